"""Writes tests/golden/ref_settings_subset.json: the general settings and the
physics-stage keys (zones and radiation sources included) of the reference's
sample settings file
(resources/autosave.settings.json of the reference repository), in the
file's own nested layout and string values, for the settings reader's test.
Run where the reference checkout is available:

    python tests/golden/make_settings_fixture.py <reference checkout>

(or with the ALIEN_REFERENCE environment variable naming the checkout)."""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", ".."))
from alien_b200 import settings  # noqa: E402

SAMPLE = os.path.join("resources", "autosave.settings.json")


def _key_names():
    """every key the reader looks up below "simulation parameters", with
    zones and radiation sources up to the reference's maxima"""
    colors = range(7)
    for _, key, _, color in settings._FIELDS:
        yield from ([f"{key}[{c}]" for c in colors] if color else [key])
    flows = [k for fields in settings._ZONE_FLOW.values() for _, k, _ in fields]
    for i in range(settings.P.MAX_ZONES):
        base = f"spots.{i}."
        for _, key, _ in settings._ZONE_PLAIN:
            yield base + key
        for key in flows:
            yield base + key
        for _, _, key, _, color in settings._ZONE_VALUES:
            yield base + key + ".activated"
            yield from ([base + f"{key}[{c}]" for c in colors] if color else [base + key + ".value"])
    for i in range(settings.P.MAX_RADIATION_SOURCES):
        for _, key, _ in settings._SOURCE_FIELDS:
            yield f"particle sources.{i}." + key


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("ALIEN_REFERENCE", "")
    if not ref:
        sys.exit("usage: make_settings_fixture.py <reference checkout>")
    with open(os.path.join(ref, SAMPLE), encoding="utf-8") as f:
        tree = json.load(f)
    out = {"general": {k: tree["general"][k] for k in ("time step", "world size")}}
    sp = tree["simulation parameters"]
    keep = {}
    for name in _key_names():
        parts = name.split(".")
        node = sp
        for p in parts[:-1]:
            node = node.get(p, {}) if isinstance(node, dict) else {}
        if isinstance(node, dict) and parts[-1] in node and not isinstance(node[parts[-1]], dict):
            dst = keep
            for p in parts[:-1]:
                dst = dst.setdefault(p, {})
            dst[parts[-1]] = node[parts[-1]]
    out["simulation parameters"] = keep
    with open(os.path.join(HERE, "ref_settings_subset.json"), "w", encoding="utf-8") as f:
        json.dump(out, f, indent=2)


if __name__ == "__main__":
    main()
