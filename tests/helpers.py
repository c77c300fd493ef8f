"""Comparison helpers shared by the parity tests.

Objects are matched by id (the reference's own tests sort by id,
EngineTests/IntegrationTestFramework.cpp:135-142).  Floating-point fields
are compared with the one-step tolerance of the engine against the FP64
oracle: |a - b| <= RTOL * max(|b|, 1) per component (bond angles in degrees
with max(|b|, 360)).  Positions are compared through the torus-wrapped
difference, scaled by max(|b|, |position before the step|, 1) when the
input state is given: a coordinate that crossed the seam (511.99 + 0.02 ->
0.01 on a 512-wide torus) was computed in FP32 at its pre-wrap magnitude,
where one unit in the last place is 6e-5, and carries that rounding after
the wrap; an object created in the steps compared has no earlier position,
and near the low seam its scale is the world's extent.  Integer and index fields (ids, bond partners, counts, living
states) must match exactly.
"""
from __future__ import annotations

import numpy as np

RTOL = 1e-5
# a new object this close to the low seam may have crossed it in its first
# steps (speeds are at most a few units per step)
SEAM_MARGIN = 4.0


def _wrapped_diff(a, b, size):
    d = a - b
    return d - np.round(d / size) * size


def index_by_id(cells):
    order = np.argsort(cells["id"], kind="stable")
    return order


def partner_ids(cells):
    """(n, 6) array of partner ids (0 = none), per cell in the given order."""
    ids = cells["id"]
    n = cells["numConnections"].astype(np.int64)
    idx = cells["connections"]["cellIndex"].astype(np.int64)
    out = np.zeros((len(cells), 6), np.uint64)
    mask = np.arange(6)[None, :] < n[:, None]
    safe = np.where(mask, idx, 0)
    out[mask] = ids[safe[mask]]
    return out


def topology(cells):
    """set of directed bonds (id, partner id)"""
    p = partner_ids(cells)
    ids = cells["id"]
    s = set()
    for i in range(len(cells)):
        for k in range(int(cells["numConnections"][i])):
            s.add((int(ids[i]), int(p[i, k])))
    return s


def rel_err(a, b, scale=1.0):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.abs(a - b) / np.maximum(np.abs(b), scale)


def position_scale(ref_sorted, before=None, world=None):
    """max(|b|, |position before the step|, 1) per component, for objects
    sorted by id.  Objects created in the step have no earlier position: one
    that lies within ``SEAM_MARGIN`` of the low seam may have been created
    just below the high seam and crossed it, so that component is scaled by
    the world's extent"""
    scale = np.maximum(np.abs(ref_sorted["pos"].astype(np.float64)), 1.0)
    known = np.zeros(len(ref_sorted), bool)
    if before is not None and len(before):
        b = before[np.argsort(before["id"], kind="stable")]
        at = np.searchsorted(b["id"], ref_sorted["id"])
        at = np.minimum(at, len(b) - 1)
        known = b["id"][at] == ref_sorted["id"]
        scale[known] = np.maximum(scale[known], np.abs(b["pos"][at[known]].astype(np.float64)))
    if before is not None and world is not None:
        near = (~known)[:, None] & (np.abs(ref_sorted["pos"].astype(np.float64)) < SEAM_MARGIN)
        scale = np.where(near, np.maximum(scale, np.asarray(world, np.float64)[None, :]), scale)
    return scale


def compare_cells(got, ref, world, rtol=RTOL, check_bonds=True, report=None, before=None):
    """Returns a dict of max errors; asserts exact integer agreement.
    ``before``: the cells of the input state (position scale)."""
    assert len(got) == len(ref), f"cell count {len(got)} != {len(ref)}"
    og, orr = index_by_id(got), index_by_id(ref)
    g = got[og]
    r = ref[orr]
    assert np.array_equal(g["id"], r["id"]), "cell id sets differ"
    errs = {}
    W, H = world
    dpos = np.stack([_wrapped_diff(g["pos"][:, 0].astype(np.float64), r["pos"][:, 0].astype(np.float64), W),
                     _wrapped_diff(g["pos"][:, 1].astype(np.float64), r["pos"][:, 1].astype(np.float64), H)], axis=1)
    errs["pos"] = float(np.max(np.abs(dpos) / position_scale(r, before, world), initial=0))
    errs["vel"] = float(np.max(rel_err(g["vel"], r["vel"]), initial=0))
    errs["energy"] = float(np.max(rel_err(g["energy"], r["energy"]), initial=0))
    assert np.array_equal(g["livingState"], r["livingState"]), "living states differ"
    assert np.array_equal(g["age"], r["age"]), "ages differ"
    assert np.array_equal(g["numConnections"], r["numConnections"]), "bond counts differ"
    if check_bonds:
        # cellIndex refers to positions in the transfer array as returned
        pg = partner_ids(got)[og]
        pr = partner_ids(ref)[orr]
        assert np.array_equal(pg, pr), "bond partners (order included) differ"
        n = r["numConnections"].astype(np.int64)
        mask = np.arange(6)[None, :] < n[:, None]
        errs["bondDist"] = float(np.max(rel_err(g["connections"]["distance"][mask], r["connections"]["distance"][mask]), initial=0))
        # angles of bonds created this step derive from FP32 positions through
        # asin: their error floor is absolute (~1e-6 rad), so they are scaled
        # by the full circle (360 degrees) instead of their own magnitude
        errs["bondAngle"] = float(np.max(rel_err(g["connections"]["angleFromPrevious"][mask],
                                                 r["connections"]["angleFromPrevious"][mask], 360.0), initial=0))
    for k, v in errs.items():
        assert v <= rtol, f"{k}: max relative error {v:.3g} > {rtol}"
    return errs


def compare_particles(got, ref, world, rtol=RTOL, before=None):
    assert len(got) == len(ref), f"particle count {len(got)} != {len(ref)}"
    g = got[np.argsort(got["id"], kind="stable")]
    r = ref[np.argsort(ref["id"], kind="stable")]
    assert np.array_equal(g["id"], r["id"]), "particle id sets differ"
    W, H = world
    dpos = np.stack([_wrapped_diff(g["pos"][:, 0].astype(np.float64), r["pos"][:, 0].astype(np.float64), W),
                     _wrapped_diff(g["pos"][:, 1].astype(np.float64), r["pos"][:, 1].astype(np.float64), H)], axis=1)
    errs = {
        "ppos": float(np.max(np.abs(dpos) / position_scale(r, before, world), initial=0)),
        "pvel": float(np.max(rel_err(g["vel"], r["vel"]), initial=0)),
        "penergy": float(np.max(rel_err(g["energy"], r["energy"]), initial=0)),
    }
    for k, v in errs.items():
        assert v <= rtol, f"{k}: max relative error {v:.3g} > {rtol}"
    return errs


def slot_sets(cells, world):
    """order-independent cell-map contents: slot -> frozenset(ids)"""
    W, H = world
    x = np.floor(cells["pos"][:, 0].astype(np.float64)).astype(np.int64) % W
    y = np.floor(cells["pos"][:, 1].astype(np.float64)).astype(np.int64) % H
    slots = x + y * W
    out = {}
    for s, i in zip(slots.tolist(), cells["id"].tolist()):
        out.setdefault(s, set()).add(i)
    return {k: frozenset(v) for k, v in out.items()}


def total_energy(data):
    return float(np.sum(data.cells["energy"], dtype=np.float64) + np.sum(data.particles["energy"], dtype=np.float64))
