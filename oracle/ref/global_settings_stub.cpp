// Minimal GlobalSettings for the reference-engine harness (test
// infrastructure).  The reference's own implementation
// (source/Base/GlobalSettings.cpp) needs Boost property trees; the engine
// only asks isDebugMode(), and the harness answers false so that kernels are
// not synchronised one by one (Macros.cuh:75-101).
#include "Base/GlobalSettings.h"

struct GlobalSettingsImpl {};

GlobalSettings& GlobalSettings::get()
{
    static GlobalSettings instance;
    return instance;
}
GlobalSettings::GlobalSettings() {}
GlobalSettings::~GlobalSettings() {}
bool GlobalSettings::isDebugMode() const { return false; }
void GlobalSettings::setDebugMode(bool) const {}
