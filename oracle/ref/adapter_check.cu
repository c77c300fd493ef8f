// Compile-only check of include/alien_b200_reference_facade.hpp against the
// reference's own headers (TEST INFRASTRUCTURE, built by oracle/ref/Makefile
// when the reference sources are present): the adapter's static layout
// assertions hold, and every member function compiles.
#include "alien_b200_reference_facade.hpp"

void adapterCompileCheck(Settings const& settings, DataTO const& data, SimulationParameters const& parameters)
{
    alien_b200::B200SimulationFacade facade(0, settings);
    facade.setSimulationParameters(parameters);
    facade.setSimulationData(data);
    facade.calcTimestep(1, false);
    facade.getSimulationData(int2{0, 0}, int2{10, 10}, data);
    ArraySizes sizes = facade.getArraySizes();
    facade.resizeArraysIfNecessary(sizes);
    facade.setCurrentTimestep(facade.getCurrentTimestep());
    RawStatisticsData statistics = facade.getRawStatistics();
    (void)statistics;
    facade.resetTimeIntervalStatistics();
    facade.clear();
}
