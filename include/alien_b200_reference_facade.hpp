/* alien_b200_reference_facade.hpp - the drop-in adapter for the reference's
 * host code: a class with the physics-stage interface of _SimulationCudaFacade
 * (source/EngineGpuKernels/SimulationCudaFacade.cuh:27-139) that forwards to
 * the C ABI of libalien_b200.so.  It is compiled inside the reference tree
 * (it includes the reference's own headers: TOs.cuh, Settings.h,
 * ArraySizes.h, RawStatisticsData.h); the layout checks below make the
 * transfer objects and the statistics byte-identical to this library's. */
#pragma once

#include <cstring>
#include <stdexcept>

#include "alien_b200.h"
#include "EngineGpuKernels/TOs.cuh"
#include "EngineInterface/ArraySizes.h"
#include "EngineInterface/RawStatisticsData.h"
#include "EngineInterface/Settings.h"

static_assert(sizeof(CellTO) == sizeof(AlienCellTO) && sizeof(ParticleTO) == sizeof(AlienParticleTO), "transfer objects");
static_assert(sizeof(ConnectionTO) == sizeof(AlienConnectionTO) && sizeof(DataTO) == sizeof(AlienDataTO), "transfer objects");
static_assert(offsetof(CellTO, pos) == offsetof(AlienCellTO, pos) && offsetof(CellTO, signal) == offsetof(AlienCellTO, signal)
                  && offsetof(CellTO, metadata) == offsetof(AlienCellTO, metadata),
              "CellTO layout");
static_assert(sizeof(RawStatisticsData) == sizeof(AlienRawStatisticsData), "RawStatisticsData");
static_assert(offsetof(RawStatisticsData, histogram) == offsetof(AlienRawStatisticsData, histogram), "RawStatisticsData.histogram");
static_assert(offsetof(TimestepStatistics, totalEnergy) == offsetof(AlienTimestepStatistics, totalEnergy), "TimestepStatistics");
static_assert(offsetof(AccumulatedStatistics, numNeuronActivities) == offsetof(AlienAccumulatedStatistics, numNeuronActivities),
              "AccumulatedStatistics");
static_assert(sizeof(ArraySizes) == sizeof(AlienArraySizes), "ArraySizes");

namespace alien_b200
{

inline void check(int status)
{
    if (status != ALIEN_B200_OK) {
        char text[512];
        alien_b200_last_error(text, sizeof(text));
        throw std::runtime_error(text);   // the reference's error convention (Macros.cuh:14-59)
    }
}

inline AlienPhysicsParams toB200(SimulationParameters const& p)
{
    AlienPhysicsParams a;
    alien_b200_default_parameters(&a);
    a.timestepSize = p.timestepSize;
    a.motionType = p.motionType;
    if (p.motionType == MotionType_Fluid) {
        a.smoothingLength = p.motionData.fluidMotion.smoothingLength;
        a.viscosityStrength = p.motionData.fluidMotion.viscosityStrength;
        a.pressureStrength = p.motionData.fluidMotion.pressureStrength;
    } else {
        a.cellMaxCollisionDistance = p.motionData.collisionMotion.cellMaxCollisionDistance;
        a.cellRepulsionStrength = p.motionData.collisionMotion.cellRepulsionStrength;
    }
    a.innerFriction = p.innerFriction;
    a.cellMaxVelocity = p.cellMaxVelocity;
    a.cellMinDistance = p.cellMinDistance;
    a.cellMaxForceDecayProb = p.cellMaxForceDecayProb;
    a.radiationProb = p.radiationProb;
    a.radiationVelocityMultiplier = p.radiationVelocityMultiplier;
    a.radiationVelocityPerturbation = p.radiationVelocityPerturbation;
    a.cellDeathConsequences = p.cellDeathConsequences;
    a.friction = p.baseValues.friction;
    a.rigidity = p.baseValues.rigidity;
    a.cellFusionVelocity = p.baseValues.cellFusionVelocity;
    a.cellMaxBindingEnergy = p.baseValues.cellMaxBindingEnergy;
    for (int c = 0; c < MAX_COLORS; ++c) {
        a.cellMaxBindingDistance[c] = p.cellMaxBindingDistance[c];
        a.radiationMinCellAge[c] = p.radiationMinCellAge[c];
        a.highRadiationFactor[c] = p.highRadiationFactor[c];
        a.highRadiationMinCellEnergy[c] = p.highRadiationMinCellEnergy[c];
        a.cellMaxAge[c] = p.cellMaxAge[c];
        a.particleSplitEnergy[c] = p.particleSplitEnergy[c];
        a.radiationAbsorption[c] = p.baseValues.radiationAbsorption[c];
        a.radiationCellAgeStrength[c] = p.baseValues.radiationCellAgeStrength[c];
        a.cellMaxForce[c] = p.baseValues.cellMaxForce[c];
        a.cellMinEnergy[c] = p.baseValues.cellMinEnergy[c];
        a.cellDeathProbability[c] = p.baseValues.cellDeathProbability[c];
    }
    a.radiationDisableSources = p.baseValues.radiationDisableSources;
    a.externalEnergy = p.externalEnergy;
    a.externalEnergyBackflowLimit = p.externalEnergyBackflowLimit;
    for (int c = 0; c < MAX_COLORS; ++c) a.externalEnergyBackflowFactor[c] = p.externalEnergyBackflowFactor[c];
    // zones (SimulationParametersZone.h): position, velocity, shape, flow
    // field and the physics-stage values with their activation flags
    a.numZones = p.numZones;
    for (int i = 0; i < p.numZones && i < ALIEN_B200_MAX_ZONES; ++i) {
        SimulationParametersZone const& r = p.zone[i];
        AlienZone& z = a.zones[i];
        z.posX = r.posX;
        z.posY = r.posY;
        z.velX = r.velX;
        z.velY = r.velY;
        z.fadeoutRadius = r.fadeoutRadius;
        z.shapeType = r.shapeType;
        if (r.shapeType == SpotShapeType_Circular) {
            z.coreRadius = r.shapeData.circularSpot.coreRadius;
        } else {
            z.width = r.shapeData.rectangularSpot.width;
            z.height = r.shapeData.rectangularSpot.height;
        }
        z.flowType = r.flowType;
        if (r.flowType == FlowType_Radial) {
            z.flowOrientation = r.flowData.radialFlow.orientation;
            z.flowStrength = r.flowData.radialFlow.strength;
            z.flowDriftAngle = r.flowData.radialFlow.driftAngle;
        } else if (r.flowType == FlowType_Central) {
            z.flowStrength = r.flowData.centralFlow.strength;
        } else if (r.flowType == FlowType_Linear) {
            z.flowAngle = r.flowData.linearFlow.angle;
            z.flowStrength = r.flowData.linearFlow.strength;
        }
        z.friction = r.values.friction;
        z.rigidity = r.values.rigidity;
        z.radiationDisableSources = r.values.radiationDisableSources;
        z.cellFusionVelocity = r.values.cellFusionVelocity;
        z.cellMaxBindingEnergy = r.values.cellMaxBindingEnergy;
        for (int c = 0; c < MAX_COLORS; ++c) {
            z.radiationAbsorption[c] = r.values.radiationAbsorption[c];
            z.radiationCellAgeStrength[c] = r.values.radiationCellAgeStrength[c];
            z.cellMaxForce[c] = r.values.cellMaxForce[c];
            z.cellMinEnergy[c] = r.values.cellMinEnergy[c];
            z.cellDeathProbability[c] = r.values.cellDeathProbability[c];
        }
        z.frictionActivated = r.activatedValues.friction;
        z.rigidityActivated = r.activatedValues.rigidity;
        z.radiationAbsorptionActivated = r.activatedValues.radiationAbsorption;
        z.radiationCellAgeStrengthActivated = r.activatedValues.radiationCellAgeStrength;
        z.radiationDisableSourcesActivated = r.activatedValues.radiationDisableSources;
        z.cellMaxForceActivated = r.activatedValues.cellMaxForce;
        z.cellMinEnergyActivated = r.activatedValues.cellMinEnergy;
        z.cellDeathProbabilityActivated = r.activatedValues.cellDeathProbability;
        z.cellFusionVelocityActivated = r.activatedValues.cellFusionVelocity;
        z.cellMaxBindingEnergyActivated = r.activatedValues.cellMaxBindingEnergy;
    }
    // radiation sources (RadiationSource.h)
    a.numRadiationSources = p.numRadiationSources;
    for (int i = 0; i < p.numRadiationSources && i < ALIEN_B200_MAX_RADIATION_SOURCES; ++i) {
        RadiationSource const& r = p.radiationSource[i];
        AlienRadiationSource& s = a.radiationSources[i];
        s.strength = r.strength;
        s.posX = r.posX;
        s.posY = r.posY;
        s.velX = r.velX;
        s.velY = r.velY;
        s.useAngle = r.useAngle;
        s.angle = r.angle;
        s.shapeType = r.shapeType;
        if (r.shapeType == RadiationSourceShapeType_Circular) {
            s.radius = r.shapeData.circularRadiationSource.radius;
        } else {
            s.width = r.shapeData.rectangularRadiationSource.width;
            s.height = r.shapeData.rectangularRadiationSource.height;
        }
    }
    a.particleTransformationAllowed = p.particleTransformationAllowed;
    a.cellAgeLimiter = p.features.cellAgeLimiter;
    a.cellColorTransitionRules = p.features.cellColorTransitionRules;
    a.advancedAbsorptionControl = p.features.advancedAbsorptionControl;
    a.externalEnergyControl = p.features.externalEnergyControl;
    a.cellNumExecutionOrderNumbers = p.cellNumExecutionOrderNumbers;
    return a;
}

class B200SimulationFacade
{
public:
    B200SimulationFacade(uint64_t timestep, Settings const& settings)
        : _world{settings.generalSettings.worldSizeX, settings.generalSettings.worldSizeY}
    {
        auto params = toB200(settings.simulationParameters);
        check(alien_b200_create(&_world, &params, timestep, &_sim));
    }
    ~B200SimulationFacade() { alien_b200_destroy(_sim); }

    void calcTimestep(uint64_t timesteps, bool /*forceUpdateStatistics*/) { check(alien_b200_calc_timesteps(_sim, timesteps)); }
    void setSimulationData(DataTO const& to) { check(alien_b200_set_data(_sim, reinterpret_cast<AlienDataTO const*>(&to))); }
    void getSimulationData(int2 const& ul, int2 const& lr, DataTO const& to)
    {
        check(alien_b200_get_data(_sim, {ul.x, ul.y}, {lr.x, lr.y}, reinterpret_cast<AlienDataTO const*>(&to)));
    }
    void setSimulationParameters(SimulationParameters const& p)
    {
        auto a = toB200(p);
        check(alien_b200_set_parameters(_sim, &a));
    }
    ArraySizes getArraySizes() const
    {
        AlienArraySizes s;
        check(alien_b200_get_array_sizes(_sim, &s));
        return {s.cellArraySize, s.particleArraySize, s.auxiliaryDataSize};
    }
    void resizeArraysIfNecessary(ArraySizes const& add)
    {
        AlienArraySizes s{add.cellArraySize, add.particleArraySize, add.auxiliaryDataSize};
        check(alien_b200_resize_arrays_if_necessary(_sim, &s));
    }
    uint64_t getCurrentTimestep() const
    {
        uint64_t t;
        check(alien_b200_get_current_timestep(_sim, &t));
        return t;
    }
    void setCurrentTimestep(uint64_t t) { check(alien_b200_set_current_timestep(_sim, t)); }
    void clear() { check(alien_b200_clear(_sim)); }
    RawStatisticsData getRawStatistics()
    {
        AlienRawStatisticsData a;
        check(alien_b200_get_raw_statistics_data(_sim, &a));
        RawStatisticsData r;
        std::memcpy(&r, &a, sizeof(r));  // the same layout (static_asserts above)
        return r;
    }
    void resetTimeIntervalStatistics() { check(alien_b200_reset_time_interval_statistics(_sim)); }

private:
    AlienGeneralSettings _world;
    alien_b200_simulation* _sim = nullptr;
};

}  // namespace alien_b200
