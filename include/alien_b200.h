/*
 * alien_b200.h - C ABI of the B200-native ALIEN physics-stage engine.
 *
 * The functions below replace, one for one, the engine surface that the
 * reference's host code drives for the per-timestep physics stage:
 *
 *   reference (chrxh/alien 4.12.2)                          this ABI
 *   -----------------------------------------------------   -------------------------------
 *   _SimulationCudaFacade(timestep, Settings)                alien_b200_create
 *     source/EngineGpuKernels/SimulationCudaFacade.cuh:37
 *   ~_SimulationCudaFacade()            (.cu:89-112)         alien_b200_destroy
 *   calcTimestep(timesteps, forceUpdateStatistics)  (:42)    alien_b200_calc_timesteps
 *   setSimulationData(DataTO const&)                (:51)    alien_b200_set_data
 *   getSimulationData(upperLeft, lowerRight, DataTO) (:46)   alien_b200_get_data
 *   setSimulationParameters(SimulationParameters)  (:74-76)  alien_b200_set_parameters
 *   getSimulationParameters()                       (:73)    alien_b200_get_parameters
 *   getArraySizes()                                 (:78)    alien_b200_get_array_sizes
 *   resizeArraysIfNecessary(ArraySizes)             (:91)    alien_b200_resize_arrays_if_necessary
 *   getCurrentTimestep / setCurrentTimestep      (:86-87)    alien_b200_get/set_current_timestep
 *   clear()                                         (:89)    alien_b200_clear
 *   getRawStatistics()                              (:80)    alien_b200_get_raw_statistics
 *
 * Data crosses the boundary in the reference's own transfer format: the
 * structs AlienCellTO / AlienParticleTO / AlienDataTO below are byte-for-byte
 * the reference's CellTO / ParticleTO / DataTO
 * (source/EngineGpuKernels/TOs.cuh:10-236); the static asserts at the end pin
 * every offset.  Parameters cross as AlienPhysicsParams, the subset of
 * SimulationParameters (source/EngineInterface/SimulationParameters.h:18-206)
 * that the physics stage reads, with the reference's field names.
 *
 * Conventions: every function returns an int status (ALIEN_B200_OK == 0);
 * no C++ exception crosses the ABI; alien_b200_last_error() returns the text
 * of the last failure on the calling thread.  A handle is not thread-safe:
 * callers serialise calls per handle (the reference does the same through
 * EngineWorkerGuard, source/EngineImpl/EngineWorker.cpp:608-632).
 */
#ifndef ALIEN_B200_H
#define ALIEN_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ALIEN_B200_MAX_CELL_BONDS 6  /* EngineInterface/EngineConstants.h:3 */
#define ALIEN_B200_MAX_CHANNELS 8    /* EngineInterface/EngineConstants.h:4 */
#define ALIEN_B200_MAX_COLORS 7      /* EngineInterface/EngineConstants.h:6 */

/* status codes */
#define ALIEN_B200_OK 0
#define ALIEN_B200_ERR_INVALID_ARGUMENT 1
#define ALIEN_B200_ERR_OUT_OF_MEMORY 2
#define ALIEN_B200_ERR_CUDA 3
#define ALIEN_B200_ERR_DEVICE_FLAG 4
#define ALIEN_B200_ERR_UNSUPPORTED 5
#define ALIEN_B200_ERR_CAPACITY 6
#define ALIEN_B200_ERR_NO_DEVICE 7

/* motion types, EngineInterface/Motion.h:38-43 */
#define ALIEN_B200_MOTION_FLUID 0
#define ALIEN_B200_MOTION_COLLISION 1

/* living states, EngineInterface/CellFunctionConstants.h:25-35 */
#define ALIEN_B200_LIVING_READY 0
#define ALIEN_B200_LIVING_UNDER_CONSTRUCTION 1
#define ALIEN_B200_LIVING_ACTIVATING 2
#define ALIEN_B200_LIVING_DETACHING 3
#define ALIEN_B200_LIVING_REVIVING 4
#define ALIEN_B200_LIVING_DYING 5

/* cell death consequences, EngineInterface/SimulationParametersTypes.h */
#define ALIEN_B200_DEATH_NONE 0
#define ALIEN_B200_DEATH_CREATURE_DIES 1
#define ALIEN_B200_DEATH_DETACHED_PARTS_DIE 2

#define ALIEN_B200_CELL_FUNCTION_CONSTRUCTOR 2
#define ALIEN_B200_CELL_FUNCTION_NONE 11

#if defined(__cplusplus)
#define ALIEN_B200_ALIGN8 alignas(8)
#else
#define ALIEN_B200_ALIGN8 _Alignas(8)
#endif

/* float2 / int2 with CUDA's alignment (float2 is 8-byte aligned) */
typedef struct AlienFloat2 {
    ALIEN_B200_ALIGN8 float x;
    float y;
} AlienFloat2;

typedef struct AlienInt2 {
    int32_t x;
    int32_t y;
} AlienInt2;

/* ConnectionTO, TOs.cuh:30-35 */
typedef struct AlienConnectionTO {
    int32_t cellIndex; /* index into the same cell array */
    float distance;
    float angleFromPrevious;
} AlienConnectionTO;

/* SignalTO, TOs.cuh:37-43 */
typedef struct AlienSignalTO {
    float channels[ALIEN_B200_MAX_CHANNELS];
    uint8_t origin;
    float targetX;
    float targetY;
} AlienSignalTO;

/* CellMetadataTO, TOs.cuh:21-28 */
typedef struct AlienCellMetadataTO {
    uint16_t nameSize;
    uint64_t nameDataIndex;
    uint16_t descriptionSize;
    uint64_t descriptionDataIndex;
} AlienCellMetadataTO;

/* CellTO, TOs.cuh:158-193 (304 bytes).  The cell-function union
 * (CellFunctionTO, TOs.cuh:143-156, 64 bytes) is carried opaquely: the
 * physics stage never reads it, and egress returns it unchanged. */
typedef struct AlienCellTO {
    uint64_t id;
    AlienConnectionTO connections[ALIEN_B200_MAX_CELL_BONDS];
    AlienFloat2 pos;
    AlienFloat2 vel;
    float energy;
    float stiffness;
    uint8_t color;
    uint8_t maxConnections;
    uint8_t numConnections;
    uint8_t barrier;
    uint32_t age;
    int32_t livingState;
    uint32_t creatureId;
    uint32_t mutationId;
    uint8_t ancestorMutationId;
    float genomeComplexity;
    uint8_t executionOrderNumber;
    int8_t inputExecutionOrderNumber;
    uint8_t outputBlocked;
    int32_t cellFunction;
    uint64_t cellFunctionData[8];
    AlienSignalTO signal;
    uint32_t activationTime;
    uint16_t detectedByCreatureId;
    uint8_t cellFunctionUsed;
    AlienCellMetadataTO metadata;
    uint8_t selected;
} AlienCellTO;

/* ParticleTO, TOs.cuh:10-19 (40 bytes) */
typedef struct AlienParticleTO {
    uint64_t id;
    float energy;
    AlienFloat2 pos;
    AlienFloat2 vel;
    uint8_t color;
    uint8_t selected;
} AlienParticleTO;

/* DataTO, TOs.cuh:195-236: caller-owned host buffers */
typedef struct AlienDataTO {
    uint64_t* numCells;
    AlienCellTO* cells;
    uint64_t* numParticles;
    AlienParticleTO* particles;
    uint64_t* numAuxiliaryData;
    uint8_t* auxiliaryData;
} AlienDataTO;

/* ArraySizes, EngineInterface/ArraySizes.h:5-10 */
typedef struct AlienArraySizes {
    uint64_t cellArraySize;
    uint64_t particleArraySize;
    uint64_t auxiliaryDataSize;
} AlienArraySizes;

/* GeneralSettings, EngineInterface/GeneralSettings.h:3-7 */
typedef struct AlienGeneralSettings {
    int32_t worldSizeX;
    int32_t worldSizeY;
} AlienGeneralSettings;

/* Zones (SimulationParametersZone, EngineInterface/SimulationParametersZone.h):
 * regions in which parameter values blend from the base values into the
 * zone's own (SpotCalculator.cuh:78-93, 183-232) and which may carry a flow
 * field (FlowFieldKernels.cu:48-89).  Only the physics-stage values are
 * carried; each has an `activated` flag as in
 * SimulationParametersZoneActivatedValues.h.  Zones and radiation sources
 * move by their velocity after every timestep
 * (SimulationParametersUpdateService.cu:52-78). */
#define ALIEN_B200_MAX_ZONES 20              /* EngineConstants.h:8 */
#define ALIEN_B200_MAX_RADIATION_SOURCES 40  /* EngineConstants.h:7 */
enum {
    ALIEN_B200_SHAPE_CIRCULAR = 0,
    ALIEN_B200_SHAPE_RECTANGULAR = 1,
};
enum {
    ALIEN_B200_FLOW_NONE = 0,
    ALIEN_B200_FLOW_RADIAL = 1,
    ALIEN_B200_FLOW_CENTRAL = 2,
    ALIEN_B200_FLOW_LINEAR = 3,
};
typedef struct AlienZone {
    float posX, posY, velX, velY;
    float fadeoutRadius;
    int32_t shapeType;          /* ALIEN_B200_SHAPE_*: circular uses coreRadius, rectangular width x height */
    float coreRadius, width, height;
    int32_t flowType;           /* ALIEN_B200_FLOW_* */
    int32_t flowOrientation;    /* radial: 0 clockwise, 1 counter-clockwise */
    float flowStrength;         /* radial / central / linear */
    float flowDriftAngle;       /* radial, degrees */
    float flowAngle;            /* linear, degrees */
    /* values (SimulationParametersZoneValues.h) */
    float friction;
    float rigidity;
    float radiationAbsorption[ALIEN_B200_MAX_COLORS];
    float radiationCellAgeStrength[ALIEN_B200_MAX_COLORS];
    float cellMaxForce[ALIEN_B200_MAX_COLORS];
    float cellMinEnergy[ALIEN_B200_MAX_COLORS];
    float cellDeathProbability[ALIEN_B200_MAX_COLORS];
    float cellFusionVelocity;
    float cellMaxBindingEnergy;
    uint8_t radiationDisableSources;
    /* activated flags of the values above, in their order */
    uint8_t frictionActivated, rigidityActivated, radiationAbsorptionActivated, radiationCellAgeStrengthActivated;
    uint8_t cellMaxForceActivated, cellMinEnergyActivated, cellDeathProbabilityActivated, cellFusionVelocityActivated;
    uint8_t cellMaxBindingEnergyActivated, radiationDisableSourcesActivated;
    uint8_t reserved[1];
} AlienZone;

/* RadiationSource (EngineInterface/RadiationSource.h): new energy particles
 * (radiation, deleted cells) appear at an active source, chosen in
 * proportion to the strengths (RadiationProcessor.cuh:248-364). */
typedef struct AlienRadiationSource {
    float strength;
    float posX, posY, velX, velY;
    int32_t useAngle;
    float angle;                /* degrees */
    int32_t shapeType;          /* ALIEN_B200_SHAPE_*: circular uses radius, rectangular width x height */
    float radius, width, height;
} AlienRadiationSource;

/* The physics-stage subset of SimulationParameters
 * (EngineInterface/SimulationParameters.h:18-206, base values from
 * SimulationParametersZoneValues.h:10-30, motion from Motion.h:7-36).
 * alien_b200_default_parameters() fills the reference defaults. */
typedef struct AlienPhysicsParams {
    float timestepSize;                       /* SimulationParameters.h:61 */
    int32_t motionType;                       /* :62 */
    float smoothingLength;                    /* Motion.h:9 */
    float viscosityStrength;                  /* Motion.h:10 */
    float pressureStrength;                   /* Motion.h:11 */
    float cellMaxCollisionDistance;           /* Motion.h:22 */
    float cellRepulsionStrength;              /* Motion.h:23 */
    float innerFriction;                      /* :65 */
    float cellMaxVelocity;                    /* :66 */
    float cellMaxBindingDistance[ALIEN_B200_MAX_COLORS]; /* :67 */
    float cellMinDistance;                    /* :70 */
    float cellMaxForceDecayProb;              /* :71 */
    float radiationProb;                      /* :79 */
    float radiationVelocityMultiplier;        /* :80 */
    float radiationVelocityPerturbation;      /* :81 */
    int32_t radiationMinCellAge[ALIEN_B200_MAX_COLORS];  /* :82 */
    float highRadiationFactor[ALIEN_B200_MAX_COLORS];    /* :85 */
    float highRadiationMinCellEnergy[ALIEN_B200_MAX_COLORS]; /* :86 */
    int32_t cellDeathConsequences;            /* :87 */
    int32_t cellMaxAge[ALIEN_B200_MAX_COLORS];           /* :88 */
    float particleSplitEnergy[ALIEN_B200_MAX_COLORS];    /* :114 */
    /* baseValues (SimulationParametersZoneValues.h) */
    float friction;                           /* :12 */
    float rigidity;                           /* :13 */
    float radiationAbsorption[ALIEN_B200_MAX_COLORS];    /* :14 */
    float radiationCellAgeStrength[ALIEN_B200_MAX_COLORS]; /* :17 */
    float cellMaxForce[ALIEN_B200_MAX_COLORS];           /* :19 */
    float cellMinEnergy[ALIEN_B200_MAX_COLORS];          /* :20 */
    float cellDeathProbability[ALIEN_B200_MAX_COLORS];   /* :21 */
    float cellFusionVelocity;                 /* :23 */
    float cellMaxBindingEnergy;               /* :24 */
    int32_t numZones;                         /* :39, zones[0, numZones) */
    int32_t numRadiationSources;              /* :27, radiationSources[0, numRadiationSources) */
    /* features outside the physics stage: must be zero (checked; a nonzero
     * value returns ALIEN_B200_ERR_UNSUPPORTED) */
    uint8_t particleTransformationAllowed;    /* :111 */
    uint8_t cellAgeLimiter;                   /* Features.h */
    uint8_t cellColorTransitionRules;         /* Features.h */
    uint8_t advancedAbsorptionControl;        /* Features.h */
    /* external energy (Features.h, SimulationParameters.h:31-36): with it on,
     * a new energy particle of color c sends externalEnergyBackflowFactor[c]
     * of its energy to the external energy pool (RadiationProcessor.cuh:
     * 345-354) */
    uint8_t externalEnergyControl;
    uint8_t radiationDisableSources;          /* ZoneValues.h:18, base value */
    uint8_t reserved[2];
    /* cell functions: a cell with a function runs it in the steps where
     * timestep % cellNumExecutionOrderNumbers equals its execution order
     * number (CellFunctionProcessor.cuh:241-244); only the neuron function is
     * part of this engine */
    int32_t cellNumExecutionOrderNumbers;     /* :72 */
    float externalEnergy;                     /* :31, the pool (updated by the steps) */
    float externalEnergyBackflowFactor[ALIEN_B200_MAX_COLORS]; /* :34 */
    float externalEnergyBackflowLimit;        /* :36 */
    AlienZone zones[ALIEN_B200_MAX_ZONES];    /* :40 */
    AlienRadiationSource radiationSources[ALIEN_B200_MAX_RADIATION_SOURCES]; /* :28 */
} AlienPhysicsParams;

/* Subset of RawStatisticsData (EngineGpuKernels/SimulationStatistics.cuh)
 * that the physics stage maintains. */
typedef struct AlienRawStatistics {
    uint64_t timestep;
    uint64_t numCells;
    uint64_t numParticles;
    uint64_t numConnections;          /* directed bonds: sum of numConnections */
    uint64_t numCellsByColor[ALIEN_B200_MAX_COLORS];
    double totalCellEnergy;
    double totalParticleEnergy;
} AlienRawStatistics;

/* RawStatisticsData (EngineInterface/RawStatisticsData.h:5-56), byte for
 * byte: the timeline of the current timestep, the statistics accumulated
 * since the last alien_b200_reset_time_interval_statistics, and the age
 * histogram.  Fields that count cell functions outside the physics stage
 * (self-replicators, colonies, viruses, genome sizes and complexity,
 * constructor, attacker, muscle, ... activities) are 0: the engine accepts
 * no cell carrying those functions. */
#define ALIEN_B200_MAX_HISTOGRAM_SLOTS 20    /* EngineConstants.h:9 */
typedef struct AlienTimestepStatistics {
    int32_t numCells[ALIEN_B200_MAX_COLORS];
    int32_t numSelfReplicators[ALIEN_B200_MAX_COLORS];
    int32_t numColonies[ALIEN_B200_MAX_COLORS];
    int32_t numViruses[ALIEN_B200_MAX_COLORS];
    int32_t numFreeCells[ALIEN_B200_MAX_COLORS];     /* cells with mutationId 1 (Const::MutationIdForFreeCell) */
    int32_t numParticles[ALIEN_B200_MAX_COLORS];
    uint64_t numGenomeCells[ALIEN_B200_MAX_COLORS];
    float genomeComplexity[ALIEN_B200_MAX_COLORS];
    float maxGenomeComplexityOfColonies[ALIEN_B200_MAX_COLORS];
    double genomeComplexityVariance[ALIEN_B200_MAX_COLORS];
    float totalEnergy[ALIEN_B200_MAX_COLORS];        /* cells and energy particles of the color */
} AlienTimestepStatistics;
typedef struct AlienAccumulatedStatistics {
    uint64_t numCreatedCells[ALIEN_B200_MAX_COLORS];
    uint64_t numCreatedReplicators[ALIEN_B200_MAX_COLORS];
    uint64_t numAttacks[ALIEN_B200_MAX_COLORS];
    uint64_t numMuscleActivities[ALIEN_B200_MAX_COLORS];
    uint64_t numDefenderActivities[ALIEN_B200_MAX_COLORS];
    uint64_t numTransmitterActivities[ALIEN_B200_MAX_COLORS];
    uint64_t numInjectionActivities[ALIEN_B200_MAX_COLORS];
    uint64_t numCompletedInjections[ALIEN_B200_MAX_COLORS];
    uint64_t numNervePulses[ALIEN_B200_MAX_COLORS];
    uint64_t numNeuronActivities[ALIEN_B200_MAX_COLORS]; /* neuron cells that ran (NeuronProcessor.cuh:70) */
    uint64_t numSensorActivities[ALIEN_B200_MAX_COLORS];
    uint64_t numSensorMatches[ALIEN_B200_MAX_COLORS];
    uint64_t numReconnectorCreated[ALIEN_B200_MAX_COLORS];
    uint64_t numReconnectorRemoved[ALIEN_B200_MAX_COLORS];
    uint64_t numDetonations[ALIEN_B200_MAX_COLORS];
} AlienAccumulatedStatistics;
typedef struct AlienTimelineStatistics {
    AlienTimestepStatistics timestep;
    AlienAccumulatedStatistics accumulated;
} AlienTimelineStatistics;
/* ages of the cells that are not barriers: maxValue = the largest age,
 * slot = age * 20 / (maxValue + 1) (StatisticsKernels.cu:85-105) */
typedef struct AlienHistogramData {
    int32_t maxValue;
    int32_t numCellsByColorBySlot[ALIEN_B200_MAX_COLORS][ALIEN_B200_MAX_HISTOGRAM_SLOTS];
} AlienHistogramData;
typedef struct AlienRawStatisticsData {
    AlienTimelineStatistics timeline;
    AlienHistogramData histogram;
} AlienRawStatisticsData;

typedef struct alien_b200_simulation alien_b200_simulation;

/* library / defaults */
int alien_b200_version(void);
/* Makes `device` the CUDA device of the calling thread for handles created
 * afterwards (the reference picks the device with the highest compute
 * capability itself, SimulationCudaFacade.cu:517-576). */
int alien_b200_select_device(int device);
void alien_b200_default_parameters(AlienPhysicsParams* params);
int alien_b200_last_error(char* buffer, size_t size);

/* facade.  alien_b200_create replaces the _SimulationCudaFacade constructor
 * (SimulationCudaFacade.cu:51-87): it selects the device (the current CUDA
 * device of the calling thread), and allocates the world-sized structures. */
int alien_b200_create(const AlienGeneralSettings* general, const AlienPhysicsParams* params,
                      uint64_t timestep, alien_b200_simulation** out);
int alien_b200_destroy(alien_b200_simulation* sim);
/* Particle storage grows as the steps need it: every 64 steps when half of
 * it is used, and inside a step whose new particles would not fit (the
 * world halts before writing them; the call grows the storage on the
 * device, completes the step and the remaining steps).  Results equal a run
 * whose storage was large enough from the start; nothing is dropped. */
int alien_b200_calc_timesteps(alien_b200_simulation* sim, uint64_t timesteps);
int alien_b200_set_data(alien_b200_simulation* sim, const AlienDataTO* data);
int alien_b200_get_data(alien_b200_simulation* sim, AlienInt2 upperLeft, AlienInt2 lowerRight,
                        const AlienDataTO* data);
int alien_b200_set_parameters(alien_b200_simulation* sim, const AlienPhysicsParams* params);
int alien_b200_get_parameters(alien_b200_simulation* sim, AlienPhysicsParams* params);
int alien_b200_get_array_sizes(alien_b200_simulation* sim, AlienArraySizes* sizes);
int alien_b200_resize_arrays_if_necessary(alien_b200_simulation* sim, const AlienArraySizes* additionals);
int alien_b200_get_current_timestep(alien_b200_simulation* sim, uint64_t* timestep);
int alien_b200_set_current_timestep(alien_b200_simulation* sim, uint64_t timestep);
int alien_b200_clear(alien_b200_simulation* sim);
int alien_b200_get_raw_statistics(alien_b200_simulation* sim, AlienRawStatistics* statistics);
/* _SimulationCudaFacade::getRawStatistics (SimulationCudaFacade.cu:420-440)
 * with the reference's RawStatisticsData layout, computed at the call (the
 * reference refreshes it at most every 30 ms of stepping and at the end of
 * calcTimestep); energies are 2^-16 fixed-point sums, independent of order. */
int alien_b200_get_raw_statistics_data(alien_b200_simulation* sim, AlienRawStatisticsData* statistics);
/* resetTimeIntervalStatistics (SimulationCudaFacade.cu:452-455): clears the
 * accumulated statistics. */
int alien_b200_reset_time_interval_statistics(alien_b200_simulation* sim);

/* The density map (DensityMap, source/EngineGpuKernels/DensityMap.cuh:8-230)
 * that the reference fills in every step (cleared at SimulationKernels.cu:33,
 * DensityMap::addCell for every cell in the pair-force kernels at :39 and
 * :47) and that only its sensor cells read.  Built on request here, with the
 * reference's layout: slots of 8 x 8 (PreprocessedSimulationData.cuh:13),
 * sizeX = worldSizeX / 8, sizeY = worldSizeY / 8, entry x + y * sizeX, and
 * the packed byte counters of addCell (per color and a total byte; mutant
 * buckets; genome-complexity buckets; carries between byte lanes as in the
 * reference's 64-bit adds).  The map is the one the last step filled: every
 * live cell at its position after that step's overlap correction, the
 * other-mutant buckets at that step's timestep (the current one minus 1).
 * Without a step since the world was set, the cells at their set positions
 * and the current timestep.  Cells the last step removed are not in it.
 * sizeX and sizeY are always written; each array that is not null receives
 * sizeX * sizeY entries (call once with null arrays for the size). */
typedef struct AlienDensityMap {
    int32_t sizeX, sizeY;
    uint64_t* color;            /* byte c: cells of color c; byte 7: all cells */
    uint64_t* otherMutant;      /* mutationId >= 2: all bytes but bucket (id + timestep / 23) % 8 */
    uint64_t* sameMutant1;      /* mutationId >= 2: byte id % 3 and byte 3 + id % 5 */
    uint64_t* sameMutant2;      /* mutationId >= 2: byte id % 7 */
    uint32_t* specificMutant;   /* byte 0: mutationId 0, byte 1: mutationId 1 */
    uint64_t* lessComplexity1;  /* genome-complexity buckets (bit length of complexity * 10) */
    uint64_t* lessComplexity2;
    uint64_t* moreComplexity1;
    uint64_t* moreComplexity2;
} AlienDensityMap;
int alien_b200_get_density_map(alien_b200_simulation* sim, AlienDensityMap* map);

/* Device-resident timing hook: steps `timesteps` times on the handle's
 * stream without the end-of-call synchronisation and error read-back that
 * alien_b200_calc_timesteps performs.  For benchmarks that bracket the
 * steps with their own events; errors surface at the next synchronising
 * call.  No counterpart in the reference (its calcTimestep synchronises
 * after every step, SimulationCudaFacade.cu:578-582). */
int alien_b200_enqueue_timesteps(alien_b200_simulation* sim, uint64_t timesteps);
/* Steps `timesteps` times on the handle's stream between two CUDA events
 * (the stream is synchronised first) and returns the elapsed milliseconds. */
int alien_b200_time_timesteps(alien_b200_simulation* sim, uint64_t timesteps, double* milliseconds);
/* The CUDA stream (cudaStream_t) all of the handle's work is issued on. */
void* alien_b200_stream(alien_b200_simulation* sim);
/* Number of kernel launches issued by the handle since creation. */
uint64_t alien_b200_kernel_launch_count(alien_b200_simulation* sim);
/* Steps `timesteps` times launch by launch (no graph) with a CUDA event
 * after every kernel; kernelMs[k] receives the summed milliseconds of the
 * k-th kernel of the step, alien_b200_step_kernel_name(k) its name (valid on
 * the calling thread until the next timed call).  A profiling hook without
 * a reference counterpart. */
int alien_b200_timed_timesteps(alien_b200_simulation* sim, uint64_t timesteps, double* kernelMs, int maxKernels,
                               int* numKernels);
const char* alien_b200_step_kernel_name(int index);

/* Launch configuration of the pair-force kernel.  It processes the world in
 * regions of tiles (one CTA each, staged in shared memory); the region
 * shape is one of ALIEN_B200_REGION_CHOICES candidates per motion type (0
 * fluid, 1 collision; candidates[m][i] = tiles in x, y; the first is the
 * default).  A cell's neighbours are visited in the same order whatever the
 * shape, so the choice changes no result, only the speed.  Unless the
 * caller fixes it (regionChoiceFixed[m] = candidate index + 1), an
 * autotuner chooses it at the first step of every new layout (set_data, a
 * batch): it bins the current state, times the pair kernel with every
 * candidate (three launches each after one untimed) and keeps the fastest
 * (alien_b200_choose_region).  The state is not changed.  No counterpart in
 * the reference, whose launch shapes are fixed (KERNEL_CALL, Macros.cuh:75-83)
 * or computed by calcOptimalThreadsForFluidKernel
 * (SimulationKernelsLauncher.cu:18-22). */
#define ALIEN_B200_REGION_CHOICES 6
typedef struct AlienLaunchConfig {
    int32_t regionTiles[2][2];      /* shape in use (tiles x, y), per motion type */
    int32_t regionChoice[2];        /* its index among the candidates */
    int32_t regionChoiceFixed[2];   /* fixed by the caller: index + 1; 0 = autotune */
    int32_t tuned;                  /* 1 once the autotuner ran on this layout */
    float tunedMs[2][ALIEN_B200_REGION_CHOICES];  /* measured ms per launch (0 = not measured) */
    int32_t candidates[2][ALIEN_B200_REGION_CHOICES][2];
} AlienLaunchConfig;
/* Only regionChoiceFixed is read: 0 returns a motion type to the autotuner. */
int alien_b200_set_launch_config(alien_b200_simulation* sim, const AlienLaunchConfig* config);
int alien_b200_get_launch_config(alien_b200_simulation* sim, AlienLaunchConfig* config);
/* The autotuner's rule on n measured times (ms per launch of each candidate
 * in order; entries <= 0 are skipped): the fastest, where a later candidate
 * must beat the best earlier one by more than 2 %.  Returns the index. */
int alien_b200_choose_region(const float* milliseconds, int n);

/* The cell map of the current state as the step's own binning kernels
 * build it (tile histogram, scan, scatter, tile-ordered staging), read back
 * without stepping: for each binned cell in the map's tile order its id, its
 * slot (x + y * worldSizeX, the slot of CellMap::set_block, Map.cuh:95-130),
 * its tile (tiles of ceil(interaction radius) slots, row-major) and its map
 * flags (bit 0 barrier, bit 1 visible to scans: among the first 10 cells of
 * its slot in storage order, Map.cuh:117-125; bit 2 first cell of its slot,
 * CellMap::getFirst).  Host buffers of `capacity` entries each; *count
 * receives the number of binned cells (ALIEN_B200_ERR_CAPACITY when it
 * exceeds capacity, nothing written).  A test and debugging hook with no
 * counterpart in the reference (its map is a device-internal pointer grid);
 * the state is unchanged. */
int alien_b200_debug_cell_map(alien_b200_simulation* sim, uint64_t capacity, uint64_t* ids, uint32_t* slots, uint32_t* tiles,
                              uint8_t* flags, uint64_t* count);

/* Statistics of transfer objects that already sit in device memory,
 * computed without allocating anything on the device.  No counterpart in
 * the reference.  For callers that cannot call cudaMalloc when they need the
 * numbers: a host runtime that reserved the whole HBM budget up front and
 * lends out only its own buffers, or code running while another component
 * owns the allocator.  cells / particles / statistics are device pointers
 * owned by the caller (statistics: one AlienRawStatistics written on
 * `stream`, a cudaStream_t or NULL); the result equals
 * alien_b200_get_raw_statistics for the same objects.  The only scratch is a
 * fixed 640 KiB (655,360 B) array inside the library that every GPU loading
 * it keeps until exit, which bounds one call to 8,388,608 cells and as many
 * particles; larger inputs return ALIEN_B200_ERR_CAPACITY.  The first call
 * on a device is its set-up: it loads the entry point's code and array onto
 * that device (CUDA loads modules lazily by default, and that load may need
 * device memory) and looks up the array's device address.  So make the
 * first call on each device before reserving the remaining device memory
 * and before any stream capture; later calls need no device memory.  A
 * cudaDeviceReset invalidates the looked-up address: do not call again on a
 * device that was reset.  A CUDA error pending from earlier work is
 * returned as ALIEN_B200_ERR_CUDA without launching and is left in place.
 * Calls that overlap on the GPU share the array and race. */
int alien_b200_statistics_no_alloc(const AlienCellTO* cells, uint64_t numCells, const AlienParticleTO* particles,
                                   uint64_t numParticles, uint64_t timestep, AlienRawStatistics* statistics,
                                   void* stream);

#ifdef __cplusplus
} /* extern "C" */
#endif

/* ---- layout pins: must equal the reference's TOs.cuh layout ---- */
#ifdef __cplusplus
#define ALIEN_B200_STATIC_ASSERT(c, m) static_assert(c, m)
#else
#define ALIEN_B200_STATIC_ASSERT(c, m) _Static_assert(c, m)
#endif
ALIEN_B200_STATIC_ASSERT(sizeof(AlienCellTO) == 304, "CellTO is 304 bytes");
ALIEN_B200_STATIC_ASSERT(sizeof(AlienParticleTO) == 40, "ParticleTO is 40 bytes");
ALIEN_B200_STATIC_ASSERT(sizeof(AlienConnectionTO) == 12, "ConnectionTO is 12 bytes");
ALIEN_B200_STATIC_ASSERT(sizeof(AlienSignalTO) == 44, "SignalTO is 44 bytes");
ALIEN_B200_STATIC_ASSERT(sizeof(AlienCellMetadataTO) == 32, "CellMetadataTO is 32 bytes");
ALIEN_B200_STATIC_ASSERT(offsetof(AlienCellTO, connections) == 8, "CellTO.connections");
ALIEN_B200_STATIC_ASSERT(offsetof(AlienCellTO, pos) == 80, "CellTO.pos");
ALIEN_B200_STATIC_ASSERT(offsetof(AlienCellTO, vel) == 88, "CellTO.vel");
ALIEN_B200_STATIC_ASSERT(offsetof(AlienCellTO, energy) == 96, "CellTO.energy");
ALIEN_B200_STATIC_ASSERT(offsetof(AlienCellTO, stiffness) == 100, "CellTO.stiffness");
ALIEN_B200_STATIC_ASSERT(offsetof(AlienCellTO, color) == 104, "CellTO.color");
ALIEN_B200_STATIC_ASSERT(offsetof(AlienCellTO, barrier) == 107, "CellTO.barrier");
ALIEN_B200_STATIC_ASSERT(offsetof(AlienCellTO, age) == 108, "CellTO.age");
ALIEN_B200_STATIC_ASSERT(offsetof(AlienCellTO, livingState) == 112, "CellTO.livingState");
ALIEN_B200_STATIC_ASSERT(offsetof(AlienCellTO, creatureId) == 116, "CellTO.creatureId");
ALIEN_B200_STATIC_ASSERT(offsetof(AlienCellTO, ancestorMutationId) == 124, "CellTO.ancestorMutationId");
ALIEN_B200_STATIC_ASSERT(offsetof(AlienCellTO, genomeComplexity) == 128, "CellTO.genomeComplexity");
ALIEN_B200_STATIC_ASSERT(offsetof(AlienCellTO, executionOrderNumber) == 132, "CellTO.executionOrderNumber");
ALIEN_B200_STATIC_ASSERT(offsetof(AlienCellTO, cellFunction) == 136, "CellTO.cellFunction");
ALIEN_B200_STATIC_ASSERT(offsetof(AlienCellTO, cellFunctionData) == 144, "CellTO.cellFunctionData");
ALIEN_B200_STATIC_ASSERT(offsetof(AlienCellTO, signal) == 208, "CellTO.signal");
ALIEN_B200_STATIC_ASSERT(offsetof(AlienCellTO, activationTime) == 252, "CellTO.activationTime");
ALIEN_B200_STATIC_ASSERT(offsetof(AlienCellTO, detectedByCreatureId) == 256, "CellTO.detectedByCreatureId");
ALIEN_B200_STATIC_ASSERT(offsetof(AlienCellTO, cellFunctionUsed) == 258, "CellTO.cellFunctionUsed");
ALIEN_B200_STATIC_ASSERT(offsetof(AlienCellTO, metadata) == 264, "CellTO.metadata");
ALIEN_B200_STATIC_ASSERT(offsetof(AlienCellTO, selected) == 296, "CellTO.selected");
ALIEN_B200_STATIC_ASSERT(offsetof(AlienParticleTO, energy) == 8, "ParticleTO.energy");
ALIEN_B200_STATIC_ASSERT(offsetof(AlienParticleTO, pos) == 16, "ParticleTO.pos");
ALIEN_B200_STATIC_ASSERT(offsetof(AlienParticleTO, vel) == 24, "ParticleTO.vel");
ALIEN_B200_STATIC_ASSERT(offsetof(AlienParticleTO, color) == 32, "ParticleTO.color");
ALIEN_B200_STATIC_ASSERT(offsetof(AlienSignalTO, targetX) == 36, "SignalTO.targetX");
ALIEN_B200_STATIC_ASSERT(offsetof(AlienCellMetadataTO, nameDataIndex) == 8, "CellMetadataTO.nameDataIndex");
ALIEN_B200_STATIC_ASSERT(offsetof(AlienCellMetadataTO, descriptionDataIndex) == 24, "CellMetadataTO.descriptionDataIndex");
ALIEN_B200_STATIC_ASSERT(sizeof(AlienZone) == 224, "AlienZone is 224 bytes");
ALIEN_B200_STATIC_ASSERT(sizeof(AlienRadiationSource) == 44, "AlienRadiationSource is 44 bytes");
ALIEN_B200_STATIC_ASSERT(sizeof(AlienTimestepStatistics) == 368, "TimestepStatistics is 368 bytes");
ALIEN_B200_STATIC_ASSERT(offsetof(AlienTimestepStatistics, numGenomeCells) == 168, "TimestepStatistics.numGenomeCells");
ALIEN_B200_STATIC_ASSERT(offsetof(AlienTimestepStatistics, genomeComplexityVariance) == 280, "TimestepStatistics.genomeComplexityVariance");
ALIEN_B200_STATIC_ASSERT(offsetof(AlienTimestepStatistics, totalEnergy) == 336, "TimestepStatistics.totalEnergy");
ALIEN_B200_STATIC_ASSERT(sizeof(AlienAccumulatedStatistics) == 840, "AccumulatedStatistics is 840 bytes");
ALIEN_B200_STATIC_ASSERT(sizeof(AlienHistogramData) == 564, "HistogramData is 564 bytes");
ALIEN_B200_STATIC_ASSERT(offsetof(AlienRawStatisticsData, histogram) == 1208, "RawStatisticsData.histogram");
ALIEN_B200_STATIC_ASSERT(sizeof(AlienRawStatisticsData) == 1776, "RawStatisticsData is 1776 bytes");

#endif /* ALIEN_B200_H */
