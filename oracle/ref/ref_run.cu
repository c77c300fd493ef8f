// ref_run - drives the reference's own CUDA engine (_SimulationCudaFacade,
// source/EngineGpuKernels/SimulationCudaFacade.cuh:27-139) at the DataTO
// level.  TEST INFRASTRUCTURE: it is the reference arm of the benchmark and
// the pin of the CPU oracle; the B200 engine never calls it.
//
//   ref_run <input> <output> [<density map output>]
//
// input : "ALRF" u32 version, i32 W, i32 H, u64 timestep, u64 warmup,
//         u64 steps, AlienPhysicsParams, u64 numCells, u64 numParticles,
//         u64 numAux, CellTO[numCells], ParticleTO[numParticles], aux bytes
// output: "ALRO" u32 version, u64 numCells, u64 numParticles, u64 numAux,
//         double seconds (timed steps, wall clock around calcTimestep),
//         u64 timestep, CellTO[], ParticleTO[], aux bytes
// density map output (optional): "ALDM" i32 sizeX, i32 sizeY, then the
//         reference's DensityMap arrays as the last step filled them
//         (DensityMap.cuh:8-230), sizeX*sizeY entries each: color,
//         otherMutant, sameMutant1, sameMutant2 (u64), specificMutant (u32),
//         lessComplexity1, lessComplexity2, moreComplexity1,
//         moreComplexity2 (u64)
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <type_traits>
#include <vector>

#include "EngineGpuKernels/SimulationCudaFacade.cuh"
#include "EngineGpuKernels/SimulationData.cuh"
#include "EngineGpuKernels/TOs.cuh"
#include "EngineInterface/Settings.h"

#include "../../include/alien_b200.h"

// Read access to private members for the density-map output: an explicit
// instantiation may name a private member, and the friend function it
// defines hands out the member pointer (standard C++; nothing of the
// reference's classes changes).
template <class Tag, typename Tag::type Member>
struct MemberAccess {
    friend typename Tag::type memberOf(Tag) { return Member; }
};
#define AB_MEMBER(TAG, CLASS, TYPE, NAME)                              \
    struct TAG {                                                       \
        using type = TYPE CLASS::*;                                    \
        friend type memberOf(TAG);                                     \
    };                                                                 \
    template struct MemberAccess<TAG, &CLASS::NAME>;
AB_MEMBER(FacadeData, _SimulationCudaFacade, std::shared_ptr<SimulationData>, _cudaSimulationData)
AB_MEMBER(MapSize, DensityMap, int2, _densityMapSize)
AB_MEMBER(MapColor, DensityMap, uint64_t*, _colorDensityMap)
AB_MEMBER(MapOther, DensityMap, uint64_t*, _otherMutantDensityMap)
AB_MEMBER(MapSame1, DensityMap, uint64_t*, _sameMutantDensityMap1)
AB_MEMBER(MapSame2, DensityMap, uint64_t*, _sameMutantDensityMap2)
AB_MEMBER(MapSpecific, DensityMap, uint32_t*, _specificMutantDensityMap)
AB_MEMBER(MapLess1, DensityMap, uint64_t*, _lessGenomeComplexityDensityMap1)
AB_MEMBER(MapLess2, DensityMap, uint64_t*, _lessGenomeComplexityDensityMap2)
AB_MEMBER(MapMore1, DensityMap, uint64_t*, _moreGenomeComplexityDensityMap1)
AB_MEMBER(MapMore2, DensityMap, uint64_t*, _moreGenomeComplexityDensityMap2)
#undef AB_MEMBER

static_assert(sizeof(CellTO) == sizeof(AlienCellTO), "CellTO layout");
static_assert(sizeof(ParticleTO) == sizeof(AlienParticleTO), "ParticleTO layout");

namespace
{
template <class T>
void readOrThrow(FILE* f, T* p, size_t n = 1)
{
    if (n && fread(p, sizeof(T), n, f) != n) throw std::runtime_error("short read");
}
template <class T>
void writeOrThrow(FILE* f, T const* p, size_t n = 1)
{
    if (n && fwrite(p, sizeof(T), n, f) != n) throw std::runtime_error("short write");
}

// AlienPhysicsParams -> SimulationParameters (the fields the physics stage
// reads; everything else keeps the reference defaults)
SimulationParameters toReference(AlienPhysicsParams const& a)
{
    SimulationParameters p;
    p.timestepSize = a.timestepSize;
    p.motionType = a.motionType;
    p.cellNumExecutionOrderNumbers = a.cellNumExecutionOrderNumbers;
    if (a.motionType == MotionType_Fluid) {
        p.motionData.fluidMotion.smoothingLength = a.smoothingLength;
        p.motionData.fluidMotion.viscosityStrength = a.viscosityStrength;
        p.motionData.fluidMotion.pressureStrength = a.pressureStrength;
    } else {
        p.motionData.collisionMotion.cellMaxCollisionDistance = a.cellMaxCollisionDistance;
        p.motionData.collisionMotion.cellRepulsionStrength = a.cellRepulsionStrength;
    }
    p.innerFriction = a.innerFriction;
    p.cellMaxVelocity = a.cellMaxVelocity;
    p.cellMinDistance = a.cellMinDistance;
    p.cellMaxForceDecayProb = a.cellMaxForceDecayProb;
    p.radiationProb = a.radiationProb;
    p.radiationVelocityMultiplier = a.radiationVelocityMultiplier;
    p.radiationVelocityPerturbation = a.radiationVelocityPerturbation;
    p.cellDeathConsequences = a.cellDeathConsequences;
    p.baseValues.friction = a.friction;
    p.baseValues.rigidity = a.rigidity;
    p.baseValues.cellFusionVelocity = a.cellFusionVelocity;
    p.baseValues.cellMaxBindingEnergy = a.cellMaxBindingEnergy;
    for (int c = 0; c < MAX_COLORS; ++c) {
        p.cellMaxBindingDistance[c] = a.cellMaxBindingDistance[c];
        p.radiationMinCellAge[c] = a.radiationMinCellAge[c];
        p.highRadiationFactor[c] = a.highRadiationFactor[c];
        p.highRadiationMinCellEnergy[c] = a.highRadiationMinCellEnergy[c];
        p.cellMaxAge[c] = a.cellMaxAge[c];
        p.particleSplitEnergy[c] = a.particleSplitEnergy[c];
        p.baseValues.radiationAbsorption[c] = a.radiationAbsorption[c];
        p.baseValues.radiationCellAgeStrength[c] = a.radiationCellAgeStrength[c];
        p.baseValues.cellMaxForce[c] = a.cellMaxForce[c];
        p.baseValues.cellMinEnergy[c] = a.cellMinEnergy[c];
        p.baseValues.cellDeathProbability[c] = a.cellDeathProbability[c];
        p.externalEnergyBackflowFactor[c] = a.externalEnergyBackflowFactor[c];
    }
    p.baseValues.radiationDisableSources = a.radiationDisableSources != 0;
    p.features.externalEnergyControl = a.externalEnergyControl != 0;
    p.externalEnergy = a.externalEnergy;
    p.externalEnergyBackflowLimit = a.externalEnergyBackflowLimit;

    p.numZones = a.numZones;
    for (int i = 0; i < a.numZones; ++i) {
        AlienZone const& z = a.zones[i];
        SimulationParametersZone& r = p.zone[i];
        r.posX = z.posX;
        r.posY = z.posY;
        r.velX = z.velX;
        r.velY = z.velY;
        r.fadeoutRadius = z.fadeoutRadius;
        r.shapeType = z.shapeType;
        if (z.shapeType == SpotShapeType_Circular) {
            r.shapeData.circularSpot.coreRadius = z.coreRadius;
        } else {
            r.shapeData.rectangularSpot.width = z.width;
            r.shapeData.rectangularSpot.height = z.height;
        }
        r.flowType = z.flowType;
        if (z.flowType == FlowType_Radial) {
            r.flowData.radialFlow.orientation = z.flowOrientation;
            r.flowData.radialFlow.strength = z.flowStrength;
            r.flowData.radialFlow.driftAngle = z.flowDriftAngle;
        } else if (z.flowType == FlowType_Central) {
            r.flowData.centralFlow.strength = z.flowStrength;
        } else if (z.flowType == FlowType_Linear) {
            r.flowData.linearFlow.angle = z.flowAngle;
            r.flowData.linearFlow.strength = z.flowStrength;
        }
        r.values.friction = z.friction;
        r.values.rigidity = z.rigidity;
        r.values.radiationDisableSources = z.radiationDisableSources != 0;
        r.values.cellFusionVelocity = z.cellFusionVelocity;
        r.values.cellMaxBindingEnergy = z.cellMaxBindingEnergy;
        for (int c = 0; c < MAX_COLORS; ++c) {
            r.values.radiationAbsorption[c] = z.radiationAbsorption[c];
            r.values.radiationCellAgeStrength[c] = z.radiationCellAgeStrength[c];
            r.values.cellMaxForce[c] = z.cellMaxForce[c];
            r.values.cellMinEnergy[c] = z.cellMinEnergy[c];
            r.values.cellDeathProbability[c] = z.cellDeathProbability[c];
        }
        r.activatedValues.friction = z.frictionActivated != 0;
        r.activatedValues.rigidity = z.rigidityActivated != 0;
        r.activatedValues.radiationAbsorption = z.radiationAbsorptionActivated != 0;
        r.activatedValues.radiationCellAgeStrength = z.radiationCellAgeStrengthActivated != 0;
        r.activatedValues.radiationDisableSources = z.radiationDisableSourcesActivated != 0;
        r.activatedValues.cellMaxForce = z.cellMaxForceActivated != 0;
        r.activatedValues.cellMinEnergy = z.cellMinEnergyActivated != 0;
        r.activatedValues.cellDeathProbability = z.cellDeathProbabilityActivated != 0;
        r.activatedValues.cellFusionVelocity = z.cellFusionVelocityActivated != 0;
        r.activatedValues.cellMaxBindingEnergy = z.cellMaxBindingEnergyActivated != 0;
    }
    p.numRadiationSources = a.numRadiationSources;
    for (int i = 0; i < a.numRadiationSources; ++i) {
        AlienRadiationSource const& s = a.radiationSources[i];
        RadiationSource& r = p.radiationSource[i];
        r.strength = s.strength;
        r.posX = s.posX;
        r.posY = s.posY;
        r.velX = s.velX;
        r.velY = s.velY;
        r.useAngle = s.useAngle != 0;
        r.angle = s.angle;
        r.shapeType = s.shapeType;
        if (s.shapeType == RadiationSourceShapeType_Circular) {
            r.shapeData.circularRadiationSource.radius = s.radius;
        } else {
            r.shapeData.rectangularRadiationSource.width = s.width;
            r.shapeData.rectangularRadiationSource.height = s.height;
        }
    }
    return p;
}
}  // namespace

int main(int argc, char** argv)
{
    if (argc != 3 && argc != 4) {
        fprintf(stderr, "usage: ref_run <input> <output> [<density map output>]\n");
        return 2;
    }
    try {
        FILE* in = fopen(argv[1], "rb");
        if (!in) throw std::runtime_error("cannot open input");
        char magic[4];
        uint32_t version;
        int32_t W, H;
        uint64_t timestep, warmup, steps, nc, np, na;
        AlienPhysicsParams params;
        readOrThrow(in, magic, 4);
        if (std::memcmp(magic, "ALRF", 4) != 0) throw std::runtime_error("bad magic");
        readOrThrow(in, &version);
        readOrThrow(in, &W);
        readOrThrow(in, &H);
        readOrThrow(in, &timestep);
        readOrThrow(in, &warmup);
        readOrThrow(in, &steps);
        readOrThrow(in, &params);
        readOrThrow(in, &nc);
        readOrThrow(in, &np);
        readOrThrow(in, &na);
        std::vector<CellTO> cells(nc + 1);
        std::vector<ParticleTO> particles(np + 1);
        std::vector<uint8_t> aux(na + 1);
        readOrThrow(in, cells.data(), nc);
        readOrThrow(in, particles.data(), np);
        readOrThrow(in, aux.data(), na);
        fclose(in);

        Settings settings;
        settings.generalSettings.worldSizeX = W;
        settings.generalSettings.worldSizeY = H;
        settings.simulationParameters = toReference(params);
        // never destroyed: when a CUDA call inside the facade throws, its
        // destructor (run during unwinding) throws again from cudaFree and
        // aborts the process before the first error is reported
        auto* facade = new _SimulationCudaFacade(timestep, settings);

        // pre-size the arrays as the reference's own setSimulationData path
        // does (exact counts; the facade keeps 3x headroom), plus room for
        // particles from dying cells, so that no timed step includes a
        // resize.  Larger requests overflow the int bound of the dynamic
        // memory in SimulationData::resizeObjects (SimulationData.cu:93):
        // for cell arrays above 6,391,320 entries, i.e. worlds above about
        // 1.83M cells, it wraps to an undersized buffer and the reference's
        // kernels fail; oracle/refrun.py refuses such worlds.
        ArraySizes additional{nc, np + nc / 4, na};
        facade->resizeArraysIfNecessary(additional);

        DataTO to;
        uint64_t ncIn = nc, npIn = np, naIn = na;
        to.numCells = &ncIn;
        to.cells = cells.data();
        to.numParticles = &npIn;
        to.particles = particles.data();
        to.numAuxiliaryData = &naIn;
        to.auxiliaryData = aux.data();
        facade->setSimulationData(to);

        facade->calcTimestep(warmup, false);
        auto t0 = std::chrono::steady_clock::now();
        facade->calcTimestep(steps, false);
        auto t1 = std::chrono::steady_clock::now();
        double seconds = std::chrono::duration<double>(t1 - t0).count();

        ArraySizes sizes = facade->getArraySizes();
        DataTO out;
        out.init(sizes);
        facade->getSimulationData({-10, -10}, {W + 10, H + 10}, out);
        uint64_t ts = facade->getCurrentTimestep();

        FILE* o = fopen(argv[2], "wb");
        if (!o) throw std::runtime_error("cannot open output");
        writeOrThrow(o, "ALRO", 4);
        uint32_t v = 1;
        writeOrThrow(o, &v);
        writeOrThrow(o, out.numCells);
        writeOrThrow(o, out.numParticles);
        writeOrThrow(o, out.numAuxiliaryData);
        writeOrThrow(o, &seconds);
        writeOrThrow(o, &ts);
        writeOrThrow(o, out.cells, *out.numCells);
        writeOrThrow(o, out.particles, *out.numParticles);
        writeOrThrow(o, out.auxiliaryData, *out.numAuxiliaryData);
        fclose(o);
        out.destroy();
        if (argc == 4) {
            DensityMap const& dm = ((*facade).*memberOf(FacadeData{}))->preprocessedSimulationData.densityMap;
            int2 const size = dm.*memberOf(MapSize{});
            const size_t n = static_cast<size_t>(size.x) * size.y;
            FILE* d = fopen(argv[3], "wb");
            if (!d) throw std::runtime_error("cannot open density map output");
            writeOrThrow(d, "ALDM", 4);
            writeOrThrow(d, &size.x);
            writeOrThrow(d, &size.y);
            auto put = [&](auto* devicePtr) {
                std::vector<std::remove_pointer_t<decltype(devicePtr)>> host(n);
                if (cudaMemcpy(host.data(), devicePtr, n * sizeof(host[0]), cudaMemcpyDeviceToHost) != cudaSuccess)
                    throw std::runtime_error("density map copy failed");
                writeOrThrow(d, host.data(), n);
            };
            put(dm.*memberOf(MapColor{}));
            put(dm.*memberOf(MapOther{}));
            put(dm.*memberOf(MapSame1{}));
            put(dm.*memberOf(MapSame2{}));
            put(dm.*memberOf(MapSpecific{}));
            put(dm.*memberOf(MapLess1{}));
            put(dm.*memberOf(MapLess2{}));
            put(dm.*memberOf(MapMore1{}));
            put(dm.*memberOf(MapMore2{}));
            fclose(d);
        }
        // process exit releases the facade's device memory
        fflush(nullptr);
        std::_Exit(0);
    } catch (std::exception const& e) {
        fprintf(stderr, "ref_run: %s\n", e.what());
        return 1;
    }
    return 0;
}
