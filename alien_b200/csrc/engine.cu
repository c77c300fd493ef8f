// engine.cu - host side of the B200 engine: the arena of worlds, the step
// launch sequence, data transfer and the C ABI declared in
// include/alien_b200.h.
//
// Arena  : one set of SoA device arrays for N independent worlds; one step
//          of all worlds is one launch per phase (kernels.cuh), replayed from
//          a CUDA graph.
// Facade : alien_b200_simulation = an arena of one world, the counterpart of
//          _SimulationCudaFacade (source/EngineGpuKernels/SimulationCudaFacade.cuh:27-139).
// Batch  : alien_b200_batch = an arena of many worlds stepped together.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/alien_b200.h"
#include "../../include/alien_b200_batch.h"
#include "device_common.cuh"
#include "io_kernels.cuh"
#include "kernels.cuh"
#include "rigidity.cuh"

namespace ab {

thread_local std::string g_lastError;

void setLastError(const std::string& message) { g_lastError = message; }

struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define AB_CK(x)                                                                                           \
    do {                                                                                                   \
        cudaError_t e_ = (x);                                                                              \
        if (e_ != cudaSuccess) {                                                                           \
            throw Error(e_ == cudaErrorMemoryAllocation ? ALIEN_B200_ERR_OUT_OF_MEMORY : ALIEN_B200_ERR_CUDA, \
                        std::string(#x) + ": " + cudaGetErrorString(e_));                                  \
        }                                                                                                  \
    } while (0)

#define launch(kernel, ...) launchNamed(#kernel, kernel, __VA_ARGS__)
#define launchSmem(kernel, ...) launchNamedSmem(#kernel, kernel, __VA_ARGS__)

static inline long long roundUp(long long v, long long m) { return (v + m - 1) / m * m; }
static inline int divUp(long long v, long long m) { return static_cast<int>((v + m - 1) / m); }

// Device arrays of an arena, allocated stream-ordered from the device's
// default memory pool on the arena's stream.  The pool keeps freed blocks
// (its release threshold is raised once per device), so a rebuild with the
// same layout, or a new arena after a finished one (the serving loop), gets
// its arrays back without cudaMalloc, and freeing never synchronises the
// device.
class DeviceMemory {
public:
    ~DeviceMemory() { freeAll(); }
    void setStream(cudaStream_t stream) { stream_ = stream; }
    // counting mode: allocations only add up their sizes (reserveBytes)
    void setCountOnly(bool on) { countOnly_ = on; }
    template <class T>
    T* alloc(size_t n)
    {
        const size_t bytes = std::max<size_t>(n, 1) * sizeof(T);
        if (countOnly_) {
            bytes_ += bytes;
            return nullptr;
        }
        void* p = nullptr;
        cudaError_t e = cudaMallocAsync(&p, bytes, stream_);
        if (e != cudaSuccess) {
            cudaGetLastError();
            throw Error(ALIEN_B200_ERR_OUT_OF_MEMORY, "device allocation of " + std::to_string(bytes) + " bytes failed");
        }
        live_.emplace_back(p, bytes);
        bytes_ += bytes;
        return static_cast<T*>(p);
    }
    // one allocation returned in stream order (a replaced array)
    void release(const void* p)
    {
        for (size_t i = 0; i < live_.size(); ++i) {
            if (live_[i].first != p) continue;
            cudaFreeAsync(live_[i].first, stream_);
            bytes_ -= live_[i].second;
            live_[i] = live_.back();
            live_.pop_back();
            return;
        }
    }
    void freeAll()
    {
        for (auto& a : live_) cudaFreeAsync(a.first, stream_);
        live_.clear();
        bytes_ = 0;
    }
    size_t bytes() const { return bytes_; }

private:
    cudaStream_t stream_ = nullptr;
    std::vector<std::pair<void*, size_t>> live_;
    size_t bytes_ = 0;
    bool countOnly_ = false;
};

// A device buffer that keeps its allocation across arena rebuilds and only
// grows: the transfer-object staging of set_data and the egress buffers of
// get_data, whose sizes repeat from call to call.
class GrowBuffer {
public:
    ~GrowBuffer()
    {
        if (p_) cudaFree(p_);
    }
    void* ensure(size_t bytes)
    {
        if (bytes <= cap_) return p_;
        if (p_) cudaFree(p_);
        p_ = nullptr;
        cap_ = 0;
        if (cudaMalloc(&p_, bytes) != cudaSuccess) {
            cudaGetLastError();
            p_ = nullptr;
            throw Error(ALIEN_B200_ERR_OUT_OF_MEMORY, "cudaMalloc of " + std::to_string(bytes) + " bytes failed");
        }
        cap_ = bytes;
        return p_;
    }
    size_t bytes() const { return cap_; }
    void release()
    {
        if (p_) cudaFree(p_);
        p_ = nullptr;
        cap_ = 0;
    }

private:
    void* p_ = nullptr;
    size_t cap_ = 0;
};

// parameters the physics stage cannot honour are rejected, not ignored
static void validateParams(const AlienPhysicsParams& p, int W, int H)
{
    if (p.numZones < 0 || p.numZones > ALIEN_B200_MAX_ZONES)
        throw Error(ALIEN_B200_ERR_INVALID_ARGUMENT, "numZones must lie in [0, 20]");
    if (p.numRadiationSources < 0 || p.numRadiationSources > ALIEN_B200_MAX_RADIATION_SOURCES)
        throw Error(ALIEN_B200_ERR_INVALID_ARGUMENT, "numRadiationSources must lie in [0, 40]");
    if (p.particleTransformationAllowed)
        throw Error(ALIEN_B200_ERR_UNSUPPORTED, "particle-to-cell transformation is outside the physics stage");
    if (p.cellAgeLimiter || p.cellColorTransitionRules || p.advancedAbsorptionControl)
        throw Error(ALIEN_B200_ERR_UNSUPPORTED, "feature flags of cell functions (age limiter, color transitions, absorption control) must be off");
    for (int i = 0; i < p.numZones; ++i) {
        const AlienZone& z = p.zones[i];
        if (z.shapeType != ALIEN_B200_SHAPE_CIRCULAR && z.shapeType != ALIEN_B200_SHAPE_RECTANGULAR)
            throw Error(ALIEN_B200_ERR_INVALID_ARGUMENT, "zone shape type must be 0 (circular) or 1 (rectangular)");
        if (z.flowType < ALIEN_B200_FLOW_NONE || z.flowType > ALIEN_B200_FLOW_LINEAR)
            throw Error(ALIEN_B200_ERR_INVALID_ARGUMENT, "zone flow type must lie in [0, 3]");
    }
    for (int i = 0; i < p.numRadiationSources; ++i)
        if (p.radiationSources[i].shapeType != ALIEN_B200_SHAPE_CIRCULAR && p.radiationSources[i].shapeType != ALIEN_B200_SHAPE_RECTANGULAR)
            throw Error(ALIEN_B200_ERR_INVALID_ARGUMENT, "radiation source shape type must be 0 (circular) or 1 (rectangular)");
    if (p.cellNumExecutionOrderNumbers < 1)
        throw Error(ALIEN_B200_ERR_INVALID_ARGUMENT, "cellNumExecutionOrderNumbers must be at least 1");
    if (p.motionType != ALIEN_B200_MOTION_FLUID && p.motionType != ALIEN_B200_MOTION_COLLISION)
        throw Error(ALIEN_B200_ERR_INVALID_ARGUMENT, "motionType must be 0 (fluid) or 1 (collision)");
    if (!(p.smoothingLength > 0.0f) || !(p.cellMaxCollisionDistance > 0.0f))
        throw Error(ALIEN_B200_ERR_INVALID_ARGUMENT, "interaction radii must be positive");
    const int r = p.motionType == ALIEN_B200_MOTION_FLUID ? static_cast<int>(ceilf(p.smoothingLength * 2.0f))
                                                          : static_cast<int>(ceilf(p.cellMaxCollisionDistance));
    if (r > kMaxRadius) throw Error(ALIEN_B200_ERR_UNSUPPORTED, "interaction radius above 15 slots");
    if (W < 2 * r + 1 || H < 2 * r + 1) throw Error(ALIEN_B200_ERR_INVALID_ARGUMENT, "world smaller than the interaction window");
}

static int scanRadius(const AlienPhysicsParams& p)
{
    return std::max(1, p.motionType == ALIEN_B200_MOTION_FLUID ? static_cast<int>(ceilf(p.smoothingLength * 2.0f))
                                                               : static_cast<int>(ceilf(p.cellMaxCollisionDistance)));
}

struct WorldSetup {
    int W = 0, H = 0;
    AlienPhysicsParams params{};
    uint64_t timestep = 0;
    const AlienCellTO* cells = nullptr;
    uint64_t numCells = 0;
    const AlienParticleTO* particles = nullptr;
    uint64_t numParticles = 0;
    const uint8_t* aux = nullptr;
    uint64_t numAux = 0;
    uint64_t extraParticles = 0;  // capacity beyond the default
};

struct HostWorld {
    WorldInfo info;
    AlienPhysicsParams params;
    // opaque auxiliary bytes, returned unchanged: on the device (at
    // info.auxBase in the arena's aux array) when the arena holds neurons,
    // which read their weights there, else kept here on the host
    uint64_t auxSize = 0;
    std::vector<uint8_t> aux;
    // live arenas: an unused world slot, and what the admission check found
    bool vacant = false;
    uint32_t neurons = 0, signals = 0;
    // the timestep the world was set with (its step counter has not moved
    // past it when no step ran since)
    uint64_t setTimestep = 0;
};

// first-fit ranges of [0, capacity): the cell blocks, particle blocks, tiles,
// particle-map slots and auxiliary bytes of a live arena
class RangePool {
public:
    void init(long long capacity)
    {
        cap_ = capacity;
        free_.clear();
        if (capacity > 0) free_[0] = capacity;
    }
    // start of a free range of n units, or -1
    long long alloc(long long n)
    {
        if (n <= 0) return 0;
        for (auto it = free_.begin(); it != free_.end(); ++it)
            if (it->second >= n) {
                const long long start = it->first, len = it->second;
                free_.erase(it);
                if (len > n) free_[start + n] = len - n;
                return start;
            }
        return -1;
    }
    void release(long long start, long long n)
    {
        if (n <= 0) return;
        auto next = free_.lower_bound(start);
        if (next != free_.end() && next->first == start + n) {
            n += next->second;
            next = free_.erase(next);
        }
        if (next != free_.begin()) {
            auto prev = std::prev(next);
            if (prev->first + prev->second == start) {
                start = prev->first;
                n += prev->second;
                free_.erase(prev);
            }
        }
        free_[start] = n;
    }
    // one past the last used unit (the launches cover [0, highWater))
    long long highWater() const
    {
        if (free_.empty()) return cap_;
        const auto last = std::prev(free_.end());
        return last->first + last->second == cap_ ? last->first : cap_;
    }
    long long capacity() const { return cap_; }

private:
    long long cap_ = 0;
    std::map<long long, long long> free_;
};

class Arena {
public:
    explicit Arena(cudaStream_t stream) : stream_(stream) { mem_.setStream(stream); }
    ~Arena()
    {
        releaseGraph();
        if (checkStream_) cudaStreamDestroy(checkStream_);
        if (readback_) cudaFreeHost(readback_);
    }

    void build(const std::vector<WorldSetup>& setups);
    // live arenas (alien_b200_arena_create): memory for a stated capacity is
    // reserved once; worlds are admitted into free ranges and evicted while
    // the other worlds keep their state, all in stream order behind the
    // steps already enqueued
    void reserve(const AlienArenaCapacity& capacity);
    int admit(const WorldSetup& ws, uint64_t steps, int slot = -1);
    void evict(int w);
    bool live() const { return live_; }
    bool resident(int w) const { return w >= 0 && w < numWorlds() && !worlds_[w].vacant && (!live_ || w != vacant_); }
    int residentWorlds() const;
    static uint64_t reserveBytes(const AlienArenaCapacity& capacity);
    void enqueueStep();
    void enqueueSteps(uint64_t n);
    // n graph steps bracketed by CUDA events on the arena's stream
    double timeSteps(uint64_t n);
    // n steps without the graph, an event after every launch; returns the
    // summed milliseconds per launch position of the step
    std::vector<double> timedSteps(uint64_t n);
    void calcTimesteps(uint64_t n);
    // waits for the enqueued work and completes halted worlds; throws
    // ALIEN_B200_ERR_CAPACITY when particles were dropped
    void sync();
    // the same without the report (entry points that read a world's state)
    void settle();
    void setParams(int w, const AlienPhysicsParams& p);
    // the parameters as the steps left them: zone and source positions,
    // the external energy pool
    AlienPhysicsParams params(int w);
    void syncParamsFromDevice();
    std::vector<WorldCounters> readCounters();
    void getData(int w, bool useRect, AlienInt2 ul, AlienInt2 lr, const AlienDataTO* out);
    void countData(int w, uint64_t* cells, uint64_t* particles);
    AlienRawStatistics statistics(int w);
    AlienRawStatisticsData statisticsData(int w);
    // the density map of the last step (alien_b200_get_density_map)
    void densityMap(int w, AlienDensityMap* out);
    void resetTimeIntervalStatistics(int w);
    void setTimestep(int w, uint64_t t);
    void setStepBudget(int w, uint64_t steps);
    void compactParticles(int w);
    void ensureParticleCapacity();
    // more particle room for world w (the arena rebuilt, or in a live arena
    // the world's particles moved), with no change of state
    void growParticles(int w, uint64_t extra);
    // the cell map of the current state, built by the step's own binning
    // kernels and read back in tile order (alien_b200_debug_cell_map)
    uint64_t cellMap(uint64_t capacity, uint64_t* ids, uint32_t* slots, uint32_t* tiles, uint8_t* flags);
    // launch configuration of the pair kernel: region shape per motion
    // type, fixed by the caller (candidate index + 1) or chosen by the
    // autotuner (0)
    void setRegionChoice(int motion, int choicePlusOne);
    AlienLaunchConfig launchConfig() const;
    void autotune();

    int numWorlds() const { return static_cast<int>(worlds_.size()); }
    const HostWorld& world(int w) const { return worlds_[w]; }
    uint64_t launches() const { return launches_; }
    size_t deviceBytes() const
    {
        return mem_.bytes() + egressCells_.bytes() + egressParts_.bytes() + stageCells_.bytes() + stageParts_.bytes();
    }
    int kernelsPerStep() const { return kernelsPerStep_; }
    cudaStream_t stream() const { return stream_; }

private:
    template <class K, class... A>
    void launchNamed(const char* name, K kernel, int grid, int block, A... args)
    {
        launchNamedSmem(name, kernel, grid, block, 0, args...);
    }
    template <class K, class... A>
    void launchNamedSmem(const char* name, K kernel, int grid, int block, size_t smem, A... args)
    {
        if (grid <= 0) return;
        kernel<<<grid, block, smem, stream_>>>(args...);
        ++launches_;
        AB_CK(cudaGetLastError());
        if (timingEvents_) {
            cudaEvent_t e;
            AB_CK(cudaEventCreate(&e));
            AB_CK(cudaEventRecord(e, stream_));
            timingEvents_->push_back(e);
            timingNames_.push_back(name);
        }
    }
    std::vector<cudaEvent_t>* timingEvents_ = nullptr;
    std::vector<const char*> timingNames_;

public:
    std::vector<std::string> lastTimedNames;

private:
    void scan(const uint32_t* in, long long n, uint32_t* out);
    // pair-kernel region shapes: the candidates' index in use per motion type,
    // fixed by the caller (index + 1) or chosen by the autotuner
    int regionChoice_[2] = {0, 0};
    int regionChoiceFixed_[2] = {0, 0};
    const int* regionShape(int motion) const { return kRegionChoices[motion][regionChoice_[motion]]; }
    static void assignRegions(WorldInfo& wi, const int* shape);
    static int maxRegions(const WorldInfo& wi);
    void applyRegionShapes();
    template <int Motion>
    void launchPairs()
    {
        launchSmem(kPairsRegion<Motion>, s_.numRegions, kRegionThreads, regionDynSmem<Motion>(), s_);
    }
    void allocCellAndParticleArrays(size_t C, size_t P, long long tiles, long long pmapSlots, int cellBlocks, int partBlocks,
                                    bool clusters);
    void allocParticleArrays(size_t P, int partBlocks);
    void allocParticleArrays(DevState& target, size_t P, int partBlocks);
    // halted worlds (kEventWorld): their particle ranges grown, their step
    // completed by the resume launches, then the steps they missed run with
    // every other world parked; returns whether particles were dropped
    bool resumeHalted();
    // the particle arrays of an arena laid out once (batch or single world)
    // allocated again on the device with the ranges newCap[w] (0: as it
    // is); the used slots move with their step's split records, nothing else
    // of the state changes
    void growParticleArrays(const std::vector<long long>& newCap);
    // growParticleArrays, or an export and rebuild when the device has no
    // room for both sets of arrays
    void growOrRebuild(const std::vector<long long>& newCap);
    bool droppedPending_ = false;  // a resume dropped particles: the next sync() reports it
    bool stepsPending_ = false;    // steps were enqueued since settle() last read the error word
    // page-locked landing place of the small per-step reads (the error word,
    // a world's statistics and counters): a copy into pageable memory goes
    // through a staging buffer and adds to every step's wait
    struct Readback {
        uint32_t flags;
        StatsAcc stats;
        WorldCounters counters;
    };
    Readback* readback_ = nullptr;
    Readback& readback()
    {
        if (!readback_) AB_CK(cudaMallocHost(reinterpret_cast<void**>(&readback_), sizeof(Readback)));
        return *readback_;
    }
    // live arenas
    bool live_ = false;
    AlienArenaCapacity capacity_{};
    RangePool cellPool_, partPool_, tilePool_, pmapPool_, auxPool_;  // cells and particles in blocks of kBlock
    int regionCap_ = 0;
    long long regionsReserved_ = 0;  // the most regions the resident worlds can take (every candidate shape)
    int vacant_ = -1;  // the world slot of every unused block (never active)
    cudaStream_t checkStream_ = nullptr;
    bool layoutDirty_ = false;  // admissions or evictions since the last layout update
    void updateLiveLayout();
    void refreshLayout()
    {
        if (layoutDirty_) {
            layoutDirty_ = false;
            updateLiveLayout();
        }
    }
    // a resident world re-admitted (same slot) from its current state, for
    // a new interaction radius
    void relocate(int w, uint64_t extraParticles, const AlienPhysicsParams* newParams);
    // a resident world's particles moved to a larger free range on the
    // device, with the step's split records when stepScratch (a halted
    // world); false when no range of that size is free
    bool moveParticles(int w, long long newCap, bool stepScratch = false);
    void releaseGraph()
    {
        if (graphExec_) cudaGraphExecDestroy(graphExec_);
        graphExec_ = nullptr;
    }
    // a world's live objects read back for a rebuild, with the state their
    // transfer objects do not hold (kGatherCarried) on the device
    struct Carried {
        std::vector<AlienCellTO> cells;
        std::vector<AlienParticleTO> parts;
        float* density = nullptr;
        unsigned long long* last = nullptr;
    };
    void exportWorld(int w, Carried& out);
    // the arena built again from exported worlds (extra particle room per
    // world); fluid densities continue when keepDensity, else start at 1 as
    // after a parameter change (prepareForSimulationParametersChanges)
    void rebuildFromHost(std::vector<Carried>& worlds, const std::vector<uint64_t>& extra, bool keepDensity);

    cudaStream_t stream_;
    DeviceMemory mem_;
    std::vector<HostWorld> worlds_;
    DevState s_{};
    StatsAcc* stats_ = nullptr;
    TimelineAcc* timeline_ = nullptr;
    AlienCellTO* cold_ = nullptr;
    int* rankCells_ = nullptr;
    int* rankParts_ = nullptr;
    uint32_t* blockCount_ = nullptr;
    GrowBuffer egressCells_, egressParts_, stageCells_, stageParts_;
    long long maxWorldCells_ = 0, maxWorldParts_ = 0;
    uint64_t launches_ = 0;
    int kernelsPerStep_ = 0;
    int partGrid_ = 1;  // blocks of the particle part of a combined launch
    int overflowGrid_ = 1;  // blocks of kPairsOverflow (a grid-stride loop over the deferred cells)
    int statsGrid_ = 1;  // blocks of a statistics reduction
    cudaGraphExec_t graphExec_ = nullptr;
    uint64_t stepsSinceCheck_ = 0;
    bool hasFluid_ = false, hasCollision_ = false, hasNeurons_ = false;
    bool hasWorldParams_ = false;  // some world has zones, radiation sources or external energy (kWorldsEnd)
    bool hasRigidity_ = false;     // some world enables rigidity: the cluster arrays exist and the step runs the cluster pass
    static bool needsWorldParams(const AlienPhysicsParams& p)
    {
        return p.numZones > 0 || p.numRadiationSources > 0 || p.externalEnergyControl;
    }
    bool tuned_ = false;              // the autotuner ran on this layout
    bool motionTuned_[2] = {false, false};  // the autotuner chose the motion type's region shape
    float tunedMs_[2][kNumRegionChoices] = {};
    void binCurrentState();
    bool signalsLive_ = false;  // some cell has a function or a nonzero signal channel
};

// ------------------------------------------------------------- build -----
// cell functions: neurons run in this engine (kNeuron); any other function
// would need the rest of the cell-function stage.  Checked before build()
// changes anything.
static void validateCells(const std::vector<WorldSetup>& setups)
{
    for (const WorldSetup& ws : setups)
        for (uint64_t i = 0; i < ws.numCells; ++i) {
            const AlienCellTO& c = ws.cells[i];
            if (c.numConnections > ALIEN_B200_MAX_CELL_BONDS)
                throw Error(ALIEN_B200_ERR_INVALID_ARGUMENT, "numConnections above 6 (cell id " + std::to_string(c.id) + ")");
            for (int k = 0; k < c.numConnections; ++k)
                if (c.connections[k].cellIndex < 0 || static_cast<uint64_t>(c.connections[k].cellIndex) >= ws.numCells)
                    throw Error(ALIEN_B200_ERR_INVALID_ARGUMENT,
                                "connection cellIndex out of range (cell id " + std::to_string(c.id) + ")");
            if (c.cellFunction == kCellFunctionNone) continue;
            if (c.cellFunction != kCellFunctionNeuron)
                throw Error(ALIEN_B200_ERR_UNSUPPORTED, "cell id " + std::to_string(c.id) + " has cell function "
                                                            + std::to_string(c.cellFunction)
                                                            + "; only neurons (0) and cells without function (11) are supported");
            const uint64_t at = c.cellFunctionData[0];  // NeuronTO.weightsAndBiasesDataIndex
            const uint64_t bytes = sizeof(float) * kNeuronTableStride;
            if (at > ws.numAux || ws.numAux - at < bytes)
                throw Error(ALIEN_B200_ERR_INVALID_ARGUMENT,
                            "neuron data of cell id " + std::to_string(c.id) + " lies outside the auxiliary data");
        }
}

// the pair-phase regions stage up to RegionShape<>::Cap records in dynamic
// shared memory (above the 48 KB default): set before any arena's first step
static void setRegionKernelAttributes()
{
    AB_CK(cudaFuncSetAttribute(kPairsRegion<ALIEN_B200_MOTION_FLUID>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               static_cast<int>(regionDynSmem<ALIEN_B200_MOTION_FLUID>())));
    AB_CK(cudaFuncSetAttribute(kPairsRegion<ALIEN_B200_MOTION_COLLISION>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               static_cast<int>(regionDynSmem<ALIEN_B200_MOTION_COLLISION>())));
}

// the per-cell, per-particle, per-tile and per-block arrays of the arena
// (the cluster arrays of rigidity only when asked for)
void Arena::allocCellAndParticleArrays(size_t C, size_t P, long long tiles, long long pmapSlots, int cellBlocks, int partBlocks,
                                       bool clusters)
{
    DevState& s = s_;
    s.id = mem_.alloc<unsigned long long>(C);
    s.posA = mem_.alloc<float2>(C);
    s.push = mem_.alloc<float2>(C);
    s.dpos = mem_.alloc<float2>(C);
    s.velA = mem_.alloc<float2>(C);
    s.velB = mem_.alloc<float2>(C);
    s.energy = mem_.alloc<float>(C);
    s.stiffness = mem_.alloc<float>(C);
    s.density = mem_.alloc<float>(C);
    s.densNew = mem_.alloc<float>(C);
    s.color = mem_.alloc<uint8_t>(C);
    s.maxConn = mem_.alloc<uint8_t>(C);
    s.numConn = mem_.alloc<uint8_t>(C);
    s.barrier = mem_.alloc<uint8_t>(C);
    s.alive = mem_.alloc<uint8_t>(C);
    s.triMask = mem_.alloc<uint8_t>(C);
    s.livingState = mem_.alloc<uint8_t>(C);
    s.nextState = mem_.alloc<uint8_t>(C);
    s.flags = mem_.alloc<uint32_t>(C);
    s.age = mem_.alloc<uint32_t>(C);
    s.activationTime = mem_.alloc<uint32_t>(C);
    s.creatureId = mem_.alloc<uint32_t>(C);
    s.coldIdx = mem_.alloc<uint32_t>(C);
    s.bond = mem_.alloc<int>(C * kMaxBonds);
    s.bondDist = mem_.alloc<float>(C * kMaxBonds);
    s.bondAngle = mem_.alloc<float>(C * kMaxBonds);
    s.force = mem_.alloc<float2>(C);
    s.force1 = mem_.alloc<float2>(C);
    s.angleAcc = mem_.alloc<long long>(C * 4);
    s.energyAcc = mem_.alloc<long long>(C);
    s.best = mem_.alloc<int>(C);
    s.newPartner = mem_.alloc<int>(C);
    if (clusters) {
        s.clusterLab[0] = mem_.alloc<int>(C);
        s.clusterLab[1] = mem_.alloc<int>(C);
        s.clusterCount = mem_.alloc<uint32_t>(C);
        s.clusterAcc = mem_.alloc<long long>(C * kAccFields);
        s.clusterChanged = mem_.alloc<uint32_t>(kClusterRounds);
    }
    s.addNum = mem_.alloc<uint8_t>(C);
    s.addBond = mem_.alloc<int>(C * kMaxBonds);
    s.addDist = mem_.alloc<float>(C * kMaxBonds);
    s.addAngle = mem_.alloc<float>(C * kMaxBonds);
    s.radPos = mem_.alloc<float2>(C);
    s.radVel = mem_.alloc<float2>(C);
    s.radEnergy = mem_.alloc<float>(C);
    s.tileOf = mem_.alloc<uint32_t>(C);
    s.slotOf = mem_.alloc<uint32_t>(C);
    s.tileOff = mem_.alloc<uint32_t>(C);
    s.sorted = mem_.alloc<uint32_t>(C);
    s.slotInTile = mem_.alloc<uint8_t>(C);
    s.sortedSlot = mem_.alloc<uint8_t>(C);
    s.stagedPV = mem_.alloc<float4>(C);
    s.stagedMeta = mem_.alloc<int4>(C);
    s.tileCount = mem_.alloc<uint32_t>(static_cast<size_t>(tiles) + 1);
    s.pairOverflowCount = s.tileCount + tiles;
    s.pairOverflow = mem_.alloc<uint32_t>(C);
    s.tileStart = mem_.alloc<uint32_t>(static_cast<size_t>(tiles) + 1);
    s.scanPartials = mem_.alloc<uint32_t>(static_cast<size_t>(divUp(tiles, kScanTile)) + 2);

    allocParticleArrays(P, partBlocks);
    s.pmap = mem_.alloc<int>(static_cast<size_t>(pmapSlots));
    s.blockRad = mem_.alloc<uint32_t>(cellBlocks);
    s.blockDel = mem_.alloc<uint32_t>(cellBlocks);
}

void Arena::allocParticleArrays(size_t P, int partBlocks)
{
    allocParticleArrays(s_, P, partBlocks);
}

void Arena::allocParticleArrays(DevState& s, size_t P, int partBlocks)
{
    s.pid = mem_.alloc<unsigned long long>(P);
    s.ppos = mem_.alloc<float2>(P);
    s.pvel = mem_.alloc<float2>(P);
    s.penergy = mem_.alloc<float>(P);
    s.pcolor = mem_.alloc<uint8_t>(P);
    s.palive = mem_.alloc<uint8_t>(P);
    s.pselected = mem_.alloc<uint8_t>(P);
    s.pflag = mem_.alloc<uint32_t>(P);
    s.plast = mem_.alloc<unsigned long long>(P);
    s.ptarget = mem_.alloc<int>(P);
    s.pslot = mem_.alloc<int>(P);
    s.pmerge = mem_.alloc<long long>(P * 3);
    s.splitPos = mem_.alloc<float2>(P);
    s.splitVel = mem_.alloc<float2>(P);
    s.splitEnergy = mem_.alloc<float>(P);
    s.blockSplit = mem_.alloc<uint32_t>(partBlocks);
}

void Arena::build(const std::vector<WorldSetup>& setups)
{
    for (const WorldSetup& ws : setups) {
        if (ws.W <= 0 || ws.H <= 0) throw Error(ALIEN_B200_ERR_INVALID_ARGUMENT, "world size must be positive");
        validateParams(ws.params, ws.W, ws.H);
    }
    // upload the transfer objects and check them on the device before the
    // arena changes (a rejected set_data leaves the previous world in place)
    const int nWorlds = static_cast<int>(setups.size());
    std::vector<AlienCellTO*> stagedCells(nWorlds, nullptr);
    std::vector<AlienParticleTO*> stagedParts(nWorlds, nullptr);
    std::vector<void*> asyncStage;
    auto freeAsyncStage = [&] {
        for (void* p : asyncStage) cudaFreeAsync(p, stream_);
        asyncStage.clear();
    };
    {
        // all worlds' objects side by side in the staging buffers
        size_t totalCells = 0, totalParts = 0;
        for (const WorldSetup& ws : setups) {
            totalCells += ws.numCells;
            totalParts += ws.numParticles;
        }
        AlienCellTO* cellBase = nullptr;
        AlienParticleTO* partBase = nullptr;
        if (nWorlds == 1) {
            // a single-world handle keeps its staging: set_data repeats with the same sizes
            AB_CK(cudaStreamSynchronize(stream_));  // earlier copies out of the staging buffers are done
            cellBase = static_cast<AlienCellTO*>(stageCells_.ensure(sizeof(AlienCellTO) * std::max<size_t>(totalCells, 1)));
            partBase = static_cast<AlienParticleTO*>(stageParts_.ensure(sizeof(AlienParticleTO) * std::max<size_t>(totalParts, 1)));
        } else {
            // a batch is built once: stream-ordered staging, released without
            // synchronising the device (other arenas keep stepping meanwhile)
            AB_CK(cudaMallocAsync(reinterpret_cast<void**>(&cellBase), sizeof(AlienCellTO) * std::max<size_t>(totalCells, 1), stream_));
            AB_CK(cudaMallocAsync(reinterpret_cast<void**>(&partBase), sizeof(AlienParticleTO) * std::max<size_t>(totalParts, 1),
                                  stream_));
            asyncStage = {cellBase, partBase};
        }
        size_t c0 = 0, p0 = 0;
        for (int w = 0; w < nWorlds; ++w) {
            if (setups[w].numCells) stagedCells[w] = cellBase + c0;
            if (setups[w].numParticles) stagedParts[w] = partBase + p0;
            c0 += setups[w].numCells;
            p0 += setups[w].numParticles;
        }
    }
    uint32_t neuronsTotal = 0, signalsTotal = 0;
    {
        IngestCheck* dCheck = nullptr;
        AB_CK(cudaMallocAsync(reinterpret_cast<void**>(&dCheck), sizeof(IngestCheck) * std::max(nWorlds, 1), stream_));
        AB_CK(cudaMemsetAsync(dCheck, 0, sizeof(IngestCheck) * std::max(nWorlds, 1), stream_));
        try {
            for (int w = 0; w < nWorlds; ++w) {
                const WorldSetup& ws = setups[w];
                const long long nc = static_cast<long long>(ws.numCells), np = static_cast<long long>(ws.numParticles);
                if (nc) {
                    AB_CK(cudaMemcpyAsync(stagedCells[w], ws.cells, sizeof(AlienCellTO) * nc, cudaMemcpyHostToDevice, stream_));
                    launch(kCheckCells, divUp(nc, kBlock), kBlock, static_cast<const AlienCellTO*>(stagedCells[w]), nc,
                           static_cast<unsigned long long>(ws.numAux), dCheck + w);
                }
                if (np) {
                    AB_CK(cudaMemcpyAsync(stagedParts[w], ws.particles, sizeof(AlienParticleTO) * np, cudaMemcpyHostToDevice,
                                          stream_));
                }
            }
            std::vector<IngestCheck> checks(std::max(nWorlds, 1));
            AB_CK(cudaMemcpyAsync(checks.data(), dCheck, sizeof(IngestCheck) * checks.size(), cudaMemcpyDeviceToHost, stream_));
            AB_CK(cudaStreamSynchronize(stream_));
            bool bad = false;
            for (int w = 0; w < nWorlds; ++w) {
                const IngestCheck& c = checks[w];
                bad |= c.badBondCount || c.badBondIndex || c.otherFunction || c.neuronOutOfAux;
                neuronsTotal += c.neurons;
                signalsTotal += c.nonzeroSignal;
            }
            if (bad) {
                validateCells(setups);  // the host scan names the first offending cell
                throw Error(ALIEN_B200_ERR_INVALID_ARGUMENT, "invalid cell transfer objects");
            }
        } catch (...) {
            cudaFreeAsync(dCheck, stream_);
            freeAsyncStage();
            cudaStreamSynchronize(stream_);
            throw;
        }
        AB_CK(cudaFreeAsync(dCheck, stream_));
    }
    releaseGraph();
    AB_CK(cudaStreamSynchronize(stream_));
    mem_.freeAll();
    worlds_.clear();
    tuned_ = false;  // a new layout is tuned again at its first step
    motionTuned_[0] = motionTuned_[1] = false;
    std::memset(tunedMs_, 0, sizeof(tunedMs_));
    for (int m = 0; m < 2; ++m) regionChoice_[m] = regionChoiceFixed_[m] ? regionChoiceFixed_[m] - 1 : 0;
    const int n = static_cast<int>(setups.size());
    long long cellSlots = 0, partSlots = 0, tiles = 0, pmapSlots = 0, coldTotal = 0, auxTotal = 0;
    int regions = 0, regionsCap = 0;  // regions of the current shapes; most regions any candidate shape gives
    int cellBlocks = 0, partBlocks = 0;
    maxWorldCells_ = maxWorldParts_ = 0;
    for (int w = 0; w < n; ++w) {
        const WorldSetup& ws = setups[w];
        if (ws.W <= 0 || ws.H <= 0) throw Error(ALIEN_B200_ERR_INVALID_ARGUMENT, "world size must be positive");
        validateParams(ws.params, ws.W, ws.H);
        if (ws.numCells > (1ull << 30) || ws.numParticles > (1ull << 30))
            throw Error(ALIEN_B200_ERR_CAPACITY, "more than 2^30 objects in one world");
        HostWorld hw;
        hw.params = ws.params;
        hw.setTimestep = ws.timestep;
        WorldInfo& wi = hw.info;
        wi.W = ws.W;
        wi.H = ws.H;
        wi.radiusInt = scanRadius(ws.params);
        wi.T = wi.radiusInt;
        wi.nTX = divUp(ws.W, wi.T);
        wi.nTY = divUp(ws.H, wi.T);
        wi.motionType = ws.params.motionType;
        wi.paramIndex = w;
        wi.tileBase = tiles;
        tiles += static_cast<long long>(wi.nTX) * wi.nTY;
        wi.cellCap = roundUp(std::max<long long>(static_cast<long long>(ws.numCells), 1), kBlock);
        const long long np = static_cast<long long>(ws.numParticles), nc = static_cast<long long>(ws.numCells);
        wi.partCap = roundUp(np + nc + std::max<long long>(4096, (np + nc) / 2) + static_cast<long long>(ws.extraParticles), kBlock);
        wi.cellBase = cellSlots;
        wi.partBase = partSlots;
        wi.firstCellBlock = cellBlocks;
        wi.numCellBlocks = static_cast<int>(wi.cellCap / kBlock);
        wi.firstPartBlock = partBlocks;
        wi.numPartBlocks = static_cast<int>(wi.partCap / kBlock);
        wi.pmapBase = pmapSlots;
        assignRegions(wi, regionShape(wi.motionType));
        regionsCap += maxRegions(wi);
        wi.regionBase = regions;
        regions += wi.nRX * wi.nRY;
        pmapSlots += static_cast<long long>(ws.W) * ws.H;
        cellSlots += wi.cellCap;
        partSlots += wi.partCap;
        cellBlocks += wi.numCellBlocks;
        partBlocks += wi.numPartBlocks;
        coldTotal += nc;
        maxWorldCells_ = std::max(maxWorldCells_, wi.cellCap);
        maxWorldParts_ = std::max(maxWorldParts_, wi.partCap);
        hw.auxSize = ws.numAux;
        hw.info.auxBase = auxTotal;
        auxTotal += static_cast<long long>(ws.numAux);
        worlds_.push_back(std::move(hw));
    }
    hasNeurons_ = neuronsTotal > 0;
    signalsLive_ = hasNeurons_ || signalsTotal > 0;
    hasFluid_ = hasCollision_ = hasWorldParams_ = hasRigidity_ = false;
    for (const HostWorld& hw : worlds_) {
        hasWorldParams_ |= needsWorldParams(hw.params);
        hasRigidity_ |= rigidityEnabled(hw.params);
        if (hw.info.motionType == ALIEN_B200_MOTION_FLUID)
            hasFluid_ = true;
        else
            hasCollision_ = true;
    }
    if (cellSlots >= (1ll << 31) || partSlots >= (1ll << 31) || tiles >= (1ll << 32) - 2)
        throw Error(ALIEN_B200_ERR_CAPACITY, "arena exceeds 2^31 slots");

    setRegionKernelAttributes();
    DevState& s = s_;
    s = DevState{};
    s.numWorlds = n;
    s.numCellBlocks = cellBlocks;
    s.numPartBlocks = partBlocks;
    {
        // particle parts of the combined launches stride over the used
        // particle blocks with at most 16 blocks per SM
        int device = 0, sms = 0;
        AB_CK(cudaGetDevice(&device));
        AB_CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
        partGrid_ = std::max(1, std::min(partBlocks, 16 * std::max(sms, 1)));
        statsGrid_ = 4 * std::max(sms, 1);
        overflowGrid_ = std::max(1, std::min(cellBlocks, 2 * std::max(sms, 1)));
    }
    s.cellSlots = cellSlots;
    s.partSlots = partSlots;
    s.numTiles = tiles;
    const size_t C = static_cast<size_t>(cellSlots), P = static_cast<size_t>(partSlots);

    auto* worldsDev = mem_.alloc<WorldInfo>(n);
    s.worlds = worldsDev;
    s.counters = mem_.alloc<WorldCounters>(n);
    auto* paramsDev = mem_.alloc<AlienPhysicsParams>(n);
    s.params = paramsDev;
    auto* rgw = mem_.alloc<int>(regionsCap);
    s.regionWorld = rgw;
    s.numRegions = regions;
    auto* cbw = mem_.alloc<int>(cellBlocks);
    auto* pbw = mem_.alloc<int>(partBlocks);
    s.cellBlockWorld = cbw;
    s.partBlockWorld = pbw;
    s.errorFlags = mem_.alloc<uint32_t>(1);

    allocCellAndParticleArrays(C, P, tiles, pmapSlots, cellBlocks, partBlocks, hasRigidity_);

    stats_ = mem_.alloc<StatsAcc>(n);
    timeline_ = mem_.alloc<TimelineAcc>(1);
    s.neuronActivity = mem_.alloc<unsigned long long>(static_cast<size_t>(n) * ALIEN_B200_MAX_COLORS);
    cold_ = mem_.alloc<AlienCellTO>(static_cast<size_t>(coldTotal));
    s.cold = cold_;
    s.fnInfo = nullptr;
    s.aux = nullptr;
    if (signalsLive_) s.fnInfo = mem_.alloc<uchar4>(C);  // filled by kIngestCells
    if (hasNeurons_) {
        // neuron weights and biases are read where they lie in the
        // auxiliary data, uploaded once per build straight from the
        // caller's buffers (the build synchronises before it returns); the
        // device copy is the only one
        long long auxBytes = 0;
        for (const HostWorld& hw : worlds_) auxBytes += static_cast<long long>(hw.auxSize);
        uint8_t* auxDev = mem_.alloc<uint8_t>(static_cast<size_t>(std::max<long long>(auxBytes, 1)));
        for (size_t w = 0; w < worlds_.size(); ++w)
            if (worlds_[w].auxSize)
                AB_CK(cudaMemcpyAsync(auxDev + worlds_[w].info.auxBase, setups[w].aux, worlds_[w].auxSize,
                                      cudaMemcpyHostToDevice, stream_));
        s.aux = auxDev;
    } else {
        for (size_t w = 0; w < worlds_.size(); ++w)
            if (worlds_[w].auxSize) worlds_[w].aux.assign(setups[w].aux, setups[w].aux + worlds_[w].auxSize);
    }
    rankCells_ = mem_.alloc<int>(C);
    rankParts_ = mem_.alloc<int>(P);
    blockCount_ = mem_.alloc<uint32_t>(static_cast<size_t>(std::max(cellBlocks, partBlocks)) + 2);

    // host-side tables
    std::vector<WorldInfo> infos(n);
    std::vector<AlienPhysicsParams> params(n);
    std::vector<int> cbwHost(cellBlocks), pbwHost(partBlocks), rgwHost(regions);
    std::vector<WorldCounters> counters(n);
    for (int w = 0; w < n; ++w) {
        infos[w] = worlds_[w].info;
        params[w] = worlds_[w].params;
        for (int b = 0; b < infos[w].numCellBlocks; ++b) cbwHost[infos[w].firstCellBlock + b] = w;
        for (int b = 0; b < infos[w].numPartBlocks; ++b) pbwHost[infos[w].firstPartBlock + b] = w;
        for (int r = 0; r < infos[w].nRX * infos[w].nRY; ++r) rgwHost[infos[w].regionBase + r] = w;
        WorldCounters& wc = counters[w];
        std::memset(&wc, 0, sizeof(wc));
        wc.timestep = setups[w].timestep;
        wc.nextId = 1;
        wc.numCells = static_cast<unsigned int>(setups[w].numCells);
        wc.numParticles = static_cast<unsigned int>(setups[w].numParticles);
        wc.stepsRemaining = ~0ull;
        wc.active = 1;
        wc.signalsFresh = 1;
        wc.externalEnergy = setups[w].params.externalEnergy;
        wc.lastStepped = ~0ull;
    }
    AB_CK(cudaMemcpyAsync(worldsDev, infos.data(), sizeof(WorldInfo) * n, cudaMemcpyHostToDevice, stream_));
    AB_CK(cudaMemcpyAsync(paramsDev, params.data(), sizeof(AlienPhysicsParams) * n, cudaMemcpyHostToDevice, stream_));
    AB_CK(cudaMemcpyAsync(s.counters, counters.data(), sizeof(WorldCounters) * n, cudaMemcpyHostToDevice, stream_));
    if (cellBlocks) AB_CK(cudaMemcpyAsync(cbw, cbwHost.data(), sizeof(int) * cellBlocks, cudaMemcpyHostToDevice, stream_));
    if (partBlocks) AB_CK(cudaMemcpyAsync(pbw, pbwHost.data(), sizeof(int) * partBlocks, cudaMemcpyHostToDevice, stream_));
    if (regions) AB_CK(cudaMemcpyAsync(rgw, rgwHost.data(), sizeof(int) * regions, cudaMemcpyHostToDevice, stream_));
    AB_CK(cudaMemsetAsync(s.errorFlags, 0, sizeof(uint32_t), stream_));
    AB_CK(cudaMemsetAsync(s.alive, 0, C, stream_));
    AB_CK(cudaMemsetAsync(s.palive, 0, P, stream_));
    AB_CK(cudaMemsetAsync(s.pflag, 0, P * sizeof(uint32_t), stream_));
    AB_CK(cudaMemsetAsync(s.pmap, 0xff, static_cast<size_t>(pmapSlots) * sizeof(int), stream_));
    AB_CK(cudaMemsetAsync(s.flags, 0, C * sizeof(uint32_t), stream_));
    AB_CK(cudaMemsetAsync(s.angleAcc, 0, C * 4 * sizeof(long long), stream_));
    AB_CK(cudaMemsetAsync(s.dpos, 0, C * sizeof(float2), stream_));
    AB_CK(cudaMemsetAsync(s.push, 0, C * sizeof(float2), stream_));
    AB_CK(cudaMemsetAsync(s.neuronActivity, 0, sizeof(unsigned long long) * n * ALIEN_B200_MAX_COLORS, stream_));
    AB_CK(cudaMemsetAsync(s.energyAcc, 0, C * sizeof(long long), stream_));
    AB_CK(cudaMemsetAsync(s.newPartner, 0xff, C * sizeof(int), stream_));
    AB_CK(cudaMemsetAsync(s.best, 0xff, C * sizeof(int), stream_));

    // ingest: host TOs -> device staging -> SoA (cudaCreateDataFromTO)
    long long coldBase = 0;
    for (int w = 0; w < n; ++w) {
        const WorldSetup& ws = setups[w];
        const long long nc = static_cast<long long>(ws.numCells), np = static_cast<long long>(ws.numParticles);
        const AlienCellTO* dCells = stagedCells[w];
        const AlienParticleTO* dParts = stagedParts[w];
        if (nc)
            AB_CK(cudaMemcpyAsync(cold_ + coldBase, dCells, sizeof(AlienCellTO) * static_cast<size_t>(nc), cudaMemcpyDeviceToDevice,
                                  stream_));
        launch(kIngestCells, divUp(nc, kBlock), kBlock, s, w, static_cast<const AlienCellTO*>(dCells), nc, cold_, coldBase);
        launch(kIngestParticles, divUp(np, kBlock), kBlock, s, w, static_cast<const AlienParticleTO*>(dParts), np);
        launch(kMaxId, divUp(std::max(nc, np), kBlock), kBlock, s, w, static_cast<const AlienCellTO*>(dCells), nc,
               static_cast<const AlienParticleTO*>(dParts), np);
        coldBase += nc;
    }
    freeAsyncStage();
    if (hasWorldParams_) launch(kWorldsBegin, divUp(n, kBlock), kBlock, s);
    sync();
}

// ------------------------------------------------------- live arenas -----
namespace {
constexpr int kMaxLiveWorlds = 65534;  // world indices travel in 16 bits of the staged records
}

static void validateCapacity(const AlienArenaCapacity& c)
{
    if (c.maxWorlds < 1 || c.maxWorlds > kMaxLiveWorlds)
        throw Error(ALIEN_B200_ERR_INVALID_ARGUMENT, "maxWorlds must lie in [1, 65534]");
    if (c.cellSlots == 0 || c.particleSlots == 0 || c.tiles == 0 || c.particleMapSlots == 0)
        throw Error(ALIEN_B200_ERR_INVALID_ARGUMENT, "capacities must be positive");
    if (c.cellSlots >= (1ull << 31) || c.particleSlots >= (1ull << 31) || c.tiles >= (1ull << 32) - 2 ||
        c.particleMapSlots >= (1ull << 40))
        throw Error(ALIEN_B200_ERR_CAPACITY, "arena capacity exceeds 2^31 slots");
}

int Arena::residentWorlds() const
{
    int n = 0;
    for (int w = 0; w < numWorlds(); ++w) n += resident(w) ? 1 : 0;
    return n;
}

uint64_t Arena::reserveBytes(const AlienArenaCapacity& c)
{
    validateCapacity(c);
    Arena probe(nullptr);
    probe.mem_.setCountOnly(true);
    const int n = c.maxWorlds + 1;
    const long long cellBlocks = divUp(static_cast<long long>(c.cellSlots), kBlock);
    const long long partBlocks = divUp(static_cast<long long>(c.particleSlots), kBlock);
    const size_t C = static_cast<size_t>(cellBlocks) * kBlock, P = static_cast<size_t>(partBlocks) * kBlock;
    const int regionCap = static_cast<int>(std::min<long long>(static_cast<long long>(c.tiles) / 16 + 4ll * n + 16, 1ll << 30));
    probe.mem_.alloc<WorldInfo>(n);
    probe.mem_.alloc<WorldCounters>(n);
    probe.mem_.alloc<AlienPhysicsParams>(n);
    probe.mem_.alloc<int>(regionCap);
    probe.mem_.alloc<int>(cellBlocks);
    probe.mem_.alloc<int>(partBlocks);
    probe.mem_.alloc<uint32_t>(1);
    probe.allocCellAndParticleArrays(C, P, static_cast<long long>(c.tiles), static_cast<long long>(c.particleMapSlots),
                                     static_cast<int>(cellBlocks), static_cast<int>(partBlocks), true);
    probe.mem_.alloc<StatsAcc>(n);
    probe.mem_.alloc<TimelineAcc>(1);
    probe.mem_.alloc<unsigned long long>(static_cast<size_t>(n) * ALIEN_B200_MAX_COLORS);
    probe.mem_.alloc<AlienCellTO>(C);
    probe.mem_.alloc<uchar4>(C);
    probe.mem_.alloc<uint8_t>(std::max<uint64_t>(c.auxBytes, 1));
    probe.mem_.alloc<int>(C);
    probe.mem_.alloc<int>(P);
    probe.mem_.alloc<uint32_t>(static_cast<size_t>(std::max(cellBlocks, partBlocks)) + 2);
    return probe.mem_.bytes();
}

void Arena::reserve(const AlienArenaCapacity& c)
{
    validateCapacity(c);
    setRegionKernelAttributes();
    releaseGraph();
    AB_CK(cudaStreamSynchronize(stream_));
    mem_.freeAll();
    worlds_.clear();
    live_ = true;
    capacity_ = c;
    tuned_ = false;
    motionTuned_[0] = motionTuned_[1] = false;
    std::memset(tunedMs_, 0, sizeof(tunedMs_));
    for (int m = 0; m < 2; ++m) regionChoice_[m] = regionChoiceFixed_[m] ? regionChoiceFixed_[m] - 1 : 0;
    if (!checkStream_) {
        // admissions are staged and checked at the highest stream priority,
        // so that their small kernels get SMs between the blocks of the steps
        int least = 0, greatest = 0;
        AB_CK(cudaDeviceGetStreamPriorityRange(&least, &greatest));
        AB_CK(cudaStreamCreateWithPriority(&checkStream_, cudaStreamNonBlocking, greatest));
    }

    const int n = c.maxWorlds + 1;
    vacant_ = c.maxWorlds;
    const long long cellBlocks = divUp(static_cast<long long>(c.cellSlots), kBlock);
    const long long partBlocks = divUp(static_cast<long long>(c.particleSlots), kBlock);
    const size_t C = static_cast<size_t>(cellBlocks) * kBlock, P = static_cast<size_t>(partBlocks) * kBlock;
    const long long tiles = static_cast<long long>(c.tiles), pmapSlots = static_cast<long long>(c.particleMapSlots);
    regionCap_ = static_cast<int>(std::min<long long>(tiles / 16 + 4ll * n + 16, 1ll << 30));

    DevState& s = s_;
    s = DevState{};
    s.numWorlds = n;
    s.worlds = mem_.alloc<WorldInfo>(n);
    s.counters = mem_.alloc<WorldCounters>(n);
    s.params = mem_.alloc<AlienPhysicsParams>(n);
    s.regionWorld = mem_.alloc<int>(regionCap_);
    s.cellBlockWorld = mem_.alloc<int>(cellBlocks);
    s.partBlockWorld = mem_.alloc<int>(partBlocks);
    s.errorFlags = mem_.alloc<uint32_t>(1);
    allocCellAndParticleArrays(C, P, tiles, pmapSlots, static_cast<int>(cellBlocks), static_cast<int>(partBlocks), true);
    stats_ = mem_.alloc<StatsAcc>(n);
    timeline_ = mem_.alloc<TimelineAcc>(1);
    s.neuronActivity = mem_.alloc<unsigned long long>(static_cast<size_t>(n) * ALIEN_B200_MAX_COLORS);
    cold_ = mem_.alloc<AlienCellTO>(C);  // a world's transfer objects at its cell slots
    s.cold = cold_;
    s.fnInfo = mem_.alloc<uchar4>(C);
    s.aux = mem_.alloc<uint8_t>(std::max<uint64_t>(c.auxBytes, 1));
    rankCells_ = mem_.alloc<int>(C);
    rankParts_ = mem_.alloc<int>(P);
    blockCount_ = mem_.alloc<uint32_t>(static_cast<size_t>(std::max(cellBlocks, partBlocks)) + 2);

    // every slot vacant: world tables zero (inactive, no cells), default
    // parameters, every block and region on the vacant slot
    worlds_.assign(n, HostWorld{});
    std::vector<AlienPhysicsParams> params(n);
    for (int w = 0; w < n; ++w) {
        worlds_[w].vacant = true;
        std::memset(&worlds_[w].info, 0, sizeof(WorldInfo));
        alien_b200_default_parameters(&params[w]);
        worlds_[w].params = params[w];
        worlds_[w].info.paramIndex = w;
    }
    std::vector<WorldInfo> infos(n);
    for (int w = 0; w < n; ++w) infos[w] = worlds_[w].info;
    AB_CK(cudaMemcpyAsync(const_cast<WorldInfo*>(s.worlds), infos.data(), sizeof(WorldInfo) * n, cudaMemcpyHostToDevice, stream_));
    AB_CK(cudaMemcpyAsync(s.params, params.data(), sizeof(AlienPhysicsParams) * n, cudaMemcpyHostToDevice, stream_));
    AB_CK(cudaMemsetAsync(s.counters, 0, sizeof(WorldCounters) * n, stream_));
    const std::vector<int> vacantCells(cellBlocks, vacant_), vacantParts(partBlocks, vacant_), vacantRegions(regionCap_, vacant_);
    AB_CK(cudaMemcpyAsync(const_cast<int*>(s.cellBlockWorld), vacantCells.data(), sizeof(int) * cellBlocks, cudaMemcpyHostToDevice,
                          stream_));
    AB_CK(cudaMemcpyAsync(const_cast<int*>(s.partBlockWorld), vacantParts.data(), sizeof(int) * partBlocks, cudaMemcpyHostToDevice,
                          stream_));
    AB_CK(cudaMemcpyAsync(const_cast<int*>(s.regionWorld), vacantRegions.data(), sizeof(int) * regionCap_, cudaMemcpyHostToDevice,
                          stream_));
    AB_CK(cudaMemsetAsync(s.errorFlags, 0, sizeof(uint32_t), stream_));
    AB_CK(cudaMemsetAsync(s.alive, 0, C, stream_));
    AB_CK(cudaMemsetAsync(s.palive, 0, P, stream_));
    AB_CK(cudaMemsetAsync(s.pflag, 0, P * sizeof(uint32_t), stream_));
    AB_CK(cudaMemsetAsync(s.pmap, 0xff, static_cast<size_t>(pmapSlots) * sizeof(int), stream_));
    AB_CK(cudaMemsetAsync(s.flags, 0, C * sizeof(uint32_t), stream_));
    AB_CK(cudaMemsetAsync(s.angleAcc, 0, C * 4 * sizeof(long long), stream_));
    AB_CK(cudaMemsetAsync(s.dpos, 0, C * sizeof(float2), stream_));
    AB_CK(cudaMemsetAsync(s.push, 0, C * sizeof(float2), stream_));
    AB_CK(cudaMemsetAsync(s.neuronActivity, 0, sizeof(unsigned long long) * n * ALIEN_B200_MAX_COLORS, stream_));
    AB_CK(cudaMemsetAsync(s.energyAcc, 0, C * sizeof(long long), stream_));
    AB_CK(cudaMemsetAsync(s.newPartner, 0xff, C * sizeof(int), stream_));
    AB_CK(cudaMemsetAsync(s.best, 0xff, C * sizeof(int), stream_));
    regionsReserved_ = 0;
    cellPool_.init(cellBlocks);
    partPool_.init(partBlocks);
    tilePool_.init(tiles);
    pmapPool_.init(pmapSlots);
    auxPool_.init(static_cast<long long>(c.auxBytes));
    maxWorldCells_ = maxWorldParts_ = 0;
    updateLiveLayout();
    sync();
}

// launch extents (the used prefix of each range), region tables of the
// resident worlds and the step's optional phases, after an admission or an
// eviction; the next step captures a new graph
void Arena::updateLiveLayout()
{
    DevState& s = s_;
    s.numCellBlocks = static_cast<int>(cellPool_.highWater());
    s.numPartBlocks = static_cast<int>(partPool_.highWater());
    s.numTiles = tilePool_.highWater();
    s.pairOverflowCount = s.tileCount + s.numTiles;  // cleared with the used tile counts every step
    s.cellSlots = static_cast<long long>(s.numCellBlocks) * kBlock;
    s.partSlots = static_cast<long long>(s.numPartBlocks) * kBlock;
    int device = 0, sms = 0;
    AB_CK(cudaGetDevice(&device));
    AB_CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    partGrid_ = std::max(1, std::min(s.numPartBlocks, 16 * std::max(sms, 1)));
    statsGrid_ = 4 * std::max(sms, 1);
    overflowGrid_ = std::max(1, std::min(s.numCellBlocks, 2 * std::max(sms, 1)));
    hasFluid_ = hasCollision_ = hasWorldParams_ = hasRigidity_ = hasNeurons_ = signalsLive_ = false;
    for (const HostWorld& hw : worlds_) {
        if (hw.vacant) continue;
        hasWorldParams_ |= needsWorldParams(hw.params);
        hasRigidity_ |= rigidityEnabled(hw.params);
        hasNeurons_ |= hw.neurons > 0;
        signalsLive_ |= hw.neurons > 0 || hw.signals > 0;
        if (hw.info.motionType == ALIEN_B200_MOTION_FLUID)
            hasFluid_ = true;
        else
            hasCollision_ = true;
        maxWorldCells_ = std::max(maxWorldCells_, hw.info.cellCap);
        maxWorldParts_ = std::max(maxWorldParts_, hw.info.partCap);
    }
    // a motion type the autotuner has not seen yet is tuned at the next step
    if ((hasFluid_ && !motionTuned_[ALIEN_B200_MOTION_FLUID]) || (hasCollision_ && !motionTuned_[ALIEN_B200_MOTION_COLLISION]))
        tuned_ = false;
    applyRegionShapes();
}

int Arena::admit(const WorldSetup& ws, uint64_t steps, int slot)
{
    if (!live_) throw Error(ALIEN_B200_ERR_INVALID_ARGUMENT, "not a live arena");
    if (ws.W <= 0 || ws.H <= 0) throw Error(ALIEN_B200_ERR_INVALID_ARGUMENT, "world size must be positive");
    validateParams(ws.params, ws.W, ws.H);
    if (ws.numCells > (1ull << 30) || ws.numParticles > (1ull << 30))
        throw Error(ALIEN_B200_ERR_CAPACITY, "more than 2^30 objects in one world");

    // the world's extents, as build() lays out a world
    HostWorld hw;
    hw.params = ws.params;
    hw.setTimestep = ws.timestep;
    WorldInfo& wi = hw.info;
    std::memset(&wi, 0, sizeof(wi));
    wi.W = ws.W;
    wi.H = ws.H;
    wi.radiusInt = scanRadius(ws.params);
    wi.T = wi.radiusInt;
    wi.nTX = divUp(ws.W, wi.T);
    wi.nTY = divUp(ws.H, wi.T);
    wi.motionType = ws.params.motionType;
    const long long nc = static_cast<long long>(ws.numCells), np = static_cast<long long>(ws.numParticles);
    wi.cellCap = roundUp(std::max<long long>(nc, 1), kBlock);
    wi.partCap = roundUp(np + nc + std::max<long long>(4096, (np + nc) / 2) + static_cast<long long>(ws.extraParticles), kBlock);
    wi.numCellBlocks = static_cast<int>(wi.cellCap / kBlock);
    wi.numPartBlocks = static_cast<int>(wi.partCap / kBlock);
    const long long tiles = static_cast<long long>(wi.nTX) * wi.nTY, pmapSlots = static_cast<long long>(ws.W) * ws.H;
    const int worldRegions = maxRegions(wi);
    const long long regionsAfter = regionsReserved_ + worldRegions;

    // a free world slot and free ranges, or nothing changes
    int w = slot;
    if (w < 0) {
        for (int i = 0; i < vacant_; ++i)
            if (worlds_[i].vacant) {
                w = i;
                break;
            }
    }
    if (w < 0 || w >= vacant_ || !worlds_[w].vacant) throw Error(ALIEN_B200_ERR_CAPACITY, "no free world slot in the arena");
    if (regionsAfter > regionCap_) throw Error(ALIEN_B200_ERR_CAPACITY, "the arena's region table is full");
    const long long cb = cellPool_.alloc(wi.numCellBlocks);
    const long long pb = cb < 0 ? -1 : partPool_.alloc(wi.numPartBlocks);
    const long long tb = pb < 0 ? -1 : tilePool_.alloc(tiles);
    const long long mb = tb < 0 ? -1 : pmapPool_.alloc(pmapSlots);
    const long long ab = mb < 0 ? -1 : auxPool_.alloc(static_cast<long long>(ws.numAux));
    auto releaseRanges = [&] {
        if (cb >= 0) cellPool_.release(cb, wi.numCellBlocks);
        if (pb >= 0) partPool_.release(pb, wi.numPartBlocks);
        if (tb >= 0) tilePool_.release(tb, tiles);
        if (mb >= 0) pmapPool_.release(mb, pmapSlots);
        if (ab >= 0) auxPool_.release(ab, static_cast<long long>(ws.numAux));
    };
    if (ab < 0) {
        releaseRanges();
        throw Error(ALIEN_B200_ERR_CAPACITY, cb < 0   ? "no free cell range in the arena"
                                             : pb < 0 ? "no free particle range in the arena"
                                             : tb < 0 ? "no free tile range in the arena"
                                             : mb < 0 ? "no free particle-map range in the arena"
                                                      : "no free auxiliary-data range in the arena");
    }

    // the transfer objects, staged and checked on the check stream while
    // the enqueued steps run
    AlienCellTO* dCells = nullptr;
    AlienParticleTO* dParts = nullptr;
    uint8_t* dAux = nullptr;
    IngestCheck* dCheck = nullptr;
    IngestCheck check{};
    try {
        AB_CK(cudaMallocAsync(reinterpret_cast<void**>(&dCells), sizeof(AlienCellTO) * std::max<long long>(nc, 1), checkStream_));
        AB_CK(cudaMallocAsync(reinterpret_cast<void**>(&dParts), sizeof(AlienParticleTO) * std::max<long long>(np, 1), checkStream_));
        AB_CK(cudaMallocAsync(reinterpret_cast<void**>(&dCheck), sizeof(IngestCheck), checkStream_));
        AB_CK(cudaMemsetAsync(dCheck, 0, sizeof(IngestCheck), checkStream_));
        if (nc) {
            AB_CK(cudaMemcpyAsync(dCells, ws.cells, sizeof(AlienCellTO) * nc, cudaMemcpyHostToDevice, checkStream_));
            kCheckCells<<<divUp(nc, kBlock), kBlock, 0, checkStream_>>>(dCells, nc, static_cast<unsigned long long>(ws.numAux), dCheck);
            AB_CK(cudaGetLastError());
        }
        if (np) AB_CK(cudaMemcpyAsync(dParts, ws.particles, sizeof(AlienParticleTO) * np, cudaMemcpyHostToDevice, checkStream_));
        // the auxiliary bytes too: a large copy from pageable memory on the
        // arena's stream would wait there behind the enqueued steps
        if (ws.numAux) {
            AB_CK(cudaMallocAsync(reinterpret_cast<void**>(&dAux), ws.numAux, checkStream_));
            AB_CK(cudaMemcpyAsync(dAux, ws.aux, ws.numAux, cudaMemcpyHostToDevice, checkStream_));
        }
        AB_CK(cudaMemcpyAsync(&check, dCheck, sizeof(IngestCheck), cudaMemcpyDeviceToHost, checkStream_));
        AB_CK(cudaStreamSynchronize(checkStream_));
        if (check.badBondCount || check.badBondIndex || check.otherFunction || check.neuronOutOfAux) {
            validateCells({ws});  // the host scan names the first offending cell
            throw Error(ALIEN_B200_ERR_INVALID_ARGUMENT, "invalid cell transfer objects");
        }
    } catch (...) {
        if (dCells) cudaFreeAsync(dCells, checkStream_);
        if (dParts) cudaFreeAsync(dParts, checkStream_);
        if (dAux) cudaFreeAsync(dAux, checkStream_);
        if (dCheck) cudaFreeAsync(dCheck, checkStream_);
        cudaStreamSynchronize(checkStream_);
        releaseRanges();
        throw;
    }
    AB_CK(cudaFreeAsync(dCheck, checkStream_));
    cudaEvent_t staged;
    AB_CK(cudaEventCreateWithFlags(&staged, cudaEventDisableTiming));
    AB_CK(cudaEventRecord(staged, checkStream_));
    AB_CK(cudaStreamWaitEvent(stream_, staged, 0));
    cudaEventDestroy(staged);

    wi.paramIndex = w;
    wi.tileBase = tb;
    wi.cellBase = cb * kBlock;
    wi.firstCellBlock = static_cast<int>(cb);
    wi.partBase = pb * kBlock;
    wi.firstPartBlock = static_cast<int>(pb);
    wi.pmapBase = mb;
    wi.auxBase = ab;
    hw.auxSize = ws.numAux;
    hw.vacant = false;
    hw.neurons = check.neurons;
    hw.signals = check.nonzeroSignal;
    worlds_[w] = hw;
    regionsReserved_ += worldRegions;
    maxWorldCells_ = std::max(maxWorldCells_, wi.cellCap);  // egress buffers
    maxWorldParts_ = std::max(maxWorldParts_, wi.partCap);

    // the world's tables and ranges, in stream order behind the enqueued steps
    const DevState& s = s_;
    WorldCounters wc;
    std::memset(&wc, 0, sizeof(wc));
    wc.timestep = ws.timestep;
    wc.nextId = 1;
    wc.numCells = static_cast<unsigned int>(nc);
    wc.numParticles = static_cast<unsigned int>(np);
    wc.stepsRemaining = steps == 0 ? ~0ull : steps;
    wc.active = 1;
    wc.signalsFresh = 1;
    wc.externalEnergy = ws.params.externalEnergy;
    wc.lastStepped = ~0ull;
    AB_CK(cudaMemcpyAsync(s.counters + w, &wc, sizeof(wc), cudaMemcpyHostToDevice, stream_));
    AB_CK(cudaMemcpyAsync(s.params + w, &hw.params, sizeof(AlienPhysicsParams), cudaMemcpyHostToDevice, stream_));
    AB_CK(cudaMemcpyAsync(const_cast<WorldInfo*>(s.worlds) + w, &wi, sizeof(WorldInfo), cudaMemcpyHostToDevice, stream_));
    const std::vector<int> cbw(wi.numCellBlocks, w), pbw(wi.numPartBlocks, w);
    AB_CK(cudaMemcpyAsync(const_cast<int*>(s.cellBlockWorld) + cb, cbw.data(), sizeof(int) * cbw.size(), cudaMemcpyHostToDevice, stream_));
    AB_CK(cudaMemcpyAsync(const_cast<int*>(s.partBlockWorld) + pb, pbw.data(), sizeof(int) * pbw.size(), cudaMemcpyHostToDevice, stream_));
    const size_t c0 = static_cast<size_t>(wi.cellBase), cn = static_cast<size_t>(wi.cellCap);
    const size_t p0 = static_cast<size_t>(wi.partBase), pn = static_cast<size_t>(wi.partCap);
    AB_CK(cudaMemsetAsync(s.alive + c0, 0, cn, stream_));
    AB_CK(cudaMemsetAsync(s.flags + c0, 0, cn * sizeof(uint32_t), stream_));
    AB_CK(cudaMemsetAsync(s.angleAcc + 4 * c0, 0, cn * 4 * sizeof(long long), stream_));
    AB_CK(cudaMemsetAsync(s.dpos + c0, 0, cn * sizeof(float2), stream_));
    AB_CK(cudaMemsetAsync(s.push + c0, 0, cn * sizeof(float2), stream_));
    AB_CK(cudaMemsetAsync(s.energyAcc + c0, 0, cn * sizeof(long long), stream_));
    AB_CK(cudaMemsetAsync(s.newPartner + c0, 0xff, cn * sizeof(int), stream_));
    AB_CK(cudaMemsetAsync(s.best + c0, 0xff, cn * sizeof(int), stream_));
    AB_CK(cudaMemsetAsync(s.palive + p0, 0, pn, stream_));
    AB_CK(cudaMemsetAsync(s.pflag + p0, 0, pn * sizeof(uint32_t), stream_));
    AB_CK(cudaMemsetAsync(s.pmap + mb, 0xff, static_cast<size_t>(pmapSlots) * sizeof(int), stream_));
    AB_CK(cudaMemsetAsync(s.neuronActivity + static_cast<size_t>(w) * ALIEN_B200_MAX_COLORS, 0,
                          sizeof(unsigned long long) * ALIEN_B200_MAX_COLORS, stream_));
    if (ws.numAux) {
        AB_CK(cudaMemcpyAsync(const_cast<uint8_t*>(s_.aux) + ab, dAux, ws.numAux, cudaMemcpyDeviceToDevice, stream_));
        AB_CK(cudaFreeAsync(dAux, stream_));
    }
    if (nc) AB_CK(cudaMemcpyAsync(cold_ + c0, dCells, sizeof(AlienCellTO) * nc, cudaMemcpyDeviceToDevice, stream_));
    launch(kIngestCells, divUp(nc, kBlock), kBlock, s, w, static_cast<const AlienCellTO*>(dCells), nc, cold_,
           static_cast<long long>(c0));
    launch(kIngestParticles, divUp(np, kBlock), kBlock, s, w, static_cast<const AlienParticleTO*>(dParts), np);
    launch(kMaxId, divUp(std::max(nc, np), kBlock), kBlock, s, w, static_cast<const AlienCellTO*>(dCells), nc,
           static_cast<const AlienParticleTO*>(dParts), np);
    AB_CK(cudaFreeAsync(dCells, stream_));
    AB_CK(cudaFreeAsync(dParts, stream_));
    // the launch extents and region tables follow at the next step, once for
    // all admissions and evictions since the last one
    layoutDirty_ = true;
    if (needsWorldParams(hw.params)) launch(kWorldsBegin, divUp(numWorlds(), kBlock), kBlock, s_);
    return w;
}

void Arena::evict(int w)
{
    if (!live_) throw Error(ALIEN_B200_ERR_INVALID_ARGUMENT, "not a live arena");
    if (!resident(w)) throw Error(ALIEN_B200_ERR_INVALID_ARGUMENT, "world " + std::to_string(w) + " is not resident");
    HostWorld& hw = worlds_[w];
    const WorldInfo wi = hw.info;
    const DevState& s = s_;
    // the world stops being stepped and its blocks fall to the vacant slot
    WorldCounters wc;
    std::memset(&wc, 0, sizeof(wc));
    AB_CK(cudaMemcpyAsync(s.counters + w, &wc, sizeof(wc), cudaMemcpyHostToDevice, stream_));
    const std::vector<int> cbw(wi.numCellBlocks, vacant_), pbw(wi.numPartBlocks, vacant_);
    AB_CK(cudaMemcpyAsync(const_cast<int*>(s.cellBlockWorld) + wi.firstCellBlock, cbw.data(), sizeof(int) * cbw.size(),
                          cudaMemcpyHostToDevice, stream_));
    AB_CK(cudaMemcpyAsync(const_cast<int*>(s.partBlockWorld) + wi.firstPartBlock, pbw.data(), sizeof(int) * pbw.size(),
                          cudaMemcpyHostToDevice, stream_));
    AB_CK(cudaMemsetAsync(s.alive + wi.cellBase, 0, static_cast<size_t>(wi.cellCap), stream_));
    AB_CK(cudaMemsetAsync(s.palive + wi.partBase, 0, static_cast<size_t>(wi.partCap), stream_));
    regionsReserved_ -= maxRegions(wi);
    cellPool_.release(wi.firstCellBlock, wi.numCellBlocks);
    partPool_.release(wi.firstPartBlock, wi.numPartBlocks);
    tilePool_.release(wi.tileBase, static_cast<long long>(wi.nTX) * wi.nTY);
    pmapPool_.release(wi.pmapBase, static_cast<long long>(wi.W) * wi.H);
    auxPool_.release(wi.auxBase, static_cast<long long>(hw.auxSize));
    HostWorld empty;
    empty.vacant = true;
    std::memset(&empty.info, 0, sizeof(WorldInfo));
    empty.info.paramIndex = w;
    empty.params = hw.params;
    hw = empty;
    AB_CK(cudaMemcpyAsync(const_cast<WorldInfo*>(s.worlds) + w, &hw.info, sizeof(WorldInfo), cudaMemcpyHostToDevice, stream_));
    layoutDirty_ = true;
}

bool Arena::moveParticles(int w, long long newCap, bool stepScratch)
{
    WorldInfo& wi = worlds_[w].info;
    const int newBlocks = static_cast<int>(divUp(newCap, kBlock));
    const long long pb = partPool_.alloc(newBlocks);
    if (pb < 0) return false;
    WorldCounters c;
    AB_CK(cudaMemcpyAsync(&c, s_.counters + w, sizeof(c), cudaMemcpyDeviceToHost, stream_));
    AB_CK(cudaStreamSynchronize(stream_));
    const size_t n = c.numParticles;  // used slots
    const size_t from = static_cast<size_t>(wi.partBase), to = static_cast<size_t>(pb) * kBlock;
    const size_t cap = static_cast<size_t>(newBlocks) * kBlock;
    const DevState& s = s_;
    AB_CK(cudaMemsetAsync(s.palive + to, 0, cap, stream_));
    AB_CK(cudaMemsetAsync(s.pflag + to, 0, cap * sizeof(uint32_t), stream_));
    if (n) {
        // the persistent particle state; the rest is per-step scratch
        AB_CK(cudaMemcpyAsync(s.pid + to, s.pid + from, n * sizeof(unsigned long long), cudaMemcpyDeviceToDevice, stream_));
        AB_CK(cudaMemcpyAsync(s.plast + to, s.plast + from, n * sizeof(unsigned long long), cudaMemcpyDeviceToDevice, stream_));
        AB_CK(cudaMemcpyAsync(s.ppos + to, s.ppos + from, n * sizeof(float2), cudaMemcpyDeviceToDevice, stream_));
        AB_CK(cudaMemcpyAsync(s.pvel + to, s.pvel + from, n * sizeof(float2), cudaMemcpyDeviceToDevice, stream_));
        AB_CK(cudaMemcpyAsync(s.penergy + to, s.penergy + from, n * sizeof(float), cudaMemcpyDeviceToDevice, stream_));
        AB_CK(cudaMemcpyAsync(s.pcolor + to, s.pcolor + from, n, cudaMemcpyDeviceToDevice, stream_));
        AB_CK(cudaMemcpyAsync(s.pselected + to, s.pselected + from, n, cudaMemcpyDeviceToDevice, stream_));
        AB_CK(cudaMemcpyAsync(s.palive + to, s.palive + from, n, cudaMemcpyDeviceToDevice, stream_));
        if (stepScratch) {
            // what the halted step's split emission reads (kEventEmit)
            AB_CK(cudaMemcpyAsync(s.pflag + to, s.pflag + from, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, stream_));
            AB_CK(cudaMemcpyAsync(s.splitPos + to, s.splitPos + from, n * sizeof(float2), cudaMemcpyDeviceToDevice, stream_));
            AB_CK(cudaMemcpyAsync(s.splitVel + to, s.splitVel + from, n * sizeof(float2), cudaMemcpyDeviceToDevice, stream_));
            AB_CK(cudaMemcpyAsync(s.splitEnergy + to, s.splitEnergy + from, n * sizeof(float), cudaMemcpyDeviceToDevice, stream_));
            AB_CK(cudaMemcpyAsync(s.blockSplit + pb, s.blockSplit + wi.firstPartBlock, divUp(n, kBlock) * sizeof(uint32_t),
                                  cudaMemcpyDeviceToDevice, stream_));
        }
    }
    const std::vector<int> mine(newBlocks, w), vacant(wi.numPartBlocks, vacant_);
    AB_CK(cudaMemcpyAsync(const_cast<int*>(s.partBlockWorld) + pb, mine.data(), sizeof(int) * mine.size(), cudaMemcpyHostToDevice,
                          stream_));
    AB_CK(cudaMemcpyAsync(const_cast<int*>(s.partBlockWorld) + wi.firstPartBlock, vacant.data(), sizeof(int) * vacant.size(),
                          cudaMemcpyHostToDevice, stream_));
    AB_CK(cudaMemsetAsync(s.palive + from, 0, static_cast<size_t>(wi.partCap), stream_));
    partPool_.release(wi.firstPartBlock, wi.numPartBlocks);
    wi.partBase = static_cast<long long>(to);
    wi.firstPartBlock = static_cast<int>(pb);
    wi.numPartBlocks = newBlocks;
    wi.partCap = static_cast<long long>(cap);
    AB_CK(cudaMemcpyAsync(const_cast<WorldInfo*>(s.worlds) + w, &wi, sizeof(WorldInfo), cudaMemcpyHostToDevice, stream_));
    maxWorldParts_ = std::max(maxWorldParts_, wi.partCap);
    layoutDirty_ = true;
    AB_CK(cudaStreamSynchronize(stream_));
    return true;
}

void Arena::relocate(int w, uint64_t extraParticles, const AlienPhysicsParams* newParams)
{
    syncParamsFromDevice();  // zones, sources and the pool as the steps left them
    const std::vector<WorldCounters> c = readCounters();
    const HostWorld old = worlds_[w];
    Carried carried;
    exportWorld(w, carried);
    std::vector<uint8_t> aux(std::max<uint64_t>(old.auxSize, 1));
    if (old.auxSize)
        AB_CK(cudaMemcpyAsync(aux.data(), s_.aux + old.info.auxBase, old.auxSize, cudaMemcpyDeviceToHost, stream_));
    std::vector<unsigned long long> neurons(ALIEN_B200_MAX_COLORS);
    AB_CK(cudaMemcpyAsync(neurons.data(), s_.neuronActivity + static_cast<size_t>(w) * ALIEN_B200_MAX_COLORS,
                          sizeof(unsigned long long) * ALIEN_B200_MAX_COLORS, cudaMemcpyDeviceToHost, stream_));
    AB_CK(cudaStreamSynchronize(stream_));
    WorldSetup ws;
    ws.W = old.info.W;
    ws.H = old.info.H;
    ws.params = newParams ? *newParams : old.params;
    if (newParams) ws.params.externalEnergy = old.params.externalEnergy;
    ws.timestep = c[w].timestep;
    ws.cells = carried.cells.data();
    ws.numCells = carried.cells.size();
    ws.particles = carried.parts.data();
    ws.numParticles = carried.parts.size();
    ws.aux = aux.data();
    ws.numAux = old.auxSize;
    ws.extraParticles = extraParticles;
    evict(w);
    admit(ws, 0, w);
    // the absorbers continue; densities start again after a parameter change
    const long long nc = static_cast<long long>(ws.numCells), np = static_cast<long long>(ws.numParticles);
    launch(kRestoreCarried, static_cast<int>(divUp(std::max<long long>(std::max(nc, np), 1), kBlock)), kBlock, s_, w,
           newParams ? nullptr : static_cast<const float*>(carried.density), nc, static_cast<const unsigned long long*>(carried.last),
           np);
    AB_CK(cudaFreeAsync(carried.density, stream_));
    AB_CK(cudaFreeAsync(carried.last, stream_));
    // ids, budget and activity continue where they were
    WorldCounters now;
    AB_CK(cudaMemcpyAsync(&now, s_.counters + w, sizeof(now), cudaMemcpyDeviceToHost, stream_));
    AB_CK(cudaStreamSynchronize(stream_));
    now.nextId = std::max(now.nextId, c[w].nextId);
    now.stepsRemaining = c[w].stepsRemaining;
    now.active = c[w].active;
    AB_CK(cudaMemcpyAsync(s_.counters + w, &now, sizeof(now), cudaMemcpyHostToDevice, stream_));
    AB_CK(cudaMemcpyAsync(s_.neuronActivity + static_cast<size_t>(w) * ALIEN_B200_MAX_COLORS, neurons.data(),
                          sizeof(unsigned long long) * ALIEN_B200_MAX_COLORS, cudaMemcpyHostToDevice, stream_));
    sync();
}

// -------------------------------------------------------------- scan -----
// exclusive scan of in[0, n) into out[0, n], out[n] = total; in and out are
// device allocations (16-byte aligned, as kScanDown's vector accesses need)
void Arena::scan(const uint32_t* in, long long n, uint32_t* out)
{
    const int blocks = divUp(n, kScanTile);
    launch(kScanReduce, blocks, kBlock, in, n, s_.scanPartials);
    if (blocks <= kScanFusedBlocks) {
        launch(kScanDown<true>, blocks, kBlock, in, n, static_cast<const uint32_t*>(s_.scanPartials), out);
        return;
    }
    launch(kScanPartials<1024>, 1, 1024, s_.scanPartials, blocks);
    launch(kScanDown<false>, blocks, kBlock, in, n, static_cast<const uint32_t*>(s_.scanPartials), out);
}

// -------------------------------------------------------------- step -----
// the launch sequence of one timestep for every world of the arena
void Arena::enqueueStep()
{
    const DevState& s = s_;
    const int cells = s.numCellBlocks, both = s.numCellBlocks + partGrid_;
    const uint64_t before = launches_;
    AB_CK(cudaMemsetAsync(s.tileCount, 0, sizeof(uint32_t) * (static_cast<size_t>(s.numTiles) + 1), stream_));
    launch(kBin, both, kBlock, s);
    scan(s.tileCount, s.numTiles, s.tileStart);
    launch(kScatter, cells, kBlock, s);
    launch(kStage, cells, kBlock, s);
    if (hasFluid_) launchPairs<ALIEN_B200_MOTION_FLUID>();
    if (hasCollision_) launchPairs<ALIEN_B200_MOTION_COLLISION>();
    launch(kPairsOverflow, overflowGrid_, kBlock, s);
    launch(kApplyBond1, both, kBlock, s);
    launch(kVerletPos, both, kBlock, s);
    launch(kBond2, both, kBlock, s);
    launch(kVerletVel, both, kBlock, s);
    launch(kTransition, both, kBlock, s);
    if (hasRigidity_) {
        launch(kClusterInit, cells, kBlock, s);
        for (int r = 0; r < kClusterRounds; ++r) {
            launch(kClusterGather, cells, kBlock, s, r);
            launch(kClusterScatter, cells, kBlock, s, r);
        }
        launch(kClusterSum1, cells, kBlock, s);
        launch(kClusterSum2, cells, kBlock, s);
        launch(kClusterApply, cells, kBlock, s);
    }
    launch(kResolve, cells, kBlock, s);
    if (hasNeurons_) launch(kNeuron, cells, kBlock, s);
    if (signalsLive_) launch(kSignalReset, cells, kBlock, s);
    launch(kCommit, cells, kBlock, s);
    launch(kEventCount, both, kBlock, s);
    launch(kEventWorld, s.numWorlds, kEventWorldThreads, s);
    launch(kEventEmit, both, kBlock, s);
    if (hasWorldParams_) launch(kWorldsEnd, divUp(s.numWorlds, kBlock), kBlock, s);
    kernelsPerStep_ = static_cast<int>(launches_ - before);
}

void Arena::enqueueSteps(uint64_t n)
{
    if (n == 0) return;
    refreshLayout();
    if (live_ && residentWorlds() == 0) return;
    if (!tuned_) autotune();
    if (!graphExec_) {
        cudaGraph_t graph;
        AB_CK(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
        const uint64_t before = launches_;
        try {
            enqueueStep();
        } catch (...) {
            cudaStreamEndCapture(stream_, &graph);
            throw;
        }
        launches_ = before;  // captured, not launched
        AB_CK(cudaStreamEndCapture(stream_, &graph));
        cudaError_t e = cudaGraphInstantiate(&graphExec_, graph, 0);
        cudaGraphDestroy(graph);
        AB_CK(e);
    }
    stepsPending_ = true;
    for (uint64_t i = 0; i < n; ++i) {
        AB_CK(cudaGraphLaunch(graphExec_, stream_));
        launches_ += kernelsPerStep_;
    }
}

std::vector<double> Arena::timedSteps(uint64_t n)
{
    refreshLayout();
    if (!tuned_) autotune();
    std::vector<double> sums;
    std::vector<cudaEvent_t> events;
    for (uint64_t i = 0; i < n; ++i) {
        events.clear();
        cudaEvent_t start;
        AB_CK(cudaEventCreate(&start));
        AB_CK(cudaEventRecord(start, stream_));
        events.push_back(start);
        timingEvents_ = &events;
        timingNames_.clear();
        stepsPending_ = true;
        try {
            enqueueStep();
        } catch (...) {
            timingEvents_ = nullptr;
            throw;
        }
        timingEvents_ = nullptr;
        lastTimedNames.assign(timingNames_.begin(), timingNames_.end());
        AB_CK(cudaStreamSynchronize(stream_));
        if (sums.size() < events.size() - 1) sums.resize(events.size() - 1, 0.0);
        for (size_t k = 1; k < events.size(); ++k) {
            float ms = 0.0f;
            AB_CK(cudaEventElapsedTime(&ms, events[k - 1], events[k]));
            sums[k - 1] += ms;
        }
        for (cudaEvent_t e : events) cudaEventDestroy(e);
    }
    sync();
    return sums;
}

double Arena::timeSteps(uint64_t n)
{
    enqueueSteps(0);
    if (!graphExec_) {  // build the graph outside the timed region
        enqueueSteps(1);
        sync();
    }
    cudaEvent_t a, b;
    AB_CK(cudaEventCreate(&a));
    AB_CK(cudaEventCreate(&b));
    AB_CK(cudaStreamSynchronize(stream_));
    AB_CK(cudaEventRecord(a, stream_));
    enqueueSteps(n);
    AB_CK(cudaEventRecord(b, stream_));
    AB_CK(cudaEventSynchronize(b));
    float ms = 0.0f;
    AB_CK(cudaEventElapsedTime(&ms, a, b));
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    sync();
    return ms;
}

void Arena::sync()
{
    settle();
    if (droppedPending_) {
        droppedPending_ = false;
        throw Error(ALIEN_B200_ERR_CAPACITY, "particle capacity exceeded: energy particles were dropped");
    }
}

void Arena::settle()
{
    // only the steps set the error word: without steps since the last read
    // there is nothing to wait for or to complete
    if (!s_.errorFlags || !stepsPending_) return;
    stepsPending_ = false;
    for (;;) {
        // the error word is read in stream order: one wait covers the work and the read
        uint32_t& landed = readback().flags;
        AB_CK(cudaMemcpyAsync(&landed, s_.errorFlags, sizeof(landed), cudaMemcpyDeviceToHost, stream_));
        AB_CK(cudaStreamSynchronize(stream_));
        const uint32_t flags = landed;
        if (!flags) return;
        AB_CK(cudaMemsetAsync(s_.errorFlags, 0, sizeof(uint32_t), stream_));
        if (flags & kErrDropped) droppedPending_ = true;
        if (!(flags & kErrHalted)) {
            AB_CK(cudaStreamSynchronize(stream_));
            return;
        }
        if (resumeHalted()) droppedPending_ = true;
    }
}

bool Arena::resumeHalted()
{
    std::vector<WorldCounters> c = readCounters();
    std::vector<int> halted;
    for (int w = 0; w < numWorlds(); ++w)
        if (resident(w) && c[w].halted) halted.push_back(w);
    if (halted.empty()) return false;
    // room for the step's new particles with half the range free, at least
    // three times the old range (the growth rule of ensureParticleCapacity)
    std::vector<long long> newCap(numWorlds(), 0);
    std::vector<int> cannotGrow;
    for (int w : halted) {
        const long long need = static_cast<long long>(c[w].numParticles) + c[w].evRad + c[w].evDel + c[w].evSplit;
        const long long want = roundUp(std::max(3 * worlds_[w].info.partCap, 2 * need), kBlock);
        if (!live_)
            newCap[w] = want;
        else if (!moveParticles(w, want, true))
            cannotGrow.push_back(w);  // no free range: the resume drops the excess
    }
    if (!live_) {
        try {
            growParticleArrays(newCap);
        } catch (const Error& e) {
            // no memory, or more than 2^31 particle slots: the arrays are
            // unchanged and the resume drops the excess
            if (e.code != ALIEN_B200_ERR_OUT_OF_MEMORY && e.code != ALIEN_B200_ERR_CAPACITY) throw;
            cannotGrow = halted;
        }
    }
    refreshLayout();
    DevState r = s_;
    r.resume = 1;
    launch(kEventWorld, r.numWorlds, kEventWorldThreads, r);
    launch(kEventEmit, r.numCellBlocks + partGrid_, kBlock, r);
    if (hasWorldParams_) launch(kWorldsEnd, divUp(r.numWorlds, kBlock), kBlock, r);
    std::vector<uint64_t> missed(numWorlds(), 0);
    uint64_t most = 0;
    for (int w : halted) {
        missed[w] = c[w].missedSteps;
        most = std::max(most, missed[w]);
    }
    // the missed steps: each world that missed some gets that many as its
    // budget, every other world is parked; afterwards budgets and activity
    // are what an uninterrupted run would have left
    const std::vector<WorldCounters> saved = readCounters();
    std::vector<WorldCounters> now = saved;
    for (int w : cannotGrow) now[w].dropExcess = 1;
    if (most == 0) {
        AB_CK(cudaMemcpyAsync(s_.counters, now.data(), sizeof(WorldCounters) * now.size(), cudaMemcpyHostToDevice, stream_));
        AB_CK(cudaStreamSynchronize(stream_));
        return false;
    }
    for (int w = 0; w < numWorlds(); ++w) {
        now[w].active = missed[w] ? 1u : 0u;
        if (missed[w]) now[w].stepsRemaining = missed[w];
    }
    AB_CK(cudaMemcpyAsync(s_.counters, now.data(), sizeof(WorldCounters) * now.size(), cudaMemcpyHostToDevice, stream_));
    enqueueSteps(most);
    const bool before = droppedPending_;
    droppedPending_ = false;
    settle();  // halts within the missed steps complete here
    const bool dropped = droppedPending_;
    droppedPending_ = before;
    now = readCounters();
    for (int w = 0; w < numWorlds(); ++w) {
        if (missed[w]) {
            const uint64_t b = saved[w].stepsRemaining;
            now[w].stepsRemaining = b == ~0ull ? ~0ull : b - missed[w];
            now[w].active = now[w].stepsRemaining != 0 ? 1u : 0u;
        } else {
            now[w].active = saved[w].active;
        }
    }
    AB_CK(cudaMemcpyAsync(s_.counters, now.data(), sizeof(WorldCounters) * now.size(), cudaMemcpyHostToDevice, stream_));
    AB_CK(cudaStreamSynchronize(stream_));
    return dropped;
}

void Arena::growParticleArrays(const std::vector<long long>& newCap)
{
    const std::vector<WorldCounters> c = readCounters();
    const int n = numWorlds();
    std::vector<WorldInfo> infos(n);
    long long partSlots = 0;
    int partBlocks = 0;
    for (int w = 0; w < n; ++w) {
        WorldInfo wi = worlds_[w].info;
        if (newCap[w] > wi.partCap) wi.partCap = roundUp(newCap[w], kBlock);
        wi.partBase = partSlots;
        wi.firstPartBlock = partBlocks;
        wi.numPartBlocks = static_cast<int>(wi.partCap / kBlock);
        partSlots += wi.partCap;
        partBlocks += wi.numPartBlocks;
        infos[w] = wi;
    }
    if (partSlots >= (1ll << 31)) throw Error(ALIEN_B200_ERR_CAPACITY, "arena exceeds 2^31 particle slots");
    const DevState old = s_;
    const int* oldRankParts = rankParts_;
    const uint32_t* oldBlockCount = blockCount_;
    const size_t P = static_cast<size_t>(partSlots);
    // the new arrays beside the old ones; a failed allocation leaves the arena as it was
    DevState s = s_;
    s.pid = nullptr;  // allocated so far: the non-null new pointers
    s.ppos = s.pvel = s.splitPos = s.splitVel = nullptr;
    s.penergy = s.splitEnergy = nullptr;
    s.pcolor = s.palive = s.pselected = nullptr;
    s.pflag = s.blockSplit = nullptr;
    s.plast = nullptr;
    s.ptarget = s.pslot = nullptr;
    s.pmerge = nullptr;
    int* pbw = nullptr;
    int* rankParts = nullptr;
    uint32_t* blockCount = nullptr;
    try {
        allocParticleArrays(s, P, partBlocks);
        pbw = mem_.alloc<int>(partBlocks);
        rankParts = mem_.alloc<int>(P);
        blockCount = mem_.alloc<uint32_t>(static_cast<size_t>(std::max(s.numCellBlocks, partBlocks)) + 2);
    } catch (...) {
        for (const void* p : {static_cast<const void*>(s.pid), static_cast<const void*>(s.ppos), static_cast<const void*>(s.pvel),
                              static_cast<const void*>(s.penergy), static_cast<const void*>(s.pcolor),
                              static_cast<const void*>(s.palive), static_cast<const void*>(s.pselected),
                              static_cast<const void*>(s.pflag), static_cast<const void*>(s.plast),
                              static_cast<const void*>(s.ptarget), static_cast<const void*>(s.pslot),
                              static_cast<const void*>(s.pmerge), static_cast<const void*>(s.splitPos),
                              static_cast<const void*>(s.splitVel), static_cast<const void*>(s.splitEnergy),
                              static_cast<const void*>(s.blockSplit), static_cast<const void*>(pbw),
                              static_cast<const void*>(rankParts), static_cast<const void*>(blockCount)})
            if (p) mem_.release(p);
        throw;
    }
    AB_CK(cudaMemsetAsync(s.palive, 0, P, stream_));
    AB_CK(cudaMemsetAsync(s.pflag, 0, P * sizeof(uint32_t), stream_));
    std::vector<int> pbwHost(partBlocks);
    for (int w = 0; w < n; ++w) {
        const WorldInfo& from = worlds_[w].info;
        const WorldInfo& to = infos[w];
        for (int b = 0; b < to.numPartBlocks; ++b) pbwHost[to.firstPartBlock + b] = w;
        const size_t k = c[w].numParticles, a = static_cast<size_t>(from.partBase), z = static_cast<size_t>(to.partBase);
        if (!k) continue;
        auto move = [&](auto* dst, const auto* src, size_t items) {
            AB_CK(cudaMemcpyAsync(dst + z, src + a, items * sizeof(*src), cudaMemcpyDeviceToDevice, stream_));
        };
        move(s.pid, old.pid, k);
        move(s.plast, old.plast, k);
        move(s.ppos, old.ppos, k);
        move(s.pvel, old.pvel, k);
        move(s.penergy, old.penergy, k);
        move(s.pcolor, old.pcolor, k);
        move(s.pselected, old.pselected, k);
        move(s.palive, old.palive, k);
        move(s.pflag, old.pflag, k);
        move(s.splitPos, old.splitPos, k);
        move(s.splitVel, old.splitVel, k);
        move(s.splitEnergy, old.splitEnergy, k);
        AB_CK(cudaMemcpyAsync(s.blockSplit + to.firstPartBlock, old.blockSplit + from.firstPartBlock,
                              divUp(k, kBlock) * sizeof(uint32_t), cudaMemcpyDeviceToDevice, stream_));
    }
    AB_CK(cudaMemcpyAsync(pbw, pbwHost.data(), sizeof(int) * partBlocks, cudaMemcpyHostToDevice, stream_));
    for (const void* p : {static_cast<const void*>(old.pid), static_cast<const void*>(old.ppos), static_cast<const void*>(old.pvel),
                          static_cast<const void*>(old.penergy), static_cast<const void*>(old.pcolor),
                          static_cast<const void*>(old.palive), static_cast<const void*>(old.pselected),
                          static_cast<const void*>(old.pflag), static_cast<const void*>(old.plast),
                          static_cast<const void*>(old.ptarget), static_cast<const void*>(old.pslot),
                          static_cast<const void*>(old.pmerge), static_cast<const void*>(old.splitPos),
                          static_cast<const void*>(old.splitVel), static_cast<const void*>(old.splitEnergy),
                          static_cast<const void*>(old.blockSplit), static_cast<const void*>(old.partBlockWorld),
                          static_cast<const void*>(oldRankParts), static_cast<const void*>(oldBlockCount)})
        mem_.release(p);
    s.partBlockWorld = pbw;
    s.numPartBlocks = partBlocks;
    s.partSlots = partSlots;
    s_ = s;
    rankParts_ = rankParts;
    blockCount_ = blockCount;
    int device = 0, sms = 0;
    AB_CK(cudaGetDevice(&device));
    AB_CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    partGrid_ = std::max(1, std::min(partBlocks, 16 * std::max(sms, 1)));
    for (int w = 0; w < n; ++w) {
        worlds_[w].info = infos[w];
        maxWorldParts_ = std::max(maxWorldParts_, infos[w].partCap);
    }
    AB_CK(cudaMemcpyAsync(const_cast<WorldInfo*>(s_.worlds), infos.data(), sizeof(WorldInfo) * n, cudaMemcpyHostToDevice, stream_));
    releaseGraph();  // the graph holds the old arrays
    AB_CK(cudaStreamSynchronize(stream_));
}

std::vector<WorldCounters> Arena::readCounters()
{
    std::vector<WorldCounters> c(worlds_.size());
    AB_CK(cudaMemcpyAsync(c.data(), s_.counters, sizeof(WorldCounters) * c.size(), cudaMemcpyDeviceToHost, stream_));
    AB_CK(cudaStreamSynchronize(stream_));
    return c;
}

// keep at least half of each world's particle slots free: compact when the
// used slots pass 50 %, grow (rebuild) when live particles pass 50 %
void Arena::ensureParticleCapacity()
{
    settle();
    std::vector<WorldCounters> c = readCounters();
    {
        // a world that could not grow halts again (and tries to grow) from now on
        bool any = false;
        for (WorldCounters& x : c) {
            any |= x.dropExcess != 0;
            x.dropExcess = 0;
        }
        if (any) AB_CK(cudaMemcpyAsync(s_.counters, c.data(), sizeof(WorldCounters) * c.size(), cudaMemcpyHostToDevice, stream_));
    }
    std::vector<int> grow;
    for (int w = 0; w < numWorlds(); ++w) {
        if (!resident(w)) continue;
        const long long cap = worlds_[w].info.partCap;
        if (c[w].numParticles * 2ll <= cap) continue;
        compactParticles(w);
        uint64_t live = 0, dummy = 0;
        countData(w, &dummy, &live);
        if (static_cast<long long>(live) * 2 > cap) grow.push_back(w);
    }
    if (grow.empty()) return;
    if (live_) {
        // a live arena moves only the particles of the worlds that need room;
        // without a free range of three times the size a world keeps its
        // range (an overflow is then reported by the next synchronisation)
        for (int w : grow) moveParticles(w, 3 * worlds_[w].info.partCap);
        return;
    }
    // resize (the counterpart of _SimulationCudaFacade::resizeArrays,
    // SimulationCudaFacade.cu:619-655): the particle arrays are allocated
    // again on the device with three times the room for these worlds; the
    // growth changes no state
    std::vector<long long> newCap(numWorlds(), 0);
    for (int w : grow) newCap[w] = 3 * worlds_[w].info.partCap;
    growOrRebuild(newCap);
}

void Arena::growParticles(int w, uint64_t extra)
{
    if (live_) {
        moveParticles(w, worlds_[w].info.partCap + static_cast<long long>(extra));
        return;
    }
    std::vector<long long> newCap(numWorlds(), 0);
    newCap[w] = worlds_[w].info.partCap + static_cast<long long>(extra);
    growOrRebuild(newCap);
}

void Arena::growOrRebuild(const std::vector<long long>& newCap)
{
    try {
        growParticleArrays(newCap);
        return;
    } catch (const Error& e) {
        if (e.code != ALIEN_B200_ERR_OUT_OF_MEMORY) throw;
    }
    // no room for the new arrays beside the old ones: export, rebuild larger
    // (the old arena is released first), re-import; densities and absorbers
    // continue
    std::vector<Carried> carried(numWorlds());
    std::vector<uint64_t> extra(numWorlds(), 0);
    for (int w = 0; w < numWorlds(); ++w) {
        exportWorld(w, carried[w]);
        extra[w] = newCap[w] > worlds_[w].info.partCap ? static_cast<uint64_t>(newCap[w] - worlds_[w].info.partCap) : 0;
    }
    rebuildFromHost(carried, extra, true);
}

void Arena::exportWorld(int w, Carried& out)
{
    uint64_t nc = 0, np = 0, na = worlds_[w].auxSize;
    countData(w, &nc, &np);
    out.cells.resize(std::max<uint64_t>(nc, 1));
    out.parts.resize(std::max<uint64_t>(np, 1));
    std::vector<uint8_t> auxTmp(std::max<uint64_t>(na, 1));
    AlienDataTO to{&nc, out.cells.data(), &np, out.parts.data(), &na, auxTmp.data()};
    getData(w, false, AlienInt2{0, 0}, AlienInt2{0, 0}, &to);  // leaves the egress ranks of world w
    out.cells.resize(nc);
    out.parts.resize(np);
    const WorldInfo& wi = worlds_[w].info;
    AB_CK(cudaMallocAsync(reinterpret_cast<void**>(&out.density), sizeof(float) * std::max<uint64_t>(nc, 1), stream_));
    AB_CK(cudaMallocAsync(reinterpret_cast<void**>(&out.last), sizeof(unsigned long long) * std::max<uint64_t>(np, 1), stream_));
    launch(kGatherCarried, static_cast<int>(divUp(std::max(wi.cellCap, wi.partCap), kBlock)), kBlock, s_, w,
           static_cast<const int*>(rankCells_), static_cast<const int*>(rankParts_), out.density, out.last);
}

void Arena::rebuildFromHost(std::vector<Carried>& worlds, const std::vector<uint64_t>& extra, bool keepDensity)
{
    syncParamsFromDevice();  // zones, sources and the pool as the steps left them
    std::vector<WorldCounters> c = readCounters();
    std::vector<HostWorld> old = worlds_;
    std::vector<WorldSetup> setups(old.size());
    // auxiliary bytes held only on the device come back to the host first
    std::vector<std::vector<uint8_t>> auxHost(old.size());
    for (size_t w = 0; w < old.size(); ++w)
        if (old[w].auxSize && old[w].aux.empty()) {
            auxHost[w].resize(old[w].auxSize);
            AB_CK(cudaMemcpyAsync(auxHost[w].data(), s_.aux + old[w].info.auxBase, old[w].auxSize, cudaMemcpyDeviceToHost,
                                  stream_));
        }
    AB_CK(cudaStreamSynchronize(stream_));
    for (size_t w = 0; w < old.size(); ++w) {
        WorldSetup& ws = setups[w];
        ws.W = old[w].info.W;
        ws.H = old[w].info.H;
        ws.params = old[w].params;
        ws.timestep = c[w].timestep;
        ws.cells = worlds[w].cells.data();
        ws.numCells = worlds[w].cells.size();
        ws.particles = worlds[w].parts.data();
        ws.numParticles = worlds[w].parts.size();
        ws.aux = old[w].aux.empty() ? auxHost[w].data() : old[w].aux.data();
        ws.numAux = old[w].auxSize;
        ws.extraParticles = extra[w];
    }
    std::vector<unsigned long long> neurons(old.size() * ALIEN_B200_MAX_COLORS);
    AB_CK(cudaMemcpyAsync(neurons.data(), s_.neuronActivity, sizeof(unsigned long long) * neurons.size(), cudaMemcpyDeviceToHost,
                          stream_));
    AB_CK(cudaStreamSynchronize(stream_));
    build(setups);
    for (size_t w = 0; w < old.size(); ++w) {
        const long long nc = static_cast<long long>(worlds[w].cells.size()), np = static_cast<long long>(worlds[w].parts.size());
        launch(kRestoreCarried, static_cast<int>(divUp(std::max<long long>(std::max(nc, np), 1), kBlock)), kBlock, s_,
               static_cast<int>(w), keepDensity ? static_cast<const float*>(worlds[w].density) : nullptr, nc,
               static_cast<const unsigned long long*>(worlds[w].last), np);
        AB_CK(cudaFreeAsync(worlds[w].density, stream_));
        AB_CK(cudaFreeAsync(worlds[w].last, stream_));
        worlds[w].density = nullptr;
        worlds[w].last = nullptr;
    }
    // the accumulated statistics belong to the worlds, not to the layout
    AB_CK(cudaMemcpyAsync(s_.neuronActivity, neurons.data(), sizeof(unsigned long long) * neurons.size(), cudaMemcpyHostToDevice,
                          stream_));
    // ids continue where they were, not at max(id)+1 of the surviving objects
    std::vector<WorldCounters> now = readCounters();
    for (size_t w = 0; w < old.size(); ++w) {
        now[w].nextId = std::max(now[w].nextId, c[w].nextId);
        now[w].stepsRemaining = c[w].stepsRemaining;
        now[w].active = c[w].active;
    }
    AB_CK(cudaMemcpy(s_.counters, now.data(), sizeof(WorldCounters) * now.size(), cudaMemcpyHostToDevice));
}

void Arena::calcTimesteps(uint64_t n)
{
    // particle storage is checked (and compacted or grown) after at most 64
    // steps, counted across calls, so that many short calls cost one wait each
    const uint64_t chunk = 64;
    while (n > 0) {
        const uint64_t k = std::min(n, chunk - stepsSinceCheck_);
        enqueueSteps(k);
        n -= k;
        stepsSinceCheck_ += k;
        if (stepsSinceCheck_ >= chunk) {
            sync();
            ensureParticleCapacity();
            stepsSinceCheck_ = 0;
        }
    }
    sync();
}

void Arena::setParams(int w, const AlienPhysicsParams& p)
{
    settle();
    HostWorld& hw = worlds_[w];
    validateParams(p, hw.info.W, hw.info.H);
    // the tile grid depends on the interaction radius, and the cluster arrays
    // exist only in arenas built with rigidity
    const bool relayout = scanRadius(p) != hw.info.radiusInt || p.motionType != hw.info.motionType ||
                          (rigidityEnabled(p) && !s_.clusterAcc);
    if (relayout && live_) {
        relocate(w, 0, &p);
        return;
    }
    if (relayout) {
        // rebuild the arena; densities start again, as after every
        // parameter change (kResetDensity below)
        std::vector<Carried> carried(numWorlds());
        for (int v = 0; v < numWorlds(); ++v) exportWorld(v, carried[v]);
        hw.params = p;
        rebuildFromHost(carried, std::vector<uint64_t>(numWorlds(), 0), false);
        return;
    }
    hw.params = p;
    AB_CK(cudaMemcpyAsync(s_.params + w, &p, sizeof(p), cudaMemcpyHostToDevice, stream_));
    // prepareForSimulationParametersChanges -> cudaResetDensity (SimulationKernelsLauncher.cu:93-97)
    launch(kResetDensity, hw.info.numCellBlocks, kBlock, s_, w);
    // the external energy pool takes the parameters' value, and the active
    // sources follow the new zones and sources
    std::vector<WorldCounters> c = readCounters();
    c[w].externalEnergy = p.externalEnergy;
    AB_CK(cudaMemcpyAsync(s_.counters + w, &c[w], sizeof(WorldCounters), cudaMemcpyHostToDevice, stream_));
    bool any = false, rigid = false;
    for (const HostWorld& x : worlds_) {
        any |= needsWorldParams(x.params);
        rigid |= rigidityEnabled(x.params);
    }
    if (any != hasWorldParams_ || rigid != hasRigidity_) {
        hasWorldParams_ = any;
        hasRigidity_ = rigid;
        releaseGraph();  // the step gains or loses its kWorldsEnd launch or its cluster pass
    }
    if (hasWorldParams_) launch(kWorldsBegin, divUp(numWorlds(), kBlock), kBlock, s_);
    sync();
}

void Arena::syncParamsFromDevice()
{
    if (!hasWorldParams_ || worlds_.empty()) return;
    std::vector<AlienPhysicsParams> dev(worlds_.size());
    AB_CK(cudaMemcpyAsync(dev.data(), s_.params, sizeof(AlienPhysicsParams) * dev.size(), cudaMemcpyDeviceToHost, stream_));
    std::vector<WorldCounters> c = readCounters();
    for (size_t w = 0; w < worlds_.size(); ++w) {
        AlienPhysicsParams& h = worlds_[w].params;
        for (int i = 0; i < ALIEN_B200_MAX_ZONES; ++i) {
            h.zones[i].posX = dev[w].zones[i].posX;
            h.zones[i].posY = dev[w].zones[i].posY;
        }
        for (int i = 0; i < ALIEN_B200_MAX_RADIATION_SOURCES; ++i) {
            h.radiationSources[i].posX = dev[w].radiationSources[i].posX;
            h.radiationSources[i].posY = dev[w].radiationSources[i].posY;
        }
        h.externalEnergy = static_cast<float>(c[w].externalEnergy);
    }
}

AlienPhysicsParams Arena::params(int w)
{
    syncParamsFromDevice();
    return worlds_[w].params;
}

void Arena::setStepBudget(int w, uint64_t steps)
{
    settle();
    std::vector<WorldCounters> c = readCounters();
    c[w].stepsRemaining = steps == 0 ? ~0ull : steps;
    c[w].active = 1;
    AB_CK(cudaMemcpy(s_.counters, c.data(), sizeof(WorldCounters) * c.size(), cudaMemcpyHostToDevice));
}

void Arena::setTimestep(int w, uint64_t t)
{
    settle();
    worlds_[w].setTimestep = t;
    std::vector<WorldCounters> c = readCounters();
    c[w].timestep = t;
    AB_CK(cudaMemcpy(s_.counters, c.data(), sizeof(WorldCounters) * c.size(), cudaMemcpyHostToDevice));
}

// ----------------------------------------------------------- egress ------
void Arena::countData(int w, uint64_t* cells, uint64_t* particles)
{
    const WorldInfo& wi = worlds_[w].info;
    launch(kSelectCells, wi.numCellBlocks, kBlock, s_, w, 0, 0, 0, 0, 0, rankCells_, blockCount_);
    launch(kScanPartials<kBlock>, 1, kBlock, blockCount_, wi.numCellBlocks);
    uint32_t nc = 0, np = 0;
    AB_CK(cudaMemcpyAsync(&nc, blockCount_ + wi.numCellBlocks, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream_));
    AB_CK(cudaStreamSynchronize(stream_));
    launch(kSelectParticles, wi.numPartBlocks, kBlock, s_, w, 0, 0, 0, 0, 0, rankParts_, blockCount_);
    launch(kScanPartials<kBlock>, 1, kBlock, blockCount_, wi.numPartBlocks);
    AB_CK(cudaMemcpyAsync(&np, blockCount_ + wi.numPartBlocks, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream_));
    AB_CK(cudaStreamSynchronize(stream_));
    *cells = nc;
    *particles = np;
}

void Arena::getData(int w, bool useRect, AlienInt2 ul, AlienInt2 lr, const AlienDataTO* out)
{
    if (!out || !out->numCells || !out->numParticles || !out->numAuxiliaryData)
        throw Error(ALIEN_B200_ERR_INVALID_ARGUMENT, "DataTO counters must not be null");
    settle();  // a halted world completes its step before it is read
    const WorldInfo& wi = worlds_[w].info;
    AlienCellTO* egressCells = static_cast<AlienCellTO*>(
        egressCells_.ensure(sizeof(AlienCellTO) * static_cast<size_t>(std::max<long long>(maxWorldCells_, 1))));
    AlienParticleTO* egressParts = static_cast<AlienParticleTO*>(
        egressParts_.ensure(sizeof(AlienParticleTO) * static_cast<size_t>(std::max<long long>(maxWorldParts_, 1))));
    const int u = useRect ? 1 : 0;
    uint32_t nc = 0, np = 0;
    launch(kSelectCells, wi.numCellBlocks, kBlock, s_, w, u, ul.x, ul.y, lr.x, lr.y, rankCells_, blockCount_);
    launch(kScanPartials<kBlock>, 1, kBlock, blockCount_, wi.numCellBlocks);
    launch(kFinishRanks, wi.numCellBlocks, kBlock, wi.cellBase, rankCells_, static_cast<const uint32_t*>(blockCount_));
    AB_CK(cudaMemcpyAsync(&nc, blockCount_ + wi.numCellBlocks, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream_));
    launch(kEgressCells, wi.numCellBlocks, kBlock, s_, w, static_cast<const int*>(rankCells_), static_cast<const AlienCellTO*>(cold_),
           egressCells);
    AB_CK(cudaStreamSynchronize(stream_));
    launch(kSelectParticles, wi.numPartBlocks, kBlock, s_, w, u, ul.x, ul.y, lr.x, lr.y, rankParts_, blockCount_);
    launch(kScanPartials<kBlock>, 1, kBlock, blockCount_, wi.numPartBlocks);
    launch(kFinishRanks, wi.numPartBlocks, kBlock, wi.partBase, rankParts_, static_cast<const uint32_t*>(blockCount_));
    AB_CK(cudaMemcpyAsync(&np, blockCount_ + wi.numPartBlocks, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream_));
    launch(kEgressParticles, wi.numPartBlocks, kBlock, s_, w, static_cast<const int*>(rankParts_), egressParts);
    AB_CK(cudaStreamSynchronize(stream_));
    if (nc && !out->cells) throw Error(ALIEN_B200_ERR_INVALID_ARGUMENT, "DataTO.cells is null");
    if (np && !out->particles) throw Error(ALIEN_B200_ERR_INVALID_ARGUMENT, "DataTO.particles is null");
    if (nc) AB_CK(cudaMemcpyAsync(out->cells, egressCells, sizeof(AlienCellTO) * nc, cudaMemcpyDeviceToHost, stream_));
    if (np) AB_CK(cudaMemcpyAsync(out->particles, egressParts, sizeof(AlienParticleTO) * np, cudaMemcpyDeviceToHost, stream_));
    const HostWorld& hw = worlds_[w];
    if (hw.auxSize) {
        if (!out->auxiliaryData) throw Error(ALIEN_B200_ERR_INVALID_ARGUMENT, "DataTO.auxiliaryData is null");
        if (hw.aux.empty())
            AB_CK(cudaMemcpyAsync(out->auxiliaryData, s_.aux + hw.info.auxBase, hw.auxSize, cudaMemcpyDeviceToHost, stream_));
        else
            std::memcpy(out->auxiliaryData, hw.aux.data(), hw.auxSize);
    }
    AB_CK(cudaStreamSynchronize(stream_));
    *out->numCells = nc;
    *out->numParticles = np;
    *out->numAuxiliaryData = hw.auxSize;
}

void Arena::compactParticles(int w)
{
    const WorldInfo& wi = worlds_[w].info;
    launch(kSelectParticles, wi.numPartBlocks, kBlock, s_, w, 0, 0, 0, 0, 0, rankParts_, blockCount_);
    launch(kScanPartials<kBlock>, 1, kBlock, blockCount_, wi.numPartBlocks);
    launch(kFinishRanks, wi.numPartBlocks, kBlock, wi.partBase, rankParts_, static_cast<const uint32_t*>(blockCount_));
    uint32_t live = 0;
    AB_CK(cudaMemcpyAsync(&live, blockCount_ + wi.numPartBlocks, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream_));
    AB_CK(cudaStreamSynchronize(stream_));
    const size_t cap = static_cast<size_t>(wi.partCap);
    unsigned long long *tid, *tlast;
    float2 *tpos, *tvel;
    float* te;
    uint8_t *tc, *tsel;
    AB_CK(cudaMallocAsync(reinterpret_cast<void**>(&tid), cap * 8, stream_));
    AB_CK(cudaMallocAsync(reinterpret_cast<void**>(&tlast), cap * 8, stream_));
    AB_CK(cudaMallocAsync(reinterpret_cast<void**>(&tpos), cap * 8, stream_));
    AB_CK(cudaMallocAsync(reinterpret_cast<void**>(&tvel), cap * 8, stream_));
    AB_CK(cudaMallocAsync(reinterpret_cast<void**>(&te), cap * 4, stream_));
    AB_CK(cudaMallocAsync(reinterpret_cast<void**>(&tc), cap, stream_));
    AB_CK(cudaMallocAsync(reinterpret_cast<void**>(&tsel), cap, stream_));
    launch(kCompactParticlesGather, wi.numPartBlocks, kBlock, s_, w, static_cast<const int*>(rankParts_), tid, tpos, tvel, te, tc, tsel,
           tlast);
    launch(kCompactParticlesScatter, wi.numPartBlocks, kBlock, s_, w, static_cast<long long>(live),
           static_cast<const unsigned long long*>(tid), static_cast<const float2*>(tpos), static_cast<const float2*>(tvel),
           static_cast<const float*>(te), static_cast<const uint8_t*>(tc), static_cast<const uint8_t*>(tsel),
           static_cast<const unsigned long long*>(tlast));
    for (void* p : {static_cast<void*>(tid), static_cast<void*>(tlast), static_cast<void*>(tpos), static_cast<void*>(tvel),
                    static_cast<void*>(te), static_cast<void*>(tc), static_cast<void*>(tsel)})
        AB_CK(cudaFreeAsync(p, stream_));
    std::vector<WorldCounters> c = readCounters();
    c[w].numParticles = live;
    c[w].deadParticles = 0;
    AB_CK(cudaMemcpyAsync(s_.counters + w, &c[w], sizeof(WorldCounters), cudaMemcpyHostToDevice, stream_));
    AB_CK(cudaStreamSynchronize(stream_));
}

// the cell map and staged records of the current state, by the step's own
// binning kernels without the rest of the step (no radiation, no particle
// map); everything written here is rebuilt by the next step
void Arena::binCurrentState()
{
    refreshLayout();
    const DevState& s = s_;
    AB_CK(cudaMemsetAsync(s.tileCount, 0, sizeof(uint32_t) * (static_cast<size_t>(s.numTiles) + 1), stream_));
    launch(kBinMap, s.numCellBlocks, kBlock, s);
    scan(s.tileCount, s.numTiles, s.tileStart);
    launch(kScatter, s.numCellBlocks, kBlock, s);
    launch(kStage, s.numCellBlocks, kBlock, s);
}

// Region shape of a world for the pair kernel: regW x regH tiles (the
// shape, clamped to the world) with a one-tile halo that never overlaps the
// region itself and lies within half a world (so that a seam shift gives
// the minimal image); worlds too small for that take the global path.
void Arena::assignRegions(WorldInfo& wi, const int* shape)
{
    if (wi.nTX >= 4 && wi.nTY >= 4 && wi.W >= 4 * wi.T && wi.H >= 4 * wi.T) {
        wi.regW = std::min(shape[0], wi.nTX - 2);
        wi.regH = std::min(shape[1], wi.nTY - 2);
        wi.regionShared = 1;
    } else {
        wi.regW = std::min(shape[0], wi.nTX);
        wi.regH = std::min(shape[1], wi.nTY);
        wi.regionShared = 0;
    }
    if (wi.regionShared && wi.motionType == ALIEN_B200_MOTION_FLUID) {
        // the region at the right (top) seam shifts its tiles down by the
        // world size, which is exact when its halo starts in the world's
        // upper half: narrower regions where a world is only a few regions
        // wide (regW = 1 always satisfies it, as nTX >= 4)
        auto exact = [&](int reg, int nT, int size) {
            const int last = (divUp(nT, reg) - 1) * reg;
            return last >= 1 && 2ll * (last - 1) * wi.T >= size;
        };
        while (wi.regW > 1 && !exact(wi.regW, wi.nTX, wi.W)) --wi.regW;
        while (wi.regH > 1 && !exact(wi.regH, wi.nTY, wi.H)) --wi.regH;
    }
    wi.nRX = divUp(wi.nTX, wi.regW);
    wi.nRY = divUp(wi.nTY, wi.regH);
}

int Arena::maxRegions(const WorldInfo& wi)
{
    int most = 0;
    for (int i = 0; i < kNumRegionChoices; ++i) {
        WorldInfo t = wi;
        assignRegions(t, kRegionChoices[wi.motionType][i]);
        most = std::max(most, t.nRX * t.nRY);
    }
    return most;
}

// region tables of the shapes in use: every world's regions, regionBase and
// the world of each region, uploaded on the arena's stream
void Arena::applyRegionShapes()
{
    std::vector<WorldInfo> infos(worlds_.size());
    std::vector<int> rgw;
    for (size_t w = 0; w < worlds_.size(); ++w) {
        WorldInfo& wi = worlds_[w].info;
        if (worlds_[w].vacant) {
            wi.nRX = wi.nRY = 0;  // an unused slot of a live arena has no regions
        } else {
            assignRegions(wi, regionShape(wi.motionType));
        }
        wi.regionBase = static_cast<int>(rgw.size());
        rgw.insert(rgw.end(), static_cast<size_t>(wi.nRX) * wi.nRY, static_cast<int>(w));
        infos[w] = wi;
    }
    s_.numRegions = static_cast<int>(rgw.size());
    // copies from pageable host memory are staged before the calls return,
    // so the temporaries may go without waiting for the stream (a live
    // arena keeps its enqueued steps running through an admission)
    if (!infos.empty())
        AB_CK(cudaMemcpyAsync(const_cast<WorldInfo*>(s_.worlds), infos.data(), sizeof(WorldInfo) * infos.size(),
                              cudaMemcpyHostToDevice, stream_));
    if (!rgw.empty())
        AB_CK(cudaMemcpyAsync(const_cast<int*>(s_.regionWorld), rgw.data(), sizeof(int) * rgw.size(), cudaMemcpyHostToDevice,
                              stream_));
    if (!live_) AB_CK(cudaStreamSynchronize(stream_));
    releaseGraph();
}

void Arena::setRegionChoice(int motion, int choicePlusOne)
{
    if (motion != ALIEN_B200_MOTION_FLUID && motion != ALIEN_B200_MOTION_COLLISION)
        throw Error(ALIEN_B200_ERR_INVALID_ARGUMENT, "motion type must be 0 (fluid) or 1 (collision)");
    if (choicePlusOne < 0 || choicePlusOne > kNumRegionChoices)
        throw Error(ALIEN_B200_ERR_INVALID_ARGUMENT, "region choice must be 0 (autotune) or 1.." + std::to_string(kNumRegionChoices));
    regionChoiceFixed_[motion] = choicePlusOne;
    if (choicePlusOne && regionChoice_[motion] != choicePlusOne - 1) {
        regionChoice_[motion] = choicePlusOne - 1;
        if (!worlds_.empty()) applyRegionShapes();
    }
}

AlienLaunchConfig Arena::launchConfig() const
{
    AlienLaunchConfig c;
    std::memset(&c, 0, sizeof(c));
    for (int m = 0; m < 2; ++m) {
        c.regionTiles[m][0] = regionShape(m)[0];
        c.regionTiles[m][1] = regionShape(m)[1];
        c.regionChoice[m] = regionChoice_[m];
        c.regionChoiceFixed[m] = regionChoiceFixed_[m];
        for (int i = 0; i < kNumRegionChoices; ++i) {
            c.tunedMs[m][i] = tunedMs_[m][i];
            c.candidates[m][i][0] = kRegionChoices[m][i][0];
            c.candidates[m][i][1] = kRegionChoices[m][i][1];
        }
    }
    c.tuned = tuned_ ? 1 : 0;
    return c;
}

// The autotuner: for every motion type present whose region shape the
// caller did not fix, the pair kernel of the current state is launched with
// each candidate shape (one untimed launch, then three between CUDA events)
// and the fastest is kept (alien_b200_choose_region).  The pair kernel reads
// only the staged records and overwrites its own outputs, which the next
// step recomputes, and a cell's neighbours are visited in the same order
// whatever the region shape, so tuning changes neither the state nor any
// result.  Runs once per
// arena layout, before its first step and before the step graph is
// captured.
void Arena::autotune()
{
    tuned_ = true;
    const bool need[2] = {hasFluid_ && !regionChoiceFixed_[ALIEN_B200_MOTION_FLUID] && !motionTuned_[ALIEN_B200_MOTION_FLUID],
                          hasCollision_ && !regionChoiceFixed_[ALIEN_B200_MOTION_COLLISION] &&
                              !motionTuned_[ALIEN_B200_MOTION_COLLISION]};
    if (!need[0] && !need[1]) return;
    std::vector<WorldCounters> c = readCounters();
    long long cells = 0;
    for (const WorldCounters& x : c) cells += x.active ? x.numCells : 0;
    if (cells == 0) return;
    binCurrentState();
    cudaEvent_t ev[4];
    for (cudaEvent_t& e : ev) AB_CK(cudaEventCreate(&e));
    try {
        for (int m = 0; m < 2; ++m) {
            if (!need[m]) continue;
            motionTuned_[m] = true;
            for (int i = 0; i < kNumRegionChoices; ++i) tunedMs_[m][i] = 0.0f;
            for (int i = 0; i < kNumRegionChoices; ++i) {
                regionChoice_[m] = i;
                applyRegionShapes();
                for (int rep = 0; rep < 4; ++rep) {
                    // deferred cells are listed again by every launch
                    AB_CK(cudaMemsetAsync(s_.pairOverflowCount, 0, sizeof(uint32_t), stream_));
                    if (rep > 0) AB_CK(cudaEventRecord(ev[rep], stream_));
                    if (m == ALIEN_B200_MOTION_FLUID)
                        launchPairs<ALIEN_B200_MOTION_FLUID>();
                    else
                        launchPairs<ALIEN_B200_MOTION_COLLISION>();
                    if (rep > 0) {
                        AB_CK(cudaEventRecord(ev[0], stream_));
                        AB_CK(cudaEventSynchronize(ev[0]));
                        float ms = 0.0f;
                        AB_CK(cudaEventElapsedTime(&ms, ev[rep], ev[0]));
                        tunedMs_[m][i] += ms / 3.0f;
                    }
                }
            }
            regionChoice_[m] = alien_b200_choose_region(tunedMs_[m], kNumRegionChoices);
        }
    } catch (...) {
        for (cudaEvent_t& e : ev) cudaEventDestroy(e);
        throw;
    }
    for (cudaEvent_t& e : ev) cudaEventDestroy(e);
    applyRegionShapes();
}

uint64_t Arena::cellMap(uint64_t capacity, uint64_t* ids, uint32_t* slots, uint32_t* tiles, uint8_t* flags)
{
    settle();
    const DevState& s = s_;
    binCurrentState();
    uint32_t total = 0;
    AB_CK(cudaMemcpyAsync(&total, s.tileStart + s.numTiles, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream_));
    AB_CK(cudaStreamSynchronize(stream_));
    if (total > capacity) return total;
    const size_t n = std::max<size_t>(total, 1);
    unsigned long long* dIds = nullptr;
    uint32_t *dSlots = nullptr, *dTiles = nullptr;
    uint8_t* dFlags = nullptr;
    AB_CK(cudaMallocAsync(reinterpret_cast<void**>(&dIds), n * 8, stream_));
    AB_CK(cudaMallocAsync(reinterpret_cast<void**>(&dSlots), n * 4, stream_));
    AB_CK(cudaMallocAsync(reinterpret_cast<void**>(&dTiles), n * 4, stream_));
    AB_CK(cudaMallocAsync(reinterpret_cast<void**>(&dFlags), n, stream_));
    launch(kExportCellMap, divUp(total, kBlock), kBlock, s, dIds, dSlots, dTiles, dFlags);
    if (total) {
        AB_CK(cudaMemcpyAsync(ids, dIds, total * 8ull, cudaMemcpyDeviceToHost, stream_));
        AB_CK(cudaMemcpyAsync(slots, dSlots, total * 4ull, cudaMemcpyDeviceToHost, stream_));
        AB_CK(cudaMemcpyAsync(tiles, dTiles, total * 4ull, cudaMemcpyDeviceToHost, stream_));
        AB_CK(cudaMemcpyAsync(flags, dFlags, total, cudaMemcpyDeviceToHost, stream_));
    }
    for (void* p : {static_cast<void*>(dIds), static_cast<void*>(dSlots), static_cast<void*>(dTiles), static_cast<void*>(dFlags)})
        AB_CK(cudaFreeAsync(p, stream_));
    AB_CK(cudaStreamSynchronize(stream_));
    return total;
}

AlienRawStatisticsData Arena::statisticsData(int w)
{
    settle();
    AB_CK(cudaMemsetAsync(timeline_, 0, sizeof(TimelineAcc), stream_));
    const WorldInfo& wi = worlds_[w].info;
    const long long slots = std::max(wi.cellCap, wi.partCap);
    const int grid = static_cast<int>(std::max<long long>(1, std::min<long long>(statsGrid_, (slots + kBlock - 1) / kBlock)));
    launch(kStatsTimeline, grid, kBlock, s_, w, timeline_);
    launch(kStatsHistogram, grid, kBlock, s_, w, timeline_);
    TimelineAcc a;
    AB_CK(cudaMemcpyAsync(&a, timeline_, sizeof(a), cudaMemcpyDeviceToHost, stream_));
    unsigned long long neurons[ALIEN_B200_MAX_COLORS];
    AB_CK(cudaMemcpyAsync(neurons, s_.neuronActivity + static_cast<size_t>(w) * ALIEN_B200_MAX_COLORS, sizeof(neurons),
                          cudaMemcpyDeviceToHost, stream_));
    AB_CK(cudaStreamSynchronize(stream_));
    AlienRawStatisticsData r;
    std::memset(&r, 0, sizeof(r));
    AlienTimestepStatistics& t = r.timeline.timestep;
    for (int c = 0; c < ALIEN_B200_MAX_COLORS; ++c) {
        t.numCells[c] = static_cast<int32_t>(a.cells[c]);
        t.numFreeCells[c] = static_cast<int32_t>(a.freeCells[c]);
        t.numParticles[c] = static_cast<int32_t>(a.particles[c]);
        t.totalEnergy[c] = static_cast<float>(static_cast<double>(a.energyFix[c]) / 65536.0);
        r.timeline.accumulated.numNeuronActivities[c] = neurons[c];
        for (int k = 0; k < ALIEN_B200_MAX_HISTOGRAM_SLOTS; ++k)
            r.histogram.numCellsByColorBySlot[c][k] = static_cast<int32_t>(a.histogram[c][k]);
    }
    r.histogram.maxValue = static_cast<int32_t>(a.maxAge);
    return r;
}

void Arena::resetTimeIntervalStatistics(int w)
{
    AB_CK(cudaMemsetAsync(s_.neuronActivity + static_cast<size_t>(w) * ALIEN_B200_MAX_COLORS, 0,
                          sizeof(unsigned long long) * ALIEN_B200_MAX_COLORS, stream_));
    AB_CK(cudaStreamSynchronize(stream_));
}

void Arena::densityMap(int w, AlienDensityMap* out)
{
    settle();
    const HostWorld& hw = worlds_[w];
    const WorldInfo& wi = hw.info;
    out->sizeX = wi.W / kDensitySlot;
    out->sizeY = wi.H / kDensitySlot;
    uint64_t* host64[8] = {out->color, out->otherMutant, out->sameMutant1, out->sameMutant2, out->lessComplexity1,
                           out->lessComplexity2, out->moreComplexity1, out->moreComplexity2};
    bool any = out->specificMutant != nullptr;
    for (uint64_t* p : host64) any |= p != nullptr;
    const size_t n = static_cast<size_t>(out->sizeX) * static_cast<size_t>(out->sizeY);
    if (!any || n == 0) return;
    // one zeroed device block: eight u64 maps, then the u32 map
    const size_t bytes = n * (8 * sizeof(unsigned long long) + sizeof(unsigned int));
    unsigned long long* d = nullptr;
    AB_CK(cudaMallocAsync(reinterpret_cast<void**>(&d), bytes, stream_));
    try {
        AB_CK(cudaMemsetAsync(d, 0, bytes, stream_));
        DensityMapOut m;
        m.color = d;
        m.otherMutant = d + n;
        m.sameMutant1 = d + 2 * n;
        m.sameMutant2 = d + 3 * n;
        m.lessComplexity1 = d + 4 * n;
        m.lessComplexity2 = d + 5 * n;
        m.moreComplexity1 = d + 6 * n;
        m.moreComplexity2 = d + 7 * n;
        m.specificMutant = reinterpret_cast<unsigned int*>(d + 8 * n);
        m.sizeX = out->sizeX;
        m.sizeY = out->sizeY;
        WorldCounters c;
        AB_CK(cudaMemcpyAsync(&c, s_.counters + w, sizeof(c), cudaMemcpyDeviceToHost, stream_));
        AB_CK(cudaStreamSynchronize(stream_));
        // the step that filled the map: the last one, or none since the world was set
        m.timestep = c.timestep != hw.setTimestep && c.timestep > 0 ? c.timestep - 1 : c.timestep;
        if (c.numCells) launch(kDensityMap, static_cast<int>(divUp(static_cast<long long>(c.numCells), kBlock)), kBlock, s_, w, m);
        const unsigned long long* dev64[8] = {m.color, m.otherMutant, m.sameMutant1, m.sameMutant2, m.lessComplexity1,
                                              m.lessComplexity2, m.moreComplexity1, m.moreComplexity2};
        for (int k = 0; k < 8; ++k)
            if (host64[k])
                AB_CK(cudaMemcpyAsync(host64[k], dev64[k], n * sizeof(unsigned long long), cudaMemcpyDeviceToHost, stream_));
        if (out->specificMutant)
            AB_CK(cudaMemcpyAsync(out->specificMutant, m.specificMutant, n * sizeof(unsigned int), cudaMemcpyDeviceToHost,
                                  stream_));
        AB_CK(cudaFreeAsync(d, stream_));
        AB_CK(cudaStreamSynchronize(stream_));
    } catch (...) {
        cudaFreeAsync(d, stream_);
        cudaStreamSynchronize(stream_);
        throw;
    }
}

AlienRawStatistics Arena::statistics(int w)
{
    settle();
    AB_CK(cudaMemsetAsync(stats_ + w, 0, sizeof(StatsAcc), stream_));
    {
        const WorldInfo& wi = worlds_[w].info;
        const long long slots = std::max(wi.cellCap, wi.partCap);
        const int grid = static_cast<int>(std::max<long long>(1, std::min<long long>(statsGrid_, (slots + kBlock - 1) / kBlock)));
        launch(kStatsWorld, grid, kBlock, s_, w, stats_);
    }
    Readback& rb = readback();
    AB_CK(cudaMemcpyAsync(&rb.stats, stats_ + w, sizeof(StatsAcc), cudaMemcpyDeviceToHost, stream_));
    AB_CK(cudaMemcpyAsync(&rb.counters, s_.counters + w, sizeof(WorldCounters), cudaMemcpyDeviceToHost, stream_));
    AB_CK(cudaStreamSynchronize(stream_));
    const StatsAcc a = rb.stats;
    const WorldCounters c = rb.counters;
    AlienRawStatistics r;
    std::memset(&r, 0, sizeof(r));
    r.timestep = c.timestep;
    r.numCells = a.numCells;
    r.numParticles = a.numParticles;
    r.numConnections = a.numConnections;
    for (int i = 0; i < ALIEN_B200_MAX_COLORS; ++i) r.numCellsByColor[i] = a.numCellsByColor[i];
    r.totalCellEnergy = static_cast<double>(a.cellEnergyFix) / 65536.0;
    r.totalParticleEnergy = static_cast<double>(a.particleEnergyFix) / 65536.0;
    return r;
}

template <class F>
static int guarded(F&& f)
{
    try {
        f();
        return ALIEN_B200_OK;
    } catch (const Error& e) {
        g_lastError = e.what();
        return e.code;
    } catch (const std::bad_alloc&) {
        g_lastError = "host allocation failed";
        return ALIEN_B200_ERR_OUT_OF_MEMORY;
    } catch (const std::exception& e) {
        g_lastError = e.what();
        return ALIEN_B200_ERR_CUDA;
    }
}

static void ensureDevice()
{
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0) {
        cudaGetLastError();
        throw Error(ALIEN_B200_ERR_NO_DEVICE, "no CUDA device available");
    }
    // the default memory pool of the current device keeps freed arena
    // blocks for reuse instead of returning them at every synchronisation
    // (a per-process setting of this library's allocations; other users of
    // the pool see it too)
    static std::mutex m;
    static bool configured[64] = {};
    int device = 0;
    AB_CK(cudaGetDevice(&device));
    std::lock_guard<std::mutex> lock(m);
    if (device >= 0 && device < 64 && !configured[device]) {
        cudaMemPool_t pool;
        AB_CK(cudaDeviceGetDefaultMemPool(&pool, device));
        uint64_t threshold = UINT64_MAX;
        AB_CK(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &threshold));
        configured[device] = true;
    }
}

static void checkDataTO(const AlienDataTO* d)
{
    if (!d || !d->numCells || !d->numParticles || !d->numAuxiliaryData)
        throw Error(ALIEN_B200_ERR_INVALID_ARGUMENT, "DataTO counters must not be null");
    if (*d->numCells && !d->cells) throw Error(ALIEN_B200_ERR_INVALID_ARGUMENT, "DataTO.cells is null");
    if (*d->numParticles && !d->particles) throw Error(ALIEN_B200_ERR_INVALID_ARGUMENT, "DataTO.particles is null");
    if (*d->numAuxiliaryData && !d->auxiliaryData) throw Error(ALIEN_B200_ERR_INVALID_ARGUMENT, "DataTO.auxiliaryData is null");
    // the per-cell checks run on the device during the build (kCheckCells)
}

static WorldSetup setupFrom(const AlienGeneralSettings& g, const AlienPhysicsParams& p, uint64_t timestep, const AlienDataTO* d)
{
    WorldSetup ws;
    ws.W = g.worldSizeX;
    ws.H = g.worldSizeY;
    ws.params = p;
    ws.timestep = timestep;
    if (d) {
        ws.cells = d->cells;
        ws.numCells = *d->numCells;
        ws.particles = d->particles;
        ws.numParticles = *d->numParticles;
        ws.aux = d->auxiliaryData;
        ws.numAux = *d->numAuxiliaryData;
    }
    return ws;
}

}  // namespace ab

using namespace ab;

struct alien_b200_simulation {
    cudaStream_t stream = nullptr;
    AlienGeneralSettings general{};
    AlienPhysicsParams params{};
    uint64_t extraParticles = 0;
    std::unique_ptr<Arena> arena;
};

struct alien_b200_batch {
    cudaStream_t stream = nullptr;
    std::unique_ptr<Arena> arena;
};

extern "C" {

int alien_b200_version(void) { return 1; }

int alien_b200_select_device(int device)
{
    return guarded([&] {
        ensureDevice();
        AB_CK(cudaSetDevice(device));
    });
}

void alien_b200_default_parameters(AlienPhysicsParams* p)
{
    if (!p) return;
    std::memset(p, 0, sizeof(*p));
    p->timestepSize = 1.0f;
    p->motionType = ALIEN_B200_MOTION_FLUID;
    p->smoothingLength = 0.8f;
    p->viscosityStrength = 0.1f;
    p->pressureStrength = 0.1f;
    p->cellMaxCollisionDistance = 1.3f;
    p->cellRepulsionStrength = 0.08f;
    p->innerFriction = 0.3f;
    p->cellMaxVelocity = 2.0f;
    p->cellMinDistance = 0.3f;
    p->cellMaxForceDecayProb = 0.2f;
    p->radiationProb = 0.03f;
    p->radiationVelocityMultiplier = 1.0f;
    p->radiationVelocityPerturbation = 0.5f;
    p->cellDeathConsequences = ALIEN_B200_DEATH_DETACHED_PARTS_DIE;
    p->friction = 0.001f;
    p->rigidity = 0.0f;
    p->cellFusionVelocity = 0.6f;
    p->cellMaxBindingEnergy = 3.4028234663852886e38f;
    p->cellNumExecutionOrderNumbers = 6;
    for (int i = 0; i < ALIEN_B200_MAX_COLORS; ++i) {
        p->cellMaxBindingDistance[i] = 3.6f;
        p->radiationMinCellAge[i] = 0;
        p->highRadiationFactor[i] = 0.0f;
        p->highRadiationMinCellEnergy[i] = 500.0f;
        p->cellMaxAge[i] = 2147483647;
        p->particleSplitEnergy[i] = 3.4028234663852886e38f;
        p->radiationAbsorption[i] = 1.0f;
        p->radiationCellAgeStrength[i] = 0.00002f;
        p->cellMaxForce[i] = 0.8f;
        p->cellMinEnergy[i] = 50.0f;
        p->cellDeathProbability[i] = 0.001f;
    }
    p->externalEnergyBackflowLimit = 3.4028234663852886e38f;
    // zones (SimulationParametersZone.h): circular, core and fade-out radius
    // 100, radial-flow strength 0.001, the base values, nothing activated
    for (AlienZone& z : p->zones) {
        z.fadeoutRadius = 100.0f;
        z.shapeType = ALIEN_B200_SHAPE_CIRCULAR;
        z.coreRadius = 100.0f;
        z.width = 100.0f;
        z.height = 200.0f;
        z.flowType = ALIEN_B200_FLOW_NONE;
        z.flowStrength = 0.001f;
        z.friction = p->friction;
        z.rigidity = p->rigidity;
        z.cellFusionVelocity = p->cellFusionVelocity;
        z.cellMaxBindingEnergy = p->cellMaxBindingEnergy;
        for (int c = 0; c < ALIEN_B200_MAX_COLORS; ++c) {
            z.radiationAbsorption[c] = p->radiationAbsorption[c];
            z.radiationCellAgeStrength[c] = p->radiationCellAgeStrength[c];
            z.cellMaxForce[c] = p->cellMaxForce[c];
            z.cellMinEnergy[c] = p->cellMinEnergy[c];
            z.cellDeathProbability[c] = p->cellDeathProbability[c];
        }
    }
    // radiation sources (RadiationSource.h): circular of radius 1
    for (AlienRadiationSource& r : p->radiationSources) {
        r.radius = 1.0f;
        r.width = 100.0f;
        r.height = 200.0f;
    }
}

int alien_b200_last_error(char* buffer, size_t size)
{
    if (!buffer || size == 0) return static_cast<int>(g_lastError.size());
    std::snprintf(buffer, size, "%s", g_lastError.c_str());
    return static_cast<int>(g_lastError.size());
}

int alien_b200_create(const AlienGeneralSettings* general, const AlienPhysicsParams* params, uint64_t timestep,
                      alien_b200_simulation** out)
{
    return guarded([&] {
        if (!general || !params || !out) throw Error(ALIEN_B200_ERR_INVALID_ARGUMENT, "null argument");
        *out = nullptr;
        ensureDevice();
        validateParams(*params, general->worldSizeX, general->worldSizeY);
        auto sim = std::make_unique<alien_b200_simulation>();
        sim->general = *general;
        sim->params = *params;
        AB_CK(cudaStreamCreateWithFlags(&sim->stream, cudaStreamNonBlocking));
        sim->arena = std::make_unique<Arena>(sim->stream);
        sim->arena->build({setupFrom(*general, *params, timestep, nullptr)});
        *out = sim.release();
    });
}

int alien_b200_destroy(alien_b200_simulation* sim)
{
    return guarded([&] {
        if (!sim) return;
        if (sim->stream) cudaStreamSynchronize(sim->stream);
        sim->arena.reset();
        if (sim->stream) cudaStreamDestroy(sim->stream);
        delete sim;
    });
}

int alien_b200_calc_timesteps(alien_b200_simulation* sim, uint64_t timesteps)
{
    return guarded([&] {
        if (!sim) throw Error(ALIEN_B200_ERR_INVALID_ARGUMENT, "null handle");
        sim->arena->calcTimesteps(timesteps);
    });
}

int alien_b200_enqueue_timesteps(alien_b200_simulation* sim, uint64_t timesteps)
{
    return guarded([&] {
        if (!sim) throw Error(ALIEN_B200_ERR_INVALID_ARGUMENT, "null handle");
        sim->arena->enqueueSteps(timesteps);
    });
}

void* alien_b200_stream(alien_b200_simulation* sim) { return sim ? static_cast<void*>(sim->stream) : nullptr; }

int alien_b200_time_timesteps(alien_b200_simulation* sim, uint64_t timesteps, double* milliseconds)
{
    return guarded([&] {
        if (!sim || !milliseconds) throw Error(ALIEN_B200_ERR_INVALID_ARGUMENT, "null argument");
        *milliseconds = sim->arena->timeSteps(timesteps);
    });
}

thread_local std::vector<std::string> g_timedNames;

const char* alien_b200_step_kernel_name(int index)
{
    return index >= 0 && index < static_cast<int>(g_timedNames.size()) ? g_timedNames[index].c_str() : nullptr;
}

static int timedInto(Arena& a, uint64_t timesteps, double* kernelMs, int maxKernels, int* numKernels)
{
    std::vector<double> sums = a.timedSteps(timesteps);
    g_timedNames = a.lastTimedNames;
    const int n = static_cast<int>(sums.size());
    if (numKernels) *numKernels = n;
    for (int k = 0; k < n && k < maxKernels; ++k) kernelMs[k] = sums[k];
    return n;
}

int alien_b200_timed_timesteps(alien_b200_simulation* sim, uint64_t timesteps, double* kernelMs, int maxKernels, int* numKernels)
{
    return guarded([&] {
        if (!sim || (!kernelMs && maxKernels > 0)) throw Error(ALIEN_B200_ERR_INVALID_ARGUMENT, "null argument");
        timedInto(*sim->arena, timesteps, kernelMs, maxKernels, numKernels);
    });
}

uint64_t alien_b200_kernel_launch_count(alien_b200_simulation* sim) { return sim && sim->arena ? sim->arena->launches() : 0; }

int alien_b200_set_data(alien_b200_simulation* sim, const AlienDataTO* data)
{
    return guarded([&] {
        if (!sim) throw Error(ALIEN_B200_ERR_INVALID_ARGUMENT, "null handle");
        checkDataTO(data);
        const uint64_t t = sim->arena->readCounters()[0].timestep;
        WorldSetup ws = setupFrom(sim->general, sim->arena->params(0), t, data);
        ws.extraParticles = sim->extraParticles;
        sim->arena->build({ws});
    });
}

int alien_b200_get_data(alien_b200_simulation* sim, AlienInt2 upperLeft, AlienInt2 lowerRight, const AlienDataTO* data)
{
    return guarded([&] {
        if (!sim) throw Error(ALIEN_B200_ERR_INVALID_ARGUMENT, "null handle");
        sim->arena->getData(0, true, upperLeft, lowerRight, data);
    });
}

int alien_b200_set_parameters(alien_b200_simulation* sim, const AlienPhysicsParams* params)
{
    return guarded([&] {
        if (!sim || !params) throw Error(ALIEN_B200_ERR_INVALID_ARGUMENT, "null argument");
        sim->arena->setParams(0, *params);
        sim->params = *params;
    });
}

int alien_b200_get_parameters(alien_b200_simulation* sim, AlienPhysicsParams* params)
{
    return guarded([&] {
        if (!sim || !params) throw Error(ALIEN_B200_ERR_INVALID_ARGUMENT, "null argument");
        *params = sim->arena->params(0);
    });
}

int alien_b200_get_array_sizes(alien_b200_simulation* sim, AlienArraySizes* sizes)
{
    return guarded([&] {
        if (!sim || !sizes) throw Error(ALIEN_B200_ERR_INVALID_ARGUMENT, "null argument");
        const WorldInfo& wi = sim->arena->world(0).info;
        sizes->cellArraySize = static_cast<uint64_t>(wi.cellCap);
        sizes->particleArraySize = static_cast<uint64_t>(wi.partCap);
        sizes->auxiliaryDataSize = sim->arena->world(0).auxSize;
    });
}

int alien_b200_resize_arrays_if_necessary(alien_b200_simulation* sim, const AlienArraySizes* additionals)
{
    return guarded([&] {
        if (!sim || !additionals) throw Error(ALIEN_B200_ERR_INVALID_ARGUMENT, "null argument");
        // cells enter only through set_data, which sizes the arrays itself;
        // particle headroom is kept for the next set_data and applied now
        sim->extraParticles = std::max<uint64_t>(sim->extraParticles, additionals->particleArraySize);
        const WorldInfo& wi = sim->arena->world(0).info;
        uint64_t nc = 0, np = 0;
        sim->arena->countData(0, &nc, &np);
        if (np + additionals->particleArraySize + 4096 > static_cast<uint64_t>(wi.partCap) / 2)
            sim->arena->growParticles(0, sim->extraParticles);
    });
}

int alien_b200_get_current_timestep(alien_b200_simulation* sim, uint64_t* timestep)
{
    return guarded([&] {
        if (!sim || !timestep) throw Error(ALIEN_B200_ERR_INVALID_ARGUMENT, "null argument");
        *timestep = sim->arena->readCounters()[0].timestep;
    });
}

int alien_b200_set_current_timestep(alien_b200_simulation* sim, uint64_t timestep)
{
    return guarded([&] {
        if (!sim) throw Error(ALIEN_B200_ERR_INVALID_ARGUMENT, "null handle");
        sim->arena->setTimestep(0, timestep);
    });
}

int alien_b200_clear(alien_b200_simulation* sim)
{
    return guarded([&] {
        if (!sim) throw Error(ALIEN_B200_ERR_INVALID_ARGUMENT, "null handle");
        const uint64_t t = sim->arena->readCounters()[0].timestep;
        sim->arena->build({setupFrom(sim->general, sim->arena->params(0), t, nullptr)});
    });
}

int alien_b200_get_raw_statistics(alien_b200_simulation* sim, AlienRawStatistics* statistics)
{
    return guarded([&] {
        if (!sim || !statistics) throw Error(ALIEN_B200_ERR_INVALID_ARGUMENT, "null argument");
        *statistics = sim->arena->statistics(0);
    });
}

int alien_b200_debug_cell_map(alien_b200_simulation* sim, uint64_t capacity, uint64_t* ids, uint32_t* slots, uint32_t* tiles,
                              uint8_t* flags, uint64_t* count)
{
    return guarded([&] {
        if (!sim || !count || (capacity && (!ids || !slots || !tiles || !flags)))
            throw Error(ALIEN_B200_ERR_INVALID_ARGUMENT, "null argument");
        *count = sim->arena->cellMap(capacity, ids, slots, tiles, flags);
        if (*count > capacity)
            throw Error(ALIEN_B200_ERR_CAPACITY, "cell map holds " + std::to_string(*count) + " cells, capacity "
                                                     + std::to_string(capacity));
    });
}

int alien_b200_choose_region(const float* milliseconds, int n)
{
    // the fastest candidate; a later one must beat the best earlier one by
    // more than 2 % (timing noise must not flip the choice between nearly
    // equal shapes, and the first candidate is the default)
    int best = -1;
    for (int i = 0; i < n && i < kNumRegionChoices; ++i) {
        if (!(milliseconds[i] > 0.0f)) continue;
        if (best < 0 || milliseconds[i] < 0.98f * milliseconds[best]) best = i;
    }
    return best < 0 ? 0 : best;
}

int alien_b200_set_launch_config(alien_b200_simulation* sim, const AlienLaunchConfig* config)
{
    return guarded([&] {
        if (!sim || !config) throw Error(ALIEN_B200_ERR_INVALID_ARGUMENT, "null argument");
        for (int m = 0; m < 2; ++m) sim->arena->setRegionChoice(m, config->regionChoiceFixed[m]);
    });
}

int alien_b200_get_launch_config(alien_b200_simulation* sim, AlienLaunchConfig* config)
{
    return guarded([&] {
        if (!sim || !config) throw Error(ALIEN_B200_ERR_INVALID_ARGUMENT, "null argument");
        *config = sim->arena->launchConfig();
    });
}

int alien_b200_get_raw_statistics_data(alien_b200_simulation* sim, AlienRawStatisticsData* statistics)
{
    return guarded([&] {
        if (!sim || !statistics) throw Error(ALIEN_B200_ERR_INVALID_ARGUMENT, "null argument");
        *statistics = sim->arena->statisticsData(0);
    });
}

int alien_b200_get_density_map(alien_b200_simulation* sim, AlienDensityMap* map)
{
    return guarded([&] {
        if (!sim || !map) throw Error(ALIEN_B200_ERR_INVALID_ARGUMENT, "null argument");
        sim->arena->densityMap(0, map);
    });
}

int alien_b200_reset_time_interval_statistics(alien_b200_simulation* sim)
{
    return guarded([&] {
        if (!sim) throw Error(ALIEN_B200_ERR_INVALID_ARGUMENT, "null handle");
        sim->arena->resetTimeIntervalStatistics(0);
    });
}

// ------------------------------------------------------------- batch -----
int alien_b200_batch_get_raw_statistics_data(alien_b200_batch* b, int world, AlienRawStatisticsData* statistics)
{
    return guarded([&] {
        if (!b || !statistics || !b->arena->resident(world))
            throw Error(ALIEN_B200_ERR_INVALID_ARGUMENT, "invalid world");
        *statistics = b->arena->statisticsData(world);
    });
}

int alien_b200_batch_reset_time_interval_statistics(alien_b200_batch* b, int world)
{
    return guarded([&] {
        if (!b || !b->arena->resident(world)) throw Error(ALIEN_B200_ERR_INVALID_ARGUMENT, "invalid world");
        b->arena->resetTimeIntervalStatistics(world);
    });
}

int alien_b200_batch_set_launch_config(alien_b200_batch* b, const AlienLaunchConfig* config)
{
    return guarded([&] {
        if (!b || !config) throw Error(ALIEN_B200_ERR_INVALID_ARGUMENT, "null argument");
        for (int m = 0; m < 2; ++m) b->arena->setRegionChoice(m, config->regionChoiceFixed[m]);
    });
}

int alien_b200_batch_get_launch_config(alien_b200_batch* b, AlienLaunchConfig* config)
{
    return guarded([&] {
        if (!b || !config) throw Error(ALIEN_B200_ERR_INVALID_ARGUMENT, "null argument");
        *config = b->arena->launchConfig();
    });
}

int alien_b200_arena_bytes(const AlienArenaCapacity* capacity, uint64_t* bytes)
{
    return guarded([&] {
        if (!capacity || !bytes) throw Error(ALIEN_B200_ERR_INVALID_ARGUMENT, "null argument");
        *bytes = Arena::reserveBytes(*capacity);
    });
}

int alien_b200_arena_create(const AlienArenaCapacity* capacity, alien_b200_batch** out)
{
    return guarded([&] {
        if (!capacity || !out) throw Error(ALIEN_B200_ERR_INVALID_ARGUMENT, "null argument");
        *out = nullptr;
        ensureDevice();
        auto b = std::make_unique<alien_b200_batch>();
        AB_CK(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
        b->arena = std::make_unique<Arena>(b->stream);
        b->arena->reserve(*capacity);
        *out = b.release();
    });
}

int alien_b200_world_admit(alien_b200_batch* b, const AlienGeneralSettings* general, const AlienPhysicsParams* params,
                           const AlienDataTO* data, uint64_t timestep, uint64_t steps, int* world)
{
    return guarded([&] {
        if (!b || !general || !params || !data || !world) throw Error(ALIEN_B200_ERR_INVALID_ARGUMENT, "null argument");
        if (!b->arena->live()) throw Error(ALIEN_B200_ERR_INVALID_ARGUMENT, "not a live arena (alien_b200_arena_create)");
        checkDataTO(data);
        *world = -1;
        *world = b->arena->admit(setupFrom(*general, *params, timestep, data), steps);
    });
}

int alien_b200_world_evict(alien_b200_batch* b, int world)
{
    return guarded([&] {
        if (!b) throw Error(ALIEN_B200_ERR_INVALID_ARGUMENT, "null handle");
        b->arena->evict(world);
    });
}

int alien_b200_arena_num_resident(alien_b200_batch* b) { return b && b->arena ? b->arena->residentWorlds() : -1; }

int alien_b200_batch_create(int numWorlds, const AlienGeneralSettings* general, const AlienPhysicsParams* params,
                            const AlienDataTO* data, uint64_t timestep, alien_b200_batch** out)
{
    return guarded([&] {
        if (numWorlds <= 0 || numWorlds > 65535 || !general || !params || !data || !out)
            throw Error(ALIEN_B200_ERR_INVALID_ARGUMENT, "invalid batch arguments");
        *out = nullptr;
        ensureDevice();
        std::vector<WorldSetup> setups;
        for (int w = 0; w < numWorlds; ++w) {
            checkDataTO(&data[w]);
            setups.push_back(setupFrom(general[w], params[w], timestep, &data[w]));
        }
        auto b = std::make_unique<alien_b200_batch>();
        AB_CK(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
        b->arena = std::make_unique<Arena>(b->stream);
        b->arena->build(setups);
        *out = b.release();
    });
}

int alien_b200_batch_destroy(alien_b200_batch* b)
{
    return guarded([&] {
        if (!b) return;
        if (b->stream) cudaStreamSynchronize(b->stream);
        b->arena.reset();
        if (b->stream) cudaStreamDestroy(b->stream);
        delete b;
    });
}

int alien_b200_batch_num_worlds(alien_b200_batch* b) { return b && b->arena ? b->arena->numWorlds() : 0; }

int alien_b200_batch_calc_timesteps(alien_b200_batch* b, uint64_t timesteps)
{
    return guarded([&] {
        if (!b) throw Error(ALIEN_B200_ERR_INVALID_ARGUMENT, "null handle");
        b->arena->calcTimesteps(timesteps);
    });
}

int alien_b200_batch_enqueue_timesteps(alien_b200_batch* b, uint64_t timesteps)
{
    return guarded([&] {
        if (!b) throw Error(ALIEN_B200_ERR_INVALID_ARGUMENT, "null handle");
        b->arena->enqueueSteps(timesteps);
    });
}

int alien_b200_batch_synchronize(alien_b200_batch* b)
{
    return guarded([&] {
        if (!b) throw Error(ALIEN_B200_ERR_INVALID_ARGUMENT, "null handle");
        b->arena->sync();
        b->arena->ensureParticleCapacity();
    });
}

int alien_b200_batch_get_data(alien_b200_batch* b, int world, const AlienDataTO* data)
{
    return guarded([&] {
        if (!b || !b->arena->resident(world)) throw Error(ALIEN_B200_ERR_INVALID_ARGUMENT, "invalid world");
        b->arena->getData(world, false, AlienInt2{0, 0}, AlienInt2{0, 0}, data);
    });
}

int alien_b200_batch_get_array_sizes(alien_b200_batch* b, int world, AlienArraySizes* sizes)
{
    return guarded([&] {
        if (!b || !sizes || !b->arena->resident(world)) throw Error(ALIEN_B200_ERR_INVALID_ARGUMENT, "invalid world");
        const WorldInfo& wi = b->arena->world(world).info;
        sizes->cellArraySize = static_cast<uint64_t>(wi.cellCap);
        sizes->particleArraySize = static_cast<uint64_t>(wi.partCap);
        sizes->auxiliaryDataSize = b->arena->world(world).auxSize;
    });
}

int alien_b200_batch_set_step_budget(alien_b200_batch* b, int world, uint64_t steps)
{
    return guarded([&] {
        if (!b || !b->arena->resident(world)) throw Error(ALIEN_B200_ERR_INVALID_ARGUMENT, "invalid world");
        b->arena->setStepBudget(world, steps);
    });
}

int alien_b200_batch_world_status(alien_b200_batch* b, int world, uint64_t* timestep, uint64_t* stepsRemaining, int* active)
{
    return guarded([&] {
        if (!b || !b->arena->resident(world)) throw Error(ALIEN_B200_ERR_INVALID_ARGUMENT, "invalid world");
        b->arena->settle();
        std::vector<WorldCounters> c = b->arena->readCounters();
        if (timestep) *timestep = c[world].timestep;
        if (stepsRemaining) *stepsRemaining = c[world].stepsRemaining == ~0ull ? 0 : c[world].stepsRemaining;
        if (active) *active = static_cast<int>(c[world].active);
    });
}

int alien_b200_batch_num_active(alien_b200_batch* b)
{
    if (!b || !b->arena) return -1;
    try {
        b->arena->settle();
        std::vector<WorldCounters> c = b->arena->readCounters();
        int n = 0;
        for (const WorldCounters& x : c) n += x.active ? 1 : 0;
        return n;
    } catch (...) {
        return -1;
    }
}

uint64_t alien_b200_batch_device_bytes(alien_b200_batch* b) { return b && b->arena ? b->arena->deviceBytes() : 0; }

int alien_b200_batch_get_raw_statistics(alien_b200_batch* b, int world, AlienRawStatistics* statistics)
{
    return guarded([&] {
        if (!b || !statistics || !b->arena->resident(world))
            throw Error(ALIEN_B200_ERR_INVALID_ARGUMENT, "invalid world");
        *statistics = b->arena->statistics(world);
    });
}

int alien_b200_batch_get_density_map(alien_b200_batch* b, int world, AlienDensityMap* map)
{
    return guarded([&] {
        if (!b || !map || !b->arena->resident(world)) throw Error(ALIEN_B200_ERR_INVALID_ARGUMENT, "invalid world");
        b->arena->densityMap(world, map);
    });
}

void* alien_b200_batch_stream(alien_b200_batch* b) { return b ? static_cast<void*>(b->stream) : nullptr; }

uint64_t alien_b200_batch_kernel_launch_count(alien_b200_batch* b) { return b && b->arena ? b->arena->launches() : 0; }

int alien_b200_batch_kernels_per_step(alien_b200_batch* b) { return b && b->arena ? b->arena->kernelsPerStep() : 0; }

int alien_b200_batch_time_timesteps(alien_b200_batch* b, uint64_t timesteps, double* milliseconds)
{
    return guarded([&] {
        if (!b || !milliseconds) throw Error(ALIEN_B200_ERR_INVALID_ARGUMENT, "null argument");
        *milliseconds = b->arena->timeSteps(timesteps);
    });
}

int alien_b200_batch_timed_timesteps(alien_b200_batch* b, uint64_t timesteps, double* kernelMs, int maxKernels, int* numKernels)
{
    return guarded([&] {
        if (!b || (!kernelMs && maxKernels > 0)) throw Error(ALIEN_B200_ERR_INVALID_ARGUMENT, "null argument");
        timedInto(*b->arena, timesteps, kernelMs, maxKernels, numKernels);
    });
}

}  // extern "C"
