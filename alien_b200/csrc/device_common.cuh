// device_common.cuh - device-side state layout and helpers of the B200 engine.
//
// State is structure-of-arrays in HBM.  All worlds of an arena share one set
// of arrays: world w owns the cell slots [cellBase, cellBase + cellCap) and
// the particle slots [partBase, partBase + partCap), both padded to whole
// 256-slot blocks so that every block of a per-object kernel belongs to one
// world (cellBlockWorld / partBlockWorld).  Deleted objects stay as
// tombstones (alive == 0) until a stable compaction; storage order is
// ingest order, new particles are appended.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/alien_b200.h"

namespace ab {

constexpr int kBlock = 256;           // threads per block of per-object kernels
constexpr int kCellFunctionNeuron = 0;  // CellFunction_Neuron, CellFunctionConstants.h:8
constexpr int kCellFunctionNone = 11;   // CellFunction_None, CellFunctionConstants.h:21
constexpr int kMaxBonds = 6;          // MAX_CELL_BONDS, EngineConstants.h:3
constexpr int kSlotScanLevels = 10;   // Map.cuh:117, CellProcessor.cuh:165
constexpr float kNearZero = 1.0e-4f;  // Base/Definitions.h:27
constexpr float kPi = 3.1415926535897932384626433832795f;
constexpr float kFixScale = 4294967296.0f;  // 2^32: fixed-point force/energy sums
constexpr double kFixInv = 1.0 / 4294967296.0;

// per-cell step flags (32-bit so that partners can set them with atomicOr)
enum : uint32_t {
    kFlagDelAll = 1u,          // delete all bonds that existed before this step's additions
    kFlagDelCell = 2u,         // cell is deleted at the end of the step
    kFlagDetach = 4u,          // a partner's bond overstretched (checkConnections)
    kFlagSetDying = 8u,        // decay: cell becomes Dying
    kFlagNewDying = 16u,       // ... and was not Dying before
    kFlagDetachFromDying = 32u,  // a newly dying partner detaches this cell
    kFlagRadiation = 64u,      // cell emits a radiation particle this step
};

// staged per-cell record flags (int4.y)
enum : int {
    kStageBarrier = 1,
    kStageVisible = 2,   // among the first kSlotScanLevels cells of its slot
    kStageHead = 4,      // first cell of its slot (CellMap::getFirst)
};

// counter-based random draw sites
enum : uint32_t {
    kSiteForceDecay = 1, kSiteRadiation = 2, kSiteRadiationEnergy = 3, kSiteRadiationAngle = 4,
    kSiteDeath = 5, kSiteSplit = 6, kSiteSplitAngle = 7,
};

struct WorldInfo {
    int W, H;             // world size in slots
    int T;                // tile side in slots (= scan radius, >= 1)
    int nTX, nTY;         // tile grid
    int radiusInt;        // scan radius in slots
    int motionType;
    int paramIndex;
    long long tileBase;   // first tile of this world in the arena's tile arrays
    long long cellBase, cellCap;
    long long partBase, partCap;
    long long pmapBase;   // first slot of this world's particle map
    int firstCellBlock, numCellBlocks;
    int firstPartBlock, numPartBlocks;
    // pair-phase regions: regW x regH tiles per CTA, nRX x nRY regions,
    // first CTA regionBase; regionShared = 0 for worlds too small for them
    int regW, regH, nRX, nRY, regionBase, regionShared;
    long long auxBase;  // offset of the world's auxiliary data in DevState::aux
};

struct WorldCounters {
    unsigned long long timestep;
    unsigned long long nextId;
    unsigned int numCells;        // used cell slots (live + tombstones)
    unsigned int numParticles;    // used particle slots (live + tombstones)
    unsigned int deadCells;
    unsigned int deadParticles;
    unsigned int droppedParticles;  // appends refused for lack of capacity
    // 1: no larger particle range could be had; the world's steps drop what
    // does not fit instead of halting (until the next capacity check)
    unsigned int dropExcess;
    // event bases of the current step (ids and slots of appended particles)
    unsigned long long radIdBase, splitIdBase, delIdBase;
    unsigned int radSlotBase, splitSlotBase, delSlotBase, numEvents;
    // a world steps while active; stepsRemaining counts down to 0 and then
    // clears active (~0 = no limit)
    unsigned long long stepsRemaining;
    unsigned int active;
    // 1 while the world waits for particle storage: its step stopped before
    // the new particles were written (kEventWorld), nothing of the world
    // changes until the host has grown its range and completed the step
    unsigned int halted;
    // events counted this step (radiation, deleted cells, particle splits):
    // the event scans run only when there are any
    unsigned int evRad, evDel, evSplit;
    // set at ingest: the next step clears the signals of cells without
    // function (after that no step writes them)
    unsigned int signalsFresh;
    // the external energy pool and this step's backflow into it (2^-24 fixed
    // point, added to the pool at the end of the step)
    double externalEnergy;
    long long backflowFix;
    // radiation sources active in this step (bit i: source i)
    unsigned long long activeSources;
    // the timestep a completed step left (zones and sources move once per step)
    unsigned long long lastStepped;
    // steps the world would have taken while halted (within its budget):
    // the host runs them after it completes the halted step
    unsigned long long missedSteps;
};

// bits of DevState::errorFlags
constexpr unsigned int kErrDropped = 1u;  // particles dropped for lack of storage
constexpr unsigned int kErrHalted = 8u;   // a world halted for storage (WorldCounters::halted)

struct DevState {
    int numWorlds;
    int numCellBlocks, numPartBlocks;
    long long cellSlots, partSlots;
    long long numTiles;
    const WorldInfo* worlds;
    WorldCounters* counters;
    AlienPhysicsParams* params;  // zone and source positions move with the steps
    const int* cellBlockWorld;
    const int* partBlockWorld;
    const int* regionWorld;  // world of each pair-phase CTA
    int numRegions;
    unsigned int* errorFlags;
    // 1 in the launches that complete halted steps (kEventWorld, kEventEmit,
    // kWorldsEnd): only halted worlds take part, and what does not fit is
    // dropped instead of halting again
    int resume;

    // cells
    unsigned long long* id;
    float2* posA;     // position at the start of the step (FP32 state between steps)
    float2* push;     // overlap push of the pair phase (displacement before the Verlet update)
    float2* dpos;     // displacement since the step start after the Verlet update (push plus
                      // the Verlet increment); folded into posA by the next step's binning
    float2* velA;
    float2* velB;
    float* energy;
    float* stiffness;
    float* density;
    float* densNew;
    uint8_t* color;
    uint8_t* maxConn;
    uint8_t* numConn;
    uint8_t* barrier;
    uint8_t* alive;
    uint8_t* triMask;         // per cell, angle-force steps: bit k = bond k's partner is bonded to the previous partner
    uint8_t* livingState;
    uint8_t* nextState;
    uint32_t* flags;
    uint32_t* age;
    uint32_t* activationTime;
    uint32_t* creatureId;
    uint32_t* coldIdx;
    AlienCellTO* cold;        // ingest copies (signals and cellFunctionUsed of neuron cells change here)
    uchar4* fnInfo;           // per cell: (function: 0 none / 1 neuron, execution order, input order as int8, output
                              // blocked); null when no cell has a function or a signal
    const uint8_t* aux;       // the worlds' auxiliary data (world w at worlds[w].auxBase); null without neurons
    int* bond;          // [slot * 6 + k] partner slot
    float* bondDist;
    float* bondAngle;
    float2* force;      // pair force, then bond force #2 (own part)
    float2* force1;     // bond force #1 (total)
    long long* angleAcc;  // [slot * 4]: scattered angle forces, pass 1 (x,y), pass 2 (x,y)
    long long* energyAcc; // absorbed particle energy
    int* best;          // fusion choice (partner slot) or -1
    int* newPartner;    // partner slot of the bond added this step or -1
    // pair-add scratch (written for paired cells only)
    uint8_t* addNum;
    int* addBond;
    float* addDist;
    float* addAngle;
    // radiation emission scratch
    float2* radPos;
    float2* radVel;
    float* radEnergy;

    // tiles
    uint32_t* tileOf;
    uint32_t* slotOf;      // slot (x + y * W) of the cell at binning
    uint32_t* tileOff;
    uint32_t* tileCount;
    uint32_t* tileStart;   // numTiles + 1 entries (exclusive scan of tileCount)
    uint32_t* sorted;      // cell slots grouped by tile
    uint8_t* slotInTile;   // per cell: its slot within its tile at binning
    uint8_t* sortedSlot;   // beside sorted: the listed cell's slot within the tile
    uint32_t* pairOverflow;       // staged indices of cells the pair regions defer to kPairsOverflow
    uint32_t* pairOverflowCount;  // = tileCount + numTiles: cleared with the tile counts every step
    float4* stagedPV;      // (pos.x, pos.y, vel.x, vel.y) in sorted order
    int4* stagedMeta;      // (cell slot, flags | world << 16, density bits, energy bits)

    // particles
    unsigned long long* pid;
    float2* ppos;
    float2* pvel;
    float* penergy;
    uint8_t* pcolor;
    uint8_t* palive;
    uint8_t* pselected;
    uint32_t* pflag;      // bit0 incoming merge, bit1 split emission
    unsigned long long* plast;  // id of the last absorbing cell, ~0 = none
    int* ptarget;
    int* pslot;
    long long* pmerge;    // [slot * 3]: merged energy, momentum x, momentum y
    float2* splitPos;
    float2* splitVel;
    float* splitEnergy;
    int* pmap;            // per-world dense particle maps (-1 = empty)

    // accumulated statistics, per world and color: neuron cells that ran
    unsigned long long* neuronActivity;

    // rigidity clusters (allocated when some world enables rigidity)
    int* clusterLab[2];         // cluster labels, two buffers of the propagation rounds
    uint32_t* clusterCount;     // per cluster: cells
    long long* clusterAcc;      // [cluster * 6]: velocity, offset from the label cell, angular mass and
                                // momentum (fixed point)
    uint32_t* clusterChanged;   // per propagation round: some label changed

    // event scan scratch (per block)
    uint32_t* blockRad;
    uint32_t* blockDel;
    uint32_t* blockSplit;

    // scan scratch
    uint32_t* scanPartials;
};

// ---------------------------------------------------------------- math ----

__device__ __forceinline__ float2 f2(float x, float y) { return make_float2(x, y); }
__device__ __forceinline__ float2 operator+(float2 a, float2 b) { return f2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 operator-(float2 a, float2 b) { return f2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 operator*(float2 a, float m) { return f2(a.x * m, a.y * m); }
__device__ __forceinline__ float2 operator/(float2 a, float m) { return f2(a.x / m, a.y / m); }
__device__ __forceinline__ float dot2(float2 a, float2 b) { return a.x * b.x + a.y * b.y; }
__device__ __forceinline__ float len2(float2 a) { return sqrtf(a.x * a.x + a.y * a.y); }
__device__ __forceinline__ float lensq2(float2 a) { return a.x * a.x + a.y * a.y; }

// Math::normalized, Math.cuh:246-261
__device__ __forceinline__ float2 normalized2(float2 a)
{
    float l = len2(a);
    if (l > kNearZero) return f2(a.x / l, a.y / l);
    return f2(1.0f, 0.0f);
}
// Math::rotateQuarterClockwise / CounterClockwise, Math.cuh:157-169
__device__ __forceinline__ float2 rotCW(float2 a) { return f2(-a.y, a.x); }
__device__ __forceinline__ float2 rotCCW(float2 a) { return f2(a.y, -a.x); }

// Math::angleOfVector, Math.cuh:140-155 (degrees clockwise from (0,-1)).
// The reference evaluates 90 - asin(-v.y/|v|) (v.x >= 0) or asin(..) + 270;
// both branches equal 90 - atan2(-v.y, v.x) taken mod 360, which is evaluated
// here because asin loses ~sqrt(eps) radians for near-vertical vectors.
__device__ __forceinline__ float angleOfVector(float2 v)
{
    float l = len2(v);
    if (l < kNearZero) return 0.0f;
    float a = 90.0f - atan2f(-v.y, v.x) * (180.0f / kPi);
    return a < 0.0f ? a + 360.0f : a;
}
// Math::unitVectorOfAngle, Math.cuh:134-138
__device__ __forceinline__ float2 unitVectorOfAngle(float a)
{
    a *= kPi / 180.0f;
    return f2(sinf(a), -cosf(a));
}
// Math::subtractAngle, Math.cuh:300-310
__device__ __forceinline__ float subtractAngle(float a, float b)
{
    float d = a - b;
    if (d > 360.0f) d -= 360.0f;
    if (d < 0.0f) d += 360.0f;
    return d;
}
// Math::isAngleInBetween, Math.cuh:223-236
__device__ __forceinline__ bool isAngleInBetween(float a1, float a2, float c)
{
    if (a1 == a2 && a1 != c) return false;
    if (c < a1) {
        c += 360.0f;
        a2 += 360.0f;
    }
    if (a2 < c) a2 += 360.0f;
    return a2 - a1 < 360.0f;
}
// Math::crossing, Math.cuh:363-395
__device__ inline bool crossing(float2 s, float2 e, float2 os, float2 oe)
{
    if ((s.x == os.x && s.y == os.y) || (s.x == oe.x && s.y == oe.y) || (e.x == os.x && e.y == os.y)
        || (e.x == oe.x && e.y == oe.y))
        return false;
    float2 v1 = e - s, v2 = oe - os;
    float divisor = v2.x * v1.y - v2.y * v1.x;
    if (fabsf(divisor) < kNearZero) return false;
    float mue = (v1.x * (os.y - s.y) - v1.y * (os.x - s.x)) / divisor;
    if (mue < -kNearZero || mue > 1 + kNearZero) return false;
    float lambda;
    if (fabsf(v1.x) > kNearZero)
        lambda = (os.x - s.x + mue * v2.x) / v1.x;
    else if (fabsf(v1.y) > kNearZero)
        lambda = (os.y - s.y + mue * v2.y) / v1.y;
    else
        return false;
    return lambda >= kNearZero && lambda <= 1 - kNearZero;
}

// floorInt, Base.cuh:83-90
__device__ __forceinline__ int floorInt(float v)
{
    int r = static_cast<int>(v);
    if (r > v) --r;
    return r;
}
__device__ __noinline__ int wrapIntOutside(int v, int size) { return ((v % size) + size) % size; }
__device__ __forceinline__ int wrapInt(int v, int size)
{
    if (static_cast<unsigned>(v) < static_cast<unsigned>(size)) return v;  // the usual case: already inside
    return wrapIntOutside(v, size);
}

// BaseMap::correctPosition(float2&), Map.cuh:20-26
__device__ __forceinline__ float2 correctPosition(float2 p, int W, int H)
{
    int ix = floorInt(p.x), iy = floorInt(p.y);
    float fx = p.x - static_cast<float>(ix), fy = p.y - static_cast<float>(iy);
    ix = wrapInt(ix, W);
    iy = wrapInt(iy, H);
    return f2(static_cast<float>(ix) + fx, static_cast<float>(iy) + fy);
}

// IEEE remainder(x, size) (BaseMap::correctDirection, Map.cuh:35-39).  For
// |x| < 1.5*size the quotient rounds to -1, 0 or 1 and x -/+ size is exact
// (Sterbenz), so the branch form below equals remainderf bit for bit; other
// inputs take remainderf itself.
__device__ __forceinline__ float wrapDelta(float x, float size)
{
    float ax = fabsf(x);
    if (ax <= 0.5f * size) return x;
    if (ax < 1.5f * size) return x > 0.0f ? x - size : x + size;
    return remainderf(x, size);
}
__device__ __forceinline__ float2 correctDirection(float2 d, int W, int H)
{
    return f2(wrapDelta(d.x, static_cast<float>(W)), wrapDelta(d.y, static_cast<float>(H)));
}
__device__ __forceinline__ int slotX(float x, int W) { return wrapInt(floorInt(x), W); }

// b - a on a torus of the given size for coordinates in [0, size): the
// minimal-image difference that BaseMap::correctDirection gives, computed
// without rounding at the world's scale.  Across the seam the large
// coordinate is brought down by the size first (x - size is exact for x in
// [size/2, size)), so the result carries only the rounding of a small
// difference, as for two cells away from the seam (where b - a is exact).
__device__ __forceinline__ float seamDiff(float b, float a, float size)
{
    const float d = b - a;
    if (d > 0.5f * size) return (b - size) - a;
    if (d < -0.5f * size) return b - (a - size);
    return d;
}
__device__ __forceinline__ float2 seamDiff2(float2 b, float2 a, int W, int H)
{
    return f2(seamDiff(b.x, a.x, static_cast<float>(W)), seamDiff(b.y, a.y, static_cast<float>(H)));
}

// counter-based draw: SplitMix64 finaliser (Steele, Lea & Flood, OOPSLA 2014)
// of (timestep, site), xor the object id, finalised again; 24 high bits.
__device__ __forceinline__ uint64_t splitmix64(uint64_t z)
{
    z += 0x9e3779b97f4a7c15ULL;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}
__device__ __forceinline__ float draw(uint64_t id, uint64_t step, uint32_t site)
{
    uint64_t h = splitmix64(splitmix64(step ^ (static_cast<uint64_t>(site) << 56)) ^ id);
    return static_cast<float>(h >> 40) * (1.0f / 16777216.0f);
}

// fixed-point (2^-32) accumulation: integer sums do not depend on order
__device__ __forceinline__ long long toFix(float v) { return __float2ll_rn(v * kFixScale); }
__device__ __forceinline__ float fromFix(long long q) { return static_cast<float>(static_cast<double>(q) * kFixInv); }

// calcKernel / calcKernel_d, CellProcessor.cuh:92-119
__device__ __forceinline__ float sphKernel(float q)
{
    float r;
    if (q < 1.0f)
        r = 2.0f / 3.0f - q * q + 0.5f * q * q * q;
    else if (q < 2.0f) {
        r = 2.0f - q;
        r = r * r * r / 6.0f;
    } else
        r = 0.0f;
    return r * (3.0f / (2.0f * kPi));
}
__device__ __forceinline__ float sphKernelD(float q)
{
    float r;
    if (q < 1.0f)
        r = -2.0f * q + 3.0f / 2.0f * q * q;
    else if (q < 2.0f)
        r = -0.5f * (2.0f - q) * (2.0f - q);
    else
        r = 0.0f;
    return r * (3.0f / (2.0f * kPi));
}

// exclusive scan across a block of Threads threads (a multiple of 32);
// *total = block sum
template <int Threads>
__device__ __forceinline__ uint32_t blockExclusiveScanN(uint32_t v, uint32_t* total)
{
    static_assert(Threads % 32 == 0 && Threads <= 1024, "block size");
    __shared__ uint32_t warpSums[Threads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warpSums[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t ws = lane < Threads / 32 ? warpSums[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, ws, o);
            if (lane >= o) ws += y;
        }
        if (lane < Threads / 32) warpSums[lane] = ws;
    }
    __syncthreads();
    uint32_t warpOffset = warp > 0 ? warpSums[warp - 1] : 0;
    if (total) *total = warpSums[Threads / 32 - 1];
    uint32_t r = warpOffset + x - v;
    __syncthreads();
    return r;
}

// exclusive scan across a block of kBlock threads; *total = block sum
__device__ __forceinline__ uint32_t blockExclusiveScan(uint32_t v, uint32_t* total)
{
    return blockExclusiveScanN<kBlock>(v, total);
}

__device__ __forceinline__ void setError(const DevState& s, uint32_t bit) { atomicOr(s.errorFlags, bit); }

// Positions within a step are the step-start position posA (exact FP32
// state) plus the small displacement dpos accumulated by the step, so that
// bond lengths and angles after the Verlet update are computed from exact
// start differences and small increments instead of from positions rounded
// at the world's scale (ulp 2.4e-4 at 4096).  The position a step produces
// is rounded once, when the next step's binning (or an egress) folds dpos
// into posA.
__device__ __forceinline__ float2 stepPos(const DevState& s, long long g, int W, int H)
{
    return correctPosition(s.posA[g] + s.dpos[g], W, H);
}
// displacement from cell a to cell b at the step's current positions
__device__ __forceinline__ float2 stepDisp(const DevState& s, long long a, long long b, int W, int H)
{
    return seamDiff2(s.posA[b], s.posA[a], W, H) + (s.dpos[b] - s.dpos[a]);
}

}  // namespace ab
