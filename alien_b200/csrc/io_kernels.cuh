// io_kernels.cuh - data transfer between the reference's DataTO format and
// the engine's SoA state, statistics, and stable particle compaction.
//
// Ingest restates cudaCreateDataFromTO / ObjectFactory::createCellFromTO
// (source/EngineGpuKernels/DataAccessKernels.cu:363-387,
// ObjectFactory.cuh:46-86); egress restates cudaGetCellDataWithoutConnections
// + cudaResolveConnections + cudaGetParticleData (DataAccessKernels.cu
// :312-362) with a stable, rank-based order instead of atomic slots.  All
// kernels here work on one world w; their grid covers the world's padded
// slot range block by block.
#pragma once

#include "device_common.cuh"

namespace ab {

// ---- ingest ----
// Checks of the transfer objects, run on the uploaded copy before the arena
// changes: counts of cells with more than 6 bonds, bond indices outside the
// array, cell functions other than neuron / none, neuron data outside the
// auxiliary data, neurons and nonzero signal channels (block counts, one
// atomic per block and counter).
struct IngestCheck {
    unsigned int badBondCount, badBondIndex, otherFunction, neuronOutOfAux, neurons, nonzeroSignal;
};

__global__ void __launch_bounds__(kBlock) kCheckCells(const AlienCellTO* to, long long n, unsigned long long numAux,
                                                      IngestCheck* out)
{
    const long long i = static_cast<long long>(blockIdx.x) * kBlock + threadIdx.x;
    bool badCount = false, badIndex = false, other = false, outOfAux = false, neuron = false, signal = false;
    if (i < n) {
        const AlienCellTO& c = to[i];
        if (c.numConnections > kMaxBonds) {
            badCount = true;
        } else {
            for (int k = 0; k < c.numConnections; ++k) {
                const int idx = c.connections[k].cellIndex;
                if (idx < 0 || idx >= n) badIndex = true;
            }
        }
        if (c.cellFunction == kCellFunctionNeuron) {
            neuron = true;
            const unsigned long long at = c.cellFunctionData[0];
            const unsigned long long bytes = sizeof(float) * ALIEN_B200_MAX_CHANNELS * (ALIEN_B200_MAX_CHANNELS + 1);
            outOfAux = at > numAux || numAux - at < bytes;
        } else if (c.cellFunction != kCellFunctionNone) {
            other = true;
        }
#pragma unroll
        for (int ch = 0; ch < ALIEN_B200_MAX_CHANNELS; ++ch) signal |= c.signal.channels[ch] != 0.0f;
    }
    const int nBadCount = __syncthreads_count(badCount), nBadIndex = __syncthreads_count(badIndex);
    const int nOther = __syncthreads_count(other), nOutOfAux = __syncthreads_count(outOfAux);
    const int nNeuron = __syncthreads_count(neuron), nSignal = __syncthreads_count(signal);
    if (threadIdx.x == 0) {
        if (nBadCount) atomicAdd(&out->badBondCount, static_cast<unsigned int>(nBadCount));
        if (nBadIndex) atomicAdd(&out->badBondIndex, static_cast<unsigned int>(nBadIndex));
        if (nOther) atomicAdd(&out->otherFunction, static_cast<unsigned int>(nOther));
        if (nOutOfAux) atomicAdd(&out->neuronOutOfAux, static_cast<unsigned int>(nOutOfAux));
        if (nNeuron) atomicAdd(&out->neurons, static_cast<unsigned int>(nNeuron));
        if (nSignal) atomicAdd(&out->nonzeroSignal, static_cast<unsigned int>(nSignal));
    }
}
__global__ void __launch_bounds__(kBlock) kIngestCells(DevState s, int w, const AlienCellTO* to, long long n, AlienCellTO* cold,
                                                       long long coldBase)
{
    const long long i = static_cast<long long>(blockIdx.x) * kBlock + threadIdx.x;
    if (i >= n) return;
    const WorldInfo& wi = s.worlds[w];
    const long long g = wi.cellBase + i;
    const AlienCellTO& c = to[i];
    // cold[coldBase + i] is a copy of to[i], made by one device-to-device copy
    s.coldIdx[g] = static_cast<uint32_t>(coldBase + i);
    s.id[g] = c.id;
    s.posA[g] = correctPosition(f2(c.pos.x, c.pos.y), wi.W, wi.H);
    s.dpos[g] = f2(0.0f, 0.0f);
    s.velA[g] = f2(c.vel.x, c.vel.y);
    s.energy[g] = c.energy;
    s.stiffness[g] = c.stiffness;
    s.density[g] = 1.0f;  // ObjectFactory.cuh:84
    s.color[g] = c.color;
    s.maxConn[g] = c.maxConnections;
    const int n6 = c.numConnections > kMaxBonds ? kMaxBonds : c.numConnections;
    s.numConn[g] = static_cast<uint8_t>(n6);
    s.barrier[g] = c.barrier ? 1 : 0;
    s.alive[g] = 1;
    s.livingState[g] = static_cast<uint8_t>(c.livingState);
    s.age[g] = c.age;
    s.activationTime[g] = c.activationTime;
    s.creatureId[g] = c.creatureId;
    if (s.fnInfo)
        s.fnInfo[g] = make_uchar4(c.cellFunction == kCellFunctionNeuron ? 1 : 0, c.executionOrderNumber,
                                  static_cast<uint8_t>(c.inputExecutionOrderNumber), c.outputBlocked ? 1 : 0);
    for (int k = 0; k < kMaxBonds; ++k) {
        const bool used = k < n6;
        s.bond[g * kMaxBonds + k] = used ? static_cast<int>(wi.cellBase + c.connections[k].cellIndex) : -1;
        s.bondDist[g * kMaxBonds + k] = c.connections[k].distance;
        s.bondAngle[g * kMaxBonds + k] = c.connections[k].angleFromPrevious;
    }
}

__global__ void __launch_bounds__(kBlock) kIngestParticles(DevState s, int w, const AlienParticleTO* to, long long n)
{
    const long long i = static_cast<long long>(blockIdx.x) * kBlock + threadIdx.x;
    if (i >= n) return;
    const WorldInfo& wi = s.worlds[w];
    const long long q = wi.partBase + i;
    const AlienParticleTO& p = to[i];
    s.pid[q] = p.id;
    s.ppos[q] = correctPosition(f2(p.pos.x, p.pos.y), wi.W, wi.H);
    s.pvel[q] = f2(p.vel.x, p.vel.y);
    s.penergy[q] = p.energy;
    s.pcolor[q] = p.color;
    s.pselected[q] = p.selected;
    s.palive[q] = 1;
    s.plast[q] = ~0ull;
}

// ids stay unique: the world's id counter continues after the largest id
// (cudaAdaptNumberGenerator, DataAccessKernels.cu:389-410)
__global__ void __launch_bounds__(kBlock) kMaxId(DevState s, int w, const AlienCellTO* cells, long long nc,
                                                 const AlienParticleTO* parts, long long np)
{
    __shared__ unsigned long long warpMax[kBlock / 32];
    const long long i = static_cast<long long>(blockIdx.x) * kBlock + threadIdx.x;
    unsigned long long m = 0;
    if (i < nc) m = cells[i].id + 1;
    if (i < np && parts[i].id + 1 > m) m = parts[i].id + 1;
    // block maximum first: one atomic per block instead of one per object
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long other = __shfl_down_sync(0xffffffffu, m, o);
        m = other > m ? other : m;
    }
    if ((threadIdx.x & 31) == 0) warpMax[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = 1; k < kBlock / 32; ++k) m = warpMax[k] > m ? warpMax[k] : m;
        if (m) atomicMax(&s.counters[w].nextId, m);
    }
}

// ---- selection + ranks (egress and compaction) ----
__device__ __forceinline__ bool inRect(float2 p, int ulx, int uly, int lrx, int lry)
{
    return p.x >= ulx && p.x <= lrx && p.y >= uly && p.y <= lry;  // isContainedInRect, Base.cuh:92-97
}

// rank[g] = 1 if the cell is selected (0 otherwise); blockCount = block sums
__global__ void __launch_bounds__(kBlock) kSelectCells(DevState s, int w, int useRect, int ulx, int uly, int lrx, int lry,
                                                       int* rank, uint32_t* blockCount)
{
    const WorldInfo& wi = s.worlds[w];
    const long long g = wi.cellBase + static_cast<long long>(blockIdx.x) * kBlock + threadIdx.x;
    uint32_t v = 0;
    if (g < wi.cellBase + s.counters[w].numCells && s.alive[g])
        v = (!useRect || inRect(stepPos(s, g, wi.W, wi.H), ulx, uly, lrx, lry)) ? 1u : 0u;
    uint32_t total;
    const uint32_t ex = blockExclusiveScan(v, &total);
    rank[g] = v ? static_cast<int>(ex) : -1;
    if (threadIdx.x == 0) blockCount[blockIdx.x] = total;
}

__global__ void __launch_bounds__(kBlock) kSelectParticles(DevState s, int w, int useRect, int ulx, int uly, int lrx, int lry,
                                                           int* rank, uint32_t* blockCount)
{
    const WorldInfo& wi = s.worlds[w];
    const long long q = wi.partBase + static_cast<long long>(blockIdx.x) * kBlock + threadIdx.x;
    uint32_t v = 0;
    if (q < wi.partBase + s.counters[w].numParticles && s.palive[q])
        v = (!useRect || inRect(s.ppos[q], ulx, uly, lrx, lry)) ? 1u : 0u;
    uint32_t total;
    const uint32_t ex = blockExclusiveScan(v, &total);
    rank[q] = v ? static_cast<int>(ex) : -1;
    if (threadIdx.x == 0) blockCount[blockIdx.x] = total;
}

// blockCount (exclusive scan, numBlocks + 1 entries) -> global ranks
__global__ void __launch_bounds__(kBlock) kFinishRanks(long long base, int* rank, const uint32_t* blockOffset)
{
    const long long i = base + static_cast<long long>(blockIdx.x) * kBlock + threadIdx.x;
    if (rank[i] >= 0) rank[i] += static_cast<int>(blockOffset[blockIdx.x]);
}

// ---- egress (createCellTO, DataAccessKernels.cu:18-110) ----
__global__ void __launch_bounds__(kBlock) kEgressCells(DevState s, int w, const int* rank, const AlienCellTO* cold, AlienCellTO* out)
{
    const WorldInfo& wi = s.worlds[w];
    const long long g = wi.cellBase + static_cast<long long>(blockIdx.x) * kBlock + threadIdx.x;
    const int r = rank[g];
    if (r < 0) return;
    AlienCellTO c = cold[s.coldIdx[g]];
    c.id = s.id[g];
    const float2 p = stepPos(s, g, wi.W, wi.H), v = s.velA[g];
    c.pos.x = p.x;
    c.pos.y = p.y;
    c.vel.x = v.x;
    c.vel.y = v.y;
    c.energy = s.energy[g];
    c.stiffness = s.stiffness[g];
    c.color = s.color[g];
    c.maxConnections = s.maxConn[g];
    const int n = s.numConn[g];
    c.numConnections = static_cast<uint8_t>(n);
    c.barrier = s.barrier[g];
    c.livingState = s.livingState[g];
    c.age = s.age[g];
    c.activationTime = s.activationTime[g];
    for (int k = 0; k < kMaxBonds; ++k) {
        if (k < n) {
            c.connections[k].cellIndex = rank[s.bond[g * kMaxBonds + k]];  // -1 when the partner is not exported
            c.connections[k].distance = s.bondDist[g * kMaxBonds + k];
            c.connections[k].angleFromPrevious = s.bondAngle[g * kMaxBonds + k];
        } else {
            c.connections[k].cellIndex = 0;
            c.connections[k].distance = 0.0f;
            c.connections[k].angleFromPrevious = 0.0f;
        }
    }
    out[r] = c;
}

__global__ void __launch_bounds__(kBlock) kEgressParticles(DevState s, int w, const int* rank, AlienParticleTO* out)
{
    const WorldInfo& wi = s.worlds[w];
    const long long q = wi.partBase + static_cast<long long>(blockIdx.x) * kBlock + threadIdx.x;
    const int r = rank[q];
    if (r < 0) return;
    AlienParticleTO p;
    memset(&p, 0, sizeof(p));
    p.id = s.pid[q];
    p.energy = s.penergy[q];
    const float2 pos = s.ppos[q], vel = s.pvel[q];
    p.pos.x = pos.x;
    p.pos.y = pos.y;
    p.vel.x = vel.x;
    p.vel.y = vel.y;
    p.color = s.pcolor[q];
    p.selected = s.pselected[q];
    out[r] = p;
}

// ---- stable particle compaction of one world (GarbageCollectorKernels.cu
// :177-196 without the reordering): live particles move to partBase + rank
__global__ void __launch_bounds__(kBlock) kCompactParticlesGather(DevState s, int w, const int* rank, unsigned long long* tid,
                                                                  float2* tpos, float2* tvel, float* tenergy, uint8_t* tcolor,
                                                                  uint8_t* tsel, unsigned long long* tlast)
{
    const WorldInfo& wi = s.worlds[w];
    const long long q = wi.partBase + static_cast<long long>(blockIdx.x) * kBlock + threadIdx.x;
    const int r = rank[q];
    if (r < 0) return;
    tid[r] = s.pid[q];
    tpos[r] = s.ppos[q];
    tvel[r] = s.pvel[q];
    tenergy[r] = s.penergy[q];
    tcolor[r] = s.pcolor[q];
    tsel[r] = s.pselected[q];
    tlast[r] = s.plast[q];
}

__global__ void __launch_bounds__(kBlock) kCompactParticlesScatter(DevState s, int w, long long count, const unsigned long long* tid,
                                                                   const float2* tpos, const float2* tvel, const float* tenergy,
                                                                   const uint8_t* tcolor, const uint8_t* tsel,
                                                                   const unsigned long long* tlast)
{
    const WorldInfo& wi = s.worlds[w];
    const long long r = static_cast<long long>(blockIdx.x) * kBlock + threadIdx.x;
    if (r >= wi.partCap) return;
    const long long q = wi.partBase + r;
    if (r < count) {
        s.pid[q] = tid[r];
        s.ppos[q] = tpos[r];
        s.pvel[q] = tvel[r];
        s.penergy[q] = tenergy[r];
        s.pcolor[q] = tcolor[r];
        s.pselected[q] = tsel[r];
        s.plast[q] = tlast[r];
        s.palive[q] = 1;
    } else {
        s.palive[q] = 0;
    }
}

// ---- statistics (subset of RawStatisticsData; StatisticsKernels.cu:5-105) ----
// Timeline and age histogram of world w (RawStatisticsData): counts and
// fixed-point energies per color, accumulated per block in shared memory and
// added to `acc` with one atomic per block and field.
struct TimelineAcc {
    unsigned long long cells[ALIEN_B200_MAX_COLORS];
    unsigned long long freeCells[ALIEN_B200_MAX_COLORS];
    unsigned long long particles[ALIEN_B200_MAX_COLORS];
    long long energyFix[ALIEN_B200_MAX_COLORS];  // 2^-16 fixed point
    unsigned int maxAge;                          // of the cells that are not barriers
    unsigned int pad;
    unsigned int histogram[ALIEN_B200_MAX_COLORS][ALIEN_B200_MAX_HISTOGRAM_SLOTS];
};
constexpr uint32_t kMutationIdForFreeCell = 1;  // Const::MutationIdForFreeCell, CellFunctionConstants.h:176

// StatisticsKernels.cu:12-46 (timestep statistics) and 73-83 (largest age)
__global__ void __launch_bounds__(kBlock) kStatsTimeline(DevState s, int w, TimelineAcc* acc)
{
    __shared__ unsigned long long sh[4][ALIEN_B200_MAX_COLORS];
    __shared__ unsigned int shMax;
    if (threadIdx.x < 4 * ALIEN_B200_MAX_COLORS) (&sh[0][0])[threadIdx.x] = 0;
    if (threadIdx.x == 0) shMax = 0;
    __syncthreads();
    const WorldInfo& wi = s.worlds[w];
    const WorldCounters& wc = s.counters[w];
    const long long stride = static_cast<long long>(gridDim.x) * kBlock;
    unsigned int myMax = 0;
    for (long long g = wi.cellBase + static_cast<long long>(blockIdx.x) * kBlock + threadIdx.x; g < wi.cellBase + wc.numCells;
         g += stride) {
        if (!s.alive[g]) continue;
        const int col = s.color[g] % ALIEN_B200_MAX_COLORS;
        atomicAdd(&sh[0][col], 1ull);
        if (s.cold[s.coldIdx[g]].mutationId == kMutationIdForFreeCell) atomicAdd(&sh[1][col], 1ull);
        atomicAdd(&sh[3][col], static_cast<unsigned long long>(__double2ll_rn(static_cast<double>(s.energy[g]) * 65536.0)));
        if (!s.barrier[g]) myMax = max(myMax, s.age[g]);
    }
    for (long long q = wi.partBase + static_cast<long long>(blockIdx.x) * kBlock + threadIdx.x; q < wi.partBase + wc.numParticles;
         q += stride) {
        if (!s.palive[q]) continue;
        const int col = s.pcolor[q] % ALIEN_B200_MAX_COLORS;
        atomicAdd(&sh[2][col], 1ull);
        atomicAdd(&sh[3][col], static_cast<unsigned long long>(__double2ll_rn(static_cast<double>(s.penergy[q]) * 65536.0)));
    }
    atomicMax(&shMax, myMax);
    __syncthreads();
    if (threadIdx.x < 4 * ALIEN_B200_MAX_COLORS) {
        const int f = threadIdx.x / ALIEN_B200_MAX_COLORS, c = threadIdx.x % ALIEN_B200_MAX_COLORS;
        const unsigned long long v = sh[f][c];
        if (v) {
            unsigned long long* dst = f == 0 ? &acc->cells[c]
                                     : f == 1 ? &acc->freeCells[c]
                                     : f == 2 ? &acc->particles[c]
                                              : reinterpret_cast<unsigned long long*>(&acc->energyFix[c]);
            atomicAdd(dst, v);
        }
    }
    if (threadIdx.x == 0 && shMax) atomicMax(&acc->maxAge, shMax);
}

// StatisticsKernels.cu:90-105: age histogram with the largest age of kStatsTimeline
__global__ void __launch_bounds__(kBlock) kStatsHistogram(DevState s, int w, TimelineAcc* acc)
{
    __shared__ unsigned int sh[ALIEN_B200_MAX_COLORS][ALIEN_B200_MAX_HISTOGRAM_SLOTS];
    for (int i = threadIdx.x; i < ALIEN_B200_MAX_COLORS * ALIEN_B200_MAX_HISTOGRAM_SLOTS; i += kBlock) (&sh[0][0])[i] = 0;
    __syncthreads();
    const WorldInfo& wi = s.worlds[w];
    const WorldCounters& wc = s.counters[w];
    const unsigned long long maxAge = acc->maxAge;
    const long long stride = static_cast<long long>(gridDim.x) * kBlock;
    for (long long g = wi.cellBase + static_cast<long long>(blockIdx.x) * kBlock + threadIdx.x; g < wi.cellBase + wc.numCells;
         g += stride) {
        if (!s.alive[g] || s.barrier[g]) continue;
        const int slot = static_cast<int>(static_cast<unsigned long long>(s.age[g]) * ALIEN_B200_MAX_HISTOGRAM_SLOTS / (maxAge + 1));
        atomicAdd(&sh[s.color[g] % ALIEN_B200_MAX_COLORS][slot], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < ALIEN_B200_MAX_COLORS * ALIEN_B200_MAX_HISTOGRAM_SLOTS; i += kBlock) {
        const unsigned int v = (&sh[0][0])[i];
        if (v) atomicAdd(&(&acc->histogram[0][0])[i], v);
    }
}

struct StatsAcc {
    unsigned long long numCells, numParticles, numConnections;
    unsigned long long numCellsByColor[ALIEN_B200_MAX_COLORS];
    long long cellEnergyFix, particleEnergyFix;  // 2^-16 fixed point: order-independent sums
};

__device__ __forceinline__ unsigned long long warpSumU64(unsigned long long v)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// statistics of world w (getRawStatistics): a grid of a few blocks per SM
// strides over the world's used cell and particle slots; each thread keeps
// its partial counts in registers, each block sums them (warp shuffles, then
// shared memory) and adds the block totals with one atomic per counter.
// All sums are integers (energies in 2^-16 fixed point), so the result does
// not depend on the order of the atomics.
constexpr int kStatsFields = 4 + ALIEN_B200_MAX_COLORS + 1;  // cells, bonds, cellE, parts, colors..., partE
__global__ void __launch_bounds__(kBlock) kStatsWorld(DevState s, int w, StatsAcc* acc)
{
    __shared__ unsigned long long red[kStatsFields][kBlock / 32];
    const WorldInfo& wi = s.worlds[w];
    const WorldCounters& wc = s.counters[w];
    const long long stride = static_cast<long long>(gridDim.x) * kBlock;
    unsigned int cells = 0, bonds = 0, parts = 0;
    unsigned int byColor[ALIEN_B200_MAX_COLORS] = {};
    long long cellE = 0, partE = 0;
    // four slots per thread and iteration, as vector loads: ranges start at
    // a multiple of 256 slots and their capacity is a multiple of 256, so
    // the quads are aligned and lie inside the arrays; slots past the count
    // and dead slots are skipped
    const long long nCells = wc.numCells, cellQuads = (nCells + 3) / 4;
#pragma unroll 2
    for (long long i = static_cast<long long>(blockIdx.x) * kBlock + threadIdx.x; i < cellQuads; i += stride) {
        const long long g = wi.cellBase + 4 * i;
        const uchar4 al = *reinterpret_cast<const uchar4*>(s.alive + g);
        const uchar4 nc = *reinterpret_cast<const uchar4*>(s.numConn + g);
        const float4 e = *reinterpret_cast<const float4*>(s.energy + g);
        const uchar4 co = *reinterpret_cast<const uchar4*>(s.color + g);
        const long long left = nCells - 4 * i;
        const bool a[4] = {al.x != 0, al.y != 0 && left > 1, al.z != 0 && left > 2, al.w != 0 && left > 3};
        const unsigned int n4[4] = {nc.x, nc.y, nc.z, nc.w};
        const float e4[4] = {e.x, e.y, e.z, e.w};
        const int c4[4] = {co.x % ALIEN_B200_MAX_COLORS, co.y % ALIEN_B200_MAX_COLORS, co.z % ALIEN_B200_MAX_COLORS,
                           co.w % ALIEN_B200_MAX_COLORS};
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            if (!a[k]) continue;
            ++cells;
            bonds += n4[k];
            cellE += __double2ll_rn(static_cast<double>(e4[k]) * 65536.0);
#pragma unroll
            for (int c = 0; c < ALIEN_B200_MAX_COLORS; ++c) byColor[c] += c4[k] == c ? 1u : 0u;
        }
    }
    const long long nParts = wc.numParticles, partQuads = (nParts + 3) / 4;
#pragma unroll 2
    for (long long i = static_cast<long long>(blockIdx.x) * kBlock + threadIdx.x; i < partQuads; i += stride) {
        const long long q = wi.partBase + 4 * i;
        const uchar4 al = *reinterpret_cast<const uchar4*>(s.palive + q);
        const float4 e = *reinterpret_cast<const float4*>(s.penergy + q);
        const long long left = nParts - 4 * i;
        const bool a[4] = {al.x != 0, al.y != 0 && left > 1, al.z != 0 && left > 2, al.w != 0 && left > 3};
        const float e4[4] = {e.x, e.y, e.z, e.w};
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            if (!a[k]) continue;
            ++parts;
            partE += __double2ll_rn(static_cast<double>(e4[k]) * 65536.0);
        }
    }
    unsigned long long v[kStatsFields];
    v[0] = cells;
    v[1] = bonds;
    v[2] = static_cast<unsigned long long>(cellE);
    v[3] = parts;
#pragma unroll
    for (int c = 0; c < ALIEN_B200_MAX_COLORS; ++c) v[4 + c] = byColor[c];
    v[4 + ALIEN_B200_MAX_COLORS] = static_cast<unsigned long long>(partE);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int f = 0; f < kStatsFields; ++f) {
        const unsigned long long t = warpSumU64(v[f]);
        if (lane == 0) red[f][warp] = t;
    }
    __syncthreads();
    if (threadIdx.x < kStatsFields) {
        unsigned long long t = 0;
        for (int i = 0; i < kBlock / 32; ++i) t += red[threadIdx.x][i];
        if (t) {
            StatsAcc& a = acc[w];
            unsigned long long* dst;
            const int f = threadIdx.x;
            if (f == 0) dst = &a.numCells;
            else if (f == 1) dst = &a.numConnections;
            else if (f == 2) dst = reinterpret_cast<unsigned long long*>(&a.cellEnergyFix);
            else if (f == 3) dst = &a.numParticles;
            else if (f < 4 + ALIEN_B200_MAX_COLORS) dst = &a.numCellsByColor[f - 4];
            else dst = reinterpret_cast<unsigned long long*>(&a.particleEnergyFix);
            atomicAdd(dst, t);
        }
    }
}

// prepareForSimulationParametersChanges -> resetDensity (CellProcessor.cuh:860-870)
__global__ void __launch_bounds__(kBlock) kResetDensity(DevState s, int w)
{
    const WorldInfo& wi = s.worlds[w];
    const long long g = wi.cellBase + static_cast<long long>(blockIdx.x) * kBlock + threadIdx.x;
    if (g < wi.cellBase + wi.cellCap) s.density[g] = 1.0f;
}

// state the transfer objects do not hold, carried through an arena rebuild
// (more particle room, a new interaction radius): the fluid density of each
// live cell and the last absorbing cell of each live particle, in egress
// order (rank from kSelectCells / kSelectParticles), and back after ingest
__global__ void __launch_bounds__(kBlock) kGatherCarried(DevState s, int w, const int* cellRank, const int* partRank,
                                                         float* density, unsigned long long* last)
{
    const WorldInfo& wi = s.worlds[w];
    const long long i = static_cast<long long>(blockIdx.x) * kBlock + threadIdx.x;
    if (i < wi.cellCap) {
        const int r = cellRank[wi.cellBase + i];
        if (r >= 0) density[r] = s.density[wi.cellBase + i];
    }
    if (i < wi.partCap) {
        const int r = partRank[wi.partBase + i];
        if (r >= 0) last[r] = s.plast[wi.partBase + i];
    }
}

__global__ void __launch_bounds__(kBlock) kRestoreCarried(DevState s, int w, const float* density, long long nc,
                                                          const unsigned long long* last, long long np)
{
    const WorldInfo& wi = s.worlds[w];
    const long long i = static_cast<long long>(blockIdx.x) * kBlock + threadIdx.x;
    if (density && i < nc) s.density[wi.cellBase + i] = density[i];
    if (i < np) s.plast[wi.partBase + i] = last[i];
}

// ----------------------------------------------------------- density map --
// DensityMap (DensityMap.cuh:8-230), the coarse map the reference fills in
// every step (clear at SimulationKernels.cu:33, addCell for every cell in
// the pair-force kernels :39 and :47) and that only sensor cells read.  Here
// it is built on request, from the state the last step left: each live cell
// at its position after that step's overlap correction (posA + push, the
// position the reference's cell holds when its own thread adds it), on
// slots of 8 x 8 (PreprocessedSimulationData.cuh:13), with the packed byte
// counters of addCell (DensityMap.cuh:150-205; carries between the byte
// lanes as in the reference's 64-bit adds).
constexpr int kDensitySlot = 8;
struct DensityMapOut {
    unsigned long long *color, *otherMutant, *sameMutant1, *sameMutant2;
    unsigned int* specificMutant;
    unsigned long long *lessComplexity1, *lessComplexity2, *moreComplexity1, *moreComplexity2;
    int sizeX, sizeY;
    unsigned long long timestep;  // of the step that filled the map (other-mutant buckets)
};

__global__ void __launch_bounds__(kBlock) kDensityMap(DevState s, int w, DensityMapOut m)
{
    const WorldInfo& wi = s.worlds[w];
    const long long i = static_cast<long long>(blockIdx.x) * kBlock + threadIdx.x;
    if (i >= s.counters[w].numCells) return;
    const long long g = wi.cellBase + i;
    if (!s.alive[g]) return;
    const float2 pos = s.posA[g] + s.push[g];
    // toInt (Base.cuh:29-32) truncates; the index is checked as a whole
    const long long index = static_cast<long long>(static_cast<int>(pos.x) / kDensitySlot) +
                            static_cast<long long>(static_cast<int>(pos.y) / kDensitySlot) * m.sizeX;
    if (index < 0 || index >= static_cast<long long>(m.sizeX) * m.sizeY) return;
    const int color = s.color[g] % ALIEN_B200_MAX_COLORS;
    atomicAdd(m.color + index, (1ull << (color * 8)) | (1ull << 56));
    const AlienCellTO& c = s.cold[s.coldIdx[g]];
    const uint32_t mutationId = c.mutationId;
    if (mutationId == 0) {
        atomicAdd(m.specificMutant + index, 1u);
        return;
    }
    if (mutationId == 1) {
        atomicAdd(m.specificMutant + index, 0x100u);
        return;
    }
    const unsigned long long other = (static_cast<unsigned long long>(mutationId) + m.timestep / 23) % 8;
    atomicAdd(m.otherMutant + index, 0x0101010101010101ull ^ (1ull << (other * 8)));
    const unsigned long long b1 = mutationId % 3, b2 = mutationId % 5, b3 = mutationId % 7;
    atomicAdd(m.sameMutant1 + index, (1ull << (b1 * 8)) | (1ull << ((b2 + 3) * 8)));
    atomicAdd(m.sameMutant2 + index, 1ull << (b3 * 8));
    // complexity bucket: the bit length of toInt(complexity * 10)
    const int bucket = 32 - __clz(static_cast<int>(c.genomeComplexity * 10.0f));
    const unsigned long long lanes = 0x0101010101010101ull;
    if (bucket < 8) {
        atomicAdd(m.lessComplexity1 + index, lanes << (bucket * 8));  // byte lanes bucket..7
        atomicAdd(m.lessComplexity2 + index, lanes);
        atomicAdd(m.moreComplexity1 + index, lanes >> ((7 - bucket) * 8));  // byte lanes 0..bucket
    } else if (bucket < 16) {
        atomicAdd(m.lessComplexity2 + index, lanes << ((bucket - 8) * 8));
        atomicAdd(m.moreComplexity2 + index, lanes >> ((15 - bucket) * 8));
        atomicAdd(m.moreComplexity1 + index, lanes);
    }
}

}  // namespace ab
