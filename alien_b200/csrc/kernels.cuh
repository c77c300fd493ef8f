// kernels.cuh - the per-timestep physics stage of the B200 engine.
//
// One timestep = the launch sequence in Arena::enqueueStep (engine.cu).  The
// phases follow _SimulationKernelsLauncher::calcTimestep
// (source/EngineGpuKernels/SimulationKernelsLauncher.cu:25-91) for the
// physics kernels; every phase boundary that the reference crosses by racing
// threads inside one kernel is a kernel boundary here, so each kernel reads
// only values that are final (deterministic step definition, identical to
// the CPU oracle):
//
//   kBin        cell map binning by tile + radiation + per-step resets,
//               particle map (physics_init / physics_fillMaps)
//   scan        exclusive scan of per-tile counts
//   kScatter    cell slots grouped by tile
//   kStage      per-slot rank (scan visibility) + sorted SoA copy
//   kPairs*     fluid or collision pair forces (physics_calc*Forces)
//   kApplyBond1 checkForces, applyForces, bond forces #1, | particle movement
//               verletPositionUpdate (steps without angle forces)
//   kVerletPos  verletPositionUpdate (angle-force steps) | particle targets
//   kBond2      checkConnections, bond forces #2         | particle merges
//   kVerletVel  verletVelocityUpdate, aging              | absorption
//   kTransition living-state transition, inner friction, | splitting,
//               friction, decay                          | particle map reset
//   kResolve    new living states, bond additions (scratch)
//   kCommit     bond additions, cell deletion, bond deletion
//   kEvent*     ids and slots of new energy particles, append
#pragma once

#include "device_common.cuh"
#include "zones.cuh"

namespace ab {

// ------------------------------------------------------------ helpers ----

struct CellCtx {
    int w;
    long long g;
    bool valid;
};

__device__ __forceinline__ CellCtx cellCtx(const DevState& s)
{
    CellCtx c;
    int b = blockIdx.x;
    c.g = static_cast<long long>(b) * kBlock + threadIdx.x;
    // every launched cell slot lies inside the arena (the cell blocks tile
    // it exactly), so the alive flag is loaded together with the world
    // lookup instead of after it
    const bool alive = s.alive[c.g];
    c.w = s.cellBlockWorld[b];
    const WorldInfo& wi = s.worlds[c.w];
    const WorldCounters& wc = s.counters[c.w];
    c.valid = wc.active && c.g < wi.cellBase + wc.numCells && alive;
    return c;
}

// particle part of a combined launch: blocks [numCellBlocks, numCellBlocks + numPartBlocks)
struct PartCtx {
    int w;
    long long q;
    bool inRange;  // slot used at step start (orig particles)
};
__device__ __forceinline__ PartCtx partCtx(const DevState& s, int pb)
{
    PartCtx c;
    c.w = s.partBlockWorld[pb];
    c.q = static_cast<long long>(pb) * kBlock + threadIdx.x;
    const WorldInfo& wi = s.worlds[c.w];
    const WorldCounters& wc = s.counters[c.w];
    c.inRange = wc.active && c.q < wi.partBase + wc.numParticles;
    return c;
}

// The particle part of a combined launch: the grid's blocks past the cell
// blocks stride over the particle blocks, skipping inactive worlds (unless
// SkipInactive is false) and the blocks past a world's used slots
// (partBase + usedSlots(counters)), so its cost follows the live particles
// rather than the capacity.  Everything f sees is block-uniform, so f may
// synchronise the block; f's return ends one particle block for the calling
// thread.
template <bool SkipInactive = true, class UsedSlots, class F>
__device__ __forceinline__ void forParticleBlocks(const DevState& s, UsedSlots usedSlots, F f, int firstBlock)
{
    const int stride = gridDim.x - firstBlock;
    for (int pb = blockIdx.x - firstBlock; pb < s.numPartBlocks; pb += stride) {
        const int w = s.partBlockWorld[pb];
        const WorldInfo& wi = s.worlds[w];
        const WorldCounters& wc = s.counters[w];
        const long long end = wi.partBase + static_cast<long long>(usedSlots(wc));
        if ((SkipInactive && !wc.active) || static_cast<long long>(pb) * kBlock >= end) {
            // on to the first block of the next world in this block's stride
            // (an unused block of a live arena belongs to no range: the next one)
            const int next = max(wi.firstPartBlock + wi.numPartBlocks, pb + 1);
            pb += ((next - pb + stride - 1) / stride - 1) * stride;
            continue;
        }
        PartCtx c;
        c.w = w;
        c.q = static_cast<long long>(pb) * kBlock + threadIdx.x;
        c.inRange = c.q < end;
        f(c, pb);
    }
}
template <bool SkipInactive = true, class UsedSlots, class F>
__device__ __forceinline__ void forParticleBlocks(const DevState& s, UsedSlots usedSlots, F f)
{
    forParticleBlocks<SkipInactive>(s, usedSlots, f, s.numCellBlocks);
}
__device__ __forceinline__ unsigned int usedParticles(const WorldCounters& wc) { return wc.numParticles; }

// bonds[] holds kMaxBonds entries, unused ones -1: a fixed-trip compare
// keeps the list in registers
__device__ __forceinline__ bool isBondedTo(const int* bonds, int j)
{
    bool r = false;
#pragma unroll
    for (int k = 0; k < kMaxBonds; ++k) r |= (bonds[k] == j);
    return r;
}


constexpr int kMaxRadius = 15;

// Calls f(tile) once for every tile that the (2r+1)^2-slot scan window of
// slot (sx, sy) touches.  Along each axis the wrapped slots s-r..s+r map to
// non-decreasing tiles with at most one wrap (the world is at least 2r+1
// wide), so skipping repeats of the previous tile lists each tile once.
template <class F>
__device__ __forceinline__ void forEachWindowTile(const WorldInfo& wi, int sx, int sy, F&& f)
{
    const int r = wi.radiusInt;
    int prevTy = -1;
    for (int dy = -r; dy <= r; ++dy) {
        int y = sy + dy;
        y += y < 0 ? wi.H : 0;
        y -= y >= wi.H ? wi.H : 0;
        const int ty = y / wi.T;
        if (ty == prevTy) continue;
        prevTy = ty;
        int prevTx = -1;
        for (int dx = -r; dx <= r; ++dx) {
            int x = sx + dx;
            x += x < 0 ? wi.W : 0;
            x -= x >= wi.W ? wi.W : 0;
            const int tx = x / wi.T;
            if (tx == prevTx) continue;
            prevTx = tx;
            f(wi.tileBase + tx + static_cast<long long>(ty) * wi.nTX);
        }
    }
}

// the previous step's position of the cell: its start position plus the
// displacement the step accumulated, rounded once (the FP32 state the
// reference keeps in Cell::pos)
__device__ __forceinline__ float2 foldDisplacement(const DevState& s, const WorldInfo& wi, long long g, float2 pos, float2 d)
{
    if (d.x == 0.0f && d.y == 0.0f) return pos;
    pos = correctPosition(pos + d, wi.W, wi.H);
    s.posA[g] = pos;
    s.dpos[g] = f2(0.0f, 0.0f);
    return pos;
}

// the cell's slot and tile at binning, its slot within the tile (T <= 15,
// so below 225) and its arrival rank in the tile
__device__ __forceinline__ void binCell(const DevState& s, const WorldInfo& wi, long long g, float2 pos)
{
    const int sx = slotX(pos.x, wi.W), sy = slotX(pos.y, wi.H);
    const int tx = sx / wi.T, ty = sy / wi.T;
    const uint32_t tile = static_cast<uint32_t>(wi.tileBase + tx + static_cast<long long>(ty) * wi.nTX);
    s.tileOf[g] = tile;
    s.slotOf[g] = static_cast<uint32_t>(sx + sy * wi.W);
    s.slotInTile[g] = static_cast<uint8_t>((sx - tx * wi.T) + (sy - ty * wi.T) * wi.T);
    s.tileOff[g] = atomicAdd(&s.tileCount[tile], 1u);
}

// the radiation factor (CellProcessor.cuh:730-745) is a sum of the high-
// energy factor and the age strength, the latter blended from the base and
// the zones that activate it with nonnegative weights: with no positive term
// among them no cell of the world can emit, whatever its draw
__device__ __forceinline__ bool radiationPossible(const AlienPhysicsParams& p)
{
    bool any = false;
#pragma unroll
    for (int c = 0; c < ALIEN_B200_MAX_COLORS; ++c) any |= p.highRadiationFactor[c] > 0.0f || p.radiationCellAgeStrength[c] > 0.0f;
    for (int i = 0; i < p.numZones && !any; ++i)
        if (p.zones[i].radiationCellAgeStrengthActivated)
            for (int c = 0; c < ALIEN_B200_MAX_COLORS; ++c) any |= p.zones[i].radiationCellAgeStrength[c] > 0.0f;
    return any;
}

// ---------------------------------------------------------------- kBin ----
// cells: reset per-step scratch, tile binning (CellMap::set_block,
// Map.cuh:95-130, by tile instead of a pointer chain), radiation
// (CellProcessor::radiation, CellProcessor.cuh:725-773).
// particles: reset, particle map (ParticleMap::set_block, Map.cuh:236-258;
// the highest storage index wins).
__global__ void __launch_bounds__(kBlock, 8) kBin(DevState s)
{
    if (blockIdx.x < s.numCellBlocks) {
        // per-step scratch needs no reset here: flags are cleared by
        // kEventEmit, the fixed-point accumulators and newPartner by the
        // kernels that consume them, and best is written for every live cell
        // own fields before the world lookup (every launched cell slot lies
        // inside the arena)
        float2 pos = s.posA[static_cast<long long>(blockIdx.x) * kBlock + threadIdx.x];
        const float2 d = s.dpos[static_cast<long long>(blockIdx.x) * kBlock + threadIdx.x];
        const bool barrierG = s.barrier[static_cast<long long>(blockIdx.x) * kBlock + threadIdx.x];
        CellCtx c = cellCtx(s);
        const long long g = c.g;
        if (!c.valid) return;
        const WorldInfo& wi = s.worlds[c.w];
        const AlienPhysicsParams& p = s.params[wi.paramIndex];
        pos = foldDisplacement(s, wi, g, pos, d);
        binCell(s, wi, g, pos);

        if (barrierG || !(p.radiationProb > 0.0f)) return;  // a draw in [0, 1) never falls below 0
        if (!radiationPossible(p)) return;  // the emission factor is 0 for every cell of the world
        const uint64_t T = s.counters[c.w].timestep;
        const uint64_t id = s.id[g];
        if (!(draw(id, T, kSiteRadiation) < p.radiationProb)) return;
        int col = s.color[g] % ALIEN_B200_MAX_COLORS;
        float e = s.energy[g];
        float factor = 0.0f;
        if (e > p.highRadiationMinCellEnergy[col]) factor += p.highRadiationFactor[col];
        if (static_cast<long long>(s.age[g]) > static_cast<long long>(p.radiationMinCellAge[col]))
            factor += zoneParam<kZRadiationCellAgeStrength>(p, wi.W, wi.H, pos, p.radiationCellAgeStrength[col], col);
        if (!(factor > 0.0f)) return;
        float loss = e * factor;
        loss = loss / p.radiationProb;
        loss = 2.0f * loss * draw(id, T, kSiteRadiationEnergy);
        if (e > 1.0f) {
            float2 v = s.velA[g];
            float2 pv = v * p.radiationVelocityMultiplier
                + unitVectorOfAngle(draw(id, T, kSiteRadiationAngle) * 360.0f) * p.radiationVelocityPerturbation;
            float2 pp = pos + normalized2(pv) * 1.5f - pv;
            pp = correctPosition(pp, wi.W, wi.H);
            if (loss > e - 1.0f) loss = e - 1.0f;
            s.energy[g] = e - loss;
            // createEnergyParticle (RadiationProcessor.cuh:248-364): at an
            // active radiation source if there is one, the external-energy
            // backflow, and no particle for energy <= NEAR_ZERO
            WorldCounters& wcr = s.counters[c.w];
            placeAtSource(p, wcr.activeSources, id, T, kSiteSourceRadiation, pp, pv);
            pp = correctPosition(pp, wi.W, wi.H);
            const float kept = backflow(p, wcr, col, loss);
            if (kept > kNearZero) {
                s.radPos[g] = pp;
                s.radVel[g] = pv;
                s.radEnergy[g] = kept;
                atomicOr(&s.flags[g], kFlagRadiation);
            }
        }
    } else {
        forParticleBlocks(s, usedParticles, [&](const PartCtx& c, int) {
            const long long q = c.q;
            s.pflag[q] = 0;
            s.ptarget[q] = -1;
            s.pslot[q] = -1;
            s.pmerge[3 * q + 0] = 0;
            s.pmerge[3 * q + 1] = 0;
            s.pmerge[3 * q + 2] = 0;
            if (!c.inRange || !s.palive[q]) return;
            const WorldInfo& wi = s.worlds[c.w];
            float2 pp = s.ppos[q];
            int slot = slotX(pp.x, wi.W) + slotX(pp.y, wi.H) * wi.W;
            s.pslot[q] = slot;
            atomicMax(&s.pmap[wi.pmapBase + slot], static_cast<int>(q));
        });
    }
}

// ------------------------------------------------------------- scan ------
// exclusive scan of n uint32 values: kScanReduce -> kScanPartials -> kScanDown
constexpr int kScanItems = 8;
constexpr int kScanTile = kBlock * kScanItems;

__global__ void __launch_bounds__(kBlock) kScanReduce(const uint32_t* in, long long n, uint32_t* partials)
{
    long long base = static_cast<long long>(blockIdx.x) * kScanTile;
    uint32_t sum = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        long long k = base + static_cast<long long>(i) * kBlock + threadIdx.x;
        if (k < n) sum += in[k];
    }
    uint32_t total;
    blockExclusiveScan(sum, &total);
    if (threadIdx.x == 0) partials[blockIdx.x] = total;
}

// one block of Threads threads; sequential chunks of Threads
template <int Threads>
__global__ void __launch_bounds__(Threads) kScanPartials(uint32_t* partials, int numPartials)
{
    uint32_t carry = 0;
    for (int base = 0; base < numPartials; base += Threads) {
        int k = base + threadIdx.x;
        uint32_t v = k < numPartials ? partials[k] : 0;
        uint32_t total;
        uint32_t ex = blockExclusiveScanN<Threads>(v, &total);
        if (k < numPartials) partials[k] = carry + ex;
        carry += total;
    }
    if (threadIdx.x == 0) partials[numPartials] = carry;
}

// in and out are 16-byte aligned (device allocations), so a thread's eight
// items are two 16-byte loads and stores wherever all eight lie below n.
// With PrefixFromTotals the partials are kScanReduce's block totals as they
// are, and every block sums those of the blocks before it (no kScanPartials
// launch; for scans of at most kScanFusedBlocks blocks, where that costs at
// most kScanFusedBlocks^2 / 2 reads from L2); otherwise they are already
// scanned.
constexpr int kScanFusedBlocks = 2048;
template <bool PrefixFromTotals>
__global__ void __launch_bounds__(kBlock) kScanDown(const uint32_t* in, long long n, const uint32_t* partials, uint32_t* out)
{
    static_assert(kScanItems == 8, "two uint4 per thread");
    long long base = static_cast<long long>(blockIdx.x) * kScanTile + static_cast<long long>(threadIdx.x) * kScanItems;
    const bool full = base + kScanItems <= n;
    uint32_t v[kScanItems];
    if (full) {
        const uint4 a = *reinterpret_cast<const uint4*>(in + base);
        const uint4 b = *reinterpret_cast<const uint4*>(in + base + 4);
        v[0] = a.x, v[1] = a.y, v[2] = a.z, v[3] = a.w, v[4] = b.x, v[5] = b.y, v[6] = b.z, v[7] = b.w;
    } else {
#pragma unroll
        for (int i = 0; i < kScanItems; ++i) v[i] = base + i < n ? in[base + i] : 0;
    }
    uint32_t prefix;
    if (PrefixFromTotals) {
        uint32_t pre = 0;
        for (int k = threadIdx.x; k < static_cast<int>(blockIdx.x); k += kBlock) pre += partials[k];
        blockExclusiveScan(pre, &prefix);
    } else {
        prefix = partials[blockIdx.x];
    }
    uint32_t sum = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) sum += v[i];
    uint32_t total;
    uint32_t ex = blockExclusiveScan(sum, &total) + prefix;
    uint32_t o[kScanItems];
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        o[i] = ex;
        ex += v[i];
    }
    if (full) {
        *reinterpret_cast<uint4*>(out + base) = make_uint4(o[0], o[1], o[2], o[3]);
        *reinterpret_cast<uint4*>(out + base + 4) = make_uint4(o[4], o[5], o[6], o[7]);
        if (base + kScanItems == n) out[n] = ex;
    } else {
#pragma unroll
        for (int i = 0; i < kScanItems; ++i) {
            if (base + i < n) out[base + i] = o[i];
            if (base + i == n - 1) out[n] = o[i] + v[i];
        }
    }
}

// ----------------------------------------------------------- kScatter ----
__global__ void __launch_bounds__(kBlock) kScatter(DevState s)
{
    const long long g0 = static_cast<long long>(blockIdx.x) * kBlock + threadIdx.x;
    const uint32_t t = s.tileOf[g0], off = s.tileOff[g0];  // before the world lookup
    const uint8_t local = s.slotInTile[g0];
    CellCtx c = cellCtx(s);
    if (!c.valid) return;
    const uint32_t k = s.tileStart[t] + off;
    s.sorted[k] = static_cast<uint32_t>(c.g);
    s.sortedSlot[k] = local;  // beside the tile's list, for the slot ranks of kStage
}

// ------------------------------------------------------------- kStage ----
// Rank of each cell among the cells of its slot in storage order (the
// reference chains at most 11 cells per slot and scans 10 of them,
// Map.cuh:113-125, CellProcessor.cuh:165) and a tile-sorted SoA copy of the
// fields the pair phase reads, each tile's records in storage order.
__global__ void __launch_bounds__(kBlock) kStage(DevState s)
{
    long long k = static_cast<long long>(blockIdx.x) * kBlock + threadIdx.x;
    // the launch covers the cell slots, so sorted[k] is inside the array
    // whether or not k is below the number of binned cells (one thread per
    // listed cell: the record writes stay contiguous, which measured faster
    // than one thread per cell in storage order with scattered records)
    const uint32_t total = s.tileStart[s.numTiles];
    const uint32_t g = s.sorted[k];
    const uint8_t slot = s.sortedSlot[k];  // slot within the tile
    if (k >= total) return;
    // the cell's fields, all in flight together
    const int w = s.cellBlockWorld[g / kBlock];
    const uint32_t t = s.tileOf[g];
    const float2 pos = s.posA[g];
    const float2 vel = s.velA[g];
    const bool barrierG = s.barrier[g];
    const int nc = s.numConn[g];
    const int mc = s.maxConn[g];
    const float dens = s.density[g];
    const float energy = s.energy[g];
    const uint32_t k0 = s.tileStart[t], k1 = s.tileStart[t + 1];
    int rank = 0, rankInTile = 0;
#pragma unroll 4
    for (uint32_t m = k0; m < k1; ++m) {
        uint32_t g2 = s.sorted[m];
        if (g2 >= g) continue;
        ++rankInTile;
        rank += s.sortedSlot[m] == slot;
    }
    // records of a tile in storage order: a fixed visiting order for the
    // pair phase, whatever order the binning atomics produced
    k = k0 + rankInTile;
    int fl = (barrierG ? kStageBarrier : 0) | (rank < kSlotScanLevels ? kStageVisible : 0) | (rank == 0 ? kStageHead : 0);
    fl |= (nc & 0xf) << 4;
    fl |= mc << 8;
    fl |= w << 16;
    s.stagedPV[k] = make_float4(pos.x, pos.y, vel.x, vel.y);
    s.stagedMeta[k] = make_int4(static_cast<int>(g), fl, __float_as_int(dens), __float_as_int(energy));
}

// ------------------------------------------------- cell-map read-back ----
// The binning of kBin alone (no radiation, no particles, no step counters):
// with the scan, kScatter and kStage it builds the cell map of the current
// state for alien_b200_debug_cell_map.  Everything it writes is rebuilt by
// the next step.
__global__ void __launch_bounds__(kBlock) kBinMap(DevState s)
{
    const float2 pos = s.posA[static_cast<long long>(blockIdx.x) * kBlock + threadIdx.x];
    const float2 d = s.dpos[static_cast<long long>(blockIdx.x) * kBlock + threadIdx.x];
    CellCtx c = cellCtx(s);
    if (!c.valid) return;
    const WorldInfo& wi = s.worlds[c.w];
    binCell(s, wi, c.g, foldDisplacement(s, wi, c.g, pos, d));
}

// the staged records in tile order: id, slot, tile (relative to the world's
// first tile) and the record's map flags (barrier, visible, slot head)
__global__ void __launch_bounds__(kBlock) kExportCellMap(DevState s, unsigned long long* ids, uint32_t* slots, uint32_t* tiles,
                                                         uint8_t* flags)
{
    const long long k = static_cast<long long>(blockIdx.x) * kBlock + threadIdx.x;
    if (k >= s.tileStart[s.numTiles]) return;
    const int4 meta = s.stagedMeta[k];
    const long long g = meta.x;
    const WorldInfo& wi = s.worlds[(meta.y >> 16) & 0xffff];
    ids[k] = s.id[g];
    slots[k] = s.slotOf[g];
    tiles[k] = static_cast<uint32_t>(s.tileOf[g] - wi.tileBase);
    flags[k] = static_cast<uint8_t>(meta.y & (kStageBarrier | kStageVisible | kStageHead));
}

// ---------------------------------------------------------- pair laws ----
// The pair phase of the two motion types as accumulators: begin() with the
// cell's staged record, near() as a cheap reject on the squared distance,
// visit() for the survivors, end() writes the cell's results.  Neighbours
// are visited tile by tile (3x3 tiles around the cell, in row order) and,
// within a tile, in storage order, so the FP32 sums are reproducible run to
// run and identical alone or in a batch.  Two enumerations feed the laws:
// kPairsRegion (shared-memory regions, the fast path) and pairsGlobal (tile
// lists in global memory, for regions that do not fit).

// sqrtf(q) <= R decided exactly (the reject bound is above R^2)
__device__ __forceinline__ bool withinRadius(float q, float R, float& d)
{
    d = sqrtf(q);
    return d <= R;
}

// CellProcessor::calcFluidForces_reconnectCells_correctOverlap,
// CellProcessor.cuh:122-283.  pd = p_i - p_j already corrected for the torus.
struct FluidLaw {
    const DevState* s;
    const AlienPhysicsParams* p;
    int g, W, H;
    float h, invH, invH2, invH3, R, R2reject, minDist, fusionVelocity, maxBindingEnergy;
    float2 pi, vi;
    bool barrierI, fusionI;
    float densI, invDensI;
    int bondsI[kMaxBonds];
    float dens;
    float2 Fp, Fv, dx;
    int bestBarrier;
    float bestBarrierDist;
    int best;
    unsigned long long bestId;

    // the state near() and relevant() need (the scan), then the rest (the law)
    __device__ __forceinline__ void beginScan(const DevState& st, const WorldInfo& wi, int4 me)
    {
        s = &st;
        p = &st.params[wi.paramIndex];
        g = me.x;
        h = p->smoothingLength;
        R = h * 2.0f;
        R2reject = R * R * 1.0001f + 1e-6f;
    }

    __device__ __forceinline__ void beginLaw(const WorldInfo& wi, int4 me, float2 pos, float2 vel)
    {
        const DevState& st = *s;
        W = wi.W;
        H = wi.H;
        invH = 1.0f / h;
        invH2 = invH * invH;
        invH3 = invH2 * invH;
        minDist = p->cellMinDistance;
        // zone values at the cell (CellProcessor.cuh:149-152)
        fusionVelocity = zoneParam<kZCellFusionVelocity>(*p, W, H, pos, p->cellFusionVelocity);
        maxBindingEnergy = zoneParam<kZCellMaxBindingEnergy>(*p, W, H, pos, p->cellMaxBindingEnergy);
        pi = pos;
        vi = vel;
        barrierI = me.y & kStageBarrier;
        const int nI = (me.y >> 4) & 0xf, maxI = (me.y >> 8) & 0xff;
        densI = __int_as_float(me.z);
        invDensI = __frcp_rn(densI);
        fusionI = !barrierI && nI < maxI && __int_as_float(me.w) <= maxBindingEnergy;
#pragma unroll
        for (int m = 0; m < kMaxBonds; ++m) bondsI[m] = m < nI ? st.bond[static_cast<long long>(g) * kMaxBonds + m] : -1;
        dens = 0.0f;
        Fp = Fv = dx = f2(0.0f, 0.0f);
        bestBarrier = -1;
        bestBarrierDist = 0.0f;
        best = -1;
        bestId = ~0ull;
    }

    __device__ __forceinline__ void begin(const DevState& st, const WorldInfo& wi, int4 me, float2 pos, float2 vel)
    {
        beginScan(st, wi, me);
        beginLaw(wi, me, pos, vel);
    }

    __device__ __forceinline__ bool near(float2 pd) const { return pd.x * pd.x + pd.y * pd.y <= R2reject; }
    // every candidate within the radius contributes (density, push)
    __device__ __forceinline__ bool relevant(const int4*, int, float2) const { return true; }

    __device__ __forceinline__ void visit(int4 om, float2 vj, float2 pd)
    {
        if (!(om.y & kStageVisible)) return;
        float d;
        if (!withinRadius(pd.x * pd.x + pd.y * pd.y, R, d)) return;
        const int j = om.x;
        if (om.y & kStageBarrier) {
            if (bestBarrier < 0 || d < bestBarrierDist || (d == bestBarrierDist && j < bestBarrier)) {
                bestBarrier = j;
                bestBarrierDist = d;
            }
            return;
        }
        const float q = d * invH;
        dens += sphKernel(q) * invH2;
        if (j == g) return;
        if (!barrierI && d < minDist) dx = dx + pd * (minDist / 5.0f);
        if (isBondedTo(bondsI, j)) return;
        const float2 vd = vi - vj;
        // rho_i / rho_i^2 + rho_j / rho_j^2 (CellProcessor.cuh:205) as reciprocals
        const float invDensJ = __frcp_rn(__int_as_float(om.z));
        const float factor = invDensI + invDensJ;
        if (fabsf(d) > kNearZero) {
            const float kd = sphKernelD(q) * invH3;
            Fp = Fp + pd * (-factor * kd * __frcp_rn(d));
            Fv = Fv + vd * (invDensJ * d * kd * __frcp_rn(d * d + 0.25f));
        }
        if (fusionI && len2(vd) >= fusionVelocity) {
            const int nJ = (om.y >> 4) & 0xf, maxJ = (om.y >> 8) & 0xff;
            if (nJ < maxJ && __int_as_float(om.w) <= maxBindingEnergy) {
                const unsigned long long idJ = s->id[j];
                if (idJ < bestId) {
                    bestId = idJ;
                    best = j;
                }
            }
        }
    }

    __device__ __forceinline__ void end()
    {
        const DevState& st = *s;
        float2 F = f2(0.0f, 0.0f);
        if (bestBarrier >= 0) {
            const long long b = bestBarrier;
            const float2 pb = st.posA[b];
            float2 rr = f2(0.0f, 0.0f);
            const int nb = st.numConn[b];
            if (nb <= 1) {
                rr = seamDiff2(pi, pb, W, H);
            } else {
                const float angleToCell = angleOfVector(seamDiff2(pi, pb, W, H));
                for (int m = 0; m < nb; ++m) {
                    const int c1 = st.bond[b * kMaxBonds + m], c2 = st.bond[b * kMaxBonds + (m + 1) % nb];
                    const float a1 = angleOfVector(seamDiff2(st.posA[c1], pb, W, H));
                    const float a2 = angleOfVector(seamDiff2(st.posA[c2], pb, W, H));
                    if (isAngleInBetween(a1, a2, angleToCell)) {
                        rr = rotCCW(st.posA[c2] - st.posA[c1]);
                        break;
                    }
                }
            }
            const float2 vb = st.velA[b];
            const float2 vr = vi - vb;
            const float dvr = dot2(vr, rr);
            if (dvr < 0.0f) {
                const float trr = fmaxf(0.05f, lensq2(rr));
                const float td = fmaxf(0.05f, bestBarrierDist);
                // (vr - rr*2*dvr/trr + vb - vi) / td of CellProcessor.cuh:272 with
                // vr + vb - vi = 0 cancelled algebraically (the FP32 form loses
                // ~ulp(|v|)/td to that cancellation)
                F = rr * (-2.0f * dvr / trr) / td;
            }
        }
        F = F + (Fp * p->pressureStrength + Fv * p->viscosityStrength);
        st.force[g] = F;
        st.push[g] = dx;
        st.densNew[g] = dens;
        st.best[g] = best;
    }
};

// CellProcessor::calcCollisions_reconnectCells_correctOverlap,
// CellProcessor.cuh:285-365 with CellMap::executeForEach (Map.cuh:175-196,
// distance test on the uncorrected difference).  The reference adds each
// pair force to both cells from the scanning cell; here every cell gathers
// f(i,j) from its own scan and -f(j,i) from the scans that see it.  near()
// and visit() take raw = p_j - p_i as stored: candidates across the torus
// seam never pass the uncorrected test, and for |raw| <= R < W/2 the
// corrected displacement is -raw exactly.
__device__ __forceinline__ float2 collisionForce(float2 pd, float d, float2 vCell, float2 vOther, bool barrierCell,
                                                 const AlienPhysicsParams& p)
{
    const float2 vd = vCell - vOther;
    const bool approaching = dot2(pd, vd) < 0.0f;
    const float bf = barrierCell ? 2.0f : 1.0f;
    if (len2(vCell) > 0.5f && approaching) {
        const float ds = d * d + 0.25f;
        return pd * dot2(vd, pd) / (-2.0f * ds) * bf;
    }
    return normalized2(pd) * (p.cellMaxCollisionDistance - len2(pd)) * p.cellRepulsionStrength * bf;
}

struct CollisionLaw {
    const DevState* s;
    const AlienPhysicsParams* p;
    int g;
    float R, R2reject, minDist, minDist2Keep, fusionVelocity, maxBindingEnergy;
    float2 pi, vi;
    bool barrierI, visibleI, fusionI;
    float densI;
    int bondsI[kMaxBonds];
    float2 F, dx;
    int best;
    unsigned long long bestId;

    // the state near() and relevant() need (the scan), then the rest (the law)
    __device__ __forceinline__ void beginScan(const DevState& st, const WorldInfo& wi, int4 me)
    {
        s = &st;
        p = &st.params[wi.paramIndex];
        g = me.x;
        R = p->cellMaxCollisionDistance;
        R2reject = R * R * 1.0001f + 1e-6f;
        minDist = p->cellMinDistance;
        minDist2Keep = minDist * minDist * 1.0001f + 1e-6f;
        barrierI = me.y & kStageBarrier;
        const int nI = (me.y >> 4) & 0xf;
#pragma unroll
        for (int m = 0; m < kMaxBonds; ++m) bondsI[m] = m < nI ? st.bond[static_cast<long long>(g) * kMaxBonds + m] : -1;
    }

    __device__ __forceinline__ void beginLaw(const WorldInfo& wi, int4 me, float2 pos, float2 vel)
    {
        // zone values at the cell (CellProcessor.cuh:344-353)
        fusionVelocity = zoneParam<kZCellFusionVelocity>(*p, wi.W, wi.H, pos, p->cellFusionVelocity);
        maxBindingEnergy = zoneParam<kZCellMaxBindingEnergy>(*p, wi.W, wi.H, pos, p->cellMaxBindingEnergy);
        pi = pos;
        vi = vel;
        visibleI = me.y & kStageVisible;
        const int nI = (me.y >> 4) & 0xf, maxI = (me.y >> 8) & 0xff;
        densI = __int_as_float(me.z);
        fusionI = !barrierI && nI < maxI && __int_as_float(me.w) <= maxBindingEnergy;
        F = dx = f2(0.0f, 0.0f);
        best = -1;
        bestId = ~0ull;
    }

    __device__ __forceinline__ void begin(const DevState& st, const WorldInfo& wi, int4 me, float2 pos, float2 vel)
    {
        beginScan(st, wi, me);
        beginLaw(wi, me, pos, vel);
    }

    __device__ __forceinline__ bool near(float2 raw) const { return raw.x * raw.x + raw.y * raw.y <= R2reject; }
    // visit() changes nothing for the cell itself, and for a bonded partner
    // it only adds the overlap push, which needs d < minDist and a cell that
    // is not a barrier; such candidates are dropped here (the bound on q is
    // above minDist^2 by more than the rounding of sqrtf, so no candidate
    // with sqrtf(q) < minDist is dropped)
    __device__ __forceinline__ bool relevant(const int4* meta, int m, float2 raw) const
    {
        const int j = meta[m].x;
        if (j == g) return false;
        if (!isBondedTo(bondsI, j)) return true;
        return !barrierI && raw.x * raw.x + raw.y * raw.y <= minDist2Keep;
    }

    __device__ __forceinline__ void visit(int4 om, float2 vj, float2 raw)
    {
        const int j = om.x;
        if (j == g) return;
        float d;
        if (!withinRadius(raw.x * raw.x + raw.y * raw.y, R, d)) return;
        const bool visibleJ = om.y & kStageVisible;
        if (!visibleJ && !visibleI) return;
        const float2 pd = f2(-raw.x, -raw.y);
        const bool bonded = isBondedTo(bondsI, j);
        if (visibleJ) {  // i's own scan sees j
            if (!barrierI && d < minDist) dx = dx + pd * (minDist / 5.0f);
            if (!bonded) {
                F = F + collisionForce(pd, d, vi, vj, barrierI, *p);
                const float2 vd = vi - vj;
                if (fusionI && len2(vd) >= fusionVelocity && dot2(pd, vd) < 0.0f) {
                    const int nJ = (om.y >> 4) & 0xf, maxJ = (om.y >> 8) & 0xff;
                    if (nJ < maxJ && !(om.y & kStageBarrier) && __int_as_float(om.w) <= maxBindingEnergy) {
                        const unsigned long long idJ = s->id[j];
                        if (idJ < bestId) {
                            bestId = idJ;
                            best = j;
                        }
                    }
                }
            }
        }
        if (visibleI && !bonded)  // j's scan sees i and applies -f(j,i) to i
            F = F - collisionForce(raw, d, vj, vi, om.y & kStageBarrier, *p);
    }

    __device__ __forceinline__ void end()
    {
        const DevState& st = *s;
        st.force[g] = F;
        st.push[g] = dx;
        st.densNew[g] = densI;
        st.best[g] = best;
    }
};

// the pair phase of the staged cell k, neighbours from the global tile lists
// (tiles in the same row order as the regions' 3x3 scan)
template <int Motion>
__device__ __forceinline__ void pairsGlobalCell(const DevState& s, long long k)
{
    const int4 me = s.stagedMeta[k];
    const float4 mpv = s.stagedPV[k];
    const int w = (me.y >> 16) & 0xffff;
    const WorldInfo& wi = s.worlds[w];
    const float2 pi = f2(mpv.x, mpv.y);
    const int sx = slotX(pi.x, wi.W), sy = slotX(pi.y, wi.H);
    if (Motion == ALIEN_B200_MOTION_FLUID) {
        FluidLaw law;
        law.begin(s, wi, me, pi, f2(mpv.z, mpv.w));
        forEachWindowTile(wi, sx, sy, [&](long long t) {
            const uint32_t k0 = s.tileStart[t], k1 = s.tileStart[t + 1];
            for (uint32_t m = k0; m < k1; ++m) {
                const float4 opv = s.stagedPV[m];
                const float2 pd = seamDiff2(pi, f2(opv.x, opv.y), wi.W, wi.H);
                if (law.near(pd)) law.visit(s.stagedMeta[m], f2(opv.z, opv.w), pd);
            }
        });
        law.end();
    } else {
        CollisionLaw law;
        law.begin(s, wi, me, pi, f2(mpv.z, mpv.w));
        forEachWindowTile(wi, sx, sy, [&](long long t) {
            const uint32_t k0 = s.tileStart[t], k1 = s.tileStart[t + 1];
            for (uint32_t m = k0; m < k1; ++m) {
                const float4 opv = s.stagedPV[m];
                const float2 raw = f2(opv.x, opv.y) - pi;
                if (law.near(raw)) law.visit(s.stagedMeta[m], f2(opv.z, opv.w), raw);
            }
        });
        law.end();
    }
}

// Cells that the region kernels cannot stage (rows denser than the shared
// buffer, worlds too small for regions) are appended to the overflow list
// and handled by kPairsOverflow after the region kernels, one thread per
// cell, so that the region kernels carry none of this path's registers.
// The visiting order is the regions' (tiles in row order, storage order
// within a tile), so a cell's sums do not depend on the path.
__device__ __forceinline__ void pairsDefer(const DevState& s, long long k)
{
    const uint32_t at = atomicAdd(s.pairOverflowCount, 1u);
    s.pairOverflow[at] = static_cast<uint32_t>(k);  // at most one entry per staged cell
}

__global__ void __launch_bounds__(kBlock) kPairsOverflow(DevState s)
{
    const uint32_t n = *s.pairOverflowCount;
    for (uint32_t i = blockIdx.x * kBlock + threadIdx.x; i < n; i += gridDim.x * kBlock) {
        const long long k = s.pairOverflow[i];
        if (s.worlds[(s.stagedMeta[k].y >> 16) & 0xffff].motionType == ALIEN_B200_MOTION_FLUID)
            pairsGlobalCell<ALIEN_B200_MOTION_FLUID>(s, k);
        else
            pairsGlobalCell<ALIEN_B200_MOTION_COLLISION>(s, k);
    }
}

// ------------------------------------------------------- kPairsRegion ----
// One CTA per region of regW x regH tiles (up to RegionShape<Motion>: 24 x 16
// for collision worlds, 64 x 8 for fluid worlds) of one world.  It
// copies the staged records of the region and of its one-tile halo from the
// tile-sorted arrays into shared memory, all (regW+2) x (regH+2) local tiles
// in row-major order (each tile a contiguous run in storage order), so that
// the tiles of one row of a cell's window are one contiguous run.  A local
// row is at most three contiguous global runs (left halo tile, own tiles,
// right halo tile), so the copy finds its source with a search over rows.
// Fluid worlds shift halo tiles that lie across the torus seam by +-W / +-H,
// so that plain differences are the minimal-image displacements; collision
// worlds keep stored positions (the reference's distance test is on the
// uncorrected difference, so candidates across the seam never pass).
// Every cell scans only the tiles of its 3x3 window that the disc of radius
// R around it reaches (a neighbour tile is skipped when the cell is farther
// than R, plus a rounding margin, from the shared edge: such tiles hold no
// candidate within R), appending candidates that pass the cheap distance
// reject to a per-thread hit list in shared memory, and runs the pair law on
// the hits afterwards: the scan loop stays convergent across the warp, and
// the law runs once per hit instead of once per scan iteration in which any
// lane had a hit.  The scan loop holds only the state the reject needs (the
// law's accumulators start after it), and a cell with more than HitCap hits
// scans a second time, visiting on the way in the same order.  Hits are
// visited in scan order (row by row, tile by tile, storage order), the order
// of the full 3x3 scan minus candidates that the law ignores, so the FP32
// sums do not depend on the pruning.
// Rows of regions whose records exceed the shared buffer even alone, and
// worlds too small for regions, defer their cells to kPairsOverflow.
constexpr int kRegionThreads = 256;
// Region shape per motion type (tiles per region, shared-buffer records,
// hit-list entries per thread, resident CTAs per SM), from a sweep of shapes
// on the B200.  Dense regions
// are processed in bands of rows, so the buffer size bounds no world.  The
// visiting order does not depend on the shape; the FP32 results of different
// builds can still differ in the last bit where the compiler contracts
// multiply-adds differently.
template <int Motion>
struct RegionShape;
template <>
struct RegionShape<ALIEN_B200_MOTION_FLUID> {
    static constexpr int W = 64, H = 8, Cap = 1536, HitCap = 24, MinBlocks = 3;
};
template <>
struct RegionShape<ALIEN_B200_MOTION_COLLISION> {
    static constexpr int W = 24, H = 16, Cap = 1152, HitCap = 24, MinBlocks = 4;
};
// Candidate region shapes (tiles x, y) per motion type for the autotuner
// (engine.cu, Arena::autotune), each within RegionShape<Motion>; the first
// is the default.  A cell's neighbours are visited in the same order
// whatever the shape, so the choice changes no result.
constexpr int kNumRegionChoices = ALIEN_B200_REGION_CHOICES;
// (small shapes for small worlds, whose large regions are fewer than the SMs)
constexpr int kRegionChoices[2][kNumRegionChoices][2] = {
    {{64, 8}, {32, 8}, {48, 8}, {40, 8}, {24, 8}, {16, 8}},    // fluid
    {{24, 16}, {16, 16}, {24, 8}, {12, 16}, {16, 8}, {8, 8}},  // collision
};
// candidates whose positions one thread loads together in the region scan
constexpr int kScanGroup = 4;

template <int Motion>
constexpr size_t regionDynSmem()
{
    return static_cast<size_t>(RegionShape<Motion>::Cap) * (sizeof(int4) + 2 * sizeof(float2))
           + static_cast<size_t>(RegionShape<Motion>::HitCap) * kRegionThreads * sizeof(uint16_t);
}

template <int Motion>
__global__ void __launch_bounds__(kRegionThreads, RegionShape<Motion>::MinBlocks) kPairsRegion(DevState s)
{
    constexpr int kRegionCap = RegionShape<Motion>::Cap;
    constexpr int kHitCap = RegionShape<Motion>::HitCap;
    constexpr int kRegionMaxH = RegionShape<Motion>::H;
    constexpr int kRegionMaxTiles = (RegionShape<Motion>::W + 2) * (RegionShape<Motion>::H + 2);
    extern __shared__ int4 dyn[];
    int4* sMeta = dyn;
    float2* sPos = reinterpret_cast<float2*>(sMeta + kRegionCap);
    float2* sVel = sPos + kRegionCap;
    uint16_t* sHits = reinterpret_cast<uint16_t*>(sVel + kRegionCap);  // [kHitCap][kRegionThreads]
    __shared__ int tStart[kRegionMaxTiles + 1];  // shared-memory offset of each local tile
    __shared__ int tGlobal[kRegionMaxTiles];     // first sorted index of the tile
    __shared__ float2 tShift[kRegionMaxTiles];
    __shared__ int rowOwn[kRegionMaxH + 1];      // own records before own row r

    const int w = s.regionWorld[blockIdx.x];
    const WorldInfo& wi = s.worlds[w];
    if ((wi.motionType == ALIEN_B200_MOTION_FLUID) != (Motion == ALIEN_B200_MOTION_FLUID)) return;
    if (!s.counters[w].active) return;
    const int idx = blockIdx.x - wi.regionBase;
    const int rx = idx % wi.nRX, ry = idx / wi.nRX;
    const int tx0 = rx * wi.regW, ty0 = ry * wi.regH;
    const int ownW = min(wi.regW, wi.nTX - tx0), ownH = min(wi.regH, wi.nTY - ty0);

    if (!wi.regionShared) {
        // world too small for halo regions: its own tiles from global memory
        for (int ly = 0; ly < ownH; ++ly)
            for (int lx = 0; lx < ownW; ++lx) {
                const long long t = wi.tileBase + (tx0 + lx) + static_cast<long long>(ty0 + ly) * wi.nTX;
                for (uint32_t k = s.tileStart[t] + threadIdx.x; k < s.tileStart[t + 1]; k += kRegionThreads)
                    pairsDefer(s, k);
            }
        return;
    }

    const int LW = ownW + 2, LH = ownH + 2, NT = LW * LH;
    // Fluid worlds see neighbours across the torus seam as minimal images:
    // halo tiles that wrap are shifted by -+W / -+H.  A region that touches
    // the right (top) seam shifts all its other tiles down by W (H) instead
    // and leaves the wrapped halo as stored, so that every shift subtracts
    // the world size from a coordinate in its upper half, which is exact
    // (the region is narrower than half the world, and no region touches
    // both seams of an axis).  Differences are then the ones the global
    // path computes with seamDiff, bit for bit, for every region shape.
    float2 seamFlip = f2(0.0f, 0.0f);
    if (Motion == ALIEN_B200_MOTION_FLUID) {
        if (tx0 + ownW == wi.nTX) seamFlip.x = -static_cast<float>(wi.W);
        if (ty0 + ownH == wi.nTY) seamFlip.y = -static_cast<float>(wi.H);
    }
    const float2 ownShift = seamFlip;  // shift of the region's own tiles
    // 1. local tile table (row-major over the region and its halo); every
    //    thread handles a contiguous chunk of tiles for the offsets
    {
        const int chunk = (NT + kRegionThreads - 1) / kRegionThreads;
        const int c0 = min(NT, static_cast<int>(threadIdx.x) * chunk), c1 = min(NT, c0 + chunk);
        uint32_t cnt = 0;
        for (int lt = c0; lt < c1; ++lt) {
            const int lx = lt % LW, ly = lt / LW;
            int gx = tx0 - 1 + lx, gy = ty0 - 1 + ly;
            float2 sh = f2(0.0f, 0.0f);
            if (gx < 0) {
                gx += wi.nTX;
                sh.x = -static_cast<float>(wi.W);
            } else if (gx >= wi.nTX) {
                gx -= wi.nTX;
                sh.x = static_cast<float>(wi.W);
            }
            if (gy < 0) {
                gy += wi.nTY;
                sh.y = -static_cast<float>(wi.H);
            } else if (gy >= wi.nTY) {
                gy -= wi.nTY;
                sh.y = static_cast<float>(wi.H);
            }
            sh = sh + seamFlip;
            const long long t = wi.tileBase + gx + static_cast<long long>(gy) * wi.nTX;
            const uint32_t k0 = s.tileStart[t];
            const uint32_t n = s.tileStart[t + 1] - k0;
            tGlobal[lt] = static_cast<int>(k0);
            tStart[lt] = static_cast<int>(n);  // count for now
            tShift[lt] = Motion == ALIEN_B200_MOTION_FLUID ? sh : f2(0.0f, 0.0f);
            cnt += n;
        }
        uint32_t total;
        uint32_t off = blockExclusiveScanN<kRegionThreads>(cnt, &total);
        for (int lt = c0; lt < c1; ++lt) {
            const int n = tStart[lt];
            tStart[lt] = static_cast<int>(off);
            off += n;
        }
        if (threadIdx.x == 0) tStart[NT] = static_cast<int>(total);
    }
    __syncthreads();
    static_assert(kRegionMaxH < 32, "own rows are scanned by one warp");
    if (threadIdx.x < 32) {
        // own records of rows 1..r (own row segments are [tStart[r*LW+1], tStart[r*LW+ownW+1])),
        // an inclusive scan over the rows in warp 0
        const int r = threadIdx.x;
        int acc = r >= 1 && r <= ownH ? tStart[r * LW + ownW + 1] - tStart[r * LW + 1] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, acc, o);
            if (r >= o) acc += y;
        }
        if (r <= ownH) rowOwn[r] = acc;
    }
    __syncthreads();
    uint16_t* myHits = sHits + threadIdx.x;
    const float T = static_cast<float>(wi.T);
    // Own rows in bands whose local rows (the band and one halo row on either
    // side) fit the shared buffer: one band for the usual region, several for
    // a dense one.  Every thread derives the same bands from tStart.  A single
    // own row that does not fit even alone is deferred to kPairsOverflow.
    int band0 = 1;
    while (band0 <= ownH) {
        const int base = tStart[(band0 - 1) * LW];
        if (tStart[(band0 + 2) * LW] - base > kRegionCap) {
            const int ly = band0;
            for (int lx = 1; lx <= ownW; ++lx) {
                const int q = ly * LW + lx;
                const int k0 = tGlobal[q], n = tStart[q + 1] - tStart[q];
                for (int k = k0 + threadIdx.x; k < k0 + n; k += kRegionThreads) pairsDefer(s, k);
            }
            ++band0;
            continue;
        }
        int band1 = band0;  // last own row of the band
        while (band1 < ownH && tStart[(band1 + 3) * LW] - base <= kRegionCap) ++band1;
        const int end = tStart[(band1 + 2) * LW];
        // 2. copy local rows band0-1 .. band1+1: a record's local row by binary
        //    search over the row starts, then one of the row's three global runs
        for (int e = base + threadIdx.x; e < end; e += kRegionThreads) {
            int lo = band0 - 1, hi = band1 + 1;
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (tStart[mid * LW] <= e)
                    lo = mid;
                else
                    hi = mid - 1;
            }
            const int b = lo * LW;
            const int q = e < tStart[b + 1] ? b : (e < tStart[b + LW - 1] ? b + 1 : b + LW - 1);
            const int src = tGlobal[q] + (e - tStart[q]);
            const float2 sh = tShift[q];
            const float4 pv = s.stagedPV[src];
            sPos[e - base] = f2(pv.x + sh.x, pv.y + sh.y);
            sVel[e - base] = f2(pv.z, pv.w);
            sMeta[e - base] = s.stagedMeta[src];
        }
        __syncthreads();
        // 3. pair law of every own cell of the band against the tiles its
        //    disc reaches (shared-memory index = record offset - base)
        int ly = band0;  // own row of o; o only grows, so the search continues from the last row
        for (int o = rowOwn[band0 - 1] + threadIdx.x; o < rowOwn[band1]; o += kRegionThreads) {
            while (rowOwn[ly] <= o) ++ly;
            const int e = tStart[ly * LW + 1] + (o - rowOwn[ly - 1]) - base;
            const float2 pi = sPos[e];
            const float2 piG = pi - ownShift;  // the stored position (exact)
            // own tile column as binned (own tiles are not shifted)
            const int gx = slotX(piG.x, wi.W) / wi.T;
            const int lx = min(max(gx - tx0 + 1, 1), ownW);
            const int gy = ty0 + ly - 1;
            auto scan = [&](auto& law, auto diff) {
                const int4 me = sMeta[e];
                law.beginScan(s, wi, me);
                // reach: R plus a margin above the rounding of positions up to the world size
                const float reach = law.R * 1.0001f + 1e-3f + 4.0f * static_cast<float>(max(wi.W, wi.H)) * 1.2e-7f;
                const float left = static_cast<float>(gx) * T, right = fminf(static_cast<float>(gx + 1) * T, static_cast<float>(wi.W));
                const float bottom = static_cast<float>(gy) * T, top = fminf(static_cast<float>(gy + 1) * T, static_cast<float>(wi.H));
                const int c0 = lx - (piG.x - reach < left ? 1 : 0), c1 = lx + (piG.x + reach >= right ? 1 : 0);
                const int r0 = ly - (piG.y - reach < bottom ? 1 : 0), r1 = ly + (piG.y + reach >= top ? 1 : 0);
                // scan: the hits in scan order (the first kHitCap kept, all
                // counted).  Candidates go in groups of kScanGroup: the
                // group's positions are loaded before any of its hits is
                // stored (the hit list shares the shared-memory buffer, so
                // a load after a store could not be moved ahead of it), then
                // its hits are appended in order
                int nh = 0;
                auto push = [&](int m) {
                    if (nh < kHitCap) myHits[nh * kRegionThreads] = static_cast<uint16_t>(m);
                    ++nh;
                };
                if (Motion == ALIEN_B200_MOTION_FLUID) {
                    // Fluid: the window's rows are one stream of candidates,
                    // in row order and record order within a row, grouped
                    // across the row boundaries, so that lanes with rows of
                    // different lengths stay together and only the stream's
                    // last group is partly empty (fluid1m's pair kernel
                    // 0.108 -> 0.104 ms; the collision kernel, with fewer
                    // registers to spare, was slower this way)
                    const int rows = r1 - r0 + 1;
                    const int s0 = tStart[r0 * LW + c0] - base, e0 = tStart[r0 * LW + c1 + 1] - base;
                    const int s1 = rows > 1 ? tStart[(r0 + 1) * LW + c0] - base : 0;
                    const int e1 = rows > 1 ? tStart[(r0 + 1) * LW + c1 + 1] - base : 0;
                    const int s2 = rows > 2 ? tStart[(r0 + 2) * LW + c0] - base : 0;
                    const int e2 = rows > 2 ? tStart[(r0 + 2) * LW + c1 + 1] - base : 0;
                    const int n0 = e0 - s0, n01 = n0 + (e1 - s1), total = n01 + (e2 - s2);
                    // record of stream position i (i < total)
                    auto record = [&](int i) { return i < n0 ? s0 + i : (i < n01 ? s1 + (i - n0) : s2 + (i - n01)); };
#pragma unroll 1
                    for (int i0 = 0; i0 < total; i0 += kScanGroup) {
                        int mm[kScanGroup];
#pragma unroll
                        for (int u = 0; u < kScanGroup; ++u) mm[u] = record(min(i0 + u, total - 1));
                        float2 dm[kScanGroup];
#pragma unroll
                        for (int u = 0; u < kScanGroup; ++u) dm[u] = diff(mm[u]);
                        bool cand[kScanGroup];
#pragma unroll
                        for (int u = 0; u < kScanGroup; ++u) cand[u] = i0 + u < total && law.near(dm[u]);
#pragma unroll
                        for (int u = 0; u < kScanGroup; ++u)
                            if (cand[u] && law.relevant(sMeta, mm[u], dm[u])) push(mm[u]);
                    }
                } else {
#pragma unroll 1
                    for (int r = r0; r <= r1; ++r) {
                        const int b0 = tStart[r * LW + c0] - base, b1 = tStart[r * LW + c1 + 1] - base;
#pragma unroll 1
                        for (int m0 = b0; m0 < b1; m0 += kScanGroup) {
                            float2 dm[kScanGroup];
#pragma unroll
                            for (int u = 0; u < kScanGroup; ++u) dm[u] = diff(min(m0 + u, b1 - 1));
                            bool cand[kScanGroup];
#pragma unroll
                            for (int u = 0; u < kScanGroup; ++u) cand[u] = m0 + u < b1 && law.near(dm[u]);
#pragma unroll
                            for (int u = 0; u < kScanGroup; ++u)
                                if (cand[u] && law.relevant(sMeta, m0 + u, dm[u])) push(m0 + u);
                        }
                    }
                }
                // law over the hits; a cell with more hits than the list holds
                // scans again and visits on the way, in the same order
                law.beginLaw(wi, me, piG, sVel[e]);
                if (nh <= kHitCap) {
                    for (int i = 0; i < nh; ++i) {
                        const int m = myHits[i * kRegionThreads];
                        law.visit(sMeta[m], sVel[m], diff(m));
                    }
                } else {
#pragma unroll 1
                    for (int r = r0; r <= r1; ++r) {
                        const int b0 = tStart[r * LW + c0] - base, b1 = tStart[r * LW + c1 + 1] - base;
                        for (int m = b0; m < b1; ++m) {
                            const float2 dm = diff(m);
                            if (law.near(dm) && law.relevant(sMeta, m, dm)) law.visit(sMeta[m], sVel[m], dm);
                        }
                    }
                }
                law.end();
            };
            if (Motion == ALIEN_B200_MOTION_FLUID) {
                FluidLaw law;
                scan(law, [&](int m) { return pi - sPos[m]; });
            } else {
                CollisionLaw law;
                scan(law, [&](int m) { return sPos[m] - pi; });
            }
        }
        __syncthreads();  // the next band overwrites the buffer
        band0 = band1 + 1;
    }
}

// ------------------------------------------------------- bond forces -----
// CellProcessor::calcConnectionForces, CellProcessor.cuh:408-491: spring
// forces in bond order; angle forces (every third step) are scattered to
// the two partners as fixed-point integers into angleAcc[4*j + accOffset].
// The bond row of a cell and its partners' positions and stiffnesses are
// gathered first (all loads of a cell in flight together), then the forces
// are summed in bond order.
struct BondRow {
    int n;
    int j[kMaxBonds];
    float2 disp[kMaxBonds];  // corrected partner - cell
};

// the bond vectors at the step's current positions: the minimal-image
// difference of the step-start positions (exact for partners, also across
// the seam) plus the difference of the in-step displacements D (the overlap
// push before the Verlet update, the total displacement after it)
__device__ __forceinline__ void loadBondRow(const DevState& s, long long g, int n, const float2* __restrict__ D, int W, int H,
                                            BondRow& r)
{
    r.n = n;
    const int2* row = reinterpret_cast<const int2*>(s.bond + g * kMaxBonds);
    const float2 pi = s.posA[g], di = D[g];
#pragma unroll
    for (int h = 0; h < kMaxBonds / 2; ++h) {
        const int2 jj = 2 * h < r.n ? row[h] : make_int2(0, 0);
        r.j[2 * h] = jj.x;
        r.j[2 * h + 1] = jj.y;
    }
    float2 pj[kMaxBonds], dj[kMaxBonds];
#pragma unroll
    for (int k = 0; k < kMaxBonds; ++k) {
        pj[k] = k < r.n ? s.posA[r.j[k]] : pi;
        dj[k] = k < r.n ? D[r.j[k]] : di;
    }
#pragma unroll
    for (int k = 0; k < kMaxBonds; ++k) r.disp[k] = seamDiff2(pj[k], pi, W, H) + (dj[k] - di);
}

// the triangle test of the angle forces depends only on the bond rows, which
// do not change between the two bond-force kernels of a step: the first
// computes and stores it, the second reads it back
enum TriMode { kTriStore, kTriLoad };

__device__ __forceinline__ float2 bondForce(const DevState& s, long long g, const BondRow& r, bool considerAngles,
                                            float minDist, int accOffset, TriMode triMode)
{
    float2 F = f2(0.0f, 0.0f);
    const int n = r.n;
    if (n == 0 || s.barrier[g]) return F;
    const long long bb = g * kMaxBonds;
    const float si = s.stiffness[g];
    const float s2 = si * si;
    float sj[kMaxBonds], bd[kMaxBonds], len[kMaxBonds];
    float2 nrm[kMaxBonds];  // Math::normalized: unit vector, (1, 0) below NEAR_ZERO
    const float2* bdRow = reinterpret_cast<const float2*>(s.bondDist + bb);
#pragma unroll
    for (int h = 0; h < kMaxBonds / 2; ++h) {
        const float2 d = 2 * h < n ? bdRow[h] : f2(0.0f, 0.0f);
        bd[2 * h] = d.x;
        bd[2 * h + 1] = d.y;
    }
#pragma unroll
    for (int k = 0; k < kMaxBonds; ++k) sj[k] = k < n ? s.stiffness[r.j[k]] : 0.0f;
#pragma unroll
    for (int k = 0; k < kMaxBonds; ++k) {
        len[k] = len2(r.disp[k]);
        const float inv = __frcp_rn(len[k]);
        nrm[k] = len[k] > kNearZero ? r.disp[k] * inv : f2(1.0f, 0.0f);
    }
    // spring forces in bond order: normalized(d) * (|d| - rest) * (s_i^2 + s_j^2) / 6
#pragma unroll
    for (int k = 0; k < kMaxBonds; ++k)
        if (k < n) F = F + nrm[k] * ((len[k] - bd[k]) * (s2 + sj[k] * sj[k]) * (1.0f / 6.0f));
    if (!considerAngles || n < 2) return F;
    // angle forces: partner rows for the triangle test, then the forces in bond order
    int nj[kMaxBonds];
    float ang[kMaxBonds];  // angle of every bond vector, once
    unsigned triBits = triMode == kTriLoad ? s.triMask[g] : 0u;
#pragma unroll
    for (int k = 0; k < kMaxBonds; ++k) nj[k] = triMode == kTriStore && k < n ? s.numConn[r.j[k]] : 0;
#pragma unroll
    for (int k = 0; k < kMaxBonds; ++k) {
        const float a = 90.0f - atan2f(-r.disp[k].y, r.disp[k].x) * (180.0f / kPi);
        ang[k] = k < n && len[k] >= kNearZero ? (a < 0.0f ? a + 360.0f : a) : 0.0f;
    }
#pragma unroll
    for (int k = 0; k < kMaxBonds; ++k) {
        if (k >= n || !(n > 2 || k == 0)) continue;
        const int last = k == 0 ? n - 1 : k - 1;
        int jl = r.j[0];
        float pa = ang[0], lenPrev = len[0];
        float2 nrmPrev = nrm[0];
#pragma unroll
        for (int m = 1; m < kMaxBonds; ++m)
            if (m == last) {
                jl = r.j[m];
                pa = ang[m];
                lenPrev = len[m];
                nrmPrev = nrm[m];
            }
        const int j = r.j[k];
        bool tri;
        if (triMode == kTriLoad) {
            tri = (triBits >> k) & 1u;
        } else {
            const int2* prow = reinterpret_cast<const int2*>(s.bond + static_cast<long long>(j) * kMaxBonds);
            tri = false;
#pragma unroll
            for (int h = 0; h < kMaxBonds / 2; ++h) {
                if (2 * h < nj[k]) {
                    const int2 pp = prow[h];
                    tri |= pp.x == jl;
                    tri |= (2 * h + 1 < nj[k]) && pp.y == jl;
                }
            }
            if (tri) triBits |= 1u << k;
        }
        if (tri) continue;
        const float act = subtractAngle(ang[k], pa);
        if (act < 0.0f) continue;
        const float ref = s.bondAngle[bb + k];
        const float strength = fabsf(ref - act) * (1.0f / 2000.0f) * s2;
        const float sign = ref < act ? -1.0f : 1.0f;
        const float2 f1 = rotCW(nrm[k] * (sign * strength * __frcp_rn(fmaxf(len[k], minDist))));
        const float2 f2v = rotCCW(nrmPrev * (sign * strength * __frcp_rn(fmaxf(lenPrev, minDist))));
        if (!s.barrier[j]) {
            atomicAdd(reinterpret_cast<unsigned long long*>(&s.angleAcc[4LL * j + accOffset]),
                      static_cast<unsigned long long>(toFix(f1.x)));
            atomicAdd(reinterpret_cast<unsigned long long*>(&s.angleAcc[4LL * j + accOffset + 1]),
                      static_cast<unsigned long long>(toFix(f1.y)));
        }
        if (!s.barrier[jl]) {
            atomicAdd(reinterpret_cast<unsigned long long*>(&s.angleAcc[4LL * jl + accOffset]),
                      static_cast<unsigned long long>(toFix(f2v.x)));
            atomicAdd(reinterpret_cast<unsigned long long*>(&s.angleAcc[4LL * jl + accOffset + 1]),
                      static_cast<unsigned long long>(toFix(f2v.y)));
        }
        F = F - (f1 + f2v);
    }
    if (triMode == kTriStore) s.triMask[g] = static_cast<uint8_t>(triBits);
    return F;
}

// verletPositionUpdate (CellProcessor.cuh:525-544) of cell g as an
// increment: its overlap push plus
// v * dt + F * dt^2 / 2 with the bond force F1 and the fixed-point angle
// forces (ax, ay); stores the total force of a non-barrier cell and returns
// the cell's displacement since the step start.  The position itself is
// rounded once, when the next step folds the displacement in.
__device__ __forceinline__ float2 verletIncrement(const DevState& s, long long g, const AlienPhysicsParams& p, bool barrierG,
                                                  float2 v, float2 F1, long long ax, long long ay)
{
    const float dt = p.timestepSize;
    const float2 d = s.push[g];
    if (barrierG) {
        s.force1[g] = F1;
        return d + v * dt;
    }
    const float2 F = F1 + f2(fromFix(ax), fromFix(ay));
    s.force1[g] = F;
    return d + (v * dt + F * dt * dt / 2.0f);
}

// -------------------------------------------------------- kApplyBond1 ----
// cells: checkForces + applyForces (CellProcessor.cuh:367-406), bond forces
// #1 at the overlap-corrected positions.  particles: movement
// (RadiationProcessor::movement, RadiationProcessor.cuh:61-70).
__global__ void __launch_bounds__(kBlock, 5) kApplyBond1(DevState s)
{
    if (blockIdx.x < s.numCellBlocks) {
        // own fields before the world lookup and the first store (every
        // launched cell slot lies inside the arena; no other cell writes
        // them in this kernel)
        const long long g0 = static_cast<long long>(blockIdx.x) * kBlock + threadIdx.x;
        const bool barrierG = s.barrier[g0];
        const int n = s.numConn[g0];
        const int col = s.color[g0] % ALIEN_B200_MAX_COLORS;
        float2 F = s.force[g0];
        float2 v = s.velA[g0];
        CellCtx c = cellCtx(s);
        if (!c.valid) return;
        const long long g = c.g;
        const WorldInfo& wi = s.worlds[c.w];
        const AlienPhysicsParams& p = s.params[wi.paramIndex];
        const uint64_t T = s.counters[c.w].timestep;
        if (!barrierG) {
            float maxForce = p.cellMaxForce[col];
            if (p.numZones > 0) {
                // the cell where the reference's applyForces finds it: after
                // the overlap push; flow fields (FlowFieldKernels.cu:48-70)
                // add to the pair force before checkForces reads it
                const float2 pushed = correctPosition(s.posA[g] + s.push[g], wi.W, wi.H);
                F = F + flowAcceleration(p, pushed, wi.W, wi.H);
                maxForce = zoneParam<kZCellMaxForce>(p, wi.W, wi.H, pushed, maxForce, col);
            }
            if (len2(F) > maxForce) {
                if (draw(s.id[g], T, kSiteForceDecay) < p.cellMaxForceDecayProb) atomicOr(&s.flags[g], kFlagDelAll);
            }
            v = v + F;
            if (len2(v) > p.cellMaxVelocity) v = normalized2(v) * p.cellMaxVelocity;
            s.velA[g] = v;
        }
        BondRow r;
        loadBondRow(s, g, n, s.push, wi.W, wi.H, r);
        const float2 F1 = bondForce(s, g, r, T % 3 == 0, p.cellMinDistance, 0, kTriStore);
        if (T % 3 == 0) {
            s.force1[g] = F1;  // angle forces of other cells still arrive: kVerletPos
        } else {
            // no angle forces this step: verletPositionUpdate here, with the
            // arithmetic of kVerletPos for empty accumulators
            s.dpos[g] = verletIncrement(s, g, p, barrierG, v, F1, 0, 0);
        }
        if (p.motionType == ALIEN_B200_MOTION_FLUID) s.density[g] = s.densNew[g];
    } else {
        forParticleBlocks(s, usedParticles, [&](const PartCtx& c, int) {
            if (!c.inRange || !s.palive[c.q]) return;
            const WorldInfo& wi = s.worlds[c.w];
            const AlienPhysicsParams& p = s.params[wi.paramIndex];
            float2 v = s.pvel[c.q];
            if (p.numZones > 0) {  // flow fields (FlowFieldKernels.cu:71-87), then movement
                v = v + flowAcceleration(p, s.ppos[c.q], wi.W, wi.H);
                s.pvel[c.q] = v;
            }
            s.ppos[c.q] = correctPosition(s.ppos[c.q] + v * p.timestepSize, wi.W, wi.H);
        });
    }
}

// --------------------------------------------------------- kVerletPos ----
// cells: verletPositionUpdate (CellProcessor.cuh:525-544) in steps with
// timestep % 3 == 0, after the angle forces of all cells have arrived; in the
// other steps kApplyBond1 has done it already.
// particles: merge target (RadiationProcessor::collision, :78-80).
__global__ void __launch_bounds__(kBlock, 8) kVerletPos(DevState s)
{
    if (blockIdx.x < s.numCellBlocks) {
        if (s.counters[s.cellBlockWorld[blockIdx.x]].timestep % 3 != 0) return;
        // own fields before the world lookup (every launched cell slot lies
        // inside the arena; no other cell writes them in this kernel)
        const long long g0 = static_cast<long long>(blockIdx.x) * kBlock + threadIdx.x;
        const bool barrierG = s.barrier[g0];
        const float2 v = s.velA[g0];
        const float2 F1 = s.force1[g0];
        const longlong2 a = *reinterpret_cast<const longlong2*>(s.angleAcc + 4 * g0);
        CellCtx c = cellCtx(s);
        if (!c.valid) return;
        const long long g = c.g;
        const WorldInfo& wi = s.worlds[c.w];
        const AlienPhysicsParams& p = s.params[wi.paramIndex];
        long long ax = 0, ay = 0;
        if (!barrierG) {
            // angle forces are scattered only in these steps and consumed here
            // (barrier cells receive none)
            ax = a.x;
            ay = a.y;
            if (ax | ay) *reinterpret_cast<longlong2*>(s.angleAcc + 4 * g) = make_longlong2(0, 0);
        }
        s.dpos[g] = verletIncrement(s, g, p, barrierG, v, F1, ax, ay);
    } else {
        forParticleBlocks(s, usedParticles, [&](const PartCtx& c, int) {
            if (!c.inRange || !s.palive[c.q]) return;
            const WorldInfo& wi = s.worlds[c.w];
            const float2 pp = s.ppos[c.q];
            const int o = s.pmap[wi.pmapBase + slotX(pp.x, wi.W) + slotX(pp.y, wi.H) * wi.W];
            if (o >= 0 && o != c.q && lensq2(pp - s.ppos[o]) < 0.5f) s.ptarget[c.q] = o;
        });
    }
}

// ------------------------------------------------------------- kBond2 ----
// cells: checkConnections (CellProcessor.cuh:493-523) at the new positions,
// bond forces #2.  particles: merges into particles that do not merge
// themselves (RadiationProcessor.cuh:82-96 under the fixed rule).
__global__ void __launch_bounds__(kBlock, 5) kBond2(DevState s)
{
    if (blockIdx.x < s.numCellBlocks) {
        // own fields before the world lookup (every launched cell slot lies
        // inside the arena; no other cell writes them in this kernel)
        const long long g0 = static_cast<long long>(blockIdx.x) * kBlock + threadIdx.x;
        const bool barrierG = s.barrier[g0];
        const int n = s.numConn[g0];
        const int col = s.color[g0] % ALIEN_B200_MAX_COLORS;
        CellCtx c = cellCtx(s);
        if (!c.valid) return;
        const long long g = c.g;
        const WorldInfo& wi = s.worlds[c.w];
        const AlienPhysicsParams& p = s.params[wi.paramIndex];
        const uint64_t T = s.counters[c.w].timestep;
        BondRow r;
        loadBondRow(s, g, n, s.dpos, wi.W, wi.H, r);
        if (!barrierG) {
            const float maxDist = p.cellMaxBindingDistance[col];
            bool destroy = false;
#pragma unroll
            for (int k = 0; k < kMaxBonds; ++k)
                if (k < r.n && len2(r.disp[k]) > maxDist) destroy = true;
            if (destroy) {
                atomicOr(&s.flags[g], kFlagDelAll);
#pragma unroll
                for (int k = 0; k < kMaxBonds; ++k)
                    if (k < r.n) atomicOr(&s.flags[r.j[k]], kFlagDetach);
            }
        }
        s.force[g] = bondForce(s, g, r, T % 3 == 0, p.cellMinDistance, 2, kTriLoad);
    } else {
        forParticleBlocks(s, usedParticles, [&](const PartCtx& c, int) {
            if (!c.inRange || !s.palive[c.q]) return;
            const long long q = c.q;
            const int o = s.ptarget[q];
            if (o < 0 || s.ptarget[o] >= 0) return;
            const float eq = s.penergy[q];
            if (!(eq > kNearZero && s.penergy[o] > kNearZero)) return;
            const float2 vq = s.pvel[q];
            atomicOr(&s.pflag[o], 1u);
            atomicAdd(reinterpret_cast<unsigned long long*>(&s.pmerge[3LL * o + 0]), static_cast<unsigned long long>(toFix(eq)));
            atomicAdd(reinterpret_cast<unsigned long long*>(&s.pmerge[3LL * o + 1]), static_cast<unsigned long long>(toFix(eq * vq.x)));
            atomicAdd(reinterpret_cast<unsigned long long*>(&s.pmerge[3LL * o + 2]), static_cast<unsigned long long>(toFix(eq * vq.y)));
            s.palive[q] = 0;
            atomicAdd(&s.counters[c.w].deadParticles, 1u);
        });
    }
}

// head cell (rank 0) of a slot, from the staged tile lists
__device__ __forceinline__ int slotHead(const DevState& s, const WorldInfo& wi, float2 pos)
{
    const int sx = slotX(pos.x, wi.W), sy = slotX(pos.y, wi.H);
    const long long t = wi.tileBase + sx / wi.T + static_cast<long long>(sy / wi.T) * wi.nTX;
    const uint32_t k0 = s.tileStart[t], k1 = s.tileStart[t + 1];
    for (uint32_t m = k0; m < k1; ++m) {
        const int4 om = s.stagedMeta[m];
        if (!(om.y & kStageHead)) continue;
        const float4 opv = s.stagedPV[m];
        if (slotX(opv.x, wi.W) == sx && slotX(opv.y, wi.H) == sy) return om.x;
    }
    return -1;
}

// --------------------------------------------------------- kVerletVel ----
// cells: verletVelocityUpdate (CellProcessor.cuh:546-559), detaching from
// checkConnections, aging (CellProcessor.cuh:561-593).
// particles: merged particles, absorption into / reflection at the cell
// under the particle (RadiationProcessor.cuh:97-168).
__global__ void __launch_bounds__(kBlock, 8) kVerletVel(DevState s)
{
    if (blockIdx.x < s.numCellBlocks) {
        // the cell's own fields are loaded before the world lookup and the
        // first store (every launched cell slot lies inside the arena, and
        // the cell part writes only the cell's own fields)
        const long long g0 = static_cast<long long>(blockIdx.x) * kBlock + threadIdx.x;
        const float2 v = s.velA[g0];
        const bool barrierG = s.barrier[g0];
        const float2 F = s.force[g0];
        const float2 F1 = s.force1[g0];
        const int ls0 = s.livingState[g0];
        const uint32_t fl = s.flags[g0];
        const uint32_t age = s.age[g0];
        const uint32_t at = s.activationTime[g0];
        CellCtx c = cellCtx(s);
        if (!c.valid) return;
        const long long g = c.g;
        const WorldInfo& wi = s.worlds[c.w];
        const AlienPhysicsParams& p = s.params[wi.paramIndex];
        if (barrierG) {
            s.velB[g] = v;
        } else {
            long long ax = 0, ay = 0;
            if (s.counters[c.w].timestep % 3 == 0) {
                const longlong2 a = *reinterpret_cast<const longlong2*>(s.angleAcc + 4 * g + 2);
                ax = a.x;
                ay = a.y;
                if (ax | ay) *reinterpret_cast<longlong2*>(s.angleAcc + 4 * g + 2) = make_longlong2(0, 0);
            }
            const float2 F2 = F + f2(fromFix(ax), fromFix(ay));
            s.velB[g] = v + (F2 + F1) / 2.0f * p.timestepSize;
        }
        int ls = ls0;
        if (fl & kFlagDetach) {
            ls = ALIEN_B200_LIVING_DETACHING;
            s.livingState[g] = static_cast<uint8_t>(ls);
        }
        if (!barrierG) {
            s.age[g] = age + 1;
            if (ls == ALIEN_B200_LIVING_READY && at > 0) s.activationTime[g] = at - 1;
        }
    } else {
        forParticleBlocks(s, usedParticles, [&](const PartCtx& c, int) {
            if (!c.inRange || !s.palive[c.q]) return;
            const long long q = c.q;
            const WorldInfo& wi = s.worlds[c.w];
            const AlienPhysicsParams& p = s.params[wi.paramIndex];
            if (s.pflag[q] & 1u) {
                const float eq = s.penergy[q];
                const float e = eq + fromFix(s.pmerge[3 * q + 0]);
                const float2 vq = s.pvel[q];
                s.pvel[q] = f2((eq * vq.x + fromFix(s.pmerge[3 * q + 1])) / e, (eq * vq.y + fromFix(s.pmerge[3 * q + 2])) / e);
                s.penergy[q] = e;
                s.plast[q] = ~0ull;
                return;
            }
            if (s.ptarget[q] >= 0) return;
            const float2 pp = s.ppos[q], pv = s.pvel[q];
            const int cell = slotHead(s, wi, pp + pv);
            if (cell < 0) return;
            if (s.barrier[cell]) {
                const float2 vc = s.velA[cell];
                const float2 vr = pv - vc;
                // the cell where the particle phase finds it: after the overlap push
                const float2 r = seamDiff2(pp, s.posA[cell], wi.W, wi.H) - s.push[cell];
                const float dvr = dot2(vr, r);
                if (dvr < 0.0f) {
                    const float trr = fmaxf(0.1f, lensq2(r));
                    s.pvel[q] = vr - r * 2.0f * dvr / trr + vc;
                }
                return;
            }
            const unsigned long long cellId = s.id[cell];
            if (s.plast[q] == cellId) return;
            const int cellColor = s.color[cell] % ALIEN_B200_MAX_COLORS;
            float absorption = p.radiationAbsorption[cellColor];
            if (p.numZones > 0)  // at the cell after the overlap push (RadiationProcessor.cuh:111-116)
                absorption = zoneParam<kZRadiationAbsorption>(p, wi.W, wi.H, correctPosition(s.posA[cell] + s.push[cell], wi.W, wi.H),
                                                              absorption, cellColor);
            if (absorption < kNearZero) return;
            float e = s.penergy[q];
            float transfer = e * absorption;
            if (e < 0.01f) transfer = e;
            atomicAdd(reinterpret_cast<unsigned long long*>(&s.energyAcc[cell]), static_cast<unsigned long long>(toFix(transfer)));
            e -= transfer;
            s.penergy[q] = e;
            if (e < kNearZero) {
                s.palive[q] = 0;
                atomicAdd(&s.counters[c.w].deadParticles, 1u);
            } else {
                s.plast[q] = cellId;
            }
        });
    }
}

// -------------------------------------------------------- kTransition ----
// cells: living-state transition (CellProcessor.cuh:596-664; the new state
// is applied in kResolve, after every cell has read its partners' states),
// absorbed energy, inner friction (every third step: one Jacobi sweep with
// one pair average per bond, CellProcessor.cuh:678-705), friction and decay.
// particles: splitting (RadiationProcessor::splitting, :172-204).
__global__ void __launch_bounds__(kBlock, 5) kTransition(DevState s)
{
    if (blockIdx.x < s.numCellBlocks) {
        // the cell's own fields are loaded before the world lookup and the
        // first store (every launched cell slot lies inside the arena; the
        // cell part reads no field that another cell writes in this kernel)
        const long long g0 = static_cast<long long>(blockIdx.x) * kBlock + threadIdx.x;
        const int n = s.numConn[g0];
        const uint32_t cr = s.creatureId[g0];
        const float2 vi = s.velB[g0];
        const int orig = s.livingState[g0];
        const bool barrierG = s.barrier[g0];
        const long long ea = s.energyAcc[g0];
        const float e0 = s.energy[g0];
        const int col = s.color[g0] % ALIEN_B200_MAX_COLORS;
        const uint32_t age = s.age[g0];
        CellCtx c = cellCtx(s);
        if (!c.valid) return;
        const long long g = c.g;
        const WorldInfo& wi = s.worlds[c.w];
        const AlienPhysicsParams& p = s.params[wi.paramIndex];
        const uint64_t T = s.counters[c.w].timestep;
        const bool innerFriction = T % 3 == 0;  // SimulationKernelsLauncher.cu:32
        bool sameDetaching = false, otherDetaching = false, sameReviving = false, activating = false;
        float2 acc = f2(0.0f, 0.0f);
        // the bond row, then the partners' states (and velocities on inner-
        // friction steps) with all loads of a cell in flight together
        int jb[kMaxBonds];
        const int2* row = reinterpret_cast<const int2*>(s.bond + g * kMaxBonds);
#pragma unroll
        for (int h = 0; h < kMaxBonds / 2; ++h) {
            const int2 jj = 2 * h < n ? row[h] : make_int2(0, 0);
            jb[2 * h] = jj.x;
            jb[2 * h + 1] = jj.y;
        }
        int lsj[kMaxBonds];
        uint32_t crj[kMaxBonds];
#pragma unroll
        for (int k = 0; k < kMaxBonds; ++k) {
            lsj[k] = k < n ? s.livingState[jb[k]] : ALIEN_B200_LIVING_READY;
            crj[k] = k < n ? s.creatureId[jb[k]] : cr;
        }
#pragma unroll
        for (int k = 0; k < kMaxBonds; ++k) {
            if (k >= n) continue;
            const int ls = lsj[k];
            if (crj[k] == cr) {
                if (ls == ALIEN_B200_LIVING_DETACHING) sameDetaching = true;
                else if (ls == ALIEN_B200_LIVING_REVIVING) sameReviving = true;
                else if (ls == ALIEN_B200_LIVING_ACTIVATING) activating = true;
            } else if (ls == ALIEN_B200_LIVING_DETACHING) {
                otherDetaching = true;
            }
        }
        if (innerFriction) {
            float2 vj[kMaxBonds];
            uint8_t bj[kMaxBonds];
#pragma unroll
            for (int k = 0; k < kMaxBonds; ++k) {
                bj[k] = k < n ? s.barrier[jb[k]] : 1;
                vj[k] = k < n ? s.velB[jb[k]] : vi;
            }
#pragma unroll
            for (int k = 0; k < kMaxBonds; ++k)
                if (k < n && !bj[k]) acc = acc + (vj[k] - vi);
        }
        int ls = orig;
        const int dc = p.cellDeathConsequences;
        if (barrierG)
            ls = ALIEN_B200_LIVING_READY;
        else if (orig == ALIEN_B200_LIVING_ACTIVATING || orig == ALIEN_B200_LIVING_REVIVING)
            ls = ALIEN_B200_LIVING_READY;
        else if (orig == ALIEN_B200_LIVING_UNDER_CONSTRUCTION) {
            if (activating) ls = ALIEN_B200_LIVING_ACTIVATING;
            if (otherDetaching && dc != ALIEN_B200_DEATH_NONE) ls = ALIEN_B200_LIVING_DETACHING;
        } else if (orig == ALIEN_B200_LIVING_DETACHING) {
            if (sameReviving && dc == ALIEN_B200_DEATH_DETACHED_PARTS_DIE) ls = ALIEN_B200_LIVING_REVIVING;
            if (dc == ALIEN_B200_DEATH_NONE) ls = ALIEN_B200_LIVING_READY;
        } else if (orig == ALIEN_B200_LIVING_READY) {
            if (sameDetaching && dc != ALIEN_B200_DEATH_NONE) ls = ALIEN_B200_LIVING_DETACHING;
        }
        s.nextState[g] = static_cast<uint8_t>(ls);
        float e = e0;
        if (ea) {
            e += fromFix(ea);
            s.energy[g] = e;
            s.energyAcc[g] = 0;
        }
        if (barrierG) {
            s.velA[g] = vi;
            return;
        }
        // zone values at the cell's position after the Verlet update
        float friction = p.friction, maxBindingEnergy = p.cellMaxBindingEnergy;
        float deathProbability = p.cellDeathProbability[col], minEnergy = p.cellMinEnergy[col];
        if (p.numZones > 0) {
            const float2 pos = stepPos(s, g, wi.W, wi.H);
            friction = zoneParam<kZFriction>(p, wi.W, wi.H, pos, friction);
            maxBindingEnergy = zoneParam<kZCellMaxBindingEnergy>(p, wi.W, wi.H, pos, maxBindingEnergy);
            deathProbability = zoneParam<kZCellDeathProbability>(p, wi.W, wi.H, pos, deathProbability, col);
            minEnergy = zoneParam<kZCellMinEnergy>(p, wi.W, wi.H, pos, minEnergy, col);
        }
        // applyInnerFriction (every third step) + applyFriction
        // (CellProcessor.cuh:678-723)
        const float2 vf = innerFriction ? vi + acc * (p.innerFriction / 2.0f) : vi;
        s.velA[g] = vf * (1.0f - friction);
        // decay (CellProcessor.cuh:775-858) on the state after the transition
        uint32_t f = 0;
        if (e > maxBindingEnergy) f |= kFlagDelAll;
        if (ls == ALIEN_B200_LIVING_DYING || ls == ALIEN_B200_LIVING_DETACHING) {
            if (draw(s.id[g], T, kSiteDeath) < deathProbability) f |= kFlagDelCell;
        }
        bool destroy = e < minEnergy;
        const long long maxAge = p.cellMaxAge[col];
        if (maxAge > 0 && static_cast<long long>(age) > maxAge) destroy = true;
        if (destroy) {
            f |= kFlagSetDying;
            if (ls != ALIEN_B200_LIVING_DYING) {
                f |= kFlagNewDying;
                for (int k = 0; k < n; ++k) atomicOr(&s.flags[s.bond[g * kMaxBonds + k]], kFlagDetachFromDying);
            }
        }
        if (f) atomicOr(&s.flags[g], f);
    } else {
        forParticleBlocks(s, usedParticles, [&](const PartCtx& c, int) {
            if (!c.inRange) return;
            const long long q = c.q;
            const WorldInfo& wi = s.worlds[c.w];
            if (s.pslot[q] >= 0) s.pmap[wi.pmapBase + s.pslot[q]] = -1;
            if (!s.palive[q]) return;
            const AlienPhysicsParams& p = s.params[wi.paramIndex];
            const uint64_t T = s.counters[c.w].timestep;
            const unsigned long long id = s.pid[q];
            if (draw(id, T, kSiteSplit) >= 0.01f) return;
            float e = s.penergy[q];
            if (!(e > p.particleSplitEnergy[s.pcolor[q] % ALIEN_B200_MAX_COLORS])) return;
            e *= 0.5f;
            s.penergy[q] = e;
            float2 vp = unitVectorOfAngle(draw(id, T, kSiteSplitAngle) * 360.0f);
            const float2 pp = s.ppos[q];
            const float2 otherPos = correctPosition(pp + vp / 5.0f, wi.W, wi.H);
            s.ppos[q] = correctPosition(pp - vp / 5.0f, wi.W, wi.H);
            vp = vp * (p.radiationVelocityPerturbation / (e + 1.0f));
            const float2 pv = s.pvel[q];
            s.pvel[q] = pv - vp;
            if (e > kNearZero) {
                s.splitPos[q] = otherPos;
                s.splitVel[q] = pv + vp;
                s.splitEnergy[q] = e;
                s.pflag[q] |= 2u;
            }
        });
    }
}

// ------------------------------------------------------------ kNeuron ----
// The neuron cell function: CellFunctionProcessor::collectCellFunctionOperations
// (CellFunctionProcessor.cuh:33-50) selects the cells whose execution order
// number is timestep % cellNumExecutionOrderNumbers, that are neither under
// construction nor activating and whose activation time is 0;
// NeuronProcessor::processCell (NeuronProcessor.cuh:33-74) sums the signals of
// the bonded cells of the cell's input execution order number
// (CellFunctionProcessor::calcInputSignal, :128-164; each channel clamped to
// [-10, 10] after every addition, in bond order), marks the function used
// (updateInvocationState, :176-186), and writes act(W x + b).  Inputs never run
// in the same step as the cells reading them (a different execution order
// number), so reading and writing signals in one pass needs no snapshot.  The
// matrix-vector sum runs in column order (the reference adds the 64 products
// with shared-memory atomics in arbitrary order).
constexpr int kNeuronTableStride = ALIEN_B200_MAX_CHANNELS * (ALIEN_B200_MAX_CHANNELS + 1);

__device__ __forceinline__ float neuronActivation(int function, float x)
{
    switch (function) {
    case 0: return 2.0f / (1.0f + expf(-x)) - 1.0f;       // sigmoid
    case 1: return x >= kNearZero ? 1.0f : 0.0f;          // binary step
    case 2: return fmaxf(-1.0f, fminf(1.0f, x));         // identity
    case 3: return fminf(1.0f, fabsf(x));                 // abs
    case 4: return expf(-2.0f * x * x);                   // gaussian
    }
    return 0.0f;
}

// a float of the auxiliary data at any byte offset (the reference's
// converter does not promise 4-byte alignment)
__device__ __forceinline__ float auxFloat(const uint8_t* p, bool aligned)
{
    if (aligned) return *reinterpret_cast<const float*>(p);
    const uint32_t u = static_cast<uint32_t>(p[0]) | static_cast<uint32_t>(p[1]) << 8 | static_cast<uint32_t>(p[2]) << 16
                       | static_cast<uint32_t>(p[3]) << 24;
    return __uint_as_float(u);
}

__global__ void __launch_bounds__(kBlock) kNeuron(DevState s)
{
    CellCtx c = cellCtx(s);
    if (!c.valid) return;
    const long long g = c.g;
    const uchar4 fi = s.fnInfo[g];
    if (fi.x != 1) return;
    const int w = c.w;
    const WorldCounters& wc = s.counters[w];
    const AlienPhysicsParams& p = s.params[w];
    if (static_cast<uint64_t>(fi.y) != wc.timestep % static_cast<uint64_t>(p.cellNumExecutionOrderNumbers)) return;
    const int ls = s.livingState[g];
    if (ls == ALIEN_B200_LIVING_UNDER_CONSTRUCTION || ls == ALIEN_B200_LIVING_ACTIVATING || s.activationTime[g] != 0) return;
    AlienCellTO& me = s.cold[s.coldIdx[g]];

    float in[ALIEN_B200_MAX_CHANNELS];
#pragma unroll
    for (int ch = 0; ch < ALIEN_B200_MAX_CHANNELS; ++ch) in[ch] = 0.0f;
    uint8_t origin = 0;
    float tx = 0.0f, ty = 0.0f;
    const int inputOrder = static_cast<int8_t>(fi.z);
    if (inputOrder != -1 && inputOrder != static_cast<int>(fi.y)) {
        int sensors = 0;
        const int n = s.numConn[g];
        for (int k = 0; k < n; ++k) {
            const int j = s.bond[g * kMaxBonds + k];
            const uchar4 fj = s.fnInfo[j];
            const int lsj = s.livingState[j];
            if (fj.w || lsj == ALIEN_B200_LIVING_UNDER_CONSTRUCTION || lsj == ALIEN_B200_LIVING_ACTIVATING) continue;
            if (static_cast<int>(fj.y) != inputOrder) continue;
            const AlienSignalTO& sig = s.cold[s.coldIdx[j]].signal;
#pragma unroll
            for (int ch = 0; ch < ALIEN_B200_MAX_CHANNELS; ++ch) in[ch] = fmaxf(-10.0f, fminf(10.0f, in[ch] + sig.channels[ch]));
            if (sig.origin == 1) {  // SignalOrigin_Sensor
                origin = 1;
                tx += sig.targetX;
                ty += sig.targetY;
                ++sensors;
            }
        }
        if (sensors > 0) {
            tx /= static_cast<float>(sensors);
            ty /= static_cast<float>(sensors);
        }
    }
    if (me.cellFunctionUsed == 0) {
        bool used = false;
#pragma unroll
        for (int ch = 0; ch < ALIEN_B200_MAX_CHANNELS - 1; ++ch) used |= in[ch] != 0.0f;
        if (used) me.cellFunctionUsed = 1;
    }
    // NeuronFunction::NeuronState in the auxiliary data: weights [8 x 8]
    // row-major, then 8 biases (NeuronTO.weightsAndBiasesDataIndex)
    const uint8_t* wb = s.aux + s.worlds[w].auxBase + me.cellFunctionData[0];
    const bool aligned = (reinterpret_cast<uintptr_t>(wb) & 3) == 0;
    const int32_t* act = reinterpret_cast<const int32_t*>(&me.cellFunctionData[1]);  // NeuronTO.activationFunctions
    float out[ALIEN_B200_MAX_CHANNELS];
#pragma unroll
    for (int r = 0; r < ALIEN_B200_MAX_CHANNELS; ++r) {
        float sum = auxFloat(wb + 4 * (ALIEN_B200_MAX_CHANNELS * ALIEN_B200_MAX_CHANNELS + r), aligned);
#pragma unroll
        for (int col = 0; col < ALIEN_B200_MAX_CHANNELS; ++col)
            sum += auxFloat(wb + 4 * (r * ALIEN_B200_MAX_CHANNELS + col), aligned) * in[col];
        out[r] = neuronActivation(act[r], sum);
    }
#pragma unroll
    for (int r = 0; r < ALIEN_B200_MAX_CHANNELS; ++r) me.signal.channels[r] = out[r];
    me.signal.origin = origin;
    me.signal.targetX = tx;
    me.signal.targetY = ty;
    // statistics.incNumNeuronActivities (NeuronProcessor.cuh:70): one atomic
    // per warp, world and color
    const unsigned key = static_cast<unsigned>(w) * ALIEN_B200_MAX_COLORS + s.color[g] % ALIEN_B200_MAX_COLORS;
    const unsigned peers = __match_any_sync(__activemask(), key);
    if ((threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(&s.neuronActivity[key], static_cast<unsigned long long>(__popc(peers)));
}

// -------------------------------------------------------- kSignalReset ----
// CellFunctionProcessor::resetFetchedSignals (CellFunctionProcessor.cuh:69-112,
// run by the friction kernel after the cell functions, SimulationKernels.cu
// :153-158): a cell without function loses its signal channels every step; a
// cell with a function loses them in the step after the last of its readers
// ran (the bonded cells whose input execution order number is this cell's
// execution order number; without readers, the step after the cell's own).
// Reads only execution order numbers, which no step changes.
__global__ void __launch_bounds__(kBlock) kSignalReset(DevState s)
{
    CellCtx c = cellCtx(s);
    if (!c.valid) return;
    const long long g = c.g;
    const uchar4 fi = s.fnInfo[g];
    bool reset;
    if (fi.x == 0) {
        // without function: cleared every step, so only the first step after
        // ingest finds anything to clear
        reset = s.counters[c.w].signalsFresh != 0;
    } else {
        const int orders = s.params[c.w].cellNumExecutionOrderNumbers;
        const int current = static_cast<int>(s.counters[c.w].timestep % static_cast<uint64_t>(orders));
        const int own = fi.y;
        int maxOther = -1;
        if (!fi.w) {
            const int n = s.numConn[g];
            for (int k = 0; k < n; ++k) {
                const uchar4 fo = s.fnInfo[s.bond[g * kMaxBonds + k]];
                const int other = fo.y;
                if (static_cast<int8_t>(fo.z) != own) continue;
                if (maxOther == -1) {
                    maxOther = other;
                } else if ((maxOther > own && (other > maxOther || other < own)) || (maxOther < own && other > maxOther && other < own)) {
                    maxOther = other;
                }
            }
        }
        reset = (maxOther == -1 && current == (own + 1) % orders) || (maxOther != -1 && maxOther == current);
    }
    if (reset) {
        AlienSignalTO& sig = s.cold[s.coldIdx[g]].signal;
#pragma unroll
        for (int ch = 0; ch < ALIEN_B200_MAX_CHANNELS; ++ch) sig.channels[ch] = 0.0f;
    }
}

// ---------------------------------------------------- bond additions -----
// CellConnectionProcessor::tryAddConnectionOneWay (CellConnectionProcessor.cuh
// :274-427, angle alignment None) on a register copy of the bond list;
// partner lists are read from the arrays, which no thread changes in this
// phase.
struct BondList {
    int n;
    int b[kMaxBonds];
    float d[kMaxBonds], a[kMaxBonds];
};

__device__ inline void loadBonds(const DevState& s, long long g, BondList& l)
{
    l.n = s.numConn[g];
    for (int k = 0; k < kMaxBonds; ++k) {
        l.b[k] = s.bond[g * kMaxBonds + k];
        l.d[k] = s.bondDist[g * kMaxBonds + k];
        l.a[k] = s.bondAngle[g * kMaxBonds + k];
    }
}

__device__ inline bool tryAddOneWay(const DevState& s, const WorldInfo& wi, long long c1, long long c2, float2 posDelta, BondList& out)
{
    loadBonds(s, c1, out);
    const int n = out.n;
    if (n == kMaxBonds) return false;
    if (n >= 2) {  // wouldResultInOverlappingConnection, CellConnectionProcessor.cuh:476-500
        // on the positions as the reference stores them (absolute, rounded)
        const float2 p1 = stepPos(s, c1, wi.W, wi.H), p2 = stepPos(s, c2, wi.W, wi.H);
        for (int k = 0; k < n; ++k) {
            const int cc = out.b[k], nc = out.b[(k + 1) % n];
            const int ncc = s.numConn[cc];
            bool both = false;
            for (int m = 0; m < ncc; ++m) both |= (s.bond[static_cast<long long>(cc) * kMaxBonds + m] == nc);
            if (!both) continue;
            if (crossing(p1, p2, stepPos(s, cc, wi.W, wi.H), stepPos(s, nc, wi.W, wi.H))) return false;
        }
    }
    const float newAngle = angleOfVector(posDelta);
    const float desired = len2(posDelta);
    if (n == 0) {
        out.n = 1;
        out.b[0] = static_cast<int>(c2);
        out.d[0] = desired;
        out.a[0] = 360.0f;
        return true;
    }
    if (n == 1) {
        const float prevAngle = angleOfVector(stepDisp(s, c1, out.b[0], wi.W, wi.H));
        float diff = newAngle - prevAngle;
        if (diff < 0) diff += 360.0f;
        if (fabsf(diff) < kNearZero || fabsf(diff - 360.0f) < kNearZero || fabsf(diff + 360.0f) < kNearZero) return false;
        out.a[1] = diff;
        out.a[0] = 360.0f - diff;
        out.n = 2;
        out.b[1] = static_cast<int>(c2);
        out.d[1] = desired;
        return true;
    }
    int index = 0;
    float prevAngle = 0.0f, nextAngle = 0.0f;
    for (; index < n; ++index) {
        const int prevIndex = (index + n - 1) % n;
        prevAngle = angleOfVector(stepDisp(s, c1, out.b[prevIndex], wi.W, wi.H));
        nextAngle = angleOfVector(stepDisp(s, c1, out.b[index], wi.W, wi.H));
        if (isAngleInBetween(prevAngle, nextAngle, newAngle) || prevIndex == index) break;
    }
    if (index == n) return false;
    const float refAngle = out.a[index];
    const float d1 = subtractAngle(newAngle, prevAngle), d2 = subtractAngle(nextAngle, prevAngle);
    const float fraction = d2 != 0.0f ? d1 / d2 : 0.5f;
    const float afp = fminf(refAngle * fraction, refAngle);
    if (afp < kNearZero) return false;
    if (index == 0) index = n;
    for (int j = n; j > index; --j) {
        out.b[j] = out.b[j - 1];
        out.d[j] = out.d[j - 1];
        out.a[j] = out.a[j - 1];
    }
    out.b[index] = static_cast<int>(c2);
    out.d[index] = desired;
    out.a[index] = afp;
    out.a[(index + 1) % (n + 1)] = refAngle - afp;
    out.n = n + 1;
    return true;
}

// ----------------------------------------------------------- kResolve ----
// dying / detaching resolution of decay (CellProcessor.cuh:840-850) and the
// bond additions of mutually chosen fusion pairs (processAddOperations,
// CellConnectionProcessor.cuh:130-143, 211-272), written to scratch.
__global__ void __launch_bounds__(kBlock, 8) kResolve(DevState s)
{
    // own fields before the world lookup (every launched cell slot lies
    // inside the arena; no other cell writes them in this kernel)
    const long long g0 = static_cast<long long>(blockIdx.x) * kBlock + threadIdx.x;
    const uint32_t f = s.flags[g0];
    const int next = s.nextState[g0];
    const int j = s.best[g0];
    CellCtx c = cellCtx(s);
    if (!c.valid) return;
    const long long g = c.g;
    int ls = next;
    if (f & kFlagSetDying)
        ls = ALIEN_B200_LIVING_DYING;
    else if ((f & kFlagDetachFromDying) && ls != ALIEN_B200_LIVING_DYING)
        ls = ALIEN_B200_LIVING_DETACHING;
    s.livingState[g] = static_cast<uint8_t>(ls);

    if (j < 0 || j <= g || s.best[j] != g) return;
    const WorldInfo& wi = s.worlds[c.w];
    const bool gFirst = s.id[g] < s.id[j];
    const long long c1 = gFirst ? g : j, c2 = gFirst ? j : g;
    const float2 pd = stepDisp(s, c1, c2, wi.W, wi.H);
    BondList l1, l2;
    if (!tryAddOneWay(s, wi, c1, c2, pd, l1)) return;
    if (!tryAddOneWay(s, wi, c2, c1, pd * -1.0f, l2)) return;
    const BondList* lists[2] = {&l1, &l2};
    const long long cs[2] = {c1, c2};
    for (int m = 0; m < 2; ++m) {
        const long long x = cs[m];
        s.addNum[x] = static_cast<uint8_t>(lists[m]->n);
        for (int k = 0; k < kMaxBonds; ++k) {
            s.addBond[x * kMaxBonds + k] = k < lists[m]->n ? lists[m]->b[k] : -1;
            s.addDist[x * kMaxBonds + k] = lists[m]->d[k];
            s.addAngle[x * kMaxBonds + k] = lists[m]->a[k];
        }
    }
    s.newPartner[c1] = static_cast<int>(c2);
    s.newPartner[c2] = static_cast<int>(c1);
}

// ------------------------------------------------------------ kCommit ----
// bond additions, cell deletion (processDeleteCellOperations,
// CellConnectionProcessor.cuh:145-174) and bond deletion
// (processDeleteConnectionOperations :176-209 with deleteConnectionOneWay
// :429-448): a bond is dropped when its partner is deleted, or when either
// end scheduled "delete all bonds" and the bond is not this step's addition.
__global__ void __launch_bounds__(kBlock, 8) kCommit(DevState s)
{
    // own fields before the world lookup (every launched cell slot lies
    // inside the arena; no other cell writes them in this kernel)
    const long long g0 = static_cast<long long>(blockIdx.x) * kBlock + threadIdx.x;
    const uint32_t f = s.flags[g0];
    const int np = s.newPartner[g0];
    const int n0 = s.numConn[g0];
    CellCtx c = cellCtx(s);
    if (!c.valid) return;
    const long long g = c.g;
    if (f & kFlagDelCell) {
        s.alive[g] = 0;
        atomicAdd(&s.counters[c.w].deadCells, 1u);
        return;
    }
    const bool delAllG = f & kFlagDelAll;
    BondList l;
    if (np >= 0) {
        s.newPartner[g] = -1;
        l.n = s.addNum[g];
        for (int k = 0; k < kMaxBonds; ++k) {
            l.b[k] = s.addBond[g * kMaxBonds + k];
            l.d[k] = s.addDist[g * kMaxBonds + k];
            l.a[k] = s.addAngle[g * kMaxBonds + k];
        }
    } else {
        // most cells keep their bonds: look at the partners' flags first and
        // read rest lengths and angles only when a bond goes
        const int n = n0;
        int jb[kMaxBonds];
        const int2* row = reinterpret_cast<const int2*>(s.bond + g * kMaxBonds);
#pragma unroll
        for (int h = 0; h < kMaxBonds / 2; ++h) {
            const int2 jj = 2 * h < n ? row[h] : make_int2(0, 0);
            jb[2 * h] = jj.x;
            jb[2 * h + 1] = jj.y;
        }
        uint32_t fj[kMaxBonds];
#pragma unroll
        for (int k = 0; k < kMaxBonds; ++k) fj[k] = k < n ? s.flags[jb[k]] : 0u;
        bool any = false;
#pragma unroll
        for (int k = 0; k < kMaxBonds; ++k)
            any |= k < n && ((fj[k] & kFlagDelCell) || delAllG || (fj[k] & kFlagDelAll));
        if (!any) return;
        loadBonds(s, g, l);
    }
    int drop[kMaxBonds];
    int nd = 0;
    for (int k = 0; k < l.n; ++k) {
        const int j = l.b[k];
        const uint32_t fj = s.flags[j];
        if ((fj & kFlagDelCell) || ((delAllG || (fj & kFlagDelAll)) && j != np)) drop[nd++] = j;
    }
    if (np < 0 && nd == 0) return;
    for (int m = 0; m < nd; ++m) {
        const int n = l.n;
        for (int k = 0; k < n; ++k) {
            if (l.b[k] != drop[m]) continue;
            const float add = l.a[k];
            for (int j = k; j < n - 1; ++j) {
                l.b[j] = l.b[j + 1];
                l.d[j] = l.d[j + 1];
                l.a[j] = l.a[j + 1];
            }
            if (k < n - 1)
                l.a[k] += add;
            else
                l.a[0] += add;
            l.b[n - 1] = -1;
            l.n = n - 1;
            break;
        }
    }
    s.numConn[g] = static_cast<uint8_t>(l.n);
    for (int k = 0; k < kMaxBonds; ++k) {
        s.bond[g * kMaxBonds + k] = k < l.n ? l.b[k] : -1;
        s.bondDist[g * kMaxBonds + k] = l.d[k];
        s.bondAngle[g * kMaxBonds + k] = l.a[k];
    }
}

// ------------------------------------------------------------- events ----
// New energy particles (RadiationProcessor::createEnergyParticle without
// sources, :248-364, and ObjectFactory::createParticle, ObjectFactory.cuh
// :242-256) in the order radiation (cell order), splitting (particle order),
// deleted cells (cell order); ids continue the world's id counter.  A
// deleted cell makes a particle when it has energy above NEAR_ZERO.

__global__ void __launch_bounds__(kBlock) kEventCount(DevState s)
{
    __shared__ uint32_t red[2][kBlock / 32];
    // block sums of a and b in thread 0
    auto blockSums = [&](uint32_t a, uint32_t b, uint32_t& ta, uint32_t& tb) {
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        a = __reduce_add_sync(0xffffffffu, a);
        b = __reduce_add_sync(0xffffffffu, b);
        __syncthreads();
        if (lane == 0) {
            red[0][warp] = a;
            red[1][warp] = b;
        }
        __syncthreads();
        ta = tb = 0;
        if (threadIdx.x == 0)
            for (int i = 0; i < kBlock / 32; ++i) {
                ta += red[0][i];
                tb += red[1][i];
            }
    };
    if (blockIdx.x < s.numCellBlocks) {
        const long long g = static_cast<long long>(blockIdx.x) * kBlock + threadIdx.x;
        const uint32_t fl = s.flags[g];  // before the world lookup: every cell slot is inside the arena
        const int w = s.cellBlockWorld[blockIdx.x];
        WorldCounters& wc = s.counters[w];
        // a halted world keeps its step's flags and block counts until the
        // host completes that step (the test is uniform across the block)
        if (wc.halted) return;
        uint32_t a = 0, b = 0;
        if (g < s.worlds[w].cellBase + wc.numCells) {
            a = (fl & kFlagRadiation) ? 1u : 0u;
            if (fl & kFlagDelCell) {
                // the deleted cell's energy particle (createEnergyParticle):
                // the external-energy backflow is recorded here, once
                const AlienPhysicsParams& p = s.params[s.worlds[w].paramIndex];
                b = backflow(p, wc, s.color[g] % ALIEN_B200_MAX_COLORS, s.energy[g]) > kNearZero ? 1u : 0u;
            }
            // the step's flags end here, except on the cells kEventEmit
            // still reads (radiation and deletion events)
            if (fl && !a && !b) s.flags[g] = 0;
        }
        uint32_t ta, tb;
        blockSums(a, b, ta, tb);
        if (threadIdx.x == 0) {
            s.blockRad[blockIdx.x] = ta;
            s.blockDel[blockIdx.x] = tb;
            if (ta) atomicAdd(&wc.evRad, ta);
            if (tb) atomicAdd(&wc.evDel, tb);
        }
    } else {
        forParticleBlocks(s, usedParticles, [&](const PartCtx& c, int pb) {
            const uint32_t a = c.inRange && (s.pflag[c.q] & 2u) ? 1u : 0u;
            uint32_t ta, tb;
            blockSums(a, 0u, ta, tb);
            if (threadIdx.x == 0) {
                s.blockSplit[pb] = ta;
                if (ta) atomicAdd(&s.counters[c.w].evSplit, ta);
            }
        });
    }
}

// exclusive scan of arr[first .. first+count) in place by one block of
// Threads threads: each thread scans a contiguous chunk, the chunk sums are
// scanned across the block; returns the total
template <int Threads>
__device__ uint32_t blockScanBlocks(uint32_t* arr, int first, int count)
{
    const int chunk = (count + Threads - 1) / Threads;
    const int b0 = threadIdx.x * chunk;
    const int b1 = min(b0 + chunk, count);
    uint32_t sum = 0;
    for (int k = b0; k < b1; ++k) sum += arr[first + k];
    uint32_t total;
    uint32_t run = blockExclusiveScanN<Threads>(sum, &total);
    for (int k = b0; k < b1; ++k) {
        const uint32_t v = arr[first + k];
        arr[first + k] = run;
        run += v;
    }
    return total;
}

// one block per world: block offsets, id and slot bases, timestep advance;
// the block scans run only for the kinds of events the step produced (1024
// threads ran slower than 256 on a 4M-cell world's 15,625 block counts).
//
// A step whose new particles do not fit the world's particle range halts the
// world here, before anything of the emission is written: the world turns
// inactive with its step's flags, block counts and event scratch in place,
// counts the steps it misses, and sets kErrHalted.  The host grows the range
// (on the device, nothing else of the world moves) and relaunches kEventWorld,
// kEventEmit and kWorldsEnd with DevState::resume set, which complete the
// halted step exactly as an uninterrupted step would have; then it runs the
// missed steps.  In the resume launches a world that still does not fit (no
// larger range was free) drops the excess and sets kErrDropped, and so do its
// steps until the next capacity check (WorldCounters::dropExcess).
constexpr int kEventWorldThreads = kBlock;
__global__ void __launch_bounds__(kEventWorldThreads) kEventWorld(DevState s)
{
    const int w = blockIdx.x;
    WorldCounters& wc = s.counters[w];
    const uint32_t evR = wc.evRad, evD = wc.evDel, evS = wc.evSplit;
    const bool halted = wc.halted != 0;
    const uint32_t slot0 = wc.numParticles;  // the used slots before this step's appends
    __syncthreads();
    if (s.resume) {
        if (!halted) {
            // completed worlds emit nothing in the resume launch
            if (threadIdx.x == 0) wc.numEvents = 0;
            return;
        }
    } else if (halted) {
        if (threadIdx.x == 0 && (wc.stepsRemaining == ~0ull || wc.missedSteps + 1 < wc.stepsRemaining)) ++wc.missedSteps;
        return;
    } else if (!wc.active) {
        if (threadIdx.x == 0) {
            wc.numEvents = 0;
            wc.evRad = wc.evDel = wc.evSplit = 0;
        }
        return;
    }
    const WorldInfo& wi = s.worlds[w];
    if (!s.resume && !wc.dropExcess &&
        static_cast<unsigned long long>(slot0) + evR + evD + evS > static_cast<unsigned long long>(wi.partCap)) {
        if (threadIdx.x == 0) {
            wc.halted = 1;
            wc.active = 0;
            wc.numEvents = 0;
            wc.missedSteps = 0;
            atomicOr(s.errorFlags, kErrHalted);
        }
        return;
    }
    // particle blocks holding used slots (the count before this step's appends)
    const int usedPartBlocks = static_cast<int>((wc.numParticles + kBlock - 1) / kBlock);
    const uint32_t R = evR ? blockScanBlocks<kEventWorldThreads>(s.blockRad, wi.firstCellBlock, wi.numCellBlocks) : 0u;
    const uint32_t D = evD ? blockScanBlocks<kEventWorldThreads>(s.blockDel, wi.firstCellBlock, wi.numCellBlocks) : 0u;
    const uint32_t S = evS ? blockScanBlocks<kEventWorldThreads>(s.blockSplit, wi.firstPartBlock, usedPartBlocks) : 0u;
    if (threadIdx.x != 0) return;
    if (halted) {
        wc.halted = 0;
        wc.active = 1;
    }
    wc.evRad = wc.evDel = wc.evSplit = 0;
    const unsigned long long id0 = wc.nextId;
    wc.radIdBase = id0;
    wc.splitIdBase = id0 + R;
    wc.delIdBase = id0 + R + S;
    wc.radSlotBase = slot0;
    wc.splitSlotBase = slot0 + R;
    wc.delSlotBase = slot0 + R + S;
    wc.numEvents = R + S + D;
    wc.nextId = id0 + R + S + D;
    const unsigned long long want = static_cast<unsigned long long>(slot0) + R + S + D;
    if (want > static_cast<unsigned long long>(wi.partCap)) {
        wc.droppedParticles += static_cast<uint32_t>(want - wi.partCap);
        wc.numParticles = static_cast<uint32_t>(wi.partCap);
        atomicOr(s.errorFlags, kErrDropped);
    } else {
        wc.numParticles = static_cast<uint32_t>(want);
    }
    wc.timestep += 1;
    wc.lastStepped = wc.timestep;  // kWorldsEnd: this world completed a step
    wc.signalsFresh = 0;
    if (wc.stepsRemaining != ~0ull && --wc.stepsRemaining == 0) wc.active = 0;
}

// the active radiation sources of every world before its first step
__global__ void kWorldsBegin(DevState s)
{
    const int w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= s.numWorlds) return;
    const WorldInfo& wi = s.worlds[w];
    s.counters[w].activeSources = activeSources(s.params[wi.paramIndex], wi.W, wi.H);
}

// The end of a step for worlds with zones, radiation sources or external
// energy (launched after kEventEmit, which still uses the step's sources and
// pool): the pool takes the step's backflow, zones and sources move
// (SimulationParametersUpdateService.cu:52-78) and the next step's active
// sources follow their new positions.  A world that did not step (inactive)
// has nothing to add and does not move.
__global__ void kWorldsEnd(DevState s)
{
    const int w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= s.numWorlds) return;
    WorldCounters& wc = s.counters[w];
    // a halted world's step ends when the host completes it (resume launch)
    if (wc.halted) return;
    if (wc.backflowFix) {
        wc.externalEnergy += static_cast<double>(wc.backflowFix) / kBackflowScale;
        wc.backflowFix = 0;
    }
    if (wc.lastStepped != wc.timestep) return;
    wc.lastStepped = ~0ull;
    const WorldInfo& wi = s.worlds[w];
    AlienPhysicsParams& p = s.params[wi.paramIndex];
    if (p.numZones > 0 || p.numRadiationSources > 0) {
        moveZonesAndSources(p, wi.W, wi.H);
        wc.activeSources = activeSources(p, wi.W, wi.H);
    }
}

__device__ __forceinline__ void emitParticle(const DevState& s, const WorldInfo& wi, uint32_t slotRel, unsigned long long id,
                                             float2 pos, float2 vel, float energy, uint8_t color)
{
    if (slotRel >= wi.partCap) return;
    const long long q = wi.partBase + slotRel;
    pos = correctPosition(pos, wi.W, wi.H);
    s.pid[q] = id;
    s.ppos[q] = pos;
    s.pvel[q] = vel;
    s.penergy[q] = energy;
    s.pcolor[q] = color;
    s.pselected[q] = 0;
    s.palive[q] = 1;
    s.plast[q] = ~0ull;
    // per-step scratch of a new slot (kBin resets the used slots at step start)
    s.pflag[q] = 0;
    s.ptarget[q] = -1;
    s.pslot[q] = -1;
    s.pmerge[3 * q + 0] = 0;
    s.pmerge[3 * q + 1] = 0;
    s.pmerge[3 * q + 2] = 0;
}

__global__ void __launch_bounds__(kBlock) kEventEmit(DevState s)
{
    if (blockIdx.x < s.numCellBlocks) {
        const int w = s.cellBlockWorld[blockIdx.x];
        const WorldCounters& wc = s.counters[w];
        const long long g = static_cast<long long>(blockIdx.x) * kBlock + threadIdx.x;
        // without events kEventCount has cleared every flag already
        if (wc.numEvents == 0) return;
        const WorldInfo& wi = s.worlds[w];
        // the same for a block without events: its event count is the
        // difference of consecutive block offsets (the world's total after
        // its last block; offsets stay zero for a kind the step did not
        // produce); the test is uniform across the block, ahead of its scans
        {
            const int b = blockIdx.x, lastBlock = wi.firstCellBlock + wi.numCellBlocks - 1;
            const uint32_t totalRad = static_cast<uint32_t>(wc.splitIdBase - wc.radIdBase);
            const uint32_t totalDel = static_cast<uint32_t>(wc.nextId - wc.delIdBase);
            const uint32_t nRad = (b < lastBlock ? s.blockRad[b + 1] : totalRad) - s.blockRad[b];
            const uint32_t nDel = (b < lastBlock ? s.blockDel[b + 1] : totalDel) - s.blockDel[b];
            if (nRad == 0 && nDel == 0) return;
        }
        const uint32_t fl = s.flags[g];
        if (fl) s.flags[g] = 0;  // the step's flags end here
        const bool inRange = g < wi.cellBase + wc.numCells;
        const uint32_t rad = inRange && (fl & kFlagRadiation) ? 1u : 0u;
        const AlienPhysicsParams& p = s.params[wi.paramIndex];
        const float kept = inRange && (fl & kFlagDelCell) ? backflowKept(p, wc, s.color[g] % ALIEN_B200_MAX_COLORS, s.energy[g]) : 0.0f;
        const uint32_t del = kept > kNearZero ? 1u : 0u;
        const uint32_t rr = blockExclusiveScan(rad, nullptr) + s.blockRad[blockIdx.x];
        const uint32_t dr = blockExclusiveScan(del, nullptr) + s.blockDel[blockIdx.x];
        if (rad) emitParticle(s, wi, wc.radSlotBase + rr, wc.radIdBase + rr, s.radPos[g], s.radVel[g], s.radEnergy[g], s.color[g]);
        if (del) {
            float2 pos = stepPos(s, g, wi.W, wi.H), vel = s.velA[g];
            placeAtSource(p, wc.activeSources, s.id[g], wc.timestep - 1, kSiteSourceDeletedCell, pos, vel);
            emitParticle(s, wi, wc.delSlotBase + dr, wc.delIdBase + dr, correctPosition(pos, wi.W, wi.H), vel, kept, s.color[g]);
        }
    } else {
        // splits come from the slots used before this step's appends
        // (radSlotBase); appended particles carry no split.  A world whose
        // step budget ended with this step is inactive already and still
        // emits; worlds without events are skipped by their used slots
        forParticleBlocks<false>(s, [](const WorldCounters& wc) { return wc.numEvents ? wc.radSlotBase : 0u; },
                                 [&](const PartCtx& c, int pb) {
            const WorldCounters& wc = s.counters[c.w];
            if (wc.numEvents == 0) return;
            const WorldInfo& wi = s.worlds[c.w];
            const long long q = c.q;
            const uint32_t split = c.inRange && (s.pflag[q] & 2u) ? 1u : 0u;
            const uint32_t sr = blockExclusiveScan(split, nullptr) + s.blockSplit[pb];
            if (split)
                emitParticle(s, wi, wc.splitSlotBase + sr, wc.splitIdBase + sr, s.splitPos[q], s.splitVel[q], s.splitEnergy[q],
                             s.pcolor[q]);
        });
    }
}

}  // namespace ab
