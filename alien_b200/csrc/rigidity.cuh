// Rigidity clusters (ClusterProcessor.cuh:8-168, launched in every third step
// after friction, SimulationKernelsLauncher.cu:74-83): the cells of a bonded
// cluster move partly as one rigid body.  A cell's velocity is blended,
// with weight rigidity * stiffness^2, into the velocity the cluster's mean
// motion and rotation give at its position.
//
// Deterministic definition (the reference finds clusters with three passes
// of lock-free label walks whose outcome depends on thread timing, and sums
// with float atomics):
// * cluster = the smallest storage index reachable through bonds, found by
//   synchronous Shiloach-Vishkin rounds (Shiloach and Vishkin 1982; the
//   hooking and shortcutting steps of FastSV, Zhang, Azad and Hu 2020): each
//   round reads the previous round's labels only, and its scattered hooks
//   are atomic minima, whose result does not depend on their order.  The
//   labels stop changing once they equal that minimum, in a number of rounds
//   that grows with the logarithm of the cluster's diameter (a 5000-cell
//   chain in random storage order: 14); a round whose predecessor changed
//   nothing returns at once.  A cluster still changing after kClusterRounds
//   rounds keeps its partial labels and acts as several rigid parts, as
//   large clusters do in the reference's heuristic; the oracle runs the same
//   rounds.
// * cluster sums (velocity, position, count, angular mass and momentum) are
//   fixed-point int64 atomics: order-independent.
// * positions enter as displacements from the cluster's label cell (minimal
//   image across the torus seam, from the step-start positions plus the
//   in-step displacements), so a cell's offset from the cluster centre keeps
//   FP32 precision at any world coordinate.  The reference moves the cells
//   in the last third of the world by one world size when the cluster has a
//   cell in the first third; both give the same offsets for clusters
//   smaller than a third of the world.
#pragma once

#include "device_common.cuh"
#include "kernels.cuh"
#include "zones.cuh"

namespace ab {

constexpr int kClusterRounds = 12;
constexpr double kClusterVelScale = 4294967296.0;   // 2^32: velocity and offset sums
constexpr double kClusterMassScale = 16777216.0;    // 2^24: angular mass (squared offsets)
constexpr double kClusterMomScale = 268435456.0;    // 2^28: angular momentum
enum { kAccVelX, kAccVelY, kAccPosX, kAccPosY, kAccMass, kAccMom, kAccFields };

// _SimulationKernelsLauncher::isRigidityUpdateEnabled (SimulationKernelsLauncher.cu:99-107)
__host__ __device__ inline bool rigidityEnabled(const AlienPhysicsParams& p)
{
    for (int i = 0; i < p.numZones; ++i)
        if (p.zones[i].rigidity != 0.0f) return true;
    return p.rigidity != 0.0f;
}

// the cell's world runs the cluster pass in this step
struct ClusterCtx {
    long long g;
    int w;
    bool on;
};
__device__ __forceinline__ ClusterCtx clusterCtx(const DevState& s)
{
    const CellCtx c = cellCtx(s);
    ClusterCtx k{c.g, c.w, false};
    if (!c.valid) return k;
    const AlienPhysicsParams& p = s.params[s.worlds[c.w].paramIndex];
    k.on = s.counters[c.w].timestep % 3 == 0 && rigidityEnabled(p);  // SimulationKernelsLauncher.cu:33
    return k;
}

__device__ __forceinline__ unsigned long long toFixScaled(float v, double scale)
{
    return static_cast<unsigned long long>(__double2ll_rn(static_cast<double>(v) * scale));
}
__device__ __forceinline__ double fromFixScaled(long long q, double scale) { return static_cast<double>(q) / scale; }

// initClusterData (ClusterProcessor.cuh:24-40)
__global__ void __launch_bounds__(kBlock) kClusterInit(DevState s)
{
    if (blockIdx.x == 0 && threadIdx.x < kClusterRounds) s.clusterChanged[threadIdx.x] = 0;
    const ClusterCtx c = clusterCtx(s);
    if (!c.on) return;
    s.clusterLab[0][c.g] = static_cast<int>(c.g);
    s.clusterCount[c.g] = 0;
#pragma unroll
    for (int f = 0; f < kAccFields; ++f) s.clusterAcc[c.g * kAccFields + f] = 0;
}

// a round of label propagation (replaces findClusterIteration,
// ClusterProcessor.cuh:42-66), gather half: shortcut (the label's label) and
// aggressive hooking (the partners' labels' labels)
__global__ void __launch_bounds__(kBlock) kClusterGather(DevState s, int r)
{
    if (r > 0 && s.clusterChanged[r - 1] == 0) return;  // converged: both label buffers agree
    const ClusterCtx c = clusterCtx(s);
    if (!c.on) return;
    const int* f = s.clusterLab[r & 1];
    int* g = s.clusterLab[(r + 1) & 1];
    const int fu = f[c.g];
    int m = min(fu, f[fu]);
    const int n = s.numConn[c.g];
    for (int k = 0; k < n; ++k) m = min(m, f[f[s.bond[c.g * kMaxBonds + k]]]);
    g[c.g] = m;
    if (m != fu) s.clusterChanged[r] = 1;
}

// scatter half: the partners' labels' labels hook the cell's label (atomic
// minima into the new labels, after the gather half wrote them)
__global__ void __launch_bounds__(kBlock) kClusterScatter(DevState s, int r)
{
    if (r > 0 && s.clusterChanged[r - 1] == 0) return;
    const ClusterCtx c = clusterCtx(s);
    if (!c.on) return;
    const int* f = s.clusterLab[r & 1];
    int* g = s.clusterLab[(r + 1) & 1];
    const int fu = f[c.g];
    const int n = s.numConn[c.g];
    int m = fu;
    for (int k = 0; k < n; ++k) m = min(m, f[f[s.bond[c.g * kMaxBonds + k]]]);
    if (m < fu && atomicMin(&g[fu], m) > m) s.clusterChanged[r] = 1;
}

// the labels after the last round
__device__ __forceinline__ int clusterOf(const DevState& s, long long g) { return s.clusterLab[kClusterRounds & 1][g]; }

// accumulateClusterPosAndVel and findClusterBoundaries (ClusterProcessor.cuh:68-108)
__global__ void __launch_bounds__(kBlock) kClusterSum1(DevState s)
{
    const ClusterCtx c = clusterCtx(s);
    if (!c.on) return;
    const WorldInfo& wi = s.worlds[c.w];
    const int cl = clusterOf(s, c.g);
    const float2 rel = stepDisp(s, cl, c.g, wi.W, wi.H);
    const float2 v = s.velA[c.g];
    unsigned long long* acc = reinterpret_cast<unsigned long long*>(s.clusterAcc + static_cast<long long>(cl) * kAccFields);
    atomicAdd(acc + kAccVelX, toFixScaled(v.x, kClusterVelScale));
    atomicAdd(acc + kAccVelY, toFixScaled(v.y, kClusterVelScale));
    atomicAdd(acc + kAccPosX, toFixScaled(rel.x, kClusterVelScale));
    atomicAdd(acc + kAccPosY, toFixScaled(rel.y, kClusterVelScale));
    atomicAdd(&s.clusterCount[cl], 1u);
}

// the cluster's mean velocity and position, and the cell's offset from it
struct ClusterFrame {
    float2 vel, r;
};
__device__ __forceinline__ ClusterFrame clusterFrame(const DevState& s, long long g, int cl, const WorldInfo& wi)
{
    const long long* acc = s.clusterAcc + static_cast<long long>(cl) * kAccFields;
    const double n = static_cast<double>(s.clusterCount[cl]);
    const float2 rel = stepDisp(s, cl, g, wi.W, wi.H);
    ClusterFrame f;
    f.vel = f2(static_cast<float>(fromFixScaled(acc[kAccVelX], kClusterVelScale) / n),
               static_cast<float>(fromFixScaled(acc[kAccVelY], kClusterVelScale) / n));
    f.r = f2(static_cast<float>(static_cast<double>(rel.x) - fromFixScaled(acc[kAccPosX], kClusterVelScale) / n),
             static_cast<float>(static_cast<double>(rel.y) - fromFixScaled(acc[kAccPosY], kClusterVelScale) / n));
    return f;
}

// accumulateClusterAngularProp (ClusterProcessor.cuh:110-136)
__global__ void __launch_bounds__(kBlock) kClusterSum2(DevState s)
{
    const ClusterCtx c = clusterCtx(s);
    if (!c.on) return;
    const WorldInfo& wi = s.worlds[c.w];
    const int cl = clusterOf(s, c.g);
    const ClusterFrame f = clusterFrame(s, c.g, cl, wi);
    const float2 dv = s.velA[c.g] - f.vel;
    const float mass = dot2(f.r, f.r);  // Math::lengthSquared
    const float mom = f.r.x * dv.y - f.r.y * dv.x;  // Physics::angularMomentum
    unsigned long long* acc = reinterpret_cast<unsigned long long*>(s.clusterAcc + static_cast<long long>(cl) * kAccFields);
    atomicAdd(acc + kAccMass, toFixScaled(mass, kClusterMassScale));
    atomicAdd(acc + kAccMom, toFixScaled(mom, kClusterMomScale));
}

// applyClusterData (ClusterProcessor.cuh:138-168)
__global__ void __launch_bounds__(kBlock) kClusterApply(DevState s)
{
    const ClusterCtx c = clusterCtx(s);
    if (!c.on) return;
    const WorldInfo& wi = s.worlds[c.w];
    const AlienPhysicsParams& p = s.params[wi.paramIndex];
    const int cl = clusterOf(s, c.g);
    const ClusterFrame f = clusterFrame(s, c.g, cl, wi);
    const long long* acc = s.clusterAcc + static_cast<long long>(cl) * kAccFields;
    const float mass = static_cast<float>(fromFixScaled(acc[kAccMass], kClusterMassScale));
    const float mom = static_cast<float>(fromFixScaled(acc[kAccMom], kClusterMomScale));
    // Physics::angularVelocity (Physics.cuh:191-197)
    const float angularVel = fabsf(mass) < kNearZero ? 0.0f : mom / mass * (180.0f / kPi);
    const float stiffness = s.stiffness[c.g];
    const float rigidity =
        zoneParam<kZRigidity>(p, wi.W, wi.H, stepPos(s, c.g, wi.W, wi.H), p.rigidity) * stiffness * stiffness;
    // Physics::tangentialVelocity (Physics.cuh:181-184)
    const float2 tangential = f2(f.vel.x - angularVel * f.r.y * (kPi / 180.0f), f.vel.y + angularVel * f.r.x * (kPi / 180.0f));
    s.velA[c.g] = s.velA[c.g] * (1.0f - rigidity) + tangential * rigidity;
}

}  // namespace ab
