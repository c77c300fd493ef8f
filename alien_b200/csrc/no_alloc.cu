// no_alloc.cu - statistics of device-resident transfer objects without any
// device allocation (alien_b200_statistics_no_alloc, include/alien_b200.h).
//
// Some callers cannot allocate device memory at the moment they need an
// answer: a host runtime that reserved the whole HBM budget up front and
// hands out only its own buffers, code running while another component owns
// the allocator (a memory pool under stream-ordered use, an allocator that
// must not be re-entered), or a process whose allocation calls are forbidden
// for latency reasons.  This entry point takes the caller's device buffers
// and keeps its only scratch, the per-block partial sums, in a fixed
// file-scope device array.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/alien_b200.h"

namespace {

constexpr int kThreads = 256;
constexpr int kItemsPerThread = 8;
constexpr int kItemsPerBlock = kThreads * kItemsPerThread;  // 2048 objects per block
constexpr int kMaxBlocks = 4096;                              // per object kind
// largest accepted numCells and numParticles: 8,388,608 each
constexpr unsigned long long kMaxObjects = static_cast<unsigned long long>(kMaxBlocks) * kItemsPerBlock;

struct Partial {
    unsigned long long count, connections;
    unsigned long long byColor[ALIEN_B200_MAX_COLORS];
    long long energyFix;  // 2^-16 fixed point, as the arena statistics
};

static_assert(sizeof(Partial) == 80, "the scratch size stated in the header assumes 80-byte partials");

// Scratch: one partial per block for cells, then one per block for
// particles (2 x 4096 x 80 B = 640 KiB).  Every GPU that loads the library
// holds it until the process exits.  Each call overwrites the partials of
// the blocks it launches before reading them, so nothing needs clearing; two
// calls that overlap on the GPU share this array and race.
static __device__ __align__(256) Partial g_scratch[2 * kMaxBlocks];


__device__ __forceinline__ unsigned long long warpSum(unsigned long long v)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// block sum of v, valid in thread 0
__device__ unsigned long long blockSum(unsigned long long v, unsigned long long* warpSums)
{
    v = warpSum(v);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) warpSums[warp] = v;
    __syncthreads();
    unsigned long long t = 0;
    if (threadIdx.x == 0)
        for (int i = 0; i < kThreads / 32; ++i) t += warpSums[i];
    return t;
}

// pass 1: blocks [0, cellBlocks) reduce cells, the rest particles; each
// writes its own partial
__global__ void __launch_bounds__(kThreads) kPartials(const AlienCellTO* cells, unsigned long long numCells,
                                                      const AlienParticleTO* particles, unsigned long long numParticles,
                                                      int cellBlocks, Partial* scratch)
{
    __shared__ unsigned long long warpSums[kThreads / 32];
    const bool cellBlock = static_cast<int>(blockIdx.x) < cellBlocks;
    const int b = cellBlock ? blockIdx.x : blockIdx.x - cellBlocks;
    const unsigned long long base = static_cast<unsigned long long>(b) * kItemsPerBlock;
    unsigned long long count = 0, connections = 0, byColor[ALIEN_B200_MAX_COLORS] = {};
    long long energy = 0;
    for (int i = 0; i < kItemsPerThread; ++i) {
        const unsigned long long k = base + static_cast<unsigned long long>(i) * kThreads + threadIdx.x;
        if (cellBlock) {
            if (k >= numCells) continue;
            const AlienCellTO& c = cells[k];
            ++count;
            connections += c.numConnections;
            ++byColor[c.color % ALIEN_B200_MAX_COLORS];
            energy += __double2ll_rn(static_cast<double>(c.energy) * 65536.0);
        } else {
            if (k >= numParticles) continue;
            ++count;
            energy += __double2ll_rn(static_cast<double>(particles[k].energy) * 65536.0);
        }
    }
    Partial p;
    p.count = blockSum(count, warpSums);
    p.connections = blockSum(connections, warpSums);
    for (int c = 0; c < ALIEN_B200_MAX_COLORS; ++c) p.byColor[c] = blockSum(byColor[c], warpSums);
    p.energyFix = static_cast<long long>(blockSum(static_cast<unsigned long long>(energy), warpSums));
    if (threadIdx.x == 0) scratch[cellBlock ? b : kMaxBlocks + b] = p;
}

// pass 2: one block sums the partials in block order (integer sums) and
// writes the result
__global__ void __launch_bounds__(kThreads) kFinish(int cellBlocks, int particleBlocks, const Partial* scratch,
                                                    unsigned long long timestep, AlienRawStatistics* out)
{
    __shared__ unsigned long long warpSums[kThreads / 32];
    unsigned long long cellCount = 0, connections = 0, particleCount = 0, byColor[ALIEN_B200_MAX_COLORS] = {};
    long long cellEnergy = 0, particleEnergy = 0;
    for (int b = threadIdx.x; b < cellBlocks; b += kThreads) {
        const Partial& p = scratch[b];
        cellCount += p.count;
        connections += p.connections;
        for (int c = 0; c < ALIEN_B200_MAX_COLORS; ++c) byColor[c] += p.byColor[c];
        cellEnergy += p.energyFix;
    }
    for (int b = threadIdx.x; b < particleBlocks; b += kThreads) {
        const Partial& p = scratch[kMaxBlocks + b];
        particleCount += p.count;
        particleEnergy += p.energyFix;
    }
    AlienRawStatistics r;
    r.timestep = timestep;
    r.numCells = blockSum(cellCount, warpSums);
    r.numParticles = blockSum(particleCount, warpSums);
    r.numConnections = blockSum(connections, warpSums);
    for (int c = 0; c < ALIEN_B200_MAX_COLORS; ++c) r.numCellsByColor[c] = blockSum(byColor[c], warpSums);
    const long long ce = static_cast<long long>(blockSum(static_cast<unsigned long long>(cellEnergy), warpSums));
    const long long pe = static_cast<long long>(blockSum(static_cast<unsigned long long>(particleEnergy), warpSums));
    r.totalCellEnergy = static_cast<double>(ce) / 65536.0;
    r.totalParticleEnergy = static_cast<double>(pe) / 65536.0;
    if (threadIdx.x == 0) *out = r;
}

// device address of g_scratch, looked up once per device with that device
// current (the symbol's name is only a host-side stand-in).  The cache lives
// as long as the process: after a cudaDeviceReset of a device the address
// it holds for that device is stale, so a caller that resets a device must
// not call this entry point on it again.
constexpr int kMaxDevices = 64;
std::mutex g_setupMutex;
Partial* g_scratchAddress[kMaxDevices] = {};

}  // namespace

namespace ab {
void setLastError(const std::string& message);  // engine.cu: text for alien_b200_last_error
}

namespace {
int fail(int code, const std::string& message)
{
    ab::setLastError(message);
    return code;
}
}  // namespace

extern "C" int alien_b200_statistics_no_alloc(const AlienCellTO* cells, uint64_t numCells, const AlienParticleTO* particles,
                                              uint64_t numParticles, uint64_t timestep, AlienRawStatistics* statistics,
                                              void* stream)
{
    if (!statistics) return fail(ALIEN_B200_ERR_INVALID_ARGUMENT, "statistics output pointer is null");
    if ((numCells && !cells) || (numParticles && !particles))
        return fail(ALIEN_B200_ERR_INVALID_ARGUMENT, "input pointer is null");
    if (numCells > kMaxObjects || numParticles > kMaxObjects)
        return fail(ALIEN_B200_ERR_CAPACITY, "alien_b200_statistics_no_alloc accepts at most " + std::to_string(kMaxObjects)
                                                 + " cells and as many particles per call (fixed scratch of "
                                                 + std::to_string(kMaxBlocks) + " blocks)");
    int device = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess) return fail(ALIEN_B200_ERR_NO_DEVICE, cudaGetErrorString(e));
    if (device < 0 || device >= kMaxDevices) return fail(ALIEN_B200_ERR_UNSUPPORTED, "device index above 63");
    Partial* scratch = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_setupMutex);
        if (!g_scratchAddress[device]) {
            // set-up on this device: with lazy module loading (the CUDA 12
            // default) the array and both kernels are brought onto the GPU
            // here, which may itself need device memory; later calls need
            // none
            void* p = nullptr;
            e = cudaGetSymbolAddress(&p, g_scratch);
            if (e != cudaSuccess) return fail(ALIEN_B200_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
            cudaFuncAttributes attr;
            e = cudaFuncGetAttributes(&attr, kPartials);
            if (e == cudaSuccess) e = cudaFuncGetAttributes(&attr, kFinish);
            if (e != cudaSuccess) return fail(ALIEN_B200_ERR_CUDA, std::string("kernel load: ") + cudaGetErrorString(e));
            g_scratchAddress[device] = static_cast<Partial*>(p);
        }
        scratch = g_scratchAddress[device];
    }
    const int cellBlocks = static_cast<int>((numCells + kItemsPerBlock - 1) / kItemsPerBlock);
    const int particleBlocks = static_cast<int>((numParticles + kItemsPerBlock - 1) / kItemsPerBlock);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // an error left by the caller's earlier work is the caller's to read:
    // report it without launching and without clearing it, so that the
    // error read after the launches below can only be theirs
    e = cudaPeekAtLastError();
    if (e != cudaSuccess)
        return fail(ALIEN_B200_ERR_CUDA, std::string("an earlier CUDA error is pending (not cleared): ") + cudaGetErrorString(e));
    if (cellBlocks + particleBlocks > 0)
        kPartials<<<cellBlocks + particleBlocks, kThreads, 0, s>>>(cells, numCells, particles, numParticles, cellBlocks, scratch);
    kFinish<<<1, kThreads, 0, s>>>(cellBlocks, particleBlocks, scratch, timestep, statistics);
    e = cudaGetLastError();
    if (e != cudaSuccess) return fail(ALIEN_B200_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(e));
    return ALIEN_B200_OK;
}
