// Fluid moments without any allocation: lbm_fluid_moments_noalloc (include/lbm_b200.h).
//
// Some callers cannot call cudaMalloc: a plugin inside a host program whose allocator owns the device memory (an
// MD engine's context, or a framework's caching allocator that has claimed the pool) must not allocate behind the
// owner's back, and a time-critical loop cannot afford the device synchronization that cudaMalloc and cudaFree may
// imply.  This entry point computes what the moments pass of the kernel computes (mass, momentum and the largest
// speed of the fluid, as lbm_get_fluid_mach_number) on a state array and an output array that the caller owns,
// and keeps its per-block partial sums in the file-scope device array below instead of allocated scratch.
//
// The scratch holds one record of 8 doubles per chunk of kChunkNodes nodes, for at most kMaxChunks chunks, so the
// lattice may have at most kMaxChunks*kChunkNodes nodes (67,108,864); larger ones are rejected.  Every GPU that
// loads the library holds the array (128 KB) until the process exits.  All calls share it, so calls that overlap on
// the GPU (on different streams) race; each call overwrites every record it reads, so nothing needs clearing.
#include "lbm_internal.h"
#include "lbm_device.cuh"
#include <cuda_runtime.h>
#include <mutex>
#include <string>

namespace lbm {

namespace {

constexpr long long kChunkNodes = 32768;
constexpr int kMaxChunks = 2048;
constexpr int kRecord = 8;      // sum of deviations, momentum x/y/z, unused x3, max |j/rho|^2
constexpr int kThreads = 256;
constexpr int kMaxDevices = 64;

// The scratch of the partial sums, one record per chunk.  In host code its name is only a stand-in for the device
// symbol: its device address comes from cudaGetSymbolAddress.
static __device__ __align__(256) double noallocPartials[kMaxChunks*kRecord];

std::mutex setupMutex;
struct ScratchEntry {
    void* context;      // the context whose module gave `address`
    double* address;
};
ScratchEntry scratch[kMaxDevices] = {};

// The current CUDA context (CUcontext), through the driver entry point that the runtime hands out, so that the
// library needs no link to the driver library; nullptr if there is none yet or the entry point is unavailable.
void* currentContext() {
    typedef int (*CtxGetCurrent)(void**);
    static CtxGetCurrent getCurrent = [] {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult found;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &fn, cudaEnableDefault, &found) != cudaSuccess ||
                found != cudaDriverEntryPointSuccess)
            fn = nullptr;
        return (CtxGetCurrent) fn;
    }();
    void* context = nullptr;
    if (getCurrent == nullptr || getCurrent(&context) != 0)
        return nullptr;
    return context;
}

// The device address of the scratch on the current device, looked up with that device current: once per device, and
// again whenever the device's context is not the one of the last lookup (after cudaDeviceReset the runtime creates a
// new context, whose copy of the array may sit elsewhere).
double* scratchAddress(int device) {
    std::lock_guard<std::mutex> lock(setupMutex);
    ScratchEntry& entry = scratch[device];
    void* context = currentContext();
    if (entry.address == nullptr || context == nullptr || context != entry.context) {
        void* ptr = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&ptr, noallocPartials);
        if (e != cudaSuccess)
            throw Error(LBM_ERR_CUDA, std::string("lbm_fluid_moments_noalloc: cudaGetSymbolAddress failed: ") +
                        cudaGetErrorString(e));
        entry.address = static_cast<double*>(ptr);
        entry.context = currentContext();     // the lookup made the context current if it was not yet
    }
    return entry.address;
}

// One block per chunk: the sums over the chunk's fluid nodes (deviations [q*N + node]) in a fixed order.
__global__ void __launch_bounds__(kThreads) chunkKernel(const double* __restrict__ state, long long n,
                                                        const unsigned char* __restrict__ isFluid, double* partials) {
    long long begin = blockIdx.x*kChunkNodes, end = begin + kChunkNodes < n ? begin + kChunkNodes : n;
    double acc[kRecord] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (long long node = begin + threadIdx.x; node < end; node += kThreads) {
        if (isFluid != nullptr && !isFluid[node])
            continue;
        double dr = 0, jx = 0, jy = 0, jz = 0;
        for (int q = 0; q < 19; q++) {
            double f = state[(long long) q*n + node];
            dr += f;
            jx += cxOf(q)*f;
            jy += cyOf(q)*f;
            jz += czOf(q)*f;
        }
        double rho = 1.0 + dr;
        acc[0] += dr;
        acc[1] += jx;
        acc[2] += jy;
        acc[3] += jz;
        acc[7] = fmax(acc[7], (jx*jx + jy*jy + jz*jz)/(rho*rho));
    }
    __shared__ double red[kThreads/32][kRecord];
    int lane = threadIdx.x%32, warp = threadIdx.x/32;
    for (int k = 0; k < kRecord; k++)
        for (int o = 16; o > 0; o >>= 1) {
            double other = __shfl_down_sync(0xffffffffu, acc[k], o);
            acc[k] = (k == kRecord-1 ? fmax(acc[k], other) : acc[k] + other);
        }
    if (lane == 0)
        for (int k = 0; k < kRecord; k++)
            red[warp][k] = acc[k];
    __syncthreads();
    if (threadIdx.x < kRecord) {
        int k = threadIdx.x;
        double s = red[0][k];
        for (int w = 1; w < kThreads/32; w++)
            s = (k == kRecord-1 ? fmax(s, red[w][k]) : s + red[w][k]);
        partials[kRecord*(long long) blockIdx.x + k] = s;
    }
}

// One block: the records of the chunks in chunk order; moments = {mass deviation, momentum x/y/z, Mach number}.
__global__ void __launch_bounds__(32) finishChunksKernel(const double* partials, int chunks, double* moments) {
    if (threadIdx.x < 4) {
        double s = 0;
        for (int c = 0; c < chunks; c++)
            s += partials[kRecord*c + threadIdx.x];
        moments[threadIdx.x] = s;
    }
    else if (threadIdx.x == 4) {
        double m = 0;
        for (int c = 0; c < chunks; c++)
            m = fmax(m, partials[kRecord*c + kRecord-1]);
        moments[4] = sqrt(3.0*m);
    }
}

} // namespace
} // namespace lbm

extern "C" LbmStatus lbm_fluid_moments_noalloc(const double* state, long long num_nodes, const unsigned char* is_fluid,
                                               double* moments, void* stream) {
    using namespace lbm;
    if (state == nullptr || moments == nullptr || num_nodes <= 0) {
        setLastError("lbm_fluid_moments_noalloc: null array or no nodes");
        return LBM_ERR_INVALID_ARGUMENT;
    }
    if (num_nodes > (long long) kMaxChunks*kChunkNodes) {
        setLastError("lbm_fluid_moments_noalloc: " + std::to_string(num_nodes) + " nodes is more than the " +
                     std::to_string((long long) kMaxChunks*kChunkNodes) + " that its fixed scratch array can reduce");
        return LBM_ERR_INVALID_ARGUMENT;
    }
    try {
        int device = 0;
        cudaError_t e = cudaGetDevice(&device);
        if (e != cudaSuccess)
            throw Error(LBM_ERR_CUDA, std::string("lbm_fluid_moments_noalloc: ") + cudaGetErrorString(e));
        if (device < 0 || device >= kMaxDevices)
            throw Error(LBM_ERR_NOT_SUPPORTED, "lbm_fluid_moments_noalloc: device ordinal out of range");
        double* partials = scratchAddress(device);
        int chunks = (int) ((num_nodes + kChunkNodes - 1)/kChunkNodes);
        cudaStream_t s = (cudaStream_t) stream;
        chunkKernel<<<chunks, kThreads, 0, s>>>(state, num_nodes, is_fluid, partials);
        finishChunksKernel<<<1, 32, 0, s>>>(partials, chunks, moments);
        e = cudaGetLastError();
        if (e != cudaSuccess)
            throw Error(LBM_ERR_CUDA, std::string("lbm_fluid_moments_noalloc: ") + cudaGetErrorString(e));
        return LBM_OK;
    }
    catch (const Error& err) {
        setLastError(err.what());
        return err.status;
    }
}
