// Tensor-core 3x3x3 convolutions of the learned warm start (include/lbm_b200_warmstart.h), written for sm_100a:
//
//  convForwardKernel    y[voxel][cout] = sum_k A[voxel][k] W[cout][k], k = tap*cin + ci, A the implicit im2col of x
//                       (zero padding); one CTA per 128 voxels, all cout in one N tile (<= 256)
//  convWeightGradKernel dW[cout][k] = sum_voxels dy[voxel][cout] A[voxel][k]; CTAs over (cout tile, k tile, voxel
//                       split), the K dimension of the GEMM being the voxels; results added with FP32 atomics
//
// The GEMM core: 128 x N tiles, K in stages of 64 BF16 (one 128-byte row).  All 128 threads gather a stage into
// shared memory in the canonical K-major layout with the 128-byte swizzle (8-row atoms of 128-byte rows, the 16-byte
// chunk index XOR the row within the atom), make it visible to the tensor core's proxy, and one thread issues four
// tcgen05.mma (K = 16 each, BF16 x BF16 -> FP32 in tensor memory) and commits them to an mbarrier that every
// thread waits on (bounded: a wait that gives up sets the status flag and the CTA leaves after freeing its tensor
// memory).  The epilogue reads the accumulators with tcgen05.ld (warp w owns lanes 32w..32w+31 = rows of the tile).
// Descriptor layouts: the shared-memory matrix descriptor (start >> 4, leading offset, stride offset 1024 B >> 4,
// version 1, swizzle mode 2 = 128 B) and the instruction descriptor (F32 accumulator, BF16 A and B, both K-major,
// N >> 3, M >> 4) of the PTX ISA's tcgen05 matrix and instruction descriptor formats.
#include "lbm_b200_warmstart.h"
#include "lbm_internal.h"
#include <cuda_bf16.h>
#include <algorithm>
#include <cstdint>
#include <string>

namespace {

constexpr int kThreads = 128;
constexpr int kTileM = 128;
constexpr int kChunk = 64;                     // BF16 per stage row
constexpr long long kSpinLimit = 1LL << 24;    // polls of an mbarrier before giving up

__device__ int convStatus;
// Polls of the waits for the tensor cores (kSpinLimit unless lbm_conv3d_set_wait_limit lowered it).  The drain of a
// stage whose wait gave up always uses kSpinLimit.
__device__ long long convWaitPolls = kSpinLimit;

__device__ __forceinline__ uint32_t smemAddr(const void* p) {
    return (uint32_t) __cvta_generic_to_shared(p);
}

// Shared-memory matrix descriptor of a K-major operand tile with the 128-byte swizzle.
__device__ __forceinline__ uint64_t smemDescriptor(uint32_t addr) {
    return (uint64_t) ((addr >> 4) & 0x3FFFu)
         | ((uint64_t) 1 << 16)                    // leading byte offset (16 B; unused for swizzled K-major)
         | ((uint64_t) (1024 >> 4) << 32)          // stride byte offset: 8-row atoms 1024 B apart
         | ((uint64_t) 1 << 46)                    // descriptor version of sm_100
         | ((uint64_t) 2 << 61);                   // 128-byte swizzle
}

// Instruction descriptor: FP32 accumulator, BF16 A and B, both K-major, M = 128, N = n.
__device__ __forceinline__ uint32_t instrDescriptor(int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t) (n >> 3) << 17) | ((uint32_t) (kTileM >> 4) << 24);
}

// Byte offset of 16-byte chunk `chunk` (0..7) of row `row` in a swizzled tile.
__device__ __forceinline__ uint32_t swizzled(int row, int chunk) {
    return (uint32_t) (row*128 + ((chunk ^ (row & 7)) << 4));
}

__device__ __forceinline__ void mmaBf16(uint32_t tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accumulate) {
    asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                 "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
                 :: "r"(tmem), "l"(a), "l"(b), "r"(idesc), "r"(accumulate) : "memory");
}

__device__ __forceinline__ void commitTo(uint32_t mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" :: "r"(mbar) : "memory");
}

__device__ __forceinline__ bool waitParity(uint32_t mbar, uint32_t parity, long long limit) {
    for (long long i = 0; i < limit; i++) {
        uint32_t done;
        asm volatile("{\n\t.reg .pred P1;\n\tmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
                     "selp.b32 %0, 1, 0, P1;\n\t}" : "=r"(done) : "r"(mbar), "r"(parity) : "memory");
        if (done)
            return true;
    }
    return false;
}

__device__ __forceinline__ void fenceAfterSync() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fenceBeforeSync() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}

// 8 consecutive FP32 accumulator columns of this thread's row (lane) from tensor memory.
__device__ __forceinline__ void tmemLoad8(uint32_t addr, float v[8]) {
    uint32_t r[8];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                 : "r"(addr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
    for (int i = 0; i < 8; i++)
        v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ uint32_t tmemColumns(int n) {
    return n <= 32 ? 32u : (n <= 64 ? 64u : (n <= 128 ? 128u : 256u));
}

// Setup common to both kernels: 1024-byte aligned tiles, tensor memory of `ncols` columns (warp 0), the mbarrier.
struct Stage {
    uint8_t* tileA;
    uint8_t* tileB;
    uint32_t mbar;
    uint32_t tmem;
};

__device__ __forceinline__ Stage setupStage(uint8_t* raw, int rowsB, uint32_t ncols) {
    uint32_t s = smemAddr(raw);
    uint8_t* base = raw + ((1024 - (s & 1023)) & 1023);
    Stage st;
    st.tileA = base;
    st.tileB = base + kTileM*128;
    uint64_t* bar = reinterpret_cast<uint64_t*>(st.tileB + rowsB*128);
    uint32_t* slot = reinterpret_cast<uint32_t*>(bar + 1);
    st.mbar = smemAddr(bar);
    if (threadIdx.x/32 == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" :: "r"(smemAddr(slot)), "r"(ncols) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(st.mbar), "r"(1) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    fenceBeforeSync();
    __syncthreads();
    fenceAfterSync();
    st.tmem = *slot;
    return st;
}

__device__ __forceinline__ void releaseStage(const Stage& st, uint32_t ncols) {
    fenceBeforeSync();
    __syncthreads();
    if (threadIdx.x/32 == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(st.tmem), "r"(ncols) : "memory");
}

// One stage: the tiles are in shared memory; thread 0 issues the four K = 16 MMAs and commits; all threads wait.
// Returns false (for every thread) if the wait gave up; the caller then drains the stage (drainStage) before it
// frees the tensor memory that the MMAs may still be writing.
__device__ __forceinline__ bool runStage(const Stage& st, uint32_t idesc, int stage, long long limit) {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (threadIdx.x == 0) {
        fenceAfterSync();
        uint32_t a = smemAddr(st.tileA), b = smemAddr(st.tileB);
        for (int j = 0; j < 4; j++)
            mmaBf16(st.tmem, smemDescriptor(a + 32*j), smemDescriptor(b + 32*j), idesc, (stage > 0 || j > 0) ? 1u : 0u);
        commitTo(st.mbar);
    }
    bool ok = waitParity(st.mbar, (uint32_t) (stage & 1), limit);
    return __syncthreads_and(ok) != 0;
}

// After a wait that gave up: wait once more, with the full limit, for the MMAs of that stage (the only ones in flight),
// so that the tensor memory and the shared-memory tiles are released only when the tensor cores are done with them.
__device__ __forceinline__ void drainStage(const Stage& st, int stage) {
    waitParity(st.mbar, (uint32_t) (stage & 1), kSpinLimit);
    __syncthreads();
}

__global__ void __launch_bounds__(kThreads)
convForwardKernel(const __nv_bfloat16* __restrict__ x, const __nv_bfloat16* __restrict__ w, const float* __restrict__ bias,
                  __nv_bfloat16* __restrict__ y, int batch, int D, int H, int W, int cin, int cout, int relu) {
    extern __shared__ uint8_t smemRaw[];
    const uint32_t ncols = tmemColumns(cout);
    Stage st = setupStage(smemRaw, cout, ncols);
    const int tid = threadIdx.x, warp = tid/32, lane = tid%32;
    const long long M = (long long) batch*D*H*W;
    const int K = 27*cin, stages = (K + kChunk - 1)/kChunk;
    const uint32_t idesc = instrDescriptor(cout);
    // The voxel of this thread's row of A.
    const long long m = (long long) blockIdx.x*kTileM + tid;
    const bool valid = m < M;
    int vx = 0, vy = 0, vz = 0, vn = 0;
    if (valid) {
        long long r = m;
        vx = (int) (r%W); r /= W;
        vy = (int) (r%H); r /= H;
        vz = (int) (r%D); vn = (int) (r/D);
    }
    const long long limit = convWaitPolls;
    bool ok = true;
    int failedStage = -1;
    for (int c = 0; c < stages && ok; c++) {
        for (int kv = 0; kv < 8; kv++) {
            int k = c*kChunk + kv*8;
            uint4 val = make_uint4(0, 0, 0, 0);
            if (valid && k < K) {
                int tap = k/cin, ci = k - tap*cin;
                int zz = vz + tap/9 - 1, yy = vy + (tap/3)%3 - 1, xx = vx + tap%3 - 1;
                if (zz >= 0 && zz < D && yy >= 0 && yy < H && xx >= 0 && xx < W)
                    val = __ldg(reinterpret_cast<const uint4*>(x + ((((long long) vn*D + zz)*H + yy)*W + xx)*cin + ci));
            }
            *reinterpret_cast<uint4*>(st.tileA + swizzled(tid, kv)) = val;
        }
        for (int i = tid; i < cout*8; i += kThreads) {
            int row = i >> 3, kv = i & 7, k = c*kChunk + kv*8;
            uint4 val = make_uint4(0, 0, 0, 0);
            if (k < K)
                val = __ldg(reinterpret_cast<const uint4*>(w + (long long) row*K + k));
            *reinterpret_cast<uint4*>(st.tileB + swizzled(row, kv)) = val;
        }
        ok = runStage(st, idesc, c, limit);
        if (!ok)
            failedStage = c;
    }
    if (!ok)
        drainStage(st, failedStage);
    fenceAfterSync();
    if (ok) {
        const int row = warp*32 + lane;
        const long long mo = (long long) blockIdx.x*kTileM + row;
        for (int col = 0; col < cout; col += 8) {
            float v[8];
            tmemLoad8(st.tmem + ((uint32_t) (warp*32) << 16) + (uint32_t) col, v);
            if (mo < M) {
                __align__(16) __nv_bfloat16 out[8];
                for (int i = 0; i < 8; i++) {
                    float t = v[i] + (bias ? bias[col + i] : 0.0f);
                    out[i] = __float2bfloat16_rn(relu ? fmaxf(t, 0.0f) : t);
                }
                *reinterpret_cast<uint4*>(y + mo*cout + col) = *reinterpret_cast<const uint4*>(out);
            }
        }
    }
    else if (tid == 0)
        atomicExch(&convStatus, (int) LBM_ERR_DEVICE_TIMEOUT);
    releaseStage(st, ncols);
}

// dW[cout][k] += sum_m dy[m][cout] A[m][k]: A tile rows = cout (tile of 128), B tile rows = k (tile of nt), the GEMM's
// K = voxels in stages of 64.  Both tiles are gathered transposed (voxel along the 128-byte rows).
__global__ void __launch_bounds__(kThreads)
convWeightGradKernel(const __nv_bfloat16* __restrict__ x, const __nv_bfloat16* __restrict__ dy, float* __restrict__ dw,
                     int batch, int D, int H, int W, int cin, int cout, int nt) {
    extern __shared__ uint8_t smemRaw[];
    const uint32_t ncols = tmemColumns(nt);
    Stage st = setupStage(smemRaw, nt, ncols);
    const int tid = threadIdx.x, warp = tid/32, lane = tid%32;
    const long long M = (long long) batch*D*H*W;
    const int K = 27*cin;
    const int co0 = blockIdx.x*kTileM, k0 = blockIdx.y*nt;
    const long long stagesTotal = (M + kChunk - 1)/kChunk;
    const uint32_t idesc = instrDescriptor(nt);
    const int col = tid%kChunk, half = tid/kChunk;       // this thread's voxel column and row-group parity
    const long long limit = convWaitPolls;
    bool ok = true;
    int stage = 0;
    for (long long c = blockIdx.z; c < stagesTotal && ok; c += gridDim.z, stage++) {
        const long long m = c*kChunk + col;
        const bool valid = m < M;
        int vx = 0, vy = 0, vz = 0, vn = 0;
        if (valid) {
            long long r = m;
            vx = (int) (r%W); r /= W;
            vy = (int) (r%H); r /= H;
            vz = (int) (r%D); vn = (int) (r/D);
        }
        const uint32_t colOffset = (uint32_t) ((col & 7)*2);
        // A: rows cout (16 groups of 8), column = this voxel.
        for (int g = half; g < kTileM/8; g += 2) {
            int co = co0 + 8*g;
            uint4 val = make_uint4(0, 0, 0, 0);
            if (valid && co < cout)
                val = __ldg(reinterpret_cast<const uint4*>(dy + m*cout + co));
            const __nv_bfloat16* e = reinterpret_cast<const __nv_bfloat16*>(&val);
            for (int i = 0; i < 8; i++)
                *reinterpret_cast<__nv_bfloat16*>(st.tileA + swizzled(8*g + i, col >> 3) + colOffset) = e[i];
        }
        // B: rows k = k0 + 8 g + i (one tap and 8 channels per group), column = this voxel.
        for (int g = half; g < nt/8; g += 2) {
            int k = k0 + 8*g;
            uint4 val = make_uint4(0, 0, 0, 0);
            if (valid && k < K) {
                int tap = k/cin, ci = k - tap*cin;
                int zz = vz + tap/9 - 1, yy = vy + (tap/3)%3 - 1, xx = vx + tap%3 - 1;
                if (zz >= 0 && zz < D && yy >= 0 && yy < H && xx >= 0 && xx < W)
                    val = __ldg(reinterpret_cast<const uint4*>(x + ((((long long) vn*D + zz)*H + yy)*W + xx)*cin + ci));
            }
            const __nv_bfloat16* e = reinterpret_cast<const __nv_bfloat16*>(&val);
            for (int i = 0; i < 8; i++)
                *reinterpret_cast<__nv_bfloat16*>(st.tileB + swizzled(8*g + i, col >> 3) + colOffset) = e[i];
        }
        ok = runStage(st, idesc, stage, limit);
        if (!ok)
            drainStage(st, stage);
    }
    fenceAfterSync();
    if (ok && stage > 0) {
        const int row = warp*32 + lane, co = co0 + row;
        for (int c0 = 0; c0 < nt; c0 += 8) {
            float v[8];
            tmemLoad8(st.tmem + ((uint32_t) (warp*32) << 16) + (uint32_t) c0, v);
            if (co < cout)
                for (int i = 0; i < 8; i++) {
                    int k = k0 + c0 + i;
                    if (k < K)
                        atomicAdd(&dw[(long long) co*K + k], v[i]);
                }
        }
    }
    else if (!ok && tid == 0)
        atomicExch(&convStatus, (int) LBM_ERR_DEVICE_TIMEOUT);
    releaseStage(st, ncols);
}

size_t stageBytes(int rowsB) {
    return 1024 + (size_t) kTileM*128 + (size_t) rowsB*128 + 64;
}

LbmStatus launchError(cudaError_t e) {
    lbm::setLastError(std::string("conv3d: ") + cudaGetErrorString(e));
    return LBM_ERR_CUDA;
}

LbmStatus invalid(const char* message) {
    lbm::setLastError(message);
    return LBM_ERR_INVALID_ARGUMENT;
}

} // namespace

extern "C" {

LbmStatus lbm_conv3d_forward(const void* x, const void* w, const float* bias, void* y, int batch, int depth, int height,
                             int width, int cin, int cout, int relu, void* stream) {
    if (!x || !w || !y || batch <= 0 || depth <= 0 || height <= 0 || width <= 0)
        return invalid("lbm_conv3d_forward: null pointer or empty volume");
    if (cin <= 0 || cin%8 != 0 || cout < 16 || cout > 256 || cout%16 != 0)
        return invalid("lbm_conv3d_forward: cin must be a multiple of 8 and cout a multiple of 16 up to 256");
    long long voxels = (long long) batch*depth*height*width;
    size_t smem = stageBytes(cout);
    cudaError_t e = cudaFuncSetAttribute(convForwardKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem);
    if (e != cudaSuccess)
        return launchError(e);
    unsigned grid = (unsigned) ((voxels + kTileM - 1)/kTileM);
    convForwardKernel<<<grid, kThreads, smem, (cudaStream_t) stream>>>(
        (const __nv_bfloat16*) x, (const __nv_bfloat16*) w, bias, (__nv_bfloat16*) y, batch, depth, height, width, cin,
        cout, relu);
    e = cudaGetLastError();
    return e == cudaSuccess ? LBM_OK : launchError(e);
}

LbmStatus lbm_conv3d_weight_grad(const void* x, const void* dy, float* dw, int batch, int depth, int height, int width,
                                 int cin, int cout, void* stream) {
    if (!x || !dy || !dw || batch <= 0 || depth <= 0 || height <= 0 || width <= 0)
        return invalid("lbm_conv3d_weight_grad: null pointer or empty volume");
    if (cin <= 0 || cin%8 != 0 || cout < 16 || cout > 256 || cout%16 != 0)
        return invalid("lbm_conv3d_weight_grad: cin must be a multiple of 8 and cout a multiple of 16 up to 256");
    long long voxels = (long long) batch*depth*height*width;
    int K = 27*cin;
    int nt = ((K + 15)/16)*16;
    if (nt > 256)
        nt = 256;
    int device = 0, sms = 148;
    cudaGetDevice(&device);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    unsigned gx = (unsigned) ((cout + kTileM - 1)/kTileM), gy = (unsigned) ((K + nt - 1)/nt);
    long long stages = (voxels + kChunk - 1)/kChunk;
    long long gz = std::max(1LL, std::min(stages, (long long) (4*sms)/(long long) (gx*gy) + 1));
    size_t smem = stageBytes(nt);
    cudaError_t e = cudaFuncSetAttribute(convWeightGradKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem);
    if (e != cudaSuccess)
        return launchError(e);
    convWeightGradKernel<<<dim3(gx, gy, (unsigned) gz), kThreads, smem, (cudaStream_t) stream>>>(
        (const __nv_bfloat16*) x, (const __nv_bfloat16*) dy, dw, batch, depth, height, width, cin, cout, nt);
    e = cudaGetLastError();
    return e == cudaSuccess ? LBM_OK : launchError(e);
}

LbmStatus lbm_conv3d_status(void* stream) {
    cudaError_t e = cudaStreamSynchronize((cudaStream_t) stream);
    if (e != cudaSuccess)
        return launchError(e);
    int status = 0;
    e = cudaMemcpyFromSymbol(&status, convStatus, sizeof(int));
    if (e != cudaSuccess)
        return launchError(e);
    int zero = 0;
    cudaMemcpyToSymbol(convStatus, &zero, sizeof(int));
    if (status != 0) {
        lbm::setLastError("conv3d: a wait for the tensor cores timed out");
        return (LbmStatus) status;
    }
    return LBM_OK;
}

LbmStatus lbm_conv3d_set_wait_limit(long long polls) {
    long long value = polls >= 0 ? polls : kSpinLimit;
    cudaError_t e = cudaMemcpyToSymbol(convWaitPolls, &value, sizeof(long long));
    return e == cudaSuccess ? LBM_OK : launchError(e);
}

} // extern "C"
