// Bead dynamics on the device (include/lbm_b200_md.h): the forces and the leapfrog integrator that OpenMM would
// provide around the LBM force kernel in the benchmark configurations.  Harmonic bonds, and WCA or truncated
// Lennard-Jones pairs found with a cell list: particles are binned by cell with atomics into fixed-capacity bins,
// and one warp per particle visits the 27 cells around its own (a lane per cell, taking the cell's particles in index
// order, and a lane for the bonds), the lanes' forces summed by a fixed shuffle tree (so every force is summed in one
// order); a cell over its capacity is scanned over all particles instead (a brute-force pass serves boxes with fewer
// than 3 cells along an axis).
#include "lbm_internal.h"
#include "lbm_b200_md.h"
#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

namespace lbm {

#define CUDA_CHECK(call) do { cudaError_t e_ = (call); if (e_ != cudaSuccess) \
    throw Error(LBM_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); } while (0)

namespace {

struct MdView {
    int n;
    double box[3];
    double invBox[3];
    int ncell[3];
    double cellSize[3];
    double k, r0;
    int pairType;
    double sigma2, eps, rc2;
    const double* invMass;
    const int* bondOffset;
    const int* bondPartner;
    const unsigned* cellKey;   // cell of each particle
    const unsigned* binCount;  // particles per cell (cleared after each force pass)
    const int* bins;           // binCapacity per cell: the particles of the cell, in arbitrary order
    int binCapacity;
};

constexpr int kMaxBinCapacity = 16;

// Minimum image.  d/box is taken as d*(1/box): the two differ by an ulp at most, which can move rint() only for a
// separation of half a box, far beyond every cutoff and bond length (the box holds at least 3 cells of the cutoff).
__device__ __forceinline__ void minimumImage(const MdView& v, double d[3]) {
    for (int a = 0; a < 3; a++)
        d[a] -= v.box[a]*rint(d[a]*v.invBox[a]);
}

__device__ __forceinline__ int cellOf(const MdView& v, const double* x, int a) {
    double s = x[a] - floor(x[a]/v.box[a])*v.box[a];
    int c = (int) (s/v.cellSize[a]);
    return c >= v.ncell[a] ? v.ncell[a] - 1 : c;
}

__device__ __forceinline__ bool bonded(const MdView& v, int i, int j) {
    for (int b = v.bondOffset[i]; b < v.bondOffset[i+1]; b++)
        if (v.bondPartner[b] == j)
            return true;
    return false;
}

// Pair force on i from j (d = x_i - x_j, minimum image), added to f.
__device__ __forceinline__ void pairForce(const MdView& v, const double d[3], double f[3]) {
    double r2 = d[0]*d[0] + d[1]*d[1] + d[2]*d[2];
    if (r2 >= v.rc2 || r2 == 0.0)
        return;
    double s2 = v.sigma2/r2, s6 = s2*s2*s2;
    double scale = 24.0*v.eps*s6*(2.0*s6 - 1.0)/r2;
    for (int a = 0; a < 3; a++)
        f[a] += scale*d[a];
}

__device__ void bondForces(const MdView& v, const double* pos, int i, double f[3]) {
    for (int b = v.bondOffset[i]; b < v.bondOffset[i+1]; b++) {
        int j = v.bondPartner[b];
        double d[3] = {pos[3*i] - pos[3*j], pos[3*i+1] - pos[3*j+1], pos[3*i+2] - pos[3*j+2]};
        minimumImage(v, d);
        double r = sqrt(d[0]*d[0] + d[1]*d[1] + d[2]*d[2]);
        if (r == 0.0)
            continue;
        double scale = -v.k*(r - v.r0)/r;
        for (int a = 0; a < 3; a++)
            f[a] += scale*d[a];
    }
}

__global__ void binKernel(MdView v, const double* pos, unsigned* cellKey, unsigned* binCount, int* bins) {
    for (int i = blockIdx.x*blockDim.x + threadIdx.x; i < v.n; i += gridDim.x*blockDim.x) {
        const double* x = &pos[3*i];
        const unsigned key = (unsigned) (cellOf(v, x, 0) + v.ncell[0]*(cellOf(v, x, 1) + v.ncell[1]*cellOf(v, x, 2)));
        cellKey[i] = key;
        const unsigned slot = atomicAdd(&binCount[key], 1u);
        if (slot < (unsigned) v.binCapacity)
            bins[(size_t) key*v.binCapacity + slot] = i;
    }
}

__global__ void clearBinsKernel(int n, const unsigned* cellKey, unsigned* binCount) {
    for (int i = blockIdx.x*blockDim.x + threadIdx.x; i < n; i += gridDim.x*blockDim.x)
        binCount[cellKey[i]] = 0u;
}

__device__ __forceinline__ void pairWith(const MdView& v, const double* pos, int i, const double* x, int j, double f[3]) {
    if (j == i || bonded(v, i, j))
        return;
    double d[3] = {x[0] - pos[3*j], x[1] - pos[3*j+1], x[2] - pos[3*j+2]};
    minimumImage(v, d);
    pairForce(v, d, f);
}

// The same forces with one warp per particle, for latency: lane c < 27 takes the neighbouring cell c (its members in
// index order), lane 27 the bonds, and the lanes' forces are summed by a fixed shuffle tree.
__global__ void __launch_bounds__(256) cellForceWarpKernel(MdView v, const double* pos, double* forces) {
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x*blockDim.x) >> 5;
    for (int i = (blockIdx.x*blockDim.x + threadIdx.x) >> 5; i < v.n; i += warps) {
        double f[3] = {0, 0, 0};
        const double x[3] = {pos[3*i], pos[3*i+1], pos[3*i+2]};
        if (lane == 27)
            bondForces(v, pos, i, f);
        else if (lane < 27 && v.pairType != LBM_PAIR_NONE) {
            const int c[3] = {cellOf(v, x, 0), cellOf(v, x, 1), cellOf(v, x, 2)};
            const int cx = (c[0] + lane%3 - 1 + v.ncell[0])%v.ncell[0];
            const int cy = (c[1] + (lane/3)%3 - 1 + v.ncell[1])%v.ncell[1];
            const int cz = (c[2] + lane/9 - 1 + v.ncell[2])%v.ncell[2];
            const unsigned cell = (unsigned) (cx + v.ncell[0]*(cy + v.ncell[1]*cz));
            const int count = (int) v.binCount[cell];
            if (count <= v.binCapacity) {
                int member[kMaxBinCapacity];
                for (int e = 0; e < count; e++) {
                    int j = v.bins[(size_t) cell*v.binCapacity + e], p = e;
                    while (p > 0 && member[p-1] > j) {
                        member[p] = member[p-1];
                        p--;
                    }
                    member[p] = j;
                }
                for (int e = 0; e < count; e++)
                    pairWith(v, pos, i, x, member[e], f);
            }
            else
                for (int j = 0; j < v.n; j++)
                    if (v.cellKey[j] == cell)
                        pairWith(v, pos, i, x, j, f);
        }
        for (int a = 0; a < 3; a++)
            for (int o = 16; o > 0; o >>= 1)
                f[a] += __shfl_down_sync(0xffffffffu, f[a], o);
        if (lane == 0)
            for (int a = 0; a < 3; a++)
                forces[3*i+a] = f[a];
    }
}

__global__ void bruteForceKernel(MdView v, const double* pos, double* forces) {
    for (int i = blockIdx.x*blockDim.x + threadIdx.x; i < v.n; i += gridDim.x*blockDim.x) {
        double f[3] = {0, 0, 0};
        bondForces(v, pos, i, f);
        if (v.pairType != LBM_PAIR_NONE)
            for (int j = 0; j < v.n; j++) {
                if (j == i || bonded(v, i, j))
                    continue;
                double d[3] = {pos[3*i] - pos[3*j], pos[3*i+1] - pos[3*j+1], pos[3*i+2] - pos[3*j+2]};
                minimumImage(v, d);
                pairForce(v, d, f);
            }
        for (int a = 0; a < 3; a++)
            forces[3*i+a] = f[a];
    }
}

__global__ void leapfrogKernel(int n, const double* invMass, double dt, double* pos, double* vel, const double* f) {
    for (int t = blockIdx.x*blockDim.x + threadIdx.x; t < 3*n; t += gridDim.x*blockDim.x) {
        double v = vel[t] + dt*f[t]*invMass[t/3];
        vel[t] = v;
        pos[t] += dt*v;
    }
}

__global__ void kineticKernel(int n, const double* invMass, const double* vel, double* out) {
    __shared__ double red[32];
    double s = 0;
    for (int t = threadIdx.x; t < 3*n; t += blockDim.x)
        s += vel[t]*vel[t]/invMass[t/3];
    for (int o = 16; o > 0; o >>= 1)
        s += __shfl_down_sync(0xffffffffu, s, o);
    if (threadIdx.x%32 == 0)
        red[threadIdx.x/32] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double total = 0;
        for (int w = 0; w < (int) blockDim.x/32; w++)
            total += red[w];
        *out = total;
    }
}

int gridFor(long long work) {
    return (int) std::max(1LL, std::min(2368LL, (work + 255)/256));
}

} // namespace

struct MdEngine {
    MdView view;
    int device;
    double* invMass = nullptr;
    int* bondOffset = nullptr;
    int* bondPartner = nullptr;
    unsigned* cellKey = nullptr;
    unsigned* binCount = nullptr;
    int* bins = nullptr;
    double* scalar = nullptr;
    bool brute = true;
    long long ncells = 0;
    long long launches = 0;

    MdEngine(int n, const double* masses, const double box[3], int numBonds, const int* bonds, double k, double r0,
             int pairType, double sigma, double eps, double cutoff, int dev) : device(dev) {
        if (n <= 0 || masses == nullptr || box == nullptr || (numBonds > 0 && bonds == nullptr))
            throw Error(LBM_ERR_INVALID_ARGUMENT, "lbm_md_create: invalid arguments");
        if (pairType != LBM_PAIR_NONE && pairType != LBM_PAIR_WCA && pairType != LBM_PAIR_LJ)
            throw Error(LBM_ERR_INVALID_ARGUMENT, "lbm_md_create: unknown pair type");
        CUDA_CHECK(cudaSetDevice(device));
        view = MdView();
        view.n = n;
        for (int a = 0; a < 3; a++) {
            view.box[a] = box[a];
            view.invBox[a] = 1.0/box[a];
        }
        view.k = k;
        view.r0 = r0;
        view.pairType = pairType;
        view.sigma2 = sigma*sigma;
        view.eps = eps;
        double rc = (pairType == LBM_PAIR_WCA ? std::pow(2.0, 1.0/6.0)*sigma : cutoff);
        view.rc2 = rc*rc;
        brute = false;
        ncells = 1;
        for (int a = 0; a < 3; a++) {
            view.ncell[a] = std::max(1, (int) std::floor(box[a]/rc));
            view.cellSize[a] = box[a]/view.ncell[a];
            if (view.ncell[a] < 3)
                brute = true;
            ncells *= view.ncell[a];
        }
        if (pairType == LBM_PAIR_NONE)
            brute = true;
        // Bin capacity: WCA cells (no smaller than 2^(1/6) sigma) hold few particles of a repulsive fluid; truncated
        // Lennard-Jones cells (no smaller than the cutoff) hold a liquid's.  The bins stay under 2 GB: larger boxes
        // take fewer, larger cells.
        view.binCapacity = pairType == LBM_PAIR_WCA ? 8 : kMaxBinCapacity;
        while (!brute && ncells*view.binCapacity*(long long) sizeof(int) > (2LL << 30)) {
            int a = view.ncell[0] >= view.ncell[1] && view.ncell[0] >= view.ncell[2] ? 0 : (view.ncell[1] >= view.ncell[2] ? 1 : 2);
            ncells /= view.ncell[a];
            view.ncell[a] = std::max(3, view.ncell[a]/2);
            view.cellSize[a] = box[a]/view.ncell[a];
            ncells *= view.ncell[a];
        }
        // Bonds as adjacency lists (CSR).
        std::vector<int> count(n + 1, 0), offset(n + 1, 0), partner(2*(size_t) numBonds);
        for (int b = 0; b < numBonds; b++) {
            int i = bonds[2*b], j = bonds[2*b+1];
            if (i < 0 || i >= n || j < 0 || j >= n || i == j)
                throw Error(LBM_ERR_INVALID_ARGUMENT, "lbm_md_create: a bond has an invalid particle index");
            count[i]++;
            count[j]++;
        }
        for (int i = 0; i < n; i++)
            offset[i+1] = offset[i] + count[i];
        std::vector<int> fill(offset.begin(), offset.end() - 1);
        for (int b = 0; b < numBonds; b++) {
            int i = bonds[2*b], j = bonds[2*b+1];
            partner[fill[i]++] = j;
            partner[fill[j]++] = i;
        }
        std::vector<double> inv(n);
        for (int i = 0; i < n; i++) {
            if (!(masses[i] > 0))
                throw Error(LBM_ERR_INVALID_ARGUMENT, "lbm_md_create: masses must be positive");
            inv[i] = 1.0/masses[i];
        }
        try {
            CUDA_CHECK(cudaMalloc(&invMass, sizeof(double)*n));
            CUDA_CHECK(cudaMemcpy(invMass, inv.data(), sizeof(double)*n, cudaMemcpyHostToDevice));
            CUDA_CHECK(cudaMalloc(&bondOffset, sizeof(int)*(n + 1)));
            CUDA_CHECK(cudaMemcpy(bondOffset, offset.data(), sizeof(int)*(n + 1), cudaMemcpyHostToDevice));
            CUDA_CHECK(cudaMalloc(&bondPartner, sizeof(int)*std::max<size_t>(1, partner.size())));
            if (!partner.empty())
                CUDA_CHECK(cudaMemcpy(bondPartner, partner.data(), sizeof(int)*partner.size(), cudaMemcpyHostToDevice));
            CUDA_CHECK(cudaMalloc(&scalar, sizeof(double)*4));
            if (!brute) {
                CUDA_CHECK(cudaMalloc(&cellKey, sizeof(unsigned)*n));
                CUDA_CHECK(cudaMalloc(&binCount, sizeof(unsigned)*ncells));
                CUDA_CHECK(cudaMemset(binCount, 0, sizeof(unsigned)*ncells));
                CUDA_CHECK(cudaMalloc(&bins, sizeof(int)*(size_t) ncells*view.binCapacity));
            }
        }
        catch (...) {
            release();
            throw;
        }
        view.invMass = invMass;
        view.bondOffset = bondOffset;
        view.bondPartner = bondPartner;
        view.cellKey = cellKey;
        view.binCount = binCount;
        view.bins = bins;
    }
    void release() {
        cudaFree(invMass); cudaFree(bondOffset); cudaFree(bondPartner); cudaFree(cellKey); cudaFree(binCount);
        cudaFree(bins);
        cudaFree(scalar);
        invMass = nullptr; bondOffset = bondPartner = bins = nullptr;
        cellKey = binCount = nullptr;
        scalar = nullptr;
    }
    ~MdEngine() { release(); }

    void forces(const double* pos, double* out, cudaStream_t s) {
        CUDA_CHECK(cudaSetDevice(device));
        int n = view.n;
        if (brute) {
            bruteForceKernel<<<gridFor(n), 256, 0, s>>>(view, pos, out);
            CUDA_CHECK(cudaGetLastError());
            launches++;
            return;
        }
        binKernel<<<gridFor(n), 256, 0, s>>>(view, pos, cellKey, binCount, bins);
        cellForceWarpKernel<<<gridFor(32LL*n), 256, 0, s>>>(view, pos, out);
        // Empty the occupied bins, so that the next call starts from empty cells.
        clearBinsKernel<<<gridFor(n), 256, 0, s>>>(n, cellKey, binCount);
        CUDA_CHECK(cudaGetLastError());
        launches += 3;
    }
};

} // namespace lbm

struct LbmMd {
    lbm::MdEngine* impl;
};

extern "C" {

LbmStatus lbm_md_create(int n, const double* masses, const double box[3], int num_bonds, const int* bonds, double k,
                        double r0, int pair_type, double sigma, double epsilon, double cutoff, int device, LbmMd** md) {
    if (!md)
        return LBM_ERR_INVALID_ARGUMENT;
    *md = nullptr;
    try {
        LbmMd* m = new LbmMd;
        try {
            m->impl = new lbm::MdEngine(n, masses, box, num_bonds, bonds, k, r0, pair_type, sigma, epsilon, cutoff, device);
        }
        catch (...) {
            delete m;
            throw;
        }
        *md = m;
        return LBM_OK;
    }
    catch (const lbm::Error& e) {
        lbm::setLastError(e.what());
        return e.status;
    }
}

void lbm_md_destroy(LbmMd* md) {
    if (md) {
        delete md->impl;
        delete md;
    }
}

LbmStatus lbm_md_compute_forces(LbmMd* md, const double* positions, double* forces, void* stream) {
    if (!md || !positions || !forces)
        return LBM_ERR_INVALID_ARGUMENT;
    try {
        md->impl->forces(positions, forces, (cudaStream_t) stream);
        return LBM_OK;
    }
    catch (const lbm::Error& e) {
        lbm::setLastError(e.what());
        return e.status;
    }
}

LbmStatus lbm_md_integrate(LbmMd* md, double dt, double* positions, double* velocities, const double* forces, void* stream) {
    if (!md || !positions || !velocities || !forces)
        return LBM_ERR_INVALID_ARGUMENT;
    int n = md->impl->view.n;
    lbm::leapfrogKernel<<<lbm::gridFor(3LL*n), 256, 0, (cudaStream_t) stream>>>(n, md->impl->invMass, dt, positions,
                                                                                 velocities, forces);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        lbm::setLastError(cudaGetErrorString(e));
        return LBM_ERR_CUDA;
    }
    md->impl->launches++;
    return LBM_OK;
}

LbmStatus lbm_md_kernel_launches(LbmMd* md, long long* launches) {
    if (!md || !launches)
        return LBM_ERR_INVALID_ARGUMENT;
    *launches = md->impl->launches;
    return LBM_OK;
}

LbmStatus lbm_md_kinetic(LbmMd* md, const double* velocities, double* twice_kinetic, void* stream) {
    if (!md || !velocities || !twice_kinetic)
        return LBM_ERR_INVALID_ARGUMENT;
    cudaStream_t s = (cudaStream_t) stream;
    lbm::kineticKernel<<<1, 1024, 0, s>>>(md->impl->view.n, md->impl->invMass, velocities, md->impl->scalar);
    cudaError_t e = cudaMemcpyAsync(twice_kinetic, md->impl->scalar, sizeof(double), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        lbm::setLastError(cudaGetErrorString(e));
        return LBM_ERR_CUDA;
    }
    return LBM_OK;
}

} // extern "C"
