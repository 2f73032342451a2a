// Allocation-free variant of the CFL wave-speed reduction.
//
// Some callers cannot let a library allocate device memory: a host code that
// carves all of its GPU memory out of one pool at start-up (as an MPI-era
// solver sizing its arrays once) cannot tolerate a cudaMalloc in its time
// loop, because cudaMalloc can fail once the pool owns the device and it
// synchronises the whole device when it succeeds. mc3d_cfl_max_noalloc gives
// them the per-step reduction without any allocation: the per-block partial
// maxima live in a file-scope device array, sized here once for every GPU
// that loads the library.
#include <cmath>
#include <mutex>

#include "mc3d_internal.h"

namespace {

constexpr int NA_BLOCK = 256;            // points per partial maximum
constexpr int NA_MAX_PARTIALS = 65536;   // -> at most 16,777,216 points (a 256^3 block)
constexpr int NA_MAX_DEVICES = 64;
constexpr double NA_GAMMA = 1.4;         // src/IdealGas.hpp:38

// Scratch of the reduction: one partial maximum per 256-point block. In host
// code this name is only a stand-in for the device symbol; the device address
// comes from cudaGetSymbolAddress below.
__device__ __align__(256) double g_cfl_partials[NA_MAX_PARTIALS];

std::mutex g_na_mu;
double *g_na_addr[NA_MAX_DEVICES] = {};

__device__ __forceinline__ double na_max(double a, double b) {
    // NaN wins, so a non-finite state shows in the result
    return (a > b || a != a) ? a : b;
}

__device__ __forceinline__ double na_block_max(double v, double *red) {
    for (int o = 16; o > 0; o >>= 1) v = na_max(v, __shfl_xor_sync(0xffffffffu, v, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x < 32) {
        v = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) v = na_max(v, __shfl_xor_sync(0xffffffffu, v, o));
    }
    return v;
}

// One block per 256 points: J11(|U|+c)/dxi + J22(|V|+c)/deta + J33(|W|+c)/dzeta,
// the wave-speed sum of calcDtFromCFL (src/CurvilinearCSolver_Core.cpp:196-198),
// maximised over the block into partials[blockIdx.x].
__global__ void __launch_bounds__(NA_BLOCK) na_cfl_partials(long long n, const double *__restrict__ r0,
                                                            const double *__restrict__ r1,
                                                            const double *__restrict__ r2,
                                                            const double *__restrict__ r3,
                                                            const double *__restrict__ r4, const double *J11,
                                                            const double *J22, const double *J33, double c11,
                                                            double c22, double c33, double i0, double i1, double i2,
                                                            double *partials) {
    __shared__ double red[NA_BLOCK / 32];
    long long i = (long long)blockIdx.x * NA_BLOCK + threadIdx.x;
    double v = 0.0;
    if (i < n) {
        double rho = r0[i];
        double u = r1[i] / rho, w1 = r2[i] / rho, w2 = r3[i] / rho;
        double p = (NA_GAMMA - 1) * (r4[i] - 0.5 * rho * (u * u + w1 * w1 + w2 * w2));
        double c = sqrt(NA_GAMMA * p / rho);
        double j11 = J11 ? J11[i] : c11, j22 = J22 ? J22[i] : c22, j33 = J33 ? J33[i] : c33;
        v = j11 * (fabs(u) + c) * i0 + j22 * (fabs(w1) + c) * i1 + j33 * (fabs(w2) + c) * i2;
        if (!isfinite(v)) v = __longlong_as_double(0x7ff8000000000000ll);
    }
    v = na_block_max(v, red);
    if (threadIdx.x == 0) partials[blockIdx.x] = v;
}

// One block: maximum of the first `count` partials into *out.
__global__ void __launch_bounds__(1024) na_cfl_final(const double *partials, int count, double *out) {
    __shared__ double red[32];
    double v = 0.0;
    for (int k = threadIdx.x; k < count; k += blockDim.x) v = na_max(v, partials[k]);
    v = na_block_max(v, red);
    if (threadIdx.x == 0) *out = v;
}

// Device address of the scratch array on the current device, looked up once
// per device with that device current. CUDA loads a library's modules and
// kernels on first use, and loading claims device memory (this file's module
// holds the 512 KiB array); so the first call here also loads both kernels,
// and every later call on the device neither loads nor allocates anything.
int na_scratch(double **out) {
    int dev = 0;
    MC3D_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= NA_MAX_DEVICES) return mc3d::fail(MC3D_ERR_ARG, "device index out of range");
    std::lock_guard<std::mutex> lock(g_na_mu);
    if (!g_na_addr[dev]) {
        double *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress((void **)&p, g_cfl_partials);
        if (e != cudaSuccess)
            return mc3d::fail(MC3D_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        cudaFuncAttributes fa;
        e = cudaFuncGetAttributes(&fa, na_cfl_partials);
        if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, na_cfl_final);
        if (e != cudaSuccess)
            return mc3d::fail(MC3D_ERR_CUDA, std::string("cudaFuncGetAttributes: ") + cudaGetErrorString(e));
        g_na_addr[dev] = p;
    }
    *out = g_na_addr[dev];
    return MC3D_OK;
}

}  // namespace

extern "C" int mc3d_cfl_max_noalloc(const double *rho, const double *rhoU, const double *rhoV, const double *rhoW,
                                    const double *rhoE, const double *J11, const double *J22, const double *J33,
                                    double J11c, double J22c, double J33c, int Nx, int Ny, int Nz, double dxi,
                                    double deta, double dzeta, double *out_max, void *stream) {
    if (!rho || !rhoU || !rhoV || !rhoW || !rhoE || !out_max) return mc3d::fail(MC3D_ERR_ARG, "null argument");
    if (Nx <= 0 || Ny <= 0 || Nz <= 0 || !(dxi > 0) || !(deta > 0) || !(dzeta > 0))
        return mc3d::fail(MC3D_ERR_ARG, "grid sizes and spacings must be positive");
    long long n = (long long)Nx * Ny * Nz;
    long long blocks = (n + NA_BLOCK - 1) / NA_BLOCK;
    if (blocks > NA_MAX_PARTIALS)
        return mc3d::fail(MC3D_ERR_ARG, "mc3d_cfl_max_noalloc: " + std::to_string(n) +
                                            " points exceed its fixed scratch limit of 16777216 points (256^3)");
    double *partials = nullptr;
    int rc = na_scratch(&partials);
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    na_cfl_partials<<<(unsigned)blocks, NA_BLOCK, 0, st>>>(n, rho, rhoU, rhoV, rhoW, rhoE, J11, J22, J33, J11c, J22c,
                                                          J33c, 1.0 / dxi, 1.0 / deta, 1.0 / dzeta, partials);
    MC3D_CUDA_TRY(cudaGetLastError());
    na_cfl_final<<<1, 1024, 0, st>>>(partials, (int)blocks, out_max);
    MC3D_CUDA_TRY(cudaGetLastError());
    return MC3D_OK;
}
