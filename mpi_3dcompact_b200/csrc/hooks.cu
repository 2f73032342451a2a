// Device reductions behind the reference drivers' diagnostic hooks:
//   HIT turbulence statistics, one line of turbdata.out
//     (tests/hit/Samtaney_D4/MPI_3DCompact.cpp:370-555, fullStepTemporalHook);
//   span-averaged wall values of the cylinder (src/MPI_3DCompact.cpp:408-485)
//   and its wake strip, V along xi3 at one (xi1, xi2) point (:488-527).
#include "mc3d_internal.h"
#include "pointwise_common.cuh"

namespace mc3d {
namespace {

constexpr int HB = 256;   // threads per block of the reductions

__device__ __forceinline__ void block_sums(double *v, int nv, double *partial, int stride) {
    __shared__ double red[HB / 32][TURB_NSUM];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int k = 0; k < nv; k++) {
        double s = v[k];
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) red[w][k] = s;
    }
    __syncthreads();
    if (threadIdx.x < nv) {
        double t = 0;
        for (int q = 0; q < HB / 32; q++) t += red[q][threadIdx.x];
        partial[threadIdx.x * stride + blockIdx.x] = t;
    }
}

// Per point (tests/hit/Samtaney_D4/MPI_3DCompact.cpp:408-458): Cartesian
// velocity gradients from the xi-derivatives d[3*var + dir] and the metrics,
// dilatation, vorticity, turbulent dissipation 2 mu S^d_ij du_i/dx_j, and the
// sums of pass 1: rho, mu, dissipation, |u|^2/3, (dudx^2 + dvdy^2 + dwdz^2)/3,
// |u|^2, c, dudx^2, rho |u|^2; pass 2 (means known): (rho - mean)^2, dil^2,
// |omega|^2.
template <typename R>
__global__ void __launch_bounds__(HB) turb_kernel(Grid3 g, P5c<R> pr, DerivPtrs12c<R> dp, Metrics<R> m, double mu_ref,
                                                  int pass, double mean_rho, double *partial) {
    double acc[TURB_NSUM];
    for (int k = 0; k < TURB_NSUM; k++) acc[k] = 0.0;
    const long long n = g.n();
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const double rho = pr.p[0][i], U = pr.p[1][i], V = pr.p[2][i], W = pr.p[3][i], T = pr.p[4][i];
        double gu[3][3];   // gu[a][b] = d u_a / d x_b
        for (int a = 0; a < 3; a++) {
            const double d1 = dp.p[3 * a][i], d2 = dp.p[3 * a + 1][i], d3 = dp.p[3 * a + 2][i];
            for (int b = 0; b < 3; b++)
                gu[a][b] = (double)met(m, 1 + b, i) * d1 + (double)met(m, 4 + b, i) * d2 + (double)met(m, 7 + b, i) * d3;
        }
        const double dil = gu[0][0] + gu[1][1] + gu[2][2];
        if (pass == 1) {
            const double mu = mu_ref * pow(T, 0.76);
            const double p = rho * R_GAS * T;
            double diss = 0.0;
            for (int a = 0; a < 3; a++)
                for (int b = 0; b < 3; b++) {
                    const double s = 0.5 * (gu[a][b] + gu[b][a]) - (a == b ? (1.0 / 3.0) * dil : 0.0);
                    diss += s * gu[a][b];
                }
            diss *= 2 * mu;
            const double uvar = U * U + V * V + W * W;
            acc[0] += rho;
            acc[1] += mu;
            acc[2] += diss;
            acc[3] += uvar / 3.0;
            acc[4] += (gu[0][0] * gu[0][0] + gu[1][1] * gu[1][1] + gu[2][2] * gu[2][2]) / 3.0;
            acc[5] += uvar;
            acc[6] += sqrt(GAMMA * p / rho);
            acc[7] += gu[0][0] * gu[0][0];
            acc[8] += rho * uvar;
        } else {
            const double wx = gu[2][1] - gu[1][2], wy = gu[0][2] - gu[2][0], wz = gu[1][0] - gu[0][1];
            acc[0] += (rho - mean_rho) * (rho - mean_rho);
            acc[1] += dil * dil;
            acc[2] += wx * wx + wy * wy + wz * wz;
        }
    }
    block_sums(acc, pass == 1 ? 9 : 3, partial, gridDim.x);
}

// Span average over xi3 of p, U, V, W on the j = 0 face, summed as x/Nz in k
// order (src/MPI_3DCompact.cpp:449-461); primitives from the FP64 state.
__global__ void wall_span_kernel(Grid3 g, Q5c q, double *out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < g.Nx; i += gridDim.x * blockDim.x) {
        double ap = 0, au = 0, av = 0, aw = 0;
        const double nz = (double)g.Nz;
        for (int k = 0; k < g.Nz; k++) {
            const long long p = i + (long long)g.Nx * g.Ny * k;
            const double rho = q.p[0][p];
            const double U = q.p[1][p] / rho, V = q.p[2][p] / rho, W = q.p[3][p] / rho;
            const double pr = (GAMMA - 1) * (q.p[4][p] - 0.5 * rho * (U * U + V * V + W * W));
            ap += pr / nz;
            au += U / nz;
            av += V / nz;
            aw += W / nz;
        }
        out[i] = ap;
        out[g.Nx + i] = au;
        out[2 * g.Nx + i] = av;
        out[3 * g.Nx + i] = aw;
    }
}

// V = rhoV / rho along xi3 at (i, j) (src/MPI_3DCompact.cpp:491-507)
__global__ void wake_strip_kernel(Grid3 g, Q5c q, int i, int j, double *out) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < g.Nz; k += gridDim.x * blockDim.x) {
        const long long p = i + (long long)g.Nx * (j + (long long)g.Ny * k);
        out[k] = q.p[2][p] / q.p[0][p];
    }
}

}  // namespace

template <typename R>
int launch_turb_sums(const Grid3 &g, const R *const prim[5], const R *const d[12], const Metrics<R> &m,
                     double mu_ref, int pass, double mean_rho, double *partial, int nblocks, cudaStream_t st) {
    P5c<R> P;
    DerivPtrs12c<R> D;
    for (int v = 0; v < 5; v++) P.p[v] = prim[v];
    for (int k = 0; k < 12; k++) D.p[k] = d[k];
    turb_kernel<R><<<nblocks, HB, 0, st>>>(g, P, D, m, mu_ref, pass, mean_rho, partial);
    MC3D_CUDA_TRY(cudaGetLastError());
    return MC3D_OK;
}
template int launch_turb_sums<float>(const Grid3 &, const float *const[5], const float *const[12],
                                     const Metrics<float> &, double, int, double, double *, int, cudaStream_t);
template int launch_turb_sums<double>(const Grid3 &, const double *const[5], const double *const[12],
                                      const Metrics<double> &, double, int, double, double *, int, cudaStream_t);

int launch_wall_span_average(const Grid3 &g, const double *const q[5], double *out, cudaStream_t st) {
    Q5c qq;
    for (int v = 0; v < 5; v++) qq.p[v] = q[v];
    wall_span_kernel<<<(g.Nx + 127) / 128, 128, 0, st>>>(g, qq, out);
    MC3D_CUDA_TRY(cudaGetLastError());
    return MC3D_OK;
}

int launch_wake_strip(const Grid3 &g, const double *const q[5], int i, int j, double *out, cudaStream_t st) {
    Q5c qq;
    for (int v = 0; v < 5; v++) qq.p[v] = q[v];
    wake_strip_kernel<<<(g.Nz + 127) / 128, 128, 0, st>>>(g, qq, i, j, out);
    MC3D_CUDA_TRY(cudaGetLastError());
    return MC3D_OK;
}

}  // namespace mc3d
