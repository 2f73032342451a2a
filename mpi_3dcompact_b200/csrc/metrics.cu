// Grid metrics from mesh coordinates on the device, FP64:
// AbstractSingleBlockMesh::solveForJacobians (src/AbstractSingleBlockMesh.cpp:23-1308).
//
// Along periodic directions the reference differentiates with TPB operators
// (calc1stDerivField_TPB, src/Pade6.cpp:220-249, src/Penta10.cpp:175-207,
// src/CD2.cpp:144-150): the RHS stencil reads ghost values supplied by the
// caller, the line's wrapped values with the coordinates translated by the
// periodic displacement, and the periodic system is then solved as usual.
// tpb_rhs_kernel forms that RHS (ghosts built as the reference builds them:
// (X - T) W before a line's start, (X + T) W after its end); the solve is the
// solver's own line solve with an identity RHS stencil.
#include "mc3d_internal.h"

namespace mc3d {
namespace {

__device__ __forceinline__ long long line_base(const Grid3 &g, int dir, long long p, int &n) {
    // position n along dir of point p, and the index of the line's first point
    const long long i = p % g.Nx, j = (p / g.Nx) % g.Ny, k = p / ((long long)g.Nx * g.Ny);
    if (dir == 0) {
        n = (int)i;
        return p - i;
    }
    if (dir == 1) {
        n = (int)j;
        return p - j * g.Nx;
    }
    n = (int)k;
    return p - k * (long long)g.Nx * g.Ny;
}

__global__ void tpb_rhs_kernel(Grid3 g, int dir, const double *__restrict__ f, TpbArgs a, double *__restrict__ rhs) {
    const long long n_all = g.n();
    const long long stride = dir == 0 ? 1 : (dir == 1 ? (long long)g.Nx : (long long)g.Nx * g.Ny);
    const int N = a.N, H = a.H;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n_all;
         p += (long long)gridDim.x * blockDim.x) {
        int n;
        const long long b = line_base(g, dir, p, n);
        // line value at index idx in [-H, N+H): ghosts outside [0, N)
        auto F = [&](int idx) -> double {
            if (idx >= 0 && idx < N) return f[b + idx * stride];
            double sign;
            int w;
            if (idx < 0) {
                sign = -1.0;
                w = N + idx;                        // Nm_m at N - m
                if (a.nm3_from_nm2 && idx == -3) w = N - 2;
            } else {
                sign = 1.0;
                w = idx - N;                        // Np_m at m - 1
            }
            double v = 0.0;
            for (int t = 0; t < a.nterms; t++) {
                const double xt = __dadd_rn(a.X[t][b + w * stride], sign * a.T[t]);
                const double term = a.W[t] ? __dmul_rn(xt, a.W[t][b + w * stride]) : xt;
                v = t == 0 ? term : __dadd_rn(v, term);
            }
            return v;
        };
        double acc;
        if (a.explicit_cd2) {
            // (a phi[i+1] + c phi[i-1]) / h; row 0: a Nm1 + c phi[1]; row N-1: a phi[N-2] + c Np1
            const double ca = a.st[2], cc = a.st[0];
            if (n == 0)
                acc = __dadd_rn(__dmul_rn(ca, F(-1)), __dmul_rn(cc, F(1)));
            else if (n == N - 1)
                acc = __dadd_rn(__dmul_rn(ca, F(N - 2)), __dmul_rn(cc, F(N)));
            else
                acc = __dadd_rn(__dmul_rn(ca, F(n + 1)), __dmul_rn(cc, F(n - 1)));
        } else {
            acc = 0.0;
            bool first = true;
            for (int k = 0; k <= 2 * H; k++) {
                if (a.st[k] == 0.0) continue;
                const double term = __dmul_rn(a.st[k], F(n + k - H));
                acc = first ? term : __dadd_rn(acc, term);
                first = false;
            }
        }
        rhs[p] = __ddiv_rn(acc, a.dh);
    }
}

__global__ void mul_kernel(long long n, const double *__restrict__ a, const double *__restrict__ b,
                           double *__restrict__ o) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        o[i] = __dmul_rn(a[i], b[i]);
}

__global__ void sub_kernel(long long n, const double *__restrict__ a, const double *__restrict__ b,
                           double *__restrict__ o) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        o[i] = __dsub_rn(a[i], b[i]);
}

// x J_i1 + y J_i2 + z J_i3 (src/AbstractSingleBlockMesh.cpp:1069-1073), left to right
__global__ void dot3_kernel(long long n, const double *__restrict__ x, const double *__restrict__ y,
                            const double *__restrict__ z, const double *__restrict__ a, const double *__restrict__ b,
                            const double *__restrict__ c, double *__restrict__ o) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        o[i] = __dadd_rn(__dadd_rn(__dmul_rn(x[i], a[i]), __dmul_rn(y[i], b[i])), __dmul_rn(z[i], c[i]));
}

// J = 1 / ((1/3)(Jdet1 + Jdet2 + Jdet3)), J_ij *= J (src/AbstractSingleBlockMesh.cpp:1298-1308)
__global__ void jac_finish_kernel(long long n, const double *__restrict__ d1, const double *__restrict__ d2,
                                  const double *__restrict__ d3, MetOut9 m, double *__restrict__ J) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const double j = __drcp_rn(__dmul_rn(1.0 / 3.0, __dadd_rn(__dadd_rn(d1[i], d2[i]), d3[i])));
        J[i] = j;
        for (int c = 0; c < 9; c++) m.p[c][i] = __dmul_rn(j, m.p[c][i]);
    }
}

int blocks_for(long long n) { return (int)std::min<long long>((n + 255) / 256, 148 * 16); }

}  // namespace

int launch_tpb_rhs(const Grid3 &g, int dir, const double *f, const TpbArgs &a, double *rhs, cudaStream_t st) {
    if (a.H < 1 || a.H > 3 || a.nterms < 1 || a.nterms > 3 || a.N <= 2 * a.H) return MC3D_ERR_ARG;
    for (int t = 0; t < a.nterms; t++)
        if (!a.X[t]) return MC3D_ERR_ARG;
    tpb_rhs_kernel<<<blocks_for(g.n()), 256, 0, st>>>(g, dir, f, a, rhs);
    MC3D_CUDA_TRY(cudaGetLastError());
    return MC3D_OK;
}

int launch_metric_mul(long long n, const double *a, const double *b, double *o, cudaStream_t st) {
    mul_kernel<<<blocks_for(n), 256, 0, st>>>(n, a, b, o);
    MC3D_CUDA_TRY(cudaGetLastError());
    return MC3D_OK;
}

int launch_metric_sub(long long n, const double *a, const double *b, double *o, cudaStream_t st) {
    sub_kernel<<<blocks_for(n), 256, 0, st>>>(n, a, b, o);
    MC3D_CUDA_TRY(cudaGetLastError());
    return MC3D_OK;
}

int launch_metric_dot3(long long n, const double *const xyz[3], const double *const abc[3], double *o,
                       cudaStream_t st) {
    dot3_kernel<<<blocks_for(n), 256, 0, st>>>(n, xyz[0], xyz[1], xyz[2], abc[0], abc[1], abc[2], o);
    MC3D_CUDA_TRY(cudaGetLastError());
    return MC3D_OK;
}

int launch_metric_finish(long long n, const double *const jdet[3], double *const jij[9], double *J, cudaStream_t st) {
    MetOut9 m;
    for (int c = 0; c < 9; c++) m.p[c] = jij[c];
    jac_finish_kernel<<<blocks_for(n), 256, 0, st>>>(n, jdet[0], jdet[1], jdet[2], m, J);
    MC3D_CUDA_TRY(cudaGetLastError());
    return MC3D_OK;
}

}  // namespace mc3d
