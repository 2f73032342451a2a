// Right-hand side of the TPB ("transformed periodic boundary") form of a
// periodic first derivative with ghost planes supplied by the caller:
// AbstractDerivatives::calc1stDerivField_TPB (src/AbstractDerivatives.hpp:45,
// :47), with the row arithmetic of Pade6::multRHS1stDerivPeriodic_TPB
// (src/Pade6.cpp:220-249), Penta10::multRHS1stDerivPeriodic_TPB
// (src/Penta10.cpp:175-207) and CD2::Compact1stPeriodic_TPB
// (src/CD2.cpp:144-151). The line solve that follows is the operator's own
// periodic solve with an identity right-hand-side stencil.
#include "mc3d_internal.h"

namespace mc3d {
namespace {

template <typename R>
__device__ __forceinline__ R mul_rn(R a, R b) {
    if constexpr (sizeof(R) == 8) return __dmul_rn(a, b);
    else return __fmul_rn(a, b);
}
template <typename R>
__device__ __forceinline__ R add_rn(R a, R b) {
    if constexpr (sizeof(R) == 8) return __dadd_rn(a, b);
    else return __fadd_rn(a, b);
}
template <typename R>
__device__ __forceinline__ R div_rn(R a, R b) {
    if constexpr (sizeof(R) == 8) return __ddiv_rn(a, b);
    else return __fdiv_rn(a, b);
}

// One thread per point. Ghost plane q of a point: the index of its line among
// the lines along dir, x fastest over the other two directions (dir 0:
// k Ny + j, dir 1: k Nx + i, dir 2: j Nx + i). Ghost m before the line
// (value at index -m) is planes[G - m], ghost m after it (index N - 1 + m) is
// planes[G + m - 1]. Every sum runs in stencil order, zero coefficients
// skipped, and is divided by dh, as the reference's rows are.
template <typename R>
__global__ void tpb_planes_rhs_kernel(Grid3 g, int dir, const R *__restrict__ f, TpbPlanes<R> gp, double dh,
                                      R *__restrict__ rhs) {
    const long long n_all = g.n();
    const long long stride = dir == 0 ? 1 : (dir == 1 ? (long long)g.Nx : (long long)g.Nx * g.Ny);
    const int N = dir == 0 ? g.Nx : (dir == 1 ? g.Ny : g.Nz);
    const int G = gp.G, H = gp.H;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n_all;
         p += (long long)gridDim.x * blockDim.x) {
        const long long i = p % g.Nx, j = (p / g.Nx) % g.Ny, k = p / ((long long)g.Nx * g.Ny);
        const int n = (int)(dir == 0 ? i : (dir == 1 ? j : k));
        const long long b = p - (long long)n * stride;
        const long long q = dir == 0 ? k * g.Ny + j : (dir == 1 ? k * g.Nx + i : j * g.Nx + i);
        auto F = [&](int idx) -> R {
            if (idx >= 0 && idx < N) return f[b + (long long)idx * stride];
            return idx < 0 ? gp.p[G + idx][q] : gp.p[G + idx - N][q];
        };
        R acc;
        if (gp.explicit_cd2) {
            // (a phi[i+1] + c phi[i-1]) / dd; row 0: a Nm1 + c phi[1]; row N-1: a phi[N-2] + c Np1
            const R ca = (R)gp.st[2], cc = (R)gp.st[0];
            if (n == 0) acc = add_rn(mul_rn(ca, F(-1)), mul_rn(cc, F(1)));
            else if (n == N - 1) acc = add_rn(mul_rn(ca, F(N - 2)), mul_rn(cc, F(N)));
            else acc = add_rn(mul_rn(ca, F(n + 1)), mul_rn(cc, F(n - 1)));
        } else {
            acc = R(0);
            bool first = true;
            for (int kk = 0; kk <= 2 * H; kk++) {
                if (gp.st[kk] == 0.0) continue;
                const R term = mul_rn((R)gp.st[kk], F(n + kk - H));
                acc = first ? term : add_rn(acc, term);
                first = false;
            }
        }
        rhs[p] = div_rn(acc, (R)dh);
    }
}

}  // namespace

template <typename R>
int launch_tpb_planes_rhs(const Grid3 &g, int dir, const R *f, const TpbPlanes<R> &gp, double dh, R *rhs,
                          cudaStream_t st) {
    const long long n = g.n();
    const int blocks = (int)std::min<long long>((n + 255) / 256, 148 * 16);
    tpb_planes_rhs_kernel<R><<<blocks, 256, 0, st>>>(g, dir, f, gp, dh, rhs);
    MC3D_CUDA_TRY(cudaGetLastError());
    return MC3D_OK;
}

template int launch_tpb_planes_rhs<float>(const Grid3 &, int, const float *, const TpbPlanes<float> &, double, float *,
                                          cudaStream_t);
template int launch_tpb_planes_rhs<double>(const Grid3 &, int, const double *, const TpbPlanes<double> &, double,
                                           double *, cudaStream_t);

}  // namespace mc3d
