// Pointwise kernels of the time step: primitives, the fused velocity-gradient /
// stress / heat-flux / contravariant-flux evaluation (with the Vreman closure
// inline), the RK register updates, the CFL reduction and the dt bookkeeping.
// Grid-stride loops over x-fastest fields; one thread per point per iteration.
#include <cmath>

#include "pointwise_common.cuh"

namespace mc3d {

__device__ __forceinline__ float mu_of_T(float T, double mu_ref) { return (float)mu_ref * powf(T, 0.76f); }
__device__ __forceinline__ double mu_of_T(double T, double mu_ref) { return mu_ref * pow(T, 0.76); }

// ---- primitives U, V, W, T (updateNonConservedData, Core.cpp:1158-1197) ----
// rho, U, V, W, T of one point from the FP64 conserved state (solveU, solvep,
// solveT of src/IdealGas.hpp:56-70)
template <typename R>
__device__ __forceinline__ void prims_of(double rho, double ru, double rv, double rw, double re, R *const *P,
                                         long long i) {
    double u = ru / rho, v = rv / rho, w = rw / rho;
    double p = (GAMMA - 1) * (re - 0.5 * rho * (u * u + v * v + w * w));
    P[0][i] = (R)rho;
    P[1][i] = (R)u;
    P[2][i] = (R)v;
    P[3][i] = (R)w;
    P[4][i] = (R)(p / (rho * R_GAS));
}

template <typename R>
struct P5 {
    R *p[5];
};

template <typename R>
__global__ void primitives_kernel(Grid3 g, const double *__restrict__ r0, const double *__restrict__ r1,
                                  const double *__restrict__ r2, const double *__restrict__ r3,
                                  const double *__restrict__ r4, P5<R> P) {
    long long n = g.n();
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        prims_of<R>(r0[i], r1[i], r2[i], r3[i], r4[i], P.p, i);
}

// Primitives of the stage-1 state together with the CFL wave-speed maximum of
// calcDtFromCFL (src/CurvilinearCSolver_Core.cpp:189-212), which reads the same
// state: max over points of J11 (|U| + c)/dxi + J22 (|V| + c)/deta + J33 (|W| + c)/dzeta.
template <typename R>
__global__ void primitives_cfl_kernel(Grid3 g, const double *__restrict__ r0, const double *__restrict__ r1,
                                      const double *__restrict__ r2, const double *__restrict__ r3,
                                      const double *__restrict__ r4, P5<R> P, Metrics<R> m, double i0, double i1,
                                      double i2, unsigned long long *umax) {
    __shared__ double red[32];
    double best = 0.0;
    bool bad = false;
    const long long n = g.n();
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const double rho = r0[i], q1 = r1[i], q2 = r2[i], q3 = r3[i], q4 = r4[i];
        prims_of<R>(rho, q1, q2, q3, q4, P.p, i);
        const double u = q1 / rho, v = q2 / rho, w = q3 / rho;
        const double p = (GAMMA - 1) * (q4 - 0.5 * rho * (u * u + v * v + w * w));
        const double c = sqrt(GAMMA * p / rho);
        const double uc = (double)met(m, 1, i) * (fabs(u) + c) * i0 + (double)met(m, 5, i) * (fabs(v) + c) * i1 +
                          (double)met(m, 9, i) * (fabs(w) + c) * i2;
        if (!isfinite(uc)) bad = true;
        else if (uc > best) best = uc;
    }
    for (int o = 16; o > 0; o >>= 1) best = fmax(best, __shfl_xor_sync(0xffffffffu, best, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = best;
    __syncthreads();
    if (threadIdx.x < 32) {
        double b = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) b = fmax(b, __shfl_xor_sync(0xffffffffu, b, o));
        if (threadIdx.x == 0) atomicMax(umax, (unsigned long long)__double_as_longlong(b));
    }
    // a non-finite state poisons the maximum: dt becomes NaN and the host check reports it
    if (bad) atomicMax(umax, 0x7ff8000000000000ull);
}

template <typename R>
int launch_primitives_cfl(const Grid3 &g, const double *const q[5], R *const prim[5], const Metrics<R> &m,
                          const double dxi[3], unsigned long long *umax, cudaStream_t st) {
    P5<R> P;
    for (int v = 0; v < 5; v++) P.p[v] = prim[v];
    primitives_cfl_kernel<R><<<grid_for(g.n(), 256), 256, 0, st>>>(g, q[0], q[1], q[2], q[3], q[4], P, m,
                                                                   1.0 / dxi[0], 1.0 / dxi[1], 1.0 / dxi[2], umax);
    MC3D_CUDA_TRY(cudaGetLastError());
    return MC3D_OK;
}
template int launch_primitives_cfl<float>(const Grid3 &, const double *const[5], float *const[5],
                                          const Metrics<float> &, const double[3], unsigned long long *, cudaStream_t);
template int launch_primitives_cfl<double>(const Grid3 &, const double *const[5], double *const[5],
                                           const Metrics<double> &, const double[3], unsigned long long *,
                                           cudaStream_t);

template <typename R>
int launch_primitives(const Grid3 &g, const double *const q[5], R *const prim[5], cudaStream_t st) {
    P5<R> P;
    for (int v = 0; v < 5; v++) P.p[v] = prim[v];
    primitives_kernel<R><<<grid_for(g.n(), 256), 256, 0, st>>>(g, q[0], q[1], q[2], q[3], q[4], P);
    MC3D_CUDA_TRY(cudaGetLastError());
    return MC3D_OK;
}

// ---- Vreman eddy viscosity (src/VremanSGS.hpp:43-96) ----
template <typename R>
__device__ __forceinline__ R vreman_mu(const R gu[3][3], R rho, R d1) {
    R d1v1 = gu[0][0], d2v1 = gu[0][1], d3v1 = gu[0][2];
    R d1v2 = gu[1][0], d2v2 = gu[1][1], d3v2 = gu[1][2];
    R d1v3 = gu[2][0], d2v3 = gu[2][1], d3v3 = gu[2][2];
    R b11 = d1 * d1v1 * d1v1 + d1 * d2v1 * d2v1 + d1 * d3v1 * d3v1;
    R b12 = d1 * d1v1 * d1v2 + d1 * d2v1 * d2v2 + d1 * d3v1 * d3v2;
    R b13 = d1 * d1v1 * d1v3 + d1 * d2v1 * d2v3 + d1 * d3v1 * d3v3;
    R b22 = d1 * d1v2 * d1v2 + d1 * d2v2 * d2v2 + d1 * d3v2 * d3v2;
    R b23 = d1 * d1v2 * d1v3 + d1 * d2v2 * d2v3 + d1 * d3v2 * d3v3;
    R b33 = d1 * d1v3 * d1v3 + d1 * d2v3 * d2v3 + d1 * d3v3 * d3v3;
    // the reference sums d2v3^2 twice and omits d3v2^2 (VremanSGS.hpp:74-76)
    R abeta = d1v1 * d1v1 + d1v2 * d1v2 + d1v3 * d1v3 + d2v1 * d2v1 + d2v2 * d2v2 + d2v3 * d2v3 + d3v1 * d3v1 +
              d2v3 * d2v3 + d3v3 * d3v3;
    R bbeta = b11 * b22 - (b12 * b12) + b11 * b33 - (b13 * b13) + b22 * b33 - (b23 * b23);
    const R eps = (R)1e-12;
    if (bbeta < eps) bbeta = eps;
    R ss = sqrt(bbeta / (abeta + eps));
    const R c = (R)(2.5 * 0.17 * 0.17);
    R mu = c * rho * ss;
    R cap = (R)0.05 * d1 * sqrt((R)2.0 * abeta);
    return mu < cap ? mu : cap;
}

// Filter width squared d1 = (dxi deta dzeta / J)^(2/3) of VremanSGS.hpp:49-52.
template <typename R>
__device__ __forceinline__ R vreman_d1(double dvol, R J) {
    double del = pow(dvol / (double)J, 1.0 / 3.0);
    return (R)(del * del);
}

template <typename R>
__device__ __forceinline__ void velocity_gradient(const Metrics<R> &m, long long i, const R *const *d, R gu[3][3]) {
    // gradU[a][b] = J1b dUa1 + J2b dUa2 + J3b dUa3  (Core.cpp:548-561)
#pragma unroll
    for (int a = 0; a < 3; a++) {
        R d1 = d[3 * a][i], d2 = d[3 * a + 1][i], d3 = d[3 * a + 2][i];
#pragma unroll
        for (int b = 0; b < 3; b++) gu[a][b] = met(m, 1 + b, i) * d1 + met(m, 4 + b, i) * d2 + met(m, 7 + b, i) * d3;
    }
}

struct DerivPtrs12 {
    const void *p[12];
};
struct OutPtrs15 {
    void *p[15];
};

// Paired access to two consecutive points: one 8/16-byte load or store.
template <typename T>
struct Pair;
template <>
struct Pair<float> {
    using V = float2;
};
template <>
struct Pair<double> {
    using V = double2;
};
template <typename T>
__device__ __forceinline__ void ld_pair(const T *p, long long i, bool two, double (&o)[2]) {
    if (two) {
        typename Pair<T>::V v = *reinterpret_cast<const typename Pair<T>::V *>(p + i);
        o[0] = (double)v.x;
        o[1] = (double)v.y;
    } else {
        o[0] = (double)p[i];
        o[1] = 0.0;
    }
}
template <typename T>
__device__ __forceinline__ void st_pair(T *p, long long i, bool two, double x0, double x1) {
    if (two) {
        typename Pair<T>::V v;
        v.x = (T)x0;
        v.y = (T)x1;
        *reinterpret_cast<typename Pair<T>::V *>(p + i) = v;
    } else {
        p[i] = (T)x0;
    }
}

template <typename T, int NP>
__device__ __forceinline__ void ld_np(const T *p, long long i, bool two, T (&o)[NP]) {
    if (NP == 2 && two) {
        typename Pair<T>::V v = *reinterpret_cast<const typename Pair<T>::V *>(p + i);
        o[0] = v.x;
        o[NP - 1] = v.y;
    } else {
#pragma unroll
        for (int k = 0; k < NP; k++) o[k] = k == 0 ? p[i] : T(0);
    }
}
template <typename T, int NP>
__device__ __forceinline__ void st_np(T *p, long long i, bool two, const T (&x)[NP]) {
    if (NP == 2 && two) {
        typename Pair<T>::V v;
        v.x = x[0];
        v.y = x[NP - 1];
        *reinterpret_cast<typename Pair<T>::V *>(p + i) = v;
    } else {
        p[i] = x[0];
    }
}

// ---- fluxes: preStepDerivatives, Core.cpp:615-752 ----
// Metric forms: per-point fields, ten constants, or constants with zero
// off-diagonal J_ab (rectilinear box). The diagonal form leaves out the terms
// that multiply a zero metric, which changes no finite result.
enum MetForm { MET_FIELD = 0, MET_CONST = 1, MET_DIAG = 2 };

template <typename R, int MET>
__device__ __forceinline__ void flux_point(R rho, R U, R V, R W, R T, R Tm, const R (&dd)[12], const R (&mj)[10],
                                           R msgs, R ksgs, R tk, const Metrics<R> &m, const FluxParams &fp, R d1c,
                                           R iJc, double dvol, R (&o)[15], const double *qc = nullptr) {
    constexpr bool DIAG = MET == MET_DIAG;
    const R J = MET == MET_FIELD ? mj[0] : m.c[0];
    const R J11 = MET == MET_FIELD ? mj[1] : m.c[1], J12 = MET == MET_FIELD ? mj[2] : m.c[2],
            J13 = MET == MET_FIELD ? mj[3] : m.c[3];
    const R J21 = MET == MET_FIELD ? mj[4] : m.c[4], J22 = MET == MET_FIELD ? mj[5] : m.c[5],
            J23 = MET == MET_FIELD ? mj[6] : m.c[6];
    const R J31 = MET == MET_FIELD ? mj[7] : m.c[7], J32 = MET == MET_FIELD ? mj[8] : m.c[8],
            J33 = MET == MET_FIELD ? mj[9] : m.c[9];
    // p and rhoE from the ideal-gas relations (src/IdealGas.hpp:64-78)
    R p = rho * (R)R_GAS * T;
    R rhoU = rho * U, rhoV = rho * V, rhoW = rho * W;
    // with DSM, p (and T, mu) carry -tau_kk / 2 but rhoE is the state's (Core.cpp:573-584)
    R rhoE = (fp.les == 3 ? p + (R)0.5 * tk : p) / (R)(GAMMA - 1.0) + (R)0.5 * rho * (U * U + V * V + W * W);
    if (qc) {
        // the conserved state where it no longer matches the primitives; with
        // DSM T there is the temperature of p - tau_kk/2 at the conserved rho
        rho = (R)qc[0];
        if (fp.les == 3) p = rho * (R)R_GAS * T;
        rhoU = (R)qc[1];
        rhoV = (R)qc[2];
        rhoW = (R)qc[3];
        rhoE = (R)qc[4];
    }
    R mu = mu_of_T(Tm, fp.mu_ref);
    R Ucurv = DIAG ? J11 * U : J11 * U + J12 * V + J13 * W;
    R Vcurv = DIAG ? J22 * V : J21 * U + J22 * V + J23 * W;
    R Wcurv = DIAG ? J33 * W : J31 * U + J32 * V + J33 * W;

    // gradU[a][b] = J1b dUa1 + J2b dUa2 + J3b dUa3  (Core.cpp:548-561)
    R gu[3][3];
#pragma unroll
    for (int a = 0; a < 3; a++) {
        R d1 = dd[3 * a], d2 = dd[3 * a + 1], d3 = dd[3 * a + 2];
        gu[a][0] = DIAG ? J11 * d1 : J11 * d1 + J21 * d2 + J31 * d3;
        gu[a][1] = DIAG ? J22 * d2 : J12 * d1 + J22 * d2 + J32 * d3;
        gu[a][2] = DIAG ? J33 * d3 : J13 * d1 + J23 * d2 + J33 * d3;
    }

    R mu_eff, k_eff;
    if (fp.les) {
        R mu_sgs;
        if (fp.les == 1) mu_sgs = vreman_mu<R>(gu, rho, MET != MET_FIELD ? d1c : vreman_d1<R>(dvol, J));
        else mu_sgs = msgs;
        mu_eff = mu + mu_sgs;
        if (fp.les == 3) k_eff = (R)CP * mu / (R)PR + ksgs;   // Core.cpp:636-639
        else k_eff = (R)CP * (mu / (R)PR + mu_sgs / (R)fp.pr_t);
        if (mu_eff < (R)0) mu_eff = 0;
        if (k_eff < (R)0) k_eff = 0;
    } else {
        mu_eff = mu;
        k_eff = (R)(CP / PR) * mu;
    }
    R dUdx = gu[0][0], dUdy = gu[0][1], dUdz = gu[0][2];
    R dVdx = gu[1][0], dVdy = gu[1][1], dVdz = gu[1][2];
    R dWdx = gu[2][0], dWdy = gu[2][1], dWdz = gu[2][2];
    const R c43 = (R)(4.0 / 3.0), c23 = (R)(2.0 / 3.0);
    R t11 = (c43 * dUdx - c23 * dVdy - c23 * dWdz) * mu_eff;
    R t22 = (-c23 * dUdx + c43 * dVdy - c23 * dWdz) * mu_eff;
    R t33 = (-c23 * dUdx - c23 * dVdy + c43 * dWdz) * mu_eff;
    R t12 = (dUdy + dVdx) * mu_eff;
    R t13 = (dUdz + dWdx) * mu_eff;
    R t23 = (dVdz + dWdy) * mu_eff;
    const R t21 = t12, t31 = t13, t32 = t23;

    R dT1 = dd[9], dT2 = dd[10], dT3 = dd[11];
    R q1 = k_eff * (DIAG ? J11 * dT1 : J11 * dT1 + J21 * dT2 + J31 * dT3);
    R q2 = k_eff * (DIAG ? J22 * dT2 : J12 * dT1 + J22 * dT2 + J32 * dT3);
    R q3 = k_eff * (DIAG ? J33 * dT3 : J13 * dT1 + J23 * dT2 + J33 * dT3);
    R b1 = U * t11 + V * t12 + W * t13 + q1;
    R b2 = U * t21 + V * t22 + W * t23 + q2;
    R b3 = U * t31 + V * t32 + W * t33 + q3;

    R iJ = MET != MET_FIELD ? iJc : (R)1 / J;
    o[0] = iJ * (rho * Ucurv);
    o[5] = iJ * (rho * Vcurv);
    o[10] = iJ * (rho * Wcurv);

    R f1, f2, f3, g1, g2, g3;
    f1 = rhoU * Ucurv + J11 * p;
    f2 = DIAG ? rhoU * Vcurv : rhoU * Vcurv + J21 * p;
    f3 = DIAG ? rhoU * Wcurv : rhoU * Wcurv + J31 * p;
    g1 = DIAG ? J11 * t11 : J11 * t11 + J12 * t21 + J13 * t31;
    g2 = DIAG ? J22 * t21 : J21 * t11 + J22 * t21 + J23 * t31;
    g3 = DIAG ? J33 * t31 : J31 * t11 + J32 * t21 + J33 * t31;
    o[1] = iJ * (f1 - g1);
    o[6] = iJ * (f2 - g2);
    o[11] = iJ * (f3 - g3);

    f1 = DIAG ? rhoV * Ucurv : rhoV * Ucurv + J12 * p;
    f2 = rhoV * Vcurv + J22 * p;
    f3 = DIAG ? rhoV * Wcurv : rhoV * Wcurv + J32 * p;
    g1 = DIAG ? J11 * t12 : J11 * t12 + J12 * t22 + J13 * t32;
    g2 = DIAG ? J22 * t22 : J21 * t12 + J22 * t22 + J23 * t32;
    g3 = DIAG ? J33 * t32 : J31 * t12 + J32 * t22 + J33 * t32;
    o[2] = iJ * (f1 - g1);
    o[7] = iJ * (f2 - g2);
    o[12] = iJ * (f3 - g3);

    f1 = DIAG ? rhoW * Ucurv : rhoW * Ucurv + J13 * p;
    f2 = DIAG ? rhoW * Vcurv : rhoW * Vcurv + J23 * p;
    f3 = rhoW * Wcurv + J33 * p;
    g1 = DIAG ? J11 * t13 : J11 * t13 + J12 * t23 + J13 * t33;
    g2 = DIAG ? J22 * t23 : J21 * t13 + J22 * t23 + J23 * t33;
    g3 = DIAG ? J33 * t33 : J31 * t13 + J32 * t23 + J33 * t33;
    o[3] = iJ * (f1 - g1);
    o[8] = iJ * (f2 - g2);
    o[13] = iJ * (f3 - g3);

    R ep = rhoE + p;
    f1 = ep * Ucurv;
    f2 = ep * Vcurv;
    f3 = ep * Wcurv;
    g1 = DIAG ? J11 * b1 : J11 * b1 + J12 * b2 + J13 * b3;
    g2 = DIAG ? J22 * b2 : J21 * b1 + J22 * b2 + J23 * b3;
    g3 = DIAG ? J33 * b3 : J31 * b1 + J32 * b2 + J33 * b3;
    o[4] = iJ * (f1 - g1);
    o[9] = iJ * (f2 - g2);
    o[14] = iJ * (f3 - g3);
}

// NP consecutive points per thread (2 in FP32: paired 8-byte accesses), all
// inputs of the iteration loaded before its 15 stores. WALL: mu on wall points
// from Tmu, and the conserved state on the faces of fp.cons_mask.
template <typename R, int MET, int NP, bool WALL>
__global__ void __launch_bounds__(256, 2) flux_kernel(Grid3 g, const R *__restrict__ r0, const R *__restrict__ r1,
                                                      const R *__restrict__ r2, const R *__restrict__ r3,
                                                      const R *__restrict__ r4, DerivPtrs12 dp, Metrics<R> m,
                                                      FluxParams fp, const R *__restrict__ mu_sgs_f,
                                                      const R *__restrict__ ksgs_f, const R *__restrict__ taukk_f,
                                                      const R *__restrict__ Tmu, OutPtrs15 op) {
    const R *const *d = reinterpret_cast<const R *const *>(dp.p);
    R *const *F = reinterpret_cast<R *const *>(op.p);
    const double dvol = fp.dxi[0] * fp.dxi[1] * fp.dxi[2];
    const R d1c = MET != MET_FIELD ? vreman_d1<R>(dvol, m.c[0]) : R(0);   // filter width of a uniform block
    const R iJc = MET != MET_FIELD ? (R)1 / m.c[0] : R(0);
    const long long n = g.n(), nit = (n + NP - 1) / NP;
    for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < nit; j += (long long)gridDim.x * blockDim.x) {
        const long long i = NP * j;
        const bool two = i + 1 < n;
        R rho[NP], U[NP], V[NP], Wv[NP], T[NP], dd[12][NP], mj[10][NP], ms[NP], ks[NP], tk[NP];
        ld_np<R, NP>(r0, i, two, rho);
        ld_np<R, NP>(r1, i, two, U);
        ld_np<R, NP>(r2, i, two, V);
        ld_np<R, NP>(r3, i, two, Wv);
        ld_np<R, NP>(r4, i, two, T);
#pragma unroll
        for (int k = 0; k < 12; k++) ld_np<R, NP>(d[k], i, two, dd[k]);
        if (MET == MET_FIELD) {
#pragma unroll
            for (int c = 0; c < 10; c++) ld_np<R, NP>(m.m[c], i, two, mj[c]);
        }
        if (fp.les >= 2) ld_np<R, NP>(mu_sgs_f, i, two, ms);
        if (fp.les == 3) {
            ld_np<R, NP>(ksgs_f, i, two, ks);
            if (taukk_f) {
                ld_np<R, NP>(taukk_f, i, two, tk);
            } else {
#pragma unroll
                for (int q = 0; q < NP; q++) tk[q] = R(0);
            }
        }
        R out[15][NP];
#pragma unroll
        for (int q = 0; q < NP; q++) {
            R dq[12], mq[10], oq[15];
#pragma unroll
            for (int k = 0; k < 12; k++) dq[k] = dd[k][q];
#pragma unroll
            for (int c = 0; c < 10; c++) mq[c] = MET == MET_FIELD ? mj[c][q] : R(0);
            // (q == 1 without `two` is the padding point past the grid's end)
            const bool real = NP == 1 || two || q == 0;
            R Tm = T[q];
            if (WALL && fp.les != 3 && real && on_faces(g, i + q, fp.wall_mask)) Tm = Tmu[i + q];
            double qc[5];
            const bool cons = WALL && fp.cons_mask && real && on_faces(g, i + q, fp.cons_mask);
            if (cons)
                for (int v = 0; v < 5; v++) qc[v] = fp.cons[v][i + q];
            flux_point<R, MET>(rho[q], U[q], V[q], Wv[q], T[q], Tm, dq, mq, fp.les >= 2 ? ms[q] : R(0),
                               fp.les == 3 ? ks[q] : R(0), fp.les == 3 ? tk[q] : R(0), m, fp, d1c, iJc, dvol, oq,
                               cons ? qc : nullptr);
#pragma unroll
            for (int k = 0; k < 15; k++) out[k][q] = oq[k];
        }
#pragma unroll
        for (int k = 0; k < 15; k++) st_np<R, NP>(F[k], i, two, out[k]);
    }
}

template <typename R>
int launch_flux(const Grid3 &g, const R *const q[5], const R *const d[12], const Metrics<R> &m,
                const FluxParams &p, const R *mu_sgs, const R *k_sgs, const R *taukk, const R *Tmu, R *const F[15],
                cudaStream_t st) {
    DerivPtrs12 dp;
    for (int i = 0; i < 12; i++) dp.p[i] = d[i];
    OutPtrs15 op;
    for (int i = 0; i < 15; i++) op.p[i] = F[i];
    constexpr int NP = sizeof(R) == 4 ? 2 : 1;
    const int grid = grid_for((g.n() + NP - 1) / NP, 256);
    bool diag = m.constant;
    for (int c : {2, 3, 4, 6, 7, 8}) diag = diag && m.c[c] == R(0);
#define MC3D_FLUX(MF, WL) \
    flux_kernel<R, MF, NP, WL><<<grid, 256, 0, st>>>(g, q[0], q[1], q[2], q[3], q[4], dp, m, p, mu_sgs, k_sgs, taukk, Tmu, op)
    const bool wall = p.wall_mask != 0 || p.cons_mask != 0;
    if (!m.constant) {
        if (wall) MC3D_FLUX(MET_FIELD, true);
        else MC3D_FLUX(MET_FIELD, false);
    } else if (!diag) {
        if (wall) MC3D_FLUX(MET_CONST, true);
        else MC3D_FLUX(MET_CONST, false);
    } else {
        if (wall) MC3D_FLUX(MET_DIAG, true);
        else MC3D_FLUX(MET_DIAG, false);
    }
#undef MC3D_FLUX
    MC3D_CUDA_TRY(cudaGetLastError());
    return MC3D_OK;
}

template <typename R>
__global__ void vreman_kernel(Grid3 g, const R *__restrict__ r0, DerivPtrs12 dp, Metrics<R> m, FluxParams fp,
                              R *mu_sgs) {
    const R *const *d = reinterpret_cast<const R *const *>(dp.p);
    const double dvol = fp.dxi[0] * fp.dxi[1] * fp.dxi[2];
    long long n = g.n();
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        R gu[3][3];
        velocity_gradient<R>(m, i, d, gu);
        // getSGSViscosity reads the conserved rho (Core.cpp:567)
        const R rho = fp.cons_mask && on_faces(g, i, fp.cons_mask) ? (R)fp.cons[0][i] : (R)r0[i];
        mu_sgs[i] = vreman_mu<R>(gu, rho, vreman_d1<R>(dvol, met(m, 0, i)));
    }
}

template <typename R>
int launch_vreman(const Grid3 &g, const R *const q[5], const R *const d[12], const Metrics<R> &m,
                  const FluxParams &p, R *mu_sgs, cudaStream_t st) {
    DerivPtrs12 dp;
    for (int i = 0; i < 12; i++) dp.p[i] = d[i];
    vreman_kernel<R><<<grid_for(g.n(), 256), 256, 0, st>>>(g, q[0], dp, m, p, mu_sgs);
    MC3D_CUDA_TRY(cudaGetLastError());
    return MC3D_OK;
}

// ---- RK register updates ----
// RK4 (src/RK4.hpp:47-125), TVDRK3 (src/TVDRK3.hpp:50-133) and the 2N-storage
// KenRK4 / LSLDDRK4 (src/KenRK4.hpp:53-152, src/LSLDDRK4.hpp:93-320).
struct Q5 {
    double *p[5];
};
template <typename R>
struct K5 {
    const R *p[5];
};

// Two consecutive points per thread: one 8/16-byte access per array, and every
// array the stage reads is loaded before any store of the iteration (the
// register arrays are written in place, so stores would otherwise order the
// following loads behind them).
// Stage kinds: the scheme and where the stage sits in it (first, middle,
// last), which fixes the registers it reads and writes.
enum RkMode { RKM_RK4_1, RKM_RK4_MID, RKM_RK4_LAST, RKM_TVD_1, RKM_TVD_2, RKM_TVD_3, RKM_2N_1, RKM_2N_MID, RKM_2N_LAST };

template <typename R, int M>
__global__ void __launch_bounds__(256) rk_kernel(Grid3 g, RkStage rs, K5<R> k2, Q5 q1, Q5 qk, Q5 q2, P5<R> prim,
                                                 int want_prims) {
    const long long n = g.n();
    constexpr bool rk4 = M <= RKM_RK4_LAST, tvd = M >= RKM_TVD_1 && M <= RKM_TVD_3, two_n = M >= RKM_2N_1;
    constexpr bool last = M == RKM_RK4_LAST || M == RKM_TVD_3 || M == RKM_2N_LAST;
    // registers read / written by this stage
    constexpr bool rd_q1 = M != RKM_RK4_LAST;
    constexpr bool rd_qk = M == RKM_TVD_2 || M == RKM_TVD_3 || M == RKM_2N_MID || M == RKM_2N_LAST;
    constexpr bool rd_q2 = M == RKM_RK4_MID || M == RKM_RK4_LAST;
    constexpr bool wr_q1 = two_n;
    constexpr bool wr_qk = !last;
    constexpr bool wr_q2 = rk4 || last;
    constexpr bool first = M == RKM_RK4_1 || M == RKM_TVD_1 || M == RKM_2N_1;
    const long long npairs = (n + 1) / 2;
    for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < npairs;
         j += (long long)gridDim.x * blockDim.x) {
        const long long i = 2 * j;
        const bool two = i + 1 < n;
        double K[5][2], A[5][2], B[5][2], C[5][2];
#pragma unroll
        for (int v = 0; v < 5; v++) {
            ld_pair<R>(k2.p[v], i, two, K[v]);
            if (rd_q1) ld_pair<double>(q1.p[v], i, two, A[v]);
            if (rd_qk) ld_pair<double>(qk.p[v], i, two, B[v]);
            if (rd_q2) ld_pair<double>(q2.p[v], i, two, C[v]);
        }
        double nk[5][2], o1[5][2], ok[5][2], o2[5][2];
#pragma unroll
        for (int v = 0; v < 5; v++) {
#pragma unroll
            for (int p = 0; p < 2; p++) {
                const double k = K[v][p];
                nk[v][p] = o1[v][p] = ok[v][p] = o2[v][p] = 0.0;
                if (rk4) {
                    // src/RK4.hpp:47-125
                    if (first) {
                        double b1 = A[v][p];
                        o2[v][p] = b1 + rs.a * k;
                        ok[v][p] = nk[v][p] = b1 + rs.b * k;
                    } else if (!last) {
                        o2[v][p] = C[v][p] + rs.a * k;
                        ok[v][p] = nk[v][p] = A[v][p] + rs.b * k;
                    } else {
                        o2[v][p] = C[v][p] + rs.a * k;
                    }
                } else if (tvd) {
                    // src/TVDRK3.hpp:50-133
                    if (first) ok[v][p] = nk[v][p] = A[v][p] + 1.0 * k;
                    else if (M == RKM_TVD_2) ok[v][p] = nk[v][p] = 0.75 * A[v][p] + 0.25 * B[v][p] + 0.25 * k;
                    else o2[v][p] = (1.0 / 3.0) * A[v][p] + (2.0 / 3.0) * B[v][p] + (2.0 / 3.0) * k;
                } else {
                    // 2N low-storage schemes (src/KenRK4.hpp:53-152, src/LSLDDRK4.hpp:93-320)
                    if (first) {
                        ok[v][p] = nk[v][p] = A[v][p] + rs.b * k;
                        o1[v][p] = k;
                    } else {
                        double r = k + rs.a * A[v][p];
                        o1[v][p] = r;
                        if (!last) ok[v][p] = nk[v][p] = B[v][p] + rs.b * r;
                        else o2[v][p] = B[v][p] + rs.b * r;
                    }
                }
            }
        }
        const bool put_q1 = wr_q1 && !(last && (rs.skip_last & 1));
        const bool put_q2 = wr_q2 && !(last && (rs.skip_last & 2));
#pragma unroll
        for (int v = 0; v < 5; v++) {
            if (put_q1) st_pair<double>(q1.p[v], i, two, o1[v][0], o1[v][1]);
            if (wr_qk) st_pair<double>(qk.p[v], i, two, ok[v][0], ok[v][1]);
            if (put_q2) st_pair<double>(q2.p[v], i, two, o2[v][0], o2[v][1]);
        }
        // the final state in the working precision, for the filter that follows
        if (last && want_prims == 2) {
#pragma unroll
            for (int v = 0; v < 5; v++) st_pair<R>(prim.p[v], i, two, (R)o2[v][0], (R)o2[v][1]);
        }
        // primitives of the next stage state (updateNonConservedData, Core.cpp:1165-1177)
        if (!last && want_prims == 1) {
            double pr[5][2];
#pragma unroll
            for (int p = 0; p < 2; p++) {
                double rho = nk[0][p];
                double u = nk[1][p] / rho, vv = nk[2][p] / rho, w = nk[3][p] / rho;
                double pp = (GAMMA - 1) * (nk[4][p] - 0.5 * rho * (u * u + vv * vv + w * w));
                pr[0][p] = rho;
                pr[1][p] = u;
                pr[2][p] = vv;
                pr[3][p] = w;
                pr[4][p] = pp / (rho * R_GAS);
            }
#pragma unroll
            for (int v = 0; v < 5; v++) st_pair<R>(prim.p[v], i, two, pr[v][0], pr[v][1]);
        }
    }
}

template <typename R>
int launch_rk_update(const Grid3 &g, const RkStage &rs, const R *const k2[5], double *const q1[5],
                     double *const qk[5], double *const q2[5], R *const prim[5], cudaStream_t st,
                     bool copy_final) {
    K5<R> k;
    Q5 a, b, c;
    P5<R> P;
    for (int v = 0; v < 5; v++) {
        k.p[v] = k2[v];
        a.p[v] = q1[v];
        b.p[v] = qk[v];
        c.p[v] = q2[v];
        P.p[v] = prim ? prim[v] : nullptr;
    }
    const bool first = rs.stage == 1, last = rs.stage >= rs.nstages;
    int mode;
    if (rs.scheme == MC3D_RK4) mode = first ? RKM_RK4_1 : (last ? RKM_RK4_LAST : RKM_RK4_MID);
    else if (rs.scheme == MC3D_TVDRK3) mode = first ? RKM_TVD_1 : (last ? RKM_TVD_3 : RKM_TVD_2);
    else mode = first ? RKM_2N_1 : (last ? RKM_2N_LAST : RKM_2N_MID);
    // 1: primitives of the next stage state; 2 (last stage): the final state in R
    const int grid = grid_for((g.n() + 1) / 2, 256), wp = prim == nullptr ? 0 : (copy_final ? 2 : 1);
    switch (mode) {
        case RKM_RK4_1: rk_kernel<R, RKM_RK4_1><<<grid, 256, 0, st>>>(g, rs, k, a, b, c, P, wp); break;
        case RKM_RK4_MID: rk_kernel<R, RKM_RK4_MID><<<grid, 256, 0, st>>>(g, rs, k, a, b, c, P, wp); break;
        case RKM_RK4_LAST: rk_kernel<R, RKM_RK4_LAST><<<grid, 256, 0, st>>>(g, rs, k, a, b, c, P, wp); break;
        case RKM_TVD_1: rk_kernel<R, RKM_TVD_1><<<grid, 256, 0, st>>>(g, rs, k, a, b, c, P, wp); break;
        case RKM_TVD_2: rk_kernel<R, RKM_TVD_2><<<grid, 256, 0, st>>>(g, rs, k, a, b, c, P, wp); break;
        case RKM_TVD_3: rk_kernel<R, RKM_TVD_3><<<grid, 256, 0, st>>>(g, rs, k, a, b, c, P, wp); break;
        case RKM_2N_1: rk_kernel<R, RKM_2N_1><<<grid, 256, 0, st>>>(g, rs, k, a, b, c, P, wp); break;
        case RKM_2N_MID: rk_kernel<R, RKM_2N_MID><<<grid, 256, 0, st>>>(g, rs, k, a, b, c, P, wp); break;
        default: rk_kernel<R, RKM_2N_LAST><<<grid, 256, 0, st>>>(g, rs, k, a, b, c, P, wp); break;
    }
    MC3D_CUDA_TRY(cudaGetLastError());
    return MC3D_OK;
}

// setInitialConditions without walls (src/CurvilinearCSolver_BC.cpp:31-59):
// rhoU = rho U, ..., rhoE = p/(gamma-1) + (1/2) rho |U|^2, rounded as the host
// restatement does; *bad is set where the state is non-finite or rho <= 0.
__global__ void init_conserved_kernel(long long n, const double *__restrict__ rho, const double *__restrict__ U,
                                      const double *__restrict__ V, const double *__restrict__ W,
                                      const double *__restrict__ p, Q5 q, int *bad) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const double r = rho[i], u = U[i], v = V[i], w = W[i], pp = p[i];
        const double e = __dadd_rn(__ddiv_rn(pp, GAMMA - 1.0),
                                   __dmul_rn(__dmul_rn(0.5, r), __dadd_rn(__dadd_rn(__dmul_rn(u, u), __dmul_rn(v, v)),
                                                                        __dmul_rn(w, w))));
        q.p[0][i] = r;
        q.p[1][i] = __dmul_rn(r, u);
        q.p[2][i] = __dmul_rn(r, v);
        q.p[3][i] = __dmul_rn(r, w);
        q.p[4][i] = e;
        if (!isfinite(e) || !(r > 0)) atomicOr(bad, 1);
    }
}

int launch_init_conserved(long long n, const double *const prim[5], double *const q[5], int *bad, cudaStream_t st) {
    Q5 o;
    for (int v = 0; v < 5; v++) o.p[v] = q[v];
    init_conserved_kernel<<<(int)std::min<long long>((n + 255) / 256, 148 * 16), 256, 0, st>>>(
        n, prim[0], prim[1], prim[2], prim[3], prim[4], o, bad);
    MC3D_CUDA_TRY(cudaGetLastError());
    return MC3D_OK;
}

template <typename R>
__global__ void to_real_kernel(Grid3 g, Q5 src, K5<R> dst) {
    long long n = g.n();
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
#pragma unroll
        for (int v = 0; v < 5; v++)
            if (dst.p[v]) const_cast<R *>(dst.p[v])[i] = (R)src.p[v][i];
    }
}

template <typename R>
int launch_to_real(const Grid3 &g, const double *const src[5], R *const dst[5], cudaStream_t st) {
    Q5 s;
    K5<R> d;
    for (int v = 0; v < 5; v++) {
        s.p[v] = const_cast<double *>(src[v]);
        d.p[v] = dst[v];
    }
    to_real_kernel<R><<<grid_for(g.n(), 256), 256, 0, st>>>(g, s, d);
    MC3D_CUDA_TRY(cudaGetLastError());
    return MC3D_OK;
}

// ---- CFL (calcDtFromCFL, Core.cpp:189-237) ----
template <typename R>
__global__ void cfl_kernel(Grid3 g, Q5 q, Metrics<R> m, double i0, double i1, double i2, unsigned long long *umax) {
    __shared__ double red[32];
    double best = 0.0;
    bool bad = false;
    long long n = g.n();
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        double rho = q.p[0][i];
        double u = q.p[1][i] / rho, v = q.p[2][i] / rho, w = q.p[3][i] / rho;
        double p = (GAMMA - 1) * (q.p[4][i] - 0.5 * rho * (u * u + v * v + w * w));
        double c = sqrt(GAMMA * p / rho);
        double uc = (double)met(m, 1, i) * (fabs(u) + c) * i0 + (double)met(m, 5, i) * (fabs(v) + c) * i1 +
                    (double)met(m, 9, i) * (fabs(w) + c) * i2;
        if (!isfinite(uc)) bad = true;
        else if (uc > best) best = uc;
    }
    for (int o = 16; o > 0; o >>= 1) best = fmax(best, __shfl_xor_sync(0xffffffffu, best, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = best;
    __syncthreads();
    if (threadIdx.x < 32) {
        double b = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) b = fmax(b, __shfl_xor_sync(0xffffffffu, b, o));
        if (threadIdx.x == 0) atomicMax(umax, (unsigned long long)__double_as_longlong(b));
    }
    // a non-finite state poisons the maximum: dt becomes NaN and the host check reports it
    if (bad) atomicMax(umax, 0x7ff8000000000000ull);
}

template <typename R>
int launch_cfl(const Grid3 &g, const double *const q[5], const Metrics<R> &m, const double dxi[3],
               unsigned long long *umax, cudaStream_t st) {
    Q5 s;
    for (int v = 0; v < 5; v++) s.p[v] = const_cast<double *>(q[v]);
    cfl_kernel<R><<<grid_for(g.n(), 256), 256, 0, st>>>(g, s, m, 1.0 / dxi[0], 1.0 / dxi[1], 1.0 / dxi[2], umax);
    MC3D_CUDA_TRY(cudaGetLastError());
    return MC3D_OK;
}

__global__ void finalize_dt_kernel(TimeState *ts, int ts_type, double cfl, double dt_const, int first) {
    double m = __longlong_as_double((long long)ts->umax_bits);
    ts->cfl_max = m;
    if (!isfinite(m)) ts->nonfinite = 1;
    ts->dt = (ts_type == MC3D_CONST_CFL) ? cfl / m : dt_const;
    ts->time_step += 1;
    if (!first) ts->time += ts->dt;
    ts->umax_bits = 0ull;
}

int launch_finalize_dt(TimeState *ts, int ts_type, double cfl, double dt_const, int first_step, cudaStream_t st) {
    finalize_dt_kernel<<<1, 1, 0, st>>>(ts, ts_type, cfl, dt_const, first_step);
    MC3D_CUDA_TRY(cudaGetLastError());
    return MC3D_OK;
}

__global__ void integrals_kernel(Grid3 g, Q5 q, double *acc) {
    __shared__ double r1[32], r2[32];
    double ke = 0, ms = 0;
    long long n = g.n();
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        double rho = q.p[0][i];
        double a = q.p[1][i], b = q.p[2][i], c = q.p[3][i];
        ke += 0.5 * (a * a + b * b + c * c) / rho;
        ms += rho;
    }
    for (int o = 16; o > 0; o >>= 1) {
        ke += __shfl_xor_sync(0xffffffffu, ke, o);
        ms += __shfl_xor_sync(0xffffffffu, ms, o);
    }
    if ((threadIdx.x & 31) == 0) {
        r1[threadIdx.x >> 5] = ke;
        r2[threadIdx.x >> 5] = ms;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0, b = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) {
            a += r1[w];
            b += r2[w];
        }
        atomicAdd(acc, a);
        atomicAdd(acc + 1, b);
    }
}

int launch_integrals(const Grid3 &g, const double *const q[5], double *acc2, cudaStream_t st) {
    Q5 s;
    for (int v = 0; v < 5; v++) s.p[v] = const_cast<double *>(q[v]);
    integrals_kernel<<<grid_for(g.n(), 256), 256, 0, st>>>(g, s, acc2);
    MC3D_CUDA_TRY(cudaGetLastError());
    return MC3D_OK;
}

#define MC3D_INST(R)                                                                                              \
    template int launch_primitives<R>(const Grid3 &, const double *const[5], R *const[5], cudaStream_t);          \
    template int launch_flux<R>(const Grid3 &, const R *const[5], const R *const[12], const Metrics<R> &,         \
                                const FluxParams &, const R *, const R *, const R *, const R *, R *const[15],    \
                                cudaStream_t);                                                                   \
    template int launch_vreman<R>(const Grid3 &, const R *const[5], const R *const[12], const Metrics<R> &,       \
                                  const FluxParams &, R *, cudaStream_t);                                         \
    template int launch_rk_update<R>(const Grid3 &, const RkStage &, const R *const[5], double *const[5],         \
                                     double *const[5], double *const[5], R *const[5], cudaStream_t, bool);        \
    template int launch_to_real<R>(const Grid3 &, const double *const[5], R *const[5], cudaStream_t);             \
    template int launch_cfl<R>(const Grid3 &, const double *const[5], const Metrics<R> &, const double[3],        \
                               unsigned long long *, cudaStream_t);
MC3D_INST(float)
MC3D_INST(double)
#undef MC3D_INST

}  // namespace mc3d
