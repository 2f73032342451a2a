// Dynamic Smagorinsky model (Germano-Lilly, test-filter ratio^2 = 4) and the
// averaging of SGS coefficients, as pointwise kernels around the batched
// test-filter sweeps the solver issues:
//
//   dsm_prep_mu      S_ij, |S|, M_ij(2), L_ij(t), 2 rho |S|^2 and the
//                    momenta: the 24 fields filtered together
//   dsm_finish_mu    M_ij, L_ij from the filtered fields; Lkk, C_I
//                    denominator, L_ij M_ij, M_ij M_ij (averaged next)
//   dsm_mu_taukk     mu_sgs, tau_kk and the temperature of the pressure
//                    with the SGS normal stresses
//   dsm_prep_k       N_i, K_i, rho T, gradT: the 10 fields filtered together
//   dsm_finish_k     N_i N_i and N_i K_i (averaged next)
//   dsm_ksgs         k_sgs
//
// DSMSGS::calcMuSGSTaukk / calcKSGS (src/DSMSGS.hpp:130-443) and the solver's
// use of tau_kk (src/CurvilinearCSolver_Core.cpp:567-606).
//
// Averaging (AbstractSGS::doAveraging, src/AbstractSGS.cpp:13-160): XI1/XI2/
// XI3 replace a field by its mean along one grid direction (line_mean),
// GLOBAL by its mean over the block (global_sum + fill_value); LOCAL is three
// filter sweeps issued by the solver.
#include <cmath>

#include "pointwise_common.cuh"

namespace mc3d {

namespace {

constexpr double TFR2 = 2.0 * 2.0;   // testFilterRatioSquare (src/DSMSGS.hpp:55)

template <typename R>
__device__ __forceinline__ void grad_u(const Metrics<R> &m, long long i, const R *const *d, R gu[3][3]) {
    // gradU[a][b] = J1b dUa1 + J2b dUa2 + J3b dUa3 (Core.cpp:548-561)
#pragma unroll
    for (int a = 0; a < 3; a++) {
        R d1 = d[3 * a][i], d2 = d[3 * a + 1][i], d3 = d[3 * a + 2][i];
#pragma unroll
        for (int b = 0; b < 3; b++) gu[a][b] = met(m, 1 + b, i) * d1 + met(m, 4 + b, i) * d2 + met(m, 7 + b, i) * d3;
    }
}

template <typename R>
__global__ void dsm_prep_mu_kernel(Grid3 g, DsmPrepMu<R> a, Metrics<R> m) {
    const long long n = g.n();
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        R gu[3][3];
        grad_u<R>(m, i, a.d, gu);
        const R rho = (R)a.q[0][i], ru = (R)a.q[1][i], rv = (R)a.q[2][i], rw = (R)a.q[3][i];
        const R S00 = gu[0][0], S11 = gu[1][1], S22 = gu[2][2];
        const R S01 = (R)0.5 * (gu[0][1] + gu[1][0]);
        const R S02 = (R)0.5 * (gu[0][2] + gu[2][0]);
        const R S12 = (R)0.5 * (gu[1][2] + gu[2][1]);
        const R Smag = sqrt((R)2.0 * (S00 * S00 + S11 * S11 + S22 * S22) + (R)4.0 * (S01 * S01 + S02 * S02 + S12 * S12));
        const R tr = S00 + S11 + S22, third = (R)(1.0 / 3.0);
        R *const *o = a.out;
        o[0][i] = (R)2.0 * rho * Smag * (S00 - third * tr);
        o[1][i] = (R)2.0 * rho * Smag * S01;
        o[2][i] = (R)2.0 * rho * Smag * S02;
        o[3][i] = (R)2.0 * rho * Smag * (S11 - third * tr);
        o[4][i] = (R)2.0 * rho * Smag * S12;
        o[5][i] = (R)2.0 * rho * Smag * (S22 - third * tr);
        o[6][i] = S00;
        o[7][i] = S01;
        o[8][i] = S02;
        o[9][i] = S11;
        o[10][i] = S12;
        o[11][i] = S22;
        o[12][i] = Smag;
        o[13][i] = rho;
        o[14][i] = ru * ru / rho;
        o[15][i] = ru * rv / rho;
        o[16][i] = ru * rw / rho;
        o[17][i] = rv * rv / rho;
        o[18][i] = rv * rw / rho;
        o[19][i] = rw * rw / rho;
        o[20][i] = (R)2.0 * rho * Smag * Smag;
        o[21][i] = ru;
        o[22][i] = rv;
        o[23][i] = rw;
        a.smag[i] = Smag;
    }
}

template <typename R>
__global__ void dsm_finish_mu_kernel(Grid3 g, DsmFinishMu<R> a) {
    const long long n = g.n();
    const R third = (R)(1.0 / 3.0);
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const R *const *h = a.hat;   // the 24 filtered fields of dsm_prep_mu
        const R rho_h = h[13][i], Smag_h = h[12][i];
        const R Sh00 = h[6][i], Sh01 = h[7][i], Sh02 = h[8][i], Sh11 = h[9][i], Sh12 = h[10][i], Sh22 = h[11][i];
        const R trh = Sh00 + Sh11 + Sh22;
        const R c = (R)(2.0 * TFR2) * rho_h * Smag_h;
        const R M00 = h[0][i] - c * (Sh00 - third * trh);
        const R M01 = h[1][i] - c * Sh01;
        const R M02 = h[2][i] - c * Sh02;
        const R M11 = h[3][i] - c * (Sh11 - third * trh);
        const R M12 = h[4][i] - c * Sh12;
        const R M22 = h[5][i] - c * (Sh22 - third * trh);
        const R ruh = h[21][i], rvh = h[22][i], rwh = h[23][i];
        const R L00 = h[14][i] - ruh * ruh / rho_h;
        const R L01 = h[15][i] - ruh * rvh / rho_h;
        const R L02 = h[16][i] - ruh * rwh / rho_h;
        const R L11 = h[17][i] - rvh * rvh / rho_h;
        const R L12 = h[18][i] - rvh * rwh / rho_h;
        const R L22 = h[19][i] - rwh * rwh / rho_h;
        const R Lkk = L00 + L11 + L22;
        a.out[0][i] = Lkk;
        a.out[1][i] = a.use_taukk ? (R)(2.0 * TFR2) * rho_h * Smag_h * Smag_h - h[20][i] : R(0);
        a.out[2][i] = (L00 - third * Lkk) * M00 + (L11 - third * Lkk) * M11 + (L22 - third * Lkk) * M22 +
                      (R)2.0 * L01 * M01 + (R)2.0 * L02 * M02 + (R)2.0 * L12 * M12;
        a.out[3][i] = M00 * M00 + M11 * M11 + M22 * M22 + (R)2.0 * M01 * M01 + (R)2.0 * M02 * M02 + (R)2.0 * M12 * M12;
    }
}

template <typename R>
__global__ void dsm_mu_taukk_kernel(Grid3 g, DsmMuTaukk<R> a) {
    const long long n = g.n();
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const double rho = a.q[0][i];
        const R rhoR = (R)rho, Smag = a.smag[i];
        const long long ia = a.avg_scalar ? 0 : i;
        a.mu_sgs[i] = rhoR * Smag * a.avg[2][ia] / a.avg[3][ia];
        const R tk = a.use_taukk ? (R)2.0 * rhoR * Smag * Smag * a.avg[0][ia] / a.avg[1][ia] : R(0);
        a.taukk[i] = tk;
        // p of updateNonConservedData less tau_kk / 2, and the temperature of that pressure
        const double u = a.q[1][i] / rho, v = a.q[2][i] / rho, w = a.q[3][i] / rho;
        double p = (GAMMA - 1) * (a.q[4][i] - 0.5 * rho * (u * u + v * v + w * w));
        if (a.cons_mask && on_faces(g, i, a.cons_mask)) p = (double)a.rho_prim[i] * R_GAS * (double)a.T[i];
        const R pn = (R)p - (R)0.5 * tk;
        a.T[i] = pn / (rhoR * (R)R_GAS);
    }
}

template <typename R>
__global__ void dsm_prep_k_kernel(Grid3 g, DsmPrepK<R> a, Metrics<R> m) {
    const long long n = g.n();
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const R dT1 = a.dT[0][i], dT2 = a.dT[1][i], dT3 = a.dT[2][i];
        // gradT = J^T dT (Core.cpp:596-600)
        const R g0 = met(m, 1, i) * dT1 + met(m, 4, i) * dT2 + met(m, 7, i) * dT3;
        const R g1 = met(m, 2, i) * dT1 + met(m, 5, i) * dT2 + met(m, 8, i) * dT3;
        const R g2 = met(m, 3, i) * dT1 + met(m, 6, i) * dT2 + met(m, 9, i) * dT3;
        const R rho = (R)a.q[0][i], T = a.T[i], Smag = a.smag[i];
        R *const *o = a.out;
        o[0][i] = rho * Smag * g0;
        o[1][i] = rho * Smag * g1;
        o[2][i] = rho * Smag * g2;
        o[3][i] = (R)a.q[1][i] * T;
        o[4][i] = (R)a.q[2][i] * T;
        o[5][i] = (R)a.q[3][i] * T;
        o[6][i] = rho * T;
        o[7][i] = g0;
        o[8][i] = g1;
        o[9][i] = g2;
    }
}

template <typename R>
__global__ void dsm_finish_k_kernel(Grid3 g, DsmFinishK<R> a) {
    const long long n = g.n();
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const R *const *h = a.hat;   // the 10 filtered fields of dsm_prep_k
        const R c = (R)TFR2 * a.rho_hat[i] * a.smag_hat[i];
        const R N0 = c * h[7][i] - h[0][i], N1 = c * h[8][i] - h[1][i], N2 = c * h[9][i] - h[2][i];
        // K_i divides by rho, not rho_hat (src/DSMSGS.hpp:406-408)
        const R rho = (R)a.q[0][i], rT = h[6][i];
        const R K0 = -a.ru_hat[0][i] * rT / rho + h[3][i];
        const R K1 = -a.ru_hat[1][i] * rT / rho + h[4][i];
        const R K2 = -a.ru_hat[2][i] * rT / rho + h[5][i];
        a.out[0][i] = N0 * N0 + N1 * N1 + N2 * N2;
        a.out[1][i] = K0 * N0 + K1 * N1 + K2 * N2;
    }
}

template <typename R>
__global__ void dsm_ksgs_kernel(Grid3 g, const double *__restrict__ rho, const R *__restrict__ smag,
                                const R *__restrict__ nini, const R *__restrict__ niki, R *__restrict__ ksgs,
                                int avg_scalar) {
    const long long n = g.n();
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const long long ia = avg_scalar ? 0 : i;
        const R c_over_prt = niki[ia] / nini[ia];
        ksgs[i] = -(R)CP * c_over_prt * (R)rho[i] * smag[i];
    }
}

// ---- averaging ----
// mean along direction DIR of every line: each term divided by the line length
// and summed in index order, as the reference's XI*_AVG loops do
template <typename R, int DIR>
__global__ void line_mean_kernel(Grid3 g, AvgBatch<R> b) {
    const int f = blockIdx.y;
    const long long nlines = DIR == 0 ? (long long)g.Ny * g.Nz : (DIR == 1 ? (long long)g.Nx * g.Nz : (long long)g.Nx * g.Ny);
    const int N = DIR == 0 ? g.Nx : (DIR == 1 ? g.Ny : g.Nz);
    for (long long l = blockIdx.x * (long long)blockDim.x + threadIdx.x; l < nlines;
         l += (long long)gridDim.x * blockDim.x) {
        long long base, stride;
        if (DIR == 0) {
            base = l * g.Nx;
            stride = 1;
        } else if (DIR == 1) {
            const long long i = l % g.Nx, k = l / g.Nx;
            base = i + (long long)g.Nx * g.Ny * k;
            stride = g.Nx;
        } else {
            base = l;
            stride = (long long)g.Nx * g.Ny;
        }
        const R *in = b.in[f];
        R s = 0;
        for (int j = 0; j < N; j++) s += in[base + j * stride] / (R)N;
        R *out = b.out[f];
        for (int j = 0; j < N; j++) out[base + j * stride] = s;
    }
}

// block partial sums (FP64) of every field; partial[f * gridDim.x + block]
template <typename R>
__global__ void __launch_bounds__(256) global_sum_kernel(Grid3 g, AvgBatch<R> b, double *partial) {
    __shared__ double red[8];
    const int f = blockIdx.y;
    const long long n = g.n();
    double s = 0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        s += (double)b.in[f][i];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0;
        for (int w = 0; w < 8; w++) t += red[w];
        partial[f * gridDim.x + blockIdx.x] = t;
    }
}

// out[f][i] = (sum of the partials of field f) / n, the block mean, for i < nfill
template <typename R>
__global__ void fill_mean_kernel(Grid3 g, AvgBatch<R> b, const double *partial, int nparts, long long nfill) {
    const int f = blockIdx.y;
    __shared__ double mean;
    if (threadIdx.x == 0) {
        double t = 0;
        for (int k = 0; k < nparts; k++) t += partial[f * nparts + k];
        mean = t / (double)g.n();
    }
    __syncthreads();
    const R m = (R)mean;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nfill; i += (long long)gridDim.x * blockDim.x)
        b.out[f][i] = m;
}

}  // namespace

template <typename R>
int launch_dsm_prep_mu(const Grid3 &g, const DsmPrepMu<R> &a, const Metrics<R> &m, cudaStream_t st) {
    dsm_prep_mu_kernel<R><<<grid_for(g.n(), 256), 256, 0, st>>>(g, a, m);
    MC3D_CUDA_TRY(cudaGetLastError());
    return MC3D_OK;
}
template <typename R>
int launch_dsm_finish_mu(const Grid3 &g, const DsmFinishMu<R> &a, cudaStream_t st) {
    dsm_finish_mu_kernel<R><<<grid_for(g.n(), 256), 256, 0, st>>>(g, a);
    MC3D_CUDA_TRY(cudaGetLastError());
    return MC3D_OK;
}
template <typename R>
int launch_dsm_mu_taukk(const Grid3 &g, const DsmMuTaukk<R> &a, cudaStream_t st) {
    dsm_mu_taukk_kernel<R><<<grid_for(g.n(), 256), 256, 0, st>>>(g, a);
    MC3D_CUDA_TRY(cudaGetLastError());
    return MC3D_OK;
}
template <typename R>
int launch_dsm_prep_k(const Grid3 &g, const DsmPrepK<R> &a, const Metrics<R> &m, cudaStream_t st) {
    dsm_prep_k_kernel<R><<<grid_for(g.n(), 256), 256, 0, st>>>(g, a, m);
    MC3D_CUDA_TRY(cudaGetLastError());
    return MC3D_OK;
}
template <typename R>
int launch_dsm_finish_k(const Grid3 &g, const DsmFinishK<R> &a, cudaStream_t st) {
    dsm_finish_k_kernel<R><<<grid_for(g.n(), 256), 256, 0, st>>>(g, a);
    MC3D_CUDA_TRY(cudaGetLastError());
    return MC3D_OK;
}
template <typename R>
int launch_dsm_ksgs(const Grid3 &g, const double *rho, const R *smag, const R *nini, const R *niki, R *ksgs,
                    int avg_scalar, cudaStream_t st) {
    dsm_ksgs_kernel<R><<<grid_for(g.n(), 256), 256, 0, st>>>(g, rho, smag, nini, niki, ksgs, avg_scalar);
    MC3D_CUDA_TRY(cudaGetLastError());
    return MC3D_OK;
}

template <typename R>
int launch_average(const Grid3 &g, int mode, const AvgBatch<R> &b, double *scratch, size_t scratch_doubles,
                   cudaStream_t st, bool mean_only) {
    if (b.nf <= 0) return MC3D_OK;
    if (b.nf > 8) return fail(MC3D_ERR_ARG, "at most 8 fields per average");
    if (mode == MC3D_AVG_XI1 || mode == MC3D_AVG_XI2 || mode == MC3D_AVG_XI3) {
        const long long nl = mode == MC3D_AVG_XI1 ? (long long)g.Ny * g.Nz
                             : mode == MC3D_AVG_XI2 ? (long long)g.Nx * g.Nz : (long long)g.Nx * g.Ny;
        dim3 grid((unsigned)std::min<long long>((nl + 127) / 128, 148 * 8), b.nf);
        if (mode == MC3D_AVG_XI1) line_mean_kernel<R, 0><<<grid, 128, 0, st>>>(g, b);
        else if (mode == MC3D_AVG_XI2) line_mean_kernel<R, 1><<<grid, 128, 0, st>>>(g, b);
        else line_mean_kernel<R, 2><<<grid, 128, 0, st>>>(g, b);
        MC3D_CUDA_TRY(cudaGetLastError());
        return MC3D_OK;
    }
    if (mode == MC3D_AVG_GLOBAL) {
        int parts = 148 * 4;
        if ((size_t)parts * b.nf > scratch_doubles) parts = (int)(scratch_doubles / b.nf);
        if (parts < 1) return fail(MC3D_ERR_ARG, "averaging scratch too small");
        global_sum_kernel<R><<<dim3(parts, b.nf), 256, 0, st>>>(g, b, scratch);
        MC3D_CUDA_TRY(cudaGetLastError());
        // (mean_only: one block per field writes element 0)
        fill_mean_kernel<R><<<dim3(mean_only ? 1 : grid_for(g.n(), 256), b.nf), 256, 0, st>>>(
            g, b, scratch, parts, mean_only ? 1LL : g.n());
        MC3D_CUDA_TRY(cudaGetLastError());
        return MC3D_OK;
    }
    return fail(MC3D_ERR_ARG, "averaging mode is not a reduction");
}

#define MC3D_DSM_INST(R)                                                                                         \
    template int launch_dsm_prep_mu<R>(const Grid3 &, const DsmPrepMu<R> &, const Metrics<R> &, cudaStream_t);   \
    template int launch_dsm_finish_mu<R>(const Grid3 &, const DsmFinishMu<R> &, cudaStream_t);                  \
    template int launch_dsm_mu_taukk<R>(const Grid3 &, const DsmMuTaukk<R> &, cudaStream_t);                    \
    template int launch_dsm_prep_k<R>(const Grid3 &, const DsmPrepK<R> &, const Metrics<R> &, cudaStream_t);     \
    template int launch_dsm_finish_k<R>(const Grid3 &, const DsmFinishK<R> &, cudaStream_t);                    \
    template int launch_dsm_ksgs<R>(const Grid3 &, const double *, const R *, const R *, const R *, R *,          \
                                    int, cudaStream_t);                                                                   \
    template int launch_average<R>(const Grid3 &, int, const AvgBatch<R> &, double *, size_t, cudaStream_t, bool);
MC3D_DSM_INST(float)
MC3D_DSM_INST(double)
#undef MC3D_DSM_INST

}  // namespace mc3d
