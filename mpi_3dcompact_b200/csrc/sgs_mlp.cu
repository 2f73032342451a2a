// Learned SGS closure in the time step, and the kernels that make its training
// data from this solver's own DNS fields. No counterpart in the reference.
//
// Features of a point (dimensionless, from the resolved state and the grid):
//   x0 log(1 + rho Delta^2 |S| / mu)       grid Reynolds number of the strain
//   x1 W:W / (S:S + W:W)                  rotation fraction
//   x2 tr(S^3) / (S:S)^(3/2)              strain shape
//   x3 tr(S W W) / (S:S + W:W)^(3/2)      strain-rotation alignment
//   x4 tr(S S W W) / (S:S + W:W)^2
//   x5 tr(grad u) / (S:S + W:W)^(1/2)     dilatation
//   x6 Delta |grad T| / T
//   x7 Delta |S| / c                      grid-scale strain Mach number
//   x8 log(rho)
// with S, W the symmetric and antisymmetric parts of grad u, |S| = (2 S:S)^(1/2)
// and Delta = (dxi deta dzeta / J)^(1/3) (the Vreman/DSM grid scale,
// src/VremanSGS.hpp:49-52). Outputs: C (mu_t = rho C Delta^2 |S|) and Pr_t;
// k_sgs = cp mu_t / Pr_t (the form of DSM's k_sgs in the flux, Core.cpp:636-639).
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>

#include "mlp_tc.cuh"

namespace mc3d {

namespace {

template <typename R>
__device__ __forceinline__ float metf(const Metrics<R> &m, int c, long long i) {
    return (float)(m.constant ? m.c[c] : m.m[c][i]);
}

// Warpgroups per CTA of the tensor-core kernels: 256 threads and 63.5 KB of
// shared memory per CTA (the weight image and two activation tiles), so three
// CTAs share an SM and hold 3 x 128 of its 512 TMEM columns. (Four warpgroups
// per CTA at 64 registers, two CTAs and 32 warps per SM, took 220 us per
// 128^3 pass against 212 us: more instructions at the lower register count.)
constexpr int TC_NWG = 2;
constexpr size_t TC_SMEM = 1024 + MLPT_BYTES + TC_NWG * MLPT_TILE + 16 * TC_NWG;

// Fused closure evaluation: features of every point, the network on the
// tensor cores, mu_sgs and k_sgs; *flag counts the points with a feature
// outside the training range (those features are clamped to the range before
// the network). Persistent CTAs; each warpgroup walks tiles of 128 points,
// thread r of the warpgroup owning point r of the tile.
template <typename R>
__global__ void __launch_bounds__(TC_NWG * 128, 3)
    sgs_mlp_kernel(Grid3 g, const R *__restrict__ rho_f, const R *__restrict__ T_f, DerivPtrs12c<R> dp,
                   Metrics<R> m, double dvol, double mu_ref, const uint4 *__restrict__ img, MlpNorm nrm, R *mu_sgs,
                   R *ksgs, int *flag) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    const TcCta c = tc_setup<TC_NWG>(smem_raw, img);
    const int wg = threadIdx.x >> 7, r = threadIdx.x & 127, lane = threadIdx.x & 31;
    unsigned char *tile = c.img + MLPT_BYTES + wg * MLPT_TILE;
    unsigned phase = 0;
    const long long n = g.n(), ntiles = (n + 127) / 128;
    const float delta_c = m.constant ? cbrtf((float)(dvol / (double)m.c[0])) : 0.f;   // Delta of a uniform block
    for (long long t = (long long)blockIdx.x * TC_NWG + wg; t < ntiles; t += (long long)gridDim.x * TC_NWG) {
        const long long i = t * 128 + r;
        const bool ok = i < n;
        float scale = 0.0f;
        bool out_of_range = false;
        float xn[MLP_IN];
        if (ok) {
            float gu[3][3], gT[3];
#pragma unroll
            for (int a = 0; a < 3; a++) {
                const float d1 = (float)dp.p[3 * a][i], d2 = (float)dp.p[3 * a + 1][i], d3 = (float)dp.p[3 * a + 2][i];
#pragma unroll
                for (int b = 0; b < 3; b++)
                    gu[a][b] = metf(m, 1 + b, i) * d1 + metf(m, 4 + b, i) * d2 + metf(m, 7 + b, i) * d3;
            }
            {
                const float d1 = (float)dp.p[9][i], d2 = (float)dp.p[10][i], d3 = (float)dp.p[11][i];
#pragma unroll
                for (int b = 0; b < 3; b++)
                    gT[b] = metf(m, 1 + b, i) * d1 + metf(m, 4 + b, i) * d2 + metf(m, 7 + b, i) * d3;
            }
            const float rhof = (float)rho_f[i], T = (float)T_f[i];
            const float delta = m.constant ? delta_c : cbrtf((float)dvol / metf(m, 0, i));
            const float mu = (float)mu_ref * __powf(T, 0.76f);
            float x[MLP_IN];
            const float smag = mlp_features(gu, rhof, T, gT, delta, mu, x);
            scale = rhof * delta * delta * smag;   // mu_t / C
#pragma unroll
            for (int k = 0; k < MLP_IN; k++) {
                if (!(x[k] >= nrm.lo[k] && x[k] <= nrm.hi[k])) out_of_range = true;   // NaN counts as outside
                const float xc = fminf(fmaxf(x[k], nrm.lo[k]), nrm.hi[k]);
                xn[k] = (xc - nrm.mean[k]) * nrm.inv_std[k];
            }
        } else {
#pragma unroll
            for (int k = 0; k < MLP_IN; k++) xn[k] = 0.0f;
        }
        const unsigned outside = __ballot_sync(0xffffffffu, out_of_range);
        if (outside && lane == 0) atomicAdd(flag, __popc(outside));
        tc_put_input(tile, r, xn);
        float o0, o1;
        if (!tc_forward(c, wg, r, phase, o0, o1)) break;
        if (ok) {
            const float C = fmaxf(0.0f, o0 * nrm.ystd[0] + nrm.ymean[0]);
            const float prt = fminf(10.0f, fmaxf(0.1f, o1 * nrm.ystd[1] + nrm.ymean[1]));
            const float mt = C * scale;
            mu_sgs[i] = (R)mt;
            ksgs[i] = (R)__fdividef((float)CP * mt, prt);
        }
    }
    tc_teardown<TC_NWG>(c);
}

// standalone inference: x [n][9] (raw features, normalised without clamping)
// -> out [n][2] (raw outputs)
__global__ void __launch_bounds__(TC_NWG * 128, 3)
    mlp_infer_kernel(const uint4 *__restrict__ img, MlpNorm nrm, const float *__restrict__ x, int n,
                     float *__restrict__ out) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    const TcCta c = tc_setup<TC_NWG>(smem_raw, img);
    const int wg = threadIdx.x >> 7, r = threadIdx.x & 127;
    unsigned char *tile = c.img + MLPT_BYTES + wg * MLPT_TILE;
    unsigned phase = 0;
    const long long ntiles = ((long long)n + 127) / 128;
    for (long long t = (long long)blockIdx.x * TC_NWG + wg; t < ntiles; t += (long long)gridDim.x * TC_NWG) {
        const long long p = t * 128 + r;
        float xn[MLP_IN];
#pragma unroll
        for (int k = 0; k < MLP_IN; k++) xn[k] = p < n ? (x[p * MLP_IN + k] - nrm.mean[k]) * nrm.inv_std[k] : 0.0f;
        tc_put_input(tile, r, xn);
        float o0, o1;
        if (!tc_forward(c, wg, r, phase, o0, o1)) break;
        if (p < n) {
            out[p * 2 + 0] = o0;
            out[p * 2 + 1] = o1;
        }
    }
    tc_teardown<TC_NWG>(c);
}

// grid of the persistent tensor-core kernels: as many CTAs as fit on the SMs
// together (shared memory, registers, threads, TMEM columns; counted here from
// the kernel's attributes, with the largest shared-memory carveout requested),
// and no more than there are tile pairs
template <typename K>
int tc_grid(K kern, KernelLaunchState &st, long long n, int *blocks) {
    if (int rc = open_kernel(kern, st, TC_SMEM, TC_NWG * 128, nullptr)) return rc;
    int dev = 0;
    MC3D_CUDA_TRY(cudaGetDevice(&dev));
    int ctas = st.ctas[dev].load();
    if (ctas <= 0) {   // first launch on this device: the CTAs that fit, counted once
        MC3D_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout,
                                           (int)cudaSharedmemCarveoutMaxShared));
        int nsm = 0, smem_sm = 0, resv = 0, regs_sm = 0, thr_sm = 0;
        MC3D_CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
        MC3D_CUDA_TRY(cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev));
        MC3D_CUDA_TRY(cudaDeviceGetAttribute(&resv, cudaDevAttrReservedSharedMemoryPerBlock, dev));
        MC3D_CUDA_TRY(cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, dev));
        MC3D_CUDA_TRY(cudaDeviceGetAttribute(&thr_sm, cudaDevAttrMaxThreadsPerMultiProcessor, dev));
        cudaFuncAttributes fa{};
        MC3D_CUDA_TRY(cudaFuncGetAttributes(&fa, kern));
        const int threads = TC_NWG * 128;
        int per = std::min(smem_sm / (int)(TC_SMEM + resv), thr_sm / threads);
        if (fa.numRegs > 0) per = std::min(per, regs_sm / (fa.numRegs * threads));
        per = std::max(1, std::min(per, 512 / (TC_NWG * MLPT_NCOL)));
        ctas = nsm * per;
        st.ctas[dev].store(ctas);
    }
    const long long need = (n + 128LL * TC_NWG - 1) / (128LL * TC_NWG);
    *blocks = (int)std::max(1LL, std::min<long long>(need, (long long)ctas));
    return MC3D_OK;
}

// ---- training data -----------------------------------------------------------
// box filter of factor f of the DNS state (FP64, fine grid Nx*Ny*Nz) onto the
// coarse grid: rho, rhoU_i, rhoU_i U_j (6), rho T, rhoU_i T (3): 14 fields
__global__ void box_filter_kernel(Grid3 gf, int f, Q5c q, CoarseOut out) {
    const Grid3 gc{gf.Nx / f, gf.Ny / f, gf.Nz / f};
    const long long nc = gc.n();
    const double w = 1.0 / ((double)f * f * f);
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < nc; c += (long long)gridDim.x * blockDim.x) {
        const long long ci = c % gc.Nx, cj = (c / gc.Nx) % gc.Ny, ck = c / ((long long)gc.Nx * gc.Ny);
        double acc[14];
        for (int k = 0; k < 14; k++) acc[k] = 0.0;
        for (int dk = 0; dk < f; dk++)
            for (int dj = 0; dj < f; dj++)
                for (int di = 0; di < f; di++) {
                    const long long i = (ci * f + di) + (long long)gf.Nx * ((cj * f + dj) + (long long)gf.Ny * (ck * f + dk));
                    const double rho = q.p[0][i], ru = q.p[1][i], rv = q.p[2][i], rw = q.p[3][i];
                    const double u = ru / rho, v = rv / rho, wv = rw / rho;
                    const double p = (GAMMA - 1) * (q.p[4][i] - 0.5 * rho * (u * u + v * v + wv * wv));
                    const double T = p / (rho * R_GAS);
                    const double vals[14] = {rho, ru, rv, rw, ru * u, ru * v, ru * wv, rv * v, rv * wv, rw * wv,
                                             rho * T, ru * T, rv * T, rw * T};
                    for (int k = 0; k < 14; k++) acc[k] += vals[k];
                }
        for (int k = 0; k < 14; k++) out.p[k][c] = acc[k] * w;
    }
}

// features and least-squares targets on the coarse grid. gd[3*var + dir]:
// d/dxi_dir of u, v, w, T (Favre-filtered) with box metrics J_ii = jd[dir].
// C = -tau^d_ij S^d_ij / (2 rho Delta^2 |S| S^d:S^d); kappa_t = -q_j dT_j / |dT|^2,
// Pr_t = mu_t / kappa_t clipped to [0.1, 10] (0.9 where it is undefined).
__global__ void training_pairs_kernel(Grid3 gc, CoarseIn c, GradIn gd, double jd0, double jd1, double jd2,
                                      double delta, double mu_ref, float *__restrict__ x, float *__restrict__ y) {
    const long long n = gc.n();
    const double jd[3] = {jd0, jd1, jd2};
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const double rho = c.p[0][i];
        const double ut[3] = {c.p[1][i] / rho, c.p[2][i] / rho, c.p[3][i] / rho};
        const double T = c.p[10][i] / rho;
        double gu[3][3], gT[3];
        for (int a = 0; a < 3; a++)
            for (int b = 0; b < 3; b++) gu[a][b] = jd[b] * gd.p[3 * a + b][i];
        for (int b = 0; b < 3; b++) gT[b] = jd[b] * gd.p[9 + b][i];
        const double mu = mu_ref * pow(T, 0.76);
        float guf[3][3], gTf[3], f[MLP_IN];
        for (int a = 0; a < 3; a++) {
            gTf[a] = (float)gT[a];
            for (int b = 0; b < 3; b++) guf[a][b] = (float)gu[a][b];
        }
        mlp_features(guf, (float)rho, (float)T, gTf, (float)delta, (float)mu, f);
        // SGS stress and heat flux of the box filter
        const int ij[6][2] = {{0, 0}, {0, 1}, {0, 2}, {1, 1}, {1, 2}, {2, 2}};
        double tau[3][3];
        for (int k = 0; k < 6; k++) {
            const int a = ij[k][0], b = ij[k][1];
            tau[a][b] = tau[b][a] = c.p[4 + k][i] - c.p[1 + a][i] * c.p[1 + b][i] / rho;
        }
        const double trt = (tau[0][0] + tau[1][1] + tau[2][2]) / 3.0;
        double S[3][3], trs = 0;
        for (int a = 0; a < 3; a++)
            for (int b = 0; b < 3; b++) S[a][b] = 0.5 * (gu[a][b] + gu[b][a]);
        trs = (S[0][0] + S[1][1] + S[2][2]) / 3.0;
        double ts = 0, ss = 0, s2 = 0;
        for (int a = 0; a < 3; a++)
            for (int b = 0; b < 3; b++) {
                const double sd = S[a][b] - (a == b ? trs : 0.0);
                const double td = tau[a][b] - (a == b ? trt : 0.0);
                ts += td * sd;
                ss += sd * sd;
                s2 += S[a][b] * S[a][b];
            }
        const double smag = sqrt(2.0 * s2);
        const double denom = 2.0 * rho * delta * delta * smag * ss;
        const double C = denom > 0 ? -ts / denom : 0.0;
        double qd = 0, g2 = 0;
        for (int b = 0; b < 3; b++) {
            const double qb = c.p[11 + b][i] - c.p[1 + b][i] * c.p[10][i] / rho;
            qd += qb * gT[b];
            g2 += gT[b] * gT[b];
        }
        const double kappa = g2 > 0 ? -qd / g2 : 0.0;
        const double mut = rho * C * delta * delta * smag;
        double prt = 0.9;
        if (kappa > 0 && mut > 0) prt = fmin(10.0, fmax(0.1, mut / kappa));
        for (int k = 0; k < MLP_IN; k++) x[i * MLP_IN + k] = (float)f[k];
        y[i * 2 + 0] = (float)C;
        y[i * 2 + 1] = (float)prt;
    }
}

}  // namespace

template <typename R>
int launch_sgs_mlp(const Grid3 &g, const R *rho, const R *T, const R *const d[12], const Metrics<R> &m, double dvol,
                   double mu_ref, const MlpDev &mlp, R *mu_sgs, R *ksgs, int *flag, cudaStream_t st) {
    DerivPtrs12c<R> dp;
    for (int k = 0; k < 12; k++) dp.p[k] = d[k];
    static KernelLaunchState ks;
    int blocks = 0;
    if (int rc = tc_grid(sgs_mlp_kernel<R>, ks, g.n(), &blocks)) return rc;
    sgs_mlp_kernel<R><<<blocks, TC_NWG * 128, TC_SMEM, st>>>(g, rho, T, dp, m, dvol, mu_ref,
                                                              reinterpret_cast<const uint4 *>(mlp.Tw), mlp.norm,
                                                              mu_sgs, ksgs, flag);
    MC3D_CUDA_TRY(cudaGetLastError());
    return MC3D_OK;
}
template int launch_sgs_mlp<float>(const Grid3 &, const float *, const float *, const float *const[12],
                                   const Metrics<float> &, double, double, const MlpDev &, float *, float *, int *,
                                   cudaStream_t);
template int launch_sgs_mlp<double>(const Grid3 &, const double *, const double *, const double *const[12],
                                    const Metrics<double> &, double, double, const MlpDev &, double *, double *, int *,
                                    cudaStream_t);

int mlp_infer_bf16(const MlpDev &m, const float *x, int n, float *out, cudaStream_t st) {
    if (n <= 0) return MC3D_OK;
    static KernelLaunchState ks;
    int blocks = 0;
    if (int rc = tc_grid(mlp_infer_kernel, ks, n, &blocks)) return rc;
    mlp_infer_kernel<<<blocks, TC_NWG * 128, TC_SMEM, st>>>(reinterpret_cast<const uint4 *>(m.Tw), m.norm, x, n, out);
    MC3D_CUDA_TRY(cudaGetLastError());
    return MC3D_OK;
}

int mlp_wait_timeouts(int *count) {
    MC3D_CUDA_TRY(cudaMemcpyFromSymbol(count, g_mlp_wait_timeouts, sizeof(int)));
    return MC3D_OK;
}

int launch_box_filter(const Grid3 &gf, int f, const double *const q[5], double *const out[14], cudaStream_t st) {
    Q5c qq;
    CoarseOut o;
    for (int v = 0; v < 5; v++) qq.p[v] = q[v];
    for (int k = 0; k < 14; k++) o.p[k] = out[k];
    const long long nc = (long long)(gf.Nx / f) * (gf.Ny / f) * (gf.Nz / f);
    box_filter_kernel<<<(int)std::min<long long>((nc + 255) / 256, 148 * 16), 256, 0, st>>>(gf, f, qq, o);
    MC3D_CUDA_TRY(cudaGetLastError());
    return MC3D_OK;
}

int launch_training_pairs(const Grid3 &gc, const double *const coarse[14], const double *const grads[12],
                          const double jd[3], double delta, double mu_ref, float *x, float *y, cudaStream_t st) {
    CoarseIn c;
    GradIn gd;
    for (int k = 0; k < 14; k++) c.p[k] = coarse[k];
    for (int k = 0; k < 12; k++) gd.p[k] = grads[k];
    training_pairs_kernel<<<(int)std::min<long long>((gc.n() + 255) / 256, 148 * 16), 256, 0, st>>>(
        gc, c, gd, jd[0], jd[1], jd[2], delta, mu_ref, x, y);
    MC3D_CUDA_TRY(cudaGetLastError());
    return MC3D_OK;
}

}  // namespace mc3d
