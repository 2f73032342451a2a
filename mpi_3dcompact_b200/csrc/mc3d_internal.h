// Internal declarations shared by the host and device translation units.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/mc3d.h"

namespace mc3d {

// ---- error plumbing ----------------------------------------------------
void set_error(const std::string &msg);
int fail(int code, const std::string &msg);
#define MC3D_CUDA_TRY(expr)                                                                      \
    do {                                                                                         \
        cudaError_t _e = (expr);                                                                 \
        if (_e != cudaSuccess)                                                                   \
            return ::mc3d::fail(_e == cudaErrorMemoryAllocation ? MC3D_ERR_OOM : MC3D_ERR_CUDA,  \
                                std::string(#expr) + ": " + cudaGetErrorString(_e));            \
    } while (0)

// Launch settings of one kernel instantiation, kept per device because the
// dynamic shared-memory attribute is set per device and the persistent CTA
// count follows the device's SM count: the size the kernel has been opened
// for (0: not yet) and the CTA count for that size, indexed by device ordinal.
constexpr int MAX_DEVICES = 64;
struct KernelLaunchState {
    std::atomic<int> smem[MAX_DEVICES];
    std::atomic<int> ctas[MAX_DEVICES];
};

// Opens `kern` for `smem` bytes of dynamic shared memory on the current
// device (once per device and size) and, when ctas is given, returns the
// number of CTAs of `threads` threads that fill the device.
template <typename K>
inline int open_kernel(K kern, KernelLaunchState &st, size_t smem, int threads, int *ctas) {
    int dev = 0;
    MC3D_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= MAX_DEVICES) return fail(MC3D_ERR_ARG, "device index out of range");
    if ((int)smem > st.smem[dev].load()) {
        MC3D_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        if (ctas) {
            int nsm = 0, per = 0;
            MC3D_CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
            MC3D_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, threads, smem));
            st.ctas[dev].store(nsm * (per > 0 ? per : 1));
        }
        st.smem[dev].store((int)smem);
    }
    if (ctas) {
        *ctas = st.ctas[dev].load();
        if (*ctas <= 0) {   // another thread opened the kernel without a CTA count
            int nsm = 0, per = 0;
            MC3D_CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
            MC3D_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, threads, smem));
            *ctas = nsm * (per > 0 ? per : 1);
            st.ctas[dev].store(*ctas);
        }
    }
    return MC3D_OK;
}

// ---- one compact operator along one direction ---------------------------
// Line kinds: periodic kinds are even.
enum LineKind { K_EXPL_PER = 0, K_EXPL_DIR = 1, K_TRI_PER = 2, K_TRI_DIR = 3, K_PEN_PER = 4, K_PEN_DIR = 5 };

// Host-side description, all factors in FP64 (computed with the reference's
// own elimination order so the GPU reproduces its factors exactly).
struct LineOpHost {
    int N = 0;
    int kind = 0;
    int H = 0;            // interior stencil half-width == boundary rows per end
    int bw = 0;           // boundary row width (Dirichlet)
    bool deriv = false;   // multiply the RHS by 1/dh
    double inv_dh = 1.0;
    double st[11] = {0};  // interior stencil, st[k] multiplies phi[n + k - H]
    std::vector<double> head, tail;   // [H][bw]: rows 0..H-1 on phi[0..bw-1];
                                      // row N-1-r on phi[N-bw..N-1] (ascending)
    // packed factor arrays (see pack layout in coeffs.cpp)
    std::vector<double> arr;
    double sc[4] = {0};   // kind-specific scalars
    double Hm[16] = {0};  // penta cyclic capacitance inverse
    double cp[6] = {0};   // penta cyclic corner values
    // Rows [stat_lo, stat_hi) where every elimination factor, rounded to the
    // working precision, is exactly constant (Toeplitz interior: the factors
    // reach their fixed point a few dozen rows from the ends); stat_c holds
    // those constants.
    int stat_lo = 0, stat_hi = 0;
    double stat_c[5] = {0};
    // Rows [corr_lo, corr_hi) where the cyclic correction columns are below
    // 2^-64 (FP64) / 2^-32 (FP32) of their peak, so the correction is skipped.
    int corr_lo = 0, corr_hi = 0;
    // Segmented solve: S segments of L = N/S rows per line; homogeneous
    // responses of the local forward (to the two incoming eliminated values)
    // and backward (to the two outgoing solution values) recurrences, per row.
    int S = 1;
    std::vector<double> sfa, sfb, sba, sbb;
    // rows from a segment's start (kf) / end (kb) over which the forward /
    // backward responses are above the precision's cut-off (set at upload)
    int seg_kf = 0, seg_kb = 0;
    int L = 0;   // segment length of the register-resident kernel (0: not used)
};

// Segment length of the register-resident line solve for a line of N points
// in a precision (0 when the line goes to the shared-memory kernels).
int reg_segment_len(int N, int kind, int precision);

LineOpHost build_deriv_op(int fd_type, int bc_type, int N, double dh);
LineOpHost build_filter_op(int filter_type, double alphaF, int bc_type, int N);
LineOpHost build_testfilter_op(int type, int bc_type, int N);

// Device-side view (trivially copyable, passed by value to kernels).
template <typename R>
struct LineOpDev {
    int N, kind, H, bw;
    R inv_dh;
    R st[11];
    R sc[4];
    R Hm[16];
    R cp[6];
    const R *head;   // [H][bw]
    const R *tail;   // [H][bw]
    const R *a0;     // tri: m | penta: m1 (m1[N-1] = mL)
    const R *a1;     // tri: rw | penta: m2
    const R *a2;     // tri: c  | penta: rD
    const R *a3;     // tri: z  | penta: C
    const R *a4;     // penta: f
    const R *z0, *z1, *z2, *z3;   // penta cyclic Woodbury columns
    int stat_lo, stat_hi, corr_lo, corr_hi;
    R stat_c[5];
    int S;                         // segments per line (1 = whole-line kernel)
    const R *sfa, *sfb, *sba, *sbb;
    int seg_kf, seg_kb;
    // Register-resident segmented solve (segment length L = N/S rows, 0 when
    // the line length does not suit it). Row-interleaved copies of the
    // factors so one vector load fetches a row's coefficients:
    //   pf  [N][2]  forward  (m1_n, m2_{n-1}) | tri (m_n, 0); zero where unused
    //   pb  [N][4]  backward (C_n, f_n, rD_n, 0) | tri (c_n, 0, rw_n, 0)
    //   pz  [N][4]  penta cyclic columns (z0..z3)_n
    //   sf2 [N][2]  (sfa, sfb)_n,  sb2 [N][2]  (sba, sbb)_n
    //   hp, tp [H][MC3D_BWMAX]  Dirichlet boundary rows, zero padded (head on
    //   phi[0..BWMAX-1], tail right-aligned on phi[N-BWMAX..N-1])
    int L;
    const R *pf, *pb, *pz, *sf2, *sb2, *hp, *tp;
    // FP32 derivative form of the register-resident solve (H <= 3): asym is 1
    // when the interior stencil is antisymmetric with a zero centre, sta[k-1]
    // = st[H+k] / dh; the backward factors pre-multiplied by the reciprocal
    // pivot, stat_b = (C rD, f rD, rD) of the stationary rows and
    //   pbs [N][4]  (C_n rD_n, f_n rD_n, rD_n, 0) | tri (c_n rw_n, 0, rw_n, 0)
    int asym;
    R sta[3];
    R stat_b[3];
    const R *pbs;
};
constexpr int MC3D_BWMAX = 11;   // widest boundary row (11-point filter closures)

// Device copy of an operator in one precision.
struct LineOpBuf {
    void *dev = nullptr;          // single allocation holding every array
    LineOpDev<float> f32{};
    LineOpDev<double> f64{};
    int precision = MC3D_FP64;
    int device = 0;
};
int upload_line_op(const LineOpHost &h, int precision, LineOpBuf &out);
void free_line_op(LineOpBuf &b);

// ---- sweep launch ---------------------------------------------------------
enum EpiMode {
    EPI_STORE = 0,      // out[f] = v
    EPI_STORE_NEG = 1,  // out[f] = -v
    EPI_SUB = 2,        // out[f] -= v
    EPI_RHS_FINAL = 3,  // k2 assembly of solveContinuity..solveEnergy
    EPI_STORE_F64 = 4,  // out64[f] = (double)v
};

struct Grid3 {
    int Nx, Ny, Nz;
    __host__ __device__ long long n() const { return (long long)Nx * Ny * Nz; }
};

// Extra inputs of the k2 assembly epilogue (RHS_FINAL).
template <typename R>
struct RhsFinalArgs {
    const double *dt;        // device scalar (FP64 time accumulator)
    const R *J;              // metric Jacobian field or nullptr (constant)
    R Jc;                    // constant J when J == nullptr
    int quirk;               // momentum k2 carry-over
};

template <typename R>
struct SweepBatch {
    int nf;
    const R *in[16];
    R *out[16];            // EPI_STORE/NEG/SUB target, or the k2 arrays for RHS_FINAL
    const R *aux[16];      // RHS_FINAL: partial RHS arrays
    double *out64[16];     // EPI_STORE_F64 targets
    int eq[16];            // RHS_FINAL: equation index 0..4 of field f
};

template <typename R>
int launch_sweep(int dir, const Grid3 &g, const LineOpDev<R> &op, const SweepBatch<R> &b, int epi,
                 const RhsFinalArgs<R> &rf, const int bc_types[3], bool filter_passthrough,
                 cudaStream_t st);

// ---- pointwise kernels ----------------------------------------------------
template <typename R>
struct Metrics {
    const R *m[10];          // J, J11..J33 (nullptr when constant)
    R c[10];                 // constants
    bool constant;
};

struct FluxParams {
    double mu_ref;
    double dxi[3];
    int les;                 // 0 none, 1 Vreman inline, 2 mu_sgs field, 3 DSM fields
    double pr_t;
    int wall_mask;           // bit f: face f is a wall (mu there from the saved temperature)
    // bit f: on face f the conserved state cons[] differs from the one the
    // primitives were formed from (a sponge relaxation after the previous
    // step); the convective terms there take rho, rhoU, rhoV, rhoW, rhoE from
    // cons[] and p from the primitives, as preStepDerivatives reads them
    int cons_mask;
    const double *cons[5];
};

template <typename R>
int launch_primitives(const Grid3 &g, const double *const q[5], R *const prim[5], cudaStream_t st);
// conserved state of primitive fields rho, U, V, W, p (device); *bad |= 1 on a
// non-finite value or rho <= 0
int launch_init_conserved(long long n, const double *const prim[5], double *const q[5], int *bad, cudaStream_t st);
// primitives and the CFL wave-speed maximum (atomicMax into *umax, as launch_cfl)
template <typename R>
int launch_primitives_cfl(const Grid3 &g, const double *const q[5], R *const prim[5], const Metrics<R> &m,
                          const double dxi[3], unsigned long long *umax, cudaStream_t st);

// prim = rho, U, V, W, T of the stage state
// les 3 (DSM): mu_sgs, k_sgs and tau_kk fields; T in prim[4] is the
// temperature of p - tau_kk / 2, rhoE that of p
// with walls (p.wall_mask), mu on wall points comes from Tmu: the temperature
// before the wall treatment, which preStepBCHandling leaves mu at
template <typename R>
int launch_flux(const Grid3 &g, const R *const prim[5], const R *const d[12], const Metrics<R> &m,
                const FluxParams &p, const R *mu_sgs, const R *k_sgs, const R *taukk, const R *Tmu,
                R *const F[15], cudaStream_t st);

template <typename R>
int launch_vreman(const Grid3 &g, const R *const prim[5], const R *const d[12], const Metrics<R> &m,
                  const FluxParams &p, R *mu_sgs, cudaStream_t st);

// RK register update for one stage: see rk.cu for the per-scheme formulas.
struct RkStage {
    int scheme;        // MC3D_* RK type
    int stage;         // 1-based
    int nstages;
    double a, b;       // scheme coefficients of this stage
    // last stage: leave out writes nothing reads after the step; bit 0 the
    // 2N register (the next step starts from q1, written by the filter or the
    // final-state copy), bit 1 the FP64 final state when the filter takes its
    // working-precision copy and no statistics read it
    int skip_last;
};
// prim (optional, may be null): also write rho, U, V, W, T of the new stage
// state, or with copy_final on the last stage the final state in R instead
template <typename R>
int launch_rk_update(const Grid3 &g, const RkStage &rs, const R *const k2[5], double *const q1[5],
                     double *const qk[5], double *const q2[5], R *const prim[5], cudaStream_t st,
                     bool copy_final = false);

template <typename R>
int launch_to_real(const Grid3 &g, const double *const src[5], R *const dst[5], cudaStream_t st);

// CFL: max over points of J11(|U|+c)/dxi + J22(|V|+c)/deta + J33(|W|+c)/dzeta into *umax
// (FP64, non-negative values compared as integers with atomicMax).
template <typename R>
int launch_cfl(const Grid3 &g, const double *const q[5], const Metrics<R> &m, const double dxi[3],
               unsigned long long *umax, cudaStream_t st);

// dt/time/timeStep bookkeeping of calcDtFromCFL (Core.cpp:189-237) on device.
struct TimeState {
    double dt, time, cfl_max;
    long long time_step;
    unsigned long long umax_bits;
    int nonfinite;
};
int launch_finalize_dt(TimeState *ts, int ts_type, double cfl, double dt_const, int first_step,
                       cudaStream_t st);

// ---- learned SGS closure (mlp.cu) --------------------------------------------
constexpr int MLP_IN = 9, MLP_OUT = 2;
constexpr int MLP_NPARAM = 9090;   // 9*64+64 + 2*(64*64+64) + 64*2+2
constexpr int MLPT_BYTES = 29696;  // weight image of the tensor-core inference (mlp_common.cuh)
// input normalisation x_n = (x - mean) * inv_std, and the training range [lo, hi]
struct MlpNorm {
    float mean[MLP_IN], inv_std[MLP_IN], lo[MLP_IN], hi[MLP_IN];
    float ymean[MLP_OUT], ystd[MLP_OUT];   // targets: y = out * ystd + ymean
};
struct MlpDev {
    float *P = nullptr, *G = nullptr, *M = nullptr, *V = nullptr;   // FP32 master, grads, Adam moments
    unsigned char *Tw = nullptr;   // BF16 weight image of the tensor-core inference (MLPT_BYTES)
    MlpNorm norm{};
    long long t = 0;                                                 // Adam step
};
int mlp_pack(const MlpDev &m, cudaStream_t st);
int mlp_forward_fp32(const MlpDev &m, const float *x, int n, float *act, float *out, cudaStream_t st);
// forward, backward and the weight gradients accumulated into m.G (no update)
int mlp_gradient(MlpDev &m, const float *x, const float *y, int n, float *act, float *out, float *delta,
                 double *loss, cudaStream_t st);
int mlp_train_step(MlpDev &m, const float *x, const float *y, int n, float lr, float *act, float *out, float *delta,
                   double *loss, cudaStream_t st);
// tensor-core inference of raw features x [n][9] -> raw outputs [n][2] (sgs_mlp.cu)
int mlp_infer_bf16(const MlpDev &m, const float *x, int n, float *out, cudaStream_t st);
// MMA completions that did not arrive within the wait limit (tensor-core inference)
int mlp_wait_timeouts(int *count);
const MlpDev *mlp_dev(mc3d_mlp m);
// fused closure in the time step: d[12] the xi-derivatives of U, V, W, T
template <typename R>
int launch_sgs_mlp(const Grid3 &g, const R *rho, const R *T, const R *const d[12], const Metrics<R> &m, double dvol,
                   double mu_ref, const MlpDev &mlp, R *mu_sgs, R *ksgs, int *flag, cudaStream_t st);
int launch_box_filter(const Grid3 &gf, int f, const double *const q[5], double *const out[14], cudaStream_t st);
int launch_training_pairs(const Grid3 &gc, const double *const coarse[14], const double *const grads[12],
                          const double jd[3], double delta, double mu_ref, float *x, float *y, cudaStream_t st);

// ---- boundary conditions (bc.cu) -------------------------------------------
// face: 0 X0, 1 X1, 2 Y0, 3 Y1, 4 Z0, 5 Z1
template <typename R>
int launch_wall_prestep(const Grid3 &g, int face, int neumann, int fd_type, double vt1, double vt2,
                        double *const q[5], R *const prim[5], cudaStream_t st);
// Tmu = T on the points of the faces in wall_mask
template <typename R>
int launch_wall_save_T(const Grid3 &g, int wall_mask, const R *T, R *Tmu, cudaStream_t st);
template <typename R>
int launch_face_k2(const Grid3 &g, int face, int wall, const R *cont, const R *J, R Jc, const double *dt,
                   R *const k2[5], cudaStream_t st);
template <typename R>
int launch_sponge_source(const Grid3 &g, const double *sigma, const double *const avg[5], const double *const q[5],
                         const R *J, R Jc, R *const rhs[5], cudaStream_t st);

// ---- dynamic Smagorinsky model and SGS averaging (dsm.cu) ---------------
template <typename R>
struct DsmPrepMu {
    const R *d[9];        // dU/dxi_d, dV/dxi_d, dW/dxi_d: d[3 * var + dir]
    const double *q[4];   // stage state rho, rhoU, rhoV, rhoW
    R *out[24];           // M_ij(2) x6, S_ij x6, |S|, rho, L_ij(t) x6, 2 rho |S|^2, rhoU, rhoV, rhoW
    R *smag;              // |S| kept for the later kernels
};
template <typename R>
struct DsmFinishMu {
    const R *hat[24];     // the test-filtered out[] of DsmPrepMu
    R *out[4];            // Lkk, C_I denominator, L_ij M_ij, M_ij M_ij
    int use_taukk;
};
template <typename R>
struct DsmMuTaukk {
    const double *q[5];
    const R *smag;
    const R *avg[4];      // averaged Lkk, C_I denominator, L_ij M_ij, M_ij M_ij
    int avg_scalar;       // 1: avg[k][0] holds the value of every point (the GLOBAL mean)
    R *mu_sgs, *taukk;
    R *T;                 // temperature of p - tau_kk / 2 (written in place)
    int use_taukk;
    // on the faces in cons_mask p is that of the primitives (rho_prim R T), not of q
    int cons_mask;
    const R *rho_prim;
};
template <typename R>
struct DsmPrepK {
    const R *dT[3];
    const double *q[4];
    const R *T, *smag;
    R *out[10];           // N_i(RHS) x3, rhoU_i T x3, rho T, gradT x3
};
template <typename R>
struct DsmFinishK {
    const R *hat[10];     // the test-filtered out[] of DsmPrepK
    const R *rho_hat, *smag_hat, *ru_hat[3];
    const double *q[4];
    R *out[2];            // N_i N_i, N_i K_i
};
template <typename R>
struct AvgBatch {
    int nf;
    const R *in[8];
    R *out[8];
};
template <typename R>
int launch_dsm_prep_mu(const Grid3 &g, const DsmPrepMu<R> &a, const Metrics<R> &m, cudaStream_t st);
template <typename R>
int launch_dsm_finish_mu(const Grid3 &g, const DsmFinishMu<R> &a, cudaStream_t st);
template <typename R>
int launch_dsm_mu_taukk(const Grid3 &g, const DsmMuTaukk<R> &a, cudaStream_t st);
template <typename R>
int launch_dsm_prep_k(const Grid3 &g, const DsmPrepK<R> &a, const Metrics<R> &m, cudaStream_t st);
template <typename R>
int launch_dsm_finish_k(const Grid3 &g, const DsmFinishK<R> &a, cudaStream_t st);
template <typename R>
int launch_dsm_ksgs(const Grid3 &g, const double *rho, const R *smag, const R *nini, const R *niki, R *ksgs,
                    int avg_scalar, cudaStream_t st);
// XI1/XI2/XI3 line means or the GLOBAL block mean of up to 8 fields (in may equal out);
// scratch holds the FP64 partial sums of GLOBAL
template <typename R>
// mean_only (GLOBAL): write the mean into element 0 of each output only
int launch_average(const Grid3 &g, int mode, const AvgBatch<R> &b, double *scratch, size_t scratch_doubles,
                   cudaStream_t st, bool mean_only = false);

int launch_integrals(const Grid3 &g, const double *const q[5], double *acc2, cudaStream_t st);
int launch_nonfinite_check(const Grid3 &g, const double *const q[5], int *flag, cudaStream_t st);

// ---- grid metrics (metrics.cu) -----------------------------------------------
// RHS of the reference's TPB derivative along `dir` (periodic lines whose
// stencil reads ghost values): row n = (sum_k st[k] F[n+k-H]) / dh with F the
// line values inside [0, N) and, outside, sum_t (X_t -+ T[t]) W_t at the wrapped
// index (N-m before the start, m-1 after the end; W_t == nullptr: 1). CD2
// (explicit_cd2) uses the reference's mirrored end rows. nm3_from_nm2: the
// Nm3 ghost is the Nm2 one.
struct TpbArgs {
    int N, H, nterms, explicit_cd2, nm3_from_nm2;
    double st[7];
    double dh;
    double T[3];
    const double *X[3];
    const double *W[3];
};
struct MetOut9 {
    double *p[9];
};
int launch_tpb_rhs(const Grid3 &g, int dir, const double *f, const TpbArgs &a, double *rhs, cudaStream_t st);

// TPB right-hand side from caller-supplied ghost planes (tpb.cu): G planes per
// side (p[0..G-1] = Nm_G..Nm_1, p[G..2G-1] = Np_1..Np_G), interior stencil
// st[0..2H] (explicit_cd2: the reference's CD2 end rows)
template <typename R>
struct TpbPlanes {
    const R *p[6];
    int G, H, explicit_cd2;
    double st[7];
};
template <typename R>
int launch_tpb_planes_rhs(const Grid3 &g, int dir, const R *f, const TpbPlanes<R> &gp, double dh, R *rhs,
                          cudaStream_t st);

// ---- running statistics (stats.cu) ------------------------------------------
struct StatsIn {
    const double *q[5];      // filtered conserved state (rho1 .. rhoE1)
    const double *rho2;      // density before the filter
};
struct StatsOut {
    double *p[9];
};
// One Stats::updateStatsFields with time increment dt and old weights ovw /
// otw: v = UAVG, VAVG, WAVG, URMS, VRMS, WRMS, UVREY, UWREY, VWREY; t = RHOAVG,
// RHORMS, PAVG, PRMS, TAVG, TRMS.
int launch_stats_update(const Grid3 &g, const StatsIn &in, double *const v[9], double *const t[6], double dt,
                        double ovw, double otw, int avg_type, int vel, int thermo, cudaStream_t st);

// updateSponge: relax the sponge target toward q, then set the SPONGE faces
// (bit f of sponge_faces: face X0, X1, Y0, Y1, Z0, Z1) to it
int launch_sponge_relax(const Grid3 &g, double *const q[5], double *const avg[5], const TimeState *ts, double avg_t,
                        double p_inf, int sponge_faces, cudaStream_t st);

// ---- diagnostic hooks of the reference drivers (hooks.cu) --------------------
constexpr int TURB_NSUM = 9;   // block sums of the HIT statistics, pass 1
// pass 1: sums of rho, mu, dissipation, |u|^2/3, (u_x^2+v_y^2+w_z^2)/3, |u|^2,
// c, u_x^2, rho |u|^2; pass 2: sums of (rho - mean_rho)^2, dil^2, |omega|^2.
// partial[k * nblocks + block]
template <typename R>
int launch_turb_sums(const Grid3 &g, const R *const prim[5], const R *const d[12], const Metrics<R> &m,
                     double mu_ref, int pass, double mean_rho, double *partial, int nblocks, cudaStream_t st);
// out[4][Nx]: span averages of p, U, V, W on the j = 0 face
int launch_wall_span_average(const Grid3 &g, const double *const q[5], double *out, cudaStream_t st);
int launch_wake_strip(const Grid3 &g, const double *const q[5], int i, int j, double *out, cudaStream_t st);

// CTAs of the TMA-staged line solves on the current device whose tile load
// did not arrive within the wait limit (their results are invalid)
int tma_wait_timeouts(int *count);

// ---- checkpoint files (checkpoint.cpp) ----------------------------------------
int write_solution_dump(const char *path, int time_step, double time, int Nx, int Ny, int Nz,
                        const double *const fields[8]);
int read_solution_header(const char *path, int *time_step, double *time, int *Nx, int *Ny, int *Nz);
int read_solution_fields(const char *path, long long n, double *const fields[8]);
int write_sponge_avg(const char *path, long long n, const double *const fields[5]);
int read_sponge_avg(const char *path, long long n, double *const fields[5]);
int launch_metric_mul(long long n, const double *a, const double *b, double *o, cudaStream_t st);
int launch_metric_sub(long long n, const double *a, const double *b, double *o, cudaStream_t st);
int launch_metric_dot3(long long n, const double *const xyz[3], const double *const abc[3], double *o,
                       cudaStream_t st);
int launch_metric_finish(long long n, const double *const jdet[3], double *const jij[9], double *J, cudaStream_t st);

}  // namespace mc3d
