// GPU CurvilinearCSolver: one block resident on one device, driven by the RK
// schemes of the reference. Host code only sequences kernels on one stream;
// dt, time and the time-step counter live on the device (FP64) so a step
// needs no host synchronisation.
//
// Stage data flow (per RK stage; every array is a full Nx*Ny*Nz field):
//   primitives(qP) -> U,V,W,T                           (Core.cpp:1158-1197)
//   3 sweeps: d/dxi_d of U,V,W,T -> 12 derivatives        (Core.cpp:239-348)
//   flux: gradU, Vreman, tau, q, 15 flux components       (Core.cpp:548-752)
//   (DSM: gradients of U,V,W; DSM mu_sgs/tau_kk with two test-filtered
//    batches; gradient of the tau_kk-corrected T; k_sgs; then the flux)
//   3 sweeps: -dF/dxi1, -dG/dxi2, -dH/dxi3 -> k2          (Core.cpp:350-466, 790-947)
//   RK register update                                    (RK4.hpp, LSLDDRK4.hpp, ...)
//   filter (last stage or every stage)                   (Core.cpp:949-1155)
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "mc3d_internal.h"

struct mc3d_solver_s {
    mc3d_config cfg;
    int device = 0;
    cudaStream_t stream = nullptr;
    mc3d::Grid3 g{};
    int prec = MC3D_FP64;
    double dxi[3] = {0, 0, 0};
    mc3d::LineOpBuf dop[3], fop[3], vop[3], top[3];   // derivative, filter, Vreman averaging, DSM test filter
    double *q1[5] = {}, *qk[5] = {}, *q2[5] = {};
    void *k2[5] = {}, *rhs[5] = {}, *prim[5] = {}, *der[12] = {}, *flux[15] = {};
    void *tA[5] = {}, *tB[5] = {}, *tC[5] = {}, *mu_sgs = nullptr;
    // DSM work fields: two banks of 24, |S|, tau_kk, k_sgs; FP64 partial sums of GLOBAL averaging
    void *dA[24] = {}, *dB[24] = {}, *smag = nullptr, *taukk = nullptr, *ksgs = nullptr;
    double *avg_scratch = nullptr;
    // sponge: strength and target state (FP64); walls present
    double *sigma = nullptr, *spg_avg[5] = {};
    bool have_sponge = false, have_walls = false, sigma_set = false;
    long long sponge_pts = 0;   // points with a nonzero sponge strength
    // walls: temperature that mu at wall points follows (set_initial fills it
    // with the initial temperature for the first stage; later stages save it
    // before the wall treatment)
    void *Tmu = nullptr;
    int wall_mask = 0;
    bool tmu_from_init = false;
    // learned closure (LESMODEL = MLP): the network, its out-of-range flag and the DSM fallbacks
    mc3d_mlp mlp = nullptr;
    int *mlp_flag = nullptr, *mlp_flag_host = nullptr;
    long long mlp_fallbacks = 0;
    double *met64[10] = {};
    void *metR[10] = {};
    bool const_met = true;
    double met_c[10] = {0};
    bool have_metrics = false;
    // the mesh behind the metrics, for SolutionDump files: coordinates given to
    // set_mesh / restart, or the box lengths of set_box_metrics
    std::vector<double> mesh_xyz[3];
    double box_L[3] = {0, 0, 0};
    int mesh_kind = 0;   // 0 none, 1 coordinates, 2 box
    mc3d::TimeState *ts = nullptr;
    double *acc = nullptr;
    int host_time_step = 0;
    int filter_time_step = 0;
    bool tc_fresh = false;   // tC holds the working-precision copy of the state the filter reads
    // prim and the CFL maximum already hold the primitives of the next step:
    // formed before a sponge relaxation changed rho1..rhoE1
    bool prims_ready = false;
    // faces whose conserved state the current stage takes in place of the
    // primitives' (set for stage 1 after a sponge relaxation)
    int cons_mask = 0;
    // running statistics (FP64): velocity (9) and thermodynamic (6) fields, their
    // time weights and the time of the last update
    double *stv[9] = {}, *stt[6] = {};
    double st_vw = 0.0, st_tw = 0.0, st_prev = 0.0;
    double *hook_scratch = nullptr;   // block partials of the diagnostic reductions
    int lsldd_half = 1;
    // GPU.STORAGE = LEAN: work arrays along xi1 / xi2 hold one slab of slab_nz
    // xi3-planes; q2 is qk for the 2N schemes; k2 accumulates the divergence
    bool lean = false;
    int slab_nz = 0;
    // stage-level driving (mc3d_solver_pre_step .. mc3d_solver_post_step): the
    // last call made in the current time step, its stage, the step's stage
    // count, whether it filters, and the sponge faces relaxed before it
    int phase = 0;
    int cur_stage = 0, cur_ns = 0, cur_relaxed = 0;
    bool cur_filter_now = false;
    long long stages = 0;
    long long launches = 0;
    bool initialized = false;
    std::vector<void *> allocs;
    // optional per-kernel-class CUDA-event timing (mc3d_solver_set_timing)
    bool timing = false;
    struct Rec { int cls; size_t ev; double bytes; };
    std::vector<cudaEvent_t> events;
    std::vector<Rec> recs;
    size_t ev_used = 0;
    std::string report;
};

namespace mc3d {

// FP64 partial sums of GLOBAL averaging: up to 148 x 4 blocks for up to 8 fields
constexpr size_t AVG_SCRATCH = 148 * 4 * 8;

// kernel classes for the optional event timing
enum KClass { KC_SWEEP = 0, KC_FLUX, KC_PRIM, KC_RK, KC_CFL, KC_TOREAL, KC_VREMAN, KC_SGS, KC_BC, KC_COUNT };
static const char *KC_NAME[KC_COUNT] = {"sweep_linesolve", "flux", "primitives", "rk_update", "cfl_dt", "to_fp32",
                                        "vreman", "sgs_pointwise", "boundary"};

static int tic(mc3d_solver s, int cls, double bytes) {
    if (!s->timing) return MC3D_OK;
    while (s->events.size() < s->ev_used + 2) {
        cudaEvent_t e;
        MC3D_CUDA_TRY(cudaEventCreate(&e));
        s->events.push_back(e);
    }
    MC3D_CUDA_TRY(cudaEventRecord(s->events[s->ev_used], s->stream));
    s->recs.push_back({cls, s->ev_used, bytes});
    s->ev_used += 2;
    return MC3D_OK;
}
static int toc(mc3d_solver s) {
    if (!s->timing) return MC3D_OK;
    MC3D_CUDA_TRY(cudaEventRecord(s->events[s->recs.back().ev + 1], s->stream));
    return MC3D_OK;
}

static const double RK4_A[4] = {1.0 / 6.0, 1.0 / 3.0, 1.0 / 3.0, 1.0 / 6.0};
static const double RK4_B[3] = {1.0 / 2.0, 1.0 / 2.0, 1.0};
// src/KenRK4.hpp:30-40
static const double KEN_A[5] = {0.0, -6234157559845.0 / 12983515589748.0, -6194124222391.0 / 4410992767914.0,
                                -31623096876824.0 / 15682348800105.0, -12251185447671.0 / 11596622555746.0};
static const double KEN_B[5] = {494393426753.0 / 4806282396855.0, 4047970641027.0 / 5463924506627.0,
                                9795748752853.0 / 13190207949281.0, 4009051133189.0 / 8539092990294.0,
                                1348533437543.0 / 7166442652324.0};
// src/LSLDDRK4.hpp:40-78
static const double LS_A1[5] = {0.0, -0.60512264332862261228, -2.04375640234761394333, -0.74069990637544192841,
                                -4.42317651302968168941};
static const double LS_B1[5] = {0.26874543888713438496, 0.8014706973220802933, 0.50515704269422722538,
                                0.56235680379000296407, 0.05900655127758823335};
static const double LS_A2[6] = {0.0, -0.44127377153877382565, -1.073982008079781868, -1.7063570791256758809,
                                -2.7979293162682443056, -4.0913537120919160454};
static const double LS_B2[6] = {0.11584888181285561688, 0.37287699051652864918, 0.73795368921435295698,
                                0.57981109366311039538, 1.031284991300145194, 0.15};

static int salloc(mc3d_solver s, void **p, size_t bytes) {
    cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaSuccess) return fail(MC3D_ERR_OOM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    s->allocs.push_back(*p);
    MC3D_CUDA_TRY(cudaMemsetAsync(*p, 0, bytes, s->stream));
    return MC3D_OK;
}

template <typename R>
static Metrics<R> metrics_of(mc3d_solver s) {
    Metrics<R> m;
    m.constant = s->const_met;
    for (int i = 0; i < 10; i++) {
        m.c[i] = (R)s->met_c[i];
        m.m[i] = s->const_met ? nullptr : (const R *)s->metR[i];
    }
    return m;
}

template <typename R>
static const LineOpDev<R> &opdev(const LineOpBuf &b);
template <>
const LineOpDev<float> &opdev<float>(const LineOpBuf &b) { return b.f32; }
template <>
const LineOpDev<double> &opdev<double>(const LineOpBuf &b) { return b.f64; }

template <typename R>
static int sweep_on(mc3d_solver s, const Grid3 &g, int dir, const LineOpBuf &op, int nf, const void *const *in,
                    void *const *out, int epi, const void *const *aux, double *const *out64, bool filter, bool quirk);

template <typename R>
static int sweep(mc3d_solver s, int dir, const LineOpBuf &op, int nf, const void *const *in, void *const *out,
                 int epi, const void *const *aux, double *const *out64, bool filter) {
    return sweep_on<R>(s, s->g, dir, op, nf, in, out, epi, aux, out64, filter, s->cfg.reference_quirks != 0);
}

// one batched line solve along dir over the block (or slab) g; `quirk` turns
// on the momentum k2 carry-over of the k2-assembly epilogue
template <typename R>
static int sweep_on(mc3d_solver s, const Grid3 &g, int dir, const LineOpBuf &op, int nf, const void *const *in,
                    void *const *out, int epi, const void *const *aux, double *const *out64, bool filter, bool quirk) {
    SweepBatch<R> b{};
    b.nf = nf;
    for (int f = 0; f < nf; f++) {
        b.in[f] = (const R *)in[f];
        b.out[f] = out ? (R *)out[f] : nullptr;
        b.aux[f] = aux ? (const R *)aux[f] : nullptr;
        b.out64[f] = out64 ? out64[f] : nullptr;
        b.eq[f] = f;
    }
    RhsFinalArgs<R> rf{};
    rf.dt = &s->ts->dt;
    rf.J = s->const_met ? nullptr : (const R *)s->metR[0];
    rf.Jc = (R)s->met_c[0];
    rf.quirk = quirk;
    s->launches++;
    // algorithmic bytes: every field read once and written once, plus the
    // epilogue's extra operands (partial RHS, previous k2, FP64 store)
    double per = 2.0 * sizeof(R);
    if (epi == EPI_SUB) per = 3.0 * sizeof(R);
    if (epi == EPI_STORE_F64) per = sizeof(R) + 8.0;
    double bytes = per * nf * (double)g.n();
    if (epi == EPI_RHS_FINAL) bytes = (3.0 * nf + (quirk ? 3.0 : 0.0)) * sizeof(R) * (double)g.n();
    int rc = tic(s, KC_SWEEP, bytes);
    if (rc) return rc;
    rc = launch_sweep<R>(dir, g, opdev<R>(op), b, epi, rf, s->cfg.bc_type, filter, s->stream);
    if (rc) return rc;
    return toc(s);
}

// Three directional filter sweeps in the rotating order of
// filterConservedData (Core.cpp:996-1134): filterTimeStep%3 == 1: Y,Z,X;
// == 2: Z,X,Y; == 0: X,Y,Z. in -> out (both FP64 state arrays).
template <typename R>
static int filter_state(mc3d_solver s, double *const in[5], double *const out[5], const LineOpBuf *ops,
                        const int order[3]) {
    int rc;
    void *src0[5];
    if (s->prec == MC3D_FP64) {
        for (int v = 0; v < 5; v++) src0[v] = in[v];
    } else {
        // the last RK stage of a filtered step already wrote the copy
        if (!s->tc_fresh) {
            R *dst[5];
            for (int v = 0; v < 5; v++) dst[v] = (R *)s->tC[v];
            s->launches++;
            if ((rc = tic(s, KC_TOREAL, (8.0 + sizeof(R)) * 5 * (double)s->g.n()))) return rc;
            if ((rc = launch_to_real<R>(s->g, in, dst, s->stream))) return rc;
            if ((rc = toc(s))) return rc;
        }
        s->tc_fresh = false;
        for (int v = 0; v < 5; v++) src0[v] = s->tC[v];
    }
    if ((rc = sweep<R>(s, order[0], ops[order[0]], 5, src0, s->tA, EPI_STORE, nullptr, nullptr, true))) return rc;
    if ((rc = sweep<R>(s, order[1], ops[order[1]], 5, s->tA, s->tB, EPI_STORE, nullptr, nullptr, true))) return rc;
    if (s->prec == MC3D_FP64) {
        void *o[5];
        for (int v = 0; v < 5; v++) o[v] = out[v];
        return sweep<R>(s, order[2], ops[order[2]], 5, s->tB, o, EPI_STORE, nullptr, nullptr, true);
    }
    return sweep<R>(s, order[2], ops[order[2]], 5, s->tB, nullptr, EPI_STORE_F64, nullptr, out, true);
}

// filterConservedData with LEAN storage: one conserved field at a time through
// two full work fields (the xi3-flux fields, free once k2 is assembled)
template <typename R>
static int filter_state_lean(mc3d_solver s, double *const in[5], double *const out[5], const int order[3]) {
    int rc;
    void *t0 = s->tA[0], *t1 = s->tB[0];
    for (int v = 0; v < 5; v++) {
        void *a[1], *b[1] = {t1};
        if (s->prec == MC3D_FP64) {
            a[0] = in[v];
        } else {
            const double *src[5] = {in[v], in[v], in[v], in[v], in[v]};
            R *dst[5] = {(R *)t0, nullptr, nullptr, nullptr, nullptr};
            s->launches++;
            if ((rc = tic(s, KC_TOREAL, (8.0 + sizeof(R)) * (double)s->g.n()))) return rc;
            if ((rc = launch_to_real<R>(s->g, src, dst, s->stream))) return rc;
            if ((rc = toc(s))) return rc;
            a[0] = t0;
        }
        if ((rc = sweep<R>(s, order[0], s->fop[order[0]], 1, a, b, EPI_STORE, nullptr, nullptr, true))) return rc;
        void *c[1] = {t0};
        if ((rc = sweep<R>(s, order[1], s->fop[order[1]], 1, b, c, EPI_STORE, nullptr, nullptr, true))) return rc;
        if (s->prec == MC3D_FP64) {
            void *o[1] = {out[v]};
            if ((rc = sweep<R>(s, order[2], s->fop[order[2]], 1, c, o, EPI_STORE, nullptr, nullptr, true))) return rc;
        } else {
            double *o64[1] = {out[v]};
            if ((rc = sweep<R>(s, order[2], s->fop[order[2]], 1, c, nullptr, EPI_STORE_F64, nullptr, o64, true)))
                return rc;
        }
    }
    return MC3D_OK;
}

template <typename R>
static int filter_conserved(mc3d_solver s, bool last) {
    double **in = last ? s->q2 : s->qk;
    double **out = last ? s->q1 : s->qk;
    if (s->host_time_step % s->cfg.filter_step == 0) {
        s->filter_time_step++;
        int r = s->filter_time_step % 3;
        int order[3];
        if (r == 1) { order[0] = 1; order[1] = 2; order[2] = 0; }
        else if (r == 2) { order[0] = 2; order[1] = 0; order[2] = 1; }
        else { order[0] = 0; order[1] = 1; order[2] = 2; }
        if (s->lean) return filter_state_lean<R>(s, in, out, order);
        return filter_state<R>(s, in, out, s->fop, order);
    }
    if (last) {
        size_t bytes = (size_t)s->g.n() * sizeof(double);
        for (int v = 0; v < 5; v++)
            MC3D_CUDA_TRY(cudaMemcpyAsync(s->q1[v], s->q2[v], bytes, cudaMemcpyDeviceToDevice, s->stream));
    }
    return MC3D_OK;
}

// rho, U, V, W, T of `q` into s->prim (updateNonConservedData, Core.cpp:1158-1197)
template <typename R>
static int primitives(mc3d_solver s, double *const q[5]) {
    int rc;
    R *prim[5];
    for (int v = 0; v < 5; v++) prim[v] = (R *)s->prim[v];
    s->launches++;
    if ((rc = tic(s, KC_PRIM, (5.0 * 8 + 5.0 * sizeof(R)) * (double)s->g.n()))) return rc;
    if ((rc = launch_primitives<R>(s->g, q, prim, s->stream))) return rc;
    return toc(s);
}

static bool is_wall_kind(int k) {
    return k == MC3D_BC_ADIABATIC_WALL || k == MC3D_BC_CONST_T_WALL || k == MC3D_BC_MOVING_ADIABATIC_WALL;
}

// preStepBCHandling (src/CurvilinearCSolver_BC.cpp:372-700) on the stage
// state qP and its primitives: no-slip walls of all faces X0..Z1 first, then
// the moving walls.
template <typename R>
static int wall_prestep(mc3d_solver s, double *const *qP) {
    if (!s->have_walls) return MC3D_OK;
    int rc;
    R *pr[5];
    for (int v = 0; v < 5; v++) pr[v] = (R *)s->prim[v];
    // mu keeps updateNonConservedData's value on the walls: keep that temperature
    if (!s->tmu_from_init) {
        s->launches += 6;
        if ((rc = launch_wall_save_T<R>(s->g, s->wall_mask, pr[4], (R *)s->Tmu, s->stream))) return rc;
    }
    s->tmu_from_init = false;
    for (int pass = 0; pass < 2; pass++)
        for (int f = 0; f < 6; f++) {
            const int k = s->cfg.bc_kind[f];
            const bool noslip = k == MC3D_BC_ADIABATIC_WALL || k == MC3D_BC_CONST_T_WALL;
            if (pass == 0 ? !noslip : k != MC3D_BC_MOVING_ADIABATIC_WALL) continue;
            const int neumann = k != MC3D_BC_CONST_T_WALL;
            const double *vt = s->cfg.wall_velocity[f];
            s->launches++;
            if ((rc = tic(s, KC_BC, 0.0))) return rc;
            if ((rc = launch_wall_prestep<R>(s->g, f, neumann, s->cfg.fd_type[f >> 1], pass ? vt[0] : 0.0,
                                             pass ? vt[1] : 0.0, qP, pr, s->stream)))
                return rc;
            if ((rc = toc(s))) return rc;
        }
    return MC3D_OK;
}

// postStepBCHandling (src/CurvilinearCSolver_BC.cpp:702-842): wall faces keep
// -dt J dF_mass/dxi_d in the continuity k2, sponge faces zero the k2 entirely.
template <typename R>
static int face_poststep(mc3d_solver s) {
    int rc;
    R *k2[5];
    for (int v = 0; v < 5; v++) k2[v] = (R *)s->k2[v];
    const R *J = s->const_met ? nullptr : (const R *)s->metR[0];
    for (int pass = 0; pass < 2; pass++)
        for (int f = 0; f < 6; f++) {
            const int k = s->cfg.bc_kind[f];
            if (pass == 0 ? !is_wall_kind(k) : k != MC3D_BC_SPONGE) continue;
            s->launches++;
            if ((rc = tic(s, KC_BC, 0.0))) return rc;
            if ((rc = launch_face_k2<R>(s->g, f, pass == 0, (const R *)s->tB[f >> 1], J, (R)s->met_c[0], &s->ts->dt,
                                        k2, s->stream)))
                return rc;
            if ((rc = toc(s))) return rc;
        }
    return MC3D_OK;
}

// Test-filter sweeps of nf fields along Y, Z, X (DSMSGS::filterQuantity,
// src/DSMSGS.hpp:120-128) in batches of at most 16: in -> tmp -> in -> tmp, so
// the filtered fields end in tmp and in is overwritten.
template <typename R>
static int test_filter3(mc3d_solver s, int nf, void *const *in, void *const *tmp) {
    int rc;
    for (int b0 = 0; b0 < nf; b0 += 16) {
        const int nb = std::min(16, nf - b0);
        if ((rc = sweep<R>(s, 1, s->top[1], nb, in + b0, tmp + b0, EPI_STORE, nullptr, nullptr, true))) return rc;
        if ((rc = sweep<R>(s, 2, s->top[2], nb, tmp + b0, in + b0, EPI_STORE, nullptr, nullptr, true))) return rc;
        if ((rc = sweep<R>(s, 0, s->top[0], nb, in + b0, tmp + b0, EPI_STORE, nullptr, nullptr, true))) return rc;
    }
    return MC3D_OK;
}

// AbstractSGS::doAveraging (src/AbstractSGS.cpp:13-160) of nf fields f[]:
// LOCAL filters them along Y, Z, X with `ops` (f -> t -> f -> t: the result is
// in t); XI1/XI2/XI3/GLOBAL average in place; NONE leaves them. Returns the
// arrays that hold the result in res[].
template <typename R>
// scalar (optional): the caller reads element 0 of each result for every
// point, so GLOBAL averaging writes the mean there only (*scalar = 1)
static int sgs_average(mc3d_solver s, int nf, void *const *f, void *const *t, const LineOpBuf *ops, void **res,
                       int *scalar = nullptr) {
    int rc;
    const int mode = s->cfg.les_averaging;
    const bool mean_only = scalar && mode == MC3D_AVG_GLOBAL;
    if (scalar) *scalar = mean_only ? 1 : 0;
    for (int i = 0; i < nf; i++) res[i] = f[i];
    if (mode == MC3D_AVG_NONE) return MC3D_OK;
    if (mode == MC3D_AVG_LOCAL) {
        if ((rc = sweep<R>(s, 1, ops[1], nf, f, t, EPI_STORE, nullptr, nullptr, true))) return rc;
        if ((rc = sweep<R>(s, 2, ops[2], nf, t, f, EPI_STORE, nullptr, nullptr, true))) return rc;
        if ((rc = sweep<R>(s, 0, ops[0], nf, f, t, EPI_STORE, nullptr, nullptr, true))) return rc;
        for (int i = 0; i < nf; i++) res[i] = t[i];
        return MC3D_OK;
    }
    AvgBatch<R> b{};
    b.nf = nf;
    for (int i = 0; i < nf; i++) {
        b.in[i] = (const R *)f[i];
        b.out[i] = (R *)f[i];
    }
    s->launches += mode == MC3D_AVG_GLOBAL ? 2 : 1;
    if ((rc = tic(s, KC_SGS, (mean_only ? 1.0 : 2.0) * nf * sizeof(R) * (double)s->g.n()))) return rc;
    if ((rc = launch_average<R>(s->g, mode, b, s->avg_scratch, AVG_SCRATCH, s->stream, mean_only))) return rc;
    return toc(s);
}

// DSMSGS::calcMuSGSTaukk (src/DSMSGS.hpp:130-331) on the stage state qP, then
// p -= tau_kk / 2 and T of that pressure into prim[4] (Core.cpp:567-585).
template <typename R>
static int dsm_mu_taukk(mc3d_solver s, double *const *qP, const Metrics<R> &m) {
    int rc;
    const double n = (double)s->g.n();
    DsmPrepMu<R> a{};
    for (int i = 0; i < 9; i++) a.d[i] = (const R *)s->der[i];
    for (int v = 0; v < 4; v++) a.q[v] = qP[v];
    for (int i = 0; i < 24; i++) a.out[i] = (R *)s->dA[i];
    a.smag = (R *)s->smag;
    s->launches++;
    if ((rc = tic(s, KC_SGS, (9.0 * sizeof(R) + 4.0 * 8 + 25.0 * sizeof(R)) * n))) return rc;
    if ((rc = launch_dsm_prep_mu<R>(s->g, a, m, s->stream))) return rc;
    if ((rc = toc(s))) return rc;
    if ((rc = test_filter3<R>(s, 24, s->dA, s->dB))) return rc;   // filtered fields in dB
    DsmFinishMu<R> fm{};
    for (int i = 0; i < 24; i++) fm.hat[i] = (const R *)s->dB[i];
    for (int i = 0; i < 4; i++) fm.out[i] = (R *)s->dA[i];
    fm.use_taukk = s->cfg.dsm_use_taukk;
    s->launches++;
    if ((rc = tic(s, KC_SGS, 28.0 * sizeof(R) * n))) return rc;
    if ((rc = launch_dsm_finish_mu<R>(s->g, fm, s->stream))) return rc;
    if ((rc = toc(s))) return rc;
    void *avg[4];
    int avg_scalar = 0;
    if ((rc = sgs_average<R>(s, 4, s->dA, s->dA + 4, s->top, avg, &avg_scalar))) return rc;
    DsmMuTaukk<R> mt{};
    for (int v = 0; v < 5; v++) mt.q[v] = qP[v];
    mt.smag = (const R *)s->smag;
    for (int i = 0; i < 4; i++) mt.avg[i] = (const R *)avg[i];
    mt.avg_scalar = avg_scalar;
    mt.mu_sgs = (R *)s->mu_sgs;
    mt.taukk = (R *)s->taukk;
    mt.T = (R *)s->prim[4];
    mt.use_taukk = s->cfg.dsm_use_taukk;
    mt.cons_mask = s->cons_mask;
    mt.rho_prim = (const R *)s->prim[0];
    s->launches++;
    if ((rc = tic(s, KC_SGS, (5.0 * 8 + (avg_scalar ? 4.0 : 8.0) * sizeof(R)) * n))) return rc;
    if ((rc = launch_dsm_mu_taukk<R>(s->g, mt, s->stream))) return rc;
    return toc(s);
}

// DSMSGS::calcKSGS (src/DSMSGS.hpp:333-443) with gradT of the corrected T.
template <typename R>
static int dsm_ksgs(mc3d_solver s, double *const *qP, const Metrics<R> &m) {
    int rc;
    const double n = (double)s->g.n();
    DsmPrepK<R> a{};
    for (int i = 0; i < 3; i++) a.dT[i] = (const R *)s->der[9 + i];
    for (int v = 0; v < 4; v++) a.q[v] = qP[v];
    a.T = (const R *)s->prim[4];
    a.smag = (const R *)s->smag;
    for (int i = 0; i < 10; i++) a.out[i] = (R *)s->dA[i];
    s->launches++;
    if ((rc = tic(s, KC_SGS, (5.0 * sizeof(R) + 4.0 * 8 + 10.0 * sizeof(R)) * n))) return rc;
    if ((rc = launch_dsm_prep_k<R>(s->g, a, m, s->stream))) return rc;
    if ((rc = toc(s))) return rc;
    if ((rc = test_filter3<R>(s, 10, s->dA, s->dA + 10))) return rc;   // filtered fields in dA[10..19]
    DsmFinishK<R> fk{};
    for (int i = 0; i < 10; i++) fk.hat[i] = (const R *)s->dA[10 + i];
    fk.smag_hat = (const R *)s->dB[12];
    fk.rho_hat = (const R *)s->dB[13];
    for (int i = 0; i < 3; i++) fk.ru_hat[i] = (const R *)s->dB[21 + i];
    for (int v = 0; v < 4; v++) fk.q[v] = qP[v];
    fk.out[0] = (R *)s->dA[0];
    fk.out[1] = (R *)s->dA[1];
    s->launches++;
    if ((rc = tic(s, KC_SGS, (15.0 * sizeof(R) + 8.0 + 2.0 * sizeof(R)) * n))) return rc;
    if ((rc = launch_dsm_finish_k<R>(s->g, fk, s->stream))) return rc;
    if ((rc = toc(s))) return rc;
    void *avg[2];
    int avg_scalar = 0;
    if ((rc = sgs_average<R>(s, 2, s->dA, s->dA + 2, s->top, avg, &avg_scalar))) return rc;
    s->launches++;
    if ((rc = tic(s, KC_SGS, (8.0 + (avg_scalar ? 2.0 : 4.0) * sizeof(R)) * n))) return rc;
    if ((rc = launch_dsm_ksgs<R>(s->g, qP[0], (const R *)s->smag, (const R *)avg[0], (const R *)avg[1],
                                 (R *)s->ksgs, avg_scalar, s->stream)))
        return rc;
    return toc(s);
}

// preStepDerivatives and the first two divergence sweeps of one stage
// (Core.cpp:468-787, the RHS up to the last direction); s->prim holds rho, U,
// V, W, T of the stage state qP.
template <typename R>
static int stage_rhs(mc3d_solver s, double *const *qP) {
    int rc;
    bool dsm = s->cfg.les_model == MC3D_DSM;
    // gradients of U, V, W, T in each direction: der[3*var + dir]; with DSM
    // the T gradient waits for the tau_kk correction of T
    for (int d = 0; d < 3; d++) {
        void *out[4] = {s->der[0 + d], s->der[3 + d], s->der[6 + d], s->der[9 + d]};
        if ((rc = sweep<R>(s, d, s->dop[d], dsm ? 3 : 4, s->prim + 1, out, EPI_STORE, nullptr, nullptr, false)))
            return rc;
    }
    const R *pr[5];
    for (int v = 0; v < 5; v++) pr[v] = (const R *)s->prim[v];
    Metrics<R> m = metrics_of<R>(s);
    FluxParams fp{};
    fp.mu_ref = s->cfg.mu_ref;
    for (int i = 0; i < 3; i++) fp.dxi[i] = s->dxi[i];
    fp.pr_t = 0.9;   // src/CurvilinearCSolver.hpp:232
    fp.les = 0;
    fp.wall_mask = s->wall_mask;
    fp.cons_mask = s->cons_mask;
    for (int v = 0; v < 5; v++) fp.cons[v] = qP[v];
    const R *dd[12];
    for (int i = 0; i < 12; i++) dd[i] = (const R *)s->der[i];
    const R *mu_sgs = (const R *)s->mu_sgs;
    if (s->cfg.les_model == MC3D_VREMAN) {
        if (s->cfg.les_averaging == MC3D_AVG_NONE) {
            fp.les = 1;
        } else {
            // mu_sgs, then doAveraging with Compact10(-0.49) filters (VremanSGS.hpp:38-40)
            s->launches++;
            if ((rc = tic(s, KC_VREMAN, 11.0 * sizeof(R) * (double)s->g.n()))) return rc;
            if ((rc = launch_vreman<R>(s->g, pr, dd, m, fp, (R *)s->mu_sgs, s->stream))) return rc;
            if ((rc = toc(s))) return rc;
            void *a[1] = {s->mu_sgs}, *t1[1] = {s->tA[0]}, *res[1];
            if ((rc = sgs_average<R>(s, 1, a, t1, s->vop, res))) return rc;
            mu_sgs = (const R *)res[0];
            fp.les = 2;
        }
    } else if (s->cfg.les_model == MC3D_MLPSGS) {
        // learned closure; the stage goes to DSM when more than mlp_fallback_frac
        // of the points have a feature outside the training range
        MC3D_CUDA_TRY(cudaMemsetAsync(s->mlp_flag, 0, sizeof(int), s->stream));
        s->launches++;
        if ((rc = tic(s, KC_SGS, (14.0 + 2.0) * sizeof(R) * (double)s->g.n()))) return rc;
        if ((rc = launch_sgs_mlp<R>(s->g, pr[0], pr[4], dd, m, s->dxi[0] * s->dxi[1] * s->dxi[2], s->cfg.mu_ref,
                                    *mlp_dev(s->mlp), (R *)s->mu_sgs, (R *)s->ksgs, s->mlp_flag, s->stream)))
            return rc;
        if ((rc = toc(s))) return rc;
        MC3D_CUDA_TRY(cudaMemcpyAsync(s->mlp_flag_host, s->mlp_flag, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
        MC3D_CUDA_TRY(cudaStreamSynchronize(s->stream));
        if ((double)*s->mlp_flag_host > s->cfg.mlp_fallback_frac * (double)s->g.n()) {
            s->mlp_fallbacks++;
            dsm = true;
        } else {
            fp.les = 3;   // mu_sgs and k_sgs fields, no tau_kk
        }
    }
    if (dsm) {
        if ((rc = dsm_mu_taukk<R>(s, qP, m))) return rc;
        for (int d = 0; d < 3; d++) {
            void *in[1] = {s->prim[4]}, *out[1] = {s->der[9 + d]};
            if ((rc = sweep<R>(s, d, s->dop[d], 1, in, out, EPI_STORE, nullptr, nullptr, false))) return rc;
        }
        if ((rc = dsm_ksgs<R>(s, qP, m))) return rc;
        fp.les = 3;
    }
    R *F[15];
    for (int i = 0; i < 15; i++) F[i] = (R *)s->flux[i];
    s->launches++;
    {
        double b = (5.0 + 12.0 + 15.0) * sizeof(R) + (fp.les >= 2 ? sizeof(R) : 0) + (fp.les == 3 ? 2.0 * sizeof(R) : 0) +
                   (s->const_met ? 0 : 10.0 * sizeof(R));
        if ((rc = tic(s, KC_FLUX, b * (double)s->g.n()))) return rc;
    }
    if ((rc = launch_flux<R>(s->g, pr, dd, m, fp, mu_sgs, (const R *)s->ksgs, dsm ? (const R *)s->taukk : nullptr,
                             (const R *)s->Tmu, F, s->stream)))
        return rc;
    if ((rc = toc(s))) return rc;
    // divergence of the contravariant fluxes, accumulated into the RHS, then k2
    if ((rc = sweep<R>(s, 0, s->dop[0], 5, s->flux + 0, s->rhs, EPI_STORE_NEG, nullptr, nullptr, false))) return rc;
    if ((rc = sweep<R>(s, 1, s->dop[1], 5, s->flux + 5, s->rhs, EPI_SUB, nullptr, nullptr, false))) return rc;
    if (s->have_sponge) {
        R *rh[5];
        const double *qc[5], *ac[5];
        for (int v = 0; v < 5; v++) {
            rh[v] = (R *)s->rhs[v];
            qc[v] = qP[v];
            ac[v] = s->spg_avg[v];
        }
        s->launches++;
        // sigma everywhere; state, target, right-hand side (and J) where sigma is nonzero
        const double per_pt = 10.0 * 8 + 10.0 * sizeof(R) + (s->const_met ? 0.0 : sizeof(R));
        if ((rc = tic(s, KC_BC, 8.0 * (double)s->g.n() + per_pt * (double)s->sponge_pts))) return rc;
        if ((rc = launch_sponge_source<R>(s->g, s->sigma, ac, qc, s->const_met ? nullptr : (const R *)s->metR[0],
                                          (R)s->met_c[0], rh, s->stream)))
            return rc;
        if ((rc = toc(s))) return rc;
    }
    return MC3D_OK;
}

// preStepDerivatives and the first two divergence sweeps with LEAN storage.
// The xi3-derivatives of U, V, W, T are formed over the whole block; then,
// slab by slab of xi3-planes, the xi1- and xi2-derivatives, the SGS closure,
// the 15 fluxes (the xi3-fluxes into their full fields) and the xi1- and
// xi2-divergences, accumulated straight into k2. With the momentum carry-over
// (Core.cpp:839,872,904) the momentum k2 starts from its previous value, so
// k2 ends as (k2_prev + RHS) dt J there and RHS dt J elsewhere, as in
// solveXMomentum etc.
template <typename R>
static int stage_rhs_lean(mc3d_solver s, double *const *qP) {
    if (!s->const_met) return fail(MC3D_ERR_CONFIG, "GPU.STORAGE = LEAN needs constant metrics (a uniform box)");
    int rc;
    const Grid3 G = s->g;
    const size_t plane = (size_t)G.Nx * G.Ny;
    {
        void *out[4] = {s->der[2], s->der[5], s->der[8], s->der[11]};
        if ((rc = sweep<R>(s, 2, s->dop[2], 4, s->prim + 1, out, EPI_STORE, nullptr, nullptr, false))) return rc;
    }
    const Metrics<R> m = metrics_of<R>(s);
    FluxParams fp{};
    fp.mu_ref = s->cfg.mu_ref;
    for (int i = 0; i < 3; i++) fp.dxi[i] = s->dxi[i];
    fp.pr_t = 0.9;   // src/CurvilinearCSolver.hpp:232
    const bool mlp = s->cfg.les_model == MC3D_MLPSGS;
    fp.les = s->cfg.les_model == MC3D_VREMAN ? 1 : (mlp ? 3 : 0);
    if (mlp) MC3D_CUDA_TRY(cudaMemsetAsync(s->mlp_flag, 0, sizeof(int), s->stream));
    const bool quirk = s->cfg.reference_quirks != 0;
    for (int k0 = 0; k0 < G.Nz; k0 += s->slab_nz) {
        const int nz = std::min(s->slab_nz, G.Nz - k0);
        const Grid3 gs{G.Nx, G.Ny, nz};
        const size_t off = (size_t)k0 * plane;
        void *pr[5], *k2s[5];
        for (int v = 0; v < 5; v++) {
            pr[v] = (R *)s->prim[v] + off;
            k2s[v] = (R *)s->k2[v] + off;
            fp.cons[v] = qP[v] + off;
        }
        for (int d = 0; d < 2; d++) {
            void *out[4] = {s->der[0 + d], s->der[3 + d], s->der[6 + d], s->der[9 + d]};
            if ((rc = sweep_on<R>(s, gs, d, s->dop[d], 4, pr + 1, out, EPI_STORE, nullptr, nullptr, false, quirk)))
                return rc;
        }
        const R *dd[12], *prc[5];
        for (int var = 0; var < 4; var++) {
            dd[3 * var + 0] = (const R *)s->der[3 * var + 0];
            dd[3 * var + 1] = (const R *)s->der[3 * var + 1];
            dd[3 * var + 2] = (const R *)s->der[3 * var + 2] + off;
        }
        for (int v = 0; v < 5; v++) prc[v] = (const R *)pr[v];
        if (mlp) {
            s->launches++;
            if ((rc = tic(s, KC_SGS, (14.0 + 2.0) * sizeof(R) * (double)gs.n()))) return rc;
            if ((rc = launch_sgs_mlp<R>(gs, prc[0], prc[4], dd, m, s->dxi[0] * s->dxi[1] * s->dxi[2], s->cfg.mu_ref,
                                        *mlp_dev(s->mlp), (R *)s->mu_sgs, (R *)s->ksgs, s->mlp_flag, s->stream)))
                return rc;
            if ((rc = toc(s))) return rc;
        }
        R *F[15];
        for (int i = 0; i < 10; i++) F[i] = (R *)s->flux[i];
        for (int i = 10; i < 15; i++) F[i] = (R *)s->flux[i] + off;
        s->launches++;
        {
            const double b = (5.0 + 12.0 + 15.0) * sizeof(R) + (mlp ? 2.0 * sizeof(R) : 0.0);
            if ((rc = tic(s, KC_FLUX, b * (double)gs.n()))) return rc;
        }
        if ((rc = launch_flux<R>(gs, prc, dd, m, fp, (const R *)s->mu_sgs, (const R *)s->ksgs, nullptr, nullptr, F,
                                 s->stream)))
            return rc;
        if ((rc = toc(s))) return rc;
        void *fx[5] = {F[0], F[1], F[2], F[3], F[4]}, *fy[5] = {F[5], F[6], F[7], F[8], F[9]};
        if (quirk) {
            void *ince[2] = {fx[0], fx[4]}, *outce[2] = {k2s[0], k2s[4]};
            if ((rc = sweep_on<R>(s, gs, 0, s->dop[0], 2, ince, outce, EPI_STORE_NEG, nullptr, nullptr, false, quirk)))
                return rc;
            if ((rc = sweep_on<R>(s, gs, 0, s->dop[0], 3, fx + 1, k2s + 1, EPI_SUB, nullptr, nullptr, false, quirk)))
                return rc;
        } else if ((rc = sweep_on<R>(s, gs, 0, s->dop[0], 5, fx, k2s, EPI_STORE_NEG, nullptr, nullptr, false, quirk))) {
            return rc;
        }
        if ((rc = sweep_on<R>(s, gs, 1, s->dop[1], 5, fy, k2s, EPI_SUB, nullptr, nullptr, false, quirk))) return rc;
    }
    if (mlp) {
        // no DSM fallback with LEAN storage: such stages are counted
        MC3D_CUDA_TRY(cudaMemcpyAsync(s->mlp_flag_host, s->mlp_flag, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
        MC3D_CUDA_TRY(cudaStreamSynchronize(s->stream));
        if ((double)*s->mlp_flag_host > s->cfg.mlp_fallback_frac * (double)s->g.n()) s->mlp_fallbacks++;
    }
    return MC3D_OK;
}

// solveContinuity .. solveEnergy (Core.cpp:790-947): the third divergence
// sweep assembles k2 = dt J (partial RHS - dH/dxi3) in its epilogue (LEAN:
// k2 holds the partial RHS itself, and the assembly runs in place)
template <typename R>
static int stage_solve(mc3d_solver s) {
    if (s->lean)
        return sweep_on<R>(s, s->g, 2, s->dop[2], 5, s->flux + 10, s->k2, EPI_RHS_FINAL, s->k2, nullptr, false, false);
    return sweep<R>(s, 2, s->dop[2], 5, s->flux + 10, s->k2, EPI_RHS_FINAL, s->rhs, nullptr, false);
}

// postStepBCHandling (src/CurvilinearCSolver_BC.cpp:702-842) on k2
template <typename R>
static int stage_post(mc3d_solver s) {
    if (!s->have_walls && !s->have_sponge) return MC3D_OK;
    int rc;
    // wall faces need the wall-normal derivative of the mass flux alone
    for (int d = 0; d < 3; d++) {
        if (!is_wall_kind(s->cfg.bc_kind[2 * d]) && !is_wall_kind(s->cfg.bc_kind[2 * d + 1])) continue;
        void *in[1] = {s->flux[5 * d]}, *out[1] = {s->tB[d]};
        if ((rc = sweep<R>(s, d, s->dop[d], 1, in, out, EPI_STORE, nullptr, nullptr, false))) return rc;
    }
    return face_poststep<R>(s);
}

// MC3D_ERR_TIMEOUT when a line-solve tile load or a tensor-core MMA of the
// learned closure gave up waiting on this device
static int tma_timeouts_failed(mc3d_solver s) {
    (void)s;
    int n = 0, nm = 0;
    if (int rc = tma_wait_timeouts(&n)) return rc;
    if (n) return fail(MC3D_ERR_TIMEOUT, "a line-solve tile load did not arrive within the wait limit");
    if (int rc = mlp_wait_timeouts(&nm)) return rc;
    return nm ? fail(MC3D_ERR_TIMEOUT, "a tensor-core MMA of the learned closure did not complete within the wait limit")
              : MC3D_OK;
}

// bit f: face f is a SPONGE
static int sponge_faces(mc3d_solver s) {
    int faces = 0;
    for (int f = 0; f < 6; f++)
        if (s->cfg.bc_kind[f] == MC3D_BC_SPONGE) faces |= 1 << f;
    return faces;
}

// primitives of rho1..rhoE1 (updateNonConservedData, Core.cpp:1165-1177) and
// the CFL maximum over them, which calcDtFromCFL (Core.cpp:189-237) reads
template <typename R>
static int primitives_cfl(mc3d_solver s) {
    R *prim[5];
    for (int v = 0; v < 5; v++) prim[v] = (R *)s->prim[v];
    s->launches++;
    int rc;
    if ((rc = tic(s, KC_PRIM, (5.0 * 8 + 5.0 * sizeof(R)) * (double)s->g.n()))) return rc;
    if ((rc = launch_primitives_cfl<R>(s->g, s->q1, prim, metrics_of<R>(s), s->dxi, &s->ts->umax_bits, s->stream)))
        return rc;
    return toc(s);
}

static int stages_of(mc3d_solver s) {
    const int scheme = s->cfg.rk_type;
    return scheme == MC3D_RK4 ? 4 : scheme == MC3D_TVDRK3 ? 3 : scheme == MC3D_KENRK4 ? 5 : (s->lsldd_half == 1 ? 5 : 6);
}

// preStep (src/CurvilinearCSolver.hpp:310-318): calcDtFromCFL on the current
// state, fused into the primitives of stage 1, which read the same state
// (unless a sponge relaxation after the previous step formed both already)
template <typename R>
static int step_begin(mc3d_solver s) {
    int rc;
    const int first = s->host_time_step == s->cfg.time_step0;
    if (!s->prims_ready)
        if ((rc = primitives_cfl<R>(s))) return rc;
    s->cur_relaxed = s->prims_ready ? sponge_faces(s) : 0;
    s->prims_ready = false;
    s->launches++;
    if ((rc = launch_finalize_dt(s->ts, s->cfg.ts_type, s->cfg.cfl, s->cfg.dt, first, s->stream))) return rc;
    s->host_time_step++;
    s->cur_filter_now = s->host_time_step % s->cfg.filter_step == 0;
    s->cur_ns = stages_of(s);
    s->cur_stage = 0;
    return MC3D_OK;
}

// preSubStep (src/CurvilinearCSolver.hpp:320-327) of stage st: stage 1 works
// on q1 (filtered at the end of the previous step); later stages on qk, whose
// primitives the RK update of the previous stage already wrote unless a
// sub-step filter changed qk since. preStepBCHandling, then
// preStepDerivatives with the first two divergence sweeps.
template <typename R>
static int stage_begin(mc3d_solver s, int st) {
    int rc;
    if (st > 1 && s->cfg.substep_filtering)
        if ((rc = primitives<R>(s, s->qk))) return rc;
    if ((rc = wall_prestep<R>(s, st == 1 ? s->q1 : s->qk))) return rc;
    s->cons_mask = st == 1 ? s->cur_relaxed : 0;
    rc = s->lean ? stage_rhs_lean<R>(s, st == 1 ? s->q1 : s->qk) : stage_rhs<R>(s, st == 1 ? s->q1 : s->qk);
    s->cons_mask = 0;
    return rc;
}

// updateConservedData of the scheme's stage st (RK4.hpp:47-125,
// TVDRK3.hpp:50-133, KenRK4.hpp:53-152, LSLDDRK4.hpp:93-320); except after a
// step's last stage or with sub-step filtering, the same pass writes the
// primitives of the next stage's state (updateNonConservedData)
template <typename R>
static int stage_rk(mc3d_solver s, int st) {
    int rc;
    const int scheme = s->cfg.rk_type, ns = s->cur_ns;
    RkStage rs{};
    rs.scheme = scheme;
    rs.stage = st;
    rs.nstages = ns;
    if (scheme == MC3D_RK4) {
        rs.a = RK4_A[st - 1];
        rs.b = st < 4 ? RK4_B[st - 1] : 0.0;
    } else if (scheme == MC3D_KENRK4) {
        rs.a = KEN_A[st - 1];
        rs.b = KEN_B[st - 1];
    } else if (scheme == MC3D_LSLDDRK4) {
        rs.a = s->lsldd_half == 1 ? LS_A1[st - 1] : LS_A2[st - 1];
        rs.b = s->lsldd_half == 1 ? LS_B1[st - 1] : LS_B2[st - 1];
    }
    const R *k2[5];
    R *pw[5];
    for (int v = 0; v < 5; v++) {
        k2[v] = (const R *)s->k2[v];
        pw[v] = (R *)s->prim[v];
    }
    const bool fuse_prims = st < ns && !s->cfg.substep_filtering;
    // last stage of a filtered step (FP32 path): the filter's working copy
    const bool copy_final = !s->lean && st == ns && s->cur_filter_now && s->prec != MC3D_FP64;
    if (copy_final)
        for (int v = 0; v < 5; v++) pw[v] = (R *)s->tC[v];
    // after the last stage the step continues from q1 (filter_conserved), so
    // the 2N register is dead there, and so is the FP64 final state q2 when
    // the filter reads its working copy and no statistics read q2
    const bool two_n = scheme == MC3D_KENRK4 || scheme == MC3D_LSLDDRK4;
    const bool stats = s->cfg.velocity_stats || s->cfg.thermo_stats;
    rs.skip_last = (two_n ? 1 : 0) | (copy_final && !stats ? 2 : 0);
    s->launches++;
    {
        // reads k2 and the FP64 registers the scheme touches, writes the updated ones
        double b = 5.0 * sizeof(R);
        if (scheme == MC3D_RK4) b += st == 1 ? 5.0 * 8 * 3 : (st < 4 ? 5.0 * 8 * 4 : 5.0 * 8 * 2);
        else if (scheme == MC3D_TVDRK3) b += st == 1 ? 5.0 * 8 * 2 : 5.0 * 8 * 3;
        else b += st == 1 ? 5.0 * 8 * 3 : 5.0 * 8 * 4;
        if (st == ns) b -= 5.0 * 8 * ((rs.skip_last & 1) + ((rs.skip_last >> 1) & 1));
        if (fuse_prims || copy_final) b += 5.0 * sizeof(R);
        if ((rc = tic(s, KC_RK, b * (double)s->g.n()))) return rc;
    }
    if ((rc = launch_rk_update<R>(s->g, rs, k2, s->q1, s->qk, s->q2, (fuse_prims || copy_final) ? pw : nullptr,
                                  s->stream, copy_final)))
        return rc;
    if ((rc = toc(s))) return rc;
    if (copy_final) s->tc_fresh = true;
    return MC3D_OK;
}

// updateData (src/CurvilinearCSolver.hpp:346-353): filterConservedData after
// the last stage (or every stage with sub-step filtering); the primitives of
// the next state come from the RK update or from the next stage / step
template <typename R>
static int stage_end(mc3d_solver s, int st) {
    int rc;
    const bool last = st == s->cur_ns;
    if (last || s->cfg.substep_filtering)
        if ((rc = filter_conserved<R>(s, last))) return rc;
    s->stages++;
    return MC3D_OK;
}

// postStep (src/CurvilinearCSolver.hpp:355-375): LSLDDRK4 alternates its
// halves; statistics; the optional sponge relaxation.
static int step_end(mc3d_solver s);

template <typename R>
static int one_step(mc3d_solver s) {
    int rc;
    if ((rc = step_begin<R>(s))) return rc;
    for (int st = 1; st <= s->cur_ns; st++) {
        if ((rc = stage_begin<R>(s, st))) return rc;
        if ((rc = stage_solve<R>(s))) return rc;
        if ((rc = stage_post<R>(s))) return rc;
        if ((rc = stage_rk<R>(s, st))) return rc;
        if ((rc = stage_end<R>(s, st))) return rc;
    }
    return step_end(s);
}

}  // namespace mc3d

namespace mc3d {
// The default stream of the solvers on a device: one non-blocking stream per
// device, created with the first solver and kept until exit, so solvers that
// their caller does not place (mc3d_solver_set_stream) queue one after the
// other and mc3d_solver_sync waits for all of them.
static cudaError_t device_stream(int device, cudaStream_t *out) {
    static std::mutex mu;
    static std::map<int, cudaStream_t> streams;
    std::lock_guard<std::mutex> lk(mu);
    auto it = streams.find(device);
    if (it != streams.end()) {
        *out = it->second;
        return cudaSuccess;
    }
    cudaStream_t st = nullptr;
    cudaError_t e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    if (e != cudaSuccess) return e;
    streams[device] = st;
    *out = st;
    return cudaSuccess;
}
}  // namespace mc3d

using namespace mc3d;

extern "C" {

int mc3d_solver_create(const mc3d_config *cfg, int device, mc3d_solver *out) {
    if (!cfg || !out) return fail(MC3D_ERR_ARG, "null argument");
    *out = nullptr;
    const mc3d_config &c = *cfg;
    if (c.Nx <= 10 || c.Ny <= 10 || c.Nz <= 10)
        return fail(MC3D_ERR_CONFIG, "Number of grid points in any direction must be greater than 10");
    if (c.precision != MC3D_FP64 && c.precision != MC3D_FP32BULK) return fail(MC3D_ERR_CONFIG, "bad precision");
    if (c.les_model == MC3D_DSM && c.dsm_test_filter != 1 && c.dsm_test_filter != 2)
        return fail(MC3D_ERR_CONFIG, "DSMTESTFILTER must be 1 or 2");
    if (c.les_averaging < MC3D_AVG_NONE || c.les_averaging > MC3D_AVG_GLOBAL)
        return fail(MC3D_ERR_CONFIG, "unknown LESAVERAGING");
    if (c.les_model == MC3D_MLPSGS && !(c.mlp_fallback_frac >= 0.0 && c.mlp_fallback_frac <= 1.0))
        return fail(MC3D_ERR_CONFIG, "MLPFALLBACKFRAC must lie in [0, 1]");
    for (int f = 0; f < 6; f++)
        if (c.bc_kind[f] == MC3D_BC_INLET)
            return fail(MC3D_ERR_CONFIG, "INLET faces have no boundary treatment in the reference solver");
    if (c.filter_step < 1) return fail(MC3D_ERR_CONFIG, "FILTERSTEP must be >= 1");
    if (c.lean_storage) {
        for (int d = 0; d < 3; d++)
            if (c.bc_type[d] != MC3D_PERIODIC_SOLVE)
                return fail(MC3D_ERR_CONFIG, "GPU.STORAGE = LEAN needs periodic directions");
        for (int f = 0; f < 6; f++)
            if (is_wall_kind(c.bc_kind[f]) || c.bc_kind[f] == MC3D_BC_SPONGE)
                return fail(MC3D_ERR_CONFIG, "GPU.STORAGE = LEAN has no walls or sponges");
        if (c.les_model == MC3D_DSM || (c.les_model == MC3D_VREMAN && c.les_averaging != MC3D_AVG_NONE))
            return fail(MC3D_ERR_CONFIG, "GPU.STORAGE = LEAN takes NOMODEL, VREMAN without averaging or MLP");
        if (c.substep_filtering || c.velocity_stats || c.thermo_stats || c.sponge_relax)
            return fail(MC3D_ERR_CONFIG, "GPU.STORAGE = LEAN has no sub-step filtering, statistics or relaxation");
        if (c.lean_slab < 0) return fail(MC3D_ERR_CONFIG, "GPU.LEANSLAB must be >= 0");
    }
    MC3D_CUDA_TRY(cudaSetDevice(device));
    mc3d_solver s = new mc3d_solver_s();
    s->cfg = c;
    s->device = device;
    s->prec = c.precision;
    s->g = Grid3{c.Nx, c.Ny, c.Nz};
    s->host_time_step = c.time_step0;
    for (int f = 0; f < 6; f++) {
        s->have_walls = s->have_walls || is_wall_kind(c.bc_kind[f]);
        s->have_sponge = s->have_sponge || c.bc_kind[f] == MC3D_BC_SPONGE;
        if (is_wall_kind(c.bc_kind[f])) s->wall_mask |= 1 << f;
    }
    cudaError_t e = device_stream(device, &s->stream);
    if (e != cudaSuccess) {
        delete s;
        return fail(MC3D_ERR_CUDA, std::string("cudaStreamCreate: ") + cudaGetErrorString(e));
    }
    int N[3] = {c.Nx, c.Ny, c.Nz};
    int rc = MC3D_OK;
    try {
        for (int d = 0; d < 3; d++) {
            // Domain with unit extents (src/Domain.hpp:45-79)
            s->dxi[d] = c.bc_type[d] == MC3D_PERIODIC_SOLVE ? 1.0 / N[d] : 1.0 / (N[d] - 1.0);
            LineOpHost dh = build_deriv_op(c.fd_type[d], c.bc_type[d], N[d], s->dxi[d]);
            LineOpHost fh = build_filter_op(c.filter_type, c.alphaF, c.bc_type[d], N[d]);
            LineOpHost vh = build_filter_op(MC3D_COMPACT10, -0.49, c.bc_type[d], N[d]);
            if ((rc = upload_line_op(dh, c.precision, s->dop[d]))) break;
            if ((rc = upload_line_op(fh, c.precision, s->fop[d]))) break;
            if ((rc = upload_line_op(vh, c.precision, s->vop[d]))) break;
            if (c.les_model == MC3D_DSM || c.les_model == MC3D_MLPSGS) {
                // DSMTESTFILTER 1 -> Pade, 2 -> explicit (src/DSMSGS.hpp:57-67)
                LineOpHost th = build_testfilter_op(c.dsm_test_filter == 1 ? MC3D_TESTFILTER_PADE : MC3D_TESTFILTER_EXP,
                                                    c.bc_type[d], N[d]);
                if ((rc = upload_line_op(th, c.precision, s->top[d]))) break;
            }
        }
    } catch (const std::exception &ex) {
        rc = fail(MC3D_ERR_CONFIG, ex.what());
    }
    size_t n = (size_t)s->g.n();
    size_t rb = c.precision == MC3D_FP64 ? sizeof(double) : sizeof(float);
    s->lean = c.lean_storage != 0;
    if (s->lean) {
        const long long plane = (long long)c.Nx * c.Ny;
        s->slab_nz = c.lean_slab > 0 ? std::min(c.lean_slab, c.Nz)
                                     : (int)std::max(1LL, std::min((long long)c.Nz, (1LL << 26) / plane));
        const size_t ns = (size_t)plane * s->slab_nz;
        const bool two_n = c.rk_type == MC3D_KENRK4 || c.rk_type == MC3D_LSLDDRK4;
        for (int v = 0; v < 5 && !rc; v++) {
            rc = rc ? rc : salloc(s, (void **)&s->q1[v], n * sizeof(double));
            rc = rc ? rc : salloc(s, (void **)&s->qk[v], n * sizeof(double));
            if (two_n) s->q2[v] = s->qk[v];   // the 2N schemes write the final state over the stage state
            else rc = rc ? rc : salloc(s, (void **)&s->q2[v], n * sizeof(double));
            rc = rc ? rc : salloc(s, &s->k2[v], n * rb);
            rc = rc ? rc : salloc(s, &s->prim[v], n * rb);
        }
        for (int var = 0; var < 4 && !rc; var++) {
            rc = salloc(s, &s->der[3 * var + 0], ns * rb);
            if (!rc) rc = salloc(s, &s->der[3 * var + 1], ns * rb);
            if (!rc) rc = salloc(s, &s->der[3 * var + 2], n * rb);
        }
        for (int i = 0; i < 15 && !rc; i++) rc = salloc(s, &s->flux[i], (i < 10 ? ns : n) * rb);
        if (!rc) {
            // the filter's two work fields are the xi3-flux fields
            s->tA[0] = s->flux[10];
            s->tB[0] = s->flux[11];
        }
        if (c.les_model == MC3D_MLPSGS) {
            if (!rc) rc = salloc(s, &s->mu_sgs, ns * rb);
            if (!rc) rc = salloc(s, &s->ksgs, ns * rb);
            if (!rc) rc = salloc(s, (void **)&s->mlp_flag, sizeof(int));
            if (!rc) {
                cudaError_t he = cudaMallocHost((void **)&s->mlp_flag_host, sizeof(int));
                if (he != cudaSuccess) rc = fail(MC3D_ERR_OOM, "cudaMallocHost");
            }
        }
    }
    for (int v = 0; v < 5 && !rc && !s->lean; v++) {
        rc = rc ? rc : salloc(s, (void **)&s->q1[v], n * sizeof(double));
        rc = rc ? rc : salloc(s, (void **)&s->qk[v], n * sizeof(double));
        rc = rc ? rc : salloc(s, (void **)&s->q2[v], n * sizeof(double));
        rc = rc ? rc : salloc(s, &s->k2[v], n * rb);
        rc = rc ? rc : salloc(s, &s->rhs[v], n * rb);
        rc = rc ? rc : salloc(s, &s->tA[v], n * rb);
        rc = rc ? rc : salloc(s, &s->tB[v], n * rb);
        if (!rc && c.precision != MC3D_FP64) rc = salloc(s, &s->tC[v], n * rb);
    }
    for (int v = 0; v < 5 && !rc && !s->lean; v++) rc = salloc(s, &s->prim[v], n * rb);
    for (int v = 0; v < 12 && !rc && !s->lean; v++) rc = salloc(s, &s->der[v], n * rb);
    for (int v = 0; v < 15 && !rc && !s->lean; v++) rc = salloc(s, &s->flux[v], n * rb);
    if (!rc && !s->lean && c.les_model != MC3D_NOMODEL) rc = salloc(s, &s->mu_sgs, n * rb);
    if (c.velocity_stats)
        for (int k = 0; k < 9 && !rc; k++) rc = salloc(s, (void **)&s->stv[k], n * sizeof(double));
    if (c.thermo_stats)
        for (int k = 0; k < 6 && !rc; k++) rc = salloc(s, (void **)&s->stt[k], n * sizeof(double));
    s->st_prev = c.time0;   // Stats takes the solver's time at construction (src/Stats.hpp:58)
    if (c.les_model == MC3D_MLPSGS && !s->lean) {
        if (!rc) rc = salloc(s, (void **)&s->mlp_flag, sizeof(int));
        if (!rc) {
            cudaError_t he = cudaMallocHost((void **)&s->mlp_flag_host, sizeof(int));
            if (he != cudaSuccess) rc = fail(MC3D_ERR_OOM, "cudaMallocHost");
        }
    }
    if ((c.les_model == MC3D_DSM || c.les_model == MC3D_MLPSGS) && !s->lean) {
        for (int i = 0; i < 24 && !rc; i++) rc = salloc(s, &s->dA[i], n * rb);
        for (int i = 0; i < 24 && !rc; i++) rc = salloc(s, &s->dB[i], n * rb);
        if (!rc) rc = salloc(s, &s->smag, n * rb);
        if (!rc) rc = salloc(s, &s->taukk, n * rb);
        if (!rc) rc = salloc(s, &s->ksgs, n * rb);
    }
    if (!rc && c.les_model != MC3D_NOMODEL) rc = salloc(s, (void **)&s->avg_scratch, AVG_SCRATCH * sizeof(double));
    if (s->have_walls && !rc) rc = salloc(s, &s->Tmu, n * rb);
    if (s->have_sponge) {
        if (!rc) rc = salloc(s, (void **)&s->sigma, n * sizeof(double));
        for (int v = 0; v < 5 && !rc; v++) rc = salloc(s, (void **)&s->spg_avg[v], n * sizeof(double));
    }
    if (!rc) rc = salloc(s, (void **)&s->ts, sizeof(TimeState));
    if (!rc) rc = salloc(s, (void **)&s->acc, 2 * sizeof(double));
    if (!rc) {
        TimeState t{};
        t.time = c.time0;
        t.time_step = c.time_step0;
        t.dt = c.ts_type == MC3D_CONST_DT ? c.dt : 0.0;
        e = cudaMemcpyAsync(s->ts, &t, sizeof(t), cudaMemcpyHostToDevice, s->stream);
        if (e != cudaSuccess) rc = fail(MC3D_ERR_CUDA, cudaGetErrorString(e));
    }
    if (!rc) {
        e = cudaStreamSynchronize(s->stream);
        if (e != cudaSuccess) rc = fail(MC3D_ERR_CUDA, cudaGetErrorString(e));
    }
    if (rc) {
        mc3d_solver_destroy(s);
        return rc;
    }
    *out = s;
    return MC3D_OK;
}

int mc3d_solver_destroy(mc3d_solver s) {
    if (!s) return MC3D_OK;
    cudaSetDevice(s->device);
    if (s->stream) cudaStreamSynchronize(s->stream);
    for (cudaEvent_t e : s->events) cudaEventDestroy(e);
    for (void *p : s->allocs) cudaFree(p);
    if (s->mlp_flag_host) cudaFreeHost(s->mlp_flag_host);
    for (int d = 0; d < 3; d++) {
        free_line_op(s->dop[d]);
        free_line_op(s->fop[d]);
        free_line_op(s->vop[d]);
        free_line_op(s->top[d]);
    }
    // (the device's shared stream stays for the other solvers)
    delete s;
    return MC3D_OK;
}

static int upload_metrics(mc3d_solver s, const double *const h[10], const double *cvals) {
    size_t n = (size_t)s->g.n();
    int rc;
    if (h) {
        // constant metrics (uniform Cartesian blocks such as the HIT box) are
        // carried as 10 scalars instead of 10 resident fields
        bool cst = true;
        for (int c = 0; c < 10 && cst; c++) {
            double v0 = h[c][0], scale = std::fabs(v0) > 0 ? std::fabs(v0) : 1.0;
            for (size_t i = 1; i < n; i++)
                if (std::fabs(h[c][i] - v0) > 1e-13 * scale) { cst = false; break; }
        }
        s->const_met = cst;
        for (int c = 0; c < 10; c++) s->met_c[c] = h[c][0];
        if (!cst) {
            size_t rb = s->prec == MC3D_FP64 ? sizeof(double) : sizeof(float);
            for (int c = 0; c < 10; c++) {
                if (!s->met64[c] && (rc = salloc(s, (void **)&s->met64[c], n * sizeof(double)))) return rc;
                MC3D_CUDA_TRY(cudaMemcpyAsync(s->met64[c], h[c], n * sizeof(double), cudaMemcpyHostToDevice, s->stream));
                if (s->prec == MC3D_FP64) {
                    s->metR[c] = s->met64[c];
                } else {
                    if (!s->metR[c] && (rc = salloc(s, &s->metR[c], n * rb))) return rc;
                    std::vector<float> tmp(n);
                    for (size_t i = 0; i < n; i++) tmp[i] = (float)h[c][i];
                    MC3D_CUDA_TRY(cudaMemcpyAsync(s->metR[c], tmp.data(), n * sizeof(float), cudaMemcpyHostToDevice, s->stream));
                    MC3D_CUDA_TRY(cudaStreamSynchronize(s->stream));
                }
            }
        }
    } else {
        s->const_met = true;
        for (int c = 0; c < 10; c++) s->met_c[c] = cvals[c];
    }
    s->have_metrics = true;
    MC3D_CUDA_TRY(cudaStreamSynchronize(s->stream));
    return MC3D_OK;
}

int mc3d_solver_set_metrics(mc3d_solver s, const double *const metrics[10]) {
    if (!s || !metrics) return fail(MC3D_ERR_ARG, "null argument");
    for (int c = 0; c < 10; c++)
        if (!metrics[c]) return fail(MC3D_ERR_ARG, "null metric field");
    MC3D_CUDA_TRY(cudaSetDevice(s->device));
    return upload_metrics(s, metrics, nullptr);
}

int mc3d_solver_set_box_metrics(mc3d_solver s, double Lx, double Ly, double Lz) {
    if (!s) return fail(MC3D_ERR_ARG, "null solver");
    if (!(Lx > 0 && Ly > 0 && Lz > 0)) return fail(MC3D_ERR_ARG, "box lengths must be positive");
    MC3D_CUDA_TRY(cudaSetDevice(s->device));
    double c[10] = {1.0 / (Lx * Ly * Lz), 1.0 / Lx, 0, 0, 0, 1.0 / Ly, 0, 0, 0, 1.0 / Lz};
    int rc = upload_metrics(s, nullptr, c);
    if (rc) return rc;
    s->box_L[0] = Lx;
    s->box_L[1] = Ly;
    s->box_L[2] = Lz;
    s->mesh_kind = 2;
    for (auto &v : s->mesh_xyz) std::vector<double>().swap(v);
    return MC3D_OK;
}

namespace mc3d {

// Translation of each PERIODIC_SOLVE direction (handlePeriodicStuff,
// src/AbstractSingleBlockMesh.cpp:2019-2083). The xi1 branch tests the Y faces
// (:2034), so x takes PERIODICDISPX only when the Y faces are PERIODIC;
// INTERNALLY_PERIODIC faces translate by zero; the reference leaves any other
// combination unset, zero here.
static void periodic_translations(const mc3d_config &c, double T[3][3]) {
    for (int d = 0; d < 3; d++) {
        for (int e = 0; e < 3; e++) T[d][e] = 0.0;
        if (c.bc_type[d] != MC3D_PERIODIC_SOLVE) continue;
        const int face = d == 0 ? 2 : 2 * d;
        if (c.bc_kind[face] == MC3D_BC_PERIODIC && c.bc_kind[face + 1] == MC3D_BC_PERIODIC)
            for (int e = 0; e < 3; e++) T[d][e] = c.periodic_disp[d][e];
    }
}

// Operators of one metric direction: the derivative, and for periodic
// directions the same left-hand side with an identity RHS stencil (the solve
// of a TPB right-hand side built by tpb_rhs_kernel).
struct MetricDir {
    LineOpBuf deriv, solve;
    bool periodic = false, cd2 = false;
    int H = 0;
    double st[7] = {0};
    double dh = 1.0;
};

// One metric derivative along d, in -> out. On a periodic direction whose
// translation or ghost quirk changes the ghosts, the reference's TPB
// derivative: the RHS with ghosts sum_t (X_t -+ T_t) W_t at the wrapped indices
// (tmp), then the periodic solve; otherwise the solver's plain derivative.
static int metric_deriv(mc3d_solver s, int d, const MetricDir &md, const double *in, double *out, double *tmp,
                        int nterms, const double *T, const double *const *X, const double *const *W, bool nm3_quirk) {
    bool tpb = md.periodic && nm3_quirk;
    for (int t = 0; t < nterms && md.periodic; t++) tpb = tpb || T[t] != 0.0;
    SweepBatch<double> b{};
    b.nf = 1;
    RhsFinalArgs<double> rf{};
    if (!tpb) {
        b.in[0] = in;
        b.out[0] = out;
        return launch_sweep<double>(d, s->g, md.deriv.f64, b, EPI_STORE, rf, s->cfg.bc_type, false, s->stream);
    }
    TpbArgs a{};
    a.N = d == 0 ? s->g.Nx : (d == 1 ? s->g.Ny : s->g.Nz);
    a.H = md.H;
    a.nterms = nterms;
    a.explicit_cd2 = md.cd2 ? 1 : 0;
    a.nm3_from_nm2 = nm3_quirk ? 1 : 0;
    for (int k = 0; k < 7; k++) a.st[k] = md.st[k];
    a.dh = md.dh;
    for (int t = 0; t < nterms; t++) {
        a.T[t] = T[t];
        a.X[t] = X[t];
        a.W[t] = W ? W[t] : nullptr;
    }
    if (md.cd2) return launch_tpb_rhs(s->g, d, in, a, out, s->stream);   // explicit: the RHS is the derivative
    int rc = launch_tpb_rhs(s->g, d, in, a, tmp, s->stream);
    if (rc) return rc;
    b.in[0] = tmp;
    b.out[0] = out;
    return launch_sweep<double>(d, s->g, md.solve.f64, b, EPI_STORE, rf, s->cfg.bc_type, false, s->stream);
}

// solveForJacobians (src/AbstractSingleBlockMesh.cpp:23-1308) on the device.
static int compute_metrics(mc3d_solver s, const double *hx, const double *hy, const double *hz,
                           std::vector<std::vector<double>> &host) {
    const long long n = s->g.n();
    const size_t bytes = (size_t)n * sizeof(double);
    const int Ns[3] = {s->g.Nx, s->g.Ny, s->g.Nz};
    std::vector<void *> mine;
    MetricDir md[3];
    int rc = MC3D_OK;
    auto dalloc = [&](size_t b) -> double * {
        void *p = nullptr;
        if (cudaMalloc(&p, b) != cudaSuccess) return nullptr;
        mine.push_back(p);
        return (double *)p;
    };
    auto cleanup = [&]() {
        cudaStreamSynchronize(s->stream);
        for (void *p : mine) cudaFree(p);
        for (int d = 0; d < 3; d++) {
            free_line_op(md[d].deriv);
            free_line_op(md[d].solve);
        }
    };
    // x, y, z; xE1j = dx/dxi_j, xE2j = dy/dxi_j; the nine cofactors; temporaries
    double *X[3], *xE1[3], *xE2[3], *Jr[9], *t0, *t1, *t2, *tr, *Jf;
    double **slots[] = {&X[0], &X[1], &X[2], &xE1[0], &xE1[1], &xE1[2], &xE2[0], &xE2[1], &xE2[2], &Jr[0], &Jr[1],
                        &Jr[2], &Jr[3], &Jr[4], &Jr[5], &Jr[6], &Jr[7], &Jr[8], &t0, &t1, &t2, &tr, &Jf};
    for (double **sl : slots)
        if (!(*sl = dalloc(bytes))) {
            cleanup();
            return fail(MC3D_ERR_OOM, "device allocation for the metric computation failed");
        }
    const double *hs[3] = {hx, hy, hz};
    for (int c = 0; c < 3; c++)
        if (cudaMemcpyAsync(X[c], hs[c], bytes, cudaMemcpyHostToDevice, s->stream) != cudaSuccess) {
            cleanup();
            return fail(MC3D_ERR_CUDA, "mesh upload failed");
        }
    try {
        for (int d = 0; d < 3 && !rc; d++) {
            LineOpHost h = build_deriv_op(s->cfg.fd_type[d], s->cfg.bc_type[d], Ns[d], s->dxi[d]);
            if ((rc = upload_line_op(h, MC3D_FP64, md[d].deriv))) break;
            md[d].periodic = s->cfg.bc_type[d] == MC3D_PERIODIC_SOLVE;
            md[d].cd2 = s->cfg.fd_type[d] == MC3D_CD2;
            md[d].H = h.H;
            for (int k = 0; k <= 2 * h.H && k < 7; k++) md[d].st[k] = h.st[k];
            md[d].dh = s->dxi[d];
            if (md[d].periodic && !md[d].cd2) {
                LineOpHost sv = h;
                for (double &v : sv.st) v = 0.0;
                sv.st[sv.H] = 1.0;
                sv.deriv = false;
                sv.inv_dh = 1.0;
                rc = upload_line_op(sv, MC3D_FP64, md[d].solve);
            }
        }
    } catch (const std::exception &e) {
        cleanup();
        return fail(MC3D_ERR_CONFIG, e.what());
    }
    if (rc) {
        cleanup();
        return fail(rc, "metric operator setup failed");
    }
    double T[3][3];
    periodic_translations(s->cfg, T);
    const bool q = s->cfg.reference_quirks != 0;
    auto penta = [&](int d) { return s->cfg.fd_type[d] == MC3D_PENTA10; };
#define MC3D_MTRY(x)      \
    if ((rc = (x))) {     \
        cleanup();        \
        return rc;        \
    }
    // xE1j, xE2j (:39-303); d y / d xi3 of a BW7 scheme passes Nm2 as Nm3 (:273)
    for (int j = 0; j < 3; j++) {
        const double *xc[1] = {X[0]}, *yc[1] = {X[1]};
        MC3D_MTRY(metric_deriv(s, j, md[j], X[0], xE1[j], tr, 1, &T[j][0], xc, nullptr, false));
        MC3D_MTRY(metric_deriv(s, j, md[j], X[1], xE2[j], tr, 1, &T[j][1], yc, nullptr, q && j == 2 && penta(2)));
    }
    // cofactors from the off-diagonal derivatives of Va_j = xE1j y, Vb_j = xE1j z,
    // Vc_j = xE2j z (:320-1023): J_ab = dV[j1]/dxi[k1] - dV[j2]/dxi[k2]
    static const int tab[9][5] = {{2, 1, 2, 2, 1}, {1, 2, 1, 1, 2}, {0, 1, 2, 2, 1},
                                  {2, 2, 0, 0, 2}, {1, 0, 2, 2, 0}, {0, 2, 0, 0, 2},
                                  {2, 0, 1, 1, 0}, {1, 1, 0, 0, 1}, {0, 0, 1, 1, 0}};
    auto dV = [&](int fam, int j, int k, double *out) -> int {
        const double *w = fam == 2 ? xE2[j] : xE1[j];
        const int c = fam == 0 ? 1 : 2;
        int r = launch_metric_mul(n, w, X[c], t0, s->stream);
        if (r) return r;
        const double *xc[1] = {X[c]}, *wc[1] = {w};
        // d Vc3 / d xi1 of a BW7 scheme passes Nm2 as Nm3 (:706)
        return metric_deriv(s, k, md[k], t0, out, tr, 1, &T[k][c], xc, wc,
                            q && fam == 2 && j == 2 && k == 0 && penta(0));
    };
    for (int ab = 0; ab < 9; ab++) {
        MC3D_MTRY(dV(tab[ab][0], tab[ab][1], tab[ab][2], t1));
        MC3D_MTRY(dV(tab[ab][0], tab[ab][3], tab[ab][4], t2));
        MC3D_MTRY(launch_metric_sub(n, t1, t2, Jr[ab], s->stream));
    }
    // determinant: (1/3) sum_i d(x J_i1 + y J_i2 + z J_i3)/dxi_i (:1058-1296)
    double *jd[3] = {xE1[0], xE1[1], xE1[2]};
    for (int i = 0; i < 3; i++) {
        const double *xyz[3] = {X[0], X[1], X[2]};
        const double *abc[3] = {Jr[3 * i], Jr[3 * i + 1], Jr[3 * i + 2]};
        MC3D_MTRY(launch_metric_dot3(n, xyz, abc, t0, s->stream));
        MC3D_MTRY(metric_deriv(s, i, md[i], t0, jd[i], tr, 3, T[i], xyz, abc, false));
    }
    const double *jdc[3] = {jd[0], jd[1], jd[2]};
    MC3D_MTRY(launch_metric_finish(n, jdc, Jr, Jf, s->stream));
#undef MC3D_MTRY
    host.assign(10, std::vector<double>((size_t)n));
    const double *src[10] = {Jf, Jr[0], Jr[1], Jr[2], Jr[3], Jr[4], Jr[5], Jr[6], Jr[7], Jr[8]};
    for (int c = 0; c < 10; c++)
        if (cudaMemcpyAsync(host[c].data(), src[c], bytes, cudaMemcpyDeviceToHost, s->stream) != cudaSuccess) {
            cleanup();
            return fail(MC3D_ERR_CUDA, "metric download failed");
        }
    cudaError_t e = cudaStreamSynchronize(s->stream);
    cleanup();
    if (e != cudaSuccess) return fail(MC3D_ERR_CUDA, cudaGetErrorString(e));
    return MC3D_OK;
}

}  // namespace mc3d

int mc3d_solver_set_mesh(mc3d_solver s, const double *x, const double *y, const double *z) {
    if (!s || !x || !y || !z) return fail(MC3D_ERR_ARG, "null argument");
    MC3D_CUDA_TRY(cudaSetDevice(s->device));
    std::vector<std::vector<double>> h;
    int rc = mc3d::compute_metrics(s, x, y, z, h);
    if (rc) return rc;
    const double *p[10];
    for (int c = 0; c < 10; c++) p[c] = h[c].data();
    rc = upload_metrics(s, p, nullptr);
    if (rc) return rc;
    const size_t n = (size_t)s->g.n();
    s->mesh_xyz[0].assign(x, x + n);
    s->mesh_xyz[1].assign(y, y + n);
    s->mesh_xyz[2].assign(z, z + n);
    s->mesh_kind = 1;
    return MC3D_OK;
}

int mc3d_solver_get_metrics(mc3d_solver s, double *const metrics[10]) {
    if (!s || !metrics) return fail(MC3D_ERR_ARG, "null argument");
    for (int c = 0; c < 10; c++)
        if (!metrics[c]) return fail(MC3D_ERR_ARG, "null metric field");
    if (!s->have_metrics) return fail(MC3D_ERR_CONFIG, "no metrics set");
    MC3D_CUDA_TRY(cudaSetDevice(s->device));
    const size_t n = (size_t)s->g.n();
    for (int c = 0; c < 10; c++) {
        if (s->const_met) {
            for (size_t i = 0; i < n; i++) metrics[c][i] = s->met_c[c];
        } else {
            MC3D_CUDA_TRY(cudaMemcpyAsync(metrics[c], s->met64[c], n * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
        }
    }
    MC3D_CUDA_TRY(cudaStreamSynchronize(s->stream));
    return MC3D_OK;
}

static int set_initial_impl(mc3d_solver s, const double *rho, const double *U, const double *V, const double *W,
                            const double *p, bool device) {
    if (!s || !rho || !U || !V || !W || !p) return fail(MC3D_ERR_ARG, "null argument");
    if (!s->have_metrics) return fail(MC3D_ERR_CONFIG, "set the metrics before the initial condition");
    MC3D_CUDA_TRY(cudaSetDevice(s->device));
    size_t n = (size_t)s->g.n();
    s->prims_ready = false;
    if (!s->have_walls) {
        // no wall treatment: the conserved state is formed on the device. Host
        // primitives go through the (not yet used) q2 registers.
        if (s->have_sponge && !s->sigma_set)
            return fail(MC3D_ERR_CONFIG, "set the sponge strength before the initial condition");
        const double *src[5] = {rho, U, V, W, p};
        const double *dp[5];
        for (int v = 0; v < 5; v++) {
            if (device) {
                dp[v] = src[v];
            } else {
                MC3D_CUDA_TRY(cudaMemcpyAsync(s->q2[v], src[v], n * 8, cudaMemcpyHostToDevice, s->stream));
                dp[v] = s->q2[v];
            }
        }
        int *bad = s->ts ? &s->ts->nonfinite : nullptr;
        MC3D_CUDA_TRY(cudaMemsetAsync(bad, 0, sizeof(int), s->stream));
        int rc = launch_init_conserved((long long)n, dp, s->q1, bad, s->stream);
        if (rc) return rc;
        for (int v = 0; v < 5; v++) {
            MC3D_CUDA_TRY(cudaMemsetAsync(s->k2[v], 0, n * (s->prec == MC3D_FP64 ? 8 : 4), s->stream));
            // the sponge target starts as the initial state (src/CurvilinearCSolver_BC.cpp:325-341)
            if (s->have_sponge)
                MC3D_CUDA_TRY(cudaMemcpyAsync(s->spg_avg[v], s->q1[v], n * 8, cudaMemcpyDeviceToDevice, s->stream));
        }
        int hbad = 0;
        MC3D_CUDA_TRY(cudaMemcpyAsync(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
        MC3D_CUDA_TRY(cudaStreamSynchronize(s->stream));
        if (hbad) {
            MC3D_CUDA_TRY(cudaMemset(bad, 0, sizeof(int)));
            return fail(MC3D_ERR_NONFINITE, "non-finite or non-positive initial state");
        }
        s->initialized = true;
        return MC3D_OK;
    }
    // conserved state of setInitialConditions (src/CurvilinearCSolver_BC.cpp:31-59)
    std::vector<double> h[5];
    std::vector<double> hr(n), hu(n), hv(n), hw(n), hp(n);
    if (device) {
        MC3D_CUDA_TRY(cudaMemcpy(hr.data(), rho, n * 8, cudaMemcpyDeviceToHost));
        MC3D_CUDA_TRY(cudaMemcpy(hu.data(), U, n * 8, cudaMemcpyDeviceToHost));
        MC3D_CUDA_TRY(cudaMemcpy(hv.data(), V, n * 8, cudaMemcpyDeviceToHost));
        MC3D_CUDA_TRY(cudaMemcpy(hw.data(), W, n * 8, cudaMemcpyDeviceToHost));
        MC3D_CUDA_TRY(cudaMemcpy(hp.data(), p, n * 8, cudaMemcpyDeviceToHost));
        rho = hr.data(); U = hu.data(); V = hv.data(); W = hw.data(); p = hp.data();
    }
    const double gamma = 1.4, Rg = 1.0 / 1.4;
    if (s->have_sponge && !s->sigma_set) return fail(MC3D_ERR_CONFIG, "set the sponge strength before the initial condition");
    std::vector<double> uu(U, U + n), vv(V, V + n), ww(W, W + n), T;
    if (s->have_walls) {
        // wall conditions of setInitialConditions (src/CurvilinearCSolver_BC.cpp:60-313): no-slip
        // faces X0..Z1, then moving walls; the Neumann wall temperature uses the
        // scheme of the wall-normal direction. On X1 the reference takes it for
        // CONST_T_WALL rather than ADIABATIC_WALL (:98).
        T.resize(n);
        for (size_t i = 0; i < n; i++) T[i] = p[i] / (rho[i] * Rg);
        // mu of the first stage stays that of this temperature on the walls
        if (s->prec == MC3D_FP64) {
            MC3D_CUDA_TRY(cudaMemcpy(s->Tmu, T.data(), n * 8, cudaMemcpyHostToDevice));
        } else {
            std::vector<float> tf(T.begin(), T.end());
            MC3D_CUDA_TRY(cudaMemcpy(s->Tmu, tf.data(), n * 4, cudaMemcpyHostToDevice));
        }
        s->tmu_from_init = true;
        const long long Nx = s->g.Nx, Ny = s->g.Ny, Nz = s->g.Nz;
        const long long dimn[3] = {Nx, Ny, Nz}, strd[3] = {1, Nx, Nx * Ny};
        for (int pass = 0; pass < 2; pass++)
            for (int f = 0; f < 6; f++) {
                const int k = s->cfg.bc_kind[f], d = f >> 1, side = f & 1;
                const bool noslip = k == MC3D_BC_ADIABATIC_WALL || k == MC3D_BC_CONST_T_WALL;
                if (pass == 0 ? !noslip : k != MC3D_BC_MOVING_ADIABATIC_WALL) continue;
                bool neumann = pass == 1 || (f == 1 ? k == MC3D_BC_CONST_T_WALL : k == MC3D_BC_ADIABATIC_WALL);
                const double v1 = pass ? s->cfg.wall_velocity[f][0] : 0.0, v2 = pass ? s->cfg.wall_velocity[f][1] : 0.0;
                const long long step = side ? -strd[d] : strd[d];
                for (long long kk = 0; kk < Nz; kk++)
                    for (long long jj = 0; jj < Ny; jj++)
                        for (long long ii = 0; ii < Nx; ii++) {
                            const long long c3[3] = {ii, jj, kk};
                            if (c3[d] != (side ? dimn[d] - 1 : 0)) continue;
                            const long long i = ii + Nx * (jj + Ny * kk);
                            double uw[3];
                            uw[d] = 0.0;
                            uw[d == 0 ? 1 : 0] = v1;
                            uw[d == 2 ? 1 : 2] = v2;
                            uu[i] = uw[0];
                            vv[i] = uw[1];
                            ww[i] = uw[2];
                            if (neumann) {
                                double f6[6];
                                for (int m = 0; m < 6; m++) f6[m] = (m < dimn[d] - 1) ? T[i + (m + 1) * step] : 0.0;
                                T[i] = mc3d_calc_neumann(s->cfg.fd_type[d], f6);
                            }
                        }
            }
    }
    for (int v = 0; v < 5; v++) h[v].resize(n);
    for (size_t i = 0; i < n; i++) {
        double r = rho[i];
        h[0][i] = r;
        h[1][i] = r * uu[i];
        h[2][i] = r * vv[i];
        h[3][i] = r * ww[i];
        // with walls p and rhoE follow from rho and T everywhere (src/CurvilinearCSolver_BC.cpp:314-323)
        const double pp = s->have_walls ? r * Rg * T[i] : p[i];
        h[4][i] = pp / (gamma - 1.0) + 0.5 * r * (uu[i] * uu[i] + vv[i] * vv[i] + ww[i] * ww[i]);
        if (!std::isfinite(h[4][i]) || !(r > 0)) return fail(MC3D_ERR_NONFINITE, "non-finite or non-positive initial state");
    }
    for (int v = 0; v < 5; v++) {
        MC3D_CUDA_TRY(cudaMemcpyAsync(s->q1[v], h[v].data(), n * 8, cudaMemcpyHostToDevice, s->stream));
        MC3D_CUDA_TRY(cudaMemsetAsync(s->k2[v], 0, n * (s->prec == MC3D_FP64 ? 8 : 4), s->stream));
        // the sponge target starts as the initial state (src/CurvilinearCSolver_BC.cpp:325-341)
        if (s->have_sponge)
            MC3D_CUDA_TRY(cudaMemcpyAsync(s->spg_avg[v], h[v].data(), n * 8, cudaMemcpyHostToDevice, s->stream));
    }
    MC3D_CUDA_TRY(cudaStreamSynchronize(s->stream));
    s->initialized = true;
    return MC3D_OK;
}

int mc3d_solver_set_initial(mc3d_solver s, const double *rho, const double *U, const double *V, const double *W,
                            const double *p) {
    return set_initial_impl(s, rho, U, V, W, p, false);
}
int mc3d_solver_set_initial_device(mc3d_solver s, const double *rho, const double *U, const double *V,
                                   const double *W, const double *p) {
    return set_initial_impl(s, rho, U, V, W, p, true);
}

int mc3d_solver_set_mlp(mc3d_solver s, mc3d_mlp m) {
    if (!s || !m) return fail(MC3D_ERR_ARG, "null argument");
    if (s->cfg.les_model != MC3D_MLPSGS) return fail(MC3D_ERR_CONFIG, "LESMODEL is not MLP");
    s->mlp = m;
    return MC3D_OK;
}

int mc3d_solver_mlp_fallbacks(mc3d_solver s, long long *stages) {
    if (!s || !stages) return fail(MC3D_ERR_ARG, "null argument");
    *stages = s->mlp_fallbacks;
    return MC3D_OK;
}

int mc3d_solver_set_sponge(mc3d_solver s, const double *sigma) {
    if (!s || !sigma) return fail(MC3D_ERR_ARG, "null argument");
    if (!s->have_sponge) return fail(MC3D_ERR_CONFIG, "no face is a SPONGE");
    MC3D_CUDA_TRY(cudaSetDevice(s->device));
    MC3D_CUDA_TRY(cudaMemcpyAsync(s->sigma, sigma, (size_t)s->g.n() * 8, cudaMemcpyHostToDevice, s->stream));
    MC3D_CUDA_TRY(cudaStreamSynchronize(s->stream));
    s->sigma_set = true;
    s->sponge_pts = 0;
    for (long long i = 0; i < s->g.n(); i++) s->sponge_pts += sigma[i] != 0.0;
    return MC3D_OK;
}

int mc3d_solver_set_sponge_avg(mc3d_solver s, const double *const avg[5]) {
    if (!s || !avg) return fail(MC3D_ERR_ARG, "null argument");
    if (!s->have_sponge) return fail(MC3D_ERR_CONFIG, "no face is a SPONGE");
    MC3D_CUDA_TRY(cudaSetDevice(s->device));
    for (int v = 0; v < 5; v++) {
        if (!avg[v]) return fail(MC3D_ERR_ARG, "null argument");
        MC3D_CUDA_TRY(cudaMemcpyAsync(s->spg_avg[v], avg[v], (size_t)s->g.n() * 8, cudaMemcpyHostToDevice, s->stream));
    }
    MC3D_CUDA_TRY(cudaStreamSynchronize(s->stream));
    return MC3D_OK;
}

// postStep's Stats::updateStatsFields (src/CurvilinearCSolver.hpp:362-364,
// src/Stats.cpp:127-223): time weights from the device time, fields on device.
static int stats_update(mc3d_solver s) {
    mc3d::TimeState t;
    MC3D_CUDA_TRY(cudaMemcpyAsync(&t, s->ts, sizeof(t), cudaMemcpyDeviceToHost, s->stream));
    MC3D_CUDA_TRY(cudaStreamSynchronize(s->stream));
    const double dt = t.time - s->st_prev;
    if (dt != 0.0) {
        mc3d::StatsIn in{};
        for (int v = 0; v < 5; v++) in.q[v] = s->q1[v];
        in.rho2 = s->q2[0];
        double *v9[9], *t6[6];
        for (int k = 0; k < 9; k++) v9[k] = s->stv[k];
        for (int k = 0; k < 6; k++) t6[k] = s->stt[k];
        int rc = mc3d::launch_stats_update(s->g, in, v9, t6, dt, s->st_vw, s->st_tw, s->cfg.stats_avg_type,
                                           s->cfg.velocity_stats, s->cfg.thermo_stats, s->stream);
        if (rc) return rc;
        if (s->cfg.velocity_stats) s->st_vw += dt;
        if (s->cfg.thermo_stats) s->st_tw += dt;
    }
    s->st_prev = t.time;
    return MC3D_OK;
}

}  // extern "C"

namespace mc3d {

// postStep (src/CurvilinearCSolver.hpp:355-375). The statistics read the
// primitives of the filtered state and rho2, neither of which the sponge
// relaxation changes, so they are updated first.
static int step_end(mc3d_solver s) {
    int rc;
    if (s->cfg.rk_type == MC3D_LSLDDRK4) s->lsldd_half = s->lsldd_half == 1 ? 2 : 1;
    if ((s->cfg.velocity_stats || s->cfg.thermo_stats) && s->host_time_step % s->cfg.stats_interval == 0)
        if ((rc = ::stats_update(s))) return rc;
    if (s->cfg.sponge_relax && s->have_sponge) {
        // updateSponge changes rho1..rhoE1 alone: the primitives, and with
        // them the next step's CFL and stage-1 derivatives, stay those of the
        // filtered state, so they are formed before the relaxation
        if ((rc = s->prec == MC3D_FP64 ? primitives_cfl<double>(s) : primitives_cfl<float>(s))) return rc;
        s->prims_ready = true;
        s->launches++;
        if ((rc = launch_sponge_relax(s->g, s->q1, s->spg_avg, s->ts, s->cfg.sponge_avg_time, s->cfg.sponge_p_inf,
                                      sponge_faces(s), s->stream)))
            return rc;
    }
    return MC3D_OK;
}
constexpr int HOOK_BLOCKS = 148 * 4;

template <typename R>
static int turbdata_impl(mc3d_solver s, double k0, double out[11]) {
    int rc;
    if (!s->hook_scratch && (rc = salloc(s, (void **)&s->hook_scratch, (size_t)TURB_NSUM * HOOK_BLOCKS * 8))) return rc;
    // the driver's computeGradient of U, V, W of the current (filtered) state
    if ((rc = primitives<R>(s, s->q1))) return rc;
    for (int d = 0; d < 3; d++) {
        void *o[3] = {s->der[0 + d], s->der[3 + d], s->der[6 + d]};
        if ((rc = sweep<R>(s, d, s->dop[d], 3, s->prim + 1, o, EPI_STORE, nullptr, nullptr, false))) return rc;
    }
    const R *pr[5], *dd[12];
    for (int v = 0; v < 5; v++) pr[v] = (const R *)s->prim[v];
    for (int k = 0; k < 12; k++) dd[k] = (const R *)s->der[k];
    Metrics<R> m = metrics_of<R>(s);
    const double nall = (double)s->g.n();
    std::vector<double> part((size_t)TURB_NSUM * HOOK_BLOCKS);
    double sum1[TURB_NSUM] = {0}, sum2[3] = {0};
    for (int pass = 1; pass <= 2; pass++) {
        const double mean_rho = sum1[0] / nall;
        if ((rc = launch_turb_sums<R>(s->g, pr, dd, m, s->cfg.mu_ref, pass, mean_rho, s->hook_scratch, HOOK_BLOCKS,
                                      s->stream)))
            return rc;
        const int nk = pass == 1 ? TURB_NSUM : 3;
        MC3D_CUDA_TRY(cudaMemcpyAsync(part.data(), s->hook_scratch, (size_t)nk * HOOK_BLOCKS * 8,
                                      cudaMemcpyDeviceToHost, s->stream));
        MC3D_CUDA_TRY(cudaStreamSynchronize(s->stream));
        for (int k = 0; k < nk; k++)
            for (int b = 0; b < HOOK_BLOCKS; b++) (pass == 1 ? sum1 : sum2)[k] += part[(size_t)k * HOOK_BLOCKS + b];
    }
    TimeState t;
    MC3D_CUDA_TRY(cudaMemcpy(&t, s->ts, sizeof(t), cudaMemcpyDeviceToHost));
    // tests/hit/Samtaney_D4/MPI_3DCompact.cpp:522-555
    const double meanRho = sum1[0] / nall, meanMu = sum1[1] / nall;
    const double meanTurbDiss = (sum1[2] / nall) / meanRho;
    const double uprime = std::sqrt(sum1[3] / nall), uiprime = std::sqrt(sum1[4] / nall);
    const double urms = std::sqrt(sum1[5] / nall), meanSOS = sum1[6] / nall;
    const double meanKE = sum1[8] / nall;
    const double rhoprime = std::sqrt(sum2[0] / nall), dilprime = std::sqrt(sum2[1] / nall);
    const double vortprime = std::sqrt(sum2[2] / nall);
    const double meanNu = meanMu / meanRho;
    const double taylorMicro = uprime / uiprime;
    const double pi = 3.14159265358979323846;
    out[0] = t.time;
    out[1] = std::sqrt(2 * pi) / k0 / uprime;
    out[2] = uprime * taylorMicro / meanNu;
    out[3] = urms / meanSOS;
    out[4] = meanTurbDiss;
    out[5] = uprime;
    out[6] = std::pow(std::pow(meanNu, 3.0) / meanTurbDiss, 0.25);
    out[7] = rhoprime;
    out[8] = dilprime;
    out[9] = vortprime;
    out[10] = meanKE;
    return MC3D_OK;
}
}  // namespace mc3d

extern "C" {

int mc3d_solver_turbdata(mc3d_solver s, double k0, double out[11]) {
    if (!s || !out) return fail(MC3D_ERR_ARG, "null argument");
    if (!s->initialized) return fail(MC3D_ERR_CONFIG, "no state");
    if (s->lean) return fail(MC3D_ERR_CONFIG, "turbdata needs the full-field gradients of GPU.STORAGE = FULL");
    MC3D_CUDA_TRY(cudaSetDevice(s->device));
    return s->prec == MC3D_FP64 ? mc3d::turbdata_impl<double>(s, k0, out) : mc3d::turbdata_impl<float>(s, k0, out);
}

int mc3d_solver_wall_span_average(mc3d_solver s, double *p, double *U, double *V, double *W) {
    if (!s || !p || !U || !V || !W) return fail(MC3D_ERR_ARG, "null argument");
    if (!s->initialized) return fail(MC3D_ERR_CONFIG, "no state");
    MC3D_CUDA_TRY(cudaSetDevice(s->device));
    int rc;
    const size_t need = (size_t)4 * s->g.Nx;
    double *buf = nullptr;
    MC3D_CUDA_TRY(cudaMallocAsync((void **)&buf, need * 8, s->stream));
    if ((rc = mc3d::launch_wall_span_average(s->g, s->q1, buf, s->stream))) {
        cudaFreeAsync(buf, s->stream);
        return rc;
    }
    double *dst[4] = {p, U, V, W};
    for (int k = 0; k < 4; k++)
        MC3D_CUDA_TRY(cudaMemcpyAsync(dst[k], buf + (size_t)k * s->g.Nx, s->g.Nx * 8, cudaMemcpyDeviceToHost, s->stream));
    MC3D_CUDA_TRY(cudaFreeAsync(buf, s->stream));
    MC3D_CUDA_TRY(cudaStreamSynchronize(s->stream));
    return MC3D_OK;
}

int mc3d_solver_wake_strip(mc3d_solver s, int i, int j, double *V) {
    if (!s || !V) return fail(MC3D_ERR_ARG, "null argument");
    if (!s->initialized) return fail(MC3D_ERR_CONFIG, "no state");
    if (i < 0 || i >= s->g.Nx || j < 0 || j >= s->g.Ny) return fail(MC3D_ERR_ARG, "strip point outside the grid");
    MC3D_CUDA_TRY(cudaSetDevice(s->device));
    int rc;
    double *buf = nullptr;
    MC3D_CUDA_TRY(cudaMallocAsync((void **)&buf, (size_t)s->g.Nz * 8, s->stream));
    if ((rc = mc3d::launch_wake_strip(s->g, s->q1, i, j, buf, s->stream))) {
        cudaFreeAsync(buf, s->stream);
        return rc;
    }
    MC3D_CUDA_TRY(cudaMemcpyAsync(V, buf, (size_t)s->g.Nz * 8, cudaMemcpyDeviceToHost, s->stream));
    MC3D_CUDA_TRY(cudaFreeAsync(buf, s->stream));
    MC3D_CUDA_TRY(cudaStreamSynchronize(s->stream));
    return MC3D_OK;
}

int mc3d_solver_get_stats(mc3d_solver s, double *const velocity[9], double *const thermo[6], double weights[2]) {
    if (!s) return fail(MC3D_ERR_ARG, "null solver");
    MC3D_CUDA_TRY(cudaSetDevice(s->device));
    const size_t bytes = (size_t)s->g.n() * sizeof(double);
    for (int k = 0; k < 9 && velocity; k++) {
        if (!velocity[k]) continue;
        if (!s->cfg.velocity_stats) return fail(MC3D_ERR_CONFIG, "VELOCITYSTATS is off");
        MC3D_CUDA_TRY(cudaMemcpyAsync(velocity[k], s->stv[k], bytes, cudaMemcpyDeviceToHost, s->stream));
    }
    for (int k = 0; k < 6 && thermo; k++) {
        if (!thermo[k]) continue;
        if (!s->cfg.thermo_stats) return fail(MC3D_ERR_CONFIG, "THERMOSTATS is off");
        MC3D_CUDA_TRY(cudaMemcpyAsync(thermo[k], s->stt[k], bytes, cudaMemcpyDeviceToHost, s->stream));
    }
    MC3D_CUDA_TRY(cudaStreamSynchronize(s->stream));
    if (weights) {
        weights[0] = s->st_vw;
        weights[1] = s->st_tw;
    }
    return MC3D_OK;
}

// Stats::dumpStatsFields (src/Stats.cpp:3-125): the weight, then the fields
static int write_stats_file(const std::string &path, double w, double *const *dev, int nf, size_t n,
                            cudaStream_t st) {
    std::vector<double> h(n);
    FILE *f = std::fopen(path.c_str(), "wb");
    if (!f) return fail(MC3D_ERR_ARG, "cannot write " + path);
    bool ok = std::fwrite(&w, sizeof(double), 1, f) == 1;
    for (int k = 0; k < nf && ok; k++) {
        if (cudaMemcpyAsync(h.data(), dev[k], n * sizeof(double), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess) {
            std::fclose(f);
            return fail(MC3D_ERR_CUDA, "stats download failed");
        }
        ok = std::fwrite(h.data(), sizeof(double), n, f) == n;
    }
    std::fclose(f);
    return ok ? MC3D_OK : fail(MC3D_ERR_ARG, "write failed: " + path);
}

static int read_stats_file(const std::string &path, double &w, double *const *dev, int nf, size_t n,
                           cudaStream_t st) {
    std::vector<double> h(n);
    FILE *f = std::fopen(path.c_str(), "rb");
    if (!f) return fail(MC3D_ERR_ARG, "ERROR: Couldn't open file " + path);
    bool ok = std::fread(&w, sizeof(double), 1, f) == 1;
    for (int k = 0; k < nf && ok; k++) {
        ok = std::fread(h.data(), sizeof(double), n, f) == n;
        if (ok && (cudaMemcpyAsync(dev[k], h.data(), n * sizeof(double), cudaMemcpyHostToDevice, st) != cudaSuccess ||
                   cudaStreamSynchronize(st) != cudaSuccess)) {
            std::fclose(f);
            return fail(MC3D_ERR_CUDA, "stats upload failed");
        }
    }
    std::fclose(f);
    return ok ? MC3D_OK : fail(MC3D_ERR_ARG, "short file: " + path);
}

int mc3d_solver_dump_stats(mc3d_solver s, const char *velocity_path, const char *thermo_path) {
    if (!s) return fail(MC3D_ERR_ARG, "null solver");
    MC3D_CUDA_TRY(cudaSetDevice(s->device));
    int ts;
    int rc = mc3d_solver_info(s, &ts, nullptr, nullptr, nullptr);
    if (rc) return rc;
    const size_t n = (size_t)s->g.n();
    if (s->cfg.velocity_stats) {
        const std::string p = velocity_path ? velocity_path : "VelocityStats." + std::to_string(ts);
        if ((rc = write_stats_file(p, s->st_vw, s->stv, 9, n, s->stream))) return rc;
    }
    if (s->cfg.thermo_stats) {
        const std::string p = thermo_path ? thermo_path : "ThermoStats." + std::to_string(ts);
        if ((rc = write_stats_file(p, s->st_tw, s->stt, 6, n, s->stream))) return rc;
    }
    return MC3D_OK;
}

int mc3d_solver_read_stats(mc3d_solver s, const char *velocity_path, const char *thermo_path) {
    if (!s) return fail(MC3D_ERR_ARG, "null solver");
    MC3D_CUDA_TRY(cudaSetDevice(s->device));
    const size_t n = (size_t)s->g.n();
    int rc;
    if (velocity_path) {
        if (!s->cfg.velocity_stats) return fail(MC3D_ERR_CONFIG, "VELOCITYSTATS is off");
        if ((rc = read_stats_file(velocity_path, s->st_vw, s->stv, 9, n, s->stream))) return rc;
    }
    if (thermo_path) {
        if (!s->cfg.thermo_stats) return fail(MC3D_ERR_CONFIG, "THERMOSTATS is off");
        if ((rc = read_stats_file(thermo_path, s->st_tw, s->stt, 6, n, s->stream))) return rc;
    }
    return MC3D_OK;
}

int mc3d_solver_step(mc3d_solver s, int nsteps) {
    if (!s) return fail(MC3D_ERR_ARG, "null solver");
    if (!s->initialized) return fail(MC3D_ERR_CONFIG, "no initial condition");
    if (s->cfg.les_model == MC3D_MLPSGS && !s->mlp) return fail(MC3D_ERR_CONFIG, "LESMODEL = MLP needs mc3d_solver_set_mlp");
    MC3D_CUDA_TRY(cudaSetDevice(s->device));
    if (s->phase != 0) return fail(MC3D_ERR_CONFIG, "a time step driven stage by stage is in progress");
    for (int i = 0; i < nsteps; i++) {
        int rc = s->prec == MC3D_FP64 ? one_step<double>(s) : one_step<float>(s);
        if (rc) return rc;
    }
    return MC3D_OK;
}

// ---- stage-level driving: the calls AbstractRK::executeSolverLoop makes ----
// Phases of a time step: 0 between steps, 1 ready for a stage's preSubStep,
// 2 preSubStep done, 3 solveEqnSet done, 4 postSubStep done, 5 RK update done,
// 6 last stage done (postStep next).
static int stage_ready(mc3d_solver s, int phase, const char *what) {
    if (!s) return fail(MC3D_ERR_ARG, "null solver");
    if (!s->initialized) return fail(MC3D_ERR_CONFIG, "no initial condition");
    if (s->cfg.les_model == MC3D_MLPSGS && !s->mlp) return fail(MC3D_ERR_CONFIG, "LESMODEL = MLP needs mc3d_solver_set_mlp");
    if (s->phase != phase)
        return fail(MC3D_ERR_CONFIG, std::string(what) + " out of order (the reference's RK loop order is preStep, "
                                     "then per stage preSubStep, solveEqnSet, postSubStep, updateConservedData, "
                                     "updateData, then postStep)");
    MC3D_CUDA_TRY(cudaSetDevice(s->device));
    return MC3D_OK;
}

int mc3d_solver_pre_step(mc3d_solver s) {
    if (int rc = stage_ready(s, 0, "preStep")) return rc;
    int rc = s->prec == MC3D_FP64 ? step_begin<double>(s) : step_begin<float>(s);
    if (rc) return rc;
    s->phase = 1;
    return MC3D_OK;
}

int mc3d_solver_stage_count(mc3d_solver s, int *stages) {
    if (!s || !stages) return fail(MC3D_ERR_ARG, "null argument");
    *stages = s->phase == 0 ? stages_of(s) : s->cur_ns;
    return MC3D_OK;
}

int mc3d_solver_pre_substep(mc3d_solver s, int rk_step) {
    if (int rc = stage_ready(s, 1, "preSubStep")) return rc;
    if (rk_step != s->cur_stage + 1 || rk_step > s->cur_ns)
        return fail(MC3D_ERR_CONFIG, "preSubStep: rkStep " + std::to_string(rk_step) + " where stage " +
                                         std::to_string(s->cur_stage + 1) + " of " + std::to_string(s->cur_ns) +
                                         " is next");
    int rc = s->prec == MC3D_FP64 ? stage_begin<double>(s, rk_step) : stage_begin<float>(s, rk_step);
    if (rc) return rc;
    s->cur_stage = rk_step;
    s->phase = 2;
    return MC3D_OK;
}

int mc3d_solver_solve_eqn_set(mc3d_solver s) {
    if (int rc = stage_ready(s, 2, "solveEqnSet")) return rc;
    int rc = s->prec == MC3D_FP64 ? stage_solve<double>(s) : stage_solve<float>(s);
    if (rc) return rc;
    s->phase = 3;
    return MC3D_OK;
}

int mc3d_solver_post_substep(mc3d_solver s) {
    if (int rc = stage_ready(s, 3, "postSubStep")) return rc;
    int rc = s->prec == MC3D_FP64 ? stage_post<double>(s) : stage_post<float>(s);
    if (rc) return rc;
    s->phase = 4;
    return MC3D_OK;
}

int mc3d_rk_update(mc3d_solver s, int scheme, int rk_step, int dual_step) {
    if (int rc = stage_ready(s, 4, "updateConservedData")) return rc;
    if (scheme != s->cfg.rk_type)
        return fail(MC3D_ERR_CONFIG, "updateConservedData: the RK scheme differs from the solver's RKTYPE");
    if (rk_step != s->cur_stage) return fail(MC3D_ERR_CONFIG, "updateConservedData: rkStep is not the current stage");
    if (scheme == MC3D_LSLDDRK4 && dual_step != s->lsldd_half)
        return fail(MC3D_ERR_CONFIG, "updateConservedData: LSLDDRK4 dual step " + std::to_string(dual_step) +
                                         " where " + std::to_string(s->lsldd_half) + " is current");
    int rc = s->prec == MC3D_FP64 ? stage_rk<double>(s, rk_step) : stage_rk<float>(s, rk_step);
    if (rc) return rc;
    s->phase = 5;
    return MC3D_OK;
}

int mc3d_solver_update_data(mc3d_solver s, int rk_last) {
    if (int rc = stage_ready(s, 5, "updateData")) return rc;
    if ((rk_last != 0) != (s->cur_stage == s->cur_ns))
        return fail(MC3D_ERR_CONFIG, "updateData: rkLast disagrees with the scheme's stage count");
    int rc = s->prec == MC3D_FP64 ? stage_end<double>(s, s->cur_stage) : stage_end<float>(s, s->cur_stage);
    if (rc) return rc;
    s->phase = rk_last ? 6 : 1;
    return MC3D_OK;
}

int mc3d_solver_post_step(mc3d_solver s) {
    if (int rc = stage_ready(s, 6, "postStep")) return rc;
    int rc = step_end(s);
    if (rc) return rc;
    s->phase = 0;
    return MC3D_OK;
}

int mc3d_solver_get_conserved(mc3d_solver s, double *rho, double *rhoU, double *rhoV, double *rhoW, double *rhoE) {
    if (!s) return fail(MC3D_ERR_ARG, "null solver");
    MC3D_CUDA_TRY(cudaSetDevice(s->device));
    double *dst[5] = {rho, rhoU, rhoV, rhoW, rhoE};
    size_t n = (size_t)s->g.n();
    for (int v = 0; v < 5; v++)
        if (dst[v]) MC3D_CUDA_TRY(cudaMemcpyAsync(dst[v], s->q1[v], n * 8, cudaMemcpyDeviceToHost, s->stream));
    MC3D_CUDA_TRY(cudaStreamSynchronize(s->stream));
    TimeState t;
    MC3D_CUDA_TRY(cudaMemcpy(&t, s->ts, sizeof(t), cudaMemcpyDeviceToHost));
    if (t.nonfinite) return fail(MC3D_ERR_NONFINITE, "the state became non-finite");
    if (int rc_tma = tma_timeouts_failed(s)) return rc_tma;
    return MC3D_OK;
}

int mc3d_solver_copy_conserved_device(mc3d_solver s, double *const dst[5]) {
    if (!s || !dst) return fail(MC3D_ERR_ARG, "null argument");
    MC3D_CUDA_TRY(cudaSetDevice(s->device));
    size_t n = (size_t)s->g.n();
    for (int v = 0; v < 5; v++)
        if (dst[v]) MC3D_CUDA_TRY(cudaMemcpyAsync(dst[v], s->q1[v], n * 8, cudaMemcpyDeviceToDevice, s->stream));
    MC3D_CUDA_TRY(cudaStreamSynchronize(s->stream));
    return MC3D_OK;
}

int mc3d_solver_conserved_device(mc3d_solver s, double *ptrs[5]) {
    if (!s || !ptrs) return fail(MC3D_ERR_ARG, "null argument");
    for (int v = 0; v < 5; v++) ptrs[v] = s->q1[v];
    return MC3D_OK;
}

// ---- checkpoints and the driver loop ------------------------------------------

// The time origin of a (re)start: time step and time of the state, the counters
// a fresh solver starts with (src/MPI_3DCompact.cpp:99-101 sets opt->timeStep
// and opt->time, which the solver takes over in its constructor,
// src/CurvilinearCSolver.hpp:147-148).
static int set_time_origin(mc3d_solver s, int time_step, double time) {
    s->cfg.time_step0 = time_step;
    s->cfg.time0 = time;
    s->st_prev = time;
    s->host_time_step = time_step;
    s->filter_time_step = 0;
    s->lsldd_half = 1;
    mc3d::TimeState t{};
    t.time = time;
    t.time_step = time_step;
    t.dt = s->cfg.ts_type == MC3D_CONST_DT ? s->cfg.dt : 0.0;
    MC3D_CUDA_TRY(cudaMemcpyAsync(s->ts, &t, sizeof(t), cudaMemcpyHostToDevice, s->stream));
    MC3D_CUDA_TRY(cudaStreamSynchronize(s->stream));
    return MC3D_OK;
}

int mc3d_solver_dump(mc3d_solver s, const char *path, const double *x, const double *y, const double *z) {
    if (!s) return fail(MC3D_ERR_ARG, "null solver");
    if (!s->initialized) return fail(MC3D_ERR_CONFIG, "no state to dump");
    MC3D_CUDA_TRY(cudaSetDevice(s->device));
    const size_t n = (size_t)s->g.n();
    std::vector<double> q[5], box[3];
    for (auto &v : q) v.resize(n);
    int rc = mc3d_solver_get_conserved(s, q[0].data(), q[1].data(), q[2].data(), q[3].data(), q[4].data());
    if (rc) return rc;
    int ts;
    double time;
    if ((rc = mc3d_solver_info(s, &ts, &time, nullptr, nullptr))) return rc;
    const double *xyz[3] = {x, y, z};
    if (!x || !y || !z) {
        if (s->mesh_kind == 1) {
            for (int c = 0; c < 3; c++) xyz[c] = s->mesh_xyz[c].data();
        } else if (s->mesh_kind == 2) {
            // the box x = L*xi with Domain's xi (src/Domain.hpp:44-56)
            const int N[3] = {s->g.Nx, s->g.Ny, s->g.Nz};
            for (int c = 0; c < 3; c++) {
                std::vector<double> xi(N[c]);
                for (int i = 0; i < N[c]; i++)
                    xi[i] = s->cfg.bc_type[c] == MC3D_PERIODIC_SOLVE ? (double)i * 1.0 / (double)N[c]
                                                                     : ((double)i / ((double)N[c] - 1.0)) * 1.0;
                box[c].resize(n);
                for (int k = 0; k < s->g.Nz; k++)
                    for (int j = 0; j < s->g.Ny; j++)
                        for (int i = 0; i < s->g.Nx; i++) {
                            const int ix[3] = {i, j, k};
                            box[c][i + (size_t)s->g.Nx * (j + (size_t)s->g.Ny * k)] = s->box_L[c] * xi[ix[c]];
                        }
                xyz[c] = box[c].data();
            }
        } else {
            return fail(MC3D_ERR_CONFIG, "no mesh: pass x, y, z (metrics were given directly)");
        }
    }
    const std::string name = path ? std::string(path) : "SolutionDump." + std::to_string(ts);
    const double *f[8] = {xyz[0], xyz[1], xyz[2], q[0].data(), q[1].data(), q[2].data(), q[3].data(), q[4].data()};
    return write_solution_dump(name.c_str(), ts, time, s->g.Nx, s->g.Ny, s->g.Nz, f);
}

int mc3d_solver_restart(mc3d_solver s, const char *path, int grid_only) {
    if (!s || !path) return fail(MC3D_ERR_ARG, "null argument");
    int ts, Nx, Ny, Nz;
    double time;
    int rc = read_solution_header(path, &ts, &time, &Nx, &Ny, &Nz);
    if (rc) return rc;
    if (Nx != s->g.Nx || Ny != s->g.Ny || Nz != s->g.Nz)
        return fail(MC3D_ERR_CONFIG, std::string("grid of ") + path + " differs from the solver's");
    const long long n = s->g.n();
    std::vector<double> f[8];
    double *fp[8];
    for (int k = 0; k < 8; k++) {
        if (grid_only && k >= 3) {
            fp[k] = nullptr;
            continue;
        }
        f[k].resize((size_t)n);
        fp[k] = f[k].data();
    }
    if ((rc = read_solution_fields(path, n, fp))) return rc;
    // AlgebraicSingleBlockMesh::getMesh reads the grid of a restart (src/AlgebraicSingleBlockMesh.hpp:77-101)
    if ((rc = mc3d_solver_set_mesh(s, fp[0], fp[1], fp[2]))) return rc;
    if (s->have_sponge && !s->sigma_set) {
        // SpongeBC builds its strength field from the mesh (src/SpongeBC.cpp:65-189)
        std::vector<double> sig((size_t)n);
        if ((rc = mc3d_sponge_sigma(&s->cfg, fp[0], fp[1], fp[2], sig.data()))) return rc;
        if ((rc = mc3d_solver_set_sponge(s, sig.data()))) return rc;
    }
    if (grid_only) return MC3D_OK;
    // src/MPI_3DCompact.cpp:248-262 with IdealGas::solveU / solvep (src/IdealGas.hpp:58-64)
    const double gamma = 1.4;
    std::vector<double> U((size_t)n), V((size_t)n), W((size_t)n), p((size_t)n);
    for (long long i = 0; i < n; i++) {
        const double rho = f[3][i];
        U[i] = f[4][i] / rho;
        V[i] = f[5][i] / rho;
        W[i] = f[6][i] / rho;
        p[i] = (gamma - 1) * (f[7][i] - 0.5 * rho * (U[i] * U[i] + V[i] * V[i] + W[i] * W[i]));
    }
    MC3D_CUDA_TRY(cudaSetDevice(s->device));
    if ((rc = set_time_origin(s, ts, time))) return rc;
    return mc3d_solver_set_initial(s, f[3].data(), U.data(), V.data(), W.data(), p.data());
}

int mc3d_solver_dump_sponge_avg(mc3d_solver s, const char *path) {
    if (!s) return fail(MC3D_ERR_ARG, "null solver");
    if (!s->have_sponge) return fail(MC3D_ERR_CONFIG, "no face is a SPONGE");
    MC3D_CUDA_TRY(cudaSetDevice(s->device));
    const size_t n = (size_t)s->g.n();
    std::vector<double> a[5];
    const double *ap[5];
    for (int v = 0; v < 5; v++) {
        a[v].resize(n);
        MC3D_CUDA_TRY(cudaMemcpyAsync(a[v].data(), s->spg_avg[v], n * 8, cudaMemcpyDeviceToHost, s->stream));
        ap[v] = a[v].data();
    }
    MC3D_CUDA_TRY(cudaStreamSynchronize(s->stream));
    int ts;
    int rc = mc3d_solver_info(s, &ts, nullptr, nullptr, nullptr);
    if (rc) return rc;
    const std::string name = path ? std::string(path) : "SpongeAvgDump." + std::to_string(ts);
    return write_sponge_avg(name.c_str(), (long long)n, ap);
}

int mc3d_solver_read_sponge_avg(mc3d_solver s, const char *path) {
    if (!s || !path) return fail(MC3D_ERR_ARG, "null argument");
    const size_t n = (size_t)s->g.n();
    std::vector<double> a[5];
    double *ap[5];
    for (int v = 0; v < 5; v++) {
        a[v].resize(n);
        ap[v] = a[v].data();
    }
    int rc = read_sponge_avg(path, (long long)n, ap);
    if (rc) return rc;
    const double *cp[5] = {ap[0], ap[1], ap[2], ap[3], ap[4]};
    return mc3d_solver_set_sponge_avg(s, cp);
}

int mc3d_solver_start(mc3d_solver s) {
    if (!s) return fail(MC3D_ERR_ARG, "null solver");
    int rc = MC3D_OK;
    if (s->cfg.from_restart || s->cfg.only_grid_from_restart)
        rc = mc3d_solver_restart(s, s->cfg.restart_file, s->cfg.only_grid_from_restart);
    if (!rc && s->cfg.sponge_avg_from_restart) rc = mc3d_solver_read_sponge_avg(s, s->cfg.sponge_avg_file);
    if (!rc && (s->cfg.velocity_stats_from_restart || s->cfg.thermo_stats_from_restart))
        rc = mc3d_solver_read_stats(s, s->cfg.velocity_stats_from_restart ? s->cfg.velocity_stats_file : nullptr,
                                    s->cfg.thermo_stats_from_restart ? s->cfg.thermo_stats_file : nullptr);
    return rc;
}

int mc3d_solver_run(mc3d_solver s, const char *dir) {
    if (!s) return fail(MC3D_ERR_ARG, "null solver");
    const std::string base = dir ? std::string(dir) + "/" : std::string();
    auto dump = [&](int ts) -> int {
        int rc = mc3d_solver_dump(s, (base + "SolutionDump." + std::to_string(ts)).c_str(), nullptr, nullptr, nullptr);
        if (!rc && s->have_sponge)
            rc = mc3d_solver_dump_sponge_avg(s, (base + "SpongeAvgDump." + std::to_string(ts)).c_str());
        if (!rc && (s->cfg.velocity_stats || s->cfg.thermo_stats))
            rc = mc3d_solver_dump_stats(s, (base + "VelocityStats." + std::to_string(ts)).c_str(),
                                        (base + "ThermoStats." + std::to_string(ts)).c_str());
        return rc;
    };
    bool end = false;
    while (!end) {
        int rc = mc3d_solver_step(s, 1);
        if (rc) return rc;
        int ts;
        double time;
        if ((rc = mc3d_solver_info(s, &ts, &time, nullptr, nullptr))) return rc;
        // postStep (src/CurvilinearCSolver.hpp:367-369), then checkEnd (Core.cpp:1785-1824)
        if (ts % s->cfg.dump_step == 0 && (rc = dump(ts))) return rc;
        const std::string kill = base + "killsolver";
        if (FILE *kf = std::fopen(kill.c_str(), "r")) {
            std::fclose(kf);
            std::remove(kill.c_str());
            end = true;
        }
        if (time >= s->cfg.max_time || ts >= s->cfg.max_time_step) end = true;
        if (end && (rc = dump(ts))) return rc;
    }
    return MC3D_OK;
}

int mc3d_solver_info(mc3d_solver s, int *time_step, double *time, double *dt, long long *stages) {
    if (!s) return fail(MC3D_ERR_ARG, "null solver");
    MC3D_CUDA_TRY(cudaSetDevice(s->device));
    MC3D_CUDA_TRY(cudaStreamSynchronize(s->stream));
    TimeState t;
    MC3D_CUDA_TRY(cudaMemcpy(&t, s->ts, sizeof(t), cudaMemcpyDeviceToHost));
    if (time_step) *time_step = (int)t.time_step;
    if (time) *time = t.time;
    if (dt) *dt = t.dt;
    if (stages) *stages = s->stages;
    if (t.nonfinite) return fail(MC3D_ERR_NONFINITE, "the state became non-finite");
    if (int rc_tma = tma_timeouts_failed(s)) return rc_tma;
    return MC3D_OK;
}

int mc3d_solver_integrals(mc3d_solver s, double *kinetic, double *mass) {
    if (!s) return fail(MC3D_ERR_ARG, "null solver");
    MC3D_CUDA_TRY(cudaSetDevice(s->device));
    MC3D_CUDA_TRY(cudaMemsetAsync(s->acc, 0, 2 * sizeof(double), s->stream));
    int rc = launch_integrals(s->g, s->q1, s->acc, s->stream);
    if (rc) return rc;
    double h[2];
    MC3D_CUDA_TRY(cudaMemcpyAsync(h, s->acc, sizeof(h), cudaMemcpyDeviceToHost, s->stream));
    MC3D_CUDA_TRY(cudaStreamSynchronize(s->stream));
    if (kinetic) *kinetic = h[0];
    if (mass) *mass = h[1];
    return MC3D_OK;
}

int mc3d_solver_stream(mc3d_solver s, void **stream) {
    if (!s || !stream) return fail(MC3D_ERR_ARG, "null argument");
    *stream = (void *)s->stream;
    return MC3D_OK;
}

int mc3d_solver_set_stream(mc3d_solver s, void *stream) {
    if (!s) return fail(MC3D_ERR_ARG, "null solver");
    MC3D_CUDA_TRY(cudaSetDevice(s->device));
    MC3D_CUDA_TRY(cudaStreamSynchronize(s->stream));
    if (stream) {
        s->stream = (cudaStream_t)stream;
        return MC3D_OK;
    }
    cudaError_t e = device_stream(s->device, &s->stream);
    if (e != cudaSuccess) return fail(MC3D_ERR_CUDA, std::string("cudaStreamCreate: ") + cudaGetErrorString(e));
    return MC3D_OK;
}

int mc3d_solver_launch_count(mc3d_solver s, long long *count) {
    if (!s || !count) return fail(MC3D_ERR_ARG, "null argument");
    *count = s->launches;
    return MC3D_OK;
}

int mc3d_solver_set_timing(mc3d_solver s, int enable) {
    if (!s) return fail(MC3D_ERR_ARG, "null solver");
    MC3D_CUDA_TRY(cudaSetDevice(s->device));
    MC3D_CUDA_TRY(cudaStreamSynchronize(s->stream));
    s->timing = enable != 0;
    s->recs.clear();
    s->ev_used = 0;
    return MC3D_OK;
}

const char *mc3d_solver_timing_report(mc3d_solver s) {
    if (!s) {
        fail(MC3D_ERR_ARG, "null solver");
        return nullptr;
    }
    cudaSetDevice(s->device);
    if (cudaStreamSynchronize(s->stream) != cudaSuccess) {
        fail(MC3D_ERR_CUDA, "stream synchronisation failed");
        return nullptr;
    }
    double ms[KC_COUNT] = {0}, by[KC_COUNT] = {0};
    long long cnt[KC_COUNT] = {0};
    for (const auto &r : s->recs) {
        float t = 0;
        if (cudaEventElapsedTime(&t, s->events[r.ev], s->events[r.ev + 1]) != cudaSuccess) continue;
        ms[r.cls] += t;
        by[r.cls] += r.bytes;
        cnt[r.cls]++;
    }
    std::string o = "{";
    char buf[256];
    bool firstk = true;
    for (int c = 0; c < KC_COUNT; c++) {
        if (!cnt[c]) continue;
        snprintf(buf, sizeof(buf), "%s\"%s\": {\"launches\": %lld, \"ms\": %.6f, \"bytes\": %.6e}", firstk ? "" : ", ",
                 KC_NAME[c], cnt[c], ms[c], by[c]);
        o += buf;
        firstk = false;
    }
    o += "}";
    s->report = o;
    return s->report.c_str();
}

}  // extern "C"

// ---- SGS models on their own: the AbstractSGS drop-in ----
// The object keeps an internal solver record that holds only what the SGS
// kernels read: the model settings, the test-filter and averaging operators,
// the work fields, and metrics whose J_ij factors are the identity (so the
// kernels take the caller's physical gradients as they are) and whose J is
// the caller's.
struct mc3d_sgs_s {
    mc3d_solver rec = nullptr;
    cudaStream_t home = nullptr;   // the record's own stream, restored after each call
    void *taukk_own = nullptr;
};

extern "C" {

int mc3d_sgs_create(int model, int averaging, int test_filter, int use_taukk, int Nx, int Ny, int Nz,
                    const int bc_types[3], const double dxi[3], const void *J, double Jc, int precision, int device,
                    mc3d_sgs *out) {
    if (!out || !bc_types || !dxi) return fail(MC3D_ERR_ARG, "null argument");
    *out = nullptr;
    if (model != MC3D_VREMAN && model != MC3D_DSM && model != MC3D_MLPSGS)
        return fail(MC3D_ERR_CONFIG, "model must be VREMAN, DSM or MLP");
    if (averaging < MC3D_AVG_NONE || averaging > MC3D_AVG_GLOBAL) return fail(MC3D_ERR_CONFIG, "unknown LESAVERAGING");
    if (model == MC3D_DSM && test_filter != 1 && test_filter != 2)
        return fail(MC3D_ERR_CONFIG, "DSMTESTFILTER must be 1 or 2");
    if (precision != MC3D_FP64 && precision != MC3D_FP32BULK) return fail(MC3D_ERR_CONFIG, "bad precision");
    if (Nx <= 10 || Ny <= 10 || Nz <= 10)
        return fail(MC3D_ERR_CONFIG, "Number of grid points in any direction must be greater than 10");
    for (int d = 0; d < 3; d++)
        if (!(dxi[d] > 0)) return fail(MC3D_ERR_ARG, "dxi must be positive");
    if (!J && !(Jc != 0.0)) return fail(MC3D_ERR_ARG, "J: a field or a nonzero constant");
    MC3D_CUDA_TRY(cudaSetDevice(device));
    mc3d_sgs o = new mc3d_sgs_s();
    mc3d_solver s = new mc3d_solver_s();
    o->rec = s;
    mc3d_config_default(&s->cfg);
    s->cfg.Nx = Nx;
    s->cfg.Ny = Ny;
    s->cfg.Nz = Nz;
    s->cfg.les_model = model;
    s->cfg.les_averaging = averaging;
    s->cfg.dsm_test_filter = test_filter;
    s->cfg.dsm_use_taukk = use_taukk != 0;
    s->cfg.precision = precision;
    for (int d = 0; d < 3; d++) s->cfg.bc_type[d] = bc_types[d];
    s->device = device;
    s->prec = precision;
    s->g = Grid3{Nx, Ny, Nz};
    for (int d = 0; d < 3; d++) s->dxi[d] = dxi[d];
    int rc = MC3D_OK;
    cudaError_t e = device_stream(device, &s->stream);
    if (e != cudaSuccess) rc = fail(MC3D_ERR_CUDA, std::string("cudaStreamCreate: ") + cudaGetErrorString(e));
    o->home = s->stream;
    const int N[3] = {Nx, Ny, Nz};
    try {
        for (int d = 0; d < 3 && !rc && model != MC3D_MLPSGS; d++) {
            if (model == MC3D_VREMAN) {
                // VremanSGS averages with Compact10 filters of alpha -0.49 (src/VremanSGS.hpp:38-40)
                rc = upload_line_op(build_filter_op(MC3D_COMPACT10, -0.49, bc_types[d], N[d]), precision, s->vop[d]);
            } else {
                // DSMTESTFILTER 1 -> Pade, 2 -> explicit (src/DSMSGS.hpp:57-67)
                rc = upload_line_op(build_testfilter_op(test_filter == 1 ? MC3D_TESTFILTER_PADE : MC3D_TESTFILTER_EXP,
                                                        bc_types[d], N[d]),
                                    precision, s->top[d]);
            }
        }
    } catch (const std::exception &ex) {
        rc = fail(MC3D_ERR_CONFIG, ex.what());
    }
    const size_t n = (size_t)s->g.n(), rb = precision == MC3D_FP64 ? 8 : 4;
    for (int v = 0; v < 5 && !rc; v++) rc = salloc(s, &s->prim[v], n * rb);
    if (!rc) rc = salloc(s, (void **)&s->avg_scratch, AVG_SCRATCH * sizeof(double));
    if (model == MC3D_VREMAN && !rc) rc = salloc(s, &s->tA[0], n * rb);
    if (model == MC3D_DSM) {
        for (int i = 0; i < 24 && !rc; i++) rc = salloc(s, &s->dA[i], n * rb);
        for (int i = 0; i < 24 && !rc; i++) rc = salloc(s, &s->dB[i], n * rb);
        if (!rc) rc = salloc(s, &s->smag, n * rb);
        if (!rc) rc = salloc(s, &o->taukk_own, n * rb);
    }
    if (model == MC3D_MLPSGS) {
        if (!rc) rc = salloc(s, (void **)&s->mlp_flag, sizeof(int));
        if (!rc && cudaMallocHost((void **)&s->mlp_flag_host, sizeof(int)) != cudaSuccess)
            rc = fail(MC3D_ERR_OOM, "cudaMallocHost");
    }
    // metrics: J_ij = identity, J from the caller
    s->const_met = J == nullptr;
    for (int c = 0; c < 10; c++) s->met_c[c] = 0.0;
    s->met_c[0] = J ? 1.0 : Jc;
    s->met_c[1] = s->met_c[5] = s->met_c[9] = 1.0;
    if (J && !rc) {
        void *ones = nullptr, *zeros = nullptr;
        rc = salloc(s, &zeros, n * rb);
        if (!rc) rc = salloc(s, &ones, n * rb);
        if (!rc) {
            std::vector<char> h(n * rb);
            if (precision == MC3D_FP64) std::fill((double *)h.data(), (double *)h.data() + n, 1.0);
            else std::fill((float *)h.data(), (float *)h.data() + n, 1.0f);
            e = cudaMemcpy(ones, h.data(), n * rb, cudaMemcpyHostToDevice);
            if (e != cudaSuccess) rc = fail(MC3D_ERR_CUDA, cudaGetErrorString(e));
        }
        for (int c = 1; c < 10 && !rc; c++) s->metR[c] = (c == 1 || c == 5 || c == 9) ? ones : zeros;
        s->metR[0] = const_cast<void *>(J);
    }
    if (!rc) {
        e = cudaStreamSynchronize(s->stream);
        if (e != cudaSuccess) rc = fail(MC3D_ERR_CUDA, cudaGetErrorString(e));
    }
    if (rc) {
        mc3d_sgs_destroy(o);
        return rc;
    }
    *out = o;
    return MC3D_OK;
}

int mc3d_sgs_destroy(mc3d_sgs o) {
    if (!o) return MC3D_OK;
    if (o->rec) {
        o->rec->stream = o->home;
        mc3d_solver_destroy(o->rec);
    }
    delete o;
    return MC3D_OK;
}

}  // extern "C"

template <typename R>
static int sgs_viscosity_t(mc3d_sgs o, const void *const gradU[9], const double *const q[5], void *mu_sgs) {
    mc3d_solver s = o->rec;
    int rc;
    R *pr[5];
    for (int v = 0; v < 5; v++) pr[v] = (R *)s->prim[v];
    if ((rc = launch_to_real<R>(s->g, q, pr, s->stream))) return rc;
    const R *dd[12];
    for (int i = 0; i < 12; i++) dd[i] = (const R *)gradU[i < 9 ? i : 0];
    FluxParams fp{};
    for (int d = 0; d < 3; d++) fp.dxi[d] = s->dxi[d];
    const R *prc[5] = {pr[0], pr[1], pr[2], pr[3], pr[4]};
    if ((rc = launch_vreman<R>(s->g, prc, dd, metrics_of<R>(s), fp, (R *)mu_sgs, s->stream))) return rc;
    void *a[1] = {mu_sgs}, *t1[1] = {s->tA[0]}, *res[1];
    if ((rc = sgs_average<R>(s, 1, a, t1, s->vop, res))) return rc;
    if (res[0] != mu_sgs)
        MC3D_CUDA_TRY(cudaMemcpyAsync(mu_sgs, res[0], (size_t)s->g.n() * sizeof(R), cudaMemcpyDeviceToDevice,
                                      s->stream));
    return MC3D_OK;
}

template <typename R>
static int sgs_mu_taukk_t(mc3d_sgs o, const void *const gradU[9], const double *const q[5], void *mu_sgs,
                          void *taukk) {
    mc3d_solver s = o->rec;
    for (int i = 0; i < 9; i++) s->der[i] = const_cast<void *>(gradU[i]);
    s->mu_sgs = mu_sgs;
    s->taukk = taukk ? taukk : o->taukk_own;
    s->cons_mask = 0;
    // (the kernel also forms the temperature of p - tau_kk / 2, which the
    // solver uses; here it lands in a work field)
    return dsm_mu_taukk<R>(s, const_cast<double *const *>(q), metrics_of<R>(s));
}

template <typename R>
static int sgs_ksgs_t(mc3d_sgs o, const void *const gradT[3], const double *const q[5], const void *T, void *k_sgs) {
    mc3d_solver s = o->rec;
    for (int i = 0; i < 3; i++) s->der[9 + i] = const_cast<void *>(gradT[i]);
    void *keep = s->prim[4];
    s->prim[4] = const_cast<void *>(T);
    s->ksgs = k_sgs;
    int rc = dsm_ksgs<R>(s, const_cast<double *const *>(q), metrics_of<R>(s));
    s->prim[4] = keep;
    return rc;
}

// the learned closure on the caller's gradients: calcMuSGSTaukk keeps the
// velocity gradients and the mu_sgs destination (tau_kk is zero), calcKSGS
// runs the fused closure kernel for both outputs
template <typename R>
static int sgs_mlp_mu_t(mc3d_sgs o, const void *const gradU[9], void *mu_sgs, void *taukk) {
    mc3d_solver s = o->rec;
    for (int i = 0; i < 9; i++) s->der[i] = const_cast<void *>(gradU[i]);
    s->mu_sgs = mu_sgs;
    if (taukk) MC3D_CUDA_TRY(cudaMemsetAsync(taukk, 0, (size_t)s->g.n() * sizeof(R), s->stream));
    return MC3D_OK;
}

template <typename R>
static int sgs_mlp_k_t(mc3d_sgs o, const void *const gradT[3], const double *const q[5], const void *T, void *k_sgs) {
    mc3d_solver s = o->rec;
    if (!s->mlp) return fail(MC3D_ERR_CONFIG, "no closure attached (mc3d_sgs_set_mlp)");
    if (!s->mu_sgs) return fail(MC3D_ERR_CONFIG, "calcKSGS of the learned closure needs calcMuSGSTaukk first");
    int rc;
    const double *src[5] = {q[0], nullptr, nullptr, nullptr, nullptr};
    R *dst[5] = {(R *)s->prim[0], nullptr, nullptr, nullptr, nullptr};
    if ((rc = launch_to_real<R>(s->g, src, dst, s->stream))) return rc;
    const R *dd[12];
    for (int i = 0; i < 9; i++) dd[i] = (const R *)s->der[i];
    for (int i = 0; i < 3; i++) dd[9 + i] = (const R *)gradT[i];
    MC3D_CUDA_TRY(cudaMemsetAsync(s->mlp_flag, 0, sizeof(int), s->stream));
    return launch_sgs_mlp<R>(s->g, (const R *)s->prim[0], (const R *)T, dd, metrics_of<R>(s),
                             s->dxi[0] * s->dxi[1] * s->dxi[2], s->cfg.mu_ref, *mlp_dev(s->mlp), (R *)s->mu_sgs,
                             (R *)k_sgs, s->mlp_flag, s->stream);
}

extern "C" {

int mc3d_sgs_set_mlp(mc3d_sgs o, mc3d_mlp mlp, double mu_ref) {
    if (!o || !mlp) return fail(MC3D_ERR_ARG, "null argument");
    if (o->rec->cfg.les_model != MC3D_MLPSGS) return fail(MC3D_ERR_CONFIG, "the SGS object's model is not MLP");
    if (!(mu_ref > 0)) return fail(MC3D_ERR_ARG, "mu_ref must be positive");
    o->rec->mlp = mlp;
    o->rec->cfg.mu_ref = mu_ref;
    return MC3D_OK;
}

int mc3d_sgs_mlp_out_of_range(mc3d_sgs o, long long *points) {
    if (!o || !points) return fail(MC3D_ERR_ARG, "null argument");
    mc3d_solver s = o->rec;
    if (s->cfg.les_model != MC3D_MLPSGS) return fail(MC3D_ERR_CONFIG, "the SGS object's model is not MLP");
    MC3D_CUDA_TRY(cudaSetDevice(s->device));
    MC3D_CUDA_TRY(cudaMemcpy(s->mlp_flag_host, s->mlp_flag, sizeof(int), cudaMemcpyDeviceToHost));
    *points = *s->mlp_flag_host;
    return MC3D_OK;
}

static int sgs_call(mc3d_sgs o, void *stream) {
    if (!o) return fail(MC3D_ERR_ARG, "null argument");
    MC3D_CUDA_TRY(cudaSetDevice(o->rec->device));
    o->rec->stream = (cudaStream_t)stream;
    return MC3D_OK;
}

int mc3d_sgs_get_viscosity(mc3d_sgs o, const void *const gradU[9], const double *const q[5], void *mu_sgs,
                           void *stream) {
    if (int rc = sgs_call(o, stream)) return rc;
    if (!gradU || !q || !mu_sgs) return fail(MC3D_ERR_ARG, "null argument");
    int rc = MC3D_OK;
    if (o->rec->cfg.les_model == MC3D_VREMAN)
        rc = o->rec->prec == MC3D_FP64 ? sgs_viscosity_t<double>(o, gradU, q, mu_sgs)
                                       : sgs_viscosity_t<float>(o, gradU, q, mu_sgs);
    o->rec->stream = o->home;
    return rc;
}

int mc3d_sgs_calc_mu_taukk(mc3d_sgs o, const void *const gradU[9], const double *const q[5], void *mu_sgs,
                           void *taukk, void *stream) {
    if (int rc = sgs_call(o, stream)) return rc;
    if (!gradU || !q || !mu_sgs) return fail(MC3D_ERR_ARG, "null argument");
    int rc = MC3D_OK;
    if (o->rec->cfg.les_model == MC3D_DSM)
        rc = o->rec->prec == MC3D_FP64 ? sgs_mu_taukk_t<double>(o, gradU, q, mu_sgs, taukk)
                                       : sgs_mu_taukk_t<float>(o, gradU, q, mu_sgs, taukk);
    if (o->rec->cfg.les_model == MC3D_MLPSGS)
        rc = o->rec->prec == MC3D_FP64 ? sgs_mlp_mu_t<double>(o, gradU, mu_sgs, taukk)
                                       : sgs_mlp_mu_t<float>(o, gradU, mu_sgs, taukk);
    o->rec->stream = o->home;
    return rc;
}

int mc3d_sgs_calc_ksgs(mc3d_sgs o, const void *const gradT[3], const double *const q[5], const void *T,
                       void *k_sgs, void *stream) {
    if (int rc = sgs_call(o, stream)) return rc;
    if (!gradT || !q || !T || !k_sgs) return fail(MC3D_ERR_ARG, "null argument");
    int rc = MC3D_OK;
    if (o->rec->cfg.les_model == MC3D_DSM)
        rc = o->rec->prec == MC3D_FP64 ? sgs_ksgs_t<double>(o, gradT, q, T, k_sgs)
                                       : sgs_ksgs_t<float>(o, gradT, q, T, k_sgs);
    if (o->rec->cfg.les_model == MC3D_MLPSGS)
        rc = o->rec->prec == MC3D_FP64 ? sgs_mlp_k_t<double>(o, gradT, q, T, k_sgs)
                                       : sgs_mlp_k_t<float>(o, gradT, q, T, k_sgs);
    o->rec->stream = o->home;
    return rc;
}

int mc3d_solver_sync(mc3d_solver s) {
    if (!s) return fail(MC3D_ERR_ARG, "null solver");
    MC3D_CUDA_TRY(cudaSetDevice(s->device));
    MC3D_CUDA_TRY(cudaStreamSynchronize(s->stream));
    return MC3D_OK;
}

}  // extern "C"
