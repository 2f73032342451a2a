/*
 * mc3d: B200-native CurvilinearCSolver time step (compact derivatives, compact
 * filtering, SGS model and RK stage update) behind a plain C ABI.
 *
 * Conventions
 *   - Every function returns an int status (MC3D_OK = 0) and never aborts the
 *     process; mc3d_last_error() returns the calling thread's last message.
 *   - Fields are 3-D arrays of Nx*Ny*Nz values in x-fastest order
 *     (index i + Nx*(j + Ny*k)), the global order of the reference's dumps
 *     (src/CurvilinearCSolver_Core.cpp:1333-1436).
 *   - "device" pointers live on the solver's / operator's CUDA device; "host"
 *     pointers are ordinary CPU memory.
 *   - Directions: 0 = xi1 (x), 1 = xi2 (y), 2 = xi3 (z), as
 *     AbstractDerivatives::Direct {DIRX, DIRY, DIRZ} (src/AbstractDerivatives.hpp:32).
 *
 * Reference interfaces each group replaces (paths within emathew1/MPI_3DCompact):
 *   mc3d_deriv_*   AbstractDerivatives (src/AbstractDerivatives.hpp:13-54):
 *                  calc1stDerivField(in, out) and calcNeumann(f); concrete
 *                  Pade6 (src/Pade6.hpp:11), Penta10 (src/Penta10.hpp:7),
 *                  CD2 (src/CD2.hpp).
 *   mc3d_filter_*  AbstractFilter (src/AbstractFilter.hpp:13-35): filterField(in,
 *                  out); Compact8Filter (src/Compact8Filter.hpp:9),
 *                  Compact10Filter (src/Compact10Filter.hpp:9).
 *   mc3d_solver_*  AbstractCSolver + CurvilinearCSolver (src/AbstractCSolver.hpp:14,
 *                  src/CurvilinearCSolver.hpp:25) driven by an AbstractRK
 *                  (src/AbstractRK.hpp:6): RK4, TVDRK3, KenRK4, LSLDDRK4, with
 *                  the AbstractSGS models (src/AbstractSGS.hpp:10) NOMODEL and
 *                  VREMAN.
 *   mc3d_config_*  Options (src/Options.hpp:13-598): the MPI_3DCompact.in keys.
 */
#ifndef MC3D_H
#define MC3D_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---- */
#define MC3D_OK 0
#define MC3D_ERR_CONFIG 1    /* invalid option or unsupported combination        */
#define MC3D_ERR_CUDA 2      /* a CUDA runtime call failed                        */
#define MC3D_ERR_NONFINITE 3 /* the state became NaN/Inf                          */
#define MC3D_ERR_OOM 4       /* device allocation failed                          */
#define MC3D_ERR_TIMEOUT 5   /* a bounded device wait gave up                     */
#define MC3D_ERR_ARG 6       /* null handle / bad argument                        */

/* ---- enumerations (values follow src/Options.hpp:19-37 where it has them) ---- */
enum { MC3D_CONST_DT = 0, MC3D_CONST_CFL = 1 };                 /* TimeSteppingType */
enum { MC3D_PERIODIC_SOLVE = 0, MC3D_DIRICHLET_SOLVE = 1 };     /* BCType           */
enum { MC3D_CD2 = 0, MC3D_PADE6 = 1, MC3D_PENTA10 = 2 };        /* FDType           */
enum { MC3D_COMPACT8 = 0, MC3D_COMPACT10 = 1,                  /* FilterType       */
       MC3D_TESTFILTER_PADE = 2, MC3D_TESTFILTER_EXP = 3 };      /* DSM test filters */
enum { MC3D_NOMODEL = 0, MC3D_VREMAN = 1, MC3D_DSM = 2,        /* LESModel         */
       MC3D_MLPSGS = 3 };   /* learned closure (LESMODEL = MLP), an addition with DSM as its fallback */
enum { MC3D_AVG_NONE = 0, MC3D_AVG_XI1 = 1, MC3D_AVG_XI2 = 2, MC3D_AVG_XI3 = 3,
       MC3D_AVG_LOCAL = 4, MC3D_AVG_GLOBAL = 5 };               /* StatsAvgType     */
enum { MC3D_TVDRK3 = 0, MC3D_RK4 = 1, MC3D_KENRK4 = 2, MC3D_LSLDDRK4 = 3 }; /* RKType */
/* BCKind (src/Options.hpp:21-27) */
enum { MC3D_BC_PERIODIC = 0, MC3D_BC_INTERNALLY_PERIODIC = 1, MC3D_BC_SPONGE = 2,
       MC3D_BC_ADIABATIC_WALL = 3, MC3D_BC_CONST_T_WALL = 4, MC3D_BC_MOVING_ADIABATIC_WALL = 5,
       MC3D_BC_INLET = 6 };
enum { MC3D_SPONGE_RECTILINEAR = 0, MC3D_SPONGE_CYLINDRICAL = 1 };   /* SpongeKind */
/* precision of the bulk arithmetic; metrics, LU factors, the conserved state,
 * the RK registers and the time accumulators are FP64 in both */
enum { MC3D_FP64 = 0, MC3D_FP32BULK = 1 };

/* The options of the time step (src/Options.hpp:46-118 members). */
typedef struct mc3d_config {
    int Nx, Ny, Nz;
    int bc_type[3];          /* BCType per direction                         */
    int bc_kind[6];          /* BCKind for X0, X1, Y0, Y1, Z0, Z1             */
    int fd_type[3];          /* FDType per direction                         */
    int filter_type;         /* FilterType                                   */
    double alphaF;           /* SOLVER.ALPHAF                                */
    double mu_ref;           /* SOLVER.MU_REF                                */
    int rk_type;             /* SOLVER.RKTYPE                                */
    int ts_type;             /* TIMESTEPPING.TSTYPE                          */
    double cfl;              /* TIMESTEPPING.CFL                             */
    double dt;               /* TIMESTEPPING.DT                              */
    int filter_step;         /* TIMESTEPPING.FILTERSTEP                      */
    int substep_filtering;   /* TIMESTEPPING.SUBSTEPFILTERING                */
    int max_time_step;       /* TIMESTEPPING.MAXTIMESTEP                     */
    double max_time;         /* TIMESTEPPING.MAXTIME                         */
    int les_model;           /* LES.LESMODEL                                 */
    int les_averaging;       /* LES.LESAVERAGING                             */
    int time_step0;          /* starting time step (restart)                 */
    double time0;            /* starting time                                */
    /* [GPU] section: keys the reference does not have */
    int precision;           /* GPU.PRECISION = FP64 | FP32BULK              */
    int reference_quirks;    /* GPU.REFERENCEQUIRKS (default 1): keep the
                                reference's momentum k2 carry-over
                                (src/CurvilinearCSolver_Core.cpp:839,872,904) */
    int dsm_test_filter;     /* LES.DSMTESTFILTER (default 1): 1 = Pade test
                                filter, 2 = explicit (src/DSMSGS.hpp:57-67)   */
    int dsm_use_taukk;       /* LES.DSMUSETAUKK (default 1)                  */
    /* [SPONGE] (src/Options.hpp:161-175, read when a face is SPONGE) */
    int sponge_kind;         /* SPONGE.KIND: MC3D_SPONGE_*                   */
    double sponge_strength;  /* SPONGE.STRENGTH (default 1)                  */
    double sponge_rect_perc[6];  /* SPONGE.RECT{X,Y,Z}{0,1}PERC, X0 X1 Y0 Y1 Z0 Z1 */
    int sponge_cyl_orient;   /* SPONGE.CYLAXIS_ORIENT                        */
    double sponge_cyl_axis[3];   /* SPONGE.CYLAXIS_X, _Y, _Z                 */
    double sponge_rmin;      /* SPONGE.RMIN                                  */
    /* tangential velocity of MOVING_ADIABATIC_WALL faces X0 X1 Y0 Y1 Z0 Z1:
     * (V, W) on X faces, (U, W) on Y faces, (U, V) on Z faces; the reference
     * sets them to zero in its constructor (src/CurvilinearCSolver.hpp:219-221) */
    double wall_velocity[6][2];
    /* LESMODEL = MLP: a stage falls back to DSM when more than this fraction
     * of its points has a feature outside the closure's training range; the
     * features of the other out-of-range points are clamped to the range
     * (LES.MLPFALLBACKFRAC, default 1e-3; 0 = any point). No counterpart in
     * the reference. */
    double mlp_fallback_frac;
    /* BC.PERIODICDISP{X,Y,Z}_{X,Y,Z}: displacement of the X1 (Y1, Z1) face
     * from the X0 (Y0, Z0) face, row = face pair, column = component; read
     * for PERIODIC faces (src/Options.hpp:152-160), used by mc3d_solver_set_mesh */
    double periodic_disp[3][3];
    int dump_step;           /* TIMESTEPPING.DUMPSTEP (default 1000, src/Options.hpp:237) */
    /* [RESTART] (src/Options.hpp:186-193, :365-391): FROMRESTART,
     * ONLYGRIDFROMRESTART, FILENAME; SPONGEAVGFROMRESTART, SPONGEAVGFILENAME.
     * With either restart flag DOMAIN.N* come from the file's header
     * (src/MPI_3DCompact.cpp:80-110); mc3d_solver_start applies them. */
    int from_restart, only_grid_from_restart, sponge_avg_from_restart;
    char restart_file[512];
    char sponge_avg_file[512];
    /* [STATS] (src/Options.hpp:194-201, :392-417): running statistics updated
     * every stats_interval steps (default 5); stats_avg_type is STATSAVGTYPE
     * (MC3D_AVG_*: only XI1/XI3 average, as Stats::doAveraging does) */
    int velocity_stats, thermo_stats, stats_interval, stats_avg_type;
    int velocity_stats_from_restart, thermo_stats_from_restart;
    char velocity_stats_file[512];
    char thermo_stats_file[512];
    /* SPONGE.AVGTIME (default 1), SPONGE.PINF (default 1/gamma), read with the
     * sponge (src/Options.hpp:321-322); sponge_relax turns on the relaxation of
     * the sponge target toward the state after every step
     * (CurvilinearCSolver::updateSponge, src/CurvilinearCSolver_BC.cpp:843-928),
     * which the reference leaves commented out in postStep (default 0). No key. */
    double sponge_avg_time, sponge_p_inf;
    int sponge_relax;
    /* GPU.STORAGE = FULL | LEAN (default FULL; no key in the reference). LEAN
     * holds the periodic-box time step in 19 work fields of the working
     * precision and 10 FP64 fields of the block instead of about 60 (a 1024^3
     * block on one 180 GB GPU): the 2N schemes update the stage state in
     * place, k2 accumulates the flux divergence (with the momentum carry-over
     * when REFERENCEQUIRKS is on), and everything along xi1 and xi2 runs in
     * slabs of xi3-planes, so only the xi3-gradients and xi3-fluxes are full
     * fields. For periodic blocks with constant metrics, LESMODEL NOMODEL,
     * VREMAN (no averaging) or MLP (no DSM fallback: stages past
     * MLPFALLBACKFRAC are counted and keep the clamped network), no
     * sub-step filtering and no statistics. GPU.LEANSLAB (lean_slab):
     * xi3-planes per slab (0: about 2^26 points). */
    int lean_storage;
    int lean_slab;
} mc3d_config;

/* ---- configuration ---- */
int mc3d_config_default(mc3d_config *cfg);
/* Parse an MPI_3DCompact.in file: same sections, keys, enum strings, defaults
 * and required keys as Options (src/Options.hpp:128-428, src/Options.cpp:3-312);
 * LESMODEL also accepts NONE for NOMODEL. Unsupported but valid settings are
 * reported as MC3D_ERR_CONFIG. */
int mc3d_config_from_ini(const char *path, mc3d_config *cfg);

/* SpongeBC::initRectSpongeBC / initCylSpongeBC (src/SpongeBC.cpp:65-360):
 * the sponge strength sigma of every point from the mesh coordinates (host
 * arrays, x-fastest, Nx*Ny*Nz each) and the [SPONGE] options of cfg. */
int mc3d_sponge_sigma(const mc3d_config *cfg, const double *x, const double *y, const double *z, double *sigma);

/* ---- last error of the calling thread ---- */
const char *mc3d_last_error(void);

/* ---- compact-derivative and filter operators ---- */
typedef struct mc3d_op_s *mc3d_op;

/* Replaces `new Pade6/Penta10/CD2(Domain*, BCType, Direct)` (src/Pade6.hpp:39,
 * src/Penta10.hpp:38, src/CD2.hpp:30). `dh` is the computational spacing
 * (Domain::dx/dy/dz, src/Domain.hpp:45-79). precision: MC3D_FP64 -> fields are
 * double, MC3D_FP32BULK -> fields are float. */
int mc3d_deriv_create(int fd_type, int bc_type, int dir, int Nx, int Ny, int Nz, double dh,
                      int precision, int device, mc3d_op *out);

/* Replaces `new Compact8Filter/Compact10Filter(alphaF, Domain*, BC*, BCType,
 * Direct)` (src/Compact8Filter.hpp:28, src/Compact10Filter.hpp:30), and with
 * filter_type MC3D_TESTFILTER_PADE / MC3D_TESTFILTER_EXP (alphaF unused) the
 * DSM test filters `new CommN5PadeTestFilter/CommN5ExpTestFilter(Domain*, BC*,
 * BCType, Direct)` (src/CommN5PadeTestFilter.hpp:32, src/CommN5ExpTestFilter.hpp:16).
 * bc_types[3] are the BC types of all three directions: lines lying on a
 * Dirichlet face of another direction pass through (src/Compact10Filter.cpp:166-252). */
int mc3d_filter_create(int filter_type, double alphaF, int dir, const int bc_types[3], int Nx, int Ny,
                       int Nz, int precision, int device, mc3d_op *out);

/* calc1stDerivField / filterField on `nfields` device fields at once:
 * out[f] = op(in[f]). `stream` is a cudaStream_t (NULL = legacy default).
 * in[f] and out[f] may not alias. FP32 lines of 128-256 points (y and z lines
 * also of 512 and 1024) go through the TMA-staged kernels. Lines of up to
 * 1024 points in FP32 and 512 in FP64 run in every direction; longer FP64
 * lines run while the shared-memory tile of the 32 lines fits, and give
 * MC3D_ERR_CONFIG beyond (1024 points). Calls may overlap solver steps and other
 * calls on other streams; each result is the same as when it runs alone. */
int mc3d_op_apply(mc3d_op op, const void *const *in, void *const *out, int nfields, void *stream);

/* calc1stDerivField_TPB (src/AbstractDerivatives.hpp:45 for Pade6 and CD2,
 * :47 for Penta10; src/Pade6.cpp:48-107, src/Penta10.cpp:175-207,
 * src/CD2.cpp:48-151) of a periodic derivative operator: the line's values
 * beyond its ends come from caller-supplied ghost planes instead of wrapping
 * around (the reference uses it for translated periodic meshes), then the
 * periodic system is solved. *per_side = 2 (Pade6, CD2: Nm2 Nm1 | Np1 Np2)
 * or 3 (Penta10: Nm3 Nm2 Nm1 | Np1 Np2 Np3). ghosts[f * 2 * per_side + m] are
 * device planes of the op's precision, in the reference's argument order
 * (Nm_{per_side} .. Nm1, Np1 .. Np_{per_side}); Nm_m holds the value at index
 * -m of each line, Np_m the value at N - 1 + m. A plane has one value per line
 * along dir, x fastest over the other two directions: dir 0: [k*Ny + j],
 * dir 1: [k*Nx + i], dir 2: [j*Nx + i] (the reference's y-pencil planes are
 * [i*Nz + k]). The first call allocates the operator's one-field scratch. */
int mc3d_op_tpb_ghosts(mc3d_op op, int *per_side);
int mc3d_op_apply_tpb(mc3d_op op, const void *const *in, void *const *out, int nfields,
                      const void *const *ghosts, void *stream);
int mc3d_op_destroy(mc3d_op op);

/* AbstractDerivatives::calcNeumann (src/Pade6.cpp:395-397, src/CD2.cpp:183):
 * the wall value giving a zero normal derivative from f[1..5]. Host-side. */
double mc3d_calc_neumann(int fd_type, const double *f);

/* ---- learned SGS closure: no counterpart in the reference, where VremanSGS /
 * DSMSGS (src/VremanSGS.hpp, src/DSMSGS.hpp) are the models. A 9-64-64-64-2
 * GELU MLP from invariants of the resolved velocity gradient and the grid
 * scale to C (mu_t = rho C Delta^2 |S|) and Pr_t. Arrays are device FP32:
 * x [n][9] raw features, y [n][2]. ---- */
typedef struct mc3d_mlp_s *mc3d_mlp;
int mc3d_mlp_create(unsigned long long seed, int device, mc3d_mlp *out);
int mc3d_mlp_destroy(mc3d_mlp m);
/* feature mean/std (normalisation), training range lo/hi (outside it the
 * solver falls back to DSM), target mean/std (outputs are normalised targets) */
int mc3d_mlp_set_normalization(mc3d_mlp m, const float *mean, const float *std, const float *lo, const float *hi,
                               const float *ymean, const float *ystd);
int mc3d_mlp_get_normalization(mc3d_mlp m, float *out);
/* one Adam step (lr) on MSE against normalised targets y; loss (host, may be NULL) */
int mc3d_mlp_train_step(mc3d_mlp m, const float *x, const float *y, int n, float lr, double *loss, void *stream);
/* the gradient that step would use, without the update: G (host, MLP_NPARAM =
 * 9090 floats, in the parameter order of mc3d_mlp_get_params) = d loss / dP
 * with loss = mean_b sum_o (out_bo - y_bo)^2, computed by the same FP32
 * forward, backward and weight-gradient kernels; loss (host, may be NULL) */
int mc3d_mlp_gradient(mc3d_mlp m, const float *x, const float *y, int n, float *G, double *loss, void *stream);
/* FP32 forward on CUDA cores, and the BF16 tensor-core inference (tcgen05
 * MMAs on tiles of 128 points, FP32 accumulators in tensor memory, the kernel
 * of the closure in the time step) */
int mc3d_mlp_forward(mc3d_mlp m, const float *x, float *y, int n, void *stream);
int mc3d_mlp_infer_bf16(mc3d_mlp m, const float *x, float *y, int n, void *stream);
int mc3d_mlp_get_params(mc3d_mlp m, float *P);          /* host, 9090 floats */
int mc3d_mlp_set_params(mc3d_mlp m, const float *P);
int mc3d_mlp_save(mc3d_mlp m, const char *path);
int mc3d_mlp_load(mc3d_mlp m, const char *path);
/* training data from DNS fields (device FP64): box filter of factor f of the
 * conserved state into 14 coarse fields (rho, rhoU_i, rhoU_iU_j, rhoT, rhoU_iT),
 * and features + least-squares targets from them and the xi-derivatives
 * grads[3*var + dir] of the Favre-filtered u, v, w, T (box metrics jd[3]) */
int mc3d_sgs_box_filter(const double *const q[5], int Nx, int Ny, int Nz, int f, double *const out[14],
                        void *stream);
int mc3d_sgs_training_pairs(const double *const coarse[14], const double *const grads[12], int Nx, int Ny, int Nz,
                            const double jd[3], double delta, double mu_ref, float *x, float *y, void *stream);

/* ---- solver: CurvilinearCSolver + AbstractRK on one GPU ---- */
typedef struct mc3d_solver_s *mc3d_solver;

int mc3d_solver_create(const mc3d_config *cfg, int device, mc3d_solver *out);
int mc3d_solver_destroy(mc3d_solver s);

/* Metrics J, J11, J12, J13, J21, J22, J23, J31, J32, J33 (host, FP64), as
 * AbstractSingleBlockMesh::solveForJacobians produces them
 * (src/AbstractSingleBlockMesh.cpp:23-1439). */
int mc3d_solver_set_metrics(mc3d_solver s, const double *const metrics[10]);
/* The uniform periodic box x = L*xi (the HIT mesh,
 * tests/hit/Samtaney_D4/AlgebraicSingleBlockMesh.hpp:154-156). */
int mc3d_solver_set_box_metrics(mc3d_solver s, double Lx, double Ly, double Lz);
/* Metrics computed on the device, in FP64, from the mesh coordinates x, y, z
 * (host, Nx*Ny*Nz each, x fastest): AbstractSingleBlockMesh::solveForJacobians
 * (src/AbstractSingleBlockMesh.cpp:23-1308) with the solver's derivative
 * schemes, TPB derivatives along periodic directions translated as
 * handlePeriodicStuff does (:2019-2083, from cfg.periodic_disp), and with
 * cfg.reference_quirks the two BW7 calls that pass their Nm2 ghost as Nm3
 * (:273, :706). Replaces mc3d_solver_set_metrics. */
int mc3d_solver_set_mesh(mc3d_solver s, const double *x, const double *y, const double *z);
/* Copy the FP64 metrics J, J11..J33 the solver holds into 10 host arrays. */
int mc3d_solver_get_metrics(mc3d_solver s, double *const metrics[10]);

/* The learned closure a LESMODEL = MLP solver evaluates (kept by reference;
 * it must outlive the solver). */
int mc3d_solver_set_mlp(mc3d_solver s, mc3d_mlp m);
/* RK stages that fell back to DSM because a feature left the training range */
int mc3d_solver_mlp_fallbacks(mc3d_solver s, long long *stages);

/* Sponge strength sigma (host, FP64, x-fastest; e.g. from mc3d_sponge_sigma),
 * required before set_initial when a face is SPONGE (SpongeBC::sigma,
 * src/SpongeBC.cpp:42-61). */
int mc3d_solver_set_sponge(mc3d_solver s, const double *sigma);
/* Sponge target state rho, rhoU, rhoV, rhoW, rhoE (host, FP64), in place of
 * the initial conserved state (SpongeBC::readSpongeAvgFromRestart,
 * src/SpongeBC.cpp:426-487); call after set_initial. */
int mc3d_solver_set_sponge_avg(mc3d_solver s, const double *const avg[5]);

/* setInitialConditions from primitive fields (host, FP64): rho, U, V, W, p,
 * with the wall conditions of the BC kinds (no-slip / moving velocity, the
 * Neumann wall temperature, p and rhoE from rho and T) and the sponge target
 * state (src/CurvilinearCSolver_BC.cpp:3-369). */
int mc3d_solver_set_initial(mc3d_solver s, const double *rho, const double *U, const double *V,
                            const double *W, const double *p);
/* Same from device FP64 primitive fields (no host copy). */
int mc3d_solver_set_initial_device(mc3d_solver s, const double *rho, const double *U, const double *V,
                                   const double *W, const double *p);

/* Advance `nsteps` time steps (preStep .. postStep of AbstractRK::executeSolverLoop,
 * e.g. src/RK4.hpp:127-178). For LSLDDRK4 the 5- and 6-stage halves alternate,
 * one half per step. Asynchronous on the solver's stream. */
int mc3d_solver_step(mc3d_solver s, int nsteps);

/* ---- the same time step driven stage by stage ----
 * The virtuals of AbstractCSolver that AbstractRK::executeSolverLoop calls
 * (src/AbstractCSolver.hpp:82-87, e.g. the loop of src/RK4.hpp:127-178 and
 * src/LSLDDRK4.hpp:324-459), and AbstractRK::updateConservedData
 * (src/AbstractRK.hpp:15), so a GPU-backed RK object and solver drop in
 * behind the reference's loop. Called in the reference's order, they give the
 * state mc3d_solver_step gives, bit for bit; a call out of order returns
 * MC3D_ERR_CONFIG and changes nothing. All asynchronous on the solver's stream.
 *   preStep        calcDtFromCFL (src/CurvilinearCSolver.hpp:310-318)
 *   preSubStep     preStepBCHandling + preStepDerivatives of stage rkStep and
 *                  the first two directions of the flux divergence
 *                  (src/CurvilinearCSolver.hpp:320-327)
 *   solveEqnSet    solveContinuity .. solveEnergy: the third direction of the
 *                  divergence with the k2 assembly (Core.cpp:790-947)
 *   postSubStep    postStepBCHandling (src/CurvilinearCSolver_BC.cpp:702-842)
 *   rk_update      updateConservedData of `scheme` (MC3D_RK4 ..), stage
 *                  rkStep; dual_step: LSLDDRK4's rkDualStepStep (1: the
 *                  5-stage half, 2: the 6-stage half), ignored otherwise
 *   updateData     filterConservedData when rkLast (or SUBSTEPFILTERING) and
 *                  updateNonConservedData (src/CurvilinearCSolver.hpp:346-353)
 *   postStep       statistics and the optional sponge relaxation
 *                  (src/CurvilinearCSolver.hpp:355-375)
 * mc3d_solver_stage_count: the stages of the current time step (or of the
 * next one between steps): RK4 4, TVDRK3 3, KENRK4 5, LSLDDRK4 5 or 6. */
int mc3d_solver_pre_step(mc3d_solver s);
int mc3d_solver_stage_count(mc3d_solver s, int *stages);
int mc3d_solver_pre_substep(mc3d_solver s, int rk_step);
int mc3d_solver_solve_eqn_set(mc3d_solver s);
int mc3d_solver_post_substep(mc3d_solver s);
int mc3d_rk_update(mc3d_solver s, int scheme, int rk_step, int dual_step);
int mc3d_solver_update_data(mc3d_solver s, int rk_last);
int mc3d_solver_post_step(mc3d_solver s);

/* Copy the conserved state rho1, rhoU1, rhoV1, rhoW1, rhoE1 (FP64) to host. */
int mc3d_solver_get_conserved(mc3d_solver s, double *rho, double *rhoU, double *rhoV, double *rhoW,
                              double *rhoE);
/* Device-to-device copy of the conserved state into caller buffers (FP64). */
int mc3d_solver_copy_conserved_device(mc3d_solver s, double *const dst[5]);
/* Device pointers (FP64) of the five conserved fields. */
int mc3d_solver_conserved_device(mc3d_solver s, double *ptrs[5]);

/* ---- checkpoint files in the reference's formats ---- */
/* SolutionDump (CurvilinearCSolver::dumpSolution, src/CurvilinearCSolver_Core.cpp:1333-1405):
 * 5 FP64 header values (time step, time, Nx, Ny, Nz), then x, y, z, rho,
 * rhoU, rhoV, rhoW, rhoE, Nx*Ny*Nz FP64 values each, x fastest. */
int mc3d_dump_read_header(const char *path, int *time_step, double *time, int *Nx, int *Ny, int *Nz);
/* fields[0..7] = x, y, z, rho, rhoU, rhoV, rhoW, rhoE (NULL entries are
 * skipped); n = Nx*Ny*Nz must match the header. */
int mc3d_dump_read_fields(const char *path, long long n, double *const fields[8]);
int mc3d_dump_write(const char *path, int time_step, double time, int Nx, int Ny, int Nz,
                    const double *const fields[8]);
/* The solver's conserved state, time step and time as a SolutionDump. path
 * NULL: "SolutionDump.<time step>" in the working directory. x, y, z NULL:
 * the mesh of mc3d_solver_set_mesh / mc3d_solver_restart, or the box of
 * mc3d_solver_set_box_metrics (x = L*xi). */
int mc3d_solver_dump(mc3d_solver s, const char *path, const double *x, const double *y, const double *z);
/* Restart from a SolutionDump (src/MPI_3DCompact.cpp:80-271): metrics from
 * the file's mesh (as mc3d_solver_set_mesh); unless grid_only
 * (RESTART.ONLYGRIDFROMRESTART) also the conserved state, turned into
 * primitives by IdealGas::solveU/solvep (src/IdealGas.hpp:58-64) and set as
 * the initial condition, with the file's time step and time (so the first
 * step after it again leaves time unchanged, Core.cpp:221-228; the filter
 * direction rotation and the LSLDDRK4 halves start over). */
int mc3d_solver_restart(mc3d_solver s, const char *path, int grid_only);
/* SpongeAvgDump (SpongeBC::dumpSpongeAvg, src/SpongeBC.cpp:363-424): the five
 * sponge target fields, no header; path NULL: "SpongeAvgDump.<time step>". */
int mc3d_solver_dump_sponge_avg(mc3d_solver s, const char *path);
/* readSpongeAvgFromRestart (src/SpongeBC.cpp:426-480): the sponge target
 * from such a file (after the initial condition, which sets it otherwise). */
int mc3d_solver_read_sponge_avg(mc3d_solver s, const char *path);
/* The reference's driver loop for a configuration (src/MPI_3DCompact.cpp
 * with AbstractRK::executeSolverLoop and CurvilinearCSolver::postStep,
 * src/CurvilinearCSolver.hpp:355-375): when cfg.from_restart /
 * only_grid_from_restart / sponge_avg_from_restart are set, mc3d_solver_start
 * reads those files first; mc3d_solver_run then steps until checkEnd
 * (time >= MAXTIME, time step >= MAXTIMESTEP, or a file "killsolver" in dir,
 * removed when found, src/CurvilinearCSolver_Core.cpp:1750-1824), writing
 * SolutionDump.<step> (and SpongeAvgDump.<step> with sponges) into dir (NULL:
 * working directory) every DUMPSTEP steps and at the end. */
int mc3d_solver_start(mc3d_solver s);
int mc3d_solver_run(mc3d_solver s, const char *dir);

/* ---- diagnostic hooks of the reference drivers, as device reductions ---- */
/* One turbdata.out line of the HIT driver (tests/hit/Samtaney_D4/MPI_3DCompact.cpp:370-555)
 * for the current state: out = time, tau = sqrt(2 pi)/k0/u', Re_lambda, Mt,
 * dissipation / mean rho, u', Kolmogorov length, rho', dilatation', vorticity',
 * mean rho|u|^2 (the driver passes k0 = 8). */
int mc3d_solver_turbdata(mc3d_solver s, double k0, double out[11]);
/* The cylinder driver's surface data (src/MPI_3DCompact.cpp:408-485): p, U, V,
 * W on the j = 0 face averaged over xi3, Nx values each (host arrays). */
int mc3d_solver_wall_span_average(mc3d_solver s, double *p, double *U, double *V, double *W);
/* The cylinder driver's wake strip (src/MPI_3DCompact.cpp:488-527): V along
 * xi3 at the grid point (i, j) (the driver takes i = 0, j = 143), Nz values
 * (host array). MC3D_ERR_ARG when (i, j) lies outside the grid. */
int mc3d_solver_wake_strip(mc3d_solver s, int i, int j, double *V);

/* ---- running statistics (Stats, src/Stats.cpp:127-347) ---- */
/* With cfg.velocity_stats / thermo_stats set, every mc3d_solver_step updates
 * them after each stats_interval-th time step (postStep): time-weighted
 * means, RMS and Reynolds stresses of U, V, W of the filtered state and of
 * rho (the unfiltered rho2), p, T, with the XI1/XI3 index averaging of
 * STATSAVGTYPE; FP64 on the device. Copies to host: velocity[9] = UAVG, VAVG,
 * WAVG, URMS, VRMS, WRMS, UVREY, UWREY, VWREY; thermo[6] = RHOAVG, RHORMS,
 * PAVG, PRMS, TAVG, TRMS (NULL arrays skipped); weights[2] = the two
 * accumulated time weights. */
int mc3d_solver_get_stats(mc3d_solver s, double *const velocity[9], double *const thermo[6], double weights[2]);
/* VelocityStats / ThermoStats files (Stats::dumpStatsFields, src/Stats.cpp:3-125:
 * the weight, then the fields, x fastest); NULL paths: "VelocityStats.<step>"
 * and "ThermoStats.<step>" in the working directory. mc3d_solver_run writes
 * them with each SolutionDump. */
int mc3d_solver_dump_stats(mc3d_solver s, const char *velocity_path, const char *thermo_path);
/* Statistics from such files (STATS.*STATSFROMRESTART, Stats.hpp:60-266);
 * NULL paths are skipped; mc3d_solver_start reads the configured ones. */
int mc3d_solver_read_stats(mc3d_solver s, const char *velocity_path, const char *thermo_path);

/* Time-step counter, time, last dt and total RK stages run (synchronises). */
int mc3d_solver_info(mc3d_solver s, int *time_step, double *time, double *dt, long long *stages);

/* Kinetic-energy and mass integrals sum(rho|u|^2/2), sum(rho) over the grid
 * (FP64 device reduction, synchronises). */
int mc3d_solver_integrals(mc3d_solver s, double *kinetic, double *mass);

/* The cudaStream_t the solver launches on (for event timing). By default every
 * solver on a device launches on one non-blocking stream of that device
 * (created at the first solver, kept until exit); mc3d_solver_set_stream
 * moves a solver to a stream of the caller's. */
int mc3d_solver_stream(mc3d_solver s, void **stream);
/* Binds the solver to `stream` (a cudaStream_t of the solver's device; NULL:
 * the device's shared stream). Work already queued on the previous stream is
 * completed first; every later call queues the solver's kernels on the new
 * stream. Solvers on different streams run concurrently and independently:
 * their kernels share no memory. Like the reference's one solver per MPI rank,
 * a solver is driven from one host thread at a time. */
int mc3d_solver_set_stream(mc3d_solver s, void *stream);
/* Total number of kernels this solver has launched so far (launch accounting). */
int mc3d_solver_launch_count(mc3d_solver s, long long *count);
int mc3d_solver_sync(mc3d_solver s);

/* Optional CUDA-event timing of every kernel the solver launches, grouped by
 * kernel class. Enabling clears earlier records. The report is a JSON object
 * {"class": {"launches": L, "ms": T, "bytes": B}, ...} with B the algorithmic
 * bytes those launches must move; the string is owned by the solver and valid
 * until the next call (synchronises). */
int mc3d_solver_set_timing(mc3d_solver s, int enable);
const char *mc3d_solver_timing_report(mc3d_solver s);

/* Number of bounded waits on `device` that gave up: line-solve CTAs whose TMA
 * tile load did not arrive (they skipped their tile) plus learned-closure
 * warpgroups whose tensor-core MMAs did not complete (they stopped); the
 * results of those launches are invalid. mc3d_solver_info and
 * mc3d_solver_get_conserved return MC3D_ERR_TIMEOUT when it is nonzero. */
int mc3d_tma_wait_timeouts(int device, int *count);

/* ---- SGS models on their own (AbstractSGS, src/AbstractSGS.hpp:10-42) ----
 * A GPU VremanSGS / DSMSGS (src/VremanSGS.hpp:13-41, src/DSMSGS.hpp:20-118)
 * that a caller drives with its own gradients: model MC3D_VREMAN | MC3D_DSM,
 * LESAVERAGING (MC3D_AVG_*), DSMTESTFILTER (1 Pade, 2 explicit), DSMUSETAUKK,
 * the block, the BC types of the three directions (periodic / Dirichlet
 * test-filter and averaging closures), the computational spacings
 * dxi[3] = Domain::dx, dy, dz and the metric Jacobian J (a device field of the
 * object's precision, or NULL with the constant Jc; Vreman's filter width is
 * (dx dy dz / J)^(1/3)). Fields are device arrays, x fastest: gradients and
 * outputs in the object's precision (double for MC3D_FP64, float for
 * MC3D_FP32BULK), the conserved rho..rhoE always FP64 (calcKSGS reads rho ..
 * rhoW only; q[4] may be NULL there). gradU[3*a + b] = d u_a / d x_b and
 * gradT[b] = d T / d x_b are physical gradients (preStepDerivatives'
 * J^T-transformed ones, Core.cpp:548-561, :596-600). As in the reference,
 * each model implements only its own virtuals and the others do nothing:
 * Vreman getSGSViscosity (mu_sgs, averaged with Compact10(-0.49) filters
 * when LOCAL); DSM calcMuSGSTaukk (mu_sgs and, with taukk non-NULL, tau_kk)
 * and calcKSGS (k_sgs; it reuses the filtered fields of the preceding
 * calcMuSGSTaukk, so call it after that one on the same state), averaged per
 * doAveraging (src/AbstractSGS.cpp:13-160). The object holds its work
 * fields (DSM: 49 fields of the block).
 * MC3D_MLPSGS (the learned closure; averaging, test_filter and use_taukk are
 * ignored) takes its network and mu_ref from mc3d_sgs_set_mlp and works as a
 * DSM-shaped pair: calcMuSGSTaukk keeps gradU and the mu_sgs destination and
 * zeroes tau_kk (when given), then calcKSGS evaluates the closure (features
 * of gradU, gradT, rho = q[0] and T; the tcgen05 network) into mu_sgs and
 * k_sgs. Features outside the closure's training range are clamped; their
 * points are counted (mc3d_sgs_mlp_out_of_range, the last calcKSGS). There
 * is no fallback here: a caller that wants DSM for such states runs a DSM
 * object. */
typedef struct mc3d_sgs_s *mc3d_sgs;
int mc3d_sgs_create(int model, int averaging, int test_filter, int use_taukk, int Nx, int Ny, int Nz,
                    const int bc_types[3], const double dxi[3], const void *J, double Jc, int precision,
                    int device, mc3d_sgs *out);
int mc3d_sgs_destroy(mc3d_sgs sgs);
int mc3d_sgs_get_viscosity(mc3d_sgs sgs, const void *const gradU[9], const double *const q[5], void *mu_sgs,
                           void *stream);
int mc3d_sgs_calc_mu_taukk(mc3d_sgs sgs, const void *const gradU[9], const double *const q[5], void *mu_sgs,
                           void *taukk, void *stream);
int mc3d_sgs_calc_ksgs(mc3d_sgs sgs, const void *const gradT[3], const double *const q[5], const void *T,
                       void *k_sgs, void *stream);
int mc3d_sgs_set_mlp(mc3d_sgs sgs, mc3d_mlp mlp, double mu_ref);
/* points of the last learned-closure calcKSGS with a feature outside the
 * training range (synchronises the device) */
int mc3d_sgs_mlp_out_of_range(mc3d_sgs sgs, long long *points);

/* ---- allocation-free CFL reduction ----
 * No counterpart in the reference: an extra entry point for callers that must
 * not have the library allocate device memory (a host code that hands all GPU
 * memory to its own pool at start-up, where a cudaMalloc in the time loop
 * could fail or would synchronise the device). Computes the CFL wave-speed
 * maximum max(J11(|U|+c)/dxi + J22(|V|+c)/deta + J33(|W|+c)/dzeta) over the
 * FP64 conserved fields (device pointers, x-fastest) into *out_max (device
 * pointer to one double). J11/J22/J33 may be NULL, then J11c/J22c/J33c are
 * used. It allocates nothing: the per-block partial maxima sit in a fixed
 * 512 KiB device array inside the library, which every GPU that loads the
 * library holds until the process exits; fields larger than 16,777,216
 * points (256^3) are rejected with MC3D_ERR_ARG. The first call on a device
 * sets up: it looks up that array's address (cudaGetSymbolAddress) and loads
 * the two kernels, and CUDA's on-demand module loading claims device memory
 * for that (the array and the kernels' code). Make the first call on each
 * device at start-up, before the caller's pool takes the device's memory and
 * before any stream capture; every later call allocates and loads nothing.
 * All calls share the array: calls that overlap on the GPU (different
 * streams, no ordering) race; no scratch value needs to start at zero, every
 * slot a call reads is written by the same call. A non-finite wave speed
 * anywhere (a NaN or infinite state) makes *out_max NaN, on purpose: the
 * reference's `UChar > lmax` loop (src/CurvilinearCSolver_Core.cpp:200-205)
 * skips NaN points instead, so check the result before dividing by it.
 * Asynchronous on `stream`. */
int mc3d_cfl_max_noalloc(const double *rho, const double *rhoU, const double *rhoV, const double *rhoW,
                         const double *rhoE, const double *J11, const double *J22, const double *J33,
                         double J11c, double J22c, double J33c, int Nx, int Ny, int Nz, double dxi, double deta,
                         double dzeta, double *out_max, void *stream);

/* ---- host utilities ---- */
/* The combined-LCG shuffle generator of the reference's HIT IC generator
 * (tests/hit/generate_init_hit.f90:16-81). state[0..2] = ix1..ix3 and
 * table[0..96] = r(1..97) are updated in place; n values go to out. */
int mc3d_hit_randvec(int *state, double *table, long long n, double *out);

#ifdef __cplusplus
}
#endif
#endif
