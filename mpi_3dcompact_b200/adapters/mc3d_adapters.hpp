// GPU objects behind the reference solver's own plugin interfaces
// (emathew1/MPI_3DCompact): include this after the reference's headers and
// link libmc3d.so (include/mc3d.h) and the CUDA runtime.
//
//   reference interface                             GPU object here
//   AbstractDerivatives (src/AbstractDerivatives.hpp)   GpuPade6, GpuPenta10, GpuCD2
//   AbstractFilter      (src/AbstractFilter.hpp)        GpuCompact8Filter, GpuCompact10Filter,
//                                                       GpuCommN5PadeTestFilter, GpuCommN5ExpTestFilter
//   AbstractCSolver     (src/AbstractCSolver.hpp)       GpuCurvilinearCSolver
//   AbstractRK          (src/AbstractRK.hpp)            GpuRK (RK4, TVDRK3, KenRK4, LSLDDRK4)
//   AbstractSGS         (src/AbstractSGS.hpp)           GpuVremanSGS, GpuDSMSGS
//
// Field pointers passed to the operators and SGS objects are DEVICE arrays in
// the library's resident layout (the whole block, x fastest:
// i + Nx*(j + Ny*k)), FP64 unless an object was made with MC3D_FP32BULK; the
// reference's host pencils are not used. Errors of the C ABI surface as
// std::runtime_error with the library's message (the reference prints and
// calls MPI_Abort instead).
#ifndef MC3D_ADAPTERS_HPP
#define MC3D_ADAPTERS_HPP

#include <cuda_runtime.h>

#include <cstdio>
#include <stdexcept>
#include <string>

#include "mc3d.h"

namespace mc3d_adapters {

inline void check(int rc, const char *what) {
    if (rc != MC3D_OK) throw std::runtime_error(std::string(what) + ": " + mc3d_last_error());
}

inline int to_bc(Options::BCType t) {
    return t == Options::PERIODIC_SOLVE ? MC3D_PERIODIC_SOLVE : MC3D_DIRICHLET_SOLVE;
}

// ---- derivatives: new Pade6/Penta10/CD2(Domain*, BCType, Direct) ----------
class GpuDerivatives : public AbstractDerivatives {
   public:
    mc3d_op op = nullptr;
    int fdType;
    void *stream;

    GpuDerivatives(int fd_type, Domain *dom, Options::BCType bcType, Direct currentDir, int precision = MC3D_FP64,
                   int device = 0, void *stream = nullptr)
        : fdType(fd_type), stream(stream) {
        // the fields AbstractDerivatives carries (src/Pade6.hpp:39-75)
        Nx = dom->gNx;
        Ny = dom->gNy;
        Nz = dom->gNz;
        dx = dom->dx;
        dy = dom->dy;
        dz = dom->dz;
        this->currentDir = currentDir;
        this->bcType = bcType;
        N = currentDir == DIRX ? Nx : (currentDir == DIRY ? Ny : Nz);
        dd = currentDir == DIRX ? dx : (currentDir == DIRY ? dy : dz);
        rhsBandwidth = fd_type == MC3D_PENTA10 ? BW7 : BW5;
        lhsBandwidth = fd_type == MC3D_PENTA10 ? BW5 : BW3;
        check(mc3d_deriv_create(fd_type, to_bc(bcType), (int)currentDir, Nx, Ny, Nz, dd, precision, device, &op),
              "mc3d_deriv_create");
    }
    ~GpuDerivatives() { mc3d_op_destroy(op); }

    void calc1stDerivField(double *dataIn, double *dataOut) {
        const void *in[1] = {dataIn};
        void *out[1] = {dataOut};
        check(mc3d_op_apply(op, in, out, 1, stream), "calc1stDerivField");
    }

    // BW5 signature (Pade6, CD2); a BW7 scheme (Penta10) needs Nm3 / Np3 too
    void calc1stDerivField_TPB(double *dataIn, double *dataOut, double *Nm2, double *Nm1, double *Np1, double *Np2) {
        if (fdType == MC3D_PENTA10)
            throw std::runtime_error("calc1stDerivField_TPB: Penta10 reads Nm3 and Np3 (the BW7 signature)");
        const void *g[4] = {Nm2, Nm1, Np1, Np2};
        tpb(dataIn, dataOut, g);
    }
    // BW7 signature (Penta10); a BW5 scheme reads Nm2 .. Np2 of it
    void calc1stDerivField_TPB(double *dataIn, double *dataOut, double *Nm3, double *Nm2, double *Nm1, double *Np1,
                               double *Np2, double *Np3) {
        if (fdType == MC3D_PENTA10) {
            const void *g[6] = {Nm3, Nm2, Nm1, Np1, Np2, Np3};
            tpb(dataIn, dataOut, g);
        } else {
            const void *g[4] = {Nm2, Nm1, Np1, Np2};
            tpb(dataIn, dataOut, g);
        }
    }

    // calcNeumann reads six host values along the wall normal (src/Pade6.cpp:395-397)
    double calcNeumann(double *f) { return mc3d_calc_neumann(fdType, f); }

   private:
    void tpb(double *dataIn, double *dataOut, const void *const *ghosts) {
        const void *in[1] = {dataIn};
        void *out[1] = {dataOut};
        check(mc3d_op_apply_tpb(op, in, out, 1, ghosts, stream), "calc1stDerivField_TPB");
    }
};

struct GpuPade6 : GpuDerivatives {
    GpuPade6(Domain *dom, Options::BCType bc, Direct dir, int prec = MC3D_FP64, int dev = 0, void *st = nullptr)
        : GpuDerivatives(MC3D_PADE6, dom, bc, dir, prec, dev, st) {}
};
struct GpuPenta10 : GpuDerivatives {
    GpuPenta10(Domain *dom, Options::BCType bc, Direct dir, int prec = MC3D_FP64, int dev = 0, void *st = nullptr)
        : GpuDerivatives(MC3D_PENTA10, dom, bc, dir, prec, dev, st) {}
};
struct GpuCD2 : GpuDerivatives {
    GpuCD2(Domain *dom, Options::BCType bc, Direct dir, int prec = MC3D_FP64, int dev = 0, void *st = nullptr)
        : GpuDerivatives(MC3D_CD2, dom, bc, dir, prec, dev, st) {}
};

// ---- filters: new Compact10Filter(alphaF, Domain*, BC*, BCType, Direct) ----
class GpuFilter : public AbstractFilter {
   public:
    mc3d_op op = nullptr;
    void *stream;

    GpuFilter(int filter_type, double alphaF, Domain *dom, BC *bc, Options::BCType bcType,
              AbstractDerivatives::Direct currentDir, int precision = MC3D_FP64, int device = 0, void *stream = nullptr)
        : stream(stream) {
        Nx = dom->gNx;
        Ny = dom->gNy;
        Nz = dom->gNz;
        N = currentDir == AbstractDerivatives::DIRX ? Nx : (currentDir == AbstractDerivatives::DIRY ? Ny : Nz);
        this->currentDir = currentDir;
        this->bcType = bcType;
        this->bc = bc;
        // lines on the Dirichlet faces of the other directions pass through
        // (src/Compact10Filter.cpp:166-252): the filter needs all three BC types
        const int bcs[3] = {to_bc(bc->bcXType), to_bc(bc->bcYType), to_bc(bc->bcZType)};
        check(mc3d_filter_create(filter_type, alphaF, (int)currentDir, bcs, Nx, Ny, Nz, precision, device, &op),
              "mc3d_filter_create");
    }
    ~GpuFilter() { mc3d_op_destroy(op); }

    void filterField(double *dataIn, double *dataOut) {
        const void *in[1] = {dataIn};
        void *out[1] = {dataOut};
        check(mc3d_op_apply(op, in, out, 1, stream), "filterField");
    }
};

struct GpuCompact8Filter : GpuFilter {
    GpuCompact8Filter(double a, Domain *dom, BC *bc, Options::BCType t, AbstractDerivatives::Direct d,
                      int prec = MC3D_FP64, int dev = 0, void *st = nullptr)
        : GpuFilter(MC3D_COMPACT8, a, dom, bc, t, d, prec, dev, st) {}
};
struct GpuCompact10Filter : GpuFilter {
    GpuCompact10Filter(double a, Domain *dom, BC *bc, Options::BCType t, AbstractDerivatives::Direct d,
                       int prec = MC3D_FP64, int dev = 0, void *st = nullptr)
        : GpuFilter(MC3D_COMPACT10, a, dom, bc, t, d, prec, dev, st) {}
};
struct GpuCommN5PadeTestFilter : GpuFilter {
    GpuCommN5PadeTestFilter(Domain *dom, BC *bc, Options::BCType t, AbstractDerivatives::Direct d,
                            int prec = MC3D_FP64, int dev = 0, void *st = nullptr)
        : GpuFilter(MC3D_TESTFILTER_PADE, 0.0, dom, bc, t, d, prec, dev, st) {}
};
struct GpuCommN5ExpTestFilter : GpuFilter {
    GpuCommN5ExpTestFilter(Domain *dom, BC *bc, Options::BCType t, AbstractDerivatives::Direct d,
                           int prec = MC3D_FP64, int dev = 0, void *st = nullptr)
        : GpuFilter(MC3D_TESTFILTER_EXP, 0.0, dom, bc, t, d, prec, dev, st) {}
};

// ---- the solver: CurvilinearCSolver(C2Decomp*, Domain*, BC*, TimeStepping*, Options*) ----
// The device-resident solver reads its options from the same
// MPI_3DCompact.in the reference's Options parsed. Its state stays on the
// device; rho0 .. p0 are the host initial fields setInitialConditions
// uploads (as the reference's setInitialConditions reads them).
class GpuCurvilinearCSolver : public AbstractCSolver {
   public:
    mc3d_solver s = nullptr;
    mc3d_config cfg;
    int device;

    GpuCurvilinearCSolver(const char *ini_path, Options *opt, Domain *dom, BC *bc, TimeStepping *ts,
                          int precision = MC3D_FP64, int device = 0)
        : device(device) {
        check(mc3d_config_from_ini(ini_path, &cfg), "mc3d_config_from_ini");
        cfg.precision = precision;
        this->opt = opt;
        this->dom = dom;
        this->bc = bc;
        this->ts = ts;
        mpiRank = 0;
        totRank = 1;
        rkStep = 1;
        rkLast = false;
        endFlag = false;
        timeStep = opt->timeStep;
        time = opt->time;
        baseDirection = 1;
        useTiming = false;
        rho0 = p0 = U0 = V0 = W0 = nullptr;
    }
    ~GpuCurvilinearCSolver() { mc3d_solver_destroy(s); }

    // device state and operators for the block (the reference allocates its
    // host arrays here)
    void initializeSolverData() { check(mc3d_solver_create(&cfg, device, &s), "mc3d_solver_create"); }
    // metrics: from the mesh coordinates (host, x fastest) or the uniform box
    void setMesh(const double *x, const double *y, const double *z) {
        check(mc3d_solver_set_mesh(s, x, y, z), "mc3d_solver_set_mesh");
    }
    void setBoxMetrics(double Lx, double Ly, double Lz) {
        check(mc3d_solver_set_box_metrics(s, Lx, Ly, Lz), "mc3d_solver_set_box_metrics");
    }
    void setInitialConditions() { check(mc3d_solver_set_initial(s, rho0, U0, V0, W0, p0), "setInitialConditions"); }

    void preStep() { check(mc3d_solver_pre_step(s), "preStep"); }
    void preSubStep() { check(mc3d_solver_pre_substep(s, rkStep), "preSubStep"); }
    void solveEqnSet() { check(mc3d_solver_solve_eqn_set(s), "solveEqnSet"); }
    void postSubStep() { check(mc3d_solver_post_substep(s), "postSubStep"); }
    void updateData() { check(mc3d_solver_update_data(s, rkLast ? 1 : 0), "updateData"); }
    void postStep() {
        check(mc3d_solver_post_step(s), "postStep");
        double dt = 0.0;
        long long stages = 0;
        check(mc3d_solver_info(s, &timeStep, &time, &dt, &stages), "mc3d_solver_info");
        // checkEnd (src/CurvilinearCSolver_Core.cpp:1785-1830)
        if (timeStep >= ts->maxTimeStep || time >= ts->maxTime) endFlag = true;
    }
    void reportAll() {
        double dt = 0.0;
        long long stages = 0;
        check(mc3d_solver_info(s, &timeStep, &time, &dt, &stages), "mc3d_solver_info");
        printf("step %d  time %.10g  dt %.10g  RK stages %lld\n", timeStep, time, dt, stages);
    }
    // the RHS hook sources are per-point host callbacks of the CPU solver; the
    // device path has none (only the built-in sponge source)
    double contRHSSource(int) { return 0.0; }
    double xmomRHSSource(int) { return 0.0; }
    double ymomRHSSource(int) { return 0.0; }
    double zmomRHSSource(int) { return 0.0; }
    double engyRHSSource(int) { return 0.0; }
    // conserved state rho1 .. rhoE1 back to host arrays
    void getConserved(double *r, double *ru, double *rv, double *rw, double *re) {
        check(mc3d_solver_get_conserved(s, r, ru, rv, rw, re), "mc3d_solver_get_conserved");
    }
};

// ---- RK: new RK4/TVDRK3/KenRK4/LSLDDRK4(AbstractCSolver*) -------------------
// executeSolverLoop is the reference's loop (src/RK4.hpp:127-178,
// src/LSLDDRK4.hpp:324-459) over the solver's virtuals;
// updateConservedData is the scheme's register update on the device.
class GpuRK : public AbstractRK {
   public:
    int scheme;
    int dualStep = 1;   // LSLDDRK4's rkDualStepStep

    GpuRK(AbstractCSolver *cs, int scheme) : scheme(scheme) {
        this->cs = cs;
        mpiRank = 0;
    }
    mc3d_solver handle() const { return static_cast<GpuCurvilinearCSolver *>(cs)->s; }

    void updateConservedData() { check(mc3d_rk_update(handle(), scheme, cs->rkStep, dualStep), "updateConservedData"); }

    void executeSolverLoop() {
        while (!cs->endFlag) {
            cs->rkLast = false;
            cs->preStep();
            int ns = 0;
            check(mc3d_solver_stage_count(handle(), &ns), "mc3d_solver_stage_count");
            for (int st = 1; st <= ns; st++) {
                cs->rkStep = st;
                cs->rkLast = st == ns;
                cs->preSubStep();
                cs->solveEqnSet();
                cs->postSubStep();
                updateConservedData();
                cs->updateData();
            }
            cs->postStep();
            if (scheme == MC3D_LSLDDRK4) dualStep = dualStep == 1 ? 2 : 1;
        }
    }
};

// ---- SGS: new VremanSGS(AbstractCSolver*) / DSMSGS(AbstractCSolver*) ---------
// The outputs mu_sgs, taukk and k_sgs are device fields the object owns.
class GpuSGS : public AbstractSGS {
   public:
    mc3d_sgs sgs = nullptr;
    void *stream;
    int prec;

    GpuSGS(int model, int averaging, int test_filter, bool use_taukk, Domain *dom, BC *bc, const void *J_device,
           double Jc, int precision = MC3D_FP64, int device = 0, void *stream = nullptr)
        : stream(stream), prec(precision) {
        mpiRank = 0;
        cs = nullptr;
        Nx = dom->gNx;
        Ny = dom->gNy;
        Nz = dom->gNz;
        N = Nx * Ny * Nz;
        filtX = filtY = filtZ = nullptr;
        coeffRangeFlag = false;
        C = CI = Prt = nullptr;
        const int bcs[3] = {to_bc(bc->bcXType), to_bc(bc->bcYType), to_bc(bc->bcZType)};
        const double dxi[3] = {dom->dx, dom->dy, dom->dz};
        check(mc3d_sgs_create(model, averaging, test_filter, use_taukk ? 1 : 0, Nx, Ny, Nz, bcs, dxi, J_device, Jc,
                              precision, device, &sgs),
              "mc3d_sgs_create");
        const size_t bytes = (size_t)N * (precision == MC3D_FP64 ? sizeof(double) : sizeof(float));
        if (cudaMalloc((void **)&mu_sgs, bytes) != cudaSuccess || cudaMalloc((void **)&taukk, bytes) != cudaSuccess ||
            cudaMalloc((void **)&k_sgs, bytes) != cudaSuccess)
            throw std::runtime_error("GpuSGS: device allocation failed");
    }
    ~GpuSGS() {
        mc3d_sgs_destroy(sgs);
        cudaFree(mu_sgs);
        cudaFree(taukk);
        cudaFree(k_sgs);
    }

    void getSGSViscosity(double *gradU[3][3], double *rho, double *rhoU, double *rhoV, double *rhoW, double *rhoE) {
        const void *g[9];
        flat(gradU, g);
        const double *q[5] = {rho, rhoU, rhoV, rhoW, rhoE};
        check(mc3d_sgs_get_viscosity(sgs, g, q, mu_sgs, stream), "getSGSViscosity");
    }
    void calcMuSGSTaukk(double *gradU[3][3], double *rho, double *rhoU, double *rhoV, double *rhoW, double *rhoE) {
        const void *g[9];
        flat(gradU, g);
        const double *q[5] = {rho, rhoU, rhoV, rhoW, rhoE};
        check(mc3d_sgs_calc_mu_taukk(sgs, g, q, mu_sgs, taukk, stream), "calcMuSGSTaukk");
    }
    void calcKSGS(double *gradT[3], double *rho, double *rhoU, double *rhoV, double *rhoW, double *T) {
        const void *g[3] = {gradT[0], gradT[1], gradT[2]};
        const double *q[5] = {rho, rhoU, rhoV, rhoW, nullptr};
        check(mc3d_sgs_calc_ksgs(sgs, g, q, T, k_sgs, stream), "calcKSGS");
    }

   private:
    static void flat(double *gradU[3][3], const void **g) {
        for (int a = 0; a < 3; a++)
            for (int b = 0; b < 3; b++) g[3 * a + b] = gradU[a][b];
    }
};

struct GpuVremanSGS : GpuSGS {
    GpuVremanSGS(int averaging, Domain *dom, BC *bc, const void *J, double Jc, int prec = MC3D_FP64, int dev = 0,
                 void *st = nullptr)
        : GpuSGS(MC3D_VREMAN, averaging, 1, false, dom, bc, J, Jc, prec, dev, st) {}
};
struct GpuDSMSGS : GpuSGS {
    GpuDSMSGS(int averaging, int test_filter, bool use_taukk, Domain *dom, BC *bc, const void *J, double Jc,
              int prec = MC3D_FP64, int dev = 0, void *st = nullptr)
        : GpuSGS(MC3D_DSM, averaging, test_filter, use_taukk, dom, bc, J, Jc, prec, dev, st) {}
};
// The learned closure behind the same interface, driven as DSM is
// (calcMuSGSTaukk, then calcKSGS, which fills mu_sgs and k_sgs; tau_kk is
// zero). `net` is a loaded closure (mc3d_mlp_create + mc3d_mlp_load), owned by
// the caller; mu_ref is Options::mu_ref.
struct GpuMlpSGS : GpuSGS {
    GpuMlpSGS(mc3d_mlp net, double mu_ref, Domain *dom, BC *bc, const void *J, double Jc, int prec = MC3D_FP64,
              int dev = 0, void *st = nullptr)
        : GpuSGS(MC3D_MLPSGS, MC3D_AVG_NONE, 1, false, dom, bc, J, Jc, prec, dev, st) {
        check(mc3d_sgs_set_mlp(sgs, net, mu_ref), "mc3d_sgs_set_mlp");
    }
};

}  // namespace mc3d_adapters

#endif
