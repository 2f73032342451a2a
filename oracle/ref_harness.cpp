/*
 * CPU oracle harness: drives the reference solver (emathew1/MPI_3DCompact,
 * compiled unchanged from its own sources with the single-rank shims in
 * oracle/ref_shims) so its outputs can pin the numpy restatement and the GPU
 * path. Test infrastructure only: the product never links or runs this.
 *
 * It replaces the reference's driver (src/MPI_3DCompact.cpp:34-316) with a
 * harness that supplies the mesh, the initial condition and the solver hooks
 * (src/MPI_3DCompact.cpp:318-543 define them for the cylinder case; here they
 * are empty, as in the HIT case tests/hit/Samtaney_D4/MPI_3DCompact.cpp).
 *
 * Run inside a directory holding MPI_3DCompact.in. Modes:
 *   run  <mesh> <ic.bin> <out.bin>        N steps (TIMESTEPPING.MAXTIMESTEP),
 *                                          then dump the conserved state.
 *   ops  <scheme> <dir> <in.bin> <out.bin> one operator on one field:
 *        scheme = PADE6|PENTA10|CD2 (derivative), COMPACT8|COMPACT10 (filter,
 *        SOLVER.ALPHAF) or TESTPADE|TESTEXP (the DSM test filters
 *        CommN5PadeTestFilter / CommN5ExpTestFilter); dir = 0,1,2.
 *   metrics <mesh> <out.bin>               J, J11..J33 from solveForJacobians.
 *   restart <SolutionDump> <out.bin>       restart as src/MPI_3DCompact.cpp:80-271
 *        does (time step, time, mesh and conserved state from the dump,
 *        primitives through IdealGas::solveU/solvep), run to MAXTIMESTEP.
 * <mesh> is "cube:<L>" (x = L*xi, the HIT box), "file:<path>" (x,y,z FP64)
 * or "dump:<path>" (x,y,z after the 5-value header of a SolutionDump file,
 * as AlgebraicSingleBlockMesh::getMesh reads a restart grid,
 * src/AlgebraicSingleBlockMesh.hpp:77-101).
 * Every "run"/"restart" also leaves the reference's own SolutionDump.<step>
 * (written by CurvilinearCSolver::checkEnd at the last step).
 * All binary fields are FP64, x-fastest global order (i + Nx*(j + Ny*k)).
 */
#include <mpi.h>
#include <cmath>
#include <new>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

using namespace std;

#include "C2Decomp.hpp"
#include "Macros.hpp"
#include "Options.hpp"
#include "TimeStepping.hpp"
#include "Domain.hpp"
#include "BC.hpp"
#include "AbstractCSolver.hpp"
#include "CurvilinearCSolver.hpp"
#include "AbstractSingleBlockMesh.hpp"
#include "AbstractRK.hpp"
#include "TVDRK3.hpp"
#include "RK4.hpp"
#include "KenRK4.hpp"
#include "LSLDDRK4.hpp"
#include "CommN5PadeTestFilter.hpp"
#include "CommN5ExpTestFilter.hpp"

// Every allocation of the reference starts zero-filled. Its C2Decomp::alloc*
// arrays come from new[] and are not cleared, and solveForJacobians reads some
// of that memory before writing it on meshes with a wall direction (restarts
// of the same mesh gave different metrics until allocations were zeroed); the
// GPU context zero-initialises its buffers, so the oracle runs do the same.
void *operator new[](size_t n) {
    void *p = calloc(n ? n : 1, 1);
    if (!p) throw std::bad_alloc();
    return p;
}
void *operator new(size_t n) {
    void *p = calloc(n ? n : 1, 1);
    if (!p) throw std::bad_alloc();
    return p;
}
void operator delete[](void *p) noexcept { free(p); }
void operator delete(void *p) noexcept { free(p); }
void operator delete[](void *p, size_t) noexcept { free(p); }
void operator delete(void *p, size_t) noexcept { free(p); }

// wall-clock stamp at the end of every time step (postStep -> fullStepTemporalHook)
static std::vector<double> g_step_stamps;
// MC3D_REF_UPDATE_SPONGE=1: call updateSponge where postStep has it commented
// out (src/CurvilinearCSolver.hpp:355-359), i.e. right after this hook
static bool update_sponge_on() {
    const char *e = getenv("MC3D_REF_UPDATE_SPONGE");
    return e && e[0] == '1';
}

// ---- solver hooks (the reference leaves their bodies to the driver) ----
// Built with MC3D_REF_DRIVER_HOOKS, the harness links the hooks of one of the
// reference's own drivers instead (tests/hit/Samtaney_D4/MPI_3DCompact.cpp or
// src/MPI_3DCompact.cpp, compiled with their main renamed), which append to
// turbdata.out / cylinder{P,U,V,W}.dat / VWakeStrip.dat in the run directory;
// the step stamps are then not recorded.
#ifndef MC3D_REF_DRIVER_HOOKS
void CurvilinearCSolver::initialHook() {}
void CurvilinearCSolver::fullStepTemporalHook() {
    g_step_stamps.push_back(MPI_Wtime());
    if (update_sponge_on()) updateSponge();
}
void CurvilinearCSolver::subStepTemporalHook() {}
void CurvilinearCSolver::preStepBoundaryHook() {}
void CurvilinearCSolver::postStepBoundaryHook() {}
double CurvilinearCSolver::contRHSSource(int) { return 0.0; }
double CurvilinearCSolver::xmomRHSSource(int) { return 0.0; }
double CurvilinearCSolver::ymomRHSSource(int) { return 0.0; }
double CurvilinearCSolver::zmomRHSSource(int) { return 0.0; }
double CurvilinearCSolver::engyRHSSource(int) { return 0.0; }
#endif

static void die(const string &m) {
    fprintf(stderr, "mc3d_ref: %s\n", m.c_str());
    exit(2);
}

static vector<double> read_bin(const string &path, size_t n, size_t skip = 0) {
    vector<double> v(n);
    FILE *f = fopen(path.c_str(), "rb");
    if (!f) die("cannot open " + path);
    if (skip && fseek(f, (long)(skip * sizeof(double)), SEEK_SET) != 0) die("seek " + path);
    if (fread(v.data(), sizeof(double), n, f) != n) die("short read " + path);
    fclose(f);
    return v;
}

// Mesh plugin: the harness's own getMesh (the reference's AlgebraicSingleBlockMesh
// hard-codes its geometry, so each test supplies one here).
class HarnessMesh : public AbstractSingleBlockMesh {
  public:
    string spec;
    HarnessMesh(C2Decomp *c2d_, AbstractCSolver *cs_, Domain *dom, const string &spec_) : spec(spec_) {
        mpiRank = 0;
        cs = cs_;
        c2d = c2d_;
        d = dom;
        derivX = cs->derivX;
        derivY = cs->derivY;
        derivZ = cs->derivZ;
        d->getPencilDecompInfo(pxSize, pySize, pzSize, pxStart, pyStart, pzStart, pxEnd, pyEnd, pzEnd);
        max_xi = d->gLx;
        max_eta = d->gLy;
        max_zta = d->gLz;
        Nx = d->gNx;
        Ny = d->gNy;
        Nz = d->gNz;
        allocateForMesh();
        getMesh();
        // handlePeriodicStuff leaves a periodic direction's translation unset
        // when its faces are neither both PERIODIC (as tested, the Y faces for
        // x, src/AbstractSingleBlockMesh.cpp:2034) nor INTERNALLY_PERIODIC; the
        // members are otherwise uninitialised, so they start from zero here
        for (int c = 0; c < 3; c++)
            periodicXTranslation[c] = periodicYTranslation[c] = periodicZTranslation[c] = 0.0;
        handlePeriodicStuff();
        solveForJacobians();
    }
    void getMesh() {
        vector<double> X, Y, Z;
        double L = 0;
        bool cube = spec.compare(0, 5, "cube:") == 0;
        if (cube) {
            L = atof(spec.c_str() + 5);
        } else if (spec.compare(0, 5, "file:") == 0 || spec.compare(0, 5, "dump:") == 0) {
            size_t n = (size_t)Nx * Ny * Nz;
            vector<double> all = read_bin(spec.substr(5), 3 * n, spec[0] == 'd' ? 5 : 0);
            X.assign(all.begin(), all.begin() + n);
            Y.assign(all.begin() + n, all.begin() + 2 * n);
            Z.assign(all.begin() + 2 * n, all.end());
        } else {
            die("bad mesh spec " + spec);
        }
        for (int i = 0; i < 3; i++) { x_min[i] = 1e300; x_max[i] = -1e300; }
        FOR_Z_YPEN {
            FOR_Y_YPEN {
                FOR_X_YPEN {
                    int ip = GETMAJIND_YPEN;
                    int ii = GETGLOBALXIND_YPEN, jj = GETGLOBALYIND_YPEN, kk = GETGLOBALZIND_YPEN;
                    size_t g = (size_t)ii + (size_t)Nx * (jj + (size_t)Ny * kk);
                    if (cube) {
                        x[ip] = L * d->x[ii];
                        y[ip] = L * d->y[jj];
                        z[ip] = L * d->z[kk];
                    } else {
                        x[ip] = X[g];
                        y[ip] = Y[g];
                        z[ip] = Z[g];
                    }
                    x_min[0] = fmin(x_min[0], x[ip]); x_max[0] = fmax(x_max[0], x[ip]);
                    x_min[1] = fmin(x_min[1], y[ip]); x_max[1] = fmax(x_max[1], y[ip]);
                    x_min[2] = fmin(x_min[2], z[ip]); x_max[2] = fmax(x_max[2], z[ip]);
                }
            }
        }
    }
};

struct Setup {
    Options *opt;
    TimeStepping *ts;
    BC *bc;
    Domain *d;
    C2Decomp *c2d;
};

static Setup make_setup() {
    Setup s;
    s.opt = new Options(0);
    s.ts = new TimeStepping(s.opt);
    bool periodicBC[3];
    s.bc = new BC(s.opt, periodicBC);
    s.d = new Domain(s.opt, 1.0, 1.0, 1.0);
    s.c2d = new C2Decomp(s.opt->Nx, s.opt->Ny, s.opt->Nz, s.opt->pRow, s.opt->pCol, periodicBC);
    s.d->setPencilDecompInfo(s.c2d);
    return s;
}

// global x-fastest <-> reference y-pencil "major" layout (i*Nz*Ny + k*Ny + j)
static inline size_t ymaj(int i, int j, int k, int Ny, int Nz) { return (size_t)i * Nz * Ny + (size_t)k * Ny + j; }
static inline size_t glob(int i, int j, int k, int Nx, int Ny) { return (size_t)i + (size_t)Nx * (j + (size_t)Ny * k); }

static void write_fields(const string &path, const vector<double *> &fields, int Nx, int Ny, int Nz,
                         const double *hdr, int nhdr) {
    FILE *f = fopen(path.c_str(), "wb");
    if (!f) die("cannot write " + path);
    fwrite(hdr, sizeof(double), nhdr, f);
    vector<double> buf((size_t)Nx * Ny * Nz);
    for (double *fld : fields) {
        for (int k = 0; k < Nz; k++)
            for (int j = 0; j < Ny; j++)
                for (int i = 0; i < Nx; i++) buf[glob(i, j, k, Nx, Ny)] = fld[ymaj(i, j, k, Ny, Nz)];
        fwrite(buf.data(), sizeof(double), buf.size(), f);
    }
    fclose(f);
}

static int mode_run(const string &mesh, const string &icpath, const string &out, const string &restart = "") {
    Setup s = make_setup();
    int Nx = s.opt->Nx, Ny = s.opt->Ny, Nz = s.opt->Nz;
    size_t n = (size_t)Nx * Ny * Nz;
    if (!restart.empty()) {
        // src/MPI_3DCompact.cpp:80-110: time step, time and sizes from the header
        vector<double> h = read_bin(restart, 5);
        if ((int)h[2] != Nx || (int)h[3] != Ny || (int)h[4] != Nz) die("restart file sizes differ from DOMAIN");
        s.opt->timeStep = (int)h[0];
        s.opt->time = h[1];
    }
    CurvilinearCSolver *cs = new CurvilinearCSolver(s.c2d, s.d, s.bc, s.ts, s.opt);
    // The reference allocates solver arrays with new[] and never clears them;
    // the momentum update accumulates into rho{U,V,W}k2 (Core.cpp:839,872,904),
    // so every array starts from zero here, as the GPU context does.
    double *arrs[] = {cs->rhok, cs->rhok2, cs->rho2, cs->rhoUk, cs->rhoUk2, cs->rhoU2, cs->rhoVk, cs->rhoVk2,
                      cs->rhoV2, cs->rhoWk, cs->rhoWk2, cs->rhoW2, cs->rhoEk, cs->rhoEk2, cs->rhoE2};
    for (double *a : arrs) memset(a, 0, n * sizeof(double));
    cs->msh = new HarnessMesh(s.c2d, cs, s.d, mesh);
    AbstractRK *rk = nullptr;
    if (s.opt->rkType == Options::TVDRK3) rk = new TVDRK3(cs);
    else if (s.opt->rkType == Options::RK4) rk = new RK4(cs);
    else if (s.opt->rkType == Options::KENRK4) rk = new KenRK4(cs);
    else if (s.opt->rkType == Options::LSLDDRK4) rk = new LSLDDRK4(cs);
    else die("unknown RK type");

    if (restart.empty()) {
        vector<double> ic = read_bin(icpath, 5 * n);
        for (int k = 0; k < Nz; k++)
            for (int j = 0; j < Ny; j++)
                for (int i = 0; i < Nx; i++) {
                    size_t g = glob(i, j, k, Nx, Ny), ip = ymaj(i, j, k, Ny, Nz);
                    cs->rho0[ip] = ic[g];
                    cs->U0[ip] = ic[n + g];
                    cs->V0[ip] = ic[2 * n + g];
                    cs->W0[ip] = ic[3 * n + g];
                    cs->p0[ip] = ic[4 * n + g];
                }
    } else {
        // src/MPI_3DCompact.cpp:220-262: conserved fields after the header and
        // the mesh, primitives through the solver's IdealGas
        vector<double> q = read_bin(restart, 5 * n, 5 + 3 * n);
        for (int k = 0; k < Nz; k++)
            for (int j = 0; j < Ny; j++)
                for (int i = 0; i < Nx; i++) {
                    size_t g = glob(i, j, k, Nx, Ny), ip = ymaj(i, j, k, Ny, Nz);
                    cs->rho0[ip] = q[g];
                    cs->U0[ip] = cs->ig->solveU(q[g], q[n + g]);
                    cs->V0[ip] = cs->ig->solveU(q[g], q[2 * n + g]);
                    cs->W0[ip] = cs->ig->solveU(q[g], q[3 * n + g]);
                    cs->p0[ip] = cs->ig->solvep(q[g], q[4 * n + g], cs->U0[ip], cs->V0[ip], cs->W0[ip]);
                }
    }
    cs->setInitialConditions();

    double t0 = MPI_Wtime();
    rk->executeSolverLoop();
    double t1 = MPI_Wtime();
    fprintf(stderr, "mc3d_ref: wall %.6f s for %d steps\n", t1 - t0, cs->timeStep);
    {
        FILE *st = fopen("step_times.txt", "w");
        if (st) {
            double prev = t0;
            for (double s : g_step_stamps) {
                fprintf(st, "%.9f\n", s - prev);
                prev = s;
            }
            fclose(st);
        }
    }

    double hdr[8] = {(double)cs->timeStep, cs->time, (double)Nx, (double)Ny, (double)Nz, s.ts->dt, t1 - t0, 0.0};
    vector<double *> f = {cs->rho1, cs->rhoU1, cs->rhoV1, cs->rhoW1, cs->rhoE1};
    write_fields(out, f, Nx, Ny, Nz, hdr, 8);
    return 0;
}

static int mode_metrics(const string &mesh, const string &out) {
    Setup s = make_setup();
    int Nx = s.opt->Nx, Ny = s.opt->Ny, Nz = s.opt->Nz;
    CurvilinearCSolver *cs = new CurvilinearCSolver(s.c2d, s.d, s.bc, s.ts, s.opt);
    HarnessMesh *m = new HarnessMesh(s.c2d, cs, s.d, mesh);
    double hdr[8] = {0, 0, (double)Nx, (double)Ny, (double)Nz, 0, 0, 0};
    vector<double *> f = {m->J, m->J11, m->J12, m->J13, m->J21, m->J22, m->J23, m->J31, m->J32, m->J33};
    write_fields(out, f, Nx, Ny, Nz, hdr, 8);
    return 0;
}

// one operator on one field, in the pencil layout the reference uses for it
static int mode_ops(const string &scheme, int dir, const string &in, const string &out) {
    Setup s = make_setup();
    int Nx = s.opt->Nx, Ny = s.opt->Ny, Nz = s.opt->Nz;
    size_t n = (size_t)Nx * Ny * Nz;
    vector<double> src = read_bin(in, n), pin(n), pout(n), dst(n);
    AbstractDerivatives::Direct D = dir == 0 ? AbstractDerivatives::DIRX
                                   : dir == 1 ? AbstractDerivatives::DIRY : AbstractDerivatives::DIRZ;
    Options::BCType bct = dir == 0 ? s.bc->bcXType : dir == 1 ? s.bc->bcYType : s.bc->bcZType;
    // pencil "major" index of (i,j,k) for the operator's direction
    auto pidx = [&](int i, int j, int k) -> size_t {
        if (dir == 0) return (size_t)k * Nx * Ny + (size_t)j * Nx + i;
        if (dir == 1) return (size_t)i * Nz * Ny + (size_t)k * Ny + j;
        return (size_t)j * Nx * Nz + (size_t)i * Nz + k;
    };
    for (int k = 0; k < Nz; k++)
        for (int j = 0; j < Ny; j++)
            for (int i = 0; i < Nx; i++) pin[pidx(i, j, k)] = src[glob(i, j, k, Nx, Ny)];
    if (scheme == "PADE6" || scheme == "PENTA10" || scheme == "CD2") {
        AbstractDerivatives *op;
        if (scheme == "PADE6") op = new Pade6(s.d, bct, D);
        else if (scheme == "PENTA10") op = new Penta10(s.d, bct, D);
        else op = new CD2(s.d, bct, D);
        op->calc1stDerivField(pin.data(), pout.data());
    } else if (scheme == "COMPACT8" || scheme == "COMPACT10" || scheme == "TESTPADE" || scheme == "TESTEXP") {
        AbstractFilter *op;
        if (scheme == "COMPACT8") op = new Compact8Filter(s.opt->alphaF, s.d, s.bc, bct, D);
        else if (scheme == "COMPACT10") op = new Compact10Filter(s.opt->alphaF, s.d, s.bc, bct, D);
        else if (scheme == "TESTPADE") op = new CommN5PadeTestFilter(s.d, s.bc, bct, D);
        else op = new CommN5ExpTestFilter(s.d, s.bc, bct, D);
        op->filterField(pin.data(), pout.data());
    } else {
        die("unknown operator " + scheme);
    }
    for (int k = 0; k < Nz; k++)
        for (int j = 0; j < Ny; j++)
            for (int i = 0; i < Nx; i++) dst[glob(i, j, k, Nx, Ny)] = pout[pidx(i, j, k)];
    FILE *f = fopen(out.c_str(), "wb");
    if (!f) die("cannot write " + out);
    fwrite(dst.data(), sizeof(double), n, f);
    fclose(f);
    return 0;
}

int main(int argc, char **argv) {
    MPI_Init(&argc, &argv);
    if (argc < 2) die("usage: mc3d_ref run|ops|metrics|restart ...");
    string mode = argv[1];
    int rc = 2;
    if (mode == "run" && argc == 5) rc = mode_run(argv[2], argv[3], argv[4]);
    else if (mode == "ops" && argc == 6) rc = mode_ops(argv[2], atoi(argv[3]), argv[4], argv[5]);
    else if (mode == "metrics" && argc == 4) rc = mode_metrics(argv[2], argv[3]);
    else if (mode == "restart" && argc == 4) rc = mode_run(string("dump:") + argv[2], "", argv[3], argv[2]);
    else die("bad arguments");
    MPI_Finalize();
    return rc;
}
