/*
 * Test driver of the GPU adapters (mpi_3dcompact_b200/adapters/mc3d_adapters.hpp):
 * each GPU object is used through the reference's own base-class pointer
 * (AbstractDerivatives*, AbstractFilter*, AbstractCSolver* + AbstractRK*,
 * AbstractSGS*) exactly as the reference's solver calls them. Built by
 * oracle/Makefile against the reference's headers and objects (compiled
 * unchanged, single-rank shims); test infrastructure only.
 *
 * Run inside a directory holding MPI_3DCompact.in. Modes:
 *   ops <seed>    every derivative (calc1stDerivField, calc1stDerivField_TPB
 *                 with random ghost planes) and filter (filterField) of the
 *                 config's BC types along x, y, z: the reference's class on
 *                 its pencil layout and the GPU adapter on the device, same
 *                 input; prints "op <name> <dir> <kind> <max |gpu-ref| / max |ref|>"
 *   solver <ic.bin> <out.bin>   GpuCurvilinearCSolver + GpuRK driven by the
 *                 reference's loop through the base classes until endFlag
 *                 (MAXTIMESTEP), on the 2*pi box; writes the conserved state
 *                 (x fastest, after a header: time step, time) and prints the
 *                 largest difference from mc3d_solver_step on the same input
 *   sgs <in.bin> <out.bin> [closure.bin]   GpuVremanSGS or GpuDSMSGS
 *                 (LES.LESMODEL), or with a closure file GpuMlpSGS (the
 *                 learned closure, SOLVER.MU_REF), via AbstractSGS*:
 *                 in = gradU (9), rho..rhoE (5), T, gradT (3);
 *                 out = mu_sgs, taukk, k_sgs (FP64, x fastest)
 */
#include <mpi.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <random>
#include <string>
#include <vector>

using namespace std;

#include "AbstractCSolver.hpp"
#include "AbstractRK.hpp"
#include "AbstractSGS.hpp"
#include "BC.hpp"
#include "C2Decomp.hpp"
#include "CD2.hpp"
#include "CommN5ExpTestFilter.hpp"
#include "CommN5PadeTestFilter.hpp"
#include "Compact10Filter.hpp"
#include "Compact8Filter.hpp"
#include "Domain.hpp"
#include "Options.hpp"
#include "Pade6.hpp"
#include "Penta10.hpp"
#include "TimeStepping.hpp"
#include "mc3d_adapters.hpp"

using namespace mc3d_adapters;

static void die(const string &m) {
    fprintf(stderr, "adapter_driver: %s\n", m.c_str());
    exit(2);
}

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

static inline size_t glob(int i, int j, int k, int Nx, int Ny) { return (size_t)i + (size_t)Nx * (j + (size_t)Ny * k); }

static vector<double> read_bin(const string &path, size_t n) {
    vector<double> v(n);
    FILE *f = fopen(path.c_str(), "rb");
    if (!f || fread(v.data(), sizeof(double), n, f) != n) die("cannot read " + path);
    fclose(f);
    return v;
}

struct Dev {
    double *p = nullptr;
    size_t n = 0;
    explicit Dev(size_t n_) : n(n_) {
        if (cudaMalloc((void **)&p, n * sizeof(double)) != cudaSuccess) die("cudaMalloc");
    }
    Dev(const Dev &) = delete;
    ~Dev() { cudaFree(p); }
    void put(const double *h) { cudaMemcpy(p, h, n * sizeof(double), cudaMemcpyHostToDevice); }
    void get(double *h) const { cudaMemcpy(h, p, n * sizeof(double), cudaMemcpyDeviceToHost); }
};

static double rel_max(const vector<double> &a, const vector<double> &b) {
    double num = 0, den = 0;
    for (size_t i = 0; i < a.size(); i++) {
        num = max(num, fabs(a[i] - b[i]));
        den = max(den, fabs(b[i]));
    }
    return den > 0 ? num / den : num;
}

// ---- ops ------------------------------------------------------------------
static int mode_ops(int seed) {
    Setup s = make_setup();
    const int Nx = s.opt->Nx, Ny = s.opt->Ny, Nz = s.opt->Nz;
    const size_t n = (size_t)Nx * Ny * Nz;
    mt19937_64 rng(seed);
    normal_distribution<double> nd(0.0, 1.0);
    vector<double> f(n);
    for (double &v : f) v = nd(rng);
    Dev din(n), dout(n);
    din.put(f.data());
    const char *dname = "xyz";
    for (int dir = 0; dir < 3; dir++) {
        const AbstractDerivatives::Direct D =
            dir == 0 ? AbstractDerivatives::DIRX : dir == 1 ? AbstractDerivatives::DIRY : AbstractDerivatives::DIRZ;
        const Options::BCType bct = dir == 0 ? s.bc->bcXType : dir == 1 ? s.bc->bcYType : s.bc->bcZType;
        // the reference's pencil "major" index of (i,j,k) for this direction and
        // its ghost-plane index (src/Pade6.cpp:48-107)
        auto pidx = [&](int i, int j, int k) -> size_t {
            if (dir == 0) return (size_t)k * Nx * Ny + (size_t)j * Nx + i;
            if (dir == 1) return (size_t)i * Nz * Ny + (size_t)k * Ny + j;
            return (size_t)j * Nx * Nz + (size_t)i * Nz + k;
        };
        auto ref_plane = [&](int i, int j, int k) -> size_t {
            if (dir == 0) return (size_t)k * Ny + j;
            if (dir == 1) return (size_t)i * Nz + k;
            return (size_t)j * Nx + i;
        };
        auto our_plane = [&](int i, int j, int k) -> size_t {
            if (dir == 0) return (size_t)k * Ny + j;
            if (dir == 1) return (size_t)k * Nx + i;
            return (size_t)j * Nx + i;
        };
        const size_t np = dir == 0 ? (size_t)Ny * Nz : dir == 1 ? (size_t)Nx * Nz : (size_t)Nx * Ny;
        vector<double> pin(n), pout(n), got(n), ref(n);
        for (int k = 0; k < Nz; k++)
            for (int j = 0; j < Ny; j++)
                for (int i = 0; i < Nx; i++) pin[pidx(i, j, k)] = f[glob(i, j, k, Nx, Ny)];
        auto unpencil = [&]() {
            for (int k = 0; k < Nz; k++)
                for (int j = 0; j < Ny; j++)
                    for (int i = 0; i < Nx; i++) ref[glob(i, j, k, Nx, Ny)] = pout[pidx(i, j, k)];
        };
        // six ghost planes (Nm3 .. Np3), in both layouts
        vector<vector<double>> gref(6, vector<double>(np)), gour(6, vector<double>(np));
        for (int m = 0; m < 6; m++)
            for (int k = 0; k < Nz; k++)
                for (int j = 0; j < Ny; j++)
                    for (int i = 0; i < Nx; i++) {
                        if ((dir == 0 && i) || (dir == 1 && j) || (dir == 2 && k)) continue;
                        const double v = nd(rng);
                        gref[m][ref_plane(i, j, k)] = v;
                        gour[m][our_plane(i, j, k)] = v;
                    }
        vector<Dev *> gdev;
        for (int m = 0; m < 6; m++) {
            gdev.push_back(new Dev(np));
            gdev[m]->put(gour[m].data());
        }
        const char *schemes[3] = {"PADE6", "PENTA10", "CD2"};
        for (int sc = 0; sc < 3; sc++) {
            AbstractDerivatives *r, *g;
            if (sc == 0) {
                r = new Pade6(s.d, bct, D);
                g = new GpuPade6(s.d, bct, D);
            } else if (sc == 1) {
                r = new Penta10(s.d, bct, D);
                g = new GpuPenta10(s.d, bct, D);
            } else {
                r = new CD2(s.d, bct, D);
                g = new GpuCD2(s.d, bct, D);
            }
            r->calc1stDerivField(pin.data(), pout.data());
            unpencil();
            g->calc1stDerivField(din.p, dout.p);
            dout.get(got.data());
            printf("op %s %c deriv %.3e\n", schemes[sc], dname[dir], rel_max(got, ref));
            if (bct == Options::PERIODIC_SOLVE) {
                double *G[6], *R[6];
                for (int m = 0; m < 6; m++) {
                    G[m] = gdev[m]->p;
                    R[m] = gref[m].data();
                }
                if (sc == 1) {
                    r->calc1stDerivField_TPB(pin.data(), pout.data(), R[0], R[1], R[2], R[3], R[4], R[5]);
                    g->calc1stDerivField_TPB(din.p, dout.p, G[0], G[1], G[2], G[3], G[4], G[5]);
                } else {
                    r->calc1stDerivField_TPB(pin.data(), pout.data(), R[1], R[2], R[3], R[4]);
                    g->calc1stDerivField_TPB(din.p, dout.p, G[1], G[2], G[3], G[4]);
                }
                unpencil();
                dout.get(got.data());
                printf("op %s %c tpb %.3e\n", schemes[sc], dname[dir], rel_max(got, ref));
            }
            // calcNeumann on six host values
            double w[6] = {1.0, 1.1, 1.3, 1.6, 2.0, 2.5};
            printf("op %s %c neumann %.3e\n", schemes[sc], dname[dir],
                   fabs(g->calcNeumann(w) - r->calcNeumann(w)) / fabs(r->calcNeumann(w)));
            delete r;
            delete g;
        }
        const char *filters[4] = {"COMPACT8", "COMPACT10", "TESTPADE", "TESTEXP"};
        for (int fc = 0; fc < 4; fc++) {
            AbstractFilter *r, *g;
            if (fc == 0) {
                r = new Compact8Filter(s.opt->alphaF, s.d, s.bc, bct, D);
                g = new GpuCompact8Filter(s.opt->alphaF, s.d, s.bc, bct, D);
            } else if (fc == 1) {
                r = new Compact10Filter(s.opt->alphaF, s.d, s.bc, bct, D);
                g = new GpuCompact10Filter(s.opt->alphaF, s.d, s.bc, bct, D);
            } else if (fc == 2) {
                r = new CommN5PadeTestFilter(s.d, s.bc, bct, D);
                g = new GpuCommN5PadeTestFilter(s.d, s.bc, bct, D);
            } else {
                r = new CommN5ExpTestFilter(s.d, s.bc, bct, D);
                g = new GpuCommN5ExpTestFilter(s.d, s.bc, bct, D);
            }
            r->filterField(pin.data(), pout.data());
            unpencil();
            g->filterField(din.p, dout.p);
            dout.get(got.data());
            printf("op %s %c filter %.3e\n", filters[fc], dname[dir], rel_max(got, ref));
            delete r;
            delete g;
        }
        for (Dev *d : gdev) delete d;
    }
    return 0;
}

// ---- solver + RK through the base classes ---------------------------------
static int mode_solver(const string &icpath, const string &outpath) {
    Setup s = make_setup();
    const int Nx = s.opt->Nx, Ny = s.opt->Ny, Nz = s.opt->Nz;
    const size_t n = (size_t)Nx * Ny * Nz;
    vector<double> ic = read_bin(icpath, 5 * n);
    const double L = 6.283185307179586;
    GpuCurvilinearCSolver *g = new GpuCurvilinearCSolver("MPI_3DCompact.in", s.opt, s.d, s.bc, s.ts);
    AbstractCSolver *cs = g;
    cs->initializeSolverData();
    g->setBoxMetrics(L, L, L);
    cs->rho0 = ic.data();
    cs->U0 = ic.data() + n;
    cs->V0 = ic.data() + 2 * n;
    cs->W0 = ic.data() + 3 * n;
    cs->p0 = ic.data() + 4 * n;
    cs->setInitialConditions();
    AbstractRK *rk = new GpuRK(cs, g->cfg.rk_type);
    rk->executeSolverLoop();
    vector<double> q(5 * n);
    g->getConserved(q.data(), q.data() + n, q.data() + 2 * n, q.data() + 3 * n, q.data() + 4 * n);
    // the same steps through mc3d_solver_step
    mc3d_solver d = nullptr;
    check(mc3d_solver_create(&g->cfg, 0, &d), "mc3d_solver_create");
    check(mc3d_solver_set_box_metrics(d, L, L, L), "set_box_metrics");
    check(mc3d_solver_set_initial(d, ic.data(), ic.data() + n, ic.data() + 2 * n, ic.data() + 3 * n,
                                  ic.data() + 4 * n),
          "set_initial");
    check(mc3d_solver_step(d, cs->timeStep - s.opt->timeStep), "mc3d_solver_step");
    vector<double> qd(5 * n);
    check(mc3d_solver_get_conserved(d, qd.data(), qd.data() + n, qd.data() + 2 * n, qd.data() + 3 * n,
                                    qd.data() + 4 * n),
          "get_conserved");
    double diff = 0;
    for (size_t i = 0; i < 5 * n; i++) diff = max(diff, fabs(q[i] - qd[i]));
    int ts2 = 0;
    double t2 = 0, dt2 = 0;
    long long st2 = 0;
    check(mc3d_solver_info(d, &ts2, &t2, &dt2, &st2), "info");
    mc3d_solver_destroy(d);
    printf("solver steps %d time %.17g vs_step_max_abs_diff %.3e same_time %d\n", cs->timeStep, cs->time, diff,
           (int)(ts2 == cs->timeStep && t2 == cs->time));
    FILE *f = fopen(outpath.c_str(), "wb");
    if (!f) die("cannot write " + outpath);
    const double hdr[2] = {(double)cs->timeStep, cs->time};
    fwrite(hdr, sizeof(double), 2, f);
    fwrite(q.data(), sizeof(double), q.size(), f);
    fclose(f);
    delete rk;
    delete g;
    return 0;
}

// ---- SGS through AbstractSGS ----------------------------------------------
static int mode_sgs(const string &inpath, const string &outpath, const char *closure) {
    Setup s = make_setup();
    const int Nx = s.opt->Nx, Ny = s.opt->Ny, Nz = s.opt->Nz;
    const size_t n = (size_t)Nx * Ny * Nz;
    vector<double> in = read_bin(inpath, 18 * n);
    vector<Dev *> f;
    for (int c = 0; c < 18; c++) {
        f.push_back(new Dev(n));
        f[c]->put(in.data() + c * n);
    }
    // the HIT box: J = 1/(2 pi)^3
    const double L = 6.283185307179586, Jc = 1.0 / (L * L * L);
    const Options::StatsAvgType a = s.opt->musgsAvgType;
    const int avg = a == Options::NONE      ? MC3D_AVG_NONE
                    : a == Options::XI1_AVG ? MC3D_AVG_XI1
                    : a == Options::XI2_AVG ? MC3D_AVG_XI2
                    : a == Options::XI3_AVG ? MC3D_AVG_XI3
                    : a == Options::LOCAL   ? MC3D_AVG_LOCAL
                                            : MC3D_AVG_GLOBAL;
    AbstractSGS *sgs;
    mc3d_mlp net = nullptr;
    if (closure) {
        if (mc3d_mlp_create(0, 0, &net) != MC3D_OK || mc3d_mlp_load(net, closure) != MC3D_OK)
            die(string("closure: ") + mc3d_last_error());
        sgs = new GpuMlpSGS(net, s.opt->mu_ref, s.d, s.bc, nullptr, Jc);
    } else if (s.opt->lesModel == Options::VREMAN) {
        sgs = new GpuVremanSGS(avg, s.d, s.bc, nullptr, Jc);
    } else {
        sgs = new GpuDSMSGS(avg, s.opt->testFilterType, s.opt->useTaukk, s.d, s.bc, nullptr, Jc);
    }
    double *gu[3][3];
    for (int a2 = 0; a2 < 3; a2++)
        for (int b = 0; b < 3; b++) gu[a2][b] = f[3 * a2 + b]->p;
    double *gT[3] = {f[15]->p, f[16]->p, f[17]->p};
    sgs->getSGSViscosity(gu, f[9]->p, f[10]->p, f[11]->p, f[12]->p, f[13]->p);
    sgs->calcMuSGSTaukk(gu, f[9]->p, f[10]->p, f[11]->p, f[12]->p, f[13]->p);
    sgs->calcKSGS(gT, f[9]->p, f[10]->p, f[11]->p, f[12]->p, f[14]->p);
    if (cudaDeviceSynchronize() != cudaSuccess) die("CUDA error");
    vector<double> out(3 * n);
    cudaMemcpy(out.data(), sgs->mu_sgs, n * 8, cudaMemcpyDeviceToHost);
    cudaMemcpy(out.data() + n, sgs->taukk, n * 8, cudaMemcpyDeviceToHost);
    cudaMemcpy(out.data() + 2 * n, sgs->k_sgs, n * 8, cudaMemcpyDeviceToHost);
    FILE *fo = fopen(outpath.c_str(), "wb");
    if (!fo) die("cannot write " + outpath);
    fwrite(out.data(), sizeof(double), out.size(), fo);
    fclose(fo);
    printf("sgs ok\n");
    delete sgs;
    if (net) mc3d_mlp_destroy(net);
    for (Dev *d : f) delete d;
    return 0;
}

int main(int argc, char **argv) {
    MPI_Init(&argc, &argv);
    if (argc < 2) die("usage: adapter_driver ops <seed> | solver <ic> <out> | sgs <in> <out> [closure]");
    const string mode = argv[1];
    int rc = 2;
    try {
        if (mode == "ops" && argc == 3) rc = mode_ops(atoi(argv[2]));
        else if (mode == "solver" && argc == 4) rc = mode_solver(argv[2], argv[3]);
        else if (mode == "sgs" && (argc == 4 || argc == 5)) rc = mode_sgs(argv[2], argv[3], argc == 5 ? argv[4] : nullptr);
        else die("bad arguments");
    } catch (const std::exception &e) {
        die(e.what());
    }
    MPI_Finalize();
    return rc;
}
