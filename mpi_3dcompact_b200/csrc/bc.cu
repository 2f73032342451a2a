// Boundary conditions of the time step on the device (src/CurvilinearCSolver_BC.cpp):
//
//   wall_prestep   preStepBCHandling on one wall face (:372-700): wall
//                  velocity (zero, or the moving-wall tangential velocity),
//                  the Neumann wall temperature of adiabatic walls from the six
//                  (CD2: two) points inward along the wall normal, p = rho R T
//                  and rhoE; both the stage state (FP64) and its primitives;
//   face_k2        postStepBCHandling on one face (:702-842): walls keep
//                  only -dt J d(rho U^xi_d)/dxi_d in the continuity k2 and
//                  zero the others, sponge faces zero all five;
//   sponge_source  sigma (avg - q) / J added to the RHS of every equation
//                  (solveContinuity .. solveEnergy, Core.cpp:790-947, with
//                  calcSpongeSource of src/CurvilinearCSolver.hpp:293-295).
#include <cmath>

#include "pointwise_common.cuh"

namespace mc3d {

namespace {

// point (a, b) of face f (0 X0, 1 X1, 2 Y0, 3 Y1, 4 Z0, 5 Z1): its index and
// the index step one point inward along the wall normal
struct FacePoint {
    long long idx, step;
};
__device__ __forceinline__ FacePoint face_point(const Grid3 &g, int f, int a, int b) {
    const int d = f >> 1, side = f & 1;
    long long i, j, k, step;
    if (d == 0) {
        i = side ? g.Nx - 1 : 0;
        j = a;
        k = b;
        step = 1;
    } else if (d == 1) {
        i = a;
        j = side ? g.Ny - 1 : 0;
        k = b;
        step = g.Nx;
    } else {
        i = a;
        j = b;
        k = side ? g.Nz - 1 : 0;
        step = (long long)g.Nx * g.Ny;
    }
    FacePoint p;
    p.idx = i + (long long)g.Nx * (j + (long long)g.Ny * k);
    p.step = side ? -step : step;
    return p;
}

__device__ __forceinline__ void face_dims(const Grid3 &g, int f, int &na, int &nb) {
    const int d = f >> 1;
    na = d == 0 ? g.Ny : g.Nx;
    nb = d == 2 ? g.Ny : g.Nz;
}

template <typename R>
__global__ void wall_prestep_kernel(Grid3 g, int f, int neumann, int fd_type, double vt1, double vt2, Q5d q,
                                    P5w<R> prim) {
    int na, nb;
    face_dims(g, f, na, nb);
    const long long np = (long long)na * nb;
    const int d = f >> 1;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < np; t += (long long)gridDim.x * blockDim.x) {
        const FacePoint fp = face_point(g, f, (int)(t % na), (int)(t / na));
        const long long i = fp.idx;
        R T = prim.p[4][i];
        if (neumann) {
            // AbstractDerivatives::calcNeumann (src/Pade6.cpp:395-397, src/CD2.cpp:183)
            const R *Tp = prim.p[4];
            if (fd_type == MC3D_CD2) {
                T = (Tp[i + fp.step] * (R)4.0 - Tp[i + 2 * fp.step] * (R)1.0) / (R)3.0;
            } else {
                T = (Tp[i + fp.step] * (R)360.0 - Tp[i + 2 * fp.step] * (R)450.0 + Tp[i + 3 * fp.step] * (R)400.0 -
                     Tp[i + 4 * fp.step] * (R)225.0 + Tp[i + 5 * fp.step] * (R)72.0 - Tp[i + 6 * fp.step] * (R)10.0) /
                    (R)147.0;
            }
        }
        // wall velocity: zero normal component, tangential (vt1, vt2) in axis order
        double u[3];
        u[d] = 0.0;
        u[d == 0 ? 1 : 0] = vt1;
        u[d == 2 ? 1 : 2] = vt2;
        const double rho = q.p[0][i];
        q.p[1][i] = rho * u[0];
        q.p[2][i] = rho * u[1];
        q.p[3][i] = rho * u[2];
        // solvep_idealgas, solverhoE (src/IdealGas.hpp:66-80)
        const double p = rho * R_GAS * (double)T;
        q.p[4][i] = p / (GAMMA - 1.0) + 0.5 * rho * (u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
        prim.p[1][i] = (R)u[0];
        prim.p[2][i] = (R)u[1];
        prim.p[3][i] = (R)u[2];
        prim.p[4][i] = T;
    }
}

template <typename R>
__global__ void wall_save_T_kernel(Grid3 g, int f, const R *T, R *Tmu) {
    int na, nb;
    face_dims(g, f, na, nb);
    const long long np = (long long)na * nb;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < np; t += (long long)gridDim.x * blockDim.x) {
        const long long i = face_point(g, f, (int)(t % na), (int)(t / na)).idx;
        Tmu[i] = T[i];
    }
}

template <typename R>
__global__ void face_k2_kernel(Grid3 g, int f, int wall, const R *cont, const R *J, R Jc, const double *dt,
                               P5w<R> k2) {
    int na, nb;
    face_dims(g, f, na, nb);
    const long long np = (long long)na * nb;
    const R mdt = (R)(-*dt);
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < np; t += (long long)gridDim.x * blockDim.x) {
        const long long i = face_point(g, f, (int)(t % na), (int)(t / na)).idx;
        k2.p[0][i] = wall ? mdt * (J ? J[i] : Jc) * cont[i] : R(0);
        k2.p[1][i] = R(0);
        k2.p[2][i] = R(0);
        k2.p[3][i] = R(0);
        k2.p[4][i] = R(0);
    }
}

template <typename R>
__global__ void sponge_source_kernel(Grid3 g, const double *__restrict__ sigma, Q5c avg, Q5c q, const R *J, R Jc,
                                     P5w<R> rhs) {
    const long long n = g.n();
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const double s = sigma[i];
        // outside the sponge (sigma = 0) a finite state adds a zero: the state,
        // the target and the right-hand side there are not read (a cylindrical
        // sponge covers a few of the radial lines)
        if (s == 0.0) continue;
        const R Jv = J ? J[i] : Jc;
#pragma unroll
        for (int e = 0; e < 5; e++) rhs.p[e][i] += (R)(s * (avg.p[e][i] - q.p[e][i])) / Jv;
    }
}

inline int face_blocks(const Grid3 &g, int f) {
    const int d = f >> 1;
    const long long np = (long long)(d == 0 ? g.Ny : g.Nx) * (d == 2 ? g.Ny : g.Nz);
    long long b = (np + 255) / 256;
    return (int)(b < 1 ? 1 : (b > 148 * 8 ? 148 * 8 : b));
}

}  // namespace

template <typename R>
int launch_wall_prestep(const Grid3 &g, int face, int neumann, int fd_type, double vt1, double vt2,
                        double *const q[5], R *const prim[5], cudaStream_t st) {
    Q5d qq;
    P5w<R> pp;
    for (int v = 0; v < 5; v++) {
        qq.p[v] = q[v];
        pp.p[v] = prim[v];
    }
    wall_prestep_kernel<R><<<face_blocks(g, face), 256, 0, st>>>(g, face, neumann, fd_type, vt1, vt2, qq, pp);
    MC3D_CUDA_TRY(cudaGetLastError());
    return MC3D_OK;
}

template <typename R>
int launch_wall_save_T(const Grid3 &g, int wall_mask, const R *T, R *Tmu, cudaStream_t st) {
    for (int f = 0; f < 6; f++) {
        if (!(wall_mask >> f & 1)) continue;
        wall_save_T_kernel<R><<<face_blocks(g, f), 256, 0, st>>>(g, f, T, Tmu);
        MC3D_CUDA_TRY(cudaGetLastError());
    }
    return MC3D_OK;
}

template <typename R>
int launch_face_k2(const Grid3 &g, int face, int wall, const R *cont, const R *J, R Jc, const double *dt,
                   R *const k2[5], cudaStream_t st) {
    P5w<R> kk;
    for (int v = 0; v < 5; v++) kk.p[v] = k2[v];
    face_k2_kernel<R><<<face_blocks(g, face), 256, 0, st>>>(g, face, wall, cont, J, Jc, dt, kk);
    MC3D_CUDA_TRY(cudaGetLastError());
    return MC3D_OK;
}

template <typename R>
int launch_sponge_source(const Grid3 &g, const double *sigma, const double *const avg[5], const double *const q[5],
                         const R *J, R Jc, R *const rhs[5], cudaStream_t st) {
    Q5c a, qq;
    P5w<R> r;
    for (int v = 0; v < 5; v++) {
        a.p[v] = avg[v];
        qq.p[v] = q[v];
        r.p[v] = rhs[v];
    }
    sponge_source_kernel<R><<<grid_for(g.n(), 256), 256, 0, st>>>(g, sigma, a, qq, J, Jc, r);
    MC3D_CUDA_TRY(cudaGetLastError());
    return MC3D_OK;
}

#define MC3D_BC_INST(R)                                                                                          \
    template int launch_wall_save_T<R>(const Grid3 &, int, const R *, R *, cudaStream_t);                        \
    template int launch_wall_prestep<R>(const Grid3 &, int, int, int, double, double, double *const[5],           \
                                        R *const[5], cudaStream_t);                                              \
    template int launch_face_k2<R>(const Grid3 &, int, int, const R *, const R *, R, const double *, R *const[5], \
                                   cudaStream_t);                                                                \
    template int launch_sponge_source<R>(const Grid3 &, const double *, const double *const[5],                  \
                                         const double *const[5], const R *, R, R *const[5], cudaStream_t);
MC3D_BC_INST(float)
MC3D_BC_INST(double)
#undef MC3D_BC_INST

// updateSponge (src/CurvilinearCSolver_BC.cpp:843-928): the sponge target
// relaxes toward the state with eps = 1/(avgT/dt + 1), its energy blended
// toward the back pressure with epsP = 0.005 (src/SpongeBC.cpp:37); then the
// points of every SPONGE face take the target state.
__global__ void sponge_relax_kernel(Grid3 g, Q5d q, Q5d avg, const TimeState *ts, double avg_t, double p_inf,
                                    int sponge_faces) {
    const double eps = 1.0 / (avg_t / ts->dt + 1.0);
    const double eps_p = 0.005;
    const long long n = g.n();
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        double a[5];
        for (int v = 0; v < 5; v++) a[v] = avg.p[v][i] + eps * (q.p[v][i] - avg.p[v][i]);
        a[4] = eps_p * a[4] + (1.0 - eps_p) * (p_inf / (GAMMA - 1.0) + 0.5 * (a[1] * a[1] + a[2] * a[2] + a[3] * a[3]) / a[0]);
        for (int v = 0; v < 5; v++) avg.p[v][i] = a[v];
        const long long x = i % g.Nx, y = (i / g.Nx) % g.Ny, z = i / ((long long)g.Nx * g.Ny);
        const bool on = ((sponge_faces & 1) && x == 0) || ((sponge_faces & 2) && x == g.Nx - 1) ||
                        ((sponge_faces & 4) && y == 0) || ((sponge_faces & 8) && y == g.Ny - 1) ||
                        ((sponge_faces & 16) && z == 0) || ((sponge_faces & 32) && z == g.Nz - 1);
        if (on)
            for (int v = 0; v < 5; v++) q.p[v][i] = a[v];
    }
}

int launch_sponge_relax(const Grid3 &g, double *const q[5], double *const avg[5], const TimeState *ts, double avg_t,
                        double p_inf, int sponge_faces, cudaStream_t st) {
    Q5d qq, aa;
    for (int v = 0; v < 5; v++) {
        qq.p[v] = q[v];
        aa.p[v] = avg[v];
    }
    sponge_relax_kernel<<<grid_for(g.n(), 256), 256, 0, st>>>(g, qq, aa, ts, avg_t, p_inf, sponge_faces);
    MC3D_CUDA_TRY(cudaGetLastError());
    return MC3D_OK;
}

}  // namespace mc3d
