// Running statistics of the solver, FP64 on the device:
// Stats::updateStatsFields and Stats::doAveraging (src/Stats.cpp:127-347).
// The arithmetic follows the reference's expressions term by term with
// explicitly rounded operations (no contraction), so each point reproduces
// its update exactly given the same state.
#include "mc3d_internal.h"
#include "pointwise_common.cuh"

namespace mc3d {
namespace {

__device__ __forceinline__ double m_(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double a_(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double s_(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double d_(double a, double b) { return __ddiv_rn(a, b); }

// (ow (R R + A A) + dt x x) / nw
__device__ __forceinline__ double second(double ow, double nw, double dt, double R, double A, double x) {
    return d_(a_(m_(ow, a_(m_(R, R), m_(A, A))), m_(m_(dt, x), x)), nw);
}
// (ow (C + A B) + dt x y) / nw
__device__ __forceinline__ double cross(double ow, double nw, double dt, double C, double A, double B, double x,
                                        double y) {
    return d_(a_(m_(ow, a_(C, m_(A, B))), m_(m_(dt, x), y)), nw);
}
// (ow A + dt x) / nw
__device__ __forceinline__ double first(double ow, double nw, double dt, double A, double x) {
    return d_(a_(m_(ow, A), m_(dt, x)), nw);
}

// U, V, W, p, T of the filtered state (updateNonConservedData, Core.cpp:1165-1177)
__device__ __forceinline__ void state_prims(const StatsIn &in, long long i, double &U, double &V, double &W,
                                            double &p, double &T) {
    const double rho = in.q[0][i];
    U = d_(in.q[1][i], rho);
    V = d_(in.q[2][i], rho);
    W = d_(in.q[3][i], rho);
    const double ke = m_(m_(0.5, rho), a_(a_(m_(U, U), m_(V, V)), m_(W, W)));
    p = m_(GAMMA - 1, s_(in.q[4][i], ke));
    T = d_(p, m_(rho, R_GAS));
}

__global__ void stats_accumulate_kernel(long long n, StatsIn in, StatsOut v, StatsOut t, double dt, double ovw,
                                        double nvw, double otw, double ntw, int vel, int thermo) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        double U, V, W, p, T;
        state_prims(in, i, U, V, W, p, T);
        if (vel) {
            const double UA = v.p[0][i], VA = v.p[1][i], WA = v.p[2][i];
            v.p[3][i] = second(ovw, nvw, dt, v.p[3][i], UA, U);
            v.p[4][i] = second(ovw, nvw, dt, v.p[4][i], VA, V);
            v.p[5][i] = second(ovw, nvw, dt, v.p[5][i], WA, W);
            v.p[6][i] = cross(ovw, nvw, dt, v.p[6][i], UA, VA, U, V);
            v.p[7][i] = cross(ovw, nvw, dt, v.p[7][i], UA, WA, U, W);
            v.p[8][i] = cross(ovw, nvw, dt, v.p[8][i], VA, WA, V, W);
            v.p[0][i] = first(ovw, nvw, dt, UA, U);
            v.p[1][i] = first(ovw, nvw, dt, VA, V);
            v.p[2][i] = first(ovw, nvw, dt, WA, W);
        }
        if (thermo) {
            const double rho = in.rho2[i];   // Stats takes rho from rho2 (src/Stats.hpp:45)
            const double RA = t.p[0][i], PA = t.p[2][i], TA = t.p[4][i];
            t.p[1][i] = second(otw, ntw, dt, t.p[1][i], RA, rho);
            t.p[3][i] = second(otw, ntw, dt, t.p[3][i], PA, p);
            t.p[5][i] = second(otw, ntw, dt, t.p[5][i], TA, T);
            t.p[0][i] = first(otw, ntw, dt, RA, rho);
            t.p[2][i] = first(otw, ntw, dt, PA, p);
            t.p[4][i] = first(otw, ntw, dt, TA, T);
        }
    }
}

// XI1 (dir 0) or XI3 (dir 2) index mean of every line, summed as phi/N in
// index order and written back to the whole line (Stats.cpp:227-264, 297-335)
__global__ void stats_line_mean_kernel(Grid3 g, int dir, StatsOut f, int nf) {
    const long long nlines = dir == 0 ? (long long)g.Ny * g.Nz : (long long)g.Nx * g.Ny;
    const int N = dir == 0 ? g.Nx : g.Nz;
    const long long stride = dir == 0 ? 1 : (long long)g.Nx * g.Ny;
    const double Nd = (double)N;
    for (long long l = blockIdx.x * (long long)blockDim.x + threadIdx.x; l < nlines * nf;
         l += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(l / nlines);
        const long long line = l - k * nlines;
        const long long base = dir == 0 ? line * g.Nx : line;
        double *p = f.p[k];
        double acc = 0.0;
        for (int n = 0; n < N; n++) acc = a_(acc, d_(p[base + n * stride], Nd));
        for (int n = 0; n < N; n++) p[base + n * stride] = acc;
    }
}

// RMS = sqrt(|<x^2> - <x>^2|), Reynolds stresses <xy> - <x><y> (Stats.cpp:158-167, :205-211)
__global__ void stats_finish_kernel(long long n, StatsOut v, StatsOut t, int vel, int thermo) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        if (vel) {
            const double UA = v.p[0][i], VA = v.p[1][i], WA = v.p[2][i];
            v.p[3][i] = sqrt(fabs(s_(v.p[3][i], m_(UA, UA))));
            v.p[4][i] = sqrt(fabs(s_(v.p[4][i], m_(VA, VA))));
            v.p[5][i] = sqrt(fabs(s_(v.p[5][i], m_(WA, WA))));
            v.p[6][i] = s_(v.p[6][i], m_(UA, VA));
            v.p[7][i] = s_(v.p[7][i], m_(UA, WA));
            v.p[8][i] = s_(v.p[8][i], m_(VA, WA));
        }
        if (thermo) {
            t.p[1][i] = sqrt(fabs(s_(t.p[1][i], m_(t.p[0][i], t.p[0][i]))));
            t.p[3][i] = sqrt(fabs(s_(t.p[3][i], m_(t.p[2][i], t.p[2][i]))));
            t.p[5][i] = sqrt(fabs(s_(t.p[5][i], m_(t.p[4][i], t.p[4][i]))));
        }
    }
}

int blocks_n(long long n) { return (int)std::min<long long>((n + 255) / 256, 148 * 16); }

}  // namespace

int launch_stats_update(const Grid3 &g, const StatsIn &in, double *const v[9], double *const t[6], double dt,
                        double ovw, double otw, int avg_type, int vel, int thermo, cudaStream_t st) {
    const long long n = g.n();
    StatsOut vo{}, to{};
    for (int k = 0; k < 9; k++) vo.p[k] = v[k];
    for (int k = 0; k < 6; k++) to.p[k] = t[k];
    stats_accumulate_kernel<<<blocks_n(n), 256, 0, st>>>(n, in, vo, to, dt, ovw, ovw + dt, otw, otw + dt, vel, thermo);
    MC3D_CUDA_TRY(cudaGetLastError());
    if (avg_type == MC3D_AVG_XI1 || avg_type == MC3D_AVG_XI3) {
        const int dir = avg_type == MC3D_AVG_XI1 ? 0 : 2;
        const long long nlines = dir == 0 ? (long long)g.Ny * g.Nz : (long long)g.Nx * g.Ny;
        if (vel) {
            stats_line_mean_kernel<<<blocks_n(nlines * 9), 256, 0, st>>>(g, dir, vo, 9);
            MC3D_CUDA_TRY(cudaGetLastError());
        }
        if (thermo) {
            stats_line_mean_kernel<<<blocks_n(nlines * 6), 256, 0, st>>>(g, dir, to, 6);
            MC3D_CUDA_TRY(cudaGetLastError());
        }
    }
    stats_finish_kernel<<<blocks_n(n), 256, 0, st>>>(n, vo, to, vel, thermo);
    MC3D_CUDA_TRY(cudaGetLastError());
    return MC3D_OK;
}

}  // namespace mc3d
