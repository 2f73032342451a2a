// Constants and helpers shared by the pointwise kernels (pointwise.cu, dsm.cu).
#pragma once
#include "mc3d_internal.h"

namespace mc3d {

constexpr double GAMMA = 1.4;        // src/IdealGas.hpp:38-46
constexpr double PR = 0.7;
constexpr double R_GAS = (1.0 / 1.4) / 1.0 / 1.0;
constexpr double CP = R_GAS * GAMMA / (GAMMA - 1.0);

inline int grid_for(long long n, int block) {
    long long g = (n + block - 1) / block;
    int sms = 148;
    long long cap = (long long)sms * 16;
    if (g > cap) g = cap;
    if (g < 1) g = 1;
    return (int)g;
}

// kernel-argument bundles of five field pointers
struct Q5d {
    double *p[5];
};
struct Q5c {
    const double *p[5];
};
template <typename R>
struct P5w {
    R *p[5];
};

template <typename R>
struct P5c {
    const R *p[5];
};

template <typename R>
struct DerivPtrs12c {
    const R *p[12];
};
struct CoarseOut {
    double *p[14];
};
struct CoarseIn {
    const double *p[14];
};
struct GradIn {
    const double *p[12];
};

template <typename R>
__device__ __forceinline__ R met(const Metrics<R> &m, int c, long long i) {
    return m.constant ? m.c[c] : m.m[c][i];
}

// is linear index i on one of the faces in mask (bit f: 0 X0, 1 X1, 2 Y0, 3 Y1, 4 Z0, 5 Z1)
__device__ __forceinline__ bool on_faces(const Grid3 &g, long long i, int mask) {
    const long long ix = i % g.Nx, r = i / g.Nx, iy = r % g.Ny, iz = r / g.Ny;
    return ((mask & 1) && ix == 0) || ((mask & 2) && ix == g.Nx - 1) || ((mask & 4) && iy == 0) ||
           ((mask & 8) && iy == g.Ny - 1) || ((mask & 16) && iz == 0) || ((mask & 32) && iz == g.Nz - 1);
}

}  // namespace mc3d
