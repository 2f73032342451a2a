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

}  // namespace mc3d
