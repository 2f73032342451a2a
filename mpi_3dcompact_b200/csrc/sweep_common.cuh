// Device helpers shared by the line-solve kernels (sweeps.cu, sweeps_reg_*.cu).
#pragma once
#include <cstdint>

#include "mc3d_internal.h"

namespace mc3d {


constexpr int W = 32;       // lines per tile
constexpr int SP = W + 1;   // shared-memory row pitch (elements)

template <typename R>
__device__ __forceinline__ R ldc(const R *p) {
    return __ldg(p);
}

// Asynchronous global->shared element copy (cp.async, L1-allocating), so a
// whole tile is in flight at once without staging through registers.
template <typename R>
__device__ __forceinline__ void cp_async_elem(R *dst, const R *src) {
    unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    if (sizeof(R) == 4)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(src) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
    asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
}

// Tile geometry: line `lane` of tile `tile` starts at base(lane) and advances by
// `stride`; for DIR 0 the tile's lines are one contiguous block of len*N values.
struct TileGeom {
    long long base;   // element 0 of this lane's line
    long long stride;
    bool active;
    int j, k, i;      // grid coordinates of the line (the running one is unused)
};

template <int DIR>
__device__ __forceinline__ TileGeom tile_geom(const Grid3 &g, int tile, int lane) {
    TileGeom t;
    if (DIR == 0) {
        long long L = (long long)tile * W + lane;
        long long nl = (long long)g.Ny * g.Nz;
        t.active = L < nl;
        t.base = L * g.Nx;
        t.stride = 1;
        t.j = (int)(L % g.Ny);
        t.k = (int)(L / g.Ny);
        t.i = 0;
    } else if (DIR == 1) {
        int tx = (g.Nx + W - 1) / W;
        int k = tile / tx;
        int i = (tile % tx) * W + lane;
        t.active = i < g.Nx;
        t.base = (long long)i + (long long)g.Nx * g.Ny * k;
        t.stride = g.Nx;
        t.i = i;
        t.k = k;
        t.j = 0;
    } else {
        long long L = (long long)tile * W + lane;
        long long nl = (long long)g.Nx * g.Ny;
        t.active = L < nl;
        t.base = L;
        t.stride = (long long)g.Nx * g.Ny;
        t.i = (int)(L % g.Nx);
        t.j = (int)(L / g.Nx);
        t.k = 0;
    }
    return t;
}

template <int DIR>
__host__ __device__ __forceinline__ int tile_count(const Grid3 &g) {
    if (DIR == 0) return (int)(((long long)g.Ny * g.Nz + W - 1) / W);
    if (DIR == 1) return ((g.Nx + W - 1) / W) * g.Nz;
    return (int)(((long long)g.Nx * g.Ny + W - 1) / W);
}

// rows per register block of the line solves
constexpr int UB = 8;

// elements of the segment-chain area of the register-resident solve: the
// local end states of both passes ([2][S][2][W]) and the last two values of
// the last segment ([2][W])
__host__ __device__ constexpr int reg_chain_elems(int S) { return 4 * S * W + 2 * W; }

// shared-memory bytes of the register-resident kernel: chain states and, for
// x lines, the transposed tile
inline size_t reg_smem_bytes(int dir, int N, int S, size_t esize) {
    return ((size_t)reg_chain_elems(S) + (dir == 0 ? (size_t)N * (W + 1) : 0)) * esize;
}

// Register-resident segmented line solve along DIR (sweep_reg.cuh); returns
// MC3D_ERR_CONFIG, without recording an error, for operators it does not cover.
template <int DIR, typename R>
int launch_sweep_reg(const Grid3 &g, const LineOpDev<R> &op, const SweepBatch<R> &b, int epi,
                     const RhsFinalArgs<R> &rf, int px, int py, int pz, cudaStream_t st);

// FP32 x-line solves staged through shared memory by TMA (sweep_tma.cuh,
// sweeps_tma.cu);
// MC3D_ERR_CONFIG, without recording an error, when the case is not covered
// (or MC3D_NO_TMA=1 is set).
int launch_sweep_tma_x(const Grid3 &g, const LineOpDev<float> &op, const SweepBatch<float> &b, int epi, int px,
                       int py, int pz, cudaStream_t st);
// the same for y (dir 1) and z (dir 2) lines
int launch_sweep_tma_yz(int dir, const Grid3 &g, const LineOpDev<float> &op, const SweepBatch<float> &b, int epi,
                        const RhsFinalArgs<float> &rf, int px, int py, int pz, cudaStream_t st);

}  // namespace mc3d
