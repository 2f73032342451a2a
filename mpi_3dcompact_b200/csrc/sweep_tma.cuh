// Line solves staged by the Tensor Memory Accelerator.
//
// x lines: the tile of a CTA, 32 consecutive x-lines of N values, is one contiguous
// block of global memory. One thread brings it into shared memory as N/32
// boxes of 32 x-values by 32 lines (cp.async.bulk.tensor, completion counted
// on an mbarrier), stored with the 128-byte swizzle: within each 1024-byte
// group of 8 box rows the 16-byte chunk index is XORed with the row index.
// Lane l owns line l, so it reads its rows four at a time (one 16-byte
// shared load per four rows, the 8 lanes of each load phase hitting 8
// different chunks). After the solve the lanes write their rows back into the
// same swizzled tile and one thread stores the boxes (TMA store, clipped at
// the grid's last line). Compared with the register kernel's x path this
// replaces one asynchronous copy per element and the transposed tile with a
// few bulk-copy instructions per CTA.
//
// y and z lines: the tile's 32 lines are 32 consecutive points of the x index
// (y lines) or of the flattened x-y index (z lines); one box of 32 points by
// the N rows of the lines (a {32, N, 1} box of the 3-D field for y, a {32, N}
// box of the [Nz][Nx*Ny] view for z) lands as N rows of 128 bytes with the
// same swizzle, so the 32 lanes reading one row hit 32 banks. The epilogue
// computes the caller's operation (operands the operation reads still come
// from global memory, a block of rows ahead) into the tile, and one thread
// stores the box.
#pragma once
#include <cuda.h>

#include "sweep_reg.cuh"

namespace mc3d {

constexpr int TMA_MAXF = 8;   // fields per launch
constexpr int TMA_BOX = 32;   // box edge: 32 x-values (128 bytes, the swizzle span) by 32 lines

struct TmaMaps {
    CUtensorMap in[TMA_MAXF];
    CUtensorMap out[TMA_MAXF];
};

// CTAs whose tile load did not complete within the wait limit
__device__ int g_tma_wait_timeouts;

__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

// byte offset of (line l, x) in the swizzled tile
__device__ __forceinline__ unsigned swz_off(int l, int x) {
    const int bx = x >> 5, c = (x >> 2) & 7;
    return (unsigned)(bx * 4096 + l * 128 + ((c ^ (l & 7)) << 4) + ((x & 3) << 2));
}

__device__ __forceinline__ float4 lds4(const unsigned char *tile, unsigned off) {
    return *reinterpret_cast<const float4 *>(tile + off);
}

template <int KIND, int H, int L, int E>
__global__ void __launch_bounds__(512) sweep_tma_x_kernel(Grid3 g, LineOpDev<float> op,
                                                          const __grid_constant__ TmaMaps maps, int pass_y,
                                                          int pass_z) {
    using R = float;
    constexpr bool PER = (KIND % 2) == 0;
    constexpr int NV = L + 2 * H;
    constexpr int HC = (H + 3) / 4;   // 16-byte halo chunks on each side
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    __shared__ __align__(8) unsigned long long bar;
    const unsigned base = smem_u32(smem_raw);
    unsigned char *tile = smem_raw + ((1024u - (base & 1023u)) & 1023u);   // boxes need 1024-byte alignment
    const int N = op.N, nbox = N / TMA_BOX;
    R *sh = reinterpret_cast<R *>(tile + nbox * 4096);
    const int S = blockDim.x >> 5;
    const int lane = threadIdx.x & 31, seg = threadIdx.x >> 5, a = seg * L;
    const int f = blockIdx.y;
    const int line0 = blockIdx.x * W;
    const unsigned bar_a = smem_u32(&bar);

    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar_a) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar_a), "r"(nbox * 4096)
                     : "memory");
        const unsigned long long tm = reinterpret_cast<unsigned long long>(&maps.in[f]);
        for (int bx = 0; bx < nbox; bx++)
            asm volatile(
                "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
                "[%4];" ::"r"(smem_u32(tile + bx * 4096)),
                "l"(tm), "r"(bx * TMA_BOX), "r"(line0), "r"(bar_a)
                : "memory");
    }
    __syncthreads();   // the barrier is initialised before anyone waits on it
    unsigned done = 0;
    for (int it = 0; it < (1 << 22) && !done; it++)
        asm volatile(
            "{\n.reg .pred p;\nmbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0;\nselp.u32 %0, 1, 0, p;\n}"
            : "=r"(done)
            : "r"(bar_a)
            : "memory");
    // the whole CTA gives up together when the copy did not arrive in time
    if (!__syncthreads_and(done != 0)) {
        if (threadIdx.x == 0) atomicAdd(&g_tma_wait_timeouts, 1);
        return;
    }

    const TileGeom t = tile_geom<0>(g, blockIdx.x, lane);
    const bool pass = (pass_y && (t.j == 0 || t.j == g.Ny - 1)) || (pass_z && (t.k == 0 || t.k == g.Nz - 1));
    const bool work = t.active && !pass;

    // ---- rows a-H .. a+L+H-1 of this lane's line (periodic wrap / zero) ----
    R v[NV];
#pragma unroll
    for (int q = 0; q < L / 4; q++) {
        const float4 w = lds4(tile, swz_off(lane, a + 4 * q));
        v[H + 4 * q + 0] = w.x;
        v[H + 4 * q + 1] = w.y;
        v[H + 4 * q + 2] = w.z;
        v[H + 4 * q + 3] = w.w;
    }
#pragma unroll
    for (int hc = 0; hc < HC; hc++) {
        int n = a - 4 * (hc + 1);
        bool in = true;
        if (n < 0) {
            n += N;
            in = PER;
        }
        const float4 w = in ? lds4(tile, swz_off(lane, n)) : make_float4(0.f, 0.f, 0.f, 0.f);
        const R e[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int k = H - 4 * (hc + 1) + j;
            if (k >= 0) v[k] = e[j];
        }
        int m = a + L + 4 * hc;
        bool in2 = true;
        if (m >= N) {
            m -= N;
            in2 = PER;
        }
        const float4 w2 = in2 ? lds4(tile, swz_off(lane, m)) : make_float4(0.f, 0.f, 0.f, 0.f);
        const R e2[4] = {w2.x, w2.y, w2.z, w2.w};
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int k = H + L + 4 * hc + j;
            if (k < NV) v[k] = e2[j];
        }
    }

    R y[L];
    reg_solve<R, KIND, H, L>(op, v, y, work, lane, seg, S, a, sh);

    // ---- solution rows back into the tile (pass-through lines keep their input), then the TMA store ----
    if (work) {
#pragma unroll
        for (int q = 0; q < L / 4; q++) {
            float4 w;
            w.x = E == EPI_STORE_NEG ? -y[4 * q + 0] : y[4 * q + 0];
            w.y = E == EPI_STORE_NEG ? -y[4 * q + 1] : y[4 * q + 1];
            w.z = E == EPI_STORE_NEG ? -y[4 * q + 2] : y[4 * q + 2];
            w.w = E == EPI_STORE_NEG ? -y[4 * q + 3] : y[4 * q + 3];
            *reinterpret_cast<float4 *>(tile + swz_off(lane, a + 4 * q)) = w;
        }
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned long long tm = reinterpret_cast<unsigned long long>(&maps.out[f]);
        for (int bx = 0; bx < nbox; bx++)
            asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.tile.bulk_group [%0, {%1, %2}], [%3];" ::"l"(tm),
                         "r"(bx * TMA_BOX), "r"(line0), "r"(smem_u32(tile + bx * 4096))
                         : "memory");
        asm volatile("cp.async.bulk.commit_group;" ::: "memory");
        asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
    }
}

// byte offset of row n, lane l in a strided-line tile
__device__ __forceinline__ unsigned swz_row(int n, int l) {
    return (unsigned)(n * 128 + ((((l >> 2) ^ (n & 7))) << 4) + ((l & 3) << 2));
}

// the caller's operation on this lane's L solution rows, written into the
// tile (row a + r); old output, partial RHS and J come from global memory,
// the next block's ahead of this block's shared stores
template <int E, int L>
__device__ __forceinline__ void tma_tile_rows(const SweepBatch<float> &b, const RhsFinalArgs<float> &rf, int f,
                                              int off0, int stride, const float (&y)[L], unsigned char *tile,
                                              int a, int lane) {
    using R = float;
    constexpr int NB = L / UB;
    constexpr bool RD_OLD = E == EPI_SUB || E == EPI_RHS_FINAL;
    constexpr bool RD_AUX = E == EPI_RHS_FINAL;
    const R dt = (E == EPI_RHS_FINAL) ? (R)(*rf.dt) : R(0);
    const bool mom = (E == EPI_RHS_FINAL) && rf.quirk && b.eq[f] >= 1 && b.eq[f] <= 3;
    const bool rd_old = E == EPI_SUB || mom;
    const R *o = b.out[f];
    const R *ax = b.aux[f];
    const R *jp = rf.J;
    R old[2][UB], aux[2][UB], jj[2][UB];
    auto fetch = [&](int blk, int slot) {
#pragma unroll
        for (int u = 0; u < UB; u++) {
            const int off = off0 + (blk * UB + u) * stride;
            if (RD_OLD) old[slot][u] = rd_old ? o[off] : R(0);
            if (RD_AUX) {
                aux[slot][u] = ax[off];
                jj[slot][u] = jp ? jp[off] : rf.Jc;
            }
        }
    };
    if (RD_OLD || RD_AUX) fetch(0, 0);
#pragma unroll
    for (int blk = 0; blk < NB; blk++) {
        const int cur = blk & 1;
        if ((RD_OLD || RD_AUX) && blk + 1 < NB) fetch(blk + 1, cur ^ 1);
#pragma unroll
        for (int u = 0; u < UB; u++) {
            const int r = blk * UB + u;
            const R v = y[r];
            R w = v;
            if (E == EPI_STORE_NEG) w = -v;
            if (E == EPI_SUB) w = old[cur][u] - v;
            if (E == EPI_RHS_FINAL) {
                // solveContinuity .. solveEnergy (src/CurvilinearCSolver_Core.cpp:790-947)
                const R tt = aux[cur][u] - v;
                const R dtJ = dt * jj[cur][u];
                w = mom ? (old[cur][u] + tt) * dtJ : tt * dtJ;
            }
            *reinterpret_cast<R *>(tile + swz_row(a + r, lane)) = w;
        }
    }
}

template <int DIR, int KIND, int H, int L, int E>
__global__ void __launch_bounds__(512) sweep_tma_yz_kernel(Grid3 g, LineOpDev<float> op, SweepBatch<float> b,
                                                           RhsFinalArgs<float> rf, const __grid_constant__ TmaMaps maps,
                                                           int pass_x, int pass_y, int pass_z) {
    using R = float;
    constexpr bool PER = (KIND % 2) == 0;
    constexpr int NV = L + 2 * H;
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    __shared__ __align__(8) unsigned long long bar;
    const unsigned base = smem_u32(smem_raw);
    unsigned char *tile = smem_raw + ((1024u - (base & 1023u)) & 1023u);
    const int N = op.N;
    R *sh = reinterpret_cast<R *>(tile + N * 128);
    const int S = blockDim.x >> 5;
    const int lane = threadIdx.x & 31, seg = threadIdx.x >> 5, a = seg * L;
    const int f = blockIdx.y;
    int c0, c2 = 0;
    if (DIR == 1) {
        const int tx = (g.Nx + W - 1) / W;
        c0 = (blockIdx.x % tx) * W;
        c2 = blockIdx.x / tx;
    } else {
        c0 = blockIdx.x * W;
    }
    const unsigned bar_a = smem_u32(&bar);

    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar_a) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar_a), "r"(N * 128) : "memory");
        const unsigned long long tm = reinterpret_cast<unsigned long long>(&maps.in[f]);
        if (DIR == 1)
            asm volatile(
                "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, "
                "%4}], [%5];" ::"r"(smem_u32(tile)),
                "l"(tm), "r"(c0), "r"(0), "r"(c2), "r"(bar_a)
                : "memory");
        else
            asm volatile(
                "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
                "[%4];" ::"r"(smem_u32(tile)),
                "l"(tm), "r"(c0), "r"(0), "r"(bar_a)
                : "memory");
    }
    __syncthreads();
    unsigned done = 0;
    for (int it = 0; it < (1 << 22) && !done; it++)
        asm volatile(
            "{\n.reg .pred p;\nmbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0;\nselp.u32 %0, 1, 0, p;\n}"
            : "=r"(done)
            : "r"(bar_a)
            : "memory");
    if (!__syncthreads_and(done != 0)) {
        if (threadIdx.x == 0) atomicAdd(&g_tma_wait_timeouts, 1);
        return;
    }

    const TileGeom t = tile_geom<DIR>(g, blockIdx.x, lane);
    bool pass;
    if (DIR == 1) pass = (pass_x && (t.i == 0 || t.i == g.Nx - 1)) || (pass_z && (t.k == 0 || t.k == g.Nz - 1));
    else pass = (pass_y && (t.j == 0 || t.j == g.Ny - 1)) || (pass_x && (t.i == 0 || t.i == g.Nx - 1));
    const bool work = t.active && !pass;

    // ---- rows a-H .. a+L+H-1 of this lane's line (periodic wrap / zero) ----
    R v[NV];
#pragma unroll
    for (int k = 0; k < NV; k++) {
        int n = a - H + k;
        bool in = true;
        if (k < H && n < 0) {
            n += N;
            in = PER;
        }
        if (k >= H + L && n >= N) {
            n -= N;
            in = PER;
        }
        v[k] = in ? *reinterpret_cast<const R *>(tile + swz_row(n, lane)) : R(0);
    }

    R y[L];
    reg_solve<R, KIND, H, L>(op, v, y, work, lane, seg, S, a, sh);

    // ---- the operation's values into the tile (pass-through lines keep their input), then the TMA store ----
    if (work) tma_tile_rows<E, L>(b, rf, f, (int)t.base + a * (int)t.stride, (int)t.stride, y, tile, a, lane);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned long long tm = reinterpret_cast<unsigned long long>(&maps.out[f]);
        if (DIR == 1)
            asm volatile("cp.async.bulk.tensor.3d.global.shared::cta.tile.bulk_group [%0, {%1, %2, %3}], [%4];" ::"l"(tm),
                         "r"(c0), "r"(0), "r"(c2), "r"(smem_u32(tile))
                         : "memory");
        else
            asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.tile.bulk_group [%0, {%1, %2}], [%3];" ::"l"(tm),
                         "r"(c0), "r"(0), "r"(smem_u32(tile))
                         : "memory");
        asm volatile("cp.async.bulk.commit_group;" ::: "memory");
        asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
    }
}

}  // namespace mc3d
