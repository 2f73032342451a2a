// Line solves staged by the Tensor Memory Accelerator.
//
// x lines: the tile of a CTA, 32 consecutive x-lines of N values, is one contiguous
// block of global memory. One thread brings it into shared memory as N/32
// boxes of 32 x-values by 32 lines (cp.async.bulk.tensor, completion counted
// on an mbarrier), stored with the 128-byte swizzle: within each 1024-byte
// group of 8 box rows the 16-byte chunk index is XORed with the row index.
// Lane l owns line l, so it reads its rows four at a time (one 16-byte
// shared load per four rows, the 8 lanes of each load phase hitting 8
// different chunks). After the solve the lanes write their rows into a second
// swizzled tile and one thread stores its boxes (TMA store, clipped at the
// grid's last line). CTAs are persistent: the next tile's load runs during
// the solve. Compared with the register kernel's x path this replaces one
// asynchronous copy per element and the transposed tile with a few
// bulk-copy instructions per CTA.
//
// y and z lines: the tile's 32 lines are 32 consecutive points of the x index
// (y lines) or of the flattened x-y index (z lines); boxes of 32 points by up
// to 256 rows of the lines ({32, rows, 1} boxes of the 3-D field for y,
// {32, rows} boxes of the [Nz][Nx*Ny] view for z; lines of 512 or 1024 take
// two or four) land as N rows of 128 bytes with the same swizzle, so the 32
// lanes reading one row hit 32 banks. Plain and
// negated stores run persistent CTAs that load the next tile during the
// solve and store directly (one 128-byte row per warp instruction); the
// operations that read operands (accumulate, k2 assembly) run one CTA per
// tile, bring their operand tiles in by TMA during the solve and store by TMA.
#pragma once
#include <cuda.h>

#include "sweep_reg.cuh"

namespace mc3d {

constexpr int TMA_MAXF = 8;   // fields per launch
constexpr int TMA_BOX = 32;   // box edge: 32 x-values (128 bytes, the swizzle span) by 32 lines
constexpr int TMA_ROWS = 256; // rows per box of a y/z tile (the largest box extent); longer lines take several

struct TmaMaps {
    CUtensorMap in[TMA_MAXF];
    CUtensorMap out[TMA_MAXF];
    CUtensorMap aux[TMA_MAXF];   // partial RHS of the k2 assembly
};

// CTAs whose tile load did not complete within the wait limit
__device__ int g_tma_wait_timeouts;

__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

// byte offset of (line l, x) in the swizzled tile: box x/32, row l, chunk
// ((x/4) % 8) ^ (l % 8); written as a lane constant XORed with the chunk so
// that one register per lane serves every row
__device__ __forceinline__ unsigned swz_off(int l, int x) {
    const unsigned lane_part = (unsigned)(l * 128 + ((l & 7) << 4));
    return (unsigned)((x >> 5) * 4096) + (lane_part ^ (unsigned)(((x >> 2) & 7) << 4)) + (unsigned)((x & 3) << 2);
}

// A tile that the lanes have read with ordinary shared-memory loads (the
// generic proxy) is refilled by a TMA load (the async proxy). The CTA barrier
// alone orders the two only within the generic proxy: without a proxy fence
// the bulk copy may land in the tile before every lane's earlier loads have
// read it, and those lanes then solve with rows of the next tile. Each thread
// fences its own reads, then the barrier hands that ordering to the thread
// that issues the copy (the write-after-read form of the proxy rule of the
// PTX memory model; the read-after-write form is the fence before each TMA
// store).
__device__ __forceinline__ void tile_reads_done() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ float4 lds4(const unsigned char *tile, unsigned off) {
    return *reinterpret_cast<const float4 *>(tile + off);
}

// byte offset of row n, lane l in a strided-line tile: chunk (l/4) ^ (n % 8),
// as a lane constant XORed with the row's chunk mask
__device__ __forceinline__ unsigned swz_row(int n, int l) {
    const unsigned lane_part = (unsigned)(((l >> 2) << 4) | ((l & 3) << 2));
    return (unsigned)(n * 128) + (lane_part ^ (unsigned)((n & 7) << 4));
}

// y/z lines, operations that read operands (accumulate: the previous output;
// k2 assembly: the partial RHS and, for momentum with the carry-over, the
// previous k2): one CTA per tile. The input tile arrives by TMA; once every
// lane holds its rows the same buffer receives the first operand tile while
// the lanes solve, then (k2 assembly of momentum) the second; the results go
// back into the buffer and leave by one TMA store.
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
    // the tile's boxes of `m` (thread 0)
    auto load = [&](const CUtensorMap *m) {
        const unsigned long long tm = reinterpret_cast<unsigned long long>(m);
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar_a), "r"(N * 128) : "memory");
        for (int r0 = 0; r0 < N; r0 += TMA_ROWS) {
            if (DIR == 1)
                asm volatile(
                    "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, "
                    "%3, %4}], [%5];" ::"r"(smem_u32(tile + r0 * 128)),
                    "l"(tm), "r"(c0), "r"(r0), "r"(c2), "r"(bar_a)
                    : "memory");
            else
                asm volatile(
                    "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, "
                    "%3}], [%4];" ::"r"(smem_u32(tile + r0 * 128)),
                    "l"(tm), "r"(c0), "r"(r0), "r"(bar_a)
                    : "memory");
        }
    };
    // bounded wait for the phase of the given parity; the CTA decides together
    auto wait = [&](unsigned parity) -> bool {
        unsigned done = 0;
        for (int it = 0; it < (1 << 22) && !done; it++)
            asm volatile(
                "{\n.reg .pred p;\nmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\nselp.u32 %0, 1, 0, p;\n}"
                : "=r"(done)
                : "r"(bar_a), "r"(parity)
                : "memory");
        if (__syncthreads_and(done != 0)) return true;
        if (threadIdx.x == 0) atomicAdd(&g_tma_wait_timeouts, 1);
        return false;
    };
    auto at = [&](int r) -> R & { return *reinterpret_cast<R *>(tile + swz_row(a + r, lane)); };

    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar_a) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        load(&maps.in[f]);
    }
    __syncthreads();
    if (!wait(0)) return;

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
    tile_reads_done();
    __syncthreads();   // every lane holds its rows: the tile takes the first operand
    const bool mom = E == EPI_RHS_FINAL && rf.quirk && b.eq[f] >= 1 && b.eq[f] <= 3;
    if (threadIdx.x == 0) load(E == EPI_SUB ? &maps.out[f] : &maps.aux[f]);

    R y[L];
    reg_solve<R, KIND, H, L>(op, v, y, work, lane, seg, S, a, sh);

    if (!wait(1)) return;
    // accumulate: old - v; k2 assembly: tt = aux - v (src/CurvilinearCSolver_Core.cpp:790-947)
#pragma unroll
    for (int r = 0; r < L; r++) y[r] = at(r) - y[r];
    if (E == EPI_RHS_FINAL) {
        if (mom) {
            tile_reads_done();
            __syncthreads();   // every lane has read the partial RHS
            if (threadIdx.x == 0) load(&maps.out[f]);
            if (!wait(0)) return;
#pragma unroll
            for (int r = 0; r < L; r++) y[r] = at(r) + y[r];
        }
        const R dt = (R)(*rf.dt);
        if (!rf.J) {
            const R dtJ = dt * rf.Jc;
#pragma unroll
            for (int r = 0; r < L; r++) y[r] = y[r] * dtJ;
        } else if (t.active) {
            const int off0 = (int)t.base + a * (int)t.stride, stride = (int)t.stride;
#pragma unroll
            for (int r = 0; r < L; r++) y[r] = y[r] * (dt * rf.J[off0 + r * stride]);
        }
    }
    __syncthreads();   // every lane has read its operands
#pragma unroll
    for (int r = 0; r < L; r++) at(r) = y[r];
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned long long tm = reinterpret_cast<unsigned long long>(&maps.out[f]);
        for (int r0 = 0; r0 < N; r0 += TMA_ROWS) {
            if (DIR == 1)
                asm volatile("cp.async.bulk.tensor.3d.global.shared::cta.tile.bulk_group [%0, {%1, %2, %3}], [%4];" ::
                                 "l"(tm),
                             "r"(c0), "r"(r0), "r"(c2), "r"(smem_u32(tile + r0 * 128))
                             : "memory");
            else
                asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.tile.bulk_group [%0, {%1, %2}], [%3];" ::"l"(tm),
                             "r"(c0), "r"(r0), "r"(smem_u32(tile + r0 * 128))
                             : "memory");
        }
        asm volatile("cp.async.bulk.commit_group;" ::: "memory");
        asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
    }
}

// Persistent form of the y/z kernel (plain and negated stores): each CTA
// walks the (field, tile) items gridDim.x apart; as soon as the lanes hold the
// current tile in registers, one thread starts the TMA load of the next item
// into the same buffer, so the load overlaps the solve and the epilogue
// (direct global stores, 128 bytes per warp and row).
template <int DIR, int KIND, int H, int L, int E>
__global__ void __launch_bounds__(512) sweep_tma_yz_persist_kernel(Grid3 g, LineOpDev<float> op, SweepBatch<float> b,
                                                                   RhsFinalArgs<float> rf,
                                                                   const __grid_constant__ TmaMaps maps, int pass_x,
                                                                   int pass_y, int pass_z) {
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
    const int ntiles = tile_count<DIR>(g);
    const int nitems = ntiles * b.nf;
    const int tx = (g.Nx + W - 1) / W;
    const unsigned bar_a = smem_u32(&bar);
    // TMA load of item w into the tile
    auto issue = [&](int w) {
        const int f = w / ntiles, tl = w - f * ntiles;
        const unsigned long long tm = reinterpret_cast<unsigned long long>(&maps.in[f]);
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar_a), "r"(N * 128) : "memory");
        for (int r0 = 0; r0 < N; r0 += TMA_ROWS) {
            if (DIR == 1)
                asm volatile(
                    "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, "
                    "%3, %4}], [%5];" ::"r"(smem_u32(tile + r0 * 128)),
                    "l"(tm), "r"((tl % tx) * W), "r"(r0), "r"(tl / tx), "r"(bar_a)
                    : "memory");
            else
                asm volatile(
                    "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, "
                    "%3}], [%4];" ::"r"(smem_u32(tile + r0 * 128)),
                    "l"(tm), "r"(tl * W), "r"(r0), "r"(bar_a)
                    : "memory");
        }
    };
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar_a) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        if ((int)blockIdx.x < nitems) issue(blockIdx.x);
    }
    __syncthreads();
    unsigned phase = 0;
    for (int w = blockIdx.x; w < nitems; w += gridDim.x) {
        unsigned done = 0;
        for (int it = 0; it < (1 << 22) && !done; it++)
            asm volatile(
                "{\n.reg .pred p;\nmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\nselp.u32 %0, 1, 0, p;\n}"
                : "=r"(done)
                : "r"(bar_a), "r"(phase)
                : "memory");
        if (!__syncthreads_and(done != 0)) {
            if (threadIdx.x == 0) atomicAdd(&g_tma_wait_timeouts, 1);
            return;
        }
        phase ^= 1u;
        const int f = w / ntiles, tl = w - f * ntiles;
        const TileGeom t = tile_geom<DIR>(g, tl, lane);
        bool pass = false;   // (no pass-through lines with the derivatives, H <= 3)
        if (H > 3) {
            if (DIR == 1) pass = (pass_x && (t.i == 0 || t.i == g.Nx - 1)) || (pass_z && (t.k == 0 || t.k == g.Nz - 1));
            else pass = (pass_y && (t.j == 0 || t.j == g.Ny - 1)) || (pass_x && (t.i == 0 || t.i == g.Nx - 1));
        }
        const bool work = t.active && !pass;
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
        // the buffer takes the next item at the barrier that ends pass 1
        auto refill = [&](int ph) {
            if (ph == 0) tile_reads_done();
            else if (threadIdx.x == 0 && w + (int)gridDim.x < nitems) issue(w + gridDim.x);
        };
        R y[L];
        reg_solve<R, KIND, H, L>(op, v, y, work, lane, seg, S, a, sh, refill);
        if (t.active) reg_store_rows<R, E, L>(b, rf, f, (int)t.base + a * (int)t.stride, (int)t.stride, y);
    }
}

// Persistent form of the x kernel: each CTA walks the (field, tile) items
// gridDim.x apart with two tiles, one receiving the next item's TMA load
// while the lanes solve the current one, the other holding the solution rows
// for the TMA store (whose shared-memory reads are awaited before the tile is
// written again).
template <int KIND, int H, int L, int E>
__global__ void __launch_bounds__(512) sweep_tma_x_persist_kernel(Grid3 g, LineOpDev<float> op,
                                                                  const __grid_constant__ TmaMaps maps, int nf,
                                                                  int pass_y, int pass_z) {
    using R = float;
    constexpr bool PER = (KIND % 2) == 0;
    constexpr int NV = L + 2 * H;
    constexpr int HC = (H + 3) / 4;
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    __shared__ __align__(8) unsigned long long bar;
    const unsigned base = smem_u32(smem_raw);
    unsigned char *tin = smem_raw + ((1024u - (base & 1023u)) & 1023u);
    const int N = op.N, nbox = N / TMA_BOX;
    unsigned char *tout = tin + nbox * 4096;
    R *sh = reinterpret_cast<R *>(tout + nbox * 4096);
    const int S = blockDim.x >> 5;
    const int lane = threadIdx.x & 31, seg = threadIdx.x >> 5, a = seg * L;
    const int ntiles = tile_count<0>(g);
    const int nitems = ntiles * nf;
    const unsigned bar_a = smem_u32(&bar);
    auto issue = [&](int w) {
        const int f = w / ntiles, tl = w - f * ntiles;
        const unsigned long long tm = reinterpret_cast<unsigned long long>(&maps.in[f]);
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar_a), "r"(nbox * 4096)
                     : "memory");
        for (int bx = 0; bx < nbox; bx++)
            asm volatile(
                "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
                "[%4];" ::"r"(smem_u32(tin + bx * 4096)),
                "l"(tm), "r"(bx * TMA_BOX), "r"(tl * W), "r"(bar_a)
                : "memory");
    };
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar_a) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        if ((int)blockIdx.x < nitems) issue(blockIdx.x);
    }
    __syncthreads();
    unsigned phase = 0;
    for (int w = blockIdx.x; w < nitems; w += gridDim.x) {
        unsigned done = 0;
        for (int it = 0; it < (1 << 22) && !done; it++)
            asm volatile(
                "{\n.reg .pred p;\nmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\nselp.u32 %0, 1, 0, p;\n}"
                : "=r"(done)
                : "r"(bar_a), "r"(phase)
                : "memory");
        if (!__syncthreads_and(done != 0)) {
            if (threadIdx.x == 0) {
                atomicAdd(&g_tma_wait_timeouts, 1);
                asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
            }
            return;
        }
        phase ^= 1u;
        const int f = w / ntiles, tl = w - f * ntiles;
        const TileGeom t = tile_geom<0>(g, tl, lane);
        const bool pass = (pass_y && (t.j == 0 || t.j == g.Ny - 1)) || (pass_z && (t.k == 0 || t.k == g.Nz - 1));
        const bool work = t.active && !pass;
        R v[NV];
#pragma unroll
        for (int q = 0; q < L / 4; q++) {
            const float4 x4 = lds4(tin, swz_off(lane, a + 4 * q));
            v[H + 4 * q + 0] = x4.x;
            v[H + 4 * q + 1] = x4.y;
            v[H + 4 * q + 2] = x4.z;
            v[H + 4 * q + 3] = x4.w;
        }
#pragma unroll
        for (int hc = 0; hc < HC; hc++) {
            int n = a - 4 * (hc + 1);
            bool in = true;
            if (n < 0) {
                n += N;
                in = PER;
            }
            const float4 x4 = in ? lds4(tin, swz_off(lane, n)) : make_float4(0.f, 0.f, 0.f, 0.f);
            const R e[4] = {x4.x, x4.y, x4.z, x4.w};
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
            const float4 x5 = in2 ? lds4(tin, swz_off(lane, m)) : make_float4(0.f, 0.f, 0.f, 0.f);
            const R e2[4] = {x5.x, x5.y, x5.z, x5.w};
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const int k = H + L + 4 * hc + j;
                if (k < NV) v[k] = e2[j];
            }
        }
        // the input tile takes the next item at the barrier that ends pass 1;
        // the output tile is written after the solve's second barrier, which
        // the issuing thread reaches only once the previous store has read it
        auto refill = [&](int ph) {
            if (ph == 0) {
                tile_reads_done();
            } else if (threadIdx.x == 0) {
                if (w + (int)gridDim.x < nitems) issue(w + gridDim.x);
                asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");   // previous store has read tout
            }
        };
        R y[L];
        // (negated store: the solve itself yields -y)
        static_assert(E != EPI_STORE_NEG || H <= 3, "negated x stores are derivative sweeps");
        reg_solve<R, KIND, H, L, E == EPI_STORE_NEG>(op, v, y, work, lane, seg, S, a, sh, refill);
        // (pass-through lines: y holds their input)
        if (t.active) {
#pragma unroll
            for (int q = 0; q < L / 4; q++) {
                float4 o4;
                o4.x = y[4 * q + 0];
                o4.y = y[4 * q + 1];
                o4.z = y[4 * q + 2];
                o4.w = y[4 * q + 3];
                *reinterpret_cast<float4 *>(tout + swz_off(lane, a + 4 * q)) = o4;
            }
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (threadIdx.x == 0) {
            const unsigned long long tm = reinterpret_cast<unsigned long long>(&maps.out[f]);
            for (int bx = 0; bx < nbox; bx++)
                asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.tile.bulk_group [%0, {%1, %2}], [%3];" ::"l"(tm),
                             "r"(bx * TMA_BOX), "r"(tl * W), "r"(smem_u32(tout + bx * 4096))
                             : "memory");
            asm volatile("cp.async.bulk.commit_group;" ::: "memory");
        }
    }
    if (threadIdx.x == 0) asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
}

}  // namespace mc3d
