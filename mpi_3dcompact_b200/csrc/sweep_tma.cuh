// x-line solves staged by the Tensor Memory Accelerator.
//
// The tile of a CTA, 32 consecutive x-lines of N values, is one contiguous
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
#pragma once
#include <cuda.h>

#include "sweep_reg.cuh"

namespace mc3d {

constexpr int TMA_MAXF = 8;   // fields per launch
constexpr int TMA_BOX = 32;   // box edge: 32 x-values (128 bytes, the swizzle span) by 32 lines

struct TmaMapsX {
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
                                                          const __grid_constant__ TmaMapsX maps, int pass_y,
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

}  // namespace mc3d
