// Tensor-core (tcgen05) evaluation of the learned closure's network on tiles
// of 128 points, one tile per warpgroup at a time.
//
//   layer 1  D[128 x 64]  = A1[128 x 16] W1'[16 x 64]          (one MMA, K = 16)
//   layer l  D[128 x N_l] = A[128 x 64] W_l'[64 x N_l]         (four MMAs, K = 16 each)
//                         + Ac[128 x 16] B_l'[16 x N_l]        (the bias, one MMA)
// BF16 operands in shared memory, FP32 accumulators in tensor memory (TMEM
// lane = point, column = output). The accumulator of a layer is read back by
// the warpgroup's own threads (tcgen05.ld, thread = point), rounded to BF16
// pairs, put through the GELU in packed BF16 arithmetic in registers and
// written into the operand tile of the next layer, whose MMAs one thread then
// issues; tcgen05.commit on an mbarrier signals their completion. The biases ride on the tensor cores: layer 1's
// input carries two constant-one columns against the rows (b_hi, b_lo) of W1
// (b = b_hi + b_lo to 16 bits), the other layers add Ac B_l with the same two
// columns. Operands use the K-major layout without swizzle: 8-row core
// matrices of 8 rows x 16 bytes, the 16-byte K-chunks 128 bytes apart (LBO),
// 8-row groups 1024 bytes apart for K = 64 and 256 bytes apart for K = 16 (SBO).
//
// Used by the standalone inference and by the closure fused into the SGS pass
// of the time step, both in sgs_mlp.cu, the one file that includes this header
// (it defines the device counter of wait timeouts). Single-GPU code: every
// operand is in this CTA's shared memory; no TMA and no multicast.
#pragma once
#include <cuda_bf16.h>

#include "mlp_common.cuh"

namespace mc3d {

// shared-memory matrix descriptor (tcgen05): start address, leading (K) and
// stride (M/N) byte offsets in 16-byte units, descriptor version 1, no swizzle
__device__ __forceinline__ unsigned long long tc_desc(unsigned saddr, unsigned lbo, unsigned sbo) {
    return (unsigned long long)((saddr & 0x3FFFFu) >> 4) | ((unsigned long long)(lbo >> 4) << 16) |
           ((unsigned long long)(sbo >> 4) << 32) | (1ull << 46);
}
__device__ __forceinline__ void tc_mma(unsigned tmem_d, unsigned long long a, unsigned long long b, unsigned idesc,
                                       unsigned accumulate) {
    asm volatile(
        "{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\n"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
        "l"(a), "l"(b), "r"(idesc), "r"(accumulate)
        : "memory");
}
__device__ __forceinline__ void tc_commit(unsigned mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
                 : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
// shared-memory writes of the generic proxy made visible to the tensor cores
__device__ __forceinline__ void tc_proxy_fence() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
// barrier of the 128 threads of warpgroup wg (named barrier 1 + wg; immediate
// ids, so the kernel reserves only the barriers it uses)
__device__ __forceinline__ void wg_bar(int wg) {
    if (wg == 0) asm volatile("bar.sync 1, 128;" ::: "memory");
    else if (wg == 1) asm volatile("bar.sync 2, 128;" ::: "memory");
    else if (wg == 2) asm volatile("bar.sync 3, 128;" ::: "memory");
    else asm volatile("bar.sync 4, 128;" ::: "memory");
}

__device__ __forceinline__ void tc_ld32(unsigned taddr, unsigned (&v)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
          "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
          "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
          "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
        : "r"(taddr)
        : "memory");
}
__device__ __forceinline__ void tc_ld2(unsigned taddr, unsigned &a, unsigned &b) {
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x2.b32 {%0, %1}, [%2];" : "=r"(a), "=r"(b) : "r"(taddr) : "memory");
}

// bounded wait on phase `parity` of an mbarrier; false when it gave up
__device__ __forceinline__ bool tc_mbar_wait(unsigned bar, unsigned parity) {
    unsigned done = 0;
    for (int it = 0; it < (1 << 22) && !done; it++)
        asm volatile(
            "{\n.reg .pred p;\nmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\nselp.u32 %0, 1, 0, p;\n}"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
    return done != 0;
}

// CTAs whose MMA completion did not arrive within the wait limit
__device__ int g_mlp_wait_timeouts;

// Per-CTA state: shared-memory base of the weight image, TMEM base, and per
// warpgroup the activation tile, the mbarrier, its phase and a status word.
struct TcCta {
    unsigned char *img;   // MLPT_BYTES, then NWG activation tiles
    unsigned tmem;
    unsigned long long *bar;
    int *status;
};

// Carve the dynamic shared memory, copy the weight image, allocate TMEM
// (warp 0) and initialise the barriers. Every thread of the CTA calls it.
template <int NWG>
__device__ __forceinline__ TcCta tc_setup(unsigned char *smem_raw, const uint4 *__restrict__ image) {
    TcCta c;
    const unsigned base = (unsigned)__cvta_generic_to_shared(smem_raw);
    c.img = smem_raw + ((1024u - (base & 1023u)) & 1023u);
    unsigned char *tail = c.img + MLPT_BYTES + NWG * MLPT_TILE;
    c.bar = reinterpret_cast<unsigned long long *>(tail);
    c.status = reinterpret_cast<int *>(tail + 8 * NWG);
    unsigned *tslot = reinterpret_cast<unsigned *>(tail + 12 * NWG);
    uint4 *dst = reinterpret_cast<uint4 *>(c.img);
    for (int k = threadIdx.x; k < MLPT_BYTES / 16; k += blockDim.x) dst[k] = image[k];
    if (threadIdx.x < 32) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         (unsigned)__cvta_generic_to_shared(tslot)),
                     "r"(NWG * MLPT_NCOL)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (threadIdx.x == 0) {
        for (int w = 0; w < NWG; w++) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"((unsigned)__cvta_generic_to_shared(&c.bar[w]))
                         : "memory");
            c.status[w] = 1;
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    tc_proxy_fence();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    c.tmem = *tslot;
    return c;
}

// Every thread of the CTA: wait for the last MMAs of warpgroups that gave up
// (bounded), then warp 0 frees the TMEM columns.
template <int NWG>
__device__ __forceinline__ void tc_teardown(const TcCta &c) {
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (threadIdx.x < 32)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(c.tmem), "r"(NWG * MLPT_NCOL)
                     : "memory");
}

// address of row r's 16-byte chunk c in an activation tile (K64 layout)
__device__ __forceinline__ unsigned char *tc_row_chunk(unsigned char *tile, int r, int c) {
    return tile + tc_off64(r, 8 * c);
}

// Layer-1 input of row r: the nine normalised features, the two bias columns
// (one) and zeros, BF16, chunks 0 and 1 of the row.
__device__ __forceinline__ void tc_put_input(unsigned char *tile, int r, const float (&xn)[MLP_IN]) {
    uint4 c0, c1;
    c0.x = pack_bf2(xn[0], xn[1]);
    c0.y = pack_bf2(xn[2], xn[3]);
    c0.z = pack_bf2(xn[4], xn[5]);
    c0.w = pack_bf2(xn[6], xn[7]);
    c1.x = pack_bf2(xn[8], 1.0f);
    c1.y = pack_bf2(1.0f, 0.0f);
    c1.z = 0u;
    c1.w = 0u;
    *reinterpret_cast<uint4 *>(tc_row_chunk(tile, r, 0)) = c0;
    *reinterpret_cast<uint4 *>(tc_row_chunk(tile, r, 1)) = c1;
}

// accumulator columns [c0, c0 + 32) of this thread's row -> BF16 pairs ->
// GELU -> chunks c0/8 .. c0/8 + 3 of the row
__device__ __forceinline__ void tc_gelu_half(unsigned taddr, unsigned char *tile, int r, int c0) {
    unsigned v[32];
    tc_ld32(taddr + (unsigned)c0, v);
    tc_wait_ld();
#pragma unroll
    for (int q = 0; q < 4; q++) {
        uint4 o;
        o.x = gelu2_bf16x2(pack_bf2(__uint_as_float(v[8 * q + 0]), __uint_as_float(v[8 * q + 1])));
        o.y = gelu2_bf16x2(pack_bf2(__uint_as_float(v[8 * q + 2]), __uint_as_float(v[8 * q + 3])));
        o.z = gelu2_bf16x2(pack_bf2(__uint_as_float(v[8 * q + 4]), __uint_as_float(v[8 * q + 5])));
        o.w = gelu2_bf16x2(pack_bf2(__uint_as_float(v[8 * q + 6]), __uint_as_float(v[8 * q + 7])));
        *reinterpret_cast<uint4 *>(tc_row_chunk(tile, r, c0 / 8 + q)) = o;
    }
}

// Issue (one thread) the MMAs of a layer and wait for them; the status word
// tells the warpgroup whether they completed within the wait limit.
__device__ __forceinline__ void tc_layer_issue(const TcCta &c, int wg, unsigned tile_s, int layer, unsigned &phase) {
    const unsigned img = (unsigned)__cvta_generic_to_shared(c.img);
    const unsigned d = c.tmem + (unsigned)(wg * MLPT_NCOL);
    const unsigned bar = (unsigned)__cvta_generic_to_shared(&c.bar[wg]);
    tc_fence_after();
    if (layer == 1) {
        tc_mma(d, tc_desc(tile_s, 128, 1024), tc_desc(img + MLPT_W1, 128, 256), tc_idesc(64), 0u);
    } else {
        const int w = layer == 2 ? MLPT_W2 : layer == 3 ? MLPT_W3 : MLPT_W4;
        const int b = layer == 2 ? MLPT_B2 : layer == 3 ? MLPT_B3 : MLPT_B4;
        const unsigned id = tc_idesc(layer == 4 ? 16 : 64);
#pragma unroll
        for (int kk = 0; kk < 4; kk++)
            tc_mma(d, tc_desc(tile_s + kk * 256, 128, 1024), tc_desc(img + w + kk * 256, 128, 1024), id,
                   kk > 0 ? 1u : 0u);
        tc_mma(d, tc_desc(img + MLPT_AC, 128, 256), tc_desc(img + b, 128, 256), id, 1u);
    }
    tc_commit(bar);
    const bool ok = tc_mbar_wait(bar, phase);
    if (!ok) {
        atomicAdd(&g_mlp_wait_timeouts, 1);
        tc_mbar_wait(bar, phase);   // once more, for the copies still in flight
    }
    c.status[wg] = ok ? 1 : 0;
}

// The network on the warpgroup's tile whose layer-1 inputs the 128 threads
// have written (row r = this thread's point). Returns false, uniformly over
// the warpgroup, when an MMA did not complete in time; otherwise the two raw
// outputs of row r. One tile per warpgroup and three CTAs of two warpgroups
// per SM; the issuing thread alone waits on the mbarrier while the others
// wait at the warpgroup barrier. Measured alternatives on the 128^3 pass (212
// us here): every thread polling the mbarrier, 227 us (the polling takes
// issue slots); two tiles in flight per warpgroup, the MMAs of one under the
// activation work of the other, 242 us (128 TMEM columns and 32 KB of tiles
// per warpgroup leave 16 warps per SM instead of 24).
__device__ __forceinline__ bool tc_forward(const TcCta &c, int wg, int r, unsigned &phase, float &o0, float &o1) {
    unsigned char *tile = c.img + MLPT_BYTES + wg * MLPT_TILE;
    const unsigned tile_s = (unsigned)__cvta_generic_to_shared(tile);
    const unsigned trow = c.tmem + ((unsigned)(r & ~31) << 16) + (unsigned)(wg * MLPT_NCOL);
    const bool leader = r == 0;
#pragma unroll 1
    for (int layer = 1; layer <= 4; layer++) {
        if (layer > 1) {
            tc_gelu_half(trow, tile, r, 0);
            tc_gelu_half(trow, tile, r, 32);
        }
        tc_proxy_fence();
        tc_fence_before();
        wg_bar(wg);
        if (leader) tc_layer_issue(c, wg, tile_s, layer, phase);
        phase ^= 1u;
        wg_bar(wg);
        tc_fence_after();
        if (!c.status[wg]) return false;
    }
    unsigned a, b;
    tc_ld2(trow, a, b);
    tc_wait_ld();
    tc_fence_before();
    o0 = __uint_as_float(a);
    o1 = __uint_as_float(b);
    return true;
}


}  // namespace mc3d
