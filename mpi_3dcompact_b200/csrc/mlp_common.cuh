// Device pieces of the learned SGS closure shared by mlp.cu and sgs_mlp.cu:
// the BF16 weight image of the tensor-core inference (mlp_tc.cuh), GELU, and
// the features of a point.
#pragma once
#include <cuda_bf16.h>

#include "pointwise_common.cuh"

namespace mc3d {

// ---- weight image of the tensor-core inference (bytes), built by mlp_pack
// and copied once into each CTA's shared memory; K16 / K64 name the operand
// layouts of tc_off16 / tc_off64 below
constexpr int MLPT_W1 = 0;         // [64][16]  K16 layout: W1 (9 columns), b1_hi, b1_lo
constexpr int MLPT_W2 = 2048;      // [64][64]  K64 layout
constexpr int MLPT_W3 = 10240;     // [64][64]
constexpr int MLPT_W4 = 18432;     // [16][64]  rows 0..1 used
constexpr int MLPT_B2 = 20480;     // [64][16]  columns 0, 1: b_hi, b_lo
constexpr int MLPT_B3 = 22528;     // [64][16]
constexpr int MLPT_B4 = 24576;     // [16][16]
constexpr int MLPT_AC = 25600;     // [128][16] columns 0, 1 equal to one
static_assert(MLPT_BYTES == MLPT_AC + 128 * 16 * 2, "image size");   // (a multiple of 1024)
constexpr int MLPT_TILE = 16384;   // one warpgroup's activation tile [128][64] BF16
constexpr int MLPT_NCOL = 64;      // TMEM columns per warpgroup

// byte offset of element (r, k) in the K-major no-swizzle layouts
__host__ __device__ constexpr int tc_off16(int r, int k) {
    return (r >> 3) * 256 + (k >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2;
}
__host__ __device__ constexpr int tc_off64(int r, int k) {
    return (r >> 3) * 1024 + (k >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2;
}

// instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B, both
// K-major, M = 128, N = n
__host__ __device__ constexpr unsigned tc_idesc(int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((unsigned)(n >> 3) << 17) | ((unsigned)(128 >> 4) << 24);
}

// GELU in its tanh form, 0.5 x (1 + tanh(sqrt(2/pi) (x + 0.044715 x^3))): the
// training kernels use tanhf in FP32, the tensor-core inference gelu2_bf16x2
constexpr float GELU_K0 = 0.7978845608028654f, GELU_K1 = 0.044715f;
__device__ __forceinline__ float gelu(float x) {
    return 0.5f * x * (1.0f + tanhf(GELU_K0 * (x + GELU_K1 * x * x * x)));
}
__device__ __forceinline__ float gelu_grad(float x) {
    const float t = tanhf(GELU_K0 * (x + GELU_K1 * x * x * x));
    return 0.5f * (1.0f + t) + 0.5f * x * (1.0f - t * t) * GELU_K0 * (1.0f + 3.0f * GELU_K1 * x * x);
}
// two FP32 values as a BF16 pair (lo in the low half), round to nearest even
__device__ __forceinline__ unsigned pack_bf2(float lo, float hi) {
    __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<unsigned *>(&v);
}

// Twice the same GELU on a BF16 pair in five packed instructions (six with
// the conversion of the FP32 accumulator pair), as the
// tensor-core inference uses it (its operands are BF16 anyway): u = x (K0 +
// K0 K1 x^2), 2 gelu = x + x tanh(u), every step rounded to BF16 and tanh by
// the hardware's tanh.approx.bf16x2; the factor 1/2 sits in the next layer's
// weights (mlp_pack halves them, exactly), so the products are those of
// h = x / 2, gelu = h + h tanh(u) bit for bit. Against GELU in FP32 rounded
// once to BF16 this moves the shipped network's outputs by at most 0.6% of
// their range on standard-normal inputs (numpy emulation with exact tanh).
__device__ __forceinline__ unsigned gelu2_bf16x2(unsigned x) {
    const unsigned k01 = pack_bf2(GELU_K0 * GELU_K1, GELU_K0 * GELU_K1), k0 = pack_bf2(GELU_K0, GELU_K0);
    unsigned y;
    asm("{\n.reg .b32 x2, t, u, th;\n"
        "mul.rn.bf16x2 x2, %1, %1;\n"
        "fma.rn.bf16x2 t, x2, %2, %3;\n"
        "mul.rn.bf16x2 u, %1, t;\n"
        "tanh.approx.bf16x2 th, u;\n"
        "fma.rn.bf16x2 %0, %1, th, %1;\n}"
        : "=r"(y)
        : "r"(x), "r"(k01), "r"(k0));
    return y;
}

// Features of one point (see sgs_mlp.cu), in FP32: the inference and the
// training data both use this function. Quotients by the hardware reciprocal
// (__fdividef, 2 ulp), logarithm and square roots as the library rounds them;
// returns |S| = (2 S:S)^(1/2).
__device__ __forceinline__ float mlp_features(const float gu[3][3], float rho, float T, const float gT[3], float delta,
                                              float mu, float *x) {
    float S[3][3], Wm[3][3];
    float s2 = 0.f, w2 = 0.f;
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
        for (int b = 0; b < 3; b++) {
            S[a][b] = 0.5f * (gu[a][b] + gu[b][a]);
            Wm[a][b] = 0.5f * (gu[a][b] - gu[b][a]);
            s2 += S[a][b] * S[a][b];
            w2 += Wm[a][b] * Wm[a][b];
        }
    float trS3 = 0.f, trSW2 = 0.f, trS2W2 = 0.f;
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
        for (int b = 0; b < 3; b++) {
            float p = 0.f, q = 0.f;
#pragma unroll
            for (int k = 0; k < 3; k++) {
                p += S[a][k] * S[k][b];
                q += Wm[a][k] * Wm[k][b];
            }
            // p = (S S)_ab, q = (W W)_ab
            trS3 += p * S[b][a];
            trSW2 += S[a][b] * q;
            trS2W2 += p * q;
        }
    const float eps = 1e-30f, sw = s2 + w2;
    const float rs = sqrtf(s2), rsw = sqrtf(sw);
    const float smag = 1.41421356f * rs;
    const float c = sqrtf((float)(GAMMA * R_GAS) * T);
    const float gTm = sqrtf(gT[0] * gT[0] + gT[1] * gT[1] + gT[2] * gT[2]);
    x[0] = log1pf(__fdividef(rho * delta * delta * smag, mu));
    x[1] = __fdividef(w2, sw + eps);
    x[2] = __fdividef(trS3, s2 * rs + eps);
    x[3] = __fdividef(trSW2, sw * rsw + eps);
    x[4] = __fdividef(trS2W2, sw * sw + eps);
    x[5] = __fdividef(gu[0][0] + gu[1][1] + gu[2][2], rsw + eps);
    x[6] = __fdividef(delta * gTm, T);
    x[7] = __fdividef(delta * smag, c);
    x[8] = logf(rho);
    return smag;
}

}  // namespace mc3d
