// Device pieces of the learned SGS closure shared by mlp.cu and sgs_mlp.cu:
// the packed BF16 weight layout, GELU, and the tensor-core evaluation of a
// 16-point tile (mma.sync m16n8k16, BF16 inputs, FP32 accumulate).
#pragma once
#include <cuda_bf16.h>

#include "pointwise_common.cuh"

namespace mc3d {

// bf16 inference copies, rows padded so the B-fragment loads of a warp hit 32
// distinct banks: W1 [64][24] (9 used), W2 and W3 [64][72] (64 used), W4 [8][72]
// (2 x 64 used); the biases follow as FP32 in MlpDev::Bc [64 | 64 | 64 | 2]
constexpr int MLPH_P1 = 24, MLPH_P = 72;
constexpr int MLPH_W1 = 0;
constexpr int MLPH_W2 = MLPH_W1 + 64 * MLPH_P1;
constexpr int MLPH_W3 = MLPH_W2 + 64 * MLPH_P;
constexpr int MLPH_W4 = MLPH_W3 + 64 * MLPH_P;
constexpr int MLPH_N = MLPH_W4 + 8 * MLPH_P;
static_assert(MLPH_N == MLP_NHALF, "packed size");

// GELU in its tanh form, 0.5 x (1 + tanh(sqrt(2/pi) (x + 0.044715 x^3))): the
// training kernels use tanhf, the tensor-core inference the hardware tanh.approx
constexpr float GELU_K0 = 0.7978845608028654f, GELU_K1 = 0.044715f;
__device__ __forceinline__ float gelu(float x) {
    return 0.5f * x * (1.0f + tanhf(GELU_K0 * (x + GELU_K1 * x * x * x)));
}
__device__ __forceinline__ float gelu_grad(float x) {
    const float t = tanhf(GELU_K0 * (x + GELU_K1 * x * x * x));
    return 0.5f * (1.0f + t) + 0.5f * x * (1.0f - t * t) * GELU_K0 * (1.0f + 3.0f * GELU_K1 * x * x);
}
__device__ __forceinline__ float tanh_approx(float x) {
    float y;
    asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
// the same function in six instructions: u = x (K0 + K0 K1 x^2), h = x / 2,
// gelu = h + h tanh(u)
__device__ __forceinline__ float gelu_fast(float x) {
    const float u = x * fmaf(GELU_K0 * GELU_K1, x * x, GELU_K0);
    const float h = 0.5f * x;
    return fmaf(h, tanh_approx(u), h);
}

// ---------------------------------------------------------------------------
// BF16 tensor-core inference of one warp's 32 points (two m16 tiles). The
// normalised features of point p are in xs[p * XS + 0..15] (bf16, zero
// padded); outputs of point p go to ys[p * 2 + 0..1].
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned pack_bf2(float lo, float hi) {
    __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<unsigned *>(&v);
}

__device__ __forceinline__ void mma_bf16(float (&c)[4], const unsigned (&a)[4], unsigned b0, unsigned b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// one hidden layer on a 16-point tile: A fragments of K = 16 * KT columns in a[KT][4],
// weights W [64][PITCH] (bf16, row-major), bias b; writes the GELU output as A fragments
template <int KT, int PITCH>
__device__ __forceinline__ void mlp_layer(const unsigned (&a)[KT][4], const __nv_bfloat16 *W, const float *bias,
                                          unsigned (&next)[4][4], int g, int t) {
#pragma unroll
    for (int j = 0; j < 4; j++) {   // next layer's k-tile j = this layer's n-tiles 2j, 2j+1
        float c[2][4];
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const int n0 = (2 * j + h) * 8;
            const float bl = bias[n0 + 2 * t], bh = bias[n0 + 2 * t + 1];
            c[h][0] = bl;
            c[h][1] = bh;
            c[h][2] = bl;
            c[h][3] = bh;
#pragma unroll
            for (int kt = 0; kt < KT; kt++) {
                const __nv_bfloat16 *wr = W + (size_t)(n0 + g) * PITCH + kt * 16 + 2 * t;
                const unsigned b0 = *reinterpret_cast<const unsigned *>(wr);
                const unsigned b1 = *reinterpret_cast<const unsigned *>(wr + 8);
                mma_bf16(c[h], a[kt], b0, b1);
            }
        }
        next[j][0] = pack_bf2(gelu_fast(c[0][0]), gelu_fast(c[0][1]));
        next[j][1] = pack_bf2(gelu_fast(c[0][2]), gelu_fast(c[0][3]));
        next[j][2] = pack_bf2(gelu_fast(c[1][0]), gelu_fast(c[1][1]));
        next[j][3] = pack_bf2(gelu_fast(c[1][2]), gelu_fast(c[1][3]));
    }
}

// 16 points starting at row r0 of xs (bf16 [..][XS]); outputs (raw network
// outputs) to ys[(r0 + row) * 2 + o]; Hw packed weights, bias the compact biases
template <int XS>
__device__ __forceinline__ void mlp_tile16(const __nv_bfloat16 *xs, int r0, const __nv_bfloat16 *Hw,
                                           const float *bias, float *ys, int lane) {
    const int g = lane >> 2, t = lane & 3;
    unsigned a1[1][4];
    {
        const __nv_bfloat16 *r = xs + (size_t)(r0 + g) * XS, *r8 = xs + (size_t)(r0 + g + 8) * XS;
        a1[0][0] = *reinterpret_cast<const unsigned *>(r + 2 * t);
        a1[0][1] = *reinterpret_cast<const unsigned *>(r8 + 2 * t);
        a1[0][2] = *reinterpret_cast<const unsigned *>(r + 2 * t + 8);
        a1[0][3] = *reinterpret_cast<const unsigned *>(r8 + 2 * t + 8);
    }
    unsigned h1[4][4], h2[4][4], h3[4][4];
    mlp_layer<1, MLPH_P1>(a1, Hw + MLPH_W1, bias, h1, g, t);
    mlp_layer<4, MLPH_P>(h1, Hw + MLPH_W2, bias + 64, h2, g, t);
    mlp_layer<4, MLPH_P>(h2, Hw + MLPH_W3, bias + 128, h3, g, t);
    // output layer: n-tile 0 of W4 padded to 8 rows
    float c[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
    for (int kt = 0; kt < 4; kt++) {
        const __nv_bfloat16 *wr = Hw + MLPH_W4 + (size_t)g * MLPH_P + kt * 16 + 2 * t;
        mma_bf16(c, h3[kt], *reinterpret_cast<const unsigned *>(wr), *reinterpret_cast<const unsigned *>(wr + 8));
    }
    if (t == 0) {
        ys[(r0 + g) * 2 + 0] = c[0] + bias[192];
        ys[(r0 + g) * 2 + 1] = c[1] + bias[193];
        ys[(r0 + g + 8) * 2 + 0] = c[2] + bias[192];
        ys[(r0 + g + 8) * 2 + 1] = c[3] + bias[193];
    }
}

// Features of one point (see sgs_mlp.cu), in FP32: the inference and the
// training data both use this function.
__device__ __forceinline__ void mlp_features(const float gu[3][3], float rho, float T, const float gT[3], float delta,
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
    const float smag = sqrtf(2.0f * s2);
    const float c = sqrtf((float)(GAMMA * R_GAS) * T);
    const float gTm = sqrtf(gT[0] * gT[0] + gT[1] * gT[1] + gT[2] * gT[2]);
    x[0] = log1pf(rho * delta * delta * smag / mu);
    x[1] = w2 / (sw + eps);
    x[2] = trS3 / (s2 * sqrtf(s2) + eps);
    x[3] = trSW2 / (sw * sqrtf(sw) + eps);
    x[4] = trS2W2 / (sw * sw + eps);
    x[5] = (gu[0][0] + gu[1][1] + gu[2][2]) / (sqrtf(sw) + eps);
    x[6] = delta * gTm / T;
    x[7] = delta * smag / c;
    x[8] = logf(rho);
}

}  // namespace mc3d
