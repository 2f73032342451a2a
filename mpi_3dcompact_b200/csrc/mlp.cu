// Learned SGS closure: a 9 -> 64 -> 64 -> 64 -> 2 MLP (GELU) mapping local
// invariants of the resolved velocity-gradient tensor and the grid scale to
// the Smagorinsky-form coefficient C (nu_t = C Delta^2 |S|) and the turbulent
// Prandtl number. No counterpart in the reference: it stands in for
// VremanSGS / DSMSGS (src/VremanSGS.hpp, src/DSMSGS.hpp) behind the same
// solver path, with DSM kept as the fallback.
//
// Training (FP32, CUDA cores): mlp_forward stores pre- and post-activations,
// mlp_backward the per-sample deltas and the MSE, mlp_wgrad reduces the weight
// and bias gradients over the batch (split over the batch, one atomic add per
// split), mlp_adam applies Adam with bias correction.
// Inference (BF16 tensor cores, FP32 accumulate in tensor memory) runs on
// tcgen05 MMAs over tiles of 128 points (mlp_tc.cuh, kernels in sgs_mlp.cu);
// mlp_pack writes its weight image after every change of the parameters.
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <string>
#include <vector>

#include "mlp_common.cuh"

namespace mc3d {

// parameter offsets (floats) of the FP32 master copy
constexpr int MLP_W1 = 0;                          // [64][9]
constexpr int MLP_B1 = MLP_W1 + 64 * MLP_IN;       // [64]
constexpr int MLP_W2 = MLP_B1 + 64;                // [64][64]
constexpr int MLP_B2 = MLP_W2 + 64 * 64;
constexpr int MLP_W3 = MLP_B2 + 64;
constexpr int MLP_B3 = MLP_W3 + 64 * 64;
constexpr int MLP_W4 = MLP_B3 + 64;                // [2][64]
constexpr int MLP_B4 = MLP_W4 + MLP_OUT * 64;
constexpr int MLP_NP = MLP_B4 + MLP_OUT;           // 9090
static_assert(MLP_NP == MLP_NPARAM, "parameter count");

namespace {

// ---------------------------------------------------------------------------
// training kernels (thread per sample, parameters staged in shared memory)
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(128) mlp_forward_kernel(const float *__restrict__ P, const float *__restrict__ x,
                                                           int n, MlpNorm nrm, float *__restrict__ act,
                                                           float *__restrict__ out) {
    extern __shared__ float sp[];
    for (int k = threadIdx.x; k < MLP_NP; k += blockDim.x) sp[k] = P[k];
    __syncthreads();
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= n) return;
    float a0[MLP_IN];
#pragma unroll
    for (int k = 0; k < MLP_IN; k++) a0[k] = (x[(size_t)b * MLP_IN + k] - nrm.mean[k]) * nrm.inv_std[k];
    float h[64], z[64];
    // layer 1
#pragma unroll 4
    for (int o = 0; o < 64; o++) {
        float s = sp[MLP_B1 + o];
#pragma unroll
        for (int k = 0; k < MLP_IN; k++) s += sp[MLP_W1 + o * MLP_IN + k] * a0[k];
        z[o] = s;
    }
    // act layout: [6][n][64]: z1, h1, z2, h2, z3, h3
#pragma unroll 4
    for (int o = 0; o < 64; o++) {
        h[o] = gelu(z[o]);
        if (act) {
            act[(size_t)0 * n * 64 + (size_t)b * 64 + o] = z[o];
            act[(size_t)1 * n * 64 + (size_t)b * 64 + o] = h[o];
        }
    }
    for (int layer = 0; layer < 2; layer++) {
        const int W = layer == 0 ? MLP_W2 : MLP_W3, B = layer == 0 ? MLP_B2 : MLP_B3;
#pragma unroll 2
        for (int o = 0; o < 64; o++) {
            float s = sp[B + o];
#pragma unroll
            for (int k = 0; k < 64; k++) s += sp[W + o * 64 + k] * h[k];
            z[o] = s;
        }
#pragma unroll 4
        for (int o = 0; o < 64; o++) {
            h[o] = gelu(z[o]);
            if (act) {
                act[(size_t)(2 + 2 * layer) * n * 64 + (size_t)b * 64 + o] = z[o];
                act[(size_t)(3 + 2 * layer) * n * 64 + (size_t)b * 64 + o] = h[o];
            }
        }
    }
#pragma unroll
    for (int o = 0; o < MLP_OUT; o++) {
        float s = sp[MLP_B4 + o];
#pragma unroll
        for (int k = 0; k < 64; k++) s += sp[MLP_W4 + o * 64 + k] * h[k];
        out[(size_t)b * MLP_OUT + o] = s;
    }
}

// deltas of every layer for MSE loss = (1/n) sum_b sum_o (out - y)^2; loss accumulated
__global__ void __launch_bounds__(128) mlp_backward_kernel(const float *__restrict__ P, const float *__restrict__ act,
                                                            const float *__restrict__ out, const float *__restrict__ y,
                                                            int n, float *__restrict__ delta, double *loss) {
    extern __shared__ float sp[];
    for (int k = threadIdx.x; k < MLP_NP; k += blockDim.x) sp[k] = P[k];
    __syncthreads();
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    double l = 0.0;
    if (b < n) {
        float d4[MLP_OUT];
#pragma unroll
        for (int o = 0; o < MLP_OUT; o++) {
            const float e = out[(size_t)b * MLP_OUT + o] - y[(size_t)b * MLP_OUT + o];
            l += (double)e * e;
            d4[o] = 2.0f * e / (float)n;
            delta[(size_t)3 * n * 64 + (size_t)b * MLP_OUT + o] = d4[o];
        }
        float d[64], dn[64];
        // delta3 = (W4^T d4) * gelu'(z3)
#pragma unroll 4
        for (int k = 0; k < 64; k++) {
            float s = 0;
#pragma unroll
            for (int o = 0; o < MLP_OUT; o++) s += sp[MLP_W4 + o * 64 + k] * d4[o];
            d[k] = s * gelu_grad(act[(size_t)4 * n * 64 + (size_t)b * 64 + k]);
            delta[(size_t)2 * n * 64 + (size_t)b * 64 + k] = d[k];
        }
        for (int layer = 1; layer >= 0; layer--) {
            // delta_{l} = (W_{l+1}^T delta_{l+1}) * gelu'(z_l); W_{l+1} = W3 (layer 1) or W2 (layer 0)
            const int W = layer == 1 ? MLP_W3 : MLP_W2;
            const size_t zoff = (size_t)(2 * layer) * n * 64;
#pragma unroll 2
            for (int k = 0; k < 64; k++) {
                float s = 0;
#pragma unroll
                for (int o = 0; o < 64; o++) s += sp[W + o * 64 + k] * d[o];
                dn[k] = s * gelu_grad(act[zoff + (size_t)b * 64 + k]);
            }
#pragma unroll
            for (int k = 0; k < 64; k++) {
                d[k] = dn[k];
                delta[(size_t)layer * n * 64 + (size_t)b * 64 + k] = d[k];
            }
        }
    }
    // block-reduce the loss
    for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(loss, l / (double)n);
}

// G[layer] += sum_b delta[b][o] * a_prev[b][i]; bias gradients in the extra column
__global__ void mlp_wgrad_kernel(const float *__restrict__ x, MlpNorm nrm, const float *__restrict__ act,
                                 const float *__restrict__ delta, int n, int layer, float *__restrict__ G) {
    const int nin = layer == 0 ? MLP_IN : 64, nout = layer == 3 ? MLP_OUT : 64;
    const int o = blockIdx.x;                  // output row
    const int i = threadIdx.x;                 // input column, i == nin: bias
    if (o >= nout || i > nin) return;
    const int splits = gridDim.y;
    const int b0 = (int)((long long)n * blockIdx.y / splits), b1 = (int)((long long)n * (blockIdx.y + 1) / splits);
    const float *dl = layer == 3 ? delta + (size_t)3 * n * 64 : delta + (size_t)layer * n * 64;
    const int dstride = layer == 3 ? MLP_OUT : 64;
    const float *ap = layer == 0 ? nullptr : act + (size_t)(2 * layer - 1) * n * 64;   // h_{layer}
    float s = 0;
    for (int b = b0; b < b1; b++) {
        const float dv = dl[(size_t)b * dstride + o];
        float a;
        if (i == nin) a = 1.0f;
        else if (layer == 0) a = (x[(size_t)b * MLP_IN + i] - nrm.mean[i]) * nrm.inv_std[i];
        else a = ap[(size_t)b * 64 + i];
        s += dv * a;
    }
    const int W = layer == 0 ? MLP_W1 : layer == 1 ? MLP_W2 : layer == 2 ? MLP_W3 : MLP_W4;
    const int B = layer == 0 ? MLP_B1 : layer == 1 ? MLP_B2 : layer == 2 ? MLP_B3 : MLP_B4;
    atomicAdd(i == nin ? &G[B + o] : &G[W + o * nin + i], s);
}

__global__ void mlp_adam_kernel(float *P, float *G, float *M, float *V, float lr, float b1t, float b2t) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= MLP_NP) return;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    const float g = G[k];
    const float m = b1 * M[k] + (1.0f - b1) * g;
    const float v = b2 * V[k] + (1.0f - b2) * g * g;
    M[k] = m;
    V[k] = v;
    const float mh = m / (1.0f - b1t), vh = v / (1.0f - b2t);
    P[k] -= lr * mh / (sqrtf(vh) + eps);
    G[k] = 0.0f;
}

// The weight image of the tensor-core inference (layout in mlp_common.cuh),
// written over a zeroed buffer: one thread per element of the eight blocks.
// A bias b is carried as the BF16 pair (b_hi, b_lo), b_hi = bf16(b) and
// b_lo = bf16(b - b_hi), against two constant-one input columns.
__device__ __forceinline__ void bias_pair(float b, __nv_bfloat16 &hi, __nv_bfloat16 &lo) {
    hi = __float2bfloat16_rn(b);
    lo = __float2bfloat16_rn(b - __bfloat162float(hi));
}

__global__ void mlp_pack_kernel(const float *__restrict__ P, unsigned char *__restrict__ img) {
    // element counts of W1 [64][16], W2, W3 [64][64], W4 [16][64], B2, B3 [64][16], B4 [16][16], Ac [128][16]
    constexpr int n1 = 64 * 16, n2 = 64 * 64, n4 = 16 * 64, nb = 64 * 16, nb4 = 16 * 16, nac = 128 * 16;
    constexpr int total = n1 + 2 * n2 + n4 + 2 * nb + nb4 + nac;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < total; e += gridDim.x * blockDim.x) {
        int k = e, off;
        __nv_bfloat16 v = __float2bfloat16_rn(0.0f);
        if (k < n1) {   // W1 and the layer-1 bias
            const int o = k / 16, c = k % 16;
            __nv_bfloat16 hi, lo;
            bias_pair(P[MLP_B1 + o], hi, lo);
            if (c < MLP_IN) v = __float2bfloat16_rn(P[MLP_W1 + o * MLP_IN + c]);
            else if (c == MLP_IN) v = hi;
            else if (c == MLP_IN + 1) v = lo;
            off = MLPT_W1 + tc_off16(o, c);
        } else if ((k -= n1) < 2 * n2) {   // W2, W3, halved: their inputs are twice GELU (gelu2_bf16x2)
            const int w = k < n2 ? MLP_W2 : MLP_W3, kk = k % n2, o = kk / 64, c = kk % 64;
            v = __float2bfloat16_rn(0.5f * P[w + o * 64 + c]);
            off = (k < n2 ? MLPT_W2 : MLPT_W3) + tc_off64(o, c);
        } else if ((k -= 2 * n2) < n4) {   // W4, halved likewise; rows past the outputs zero
            const int o = k / 64, c = k % 64;
            if (o < MLP_OUT) v = __float2bfloat16_rn(0.5f * P[MLP_W4 + o * 64 + c]);
            off = MLPT_W4 + tc_off64(o, c);
        } else if ((k -= n4) < 2 * nb + nb4) {   // bias blocks of layers 2, 3, 4
            const int blk = k < nb ? 0 : k < 2 * nb ? 1 : 2, kk = k - blk * nb, o = kk / 16, c = kk % 16;
            const int nout = blk == 2 ? MLP_OUT : 64;
            if (o < nout && c < 2) {
                __nv_bfloat16 hi, lo;
                bias_pair(P[(blk == 0 ? MLP_B2 : blk == 1 ? MLP_B3 : MLP_B4) + o], hi, lo);
                v = c == 0 ? hi : lo;
            }
            off = (blk == 0 ? MLPT_B2 : blk == 1 ? MLPT_B3 : MLPT_B4) + tc_off16(o, c);
        } else {   // the constant-one columns of the bias MMAs
            k -= 2 * nb + nb4;
            const int r = k / 16, c = k % 16;
            if (c < 2) v = __float2bfloat16_rn(1.0f);
            off = MLPT_AC + tc_off16(r, c);
        }
        *reinterpret_cast<__nv_bfloat16 *>(img + off) = v;
    }
}

}  // namespace

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
int mlp_pack(const MlpDev &m, cudaStream_t st) {
    MC3D_CUDA_TRY(cudaMemsetAsync(m.Tw, 0, MLPT_BYTES, st));
    mlp_pack_kernel<<<16, 256, 0, st>>>(m.P, m.Tw);
    MC3D_CUDA_TRY(cudaGetLastError());
    return MC3D_OK;
}

int mlp_forward_fp32(const MlpDev &m, const float *x, int n, float *act, float *out, cudaStream_t st) {
    const size_t smem = MLP_NP * sizeof(float);
    static KernelLaunchState fwd, bwd;
    int rc;
    if ((rc = open_kernel(mlp_forward_kernel, fwd, smem, 128, nullptr))) return rc;
    if ((rc = open_kernel(mlp_backward_kernel, bwd, smem, 128, nullptr))) return rc;
    mlp_forward_kernel<<<(n + 127) / 128, 128, smem, st>>>(m.P, x, n, m.norm, act, out);
    MC3D_CUDA_TRY(cudaGetLastError());
    return MC3D_OK;
}

int mlp_gradient(MlpDev &m, const float *x, const float *y, int n, float *act, float *out, float *delta,
                 double *loss, cudaStream_t st) {
    int rc;
    if ((rc = mlp_forward_fp32(m, x, n, act, out, st))) return rc;
    const size_t smem = MLP_NP * sizeof(float);
    mlp_backward_kernel<<<(n + 127) / 128, 128, smem, st>>>(m.P, act, out, y, n, delta, loss);
    MC3D_CUDA_TRY(cudaGetLastError());
    const int splits = std::max(1, std::min(128, n / 512));
    for (int layer = 0; layer < 4; layer++) {
        const int nout = layer == 3 ? MLP_OUT : 64, nin = layer == 0 ? MLP_IN : 64;
        mlp_wgrad_kernel<<<dim3(nout, splits), nin + 1, 0, st>>>(x, m.norm, act, delta, n, layer, m.G);
        MC3D_CUDA_TRY(cudaGetLastError());
    }
    return MC3D_OK;
}

int mlp_train_step(MlpDev &m, const float *x, const float *y, int n, float lr, float *act, float *out, float *delta,
                   double *loss, cudaStream_t st) {
    int rc;
    if ((rc = mlp_gradient(m, x, y, n, act, out, delta, loss, st))) return rc;
    m.t += 1;
    const float b1t = (float)std::pow(0.9, (double)m.t), b2t = (float)std::pow(0.999, (double)m.t);
    mlp_adam_kernel<<<(MLP_NP + 255) / 256, 256, 0, st>>>(m.P, m.G, m.M, m.V, lr, b1t, b2t);
    MC3D_CUDA_TRY(cudaGetLastError());
    return mlp_pack(m, st);
}

}  // namespace mc3d
