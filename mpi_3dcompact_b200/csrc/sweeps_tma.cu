// TMA-staged line solves (kernels in sweep_tma.cuh): tensor maps and launches.
#include <algorithm>
#include <cstdlib>
#include <map>
#include <mutex>
#include <tuple>

#include "sweep_tma.cuh"

namespace mc3d {
namespace {

// cuTensorMapEncodeTiled through the runtime's driver entry point, so the
// library loads without libcuda on hosts that only build or test it
using EncodeTiledFn = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                   const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiledFn encode_tiled() {
    static EncodeTiledFn fn = [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            return (EncodeTiledFn) nullptr;
        return reinterpret_cast<EncodeTiledFn>(p);
    }();
    return fn;
}

// FP32 tensor map (rank 2 or 3, innermost first; strides in bytes of the
// outer dimensions) with the 128-byte swizzle; cached per (address, shape,
// strides, box) since a run reuses a fixed set of field buffers.
bool tensor_map(const void *p, int rank, const cuuint64_t *dims, const cuuint64_t *strides, const cuuint32_t *box,
                CUtensorMap *out) {
    using Key = std::tuple<const void *, int, cuuint64_t, cuuint64_t, cuuint64_t, cuuint64_t, cuuint64_t, cuuint32_t,
                           cuuint32_t, cuuint32_t>;
    static std::mutex mu;
    static std::map<Key, CUtensorMap> cache;
    std::lock_guard<std::mutex> lk(mu);
    const Key key{p,          rank,   dims[0], dims[1], rank > 2 ? dims[2] : 0, strides[0], rank > 2 ? strides[1] : 0,
                  box[0],     box[1], rank > 2 ? box[2] : 0};
    auto it = cache.find(key);
    if (it != cache.end()) {
        *out = it->second;
        return true;
    }
    if (((uintptr_t)p & 15) != 0) return false;
    for (int i = 0; i < rank - 1; i++)
        if (strides[i] % 16 != 0) return false;
    const cuuint32_t estr[3] = {1, 1, 1};
    const EncodeTiledFn enc = encode_tiled();
    if (!enc) return false;
    CUtensorMap m;
    if (enc(&m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, (cuuint32_t)rank, const_cast<void *>(p), dims, strides, box, estr,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return false;
    if (cache.size() > 4096) cache.clear();
    cache.emplace(key, m);
    *out = m;
    return true;
}

// x lines: [Ny*Nz lines][Nx] with 32 x 32 boxes
bool tensor_map_x(const void *p, int nx, long long lines, CUtensorMap *out) {
    const cuuint64_t dims[2] = {(cuuint64_t)nx, (cuuint64_t)lines};
    const cuuint64_t strides[1] = {(cuuint64_t)nx * 4};
    const cuuint32_t box[2] = {(cuuint32_t)TMA_BOX, (cuuint32_t)W};
    return tensor_map(p, 2, dims, strides, box, out);
}

// y lines: the [Nz][Ny][Nx] field with {32, min(Ny, 256), 1} boxes; z lines:
// the [Nz][Nx*Ny] view with {32, min(Nz, 256)} boxes
bool tensor_map_yz(int dir, const void *p, const Grid3 &g, CUtensorMap *out) {
    if (dir == 1) {
        const cuuint64_t dims[3] = {(cuuint64_t)g.Nx, (cuuint64_t)g.Ny, (cuuint64_t)g.Nz};
        const cuuint64_t strides[2] = {(cuuint64_t)g.Nx * 4, (cuuint64_t)g.Nx * g.Ny * 4};
        const cuuint32_t box[3] = {(cuuint32_t)W, (cuuint32_t)std::min(g.Ny, TMA_ROWS), 1};
        return tensor_map(p, 3, dims, strides, box, out);
    }
    const cuuint64_t dims[2] = {(cuuint64_t)g.Nx * g.Ny, (cuuint64_t)g.Nz};
    const cuuint64_t strides[1] = {(cuuint64_t)g.Nx * g.Ny * 4};
    const cuuint32_t box[2] = {(cuuint32_t)W, (cuuint32_t)std::min(g.Nz, TMA_ROWS)};
    return tensor_map(p, 2, dims, strides, box, out);
}

template <int DIR, int KIND, int H, int L, int E>
int launch_tma_yz_epi(const Grid3 &g, const LineOpDev<float> &op, const SweepBatch<float> &b,
                      const RhsFinalArgs<float> &rf, const TmaMaps &maps, int px, int py, int pz, cudaStream_t st) {
    const int S = op.N / L;
    const size_t smem = 1024 + (size_t)op.N * 128 + (size_t)reg_chain_elems(S) * sizeof(float);
    // plain, negated and FP64 stores: persistent CTAs with the next tile's load in
    // flight; the operations that read operands: one CTA per tile, the
    // operand tiles arriving by TMA during the solve
    if constexpr (E == EPI_STORE || E == EPI_STORE_NEG || E == EPI_STORE_F64) {
        auto kern = sweep_tma_yz_persist_kernel<DIR, KIND, H, L, E>;
        static KernelLaunchState ls;
        int ctas = 0;
        if (int rc = open_kernel(kern, ls, smem, 32 * S, &ctas)) return rc;
        const int items = tile_count<DIR>(g) * b.nf;
        kern<<<items < ctas ? items : ctas, 32 * S, smem, st>>>(g, op, b, rf, maps, px, py, pz);
        MC3D_CUDA_TRY(cudaGetLastError());
        return MC3D_OK;
    } else {
        auto kern = sweep_tma_yz_kernel<DIR, KIND, H, L, E>;
        static KernelLaunchState ls;
        if (int rc = open_kernel(kern, ls, smem, 32 * S, nullptr)) return rc;
        dim3 grid(tile_count<DIR>(g), b.nf);
        kern<<<grid, 32 * S, smem, st>>>(g, op, b, rf, maps, px, py, pz);
        MC3D_CUDA_TRY(cudaGetLastError());
        return MC3D_OK;
    }
}

template <int DIR, int KIND, int H>
int launch_tma_yz_kind(const Grid3 &g, const LineOpDev<float> &op, const SweepBatch<float> &b, int epi,
                       const RhsFinalArgs<float> &rf, const TmaMaps &maps, int px, int py, int pz, cudaStream_t st) {
    if (epi == EPI_STORE) return launch_tma_yz_epi<DIR, KIND, H, 64, EPI_STORE>(g, op, b, rf, maps, px, py, pz, st);
    if constexpr (H >= 4) {
        if (epi == EPI_STORE_F64)
            return launch_tma_yz_epi<DIR, KIND, H, 64, EPI_STORE_F64>(g, op, b, rf, maps, px, py, pz, st);
    }
    if constexpr (H <= 3) {
        if (epi == EPI_STORE_NEG)
            return launch_tma_yz_epi<DIR, KIND, H, 64, EPI_STORE_NEG>(g, op, b, rf, maps, px, py, pz, st);
        if (epi == EPI_SUB) return launch_tma_yz_epi<DIR, KIND, H, 64, EPI_SUB>(g, op, b, rf, maps, px, py, pz, st);
        if (epi == EPI_RHS_FINAL)
            return launch_tma_yz_epi<DIR, KIND, H, 64, EPI_RHS_FINAL>(g, op, b, rf, maps, px, py, pz, st);
    }
    return MC3D_ERR_CONFIG;
}

template <int KIND, int H, int L, int E>
int launch_tma_epi(const Grid3 &g, const LineOpDev<float> &op, const TmaMaps &maps, int nf, int py, int pz,
                   cudaStream_t st) {
    // input and output tiles, chain states; persistent CTAs, as many as fit
    const int S = op.N / L;
    const size_t smem = 1024 + 2 * (size_t)(op.N / TMA_BOX) * 4096 + (size_t)reg_chain_elems(S) * sizeof(float);
    auto kern = sweep_tma_x_persist_kernel<KIND, H, L, E>;
    static KernelLaunchState ls;
    int ctas = 0;
    if (int rc = open_kernel(kern, ls, smem, 32 * S, &ctas)) return rc;
    const int items = tile_count<0>(g) * nf;
    kern<<<items < ctas ? items : ctas, 32 * S, smem, st>>>(g, op, maps, nf, py, pz);
    MC3D_CUDA_TRY(cudaGetLastError());
    return MC3D_OK;
}

template <int KIND, int H>
int launch_tma_kind(const Grid3 &g, const LineOpDev<float> &op, const TmaMaps &maps, int nf, int epi, int py, int pz,
                    cudaStream_t st) {
    if (epi == EPI_STORE) return launch_tma_epi<KIND, H, 64, EPI_STORE>(g, op, maps, nf, py, pz, st);
    if constexpr (H <= 3) {
        if (epi == EPI_STORE_NEG) return launch_tma_epi<KIND, H, 64, EPI_STORE_NEG>(g, op, maps, nf, py, pz, st);
    }
    return MC3D_ERR_CONFIG;
}

}  // namespace

int launch_sweep_tma_x(const Grid3 &g, const LineOpDev<float> &op, const SweepBatch<float> &b, int epi, int px,
                       int py, int pz, cudaStream_t st) {
    static const bool disabled = [] {
        const char *e = std::getenv("MC3D_NO_TMA");
        return e && e[0] == '1';
    }();
    if (disabled) return MC3D_ERR_CONFIG;
    // stores and negated stores (the latter without pass-through lines) of
    // lines up to 256 values in 64-row segments
    if (!(epi == EPI_STORE || (epi == EPI_STORE_NEG && !px && !py && !pz))) return MC3D_ERR_CONFIG;
    if (op.L != 64 || op.N % TMA_BOX != 0 || op.N > 256 || op.N != g.Nx) return MC3D_ERR_CONFIG;
    if (b.nf < 1 || b.nf > TMA_MAXF) return MC3D_ERR_CONFIG;
    const long long lines = (long long)g.Ny * g.Nz;
    TmaMaps maps;
    for (int f = 0; f < b.nf; f++)
        if (!tensor_map_x(b.in[f], g.Nx, lines, &maps.in[f]) || !tensor_map_x(b.out[f], g.Nx, lines, &maps.out[f]))
            return MC3D_ERR_CONFIG;
    if (op.kind == K_TRI_PER && op.H == 2) return launch_tma_kind<K_TRI_PER, 2>(g, op, maps, b.nf, epi, py, pz, st);
    if (op.kind == K_TRI_DIR && op.H == 2) return launch_tma_kind<K_TRI_DIR, 2>(g, op, maps, b.nf, epi, py, pz, st);
    if (op.kind == K_PEN_PER && op.H == 3) return launch_tma_kind<K_PEN_PER, 3>(g, op, maps, b.nf, epi, py, pz, st);
    if (op.kind == K_PEN_DIR && op.H == 3) return launch_tma_kind<K_PEN_DIR, 3>(g, op, maps, b.nf, epi, py, pz, st);
    if (op.kind == K_TRI_PER && op.H == 4) return launch_tma_kind<K_TRI_PER, 4>(g, op, maps, b.nf, epi, py, pz, st);
    if (op.kind == K_TRI_DIR && op.H == 4) return launch_tma_kind<K_TRI_DIR, 4>(g, op, maps, b.nf, epi, py, pz, st);
    if (op.kind == K_TRI_PER && op.H == 5) return launch_tma_kind<K_TRI_PER, 5>(g, op, maps, b.nf, epi, py, pz, st);
    if (op.kind == K_TRI_DIR && op.H == 5) return launch_tma_kind<K_TRI_DIR, 5>(g, op, maps, b.nf, epi, py, pz, st);
    if (op.kind == K_PEN_PER && op.H == 5) return launch_tma_kind<K_PEN_PER, 5>(g, op, maps, b.nf, epi, py, pz, st);
    if (op.kind == K_PEN_DIR && op.H == 5) return launch_tma_kind<K_PEN_DIR, 5>(g, op, maps, b.nf, epi, py, pz, st);
    return MC3D_ERR_CONFIG;
}

int launch_sweep_tma_yz(int dir, const Grid3 &g, const LineOpDev<float> &op, const SweepBatch<float> &b, int epi,
                        const RhsFinalArgs<float> &rf, int px, int py, int pz, cudaStream_t st) {
    static const bool disabled = [] {
        const char *e = std::getenv("MC3D_NO_TMA");
        return e && e[0] == '1';
    }();
    if (disabled || (dir != 1 && dir != 2)) return MC3D_ERR_CONFIG;
    // the operations of the derivative and filter sweeps; pass-through lines
    // only with the plain and FP64 stores of the filters
    if (!(epi == EPI_STORE || epi == EPI_STORE_NEG || epi == EPI_SUB || epi == EPI_RHS_FINAL || epi == EPI_STORE_F64))
        return MC3D_ERR_CONFIG;
    if (epi != EPI_STORE && epi != EPI_STORE_F64 && (px || py || pz)) return MC3D_ERR_CONFIG;
    // lines up to 256 rows in one box, up to 1024 in boxes of 256 rows
    const int n = dir == 1 ? g.Ny : g.Nz;
    if (op.L != 64 || op.N != n || n > 4 * TMA_ROWS || (n > TMA_ROWS && n % TMA_ROWS != 0)) return MC3D_ERR_CONFIG;
    if (b.nf < 1 || b.nf > TMA_MAXF) return MC3D_ERR_CONFIG;
    TmaMaps maps;
    // input tiles for every operation; the output (TMA store and previous
    // values) and partial-RHS tiles for the operations that read operands
    const bool operands = epi == EPI_SUB || epi == EPI_RHS_FINAL;
    for (int f = 0; f < b.nf; f++) {
        if (!tensor_map_yz(dir, b.in[f], g, &maps.in[f])) return MC3D_ERR_CONFIG;
        if (operands && !tensor_map_yz(dir, b.out[f], g, &maps.out[f])) return MC3D_ERR_CONFIG;
        if (epi == EPI_RHS_FINAL && !tensor_map_yz(dir, b.aux[f], g, &maps.aux[f])) return MC3D_ERR_CONFIG;
    }
#define MC3D_TCASE(K, HH)                                                                                    \
    if (op.kind == K && op.H == HH)                                                                          \
        return dir == 1 ? launch_tma_yz_kind<1, K, HH>(g, op, b, epi, rf, maps, px, py, pz, st)              \
                        : launch_tma_yz_kind<2, K, HH>(g, op, b, epi, rf, maps, px, py, pz, st);
    MC3D_TCASE(K_TRI_PER, 2)
    MC3D_TCASE(K_TRI_DIR, 2)
    MC3D_TCASE(K_PEN_PER, 3)
    MC3D_TCASE(K_PEN_DIR, 3)
    MC3D_TCASE(K_TRI_PER, 4)
    MC3D_TCASE(K_TRI_DIR, 4)
    MC3D_TCASE(K_TRI_PER, 5)
    MC3D_TCASE(K_TRI_DIR, 5)
    MC3D_TCASE(K_PEN_PER, 5)
    MC3D_TCASE(K_PEN_DIR, 5)
#undef MC3D_TCASE
    return MC3D_ERR_CONFIG;
}

int tma_wait_timeouts(int *count) {
    MC3D_CUDA_TRY(cudaMemcpyFromSymbol(count, g_tma_wait_timeouts, sizeof(int)));
    return MC3D_OK;
}

}  // namespace mc3d

extern "C" int mc3d_tma_wait_timeouts(int device, int *count) {
    if (!count) return mc3d::fail(MC3D_ERR_ARG, "null argument");
    MC3D_CUDA_TRY(cudaSetDevice(device));
    int a = 0, b = 0;
    if (int rc = mc3d::tma_wait_timeouts(&a)) return rc;
    if (int rc = mc3d::mlp_wait_timeouts(&b)) return rc;
    *count = a + b;
    return MC3D_OK;
}
