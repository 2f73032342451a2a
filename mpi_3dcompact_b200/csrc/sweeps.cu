// Batched compact line solves along one grid direction.
//
// One CTA = one warp = one tile of W = 32 lines of one field. The tile is
// staged whole in shared memory as s[n][w] (line w, element n, row pitch
// W+1 words so that both the thread-per-line sweeps and the coalesced
// global<->shared copies are bank-conflict free), then each lane runs the
// elimination for its own line in place:
//   forward:  RHS stencil from a register window of 2H+1 inputs, then the
//             RHS half of Thomas (tridiagonal) or of the pentadiagonal
//             elimination, with multipliers precomputed in FP64 on the host;
//   backward: substitution with the precomputed reciprocal pivots;
//   cyclic:   Sherman-Morrison (tri) or rank-4 Woodbury (penta) correction.
// The epilogue streams the tile back with coalesced accesses and applies the
// caller's operation (store, negate, accumulate, or the k2 assembly).
//
// Reference loops this replaces: Pade6/Penta10/CD2::calc1stDerivField
// (src/Pade6.cpp:3-46), Compact8/10Filter::filterField
// (src/Compact10Filter.cpp:166-252) with src/Utils.cpp:4-191 per line.
#include <cstdio>

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
__device__ __forceinline__ int tile_count(const Grid3 &g) {
    if (DIR == 0) return (int)(((long long)g.Ny * g.Nz + W - 1) / W);
    if (DIR == 1) return ((g.Nx + W - 1) / W) * g.Nz;
    return (int)(((long long)g.Nx * g.Ny + W - 1) / W);
}

// ---------------------------------------------------------------------------
// per-line solve, in place on col[n * SP], n = 0 .. N-1 (+ H wrap rows)
// ---------------------------------------------------------------------------
template <typename R, int KIND, int H>
__device__ __forceinline__ R stencil(const R (&win)[2 * H + 1], const LineOpDev<R> &op) {
    R s = op.st[0] * win[0];
#pragma unroll
    for (int k = 1; k < 2 * H + 1; k++) s += op.st[k] * win[k];
    return s;
}

template <typename R, int KIND, int H>
__device__ __forceinline__ R stencil_mirror(const R (&win)[2 * H + 1], const LineOpDev<R> &op) {
    R s = op.st[2 * H] * win[0];
#pragma unroll
    for (int k = 1; k < 2 * H + 1; k++) s += op.st[2 * H - k] * win[k];
    return s;
}

template <typename R, int KIND, int H>
__device__ void solve_line(R *col, const LineOpDev<R> &op) {
    constexpr bool PER = (KIND % 2) == 0;
    constexpr bool TRI = KIND == K_TRI_PER || KIND == K_TRI_DIR;
    constexpr bool PEN = KIND == K_PEN_PER || KIND == K_PEN_DIR;
    const int N = op.N;

    // window of inputs phi[n-H .. n+H] for n = 0
    R win[2 * H + 1];
#pragma unroll
    for (int k = 0; k < 2 * H + 1; k++) {
        int idx = k - H;
        if (idx < 0) win[k] = PER ? col[(idx + N) * SP] : R(0);
        else win[k] = col[idx * SP];
    }
    // Dirichlet boundary rows read inputs the in-place sweep overwrites: evaluate first
    R headr[H], tailr[H];
    if (!PER) {
#pragma unroll
        for (int r = 0; r < H; r++) {
            R h = 0, t = 0;
            for (int k = 0; k < op.bw; k++) {
                h += ldc(op.head + r * op.bw + k) * col[k * SP];
                t += ldc(op.tail + r * op.bw + k) * col[(N - op.bw + k) * SP];
            }
            headr[r] = h * op.inv_dh;
            tailr[r] = t * op.inv_dh;
        }
    }

    R xp = 0, xpp = 0;   // B[n-1], B[n-2] of the forward elimination
    auto process = [&](int n, R rhs) {
        if (TRI) {
            R x = (n == 0) ? rhs : rhs - ldc(op.a0 + n) * xp;
            col[n * SP] = x;
            xp = x;
        } else if (PEN) {
            R b = rhs;
            if (n >= 2) b -= ldc(op.a1 + (n - 1)) * xpp;
            if (n >= 1) b -= ldc(op.a0 + n) * xp;
            col[n * SP] = b;
            xpp = xp;
            xp = b;
        } else {
            col[n * SP] = rhs;
        }
    };
    auto advance = [&](int n) {
#pragma unroll
        for (int k = 0; k < 2 * H; k++) win[k] = win[k + 1];
        // rows N .. N+H-1 hold the wrap copy (periodic) or zeros (Dirichlet)
        win[2 * H] = col[(n + H + 1) * SP];
    };

#pragma unroll
    for (int r = 0; r < H; r++) {
        R rhs;
        if (PER) {
            if (KIND == K_EXPL_PER && r == 0) rhs = stencil_mirror<R, KIND, H>(win, op) * op.inv_dh;
            else rhs = stencil<R, KIND, H>(win, op) * op.inv_dh;
        } else {
            rhs = headr[r];
        }
        process(r, rhs);
        advance(r);
    }
    for (int n = H; n < N - H; n++) {
        R rhs = stencil<R, KIND, H>(win, op) * op.inv_dh;
        process(n, rhs);
        advance(n);
    }
#pragma unroll
    for (int r = 0; r < H; r++) {
        int n = N - H + r;
        R rhs;
        if (PER) {
            if (KIND == K_EXPL_PER && r == H - 1) rhs = stencil_mirror<R, KIND, H>(win, op) * op.inv_dh;
            else rhs = stencil<R, KIND, H>(win, op) * op.inv_dh;
        } else {
            rhs = tailr[H - 1 - r];
        }
        process(n, rhs);
        if (r < H - 1) advance(n);
    }

    if (TRI) {
        // backward substitution (src/Utils.cpp:16-19)
        R x = col[(N - 1) * SP] * ldc(op.a1 + (N - 1));
        col[(N - 1) * SP] = x;
        const R xN1 = x;
        for (int n = N - 2; n >= 0; n--) {
            x = (col[n * SP] - ldc(op.a2 + n) * x) * ldc(op.a1 + n);
            col[n * SP] = x;
        }
        if (PER) {
            // Sherman-Morrison (src/Utils.cpp:43-45)
            R fact = (x + op.sc[0] * xN1 * op.sc[1]) * op.sc[2];
            for (int n = 0; n < N; n++) col[n * SP] -= fact * ldc(op.a3 + n);
        }
    } else if (PEN) {
        // backward substitution (src/Utils.cpp:75-82)
        R x1 = col[(N - 1) * SP] * ldc(op.a2 + (N - 1));
        R x2 = (col[(N - 2) * SP] - ldc(op.a3 + (N - 2)) * x1) * ldc(op.a2 + (N - 2));
        col[(N - 1) * SP] = x1;
        col[(N - 2) * SP] = x2;
        const R yN1 = x1, yN2 = x2;
        R xa = x2, xb = x1;   // x[n+1], x[n+2]
        for (int n = N - 3; n >= 0; n--) {
            R x = (col[n * SP] - ldc(op.a4 + n) * xb - ldc(op.a3 + n) * xa) * ldc(op.a2 + n);
            col[n * SP] = x;
            xb = xa;
            xa = x;
        }
        if (PER) {
            // Woodbury correction (src/Utils.cpp:158-190)
            const R y0 = xa, y1 = xb;
            R r0 = op.cp[0] * yN2 + op.cp[1] * yN1;
            R r1 = op.cp[2] * yN1;
            R r2 = op.cp[3] * y0;
            R r3 = op.cp[4] * y0 + op.cp[5] * y1;
            R s0 = op.Hm[0] * r0 + op.Hm[1] * r1 + op.Hm[2] * r2 + op.Hm[3] * r3;
            R s1 = op.Hm[4] * r0 + op.Hm[5] * r1 + op.Hm[6] * r2 + op.Hm[7] * r3;
            R s2 = op.Hm[8] * r0 + op.Hm[9] * r1 + op.Hm[10] * r2 + op.Hm[11] * r3;
            R s3 = op.Hm[12] * r0 + op.Hm[13] * r1 + op.Hm[14] * r2 + op.Hm[15] * r3;
            for (int n = 0; n < N; n++) {
                R sum = ldc(op.z0 + n) * s0 + ldc(op.z1 + n) * s1 + ldc(op.z2 + n) * s2 + ldc(op.z3 + n) * s3;
                col[n * SP] -= sum;
            }
        }
    }
}

// ---------------------------------------------------------------------------
// epilogue
// ---------------------------------------------------------------------------
template <typename R>
__device__ __forceinline__ void epi_apply(int epi, const SweepBatch<R> &b, const RhsFinalArgs<R> &rf, int f,
                                          long long idx, R v) {
    switch (epi) {
        case EPI_STORE: b.out[f][idx] = v; break;
        case EPI_STORE_NEG: b.out[f][idx] = -v; break;
        case EPI_SUB: b.out[f][idx] -= v; break;
        case EPI_STORE_F64: b.out64[f][idx] = (double)v; break;
        case EPI_RHS_FINAL: {
            // solveContinuity .. solveEnergy (src/CurvilinearCSolver_Core.cpp:790-947)
            // with zero sponge and zero hook sources: (src)/J == 0.
            R t = b.aux[f][idx] - v;
            R J = rf.J ? rf.J[idx] : rf.Jc;
            R dtJ = (R)(*rf.dt) * J;
            int e = b.eq[f];
            R k2;
            if (e >= 1 && e <= 3 && rf.quirk) k2 = (b.out[f][idx] + t) * dtJ;
            else k2 = t * dtJ;
            b.out[f][idx] = k2;
            break;
        }
    }
}

template <int DIR, typename R, int KIND, int H>
__global__ void __launch_bounds__(32) sweep_kernel(Grid3 g, LineOpDev<R> op, SweepBatch<R> b, int epi,
                                                   RhsFinalArgs<R> rf, int pass_y, int pass_z, int pass_x) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    R *s = reinterpret_cast<R *>(smem_raw);
    const int lane = threadIdx.x;
    const int tile = blockIdx.x;
    const int f = blockIdx.y;
    const int N = op.N;
    const R *in = b.in[f];
    TileGeom t = tile_geom<DIR>(g, tile, lane);

    // ---- load (coalesced) into s[n][lane] ----
    int nl = W;   // lines in this tile (DIR 0 / 2 may be partial)
    if (DIR == 0) {
        long long nlines = (long long)g.Ny * g.Nz;
        long long rem = nlines - (long long)tile * W;
        nl = rem < W ? (int)rem : W;
        const R *src = in + (long long)tile * W * N;
        int tot = nl * N;
        int q = lane / N, r = lane % N;   // e = lane + 32*it -> (q, r) = divmod(e, N)
        for (int e = lane; e < tot; e += 32) {
            cp_async_elem(&s[r * SP + q], src + e);
            r += 32;
            while (r >= N) { r -= N; q++; }
        }
    } else {
        if (t.active) {
            for (int n = 0; n < N; n++) cp_async_elem(&s[n * SP + lane], in + t.base + (long long)n * t.stride);
        }
    }
    cp_async_wait_all();
    __syncwarp();
    // wrap rows N .. N+H-1: periodic copy of rows 0..H-1, zero for Dirichlet
    if (t.active) {
        constexpr bool PER = (KIND % 2) == 0;
#pragma unroll
        for (int h = 0; h < H; h++) s[(N + h) * SP + lane] = PER ? s[h * SP + lane] : R(0);
    }
    __syncwarp();

    // ---- solve ----
    bool pass = false;
    if (DIR == 0) pass = (pass_y && (t.j == 0 || t.j == g.Ny - 1)) || (pass_z && (t.k == 0 || t.k == g.Nz - 1));
    if (DIR == 1) pass = (pass_x && (t.i == 0 || t.i == g.Nx - 1)) || (pass_z && (t.k == 0 || t.k == g.Nz - 1));
    if (DIR == 2) pass = (pass_y && (t.j == 0 || t.j == g.Ny - 1)) || (pass_x && (t.i == 0 || t.i == g.Nx - 1));
    if (t.active && !pass) solve_line<R, KIND, H>(s + lane, op);
    __syncwarp();

    // ---- epilogue (coalesced) ----
    if (DIR == 0) {
        long long off = (long long)tile * W * N;
        int tot = nl * N;
        int q = lane / N, r = lane % N;
        for (int e = lane; e < tot; e += 32) {
            epi_apply<R>(epi, b, rf, f, off + e, s[r * SP + q]);
            r += 32;
            while (r >= N) { r -= N; q++; }
        }
    } else {
        if (t.active) {
#pragma unroll 4
            for (int n = 0; n < N; n++) epi_apply<R>(epi, b, rf, f, t.base + (long long)n * t.stride, s[n * SP + lane]);
        }
    }
}

template <int DIR, typename R, int KIND, int H>
static int launch_one(const Grid3 &g, const LineOpDev<R> &op, const SweepBatch<R> &b, int epi,
                      const RhsFinalArgs<R> &rf, int px, int py, int pz, cudaStream_t st) {
    size_t smem = (size_t)(op.N + H) * SP * sizeof(R);
    auto kern = sweep_kernel<DIR, R, KIND, H>;
    static thread_local int configured_smem = -1;
    if ((int)smem > configured_smem) {
        MC3D_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        configured_smem = (int)smem;
    }
    int tiles;
    if (DIR == 0) tiles = (int)(((long long)g.Ny * g.Nz + W - 1) / W);
    else if (DIR == 1) tiles = ((g.Nx + W - 1) / W) * g.Nz;
    else tiles = (int)(((long long)g.Nx * g.Ny + W - 1) / W);
    dim3 grid(tiles, b.nf);
    kern<<<grid, 32, smem, st>>>(g, op, b, epi, rf, py, pz, px);
    MC3D_CUDA_TRY(cudaGetLastError());
    return MC3D_OK;
}

template <int DIR, typename R>
static int dispatch_kind(const Grid3 &g, const LineOpDev<R> &op, const SweepBatch<R> &b, int epi,
                         const RhsFinalArgs<R> &rf, int px, int py, int pz, cudaStream_t st) {
#define MC3D_CASE(K, HH) \
    if (op.kind == K && op.H == HH) return launch_one<DIR, R, K, HH>(g, op, b, epi, rf, px, py, pz, st);
    MC3D_CASE(K_TRI_PER, 2)   // Pade6 periodic
    MC3D_CASE(K_TRI_DIR, 2)   // Pade6 Dirichlet
    MC3D_CASE(K_PEN_PER, 3)   // Penta10 periodic
    MC3D_CASE(K_PEN_DIR, 3)   // Penta10 Dirichlet
    MC3D_CASE(K_EXPL_PER, 1)  // CD2 periodic
    MC3D_CASE(K_EXPL_DIR, 1)  // CD2 Dirichlet
    MC3D_CASE(K_TRI_PER, 4)   // Compact8 periodic
    MC3D_CASE(K_TRI_DIR, 4)   // Compact8 Dirichlet
    MC3D_CASE(K_TRI_PER, 5)   // Compact10 periodic
    MC3D_CASE(K_TRI_DIR, 5)   // Compact10 Dirichlet
#undef MC3D_CASE
    return fail(MC3D_ERR_CONFIG, "no line-solve kernel for this operator");
}

template <typename R>
int launch_sweep(int dir, const Grid3 &g, const LineOpDev<R> &op, const SweepBatch<R> &b, int epi,
                 const RhsFinalArgs<R> &rf, const int bc_types[3], bool filter_passthrough, cudaStream_t st) {
    if (b.nf <= 0) return MC3D_OK;
    if (b.nf > 16) return fail(MC3D_ERR_ARG, "at most 16 fields per sweep");
    size_t smem = (size_t)(op.N + op.H) * SP * sizeof(R);
    if (smem > 227 * 1024) return fail(MC3D_ERR_CONFIG, "line too long for the shared-memory tile");
    int px = filter_passthrough && bc_types[0] == MC3D_DIRICHLET_SOLVE;
    int py = filter_passthrough && bc_types[1] == MC3D_DIRICHLET_SOLVE;
    int pz = filter_passthrough && bc_types[2] == MC3D_DIRICHLET_SOLVE;
    if (dir == 0) return dispatch_kind<0, R>(g, op, b, epi, rf, px, py, pz, st);
    if (dir == 1) return dispatch_kind<1, R>(g, op, b, epi, rf, px, py, pz, st);
    return dispatch_kind<2, R>(g, op, b, epi, rf, px, py, pz, st);
}

template int launch_sweep<float>(int, const Grid3 &, const LineOpDev<float> &, const SweepBatch<float> &, int,
                                 const RhsFinalArgs<float> &, const int[3], bool, cudaStream_t);
template int launch_sweep<double>(int, const Grid3 &, const LineOpDev<double> &, const SweepBatch<double> &, int,
                                  const RhsFinalArgs<double> &, const int[3], bool, cudaStream_t);

}  // namespace mc3d
