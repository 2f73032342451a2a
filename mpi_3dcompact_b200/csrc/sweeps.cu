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
#include <cstdint>
#include <cstdio>

#include "sweep_common.cuh"

namespace mc3d {

// ---------------------------------------------------------------------------
// per-line solve, in place on col[n * SP]. Rows N .. N+H-1 hold the periodic
// wrap copy of rows 0..H-1 (zeros on Dirichlet lines); the tile has UB more
// pad rows so blocked loads never leave it.
//
// Register blocking: every pass handles UB rows at a time and issues all of
// the block's shared-memory and coefficient loads before the block's
// dependent FMA chain, so the per-row latency is one FMA, not one load.
// The periodic (Sherman-Morrison / Woodbury) correction is returned as up to
// four per-line scalars and applied in the epilogue.
// ---------------------------------------------------------------------------

template <int H, typename R>
__device__ __forceinline__ R win_at(const R (&w)[2 * H], const R (&in)[UB], int j) {
    return j < 2 * H ? w[j] : in[j - 2 * H];
}

template <typename R, int KIND, int H>
__device__ __forceinline__ void solve_line(R *col, const LineOpDev<R> &op, R corr[4]) {
    constexpr bool PER = (KIND % 2) == 0;
    constexpr bool TRI = KIND == K_TRI_PER || KIND == K_TRI_DIR;
    constexpr bool PEN = KIND == K_PEN_PER || KIND == K_PEN_DIR;
    const int N = op.N;

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
    // window phi[n0-H .. n0+H-1] for n0 = 0
    R w[2 * H];
#pragma unroll
    for (int k = 0; k < 2 * H; k++) {
        int idx = k - H;
        if (idx < 0) w[k] = PER ? col[(idx + N) * SP] : R(0);
        else w[k] = col[idx * SP];
    }

    // ---- pass 1: RHS stencil + forward elimination ----
    R xp = 0, xpp = 0;
    for (int n0 = 0; n0 < N; n0 += UB) {
        R in[UB], ca[UB], cb[UB], rhs[UB];
#pragma unroll
        for (int u = 0; u < UB; u++) in[u] = col[(n0 + H + u) * SP];
        const bool stat = n0 >= op.stat_lo && n0 + UB <= op.stat_hi;   // uniform across the warp
        if (stat) {
#pragma unroll
            for (int u = 0; u < UB; u++) {
                ca[u] = op.stat_c[0];
                cb[u] = op.stat_c[1];
            }
        } else {
#pragma unroll
            for (int u = 0; u < UB; u++) {
                int n = n0 + u;
                ca[u] = (TRI || PEN) && n < N ? ldc(op.a0 + n) : R(0);
                cb[u] = PEN && n >= 2 && n < N ? ldc(op.a1 + (n - 1)) : R(0);
            }
        }
#pragma unroll
        for (int u = 0; u < UB; u++) {
            R acc = op.st[0] * win_at<H>(w, in, u);
#pragma unroll
            for (int k = 1; k < 2 * H + 1; k++) acc += op.st[k] * win_at<H>(w, in, u + k);
            rhs[u] = acc * op.inv_dh;
            int n = n0 + u;
            if (!PER) {
#pragma unroll
                for (int r = 0; r < H; r++) {
                    if (n == r) rhs[u] = headr[r];
                    if (n == N - 1 - r) rhs[u] = tailr[r];
                }
            } else if (KIND == K_EXPL_PER) {
                // the reference's periodic CD2 end rows use the mirrored pair (src/CD2.cpp:131-132)
                if (n == 0 || n == N - 1) {
                    R m = op.st[2 * H] * win_at<H>(w, in, u);
#pragma unroll
                    for (int k = 1; k < 2 * H + 1; k++) m += op.st[2 * H - k] * win_at<H>(w, in, u + k);
                    rhs[u] = m * op.inv_dh;
                }
            }
        }
#pragma unroll
        for (int u = 0; u < UB; u++) {
            int n = n0 + u;
            R x;
            if (TRI) {
                x = (n == 0) ? rhs[u] : rhs[u] - ca[u] * xp;
                xp = x;
            } else if (PEN) {
                x = rhs[u];
                if (n >= 2) x -= cb[u] * xpp;
                if (n >= 1) x -= ca[u] * xp;
                xpp = xp;
                xp = x;
            } else {
                x = rhs[u];
            }
            if (n < N) col[n * SP] = x;
        }
#pragma unroll
        for (int k = 0; k < 2 * H; k++) w[k] = win_at<H>(w, in, UB + k);
    }

    corr[0] = corr[1] = corr[2] = corr[3] = R(0);
    if (!(TRI || PEN)) return;

    // ---- pass 2: backward substitution (src/Utils.cpp:16-19, :75-82) ----
    R xa = 0, xb = 0;   // x[n+1], x[n+2] (zero beyond the line end)
    R xN1 = 0, xN2 = 0;
    for (int n1 = N - 1; n1 >= 0; n1 -= UB) {
        R bb[UB], c1[UB], c2[UB], rr[UB];
        const bool stat = n1 - UB + 1 >= op.stat_lo && n1 < op.stat_hi;
#pragma unroll
        for (int u = 0; u < UB; u++) {
            int n = n1 - u;
            bool ok = n >= 0;
            bb[u] = ok ? col[n * SP] : R(0);
            if (stat) {
                c1[u] = TRI ? op.stat_c[2] : op.stat_c[3];
                c2[u] = TRI ? R(0) : op.stat_c[4];
                rr[u] = TRI ? op.stat_c[1] : op.stat_c[2];
            } else if (TRI) {
                c1[u] = ok ? ldc(op.a2 + n) : R(0);   // upper band c
                rr[u] = ok ? ldc(op.a1 + n) : R(0);   // 1/pivot
                c2[u] = R(0);
            } else {
                c1[u] = ok ? ldc(op.a3 + n) : R(0);   // modified first upper band C
                c2[u] = ok ? ldc(op.a4 + n) : R(0);   // second upper band f
                rr[u] = ok ? ldc(op.a2 + n) : R(0);   // 1/pivot
            }
        }
#pragma unroll
        for (int u = 0; u < UB; u++) {
            int n = n1 - u;
            R x;
            if (TRI) x = (bb[u] - c1[u] * xa) * rr[u];
            else x = (bb[u] - c2[u] * xb - c1[u] * xa) * rr[u];
            if (n >= 0) {
                col[n * SP] = x;
                if (n == N - 1) xN1 = x;
                if (n == N - 2) xN2 = x;
                xb = xa;
                xa = x;
            }
        }
    }
    if (KIND == K_TRI_PER) {
        // Sherman-Morrison factor (src/Utils.cpp:43): x[0] = xa
        corr[0] = (xa + op.sc[0] * xN1 * op.sc[1]) * op.sc[2];
    } else if (KIND == K_PEN_PER) {
        // Woodbury (src/Utils.cpp:158-181): r = V y, s = H r; y0 = xa, y1 = xb
        R r0 = op.cp[0] * xN2 + op.cp[1] * xN1;
        R r1 = op.cp[2] * xN1;
        R r2 = op.cp[3] * xa;
        R r3 = op.cp[4] * xa + op.cp[5] * xb;
        corr[0] = op.Hm[0] * r0 + op.Hm[1] * r1 + op.Hm[2] * r2 + op.Hm[3] * r3;
        corr[1] = op.Hm[4] * r0 + op.Hm[5] * r1 + op.Hm[6] * r2 + op.Hm[7] * r3;
        corr[2] = op.Hm[8] * r0 + op.Hm[9] * r1 + op.Hm[10] * r2 + op.Hm[11] * r3;
        corr[3] = op.Hm[12] * r0 + op.Hm[13] * r1 + op.Hm[14] * r2 + op.Hm[15] * r3;
    }
}

// periodic correction of element n (src/Utils.cpp:45 and :183-190)
template <typename R, int KIND>
__device__ __forceinline__ R corrected(R x, int n, const LineOpDev<R> &op, const R c[4]) {
    if (n >= op.corr_lo && n < op.corr_hi) return x;   // columns below 2^-64 of their peak
    if (KIND == K_TRI_PER) return x - c[0] * ldc(op.a3 + n);
    if (KIND == K_PEN_PER) {
        R sum = ldc(op.z0 + n) * c[0] + ldc(op.z1 + n) * c[1] + ldc(op.z2 + n) * c[2] + ldc(op.z3 + n) * c[3];
        return x - sum;
    }
    return x;
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

// Row loop of the strided-direction epilogue, one copy per mode, with the
// row address advanced by the line stride.
template <typename R, int KIND, int E>
__device__ __forceinline__ void epi_rows_t(const SweepBatch<R> &b, const RhsFinalArgs<R> &rf, int f, long long base,
                                           long long stride, const R *col, const LineOpDev<R> &op, const R corr[4]) {
    const int N = op.N;
    R *__restrict__ o = (E == EPI_STORE_F64) ? nullptr : b.out[f] + base;
    double *__restrict__ o64 = (E == EPI_STORE_F64) ? b.out64[f] + base : nullptr;
    const R *__restrict__ a = (E == EPI_RHS_FINAL) ? b.aux[f] + base : nullptr;
    const R *__restrict__ Jp = (E == EPI_RHS_FINAL && rf.J) ? rf.J + base : nullptr;
    R dt = (E == EPI_RHS_FINAL) ? (R)(*rf.dt) : R(0);
    const bool mom = (E == EPI_RHS_FINAL) && rf.quirk && b.eq[f] >= 1 && b.eq[f] <= 3;
#pragma unroll 4
    for (int n = 0; n < N; n++) {
        long long off = (long long)n * stride;
        R v = corrected<R, KIND>(col[n * SP], n, op, corr);
        if (E == EPI_STORE) o[off] = v;
        if (E == EPI_STORE_NEG) o[off] = -v;
        if (E == EPI_SUB) o[off] = o[off] - v;
        if (E == EPI_STORE_F64) o64[off] = (double)v;
        if (E == EPI_RHS_FINAL) {
            // solveContinuity .. solveEnergy (src/CurvilinearCSolver_Core.cpp:790-947)
            R t = a[off] - v;
            R dtJ = dt * (Jp ? Jp[off] : rf.Jc);
            o[off] = mom ? (o[off] + t) * dtJ : t * dtJ;
        }
    }
}

template <typename R, int KIND>
__device__ __forceinline__ void epi_rows(int epi, const SweepBatch<R> &b, const RhsFinalArgs<R> &rf, int f,
                                         long long base, long long stride, const R *col, const LineOpDev<R> &op,
                                         const R corr[4]) {
    switch (epi) {
        case EPI_STORE: epi_rows_t<R, KIND, EPI_STORE>(b, rf, f, base, stride, col, op, corr); break;
        case EPI_STORE_NEG: epi_rows_t<R, KIND, EPI_STORE_NEG>(b, rf, f, base, stride, col, op, corr); break;
        case EPI_SUB: epi_rows_t<R, KIND, EPI_SUB>(b, rf, f, base, stride, col, op, corr); break;
        case EPI_STORE_F64: epi_rows_t<R, KIND, EPI_STORE_F64>(b, rf, f, base, stride, col, op, corr); break;
        case EPI_RHS_FINAL: epi_rows_t<R, KIND, EPI_RHS_FINAL>(b, rf, f, base, stride, col, op, corr); break;
    }
}

template <int DIR, typename R, int KIND, int H>
__global__ void __launch_bounds__(32) sweep_kernel(Grid3 g, LineOpDev<R> op, SweepBatch<R> b, int epi,
                                                   RhsFinalArgs<R> rf, int pass_y, int pass_z, int pass_x) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int N = op.N;
    R *s = reinterpret_cast<R *>(smem_raw);
    R *scorr = s + (size_t)(N + H + UB) * SP;   // [W][4] per-line correction scalars
    const int lane = threadIdx.x;
    const int tile = blockIdx.x;
    const int f = blockIdx.y;
    const R *in = b.in[f];
    TileGeom t = tile_geom<DIR>(g, tile, lane);

    // ---- load (coalesced) into s[n][line] ----
    int nl = W;   // lines in this tile (DIR 0 / 2 may be partial)
    if (DIR == 0) {
        long long nlines = (long long)g.Ny * g.Nz;
        long long rem = nlines - (long long)tile * W;
        nl = rem < W ? (int)rem : W;
        const R *src = in + (long long)tile * W * N;
        for (int l = 0; l < nl; l++)
            for (int i = lane; i < N; i += 32) cp_async_elem(&s[i * SP + l], src + (long long)l * N + i);
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
    R corr[4] = {R(0), R(0), R(0), R(0)};
    if (t.active && !pass) solve_line<R, KIND, H>(s + lane, op, corr);

    // ---- epilogue (coalesced) ----
    if (DIR == 0) {
#pragma unroll
        for (int c = 0; c < 4; c++) scorr[lane * 4 + c] = corr[c];
        __syncwarp();
        long long off = (long long)tile * W * N;
        for (int l = 0; l < nl; l++) {
            R cl[4] = {scorr[l * 4 + 0], scorr[l * 4 + 1], scorr[l * 4 + 2], scorr[l * 4 + 3]};
            for (int i = lane; i < N; i += 32)
                epi_apply<R>(epi, b, rf, f, off + (long long)l * N + i, corrected<R, KIND>(s[i * SP + l], i, op, cl));
        }
    } else {
        __syncwarp();
        if (t.active) epi_rows<R, KIND>(epi, b, rf, f, t.base, t.stride, s + lane, op, corr);
    }
}

template <int DIR, typename R, int KIND, int H>
static int launch_one(const Grid3 &g, const LineOpDev<R> &op, const SweepBatch<R> &b, int epi,
                      const RhsFinalArgs<R> &rf, int px, int py, int pz, cudaStream_t st) {
    size_t smem = ((size_t)(op.N + H + UB) * SP + 4 * W) * sizeof(R);
    auto kern = sweep_kernel<DIR, R, KIND, H>;
    static KernelLaunchState ls;
    if (int rc = open_kernel(kern, ls, smem, 0, nullptr)) return rc;
    int tiles;
    if (DIR == 0) tiles = (int)(((long long)g.Ny * g.Nz + W - 1) / W);
    else if (DIR == 1) tiles = ((g.Nx + W - 1) / W) * g.Nz;
    else tiles = (int)(((long long)g.Nx * g.Ny + W - 1) / W);
    dim3 grid(tiles, b.nf);
    kern<<<grid, 32, smem, st>>>(g, op, b, epi, rf, py, pz, px);
    MC3D_CUDA_TRY(cudaGetLastError());
    return MC3D_OK;
}

// ---------------------------------------------------------------------------
// Segmented line solve: one CTA of S warps per tile of W lines; warp w owns
// rows [w L, (w+1) L) of every line (L = N/S), staged in its own shared-memory
// region with H halo rows on each side. Each warp runs the local RHS + forward
// elimination with zero incoming state, the S per-line segment states are
// chained (sequential over S, using the precomputed homogeneous responses),
// the local backward substitution folds in the forward superposition, the
// backward states are chained the same way, and the epilogue folds in the
// backward superposition and the cyclic correction. Dependency chains are S
// times shorter and S times more warps share each tile than in sweep_kernel.
//
// Row pitch: x-lines (DIR 0) are transposed on load into rows of W+1 words
// (bank-conflict-free scatter); strided lines (DIR 1, 2) are 128-byte rows of
// W words filled with 16-byte asynchronous copies when the field is aligned.
// ---------------------------------------------------------------------------
template <int DIR>
constexpr int seg_pitch() { return DIR == 0 ? W + 1 : W; }

template <typename R>
__device__ __forceinline__ void cp_async_16(R *dst, const R *src) {
    unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src) : "memory");
}

// strided-direction epilogue of one warp's segment rows, in blocks of UB rows
template <typename R, int KIND, int E, int P>
__device__ __forceinline__ void seg_epi_rows(const SweepBatch<R> &b, const RhsFinalArgs<R> &rf, int f, long long base,
                                             long long stride, const R *col, int a, int L, int kb,
                                             const LineOpDev<R> &op, const R corr[4], R Y1, R Y2, bool fold) {
    R *__restrict__ o = (E == EPI_STORE_F64) ? nullptr : b.out[f] + base + (long long)a * stride;
    double *__restrict__ o64 = (E == EPI_STORE_F64) ? b.out64[f] + base + (long long)a * stride : nullptr;
    const R *__restrict__ ax = (E == EPI_RHS_FINAL) ? b.aux[f] + base + (long long)a * stride : nullptr;
    const R *__restrict__ Jp = (E == EPI_RHS_FINAL && rf.J) ? rf.J + base + (long long)a * stride : nullptr;
    R dt = (E == EPI_RHS_FINAL) ? (R)(*rf.dt) : R(0);
    const bool mom = (E == EPI_RHS_FINAL) && rf.quirk && b.eq[f] >= 1 && b.eq[f] <= 3;
    const int fold_from = fold ? L - kb : L;   // rows of the segment carrying the backward superposition
    for (int r0 = 0; r0 < L; r0 += UB) {
        const bool fb = r0 + UB > fold_from;
        const bool cw = a + r0 >= op.corr_lo && a + r0 + UB <= op.corr_hi;   // inside the no-correction window
        R v[UB], t[UB], jj[UB], old[UB];
#pragma unroll
        for (int u = 0; u < UB; u++) {
            int r = r0 + u, n = a + r;
            v[u] = col[r * P];
            if (fb && r >= fold_from) v[u] += ldc(op.sba + n) * Y1 + ldc(op.sbb + n) * Y2;
            if (!cw) v[u] = corrected<R, KIND>(v[u], n, op, corr);
            long long off = (long long)r * stride;
            if (E == EPI_RHS_FINAL) {
                t[u] = ax[off];
                jj[u] = Jp ? Jp[off] : rf.Jc;
                old[u] = mom ? o[off] : R(0);
            } else if (E == EPI_SUB) {
                old[u] = o[off];
            }
        }
#pragma unroll
        for (int u = 0; u < UB; u++) {
            long long off = (long long)(r0 + u) * stride;
            if (E == EPI_STORE) o[off] = v[u];
            if (E == EPI_STORE_NEG) o[off] = -v[u];
            if (E == EPI_SUB) o[off] = old[u] - v[u];
            if (E == EPI_STORE_F64) o64[off] = (double)v[u];
            if (E == EPI_RHS_FINAL) {
                // solveContinuity .. solveEnergy (src/CurvilinearCSolver_Core.cpp:790-947)
                R tt = t[u] - v[u];
                R dtJ = dt * jj[u];
                o[off] = mom ? (old[u] + tt) * dtJ : tt * dtJ;
            }
        }
    }
}

// x-direction epilogue: warp `seg` streams its rows of every line, lanes along x
template <typename R, int KIND, int E, int P, int H_OF_REG>
__device__ __forceinline__ void seg_epi_x(const SweepBatch<R> &b, const RhsFinalArgs<R> &rf, int f, long long off0,
                                          int N, const R *reg, int a, int L, int kb, int nl, const R *scorr,
                                          const R *Yb, const LineOpDev<R> &op, bool fold, int lane) {
    R dt = (E == EPI_RHS_FINAL) ? (R)(*rf.dt) : R(0);
    const bool mom = (E == EPI_RHS_FINAL) && rf.quirk && b.eq[f] >= 1 && b.eq[f] <= 3;
    const int fold_from = fold ? L - kb : L;
    for (int l = 0; l < nl; l++) {
        R cl[4] = {scorr[l * 4 + 0], scorr[l * 4 + 1], scorr[l * 4 + 2], scorr[l * 4 + 3]};
        R Y1 = Yb[l], Y2 = Yb[W + l];
        long long lo = off0 + (long long)l * N + a;
        for (int r = lane; r < L; r += 32) {
            int n = a + r;
            R v = reg[(H_OF_REG + r) * P + l];
            if (r >= fold_from) v += ldc(op.sba + n) * Y1 + ldc(op.sbb + n) * Y2;
            v = corrected<R, KIND>(v, n, op, cl);
            long long idx = lo + r;
            if (E == EPI_STORE) b.out[f][idx] = v;
            if (E == EPI_STORE_NEG) b.out[f][idx] = -v;
            if (E == EPI_SUB) b.out[f][idx] -= v;
            if (E == EPI_STORE_F64) b.out64[f][idx] = (double)v;
            if (E == EPI_RHS_FINAL) {
                R tt = b.aux[f][idx] - v;
                R dtJ = dt * (rf.J ? rf.J[idx] : rf.Jc);
                b.out[f][idx] = mom ? (b.out[f][idx] + tt) * dtJ : tt * dtJ;
            }
        }
    }
}

template <int DIR, typename R, int KIND, int H, int S>
__global__ void __launch_bounds__(32 * S) sweep_seg_kernel(Grid3 g, LineOpDev<R> op, SweepBatch<R> b, int epi,
                                                           RhsFinalArgs<R> rf, int pass_y, int pass_z, int pass_x,
                                                           int vec16) {
    constexpr bool PER = (KIND % 2) == 0;
    constexpr bool TRI = KIND == K_TRI_PER || KIND == K_TRI_DIR;
    constexpr int P = seg_pitch<DIR>();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int N = op.N, L = N / S;
    const int RG = L + 2 * H + UB;   // rows per segment region (UB keeps regions 16-byte aligned)
    R *s = reinterpret_cast<R *>(smem_raw);
    R *fwdEnd = s + (size_t)S * RG * P;   // [S][2][W]
    R *fwdIn = fwdEnd + S * 2 * W;
    R *bwdStart = fwdIn + S * 2 * W;
    R *bwdNext = bwdStart + S * 2 * W;
    R *scorr = bwdNext + S * 2 * W;       // [W][4]
    const int lane = threadIdx.x & 31, seg = threadIdx.x >> 5;
    const int tile = blockIdx.x, f = blockIdx.y;
    const int a = seg * L, bEnd = a + L;
    const R *in = b.in[f];
    TileGeom t = tile_geom<DIR>(g, tile, lane);
    R *reg = s + (size_t)seg * RG * P;    // this warp's segment region
    R *col = reg + lane;                  // ... line `lane`

    // ---- load: warp `seg` brings its own rows of every line ----
    int nl = W;
    if (DIR == 0) {
        long long rem = (long long)g.Ny * g.Nz - (long long)tile * W;
        nl = rem < W ? (int)rem : W;
        const R *src = in + (long long)tile * W * N;
        for (int l = 0; l < nl; l++)
            for (int i = a + lane; i < bEnd; i += 32) cp_async_elem(&reg[(H + i - a) * P + l], src + (long long)l * N + i);
    } else if (vec16) {
        // 16-byte chunks of 128-byte rows: CPR chunks per row, 32/CPR rows per pass
        constexpr int EPC = 16 / sizeof(R), CPR = W / EPC, RPP = 32 / CPR;
        TileGeom t0 = tile_geom<DIR>(g, tile, 0);
        long long nvalid = DIR == 1 ? (long long)g.Nx - t0.i : (long long)g.Nx * g.Ny - (long long)tile * W;
        const int c = lane % CPR;
        if (c * EPC < nvalid)
            for (int r = lane / CPR; r < L; r += RPP)
                cp_async_16(&reg[(H + r) * P + c * EPC], in + t0.base + (long long)(a + r) * t0.stride + c * EPC);
    } else if (t.active) {
        for (int n = a; n < bEnd; n++) cp_async_elem(&col[(H + n - a) * P], in + t.base + (long long)n * t.stride);
    }
    cp_async_wait_all();
    __syncthreads();
    // halos: rows a-H..a-1 and b..b+H-1 (periodic wrap, zero beyond a Dirichlet end)
    if (t.active) {
        const int prev = (seg + S - 1) % S, next = (seg + 1) % S;
        const R *pr = s + (size_t)prev * RG * P + lane, *nx = s + (size_t)next * RG * P + lane;
#pragma unroll
        for (int h = 0; h < H; h++) {
            col[h * P] = (PER || seg > 0) ? pr[(L + h) * P] : R(0);
            col[(H + L + h) * P] = (PER || seg < S - 1) ? nx[(H + h) * P] : R(0);
        }
    }
    bool pass = false;
    if (DIR == 0) pass = (pass_y && (t.j == 0 || t.j == g.Ny - 1)) || (pass_z && (t.k == 0 || t.k == g.Nz - 1));
    if (DIR == 1) pass = (pass_x && (t.i == 0 || t.i == g.Nx - 1)) || (pass_z && (t.k == 0 || t.k == g.Nz - 1));
    if (DIR == 2) pass = (pass_y && (t.j == 0 || t.j == g.Ny - 1)) || (pass_x && (t.i == 0 || t.i == g.Nx - 1));
    const bool work = t.active && !pass;
    // Dirichlet boundary rows (first / last segment) read inputs the in-place sweep overwrites
    R headr[H], tailr[H];
    if (!PER && work) {
#pragma unroll
        for (int r = 0; r < H; r++) {
            R hsum = 0, tsum = 0;
            if (seg == 0)
                for (int k = 0; k < op.bw; k++) hsum += ldc(op.head + r * op.bw + k) * col[(H + k) * P];
            if (seg == S - 1)
                for (int k = 0; k < op.bw; k++) tsum += ldc(op.tail + r * op.bw + k) * col[(H + L - op.bw + k) * P];
            headr[r] = hsum * op.inv_dh;
            tailr[r] = tsum * op.inv_dh;
        }
    }
    __syncthreads();

    // ---- pass 1: RHS + local forward elimination (zero incoming state) ----
    R xp = 0, xpp = 0;
    if (work) {
        R w[2 * H];
#pragma unroll
        for (int k = 0; k < 2 * H; k++) w[k] = col[k * P];
        for (int n0 = a; n0 < bEnd; n0 += UB) {
            R inb[UB], rhs[UB];
#pragma unroll
            for (int u = 0; u < UB; u++) inb[u] = col[(n0 - a + 2 * H + u) * P];
#pragma unroll
            for (int u = 0; u < UB; u++) {
                R acc = op.st[0] * win_at<H>(w, inb, u);
#pragma unroll
                for (int k = 1; k < 2 * H + 1; k++) acc += op.st[k] * win_at<H>(w, inb, u + k);
                rhs[u] = acc * op.inv_dh;
            }
            const bool clean = n0 >= 2 && n0 >= op.stat_lo && n0 + UB <= op.stat_hi && (PER || n0 >= H) &&
                               (PER || n0 + UB <= N - H);
            if (clean) {
                // stationary interior: constant factors, no boundary rows
                const R ca = op.stat_c[0], cb = op.stat_c[1];
#pragma unroll
                for (int u = 0; u < UB; u++) {
                    R x = TRI ? rhs[u] - ca * xp : rhs[u] - cb * xpp - ca * xp;
                    xpp = xp;
                    xp = x;
                    col[(H + n0 - a + u) * P] = x;
                }
            } else {
#pragma unroll
                for (int u = 0; u < UB; u++) {
                    int n = n0 + u;
                    if (!PER) {
#pragma unroll
                        for (int r = 0; r < H; r++) {
                            if (n == r) rhs[u] = headr[r];
                            if (n == N - 1 - r) rhs[u] = tailr[r];
                        }
                    }
                    R ca = ldc(op.a0 + n);
                    R x;
                    if (TRI) {
                        x = (n == 0) ? rhs[u] : rhs[u] - ca * xp;
                    } else {
                        x = rhs[u];
                        if (n >= 2) x -= ldc(op.a1 + (n - 1)) * xpp;
                        if (n >= 1) x -= ca * xp;
                    }
                    xpp = xp;
                    xp = x;
                    col[(H + n - a) * P] = x;
                }
            }
#pragma unroll
            for (int k = 0; k < 2 * H; k++) w[k] = win_at<H>(w, inb, UB + k);
        }
    }
    fwdEnd[(seg * 2 + 0) * W + lane] = xp;    // local B_{b-1}
    fwdEnd[(seg * 2 + 1) * W + lane] = xpp;   // local B_{b-2}
    __syncthreads();

    // ---- chain the forward states: final B_{a-1}, B_{a-2} of every segment ----
    if (seg == 0) {
        R X1 = 0, X2 = 0;
        fwdIn[lane] = 0;
        fwdIn[W + lane] = 0;
        for (int ws = 1; ws < S; ws++) {
            int e1 = ws * L - 1, e2 = e1 - 1;
            R n1 = fwdEnd[((ws - 1) * 2 + 0) * W + lane] + ldc(op.sfa + e1) * X1 + ldc(op.sfb + e1) * X2;
            R n2 = fwdEnd[((ws - 1) * 2 + 1) * W + lane] + ldc(op.sfa + e2) * X1 + ldc(op.sfb + e2) * X2;
            X1 = work ? n1 : R(0);
            X2 = work ? n2 : R(0);
            fwdIn[(ws * 2 + 0) * W + lane] = X1;
            fwdIn[(ws * 2 + 1) * W + lane] = X2;
        }
    }
    __syncthreads();

    // ---- pass 2: local backward substitution on the superposed RHS ----
    R xa = 0, xb = 0;
    if (work) {
        const R X1 = fwdIn[(seg * 2 + 0) * W + lane], X2 = fwdIn[(seg * 2 + 1) * W + lane];
        const int fold_to = seg > 0 ? a + op.seg_kf : a;   // rows [a, fold_to) carry the forward superposition
        for (int n1 = bEnd - 1; n1 >= a; n1 -= UB) {
            R bb[UB], c1[UB], c2[UB], rr[UB];
            const bool stat = n1 - UB + 1 >= op.stat_lo && n1 < op.stat_hi;
            const bool ff = n1 - UB + 1 < fold_to;
#pragma unroll
            for (int u = 0; u < UB; u++) {
                int n = n1 - u;
                bb[u] = col[(H + n - a) * P];
                if (ff && n < fold_to) bb[u] += ldc(op.sfa + n) * X1 + (TRI ? R(0) : ldc(op.sfb + n) * X2);
                if (stat) {
                    c1[u] = TRI ? op.stat_c[2] : op.stat_c[3];
                    c2[u] = TRI ? R(0) : op.stat_c[4];
                    rr[u] = TRI ? op.stat_c[1] : op.stat_c[2];
                } else if (TRI) {
                    c1[u] = ldc(op.a2 + n);
                    rr[u] = ldc(op.a1 + n);
                    c2[u] = R(0);
                } else {
                    c1[u] = ldc(op.a3 + n);
                    c2[u] = ldc(op.a4 + n);
                    rr[u] = ldc(op.a2 + n);
                }
            }
#pragma unroll
            for (int u = 0; u < UB; u++) {
                int n = n1 - u;
                R x = TRI ? (bb[u] - c1[u] * xa) * rr[u] : (bb[u] - c2[u] * xb - c1[u] * xa) * rr[u];
                col[(H + n - a) * P] = x;
                xb = xa;
                xa = x;
            }
        }
    }
    bwdStart[(seg * 2 + 0) * W + lane] = xa;   // local x_a
    bwdStart[(seg * 2 + 1) * W + lane] = xb;   // local x_{a+1}
    __syncthreads();

    // ---- chain the backward states; periodic correction scalars ----
    if (seg == 0) {
        R Y1 = 0, Y2 = 0;
        bwdNext[((S - 1) * 2 + 0) * W + lane] = 0;
        bwdNext[((S - 1) * 2 + 1) * W + lane] = 0;
        for (int ws = S - 2; ws >= 0; ws--) {
            int s0 = (ws + 1) * L;
            R n1 = bwdStart[((ws + 1) * 2 + 0) * W + lane] + ldc(op.sba + s0) * Y1 + ldc(op.sbb + s0) * Y2;
            R n2 = bwdStart[((ws + 1) * 2 + 1) * W + lane] + ldc(op.sba + s0 + 1) * Y1 + ldc(op.sbb + s0 + 1) * Y2;
            Y1 = work ? n1 : R(0);
            Y2 = work ? n2 : R(0);
            bwdNext[(ws * 2 + 0) * W + lane] = Y1;
            bwdNext[(ws * 2 + 1) * W + lane] = Y2;
        }
        R c[4] = {R(0), R(0), R(0), R(0)};
        if (work && PER) {
            // final x_0, x_1 (first segment, folded) and x_{N-1}, x_{N-2} (last segment)
            R x0 = bwdStart[0 * W + lane] + ldc(op.sba + 0) * Y1 + ldc(op.sbb + 0) * Y2;
            R x1 = bwdStart[1 * W + lane] + ldc(op.sba + 1) * Y1 + ldc(op.sbb + 1) * Y2;
            const R *last = s + (size_t)(S - 1) * RG * P + lane;
            R xN1 = last[(H + L - 1) * P], xN2 = last[(H + L - 2) * P];
            if (KIND == K_TRI_PER) {
                c[0] = (x0 + op.sc[0] * xN1 * op.sc[1]) * op.sc[2];
            } else {
                R r0 = op.cp[0] * xN2 + op.cp[1] * xN1;
                R r1 = op.cp[2] * xN1;
                R r2 = op.cp[3] * x0;
                R r3 = op.cp[4] * x0 + op.cp[5] * x1;
                c[0] = op.Hm[0] * r0 + op.Hm[1] * r1 + op.Hm[2] * r2 + op.Hm[3] * r3;
                c[1] = op.Hm[4] * r0 + op.Hm[5] * r1 + op.Hm[6] * r2 + op.Hm[7] * r3;
                c[2] = op.Hm[8] * r0 + op.Hm[9] * r1 + op.Hm[10] * r2 + op.Hm[11] * r3;
                c[3] = op.Hm[12] * r0 + op.Hm[13] * r1 + op.Hm[14] * r2 + op.Hm[15] * r3;
            }
        }
#pragma unroll
        for (int k = 0; k < 4; k++) scorr[lane * 4 + k] = c[k];
    }
    __syncthreads();

    // ---- epilogue: backward superposition, cyclic correction, output ----
    const bool fold = seg < S - 1;
    const int kb = op.seg_kb;
    if (DIR == 0) {
        long long off0 = (long long)tile * W * N;
        const R *Yb = bwdNext + seg * 2 * W;
#define MC3D_EPX(E) seg_epi_x<R, KIND, E, P, H>(b, rf, f, off0, N, reg, a, L, kb, nl, scorr, Yb, op, fold, lane)
        switch (epi) {
            case EPI_STORE: MC3D_EPX(EPI_STORE); break;
            case EPI_STORE_NEG: MC3D_EPX(EPI_STORE_NEG); break;
            case EPI_SUB: MC3D_EPX(EPI_SUB); break;
            case EPI_STORE_F64: MC3D_EPX(EPI_STORE_F64); break;
            case EPI_RHS_FINAL: MC3D_EPX(EPI_RHS_FINAL); break;
        }
#undef MC3D_EPX
    } else if (t.active) {
        R cl[4] = {scorr[lane * 4 + 0], scorr[lane * 4 + 1], scorr[lane * 4 + 2], scorr[lane * 4 + 3]};
        R Y1 = bwdNext[(seg * 2 + 0) * W + lane], Y2 = bwdNext[(seg * 2 + 1) * W + lane];
        const R *c0 = col + H * P;
#define MC3D_EPR(E) seg_epi_rows<R, KIND, E, P>(b, rf, f, t.base, t.stride, c0, a, L, kb, op, cl, Y1, Y2, fold)
        switch (epi) {
            case EPI_STORE: MC3D_EPR(EPI_STORE); break;
            case EPI_STORE_NEG: MC3D_EPR(EPI_STORE_NEG); break;
            case EPI_SUB: MC3D_EPR(EPI_SUB); break;
            case EPI_STORE_F64: MC3D_EPR(EPI_STORE_F64); break;
            case EPI_RHS_FINAL: MC3D_EPR(EPI_RHS_FINAL); break;
        }
#undef MC3D_EPR
    }
}

template <int S>
constexpr size_t seg_smem_elems(int N, int H, int P) {
    return (size_t)S * (N / S + 2 * H + UB) * P + 4 * S * 2 * W + 4 * W;
}

template <int DIR, typename R, int KIND, int H, int S>
static int launch_seg(const Grid3 &g, const LineOpDev<R> &op, const SweepBatch<R> &b, int epi,
                      const RhsFinalArgs<R> &rf, int px, int py, int pz, cudaStream_t st) {
    size_t smem = seg_smem_elems<S>(op.N, H, seg_pitch<DIR>()) * sizeof(R);
    auto kern = sweep_seg_kernel<DIR, R, KIND, H, S>;
    static KernelLaunchState ls;
    if (int rc = open_kernel(kern, ls, smem, 0, nullptr)) return rc;
    int tiles;
    if (DIR == 0) tiles = (int)(((long long)g.Ny * g.Nz + W - 1) / W);
    else if (DIR == 1) tiles = ((g.Nx + W - 1) / W) * g.Nz;
    else tiles = (int)(((long long)g.Nx * g.Ny + W - 1) / W);
    // 16-byte copies need 16-byte aligned rows: field bases and the line stride
    int vec16 = 0;
    if (DIR != 0) {
        const int epc = 16 / sizeof(R);
        long long inner = DIR == 1 ? g.Nx : (long long)g.Nx * g.Ny;
        vec16 = (inner % epc == 0);
        for (int f = 0; f < b.nf && vec16; f++) vec16 = ((uintptr_t)b.in[f] % 16) == 0;
    }
    dim3 grid(tiles, b.nf);
    kern<<<grid, 32 * S, smem, st>>>(g, op, b, epi, rf, py, pz, px, vec16);
    MC3D_CUDA_TRY(cudaGetLastError());
    return MC3D_OK;
}

template <int DIR, typename R>
static int dispatch_kind(const Grid3 &g, const LineOpDev<R> &op, const SweepBatch<R> &b, int epi,
                         const RhsFinalArgs<R> &rf, int px, int py, int pz, cudaStream_t st) {
#define MC3D_CASE(K, HH)                                                                             \
    if (op.kind == K && op.H == HH) {                                                                \
        if constexpr (K >= K_TRI_PER) {                                                              \
            if (op.S == 4) return launch_seg<DIR, R, K, HH, 4>(g, op, b, epi, rf, px, py, pz, st);   \
            if (op.S == 2) return launch_seg<DIR, R, K, HH, 2>(g, op, b, epi, rf, px, py, pz, st);   \
        }                                                                                            \
        return launch_one<DIR, R, K, HH>(g, op, b, epi, rf, px, py, pz, st);                         \
    }
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
    MC3D_CASE(K_PEN_PER, 5)   // DSM Pade test filter periodic
    MC3D_CASE(K_PEN_DIR, 5)   // DSM Pade test filter Dirichlet
    MC3D_CASE(K_EXPL_PER, 3)  // DSM explicit test filter periodic
    MC3D_CASE(K_EXPL_DIR, 3)  // DSM explicit test filter Dirichlet
#undef MC3D_CASE
    return fail(MC3D_ERR_CONFIG, "no line-solve kernel for this operator");
}

template <typename R>
int launch_sweep(int dir, const Grid3 &g, const LineOpDev<R> &op, const SweepBatch<R> &b, int epi,
                 const RhsFinalArgs<R> &rf, const int bc_types[3], bool filter_passthrough, cudaStream_t st) {
    if (b.nf <= 0) return MC3D_OK;
    if (b.nf > 16) return fail(MC3D_ERR_ARG, "at most 16 fields per sweep");
    int px = filter_passthrough && bc_types[0] == MC3D_DIRICHLET_SOLVE;
    int py = filter_passthrough && bc_types[1] == MC3D_DIRICHLET_SOLVE;
    int pz = filter_passthrough && bc_types[2] == MC3D_DIRICHLET_SOLVE;
    if (op.L > 0 && g.n() < (1LL << 31) &&   // register-resident kernels index fields with 32-bit offsets
        reg_smem_bytes(dir, op.N, op.N / op.L, sizeof(R)) <= 227 * 1024) {
        int rc = dir == 0 ? launch_sweep_reg<0, R>(g, op, b, epi, rf, px, py, pz, st)
                 : dir == 1 ? launch_sweep_reg<1, R>(g, op, b, epi, rf, px, py, pz, st)
                            : launch_sweep_reg<2, R>(g, op, b, epi, rf, px, py, pz, st);
        if (rc != MC3D_ERR_CONFIG) return rc;
    }
    size_t smem = ((size_t)(op.N + op.H + UB) * SP + 4 * W) * sizeof(R);
    if (op.S == 4) smem = seg_smem_elems<4>(op.N, op.H, W + 1) * sizeof(R);
    if (op.S == 2) smem = seg_smem_elems<2>(op.N, op.H, W + 1) * sizeof(R);
    if (smem > 227 * 1024) return fail(MC3D_ERR_CONFIG, "line too long for the shared-memory tile");
    if (dir == 0) return dispatch_kind<0, R>(g, op, b, epi, rf, px, py, pz, st);
    if (dir == 1) return dispatch_kind<1, R>(g, op, b, epi, rf, px, py, pz, st);
    return dispatch_kind<2, R>(g, op, b, epi, rf, px, py, pz, st);
}

template int launch_sweep<float>(int, const Grid3 &, const LineOpDev<float> &, const SweepBatch<float> &, int,
                                 const RhsFinalArgs<float> &, const int[3], bool, cudaStream_t);
template int launch_sweep<double>(int, const Grid3 &, const LineOpDev<double> &, const SweepBatch<double> &, int,
                                  const RhsFinalArgs<double> &, const int[3], bool, cudaStream_t);

}  // namespace mc3d
