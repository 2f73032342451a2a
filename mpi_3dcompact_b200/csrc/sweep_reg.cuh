// Register-resident segmented line solve.
//
// One CTA = S warps on a tile of W = 32 lines of one field; warp w owns rows
// [w L, (w+1) L) of every line (L = N/S, a compile-time 32 or 64) and each
// lane keeps its line's L rows, plus H halo rows on either side, in registers
// for the whole solve:
//   load      strided lines (y, z): one coalesced 128-byte row per warp load,
//             straight into registers; x lines: the tile is staged transposed
//             in shared memory once and each lane reads its line from there;
//   pass 1    RHS stencil from registers and the forward elimination with a
//             zero incoming state;
//   chain     warp 0 chains the S segment end states (host-computed
//             homogeneous responses at the segment ends);
//   fold      the incoming forward state is propagated through the segment's
//             first rows by the elimination's own recurrence (no per-row
//             response loads), while it is above the precision's cut-off;
//   pass 2    backward substitution with a zero incoming state;
//   chain     the backward states, then the cyclic correction scalars;
//   epilogue  the backward state is propagated up the segment by the
//             substitution's recurrence, the cyclic correction is applied in
//             the rows where its columns matter, and the caller's operation
//             (store, negate, accumulate, k2 assembly, FP64 store) is applied.
// Row factors come from row-interleaved copies (one vector load per row) and
// only in rows that are not on the Toeplitz fixed point.
//
// Reference loops this replaces: Pade6/Penta10::calc1stDerivField
// (src/Pade6.cpp:3-46, src/Penta10.cpp:3-47), Compact8/10Filter::filterField
// (src/Compact10Filter.cpp:166-252) with src/Utils.cpp:4-191 per line.
#pragma once
#include "sweep_common.cuh"

namespace mc3d {

template <typename R>
struct RegVec;
template <>
struct RegVec<float> {
    static __device__ __forceinline__ void ld2(const float *p, float &a, float &b) {
        float2 v = __ldg(reinterpret_cast<const float2 *>(p));
        a = v.x;
        b = v.y;
    }
    static __device__ __forceinline__ void ld4(const float *p, float &a, float &b, float &c, float &d) {
        float4 v = __ldg(reinterpret_cast<const float4 *>(p));
        a = v.x;
        b = v.y;
        c = v.z;
        d = v.w;
    }
};
template <>
struct RegVec<double> {
    static __device__ __forceinline__ void ld2(const double *p, double &a, double &b) {
        double2 v = __ldg(reinterpret_cast<const double2 *>(p));
        a = v.x;
        b = v.y;
    }
    static __device__ __forceinline__ void ld4(const double *p, double &a, double &b, double &c, double &d) {
        double2 v = __ldg(reinterpret_cast<const double2 *>(p));
        double2 w = __ldg(reinterpret_cast<const double2 *>(p) + 1);
        a = v.x;
        b = v.y;
        c = w.x;
        d = w.y;
    }
};

// strided lines: write this lane's L rows (row a + r at off0 + r * stride).
// Operands the operation reads (previous output, partial RHS, J) are loaded a
// block of UB rows ahead of the block being stored, in program order before
// those stores, so each block costs one memory round trip at most and the
// loads overlap the previous block's stores.
template <typename R, int E, int L, bool PREFETCH = true>
__device__ __forceinline__ void reg_store_rows(const SweepBatch<R> &b, const RhsFinalArgs<R> &rf, int f, int off0,
                                               int stride, const R (&y)[L]) {
    constexpr int NB = L / UB;
    constexpr bool RD_OLD = E == EPI_SUB || E == EPI_RHS_FINAL;   // RHS_FINAL: only momentum with the quirk
    constexpr bool RD_AUX = E == EPI_RHS_FINAL;
    const R dt = (E == EPI_RHS_FINAL) ? (R)(*rf.dt) : R(0);
    const bool mom = (E == EPI_RHS_FINAL) && rf.quirk && b.eq[f] >= 1 && b.eq[f] <= 3;
    const bool rd_old = E == EPI_SUB || mom;
    R *o = b.out[f];
    double *o64 = b.out64[f];
    const R *ax = b.aux[f];
    const R *jp = rf.J;
    // FP32: the next block's operands are fetched while this block is stored;
    // FP64 (twice the registers per value), or PREFETCH false: each block
    // fetches its own.
    constexpr bool AHEAD = PREFETCH && sizeof(R) == 4;
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
    if (AHEAD && (RD_OLD || RD_AUX)) fetch(0, 0);
#pragma unroll
    for (int blk = 0; blk < NB; blk++) {
        const int cur = AHEAD ? (blk & 1) : 0;
        if (AHEAD && (RD_OLD || RD_AUX) && blk + 1 < NB) fetch(blk + 1, cur ^ 1);
        if (!AHEAD && (RD_OLD || RD_AUX)) fetch(blk, 0);
#pragma unroll
        for (int u = 0; u < UB; u++) {
            const int r = blk * UB + u;
            const int off = off0 + r * stride;
            const R v = y[r];
            if (E == EPI_STORE) o[off] = v;
            if (E == EPI_STORE_NEG) o[off] = -v;
            if (E == EPI_SUB) o[off] = old[cur][u] - v;
            if (E == EPI_STORE_F64) o64[off] = (double)v;
            if (E == EPI_RHS_FINAL) {
                // solveContinuity .. solveEnergy (src/CurvilinearCSolver_Core.cpp:790-947)
                // with zero sponge and zero hook sources
                R tt = aux[cur][u] - v;
                R dtJ = dt * jj[cur][u];
                o[off] = mom ? (old[cur][u] + tt) * dtJ : tt * dtJ;
            }
        }
    }
}

// x lines: warp `seg` writes rows [a, a+L) of the tile's nl lines, lanes
// along x. The read operands of a group of lines are loaded before any of the
// group's stores.
template <typename R, int E, int L>
__device__ __forceinline__ void reg_copy_out(const SweepBatch<R> &b, const RhsFinalArgs<R> &rf, int f, int tile0,
                                             int N, int nl, int a, int lane, const R *tile) {
    constexpr int P = W + 1;
    constexpr int Q = L / 32;    // elements per lane and line
    constexpr int G = 8 / Q;     // lines per group: 8 elements per lane in flight
    constexpr bool RD_OLD = E == EPI_SUB || E == EPI_RHS_FINAL;
    constexpr bool RD_AUX = E == EPI_RHS_FINAL;
    const R dt = (E == EPI_RHS_FINAL) ? (R)(*rf.dt) : R(0);
    const bool mom = (E == EPI_RHS_FINAL) && rf.quirk && b.eq[f] >= 1 && b.eq[f] <= 3;
    const bool rd_old = E == EPI_SUB || mom;
    R *o = b.out[f];
    double *o64 = b.out64[f];
    const R *ax = b.aux[f];
    const R *jp = rf.J;
    for (int l0 = 0; l0 < nl; l0 += G) {
        R old[G][Q], aux[G][Q], jj[G][Q];
        if (RD_OLD || RD_AUX) {
#pragma unroll
            for (int gl = 0; gl < G; gl++) {
                if (l0 + gl < nl) {
                    const int line0 = (tile0 + l0 + gl) * N + a + lane;
#pragma unroll
                    for (int q = 0; q < Q; q++) {
                        const int off = line0 + 32 * q;
                        if (RD_OLD) old[gl][q] = rd_old ? o[off] : R(0);
                        if (RD_AUX) {
                            aux[gl][q] = ax[off];
                            jj[gl][q] = jp ? jp[off] : rf.Jc;
                        }
                    }
                }
            }
        }
#pragma unroll
        for (int gl = 0; gl < G; gl++) {
            if (l0 + gl < nl) {
                const int l = l0 + gl;
                const int line0 = (tile0 + l) * N + a + lane;
#pragma unroll
                for (int q = 0; q < Q; q++) {
                    const int off = line0 + 32 * q;
                    const R v = tile[(a + lane + 32 * q) * P + l];
                    if (E == EPI_STORE) o[off] = v;
                    if (E == EPI_STORE_NEG) o[off] = -v;
                    if (E == EPI_SUB) o[off] = old[gl][q] - v;
                    if (E == EPI_STORE_F64) o64[off] = (double)v;
                    if (E == EPI_RHS_FINAL) {
                        R tt = aux[gl][q] - v;
                        R dtJ = dt * jj[gl][q];
                        o[off] = mom ? (old[gl][q] + tt) * dtJ : tt * dtJ;
                    }
                }
            }
        }
    }
}

// E: the caller's operation (EpiMode), compiled into the kernel so that each
// instantiation carries one epilogue only.
// The solve of one tile once each lane holds rows a-H .. a+L+H-1 of its line
// in v: Dirichlet boundary rows, pass 1, the forward chain and fold, pass 2,
// the backward chain, fold and cyclic correction; y gets the solution rows
// a .. a+L-1. sh: the chain-state area of the shared memory (reg_chain_elems:
// the segments' local end states of both passes and the last segment's last
// two values). Every thread of the CTA calls it (it synchronises the CTA
// twice; each warp then chains the states it needs itself).
// NEG (the FP32 derivative form only): solve for the negated right-hand
// side, so that a negated store needs no negation of its own.
// hook(0) runs in every thread just before the barrier that ends pass 1 and
// hook(1) just after it: v is dead from there on, so a caller that loaded v
// from a shared-memory tile can hand the tile to its next load there instead
// of spending a barrier of its own.
struct NoFwdHook {
    __device__ __forceinline__ void operator()(int) const {}
};
template <typename R, int KIND, int H, int L, bool NEG = false, typename FwdHook = NoFwdHook>
__device__ __forceinline__ void reg_solve(const LineOpDev<R> &op, const R (&v)[L + 2 * H], R (&y)[L], bool work,
                                          int lane, int seg, int S, int a, R *sh, const FwdHook &hook = FwdHook()) {
    constexpr bool PER = (KIND % 2) == 0;
    constexpr bool TRI = KIND == K_TRI_PER || KIND == K_TRI_DIR;
    constexpr int NB = L / UB;
    // FP32 first derivatives (H <= 3; the launchers send only antisymmetric
    // stencils and no pass-through lines here): RHS as the 2H products of the
    // stencil without its zero centre, 1/dh in the coefficients; pass 1 keeps each
    // eliminated row times its pivot reciprocal rD_n (the multiply off the
    // recurrence's path) and the backward factors come pre-multiplied by it,
    // so pass 2 is two FMAs a row with one on its path; every lane's line is
    // solved (lanes past the block's last line hold zeros and are not stored).
    constexpr bool FAST = sizeof(R) == 4 && H <= 3;
    static_assert(FAST || !NEG, "a negated right-hand side only in the FP32 derivative form");
    if constexpr (FAST) work = true;
    using V = RegVec<R>;
    const int N = op.N;
    R *fwdEnd = sh;                    // [S][2][W] local end states of pass 1
    R *bwdStart = fwdEnd + S * 2 * W;  // [S][2][W] local start values of pass 2
    R *lastx = bwdStart + S * 2 * W;   // [2][W] x_{N-1}, x_{N-2}

    // ---- Dirichlet boundary rows (first / last segment) ----
    R headr[H], tailr[H];
    if (!PER) {
#pragma unroll
        for (int r = 0; r < H; r++) {
            R hs = 0, ts = 0;
            if (seg == 0) {
#pragma unroll
                for (int k = 0; k < MC3D_BWMAX; k++) hs += ldc(op.hp + r * MC3D_BWMAX + k) * v[H + k];
            }
            if (seg == S - 1) {
#pragma unroll
                for (int k = 0; k < MC3D_BWMAX; k++) ts += ldc(op.tp + r * MC3D_BWMAX + k) * v[H + L - MC3D_BWMAX + k];
            }
            headr[r] = hs * (NEG ? -op.inv_dh : op.inv_dh);
            tailr[r] = ts * (NEG ? -op.inv_dh : op.inv_dh);
        }
    }

    // ---- pass 1: RHS + local forward elimination (zero incoming state) ----
    // Pass-through and inactive lines keep their input in y.
    R y1 = 0, y2 = 0;   // y_{n-1}, y_{n-2}
#pragma unroll
    for (int blk = 0; blk < NB; blk++) {
        const int n0 = a + blk * UB;
        R rhs[UB];
#pragma unroll
        for (int u = 0; u < UB; u++) {
            const int r = blk * UB + u;
            if constexpr (FAST) {
                // 2H products, the zero centre skipped; the row's lowest value first
                R acc = (NEG ? op.sta[H - 1] : -op.sta[H - 1]) * v[r];
#pragma unroll
                for (int k = H - 1; k >= 1; k--) acc += (NEG ? op.sta[k - 1] : -op.sta[k - 1]) * v[r + H - k];
#pragma unroll
                for (int k = 1; k <= H; k++) acc += (NEG ? -op.sta[k - 1] : op.sta[k - 1]) * v[r + H + k];
                rhs[u] = acc;
            } else {
                R acc = op.st[0] * v[r];
#pragma unroll
                for (int k = 1; k < 2 * H + 1; k++) acc += op.st[k] * v[r + k];
                rhs[u] = acc * op.inv_dh;
            }
        }
        const bool stat = n0 >= op.stat_lo && n0 + UB <= op.stat_hi && (PER || (n0 >= H && n0 + UB <= N - H));
        if (stat) {
            const R m1 = op.stat_c[0], m2 = op.stat_c[1];
            const R rDs = FAST ? op.stat_b[2] : R(1);
#pragma unroll
            for (int u = 0; u < UB; u++) {
                R x = TRI ? rhs[u] - m1 * y1 : rhs[u] - m2 * y2 - m1 * y1;
                y2 = y1;
                y1 = x;
                if constexpr (FAST) y[blk * UB + u] = rDs * x;
                else y[blk * UB + u] = work ? x : v[H + blk * UB + u];
            }
        } else {
#pragma unroll
            for (int u = 0; u < UB; u++) {
                const int n = n0 + u;
                R rr = rhs[u];
                if (!PER) {
#pragma unroll
                    for (int q = 0; q < H; q++) {
                        if (n == q) rr = headr[q];
                        if (n == N - 1 - q) rr = tailr[q];
                    }
                }
                R m1, m2;
                V::ld2(op.pf + 2 * n, m1, m2);
                R x = TRI ? rr - m1 * y1 : rr - m2 * y2 - m1 * y1;
                y2 = y1;
                y1 = x;
                if constexpr (FAST) y[blk * UB + u] = ldc(op.pbs + 4 * n + 2) * x;
                else y[blk * UB + u] = work ? x : v[H + blk * UB + u];
            }
        }
    }
    fwdEnd[(seg * 2 + 0) * W + lane] = y1;
    fwdEnd[(seg * 2 + 1) * W + lane] = y2;
    hook(0);
    __syncthreads();
    hook(1);

    // ---- chain the forward states up to this segment: its incoming (y_{a-1}, y_{a-2}) ----
    // (each warp runs the chain of the segments before its own, so no further
    // barrier is needed)
    R F1 = 0, F2 = 0;
    for (int ws = 1; ws <= seg; ws++) {
        const int e1 = ws * L - 1, e2 = e1 - 1;
        R s1a, s1b, s2a, s2b;
        V::ld2(op.sf2 + 2 * e1, s1a, s1b);
        V::ld2(op.sf2 + 2 * e2, s2a, s2b);
        R n1 = fwdEnd[((ws - 1) * 2 + 0) * W + lane] + s1a * F1 + s1b * F2;
        R n2 = fwdEnd[((ws - 1) * 2 + 1) * W + lane] + s2a * F1 + s2b * F2;
        F1 = work ? n1 : R(0);
        F2 = work ? n2 : R(0);
    }

    // ---- forward fold: propagate the incoming state through the first kf rows ----
    if (seg > 0) {
        const int kf = op.seg_kf;
#pragma unroll
        for (int blk = 0; blk < NB; blk++) {
            if (blk * UB < kf) {
                const int n0 = a + blk * UB;
                const bool stat = n0 >= op.stat_lo && n0 + UB <= op.stat_hi;
                if (stat) {
                    const R m1 = op.stat_c[0], m2 = op.stat_c[1];
                    const R rDs = FAST ? op.stat_b[2] : R(1);
#pragma unroll
                    for (int u = 0; u < UB; u++) {
                        R F = TRI ? -(m1 * F1) : -(m2 * F2) - m1 * F1;
                        if constexpr (FAST) y[blk * UB + u] += rDs * F;
                        else y[blk * UB + u] += F;
                        F2 = F1;
                        F1 = F;
                    }
                } else {
#pragma unroll
                    for (int u = 0; u < UB; u++) {
                        R m1, m2;
                        V::ld2(op.pf + 2 * (n0 + u), m1, m2);
                        R F = TRI ? -(m1 * F1) : -(m2 * F2) - m1 * F1;
                        if constexpr (FAST) y[blk * UB + u] += ldc(op.pbs + 4 * (n0 + u) + 2) * F;
                        else y[blk * UB + u] += F;
                        F2 = F1;
                        F1 = F;
                    }
                }
            }
        }
    }

    // ---- pass 2: local backward substitution (zero incoming state) ----
    {
        R x1 = 0, x2 = 0;   // x_{n+1}, x_{n+2}
#pragma unroll
        for (int blk = NB - 1; blk >= 0; blk--) {
            const int n0 = a + blk * UB;
            const bool stat = n0 >= op.stat_lo && n0 + UB <= op.stat_hi;
            if (stat) {
                if constexpr (FAST) {
                    const R Cs = op.stat_b[0], fs = op.stat_b[1];
#pragma unroll
                    for (int u = UB - 1; u >= 0; u--) {
                        const int r = blk * UB + u;
                        R t = y[r];
                        if (!TRI) t -= fs * x2;
                        const R x = t - Cs * x1;
                        x2 = x1;
                        x1 = x;
                        y[r] = x;
                    }
                } else {
                    const R C = TRI ? op.stat_c[2] : op.stat_c[3];
                    const R fv = TRI ? R(0) : op.stat_c[4];
                    const R rD = TRI ? op.stat_c[1] : op.stat_c[2];
#pragma unroll
                    for (int u = UB - 1; u >= 0; u--) {
                        const int r = blk * UB + u;
                        R x = TRI ? (y[r] - C * x1) * rD : (y[r] - fv * x2 - C * x1) * rD;
                        x2 = x1;
                        x1 = x;
                        if (work) y[r] = x;
                    }
                }
            } else {
#pragma unroll
                for (int u = UB - 1; u >= 0; u--) {
                    const int r = blk * UB + u;
                    R C, fv, rD, pad;
                    if constexpr (FAST) {
                        V::ld4(op.pbs + 4 * (n0 + u), C, fv, rD, pad);
                        R t = y[r];
                        if (!TRI) t -= fv * x2;
                        const R x = t - C * x1;
                        x2 = x1;
                        x1 = x;
                        y[r] = x;
                    } else {
                        V::ld4(op.pb + 4 * (n0 + u), C, fv, rD, pad);
                        R x = TRI ? (y[r] - C * x1) * rD : (y[r] - fv * x2 - C * x1) * rD;
                        x2 = x1;
                        x1 = x;
                        if (work) y[r] = x;
                    }
                }
            }
        }
    }
    bwdStart[(seg * 2 + 0) * W + lane] = y[0];
    bwdStart[(seg * 2 + 1) * W + lane] = y[1];
    if (seg == S - 1) {
        lastx[lane] = y[L - 1];
        lastx[W + lane] = y[L - 2];
    }
    __syncthreads();

    // ---- chain the backward states down to this segment (periodic lines: down
    // to the first, for the cyclic correction scalars); every warp runs it ----
    R G1 = 0, G2 = 0;   // incoming backward state of this segment
    R c[4] = {R(0), R(0), R(0), R(0)};
    {
        R Y1 = 0, Y2 = 0;
        const int wlo = PER ? 0 : seg;
        for (int ws = S - 2; ws >= wlo; ws--) {
            const int s0 = (ws + 1) * L;
            R b1a, b1b, b2a, b2b;
            V::ld2(op.sb2 + 2 * s0, b1a, b1b);
            V::ld2(op.sb2 + 2 * (s0 + 1), b2a, b2b);
            R n1 = bwdStart[((ws + 1) * 2 + 0) * W + lane] + b1a * Y1 + b1b * Y2;
            R n2 = bwdStart[((ws + 1) * 2 + 1) * W + lane] + b2a * Y1 + b2b * Y2;
            Y1 = work ? n1 : R(0);
            Y2 = work ? n2 : R(0);
            if (ws == seg) {
                G1 = Y1;
                G2 = Y2;
            }
        }
        if (work && PER) {
            // final x_0, x_1 (first segment, folded) and x_{N-1}, x_{N-2} (last segment)
            R b0a, b0b, b1a, b1b;
            V::ld2(op.sb2 + 0, b0a, b0b);
            V::ld2(op.sb2 + 2, b1a, b1b);
            R x0 = bwdStart[0 * W + lane] + b0a * Y1 + b0b * Y2;
            R x1 = bwdStart[1 * W + lane] + b1a * Y1 + b1b * Y2;
            R xN1 = lastx[lane], xN2 = lastx[W + lane];
            if (KIND == K_TRI_PER) {
                // Sherman-Morrison factor (src/Utils.cpp:43)
                c[0] = (x0 + op.sc[0] * xN1 * op.sc[1]) * op.sc[2];
            } else {
                // Woodbury (src/Utils.cpp:158-181)
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
    }

    // ---- backward fold: propagate the incoming state up through the last kb rows ----
    if (seg < S - 1) {
        const int kb = op.seg_kb;
#pragma unroll
        for (int blk = NB - 1; blk >= 0; blk--) {
            if ((blk + 1) * UB > L - kb) {
                const int n0 = a + blk * UB;
                const bool stat = n0 >= op.stat_lo && n0 + UB <= op.stat_hi;
                if (stat) {
                    const R C = FAST ? op.stat_b[0] : (TRI ? op.stat_c[2] : op.stat_c[3]);
                    const R fv = FAST ? op.stat_b[1] : (TRI ? R(0) : op.stat_c[4]);
                    const R rD = TRI ? op.stat_c[1] : op.stat_c[2];
#pragma unroll
                    for (int u = UB - 1; u >= 0; u--) {
                        R G;
                        if constexpr (FAST) G = TRI ? -(C * G1) : -(fv * G2) - C * G1;
                        else G = TRI ? (R(0) - C * G1) * rD : (R(0) - fv * G2 - C * G1) * rD;
                        y[blk * UB + u] += G;
                        G2 = G1;
                        G1 = G;
                    }
                } else {
#pragma unroll
                    for (int u = UB - 1; u >= 0; u--) {
                        R C, fv, rD, pad, G;
                        if constexpr (FAST) {
                            V::ld4(op.pbs + 4 * (n0 + u), C, fv, rD, pad);
                            G = TRI ? -(C * G1) : -(fv * G2) - C * G1;
                        } else {
                            V::ld4(op.pb + 4 * (n0 + u), C, fv, rD, pad);
                            G = TRI ? (R(0) - C * G1) * rD : (R(0) - fv * G2 - C * G1) * rD;
                        }
                        y[blk * UB + u] += G;
                        G2 = G1;
                        G1 = G;
                    }
                }
            }
        }
    }

    // ---- cyclic correction (src/Utils.cpp:45 and :183-190) where its columns matter ----
    if (PER) {
        const R c0 = c[0], c1 = c[1], c2 = c[2], c3 = c[3];
#pragma unroll
        for (int blk = 0; blk < NB; blk++) {
            const int n0 = a + blk * UB;
            if (!(n0 >= op.corr_lo && n0 + UB <= op.corr_hi)) {
#pragma unroll
                for (int u = 0; u < UB; u++) {
                    const int n = n0 + u;
                    if (KIND == K_TRI_PER) {
                        y[blk * UB + u] -= c0 * ldc(op.a3 + n);
                    } else {
                        R z0, z1, z2, z3;
                        V::ld4(op.pz + 4 * n, z0, z1, z2, z3);
                        if constexpr (FAST) {
                            // four FMAs into the row
                            R t = y[blk * UB + u] - z0 * c0;
                            t -= z1 * c1;
                            t -= z2 * c2;
                            y[blk * UB + u] = t - z3 * c3;
                        } else {
                            R sum = z0 * c0 + z1 * c1 + z2 * c2 + z3 * c3;
                            y[blk * UB + u] -= sum;
                        }
                    }
                }
            }
        }
    }

}

template <int DIR, typename R, int KIND, int H, int L, int E>
__global__ void __launch_bounds__(512) sweep_reg_kernel(Grid3 g, LineOpDev<R> op, SweepBatch<R> b,
                                                        RhsFinalArgs<R> rf, int pass_y, int pass_z, int pass_x) {
    constexpr bool PER = (KIND % 2) == 0;
    constexpr int NV = L + 2 * H;
    constexpr int P = W + 1;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    R *sh = reinterpret_cast<R *>(smem_raw);
    const int S = blockDim.x >> 5;
    const int lane = threadIdx.x & 31, seg = threadIdx.x >> 5;
    const int N = op.N, a = seg * L;
    const int f = blockIdx.y;
    R *tile = sh + reg_chain_elems(S);   // x lines: [N][W+1], after the chain states

    const TileGeom t = tile_geom<DIR>(g, blockIdx.x, lane);
    bool pass = false;
    if (DIR == 0) pass = (pass_y && (t.j == 0 || t.j == g.Ny - 1)) || (pass_z && (t.k == 0 || t.k == g.Nz - 1));
    if (DIR == 1) pass = (pass_x && (t.i == 0 || t.i == g.Nx - 1)) || (pass_z && (t.k == 0 || t.k == g.Nz - 1));
    if (DIR == 2) pass = (pass_y && (t.j == 0 || t.j == g.Ny - 1)) || (pass_x && (t.i == 0 || t.i == g.Nx - 1));
    const bool work = t.active && !pass;

    // ---- load rows a-H .. a+L+H-1 of this lane's line (periodic wrap / zero) ----
    R v[NV];
    int nl = W;
    if (DIR == 0) {
        const long long rem = (long long)g.Ny * g.Nz - (long long)blockIdx.x * W;
        nl = rem < W ? (int)rem : W;
        const R *src = b.in[f] + (size_t)blockIdx.x * W * N;
        for (int l = 0; l < nl; l++) {
#pragma unroll
            for (int i0 = 0; i0 < L; i0 += 32) cp_async_elem(&tile[(a + i0 + lane) * P + l], src + l * N + a + i0 + lane);
        }
        cp_async_wait_all();
        __syncthreads();
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
            v[k] = in ? tile[n * P + lane] : R(0);
        }
    } else {
        const R *src = b.in[f] + (int)t.base;
        const int stride = (int)t.stride;
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
            v[k] = (t.active && in) ? src[n * stride] : R(0);
        }
    }

    R y[L];
    reg_solve<R, KIND, H, L>(op, v, y, work, lane, seg, S, a, sh);

    // ---- epilogue ----
    if (DIR == 0) {
        if (t.active) {
#pragma unroll
            for (int r = 0; r < L; r++) tile[(a + r) * P + lane] = y[r];
        }
        __syncwarp();
        const int tile0 = blockIdx.x * W;
        reg_copy_out<R, E, L>(b, rf, f, tile0, N, nl, a, lane, tile);
    } else if (t.active) {
        const int off0 = (int)t.base + a * (int)t.stride;
        reg_store_rows<R, E, L>(b, rf, f, off0, (int)t.stride, y);
    }
}

template <int DIR, typename R, int KIND, int H, int L, int E>
static int launch_reg_epi(const Grid3 &g, const LineOpDev<R> &op, const SweepBatch<R> &b, const RhsFinalArgs<R> &rf,
                          int px, int py, int pz, cudaStream_t st) {
    const int S = op.N / L;
    size_t smem = reg_smem_bytes(DIR, op.N, S, sizeof(R));
    auto kern = sweep_reg_kernel<DIR, R, KIND, H, L, E>;
    static KernelLaunchState ls;
    if (int rc = open_kernel(kern, ls, smem, 0, nullptr)) return rc;
    int tiles;
    if (DIR == 0) tiles = (int)(((long long)g.Ny * g.Nz + W - 1) / W);
    else if (DIR == 1) tiles = ((g.Nx + W - 1) / W) * g.Nz;
    else tiles = (int)(((long long)g.Nx * g.Ny + W - 1) / W);
    dim3 grid(tiles, b.nf);
    kern<<<grid, 32 * S, smem, st>>>(g, op, b, rf, py, pz, px);
    MC3D_CUDA_TRY(cudaGetLastError());
    return MC3D_OK;
}

// Epilogues instantiated per operator family: derivatives (H <= 3) store,
// negate, accumulate or assemble k2; filters (H >= 4) store in the working
// precision or in FP64. Other combinations go to the shared-memory kernels.
template <int DIR, typename R, int KIND, int H, int L>
static int launch_reg_one(const Grid3 &g, const LineOpDev<R> &op, const SweepBatch<R> &b, int epi,
                          const RhsFinalArgs<R> &rf, int px, int py, int pz, cudaStream_t st) {
    if (epi == EPI_STORE) return launch_reg_epi<DIR, R, KIND, H, L, EPI_STORE>(g, op, b, rf, px, py, pz, st);
    if constexpr (H <= 3) {
        if (epi == EPI_STORE_NEG) return launch_reg_epi<DIR, R, KIND, H, L, EPI_STORE_NEG>(g, op, b, rf, px, py, pz, st);
        if (epi == EPI_SUB) return launch_reg_epi<DIR, R, KIND, H, L, EPI_SUB>(g, op, b, rf, px, py, pz, st);
        if (epi == EPI_RHS_FINAL) return launch_reg_epi<DIR, R, KIND, H, L, EPI_RHS_FINAL>(g, op, b, rf, px, py, pz, st);
    } else {
        if (epi == EPI_STORE_F64) return launch_reg_epi<DIR, R, KIND, H, L, EPI_STORE_F64>(g, op, b, rf, px, py, pz, st);
    }
    return MC3D_ERR_CONFIG;
}

// Register-resident launch for direction DIR; returns MC3D_ERR_CONFIG (without
// recording an error) when the operator is not one this kernel handles.
template <int DIR, typename R>
int launch_sweep_reg(const Grid3 &g, const LineOpDev<R> &op, const SweepBatch<R> &b, int epi,
                     const RhsFinalArgs<R> &rf, int px, int py, int pz, cudaStream_t st) {
    if constexpr (sizeof(R) == 4) {
        // the FP32 solve of H <= 3 takes antisymmetric stencils and no
        // pass-through lines (reg_solve); anything else goes to the
        // shared-memory kernels
        if (op.H <= 3 && (px || py || pz || !op.asym)) return MC3D_ERR_CONFIG;
        const int rc = DIR == 0 ? launch_sweep_tma_x(g, op, b, epi, px, py, pz, st)
                                : launch_sweep_tma_yz(DIR, g, op, b, epi, rf, px, py, pz, st);
        if (rc != MC3D_ERR_CONFIG) return rc;
    }
#define MC3D_RCASE(K, HH, LL)                                                  \
    if (op.kind == K && op.H == HH && op.L == LL)                              \
        return launch_reg_one<DIR, R, K, HH, LL>(g, op, b, epi, rf, px, py, pz, st);
#define MC3D_RKINDS(LL)            \
    MC3D_RCASE(K_TRI_PER, 2, LL)   \
    MC3D_RCASE(K_TRI_DIR, 2, LL)   \
    MC3D_RCASE(K_PEN_PER, 3, LL)   \
    MC3D_RCASE(K_PEN_DIR, 3, LL)   \
    MC3D_RCASE(K_TRI_PER, 4, LL)   \
    MC3D_RCASE(K_TRI_DIR, 4, LL)   \
    MC3D_RCASE(K_TRI_PER, 5, LL)   \
    MC3D_RCASE(K_TRI_DIR, 5, LL)   \
    MC3D_RCASE(K_PEN_PER, 5, LL)   \
    MC3D_RCASE(K_PEN_DIR, 5, LL)
    MC3D_RKINDS(32)
    if constexpr (sizeof(R) == 4) {
        MC3D_RKINDS(64)
    }
#undef MC3D_RKINDS
#undef MC3D_RCASE
    return MC3D_ERR_CONFIG;
}

}  // namespace mc3d
