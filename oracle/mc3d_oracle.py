"""CPU oracle: a numpy restatement of the reference CurvilinearCSolver time step.

TEST INFRASTRUCTURE ONLY. Nothing in the product package imports this module;
only tests/, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg
may call it, and only as the checker. Every function cites the file:line of
emathew1/MPI_3DCompact (paths relative to that project) whose arithmetic it
restates. The restatement itself is pinned against the reference's own C++,
compiled unchanged into ``oracle/_ref/mc3d_ref`` (see oracle/Makefile), through
the fixtures in tests/golden/.

Layout: every field is a float64 array shaped (Nz, Ny, Nx) (x fastest), the
global order the reference uses for its dumps (CurvilinearCSolver_Core.cpp:1333).
Direction d in {0,1,2} = xi1 (x, axis 2), xi2 (y, axis 1), xi3 (z, axis 0).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

PERIODIC, DIRICHLET = 0, 1
_AXIS = {0: 2, 1: 1, 2: 0}


def _to_lines(f, d):
    return np.moveaxis(f, _AXIS[d], -1)


def _from_lines(f, d):
    return np.moveaxis(f, -1, _AXIS[d])


# --------------------------------------------------------------------------
# Banded solvers (src/Utils.cpp:4-191), vectorised over leading axes.
# --------------------------------------------------------------------------
def solve_tri(a, b, c, d):
    """Thomas algorithm, src/Utils.cpp:4-20 (a[0] and c[n-1] unused)."""
    n = d.shape[-1]
    work = np.array(b, dtype=np.float64, copy=True)
    x = np.array(d, dtype=np.float64, copy=True)
    for ip in range(1, n):
        m = a[ip] / work[ip - 1]
        work[ip] = work[ip] - m * c[ip - 1]
        x[..., ip] = x[..., ip] - m * x[..., ip - 1]
    x[..., n - 1] /= work[n - 1]
    for ip in range(n - 2, -1, -1):
        x[..., ip] = (x[..., ip] - c[ip] * x[..., ip + 1]) / work[ip]
    return x


def cyclic(a, b, c, alpha, beta, r):
    """Sherman-Morrison cyclic tridiagonal, src/Utils.cpp:22-46."""
    n = r.shape[-1]
    gamma = -b[0]
    bb = np.array(b, dtype=np.float64, copy=True)
    bb[0] = b[0] - gamma
    bb[n - 1] = b[n - 1] - alpha * beta / gamma
    x = solve_tri(a, bb, c, r)
    u = np.zeros(n)
    u[0] = gamma
    u[n - 1] = alpha
    z = solve_tri(a, bb, c, u)
    fact = (x[..., 0] + beta * x[..., n - 1] / gamma) / (1.0 + z[0] + beta * z[n - 1] / gamma)
    return x - fact[..., None] * z


def solve_penta(e, a, d, c, f, b):
    """Pentadiagonal elimination, src/Utils.cpp:48-83 (band layout of :50-57)."""
    size = b.shape[-1]
    x = np.array(a, dtype=np.float64, copy=True)        # lower band, becomes multipliers
    B = np.array(b, dtype=np.float64, copy=True)
    C = np.array(c, dtype=np.float64, copy=True)
    D = np.array(d, dtype=np.float64, copy=True)
    xs = np.zeros(b.shape)
    for ip in range(1, size - 1):
        xmult = x[ip - 1] / D[ip - 1]
        D[ip] = D[ip] - xmult * C[ip - 1]
        C[ip] = C[ip] - xmult * f[ip - 1]
        B[..., ip] = B[..., ip] - xmult * B[..., ip - 1]
        xmult = e[ip - 1] / D[ip - 1]
        x[ip] = x[ip] - xmult * C[ip - 1]
        D[ip + 1] = D[ip + 1] - xmult * f[ip - 1]
        B[..., ip + 1] = B[..., ip + 1] - xmult * B[..., ip - 1]
    xmult = x[size - 2] / D[size - 2]
    D[size - 1] = D[size - 1] - xmult * C[size - 2]
    xs[..., size - 1] = (B[..., size - 1] - xmult * B[..., size - 2]) / D[size - 1]
    xs[..., size - 2] = (B[..., size - 2] - C[size - 2] * xs[..., size - 1]) / D[size - 2]
    for ip in range(size - 3, -1, -1):
        xs[..., ip] = (B[..., ip] - f[ip] * xs[..., ip + 2] - C[ip] * xs[..., ip + 1]) / D[ip]
    return xs


def _inv4_adjugate(m):
    """4x4 inverse by adjugate / determinant, src/Utils.cpp:193-224."""
    def minor(r0, r1, r2, c0, c1, c2):
        return (m[r0, c0] * (m[r1, c1] * m[r2, c2] - m[r2, c1] * m[r1, c2])
                - m[r0, c1] * (m[r1, c0] * m[r2, c2] - m[r2, c0] * m[r1, c2])
                + m[r0, c2] * (m[r1, c0] * m[r2, c1] - m[r2, c0] * m[r1, c1]))
    adj = np.array([
        [minor(1, 2, 3, 1, 2, 3), -minor(0, 2, 3, 1, 2, 3), minor(0, 1, 3, 1, 2, 3), -minor(0, 1, 2, 1, 2, 3)],
        [-minor(1, 2, 3, 0, 2, 3), minor(0, 2, 3, 0, 2, 3), -minor(0, 1, 3, 0, 2, 3), minor(0, 1, 2, 0, 2, 3)],
        [minor(1, 2, 3, 0, 1, 3), -minor(0, 2, 3, 0, 1, 3), minor(0, 1, 3, 0, 1, 3), -minor(0, 1, 2, 0, 1, 3)],
        [-minor(1, 2, 3, 0, 1, 2), minor(0, 2, 3, 0, 1, 2), -minor(0, 1, 3, 0, 1, 2), minor(0, 1, 2, 0, 1, 2)]])
    det = (m[0, 0] * minor(1, 2, 3, 1, 2, 3) - m[0, 1] * minor(1, 2, 3, 0, 2, 3)
           + m[0, 2] * minor(1, 2, 3, 0, 1, 3) - m[0, 3] * minor(1, 2, 3, 0, 1, 2))
    return adj * (1.0 / det)


def cyclic_penta(e2, e1, d0, f1, f2, rhs, cp):
    """Cyclic pentadiagonal via a rank-4 Woodbury correction, src/Utils.cpp:85-191.
    Arguments follow the reference call cyclicPenta(offlower2, offlower, diag,
    offupper, offupper2, RHS, cpvec) (src/Penta10.cpp:254-261)."""
    n = rhs.shape[-1]
    U = np.zeros((4, n))
    V = np.zeros((4, n))
    U[0, 0] = U[1, 1] = U[2, n - 2] = U[3, n - 1] = 1.0
    V[0, n - 2], V[0, n - 1], V[1, n - 1] = cp[0], cp[1], cp[2]
    V[2, 0], V[3, 0], V[3, 1] = cp[3], cp[4], cp[5]
    Z = np.stack([solve_penta(e2, e1, d0, f1, f2, U[i]) for i in range(4)])
    y = solve_penta(e2, e1, d0, f1, f2, rhs)
    P = np.empty((4, 4))
    for i in range(4):
        for j in range(4):
            s = 0.0
            for k in range(n):
                s += V[i, k] * Z[j, k]
            P[i, j] = s
    P += np.eye(4)
    H = _inv4_adjugate(P)
    # r[i] = sum_k V[i,k] y[k]; V rows have nonzeros only at k in {0,1,n-2,n-1}
    r = [np.zeros(y.shape[:-1]) + 0.0 for _ in range(4)]
    for i in range(4):
        for k in (0, 1, n - 2, n - 1) if n > 3 else range(n):
            if V[i, k] != 0.0:
                r[i] = r[i] + V[i, k] * y[..., k]
    s = [H[i, 0] * r[0] + H[i, 1] * r[1] + H[i, 2] * r[2] + H[i, 3] * r[3] for i in range(4)]
    corr = Z[0] * s[0][..., None] + Z[1] * s[1][..., None] + Z[2] * s[2][..., None] + Z[3] * s[3][..., None]
    return y - corr


# --------------------------------------------------------------------------
# Compact first derivatives (src/Pade6.*, src/Penta10.*, src/CD2.*)
# --------------------------------------------------------------------------
def _roll(phi, s):
    """phi[(i + s) mod N] along the last axis."""
    return np.roll(phi, -s, axis=-1)


def pade6_lhs(n, bc):
    """Band arrays of src/Pade6.hpp:183-215 (first derivative)."""
    alpha = 1.0 / 3.0
    lo = np.full(n, alpha)
    up = np.full(n, alpha)
    dg = np.ones(n)
    if bc == DIRICHLET:
        alpha11, alpha21, alpha22 = 2.0, 1.0 / 6.0, 1.0 / 2.0
        up[0], up[1], lo[1] = alpha11, alpha22, alpha21
        lo[n - 1], lo[n - 2], up[n - 2] = alpha11, alpha22, alpha21
    return lo, dg, up


def pade6_deriv_lines(phi, dh, bc):
    """src/Pade6.cpp:187-218 (periodic RHS), :284-313 (Dirichlet RHS),
    :351-384 (cyclic / solveTri)."""
    n = phi.shape[-1]
    a_1d, b_1d = 14.0 / 9.0, 1.0 / 9.0
    cc2, cc3, cc4, cc5 = -b_1d / 4.0, -a_1d / 2.0, a_1d / 2.0, b_1d / 4.0
    lo, dg, up = pade6_lhs(n, bc)
    if bc == PERIODIC:
        rhs = cc2 * _roll(phi, -2) + cc3 * _roll(phi, -1) + cc4 * _roll(phi, 1) + cc5 * _roll(phi, 2)
        rhs = rhs / dh
        return cyclic(lo, dg, up, 1.0 / 3.0, 1.0 / 3.0, rhs)
    a1, b1, c1, d1, e1, f1 = -5.0 / 2.0, 2.0, 1.0 / 2.0, 0.0, 0.0, 0.0
    a2, b2, c2, d2, e2 = -5.0 / 9.0, -1.0 / 2.0, 1.0, 1.0 / 18.0, 0.0
    rhs = np.zeros(phi.shape)
    p = phi
    rhs[..., 0] = a1 * p[..., 0] + b1 * p[..., 1] + c1 * p[..., 2] + d1 * p[..., 3] + e1 * p[..., 4] + f1 * p[..., 5]
    rhs[..., 1] = a2 * p[..., 0] + b2 * p[..., 1] + c2 * p[..., 2] + d2 * p[..., 3] + e2 * p[..., 4]
    rhs[..., 2:n - 2] = (cc2 * p[..., 0:n - 4] + cc3 * p[..., 1:n - 3] + cc4 * p[..., 3:n - 1] + cc5 * p[..., 4:n])
    rhs[..., n - 2] = (-e2 * p[..., n - 5] - d2 * p[..., n - 4] - c2 * p[..., n - 3] - b2 * p[..., n - 2] - a2 * p[..., n - 1])
    rhs[..., n - 1] = (-f1 * p[..., n - 6] - e1 * p[..., n - 5] - d1 * p[..., n - 4] - c1 * p[..., n - 3]
                       - b1 * p[..., n - 2] - a1 * p[..., n - 1])
    rhs = rhs / dh
    return solve_tri(lo, dg, up, rhs)


def penta10_lhs(n, bc):
    """Band arrays of src/Penta10.hpp:116-175 (penta layout: lower bands skip
    the last index, src/Utils.cpp:50-57)."""
    beta, alpha = 1.0 / 20.0, 1.0 / 2.0
    dg = np.ones(n)
    lo = np.full(n, alpha)
    up = np.full(n, alpha)
    lo2 = np.full(n, beta)
    up2 = np.full(n, beta)
    if bc == DIRICHLET:
        beta1, alpha1 = 0.0, 5.0
        beta2, alpha2_1, alpha2_2 = 0.0, 1.0 / 12.0, 5.0 / 4.0
        beta3_1 = beta3_2 = 1.0 / 36.0
        alpha3_1 = alpha3_2 = 4.0 / 9.0
        up[0], up[1], up[2] = alpha1, alpha2_2, alpha3_2
        lo[0], lo[1] = alpha2_1, alpha3_1
        up2[0], up2[1], up2[2] = beta1, beta2, beta3_2
        lo2[0] = beta3_1
        up[n - 2], up[n - 3] = alpha2_1, alpha3_1
        lo[n - 2], lo[n - 3], lo[n - 4] = alpha1, alpha2_2, alpha3_2
        up2[n - 3] = beta3_1
        lo2[n - 3], lo2[n - 4], lo2[n - 5] = beta1, beta2, beta3_2
    return lo2, lo, dg, up, up2


def penta10_deriv_lines(phi, dh, bc):
    """src/Penta10.cpp:141-173 (periodic RHS), :211-252 (Dirichlet RHS),
    :254-282 (cyclicPenta / solvePenta)."""
    n = phi.shape[-1]
    a, b, c = 17.0 / 12.0, 101.0 / 150.0, 1.0 / 100.0
    cc1, cc2, cc3, cc4, cc5, cc6 = -c / 6.0, -b / 4.0, -a / 2.0, a / 2.0, b / 4.0, c / 6.0
    lo2, lo, dg, up, up2 = penta10_lhs(n, bc)
    p = phi
    if bc == PERIODIC:
        rhs = (cc1 * _roll(p, -3) + cc2 * _roll(p, -2) + cc3 * _roll(p, -1)
               + cc4 * _roll(p, 1) + cc5 * _roll(p, 2) + cc6 * _roll(p, 3))
        rhs = rhs / dh
        beta, alpha = 1.0 / 20.0, 1.0 / 2.0
        cp = [beta, alpha, beta, beta, alpha, beta]
        return cyclic_penta(lo2, lo, dg, up, up2, rhs, cp)
    a1, b1, c1, d1, e1, f1, g1, h1, i1 = (-197.0 / 60.0, -5.0 / 12.0, 5.0, -5.0 / 3.0, 5.0 / 12.0, -1.0 / 20.0,
                                          0.0, 0.0, 0.0)
    a2, b2, c2, d2, e2, f2, g2, h2 = (-79.0 / 240.0, -77.0 / 60.0, 55.0 / 48.0, 5.0 / 9.0, -5.0 / 48.0,
                                      1.0 / 60.0, -1.0 / 720.0, 0.0)
    a3, b3, c3, d3, e3, f3, g3 = (-25.0 / 54.0 / 4.0, -40.0 / 27.0 / 2.0, 0.0, 40.0 / 27.0 / 2.0,
                                  25.0 / 54.0 / 4.0, 0.0, 0.0)
    rhs = np.zeros(p.shape)
    rhs[..., 0] = (a1 * p[..., 0] + b1 * p[..., 1] + c1 * p[..., 2] + d1 * p[..., 3] + e1 * p[..., 4]
                   + f1 * p[..., 5] + g1 * p[..., 6] + h1 * p[..., 7] + i1 * p[..., 8])
    rhs[..., 1] = (a2 * p[..., 0] + b2 * p[..., 1] + c2 * p[..., 2] + d2 * p[..., 3] + e2 * p[..., 4]
                   + f2 * p[..., 5] + g2 * p[..., 6] + h2 * p[..., 7])
    rhs[..., 2] = (a3 * p[..., 0] + b3 * p[..., 1] + c3 * p[..., 2] + d3 * p[..., 3] + e3 * p[..., 4]
                   + f3 * p[..., 5] + g3 * p[..., 6])
    rhs[..., 3:n - 3] = (cc1 * p[..., 0:n - 6] + cc2 * p[..., 1:n - 5] + cc3 * p[..., 2:n - 4]
                         + cc4 * p[..., 4:n - 2] + cc5 * p[..., 5:n - 1] + cc6 * p[..., 6:n])
    rhs[..., n - 3] = (-g3 * p[..., n - 7] - f3 * p[..., n - 6] - e3 * p[..., n - 5] - d3 * p[..., n - 4]
                       - c3 * p[..., n - 3] - b3 * p[..., n - 2] - a3 * p[..., n - 1])
    rhs[..., n - 2] = (-h2 * p[..., n - 8] - g2 * p[..., n - 7] - f2 * p[..., n - 6] - e2 * p[..., n - 5]
                       - d2 * p[..., n - 4] - c2 * p[..., n - 3] - b2 * p[..., n - 2] - a2 * p[..., n - 1])
    rhs[..., n - 1] = (-i1 * p[..., n - 9] - h1 * p[..., n - 8] - g1 * p[..., n - 7] - f1 * p[..., n - 6]
                       - e1 * p[..., n - 5] - d1 * p[..., n - 4] - c1 * p[..., n - 3] - b1 * p[..., n - 2]
                       - a1 * p[..., n - 1])
    rhs = rhs / dh
    return solve_penta(lo2, lo, dg, up, up2, rhs)


def cd2_deriv_lines(phi, dh, bc):
    """Explicit two-point difference exactly as src/CD2.cpp:129-183 computes it:
    with a=-1/2, c=+1/2 (src/CD2.hpp:56-58) the interior and node N-1 rows are
    (a*phi[i+1] + c*phi[i-1])/h, i.e. the NEGATIVE of the central difference,
    while node 0 of a Dirichlet line is the positive one-sided (-3/2, 2, -1/2)/h.
    The sign quirk is reproduced, not corrected."""
    n = phi.shape[-1]
    a, c = -0.5, 0.5
    aa, bb, cc = -1.5, 2.0, -0.5
    out = np.empty(phi.shape)
    out[..., 1:n - 1] = (a * phi[..., 2:n] + c * phi[..., 0:n - 2]) / dh
    if bc == PERIODIC:
        out[..., 0] = (a * phi[..., n - 1] + c * phi[..., 1]) / dh
        out[..., n - 1] = (a * phi[..., n - 2] + c * phi[..., 0]) / dh
    else:
        out[..., 0] = (aa * phi[..., 0] + bb * phi[..., 1] + cc * phi[..., 2]) / dh
        out[..., n - 1] = (aa * phi[..., n - 1] + bb * phi[..., n - 2] + cc * phi[..., n - 3]) / dh
    return out


def deriv(f, d, scheme, bc, dh):
    """calc1stDerivField for one direction (src/AbstractDerivatives.hpp:45)."""
    lines = _to_lines(f, d)
    if scheme == "PADE6":
        out = pade6_deriv_lines(lines, dh, bc)
    elif scheme == "PENTA10":
        out = penta10_deriv_lines(lines, dh, bc)
    elif scheme == "CD2":
        out = cd2_deriv_lines(lines, dh, bc)
    else:
        raise ValueError(scheme)
    return np.ascontiguousarray(_from_lines(out, d))


# --------------------------------------------------------------------------
# Compact filters (src/Compact8Filter.*, src/Compact10Filter.*)
# --------------------------------------------------------------------------
def compact10_coeffs(af):
    """Interior and boundary (scheme 1) coefficients, src/Compact10Filter.hpp:58-134."""
    a = [(193.0 + 126.0 * af) / 256.0, (105.0 + 302.0 * af) / 256.0, (-15.0 + 30.0 * af) / 64.0,
         (45.0 - 90.0 * af) / 512.0, (-5.0 + 10.0 * af) / 256.0, (1.0 - 2.0 * af) / 512.0]
    fb2 = [(1.0 + 1022.0 * af) / 1024.0, (507.0 + 10.0 * af) / 512.0, (45.0 + 934.0 * af) / 1024.0,
           (-15.0 + 30.0 * af) / 128.0, (105.0 - 210.0 * af) / 512.0, (-63.0 + 126.0 * af) / 256.0,
           (105.0 - 210.0 * af) / 512.0, (-15.0 + 30.0 * af) / 128.0, (45.0 - 90.0 * af) / 1024.0,
           (-5.0 + 10.0 * af) / 512.0, (1.0 - 2.0 * af) / 1024.0]
    fb3 = [(-1.0 + 2.0 * af) / 1024.0, (5.0 + 502.0 * af) / 512.0, (979.0 + 90.0 * af) / 1024.0,
           (15.0 + 98.0 * af) / 128.0, (-105.0 + 210.0 * af) / 512.0, (63.0 - 126.0 * af) / 256.0,
           (-105.0 + 210.0 * af) / 512.0, (15.0 - 30.0 * af) / 128.0, (-45.0 + 90.0 * af) / 1024.0,
           (5.0 - 10.0 * af) / 512.0, (-1.0 + 2.0 * af) / 1024.0]
    fb4 = [(1.0 - 2.0 * af) / 1024.0, (-5.0 + 10.0 * af) / 512.0, (45.0 + 934.0 * af) / 1024.0,
           (113.0 + 30.0 * af) / 128.0, (105.0 + 302.0 * af) / 512.0, (-63.0 + 126.0 * af) / 256.0,
           (105.0 - 210.0 * af) / 512.0, (-15.0 + 30.0 * af) / 128.0, (45.0 - 90.0 * af) / 1024.0,
           (-5.0 + 10.0 * af) / 512.0, (1.0 - 2.0 * af) / 1024.0]
    fb5 = [(-1.0 + 2.0 * af) / 1024.0, (5.0 - 10.0 * af) / 512.0, (-45.0 + 90.0 * af) / 1024.0,
           (15.0 + 98.0 * af) / 128.0, (407.0 + 210.0 * af) / 512.0, (63.0 + 130.0 * af) / 256.0,
           (-105.0 + 210.0 * af) / 512.0, (15.0 - 30.0 * af) / 128.0, (-45.0 + 90.0 * af) / 1024.0,
           (5.0 - 10.0 * af) / 512.0, (-1.0 + 2.0 * af) / 1024.0]
    return a, [fb2, fb3, fb4, fb5]


def compact8_coeffs(af):
    """Interior and boundary coefficients, src/Compact8Filter.hpp:55-94."""
    a = [(93.0 + 70.0 * af) / 128.0, (7.0 + 18.0 * af) / 16.0, (-7.0 + 14.0 * af) / 32.0,
         (1.0 - 2.0 * af) / 16.0, (-1.0 + 2.0 * af) / 128.0]
    fb2 = [1.0 / 256.0 + 127.0 * af / 128.0, 31.0 / 32.0 + 1.0 * af / 16.0, 7.0 / 64.0 + 25.0 * af / 32.0,
           -7.0 / 32.0 + 7.0 * af / 16.0, 7.0 * (5.0 - 10.0 * af) / 128.0, -7.0 / 32.0 + 7.0 * af / 16.0,
           7.0 / 64.0 - 7.0 * af / 32.0, -1.0 / 32.0 + 1.0 * af / 16.0, 1.0 / 256.0 - 1.0 * af / 128.0]
    fb3 = [-1.0 / 256.0 + 1.0 * af / 128.0, 1.0 / 32.0 + 15.0 * af / 16.0, 57.0 / 64.0 + 7.0 * af / 32.0,
           7.0 / 32.0 + 9.0 * af / 16.0, 7.0 * (-5.0 + 10.0 * af) / 128.0, 7.0 / 32.0 - 7.0 * af / 16.0,
           -7.0 / 64.0 + 7.0 * af / 32.0, 1.0 / 32.0 - 1.0 * af / 16.0, -1.0 / 256.0 + 1.0 * af / 128.0]
    fb4 = [1.0 / 256.0 - 1.0 * af / 128.0, -1.0 / 32.0 + 1.0 * af / 16.0, 7.0 / 64.0 + 25.0 * af / 32.0,
           25.0 / 32.0 + 7.0 * af / 16.0, 35.0 / 128.0 + 29.0 * af / 64.0, -7.0 / 32.0 + 7.0 * af / 16.0,
           7.0 / 64.0 - 7.0 * af / 32.0, -1.0 / 32.0 + 1.0 * af / 16.0, 1.0 / 256.0 - 1.0 * af / 128.0]
    return a, [fb2, fb3, fb4]


def filter_lines(phi, ftype, af, bc):
    """One-direction compact filter on lines: src/Compact10Filter.cpp:5-141 and
    src/Compact8Filter.cpp:5-117 (periodic cyclic / Dirichlet solveTri)."""
    n = phi.shape[-1]
    if ftype == "COMPACT10":
        a, fbs = compact10_coeffs(af)
    elif ftype == "COMPACT8":
        a, fbs = compact8_coeffs(af)
    else:
        raise ValueError(ftype)
    H = len(a) - 1
    cc = [a[0]] + [a[k] / 2.0 for k in range(1, H + 1)]
    lo = np.full(n, af)
    up = np.full(n, af)
    dg = np.ones(n)
    # the reference sums the symmetric stencil from the far-left point to the far-right point
    rhs = np.zeros(phi.shape)
    if bc == PERIODIC:
        for s in range(-H, H + 1):
            rhs = rhs + cc[abs(s)] * _roll(phi, s)
        return cyclic(lo, dg, up, af, af, rhs)
    lo[0] = up[0] = lo[n - 1] = up[n - 1] = 0.0
    for s in range(-H, H + 1):
        rhs[..., H:n - H] = rhs[..., H:n - H] + cc[abs(s)] * phi[..., H + s:n - H + s]
    rhs[..., 0] = phi[..., 0]
    rhs[..., n - 1] = phi[..., n - 1]
    w = len(fbs[0])
    for r, fb in enumerate(fbs, start=1):
        acc = np.zeros(phi.shape[:-1])
        acc2 = np.zeros(phi.shape[:-1])
        for k in range(w):
            acc = acc + fb[k] * phi[..., k]
            acc2 = acc2 + fb[k] * phi[..., n - 1 - k]
        rhs[..., r] = acc
        rhs[..., n - 1 - r] = acc2
    return solve_tri(lo, dg, up, rhs)


def filt(f, d, ftype, af, bcs):
    """filterField along direction d (src/Compact10Filter.cpp:166-252): lines on
    a Dirichlet face of either other direction pass through unfiltered."""
    lines = _to_lines(f, d)
    out = filter_lines(lines, ftype, af, bcs[d])
    others = [o for o in range(3) if o != d]
    mask = np.zeros(f.shape, dtype=bool)
    for o in others:
        if bcs[o] == DIRICHLET:
            ax = _AXIS[o]
            sl0 = [slice(None)] * 3
            sl1 = [slice(None)] * 3
            sl0[ax] = 0
            sl1[ax] = f.shape[ax] - 1
            mask[tuple(sl0)] = True
            mask[tuple(sl1)] = True
    res = np.ascontiguousarray(_from_lines(out, d))
    res[mask] = f[mask]
    return res


# --------------------------------------------------------------------------
# DSM test filters (src/CommN5PadeTestFilter.{hpp,cpp},
# src/CommN5ExpTestFilter.{hpp,cpp}): commutative filters of filter-width
# ratio 2, with the same one-sided closures at Dirichlet ends.
# --------------------------------------------------------------------------
TF_B = [[31.0 / 32.0, 5.0 / 32.0, -5.0 / 16.0, 5.0 / 16.0, -5.0 / 32.0, 1.0 / 32.0],    # node 0 (w*_n1)
        [1.0 / 32.0, 27.0 / 32.0, 5.0 / 16.0, -5.0 / 16.0, 5.0 / 32.0, -1.0 / 32.0],    # node 1 (w*_n2)
        [-1.0 / 32.0, 5.0 / 32.0, 11.0 / 16.0, 5.0 / 16.0, -5.0 / 32.0, 1.0 / 32.0]]    # node 2 (w*_n3)
TF_W = [11.0 / 16.0, 15.0 / 64.0, -3.0 / 32.0, 1.0 / 64.0]                             # w0..w3
TF_WI = [7.0 / 24.0, 175.0 / 768.0, 5.0 / 48.0, 35.0 / 1536.0, 0.0, -1.0 / 1536.0]     # wi0..wi5
TF_V = (7.0 / 12.0, 0.0, 5.0 / 24.0)                                                    # v0, v1, v2


def _closure_rows(phi, rhs, rows):
    """Boundary rows of the test filters: node r on phi[0..5] and its mirror
    node N-1-r on phi[N-1], phi[N-2], ... (CommN5ExpTestFilter.cpp:22-48)."""
    n = phi.shape[-1]
    for r in rows:
        b = TF_B[r]
        acc = b[0] * phi[..., 0]
        acc2 = b[0] * phi[..., n - 1]
        for k in range(1, 6):
            acc = acc + b[k] * phi[..., k]
            acc2 = acc2 + b[k] * phi[..., n - 1 - k]
        rhs[..., r] = acc
        rhs[..., n - 1 - r] = acc2


def exp_test_filter_lines(phi, bc):
    """CommN5ExpTestFilter::FilterPeriodic / FilterDirichlet
    (src/CommN5ExpTestFilter.cpp:3-50): explicit 7-point filter."""
    n = phi.shape[-1]
    w = TF_W
    out = np.zeros(phi.shape)
    if bc == PERIODIC:
        acc = w[3] * _roll(phi, -3)
        for s in (-2, -1, 0, 1, 2, 3):
            acc = acc + w[abs(s)] * _roll(phi, s)
        return acc
    acc = w[3] * phi[..., 0:n - 6]
    for s in (-2, -1, 0, 1, 2, 3):
        acc = acc + w[abs(s)] * phi[..., 3 + s:n - 3 + s]
    out[..., 3:n - 3] = acc
    _closure_rows(phi, out, (0, 1, 2))
    return out


def pade_test_filter_lines(phi, bc):
    """CommN5PadeTestFilter::FilterPeriodic / FilterDirichlet
    (src/CommN5PadeTestFilter.cpp:3-130, LHS of CommN5PadeTestFilter.hpp:56-178):
    11-point RHS, pentadiagonal LHS (v2, v1, v0, v1, v2) with v1 = 0."""
    n = phi.shape[-1]
    v0, v1, v2 = TF_V
    wi = TF_WI
    dg = np.full(n, v0)
    lo, up = np.full(n, v1), np.full(n, v1)
    lo2, up2 = np.full(n, v2), np.full(n, v2)
    if bc == PERIODIC:
        rhs = wi[5] * _roll(phi, -5)
        for s in range(-4, 6):
            rhs = rhs + wi[abs(s)] * _roll(phi, s)
        return cyclic_penta(lo2, lo, dg, up, up2, rhs, [v2, v1, v2, v2, v1, v2])
    # nodes 0..4 and N-5..N-1 are explicitly filtered (identity LHS rows)
    for r in range(5):
        dg[r] = dg[n - 1 - r] = 1.0
        up[r] = up2[r] = 0.0
    lo[0:4] = 0.0
    lo2[0:3] = 0.0
    lo2[n - 7:n - 2] = 0.0
    lo[n - 6:n - 1] = 0.0
    up[n - 5:n - 1] = 0.0
    up2[n - 5:n - 2] = 0.0
    rhs = np.zeros(phi.shape)
    acc = wi[5] * phi[..., 0:n - 10]
    for s in range(-4, 6):
        acc = acc + wi[abs(s)] * phi[..., 5 + s:n - 5 + s]
    rhs[..., 5:n - 5] = acc
    _closure_rows(phi, rhs, (0, 1, 2))
    w = TF_W
    for r in (3, 4):   # 7-point rows (CommN5PadeTestFilter.cpp:106-111, :125-130)
        a = w[3] * phi[..., r - 3]
        a2 = w[3] * phi[..., n - 1 - r + 3]
        for s in (-2, -1, 0, 1, 2, 3):
            a = a + w[abs(s)] * phi[..., r + s]
            a2 = a2 + w[abs(s)] * phi[..., n - 1 - r - s]
        rhs[..., r] = a
        rhs[..., n - 1 - r] = a2
    return solve_penta(lo2, lo, dg, up, up2, rhs)


def test_filter(f, d, ftype, bcs):
    """filterField of the DSM test filter along d, with the Dirichlet-face
    pass-through of src/CommN5PadeTestFilter.cpp:134-241. ftype is the
    LES.DSMTESTFILTER value: 1 = Pade, 2 = explicit (src/DSMSGS.hpp:57-67)."""
    lines = _to_lines(f, d)
    out = pade_test_filter_lines(lines, bcs[d]) if ftype == 1 else exp_test_filter_lines(lines, bcs[d])
    others = [o for o in range(3) if o != d]
    mask = np.zeros(f.shape, dtype=bool)
    for o in others:
        if bcs[o] == DIRICHLET:
            ax = _AXIS[o]
            sl0 = [slice(None)] * 3
            sl1 = [slice(None)] * 3
            sl0[ax] = 0
            sl1[ax] = f.shape[ax] - 1
            mask[tuple(sl0)] = True
            mask[tuple(sl1)] = True
    res = np.ascontiguousarray(_from_lines(out, d))
    res[mask] = f[mask]
    return res


# --------------------------------------------------------------------------
# Ideal gas (src/IdealGas.hpp:9-80)
# --------------------------------------------------------------------------
GAMMA, PR = 1.4, 0.7
P_REF = 1.0 / GAMMA
R_GAS = P_REF / 1.0 / 1.0
CP = R_GAS * GAMMA / (GAMMA - 1.0)


def primitives(q, mu_ref):
    """updateNonConservedData, src/CurvilinearCSolver_Core.cpp:1158-1197."""
    rho, ru, rv, rw, re = q
    U, V, W = ru / rho, rv / rho, rw / rho
    p = (GAMMA - 1) * (re - 0.5 * rho * (U * U + V * V + W * W))
    T = p / (rho * R_GAS)
    mu = mu_ref * np.power(T / 1.0, 0.76)
    sos = np.sqrt(GAMMA * p / rho)
    return U, V, W, p, T, mu, sos


# --------------------------------------------------------------------------
# Time-integration coefficients (src/RK4.hpp:27-34, src/TVDRK3.hpp,
# src/KenRK4.hpp:30-40, src/LSLDDRK4.hpp:40-78)
# --------------------------------------------------------------------------
KENRK4_A = [0.0, -6234157559845.0 / 12983515589748.0, -6194124222391.0 / 4410992767914.0,
            -31623096876824.0 / 15682348800105.0, -12251185447671.0 / 11596622555746.0]
KENRK4_B = [494393426753.0 / 4806282396855.0, 4047970641027.0 / 5463924506627.0,
            9795748752853.0 / 13190207949281.0, 4009051133189.0 / 8539092990294.0,
            1348533437543.0 / 7166442652324.0]
LSLDD_A1 = [0.0, -0.60512264332862261228, -2.04375640234761394333, -0.74069990637544192841,
            -4.42317651302968168941]
LSLDD_B1 = [0.26874543888713438496, 0.8014706973220802933, 0.50515704269422722538,
            0.56235680379000296407, 0.05900655127758823335]
LSLDD_A2 = [0.0, -0.44127377153877382565, -1.073982008079781868, -1.7063570791256758809,
            -2.7979293162682443056, -4.0913537120919160454]
LSLDD_B2 = [0.11584888181285561688, 0.37287699051652864918, 0.73795368921435295698,
            0.57981109366311039538, 1.031284991300145194, 0.15]


@dataclass
class Config:
    """The MPI_3DCompact.in options the time step reads (src/Options.hpp:133-206)."""
    N: tuple = (16, 16, 16)                # (Nx, Ny, Nz)
    bc: tuple = (PERIODIC, PERIODIC, PERIODIC)
    fd: tuple = ("PADE6", "PADE6", "PADE6")
    filter: str = "COMPACT10"
    alphaF: float = 0.49
    mu_ref: float = 0.001
    rk: str = "RK4"
    ts_type: str = "CONST_CFL"
    cfl: float = 0.5
    dt: float = -1.0
    filter_step: int = 1
    substep_filtering: bool = False
    les: str = "NOMODEL"
    les_avg: str = "NONE"
    dsm_test_filter: int = 1               # LES.DSMTESTFILTER (1 Pade, 2 explicit)
    dsm_use_taukk: bool = True             # LES.DSMUSETAUKK
    # face kinds X0, X1, Y0, Y1, Z0, Z1 (src/Options.hpp:21-27); None: PERIODIC on
    # periodic directions, ADIABATIC_WALL on the others
    bc_kind: tuple = None
    # [SPONGE]: dict(kind="RECTILINEAR"|"CYLINDRICAL", strength, rect_perc[6], orient, cyl_axis[3], rmin)
    sponge: dict = None
    # periodic translation of each periodic direction's faces along its own axis
    # (BC.PERIODICDISP*), for the reference runs; None: the 2*pi HIT box
    periodic_box: tuple = None
    # full BC.PERIODICDISP{X,Y,Z}_{X,Y,Z} table (row = face pair, column =
    # component); None: periodic_box on the diagonal
    periodic_disp: tuple = None
    # [STATS]: dict(velocity=bool, thermo=bool, avg="NONE"|"XI1_AVG"|"XI2_AVG"|"XI3_AVG", interval=int)
    stats: dict = None
    # updateSponge after every step (commented out in the reference's postStep):
    # dict(avg_time=float, p_inf=float) or None
    sponge_relax: dict = None

    def kinds(self):
        if self.bc_kind is not None:
            return tuple(self.bc_kind)
        return tuple("PERIODIC" if self.bc[f // 2] == PERIODIC else "ADIABATIC_WALL" for f in range(6))


def _ramp(strength, s):
    return strength * (0.068 * np.power(s, 2.0) + 0.845 * np.power(s, 8.0))


def sponge_sigma(cfg, x, y, z):
    """SpongeBC::initRectSpongeBC / initCylSpongeBC (src/SpongeBC.cpp:65-262):
    sponge strength from the mesh coordinates (fields shaped (Nz, Ny, Nx))."""
    sp, k = cfg.sponge, cfg.kinds()
    X = (x, y, z)
    mn = [float(np.min(a)) for a in X]
    mx = [float(np.max(a)) for a in X]
    sigma = np.zeros(x.shape)
    st = sp.get("strength", 1.0)
    if sp.get("kind", "RECTILINEAR") == "RECTILINEAR":
        perc = sp.get("rect_perc", [0.0] * 6)
        for d in range(3):
            L0 = perc[2 * d] * (mx[d] - mn[d])
            L1 = perc[2 * d + 1] * (mx[d] - mn[d])
            if k[2 * d] == "SPONGE":
                dd = X[d] - mn[d]
                m = dd < L0
                sigma = np.where(m, np.fmax(_ramp(st, (L0 - dd) / L0), sigma), sigma)
            if k[2 * d + 1] == "SPONGE":
                dd = mx[d] - X[d]
                m = dd < L1
                sigma = np.where(m, np.fmax(_ramp(st, (X[d] - (mx[d] - L1)) / L1), sigma), sigma)
        return sigma
    if sp.get("orient", 2) != 2:
        raise NotImplementedError("cylindrical sponge orientation")
    ax = sp["cyl_axis"]
    rmax = max(max(abs(mn[0] - ax[0]), abs(mx[0] - ax[0])), max(abs(mn[1] - ax[1]), abs(mx[1] - ax[1])))
    rmin = sp["rmin"]
    if k[3] == "SPONGE":
        r = np.sqrt(np.power(x - ax[0], 2.0) + np.power(y - ax[1], 2.0))
        m = r > rmin
        sigma = np.where(m, np.fmax(_ramp(st, (r - rmin) / (rmax - rmin)), sigma), sigma)
    return sigma


_WALLS = ("ADIABATIC_WALL", "CONST_T_WALL", "MOVING_ADIABATIC_WALL")


def _face_slices(f, shape):
    """(face slice, slices of the points 1..6 inward) of face f on (Nz, Ny, Nx) arrays."""
    ax = _AXIS[f // 2]
    n = shape[ax]
    side = f % 2
    sl = [slice(None)] * 3
    sl[ax] = n - 1 if side else 0
    inward = []
    for m in range(1, 7):
        t = [slice(None)] * 3
        t[ax] = n - 1 - m if side else m
        inward.append(tuple(t))
    return tuple(sl), inward


def calc_neumann(scheme, f):
    """calcNeumann (src/Pade6.cpp:395-397, src/Penta10.cpp:284-286, src/CD2.cpp:183)."""
    if scheme == "CD2":
        return (f[0] * 4.0 - f[1] * 1.0) / 3.0
    return (f[0] * 360.0 - f[1] * 450.0 + f[2] * 400.0 - f[3] * 225.0 + f[4] * 72.0 - f[5] * 10.0) / 147.0


@dataclass
class State:
    q1: list                                 # rho1, rhoU1, rhoV1, rhoW1, rhoE1
    qk: list = None
    k2: list = None
    q2: list = None
    time: float = 0.0
    time_step: int = 0
    filter_time_step: int = 0
    dt: float = 0.0
    history: list = field(default_factory=list)


class Oracle:
    """The CurvilinearCSolver time step on one block (src/CurvilinearCSolver.hpp:25-379)."""

    def __init__(self, cfg: Config, metrics=None, sigma=None):
        self.cfg = cfg
        self.sigma = sigma
        self.kinds = cfg.kinds()
        self.walls = any(k in _WALLS for k in self.kinds)
        self.sponge_on = any(k == "SPONGE" for k in self.kinds)
        if self.sponge_on and sigma is None:
            raise ValueError("sponge faces need sigma")
        Nx, Ny, Nz = cfg.N
        # Domain with Lx=Ly=Lz=1 (src/Domain.hpp:45-79)
        self.dxi = [1.0 / n if b == PERIODIC else 1.0 / (n - 1.0) for n, b in zip(cfg.N, cfg.bc)]
        if metrics is None:
            raise ValueError("metrics (J, J11..J33) are required")
        self.J = metrics[0]
        self.Jm = [[metrics[1], metrics[2], metrics[3]],
                   [metrics[4], metrics[5], metrics[6]],
                   [metrics[7], metrics[8], metrics[9]]]
        self.pr_t = 0.9

    # -- operators --------------------------------------------------------
    def d(self, f, direction):
        c = self.cfg
        return deriv(f, direction, c.fd[direction], c.bc[direction], self.dxi[direction])

    def grad(self, f):
        return [self.d(f, 0), self.d(f, 1), self.d(f, 2)]

    def f3(self, f, order, ftype, af):
        for d in order:
            f = filt(f, d, ftype, af, self.cfg.bc)
        return f

    # -- SGS (src/VremanSGS.hpp:43-96, src/AbstractSGS.cpp:13-160) ---------
    def vreman(self, gu, rho):
        J = self.J
        vol = self.dxi[0] * self.dxi[1] * self.dxi[2] / J
        d1 = np.power(vol, 1.0 / 3.0) ** 2
        d1v1, d2v1, d3v1 = gu[0][0], gu[0][1], gu[0][2]
        d1v2, d2v2, d3v2 = gu[1][0], gu[1][1], gu[1][2]
        d1v3, d2v3, d3v3 = gu[2][0], gu[2][1], gu[2][2]
        b11 = d1 * d1v1 * d1v1 + d1 * d2v1 * d2v1 + d1 * d3v1 * d3v1
        b12 = d1 * d1v1 * d1v2 + d1 * d2v1 * d2v2 + d1 * d3v1 * d3v2
        b13 = d1 * d1v1 * d1v3 + d1 * d2v1 * d2v3 + d1 * d3v1 * d3v3
        b22 = d1 * d1v2 * d1v2 + d1 * d2v2 * d2v2 + d1 * d3v2 * d3v2
        b23 = d1 * d1v2 * d1v3 + d1 * d2v2 * d2v3 + d1 * d3v2 * d3v3
        b33 = d1 * d1v3 * d1v3 + d1 * d2v3 * d2v3 + d1 * d3v3 * d3v3
        # the reference sums d2v3^2 twice and omits d3v2^2 (VremanSGS.hpp:74-76)
        abeta = (d1v1 * d1v1 + d1v2 * d1v2 + d1v3 * d1v3 + d2v1 * d2v1 + d2v2 * d2v2 + d2v3 * d2v3
                 + d3v1 * d3v1 + d2v3 * d2v3 + d3v3 * d3v3)
        bbeta = b11 * b22 - (b12 * b12) + b11 * b33 - (b13 * b13) + b22 * b33 - (b23 * b23)
        eps = 1e-12
        bbeta = np.where(bbeta < eps, eps, bbeta)
        ss = np.sqrt(bbeta / (abeta + eps))
        c = 2.5 * 0.17 * 0.17
        mu_sgs = c * rho * ss
        mu_sgs = np.minimum(mu_sgs, 0.05 * d1 * np.sqrt(2.0 * abeta))
        # VremanSGS averages with a Compact10 filter of alpha = -0.49 (VremanSGS.hpp:38-40)
        return self.average(mu_sgs, lambda f, d: filt(f, d, "COMPACT10", -0.49, self.cfg.bc))

    def average(self, phi, filt1):
        """AbstractSGS::doAveraging (src/AbstractSGS.cpp:13-160) for LESAVERAGING:
        XI1/XI2/XI3 replace phi by its mean along xi1/xi2/xi3, GLOBAL by its
        mean over the block, LOCAL applies the SGS model's filter along Y, Z, X
        (filt1(f, d) filters f along d); NONE leaves it."""
        a = self.cfg.les_avg
        if a == "NONE":
            return phi
        if a == "LOCAL":
            for d in (1, 2, 0):
                phi = filt1(phi, d)
            return phi
        if a == "GLOBAL":
            return np.full(phi.shape, np.sum(phi) / phi.size)
        ax = {"XI1_AVG": 2, "XI2_AVG": 1, "XI3_AVG": 0}[a]
        m = np.sum(phi / phi.shape[ax], axis=ax, keepdims=True)
        return np.broadcast_to(m, phi.shape).copy()

    # -- dynamic Smagorinsky (src/DSMSGS.hpp:130-447) -------------------------
    def _fq(self, phi):
        """DSMSGS::filterQuantity: test filter along Y, Z, X (DSMSGS.hpp:120-128)."""
        for d in (1, 2, 0):
            phi = test_filter(phi, d, self.cfg.dsm_test_filter, self.cfg.bc)
        return phi

    def dsm_mu_taukk(self, gu, rho, ru, rv, rw):
        """DSMSGS::calcMuSGSTaukk (DSMSGS.hpp:130-331): returns mu_sgs, taukk and
        the filtered quantities calcKSGS reuses."""
        tfr2 = 2.0 * 2.0
        avg = lambda f: self.average(f, lambda g, d: test_filter(g, d, self.cfg.dsm_test_filter, self.cfg.bc))
        S00, S11, S22 = gu[0][0], gu[1][1], gu[2][2]
        S01 = 0.5 * (gu[0][1] + gu[1][0])
        S02 = 0.5 * (gu[0][2] + gu[2][0])
        S12 = 0.5 * (gu[1][2] + gu[2][1])
        Smag = np.sqrt(2.0 * (S00 * S00 + S11 * S11 + S22 * S22) + 4.0 * (S01 * S01 + S02 * S02 + S12 * S12))
        tr = S00 + S11 + S22
        M2 = [2.0 * rho * Smag * (S00 - (1.0 / 3.0) * tr), 2.0 * rho * Smag * S01, 2.0 * rho * Smag * S02,
              2.0 * rho * Smag * (S11 - (1.0 / 3.0) * tr), 2.0 * rho * Smag * S12,
              2.0 * rho * Smag * (S22 - (1.0 / 3.0) * tr)]
        M = [self._fq(m) for m in M2]              # M00, M01, M02, M11, M12, M22
        rho_hat = self._fq(rho)
        Sh = [self._fq(x) for x in (S00, S01, S02, S11, S12, S22)]
        Smag_hat = self._fq(Smag)
        trh = Sh[0] + Sh[3] + Sh[5]
        c = 2.0 * tfr2 * rho_hat * Smag_hat
        M = [M[0] - c * (Sh[0] - (1.0 / 3.0) * trh), M[1] - c * Sh[1], M[2] - c * Sh[2],
             M[3] - c * (Sh[3] - (1.0 / 3.0) * trh), M[4] - c * Sh[4], M[5] - c * (Sh[5] - (1.0 / 3.0) * trh)]
        Lt = [ru * ru / rho, ru * rv / rho, ru * rw / rho, rv * rv / rho, rv * rw / rho, rw * rw / rho]
        L = [self._fq(x) for x in Lt]
        ruh, rvh, rwh = self._fq(ru), self._fq(rv), self._fq(rw)
        L = [L[0] - ruh * ruh / rho_hat, L[1] - ruh * rvh / rho_hat, L[2] - ruh * rwh / rho_hat,
             L[3] - rvh * rvh / rho_hat, L[4] - rvh * rwh / rho_hat, L[5] - rwh * rwh / rho_hat]
        if self.cfg.dsm_use_taukk:
            alpha_hat = self._fq(2.0 * rho * Smag * Smag)
            CIdenom = 2.0 * tfr2 * rho_hat * Smag_hat * Smag_hat - alpha_hat
        Lkk = L[0] + L[3] + L[5]
        LijMij = ((L[0] - (1.0 / 3.0) * Lkk) * M[0] + (L[3] - (1.0 / 3.0) * Lkk) * M[3]
                  + (L[5] - (1.0 / 3.0) * Lkk) * M[5] + 2.0 * L[1] * M[1] + 2.0 * L[2] * M[2] + 2.0 * L[4] * M[4])
        MijMij = (M[0] * M[0] + M[3] * M[3] + M[5] * M[5] + 2.0 * M[1] * M[1] + 2.0 * M[2] * M[2]
                  + 2.0 * M[4] * M[4])
        if self.cfg.dsm_use_taukk:
            Lkk_avg = avg(Lkk)
            CIdenom_avg = avg(CIdenom)
        LijMij_avg = avg(LijMij)
        MijMij_avg = avg(MijMij)
        mu_sgs = rho * Smag * LijMij_avg / MijMij_avg
        if self.cfg.dsm_use_taukk:
            taukk = 2.0 * rho * Smag * Smag * Lkk_avg / CIdenom_avg
        else:
            taukk = np.zeros(rho.shape)
        ctx = dict(Smag=Smag, rho_hat=rho_hat, Smag_hat=Smag_hat, ruh=ruh, rvh=rvh, rwh=rwh)
        return mu_sgs, taukk, ctx

    def dsm_ksgs(self, gradT, rho, ru, rv, rw, T, ctx):
        """DSMSGS::calcKSGS (DSMSGS.hpp:333-443); K_i divides by rho, not
        rho_hat (DSMSGS.hpp:406-408)."""
        tfr2 = 2.0 * 2.0
        avg = lambda f: self.average(f, lambda g, d: test_filter(g, d, self.cfg.dsm_test_filter, self.cfg.bc))
        Smag, rho_hat, Smag_hat = ctx["Smag"], ctx["rho_hat"], ctx["Smag_hat"]
        NR = [self._fq(rho * Smag * g) for g in gradT]
        KR = [self._fq(x * T) for x in (ru, rv, rw)]
        rhoT_hat = self._fq(rho * T)
        gh = [self._fq(g) for g in gradT]
        N = [tfr2 * rho_hat * Smag_hat * gh[i] - NR[i] for i in range(3)]
        uh = (ctx["ruh"], ctx["rvh"], ctx["rwh"])
        K = [-uh[i] * rhoT_hat / rho + KR[i] for i in range(3)]
        NiNi = N[0] * N[0] + N[1] * N[1] + N[2] * N[2]
        NiKi = K[0] * N[0] + K[1] * N[1] + K[2] * N[2]
        NiNi_avg = avg(NiNi)
        NiKi_avg = avg(NiKi)
        return -CP * (NiKi_avg / NiNi_avg) * rho * Smag

    # -- one stage: preStepDerivatives + solveEqnSet (Core.cpp:468-947) ----
    def rhs(self, qP, k2, prims=None):
        """preStepDerivatives + solveEqnSet + postStepBCHandling on the stage
        state qP with the primitives `prims` (U, V, W, p, T, mu, sos) of
        updateNonConservedData as preStepBCHandling left them."""
        c = self.cfg
        J, Jm = self.J, self.Jm
        rhoP, ruP, rvP, rwP, reP = qP
        U, V, W, p, T, mu, sos = prims if prims is not None else primitives(qP, c.mu_ref)
        Ucurv = Jm[0][0] * U + Jm[0][1] * V + Jm[0][2] * W
        Vcurv = Jm[1][0] * U + Jm[1][1] * V + Jm[1][2] * W
        Wcurv = Jm[2][0] * U + Jm[2][1] * V + Jm[2][2] * W
        dU, dV, dW = self.grad(U), self.grad(V), self.grad(W)

        def phys(dq, j):   # Core.cpp:548-561: d/dx_j = sum_i J_ij d/dxi_i
            return Jm[0][j] * dq[0] + Jm[1][j] * dq[1] + Jm[2][j] * dq[2]
        gu = [[phys(dU, 0), phys(dU, 1), phys(dU, 2)],
              [phys(dV, 0), phys(dV, 1), phys(dV, 2)],
              [phys(dW, 0), phys(dW, 1), phys(dW, 2)]]
        les = c.les != "NOMODEL"
        mu_sgs = k_sgs = None
        if c.les == "VREMAN":
            mu_sgs = self.vreman(gu, rhoP)
        elif c.les == "DSM":
            mu_sgs, taukk, ctx = self.dsm_mu_taukk(gu, rhoP, ruP, rvP, rwP)
            # pressure with the SGS normal stresses; T, mu follow (Core.cpp:573-584)
            p = p - 0.5 * taukk
            T = p / (rhoP * R_GAS)
            mu = c.mu_ref * np.power(T / 1.0, 0.76)
        elif les:
            raise NotImplementedError(c.les)
        dT = self.grad(T)
        if c.les == "DSM":
            gradT = [phys(dT, 0), phys(dT, 1), phys(dT, 2)]   # Core.cpp:596-600
            k_sgs = self.dsm_ksgs(gradT, rhoP, ruP, rvP, rwP, T, ctx)
        dUdx, dUdy, dUdz = gu[0]
        dVdx, dVdy, dVdz = gu[1]
        dWdx, dWdy, dWdz = gu[2]
        t11 = (4.0 / 3.0) * dUdx - (2.0 / 3.0) * dVdy - (2.0 / 3.0) * dWdz
        t22 = -(2.0 / 3.0) * dUdx + (4.0 / 3.0) * dVdy - (2.0 / 3.0) * dWdz
        t33 = -(2.0 / 3.0) * dUdx - (2.0 / 3.0) * dVdy + (4.0 / 3.0) * dWdz
        t12 = dUdy + dVdx
        t13 = dUdz + dWdx
        t23 = dVdz + dWdy
        if les:
            mu_eff = mu + mu_sgs
            if c.les == "DSM":
                k_eff = CP * mu / PR + k_sgs               # Core.cpp:637-639
            else:
                k_eff = CP * (mu / PR + mu_sgs / self.pr_t)
            mu_eff = np.where(mu_eff < 0.0, 0.0, mu_eff)
            k_eff = np.where(k_eff < 0.0, 0.0, k_eff)
        else:
            mu_eff = mu
            k_eff = (CP / PR) * mu
        t11, t22, t33, t12, t13, t23 = (t * mu_eff for t in (t11, t22, t33, t12, t13, t23))
        t21, t31, t32 = t12, t13, t23
        q1 = k_eff * (Jm[0][0] * dT[0] + Jm[1][0] * dT[1] + Jm[2][0] * dT[2])
        q2 = k_eff * (Jm[0][1] * dT[0] + Jm[1][1] * dT[1] + Jm[2][1] * dT[2])
        q3 = k_eff * (Jm[0][2] * dT[0] + Jm[1][2] * dT[1] + Jm[2][2] * dT[2])
        b1 = U * t11 + V * t12 + W * t13 + q1
        b2 = U * t21 + V * t22 + W * t23 + q2
        b3 = U * t31 + V * t32 + W * t33 + q3
        iJ = 1.0 / J
        cont = [iJ * (rhoP * Ucurv), iJ * (rhoP * Vcurv), iJ * (rhoP * Wcurv)]

        def mom(rq, tcol, row):
            F1 = rq * Ucurv + Jm[0][row] * p
            F2 = rq * Vcurv + Jm[1][row] * p
            F3 = rq * Wcurv + Jm[2][row] * p
            G1 = Jm[0][0] * tcol[0] + Jm[0][1] * tcol[1] + Jm[0][2] * tcol[2]
            G2 = Jm[1][0] * tcol[0] + Jm[1][1] * tcol[1] + Jm[1][2] * tcol[2]
            G3 = Jm[2][0] * tcol[0] + Jm[2][1] * tcol[1] + Jm[2][2] * tcol[2]
            return [iJ * (F1 - G1), iJ * (F2 - G2), iJ * (F3 - G3)]
        m1 = mom(ruP, (t11, t21, t31), 0)
        m2 = mom(rvP, (t12, t22, t32), 1)
        m3 = mom(rwP, (t13, t23, t33), 2)
        F1, F2, F3 = (reP + p) * Ucurv, (reP + p) * Vcurv, (reP + p) * Wcurv
        G1 = Jm[0][0] * b1 + Jm[0][1] * b2 + Jm[0][2] * b3
        G2 = Jm[1][0] * b1 + Jm[1][1] * b2 + Jm[1][2] * b3
        G3 = Jm[2][0] * b1 + Jm[2][1] * b2 + Jm[2][2] * b3
        en = [iJ * (F1 - G1), iJ * (F2 - G2), iJ * (F3 - G3)]
        comps = [cont, m1, m2, m3, en]
        div = [[self.d(comp[0], 0), self.d(comp[1], 1), self.d(comp[2], 2)] for comp in comps]
        dt = self.state.dt
        # sponge source sigma (avg - phi) (src/CurvilinearCSolver.hpp:293-295)
        if self.sponge_on:
            spg = [self.sigma * (self.spg_avg[e] - qP[e]) for e in range(5)]
        else:
            spg = [0.0] * 5
        # solveContinuity/X/Y/ZMomentum/Energy, Core.cpp:790-947 (zero hooks)
        new = [None] * 5
        new[0] = dt * J * (-div[0][0] - div[0][1] - div[0][2] + (spg[0] + 0.0) / J)
        for e in (1, 2, 3):
            # momentum accumulates into the previous k2 (Core.cpp:839,872,904)
            t = k2[e] + (-div[e][0] - div[e][1] - div[e][2] + (spg[e] + 0.0) / J)
            new[e] = t * (dt * J)
        t = -div[4][0] - div[4][1] - div[4][2] + (spg[4] + 0.0) / J
        new[4] = t * (dt * J)
        # postStepBCHandling (src/CurvilinearCSolver_BC.cpp:702-842): walls keep the
        # wall-normal mass-flux derivative in the continuity k2, sponge faces zero all
        if self.walls or self.sponge_on:
            for f in range(6):
                if self.kinds[f] in _WALLS:
                    sl, _ = _face_slices(f, rhoP.shape)
                    new[0][sl] = -dt * J[sl] * div[0][f // 2][sl]
                    for e in (1, 2, 3, 4):
                        new[e][sl] = 0.0
            for f in range(6):
                if self.kinds[f] == "SPONGE":
                    sl, _ = _face_slices(f, rhoP.shape)
                    for e in range(5):
                        new[e][sl] = 0.0
        return new

    def wall_prestep(self, qP, prims):
        """preStepBCHandling (src/CurvilinearCSolver_BC.cpp:372-700): no-slip walls
        of faces X0..Z1, then moving walls; modifies the stage state qP in place
        and returns the primitives with U, V, W, T, p replaced on the walls (mu
        and sos keep their values)."""
        U, V, W, p, T, mu, sos = [a.copy() if isinstance(a, np.ndarray) else a for a in prims]
        rho, ru, rv, rw, re = qP
        for pass_ in (0, 1):
            for f in range(6):
                k = self.kinds[f]
                if pass_ == 0 and k not in ("ADIABATIC_WALL", "CONST_T_WALL"):
                    continue
                if pass_ == 1 and k != "MOVING_ADIABATIC_WALL":
                    continue
                sl, inward = _face_slices(f, rho.shape)
                if k != "CONST_T_WALL":
                    T[sl] = calc_neumann(self.cfg.fd[f // 2], [T[t] for t in inward])
                U[sl] = 0.0
                V[sl] = 0.0
                W[sl] = 0.0
                ru[sl] = 0.0
                rv[sl] = 0.0
                rw[sl] = 0.0
                p[sl] = rho[sl] * R_GAS * T[sl]
                re[sl] = p[sl] / (GAMMA - 1.0) + 0.5 * rho[sl] * (U[sl] * U[sl] + V[sl] * V[sl] + W[sl] * W[sl])
        return U, V, W, p, T, mu, sos

    # -- time-step bookkeeping ---------------------------------------------
    def cfl(self, q):
        """calcDtFromCFL, Core.cpp:189-237 (diagonal metrics only)."""
        c, st = self.cfg, self.state
        U, V, W, p, T, mu, sos = self._prims
        uc = (self.Jm[0][0] * (np.abs(U) + sos) / self.dxi[0] + self.Jm[1][1] * (np.abs(V) + sos) / self.dxi[1]
              + self.Jm[2][2] * (np.abs(W) + sos) / self.dxi[2])
        m = float(np.max(uc))
        if c.ts_type == "CONST_CFL":
            st.dt = c.cfl / m
        else:
            st.dt = c.dt
        if st.time_step == self.start_step:
            st.time_step += 1
        else:
            st.time_step += 1
            st.time += st.dt

    def filter_conserved(self, qin, last):
        """filterConservedData, Core.cpp:949-1155: direction order rotates with
        filterTimeStep % 3 (1: Y,Z,X; 2: Z,X,Y; 0: X,Y,Z); otherwise copy."""
        c, st = self.cfg, self.state
        if st.time_step % c.filter_step == 0:
            st.filter_time_step += 1
            r = st.filter_time_step % 3
            order = (1, 2, 0) if r == 1 else ((2, 0, 1) if r == 2 else (0, 1, 2))
            return [self.f3(f, order, c.filter, c.alphaF) for f in qin]
        return [f.copy() for f in qin] if last else qin

    def init(self, rho0, U0, V0, W0, p0, time=0.0, time_step=0):
        """setInitialConditions, src/CurvilinearCSolver_BC.cpp:3-59 (periodic:
        no walls, no sponge)."""
        z = np.zeros_like(rho0)
        if self.walls:
            # wall conditions of setInitialConditions (src/CurvilinearCSolver_BC.cpp:60-323):
            # on X1 the Neumann temperature is taken for CONST_T_WALL (:98)
            U0, V0, W0 = U0.copy(), V0.copy(), W0.copy()
            T = p0 / (rho0 * R_GAS)
            mu_init = self.cfg.mu_ref * np.power(T / 1.0, 0.76)   # mu is not updated after the walls
            for pass_ in (0, 1):
                for f in range(6):
                    k = self.kinds[f]
                    if pass_ == 0 and k not in ("ADIABATIC_WALL", "CONST_T_WALL"):
                        continue
                    if pass_ == 1 and k != "MOVING_ADIABATIC_WALL":
                        continue
                    sl, inward = _face_slices(f, rho0.shape)
                    U0[sl] = 0.0
                    V0[sl] = 0.0
                    W0[sl] = 0.0
                    neumann = pass_ == 1 or (k == "CONST_T_WALL" if f == 1 else k == "ADIABATIC_WALL")
                    if neumann:
                        T[sl] = calc_neumann(self.cfg.fd[f // 2], [T[t] for t in inward])
            p0 = rho0 * R_GAS * T
        rhoE = p0 / (GAMMA - 1.0) + 0.5 * rho0 * (U0 * U0 + V0 * V0 + W0 * W0)
        q1 = [rho0.copy(), rho0 * U0, rho0 * V0, rho0 * W0, rhoE]
        if self.sponge_on:
            self.spg_avg = [a.copy() for a in q1]
        self.state = State(q1=q1, qk=[z.copy() for _ in range(5)], k2=[z.copy() for _ in range(5)],
                           q2=[z.copy() for _ in range(5)], time=time, time_step=time_step)
        self.start_step = time_step
        self.stats = Stats(self.cfg.stats, rho0.shape, time) if self.cfg.stats else None
        T0 = p0 / (rho0 * R_GAS)
        self._prims = (U0, V0, W0, p0, T0, self.cfg.mu_ref * np.power(T0, 0.76), np.sqrt(GAMMA * p0 / rho0))
        if self.walls:
            # arrays as setInitialConditions leaves them: wall U, V, W, T; p and sos
            # from rho and T; mu still that of the initial temperature
            self._prims = (U0, V0, W0, p0, T, mu_init, np.sqrt(GAMMA * p0 / rho0))

    def _stage(self, qP, rk_step, last, update):
        st = self.state
        prims = self.wall_prestep(qP, self._prims) if self.walls else self._prims
        st.k2 = self.rhs(qP, st.k2, prims)
        update(rk_step)
        if last or self.cfg.substep_filtering:
            if last:
                st.q1 = self.filter_conserved(st.q2, True)
            else:
                st.qk = self.filter_conserved(st.qk, False)
        src = st.q1 if last else st.qk
        self._prims = primitives(src, self.cfg.mu_ref)

    def step(self):
        """One time step then postStep (src/CurvilinearCSolver.hpp:355-375): the
        sponge relaxation when switched on and the statistics update every
        STATS.INTERVAL steps. The statistics read the primitives of the
        filtered state and rho2, which the relaxation leaves as they were, so
        they are taken before it."""
        self._advance()
        st = self.state
        if self.stats is not None and st.time_step % self.stats.interval == 0:
            self.stats.update(st.time, st.q1, st.q2)
        if self.cfg.sponge_relax and self.sponge_on:
            self.update_sponge()

    def update_sponge(self):
        """CurvilinearCSolver::updateSponge (src/CurvilinearCSolver_BC.cpp:843-928):
        the target relaxes toward rho1..rhoE1 with eps = 1/(avgT/dt + 1), its
        energy is blended toward the back pressure (epsP = 0.005,
        src/SpongeBC.cpp:37), and the SPONGE faces take the target state.
        Only rho1..rhoE1 change: the primitives of the filtered state, which
        the next step's CFL and first-stage derivatives read, stay as they were."""
        st, sr = self.state, self.cfg.sponge_relax
        eps = 1.0 / (sr.get("avg_time", 1.0) / st.dt + 1.0)
        a = [self.spg_avg[v] + eps * (st.q1[v] - self.spg_avg[v]) for v in range(5)]
        eps_p, p_inf = 0.005, sr.get("p_inf", 1.0 / 1.4)
        a[4] = eps_p * a[4] + (1.0 - eps_p) * (p_inf / (GAMMA - 1.0) + 0.5 * (a[1] * a[1] + a[2] * a[2] + a[3] * a[3]) / a[0])
        self.spg_avg = a
        for f in range(6):
            if self.kinds[f] == "SPONGE":
                sl = _face_slices(f, a[0].shape)[0]
                for v in range(5):
                    st.q1[v][sl] = a[v][sl]

    def _advance(self):
        """One time step (or the LSLDDRK4 two-step pair's half): src/RK4.hpp:127-178,
        src/TVDRK3.hpp, src/KenRK4.hpp:154-217, src/LSLDDRK4.hpp:324-459."""
        c, st = self.cfg, self.state
        self.cfl(st.q1)
        if c.rk == "RK4":
            a = [1.0 / 6.0, 1.0 / 3.0, 1.0 / 3.0, 1.0 / 6.0]
            b = [0.5, 0.5, 1.0]

            def upd(s):   # RK4.hpp:47-125
                k2 = st.k2
                if s == 1:
                    st.q2 = [st.q1[i] + a[0] * k2[i] for i in range(5)]
                    st.qk = [st.q1[i] + b[0] * k2[i] for i in range(5)]
                elif s in (2, 3):
                    st.q2 = [st.q2[i] + a[s - 1] * k2[i] for i in range(5)]
                    st.qk = [st.q1[i] + b[s - 1] * k2[i] for i in range(5)]
                else:
                    st.q2 = [st.q2[i] + a[3] * k2[i] for i in range(5)]
            for s in range(1, 5):
                self._stage(st.q1 if s == 1 else st.qk, s, s == 4, upd)
        elif c.rk == "TVDRK3":
            def upd(s):   # TVDRK3.hpp:50-133
                k2 = st.k2
                if s == 1:
                    st.qk = [st.q1[i] + 1.0 * k2[i] for i in range(5)]
                elif s == 2:
                    st.qk = [(3.0 / 4.0) * st.q1[i] + (1.0 / 4.0) * st.qk[i] + (1.0 / 4.0) * k2[i] for i in range(5)]
                else:
                    st.q2 = [(1.0 / 3.0) * st.q1[i] + (2.0 / 3.0) * st.qk[i] + (2.0 / 3.0) * k2[i]
                             for i in range(5)]
            for s in range(1, 4):
                self._stage(st.q1 if s == 1 else st.qk, s, s == 3, upd)
        elif c.rk in ("KENRK4", "LSLDDRK4"):
            if c.rk == "KENRK4":
                A, B = KENRK4_A, KENRK4_B
            else:
                half = getattr(self, "_lsldd_half", 1)
                A, B = (LSLDD_A1, LSLDD_B1) if half == 1 else (LSLDD_A2, LSLDD_B2)
            ns = len(A)

            def upd(s):   # 2N-storage form: KenRK4.hpp:53-152, LSLDDRK4.hpp:93-320
                k2 = st.k2
                if s == 1:
                    st.qk = [st.q1[i] + B[0] * k2[i] for i in range(5)]
                    st.q1 = [k2[i].copy() for i in range(5)]
                else:
                    st.q1 = [k2[i] + A[s - 1] * st.q1[i] for i in range(5)]
                    if s < ns:
                        st.qk = [st.qk[i] + B[s - 1] * st.q1[i] for i in range(5)]
                    else:
                        st.q2 = [st.qk[i] + B[s - 1] * st.q1[i] for i in range(5)]
            for s in range(1, ns + 1):
                self._stage(st.q1 if s == 1 else st.qk, s, s == ns, upd)
            if c.rk == "LSLDDRK4":
                self._lsldd_half = 2 if getattr(self, "_lsldd_half", 1) == 1 else 1
        else:
            raise ValueError(c.rk)

    def stages_per_step(self):
        c = self.cfg
        if c.rk == "RK4":
            return 4
        if c.rk == "TVDRK3":
            return 3
        if c.rk == "KENRK4":
            return 5
        return 5 if getattr(self, "_lsldd_half", 1) == 1 else 6


def ogrid_mesh(N, r0=0.5, ratio=1.08, span=2.0):
    """O-grid around a cylinder of radius r0: xi1 = theta (periodic, internally),
    xi2 = r (geometric spacing, wall at r0), xi3 = z (periodic, `span` long);
    coordinates shaped (Nz, Ny, Nx)."""
    Nx, Ny, Nz = N
    th = 2.0 * math.pi * np.arange(Nx) / Nx
    r = r0 * np.cumprod(np.concatenate([[1.0], np.full(Ny - 1, ratio)]))
    zz = span * np.arange(Nz) / Nz
    Z, Rr, TH = np.meshgrid(zz, r, th, indexing="ij")
    return Rr * np.cos(TH), Rr * np.sin(TH), Z


# --------------------------------------------------------------------------
# Grid metrics (src/AbstractSingleBlockMesh.cpp:23-1308, :2019-2083)
# --------------------------------------------------------------------------
def periodic_disp_table(cfg: Config):
    """BC.PERIODICDISP* as the reference runs set them: cfg.periodic_disp, else
    periodic_box (or 2*pi) on the diagonal of each PERIODIC face pair."""
    kinds = cfg.kinds()
    t = np.zeros((3, 3))
    for d in range(3):
        if kinds[2 * d] == "PERIODIC":
            if cfg.periodic_disp is not None:
                t[d] = cfg.periodic_disp[d]
            else:
                t[d, d] = (cfg.periodic_box[d] if cfg.periodic_box is not None else 2.0 * math.pi)
    return t


def periodic_translations(cfg: Config):
    """handlePeriodicStuff (src/AbstractSingleBlockMesh.cpp:2019-2083): the
    translation of each PERIODIC_SOLVE direction. The xi1 test reads the Y
    faces (:2034), so an x-periodic block takes PERIODICDISPX only when its Y
    faces are PERIODIC; INTERNALLY_PERIODIC faces translate by zero; any other
    combination leaves the translation unset in the reference (zero here)."""
    kinds = cfg.kinds()
    disp = periodic_disp_table(cfg)
    T = np.zeros((3, 3))
    for d in range(3):
        if cfg.bc[d] != PERIODIC:
            continue
        test = 2 if d == 0 else 2 * d       # the xi1 branch looks at Y0/Y1
        if kinds[test] == "PERIODIC" and kinds[test + 1] == "PERIODIC":
            T[d] = disp[d]
        # INTERNALLY_PERIODIC and the unset case: zero
    return T


def _tpb_lines(phi, gm, gp, scheme, dh):
    """calc1stDeriv_TPB of periodic lines (src/Pade6.cpp:220-249,359-363,
    src/Penta10.cpp:175-207,263-269, src/CD2.cpp:144-150): the RHS stencil reads
    the ghost values gm[..., m-1] = Nm_m (before index 0) and gp[..., m-1] =
    Np_m (after index N-1) instead of the wrapped line values."""
    n = phi.shape[-1]
    if scheme == "CD2":
        out = cd2_deriv_lines(phi, dh, PERIODIC)
        a, c = -0.5, 0.5
        out[..., 0] = (a * gm[..., 0] + c * phi[..., 1]) / dh
        out[..., n - 1] = (a * phi[..., n - 2] + c * gp[..., 0]) / dh
        return out
    if scheme == "PADE6":
        a_1d, b_1d = 14.0 / 9.0, 1.0 / 9.0
        st = [-b_1d / 4.0, -a_1d / 2.0, 0.0, a_1d / 2.0, b_1d / 4.0]
        H = 2
    else:
        a, b, c = 17.0 / 12.0, 101.0 / 150.0, 1.0 / 100.0
        st = [-c / 6.0, -b / 4.0, -a / 2.0, 0.0, a / 2.0, b / 4.0, c / 6.0]
        H = 3
    ext = np.concatenate([gm[..., ::-1], phi, gp], axis=-1)     # [Nm_H..Nm_1, phi, Np_1..Np_H]
    rhs = np.zeros(phi.shape)
    for k, s in enumerate(st):
        if s != 0.0:
            rhs = rhs + s * ext[..., k:k + n]
    rhs = rhs / dh
    if scheme == "PADE6":
        lo, dg, up = pade6_lhs(n, PERIODIC)
        return cyclic(lo, dg, up, 1.0 / 3.0, 1.0 / 3.0, rhs)
    lo2, lo, dg, up, up2 = penta10_lhs(n, PERIODIC)
    beta, alpha = 1.0 / 20.0, 1.0 / 2.0
    return cyclic_penta(lo2, lo, dg, up, up2, rhs, [beta, alpha, beta, beta, alpha, beta])


def _deriv_tpb(cfg, dxi, f, d, ghost):
    """One metric derivative along d: TPB with ghost(idx, sign) giving the
    translated line values at wrapped indices (sign -1 before the start, +1
    after the end) on PERIODIC_SOLVE directions, the plain derivative else."""
    scheme = cfg.fd[d]
    if cfg.bc[d] != PERIODIC:
        return deriv(f, d, scheme, cfg.bc[d], dxi[d])
    H = {"PADE6": 2, "PENTA10": 3, "CD2": 2}[scheme]
    n = f.shape[_AXIS[d]]
    lines = _to_lines(f, d)
    gm = np.stack([ghost(n - m, -1) for m in range(1, H + 1)], axis=-1)   # Nm_1..Nm_H
    gp = np.stack([ghost(m - 1, +1) for m in range(1, H + 1)], axis=-1)   # Np_1..Np_H
    return np.ascontiguousarray(_from_lines(_tpb_lines(lines, gm, gp, scheme, dxi[d]), d))


def solve_for_jacobians(cfg: Config, x, y, z, quirks=True):
    """AbstractSingleBlockMesh::solveForJacobians (src/AbstractSingleBlockMesh.cpp:23-1308):
    xE_ij = d(x, y)/dxi_j (:39-303), V products (:320-333), their off-diagonal
    derivatives (:335-1008), cofactors J_ij (:1010-1023), determinant from
    (1/3) sum_i d(x . J_i)/dxi_i (:1058-1296), J = 1/det and J_ij *= J
    (:1298-1308). Periodic directions use the TPB derivatives with the ghost
    values translated by handlePeriodicStuff. With `quirks`, two BW7 calls
    pass their Nm2 ghost as the Nm3 ghost: d y/d xi3 (:273) and d Vc3/d xi1
    (:706). Returns [J, J11, ..., J33]."""
    dxi = [1.0 / n if b == PERIODIC else 1.0 / (n - 1.0) for n, b in zip(cfg.N, cfg.bc)]
    T = periodic_translations(cfg)
    X = [x, y, z]

    def line_at(a, d, idx):
        return np.take(_to_lines(a, d), idx, axis=-1)

    def coord_ghost(c, d):
        return lambda idx, sg: line_at(X[c], d, idx) + sg * T[d, c]

    def deriv_of(f, d, ghost):
        return _deriv_tpb(cfg, dxi, f, d, ghost)

    # xE1j = dx/dxi_j, xE2j = dy/dxi_j
    def nm3_as_nm2(g, d):
        # the Nm3 ghost (index N-3, before the start) replaced by the Nm2 one
        n = x.shape[_AXIS[d]]
        return lambda idx, sg: g(n - 2, sg) if (sg < 0 and idx == n - 3) else g(idx, sg)

    xE1 = [deriv_of(x, j, coord_ghost(0, j)) for j in range(3)]
    xE2 = []
    for j in range(3):
        g = coord_ghost(1, j)
        if quirks and j == 2 and cfg.fd[2] == "PENTA10":
            g = nm3_as_nm2(g, 2)
        xE2.append(deriv_of(y, j, g))

    def vprod(w, c, j):
        # V = w_j * X_c with ghosts (X_c +- T_c) * w_j
        f = w[j] * X[c]

        def ghost_for(k):
            return lambda idx, sg: (line_at(X[c], k, idx) + sg * T[k, c]) * line_at(w[j], k, idx)
        return f, ghost_for

    Va = [vprod(xE1, 1, j) for j in range(3)]   # xE1j * y
    Vb = [vprod(xE1, 2, j) for j in range(3)]   # xE1j * z
    Vc = [vprod(xE2, 2, j) for j in range(3)]   # xE2j * z

    def dV(V, j, k):
        f, gf = V[j]
        g = gf(k)
        if quirks and V is Vc and j == 2 and k == 0 and cfg.fd[0] == "PENTA10":
            g = nm3_as_nm2(g, 0)
        return deriv_of(f, k, g)

    # 0-based: dV?[j][k] = d V?_j / d xi_k
    J11 = dV(Vc, 1, 2) - dV(Vc, 2, 1)
    J12 = dV(Vb, 2, 1) - dV(Vb, 1, 2)
    J13 = dV(Va, 1, 2) - dV(Va, 2, 1)
    J21 = dV(Vc, 2, 0) - dV(Vc, 0, 2)
    J22 = dV(Vb, 0, 2) - dV(Vb, 2, 0)
    J23 = dV(Va, 2, 0) - dV(Va, 0, 2)
    J31 = dV(Vc, 0, 1) - dV(Vc, 1, 0)
    J32 = dV(Vb, 1, 0) - dV(Vb, 0, 1)
    J33 = dV(Va, 0, 1) - dV(Va, 1, 0)
    Jr = [[J11, J12, J13], [J21, J22, J23], [J31, J32, J33]]
    jd = []
    for i in range(3):
        pre = x * Jr[i][0] + y * Jr[i][1] + z * Jr[i][2]

        def ghost(idx, sg, i=i):
            return sum((line_at(X[c], i, idx) + sg * T[i, c]) * line_at(Jr[i][c], i, idx) for c in range(3))
        jd.append(deriv_of(pre, i, ghost))
    J = 1.0 / ((1.0 / 3.0) * (jd[0] + jd[1] + jd[2]))
    return [J] + [J * Jr[a][b] for a in range(3) for b in range(3)]


# --------------------------------------------------------------------------
# Checkpoints (src/CurvilinearCSolver_Core.cpp:1333-1405, src/MPI_3DCompact.cpp:80-271)
# --------------------------------------------------------------------------
def parse_solution_dump(raw: bytes):
    """A SolutionDump file as dumpSolution writes it: 5 FP64 header values
    (time step, time, Nx, Ny, Nz) then x, y, z, rho, rhoU, rhoV, rhoW, rhoE,
    Nx*Ny*Nz FP64 values each, x fastest. Returns (header, 8 fields (Nz, Ny, Nx))."""
    a = np.frombuffer(raw, dtype=np.float64)
    ts, t, nx, ny, nz = a[:5]
    nx, ny, nz = int(nx), int(ny), int(nz)
    n = nx * ny * nz
    if a.size != 5 + 8 * n:
        raise ValueError("not a SolutionDump of its header's size")
    fields = [a[5 + k * n:5 + (k + 1) * n].reshape(nz, ny, nx).copy() for k in range(8)]
    return {"time_step": int(ts), "time": float(t), "N": (nx, ny, nz)}, fields


def restart_primitives(q):
    """src/MPI_3DCompact.cpp:248-262: rho, U, V, W, p of a restart from its
    conserved fields through IdealGas::solveU / solvep (src/IdealGas.hpp:58-64)."""
    rho, ru, rv, rw, re = q
    U, V, W = ru / rho, rv / rho, rw / rho
    p = (1.4 - 1) * (re - 0.5 * rho * (U * U + V * V + W * W))
    return rho, U, V, W, p


def cube_metrics(N, L=2.0 * math.pi):
    """Analytic metrics of the periodic cube x = L*xi (the HIT box of
    tests/hit/Samtaney_D4/AlgebraicSingleBlockMesh.hpp:154-156): J_ii = 1/L,
    J = 1/L^3, off-diagonals zero."""
    Nx, Ny, Nz = N
    shp = (Nz, Ny, Nx)
    z = np.zeros(shp)
    d = np.full(shp, 1.0 / L)
    return [np.full(shp, 1.0 / L ** 3), d, z, z, z, d.copy(), z, z, z, d.copy()]


class Stats:
    """Running statistics of the solver (src/Stats.hpp:30-266, src/Stats.cpp:127-347):
    time-weighted means, RMS and Reynolds stresses of U, V, W and means / RMS of
    rho, p, T, updated every `interval` time steps in postStep
    (src/CurvilinearCSolver.hpp:362-364). Velocity, p and T are those of the
    filtered state; rho is rho2, the state before the filter (Stats.hpp:45)."""

    def __init__(self, spec, shape, time):
        self.spec = dict(spec)
        self.velocity = self.spec.get("velocity", True)
        self.thermo = self.spec.get("thermo", True)
        self.avg = self.spec.get("avg", "NONE")
        self.interval = self.spec.get("interval", 1)
        self.prev_time = time                    # Stats.hpp:58
        self.vw = 0.0
        self.tw = 0.0
        z = np.zeros(shape)
        # UAVG, VAVG, WAVG, URMS, VRMS, WRMS, UVREY, UWREY, VWREY (the dump order)
        self.v = [z.copy() for _ in range(9)]
        # RHOAVG, RHORMS, PAVG, PRMS, TAVG, TRMS
        self.t = [z.copy() for _ in range(6)]

    def _average(self, phi):
        """Stats::doAveraging (src/Stats.cpp:225-347): index means along xi1 or
        xi3 summed term by term as phi/N; the XI2 branch averages the solver's
        scratch array instead of phi (:268-296), which leaves phi unchanged;
        other types do nothing."""
        if self.avg == "XI1_AVG":
            n = phi.shape[2]
            acc = np.zeros(phi.shape[:2])
            for i in range(n):
                acc = acc + phi[:, :, i] / float(n)
            return np.repeat(acc[:, :, None], n, axis=2)
        if self.avg == "XI3_AVG":
            n = phi.shape[0]
            acc = np.zeros(phi.shape[1:])
            for k in range(n):
                acc = acc + phi[k] / float(n)
            return np.repeat(acc[None], n, axis=0)
        return phi

    def update(self, time, q1, q2):
        """Stats::updateStatsFields (src/Stats.cpp:127-223)."""
        dt = time - self.prev_time
        rho1, ru, rv, rw, re = q1
        U, V, W = ru / rho1, rv / rho1, rw / rho1
        p = (GAMMA - 1) * (re - 0.5 * rho1 * (U * U + V * V + W * W))
        T = p / (rho1 * R_GAS)
        if self.velocity and dt != 0.0:
            ow, nw = self.vw, self.vw + dt
            UA, VA, WA, UR, VR, WR, UV, UW, VW = self.v
            UR = (ow * (UR * UR + UA * UA) + dt * U * U) / nw
            VR = (ow * (VR * VR + VA * VA) + dt * V * V) / nw
            WR = (ow * (WR * WR + WA * WA) + dt * W * W) / nw
            UV = (ow * (UV + UA * VA) + dt * U * V) / nw
            UW = (ow * (UW + UA * WA) + dt * U * W) / nw
            VW = (ow * (VW + VA * WA) + dt * V * W) / nw
            UA = (ow * UA + dt * U) / nw
            VA = (ow * VA + dt * V) / nw
            WA = (ow * WA + dt * W) / nw
            UR, VR, WR, UV, UW, VW, UA, VA, WA = [self._average(a) for a in (UR, VR, WR, UV, UW, VW, UA, VA, WA)]
            UR = np.sqrt(np.abs(UR - UA * UA))
            VR = np.sqrt(np.abs(VR - VA * VA))
            WR = np.sqrt(np.abs(WR - WA * WA))
            UV = UV - UA * VA
            UW = UW - UA * WA
            VW = VW - VA * WA
            self.v = [UA, VA, WA, UR, VR, WR, UV, UW, VW]
            self.vw = nw
        if self.thermo and dt != 0.0:
            rho = q2[0]
            ow, nw = self.tw, self.tw + dt
            RA, RR, PA, PR, TA, TR = self.t
            RR = (ow * (RR * RR + RA * RA) + dt * rho * rho) / nw
            PR = (ow * (PR * PR + PA * PA) + dt * p * p) / nw
            TR = (ow * (TR * TR + TA * TA) + dt * T * T) / nw
            RA = (ow * RA + dt * rho) / nw
            PA = (ow * PA + dt * p) / nw
            TA = (ow * TA + dt * T) / nw
            RR, PR, TR, RA, PA, TA = [self._average(a) for a in (RR, PR, TR, RA, PA, TA)]
            RR = np.sqrt(np.abs(RR - RA * RA))
            PR = np.sqrt(np.abs(PR - PA * PA))
            TR = np.sqrt(np.abs(TR - TA * TA))
            self.t = [RA, RR, PA, PR, TA, TR]
            self.tw = nw
        self.prev_time = time


def hit_turbdata(o: "Oracle", k0=8.0):
    """The HIT driver's turbdata.out line (tests/hit/Samtaney_D4/MPI_3DCompact.cpp:
    370-555) for the oracle's current state: gradients of U, V, W of the filtered
    state, Cartesian components through the metrics (:410-420), dissipation
    2 mu S^d_ij du_i/dx_j (:430-450), block means (:480-495, :511-515) and the
    11 output values (:522-552)."""
    st = o.state
    U, V, W, p, T, mu, sos = primitives(st.q1, o.cfg.mu_ref)
    rho = st.q1[0]
    d = [o.grad(f) for f in (U, V, W)]          # d[var][dir]
    Jm = o.Jm
    gu = [[Jm[0][b] * d[a][0] + Jm[1][b] * d[a][1] + Jm[2][b] * d[a][2] for b in range(3)] for a in range(3)]
    dil = gu[0][0] + gu[1][1] + gu[2][2]
    diss = 0.0
    for a in range(3):
        for b in range(3):
            s = 0.5 * (gu[a][b] + gu[b][a]) - ((1.0 / 3.0) * dil if a == b else 0.0)
            diss = diss + s * gu[a][b]
    diss = diss * 2 * mu
    uvar = U * U + V * V + W * W
    mean = (lambda f: float(np.mean(f)))
    meanRho, meanMu = mean(rho), mean(mu)
    meanTurbDiss = mean(diss) / meanRho
    uprime, uiprime = math.sqrt(mean(uvar / 3.0)), math.sqrt(mean((gu[0][0] ** 2 + gu[1][1] ** 2 + gu[2][2] ** 2) / 3.0))
    urms, meanSOS = math.sqrt(mean(uvar)), mean(sos)
    wx, wy, wz = gu[2][1] - gu[1][2], gu[0][2] - gu[2][0], gu[1][0] - gu[0][1]
    rhoprime = math.sqrt(mean((rho - meanRho) ** 2))
    dilprime = math.sqrt(mean(dil * dil))
    vortprime = math.sqrt(mean(wx * wx + wy * wy + wz * wz))
    meanNu = meanMu / meanRho
    taylor = uprime / uiprime
    return [st.time, math.sqrt(2 * math.pi) / k0 / uprime, uprime * taylor / meanNu, urms / meanSOS, meanTurbDiss,
            uprime, (meanNu ** 3 / meanTurbDiss) ** 0.25, rhoprime, dilprime, vortprime, mean(rho * uvar)]


def wall_span_average(q):
    """The cylinder driver's surface averages (src/MPI_3DCompact.cpp:408-461):
    p, U, V, W on the j = 0 face summed as x/Nz over xi3."""
    U, V, W, p, T, mu, sos = primitives([a[:, 0, :] for a in q], 1.0)
    nz = q[0].shape[0]
    out = []
    for f in (p, U, V, W):
        acc = np.zeros(f.shape[1])
        for k in range(nz):
            acc = acc + f[k] / float(nz)
        out.append(acc)
    return out


def parse_stats_file(raw: bytes, nfields, shape):
    """VelocityStats / ThermoStats as Stats::dumpStatsFields writes them
    (src/Stats.cpp:3-125): the weight, then the fields, x fastest."""
    a = np.frombuffer(raw, dtype=np.float64)
    n = int(np.prod(shape))
    if a.size != 1 + nfields * n:
        raise ValueError("not a stats file of this size")
    return float(a[0]), [a[1 + k * n:1 + (k + 1) * n].reshape(shape).copy() for k in range(nfields)]


def run(cfg: Config, ic, nsteps, metrics=None, sigma=None, time=0.0, time_step=0):
    """Run `nsteps` time steps from primitive ICs (rho, U, V, W, p), starting
    at `time` / `time_step` (a restart), and return (conserved state
    rho1..rhoE1, state object)."""
    o = Oracle(cfg, metrics if metrics is not None else cube_metrics(cfg.N), sigma=sigma)
    o.init(*ic, time=time, time_step=time_step)
    for _ in range(nsteps):
        o.step()
    return o.state.q1, o.state
