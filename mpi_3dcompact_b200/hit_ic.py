"""Seeded initial condition for decaying homogeneous isotropic turbulence.

Restates the algorithm of the reference's generator
tests/hit/generate_init_hit.f90 (emathew1/MPI_3DCompact):
  * the combined-LCG shuffle generator randset/randvec (:16-81);
  * random phases phi1..phi3 in (-pi, pi] (:223-229);
  * spectrum E(k) = (k/k0)^4 exp(-2 (k/k0)^2) (:277);
  * the solenoidal two-angle construction of u_hat (:301-329);
  * Hermitian symmetry on the kx=0 plane, zeroed Nyquist planes and mean (:338-356);
  * the unnormalised complex-to-real 3-D transform (FFTW c2r, :359).
The reference writes an ASCII Tecplot box of N+1 points; the solver grid is
the periodic N^3 part of it, which is what this returns. Velocities are then
scaled to a target turbulent Mach number (rms |u| / c, c = 1 for p = 1/gamma,
rho = 1) as BASELINE's HIT configurations ask.
"""
from __future__ import annotations

import math

import numpy as np

_M1, _IA1, _IC1 = 259200, 7141, 54773
_M2, _IA2, _IC2 = 134456, 8121, 28441
_M3, _IA3, _IC3 = 243000, 4561, 51349
_RM1, _RM2 = 1.0 / _M1, 1.0 / _M2


class _Gen:
    """randset/randvec of generate_init_hit.f90:16-81."""

    def __init__(self, idum: int):
        ix1 = (_IC1 - idum) % _M1
        ix1 = (_IA1 * ix1 + _IC1) % _M1
        ix2 = ix1 % _M2
        ix1 = (_IA1 * ix1 + _IC1) % _M1
        ix3 = ix1 % _M3
        r = [0.0] * 97
        for j in range(97):
            ix1 = (_IA1 * ix1 + _IC1) % _M1
            ix2 = (_IA2 * ix2 + _IC2) % _M2
            r[j] = min(1.0, max(0.0, (float(ix1) + float(ix2) * _RM2) * _RM1))
        self.r, self.ix1, self.ix2, self.ix3 = r, ix1, ix2, ix3

    def vec(self, n: int) -> np.ndarray:
        """The next n values of randvec, vectorised: each of the three LCG
        sequences is produced by doubling (x -> A x + C composed with itself),
        and the shuffle table's output at step m is the table value written at
        the last earlier step that drew the same slot (or the initial value),
        found with one stable sort by slot. Bit-identical to the loop of
        generate_init_hit.f90:54-81 (same integer arithmetic, same FP64
        expression for the table values)."""
        if n <= 0:
            return np.empty(0)
        ix1 = _lcg(self.ix1, _IA1, _IC1, _M1, n)
        ix2 = _lcg(self.ix2, _IA2, _IC2, _M2, n)
        ix3 = _lcg(self.ix3, _IA3, _IC3, _M3, n)
        slot = ((97 * ix3) // _M3 % 97).astype(np.uint8)
        val = np.clip((ix1.astype(np.float64) + ix2.astype(np.float64) * _RM2) * _RM1, 0.0, 1.0)
        order = np.argsort(slot, kind="stable")
        ss = slot[order]
        prev = np.full(n, -1, dtype=np.int64)
        same = ss[1:] == ss[:-1]
        prev[order[1:][same]] = order[:-1][same]
        table = np.array(self.r, dtype=np.float64)
        out = np.where(prev >= 0, val[np.maximum(prev, 0)], table[slot])
        last = np.ones(n, dtype=bool)
        last[:-1] = ~same
        table[ss[last]] = val[order[last]]
        self.r = table.tolist()
        self.ix1, self.ix2, self.ix3 = int(ix1[-1]), int(ix2[-1]), int(ix3[-1])
        return out


def _lcg(x0: int, a: int, c: int, m: int, n: int) -> np.ndarray:
    """x_1..x_n of x_{k+1} = (a x_k + c) mod m."""
    out = np.empty(n, dtype=np.int64)
    out[0] = (a * x0 + c) % m
    A, Cc, filled = a, c, 1          # (A, Cc): the map x -> x_{k+filled}
    while filled < n:
        take = min(filled, n - filled)
        out[filled:filled + take] = (A * out[:take] + Cc) % m
        Cc = (A * Cc + Cc) % m
        A = (A * A) % m
        filled += take
    return out


def hit_velocity(n: int, k0: float = 4.0, seed: int = 1):
    """Random-phase solenoidal velocity on an n^3 periodic box of side 2*pi,
    arrays shaped (n, n, n) = (z, y, x). `seed` plays the role of randset's idum."""
    if n % 2:
        raise ValueError("n must be even (generate_init_hit.f90:150-153)")
    kx_max = n // 2 + 1
    shape_f = (n, n, kx_max)        # Fortran (kx, ky, kz) column-major == C (kz, ky, kx)
    g = _Gen(seed)
    cnt = kx_max * n * n
    # randvec fills phi(kx, ky, kz) in Fortran order: kx fastest
    phis = [2.0 * math.pi * (g.vec(cnt).reshape(shape_f) - 0.5) for _ in range(3)]
    tol = 1e-4
    kmin = tol
    i = np.arange(kx_max, dtype=np.float64)
    j = np.arange(n)
    kx = i[None, None, :]
    ky = np.where(j + 1 > kx_max, -(n - j).astype(np.float64), j.astype(np.float64))[None, :, None]
    kz = np.where(j + 1 > kx_max, -(n - j).astype(np.float64), j.astype(np.float64))[:, None, None]
    kxyz = np.sqrt(kx ** 2 + ky ** 2 + kz ** 2)
    kxy = np.sqrt(kx ** 2 + ky ** 2) + 0.0 * kz
    eq = (kxyz / k0) ** 4 * np.exp(-2.0 * (kxyz / k0) ** 2)
    amp = np.where(kxyz > kmin, np.sqrt(eq / (2.0 * math.pi * np.maximum(kxyz, kmin) ** 2)), 0.0)
    a = amp * np.exp(1j * phis[0]) * np.cos(phis[2])
    b = amp * np.exp(1j * phis[1]) * np.sin(phis[2])
    safe = np.maximum(kxyz * kxy, 1e-300)
    out = []
    for comp in range(3):
        if comp == 0:
            uk = np.where(kxy > kmin, (a * kxyz * ky + b * kx * kz) / safe, (a + b) / math.sqrt(2.0))
        elif comp == 1:
            uk = np.where(kxy > kmin, (b * ky * kz - a * kxyz * kx) / safe, (b - a) / math.sqrt(2.0))
        else:
            uk = -b * kxy / np.maximum(kxyz, kmin)
        uk = np.where(kxyz > kmin, uk, 0.0).astype(np.complex128)
        # Hermitian symmetry on the kx = 0 plane (:338-348), Fortran 1-based -> 0-based
        for kk in range(1, n):
            for jj in range(kx_max, n):
                uk[kk, jj, 0] = np.conj(uk[n - kk, n - jj, 0])
        for kk in range(kx_max, n):
            uk[kk, 0, 0] = np.conj(uk[n - kk, 0, 0])
        for jj in range(kx_max, n):
            uk[0, jj, 0] = np.conj(uk[0, n - jj, 0])
        # odd-ball (Nyquist) planes and the mean removed (:351-356)
        uk[:, :, kx_max - 1] = 0.0
        uk[:, kx_max - 1, :] = 0.0
        uk[kx_max - 1, :, :] = 0.0
        uk[0, 0, 0] = 0.0
        u = np.fft.irfftn(uk, s=(n, n, n), axes=(0, 1, 2)) * float(n) ** 3
        out.append(np.ascontiguousarray(u))
    return out


def _lcg_torch(torch, x0: int, a: int, c: int, m: int, n: int, device):
    """x_1..x_n of x_{k+1} = (a x_k + c) mod m on `device` (as _lcg)."""
    out = torch.empty(n, dtype=torch.int64, device=device)
    out[0] = (a * x0 + c) % m
    A, Cc, filled = a, c, 1
    while filled < n:
        take = min(filled, n - filled)
        out[filled:filled + take] = (A * out[:take] + Cc) % m
        Cc = (A * Cc + Cc) % m
        A = (A * A) % m
        filled += take
    return out


def _vec_torch(torch, g: _Gen, n: int, device):
    """_Gen.vec on `device`: the same sequence, state updated the same way."""
    ix1 = _lcg_torch(torch, g.ix1, _IA1, _IC1, _M1, n, device)
    ix2 = _lcg_torch(torch, g.ix2, _IA2, _IC2, _M2, n, device)
    ix3 = _lcg_torch(torch, g.ix3, _IA3, _IC3, _M3, n, device)
    slot = (97 * ix3) // _M3 % 97
    val = torch.clamp((ix1.double() + ix2.double() * _RM2) * _RM1, 0.0, 1.0)
    last_state = (int(ix1[-1].item()), int(ix2[-1].item()), int(ix3[-1].item()))
    del ix1, ix2, ix3
    ss, order = torch.sort(slot, stable=True)
    same = ss[1:] == ss[:-1]
    prev = torch.full((n,), -1, dtype=torch.int64, device=device)
    prev[order[1:][same]] = order[:-1][same]
    table = torch.tensor(g.r, dtype=torch.float64, device=device)
    out = torch.where(prev >= 0, val[prev.clamp(min=0)], table[slot])
    last = torch.ones(n, dtype=torch.bool, device=device)
    last[:-1] = ~same
    table[ss[last]] = val[order[last]]
    g.r = table.cpu().tolist()
    g.ix1, g.ix2, g.ix3 = last_state
    return out


def hit_velocity_device(n: int, k0: float = 4.0, seed: int = 1, device="cuda"):
    """hit_velocity on a torch device (the same generator sequence, spectrum,
    solenoidal construction and symmetries; cuFFT for the c2r transform, so
    the field differs from the numpy one by FFT rounding only). Returns three
    float64 device tensors (n, n, n); peak device memory about 6 complex
    half-spectra (n * n * (n/2 + 1) * 16 bytes each)."""
    import torch
    if n % 2:
        raise ValueError("n must be even (generate_init_hit.f90:150-153)")
    kx_max = n // 2 + 1
    shape_f = (n, n, kx_max)
    g = _Gen(seed)
    cnt = kx_max * n * n
    phis = [2.0 * math.pi * (_vec_torch(torch, g, cnt, device).reshape(shape_f) - 0.5) for _ in range(3)]
    kmin = 1e-4
    i = torch.arange(kx_max, dtype=torch.float64, device=device)
    j = torch.arange(n, device=device)
    half = torch.where(j + 1 > kx_max, -(n - j).double(), j.double())
    kx = i[None, None, :]
    ky = half[None, :, None]
    kz = half[:, None, None]
    kxyz = torch.sqrt(kx ** 2 + ky ** 2 + kz ** 2)
    kxy = torch.sqrt(kx ** 2 + ky ** 2) + 0.0 * kz
    eq = (kxyz / k0) ** 4 * torch.exp(-2.0 * (kxyz / k0) ** 2)
    amp = torch.where(kxyz > kmin, torch.sqrt(eq / (2.0 * math.pi * torch.clamp(kxyz, min=kmin) ** 2)),
                      torch.zeros((), dtype=torch.float64, device=device))
    del eq
    a = amp * torch.exp(1j * phis[0]) * torch.cos(phis[2])
    b = amp * torch.exp(1j * phis[1]) * torch.sin(phis[2])
    del phis, amp
    safe = torch.clamp(kxyz * kxy, min=1e-300)
    out = []
    for comp in range(3):
        if comp == 0:
            uk = torch.where(kxy > kmin, (a * kxyz * ky + b * kx * kz) / safe, (a + b) / math.sqrt(2.0))
        elif comp == 1:
            uk = torch.where(kxy > kmin, (b * ky * kz - a * kxyz * kx) / safe, (b - a) / math.sqrt(2.0))
        else:
            uk = -b * kxy / torch.clamp(kxyz, min=kmin)
        uk = torch.where(kxyz > kmin, uk, torch.zeros((), dtype=uk.dtype, device=device))
        # Hermitian symmetry on the kx = 0 plane (:338-348); every source lies
        # outside the targets of its loop, so each loop is one assignment
        p0 = uk[:, :, 0]
        kk = torch.arange(1, n, device=device)
        jj = torch.arange(kx_max, n, device=device)
        p0[kk[:, None], jj[None, :]] = torch.conj(p0[(n - kk)[:, None], (n - jj)[None, :]])
        kk2 = torch.arange(kx_max, n, device=device)
        p0[kk2, 0] = torch.conj(p0[n - kk2, 0])
        p0[0, jj] = torch.conj(p0[0, n - jj])
        uk[:, :, 0] = p0
        uk[:, :, kx_max - 1] = 0.0
        uk[:, kx_max - 1, :] = 0.0
        uk[kx_max - 1, :, :] = 0.0
        uk[0, 0, 0] = 0.0
        u = torch.fft.irfftn(uk, s=(n, n, n), dim=(0, 1, 2)) * float(n) ** 3
        del uk
        out.append(u.contiguous())
    return out


def hit_initial_condition(n: int, k0: float = 4.0, seed: int = 1, mt: float = 0.3, gamma: float = 1.4):
    """Primitive ICs (rho, U, V, W, p) with rho = 1, p = 1/gamma (c = 1) and the
    velocity scaled so that sqrt(<|u|^2>)/c = mt."""
    u, v, w = hit_velocity(n, k0, seed)
    urms = math.sqrt(float(np.mean(u * u + v * v + w * w)))
    s = mt / urms if urms > 0 else 0.0
    rho = np.ones((n, n, n))
    p = np.full((n, n, n), 1.0 / gamma)
    return [rho, u * s, v * s, w * s, p]


def hit_initial_condition_device(n: int, k0: float = 4.0, seed: int = 1, mt: float = 0.3, gamma: float = 1.4,
                                 device="cuda"):
    """hit_initial_condition with the velocity drawn by hit_velocity_device,
    returned as host numpy arrays (the solver takes host initial conditions);
    for large n, where the numpy transform takes minutes."""
    import torch
    u, v, w = hit_velocity_device(n, k0, seed, device)
    urms = math.sqrt(float((u * u + v * v + w * w).mean().item()))
    s = mt / urms if urms > 0 else 0.0
    vel = [(a * s).cpu().numpy() for a in (u, v, w)]
    del u, v, w
    torch.cuda.empty_cache()
    return [np.ones((n, n, n)), vel[0], vel[1], vel[2], np.full((n, n, n), 1.0 / gamma)]


def reynolds_lambda_mu(ic, L=2.0 * math.pi):
    """mu_ref giving Re_lambda for a target (helper for the HIT configurations):
    returns (u', lambda) where u' = rms of one component and lambda the Taylor
    microscale sqrt(<u^2>/<(du/dx)^2>), spectral derivative on the periodic box."""
    rho, u, v, w, p = ic
    n = u.shape[0]
    k = np.fft.fftfreq(n, d=L / n) * 2.0 * math.pi
    du = np.real(np.fft.ifft(1j * k[None, None, :] * np.fft.fft(u, axis=2), axis=2))
    up = math.sqrt(float(np.mean(u * u + v * v + w * w)) / 3.0)
    lam = math.sqrt(float(np.mean(u * u)) / float(np.mean(du * du)))
    return up, lam
