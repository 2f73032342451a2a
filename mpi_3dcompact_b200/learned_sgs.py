"""Training of the learned SGS closure from this solver's own DNS.

No counterpart in the reference (its SGS models are VremanSGS and DSMSGS).
Pipeline, all on the GPU:

1. DNS of decaying HIT on a fine grid with ``CurvilinearCSolver``
   (LESMODEL = NOMODEL), snapshots of the conserved state;
2. box filter of factor f onto the coarse LES grid (``mc3d_sgs_box_filter``):
   rho, rhoU_i, rhoU_iU_j, rhoT, rhoU_iT;
3. Favre-filtered u, v, w, T and their compact xi-derivatives on the coarse
   grid (the solver's own ``Pade6`` operators);
4. features and least-squares targets per coarse point
   (``mc3d_sgs_training_pairs``): C = -tau^d:S^d / (2 rho Delta^2 |S| S^d:S^d)
   and Pr_t from the SGS heat flux;
5. Adam on the MSE of normalised targets (``MLPClosure.train_step``); the
   feature normalisation and the training range (outside which the solver
   falls back to DSM) come from the training set;
6. a posteriori calibration of the coefficient: LES of decaying HIT on the
   coarse grid from held-out seeds with the closure and with DSM, and the one
   scale of C whose decayed kinetic energy stays closest to DSM's is folded
   into the output normalisation (``calibrate_output_scale``). The pointwise
   least-squares coefficients of the box-filtered DNS dissipate several times
   more than the compact-filtered LES needs.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _native as N
from . import CurvilinearCSolver, MLPClosure, Options, Pade6, PERIODIC_SOLVE
from .hit_ic import hit_initial_condition, hit_initial_condition_device

C_RANGE = (-0.2, 0.5)      # clip of the pointwise least-squares coefficient
PRT_RANGE = (0.1, 10.0)
DEFAULT_FALLBACK_FRAC = 1e-3   # the library's LES.MLPFALLBACKFRAC default


def _torch():
    import torch
    return torch


def _vp_array(ts):
    return (C.c_void_p * len(ts))(*[t.data_ptr() for t in ts])


def training_pairs(q, n_fine, factor, box=2.0 * math.pi, mu_ref=1e-3):
    """Features x [n, 9] and targets y [n, 2] (torch float32 on the GPU) from
    a DNS state q (5 device FP64 tensors (N, N, N)) box-filtered by `factor`."""
    torch = _torch()
    nc = n_fine // factor
    coarse = [torch.empty((nc, nc, nc), dtype=torch.float64, device="cuda") for _ in range(14)]
    N.check(N.host_lib().mc3d_sgs_box_filter(_vp_array(q), n_fine, n_fine, n_fine, factor, _vp_array(coarse), None))
    rho = coarse[0]
    fav = [coarse[1] / rho, coarse[2] / rho, coarse[3] / rho, coarse[10] / rho]   # u, v, w, T
    grads = [torch.empty_like(rho) for _ in range(12)]
    ops = [Pade6((nc, nc, nc), PERIODIC_SOLVE, d) for d in range(3)]
    for v in range(4):
        for d in range(3):
            ops[d].calc1stDerivField(fav[v].contiguous(), grads[3 * v + d])
    n = nc ** 3
    x = torch.empty((n, 9), dtype=torch.float32, device="cuda")
    y = torch.empty((n, 2), dtype=torch.float32, device="cuda")
    jd = (C.c_double * 3)(1.0 / box, 1.0 / box, 1.0 / box)
    N.check(N.host_lib().mc3d_sgs_training_pairs(_vp_array(coarse), _vp_array(grads), nc, nc, nc, jd, box / nc,
                                                 mu_ref, C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()), None))
    torch.cuda.synchronize()
    ok = torch.isfinite(x).all(dim=1) & torch.isfinite(y).all(dim=1)
    x, y = x[ok], y[ok]
    y[:, 0].clamp_(*C_RANGE)
    y[:, 1].clamp_(*PRT_RANGE)
    return x, y


def dns_snapshots(n=128, seeds=(0,), steps=(20, 40), k0=4.0, mt=0.3, mu_ref=1e-3, precision=0):
    """Conserved-state snapshots (device FP64 tensors (n, n, n)) of HIT DNS runs
    with the given seeds, taken after each count of time steps in `steps`
    (initial fields from the device generator from 256^3 up)."""
    torch = _torch()
    out = []
    for seed in seeds:
        opt = Options(grid=n, fd="PADE6", filter="COMPACT10", alphaF=0.49, rk="RK4", mu_ref=mu_ref,
                      precision=precision)
        s = CurvilinearCSolver(opt)
        s.set_box_metrics(2.0 * math.pi)
        gen = hit_initial_condition_device if n >= 256 else hit_initial_condition
        s.set_initial_conditions(*gen(n, k0=k0, seed=seed, mt=mt))
        done = 0
        for target in steps:
            s.step(target - done)
            done = target
            snap = [torch.empty((n, n, n), dtype=torch.float64, device="cuda") for _ in range(5)]
            s.copy_conserved_device(snap)
            out.append(snap)
        del s
    return out


def fit_normalization(mlp: MLPClosure, x, y, margin=0.05):
    """Feature/target statistics of the training set into the network; the
    training range is the data range widened by `margin` of its width."""
    xd = x.double()
    mean = xd.mean(0).cpu().numpy()
    std = xd.std(0).clamp_min(1e-6).cpu().numpy()
    lo = xd.min(0).values.cpu().numpy()
    hi = xd.max(0).values.cpu().numpy()
    w = hi - lo
    yd = y.double()
    mlp.set_normalization(mean, std, lo - margin * w, hi + margin * w, yd.mean(0).cpu().numpy(),
                          yd.std(0).clamp_min(1e-6).cpu().numpy())


def train(mlp: MLPClosure, x, y, steps=2000, batch=65536, lr=1e-3, seed=0):
    """Adam on minibatches of the normalised targets; returns the loss history."""
    torch = _torch()
    nrm = mlp.normalization()
    ym = torch.tensor(nrm["ymean"], device="cuda")
    ys = torch.tensor(nrm["ystd"], device="cuda")
    yn = ((y - ym) / ys).contiguous()
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    n = x.shape[0]
    hist = []
    for it in range(steps):
        idx = torch.randint(0, n, (min(batch, n),), device="cuda", generator=g)
        hist.append(mlp.train_step(x[idx].contiguous(), yn[idx].contiguous(), lr))
    return hist


# LES of the calibration (the a posteriori configuration of the closure)
LES_SCHEME = dict(fd="PADE6", filter="COMPACT10", alphaF=0.49, rk="RK4", les_avg="GLOBAL", cfl=0.5)


def scale_output(mlp: MLPClosure, s):
    """Multiply the closure's coefficient C by s > 0 (C = max(0, out * ystd +
    ymean) scales with ymean and ystd)."""
    nrm = mlp.normalization()
    ym, ys = nrm["ymean"].copy(), nrm["ystd"].copy()
    ym[0] *= s
    ys[0] *= s
    mlp.set_normalization(nrm["mean"], nrm["std"], nrm["lo"], nrm["hi"], ym, ys)


def decayed_energy(les, mlp=None, n=128, seed=1, steps=500, chunk=50, mu_ref=2.5e-4, k0=4.0, mt=0.3, frac=1.0,
                   timing=None):
    """Kinetic energy every `chunk` steps of an FP32-bulk LES of decaying HIT
    on n^3 (LES_SCHEME) with closure `les` ("MLP" uses `mlp` with fallback
    fraction `frac`); `timing` (a dict) receives the device milliseconds of the
    steps ("ms", CUDA events on the solver's stream) and the fallback count."""
    from . import FP32BULK
    ic = hit_initial_condition(n, k0=k0, seed=seed, mt=mt)
    kw = dict(grid=n, mu_ref=mu_ref, les=les, precision=FP32BULK, **LES_SCHEME)
    if les == "MLP":
        kw["mlp_fallback_frac"] = frac
    s = CurvilinearCSolver(Options(**kw))
    s.set_box_metrics(2.0 * math.pi)
    s.set_initial_conditions(*ic)
    if les == "MLP":
        s.set_mlp(mlp)
    torch = _torch()
    stream = torch.cuda.ExternalStream(s.stream())
    ke = [s.integrals()[0]]
    done, ms = 0, 0.0
    while done < steps:
        k = min(chunk, steps - done)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        s.step(k)
        e1.record(stream)
        e1.synchronize()
        ms += e0.elapsed_time(e1)
        done += k
        ke.append(s.integrals()[0])
    if timing is not None:
        timing["ms"] = ms
        timing["fallbacks"] = s.mlp_fallbacks() if les == "MLP" else None
    return np.array(ke)


def decay_difference(ke, ke_ref):
    """Largest relative difference of the decayed energy KE(0) - KE(t) over
    the checkpoints."""
    d, r = ke[0] - ke, ke_ref[0] - ke_ref
    return float(np.max(np.abs(d[1:] - r[1:]) / np.abs(r[1:])))


def calibrate_output_scale(mlp: MLPClosure, seeds=(1, 2), scales=(0.15, 0.2, 0.25, 0.3, 0.4, 0.55, 0.7, 1.0),
                           **les_kw):
    """A posteriori calibration: the scale of C (from `scales`) minimising the
    largest decay difference to DSM over LES from `seeds` (no DSM fallback),
    applied to `mlp`; returns (scale, {scale: [difference per seed]})."""
    ref = {sd: decayed_energy("DSM", seed=sd, **les_kw) for sd in seeds}
    nrm = mlp.normalization()
    table = {}
    for sc in scales:
        scale_output(mlp, sc)
        table[sc] = [decay_difference(decayed_energy("MLP", mlp, seed=sd, **les_kw), ref[sd]) for sd in seeds]
        mlp.set_normalization(nrm["mean"], nrm["std"], nrm["lo"], nrm["hi"], nrm["ymean"], nrm["ystd"])
    best = min(table, key=lambda k: max(table[k]))
    scale_output(mlp, best)
    return best, table
