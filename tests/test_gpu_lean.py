"""GPU tests of GPU.STORAGE = LEAN, the dataflow that holds a 1024^3 block on
one GPU: the xi3-gradients and xi3-fluxes as the only full work fields,
everything along xi1 and xi2 in slabs of xi3-planes, k2 accumulating the
divergence in place, the 2N schemes' final state written over the stage
state, and the filter one field at a time.

It computes the same operations per point as STORAGE = FULL; only the order
of the momentum RHS sums differs with the reference's carry-over
((k2_prev - dF/dxi1) - dF/dxi2 - dF/dxi3 against k2_prev + ((-dF/dxi1 -
dF/dxi2) - dF/dxi3)). Bounds: FP64 within 1e-12 relative max per field of
the full path after four steps (rounding of those sums only); FP32-bulk within
1e-5 relative L2 of the FP64 full path (the error target of the FP32 path).
Slabs of 5 planes over 22 make a ragged last slab."""
import math

import numpy as np
import pytest

import mpi_3dcompact_b200 as m
from mpi_3dcompact_b200.hit_ic import hit_initial_condition
from tests import helpers as H

pytestmark = pytest.mark.gpu


def _run(storage, prec, n_xyz, steps, ic, **kw):
    opts = dict(fd="PENTA10", filter="COMPACT8", alphaF=0.45, rk="LSLDDRK4", les="VREMAN", mu_ref=0.002, cfl=0.5)
    opts.update(kw)
    s = m.CurvilinearCSolver(m.Options(grid=n_xyz, precision=prec, storage=storage, lean_slab=5, **opts))
    s.set_box_metrics(2 * math.pi)
    s.set_initial_conditions(*ic)
    s.step(steps)
    return s.conserved(), s.info()


def _ic(n_xyz, seed):
    n = max(n_xyz)
    ic = hit_initial_condition(n, k0=3.0, seed=seed, mt=0.3)
    Nx, Ny, Nz = n_xyz
    return [np.ascontiguousarray(a[:Nz, :Ny, :Nx]) for a in ic]


@pytest.mark.parametrize("kw", [dict(), dict(rk="RK4", fd="PADE6", filter="COMPACT10", alphaF=0.49, les="NOMODEL"),
                                dict(reference_quirks=False), dict(rk="KENRK4", filter_step=2)])
def test_lean_fp64_follows_full_storage(kw):
    N = (32, 24, 22)
    ic = _ic(N, 5)
    qf, inf = _run("FULL", m.FP64, N, 4, ic, **kw)
    ql, inl = _run("LEAN", m.FP64, N, 4, ic, **kw)
    for i in range(5):
        assert H.rel_max(ql[i], qf[i]) <= 1e-12, (kw, i, H.rel_max(ql[i], qf[i]))
    assert inl["time_step"] == inf["time_step"] and abs(inl["time"] - inf["time"]) <= 1e-12 * inf["time"]
    assert inl["stages"] == inf["stages"]


def test_lean_fp32bulk_holds_the_fp64_bound():
    N = (64, 64, 64)
    ic = _ic(N, 7)
    q64, _ = _run("FULL", m.FP64, N, 10, ic)
    q32, _ = _run("LEAN", m.FP32BULK, N, 10, ic)
    for i in range(5):
        assert H.rel_l2(q32[i], q64[i]) <= 1e-5, (i, H.rel_l2(q32[i], q64[i]))


def test_lean_learned_closure_runs_and_counts_out_of_range_stages():
    """LESMODEL = MLP with lean storage: no DSM fallback; stages that would have
    fallen back are counted. With a fallback fraction of 1 no stage counts and
    the lean and full FP32 paths agree to 1e-5 relative L2."""
    import os
    N = (32, 32, 32)
    ic = _ic(N, 9)
    weights = os.path.join(os.path.dirname(m.__file__), "data", "mlp_sgs_hit128.bin")
    out = []
    for storage in ("FULL", "LEAN"):
        s = m.CurvilinearCSolver(m.Options(grid=N, fd="PADE6", filter="COMPACT10", alphaF=0.49, rk="RK4", les="MLP",
                                           mu_ref=2.5e-4, precision=m.FP32BULK, storage=storage, lean_slab=5,
                                           mlp_fallback_frac=1.0))
        s.set_box_metrics(2 * math.pi)
        s.set_initial_conditions(*ic)
        mlp = m.MLPClosure()
        mlp.load(weights)
        s.set_mlp(mlp)
        s.step(3)
        out.append(s.conserved())
        assert s.mlp_fallbacks() == 0
    for i in range(5):
        assert H.rel_l2(out[1][i], out[0][i]) <= 1e-5, (i, H.rel_l2(out[1][i], out[0][i]))


def test_lean_storage_refuses_what_it_does_not_hold():
    for kw in (dict(les="DSM"), dict(les="VREMAN", les_avg="LOCAL"), dict(substep_filtering=True),
               dict(bc=(m.PERIODIC_SOLVE, m.DIRICHLET_SOLVE, m.PERIODIC_SOLVE))):
        with pytest.raises(m.Mc3dError):
            m.CurvilinearCSolver(m.Options(grid=16, storage="LEAN", **kw))
    s = m.CurvilinearCSolver(m.Options(grid=16, storage="LEAN"))
    s.set_box_metrics(2 * math.pi)
    s.set_initial_conditions(*hit_initial_condition(16, k0=3.0, seed=1, mt=0.3))
    with pytest.raises(m.Mc3dError):
        s.turbdata()
