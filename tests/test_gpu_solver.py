"""GPU parity of the full time step (C ABI mc3d_solver_* through the
CurvilinearCSolver mirror).

  * FP64 path vs the reference solver's own output (golden fixtures, 3-5 steps
    of every RK scheme, both compact schemes, both filters, Vreman with and
    without LOCAL averaging, sub-step filtering, non-cubic grids):
    max error <= 1e-12 relative per conserved field.
  * FP64 path vs the oracle after 10 steps of the 64^3-class HIT set-up
    (PADE6 / RK4 / COMPACT10 alpha_f = 0.49) on 16^3: <= 1e-12 relative.
  * General (non-constant) metric fields vs the oracle: <= 1e-12.
  * FP32-bulk vs FP64 on 32^3 HIT after 20 LSLDDRK4 steps: relative L2 per
    field <= 1e-5 (the error target stated for the FP32 path).
  * Dynamic Smagorinsky (both test filters, XI2/GLOBAL averaging) on 64^3 vs
    the oracle after two steps: 1e-12 (FP64), 1e-5 (FP32-bulk).
"""
import math
import os

import numpy as np
import pytest

import mpi_3dcompact_b200 as m
from oracle import mc3d_oracle as O
from tests import helpers as H
from tests.golden import gen_golden as G

pytestmark = pytest.mark.gpu


def _opts(cfg: O.Config, precision=m.FP64):
    return m.Options(grid=cfg.N, fd=cfg.fd, filter=cfg.filter, alphaF=cfg.alphaF, mu_ref=cfg.mu_ref, rk=cfg.rk,
                     ts_type=cfg.ts_type, cfl=cfg.cfl, dt=cfg.dt, filter_step=cfg.filter_step,
                     substep_filtering=cfg.substep_filtering, les=cfg.les, les_avg=cfg.les_avg,
                     precision=precision, dsm_test_filter=cfg.dsm_test_filter, dsm_use_taukk=cfg.dsm_use_taukk)


def _run(cfg, ic, n, precision=m.FP64, metrics=None):
    s = m.CurvilinearCSolver(_opts(cfg, precision))
    if metrics is None:
        s.set_box_metrics(2.0 * math.pi)
    else:
        s.set_metrics(metrics)
    s.set_initial_conditions(*ic)
    s.step(n)
    q = s.conserved()
    return q, s.info(), s


@pytest.mark.parametrize("name", list(G.STEP_CASES))
def test_fp64_matches_reference_solver(name):
    cfg, ic, n = H.oracle_config(name)
    q, info, _ = _run(cfg, ic, n)
    gold = H.golden_steps()
    for i in range(5):
        err = H.rel_max(q[i], gold[f"{name}_q{i}"])
        assert err <= 1e-12, (name, i, err)
    ts, t, dt = gold[f"{name}_info"]
    assert info["time_step"] == int(ts)
    assert abs(info["time"] - t) <= 1e-12 * abs(t)
    assert abs(info["dt"] - dt) <= 1e-12 * abs(dt)


def test_fp64_hit_10_steps_vs_oracle():
    cfg = O.Config(N=(16, 16, 16), fd=("PADE6",) * 3, filter="COMPACT10", alphaF=0.49, rk="RK4", mu_ref=0.002)
    from mpi_3dcompact_b200.hit_ic import hit_initial_condition
    ic = hit_initial_condition(16, k0=4.0, seed=1, mt=0.3)
    q, info, _ = _run(cfg, ic, 10)
    qo, st = O.run(cfg, ic, 10)
    for i in range(5):
        assert H.rel_max(q[i], qo[i]) <= 1e-12, i
        assert H.rel_l2(q[i], qo[i]) <= 1e-12, i
    assert info["time_step"] == st.time_step == 10
    assert info["stages"] == 40


def test_general_metrics_vs_oracle():
    """Non-constant metric fields exercise the per-point metric path."""
    cfg = O.Config(N=(16, 14, 12), fd=("PENTA10", "PADE6", "PADE6"), filter="COMPACT8", alphaF=0.45, rk="KENRK4",
                   les="VREMAN", mu_ref=0.003)
    met = O.cube_metrics(cfg.N)
    Nx, Ny, Nz = cfg.N
    z, y, x = np.meshgrid(np.arange(Nz) / Nz, np.arange(Ny) / Ny, np.arange(Nx) / Nx, indexing="ij")
    bump = 1.0 + 0.05 * np.sin(2 * math.pi * x) * np.cos(2 * math.pi * y) * np.sin(2 * math.pi * z + 0.3)
    met = [met[0] * bump] + [mm + 0.01 * np.sin(2 * math.pi * (x + 2 * y)) * (c % 4 == 0) for c, mm in
                             enumerate(met[1:], start=1)]
    ic = G.step_ic(cfg.N, 11)
    q, info, _ = _run(cfg, ic, 3, metrics=met)
    qo, st = O.run(cfg, ic, 3, metrics=met)
    for i in range(5):
        assert H.rel_max(q[i], qo[i]) <= 1e-12, i


def test_fp32bulk_vs_fp64():
    from mpi_3dcompact_b200.hit_ic import hit_initial_condition
    cfg = O.Config(N=(32, 32, 32), fd=("PENTA10",) * 3, filter="COMPACT8", alphaF=0.45, rk="LSLDDRK4",
                   les="VREMAN", mu_ref=0.001)
    ic = hit_initial_condition(32, k0=4.0, seed=2, mt=0.3)
    q64, _, _ = _run(cfg, ic, 20, precision=m.FP64)
    q32, _, _ = _run(cfg, ic, 20, precision=m.FP32BULK)
    for i in range(5):
        # momenta have zero mean: compare against the field's own scale
        assert H.rel_l2(q32[i], q64[i]) <= 1e-5, (i, H.rel_l2(q32[i], q64[i]))


def test_mass_is_conserved():
    from mpi_3dcompact_b200.hit_ic import hit_initial_condition
    cfg = O.Config(N=(24, 24, 24), fd=("PADE6",) * 3, filter="COMPACT10", alphaF=0.49, rk="RK4", mu_ref=0.002)
    ic = hit_initial_condition(24, k0=4.0, seed=3, mt=0.3)
    s = m.CurvilinearCSolver(_opts(cfg))
    s.set_box_metrics(2 * math.pi)
    s.set_initial_conditions(*ic)
    ke0, m0 = s.integrals()
    s.step(5)
    ke1, m1 = s.integrals()
    assert abs(m1 - m0) <= 1e-12 * m0
    assert 0 < ke1 < ke0          # decaying turbulence


def test_solver_rejects_unsupported_configs():
    with pytest.raises(m.Mc3dError):
        m.CurvilinearCSolver(m.Options(grid=16, les="DSM", dsm_test_filter=3))
    with pytest.raises(m.Mc3dError):
        m.CurvilinearCSolver(m.Options(grid=(16, 16, 8)))


@pytest.mark.parametrize("prec,tol", [(m.FP64, 1e-12), (m.FP32BULK, 1e-5)])
@pytest.mark.parametrize("ft,avg", [(1, "XI2_AVG"), (2, "GLOBAL")])
def test_dsm_64cube_vs_oracle(ft, avg, prec, tol):
    """Dynamic Smagorinsky on 64^3 (segmented test-filter sweeps of 24 and 10
    fields, averaging reductions) against the oracle after two steps."""
    from mpi_3dcompact_b200.hit_ic import hit_initial_condition
    cfg = O.Config(N=(64, 64, 64), fd=("PADE6",) * 3, filter="COMPACT10", alphaF=0.49, rk="RK4", mu_ref=0.001,
                   les="DSM", les_avg=avg, dsm_test_filter=ft)
    ic = hit_initial_condition(64, k0=4.0, seed=11, mt=0.3)
    q, info, _ = _run(cfg, ic, 2, precision=prec)
    qo, st = O.run(cfg, ic, 2)
    for i in range(5):
        assert H.rel_l2(q[i], qo[i]) <= tol, (i, H.rel_l2(q[i], qo[i]))


@pytest.mark.parametrize("prec,tol", [(m.FP64, 1e-12), (m.FP32BULK, 1e-5)])
def test_64cube_two_steps_vs_oracle(prec, tol):
    """64^3 lines take the segmented line-solve kernels in every sweep
    (gradients, flux divergence with all epilogues, filter)."""
    from mpi_3dcompact_b200.hit_ic import hit_initial_condition
    cfg = O.Config(N=(64, 64, 64), fd=("PENTA10",) * 3, filter="COMPACT8", alphaF=0.45, rk="LSLDDRK4",
                   les="VREMAN", mu_ref=0.001)
    ic = hit_initial_condition(64, k0=4.0, seed=6, mt=0.3)
    q, info, _ = _run(cfg, ic, 2, precision=prec)
    qo, st = O.run(cfg, ic, 2)
    for i in range(5):
        assert H.rel_l2(q[i], qo[i]) <= tol, (i, H.rel_l2(q[i], qo[i]))


def _wall_opts(cfg, precision=m.FP64):
    return m.Options(grid=cfg.N, fd=cfg.fd, filter=cfg.filter, alphaF=cfg.alphaF, mu_ref=cfg.mu_ref, rk=cfg.rk,
                     ts_type=cfg.ts_type, cfl=cfg.cfl, dt=cfg.dt, filter_step=cfg.filter_step,
                     substep_filtering=cfg.substep_filtering, les=cfg.les, les_avg=cfg.les_avg, precision=precision,
                     bc=cfg.bc, bc_kind=cfg.kinds(), sponge=cfg.sponge)


@pytest.mark.parametrize("name", list(G.WALL_CASES))
def test_boundary_cases_match_reference_solver(name):
    """Walls, sponges and the O-grid cylinder (curvilinear metrics of the
    reference) against the reference solver's output: <= 1e-12 relative."""
    cfg, ic, n, coords = G.wall_case(name)
    gold = H.golden_steps()
    opt = _wall_opts(cfg)
    s = m.CurvilinearCSolver(opt)
    s.set_metrics([gold[f"{name}_met{c}"] for c in range(10)])
    if cfg.sponge:
        s.set_sponge(m.sponge_sigma(opt, *coords))
    s.set_initial_conditions(*ic)
    s.step(n)
    q = s.conserved()
    for i in range(5):
        err = H.rel_max(q[i], gold[f"{name}_q{i}"])
        assert err <= 1e-12, (name, i, err)
    ts, t, dt = gold[f"{name}_info"]
    assert s.info()["time_step"] == int(ts)


def test_boundary_case_fp32bulk():
    """FP32-bulk on the O-grid cylinder stays within 1e-5 of the FP64 path."""
    name = "ogrid_cyl_sponge_kenrk4"
    cfg, ic, n, coords = G.wall_case(name)
    gold = H.golden_steps()
    outs = []
    for prec in (m.FP64, m.FP32BULK):
        opt = _wall_opts(cfg, prec)
        s = m.CurvilinearCSolver(opt)
        s.set_metrics([gold[f"{name}_met{c}"] for c in range(10)])
        s.set_sponge(m.sponge_sigma(opt, *coords))
        s.set_initial_conditions(*ic)
        s.step(n)
        outs.append(s.conserved())
    # momentum errors against the momentum-vector norm: the cross-stream
    # components are a 0.2% disturbance of a Mach 0.2 stream along x
    mom = np.sqrt(sum(np.sum(outs[0][i] ** 2) for i in (1, 2, 3)))
    for i in range(5):
        scale = mom if i in (1, 2, 3) else np.sqrt(np.sum(outs[0][i] ** 2))
        err = np.sqrt(np.sum((outs[1][i] - outs[0][i]) ** 2)) / scale
        assert err <= 1e-5, (i, err)


def test_fp32bulk_tma_line_solves_follow_fp64():
    """FP32-bulk on 128^3 (every line solve TMA-staged: gradients, divergences,
    k2 assembly, the filter's FP32 and FP64 stores in all three rotations)
    stays within 1e-5 relative L2 of the FP64 path after three steps."""
    import math
    from mpi_3dcompact_b200.hit_ic import hit_initial_condition
    n = 128
    ic = hit_initial_condition(n, k0=4.0, seed=3, mt=0.3)
    outs = []
    for prec in (m.FP64, m.FP32BULK):
        s = m.CurvilinearCSolver(m.Options(grid=n, fd="PENTA10", filter="COMPACT8", alphaF=0.45, mu_ref=2.5e-4,
                                           rk="LSLDDRK4", les="VREMAN", cfl=0.5, precision=prec))
        s.set_box_metrics(2 * math.pi)
        s.set_initial_conditions(*ic)
        s.step(3)
        outs.append(s.conserved())
    for i in range(5):
        err = np.linalg.norm(outs[1][i] - outs[0][i]) / np.linalg.norm(outs[0][i])
        assert err <= 1e-5, (i, err)
    assert m.tma_wait_timeouts(0) == 0


def test_ten_steps_match_reference_solver():
    """The bench's scheme for 10 time steps (55 LSLDDRK4 stages) on 64 x 24 x 16:
    FP64 within 1e-12 relative of the reference solver per conserved field,
    FP32-bulk within 1e-5 relative L2; same time step, time within the same
    tolerances."""
    cfg, ic, n = G.ten_step_case()
    gold = np.load(os.path.join(G.HERE, "ten_steps.npz"))
    for prec, tol in ((m.FP64, 1e-12), (m.FP32BULK, 1e-5)):
        s = m.CurvilinearCSolver(m.Options(grid=cfg.N, fd=cfg.fd, filter=cfg.filter, alphaF=cfg.alphaF,
                                           mu_ref=cfg.mu_ref, rk=cfg.rk, les=cfg.les, cfl=cfg.cfl, precision=prec))
        s.set_box_metrics(2.0 * np.pi)
        s.set_initial_conditions(*ic)
        s.step(n)
        q = s.conserved()
        for i in range(5):
            ref = gold[f"q{i}"]
            err = H.rel_max(q[i], ref) if prec == m.FP64 else np.linalg.norm(q[i] - ref) / np.linalg.norm(ref)
            assert err <= tol, (prec, i, err)
        info = s.info()
        assert info["time_step"] == int(gold["info"][0])
        # FP32-bulk: dt from the CFL maximum over FP32 primitives
        assert abs(info["time"] - gold["info"][1]) <= tol * gold["info"][1], (prec, info["time"])


def _hit_solver(n, prec, ic):
    s = m.CurvilinearCSolver(m.Options(grid=n, fd="PENTA10", filter="COMPACT8", alphaF=0.45, mu_ref=2.5e-4,
                                       rk="LSLDDRK4", les="VREMAN", cfl=0.5, precision=prec))
    s.set_box_metrics(2 * math.pi)
    s.set_initial_conditions(*ic)
    return s


def test_concurrent_solvers_on_own_streams_do_not_interfere():
    """Two solvers on one device, each on a stream of its own (an FP32-bulk
    256^3 case through the TMA-staged line solves and an FP64 one), stepped
    alternately without waiting so that their kernels overlap: in each of
    three trials the FP32-bulk state equals running it alone, bit for bit."""
    import torch
    from mpi_3dcompact_b200.hit_ic import hit_initial_condition
    n = 256
    ic = hit_initial_condition(n, k0=4.0, seed=1, mt=0.3)
    alone = _hit_solver(n, m.FP32BULK, ic)
    alone.step(4)
    ref = alone.conserved()
    del alone
    sa, sb = torch.cuda.Stream(), torch.cuda.Stream()
    for trial in range(3):
        a, b = _hit_solver(n, m.FP32BULK, ic), _hit_solver(n, m.FP64, ic)
        a.set_stream(sa.cuda_stream)
        b.set_stream(sb.cuda_stream)
        for _ in range(4):
            a.step(1)
            b.step(1)
        got = a.conserved()
        b.sync()
        for i in range(5):
            assert np.array_equal(got[i], ref[i]), (trial, i, float(np.nanmax(np.abs(got[i] - ref[i]))))
        del a, b
    assert m.tma_wait_timeouts(0) == 0


def test_operator_calls_on_default_stream_overlap_a_solver_step():
    """Operator calls on the legacy default stream (mc3d_op_apply with a NULL
    stream, as a reference-side adapter makes them: FP32 Penta10 along x, y
    and z of five 256^3 fields, FP64 along x) queued while an FP32-bulk solver
    steps on its own non-blocking stream: the operator results and the solver
    state both equal their solo runs bit for bit."""
    import torch
    from mpi_3dcompact_b200.hit_ic import hit_initial_condition
    n = 256
    ic = hit_initial_condition(n, k0=4.0, seed=2, mt=0.3)
    alone = _hit_solver(n, m.FP32BULK, ic)
    alone.step(2)
    ref = alone.conserved()
    del alone
    g = torch.Generator(device="cuda").manual_seed(5)
    x32 = [torch.randn(n, n, n, device="cuda", generator=g) for _ in range(5)]
    x64 = [torch.randn(n, n, n, device="cuda", generator=g, dtype=torch.float64) for _ in range(5)]
    ops32 = [m.Penta10((n, n, n), m.PERIODIC_SOLVE, d, precision=m.FP32BULK) for d in range(3)]
    op64 = m.Penta10((n, n, n), m.PERIODIC_SOLVE, 0)
    y32 = [[torch.empty_like(x32[0]) for _ in range(5)] for _ in range(3)]
    y64 = [torch.empty_like(x64[0]) for _ in range(5)]
    for d in range(3):
        ops32[d].calc1stDerivFields(x32, y32[d])
    op64.calc1stDerivFields(x64, y64)
    torch.cuda.synchronize()
    solo32 = [[t.clone() for t in y32[d]] for d in range(3)]
    solo64 = [t.clone() for t in y64]
    s = _hit_solver(n, m.FP32BULK, ic)
    own = torch.cuda.Stream()
    s.set_stream(own.cuda_stream)
    for _ in range(2):
        for d in range(3):
            for t in y32[d]:
                t.zero_()
        torch.cuda.synchronize()
        s.step(1)                      # queued on the solver's stream
        for d in range(3):             # queued on the legacy default stream meanwhile
            ops32[d].calc1stDerivFields(x32, y32[d])
            op64.calc1stDerivFields(x64, y64)
        torch.cuda.synchronize()
        for d in range(3):
            for f in range(5):
                assert torch.equal(y32[d][f], solo32[d][f]), (d, f)
        for f in range(5):
            assert torch.equal(y64[f], solo64[f]), f
    got = s.conserved()
    for i in range(5):
        assert np.array_equal(got[i], ref[i]), (i, float(np.nanmax(np.abs(got[i] - ref[i]))))
    assert m.tma_wait_timeouts(0) == 0


def test_fp32_line_solves_stay_bit_stable_under_overlapping_sweeps():
    """FP32 Penta10 derivatives of five 256^3 fields along x, y and z (the
    TMA-staged persistent kernels) on one stream while FP64 x sweeps (the
    register kernel, staging its tiles with per-element asynchronous copies)
    run on another: ten rounds, every output equal to the solo result."""
    import torch
    n = 256
    g = torch.Generator(device="cuda").manual_seed(9)
    xa = [torch.randn(n, n, n, device="cuda", generator=g) for _ in range(5)]
    xb = [torch.randn(n, n, n, device="cuda", generator=g, dtype=torch.float64) for _ in range(5)]
    opa = [m.Penta10((n, n, n), m.PERIODIC_SOLVE, d, precision=m.FP32BULK) for d in range(3)]
    opb = m.Penta10((n, n, n), m.PERIODIC_SOLVE, 0)
    ya = [[torch.empty_like(xa[0]) for _ in range(5)] for _ in range(3)]
    yb = [torch.empty_like(xb[0]) for _ in range(5)]
    sa, sb = torch.cuda.Stream(), torch.cuda.Stream()
    for d in range(3):
        opa[d].calc1stDerivFields(xa, ya[d], stream=sa.cuda_stream)
    torch.cuda.synchronize()
    ref = [[t.clone() for t in ya[d]] for d in range(3)]
    for rnd in range(10):
        for d in range(3):
            for t in ya[d]:
                t.zero_()
        torch.cuda.synchronize()
        for _ in range(3):
            opb.calc1stDerivFields(xb, yb, stream=sb.cuda_stream)
        for d in range(3):
            opa[d].calc1stDerivFields(xa, ya[d], stream=sa.cuda_stream)
            opb.calc1stDerivFields(xb, yb, stream=sb.cuda_stream)
        torch.cuda.synchronize()
        for d in range(3):
            for f in range(5):
                assert torch.equal(ya[d][f], ref[d][f]), (rnd, d, f)
    assert m.tma_wait_timeouts(0) == 0


def test_stage_by_stage_calls_equal_the_step():
    """The stage-level calls in the reference's RK loop order (preStep, then
    per stage preSubStep, solveEqnSet, postSubStep, updateConservedData,
    updateData, then postStep) give mc3d_solver_step's state bit for bit, over
    both LSLDDRK4 halves; a call out of order is refused and changes nothing."""
    import ctypes as C
    from mpi_3dcompact_b200 import _native as N
    from mpi_3dcompact_b200.hit_ic import hit_initial_condition
    lib = N.host_lib()
    n = 32
    ic = hit_initial_condition(n, k0=4.0, seed=12, mt=0.3)
    a, b = _hit_solver(n, m.FP32BULK, ic), _hit_solver(n, m.FP32BULK, ic)
    a.step(3)
    h = b._h
    assert lib.mc3d_solver_pre_substep(h, 1) == 1          # before preStep: refused
    for step in range(3):
        N.check(lib.mc3d_solver_pre_step(h))
        ns = C.c_int()
        N.check(lib.mc3d_solver_stage_count(h, C.byref(ns)))
        assert ns.value == (5 if step % 2 == 0 else 6)
        for st in range(1, ns.value + 1):
            N.check(lib.mc3d_solver_pre_substep(h, st))
            N.check(lib.mc3d_solver_solve_eqn_set(h))
            N.check(lib.mc3d_solver_post_substep(h))
            assert lib.mc3d_rk_update(h, m.LSLDDRK4, st, 2 if step % 2 == 0 else 1) == 1   # wrong half
            N.check(lib.mc3d_rk_update(h, m.LSLDDRK4, st, 1 if step % 2 == 0 else 2))
            N.check(lib.mc3d_solver_update_data(h, int(st == ns.value)))
        N.check(lib.mc3d_solver_post_step(h))
    qa, qb = a.conserved(), b.conserved()
    for i in range(5):
        assert np.array_equal(qa[i], qb[i]), i
    assert a.info() == b.info()


@pytest.mark.parametrize("prec,tol", [(m.FP64, 1e-13), (m.FP32BULK, 3e-6)])
@pytest.mark.parametrize("scheme", ["PADE6", "PENTA10", "CD2"])
def test_tpb_derivative_matches_oracle(scheme, prec, tol):
    """calc1stDerivField_TPB with caller ghost planes (mc3d_op_apply_tpb) along
    each direction against the oracle's restatement of the reference's TPB rows
    (pinned through the metric fixtures)."""
    import torch
    cls = {"PADE6": m.Pade6, "PENTA10": m.Penta10, "CD2": m.CD2}[scheme]
    rng = np.random.default_rng(3)
    shape = (20, 24, 32)          # (Nz, Ny, Nx)
    f = rng.standard_normal(shape)
    dt = torch.float64 if prec == m.FP64 else torch.float32
    G = 3 if scheme == "PENTA10" else 2
    for d in range(3):
        ax = 2 - d
        nline = shape[ax]
        pshape = tuple(s for a, s in enumerate(shape) if a != ax)
        ghosts = [rng.standard_normal(pshape) for _ in range(2 * G)]   # Nm_G .. Nm_1, Np_1 .. Np_G
        op = cls(shape, m.PERIODIC_SOLVE, d, precision=prec)
        x = torch.tensor(f, dtype=dt, device="cuda")
        y = torch.empty_like(x)
        op.calc1stDerivField_TPB(x, y, *[torch.tensor(g, dtype=dt, device="cuda") for g in ghosts])
        lines = np.moveaxis(f, ax, -1)
        gm = np.stack([ghosts[G - mm] for mm in range(1, G + 1)], axis=-1)
        gp = np.stack([ghosts[G + mm - 1] for mm in range(1, G + 1)], axis=-1)
        ref = np.moveaxis(O._tpb_lines(lines, gm, gp, scheme, 1.0 / nline), -1, ax)
        err = H.rel_max(y.double().cpu().numpy(), ref)
        assert err <= tol, (scheme, d, err)
