"""CPU tests of the oracle: the numpy restatement against golden fixtures made
by the reference solver itself (tests/golden/gen_golden.py), operator
known-answer tests, and a live comparison with oracle/_ref when it is built."""
import math
import os

import numpy as np
import pytest

from oracle import mc3d_oracle as O
from oracle import ref_runner as R
from tests import helpers as H
from tests.golden import gen_golden as G


@pytest.mark.parametrize("bname", list(G.OPS_BCS))
@pytest.mark.parametrize("op", G.OPS)
def test_oracle_ops_match_reference_fixtures(op, bname):
    gold = H.golden_ops()
    f = G.ops_input()
    bcs = G.OPS_BCS[bname]
    for d in range(3):
        ref = gold[f"{op}_{bname}_{d}"]
        if op in ("COMPACT8", "COMPACT10"):
            out = O.filt(f, d, op, G.OPS_ALPHA, bcs)
        elif op in ("TESTPADE", "TESTEXP"):
            out = O.test_filter(f, d, 1 if op == "TESTPADE" else 2, bcs)
        else:
            n = G.OPS_GRID[d]
            dh = 1.0 / n if bcs[d] == 0 else 1.0 / (n - 1.0)
            out = O.deriv(f, d, op, bcs[d], dh)
        # the restatement follows the reference's arithmetic order: bit-identical
        assert np.array_equal(out, ref), (op, bname, d, H.rel_max(out, ref))


@pytest.mark.parametrize("name", list(G.STEP_CASES))
def test_oracle_steps_match_reference_fixtures(name):
    cfg, ic, n = H.oracle_config(name)
    q, st = O.run(cfg, ic, n)
    gold = H.golden_steps()
    for i in range(5):
        assert H.rel_max(q[i], gold[f"{name}_q{i}"]) < 1e-13, (name, i)
    ts, t, dt = gold[f"{name}_info"]
    assert st.time_step == int(ts)
    assert abs(st.time - t) <= 1e-13 * abs(t)
    assert abs(st.dt - dt) <= 1e-13 * abs(dt)


def test_pade6_modified_wavenumber():
    """Known answer: d/dx sin(kx) for the periodic Pade6 scheme equals
    k'(k) cos(kx) with Lele's modified wavenumber (interior alpha=1/3,
    a=14/9, b=1/9; src/Pade6.hpp:70-75)."""
    n, k = 32, 3
    x = np.arange(n) / n
    f = np.sin(2 * math.pi * k * x)[None, None, :] * np.ones((2, 2, 1))
    out = O.deriv(f, 0, "PADE6", O.PERIODIC, 1.0 / n)
    w = 2 * math.pi * k / n
    kp = (14 / 9 * math.sin(w) + 1 / 9 / 2 * math.sin(2 * w)) / (1 + 2 / 3 * math.cos(w)) * n
    assert np.allclose(out[0, 0], kp * np.cos(2 * math.pi * k * x), atol=1e-12)


def test_filter_transfer_function():
    """Known answer: the periodic compact filter scales sin(kx) by its transfer
    function T(w) = sum_k a_k cos(kw) / (1 + 2 alpha cos w) and removes the
    Nyquist mode (src/Compact10Filter.hpp:58-63)."""
    n, af = 32, 0.45
    x = np.arange(n) / n
    for ftype in ("COMPACT8", "COMPACT10"):
        a, _ = O.compact10_coeffs(af) if ftype == "COMPACT10" else O.compact8_coeffs(af)
        for k in (2, 5, 9):
            f = np.sin(2 * math.pi * k * x)[None, None, :] * np.ones((1, 1, 1))
            out = O.filt(f, 0, ftype, af, (0, 0, 0))
            w = 2 * math.pi * k / n
            T = sum(a[m] * math.cos(m * w) for m in range(len(a))) / (1 + 2 * af * math.cos(w))
            assert np.allclose(out[0, 0], T * f[0, 0], atol=1e-13)
        nyq = np.cos(math.pi * np.arange(n))[None, None, :]
        assert np.max(np.abs(O.filt(nyq, 0, ftype, af, (0, 0, 0)))) < 1e-12


def test_cube_metrics_match_reference_metrics():
    if not R.available():
        pytest.skip("oracle/_ref not built")
    cfg = O.Config(N=(12, 12, 12))
    ref = R.run_metrics(cfg)
    for a, b in zip(ref, O.cube_metrics(cfg.N)):
        assert np.max(np.abs(a - b)) < 1e-13


@pytest.mark.parametrize("name", list(G.METRIC_CASES))
def test_oracle_metrics_match_reference_fixtures(name):
    """solveForJacobians restated (TPB ghosts, translations, both BW7 ghost
    quirks) against the reference's own metrics of the same mesh: the
    restatement follows its arithmetic order, so it is bit-identical except for
    the sign of underflowed off-diagonal terms."""
    cfg, coords = G.metric_case(name)
    got = O.solve_for_jacobians(cfg, *coords)
    gold = H.golden_metrics()
    for c in range(10):
        ref = gold[f"{name}_met{c}"]
        assert np.abs(got[c] - ref).max() <= 1e-300 + 1e-15 * np.abs(ref).max(), (name, c)


def test_oracle_metrics_quirks_matter():
    """The BW7 ghost quirks change the PENTA10 metrics (so the fixtures pin them)."""
    cfg, coords = G.metric_case("wavy_penta10")
    a = O.solve_for_jacobians(cfg, *coords, quirks=True)
    b = O.solve_for_jacobians(cfg, *coords, quirks=False)
    assert max(H.rel_max(x, y) for x, y in zip(a, b)) > 1e-6


def test_oracle_metrics_of_the_cube_are_analytic():
    cfg = O.Config(N=(12, 13, 14))
    xi = [np.arange(n) / n for n in cfg.N]
    z, y, x = np.meshgrid(2 * math.pi * xi[2], 2 * math.pi * xi[1], 2 * math.pi * xi[0], indexing="ij")
    for a, b in zip(O.solve_for_jacobians(cfg, x, y, z), O.cube_metrics(cfg.N)):
        assert np.abs(a - b).max() < 1e-13


def test_oracle_live_reference_run():
    """Live check against the reference binary on a fresh configuration."""
    if not R.available():
        pytest.skip("oracle/_ref not built")
    cfg = O.Config(N=(12, 12, 12), fd=("PENTA10",) * 3, filter="COMPACT10", alphaF=0.4, rk="KENRK4",
                   mu_ref=0.002, cfl=0.4)
    ic = G.step_ic((12, 12, 12), 9)
    ref, info = R.run_solver(cfg, ic, 4)
    q, st = O.run(cfg, ic, 4)
    for i in range(5):
        assert H.rel_max(q[i], ref[i]) < 1e-13
    assert st.time_step == info["time_step"]


def test_hit_ic_is_seeded_and_solenoidal():
    from mpi_3dcompact_b200.hit_ic import hit_initial_condition
    a = hit_initial_condition(16, k0=4.0, seed=3, mt=0.3)
    b = hit_initial_condition(16, k0=4.0, seed=3, mt=0.3)
    c = hit_initial_condition(16, k0=4.0, seed=4, mt=0.3)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)
    assert not np.array_equal(a[1], c[1])
    u, v, w = a[1], a[2], a[3]
    assert abs(math.sqrt(np.mean(u * u + v * v + w * w)) - 0.3) < 1e-12
    # spectral divergence of the generated field is at round-off level
    n = 16
    k = np.fft.fftfreq(n, d=1.0 / n)
    div = (1j * k[None, None, :] * np.fft.fftn(u) + 1j * k[None, :, None] * np.fft.fftn(v)
           + 1j * k[:, None, None] * np.fft.fftn(w))
    assert np.max(np.abs(div)) / np.max(np.abs(np.fft.fftn(u))) < 1e-10


@pytest.mark.parametrize("name", list(G.WALL_CASES))
def test_oracle_boundary_cases_match_reference_fixtures(name):
    """Walls (adiabatic, the X1 constant-temperature quirk), rectilinear and
    cylindrical sponges, an O-grid cylinder: the reference's own metrics."""
    cfg, ic, n, coords = G.wall_case(name)
    gold = H.golden_steps()
    met = [gold[f"{name}_met{c}"] for c in range(10)]
    sigma = O.sponge_sigma(cfg, *coords) if cfg.sponge else None
    q, st = O.run(cfg, ic, n, metrics=met, sigma=sigma)
    for i in range(5):
        assert H.rel_max(q[i], gold[f"{name}_q{i}"]) < 1e-12, (name, i, H.rel_max(q[i], gold[f"{name}_q{i}"]))
    ts, t, dt = gold[f"{name}_info"]
    assert st.time_step == int(ts)
    assert abs(st.dt - dt) <= 1e-13 * abs(dt)


def test_oracle_turbdata_of_the_initial_field():
    """The HIT driver's statistics of the seeded initial field: Mt as scaled,
    rho' = 0 and mean rho|u|^2 = Mt^2 c^2 with c = 1."""
    cfg, ic, n = H.oracle_config("pade6_rk4_c10")
    o = O.Oracle(cfg, O.cube_metrics(cfg.N))
    o.init(*ic)
    t = O.hit_turbdata(o, 8.0)
    assert abs(t[3] - 0.3) < 1e-12 and t[7] < 1e-14
    assert abs(t[10] - 0.09) < 1e-12


@pytest.mark.parametrize("name", list(G.RELAX_CASES))
def test_oracle_sponge_relaxation_matches_reference_fixtures(name):
    """updateSponge restatement against the reference run with the call made
    after every step: <= 1e-12 relative; the SPONGE faces carry the relaxed
    target and its pressure moves toward SPONGE.PINF."""
    cfg, ic, n, coords, base = G.relax_case(name)
    gold, relaxed = H.golden_steps(), H.golden_relax()
    o = O.Oracle(cfg, [gold[f"{base}_met{c}"] for c in range(10)], sigma=O.sponge_sigma(cfg, *coords))
    o.init(*ic)
    for _ in range(n):
        o.step()
    for i in range(5):
        err = H.rel_max(o.state.q1[i], relaxed[f"{name}_q{i}"])
        assert err <= 1e-12, (i, err)
    kinds = cfg.kinds()
    faces = [f for f in range(6) if kinds[f] == "SPONGE"]
    assert faces
    for f in faces:
        sl = O._face_slices(f, o.state.q1[0].shape)[0]
        for v in range(5):
            assert np.array_equal(o.state.q1[v][sl], o.spg_avg[v][sl])
    a = o.spg_avg
    p = (O.GAMMA - 1.0) * (a[4] - 0.5 * (a[1] ** 2 + a[2] ** 2 + a[3] ** 2) / a[0])
    p_inf = cfg.sponge_relax["p_inf"]
    assert abs(float(np.mean(p)) - p_inf) < abs(1.0 / 1.4 - p_inf)


def test_oracle_ten_steps_match_reference_fixture():
    """The oracle restatement over 10 steps of the bench's scheme (64 x 24 x 16)
    against the reference solver: <= 1e-12 relative per conserved field."""
    import os
    cfg, ic, n = G.ten_step_case()
    gold = np.load(os.path.join(G.HERE, "ten_steps.npz"))
    q, st = O.run(cfg, ic, n)
    for i in range(5):
        err = H.rel_max(q[i], gold[f"q{i}"])
        assert err <= 1e-12, (i, err)
    assert st.time_step == int(gold["info"][0])


@pytest.mark.skipif(not R.available(), reason="oracle/_ref/mc3d_ref not built")
def test_reference_ogrid_dsm_local_nonfinite_at_128x64x32():
    """The reference's own solver on BASELINE's O-grid configuration (cylinder,
    wall, cylindrical sponge, PADE6, KENRK4, COMPACT10, DSM with the Pade test
    filter and LOCAL averaging) at 128 x 64 x 32: after one time step the
    momentum and energy fields hold non-finite values (LOCAL divides by a
    locally filtered M_ij M_ij); on 64 x 32 x 16 the same set-up stays finite
    for three steps. This is why the bench quotes the configuration's
    throughput with GLOBAL averaging."""
    from mpi_3dcompact_b200.meshes import cylinder_flow_ic, cylinder_ogrid

    def cfg(N):
        return O.Config(N=N, bc=(O.PERIODIC, O.DIRICHLET, O.PERIODIC),
                        bc_kind=("INTERNALLY_PERIODIC", "INTERNALLY_PERIODIC", "ADIABATIC_WALL", "SPONGE",
                                 "PERIODIC", "PERIODIC"),
                        fd=("PADE6",) * 3, filter="COMPACT10", alphaF=0.49, rk="KENRK4", mu_ref=0.2 / 3900.0,
                        les="DSM", les_avg="LOCAL", dsm_test_filter=1,
                        sponge=dict(kind="CYLINDRICAL", strength=1.0, orient=2, cyl_axis=[0.0, 0.0, 0.0], rmin=24.0),
                        periodic_box=(0.0, 0.0, 2.0))
    for N, steps, finite in (((64, 32, 16), 3, True), ((128, 64, 32), 1, False)):
        x, y, z, _ = cylinder_ogrid(*N)
        q, info = R.run_solver(cfg(N), cylinder_flow_ic(N[::-1]), steps, coords=(x, y, z))
        assert info["time_step"] == steps
        assert all(np.isfinite(a).all() for a in q) == finite, N
    assert np.isfinite(q[0]).all() and not any(np.isfinite(a).all() for a in q[1:])


@pytest.mark.skipif(not R.available(), reason="oracle/_ref/mc3d_ref not built")
@pytest.mark.parametrize("tf", [1, 2])
def test_reference_dsm_without_averaging_is_nonfinite(tf):
    """The reference's own solver with DSM and LESAVERAGING = NONE (either test
    filter) on a 16^3 HIT state: every value of every conserved field is NaN
    after one time step. doAveraging does nothing for NONE
    (src/AbstractSGS.cpp:160-162) while DSMSGS reads the averages from separate
    work arrays (src/DSMSGS.hpp:306-316), which nothing wrote: with the
    harness's zero-filled allocations the coefficient is 0/0. The GPU path
    takes NONE as no averaging (tests/test_gpu_configs.py)."""
    from mpi_3dcompact_b200.hit_ic import hit_initial_condition
    n = 16
    ic = hit_initial_condition(n, k0=4.0, seed=3, mt=0.3)
    cfg = O.Config(N=(n,) * 3, fd=("PADE6",) * 3, filter="COMPACT10", alphaF=0.49, rk="RK4", mu_ref=0.005,
                   les="DSM", les_avg="NONE", dsm_test_filter=tf)
    q, info = R.run_solver(cfg, ic, 1)
    assert info["time_step"] == 1
    assert all(np.isnan(a).all() for a in q)


def test_device_hit_generator_matches_numpy():
    """hit_velocity_device (the generator used for the 1024^3 block) draws the
    same LCG sequence as the numpy restatement, bit for bit, and gives the same
    field to FFT rounding (run here on the CPU device)."""
    import torch
    from mpi_3dcompact_b200 import hit_ic as HI
    g1, g2 = HI._Gen(5), HI._Gen(5)
    for n in (100003, 7):
        a = HI._vec_torch(torch, g1, n, "cpu").numpy()
        assert np.array_equal(a, g2.vec(n))
        assert (g1.ix1, g1.ix2, g1.ix3) == (g2.ix1, g2.ix2, g2.ix3) and g1.r == g2.r
    ref = HI.hit_velocity(16, 4.0, 3)
    got = HI.hit_velocity_device(16, 4.0, 3, device="cpu")
    for g, r in zip(got, ref):
        assert np.abs(g.numpy() - r).max() <= 1e-14 * np.abs(r).max()


def test_oracle_turbdata_matches_reference_hook():
    """The oracle's restatement of the HIT driver's turbdata hook against the
    reference's own hook output (tests/golden/hooks.npz) on the same run."""
    from mpi_3dcompact_b200.hit_ic import hit_initial_condition
    grid, kw, n, seed = G.HOOK_HIT
    gold = np.load(os.path.join(G.HERE, "hooks.npz"))["hit_turbdata"]
    cfg = O.Config(N=grid, **kw)
    o = O.Oracle(cfg, O.cube_metrics(cfg.N))
    o.init(*hit_initial_condition(grid[0], k0=4.0, seed=seed, mt=0.3))
    rows = []
    for step in range(1, n + 1):
        o.step()
        if step % 25 == 0:
            rows.append(O.hit_turbdata(o, 8.0))
    for got, want in zip(rows, gold):
        for k, (a, b) in enumerate(zip(got, want)):
            assert abs(a - b) <= 1e-11 * abs(b) + 1e-300, (k, a, b)
