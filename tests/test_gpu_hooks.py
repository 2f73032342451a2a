"""GPU tests of the drivers' diagnostic hooks as device reductions.

* Against the reference's own hook code (tests/golden/hooks.npz, written by
  the harness built with the hooks of tests/hit/Samtaney_D4/MPI_3DCompact.cpp
  and src/MPI_3DCompact.cpp): the HIT turbdata.out lines after steps 25 and 50
  of a 24^3 run, and the cylinder's span-averaged wall p, U, V, W after step 50
  and the V strip at (i, j) = (0, 143) after each of 50 steps on a
  16 x 150 x 12 O-grid whose metrics the GPU computes from the mesh.
  Tolerances: 1e-10 relative for turbdata (sums of products of derivatives in
  another order), 1e-9 of the record's largest value for the cylinder records
  (the GPU metrics differ from the reference's by rounding, 1e-13, and 50
  steps of a wall-bounded flow carry that).
* Against the oracle's restatement on the same state: the HIT line (1e-10)
  and the wall averages (1e-14, same summation order)."""
import math
import os

import numpy as np
import pytest

import mpi_3dcompact_b200 as m
from oracle import mc3d_oracle as O
from tests import helpers as H
from tests.golden import gen_golden as G

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["pade6_rk4_c10", "mixed_rk4_noncubic"])
def test_turbdata_matches_restatement(name):
    cfg, ic, n = H.oracle_config(name)
    s = m.CurvilinearCSolver(m.Options(grid=cfg.N, fd=cfg.fd, filter=cfg.filter, alphaF=cfg.alphaF,
                                       mu_ref=cfg.mu_ref, rk=cfg.rk, cfl=cfg.cfl, les=cfg.les, les_avg=cfg.les_avg))
    s.set_box_metrics(2.0 * math.pi)
    s.set_initial_conditions(*ic)
    s.step(n)
    got = s.turbdata(8.0)
    o = O.Oracle(cfg, O.cube_metrics(cfg.N))
    o.init(*ic)
    for _ in range(n):
        o.step()
    want = O.hit_turbdata(o, 8.0)
    for k, (a, b) in enumerate(zip(got, want)):
        assert abs(a - b) <= 1e-10 * abs(b) + 1e-300, (k, a, b)


def test_turbdata_matches_reference_hook():
    from mpi_3dcompact_b200.hit_ic import hit_initial_condition
    grid, kw, n, seed = G.HOOK_HIT
    gold = np.load(os.path.join(G.HERE, "hooks.npz"))["hit_turbdata"]
    s = m.CurvilinearCSolver(m.Options(grid=grid, **kw))
    s.set_box_metrics(2.0 * math.pi)
    s.set_initial_conditions(*hit_initial_condition(grid[0], k0=4.0, seed=seed, mt=0.3))
    lines = []
    for step in range(1, n + 1):
        s.step(1)
        if step % 25 == 0:           # the driver writes a line every 25 steps
            lines.append(s.turbdata(8.0))
    assert len(lines) == len(gold) == 2
    for got, want in zip(lines, gold):
        for k, (a, b) in enumerate(zip(got, want)):
            assert abs(a - b) <= 1e-10 * abs(b) + 1e-300, (k, a, b)


def test_cylinder_hooks_match_reference_hooks():
    cfg, ic, n, coords = G.hook_cyl_case()
    gold = np.load(os.path.join(G.HERE, "hooks.npz"))
    opt = m.Options(grid=cfg.N, fd=cfg.fd, filter=cfg.filter, alphaF=cfg.alphaF, mu_ref=cfg.mu_ref, rk=cfg.rk,
                    cfl=cfg.cfl, bc=cfg.bc, bc_kind=cfg.kinds(), sponge=cfg.sponge,
                    periodic_disp=O.periodic_disp_table(cfg))
    s = m.CurvilinearCSolver(opt)
    s.set_mesh(*coords)
    s.set_sponge(m.sponge_sigma(opt, *coords))
    s.set_initial_conditions(*ic)
    strip_gold = gold["cyl_VWakeStrip"]
    assert strip_gold.shape[0] == n
    for step in range(1, n + 1):
        s.step(1)
        t = s.info()["time"]
        row = strip_gold[step - 1]
        assert abs(t - row[0]) <= 1e-12 * max(abs(row[0]), 1e-30), (step, t, row[0])
        got = s.wake_strip(0, 143)
        assert np.abs(got - row[1:]).max() <= 1e-9 * np.abs(row[1:]).max(), step
    avgs = s.wall_span_average()
    for name, got in zip(("cylinderP", "cylinderU", "cylinderV", "cylinderW"), avgs):
        row = gold[f"cyl_{name}"][-1]
        assert abs(s.info()["time"] - row[0]) <= 1e-12 * row[0]
        assert np.abs(got - row[1:]).max() <= 1e-9 * max(np.abs(row[1:]).max(), 1e-300), name


def test_wall_span_average_matches_restatement():
    name = "ogrid_cyl_sponge_kenrk4"
    cfg, ic, n, coords = G.wall_case(name)
    opt = m.Options(grid=cfg.N, fd=cfg.fd, filter=cfg.filter, alphaF=cfg.alphaF, mu_ref=cfg.mu_ref, rk=cfg.rk,
                    cfl=cfg.cfl, bc=cfg.bc, bc_kind=cfg.kinds(), sponge=cfg.sponge,
                    periodic_disp=O.periodic_disp_table(cfg))
    s = m.CurvilinearCSolver(opt)
    s.set_mesh(*coords)
    s.set_sponge(m.sponge_sigma(opt, *coords))
    s.set_initial_conditions(*ic)
    s.step(n)
    got = s.wall_span_average()
    want = O.wall_span_average(s.conserved())
    for a, b in zip(got, want):
        assert np.abs(a - b).max() <= 1e-14 * max(np.abs(b).max(), 1.0)
    # a no-slip wall: the averaged wall velocity is zero
    assert max(np.abs(a).max() for a in got[1:]) == 0.0


@pytest.mark.parametrize("name", list(G.RELAX_CASES))
def test_sponge_relaxation_matches_reference(name):
    """updateSponge after every step (left commented out in the reference's
    postStep, called by the fixture run): FP64 against the reference's state,
    <= 1e-12 relative, and the relaxation changes the result."""
    cfg, ic, n, coords, base = G.relax_case(name)
    gold, relaxed = H.golden_steps(), H.golden_relax()
    opt = m.Options(grid=cfg.N, fd=cfg.fd, filter=cfg.filter, alphaF=cfg.alphaF, mu_ref=cfg.mu_ref, rk=cfg.rk,
                    ts_type=cfg.ts_type, cfl=cfg.cfl, dt=cfg.dt, filter_step=cfg.filter_step,
                    substep_filtering=cfg.substep_filtering, les=cfg.les, les_avg=cfg.les_avg,
                    dsm_test_filter=cfg.dsm_test_filter, bc=cfg.bc, bc_kind=cfg.kinds(), sponge=cfg.sponge,
                    sponge_relax=cfg.sponge_relax)
    s = m.CurvilinearCSolver(opt)
    s.set_metrics([gold[f"{base}_met{c}"] for c in range(10)])
    s.set_sponge(m.sponge_sigma(opt, *coords))
    s.set_initial_conditions(*ic)
    s.step(n)
    got = s.conserved()
    for i in range(5):
        err = H.rel_max(got[i], relaxed[f"{name}_q{i}"])
        assert err <= 1e-12, (i, err)
    if base == name:
        assert max(H.rel_max(got[i], gold[f"{name}_q{i}"]) for i in range(5)) > 1e-6
    ts, t, dt = relaxed[f"{name}_info"]
    assert s.info()["time_step"] == int(ts)


def test_wake_strip_and_cylinder_records(tmp_path):
    """The wake strip is V = rhoV / rho of the state along xi3 at (i, j); the
    record files carry the time then the values; a strip point outside the
    grid gives the driver's -100000 fill and the ABI call rejects it."""
    name = "ogrid_cyl_sponge_kenrk4"
    cfg, ic, n, coords = G.wall_case(name)
    opt = m.Options(grid=cfg.N, fd=cfg.fd, filter=cfg.filter, alphaF=cfg.alphaF, mu_ref=cfg.mu_ref, rk=cfg.rk,
                    cfl=cfg.cfl, bc=cfg.bc, bc_kind=cfg.kinds(), sponge=cfg.sponge,
                    periodic_disp=O.periodic_disp_table(cfg))
    s = m.CurvilinearCSolver(opt)
    s.set_mesh(*coords)
    s.set_sponge(m.sponge_sigma(opt, *coords))
    s.set_initial_conditions(*ic)
    s.step(n)
    q = s.conserved()
    i, j = 3, 7
    assert np.array_equal(s.wake_strip(i, j), q[2][:, j, i] / q[0][:, j, i])
    with pytest.raises(Exception):
        s.wake_strip(0, cfg.N[1])
    s.write_cylinder_data(tmp_path, strip=(i, j))
    s.write_cylinder_data(tmp_path)   # the driver's (0, 143): outside this 24 x 20 x 12 grid
    t = s.info()["time"]
    nx, nz = cfg.N[0], cfg.N[2]
    for k, a in enumerate(s.wall_span_average()):
        raw = np.fromfile(tmp_path / f"cylinder{'PUVW'[k]}.dat", dtype=np.float64)
        assert raw.size == 2 * (1 + nx) and raw[0] == t and np.array_equal(raw[1:1 + nx], a)
    raw = np.fromfile(tmp_path / "VWakeStrip.dat", dtype=np.float64)
    assert raw.size == 2 * (1 + nz) and raw[0] == t
    assert np.array_equal(raw[1:1 + nz], q[2][:, j, i] / q[0][:, j, i])
    assert np.all(raw[2 + nz:] == -100000.0)
