"""GPU tests of checkpoints in the reference's formats: restarting from a
SolutionDump the reference wrote and stepping on against the reference's own
restart run, dumping after the same steps as the reference's dump, the sponge
average file, and the driver loop (DUMPSTEP dumps, end dump, killsolver).

Tolerances: 1e-12 of each field's largest magnitude on the periodic box; 1e-11
on the O-grid, whose restart recomputes the metrics on the GPU (determinant and
cofactors within ~1e-13 of the reference's)."""
import math
import os

import numpy as np
import pytest

import mpi_3dcompact_b200 as m
from oracle import mc3d_oracle as O
from tests.golden import gen_golden as G

pytestmark = pytest.mark.gpu

TOL = {"hit_pade6_rk4": 1e-12, "ogrid_cyl_sponge_kenrk4": 1e-11}


def _gold():
    return np.load(os.path.join(G.HERE, "checkpoint.npz"))


def _opts(cfg, **kw):
    return m.Options(grid=cfg.N, fd=cfg.fd, filter=cfg.filter, alphaF=cfg.alphaF, mu_ref=cfg.mu_ref, rk=cfg.rk,
                     cfl=cfg.cfl, les=cfg.les, les_avg=cfg.les_avg, precision=m.FP64, bc=cfg.bc,
                     bc_kind=cfg.kinds(), sponge=cfg.sponge, periodic_disp=O.periodic_disp_table(cfg), **kw)


def _rel(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


@pytest.mark.parametrize("name", list(G.CHECKPOINT_CASES))
def test_restart_from_reference_dump(name, tmp_path):
    cfg, _, _, n1, n2 = G.checkpoint_case(name)
    gold = _gold()
    path = tmp_path / f"SolutionDump.{n1}"
    path.write_bytes(gold[f"{name}_dump"].tobytes())
    s = m.CurvilinearCSolver(_opts(cfg))
    s.restart(path)
    s.step(n2)
    q = s.conserved()
    info = s.info()
    ts, t, dt = gold[f"{name}_restart_info"]
    assert info["time_step"] == int(ts)
    assert abs(info["time"] - t) <= 1e-12 * abs(t)
    for i in range(5):
        err = _rel(q[i], gold[f"{name}_restart_q{i}"])
        assert err <= TOL[name], (name, i, err)


@pytest.mark.parametrize("name", list(G.CHECKPOINT_CASES))
def test_dump_matches_reference_dump(name, tmp_path):
    cfg, ic, coords, n1, _ = G.checkpoint_case(name)
    gold = _gold()
    s = m.CurvilinearCSolver(_opts(cfg))
    if coords is None:
        s.set_box_metrics(2.0 * math.pi)
    else:
        s.set_mesh(*coords)
    if cfg.sponge:
        s.set_sponge(m.sponge_sigma(s.opt, *coords))
    s.set_initial_conditions(*ic)
    s.step(n1)
    out = tmp_path / "dump"
    s.dump(out)
    hdr, f = m.read_dump(out)
    rhdr, rf = O.parse_solution_dump(gold[f"{name}_dump"].tobytes())
    assert hdr["time_step"] == rhdr["time_step"] and hdr["N"] == rhdr["N"]
    assert abs(hdr["time"] - rhdr["time"]) <= 1e-12 * abs(rhdr["time"])
    for k in range(3):
        assert np.array_equal(f[k], rf[k]), k
    for k in range(3, 8):
        assert _rel(f[k], rf[k]) <= TOL[name], k
    if cfg.sponge:
        sp = tmp_path / "spg"
        s.dump_sponge_avg(sp)
        mine = np.fromfile(sp, dtype=np.float64)
        ref = np.frombuffer(gold[f"{name}_spongeavg"].tobytes(), dtype=np.float64)
        assert mine.size == ref.size and np.abs(mine - ref).max() <= 1e-15 * np.abs(ref).max()
        s2 = m.CurvilinearCSolver(_opts(cfg))
        s2.restart(out)
        s2.read_sponge_avg(sp)


def test_run_dumps_every_dumpstep_and_at_the_end(tmp_path):
    cfg, ic, _, _, _ = G.checkpoint_case("hit_pade6_rk4")
    s = m.CurvilinearCSolver(_opts(cfg, max_time_step=5, dump_step=2))
    s.set_box_metrics(2.0 * math.pi)
    s.set_initial_conditions(*ic)
    s.run(tmp_path)
    names = sorted(p.name for p in tmp_path.iterdir())
    assert names == ["SolutionDump.2", "SolutionDump.4", "SolutionDump.5"]
    hdr, f = m.read_dump(tmp_path / "SolutionDump.5")
    q = s.conserved()
    assert hdr["time_step"] == 5 and all(np.array_equal(f[3 + i], q[i]) for i in range(5))
    # a killsolver file ends the loop after the next step and is removed
    (tmp_path / "killsolver").write_text("")
    s2 = m.CurvilinearCSolver(_opts(cfg, max_time_step=100, dump_step=1000))
    s2.restart(tmp_path / "SolutionDump.5")
    s2.run(tmp_path)
    assert not (tmp_path / "killsolver").exists()
    assert (tmp_path / "SolutionDump.6").exists() and s2.info()["time_step"] == 6
