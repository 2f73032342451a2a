"""GPU tests of the running statistics (Stats): the solver's statistics after
the steps of each STATS_CASES configuration against the VelocityStats /
ThermoStats files the reference wrote (tests/golden/stats.npz), and the stats
files' round trip.

Compared: the time weights (1e-13) and the well-conditioned moments behind the
RMS and Reynolds-stress fields (means, mean squares, mean products; 1e-12 of
each moment's largest magnitude), since RMS = sqrt(|<x^2> - <x>^2|) amplifies
the state's last-bit differences where fluctuations are small."""
import math

import numpy as np
import pytest

import mpi_3dcompact_b200 as m
from tests.golden import gen_golden as G
from tests.test_checkpoint import stats_errors

pytestmark = pytest.mark.gpu


def _solver(name, precision=m.FP64):
    cfg, ic, n = G.stats_case(name)
    opt = m.Options(grid=cfg.N, fd=cfg.fd, filter=cfg.filter, alphaF=cfg.alphaF, mu_ref=cfg.mu_ref, rk=cfg.rk,
                    cfl=cfg.cfl, filter_step=cfg.filter_step, substep_filtering=cfg.substep_filtering, les=cfg.les,
                    les_avg=cfg.les_avg, precision=precision, stats=cfg.stats)
    s = m.CurvilinearCSolver(opt)
    s.set_box_metrics(2.0 * math.pi)
    s.set_initial_conditions(*ic)
    return s, n


@pytest.mark.parametrize("name", list(G.STATS_CASES))
def test_stats_match_reference(name):
    s, n = _solver(name)
    s.step(n)
    st = s.stats()
    e_w, e_m = stats_errors(st["velocity"], st["thermo"], st["weights"], name)
    assert e_w <= 1e-13 and e_m <= 1e-12, (name, e_w, e_m)


def test_stats_files_round_trip(tmp_path):
    s, n = _solver("pade6_rk4_xi3_every2")
    s.step(n)
    s.dump_stats(tmp_path / "v", tmp_path / "t")
    a = s.stats()
    raw = np.fromfile(tmp_path / "v", dtype=np.float64)
    assert raw[0] == a["weights"][0] and np.array_equal(raw[1:].reshape(9, -1)[3], a["velocity"][3].reshape(-1))
    s2, _ = _solver("pade6_rk4_xi3_every2")
    s2.read_stats(tmp_path / "v", tmp_path / "t")
    b = s2.stats()
    assert b["weights"] == a["weights"]
    assert all(np.array_equal(x, y) for x, y in zip(a["velocity"] + a["thermo"], b["velocity"] + b["thermo"]))


def test_fp32_bulk_stats_follow_fp64():
    s64, n = _solver("penta10_lsldd_none")
    s32, _ = _solver("penta10_lsldd_none", m.FP32BULK)
    s64.step(n)
    s32.step(n)
    a, b = s64.stats(), s32.stats()
    for x, y in zip(a["velocity"][:3] + a["thermo"][::2], b["velocity"][:3] + b["thermo"][::2]):
        assert np.abs(x - y).max() <= 1e-5 * np.abs(x).max()
