"""CPU tests of the checkpoint formats: SolutionDump / SpongeAvgDump files the
reference itself wrote (tests/golden/checkpoint.npz, from oracle/_ref), the
library's reader and writer on them, the oracle's restart restatement against
the reference's own restart, and the [RESTART] keys of MPI_3DCompact.in."""
import textwrap

import numpy as np
import pytest

import mpi_3dcompact_b200 as m
from mpi_3dcompact_b200 import _native as N
from oracle import mc3d_oracle as O
from tests.golden import gen_golden as G


def _gold():
    return np.load(G.os.path.join(G.HERE, "checkpoint.npz"))


def _write(tmp_path, name, arr):
    p = tmp_path / name
    p.write_bytes(arr.tobytes())
    return p


@pytest.mark.parametrize("name", list(G.CHECKPOINT_CASES))
def test_reference_dump_layout(name):
    """Header, mesh and state of the reference's dump: the time step it stopped
    at, its grid, the mesh it ran on and the oracle's state after those steps."""
    cfg, ic, coords, n1, _ = G.checkpoint_case(name)
    hdr, f = O.parse_solution_dump(_gold()[f"{name}_dump"].tobytes())
    assert hdr["time_step"] == n1 and hdr["N"] == tuple(cfg.N)
    if coords is None:
        xi = [np.arange(k) / k for k in cfg.N]
        z, y, x = np.meshgrid(2 * np.pi * xi[2], 2 * np.pi * xi[1], 2 * np.pi * xi[0], indexing="ij")
        coords = (x, y, z)
    for a, b in zip(f[:3], coords):
        assert np.abs(a - b).max() <= 1e-15 * max(1.0, np.abs(b).max())
    sigma = O.sponge_sigma(cfg, *coords) if cfg.sponge else None
    met = None
    if name != "hit_pade6_rk4":
        met = O.solve_for_jacobians(cfg, *coords)
    q, st = O.run(cfg, ic, n1, metrics=met, sigma=sigma)
    for i in range(5):
        assert np.abs(f[3 + i] - q[i]).max() <= 1e-13 * np.abs(q[i]).max()
    assert abs(hdr["time"] - st.time) <= 1e-14


@pytest.mark.parametrize("name", list(G.CHECKPOINT_CASES))
def test_library_reads_and_rewrites_reference_dump(name, tmp_path):
    raw = _gold()[f"{name}_dump"]
    path = _write(tmp_path, "SolutionDump.ref", raw)
    hdr, fields = m.read_dump(path)
    ohdr, ofields = O.parse_solution_dump(raw.tobytes())
    assert hdr == ohdr
    for a, b in zip(fields, ofields):
        assert np.array_equal(a, b)
    out = tmp_path / "SolutionDump.copy"
    m.write_dump(out, hdr["time_step"], hdr["time"], fields)
    assert out.read_bytes() == path.read_bytes()


@pytest.mark.parametrize("name", list(G.CHECKPOINT_CASES))
def test_oracle_restart_matches_reference_restart(name):
    """Restart restated (mesh and state from the dump, primitives by
    solveU/solvep, the dump's time step and time) against the reference's own
    restart run: bit-level agreement up to the oracle's 1e-13 budget."""
    cfg, _, coords, n1, n2 = G.checkpoint_case(name)
    gold = _gold()
    hdr, f = O.parse_solution_dump(gold[f"{name}_dump"].tobytes())
    met = O.solve_for_jacobians(cfg, *f[:3]) if name != "hit_pade6_rk4" else None
    sigma = O.sponge_sigma(cfg, *f[:3]) if cfg.sponge else None
    q, st = O.run(cfg, O.restart_primitives(f[3:]), n2, metrics=met, sigma=sigma, time=hdr["time"],
                  time_step=hdr["time_step"])
    ts, t, dt = gold[f"{name}_restart_info"]
    assert st.time_step == int(ts) == n1 + n2
    assert abs(st.time - t) <= 1e-14 * abs(t)
    for i in range(5):
        ref = gold[f"{name}_restart_q{i}"]
        assert np.abs(q[i] - ref).max() <= 1e-13 * np.abs(ref).max(), i


def test_restart_is_not_bit_continuous_in_the_reference():
    """The reference's restart leaves time unchanged on its first step and
    restarts the filter rotation, so 3 + 2 steps differ from 5 straight ones."""
    cfg, ic, _, n1, n2 = G.checkpoint_case("hit_pade6_rk4")
    gold = _gold()
    q5, st5 = O.run(cfg, ic, n1 + n2)
    ts, t, dt = gold["hit_pade6_rk4_restart_info"]
    assert t < st5.time
    assert max(np.abs(gold[f"hit_pade6_rk4_restart_q{i}"] - q5[i]).max() for i in range(5)) > 1e-9


def test_ini_restart_keys(tmp_path):
    from tests.test_capi import HIT_IN
    raw = _gold()["hit_pade6_rk4_dump"]
    dump = _write(tmp_path, "SolutionDump.3", raw)
    txt = HIT_IN.replace("\nFROMRESTART = FALSE", f"\nFROMRESTART = TRUE\nFILENAME = {dump}")
    txt = "\n".join(line for line in txt.splitlines() if not line.startswith("N") or "=" not in line
                    or line.split("=")[0].strip() not in ("NX", "NY", "NZ"))
    p = tmp_path / "MPI_3DCompact.in"
    p.write_text(textwrap.dedent(txt))
    c = m.Options.from_ini(p).c
    assert c.from_restart == 1 and (c.Nx, c.Ny, c.Nz) == (12, 12, 12)
    assert c.restart_file.decode() == str(dump)
    assert c.dump_step == 25000
    bad = txt.replace(f"FILENAME = {dump}", f"FILENAME = {tmp_path / 'missing'}")
    p.write_text(textwrap.dedent(bad))
    with pytest.raises(N.Mc3dError):
        m.Options.from_ini(p)


def _moments(v, t):
    """Means, mean squares and mean products of the stats fields: the
    well-conditioned quantities behind RMS = sqrt(|<x^2> - <x>^2|)."""
    m = [v[0], v[1], v[2], t[0], t[2], t[4]]
    m += [v[3 + k] ** 2 + v[k] ** 2 for k in range(3)]
    m += [t[2 * k + 1] ** 2 + t[2 * k] ** 2 for k in range(3)]
    m += [v[6 + k] + v[a] * v[b] for k, (a, b) in enumerate(((0, 1), (0, 2), (1, 2)))]
    return m


def stats_errors(v, t, weights, name):
    gold = np.load(G.os.path.join(G.HERE, "stats.npz"))
    gv = [gold[f"{name}_v{k}"] for k in range(9)]
    gt = [gold[f"{name}_t{k}"] for k in range(6)]
    gw = gold[f"{name}_weights"]
    e_w = float(np.max(np.abs(np.asarray(weights) - gw) / np.abs(gw)))
    e_m = max(float(np.abs(a - b).max() / np.abs(b).max()) for a, b in zip(_moments(v, t), _moments(gv, gt)))
    return e_w, e_m


@pytest.mark.parametrize("name", list(G.STATS_CASES))
def test_oracle_stats_match_reference(name):
    """Stats::updateStatsFields restated against the reference's own stats
    files: weights and moments to 1e-13."""
    cfg, ic, n = G.stats_case(name)
    o = O.Oracle(cfg, O.cube_metrics(cfg.N))
    o.init(*ic)
    for _ in range(n):
        o.step()
    e_w, e_m = stats_errors(o.stats.v, o.stats.t, [o.stats.vw, o.stats.tw], name)
    assert e_w <= 1e-13 and e_m <= 1e-13, (e_w, e_m)


def test_oracle_stats_xi2_leaves_fields_unaveraged():
    """The reference's XI2 branch averages its scratch array, not the field."""
    runs = []
    for avg in ("XI2_AVG", "NONE"):
        c, ic, n = G.stats_case("mixed_rk4_xi2")
        c.stats = dict(avg=avg, interval=1)
        o = O.Oracle(c, O.cube_metrics(c.N))
        o.init(*ic)
        for _ in range(n):
            o.step()
        runs.append(o.stats.v + o.stats.t)
    assert all(np.array_equal(a, b) for a, b in zip(*runs))
