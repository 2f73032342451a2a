"""CPU tests of the C ABI: the library loads, exports every function the header
declares, and its host logic (MPI_3DCompact.in reader, calcNeumann, the HIT
generator's random numbers) behaves like the reference. No device calls."""
import ctypes as C
import os
import textwrap

import numpy as np
import pytest

import mpi_3dcompact_b200 as m
from mpi_3dcompact_b200 import _native as N

HIT_IN = """
# HIT box in the layout of the reference's inputs
[RESTART]
FROMRESTART = FALSE
ONLYGRIDFROMRESTART = FALSE
SPONGEAVGFROMRESTART = FALSE

[TIMESTEPPING]
TSTYPE      = CONST_CFL
CFL         = 0.5
MAXTIME     = 10.0
MAXTIMESTEP = 200
FILTERSTEP  = 1
SUBSTEPFILTERING = FALSE
CHECKSTEP   = 1
DUMPSTEP    = 25000

[STATS]
INTERVAL = 1
VELOCITYSTATS = 0
THERMOSTATS = 0
STATSAVGTYPE = XI3_AVG

[BC]
BCXTYPE = PERIODIC_SOLVE
BCYTYPE = PERIODIC_SOLVE
BCZTYPE = PERIODIC_SOLVE
BCX0 = PERIODIC
BCX1 = PERIODIC
BCY0 = PERIODIC
BCY1 = PERIODIC
BCZ0 = PERIODIC
BCZ1 = PERIODIC
PERIODICDISPX_X = 6.2831853
PERIODICDISPX_Y = 0.0
PERIODICDISPX_Z = 0.0
PERIODICDISPY_X = 0.0
PERIODICDISPY_Y = 6.2831853
PERIODICDISPY_Z = 0.0
PERIODICDISPZ_X = 0.0
PERIODICDISPZ_Y = 0.0
PERIODICDISPZ_Z = 6.2831853

[DOMAIN]
NX = 256
NY = 256
NZ = 256

[PENCILDECOMP]
PROW = 0
PCOL = 0

[SOLVER]
RKTYPE = LSLDDRK4
ALPHAF = 0.45
MU_REF = 0.00033
USETIMING = FALSE
XFDTYPE = PENTA10
YFDTYPE = PENTA10
ZFDTYPE = PENTA10
FILTERTYPE = COMPACT8

[LES]
LESMODEL = VREMAN
LESAVERAGING = NONE

[GPU]
PRECISION = FP32BULK
"""


def test_library_exports_every_header_function():
    lib = N.host_lib()
    names = N.header_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_library_is_in_tree():
    assert os.path.dirname(N.LIB_PATH) == os.path.dirname(os.path.abspath(m.__file__))


def _write(tmp_path, text):
    p = tmp_path / "MPI_3DCompact.in"
    p.write_text(textwrap.dedent(text))
    return p


def test_ini_parses_hit_case(tmp_path):
    o = m.Options.from_ini(_write(tmp_path, HIT_IN))
    c = o.c
    assert (c.Nx, c.Ny, c.Nz) == (256, 256, 256)
    assert list(c.fd_type) == [N.PENTA10] * 3
    assert c.filter_type == N.COMPACT8 and c.alphaF == 0.45
    assert c.rk_type == N.LSLDDRK4 and c.ts_type == N.CONST_CFL and c.cfl == 0.5
    assert c.les_model == N.VREMAN and c.les_averaging == N.AVG_NONE
    assert c.mu_ref == 0.00033 and c.max_time_step == 200 and c.filter_step == 1
    assert c.precision == N.FP32BULK and c.reference_quirks == 1
    disp = [[c.periodic_disp[d][e] for e in range(3)] for d in range(3)]
    assert disp == [[6.2831853, 0.0, 0.0], [0.0, 6.2831853, 0.0], [0.0, 0.0, 6.2831853]]


def test_ini_defaults(tmp_path):
    txt = HIT_IN.replace("CFL         = 0.5\n", "").replace("ALPHAF = 0.45\n", "").replace("FILTERSTEP  = 1\n", "")
    c = m.Options.from_ini(_write(tmp_path, txt)).c
    assert c.cfl == 0.5 and c.alphaF == 0.45 and c.filter_step == 1   # Options.hpp:228,235,250


@pytest.mark.parametrize("drop,needle", [
    ("MU_REF = 0.00033\n", "mu_ref"),
    ("RKTYPE = LSLDDRK4\n", "RKTYPE"),
    ("LESMODEL = VREMAN\n", "LESMODEL"),
    ("NZ = 256\n", "NZ"),
    ("\nFROMRESTART = FALSE", "fromRestart"),
    ("PERIODICDISPY_Z = 0.0\n", "PERIODICDISPY_Z"),
])
def test_ini_required_keys(tmp_path, drop, needle):
    with pytest.raises(N.Mc3dError) as e:
        m.Options.from_ini(_write(tmp_path, HIT_IN.replace(drop, "")))
    assert e.value.code == 1 and needle in str(e.value)


def test_ini_rejects_bad_values(tmp_path):
    for a, b in [("RKTYPE = LSLDDRK4", "RKTYPE = RK5"), ("NX = 256", "NX = 10"),
                 ("BCX1 = PERIODIC", "BCX1 = ADIABATIC_WALL"), ("[LES]", "[LES]\nBOGUS = 1")]:
        with pytest.raises(N.Mc3dError):
            m.Options.from_ini(_write(tmp_path, HIT_IN.replace(a, b)))


def test_ini_mlp_closure_keys(tmp_path):
    txt = HIT_IN.replace("LESMODEL = VREMAN", "LESMODEL = MLP")
    c = m.Options.from_ini(_write(tmp_path, txt)).c
    assert c.les_model == N.MLPSGS and c.mlp_fallback_frac == 1e-3
    c = m.Options.from_ini(_write(tmp_path, txt.replace("[LES]", "[LES]\nMLPFALLBACKFRAC = 0.01"))).c
    assert c.mlp_fallback_frac == 0.01
    with pytest.raises(N.Mc3dError):
        m.Options.from_ini(_write(tmp_path, txt.replace("[LES]", "[LES]\nMLPFALLBACKFRAC = 2")))


def test_ini_stats_keys(tmp_path):
    txt = HIT_IN.replace("VELOCITYSTATS = 0", "VELOCITYSTATS = 1\nVELOCITYSTATSFROMRESTART = TRUE\n"
                         "VELOCITYSTATSFILENAME = VelocityStats.100")
    c = m.Options.from_ini(_write(tmp_path, txt)).c
    assert c.velocity_stats == 1 and c.thermo_stats == 0 and c.stats_interval == 1
    assert c.stats_avg_type == N.AVG_XI3 and c.velocity_stats_from_restart == 1
    assert c.velocity_stats_file.decode() == "VelocityStats.100"
    with pytest.raises(N.Mc3dError):   # the restart flag is required once the stats are on
        m.Options.from_ini(_write(tmp_path, HIT_IN.replace("VELOCITYSTATS = 0", "VELOCITYSTATS = 1")))


def test_ini_lesmodel_none_alias(tmp_path):
    c = m.Options.from_ini(_write(tmp_path, HIT_IN.replace("LESMODEL = VREMAN", "LESMODEL = NONE"))).c
    assert c.les_model == N.NOMODEL


def test_calc_neumann_matches_reference_formula():
    f = np.array([1.0, 1.1, 1.3, 1.6, 2.0, 2.5])
    want = (f[0] * 360 - f[1] * 450 + f[2] * 400 - f[3] * 225 + f[4] * 72 - f[5] * 10) / 147   # Pade6.cpp:395
    assert m.calc_neumann(N.PADE6, f) == want
    assert m.calc_neumann(N.PENTA10, f) == want
    assert m.calc_neumann(N.CD2, f) == (f[0] * 4 - f[1]) / 3                                   # CD2.cpp:183


def test_hit_randvec_matches_restatement():
    """The C generator (mc3d_hit_randvec) and the vectorised numpy restatement
    give the same sequence, also across consecutive calls of different sizes."""
    from mpi_3dcompact_b200.hit_ic import _Gen
    ga, gb = _Gen(7), _Gen(7)
    for n in (5000, 1, 300001, 97):
        a = ga.vec(n)
        b = N.hit_randvec(N.host_lib(), gb, n)
        assert np.array_equal(a, b), n
        assert (ga.ix1, ga.ix2, ga.ix3) == (gb.ix1, gb.ix2, gb.ix3) and ga.r == gb.r


def test_null_arguments_are_errors_not_crashes():
    lib = N.host_lib()
    assert lib.mc3d_solver_step(None, 1) == 6
    assert lib.mc3d_op_apply(None, None, None, 1, None) == 6
    assert lib.mc3d_config_from_ini(None, None) == 6
    assert b"null" in lib.mc3d_last_error()


@pytest.mark.parametrize("name", ["channel_sponge_rect_lsldd", "ogrid_cyl_sponge_kenrk4"])
def test_sponge_sigma_matches_oracle(name):
    """mc3d_sponge_sigma (host code) restates SpongeBC's sigma exactly."""
    import mpi_3dcompact_b200 as m
    from oracle import mc3d_oracle as O
    from tests.golden import gen_golden as G
    cfg, ic, n, coords = G.wall_case(name)
    opt = m.Options(grid=cfg.N, bc=cfg.bc, bc_kind=cfg.kinds(), sponge=cfg.sponge)
    got = m.sponge_sigma(opt, *coords)
    ref = O.sponge_sigma(cfg, *coords)
    assert np.array_equal(got, ref)
    assert ref.max() > 0.1
