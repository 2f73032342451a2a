"""GPU tests of the metric computation (mc3d_solver_set_mesh): the device
restatement of AbstractSingleBlockMesh::solveForJacobians against the
reference's own metrics of the same meshes (tests/golden/metrics.npz, made by
oracle/_ref), and a time step on GPU-computed metrics against one on the
reference's metrics.

Compared quantities are the ones the reference forms before its final
division, the determinant 1/J and the cofactors J_ij / J: J itself is 1/det,
whose relative error grows without bound where a mesh folds (det -> 0, as in
the CD2 and unset-translation fixtures), and several cofactors vanish on the
O-grid. Tolerance: 1e-11 of the largest determinant / cofactor magnitude. Both
are differences of derivatives much larger than themselves (the cofactors of
d(X W)/dxi pairs, the determinant of d(x J_i)/dxi_i whose x Sigma_i dJ_i/dxi_i
parts cancel), so the line solves' FP64 rounding (a few 1e-16 of those
derivatives) grows by one to two digits; the smooth periodic meshes stay near
1e-12, the folded Dirichlet mesh with the wide PENTA10 closures reaches ~7e-12."""
import math

import numpy as np
import pytest

import mpi_3dcompact_b200 as m
from oracle import mc3d_oracle as O
from tests import helpers as H
from tests.golden import gen_golden as G

pytestmark = pytest.mark.gpu


def _opts(cfg: O.Config, precision=m.FP64, reference_quirks=True):
    return m.Options(grid=cfg.N, fd=cfg.fd, filter=cfg.filter, alphaF=cfg.alphaF, mu_ref=cfg.mu_ref, rk=cfg.rk,
                     cfl=cfg.cfl, precision=precision, bc=cfg.bc, bc_kind=cfg.kinds(),
                     periodic_disp=O.periodic_disp_table(cfg), reference_quirks=reference_quirks)


@pytest.mark.parametrize("precision", [m.FP64, m.FP32BULK])
@pytest.mark.parametrize("name", list(G.METRIC_CASES))
def test_device_metrics_match_reference(name, precision):
    cfg, coords = G.metric_case(name)
    s = m.CurvilinearCSolver(_opts(cfg, precision))
    s.set_mesh(*coords)
    got = s.metrics()
    gold = H.golden_metrics()
    ref = [gold[f"{name}_met{c}"] for c in range(10)]
    e_det, e_cof = _errors(got, ref)
    print(f"metrics {name} precision={precision}: det {e_det:.2e} cofactors {e_cof:.2e}")
    assert e_det <= 1e-11 and e_cof <= 1e-11, (name, e_det, e_cof)


def _errors(got, ref):
    """Largest determinant and cofactor differences, each relative to the
    largest magnitude of its kind."""
    det_g, det_r = 1.0 / got[0], 1.0 / ref[0]
    e_det = np.abs(det_g - det_r).max() / np.abs(det_r).max()
    cof_g = [got[c] * det_g for c in range(1, 10)]
    cof_r = [ref[c] * det_r for c in range(1, 10)]
    scale = max(np.abs(a).max() for a in cof_r)
    e_cof = max(np.abs(a - b).max() for a, b in zip(cof_g, cof_r)) / scale
    return e_det, e_cof


def test_device_metrics_without_quirks_differ_only_where_the_quirks_act():
    cfg, coords = G.metric_case("wavy_penta10")
    s = m.CurvilinearCSolver(_opts(cfg, reference_quirks=False))
    s.set_mesh(*coords)
    got = s.metrics()
    want = O.solve_for_jacobians(cfg, *coords, quirks=False)
    e_det, e_cof = _errors(got, want)
    assert e_det <= 1e-11 and e_cof <= 1e-11
    gold = H.golden_metrics()
    assert max(H.rel_max(got[c], gold[f"wavy_penta10_met{c}"]) for c in range(10)) > 1e-6


def test_box_mesh_gives_constant_metrics():
    cfg = O.Config(N=(16, 12, 14))
    xi = [np.arange(n) / n for n in cfg.N]
    z, y, x = np.meshgrid(2 * math.pi * xi[2], 2 * math.pi * xi[1], 2 * math.pi * xi[0], indexing="ij")
    s = m.CurvilinearCSolver(_opts(cfg))
    s.set_mesh(x, y, z)
    for a, b in zip(s.metrics(), O.cube_metrics(cfg.N)):
        assert np.abs(a - b).max() < 1e-13


def test_step_on_device_metrics_matches_step_on_reference_metrics():
    """O-grid wall case run on metrics from set_mesh and on the reference's
    metrics: the same state after its steps."""
    name = "ogrid_cyl_sponge_kenrk4"
    cfg, ic, n, coords = G.wall_case(name)
    gold = H.golden_steps()
    met = [gold[f"{name}_met{c}"] for c in range(10)]
    opt = m.Options(grid=cfg.N, fd=cfg.fd, filter=cfg.filter, alphaF=cfg.alphaF, mu_ref=cfg.mu_ref, rk=cfg.rk,
                    cfl=cfg.cfl, les=cfg.les, les_avg=cfg.les_avg, precision=m.FP64, bc=cfg.bc, bc_kind=cfg.kinds(),
                    sponge=cfg.sponge, periodic_disp=O.periodic_disp_table(cfg))
    sig = m.sponge_sigma(opt, *coords) if cfg.sponge else None
    out = []
    for use_mesh in (True, False):
        s = m.CurvilinearCSolver(opt)
        if use_mesh:
            s.set_mesh(*coords)
        else:
            s.set_metrics(met)
        if sig is not None:
            s.set_sponge(sig)
        s.set_initial_conditions(*ic)
        s.step(n)
        out.append(s.conserved())
    for i in range(5):
        assert H.rel_max(out[0][i], out[1][i]) <= 1e-11, i
