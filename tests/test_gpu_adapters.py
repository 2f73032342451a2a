"""GPU tests of the drop-in boundary as a maintainer would use it: the C++
adapters of mpi_3dcompact_b200/adapters/mc3d_adapters.hpp (GpuPade6 ..
GpuCompact10Filter, GpuCurvilinearCSolver + GpuRK, GpuVremanSGS / GpuDSMSGS)
compiled against the reference's own headers into oracle/_ref/adapter_driver,
which calls them through the reference's base-class pointers
(AbstractDerivatives*, AbstractFilter*, AbstractCSolver* and AbstractRK*,
AbstractSGS*).

* Operators: each GPU object against the reference's own class on the same
  field in the same process: calc1stDerivField, calc1stDerivField_TPB with
  random ghost planes, filterField, calcNeumann. FP64, <= 1e-13 of the
  output's largest value (the compact solves round differently in the last
  bits, as the operator parity tests state).
* Solver and RK: the reference's loop (preStep, preSubStep, solveEqnSet,
  postSubStep, updateConservedData, updateData, postStep) through the base
  classes gives mc3d_solver_step's state bit for bit, and the reference
  solver's state (run live) within 1e-12 relative per conserved field.
* SGS: Vreman getSGSViscosity and DSM calcMuSGSTaukk / calcKSGS on a HIT state
  with smooth density and pressure variations, against the oracle's
  restatement of VremanSGS / DSMSGS (pinned to the reference through the
  solver fixtures): <= 1e-12 relative, k_sgs 1e-11 (well-conditioned averaging
  modes; LOCAL DSM's conditioning is covered in test_gpu_configs).
* The learned closure behind AbstractSGS (GpuMlpSGS, no counterpart in the
  reference): calcMuSGSTaukk + calcKSGS with the shipped closure against a
  numpy restatement of its features and outputs around the same network run
  by the standalone tensor-core inference (relative L2 <= 1e-2) and by the
  FP32 forward (<= 5e-2, the BF16 quantisation); tau_kk zero."""
import math
import os
import subprocess

import numpy as np
import pytest

from mpi_3dcompact_b200.hit_ic import hit_initial_condition
from oracle import mc3d_oracle as O
from oracle import ref_runner as R
from tests import helpers as H

DRIVER = os.path.join(os.path.dirname(R.REF_BIN), "adapter_driver")
pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not os.access(DRIVER, os.X_OK), reason="oracle/_ref/adapter_driver not built")]


def _drive(tmp_path, cfg, *args, steps=1):
    with open(os.path.join(tmp_path, "MPI_3DCompact.in"), "w") as f:
        f.write(R.ini_text(cfg, steps))
    r = subprocess.run([DRIVER, *args], cwd=tmp_path, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:] + r.stdout[-2000:]
    return r.stdout


@pytest.mark.parametrize("bc", [(0, 0, 0), (1, 0, 1)])
def test_operator_adapters_match_reference_classes(tmp_path, bc):
    cfg = O.Config(N=(32, 24, 20), bc=bc, alphaF=0.47)
    out = _drive(tmp_path, cfg, "ops", "7")
    rows = [ln.split() for ln in out.splitlines() if ln.startswith("op ")]
    kinds = {(r[1], r[2], r[3]) for r in rows}
    assert len(rows) == len(kinds)
    # every direction: 3 derivatives (+TPB on periodic directions, + calcNeumann) and 4 filters
    per_dir = {d: 3 * 2 + 4 + (3 if bc["xyz".index(d)] == 0 else 0) for d in "xyz"}
    for d in "xyz":
        assert sum(1 for r in rows if r[2] == d) == per_dir[d], d
    for _, name, d, kind, err in rows:
        tol = 0.0 if kind == "neumann" else 1e-13
        assert float(err) <= tol, (name, d, kind, err)
    assert any(r[3] == "tpb" for r in rows)


_SOLVER_CASES = {
    "penta10_lsldd_c8_vreman": dict(N=(24, 20, 16), fd=("PENTA10",) * 3, filter="COMPACT8", alphaF=0.45,
                                    rk="LSLDDRK4", les="VREMAN", mu_ref=0.002),
    "pade6_rk4_c10": dict(N=(20, 20, 20), fd=("PADE6",) * 3, filter="COMPACT10", alphaF=0.49, rk="RK4",
                          mu_ref=0.002),
    "pade6_kenrk4_dsm_global": dict(N=(16, 16, 16), fd=("PADE6",) * 3, filter="COMPACT10", alphaF=0.49, rk="KENRK4",
                                    les="DSM", les_avg="GLOBAL", dsm_test_filter=1, mu_ref=0.005),
    "pade6_tvdrk3_substep": dict(N=(16, 16, 16), fd=("PADE6",) * 3, filter="COMPACT8", alphaF=0.45, rk="TVDRK3",
                                 filter_step=2, substep_filtering=True, mu_ref=0.005),
}


@pytest.mark.parametrize("name", list(_SOLVER_CASES))
def test_solver_and_rk_adapters_drive_the_reference_loop(tmp_path, name):
    cfg = O.Config(**_SOLVER_CASES[name])
    n = cfg.N[0]
    ic = hit_initial_condition(n, k0=3.0, seed=4, mt=0.3)
    if cfg.N != (n, n, n):
        ic = [np.ascontiguousarray(a[:cfg.N[2], :cfg.N[1], :cfg.N[0]]) for a in ic]
    steps = 4
    with open(os.path.join(tmp_path, "ic.bin"), "wb") as f:
        for a in ic:
            f.write(np.ascontiguousarray(a, dtype=np.float64).tobytes())
    out = _drive(tmp_path, cfg, "solver", "ic.bin", "out.bin", steps=steps)
    line = [ln.split() for ln in out.splitlines() if ln.startswith("solver ")][0]
    assert int(line[2]) == steps
    assert float(line[6]) == 0.0 and line[8] == "1", line   # bit for bit mc3d_solver_step
    raw = np.fromfile(os.path.join(tmp_path, "out.bin"), dtype=np.float64)
    Nx, Ny, Nz = cfg.N
    q = raw[2:].reshape(5, Nz, Ny, Nx)
    qr, info = R.run_solver(cfg, ic, steps)
    for i in range(5):
        assert H.rel_max(q[i], qr[i]) <= 1e-12, (name, i, H.rel_max(q[i], qr[i]))
    assert abs(raw[1] - info["time"]) <= 1e-12 * info["time"]


@pytest.mark.parametrize("les,avg,tf", [("VREMAN", "NONE", 1), ("VREMAN", "LOCAL", 1), ("VREMAN", "GLOBAL", 1),
                                        ("DSM", "GLOBAL", 1), ("DSM", "XI2_AVG", 2), ("DSM", "XI1_AVG", 1)])
def test_sgs_adapters_match_oracle(tmp_path, les, avg, tf):
    n = 24
    cfg = O.Config(N=(n, n, n), fd=("PADE6",) * 3, les=les, les_avg=avg, dsm_test_filter=tf, mu_ref=0.002)
    _, U, V, W, _ = hit_initial_condition(n, k0=3.0, seed=6, mt=0.3)
    # smooth density and pressure variations, so that the temperature gradient
    # (and with it the k_sgs ratio N_i K_i / N_i N_i) is not rounding noise
    xi = 2 * math.pi * np.arange(n) / n
    z, y, x = np.meshgrid(xi, xi, xi, indexing="ij")
    rho = 1.0 + 0.05 * np.sin(x + 2 * y) * np.cos(z)
    p = (1.0 / 1.4) * (1.0 + 0.04 * np.cos(2 * x - y + z))
    o = O.Oracle(cfg, O.cube_metrics(cfg.N))
    q = [rho, rho * U, rho * V, rho * W, p / 0.4 + 0.5 * rho * (U * U + V * V + W * W)]
    T = p / (rho * (1.0 / 1.4))
    Jm = o.Jm

    def phys(dq, j):   # Core.cpp:548-561
        return Jm[0][j] * dq[0] + Jm[1][j] * dq[1] + Jm[2][j] * dq[2]
    dU, dV, dW, dT = o.grad(U), o.grad(V), o.grad(W), o.grad(T)
    gu = [[phys(d, j) for j in range(3)] for d in (dU, dV, dW)]
    gT = [phys(dT, j) for j in range(3)]
    with open(os.path.join(tmp_path, "in.bin"), "wb") as f:
        for a in [gu[a][b] for a in range(3) for b in range(3)] + q + [T] + gT:
            f.write(np.ascontiguousarray(a, dtype=np.float64).tobytes())
    _drive(tmp_path, cfg, "sgs", "in.bin", "out.bin")
    mu, tk, ks = np.fromfile(os.path.join(tmp_path, "out.bin"), dtype=np.float64).reshape(3, n, n, n)
    if les == "VREMAN":
        assert H.rel_max(mu, o.vreman(gu, q[0])) <= 1e-12
    else:
        mu_r, tk_r, ctx = o.dsm_mu_taukk(gu, q[0], q[1], q[2], q[3])
        ks_r = o.dsm_ksgs(gT, q[0], q[1], q[2], q[3], T, ctx)
        # k_sgs divides by the averaged N_i N_i: a one-ulp change of the state
        # moves it by up to 4e-13, hence its bound of 1e-11
        for name, got, ref, tol in (("mu_sgs", mu, mu_r, 1e-12), ("taukk", tk, tk_r, 1e-12),
                                    ("k_sgs", ks, ks_r, 1e-11)):
            assert np.isfinite(ref).all()
            assert H.rel_max(got, ref) <= tol, (name, H.rel_max(got, ref))


def _closure_features(gu, rho, T, gT, delta, mu):
    """The closure's nine features (csrc/mlp_common.cuh mlp_features) in
    float64 numpy, and |S|."""
    S = [[0.5 * (gu[a][b] + gu[b][a]) for b in range(3)] for a in range(3)]
    Wm = [[0.5 * (gu[a][b] - gu[b][a]) for b in range(3)] for a in range(3)]
    s2 = sum(S[a][b] ** 2 for a in range(3) for b in range(3))
    w2 = sum(Wm[a][b] ** 2 for a in range(3) for b in range(3))
    trS3 = trSW2 = trS2W2 = 0.0
    for a in range(3):
        for b in range(3):
            p = sum(S[a][k] * S[k][b] for k in range(3))
            q = sum(Wm[a][k] * Wm[k][b] for k in range(3))
            trS3 = trS3 + p * S[b][a]
            trSW2 = trSW2 + S[a][b] * q
            trS2W2 = trS2W2 + p * q
    eps, sw = 1e-30, s2 + w2
    smag = np.sqrt(2.0 * s2)
    c = np.sqrt(1.4 * (1.0 / 1.4) * T)
    gTm = np.sqrt(gT[0] ** 2 + gT[1] ** 2 + gT[2] ** 2)
    x = [np.log1p(rho * delta * delta * smag / mu), w2 / (sw + eps), trS3 / (s2 * np.sqrt(s2) + eps),
         trSW2 / (sw * np.sqrt(sw) + eps), trS2W2 / (sw * sw + eps), (gu[0][0] + gu[1][1] + gu[2][2]) / (np.sqrt(sw) + eps),
         delta * gTm / T, delta * smag / c, np.log(rho)]
    return np.stack([a.ravel() for a in x], axis=1), smag.ravel()


def test_mlp_sgs_adapter_matches_the_closure(tmp_path):
    """GpuMlpSGS through AbstractSGS* against the closure restated around the
    same network: features in float64 numpy, the network by the standalone
    tensor-core inference (mc3d_mlp_infer_bf16, the same pipeline) and by
    the FP32 forward, the outputs in numpy. Against the first the difference
    is the features' rounding (FP32 with reciprocal quotients on the GPU),
    which flips an occasional BF16 input: relative L2 <= 1e-2, max <= 5e-2
    of the largest value. Against the FP32 network the difference is the
    BF16 quantisation of this network on this state: relative L2 <= 5e-2.
    mu_ref 1e-3 keeps every feature inside the training range."""
    import torch
    import mpi_3dcompact_b200 as m
    n = 24
    mu_ref = 1e-3
    cfg = O.Config(N=(n, n, n), fd=("PADE6",) * 3, les="DSM", les_avg="GLOBAL", mu_ref=mu_ref)
    _, U, V, W, _ = hit_initial_condition(n, k0=3.0, seed=6, mt=0.3)
    xi = 2 * math.pi * np.arange(n) / n
    z, y, x = np.meshgrid(xi, xi, xi, indexing="ij")
    rho = 1.0 + 0.05 * np.sin(x + 2 * y) * np.cos(z)
    p = (1.0 / 1.4) * (1.0 + 0.04 * np.cos(2 * x - y + z))
    o = O.Oracle(cfg, O.cube_metrics(cfg.N))
    q = [rho, rho * U, rho * V, rho * W, p / 0.4 + 0.5 * rho * (U * U + V * V + W * W)]
    T = p / (rho * (1.0 / 1.4))
    Jm = o.Jm

    def phys(dq, j):
        return Jm[0][j] * dq[0] + Jm[1][j] * dq[1] + Jm[2][j] * dq[2]
    gu = [[phys(d, j) for j in range(3)] for d in (o.grad(U), o.grad(V), o.grad(W))]
    gT = [phys(o.grad(T), j) for j in range(3)]
    with open(os.path.join(tmp_path, "in.bin"), "wb") as f:
        for a in [gu[a][b] for a in range(3) for b in range(3)] + q + [T] + gT:
            f.write(np.ascontiguousarray(a, dtype=np.float64).tobytes())
    closure = os.path.join(os.path.dirname(m.__file__), "data", "mlp_sgs_hit128.bin")
    _drive(tmp_path, cfg, "sgs", "in.bin", "out.bin", closure)
    mu, tk, ks = np.fromfile(os.path.join(tmp_path, "out.bin"), dtype=np.float64).reshape(3, n, n, n)
    assert np.all(tk == 0.0)
    net = m.MLPClosure()
    net.load(closure)
    nrm = net.normalization()
    delta = 2 * math.pi / n
    feats, smag = _closure_features(gu, rho, T, gT, delta, mu_ref * T ** 0.76)
    assert ((feats >= nrm["lo"]) & (feats <= nrm["hi"])).all()
    xt = torch.tensor(feats.astype(np.float32), device="cuda")
    refs = {}
    for kind in ("bf16", "fp32"):
        yt = torch.empty((xt.shape[0], 2), dtype=torch.float32, device="cuda")
        (net.infer_bf16 if kind == "bf16" else net.forward)(xt, yt)
        torch.cuda.synchronize()
        out = yt.cpu().numpy().astype(np.float64)
        C = np.maximum(0.0, out[:, 0] * nrm["ystd"][0] + nrm["ymean"][0])
        prt = np.clip(out[:, 1] * nrm["ystd"][1] + nrm["ymean"][1], 0.1, 10.0)
        mu_r = rho.ravel() * delta * delta * smag * C
        refs[kind] = (mu_r.reshape(n, n, n), (2.5 * mu_r / prt).reshape(n, n, n))
    for i, (name, got) in enumerate((("mu_sgs", mu), ("k_sgs", ks))):
        ref, ref32 = refs["bf16"][i], refs["fp32"][i]
        assert np.abs(ref).max() > 0
        l2 = np.linalg.norm(got - ref) / np.linalg.norm(ref)
        mx = np.abs(got - ref).max() / np.abs(ref).max()
        assert l2 <= 1e-2 and mx <= 5e-2, (name, l2, mx)
        l2_32 = np.linalg.norm(got - ref32) / np.linalg.norm(ref32)
        assert l2_32 <= 5e-2, (name, l2_32)
