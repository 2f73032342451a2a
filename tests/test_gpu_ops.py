"""GPU parity of the compact operators (C ABI mc3d_op_apply through the
Pade6/Penta10/CD2/Compact8Filter/Compact10Filter and DSM test-filter
CommN5PadeTestFilter/CommN5ExpTestFilter mirrors) against fixtures made by the
reference's own operator classes.

Tolerances: FP64 max error <= 1e-13 relative to max|out| (the GPU replays the
reference elimination with precomputed factors and reciprocal pivots, so only
rounding differs); FP32 <= 3e-6 relative to max|out| (single rounding of
inputs, factors and every operation on an O(1)-conditioned banded solve).
"""
import numpy as np
import pytest

import mpi_3dcompact_b200 as m
from tests import helpers as H
from tests.golden import gen_golden as G

pytestmark = pytest.mark.gpu

TOL = {m.FP64: 1e-13, m.FP32BULK: 3e-6}


def _torch():
    import torch
    return torch


def _make(op, d, bcs, shape, prec):
    if op == "PADE6":
        return m.Pade6(shape, bcs[d], d, precision=prec)
    if op == "PENTA10":
        return m.Penta10(shape, bcs[d], d, precision=prec)
    if op == "CD2":
        return m.CD2(shape, bcs[d], d, precision=prec)
    if op == "COMPACT8":
        return m.Compact8Filter(G.OPS_ALPHA, shape, bcs, d, precision=prec)
    if op == "TESTPADE":
        return m.CommN5PadeTestFilter(shape, bcs, d, precision=prec)
    if op == "TESTEXP":
        return m.CommN5ExpTestFilter(shape, bcs, d, precision=prec)
    return m.Compact10Filter(G.OPS_ALPHA, shape, bcs, d, precision=prec)


def _is_filter(op):
    return op.startswith("COMPACT") or op.startswith("TEST")


@pytest.mark.parametrize("prec", [m.FP64, m.FP32BULK])
@pytest.mark.parametrize("bname", list(G.OPS_BCS))
@pytest.mark.parametrize("op", G.OPS)
def test_operator_matches_reference(op, bname, prec):
    torch = _torch()
    gold = H.golden_ops()
    f = G.ops_input()
    dt = torch.float64 if prec == m.FP64 else torch.float32
    x = torch.tensor(f, dtype=dt, device="cuda")
    bcs = G.OPS_BCS[bname]
    for d in range(3):
        o = _make(op, d, bcs, f.shape, prec)
        y = torch.empty_like(x)
        if _is_filter(op):
            o.filterField(x, y)
        else:
            o.calc1stDerivField(x, y)
        torch.cuda.synchronize()
        ref = gold[f"{op}_{bname}_{d}"]
        err = H.rel_max(y.double().cpu().numpy(), ref)
        assert err <= TOL[prec], (op, bname, d, err)


@pytest.mark.parametrize("prec", [m.FP64, m.FP32BULK])
def test_batched_fields_and_large_lines(prec):
    """Several fields per launch, non-multiple-of-32 batch extents and long
    lines (N = 300 > one tile row block) against the oracle."""
    torch = _torch()
    from oracle import mc3d_oracle as O
    rng = np.random.default_rng(5)
    shape = (13, 37, 300)           # (Nz, Ny, Nx)
    fields = [rng.standard_normal(shape) for _ in range(3)]
    dt = torch.float64 if prec == m.FP64 else torch.float32
    for d, n in enumerate((300, 37, 13)):
        o = m.Penta10(shape, m.PERIODIC_SOLVE, d, precision=prec)
        xs = [torch.tensor(a, dtype=dt, device="cuda") for a in fields]
        ys = [torch.empty_like(t) for t in xs]
        o.calc1stDerivFields(xs, ys)
        torch.cuda.synchronize()
        for a, y in zip(fields, ys):
            ref = O.deriv(a, d, "PENTA10", O.PERIODIC, 1.0 / n)
            assert H.rel_max(y.double().cpu().numpy(), ref) <= TOL[prec]


def test_operator_errors_are_reported():
    torch = _torch()
    with pytest.raises(m.Mc3dError):
        m.Pade6((12, 12, 10), m.PERIODIC_SOLVE, 0)        # Nx = 10 <= 10
    o = m.Pade6((12, 12, 12), m.PERIODIC_SOLVE, 0)
    x = torch.zeros((12, 12, 12), dtype=torch.float64, device="cuda")
    with pytest.raises(m.Mc3dError):
        o.calc1stDerivField(x, x)                         # in and out alias


@pytest.mark.parametrize("prec", [m.FP64, m.FP32BULK])
@pytest.mark.parametrize("bc", [m.PERIODIC_SOLVE, m.DIRICHLET_SOLVE])
@pytest.mark.parametrize("n", [64, 128, 192, 256, 512, 1024])
def test_segmented_lines_vs_oracle(n, bc, prec):
    """Lines long enough for the segmented solve (2 to 16 segments per line;
    FP32 lines of 128-256 points through the TMA-staged kernels, y and z lines
    of 512 and 1024 points through them in boxes of 256 rows, the other
    dimensions not multiples of the 32-line tile), every operator kind, every
    direction, against the oracle. FP64 lines of 1024 points do not fit the
    shared-memory tiles of the FP64 kernels (32 lines x 1024 x 8 bytes): the
    operator reports MC3D_ERR_CONFIG."""
    torch = _torch()
    from oracle import mc3d_oracle as O
    rng = np.random.default_rng(n + 7 * bc)
    dt = torch.float64 if prec == m.FP64 else torch.float32
    for d in range(3):
        shape = [12, 20, 36]
        shape[2 - d] = n                       # (Nz, Ny, Nx): direction d has n points
        shape = tuple(shape)
        f = rng.standard_normal(shape)
        x = torch.tensor(f, dtype=dt, device="cuda")
        bcs = [m.PERIODIC_SOLVE] * 3
        bcs[d] = bc
        for op in ("PADE6", "PENTA10", "COMPACT8", "COMPACT10", "TESTPADE", "TESTEXP"):
            o = _make(op, d, bcs, shape, prec)
            y = torch.empty_like(x)
            if prec == m.FP64 and n > 768:
                with pytest.raises(m.Mc3dError):
                    o.filterField(x, y) if _is_filter(op) else o.calc1stDerivField(x, y)
                continue
            if op.startswith("COMPACT"):
                o.filterField(x, y)
                ref = O.filt(f, d, op, G.OPS_ALPHA, tuple(bcs))
            elif op.startswith("TEST"):
                o.filterField(x, y)
                ref = O.test_filter(f, d, 1 if op == "TESTPADE" else 2, tuple(bcs))
            else:
                o.calc1stDerivField(x, y)
                dh = 1.0 / n if bc == m.PERIODIC_SOLVE else 1.0 / (n - 1.0)
                ref = O.deriv(f, d, op, bc, dh)
            torch.cuda.synchronize()
            err = H.rel_max(y.double().cpu().numpy(), ref)
            assert err <= TOL[prec], (op, n, d, bc, err)


@pytest.mark.parametrize("prec,n", [(m.FP64, 64), (m.FP32BULK, 64), (m.FP32BULK, 128)])
def test_register_kernel_pass_through_lines(prec, n):
    """Filter lines on the faces of the other (Dirichlet) directions pass
    through unchanged (Compact10Filter::filterField) in the register-resident
    kernels (64-point lines) and the TMA-staged ones (128-point FP32 lines), in
    every direction, against the oracle."""
    torch = _torch()
    from oracle import mc3d_oracle as O
    rng = np.random.default_rng(11)
    dt = torch.float64 if prec == m.FP64 else torch.float32
    shape = (n, n, n)
    f = rng.standard_normal(shape)
    x = torch.tensor(f, dtype=dt, device="cuda")
    for d in range(3):
        bcs = [m.DIRICHLET_SOLVE] * 3
        bcs[d] = m.PERIODIC_SOLVE
        for op in ("COMPACT8", "COMPACT10", "TESTPADE"):
            o = _make(op, d, bcs, shape, prec)
            y = torch.empty_like(x)
            o.filterField(x, y)
            if op == "TESTPADE":
                ref = O.test_filter(f, d, 1, tuple(bcs))
            else:
                ref = O.filt(f, d, op, G.OPS_ALPHA, tuple(bcs))
            torch.cuda.synchronize()
            out = y.double().cpu().numpy()
            err = H.rel_max(out, ref)
            assert err <= TOL[prec], (op, d, err)
            # the face lines are the input, bit for bit
            face = [slice(None)] * 3
            face[2 - (d + 1) % 3] = 0
            assert np.array_equal(out[tuple(face)], x.double().cpu().numpy()[tuple(face)]), (op, d)


def test_tma_line_solves_complete_their_waits():
    """The TMA-staged FP32 line solves (256-point lines: persistent x and y/z
    kernels) finish without a bounded wait giving up, and agree with the
    FP64 solve of the same field."""
    torch = _torch()
    rng = np.random.default_rng(5)
    shape = (256, 64, 256)
    f = rng.standard_normal(shape)
    x32 = torch.tensor(f, dtype=torch.float32, device="cuda")
    x64 = torch.tensor(f, dtype=torch.float64, device="cuda")
    bcs = [m.PERIODIC_SOLVE] * 3
    for d in (0, 2):
        for op in ("PENTA10", "COMPACT8"):
            y32, y64 = torch.empty_like(x32), torch.empty_like(x64)
            o32, o64 = _make(op, d, bcs, shape, m.FP32BULK), _make(op, d, bcs, shape, m.FP64)
            if op.startswith("COMPACT"):
                o32.filterField(x32, y32)
                o64.filterField(x64, y64)
            else:
                o32.calc1stDerivField(x32, y32)
                o64.calc1stDerivField(x64, y64)
            torch.cuda.synchronize()
            err = H.rel_max(y32.double().cpu().numpy(), y64.cpu().numpy())
            assert err <= TOL[m.FP32BULK], (op, d, err)
    assert m.tma_wait_timeouts(0) == 0
