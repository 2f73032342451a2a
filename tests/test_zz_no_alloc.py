"""GPU test of mc3d_cfl_max_noalloc, the entry point for callers that cannot
let the library allocate device memory (they own a fixed device pool).

It is called through the C ABI on the solver's own state, twice in a row
(before the first and before the second time step), and CFL / max must equal
the dt the solver's allocating path computed for those steps, to the FP64
tolerance of the other parity tests (1e-12 relative). Collected last so a
failure here leaves every other test already run."""
import ctypes as C
import math

import numpy as np
import pytest

import mpi_3dcompact_b200 as m
from mpi_3dcompact_b200 import _native as N

pytestmark = pytest.mark.gpu


def _noalloc_max(s, q_ptrs, n, out, stream):
    lib = N.host_lib()
    rc = lib.mc3d_cfl_max_noalloc(*[C.c_void_p(p) for p in q_ptrs], None, None, None,
                                  1.0 / (2 * math.pi), 1.0 / (2 * math.pi), 1.0 / (2 * math.pi),
                                  n, n, n, 1.0 / n, 1.0 / n, 1.0 / n, C.c_void_p(out.data_ptr()), C.c_void_p(stream))
    N.check(rc)


def test_noalloc_cfl_matches_solver_dt_twice():
    import torch
    from mpi_3dcompact_b200.hit_ic import hit_initial_condition
    n, cfl = 32, 0.5
    s = m.CurvilinearCSolver(m.Options(grid=n, fd="PENTA10", filter="COMPACT8", alphaF=0.45, rk="LSLDDRK4",
                                       les="VREMAN", mu_ref=0.001, cfl=cfl, precision=m.FP64))
    s.set_box_metrics(2 * math.pi)
    s.set_initial_conditions(*hit_initial_condition(n, k0=4.0, seed=8, mt=0.3))
    stream = s.stream()
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    for call in range(2):
        s.sync()
        free_before = torch.cuda.mem_get_info()[0]
        _noalloc_max(s, s.conserved_device_ptrs(), n, out, stream)   # ordered before the step on the same stream
        s.sync()
        if call == 1:
            # after the set-up of the first call nothing more is claimed on the device
            assert torch.cuda.mem_get_info()[0] == free_before
        s.step(1)
        dt = s.info()["dt"]
        got = cfl / out.item()
        assert abs(got - dt) <= 1e-12 * dt, (got, dt)


def test_noalloc_cfl_reports_a_non_finite_state_as_nan():
    """One NaN density makes the maximum NaN (the reference's loop would skip
    that point), so a caller sees the broken state instead of a finite dt."""
    import torch
    n = 16
    q = [torch.ones(n, n, n, dtype=torch.float64, device="cuda") for _ in range(5)]
    q[4].fill_(2.5)
    q[0][3, 4, 5] = float("nan")
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    lib = N.host_lib()
    N.check(lib.mc3d_cfl_max_noalloc(*[C.c_void_p(t.data_ptr()) for t in q], None, None, None, 1.0, 1.0, 1.0,
                                     n, n, n, 1.0 / n, 1.0 / n, 1.0 / n, C.c_void_p(out.data_ptr()), None))
    torch.cuda.synchronize()
    assert math.isnan(out.item())
    q[0][3, 4, 5] = 1.0
    N.check(lib.mc3d_cfl_max_noalloc(*[C.c_void_p(t.data_ptr()) for t in q], None, None, None, 1.0, 1.0, 1.0,
                                     n, n, n, 1.0 / n, 1.0 / n, 1.0 / n, C.c_void_p(out.data_ptr()), None))
    torch.cuda.synchronize()
    assert math.isfinite(out.item()) and out.item() > 0


def test_noalloc_rejects_fields_beyond_its_limit():
    lib = N.host_lib()
    dummy = C.c_void_p(16)      # never dereferenced: the size check comes first
    rc = lib.mc3d_cfl_max_noalloc(*([dummy] * 5), None, None, None, 1.0, 1.0, 1.0, 300, 300, 300,
                                  1.0, 1.0, 1.0, dummy, None)
    assert rc == 6
    assert b"16777216" in lib.mc3d_last_error()
