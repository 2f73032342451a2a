"""mpi_3dcompact_b200: the CurvilinearCSolver time step of emathew1/MPI_3DCompact
on one NVIDIA B200, behind the reference's operator interfaces.

Host-side mirror of the reference classes over the C ABI (include/mc3d.h):

  reference (emathew1/MPI_3DCompact)          here
  ------------------------------------------  ------------------------------------
  AbstractDerivatives / Pade6 / Penta10 / CD2  Pade6, Penta10, CD2 (.calc1stDerivField)
  AbstractFilter / Compact8Filter / ...10      Compact8Filter, Compact10Filter (.filterField)
  Options (MPI_3DCompact.in)                   Options.from_ini / Options(...)
  CurvilinearCSolver + AbstractRK              CurvilinearCSolver (.step)
  AbstractCSolver::calcNeumann                 calc_neumann

Fields are CUDA torch tensors (or any object with .data_ptr()) shaped
(Nz, Ny, Nx) = x-fastest, float64 for FP64 and float32 for FP32BULK operators.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import _native as N
from ._native import (AVG_LOCAL, AVG_NONE, CD2 as _CD2, COMPACT8, COMPACT10, CONST_CFL, CONST_DT, DIRICHLET_SOLVE,
                      FP32BULK, FP64, KENRK4, LSLDDRK4, Mc3dError, NOMODEL, PADE6 as _PADE6, PENTA10 as _PENTA10,
                      PERIODIC_SOLVE, RK4, TVDRK3, VREMAN)

DIRX, DIRY, DIRZ = 0, 1, 2

__all__ = ["Pade6", "Penta10", "CD2", "Compact8Filter", "Compact10Filter", "Options", "CurvilinearCSolver",
           "calc_neumann", "Mc3dError", "DIRX", "DIRY", "DIRZ", "FP64", "FP32BULK", "PERIODIC_SOLVE",
           "DIRICHLET_SOLVE"]


def _ptr(t):
    return C.c_void_p(t.data_ptr())


class _Operator:
    """Shared apply() of the derivative and filter operators."""

    _h = None

    def _apply(self, ins, outs, stream=None):
        if len(ins) != len(outs):
            raise ValueError("in/out field counts differ")
        n = len(ins)
        for t in list(ins) + list(outs):
            if tuple(t.shape) != self.shape:
                raise ValueError(f"field shape {tuple(t.shape)} != {self.shape}")
            if not t.is_contiguous():
                raise ValueError("fields must be contiguous")
        a = (C.c_void_p * n)(*[t.data_ptr() for t in ins])
        b = (C.c_void_p * n)(*[t.data_ptr() for t in outs])
        st = C.c_void_p(stream) if stream is not None else None
        N.check(N.host_lib().mc3d_op_apply(self._h, a, b, n, st))

    def __del__(self):
        if self._h:
            try:
                N.host_lib().mc3d_op_destroy(self._h)
            except Exception:
                pass
            self._h = None


class _Derivative(_Operator):
    _fd = None

    def __init__(self, shape, bc_type, direction, dh=None, precision=FP64, device=0):
        """`shape` = (Nz, Ny, Nx). `dh` defaults to the unit-domain spacing of
        Domain (1/N periodic, 1/(N-1) Dirichlet; src/Domain.hpp:45-79)."""
        self.shape = tuple(shape)
        nz, ny, nx = self.shape
        n = (nx, ny, nz)[direction]
        if dh is None:
            dh = 1.0 / n if bc_type == PERIODIC_SOLVE else 1.0 / (n - 1.0)
        self.direction, self.bc_type, self.dh, self.precision = direction, bc_type, dh, precision
        h = C.c_void_p()
        N.check(N.host_lib().mc3d_deriv_create(self._fd, bc_type, direction, nx, ny, nz, dh, precision, device,
                                               C.byref(h)))
        self._h = h

    def calc1stDerivField(self, dataIn, dataOut, stream=None):
        """AbstractDerivatives::calc1stDerivField (src/AbstractDerivatives.hpp:45)."""
        self._apply([dataIn], [dataOut], stream)

    def calc1stDerivFields(self, ins, outs, stream=None):
        """Batched form: one launch for several fields."""
        self._apply(ins, outs, stream)

    def calc1stDerivField_TPB(self, dataIn, dataOut, *ghosts, stream=None):
        """AbstractDerivatives::calc1stDerivField_TPB (src/AbstractDerivatives.hpp:45,
        :47): ghost planes Nm2, Nm1, Np1, Np2 (Pade6, CD2) or Nm3 .. Np3
        (Penta10), each shaped like the field without its `direction` axis."""
        w = C.c_int()
        N.check(N.host_lib().mc3d_op_tpb_ghosts(self._h, C.byref(w)))
        if len(ghosts) != 2 * w.value:
            raise ValueError(f"{type(self).__name__} takes {2 * w.value} ghost planes")
        for t in [dataIn, dataOut]:
            if tuple(t.shape) != self.shape or not t.is_contiguous():
                raise ValueError("fields must be contiguous and of the operator's shape")
        pshape = tuple(n for a, n in enumerate(self.shape) if a != 2 - self.direction)
        for gpl in ghosts:
            if tuple(gpl.shape) != pshape or not gpl.is_contiguous():
                raise ValueError(f"ghost planes must be contiguous of shape {pshape}")
        a = (C.c_void_p * 1)(dataIn.data_ptr())
        b = (C.c_void_p * 1)(dataOut.data_ptr())
        g = (C.c_void_p * len(ghosts))(*[t.data_ptr() for t in ghosts])
        st = C.c_void_p(stream) if stream is not None else None
        N.check(N.host_lib().mc3d_op_apply_tpb(self._h, a, b, 1, g, st))

    def calcNeumann(self, f):
        return calc_neumann(self._fd, f)


class Pade6(_Derivative):
    """Sixth-order tridiagonal compact first derivative (src/Pade6.hpp)."""
    _fd = _PADE6


class Penta10(_Derivative):
    """Tenth-order pentadiagonal compact first derivative (src/Penta10.hpp)."""
    _fd = _PENTA10


class CD2(_Derivative):
    """Explicit two-point difference exactly as src/CD2.cpp computes it."""
    _fd = _CD2


class _Filter(_Operator):
    _ft = None

    def __init__(self, alphaF, shape, bc_types, direction, precision=FP64, device=0):
        self.shape = tuple(shape)
        nz, ny, nx = self.shape
        self.alphaF, self.direction, self.precision = alphaF, direction, precision
        bcs = (C.c_int * 3)(*bc_types)
        h = C.c_void_p()
        N.check(N.host_lib().mc3d_filter_create(self._ft, alphaF, direction, bcs, nx, ny, nz, precision, device,
                                                C.byref(h)))
        self._h = h

    def filterField(self, dataIn, dataOut, stream=None):
        """AbstractFilter::filterField (src/AbstractFilter.hpp:33)."""
        self._apply([dataIn], [dataOut], stream)

    def filterFields(self, ins, outs, stream=None):
        self._apply(ins, outs, stream)


class Compact8Filter(_Filter):
    """Eighth-order tridiagonal compact filter (src/Compact8Filter.hpp)."""
    _ft = COMPACT8


class Compact10Filter(_Filter):
    """Tenth-order tridiagonal compact filter (src/Compact10Filter.hpp)."""
    _ft = COMPACT10


class CommN5PadeTestFilter(_Filter):
    """DSM Pade test filter (src/CommN5PadeTestFilter.hpp): 11-point RHS,
    pentadiagonal LHS. Constructed as (shape, bc_types, direction)."""
    _ft = 2

    def __init__(self, shape, bc_types, direction, precision=FP64, device=0):
        super().__init__(0.0, shape, bc_types, direction, precision, device)


class CommN5ExpTestFilter(_Filter):
    """DSM explicit 7-point test filter (src/CommN5ExpTestFilter.hpp)."""
    _ft = 3

    def __init__(self, shape, bc_types, direction, precision=FP64, device=0):
        super().__init__(0.0, shape, bc_types, direction, precision, device)


def calc_neumann(fd_type, f):
    a = np.ascontiguousarray(np.asarray(f, dtype=np.float64))
    return N.host_lib().mc3d_calc_neumann(fd_type, N.dptr(a))


_FD = {"CD2": _CD2, "PADE6": _PADE6, "PENTA10": _PENTA10}
_FILT = {"COMPACT8": COMPACT8, "COMPACT10": COMPACT10}
_RK = {"TVDRK3": TVDRK3, "RK4": RK4, "KENRK4": KENRK4, "LSLDDRK4": LSLDDRK4}
_LES = {"NOMODEL": NOMODEL, "NONE": NOMODEL, "VREMAN": VREMAN, "DSM": 2, "MLP": 3}
_AVG = {"NONE": 0, "XI1_AVG": 1, "XI2_AVG": 2, "XI3_AVG": 3, "LOCAL": 4, "GLOBAL": 5}
_BCKIND = {"PERIODIC": 0, "INTERNALLY_PERIODIC": 1, "SPONGE": 2, "ADIABATIC_WALL": 3, "CONST_T_WALL": 4,
           "MOVING_ADIABATIC_WALL": 5, "INLET": 6}


def read_dump(path):
    """A SolutionDump file: (header dict, [x, y, z, rho, rhoU, rhoV, rhoW,
    rhoE]) with arrays shaped (Nz, Ny, Nx)."""
    ts, t, nx, ny, nz = C.c_int(), C.c_double(), C.c_int(), C.c_int(), C.c_int()
    lib = N.host_lib()
    N.check(lib.mc3d_dump_read_header(str(path).encode(), C.byref(ts), C.byref(t), C.byref(nx), C.byref(ny),
                                      C.byref(nz)))
    shape = (nz.value, ny.value, nx.value)
    out = [np.empty(shape) for _ in range(8)]
    p = (C.POINTER(C.c_double) * 8)(*[N.dptr(a) for a in out])
    N.check(lib.mc3d_dump_read_fields(str(path).encode(), nx.value * ny.value * nz.value, p))
    return {"time_step": ts.value, "time": t.value, "N": (nx.value, ny.value, nz.value)}, out


def write_dump(path, time_step, time, fields):
    """Write a SolutionDump file from 8 arrays (x, y, z, rho, rhoU, rhoV, rhoW,
    rhoE) shaped (Nz, Ny, Nx)."""
    arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in fields]
    nz, ny, nx = arrs[0].shape
    p = (C.POINTER(C.c_double) * 8)(*[N.dptr(a) for a in arrs])
    N.check(N.host_lib().mc3d_dump_write(str(path).encode(), int(time_step), float(time), nx, ny, nz, p))


def tma_wait_timeouts(device=0):
    """Line-solve CTAs on `device` whose TMA tile load gave up waiting (0 in a
    healthy run)."""
    n = C.c_int()
    N.check(N.host_lib().mc3d_tma_wait_timeouts(int(device), C.byref(n)))
    return n.value


def append_turbdata_line(path, values):
    """Append one turbdata.out line: the values as the HIT driver's ofstream
    with precision 17 prints them, each followed by a space
    (tests/hit/Samtaney_D4/MPI_3DCompact.cpp:545-555)."""
    with open(path, "a") as f:
        f.write("".join(f"{float(v):.17g} " for v in values) + "\n")


def append_record(path, time, values):
    """Append time and the values as raw doubles (the cylinder driver's
    cylinder{P,U,V,W}.dat and VWakeStrip.dat records, src/MPI_3DCompact.cpp:463-483, :518-524)."""
    with open(path, "ab") as f:
        f.write(np.float64(time).tobytes())
        f.write(np.ascontiguousarray(values, dtype=np.float64).tobytes())


def sponge_sigma(opt, x, y, z):
    """SpongeBC sigma (src/SpongeBC.cpp:65-360) from mesh coordinates (host arrays)."""
    arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (x, y, z)]
    out = np.empty(arrs[0].shape)
    N.check(N.host_lib().mc3d_sponge_sigma(C.byref(opt.c), *[N.dptr(a) for a in arrs], N.dptr(out)))
    return out


class Options:
    """The MPI_3DCompact.in options of the time step (src/Options.hpp)."""

    def __init__(self, grid=(64, 64, 64), fd="PADE6", filter="COMPACT10", alphaF=0.45, mu_ref=1e-3, rk="RK4",
                 ts_type="CONST_CFL", cfl=0.5, dt=-1.0, filter_step=1, substep_filtering=False, les="NOMODEL",
                 les_avg="NONE", precision=FP64, reference_quirks=True, bc=(PERIODIC_SOLVE,) * 3,
                 dsm_test_filter=1, dsm_use_taukk=True, bc_kind=None, sponge=None, mlp_fallback_frac=1e-3,
                 periodic_disp=None, max_time_step=None, max_time=None, dump_step=None, stats=None,
                 sponge_relax=None, storage="FULL", lean_slab=0):
        c = N.Config()
        N.check(N.host_lib().mc3d_config_default(C.byref(c)))
        c.Nx, c.Ny, c.Nz = grid if isinstance(grid, (tuple, list)) else (grid, grid, grid)
        fds = fd if isinstance(fd, (tuple, list)) else (fd, fd, fd)
        for d in range(3):
            c.fd_type[d] = _FD[fds[d]]
            c.bc_type[d] = bc[d]
        c.filter_type = _FILT[filter]
        c.alphaF, c.mu_ref = alphaF, mu_ref
        c.rk_type = _RK[rk]
        c.ts_type = CONST_CFL if ts_type == "CONST_CFL" else CONST_DT
        c.cfl, c.dt = cfl, dt
        c.filter_step = filter_step
        c.substep_filtering = int(bool(substep_filtering))
        c.les_model = _LES[les]
        c.les_averaging = _AVG[les_avg]
        c.precision = precision
        c.reference_quirks = int(bool(reference_quirks))
        c.dsm_test_filter = int(dsm_test_filter)
        c.dsm_use_taukk = int(bool(dsm_use_taukk))
        c.mlp_fallback_frac = mlp_fallback_frac
        c.lean_storage = {"FULL": 0, "LEAN": 1}[storage]
        c.lean_slab = int(lean_slab)
        if max_time_step is not None:
            c.max_time_step = int(max_time_step)
        if max_time is not None:
            c.max_time = float(max_time)
        if dump_step is not None:
            c.dump_step = int(dump_step)
        if stats:   # {"velocity": bool, "thermo": bool, "avg": "NONE"|"XI1_AVG"|..., "interval": int}
            c.velocity_stats = int(bool(stats.get("velocity", True)))
            c.thermo_stats = int(bool(stats.get("thermo", True)))
            c.stats_avg_type = _AVG[stats.get("avg", "NONE")]
            c.stats_interval = int(stats.get("interval", 5))
        # BC.PERIODICDISP{X,Y,Z}_{X,Y,Z} (row = face pair, column = component)
        for d in range(3):
            for e in range(3):
                c.periodic_disp[d][e] = 0.0 if periodic_disp is None else float(periodic_disp[d][e])
        # BC kinds of the faces X0, X1, Y0, Y1, Z0, Z1 (names of src/Options.hpp:21-27);
        # default: PERIODIC on periodic directions, ADIABATIC_WALL otherwise
        kinds = bc_kind or [("PERIODIC" if bc[f // 2] == PERIODIC_SOLVE else "ADIABATIC_WALL") for f in range(6)]
        for f in range(6):
            c.bc_kind[f] = _BCKIND[kinds[f]]
        if sponge:   # {"kind": "RECTILINEAR"|"CYLINDRICAL", "strength", "rect_perc"[6], "cyl_axis"[3], "rmin", "orient"}
            c.sponge_kind = 0 if sponge.get("kind", "RECTILINEAR") == "RECTILINEAR" else 1
            c.sponge_strength = sponge.get("strength", 1.0)
            for f, v in enumerate(sponge.get("rect_perc", [0.0] * 6)):
                c.sponge_rect_perc[f] = v
            c.sponge_cyl_orient = sponge.get("orient", 2)
            for d, v in enumerate(sponge.get("cyl_axis", [0.0] * 3)):
                c.sponge_cyl_axis[d] = v
            c.sponge_rmin = sponge.get("rmin", 0.0)
        if sponge_relax:   # {"avg_time": float, "p_inf": float}: updateSponge after every step
            c.sponge_relax = 1
            c.sponge_avg_time = float(sponge_relax.get("avg_time", 1.0))
            c.sponge_p_inf = float(sponge_relax.get("p_inf", 1.0 / 1.4))
        self.c = c

    @classmethod
    def from_ini(cls, path):
        """Options(mpiRank) reading MPI_3DCompact.in (src/Options.hpp:121-428)."""
        o = cls.__new__(cls)
        o.c = N.Config()
        N.check(N.host_lib().mc3d_config_from_ini(str(path).encode(), C.byref(o.c)))
        return o

    @property
    def shape(self):
        return (self.c.Nz, self.c.Ny, self.c.Nx)


def _fp(a):
    return C.cast(C.c_void_p(a.data_ptr()), C.c_void_p)


class MLPClosure:
    """Learned SGS closure (no counterpart in the reference): a 9-64-64-64-2
    GELU MLP from velocity-gradient invariants and the grid scale to C and
    Pr_t, with FP32 training kernels and BF16 tensor-core inference. Arrays
    are CUDA float32 torch tensors: x [n, 9] raw features, y [n, 2]."""

    N_PARAMS = 9090

    def __init__(self, seed=0, device=0):
        h = C.c_void_p()
        N.check(N.host_lib().mc3d_mlp_create(int(seed), device, C.byref(h)))
        self._h = h

    def __del__(self):
        if getattr(self, "_h", None):
            try:
                N.host_lib().mc3d_mlp_destroy(self._h)
            except Exception:
                pass
            self._h = None

    def set_normalization(self, mean, std, lo, hi, ymean, ystd):
        arrs = [np.ascontiguousarray(a, dtype=np.float32) for a in (mean, std, lo, hi, ymean, ystd)]
        ptrs = [a.ctypes.data_as(C.POINTER(C.c_float)) for a in arrs]
        N.check(N.host_lib().mc3d_mlp_set_normalization(self._h, *ptrs))

    def normalization(self):
        out = np.zeros(4 * 9 + 4, dtype=np.float32)
        N.check(N.host_lib().mc3d_mlp_get_normalization(self._h, out.ctypes.data_as(C.POINTER(C.c_float))))
        return dict(mean=out[0:9], std=out[9:18], lo=out[18:27], hi=out[27:36], ymean=out[36:38], ystd=out[38:40])

    def train_step(self, x, y, lr=1e-3, stream=None):
        """One Adam step on the MSE against normalised targets y; returns the loss."""
        loss = C.c_double()
        N.check(N.host_lib().mc3d_mlp_train_step(self._h, _fp(x), _fp(y), x.shape[0], lr, C.byref(loss), stream))
        return loss.value

    def gradient(self, x, y, stream=None):
        """d loss / dP of the MSE against normalised targets y (the gradient
        train_step would use), without updating; returns (G, loss)."""
        G = np.zeros(self.N_PARAMS, dtype=np.float32)
        loss = C.c_double()
        N.check(N.host_lib().mc3d_mlp_gradient(self._h, _fp(x), _fp(y), x.shape[0],
                                               G.ctypes.data_as(C.POINTER(C.c_float)), C.byref(loss), stream))
        return G, loss.value

    def forward(self, x, y, stream=None):
        N.check(N.host_lib().mc3d_mlp_forward(self._h, _fp(x), _fp(y), x.shape[0], stream))

    def infer_bf16(self, x, y, stream=None):
        N.check(N.host_lib().mc3d_mlp_infer_bf16(self._h, _fp(x), _fp(y), x.shape[0], stream))

    def params(self):
        P = np.zeros(self.N_PARAMS, dtype=np.float32)
        N.check(N.host_lib().mc3d_mlp_get_params(self._h, P.ctypes.data_as(C.POINTER(C.c_float))))
        return P

    def set_params(self, P):
        P = np.ascontiguousarray(P, dtype=np.float32)
        N.check(N.host_lib().mc3d_mlp_set_params(self._h, P.ctypes.data_as(C.POINTER(C.c_float))))

    def save(self, path):
        N.check(N.host_lib().mc3d_mlp_save(self._h, str(path).encode()))

    def load(self, path):
        N.check(N.host_lib().mc3d_mlp_load(self._h, str(path).encode()))


class CurvilinearCSolver:
    """CurvilinearCSolver + its AbstractRK driver on one GPU
    (src/CurvilinearCSolver.hpp:25-379, src/AbstractRK.hpp:6-17)."""

    def __init__(self, opt: Options, device=0):
        self.opt = opt
        h = C.c_void_p()
        N.check(N.host_lib().mc3d_solver_create(C.byref(opt.c), device, C.byref(h)))
        self._h = h
        self.shape = opt.shape

    def __del__(self):
        if getattr(self, "_h", None):
            try:
                N.host_lib().mc3d_solver_destroy(self._h)
            except Exception:
                pass
            self._h = None

    def set_box_metrics(self, L=2.0 * np.pi, Ly=None, Lz=None):
        N.check(N.host_lib().mc3d_solver_set_box_metrics(self._h, L, Ly or L, Lz or L))

    def set_metrics(self, metrics):
        """J, J11..J33 (10 float64 arrays shaped (Nz, Ny, Nx))."""
        arrs = [np.ascontiguousarray(m, dtype=np.float64) for m in metrics]
        self._met_keep = arrs
        p = (C.POINTER(C.c_double) * 10)(*[N.dptr(a) for a in arrs])
        N.check(N.host_lib().mc3d_solver_set_metrics(self._h, p))

    def set_mesh(self, x, y, z):
        """Metrics from the mesh coordinates (3 float64 arrays shaped (Nz, Ny,
        Nx)), computed on the GPU as AbstractSingleBlockMesh::solveForJacobians
        does (src/AbstractSingleBlockMesh.cpp:23-1308)."""
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (x, y, z)]
        for a in arrs:
            if a.shape != self.shape:
                raise ValueError(f"mesh arrays must be shaped {self.shape}")
        N.check(N.host_lib().mc3d_solver_set_mesh(self._h, *[N.dptr(a) for a in arrs]))

    def dump(self, path=None, mesh=None):
        """Write the state as the reference's SolutionDump file (path None:
        SolutionDump.<time step> in the working directory); mesh (x, y, z)
        None: the solver's own mesh or box."""
        if mesh is None:
            N.check(N.host_lib().mc3d_solver_dump(self._h, None if path is None else str(path).encode(),
                                                  None, None, None))
            return
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in mesh]
        N.check(N.host_lib().mc3d_solver_dump(self._h, None if path is None else str(path).encode(),
                                              *[N.dptr(a) for a in arrs]))

    def restart(self, path, grid_only=False):
        """Restart from a SolutionDump file (src/MPI_3DCompact.cpp:80-271)."""
        N.check(N.host_lib().mc3d_solver_restart(self._h, str(path).encode(), int(bool(grid_only))))

    def dump_sponge_avg(self, path=None):
        N.check(N.host_lib().mc3d_solver_dump_sponge_avg(self._h, None if path is None else str(path).encode()))

    def read_sponge_avg(self, path):
        N.check(N.host_lib().mc3d_solver_read_sponge_avg(self._h, str(path).encode()))

    def start(self):
        """Apply the configuration's [RESTART] files (mc3d_solver_start)."""
        N.check(N.host_lib().mc3d_solver_start(self._h))

    def run(self, directory=None):
        """Step until MAXTIMESTEP / MAXTIME / a killsolver file, dumping every
        DUMPSTEP steps and at the end (mc3d_solver_run)."""
        N.check(N.host_lib().mc3d_solver_run(self._h, None if directory is None else str(directory).encode()))

    def stats(self):
        """Running statistics (Stats): {"velocity": [UAVG, VAVG, WAVG, URMS, VRMS,
        WRMS, UVREY, UWREY, VWREY] or None, "thermo": [RHOAVG, RHORMS, PAVG, PRMS,
        TAVG, TRMS] or None, "weights": (velocity, thermo)}."""
        c = self.opt.c
        v = [np.empty(self.shape) for _ in range(9)] if c.velocity_stats else None
        t = [np.empty(self.shape) for _ in range(6)] if c.thermo_stats else None
        pv = (C.POINTER(C.c_double) * 9)(*[N.dptr(a) for a in v]) if v else None
        pt = (C.POINTER(C.c_double) * 6)(*[N.dptr(a) for a in t]) if t else None
        w = (C.c_double * 2)()
        N.check(N.host_lib().mc3d_solver_get_stats(self._h, pv, pt, w))
        return {"velocity": v, "thermo": t, "weights": (w[0], w[1])}

    def turbdata(self, k0=8.0):
        """One turbdata.out line of the HIT driver for the current state: time,
        tau, Re_lambda, Mt, dissipation, u', Kolmogorov length, rho', dil',
        vorticity', mean rho|u|^2."""
        out = (C.c_double * 11)()
        N.check(N.host_lib().mc3d_solver_turbdata(self._h, float(k0), out))
        return list(out)

    def wall_span_average(self):
        """p, U, V, W on the j = 0 face averaged over xi3 (Nx values each)."""
        out = [np.empty(self.shape[2]) for _ in range(4)]
        N.check(N.host_lib().mc3d_solver_wall_span_average(self._h, *[N.dptr(a) for a in out]))
        return out

    def wake_strip(self, i=0, j=143):
        """V along xi3 at the grid point (i, j) (Nz values)."""
        out = np.empty(self.shape[0])
        N.check(N.host_lib().mc3d_solver_wake_strip(self._h, int(i), int(j), N.dptr(out)))
        return out

    def write_turbdata(self, path="turbdata.out", k0=8.0):
        """Append the HIT driver's turbdata.out line for the current state
        (tests/hit/Samtaney_D4/MPI_3DCompact.cpp:545-555)."""
        append_turbdata_line(path, self.turbdata(k0))

    def write_cylinder_data(self, directory=".", strip=(0, 143)):
        """Append the cylinder driver's records for the current state
        (src/MPI_3DCompact.cpp:463-527): time and the span-averaged wall p, U,
        V, W to cylinderP/U/V/W.dat, time and the wake strip V to
        VWakeStrip.dat; a strip point outside the grid gives the driver's
        -100000 fill."""
        t = self.info()["time"]
        for name, a in zip("PUVW", self.wall_span_average()):
            append_record(os.path.join(directory, f"cylinder{name}.dat"), t, a)
        i, j = strip
        nx, ny = self.shape[2], self.shape[1]
        v = self.wake_strip(i, j) if 0 <= i < nx and 0 <= j < ny else np.full(self.shape[0], -100000.0)
        append_record(os.path.join(directory, "VWakeStrip.dat"), t, v)

    def dump_stats(self, velocity_path=None, thermo_path=None):
        enc = (lambda p: None if p is None else str(p).encode())
        N.check(N.host_lib().mc3d_solver_dump_stats(self._h, enc(velocity_path), enc(thermo_path)))

    def read_stats(self, velocity_path=None, thermo_path=None):
        enc = (lambda p: None if p is None else str(p).encode())
        N.check(N.host_lib().mc3d_solver_read_stats(self._h, enc(velocity_path), enc(thermo_path)))

    def metrics(self):
        """The FP64 metrics J, J11..J33 the solver holds (10 arrays (Nz, Ny, Nx))."""
        out = [np.empty(self.shape) for _ in range(10)]
        p = (C.POINTER(C.c_double) * 10)(*[N.dptr(a) for a in out])
        N.check(N.host_lib().mc3d_solver_get_metrics(self._h, p))
        return out

    def set_mlp(self, mlp: MLPClosure):
        """The learned closure of a LESMODEL = MLP solver (kept alive by the solver object)."""
        self._mlp = mlp
        N.check(N.host_lib().mc3d_solver_set_mlp(self._h, mlp._h))

    def mlp_fallbacks(self):
        v = C.c_longlong()
        N.check(N.host_lib().mc3d_solver_mlp_fallbacks(self._h, C.byref(v)))
        return v.value

    def set_sponge(self, sigma):
        """Sponge strength field (SpongeBC::sigma); needed before the initial condition."""
        a = np.ascontiguousarray(sigma, dtype=np.float64)
        N.check(N.host_lib().mc3d_solver_set_sponge(self._h, N.dptr(a)))

    def set_sponge_avg(self, avg):
        """Sponge target state rho, rhoU, rhoV, rhoW, rhoE (readSpongeAvgFromRestart)."""
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in avg]
        p = (C.POINTER(C.c_double) * 5)(*[N.dptr(a) for a in arrs])
        N.check(N.host_lib().mc3d_solver_set_sponge_avg(self._h, p))

    def set_initial_conditions(self, rho, U, V, W, p):
        """setInitialConditions from primitive host arrays, with the wall
        conditions and sponge target (src/CurvilinearCSolver_BC.cpp:3-369)."""
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (rho, U, V, W, p)]
        N.check(N.host_lib().mc3d_solver_set_initial(self._h, *[N.dptr(a) for a in arrs]))

    def step(self, n=1):
        N.check(N.host_lib().mc3d_solver_step(self._h, int(n)))

    def conserved(self, out=None):
        """Host copies of rho1, rhoU1, rhoV1, rhoW1, rhoE1 (into `out`, five
        C-contiguous float64 arrays of the grid's shape, e.g. pinned buffers)."""
        if out is None:
            out = [np.empty(self.shape) for _ in range(5)]
        for a in out:
            if a.shape != self.shape or a.dtype != np.float64 or not a.flags.c_contiguous:
                raise ValueError("conserved(out=...) needs C-contiguous float64 arrays of the grid's shape")
        N.check(N.host_lib().mc3d_solver_get_conserved(self._h, *[N.dptr(a) for a in out]))
        return out

    def copy_conserved_device(self, dst):
        """Device-to-device copy of rho1..rhoE1 into 5 CUDA float64 tensors."""
        p = (C.c_void_p * 5)(*[t.data_ptr() for t in dst])
        N.check(N.host_lib().mc3d_solver_copy_conserved_device(self._h, p))

    def conserved_device_ptrs(self):
        p = (C.c_void_p * 5)()
        N.check(N.host_lib().mc3d_solver_conserved_device(self._h, p))
        return [p[i] for i in range(5)]

    def info(self):
        ts, t, dt, st = C.c_int(), C.c_double(), C.c_double(), C.c_longlong()
        N.check(N.host_lib().mc3d_solver_info(self._h, C.byref(ts), C.byref(t), C.byref(dt), C.byref(st)))
        return {"time_step": ts.value, "time": t.value, "dt": dt.value, "stages": st.value}

    def integrals(self):
        ke, m = C.c_double(), C.c_double()
        N.check(N.host_lib().mc3d_solver_integrals(self._h, C.byref(ke), C.byref(m)))
        return ke.value, m.value

    def stream(self):
        s = C.c_void_p()
        N.check(N.host_lib().mc3d_solver_stream(self._h, C.byref(s)))
        return s.value

    def set_stream(self, stream=None):
        """Queue this solver's kernels on `stream` (a cudaStream_t handle, e.g.
        torch.cuda.Stream().cuda_stream; None: the device's shared stream)."""
        N.check(N.host_lib().mc3d_solver_set_stream(self._h, C.c_void_p(stream) if stream else None))

    def launch_count(self):
        c = C.c_longlong()
        N.check(N.host_lib().mc3d_solver_launch_count(self._h, C.byref(c)))
        return c.value

    def sync(self):
        N.check(N.host_lib().mc3d_solver_sync(self._h))

    def set_timing(self, enable=True):
        N.check(N.host_lib().mc3d_solver_set_timing(self._h, int(bool(enable))))

    def timing_report(self):
        import json
        r = N.host_lib().mc3d_solver_timing_report(self._h)
        if r is None:
            N.check(2)
        return json.loads(r.decode())
