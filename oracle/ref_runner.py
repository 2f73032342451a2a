"""Runs the reference solver binary oracle/_ref/mc3d_ref (built by oracle/Makefile
from the reference's own sources). TEST INFRASTRUCTURE ONLY: used by the golden
fixture generator, the oracle's self-check tests and bench.py's reference arm.

Fields cross the process boundary as FP64 arrays shaped (Nz, Ny, Nx).
"""
from __future__ import annotations

import os
import shutil
import subprocess
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_BIN = os.path.join(HERE, "_ref", "mc3d_ref")
# the harness with the hooks of the reference's HIT driver
# (tests/hit/Samtaney_D4/MPI_3DCompact.cpp) or cylinder driver (src/MPI_3DCompact.cpp)
HOOK_BINS = {"hit": os.path.join(HERE, "_ref", "mc3d_ref_hit"), "cyl": os.path.join(HERE, "_ref", "mc3d_ref_cyl")}
HOOK_FILES = {"hit": ("turbdata.out",), "cyl": ("cylinderP.dat", "cylinderU.dat", "cylinderV.dat", "cylinderW.dat",
                                                 "VWakeStrip.dat")}

_BC = {0: "PERIODIC_SOLVE", 1: "DIRICHLET_SOLVE"}


def available() -> bool:
    return os.path.isfile(REF_BIN) and os.access(REF_BIN, os.X_OK)


def ini_text(cfg, max_steps: int, kinds=None, box=6.283185307179586) -> str:
    """MPI_3DCompact.in for an oracle Config (keys of src/Options.hpp:133-206).
    Periodic faces are translated by `box` along their own axis, as the HIT case
    sets PERIODICDISPX_X = PERIODICDISPY_Y = PERIODICDISPZ_Z = 2*pi
    (tests/hit/Samtaney_D4/MPI_3DCompact.in)."""
    Nx, Ny, Nz = cfg.N
    if kinds is None:
        kinds = cfg.kinds() if hasattr(cfg, "kinds") else \
            [k for b in cfg.bc for k in (("PERIODIC",) * 2 if b == 0 else ("ADIABATIC_WALL",) * 2)]
    elif len(kinds) == 3:
        kinds = [k for k in kinds for _ in range(2)]
    lines = [
        "[TIMESTEPPING]",
        f"TSTYPE = {cfg.ts_type}",
        f"CFL = {cfg.cfl!r}",
    ]
    if cfg.ts_type == "CONST_DT":
        lines.append(f"DT = {cfg.dt!r}")
    lines += [
        "MAXTIME = 1e30",
        f"MAXTIMESTEP = {max_steps}",
        f"FILTERSTEP = {cfg.filter_step}",
        f"SUBSTEPFILTERING = {'true' if cfg.substep_filtering else 'false'}",
        "CHECKSTEP = 1000000000",
        "DUMPSTEP = 1000000000",
        "[RESTART]",
        "FROMRESTART = false",
        "ONLYGRIDFROMRESTART = false",
        "SPONGEAVGFROMRESTART = false",
        "[STATS]",
    ]
    st = getattr(cfg, "stats", None)
    if st:
        lines += [f"VELOCITYSTATS = {'true' if st.get('velocity', True) else 'false'}",
                  f"THERMOSTATS = {'true' if st.get('thermo', True) else 'false'}",
                  "VELOCITYSTATSFROMRESTART = false", "THERMOSTATSFROMRESTART = false",
                  f"STATSAVGTYPE = {st.get('avg', 'NONE')}", f"INTERVAL = {st.get('interval', 1)}"]
    else:
        lines += ["VELOCITYSTATS = false", "THERMOSTATS = false", "STATSAVGTYPE = NONE"]
    lines += [
        "[BC]",
    ]
    for ax, name in enumerate("XYZ"):
        lines.append(f"BC{name}TYPE = {_BC[cfg.bc[ax]]}")
        lines.append(f"BC{name}0 = {kinds[2 * ax]}")
        lines.append(f"BC{name}1 = {kinds[2 * ax + 1]}")
        if kinds[2 * ax] == "PERIODIC":
            L = getattr(cfg, "periodic_box", None)
            b = L[ax] if L is not None else box
            full = getattr(cfg, "periodic_disp", None)
            for ci, c in enumerate("XYZ"):
                v = full[ax][ci] if full is not None else (b if c == name else 0.0)
                lines.append(f"PERIODICDISP{name}_{c} = {float(v)!r}")
    sp = getattr(cfg, "sponge", None)
    if "SPONGE" in kinds and sp:
        lines += ["[SPONGE]", f"KIND = {sp.get('kind', 'RECTILINEAR')}", f"STRENGTH = {sp.get('strength', 1.0)!r}"]
        relax = getattr(cfg, "sponge_relax", None)
        if relax:
            lines += [f"AVGTIME = {float(relax.get('avg_time', 1.0))!r}",
                      f"PINF = {float(relax.get('p_inf', 1.0 / 1.4))!r}"]
        if sp.get("kind", "RECTILINEAR") == "RECTILINEAR":
            for f, key in enumerate(("X0", "X1", "Y0", "Y1", "Z0", "Z1")):
                if kinds[f] == "SPONGE":
                    lines.append(f"RECT{key}PERC = {sp['rect_perc'][f]!r}")
        else:
            lines += [f"CYLAXIS_ORIENT = {sp.get('orient', 2)}", f"CYLAXIS_X = {sp['cyl_axis'][0]!r}",
                      f"CYLAXIS_Y = {sp['cyl_axis'][1]!r}", f"CYLAXIS_Z = {sp['cyl_axis'][2]!r}",
                      f"RMIN = {sp['rmin']!r}"]
    lines += [
        "[DOMAIN]",
        f"NX = {Nx}",
        f"NY = {Ny}",
        f"NZ = {Nz}",
        "[SOLVER]",
        f"ALPHAF = {cfg.alphaF!r}",
        f"MU_REF = {cfg.mu_ref!r}",
        f"XFDTYPE = {cfg.fd[0]}",
        f"YFDTYPE = {cfg.fd[1]}",
        f"ZFDTYPE = {cfg.fd[2]}",
        f"FILTERTYPE = {cfg.filter}",
        f"RKTYPE = {cfg.rk}",
        "[LES]",
        f"LESMODEL = {cfg.les}",
        f"LESAVERAGING = {cfg.les_avg}",
        f"DSMTESTFILTER = {getattr(cfg, 'dsm_test_filter', 1)}",
        f"DSMUSETAUKK = {'true' if getattr(cfg, 'dsm_use_taukk', True) else 'false'}",
    ]
    return "\n".join(lines) + "\n"


def _write(path, arrays):
    with open(path, "wb") as f:
        for a in arrays:
            f.write(np.ascontiguousarray(a, dtype=np.float64).tobytes())


def _read_fields(path, N, nf, header=8):
    Nx, Ny, Nz = N
    raw = np.fromfile(path, dtype=np.float64)
    hdr = raw[:header]
    n = Nx * Ny * Nz
    fields = [raw[header + i * n: header + (i + 1) * n].reshape(Nz, Ny, Nx).copy() for i in range(nf)]
    return hdr, fields


def run_solver(cfg, ic, nsteps, mesh="cube:6.283185307179586", timeout=3600, coords=None, dump_to=None,
               restart_from=None, sponge_dump_to=None, stats_to=None, hooks=None):
    """Run the reference solver for `nsteps` time steps from primitive ICs
    (rho, U, V, W, p). `coords` = (x, y, z) selects a mesh from file. Returns
    (conserved fields, header dict). `dump_to`: copy the SolutionDump.<step>
    file the reference writes when it reaches its last step
    (CurvilinearCSolver::checkEnd, src/CurvilinearCSolver_Core.cpp:1820-1823)
    to this path. `restart_from`: start from a SolutionDump file instead of
    `ic` (mesh, conserved state, time step and time from the file, as
    src/MPI_3DCompact.cpp:80-271 restarts); nsteps then counts from its step.
    `sponge_dump_to`: copy the SpongeAvgDump.<step> written with it;
    `stats_to`: (velocity, thermo) paths for the VelocityStats.<step> /
    ThermoStats.<step> files written with it (cfg.stats enabled);
    `hooks`: "hit" or "cyl" runs the harness with that reference driver's
    hooks and returns the files they wrote in info["hooks"] (name -> bytes)."""
    binary = REF_BIN if hooks is None else HOOK_BINS[hooks]
    if not (os.path.isfile(binary) and os.access(binary, os.X_OK)):
        raise RuntimeError(f"{binary} is not built (make -C oracle all hooks)")
    if restart_from is not None:
        nsteps += int(np.fromfile(restart_from, dtype=np.float64, count=1)[0])   # MAXTIMESTEP is absolute
    with tempfile.TemporaryDirectory() as d:
        with open(os.path.join(d, "MPI_3DCompact.in"), "w") as f:
            f.write(ini_text(cfg, nsteps))
        if restart_from is not None:
            shutil.copy(restart_from, os.path.join(d, "restart.bin"))
            cmd = [binary, "restart", "restart.bin", "out.bin"]
        else:
            _write(os.path.join(d, "ic.bin"), ic)
            if coords is not None:
                _write(os.path.join(d, "mesh.bin"), coords)
                mesh = "file:mesh.bin"
            cmd = [binary, "run", mesh, "ic.bin", "out.bin"]
        t0 = time.perf_counter()
        env = dict(os.environ)
        env["MC3D_REF_UPDATE_SPONGE"] = "1" if getattr(cfg, "sponge_relax", None) else "0"
        r = subprocess.run(cmd, cwd=d, capture_output=True, text=True, timeout=timeout, env=env)
        wall = time.perf_counter() - t0
        if r.returncode != 0:
            raise RuntimeError("mc3d_ref failed: " + r.stderr[-2000:] + r.stdout[-2000:])
        hdr, fields = _read_fields(os.path.join(d, "out.bin"), cfg.N, 5)
        if dump_to is not None:
            shutil.copy(os.path.join(d, f"SolutionDump.{int(hdr[0])}"), dump_to)
        if sponge_dump_to is not None:
            shutil.copy(os.path.join(d, f"SpongeAvgDump.{int(hdr[0])}"), sponge_dump_to)
        if stats_to is not None:
            for name, dst in zip(("VelocityStats", "ThermoStats"), stats_to):
                if dst is not None:
                    shutil.copy(os.path.join(d, f"{name}.{int(hdr[0])}"), dst)
        st = os.path.join(d, "step_times.txt")
        step_s = [float(x) for x in open(st).read().split()] if os.path.exists(st) else []
        hook_out = {}
        for name in HOOK_FILES.get(hooks, ()):
            fp = os.path.join(d, name)
            hook_out[name] = open(fp, "rb").read() if os.path.exists(fp) else b""
    info = {"time_step": int(hdr[0]), "time": hdr[1], "dt": hdr[5], "solver_wall_s": hdr[6], "wall_s": wall,
            "step_s": step_s, "hooks": hook_out}
    return fields, info


def run_metrics(cfg, mesh="cube:6.283185307179586", coords=None):
    """J, J11..J33 as the reference's solveForJacobians computes them."""
    with tempfile.TemporaryDirectory() as d:
        with open(os.path.join(d, "MPI_3DCompact.in"), "w") as f:
            f.write(ini_text(cfg, 1))
        if coords is not None:
            _write(os.path.join(d, "mesh.bin"), coords)
            mesh = "file:mesh.bin"
        r = subprocess.run([REF_BIN, "metrics", mesh, "m.bin"], cwd=d, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("mc3d_ref metrics failed: " + r.stderr[-2000:])
        _, fields = _read_fields(os.path.join(d, "m.bin"), cfg.N, 10)
    return fields


def run_op(cfg, scheme, direction, field):
    """One derivative (PADE6|PENTA10|CD2) or filter (COMPACT8|COMPACT10, alpha
    = cfg.alphaF) along `direction` with the reference's own operator class."""
    with tempfile.TemporaryDirectory() as d:
        with open(os.path.join(d, "MPI_3DCompact.in"), "w") as f:
            f.write(ini_text(cfg, 1))
        _write(os.path.join(d, "in.bin"), [field])
        r = subprocess.run([REF_BIN, "ops", scheme, str(direction), "in.bin", "out.bin"], cwd=d,
                           capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("mc3d_ref ops failed: " + r.stderr[-2000:])
        Nx, Ny, Nz = cfg.N
        return np.fromfile(os.path.join(d, "out.bin"), dtype=np.float64).reshape(Nz, Ny, Nx)
