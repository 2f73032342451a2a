#!/usr/bin/env python
"""Throughput of the CurvilinearCSolver time step on B200: grid-point RK stages
per second for decaying HIT on a 256^3 periodic box (Penta10 derivatives,
Compact8 filter alpha_f = 0.45, LSLDDRK4, Vreman SGS), FP32-bulk arithmetic
with FP64 state/accumulators, next to the FP64 GPU path on the same input.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One "step" is one time step of the solver (LSLDDRK4 alternates 5- and
6-stage halves; the metric counts the stages actually run). N > 1 runs
independent replicas (one per rank, different seeds): the path has no
exchange between GPUs. Rank 0 prints one JSON line.

At N = 1 the line also carries "cylinder": the curvilinear O-grid configuration
(512 x 256 x 64 around a cylinder, wall + cylindrical sponge, PADE6 with
boundary closures, KENRK4, COMPACT10, DSM, FP32-bulk, metrics computed on the
GPU from the mesh), and "learned_sgs": a posteriori 128^3 LES of the
same HIT (PADE6, RK4, COMPACT10 alpha_f = 0.49, FP32-bulk, 500 steps) with
the learned closure shipped in mpi_3dcompact_b200/data (DSM with GLOBAL
averaging as its fallback when more than 10% of the points leave the training
range) against DSM and against no model: device time per step, fallback
stages, kinetic-energy decay and the final energy spectrum.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import re
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "grid-pt RK stages/s, 256^3: FP32 vs FP64 GPU; learned SGS vs DSM at stated error"
UNIT = "grid-pt RK stages/s"
GRID = 256
K0, MT, RE_LAMBDA = 4.0, 0.3, 100.0
SCHEME = dict(fd="PENTA10", filter="COMPACT8", alphaF=0.45, rk="LSLDDRK4", les="VREMAN", les_avg="NONE", cfl=0.5)
WORKLOAD = ("decaying HIT 256^3 periodic box 2*pi, PENTA10 derivatives, COMPACT8 filter alpha_f=0.45 every step, "
            "LSLDDRK4, VREMAN SGS, CFL 0.5, Mt=0.3, Re_lambda~100, FP32-bulk (FP64 state, RK registers, dt/time)")
# the reference's CPU time step is timed on a 128^3 sample of the same scheme
# (one core: the reference has no threading and no MPI runtime here)
CPU_SAMPLE_GRID = 128
# FP32-bulk against FP64 after the configuration's 200 steps (untimed)
ERR_STEPS = 200
LES_GRID, LES_STEPS, LES_MU, LES_SEED = 128, 500, 2.5e-4, 5
# the learned closure's stage goes to DSM when more than this fraction of the
# points has a feature outside the training range (features are clamped): the
# library's default LES.MLPFALLBACKFRAC
LES_MLP_FALLBACK = 1e-3
LES_SCHEME = dict(fd="PADE6", filter="COMPACT10", alphaF=0.49, rk="RK4", les_avg="GLOBAL", cfl=0.5)
MLP_WEIGHTS = os.path.join(ROOT, "mpi_3dcompact_b200", "data", "mlp_sgs_hit128.bin")
PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM_GBS = 6650.0


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def max_over_ranks(x, dist=None, device="cpu"):
    """The largest x over the ranks (the slowest rank's time); x itself
    without a process group."""
    if dist is None:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(ws, points, stages, seconds):
    """Whole-job grid-point RK stages per second: ws replicas of `points`
    points each ran `stages` stages within `seconds` (the slowest rank)."""
    return ws * float(points) * stages / seconds


def lsldd_stages(first_step: int, nsteps: int) -> int:
    """Stages of LSLDDRK4 steps first_step..first_step+nsteps-1 (1-based): odd
    steps run the 5-stage half, even steps the 6-stage half."""
    return sum(5 if (s % 2) == 1 else 6 for s in range(first_step, first_step + nsteps))


def hbm_peak():
    try:
        with open(PEAKS) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def profile_traffic():
    """Per-launch DRAM traffic of the line-solve kernel from the committed ncu
    summary (a line `traffic_bytes_per_launch: <float>`), else None."""
    p = os.path.join(ROOT, "profiles", "sweep_linesolve_hit256_fp32.md")
    try:
        m = re.search(r"traffic_bytes_per_launch:\s*([0-9.eE+-]+)", open(p).read())
        return float(m.group(1)) if m else None
    except OSError:
        return None


class ClockSampler:
    """nvidia-smi clocks/throttle sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id):
        self.gpu_id = gpu_id
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(prefix="clocks_", suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu_id), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def mu_for(ic):
    up, lam = _hit_ic().reynolds_lambda_mu(ic)
    return up * lam / RE_LAMBDA


def _hit_ic():
    """The HIT initial-condition module, loaded from its file alone: the
    reference arm must not import the package (nor map libmc3d.so)."""
    import importlib.util
    name = "mc3d_hit_ic_standalone"
    if name not in sys.modules:
        spec = importlib.util.spec_from_file_location(name, os.path.join(ROOT, "mpi_3dcompact_b200", "hit_ic.py"))
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        sys.modules[name] = mod
    return sys.modules[name]


def host_cpu():
    """(CPU model name, logical cores) of this host."""
    name = "unknown"
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                name = line.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    return name, os.cpu_count()


def cpu_reference_rate(grid, min_stages, warmup_steps):
    """The reference's own C++ time step (oracle/_ref/mc3d_ref, one core) on a
    `grid`^3 sample of the same scheme, timed over the fewest whole time steps
    that run at least `min_stages` RK stages after `warmup_steps` untimed ones.
    Returns (pt-stages/s, sample text, kind, timed seconds, timed steps,
    timed stages). Imports nothing of the package: the initial condition comes
    from hit_ic.py loaded on its own."""
    from oracle import mc3d_oracle as O
    from oracle import ref_runner as R
    ic = _hit_ic().hit_initial_condition(grid, k0=K0, seed=1, mt=MT)
    cfg = O.Config(N=(grid,) * 3, fd=(SCHEME["fd"],) * 3, filter=SCHEME["filter"], alphaF=SCHEME["alphaF"],
                   rk=SCHEME["rk"], les=SCHEME["les"], les_avg=SCHEME["les_avg"], cfl=SCHEME["cfl"],
                   mu_ref=mu_for(ic))
    steps = 1
    while lsldd_stages(warmup_steps + 1, steps) < min_stages:
        steps += 1
    total = warmup_steps + steps
    if R.available():
        _, info = R.run_solver(cfg, ic, total)
        st = info["step_s"][warmup_steps:total]
        kind = "reference"
    else:   # the numpy restatement when the reference binary is not built
        o = O.Oracle(cfg, O.cube_metrics(cfg.N))
        o.init(*ic)
        st = []
        for i in range(total):
            t0 = time.perf_counter()
            o.step()
            if i >= warmup_steps:
                st.append(time.perf_counter() - t0)
        kind = "port"
    stages = lsldd_stages(warmup_steps + 1, steps)
    rate = grid ** 3 * stages / sum(st)
    sample = (f"{grid}^3 box, same scheme in FP64, {steps} timed time steps ({stages} RK stages) after "
              f"{warmup_steps} warm-up time step(s), 1 core")
    return rate, sample, kind, sum(st), steps, stages


def run_reference_arm(args):
    """The reference's CPU time step on the bench's scheme. Each of the K arm
    steps is one RK stage of a 128^3 sample (the reference's 256^3 time step
    takes minutes on one core); the stages run as whole LSLDDRK4 time steps."""
    ws, rank, _ = dist_env()
    if rank != 0:
        return 0
    w = max(1, round(args.warmup / 5.5))
    rate, sample, kind, secs, tsteps, stages = cpu_reference_rate(CPU_SAMPLE_GRID, args.steps, w)
    line = {
        "impl": "reference", "metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * secs / stages, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded HIT initial condition, "
        "k0=4, Mt=0.3)",
        "config": {"workload": WORKLOAD.replace("FP32-bulk (FP64 state, RK registers, dt/time)", "FP64"),
                   "grid": CPU_SAMPLE_GRID, "arm_step": "one RK stage (ms_per_step is per stage)",
                   "time_steps_timed": tsteps, "stages_timed": stages, "parallelism": "single rank, one core"},
        "cpu_baseline": {"value": rate, "unit": UNIT, "cores": 1, "kind": kind, "sample": sample,
                         "cpu": "{}, 1 of {} logical cores used".format(*host_cpu())},
        "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def energy_spectrum(torch, q):
    """Shell-summed kinetic energy spectrum E(k), k = 0..N/2, of a periodic
    conserved state q (5 device tensors (N, N, N))."""
    n = q[0].shape[0]
    e = None
    for c in range(1, 4):
        uh = torch.fft.fftn(q[c] / q[0]) / n ** 3
        p = 0.5 * (uh.real ** 2 + uh.imag ** 2)
        e = p if e is None else e + p
    k = torch.fft.fftfreq(n, d=1.0 / n, device=e.device, dtype=torch.float64)
    kk = torch.sqrt(k[:, None, None] ** 2 + k[None, :, None] ** 2 + k[None, None, :] ** 2)
    shell = torch.round(kk).long().clamp_(max=n)
    return torch.bincount(shell.reshape(-1), weights=e.reshape(-1), minlength=n + 1)[: n // 2 + 1].cpu().numpy()


def cylinder_block(args, local):
    """The O-grid cylinder configuration: grid-point RK stages per second with
    DSM (GLOBAL averaging), and whether the configuration's LOCAL averaging
    stays finite."""
    import numpy as np
    import torch

    import mpi_3dcompact_b200 as m

    from mpi_3dcompact_b200.meshes import cylinder_flow_ic, cylinder_ogrid
    Nx, Ny, Nz = 512, 256, 64
    r1, span = 30.0, 2.0
    x, y, z, ratio = cylinder_ogrid(Nx, Ny, Nz, 0.5, r1, span)   # (theta clockwise, r, z): J > 0
    ic = cylinder_flow_ic((Nz, Ny, Nx), 0.2, 0.01, 3)

    def make(avg):
        opt = m.Options(grid=(Nx, Ny, Nz), fd="PADE6", filter="COMPACT10", alphaF=0.49, rk="KENRK4",
                        mu_ref=0.2 / 3900.0, les="DSM", les_avg=avg, dsm_test_filter=1, precision=m.FP32BULK,
                        bc=(m.PERIODIC_SOLVE, m.DIRICHLET_SOLVE, m.PERIODIC_SOLVE),
                        bc_kind=("INTERNALLY_PERIODIC", "INTERNALLY_PERIODIC", "ADIABATIC_WALL", "SPONGE",
                                 "PERIODIC", "PERIODIC"),
                        sponge={"kind": "CYLINDRICAL", "strength": 1.0, "orient": 2, "cyl_axis": [0.0, 0.0, 0.0],
                                "rmin": 0.8 * r1},
                        periodic_disp=((0, 0, 0), (0, 0, 0), (0, 0, span)), cfl=0.5)
        s = m.CurvilinearCSolver(opt, device=local)
        t0 = time.perf_counter()
        s.set_mesh(x, y, z)
        tm = time.perf_counter() - t0
        s.set_sponge(m.sponge_sigma(opt, x, y, z))
        s.set_initial_conditions(*ic)
        return s, tm

    s, metrics_s = make("GLOBAL")
    s.step(3)
    s.sync()
    stream = torch.cuda.ExternalStream(s.stream())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    st0 = s.info()["stages"]
    e0.record(stream)
    s.step(args.cyl_steps)
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    stages = s.info()["stages"] - st0
    # per-class algorithmic bytes and device time of two more steps, for the
    # HBM roofline of the configuration (every kernel class together)
    s.set_timing(True)
    s.step(2)
    rep = s.timing_report()
    s.set_timing(False)
    del s
    peak, peak_kind = hbm_peak()
    tot_b = sum(v["bytes"] for v in rep.values())
    tot_ms = sum(v["ms"] for v in rep.values())
    roof = {"bound": "hbm", "kernels": "all kernel classes of the step", "achieved": tot_b / (tot_ms * 1e-3) / 1e9,
            "peak": peak, "unit": "GB/s", "frac": tot_b / (tot_ms * 1e-3) / 1e9 / peak, "peak_kind": peak_kind,
            "algorithmic_bytes_per_pt_stage": tot_b / (float(Nx * Ny * Nz) * (stages / args.cyl_steps) * 2)}
    sl, _ = make("LOCAL")
    local_steps = None
    for k in range(1, 4):
        sl.step(1)
        try:
            sl.info()
        except Exception:
            local_steps = k
            break
    del sl
    return {
        "workload": "O-grid cylinder 512 (theta, periodic) x 256 (r 0.5..30, geometric) x 64 (z periodic, span 2), "
                    "M 0.2, Re_D 3900, adiabatic wall, cylindrical sponge r > 24, PADE6 + boundary closures, KENRK4, "
                    "COMPACT10 alpha_f=0.49, DSM (DSMTESTFILTER=1), FP32-bulk, 1% seeded velocity perturbation",
        "metric": UNIT, "value": Nx * Ny * Nz * stages / (ms * 1e-3), "ms_per_step": ms / args.cyl_steps,
        "steps": args.cyl_steps, "averaging": "GLOBAL",
        "metrics_on_gpu_s": metrics_s,
        "roofline": roof, "kernels": rep,
        "local_averaging_nonfinite_after_steps": local_steps,
        "note": "the configuration's LOCAL averaging divides by a locally filtered M_ij M_ij and goes non-finite "
                "in the reference's own solver as well (128x64x32 O-grid, first step); radial ratio "
                "(30/0.5)^(1/255) = %.4f so that r ends at 30" % ratio,
    }


def learned_sgs_block(args, local):
    """A posteriori LES with the learned closure against DSM and no model."""
    import numpy as np
    import torch

    import mpi_3dcompact_b200 as m
    from mpi_3dcompact_b200.hit_ic import hit_initial_condition

    n, steps, chunk = LES_GRID, args.les_steps, 25
    ic = hit_initial_condition(n, k0=K0, seed=LES_SEED, mt=MT)
    out = {}
    for les in ("MLP", "DSM", "NOMODEL"):
        kw = dict(mlp_fallback_frac=args.les_fallback) if les == "MLP" else {}
        s = m.CurvilinearCSolver(m.Options(grid=n, mu_ref=LES_MU, les=les, precision=m.FP32BULK, **LES_SCHEME, **kw),
                                 device=local)
        s.set_box_metrics(2 * math.pi)
        s.set_initial_conditions(*ic)
        if les == "MLP":
            mlp = m.MLPClosure(device=local)
            mlp.load(MLP_WEIGHTS)
            s.set_mlp(mlp)
        stream = torch.cuda.ExternalStream(s.stream())
        ke = [s.integrals()[0]]
        ms = 0.0
        done = 0
        while done < steps:
            k = min(chunk, steps - done)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            s.step(k)
            e1.record(stream)
            e1.synchronize()
            ms += e0.elapsed_time(e1)
            done += k
            ke.append(s.integrals()[0])
        q = [torch.empty((n, n, n), dtype=torch.float64, device=f"cuda:{local}") for _ in range(5)]
        s.copy_conserved_device(q)
        spec = energy_spectrum(torch, q)
        out[les] = dict(ms=ms / steps, ke=np.array(ke), spec=spec, stages=s.info()["stages"],
                        fallbacks=s.mlp_fallbacks() if les == "MLP" else None,
                        finite=bool(all(torch.isfinite(t).all().item() for t in q)))
        del s, q
    mlp, dsm, nom = out["MLP"], out["DSM"], out["NOMODEL"]

    def decay_diff(a):
        da, dd = a["ke"][0] - a["ke"], dsm["ke"][0] - dsm["ke"]
        return float(np.max(np.abs(da[1:] - dd[1:]) / np.abs(dd[1:])))

    kmax = n // 3   # resolved band below the filter cut-off
    band = slice(1, kmax + 1)

    def spec_diff(a):
        return float(np.linalg.norm(a["spec"][band] - dsm["spec"][band]) / np.linalg.norm(dsm["spec"][band]))

    return {
        "workload": f"decaying HIT {n}^3 LES, PADE6, RK4, COMPACT10 alpha_f=0.49 every step, CFL 0.5, Mt=0.3, "
                    f"mu_ref={LES_MU}, FP32-bulk, {steps} steps from the seed-{LES_SEED} initial field",
        "closure": "9-64-64-64-2 GELU MLP, BF16 tcgen05 tensor-core inference (TMEM accumulators, GELU in packed "
                   "BF16) fused into the SGS pass; trained on 8 seeds of 512^3 DNS box-filtered to 128^3, coefficient "
                   "calibrated a posteriori on LES seeds 1 and 2 (mpi_3dcompact_b200/train_sgs.py)",
        "ms_per_step": {"mlp": mlp["ms"], "dsm": dsm["ms"], "nomodel": nom["ms"]},
        "mlp_speedup_over_dsm": dsm["ms"] / mlp["ms"],
        "fallback_frac": args.les_fallback, "fallback_stages": mlp["fallbacks"], "stages": mlp["stages"],
        "ke_decay_max_rel_diff_vs_dsm": {"mlp": decay_diff(mlp), "nomodel": decay_diff(nom)},
        "ke_final": {"mlp": float(mlp["ke"][-1]), "dsm": float(dsm["ke"][-1]), "nomodel": float(nom["ke"][-1]),
                     "initial": float(dsm["ke"][0])},
        "spectrum_rel_l2_vs_dsm_k1_to_%d" % kmax: {"mlp": spec_diff(mlp), "nomodel": spec_diff(nom)},
        "finite": {k: v["finite"] for k, v in out.items()},
        "timing": "CUDA events on the solver stream over 25-step chunks, summed",
    }


HBM_GRID, HBM_K0 = 1024, 8.0
HBM_WORKLOAD = ("HBM-sizing: decaying HIT 1024^3 periodic box 2*pi, PENTA10, COMPACT8 alpha_f=0.45 every step, "
                "LSLDDRK4, learned SGS closure (MLP, stages past the fallback fraction counted: no DSM fallback "
                "with lean storage), FP32-bulk with FP64 state and 2N register, GPU.STORAGE=LEAN, k0=8, Mt=0.3, "
                "Re_lambda~100, CFL 0.5")


def hbm_sizing_run(args, local):
    """the 1024^3 block held on one GPU by lean storage. The
    initial field is made on the device (the reference generator's sequence,
    cuFFT), moved to host memory to free the device for the solver, and
    uploaded by set_initial_conditions. Device time of `steps` steps after
    `warmup`, CUDA events on the solver stream; resident bytes from
    cudaMemGetInfo around the solver's creation."""
    import numpy as np
    import torch

    import mpi_3dcompact_b200 as m
    from mpi_3dcompact_b200.hit_ic import hit_velocity_device

    n = args.hbm_grid
    dev = torch.device("cuda", local)
    t0 = time.perf_counter()
    u = hit_velocity_device(n, k0=HBM_K0, seed=1, device=dev)
    scale = MT / math.sqrt(float(sum((c * c).mean() for c in u)))
    # Taylor microscale of the scaled field (spectral d/dx of u on the 2*pi box)
    k = torch.fft.rfftfreq(n, d=1.0 / n, device=dev).to(torch.float64)
    du = torch.fft.irfft(1j * k * torch.fft.rfft(u[0] * scale, dim=2), n=n, dim=2)
    up = scale * math.sqrt(float(sum((c * c).mean() for c in u)) / 3.0)
    lam = math.sqrt(float(((u[0] * scale) ** 2).mean()) / float((du * du).mean()))
    del du
    mu = up * lam / RE_LAMBDA
    host = [np.ones((n, n, n))]
    for c in u:
        host.append((c * scale).cpu().numpy())
    host.append(np.full((n, n, n), 1.0 / 1.4))
    del u, c
    torch.cuda.empty_cache()
    ic_s = time.perf_counter() - t0
    free0 = torch.cuda.mem_get_info(dev)[0]
    s = m.CurvilinearCSolver(m.Options(grid=n, fd="PENTA10", filter="COMPACT8", alphaF=0.45, rk="LSLDDRK4",
                                       les="MLP", mlp_fallback_frac=LES_MLP_FALLBACK, mu_ref=mu, cfl=0.5,
                                       precision=m.FP32BULK, storage="LEAN"), device=local)
    s.set_box_metrics(2 * math.pi)
    mlp = m.MLPClosure(device=local)
    mlp.load(MLP_WEIGHTS)
    s.set_mlp(mlp)
    torch.cuda.synchronize(dev)
    resident = free0 - torch.cuda.mem_get_info(dev)[0]
    s.set_initial_conditions(*host)
    del host
    s.step(args.warmup)
    s.sync()
    stream = torch.cuda.ExternalStream(s.stream())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    st0 = s.info()["stages"]
    fb0 = s.mlp_fallbacks()
    s.set_timing(True)
    e0.record(stream)
    s.step(args.steps)
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    rep = s.timing_report()
    s.set_timing(False)
    stages = s.info()["stages"] - st0
    ke, mass = s.integrals()
    peak, peak_kind = hbm_peak()
    sw = rep.get("sweep_linesolve", {})
    roof = None
    if sw:
        achieved = sw["bytes"] / sw["launches"] / (sw["ms"] * 1e-3 / sw["launches"]) / 1e9
        roof = {"bound": "hbm", "kernel": "sweep_linesolve", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_kind": peak_kind,
                "kernel_share": sw["ms"] / sum(v["ms"] for v in rep.values())}
    total_bytes = sum(v["bytes"] for v in rep.values())
    return {"workload": HBM_WORKLOAD, "grid": n, "metric": UNIT, "value": float(n) ** 3 * stages / (ms * 1e-3),
            "ms_per_step": ms / args.steps, "steps": args.steps, "warmup": args.warmup, "stages_timed": stages,
            "resident_device_bytes": int(resident), "resident_fp32_field_equivalents": resident / (4.0 * n ** 3),
            "algorithmic_bytes_per_pt_stage": total_bytes / (float(n) ** 3 * stages),
            "all_kernels_gbs": total_bytes / (sum(v["ms"] for v in rep.values()) * 1e-3) / 1e9,
            "mlp_out_of_range_stages": s.mlp_fallbacks() - fb0, "mu_ref": mu, "initial_field_s": ic_s,
            "finite": bool(math.isfinite(ke) and math.isfinite(mass)), "roofline": roof, "kernels": rep}


def fp32_vs_fp64(m, make, nsteps):
    """FP32-bulk against the FP64 path from the same initial field after
    `nsteps` time steps (untimed): per-field relative L2 and max differences of
    the conserved state, the decay of the kinetic energy and its curve."""
    import numpy as np
    a, b = make(m.FP32BULK), make(m.FP64)
    curve = {"step": [0], "fp32": [float(a.integrals()[0])], "fp64": [float(b.integrals()[0])]}
    for k in range(1, nsteps + 1):
        a.step(1)
        b.step(1)
        if k % 10 == 0 or k == nsteps:
            curve["step"].append(k)
            curve["fp32"].append(float(a.integrals()[0]))
            curve["fp64"].append(float(b.integrals()[0]))
    qa, qb = a.conserved(), b.conserved()
    ta, tb = a.info()["time"], b.info()["time"]
    del a, b
    names = ["rho", "rhoU", "rhoV", "rhoW", "rhoE"]
    l2 = {nm: float(np.linalg.norm(x - y) / np.linalg.norm(y)) for nm, x, y in zip(names, qa, qb)}
    mx = {nm: float(np.abs(x - y).max() / np.abs(y).max()) for nm, x, y in zip(names, qa, qb)}
    d32 = curve["fp32"][0] - np.array(curve["fp32"][1:])
    d64 = curve["fp64"][0] - np.array(curve["fp64"][1:])
    return {"steps": nsteps, "rel_l2": l2, "rel_max": mx, "max_rel_l2": max(l2.values()),
            "ke_decay_rel_diff_final": float(d32[-1] / d64[-1] - 1.0),
            "ke_decay_max_rel_diff": float(np.max(np.abs(d32 - d64) / np.abs(d64))),
            "time": {"fp32": ta, "fp64": tb}, "curve": curve}


def run_ours(args):
    import numpy as np
    import torch

    import mpi_3dcompact_b200 as m
    from mpi_3dcompact_b200.hit_ic import hit_initial_condition

    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    dist = None
    if ws > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))
    n = args.grid
    ic = hit_initial_condition(n, k0=K0, seed=1 + rank, mt=MT)
    mu = mu_for(ic)

    def make(precision):
        s = m.CurvilinearCSolver(m.Options(grid=n, mu_ref=mu, precision=precision, **SCHEME), device=local)
        s.set_box_metrics(2 * math.pi)
        s.set_initial_conditions(*ic)
        return s

    def barrier():
        if dist is not None:
            dist.barrier()

    def timed(s, steps, warmup, with_timing):
        s.step(warmup)
        s.sync()
        stream = torch.cuda.ExternalStream(s.stream())
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        st0 = s.info()["stages"]
        l0 = s.launch_count()
        if with_timing:
            s.set_timing(True)
        barrier()
        torch.cuda.synchronize()
        e0.record(stream)
        s.step(steps)
        e1.record(stream)
        torch.cuda.synchronize()
        barrier()
        ms = e0.elapsed_time(e1)
        rep = s.timing_report() if with_timing else None
        if with_timing:
            s.set_timing(False)
        return ms, s.info()["stages"] - st0, s.launch_count() - l0, rep

    gpu_id = local
    try:
        uuid = str(torch.cuda.get_device_properties(local).uuid)
        gpu_id = uuid if uuid.startswith("GPU-") else f"GPU-{uuid}"
    except Exception:
        pass
    clocks = ClockSampler(gpu_id)

    # ---- FP32-bulk, device-resident (the headline value) ----
    s32 = make(m.FP32BULK)
    clocks.start()
    ms, stages, launches, rep = timed(s32, args.steps, args.warmup, True)
    clk = clocks.stop()
    ms = max_over_ranks(ms, dist, "cuda")
    pts = float(n) ** 3
    value = job_rate(ws, pts, stages, ms * 1e-3)
    del s32

    # ---- FP64 GPU path on the same input ----
    fp64 = None
    cmp = None
    if not args.no_fp64:
        s64 = make(m.FP64)
        ms64, st64, _, _ = timed(s64, args.steps, args.warmup, False)
        del s64
        fp64 = pts * st64 / (ms64 * 1e-3)
        cmp = fp32_vs_fp64(m, make, args.err_steps)

    # ---- end to end through the C ABI with host buffers ----
    e2e = None
    if not args.no_e2e:
        se = m.CurvilinearCSolver(m.Options(grid=n, mu_ref=mu, precision=m.FP32BULK, **SCHEME), device=local)
        se.set_box_metrics(2 * math.pi)

        def pinned():
            return torch.empty(ic[0].shape, dtype=torch.float64, pin_memory=True).numpy()
        host_ic = [pinned() for _ in range(5)]        # the initial condition in pinned host memory
        for a, b in zip(host_ic, ic):
            a[...] = b
        out = [pinned() for _ in range(5)]
        torch.cuda.synchronize()
        barrier()
        t0 = time.perf_counter()
        se.set_initial_conditions(*host_ic)          # host -> device (FP64 primitives)
        for _ in range(args.steps):
            se.step(1)
            se.info()                                # per-step device -> host read of time step / dt
        se.conserved(out=out)                        # device -> host (FP64 conserved state)
        wall = time.perf_counter() - t0
        barrier()
        st_e = se.info()["stages"]
        del se
        wall = max_over_ranks(wall, dist, "cuda")
        e2e = {"value": job_rate(ws, pts, st_e, wall), "unit": UNIT,
               "h2d_bytes_per_step": int(5 * 8 * pts / args.steps),
               "d2h_bytes_per_step": int(5 * 8 * pts / args.steps + 32)}
        del out

    les = None
    if ws == 1 and not args.no_learned_sgs:
        les = learned_sgs_block(args, local)
    cyl = None
    if ws == 1 and not args.no_cylinder:
        cyl = cylinder_block(args, local)

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        # one 5-stage time step of the reference at 128^3 (about half a minute)
        rate, sample, kind, _, _, _ = cpu_reference_rate(CPU_SAMPLE_GRID, 5, 0)
        model, ncores = host_cpu()
        cpu = {"value": rate, "unit": UNIT, "cores": 1, "kind": kind, "sample": sample,
               "cpu": f"{model}, 1 of {ncores} logical cores used"}

    peak, peak_kind = hbm_peak()
    sw = rep.get("sweep_linesolve", {}) if rep else {}
    roof = None
    if sw:
        per_launch_bytes = sw["bytes"] / sw["launches"]
        per_launch_s = sw["ms"] * 1e-3 / sw["launches"]
        achieved = per_launch_bytes / per_launch_s / 1e9
        tr = profile_traffic()
        roof = {"bound": "hbm", "kernel": "sweep_linesolve (compact line solve, all directions/epilogues)",
                "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "peak_kind": peak_kind, "traffic": tr, "algorithmic_bytes_per_launch": per_launch_bytes,
                "kernel_share": sw["ms"] / sum(v["ms"] for v in rep.values())}
    if dist is not None:
        dist.destroy_process_group()
    if rank != 0:
        return 0
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (seeded HIT initial condition, k0=4, Mt=0.3)",
        "config": {"workload": WORKLOAD, "grid": n, "stages_timed": stages,
                   "l2": "inputs larger than L2: 40 resident fields of 64-128 MB", "parallelism":
                   "replicas" if ws > 1 else "single GPU"},
        "roofline": roof, "kernels": rep, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches,
        "clocks": clk, "fp32_vs_fp64_ke_curve": cmp.pop("curve") if cmp else None, "cylinder": cyl,
        "learned_sgs": les,
        # the compact results last, where a truncated record still keeps them
        "learned_vs_dsm": None if not les else {
            "mlp_ms_per_step": les["ms_per_step"]["mlp"], "dsm_ms_per_step": les["ms_per_step"]["dsm"],
            "speedup": les["mlp_speedup_over_dsm"], "fallback_frac": les["fallback_frac"],
            "fallback_stages": les["fallback_stages"],
            "ke_decay_max_rel_diff": les["ke_decay_max_rel_diff_vs_dsm"]["mlp"]},
        "fp64_value": fp64, "fp32_over_fp64": (value / ws / fp64) if fp64 else None,
        "fp64_over_cpu_reference": (fp64 / cpu["value"]) if (fp64 and cpu) else None,
        "fp32_vs_fp64": cmp,
    }
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--grid", type=int, default=GRID)
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-learned-sgs", action="store_true")
    ap.add_argument("--no-cylinder", action="store_true")
    ap.add_argument("--cyl-steps", type=int, default=5)
    ap.add_argument("--les-steps", type=int, default=LES_STEPS)
    ap.add_argument("--les-fallback", type=float, default=LES_MLP_FALLBACK,
                    help="fallback fraction of the learned closure in the 128^3 LES")
    ap.add_argument("--err-steps", type=int, default=ERR_STEPS)
    ap.add_argument("--workload", choices=["hit256", "hbm1024"], default="hit256",
                    help="hbm1024: the 1024^3 HBM-sizing configuration with lean storage")
    ap.add_argument("--hbm-grid", type=int, default=HBM_GRID)
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference_arm(args)
    if args.workload == "hbm1024":
        import torch
        ws, rank, local = dist_env()
        torch.cuda.set_device(local)
        res = hbm_sizing_run(args, local)
        if rank == 0:
            print(json.dumps({"metric": METRIC, "value": res["value"], "unit": UNIT, "n_gpus": 1,
                              "steps": args.steps, "warmup": args.warmup, "ms_per_step": res["ms_per_step"],
                              "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                              "data": "synthetic (seeded HIT initial condition, k0=8, Mt=0.3)",
                              "config": {"workload": res["workload"], "grid": res["grid"]},
                              "roofline": res["roofline"], "hbm_sizing": res}), flush=True)
        return 0
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
