"""ctypes binding of the C ABI in include/mc3d.h (libmc3d.so, built in-tree).

The product path has no fallback: if the library is missing or fails to load,
every entry point raises.
"""
from __future__ import annotations

import ctypes as C
import os
import re

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libmc3d.so")
HEADER = os.path.join(os.path.dirname(PKG), "include", "mc3d.h")

MC3D_OK = 0
ERRORS = {1: "MC3D_ERR_CONFIG", 2: "MC3D_ERR_CUDA", 3: "MC3D_ERR_NONFINITE", 4: "MC3D_ERR_OOM",
          5: "MC3D_ERR_TIMEOUT", 6: "MC3D_ERR_ARG"}

FP64, FP32BULK = 0, 1
CONST_DT, CONST_CFL = 0, 1
PERIODIC_SOLVE, DIRICHLET_SOLVE = 0, 1
CD2, PADE6, PENTA10 = 0, 1, 2
COMPACT8, COMPACT10 = 0, 1
NOMODEL, VREMAN, DSM, MLPSGS = 0, 1, 2, 3
AVG_NONE, AVG_XI1, AVG_XI2, AVG_XI3, AVG_LOCAL, AVG_GLOBAL = range(6)
TVDRK3, RK4, KENRK4, LSLDDRK4 = 0, 1, 2, 3


class Mc3dError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


class Config(C.Structure):
    _fields_ = [("Nx", C.c_int), ("Ny", C.c_int), ("Nz", C.c_int),
                ("bc_type", C.c_int * 3), ("bc_kind", C.c_int * 6), ("fd_type", C.c_int * 3),
                ("filter_type", C.c_int), ("alphaF", C.c_double), ("mu_ref", C.c_double),
                ("rk_type", C.c_int), ("ts_type", C.c_int), ("cfl", C.c_double), ("dt", C.c_double),
                ("filter_step", C.c_int), ("substep_filtering", C.c_int), ("max_time_step", C.c_int),
                ("max_time", C.c_double), ("les_model", C.c_int), ("les_averaging", C.c_int),
                ("time_step0", C.c_int), ("time0", C.c_double), ("precision", C.c_int),
                ("reference_quirks", C.c_int), ("dsm_test_filter", C.c_int), ("dsm_use_taukk", C.c_int),
                ("sponge_kind", C.c_int), ("sponge_strength", C.c_double), ("sponge_rect_perc", C.c_double * 6),
                ("sponge_cyl_orient", C.c_int), ("sponge_cyl_axis", C.c_double * 3), ("sponge_rmin", C.c_double),
                ("wall_velocity", (C.c_double * 2) * 6), ("mlp_fallback_frac", C.c_double),
                ("periodic_disp", (C.c_double * 3) * 3), ("dump_step", C.c_int),
                ("from_restart", C.c_int), ("only_grid_from_restart", C.c_int), ("sponge_avg_from_restart", C.c_int),
                ("restart_file", C.c_char * 512), ("sponge_avg_file", C.c_char * 512),
                ("velocity_stats", C.c_int), ("thermo_stats", C.c_int), ("stats_interval", C.c_int),
                ("stats_avg_type", C.c_int), ("velocity_stats_from_restart", C.c_int),
                ("thermo_stats_from_restart", C.c_int), ("velocity_stats_file", C.c_char * 512),
                ("thermo_stats_file", C.c_char * 512), ("sponge_avg_time", C.c_double),
                ("sponge_p_inf", C.c_double), ("sponge_relax", C.c_int), ("lean_storage", C.c_int),
                ("lean_slab", C.c_int)]


_lib = None


def host_lib():
    """Load libmc3d.so (raises if it is missing: there is no fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m mpi_3dcompact_b200.build`")
        lib = C.CDLL(LIB_PATH)
        vp, ip, dp = C.c_void_p, C.c_int, C.c_double
        sigs = {
            "mc3d_config_default": (ip, [C.POINTER(Config)]),
            "mc3d_config_from_ini": (ip, [C.c_char_p, C.POINTER(Config)]),
            "mc3d_last_error": (C.c_char_p, []),
            "mc3d_deriv_create": (ip, [ip, ip, ip, ip, ip, ip, dp, ip, ip, C.POINTER(vp)]),
            "mc3d_filter_create": (ip, [ip, dp, ip, C.POINTER(C.c_int), ip, ip, ip, ip, ip, C.POINTER(vp)]),
            "mc3d_op_apply": (ip, [vp, C.POINTER(vp), C.POINTER(vp), ip, vp]),
            "mc3d_op_destroy": (ip, [vp]),
            "mc3d_op_tpb_ghosts": (ip, [vp, C.POINTER(ip)]),
            "mc3d_op_apply_tpb": (ip, [vp, C.POINTER(vp), C.POINTER(vp), ip, C.POINTER(vp), vp]),
            "mc3d_calc_neumann": (dp, [ip, C.POINTER(dp)]),
            "mc3d_solver_create": (ip, [C.POINTER(Config), ip, C.POINTER(vp)]),
            "mc3d_solver_destroy": (ip, [vp]),
            "mc3d_solver_set_metrics": (ip, [vp, C.POINTER(C.POINTER(dp))]),
            "mc3d_solver_set_box_metrics": (ip, [vp, dp, dp, dp]),
            "mc3d_solver_set_mesh": (ip, [vp, C.POINTER(dp), C.POINTER(dp), C.POINTER(dp)]),
            "mc3d_solver_get_metrics": (ip, [vp, C.POINTER(C.POINTER(dp))]),
            "mc3d_dump_read_header": (ip, [C.c_char_p, C.POINTER(ip), C.POINTER(dp), C.POINTER(ip), C.POINTER(ip),
                                           C.POINTER(ip)]),
            "mc3d_dump_read_fields": (ip, [C.c_char_p, C.c_longlong, C.POINTER(C.POINTER(dp))]),
            "mc3d_dump_write": (ip, [C.c_char_p, ip, dp, ip, ip, ip, C.POINTER(C.POINTER(dp))]),
            "mc3d_solver_dump": (ip, [vp, C.c_char_p, C.POINTER(dp), C.POINTER(dp), C.POINTER(dp)]),
            "mc3d_solver_restart": (ip, [vp, C.c_char_p, ip]),
            "mc3d_solver_dump_sponge_avg": (ip, [vp, C.c_char_p]),
            "mc3d_solver_read_sponge_avg": (ip, [vp, C.c_char_p]),
            "mc3d_solver_start": (ip, [vp]),
            "mc3d_solver_get_stats": (ip, [vp, C.POINTER(C.POINTER(dp)), C.POINTER(C.POINTER(dp)), C.POINTER(dp)]),
            "mc3d_solver_dump_stats": (ip, [vp, C.c_char_p, C.c_char_p]),
            "mc3d_solver_turbdata": (ip, [vp, dp, C.POINTER(dp)]),
            "mc3d_solver_wall_span_average": (ip, [vp] + [C.POINTER(dp)] * 4),
            "mc3d_solver_wake_strip": (ip, [vp, C.c_int, C.c_int, C.POINTER(dp)]),
            "mc3d_tma_wait_timeouts": (ip, [C.c_int, C.POINTER(C.c_int)]),
            "mc3d_solver_read_stats": (ip, [vp, C.c_char_p, C.c_char_p]),
            "mc3d_solver_run": (ip, [vp, C.c_char_p]),
            "mc3d_solver_set_initial": (ip, [vp] + [C.POINTER(dp)] * 5),
            "mc3d_solver_set_initial_device": (ip, [vp] + [vp] * 5),
            "mc3d_solver_step": (ip, [vp, ip]),
            "mc3d_solver_pre_step": (ip, [vp]),
            "mc3d_solver_stage_count": (ip, [vp, C.POINTER(ip)]),
            "mc3d_solver_pre_substep": (ip, [vp, ip]),
            "mc3d_solver_solve_eqn_set": (ip, [vp]),
            "mc3d_solver_post_substep": (ip, [vp]),
            "mc3d_rk_update": (ip, [vp, ip, ip, ip]),
            "mc3d_solver_update_data": (ip, [vp, ip]),
            "mc3d_solver_post_step": (ip, [vp]),
            "mc3d_solver_get_conserved": (ip, [vp] + [C.POINTER(dp)] * 5),
            "mc3d_solver_conserved_device": (ip, [vp, C.POINTER(vp)]),
            "mc3d_solver_info": (ip, [vp, C.POINTER(ip), C.POINTER(dp), C.POINTER(dp), C.POINTER(C.c_longlong)]),
            "mc3d_solver_integrals": (ip, [vp, C.POINTER(dp), C.POINTER(dp)]),
            "mc3d_solver_stream": (ip, [vp, C.POINTER(vp)]),
            "mc3d_solver_set_stream": (ip, [vp, vp]),
            "mc3d_solver_launch_count": (ip, [vp, C.POINTER(C.c_longlong)]),
            "mc3d_solver_sync": (ip, [vp]),
            "mc3d_solver_set_timing": (ip, [vp, ip]),
            "mc3d_solver_timing_report": (C.c_char_p, [vp]),
            "mc3d_hit_randvec": (ip, [C.POINTER(C.c_int), C.POINTER(dp), C.c_longlong, C.POINTER(dp)]),
            "mc3d_cfl_max_noalloc": (ip, [vp] * 8 + [dp] * 3 + [ip] * 3 + [dp] * 3 + [vp, vp]),
            "mc3d_sponge_sigma": (ip, [C.POINTER(Config)] + [C.POINTER(dp)] * 4),
            "mc3d_mlp_create": (ip, [C.c_ulonglong, ip, C.POINTER(vp)]),
            "mc3d_mlp_destroy": (ip, [vp]),
            "mc3d_mlp_set_normalization": (ip, [vp] + [C.POINTER(C.c_float)] * 6),
            "mc3d_mlp_get_normalization": (ip, [vp, C.POINTER(C.c_float)]),
            "mc3d_mlp_train_step": (ip, [vp, vp, vp, ip, C.c_float, C.POINTER(dp), vp]),
            "mc3d_mlp_forward": (ip, [vp, vp, vp, ip, vp]),
            "mc3d_mlp_gradient": (ip, [vp, vp, vp, ip, C.POINTER(C.c_float), C.POINTER(dp), vp]),
            "mc3d_mlp_infer_bf16": (ip, [vp, vp, vp, ip, vp]),
            "mc3d_mlp_get_params": (ip, [vp, C.POINTER(C.c_float)]),
            "mc3d_mlp_set_params": (ip, [vp, C.POINTER(C.c_float)]),
            "mc3d_mlp_save": (ip, [vp, C.c_char_p]),
            "mc3d_mlp_load": (ip, [vp, C.c_char_p]),
            "mc3d_sgs_box_filter": (ip, [C.POINTER(vp), ip, ip, ip, ip, C.POINTER(vp), vp]),
            "mc3d_sgs_training_pairs": (ip, [C.POINTER(vp), C.POINTER(vp), ip, ip, ip, C.POINTER(dp), dp, dp,
                                             vp, vp, vp]),
            "mc3d_solver_set_mlp": (ip, [vp, vp]),
            "mc3d_solver_copy_conserved_device": (ip, [vp, C.POINTER(vp)]),
            "mc3d_solver_mlp_fallbacks": (ip, [vp, C.POINTER(C.c_longlong)]),
            "mc3d_solver_set_sponge": (ip, [vp, C.POINTER(dp)]),
            "mc3d_sgs_create": (ip, [ip, ip, ip, ip, ip, ip, ip, C.POINTER(ip), C.POINTER(dp), vp, dp, ip, ip,
                                     C.POINTER(vp)]),
            "mc3d_sgs_destroy": (ip, [vp]),
            "mc3d_sgs_get_viscosity": (ip, [vp, C.POINTER(vp), C.POINTER(vp), vp, vp]),
            "mc3d_sgs_calc_mu_taukk": (ip, [vp, C.POINTER(vp), C.POINTER(vp), vp, vp, vp]),
            "mc3d_sgs_calc_ksgs": (ip, [vp, C.POINTER(vp), C.POINTER(vp), vp, vp, vp]),
            "mc3d_sgs_set_mlp": (ip, [vp, vp, dp]),
            "mc3d_sgs_mlp_out_of_range": (ip, [vp, C.POINTER(C.c_longlong)]),
            "mc3d_solver_set_sponge_avg": (ip, [vp, C.POINTER(C.POINTER(dp))]),
        }
        for name, (res, args) in sigs.items():
            f = getattr(lib, name)
            f.restype = res
            f.argtypes = args
        _lib = lib
    return _lib


def header_functions():
    """Names of every function include/mc3d.h declares."""
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(mc3d_[a-z0-9_]+)\s*\(", txt)))


def check(rc):
    if rc != MC3D_OK:
        raise Mc3dError(rc, host_lib().mc3d_last_error().decode(errors="replace"))


def dptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_double))


def hit_randvec(lib, gen, n):
    """Fast path of the HIT generator's randvec (same sequence as the Python loop)."""
    st = (C.c_int * 3)(gen.ix1, gen.ix2, gen.ix3)
    tab = np.array(gen.r, dtype=np.float64)
    out = np.empty(n, dtype=np.float64)
    check(lib.mc3d_hit_randvec(st, dptr(tab), n, dptr(out)))
    gen.ix1, gen.ix2, gen.ix3 = st[0], st[1], st[2]
    gen.r = tab.tolist()
    return out
