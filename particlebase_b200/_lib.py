"""ctypes loader for ``libparticlebase_b200.so`` (the C ABI in include/pb/pb.h).

There is no CPU fallback: if the library is missing or cannot be loaded the
import fails with an error that says how to build it.
"""
from __future__ import annotations

import ctypes as C
import os

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "lib", "libparticlebase_b200.so")

PB_OK = 0
ERRORS = {
    1: "PB_ERR_ARG", 2: "PB_ERR_CUDA", 3: "PB_ERR_STATE", 4: "PB_ERR_NOCONVERGE",
    5: "PB_ERR_UNSUPPORTED", 6: "PB_ERR_OOM", 7: "PB_ERR_DEVICE", 8: "PB_ERR_NOTFOUND",
}

# pb_field
FIELD = {
    "r": 0, "v": 1, "vd": 2, "F": 3, "Fold": 4, "minv": 5, "type": 6, "cell_of": 7,
    "pid": 8, "cell_start": 9, "cell_key": 10, "neighbors": 11, "r_sorted": 12, "mass": 13,
}

VEL_FP64 = 0x1
ACC_FP64 = 0x2
HALF_SHELL = 0x4
FORCE_ENERGY = 0x1
MODE_VV = 0
MODE_GAUSS = 1


class PBError(RuntimeError):
    def __init__(self, code: int, what: str, detail: str = ""):
        super().__init__(f"{what} failed: {ERRORS.get(code, code)} {detail}".strip())
        self.code = code


class pb_particle(C.Structure):
    """Binary image of the reference's ParticleBase (ParticleBase.hh:10-18)."""

    _fields_ = [("r", C.c_double * 3), ("m", C.c_double), ("v", C.c_double * 3),
                ("is_fixed", C.c_uint8), ("a", C.c_double * 3), ("type", C.c_uint32)]


class pb_srv_config(C.Structure):
    _fields_ = [("hbm_budget", C.c_size_t), ("max_atoms", C.c_uint64), ("max_jobs", C.c_uint32),
                ("chunk_ms", C.c_float), ("flags", C.c_uint32), ("mode", C.c_int),
                ("force_threads", C.c_int), ("seg_scale", C.c_float),
                ("reserve_bytes", C.c_size_t)]


class pb_srv_job(C.Structure):
    _fields_ = [("natoms", C.c_uint32), ("cell6", C.c_float * 6), ("rc", C.c_float),
                ("sigma_eps", C.c_void_p), ("sigma_eps_rc", C.c_void_p), ("ntypes", C.c_uint32),
                ("dt", C.c_float), ("kB", C.c_float), ("steps", C.c_uint32),
                ("r3", C.c_void_p), ("v3", C.c_void_p), ("mass", C.c_void_p),
                ("type", C.c_void_p)]


class pb_srv_job_info(C.Structure):
    _fields_ = [("id", C.c_uint64), ("state", C.c_int), ("natoms", C.c_uint32),
                ("steps", C.c_uint32), ("t_submit", C.c_double), ("t_admit", C.c_double),
                ("t_done", C.c_double), ("device_status", C.c_uint32)]


class pb_srv_stats(C.Structure):
    _fields_ = [("submitted", C.c_uint64), ("done", C.c_uint64), ("failed", C.c_uint64),
                ("rejected", C.c_uint64), ("atom_steps", C.c_double),
                ("gpu_seconds", C.c_double), ("repack_seconds", C.c_double),
                ("chunks", C.c_uint64), ("repacks", C.c_uint64), ("peak_jobs", C.c_uint64),
                ("peak_atoms", C.c_uint64), ("peak_bytes", C.c_size_t)]


class pb_md_sums(C.Structure):
    _fields_ = [("mv2", C.c_double), ("fv", C.c_double), ("pe", C.c_double),
                ("pe_shift", C.c_double), ("virial", C.c_double), ("xi", C.c_double)]


_lib = None


def _declare(L: C.CDLL) -> None:
    vp, u32, f32, f64, i32 = C.c_void_p, C.c_uint32, C.c_float, C.c_double, C.c_int
    sig = {
        "pb_md_create": [u32, u32, C.POINTER(vp)],
        "pb_md_destroy": [vp],
        "pb_md_set_stream": [vp, vp],
        "pb_md_status": [vp, C.POINTER(u32)],
        "pb_md_set_cell": [vp, C.POINTER(f32)],
        "pb_md_set_lj": [vp, C.POINTER(f32), u32],
        "pb_md_set_lj_cut": [vp, C.POINTER(f32), u32],
        "pb_md_set_rmax2": [vp, f32],
        "pb_md_set_kB": [vp, f32],
        "pb_md_import": [vp, C.POINTER(pb_particle), u32],
        "pb_md_import_arrays": [vp, vp, vp, vp, vp],
        "pb_md_setup_cells": [vp, f32, i32],
        "pb_md_grid": [vp, C.POINTER(u32), C.POINTER(f32), C.POINTER(u32)],
        "pb_md_build_cells": [vp],
        "pb_md_force": [vp, u32],
        "pb_md_use_nlist": [vp, f32],
        "pb_md_make_nlist": [vp],
        "pb_md_nlist_info": [vp, C.POINTER(f64)],
        "pb_md_gr": [vp, f32, f32, vp, C.POINTER(u32)],
        "pb_md_clear_force": [vp],
        "pb_md_step_vv": [vp, f32],
        "pb_md_step_gauss": [vp, f32, f64],
        "pb_md_wrap": [vp],
        "pb_md_run": [vp, f32, i32, u32],
        "pb_md_run_timed": [vp, f32, i32, u32, C.POINTER(f32)],
        "pb_md_reduce": [vp, C.POINTER(pb_md_sums)],
        "pb_md_temperature": [vp, C.POINTER(f64)],
        "pb_md_scale_velocities": [vp, f64],
        "pb_md_adjust_velocities": [vp, f64],
        "pb_md_mean_mass": [vp, C.POINTER(f64)],
        "pb_md_correct_force": [vp, f64],
        "pb_md_set_xi": [vp, f64],
        "pb_md_minimize": [vp, u32, f32, f32],
        "pb_md_force_softcore": [vp, f32, f32],
        "pb_md_step_euler": [vp, f32],
        "pb_md_force_wait_test": [vp, u32],
        "pb_md_get": [vp, i32, vp, C.c_size_t],
        "pb_md_set": [vp, i32, vp, C.c_size_t],
        "pb_md_field_bytes": [vp, i32, C.POINTER(C.c_size_t)],
        "pb_md_size": [vp, C.POINTER(u32)],
        "pb_md_profile": [vp, f32, i32, u32, C.POINTER(f64)],
        "pb_md_pair_stats": [vp, C.POINTER(f64)],
        "pb_md_cell_build_kernels": [vp, C.POINTER(u32)],
        "pb_peak_fp32": [C.POINTER(f64)],
        "pb_cells_build_noalloc": [vp, vp, u32, C.POINTER(f32), f32, vp, vp, vp, vp, vp],
        "pb_cells_build_noalloc_limits": [C.POINTER(u32), C.POINTER(u32), C.POINTER(C.c_size_t)],
        "pb_plan_grid": [C.POINTER(f32), f32, C.POINTER(u32), C.POINTER(f32)],
        "pb_plan_columns": [u32, u32, C.POINTER(u32)],
        "pb_batch_create": [vp, u32, u32, C.POINTER(vp)],
        "pb_batch_repack": [vp, vp, vp, u32, C.POINTER(vp)],
        "pb_batch_destroy": [vp],
        "pb_batch_set_stream": [vp, vp],
        "pb_batch_size": [vp, C.POINTER(u32), C.POINTER(u32), vp],
        "pb_batch_set_system": [vp, u32, C.POINTER(f32), f32, C.POINTER(f32), u32, f32, f32],
        "pb_batch_set_lj_cut": [vp, u32, C.POINTER(f32), u32],
        "pb_batch_import": [vp, u32, vp, vp, vp, vp],
        "pb_batch_setup_cells": [vp, vp],
        "pb_batch_force": [vp, u32],
        "pb_batch_clear_force": [vp],
        "pb_batch_run": [vp, i32, u32],
        "pb_batch_run_timed": [vp, i32, u32, C.POINTER(f32)],
        "pb_batch_profile": [vp, i32, u32, C.POINTER(f64)],
        "pb_batch_set_steps_left": [vp, vp],
        "pb_batch_get_steps_left": [vp, vp],
        "pb_batch_reduce": [vp, vp],
        "pb_batch_temperature": [vp, vp],
        "pb_batch_status": [vp, vp],
        "pb_batch_scale_velocities": [vp, vp],
        "pb_batch_adjust_velocities": [vp, vp],
        "pb_batch_get": [vp, u32, i32, vp, C.c_size_t],
        "pb_batch_set": [vp, u32, i32, vp, C.c_size_t],
        "pb_batch_set_tuning": [vp, i32, f32],
        "pb_batch_estimate_bytes": [vp, vp, vp, u32, u32, C.POINTER(C.c_size_t)],
        "pb_srv_create": [C.POINTER(pb_srv_config), C.POINTER(vp)],
        "pb_srv_destroy": [vp],
        "pb_srv_submit": [vp, C.POINTER(pb_srv_job), C.POINTER(C.c_uint64)],
        "pb_srv_wait": [vp, C.c_uint64, f64],
        "pb_srv_drain": [vp, f64],
        "pb_srv_poll": [vp, vp, u32, C.POINTER(u32)],
        "pb_srv_info": [vp, C.c_uint64, C.POINTER(pb_srv_job_info)],
        "pb_srv_result": [vp, C.c_uint64, vp, vp, C.c_size_t, vp],
        "pb_srv_release": [vp, C.c_uint64],
        "pb_srv_stats_get": [vp, C.POINTER(pb_srv_stats)],
        "pb_pool_reserve": [C.c_size_t],
        "pb_pool_trim": [],
    }
    for name, args in sig.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = C.c_int
    L.pb_md_last_error.argtypes = [vp]
    L.pb_md_last_error.restype = C.c_char_p
    L.pb_batch_last_error.argtypes = [vp]
    L.pb_batch_last_error.restype = C.c_char_p
    L.pb_srv_last_error.argtypes = [vp]
    L.pb_srv_last_error.restype = C.c_char_p
    L.pb_srv_now.argtypes = [vp]
    L.pb_srv_now.restype = C.c_double
    L.pb_version.restype = C.c_char_p


def lib() -> C.CDLL:
    """Load the CUDA library (fails loudly when it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python -m particlebase_b200.build`")
        L = C.CDLL(LIB_PATH)
        _declare(L)
        _lib = L
    return _lib


def check(code: int, what: str, handle=None, batch: bool = False) -> None:
    if code != PB_OK:
        detail = ""
        if handle is not None:
            err = lib().pb_batch_last_error if batch else lib().pb_md_last_error
            detail = err(handle).decode(errors="replace")
        raise PBError(code, what, detail)
