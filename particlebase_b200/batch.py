"""Many independent LJ systems advanced together (a pb_batch handle).

No counterpart in the reference, which runs one system per process
(testMD2.cu:88-189).  Every system of a batch is computed exactly as an
``MDSystem`` computes it alone: same cell list, same force and integration
arithmetic, per-system FP64 sums in the same order, so its trajectory is
bit-identical alone and in any batch (for the same force launch tuning).

    b = Batch.from_systems(systems, gaussian=True, dt=0.005)
    b.run(100)                      # one CUDA graph per 2 steps, all systems
    T = b.temperatures()            # per-system calcTemp
    r3 = b.get(7, "r")              # positions of system 7
"""
from __future__ import annotations

import ctypes as C
from typing import Sequence

import numpy as np

from . import _lib as L
from .md import MDSystem, _fptr
from .workloads import LJSystem


class Batch:
    _DTYPES = {"r": (np.float32, 4), "v": (np.float32, 4), "vd": (np.float64, 1),
               "F": (np.float32, 4), "Fold": (np.float32, 4), "minv": (np.float32, 1),
               "mass": (np.float32, 1), "type": (np.uint16, 1)}
    _WIDTH = {"r": 16, "v": 16, "vd": 24, "F": 16, "Fold": 16, "minv": 4, "mass": 4, "type": 2}

    def __init__(self, natoms: Sequence[int], gaussian: bool = False,
                 fp64_velocities: bool | None = None, fp64_forces: bool = False,
                 _handle: C.c_void_p | None = None, half_shell: bool = False):
        self.lib = L.lib()
        self.gaussian = bool(gaussian)
        if fp64_velocities is None:
            fp64_velocities = self.gaussian
        self.fp64_velocities = bool(fp64_velocities)
        self.flags = ((L.VEL_FP64 if fp64_velocities else 0) | (L.ACC_FP64 if fp64_forces else 0) |
                      (L.HALF_SHELL if half_shell else 0))
        if _handle is None:
            n = np.ascontiguousarray(np.asarray(natoms, np.uint32))
            h = C.c_void_p()
            L.check(self.lib.pb_batch_create(_fptr(n), len(n), self.flags, C.byref(h)),
                    "pb_batch_create")
            self.h = h
        else:
            self.h = _handle
        ns, nt = C.c_uint32(), C.c_uint32()
        self._ck(self.lib.pb_batch_size(self.h, C.byref(ns), C.byref(nt), None), "size")
        self.nsys, self.total = int(ns.value), int(nt.value)
        a0 = np.empty(self.nsys + 1, np.uint32)
        self._ck(self.lib.pb_batch_size(self.h, None, None, _fptr(a0)), "size")
        self.atom0 = a0.astype(np.int64)
        self.natoms = np.diff(self.atom0)
        self.kB = np.ones(self.nsys)

    # ---------------------------------------------------------------- lifetime
    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.pb_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _ck(self, code: int, what: str) -> None:
        L.check(code, what, self.h, batch=True)

    @property
    def mode(self) -> int:
        return L.MODE_GAUSS if self.gaussian else L.MODE_VV

    # ---------------------------------------------------------------- set-up
    def set_system(self, k: int, box, rc: float, sigma_eps, ntypes: int, dt: float,
                   kB: float = 1.0) -> None:
        c = np.ascontiguousarray(np.asarray(box, np.float32).reshape(6))
        p = np.ascontiguousarray(np.asarray(sigma_eps, np.float32).reshape(-1))
        self._ck(self.lib.pb_batch_set_system(
            self.h, int(k), c.ctypes.data_as(C.POINTER(C.c_float)), C.c_float(rc),
            p.ctypes.data_as(C.POINTER(C.c_float)), int(ntypes), C.c_float(dt),
            C.c_float(kB)), "set_system")
        self.kB[k] = kB

    def set_lj_cut(self, k: int, params, ntypes: int) -> None:
        p = np.ascontiguousarray(np.asarray(params, np.float32).reshape(-1))
        self._ck(self.lib.pb_batch_set_lj_cut(self.h, int(k),
                                              p.ctypes.data_as(C.POINTER(C.c_float)),
                                              int(ntypes)), "set_lj_cut")

    def import_arrays(self, k: int, r, v=None, mass=None, types=None) -> None:
        r = np.ascontiguousarray(np.asarray(r, np.float64)[:, :3])
        keep, args = [r], [_fptr(r)]
        for a, dt in ((v, np.float64), (mass, np.float64), (types, np.uint32)):
            if a is None:
                args.append(None)
                continue
            a = np.ascontiguousarray(np.asarray(a, dt))
            if dt is np.float64 and a.ndim == 2:
                a = np.ascontiguousarray(a[:, :3])
            keep.append(a)
            args.append(_fptr(a))
        self._ck(self.lib.pb_batch_import(self.h, int(k), *args), "import")

    def add_system(self, k: int, s: LJSystem, dt: float) -> None:
        """set_system + import of a host LJSystem (per-pair cutoffs when it has them)."""
        self.set_system(k, s.box, float(s.rc), s.lj[..., :2].reshape(-1), s.ntypes, dt)
        if not np.allclose(s.lj[..., 2], s.rc):
            self.set_lj_cut(k, s.lj.reshape(-1), s.ntypes)
        self.import_arrays(k, s.r, s.v, s.mass, s.types)

    def setup_cells(self, rmax=None) -> None:
        if rmax is None:
            self._ck(self.lib.pb_batch_setup_cells(self.h, None), "setup_cells")
        else:
            r = np.ascontiguousarray(np.asarray(rmax, np.float32))
            self._ck(self.lib.pb_batch_setup_cells(self.h, _fptr(r)), "setup_cells")

    def set_tuning(self, force_threads: int = 256, seg_scale: float = 1.0) -> None:
        self._ck(self.lib.pb_batch_set_tuning(self.h, int(force_threads), C.c_float(seg_scale)),
                 "set_tuning")

    @classmethod
    def from_systems(cls, systems: Sequence[LJSystem], gaussian: bool = False, dt: float = 0.005,
                     fp64_velocities: bool | None = None, fp64_forces: bool = False,
                     tuning: tuple[int, float] | None = None,
                     half_shell: bool = False) -> "Batch":
        b = cls([s.n for s in systems], gaussian, fp64_velocities, fp64_forces,
                half_shell=half_shell)
        dts = np.broadcast_to(np.asarray(dt, np.float64), (len(systems),))
        for k, s in enumerate(systems):
            b.add_system(k, s, float(dts[k]))
        if tuning is not None:
            b.set_tuning(*tuning)
        b.setup_cells()
        return b

    def repack(self, src: Sequence[int], new_systems: dict[int, LJSystem] | None = None,
               dt: float = 0.005) -> "Batch":
        """New batch: slot k continues system src[k] of this batch, or (src[k] < 0)
        takes new_systems[k].  Cells are set up; this batch stays valid."""
        new_systems = new_systems or {}
        src_a = np.ascontiguousarray(np.asarray(src, np.int32))
        nat = np.zeros(len(src_a), np.uint32)
        for k, s in enumerate(src_a):
            if s < 0:
                nat[k] = new_systems[k].n
        h = C.c_void_p()
        self._ck(self.lib.pb_batch_repack(self.h, _fptr(src_a), _fptr(nat), len(src_a),
                                          C.byref(h)), "repack")
        out = Batch(nat, self.gaussian, self.fp64_velocities, bool(self.flags & L.ACC_FP64),
                    _handle=h, half_shell=bool(self.flags & L.HALF_SHELL))
        for k, s in enumerate(src_a):
            if s >= 0:
                out.kB[k] = self.kB[s]
            else:
                out.add_system(k, new_systems[k], dt)
        out.setup_cells()
        return out

    # ---------------------------------------------------------------- stepping
    def force(self, energy: bool = False) -> None:
        self._ck(self.lib.pb_batch_force(self.h, L.FORCE_ENERGY if energy else 0), "force")

    def clear_force(self) -> None:
        self._ck(self.lib.pb_batch_clear_force(self.h), "clear_force")

    def run(self, steps: int) -> None:
        self._ck(self.lib.pb_batch_run(self.h, self.mode, int(steps)), "run")

    def run_timed(self, steps: int) -> float:
        ms = C.c_float()
        self._ck(self.lib.pb_batch_run_timed(self.h, self.mode, int(steps), C.byref(ms)),
                 "run_timed")
        return float(ms.value)

    def profile(self, steps: int) -> dict:
        ms = (C.c_double * 3)()
        self._ck(self.lib.pb_batch_profile(self.h, self.mode, int(steps), ms), "profile")
        return {"cells": ms[0], "force": ms[1], "evolve": ms[2]}

    def set_steps_left(self, steps) -> None:
        """Per-system step budgets (None removes them): system k stops after
        steps[k] more steps while the others continue."""
        if steps is None:
            self._ck(self.lib.pb_batch_set_steps_left(self.h, None), "set_steps_left")
            return
        s = np.ascontiguousarray(np.broadcast_to(np.asarray(steps, np.uint32), (self.nsys,)))
        self._ck(self.lib.pb_batch_set_steps_left(self.h, _fptr(s)), "set_steps_left")

    def steps_left(self) -> np.ndarray:
        s = np.empty(self.nsys, np.uint32)
        self._ck(self.lib.pb_batch_get_steps_left(self.h, _fptr(s)), "get_steps_left")
        return s

    # ---------------------------------------------------------------- reductions
    def sums(self) -> np.ndarray:
        out = (L.pb_md_sums * self.nsys)()
        self._ck(self.lib.pb_batch_reduce(self.h, out), "reduce")
        names = [k for k, _ in L.pb_md_sums._fields_]
        return np.array([[getattr(o, k) for k in names] for o in out])

    def temperatures(self) -> np.ndarray:
        t = np.empty(self.nsys, np.float64)
        self._ck(self.lib.pb_batch_temperature(self.h, _fptr(t)), "temperature")
        return t

    def status(self) -> np.ndarray:
        b = np.empty(self.nsys, np.uint32)
        self._ck(self.lib.pb_batch_status(self.h, _fptr(b)), "status")
        return b

    def scale_velocities(self, s) -> None:
        f = np.ascontiguousarray(np.broadcast_to(np.asarray(s, np.float64), (self.nsys,)))
        self._ck(self.lib.pb_batch_scale_velocities(self.h, _fptr(f)), "scale")

    def adjust_velocities(self, v1) -> None:
        f = np.ascontiguousarray(np.broadcast_to(np.asarray(v1, np.float64), (self.nsys,)))
        self._ck(self.lib.pb_batch_adjust_velocities(self.h, _fptr(f)), "adjust")

    # ---------------------------------------------------------------- state
    def get(self, k: int, field: str) -> np.ndarray:
        dt, width = self._DTYPES[field]
        n = int(self.natoms[k])
        nbytes = self._WIDTH[field] * n
        out = np.empty(nbytes // np.dtype(dt).itemsize, dt)
        self._ck(self.lib.pb_batch_get(self.h, int(k), L.FIELD[field], _fptr(out), nbytes),
                 "get " + field)
        if field == "vd":
            return out.reshape(3, -1).T.copy()
        return out.reshape(-1, width) if width > 1 else out

    def set(self, k: int, field: str, arr) -> None:
        dt, _ = self._DTYPES[field]
        a = np.asarray(arr, dt)
        if field == "vd":
            a = a.reshape(-1, 3).T
        a = np.ascontiguousarray(a).reshape(-1)
        self._ck(self.lib.pb_batch_set(self.h, int(k), L.FIELD[field], _fptr(a), a.nbytes),
                 "set " + field)

    def velocities(self, k: int) -> np.ndarray:
        if self.fp64_velocities:
            return self.get(k, "vd")
        return self.get(k, "v")[:, :3].astype(np.float64)

    @staticmethod
    def estimate_bytes(systems: Sequence[LJSystem], fp64_velocities: bool = False) -> int:
        nat = np.ascontiguousarray([s.n for s in systems], np.uint32)
        cells = np.ascontiguousarray(np.stack([s.box for s in systems]).astype(np.float32))
        rmax = np.ascontiguousarray([s.rc for s in systems], np.float32)
        out = C.c_size_t()
        L.check(L.lib().pb_batch_estimate_bytes(_fptr(nat), _fptr(cells), _fptr(rmax), len(nat),
                                                L.VEL_FP64 if fp64_velocities else 0,
                                                C.byref(out)), "estimate_bytes")
        return int(out.value)


def alone(s: LJSystem, gaussian: bool, dt: float, fp64_velocities: bool | None = None,
          tuning: tuple[int, float] | None = None) -> "Batch":
    """A one-system batch (the reference point of the alone-versus-batched checks)."""
    return Batch.from_systems([s], gaussian=gaussian, dt=dt, fp64_velocities=fp64_velocities,
                              tuning=tuning)


__all__ = ["Batch", "MDSystem", "alone"]
