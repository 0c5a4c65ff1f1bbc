"""Python mirror of the reference's MD classes over the C ABI.

``MDSystem`` carries the method names of cudaParticleMD / cudaParticleVV /
GaussianThermo (cudaParticleMD.hh:32-194, cudaParticleVV.hh:14-57,
GaussianThermo.hh:14-90) so that tests and benchmarks read like the
reference's drivers (testMD2.cu:88-189):

    p = MDSystem(n, gaussian=True)
    p.setCell(cell); p.rmax2 = 2.5 ** 2; p.import_(particles)
    p.setLJparams([1.0, 1.0], 1); p.setupCutoffBlock(2.5)
    p.calcBlockID(); p.clearForce()
    for step in range(steps):
        p.calcBlockID(); p.calcForce(); t = p.calcTemp()
        p.TimeEvolution(dt); p.treatPeriodicCondition()

All computation runs in libparticlebase_b200.so on the current CUDA device.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L
from .workloads import LJSystem


def _fptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


class MDSystem:
    """One periodic LJ system resident on the GPU (a pb_md handle)."""

    def __init__(self, n: int, gaussian: bool = False, fp64_velocities: bool | None = None,
                 fp64_forces: bool = False, half_shell: bool = False):
        self.lib = L.lib()
        self.n = int(n)
        self.gaussian = bool(gaussian)
        if fp64_velocities is None:
            fp64_velocities = self.gaussian  # GaussianThermo keeps FP64 velocities (vd)
        flags = ((L.VEL_FP64 if fp64_velocities else 0) | (L.ACC_FP64 if fp64_forces else 0) |
                 (L.HALF_SHELL if half_shell else 0))
        self.fp64_velocities = bool(fp64_velocities)
        h = C.c_void_p()
        L.check(self.lib.pb_md_create(self.n, flags, C.byref(h)), "pb_md_create")
        self.h = h
        self._kB = 1.0
        self._rmax2 = 0.0
        self._e = 1e-8
        self.timestep = 0
        self.mv2 = 0.0
        self.cell = np.zeros(6, np.float32)

    # ---------------------------------------------------------------- lifetime
    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.pb_md_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _ck(self, code: int, what: str) -> None:
        L.check(code, what, self.h)

    # ---------------------------------------------------------------- set-up
    @property
    def kB(self) -> float:
        return self._kB

    @kB.setter
    def kB(self, value: float) -> None:
        self._kB = float(value)
        self._ck(self.lib.pb_md_set_kB(self.h, C.c_float(value)), "set_kB")

    @property
    def rmax2(self) -> float:
        return self._rmax2

    @rmax2.setter
    def rmax2(self, value: float) -> None:
        self._rmax2 = float(value)
        self._ck(self.lib.pb_md_set_rmax2(self.h, C.c_float(value)), "set_rmax2")

    def setE(self, e: float) -> None:
        """GaussianThermo::setE: Newton-Raphson tolerance (kept for parity)."""
        self._e = float(e)

    def setCell(self, cell) -> None:
        c = np.ascontiguousarray(np.asarray(cell, np.float32).reshape(6))
        self.cell = c.copy()
        self._ck(self.lib.pb_md_set_cell(self.h, c.ctypes.data_as(C.POINTER(C.c_float))),
                 "set_cell")

    def setLJparams(self, params, elemnum: int) -> None:
        p = np.ascontiguousarray(np.asarray(params, np.float32).reshape(-1))
        self._ck(self.lib.pb_md_set_lj(self.h, p.ctypes.data_as(C.POINTER(C.c_float)), elemnum),
                 "set_lj")

    def setLJparamsCut(self, params, elemnum: int) -> None:
        """Extension: (sigma, epsilon, rc) per type pair."""
        p = np.ascontiguousarray(np.asarray(params, np.float32).reshape(-1))
        self._ck(self.lib.pb_md_set_lj_cut(self.h, p.ctypes.data_as(C.POINTER(C.c_float)),
                                           elemnum), "set_lj_cut")

    def import_(self, particles) -> None:
        """cudaParticleMD::import + setM from a list of pb_particle records."""
        arr = (L.pb_particle * self.n)(*particles)
        self._ck(self.lib.pb_md_import(self.h, arr, self.n), "import")

    def import_arrays(self, r, v=None, mass=None, types=None) -> None:
        r = np.ascontiguousarray(np.asarray(r, np.float64)[:, :3])
        keep = [r]
        args = [_fptr(r)]
        for a, dt in ((v, np.float64), (mass, np.float64), (types, np.uint32)):
            if a is None:
                args.append(None)
            else:
                a = np.ascontiguousarray(np.asarray(a, dt))
                if dt is np.float64 and a.ndim == 2:
                    a = np.ascontiguousarray(a[:, :3])
                keep.append(a)
                args.append(_fptr(a))
        self._ck(self.lib.pb_md_import_arrays(self.h, *args), "import_arrays")

    def setM(self) -> None:
        """m = 1/minv is computed at import; kept for interface parity."""

    def setupCutoffBlock(self, rmax: float, periodic: bool = True) -> None:
        self._ck(self.lib.pb_md_setup_cells(self.h, C.c_float(rmax), int(periodic)),
                 "setup_cells")

    def grid(self):
        n = (C.c_uint32 * 3)()
        ln = (C.c_float * 3)()
        nc = C.c_uint32()
        self._ck(self.lib.pb_md_grid(self.h, n, ln, C.byref(nc)), "grid")
        return np.array(n[:], np.uint32), np.array(ln[:], np.float32), int(nc.value)

    def numBlocks(self) -> int:
        return self.grid()[2]

    # ---------------------------------------------------------------- the step
    def calcBlockID(self) -> None:
        self._ck(self.lib.pb_md_build_cells(self.h), "build_cells")

    def calcForce(self, energy: bool = False) -> None:
        self._ck(self.lib.pb_md_force(self.h, L.FORCE_ENERGY if energy else 0), "force")

    def useNList(self, thickness: float) -> None:
        """cudaParticleMD::useNList with `thickness` (cudaParticleMD.hh:167-179):
        force calls use a Verlet list of the atoms within rc + thickness,
        rebuilt by makeNList; thickness < 0 turns it off."""
        self._ck(self.lib.pb_md_use_nlist(self.h, C.c_float(thickness)), "use_nlist")

    def makeNList(self) -> None:
        """cudaParticleMD::makeNList (cudaParticleMD.cu:338-394): cell list and
        neighbour list rebuilt from the current positions."""
        self._ck(self.lib.pb_md_make_nlist(self.h), "make_nlist")

    def nlist_info(self) -> dict:
        out = (C.c_double * 3)()
        self._ck(self.lib.pb_md_nlist_info(self.h, out), "nlist_info")
        return {"mean": out[0], "max": out[1], "capacity": out[2]}

    def gr_counts(self, rstep: float, rmax: float) -> np.ndarray:
        """cudaCalcGR::calcgr: counts of the unordered pairs of the current
        positions per distance bin (bin j = round(r / rstep), 0 < j < rnum)."""
        n = C.c_uint32()
        self._ck(self.lib.pb_md_gr(self.h, C.c_float(rstep), C.c_float(rmax), None,
                                   C.byref(n)), "gr")
        out = np.zeros(n.value, np.uint64)
        self._ck(self.lib.pb_md_gr(self.h, C.c_float(rstep), C.c_float(rmax),
                                   out.ctypes.data_as(C.c_void_p), C.byref(n)), "gr")
        return out

    def force_wait_test(self, polls: int = 2000) -> None:
        """Failure-detection test hook: one force call whose hand-off wait is
        made to run out (pb_md_force_wait_test); raises nothing, sets
        PB_STATUS_WAIT_TIMEOUT in the status word."""
        self._ck(self.lib.pb_md_force_wait_test(self.h, int(polls)), "force_wait_test")

    def clearForce(self) -> None:
        self._ck(self.lib.pb_md_clear_force(self.h), "clear_force")

    def TimeEvolution(self, dt: float) -> None:
        if self.gaussian:
            self._ck(self.lib.pb_md_step_gauss(self.h, C.c_float(dt), C.c_double(self._e)),
                     "step_gauss")
        else:
            self._ck(self.lib.pb_md_step_vv(self.h, C.c_float(dt)), "step_vv")

    def treatPeriodicCondition(self) -> None:
        self._ck(self.lib.pb_md_wrap(self.h), "wrap")

    def run(self, dt: float, steps: int) -> None:
        """Whole steps (cells, force, evolution + wrap) replayed from a CUDA graph."""
        mode = L.MODE_GAUSS if self.gaussian else L.MODE_VV
        self._ck(self.lib.pb_md_run(self.h, C.c_float(dt), mode, int(steps)), "run")

    def run_timed(self, dt: float, steps: int) -> float:
        mode = L.MODE_GAUSS if self.gaussian else L.MODE_VV
        ms = C.c_float()
        self._ck(self.lib.pb_md_run_timed(self.h, C.c_float(dt), mode, int(steps), C.byref(ms)),
                 "run_timed")
        return float(ms.value)

    def profile(self, dt: float, steps: int) -> dict:
        """Per-phase device ms per step (cell build, force, evolution)."""
        mode = L.MODE_GAUSS if self.gaussian else L.MODE_VV
        ms = (C.c_double * 3)()
        self._ck(self.lib.pb_md_profile(self.h, C.c_float(dt), mode, int(steps), ms), "profile")
        return {"cells": ms[0], "force": ms[1], "evolve": ms[2]}

    def minimize(self, iters: int, alpha: float = 1e-3, max_disp: float = 0.02) -> None:
        """Extension: capped steepest descent (r += F min(alpha, max_disp/|F|)) with
        the relaxation force; used to relax random starts before dynamics."""
        self._ck(self.lib.pb_md_minimize(self.h, int(iters), C.c_float(alpha),
                                         C.c_float(max_disp)), "minimize")

    def cell_build_kernels(self) -> int:
        """Kernels one cell build launches (2: bucket build, 6: counting sort)."""
        k = C.c_uint32()
        self._ck(self.lib.pb_md_cell_build_kernels(self.h, C.byref(k)), "cell_build_kernels")
        return int(k.value)

    def pair_stats(self) -> dict:
        out = (C.c_double * 2)()
        self._ck(self.lib.pb_md_pair_stats(self.h, out), "pair_stats")
        return {"ncand": out[0], "nin": out[1]}

    # ---------------------------------------------------------------- reductions
    def sums(self) -> dict:
        s = L.pb_md_sums()
        self._ck(self.lib.pb_md_reduce(self.h, C.byref(s)), "reduce")
        return {k: getattr(s, k) for k, _ in L.pb_md_sums._fields_}

    def calcTemp(self) -> float:
        t = C.c_double()
        self._ck(self.lib.pb_md_temperature(self.h, C.byref(t)), "temperature")
        self.mv2 = float(t.value) * 3 * self.n * self._kB
        return float(t.value)

    def calcKineticE(self) -> float:
        return self.mv2 / 2.0

    def calcPotentialE(self) -> float:
        """Truncated, unshifted sum_{i<j} 4 eps [(s/r)^12 - (s/r)^6].

        The reference kernel for this (MDpairPotential, kerneltemplate.hh:570-587)
        assigns instead of accumulating; this is the intended quantity.
        """
        self.calcForce(energy=True)
        return self.sums()["pe"]

    def scaleTemp(self, temp: float) -> float:
        """scaleTemp (cudaParticleMD.cu:168-175, GaussianThermo.cu:89-96): v *= s,
        s = sqrt((3N-1)/(3N) T/T0); FP32 arithmetic for the plain class, FP64 for
        the Gaussian one, as the reference computes it."""
        t0 = self.calcTemp()
        if self.gaussian:
            s = float(np.sqrt((3 * self.n - 1) / (3 * self.n) * float(np.float32(temp))
                              / float(np.float32(t0))))
        else:
            f32 = np.float32
            s = float(np.sqrt(f32(3 * self.n - 1) / f32(3 * self.n) * f32(temp) / f32(t0),
                              dtype=np.float32))
        self._ck(self.lib.pb_md_scale_velocities(self.h, C.c_double(s)), "scale")
        return float(s)

    def adjustVelocities(self, temp: float, debug: bool = False) -> None:
        """cudaParticleMD::adjustVelocities (cudaParticleMD.cu:177-198): zero mean
        and standard deviation v1 = sqrt(kB T / m0) per axis, v1 in FP32 as the
        reference computes it."""
        m0 = C.c_double()
        self._ck(self.lib.pb_md_mean_mass(self.h, C.byref(m0)), "mean_mass")
        v1 = np.sqrt(np.float32(self._kB) * np.float32(temp) / np.float32(m0.value),
                     dtype=np.float32)
        self._ck(self.lib.pb_md_adjust_velocities(self.h, C.c_double(float(v1))), "adjust")

    def constTemp(self) -> float:
        """cudaParticleMD::constTemp (cudaParticleMD.cu:140-155): lambda =
        sum F.v / sum m v^2 (FP64 sums), F -= lambda m v; returns the temperature."""
        s = self.sums()
        lam = s["fv"] / s["mv2"] if s["mv2"] > 0 else 0.0
        if lam != 0:
            self._ck(self.lib.pb_md_correct_force(self.h, C.c_double(lam)), "correct_force")
        return float(np.float32(s["mv2"])) / (3 * self.n * self._kB)

    def calcForceSoftCore(self, rc: float, f0: float) -> None:
        """The soft-core force of initialAnnealing (potentialSC, kernelinline.hh:136-158)
        on the current cell list."""
        self._ck(self.lib.pb_md_force_softcore(self.h, C.c_float(rc), C.c_float(f0)),
                 "force_softcore")

    def stepEuler(self, dt: float) -> None:
        """calcA_F4 + propagateEuler_F4 + applyPeriodicCondition_F4 with the latest force."""
        self._ck(self.lib.pb_md_step_euler(self.h, C.c_float(dt)), "step_euler")

    def initialAnnealing(self, anealstep: int, dt: float, rc: float, f0: float, T: float) -> None:
        """cudaParticleMD::initialAnnealing (cudaParticleMD.cu:205-325): anealstep
        soft-core Euler steps with the range growing to rc, each with constTemp,
        a rescale to T, anealstep LJ velocity-Verlet steps with constTemp, and a
        final rescale."""
        for i in range(anealstep):
            rci = float(np.float32(np.float32(rc) * np.float32(i + 1)) / np.float32(anealstep))
            self.calcBlockID()
            self.calcForceSoftCore(rci, f0)
            self.constTemp()
            self.stepEuler(dt)
        self.scaleTemp(T)
        self.clearForce()
        for _ in range(anealstep):
            self.calcBlockID()
            self.calcForce()
            self.constTemp()
            self._ck(self.lib.pb_md_step_vv(self.h, C.c_float(dt)), "step_vv")
            self.treatPeriodicCondition()
        self.scaleTemp(T)

    def status(self) -> int:
        b = C.c_uint32()
        self._ck(self.lib.pb_md_status(self.h, C.byref(b)), "status")
        return int(b.value)

    # ---------------------------------------------------------------- state
    _DTYPES = {"r": (np.float32, 4), "v": (np.float32, 4), "vd": (np.float64, 1),
               "F": (np.float32, 4), "Fold": (np.float32, 4), "minv": (np.float32, 1),
               "mass": (np.float32, 1), "type": (np.uint16, 1), "cell_of": (np.uint32, 1),
               "pid": (np.uint32, 1), "cell_start": (np.uint32, 1), "cell_key": (np.uint32, 1),
               "neighbors": (np.uint32, 27), "r_sorted": (np.float32, 4)}

    def get(self, field: str) -> np.ndarray:
        nbytes = C.c_size_t()
        self._ck(self.lib.pb_md_field_bytes(self.h, L.FIELD[field], C.byref(nbytes)), "field_bytes")
        dt, width = self._DTYPES[field]
        out = np.empty(nbytes.value // np.dtype(dt).itemsize, dt)
        self._ck(self.lib.pb_md_get(self.h, L.FIELD[field], _fptr(out), nbytes.value), "get " + field)
        if field == "vd":
            return out.reshape(3, -1).T.copy()
        return out.reshape(-1, width) if width > 1 else out

    def set(self, field: str, arr) -> None:
        dt, width = self._DTYPES[field]
        a = np.asarray(arr, dt)
        if field == "vd":
            a = a.reshape(-1, 3).T
        a = np.ascontiguousarray(a).reshape(-1)
        self._ck(self.lib.pb_md_set(self.h, L.FIELD[field], _fptr(a), a.nbytes), "set " + field)

    def getPosition(self) -> np.ndarray:
        return self.get("r")

    def getForce(self) -> np.ndarray:
        return self.get("F")

    def getTypeID(self) -> np.ndarray:
        return self.get("type")

    def velocities(self) -> np.ndarray:
        """(N, 3) FP64 copy of the velocities, whichever precision is stored."""
        if self.fp64_velocities:
            return self.get("vd")
        return self.get("v")[:, :3].astype(np.float64)


def from_system(s: LJSystem, gaussian: bool = False, fp64_velocities: bool | None = None,
                fp64_forces: bool = False, per_pair_cutoff: bool | None = None,
                cell_rmax: float | None = None, half_shell: bool = False) -> MDSystem:
    """Build a ready-to-step MDSystem from a host LJSystem (reduced units).
    Cells are at least `cell_rmax` wide (default: the cutoff; a neighbour list
    needs cutoff + thickness).  half_shell: evaluate every unordered pair once
    (Newton's third law, fixed-point sums) instead of every ordered pair."""
    p = MDSystem(s.n, gaussian=gaussian, fp64_velocities=fp64_velocities, fp64_forces=fp64_forces,
                 half_shell=half_shell)
    p.setCell(s.box)
    p.kB = 1.0
    p.rmax2 = float(s.rc) ** 2
    nt = s.ntypes
    if per_pair_cutoff is None:
        per_pair_cutoff = not np.allclose(s.lj[..., 2], s.rc)
    if per_pair_cutoff:
        p.setLJparamsCut(s.lj.reshape(-1), nt)
    else:
        p.setLJparams(s.lj[..., :2].reshape(-1), nt)
    p.import_arrays(s.r, s.v, s.mass, s.types)
    p.setupCutoffBlock(float(s.rc if cell_rmax is None else cell_rmax))
    return p
