"""ctypes bindings for the test oracle.

TEST INFRASTRUCTURE ONLY.  Imported by tests/, bench.py (CPU-baseline and
reference arms) and __graft_entry__.smoke(); the product package never imports
it.

* :class:`Oracle` wraps ``oracle/liboracle.so``: the FP64 restatement of the
  reference's LJ cell-list step (``oracle/oracle.cpp``).
* :class:`RefKernels` wraps ``oracle/_ref/libpbref.so``: the reference's own
  MD kernels compiled for the CPU (``oracle/ref_harness.cpp``).  It exists
  only where the reference checkout was available at build time.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_ORACLE = os.path.join(HERE, "liboracle.so")
LIB_REF = os.path.join(HERE, "_ref", "libpbref.so")
# the reference checkout: PB_REFERENCE_DIR, else a `reference` directory beside
# this repository
REFERENCE_DIR = os.environ.get(
    "PB_REFERENCE_DIR", os.path.normpath(os.path.join(HERE, os.pardir, os.pardir, "reference")))

_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")


def build(ref: bool = True) -> None:
    """Compile the oracle (and, when the reference checkout exists, _ref)."""
    targets = ["oracle"]
    if ref and os.path.isdir(REFERENCE_DIR):
        targets.append("ref")
    subprocess.run(["make", "-s", "-C", HERE, f"REF={REFERENCE_DIR}", *targets], check=True)


def ref_available() -> bool:
    return os.path.exists(LIB_REF)


def _load(path: str) -> C.CDLL:
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} is not built (run make -C oracle)")
    return C.CDLL(path)


_lib = None
_ref = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        L = _load(LIB_ORACLE)
        L.orc_grid.argtypes = [_f32p, C.c_float, _u32p, _f32p]
        L.orc_grid_p.argtypes = [_f32p, C.c_float, C.c_int, _u32p, _f32p]
        L.orc_bin_p.argtypes = [_f32p, C.c_uint32, _f32p, C.c_float, C.c_int, _u32p]
        L.orc_neighbor_table.argtypes = [_f32p, C.c_float, C.c_int, _u32p]
        L.orc_bin.argtypes = [_f32p, C.c_uint32, _f32p, C.c_float, _u32p]
        L.orc_cell_list.argtypes = [_u32p, C.c_void_p, C.c_uint32, C.c_uint32, _u32p, _u32p]
        L.orc_wrap_f32.argtypes = [_f32p, C.c_uint32, _f32p]
        L.orc_create.restype = C.c_void_p
        L.orc_create.argtypes = [C.c_uint32, _f32p, C.c_float, _f64p, C.c_int]
        L.orc_destroy.argtypes = [C.c_void_p]
        L.orc_set_state.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.orc_set_fold.argtypes = [C.c_void_p, _f64p]
        L.orc_set_xi.argtypes = [C.c_void_p, C.c_double]
        L.orc_set_tol.argtypes = [C.c_void_p, C.c_double]
        L.orc_forces.argtypes = [C.c_void_p, _f64p]
        L.orc_run.argtypes = [C.c_void_p, C.c_uint32, C.c_double, C.c_int, C.c_void_p]
        L.orc_run.restype = C.c_int
        L.orc_steepest_descent.argtypes = [C.c_void_p, C.c_uint32, C.c_double, C.c_double]
        L.orc_kinetic.argtypes = [C.c_void_p]
        L.orc_kinetic.restype = C.c_double
        L.orc_get_xi.argtypes = [C.c_void_p]
        L.orc_get_xi.restype = C.c_double
        L.orc_get_nr_iters.argtypes = [C.c_void_p]
        L.orc_get.argtypes = [C.c_void_p, C.c_int, _f64p]
        L.orc_threads.restype = C.c_int
        L.orc_adjust_velocities.argtypes = [C.c_void_p, C.c_double]
        L.orc_scale_temp.argtypes = [C.c_void_p, C.c_double, C.c_double]
        L.orc_scale_temp.restype = C.c_double
        L.orc_forces_softcore.argtypes = [C.c_void_p, C.c_double, C.c_double]
        L.orc_const_temp.argtypes = [C.c_void_p]
        L.orc_const_temp.restype = C.c_double
        L.orc_euler.argtypes = [C.c_void_p, C.c_double]
        L.orc_initial_annealing.argtypes = [C.c_void_p, C.c_uint32, C.c_double, C.c_double,
                                            C.c_double, C.c_double, C.c_double]
        _lib = L
    return _lib


def ref() -> C.CDLL:
    global _ref
    if _ref is None:
        L = _load(LIB_REF)
        L.ref_create.restype = C.c_void_p
        L.ref_create.argtypes = [C.c_uint32, _f32p, C.c_int]
        L.ref_destroy.argtypes = [C.c_void_p]
        for n in ("ref_set_rmax2", "ref_set_kB", "ref_set_e"):
            getattr(L, n).argtypes = [C.c_void_p, C.c_float]
        L.ref_set_lj.argtypes = [C.c_void_p, _f32p, C.c_uint32]
        L.ref_import.argtypes = [C.c_void_p, _f64p, _f64p, _f64p, _u32p]
        L.ref_set_positions.argtypes = [C.c_void_p, _f32p]
        L.ref_setup_cells.argtypes = [C.c_void_p, C.c_float]
        L.ref_setup_cells.restype = C.c_int
        L.ref_setup_cells_p.argtypes = [C.c_void_p, C.c_float, C.c_int]
        L.ref_setup_cells_p.restype = C.c_int
        for n in ("ref_calc_block_id", "ref_calc_force", "ref_clear_force", "ref_wrap"):
            getattr(L, n).argtypes = [C.c_void_p]
        L.ref_calc_mv2.argtypes = [C.c_void_p]
        L.ref_calc_mv2.restype = C.c_double
        L.ref_time_evolution.argtypes = [C.c_void_p, C.c_float]
        L.ref_time_evolution.restype = C.c_int
        L.ref_run.argtypes = [C.c_void_p, C.c_float, C.c_uint32]
        L.ref_run.restype = C.c_int
        for n in ("ref_get_r", "ref_get_v", "ref_get_F", "ref_get_Fold"):
            getattr(L, n).argtypes = [C.c_void_p, _f32p]
        L.ref_get_vd.argtypes = [C.c_void_p, _f64p]
        L.ref_get_xi.argtypes = [C.c_void_p]
        L.ref_get_xi.restype = C.c_double
        L.ref_num_cells.argtypes = [C.c_void_p]
        L.ref_num_cells.restype = C.c_uint32
        L.ref_get_grid.argtypes = [C.c_void_p, _u32p, _f32p]
        L.ref_get_cells.argtypes = [C.c_void_p, _u32p, _u32p, _u32p]
        L.ref_get_neighbors.argtypes = [C.c_void_p, _u32p]
        L.ref_threads.restype = C.c_int
        L.ref_gr.argtypes = [C.c_void_p, C.c_float, C.c_float, C.c_void_p, C.c_uint32]
        L.ref_gr.restype = C.c_int
        L.ref_adjust_velocities.argtypes = [C.c_void_p, C.c_float]
        L.ref_scale_temp.argtypes = [C.c_void_p, C.c_float]
        L.ref_scale_temp.restype = C.c_double
        L.ref_calc_force_softcore.argtypes = [C.c_void_p, C.c_float, C.c_float]
        L.ref_const_temp.argtypes = [C.c_void_p, C.POINTER(C.c_double)]
        L.ref_const_temp.restype = C.c_double
        L.ref_euler.argtypes = [C.c_void_p, C.c_float]
        L.ref_initial_annealing.argtypes = [C.c_void_p, C.c_uint32, C.c_float, C.c_float,
                                            C.c_float, C.c_float]
        L.ref_set_v.argtypes = [C.c_void_p, _f32p]
        L.ref_set_F.argtypes = [C.c_void_p, _f32p]
        _ref = L
    return _ref


def _cell6(box) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(box, dtype=np.float32).reshape(6))


# ---------------------------------------------------------------- stateless


def grid(box, rc, periodic=True):
    n = np.zeros(3, np.uint32)
    ln = np.zeros(3, np.float32)
    if lib().orc_grid_p(_cell6(box), rc, int(periodic), n, ln):
        raise ValueError("cell grid needs at least 3 cells per dimension")
    return n, ln


def neighbor_table(box, rc, periodic=True):
    n, _ = grid(box, rc, periodic)
    out = np.zeros(int(np.prod(n)) * 27, np.uint32)
    lib().orc_neighbor_table(_cell6(box), rc, int(periodic), out)
    return out.reshape(-1, 27)


def bin_cells(r4, box, rc, periodic=True):
    r4 = np.ascontiguousarray(r4, np.float32).reshape(-1, 4)
    out = np.zeros(len(r4), np.uint32)
    if lib().orc_bin_p(r4.reshape(-1), len(r4), _cell6(box), rc, int(periodic), out):
        raise ValueError("bad grid")
    return out


def cell_list(cid, ncells, z=None):
    """Members per cell; within a cell by ascending FP32 z (ties: particle id)
    when z is given, else by particle id."""
    cid = np.ascontiguousarray(cid, np.uint32)
    start = np.zeros(ncells + 1, np.uint32)
    members = np.zeros(len(cid), np.uint32)
    zz = None if z is None else np.ascontiguousarray(z, np.float32)
    lib().orc_cell_list(cid, None if zz is None else zz.ctypes.data, len(cid), ncells, start, members)
    return start, members


def wrap_f32(r4, box):
    r4 = np.array(r4, np.float32, copy=True).reshape(-1, 4)
    lib().orc_wrap_f32(r4.reshape(-1), len(r4), _cell6(box))
    return r4


# ---------------------------------------------------------------- stateful


class Oracle:
    """FP64 system: positions, velocities, forces and the reference step."""

    def __init__(self, box, lj, rc_grid, r, v=None, mass=None, types=None):
        lj = np.ascontiguousarray(lj, np.float64)
        nt = int(round((lj.size / 3) ** 0.5))
        r = np.ascontiguousarray(np.asarray(r, np.float64)[:, :3])
        self.N = len(r)
        self.h = lib().orc_create(self.N, _cell6(box), rc_grid, lj.reshape(-1), nt)
        if not self.h:
            raise ValueError("oracle_create failed (grid or types)")
        v = np.zeros_like(r) if v is None else np.ascontiguousarray(v, np.float64)[:, :3]
        mass = np.ones(self.N) if mass is None else np.ascontiguousarray(mass, np.float64)
        types = np.zeros(self.N, np.uint32) if types is None else np.ascontiguousarray(types, np.uint32)
        self._keep = (r, np.ascontiguousarray(v), mass, types)
        lib().orc_set_state(self.h, *(a.ctypes.data for a in self._keep))

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_destroy(self.h)
            self.h = None

    def forces(self):
        out = np.zeros(5)
        lib().orc_forces(self.h, out)
        return {"pe": out[0], "pe_shift": out[1], "virial": out[2], "ncand": out[3], "nin": out[4]}

    def run(self, steps, dt, mode="nve", record=False):
        e = np.zeros((steps, 3)) if record else None
        rc = lib().orc_run(self.h, steps, dt, 0 if mode == "nve" else 1,
                           e.ctypes.data if record else None)
        if rc:
            raise RuntimeError("Newton-Raphson did not converge")
        return e

    def set_tol(self, tol):
        lib().orc_set_tol(self.h, tol)

    def set_xi(self, xi):
        lib().orc_set_xi(self.h, xi)

    def set_fold(self, fold):
        lib().orc_set_fold(self.h, np.ascontiguousarray(fold, np.float64).reshape(-1))

    def steepest_descent(self, iters, alpha, max_disp):
        """Capped steepest descent (extension): r += F min(alpha, max_disp/|F|)
        with the relaxation force (pair distance floored at sigma/2)."""
        lib().orc_steepest_descent(self.h, iters, alpha, max_disp)

    def adjust_velocities(self, v1):
        """adjustVelocity_F4 / _VD: zero mean, standard deviation v1 per axis."""
        lib().orc_adjust_velocities(self.h, v1)

    def scale_temp(self, T, kB=1.0):
        """scaleTemp: returns the factor sqrt((3N-1)/(3N) T/T0) applied to v."""
        return lib().orc_scale_temp(self.h, T, kB)

    def forces_softcore(self, rc, f0):
        """The soft-core force of initialAnnealing (potentialSC)."""
        lib().orc_forces_softcore(self.h, rc, f0)

    def const_temp(self):
        """constTemp's correction F -= lambda m v; returns lambda."""
        return lib().orc_const_temp(self.h)

    def euler(self, dt):
        """calcA_F4 + propagateEuler_F4 + wrap."""
        lib().orc_euler(self.h, dt)

    def initial_annealing(self, steps, dt, rc, f0, T, kB=1.0):
        lib().orc_initial_annealing(self.h, steps, dt, rc, f0, T, kB)

    def get(self, name):
        idx = {"r": 0, "v": 1, "F": 2, "Fold": 3, "pe_atom": 4}[name]
        out = np.zeros(self.N if name == "pe_atom" else 3 * self.N)
        lib().orc_get(self.h, idx, out)
        return out if name == "pe_atom" else out.reshape(-1, 3)

    @property
    def xi(self):
        return lib().orc_get_xi(self.h)

    def kinetic(self):
        return lib().orc_kinetic(self.h)


class RefKernels:
    """The reference's own MD kernels run on the CPU (oracle/_ref)."""

    def __init__(self, box, rc, r, v, mass, types, lj_sigma_eps, ntypes=1,
                 gaussian=False, rmax2=None, kB=1.0, tol=1e-8, periodic=True):
        L = ref()
        self.N = len(r)
        self.h = L.ref_create(self.N, _cell6(box), int(gaussian))
        L.ref_set_lj(self.h, np.ascontiguousarray(lj_sigma_eps, np.float32).reshape(-1), ntypes)
        L.ref_set_rmax2(self.h, float(rc * rc if rmax2 is None else rmax2))
        L.ref_set_kB(self.h, kB)
        L.ref_set_e(self.h, tol)
        L.ref_import(self.h, np.ascontiguousarray(r, np.float64)[:, :3].copy().reshape(-1),
                     np.ascontiguousarray(v, np.float64)[:, :3].copy().reshape(-1),
                     np.ascontiguousarray(mass, np.float64),
                     np.ascontiguousarray(types, np.uint32))
        if L.ref_setup_cells_p(self.h, rc, int(periodic)):
            raise ValueError("reference grid needs blocknum > 2")
        L.ref_clear_force(self.h)

    def __del__(self):
        if getattr(self, "h", None):
            ref().ref_destroy(self.h)
            self.h = None

    def set_positions(self, r4):
        ref().ref_set_positions(self.h, np.ascontiguousarray(r4, np.float32).reshape(-1))

    def calc_block_id(self):
        ref().ref_calc_block_id(self.h)

    def calc_force(self):
        ref().ref_calc_force(self.h)

    def time_evolution(self, dt):
        return ref().ref_time_evolution(self.h, dt)

    def wrap(self):
        ref().ref_wrap(self.h)

    def run(self, dt, steps):
        return ref().ref_run(self.h, dt, steps)

    def mv2(self):
        return ref().ref_calc_mv2(self.h)

    def adjust_velocities(self, v1):
        """adjustVelocity_F4 / adjustVelocity_VD with v1 = sqrt(kB T / m0) (FP32)."""
        ref().ref_adjust_velocities(self.h, v1)

    def scale_temp(self, T):
        """scaleTemp: returns the factor applied (mulArray)."""
        return ref().ref_scale_temp(self.h, T)

    def calc_force_softcore(self, rc, f0):
        """Soft-core force of initialAnnealing (potentialSC) on the current cells."""
        ref().ref_calc_force_softcore(self.h, rc, f0)

    def const_temp(self):
        """constTemp: returns (temperature, lambda); corrects F when lambda != 0."""
        lam = C.c_double()
        t = ref().ref_const_temp(self.h, C.byref(lam))
        return t, lam.value

    def euler(self, dt):
        """calcA_F4 + propagateEuler_F4 + applyPeriodicCondition_F4."""
        ref().ref_euler(self.h, dt)

    def initial_annealing(self, steps, dt, rc, f0, T):
        ref().ref_initial_annealing(self.h, steps, dt, rc, f0, T)

    def set4(self, name, arr):
        getattr(ref(), "ref_set_" + name)(self.h, np.ascontiguousarray(arr, np.float32).reshape(-1))

    def get4(self, name):
        out = np.zeros(4 * self.N, np.float32)
        getattr(ref(), "ref_get_" + name)(self.h, out)
        return out.reshape(-1, 4)

    def vd(self):
        out = np.zeros(3 * self.N)
        ref().ref_get_vd(self.h, out)
        return out.reshape(3, -1).T.copy()

    @property
    def xi(self):
        return ref().ref_get_xi(self.h)

    def grid(self):
        n = np.zeros(3, np.uint32)
        ln = np.zeros(6, np.float32)
        ref().ref_get_grid(self.h, n, ln)
        return n, ln

    def cells(self):
        nc = ref().ref_num_cells(self.h)
        bid = np.zeros(self.N, np.uint32)
        pid = np.zeros(self.N, np.uint32)
        bindex = np.zeros(nc + 1, np.uint32)
        ref().ref_get_cells(self.h, bid, pid, bindex)
        return bid, pid, bindex

    def gr_counts(self, rstep, rmax):
        """cudaCalcGR pair counts per bin (after calc_block_id), from the
        reference's own kernel; bin 0 holds nothing."""
        L = ref()
        rnum = L.ref_gr(self.h, rstep, rmax, None, 0)
        out = np.zeros(rnum, np.uint32)
        L.ref_gr(self.h, rstep, rmax, out.ctypes.data_as(C.c_void_p), rnum)
        return out

    def neighbors(self):
        nc = ref().ref_num_cells(self.h)
        out = np.zeros(nc * 27, np.uint32)
        ref().ref_get_neighbors(self.h, out)
        return out.reshape(-1, 27)


# ---- g(r) -------------------------------------------------------------------


def gr_bins(rstep, rmax):
    """Number of bins of cudaCalcGR::setup (cudaCalcGR.hh:27-31): rstepinv =
    1 / rstep (double quotient stored as FP32), rnum = trunc(rmax * rstepinv)
    in FP32."""
    inv = np.float32(1.0 / np.float64(np.float32(rstep)))
    return int(np.float32(np.float32(rmax) * inv)), inv


def _image_delta32(a, b, L):
    """x_i - x_j in FP32 with the minimum image, the coordinate above the box
    middle moved down by L first (exact), as the CUDA g(r) and neighbour-list
    kernels do."""
    L = np.float32(L)
    h = np.float32(0.5) * L
    d = (a - b).astype(np.float32)
    hi = d > h
    lo = d < -h
    d = np.where(hi, (a - L) - b, d)
    d = np.where(lo, a - (b - L), d)
    return d.astype(np.float32)


def gr_counts(r4, box, rstep, rmax):
    """Pair counts per bin of every unordered pair (i < j) of positions r4,
    restating cudaCalcGR::calcgr with calcGR_F4 (kernelinline.hh:433-449):
    bin = trunc(sqrt(r^2) * rstepinv + 0.5), counted when 0 < bin < rnum.
    Arithmetic in FP32 without fused multiply-adds, r^2 = (dx^2 + dy^2) + dz^2,
    with the exact minimum image of _image_delta32, as the CUDA kernel does
    (the reference takes the minimum image inside r^2, distance2p at
    kernelinline.hh:47-62, which can move a pair on a bin edge by one bin)."""
    rnum, inv = gr_bins(rstep, rmax)
    b = np.asarray(box, np.float32)
    r = np.asarray(r4, np.float32)[:, :3]
    n = len(r)
    counts = np.zeros(rnum, np.int64)
    Ls = [b[1] - b[0], b[3] - b[2], b[5] - b[4]]
    for i0 in range(0, n, 512):
        ri = r[i0:i0 + 512]
        d = [_image_delta32(ri[:, None, k], r[None, :, k], Ls[k]) for k in range(3)]
        r2 = ((d[0] * d[0] + d[1] * d[1]).astype(np.float32) + d[2] * d[2]).astype(np.float32)
        bins = (np.sqrt(r2).astype(np.float32) * inv + np.float32(0.5)).astype(np.float32)
        bins = np.floor(bins).astype(np.int64)
        ii = np.arange(i0, i0 + len(ri))[:, None]
        jj = np.arange(n)[None, :]
        keep = (jj > ii) & (bins > 0) & (bins < rnum)
        counts += np.bincount(bins[keep], minlength=rnum)[:rnum]
    return counts


def gr_normalise(counts, n, volume, rstep):
    """cudaCalcGR::igr2gr (cudaCalcGR.cu:118-136): g_j = counts_j * Q /
    (4 j^2 + 1/3), Q = 2 / N / (pi rstep^3) * V / N; g_0 = 0."""
    j = np.arange(len(counts), dtype=np.float64)
    q = 2.0 / n / (np.pi * rstep ** 3) * volume / n
    g = counts * q / (4 * j * j + 1.0 / 3.0)
    g[0] = 0.0
    return g
