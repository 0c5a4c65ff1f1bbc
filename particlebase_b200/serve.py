"""MD job server (a pb_srv handle): continuous batching of independent LJ
jobs into one device-resident batch.

No counterpart in the reference, which runs one system per process.  Jobs
are admitted from a FIFO queue as the HBM budget allows, packed into the
running batch at the next chunk boundary, and leave it after exactly their
own step count; each job's final state is bit-identical to running it alone
with ``MDSystem.run`` under the same precision flags.

    srv = Server(hbm_budget=120e9, gaussian=True)
    jid = srv.submit(system, steps=1000, dt=0.005)
    srv.wait(jid)
    r, v, F = srv.result(jid)
    info = srv.info(jid)   # t_submit, t_admit, t_done on the server clock
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L
from .workloads import LJSystem

STATES = {0: "queued", 1: "running", 2: "done", 3: "failed"}


class Server:
    def __init__(self, hbm_budget: float = 0, gaussian: bool = True,
                 fp64_velocities: bool | None = None, fp64_forces: bool = False,
                 chunk_ms: float = 100.0, max_atoms: int = 0, max_jobs: int = 0,
                 force_threads: int = 256, seg_scale: float = 1.0,
                 reserve: float | None = None):
        self.lib = L.lib()
        if fp64_velocities is None:
            fp64_velocities = gaussian
        self.gaussian = bool(gaussian)
        self.fp64_velocities = bool(fp64_velocities)
        cfg = L.pb_srv_config()
        cfg.hbm_budget = int(hbm_budget)
        cfg.max_atoms = int(max_atoms)
        cfg.max_jobs = int(max_jobs)
        cfg.chunk_ms = float(chunk_ms)
        cfg.flags = (L.VEL_FP64 if fp64_velocities else 0) | (L.ACC_FP64 if fp64_forces else 0)
        cfg.mode = L.MODE_GAUSS if gaussian else L.MODE_VV
        cfg.force_threads = int(force_threads)
        cfg.seg_scale = float(seg_scale)
        # device memory taken into the allocator's pool up front (None: the
        # whole budget, as a serving engine pre-allocates its memory budget)
        cfg.reserve_bytes = (C.c_size_t(-1).value if reserve is None else int(reserve))
        h = C.c_void_p()
        L.check(self.lib.pb_srv_create(C.byref(cfg), C.byref(h)), "pb_srv_create")
        self.h = h
        self.natoms: dict[int, int] = {}

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.pb_srv_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _ck(self, code: int, what: str) -> None:
        if code != L.PB_OK:
            raise L.PBError(code, what, self.lib.pb_srv_last_error(self.h).decode(errors="replace"))

    def now(self) -> float:
        return float(self.lib.pb_srv_now(self.h))

    def submit(self, s: LJSystem, steps: int, dt: float = 0.005, kB: float = 1.0) -> int:
        j = L.pb_srv_job()
        j.natoms = s.n
        j.cell6[:] = [float(x) for x in np.asarray(s.box, np.float32)]
        j.rc = float(s.rc)
        lj2 = np.ascontiguousarray(s.lj[..., :2].reshape(-1), np.float32)
        j.sigma_eps = lj2.ctypes.data
        keep = [lj2]
        if not np.allclose(s.lj[..., 2], s.rc):
            lj3 = np.ascontiguousarray(s.lj.reshape(-1), np.float32)
            j.sigma_eps_rc = lj3.ctypes.data
            keep.append(lj3)
        j.ntypes = s.ntypes
        j.dt = float(dt)
        j.kB = float(kB)
        j.steps = int(steps)
        r = np.ascontiguousarray(s.r[:, :3], np.float64)
        v = np.ascontiguousarray(s.v[:, :3], np.float64)
        m = np.ascontiguousarray(s.mass, np.float64)
        t = np.ascontiguousarray(s.types, np.uint32)
        keep += [r, v, m, t]
        j.r3, j.v3, j.mass, j.type = r.ctypes.data, v.ctypes.data, m.ctypes.data, t.ctypes.data
        jid = C.c_uint64()
        self._ck(self.lib.pb_srv_submit(self.h, C.byref(j), C.byref(jid)), "submit")
        self.natoms[int(jid.value)] = s.n
        return int(jid.value)

    def wait(self, jid: int, timeout: float = -1.0) -> None:
        self._ck(self.lib.pb_srv_wait(self.h, C.c_uint64(jid), float(timeout)), f"wait {jid}")

    def drain(self, timeout: float = -1.0) -> None:
        self._ck(self.lib.pb_srv_drain(self.h, float(timeout)), "drain")

    def poll(self, max_ids: int = 4096) -> list[int]:
        ids = np.empty(max_ids, np.uint64)
        n = C.c_uint32()
        self._ck(self.lib.pb_srv_poll(self.h, ids.ctypes.data, max_ids, C.byref(n)), "poll")
        return [int(x) for x in ids[: n.value]]

    def info(self, jid: int) -> dict:
        i = L.pb_srv_job_info()
        self._ck(self.lib.pb_srv_info(self.h, C.c_uint64(jid), C.byref(i)), f"info {jid}")
        return {"id": i.id, "state": STATES.get(i.state, i.state), "natoms": i.natoms,
                "steps": i.steps, "t_submit": i.t_submit, "t_admit": i.t_admit,
                "t_done": i.t_done, "device_status": i.device_status}

    def result(self, jid: int):
        """(positions float32 (n,4), velocities (n,3) float64 or (n,4) float32, forces (n,4))."""
        n = self.natoms[jid]
        r = np.empty((n, 4), np.float32)
        F = np.empty((n, 4), np.float32)
        if self.fp64_velocities:
            v = np.empty(3 * n, np.float64)
        else:
            v = np.empty((n, 4), np.float32)
        self._ck(self.lib.pb_srv_result(self.h, C.c_uint64(jid), r.ctypes.data, v.ctypes.data,
                                        v.nbytes, F.ctypes.data), f"result {jid}")
        if self.fp64_velocities:
            v = v.reshape(3, n).T.copy()
        return r, v, F

    def release(self, jid: int) -> None:
        self._ck(self.lib.pb_srv_release(self.h, C.c_uint64(jid)), f"release {jid}")
        self.natoms.pop(jid, None)

    def stats(self) -> dict:
        st = L.pb_srv_stats()
        self._ck(self.lib.pb_srv_stats_get(self.h, C.byref(st)), "stats")
        return {k: getattr(st, k) for k, _ in L.pb_srv_stats._fields_}
