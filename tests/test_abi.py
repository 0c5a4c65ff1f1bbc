"""C-ABI boundary and host-side logic (CPU only: no kernel is launched)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from particlebase_b200 import _lib as L
from particlebase_b200 import build as B
from particlebase_b200 import workloads as W

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def lib():
    B.build()
    return L.lib()


def declared_symbols():
    names = []
    inc = os.path.join(ROOT, "include", "pb")
    for f in sorted(os.listdir(inc)):
        txt = open(os.path.join(inc, f)).read()
        names += re.findall(r"^\s*(?:int|const char \*|void \*?)\s*\*?\s*(pb_\w+)\s*\(", txt, re.M)
    return sorted(set(names))


def test_library_exports_every_declared_symbol(lib):
    names = declared_symbols()
    assert len(names) > 30
    for n in names:
        assert hasattr(lib, n), n


def test_version(lib):
    assert b"sm_100a" in lib.pb_version()


def test_particle_record_matches_reference_layout():
    # ParticleBase (ParticleBase.hh:10-18) on x86-64: 96 bytes
    assert C.sizeof(L.pb_particle) == 96
    assert L.pb_particle.is_fixed.offset == 56
    assert L.pb_particle.a.offset == 64
    assert L.pb_particle.type.offset == 88


def test_plan_grid_bit_exact_with_oracle(lib, po):
    rng = np.random.default_rng(0)
    for _ in range(300):
        lo = rng.uniform(-5, 5, 3)
        ext = rng.uniform(7.6, 200, 3)
        cell = np.array([lo[0], lo[0] + ext[0], lo[1], lo[1] + ext[1], lo[2], lo[2] + ext[2]],
                        np.float32)
        rc = np.float32(rng.uniform(1.0, 2.5))
        n = (C.c_uint32 * 3)()
        ln = (C.c_float * 3)()
        rc_code = lib.pb_plan_grid(cell.ctypes.data_as(C.POINTER(C.c_float)), C.c_float(rc), n, ln)
        try:
            on, oln = po.grid(cell, float(rc))
        except ValueError:
            assert rc_code == 1
            continue
        assert rc_code == 0
        assert list(n) == list(on)
        assert np.array_equal(np.array(ln[:], np.float32), oln)


def test_plan_grid_rejects_two_cells(lib):
    cell = np.array([0, 5, 0, 50, 0, 50], np.float32)
    n = (C.c_uint32 * 3)()
    ln = (C.c_float * 3)()
    assert lib.pb_plan_grid(cell.ctypes.data_as(C.POINTER(C.c_float)), C.c_float(2.5), n, ln) == 1


def test_plan_columns_is_a_zorder_permutation(lib):
    for nx, ny in ((3, 3), (42, 42), (7, 13)):
        rank = (C.c_uint32 * (nx * ny))()
        assert lib.pb_plan_columns(nx, ny, rank) == 0
        r = np.array(rank[:])
        assert np.array_equal(np.sort(r), np.arange(nx * ny))
        # rank order follows the interleaved (x, y) bits
        def code(c):
            a, b = divmod(int(c), ny)
            z = 0
            for k in range(16):
                z |= ((a >> k) & 1) << (2 * k) | ((b >> k) & 1) << (2 * k + 1)
            return z
        order = np.argsort(r)
        codes = [code(c) for c in order]
        assert codes == sorted(codes)


def test_workloads_shapes():
    s = W.config_c1()
    assert s.n == 4000
    assert s.n / np.prod(s.L) == pytest.approx(0.8442, rel=1e-6)
    assert np.abs(s.v.sum(0)).max() < 1e-9
    assert (s.v ** 2).sum() / (3 * s.n) == pytest.approx(0.72, rel=1e-12)
    assert np.all((s.r >= 0) & (s.r < s.L))
    reps = W.uneven_replicas(16, seed=1)
    for r in reps:
        k = round((r.n / 4) ** (1 / 3))
        assert 4 * k ** 3 == r.n and 500 <= r.n <= 60000


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    monkeypatch.setattr(L, "_lib", None)
    monkeypatch.setattr(L, "LIB_PATH", str(tmp_path / "nope.so"))
    with pytest.raises(ImportError):
        L.lib()
