"""The cell-list build that allocates no device memory.

Some callers cannot allocate device memory themselves: a host framework that
owns all device memory through its own pool, or a latency-critical loop that
must not allocate.  pb_cells_build_noalloc serves them with every scratch
array in one fixed-size static device array.  These tests check it through
the C ABI against the regular handle-based build (pb_md_build_cells), bit for
bit, on two calls in a row with different inputs, with and without a type
array, that the calls allocate no device memory, and that oversized inputs
are rejected.  This file is collected last on purpose.
"""
import ctypes as C

import numpy as np
import pytest

from particlebase_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _perturbed(seed):
    s = W.config_c1(seed=seed)
    rng = np.random.default_rng(seed)
    r = np.mod(s.r + rng.uniform(-0.07, 0.07, s.r.shape), s.L)
    s.r = np.minimum(r.astype(np.float32), np.nextafter(np.float32(s.L[0]), np.float32(0)))
    s.r = s.r.astype(np.float64)
    return s


def _call(lib, r4, typ, n, s, start, pid, slot, rs):
    import torch
    cell6 = np.ascontiguousarray(s.box, np.float32)
    return lib.pb_cells_build_noalloc(
        C.c_void_p(r4.data_ptr()), None if typ is None else C.c_void_p(typ.data_ptr()), n,
        cell6.ctypes.data_as(C.POINTER(C.c_float)), C.c_float(s.rc),
        C.c_void_p(start.data_ptr()), C.c_void_p(pid.data_ptr()), C.c_void_p(slot.data_ptr()),
        C.c_void_p(rs.data_ptr()), C.c_void_p(torch.cuda.current_stream().cuda_stream))


def test_noalloc_build_matches_handle_build(cuda_lib):
    import torch
    from particlebase_b200.md import from_system

    lib = cuda_lib
    dev = torch.device("cuda", 0)
    # two calls in a row with a type array (the second reuses the scratch), then
    # one without: all-zero types come from the scratch array itself
    for seed, with_types in ((3, True), (4, True), (5, False)):
        s = _perturbed(seed)
        p = from_system(s)
        p.calcBlockID()
        start_ref, pid_ref, rs_ref = p.get("cell_start"), p.get("pid"), p.get("r_sorted")
        n = s.n
        ncells = len(start_ref) - 1
        r4 = torch.from_numpy(p.get("r")).to(dev)
        typ = torch.zeros(n, dtype=torch.int16, device=dev) if with_types else None
        start = torch.full((ncells + 1,), -1, dtype=torch.int32, device=dev)
        pid = torch.full((n,), -1, dtype=torch.int32, device=dev)
        slot = torch.full((n,), -1, dtype=torch.int32, device=dev)
        rs = torch.full((n, 4), -7.0, dtype=torch.float32, device=dev)
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        assert _call(lib, r4, typ, n, s, start, pid, slot, rs) == 0
        torch.cuda.synchronize()
        if seed == 4:  # the same kernels as the first call: loaded, scratch resolved
            assert torch.cuda.mem_get_info()[0] == free0, "the call allocated device memory"
        assert np.array_equal(start.cpu().numpy().view(np.uint32), start_ref)
        got_pid = pid.cpu().numpy().view(np.uint32)
        assert np.array_equal(got_pid, pid_ref)
        slot_ref = np.empty(n, np.uint32)
        slot_ref[pid_ref] = np.arange(n, dtype=np.uint32)
        assert np.array_equal(slot.cpu().numpy().view(np.uint32), slot_ref)
        assert np.array_equal(rs.cpu().numpy().view(np.uint32), rs_ref.view(np.uint32))
        if not with_types:
            assert np.all(rs.cpu().numpy()[:, 3].view(np.int32) == 0)
        p.close()


def test_noalloc_rejects_oversized_input(cuda_lib):
    lib = cuda_lib
    max_atoms, max_cells, nbytes = C.c_uint32(), C.c_uint32(), C.c_size_t()
    assert lib.pb_cells_build_noalloc_limits(C.byref(max_atoms), C.byref(max_cells),
                                             C.byref(nbytes)) == 0
    assert max_atoms.value == 131072 and max_cells.value == 65536
    cell6 = np.array([0, 100, 0, 100, 0, 100], np.float32)
    dummy = C.c_void_p(16)  # never dereferenced: the size check comes first
    rc = lib.pb_cells_build_noalloc(dummy, None, max_atoms.value + 1,
                                    cell6.ctypes.data_as(C.POINTER(C.c_float)), C.c_float(2.5),
                                    dummy, dummy, dummy, dummy, None)
    assert rc == 1  # PB_ERR_ARG
    big = np.array([0, 200, 0, 200, 0, 200], np.float32)  # 80^3 cells > 65,536
    rc = lib.pb_cells_build_noalloc(dummy, None, 1000, big.ctypes.data_as(C.POINTER(C.c_float)),
                                    C.c_float(2.5), dummy, dummy, dummy, dummy, None)
    assert rc == 1
