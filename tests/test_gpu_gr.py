"""g(r) pair counts (cudaCalcGR) through the C ABI against the oracle and the
reference kernel's golden counts.

Bar: bit-exact counts (integer histogram; the CUDA kernel and the oracle do
the same FP32 operations, and the golden system has no pair on a bin edge).
"""
import numpy as np
import pytest

from particlebase_b200 import workloads as W

pytestmark = pytest.mark.gpu


def handle(box, r, rc=2.5):
    from particlebase_b200.md import MDSystem
    p = MDSystem(len(r))
    p.setCell(np.asarray(box, np.float32))
    p.kB = 1.0
    p.rmax2 = rc * rc
    p.setLJparams(np.array([1.0, 1.0]), 1)
    p.import_arrays(r, np.zeros_like(r), np.ones(len(r)), np.zeros(len(r), np.uint32))
    p.setupCutoffBlock(rc)
    return p


def test_gr_matches_reference_golden(cuda_lib, golden, po):
    rstep, rmax = (float(x) for x in golden["gr_rstep_rmax"])
    r = golden["gr_r4"][:, :3].astype(np.float64)
    p = handle(golden["gr_box"], r)
    got = p.gr_counts(rstep, rmax)
    assert np.array_equal(got.astype(np.int64), golden["gr_counts"].astype(np.int64))


@pytest.mark.parametrize("n,rmax", [(1500, 5.0), (3000, 2.5)])
def test_gr_matches_oracle(cuda_lib, po, n, rmax):
    s = W.kob_andersen_random(n, 0.9, 1.0, seed=n)
    r = s.r.astype(np.float32).astype(np.float64)
    p = handle(s.box, r)
    got = p.gr_counts(0.02, rmax)
    exp = po.gr_counts(p.get("r"), s.box, 0.02, rmax)
    assert got.sum() > 0
    assert np.array_equal(got.astype(np.int64), exp)
    # uniform random positions: g(r) near 1 away from r = 0
    g = po.gr_normalise(exp, n, float(np.prod(s.L)), 0.02)
    assert abs(g[len(g) // 2:].mean() - 1.0) < 0.1
