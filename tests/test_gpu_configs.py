"""Parity at the configurations that are benchmarked and claimed, against the FP64 oracle.

* the full benchmark workload (C[i,j,a,b] = sum_P A[i,a,P] B[j,b,P], 27,264 pairs, 108.5
  GFLOP, C = 738M elements): plain and batched forms bit-exact (pattern, pair list, value
  bits), split form within 1e-12 relative Frobenius;
* the mixed-magnitude workload (same shapes, per-block magnitudes 10^U(-6,2)) at full size:
  split within 1e-12 relative Frobenius, batched bit-exact;
* the order-4 x order-4 permuted contraction (abcd,cdij->abij) under its decay storage rule
  and 1e-10 product screening: batched bit-exact, split within 1e-12.
The oracle runs once per workload (OpenMP over C blocks, the XMM-order restatement)."""
import numpy as np
import pytest

import oracle
import shtensor_b200 as sht
from shtensor_b200 import workloads as W
from tests.bits import bits_equal

pytestmark = pytest.mark.gpu
REL_TOL = 1e-12


@pytest.fixture(scope="module")
def bctx():
    c = sht.Context(40 << 30)
    yield c
    c.close()


def dev(ctx, h):
    t = sht.Tensor(ctx, h.block_sizes)
    t.reserve(h.index_lists() if len(h.ids) else [[] for _ in h.block_sizes])
    if h.nnz:
        t.upload(h.data)
    return t


def host(t):
    return oracle.HostTensor(t.block_sizes, t.ids, t.offsets, t.data)


def run_form(ctx, w, A, B, mode):
    C = dev(ctx, w.C)
    plan = sht.Plan(ctx, w.expr, A, B, C, w.screen_eps, sht.BlockNorm.FROBENIUS, mode)
    plan.execute(1.0, 0.0)
    pairs = plan.pairs()
    plan.close()
    ids, offs, _ = C.get_sparse_info()
    data = C.download()
    del C
    return pairs, ids, offs, data


def check_workload(ctx, w, forms):
    want = oracle.contract(w.expr, 1.0, host(w.A), host(w.B), 0.0, host(w.C), eps=w.screen_eps)
    assert len(want.pairs) > 0
    A, B = dev(ctx, w.A), dev(ctx, w.B)
    out = {}
    for mode in forms:
        pairs, ids, offs, data = run_form(ctx, w, A, B, mode)
        assert np.array_equal(pairs, want.pairs), mode
        assert np.array_equal(ids, want.C.ids) and np.array_equal(offs, want.C.offsets), mode
        if mode == sht.Mode.SPLIT:
            diff = data - want.C.data
            rel = float(np.linalg.norm(diff) / np.linalg.norm(want.C.data))
            out[mode] = (rel, float(np.abs(diff).max()))
            del diff
            assert rel <= REL_TOL, (w.name, rel)
        else:
            assert bits_equal(data, want.C.data), (w.name, mode)
            out[mode] = (0.0, 0.0)
        del data
    return out


def test_benchmark_workload_full_size(bctx):
    w = W.c1(seed=1)
    check_workload(bctx, w, [sht.Mode.PLAIN_FP64, sht.Mode.BATCHED_FP64, sht.Mode.SPLIT])


def test_mixed_magnitudes_full_size(bctx):
    w = W.c2(seed=1)
    check_workload(bctx, w, [sht.Mode.SPLIT, sht.Mode.BATCHED_FP64])


def test_permuted_order4_decay_screened(bctx):
    # a..d extent 96 in blocks of 24-48, i,j 12 in 8-16 (the configuration's extents times
    # 1/8), V blocks kept when exp(-0.5 spread) >= 0.1, pairs screened at 1e-10
    w = W.c3(seed=1)
    assert w.screen_eps == 1e-10
    check_workload(bctx, w, [sht.Mode.BATCHED_FP64, sht.Mode.SPLIT])
