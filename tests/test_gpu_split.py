"""Split-precision (Ozaki, INT8 tensor-core slices with FP64 reassembly) contraction on the
B200 against the FP64 oracle.

Bar: result pattern and pair list bit-exact; values within 1e-12 relative Frobenius of the
oracle (the FP64-accurate target), max abs error reported."""
import numpy as np
import pytest

import oracle
import shtensor_b200 as sht
from shtensor_b200 import workloads as W

pytestmark = pytest.mark.gpu
REL_TOL = 1e-12


def dev(ctx, h):
    t = sht.Tensor(ctx, h.block_sizes)
    t.reserve(h.index_lists() if len(h.ids) else [[] for _ in h.block_sizes])
    if h.nnz:
        t.upload(h.data)
    return t


def host(t):
    return oracle.HostTensor(t.block_sizes, t.ids, t.offsets, t.data)


def run_split(ctx, w, alpha=1.0, beta=0.0, Cinit=None):
    A, B = dev(ctx, w.A), dev(ctx, w.B)
    Ch = Cinit if Cinit is not None else w.C
    C = dev(ctx, Ch)
    plan = sht.Plan(ctx, w.expr, A, B, C, w.screen_eps, sht.BlockNorm.FROBENIUS, sht.Mode.SPLIT)
    plan.execute(alpha, beta)
    want = oracle.contract(w.expr, alpha, host(w.A), host(w.B), beta, host(Ch), eps=w.screen_eps)
    ids, offs, _ = C.get_sparse_info()
    got = C.download()
    assert np.array_equal(plan.pairs(), want.pairs)
    assert np.array_equal(ids, want.C.ids) and np.array_equal(offs, want.C.offsets)
    err = np.linalg.norm(got - want.C.data) / max(np.linalg.norm(want.C.data), 1e-300)
    return err, np.abs(got - want.C.data).max(), plan.report()


def test_split_tiny_c0(ctx):
    err, mx, rep = run_split(ctx, W.c0(seed=2, nblocks=4, p=0.5))
    assert rep["slices"] == 7
    assert err <= REL_TOL, (err, mx)


def test_split_c1_scaled(ctx):
    err, mx, _ = run_split(ctx, W.c1(seed=3, scale=0.3, occupancy=0.4), alpha=0.5)
    assert err <= REL_TOL, (err, mx)


def test_split_mixed_magnitudes(ctx):
    # per-block magnitudes 10^U(-6,2): per-row / per-column scaling keeps every pair accurate
    err, mx, _ = run_split(ctx, W.c2(seed=4, scale=0.3, occupancy=0.4))
    assert err <= REL_TOL, (err, mx)


def test_split_existing_c_and_beta(ctx):
    w = W.c0(seed=9, nblocks=6, p=0.4)
    rng = np.random.default_rng(2)
    grid = int(np.prod([len(b) for b in w.C.block_sizes]))
    cid = np.sort(rng.choice(grid, 30, replace=False))
    Ch = W.build_tensor(rng, w.C.block_sizes, lambda c: np.isin(np.arange(grid), cid), None, "normal")
    err, mx, _ = run_split(ctx, w, alpha=2.0, beta=-0.5, Cinit=Ch)
    assert err <= REL_TOL, (err, mx)


def test_split_slice_count_tradeoff(ctx):
    w = W.c1(seed=5, scale=0.25, occupancy=0.5)
    errs = {}
    for S in (4, 7):
        ctx.set_split_slices(S)
        try:
            errs[S] = run_split(ctx, w)[0]
        finally:
            ctx.set_split_slices(7)
    assert errs[7] <= REL_TOL and errs[4] > errs[7]


def test_split_non_finite_inputs_follow_the_fp64_forms(ctx):
    # an operand with Inf and NaN: the execute is computed by the FP64 tiles, so the result is
    # the plain form's, bit for bit (IEEE propagation), and the call does not fail
    from tests.bits import bits_equal
    w = W.c0(seed=6, nblocks=4, p=0.6)
    w.A.data[3] = np.inf
    w.B.data[5] = np.nan
    A, B = dev(ctx, w.A), dev(ctx, w.B)
    Cs, Cp = dev(ctx, w.C), dev(ctx, w.C)
    sht.contract(ctx, w.expr, 1.0, A, B, 0.0, Cs, mode=sht.Mode.SPLIT)
    sht.contract(ctx, w.expr, 1.0, A, B, 0.0, Cp, mode=sht.Mode.PLAIN_FP64)
    ctx.stream_sync()
    got, want = Cs.download(), Cp.download()
    assert np.isnan(got).any() and np.isinf(got).any()
    assert bits_equal(got, want)
    # the same plan with finite data again takes the tensor-core path
    w2 = W.c0(seed=6, nblocks=4, p=0.6)
    A.upload(w2.A.data)
    B.upload(w2.B.data)
    err, mx, _ = run_split(ctx, w2)
    assert err <= REL_TOL, (err, mx)


def test_split_queued_back_to_back(ctx):
    # two split contractions queued on one stream with no host wait between them (the second
    # accumulates into the first's output), then one synchronization: both as the oracle
    import torch
    w = W.c1(seed=13, scale=0.25, occupancy=0.4)
    A, B, C1, C2 = dev(ctx, w.A), dev(ctx, w.B), dev(ctx, w.C), dev(ctx, w.C)
    s = torch.cuda.Stream()
    sht.contract(ctx, w.expr, 1.0, A, B, 0.0, C1, mode=sht.Mode.SPLIT, stream=s)
    sht.contract(ctx, w.expr, 0.5, A, B, 0.0, C2, mode=sht.Mode.SPLIT, stream=s)
    sht.contract(ctx, w.expr, 1.0, A, B, 2.0, C1, mode=sht.Mode.SPLIT, stream=s)
    ctx.stream_sync(s)
    want = oracle.contract(w.expr, 1.0, host(w.A), host(w.B), 0.0, host(w.C))
    want3 = oracle.contract(w.expr, 1.0, host(w.A), host(w.B), 2.0, want.C)
    for C, ref in ((C1, want3.C.data), (C2, 0.5 * want.C.data)):
        got = C.download()
        assert np.linalg.norm(got - ref) <= REL_TOL * np.linalg.norm(ref)


def test_split_bounded_wait_reports_timeout(ctx):
    # a one-poll wait limit makes the pipeline waits run out: the launch stops (its in-flight
    # copies and MMAs drained under their own bound), the context records SHT_ERR_TIMEOUT, the
    # stream sync reports it once, and the context keeps working afterwards
    w = W.c1(seed=14, scale=0.25, occupancy=0.4)
    A, B, C = dev(ctx, w.A), dev(ctx, w.B), dev(ctx, w.C)
    ctx.set_wait_limit(1)
    try:
        sht.contract(ctx, w.expr, 1.0, A, B, 0.0, C, mode=sht.Mode.SPLIT)
        with pytest.raises(sht.ShtError) as ei:
            ctx.stream_sync()
        assert ei.value.status == sht.Status.ERR_TIMEOUT
    finally:
        ctx.set_wait_limit(0)
    ctx.stream_sync()  # reported once
    err, mx, _ = run_split(ctx, w)
    assert err <= REL_TOL, (err, mx)


def test_compare_entry_point(ctx):
    w = W.c1(seed=6, scale=0.25, occupancy=0.5)
    A, B = dev(ctx, w.A), dev(ctx, w.B)
    C1, C2 = dev(ctx, w.C), dev(ctx, w.C)
    sht.contract(ctx, w.expr, 1.0, A, B, 0.0, C1, mode=sht.Mode.BATCHED_FP64)
    sht.contract(ctx, w.expr, 1.0, A, B, 0.0, C2, mode=sht.Mode.SPLIT)
    mx, fro = sht.compare(C2, C1)
    assert 0.0 <= fro <= REL_TOL and mx >= 0.0


def per_block_errors(ctx, w):
    """Run the split form and return, per C block, (relative error, max abs error, max |want|)."""
    A, B, C = dev(ctx, w.A), dev(ctx, w.B), dev(ctx, w.C)
    sht.contract(ctx, w.expr, 1.0, A, B, 0.0, C, mode=sht.Mode.SPLIT)
    want = oracle.contract(w.expr, 1.0, host(w.A), host(w.B), 0.0, host(w.C))
    ids, offs, _ = C.get_sparse_info()
    assert np.array_equal(ids, want.C.ids)
    got = C.download()
    ends = np.append(offs[1:], got.size)
    out = []
    for o, e in zip(offs, ends):
        g, r = got[o:e], want.C.data[o:e]
        scale = np.abs(r).max()
        # relative to the block's largest value (no squares: values reach 1e300)
        out.append((float(np.abs(g - r).max() / scale) if scale > 0 else 0.0, float(np.abs(g - r).max()), scale))
    return out


@pytest.mark.parametrize("scales", [((1e-150, 1.0, 1e150), (1e150, 1e-160, 1.0)),
                                    ((1e-280, 1.0, 1e280), (1e10, 1e-30, 1.0)),
                                    ((1.0, 2.0, 3.0), (1e-310, 1e300, 1.0))])
def test_split_extreme_exponents(ctx, scales):
    # far-apart row / column exponents and subnormal products.  The first set stays inside the
    # scale-folded range (A rows 2^-900 .. 2^960, B columns normal); in the second an A row
    # maximum near 1e-280 and in the third a subnormal B column fall outside it, so the launch
    # scales every element on its own
    rng = np.random.default_rng(11)
    bi, bk, bj = [8, 12, 16], [20, 40], [10, 24, 6]
    sa, sb = np.array(scales[0]), np.array(scales[1])
    A = W.build_tensor(rng, [bi, bk], lambda c: np.ones(len(c[0]), bool), lambda c: sa[c[0]], "normal")
    B = W.build_tensor(rng, [bk, bj], lambda c: np.ones(len(c[0]), bool), lambda c: sb[c[1]], "normal")
    w = W.Workload("extreme", "ik, kj -> ij", A, B, W.empty_tensor([bi, bj]))
    for rel, mx, scale in per_block_errors(ctx, w):
        if scale < 1e-300:
            # subnormal results: the oracle rounds every product to the subnormal grid
            assert mx <= 64 * 5e-324 * 60, (mx, scale)
        else:
            assert rel <= 1e-13, (rel, scale)


def test_split_long_contracted_extent(ctx):
    # K = 9728: the INT32 group sums reach 7 * 127^2 * K > 2^23, beyond the 32-bit pairing of the
    # narrow reassembly, so the launch combines the groups in int64 (the wide instance)
    rng = np.random.default_rng(12)
    bi, bk, bj = [8, 24], [9728], [16, 8]
    A = W.build_tensor(rng, [bi, bk], lambda c: np.ones(len(c[0]), bool), None, "normal")
    B = W.build_tensor(rng, [bk, bj], lambda c: np.ones(len(c[0]), bool), None, "normal")
    w = W.Workload("long_k", "ik, kj -> ij", A, B, W.empty_tensor([bi, bj]))
    errs = per_block_errors(ctx, w)
    assert max(e[0] for e in errs) <= REL_TOL, errs


def test_split_contract_grows_then_reuses_pattern(ctx):
    # sht_contract plans assuming C's stored pattern covers the product and checks that at the
    # work list; a C holding only part of the product takes the second build, which grows it;
    # the next contraction into the grown C keeps the assumption
    w = W.c1(seed=7, scale=0.2, occupancy=0.3)
    rng = np.random.default_rng(8)
    Ch = W.build_tensor(rng, w.C.block_sizes, lambda c: rng.random(len(c[0])) < 0.2, None, "normal")
    A, B, C = dev(ctx, w.A), dev(ctx, w.B), dev(ctx, Ch)
    sht.contract(ctx, w.expr, 0.5, A, B, 1.5, C, mode=sht.Mode.SPLIT)
    want = oracle.contract(w.expr, 0.5, host(w.A), host(w.B), 1.5, host(Ch))
    ids, offs, _ = C.get_sparse_info()
    assert np.array_equal(ids, want.C.ids) and np.array_equal(offs, want.C.offsets)
    got = C.download()
    assert np.linalg.norm(got - want.C.data) <= REL_TOL * np.linalg.norm(want.C.data)
    # again into the grown C: the pattern holds every product block now
    Cg = oracle.HostTensor(w.C.block_sizes, ids, offs, got)
    sht.contract(ctx, w.expr, 1.0, A, B, -1.0, C, mode=sht.Mode.SPLIT)
    want2 = oracle.contract(w.expr, 1.0, host(w.A), host(w.B), -1.0, Cg)
    ids2, _, _ = C.get_sparse_info()
    assert np.array_equal(ids2, ids)
    got2 = C.download()
    assert np.linalg.norm(got2 - want2.C.data) <= REL_TOL * max(np.linalg.norm(want2.C.data), 1e-300)
