"""Block-sparse contraction on the B200 through the C ABI, against the oracle.

Bar (plain FP64): result pattern, offsets and the pair list bit-exact; values bit-exact to
the XMM-order restatement (the kernel does the same fma chain), and within 1e-13 relative
Frobenius of the reference LAPACK path frozen in tests/golden."""
import os

import numpy as np
import pytest

import oracle
import shtensor_b200 as sht
from tests.bits import bits_equal
from shtensor_b200 import workloads as W

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
MODES = [sht.Mode.PLAIN_FP64, sht.Mode.BATCHED_FP64]


def dev(ctx, h):
    t = sht.Tensor(ctx, h.block_sizes)
    t.reserve(h.index_lists() if len(h.ids) else [[] for _ in h.block_sizes])
    if h.nnz:
        t.upload(h.data)
    return t


def host(t):
    return oracle.HostTensor(t.block_sizes, t.ids, t.offsets, t.data)


def run_both(ctx, w, mode, alpha=1.0, beta=0.0, eps=0.0, Cinit=None, norm=sht.BlockNorm.FROBENIUS):
    A, B = dev(ctx, w.A), dev(ctx, w.B)
    Ch = Cinit if Cinit is not None else w.C
    C = dev(ctx, Ch)
    plan = sht.Plan(ctx, w.expr, A, B, C, eps, norm, mode)
    plan.execute(alpha, beta)
    pairs = plan.pairs()
    ids, offs, _ = C.get_sparse_info()
    data = C.download()
    want = oracle.contract(w.expr, alpha, host(w.A), host(w.B), beta, host(Ch), eps=eps, norm=int(norm))
    return pairs, ids, offs, data, want, plan.report()


@pytest.mark.parametrize("name", ["c0", "c1", "c3"])
@pytest.mark.parametrize("mode", MODES)
def test_golden_fixtures(ctx, name, mode):
    d = np.load(os.path.join(GOLD, "blocksparse.npz"))

    def ten(prefix):
        nb = d[f"{name}_{prefix}_nb"]
        flat = d[f"{name}_{prefix}_bs"]
        bs, pos = [], 0
        for n in nb:
            bs.append(list(map(int, flat[pos:pos + n])))
            pos += n
        t = sht.Tensor(ctx, bs)
        if f"{name}_{prefix}_ids" in d:
            t.reserve(W.HostBlockSparse(bs, d[f"{name}_{prefix}_ids"], None, None).index_lists())
            t.upload(d[f"{name}_{prefix}_data"])
        else:
            t.reserve([[] for _ in bs])
        return t

    A, B, C = ten("A"), ten("B"), ten("C")
    plan = sht.Plan(ctx, str(d[f"{name}_expr"][0]), A, B, C, float(d[f"{name}_eps"][0]), sht.BlockNorm.FROBENIUS,
                    mode)
    plan.execute(1.0, 0.0)
    assert np.array_equal(plan.pairs(), d[f"{name}_pairs"])
    ids, offs, _ = C.get_sparse_info()
    assert np.array_equal(ids, d[f"{name}_cids"]) and np.array_equal(offs, d[f"{name}_coffs"])
    got = C.download()
    assert bits_equal(got, d[f"{name}_cdata"])
    ref = d[f"{name}_cdata_ref"]
    assert np.linalg.norm(got - ref) <= 1e-13 * np.linalg.norm(ref)


@pytest.mark.parametrize("mode", MODES)
def test_c0_full_config_bit_exact(ctx, mode):
    w = W.c0(seed=1)
    pairs, ids, offs, data, want, rep = run_both(ctx, w, mode)
    assert np.array_equal(pairs, want.pairs)
    assert np.array_equal(ids, want.C.ids) and np.array_equal(offs, want.C.offsets)
    assert bits_equal(data, want.C.data)
    assert rep["flops"] == pytest.approx(want.flops, rel=1e-12)


@pytest.mark.parametrize("mode", MODES)
def test_c1_scaled_bit_exact(ctx, mode):
    w = W.c1(seed=2, scale=0.3, occupancy=0.4)
    pairs, ids, offs, data, want, _ = run_both(ctx, w, mode, alpha=0.75)
    assert len(pairs) > 10
    assert np.array_equal(pairs, want.pairs)
    assert np.array_equal(ids, want.C.ids) and np.array_equal(offs, want.C.offsets)
    assert bits_equal(data, want.C.data)


def test_c3_screening_bit_exact(ctx):
    w = W.c3(seed=3, scale=0.1, v_keep=0.1, t_keep=1e-4, screen_eps=1e-3)
    for norm in (sht.BlockNorm.FROBENIUS, sht.BlockNorm.MAXABS):
        pairs, ids, offs, data, want, _ = run_both(ctx, w, sht.Mode.PLAIN_FP64, eps=w.screen_eps, norm=norm)
        assert np.array_equal(pairs, want.pairs)
        assert np.array_equal(ids, want.C.ids)
        assert bits_equal(data, want.C.data)


def test_existing_c_union_and_beta(ctx):
    w = W.c0(seed=9, nblocks=8, p=0.35)
    # C starts with a few blocks of its own, some outside the product's pattern
    rng = np.random.default_rng(1)
    grid = int(np.prod([len(b) for b in w.C.block_sizes]))
    cid = np.sort(rng.choice(grid, 40, replace=False)).astype(np.int64)
    Ch = W.build_tensor(rng, w.C.block_sizes, lambda c: np.isin(np.arange(grid), cid), None, "normal")
    for beta in (0.0, 1.0, -0.5):
        pairs, ids, offs, data, want, _ = run_both(ctx, w, sht.Mode.PLAIN_FP64, alpha=2.0, beta=beta, Cinit=Ch)
        assert np.array_equal(ids, want.C.ids) and np.array_equal(offs, want.C.offsets)
        assert bits_equal(data, want.C.data), beta


def test_repeated_execute_accumulates(ctx):
    w = W.c0(seed=4, nblocks=6, p=0.4)
    A, B, C = dev(ctx, w.A), dev(ctx, w.B), dev(ctx, w.C)
    plan = sht.Plan(ctx, w.expr, A, B, C)
    plan.execute(1.0, 0.0)
    first = C.download().copy()
    plan.execute(1.0, 1.0)
    plan.execute(1.0, 1.0, graph=False)
    want = oracle.contract(w.expr, 1.0, host(w.A), host(w.B), 0.0, host(w.C))
    r2 = oracle.contract(w.expr, 1.0, host(w.A), host(w.B), 1.0, want.C)
    r3 = oracle.contract(w.expr, 1.0, host(w.A), host(w.B), 1.0, r2.C)
    assert bits_equal(first, want.C.data)
    assert bits_equal(C.download(), r3.C.data)


def test_graph_replay_matches_direct(ctx):
    import torch
    w = W.c1(seed=5, scale=0.3, occupancy=0.3)
    A, B, C = dev(ctx, w.A), dev(ctx, w.B), dev(ctx, w.C)
    plan = sht.Plan(ctx, w.expr, A, B, C, mode=sht.Mode.BATCHED_FP64)
    s = torch.cuda.Stream()
    for _ in range(3):
        plan.execute(1.0, 0.0, stream=s, graph=True)
    s.synchronize()
    want = oracle.contract(w.expr, 1.0, host(w.A), host(w.B), 0.0, host(w.C))
    assert bits_equal(C.download(), want.C.data)


def test_contract_entry_point_and_empty(ctx):
    w = W.c0(seed=6, nblocks=5, p=0.5)
    A, B, C = dev(ctx, w.A), dev(ctx, w.B), dev(ctx, w.C)
    rep = sht.contract(ctx, w.expr, 1.0, A, B, 0.0, C)
    want = oracle.contract(w.expr, 1.0, host(w.A), host(w.B), 0.0, host(w.C))
    assert rep["npairs"] == len(want.pairs)
    assert bits_equal(C.download(), want.C.data)
    E = dev(ctx, W.empty_tensor(w.A.block_sizes))
    C2 = dev(ctx, w.C)
    rep = sht.contract(ctx, w.expr, 1.0, E, B, 0.0, C2)
    assert rep["npairs"] == 0 and C2.get_nb_nzblocks_local() == 0


def test_contract_errors(ctx):
    w = W.c0(seed=6, nblocks=5, p=0.5)
    A, B, C = dev(ctx, w.A), dev(ctx, w.B), dev(ctx, w.C)
    with pytest.raises(sht.ShtError) as ei:
        sht.contract(ctx, "ijl, lk -> ikj", 1.0, A, B, 0.0, C)
    assert ei.value.status == sht.Status.ERR_SIZE
    with pytest.raises(sht.ShtError) as ei:
        sht.contract(ctx, "ijl, lk", 1.0, A, B, 0.0, C)
    assert ei.value.status == sht.Status.ERR_PARSE
    with pytest.raises(sht.ShtError):
        sht.contract(ctx, w.expr, 1.0, A, B, 0.0, A)


def test_autotune_keeps_results_bit_exact(ctx):
    w = W.c1(seed=8, scale=0.35, occupancy=0.35)
    A, B, C = dev(ctx, w.A), dev(ctx, w.B), dev(ctx, w.C)
    plan = sht.Plan(ctx, w.expr, A, B, C, mode=sht.Mode.BATCHED_FP64)
    plan.autotune()
    plan.execute(1.0, 0.0)
    want = oracle.contract(w.expr, 1.0, host(w.A), host(w.B), 0.0, host(w.C))
    assert bits_equal(C.download(), want.C.data)
    assert np.array_equal(plan.pairs(), want.pairs)


@pytest.mark.parametrize("expr,perm", [("ijl, lk -> kji", None), ("lij, kl -> ikj", None)])
def test_permuted_layouts_bit_exact(ctx, expr, perm):
    # contracted mode first in A (k-fast gathers) and permuted output modes
    rng = np.random.default_rng(21)
    sizes = {c: list(map(int, rng.integers(3, 12, 5))) for c in "ijkl"}
    ta, tb, tc = expr.replace(" ", "").replace("->", ",").split(",")
    A = W.build_tensor(rng, [sizes[c] for c in ta], lambda c: rng.random(len(c[0])) < 0.4, None, "normal")
    B = W.build_tensor(rng, [sizes[c] for c in tb], lambda c: rng.random(len(c[0])) < 0.4, None, "normal")
    wl = W.Workload("perm", expr, A, B, W.empty_tensor([sizes[c] for c in tc]))
    for mode in MODES:
        pairs, ids, offs, data, want, _ = run_both(ctx, wl, mode, alpha=-1.5)
        assert np.array_equal(pairs, want.pairs)
        assert np.array_equal(ids, want.C.ids)
        assert bits_equal(data, want.C.data)


@pytest.mark.parametrize("mode", MODES)
def test_signed_zero_and_padding_preserved(ctx, mode):
    # zero A blocks, negative beta on new (zero-filled) C blocks and contracted extents that are
    # not multiples of 4: every bit, including the sign of zero, must match the oracle
    rng = np.random.default_rng(5)
    i, l, k = [3, 5, 7], [5, 6, 7], [2, 9]
    A = W.build_tensor(rng, [i, l], lambda c: rng.random(len(c[0])) < 0.7, None, "normal")
    A.data[: A.data.size // 2] = 0.0
    B = W.build_tensor(rng, [l, k], lambda c: rng.random(len(c[0])) < 0.7, None, "normal")
    wl = W.Workload("z", "il, lk -> ik", A, B, W.empty_tensor([i, k]))
    for beta in (-1.0, -0.0, 0.5):
        pairs, ids, offs, data, want, _ = run_both(ctx, wl, mode, alpha=1.0, beta=beta)
        assert bits_equal(data, want.C.data), beta
