"""Block-sparse layer of the oracle (CPU): storage layout, filter/compress, norms, and the
contraction's canonical pair order and values against numpy.einsum on densified tensors."""
import os

import numpy as np
import pytest

import oracle
from shtensor_b200 import workloads as W

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def host(t):
    return oracle.HostTensor(t.block_sizes, t.ids, t.offsets, t.data)


def test_reserve_all_matches_reference_test_tensor():
    # test/test_tensor.cpp:39-73: dims {4,5,3,4},{5,5,8,9,2},{5,6,3,7,7,9},{4,3,2} -> 360 blocks
    bs = [[4, 5, 3, 4], [5, 5, 8, 9, 2], [5, 6, 3, 7, 7, 9], [4, 3, 2]]
    nblk = [len(b) for b in bs]
    grid = np.arange(int(np.prod(nblk)))
    gstride = np.concatenate([[1], np.cumprod(nblk)[:-1]])
    idx = [list((grid // gstride[d]) % nblk[d]) for d in range(4)]
    t = oracle.reserve(bs, idx)
    assert len(t.ids) == 360
    assert np.array_equal(t.ids, np.arange(360))
    sizes = [int(np.prod([bs[d][(i // gstride[d]) % nblk[d]] for d in range(4)])) for i in range(360)]
    assert np.array_equal(t.offsets, np.concatenate([[0], np.cumsum(sizes)[:-1]]))
    assert t.data.size == sum(sizes)


def test_reserve_sorts_and_rejects_duplicates():
    bs = [[4, 5, 3, 4], [5, 5, 8, 9, 2], [5, 6, 3, 7, 7, 9]]
    # test/test_tensor.cpp:55-59 index lists
    idx = [[0, 0, 0, 1, 2, 2, 3, 3, 3], [0, 0, 1, 0, 2, 3, 2, 3, 4], [0, 1, 1, 0, 1, 2, 0, 1, 2]]
    t = oracle.reserve(bs, idx)
    assert np.all(np.diff(t.ids) > 0)
    # rows: count prefix of mode-0 indices (BaseTensor.cpp:200-208)
    assert list(t.rows) == [0, 3, 4, 6]
    with pytest.raises(oracle.OracleError, match="duplicate"):
        oracle.reserve(bs, [[0, 0], [1, 1], [2, 2]])
    with pytest.raises(oracle.OracleError, match="range"):
        oracle.reserve(bs, [[4], [0], [0]])


def test_filter_alternating_blocks_like_reference():
    # test/test_tensor.cpp:78-120: blocks with even id zero, odd id one; FROBENIUS eps 1e-6
    bs = [[4, 5, 3, 4], [5, 5, 8, 9, 2], [5, 6, 3, 7, 7, 9], [4, 3, 2]]
    nblk = [len(b) for b in bs]
    grid = np.arange(int(np.prod(nblk)))
    gstride = np.concatenate([[1], np.cumprod(nblk)[:-1]])
    t = oracle.reserve(bs, [list((grid // gstride[d]) % nblk[d]) for d in range(4)])
    sizes = np.diff(np.concatenate([t.offsets, [t.data.size]]))
    t.data = np.repeat((t.ids % 2).astype(np.float64), sizes)
    marked = oracle.filter_blocks(t, 1e-6, 0, compress=False)
    assert np.array_equal(marked.ids < 0, t.ids % 2 == 0)
    comp = oracle.filter_blocks(t, 1e-6, 0, compress=True)
    assert np.all(comp.ids >= 0) and len(comp.ids) == 180
    assert np.all(comp.data == 1.0) and comp.data.size == sizes[t.ids % 2 == 1].sum()


def test_norms():
    rng = np.random.default_rng(0)
    x = rng.standard_normal(1001)
    assert oracle.block_norm(x, 1) == np.abs(x).max()
    assert abs(oracle.block_norm(x, 0) - np.linalg.norm(x)) <= 1e-14 * np.linalg.norm(x)
    # reference int accumulator: truncates every partial sum
    acc = 0
    for v in x:
        acc = int(acc + v * v)
    assert oracle.block_norm(x, 2) == np.sqrt(acc)


@pytest.mark.parametrize("name", ["c0", "c1", "c3"])
def test_golden_blocksparse_reproduced(name):
    d = np.load(os.path.join(GOLD, "blocksparse.npz"))

    def ten(prefix):
        nb = d[f"{name}_{prefix}_nb"]
        flat = d[f"{name}_{prefix}_bs"]
        bs, pos = [], 0
        for n in nb:
            bs.append(list(map(int, flat[pos:pos + n])))
            pos += n
        if f"{name}_{prefix}_ids" not in d:
            return oracle.HostTensor(bs, np.zeros(0, np.int64), np.zeros(0, np.int64), np.zeros(0))
        ids = d[f"{name}_{prefix}_ids"]
        t = oracle.reserve(bs, W.HostBlockSparse(bs, ids, None, None).index_lists())
        t.data = d[f"{name}_{prefix}_data"]
        return t

    A, B, C = ten("A"), ten("B"), ten("C")
    r = oracle.contract(str(d[f"{name}_expr"][0]), 1.0, A, B, 0.0, C, eps=float(d[f"{name}_eps"][0]))
    assert np.array_equal(r.pairs, d[f"{name}_pairs"])
    assert np.array_equal(r.C.ids, d[f"{name}_cids"])
    assert np.array_equal(r.C.offsets, d[f"{name}_coffs"])
    assert np.array_equal(r.C.data, d[f"{name}_cdata"])
    ref = d[f"{name}_cdata_ref"]
    assert np.linalg.norm(r.C.data - ref) <= 1e-13 * np.linalg.norm(ref)


def _check_against_einsum(w, eps=0.0):
    A, B, C = host(w.A), host(w.B), host(w.C)
    r = oracle.contract(w.expr, w.alpha, A, B, w.beta, C, eps=eps)
    # canonical order: (idC, idA, idB) ascending and complete
    p = r.pairs
    if len(p):
        key = np.lexsort((p[:, 2], p[:, 1], p[:, 0]))
        assert np.array_equal(key, np.arange(len(p)))
    assert np.array_equal(np.unique(p[:, 0]) if len(p) else p[:, 0], r.C.ids)
    if eps == 0.0:
        dC = oracle.densify(r.C)
        want = w.alpha * np.einsum(w.expr.replace(" ", ""), oracle.densify(A), oracle.densify(B))
        assert np.linalg.norm(dC - want) <= 1e-14 * max(np.linalg.norm(want), 1e-300)
    return r


def test_contract_c0_small_vs_einsum():
    r = _check_against_einsum(W.c0(seed=3, nblocks=8, p=0.3))
    assert len(r.pairs) > 0


def test_contract_c1_small_vs_einsum():
    r = _check_against_einsum(W.c1(seed=3, scale=0.25, occupancy=0.5))
    assert len(r.pairs) > 0


def test_contract_existing_c_and_beta():
    w = W.c0(seed=5, nblocks=6, p=0.4)
    A, B, C0 = host(w.A), host(w.B), host(w.C)
    r1 = oracle.contract(w.expr, 1.0, A, B, 0.0, C0)
    # second contraction into the result with beta=0.5: pattern unchanged, values scaled+added
    r2 = oracle.contract(w.expr, 2.0, A, B, 0.5, r1.C)
    assert np.array_equal(r2.C.ids, r1.C.ids)
    assert np.allclose(r2.C.data, 0.5 * r1.C.data + 2.0 * r1.C.data, rtol=1e-13, atol=1e-13)


def test_contract_empty_operands():
    w = W.c0(seed=5, nblocks=5, p=0.4)
    empty = W.empty_tensor(w.A.block_sizes)
    r = oracle.contract(w.expr, 1.0, host(empty), host(w.B), 0.0, host(w.C))
    assert len(r.pairs) == 0 and len(r.C.ids) == 0
