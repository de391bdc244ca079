"""Block-sparse tensor storage, norms, filter/compress and the device pool on the B200."""
import numpy as np
import pytest

import oracle
import shtensor_b200 as sht
from shtensor_b200 import workloads as W

pytestmark = pytest.mark.gpu

BS4 = [[4, 5, 3, 4], [5, 5, 8, 9, 2], [5, 6, 3, 7, 7, 9], [4, 3, 2]]


def test_reserve_all_layout(ctx):
    t = sht.Tensor(ctx, BS4, np.float32).reserve_all()
    assert t.get_nb_nzblocks_local() == 360
    ids, offs, rows = t.get_sparse_info()
    nblk = [len(b) for b in BS4]
    grid = np.arange(360)
    gstride = np.concatenate([[1], np.cumprod(nblk)[:-1]])
    want = oracle.reserve(BS4, [list((grid // gstride[d]) % nblk[d]) for d in range(4)])
    assert np.array_equal(ids, want.ids) and np.array_equal(offs, want.offsets) and np.array_equal(rows, want.rows)
    assert not t.download().any()


def test_reserve_index_lists_and_errors(ctx):
    bs = BS4[:3]
    idx = [[0, 0, 0, 1, 2, 2, 3, 3, 3], [0, 0, 1, 0, 2, 3, 2, 3, 4], [0, 1, 1, 0, 1, 2, 0, 1, 2]]
    t = sht.Tensor(ctx, bs).reserve(idx)
    want = oracle.reserve(bs, idx)
    ids, offs, rows = t.get_sparse_info()
    assert np.array_equal(ids, want.ids) and np.array_equal(offs, want.offsets) and np.array_equal(rows, want.rows)
    with pytest.raises(sht.ShtError):
        sht.Tensor(ctx, bs).reserve([[0, 0], [1, 1], [2, 2]])
    with pytest.raises(sht.ShtError):
        sht.Tensor(ctx, [[2, 3]])  # order < 2


def test_reserve_device_matches_host_reserve(ctx):
    # index lists in device memory, in no particular order: the same sorted ids, offsets and
    # rows as the host reserve and as the oracle's restatement; then used as a contraction
    # operand, the same result bits as the host-reserved tensor
    import torch
    w = W.c0(seed=12, nblocks=10, p=0.35)
    rng = np.random.default_rng(13)
    lists = w.A.index_lists()
    perm = rng.permutation(len(w.A.ids))
    idx = np.stack([np.asarray(v, np.int32)[perm] for v in lists])
    Ah = sht.Tensor(ctx, w.A.block_sizes).reserve(lists)
    Ad = sht.Tensor(ctx, w.A.block_sizes).reserve_device(torch.from_numpy(idx).cuda())
    want = oracle.reserve(w.A.block_sizes, [list(v) for v in lists])
    for t in (Ah, Ad):
        ids, offs, rows = t.get_sparse_info()
        assert np.array_equal(ids, want.ids) and np.array_equal(offs, want.offsets) and np.array_equal(rows, want.rows)
    assert Ad.info() == Ah.info()
    assert not Ad.download().any()
    Ah.upload(w.A.data)
    Ad.upload(w.A.data)
    B = sht.Tensor(ctx, w.B.block_sizes).reserve(w.B.index_lists())
    B.upload(w.B.data)
    Ch, Cd = sht.Tensor(ctx, w.C.block_sizes), sht.Tensor(ctx, w.C.block_sizes)
    sht.contract(ctx, w.expr, 1.0, Ah, B, 0.0, Ch, mode=sht.Mode.PLAIN_FP64)
    sht.contract(ctx, w.expr, 1.0, Ad, B, 0.0, Cd, mode=sht.Mode.PLAIN_FP64)
    assert np.array_equal(Ch.get_sparse_info()[0], Cd.get_sparse_info()[0])
    assert np.array_equal(Ch.download().view(np.uint64), Cd.download().view(np.uint64))


def test_reserve_device_errors_and_empty(ctx):
    import torch
    bs = BS4[:3]
    dup = torch.tensor([[0, 1, 0], [1, 2, 1], [2, 0, 2]], dtype=torch.int32, device="cuda")
    with pytest.raises(sht.ShtError) as ei:
        sht.Tensor(ctx, bs).reserve_device(dup)
    assert ei.value.status == sht.Status.ERR_INVALID
    out = torch.tensor([[0, 4], [1, 1], [2, 6]], dtype=torch.int32, device="cuda")  # 4 and 6 are past the grid
    with pytest.raises(sht.ShtError) as ei:
        sht.Tensor(ctx, bs).reserve_device(out)
    assert ei.value.status == sht.Status.ERR_INVALID
    t = sht.Tensor(ctx, bs).reserve_device(torch.zeros((3, 0), dtype=torch.int32, device="cuda"))
    assert t.info() == (0, 0)
    # one block of 2048 x 1024 x 1024 = 2^31 elements: rejected by the device-side size check
    # before any data is allocated
    big = sht.Tensor(ctx, [[2048, 3], [1024, 2], [1024]])
    with pytest.raises(sht.ShtError) as ei:
        big.reserve_device(torch.zeros((3, 1), dtype=torch.int32, device="cuda"))
    assert ei.value.status == sht.Status.ERR_UNSUPPORTED
    small = torch.tensor([[1], [1], [0]], dtype=torch.int32, device="cuda")  # a 3 x 2 x 1024 block
    assert big.reserve_device(small).info() == (1, 3 * 2 * 1024)


def test_reserve_device_on_side_stream_then_upload(ctx):
    # reserve on a non-blocking stream, upload on the legacy default stream: the reserve's zero
    # fill of the data must not land after the upload
    import torch
    w = W.c0(seed=21, nblocks=12, p=0.5)
    idx = torch.from_numpy(np.stack([np.asarray(v, np.int32) for v in w.A.index_lists()])).cuda()
    side = torch.cuda.Stream()
    for _ in range(3):
        t = sht.Tensor(ctx, w.A.block_sizes).reserve_device(idx, stream=side)
        t.upload(w.A.data)
        assert np.array_equal(t.download(), w.A.data)


@pytest.mark.parametrize("norm", [sht.BlockNorm.FROBENIUS, sht.BlockNorm.MAXABS, sht.BlockNorm.FROBENIUS_REFCOMPAT])
def test_norms_bit_exact(ctx, norm):
    w = W.c0(seed=2, nblocks=6, p=0.5)
    t = sht.Tensor(ctx, w.A.block_sizes).reserve(w.A.index_lists()).upload(w.A.data)
    got = t.norms(norm)
    sizes = np.diff(np.concatenate([w.A.offsets, [w.A.nnz]]))
    want = [oracle.block_norm(w.A.data[o:o + s], int(norm)) for o, s in zip(w.A.offsets, sizes)]
    assert np.array_equal(got, np.array(want))


def test_filter_compress_like_reference(ctx):
    nblk = [len(b) for b in BS4]
    t = sht.Tensor(ctx, BS4, np.float32).reserve_all()
    ids, offs, _ = t.get_sparse_info()
    sizes = np.diff(np.concatenate([offs, [t.nnz]]))
    data = np.repeat((ids % 2).astype(np.float32), sizes)
    t.upload(data)
    t.filter(1e-6, sht.BlockNorm.FROBENIUS, compress=False)
    marked, _, _ = t.get_sparse_info()
    assert np.array_equal(marked < 0, ids % 2 == 0)
    t.compress()
    ids2, offs2, _ = t.get_sparse_info()
    assert np.all(ids2 >= 0) and len(ids2) == 180
    assert np.array_equal(ids2, ids[ids % 2 == 1])
    assert np.all(t.download() == 1.0) and t.nnz == sizes[ids % 2 == 1].sum()
    assert np.array_equal(offs2, np.concatenate([[0], np.cumsum(sizes[ids % 2 == 1])[:-1]]))
    del nblk


def test_filter_values_preserved_fp64(ctx):
    w = W.c0(seed=4, nblocks=6, p=0.6)
    t = sht.Tensor(ctx, w.A.block_sizes).reserve(w.A.index_lists()).upload(w.A.data)
    norms = t.norms(sht.BlockNorm.MAXABS)
    eps = float(np.median(norms))
    t.filter(eps, sht.BlockNorm.MAXABS, compress=True)
    h = oracle.HostTensor(w.A.block_sizes, w.A.ids.copy(), w.A.offsets.copy(), w.A.data.copy())
    want = oracle.filter_blocks(h, eps, 1, compress=True)
    ids, offs, rows = t.get_sparse_info()
    assert np.array_equal(ids, want.ids) and np.array_equal(offs, want.offsets)
    assert np.array_equal(t.download(), want.data) and np.array_equal(rows, want.rows)


def test_pool_accounting_follows_reference_spec():
    # test/test_mempool.cpp:30-114 with chunk header H and 16-byte alignment
    H = 64
    pool_memory = 1024 * 8 + H
    with sht.Context(pool_memory) as c:
        c.configure_pool(H, 16)
        assert c.get_free_mem() == pool_memory - H
        p0 = c.allocate(100 * 8)
        p1 = c.allocate(100 * 4)
        assert c.get_free_mem() == pool_memory - 800 - 400 - 3 * H
        c.free(p0)
        assert c.get_free_mem() == pool_memory - 400 - 3 * H
        p2 = c.allocate(100 * 8)
        assert p2 == p0  # first fit reuses the freed chunk
        c.free(p2)
        c.free(p1)
        assert c.get_free_mem() == pool_memory - H
        u = c.allocate(pool_memory - H)
        u = c.reallocate(u, 256)
        assert c.get_free_mem() == pool_memory - 256 - 2 * H
        u = c.reallocate(u, 512)
        assert c.get_free_mem() == pool_memory - 512 - 2 * H
        u = c.reallocate(u, pool_memory - H)
        assert c.get_free_mem() == 0
        with pytest.raises(sht.ShtError) as ei:
            c.allocate(16)
        assert ei.value.status == sht.Status.ERR_OOM
        c.free(u)
        assert c.get_free_mem() == pool_memory - H


def test_handles_outlive_finalize():
    # destroying tensors and plans after the context was finalised must be safe
    w = W.c0(seed=3, nblocks=4, p=0.5)
    c = sht.Context(1 << 28)
    A = sht.Tensor(c, w.A.block_sizes).reserve(w.A.index_lists()).upload(w.A.data)
    B = sht.Tensor(c, w.B.block_sizes).reserve(w.B.index_lists()).upload(w.B.data)
    C = sht.Tensor(c, w.C.block_sizes).reserve([[] for _ in w.C.block_sizes])
    plan = sht.Plan(c, w.expr, A, B, C)
    plan.execute()
    c.close()
    plan.close()
    del A, B, C
