"""Serving loop on the B200: continuous batching of block-sparse contractions.

The bar: every request's result is bit-identical to the same contraction run alone through
sht_contract (batched and plain FP64 give the same bits), whatever the mix it was batched
with; requests that write the same tensor apply in submission order; admission defers
requests when the pool is short instead of failing them; a bad request fails alone."""
import time

import numpy as np
import pytest

import shtensor_b200 as sht
from shtensor_b200 import workloads as W
from tests.bits import bits_equal

pytestmark = pytest.mark.gpu


def dev(ctx, h):
    t = sht.Tensor(ctx, h.block_sizes)
    t.reserve(h.index_lists() if len(h.ids) else [[] for _ in h.block_sizes])
    if h.nnz:
        t.upload(h.data)
    return t


def alone(ctx, w, mode, alpha=1.0, beta=0.0, Cinit=None):
    A, B = dev(ctx, w.A), dev(ctx, w.B)
    C = dev(ctx, Cinit if Cinit is not None else w.C)
    sht.contract(ctx, w.expr, alpha, A, B, beta, C, w.screen_eps, mode=mode)
    ids, offs, _ = C.get_sparse_info()
    return ids, offs, C.download()


def small_mix(seed, n):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        k = i % 4
        s = int(rng.integers(1, 1 << 30))
        if k == 0:
            out.append(W.c0(seed=s, nblocks=int(rng.integers(4, 12)), p=float(rng.uniform(0.05, 0.4))))
        elif k == 1:
            out.append(W.c1(seed=s, scale=float(rng.uniform(0.08, 0.2)), occupancy=float(rng.uniform(0.05, 0.4))))
        elif k == 2:
            out.append(W.c2(seed=s, scale=float(rng.uniform(0.08, 0.2)), occupancy=float(rng.uniform(0.05, 0.4))))
        else:
            out.append(W.c3(seed=s, scale=0.0625))
    return out


def test_mix_equals_alone(ctx):
    ws = small_mix(11, 12)
    with sht.Server(ctx) as srv:
        held = []
        for w in ws:
            A, B, C = dev(ctx, w.A), dev(ctx, w.B), dev(ctx, w.C)
            held.append((A, B, C))
        rids = [srv.submit(w.expr, 1.0, A, B, 0.0, C, w.screen_eps) for w, (A, B, C) in zip(ws, held)]
        reps = [srv.wait(r, 60) for r in rids]
        st = srv.stats()
    assert st["completed"] == len(ws) and st["failed"] == 0
    assert max(r["batch_size"] for r in reps) > 1, "requests submitted together should share a launch"
    for w, (A, B, C), rep in zip(ws, held, reps):
        got_ids, got_offs, _ = C.get_sparse_info()
        got = C.download()
        for mode in (sht.Mode.BATCHED_FP64, sht.Mode.PLAIN_FP64):
            ids, offs, data = alone(ctx, w, mode)
            assert np.array_equal(got_ids, ids) and np.array_equal(got_offs, offs), w.name
            assert bits_equal(got, data), (w.name, mode)
        assert rep["flops"] >= 0 and rep["latency_ms"] >= rep["run_ms"] >= 0
    assert sum(r["flops"] for r in reps) > 0


def test_split_mix_equals_split_alone(ctx):
    # a split-form server: every result bit-identical to sht_contract in split mode alone; a
    # request whose operand holds a NaN is served in the batched FP64 form (its report says so)
    # and equals the FP64 forms alone
    ws = small_mix(17, 8)
    bad = W.c0(seed=5, nblocks=5, p=0.5)
    bad.A.data[7] = np.nan
    ws.append(bad)
    with sht.Server(ctx, mode=sht.Mode.SPLIT) as srv:
        held = [(dev(ctx, w.A), dev(ctx, w.B), dev(ctx, w.C)) for w in ws]
        rids = [srv.submit(w.expr, 1.0, A, B, 0.0, C, w.screen_eps) for w, (A, B, C) in zip(ws, held)]
        reps = [srv.wait(r, 60) for r in rids]
        st = srv.stats()
    assert st["completed"] == len(ws) and st["failed"] == 0
    assert [r["form"] for r in reps[:-1]] == [int(sht.Mode.SPLIT)] * (len(ws) - 1)
    assert reps[-1]["form"] == int(sht.Mode.BATCHED_FP64)
    assert max(r["batch_size"] for r in reps[:-1]) > 1, "split requests submitted together should share a launch"
    for w, (A, B, C), rep in zip(ws, held, reps):
        got_ids, got_offs, _ = C.get_sparse_info()
        got = C.download()
        ids, offs, data = alone(ctx, w, sht.Mode.SPLIT if rep["form"] == int(sht.Mode.SPLIT) else sht.Mode.PLAIN_FP64)
        assert np.array_equal(got_ids, ids) and np.array_equal(got_offs, offs), w.name
        assert bits_equal(got, data), w.name


def test_alpha_beta_and_existing_c(ctx):
    rng = np.random.default_rng(3)
    ws = [W.c1(seed=21, scale=0.12, occupancy=0.2), W.c0(seed=4, nblocks=8, p=0.3)]
    cases = [(0.75, 2.0), (-1.5, 0.0)]
    with sht.Server(ctx) as srv:
        runs = []
        for w, (alpha, beta) in zip(ws, cases):
            # C starts with a random pattern and random values
            Cp = W.build_tensor(rng, w.C.block_sizes, lambda c: rng.random(len(c[0])) < 0.3, None, "normal")
            A, B, C = dev(ctx, w.A), dev(ctx, w.B), dev(ctx, Cp)
            runs.append((w, alpha, beta, Cp, C, srv.submit(w.expr, alpha, A, B, beta, C), (A, B)))
        for w, alpha, beta, Cp, C, rid, _ in runs:
            srv.wait(rid, 60)
            ids, offs, data = alone(ctx, w, sht.Mode.PLAIN_FP64, alpha, beta, Cinit=Cp)
            got_ids, got_offs, _ = C.get_sparse_info()
            assert np.array_equal(got_ids, ids) and np.array_equal(got_offs, offs)
            assert bits_equal(C.download(), data)


def test_same_output_applies_in_order(ctx):
    w1 = W.c1(seed=5, scale=0.1, occupancy=0.3)
    rng = np.random.default_rng(6)
    # a second contraction over the same grids with other patterns and values
    A2h = W.build_tensor(rng, w1.A.block_sizes, lambda c: rng.random(len(c[0])) < 0.3, None, "normal")
    B2h = W.build_tensor(rng, w1.B.block_sizes, lambda c: rng.random(len(c[0])) < 0.3, None, "normal")
    # both write C; the second reads C's pattern after the first grew it
    A1, B1, A2, B2 = dev(ctx, w1.A), dev(ctx, w1.B), dev(ctx, A2h), dev(ctx, B2h)
    Cs = dev(ctx, w1.C)
    with sht.Server(ctx) as srv:
        r1 = srv.submit(w1.expr, 1.0, A1, B1, 0.0, Cs)
        r2 = srv.submit(w1.expr, 0.5, A2, B2, 1.0, Cs)
        rep1 = srv.wait(r1, 60)
        rep2 = srv.wait(r2, 60)
    assert rep2["batch"] > rep1["batch"]
    Cr = dev(ctx, w1.C)
    sht.contract(ctx, w1.expr, 1.0, A1, B1, 0.0, Cr, mode=sht.Mode.PLAIN_FP64)
    sht.contract(ctx, w1.expr, 0.5, A2, B2, 1.0, Cr, mode=sht.Mode.PLAIN_FP64)
    assert np.array_equal(Cs.get_sparse_info()[0], Cr.get_sparse_info()[0])
    assert bits_equal(Cs.download(), Cr.download())


def test_same_grid_shared_inputs_distinct_outputs(ctx):
    # one A, B pair read by many requests at once, each into its own C
    w = W.c1(seed=9, scale=0.15, occupancy=0.25)
    A, B = dev(ctx, w.A), dev(ctx, w.B)
    ids, offs, want = alone(ctx, w, sht.Mode.PLAIN_FP64)
    Cs = [dev(ctx, w.C) for _ in range(8)]
    with sht.Server(ctx, max_batch=4) as srv:
        rids = [srv.submit(w.expr, 1.0, A, B, 0.0, C) for C in Cs]
        reps = [srv.wait(r, 60) for r in rids]
        st = srv.stats()
    assert max(r["batch_size"] for r in reps) <= 4
    assert st["batches"] >= 2
    for C in Cs:
        assert bits_equal(C.download(), want)


def test_admission_defers_under_memory_pressure():
    # c3 at this size: V (the A operand) ~165 MB, its matrix-form copy ~210 MB per request.
    # In a 512 MB pool one request fits beside the inputs, two do not.
    w = W.c3(seed=40, scale=0.06)
    small = sht.Context(512 << 20)
    try:
        A, B = dev(small, w.A), dev(small, w.B)
        Cs = [dev(small, w.C) for _ in range(4)]
        with sht.Server(small) as srv:
            rids = [srv.submit(w.expr, 1.0, A, B, 0.0, C, w.screen_eps) for C in Cs]
            reps = [srv.wait(r, 60) for r in rids]
            st = srv.stats()
        assert st["completed"] == len(Cs) and st["failed"] == 0
        assert st["deferrals"] > 0 and st["max_active_seen"] == 1, st
        assert sum(r["deferrals"] for r in reps) > 0
        results = [C.download() for C in Cs]
    finally:
        small.close()
    ref_ctx = sht.Context(1 << 30)
    try:
        _, _, want = alone(ref_ctx, w, sht.Mode.PLAIN_FP64)
        for got in results:
            assert bits_equal(got, want)
    finally:
        ref_ctx.close()


def test_bad_request_fails_alone(ctx):
    good = W.c0(seed=2, nblocks=6, p=0.4)
    A, B, C = dev(ctx, good.A), dev(ctx, good.B), dev(ctx, good.C)
    C2 = dev(ctx, good.C)
    with sht.Server(ctx) as srv:
        r_bad = srv.submit("ijl, lk -> ijq", 1.0, A, B, 0.0, C2)  # q appears in no input
        r_good = srv.submit(good.expr, 1.0, A, B, 0.0, C)
        with pytest.raises(sht.ShtError) as ei:
            srv.wait(r_bad, 60)
        assert ei.value.status == sht.Status.ERR_PARSE
        srv.wait(r_good, 60)
        st = srv.stats()
    assert st["failed"] == 1 and st["completed"] == 1
    _, _, want = alone(ctx, good, sht.Mode.PLAIN_FP64)
    assert bits_equal(C.download(), want)
    with sht.Server(ctx) as srv:
        with pytest.raises(sht.ShtError):
            srv.poll(12345)


def test_poisson_stream_stats(ctx):
    ws = small_mix(17, 16)
    rng = np.random.default_rng(17)
    gaps = rng.exponential(1.0 / 400.0, len(ws))
    ins = [(dev(ctx, w.A), dev(ctx, w.B)) for w in ws]
    outs = [dev(ctx, w.C) for w in ws]
    with sht.Server(ctx) as srv:
        rids = []
        for w, (A, B), C, g in zip(ws, ins, outs, gaps):
            time.sleep(float(g))
            rids.append(srv.submit(w.expr, 1.0, A, B, 0.0, C, w.screen_eps))
        reps = [srv.wait(r, 60) for r in rids]
        st = srv.stats()
    assert st["completed"] == len(ws)
    assert 0 < st["p50_ms"] <= st["p99_ms"] <= st["max_ms"]
    assert st["gflops"] > 0 and st["mean_batch"] >= 1
    lat = sorted(r["latency_ms"] for r in reps)
    assert abs(lat[-1] - st["max_ms"]) < 1e-6
    for w, C in zip(ws, outs):
        _, _, want = alone(ctx, w, sht.Mode.BATCHED_FP64)
        assert bits_equal(C.download(), want)
