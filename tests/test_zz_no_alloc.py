"""The allocation-free Kernel<double> call (sht_kernel_call_static).

It serves callers that cannot allocate device memory (inside someone else's graph capture,
allocator-free plugin hosts, fully reserved devices): its scratch is a static device array.
This file is collected last on purpose.  It checks, through the C ABI, that two calls in a
row give the same bits as the allocating sht_kernel_call on the same inputs (the bit-exact
tolerance of the other stack-kernel tests), that they also give the frozen golden outputs of
the reference's own test cases (XMM order bit for bit, the reference LAPACK path within
1e-13), and that a stack larger than the static scratch is rejected.  It passes alone in a
fresh process and after the other tests."""
import os

import numpy as np
import pytest

import shtensor_b200 as sht
from tests.bits import bits_equal
from tests.golden import make_golden as G

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

CASES = [
    ("ik, kj -> ij", [8, 5], [5, 6], [8, 6], 1.0, 0.0, 20),
    ("ikl, lkmj -> mij", [6, 5, 7], [7, 5, 6, 6], [6, 6, 6], -0.5, 1.5, 20),
    ("iaP, jbP -> ijab", [13, 25, 48], [9, 32, 48], [13, 9, 25, 32], 1.0, 0.0, 6),
    ("ijl, lk -> kji", [7, 9, 11], [11, 13], [13, 9, 7], 2.0, 0.25, 50),
]


@pytest.fixture(scope="module")
def sctx():
    c = sht.Context(1 << 30)
    yield c
    c.close()


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_static_call_matches_allocating_call(sctx, case):
    import torch
    expr, sa, sb, sc, al, be, nops = case
    rng = np.random.default_rng(17)
    a = torch.from_numpy(rng.standard_normal(nops * int(np.prod(sa)))).cuda()
    b = torch.from_numpy(rng.standard_normal(nops * int(np.prod(sb)))).cuda()
    c0 = rng.standard_normal(nops * int(np.prod(sc)))
    k = sht.Kernel(sctx, expr, sa, sb, sc, al, be)
    want = torch.from_numpy(c0.copy()).cuda()
    k.call(a, b, want, nops)
    for _ in range(2):  # two calls in a row share the static scratch
        got = torch.from_numpy(c0.copy()).cuda()
        k.call_static(a, b, got, nops)
        torch.cuda.synchronize()
        assert bits_equal(got.cpu().numpy(), want.cpu().numpy())


@pytest.mark.parametrize("n", range(len(G.KERNEL_CASES)))
def test_static_call_matches_golden_outputs(sctx, n):
    import torch
    kc = np.load(os.path.join(GOLD, "kernel_cases.npz"))
    expr, sa, sb, sc, al, be, nops = G.KERNEL_CASES[n]
    k = sht.Kernel(sctx, expr, sa, sb, sc, al, be)
    a = torch.from_numpy(kc[f"{n}_a"]).cuda()
    b = torch.from_numpy(kc[f"{n}_b"]).cuda()
    for _ in range(2):
        c = torch.from_numpy(kc[f"{n}_c"].copy()).cuda()
        k.call_static(a, b, c, nops)
        torch.cuda.synchronize()
        got = c.cpu().numpy()
        assert bits_equal(got, kc[f"{n}_xmm"])
        ref = kc[f"{n}_lapack_ref"]
        assert np.linalg.norm(got - ref) <= 1e-13 * max(np.linalg.norm(ref), 1e-300)


def test_static_call_rejects_stacks_beyond_scratch(sctx):
    import torch
    k = sht.Kernel(sctx, "ik, kj -> ij", [64, 64], [64, 64], [64, 64])
    nops = 1000  # 1000 * (64 + 64) * 64 * 8 bytes = 62.5 MiB > 32 MiB
    a = torch.zeros(nops * 64 * 64, dtype=torch.float64, device="cuda")
    with pytest.raises(sht.ShtError) as ei:
        k.call_static(a, a, a.clone(), nops)
    assert ei.value.status == sht.Status.ERR_SIZE
