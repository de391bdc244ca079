"""Kernel<T> stack contraction on the B200 (parity with the oracle through the C ABI).

Bar: bit-exact against the XMM-order restatement (FP64 and FP32), and within 1e-13 relative
of the reference LAPACK path (reshape + OpenBLAS dgemm) frozen in tests/golden."""
import os

import numpy as np
import pytest

import oracle
import shtensor_b200 as sht
from tests.bits import bits_equal
from tests.golden import make_golden as G

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.fixture(scope="module")
def kc():
    return np.load(os.path.join(GOLD, "kernel_cases.npz"))


@pytest.mark.parametrize("n", range(len(G.KERNEL_CASES)))
def test_stack_fp64_device_bit_exact(ctx, kc, n):
    import torch
    expr, sa, sb, sc, al, be, nops = G.KERNEL_CASES[n]
    k = sht.Kernel(ctx, expr, sa, sb, sc, al, be, sht.KernelType.XMM)
    a = torch.from_numpy(kc[f"{n}_a"]).cuda()
    b = torch.from_numpy(kc[f"{n}_b"]).cuda()
    c = torch.from_numpy(kc[f"{n}_c"].copy()).cuda()
    k.call(a, b, c, nops)
    torch.cuda.synchronize()
    got = c.cpu().numpy()
    assert bits_equal(got, kc[f"{n}_xmm"])
    ref = kc[f"{n}_lapack_ref"]
    assert np.linalg.norm(got - ref) <= 1e-13 * max(np.linalg.norm(ref), 1e-300)


@pytest.mark.parametrize("n", range(len(G.KERNEL_CASES)))
def test_stack_fp32_host_pointers_bit_exact(ctx, kc, n):
    expr, sa, sb, sc, al, be, nops = G.KERNEL_CASES[n]
    k = sht.Kernel(ctx, expr, sa, sb, sc, al, be, sht.KernelType.LAPACK, dtype=np.float32)
    c = kc[f"{n}_c"].astype(np.float32)
    k.call(kc[f"{n}_a"].astype(np.float32), kc[f"{n}_b"].astype(np.float32), c, nops)
    assert bits_equal(c, kc[f"{n}_xmm32"])


def test_stack_large_stack_and_big_blocks(ctx):
    import torch
    rng = np.random.default_rng(11)
    for expr, sa, sb, sc, nops in [("ikl, ljk -> ij", [8, 8, 8], [8, 8, 8], [8, 8], 10000),
                                   ("iaP, jbP -> ijab", [13, 32, 64], [9, 25, 64], [13, 9, 32, 25], 3),
                                   ("ik, kj -> ij", [200, 70], [70, 150], [200, 150], 5)]:
        a = rng.standard_normal(nops * int(np.prod(sa)))
        b = rng.standard_normal(nops * int(np.prod(sb)))
        c = rng.standard_normal(nops * int(np.prod(sc)))
        want = oracle.kernel_xmm(expr, sa, sb, sc, 1.25, -0.5, a, b, c.copy(), nops)
        k = sht.Kernel(ctx, expr, sa, sb, sc, 1.25, -0.5)
        dc = torch.from_numpy(c).cuda()
        k.call(torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda(), dc, nops)
        assert bits_equal(dc.cpu().numpy(), want), expr


def test_kernel_errors(ctx):
    with pytest.raises(sht.ShtError) as ei:
        sht.Kernel(ctx, "ij, ij ->", [2, 2], [2, 2], [2, 2])
    assert ei.value.status == sht.Status.ERR_PARSE
    with pytest.raises(sht.ShtError) as ei:
        sht.Kernel(ctx, "ij, jk -> ik", [2, 3], [4, 2], [2, 2])
    assert ei.value.status == sht.Status.ERR_SIZE
    k = sht.Kernel(ctx, "ij, jk -> ik", [2, 2], [2, 2], [2, 2])
    assert "map_row" in k.get_info()
    with pytest.raises(sht.ShtError):
        k.call(np.zeros(4), np.zeros(4), np.zeros(4), -1)


def test_measured_peaks_are_plausible(ctx):
    # the in-run roofline denominators: FP64 FMA and dense INT8 tensor-core rates of this GPU
    fp64 = sht.measure_peak(ctx, "fp64")
    int8 = sht.measure_peak(ctx, "int8")
    assert 5.0 < fp64 < 200.0, fp64
    assert 100.0 < int8 < 20000.0, int8
    dmma = sht.measure_peak(ctx, "dmma")
    assert 5.0 < dmma < 200.0, dmma
    # the split kernel's operand pipeline alone: bounded by the dense INT8 rate
    pipe = sht.measure_peak(ctx, "split_pipe")
    assert 100.0 < pipe < 1.2 * int8, (pipe, int8)
    v = __import__("ctypes").c_double()
    assert sht.lib().sht_measure_peak(ctx.handle, 7, __import__("ctypes").byref(v)) == sht.Status.ERR_UNSUPPORTED
