"""Oracle pins (CPU).  The restatement in oracle/ is checked against the reference's own code
(golden fixtures made from src/Basics/ContractInfo.h and Utils.h compiled in place, plus the
LAPACK path with OpenBLAS dgemm) and against numpy.einsum(order='F'), the cross-check the
reference's test/test_kernel.cpp:44-116 carries."""
import json
import os

import numpy as np
import pytest

import oracle
from tests.golden import make_golden as G

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden")


@pytest.fixture(scope="module")
def maps():
    with open(os.path.join(GOLD, "maps.json")) as f:
        return json.load(f)


@pytest.fixture(scope="module")
def kc():
    return np.load(os.path.join(GOLD, "kernel_cases.npz"))


def test_maps_match_reference(maps):
    for case in maps["cases"]:
        m = oracle.contract_info(case["expr"], case["sa"], case["sb"], case["sc"])
        got = [list(map(int, v)) for v in (m.rowA, m.colA, m.rowB, m.colB, m.rowC, m.colC)]
        assert got == case["maps"], case["expr"]


def test_scatter_vectors_match_reference(maps):
    for case in maps["cases"]:
        mp = case["maps"]
        sizes = [case["sa"], case["sa"], case["sb"], case["sb"], case["sc"], case["sc"]]
        for i in range(6):
            got = oracle.scatter(mp[i], sizes[i])
            assert list(map(int, got)) == case["scatter"][i], (case["expr"], i)


def test_error_messages_match_reference(maps):
    for case in maps["errors"]:
        if case["message"] is None:
            continue
        with pytest.raises(oracle.OracleError) as ei:
            oracle.contract_info(case["expr"], [2, 2], [2, 2], [2, 2])
        assert str(ei.value) == case["message"]


def test_rejects_inputs_the_reference_mismaps():
    with pytest.raises(oracle.OracleError, match="free indices"):
        oracle.contract_info("ij,jk->iz", [2, 2], [2, 2], [2, 2])
    with pytest.raises(oracle.OracleError, match="order"):
        oracle.contract_info("ij,jk->ik", [2, 2, 2], [2, 2], [2, 2])
    with pytest.raises(oracle.OracleError, match="do not match"):
        oracle.contract_info("ij,jk->ik", [2, 3], [4, 2], [2, 2])


@pytest.mark.parametrize("n", range(len(G.KERNEL_CASES)))
def test_kernel_xmm_order_is_frozen(kc, n):
    expr, sa, sb, sc, al, be, nops = G.KERNEL_CASES[n]
    c = kc[f"{n}_c"].copy()
    got = oracle.kernel_xmm(expr, sa, sb, sc, al, be, kc[f"{n}_a"], kc[f"{n}_b"], c, nops)
    assert np.array_equal(got, kc[f"{n}_xmm"])
    c32 = kc[f"{n}_c"].astype(np.float32)
    got32 = oracle.kernel_xmm(expr, sa, sb, sc, al, be, kc[f"{n}_a"].astype(np.float32),
                              kc[f"{n}_b"].astype(np.float32), c32, nops)
    assert np.array_equal(got32, kc[f"{n}_xmm32"])


@pytest.mark.parametrize("n", range(len(G.KERNEL_CASES)))
def test_kernel_paths_agree_with_reference_lapack_and_einsum(kc, n):
    expr, sa, sb, sc, al, be, nops = G.KERNEL_CASES[n]
    a, b, c0 = kc[f"{n}_a"], kc[f"{n}_b"], kc[f"{n}_c"]
    xmm = kc[f"{n}_xmm"]
    ref = kc[f"{n}_lapack_ref"]
    lap = oracle.kernel_lapack(expr, sa, sb, sc, al, be, a, b, c0.copy(), nops)
    za, zb, zc = (int(np.prod(s)) for s in (sa, sb, sc))
    for op in range(nops):
        A = a[op * za:(op + 1) * za].reshape(sa, order="F")
        B = b[op * zb:(op + 1) * zb].reshape(sb, order="F")
        C0 = c0[op * zc:(op + 1) * zc].reshape(sc, order="F")
        want = al * np.einsum(expr.replace(" ", ""), A, B) + be * C0
        for got in (xmm, ref, lap):
            g = got[op * zc:(op + 1) * zc].reshape(sc, order="F")
            assert np.abs(g - want).max() <= 1e-13 * max(1.0, np.abs(want).max())


def test_beta_scaling_identity(kc):
    # test_kernel (test/test_kernel.cpp:241-285): alpha=0, beta=2 gives sum(C') = 2 sum(C)
    for n, case in enumerate(G.KERNEL_CASES):
        if case[4] != 0.0:
            continue
        assert np.isclose(kc[f"{n}_xmm"].sum(), 2.0 * kc[f"{n}_c"].sum(), atol=1e-12)


def test_reshape_matches_reference_when_built():
    if oracle.ref_lib() is None:
        pytest.skip("reference harness not built here")
    x = np.random.default_rng(3).uniform(size=3 * 4 * 5 * 6)
    for order in ([2, 0, 3, 1], [0, 1, 2, 3], [3, 2, 1, 0], [1, 3, 0, 2]):
        assert np.array_equal(oracle.reshape(x, [3, 4, 5, 6], order), oracle.reshape(x, [3, 4, 5, 6], order, ref=True))
