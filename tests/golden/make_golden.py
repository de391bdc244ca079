"""Generate the frozen golden fixtures of this directory.

Run from the repository root where the reference sources and oracle/_ref are present:

    make -C oracle && python tests/golden/make_golden.py

Fixtures (all inputs seeded with numpy's PCG64):
* ``maps.json``      -- axis maps and scatter vectors from the reference's own
                        compute_contract_info (src/Basics/ContractInfo.h, compiled in place by
                        oracle/Makefile into oracle/_ref), for the reference's test expressions
                        (test/test_kernel.cpp:306-356) and the block-sparse workloads.
* ``kernel_cases.npz`` -- per-block stack cases of test/test_kernel.cpp (expressions, sizes,
                        nb_ops=20): inputs, the reference LAPACK path (Utils::reshape + OpenBLAS
                        dgemm, KernelImpl.cpp:142-208) and the XMM-order restatement.
* ``blocksparse.npz`` -- small block-sparse contractions (c0-like, c1-like, c3-like): inputs,
                        the canonical pair list, the result pattern and values (XMM order), and
                        the reference-path values (reshape + dgemm per pair).
The GPU tests read only these files; nothing under the reference tree is read at test time.
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from shtensor_b200 import workloads as W  # noqa: E402

KERNEL_CASES = [
    # test_contract cases (test/test_kernel.cpp:306-316), alpha=1, beta=0, 20 ops
    ("ik, kj -> ij", [8, 5], [5, 6], [8, 6], 1.0, 0.0, 20),
    ("jik, kmj -> im", [6, 5, 8], [8, 4, 6], [5, 4], 1.0, 0.0, 20),
    ("ikl, lkmj -> mij", [6, 5, 7], [7, 5, 6, 6], [6, 6, 6], 1.0, 0.0, 20),
    # test_kernel cases (:318-345), alpha=0, beta=2, one op
    ("ijml, lmk -> jki", [5, 6, 8, 9], [9, 8, 7], [6, 7, 5], 0.0, 2.0, 1),
    ("ij, jk -> ik", [2, 2], [2, 2], [2, 2], 0.0, 2.0, 1),
    ("ij, jk -> ik", [5, 5], [5, 5], [5, 5], 0.0, 2.0, 1),
    ("ij, jk -> ik", [8, 8], [8, 8], [8, 8], 0.0, 2.0, 1),
    ("ij, jk -> ik", [10, 10], [10, 10], [10, 10], 0.0, 2.0, 1),
    ("ij, jk -> ik", [3, 3], [3, 3], [3, 3], 0.0, 2.0, 1),
    ("ij, jk -> ik", [4, 4], [4, 4], [4, 4], 0.0, 2.0, 1),
    ("ij, jk -> ki", [4, 4], [4, 4], [4, 4], 0.0, 2.0, 1),
    # test_timings shapes (:347-356) with both scalars non-trivial
    ("ikl, ljk -> ij", [8, 8, 8], [8, 8, 8], [8, 8], 1.5, 0.5, 4),
    ("kil, ljk -> ij", [8, 8, 8], [8, 8, 8], [8, 8], 1.5, 0.5, 4),
    ("ikl, ljk -> ji", [5, 5, 5], [5, 5, 5], [5, 5], 1.5, 0.5, 4),
    ("ik, kj -> ij", [16, 16], [16, 16], [16, 16], 1.5, 0.5, 4),
    # block-sparse workload shapes
    ("ijl, lk -> ijk", [7, 9, 11], [11, 13], [7, 9, 13], 1.0, 1.0, 3),
    ("iaP, jbP -> ijab", [5, 7, 8], [9, 6, 8], [5, 9, 7, 6], 1.0, 0.0, 2),
    ("abcd, cdij -> abij", [3, 4, 5, 6], [5, 6, 7, 8], [3, 4, 7, 8], -0.75, 0.25, 2),
    ("ijl, lkm -> ijmk", [3, 4, 5], [5, 6, 7], [3, 4, 7, 6], 1.0, 0.0, 2),
]

ERROR_CASES = ["", "ij,jk", "ij,jk->ik,", "ii,ik->k", "ij,ij->", "ij,kl->ijkl", "i$,jk->ik", "ij,jk->ik->ij"]


def mini_c1(seed):
    """c1's expression and structure with small blocks (fixture size)."""
    rng = np.random.default_rng(seed)
    i, j = [3, 5, 2], [4, 2, 3]
    a, b = [3, 5, 4, 2], [2, 6, 3]
    P = [4, 6, 5, 3]
    A = W.build_tensor(rng, [i, a, P], lambda c: rng.random(len(c[0])) < 0.35,
                       lambda c: np.exp(-np.abs(c[1] - c[2]) / 4.0), "normal")
    B = W.build_tensor(rng, [j, b, P], lambda c: rng.random(len(c[0])) < 0.35,
                       lambda c: 10.0 ** rng.uniform(-6, 2, len(c[0])), "normal")
    return W.Workload("c1", "iaP, jbP -> ijab", A, B, W.empty_tensor([i, j, a, b]))


def mini_c3(seed):
    """c3's expression with decay storage and product screening on small blocks."""
    rng = np.random.default_rng(seed)
    big = [[3, 4, 2, 3], [2, 3, 4], [3, 2, 4], [4, 2, 3]]
    small = [[2, 3], [3, 2]]

    def spread(cc):
        st = np.stack(cc[:4])
        return st.max(0) - st.min(0)

    V = W.build_tensor(rng, big, lambda cc: np.exp(-0.5 * spread(cc)) >= 0.2,
                       lambda cc: np.exp(-2.0 * spread(cc)), "normal")
    T = W.build_tensor(rng, [big[2], big[3]] + small,
                       lambda cc: np.exp(-0.5 * (np.abs(cc[0] - cc[1]) + np.abs(cc[2] - cc[3]))) >= 0.1,
                       lambda cc: np.exp(-2.0 * (np.abs(cc[0] - cc[1]) + np.abs(cc[2] - cc[3]))), "normal")
    return W.Workload("c3", "abcd, cdij -> abij", V, T, W.empty_tensor([big[0], big[1]] + small), screen_eps=0.05)


def host(t):
    return oracle.HostTensor(t.block_sizes, t.ids, t.offsets, t.data)


def main():
    if oracle.ref_lib() is None:
        raise SystemExit("oracle/_ref not built (needs the reference sources)")
    rng = np.random.default_rng(20261203)
    maps = {"cases": [], "errors": []}
    kc = {}
    for n, (expr, sa, sb, sc, al, be, nops) in enumerate(KERNEL_CASES):
        r = oracle.ref_contract_info(expr, sa, sb, sc)
        maps["cases"].append({"expr": expr, "sa": sa, "sb": sb, "sc": sc,
                              "maps": [list(map(int, v)) for v in (r.rowA, r.colA, r.rowB, r.colB, r.rowC, r.colC)],
                              "scatter": [list(map(int, v)) for v in r.scatter]})
        a = rng.uniform(-1, 1, nops * int(np.prod(sa)))
        b = rng.uniform(-1, 1, nops * int(np.prod(sb)))
        c = rng.uniform(-1, 1, nops * int(np.prod(sc)))
        kc[f"{n}_a"], kc[f"{n}_b"], kc[f"{n}_c"] = a, b, c
        kc[f"{n}_lapack_ref"] = oracle.kernel_lapack(expr, sa, sb, sc, al, be, a, b, c.copy(), nops, ref=True)
        kc[f"{n}_xmm"] = oracle.kernel_xmm(expr, sa, sb, sc, al, be, a, b, c.copy(), nops)
        a32, b32, c32 = a.astype(np.float32), b.astype(np.float32), c.astype(np.float32)
        kc[f"{n}_xmm32"] = oracle.kernel_xmm(expr, sa, sb, sc, al, be, a32, b32, c32.copy(), nops)
    for e in ERROR_CASES:
        try:
            oracle.ref_contract_info(e, [2, 2], [2, 2], [2, 2])
            msg = None
        except oracle.OracleError as ex:
            msg = str(ex)
        maps["errors"].append({"expr": e, "message": msg})
    with open(os.path.join(HERE, "maps.json"), "w") as f:
        json.dump(maps, f, indent=1)
    np.savez_compressed(os.path.join(HERE, "kernel_cases.npz"), **kc)

    bs = {}
    cases = {"c0": W.c0(seed=7, nblocks=4, p=0.4), "c1": mini_c1(7), "c3": mini_c3(7)}
    for name, w in cases.items():
        A, B, Cw = host(w.A), host(w.B), host(w.C)
        r = oracle.contract(w.expr, 1.0, A, B, 0.0, Cw, eps=w.screen_eps, norm=0)
        rr = oracle.contract(w.expr, 1.0, A, B, 0.0, Cw, eps=w.screen_eps, norm=0, ref=True)
        assert np.array_equal(r.pairs, rr.pairs)
        for tn, t in (("A", w.A), ("B", w.B)):
            bs[f"{name}_{tn}_bs"] = np.concatenate([np.asarray(x, np.int32) for x in t.block_sizes])
            bs[f"{name}_{tn}_nb"] = np.array([len(x) for x in t.block_sizes], np.int32)
            bs[f"{name}_{tn}_ids"] = t.ids
            bs[f"{name}_{tn}_data"] = t.data
        bs[f"{name}_C_bs"] = np.concatenate([np.asarray(x, np.int32) for x in w.C.block_sizes])
        bs[f"{name}_C_nb"] = np.array([len(x) for x in w.C.block_sizes], np.int32)
        bs[f"{name}_pairs"] = r.pairs
        bs[f"{name}_cids"] = r.C.ids
        bs[f"{name}_coffs"] = r.C.offsets
        bs[f"{name}_cdata"] = r.C.data
        bs[f"{name}_cdata_ref"] = rr.C.data
        bs[f"{name}_eps"] = np.array([w.screen_eps])
        bs[f"{name}_expr"] = np.array([w.expr])
    np.savez_compressed(os.path.join(HERE, "blocksparse.npz"), **bs)
    print("fixtures written:", sorted(os.listdir(HERE)))


if __name__ == "__main__":
    main()
