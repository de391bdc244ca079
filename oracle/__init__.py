"""CPU oracle for shtensor's single-rank block-sparse contraction (test infrastructure only).

This package is the checker.  Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU
legs import it; the product package ``shtensor_b200`` never does.  It wraps two shared
libraries built by ``oracle/Makefile``:

* ``liboracle.so`` -- the C++ restatement (oracle.cpp) of the reference's einsum mapping
  (src/Basics/ContractInfo.h:69-346), reshape (src/Basics/Utils.h:315-359), the XMM
  kernel's FP64/FP32 arithmetic order (src/Kernel/KernelImpl.cpp:210-770), the LAPACK path
  (KernelImpl.cpp:142-208), reserve (src/Tensor/BaseTensor.cpp:117-251), norms
  (src/Basics/BlockSpan.h:140-164), filter/compress, and the block-sparse contraction with
  this project's canonical pair order.
* ``_ref/libshtref.so`` -- the reference's own headers compiled in place, used to pin the
  restatement and as the reference-faithful CPU baseline (reshape + OpenBLAS dgemm).
"""
from __future__ import annotations

import ctypes as C
import glob
import os
from dataclasses import dataclass, field

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None
_REF = None

_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")


class OracleError(RuntimeError):
    pass


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            raise OracleError(f"{path} missing: run `make -C oracle`")
        L = C.CDLL(path)
        L.ora_contract_info.restype = C.c_int
        L.ora_scatter.restype = C.c_int
        L.ora_kernel_xmm_f64.restype = C.c_int
        L.ora_kernel_xmm_f32.restype = C.c_int
        L.ora_kernel_lapack_f64.restype = C.c_int
        L.ora_reserve.restype = C.c_int
        L.ora_block_norm.restype = C.c_double
        L.ora_block_norm.argtypes = [_f64p, C.c_int64, C.c_int]
        L.ora_filter.restype = C.c_int64
        L.ora_contract_run.restype = C.c_void_p
        for n in ("ora_result_npairs", "ora_result_nblocks", "ora_result_nnz"):
            getattr(L, n).restype = C.c_int64
            getattr(L, n).argtypes = [C.c_void_p]
        for n in ("ora_result_flops", "ora_result_seconds"):
            getattr(L, n).restype = C.c_double
            getattr(L, n).argtypes = [C.c_void_p]
        L.ora_result_pairs.argtypes = [C.c_void_p, _i64p]
        L.ora_result_index.argtypes = [C.c_void_p, _i64p, _i64p]
        L.ora_result_data.argtypes = [C.c_void_p, _f64p]
        L.ora_result_free.argtypes = [C.c_void_p]
        _LIB = L
    return _LIB


def _blas_library():
    """Locate the OpenBLAS bundled with scipy (LP64, symbols prefixed ``scipy_``)."""
    import scipy

    libs = os.path.join(os.path.dirname(os.path.dirname(scipy.__file__)), "scipy.libs")
    cands = sorted(glob.glob(os.path.join(libs, "libscipy_openblas-*.so")))
    return cands[0] if cands else None


def ref_lib(nthreads_blas: int = 1):
    """The reference-header harness, or None when it was not built (no reference sources)."""
    global _REF
    if _REF is None:
        path = os.path.join(_HERE, "_ref", "libshtref.so")
        if not os.path.exists(path):
            return None
        L = C.CDLL(path)
        L.ref_contract_info.restype = C.c_int
        L.ref_kernel_lapack_f64.restype = C.c_int
        L.ref_contract_run.restype = C.c_void_p
        L.ora_result_free.argtypes = [C.c_void_p]
        for n in ("ora_result_npairs", "ora_result_nblocks", "ora_result_nnz"):
            getattr(L, n).restype = C.c_int64
            getattr(L, n).argtypes = [C.c_void_p]
        for n in ("ora_result_flops", "ora_result_seconds"):
            getattr(L, n).restype = C.c_double
            getattr(L, n).argtypes = [C.c_void_p]
        L.ora_result_pairs.argtypes = [C.c_void_p, _i64p]
        L.ora_result_index.argtypes = [C.c_void_p, _i64p, _i64p]
        L.ora_result_data.argtypes = [C.c_void_p, _f64p]
        blas = _blas_library()
        if blas is None or L.ref_init_blas(blas.encode(), b"scipy_dgemm_",
                                          b"scipy_openblas_set_num_threads", nthreads_blas) != 0:
            return None
        _REF = L
    return _REF


def _ints(v):
    return np.ascontiguousarray(np.asarray(v, dtype=np.int32))


def _err():
    return C.create_string_buffer(512)


@dataclass
class Maps:
    rowA: list
    colA: list
    rowB: list
    colB: list
    rowC: list
    colC: list
    scatter: list = field(default_factory=list)


def contract_info(expr: str, sA, sB, sC) -> Maps:
    L = lib()
    maps = np.zeros(96, dtype=np.int32)
    counts = np.zeros(6, dtype=np.int32)
    e = _err()
    sa, sb, sc = _ints(sA), _ints(sB), _ints(sC)
    rc = L.ora_contract_info(expr.encode(), len(sa), sa.ctypes.data_as(C.c_void_p), len(sb),
                             sb.ctypes.data_as(C.c_void_p), len(sc), sc.ctypes.data_as(C.c_void_p),
                             maps.ctypes.data_as(C.c_void_p), counts.ctypes.data_as(C.c_void_p), e, 512)
    if rc != 0:
        raise OracleError(e.value.decode())
    return Maps(*[list(maps[16 * i:16 * i + counts[i]]) for i in range(6)])


def ref_contract_info(expr: str, sA, sB, sC) -> Maps:
    L = ref_lib()
    if L is None:
        raise OracleError("reference harness not built")
    maps = np.zeros(96, dtype=np.int32)
    counts = np.zeros(12, dtype=np.int32)
    cap = 1 << 20
    scat = np.zeros(cap, dtype=np.int32)
    e = _err()
    sa, sb, sc = _ints(sA), _ints(sB), _ints(sC)
    rc = L.ref_contract_info(expr.encode(), len(sa), sa.ctypes.data_as(C.c_void_p), len(sb),
                             sb.ctypes.data_as(C.c_void_p), len(sc), sc.ctypes.data_as(C.c_void_p),
                             maps.ctypes.data_as(C.c_void_p), counts.ctypes.data_as(C.c_void_p),
                             scat.ctypes.data_as(C.c_void_p), cap, e, 512)
    if rc != 0:
        raise OracleError(e.value.decode())
    out = Maps(*[list(maps[16 * i:16 * i + counts[i]]) for i in range(6)])
    pos = 0
    for i in range(6):
        n = int(counts[6 + i])
        out.scatter.append(list(scat[pos:pos + n]))
        pos += n
    return out


def scatter(map_, sizes):
    L = lib()
    m, s = _ints(map_), _ints(sizes)
    total = int(np.prod([sizes[a] for a in map_])) if len(map_) else 1
    out = np.zeros(total, dtype=np.int32)
    L.ora_scatter(m.ctypes.data_as(C.c_void_p), len(m), s.ctypes.data_as(C.c_void_p), len(s),
                  out.ctypes.data_as(C.c_void_p))
    return out


def reshape(arr: np.ndarray, sizes, order, ref: bool = False) -> np.ndarray:
    L = ref_lib() if ref else lib()
    a = np.ascontiguousarray(arr, dtype=np.float64).ravel()
    out = np.zeros_like(a)
    s, o = _ints(sizes), _ints(order)
    fn = L.ref_reshape_f64 if ref else L.ora_reshape_f64
    fn(a.ctypes.data_as(C.c_void_p), s.ctypes.data_as(C.c_void_p), o.ctypes.data_as(C.c_void_p),
       len(s), out.ctypes.data_as(C.c_void_p))
    return out


def _kernel(fn, expr, sA, sB, sC, alpha, beta, a, b, c, nb_ops, dtype):
    sa, sb, sc = _ints(sA), _ints(sB), _ints(sC)
    e = _err()
    ct = C.c_double if dtype == np.float64 else C.c_float
    rc = fn(expr.encode(), len(sa), sa.ctypes.data_as(C.c_void_p), len(sb), sb.ctypes.data_as(C.c_void_p),
            len(sc), sc.ctypes.data_as(C.c_void_p), ct(alpha), ct(beta), a.ctypes.data_as(C.c_void_p),
            b.ctypes.data_as(C.c_void_p), c.ctypes.data_as(C.c_void_p), C.c_int64(nb_ops), e, 512)
    if rc != 0:
        raise OracleError(e.value.decode())
    return c


def kernel_xmm(expr, sA, sB, sC, alpha, beta, a, b, c, nb_ops):
    """Stack kernel in the XMM arithmetic order; c is updated in place and returned."""
    L = lib()
    if c.dtype == np.float64:
        return _kernel(L.ora_kernel_xmm_f64, expr, sA, sB, sC, alpha, beta, a, b, c, nb_ops, np.float64)
    return _kernel(L.ora_kernel_xmm_f32, expr, sA, sB, sC, alpha, beta, a, b, c, nb_ops, np.float32)


def kernel_lapack(expr, sA, sB, sC, alpha, beta, a, b, c, nb_ops, ref: bool = False):
    """Stack kernel on the LAPACK path (reshape -> gemm -> reshape back)."""
    if ref:
        L = ref_lib()
        if L is None:
            raise OracleError("reference harness not built")
        return _kernel(L.ref_kernel_lapack_f64, expr, sA, sB, sC, alpha, beta, a, b, c, nb_ops, np.float64)
    return _kernel(lib().ora_kernel_lapack_f64, expr, sA, sB, sC, alpha, beta, a, b, c, nb_ops, np.float64)


@dataclass
class HostTensor:
    """Host copy of a block-sparse tensor in the reference's storage layout."""
    block_sizes: list          # per mode: list of block sizes
    ids: np.ndarray            # sorted rolled ids (int64)
    offsets: np.ndarray        # element offsets (int64)
    data: np.ndarray           # float64, blocks in id order, each column-major
    rows: np.ndarray | None = None

    @property
    def order(self):
        return len(self.block_sizes)

    def flat_sizes(self):
        nb = np.array([len(b) for b in self.block_sizes], dtype=np.int32)
        bs = np.concatenate([np.asarray(b, dtype=np.int32) for b in self.block_sizes])
        return nb, bs


def reserve(block_sizes, idx) -> HostTensor:
    """BaseTensor::reserve on the host; idx is a list of per-mode index lists (VArray<N>)."""
    L = lib()
    order = len(block_sizes)
    nb = np.array([len(b) for b in block_sizes], dtype=np.int32)
    bs = np.concatenate([np.asarray(b, dtype=np.int32) for b in block_sizes])
    n = len(idx[0]) if order else 0
    flat = np.ascontiguousarray(np.concatenate([np.asarray(v, dtype=np.int32) for v in idx])) if n else np.zeros(0, np.int32)
    ids = np.zeros(n, dtype=np.int64)
    offs = np.zeros(n, dtype=np.int64)
    rows = np.zeros(int(nb[0]), dtype=np.int64)
    nnz = C.c_int64(0)
    e = _err()
    rc = L.ora_reserve(order, nb.ctypes.data_as(C.c_void_p), bs.ctypes.data_as(C.c_void_p), C.c_int64(n),
                       flat.ctypes.data_as(C.c_void_p), ids.ctypes.data_as(C.c_void_p),
                       offs.ctypes.data_as(C.c_void_p), rows.ctypes.data_as(C.c_void_p), C.byref(nnz), e, 512)
    if rc != 0:
        raise OracleError(e.value.decode())
    return HostTensor([list(b) for b in block_sizes], ids, offs, np.zeros(nnz.value), rows)


def block_norm(data, norm: int) -> float:
    d = np.ascontiguousarray(data, dtype=np.float64)
    return float(lib().ora_block_norm(d, C.c_int64(d.size), norm))


def filter_blocks(t: HostTensor, eps: float, norm: int, compress: bool = True) -> HostTensor:
    L = lib()
    nb, bs = t.flat_sizes()
    ids = t.ids.copy()
    offs = t.offsets.copy()
    data = t.data.copy()
    rows = np.zeros(len(t.block_sizes[0]), dtype=np.int64)
    nnz = C.c_int64(0)
    n = L.ora_filter(t.order, nb.ctypes.data_as(C.c_void_p), bs.ctypes.data_as(C.c_void_p),
                     C.c_int64(len(ids)), ids.ctypes.data_as(C.c_void_p), offs.ctypes.data_as(C.c_void_p),
                     data.ctypes.data_as(C.c_void_p), C.c_double(eps), C.c_int(norm), C.c_int(int(compress)),
                     rows.ctypes.data_as(C.c_void_p), C.byref(nnz))
    return HostTensor(t.block_sizes, ids[:n].copy(), offs[:n].copy(), data[:nnz.value].copy(),
                      rows if compress else t.rows)


@dataclass
class ContractOut:
    C: HostTensor
    pairs: np.ndarray   # (npairs, 3) int64: idC, idA, idB
    flops: float
    seconds: float


def _targs(t: HostTensor):
    nb, bs = t.flat_sizes()
    ids = np.ascontiguousarray(t.ids, dtype=np.int64)
    offs = np.ascontiguousarray(t.offsets, dtype=np.int64)
    data = np.ascontiguousarray(t.data, dtype=np.float64)
    keep = (nb, bs, ids, offs, data)
    return keep, [C.c_int(t.order), nb.ctypes.data_as(C.c_void_p), bs.ctypes.data_as(C.c_void_p),
                  C.c_int64(len(ids)), ids.ctypes.data_as(C.c_void_p), offs.ctypes.data_as(C.c_void_p),
                  data.ctypes.data_as(C.c_void_p)]


def contract(expr, alpha, A: HostTensor, B: HostTensor, beta, Cin: HostTensor, eps=0.0, norm=0,
             lapack_blocks=False, nthreads=0, ref=False) -> ContractOut:
    """Block-sparse C = beta*C + alpha*A·B.  ref=True uses the reference-header harness
    (Utils::reshape + OpenBLAS dgemm per pair); otherwise the XMM-order restatement."""
    L = lib()
    kA, aA = _targs(A)
    kB, aB = _targs(B)
    kC, aC = _targs(Cin)
    e = _err()
    if ref:
        R = ref_lib()
        if R is None:
            raise OracleError("reference harness not built")
        h = R.ref_contract_run(expr.encode(), C.c_double(alpha), *aA, *aB, C.c_double(beta), *aC,
                               C.c_double(eps), C.c_int(norm), C.c_int(nthreads), e, 512)
        RL = R
    else:
        h = L.ora_contract_run(expr.encode(), C.c_double(alpha), *aA, *aB, C.c_double(beta), *aC,
                               C.c_double(eps), C.c_int(norm), C.c_int(int(lapack_blocks)), C.c_int(nthreads),
                               e, 512)
        RL = L
    if not h:
        raise OracleError(e.value.decode())
    try:
        npairs = RL.ora_result_npairs(h)
        nblk = RL.ora_result_nblocks(h)
        nnz = RL.ora_result_nnz(h)
        pairs = np.zeros(max(npairs, 1) * 3, dtype=np.int64)
        RL.ora_result_pairs(h, pairs)
        ids = np.zeros(max(nblk, 1), dtype=np.int64)
        offs = np.zeros(max(nblk, 1), dtype=np.int64)
        RL.ora_result_index(h, ids, offs)
        data = np.zeros(max(nnz, 1), dtype=np.float64)
        RL.ora_result_data(h, data)
        out = ContractOut(HostTensor(Cin.block_sizes, ids[:nblk].copy(), offs[:nblk].copy(), data[:nnz].copy()),
                          pairs[:3 * npairs].reshape(npairs, 3).copy(), RL.ora_result_flops(h),
                          RL.ora_result_seconds(h))
    finally:
        RL.ora_result_free(h)
    del kA, kB, kC
    return out


def densify(t: HostTensor) -> np.ndarray:
    """Dense column-major (Fortran-order) array of a block-sparse host tensor."""
    order = t.order
    nblk = [len(b) for b in t.block_sizes]
    starts = [np.concatenate([[0], np.cumsum(b)]).astype(np.int64) for b in t.block_sizes]
    full = np.zeros([int(s[-1]) for s in starts], dtype=np.float64, order="F")
    gstride = np.concatenate([[1], np.cumprod(nblk)[:-1]]).astype(np.int64)
    for bid, off in zip(t.ids, t.offsets):
        coords = [(int(bid) // int(gstride[d])) % nblk[d] for d in range(order)]
        dims = [t.block_sizes[d][coords[d]] for d in range(order)]
        blk = t.data[int(off):int(off) + int(np.prod(dims))].reshape(dims, order="F")
        sl = tuple(slice(int(starts[d][coords[d]]), int(starts[d][coords[d]]) + dims[d]) for d in range(order))
        full[sl] = blk
    return full
