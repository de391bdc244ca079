"""shtensor_b200 -- B200 (sm_100a) block-sparse tensor contraction, Python host binding.

A thin ctypes layer over the C ABI of ``libshtensor_b200.so`` (declared in
include/shtensor_b200.h).  Names and argument meanings mirror shtensor's C++ API:

* ``Context(pool_bytes)``                     -- Context(MPI_Comm, int64_t)      src/Shmem/Context.h:30
* ``Kernel(ctx, expr, sa, sb, sc, alpha, beta, KernelType)`` and ``.call(a, b, c, nb_ops)``
                                               -- Kernel<T>                       src/Kernel/Kernel.h:62-93
* ``Tensor(ctx, block_sizes)`` with ``reserve``/``reserve_all``/``filter``/``compress``
                                               -- Tensor<T,N>                     src/Tensor/Tensor.h:19-366
* ``contract(...)`` / ``Plan``                 -- the block-sparse contract the reference lacks

Errors raise ``ShtError`` with the library's message, like the reference's
``std::runtime_error``.  There is no CPU fallback: importing works without a GPU, but every
call that needs the device fails loudly when the library or the GPU is missing.
"""
from __future__ import annotations

import ctypes as C
import enum
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libshtensor_b200.so")
_lib = None


class ShtError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"[{Status(status).name if status in Status._value2member_map_ else status}] {msg}")
        self.status = status


class Status(enum.IntEnum):
    OK = 0
    ERR_INVALID = 1
    ERR_PARSE = 2
    ERR_SIZE = 3
    ERR_OOM = 4
    ERR_CUDA = 5
    ERR_TIMEOUT = 6
    ERR_UNSUPPORTED = 7
    ERR_STATE = 8


class KernelType(enum.IntEnum):
    LAPACK = 0
    XMM = 1


class BlockNorm(enum.IntEnum):
    FROBENIUS = 0
    MAXABS = 1
    FROBENIUS_REFCOMPAT = 2


class Mode(enum.IntEnum):
    PLAIN_FP64 = 0
    BATCHED_FP64 = 1
    SPLIT = 2


class Report(C.Structure):
    _fields_ = [("npairs", C.c_int64), ("nblocks_c", C.c_int64), ("nnz_c", C.c_int64), ("nwork", C.c_int64),
                ("flops", C.c_double), ("plan_ms", C.c_double), ("exec_ms", C.c_double),
                ("slices", C.c_int32), ("reserved", C.c_int32)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "reserved"}


class ServerConfig(C.Structure):
    _fields_ = [("max_active", C.c_int), ("max_batch", C.c_int), ("reserve_bytes", C.c_size_t),
                ("planners", C.c_int), ("ctas_per_sm", C.c_int), ("mode", C.c_int)]


class RequestReport(C.Structure):
    _fields_ = [("status", C.c_int), ("npairs", C.c_int64), ("flops", C.c_double), ("queue_ms", C.c_double),
                ("plan_ms", C.c_double), ("run_ms", C.c_double), ("gpu_ms", C.c_double), ("latency_ms", C.c_double),
                ("batch", C.c_int64), ("form", C.c_int), ("batch_size", C.c_int), ("deferrals", C.c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class ServerStats(C.Structure):
    _fields_ = [("submitted", C.c_int64), ("completed", C.c_int64), ("failed", C.c_int64), ("batches", C.c_int64),
                ("deferrals", C.c_int64), ("max_active_seen", C.c_int), ("mean_batch", C.c_double),
                ("p50_ms", C.c_double), ("p99_ms", C.c_double), ("max_ms", C.c_double), ("flops", C.c_double),
                ("span_s", C.c_double), ("gflops", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_P = C.c_void_p
_SIGS = {
    "sht_init": [C.POINTER(_P), C.c_int, C.c_size_t],
    "sht_finalize": [_P],
    "sht_pool_info": [_P, C.POINTER(C.c_size_t), C.POINTER(C.c_size_t), C.POINTER(C.c_size_t), C.POINTER(C.c_size_t)],
    "sht_pool_alloc": [_P, C.c_size_t, C.POINTER(_P)],
    "sht_pool_realloc": [_P, C.POINTER(_P), C.c_size_t, _P],
    "sht_pool_free": [_P, _P, _P],
    "sht_pool_configure": [_P, C.c_size_t, C.c_size_t],
    "sht_kernel_create": [_P, C.c_char_p, _P, C.c_int, _P, C.c_int, _P, C.c_int, C.c_double, C.c_double, C.c_int,
                          C.c_int, C.POINTER(_P)],
    "sht_kernel_call": [_P, _P, _P, _P, C.c_int64, _P],
    "sht_kernel_call_static": [_P, _P, _P, _P, C.c_int64, _P],
    "sht_kernel_info": [_P, C.c_char_p, C.c_size_t],
    "sht_kernel_destroy": [_P],
    "sht_tensor_create": [_P, C.c_int, _P, _P, C.c_int, C.POINTER(_P)],
    "sht_tensor_reserve": [_P, C.c_int64, _P],
    "sht_tensor_reserve_all": [_P],
    "sht_tensor_reserve_device": [_P, C.c_int64, _P, _P],
    "sht_tensor_info": [_P, C.POINTER(C.c_int64), C.POINTER(C.c_int64)],
    "sht_tensor_get_index": [_P, _P, _P, _P],
    "sht_tensor_upload": [_P, _P, C.c_int64, _P],
    "sht_tensor_download": [_P, _P, C.c_int64, _P],
    "sht_tensor_device_data": [_P, C.POINTER(_P)],
    "sht_tensor_norms": [_P, C.c_int, _P, _P],
    "sht_tensor_filter": [_P, C.c_double, C.c_int, C.c_int, _P],
    "sht_tensor_compress": [_P, _P],
    "sht_tensor_destroy": [_P],
    "sht_contract": [_P, C.c_char_p, C.c_double, _P, _P, C.c_double, _P, C.c_double, C.c_int, C.c_int, _P,
                     C.POINTER(Report)],
    "sht_plan_create": [_P, C.c_char_p, _P, _P, _P, C.c_double, C.c_int, C.c_int, _P, C.POINTER(_P)],
    "sht_plan_execute": [_P, C.c_double, C.c_double, _P],
    "sht_plan_execute_graph": [_P, C.c_double, C.c_double, _P],
    "sht_plan_report": [_P, C.POINTER(Report)],
    "sht_plan_pairs": [_P, _P, C.c_int64],
    "sht_plan_destroy": [_P],
    "sht_tensor_compare": [_P, _P, C.POINTER(C.c_double), C.POINTER(C.c_double), _P],
    "sht_tensor_bitdiff": [_P, _P, C.POINTER(C.c_int64), _P],
    "sht_autotune": [_P, C.c_char_p, _P],
    "sht_measure_peak": [_P, C.c_int, C.POINTER(C.c_double)],
    "sht_set_split_slices": [_P, C.c_int],
    "sht_stream_sync": [_P, _P],
    "sht_set_wait_limit": [_P, C.c_int64],
    "sht_server_create": [_P, C.POINTER(ServerConfig), C.POINTER(_P)],
    "sht_server_submit": [_P, C.c_char_p, C.c_double, _P, _P, C.c_double, _P, C.c_double, C.c_int,
                          C.POINTER(C.c_int64)],
    "sht_server_poll": [_P, C.c_int64, C.POINTER(C.c_int)],
    "sht_server_wait": [_P, C.c_int64, C.c_double, C.POINTER(RequestReport)],
    "sht_server_get_stats": [_P, C.POINTER(ServerStats)],
    "sht_server_reset_stats": [_P],
    "sht_server_destroy": [_P],
}


def lib():
    """Load the CUDA library; raises if it was not built (there is no fallback path)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m shtensor_b200.build`")
        L = C.CDLL(LIB_PATH)
        for name, args in _SIGS.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = C.c_int
        L.sht_last_error.restype = C.c_char_p
        L.sht_last_error.argtypes = []
        _lib = L
    return _lib


def exported_symbols():
    return list(_SIGS) + ["sht_last_error"]


def _check(rc: int):
    if rc != 0:
        raise ShtError(rc, lib().sht_last_error().decode(errors="replace"))


def _stream(stream):
    if stream is None:
        return None
    if isinstance(stream, int):
        return stream
    return getattr(stream, "cuda_stream", stream)


def _iarr(v):
    a = np.ascontiguousarray(np.asarray(v, dtype=np.int32))
    return a, a.ctypes.data_as(_P)


def _ptr(x):
    """Device pointer of a torch tensor, or host pointer of a numpy array."""
    if hasattr(x, "data_ptr"):
        return x.data_ptr()
    if isinstance(x, np.ndarray):
        if not x.flags.c_contiguous:
            raise ValueError("arrays must be contiguous")
        return x.ctypes.data
    if isinstance(x, int):
        return x
    raise TypeError(f"unsupported buffer {type(x)}")


class Context:
    """Device context with its memory pool (replaces Context + MemoryPool)."""

    def __init__(self, pool_bytes: int, device: int = 0):
        h = _P()
        _check(lib().sht_init(C.byref(h), device, C.c_size_t(pool_bytes)))
        self._h = h
        self.device = device

    @property
    def handle(self):
        return self._h

    def pool_info(self):
        vals = [C.c_size_t() for _ in range(4)]
        _check(lib().sht_pool_info(self._h, *[C.byref(v) for v in vals]))
        return dict(zip(("capacity", "free", "chunk_header", "alignment"), (v.value for v in vals)))

    def get_free_mem(self) -> int:
        return self.pool_info()["free"]

    def set_split_slices(self, slices: int):
        """INT8 slices per operand of split-precision plans made afterwards (1..8)."""
        _check(lib().sht_set_split_slices(self._h, slices))

    def stream_sync(self, stream=None):
        """Wait for the work queued on `stream` and raise the first failure this context's
        device work recorded (a split launch whose bounded wait ran out)."""
        _check(lib().sht_stream_sync(self._h, _stream(stream)))

    def set_wait_limit(self, polls: int):
        """Diagnostic: polls of one split-kernel pipeline wait before the launch gives up (0 =
        default)."""
        _check(lib().sht_set_wait_limit(self._h, int(polls)))

    def configure_pool(self, chunk_header: int, alignment: int):
        _check(lib().sht_pool_configure(self._h, chunk_header, alignment))

    def allocate(self, nbytes: int) -> int:
        p = _P()
        _check(lib().sht_pool_alloc(self._h, C.c_size_t(nbytes), C.byref(p)))
        return p.value

    def reallocate(self, ptr: int, nbytes: int, stream=None) -> int:
        p = _P(ptr)
        _check(lib().sht_pool_realloc(self._h, C.byref(p), C.c_size_t(nbytes), _stream(stream)))
        return p.value

    def free(self, ptr: int, stream=None):
        _check(lib().sht_pool_free(self._h, _P(ptr), _stream(stream)))

    def close(self):
        if getattr(self, "_h", None):
            _check(lib().sht_finalize(self._h))
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


class Kernel:
    """Kernel<T>: per-block stack contraction C = alpha*A·B + beta*C over nb_ops triples."""

    def __init__(self, ctx: Context, expr: str, sizes_in1, sizes_in2, sizes_out, alpha=1.0, beta=0.0,
                 kernel_type: KernelType = KernelType.XMM, dtype=np.float64):
        self.ctx = ctx
        self.dtype = np.dtype(dtype)
        if self.dtype not in (np.float32, np.float64):
            raise ValueError("dtype must be float32 or float64")
        a, pa = _iarr(sizes_in1)
        b, pb = _iarr(sizes_in2)
        c, pc = _iarr(sizes_out)
        h = _P()
        _check(lib().sht_kernel_create(ctx.handle, expr.encode(), pa, len(a), pb, len(b), pc, len(c), alpha, beta,
                                       1 if self.dtype == np.float64 else 0, int(kernel_type), C.byref(h)))
        self._h = h
        self.sizes = (list(a), list(b), list(c))

    def call(self, a, b, c, nb_ops: int, stream=None):
        """a, b, c: torch CUDA tensors (run on `stream`) or numpy arrays (staged, synchronous)."""
        _check(lib().sht_kernel_call(self._h, _P(_ptr(a)), _P(_ptr(b)), _P(_ptr(c)), C.c_int64(nb_ops),
                                     _stream(stream)))
        return c

    def call_static(self, a, b, c, nb_ops: int, stream=None):
        """Allocation-free call for callers that cannot allocate device memory: a, b, c are
        device buffers (torch CUDA tensors or raw pointers); scratch is a static device array
        of 32 MiB shared by all such calls, so calls that overlap on the GPU race."""
        _check(lib().sht_kernel_call_static(self._h, _P(_ptr(a)), _P(_ptr(b)), _P(_ptr(c)), C.c_int64(nb_ops),
                                            _stream(stream)))
        return c

    def get_info(self) -> str:
        buf = C.create_string_buffer(8192)
        _check(lib().sht_kernel_info(self._h, buf, 8192))
        return buf.value.decode()

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.sht_kernel_destroy(self._h)
            self._h = None


class Tensor:
    """Tensor<T,N>: block-sparse tensor resident in device memory."""

    def __init__(self, ctx: Context, block_sizes, dtype=np.float64):
        self.ctx = ctx  # keeps the context (and its device arena) alive while the tensor lives
        self.block_sizes = [list(map(int, b)) for b in block_sizes]
        self.dtype = np.dtype(dtype)
        nb, pnb = _iarr([len(b) for b in self.block_sizes])
        bs, pbs = _iarr([x for b in self.block_sizes for x in b])
        h = _P()
        _check(lib().sht_tensor_create(ctx.handle, len(self.block_sizes), pnb, pbs,
                                       1 if self.dtype == np.float64 else 0, C.byref(h)))
        self._h = h

    @property
    def handle(self):
        return self._h

    @property
    def order(self):
        return len(self.block_sizes)

    def reserve(self, idx):
        """idx: per-mode lists of block indices (VArray<N>)."""
        n = len(idx[0]) if len(idx) else 0
        flat = np.ascontiguousarray(np.concatenate([np.asarray(v, dtype=np.int32) for v in idx])) if n else \
            np.zeros(1, np.int32)
        _check(lib().sht_tensor_reserve(self._h, C.c_int64(n), flat.ctypes.data_as(_P)))
        return self

    def reserve_device(self, idx, nblocks=None, stream=None):
        """Reserve from index lists in device memory: idx is a CUDA int32 tensor of shape
        (order, nblocks) (mode-major, like reserve's lists), or a raw device pointer with
        nblocks given."""
        if hasattr(idx, "data_ptr"):
            if idx.dtype != __import__("torch").int32 or not idx.is_cuda or idx.dim() != 2 \
                    or idx.shape[0] != self.order:
                raise ValueError("reserve_device: a CUDA int32 tensor of shape (order, nblocks)")
            idx = idx.contiguous()
            nblocks = idx.shape[1]
            ptr = idx.data_ptr()
        else:
            ptr = int(idx)
        _check(lib().sht_tensor_reserve_device(self._h, C.c_int64(int(nblocks)), C.c_void_p(ptr or None),
                                               _stream(stream)))
        return self

    def reserve_all(self):
        _check(lib().sht_tensor_reserve_all(self._h))
        return self

    def info(self):
        nb, nnz = C.c_int64(), C.c_int64()
        _check(lib().sht_tensor_info(self._h, C.byref(nb), C.byref(nnz)))
        return nb.value, nnz.value

    def get_nb_nzblocks_local(self) -> int:
        return self.info()[0]

    @property
    def nnz(self) -> int:
        return self.info()[1]

    def get_sparse_info(self):
        """(ids, offsets, rows) like BaseTensor::SparseInfo."""
        n, _ = self.info()
        ids = np.zeros(max(n, 1), np.int64)
        offs = np.zeros(max(n, 1), np.int64)
        rows = np.zeros(len(self.block_sizes[0]), np.int64)
        _check(lib().sht_tensor_get_index(self._h, ids.ctypes.data_as(_P), offs.ctypes.data_as(_P),
                                          rows.ctypes.data_as(_P)))
        return ids[:n], offs[:n], rows

    def upload(self, data, stream=None):
        data = np.ascontiguousarray(data, dtype=self.dtype)
        _check(lib().sht_tensor_upload(self._h, data.ctypes.data_as(_P), C.c_int64(data.size), _stream(stream)))
        return self

    def download(self, out=None, stream=None):
        nnz = self.nnz
        if out is None:
            out = np.empty(nnz, dtype=self.dtype)
        _check(lib().sht_tensor_download(self._h, _P(_ptr(out)), C.c_int64(nnz), _stream(stream)))
        return out

    def device_ptr(self) -> int:
        p = _P()
        _check(lib().sht_tensor_device_data(self._h, C.byref(p)))
        return p.value or 0

    def norms(self, norm: BlockNorm = BlockNorm.FROBENIUS, stream=None):
        n, _ = self.info()
        out = np.zeros(max(n, 1), np.float64)
        _check(lib().sht_tensor_norms(self._h, int(norm), out.ctypes.data_as(_P), _stream(stream)))
        return out[:n]

    def filter(self, eps: float, norm: BlockNorm = BlockNorm.FROBENIUS, compress: bool = True, stream=None):
        _check(lib().sht_tensor_filter(self._h, eps, int(norm), int(compress), _stream(stream)))
        return self

    def compress(self, stream=None):
        _check(lib().sht_tensor_compress(self._h, _stream(stream)))
        return self

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.sht_tensor_destroy(self._h)
            self._h = None


class Plan:
    """Matching + C pattern + work list of one contraction, reusable while patterns hold."""

    def __init__(self, ctx: Context, expr: str, A: Tensor, B: Tensor, Cten: Tensor, screen_eps: float = 0.0,
                 norm: BlockNorm = BlockNorm.FROBENIUS, mode: Mode = Mode.PLAIN_FP64, stream=None):
        h = _P()
        _check(lib().sht_plan_create(ctx.handle, expr.encode(), A.handle, B.handle, Cten.handle, screen_eps,
                                     int(norm), int(mode), _stream(stream), C.byref(h)))
        self._h = h
        self.refs = (A, B, Cten)

    def execute(self, alpha: float = 1.0, beta: float = 0.0, stream=None, graph: bool = False):
        fn = lib().sht_plan_execute_graph if graph else lib().sht_plan_execute
        _check(fn(self._h, alpha, beta, _stream(stream)))

    def report(self) -> dict:
        r = Report()
        _check(lib().sht_plan_report(self._h, C.byref(r)))
        return r.as_dict()

    def pairs(self) -> np.ndarray:
        n = self.report()["npairs"]
        out = np.zeros(max(n, 1) * 3, np.int64)
        _check(lib().sht_plan_pairs(self._h, out.ctypes.data_as(_P), C.c_int64(n)))
        return out[:3 * n].reshape(n, 3)

    def autotune(self, cache_file: str | None = None, stream=None):
        _check(lib().sht_autotune(self._h, cache_file.encode() if cache_file else None, _stream(stream)))

    def close(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.sht_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()


def contract(ctx: Context, expr: str, alpha: float, A: Tensor, B: Tensor, beta: float, Cten: Tensor,
             screen_eps: float = 0.0, norm: BlockNorm = BlockNorm.FROBENIUS, mode: Mode = Mode.PLAIN_FP64,
             stream=None) -> dict:
    """C = beta*C + alpha * contract(expr, A, B) on the device; returns the report."""
    r = Report()
    _check(lib().sht_contract(ctx.handle, expr.encode(), alpha, A.handle, B.handle, beta, Cten.handle, screen_eps,
                              int(norm), int(mode), _stream(stream), C.byref(r)))
    return r.as_dict()


def measure_peak(ctx: Context, which: str = "fp64") -> float:
    """Roofline denominators measured on this GPU: 'fp64' = FP64 FMA TFLOP/s, 'int8' = dense
    INT8 tensor-core TOPS, 'dmma' = FP64 tensor-core (m8n8k4) TFLOP/s, 'split_pipe' = the split
    kernel's operand pipeline alone (stage copies from L2 + the 7-slice MMA triangle), INT8 TOPS."""
    v = C.c_double()
    _check(lib().sht_measure_peak(ctx.handle, {"fp64": 0, "int8": 1, "dmma": 2, "split_pipe": 3}[which],
                                  C.byref(v)))
    return v.value


def compare(X: Tensor, Ref: Tensor, stream=None):
    mx, fr = C.c_double(), C.c_double()
    _check(lib().sht_tensor_compare(X.handle, Ref.handle, C.byref(mx), C.byref(fr), _stream(stream)))
    return mx.value, fr.value


def bitdiff(X: Tensor, Ref: Tensor, stream=None) -> int:
    """Number of elements whose bit patterns differ (0 = bit-identical, signed zeros included)."""
    n = C.c_int64()
    _check(lib().sht_tensor_bitdiff(X.handle, Ref.handle, C.byref(n), _stream(stream)))
    return n.value


class Server:
    """Serving loop: continuous batching of contractions over device-resident tensors.

    ``submit`` queues ``C = beta*C + alpha*contract(expr, A, B)`` and returns a request id;
    ``wait`` returns the request's report (and raises if the request failed).  With
    ``mode=Mode.BATCHED_FP64`` (the default) results equal :func:`contract` in
    ``Mode.BATCHED_FP64`` (and ``Mode.PLAIN_FP64``) bit for bit; with ``mode=Mode.SPLIT`` they
    equal :func:`contract` in ``Mode.SPLIT`` (a request with non-finite values or out-of-range
    exponents is served in the batched FP64 form; its report's ``form`` says which).  The
    tensors of a request must stay alive and unmodified until it has finished.
    """

    def __init__(self, ctx: Context, max_active: int = 0, max_batch: int = 0, reserve_bytes: int = 0,
                 planners: int = 0, ctas_per_sm: int = 0, mode: "Mode" = None):
        cfg = ServerConfig(max_active, max_batch, reserve_bytes, planners, ctas_per_sm,
                           int(mode) if mode is not None else 0)
        h = _P()
        _check(lib().sht_server_create(ctx.handle, C.byref(cfg), C.byref(h)))
        self._h = h
        self.ctx = ctx
        self._refs = {}

    def submit(self, expr: str, alpha: float, A: Tensor, B: Tensor, beta: float, Cten: Tensor,
               screen_eps: float = 0.0, norm: BlockNorm = BlockNorm.FROBENIUS) -> int:
        rid = C.c_int64()
        _check(lib().sht_server_submit(self._h, expr.encode(), alpha, A.handle, B.handle, beta, Cten.handle,
                                       screen_eps, int(norm), C.byref(rid)))
        self._refs[rid.value] = (A, B, Cten)
        return rid.value

    def poll(self, rid: int) -> bool:
        st = C.c_int()
        _check(lib().sht_server_poll(self._h, rid, C.byref(st)))
        return bool(st.value)

    def wait(self, rid: int, timeout: float = -1.0) -> dict:
        rep = RequestReport()
        rc = lib().sht_server_wait(self._h, rid, timeout, C.byref(rep))
        if rc != Status.ERR_TIMEOUT:
            self._refs.pop(rid, None)
        _check(rc)
        return rep.as_dict()

    def stats(self) -> dict:
        st = ServerStats()
        _check(lib().sht_server_get_stats(self._h, C.byref(st)))
        return st.as_dict()

    def reset_stats(self):
        _check(lib().sht_server_reset_stats(self._h))

    def close(self):
        if getattr(self, "_h", None) and _lib is not None:
            _check(_lib.sht_server_destroy(self._h))
            self._h = None
            self._refs.clear()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
