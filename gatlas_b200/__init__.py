"""gatlas_b200: B200-native GEMM / GEMV / SAXPY hot path of GATLAS.

Python binding of the C ABI declared in include/gatlas.h (ctypes over the
in-tree gatlas_b200/lib/libgatlas_b200.so).  Device memory, streams and
tensors come from PyTorch; every computation runs in the library's CUDA
kernels.  There is no CPU fallback: if the library is missing, the import of
any op raises.
"""

from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libgatlas_b200.so")

GATLAS_OK = 0
ERR_INVALID, ERR_CUDA, ERR_UNSUPPORTED, ERR_TIMEOUT, ERR_NOMEM, ERR_CHECK, ERR_STATE = (
    -1, -2, -3, -4, -5, -6, -7)

ENGINES = {"buffer": 0, "image": 1, "tc_bf16": 2, "tc_split3": 3, "tc_split6": 4, "tc_fp8": 5}
DISTS = {"uniform": 0, "pow2": 1, "const": 2}


class GatlasError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"gatlas status {status}: {message}")
        self.status = status


class MatmulDesc(ctypes.Structure):
    _fields_ = [("engine", ctypes.c_int32), ("gemm", ctypes.c_int32),
                ("trans_a", ctypes.c_int32), ("trans_b", ctypes.c_int32),
                ("m", ctypes.c_uint64), ("n", ctypes.c_uint64), ("k", ctypes.c_uint64),
                ("lda", ctypes.c_uint64), ("ldb", ctypes.c_uint64), ("ldc", ctypes.c_uint64),
                ("batch", ctypes.c_uint64), ("stride_a", ctypes.c_uint64),
                ("stride_b", ctypes.c_uint64), ("stride_c", ctypes.c_uint64),
                ("alpha", ctypes.c_double), ("beta", ctypes.c_double),
                ("group_h", ctypes.c_uint32), ("group_w", ctypes.c_uint32),
                ("block_h", ctypes.c_uint32), ("block_w", ctypes.c_uint32),
                ("vector_length", ctypes.c_uint32), ("extra", ctypes.c_uint32)]


class MatvecDesc(ctypes.Structure):
    _fields_ = [("engine", ctypes.c_int32), ("gemv", ctypes.c_int32),
                ("trans_a", ctypes.c_int32), ("reserved0", ctypes.c_int32),
                ("m", ctypes.c_uint64), ("n", ctypes.c_uint64), ("lda", ctypes.c_uint64),
                ("batch", ctypes.c_uint64), ("stride_a", ctypes.c_uint64),
                ("stride_x", ctypes.c_uint64), ("stride_y", ctypes.c_uint64),
                ("alpha", ctypes.c_double), ("beta", ctypes.c_double)]


class GroupedInstance(ctypes.Structure):
    _fields_ = [("a", ctypes.c_void_p), ("b", ctypes.c_void_p), ("c", ctypes.c_void_p),
                ("m", ctypes.c_int64), ("n", ctypes.c_int64), ("k", ctypes.c_int64),
                ("lda", ctypes.c_int64), ("ldb", ctypes.c_int64), ("ldc", ctypes.c_int64),
                ("trans_a", ctypes.c_int32), ("trans_b", ctypes.c_int32),
                ("gemm", ctypes.c_int32), ("tile_n", ctypes.c_int32),
                ("alpha", ctypes.c_double), ("beta", ctypes.c_double)]


GROUPED_BUCKETS = 4


class ServerConfig(ctypes.Structure):
    _fields_ = [("budget_bytes", ctypes.c_size_t), ("gemm_engine", ctypes.c_int32),
                ("max_batch", ctypes.c_int32), ("batch_target_ms", ctypes.c_double),
                ("gemm_tflops_estimate", ctypes.c_double)]


class ServerStats(ctypes.Structure):
    _fields_ = [("budget_bytes", ctypes.c_size_t), ("peak_bytes", ctypes.c_size_t),
                ("used_bytes", ctypes.c_size_t), ("gemm_batches", ctypes.c_int64),
                ("batched_gemms", ctypes.c_int64), ("host_busy_ns", ctypes.c_int64),
                ("iterations", ctypes.c_int64), ("phase_ns", ctypes.c_int64 * 5),
                ("generate_ns", ctypes.c_int64), ("generate_launches", ctypes.c_int64)]


_lib = None


def lib() -> ctypes.CDLL:
    """Loads the in-tree library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `make -j8` at the repository "
                           "root (or __graft_entry__.build())")
    L = ctypes.CDLL(LIB_PATH)
    vp, sz, i32, u64 = ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int, ctypes.c_uint64
    L.gatlas_version.restype = i32
    L.gatlas_status_string.restype = ctypes.c_char_p
    L.gatlas_status_string.argtypes = [i32]
    L.gatlas_last_error.restype = sz
    L.gatlas_last_error.argtypes = [ctypes.c_char_p, sz]
    L.gatlas_saxpy_f32.argtypes = [i32, sz, ctypes.c_float, vp, vp, vp, vp]
    L.gatlas_saxpy_f64.argtypes = [i32, sz, ctypes.c_double, vp, vp, vp, vp]
    L.gatlas_matvec_workspace_size.argtypes = [ctypes.POINTER(MatvecDesc)]
    L.gatlas_matvec_workspace_size.restype = sz
    for n in ("gatlas_matvec_f32", "gatlas_matvec_f64"):
        getattr(L, n).argtypes = [ctypes.POINTER(MatvecDesc), vp, vp, vp, vp, sz, vp]
    L.gatlas_matmul_workspace_size.argtypes = [ctypes.POINTER(MatmulDesc)]
    L.gatlas_matmul_workspace_size.restype = sz
    for n in ("gatlas_matmul_f32", "gatlas_matmul_f64"):
        getattr(L, n).argtypes = [ctypes.POINTER(MatmulDesc), vp, vp, vp, vp, sz, vp]
    L.gatlas_matmul_supported.argtypes = [i32, ctypes.POINTER(MatmulDesc)]
    L.gatlas_matmul_tc_prepare.argtypes = [ctypes.POINTER(MatmulDesc), vp, vp, vp, sz, vp]
    L.gatlas_matmul_tc_run.argtypes = [ctypes.POINTER(MatmulDesc), vp, sz, vp, vp]
    L.gatlas_matvec_f32_noalloc.argtypes = [ctypes.POINTER(MatvecDesc), vp, vp, vp, vp]
    L.gatlas_fill_f32.argtypes = [vp, sz, i32, u64, u64, ctypes.c_float, vp]
    L.gatlas_fill_f64.argtypes = [vp, sz, i32, u64, u64, ctypes.c_double, vp]
    L.gatlas_matmul_residual_f32.argtypes = [ctypes.POINTER(MatmulDesc), vp, vp, vp,
                                             ctypes.POINTER(ctypes.c_double), vp]
    L.gatlas_device_faults.argtypes = [ctypes.POINTER(ctypes.c_int), i32]
    L.gatlas_reference_matmul.argtypes = [i32, i32, ctypes.POINTER(MatmulDesc), vp, vp, vp, vp, vp]
    L.gatlas_reference_matvec.argtypes = [i32, i32, ctypes.POINTER(MatvecDesc), vp, vp, vp, vp, vp]
    L.gatlas_reference_saxpy.argtypes = [i32, i32, sz, ctypes.c_double, vp, vp, vp, vp]
    L.gatlas_matmul_f32_host.argtypes = [ctypes.POINTER(MatmulDesc), vp, vp, vp, vp]
    L.gatlas_set_option.argtypes = [ctypes.c_char_p, ctypes.c_int64]
    L.gatlas_selftest_bounded_wait.argtypes = [ctypes.c_int64, ctypes.c_int, ctypes.POINTER(ctypes.c_int), vp]
    L.gatlas_get_option.argtypes = [ctypes.c_char_p, ctypes.POINTER(ctypes.c_int64)]
    gi = ctypes.POINTER(GroupedInstance)
    L.gatlas_grouped_workspace_size.argtypes = [i32, gi, ctypes.c_int32]
    L.gatlas_grouped_workspace_size.restype = sz
    L.gatlas_grouped_create.argtypes = [i32, gi, ctypes.c_int32, vp, sz, ctypes.POINTER(vp)]
    for n in ("gatlas_grouped_prepare", "gatlas_grouped_run", "gatlas_grouped_run_each"):
        getattr(L, n).argtypes = [vp, vp]
    L.gatlas_grouped_launch_graph.argtypes = [vp, ctypes.c_int32, vp]
    L.gatlas_grouped_info.argtypes = [vp, ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int32),
                                      ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int64)]
    L.gatlas_grouped_destroy.argtypes = [vp]
    L.gatlas_grouped_destroy.restype = None
    L.gatlas_grouped_bucket.argtypes = [ctypes.c_int64, ctypes.c_int64, ctypes.c_int64]
    L.gatlas_grouped_bucket.restype = ctypes.c_int32
    L.gatlas_grouped_set_tile_table.argtypes = [i32, ctypes.POINTER(ctypes.c_int32), ctypes.c_int32]
    L.gatlas_grouped_get_tile_table.argtypes = [i32, ctypes.POINTER(ctypes.c_int32), ctypes.c_int32]
    L.gatlas_grouped_autotune.argtypes = [i32, ctypes.c_char_p, ctypes.c_int32, u64,
                                          ctypes.POINTER(ctypes.c_int32)]
    L.gatlas_server_create.argtypes = [ctypes.POINTER(ServerConfig), ctypes.POINTER(vp)]
    L.gatlas_server_run.argtypes = [vp, vp, ctypes.c_int32, ctypes.c_int32, vp]
    L.gatlas_server_release.argtypes = [vp, vp]
    L.gatlas_server_read.argtypes = [vp, vp, vp, ctypes.c_int64]
    L.gatlas_server_stats.argtypes = [vp, ctypes.POINTER(ServerStats)]
    L.gatlas_server_destroy.argtypes = [vp]
    L.gatlas_server_destroy.restype = None
    _lib = L
    return L


def last_error() -> str:
    buf = ctypes.create_string_buffer(512)
    lib().gatlas_last_error(buf, 512)
    return buf.value.decode(errors="replace")


def check(status: int) -> int:
    if status != GATLAS_OK:
        raise GatlasError(status, last_error() or lib().gatlas_status_string(status).decode())
    return status


# ---------------------------------------------------------------------------
# torch helpers
# ---------------------------------------------------------------------------

def _torch():
    import torch
    return torch


def _ptr(t):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def _stream(stream=None):
    torch = _torch()
    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)


def _engine(engine) -> int:
    return ENGINES[engine] if isinstance(engine, str) else int(engine)


def _require_cuda(*ts):
    for t in ts:
        if t is not None and not t.is_cuda:
            raise ValueError("gatlas_b200 ops take CUDA tensors")


# ---------------------------------------------------------------------------
# ops
# ---------------------------------------------------------------------------

def saxpy(alpha, x, y, out=None, engine="buffer", stream=None):
    """out = fma(alpha, x, y) elementwise (out may be y for in-place)."""
    torch = _torch()
    _require_cuda(x, y, out)
    if out is None:
        out = torch.empty_like(y)
    n = x.numel()
    assert y.numel() == n and out.numel() == n
    assert x.dtype == y.dtype == out.dtype
    if x.dtype == torch.float32:
        fn = lib().gatlas_saxpy_f32
    elif x.dtype == torch.float64:
        fn = lib().gatlas_saxpy_f64
    else:
        raise TypeError(f"saxpy: unsupported dtype {x.dtype}")
    check(fn(_engine(engine), n, float(alpha), _ptr(x), _ptr(y), _ptr(out), _stream(stream)))
    return out


def matvec_desc(M, N, trans_a=False, gemv=False, alpha=1.0, beta=0.0, engine="buffer",
                lda=0, batch=1, stride_a=0, stride_x=0, stride_y=0) -> MatvecDesc:
    return MatvecDesc(engine=_engine(engine), gemv=int(bool(gemv)), trans_a=int(bool(trans_a)),
                      reserved0=0, m=M, n=N, lda=lda, batch=batch, stride_a=stride_a,
                      stride_x=stride_x, stride_y=stride_y, alpha=alpha, beta=beta)


def matvec(A, x, M, N, y=None, trans_a=False, gemv=False, alpha=1.0, beta=0.0,
           engine="buffer", batch=1, workspace=None, stream=None):
    """y = A·x (or alpha·A·x + beta·y).  A is flat: trans_a=False → M×N
    row-major; trans_a=True → column-major (N rows of M)."""
    torch = _torch()
    _require_cuda(A, x, y)
    if y is None:
        y = torch.zeros(batch * M, dtype=A.dtype, device=A.device)
    d = matvec_desc(M, N, trans_a, gemv, alpha, beta, engine, batch=batch)
    fn = lib().gatlas_matvec_f32 if A.dtype == torch.float32 else lib().gatlas_matvec_f64
    ws = _ptr(workspace)
    wsb = 0 if workspace is None else workspace.numel() * workspace.element_size()
    check(fn(ctypes.byref(d), _ptr(A), _ptr(x), _ptr(y), ws, wsb, _stream(stream)))
    return y


def matvec_workspace_size(M, N, trans_a=False, batch=1) -> int:
    d = matvec_desc(M, N, trans_a, batch=batch)
    return int(lib().gatlas_matvec_workspace_size(ctypes.byref(d)))


def matmul_desc(M, N, K, trans_a=False, trans_b=False, gemm=False, alpha=1.0, beta=0.0,
                engine="buffer", tile=None, batch=1, lda=0, ldb=0, ldc=0,
                stride_a=0, stride_b=0, stride_c=0) -> MatmulDesc:
    t = tuple(tile or ())
    gh, gw, bh, bw, vl, x = t + (0,) * (6 - len(t))
    return MatmulDesc(engine=_engine(engine), gemm=int(bool(gemm)), trans_a=int(bool(trans_a)),
                      trans_b=int(bool(trans_b)), m=M, n=N, k=K, lda=lda, ldb=ldb, ldc=ldc,
                      batch=batch, stride_a=stride_a, stride_b=stride_b, stride_c=stride_c,
                      alpha=alpha, beta=beta, group_h=gh, group_w=gw, block_h=bh, block_w=bw,
                      vector_length=vl, extra=x)


def matmul(A, B, M, N, K, C=None, trans_a=False, trans_b=False, gemm=False, alpha=1.0,
           beta=0.0, engine="buffer", tile=None, batch=1, workspace=None, stream=None):
    """C = op(A)·op(B) (or alpha·op(A)·op(B) + beta·C) on flat tensors in the
    reference's layouts (see include/gatlas.h)."""
    torch = _torch()
    _require_cuda(A, B, C)
    if C is None:
        C = torch.empty(batch * M * N, dtype=A.dtype, device=A.device)
    d = matmul_desc(M, N, K, trans_a, trans_b, gemm, alpha, beta, engine, tile, batch)
    fn = lib().gatlas_matmul_f32 if A.dtype == torch.float32 else lib().gatlas_matmul_f64
    ws = _ptr(workspace)
    wsb = 0 if workspace is None else workspace.numel() * workspace.element_size()
    check(fn(ctypes.byref(d), _ptr(A), _ptr(B), _ptr(C), ws, wsb, _stream(stream)))
    return C


def matmul_tc_prepare(A, B, M, N, K, workspace, trans_a=False, trans_b=False, engine="tc_split3",
                      batch=1, extra=0, stream=None):
    """Writes the BF16 pieces of A and B into `workspace` (tensor-core engines)."""
    d = matmul_desc(M, N, K, trans_a, trans_b, engine=engine, batch=batch,
                    tile=(0, 0, 0, 0, 0, extra))
    check(lib().gatlas_matmul_tc_prepare(ctypes.byref(d), _ptr(A), _ptr(B), _ptr(workspace),
                                         workspace.numel() * workspace.element_size(),
                                         _stream(stream)))


def matmul_tc_run(workspace, M, N, K, C, trans_a=False, trans_b=False, engine="tc_split3",
                  gemm=False, alpha=1.0, beta=0.0, batch=1, extra=0, stream=None):
    """Contracts the pieces prepared in `workspace` into C."""
    d = matmul_desc(M, N, K, trans_a, trans_b, gemm, alpha, beta, engine, batch=batch,
                    tile=(0, 0, 0, 0, 0, extra))
    check(lib().gatlas_matmul_tc_run(ctypes.byref(d), _ptr(workspace),
                                     workspace.numel() * workspace.element_size(), _ptr(C),
                                     _stream(stream)))
    return C


def matmul_supported(engine="buffer", tile=None, trans_a=False, trans_b=False, double=False):
    """1: prebuilt kernel; 2: compiled at run time on first use; 0: cannot run."""
    d = matmul_desc(1, 1, 1, trans_a, trans_b, engine=engine, tile=tile)
    return int(lib().gatlas_matmul_supported(int(double), ctypes.byref(d)))


def matmul_workspace_size(M, N, K, engine, trans_a=False, trans_b=False, batch=1) -> int:
    d = matmul_desc(M, N, K, trans_a, trans_b, engine=engine, batch=batch)
    return int(lib().gatlas_matmul_workspace_size(ctypes.byref(d)))


def fill(t, dist="uniform", seed=0, offset=0, value=0.0, stream=None):
    """Seeded device-side fill (same stream as the host oracle's generators)."""
    torch = _torch()
    _require_cuda(t)
    fn = lib().gatlas_fill_f32 if t.dtype == torch.float32 else lib().gatlas_fill_f64
    check(fn(_ptr(t), t.numel(), DISTS[dist] if isinstance(dist, str) else int(dist), seed,
             offset, float(value), _stream(stream)))
    return t


def residual(A, B, C, M, N, K, trans_a=False, trans_b=False, alpha=1.0, stream=None):
    """FP64 residual of C against op(A)·op(B) computed on the GPU in double:
    (||C-Cref||_F, ||Cref||_F, max|C-Cref|, sum|C-Cref|)."""
    d = matmul_desc(M, N, K, trans_a, trans_b, gemm=alpha != 1.0, alpha=alpha)
    out = (ctypes.c_double * 4)()
    check(lib().gatlas_matmul_residual_f32(ctypes.byref(d), _ptr(A), _ptr(B), _ptr(C), out,
                                           _stream(stream)))
    return tuple(out)


def _scalar(t) -> int:
    torch = _torch()
    return 0 if t.dtype == torch.float32 else 1


def reference_matmul(A, B, M, N, K, fused=True, Cin=None, trans_a=False, trans_b=False, gemm=False,
                     alpha=1.0, beta=0.0, batch=1, stream=None):
    """The paranoid check's device reference product (gatlas_reference_matmul):
    fused mad chain, or (fused=False) separately rounded products and sums."""
    torch = _torch()
    _require_cuda(A, B, Cin)
    C = torch.empty(batch * M * N, dtype=A.dtype, device=A.device)
    d = matmul_desc(M, N, K, trans_a, trans_b, gemm, alpha, beta, batch=batch)
    check(lib().gatlas_reference_matmul(_scalar(A), int(bool(fused)), ctypes.byref(d), _ptr(A), _ptr(B),
                                        _ptr(Cin), _ptr(C), _stream(stream)))
    return C


def reference_matvec(A, x, M, N, fused=True, yin=None, trans_a=False, gemv=False, alpha=1.0, beta=0.0,
                     batch=1, stream=None):
    torch = _torch()
    _require_cuda(A, x, yin)
    y = torch.empty(batch * M, dtype=A.dtype, device=A.device)
    d = matvec_desc(M, N, trans_a, gemv, alpha, beta, batch=batch)
    check(lib().gatlas_reference_matvec(_scalar(A), int(bool(fused)), ctypes.byref(d), _ptr(A), _ptr(x),
                                        _ptr(yin), _ptr(y), _stream(stream)))
    return y


def reference_saxpy(alpha, x, y, fused=True, stream=None):
    torch = _torch()
    _require_cuda(x, y)
    z = torch.empty_like(x)
    check(lib().gatlas_reference_saxpy(_scalar(x), int(bool(fused)), x.numel(), float(alpha), _ptr(x), _ptr(y),
                                       _ptr(z), _stream(stream)))
    return z


def device_faults(clear=True) -> int:
    v = ctypes.c_int(0)
    check(lib().gatlas_device_faults(ctypes.byref(v), int(clear)))
    return v.value


# ---------------------------------------------------------------------------
# grouped GEMM: many uneven instances per persistent launch
# ---------------------------------------------------------------------------

def _grouped_instances(instances):
    arr = (GroupedInstance * max(len(instances), 1))()
    for i, q in enumerate(instances):
        r = arr[i]
        r.a = q["A"].data_ptr() if q.get("A") is not None else None
        r.b = q["B"].data_ptr() if q.get("B") is not None else None
        r.c = q["C"].data_ptr() if q.get("C") is not None else None
        r.m, r.n, r.k = int(q["m"]), int(q["n"]), int(q["k"])
        r.lda, r.ldb, r.ldc = int(q.get("lda", 0)), int(q.get("ldb", 0)), int(q.get("ldc", 0))
        r.trans_a, r.trans_b = int(bool(q.get("trans_a", 0))), int(bool(q.get("trans_b", 0)))
        r.gemm = int(bool(q.get("gemm", 0)))
        r.tile_n = int(q.get("tile_n", 0))
        r.alpha, r.beta = float(q.get("alpha", 1.0)), float(q.get("beta", 0.0))
    return arr


def grouped_workspace_size(instances, engine="tc_split3") -> int:
    """Packed workspace bytes; instances as for Grouped (tensors may be omitted)."""
    arr = _grouped_instances(instances)
    return int(lib().gatlas_grouped_workspace_size(_engine(engine), arr, len(instances)))


def grouped_bucket(m, n, k) -> int:
    return int(lib().gatlas_grouped_bucket(m, n, k))


def grouped_tile_table(engine="tc_split3", table=None):
    """Returns the per-bucket tile widths; sets them first when `table` is given."""
    buf = (ctypes.c_int32 * GROUPED_BUCKETS)()
    if table is not None:
        for i, v in enumerate(table):
            buf[i] = int(v)
        check(lib().gatlas_grouped_set_tile_table(_engine(engine), buf, GROUPED_BUCKETS))
    check(lib().gatlas_grouped_get_tile_table(_engine(engine), buf, GROUPED_BUCKETS))
    return list(buf)


def grouped_autotune(engine="tc_split3", journal=None, trials=3, seed=1):
    """Times tile widths 64/128/256 per size bucket, journals every candidate
    and installs the winners; returns the table."""
    out = (ctypes.c_int32 * GROUPED_BUCKETS)()
    check(lib().gatlas_grouped_autotune(_engine(engine), journal.encode() if journal else None, trials, seed,
                                        out))
    return list(out)


class Grouped:
    """A grouped GEMM plan over instances given as dicts with keys A, B, C
    (device float32 tensors), m, n, k and optionally lda, ldb, ldc, trans_a,
    trans_b, gemm, alpha, beta, tile_n.  The tensors are bound at creation."""

    def __init__(self, instances, engine="tc_split3", workspace=None):
        self._keep = [(q.get("A"), q.get("B"), q.get("C")) for q in instances]
        self._ws = workspace
        self.engine = engine
        self._h = ctypes.c_void_p()
        arr = _grouped_instances(instances)
        wsb = 0 if workspace is None else workspace.numel() * workspace.element_size()
        check(lib().gatlas_grouped_create(_engine(engine), arr, len(instances), _ptr(workspace), wsb,
                                          ctypes.byref(self._h)))

    def prepare(self, stream=None):
        check(lib().gatlas_grouped_prepare(self._h, _stream(stream)))
        return self

    def run(self, stream=None):
        check(lib().gatlas_grouped_run(self._h, _stream(stream)))
        return self

    def launch_graph(self, with_prepare=True, stream=None):
        check(lib().gatlas_grouped_launch_graph(self._h, int(bool(with_prepare)), _stream(stream)))
        return self

    def run_each(self, stream=None):
        check(lib().gatlas_grouped_run_each(self._h, _stream(stream)))
        return self

    def info(self) -> dict:
        t, c, f, it = ctypes.c_int64(), ctypes.c_int32(), ctypes.c_double(), ctypes.c_int64()
        check(lib().gatlas_grouped_info(self._h, ctypes.byref(t), ctypes.byref(c), ctypes.byref(f),
                                        ctypes.byref(it)))
        return {"tiles": t.value, "ctas": c.value, "flops": f.value, "pack_items": it.value}

    def close(self):
        if self._h:
            lib().gatlas_grouped_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------------
# serving: continuous batching of mixed requests under a memory budget
# ---------------------------------------------------------------------------

REQ_GEMM, REQ_GEMV, REQ_SAXPY = 0, 1, 2
SERVE_MODES = {"continuous": 0, "serial": 1}


def request_dtype():
    """numpy layout of gatlas_request (72 bytes)."""
    import numpy as np
    return np.dtype([("kind", "<i4"), ("trans_a", "<i4"), ("trans_b", "<i4"), ("retain", "<i4"),
                     ("m", "<i8"), ("n", "<i8"), ("k", "<i8"), ("alpha", "<f8"), ("beta", "<f8"),
                     ("seed", "<u8"), ("arrival_ns", "<i8")], align=True)


def result_dtype():
    """numpy layout of gatlas_request_result (48 bytes)."""
    import numpy as np
    return np.dtype([("admit_ns", "<i8"), ("start_ns", "<i8"), ("done_ns", "<i8"), ("status", "<i4"),
                     ("batch", "<i4"), ("result", "<u8"), ("result_elems", "<i8")], align=True)


class Server:
    """The serving loop: Server(budget_bytes).run(requests, mode) with requests
    a numpy array of request_dtype(); returns an array of result_dtype()."""

    def __init__(self, budget_bytes, engine="tc_split3", max_batch=0, batch_target_ms=0.0,
                 gemm_tflops_estimate=0.0):
        cfg = ServerConfig(int(budget_bytes), _engine(engine), int(max_batch), float(batch_target_ms),
                           float(gemm_tflops_estimate))
        self._h = ctypes.c_void_p()
        check(lib().gatlas_server_create(ctypes.byref(cfg), ctypes.byref(self._h)))

    def run(self, requests, mode="continuous"):
        import numpy as np
        req = np.ascontiguousarray(requests, dtype=request_dtype())
        out = np.zeros(len(req), dtype=result_dtype())
        check(lib().gatlas_server_run(self._h, req.ctypes.data if len(req) else None, len(req),
                                      SERVE_MODES[mode] if isinstance(mode, str) else int(mode),
                                      out.ctypes.data if len(req) else None))
        return out

    def read(self, result_row):
        """Host copy of a retained result."""
        import numpy as np
        host = np.empty(int(result_row["result_elems"]), dtype=np.float32)
        check(lib().gatlas_server_read(self._h, ctypes.c_void_p(int(result_row["result"])), host.ctypes.data,
                                       host.size))
        return host

    def release(self, result_row):
        check(lib().gatlas_server_release(self._h, ctypes.c_void_p(int(result_row["result"]))))

    def stats(self) -> dict:
        st = ServerStats()
        check(lib().gatlas_server_stats(self._h, ctypes.byref(st)))
        out = {f: getattr(st, f) for f, _ in ServerStats._fields_}
        out["phase_ns"] = list(st.phase_ns)
        return out

    def close(self):
        if self._h:
            lib().gatlas_server_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def set_option(name: str, value: int) -> None:
    """Library options (see gatlas_set_option in include/gatlas.h): "tc_pair"
    (tiling of tensor-core contractions: 1 default, 0 128 x 256 tiles, 2 CTA
    pairs), "tc_group_rows" (raster group height, multiple of 128),
    "host_block_rows" (row block of the host-buffer pipeline, multiple of 256),
    "tc_l2_hint" (1 default: A's tiles evict-last in L2; 0 plain loads)
    and "grouped_pair" (grouped contractions on CTA pairs: 1, or single CTAs:
    0, the default)."""
    check(lib().gatlas_set_option(name.encode(), int(value)))


def get_option(name: str) -> int:
    v = ctypes.c_int64()
    check(lib().gatlas_get_option(name.encode(), ctypes.byref(v)))
    return int(v.value)


def matmul_host(A, B, M, N, K, C, trans_a=False, trans_b=False, gemm=False, alpha=1.0, beta=0.0,
                engine="tc_split3", batch=1, extra=0, stream=None, lda=0, ldb=0, ldc=0,
                stride_a=0, stride_b=0, stride_c=0):
    """C = op(A)op(B) with host (CPU, ideally pinned) float32 tensors: upload,
    contract and download in one call, ordered on the current CUDA stream.
    Leading dimensions and instance strides as in include/gatlas.h (0 = dense);
    only the M x N elements of each instance of C are written."""
    for t in (A, B, C):
        if t is not None and t.is_cuda:
            raise ValueError("matmul_host takes host tensors")
    d = matmul_desc(M, N, K, trans_a, trans_b, gemm, alpha, beta, engine, batch=batch,
                    tile=(0, 0, 0, 0, 0, extra), lda=lda, ldb=ldb, ldc=ldc,
                    stride_a=stride_a, stride_b=stride_b, stride_c=stride_c)
    check(lib().gatlas_matmul_f32_host(ctypes.byref(d), _ptr(A), _ptr(B), _ptr(C), _stream(stream)))
    return C


FAULT_SELFTEST_WAIT = 1 << 6


def selftest_bounded_wait(limit_ns=1_000_000, arrive=False, stream=None) -> bool:
    """Runs the bounded mbarrier wait every TMA kernel uses; True when the wait
    completed, False when it ran out (and set FAULT_SELFTEST_WAIT)."""
    done = ctypes.c_int(-1)
    s = None if stream is None else _stream(stream)  # NULL: the legacy default stream
    check(lib().gatlas_selftest_bounded_wait(int(limit_ns), int(bool(arrive)), ctypes.byref(done), s))
    return done.value == 1
