"""The plugin surface from Python: KernelInterface objects and Bench::run.

Thin ctypes wrapper over the gatlas_kernel_* / gatlas_bench_run entry points
of include/gatlas.h (the reference's KernelInterface, GatlasBenchmark.hpp:28-58).
"""

from __future__ import annotations

import ctypes

from . import check, lib

_declared = False


def _decl():
    global _declared
    if _declared:
        return lib()
    L = lib()
    vp, sz, i32 = ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int
    psz = ctypes.POINTER(ctypes.c_size_t)
    L.gatlas_kernel_create.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.POINTER(vp)]
    L.gatlas_kernel_destroy.argtypes = [vp]
    L.gatlas_kernel_destroy.restype = None
    L.gatlas_kernel_name.argtypes = [vp, ctypes.c_char_p, sz]
    L.gatlas_kernel_name.restype = sz
    L.gatlas_kernel_set_params.argtypes = [vp, psz, sz]
    L.gatlas_kernel_get_params.argtypes = [vp, psz, sz, psz]
    for n in ("gatlas_kernel_number_flops", "gatlas_kernel_total_variations"):
        getattr(L, n).argtypes = [vp]
        getattr(L, n).restype = sz
    for n in ("gatlas_kernel_extra_param_detail", "gatlas_kernel_global_work_items",
              "gatlas_kernel_local_work_items"):
        getattr(L, n).argtypes = [vp, psz, sz]
        getattr(L, n).restype = sz
    L.gatlas_kernel_print.argtypes = [vp, ctypes.c_char_p, sz]
    L.gatlas_kernel_print.restype = sz
    L.gatlas_kernel_paranoid_check.argtypes = [vp]
    L.gatlas_kernel_paranoid_check.restype = None
    L.gatlas_kernel_paranoid_fused.argtypes = [vp, i32]
    L.gatlas_kernel_paranoid_fused.restype = None
    L.gatlas_kernel_last_check.argtypes = [vp]
    L.gatlas_kernel_last_check.restype = ctypes.c_double
    L.gatlas_bench_run.argtypes = [vp, ctypes.c_char_p, sz, psz, sz, i32, i32, psz]
    _declared = True
    return L


def _arr(values):
    a = (ctypes.c_size_t * max(1, len(values)))(*values)
    return a


class Kernel:
    """A KernelInterface object of one family ("matmul", "matvec", "saxpy")
    and one -T type ("float4", "floatimg", "split3", ...)."""

    def __init__(self, op: str, type_: str):
        L = _decl()
        h = ctypes.c_void_p()
        check(L.gatlas_kernel_create(op.encode(), type_.encode(), ctypes.byref(h)))
        self._h = h
        self.op, self.type = op, type_

    def __del__(self):
        if getattr(self, "_h", None):
            _decl().gatlas_kernel_destroy(self._h)
            self._h = None

    def _str(self, fn) -> str:
        n = fn(self._h, None, 0)
        buf = ctypes.create_string_buffer(n + 1)
        fn(self._h, buf, n + 1)
        return buf.value.decode()

    def _vec(self, fn) -> list[int]:
        n = fn(self._h, None, 0)
        out = (ctypes.c_size_t * max(1, n))()
        fn(self._h, out, n)
        return list(out[:n])

    def kernel_name(self) -> str:
        return self._str(_decl().gatlas_kernel_name)

    def set_params(self, params) -> None:
        check(_decl().gatlas_kernel_set_params(self._h, _arr(list(params)), len(params)))

    def get_params(self):
        """(valid, params) -- the reference's getParams/validParams."""
        out = (ctypes.c_size_t * 32)()
        n = ctypes.c_size_t(0)
        ok = _decl().gatlas_kernel_get_params(self._h, out, 32, ctypes.byref(n))
        return bool(ok == 1), list(out[: n.value])

    def number_flops(self) -> int:
        return int(_decl().gatlas_kernel_number_flops(self._h))

    def total_variations(self) -> int:
        return int(_decl().gatlas_kernel_total_variations(self._h))

    def extra_param_detail(self) -> list[int]:
        return self._vec(_decl().gatlas_kernel_extra_param_detail)

    def global_work_items(self) -> list[int]:
        return self._vec(_decl().gatlas_kernel_global_work_items)

    def local_work_items(self) -> list[int]:
        return self._vec(_decl().gatlas_kernel_local_work_items)

    def print(self) -> str:
        return self._str(_decl().gatlas_kernel_print)

    def paranoid_check(self, fused: bool = True) -> None:
        """Random inputs and a device reference (paranoidCheck).  fused=False
        gives the reference the separately rounded arithmetic of the
        reference's host loops instead of the generated kernels' mad chain."""
        _decl().gatlas_kernel_paranoid_check(self._h)
        _decl().gatlas_kernel_paranoid_fused(self._h, int(bool(fused)))

    def last_check(self) -> float:
        """absdiff (normwise error for tensor-core engines and GEMV) of the
        last paranoid check."""
        return float(_decl().gatlas_kernel_last_check(self._h))

    def bench_run(self, params, trials=1, journal=None, bus_to_device=False,
                  bus_from_device=False) -> int:
        """Bench::run: microseconds, 0 when the point failed."""
        usec = ctypes.c_size_t(0)
        check(_decl().gatlas_bench_run(self._h, journal.encode() if journal else None, trials,
                                       _arr(list(params)), len(params), int(bus_to_device),
                                       int(bus_from_device), ctypes.byref(usec)))
        return int(usec.value)
