"""Oracle restatement of GATLAS's kernel parameter space and journal.

TEST INFRASTRUCTURE ONLY: the product implements the same rules in C++
(gatlas_b200/csrc/host); tests compare the two over broad sweeps, and this
module is pinned by the parameter lines the reference prints in its own
documentation (tests/golden/reference_examples.json).

Every rule cites the reference file and line it restates.
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field

# Journal run states (GatlasBenchmark.hpp:72-76)
MISSING, BUILD_IN_PROGRESS, BUILD_OK, RUN_IN_PROGRESS, RUN_OK = 0, -1, -2, -3, -4

# OpenCL's max work group size on the CUDA target: 1024 threads per block.
MAX_WORK_GROUP_SIZE = 1024


def _decode_extra(value: int, variations: list[int]) -> list[int]:
    """Mixed-radix decode of the extra parameter (KernelBaseMatmul.cpp:160-169)."""
    out = []
    shift = 1
    for i, nv in enumerate(variations):
        if i > 0:
            shift *= variations[i - 1]
        out.append((value // shift) % nv)
    return out


def _scalar_name(scalar: str) -> str:
    assert scalar in ("float", "double")
    return scalar


@dataclass
class Matmul:
    """KernelBaseMatmul + KernelMatmul{Buffer,Image} parameter rules."""

    variant: str = "buffer"   # "buffer" | "image"
    scalar: str = "float"
    vl: int = 4               # template VECTOR_LENGTH
    packed: int = 1
    gemm: int = 0
    M: int = 0
    N: int = 0
    K: int = 0
    tA: int = 0
    tB: int = 0
    gh: int = 0
    gw: int = 0
    bh: int = 0
    bw: int = 0
    x: int = 0

    def variations(self) -> list[int]:
        # buffer: inlineMNK(2), loopOrder(6) (KernelMatmulBuffer.hpp:27-29,45-46)
        # image : + globalID(2)           (KernelMatmulImage.hpp:27-30,48-50)
        return [2, 6] if self.variant == "buffer" else [2, 6, 2]

    def total_variations(self) -> int:
        return math.prod(self.variations())

    def extra_param_detail(self) -> list[int]:
        return _decode_extra(self.x, self.variations())

    def kernel_name(self) -> str:
        # KernelMatmulBuffer.hpp:58-62, KernelMatmulImage.hpp:63-67
        return f"matmul{self.variant}{_scalar_name(self.scalar)}{self.vl}"

    def group_size(self) -> int:
        # MatmulWorkGroup::groupSize (KernelBaseMatmul.cpp:86-88)
        return self.gw if self.gw == self.gh else 0

    def valid(self) -> bool:
        """KernelBaseMatmul::validParams (KernelBaseMatmul.cpp:263-291).

        VECTOR_LENGTH there is blockWidth(); a zero divisor (which would trap
        in the reference) counts as invalid."""
        VL = self.bw
        M, N, K = self.M, self.N, self.K
        try:
            return bool(
                self.packed > 0
                and M % VL == 0 and N % VL == 0 and K % VL == 0
                and M % (self.gh * self.bh) == 0
                and N % (self.gw * self.bw) == 0
                and K % (self.gh * VL) == 0
                and self.gh * self.bh <= M
                and self.gw * self.bw <= N
                and self.gh * VL <= K
                and ((self.bh % VL == 0) if self.tA else True)
                and self.x < self.total_variations()
            )
        except ZeroDivisionError:
            return False

    def params(self) -> list[int]:
        # KernelBaseMatmul::getParams order (KernelBaseMatmul.cpp:293-325)
        return [self.packed, int(bool(self.gemm)), self.M, self.N, self.K,
                int(bool(self.tA)), int(bool(self.tB)), self.gh, self.gw,
                self.bh, self.bw, self.x]

    def set_params(self, p: list[int]) -> None:
        # KernelBaseMatmul::setParams (KernelBaseMatmul.cpp:327-362)
        (self.packed, self.gemm, self.M, self.N, self.K, self.tA, self.tB,
         self.gh, self.gw, self.bh, self.bw, self.x) = [int(v) for v in p[:12]]

    def global_work_items(self) -> list[int]:
        return [self.N // self.bw, self.M // self.bh]   # KernelBaseMatmul.cpp:364-369

    def local_work_items(self) -> list[int]:
        return [self.gw, self.gh]                       # KernelBaseMatmul.cpp:371-376

    def number_flops(self) -> int:
        # KernelBaseMatmul.cpp:378-383
        if self.gemm:
            return self.packed * 2 * self.M * self.N * (self.K + 1)
        return self.packed * self.M * self.N * (2 * self.K - 1)


@dataclass
class Matvec:
    """KernelBaseMatvec + KernelMatvec{Buffer,Image} parameter rules."""

    variant: str = "buffer"
    scalar: str = "float"
    vl: int = 4
    packed: int = 1
    gemv: int = 0
    M: int = 0
    N: int = 0
    tA: int = 0
    g: int = 0
    bh: int = 0
    x: int = 0

    def variations(self) -> list[int]:
        # buffer: inlineMN(2) (KernelMatvecBuffer.hpp:27-28); image adds globalID(2)
        # (KernelMatvecImage.hpp:27-29)
        return [2] if self.variant == "buffer" else [2, 2]

    def total_variations(self) -> int:
        return math.prod(self.variations())

    def extra_param_detail(self) -> list[int]:
        return _decode_extra(self.x, self.variations())

    def kernel_name(self) -> str:
        return f"matvec{self.variant}{_scalar_name(self.scalar)}{self.vl}"

    def valid(self) -> bool:
        """KernelBaseMatvec::validParams (KernelBaseMatvec.cpp:236-257)."""
        VL = self.vl
        try:
            return bool(
                self.packed > 0
                and self.M % VL == 0 and self.N % VL == 0
                and self.M % (self.g * self.bh) == 0
                and self.N % (self.g * VL) == 0
                and self.g * self.bh <= self.M
                and self.g * VL <= self.N
                and self.bh % VL == 0
                and self.x < self.total_variations()
            )
        except ZeroDivisionError:
            return False

    def params(self) -> list[int]:
        # KernelBaseMatvec.cpp:259-288
        return [self.packed, int(bool(self.gemv)), self.M, self.N, int(bool(self.tA)),
                self.g, self.bh, self.vl, self.x]

    def set_params(self, p: list[int]) -> None:
        (self.packed, self.gemv, self.M, self.N, self.tA, self.g, self.bh,
         vl, self.x) = [int(v) for v in p[:9]]
        self.vl = vl

    def global_work_items(self) -> list[int]:
        return [self.M // self.bh]                      # KernelBaseMatvec.cpp:324-328

    def local_work_items(self) -> list[int]:
        return [self.g]                                 # KernelBaseMatvec.cpp:330-334

    def number_flops(self) -> int:
        # KernelBaseMatvec.cpp:336-341
        if self.gemv:
            return self.packed * 2 * self.M * (self.N + 1)
        return self.packed * self.M * (2 * self.N - 1)


@dataclass
class Saxpy:
    """KernelBaseSaxpy + KernelSaxpy{Buffer,Image} parameter rules."""

    variant: str = "buffer"
    scalar: str = "float"
    vl: int = 4
    packed: int = 1
    M: int = 0
    N: int = 0
    gh: int = 0
    gw: int = 0
    bh: int = 0
    bw: int = 0
    x: int = 0

    def variations(self) -> list[int]:
        # buffer: inlineMN(2) (KernelSaxpyBuffer.hpp:26-28); image adds globalID(2)
        return [2] if self.variant == "buffer" else [2, 2]

    def total_variations(self) -> int:
        return math.prod(self.variations())

    def extra_param_detail(self) -> list[int]:
        return _decode_extra(self.x, self.variations())

    def kernel_name(self) -> str:
        return f"saxpy{self.variant}{_scalar_name(self.scalar)}{self.vl}"

    def valid(self) -> bool:
        """KernelBaseSaxpy::validParams (KernelBaseSaxpy.cpp:210-231)."""
        VL = self.vl
        try:
            return bool(
                self.packed > 0
                and self.M % VL == 0 and self.N % VL == 0
                and self.M % (self.gh * self.bh) == 0
                and ((self.N % (self.gw * self.bw) == 0) if (self.gw and self.bw) else True)
                and self.gh * self.bh <= self.M
                and self.gw * self.bw <= self.N
                and self.bw % VL == 0
                and self.x < self.total_variations()
            )
        except ZeroDivisionError:
            return False

    def params(self) -> list[int]:
        # KernelBaseSaxpy.cpp:233-258
        return [self.packed, self.M, self.N, self.gh, self.gw, self.bh, self.bw,
                self.vl, self.x]

    def set_params(self, p: list[int]) -> None:
        (self.packed, self.M, self.N, self.gh, self.gw, self.bh, self.bw,
         vl, self.x) = [int(v) for v in p[:9]]
        self.vl = vl

    def global_work_items(self) -> list[int]:
        # KernelBaseSaxpy.cpp:289-294
        dims = [self.M // self.bh]
        if self.bw:
            dims.append(self.N // self.bw)
        return dims

    def local_work_items(self) -> list[int]:
        dims = [self.gh]
        if self.gw:
            dims.append(self.gw)
        return dims

    def number_flops(self) -> int:
        return self.packed * 2 * self.M * self.N       # KernelBaseSaxpy.cpp:303-305


def journal_key(kernel_name: str, params: list[int]) -> str:
    """Journal::toString (GatlasBenchmark.cpp:44-50): name_p0_p1_..._"""
    return kernel_name + "_" + "".join(f"{p}_" for p in params)


# ---------------------------------------------------------------------------
# search-space enumeration (bench*.cpp getParams)
# ---------------------------------------------------------------------------

# -T kernel type table (benchMatmul.cpp:141-160): (variant, scalar, VL, maxBH, maxWG)
MATMUL_TYPES = {
    "float1": ("buffer", "float", 1, 10, 10),
    "float2": ("buffer", "float", 2, 10, 10),
    "float4": ("buffer", "float", 4, 10, 10),
    "double1": ("buffer", "double", 1, 10, 10),
    "double2": ("buffer", "double", 2, 10, 10),
    "double4": ("buffer", "double", 4, 10, 10),
    "floatimg": ("image", "float", 4, 12, 16),
    "doubleimg": ("image", "double", 2, 12, 16),
}

# benchMatvec.cpp:131-150: maxBlockHeight 64, maxGroupSize 256 for every type
MATVEC_TYPES = {k: (v[0], v[1], v[2], 64, 256) for k, v in MATMUL_TYPES.items()}

# benchSaxpy.cpp:116-134 (maxBlockHeight / maxGroupSize set elsewhere to 8 / 256)
SAXPY_TYPES = {k: (v[0], v[1], v[2]) for k, v in MATMUL_TYPES.items()}


def matmul_search_space(kernel: Matmul, max_bh: int, max_wg: int,
                        group_size: int = -1, block_height: int = -1,
                        extra_param: int = -1) -> list[list[int]]:
    """benchMatmul.cpp getParams (:217-304)."""
    out: list[list[int]] = []
    vl = kernel.vl
    if group_size != -1:
        kernel.gh = kernel.gw = group_size
    if block_height != -1:
        kernel.bh, kernel.bw = block_height, vl
    if extra_param != -1:
        kernel.x = extra_param

    def push():
        if kernel.valid():
            out.append(kernel.params())
            return True
        return False

    if group_size != -1 and block_height != -1 and extra_param != -1:
        push()
    elif group_size != -1 and block_height != -1:
        for xp in range(kernel.total_variations()):
            kernel.x = xp
            push()
    elif group_size != -1:
        for bh in range(vl, max_bh + 1):
            kernel.bh, kernel.bw = bh, vl
            for xp in range(kernel.total_variations()):
                kernel.x = xp
                push()
    else:
        largest_possible = int(math.sqrt(MAX_WORK_GROUP_SIZE))
        largest = min(max_wg, largest_possible)
        bh_min = block_height if block_height != -1 else vl
        bh_max = block_height if block_height != -1 else max_bh
        xp_min = extra_param if extra_param != -1 else 0
        xp_max = extra_param + 1 if extra_param != -1 else kernel.total_variations()
        wg = largest
        while wg > 8:
            kernel.gh = kernel.gw = wg
            not_empty = False
            for bh in range(bh_min, bh_max + 1):
                kernel.bh, kernel.bw = bh, vl
                for xp in range(xp_min, xp_max):
                    kernel.x = xp
                    if push():
                        not_empty = True
            if not_empty:
                break
            wg -= 1
        kernel.gh = kernel.gw = 8
        for bh in range(bh_min, bh_max + 1):
            kernel.bh, kernel.bw = bh, vl
            for xp in range(xp_min, xp_max):
                kernel.x = xp
                push()
    return out


def matvec_search_space(kernel: Matvec, max_bh: int, max_wg: int,
                        group_size: int = -1, block_height: int = -1,
                        extra_param: int = -1) -> list[list[int]]:
    """benchMatvec.cpp getParams (:202-289)."""
    out: list[list[int]] = []
    vl = kernel.vl
    if group_size != -1:
        kernel.g = group_size
    if block_height != -1:
        kernel.bh = block_height
    if extra_param != -1:
        kernel.x = extra_param

    def push():
        if kernel.valid():
            out.append(kernel.params())
            return True
        return False

    if group_size != -1 and block_height != -1 and extra_param != -1:
        push()
    elif group_size != -1 and block_height != -1:
        for xp in range(kernel.total_variations()):
            kernel.x = xp
            push()
    elif group_size != -1:
        for bh in range(vl, max_bh + 1):
            kernel.bh = bh
            for xp in range(kernel.total_variations()):
                kernel.x = xp
                push()
    else:
        largest = min(max_wg, MAX_WORK_GROUP_SIZE)
        bh_min = block_height if block_height != -1 else vl
        bh_max = block_height if block_height != -1 else max_bh
        xp_min = extra_param if extra_param != -1 else 0
        xp_max = extra_param + 1 if extra_param != -1 else kernel.total_variations()
        wg = largest
        while wg > 64:
            kernel.g = wg
            not_empty = False
            for bh in range(bh_min, bh_max + 1):
                kernel.bh = bh
                for xp in range(xp_min, xp_max):
                    kernel.x = xp
                    if push():
                        not_empty = True
            if not_empty:
                break
            wg -= 1
        kernel.g = 64
        for bh in range(bh_min, bh_max + 1):
            kernel.bh = bh
            for xp in range(xp_min, xp_max):
                kernel.x = xp
                push()
    return out


# ---------------------------------------------------------------------------
# journal (GatlasBenchmark.cpp:41-137)
# ---------------------------------------------------------------------------

@dataclass
class Journal:
    path: str
    run_state: dict = field(default_factory=dict)
    times: dict = field(default_factory=dict)

    def load(self) -> bool:
        """Journal::loadMemo (GatlasBenchmark.cpp:56-73): whitespace-separated
        (key, int) pairs; negative = run state (last wins), else a time."""
        try:
            with open(self.path) as f:
                toks = f.read().split()
        except OSError:
            return False
        self.run_state.clear()
        self.times.clear()
        for i in range(0, len(toks) - 1, 2):
            key, sval = toks[i], toks[i + 1]
            try:
                value = int(sval)
            except ValueError:
                break   # operator>> into an int fails: the reference stops reading
            if value < 0:
                self.run_state[key] = value
            else:
                self.times.setdefault(key, []).append(value)
        return True

    def purge(self, delete_times: bool = False) -> int:
        """Journal::purgeMemo (GatlasBenchmark.cpp:75-105)."""
        count = 0
        lines = []
        for key in sorted(self.run_state):
            value = self.run_state[key]
            if key not in self.times:
                lines.append(f"{key}\t{value}\n")
                count += 1
            elif not delete_times:
                lines.append(f"{key}\t{value}\n")
                for t in self.times[key]:
                    lines.append(f"{key}\t{t}\n")
        with open(self.path, "w") as f:
            f.writelines(lines)
        return count

    def memo_run_state(self, key: str) -> int:
        return self.run_state.get(key, MISSING)

    def memo_time(self, key: str, trial: int) -> int:
        t = self.times.get(key)
        if t is None or trial >= len(t):
            return -1
        return t[trial]

    def take(self, key: str, value: int) -> None:
        with open(self.path, "a") as f:
            f.write(f"{key}\t{value}\n")
