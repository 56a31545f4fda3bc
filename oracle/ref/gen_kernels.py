"""Builds the reference's own generated kernels as a host library.

TEST INFRASTRUCTURE.  Recipe, run by oracle/ref/Makefile where the
reference's sources are present (cjang/GATLAS, read at REF_SRC):

1. emit: oracle/_ref/bin/emit_kernel (the reference's generators, built from
   its sources) prints the OpenCL C kernel of every point in POINTS;
2. translate: the OpenCL C is rewritten into C++ over clshim.hpp (address
   space qualifiers dropped, vector literals made constructor calls) and
   wrapped in an entry point with the refk.h signature that binds the
   kernel's arguments the way the reference's setArgs does
   (KernelMatmulBuffer.hpp:150-170, KernelMatmulImage.hpp:170-185,
   KernelMatvecBuffer.hpp:153-175, KernelMatvecImage.hpp:168-183,
   KernelSaxpyBuffer.hpp:123-140);
3. compile every kernel twice (mad fused, mad rounded separately) into
   oracle/_ref/librefk.so, and write oracle/_ref/kernels.json, the manifest
   the Python side (oracle/ref/__init__.py) loads.

Nothing emitted is committed: the sources under oracle/_ref/src are
regenerated from the reference on every build.

One change is made to the emitted buffer matmul (the only kernel with a
barrier): its K-step loop stores the next tiles of A and B into local memory
right after the work item's own reads of the previous tiles, with no barrier
between the last reads and the next stores (KernelMatmulBuffer.hpp:257-323).
On a device that runs the work group in lockstep no item stores before all
have read; a host that runs the items one after another must be told, so the
translation adds a barrier at the top of that loop.  The arithmetic is
untouched.
"""

from __future__ import annotations

import json
import os
import re
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(os.path.dirname(HERE), "_ref")

# (id, op, -T type, parameter vector in journal order)
#   matmul [packed, gemm, M, N, K, tA, tB, gh, gw, bh, bw, extra]   (KernelBaseMatmul.cpp:293-325)
#   matvec [packed, gemv, M, N, tA, g, bh, VL, extra]               (KernelBaseMatvec.cpp:259-288)
#   saxpy  [packed, M, N, gh, gw, bh, bw, VL, extra]                (KernelBaseSaxpy.cpp:233-258)
POINTS = [
    # parity cases: every layout, GEMM with packed instances, each vector width, images
    ("mm_f4_nn", "matmul", "float4", [1, 0, 256, 192, 320, 0, 0, 16, 16, 8, 4, 0]),
    ("mm_f4_tn", "matmul", "float4", [1, 0, 256, 192, 320, 1, 0, 16, 16, 8, 4, 5]),
    ("mm_f4_nt", "matmul", "float4", [1, 0, 256, 192, 320, 0, 1, 8, 8, 4, 4, 2]),
    ("mm_f4_tt_gemm_p2", "matmul", "float4", [2, 1, 128, 128, 128, 1, 1, 8, 8, 8, 4, 0]),
    ("mm_f2_gemm", "matmul", "float2", [1, 1, 128, 64, 96, 0, 0, 8, 8, 4, 2, 3]),
    ("mm_f1", "matmul", "float1", [1, 0, 64, 64, 64, 0, 0, 8, 8, 4, 1, 0]),
    ("mm_d2_gemm", "matmul", "double2", [1, 1, 128, 128, 128, 0, 1, 8, 8, 4, 2, 7]),
    ("mm_img_f_nn", "matmul", "floatimg", [1, 0, 256, 256, 256, 0, 0, 16, 16, 8, 4, 0]),
    ("mm_img_f_tn_gemm", "matmul", "floatimg", [1, 1, 128, 256, 192, 1, 0, 8, 8, 8, 4, 13]),
    ("mm_img_d", "matmul", "doubleimg", [1, 0, 128, 128, 128, 0, 0, 8, 8, 4, 2, 7]),
    ("mv_f4_n", "matvec", "float4", [1, 0, 1024, 768, 0, 64, 4, 4, 0]),
    ("mv_f4_t_gemv", "matvec", "float4", [1, 1, 1024, 768, 1, 64, 8, 4, 1]),
    ("mv_f4_n_p2", "matvec", "float4", [2, 0, 512, 256, 0, 32, 4, 4, 0]),
    ("mv_d2_t", "matvec", "double2", [1, 0, 512, 512, 1, 32, 2, 2, 0]),
    ("mv_img_f_n", "matvec", "floatimg", [1, 0, 1024, 768, 0, 64, 4, 4, 0]),
    ("mv_img_f_t_gemv", "matvec", "floatimg", [1, 1, 1024, 768, 1, 64, 4, 4, 0]),
    ("sx_f4_1d", "saxpy", "float4", [1, 250000, 4, 250, 0, 4, 0, 4, 0]),
    ("sx_f4_2d", "saxpy", "float4", [1, 512, 1024, 16, 16, 4, 4, 4, 0]),
    ("sx_d2_1d", "saxpy", "double2", [1, 65536, 2, 64, 0, 4, 0, 2, 0]),
    # the workloads' own sizes, for the timed CPU baseline
    ("bench_sgemm_1024", "matmul", "float4", [1, 0, 1024, 1024, 1024, 0, 0, 16, 16, 8, 4, 0]),
    ("bench_sgemm_8192", "matmul", "float4", [1, 0, 8192, 8192, 8192, 0, 0, 16, 16, 8, 4, 0]),
    ("bench_saxpy_2p28", "saxpy", "float4", [1, 1 << 26, 4, 256, 0, 4, 0, 4, 0]),
    ("bench_sgemv_n_16384", "matvec", "float4", [1, 0, 16384, 16384, 0, 64, 4, 4, 0]),
    ("bench_sgemv_t_16384", "matvec", "float4", [1, 0, 16384, 16384, 1, 64, 4, 4, 0]),
    ("bench_sgemv_img_n_16384", "matvec", "floatimg", [1, 0, 16384, 16384, 0, 64, 4, 4, 0]),
    ("bench_sgemv_img_t_16384", "matvec", "floatimg", [1, 0, 16384, 16384, 1, 64, 4, 4, 0]),
]

CXX = os.environ.get("CXX", "g++")
CXXFLAGS = ["-std=c++17", "-O3", "-mavx2", "-mfma", "-ffp-contract=off", "-fPIC", "-fopenmp", "-w"]


def scalar_of(type_: str) -> str:
    return "double" if type_.startswith("double") else "float"


def emit(point) -> tuple[str, dict]:
    pid, op, type_, params = point
    exe = os.path.join(OUT, "bin", "emit_kernel")
    r = subprocess.run([exe, op, type_] + [str(p) for p in params], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"{pid}: emit_kernel failed: {r.stderr.strip()}")
    src, meta_line = r.stdout.rsplit("//@", 1)
    meta = dict(kv.split("=", 1) for kv in meta_line.split())
    meta["global"] = [int(v) for v in meta["global"].split(",")]
    meta["local"] = [int(v) for v in meta["local"].split(",")]
    return src, meta


def parse_signature(src: str):
    m = re.search(r"void\s+(\w+)\s*\((.*?)\)\s*\{", src, re.S)
    if not m:
        raise RuntimeError("no kernel signature")
    name, body = m.group(1), m.group(2)
    args = []
    for raw in body.split(","):
        a = " ".join(raw.split())
        pname = re.findall(r"(\w+)$", a)[0]
        if "image2d_t" in a:
            kind = "image"
        elif "__global" in a:
            kind = "global"
        elif "__local" in a:
            kind = "local"
        else:
            kind = "value"
        ctype = a.replace("__global", "").replace("__local", "").replace("__read_only", "")
        ctype = ctype.replace("__write_only", "").strip()
        ctype = ctype[: -len(pname)].strip()
        args.append({"name": pname, "kind": kind, "ctype": ctype})
    return name, args


def translate(src: str) -> str:
    out = []
    for line in src.splitlines():
        if line.strip().startswith("#pragma OPENCL"):
            continue
        out.append(line)
    s = "\n".join(out)
    s = re.sub(r"__attribute__\(\(vec_type_hint\(\w+\)\)\)\s*", "", s)
    s = s.replace("__kernel ", "static ")
    for q in ("__global ", "__local ", "__read_only ", "__write_only ", "__constant "):
        s = s.replace(q, "")
    s = re.sub(r"\((float|double|int|uint)(\d?)\)\(", r"\1\2(", s)
    if "barrier(" in s:
        # a barrier at the top of the K-step loop (see the module docstring)
        s, n = re.subn(r"(for \(int idx = 0;[^\n]*\n(\s*)\{\n)", r"\1\2    barrier(CLK_LOCAL_MEM_FENCE);\n", s)
        if n != 1:
            raise RuntimeError("buffer matmul: K-step loop not found")
    return s


def layouts(op: str, params: list[int]) -> dict:
    """(width in scalars, height) of each image operand, as the reference
    creates them (KernelMatmulImage.hpp:100-108, KernelMatvecImage.hpp:100-107)."""
    if op == "matmul":
        P, gemm, M, N, K, tA, tB = params[:7]
        return {"A": (M, P * K) if tA else (K, P * M), "B": (K, P * N) if tB else (N, P * K),
                "C": None if gemm else (N, P * M)}
    if op == "matvec":
        P, gemv, M, N, tA = params[:5]
        return {"A": (M, P * N) if tA else (N, P * M), "B": (N, P), "C": None if gemv else (M, P)}
    return {"A": None, "B": None, "C": None}


def dims(op: str, params: list[int]) -> dict:
    if op == "matmul":
        return {"M": params[2], "N": params[3], "K": params[4]}
    if op == "matvec":
        return {"M": params[2], "N": params[3]}
    return {"M": params[1], "N": params[2]}


def wrapper(point, src: str, meta: dict) -> tuple[str, dict]:
    pid, op, type_, params = point
    name, args = parse_signature(src)
    scalar = scalar_of(type_)
    lay = layouts(op, params)
    d = dims(op, params)
    spt = 4 if scalar == "float" else 2  # scalars per 16-byte texel
    roles = ["C", "A", "B"]
    ptr_args = [a for a in args if a["kind"] in ("global", "image")]
    if len(ptr_args) != 3:
        raise RuntimeError(f"{pid}: expected 3 operand arguments, got {len(ptr_args)}")
    call = []
    image_setup = []
    role_of = {}
    for a, role in zip(ptr_args, roles):
        role_of[a["name"]] = role
    local_bytes = [0, 0]
    nlocal = 0
    for a in args:
        if a["kind"] in ("global", "image"):
            role = role_of[a["name"]]
            field = {"A": "a->A", "B": "a->B", "C": "a->C"}[role]
            if a["kind"] == "image":
                w, h = lay[role]
                image_setup.append(
                    f"    clshim::Image img{role}{{(unsigned char *){field}, {w // spt}, {h}}};")
                call.append(f"(clshim::Image *)&k->img{role}")
            else:
                call.append(f"({a['ctype']})k->{role}")
        elif a["kind"] == "local":
            call.append(f"({a['ctype']})local{nlocal}")
            if op != "matmul":
                raise RuntimeError(f"{pid}: unexpected local argument")
            g, bh, vl = params[7], params[9], params[10]
            elems = (g + 1) * g * vl * (bh if nlocal == 0 else vl)  # KernelMatmulBuffer.hpp:150-151
            local_bytes[nlocal] = elems * (8 if scalar == "double" else 4)
            nlocal += 1
        else:
            n = a["name"]
            if n in d:
                call.append(f"(int){d[n]}")
            elif n in ("alpha", "beta"):
                call.append(f"({scalar})k->{n}")
            else:
                raise RuntimeError(f"{pid}: unknown argument {n}")
    ns = f"refk_{pid}"
    g0, g1 = (meta["global"] + [1])[:2]
    l0, l1 = (meta["local"] + [1])[:2]
    code = [
        f"namespace {ns} {{",
        "using namespace clshim;",
        translate(src),
        "struct Bound {",
        "    void *A, *B, *C;",
        "    double alpha, beta;",
        "    clshim::Image imgA, imgB, imgC;",
        "};",
        "static void body(void *arg, void *local0, void *local1) {",
        "    const Bound *k = (const Bound *)arg;",
        "    (void)local0; (void)local1;",
        f"    {name}({', '.join(call)});",
        "}",
        f"}}  // namespace {ns}",
        f'extern "C" int REFK_CAT({ns}, REFK_SUFFIX)(const refk_args *a) {{',
        "\n".join(image_setup),
        f"    {ns}::Bound k;",
        "    k.A = (void *)a->A; k.B = (void *)a->B; k.C = a->C; k.alpha = a->alpha; k.beta = a->beta;",
    ]
    for role in ("A", "B", "C"):
        if any(f"img{role}{{" in s for s in image_setup):
            code.append(f"    k.img{role} = img{role};")
    code += [
        "    refk_launch L;",
        f"    L.global[0] = {g0}; L.global[1] = {g1}; L.local[0] = {l0}; L.local[1] = {l1};",
        "    for (int d = 0; d < 2; ++d) { L.group_begin[d] = a->group_begin[d]; L.group_end[d] = a->group_end[d]; }",
        f"    L.local_bytes[0] = {local_bytes[0]}; L.local_bytes[1] = {local_bytes[1]};",
        f"    L.uses_barrier = {1 if 'barrier(' in src else 0};",
        "    L.threads = a->threads;",
        f"    return refk_run_groups(&L, {ns}::body, &k);",
        "}",
    ]
    info = {"id": pid, "op": op, "type": type_, "params": params, "kernel": name,
            "global": [g0, g1], "local": [l0, l1], "scalar": scalar, "uses_barrier": "barrier(" in src,
            "images": {r: lay[r] for r in ("A", "B", "C") if lay[r] is not None and
                       any(a["kind"] == "image" and role_of[a["name"]] == r for a in args)}}
    return "\n".join(code), info


def main() -> int:
    os.makedirs(os.path.join(OUT, "src"), exist_ok=True)
    os.makedirs(os.path.join(OUT, "obj"), exist_ok=True)
    manifest = []
    tus = []
    for point in POINTS:
        src, meta = emit(point)
        with open(os.path.join(OUT, "src", point[0] + ".cl"), "w") as f:
            f.write(src)
        code, info = wrapper(point, src, meta)
        manifest.append(info)
        tu = os.path.join(OUT, "src", point[0] + ".cpp")
        with open(tu, "w") as f:
            f.write('#include "clshim.hpp"\n#include "refk.h"\n'
                    "#define REFK_CAT2(a, b) a##b\n#define REFK_CAT(a, b) REFK_CAT2(a, b)\n")
            f.write(code + "\n")
        tus.append(tu)
    objs = []
    procs = []
    for tu in tus:
        for fused, suffix in ((1, "_fma"), (0, "_sep")):
            obj = os.path.join(OUT, "obj", os.path.basename(tu)[:-4] + suffix + ".o")
            cmd = [CXX] + CXXFLAGS + [f"-DREFK_FUSED={fused}", f"-DREFK_SUFFIX={suffix}", "-I", HERE, "-c", tu,
                                      "-o", obj]
            procs.append((cmd, subprocess.Popen(cmd)))
            objs.append(obj)
            if len(procs) >= (os.cpu_count() or 4):
                cmd0, p = procs.pop(0)
                if p.wait() != 0:
                    raise RuntimeError("compile failed: " + " ".join(cmd0))
    for cmd, p in procs:
        if p.wait() != 0:
            raise RuntimeError("compile failed: " + " ".join(cmd))
    rt = os.path.join(OUT, "obj", "clshim_runtime_fma.o")
    subprocess.run([CXX] + CXXFLAGS + ["-DREFK_FUSED=1", "-I", HERE, "-c",
                    os.path.join(HERE, "clshim_runtime.cpp"), "-o", rt], check=True)
    lib = os.path.join(OUT, "librefk.so")
    subprocess.run([CXX, "-shared", "-fopenmp", "-o", lib, rt] + objs, check=True)
    with open(os.path.join(OUT, "kernels.json"), "w") as f:
        json.dump(manifest, f, indent=1)
    print(f"built {len(manifest)} reference kernels into {lib}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
