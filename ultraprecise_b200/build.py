"""Build libultraprecise.so in-tree for sm_100a.

    python -m ultraprecise_b200.build [-j N] [--clean]

Host C++ is compiled with g++, CUDA with nvcc
(-gencode arch=compute_100a,code=sm_100a), the CUDA runtime is linked
statically and NVRTC dynamically.  The device arithmetic header
(csrc/up_dev.cuh) is embedded into the library for the JIT.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
OUT_DIR = os.path.join(HERE, "_lib")
OUT = os.path.join(OUT_DIR, "libultraprecise.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA, "bin", "nvcc")
GENCODE = ["-gencode", "arch=compute_100a,code=sm_100a"]

CXX_SOURCES = ["up_host.cpp", "up_typing.cpp", "up_align.cpp", "up_codegen.cpp", "up_jit.cpp", "up_abi.cpp",
               "up_batch.cpp", "up_serve.cpp"]
CU_SOURCES = ["up_kernels.cu", "up_noalloc.cu", "up_text.cu", "up_filter.cu", "up_costmodel.cu"]
HEADERS = ["up_internal.h", "up_kernels.h", "up_dev.cuh", "up_batch.h", "up_kargs.h"]


def _newer(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.exists(d) and os.path.getmtime(d) > t for d in deps)


def _embed_header() -> str:
    """The device headers the JIT hands to NVRTC, as C string literals."""
    srcs = [("kUpDevCuh", os.path.join(CSRC, "up_dev.cuh")), ("kUpKargsH", os.path.join(CSRC, "up_kargs.h"))]
    dst = os.path.join(OBJ, "up_dev_embed.inc")
    if _newer(dst, [p for _, p in srcs]):
        with open(dst + ".tmp", "w") as f:
            for name, path in srcs:
                text = open(path).read()
                assert ')UPDEV"' not in text
                f.write(f'static const char {name}[] = R"UPDEV(' + text + ')UPDEV";\n')
        os.replace(dst + ".tmp", dst)
    return dst


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build step failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)


def build(jobs: int = 8, clean: bool = False, verbose: bool = False) -> str:
    if clean and os.path.isdir(OBJ):
        shutil.rmtree(OBJ)
    os.makedirs(OBJ, exist_ok=True)
    os.makedirs(OUT_DIR, exist_ok=True)
    embed = _embed_header()
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(INCLUDE, h) for h in os.listdir(INCLUDE)]
    cmds = []
    objs = []
    for s in CXX_SOURCES:
        src = os.path.join(CSRC, s)
        if not os.path.exists(src):
            continue
        o = os.path.join(OBJ, s + ".o")
        objs.append(o)
        if _newer(o, [src, embed] + hdrs):
            cmds.append(["g++", "-std=c++17", "-O2", "-fPIC", "-Wall", "-Wno-unused-function",
                         f"-I{CUDA}/include", f"-I{OBJ}", f"-I{CSRC}", "-c", src, "-o", o])
    for s in CU_SOURCES:
        src = os.path.join(CSRC, s)
        o = os.path.join(OBJ, s + ".o")
        objs.append(o)
        if _newer(o, [src] + hdrs):
            cmds.append([NVCC, *GENCODE, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC",
                         f"-I{CSRC}", "-c", src, "-o", o])
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        futs = [ex.submit(_run, c) for c in cmds]
        for f in futs:
            f.result()
    if cmds or not os.path.exists(OUT):
        tmp = OUT + ".tmp"
        _run(["g++", "-shared", "-o", tmp, *objs, f"-L{CUDA}/lib64", "-lcudart_static", "-lnvrtc",
              "-lz", "-ldl", "-lrt", "-lpthread", f"-Wl,-rpath,{CUDA}/lib64"])
        os.replace(tmp, OUT)
    if verbose:
        print(f"built {OUT} ({len(cmds)} compiled)")
    return OUT


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("-j", type=int, default=os.cpu_count() or 8)
    ap.add_argument("--clean", action="store_true")
    a = ap.parse_args()
    try:
        build(a.j, a.clean, verbose=True)
    except RuntimeError as e:
        print(e, file=sys.stderr)
        sys.exit(1)
