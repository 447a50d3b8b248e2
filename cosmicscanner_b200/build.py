"""Builds libcosmicscanner_b200.so in place with nvcc for sm_100a.

    python -m cosmicscanner_b200.build [--force]

Objects go to cosmicscanner_b200/_build/ (not committed); the shared library lands next
to this file so that it travels with the source tree.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libcosmicscanner_b200.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
CUDA_INCLUDE = "/usr/local/cuda/include"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _host_cxx() -> str:
    # the system g++ (the image's /opt/gcc toolchain lacks the OpenMP spec files)
    return "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"


GEN_SRC = os.path.join(HERE, "gen_mt64_jump.cpp")
GEN_INC = os.path.join(BUILD, "mt64_jump_table.inc")


def _jump_table() -> None:
    """The mt19937_64 jump table (X^(c J) mod p(X)) that omega.cu compiles in: computed at
    build time by gen_mt64_jump.cpp, which checks a jump against direct generation."""
    if os.path.exists(GEN_INC) and os.path.getmtime(GEN_INC) >= os.path.getmtime(GEN_SRC):
        return
    exe = os.path.join(BUILD, "gen_mt64_jump")
    res = subprocess.run([_host_cxx(), "-O2", "-std=c++17", GEN_SRC, "-o", exe],
                         capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"g++ failed on gen_mt64_jump.cpp:\n{res.stdout}\n{res.stderr}")
    tmp = GEN_INC + ".tmp"
    res = subprocess.run([exe, tmp], capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"gen_mt64_jump failed:\n{res.stdout}\n{res.stderr}")
    os.replace(tmp, GEN_INC)


def _sources():
    return sorted(f for f in os.listdir(CSRC) if f.endswith((".cu", ".cpp")))


def _headers_mtime() -> float:
    paths = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    paths += [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE)]
    return max(os.path.getmtime(p) for p in paths) if paths else 0.0


def _compile(src: str, force: bool, verbose: bool) -> str:
    obj = os.path.join(BUILD, src + ".o")
    path = os.path.join(CSRC, src)
    deps = [os.path.getmtime(path), _headers_mtime()]
    if src == "omega.cu":
        deps.append(os.path.getmtime(GEN_INC))
    if (not force and os.path.exists(obj) and os.path.getmtime(obj) >= max(deps)):
        return obj
    if src.endswith(".cpp"):
        # host-only translation units: the system g++ with OpenMP (small dense algebra)
        cmd = [_host_cxx(), "-O3", "-march=x86-64-v3", "-std=c++17", "-fPIC", "-fopenmp",
               "-Wall", "-Wno-unused-function", "-I", INCLUDE, "-I", CUDA_INCLUDE, "-c",
               path, "-o", obj]
    else:
        cmd = [_nvcc(), "-ccbin", _host_cxx(), *ARCH, "-lineinfo", "-O3", "-std=c++17",
               "-Xcompiler", "-fPIC,-O2,-Wall,-Wno-unused-function", "--expt-relaxed-constexpr",
               "-I", INCLUDE, "-I", BUILD, "-c", path, "-o", obj]
    if src.endswith(".cu") and verbose:
        cmd.insert(1, "-Xptxas=-v")
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src}:\n{res.stdout}\n{res.stderr}")
    if verbose and res.stderr:
        sys.stderr.write(res.stderr)
    return obj


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    _jump_table()
    srcs = _sources()
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        objs = list(ex.map(lambda s: _compile(s, force, verbose), srcs))
    newest = max(os.path.getmtime(o) for o in objs)
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < newest:
        cmd = [_nvcc(), "-ccbin", _host_cxx(), *ARCH, "-shared", "-o", LIB, *objs,
               "-lcublas", "-lcusolver", "-lcudart", "-lz", "-Xcompiler", "-fopenmp"]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"link failed:\n{res.stdout}\n{res.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
