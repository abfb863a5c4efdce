"""Build the engine's shared library, libspams_b200.so, in-tree.

    python spams-devel_b200/build.py [--jobs N] [--verbose]

The CUDA sources listed in SOURCES are compiled for sm_100a only
(``-gencode arch=compute_100a,code=sm_100a``) and linked, with the C ABI of
include/spams_b200.h, into spams-devel_b200/lib/libspams_b200.so.  Object files
go to spams-devel_b200/_build/.  Rebuilds only what changed.

The list is explicit: a stray .cu file in csrc/ is an error, not a silent
part of the library.  Before linking, the weak (template-instantiation) host
symbols of every object are compared: two objects that define the same one
would let the linker keep whichever comes first, so that is an error too.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import hashlib
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIBDIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIBDIR, "libspams_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


SOURCES = [
    "csc.cu", "dl.cu", "engine.cu", "gemm.cu", "lars.cu", "lars_chol.cu", "lars_cta.cu", "mask.cu",
    "noalloc.cu", "omp.cu", "omp_cta.cu", "refine.cu", "serve.cu", "tc_gemm.cu",
]


def sources() -> list[str]:
    present = sorted(f for f in os.listdir(CSRC) if f.endswith(".cu"))
    extra = sorted(set(present) - set(SOURCES))
    missing = sorted(set(SOURCES) - set(present))
    if extra or missing:
        raise RuntimeError(f"csrc/ does not match the source list: unlisted {extra}, missing {missing}")
    return [os.path.join(CSRC, f) for f in SOURCES]


def _weak_host_symbols(obj: str) -> set[str]:
    """Defined weak symbols of one object's host code (nm types W/V)."""
    r = subprocess.run(["nm", "--defined-only", obj], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nm failed on {obj}: {r.stderr}")
    out = set()
    for line in r.stdout.splitlines():
        parts = line.split()
        if len(parts) == 3 and parts[1] in ("W", "V"):
            out.add(parts[2])
    return out


def check_duplicate_weak(objs: list[str]) -> None:
    """Refuse a link in which two objects define the same project symbol weakly.

    Project code lives in namespace ``sc`` (mangled ``_ZN2sc``); a weak ``sc::``
    symbol in two objects means two explicit instantiations of the same
    template, and the linker would keep one of them without a word.
    """
    seen: dict[str, str] = {}
    dups = []
    for o in objs:
        for sym in _weak_host_symbols(o):
            if not sym.startswith("_ZN2sc"):
                continue
            if sym in seen and seen[sym] != o:
                dups.append((sym, os.path.basename(seen[sym]), os.path.basename(o)))
            seen.setdefault(sym, o)
    if dups:
        lines = "\n".join(f"  {s} in {a} and {b}" for s, a, b in dups[:20])
        raise RuntimeError(f"weak project symbols defined by two objects:\n{lines}")


def headers() -> list[str]:
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    hs.append(os.path.join(ROOT, "include", "spams_b200.h"))
    return hs


def _digest(paths: list[str], extra: str = "") -> str:
    h = hashlib.sha256(extra.encode())
    for p in sorted(paths):
        with open(p, "rb") as f:
            h.update(os.path.basename(p).encode())
            h.update(f.read())
    return h.hexdigest()


def _stale(target: str, deps: list[str]) -> bool:
    """Content-hash check (file copies that reset mtimes do not force rebuilds)."""
    stamp = target + ".sha256"
    if not os.path.exists(target) or not os.path.exists(stamp):
        return True
    with open(stamp) as f:
        return f.read().strip() != _digest(deps, " ".join(ARCH + NVCC_FLAGS))


def _stamp(target: str, deps: list[str]) -> None:
    with open(target + ".sha256", "w") as f:
        f.write(_digest(deps, " ".join(ARCH + NVCC_FLAGS)))


def _compile(src: str, verbose: bool) -> str:
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    if _stale(obj, [src] + headers()):
        cmd = [nvcc(), *ARCH, *NVCC_FLAGS, "-I", os.path.join(ROOT, "include"), "-c", src, "-o", obj]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src}:\n{r.stdout}\n{r.stderr}")
        if verbose and r.stderr:
            print(r.stderr, flush=True)
        _stamp(obj, [src] + headers())
    return obj


def build(jobs: int = 0, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    srcs = sources()
    jobs = jobs or min(len(srcs), os.cpu_count() or 4)
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), srcs))
    if _stale(LIB, objs):
        check_duplicate_weak(objs)
        cmd = [nvcc(), *ARCH, "-shared", "-o", LIB, *objs, "-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
        _stamp(LIB, objs)
    return LIB


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--jobs", type=int, default=0)
    ap.add_argument("--verbose", action="store_true")
    a = ap.parse_args()
    print(build(a.jobs, a.verbose))
    return 0


if __name__ == "__main__":
    sys.exit(main())
