"""Build the B200 substep library (libpdem.so) in-tree with nvcc for sm_100a.

    python peclet-dem_b200/build.py

Compiles csrc/*.cu to objects under _build/ (in parallel) and links
peclet/dem/libpdem.so, which the `peclet.dem` package loads. Floating-point flags: no FMA
contraction on device (-fmad=false) or host (-ffp-contract=off), IEEE division and square root,
so the float build reproduces the reference's arithmetic and the double build the FP64 oracle.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
OUT = os.path.join(HERE, "peclet", "dem", "libpdem.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-fmad=false", "-prec-div=true", "-prec-sqrt=true",
                "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC,-ffp-contract=off,-O2",
                "-I", CSRC, "-I", INCLUDE]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, jobs: int | None = None) -> str:
    nvcc = _nvcc()
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".hpp", ".h"))]
    headers.append(os.path.join(INCLUDE, "pdem.h"))
    sources = sorted(f for f in os.listdir(CSRC) if f.endswith(".cu"))
    objs = []

    def compile_one(src: str) -> str:
        path = os.path.join(CSRC, src)
        obj = os.path.join(BUILD, src.replace(".cu", ".o"))
        if _stale(obj, [path] + headers + [__file__]):
            cmd = [nvcc, *FLAGS, "-c", path, "-o", obj]
            if verbose:
                print(" ".join(cmd), flush=True)
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode != 0:
                raise RuntimeError(f"nvcc failed on {src}:\n{r.stdout}\n{r.stderr}")
        return obj

    with ThreadPoolExecutor(max_workers=jobs or min(8, os.cpu_count() or 4)) as ex:
        objs = list(ex.map(compile_one, sources))
    if _stale(OUT, objs):
        cmd = [nvcc, *ARCH, "-shared", "-o", OUT, *objs]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    _check_undefined(OUT)
    return OUT


def _check_undefined(lib: str) -> None:
    """A template of the library used in one file but defined in another links into an undefined
    symbol that only the loader reports: fail the build on any undefined symbol of our namespace."""
    nm = shutil.which("nm")
    if not nm:
        return
    r = subprocess.run([nm, "-D", "--undefined-only", "-C", lib], capture_output=True, text=True)
    bad = [ln.strip() for ln in r.stdout.splitlines() if "pdem::" in ln]
    if bad:
        raise RuntimeError("undefined symbols in " + lib + ":\n" + "\n".join(bad[:10]))


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
