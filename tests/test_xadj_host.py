"""The XPBD adjoint's hand-written reverses against their maps' forward-mode Jacobians, on the CPU.

tests/xadj_host_check.cu compiles the adjoint's local maps (peclet-dem_b200/csrc/pdem_xadj.cuh,
host-and-device code) for the host and compares, on random inputs drawn to visit every branch
(side flags, restitution cut-off, clamped and free impulses, friction cone, walls and pairs,
active and inactive position contacts), each hand-written reverse with the vector-Jacobian product
of its map through dual numbers. The GPU tests check the same reverses on whole rollouts; this
one covers branches those scenes may not reach, in a second."""
import os
import re
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "xadj_host_check.cu")
OUT = os.path.join(ROOT, "tests", "_build", "xadj_host_check")


def _nvcc():
    for c in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if c and os.path.exists(c):
            return c
    return None


def _build():
    nvcc = _nvcc()
    if nvcc is None:
        pytest.skip("nvcc not available")
    deps = [SRC, os.path.join(ROOT, "peclet-dem_b200", "csrc", "pdem_xadj.cuh"),
            os.path.join(ROOT, "peclet-dem_b200", "csrc", "pdem_math.cuh")]
    if os.path.exists(OUT) and all(os.path.getmtime(d) < os.path.getmtime(OUT) for d in deps):
        return OUT
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    cmd = [nvcc, "-O2", "-std=c++17", "-fmad=false", "-prec-div=true", "-prec-sqrt=true", "--expt-relaxed-constexpr",
           "-Wno-deprecated-gpu-targets", "-Xcompiler", "-ffp-contract=off",
           "-I", os.path.join(ROOT, "peclet-dem_b200", "csrc"), "-I", os.path.join(ROOT, "include"),
           "-x", "cu", SRC, "-o", OUT]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]
    return OUT


def test_hand_reverses_match_dual_jacobians():
    exe = _build()
    r = subprocess.run([exe, "20000"], capture_output=True, text=True, timeout=300)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    lines = dict(re.findall(r"^(\w+) cases .*max-rel ([0-9.e+-]+)$", r.stdout, re.M))
    assert set(lines) == {"pgs", "warm", "vn0", "pos"}, r.stdout
    assert all(float(v) < 1e-9 for v in lines.values()), lines
    # the random inputs reached many branch combinations of the PGS update
    assert int(re.search(r"branch-sets (\d+)", r.stdout).group(1)) >= 40
