"""GPU parity: the B200 step against the CPU checkers, through the C ABI.

* fp32 B200 vs the reference itself (oracle/_ref, its own headers built against the serial Kokkos
  shim) — bit-exact: candidate pairs, contacts, manifolds, colours, warm-start ledger, support
  levels and the state after every substep;
* fp32 B200 vs the oracle restatement at float — bit-exact (always available);
* fp64 B200 vs the oracle restatement at double — every product and the state within 1e-12
  relative (the FP64 acceptance bar; the implementation is expected to be bit-exact).
"""
import numpy as np
import pytest

import parity as P

pytestmark = pytest.mark.gpu


def _run_pair(api_a, api_b, name, mk, extra, steps, precision, rtol):
    sc = mk()
    a = P.build(api_a, sc, extra, precision)
    b = P.build(api_b, sc, extra, precision)
    for k in range(steps):
        a.step(sc.dt)
        b.step(sc.dt)
        bad = P.diff(P.snapshot(a), P.snapshot(b), rtol=rtol)
        assert not bad, f"{name}: substep {k}: {bad[:4]}"


@pytest.mark.parametrize("name,mk,extra,steps", P.MATRIX, ids=[m[0] for m in P.MATRIX])
def test_fp32_bitexact_vs_oracle(gpu_api, orc_api, name, mk, extra, steps):
    _run_pair(gpu_api, orc_api, name, mk, extra, steps, "fp32", 0.0)


@pytest.mark.parametrize("name,mk,extra,steps", P.MATRIX, ids=[m[0] for m in P.MATRIX])
def test_fp64_vs_oracle(gpu_api, orc_api, name, mk, extra, steps):
    _run_pair(gpu_api, orc_api, name, mk, extra, steps, "fp64", 1e-12)


@pytest.mark.parametrize("name,mk,extra,steps", P.MATRIX[:8], ids=[m[0] for m in P.MATRIX[:8]])
def test_fp32_bitexact_vs_reference(gpu_api, ref_api, name, mk, extra, steps):
    _run_pair(gpu_api, ref_api, name, mk, extra, steps, "fp32", 0.0)
