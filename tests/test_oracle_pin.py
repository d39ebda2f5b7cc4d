"""The oracle restatement (float) is bit-identical to the reference's own code (its headers built
against the serial Kokkos shim) on every branch of the substep and on the Hertz engine."""
import numpy as np
import pytest

import parity as P
import scenes as S


@pytest.mark.parametrize("name,mk,extra,steps", P.MATRIX, ids=[m[0] for m in P.MATRIX])
def test_restatement_bitexact_vs_reference(ref_api, orc_api, name, mk, extra, steps):
    sc = mk()
    a = P.build(ref_api, sc, extra, "fp32")
    b = P.build(orc_api, sc, extra, "fp32")
    for k in range(steps):
        a.step(sc.dt)
        b.step(sc.dt)
        bad = P.diff(P.snapshot(a), P.snapshot(b))
        assert not bad, f"{name}: substep {k}: {bad[:4]}"


def test_hertz_restatement_bitexact_vs_reference(ref_api, orc_api):
    sc, ex = S.spheres_in_drum()
    sc.planes = []

    def extra(s):
        ex(s)
        s.set_hertz_material(0, 1e7, 0.3)
    a = P.build(ref_api, sc, extra, "fp32")
    b = P.build(orc_api, sc, extra, "fp32")
    for k in range(4):
        a.step_hertz(2e-6, 10, 0.3)
        b.step_hertz(2e-6, 10, 0.3)
        sa, sb = P.snapshot(a, products=False), P.snapshot(b, products=False)
        ka, xa = a.debug_hertz()
        kb, xb = b.debug_hertz()
        sa.update(hk=ka, hx=xa)
        sb.update(hk=kb, hx=xb)
        bad = P.diff(sa, sb)
        assert not bad, f"hertz call {k}: {bad[:4]}"


def test_domain_getters_match_reference(ref_api, orc_api):
    """get_domain_min / get_domain_max (src/sim.hpp:1105-1110), both set_domain overloads."""
    for setup in (lambda s: s.set_domain(0.02, 0.03, 0.04), lambda s: s.set_domain((-1e-3, 0, 2e-3), (5e-3, 6e-3, 7e-3))):
        got = []
        for api in (ref_api, orc_api):
            sim = P.build(api, S.dense_spheres(), setup, "fp32")
            got.append((sim.get_domain_min(), sim.get_domain_max()))
        assert got[0] == got[1]


def test_hertz_shape_pairs_restatement_bitexact_vs_reference(ref_api, orc_api):
    """Hollow cylinders (point shells) under the Hertz engine: the shape-pair forces
    (hertzShapePairForcesKokkos, src/solver_hertz.hpp:454) and shell-wall contacts, bit-exact."""
    import hertz_cases as HC
    sc, extra = HC.shape_pairs()
    a = P.build(ref_api, sc, extra, "fp32")
    b = P.build(orc_api, sc, extra, "fp32")
    for k in range(3):
        a.step_hertz(2e-6, 10, 0.3)
        b.step_hertz(2e-6, 10, 0.3)
        sa, sb = P.snapshot(a, products=False), P.snapshot(b, products=False)
        ka, xa = a.debug_hertz()
        kb, xb = b.debug_hertz()
        assert len(ka) > 0 and np.count_nonzero(xa) > 0  # touching shell pairs carry history
        sa.update(hk=ka, hx=xa)
        sb.update(hk=kb, hx=xb)
        bad = P.diff(sa, sb)
        assert not bad, f"hertz shape pairs call {k}: {bad[:4]}"
