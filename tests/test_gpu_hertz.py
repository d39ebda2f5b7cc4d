"""GPU parity of the explicit Hertz-Mindlin engine (`step_hertz`, src/sim.hpp:628-750) through the
C ABI: tangential history keys and vectors and the state after every call, against the oracle
restatement (bit-exact at float, within 1e-12 relative at double)."""
import pytest

import parity as P
import scenes as S

pytestmark = pytest.mark.gpu


def _drum_spheres():
    sc, ex = S.spheres_in_drum()
    sc.planes = []

    def extra(s):
        ex(s)
        s.set_hertz_material(0, 1e7, 0.3)
    return sc, extra


def _dense_drum():
    sc, ex = S.spheres_in_drum(seed=21, n=240, omega=3.0)
    sc.planes = []

    def extra(s):
        ex(s)
        s.set_hertz_material(0, 5e6, 0.25)
    return sc, extra


def _shape_pairs():
    import hertz_cases as HC
    return HC.shape_pairs()


def _shape_pairs_512():
    import hertz_cases as HC
    from peclet.dem import workloads as W
    return HC.shape_pairs(seed=32, n=64, L=10e-3, shell=W.hollow_cylinder_shell())


# (name, scene, calls, substeps per call, skin fraction); the shape cases drive the shape-pair
# forces (src/solver_hertz.hpp:454) with the analytic shell and the 512-point stratified shell
CASES = [("drum_spheres", _drum_spheres, 4, 10, 0.3), ("dense_drum", _dense_drum, 3, 20, 0.2),
         ("shape_pairs", _shape_pairs, 3, 10, 0.3), ("shape_pairs_512", _shape_pairs_512, 2, 10, 0.3)]


@pytest.mark.parametrize("precision,rtol", [("fp32", 0.0), ("fp64", 1e-12)])
@pytest.mark.parametrize("name,mk,calls,substeps,skin", CASES, ids=[c[0] for c in CASES])
def test_hertz_vs_oracle(gpu_api, orc_api, name, mk, calls, substeps, skin, precision, rtol):
    sc, extra = mk()
    a = P.build(gpu_api, sc, extra, precision)
    b = P.build(orc_api, sc, extra, precision)
    for k in range(calls):
        a.step_hertz(2e-6, substeps, skin)
        b.step_hertz(2e-6, substeps, skin)
        sa, sb = P.snapshot(a, products=False), P.snapshot(b, products=False)
        ka, xa = a.debug_hertz()
        kb, xb = b.debug_hertz()
        sa.update(hk=ka, hx=xa)
        sb.update(hk=kb, hx=xb)
        bad = P.diff(sa, sb, rtol=rtol)
        assert not bad, f"{name} {precision}: hertz call {k}: {bad[:4]}"


def test_hertz_rejects_periodic(gpu_api):
    """The reference refuses the Hertz engine on periodic domains (src/sim.hpp:629-634); the B200
    step raises the same error type."""
    sc = S.polydisperse_periodic()
    sim = P.build(gpu_api, sc, lambda s: s.set_hertz_material(0, 1e7, 0.3), "fp64")
    with pytest.raises(RuntimeError):
        sim.step_hertz(2e-6, 2, 0.3)
