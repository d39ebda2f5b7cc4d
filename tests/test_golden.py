"""Golden vectors recorded from the reference's own substep (tests/golden/make_golden.py): the
oracle restatement (CPU) and the B200 step in float (GPU) must reproduce them bit for bit — state
after every substep and the intermediate products (pairs, contacts, manifolds, colours, ledger)
after the first and last substep."""
import os

import numpy as np
import pytest

import parity as P

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
import importlib.util  # noqa: E402

_spec = importlib.util.spec_from_file_location("make_golden", os.path.join(HERE, "make_golden.py"))
_mg = importlib.util.module_from_spec(_spec)
_spec.loader.exec_module(_mg)
CASES = _mg.CASES


def _check(api, name):
    mk, extra, steps = CASES[name]
    g = np.load(os.path.join(HERE, f"{name}.npz"))
    assert int(g["steps"]) == steps
    sc = mk()
    sim = P.build(api, sc, extra, "fp32")
    for k in range(steps):
        sim.step(sc.dt)
        st = P.snapshot(sim, products=k in (0, steps - 1))
        for key in P.STATE_KEYS:
            np.testing.assert_array_equal(st[key].astype(np.float32), g[f"s{k}_{key}"], err_msg=f"{name} s{k} {key}")
        if k in (0, steps - 1):
            for key in P.PRODUCT_KEYS:
                want = g[f"p{k}_{key}"]
                got = st[key]
                got = got.astype(np.float32) if want.dtype == np.float32 else got.astype(want.dtype)
                np.testing.assert_array_equal(got, want, err_msg=f"{name} p{k} {key}")


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_reproduces_golden(orc_api, name):
    _check(orc_api, name)


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(CASES))
def test_b200_fp32_reproduces_golden(gpu_api, name):
    _check(gpu_api, name)
