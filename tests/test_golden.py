"""Frozen fixtures (tests/golden/, made by tests/golden/make_golden.py)."""
import os

import numpy as np
import pytest

import abt_b200
from oracle import oracle as O
from tests.helpers import rel_err

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CASES = ["hex_orientation", "synthetic_cube"]


def load(name):
    z = dict(np.load(os.path.join(HERE, name + ".npz")))
    z["beam"] = z["beam"].view(O.OUTBEAM_DTYPE)
    z["ext"] = z["ext"].view(O.OUTBEAM_DTYPE)
    z["geo"] = dict(verts=z["verts"], face_off=z["face_off"], face_vi=z["face_vi"])
    return z


@pytest.mark.parametrize("name", CASES)
def test_oracle_reproduces_fixture(name):
    z = load(name)
    afb, afe = O.diff_main(z["theta"], z["phi"], float(z["lam"]), z["geo"], z["beam"], z["ext"])
    assert np.array_equal(afb, z["ampl_far_beam"])
    assert np.array_equal(afe, z["ampl_far_ext_diff"])
    mu, mu1, p = O.finalise(afb, afe, z["theta"], z["phi"], float(z["lam"]), z["params_in"])
    assert np.array_equal(mu, z["mueller"])
    assert np.array_equal(mu1, z["mueller_1d"])
    # asymmetry_ext_diff is 0/0 = NaN when there is no external diffraction, as in the reference
    assert np.array_equal(p, z["params"], equal_nan=True)


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES)
def test_gpu_fp64_matches_fixture(ctx, name):
    z = load(name)
    lam = float(z["lam"])
    afb, afe = ctx.diff_main(z["beam"], z["ext"], z["geo"], z["theta"], z["phi"], lam)
    assert rel_err(afb, z["ampl_far_beam"]) <= 1e-10
    assert rel_err(afe, z["ampl_far_ext_diff"]) <= 1e-10
    pin = np.frombuffer(np.ascontiguousarray(z["params_in"], dtype=np.float64).tobytes(),
                        dtype=abt_b200.PARAMS_DTYPE)[0]
    mu, mu1, p = ctx.finalise(afb, afe, z["theta"], z["phi"], lam, pin)
    assert rel_err(mu, z["mueller"]) <= 1e-10
    assert rel_err(mu1, z["mueller_1d"]) <= 1e-10
    got = np.array([p[n] for n in abt_b200.PARAM_NAMES])
    np.testing.assert_allclose(got, z["params"], rtol=1e-10)
