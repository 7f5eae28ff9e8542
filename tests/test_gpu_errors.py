"""Error handling of the C ABI: every bad input returns a status, never traps.

All faults are made on the host (bad arguments); nothing here faults a GPU.
"""
import numpy as np
import pytest

import abt_b200
from abt_b200._lib import PBT_EINVAL, PBT_ESTATE, PbtError
from tests.helpers import one_triangle, outbeams

pytestmark = pytest.mark.gpu
LAM = 0.532


def _inputs():
    rng = np.random.default_rng(0)
    th, ph = abt_b200.make_angles([0, 180], [10]), abt_b200.make_angles([0, 350], [10])
    geo = one_triangle()
    return th, ph, geo, outbeams(2, rng, 1)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_bad_face_index(ctx, precision):
    th, ph, geo, ob = _inputs()
    ob["fi"][1] = 7
    with pytest.raises(PbtError) as e:
        ctx.diff_main(ob, None, geo, th, ph, LAM, precision=precision)
    assert e.value.status == PBT_EINVAL and "fi=7" in str(e.value)


def test_bad_lambda_and_grid(ctx):
    th, ph, geo, ob = _inputs()
    for lam in (0.0, -1.0, float("nan")):
        with pytest.raises(PbtError):
            ctx.diff_main(ob, None, geo, th, ph, lam)
    with pytest.raises(PbtError) as e:
        ctx.diff_main(ob, None, geo, th[:2], ph, LAM)
    assert e.value.status == PBT_EINVAL
    # no theta above one degree: the reference's forward fix has no row to use
    with pytest.raises(PbtError) as e:
        ctx.diff_main(ob, None, geo, np.radians([0.0, 0.5, 1.0]), ph, LAM)
    assert "1 degree" in str(e.value)


def test_non_finite_inputs(ctx):
    th, ph, geo, ob = _inputs()
    g2 = dict(geo, verts=geo["verts"].copy())
    g2["verts"][0, 0] = np.nan
    with pytest.raises(PbtError):
        ctx.diff_main(ob, None, g2, th, ph, LAM)
    ob2 = ob.copy()
    ob2["ampl"][0, 3] = np.inf
    with pytest.raises(PbtError):
        ctx.diff_main(ob2, None, geo, th, ph, LAM)


def test_bad_topology(ctx):
    th, ph, geo, ob = _inputs()
    g2 = dict(geo, face_vi=np.array([1, 2, 9]))
    with pytest.raises(PbtError):
        ctx.diff_main(ob, None, g2, th, ph, LAM)
    g3 = dict(geo, face_off=np.array([0, 2]), face_vi=np.array([1, 2]))
    with pytest.raises(PbtError):
        ctx.diff_main(ob, None, g3, th, ph, LAM)


def test_divide_before_summation(ctx):
    ctx.totals_reset()
    with pytest.raises(PbtError) as e:
        ctx.divide_by_num_orientations(1, 3, 3)
    assert e.value.status == PBT_ESTATE


def test_context_survives_errors(ctx):
    """After every rejected call the context still computes."""
    th, ph, geo, ob = _inputs()
    afb, afe = ctx.diff_main(ob, None, geo, th, ph, LAM)
    assert np.isfinite(afb).all() and np.abs(afb).max() > 0
