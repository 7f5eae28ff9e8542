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


def test_bounded_wait_times_out_and_context_survives(ctx):
    """Failure detection without a GPU fault: a device wait that nothing
    completes ends by itself within its limit and is reported as
    PBT_ETIMEOUT; the next compute call on the same context succeeds."""
    import time
    t0 = time.perf_counter()
    with pytest.raises(abt_b200.PbtError) as e:
        ctx.selftest_bounded_wait(200)
    assert e.value.status == abt_b200._lib.PBT_ETIMEOUT
    assert time.perf_counter() - t0 < 5.0
    rng = np.random.default_rng(3)
    geo = one_triangle()
    th, ph = abt_b200.make_angles([0, 180], [10]), abt_b200.make_angles([0, 350], [10])
    afb, _ = ctx.diff_main(outbeams(2, rng, 1), None, geo, th, ph, 0.532, precision="fp32")
    assert np.isfinite(afb).all() and np.abs(afb).max() > 0


def test_fp32_face_vertex_limit(ctx):
    """The FP32 path fans faces of up to 16 vertices; a 20-gon is refused with
    PBT_EINVAL there, while the FP64 drop-in takes it."""
    n = 20
    a = np.arange(n) * 2 * np.pi / n
    verts = np.stack([np.cos(a), np.sin(a), np.zeros(n)], 1) + np.array([3.0, -2.0, 1.0])
    geo = abt_b200.make_geometry(verts, [list(range(1, n + 1))])
    rng = np.random.default_rng(4)
    ob = outbeams(1, rng, 1)
    th, ph = abt_b200.make_angles([0, 180], [10]), abt_b200.make_angles([0, 350], [10])
    a64, _ = ctx.diff_main(ob, None, geo, th, ph, 0.532, precision="fp64")
    assert np.isfinite(a64).all()
    with pytest.raises(PbtError) as e:
        ctx.diff_main(ob, None, geo, th, ph, 0.532, precision="fp32")
    assert e.value.status == PBT_EINVAL


def test_ragged_batch_with_empty_orientations(ctx):
    """Orientations with no outbeams at all, or no external diffraction, in a
    batch: FP32 matches the FP64 drop-in."""
    from abt_b200 import workloads as W
    from tests.helpers import mueller_rel_err
    geo, Vs, beams, exts, pin = W.rough_column_orientations(4, seed=41, n_side=2, n_len=3,
                                                            m_range=(0, 2))
    beams[1] = beams[1][:0]
    exts[2] = exts[2][:0]
    th, ph = abt_b200.make_angles([0, 180], [4]), abt_b200.make_angles([0, 356], [4])
    r32 = ctx.diff_batch(beams, exts, Vs, geo, th, ph, 0.532, pin, precision="fp32")
    r64 = ctx.diff_batch(beams, exts, Vs, geo, th, ph, 0.532, pin, precision="fp64")
    assert mueller_rel_err(r32[0], r64[0]) <= 1e-4


def test_first_bad_record_of_a_long_list_is_reported(ctx):
    """Long lists (above 65,536 records) are checked by all host threads; the
    record reported is still the first bad one, and nothing runs."""
    th, ph, geo, ob = _inputs()
    rng = np.random.default_rng(5)
    many = outbeams(70000, rng, 1)
    many["fi"][50000] = 9
    many["ampl"][60000, 3] = np.nan
    with pytest.raises(PbtError) as e:
        ctx.diff_main(many, None, geo, th, ph, LAM, precision="fp32")
    assert e.value.status == PBT_EINVAL and "outbeam 50001" in str(e.value) and "fi=9" in str(e.value)
    many["fi"][50000] = 1
    with pytest.raises(PbtError) as e:
        ctx.diff_main(many, None, geo, th, ph, LAM, precision="fp32")
    assert "outbeam 60001" in str(e.value) and "not finite" in str(e.value)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_no_outbeams_at_all(ctx, precision):
    """A call with no outbeams in either list is legal and gives zero grids, and
    a batch whose orientations are all empty gives a zero Mueller average."""
    th, ph, geo, ob = _inputs()
    afb, afe = ctx.diff_main(ob[:0], ob[:0], geo, th, ph, LAM, precision=precision)
    assert afb.shape == (len(ph), len(th), 2, 2) and not afb.any() and not afe.any()
    pin = np.zeros(3, dtype=abt_b200.PARAMS_DTYPE)
    pin["geo_cross_sec"] = 1.0
    mu, mu1, _, _ = ctx.diff_batch([ob[:0]] * 3, [ob[:0]] * 3, [geo["verts"]] * 3, geo, th, ph,
                                   LAM, pin, precision=precision)
    assert not mu.any() and not mu1.any()


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_injected_allocation_failure_reports_enomem(precision):
    """A device allocation that fails (injected on the host with
    pbt_test_fail_next_alloc) makes the call return PBT_ENOMEM with a message;
    the context stays usable and the next call gives the result of a context
    that never failed.  A fresh context has no buffers yet, so its first call
    allocates."""
    from abt_b200 import _lib
    from abt_b200._lib import PBT_ENOMEM
    th, ph, geo, ob = _inputs()
    ext = ob[:1].copy()
    ext["prop_out"] = (0.0, 0.0, -1.0)
    with abt_b200.Context(0) as ref_ctx:
        ref = ref_ctx.diff_main(ob, ext, geo, th, ph, LAM, precision=precision)
    with abt_b200.Context(0) as c:
        assert _lib.lib().pbt_test_fail_next_alloc(1) == 0
        try:
            with pytest.raises(PbtError) as e:
                c.diff_main(ob, ext, geo, th, ph, LAM, precision=precision)
        finally:
            _lib.lib().pbt_test_fail_next_alloc(0)
        assert e.value.status == PBT_ENOMEM and "injected" in str(e.value)
        got = c.diff_main(ob, ext, geo, th, ph, LAM, precision=precision)
        assert np.array_equal(got[0], ref[0]) and np.array_equal(got[1], ref[1])
        mu = c.finalise(got[0], got[1], th, ph, LAM, abt_b200.params(geo_cross_sec=1.0))[0]
        assert np.isfinite(mu).all()


def test_device_from_local_rank(monkeypatch):
    """PBT_DEVICE_LOCAL_RANK takes the launcher's node-local rank modulo the
    visible devices (the reference's MPI ranks spread over a node's GPUs); an
    unset or malformed rank gives device 0, and an explicit device is kept."""
    import torch
    from abt_b200._lib import PBT_DEVICE_LOCAL_RANK
    ndev = torch.cuda.device_count()
    names = ("LOCAL_RANK", "OMPI_COMM_WORLD_LOCAL_RANK", "MV2_COMM_WORLD_LOCAL_RANK",
             "MPI_LOCALRANKID", "SLURM_LOCALID", "PMI_LOCAL_RANK")
    for n in names:
        monkeypatch.delenv(n, raising=False)
    for env, want in (({}, 0), ({"OMPI_COMM_WORLD_LOCAL_RANK": "5"}, 5 % ndev),
                      ({"LOCAL_RANK": "x7", "SLURM_LOCALID": "3"}, 3 % ndev),
                      ({"PMI_LOCAL_RANK": "-2"}, 0)):
        for n in names:
            monkeypatch.delenv(n, raising=False)
        for k, v in env.items():
            monkeypatch.setenv(k, v)
        with abt_b200.Context(PBT_DEVICE_LOCAL_RANK) as c:
            assert c.device == want, env
    with abt_b200.Context(0) as c:
        assert c.device == 0
    with pytest.raises(PbtError) as e:
        abt_b200.Context(ndev)
    assert e.value.status == PBT_EINVAL
