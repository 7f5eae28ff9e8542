"""FP64 drop-in (reference-exact path) against the CPU oracle, through the C ABI.

Bar: <= 1e-10 relative (normwise over the grid) for diff_main / diffraction
amplitudes, and the finalise / summation / divide epilogue to <= 1e-12.
"""
import numpy as np
import pytest

import abt_b200
from abt_b200 import workloads as W
from oracle import oracle as O
from tests.helpers import mixed_polygon_geometry, one_triangle, outbeams, rel_err

pytestmark = pytest.mark.gpu

TOL_AMPL = 1e-10
LAM = 0.532


def grids():
    return [
        (abt_b200.make_angles([0, 180], [4]), abt_b200.make_angles([0, 356], [4])),
        # multi-segment theta with fine steps near the forward direction
        (abt_b200.make_angles([0, 2, 10, 180], [0.5, 2, 10]), abt_b200.make_angles([0, 350], [10])),
    ]


@pytest.mark.parametrize("gi", [0, 1])
@pytest.mark.parametrize("fast", [False, True])
def test_diff_main_random_triangles(ctx, gi, fast):
    rng = np.random.default_rng(10 + gi + 2 * fast)
    th, ph = grids()[gi]
    geo, beam, _ = W.synthetic_beam_list(n_beams=3, facets_per_beam=5, seed=5 + gi, cube=20.0)
    ext = outbeams(4, rng, len(geo["face_off"]) - 1, prop=(0, 0, -1))
    afb, afe = ctx.diff_main(beam, ext, geo, th, ph, LAM, is_fast_diff=fast, precision="fp64")
    rfb, rfe = O.diff_main(th, ph, LAM, geo, beam, ext, is_fast_diff=fast)
    assert rel_err(afb, rfb) <= TOL_AMPL
    assert rel_err(afe, rfe) <= TOL_AMPL
    if fast:
        # bins outside every field of view are exactly zero in both
        assert np.array_equal(afb == 0, rfb == 0)


def test_diff_main_polygons(ctx):
    rng = np.random.default_rng(3)
    th, ph = grids()[0]
    geo = mixed_polygon_geometry(rng)
    nf = len(geo["face_off"]) - 1
    beam = outbeams(12, rng, nf)
    beam["fi"] = np.arange(12) % nf + 1
    ext = outbeams(nf, rng, nf, prop=(0, 0, -1))
    ext["fi"] = np.arange(1, nf + 1)
    afb, afe = ctx.diff_main(beam, ext, geo, th, ph, LAM)
    rfb, rfe = O.diff_main(th, ph, LAM, geo, beam, ext)
    assert rel_err(afb, rfb) <= TOL_AMPL
    assert rel_err(afe, rfe) <= TOL_AMPL


def test_diff_main_hex_prism_orientation(ctx):
    """A stand-in orientation of a triangulated hexagonal column."""
    rng = np.random.default_rng(7)
    th, ph = grids()[0]
    geo = W.hex_prism(2.0, 4.0, n_side=1, n_len=2)
    R = W.euler_rotation(*np.radians([30, 40, 10]))
    V, beam, ext, _ = W.standin_orientation(geo, R, rng, n_internal=(0, 1))
    g2 = dict(geo, verts=V)
    afb, afe = ctx.diff_main(beam, ext, g2, th, ph, LAM)
    rfb, rfe = O.diff_main(th, ph, LAM, g2, beam, ext)
    assert rel_err(afb, rfb) <= TOL_AMPL
    assert rel_err(afe, rfe) <= TOL_AMPL


def test_diffraction_single_outbeam(ctx):
    rng = np.random.default_rng(11)
    th, ph = grids()[1]
    geo = one_triangle()
    ob = outbeams(1, rng, 1)
    for fast in (False, True):
        a = ctx.diffraction(ob, geo, th, ph, LAM, is_fast_diff=fast)
        r = O.diffraction(th, ph, LAM, geo, ob, is_fast_diff=fast)
        assert rel_err(a, r) <= TOL_AMPL


def test_empty_lists_give_zero(ctx):
    th, ph = grids()[0]
    geo = one_triangle()
    afb, afe = ctx.diff_main(None, None, geo, th, ph, LAM)
    assert not afb.any() and not afe.any()


@pytest.mark.parametrize("scaling", [False, True])
def test_finalise_matches_oracle(ctx, scaling):
    rng = np.random.default_rng(21)
    th, ph = grids()[0]
    geo, beam, _ = W.synthetic_beam_list(n_beams=2, facets_per_beam=4, seed=9, cube=10.0)
    ext = outbeams(3, rng, len(geo["face_off"]) - 1, prop=(0, 0, -1))
    rfb, rfe = O.diff_main(th, ph, LAM, geo, beam, ext)
    pin = abt_b200.params(abs=0.3, geo_cross_sec=2.5, beam_energy_out=0.7, ext_energy_out=1.9)
    mu, mu1, p = ctx.finalise(rfb, rfe, th, ph, LAM, pin, scaling=scaling)
    pvec = O.params_vec(0.3, 2.5, 0.7, 1.9)
    rmu, rmu1, rp = O.finalise(rfb, rfe, th, ph, LAM, pvec, scaling=scaling)
    assert rel_err(mu, rmu) <= 1e-12
    assert rel_err(mu1, rmu1) <= 1e-12
    got = np.array([p[n] for n in abt_b200.PARAM_NAMES])
    np.testing.assert_allclose(got, rp, rtol=1e-12, atol=0)


def test_summation_and_divide(ctx):
    rng = np.random.default_rng(31)
    th, ph = grids()[0]
    ctx.totals_reset()
    tot = O.Totals(len(ph), len(th))
    for k in range(3):
        geo, beam, _ = W.synthetic_beam_list(n_beams=1, facets_per_beam=3, seed=40 + k, cube=8.0)
        ext = outbeams(2, rng, len(geo["face_off"]) - 1, prop=(0, 0, -1))
        rfb, rfe = O.diff_main(th, ph, LAM, geo, beam, ext)
        pin = abt_b200.params(abs=0.1 * k, geo_cross_sec=1.0 + k)
        ctx.finalise(rfb, rfe, th, ph, LAM, pin, accumulate=True)
        rmu, rmu1, rp = O.finalise(rfb, rfe, th, ph, LAM, O.params_vec(0.1 * k, 1.0 + k))
        tot.add(rmu, rmu1, rp)
    mu, mu1, p = ctx.divide_by_num_orientations(3, len(th), len(ph))
    rmu, rmu1, rp = tot.averaged()
    assert rel_err(mu, rmu) <= 1e-12
    assert rel_err(mu1, rmu1) <= 1e-12
    got = np.array([p[n] for n in abt_b200.PARAM_NAMES])
    sel = [i for i, n in enumerate(abt_b200.PARAM_NAMES) if n not in ("beam_energy_out", "ext_energy_out")]
    np.testing.assert_allclose(got[sel], rp[sel], rtol=1e-12)
    ctx.totals_reset()


def test_batch_fp64_matches_oracle_loop(ctx):
    rng = np.random.default_rng(5)
    th, ph = grids()[0]
    geo = W.hex_prism(1.5, 3.0, n_side=1, n_len=1)
    beams, exts, Vs, pins = [], [], [], []
    tot = O.Totals(len(ph), len(th))
    for k in range(3):
        R = W.euler_rotation(*rng.uniform(0, 2 * np.pi, size=3))
        V, beam, ext, gcs = W.standin_orientation(geo, R, rng, n_internal=(0, 1))
        beams.append(beam)
        exts.append(ext)
        Vs.append(V)
        pins.append(abt_b200.params(abs=0.05, geo_cross_sec=gcs))
        g2 = dict(geo, verts=V)
        rfb, rfe = O.diff_main(th, ph, LAM, g2, beam, ext)
        rmu, rmu1, rp = O.finalise(rfb, rfe, th, ph, LAM, O.params_vec(0.05, gcs))
        tot.add(rmu, rmu1, rp)
    mu, mu1, pav, pper = ctx.diff_batch(beams, exts, Vs, geo, th, ph, LAM, np.array(pins),
                                        precision="fp64")
    rmu, rmu1, rp = tot.averaged()
    assert rel_err(mu, rmu) <= TOL_AMPL
    assert rel_err(mu1, rmu1) <= TOL_AMPL
    got = np.array([pav[n] for n in abt_b200.PARAM_NAMES])
    sel = [i for i, n in enumerate(abt_b200.PARAM_NAMES) if n not in ("beam_energy_out", "ext_energy_out")]
    np.testing.assert_allclose(got[sel], rp[sel], rtol=TOL_AMPL)


def test_diffraction_concurrent_callers(ctx):
    """The -memory path calls diffraction from OpenMP threads
    (src/beam_loop_mod.f90:1935-1967): concurrent callers on one context get
    the same grids as serial calls."""
    from concurrent.futures import ThreadPoolExecutor
    rng = np.random.default_rng(12)
    th, ph = grids()[0]
    geo = mixed_polygon_geometry(rng)
    obs = outbeams(16, rng, len(geo["face_off"]) - 1)
    serial = [ctx.diffraction(obs[i:i + 1], geo, th, ph, LAM) for i in range(len(obs))]
    with ThreadPoolExecutor(max_workers=8) as ex:
        conc = list(ex.map(lambda i: ctx.diffraction(obs[i:i + 1], geo, th, ph, LAM),
                           range(len(obs))))
    for a, b in zip(serial, conc):
        assert np.array_equal(a, b)


def test_diff_main_config_sized_hex_column(ctx):
    """The plain-method configuration at its own size: a hexagonal column
    (r 5 um, L 10 um, 0.26 um^2 triangles: 1,764 facets), Euler (30, 40, 10),
    stand-in outbeams (~3,500), 181 theta x 180 phi; the FP64 drop-in against
    the oracle (OpenMP facet loop, as the reference runs it)."""
    import os
    rng = np.random.default_rng(1)
    th = abt_b200.make_angles([0, 180], [1])
    ph = abt_b200.make_angles([0, 358], [2])
    geo = W.hex_prism(5.0, 10.0, n_side=7, n_len=14)
    R = W.euler_rotation(*np.radians([30, 40, 10]))
    V, beam, ext, _ = W.standin_orientation(geo, R, rng, n_internal=(0, 3))
    g2 = dict(geo, verts=V)
    afb, afe = ctx.diff_main(beam, ext, g2, th, ph, LAM)
    rfb, rfe = O.diff_main(th, ph, LAM, g2, beam, ext, nthreads=os.cpu_count() or 1)
    assert rel_err(afb, rfb) <= TOL_AMPL
    assert rel_err(afe, rfe) <= TOL_AMPL
