"""The whole orientation step on real traced lists: host tracer -> far-field
kernels -> finalise, the reference's per-orientation sequence
(src/pbt_seq_mod.f90:165-223).

Checks the consistency the reference's documentation asks of a result: the
external-diffraction and beam scattering efficiencies close to 1 for a
non-absorbing particle with large facets on a fine enough grid (README,
"far-field bins"; facets a few wavelengths across lose some energy in the
aperture diffraction itself, about 9 % per facet for 1.3 um^2 triangles at
0.532 um); the FP64 drop-in on traced lists against the C oracle; the FP32
batch within its error bars of the FP64 drop-in on a rough column's traced
lists; a physically sized asymmetry parameter for a hexagonal column."""
import numpy as np
import pytest

from abt_b200 import Context, make_angles, workloads as W
from abt_b200 import tracer as T
from oracle import oracle as O
from tests.helpers import mueller_rel_err

pytestmark = pytest.mark.gpu

LAM, RBI = 0.532, 1.31


@pytest.fixture(scope="module")
def traced():
    geo = W.hex_prism(10.0, 20.0, n_side=6, n_len=12, roughness=0.1, seed=3)
    P = T.Particle(geo, geo["apertures"])
    rng = np.random.default_rng(11)
    Vs, beams, exts, pins = [], [], [], []
    for u in rng.uniform(size=(8, 3)):
        V, beam, ext, pin, _ = T.trace(P, T.multi_euler(*u), LAM, RBI)
        Vs.append(V)
        beams.append(beam)
        exts.append(ext)
        pins.append(pin)
    return P.geometry, Vs, beams, exts, np.array(pins)


@pytest.fixture(scope="module")
def ctx():
    return Context(0)


def test_one_orientation_conserves_energy(ctx):
    """Smooth column, 144 triangles: 302 beam and 72 external-diffraction
    outbeams in the orientation below (the C oracle gives beam and external
    efficiencies 0.974 and 0.997, asymmetry 0.908 on this grid)."""
    geo = W.hex_prism(10.0, 20.0, n_side=2, n_len=4, roughness=0.0)
    P = T.Particle(geo, geo["apertures"])
    V, beam, ext, pin, en = T.trace(P, T.multi_euler(0.2, 0.4, 0.6), LAM, RBI)
    theta = make_angles([0, 180], [0.25])
    phi = make_angles([0, 359], [1])
    g = dict(P.geometry, verts=V)
    afb, afe = ctx.diff_main(beam, ext, g, theta, phi, LAM, precision="fp64")
    mu, mu1, p = ctx.finalise(afb, afe, theta, phi, LAM, pin)
    assert abs(p["scatt_eff_ext_diff"] - 1.0) < 0.02
    assert abs(p["scatt_eff_beam"] - 1.0) < 0.04
    assert 0.75 < p["asymmetry"] < 0.95
    assert p["geo_cross_sec"] == pin["geo_cross_sec"]
    # the drop-in on traced lists against the C oracle, on a coarser grid
    th2, ph2 = make_angles([0, 180], [2]), make_angles([0, 356], [4])
    g64 = ctx.diff_main(beam, ext, g, th2, ph2, LAM, precision="fp64")
    ref = O.diff_main(th2, ph2, LAM, g, beam, ext, nthreads=8)
    for a, b in zip(g64, ref):
        assert np.abs(a - b).max() <= 1e-10 * np.abs(b).max()


def test_fp32_batch_on_traced_lists(ctx, traced):
    geo, Vs, beams, exts, pins = traced
    theta = make_angles([0, 180], [0.5])
    phi = make_angles([0, 358], [2])
    r64 = ctx.diff_batch(beams, exts, Vs, geo, theta, phi, LAM, pins, precision="fp64")
    r32 = ctx.diff_batch(beams, exts, Vs, geo, theta, phi, LAM, pins, precision="fp32")
    # every element against its bin's M11, bins above 1e-6 of the peak M11
    assert mueller_rel_err(r32[0], r64[0], 1e-6) < 1e-4
    p64, p32 = r64[2], r32[2]
    for name in ("scatt", "ext", "asymmetry", "scatt_eff", "ext_eff"):
        assert abs(p32[name] - p64[name]) <= 1e-5 * abs(p64[name]), name
    assert 0.6 < p64["asymmetry"] < 0.95
    assert 0.9 < p64["scatt_eff"] / 2.0 < 1.1  # extinction paradox: Q_sca ~ 2


def test_overlapped_trace_and_average(ctx):
    """Tracing chunk c+1 on the host while the GPU averages chunk c gives the
    single-call average of all orientations (up to the rounding of combining
    the chunk averages)."""
    geo = W.hex_prism(10.0, 20.0, n_side=6, n_len=12, roughness=0.1, seed=3)
    P = T.Particle(geo, geo["apertures"])
    eul = W.uniform_euler(np.random.default_rng(7), 40)
    theta = make_angles([0, 180], [1])
    phi = make_angles([0, 356], [4])
    Vs, beams, exts, pins, _ = T.trace_batch(P, eul, LAM, RBI)
    ref = ctx.diff_batch(beams, exts, Vs, P.geometry, theta, phi, LAM, pins, precision="fp64")
    got = T.traced_orientation_average(ctx, P, eul, theta, phi, LAM, RBI, chunk=16,
                                       precision="fp64")
    assert np.allclose(got[0], ref[0], rtol=1e-12, atol=1e-12 * np.abs(ref[0]).max())
    assert np.allclose(got[1], ref[1], rtol=1e-12, atol=1e-12 * np.abs(ref[1]).max())
    for name in ("scatt", "ext", "asymmetry", "geo_cross_sec", "beam_energy_out"):
        assert got[2][name] == pytest.approx(float(ref[2][name]), rel=1e-12)
    assert got[3].tobytes() == np.atleast_1d(ref[3]).tobytes()


@pytest.mark.parametrize("plan", [(-1, 1, 2048), (0, 1, 2048), (1, 2, 1024)],
                         ids=["packed", "one-record", "packed-2bins"])
def test_large_column_traced_forward_rings(ctx, plan):
    """The large column (r 50 um, L 100 um, 22,500 triangles, n = 1.31 + 0.01i)
    traced in one orientation (about 34,000 outbeams), on a grid that keeps the
    first dark rings of the forward diffraction peak (theta 0-10 deg at 0.125 deg).
    The triangles of each face are translated copies, so per-face FP32 errors
    add up coherently, and at the dark rings the faces' contributions cancel.
    Near the forward direction the normal of the scattering plane is the cross
    product of nearly parallel unit vectors: formed from FP32 unit vectors it
    loses about six bits and left a 3e-4 Mueller error at theta = 0.25 deg.
    The FP32 form must stay within its bars of the FP64 drop-in here."""
    g = W.hex_prism(50.0, 100.0, n_side=25, n_len=50, roughness=0.0, seed=5)
    P = T.Particle(g, g["apertures"])
    e = W.uniform_euler(np.random.default_rng(5), 8)[0]
    V, beam, ext, pin, _ = T.trace(P, e, LAM, RBI, ibi=0.01)
    assert len(beam) > 20000 and len(ext) > 10000
    gv = dict(P.geometry, verts=V)
    theta, phi = make_angles([0, 10], [0.125]), make_angles([0, 356], [4])
    a64 = ctx.diff_main(beam, ext, gv, theta, phi, LAM, precision="fp64")
    ctx.set_plan(*plan)
    try:
        a32 = ctx.diff_main(beam, ext, gv, theta, phi, LAM, precision="fp32")
    finally:
        ctx.set_plan()
    m64 = ctx.finalise(a64[0], a64[1], theta, phi, LAM, pin)[0]
    m32 = ctx.finalise(a32[0], a32[1], theta, phi, LAM, pin)[0]
    assert mueller_rel_err(m32, m64, 1e-6) < 1e-4


def test_config1_analogue_traced(ctx):
    """The reference's first configuration, with the host tracer in place of
    the Fortran one: a hexagonal column r 5 um, L 10 um triangulated to about
    0.5 um^2 (900 triangles, its 8 parent faces as apertures), -rot euler
    30 40 10, lambda 0.532 um, n 1.31, 8 recursions, 181 theta x 180 phi
    (1,719 beam and 450 external-diffraction outbeams).  The FP64 drop-in
    matches the C oracle within 1e-10; the FP32 form is within its bars."""
    geo = W.hex_prism(5.0, 10.0, n_side=5, n_len=10, roughness=0.0)
    P = T.Particle(geo, geo["apertures"])
    V, beam, ext, pin, en = T.trace(P, T.euler_from_degrees(30, 40, 10), LAM, RBI)
    assert 0.97 < en["beam_energy_out"] / en["geo_cross_sec"] < 1.03
    g = dict(P.geometry, verts=V)
    theta, phi = make_angles([0, 180], [1]), make_angles([0, 358], [2])
    a64 = ctx.diff_main(beam, ext, g, theta, phi, LAM, precision="fp64")
    ref = O.diff_main(theta, phi, LAM, g, beam, ext, nthreads=8)
    for a, b in zip(a64, ref):
        assert np.abs(a - b).max() <= 1e-10 * np.abs(b).max()
    a32 = ctx.diff_main(beam, ext, g, theta, phi, LAM, precision="fp32")
    m64 = ctx.finalise(a64[0], a64[1], theta, phi, LAM, pin)
    m32 = ctx.finalise(a32[0], a32[1], theta, phi, LAM, pin)
    assert mueller_rel_err(m32[0], m64[0], 1e-6) < 1e-4
    for name in ("scatt", "ext", "asymmetry", "scatt_eff"):
        assert abs(m32[2][name] - m64[2][name]) <= 1e-5 * abs(m64[2][name]), name
