"""The whole orientation step on real traced lists: host tracer -> far-field
kernels -> finalise, the reference's per-orientation sequence
(src/pbt_seq_mod.f90:165-223).

Checks the consistency the reference's documentation asks of a result: the
external-diffraction and beam scattering efficiencies close to 1 for a
non-absorbing particle on a fine enough grid (README, "far-field bins"), the
FP32 batch within its error bars of the FP64 drop-in on these lists, and a
physically sized asymmetry parameter for a hexagonal column."""
import numpy as np
import pytest

from abt_b200 import Context, make_angles, workloads as W
from abt_b200 import tracer as T
from abt_b200.diff import PI_REF

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


def test_one_orientation_efficiencies(ctx, traced):
    geo, Vs, beams, exts, pins = traced
    theta = make_angles([0, 180], [0.25])
    phi = make_angles([0, 358], [2])
    g = dict(geo, verts=Vs[0])
    afb, afe = ctx.diff_main(beams[0], exts[0], g, theta, phi, LAM, precision="fp64")
    mu, mu1, p = ctx.finalise(afb, afe, theta, phi, LAM, pins[0])
    assert abs(p["scatt_eff_ext_diff"] - 1.0) < 0.03
    assert abs(p["scatt_eff_beam"] - 1.0) < 0.05
    assert 0.6 < p["asymmetry"] < 0.95
    assert p["geo_cross_sec"] == pins[0]["geo_cross_sec"]


def test_fp32_batch_on_traced_lists(ctx, traced):
    geo, Vs, beams, exts, pins = traced
    theta = make_angles([0, 180], [0.5])
    phi = make_angles([0, 358], [2])
    r64 = ctx.diff_batch(beams, exts, Vs, geo, theta, phi, LAM, pins, precision="fp64")
    r32 = ctx.diff_batch(beams, exts, Vs, geo, theta, phi, LAM, pins, precision="fp32")
    m64, m32 = r64[0], r32[0]
    peak = np.abs(m64).max()
    mask = np.abs(m64) > 1e-6 * peak
    err = np.abs(m32 - m64)[mask] / np.abs(m64)[mask]
    assert err.max() < 1e-4
    p64, p32 = r64[2], r32[2]
    for name in ("scatt", "ext", "asymmetry", "scatt_eff", "ext_eff"):
        assert abs(p32[name] - p64[name]) <= 1e-5 * abs(p64[name]), name
    assert 0.6 < p64["asymmetry"] < 0.95
    assert 0.9 < p64["scatt_eff"] / 2.0 < 1.1  # extinction paradox: Q_sca ~ 2
