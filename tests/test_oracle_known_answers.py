"""Known answers that pin the CPU oracle (its parity with the Fortran reference
itself is unpinned: no Fortran compiler and no reference golden vectors).

Closed forms used: simpne's exactness on quadratics, the identities of a
non-depolarising Mueller matrix (sum M_ij^2 = 4 M11^2 and
M11^2 - M12^2 - M13^2 - M14^2 = |det S|^2), the forward (q -> 0) limit of
the aperture integral |A|/lambda with the Karczewski-Wolf obliquity, linearity
in the amplitude matrix, and Parseval's theorem for the external diffraction
of a large aperture (scattering cross section ~ geometric area).
"""
import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import one_triangle

LAM = 0.532


def _ob(ampl, prop, vk7=(0, 1, 0), fi=1, fov=0.5):
    ob = np.zeros(1, dtype=O.OUTBEAM_DTYPE)
    ob["ampl"][0] = ampl
    ob["prop_out"][0] = prop
    ob["vk7"][0] = vk7
    ob["fi"][0] = fi
    ob["fov"][0] = fov
    return ob


@pytest.mark.parametrize("n", [3, 4, 7, 10, 31])
def test_simpne_exact_on_quadratics(n):
    rng = np.random.default_rng(n)
    x = np.sort(rng.uniform(-1, 2, size=n))
    y = 3 * x * x - 2 * x + 0.5
    a, b = x[0], x[-1]
    exact = (b ** 3 - a ** 3) - (b * b - a * a) + 0.5 * (b - a)
    assert abs(O.simpne(x, y) - exact) <= 1e-12 * max(1, abs(exact))


def test_mueller_of_one_amplitude_is_non_depolarising():
    rng = np.random.default_rng(1)
    a = (rng.normal(size=(5, 7, 2, 2)) + 1j * rng.normal(size=(5, 7, 2, 2)))
    mu = O.ampl_to_mueller(a)
    m11 = mu[..., 0]
    assert (m11 > 0).all()
    # a Mueller matrix of a single amplitude matrix satisfies sum_ij M_ij^2 = 4 M11^2
    np.testing.assert_allclose((mu ** 2).sum(axis=-1), 4 * m11 ** 2, rtol=1e-12)
    # and M11^2 - M12^2 - M13^2 - M14^2 = |det S|^2
    det = a[..., 0, 0] * a[..., 1, 1] - a[..., 0, 1] * a[..., 1, 0]
    np.testing.assert_allclose(m11 ** 2 - (mu[..., 1:4] ** 2).sum(-1), np.abs(det) ** 2,
                               rtol=1e-10, atol=1e-10 * (m11 ** 2).max())
    # M11 = (|S11|^2 + |S12|^2 + |S21|^2 + |S22|^2) / 2 and |M_ij| <= M11
    np.testing.assert_allclose(m11, 0.5 * (np.abs(a) ** 2).sum(axis=(2, 3)), rtol=1e-14)
    assert (np.abs(mu) <= m11[..., None] * (1 + 1e-12)).all()


def test_mueller_matches_independent_bohren_huffman():
    """The 16 forms of src/outputs_mod.f90:473-549 against an independent
    transcription of Bohren & Huffman eq. 3.16 with S1=S22, S2=S11, S3=S12, S4=S21."""
    rng = np.random.default_rng(2)
    a = rng.normal(size=(3, 4, 2, 2)) + 1j * rng.normal(size=(3, 4, 2, 2))
    mu = O.ampl_to_mueller(a)
    S2, S3, S4, S1 = a[..., 0, 0], a[..., 0, 1], a[..., 1, 0], a[..., 1, 1]
    c = np.conj
    ref = np.stack([
        0.5 * (abs(S1) ** 2 + abs(S2) ** 2 + abs(S3) ** 2 + abs(S4) ** 2),
        0.5 * (abs(S2) ** 2 - abs(S1) ** 2 + abs(S4) ** 2 - abs(S3) ** 2),
        (S2 * c(S3) + S1 * c(S4)).real,
        (S2 * c(S3) - S1 * c(S4)).imag,
        0.5 * (abs(S2) ** 2 - abs(S1) ** 2 - abs(S4) ** 2 + abs(S3) ** 2),
        0.5 * (abs(S2) ** 2 + abs(S1) ** 2 - abs(S4) ** 2 - abs(S3) ** 2),
        (S2 * c(S3) - S1 * c(S4)).real,
        (S2 * c(S3) + S1 * c(S4)).imag,
        (S2 * c(S4) + S1 * c(S3)).real,
        (S2 * c(S4) - S1 * c(S3)).real,
        (S1 * c(S2) + S3 * c(S4)).real,
        (S2 * c(S1) + S4 * c(S3)).imag,
        (S4 * c(S2) + S1 * c(S3)).imag,
        (S4 * c(S2) - S1 * c(S3)).imag,
        (S1 * c(S2) - S3 * c(S4)).imag,
        (S1 * c(S2) - S3 * c(S4)).real,
    ], axis=-1)
    np.testing.assert_allclose(mu, ref, rtol=1e-12, atol=1e-12)


@pytest.mark.parametrize("scale", [0.5, 1.0, 3.0])
def test_forward_limit_is_area_over_lambda(scale):
    """At the exact forward direction of an aperture normal to the beam the
    contour integral tends to area/lambda and the KW matrix to |Kz| = 1, so
    |S|_F = sqrt(2) A / lambda for a unit amplitude matrix.

    The facet sits 36 um off axis, so the theta = 0 bin is seen from its
    centre 3.6e-5 rad off normal (R = 1e6 um): q L ~ 1e-4.  Much closer to
    q = 0 the reference's contour formula (src/diff_mod.f90:414-420) cancels
    catastrophically in FP64 (relative error ~ 1e-16 / (q L)^2), which the
    oracle reproduces."""
    geo = one_triangle(offset=(20.0, 30.0, 0.0), scale=scale)
    th = O.make_angles([0, 180], [2])
    ph = O.make_angles([0, 358], [2])
    a = O.diffraction(th, ph, LAM, geo, _ob([1, 0, 0, 0, 0, 0, 1, 0], (0, 0, -1)))
    area = 0.5 * scale * scale
    f = np.sqrt((np.abs(a[:, 0]) ** 2).sum(axis=(1, 2)))
    np.testing.assert_allclose(f, np.sqrt(2) * area / LAM, rtol=1e-5)


def test_linear_in_amplitude():
    geo = one_triangle()
    th = O.make_angles([0, 180], [5])
    ph = O.make_angles([0, 350], [10])
    rng = np.random.default_rng(3)
    amp = rng.normal(size=8)
    prop = np.array([0.3, -0.2, -0.93])
    prop /= np.linalg.norm(prop)
    a1 = O.diffraction(th, ph, LAM, geo, _ob(amp, prop))
    a2 = O.diffraction(th, ph, LAM, geo, _ob(2 * amp, prop))
    assert np.array_equal(2 * a1, a2)


def test_diff_main_is_the_ordered_sum_of_diffraction():
    rng = np.random.default_rng(4)
    verts = rng.normal(size=(9, 3))
    geo = dict(verts=verts, face_off=np.array([0, 3, 6, 9]), face_vi=np.arange(1, 10))
    th = O.make_angles([0, 180], [10])
    ph = O.make_angles([0, 350], [10])
    obs = np.concatenate([_ob(rng.normal(size=8), p / np.linalg.norm(p), fi=k + 1)
                          for k, p in enumerate(rng.normal(size=(3, 3)))])
    afb, afe = O.diff_main(th, ph, LAM, geo, obs, obs[:1])
    acc = np.zeros_like(afb)
    for k in range(3):
        acc = acc + O.diffraction(th, ph, LAM, geo, obs[k:k + 1])
    assert np.array_equal(acc, afb)
    # external diffraction forces fov = pi/2
    e = O.diffraction(th, ph, LAM, geo, obs[:1], fov_override=O.PI_REF / 2)
    assert np.array_equal(afe, e + 0.0)


def test_parseval_external_diffraction_cross_section():
    """Fraunhofer diffraction of a large aperture scatters its geometric area."""
    # a generic triangle: an edge exactly perpendicular to a bin's q makes the
    # reference's contour term Inf * 0 = NaN (src/diff_mod.f90:414-418)
    s = 12.0
    verts = np.array([[0.0, 0.0, 0.0], [s, 0.13 * s, 0.0], [0.21 * s, s, 0.0]]) + [-3.7, -4.1, 0.0]
    geo = dict(verts=verts, face_off=np.array([0, 3]), face_vi=np.array([1, 2, 3]))
    area = 0.5 * abs(s * s - 0.13 * s * 0.21 * s)
    th = O.make_angles([0, 5, 20, 180], [0.05, 0.5, 5])
    ph = O.make_angles([0, 358], [2])
    ob = _ob([1, 0, 0, 0, 0, 0, 1, 0], (0, 0, -1), fov=np.pi / 2)
    afb, afe = O.diff_main(th, ph, LAM, geo, ob[:0], ob)
    assert np.isfinite(afe).all()
    mu, mu1, p = O.finalise(afb, afe, th, ph, LAM, O.params_vec(0.0, area))
    scatt_ext = p[13]
    assert abs(scatt_ext / area - 1) < 0.02
