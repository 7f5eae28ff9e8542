"""FP32 form (FP64 phase) against the FP64 references.

Bar (the FP32 precision target): <= 1e-4 relative on every Mueller element
at bins whose M11 exceeds 1e-6 of the peak (normalised by the bin's M11, see
helpers.mueller_rel_err); cross sections and asymmetry parameters within
1e-5 relative.
"""
import numpy as np
import pytest

import abt_b200
from abt_b200 import workloads as W
from oracle import oracle as O
from tests.helpers import mixed_polygon_geometry, mueller_rel_err, one_triangle, outbeams, rel_err

pytestmark = pytest.mark.gpu

LAM = 0.532
TOL_MU = 1e-4
TOL_PARAM = 1e-5


def _mueller(afb, afe):
    k = 2 * abt_b200.PI_REF / LAM
    return O.ampl_to_mueller((afb + afe) * k)


def test_fp32_single_facet_vs_oracle(ctx):
    rng = np.random.default_rng(1)
    th, ph = abt_b200.make_angles([0, 180], [1]), abt_b200.make_angles([0, 358], [2])
    geo = one_triangle(scale=2.0)
    beam = outbeams(1, rng, 1)
    ext = outbeams(1, rng, 1, prop=(0, 0, -1))
    afb, afe = ctx.diff_main(beam, ext, geo, th, ph, LAM, precision="fp32")
    rfb, rfe = O.diff_main(th, ph, LAM, geo, beam, ext)
    assert rel_err(afb, rfb) <= 1e-5
    assert rel_err(afe, rfe) <= 1e-5
    assert mueller_rel_err(_mueller(afb, afe), _mueller(rfb, rfe)) <= TOL_MU


def test_fp32_large_particle_phase_vs_oracle(ctx):
    """Facets spread over a 100 um cube: far-field phases ~1e3 rad (size parameter ~590)."""
    th, ph = abt_b200.make_angles([0, 180], [2]), abt_b200.make_angles([0, 356], [4])
    geo, beam, ext = W.synthetic_beam_list(n_beams=8, facets_per_beam=8, seed=3)
    afb, afe = ctx.diff_main(beam, ext, geo, th, ph, LAM, precision="fp32")
    rfb, rfe = O.diff_main(th, ph, LAM, geo, beam, ext)
    assert rel_err(afb, rfb) <= 1e-4
    assert mueller_rel_err(_mueller(afb, afe), _mueller(rfb, rfe)) <= TOL_MU


def test_fp32_polygons_and_fast_diff(ctx):
    rng = np.random.default_rng(4)
    th, ph = abt_b200.make_angles([0, 180], [2]), abt_b200.make_angles([0, 356], [4])
    geo = mixed_polygon_geometry(rng)
    nf = len(geo["face_off"]) - 1
    beam = outbeams(10, rng, nf)
    ext = outbeams(nf, rng, nf, prop=(0, 0, -1))
    ext["fi"] = np.arange(1, nf + 1)
    for fast in (False, True):
        afb, afe = ctx.diff_main(beam, ext, geo, th, ph, LAM, is_fast_diff=fast, precision="fp32")
        rfb, rfe = O.diff_main(th, ph, LAM, geo, beam, ext, is_fast_diff=fast)
        assert mueller_rel_err(_mueller(afb, afe), _mueller(rfb, rfe)) <= TOL_MU


@pytest.mark.parametrize("scaling", [False, True])
def test_batch_fp32_vs_fp64(ctx, scaling):
    rng = np.random.default_rng(8)
    th, ph = abt_b200.make_angles([0, 180], [2]), abt_b200.make_angles([0, 356], [4])
    geo = W.hex_prism(3.0, 6.0, n_side=2, n_len=3, roughness=0.05, seed=2)
    beams, exts, Vs, pins = [], [], [], []
    for k in range(5):
        R = W.euler_rotation(*rng.uniform(0, 2 * np.pi, size=3))
        V, beam, ext, gcs = W.standin_orientation(geo, R, rng, n_internal=(0, 2))
        beams.append(beam)
        exts.append(ext)
        Vs.append(V)
        pins.append(abt_b200.params(abs=0.02, geo_cross_sec=gcs, beam_energy_out=0.8 * gcs,
                                    ext_energy_out=gcs))
    pins = np.array(pins)
    r = ctx.diff_batch(beams, exts, Vs, geo, th, ph, LAM, pins, scaling=scaling, precision="fp64")
    f = ctx.diff_batch(beams, exts, Vs, geo, th, ph, LAM, pins, scaling=scaling, precision="fp32")
    assert mueller_rel_err(f[0], r[0]) <= TOL_MU
    assert rel_err(f[1], r[1]) <= TOL_MU
    for n in ("scatt", "ext", "asymmetry", "scatt_beam", "scatt_ext_diff", "asymmetry_beam",
              "asymmetry_ext_diff", "albedo"):
        assert abs(f[2][n] - r[2][n]) <= TOL_PARAM * abs(r[2][n]), n
        np.testing.assert_allclose(f[3][n], r[3][n], rtol=TOL_PARAM, err_msg=n)
    np.testing.assert_allclose(f[3]["back_scatt"], r[3]["back_scatt"], rtol=1e-4)


@pytest.mark.parametrize("fast", [False, True])
def test_batch_fp32_uneven_grid(ctx, fast):
    """The batched FP32 average against the FP64 path on a theta grid of three
    spacings (fine near the forward direction, src/input_mod.f90:114-196) and a
    phi range short of 360 degrees (the reference's phi integral then covers
    [0, phi_max] only), with and without the -fast_diff field-of-view cull."""
    rng = np.random.default_rng(21)
    th = abt_b200.make_angles([0, 2, 20, 180], [0.25, 1, 4])
    ph = abt_b200.make_angles([0, 270], [3])
    geo = W.hex_prism(3.0, 6.0, n_side=2, n_len=3, roughness=0.05, seed=4)
    beams, exts, Vs, pins = [], [], [], []
    for k in range(4):
        R = W.euler_rotation(*rng.uniform(0, 2 * np.pi, size=3))
        V, beam, ext, gcs = W.standin_orientation(geo, R, rng, n_internal=(0, 2))
        beams.append(beam)
        exts.append(ext)
        Vs.append(V)
        pins.append(abt_b200.params(abs=0.0, geo_cross_sec=gcs, beam_energy_out=0.9 * gcs,
                                    ext_energy_out=gcs))
    pins = np.array(pins)
    r = ctx.diff_batch(beams, exts, Vs, geo, th, ph, LAM, pins, is_fast_diff=fast, precision="fp64")
    f = ctx.diff_batch(beams, exts, Vs, geo, th, ph, LAM, pins, is_fast_diff=fast, precision="fp32")
    assert mueller_rel_err(f[0], r[0]) <= TOL_MU
    assert rel_err(f[1], r[1]) <= TOL_MU
    for n in ("scatt", "ext", "asymmetry", "scatt_beam", "scatt_ext_diff", "albedo"):
        assert abs(f[2][n] - r[2][n]) <= TOL_PARAM * abs(r[2][n]), n
    if fast:
        # the cull changes the result (it is not the full sum)
        full = ctx.diff_batch(beams, exts, Vs, geo, th, ph, LAM, pins, precision="fp64")
        assert rel_err(full[0], r[0]) > 1e-6


@pytest.mark.gpu
def test_fp32_fast_diff_tile_cull(ctx):
    """is_fast_diff on beam lists with small fields of view: the FP32 kernel
    skips whole (theta x phi) tiles outside a facet's cone; the result must
    still match the FP64 drop-in, which tests every bin."""
    geo, beam, _ = W.synthetic_beam_list(n_beams=30, facets_per_beam=40, seed=7)
    # narrow and wide cones, and external diffraction (a hemisphere each)
    beam["fov"] *= np.repeat(np.linspace(0.1, 2.0, 30), 40)
    ext = beam[::40].copy()
    ext["prop_out"] = (0.0, 0.0, -1.0)
    th, ph = abt_b200.make_angles([0, 180], [1]), abt_b200.make_angles([0, 358], [2])
    a32 = ctx.diff_main(beam, ext, geo, th, ph, LAM, is_fast_diff=True, precision="fp32")
    a64 = ctx.diff_main(beam, ext, geo, th, ph, LAM, is_fast_diff=True, precision="fp64")
    assert mueller_rel_err(_mueller(*a32), _mueller(*a64)) <= TOL_MU
    # the cull must not change the per-bin masking: compare against no culling
    ctx.set_plan(0, 1, 2048)   # the one-record kernel has no tile cull
    a32n = ctx.diff_main(beam, ext, geo, th, ph, LAM, is_fast_diff=True, precision="fp32")
    ctx.set_plan(-1)
    assert mueller_rel_err(_mueller(*a32), _mueller(*a32n)) <= 1e-5


def test_batch_runs_overlap_uploads(ctx):
    """A host batch large enough to be split into runs (uploads of run k+1
    overlap run k) gives the FP64 drop-in's average; a bad face index in a late
    run is still reported."""
    geo, Vs, beams, exts, pin = W.rough_column_orientations(40, seed=51, m_range=(20, 24))
    assert sum(len(b) + len(e) for b, e in zip(beams, exts)) > 3 * 262144 // 2
    th, ph = abt_b200.make_angles([0, 180], [10]), abt_b200.make_angles([0, 350], [10])
    r32 = ctx.diff_batch(beams, exts, Vs, geo, th, ph, LAM, pin, precision="fp32")
    r64 = ctx.diff_batch(beams, exts, Vs, geo, th, ph, LAM, pin, precision="fp64")
    assert mueller_rel_err(r32[0], r64[0]) <= TOL_MU
    for n in ("scatt", "ext", "asymmetry"):
        assert abs(float(r32[2][n]) - float(r64[2][n])) <= TOL_PARAM * abs(float(r64[2][n]))


def test_contiguous_batch_entry_matches_list_entry(ctx):
    """pbt_diff_batch_c (one gathered array, CSR offsets) and
    pbt_diff_batch_list_c (one array per orientation) give the same average."""
    import ctypes
    from abt_b200 import _lib
    geo, Vs, beams, exts, pin = W.rough_column_orientations(5, seed=61, n_side=2, n_len=3,
                                                            m_range=(0, 3))
    th, ph = abt_b200.make_angles([0, 180], [5]), abt_b200.make_angles([0, 350], [10])
    mu_l, m1_l, pav_l, _ = ctx.diff_batch(beams, exts, Vs, geo, th, ph, LAM, pin, precision="fp32")
    beam = np.concatenate(beams)
    ext = np.concatenate(exts)
    boff = np.concatenate([[0], np.cumsum([len(b) for b in beams])]).astype(np.int64)
    eoff = np.concatenate([[0], np.cumsum([len(e) for e in exts])]).astype(np.int64)
    V = np.concatenate([np.asfortranarray(v).ravel(order="F") for v in Vs])
    mu = np.empty((len(ph), len(th), 16), order="F")
    m1 = np.empty((len(th), 16), order="F")
    pav = np.zeros((), dtype=abt_b200.PARAMS_DTYPE)
    fo, fv = geo["face_off"], geo["face_vi"]
    _lib.check(_lib.lib().pbt_diff_batch_c(
        ctx.handle, len(beams), beam.ctypes.data, boff.ctypes.data, ext.ctypes.data,
        eoff.ctypes.data, V.ctypes.data, Vs[0].shape[0], fo.ctypes.data, fv.ctypes.data,
        len(fo) - 1, th.ctypes.data, len(th), ph.ctypes.data, len(ph), LAM, 0, 0, 1,
        pin.ctypes.data, mu.ctypes.data, m1.ctypes.data, pav.ctypes.data, None))
    assert mueller_rel_err(mu, mu_l) <= 1e-5
    assert abs(float(pav["scatt"]) - float(pav_l["scatt"])) <= 1e-6 * abs(float(pav_l["scatt"]))


@pytest.mark.gpu
def test_batch_writes_into_caller_arrays(ctx):
    """diff_batch(out=...) writes the Mueller averages into the caller's
    (here pinned) arrays, with the same values as freshly allocated ones, and
    refuses arrays of the wrong layout."""
    import torch
    geo, Vs, beams, exts, pin = W.rough_column_orientations(3, seed=62, n_side=2, n_len=3,
                                                            m_range=(0, 3))
    th, ph = abt_b200.make_angles([0, 180], [5]), abt_b200.make_angles([0, 350], [10])
    ref = ctx.diff_batch(beams, exts, Vs, geo, th, ph, LAM, pin, precision="fp32")
    mu = torch.empty(len(ph) * len(th) * 16, dtype=torch.float64, pin_memory=True).numpy()
    mu = mu.reshape((len(ph), len(th), 16), order="F")
    m1 = np.empty((len(th), 16), order="F")
    got = ctx.diff_batch(beams, exts, Vs, geo, th, ph, LAM, pin, precision="fp32", out=(mu, m1))
    assert got[0] is mu and got[1] is m1
    # same inputs, same launch plan: the same bits
    assert np.array_equal(mu, ref[0]) and np.array_equal(m1, ref[1])
    with pytest.raises(ValueError):
        ctx.diff_batch(beams, exts, Vs, geo, th, ph, LAM, pin, precision="fp32",
                       out=(np.empty((len(ph), len(th), 16)), m1))


@pytest.mark.gpu
def test_diff_main_writes_into_caller_arrays(ctx):
    """diff_main(out=...) fills the caller's (here pinned) grids with the values
    of freshly allocated ones, in both precisions, and refuses a wrong layout."""
    import torch
    rng = np.random.default_rng(8)
    th, ph = abt_b200.make_angles([0, 180], [5]), abt_b200.make_angles([0, 350], [10])
    geo = one_triangle(scale=2.0)
    beam = outbeams(3, rng, 1)
    ext = outbeams(1, rng, 1, prop=(0, 0, -1))
    shape = (len(ph), len(th), 2, 2)
    n = int(np.prod(shape)) * 16
    for prec in ("fp64", "fp32"):
        ref = ctx.diff_main(beam, ext, geo, th, ph, LAM, precision=prec)
        grids = [torch.empty(n, dtype=torch.uint8, pin_memory=True).numpy().view(np.complex128)
                 .reshape(shape, order="F") for _ in range(2)]
        got = ctx.diff_main(beam, ext, geo, th, ph, LAM, precision=prec, out=tuple(grids))
        assert got[0] is grids[0] and got[1] is grids[1]
        assert np.array_equal(got[0], ref[0]) and np.array_equal(got[1], ref[1])
    with pytest.raises(ValueError):
        ctx.diff_main(beam, ext, geo, th, ph, LAM, precision="fp32",
                      out=(np.empty(shape, np.complex128), np.empty(shape, np.complex128)))


@pytest.mark.parametrize("plan", [(1, 1, 256), (0, 1, 256), (1, 2, 512)],
                         ids=["packed", "one-record", "packed-2bins"])
def test_fp32_sums_are_reproducible(ctx, plan):
    """The FP32 form gives the same bits from run to run: each (segment, bin
    tile) adds its facet splits' FP64 sums in split order.  5,000 facets with
    256 records per work item make about 20 splits per tile, with and without
    the field-of-view cull, and in a batch of orientations."""
    geo, beam, _ = W.synthetic_beam_list(n_beams=50, facets_per_beam=100, seed=12)
    ext = beam[::7].copy()
    ext["prop_out"] = (0.0, 0.0, -1.0)
    th, ph = abt_b200.make_angles([0, 180], [2]), abt_b200.make_angles([0, 356], [4])
    ctx.set_plan(*plan)
    try:
        for fast in (False, True):
            runs = [ctx.diff_main(beam, ext, geo, th, ph, LAM, is_fast_diff=fast, precision="fp32")
                    for _ in range(3)]
            for r in runs[1:]:
                assert np.array_equal(r[0], runs[0][0]) and np.array_equal(r[1], runs[0][1])
        geo2, Vs, beams, exts, pin = W.rough_column_orientations(6, seed=63, n_side=3, n_len=6,
                                                                 m_range=(4, 8))
        b = [ctx.diff_batch(beams, exts, Vs, geo2, th, ph, LAM, pin, precision="fp32")
             for _ in range(2)]
        assert np.array_equal(b[0][0], b[1][0]) and np.array_equal(b[0][1], b[1][1])
        assert b[0][3].tobytes() == b[1][3].tobytes()
    finally:
        ctx.set_plan()


@pytest.mark.parametrize("plan", [(-1, 1, 2048), (0, 1, 2048)], ids=["packed", "one-record"])
@pytest.mark.parametrize("theta_deg", [[0, 0.5, 95, 120, 179, 180], [0, 0.25, 1.5, 90, 178.5, 180]],
                         ids=["bodge-row-backward", "bodge-row-forward"])
def test_fp32_poles_and_bodge_row_hemispheres(ctx, plan, theta_deg):
    """Bins exactly at theta = 0 and 180 deg, where s = u + sg z is zero, and a
    forward-bodge row (the first theta above 1 degree) in either hemisphere of
    the incidence direction (sg of the bodge row -1 or +1): the FP32 form stays
    within its bars of the FP64 drop-in, with external diffraction along the
    incidence direction and beams in random directions, on both kernels."""
    rng = np.random.default_rng(21)
    th = np.radians(np.array(theta_deg, dtype=np.float64))
    ph = abt_b200.make_angles([0, 350], [10])
    geo = mixed_polygon_geometry(rng)
    nf = len(geo["face_off"]) - 1
    beam = outbeams(12, rng, nf)
    ext = outbeams(nf, rng, nf, prop=(0, 0, -1))
    ext["fi"] = np.arange(1, nf + 1)
    ctx.set_plan(*plan)
    try:
        afb, afe = ctx.diff_main(beam, ext, geo, th, ph, LAM, precision="fp32")
    finally:
        ctx.set_plan()
    rfb, rfe = ctx.diff_main(beam, ext, geo, th, ph, LAM, precision="fp64")
    # normwise over the grid (the drop-in's own cancellation at q -> 0 in the
    # exact forward bin is ~1e-5 of that bin for these facet sizes)
    assert rel_err(afb + afe, rfb + rfe) <= 1e-4
    assert mueller_rel_err(_mueller(afb, afe), _mueller(rfb, rfe)) <= TOL_MU


@pytest.mark.parametrize("plan", [(-1, 1, 2048), (0, 1, 2048)], ids=["packed", "one-record"])
def test_fp32_clamp_lanes(ctx, plan):
    """Bins on the reference's clamp |ky| <= 0.999999 (src/diff_mod.f90:151):
    a triangle in the z = 0 plane with beams along (0, +-1, -1)/sqrt(2) has its
    aperture frame's y axis along +-x (x lies along the beam's projection on the
    plane), so the 15 bins within 0.08 deg of theta = 90 deg, phi = 0 or 180 deg
    have |ky| above the clamp (the kernels' rare branch, with kx^2 + kz^2 on its
    floor), next to bins just outside it.  There the reference divides kx and kz
    (below 1.4e-3) by s = 1.4e-3; formed from the bin direction in FP32 they
    carried an absolute error near 1e-7, and each clamp bin's Mueller elements
    were off by up to 5.8 times its M11 (1.9e-4 over the bins above 1e-6 of the
    peak).  The kernels form them from v = u - sigma R_1 instead: every bin within
    1e-4 of its M11, and the amplitudes normwise within 1e-4."""
    rng = np.random.default_rng(31)
    th = abt_b200.make_angles([89.8, 90.2], [0.05])
    ph = np.radians(np.concatenate([np.arange(0.0, 0.31, 0.05), np.arange(179.7, 180.31, 0.05)]))
    T, P = np.meshgrid(th, ph, indexing="ij")
    on_clamp = (np.abs(np.sin(T) * np.cos(P)) > 0.999999).T  # (phi, theta)
    assert on_clamp.sum() == 15
    geo = one_triangle(scale=2.0)
    beam = outbeams(4, rng, 1)
    s = 1.0 / np.sqrt(2.0)
    beam["prop_out"] = [(0, s, -s), (0, -s, -s), (0, s, -s), (0, -s, -s)]
    beam["vk7"] = [(1, 0, 0), (1, 0, 0), (-1, 0, 0), (-1, 0, 0)]
    ext = beam[:0]
    ctx.set_plan(*plan)
    try:
        afb, afe = ctx.diff_main(beam, ext, geo, th, ph, LAM, precision="fp32")
    finally:
        ctx.set_plan()
    rfb, rfe = ctx.diff_main(beam, ext, geo, th, ph, LAM, precision="fp64")
    assert np.isfinite(afb).all()
    assert rel_err(afb, rfb) <= 1e-4
    m32, m64 = _mueller(afb, afe), _mueller(rfb, rfe)
    assert mueller_rel_err(m32, m64) <= TOL_MU
    per_bin = np.abs(m32 - m64).max(axis=-1) / m64[..., 0]
    assert per_bin[on_clamp].max() <= TOL_MU


def test_fp32_precision_study_grid_100k_facets(ctx):
    """The precision-study grid at full size (721 theta x 360 phi, 259,560 bins)
    with half of its list (100,000 synthetic facets in a 100 um cube, phases up to
    ~1,000 rad): the FP32 batch within its bars of the FP64 drop-in, Mueller
    elements and cross sections."""
    geo, beam, _ = W.synthetic_beam_list(n_beams=1000, facets_per_beam=100, seed=2024)
    th, ph = W.grid_precision_study()
    ext = np.zeros(0, dtype=beam.dtype)
    pin = abt_b200.params(geo_cross_sec=1.0)
    f = ctx.diff_batch([beam], [ext], [geo["verts"]], geo, th, ph, LAM, pin[None], precision="fp32")
    r = ctx.diff_batch([beam], [ext], [geo["verts"]], geo, th, ph, LAM, pin[None], precision="fp64")
    assert mueller_rel_err(f[0], r[0]) <= TOL_MU
    for n in ("scatt", "asymmetry", "scatt_beam"):
        assert abs(float(f[2][n]) - float(r[2][n])) <= TOL_PARAM * abs(float(r[2][n])), n
