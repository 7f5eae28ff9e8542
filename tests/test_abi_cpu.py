"""CPU-only checks of the boundary: the built library loads and exports every
symbol include/pbt_diff.h declares; host-side logic mirrors the reference."""
import ctypes
import os
import re

import numpy as np
import pytest

import abt_b200
from abt_b200 import _lib
from abt_b200 import workloads as W
from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    src = open(os.path.join(ROOT, "include", "pbt_diff.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(pbt_\w+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    L = _lib.lib()
    declared = header_functions()
    assert len(declared) >= 12
    for name in declared:
        assert hasattr(L, name), name
    assert set(declared) == set(_lib.EXPORTS)
    assert L.pbt_version() == 10000


def test_struct_layouts_match_header():
    assert _lib.OUTBEAM_DTYPE.itemsize == 128
    assert _lib.PARAMS_DTYPE.itemsize == 18 * 8
    assert O.OUTBEAM_DTYPE == _lib.OUTBEAM_DTYPE


def test_no_device_reports_enodev():
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if has_gpu:
        pytest.skip("a GPU is present")
    for dev in (0, _lib.PBT_DEVICE_LOCAL_RANK):
        with pytest.raises(_lib.PbtError) as e:
            abt_b200.Context(dev)
        assert e.value.status == _lib.PBT_ENODEV
    # a NULL context is rejected with a status, not a crash
    assert _lib.lib().pbt_diff_main_c(None, None, 0, None, 0, None, 0, None, None, 0, None, 0,
                                      None, 0, 0.5, 0, 0, None, None) == _lib.PBT_EINVAL


@pytest.mark.parametrize("spec", [
    ([0, 180], [1]), ([0, 358], [2]), ([0, 180], [0.25]), ([0, 359], [1]),
    ([0, 2, 10, 180], [0.5, 2, 10]), ([0, 360], [1]), ([0, 180], [0.125]), ([0, 359.5], [0.5]),
])
def test_make_angles_mirror_matches_oracle(spec):
    a = abt_b200.make_angles(*spec)
    b = O.make_angles(*spec)
    assert a.shape == b.shape
    assert np.array_equal(a, b)


def test_make_angles_sizes_of_the_configs():
    assert len(abt_b200.make_angles([0, 180], [1])) == 181
    assert len(abt_b200.make_angles([0, 358], [2])) == 180
    assert len(abt_b200.make_angles([0, 180], [0.25])) == 721
    assert len(abt_b200.make_angles([0, 359], [1])) == 360
    assert len(abt_b200.make_angles([0, 180], [0.5])) == 361
    assert len(abt_b200.make_angles([0, 180], [0.125])) == 1441
    assert len(abt_b200.make_angles([0, 359.5], [0.5])) == 720
    with pytest.raises(ValueError):
        abt_b200.make_angles([0, 10], [3])


def test_synthetic_beam_list_shapes():
    geo, beam, ext = W.synthetic_beam_list(n_beams=20, facets_per_beam=100, seed=2024)
    assert len(beam) == 2000 and len(ext) == 0
    tri = geo["verts"].reshape(-1, 3, 3)
    edges = np.linalg.norm(tri - np.roll(tri, 1, axis=1), axis=2)
    assert edges.min() >= 0.3 - 1e-9 and edges.max() <= 1.5 + 1e-9
    c = tri.mean(axis=1)
    assert c.min() >= 0 and c.max() <= 100
    p = beam["prop_out"]
    assert np.allclose(np.linalg.norm(p, axis=1), 1)
    assert np.allclose((p * beam["vk7"]).sum(1), 0, atol=1e-12)
    # the facets of a beam share its amplitude and direction
    assert np.array_equal(beam["ampl"][0], beam["ampl"][99])


def test_hex_prism_is_closed_and_outward():
    geo = W.hex_prism(5.0, 10.0, n_side=2, n_len=3)
    n, a = W.facet_normals_areas(geo["verts"], geo["face_off"], geo["face_vi"])
    # area = 2 hexagons + 6 rectangles
    assert np.isclose(a.sum(), 2 * 1.5 * np.sqrt(3) * 25 + 6 * 5 * 10)
    # outward: normals point away from the centre
    c = geo["verts"][geo["face_vi"] - 1].reshape(-1, 3, 3).mean(1)
    assert ((n * c).sum(1) > 0).all()


def test_make_far_field_bins_matches_oracle():
    """make_far_field_bins through the C ABI (host only) equals the oracle's
    restatement bit for bit (both use the platform libm)."""
    import abt_b200
    from oracle import oracle as O
    th = abt_b200.make_angles([0, 2, 10, 180], [0.5, 2, 10])
    ph = abt_b200.make_angles([0, 350], [10])
    x, y, z = abt_b200.make_far_field_bins(th, ph)
    ref = O.far_field_bins(th, ph)
    assert x.shape == (len(ph), len(th))
    for a, r in zip((x, y, z), ref):
        assert np.array_equal(a.ravel(order="F"), r)
    with pytest.raises(abt_b200.PbtError):
        abt_b200.make_far_field_bins(th[:0], ph)


def test_allocation_failure_hook_counts():
    """pbt_test_fail_next_alloc (host-side failure injection) keeps a count of
    pending failures and returns the previous one; 0 clears it."""
    L = _lib.lib()
    assert L.pbt_test_fail_next_alloc(3) == 0
    assert L.pbt_test_fail_next_alloc(0) == 3
    assert L.pbt_test_fail_next_alloc(-5) == 0
    assert L.pbt_test_fail_next_alloc(0) == 0
