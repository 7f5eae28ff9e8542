"""pbt_diffraction_noalloc_c: the diffraction entry point that allocates nothing.

It serves host programs that cannot let a library allocate device memory
(their memory is reserved up front by their own pool allocator, or they may
allocate nothing after start-up).  It must give the same FP64 amplitude as
pbt_diffraction_c, within the FP64 parity tolerance of these tests (1e-10),
call after call, although every call reuses one fixed scratch array.

This file is collected last, so a failure here stops a -x run only after all
other tests have run; it passes alone in a fresh process too.
"""
import ctypes

import numpy as np
import pytest

import abt_b200
from abt_b200 import _lib
from tests.helpers import mixed_polygon_geometry, outbeams, rel_err

pytestmark = pytest.mark.gpu
LAM = 0.532


def noalloc(ob, geo, th, ph, fast):
    v = np.asfortranarray(geo["verts"], dtype=np.float64)
    fo = np.ascontiguousarray(geo["face_off"], dtype=np.int64)
    fv = np.ascontiguousarray(geo["face_vi"], dtype=np.int64)
    out = np.zeros((len(ph), len(th), 2, 2), dtype=np.complex128, order="F")
    st = _lib.lib().pbt_diffraction_noalloc_c(ob.ctypes.data, v.ctypes.data, v.shape[0],
                                              fo.ctypes.data, fv.ctypes.data, len(fo) - 1,
                                              th.ctypes.data, len(th), ph.ctypes.data, len(ph),
                                              LAM, int(fast), out.ctypes.data)
    return st, out


def test_no_alloc_matches_the_allocating_entry_point():
    rng = np.random.default_rng(77)
    geo = mixed_polygon_geometry(rng)
    nf = len(geo["face_off"]) - 1
    with abt_b200.Context(0) as ctx:
        cases = [
            (abt_b200.make_angles([0, 180], [2]), abt_b200.make_angles([0, 356], [4]), False, 1),
            (abt_b200.make_angles([0, 2, 10, 180], [0.5, 2, 5]),
             abt_b200.make_angles([0, 350], [10]), True, 5),
        ]
        for th, ph, fast, fi in cases:  # two calls in a row, different grids and facets
            ob = outbeams(1, rng, nf)
            ob["fi"] = fi
            ref = ctx.diffraction(ob, geo, th, ph, LAM, is_fast_diff=fast)
            st, out = noalloc(ob, geo, th, ph, fast)
            assert st == _lib.PBT_OK, _lib.lib().pbt_last_error_string()
            assert np.isfinite(out).all()
            assert rel_err(out, ref) <= 1e-10


def test_no_alloc_reuses_the_grid_only_when_it_is_the_same():
    """Calls alternate between two grids (A, B, A) and repeat a grid with other
    facets: the grid kept in the fixed array from the previous call is reused
    only when theta and phi are unchanged, and every result still equals the
    allocating entry point's."""
    rng = np.random.default_rng(79)
    geo = mixed_polygon_geometry(rng)
    nf = len(geo["face_off"]) - 1
    A = (abt_b200.make_angles([0, 180], [3]), abt_b200.make_angles([0, 354], [6]))
    B = (abt_b200.make_angles([0, 180], [2]), abt_b200.make_angles([0, 354], [6]))
    C = (A[0], abt_b200.make_angles([1, 355], [6]))  # A's shape, other phi values
    assert len(C[1]) == len(A[1])
    with abt_b200.Context(0) as ctx:
        for (th, ph), fi in ((A, 1), (B, 2), (A, 3), (A, 4), (C, 4), (A, 2), (B, 1)):
            ob = outbeams(1, rng, nf)
            ob["fi"] = fi
            ref = ctx.diffraction(ob, geo, th, ph, LAM)
            st, out = noalloc(ob, geo, th, ph, False)
            assert st == _lib.PBT_OK, _lib.lib().pbt_last_error_string()
            assert rel_err(out, ref) <= 1e-10


def test_no_alloc_rejects_grids_beyond_its_scratch():
    rng = np.random.default_rng(78)
    geo = mixed_polygon_geometry(rng)
    ob = outbeams(1, rng, len(geo["face_off"]) - 1)
    th = abt_b200.make_angles([0, 180], [0.25])   # 721 x 360 = 259,560 bins > 65,536
    ph = abt_b200.make_angles([0, 359], [1])
    st, _ = noalloc(ob, geo, th, ph, False)
    assert st == _lib.PBT_EINVAL
    assert b"scratch" in _lib.lib().pbt_last_error_string()


def test_no_alloc_rejects_too_many_phi_values_and_large_faces():
    """4,097 phi values (in only 12,291 bins) and a 65-vertex face are over the
    fixed limits and are refused before anything is copied."""
    rng = np.random.default_rng(79)
    geo = mixed_polygon_geometry(rng)
    ob = outbeams(1, rng, len(geo["face_off"]) - 1)
    th = np.radians([0.0, 2.0, 4.0])
    ph = np.linspace(0.0, 2 * np.pi, 4097, endpoint=False)
    st, _ = noalloc(ob, geo, th, ph, False)
    assert st == _lib.PBT_EINVAL and b"4096" in _lib.lib().pbt_last_error_string()
    # a regular 65-gon in the z = 0 plane, and a 64-gon that is accepted
    for n, want in ((65, _lib.PBT_EINVAL), (64, _lib.PBT_OK)):
        a = 2 * np.pi * np.arange(n) / n
        verts = np.stack([3 * np.cos(a), 3 * np.sin(a), np.zeros(n)], 1)
        g = abt_b200.make_geometry(verts, [list(range(1, n + 1))])
        o = outbeams(1, rng, 1)
        st, out = noalloc(o, g, abt_b200.make_angles([0, 180], [5]),
                          abt_b200.make_angles([0, 350], [10]), False)
        assert st == want, _lib.lib().pbt_last_error_string()
        if want == _lib.PBT_EINVAL:
            assert b"64" in _lib.lib().pbt_last_error_string()
        else:
            assert np.isfinite(out).all()


def test_no_alloc_calls_leave_device_memory_unchanged():
    """After a first call (which loads the device code and commits the fixed
    array), further calls change the device's free memory by nothing."""
    import torch
    rng = np.random.default_rng(80)
    geo = mixed_polygon_geometry(rng)
    ob = outbeams(1, rng, len(geo["face_off"]) - 1)
    th, ph = abt_b200.make_angles([0, 180], [2]), abt_b200.make_angles([0, 356], [4])
    st, first = noalloc(ob, geo, th, ph, False)
    assert st == _lib.PBT_OK
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info(0)
    for fast in (False, True, False):
        st, out = noalloc(ob, geo, th, ph, fast)
        assert st == _lib.PBT_OK
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info(0)
    assert free1 == free0
    assert np.array_equal(out, first)
