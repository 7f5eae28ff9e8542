"""Beam-list files: the per-orientation outbeam lists of the tracer, saved for
replay through the far-field entry points (C implementation in
csrc/beamlist.cpp, declared in include/pbt_diff.h).

    with BeamListWriter(path, theta, phi, geometry, lam) as w:
        for each orientation:   # the call site of diff_main, src/pbt_seq_mod.f90:212
            w.add(beam, ext, rotated_verts, params_in)
    bl = read_beam_list(path)
    ctx.diff_batch(bl.beams, bl.exts, bl.verts, bl.geometry, bl.theta, bl.phi,
                   bl.lam, bl.params_in, precision="fp32")
"""
import ctypes

import numpy as np

from . import _lib
from ._lib import OUTBEAM_DTYPE, PARAMS_DTYPE, check, ptr


class BeamListWriter:
    """pbt_beamlist_writer_open / _add / _close."""

    def __init__(self, path, theta, phi, geometry, lam):
        self._theta = np.ascontiguousarray(theta, dtype=np.float64)
        self._phi = np.ascontiguousarray(phi, dtype=np.float64)
        self._fo = np.ascontiguousarray(geometry["face_off"], dtype=np.int64)
        self._fv = np.ascontiguousarray(geometry["face_vi"], dtype=np.int64)
        self.nverts = int(np.asarray(geometry["verts"]).shape[0])
        h = ctypes.c_void_p()
        check(_lib.lib().pbt_beamlist_writer_open(
            str(path).encode(), ptr(self._theta), len(self._theta), ptr(self._phi), len(self._phi),
            self.nverts, ptr(self._fo), ptr(self._fv), len(self._fo) - 1, float(lam),
            ctypes.byref(h)))
        self._h = h

    def add(self, beam, ext, verts, params_in):
        """Append one orientation: outbeams, external-diffraction outbeams,
        rotated vertices (nverts,3) and its params_in record."""
        b = np.ascontiguousarray(beam if beam is not None else np.zeros(0, OUTBEAM_DTYPE),
                                 dtype=OUTBEAM_DTYPE)
        e = np.ascontiguousarray(ext if ext is not None else np.zeros(0, OUTBEAM_DTYPE),
                                 dtype=OUTBEAM_DTYPE)
        v = np.asfortranarray(verts, dtype=np.float64)
        if v.shape != (self.nverts, 3):
            raise ValueError("verts must be (%d, 3)" % self.nverts)
        p = np.array(params_in, dtype=PARAMS_DTYPE).reshape(())
        check(_lib.lib().pbt_beamlist_writer_add(self._h, ptr(b), len(b), ptr(e), len(e),
                                                 v.ctypes.data, p.ctypes.data))

    def close(self):
        if self._h:
            h, self._h = self._h, None
            check(_lib.lib().pbt_beamlist_writer_close(h))

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


class BeamList:
    """The contents of a beam-list file in pbt_diff_batch_c's layout."""

    def __init__(self, lam, theta, phi, geometry, verts, beams, exts, params_in):
        self.lam = lam
        self.theta = theta
        self.phi = phi
        self.geometry = geometry
        self.verts = verts          # list of (nverts,3)
        self.beams = beams          # list of outbeam arrays
        self.exts = exts
        self.params_in = params_in  # PARAMS_DTYPE array (norient,)

    @property
    def norient(self):
        return len(self.beams)


def read_beam_list(path):
    """pbt_beamlist_read: the whole file, copied into numpy arrays."""
    L = _lib.lib()
    h = ctypes.c_void_p()
    check(L.pbt_beamlist_read(str(path).encode(), ctypes.byref(h)))
    try:
        counts = np.zeros(8, dtype=np.int64)
        lam = ctypes.c_double()
        check(L.pbt_beamlist_info(h, counts.ctypes.data, ctypes.byref(lam)))
        no, nv, nf, nvi, nth, nph, nbt, nxt = (int(c) for c in counts)
        ptrs = [ctypes.c_void_p() for _ in range(10)]
        check(L.pbt_beamlist_arrays(h, *[ctypes.byref(q) for q in ptrs]))

        def arr(q, n, dtype):
            if n == 0:
                return np.zeros(0, dtype=dtype)
            nbytes = n * np.dtype(dtype).itemsize
            buf = (ctypes.c_char * nbytes).from_address(q.value)
            return np.frombuffer(buf, dtype=dtype).copy()

        theta = arr(ptrs[0], nth, np.float64)
        phi = arr(ptrs[1], nph, np.float64)
        fo = arr(ptrs[2], nf + 1, np.int64)
        fv = arr(ptrs[3], nvi, np.int64)
        V = arr(ptrs[4], no * nv * 3, np.float64)
        boff = arr(ptrs[5], no + 1, np.int64)
        beam = arr(ptrs[6], nbt, OUTBEAM_DTYPE)
        eoff = arr(ptrs[7], no + 1, np.int64)
        ext = arr(ptrs[8], nxt, OUTBEAM_DTYPE)
        pin = arr(ptrs[9], no, PARAMS_DTYPE)
    finally:
        L.pbt_beamlist_free(h)
    verts = [V[o * nv * 3:(o + 1) * nv * 3].reshape(3, nv).T.copy() for o in range(no)]
    beams = [beam[boff[o]:boff[o + 1]] for o in range(no)]
    exts = [ext[eoff[o]:eoff[o + 1]] for o in range(no)]
    geometry = dict(verts=verts[0] if no else np.zeros((nv, 3)), face_off=fo, face_vi=fv)
    return BeamList(lam.value, theta, phi, geometry, verts, beams, exts, pin)
