"""Host-side mirror of PBT's far-field interface over the C ABI.

Names, argument meanings and layouts follow the reference's Fortran routines
(src/diff_mod.f90 diff_main / diffraction / make_far_field_bins,
src/outputs_mod.f90 finalise / summation / divide_by_num_orientations,
src/input_mod.f90 make_angles), so that tests read like the reference's own
call sites.  Every compute call runs on the GPU through libpbt_b200.so.

Arrays:
  geometry           dict(verts=(nverts,3) float64, face_off=(nfaces+1,) int64
                     0-based CSR offsets, face_vi=1-based vertex indices)
  outbeams           numpy arrays of OUTBEAM_DTYPE
  amplitude grids    complex128 (nphi, ntheta, 2, 2), Fortran order
  Mueller grids      float64 (nphi, ntheta, 16) / (ntheta, 16), Fortran order
"""
import ctypes

import numpy as np

from . import _lib
from ._lib import OUTBEAM_DTYPE, PARAMS_DTYPE, PARAM_NAMES, PBT_PREC_FP32, PBT_PREC_FP64, check, ptr

# src/misc_submod.f90:12 -- a default-real literal widened to real(8)
PI_REF = float(np.float32(3.14159265358979))

_PREC = {"fp64": PBT_PREC_FP64, "fp32": PBT_PREC_FP32}


def make_angles(vals_deg, splits_deg):
    """make_angles (src/input_mod.f90:114-196) then the degree-to-radian step
    theta_vals*pi/180d0 (src/input_mod.f90:742): a piecewise grid given as
    values v1 s1 v2 s2 ... vn; interior segment ends are dropped."""
    v = [float(x) for x in vals_deg]
    s = [float(x) for x in splits_deg]
    if len(v) < 2 or len(s) < len(v) - 1:
        raise ValueError("need n values and n-1 splits")
    out = []
    n = len(v)
    for i in range(n - 1):
        q = (v[i + 1] - v[i]) / s[i]
        jmax = int(np.floor(abs(q) + 0.5)) * (1 if q >= 0 else -1)
        fr = np.fmod(q, 1.0)
        if float(np.float32(1e-3)) < fr < float(np.float32(1.0) - np.float32(1e-3)):
            raise ValueError("bad angle choice on segment %d: %g is not close to an integer"
                             % (i + 1, q))
        for j in range(jmax + 1):
            if i != n - 2 and j == jmax:
                continue
            out.append(v[i] + j * s[i])
    a = np.array(out, dtype=np.float64)
    return a * PI_REF / 180.0


def make_far_field_bins(theta, phi):
    """make_far_field_bins (src/diff_mod.f90:827-855) -> (xfar, yfar, zfar),
    each (nphi, ntheta) in Fortran order (pbt_make_far_field_bins_c)."""
    theta = np.ascontiguousarray(theta, dtype=np.float64)
    phi = np.ascontiguousarray(phi, dtype=np.float64)
    out = [np.zeros((len(phi), len(theta)), order="F") for _ in range(3)]
    check(_lib.lib().pbt_make_far_field_bins_c(ptr(theta), len(theta), ptr(phi), len(phi),
                                               *[o.ctypes.data for o in out]))
    return tuple(out)


def make_geometry(verts, faces):
    """Geometry dict from (nverts,3) vertices and a list of 1-based vertex index lists."""
    verts = np.asarray(verts, dtype=np.float64)
    off = np.zeros(len(faces) + 1, dtype=np.int64)
    off[1:] = np.cumsum([len(f) for f in faces])
    vi = np.concatenate([np.asarray(f, dtype=np.int64) for f in faces])
    return dict(verts=verts, face_off=off, face_vi=vi)


def params(abs=0.0, geo_cross_sec=1.0, beam_energy_out=1.0, ext_energy_out=1.0):
    """The inputs of finalise carried in output_parameters_type."""
    p = np.zeros((), dtype=PARAMS_DTYPE)
    p["abs"] = abs
    p["geo_cross_sec"] = geo_cross_sec
    p["beam_energy_out"] = beam_energy_out
    p["ext_energy_out"] = ext_energy_out
    return p


def _geo(geometry):
    v = np.asfortranarray(geometry["verts"], dtype=np.float64)
    fo = np.ascontiguousarray(geometry["face_off"], dtype=np.int64)
    fv = np.ascontiguousarray(geometry["face_vi"], dtype=np.int64)
    return v, fo, fv


def _ob(a):
    return np.ascontiguousarray(np.atleast_1d(a) if a is not None else np.zeros(0, OUTBEAM_DTYPE),
                                dtype=OUTBEAM_DTYPE)


class Context:
    """A library context on one CUDA device (pbt_ctx_create / pbt_ctx_destroy).
    device=-1 (PBT_DEVICE_LOCAL_RANK) takes the launcher's node-local rank
    modulo the visible devices; `device` holds the device the context is on."""

    def __init__(self, device=0):
        L = _lib.lib()
        h = ctypes.c_void_p()
        check(L.pbt_ctx_create(int(device), ctypes.byref(h)))
        self._h = h
        d = ctypes.c_int(-1)
        check(L.pbt_ctx_device(h, ctypes.byref(d)))
        self.device = d.value

    @property
    def handle(self):
        return self._h

    def close(self):
        if self._h:
            _lib.lib().pbt_ctx_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def last_launch_count(self):
        return int(_lib.lib().pbt_last_launch_count(self._h))

    def set_kernel_timing(self, enable=True):
        check(_lib.lib().pbt_set_kernel_timing(self._h, int(bool(enable))))

    def set_plan(self, variant=-1, bins_per_thread=1, records_per_item=2048):
        """Launch plan of the FP32 kernel (variant < 0: default)."""
        check(_lib.lib().pbt_set_plan(self._h, int(variant), int(bins_per_thread),
                                      int(records_per_item)))

    def selftest_bounded_wait(self, limit_ms=200):
        """pbt_selftest_bounded_wait_c: a device wait that nothing completes must
        give up by itself; raises PbtError(PBT_ETIMEOUT) as designed."""
        check(_lib.lib().pbt_selftest_bounded_wait_c(self._h, int(limit_ms)))

    def kernel_time_ms(self):
        """(total ms, launches) of the far-field kernels timed since the last call."""
        t = ctypes.c_double()
        n = ctypes.c_int64()
        check(_lib.lib().pbt_kernel_time_ms(self._h, ctypes.byref(t), ctypes.byref(n)))
        return t.value, n.value

    # ------------------------------------------------------------ diff_mod
    def diff_main(self, beam, ext, geometry, theta, phi, lam, is_fast_diff=False,
                  precision="fp64", out=None):
        """diff_main (src/diff_mod.f90:674-825) -> (ampl_far_beam, ampl_far_ext_diff).

        out: optional (ampl_far_beam, ampl_far_ext_diff) arrays to write into,
        complex128 of shape (nphi, ntheta, 2, 2) in Fortran order (e.g. views
        of pinned host memory, reused call after call)."""
        beam, ext = _ob(beam), _ob(ext)
        v, fo, fv = _geo(geometry)
        theta = np.ascontiguousarray(theta, dtype=np.float64)
        phi = np.ascontiguousarray(phi, dtype=np.float64)
        shape = (len(phi), len(theta), 2, 2)
        if out is None:
            afb = np.empty(shape, dtype=np.complex128, order="F")
            afe = np.empty(shape, dtype=np.complex128, order="F")
        else:
            afb, afe = out
            for a in (afb, afe):
                if (not isinstance(a, np.ndarray) or a.dtype != np.complex128 or a.shape != shape
                        or not a.flags.f_contiguous or not a.flags.writeable):
                    raise ValueError("out arrays must be writeable Fortran-ordered complex128 of "
                                     "shape (nphi, ntheta, 2, 2)")
        check(_lib.lib().pbt_diff_main_c(self._h, ptr(beam), len(beam), ptr(ext), len(ext),
                                         ptr(v), v.shape[0], ptr(fo), ptr(fv), len(fo) - 1,
                                         ptr(theta), len(theta), ptr(phi), len(phi), float(lam),
                                         int(bool(is_fast_diff)), _PREC[precision],
                                         afb.ctypes.data, afe.ctypes.data))
        return afb, afe

    def diffraction(self, outbeam, geometry, theta, phi, lam, is_fast_diff=False):
        """diffraction (src/diff_mod.f90:446-672) for one outbeam -> amplC."""
        ob = _ob(outbeam)[:1]
        v, fo, fv = _geo(geometry)
        theta = np.ascontiguousarray(theta, dtype=np.float64)
        phi = np.ascontiguousarray(phi, dtype=np.float64)
        out = np.zeros((len(phi), len(theta), 2, 2), dtype=np.complex128, order="F")
        check(_lib.lib().pbt_diffraction_c(self._h, ptr(ob), ptr(v), v.shape[0], ptr(fo), ptr(fv),
                                           len(fo) - 1, ptr(theta), len(theta), ptr(phi),
                                           len(phi), float(lam), int(bool(is_fast_diff)),
                                           out.ctypes.data))
        return out

    def diff_adjoint(self, beam, ext, geometry, theta, phi, lam, grad_ampl_far_beam,
                     grad_ampl_far_ext_diff, is_fast_diff=False):
        """Vector-Jacobian product of the FP32 diff_main (pbt_diff_adjoint_c).

        The cotangents are (nphi,ntheta,2,2) complex arrays dL/dRe + i dL/dIm;
        returns (grad_verts (nverts,3), grad_beam_ampl (nbeam,8),
        grad_ext_ampl (next,8)), the amplitude gradients as re/im of
        ampl(1,1),(2,1),(1,2),(2,2) like the records' ampl field."""
        beam, ext = _ob(beam), _ob(ext)
        v, fo, fv = _geo(geometry)
        theta = np.ascontiguousarray(theta, dtype=np.float64)
        phi = np.ascontiguousarray(phi, dtype=np.float64)
        ga = np.asfortranarray(grad_ampl_far_beam, dtype=np.complex128)
        ge = np.asfortranarray(grad_ampl_far_ext_diff, dtype=np.complex128)
        shape = (len(phi), len(theta), 2, 2)
        if ga.shape != shape or ge.shape != shape:
            raise ValueError(f"cotangent shape must be {shape}")
        gv = np.zeros((v.shape[0], 3), order="F")
        gb = np.zeros((max(len(beam), 1), 8))
        gx = np.zeros((max(len(ext), 1), 8))
        check(_lib.lib().pbt_diff_adjoint_c(self._h, ptr(beam), len(beam), ptr(ext), len(ext),
                                            ptr(v), v.shape[0], ptr(fo), ptr(fv), len(fo) - 1,
                                            ptr(theta), len(theta), ptr(phi), len(phi), float(lam),
                                            int(bool(is_fast_diff)), ga.ctypes.data,
                                            ge.ctypes.data, gv.ctypes.data, gb.ctypes.data,
                                            gx.ctypes.data))
        return gv, gb[:len(beam)], gx[:len(ext)]

    # --------------------------------------------------------- outputs_mod
    def finalise(self, ampl_far_beam, ampl_far_ext_diff, theta, phi, lam, params_in,
                 scaling=False, accumulate=False):
        """finalise (src/outputs_mod.f90:63-278) -> (mueller, mueller_1d, params)."""
        theta = np.ascontiguousarray(theta, dtype=np.float64)
        phi = np.ascontiguousarray(phi, dtype=np.float64)
        afb = np.asfortranarray(ampl_far_beam, dtype=np.complex128)
        afe = np.asfortranarray(ampl_far_ext_diff, dtype=np.complex128)
        p = np.array(params_in, dtype=PARAMS_DTYPE).copy()
        mu = np.zeros((len(phi), len(theta), 16), order="F")
        mu1 = np.zeros((len(theta), 16), order="F")
        check(_lib.lib().pbt_finalise_c(self._h, afb.ctypes.data, afe.ctypes.data, ptr(theta),
                                        len(theta), ptr(phi), len(phi), float(lam),
                                        int(bool(scaling)), p.ctypes.data, mu.ctypes.data,
                                        mu1.ctypes.data, int(bool(accumulate))))
        return mu, mu1, p

    def summation(self, mueller, mueller_1d, params_in):
        """summation (src/outputs_mod.f90:407-471) into the context's device totals."""
        mu = np.asfortranarray(mueller, dtype=np.float64)
        mu1 = np.asfortranarray(mueller_1d, dtype=np.float64)
        p = np.array(params_in, dtype=PARAMS_DTYPE)
        check(_lib.lib().pbt_summation_c(self._h, mu.ctypes.data, mu1.ctypes.data, p.ctypes.data,
                                         mu.shape[1], mu.shape[0]))

    def divide_by_num_orientations(self, num_orients, ntheta, nphi):
        """divide_by_num_orientations (src/outputs_mod.f90:13-43) of the device totals."""
        mu = np.zeros((nphi, ntheta, 16), order="F")
        mu1 = np.zeros((ntheta, 16), order="F")
        p = np.zeros((), dtype=PARAMS_DTYPE)
        check(_lib.lib().pbt_divide_by_num_orientations_c(self._h, int(num_orients),
                                                          mu.ctypes.data, mu1.ctypes.data,
                                                          p.ctypes.data))
        return mu, mu1, p

    def totals_reset(self):
        check(_lib.lib().pbt_totals_reset_c(self._h))

    # ------------------------------------------------------------ batched
    def diff_batch(self, beams, exts, verts_per_orient, geometry, theta, phi, lam,
                   params_in, is_fast_diff=False, scaling=False, precision="fp32", out=None):
        """Orientation average of norient orientations in one call.

        beams / exts: lists (one per orientation) of outbeam arrays.
        verts_per_orient: list of (nverts,3) rotated vertex arrays (topology from geometry).
        params_in: PARAMS_DTYPE array of length norient.
        out: optional (mueller_avg, mueller_1d_avg) arrays to write into, float64
        of shapes (nphi, ntheta, 16) and (ntheta, 16) in Fortran order (e.g. views
        of pinned host memory, which the device writes at full speed).
        Returns (mueller_avg, mueller_1d_avg, params_avg, params_per_orient)."""
        norient = len(beams)
        if len(exts) != norient or len(verts_per_orient) != norient:
            raise ValueError("beams, exts and verts_per_orient need one entry per orientation")
        # each orientation's arrays go to the library as they are (no host-side
        # gather; pinned arrays stay pinned): pbt_diff_batch_list_c
        bl = [_ob(b) for b in beams]
        el = [_ob(e) for e in exts]
        vl = [np.asfortranarray(v, dtype=np.float64) for v in verts_per_orient]
        nverts = vl[0].shape[0]
        if any(v.shape != (nverts, 3) for v in vl):
            raise ValueError("every orientation needs a (nverts, 3) vertex array")
        _, fo, fv = _geo(geometry)
        theta = np.ascontiguousarray(theta, dtype=np.float64)
        phi = np.ascontiguousarray(phi, dtype=np.float64)
        pin = np.ascontiguousarray(params_in, dtype=PARAMS_DTYPE)
        if out is None:
            mu = np.empty((len(phi), len(theta), 16), order="F")
            mu1 = np.empty((len(theta), 16), order="F")
        else:
            mu, mu1 = out
            for a, shape in ((mu, (len(phi), len(theta), 16)), (mu1, (len(theta), 16))):
                if (not isinstance(a, np.ndarray) or a.dtype != np.float64 or a.shape != shape
                        or not a.flags.f_contiguous or not a.flags.writeable):
                    raise ValueError("out arrays must be writeable Fortran-ordered float64 of "
                                     "shapes (nphi, ntheta, 16) and (ntheta, 16)")
        pav = np.zeros((), dtype=PARAMS_DTYPE)
        pper = np.zeros(norient, dtype=PARAMS_DTYPE)
        VP = ctypes.c_void_p * norient
        pb = VP(*[ptr(b) for b in bl])
        pe = VP(*[ptr(e) for e in el])
        pv = VP(*[v.ctypes.data for v in vl])
        nbm = np.array([len(b) for b in bl], dtype=np.int64)
        nex = np.array([len(e) for e in el], dtype=np.int64)
        check(_lib.lib().pbt_diff_batch_list_c(
            self._h, norient, ctypes.cast(pb, ctypes.c_void_p), nbm.ctypes.data,
            ctypes.cast(pe, ctypes.c_void_p), nex.ctypes.data, ctypes.cast(pv, ctypes.c_void_p),
            nverts, ptr(fo), ptr(fv), len(fo) - 1, ptr(theta), len(theta), ptr(phi), len(phi),
            float(lam), int(bool(is_fast_diff)), int(bool(scaling)), _PREC[precision], ptr(pin),
            mu.ctypes.data, mu1.ctypes.data, pav.ctypes.data, pper.ctypes.data))
        return mu, mu1, pav, pper


def params_dict(p):
    return {n: float(p[n]) for n in PARAM_NAMES}


def diff_batch_dev(ctx, stream, norient, d_beam, beam_off, d_ext, ext_off, d_verts, nverts,
                   face_off, d_face_vi, theta, phi, lam, d_params_in, d_mueller_avg, d_m1d_avg,
                   d_params_avg, d_params_per=None, is_fast_diff=False, scaling=False):
    """pbt_diff_batch_dev_c: the FP32 batched average on device-resident arrays.
    d_* are device pointers (ints) or torch CUDA tensors; beam_off, ext_off,
    face_off, theta and phi are host numpy arrays.  stream: a cudaStream_t
    handle (int), e.g. torch.cuda.current_stream().cuda_stream."""
    boff = np.ascontiguousarray(beam_off, dtype=np.int64)
    eoff = np.ascontiguousarray(ext_off, dtype=np.int64)
    fo = np.ascontiguousarray(face_off, dtype=np.int64)
    theta = np.ascontiguousarray(theta, dtype=np.float64)
    phi = np.ascontiguousarray(phi, dtype=np.float64)
    check(_lib.lib().pbt_diff_batch_dev_c(
        ctx.handle, stream, int(norient), ptr(d_beam), ptr(boff), ptr(d_ext), ptr(eoff),
        ptr(d_verts), int(nverts), ptr(fo), ptr(d_face_vi), len(fo) - 1, ptr(theta), len(theta),
        ptr(phi), len(phi), float(lam), int(bool(is_fast_diff)), int(bool(scaling)),
        PBT_PREC_FP32, ptr(d_params_in), ptr(d_mueller_avg), ptr(d_m1d_avg), ptr(d_params_avg),
        ptr(d_params_per)))


class BatchGraph:
    """pbt_diff_batch_dev_graph_c: the device-pointer FP32 batch captured as a
    CUDA graph.  Construction runs the batch once and captures it; launch()
    replays it on a stream (the device arrays are re-read at every replay)."""

    def __init__(self, ctx, stream, norient, d_beam, beam_off, d_ext, ext_off, d_verts, nverts,
                 face_off, d_face_vi, theta, phi, lam, d_params_in, d_mueller_avg, d_m1d_avg,
                 d_params_avg, d_params_per=None, is_fast_diff=False, scaling=False):
        boff = np.ascontiguousarray(beam_off, dtype=np.int64)
        eoff = np.ascontiguousarray(ext_off, dtype=np.int64)
        fo = np.ascontiguousarray(face_off, dtype=np.int64)
        theta = np.ascontiguousarray(theta, dtype=np.float64)
        phi = np.ascontiguousarray(phi, dtype=np.float64)
        h = ctypes.c_void_p()
        check(_lib.lib().pbt_diff_batch_dev_graph_c(
            ctx.handle, stream, int(norient), ptr(d_beam), ptr(boff), ptr(d_ext), ptr(eoff),
            ptr(d_verts), int(nverts), ptr(fo), ptr(d_face_vi), len(fo) - 1, ptr(theta),
            len(theta), ptr(phi), len(phi), float(lam), int(bool(is_fast_diff)),
            int(bool(scaling)), ptr(d_params_in), ptr(d_mueller_avg), ptr(d_m1d_avg),
            ptr(d_params_avg), ptr(d_params_per), ctypes.byref(h)))
        self._h = h

    def launch(self, stream):
        check(_lib.lib().pbt_graph_launch_c(self._h, stream))

    def kernel_count(self):
        return int(_lib.lib().pbt_graph_kernel_count(self._h))

    def close(self):
        if self._h:
            _lib.lib().pbt_graph_destroy_c(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
