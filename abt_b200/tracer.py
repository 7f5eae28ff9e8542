"""The near-field tracer (host, FP64): the outbeam lists the far-field stage sums.

Python face of pbt_particle_* / pbt_trace_* in include/pbt_diff.h, mirroring the
reference's orientation step ahead of diff_main (src/pbt_seq_mod.f90:165-201):

  Particle(geometry, apertures)   the particle as prepared after reading
                                  (src/input_mod.f90:2663-2680): centre of
                                  mass moved to the origin, normals, apertures
  trace(particle, euler, ...)     PROT_MPI + make_incident_beam +
                                  beam_loop_for_speed + energy_checks: the
                                  rotated vertices, beam outbeams, external-
                                  diffraction outbeams and the params record
                                  finalise reads (abs, geo_cross_sec, energies)
  trace_batch(particle, eulers)   the same for many orientations, one per host
                                  thread
  traced_orientation_average(...) trace on the host and average on the GPU,
                                  overlapped chunk by chunk
  euler_from_degrees(a, b, g)     the 'euler' rotation method's angles
  multi_euler(u1, u2, u3)         the 'multi' method's angles

The tracer runs on the host cores (OpenMP); its results feed Context.diff_main,
Context.diff_batch or a beam-list file unchanged.
"""
import ctypes

import numpy as np

from . import _lib
from ._lib import OUTBEAM_DTYPE, TRACE_ENERGY_DTYPE, TRACE_PARAMS_DTYPE, check, ptr
from .diff import PI_REF, params as _params


def euler_from_degrees(alpha, beta, gamma):
    """Angles of the 'euler' rotation method in radians: |beta| < 1e-4 degree is
    lifted to 1e-4, then each angle times pi / 180 (src/input_mod.f90:1784-1786)."""
    e = np.array([alpha, beta, gamma], dtype=np.float64)
    if abs(e[1]) < 1e-4:
        e[1] = 1e-4
    return e * PI_REF / 180.0


def multi_euler(u1, u2, u3):
    """Angles of the 'multi' method from three uniform draws in [0, 1):
    alpha = 2 pi u1, beta = acos(1 - 2 u2), gamma = 2 pi u3
    (src/input_mod.f90:1848-1855)."""
    return np.array([2 * PI_REF * u1, np.arccos(1.0 - 2.0 * u2), 2 * PI_REF * u3])


def trace_params(lam, rbi, ibi=0.0, rec=8, refl=10, thresh_area=0.1, thresh_energy=1e-4):
    """A pbt_trace_params record; the defaults are the reference's
    (src/input_mod.f90:245, :302-305)."""
    p = np.zeros((), dtype=TRACE_PARAMS_DTYPE)
    p["lambda"], p["rbi"], p["ibi"] = lam, rbi, ibi
    p["rec"], p["refl"] = rec, refl
    p["thresh_area"], p["thresh_energy"] = thresh_area, thresh_energy
    return p


class Particle:
    """A particle prepared for tracing.  geometry: dict with verts (nverts,3),
    face_off (0-based offsets) and face_vi (1-based vertex indices) of
    triangular faces; apertures: 1-based aperture per face (None: every face
    its own aperture).  .geometry holds the centred vertices, .com the centre
    of mass they were moved by, .napertures the aperture count."""

    def __init__(self, geometry, apertures=None):
        L = _lib.lib()
        v = np.asfortranarray(geometry["verts"], dtype=np.float64)
        fo = np.ascontiguousarray(geometry["face_off"], dtype=np.int64)
        fv = np.ascontiguousarray(geometry["face_vi"], dtype=np.int64)
        ap = None if apertures is None else np.ascontiguousarray(apertures, dtype=np.int64)
        if ap is not None and ap.shape != (len(fo) - 1,):
            raise ValueError("apertures must have one entry per face")
        h = ctypes.c_void_p()
        check(L.pbt_particle_create(ptr(v), v.shape[0], ptr(fo), ptr(fv), len(fo) - 1, ptr(ap),
                                    ctypes.byref(h)))
        self._h = h
        nv, nf, na = (np.zeros(1, np.int64) for _ in range(3))
        com = np.zeros(3)
        check(L.pbt_particle_info(h, ptr(nv), ptr(nf), ptr(na), ptr(com)))
        self.napertures = int(na[0])
        self.com = com
        vc = np.zeros((int(nv[0]), 3), order="F")
        check(L.pbt_particle_verts(h, ptr(vc)))
        self.geometry = dict(verts=vc, face_off=fo.copy(), face_vi=fv.copy())

    def close(self):
        if getattr(self, "_h", None):
            _lib.lib().pbt_particle_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()


def _collect(L, h, nverts):
    nb, ne = np.zeros(1, np.int64), np.zeros(1, np.int64)
    check(L.pbt_trace_sizes(h, ptr(nb), ptr(ne)))
    beam = np.zeros(int(nb[0]), dtype=OUTBEAM_DTYPE)
    ext = np.zeros(int(ne[0]), dtype=OUTBEAM_DTYPE)
    V = np.zeros((nverts, 3), order="F")
    en = np.zeros((), dtype=TRACE_ENERGY_DTYPE)
    check(L.pbt_trace_copy(h, ptr(beam), ptr(ext), ptr(V), en.ctypes.data))
    pin = _params(abs=float(en["abs"]), geo_cross_sec=float(en["geo_cross_sec"]),
                  beam_energy_out=float(en["beam_energy_out"]),
                  ext_energy_out=float(en["ext_energy_out"]))
    return V, beam, ext, pin, en


def trace(particle, euler, lam, rbi, ibi=0.0, rec=8, refl=10, thresh_area=0.1,
          thresh_energy=1e-4):
    """One orientation: rotate by euler (radians), trace, and return
    (rotated vertices (nverts,3), beam outbeams, external-diffraction outbeams,
    params record for finalise, energy record).  The params record carries
    abs, geo_cross_sec, beam_energy_out and ext_energy_out as the reference's
    output_parameters does after the beam loop."""
    L = _lib.lib()
    e = np.ascontiguousarray(euler, dtype=np.float64)
    if e.shape != (3,):
        raise ValueError("euler must hold three angles")
    prm = trace_params(lam, rbi, ibi, rec, refl, thresh_area, thresh_energy)
    h = ctypes.c_void_p()
    check(L.pbt_trace_orientation_c(particle._h, ptr(e), prm.ctypes.data, ctypes.byref(h)))
    try:
        return _collect(L, h, particle.geometry["verts"].shape[0])
    finally:
        L.pbt_trace_destroy(h)


def trace_batch(particle, eulers, lam, rbi, ibi=0.0, rec=8, refl=10, thresh_area=0.1,
                thresh_energy=1e-4):
    """Many orientations (eulers: (n,3) radians), one per host thread.  Returns
    lists (Vs, beams, exts), the params records (n,) and the energy records (n,),
    each orientation exactly as trace() gives it."""
    L = _lib.lib()
    e = np.ascontiguousarray(eulers, dtype=np.float64).reshape(-1, 3)
    n = e.shape[0]
    prm = trace_params(lam, rbi, ibi, rec, refl, thresh_area, thresh_energy)
    hs = (ctypes.c_void_p * max(n, 1))()
    check(L.pbt_trace_batch_c(particle._h, n, ptr(e), prm.ctypes.data, hs))
    Vs, beams, exts = [], [], []
    pins = np.zeros(n, dtype=_params().dtype)
    ens = np.zeros(n, dtype=TRACE_ENERGY_DTYPE)
    try:
        for i in range(n):
            V, beam, ext, pin, en = _collect(L, hs[i], particle.geometry["verts"].shape[0])
            Vs.append(V)
            beams.append(beam)
            exts.append(ext)
            pins[i] = pin
            ens[i] = en
    finally:
        for i in range(n):
            L.pbt_trace_destroy(hs[i])
    return Vs, beams, exts, pins, ens


def traced_orientation_average(ctx, particle, eulers, theta, phi, lam, rbi, ibi=0.0, rec=8,
                               refl=10, thresh_area=0.1, thresh_energy=1e-4, chunk=256,
                               precision="fp32", is_fast_diff=False, scaling=False):
    """The reference's orientation loop (src/pbt_seq_mod.f90:146-274) with the
    tracer on the host cores and the far field on the GPU, overlapped: while
    the GPU averages one chunk of orientations (Context.diff_batch), the host
    traces the next.  Returns (mueller_avg, mueller_1d_avg, params_avg,
    params_per_orientation) as Context.diff_batch does for all orientations at
    once; the chunk averages are combined weighted by their orientation counts
    in FP64, which differs from one call by rounding only."""
    from concurrent.futures import ThreadPoolExecutor

    e = np.ascontiguousarray(eulers, dtype=np.float64).reshape(-1, 3)
    n = e.shape[0]
    if n == 0:
        raise ValueError("no orientations")
    chunk = max(1, int(chunk))
    starts = list(range(0, n, chunk))
    geo = particle.geometry
    mu = mu1 = pavg = None
    per = []

    def run(s):
        return trace_batch(particle, e[s:s + chunk], lam, rbi, ibi, rec, refl, thresh_area,
                           thresh_energy)

    with ThreadPoolExecutor(max_workers=1) as ex:
        fut = ex.submit(run, starts[0])
        for c, s in enumerate(starts):
            Vs, beams, exts, pins, _ = fut.result()
            if c + 1 < len(starts):
                fut = ex.submit(run, starts[c + 1])
            m, m1, pa, pp = ctx.diff_batch(beams, exts, Vs, geo, theta, phi, lam, pins,
                                           is_fast_diff=is_fast_diff, scaling=scaling,
                                           precision=precision)
            w = len(beams) / n
            if mu is None:
                mu, mu1 = m * w, m1 * w
                pavg = np.zeros((), dtype=pa.dtype)
            else:
                mu += m * w
                mu1 += m1 * w
            for name in pa.dtype.names:
                pavg[name] = pavg[name] + w * pa[name]
            per.append(np.atleast_1d(pp))
    return mu, mu1, pavg, np.concatenate(per)
