"""ctypes binding of the C FP64 oracle (oracle/pbt_oracle.c).

TEST INFRASTRUCTURE ONLY.  Parity unpinned: the Fortran reference cannot be
run here; the oracle is checked against closed-form answers and frozen
fixtures.  Layouts follow the reference: far-field amplitude grids are
complex(8) (nphi, ntheta, 2, 2) in Fortran order (src/diff_mod.f90:717-718),
Mueller grids real(8) (nphi, ntheta, 16) (src/outputs_mod.f90:483), 1-D
Mueller (ntheta, 16) (src/outputs_mod.f90:291).
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpbt_oracle.so")

# pbt_outbeam layout (128 bytes), the fields of outbeamtype that diffraction reads
OUTBEAM_DTYPE = np.dtype([("ampl", "<f8", (8,)), ("vk7", "<f8", (3,)),
                          ("prop_out", "<f8", (3,)), ("fov", "<f8"), ("fi", "<i8")])
assert OUTBEAM_DTYPE.itemsize == 128

PARAM_NAMES = ("abs", "scatt", "ext", "albedo", "asymmetry", "abs_eff", "scatt_eff",
               "ext_eff", "geo_cross_sec", "back_scatt", "beam_energy_out",
               "ext_energy_out", "scatt_beam", "scatt_ext_diff", "asymmetry_beam",
               "asymmetry_ext_diff", "scatt_eff_beam", "scatt_eff_ext_diff")

PI_REF = float(np.float32(3.14159265358979))

_lib = None


def build():
    subprocess.check_call(["make", "-s", "-C", HERE, "libpbt_oracle.so"])


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH) or (
                os.path.getmtime(LIB_PATH) < os.path.getmtime(os.path.join(HERE, "pbt_oracle.c"))):
            build()
        L = ctypes.CDLL(LIB_PATH)
        P = ctypes.c_void_p
        I64 = ctypes.c_int64
        D = ctypes.c_double
        L.oracle_make_angles.restype = I64
        L.oracle_make_angles.argtypes = [P, P, I64, P, I64]
        L.oracle_deg_to_rad.argtypes = [P, I64]
        L.oracle_openmp.restype = ctypes.c_int
        L.oracle_openmp.argtypes = []
        L.oracle_simpne.restype = D
        L.oracle_simpne.argtypes = [I64, P, P, I64]
        L.oracle_diff_main_flat.restype = ctypes.c_int
        L.oracle_diff_main_flat.argtypes = [P, I64, P, I64, D, ctypes.c_int, P, I64, P, P, I64,
                                            P, I64, P, I64, P, P, ctypes.c_int]
        L.oracle_diffraction_flat.restype = ctypes.c_int
        L.oracle_diffraction_flat.argtypes = [P, I64, P, I64, D, ctypes.c_int, P, I64, P, P, I64,
                                              P, D, P]
        L.oracle_finalise_flat.restype = ctypes.c_int
        L.oracle_finalise_flat.argtypes = [P, P, I64, I64, P, P, D, ctypes.c_int, P, P, P]
        L.oracle_summation_flat.argtypes = [P, P, I64, P, P, I64, P, P]
        L.oracle_divide_flat.argtypes = [P, I64, P, I64, P, I64]
        L.oracle_make_far_field_bins.argtypes = [P, I64, P, I64, P, P, P]
        L.oracle_ampl_to_mueller.argtypes = [I64, P, P]
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None and a.size else None


def make_angles(vals_deg, splits_deg):
    """make_angles + degree->radian conversion (src/input_mod.f90:114-196,742)."""
    v = np.ascontiguousarray(vals_deg, dtype=np.float64)
    s = np.ascontiguousarray(splits_deg, dtype=np.float64)
    out = np.zeros(200000)
    n = lib().oracle_make_angles(_p(v), _p(s), len(v), _p(out), len(out))
    if n < 0:
        raise ValueError("bad angle choice")
    out = np.ascontiguousarray(out[:n])
    lib().oracle_deg_to_rad(_p(out), n)
    return out


def far_field_bins(theta, phi):
    nb = len(theta) * len(phi)
    xyz = np.zeros((3, nb))
    lib().oracle_make_far_field_bins(_p(theta), len(theta), _p(phi), len(phi),
                                     _p(xyz[0]), _p(xyz[1]), _p(xyz[2]))
    return xyz


def _geom(geometry):
    v = np.asfortranarray(geometry["verts"], dtype=np.float64)   # (nverts, 3)
    fo = np.ascontiguousarray(geometry["face_off"], dtype=np.int64)
    fv = np.ascontiguousarray(geometry["face_vi"], dtype=np.int64)
    return v, fo, fv


def openmp_threads(nthreads):
    """Threads oracle_diff_main_omp really uses for a request of nthreads:
    nthreads when the library was built with OpenMP, else 1."""
    return nthreads if lib().oracle_openmp() else 1


def diff_main(theta, phi, lam, geometry, beam, ext, is_fast_diff=False, nthreads=0):
    """diff_main (src/diff_mod.f90:674-825) -> (ampl_far_beam, ampl_far_ext_diff),
    complex128 arrays of shape (nphi, ntheta, 2, 2), Fortran order.
    nthreads=0: sequential facet order; >0: the reference's OpenMP loop shape."""
    theta = np.ascontiguousarray(theta, dtype=np.float64)
    phi = np.ascontiguousarray(phi, dtype=np.float64)
    v, fo, fv = _geom(geometry)
    beam = np.ascontiguousarray(beam, dtype=OUTBEAM_DTYPE)
    ext = np.ascontiguousarray(ext, dtype=OUTBEAM_DTYPE)
    nphi, nth = len(phi), len(theta)
    afb = np.zeros((nphi, nth, 2, 2), dtype=np.complex128, order="F")
    afe = np.zeros((nphi, nth, 2, 2), dtype=np.complex128, order="F")
    rc = lib().oracle_diff_main_flat(_p(theta), nth, _p(phi), nphi, lam, int(bool(is_fast_diff)),
                                     _p(v), v.shape[0], _p(fo), _p(fv), len(fo) - 1,
                                     _p(beam), len(beam), _p(ext), len(ext),
                                     afb.ctypes.data_as(ctypes.c_void_p),
                                     afe.ctypes.data_as(ctypes.c_void_p), int(nthreads))
    if rc:
        raise RuntimeError("oracle diff_main failed: %d" % rc)
    return afb, afe


def diffraction(theta, phi, lam, geometry, outbeam, is_fast_diff=False, fov_override=-1.0):
    """diffraction (src/diff_mod.f90:446-672) for one outbeam -> amplC (nphi,ntheta,2,2)."""
    theta = np.ascontiguousarray(theta, dtype=np.float64)
    phi = np.ascontiguousarray(phi, dtype=np.float64)
    v, fo, fv = _geom(geometry)
    ob = np.ascontiguousarray(np.atleast_1d(outbeam), dtype=OUTBEAM_DTYPE)
    nphi, nth = len(phi), len(theta)
    out = np.zeros((nphi, nth, 2, 2), dtype=np.complex128, order="F")
    rc = lib().oracle_diffraction_flat(_p(theta), nth, _p(phi), nphi, lam, int(bool(is_fast_diff)),
                                       _p(v), v.shape[0], _p(fo), _p(fv), len(fo) - 1,
                                       _p(ob), float(fov_override),
                                       out.ctypes.data_as(ctypes.c_void_p))
    if rc:
        raise RuntimeError("oracle diffraction failed: %d" % rc)
    return out


def params_vec(abs_=0.0, geo_cross_sec=1.0, beam_energy_out=1.0, ext_energy_out=1.0):
    p = np.zeros(18)
    p[0] = abs_
    p[8] = geo_cross_sec
    p[10] = beam_energy_out
    p[11] = ext_energy_out
    return p


def finalise(afb, afe, theta, phi, lam, params_in, scaling=False):
    """finalise (src/outputs_mod.f90:63-278) -> (mueller (nphi,ntheta,16) F-order,
    mueller_1d (ntheta,16) F-order, params (18,))."""
    theta = np.ascontiguousarray(theta, dtype=np.float64)
    phi = np.ascontiguousarray(phi, dtype=np.float64)
    nphi, nth = len(phi), len(theta)
    afb = np.asfortranarray(afb, dtype=np.complex128)
    afe = np.asfortranarray(afe, dtype=np.complex128)
    mu = np.zeros((nphi, nth, 16), order="F")
    mu1 = np.zeros((nth, 16), order="F")
    p = np.array(params_in, dtype=np.float64).copy()
    rc = lib().oracle_finalise_flat(afb.ctypes.data_as(ctypes.c_void_p),
                                    afe.ctypes.data_as(ctypes.c_void_p), nphi, nth,
                                    _p(theta), _p(phi), lam, int(bool(scaling)),
                                    mu.ctypes.data_as(ctypes.c_void_p),
                                    mu1.ctypes.data_as(ctypes.c_void_p), _p(p))
    if rc:
        raise RuntimeError("oracle finalise failed: %d" % rc)
    return mu, mu1, p


def simpne(x, y):
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.ascontiguousarray(y, dtype=np.float64)
    return lib().oracle_simpne(len(x), _p(x), _p(y), 1)


def ampl_to_mueller(ampl):
    ampl = np.asfortranarray(ampl, dtype=np.complex128)
    nb = ampl.shape[0] * ampl.shape[1]
    mu = np.zeros(ampl.shape[:2] + (16,), order="F")
    lib().oracle_ampl_to_mueller(nb, ampl.ctypes.data_as(ctypes.c_void_p),
                                 mu.ctypes.data_as(ctypes.c_void_p))
    return mu


class Totals:
    """summation + divide_by_num_orientations (src/outputs_mod.f90:407-471,13-43)."""

    def __init__(self, nphi, nth):
        self.mu = np.zeros((nphi, nth, 16), order="F")
        self.mu1 = np.zeros((nth, 16), order="F")
        self.p = np.zeros(18)
        self.n = 0

    def add(self, mu, mu1, p):
        mu = np.asfortranarray(mu)
        mu1 = np.asfortranarray(mu1)
        p = np.ascontiguousarray(p, dtype=np.float64)
        lib().oracle_summation_flat(mu.ctypes.data_as(ctypes.c_void_p),
                                    self.mu.ctypes.data_as(ctypes.c_void_p), mu.size,
                                    mu1.ctypes.data_as(ctypes.c_void_p),
                                    self.mu1.ctypes.data_as(ctypes.c_void_p), mu1.size,
                                    _p(p), _p(self.p))
        self.n += 1

    def averaged(self):
        mu, mu1, p = self.mu.copy(order="F"), self.mu1.copy(order="F"), self.p.copy()
        lib().oracle_divide_flat(mu.ctypes.data_as(ctypes.c_void_p), mu.size,
                                 mu1.ctypes.data_as(ctypes.c_void_p), mu1.size, _p(p), self.n)
        return mu, mu1, p
