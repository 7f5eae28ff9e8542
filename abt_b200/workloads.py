"""Seeded synthetic beam lists with the shapes of the benchmark configurations.

The reference's own beam lists come from its Fortran tracer (beam_loop_mod),
which is outside this package.  These generators stand in for them with the
sizes, facet geometry and value distributions the configurations name.
"""
import numpy as np

from ._lib import OUTBEAM_DTYPE
from .diff import make_angles, make_geometry

LAMBDA = 0.532


def _unit_vectors(rng, n):
    v = rng.normal(size=(n, 3))
    return v / np.linalg.norm(v, axis=1, keepdims=True)


def _perp_unit(rng, p):
    """A random unit vector orthogonal to each row of p."""
    r = _unit_vectors(rng, len(p))
    r = r - (r * p).sum(1, keepdims=True) * p
    return r / np.linalg.norm(r, axis=1, keepdims=True)


def random_triangles(rng, n, centre_lo=0.0, centre_hi=100.0, edge_lo=0.3, edge_hi=1.5):
    """n triangles with centroids U([lo,hi]^3), side lengths U[edge_lo, edge_hi]
    (resampled until the triangle inequality holds with a margin), each in a
    random plane with a random in-plane rotation.  Returns (n, 3, 3) vertices."""
    sides = np.empty((n, 3))
    todo = np.arange(n)
    while len(todo):
        s = rng.uniform(edge_lo, edge_hi, size=(len(todo), 3))
        a, b, c = s[:, 0], s[:, 1], s[:, 2]
        ok = (a + b > c * 1.05) & (a + c > b * 1.05) & (b + c > a * 1.05)
        sides[todo[ok]] = s[ok]
        todo = todo[~ok]
    a, b, c = sides[:, 0], sides[:, 1], sides[:, 2]
    x2 = (a * a + b * b - c * c) / (2 * a)
    y2 = np.sqrt(np.maximum(b * b - x2 * x2, 1e-12))
    P = np.zeros((n, 3, 2))
    P[:, 1, 0] = a
    P[:, 2, 0] = x2
    P[:, 2, 1] = y2
    P -= P.mean(axis=1, keepdims=True)
    ang = rng.uniform(0, 2 * np.pi, size=n)
    ca, sa = np.cos(ang), np.sin(ang)
    Q = np.empty_like(P)
    Q[..., 0] = ca[:, None] * P[..., 0] - sa[:, None] * P[..., 1]
    Q[..., 1] = sa[:, None] * P[..., 0] + ca[:, None] * P[..., 1]
    nrm = _unit_vectors(rng, n)
    e1 = _perp_unit(rng, nrm)
    e2 = np.cross(nrm, e1)
    centre = rng.uniform(centre_lo, centre_hi, size=(n, 3))
    return centre[:, None, :] + Q[..., 0:1] * e1[:, None, :] + Q[..., 1:2] * e2[:, None, :]


def _log_normal_amplitudes(rng, n, mu=-2.0, sigma=1.5):
    mag = np.exp(rng.normal(mu, sigma, size=(n, 4)))
    ph = rng.uniform(0, 2 * np.pi, size=(n, 4))
    z = mag * np.exp(1j * ph)
    out = np.empty((n, 8))
    out[:, 0::2] = z.real
    out[:, 1::2] = z.imag
    return out


def synthetic_beam_list(n_beams=2000, facets_per_beam=100, seed=2024, cube=100.0,
                        edge_lo=0.3, edge_hi=1.5, lam=LAMBDA):
    """Synthetic beam list fed straight to diffraction (the precision-study
    configuration): n_beams beams of facets_per_beam triangles; per beam a
    propagation direction uniform on the sphere, a perpendicular e-field
    direction and a 2x2 complex amplitude with log-normal magnitudes
    (mu=-2, sigma=1.5) and uniform phases, copied to the beam's facets.
    Returns (geometry, beam outbeams, external-diffraction outbeams (empty))."""
    rng = np.random.default_rng(seed)
    n = n_beams * facets_per_beam
    tri = random_triangles(rng, n, 0.0, cube, edge_lo, edge_hi)
    verts = tri.reshape(-1, 3)
    geometry = dict(verts=verts, face_off=np.arange(0, 3 * n + 1, 3, dtype=np.int64),
                    face_vi=np.arange(1, 3 * n + 1, dtype=np.int64))
    prop = _unit_vectors(rng, n_beams)
    vk7 = _perp_unit(rng, prop)
    ampl = _log_normal_amplitudes(rng, n_beams)
    beam = np.zeros(n, dtype=OUTBEAM_DTYPE)
    idx = np.repeat(np.arange(n_beams), facets_per_beam)
    beam["ampl"] = ampl[idx]
    beam["vk7"] = vk7[idx]
    beam["prop_out"] = prop[idx]
    # fov = 8 lambda / d over the beam's total area (src/beam_loop_mod.f90:2765-2767)
    e1 = tri[:, 1] - tri[:, 0]
    e2 = tri[:, 2] - tri[:, 0]
    area = 0.5 * np.linalg.norm(np.cross(e1, e2), axis=1)
    beam_area = np.bincount(idx, weights=area, minlength=n_beams)
    d = 2 * np.sqrt(beam_area / np.pi)
    beam["fov"] = (lam / d * 8)[idx]
    beam["fi"] = np.arange(1, n + 1)
    return geometry, beam, np.zeros(0, dtype=OUTBEAM_DTYPE)


def grid_precision_study():
    """theta 0..180 step 0.25 (721) x phi 0..359 step 1 (360)."""
    return make_angles([0, 180], [0.25]), make_angles([0, 359], [1])


def grid_small():
    """theta 0..180 step 1 (181) x phi 0..358 step 2 (180)."""
    return make_angles([0, 180], [1]), make_angles([0, 358], [2])


def euler_rotation(alpha, beta, gamma):
    """z-y-z Euler rotation matrix."""
    ca, sa, cb, sb, cg, sg = (np.cos(alpha), np.sin(alpha), np.cos(beta), np.sin(beta),
                              np.cos(gamma), np.sin(gamma))
    Rz1 = np.array([[ca, -sa, 0], [sa, ca, 0], [0, 0, 1]])
    Ry = np.array([[cb, 0, sb], [0, 1, 0], [-sb, 0, cb]])
    Rz2 = np.array([[cg, -sg, 0], [sg, cg, 0], [0, 0, 1]])
    return Rz1 @ Ry @ Rz2


def hex_prism(radius, length, n_side=4, n_len=8, roughness=0.0, seed=0):
    """Triangulated hexagonal prism centred at the origin (axis z): each
    rectangular side is an n_side x n_len grid of quads split in two
    triangles, each basal face a fan of 6 x n_side^2 triangles.  Optional
    Gaussian vertex roughness (standard deviation `roughness`) perturbs the
    interior vertices of every face along the face normal.  Faces are
    counter-clockwise seen from outside.  Returns a geometry dict whose
    "apertures" entry gives each triangle's parent face (1-6 the sides, 7 the
    top, 8 the bottom), the apertures of the reference's tracer."""
    rng = np.random.default_rng(seed)
    ang = np.arange(6) * np.pi / 3
    corners = np.stack([radius * np.cos(ang), radius * np.sin(ang)], 1)
    verts = []
    faces = []
    parent = []

    def add(p):
        verts.append(p)
        return len(verts)

    # side walls
    for k in range(6):
        a, b = corners[k], corners[(k + 1) % 6]
        nrm = np.array([a[0] + b[0], a[1] + b[1], 0.0])
        nrm /= np.linalg.norm(nrm)
        idx = np.zeros((n_side + 1, n_len + 1), dtype=np.int64)
        for i in range(n_side + 1):
            for j in range(n_len + 1):
                xy = a + (b - a) * i / n_side
                z = -length / 2 + length * j / n_len
                p = np.array([xy[0], xy[1], z])
                if roughness and 0 < i < n_side and 0 < j < n_len:
                    p = p + nrm * rng.normal(0, roughness)
                idx[i, j] = add(p)
        for i in range(n_side):
            for j in range(n_len):
                v00, v10, v01, v11 = idx[i, j], idx[i + 1, j], idx[i, j + 1], idx[i + 1, j + 1]
                faces.append([v00, v10, v11])
                faces.append([v00, v11, v01])
                parent += [k + 1, k + 1]
    # basal faces (fan of triangles subdivided per sector)
    for zsgn in (1.0, -1.0):
        z = zsgn * length / 2
        centre = add(np.array([0.0, 0.0, z]))
        for k in range(6):
            a, b = corners[k], corners[(k + 1) % 6]
            # sector subdivided into n_side^2 triangles
            rows = []
            for r in range(n_side + 1):
                row = []
                for c in range(r + 1):
                    if r == 0:
                        row.append(centre)
                        continue
                    pa = a * r / n_side
                    pb = b * r / n_side
                    xy = pa + (pb - pa) * (c / r)
                    p = np.array([xy[0], xy[1], z])
                    if roughness and 0 < r < n_side:
                        p = p + np.array([0, 0, zsgn]) * rng.normal(0, roughness)
                    row.append(add(p))
                rows.append(row)
            for r in range(n_side):
                for c in range(r + 1):
                    t1 = [rows[r][c], rows[r + 1][c], rows[r + 1][c + 1]]
                    if zsgn < 0:
                        t1 = t1[::-1]
                    faces.append(t1)
                    parent.append(7 if zsgn > 0 else 8)
                    if c < r:
                        t2 = [rows[r][c], rows[r + 1][c + 1], rows[r][c + 1]]
                        if zsgn < 0:
                            t2 = t2[::-1]
                        faces.append(t2)
                        parent.append(7 if zsgn > 0 else 8)
    geo = make_geometry(np.array(verts), faces)
    geo["apertures"] = np.array(parent, dtype=np.int64)
    return geo


def facet_normals_areas(verts, face_off, face_vi):
    """Unit normals (from the first three vertices) and areas of triangular faces."""
    v = verts[face_vi - 1]
    tri = v.reshape(-1, 3, 3) if np.all(np.diff(face_off) == 3) else None
    if tri is None:
        raise ValueError("triangles only")
    n = np.cross(tri[:, 1] - tri[:, 0], tri[:, 2] - tri[:, 0])
    a = 0.5 * np.linalg.norm(n, axis=1)
    return n / (2 * a[:, None]), a


def ext_diffraction_outbeams(V, face_off, face_vi, lam=LAMBDA):
    """The external-diffraction outbeams the tracer emits for an incident beam
    along (0,0,-1): one per lit facet, prop_out = prop_in = the incidence
    direction, vk7 = normalise(n x prop), and ampl = the incident field
    (identity, e-perp (1,0,0); src/input_mod.f90:2241-2258) times the path
    phase exp(i k dist), dist = the incident plane's z minus the facet
    centroid's z (src/beam_loop_mod.f90:2602, :530), rotated from the incident
    e-perp into vk7 by the normalised rotation of get_rot_matrix
    (src/beam_loop_mod.f90:525-533, :2611-2638).  The incident plane is put at
    the highest vertex; another choice changes every outbeam by one common
    phase.  Returns (ext outbeams, lit facet indices, cos of incidence)."""
    nrm, area = facet_normals_areas(V, face_off, face_vi)
    inc = np.array([0.0, 0.0, -1.0])
    cosi = -(nrm @ inc)
    lit = np.nonzero(cosi > 1e-6)[0]
    ext = np.zeros(len(lit), dtype=OUTBEAM_DTYPE)
    ext["fi"] = lit + 1
    ext["prop_out"] = inc
    vk7 = np.cross(nrm[lit], inc)
    vn = np.linalg.norm(vk7, axis=1)
    e1 = np.array([1.0, 0.0, 0.0])
    # a facet facing the incidence head-on has no scattering plane of its own
    vk7 = np.where(vn[:, None] > 1e-12, vk7 / np.maximum(vn, 1e-300)[:, None], e1)
    ext["vk7"] = vk7
    evo2 = np.cross(inc, e1)
    c = vk7 @ e1
    s = vk7 @ evo2
    nrm_rot = np.sqrt(np.abs(c * c + s * s))
    r11, r12, r21, r22 = c / nrm_rot, -s / nrm_rot, s / nrm_rot, c / nrm_rot
    mid_z = V[face_vi - 1].reshape(-1, 3, 3)[lit, :, 2].mean(axis=1)
    k = 2.0 * float(np.float32(np.pi)) / lam
    ph = np.exp(1j * k * (V[:, 2].max() - mid_z))
    amp = np.stack([r11 * ph, r21 * ph, r12 * ph, r22 * ph], axis=1)  # (1,1),(2,1),(1,2),(2,2)
    ext["ampl"][:, 0::2] = amp.real
    ext["ampl"][:, 1::2] = amp.imag
    ext["fov"] = np.pi / 2
    return ext, lit, cosi


def standin_orientation(geometry, R, rng, lam=LAMBDA, n_internal=(0, 6), rbi=1.31):
    """A beam list standing in for one orientation of the tracer: the particle
    rotated by R, lit from +z along (0,0,-1).  External diffraction: one
    outbeam per lit facet along the incidence direction, built as the tracer
    builds them (ext_diffraction_outbeams).  Beam outbeams: every facet
    emits 0..n reflected/refracted outgoing beams with Fresnel-like scalar
    amplitudes (uneven counts per orientation, like the tracer's output).
    Returns (rotated vertices, beam, ext, params_in record)."""
    V = geometry["verts"] @ R.T
    fo, fv = geometry["face_off"], geometry["face_vi"]
    nrm, area = facet_normals_areas(V, fo, fv)
    ext, lit, cosi = ext_diffraction_outbeams(V, fo, fv, lam)
    # outgoing beams: per facet a random number of outgoing directions
    nf = len(area)
    counts = rng.integers(n_internal[0], n_internal[1] + 1, size=nf)
    idx = np.repeat(np.arange(nf), counts)
    m = len(idx)
    beam = np.zeros(m, dtype=OUTBEAM_DTYPE)
    beam["fi"] = idx + 1
    # outgoing directions: random in the outward hemisphere of the facet
    d = _unit_vectors(rng, m)
    d = np.where(((d * nrm[idx]).sum(1) < 0)[:, None], -d, d)
    beam["prop_out"] = d
    beam["vk7"] = _perp_unit(rng, d)
    r = ((rbi - 1) / (rbi + 1)) ** 2
    mag = np.sqrt(r) * np.exp(rng.normal(-1.0, 0.8, size=(m, 4)))
    ph = rng.uniform(0, 2 * np.pi, size=(m, 4))
    z = mag * np.exp(1j * ph)
    beam["ampl"][:, 0::2] = z.real
    beam["ampl"][:, 1::2] = z.imag
    beam["fov"] = 8 * lam / 10.0
    geo = float((area[lit] * cosi[lit]).sum())
    return V, beam, ext, geo


def uniform_euler(rng, n):
    """n (alpha, beta, gamma) triples uniform on SO(3): alpha = 2 pi u1,
    beta = acos(1 - 2 u2), gamma = 2 pi u3 (the law of
    src/input_mod.f90:1848-1855)."""
    u = rng.uniform(size=(n, 3))
    return np.stack([2 * np.pi * u[:, 0], np.arccos(1 - 2 * u[:, 1]), 2 * np.pi * u[:, 2]], 1)


def grid_orientation_average():
    """361 theta x 180 phi (-theta 0 0.5 180, -phi 0 2 358)."""
    return make_angles([0, 180], [0.5]), make_angles([0, 358], [2])


def rough_column_orientations(n_orient=1024, seed=3, radius=10.0, length=20.0, roughness=0.1,
                              n_side=6, n_len=12, m_range=(2, 20), lam=LAMBDA):
    """Stand-in beam lists of the orientation-averaging workload: a Gaussian-rough
    hexagonal column (radius 10 um, length 20 um, sigma 0.1 um, 1296 triangles),
    n_orient orientations uniform on SO(3), and per orientation a maximum number
    m of outgoing beams per facet drawn from m_range, so the outgoing facet count
    is uneven across orientations (about 2,000 to 14,000).
    Returns (geometry, [V], [beam], [ext], params_in)."""
    from .diff import params as _params
    rng = np.random.default_rng(seed)
    geo = hex_prism(radius, length, n_side=n_side, n_len=n_len, roughness=roughness, seed=seed)
    eul = uniform_euler(rng, n_orient)
    Vs, beams, exts = [], [], []
    pin = np.zeros(n_orient, dtype=_params().dtype)
    for i, (a, b, c) in enumerate(eul):
        m = int(rng.integers(m_range[0], m_range[1] + 1))
        V, beam, ext, gcs = standin_orientation(geo, euler_rotation(a, b, c), rng, lam=lam,
                                                n_internal=(0, m))
        Vs.append(V)
        beams.append(beam)
        exts.append(ext)
        pin[i] = _params(geo_cross_sec=gcs, beam_energy_out=1.0, ext_energy_out=1.0)
    return geo, Vs, beams, exts, pin
