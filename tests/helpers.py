"""Error metrics and small inputs shared by the tests."""
import numpy as np

from abt_b200 import OUTBEAM_DTYPE, make_geometry


def rel_err(a, b):
    """Normwise relative error max|a-b| / max|b|."""
    a = np.asarray(a)
    b = np.asarray(b)
    den = np.max(np.abs(b))
    return float(np.max(np.abs(a - b)) / den) if den > 0 else float(np.max(np.abs(a - b)))


def mueller_rel_err(mu, mu_ref, thresh=1e-6):
    """Per-bin relative error of all 16 Mueller elements, normalised by the
    bin's reference M11, over bins whose M11 exceeds thresh * max(M11).
    |M_ij| <= M11 for a Mueller matrix of an amplitude matrix, so this is the
    relative error of every element against the bin's intensity."""
    m11 = mu_ref[..., 0]
    sel = m11 > thresh * m11.max()
    d = np.abs(mu - mu_ref)[sel].max(axis=-1)
    return float((d / m11[sel]).max())


def one_triangle(offset=(0.1, 0.2, 0.0), scale=1.0):
    verts = np.array([[0, 0, 0], [1.0, 0, 0], [0, 1.0, 0]]) * scale + np.array(offset)
    return make_geometry(verts, [[1, 2, 3]])


def outbeams(n, rng, nfaces, prop=None):
    ob = np.zeros(n, dtype=OUTBEAM_DTYPE)
    z = rng.normal(size=(n, 4)) + 1j * rng.normal(size=(n, 4))
    ob["ampl"][:, 0::2] = z.real
    ob["ampl"][:, 1::2] = z.imag
    if prop is None:
        p = rng.normal(size=(n, 3))
        p /= np.linalg.norm(p, axis=1, keepdims=True)
    else:
        p = np.tile(np.asarray(prop, float), (n, 1))
    ob["prop_out"] = p
    r = rng.normal(size=(n, 3))
    r -= (r * p).sum(1, keepdims=True) * p
    ob["vk7"] = r / np.linalg.norm(r, axis=1, keepdims=True)
    ob["fov"] = rng.uniform(0.05, 0.6, size=n)
    ob["fi"] = rng.integers(1, nfaces + 1, size=n)
    return ob


def mixed_polygon_geometry(rng):
    """Triangles, a quad and a hexagon, randomly placed and oriented."""
    verts = []
    faces = []
    for k in range(6):
        nv = [3, 3, 3, 4, 6, 5][k]
        c = rng.uniform(-10, 10, size=3)
        n = rng.normal(size=3)
        n /= np.linalg.norm(n)
        e1 = np.cross(n, rng.normal(size=3))
        e1 /= np.linalg.norm(e1)
        e2 = np.cross(n, e1)
        ang = np.sort(rng.uniform(0, 2 * np.pi, size=nv)) if nv == 3 else np.arange(nv) * 2 * np.pi / nv
        rad = rng.uniform(0.4, 1.5)
        f = []
        for a in ang:
            verts.append(c + rad * (np.cos(a) * e1 + np.sin(a) * e2))
            f.append(len(verts))
        faces.append(f)
    return make_geometry(np.array(verts), faces)
