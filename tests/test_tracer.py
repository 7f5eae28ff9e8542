"""The near-field tracer (host, FP64; no GPU needed).

The reference's tracer cannot be built here (Fortran), so these checks use
what the physics and the reference's own energy bookkeeping fix:
  * on a convex particle with no recursion beyond the first interaction, the
    outbeams are the Fresnel-reflected incident field and the external-
    diffraction records are the incident field on the lit faces -- both
    restated independently below in numpy and compared to 1e-12;
  * up to the light refracted in, propagated once inside and refracted out
    (visibility buckets, internal Fresnel, thresholds and list order
    included), a second independent numpy restatement gives the same lists;
  * the external-diffraction energy equals the illuminated geometric cross
    section, and the beam energy (plus absorption) conserves the incident
    energy to the few per cent the reference's energy checks report;
  * the lists do not depend on the number of host threads.
"""
import os
import subprocess
import sys

import numpy as np
import pytest

from abt_b200 import PbtError, _lib, workloads as W
from abt_b200 import tracer as T
from abt_b200.diff import PI_REF

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LAM, RBI = 0.532, 1.31


@pytest.fixture(scope="module")
def smooth():
    geo = W.hex_prism(5.0, 10.0, n_side=2, n_len=3, roughness=0.0)
    return geo, T.Particle(geo, geo["apertures"])


@pytest.fixture(scope="module")
def rough():
    geo = W.hex_prism(10.0, 20.0, n_side=6, n_len=12, roughness=0.1, seed=3)
    return geo, T.Particle(geo, geo["apertures"])


def _faces(V, geo):
    tri = V[geo["face_vi"] - 1].reshape(-1, 3, 3)
    n = np.cross(tri[:, 1] - tri[:, 0], tri[:, 2] - tri[:, 1])
    n /= np.linalg.norm(n, axis=1, keepdims=True)
    mid = tri.mean(axis=1)
    c = tri - mid[:, None, :]
    area = 0.5 * sum(np.linalg.norm(np.cross(c[:, k], c[:, (k + 1) % 3]), axis=1)
                     for k in range(3))
    return n, mid, area


def _ampl(z):
    """(n, 2, 2) complex from the records' ampl (column-major re/im)."""
    a = z[:, 0::2] + 1j * z[:, 1::2]
    return np.stack([np.stack([a[:, 0], a[:, 2]], 1), np.stack([a[:, 1], a[:, 3]], 1)], 1)


def test_particle_is_centred(rough):
    geo, P = rough
    assert P.napertures == 8
    V = P.geometry["verts"]
    assert np.allclose(V + P.com, geo["verts"], atol=1e-12)
    _, mid, area = _faces(V, geo)
    com = (mid * area[:, None]).sum(0) / area.sum()
    assert np.abs(com).max() < 1e-9


@pytest.mark.parametrize("euler", [(0.4, 0.9, 1.3), (2.1, 2.3, 0.2), (5.0, 1.2, 4.1)])
def test_first_interaction_matches_independent_restatement(smooth, euler):
    """rec = 0: every outbeam is the first external reflection.  Restated here
    from the physics: lit faces face the incidence (aperture normal z >= 0.01),
    path phase from the incident plane z = 1000, e-perp rotation into
    vk7 = n x prop, Fresnel r_p, r_s with real Snell's law, mirror direction,
    fov = 8 lambda / d of the lit aperture area."""
    geo, P = smooth
    V, beam, ext, pin, en = T.trace(P, np.array(euler), LAM, RBI, rec=0)
    n, mid, area = _faces(V, geo)
    ap = geo["apertures"] - 1
    apn = np.zeros((8, 3))
    np.add.at(apn, ap, n)
    apn /= np.linalg.norm(apn, axis=1, keepdims=True)
    lit = np.nonzero(apn[ap, 2] >= np.float32(0.01))[0]
    inc = np.array([0.0, 0.0, -1.0])
    k = 2 * PI_REF / LAM
    vk7 = np.cross(n[lit], inc)
    vk7 /= np.linalg.norm(vk7, axis=1, keepdims=True)
    evo2 = np.cross(inc, [1.0, 0.0, 0.0])
    c, s = vk7[:, 0], vk7 @ evo2
    rot = np.stack([np.stack([c, -s], 1), np.stack([s, c], 1)], 1) / np.sqrt(np.abs(c * c + s * s))[:, None, None]
    A = rot * np.exp(1j * k * (1000.0 - mid[lit, 2]))[:, None, None]
    # external diffraction: the incident field on every lit face, in face order
    assert np.array_equal(ext["fi"], lit + 1)
    assert np.allclose(_ampl(ext["ampl"]), A, rtol=0, atol=1e-12)
    assert np.allclose(ext["vk7"], vk7, atol=1e-12)
    assert np.all(ext["prop_out"] == inc)
    # first reflections, aperture by aperture
    ti = np.arccos(apn[ap[lit], 2])
    tt = np.arcsin(np.sin(ti) / RBI)
    rs = (np.cos(ti) - RBI * np.cos(tt)) / (np.cos(ti) + RBI * np.cos(tt))
    rp = (RBI * np.cos(ti) - np.cos(tt)) / (np.cos(tt) + RBI * np.cos(ti))
    R = np.stack([rp, rs], 1)[:, :, None] * A
    a3 = apn[ap[lit]]
    mirror = np.stack([2 * a3[:, 2] * a3[:, 0], 2 * a3[:, 2] * a3[:, 1],
                       -1 + 2 * a3[:, 2] * a3[:, 2]], 1)
    order, fov = [], []
    for a in range(8):
        sel = np.nonzero(ap[lit] == a)[0]
        if area[lit[sel]].sum() > 0.1:
            order.extend(sel)
            fov += [8 * LAM / (2 * np.sqrt(area[lit[sel]].sum() / PI_REF))] * len(sel)
    order = np.array(order)
    assert len(beam) == len(order) > 0
    assert np.array_equal(beam["fi"], lit[order] + 1)
    assert np.allclose(_ampl(beam["ampl"]), R[order], rtol=0, atol=1e-12)
    assert np.allclose(beam["prop_out"], mirror[order], atol=1e-12)
    assert np.allclose(beam["vk7"], vk7[order], atol=1e-12)
    assert np.allclose(beam["fov"], fov, rtol=1e-12)
    # cross sections of this orientation
    geo_cs = (area[lit] * n[lit, 2]).sum()
    assert pin["geo_cross_sec"] == pytest.approx(geo_cs, rel=1e-12)
    assert en["ext_energy_out"] == pytest.approx(geo_cs, rel=1e-12)


@pytest.mark.parametrize("euler", [(0.3, 0.7, 0.2), (1.0, 2.0, 0.5), (4.4, 1.57, 2.9)])
def test_energy_is_conserved(rough, euler):
    geo, P = rough
    V, beam, ext, pin, en = T.trace(P, np.array(euler), LAM, RBI)
    gcs = en["geo_cross_sec"]
    assert en["ext_energy_out"] == pytest.approx(gcs, rel=1e-12)
    assert 0.97 < en["beam_energy_out"] / gcs < 1.03
    assert en["abs"] == 0.0 and len(beam) > len(ext) > 0
    assert np.all((beam["fi"] >= 1) & (beam["fi"] <= len(geo["face_off"]) - 1))
    assert np.allclose(np.linalg.norm(beam["prop_out"], axis=1), 1.0, atol=1e-12)
    # outgoing beams leave through the face they are emitted from
    n, _, _ = _faces(V, geo)
    assert np.all((beam["prop_out"] * n[beam["fi"] - 1]).sum(1) > -0.2)
    # absorbing: what is not absorbed leaves
    _, beam2, _, pin2, en2 = T.trace(P, np.array(euler), LAM, RBI, ibi=1e-3)
    assert en2["abs"] > 0 and pin2["abs"] == en2["abs"]
    assert 0.97 < (en2["beam_energy_out"] + en2["abs"]) / gcs < 1.03
    assert en2["beam_energy_out"] < en["beam_energy_out"]


def test_recursion_limit_and_thresholds(rough):
    geo, P = rough
    e = np.array([0.5, 1.1, 0.3])
    counts = [T.trace(P, e, LAM, RBI, rec=r)[4]["nbeams"] for r in (0, 2, 4, 8)]
    assert counts[0] < counts[1] < counts[2] < counts[3]
    _, beam, ext, _, en = T.trace(P, e, LAM, RBI, thresh_area=1e9)
    assert len(beam) == 0 and en["nbeams"] == 0 and len(ext) > 0


def test_same_lists_on_one_thread(rough):
    """The lists are built in beam order whatever the number of host threads."""
    geo, P = rough
    e = np.array([1.7, 0.8, 2.2])
    V, beam, ext, pin, en = T.trace(P, e, LAM, RBI, ibi=1e-3)
    code = ("import numpy as np, sys; sys.path.insert(0, %r)\n"
            "from abt_b200 import workloads as W, tracer as T\n"
            "g = W.hex_prism(10.0, 20.0, n_side=6, n_len=12, roughness=0.1, seed=3)\n"
            "P = T.Particle(g, g['apertures'])\n"
            "V, b, x, p, e = T.trace(P, np.array([1.7, 0.8, 2.2]), 0.532, 1.31, ibi=1e-3)\n"
            "sys.stdout.buffer.write(b.tobytes() + x.tobytes() + V.tobytes() + e.tobytes())\n"
            % ROOT)
    env = dict(os.environ, OMP_NUM_THREADS="1")
    out = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True,
                         check=True).stdout
    assert out == beam.tobytes() + ext.tobytes() + V.tobytes() + en.tobytes()


def test_euler_helpers():
    e = T.euler_from_degrees(30, 0, 10)
    assert e[1] == 1e-4 * PI_REF / 180.0 and e[0] == 30 * PI_REF / 180.0
    m = T.multi_euler(0.25, 0.5, 0.75)
    assert m[0] == 2 * PI_REF * 0.25 and m[1] == np.arccos(0.0)


def test_axis_aligned_orientation(smooth):
    """A face normal along the incidence leaves e-perp = n x prop undefined:
    NaN amplitudes, on which the reference stops (src/beam_loop_mod.f90:1570);
    the 'euler' method's lift of beta to 1e-4 degree avoids it."""
    geo, P = smooth
    with pytest.raises(PbtError, match="NaN amplitude") as e:
        T.trace(P, np.zeros(3), LAM, RBI)
    assert e.value.status == _lib.PBT_ESTATE
    V, beam, ext, pin, en = T.trace(P, T.euler_from_degrees(0, 0, 0), LAM, RBI)
    assert np.isfinite(beam["ampl"]).all() and np.isfinite(ext["ampl"]).all() and len(beam) > 0


def test_bad_input_is_rejected(rough):
    geo, P = rough
    quad = dict(verts=np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0.]]),
                face_off=np.array([0, 4]), face_vi=np.array([1, 2, 3, 4]))
    with pytest.raises(PbtError, match="triangles"):
        T.Particle(quad)
    with pytest.raises(PbtError, match="aperture"):
        T.Particle(geo, np.zeros(len(geo["face_off"]) - 1, dtype=np.int64))
    bad = dict(geo, verts=geo["verts"].copy())
    bad["verts"][3, 1] = np.nan
    with pytest.raises(PbtError, match="not finite"):
        T.Particle(bad)
    with pytest.raises(PbtError) as e:
        T.trace(P, np.array([0.1, 0.2, 0.3]), LAM, 0.9)
    assert e.value.status == _lib.PBT_EINVAL
    with pytest.raises(PbtError):
        T.trace(P, np.array([0.1, np.inf, 0.3]), LAM, RBI)


def test_batch_equals_single_orientation_traces(rough):
    geo, P = rough
    eul = np.array([T.multi_euler(*u) for u in np.random.default_rng(5).uniform(size=(6, 3))])
    Vs, beams, exts, pins, ens = T.trace_batch(P, eul, LAM, RBI, ibi=1e-4)
    for i, e in enumerate(eul):
        V, beam, ext, pin, en = T.trace(P, e, LAM, RBI, ibi=1e-4)
        assert Vs[i].tobytes() == V.tobytes()
        assert beams[i].tobytes() == beam.tobytes() and exts[i].tobytes() == ext.tobytes()
        assert pins[i].tobytes() == pin.tobytes() and ens[i].tobytes() == en.tobytes()
    bad = eul.copy()
    bad[4, 2] = np.nan
    with pytest.raises(PbtError, match="orientation 5"):
        T.trace_batch(P, bad, LAM, RBI)
    assert T.trace_batch(P, np.zeros((0, 3)), LAM, RBI)[0] == []


# ---------------------------------------------------------------- second order
# An independent numpy restatement of the tracer on a convex particle up to the
# light refracted in, propagated once inside and refracted out (rec = 2,
# refl = 0: no chains of total internal reflection), following the reference's
# routines: recursion_inc, add_to_beam_tree_external, recursion_int with
# find_vis_int (its 4 x 4 bucket prefilter included), add_to_beam_tree_internal,
# recursion_ext and add_to_outbeam_tree (src/beam_loop_mod.f90).  On a convex
# particle no external beam meets the particle again.

F01 = float(np.float32(0.01))
F11 = float(np.float32(1.1))


def _snell(ti, m1, m2):
    """Angle of refraction from m1 into m2, complex Snell's law as Macke's
    form states it (src/beam_loop_mod.f90:342-383)."""
    m1, m2 = complex(m1), complex(m2)
    k1, k2 = m1.imag / m1.real, m2.imag / m2.real
    krel = (k2 - k1) / (1 + k1 * k2)
    nrel = m2.real / m1.real * (1 + k1 * k2) / (1 + k1 * k1)
    ref1, ref2 = nrel * nrel, krel * krel
    ref3 = (1 + ref2) ** 2
    ref6 = ref1 * ref3 / (1 + krel * k2) ** 2
    st2 = np.sin(ti) ** 2
    ref4 = 1 - (1 - ref2) / ref1 / ref3 * st2
    ref5 = 2 * krel / ref1 / ref3 * st2
    q2 = np.sqrt(ref4 * ref4 + ref5 * ref5)
    g = np.arccos(ref4 / q2) / 2
    ref7 = (np.cos(g) - k2 * np.sin(g)) ** 2
    return np.arcsin(np.sin(ti) / np.sqrt(st2 + ref6 * q2 * ref7))


def _trans_prop(ti, tt, prop, norm):
    if tt < float(np.float32(1e-5)):
        a, b = 0.25, 0.75
    else:
        a, b = np.sin(tt - ti) / np.sin(ti), np.sin(PI_REF - tt) / np.sin(ti)
    p = b * prop - a * norm
    return p / np.linalg.norm(p)


def _rot2(vk7, ev1, ev3):
    c = vk7 @ ev1
    evo2 = np.cross(ev3, ev1)
    evo2 /= np.linalg.norm(evo2)
    s = vk7 @ evo2
    return np.array([[c, -s], [s, c]]) / np.sqrt(abs(c * c + s * s))


def _beam_frame(prop):
    t1 = 2 * PI_REF - np.arctan2(prop[1], prop[0])
    r1 = np.array([[np.cos(t1), -np.sin(t1), 0], [np.sin(t1), np.cos(t1), 0], [0, 0, 1.0]])
    t = r1 @ prop
    t2 = np.arccos(-(t / np.linalg.norm(t))[2])
    r2 = np.array([[np.cos(t2), 0, np.sin(t2)], [0, 1.0, 0], [-np.sin(t2), 0, np.cos(t2)]])
    return r2 @ r1


def _buckets(vx, vy, px, py):
    """Index of the nearest of the 4 x 4 bucket centres (first on ties)."""
    xs = F11 * (vx.min() + (vx.max() - vx.min()) / 4 * np.arange(5))
    ys = F11 * (vy.min() + (vy.max() - vy.min()) / 4 * np.arange(5))
    cx = (xs[:4] + xs[:4] + xs[1:] + xs[1:]) / 4
    cy = (ys[:4] + ys[1:] + ys[1:] + ys[:4]) / 4
    d = np.sqrt((cx[:, None, None] - px) ** 2 + (cy[None, :, None] - py) ** 2).reshape(16, -1)
    return np.argmin(d, axis=0)


def _second_order(V, geo, lam, rbi, ibi=0.0):
    tri_i = geo["face_vi"].reshape(-1, 3) - 1
    ap = geo["apertures"] - 1
    n, mid, area = _faces(V, geo)
    na = ap.max() + 1
    apn = np.zeros((na, 3))
    np.add.at(apn, ap, n)
    apn /= np.linalg.norm(apn, axis=1, keepdims=True)
    k = 2 * PI_REF / lam
    inc = np.array([0.0, 0.0, -1.0])
    ident = np.eye(2, dtype=complex)
    out = []

    mi = complex(rbi, ibi)  # refractive index

    def fresnel_outside(ti, tt):
        ci, ct = np.cos(ti), np.cos(tt)
        return np.diag([(mi * ci - ct) / (ct + mi * ci), (ci - mi * ct) / (ci + mi * ct)]), \
            np.diag([2 * ci / (ct + mi * ci), 2 * ci / (ci + mi * ct)])

    # incidence: lit faces (convex: no blockers), in face order
    lit = [i for i in range(len(ap)) if apn[ap[i], 2] >= F01]
    fo = []
    for i in lit:
        an = apn[ap[i]]
        vk7 = np.cross(n[i], inc)
        vk7 /= np.linalg.norm(vk7)
        A = _rot2(vk7, np.array([1.0, 0, 0]), inc) @ (ident * np.exp(1j * k * (1000.0 - mid[i, 2])))
        ti = np.arccos(an[2])
        fr, ft = fresnel_outside(ti, _snell(ti, 1.0, mi))
        tt = _snell(ti, 1.0, mi)
        fo.append(dict(fi=i, ap=ap[i], e_perp=vk7, a_ext=fr @ A, a_int=ft @ A,
                       p_int=_trans_prop(ti, tt, inc, -an),
                       p_ext=np.array([2 * an[2] * an[0], 2 * an[2] * an[1], -1 + 2 * an[2] ** 2])))
    # add_to_beam_tree_external: per aperture with enough area, internal then external
    tree = []
    for a in range(na):
        fa = [o for o in fo if o["ap"] == a]
        if sum(area[o["fi"]] for o in fa) > 0.1:
            tree.append(dict(int=True, rec=1, fields=[(o["fi"], o["a_int"], o["e_perp"], False) for o in fa],
                             prop=fa[-1]["p_int"]))
            tree.append(dict(int=False, rec=1, fields=[(o["fi"], o["a_ext"], o["e_perp"], True) for o in fa],
                             prop=fa[-1]["p_ext"]))

    def emit(beam):
        d = 2 * np.sqrt(sum(area[f[0]] for f in beam["fields"]) / PI_REF)
        for fi, a, e, outgoing in beam["fields"]:
            if outgoing:
                out.append((fi, a, e, beam["prop"], lam / d * 8))

    children = []
    for beam in tree:
        if not beam["int"]:
            emit(beam)  # convex: external beams leave the particle
            continue
        prop = beam["prop"]
        R = _beam_frame(prop)
        Vr, nr, midr, apr = V @ R.T, n @ R.T, mid @ R.T, apn @ R.T
        src = {f[0]: (j, f) for j, f in enumerate(beam["fields"])}
        bv = np.concatenate([tri_i[f[0]] for f in beam["fields"]])
        box = (Vr[bv, 0].min(), Vr[bv, 0].max(), Vr[bv, 1].min(), Vr[bv, 1].max())
        f3 = _buckets(Vr[:, 0], Vr[:, 1], midr[:, 0], midr[:, 1])
        vb = _buckets(Vr[:, 0], Vr[:, 1], Vr[:, 0], Vr[:, 1])
        fo = []
        for m in range(len(ap)):
            if not (box[0] <= midr[m, 0] <= box[1] and box[2] <= midr[m, 1] <= box[3]):
                continue
            if apr[ap[m], 2] > -F01:
                continue
            hit, best = None, None
            for j in range(len(ap)):
                if j == m or f3[m] not in vb[tri_i[j]] or midr[m, 2] > midr[j, 2]:
                    continue
                x, y = Vr[tri_i[j], 0], Vr[tri_i[j], 1]
                inside = all((midr[m, 0] - x[q]) * (y[(q + 1) % 3] - y[q])
                             + (midr[m, 1] - y[q]) * (x[q] - x[(q + 1) % 3]) <= 0 for q in range(3))
                if not inside:
                    continue
                if j in src:
                    if hit is None or midr[j, 2] < midr[src[hit][1][0], 2]:
                        hit, best = j, midr[j, 2] - midr[m, 2]
                elif ap[j] != ap[m]:
                    if hit is not None and midr[j, 2] > midr[src[hit][1][0], 2]:
                        continue
                    hit = None
                    break
            if hit is None:
                continue
            _, (_, a_src, e_src, _) = src[hit]
            vk7 = np.cross(-n[m], prop)
            vk7 /= np.linalg.norm(vk7)
            A = _rot2(vk7, e_src, prop) @ a_src * np.exp(1j * k * rbi * best)
            A = A * np.exp(-2 * k * ibi * np.sqrt(best))  # the reference's attenuation
            ti = np.arccos(-apr[ap[m], 2])
            ti_f = np.arccos(-nr[m, 2])
            tir = ti >= np.arcsin(1 / rbi)
            if tir:
                fr, ft, tt = -np.eye(2), np.zeros((2, 2)), 0.0
            else:
                tt = _snell(ti, mi, 1.0)
                ci, ct = np.cos(ti), np.cos(tt)
                fr = np.diag([(ci - mi * ct) / (mi * ct + ci), (mi * ci - ct) / (mi * ci + ct)])
                ft = np.diag([2 * mi * ci / (mi * ct + ci), 2 * mi * ci / (mi * ci + ct)])
            refl = fr @ A
            pr = 0.5 * np.sum(np.abs(refl) ** 2) * area[m] * np.cos(ti_f) * rbi
            ra = apr[ap[m]]
            p_int = R.T @ np.array([2 * ra[2] * ra[0], 2 * ra[2] * ra[1], -1 + 2 * ra[2] ** 2])
            p_ext = None if tir else _trans_prop(ti, tt, prop, n[m])
            fo.append(dict(fi=m, ap=ap[m], e_perp=vk7, a_int=refl, a_ext=ft @ A, tir=tir,
                           p_int=p_int, p_ext=p_ext, pr=pr))
        # add_to_beam_tree_internal (rec 1 < 2): area and energy thresholds
        for a in range(na):
            fa = [o for o in fo if o["ap"] == a]
            if not (sum(area[o["fi"]] for o in fa) > 0.1 and sum(o["pr"] for o in fa) > 1e-4):
                continue
            if not any(o["tir"] for o in fa):
                children.append(dict(int=False, fields=[(o["fi"], o["a_ext"], o["e_perp"], True) for o in fa],
                                     prop=fa[-1]["p_ext"]))
    for beam in children:
        emit(beam)  # convex: the refracted-out light leaves
    return out


@pytest.mark.parametrize("mesh,euler,ibi", [((2, 3), (0.4, 0.9, 1.3), 0.0),
                                            ((2, 3), (2.1, 2.3, 0.2), 0.0),
                                            ((4, 6), (1.1, 1.9, 2.6), 0.0),
                                            ((4, 6), (5.5, 0.6, 0.9), 0.0),
                                            ((4, 6), (1.1, 1.9, 2.6), 2e-3),
                                            ((2, 3), (0.4, 0.9, 1.3), 1e-2)])
def test_second_order_matches_independent_restatement(mesh, euler, ibi):
    geo = W.hex_prism(5.0, 10.0, n_side=mesh[0], n_len=mesh[1], roughness=0.0)
    P = T.Particle(geo, geo["apertures"])
    V, beam, ext, pin, en = T.trace(P, np.array(euler), LAM, RBI, ibi=ibi, rec=2, refl=0)
    n0 = len(T.trace(P, np.array(euler), LAM, RBI, ibi=ibi, rec=0)[1])
    assert len(beam) > n0  # refracted-out beams beyond the first reflections
    g = dict(P.geometry, apertures=geo["apertures"])
    ref = _second_order(V, g, LAM, RBI, ibi)
    assert len(beam) == len(ref) > 0
    assert np.array_equal(beam["fi"], [r[0] + 1 for r in ref])
    assert np.allclose(_ampl(beam["ampl"]), np.array([r[1] for r in ref]), rtol=0, atol=1e-11)
    assert np.allclose(beam["vk7"], [r[2] for r in ref], atol=1e-12)
    assert np.allclose(beam["prop_out"], [r[3] for r in ref], atol=1e-12)
    assert np.allclose(beam["fov"], [r[4] for r in ref], rtol=1e-12)


def test_c_caller(tmp_path):
    """abt_b200/examples/c_trace.c, built with gcc against the library: the
    tracer through the C ABI gives what the Python face gives for the same
    prism (24 triangles, 8 apertures)."""
    exe = str(tmp_path / "c_trace")
    libdir = os.path.join(ROOT, "abt_b200")
    subprocess.check_call(["gcc", "-O2", "-std=c99", "-I", os.path.join(ROOT, "include"),
                           os.path.join(libdir, "examples", "c_trace.c"), "-o", exe,
                           "-L", libdir, "-lpbt_b200", "-Wl,-rpath," + libdir, "-lm"])
    r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    tag, nbeam, next_, ratio = r.stdout.split()
    g = W.hex_prism(5.0, 10.0, n_side=1, n_len=1, roughness=0.0)
    _, beam, ext, _, en = T.trace(T.Particle(g, g["apertures"]), np.array([0.4, 0.9, 1.3]),
                                  LAM, RBI)
    assert tag == "ok" and int(nbeam) == len(beam) and int(next_) == len(ext)
    assert float(ratio) == pytest.approx(en["beam_energy_out"] / en["geo_cross_sec"], rel=1e-9)


_DIGEST = (
    "import hashlib, sys\n"
    "import numpy as np\n"
    "sys.path.insert(0, %r)\n"
    "from abt_b200 import tracer as T, workloads as W\n"
    "h = hashlib.sha256()\n"
    "for geo, ibi in ((W.hex_prism(10.0, 20.0, n_side=6, n_len=12, roughness=0.1, seed=3), 0.0),\n"
    "                 (W.hex_prism(30.0, 60.0, n_side=14, n_len=30, roughness=0.0, seed=5), 0.01)):\n"
    "    P = T.Particle(geo, geo['apertures'])\n"
    "    eul = W.uniform_euler(np.random.default_rng(41), 3)\n"
    "    Vs, beams, exts, pins, en = T.trace_batch(P, eul, 0.532, 1.31, ibi=ibi)\n"
    "    for a in list(Vs) + list(beams) + list(exts) + [pins]:\n"
    "        h.update(np.ascontiguousarray(a).tobytes())\n"
    "print(h.hexdigest())\n")


def test_visibility_walks_give_the_same_lists():
    """The visibility test walks the candidate blockers of a centroid either over
    its bucket's member list or, from 256 candidate faces, over the faces whose
    outline box meets the centroid's cell of a finer grid (in face order, filtered
    by bucket membership): the same faces in the same order, less those whose
    inside test fails.  Traced with only the member walk and with the grid from
    the first face on, a rough column and a 7,392-triangle column give the same
    lists bit for bit."""
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    code = _DIGEST % root
    out = []
    for grid_min in ("1000000000", "0"):
        env = dict(os.environ, PBT_TRACER_GRID_MIN=grid_min, OMP_NUM_THREADS="4")
        r = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True,
                           timeout=600)
        assert r.returncode == 0, r.stderr
        out.append(r.stdout.strip())
    assert out[0] == out[1] and len(out[0]) == 64
