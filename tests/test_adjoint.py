"""Gradients of a Mueller-matrix loss with respect to facet vertices and beam
amplitudes.

CPU: the FP64 lab-frame restatement (oracle/adjoint_ref.py) against the C
oracle's forward, and its autograd gradient against FP64 central finite
differences of the oracle (h = 1e-5 um).  GPU: the adjoint kernel
(pbt_diff_adjoint_c through abt_b200.autograd) against that FP64 gradient.
"""
import numpy as np
import pytest
import torch

import abt_b200
from abt_b200 import autograd as AG
from abt_b200 import workloads as W
from oracle import adjoint_ref as AR
from oracle import oracle as O

LAM = 0.532
H_FD = 1e-5  # um


def _case(seed=8, n_internal=(0, 1)):
    rng = np.random.default_rng(seed)
    th = abt_b200.make_angles([0, 180], [4])
    ph = abt_b200.make_angles([0, 352], [8])
    geo = W.hex_prism(2.0, 4.0, n_side=1, n_len=2, roughness=0.05, seed=2)
    R0 = W.euler_rotation(*rng.uniform(0, 2 * np.pi, size=3))
    V, beam, ext, _ = W.standin_orientation(geo, R0, rng, n_internal=n_internal)
    return th, ph, dict(geo, verts=V), beam, ext


def _amp22(a8):
    """(n,8) re/im of ampl(1,1),(2,1),(1,2),(2,2) -> (n,2,2) complex, differentiably."""
    z = torch.complex(a8[:, 0::2], a8[:, 1::2])
    return torch.stack([torch.stack([z[:, 0], z[:, 2]], -1), torch.stack([z[:, 1], z[:, 3]], -1)], -2)


def _ref_S(geo, beam, ext, th, ph, V, ab, ae):
    faces = torch.as_tensor((geo["face_vi"] - 1).reshape(-1, 3))
    return AR.forward(V, faces, beam["fi"] - 1, _amp22(ab), beam["prop_out"], beam["vk7"],
                      ext["fi"] - 1, _amp22(ae), ext["prop_out"], ext["vk7"], th, ph, LAM)


def _targets(m11, m12, seed=3):
    rng = np.random.default_rng(seed)
    t11 = m11 * np.exp(0.3 * rng.normal(size=m11.shape))
    t12 = t11 * (m12 / m11 + 0.1 * rng.normal(size=m11.shape))
    return t11, t12


def _oracle_m(geo, beam, ext, th, ph):
    afb, afe = O.diff_main(th, ph, LAM, geo, beam, ext)
    m11, m12 = AG.mueller11_12(torch.from_numpy(afb), torch.from_numpy(afe), LAM)
    return m11.numpy(), m12.numpy()


def _oracle_loss(geo, beam, ext, th, ph, t11, t12):
    m11, m12 = _oracle_m(geo, beam, ext, th, ph)
    return float(AG.mueller_loss(torch.from_numpy(m11), torch.from_numpy(m12),
                                 torch.from_numpy(t11), torch.from_numpy(t12), th))


def _ref_grads(geo, beam, ext, th, ph, t11, t12):
    """FP64 autograd gradient of the loss through the lab-frame restatement."""
    V = torch.tensor(geo["verts"], requires_grad=True)
    ab = torch.tensor(beam["ampl"], requires_grad=True)
    ae = torch.tensor(ext["ampl"], requires_grad=True)
    S = _ref_S(geo, beam, ext, th, ph, V, ab, ae)
    m11, m12 = AR.mueller11_12(S, 2 * O.PI_REF / LAM)
    shp = (len(th), len(ph))
    m11 = m11.reshape(shp).T
    m12 = m12.reshape(shp).T
    L = AG.mueller_loss(m11, m12, torch.from_numpy(t11), torch.from_numpy(t12), th)
    L.backward()
    return L.item(), V.grad.numpy(), ab.grad.numpy(), ae.grad.numpy()


def test_restatement_matches_oracle_forward():
    th, ph, geo, beam, ext = _case()
    afb, afe = O.diff_main(th, ph, LAM, geo, beam, ext)
    k = 2 * O.PI_REF / LAM
    X = O.far_field_bins(th, ph)
    rho = np.linalg.norm(X, axis=0).reshape(len(th), len(ph)).T
    ref = (afb + afe) * np.exp(-1j * k * rho)[:, :, None, None]          # (nphi,ntheta,2,2)
    with torch.no_grad():
        S = _ref_S(geo, beam, ext, th, ph, torch.tensor(geo["verts"]),
                   torch.tensor(beam["ampl"]), torch.tensor(ext["ampl"])).numpy()
    S = S.reshape(len(th), len(ph), 2, 2).transpose(1, 0, 2, 3)
    scale = np.abs(ref).max()
    # theta = 0 excluded: there the reference's own FP64 contour sum loses
    # ~1e-16/(qL)^2 to cancellation (q -> 0 along the incidence direction)
    err = np.abs(S - ref)[:, 1:].max() / scale
    assert err < 1e-8, err


def test_reference_gradient_matches_finite_differences():
    th, ph, geo, beam, ext = _case()
    m11, m12 = _oracle_m(geo, beam, ext, th, ph)
    t11, t12 = _targets(m11, m12)
    L, gV, gb, ge = _ref_grads(geo, beam, ext, th, ph, t11, t12)
    assert abs(L - _oracle_loss(geo, beam, ext, th, ph, t11, t12)) < 1e-9 * abs(L)
    rng = np.random.default_rng(5)
    used = np.unique(geo["face_vi"].reshape(-1, 3)[np.concatenate([beam["fi"], ext["fi"]]) - 1])
    picks = [(int(v) - 1, int(c)) for v in rng.choice(used, 4, replace=False) for c in range(3)]
    gscale = np.abs(gV).max()
    for vi, c in picks:
        fd = []
        for s in (1, -1):
            g2 = dict(geo, verts=geo["verts"].copy())
            g2["verts"][vi, c] += s * H_FD
            fd.append(_oracle_loss(g2, beam, ext, th, ph, t11, t12))
        d = (fd[0] - fd[1]) / (2 * H_FD)
        assert abs(d - gV[vi, c]) < 1e-4 * gscale + 1e-4 * abs(d), (vi, c, d, gV[vi, c])
    # amplitude gradient: one beam and one external record, one component each
    for recs, g, j in ((beam, gb, 0), (ext, ge, 1)):
        fd = []
        for s in (1, -1):
            r2 = recs.copy()
            r2["ampl"][j, 3] += s * 1e-6
            args = (r2, ext) if recs is beam else (beam, r2)
            fd.append(_oracle_loss(geo, *args, th, ph, t11, t12))
        d = (fd[0] - fd[1]) / 2e-6
        assert abs(d - g[j, 3]) < 1e-5 * np.abs(g).max() + 1e-5 * abs(d), (d, g[j, 3])


@pytest.mark.gpu
def test_adjoint_kernel_matches_fp64_gradient(ctx):
    th, ph, geo, beam, ext = _case()
    m11, m12 = _oracle_m(geo, beam, ext, th, ph)
    t11, t12 = _targets(m11, m12)
    L_ref, gV_ref, gb_ref, ge_ref = _ref_grads(geo, beam, ext, th, ph, t11, t12)
    for fast in (False, True):
        V = torch.tensor(geo["verts"], requires_grad=True)
        ab = torch.tensor(beam["ampl"], requires_grad=True)
        ae = torch.tensor(ext["ampl"], requires_grad=True)
        afb, afe = AG.far_field(ctx, V, ab, ae, beam, ext, geo, th, ph, LAM, is_fast_diff=fast)
        m11g, m12g = AG.mueller11_12(afb, afe, LAM)
        L = AG.mueller_loss(m11g, m12g, torch.from_numpy(t11), torch.from_numpy(t12), th)
        L.backward()
        if not fast:
            assert abs(L.item() - L_ref) < 1e-4 * abs(L_ref)
            # FP32 arithmetic: normwise relative error of the gradients
            for g, r in ((V.grad.numpy(), gV_ref), (ab.grad.numpy(), gb_ref),
                         (ae.grad.numpy(), ge_ref)):
                err = np.abs(g - r).max() / np.abs(r).max()
                assert err < 1e-4, err
        else:
            assert np.all(np.isfinite(V.grad.numpy()))


@pytest.mark.gpu
def test_adjoint_vjp_is_linear_in_cotangent(ctx):
    th, ph, geo, beam, ext = _case(seed=11)
    rng = np.random.default_rng(2)
    shape = (len(ph), len(th), 2, 2)
    g1 = rng.normal(size=shape) + 1j * rng.normal(size=shape)
    g2 = rng.normal(size=shape) + 1j * rng.normal(size=shape)
    z = np.zeros(shape, np.complex128)
    a = ctx.diff_adjoint(beam, ext, geo, th, ph, LAM, g1, z)
    b = ctx.diff_adjoint(beam, ext, geo, th, ph, LAM, z, g2)
    c = ctx.diff_adjoint(beam, ext, geo, th, ph, LAM, g1, g2)
    for x, y, s in zip(a, b, c):
        assert np.abs(x + y - s).max() <= 1e-4 * np.abs(s).max()


@pytest.mark.gpu
def test_adjoint_rejects_polygons(ctx):
    from tests.helpers import mixed_polygon_geometry, outbeams
    rng = np.random.default_rng(0)
    geo = mixed_polygon_geometry(rng)
    th = abt_b200.make_angles([0, 180], [10])
    ph = abt_b200.make_angles([0, 350], [10])
    beam = outbeams(4, rng, 6)
    beam["fi"] = [4, 4, 5, 5]
    shape = (len(ph), len(th), 2, 2)
    with pytest.raises(abt_b200.PbtError):
        ctx.diff_adjoint(beam, beam[:0], geo, th, ph, LAM, np.zeros(shape, complex),
                         np.zeros(shape, complex))
