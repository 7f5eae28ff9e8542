"""torch.autograd.Function over the C ABI: differentiable far-field amplitudes.

FarFieldFP32.apply(verts, beam_ampl, ext_ampl, ...) returns the amplitude
grids (ampl_far_beam, ampl_far_ext_diff) of one orientation from the FP32
far-field sum (pbt_diff_main_c, PBT_PREC_FP32); backward calls the adjoint
(pbt_diff_adjoint_c) with the grids' cotangents and returns the gradients
with respect to the vertex coordinates and the beam amplitude matrices.
The beam topology (which facets emit, their propagation and e-perp
directions) is held fixed, as it comes from the forward trace.

Tensors are CPU float64 (vertices (nverts,3); amplitudes (n,8) = re/im of
ampl(1,1),(2,1),(1,2),(2,2)); the grids are complex128 (nphi,ntheta,2,2).
"""
import numpy as np
import torch

from ._lib import OUTBEAM_DTYPE
from .diff import PI_REF


def _records(template, ampl):
    rec = np.array(template, dtype=OUTBEAM_DTYPE, copy=True)
    if len(rec):
        rec["ampl"] = ampl
    return np.ascontiguousarray(rec)


class FarFieldFP32(torch.autograd.Function):
    @staticmethod
    def forward(fctx, verts, beam_ampl, ext_ampl, lib_ctx, beam, ext, geometry, theta, phi, lam,
                is_fast_diff):
        geo = dict(geometry, verts=verts.detach().cpu().numpy().astype(np.float64))
        b = _records(beam, beam_ampl.detach().cpu().numpy())
        e = _records(ext, ext_ampl.detach().cpu().numpy())
        afb, afe = lib_ctx.diff_main(b, e, geo, theta, phi, lam, is_fast_diff=is_fast_diff,
                                     precision="fp32")
        fctx.saved = (lib_ctx, b, e, geo, theta, phi, lam, is_fast_diff)
        return torch.from_numpy(afb), torch.from_numpy(afe)

    @staticmethod
    def backward(fctx, gafb, gafe):
        lib_ctx, b, e, geo, theta, phi, lam, fast = fctx.saved
        shape = (len(phi), len(theta), 2, 2)
        ga = gafb.detach().cpu().numpy() if gafb is not None else np.zeros(shape, np.complex128)
        ge = gafe.detach().cpu().numpy() if gafe is not None else np.zeros(shape, np.complex128)
        gv, gb, gx = lib_ctx.diff_adjoint(b, e, geo, theta, phi, lam, ga, ge, is_fast_diff=fast)
        return (torch.from_numpy(np.ascontiguousarray(gv)), torch.from_numpy(gb),
                torch.from_numpy(gx), None, None, None, None, None, None, None, None)


def far_field(lib_ctx, verts, beam_ampl, ext_ampl, beam, ext, geometry, theta, phi, lam,
              is_fast_diff=False):
    """Differentiable (ampl_far_beam, ampl_far_ext_diff) of one orientation.

    verts (nverts,3), beam_ampl (nbeam,8), ext_ampl (next,8): float64 tensors;
    beam/ext: outbeam record arrays (their ampl fields are replaced);
    geometry: dict with face_off / face_vi (its verts are replaced)."""
    return FarFieldFP32.apply(verts, beam_ampl, ext_ampl, lib_ctx, beam, ext, geometry, theta, phi,
                              lam, bool(is_fast_diff))


def mueller11_12(afb, afe, lam):
    """M11 and M12 (nphi,ntheta) of the total amplitude scaled by the
    wavenumber, as finalise forms them (src/outputs_mod.f90:104-108, 489-497)."""
    a = (afb + afe) * (2 * PI_REF / lam)
    p = a.real ** 2 + a.imag ** 2
    m11 = 0.5 * (p[..., 0, 0] + p[..., 0, 1] + p[..., 1, 0] + p[..., 1, 1])
    m12 = 0.5 * (p[..., 0, 0] - p[..., 0, 1] + p[..., 1, 0] - p[..., 1, 1])
    return m11, m12


def mueller_loss(m11, m12, t11, t12, theta):
    """sin(theta)-weighted L2 of log M11 plus L2 of -M12/M11 against targets
    (all (nphi,ntheta))."""
    w = torch.sin(torch.as_tensor(theta, dtype=torch.float64))[None, :].expand_as(m11)
    wn = w / w.sum()
    return (wn * ((torch.log(m11) - torch.log(t11)) ** 2 + (-m12 / m11 + t12 / t11) ** 2)).sum()
