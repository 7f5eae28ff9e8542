"""FP64 CPU reference for gradients of a Mueller-matrix loss (test infrastructure only).

The far-field amplitude of triangular facets is restated in the laboratory
frame with torch float64 operations, so that torch's reverse-mode autograd
gives exact gradients with respect to the facet vertices and the beam
amplitude matrices.  The restatement follows the reference's diffraction
routine (src/diff_mod.f90:446-672) mathematically:

  * the aperture frame of get_rotation_matrix2 + the in-plane rotation
    (src/diff_mod.f90:200-289, 540-559) is the frame with z = -n,
    n = unit((v1-c) x (v2-c)), and x along the propagation direction's
    component in the aperture plane;
  * the contour integral (src/diff_mod.f90:291-444) of a triangle equals
    (2 i A_s / lambda) e^{iK} g[d1, d2, d3], g the second divided difference of
    e^{ix} at the vertex phases, A_s = -area;
  * karczewski (:124-198), the scattering-plane rotation (:620-660) and the
    amplitude product follow the reference's formulas;
  * the bin direction from the facet centre and the phase k|X - c| are exact.

The beam/propagation data (prop_out, vk7, the anti-parallel sign) are held
fixed: the beam topology comes from the forward trace.  forward() agrees with
the C oracle to ~1e-9 relative (tests/test_adjoint.py), and loss gradients
are checked against central finite differences of the oracle.
"""
import numpy as np
import torch

PI_REF = float(np.float32(3.14159265358979))
LIT_0_999999 = float(np.float32(0.999999))
LIT_0_999 = float(np.float32(0.999))
LIT_0_0001 = float(np.float32(0.0001))
FAR_R = 1e6


def _unit(v):
    return v / torch.linalg.norm(v, dim=-1, keepdim=True)


def _dd_exp(t1, t2, t3):
    """Second divided difference of e^{ix} at three points (float64 torch),
    stable for close points: evaluated as an integral over the simplex with a
    series when the spread is small."""
    lo = torch.minimum(torch.minimum(t1, t2), t3)
    hi = torch.maximum(torch.maximum(t1, t2), t3)
    mid = t1 + t2 + t3 - lo - hi
    D = hi - lo
    h1 = 0.5 * (mid - lo)
    h2 = 0.5 * (hi - mid)

    def sinc(h):
        small = h.abs() < 1e-3
        hs = torch.where(small, torch.ones_like(h), h)
        return torch.where(small, 1 - h * h / 6 + h ** 4 / 120, torch.sin(hs) / hs)

    e1 = torch.complex(torch.cos(lo + h1), torch.sin(lo + h1)) * sinc(h1)
    e2 = torch.complex(torch.cos(mid + h2), torch.sin(mid + h2)) * sinc(h2)
    Ds = torch.where(D < 1e-2, torch.ones_like(D), D)
    direct = 1j * (e2 - e1) / Ds
    ya, yc = lo - mid, hi - mid
    q = [torch.ones_like(ya)]
    for n in range(1, 9):
        q.append(yc * q[-1] + ya ** n)
    fact = [1, 1, 2, 6, 24, 120, 720, 5040, 40320, 362880, 3628800]
    ser = sum((1j ** (n + 2)) / fact[n + 2] * q[n] for n in range(9))
    ser = ser * torch.complex(torch.cos(mid), torch.sin(mid))
    return torch.where(D < 1e-2, ser, direct)


def forward(verts, faces, beam_fi, beam_ampl, beam_prop, beam_vk7, ext_fi, ext_ampl, ext_prop,
            ext_vk7, theta, phi, lam):
    """Total amplitude S = ampl_far_beam + ampl_far_ext_diff without the common
    phase e^{ik|X|} and without the wavenumber factor of finalise, as a
    complex (nbins, 2, 2) tensor in the reference's bin order (phi fastest).

    verts: (nverts,3) float64 tensor (may require grad); faces: (nfaces,3)
    int64 0-based; *_ampl: (n,2,2) complex128 tensor (may require grad);
    *_prop, *_vk7: (n,3) float64 arrays; theta, phi: radians."""
    dt = torch.float64
    k = 2 * PI_REF / lam
    th = torch.as_tensor(theta, dtype=dt)
    ph = torch.as_tensor(phi, dtype=dt)
    T, P = torch.meshgrid(th, ph, indexing="ij")
    X = torch.stack([FAR_R * torch.sin(T) * torch.cos(P), FAR_R * torch.sin(T) * torch.sin(P),
                     -(FAR_R * torch.cos(T))], -1).reshape(-1, 3)
    nphi = len(phi)
    theta_i = int(np.argmax(np.asarray(theta) > PI_REF / 180))
    iph = torch.arange(X.shape[0]) % nphi
    Xh = X.reshape(len(theta), nphi, 3)[theta_i][iph]
    cp = torch.cos(ph)[iph]
    sp = torch.sin(ph)[iph]
    Tm = torch.stack([torch.stack([-sp, -cp], -1), torch.stack([cp, -sp], -1)], -2)  # T(phi)
    total = torch.zeros(X.shape[0], 2, 2, dtype=torch.complex128)
    inc = torch.tensor([0.0, 0.0, -1.0], dtype=dt)
    for fi, ampl, prop, vk7 in ((beam_fi, beam_ampl, beam_prop, beam_vk7),
                                (ext_fi, ext_ampl, ext_prop, ext_vk7)):
        for j in range(len(fi)):
            f = faces[int(fi[j])]
            V = verts[f]
            c = V.mean(0)
            e = V - c
            N = torch.linalg.cross(e[0], e[1])
            n = N / torch.linalg.norm(N)
            z = -n
            p = torch.as_tensor(prop[j], dtype=dt)
            w = p - (p @ n) * n
            x = _unit(w)
            y = torch.linalg.cross(z, x)
            # anti-parallel flip (fixed by the forward trace)
            ep = np.cross(np.asarray(vk7[j]), np.asarray(prop[j]))
            ep = ep / np.linalg.norm(ep)
            sign = -1.0 if float(ep @ z.detach().numpy()) > LIT_0_0001 else 1.0
            area = 1.5 * torch.linalg.norm(N)
            d1 = X - c
            r1 = torch.linalg.norm(d1, dim=-1)
            kh = d1 / r1[:, None]
            K = k * r1
            q = k * (p - kh)
            th3 = q @ e.T + K[:, None]
            g = _dd_exp(th3[:, 0], th3[:, 1], th3[:, 2])
            F = (2j * (-area) / lam) * g  # includes e^{iK}
            # karczewski in the aperture frame
            kx, ky, kz = kh @ x, kh @ y, kh @ z
            kyc = torch.clamp(ky, -LIT_0_999999, LIT_0_999999)
            Kx, Ky, Kz = p @ x, p @ y, p @ z
            s = torch.sqrt(1 - kyc * kyc)
            m = torch.stack([-kx * kyc / s, s, -kyc * kz / s], -1)
            frac = torch.sqrt((1 - kyc * kyc) / (1 - Ky * Ky))
            a1m = -Kz * frac
            b2m = -kz / frac
            b1m = -kx * kyc / frac + Kx * Ky * frac
            D11 = 0.5 * (a1m + b2m)
            D12 = 0.5 * b1m
            inc2 = torch.stack([inc @ x, inc @ y, inc @ z])
            kap = torch.stack([kx, kyc, kz], -1)
            fwd = (kap @ inc2).abs() >= LIT_0_999
            if bool(fwd.any()):
                dh = Xh - c
                khh = dh / torch.linalg.norm(dh, dim=-1, keepdim=True)
                kh_ap = torch.stack([khh @ x, khh @ y, khh @ z], -1)
                qh = torch.where(fwd[:, None], kh_ap, kap)
            else:
                qh = kap
            hc = _unit(torch.linalg.cross(inc2.expand_as(qh), qh))
            evo2 = _unit(torch.linalg.cross(kap, m))
            pp = (hc * m).sum(-1)
            rr = (hc * evo2).sum(-1)
            A = pp * D11 - rr * (-D12)       # rot4 . D = [[A, B], [-B, A]]
            B = pp * D12 - rr * D11
            Mx = torch.stack([torch.stack([A, B], -1), torch.stack([-B, A], -1)], -2)
            a = sign * ampl[j]
            contrib = (Mx.to(torch.complex128) @ a) @ Tm.to(torch.complex128)
            total = total + F[:, None, None] * contrib
    # remove the common phase e^{ik|X|}
    Kc = k * torch.linalg.norm(X, dim=-1)
    return total * torch.complex(torch.cos(Kc), -torch.sin(Kc))[:, None, None]


def mueller11_12(S, k):
    """M11 and M12 of the amplitude S (nbins,2,2) scaled by k (finalise, src/outputs_mod.f90:104,489-497)."""
    a = S * k
    p = (a.real ** 2 + a.imag ** 2)
    m11 = 0.5 * (p[:, 0, 0] + p[:, 0, 1] + p[:, 1, 0] + p[:, 1, 1])
    m12 = 0.5 * (p[:, 0, 0] - p[:, 0, 1] + p[:, 1, 0] - p[:, 1, 1])
    return m11, m12


def loss_from_mueller(m11, m12, t11, t12, w):
    """Log-weighted L2 of S11 plus L2 of -S12/S11, weighted by w (sin theta)."""
    wn = w / w.sum()
    return (wn * ((torch.log(m11) - torch.log(t11)) ** 2 + (-m12 / m11 + t12 / t11) ** 2)).sum()
