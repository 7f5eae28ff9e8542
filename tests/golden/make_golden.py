"""Generates the frozen fixtures in tests/golden/ from the CPU oracle.

  python tests/golden/make_golden.py

The reference (Fortran) cannot run here and ships no far-field vectors, so
these fixtures freeze the oracle's output on seeded inputs: test_golden.py
checks that the oracle still reproduces them bit for bit and that the GPU
FP64 drop-in matches them to 1e-10.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from abt_b200 import workloads as W  # noqa: E402
from oracle import oracle as O  # noqa: E402

LAM = 0.532


def case_hex():
    """One stand-in orientation of a rough hexagonal column (Euler 30, 40, 10)."""
    rng = np.random.default_rng(101)
    geo = W.hex_prism(2.0, 4.0, n_side=2, n_len=2, roughness=0.05, seed=3)
    R = W.euler_rotation(*np.radians([30.0, 40.0, 10.0]))
    V, beam, ext, gcs = W.standin_orientation(geo, R, rng, n_internal=(0, 1))
    th = O.make_angles([0, 2, 10, 180], [0.5, 2, 10])
    ph = O.make_angles([0, 350], [10])
    return dict(verts=V, face_off=geo["face_off"], face_vi=geo["face_vi"], beam=beam, ext=ext,
                theta=th, phi=ph, lam=LAM, params_in=O.params_vec(0.01, gcs, 0.9 * gcs, gcs))


def case_synthetic():
    """Facets spread over a 100 um cube (far-field phases ~1e3 rad)."""
    geo, beam, ext = W.synthetic_beam_list(n_beams=3, facets_per_beam=4, seed=7)
    th = O.make_angles([0, 180], [5])
    ph = O.make_angles([0, 350], [10])
    return dict(verts=geo["verts"], face_off=geo["face_off"], face_vi=geo["face_vi"], beam=beam,
                ext=ext, theta=th, phi=ph, lam=LAM, params_in=O.params_vec(0.0, 1.0, 1.0, 1.0))


def solve(c):
    geo = dict(verts=c["verts"], face_off=c["face_off"], face_vi=c["face_vi"])
    afb, afe = O.diff_main(c["theta"], c["phi"], c["lam"], geo, c["beam"], c["ext"])
    mu, mu1, p = O.finalise(afb, afe, c["theta"], c["phi"], c["lam"], c["params_in"])
    return dict(ampl_far_beam=afb, ampl_far_ext_diff=afe, mueller=mu, mueller_1d=mu1, params=p)


def main():
    for name, fn in (("hex_orientation", case_hex), ("synthetic_cube", case_synthetic)):
        c = fn()
        out = solve(c)
        c["beam"] = c["beam"].view(np.uint8)
        c["ext"] = c["ext"].view(np.uint8)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **c, **out)
        print(name, {k: np.asarray(v).shape for k, v in out.items()})


if __name__ == "__main__":
    main()
