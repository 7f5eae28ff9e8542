"""Beam-list files: write -> read round trip is bit-exact, damaged or foreign
files are refused, and (GPU) a replayed file gives the batch of the lists it
was written from."""
import numpy as np
import pytest

import abt_b200
from abt_b200 import PbtError
from abt_b200 import workloads as W
from abt_b200.beamlist import BeamListWriter, read_beam_list
from tests.helpers import mueller_rel_err

LAM = 0.532


def _lists(n_orient=5, seed=31):
    geo, Vs, beams, exts, pin = W.rough_column_orientations(n_orient, seed=seed, n_side=2,
                                                            n_len=4, m_range=(0, 3))
    th = abt_b200.make_angles([0, 180], [5])
    ph = abt_b200.make_angles([0, 350], [10])
    # an orientation with no outgoing beams at all is legal
    if n_orient > 1:
        beams[1] = beams[1][:0]
    return geo, Vs, beams, exts, pin, th, ph


def _write(path, geo, Vs, beams, exts, pin, th, ph):
    with BeamListWriter(path, th, ph, geo, LAM) as w:
        for V, b, e, p in zip(Vs, beams, exts, pin):
            w.add(b, e, V, p)


def test_round_trip_is_exact(tmp_path):
    geo, Vs, beams, exts, pin, th, ph = _lists()
    path = tmp_path / "orient.pbtb"
    _write(path, geo, Vs, beams, exts, pin, th, ph)
    bl = read_beam_list(path)
    assert bl.norient == len(beams)
    assert bl.lam == LAM
    assert np.array_equal(bl.theta, th) and np.array_equal(bl.phi, ph)
    assert np.array_equal(bl.geometry["face_off"], geo["face_off"])
    assert np.array_equal(bl.geometry["face_vi"], geo["face_vi"])
    for o in range(len(beams)):
        assert np.array_equal(bl.verts[o], Vs[o])
        assert bl.beams[o].tobytes() == np.ascontiguousarray(beams[o]).tobytes()
        assert bl.exts[o].tobytes() == np.ascontiguousarray(exts[o]).tobytes()
    assert bl.params_in.tobytes() == pin.tobytes()


def test_empty_file_has_no_orientations(tmp_path):
    geo, Vs, beams, exts, pin, th, ph = _lists(1)
    path = tmp_path / "empty.pbtb"
    _write(path, geo, [], [], [], [], th, ph)
    assert read_beam_list(path).norient == 0


@pytest.mark.parametrize("damage", ["flip", "truncate", "magic", "version"])
def test_damaged_files_are_refused(tmp_path, damage):
    geo, Vs, beams, exts, pin, th, ph = _lists(3)
    path = tmp_path / "d.pbtb"
    _write(path, geo, Vs, beams, exts, pin, th, ph)
    raw = bytearray(path.read_bytes())
    if damage == "flip":
        raw[len(raw) // 2] ^= 0x10
    elif damage == "truncate":
        raw = raw[:-40]
    elif damage == "magic":
        raw[0:8] = b"NOTABEAM"
    else:
        raw[8] = 99
    path.write_bytes(bytes(raw))
    with pytest.raises(PbtError):
        read_beam_list(path)


def test_writer_rejects_bad_input(tmp_path):
    geo, Vs, beams, exts, pin, th, ph = _lists(2)
    with BeamListWriter(tmp_path / "w.pbtb", th, ph, geo, LAM) as w:
        bad = exts[0].copy()
        bad["fi"][0] = len(geo["face_off"])  # one past the last face
        with pytest.raises(PbtError):
            w.add(beams[0], bad, Vs[0], pin[0])
        V = Vs[0].copy()
        V[0, 0] = np.nan
        with pytest.raises(PbtError):
            w.add(beams[0], exts[0], V, pin[0])
    with pytest.raises(PbtError):
        read_beam_list(tmp_path / "missing.pbtb")


@pytest.mark.gpu
def test_replay_matches_direct_batch(ctx, tmp_path):
    geo, Vs, beams, exts, pin, th, ph = _lists(4, seed=32)
    path = tmp_path / "r.pbtb"
    _write(path, geo, Vs, beams, exts, pin, th, ph)
    bl = read_beam_list(path)
    for prec in ("fp64", "fp32"):
        ref = ctx.diff_batch(beams, exts, Vs, geo, th, ph, LAM, pin, precision=prec)
        rep = ctx.diff_batch(bl.beams, bl.exts, bl.verts, bl.geometry, bl.theta, bl.phi, bl.lam,
                             bl.params_in, precision=prec)
        assert mueller_rel_err(rep[0], ref[0]) < (1e-12 if prec == "fp64" else 1e-5)
