"""CUDA graph of the device-pointer FP32 batch (pbt_diff_batch_dev_graph_c):
the captured graph reproduces the direct call, and a replay after the device
inputs are refilled in place computes the new inputs' average."""
import numpy as np
import pytest

import abt_b200
from abt_b200 import workloads as W
from abt_b200.diff import BatchGraph, diff_batch_dev
from tests.helpers import mueller_rel_err

LAM = 0.532


def _device_case(n_orient, seed):
    import torch
    geo, Vs, beams, exts, pin = W.rough_column_orientations(n_orient, seed=seed, n_side=3,
                                                            n_len=6, m_range=(1, 4))
    th = abt_b200.make_angles([0, 180], [2])
    ph = abt_b200.make_angles([0, 356], [4])
    dev = torch.device("cuda", 0)
    beam = np.concatenate(beams)
    ext = np.concatenate(exts)
    boff = np.concatenate([[0], np.cumsum([len(b) for b in beams])]).astype(np.int64)
    eoff = np.concatenate([[0], np.cumsum([len(e) for e in exts])]).astype(np.int64)
    V = np.concatenate([np.asfortranarray(v).ravel(order="F") for v in Vs])
    nb = len(th) * len(ph)
    d = dict(
        beam=torch.from_numpy(beam.view(np.uint8).copy()).to(dev),
        ext=torch.from_numpy(ext.view(np.uint8).copy()).to(dev),
        verts=torch.from_numpy(V).to(dev),
        fvi=torch.from_numpy(geo["face_vi"].copy()).to(dev),
        pin=torch.from_numpy(pin.view(np.uint8).copy()).to(dev),
        mu=torch.zeros(16 * nb, dtype=torch.float64, device=dev),
        m1=torch.zeros(16 * len(th), dtype=torch.float64, device=dev),
        pav=torch.zeros(18, dtype=torch.float64, device=dev),
        pper=torch.zeros(18 * n_orient, dtype=torch.float64, device=dev))
    host = dict(beam=beam, boff=boff, eoff=eoff, nverts=Vs[0].shape[0], geo=geo, th=th, ph=ph)
    return d, host


def _outputs(d, host):
    nth, nph = len(host["th"]), len(host["ph"])
    mu = d["mu"].cpu().numpy().reshape(16, nth, nph).transpose(2, 1, 0)
    return mu, d["pav"].cpu().numpy().copy()


def _direct(ctx, stream, n_orient, d, host):
    diff_batch_dev(ctx, stream, n_orient, d["beam"], host["boff"], d["ext"], host["eoff"],
                   d["verts"], host["nverts"], host["geo"]["face_off"], d["fvi"], host["th"],
                   host["ph"], LAM, d["pin"], d["mu"], d["m1"], d["pav"], d["pper"])


@pytest.mark.gpu
def test_graph_replay_matches_direct_call(ctx):
    import torch
    n = 6
    d, host = _device_case(n, seed=21)
    stream = torch.cuda.current_stream().cuda_stream
    _direct(ctx, stream, n, d, host)
    torch.cuda.synchronize()
    mu_ref, p_ref = _outputs(d, host)
    d["mu"].zero_()
    g = BatchGraph(ctx, stream, n, d["beam"], host["boff"], d["ext"], host["eoff"], d["verts"],
                   host["nverts"], host["geo"]["face_off"], d["fvi"], host["th"], host["ph"], LAM,
                   d["pin"], d["mu"], d["m1"], d["pav"], d["pper"])
    torch.cuda.synchronize()
    assert g.kernel_count() > 0
    mu_w, _ = _outputs(d, host)
    assert mueller_rel_err(mu_w, mu_ref) < 1e-5
    for _ in range(3):
        d["mu"].zero_()
        d["pav"].zero_()
        g.launch(stream)
    torch.cuda.synchronize()
    mu_g, p_g = _outputs(d, host)
    assert mueller_rel_err(mu_g, mu_ref) < 1e-5
    assert np.allclose(p_g, p_ref, rtol=1e-6, atol=0)
    g.close()


@pytest.mark.gpu
def test_graph_replay_reads_refilled_inputs(ctx):
    import torch
    n = 4
    d, host = _device_case(n, seed=22)
    stream = torch.cuda.current_stream().cuda_stream
    g = BatchGraph(ctx, stream, n, d["beam"], host["boff"], d["ext"], host["eoff"], d["verts"],
                   host["nverts"], host["geo"]["face_off"], d["fvi"], host["th"], host["ph"], LAM,
                   d["pin"], d["mu"], d["m1"], d["pav"], d["pper"])
    torch.cuda.synchronize()
    # new beam amplitudes, same sizes: refill the device array in place
    beam2 = host["beam"].copy()
    rng = np.random.default_rng(5)
    beam2["ampl"] *= rng.uniform(0.5, 2.0, size=(len(beam2), 1))
    d["beam"].copy_(torch.from_numpy(beam2.view(np.uint8).copy()))
    g.launch(stream)
    torch.cuda.synchronize()
    mu_g, _ = _outputs(d, host)
    _direct(ctx, stream, n, d, host)
    torch.cuda.synchronize()
    mu_ref, _ = _outputs(d, host)
    assert mueller_rel_err(mu_g, mu_ref) < 1e-5
    g.close()
