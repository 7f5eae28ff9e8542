"""Orientation sharding (abt_b200/shard.py): the reference's MPI split of the
orientation loop (src/mpi_mod.f90:140-164) and the sum of the ranks' totals,
on gloo ranks on the host; on the GPU, two ranks sharing cuda:0 against the
unsharded batch."""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

from abt_b200 import PARAMS_DTYPE
from abt_b200.shard import orientation_block

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _mpi_get_start_end(n, p, rank):
    """mpi_get_start_end as the reference writes it (1-based, inclusive end)."""
    n1, n2 = n // p, n % p
    start = rank * (n1 + 1) + 1
    end = (rank + 1) * (n1 + 1)
    if rank >= n2:
        start = start - rank + n2
        end = end - rank + n2 - 1
    return start, end


def test_orientation_block_is_the_reference_split():
    for n in range(1, 60):
        for p in range(1, min(n, 12) + 1):
            prev = 0
            for r in range(p):
                s, e = orientation_block(n, r, p)
                s1, e1 = _mpi_get_start_end(n, p, r)
                assert (s, e) == (s1 - 1, e1)
                assert s == prev and e - s in (n // p, n // p + 1)  # contiguous and balanced
                prev = e
            assert prev == n
    with pytest.raises(ValueError):
        orientation_block(3, 0, 4)  # more ranks than orientations (src/mpi_mod.f90:151)
    with pytest.raises(ValueError):
        orientation_block(8, 2, 2)


def _synthetic(n, nphi=5, ntheta=4, seed=0):
    rng = np.random.default_rng(seed)
    mu = rng.normal(size=(n, nphi, ntheta, 16))
    mu1 = rng.normal(size=(n, ntheta, 16))
    p = np.zeros(n, dtype=PARAMS_DTYPE)
    for name in PARAMS_DTYPE.names:
        p[name] = rng.normal(size=n)
    return mu, mu1, p


def _block_avg(mu, mu1, p, s, e):
    pav = np.zeros((), dtype=PARAMS_DTYPE)
    for name in PARAMS_DTYPE.names:
        pav[name] = p[name][s:e].sum() / (e - s)
    return (np.asfortranarray(mu[s:e].sum(0) / (e - s)), np.asfortranarray(mu1[s:e].sum(0) / (e - s)),
            pav)


def _combine_rank(rank, world, port, n, q):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    from abt_b200.shard import combine_blocks, orientation_block as ob
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    mu, mu1, p = _synthetic(n)
    s, e = ob(n, rank, world)
    out = combine_blocks(*_block_avg(mu, mu1, p, s, e), e - s, n)
    q.put((rank, out))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("world,n", [(2, 7), (3, 10)])
def test_combine_blocks_gloo(world, n):
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_combine_rank, args=(r, world, port, n, q)) for r in range(world)]
    for pr in procs:
        pr.start()
    got = dict(q.get(timeout=120) for _ in range(world))
    for pr in procs:
        pr.join(timeout=60)
        assert pr.exitcode == 0
    mu, mu1, p = _synthetic(n)
    # the blocks' totals added in rank order, then divided by n (the reference's rank 0)
    tot_mu = tot_mu1 = None
    tot_p = {}
    for r in range(world):
        s, e = orientation_block(n, r, world)
        bm, bm1, bp = _block_avg(mu, mu1, p, s, e)
        bm, bm1 = bm * (e - s), bm1 * (e - s)
        tot_mu = bm if tot_mu is None else tot_mu + bm
        tot_mu1 = bm1 if tot_mu1 is None else tot_mu1 + bm1
        for name in PARAMS_DTYPE.names:
            tot_p[name] = tot_p.get(name, 0.0) + bp[name] * (e - s) if r else bp[name] * (e - s)
    for r in range(world):
        gm, gm1, gp = got[r]
        assert gm.shape == mu.shape[1:] and gm.flags.f_contiguous
        assert np.array_equal(gm, tot_mu / n) and np.array_equal(gm1, tot_mu1 / n)
        for name in PARAMS_DTYPE.names:
            assert gp[name] == tot_p[name] / n
        # and the plain average of all orientations, to FP64 rounding
        assert np.abs(gm - mu.mean(0)).max() <= 1e-14 * np.abs(mu.mean(0)).max()


def _traced_lists(norient):
    from abt_b200 import workloads as W
    from abt_b200 import tracer as T
    geo = W.hex_prism(5.0, 10.0, n_side=3, n_len=6, roughness=0.1, seed=3)
    P = T.Particle(geo, geo["apertures"])
    rng = np.random.default_rng(5)
    Vs, beams, exts, pins = [], [], [], []
    for u in rng.uniform(size=(norient, 3)):
        V, beam, ext, pin, _ = T.trace(P, T.multi_euler(*u), 0.532, 1.31)
        Vs.append(V)
        beams.append(beam)
        exts.append(ext)
        pins.append(pin)
    return P.geometry, Vs, beams, exts, np.array(pins)


def _gpu_rank(rank, world, port, norient, precision, q):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    from abt_b200 import Context, make_angles
    from abt_b200.shard import diff_batch_sharded
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    geo, Vs, beams, exts, pins = _traced_lists(norient)
    theta, phi = make_angles([0, 180], [1.0]), make_angles([0, 356], [4])
    with Context(0) as c:
        mu, mu1, pav, blk, _ = diff_batch_sharded(c, beams, exts, Vs, geo, theta, phi, 0.532, pins,
                                                  precision=precision)
    q.put((rank, mu, mu1, pav, blk))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.gpu
@pytest.mark.parametrize("precision,tol", [("fp64", 1e-13), ("fp32", 2e-6)])
def test_sharded_average_matches_one_process(precision, tol):
    """Two ranks (gloo between them, both on cuda:0: their kernels do not wait on
    each other) average 3 and 2 of 5 traced orientations; the combined average
    equals the one-process batch over all five (FP64 path: to rounding; FP32:
    to the plan's summation order)."""
    from abt_b200 import Context, make_angles
    world, norient, port = 2, 5, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_gpu_rank, args=(r, world, port, norient, precision, q))
             for r in range(world)]
    for pr in procs:
        pr.start()
    got = {}
    for _ in range(world):
        r, mu, mu1, pav, blk = q.get(timeout=600)
        got[r] = (mu, mu1, pav, blk)
    for pr in procs:
        pr.join(timeout=120)
        assert pr.exitcode == 0
    assert got[0][3] == (0, 3) and got[1][3] == (3, 5)
    geo, Vs, beams, exts, pins = _traced_lists(norient)
    theta, phi = make_angles([0, 180], [1.0]), make_angles([0, 356], [4])
    with Context(0) as c:
        mu, mu1, pav, _ = c.diff_batch(beams, exts, Vs, geo, theta, phi, 0.532, pins, precision=precision)
    for r in range(world):
        gm, gm1, gp, _ = got[r]
        assert np.abs(gm - mu).max() <= tol * np.abs(mu).max()
        assert np.abs(gm1 - mu1).max() <= tol * np.abs(mu1).max()
        for name in ("scatt", "ext", "asymmetry", "scatt_eff", "ext_eff"):
            assert abs(gp[name] - pav[name]) <= tol * abs(pav[name]), name
