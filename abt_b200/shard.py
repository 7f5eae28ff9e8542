"""Orientation sharding: one process per GPU, each averaging a contiguous block
of the orientations, and one FP64 sum of the blocks across the ranks.

The reference's MPI driver splits its orientation loop with mpi_get_start_end
(src/mpi_mod.f90:140-164): with n orientations on p ranks the first n mod p
ranks take n // p + 1 orientations and the others n // p, in rank order.  Each
rank sums its orientations (summation, src/outputs_mod.f90:407-471), rank 0
adds the other ranks' totals to its own (mpi_send_sum, src/mpi_mod.f90:233-300)
and divides by n (divide_by_num_orientations, src/outputs_mod.f90:13-43).

Here each rank averages its block on its own GPU (Context.diff_batch, the
batched FP32 kernel or the reference-exact FP64 path), turns the average back
into the block's sums (average x block size; one FP64 rounding), and one
all-gather over torch.distributed (NCCL between GPUs, gloo between host
processes) gives every rank all the blocks' sums, which it adds in rank order,
as the reference's rank 0 does, and divides by n.  The orientations exchange
nothing else: the gather of the (nphi, ntheta, 16) + (ntheta, 16) + 18
accumulators is the only collective, once per average.
"""
import numpy as np

from ._lib import PARAMS_DTYPE

_NPARAM = len(PARAMS_DTYPE.names)


def orientation_block(n, rank, world):
    """[start, end) of rank's orientations (0-based) among n, as
    mpi_get_start_end (src/mpi_mod.f90:140-164) assigns them."""
    n, rank, world = int(n), int(rank), int(world)
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank %d is not in a world of %d" % (rank, world))
    if world > n:
        # src/mpi_mod.f90:151
        raise ValueError("number of ranks (%d) must not be greater than number of orientations (%d)"
                         % (world, n))
    n1, n2 = divmod(n, world)
    start, end = rank * (n1 + 1), (rank + 1) * (n1 + 1)
    if rank >= n2:
        start, end = start - rank + n2, end - rank + n2 - 1
    return start, end


def _flat(mu, mu1, pav):
    p = np.asarray(pav, dtype=PARAMS_DTYPE).reshape(()).view((np.float64, _NPARAM))
    return np.concatenate([np.asarray(mu, np.float64).ravel(order="F"),
                           np.asarray(mu1, np.float64).ravel(order="F"), p.ravel()])


def combine_blocks(mu, mu1, pav, count, total, group=None, device=None):
    """Average over all ranks' orientations from this rank's block average.

    mu (nphi, ntheta, 16), mu1 (ntheta, 16) and pav (a PARAMS_DTYPE scalar)
    average `count` orientations (this rank's block); `total` is the number of
    orientations over all ranks.  Every rank of `group` (default: the world)
    calls it with arrays of the same shapes.  device: where the gather runs
    (a CUDA device for NCCL; the host for gloo, the default when None).
    Returns (mueller_avg, mueller_1d_avg, params_avg) of all orientations."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)
    sums = _flat(mu, mu1, pav) * float(count)
    if device is None:
        device = torch.device("cuda", torch.cuda.current_device()) \
            if dist.get_backend(group) == "nccl" else torch.device("cpu")
    t = torch.from_numpy(sums).to(device)
    allb = torch.empty(world * t.numel(), dtype=torch.float64, device=device)
    dist.all_gather_into_tensor(allb, t, group=group)
    blocks = allb.cpu().numpy().reshape(world, -1)
    tot = blocks[0].copy()
    for r in range(1, world):
        tot = tot + blocks[r]
    tot = tot / float(total)
    nm, n1 = np.asarray(mu).size, np.asarray(mu1).size
    mu_o = tot[:nm].reshape(np.shape(mu), order="F")
    mu1_o = tot[nm:nm + n1].reshape(np.shape(mu1), order="F")
    p_o = np.zeros((), dtype=PARAMS_DTYPE)
    p_o.view((np.float64, _NPARAM))[:] = tot[nm + n1:]
    return np.asfortranarray(mu_o), np.asfortranarray(mu1_o), p_o


def diff_batch_sharded(ctx, beams, exts, verts_per_orient, geometry, theta, phi, lam, params_in,
                       group=None, device=None, **kw):
    """Context.diff_batch over all orientations, sharded across the ranks of
    `group`: this rank averages its block (orientation_block) on ctx's GPU and
    combine_blocks adds the blocks.  beams, exts, verts_per_orient and
    params_in hold every orientation (each rank reads only its block); kw goes
    to diff_batch (is_fast_diff, scaling, precision).
    Returns (mueller_avg, mueller_1d_avg, params_avg, (start, end),
    params_per_orient of the block)."""
    import torch.distributed as dist

    n = len(beams)
    s, e = orientation_block(n, dist.get_rank(group), dist.get_world_size(group))
    mu, mu1, pav, pper = ctx.diff_batch(beams[s:e], exts[s:e], verts_per_orient[s:e], geometry, theta,
                                        phi, lam, np.asarray(params_in)[s:e], **kw)
    mu, mu1, pav = combine_blocks(mu, mu1, pav, e - s, n, group=group, device=device)
    return mu, mu1, pav, (s, e), pper
