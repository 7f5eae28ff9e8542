"""Tuner for the FP32 far-field kernel's launch plan.

Times each candidate plan (kernel variant x bins per thread x facet records
per work item) on a sample of the caller's workload, with the inputs already
on the device and the kernel timed by CUDA events inside the library, and sets
the fastest on the context.  The sample is the first `sample_facets` facets of
one orientation over the full far-field grid: the per facet x bin cost does
not depend on the facet count, while the work-item granularity does depend on
the grid, which is kept.  A sample smaller than the caller's list also has fewer
facet splits per bin tile, so it favours smaller work items than the full list
wants (on 200,000 facets x 259,560 bins 2,048-8,192 records per item time the
same and 1,024 is 0.2 % slower, while a 20,000-facet sample ranks 1,024 first);
pass the whole list where one call of it is cheap.
"""
import numpy as np

from . import _lib
from .diff import diff_batch_dev

CANDIDATES = [(1, 1, 2048), (1, 1, 1024), (1, 1, 4096), (1, 2, 2048), (0, 2, 2048), (0, 1, 2048)]


def tune(ctx, beam, geometry, theta, phi, lam, sample_facets=20000, candidates=CANDIDATES,
         repeats=2, verbose=False):
    """Returns (best plan, {plan: kernel ms}) and sets the best plan on ctx."""
    import torch
    dev = torch.device("cuda", ctx.device)
    sub = np.ascontiguousarray(beam[:sample_facets])
    nb = len(theta) * len(phi)
    d_beam = torch.from_numpy(sub.view(np.uint8).copy()).to(dev)
    d_ext = torch.empty(128, dtype=torch.uint8, device=dev)
    V = np.asfortranarray(geometry["verts"], dtype=np.float64)
    d_verts = torch.from_numpy(V.ravel(order="F").copy()).to(dev)
    d_fvi = torch.from_numpy(np.ascontiguousarray(geometry["face_vi"], dtype=np.int64)).to(dev)
    pin = np.zeros(1, dtype=_lib.PARAMS_DTYPE)
    pin["geo_cross_sec"] = pin["beam_energy_out"] = pin["ext_energy_out"] = 1.0
    d_pin = torch.from_numpy(pin.view(np.uint8).copy()).to(dev)
    d_mu = torch.empty(16 * nb, dtype=torch.float64, device=dev)
    d_m1 = torch.empty(16 * len(theta), dtype=torch.float64, device=dev)
    d_pav = torch.empty(18, dtype=torch.float64, device=dev)
    boff = np.array([0, len(sub)], dtype=np.int64)
    eoff = np.array([0, 0], dtype=np.int64)
    stream = torch.cuda.current_stream(dev).cuda_stream
    times = {}
    for plan in candidates:
        ctx.set_plan(*plan)
        run = lambda: diff_batch_dev(ctx, stream, 1, d_beam, boff, d_ext, eoff, d_verts, V.shape[0],
                                     geometry["face_off"], d_fvi, theta, phi, lam, d_pin, d_mu,
                                     d_m1, d_pav)
        run()
        torch.cuda.synchronize(dev)
        ctx.set_kernel_timing(True)
        ctx.kernel_time_ms()
        for _ in range(repeats):
            run()
        torch.cuda.synchronize(dev)
        ms, n = ctx.kernel_time_ms()
        ctx.set_kernel_timing(False)
        times[plan] = ms / max(n, 1)
        if verbose:
            print("plan", plan, "%.3f ms" % times[plan], flush=True)
    best = min(times, key=times.get)
    ctx.set_plan(*best)
    return best, times
