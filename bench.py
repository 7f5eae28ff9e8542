#!/usr/bin/env python
"""Benchmark of the far-field diffraction hot path on B200.

Workload (the precision-study configuration): a synthetic beam list of
200,000 outgoing triangular facets in 2,000 beams (vertices in a 100 um cube,
edges 0.3-1.5 um, log-normal amplitudes), lambda = 0.532 um, far field
721 theta x 360 phi = 259,560 bins: 5.19e10 facet x bin evaluations per step.

One step = the batched FP32 far-field sum with FP64 phase plus its FP64
epilogue (Mueller matrix, phi/theta integrals, cross sections), inputs
resident in HBM.  Metric: facet x bin evaluations per second (whole job).

Also reported: the same metric end to end through the host C ABI
(pbt_diff_batch_list_c, pinned host buffers, copies inside the timed region)
and the roofline of the dominant kernel; in single-GPU runs also the
reference-exact FP64 drop-in's rate, the FP32-vs-FP64 Mueller error on the
full workload, the further workloads (orientation average on stand-in and on
host-traced beam lists, differentiation, large column, -fast_diff, adjoint)
and a CPU baseline (the C FP64
restatement of the reference, all host cores, bounded sample).  N-GPU runs
(replicas) time the step, e2e and roofline only.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "facet·bin evals/s & orientations/s: batched FP32 vs plain FP64 GPU @1e-4 err"
UNIT = "facet·bin/s"
LAM = 0.532
# algorithmic work per triangle facet x bin (fixed counting convention)
W_FP32 = 170.0   # FP32 flops (FMA = 2)
W_SFU = 20.0     # special-function ops
FP32_PER_SM_CLK = 128 * 2   # FP32 lanes x 2 flops
SFU_PER_SM_CLK = 16
W_FP64 = 12.0    # FP64 flops (the phase k u.c and its reduction)
FP64_PER_SM_CLK = 64 * 2    # FP64 lanes x 2 flops


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--beams", type=int, default=2000)
    ap.add_argument("--facets-per-beam", type=int, default=100)
    ap.add_argument("--fp64-facets", type=int, default=4000,
                    help="facets of the FP64 drop-in rate sample (0 = skip)")
    ap.add_argument("--no-error-check", action="store_true",
                    help="skip the full-workload FP64 run used for the FP32 error")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--no-tune", action="store_true",
                    help="keep the default launch plan instead of tuning it on the step's facet list")
    ap.add_argument("--no-graph", action="store_true",
                    help="enqueue each step through the C ABI instead of replaying a CUDA graph")
    ap.add_argument("--orient", type=int, default=1024,
                    help="orientations of the rough-column orientation average (0: skip)")
    ap.add_argument("--traced-orient", type=int, default=1024,
                    help="orientations traced on the host and averaged (0: skip)")
    ap.add_argument("--orient-fp64", type=int, default=16,
                    help="orientations timed with the FP64 drop-in and used for the error")
    ap.add_argument("--fast-diff", type=int, default=1,
                    help="1: also time the workload with is_fast_diff (field-of-view tile cull)")
    ap.add_argument("--large-orient", type=int, default=2,
                    help="orientations of the large absorbing column timed (0: skip)")
    ap.add_argument("--large-traced-orient", type=int, default=8,
                    help="orientations of the large column traced on the host (0: skip)")
    ap.add_argument("--config5", type=int, default=0,
                    help="orientations of the large absorbing column at its full size "
                         "(2048 in the configuration; opt-in, about ten minutes; 0: skip)")
    ap.add_argument("--config5-fp64", type=int, default=64,
                    help="orientations of the large absorbing column averaged in FP64 too, "
                         "for the FP32 error")
    ap.add_argument("--diff-orient", type=int, default=64,
                    help="orientations of the differentiation workload (0: skip)")
    ap.add_argument("--fd-coords", type=int, default=200,
                    help="vertex coordinates checked by FP64 central differences on each of the "
                         "first two orientations of the differentiation workload (0: skip)")
    ap.add_argument("--diffraction-calls", type=int, default=200,
                    help="per-call time of pbt_diffraction_c / pbt_diffraction_noalloc_c "
                         "(one outbeam, 181 x 180 bins; 0 = skip)")
    ap.add_argument("--adjoint-facets", type=int, default=20000,
                    help="facet sample for the adjoint / forward kernel-time ratio (0: skip)")
    return ap.parse_args()


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu_index = gpu_index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu_index),
                                       "--query-gpu=" + self.FIELDS, "--format=csv,noheader,nounits",
                                       "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.flush()
        self.f.seek(0)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.f.read().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        os.unlink(self.f.name)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None, "samples": len(sm),
                "reasons": sorted(reasons)}


def max_over_ranks(dist, ms, device):
    """The slowest rank's time (all ranks take part; dist None: one process)."""
    if dist is None:
        return ms
    import torch
    t = torch.tensor([ms], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replicas_value(world, work_per_rank, ms_step):
    """Whole-job throughput of `world` replicas: all ranks' units over the slowest time."""
    return world * work_per_rank / (ms_step / 1e3)


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        backend = "nccl" if args.impl == "ours" else "gloo"
        if backend == "nccl":
            import torch
            torch.cuda.set_device(local)  # each rank's GPU current before NCCL starts
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
        pg = dist
    return world, rank, local, pg


def workload(args):
    from abt_b200 import workloads as W
    geo, beam, ext = W.synthetic_beam_list(n_beams=args.beams, facets_per_beam=args.facets_per_beam,
                                           seed=2024)
    th, ph = W.grid_precision_study()
    return geo, beam, ext, th, ph


def orientation_average(ctx, args):
    """Batched FP32 orientation average of the rough hexagonal column (stand-in
    beam lists, 361 x 180 bins) against the plain per-orientation FP64 drop-in,
    timed on the first --orient-fp64 orientations and extrapolated by facet·bin
    count; the error of the averaged Mueller matrix and cross sections is taken
    on those orientations."""
    from abt_b200 import workloads as W
    geo, Vs, beams, exts, pin = W.rough_column_orientations(args.orient, seed=3)
    th, ph = W.grid_orientation_average()
    out = {"workload": "rough hexagonal column r 10 um, L 20 um, sigma 0.1 um (1296 triangles), "
                       "stand-in beam lists, %d orientations uniform on SO(3), 361 theta x 180 phi"
                       % args.orient}
    out.update(_average(ctx, args, geo, Vs, beams, exts, pin, th, ph))
    return out


def traced_orientation_average(ctx, args):
    """The same orientation average on beam lists from the host tracer: the
    rough column (apertures = its 8 parent faces) traced at --traced-orient
    orientations uniform on SO(3) with pbt_trace_batch_c (n = 1.31, 8
    recursions, the reference's thresholds), one orientation per host thread;
    the tracing is timed on the host cores, then the FP32 batch and the FP64
    drop-in sample are timed as in orientation_average; last, the whole loop
    with tracing (host) and averaging (GPU) overlapped chunk by chunk
    (abt_b200.tracer.traced_orientation_average, FP32, 128 orientations per
    chunk)."""
    from abt_b200 import tracer as T
    from abt_b200 import workloads as W
    g = W.hex_prism(10.0, 20.0, n_side=6, n_len=12, roughness=0.1, seed=3)
    P = T.Particle(g, g["apertures"])
    eul = W.uniform_euler(np.random.default_rng(3), args.traced_orient)
    T.trace_batch(P, eul[:8], LAM, 1.31)
    t0 = time.perf_counter()
    Vs, beams, exts, pin, en = T.trace_batch(P, eul, LAM, 1.31)
    t_trace = time.perf_counter() - t0
    th, ph = W.grid_orientation_average()
    # the whole loop with tracing and the GPU average overlapped chunk by chunk
    T.traced_orientation_average(ctx, P, eul[:64], th, ph, LAM, 1.31, chunk=32)
    t0 = time.perf_counter()
    T.traced_orientation_average(ctx, P, eul, th, ph, LAM, 1.31, chunk=128)
    t_pipe = time.perf_counter() - t0
    ratio = en["beam_energy_out"] / en["geo_cross_sec"]
    out = {"workload": "rough hexagonal column r 10 um, L 20 um, sigma 0.1 um (1296 triangles, "
                       "8 apertures), beam lists traced on the host (n = 1.31, rec 8), "
                       "%d orientations uniform on SO(3), 361 theta x 180 phi" % args.traced_orient,
           "trace_s": t_trace, "trace_orientations_per_s": args.traced_orient / t_trace,
           "trace_and_average_overlapped_s": t_pipe,
           "trace_and_average_orientations_per_s": args.traced_orient / t_pipe,
           "trace_threads": int(os.cpu_count() or 1),
           "beams_traced_per_orientation": [int(en["nbeams"].min()), int(en["nbeams"].mean()),
                                            int(en["nbeams"].max())],
           "beam_energy_over_geo_cross_section": [float(ratio.min()), float(ratio.mean()),
                                                  float(ratio.max())]}
    out.update(_average(ctx, args, P.geometry, Vs, beams, exts, pin, th, ph))
    return out


def _average(ctx, args, geo, Vs, beams, exts, pin, th, ph):
    from tests.helpers import mueller_rel_err
    norient = len(beams)
    nb = len(th) * len(ph)
    F = np.array([len(b) + len(e) for b, e in zip(beams, exts)])
    k = max(1, min(args.orient_fp64, norient))
    # FP32 batched, all orientations (host API: H2D, one persistent launch per chunk, D2H)
    ctx.diff_batch(beams[:2], exts[:2], Vs[:2], geo, th, ph, LAM, pin[:2], precision="fp32")
    ctx.set_kernel_timing(True)
    # best of two calls: the host side (gather, copies) shares the box's cores
    t32 = k32_ms = None
    for _ in range(2):
        ctx.kernel_time_ms()
        t0 = time.perf_counter()
        ctx.diff_batch(beams, exts, Vs, geo, th, ph, LAM, pin, precision="fp32")
        dt = time.perf_counter() - t0
        kms, k32_n = ctx.kernel_time_ms()
        if t32 is None or dt < t32:
            t32, k32_ms = dt, kms
    # FP32 and FP64 on the first k orientations
    f32 = ctx.diff_batch(beams[:k], exts[:k], Vs[:k], geo, th, ph, LAM, pin[:k], precision="fp32")
    # the FP64 drop-in in its steady state: best of two calls after an untimed
    # one of the same size (host buffers already allocated and touched)
    ctx.diff_batch(beams[:k], exts[:k], Vs[:k], geo, th, ph, LAM, pin[:k], precision="fp64")
    t64k = k64_ms = None
    for _ in range(2):
        ctx.kernel_time_ms()
        t0 = time.perf_counter()
        f64 = ctx.diff_batch(beams[:k], exts[:k], Vs[:k], geo, th, ph, LAM, pin[:k],
                             precision="fp64")
        dt = time.perf_counter() - t0
        kms, _ = ctx.kernel_time_ms()
        if t64k is None or dt < t64k:
            t64k, k64_ms = dt, kms
    ctx.set_kernel_timing(False)
    work = float(F.sum()) * nb
    work_k = float(F[:k].sum()) * nb
    t64 = t64k * work / work_k
    perr = max(abs(float(f32[2][n]) - float(f64[2][n])) / abs(float(f64[2][n]))
               for n in ("scatt", "ext", "asymmetry", "back_scatt"))
    return {"orientations": int(norient), "facets_total": int(F.sum()),
            "facets_per_orientation": [int(F.min()), int(F.mean()), int(F.max())], "bins": nb,
            "fp32_batched_s": t32, "fp32_orientations_per_s": norient / t32,
            "fp32_facet_bin_per_s": work / t32, "fp32_kernel_ms": k32_ms,
            "fp32_main_launches": int(k32_n),
            "fp64_dropin_sample_orientations": k, "fp64_dropin_sample_s": t64k,
            "fp64_dropin_kernel_ms": k64_ms,
            "fp64_dropin_orientations_per_s": norient / t64,
            "speedup_fp32_batched_vs_fp64_dropin": t64 / t32,
            "max_rel_mueller_err_vs_fp64": mueller_rel_err(f32[0], f64[0], 1e-6),
            "max_rel_param_err_vs_fp64": perr,
            "api": "pbt_diff_batch_list_c (host pointers, one array per orientation), wall clock"}


def large_traced(ctx, args):
    """The large column with beam lists from the host tracer: the same column
    and grid as large_case, its 8 parent faces as apertures, n = 1.31 + 0.01i,
    8 recursions, --large-traced-orient orientations uniform on SO(3) traced
    with pbt_trace_batch_c and averaged by one FP32 batch; the FP64 drop-in and
    the error on the whole first orientation."""
    import abt_b200
    from abt_b200 import tracer as T
    from abt_b200 import workloads as W
    from tests.helpers import mueller_rel_err
    g = W.hex_prism(50.0, 100.0, n_side=25, n_len=50, roughness=0.0, seed=5)
    P = T.Particle(g, g["apertures"])
    th = abt_b200.make_angles([0, 180], [0.125])
    ph = abt_b200.make_angles([0, 359.5], [0.5])
    nb = len(th) * len(ph)
    n = args.large_traced_orient
    eul = W.uniform_euler(np.random.default_rng(5), n)
    t0 = time.perf_counter()
    Vs, beams, exts, pin, en = T.trace_batch(P, eul, LAM, 1.31, ibi=0.01)
    t_trace = time.perf_counter() - t0
    geo = P.geometry
    F = np.array([len(b) + len(e) for b, e in zip(beams, exts)])
    ctx.diff_batch(beams[:1], [exts[0][:64]], Vs[:1], geo, th, ph, LAM, pin[:1], precision="fp32")
    ctx.set_kernel_timing(True)
    ctx.kernel_time_ms()
    t0 = time.perf_counter()
    ctx.diff_batch(beams, exts, Vs, geo, th, ph, LAM, pin, precision="fp32")
    t32 = time.perf_counter() - t0
    k_ms, _ = ctx.kernel_time_ms()
    g0 = dict(geo, verts=Vs[0])
    a32 = ctx.diff_main(beams[0], exts[0], g0, th, ph, LAM, precision="fp32")
    ctx.kernel_time_ms()
    t0 = time.perf_counter()
    a64 = ctx.diff_main(beams[0], exts[0], g0, th, ph, LAM, precision="fp64")
    t64 = time.perf_counter() - t0
    k64_ms, _ = ctx.kernel_time_ms()
    ctx.set_kernel_timing(False)
    m32, _, p32 = ctx.finalise(a32[0], a32[1], th, ph, LAM, pin[0])
    m64, _, p64 = ctx.finalise(a64[0], a64[1], th, ph, LAM, pin[0])
    work = float(F.sum()) * nb
    ratio = (en["beam_energy_out"] + en["abs"]) / en["geo_cross_sec"]
    return {"workload": "smooth hexagonal column r 50 um, L 100 um, 2 um^2 triangles (22,500, "
                        "8 apertures), beam lists traced on the host (n = 1.31 + 0.01i, rec 8), "
                        "%d orientations, 1441 theta x 720 phi" % n,
            "trace_s": t_trace, "outbeams_per_orientation": [int(F.min()), int(F.mean()),
                                                             int(F.max())],
            "energy_out_plus_absorbed_over_geo": [float(ratio.min()), float(ratio.max())],
            "bins": nb, "fp32_batched_s": t32, "fp32_orientations_per_s": n / t32,
            "fp32_facet_bin_per_s": work / t32, "fp32_kernel_ms": k_ms,
            "fp64_dropin_first_orientation_s": t64, "fp64_dropin_kernel_ms": k64_ms,
            "speedup_fp32_batched_vs_fp64_dropin": t64 * n / t32 * float(F.mean()) / float(F[0]),
            "max_rel_mueller_err_vs_fp64_first_orientation": mueller_rel_err(m32, m64, 1e-6),
            "mueller_err_above_1e-5_and_1e-4_of_peak": [mueller_rel_err(m32, m64, 1e-5),
                                                        mueller_rel_err(m32, m64, 1e-4)],
            "worst_bin_theta_deg_m11_over_peak": _worst_bin(m32, m64, th),
            "max_rel_param_err_vs_fp64_first_orientation": max(
                abs(float(p32[k]) - float(p64[k])) / abs(float(p64[k]))
                for k in ("scatt", "ext", "asymmetry", "back_scatt", "albedo"))}


def config5(ctx, args):
    """The large absorbing case at its stated size: the smooth hexagonal column
    r 50 um, L 100 um in 2 um^2 triangles (22,500, its 8 parent faces as
    apertures), n = 1.31 + 0.01i, --config5 orientations uniform on SO(3)
    (seed 55), 1441 theta x 720 phi.  Beam lists come from the host tracer
    (8 recursions, the reference's thresholds), traced chunk c+1 on the host
    cores while the GPU averages chunk c in FP32 (pbt_diff_batch_list_c); the
    whole loop is timed.  The FP32 average of the first --config5-fp64
    orientations is compared with their FP64 drop-in average."""
    from concurrent.futures import ThreadPoolExecutor
    import abt_b200
    from abt_b200 import tracer as T
    from abt_b200 import workloads as W
    from tests.helpers import mueller_rel_err
    g = W.hex_prism(50.0, 100.0, n_side=25, n_len=50, roughness=0.0, seed=5)
    P = T.Particle(g, g["apertures"])
    th = abt_b200.make_angles([0, 180], [0.125])
    ph = abt_b200.make_angles([0, 359.5], [0.5])
    nb = len(th) * len(ph)
    n = args.config5
    eul = W.uniform_euler(np.random.default_rng(55), n)
    chunk = 64
    geo = P.geometry

    def trace(s0):
        return T.trace_batch(P, eul[s0:s0 + chunk], LAM, 1.31, ibi=0.01)

    nout, per_orient, kept = [], [], None
    ctx.set_kernel_timing(True)
    ctx.kernel_time_ms()
    clocks = ClockSampler(ctx.device)
    clocks.start()
    t0 = time.perf_counter()
    with ThreadPoolExecutor(max_workers=1) as ex:
        starts = list(range(0, n, chunk))
        fut = ex.submit(trace, 0)
        for c, s0 in enumerate(starts):
            Vs, beams, exts, pins, _ = fut.result()
            if c + 1 < len(starts):
                fut = ex.submit(trace, starts[c + 1])
            r = ctx.diff_batch(beams, exts, Vs, geo, th, ph, LAM, pins, precision="fp32")
            nout += [len(b) + len(e) for b, e in zip(beams, exts)]
            per_orient.append(np.atleast_1d(r[3]))
            if c == 0:
                kept = (Vs, beams, exts, pins)
    t_all = time.perf_counter() - t0
    clk = clocks.stop()
    k_ms, k_n = ctx.kernel_time_ms()
    ctx.set_kernel_timing(False)
    F = np.array(nout, dtype=np.float64)
    work = float(F.sum()) * nb
    # FP32 against FP64 on the first orientations (the first chunk's lists)
    m = min(args.config5_fp64, len(kept[1]))
    Vs, beams, exts, pins = (x[:m] for x in kept)
    r32 = ctx.diff_batch(beams, exts, Vs, geo, th, ph, LAM, pins, precision="fp32")
    t0 = time.perf_counter()
    r64 = ctx.diff_batch(beams, exts, Vs, geo, th, ph, LAM, pins, precision="fp64")
    t64 = time.perf_counter() - t0
    sms = torch_sm_count()
    hz = (clk.get("sm_mhz") or 1965.0) * 1e6
    kern_s = k_ms / 1e3
    return {"workload": "smooth hexagonal column r 50 um, L 100 um, 2 um^2 triangles (22,500, "
                        "8 apertures), n = 1.31 + 0.01i, beam lists traced on the host (rec 8), "
                        "%d orientations uniform on SO(3), 1441 theta x 720 phi" % n,
            "orientations": n, "bins": nb,
            "outbeams_per_orientation": [int(F.min()), int(F.mean()), int(F.max())],
            "trace_and_fp32_average_s": t_all, "orientations_per_s": n / t_all,
            "facet_bin_per_s": work / t_all, "fp32_kernel_s": kern_s,
            "fp32_kernel_facet_bin_per_s": work / kern_s,
            "mufu_term_frac": W_SFU * work / kern_s / (sms * SFU_PER_SM_CLK * hz),
            "fp32_term_frac": W_FP32 * work / kern_s / (sms * FP32_PER_SM_CLK * hz),
            "roofline_basis": "convention per triangle facet-bin (20 MUFU, 170 FP32 flops) over "
                              "the summed kernel time; %d SMs x %.0f MHz (median sampled SM "
                              "clock of the loop)" % (sms, hz / 1e6),
            "clocks": clk,
            "error_subset_orientations": m, "fp64_dropin_subset_s": t64,
            "fp64_dropin_orientations_per_s": m / t64,
            "speedup_fp32_vs_fp64_dropin": (n / t_all) / (m / t64),
            "max_rel_mueller_err_vs_fp64_subset": mueller_rel_err(r32[0], r64[0], 1e-6),
            "mueller_err_above_1e-5_of_peak": mueller_rel_err(r32[0], r64[0], 1e-5),
            "max_rel_param_err_vs_fp64_subset": max(
                abs(float(r32[2][k]) - float(r64[2][k])) / abs(float(r64[2][k]))
                for k in ("scatt", "ext", "asymmetry", "albedo"))}


def torch_sm_count():
    import torch
    return torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count


def _worst_bin(mu, mu_ref, theta, thresh=1e-6):
    """theta (degrees) of the bin with the largest M11-normalised Mueller error
    above thresh of the peak M11, and that bin's M11 over the peak."""
    m11 = mu_ref[..., 0]
    sel = m11 > thresh * m11.max()
    e = np.where(sel, np.abs(mu - mu_ref).max(axis=-1) / np.where(sel, m11, 1.0), 0.0)
    i, j = np.unravel_index(np.argmax(e), e.shape)
    return [float(np.degrees(theta[j])), float(m11[i, j] / m11.max())]


def large_case(ctx, args):
    """The large-column workload: smooth hexagonal column r 50 um, L 100 um
    triangulated to 2 um^2 facets (22,500 triangles), stand-in beam lists of
    10-30 outgoing beams per facet (~460,000 outbeams per orientation), 1441
    theta x 720 phi (1,037,520 bins).  --large-orient orientations are averaged
    by one FP32 batch; the FP64 drop-in rate is sampled on 4,000 facets and
    the error is taken on the whole first orientation (FP64 drop-in over all
    of its outbeams, ~40 s)."""
    import abt_b200
    from abt_b200 import workloads as W
    from tests.helpers import mueller_rel_err
    geo = W.hex_prism(50.0, 100.0, n_side=25, n_len=50, roughness=0.0, seed=5)
    th = abt_b200.make_angles([0, 180], [0.125])
    ph = abt_b200.make_angles([0, 359.5], [0.5])
    nb = len(th) * len(ph)
    rng = np.random.default_rng(5)
    eul = W.uniform_euler(rng, args.large_orient)
    Vs, beams, exts = [], [], []
    pin = np.zeros(args.large_orient, dtype=abt_b200.PARAMS_DTYPE)
    for i, (a, b, c) in enumerate(eul):
        V, beam, ext, gcs = W.standin_orientation(geo, W.euler_rotation(a, b, c), rng,
                                                  n_internal=(10, 30))
        Vs.append(V)
        beams.append(beam)
        exts.append(ext)
        pin[i] = abt_b200.params(geo_cross_sec=gcs)
    F = np.array([len(b) + len(e) for b, e in zip(beams, exts)])
    ctx.diff_batch(beams[:1], [exts[0][:64]], Vs[:1], geo, th, ph, LAM, pin[:1], precision="fp32")
    ctx.set_kernel_timing(True)
    ctx.kernel_time_ms()
    t0 = time.perf_counter()
    ctx.diff_batch(beams, exts, Vs, geo, th, ph, LAM, pin, precision="fp32")
    t32 = time.perf_counter() - t0
    k_ms, k_n = ctx.kernel_time_ms()
    # FP64 drop-in rate on 4,000 facets over the full grid
    sub = beams[0][:4000]
    ctx.kernel_time_ms()
    ctx.diff_main(sub, None, dict(geo, verts=Vs[0]), th, ph, LAM, precision="fp64")
    k64_ms, _ = ctx.kernel_time_ms()
    ctx.set_kernel_timing(False)
    r64 = len(sub) * nb / (k64_ms / 1e3)
    # error on the whole first orientation
    g0 = dict(geo, verts=Vs[0])
    a32 = ctx.diff_main(beams[0], exts[0], g0, th, ph, LAM, precision="fp32")
    a64 = ctx.diff_main(beams[0], exts[0], g0, th, ph, LAM, precision="fp64")
    m32, _, p32 = ctx.finalise(a32[0], a32[1], th, ph, LAM, pin[0])
    m64, _, p64 = ctx.finalise(a64[0], a64[1], th, ph, LAM, pin[0])
    work = float(F.sum()) * nb
    return {"workload": "smooth hexagonal column r 50 um, L 100 um, 2 um^2 triangles (22,500), "
                        "stand-in beam lists (10-30 outgoing beams per facet), %d orientations, "
                        "1441 theta x 720 phi" % args.large_orient,
            "outbeams_per_orientation": [int(F.min()), int(F.mean()), int(F.max())], "bins": nb,
            "fp32_batched_s": t32, "fp32_orientations_per_s": args.large_orient / t32,
            "fp32_facet_bin_per_s": work / t32, "fp32_kernel_ms": k_ms,
            "fp32_kernel_facet_bin_per_s": work / (k_ms / 1e3),
            "fp64_dropin_facet_bin_per_s": r64,
            "fp64_dropin_orientations_per_s_extrapolated": r64 / (float(F.mean()) * nb),
            "speedup_fp32_batched_vs_fp64_dropin": (work / t32) / r64,
            "max_rel_mueller_err_vs_fp64_first_orientation": mueller_rel_err(m32, m64, 1e-6),
            "max_rel_param_err_vs_fp64_first_orientation": max(
                abs(float(p32[n]) - float(p64[n])) / abs(float(p64[n]))
                for n in ("scatt", "ext", "asymmetry"))}


def differentiation(ctx, args):
    """Gradients of the Mueller loss for a Gaussian-rough hexagonal plate
    (r 8 um, L 4 um, sigma 0.05 um, 20,808 triangles; stand-in beam lists),
    --diff-orient orientations, 181 theta x 90 phi: the target is the FP32
    forward of the geometry with N(0, 0.02^2) um vertex noise; each orientation
    runs the FP32 forward and the adjoint through torch.autograd.  On the first
    orientation the gradient is checked against FP64 central differences
    (h = 1e-5 um) of the loss of the FP64 drop-in."""
    import torch

    import abt_b200
    from abt_b200 import autograd as AG
    from abt_b200 import workloads as W
    geo = W.hex_prism(8.0, 4.0, n_side=34, n_len=17, roughness=0.05, seed=4)
    th = abt_b200.make_angles([0, 180], [1])
    ph = abt_b200.make_angles([0, 356], [4])
    rng = np.random.default_rng(4)
    eul = W.uniform_euler(rng, args.diff_orient)
    noise = rng.normal(0.0, 0.02, size=geo["verts"].shape)
    fwd_ms = adj_ms = wall = 0.0
    nrec = []
    fds = []
    for i, (a, b, c) in enumerate(eul):
        R = W.euler_rotation(a, b, c)
        V, beam, ext, _ = W.standin_orientation(geo, R, rng, n_internal=(0, 2))
        nrec.append(len(beam) + len(ext))
        tb, te = ctx.diff_main(beam, ext, dict(geo, verts=(geo["verts"] + noise) @ R.T), th, ph,
                               LAM, precision="fp32")
        t11, t12 = AG.mueller11_12(torch.from_numpy(tb), torch.from_numpy(te), LAM)
        g = dict(geo, verts=V)
        Vg = torch.tensor(V, requires_grad=True)
        ab = torch.tensor(beam["ampl"], requires_grad=True)
        ae = torch.tensor(ext["ampl"], requires_grad=True)
        ctx.set_kernel_timing(True)
        ctx.kernel_time_ms()
        t0 = time.perf_counter()
        afb, afe = AG.far_field(ctx, Vg, ab, ae, beam, ext, g, th, ph, LAM)
        f_ms, _ = ctx.kernel_time_ms()
        m11, m12 = AG.mueller11_12(afb, afe, LAM)
        AG.mueller_loss(m11, m12, t11, t12, th).backward()
        wall += time.perf_counter() - t0
        a_ms, _ = ctx.kernel_time_ms()
        ctx.set_kernel_timing(False)
        if i > 0:  # the first orientation warms up
            fwd_ms += f_ms
            adj_ms += a_ms
        if i < min(2, args.diff_orient) and args.fd_coords > 0:
            fds.append(_fd_check(ctx, geo, V, beam, ext, th, ph, t11, t12, Vg.grad.numpy(),
                                 ab.grad.numpy(), ae.grad.numpy(), np.random.default_rng(100 + i),
                                 args.fd_coords))
    n = max(1, args.diff_orient - 1)
    return {"workload": "rough hexagonal plate r 8 um, L 4 um, sigma 0.05 um (20,808 triangles), "
                        "stand-in beam lists, %d orientations, 181 theta x 90 phi, target from "
                        "0.02 um vertex noise" % args.diff_orient,
            "records_per_orientation": [int(min(nrec)), int(np.mean(nrec)), int(max(nrec))],
            "forward_kernel_ms_per_orientation": fwd_ms / n,
            "adjoint_kernel_ms_per_orientation": adj_ms / n,
            "adjoint_over_forward": adj_ms / fwd_ms if fwd_ms > 0 else None,
            "gradient_wall_ms_per_orientation": wall * 1e3 / args.diff_orient,
            "fd_checks_first_two_orientations": fds}


def _fd_check(ctx, geo, V, beam, ext, th, ph, t11, t12, gV, gb, ge, rng, ncoords, h=1e-5):
    """The adjoint's gradient of one orientation against FP64 central
    differences of the loss of the FP64 drop-in: ncoords random vertex
    coordinates of emitting facets one by one (only the outbeams on the moved
    vertex are recomputed, with pbt_diffraction_c), all 8 amplitude components of
    two beam and two external-diffraction outbeams, and four random directions
    in vertex space (relative to |grad| |direction|).  The drop-in keeps the
    reference's clamps (|kxx|, |kyy| >= 1e-6, edge slopes), its cancellation
    where kxx or kyy is small and its discontinuous frame choices (the
    anti-parallel flip, the frame flip of get_rotation_matrix2), so its loss has
    kinks and steps at a few vertices: each coordinate and each direction is
    differenced with steps h and h/10, and where the two differ by more than
    1e-4 of the largest gradient component (of |grad| for a direction) it is
    counted as not smooth and reported apart."""
    import torch
    from abt_b200 import autograd as AG

    def loss_of(A):
        p, q = AG.mueller11_12(torch.from_numpy(A), torch.from_numpy(np.zeros_like(A)), LAM)
        return float(AG.mueller_loss(p, q, t11, t12, th))

    ab, ae = ctx.diff_main(beam, ext, dict(geo, verts=V), th, ph, LAM, precision="fp64")
    A = ab + ae
    faces = geo["face_vi"].reshape(-1, 3) - 1
    allrec = np.concatenate([beam, ext])
    fi = allrec["fi"]
    used = np.unique(faces[fi - 1])
    gmax = np.abs(gV).max()

    one_face = {"face_off": np.array([0, 3], dtype=np.int64),
                "face_vi": np.array([1, 2, 3], dtype=np.int64)}

    def one(r, Vx):
        # the outbeam's facet alone, so that each call handles three vertices
        r1 = r.reshape(1).copy()
        f = int(r1["fi"][0]) - 1
        r1["fi"] = 1
        return ctx.diffraction(r1, dict(one_face, verts=Vx[faces[f]]), th, ph, LAM)

    def fd_coord(v, k, step):
        recs = allrec[np.any(faces[fi - 1] == v, axis=1)]
        Vp, Vm = V.copy(), V.copy()
        Vp[v, k] += step
        Vm[v, k] -= step
        dp = dm = 0.0
        for r in recs:
            a0 = one(r, V)
            dp = dp + one(r, Vp) - a0
            dm = dm + one(r, Vm) - a0
        return (loss_of(A + dp) - loss_of(A + dm)) / (2 * step)

    smooth_err, kink = [], []
    for v in rng.choice(used, ncoords):
        k = int(rng.integers(0, 3))
        d1, d2 = fd_coord(int(v), k, h), fd_coord(int(v), k, h / 10)
        if abs(d1 - d2) > 1e-4 * gmax:
            kink.append(abs(d1 - d2) / gmax)
        else:
            smooth_err.append(abs(d2 - gV[v, k]) / gmax)
    aerr = []
    for recs, g, j0 in ((beam, gb, 0), (ext, ge, len(beam))):
        for j in (0, len(recs) // 2):
            base = one(recs[j], V)
            for c in range(8):
                r2 = recs[j:j + 1].copy()
                r2["ampl"][0, c] += 1e-6
                dA = one(r2[0], V) - base
                d = (loss_of(A + dA) - loss_of(A - dA)) / 2e-6
                aerr.append(abs(d - g[j, c]) / np.abs(g).max())
    def fd_dir(dvec, step):
        lp = loss_of(sum(ctx.diff_main(beam, ext, dict(geo, verts=V + step * dvec), th, ph, LAM,
                                       precision="fp64")))
        lm = loss_of(sum(ctx.diff_main(beam, ext, dict(geo, verts=V - step * dvec), th, ph, LAM,
                                       precision="fp64")))
        return (lp - lm) / (2 * step)

    derr, dkink = [], []
    gnorm = np.linalg.norm(gV)
    for _ in range(4):
        dvec = rng.normal(size=V.shape)
        dvec /= np.linalg.norm(dvec)
        d1, d2 = fd_dir(dvec, h), fd_dir(dvec, h / 10)
        if abs(d1 - d2) > 1e-4 * gnorm:
            dkink.append(abs(d1 - d2) / gnorm)
        else:
            derr.append(abs(d2 - float((gV * dvec).sum())) / gnorm)
    return {"h_um": [h, h / 10], "vertex_coords": int(ncoords),
            "smooth_coords": len(smooth_err),
            "max_abs_err_over_max_grad_vertex_smooth": float(max(smooth_err)) if smooth_err else None,
            "not_smooth_coords": len(kink),
            "not_smooth_fd_spread_over_max_grad": [float(x) for x in sorted(kink)[-4:]],
            "ampl_components": len(aerr), "max_abs_err_over_max_grad_ampl": float(max(aerr)),
            "random_directions": 4, "smooth_directions": len(derr),
            "max_directional_err_over_grad_norm_smooth": float(max(derr)) if derr else None,
            "not_smooth_directions_fd_spread_over_grad_norm": [float(x) for x in dkink]}


def cpu_baseline(geo, beam, th, ph, seconds, nthreads):
    """The oracle (C FP64 restatement of diff_mod, the reference's OpenMP loop
    shape) on a bounded sample of the workload: the first n facets over the
    full far-field grid, n sized to about `seconds` of work."""
    from oracle import oracle as O
    nb = len(th) * len(ph)
    ext = np.zeros(0, dtype=O.OUTBEAM_DTYPE)
    n = max(nthreads, 2)
    t0 = time.perf_counter()
    O.diff_main(th, ph, LAM, geo, beam[:n], ext, nthreads=nthreads)
    dt = time.perf_counter() - t0
    n2 = int(min(len(beam), max(n, n * seconds / max(dt, 1e-3))))
    n2 = max(nthreads, (n2 // nthreads) * nthreads)
    t0 = time.perf_counter()
    O.diff_main(th, ph, LAM, geo, beam[:n2], ext, nthreads=nthreads)
    dt = time.perf_counter() - t0
    return {"value": n2 * nb / dt, "unit": UNIT, "cores": O.openmp_threads(nthreads), "kind": "port",
            "sample": "%d facets x %d bins (first facets of the workload), %.1f s" % (n2, nb, dt)}


def workload_config(nf, nb):
    """The `config` both arms print: the workload only, so that the two lines
    compare like for like (arm-specific details are keys of their own)."""
    return {"workload": "precision-study beam list: 200000 facets (2000 beams), 721 theta x 360 "
                        "phi, lambda 0.532 um",
            "facets": int(nf), "bins": int(nb), "orientations_per_step": 1,
            "l2": "GPU arm: a 256 MB buffer is written before every step, inside the timed "
                  "region; CPU arm: each step streams the facet list through the whole grid"}


def diffraction_call(ncalls):
    """The reference's -memory path calls diffraction once per outbeam
    (src/beam_loop_mod.f90:1935-1967) and adds each call's grid into its totals:
    the wall time of one call of pbt_diffraction_c and of pbt_diffraction_noalloc_c
    (FP64, one outbeam of the plain-method column, r 5 um, L 10 um, at Euler
    30, 40, 10 degrees, on its grid 181 x 180; host arrays in and out, the output
    arrays reused), over ncalls calls each."""
    import ctypes
    from abt_b200 import _lib
    from abt_b200 import workloads as W
    from abt_b200.diff import _geo
    L = _lib.lib()
    th, ph = W.grid_small()
    geo = W.hex_prism(5.0, 10.0, n_side=6, n_len=12)
    V, bl, _, _ = W.standin_orientation(geo, W.euler_rotation(*np.radians([30, 40, 10])),
                                        np.random.default_rng(1), n_internal=(0, 1))
    ob = np.ascontiguousarray(bl[:1])
    v, fo, fv = _geo(dict(geo, verts=V))
    out = np.zeros((len(ph), len(th), 2, 2), dtype=np.complex128, order="F")
    h = ctypes.c_void_p()
    _lib.check(L.pbt_ctx_create(0, ctypes.byref(h)))
    try:
        calls = {
            "pbt_diffraction_c": lambda: L.pbt_diffraction_c(
                h, ob.ctypes.data, v.ctypes.data, v.shape[0], fo.ctypes.data, fv.ctypes.data,
                len(fo) - 1, th.ctypes.data, len(th), ph.ctypes.data, len(ph), LAM, 0, out.ctypes.data),
            "pbt_diffraction_noalloc_c": lambda: L.pbt_diffraction_noalloc_c(
                ob.ctypes.data, v.ctypes.data, v.shape[0], fo.ctypes.data, fv.ctypes.data,
                len(fo) - 1, th.ctypes.data, len(th), ph.ctypes.data, len(ph), LAM, 0, out.ctypes.data),
        }
        res = {"grid": "181 theta x 180 phi (%d bins)" % (len(th) * len(ph)), "calls": ncalls,
               "particle": "hexagonal column r 5 um, L 10 um (%d triangles), one outbeam"
                           % (len(fo) - 1),
               "api": "host arrays in and out; the amplitude grid (%d bytes) copied back each call"
                      % out.nbytes}
        for name, f in calls.items():
            _lib.check(f())
            t = time.perf_counter()
            for _ in range(ncalls):
                _lib.check(f())
            res[name + "_ms"] = (time.perf_counter() - t) / ncalls * 1e3
        return res
    finally:
        L.pbt_ctx_destroy(h)


def fast_diff_kept_fraction(beam, geo, th, ph, sample=20000, tile_theta=8, tile_phi=16):
    """Fraction of (record, bin tile) pairs that the -fast_diff tile cull keeps,
    estimated on the host on the first `sample` records with the kernel's test:
    a record is skipped for a tile when the angle between its prop_out and the
    tile's centre exceeds fov + 2|com|/R + 1e-5 plus the tile's angular radius."""
    ob = beam[:sample]
    TH, PH = np.meshgrid(th, ph, indexing="ij")  # (ntheta, nphi)
    u = np.stack([np.sin(TH) * np.cos(PH), np.sin(TH) * np.sin(PH), -np.cos(TH)], -1)
    cen, psi = [], []
    for a in range(0, len(th), tile_theta):
        for b in range(0, len(ph), tile_phi):
            t = u[a:a + tile_theta, b:b + tile_phi].reshape(-1, 3)
            c = t.mean(0)
            c /= np.linalg.norm(c)
            cen.append(c)
            psi.append(np.arccos(np.clip(t @ c, -1, 1)).max())
    cen, psi = np.array(cen), np.array(psi)
    fo, fv, V = geo["face_off"], geo["face_vi"], geo["verts"]
    com = np.array([V[fv[fo[f - 1]:fo[f]] - 1].mean(0) for f in ob["fi"]])
    fovm = ob["fov"] + 2 * np.linalg.norm(com, axis=1) / 1e6 + 1e-5
    ang = np.arccos(np.clip(ob["prop_out"] @ cen.T, -1, 1))
    lim = fovm[:, None] + psi[None, :]
    kept = (lim >= np.pi) | (ang <= lim)
    return float(kept.mean())


def run_reference(args, world, rank):
    if rank != 0:
        return
    geo, beam, ext, th, ph = workload(args)
    nthreads = os.cpu_count() or 1
    nb = len(th) * len(ph)
    per_step = max(1.0, min(20.0, 60.0 / max(1, args.steps + args.warmup)))
    for _ in range(args.warmup):
        cpu_baseline(geo, beam, th, ph, 1.0, nthreads)
    vals = []
    last = None
    for _ in range(args.steps):
        last = cpu_baseline(geo, beam, th, ph, per_step, nthreads)
        vals.append(last["value"])
    value = statistics.mean(vals)
    ms = len(beam) * nb / value * 1e3
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 0,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": workload_config(len(beam), nb),
            "ms_per_step_basis": "extrapolated: the step's facet-bin count divided by the rate "
                                 "measured on each step's bounded facet sample",
            "cpu_baseline": dict(last, value=value),
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    world, rank, local, dist = dist_setup(args)
    if args.impl == "reference":
        run_reference(args, world, rank)
        if dist is not None:
            dist.destroy_process_group()
        return

    import torch

    import abt_b200
    from abt_b200.diff import diff_batch_dev
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    geo, beam, ext, th, ph = workload(args)
    nf = len(beam)
    nb = len(th) * len(ph)
    nverts = geo["verts"].shape[0]
    work = float(nf) * nb  # facet x bin evaluations per step (one orientation)

    ctx = abt_b200.Context(local)
    # device-resident inputs
    d_beam = torch.from_numpy(beam.view(np.uint8).copy()).to(dev)
    d_ext = torch.empty(128, dtype=torch.uint8, device=dev)
    d_verts = torch.from_numpy(np.asfortranarray(geo["verts"]).ravel(order="F").copy()).to(dev)
    d_fvi = torch.from_numpy(geo["face_vi"].copy()).to(dev)
    pin = np.zeros(1, dtype=abt_b200.PARAMS_DTYPE)
    pin["geo_cross_sec"] = 1.0
    pin["beam_energy_out"] = 1.0
    pin["ext_energy_out"] = 1.0
    d_pin = torch.from_numpy(pin.view(np.uint8).copy()).to(dev)
    d_mu = torch.empty(16 * nb, dtype=torch.float64, device=dev)
    d_m1 = torch.empty(16 * len(th), dtype=torch.float64, device=dev)
    d_pav = torch.empty(18, dtype=torch.float64, device=dev)
    d_pper = torch.empty(18, dtype=torch.float64, device=dev)
    boff = np.array([0, nf], dtype=np.int64)
    eoff = np.array([0, 0], dtype=np.int64)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)  # > 126 MB L2
    stream = torch.cuda.current_stream(dev)

    def direct():
        diff_batch_dev(ctx, stream.cuda_stream, 1, d_beam, boff, d_ext, eoff, d_verts, nverts,
                       geo["face_off"], d_fvi, th, ph, LAM, d_pin, d_mu, d_m1, d_pav, d_pper)

    # launch plan (variant x bins per thread x records per item) tuned on the step's
    # own facet list (a smaller sample has fewer facet splits per bin tile, which
    # favours smaller work items than the full list wants)
    plan = {"plan": "default (1, 1, 2048)"}
    if not args.no_tune:
        from abt_b200.tune import tune
        best, times = tune(ctx, beam, geo, th, ph, LAM, sample_facets=len(beam), repeats=1)
        plan = {"plan": list(best), "candidates_kernel_ms_%d_facets" % len(beam):
                {"%d,%d,%d" % k: round(v, 3) for k, v in times.items()}}

    # the step: one replay of the batch captured as a CUDA graph (the capture
    # runs the batch once); --no-graph enqueues it through the C ABI instead
    graph = None
    if not args.no_graph:
        from abt_b200.diff import BatchGraph
        graph = BatchGraph(ctx, stream.cuda_stream, 1, d_beam, boff, d_ext, eoff, d_verts, nverts,
                           geo["face_off"], d_fvi, th, ph, LAM, d_pin, d_mu, d_m1, d_pav, d_pper)
        step_kernels = graph.kernel_count()

        def step():
            graph.launch(stream.cuda_stream)
    else:
        step = direct

    for _ in range(max(3, args.warmup)):
        flush.zero_()
        step()
    torch.cuda.synchronize()
    # kernel time of the far-field kernel (CUDA events inside the library), same
    # conditions as a step: L2 flushed before each call
    ctx.set_kernel_timing(True)
    ctx.kernel_time_ms()
    for _ in range(2):
        flush.zero_()
        direct()
    torch.cuda.synchronize()
    kern_ms, kern_n = ctx.kernel_time_ms()
    ctx.set_kernel_timing(False)
    if dist is not None:
        dist.barrier()
    clocks = ClockSampler(local)
    clocks.start()
    launches = 0
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(args.steps):
        flush.zero_()
        step()
        launches += step_kernels if graph is not None else ctx.last_launch_count()
    e1.record(stream)
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    clk = clocks.stop()
    ms_total = e0.elapsed_time(e1)
    if graph is not None:
        graph.close()
    ms_total = max_over_ranks(dist, ms_total, dev)
    ms_step = ms_total / args.steps
    value = replicas_value(world, work, ms_step)

    extra = {}
    # Beyond the timed step, e2e and the roofline, the sections are single-GPU
    # measurements: they run in the N = 1 run only, so that an N-GPU run holds
    # its GPUs for the step alone.
    solo = world == 1
    # end to end through the host C ABI with pinned host buffers
    pinned_beam = torch.from_numpy(beam.view(np.uint8).copy()).pin_memory()
    pb = pinned_beam.numpy().view(abt_b200.OUTBEAM_DTYPE)
    pverts = torch.from_numpy(np.asfortranarray(geo["verts"]).copy()).pin_memory().numpy()
    pverts = np.asfortranarray(pverts.reshape(geo["verts"].shape))
    def pinned_like(a, order="C"):
        t = torch.empty(a.size, dtype=torch.float64 if a.dtype == np.float64 else torch.int64,
                        pin_memory=True).numpy()
        return t.reshape(a.shape, order=order)

    pfo = pinned_like(np.asarray(geo["face_off"], dtype=np.int64))
    pfo[...] = geo["face_off"]
    pfv = pinned_like(np.asarray(geo["face_vi"], dtype=np.int64))
    pfv[...] = geo["face_vi"]
    geo_p = dict(geo, verts=pverts, face_off=pfo, face_vi=pfv)
    # the Mueller outputs go to pinned host arrays owned by the caller
    pmu = pinned_like(np.empty((len(ph), len(th), 16)), order="F")
    pmu1 = pinned_like(np.empty((len(th), 16)), order="F")
    out = ctx.diff_batch([pb], [np.zeros(0, abt_b200.OUTBEAM_DTYPE)], [pverts], geo_p, th, ph, LAM,
                         pin, precision="fp32", out=(pmu, pmu1))
    t0 = time.perf_counter()
    for _ in range(args.e2e_steps):
        out = ctx.diff_batch([pb], [np.zeros(0, abt_b200.OUTBEAM_DTYPE)], [pverts], geo_p, th, ph,
                             LAM, pin, precision="fp32", out=(pmu, pmu1))
    e2e_s = max_over_ranks(dist, (time.perf_counter() - t0) / args.e2e_steps, dev)
    h2d = beam.nbytes + geo["verts"].nbytes + geo["face_off"].nbytes + geo["face_vi"].nbytes + pin.nbytes
    d2h = 16 * nb * 8 + 16 * len(th) * 8 + 2 * pin.nbytes
    e2e = {"value": world * work / e2e_s, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
           "d2h_bytes_per_step": int(d2h), "ms_per_step": e2e_s * 1e3,
           "api": "pbt_diff_batch_list_c (host pointers; inputs and Mueller outputs pinned)"}
    # the tuned plan is the step's; the further workloads (other facet counts and
    # grids) use the library's default, which sizes the work items per call
    ctx.set_plan()

    # reference-exact FP64 drop-in rate on a facet sample
    if args.fp64_facets > 0 and solo:
        sub = beam[:args.fp64_facets]
        ctx.diff_main(sub[:64], None, geo, th, ph, LAM, precision="fp64")
        ctx.set_kernel_timing(True)
        ctx.kernel_time_ms()
        t0 = time.perf_counter()
        ctx.diff_main(sub, None, geo, th, ph, LAM, precision="fp64")
        wall = time.perf_counter() - t0
        k64_ms, _ = ctx.kernel_time_ms()
        ctx.set_kernel_timing(False)
        r64 = len(sub) * nb / (k64_ms / 1e3)
        extra["fp64_dropin"] = {"value": r64, "unit": UNIT, "facets": int(len(sub)),
                                "kernel_ms": k64_ms, "call_ms": wall * 1e3,
                                "e2e_value": len(sub) * nb / wall}
        extra["fp32_vs_fp64_kernel_speedup"] = (work / (kern_ms / max(kern_n, 1) / 1e3)) / r64

    # adjoint (vector-Jacobian product) against the forward, same facets and grid
    if args.adjoint_facets > 0 and solo:
        sub = beam[:args.adjoint_facets]
        rng = np.random.default_rng(1)
        shape = (len(ph), len(th), 2, 2)
        gA = rng.normal(size=shape) + 1j * rng.normal(size=shape)
        gZ = np.zeros(shape, np.complex128)
        ctx.diff_main(sub, None, geo, th, ph, LAM, precision="fp32")
        ctx.diff_adjoint(sub[:64], None, geo, th, ph, LAM, gA, gZ)
        ctx.set_kernel_timing(True)
        ctx.kernel_time_ms()
        ctx.diff_main(sub, None, geo, th, ph, LAM, precision="fp32")
        fwd_ms, _ = ctx.kernel_time_ms()
        t0 = time.perf_counter()
        ctx.diff_adjoint(sub, None, geo, th, ph, LAM, gA, gZ)
        adj_call = time.perf_counter() - t0
        adj_ms, _ = ctx.kernel_time_ms()
        ctx.set_kernel_timing(False)
        extra["adjoint"] = {"facets": int(len(sub)), "bins": nb, "forward_kernel_ms": fwd_ms,
                            "adjoint_kernel_ms": adj_ms, "adjoint_over_forward": adj_ms / fwd_ms,
                            "adjoint_call_ms": adj_call * 1e3,
                            "value": len(sub) * nb / (adj_ms / 1e3), "unit": UNIT}

    if args.orient > 0 and solo:
        extra["orientation_average"] = orientation_average(ctx, args)
    if args.traced_orient > 0 and solo:
        extra["orientation_average_traced"] = traced_orientation_average(ctx, args)

    if args.diff_orient > 0 and solo:
        extra["differentiation"] = differentiation(ctx, args)
    if args.large_orient > 0 and solo:
        extra["large_column"] = large_case(ctx, args)
    if args.large_traced_orient > 0 and solo:
        extra["large_column_traced"] = large_traced(ctx, args)
    if args.config5 > 0 and solo:
        extra["large_column_config5"] = config5(ctx, args)

    # -fast_diff: the same workload with the field-of-view test (fov = 8 lambda / d);
    # error against the FP64 drop-in with is_fast_diff on the first 20,000 facets
    if args.fast_diff and solo:
        ctx.diff_main(beam[:64], None, geo, th, ph, LAM, is_fast_diff=True, precision="fp32")
        ctx.set_kernel_timing(True)
        ctx.kernel_time_ms()
        flush.zero_()
        ctx.diff_main(beam, None, geo, th, ph, LAM, is_fast_diff=True, precision="fp32")
        kf_ms, _ = ctx.kernel_time_ms()
        ctx.set_kernel_timing(False)
        sub = beam[:20000]
        from tests.helpers import mueller_rel_err
        a32 = ctx.diff_main(sub, None, geo, th, ph, LAM, is_fast_diff=True, precision="fp32")
        a64 = ctx.diff_main(sub, None, geo, th, ph, LAM, is_fast_diff=True, precision="fp64")
        m32, _, _ = ctx.finalise(a32[0], a32[1], th, ph, LAM, pin[0])
        m64, _, _ = ctx.finalise(a64[0], a64[1], th, ph, LAM, pin[0])
        kept = fast_diff_kept_fraction(beam, geo, th, ph)
        extra["fast_diff"] = {"kernel_ms": kf_ms, "value": work / (kf_ms / 1e3), "unit": UNIT,
                              "value_basis": "effective: every facet-bin of the workload over "
                                             "the kernel time, culled pairs included",
                              "kept_pair_fraction": kept,
                              "evaluated_value": kept * work / (kf_ms / 1e3),
                              "evaluated_basis": "facet-bins of the (record, tile) pairs the "
                                                 "cull keeps (fraction estimated on the host on "
                                                 "20,000 records) over the kernel time",
                              "speedup_vs_full_kernel": (kern_ms / max(kern_n, 1)) / kf_ms,
                              "max_rel_mueller_err_vs_fp64_fast_20000_facets":
                                  mueller_rel_err(m32, m64, 1e-6),
                              "cull": "records whose field of view misses a 8x16 (theta x phi) "
                                      "bin tile are skipped for that tile"}

    if args.diffraction_calls > 0 and solo:
        extra["diffraction_call"] = diffraction_call(args.diffraction_calls)

    # FP32 error against the FP64 drop-in on the full workload
    if not args.no_error_check and solo:
        from tests.helpers import mueller_rel_err
        f64 = ctx.diff_batch([beam], [np.zeros(0, abt_b200.OUTBEAM_DTYPE)], [geo["verts"]], geo,
                             th, ph, LAM, pin, precision="fp64")
        mu32 = d_mu.cpu().numpy().reshape(16, len(th), len(ph)).transpose(2, 1, 0)
        extra["max_rel_mueller_err_vs_fp64"] = mueller_rel_err(mu32, f64[0], 1e-6)
        extra["max_rel_param_err_vs_fp64"] = max(
            abs(float(out[2][n]) - float(f64[2][n])) / abs(float(f64[2][n]))
            for n in ("scatt", "asymmetry", "ext"))

    # roofline of the dominant kernel (k2_main_pk_kernel)
    kms = kern_ms / max(kern_n, 1)
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    mhz = clk.get("sm_mhz") or 1965.0
    traffic = None
    prof = os.path.join(ROOT, "profiles", "k2_main_traffic.json")
    if os.path.exists(prof):
        try:
            traffic = json.load(open(prof)).get("dram_bytes_per_launch_full")
        except Exception:
            traffic = None
    # binding term of t_roof = work x max(W_FP32/P_FP32, W_SFU/P_SFU, W_FP64/P_FP64)
    hz = mhz * 1e6
    terms = {}
    for name, w, per_clk, unit in (("fp32", W_FP32, FP32_PER_SM_CLK, "TFLOP/s"),
                                   ("mufu", W_SFU, SFU_PER_SM_CLK, "Tops/s"),
                                   ("fp64", W_FP64, FP64_PER_SM_CLK, "TFLOP/s")):
        a_ = w * work / (kms / 1e3)
        p_ = sms * per_clk * hz
        terms[name] = {"achieved": a_ / 1e12, "peak": p_ / 1e12, "unit": unit, "frac": a_ / p_,
                       "per_facet_bin": w}
    bound = max(terms, key=lambda n: terms[n]["frac"])
    # what the hardware actually runs (ncu counters of the same kernel on the
    # 20,000-facet case): MUFU ops issued per facet-bin and the pipe loads
    counters = None
    cprof = os.path.join(ROOT, "profiles", "k2_main_pk_counters.json")
    if os.path.exists(cprof):
        try:
            cj = json.load(open(cprof))
            mi = float(cj["mufu_instructions_per_facet_bin"])
            counters = {"mufu_issued_per_facet_bin": mi,
                        "xu_frac_issued": terms["mufu"]["frac"] * mi / W_SFU,
                        "issue_active": cj["issue_active"],
                        "fma_pipe_cycles_active": cj["fma_pipe_cycles_active"],
                        "thread_instructions_per_facet_bin": cj["thread_instructions_per_facet_bin"],
                        "limiter": "the FMA pipe (%.0f %% of cycles; a packed FP32x2 instruction "
                                   "holds it two cycles) and instruction issue (%.0f %%); the "
                                   "convention's MUFU term counts 20 special-function ops per "
                                   "facet-bin where the kernel issues %.1f"
                                   % (100 * cj["fma_pipe_cycles_active"], 100 * cj["issue_active"], mi),
                        "source": "profiles/k2_main_pk_counters.json (ncu)"}
        except Exception:
            counters = None
    roof = {"bound": bound, "achieved": terms[bound]["achieved"], "peak": terms[bound]["peak"],
            "unit": terms[bound]["unit"], "frac": terms[bound]["frac"], "traffic": traffic,
            "kernel": "k2_main_pk_kernel", "kernel_ms": kms, "units_per_launch": work,
            "terms": terms, "issued": counters,
            "peak_basis": "%d SMs x %.0f MHz (median sampled SM clock) x per-clock issue width "
                          "(FP32 128 lanes, MUFU 16, FP64 64); MEASURED_PEAKS.json has no "
                          "FP32/MUFU/FP64 figure" % (sms, mhz)}

    cpu = None
    if solo and not args.no_cpu_baseline:
        cpu = cpu_baseline(geo, beam, th, ph, args.cpu_seconds, os.cpu_count() or 1)
        # the single-thread path (the reference's seq build at -mt 0)
        cpu["single_thread"] = cpu_baseline(geo, beam, th, ph, args.cpu_seconds / 2, 1)
        if "diffraction_call" in extra:
            # the same call's work on one host core at the single-thread baseline's rate
            extra["diffraction_call"]["cpu_1thread_ms_from_cpu_baseline"] = \
                181 * 180 / cpu["single_thread"]["value"] * 1e3

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": workload_config(nf, nb),
            "precision": "FP32 with FP64 phase",
            "parallelism": "replicas" if world > 1 else "single GPU",
            "step": "CUDA graph replay of pbt_diff_batch_dev_c" if not args.no_graph
                    else "pbt_diff_batch_dev_c",
            "launch_plan": plan,
            "orientations_per_s": world * 1e3 / ms_step,
            "clocks": clk, "e2e": e2e, "gpu_launches": launches, "roofline": roof,
            "cpu_baseline": cpu}
    line.update(extra)
    if rank == 0:
        print(json.dumps(line), flush=True)
    ctx.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
