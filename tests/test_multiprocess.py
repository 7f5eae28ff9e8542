"""The N > 1 path of bench.py on CPU: gloo ranks (world size 2) for the
max-over-ranks timing, and the reference arm under torchrun, where rank 0
alone prints the line and every rank exits 0."""
import json
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    ms = bench.max_over_ranks(dist, 100.0 + 50.0 * rank, torch.device("cpu"))
    q.put((rank, ms, bench.replicas_value(world, 1e9, ms)))
    dist.barrier()
    dist.destroy_process_group()


def test_max_over_ranks_gloo():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, ms, value in out:
        assert ms == 150.0                      # every rank sees the slowest rank's time
        assert value == pytest.approx(2 * 1e9 / 0.150)


def test_reference_arm_under_torchrun():
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), "bench.py", "--impl",
           "reference", "--gpus", "2", "--steps", "1", "--warmup", "1", "--beams", "4",
           "--facets-per-beam", "10"]
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["value"] > 0 and d["cpu_baseline"]["kind"] == "port"
    # the same `config` as the GPU arm prints for this workload (40 facets, 721 x 360 bins)
    sys.path.insert(0, ROOT)
    import bench
    assert d["config"] == bench.workload_config(40, 721 * 360)
    assert "extrapolated" in d["ms_per_step_basis"]
