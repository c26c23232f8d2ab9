"""bench.py's multi-process plumbing on CPU, world size 2.

The path does not shard (every rank runs an independent replica of the whole node set), so
the only cross-rank steps are the host's: the process group, the barrier around the timed
region and the maximum of the ranks' times.  Here they run under the gloo backend in two
spawned processes, and the reference arm runs under torchrun with two ranks, of which rank 0
alone measures and prints its one line.
"""
import json
import os
import socket
import subprocess
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, port, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE="2", LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import bench
    ws, r, local = bench.dist_env()
    dist = bench.init_pg(ws, "gloo")
    try:
        dist.barrier()
        m = bench.max_over_ranks(dist, 1.5 + r)
        dist.barrier()
        out.put((r, ws, local, m))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_under_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_rank, args=(r, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(180)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    got = sorted(q.get(timeout=10) for _ in range(2))
    assert got == [(0, 2, 0, 2.5), (1, 2, 1, 2.5)]


def test_reference_arm_under_torchrun_prints_one_line():
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2", "--master-addr",
           "127.0.0.1", "--master-port", str(free_port()), "bench.py", "--impl", "reference", "--gpus", "2",
           "--workload", "periodic-di-o4-16k", "--steps", "1", "--warmup", "1"]
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["cpu_baseline"]["kind"] == "port"
