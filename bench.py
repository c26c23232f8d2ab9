#!/usr/bin/env python
"""RK3 node-steps/s of the LABFM time step on B200 (one JSON line on rank 0).

Workload (default): the doubly periodic 512x512 jittered node set (262,144 nodes), LABFM
order 6, sPTT (eps=0.25) in log-conformation form, FP64 - the configuration the metric is
quoted on.  One step = one step_rk3_4S_2R_EE: four right-hand sides with their stencils,
the low-storage RK update with the error norm, the hyperviscous filter and the mass
correction.  Inputs are seeded synthetic node sets (no dataset exists for this path).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--workload NAME] [--precision fp64|mixed]
  python bench.py --impl reference ...   (the CPU restatement of the reference, all host cores)

For N>1 (torchrun) every rank runs an independent replica on its own GPU (the path has no
exchange step on one node set); value = all ranks' node-steps / the slowest rank's time.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from sunset_viscoelastic_b200.nodesets import WORKLOADS, initial_state  # noqa: E402

METRIC = "RK3 node-steps/s"
DEFAULT_WORKLOAD = "periodic-lc-o6-262k"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=200)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--workload", default=DEFAULT_WORKLOAD, choices=sorted(WORKLOADS))
    p.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    p.add_argument("--no-cpu-baseline", action="store_true")
    return p.parse_args()


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def init_pg(ws, backend):
    if ws <= 1:
        return None
    import datetime

    import torch.distributed as dist
    os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
    dist.init_process_group(backend=backend, timeout=datetime.timedelta(seconds=300))
    return dist


def max_over_ranks(dist, x, device=None):
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def dt_for(wl, dtc, dtp):
    return wl.cfl * min(dtc, dtp)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.out = os.path.join("/tmp", f"sunset_clocks_{os.getpid()}.csv")

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.out, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        try:
            rows = [r.split(",") for r in open(self.out).read().strip().splitlines() if r.strip()]
        except OSError:
            return None
        sm, smax, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            r = [c.strip() for c in r]
            if len(r) < 9:
                continue
            try:
                sm.append(float(r[1]))
                smax = max(smax, float(r[2]))
            except ValueError:
                continue
            for k, name in enumerate(names):
                if r[5 + k].lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profiled_traffic(workload):
    """dram bytes per stage-kernel launch from the committed ncu summary, if present."""
    path = os.path.join(ROOT, "profiles", "stage_kernel_traffic.md")
    try:
        for line in open(path):
            if line.startswith(f"traffic_bytes_per_launch[{workload}]:"):
                return float(line.split(":", 1)[1].split()[0])
    except OSError:
        pass
    return None


def cpu_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def oracle_setup(wl, ns, gpu=None):
    """The CPU restatement on the workload; weights built on the host (or taken from the
    device build, which is bit-identical up to libm, to keep the sample bounded)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    O.set_threads(cpu_threads())
    o = O.for_workload(wl, ns)
    if gpu is None:
        o.setup()
    else:
        cnt, cs, links = gpu.neighbours()
        o.set_neighbours_weights(cnt, cs, links, gpu.weights())
    o.set_state(**initial_state(ns))
    return o


def run_reference(args, ws, rank):
    """--impl reference: the CPU restatement of the reference path on all host cores."""
    wl = WORKLOADS[args.workload]
    if rank != 0:
        return 0
    ns = wl.nodes()
    t0 = time.time()
    o = oracle_setup(wl, ns)
    setup_s = time.time() - t0
    dtc, dtp = o.set_tstep()
    dt = dt_for(wl, dtc, dtp)
    # bounded sample: each timed "step" is one full RK step of the whole node set
    warm = max(1, min(args.warmup, 2))
    nsteps = max(1, min(args.steps, 20))
    o.step(dt, warm)
    t = time.perf_counter()
    o.step(dt, nsteps)
    el = time.perf_counter() - t
    value = ns.n * nsteps / el
    line = {"metric": METRIC, "value": value, "unit": "node-steps/s", "impl": "reference", "n_gpus": args.gpus,
            "steps": nsteps, "warmup": warm, "ms_per_step": 1e3 * el / nsteps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded jittered lattice)",
            "config": {"workload": wl.name, "nodes": ns.n, "order": wl.order, "form": wl.form,
                       "radius_over_s": round(wl.radius_over_s, 4), "cfl": wl.cfl},
            "cpu_baseline": {"value": value, "unit": "node-steps/s", "cores": cpu_threads(), "kind": "port",
                             "sample": f"{nsteps} RK steps of the full {ns.n}-node set after {warm} warm-up steps "
                                       f"(host weight build {setup_s:.1f}s untimed)"},
            "e2e": {"value": value, "unit": "node-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse()
    ws, rank, local = dist_env()
    if args.impl == "reference":
        return run_reference(args, ws, rank)
    import torch
    from sunset_viscoelastic_b200 import labfm
    torch.cuda.set_device(local)
    dist = init_pg(ws, "nccl")
    wl = WORKLOADS[args.workload]
    ns = wl.nodes()
    g = labfm.for_workload(wl, ns, precision=args.precision, device=local).setup()
    g.set_state(**initial_state(ns))
    dtc, dtp = g.set_tstep()
    dt = dt_for(wl, dtc, dtp)
    g.step(dt, args.warmup)
    g.synchronize()
    if dist:
        dist.barrier()
    with ClockSampler(local) as clk:
        ms = g.step_timed(dt, args.steps)
    if dist:
        dist.barrier()
    ms_max = max_over_ranks(dist, ms, device=f"cuda:{local}")
    value = ws * ns.n * args.steps / (ms_max * 1e-3)

    # kernel roofline: the RK stage kernel, timed alone with CUDA events on its stream
    stage_ms, stage_bytes = g.time_stage_kernel(20)
    peak, peak_kind = measured_peaks()
    achieved = stage_bytes / (stage_ms * 1e-3) / 1e9
    traffic = profiled_traffic(wl.name)
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": traffic, "kernel": "k_stage (one RK stage: stencils + rhs + update)",
                "algorithmic_bytes_per_launch": stage_bytes, "launch_ms": stage_ms, "peak_source": peak_kind}

    # end to end through the C-ABI with host buffers: per step, copy the evolved fields in
    # from pinned host memory, run the step, copy them back
    n = ns.n
    st_in = torch.empty(7 * n, dtype=torch.float64, pin_memory=True)
    st_out = torch.empty(7 * n, dtype=torch.float64, pin_memory=True)
    s = g.state()
    q = ["cxx", "cxy", "cyy", "czz"] if wl.form == "di" else ["psixx", "psixy", "psiyy", "psizz"]
    st_in.copy_(torch.from_numpy(np.concatenate([s["ro"], s["rou"], s["rov"]] + [s[k] for k in q])))
    e2e_steps = max(3, min(args.steps, 50))
    g.run_host(st_in.data_ptr(), dt, 1, st_out.data_ptr())
    if dist:
        dist.barrier()
    t = time.perf_counter()
    for _ in range(e2e_steps):
        g.run_host(st_in.data_ptr(), dt, 1, st_out.data_ptr())
        st_in, st_out = st_out, st_in
    el = time.perf_counter() - t
    el = max_over_ranks(dist, el, device=f"cuda:{local}")
    e2e = {"value": ws * n * e2e_steps / el, "unit": "node-steps/s", "h2d_bytes_per_step": 7 * 8 * n,
           "d2h_bytes_per_step": 7 * 8 * n}

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        o = oracle_setup(wl, ns, gpu=g)
        o.step(dt, 1)
        k = 3
        t = time.perf_counter()
        o.step(dt, k)
        el = time.perf_counter() - t
        cpu = {"value": n * k / el, "unit": "node-steps/s", "cores": cpu_threads(), "kind": "port",
               "sample": f"{k} RK steps of the full {n}-node set (weights from the device build)"}

    launches_per_step = 7
    line = {"metric": METRIC, "value": value, "unit": "node-steps/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64" if args.precision == "fp64" else "f32+f64",
            "data": "synthetic (seeded jittered lattice)",
            "config": {"workload": wl.name, "nodes": n, "order": wl.order, "form": wl.form,
                       "radius_over_s": round(wl.radius_over_s, 4), "cfl": wl.cfl, "precision": args.precision,
                       "l2": "working set larger than L2 (weights)", "parallelism": f"replicas x{ws}"},
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e,
            "gpu_launches": launches_per_step * args.steps,
            "clocks": clk.summary()}
    if rank == 0:
        print(json.dumps(line), flush=True)
    g.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
