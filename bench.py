#!/usr/bin/env python
"""RK3 node-steps/s of the LABFM time step on B200 (one JSON line on rank 0).

Workload (default): the doubly periodic 1024x1024 jittered node set (1,048,576 nodes), LABFM
order 8, Oldroyd-B (Wi 2, beta 0.1) in Cholesky form - the precision configuration the metric
compares, and the largest that fits one GPU.  The headline `value` is the FP64 drop-in; the
line also carries
  * `mixed`: the mixed-precision step on the same set (node-steps/s, speed-up over FP64, its
    stage-kernel roofline, and the per-field error against the FP64 path after
    --error-steps steps);
  * `setup`: the device build of neighbours and weights (seconds, nodes/s) and the CPU
    restatement's build of the same order and radius on a bounded sample of nodes;
  * `adjoint`: the adjoint/forward cost of sunset_adjoint_run on the differentiation workload
    (262,144 nodes, order 6, log-conformation, 200 steps, checkpoints every 20), and the same
    with all 200 steps recorded in HBM (no recomputation); its finite-difference checks run
    with `--adjoint --fd-check`.
One step = one step_rk3_4S_2R_EE: four right-hand sides with their stencils, the low-storage
RK update with the error norm, the hyperviscous filter and the mass correction.  Inputs are
seeded synthetic node sets (no dataset exists for this path).

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

from sunset_viscoelastic_b200.nodesets import WORKLOADS  # noqa: E402

METRIC = "RK3 node-steps/s"
DEFAULT_WORKLOAD = "periodic-chl-o8-1m"
ADJOINT_WORKLOAD = "periodic-lc-o6-262k-adjoint"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=200)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--workload", default=DEFAULT_WORKLOAD, choices=sorted(WORKLOADS))
    p.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--layers", type=float, default=0.0,
                   help="3-D (-Ddim3): stack the workload's node set (at --nside per side) in z over this L_domain_z")
    p.add_argument("--nside", type=int, default=128, help="--layers: nodes per side of each layer")
    p.add_argument("--error-steps", type=int, default=100,
                   help="mixed precision: steps from the initial state for the per-field error report")
    p.add_argument("--no-error-check", action="store_true")
    p.add_argument("--adjoint", action="store_true",
                   help="time sunset_adjoint_run against the forward run (differentiation workload by default)")
    p.add_argument("--checkpoint", type=int, default=20, help="--adjoint: checkpoint every N steps")
    p.add_argument("--fd-check", action="store_true",
                   help="--adjoint: check dJ/dWi, dJ/dbeta and 8 Gaussian psi0 directions by central differences")
    p.add_argument("--no-mixed", action="store_true", help="leave out the mixed-precision block")
    p.add_argument("--no-adjoint", action="store_true", help="leave out the adjoint cost block")
    p.add_argument("--no-setup", action="store_true", help="leave out the setup block")
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
    """SM clock, its maximum and the active throttle reasons, sampled every 5 ms during the
    timed region through NVML (read-only queries; the same counters nvidia-smi prints).
    Falls back to nvidia-smi at 200 ms where NVML is unavailable."""

    NAMES = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
    MASKS = (0x8, 0x40, 0x20, 0x4)  # nvmlClocksEventReason* bits
    SMI_FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                  "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                  "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, cuda_device, period=0.005):
        self.dev = cuda_device
        self.period = period
        self.rows = []  # (sm_mhz, sm_max_mhz, reasons bitmask)
        self.proc = None
        self.thread = None
        self.stop = False
        self.source = None

    def _nvml_handle(self):
        import pynvml
        pynvml.nvmlInit()
        try:
            import torch
            props = torch.cuda.get_device_properties(self.dev)
            return pynvml, pynvml.nvmlDeviceGetHandleByUUID(f"GPU-{props.uuid}")
        except Exception:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.dev)

    def __enter__(self):
        import threading
        try:
            nv, h = self._nvml_handle()
            smax = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)

            def loop():
                while not self.stop:
                    try:
                        sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                        rs = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                        self.rows.append((float(sm), float(smax), int(rs)))
                    except Exception:
                        pass
                    time.sleep(self.period)

            self.thread = threading.Thread(target=loop, daemon=True)
            self.thread.start()
            self.source = f"nvml {self.period * 1e3:g} ms"
        except Exception:
            self.out = os.path.join("/tmp", f"sunset_clocks_{os.getpid()}.csv")
            try:
                self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.SMI_FIELDS}",
                                              "--format=csv,noheader,nounits", "-lms", "200"],
                                             stdout=open(self.out, "w"), stderr=subprocess.DEVNULL)
                self.source = "nvidia-smi 200 ms"
            except OSError:
                self.proc = None
        return self

    def __exit__(self, *a):
        self.stop = True
        if self.thread is not None:
            self.thread.join(timeout=5)
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            try:
                for r in open(self.out).read().strip().splitlines():
                    r = [c.strip() for c in r.split(",")]
                    if len(r) < 9:
                        continue
                    mask = 0
                    for k, m in enumerate(self.MASKS):
                        if r[5 + k].lower().startswith("active"):
                            mask |= m
                    self.rows.append((float(r[1]), float(r[2]), mask))
            except (OSError, ValueError):
                pass

    def summary(self):
        if not self.rows:
            return None
        sm = [r[0] for r in self.rows]
        reasons = sorted({n for r in self.rows for n, m in zip(self.NAMES, self.MASKS) if r[2] & m})
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": max(r[1] for r in self.rows), "reasons": reasons,
                "samples": len(sm), "source": self.source}


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profiled_traffic(workload, precision):
    """DRAM bytes (read + write) per stage-kernel launch from the committed ncu summary of
    the same workload and precision, if present."""
    path = os.path.join(ROOT, "profiles", "stage_kernel_traffic.md")
    key = f"traffic_bytes_per_launch[{workload}/{precision}]:"
    try:
        for line in open(path):
            if line.startswith(key):
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
    o.set_state(**wl.initial(ns))
    return o


ERROR_GROUPS = {"ro": ["ro"], "rou": ["rou", "rov"], "rov": ["rou", "rov"], "u": ["u", "v"], "v": ["u", "v"],
                "cxx": ["cxx", "cxy", "cyy"], "cxy": ["cxx", "cxy", "cyy"], "cyy": ["cxx", "cxy", "cyy"]}


def mixed_error(wl, ns, g, dt, nsteps, device, ref=None):
    """Per-field error of the mixed-precision handle g against the FP64 device path (which
    agrees with the FP64 restatement to ~1e-14 in the parity tests), both stepped nsteps
    from the initial state at the same dt.  Each field's error is relative to the magnitude
    of the quantity it is a component of (rho, the momentum or velocity vector, the
    conformation tensor): L_inf = max|d| / max_group max|f|, L_2 = ||d|| / max_group ||f||."""
    from sunset_viscoelastic_b200 import labfm
    own = ref is None
    if own:
        ref = labfm.for_workload(wl, ns, device=device).setup()
    st = wl.initial(ns)
    for h in (g, ref):
        h.set_state(**st)
        h.step(dt, nsteps)
    a, b = g.state(), ref.state()
    if own:
        ref.close()
    linf, l2 = {}, {}
    for k, grp in ERROR_GROUPS.items():
        d = a[k] - b[k]
        linf[k] = float(np.abs(d).max() / max(max(np.abs(b[f]).max() for f in grp), 1e-300))
        l2[k] = float(np.linalg.norm(d) / max(max(np.linalg.norm(b[f]) for f in grp), 1e-300))
    return {"against": "FP64 device path", "steps": nsteps, "linf": linf, "l2": l2,
            "max_linf": max(linf.values()), "max_l2": max(l2.values())}


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
    # bounded sample: each timed "step" is one full RK step of the whole node set (about 0.2 s
    # on 16 host threads at 262,144 nodes), at most 10 warm-up and 50 timed steps
    warm = max(1, min(args.warmup, 10))
    nsteps = max(1, min(args.steps, 50))
    o.step(dt, warm)
    t = time.perf_counter()
    o.step(dt, nsteps)
    el = time.perf_counter() - t
    nodes = o.sizes()[1]
    value = nodes * nsteps / el
    line = {"metric": METRIC, "value": value, "unit": "node-steps/s", "impl": "reference", "n_gpus": args.gpus,
            "steps": nsteps, "warmup": warm, "ms_per_step": 1e3 * el / nsteps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded jittered lattice)",
            "config": {"workload": wl.name, "nodes": nodes, "order": wl.order, "form": wl.form,
                       "radius_over_s": round(wl.radius_over_s, 4), "cfl": wl.cfl},
            "cpu_baseline": {"value": value, "unit": "node-steps/s", "cores": cpu_threads(), "kind": "port",
                             "sample": f"{nsteps} RK steps of the full {nodes}-node set after {warm} warm-up steps "
                                       f"(host weight build {setup_s:.1f}s untimed)"},
            "e2e": {"value": value, "unit": "node-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "setup": {"host_s": setup_s, "host_nodes_per_s": nodes / setup_s, "cores": cpu_threads(),
                      "what": "neighbour search, weights, sums and filter coefficients of the whole set"}}
    print(json.dumps(line), flush=True)
    return 0


def run_adjoint(args, local):
    """Adjoint/forward cost ratio of sunset_adjoint_run (J = final kinetic energy; gradients
    with respect to Wi, beta and the initial state) and, with --fd-check, its agreement with
    central finite differences (h = 1e-6) of the forward solver."""
    import torch
    from sunset_viscoelastic_b200 import labfm
    torch.cuda.set_device(local)
    wl = WORKLOADS[args.workload if args.workload != DEFAULT_WORKLOAD else ADJOINT_WORKLOAD]
    steps = args.steps
    fwd, adj, J, dWi, dbeta, grads, g, ns, st, dt = adjoint_cost(wl, steps, args.checkpoint, args.warmup, local)
    nodes = g.sizes()[1]
    g.set_state(**st)
    ms_fwd_events = g.step_timed(dt, steps)
    line = {"metric": "adjoint/forward cost", "value": adj / fwd, "unit": "x", "higher_is_better": False,
            "n_gpus": 1, "steps": steps, "warmup": args.warmup, "dtype": "f64", "data": "synthetic (seeded jittered lattice)",
            "config": {"workload": wl.name, "nodes": nodes, "order": wl.order, "form": wl.form, "Wi": wl.Wi,
                       "beta": wl.beta, "checkpoint_every": args.checkpoint,
                       "objective": "sum 1/2 rho |u|^2 vol after the run"},
            "forward_s": fwd, "forward_ms_events": ms_fwd_events, "adjoint_s": adj,
            "J": J, "dJ_dWi": dWi, "dJ_dbeta": dbeta}
    if args.fd_check:
        keys = ["ro", "rou", "rov", "psixx", "psixy", "psiyy", "psizz"]

        def fj(state=None, **over):
            h = labfm.for_workload(wl, ns, device=local, **over).setup() if over else g
            h.set_state(**st)
            if state is not None:
                buf = torch.from_numpy(np.concatenate([state[k] for k in keys])).pin_memory()
                out = torch.empty_like(buf).pin_memory()
                h.run_host(buf.data_ptr(), dt, 0, out.data_ptr())
            h.step(dt, steps)
            J1 = h.kinetic_energy()
            if over:
                h.close()
            return J1
        g.set_state(**st)
        s0 = g.state()
        base = {k: s0[k] for k in keys}
        # Central differences D(h) at h = 1e-6 (relative for the parameters), 1e-4, 1e-3 and
        # 2e-3.  The rounding of J (a few 1e-16 J an evaluation, from the whole run) divided
        # by 2h is not small against the directional derivatives at h = 1e-6; noise =
        # 2e-16 J / (2h) / |D| is a lower bound of that floor.  The errors fall from 1e-6 to
        # 1e-3 (rounding) and rise again at 2e-3 (truncation, O(h^2)).
        hsteps = [1e-6, 1e-4, 1e-3, 2e-3]
        fd = {"steps": hsteps}

        def entry(ad, diff):
            ent = {"adjoint": ad}
            D = {}
            for h in hsteps:
                D[h] = diff(h)
                ent[f"fd_h{h:g}"] = D[h]
                ent[f"rel_h{h:g}"] = abs(ad - D[h]) / abs(D[h])
                ent[f"noise_h{h:g}"] = 2e-16 * J / (2 * h) / abs(D[h])
            return ent

        for name, ad in (("Wi", dWi), ("beta", dbeta)):
            p0 = getattr(wl, name)
            fd[name] = entry(ad, lambda h: (fj(**{name: p0 * (1 + h)}) - fj(**{name: p0 * (1 - h)})) / (2 * h * p0))
        rng = np.random.default_rng(12345)
        dirs = []
        for r in range(8):
            d = {k: rng.standard_normal(nodes) for k in ("psixx", "psixy", "psiyy")}
            ad = sum(float(grads[k] @ d[k]) for k in d)

            def diff(h):
                sp, sm = dict(base), dict(base)
                for k in d:
                    sp[k] = base[k] + h * d[k]
                    sm[k] = base[k] - h * d[k]
                return (fj(sp) - fj(sm)) / (2 * h)
            dirs.append(entry(ad, diff))
        fd["psi0_directions"] = dirs
        ents = [fd["Wi"], fd["beta"]] + dirs
        for h in hsteps:
            fd[f"max_rel_h{h:g}"] = max(e[f"rel_h{h:g}"] for e in ents)
        line["fd_check"] = fd
    print(json.dumps(line), flush=True)
    g.close()
    return 0


def run_3d(args, local):
    """Node-steps/s of the 3-D step (-Ddim3): the workload's x-y node set at --nside per side,
    stacked in z over L_domain_z = --layers, FP64."""
    import dataclasses
    import torch
    from sunset_viscoelastic_b200 import labfm
    torch.cuda.set_device(local)
    wl = dataclasses.replace(WORKLOADS[args.workload], nside=args.nside)
    ns = wl.nodes()
    g = labfm.for_workload(wl, ns, device=local)
    nz, dz = g.set_layers(args.layers)
    g.setup()
    nl = g.sizes()[1]
    x = np.tile(ns.x, nz)
    y = np.tile(ns.y, nz)
    z = np.repeat(np.arange(nz) * dz, nl)
    tp = 2.0 * np.pi
    u = np.sin(tp * x) * np.cos(tp * y) * np.cos(tp * z)
    v = -np.cos(tp * x) * np.sin(tp * y) * np.cos(tp * z)
    w = 0.1 * np.sin(tp * z) * np.cos(tp * x)
    # a smooth conformation with distinct eigenvalues everywhere (the reference's closed-form 3x3
    # eigen solver has no branch for a repeated eigenvalue with nonzero off-diagonal terms)
    ro = 1.0 + 0.01 * np.cos(tp * x) * np.cos(tp * z)
    st3 = [ro, u, v, w, 1.2 + 0.1 * np.sin(tp * z), 0.05 * np.sin(tp * x) * np.sin(tp * y),
           1.1 + 0.05 * np.cos(tp * y), 0.05 * np.cos(tp * z) * np.sin(tp * x), 0.03 * np.sin(tp * z),
           1.05 + 0.02 * np.cos(tp * x)]
    g.set_state_3d(*st3)
    dtc, dtp = g.set_tstep()
    dt = dt_for(wl, dtc, dtp)
    g.step(dt, args.warmup)
    with ClockSampler(local) as clk:
        ms = g.step_timed(dt, args.steps)
    n = nl * nz
    # the derivative gather, timed live inside real steps (events around each launch)
    roof_steps = max(3, min(args.steps, 20))
    g_ms, g_bytes = g.time_stage_kernel(roof_steps)
    peak, peak_kind = measured_peaks()
    achieved = g_bytes / (g_ms * 1e-3) / 1e9
    workload3 = wl.name + f"-3d-nside{args.nside}"
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": profiled_traffic(workload3, "fp64"),
                "kernel": "k3_stage (one fused stage: x-y LABFM sums, z stencils, right-hand side, RK update)",
                "algorithmic_bytes_per_launch": g_bytes, "launch_ms": g_ms, "peak_source": peak_kind,
                "method": f"CUDA events around each of the 4 stage launches of {roof_steps} steps"}
    cpu = None
    if not args.no_cpu_baseline:
        # the CPU restatement on the same 3-D set, all host cores, one step (weights of the
        # layer taken from the device build to keep the sample bounded)
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as O
        O.set_threads(cpu_threads())
        lay = O.for_workload(wl, ns)
        cnt, cs, links = g.neighbours()
        lay.set_neighbours_weights(cnt, cs, links, g.weights())
        o3 = O.Oracle3(lay, args.layers)
        o3.set_state(*st3[:4], *st3[4:])
        t0 = time.perf_counter()
        o3.step(dt, 1)
        el = time.perf_counter() - t0
        cpu = {"value": n / el, "unit": "node-steps/s", "cores": cpu_threads(), "kind": "port",
               "sample": f"1 step of the full {n}-node 3-D set (layer weights from the device build)"}
    line = {"metric": METRIC + " (3-D)", "value": n * args.steps / (ms * 1e-3), "unit": "node-steps/s",
            "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "dtype": "f64", "data": "synthetic (seeded jittered lattice, stacked in z)",
            "config": {"workload": workload3, "nodes_per_layer": nl, "layers": nz, "dz": dz,
                       "nodes": n, "order": wl.order, "form": wl.form, "precision": "fp64"},
            "roofline": roofline, "cpu_baseline": cpu, "clocks": clk.summary()}
    print(json.dumps(line))
    return 0


def stage_roofline(g, wl, precision, steps):
    """The RK stage kernel inside real steps (the same step sequence launched kernel by kernel,
    CUDA events on the handle's stream around each step's four stage launches), against the
    measured HBM copy bandwidth."""
    roof_steps = max(3, min(steps, 50))
    stage_ms, stage_bytes = g.time_stage_kernel(roof_steps)
    peak, peak_kind = measured_peaks()
    achieved = stage_bytes / (stage_ms * 1e-3) / 1e9
    return {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "traffic": profiled_traffic(wl.name, precision), "kernel": "k_stage (one RK stage: stencils + rhs + update)",
            "algorithmic_bytes_per_launch": stage_bytes, "launch_ms": stage_ms, "peak_source": peak_kind,
            "method": f"CUDA events around the 4 back-to-back stage launches of each of {roof_steps} steps, / 4"}


def built_handle(wl, ns, precision, local, phases=None):
    """A handle through the setup calls (sunset.F90:51-60); returns it and the wall seconds of
    the setup (neighbour search, weights, sums, filter coefficients, link streams).  phases
    (a dict), if given, receives the seconds of each call."""
    from sunset_viscoelastic_b200 import labfm
    t0 = time.perf_counter()
    g = labfm.for_workload(wl, ns, precision=precision, device=local)
    calls = [("build_domain", None), ("find_neighbours", g.find_neighbours), ("calc_labf_weights", g.calc_labf_weights),
             ("calc_boundary_weights", g.calc_boundary_weights), ("calc_labf_sums", g.calc_labf_sums),
             ("filter_coefficients (+ link streams)", g.filter_coefficients)]
    t = time.perf_counter()
    if phases is not None:
        phases["build_domain"] = t - t0
    for name, fn in calls[1:]:
        fn()
        g.synchronize()
        t2 = time.perf_counter()
        if phases is not None:
            phases[name] = t2 - t
        t = t2
    return g, time.perf_counter() - t0


def timed_steps(g, dt, args, dist, local):
    g.step(dt, args.warmup)
    g.synchronize()
    if dist:
        dist.barrier()
    with ClockSampler(local) as clk:
        ms = g.step_timed(dt, args.steps)
    if dist:
        dist.barrier()
    return max_over_ranks(dist, ms, device=f"cuda:{local}"), clk.summary()


def setup_block(wl, nodes, device_s, phases):
    """The device setup against the CPU restatement's setup (neighbour search, weights, sums,
    filter coefficients) on a bounded sample: the same order and radius on a 192 x 192 set."""
    import dataclasses
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    O.set_threads(cpu_threads())
    sub = dataclasses.replace(wl, nside=min(wl.nside, 192)) if wl.periodic else wl
    sns = sub.nodes()
    t = time.perf_counter()
    o = O.for_workload(sub, sns).setup()
    el = time.perf_counter() - t
    del o
    return {"device_s": device_s, "device_nodes_per_s": nodes / device_s, "device_phases_s": phases,
            "cpu_nodes_per_s": sns.n / el, "cpu_cores": cpu_threads(), "cpu_kind": "port",
            "cpu_sample": f"the restatement's setup of {sns.n} nodes at the same order and radius ({el:.2f} s)",
            "note": "wall seconds through the C-ABI setup calls, host-side link ordering included"}


def adjoint_cost(wl, steps, checkpoint, warmup, local, reps=3):
    """(forward s, adjoint s, J, dJ/dWi, dJ/dbeta, handle, state, dt): sunset_adjoint_run from
    the initial state against the same forward run, wall clock with the device synchronised;
    each the median of `reps` runs from the initial state (the host's launch loop of a
    0.1-0.5 s run varies by several per cent between runs)."""
    from sunset_viscoelastic_b200 import labfm
    ns = wl.nodes()
    g = labfm.for_workload(wl, ns, device=local).setup()
    st = wl.initial(ns)
    g.set_state(**st)
    dtc, dtp = g.set_tstep()
    dt = dt_for(wl, dtc, dtp)
    # warm up both paths (graphs, adjoint storage), then time each from the initial state
    g.step(dt, warmup)
    g.set_state(**st)
    g.adjoint_run(dt, steps, checkpoint, state_gradient=False)  # sizes the checkpoint store
    fwds, adjs = [], []
    with ClockSampler(local) as clk:
        for _ in range(max(1, reps)):
            g.set_state(**st)
            g.synchronize()
            t = time.perf_counter()
            g.step(dt, steps)
            g.synchronize()
            fwds.append(time.perf_counter() - t)
            g.set_state(**st)
            g.synchronize()
            t = time.perf_counter()
            J, (dWi, dbeta), grads = g.adjoint_run(dt, steps, checkpoint)
            adjs.append(time.perf_counter() - t)
    adjoint_cost.clocks = clk.summary()
    adjoint_cost.samples = {"forward_s": fwds, "adjoint_s": adjs}
    return float(np.median(fwds)), float(np.median(adjs)), J, dWi, dbeta, grads, g, ns, st, dt


def main():
    args = parse()
    ws, rank, local = dist_env()
    if args.impl == "reference":
        return run_reference(args, ws, rank)
    if args.adjoint:
        return run_adjoint(args, local)
    if args.layers > 0.0:
        return run_3d(args, local)
    import torch
    torch.cuda.set_device(local)
    dist = init_pg(ws, "nccl")
    wl = WORKLOADS[args.workload]
    ns = wl.nodes()
    phases = {}
    g, setup_s = built_handle(wl, ns, args.precision, local, phases)
    g.set_state(**wl.initial(ns))
    nodes = g.sizes()[1]  # npfb: the reader's node list, FD rows of boundary nodes included
    dtc, dtp = g.set_tstep()
    dt = dt_for(wl, dtc, dtp)
    ms_max, clocks = timed_steps(g, dt, args, dist, local)
    value = ws * nodes * args.steps / (ms_max * 1e-3)
    roofline = stage_roofline(g, wl, args.precision, args.steps)

    # end to end through the C-ABI with host buffers: per step, copy the evolved fields in
    # from pinned host memory, run the step, copy them back
    n = nodes
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
        del o

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
            "clocks": clocks}
    # the blocks below run on a single rank only (replicas have nothing more to add)
    extra = ws == 1
    if args.precision == "mixed" and not args.no_error_check:
        line["error_vs_fp64"] = mixed_error(wl, ns, g, dt, args.error_steps, local)
    if extra and args.precision == "fp64" and not args.no_mixed:
        gm, _ = built_handle(wl, ns, "mixed", local)
        gm.set_state(**wl.initial(ns))
        ms_mx, clk_mx = timed_steps(gm, dt, args, None, local)
        v_mx = nodes * args.steps / (ms_mx * 1e-3)
        line["mixed"] = {"value": v_mx, "unit": "node-steps/s", "ms_per_step": ms_mx / args.steps,
                         "speedup_vs_fp64": v_mx / value, "dtype": "f32+f64",
                         "roofline": stage_roofline(gm, wl, "mixed", args.steps), "clocks": clk_mx,
                         "gpu_launches": launches_per_step * args.steps}
        if not args.no_error_check:
            line["mixed"]["error_vs_fp64"] = mixed_error(wl, ns, gm, dt, args.error_steps, local, ref=g)
        gm.close()
    if extra and not args.no_setup:
        line["setup"] = setup_block(wl, nodes, setup_s, phases)
    g.close()
    if extra and not args.no_adjoint:
        awl = WORKLOADS[ADJOINT_WORKLOAD]
        fwd, adj, J, dWi, dbeta, _, ga, _, _, _ = adjoint_cost(awl, 200, 20, args.warmup, local)
        ga.close()
        line["adjoint"] = {"value": adj / fwd, "unit": "x (adjoint / forward wall time)", "higher_is_better": False,
                           "workload": awl.name, "steps": 200, "checkpoint_every": 20, "forward_s": fwd,
                           "adjoint_s": adj, "samples": adjoint_cost.samples, "clocks": adjoint_cost.clocks,
                           "J": J, "dJ_dWi": dWi, "dJ_dbeta": dbeta,
                           "fd_check": "python bench.py --adjoint --steps 200 --fd-check"}
        # the same run with every step's stages recorded in HBM (one segment, about 52 GB at
        # 262,144 nodes): no forward recomputation
        fwd2, adj2, J2, dWi2, dbeta2, _, ga, _, _, _ = adjoint_cost(awl, 200, 200, args.warmup, local)
        ga.close()
        line["adjoint"]["all_steps_recorded"] = {
            "value": adj2 / fwd2, "checkpoint_every": 200, "forward_s": fwd2, "adjoint_s": adj2,
            "same_gradients": bool(J2 == J and dWi2 == dWi and dbeta2 == dbeta)}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
