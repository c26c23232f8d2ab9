"""Driver for profiler captures of the time-step kernels.

    python -m sunset_viscoelastic_b200.profile_step WORKLOAD [fp64|mixed] [STEPS] [NSIDE]

NSIDE (periodic workloads) replaces the node set's side, for captures on a smaller set of the
same order, radius and form.

Sets the workload up (neighbours, weights, link stream), sets the initial state, runs two
graph-launched steps, then STEPS steps launched kernel by kernel through
sunset_time_stage_kernel.  Kernel launch order after setup: the two graph steps (4 k_stage,
1 k_filter, 1 k_finalize, 1 k_tstep each), then the STEPS direct steps in the same order, so
`-k regex:k_stage -s 9 -c 1` selects stage 1 of the first direct step and
`-k regex:k_filter -s 2 -c 1` its filter.
"""
from __future__ import annotations

import dataclasses
import sys

from . import labfm
from .nodesets import WORKLOADS, initial_state


def main(argv=None) -> int:
    argv = sys.argv[1:] if argv is None else argv
    wl = WORKLOADS[argv[0]]
    precision = argv[1] if len(argv) > 1 else "fp64"
    steps = int(argv[2]) if len(argv) > 2 else 3
    if len(argv) > 3:
        wl = dataclasses.replace(wl, nside=int(argv[3]))
    ns = wl.nodes()
    g = labfm.for_workload(wl, ns, precision=precision).setup()
    g.set_state(**initial_state(ns))
    dtc, dtp = g.set_tstep()
    g.step(wl.cfl * min(dtc, dtp), 2)
    g.synchronize()
    ms, nbytes = g.time_stage_kernel(steps)
    print(f"{wl.name} {precision}: stage kernel {ms * 1e3:.1f} us/launch, {nbytes / 1e6:.1f} MB algorithmic, "
          f"{nbytes / (ms * 1e-3) / 1e9:.0f} GB/s")
    g.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
