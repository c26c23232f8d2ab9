"""Error paths of the C-ABI, each driven from the host with no GPU fault.

The reference stops the process where the library returns a code (svdlib.F90:219-222,
floating-point traps of its -ffpe-trap build); it has no conditioning check at all.  Each
case here makes the failure on the host side -- a NaN in the state, a limit on the SVD's QR
sweeps, a corrupt node file, a stencil radius whose moment matrices are near-singular -- and
checks the code the call returns and that the handle stays usable where it should.
"""
import dataclasses

import numpy as np
import pytest
import torch

from sunset_viscoelastic_b200 import labfm
from sunset_viscoelastic_b200.nodesets import WORKLOADS, initial_state, jittered_lattice
import oracle as O

pytestmark = pytest.mark.gpu


def small(name, nside, **over):
    return dataclasses.replace(WORKLOADS[name], nside=nside, **over)


def code_of(fn, *a, **kw):
    with pytest.raises(labfm.SunsetError) as e:
        fn(*a, **kw)
    return e.value.code


def test_nan_state_gives_nonfinite_from_step_and_run_host():
    wl = small("periodic-di-o4-16k", 32)
    ns = wl.nodes()
    g = labfm.for_workload(wl, ns).setup()
    st = initial_state(ns)
    g.set_state(**st)
    dtc, dtp = g.set_tstep()
    dt = wl.cfl * min(dtc, dtp)
    bad = dict(st)
    bad["u"] = st["u"].copy()
    bad["u"][17] = np.nan
    g.set_state(**bad)
    assert code_of(g.step, dt, 1) == labfm.ERR_NONFINITE
    s0 = g.state()
    keys = ["ro", "rou", "rov", "cxx", "cxy", "cyy", "czz"]
    buf = torch.from_numpy(np.concatenate([s0[k] for k in keys])).pin_memory()
    out = torch.empty_like(buf).pin_memory()
    g2 = labfm.for_workload(wl, ns).setup()
    g2.set_state(**st)
    assert code_of(g2.run_host, buf.data_ptr(), dt, 2, out.data_ptr()) == labfm.ERR_NONFINITE
    # the handle still steps a finite state afterwards
    g.set_state(**st)
    g.step(dt, 2)
    assert np.all(np.isfinite(g.state()["u"]))
    g.close()
    g2.close()


def test_run_host_rejects_bad_dt_and_nsteps():
    wl = small("periodic-di-o4-16k", 32)
    ns = wl.nodes()
    g = labfm.for_workload(wl, ns).setup()
    g.set_state(**initial_state(ns))
    buf = torch.zeros(7 * ns.n, dtype=torch.float64).pin_memory()
    out = torch.empty_like(buf).pin_memory()
    assert code_of(g.run_host, buf.data_ptr(), 0.0, 1, out.data_ptr()) == labfm.ERR_ARG
    assert code_of(g.run_host, buf.data_ptr(), -1e-4, 1, out.data_ptr()) == labfm.ERR_ARG
    assert code_of(g.run_host, buf.data_ptr(), 1e-4, -1, out.data_ptr()) == labfm.ERR_ARG
    g.close()


def test_svd_sweep_limit_gives_svd_error():
    wl = small("periodic-lc-o6-262k", 24)
    ns = wl.nodes()
    g = labfm.for_workload(wl, ns, svd_max_sweeps=1)
    g.find_neighbours()
    assert code_of(g.calc_labf_weights) == labfm.ERR_SVD
    g.close()
    # the reference's 30 sweeps converge on the same set
    g = labfm.for_workload(wl, ns)
    g.find_neighbours()
    g.calc_labf_weights()
    g.close()


def test_conditioning_matches_restatement_and_flags_the_stated_radius():
    # order 6 at the stated radius 3.2 s: near-singular moment matrices at some nodes
    wl = small("periodic-lc-o6-262k", 64, radius_over_s=3.2)
    ns = wl.nodes()
    O.set_pow_mode(True)
    try:
        ref = O.for_workload(wl, ns).setup()
    finally:
        O.set_pow_mode(False)
    cd_r, cf_r = ref.conditioning()
    g = labfm.for_workload(wl, ns)
    g.find_neighbours()
    with pytest.warns(RuntimeWarning, match="condition number"):
        g.calc_labf_weights()
    cd, cf, worst, nill = g.conditioning()
    # the device SVD is the restatement's bit for bit, so are its singular values
    assert np.array_equal(cd, cd_r) and np.array_equal(cf, cf_r)
    assert nill == int(np.sum(np.maximum(cd_r, cf_r) > 1e12)) and nill > 0
    assert worst == max(cd_r.max(), cf_r.max())
    g.close()
    # with a limit set, the same set is an error
    g = labfm.for_workload(wl, ns, cond_max=1e12)
    g.find_neighbours()
    assert code_of(g.calc_labf_weights) == labfm.ERR_ILLCOND
    assert "condition number" in g.L.sunset_last_error(g.h).decode()
    g.close()
    # the measured radius 4.2 s is well conditioned
    g = labfm.for_workload(small("periodic-lc-o6-262k", 64), ns, cond_max=1e12)
    g.setup()
    _, _, worst, nill = g.conditioning(arrays=False)
    assert nill == 0 and worst < 1e8
    g.close()


@pytest.mark.parametrize("what", ["node_type", "spacing", "nan_position", "far_position", "normal", "bcond"])
def test_corrupt_node_rows_are_rejected(what):
    ns = jittered_lattice(16)
    k = 37
    if what == "node_type":
        t = ns.node_type.copy(); t[k] = 5
        bad = dataclasses.replace(ns, node_type=t)
    elif what == "spacing":
        s = ns.s.copy(); s[k] = 0.0
        bad = dataclasses.replace(ns, s=s)
    elif what == "nan_position":
        x = ns.x.copy(); x[k] = np.nan
        bad = dataclasses.replace(ns, x=x)
    elif what == "far_position":
        y = ns.y.copy(); y[k] = 5.0
        bad = dataclasses.replace(ns, y=y)
    elif what == "normal":  # a wall node with no normal
        t = ns.node_type.copy(); t[k] = 0
        bad = dataclasses.replace(ns, node_type=t)
    else:
        bad = dataclasses.replace(ns, bcond=(7, 7, 1, 1))
    wl = small("periodic-di-o4-16k", 16)
    g = labfm.Sunset(**wl.params())
    assert code_of(g.build_domain, bad) == labfm.ERR_ARG
    g.close()
    labfm.Sunset(**wl.params()).build_domain(ns).close()  # the intact rows are accepted


def test_call_order_and_3d_scope():
    wl = small("periodic-di-o4-16k", 16)
    ns = wl.nodes()
    g = labfm.for_workload(wl, ns)
    assert code_of(g.calc_labf_weights) == labfm.ERR_ARG    # before find_neighbours
    g.setup()
    assert code_of(g.step, 1e-5, 1) == labfm.ERR_ARG        # before set_state
    assert code_of(g.kinetic_energy) == labfm.ERR_ARG       # no state to reduce yet
    assert code_of(g.mass) == labfm.ERR_ARG
    g.set_layers(0.25)
    assert code_of(g.kinetic_energy) == labfm.ERR_ARG       # a 3-D handle: before set_state_3d
    assert code_of(g.load_checkpoint, b"\0" * 64) == labfm.ERR_ARG   # not a 3-D checkpoint of this size
    assert code_of(g.save_checkpoint) == labfm.ERR_ARG      # nothing to save before set_state_3d
    g.close()
