"""Inflow/outflow boundaries and the flow-rate controller on the device, against the CPU
restatement.

Node sets: the in/out tube of the reference generator's cases 5 and 6 (gen/datclass.F90):
inflow (node_type 1) at x = 0, outflow (node_type 2) at x = lx, periodic or symmetric in y.

Reference behaviour restated (and followed by the device):
* the neighbour search over the 3x3 block of the reference's cells only: at order 4 the
  boundary nodes' radius (hovs_bound = 2.1) exceeds the cell side (hovs = 1.8), and points
  beyond the block are not neighbours (neighbours.F90:95-243);
* boundary weights of inflow/outflow nodes: links pruned to the node's own layer and FD rows,
  FD normal and 1-D LABFM tangential derivatives, the outflow's first derivatives reversed
  into the x-y frame (labf.F90:505-1039); their Laplacian weights are never set there
  (ij_w_lap is allocated without a value, labf.F90:72), taken as zero;
* the in/out branches of calc_rhs_ro and calc_rhs_rovel and the characteristic closures of
  characteristic_boundaries.F90 for inflow_type 0 (soft), 1 (hard) and 2 (inflow-outflow) and
  for the outflow; the conformation on in/out nodes (DI: zero; CHL: no streamwise advection
  at inflows, the one-sided flux closure of the c Laplacian; LC: the interior form);
* apply_time_dependent_bounds after every stage and after the filter, with the inflow
  velocity ramp of update_u_inflow evaluated at the stage times;
* velocity_control with -Dvpid (statistics.F90:214-303) after every step.

Tolerances as for the wall and periodic parity tests: weights and right-hand sides within
1e-10 of their terms, fields after 100 steps within 1e-8 (the device's sums run in a fixed
tree, the restatement's in node order), the mixed-precision step within 1e-6 of FP64.
"""
import dataclasses

import numpy as np
import pytest

from sunset_viscoelastic_b200 import labfm
from sunset_viscoelastic_b200.nodesets import WORKLOADS, initial_state, inflow_channel, inflow_state
import oracle as O

pytestmark = pytest.mark.gpu

W_TOL = 1e-10
F_TOL = 1e-8

BASE = dict(Re=10.0, Wi=0.5, beta=0.59, Ma=0.1, kolmogorov_forcing=0)
ORDER = {"di": 4, "lc": 6, "chl": 8}

# (form, inflow_type, ybc, extra settings)
CASES = [
    ("di", 1, 1, {}),
    ("di", 0, 2, {}),
    ("di", 2, 1, {}),
    ("lc", 1, 2, {}),
    ("lc", 0, 1, {}),
    ("lc", 2, 2, {}),
    ("chl", 1, 1, {}),
    ("chl", 0, 2, {}),
    ("chl", 2, 1, {}),
    ("chl", 1, 2, {"Mdiff": 1e-3}),
    ("di", 1, 1, {"fenep": True, "fenep_l2": 100.0}),
    ("lc", 1, 1, {"inflow_velocity_control": 1, "u_inflow_start": 0.8, "u_inflow_end": 1.2, "ramp_time": 0.02}),
    ("chl", 2, 2, {"inflow_velocity_control": 1, "u_inflow_start": 0.9, "u_inflow_end": 1.1, "ramp_time": 0.02,
                   "vpid": True}),
]


def case_id(c):
    form, it, ybc, extra = c
    tags = "-".join(k for k in extra if k not in ("u_inflow_start", "u_inflow_end", "ramp_time", "fenep_l2"))
    return f"{form}-in{it}-y{ybc}" + (f"-{tags}" if tags else "")


def rel(a, b, scale=None):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    s = max(np.abs(b).max(), 1e-300) if scale is None else scale
    return float(np.abs(a - b).max() / s)


def reader_nodes(o):
    """x, y of the reader's node list (boundary nodes followed by their FD rows)."""
    nd = o.nodes()
    n = o.sizes()[1]
    return type("ReaderNodes", (), {"x": nd["x"][:n], "y": nd["y"][:n], "n": n, "t": nd["node_type"][:n]})


@pytest.fixture(scope="module", params=CASES, ids=[case_id(c) for c in CASES])
def pair(request):
    form, itype, ybc, extra = request.param
    ns = inflow_channel(32, ybc=ybc)
    kw = dict(BASE, form=form, order=ORDER[form], inflow_type=itype, **extra)
    O.set_pow_mode(True)
    try:
        ref = O.Oracle(**kw).build_domain(ns).setup()
    finally:
        O.set_pow_mode(False)
    gpu = labfm.Sunset(**kw)
    gpu.build_domain(ns)
    gpu.setup()
    rn = reader_nodes(ref)
    return request.param, kw, ns, rn, ref, gpu


def test_lists_and_weights(pair):
    c, kw, ns, rn, ref, gpu = pair
    rc, rcs, rl = ref.neighbours()
    gc, gcs, gl = gpu.neighbours()
    np.testing.assert_array_equal(gc, rc)
    np.testing.assert_array_equal(gcs, rcs)
    np.testing.assert_array_equal(gl, rl)
    wr, wg = ref.weights(), gpu.weights()
    for key in ["w_grad", "w_lap", "w_hyp", "w_grad_sum", "w_lap_sum", "w_hyp_sum"]:
        e = rel(wg[key], wr[key])
        assert e <= W_TOL, (key, e)


def test_state_and_rhs(pair):
    c, kw, ns, rn, ref, gpu = pair
    st = inflow_state(rn)
    for o in (ref, gpu):
        o.set_state(**st)
    sr, sg = ref.state(), gpu.state()
    for k in ["ro", "rou", "rov", "u", "v", "cxx", "cxy", "cyy", "czz"]:
        assert rel(sg[k], sr[k], max(np.abs(sr[k]).max(), 1.0)) <= W_TOL, k
    rr, rg = ref.rhs(), gpu.rhs()
    gu = np.abs(ref.gradient(st["u"])).max()
    for k in ["ro", "rou", "rov", "xx", "xy", "yy", "zz"]:
        scale = max(gu * 10.0, np.abs(rr[k]).max(), 1e-300)
        e = rel(rg[k], rr[k], scale)
        print(f"{case_id(c)} rhs_{k}: {e:.2e} (|rhs| {np.abs(rr[k]).max():.3e})")
        assert e <= W_TOL, (k, e)


def test_steps(pair):
    c, kw, ns, rn, ref, gpu = pair
    form, itype, ybc, extra = c
    st = inflow_state(rn)
    for o in (ref, gpu):
        o.set_state(**st)
    dtc, dtp = ref.set_tstep()
    dt = 0.3 * min(dtc, dtp)
    for o in (ref, gpu):
        o.step(dt, 100)
    sr, sg = ref.state(), gpu.state()
    for k in ["ro", "rou", "rov", "u", "v", "cxx", "cxy", "cyy", "czz"]:
        e = rel(sg[k], sr[k])
        print(f"{case_id(c)} {k} after 100 steps: {e:.2e}")
        assert e <= F_TOL, (k, e)
    tr, tg = ref.time(), gpu.time()
    np.testing.assert_allclose(tg["time"], tr["time"], rtol=1e-14)
    np.testing.assert_allclose(tg["emax"], tr["emax"], rtol=1e-6)
    if extra.get("vpid"):
        fr, fg = ref.flow_control(), gpu.flow_control()
        print(f"flow control: restatement {fr}, device {fg}")
        assert fr["driving_force"][0] != 0.0
        np.testing.assert_allclose(fg["eflow_nm1"], fr["eflow_nm1"], rtol=1e-9, atol=1e-12)
        np.testing.assert_allclose(fg["sum_eflow"], fr["sum_eflow"], rtol=1e-9, atol=1e-14)
        np.testing.assert_allclose(fg["driving_force"], fr["driving_force"], rtol=1e-9, atol=1e-12)
    if itype == 1:  # hard inflow: v = 0 on the inflow nodes
        assert np.all(sg["rov"][rn.t == 1] == 0.0)


def test_mixed_precision(pair):
    c, kw, ns, rn, ref, gpu = pair
    mx = labfm.Sunset(**dict(kw, precision="mixed"))
    mx.build_domain(ns)
    mx.setup()
    st = inflow_state(rn)
    for o in (gpu, mx):
        o.set_state(**st)
    dtc, dtp = gpu.set_tstep()
    dt = 0.3 * min(dtc, dtp)
    for o in (gpu, mx):
        o.step(dt, 100)
    a, b = mx.state(), gpu.state()
    for grp in (["ro"], ["rou", "rov"], ["cxx", "cxy", "cyy", "czz"]):
        s = max(np.abs(b[k]).max() for k in grp)
        for k in grp:
            e = float(np.abs(a[k] - b[k]).max() / s)
            print(f"{case_id(c)} mixed vs FP64 {k}: {e:.2e}")
            assert e <= 1e-6, (k, e)
    mx.close()


def test_flow_controller_periodic():
    """velocity_control on a doubly periodic set: the driving force and the state after 100
    steps, and the controller's state through a dump and restart."""
    wl = dataclasses.replace(WORKLOADS["periodic-lc-o6-262k"], nside=48)
    ns = wl.nodes()
    O.set_pow_mode(True)
    try:
        ref = O.for_workload(wl, ns, vpid=True).setup()
    finally:
        O.set_pow_mode(False)
    gpu = labfm.for_workload(wl, ns, vpid=True).setup()
    st = initial_state(ns)
    for o in (ref, gpu):
        o.set_state(**st)
    dtc, dtp = ref.set_tstep()
    dt = wl.cfl * min(dtc, dtp)
    for o in (ref, gpu):
        o.step(dt, 100)
    fr, fg = ref.flow_control(), gpu.flow_control()
    print(f"flow control: restatement {fr}, device {fg}")
    assert fr["driving_force"][0] > 0.0
    np.testing.assert_allclose(fg["driving_force"], fr["driving_force"], rtol=1e-9)
    np.testing.assert_allclose(fg["sum_eflow"], fr["sum_eflow"], rtol=1e-9)
    np.testing.assert_allclose(fg["eflow_nm1"], fr["eflow_nm1"], rtol=1e-9)
    sr, sg = ref.state(), gpu.state()
    for k in ["ro", "rou", "rov", "cxx", "cxy", "cyy"]:
        assert rel(sg[k], sr[k]) <= F_TOL, k
    # a dump's header carries the controller (output.F90:272-276) and the restart loads it
    cols, hd = gpu.dump()
    np.testing.assert_array_equal(hd[:3], [fg["eflow_nm1"], fg["sum_eflow"], fg["driving_force"][0]])
    gpu2 = labfm.for_workload(wl, ns, vpid=True).setup()
    gpu2.set_restart(cols, hd)
    f2 = gpu2.flow_control()
    assert f2["driving_force"][0] == fg["driving_force"][0] and f2["sum_eflow"] == fg["sum_eflow"]
    # without -Dvpid the statistics call after a step zeroes the driving force
    gpu3 = labfm.for_workload(wl, ns).setup()
    gpu3.set_restart(cols, hd)
    assert gpu3.flow_control()["driving_force"][0] == fg["driving_force"][0]
    gpu3.step(dt, 1)
    assert gpu3.flow_control()["driving_force"][0] == 0.0
    for o in (gpu, gpu2, gpu3):
        o.close()
