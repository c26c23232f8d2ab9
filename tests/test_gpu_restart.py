"""Dumps, restart and checkpoints on the device.

* sunset_get_dump: the columns of output_layer (output.F90:272-310) -- rho - rho_char, u, v
  and c as the state holds them; vorticity and Q criterion from the device's velocity
  gradients, rotated on walls (:229-241), against the same formulas applied to the CPU
  restatement's gradients (1e-10 of the gradient scale); alpha_out, whose maximum over the
  nodes is the step's error norm.
* sunset_write_dump then the reference's restart path (nodes file -> sunset_set_lengths
  before the neighbour search, fields file -> sunset_set_restart) into a new handle: the
  same lengths, the same rho, u, v, and c through the psi transform (1e-13), dt and the
  error-norm history; with the run's time and step count carried over (the reference itself
  restarts at step 0) the runs agree after 20 more steps (1e-10).
* Binary checkpoints: a run resumed from a checkpoint -- in the same handle or a new one --
  repeats the uninterrupted run bit for bit.
"""
import dataclasses

import numpy as np
import pytest

from sunset_viscoelastic_b200 import dumpfiles as D
from sunset_viscoelastic_b200 import labfm
from sunset_viscoelastic_b200.nodesets import WORKLOADS, channel, initial_state
import oracle as O

pytestmark = pytest.mark.gpu

WL = dataclasses.replace(WORKLOADS["periodic-lc-o6-262k"], nside=40)
CH = dict(form="di", order=8, Re=1.0, Wi=0.5, beta=0.59, Ma=0.1, grav=(8.0, 0.0, 0.0), kolmogorov_forcing=0)


def lc_state(ns):
    st = initial_state(ns)
    st["cxx"] = 1.0 + 0.3 * np.sin(2 * np.pi * ns.y) ** 2
    st["cxy"] = 0.2 * np.sin(2 * np.pi * ns.x)
    return st


def fields(s):
    return np.stack([s[k] for k in ["ro", "rou", "rov", "u", "v", "psixx", "psixy", "psiyy", "psizz", "cxx", "cxy",
                                   "cyy", "czz"]])


def test_checkpoint_resumes_bit_for_bit():
    ns = WL.nodes()
    g = labfm.for_workload(WL, ns).setup()
    g.set_state(**lc_state(ns))
    dtc, dtp = g.set_tstep()
    dt = WL.cfl * min(dtc, dtp)
    g.step(dt, 30)
    ck = g.save_checkpoint()
    g.step(dt, 30)
    a, ta = fields(g.state()), g.time()
    g.load_checkpoint(ck)
    g.step(dt, 30)
    b, tb = fields(g.state()), g.time()
    assert np.array_equal(a, b)
    assert ta["itime"] == tb["itime"] == 60 and ta["time"] == tb["time"]
    h2 = labfm.for_workload(WL, ns).setup()
    h2.load_checkpoint(ck)
    h2.step(dt, 30)
    assert np.array_equal(fields(h2.state()), a)
    other = labfm.for_workload(dataclasses.replace(WL, nside=32), dataclasses.replace(WL, nside=32).nodes()).setup()
    with pytest.raises(labfm.SunsetError):
        other.load_checkpoint(ck)


def dump_check(gpu, ref, st, walls=None):
    for o in (ref, gpu):
        o.set_state(**st)
    cols, hd = gpu.dump()
    s = gpu.state()
    assert np.array_equal(cols["ro_minus_rho_char"], -1.0 + s["ro"])
    for k in ["u", "v", "cxx", "cxy", "cyy", "czz"]:
        assert np.array_equal(cols[k], s[k]), k
    gu, gv = ref.gradient(s["u"]), ref.gradient(s["v"])
    ux, uy, vx, vy = gu[:, 0], gu[:, 1], gv[:, 0], gv[:, 1]
    vort = vx - uy
    q = -0.5 * ux ** 2 - 0.5 * vy ** 2 - uy * vx
    if walls is not None:
        t, xn, yn = walls
        w = t == 0
        vort[w] = (xn * (vx - uy) - yn * (ux + vy))[w]
        a, b = xn * ux - yn * uy, yn * vx + xn * vy
        q[w] = (-0.5 * a ** 2 - 0.5 * b ** 2 - (yn * ux + xn * uy) * (xn * vx - yn * vy))[w]
    scale = max(np.abs(gu).max(), np.abs(gv).max())
    assert np.abs(cols["vort"] - vort).max() <= 1e-10 * scale
    assert np.abs(cols["qcrit"] - q).max() <= 1e-10 * scale ** 2
    return cols, hd


def test_dump_columns_periodic():
    ns = WL.nodes()
    gpu = labfm.for_workload(WL, ns).setup()
    O.set_pow_mode(True)
    try:
        ref = O.for_workload(WL, ns).setup()
    finally:
        O.set_pow_mode(False)
    st = lc_state(ns)
    dump_check(gpu, ref, st)
    dtc, dtp = gpu.set_tstep()
    gpu.step(WL.cfl * min(dtc, dtp), 3)
    cols, hd = gpu.dump()
    tm = gpu.time()
    # log-conformation: the error norm is the largest alpha_out (the zz error is zero)
    assert cols["alpha"].max() == max(tm["emax"][2], 1e-16)
    assert hd[5] == tm["emax"][2] and hd[8] == tm["dt"]


def test_dump_columns_on_walls():
    ns = channel(32)
    gpu = labfm.Sunset(**CH)
    gpu.build_domain(ns)
    gpu.setup()
    O.set_pow_mode(True)
    try:
        ref = O.Oracle(**CH).build_domain(ns).setup()
    finally:
        O.set_pow_mode(False)
    nd = ref.nodes()
    npfb = ref.sizes()[1]
    x, y, t = nd["x"][:npfb], nd["y"][:npfb], nd["node_type"][:npfb]
    st = dict(ro=np.ones(npfb), u=np.sin(2 * np.pi * x) * y * (1 - y), v=0.2 * np.cos(2 * np.pi * x) * y * (1 - y),
              cxx=np.ones(npfb), cxy=np.zeros(npfb), cyy=np.ones(npfb))
    xn, yn = np.zeros(npfb), np.where(y < 0.5, 1.0, -1.0)  # the channel's walls: y = 0 and y = 1, normals inward
    dump_check(gpu, ref, st, walls=(t, xn, yn))


def test_write_dump_and_restart(tmp_path):
    ns = WL.nodes()
    g = labfm.for_workload(WL, ns)
    g.find_neighbours()
    g.adapt_stencils()
    g.calc_labf_weights()
    g.calc_boundary_weights()
    g.calc_labf_sums()
    g.filter_coefficients()
    g.set_state(**lc_state(ns))
    dtc, dtp = g.set_tstep()
    dt = WL.cfl * min(dtc, dtp)
    g.step(dt, 10)
    g.write_dump(tmp_path, 1, g.time()["time"])
    hd, cols = D.read_fields(tmp_path / "fields_10000_1")
    nd = D.read_nodes(tmp_path / "nodes_10000")
    h, hs = g.lengths()
    assert np.array_equal(nd["h"], h) and np.array_equal(nd["h_small"], hs)
    assert nd["gi"].tolist() == list(range(1, ns.n + 1))
    assert len(open(tmp_path / "time.out").read().split()) == 5
    r = labfm.for_workload(WL, ns)
    r.set_lengths(nd["h"], nd["h_small"])  # restart: no adaptation, lengths from the nodes file
    r.setup()
    r.set_restart(cols, hd)
    assert np.array_equal(r.lengths()[0], h)
    a, b = g.state(), r.state()
    for k in ["ro", "u", "v"]:
        assert np.array_equal(a[k], b[k]), k
    for k in ["cxx", "cxy", "cyy", "psixx", "psixy", "psiyy"]:
        assert np.abs(a[k] - b[k]).max() <= 1e-13 * max(np.abs(a[k]).max(), 1.0), k
    tg, tr = g.time(), r.time()
    assert tr["dt"] == tg["dt"] and np.array_equal(tr["emax"], tg["emax"])
    # the reference restarts at step 0, where the log-conformation form's itime == 1 special
    # case (rhs_lc.F90:503) would run again; carry the run's own time and step count over
    assert tr["itime"] == 0
    r.set_time(tg["time"], tg["dt"], tg["itime"], tg["emax"])
    for o in (g, r):
        o.step(dt, 20)
    a, b = g.state(), r.state()
    for k in ["ro", "rou", "rov", "cxx", "cxy", "cyy"]:
        assert np.abs(a[k] - b[k]).max() <= 1e-10 * max(np.abs(a[k]).max(), 1e-300), k
