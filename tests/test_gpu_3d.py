"""The 3-D (-Ddim3) time step on the device against the CPU restatement: the direct, Cholesky
and log-conformation forms (sPTT / Oldroyd-B, with and without polymer diffusion) and the
Newtonian form, on jittered x-y node sets stacked in z, periodic or symmetric in y.

Reference behaviour restated (and followed by the device):
* build_3rd_dimension (setup_domain.F90:435-547): dz from the mean spacing, nz from
  L_domain_z (a ceiling that the float quotient can push up by one), layer-major nodes;
* calc_fd_weights (fd.F90:27-256): periodic central differences of forder + 1 points for
  d/dz, d2/dz2 and the z filter;
* derivatives.F90: x-y LABFM sums per layer plus the z stencil; the filter as the x-y filter
  followed by the z filter of its result;
* rhs_di.F90 with the dim3 terms: w, rho w, c_xz, c_yz, the z parts of every gradient,
  divergence and Laplacian, the 3-D upper-convected derivative;
* rhs.F90 (Cholesky) with the dim3 terms and the 3-D transforms of conf_transforms.F90:27-125;
* rhs_lc.F90 (log-conformation) with the dim3 terms: the 3x3 eigen-decomposition of c
  (conf_transforms.F90:218-397, closed form with acos and cos, so device and CPU agree to
  rounding rather than bit for bit), the rotation rates and the 3-D transforms;
* step.F90 with the dim3 error norms (row, xz, yz) and set_tstep with |u| including w;
* FENE-P with the direct form (rhs_di.F90:198-245, 454-464): the function
  f = (L^2 - 3)/(L^2 - tr c) at every node, its 3-D gradient, the quotient-rule polymer force
  and the FENE-P relaxation; FENE-P with the Cholesky form (rhs.F90:204-209, 479-500: the
  factors of J = f c); FENE-P with the log-conformation form is refused (its 3-D branch reads
  values the reference never sets);
* the flow-rate controller with dV = vol dz, kinetic energy and mass, and the host-buffer
  round trip on a 3-D handle.  Walls, inflow and outflow, output, restart and checkpoints have
  their own files (test_gpu_3d_walls.py, test_gpu_3d_inout.py, test_gpu_3d_output.py).

Tolerances as in the 2-D parity tests: state and right-hand sides within 1e-10 of their
terms, fields after 50 steps within 1e-8 (the mass correction and the reductions are summed in
a fixed tree on the device, in node order on the CPU).
"""
import dataclasses

import numpy as np
import pytest
import torch

from sunset_viscoelastic_b200 import labfm
from sunset_viscoelastic_b200.nodesets import WORKLOADS
import oracle as O

pytestmark = pytest.mark.gpu

W_TOL = 1e-10
F_TOL = 1e-8

# (workload, nside, L_domain_z, y conditions, overrides)
CASES = {
    "di-o4": ("periodic-di-o4-16k", 24, 1.0, (1, 1), {}),
    "di-o6-mdiff-ysym": ("periodic-lc-o6-262k", 20, 0.6, (2, 2), {"form": "di", "Mdiff": 1e-3}),
    "di-o8-reduced-grads": ("periodic-chl-o8-1m", 20, 0.5, (1, 1), {"form": "di", "di_full_gradients": False}),
    "newt-o6": ("periodic-lc-o6-262k", 20, 0.7, (1, 1), {"form": "newt"}),
    "chl-o8": ("periodic-chl-o8-1m", 20, 0.5, (1, 1), {"epsPTT": 0.25}),
    "chl-o6-mdiff-ysym": ("periodic-lc-o6-262k", 20, 0.6, (2, 2), {"form": "chl", "Mdiff": 1e-3}),
    "lc-o6": ("periodic-lc-o6-262k", 20, 0.5, (1, 1), {}),
    "lc-o8-oldroyd-ysym": ("periodic-chl-o8-1m", 20, 0.5, (2, 2), {"form": "lc", "epsPTT": 0.0}),
    "di-o4-fenep": ("periodic-di-o4-16k", 24, 1.0, (1, 1), {"fenep": True, "fenep_l2": 30.0}),
    "di-o6-fenep-mdiff-ysym": ("periodic-lc-o6-262k", 20, 0.6, (2, 2),
                               {"form": "di", "fenep": True, "fenep_l2": 50.0, "Mdiff": 1e-3}),
    "chl-o6-fenep": ("periodic-lc-o6-262k", 20, 0.6, (1, 1), {"form": "chl", "fenep": True, "fenep_l2": 50.0}),
    "chl-o4-fenep-mdiff-ysym": ("periodic-di-o4-16k", 24, 1.0, (2, 2),
                                {"form": "chl", "fenep": True, "fenep_l2": 30.0, "Mdiff": 1e-3}),
}


def state3(x, y, z):
    tp = 2.0 * np.pi
    return dict(
        ro=1.0 + 0.01 * np.cos(tp * x) * np.cos(tp * z),
        u=np.sin(tp * x) * np.cos(tp * y) * np.cos(tp * z),
        v=-np.cos(tp * x) * np.sin(tp * y) * np.cos(tp * z),
        w=0.1 * np.sin(tp * z) * np.cos(tp * x),
        cxx=1.2 + 0.1 * np.sin(tp * z), cxy=0.05 * np.sin(tp * x) * np.sin(tp * y), cyy=1.1 + 0.05 * np.cos(tp * y),
        cxz=0.05 * np.cos(tp * z) * np.sin(tp * x), cyz=0.03 * np.sin(tp * z), czz=1.05 + 0.02 * np.cos(tp * x))


@pytest.fixture(scope="module", params=list(CASES))
def pair(request):
    wlname, nside, Lz, ybc, over = CASES[request.param]
    wl = dataclasses.replace(WORKLOADS[wlname], nside=nside)
    ns = wl.nodes()
    ns = dataclasses.replace(ns, bcond=(1, 1) + ybc)
    kw = dict(wl.params())
    kw.update(over)
    O.set_pow_mode(True)
    try:
        layer = O.Oracle(**kw)
        layer.build_domain(ns)
        layer.setup()
    finally:
        O.set_pow_mode(False)
    ref = O.Oracle3(layer, Lz)
    gpu = labfm.Sunset(**kw)
    gpu.build_domain(ns)
    nz, dz = gpu.set_layers(Lz)
    gpu.setup()
    assert (nz, dz) == (ref.nz, ref.dz)
    nd = layer.nodes()
    nl = ref.nl
    x = np.tile(nd["x"][:nl], nz)
    y = np.tile(nd["y"][:nl], nz)
    z = np.repeat(np.arange(nz) * dz, nl)
    st = state3(x, y, z)
    return request.param, wl, kw, layer, ref, gpu, st


def test_layers(pair):
    name, wl, kw, layer, ref, gpu, st = pair
    print(f"{name}: nl {ref.nl}, nz {ref.nz}, dz {ref.dz:.6f}")
    assert ref.nz >= (kw.get("order", 4) + 1) // 2 + 2


def test_state_and_rhs(pair):
    name, wl, kw, layer, ref, gpu, st = pair
    newt = kw.get("form") == "newt"
    c = {} if newt else {k: st[k] for k in ["cxx", "cxy", "cyy", "cxz", "cyz", "czz"]}
    ref.set_state(st["ro"], st["u"], st["v"], st["w"], **c)
    gpu.set_state_3d(st["ro"], st["u"], st["v"], st["w"], **c)
    sr, sg = ref.state(), gpu.state_3d()
    for k in sr:
        e = float(np.abs(sg[k] - sr[k]).max() / max(np.abs(sr[k]).max(), 1.0))
        assert e <= W_TOL, (k, e)
    rr, rg = ref.rhs(), gpu.rhs_3d()
    for k in rr:
        scale = max(np.abs(rr[k]).max(), 1.0)
        e = float(np.abs(rg[k] - rr[k]).max() / scale)
        print(f"{name} rhs_{k}: {e:.2e} (|rhs| {np.abs(rr[k]).max():.3e})")
        assert e <= W_TOL, (k, e)
    if not newt:
        assert np.abs(rr["xz"]).max() > 0 and np.abs(rr["row"]).max() > 0


def test_steps(pair):
    name, wl, kw, layer, ref, gpu, st = pair
    newt = kw.get("form") == "newt"
    c = {} if newt else {k: st[k] for k in ["cxx", "cxy", "cyy", "cxz", "cyz", "czz"]}
    ref.set_state(st["ro"], st["u"], st["v"], st["w"], **c)
    gpu.set_state_3d(st["ro"], st["u"], st["v"], st["w"], **c)
    dcr, dpr = ref.set_tstep()
    dcg, dpg = gpu.set_tstep()
    np.testing.assert_allclose([dcg, dpg], [dcr, dpr], rtol=1e-14)
    dt = 0.3 * min(dcr, dpr)
    for o in (ref, gpu):
        o.step(dt, 50)
    sr, sg = ref.state(), gpu.state_3d()
    for k in sr:
        e = float(np.abs(sg[k] - sr[k]).max() / max(np.abs(sr[k]).max(), 1e-300))
        print(f"{name} {k} after 50 steps: {e:.2e}")
        assert e <= F_TOL, (k, e)
    tr, tg = ref.time(), gpu.time()
    np.testing.assert_allclose(tg["time"], tr["time"], rtol=1e-14)
    np.testing.assert_allclose(tg["emax"], tr["emax"], rtol=1e-6)
    # mass_and_energy_check with dV = vol dz (the device sums in a fixed tree)
    np.testing.assert_allclose(gpu.kinetic_energy(), ref.kinetic_energy(), rtol=1e-11)
    np.testing.assert_allclose(gpu.mass(), ref.mass(), rtol=1e-13)
    # PID-controlled steps (set_tstep + set_tstep_PID before each)
    for o in (ref, gpu):
        o.step(0.0, 10, pid=True)
    sr, sg = ref.state(), gpu.state_3d()
    for k in ["ro", "rou", "row", "czz"]:
        e = float(np.abs(sg[k] - sr[k]).max() / max(np.abs(sr[k]).max(), 1e-300))
        assert e <= F_TOL, (k, e)
    np.testing.assert_allclose(gpu.time()["dt"], ref.time()["dt"], rtol=1e-10)


def test_velocity_control_3d():
    """velocity_control with -Dvpid in 3-D (statistics.F90:214-303): after every step the volume
    sums over the node-layers with dV = vol dz drive driving_force(1) by the PID law, and the
    body force of the next step carries it.  Device against the restatement over 20 steps: the
    controller's state (summed in a fixed tree on the device, in node order on the CPU) and the
    fields."""
    wl = dataclasses.replace(WORKLOADS["periodic-di-o4-16k"], nside=24)
    ns = wl.nodes()
    kw = dict(wl.params(), vpid=True, kolmogorov_forcing=0)
    O.set_pow_mode(True)
    try:
        layer = O.Oracle(**kw)
        layer.build_domain(ns)
        layer.setup()
    finally:
        O.set_pow_mode(False)
    ref = O.Oracle3(layer, 1.0)
    gpu = labfm.Sunset(**kw)
    gpu.build_domain(ns)
    nz, dz = gpu.set_layers(1.0)
    gpu.setup()
    nd = layer.nodes()
    nl = ref.nl
    st = state3(np.tile(nd["x"][:nl], nz), np.tile(nd["y"][:nl], nz), np.repeat(np.arange(nz) * dz, nl))
    c = {k: st[k] for k in ["cxx", "cxy", "cyy", "cxz", "cyz", "czz"]}
    ref.set_state(st["ro"], st["u"], st["v"], st["w"], **c)
    gpu.set_state_3d(st["ro"], st["u"], st["v"], st["w"], **c)
    dcr, dpr = ref.set_tstep()
    gpu.set_tstep()
    for o in (ref, gpu):
        o.step(0.3 * min(dcr, dpr), 20)
    fr, fg = layer.flow_control(), gpu.flow_control()
    print("3-D controller:", fr, fg)
    assert abs(fr["driving_force"][0]) > 1e-3
    np.testing.assert_allclose(fg["driving_force"][0], fr["driving_force"][0], rtol=1e-9)
    np.testing.assert_allclose([fg["eflow_nm1"], fg["sum_eflow"]], [fr["eflow_nm1"], fr["sum_eflow"]], rtol=1e-9)
    sr, sg = ref.state(), gpu.state_3d()
    for k in ["ro", "rou", "rov", "row", "cxx", "czz"]:
        e = float(np.abs(sg[k] - sr[k]).max() / max(np.abs(sr[k]).max(), 1e-300))
        assert e <= F_TOL, (k, e)
    gpu.close()


def test_run_host_3d():
    """The host-buffer round trip on a 3-D handle (the evolved fields of every node-layer in,
    nsteps fixed-dt steps, out) against the same steps on a handle stepped in place."""
    wl = dataclasses.replace(WORKLOADS["periodic-di-o4-16k"], nside=24)
    ns = wl.nodes()
    kw = dict(wl.params(), form="chl", epsPTT=0.25)
    handles = []
    for _ in range(2):
        g = labfm.Sunset(**kw)
        g.build_domain(ns)
        nz, dz = g.set_layers(1.0)
        g.setup()
        handles.append(g)
    a, b = handles
    nl = a.sizes()[1]
    O.set_pow_mode(True)
    try:
        layer = O.Oracle(**kw)
        layer.build_domain(ns)
        layer.setup()
    finally:
        O.set_pow_mode(False)
    nd = layer.nodes()
    st = state3(np.tile(nd["x"][:nl], nz), np.tile(nd["y"][:nl], nz), np.repeat(np.arange(nz) * dz, nl))
    c = {k: st[k] for k in ["cxx", "cxy", "cyy", "cxz", "cyz", "czz"]}
    for g in (a, b):
        g.set_state_3d(st["ro"], st["u"], st["v"], st["w"], **c)
    s0 = a.state_3d()
    keys = ["ro", "rou", "rov", "row", "psixx", "psixy", "psiyy", "psixz", "psiyz", "psizz"]
    pin = torch.from_numpy(np.concatenate([s0[k] for k in keys])).pin_memory()
    pout = torch.zeros_like(pin).pin_memory()
    dc, dp = a.set_tstep()
    dt = 0.3 * min(dc, dp)
    a.step(dt, 10)
    b.run_host(pin.data_ptr(), dt, 10, pout.data_ptr())
    sa = a.state_3d()
    out = pout.numpy().reshape(10, -1)
    for q, k in enumerate(keys):
        e = float(np.abs(out[q] - sa[k]).max() / max(np.abs(sa[k]).max(), 1e-300))
        assert e <= 1e-12, (k, e)
    sb = b.state_3d()
    assert np.array_equal(sb["rou"], out[1])
    for g in handles:
        g.close()


def test_fenep_scope():
    """FENE-P in 3-D covers the direct and Cholesky forms; the log-conformation form is refused
    with a scope error."""
    wl = dataclasses.replace(WORKLOADS["periodic-lc-o6-262k"], nside=16)
    ns = wl.nodes()
    kw = dict(wl.params(), fenep=True, fenep_l2=30.0)
    gpu = labfm.Sunset(**kw)
    gpu.build_domain(ns)
    with pytest.raises(labfm.SunsetError, match="FENE-P"):
        gpu.set_layers(0.5)
    gpu.close()
