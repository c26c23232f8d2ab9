"""Inflow and outflow in 3-D on the device against the CPU restatement: the inflow channel
(inflow nodes at x = 0, outflow nodes at x = 2, periodic or symmetric in y) stacked in z, for the
direct, Cholesky and log-conformation forms, the three inflow types, the inflow ramp and
polymer diffusion.

Reference behaviour restated (and followed by the device):
* build_3rd_dimension (setup_domain.F90:487-532) copies node_type to every layer, so every
  layer has its inflow and outflow nodes, with the layer's boundary weights (d/dx, d/dy; the
  outflow's first derivatives reversed, labf.F90:986-991) and the z stencils;
* calc_rhs_ro's in/out branch with -w drho/dz - rho dw/dz (rhs_di.F90:155-157), the amplitudes
  with L4 = u dw/dx and the transverse, viscous and body-force terms of calc_rhs_rovel with their
  z parts (:311-359), the closures of characteristic_boundaries.F90:54-189 with their w terms
  (soft inflow: L3 with -w dv/dz, L4 = w nscbc c / L_x + rhs_row, L5 with the second transverse
  term; inflow-outflow: L4 = w nscbc c / L_x; outflow: L4 = 0 when u <= 0) and calc_rhs_nscbc
  with the row update;
* the conformation equations there: zero in the direct form (rhs_di.F90:582-590), the Cholesky
  form without streamwise advection on inflow nodes and with the one-sided flux closure of the
  conformation Laplacian (rhs.F90:558-643), the log-conformation form as in the interior;
* apply_time_dependent_bounds: u_inflow_local on its ramp at each stage's time, a hard inflow's
  momentum u_inflow_local rho, 0, 0 (characteristic_boundaries.F90:191-300);
* set_tstep's 0.8 on outflow nodes (step.F90:592-593).

Tolerances as in the other 3-D parity tests: right-hand sides within 1e-10 of their terms,
fields after 30 steps within 1e-8.
"""
import numpy as np
import pytest

from sunset_viscoelastic_b200 import labfm
from sunset_viscoelastic_b200.nodesets import inflow_channel, inflow_state
import oracle as O

pytestmark = pytest.mark.gpu

W_TOL = 1e-10
F_TOL = 1e-8
BASE = dict(Re=10.0, Wi=0.5, beta=0.59, Ma=0.1, kolmogorov_forcing=0)
ORDER = {"di": 4, "lc": 6, "chl": 8}

# (form, inflow_type, y conditions, L_domain_z, extra settings)
CASES = {
    "di-in0": ("di", 0, 1, 0.4, {}),
    "di-in1-ysym-nz32": ("di", 1, 2, 1.4, {}),
    "di-in2": ("di", 2, 1, 0.4, {}),
    "lc-in1-ramp": ("lc", 1, 1, 0.4, {"inflow_velocity_control": 1, "u_inflow_start": 0.8, "u_inflow_end": 1.2,
                                      "ramp_time": 0.02}),
    "lc-in0-ysym": ("lc", 0, 2, 0.4, {}),
    "chl-in2": ("chl", 2, 1, 0.4, {}),
    "chl-in1-mdiff": ("chl", 1, 2, 0.4, {"Mdiff": 1e-3}),
    "di-in1-fenep": ("di", 1, 1, 0.4, {"fenep": True, "fenep_l2": 100.0}),
}


def state3(x, y, z, Lz):
    """inflow_state's stream with z perturbations (w, c_xz, c_yz non-zero); v odd about the y
    boundaries, w and the rest even, so that the symmetric conditions hold."""
    st = inflow_state(type("R", (), {"x": x, "y": y}))
    kz = 2.0 * np.pi * z / Lz
    st["u"] = st["u"] * (1.0 + 0.02 * np.cos(kz))
    st["w"] = 0.03 * np.sin(kz) * np.cos(2.0 * np.pi * y) * np.cos(np.pi * x)
    st["ro"] = st["ro"] + 0.002 * np.sin(kz)
    st["cxz"] = 0.02 * np.cos(kz) * np.cos(2.0 * np.pi * y)
    st["cyz"] = 0.01 * np.sin(kz) * np.sin(2.0 * np.pi * y)
    st["czz"] = 1.05 + 0.02 * np.cos(kz)
    return st


@pytest.fixture(scope="module", params=list(CASES))
def pair(request):
    form, itype, ybc, Lz, extra = CASES[request.param]
    kw = dict(BASE, form=form, order=ORDER[form], inflow_type=itype, **extra)
    ns = inflow_channel(24, ybc=ybc)
    O.set_pow_mode(True)
    try:
        layer = O.Oracle(**kw).build_domain(ns).setup()
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
    t = np.tile(nd["node_type"][:nl], nz)
    st = state3(x, y, z, nz * dz)
    yield request.param, form, itype, ref, gpu, st, t
    gpu.close()


def set_both(ref, gpu, st):
    c = {k: st[k] for k in ["cxx", "cxy", "cyy", "cxz", "cyz", "czz"]}
    ref.set_state(st["ro"], st["u"], st["v"], st["w"], **c)
    gpu.set_state_3d(st["ro"], st["u"], st["v"], st["w"], **c)


def test_state_and_rhs(pair):
    name, form, itype, ref, gpu, st, t = pair
    io = (t == 1) | (t == 2)
    assert np.sum(t == 1) > 0 and np.sum(t == 2) > 0
    set_both(ref, gpu, st)
    sr, sg = ref.state(), gpu.state_3d()
    for k in sr:
        e = float(np.abs(sg[k] - sr[k]).max() / max(np.abs(sr[k]).max(), 1.0))
        assert e <= W_TOL, (k, e)
    rr, rg = ref.rhs(), gpu.rhs_3d()
    for k in rr:
        scale = max(np.abs(rr[k]).max(), 1.0)
        e = float(np.abs(rg[k] - rr[k]).max() / scale)
        eb = float(np.abs(rg[k][io] - rr[k][io]).max() / scale)
        print(f"{name} rhs_{k}: {e:.2e} (inflow/outflow {eb:.2e}, |rhs| there {np.abs(rr[k][io]).max():.3e})")
        assert e <= W_TOL, (k, e)
    # the closures are exercised: continuity and rho w are non-zero on the in/out node-layers
    assert np.abs(rr["ro"][io]).max() > 0 and np.abs(rr["row"][io]).max() > 0


def test_steps(pair):
    name, form, itype, ref, gpu, st, t = pair
    set_both(ref, gpu, st)
    dcr, dpr = ref.set_tstep()
    dcg, dpg = gpu.set_tstep()
    np.testing.assert_allclose([dcg, dpg], [dcr, dpr], rtol=1e-14)
    dt = 0.3 * min(dcr, dpr)
    for o in (ref, gpu):
        o.step(dt, 30)
    sr, sg = ref.state(), gpu.state_3d()
    for k in sr:
        e = float(np.abs(sg[k] - sr[k]).max() / max(np.abs(sr[k]).max(), 1e-300))
        print(f"{name} {k} after 30 steps: {e:.2e}")
        assert e <= F_TOL, (k, e)
    if itype == 1:  # hard inflow: v = w = 0 there
        for k in ("rov", "row", "v", "w"):
            assert np.all(sg[k][t == 1] == 0.0), k
    tr, tg = ref.time(), gpu.time()
    np.testing.assert_allclose(tg["time"], tr["time"], rtol=1e-14)
    np.testing.assert_allclose(tg["emax"], tr["emax"], rtol=1e-6)
    for o in (ref, gpu):
        o.step(0.0, 5, pid=True)
    sr, sg = ref.state(), gpu.state_3d()
    for k in ["ro", "rou", "row", "cxx", "czz"]:
        e = float(np.abs(sg[k] - sr[k]).max() / max(np.abs(sr[k]).max(), 1e-300))
        assert e <= F_TOL, (k, e)
    np.testing.assert_allclose(gpu.time()["dt"], ref.time()["dt"], rtol=1e-10)
