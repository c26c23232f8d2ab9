"""Walls in 3-D on the device against the CPU restatement: a channel (walls at y = 0 and 1,
node_type 0, with their FD rows and boundary weights) stacked in z, for the direct, Cholesky,
log-conformation and Newtonian forms, with and without polymer diffusion, FENE-P with the
direct and Cholesky forms.

Reference behaviour restated (and followed by the device):
* build_3rd_dimension (setup_domain.F90:487-532) copies node_type and the normals to every
  layer; a wall node's x-y operators are its boundary weights (d/dn, d/dt), its z operators
  the stencils of fd.F90 as everywhere;
* the wall closure of the flow with its dim3 terms: calc_rhs_ro's wall branch with rho dw/dz
  (rhs_di.F90:149-154), the wave amplitudes with L4 (:291-307), the isothermal wall
  (characteristic_boundaries.F90:27-52) and calc_rhs_nscbc (rhs_di.F90:601-665);
* the conformation equations on walls with the velocity gradients turned to x-y and d/dz
  unrotated, without advection (rhs_di.F90:478-590, rhs.F90:553-717, rhs_lc.F90:564-740);
  under polymer diffusion the tangential Laplacian plus the z stencil
  (derivatives.F90:306-358) and the one-sided normal second derivative over the FD rows;
* apply_time_dependent_bounds (characteristic_boundaries.F90:191-257) after every stage and
  after the filter: rho u, rho v, rho w zero on the walls.

Tolerances as in the other 3-D parity tests: right-hand sides within 1e-10 of their terms,
fields after 30 steps within 1e-8.  nz >= 32 in one case, so the blocks of 32 layers of four
nodes run as well as the node-layers in order.
"""
import numpy as np
import pytest

from sunset_viscoelastic_b200 import labfm
from sunset_viscoelastic_b200.nodesets import channel, poiseuille_state
import oracle as O

pytestmark = pytest.mark.gpu

W_TOL = 1e-10
F_TOL = 1e-8
G = 8.0
PARAMS = dict(Re=1.0, Wi=0.5, beta=0.59, Ma=0.1, grav=(G, 0.0, 0.0), kolmogorov_forcing=0)

# (form, order, L_domain_z, overrides)
CASES = {
    "di-o6": ("di", 6, 0.4, {"epsPTT": 0.25}),
    "di-o8-mdiff-nz32": ("di", 8, 1.4, {"epsPTT": 0.25, "Mdiff": 1e-3}),
    "chl-o6-mdiff": ("chl", 6, 0.4, {"epsPTT": 0.25, "Mdiff": 1e-3}),
    "lc-o6": ("lc", 6, 0.4, {"epsPTT": 0.25}),
    "newt-o8": ("newt", 8, 0.4, {}),
    "di-o6-fenep-mdiff": ("di", 6, 0.4, {"fenep": True, "fenep_l2": 30.0, "Mdiff": 1e-3}),
    "chl-o8-fenep-mdiff": ("chl", 8, 0.4, {"fenep": True, "fenep_l2": 30.0, "Mdiff": 1e-3}),
}


def state3(x, y, z, Lz):
    """Poiseuille flow with perturbations in x, y and z (w and c_xz, c_yz non-zero) whose
    velocity parts vanish on the walls; c stays positive definite."""
    st = poiseuille_state(type("P", (), {"y": y, "n": len(y)}), G, 1.0, 0.5)
    kz = 2.0 * np.pi * z / Lz
    yy = y * (1.0 - y)
    st["u"] = st["u"] + 0.3 * np.sin(2 * np.pi * x) * yy * np.cos(kz)
    st["v"] = 0.2 * np.cos(2 * np.pi * x) * yy
    st["w"] = 0.1 * yy * np.sin(kz)
    st["ro"] = 1.0 + 0.01 * np.sin(2 * np.pi * x) * np.cos(np.pi * y) * np.cos(kz)
    st["cxx"] = st["cxx"] + 0.1 * np.sin(2 * np.pi * x) ** 2 + 0.05 * np.sin(kz) ** 2
    st["cyy"] = st["cyy"] + 0.05 * np.cos(np.pi * y) ** 2
    st["czz"] = 1.05 + 0.02 * np.cos(kz)
    st["cxz"] = 0.05 * yy * np.cos(kz)
    st["cyz"] = 0.03 * yy * np.sin(kz)
    return st


@pytest.fixture(scope="module", params=list(CASES))
def pair(request):
    form, order, Lz, over = CASES[request.param]
    kw = dict(PARAMS, form=form, order=order, **over)
    ns = channel(24)
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
    wall = np.tile(nd["node_type"][:nl] == 0, nz)
    st = state3(x, y, z, nz * dz)
    yield request.param, form, ref, gpu, st, wall
    gpu.close()


def set_both(form, ref, gpu, st):
    c = {} if form == "newt" else {k: st[k] for k in ["cxx", "cxy", "cyy", "cxz", "cyz", "czz"]}
    ref.set_state(st["ro"], st["u"], st["v"], st["w"], **c)
    gpu.set_state_3d(st["ro"], st["u"], st["v"], st["w"], **c)


def test_state_and_rhs(pair):
    name, form, ref, gpu, st, wall = pair
    assert wall.sum() > 0
    set_both(form, ref, gpu, st)
    sr, sg = ref.state(), gpu.state_3d()
    for k in sr:
        e = float(np.abs(sg[k] - sr[k]).max() / max(np.abs(sr[k]).max(), 1.0))
        assert e <= W_TOL, (k, e)
    for k in ("u", "v", "w", "rou", "rov", "row"):  # hardcode_initial_conditions: at rest on walls
        assert np.all(sg[k][wall] == 0.0), k
    rr, rg = ref.rhs(), gpu.rhs_3d()
    for k in rr:
        if form == "newt" and k in ("xx", "xy", "yy", "xz", "yz", "zz"):
            continue
        scale = max(np.abs(rr[k]).max(), 1.0)
        e = float(np.abs(rg[k] - rr[k]).max() / scale)
        ew = float(np.abs(rg[k][wall] - rr[k][wall]).max() / scale)
        print(f"{name} rhs_{k}: {e:.2e} (walls {ew:.2e}, |rhs| on walls {np.abs(rr[k][wall]).max():.3e})")
        assert e <= W_TOL, (k, e)
    # the wall closure is exercised: continuity and the conformation equations are non-zero there
    assert np.abs(rr["ro"][wall]).max() > 0
    if form != "newt":
        assert np.abs(rr["xx"][wall]).max() > 0 and np.abs(rr["xz"][wall]).max() > 0


def test_steps(pair):
    name, form, ref, gpu, st, wall = pair
    set_both(form, ref, gpu, st)
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
    for k in ("u", "v", "w", "rou", "rov", "row"):  # apply_time_dependent_bounds
        assert np.all(sg[k][wall] == 0.0), k
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
