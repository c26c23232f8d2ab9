"""Walls on the device against the CPU restatement: a channel with wall nodes (node_type 0),
their FD rows, boundary weights (labf.F90:505-1039) and the wall closure of the right-hand
sides (rhs_*.F90 wall branches, characteristic_boundaries.F90:27-52,191-257).

Tolerances as for the periodic parity tests: weights and right-hand sides within 1e-10
relative (right-hand sides against the size of their terms), fields after 100 steps within
1e-8.  The transverse operators of FD rows 1-2 use atan/cos/sin/tan, where CUDA and glibc may
differ in the last bit, so those weights agree to rounding rather than bit for bit.
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
CASES = [("di", 8), ("lc", 8), ("chl", 8), ("di", 6)]


def rel(a, b, scale=None):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    s = max(np.abs(b).max(), 1e-300) if scale is None else scale
    return float(np.abs(a - b).max() / s)


def perturbed_state(y, x):
    """Poiseuille flow plus a perturbation that vanishes on the walls, with a density and
    conformation perturbation, so every term of the wall closure is non-zero."""
    st = poiseuille_state(type("P", (), {"y": y, "n": len(y)}), G, 1.0, 0.5)
    bump = np.sin(2 * np.pi * x) * y * (1.0 - y)
    st["u"] = st["u"] + 0.3 * bump
    st["v"] = 0.2 * np.cos(2 * np.pi * x) * y * (1.0 - y)
    st["ro"] = 1.0 + 0.01 * np.sin(2 * np.pi * x) * np.cos(np.pi * y)
    st["cxx"] = st["cxx"] + 0.1 * np.sin(2 * np.pi * x) ** 2
    st["cyy"] = st["cyy"] + 0.05 * np.cos(np.pi * y) ** 2
    return st


@pytest.fixture(scope="module", params=CASES, ids=[f"{f}-o{o}" for f, o in CASES])
def pair(request):
    form, order = request.param
    ns = channel(32)
    O.set_pow_mode(True)
    try:
        ref = O.Oracle(form=form, order=order, **PARAMS).build_domain(ns).setup()
    finally:
        O.set_pow_mode(False)
    gpu = labfm.Sunset(form=form, order=order, **PARAMS)
    gpu.build_domain(ns)
    gpu.setup()
    nd = ref.nodes()
    npfb = ref.sizes()[1]
    return form, order, ns, ref, gpu, nd["x"][:npfb], nd["y"][:npfb], nd["node_type"][:npfb]


def test_boundary_links_identical(pair):
    form, order, ns, ref, gpu, x, y, t = pair
    assert gpu.sizes()[:3] == ref.sizes()[:3]
    c1, s1, l1 = ref.neighbours()
    c2, s2, l2 = gpu.neighbours()
    np.testing.assert_array_equal(c2, c1)
    np.testing.assert_array_equal(s2, s1)
    for i in range(len(c1)):
        np.testing.assert_array_equal(l2[i, :c1[i]], l1[i, :c1[i]])


def test_boundary_weights(pair):
    form, order, ns, ref, gpu, x, y, t = pair
    wr, wg = ref.weights(), gpu.weights()
    c, _, _ = ref.neighbours()
    width = min(wr["w_lap"].shape[1], wg["w_lap"].shape[1])
    assert c.max() <= width
    mask = np.arange(width)[None, :] < c[:, None]
    for k in ["w_grad", "w_lap", "w_hyp"]:
        a, b = wg[k][:, :width], wr[k][:, :width]
        m = mask if a.ndim == 2 else mask[..., None]
        scale = np.abs(np.where(m, b, 0)).max(axis=tuple(range(1, b.ndim)), keepdims=True)
        d = np.abs(np.where(m, a - b, 0)) / np.maximum(scale, 1e-300)
        for name, sel in [("walls", t == 0), ("rows 1-2", (t == -1) | (t == -2)), ("other", (t < -2) | (t > 2))]:
            e = float(d[sel].max())
            print(f"{form}-o{order} {k} {name}: {e:.2e}")
            assert e <= W_TOL, (k, name, e)
    for k in ["w_grad_sum", "w_lap_sum", "w_hyp_sum", "vol"]:
        assert rel(wg[k], wr[k]) <= W_TOL, k


def test_poiseuille_is_a_fixed_point(pair):
    """The steady state is polynomial in the direct form; the log-conformation form evolves
    log c but its momentum equation reads c; the Cholesky form's momentum equation reads
    its non-polynomial variables, so there only the continuity equation is exact."""
    form, order, ns, ref, gpu, x, y, t = pair
    st = poiseuille_state(type("P", (), {"y": y, "n": len(y)}), G, 1.0, 0.5)
    gpu.set_state(**st)
    r = gpu.rhs()
    keys = {"di": ["ro", "rou", "rov", "xx", "xy", "yy"], "lc": ["ro", "rou", "rov"], "chl": ["ro"]}[form]
    worst = max(np.abs(r[k]).max() for k in keys) / G
    print(f"{form}-o{order} device max |rhs| / G at the Poiseuille state: {worst:.2e}")
    assert worst < 1e-9


def test_rhs_with_walls(pair):
    form, order, ns, ref, gpu, x, y, t = pair
    st = perturbed_state(y, x)
    for o in (ref, gpu):
        o.set_state(**st)
    sr, sg = ref.state(), gpu.state()
    for k in ["ro", "rou", "rov", "u", "v", "cxx", "cxy", "cyy"]:
        assert rel(sg[k], sr[k]) <= W_TOL, k
    assert np.all(sg["u"][t == 0] == 0.0) and np.all(sg["v"][t == 0] == 0.0)
    rr, rg = ref.rhs(), gpu.rhs()
    gu = np.abs(ref.gradient(st["u"])).max()
    cmax = max(np.abs(st["cxx"]).max(), np.abs(st["cyy"]).max())
    scale = {"ro": gu, "rou": max(gu, np.abs(rr["rou"]).max()), "rov": max(gu, np.abs(rr["rov"]).max()),
             "xx": gu * cmax, "xy": gu * cmax, "yy": gu * cmax}
    for k in ["ro", "rou", "rov", "xx", "xy", "yy"]:
        e = rel(rg[k], rr[k], scale[k])
        ew = rel(rg[k][t == 0], rr[k][t == 0], scale[k])
        print(f"{form}-o{order} rhs_{k}: {e:.2e} (walls {ew:.2e})")
        assert e <= W_TOL, (k, e)


def test_steps_with_walls(pair):
    form, order, ns, ref, gpu, x, y, t = pair
    st = perturbed_state(y, x)
    for o in (ref, gpu):
        o.set_state(**st)
    dtc, dtp = ref.set_tstep()
    assert gpu.set_tstep() == pytest.approx((dtc, dtp), rel=1e-14)
    dt = 0.3 * min(dtc, dtp)
    for o in (ref, gpu):
        o.step(dt, 100)
    sr, sg = ref.state(), gpu.state()
    for k in ["ro", "rou", "rov", "u", "v", "cxx", "cxy", "cyy"]:
        e = rel(sg[k], sr[k])
        print(f"{form}-o{order} {k} after 100 steps: {e:.2e}")
        assert e <= F_TOL, (k, e)
    assert np.all(sg["rou"][t == 0] == 0.0)
    assert abs(gpu.kinetic_energy() - ref.kinetic_energy()) <= 1e-10 * ref.kinetic_energy()


def test_mixed_precision_with_walls():
    ns = channel(32)
    f64 = labfm.Sunset(form="lc", order=8, **PARAMS)
    mx = labfm.Sunset(form="lc", order=8, precision="mixed", **PARAMS)
    for g in (f64, mx):
        g.build_domain(ns)
        g.setup()
    ref = O.Oracle(form="lc", order=8, **PARAMS).build_domain(ns)
    nd = ref.nodes()
    npfb = ref.sizes()[1]
    st = perturbed_state(nd["y"][:npfb], nd["x"][:npfb])
    for g in (f64, mx):
        g.set_state(**st)
    dtc, dtp = f64.set_tstep()
    for g in (f64, mx):
        g.step(0.3 * min(dtc, dtp), 100)
    a, b = mx.state(), f64.state()
    for grp in (["ro"], ["rou", "rov"], ["u", "v"], ["cxx", "cxy", "cyy"]):
        s = max(np.abs(b[k]).max() for k in grp)
        for k in grp:
            e = float(np.abs(a[k] - b[k]).max() / s)
            print(f"walls, mixed vs FP64 {k} after 100 steps: {e:.2e}")
            assert e <= 1e-6, (k, e)


def cylinder_state(x, y):
    """A smooth state on the cylinder channel, vanishing velocity on the cylinder and walls."""
    r = np.hypot(x, y)
    damp = (1.0 - (y / 2.0) ** 2) * (1.0 - np.exp(-50.0 * (r - 1.0) ** 2))
    n = len(x)
    return dict(ro=1.0 + 0.001 * np.sin(np.pi * x / 15.0) * np.cos(np.pi * y / 4.0), u=0.8 * damp,
                v=0.1 * np.sin(np.pi * x / 7.5) * damp, cxx=1.0 + 0.2 * damp, cxy=0.05 * damp, cyy=np.ones(n),
                czz=np.ones(n))


def test_cylinder_channel_against_restatement():
    from sunset_viscoelastic_b200.nodesets import WORKLOADS, reader_nodes
    wl = WORKLOADS["cylinder-channel-o8"]
    ns = wl.nodes()
    O.set_pow_mode(True)
    try:
        ref = O.for_workload(wl, ns).setup()
    finally:
        O.set_pow_mode(False)
    gpu = labfm.for_workload(wl, ns).setup()
    c1, s1, l1 = ref.neighbours()
    c2, s2, l2 = gpu.neighbours()
    np.testing.assert_array_equal(c2, c1)
    for i in range(len(c1)):
        np.testing.assert_array_equal(l2[i, :c1[i]], l1[i, :c1[i]])
    wr, wg = ref.weights(), gpu.weights()
    for k in ["w_grad_sum", "w_lap_sum", "w_hyp_sum", "vol"]:
        e = rel(wg[k], wr[k])
        print(f"cylinder {k}: {e:.2e}")
        assert e <= W_TOL, k
    x, y, t = reader_nodes(ns)
    st = cylinder_state(x, y)
    for o in (ref, gpu):
        o.set_state(**st)
    rr, rg = ref.rhs(), gpu.rhs()
    for k in ["ro", "rou", "rov", "xx", "xy", "yy"]:
        s = max(np.abs(rr[k]).max(), 1.0)
        e = rel(rg[k], rr[k], s)
        print(f"cylinder rhs_{k}: {e:.2e}")
        assert e <= W_TOL, (k, e)
    dtc, dtp = ref.set_tstep()
    for o in (ref, gpu):
        o.step(wl.cfl * min(dtc, dtp), 50)
    sr, sg = ref.state(), gpu.state()
    for k in ["ro", "rou", "rov", "u", "v", "cxx", "cxy", "cyy"]:
        e = rel(sg[k], sr[k])
        print(f"cylinder {k} after 50 steps: {e:.2e}")
        assert e <= F_TOL, (k, e)


# Polymer diffusion next to walls: the transverse Laplacian of c on wall nodes
# (derivatives.F90:306-358) with the one-sided FD normal correction (rhs_di.F90:556-568;
# rhs.F90 also for c_zz, which the Cholesky FENE-P source reads).
MD_CASES = [("di", 8, False), ("chl", 8, False), ("chl", 8, True), ("di", 6, True)]


@pytest.fixture(scope="module", params=MD_CASES, ids=[f"{f}-o{o}{'-fenep' if p else ''}" for f, o, p in MD_CASES])
def md_pair(request):
    form, order, fenep = request.param
    ns = channel(32)
    kw = dict(PARAMS, Mdiff=1e-2, fenep=fenep, fenep_l2=100.0)
    O.set_pow_mode(True)
    try:
        ref = O.Oracle(form=form, order=order, **kw).build_domain(ns).setup()
    finally:
        O.set_pow_mode(False)
    gpu = labfm.Sunset(form=form, order=order, **kw)
    gpu.build_domain(ns)
    gpu.setup()
    nd = ref.nodes()
    npfb = ref.sizes()[1]
    return form, order, ref, gpu, nd["x"][:npfb], nd["y"][:npfb], nd["node_type"][:npfb]


def test_rhs_with_walls_and_polymer_diffusion(md_pair):
    form, order, ref, gpu, x, y, t = md_pair
    st = perturbed_state(y, x)
    st["czz"] = 1.0 + 0.05 * np.sin(2 * np.pi * x) * np.cos(np.pi * y)
    for o in (ref, gpu):
        o.set_state(**st)
    rr, rg = ref.rhs(), gpu.rhs()
    gu = np.abs(ref.gradient(st["u"])).max()
    cmax = max(np.abs(st["cxx"]).max(), np.abs(st["cyy"]).max())
    for k in ["ro", "rou", "rov", "xx", "xy", "yy", "zz"]:
        scale = max(gu * cmax, np.abs(rr[k]).max(), 1e-300)
        e = rel(rg[k], rr[k], scale)
        ew = rel(rg[k][t == 0], rr[k][t == 0], scale)
        print(f"{form}-o{order} Mdiff rhs_{k}: {e:.2e} (walls {ew:.2e})")
        assert e <= W_TOL, (k, e)


def test_steps_with_walls_and_polymer_diffusion(md_pair):
    form, order, ref, gpu, x, y, t = md_pair
    st = perturbed_state(y, x)
    for o in (ref, gpu):
        o.set_state(**st)
    dtc, dtp = ref.set_tstep()
    dt = 0.3 * min(dtc, dtp)
    for o in (ref, gpu):
        o.step(dt, 100)
    sr, sg = ref.state(), gpu.state()
    for k in ["ro", "rou", "rov", "u", "v", "cxx", "cxy", "cyy", "czz"]:
        e = rel(sg[k], sr[k])
        print(f"{form}-o{order} Mdiff {k} after 100 steps: {e:.2e}")
        assert e <= F_TOL, (k, e)
    assert np.all(sg["rou"][t == 0] == 0.0)
