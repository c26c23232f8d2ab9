"""Known-answer tests of the CPU restatement (the oracle), run without a GPU.

The reference ships no test suite and no golden outputs, and it cannot be compiled here
(Fortran).  The restatement is pinned instead by what the reference itself solves for and
checks: the LABFM moment conditions (labf.F90:153-180), its own analytic steady state
(the Kolmogorov initial condition of setup_flow.F90:224-229 with the forcing of
rhs.F90:275, statistics.F90:552-612), mass conservation under the mass correction
(rhs_di.F90:697-717), and building blocks against independent computations.
"""
import ctypes
import dataclasses
import math
import os
import random
from fractions import Fraction

import numpy as np
import pytest

from sunset_viscoelastic_b200.nodesets import (NodeSet, WORKLOADS, channel, inflow_channel, inflow_state, initial_state,
                                               jittered_lattice, poiseuille_state)
import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))


def fixture_nodes():
    d = np.load(os.path.join(HERE, "golden", "ipart_fixture.npz"))
    b = d["box"]
    ns = NodeSet(x=d["x"], y=d["y"], node_type=d["node_type"], nx=d["nx"], ny=d["ny"], s=d["s"],
                 xmin=b[0], xmax=b[1], ymin=b[2], ymax=b[3], bcond=tuple(int(v) for v in d["bcond"]), gi=d["gi"])
    return ns, dict(zip(["L_char", "U_char", "Re", "Wi", "beta", "epsPTT", "fenep_l2", "Mdiff", "Ma"],
                        (float(v) for v in d["control"])))


# ------------------------------------------------------------------------------------ blocks
def test_svd_solve_matches_lapack():
    rng = np.random.default_rng(1)
    for n in (5, 14, 27, 44):
        A = rng.standard_normal((n, n)) + n * np.eye(n)
        b = rng.standard_normal(n)
        x = b.copy()
        O.lib().or_svd_solve(np.asfortranarray(A).ravel(order="F").copy(), n, x)
        np.testing.assert_allclose(x, np.linalg.solve(A, b), rtol=1e-10, atol=1e-12)


def test_svd_solve_skips_zero_singular_values():
    """svdlib.F90:286: an exactly singular system gives the minimum-norm-like solution
    with the zero singular value skipped, not inf/nan."""
    A = np.diag([2.0, 1.0, 0.0])
    x = np.array([2.0, 3.0, 5.0])
    O.lib().or_svd_solve(np.asfortranarray(A).ravel(order="F").copy(), 3, x)
    assert np.all(np.isfinite(x))
    np.testing.assert_allclose(x[:2], [1.0, 3.0])


def test_monomials_and_hermite_abfs():
    x, y = 0.37, -0.81
    for order in (4, 6, 8, 10):
        n = (order * order + 3 * order) // 2
        mono, abf = np.zeros(n), np.zeros(n)
        O.lib().or_monomials(order, x, y, mono)
        O.lib().or_abfs(order, x, y, abf)
        # probabilists' Hermite polynomials from numpy's HermiteE basis
        from numpy.polynomial import hermite_e as He
        m = 0
        for d in range(1, order + 1):
            for p in range(d, -1, -1):
                q = d - p
                assert mono[m] == pytest.approx(x ** p * y ** q / (math.factorial(p) * math.factorial(q)), rel=1e-13)
                hp = He.hermeval(x, [0] * p + [1])
                hq = He.hermeval(y, [0] * q + [1])
                assert abf[m] == pytest.approx(hp * hq, rel=1e-12, abs=1e-12)
                m += 1


def test_wendland_c2():
    h2 = 0.3 ** 2
    for q in (0.0, 0.5, 1.0, 1.999, 2.0, 2.5):
        w = O.lib().or_wab(q, h2)
        expect = 7.0 / (4.0 * math.pi * h2) * (2 * q + 1) * (1 - q / 2) ** 4 if 0 < q <= 2 else 0.0
        assert w == pytest.approx(expect, rel=1e-14, abs=1e-300)


def test_correctly_rounded_pow4():
    """The device's x^4 (and the restatement's set_pow_mode(True)) is the correctly
    rounded power; glibc's pow(x, 4.0), which the reference calls, is not always."""
    L = O.lib()
    rnd = random.Random(5)
    libm_wrong = 0
    for _ in range(20000):
        x = rnd.random()
        cr = float(Fraction(x) ** 4)
        assert L.or_pow4_cr(x) == cr
        libm_wrong += L.or_pow4_libm(x) != cr
    assert libm_wrong < 100


# ------------------------------------------------------------------------------ neighbours
def test_neighbour_search_matches_brute_force():
    wl = WORKLOADS["periodic-di-o4-16k"]
    ns = jittered_lattice(24, seed=9)
    o = O.Oracle(form="di", order=4, h_over_s=wl.h_over_s).build_domain(ns)
    o.find_neighbours()
    nd = o.nodes()
    cnt, cs, links = o.neighbours()
    npfb = ns.n
    x, y, h = nd["x"], nd["y"], nd["h"]
    for i in range(0, npfb, 37):
        d2 = (x[i] - x) ** 2 + (y[i] - y) ** 2
        expect = set(np.nonzero(d2 <= (2 * h[i]) ** 2)[0] + 1)
        got = links[i, :cnt[i]]
        assert set(got) == expect
        dist = d2[got - 1]
        assert np.all(np.diff(dist) >= 0)             # sorted by distance (neighbours.F90:272-314)
        assert got[0] == i + 1                         # self first


def test_mirror_points_are_periodic_images():
    ns = jittered_lattice(20, seed=3)
    o = O.Oracle(form="di", order=4, h_over_s=1.5).build_domain(ns)
    nd = o.nodes()
    np_, npfb = o.sizes()[:2]
    par = nd["irelation"][npfb:] - 1
    dx = nd["x"][npfb:] - nd["x"][par]
    dy = nd["y"][npfb:] - nd["y"][par]
    assert np.all(np.isin(np.round(dx, 12), [-1.0, 0.0, 1.0]))
    assert np.all(np.isin(np.round(dy, 12), [-1.0, 0.0, 1.0]))
    assert np.all(nd["vrelation"][npfb:] == 1)


# ------------------------------------------------------------------------- moment conditions
@pytest.mark.parametrize("order,radius,tol", [(4, 3.0, 1e-11), (6, 4.2, 1e-9), (8, 4.72, 2e-6), (8, 5.4, 2e-6)])
def test_weights_reproduce_polynomials(order, radius, tol):
    """labf.F90:153-180: the d/dx, d/dy and Laplacian weights are exact on every monomial
    up to the order.  In the stencil's scaled variables (r/h, weights times h or h^2) the
    moment conditions read sum_k w_k m(r_k) = derivative of m at 0."""
    ns = jittered_lattice(24, seed=11)
    o = O.Oracle(form="di", order=order, h_over_s=radius / 2).build_domain(ns).setup()
    nd = o.nodes()
    cnt, cs, links = o.neighbours()
    w = o.weights()
    worst = 0.0
    for i in range(0, ns.n, 53):
        j = links[i, :cs[i]] - 1
        h = nd["h_small"][i]
        X, Y = (nd["x"][j] - nd["x"][i]) / h, (nd["y"][j] - nd["y"][i]) / h
        wx, wy, wl = w["w_grad"][i, :cs[i], 0] * h, w["w_grad"][i, :cs[i], 1] * h, w["w_lap"][i, :cs[i]] * h * h
        for d in range(1, order + 1):
            for p in range(d, -1, -1):
                q = d - p
                m = X ** p * Y ** q
                worst = max(worst, abs(wx @ m - ((p, q) == (1, 0))), abs(wy @ m - ((p, q) == (0, 1))),
                            abs(wl @ m - 2.0 * ((p, q) in ((2, 0), (0, 2)))))
    # the un-truncated SVD solve meets the conditions to cond(A)*eps, ~1e9*eps at order 8
    print("order", order, "worst moment residual", worst)
    assert worst < tol, worst


def test_ipart_fixture_setup():
    """The reference's own fixture with its default parameters (order 8, hovs 2.7)."""
    ns, c = fixture_nodes()
    o = O.Oracle(form="chl", order=8, Re=c["Re"], Wi=c["Wi"], beta=c["beta"], epsPTT=c["epsPTT"],
                 fenep_l2=c["fenep_l2"], Mdiff=c["Mdiff"], Ma=c["Ma"]).build_domain(ns).setup()
    np_, npfb, nb, nplink = o.sizes()
    assert npfb == 4056 and nb == 0
    cnt, cs, links = o.neighbours()
    assert cnt.min() >= 44                # more neighbours than order-8 unknowns
    assert nplink <= 2 * 4 * math.ceil(2.0 * 2.7) ** 2  # nplink bound of setup_domain.F90:50
    w = o.weights()
    assert np.all(np.isfinite(w["w_grad"])) and np.all(np.isfinite(w["w_hyp"]))
    # node volumes tile the periodic box
    assert abs(w["vol"].sum() / (2 * math.pi) ** 2 - 1.0) < 0.05


@pytest.mark.parametrize("form,Wi,Mdiff,tol", [("di", 0.3, 1e-3, 1e-7), ("chl", 0.3, 1e-3, 1e-7), ("lc", 1.0, 0.0, 1e-5)])
def test_kolmogorov_steady_state_is_a_fixed_point(form, Wi, Mdiff, tol):
    """setup_flow.F90:224-229 with the forcing of rhs.F90:275 is an exact steady state of
    the PDE; the discrete right-hand side must vanish to discretisation accuracy, in every
    formulation (the log-conformation form has no polymer diffusion, so Mdiff = 0 there)."""
    ns, c = fixture_nodes()
    o = O.Oracle(form=form, order=8, Re=c["Re"], Wi=Wi, beta=c["beta"], epsPTT=c["epsPTT"],
                 fenep_l2=c["fenep_l2"], Mdiff=Mdiff, Ma=c["Ma"], kolmogorov_forcing=1).build_domain(ns).setup()
    x, y = ns.x, ns.y
    u = np.cos(y)
    v = np.zeros_like(y)
    cxx = 1 + (Wi * Wi / (1 + Mdiff * Wi)) * (1 - np.cos(2 * y) / (1 + 4 * Mdiff * Wi))
    cxy = -Wi * np.sin(y) / (1 + Mdiff * Wi)
    o.set_state(np.ones(ns.n), u, v, cxx, cxy, np.ones(ns.n))
    r = o.rhs()
    scale = 1.0 / c["Re"]   # size of the balanced momentum terms
    assert np.abs(r["rou"]).max() < tol * 100 * scale + tol
    assert np.abs(r["rov"]).max() < tol * 100 * scale + tol
    for k in ("xx", "xy", "yy"):
        assert np.abs(r[k]).max() < 100 * tol, (k, np.abs(r[k]).max())
    # and a perturbed state is not a fixed point (the check has teeth)
    o.set_state(np.ones(ns.n), 1.1 * u, v, cxx, cxy, np.ones(ns.n))
    assert np.abs(o.rhs()["rou"]).max() > 1e-4


def test_mass_correction_conserves_mass():
    """rhs_di.F90:697-717: after every step sum (rho - 1) vol = 0 to rounding."""
    import dataclasses
    wl = dataclasses.replace(WORKLOADS["periodic-di-o4-16k"], nside=32)
    ns = wl.nodes()
    o = O.for_workload(wl, ns).setup()
    st = initial_state(ns)
    st["ro"] = 1.0 + 0.01 * np.sin(2 * np.pi * ns.x)
    o.set_state(**st)
    dtc, dtp = o.set_tstep()
    o.step(wl.cfl * min(dtc, dtp), 10)
    vol = o.weights()["vol"]
    m = float(np.sum((o.state()["ro"] - 1.0) * vol))
    assert abs(m) < 1e-13


def test_transforms_round_trip():
    """conf_transforms.F90: c -> psi -> c for log-conformation and log-Cholesky."""
    import dataclasses
    wl = dataclasses.replace(WORKLOADS["periodic-lc-o6-262k"], nside=16)
    ns = wl.nodes()
    rng = np.random.default_rng(2)
    a = 1 + rng.random(ns.n)
    b = 0.3 * (rng.random(ns.n) - 0.5)
    d = 1 + rng.random(ns.n)
    for form in ("lc", "chl"):
        o = O.Oracle(form=form, order=6, h_over_s=wl.h_over_s).build_domain(ns)
        o.set_state(np.ones(ns.n), np.zeros(ns.n), np.zeros(ns.n), a, b, d)
        s = o.state()
        np.testing.assert_allclose(s["cxx"], a, rtol=1e-13)
        np.testing.assert_allclose(s["cxy"], b, rtol=1e-10, atol=1e-12)
        np.testing.assert_allclose(s["cyy"], d, rtol=1e-13)


# ------------------------------------------------------------------------------- wall closures
def channel_oracle(order, form="di", ncell=32, G=8.0, Wi=0.5, beta=0.59):
    o = O.Oracle(form=form, order=order, Re=1.0, Wi=Wi, beta=beta, Ma=0.1, grav=(G, 0.0, 0.0),
                 kolmogorov_forcing=0)
    o.build_domain(channel(ncell)).setup()
    return o


@pytest.mark.parametrize("order", [6, 8])
def test_boundary_operators_reproduce_polynomials(order):
    """labf.F90:505-1039 on a straight walled channel.  Wall nodes: first derivatives in the
    normal-tangent frame, the normal one a 5-point one-sided difference (exact to degree 4),
    the tangential one 6th-order 1-D LABFM (exact on polynomials in x up to degree 6).  FD
    rows 1 and 2: the same operators rotated to x-y.  Checked away from the periodic seam,
    where x^p is not periodic."""
    o = channel_oracle(order)
    nd = o.nodes()
    npfb = o.sizes()[1]
    x, y, t = nd["x"][:npfb], nd["y"][:npfb], nd["node_type"][:npfb]
    inner = (x > 0.3) & (x < 0.7)
    wall, rows = (t == 0) & inner, ((t == -1) | (t == -2)) & inner
    nsgn = np.where(y[wall] < 0.5, 1.0, -1.0)  # wall normal is +y at the bottom, -y at the top
    tsgn = -nsgn  # tangent (-n_y, n_x): -x at the bottom, +x at the top
    worst = 0.0
    for p in range(1, 5):  # normal direction
        g = o.gradient(y ** p)
        d = p * y ** (p - 1)
        worst = max(worst, np.abs(g[wall, 0] - nsgn * d[wall]).max(), np.abs(g[rows, 1] - d[rows]).max() / max(1, p))
    for p in range(1, 7):  # tangential direction
        g = o.gradient((x - 0.5) ** p)
        d = p * (x - 0.5) ** (p - 1)
        worst = max(worst, np.abs(g[wall, 1] - tsgn * d[wall]).max(), np.abs(g[rows, 0] - d[rows]).max())
    print("order", order, "worst boundary residual", worst)
    assert worst < 1e-7, worst


@pytest.mark.parametrize("order,form,tol", [(6, "di", 1e-9), (8, "di", 1e-9), (8, "lc", 1e-9)])
def test_poiseuille_is_a_fixed_point(order, form, tol):
    """Steady Oldroyd-B channel flow driven by a body force (the reference checks Poiseuille
    flow in statistics.F90:444-550): u = G y (1-y)/(2 mu), c_xy = lam u', c_xx = 1+2(lam u')^2
    is polynomial, so interior LABFM, FD rows, 1-D LABFM and the wall closure
    (rhs_di.F90:146-158,291-309,497-512; calc_rhs_nscbc, characteristic_boundaries.F90:27-52)
    must all return a zero right-hand side to rounding.  (The log-conformation form evolves
    psi = log c, which is not polynomial, so only its momentum right-hand side is checked.)"""
    G = 8.0
    o = channel_oracle(order, form, G=G)
    nd = o.nodes()
    npfb = o.sizes()[1]
    st = poiseuille_state(type("P", (), {"y": nd["y"][:npfb], "n": npfb}), G, 1.0, 0.5)
    o.set_state(**st)
    r = o.rhs()
    keys = ["ro", "rou", "rov"] + (["xx", "xy", "yy"] if form == "di" else [])
    worst = max(np.abs(r[k]).max() for k in keys) / G
    print(order, form, "max |rhs| / G", worst)
    assert worst < tol, worst


def test_cylinder_channel_stencils_and_first_steps():
    """The walled cylinder channel (labf.F90 boundary framework on a curved wall): every
    stencil is well conditioned and the restatement steps it from rest under the body
    force, the wall momentum staying zero."""
    wl = WORKLOADS["cylinder-channel-o8"]
    ns = wl.nodes()
    O.set_threads(os.cpu_count() or 1)
    o = O.for_workload(wl, ns).setup()
    nd = o.nodes()
    npfb = o.sizes()[1]
    t, sp = nd["node_type"][:npfb], nd["s"][:npfb]
    w = o.weights()
    lap = np.abs(w["w_lap"]).max(axis=1) * sp ** 2
    assert np.all(np.isfinite(lap))
    assert lap[t != 0].max() < 10.0, lap[t != 0].max()
    o.set_state(**wl.initial(ns))
    dtc, dtp = o.set_tstep()
    o.step(wl.cfl * min(dtc, dtp), 10)
    st = o.state()
    assert all(np.all(np.isfinite(st[k])) for k in ("ro", "u", "v", "cxx"))
    assert np.all(st["rou"][t == 0] == 0.0)
    assert st["u"].max() > 0.0


@pytest.mark.parametrize("form", ["di", "chl", "lc"])
def test_fenep_relaxation_agrees_across_forms(form):
    """FENE-P at rest with a uniform conformation tensor: every form must give
    dc/dt = -(f c - I) / lambda with f = (L^2 - 3) / (L^2 - tr c) (rhs_di.F90:444-449).
    The Cholesky form evolves factors of J = f c (rhs.F90:480-541, conf_transforms.F90:39-101)
    and the log-conformation form log c (rhs_lc.F90:520-535), so their right-hand sides are
    mapped back to dc/dt through the restatement's own transforms by a central difference."""
    L2, Wi = 50.0, 1.0
    wl = dataclasses.replace(WORKLOADS["periodic-di-o4-16k"], nside=16, form=form, Wi=Wi, epsPTT=0.0,
                             kolmogorov_forcing=0)
    ns = wl.nodes()
    o = O.for_workload(wl, ns, fenep=True, fenep_l2=L2).setup()
    n = ns.n
    c = dict(cxx=2.0, cxy=0.5, cyy=1.5, czz=1.0 if form == "lc" else 1.2)
    one, zero = np.ones(n), np.zeros(n)
    o.set_state(ro=one, u=zero, v=zero, **{k: v * one for k, v in c.items()})
    r = o.rhs()
    f = (L2 - 3.0) / (L2 - (c["cxx"] + c["cyy"] + c["czz"]))
    expect = {"cxx": -(f * c["cxx"] - 1.0) / Wi, "cxy": -(f * c["cxy"]) / Wi, "cyy": -(f * c["cyy"] - 1.0) / Wi,
              "czz": -(f * c["czz"] - 1.0) / Wi}
    if form == "di":
        got = {"cxx": r["xx"], "cxy": r["xy"], "cyy": r["yy"], "czz": r["zz"]}
    else:
        st = o.state()
        q = np.array([st["psixx"], st["psixy"], st["psiyy"], st["psizz"]])
        rq = np.array([r["xx"], r["xy"], r["yy"], r["zz"]])
        eps = 1e-6
        cs = []
        for sgn in (1.0, -1.0):
            o.set_raw_state(one, zero, zero, q + sgn * eps * rq)
            cs.append(o.state())
        got = {k: (cs[0][k] - cs[1][k]) / (2 * eps) for k in expect}
    keys = ["cxx", "cxy", "cyy"] + ([] if form == "lc" else ["czz"])
    for k in keys:
        err = np.abs(got[k] - expect[k]).max()
        print(form, k, "dc/dt", got[k][0], "expected", expect[k], "error", err)
        assert err <= 1e-8 * max(1.0, abs(expect[k])), (k, err)
    assert np.abs(r["ro"]).max() < 1e-12 and np.abs(r["rou"]).max() < 1e-10


def test_adapt_stencils_invariants():
    """adapt_stencils + adapt_stencils_main (labf.F90:1079-1721) restated, from the reference's
    own initial lengths: h and h_small never grow and shrink in whole steps of the
    single-precision factor 0.98, at most 26 times; only plain interior nodes change (walls and
    FD rows keep theirs); the rebuilt lists hold exactly the points within 2 h of each node;
    and the adapted stencils are well conditioned."""
    rf = float(np.float32(0.98))
    for ns, form, order in [(jittered_lattice(32, 0.3, seed=5), "lc", 6), (channel(16), "di", 8)]:
        o = O.Oracle(form=form, order=order, h_over_s=0.0).build_domain(ns)
        o.find_neighbours()
        nd0 = o.nodes()
        n = o.sizes()[1]
        h0 = nd0["h"][:n].copy()
        o.adapt_stencils()
        nd = o.nodes()
        h, hs, t = nd["h"][:n], nd["h_small"][:n], nd["node_type"][:n]
        assert np.all(h <= h0) and np.all(hs <= h)
        steps = np.log(h / h0) / np.log(rf)
        assert np.all(np.abs(steps - np.round(steps)) < 1e-6) and steps.max() <= 26
        assert np.all(h[t <= 2] == h0[t <= 2])
        assert np.sum(h < h0) > 0
        c, cs, lk = o.neighbours()
        x, y = nd["x"], nd["y"]
        for i in range(0, n, 37):
            d2 = (x - x[i]) ** 2 + (y - y[i]) ** 2
            assert c[i] == int(np.sum(d2 <= (2.0 * h[i]) ** 2)), i
        o.setup()  # the neighbour search again (same lists), weights, boundary weights, sums
        w = o.weights()
        lap = np.abs(w["w_lap"][t > 2]).max(axis=1) * nd["s"][:n][t > 2] ** 2
        print(form, order, "reduced", int(np.sum(h < h0)), "of", n, "max steps", int(steps.max()),
              "max |w_lap| s^2 interior", lap.max())
        assert lap.max() < 10.0


@pytest.mark.parametrize("form, eps, fenep", [("di", 0.25, False), ("chl", 0.25, False), ("lc", 0.0, False),
                                              ("newt", 0.0, False), ("di", 0.0, True), ("chl", 0.0, True)])
def test_3d_reduces_to_2d(form, eps, fenep):
    """3-D restatement, known answer: with w = 0, c_xz = c_yz = 0, c_zz = 1 and fields that do
    not vary in z, every layer's right-hand side is the 2-D one (the z stencils see constants;
    rho w, c_xz and c_yz stay at rest).  The log-conformation form takes eps = 0: its 3-D sPTT
    trace includes c_zz, the 2-D one does not (rhs_lc.F90:451-456).  FENE-P (direct form): the
    function f and its gradient enter the momentum and the relaxation alike in 2-D and 3-D
    (rhs_di.F90:198-245, 454-464).  FENE-P (Cholesky form): the factors of J = f c, whose
    source terms and transforms reduce to the 2-D ones when psi_xz = psi_yz = 0
    (rhs.F90:479-500, conf_transforms.F90:39-58)."""
    wl = dataclasses.replace(WORKLOADS["periodic-lc-o6-262k"], nside=16, form=form, epsPTT=eps)
    ns = wl.nodes()
    extra = dict(fenep=True, fenep_l2=30.0) if fenep else {}
    o = O.for_workload(wl, ns, kolmogorov_forcing=0, **extra).setup()
    o3 = O.Oracle3(o, 0.4)
    nl = o3.nl
    x, y = ns.x, ns.y
    tp = 2.0 * np.pi
    st = dict(ro=1.0 + 0.01 * np.cos(tp * x), u=np.sin(tp * x) * np.cos(tp * y), v=-np.cos(tp * x) * np.sin(tp * y),
              cxx=1.2 + 0.1 * np.sin(tp * x), cxy=0.1 * np.cos(tp * y), cyy=1.1 + 0.05 * np.cos(tp * x), czz=np.ones(nl))
    o.set_state(**st)
    r2 = o.rhs()
    T = lambda a: np.tile(a, o3.nz)
    zero = np.zeros(o3.n)
    o3.set_state(T(st["ro"]), T(st["u"]), T(st["v"]), zero, T(st["cxx"]), T(st["cxy"]), T(st["cyy"]), zero, zero,
                 np.ones(o3.n))
    r3 = o3.rhs()
    keys = ["ro", "rou", "rov"] + ([] if form == "newt" else ["xx", "xy", "yy"]) + (["zz"] if fenep else [])
    for k in keys:
        scale = max(np.abs(r2[k]).max(), 1.0)
        e = np.abs(r3[k].reshape(o3.nz, nl) - r2[k][None, :]).max() / scale
        assert e < 1e-9, (form, k, e)
    for k in ["row", "xz", "yz"]:
        assert np.abs(r3[k]).max() < 1e-9 * max(np.abs(r2["rou"]).max(), 1.0), (form, k)


@pytest.mark.parametrize("form, eps, mdiff, fenep", [("di", 0.25, 1e-3, False), ("chl", 0.25, 1e-3, False),
                                                     ("lc", 0.0, 0.0, False), ("newt", 0.0, 0.0, False),
                                                     ("di", 0.0, 1e-3, True), ("chl", 0.0, 1e-3, True)])
def test_3d_walls_reduce_to_2d(form, eps, mdiff, fenep):
    """3-D restatement with walls, known answer: on a channel (walls at y = 0 and 1, node_type
    0) a state that does not vary in z, with w = 0, c_xz = c_yz = 0 and c_zz = 1, gives on every
    layer the 2-D right-hand side, the wall nodes' included: the wall closure of the flow
    (rhs_di.F90:149-154, 291-307, 601-665 with characteristic_boundaries.F90:27-52; its dim3
    terms, rho dw/dz and L4, vanish), the conformation equations with the rotated velocity
    gradients, and under polymer diffusion the tangential Laplacian with the one-sided normal
    second derivative over the FD rows (rhs_di.F90:553-580, rhs.F90:631-643).  The
    log-conformation form takes eps = 0 (its 3-D trace includes c_zz).  After a few steps
    rho u, rho v and rho w stay zero on the walls (apply_time_dependent_bounds)."""
    G = 8.0
    ns = channel(24)
    extra = dict(fenep=True, fenep_l2=30.0) if fenep else {}
    o = O.Oracle(form=form, order=6, Re=1.0, Wi=0.5, beta=0.59, Ma=0.1, grav=(G, 0.0, 0.0), kolmogorov_forcing=0,
                 epsPTT=eps, Mdiff=mdiff, **extra).build_domain(ns).setup()
    o3 = O.Oracle3(o, 0.4)
    nl = o3.nl
    nd = o.nodes()
    x, y, t = nd["x"][:nl], nd["y"][:nl], nd["node_type"][:nl]
    assert np.sum(t == 0) > 0
    st = poiseuille_state(type("P", (), {"y": y, "n": nl}), G, 1.0, 0.5)
    st["u"] = st["u"] + 0.3 * np.sin(2 * np.pi * x) * y * (1.0 - y)
    st["v"] = 0.2 * np.cos(2 * np.pi * x) * y * (1.0 - y)
    st["ro"] = 1.0 + 0.01 * np.sin(2 * np.pi * x) * np.cos(np.pi * y)
    st["cxx"] = st["cxx"] + 0.1 * np.sin(2 * np.pi * x) ** 2
    st["cyy"] = st["cyy"] + 0.05 * np.cos(np.pi * y) ** 2
    o.set_state(st["ro"], st["u"], st["v"], st["cxx"], st["cxy"], st["cyy"], np.ones(nl))
    r2 = o.rhs()
    T = lambda a: np.tile(a, o3.nz)
    zero = np.zeros(o3.n)
    o3.set_state(T(st["ro"]), T(st["u"]), T(st["v"]), zero, T(st["cxx"]), T(st["cxy"]), T(st["cyy"]), zero, zero,
                 np.ones(o3.n))
    r3 = o3.rhs()
    keys = ["ro", "rou", "rov"] + ([] if form == "newt" else ["xx", "xy", "yy"])
    for k in keys:
        scale = max(np.abs(r2[k]).max(), 1.0)
        d = np.abs(r3[k].reshape(o3.nz, nl) - r2[k][None, :])
        assert d.max() / scale < 1e-9, (form, k, d.max() / scale)
        assert d[:, t == 0].max() / scale < 1e-13, (form, k, "walls")
    dc, dp = o3.set_tstep()
    o3.step(0.3 * min(dc, dp), 3)
    s3 = o3.state()
    for k in ("rou", "rov", "row", "u", "v", "w"):
        assert np.all(s3[k].reshape(o3.nz, nl)[:, t == 0] == 0.0), k
    assert all(np.isfinite(a).all() for a in s3.values())


@pytest.mark.parametrize("form, itype, extra", [("di", 0, {}), ("di", 1, {}), ("lc", 2, {}), ("chl", 0, {"Mdiff": 1e-3}),
                                                ("chl", 1, {})])
def test_3d_inout_reduces_to_2d(form, itype, extra):
    """3-D restatement with inflow and outflow nodes, known answer: on the inflow channel a state
    that does not vary in z, with w = 0, c_xz = c_yz = 0 and c_zz = 1, gives on every layer the
    2-D right-hand sides, the inflow and outflow node-layers' included (rhs_di.F90:155-157,
    311-359, characteristic_boundaries.F90:54-189 and calc_rhs_nscbc with their dim3 terms, which
    vanish here; the Cholesky form's inflow advection and one-sided flux closure,
    rhs.F90:558-643).  The log-conformation form takes eps = 0 (its 3-D trace includes c_zz)."""
    ns = inflow_channel(24, ybc=1)
    order = {"di": 4, "lc": 6, "chl": 8}[form]
    kw = dict(Re=10.0, Wi=0.5, beta=0.59, Ma=0.1, kolmogorov_forcing=0, form=form, order=order, inflow_type=itype,
              epsPTT=0.0, **extra)
    o = O.Oracle(**kw).build_domain(ns).setup()
    o3 = O.Oracle3(o, 0.4)
    nl = o3.nl
    nd = o.nodes()
    t = nd["node_type"][:nl]
    assert np.sum(t == 1) > 0 and np.sum(t == 2) > 0
    st = inflow_state(type("R", (), {"x": nd["x"][:nl], "y": nd["y"][:nl]}))
    o.set_state(**st)
    r2 = o.rhs()
    T = lambda a: np.tile(a, o3.nz)
    zero = np.zeros(o3.n)
    o3.set_state(T(st["ro"]), T(st["u"]), T(st["v"]), zero, T(st["cxx"]), T(st["cxy"]), T(st["cyy"]), zero, zero,
                 np.ones(o3.n))
    r3 = o3.rhs()
    io = (t == 1) | (t == 2)
    for k in ["ro", "rou", "rov"] + ([] if form == "di" else ["xx", "xy", "yy"]):
        scale = max(np.abs(r2[k]).max(), 1.0)
        d = np.abs(r3[k].reshape(o3.nz, nl) - r2[k][None, :])
        assert d.max() / scale < 1e-9, (form, k, d.max() / scale)
        assert d[:, io].max() / scale < 1e-11, (form, k, "inflow/outflow")
    dc, dp = o3.set_tstep()
    o3.step(0.3 * min(dc, dp), 3)
    s3 = o3.state()
    assert all(np.isfinite(a).all() for a in s3.values())
    if itype == 1:  # hard inflow: v = w = 0 there
        for k in ("rov", "row"):
            assert np.all(s3[k].reshape(o3.nz, nl)[:, t == 1] == 0.0), k


@pytest.mark.parametrize("order, tol", [(4, 2e-2), (6, 5e-4), (8, 2e-5)])
def test_shear_wave_decays_at_the_viscous_rate(order, tol):
    """Known answer in time: the shear wave u = sin(2 pi y), v = 0, rho = 1 solves the
    compressible momentum equation exactly (no advection, no pressure gradient, divergence
    free), decaying as exp(-nu k^2 t) with nu = mu_solvent / rho (load_data.F90:131-138) and
    k = 2 pi.  The Newtonian restatement on a jittered periodic set (32 nodes a wavelength)
    follows it within the error of its stencils, its hyperviscous filter and RK3, which falls
    with the order: the amplitude's error after 20 steps, relative to the decayed amount, is
    about 1e-2, 2e-4 and 3e-6 at orders 4, 6 and 8."""
    name = {4: "periodic-di-o4-16k", 6: "periodic-lc-o6-262k", 8: "periodic-chl-o8-1m"}[order]
    wl = dataclasses.replace(WORKLOADS[name], nside=32)
    ns = wl.nodes()
    o = O.for_workload(wl, ns, form="newt", kolmogorov_forcing=0, Re=1.0, beta=0.5).setup()
    n = o.sizes()[1]
    y = o.nodes()["y"][:n]
    shape = np.sin(2.0 * np.pi * y)
    one = np.ones(n)
    o.set_state(one, shape.copy(), np.zeros(n), one, np.zeros(n), one, one)
    dtc, dtp = o.set_tstep()
    dt = 0.3 * min(dtc, dtp)
    steps = 20
    o.step(dt, steps)
    u = o.state()["u"]
    amp = float(u @ shape / (shape @ shape))
    nu = 0.5 * 1.0 / 1.0  # beta * visc_total / rho with visc_total = rho_char U L / Re = 1
    exact = math.exp(-nu * (2.0 * np.pi) ** 2 * dt * steps)
    assert 1.0 - exact > 0.01  # the decay is measurable
    assert abs(amp - exact) < tol * (1.0 - exact), (order, amp, exact)


@pytest.mark.parametrize("order, tol", [(4, 5e-2), (6, 1e-3), (8, 2e-5)])
def test_shear_wave_in_z_decays_at_the_viscous_rate(order, tol):
    """The same exact solution across the layers: u = sin(2 pi z / Lz), v = w = 0, rho = 1 on a
    3-D layered set (build_3rd_dimension, setup_domain.F90:435-547; Lz = 1, dz = 0.04) decays as
    exp(-nu k^2 t), k = 2 pi / Lz, through the z finite-difference stencils (fd.F90:27-256) and
    the z filter alone.  After 20 steps the amplitude's error relative to the decay is about
    3e-2, 5e-4 and 8e-6 at orders 4, 6 and 8, and v and w stay at rounding."""
    name = {4: "periodic-di-o4-16k", 6: "periodic-lc-o6-262k", 8: "periodic-chl-o8-1m"}[order]
    wl = dataclasses.replace(WORKLOADS[name], nside=24)
    kw = dict(wl.params(), form="newt", kolmogorov_forcing=0, Re=1.0, beta=0.5)
    O.set_pow_mode(True)
    try:
        layer = O.Oracle(**kw).build_domain(wl.nodes()).setup()
    finally:
        O.set_pow_mode(False)
    r = O.Oracle3(layer, 1.0)
    Lz = r.nz * r.dz
    m = r.nl * r.nz
    shape = np.sin(2.0 * np.pi * np.repeat(np.arange(r.nz) * r.dz, r.nl) / Lz)
    z = np.zeros(m)
    r.set_state(np.ones(m), shape.copy(), z, z)
    dt = 0.3 * min(r.set_tstep())
    r.step(dt, 20)
    st = r.state()
    amp = float(st["u"] @ shape / (shape @ shape))
    exact = math.exp(-0.5 * (2.0 * np.pi / Lz) ** 2 * dt * 20)
    assert 1.0 - exact > 0.01
    assert abs(amp - exact) < tol * (1.0 - exact), (order, amp, exact)
    assert np.abs(st["v"]).max() < 1e-13 and np.abs(st["w"]).max() < 1e-13


@pytest.mark.parametrize("form", ["di", "chl", "lc"])
def test_relaxation_at_rest_is_exponential(form):
    """Known answer in time for the conformation equation: at rest with a uniform c0, the
    Oldroyd-B relaxation dc/dt = -(c - I)/lambda (rhs_di.F90:454-476, and the same relaxation
    through the Cholesky and log-conformation variables, rhs.F90:462-547, rhs_lc.F90:519-545)
    gives c(t) = I + (c0 - I) exp(-t/lambda), lambda = Wi L/U (load_data.F90:131-138).  Each form
    integrates it with RK3 in its own variables; c after 60 steps agrees with the exponential to
    1e-9 and the flow stays at rest."""
    wl = dataclasses.replace(WORKLOADS["periodic-lc-o6-262k"], nside=24)
    ns = wl.nodes()
    Wi = 0.5
    o = O.for_workload(wl, ns, form=form, kolmogorov_forcing=0, Wi=Wi, epsPTT=0.0, Mdiff=0.0).setup()
    n = o.sizes()[1]
    c0 = dict(cxx=1.5, cxy=0.2, cyy=1.2, czz=1.3)
    one = np.ones(n)
    o.set_state(one, np.zeros(n), np.zeros(n), c0["cxx"] * one, c0["cxy"] * one, c0["cyy"] * one, c0["czz"] * one)
    dtc, dtp = o.set_tstep()
    dt = 0.3 * min(dtc, dtp)
    steps = 60
    o.step(dt, steps)
    st = o.state()
    decay = math.exp(-dt * steps / Wi)
    assert 1.0 - decay > 0.02
    for k, v in c0.items():
        if k == "czz" and form != "di":
            continue  # c_zz is not evolved by the Cholesky and log-conformation forms in 2-D
        exact = (1.0 if k != "cxy" else 0.0) + (v - (1.0 if k != "cxy" else 0.0)) * decay
        assert np.abs(st[k] - exact).max() < 1e-9, (form, k, np.abs(st[k] - exact).max())
    assert np.abs(st["u"]).max() < 1e-12 and np.abs(st["v"]).max() < 1e-12


@pytest.mark.parametrize("form", ["di", "chl", "lc"])
def test_relaxation_at_rest_3d_is_exponential(form):
    """The relaxation at rest on a 3-D layered set, every component of c (c_xz, c_yz and c_zz
    included) evolved by each form in its own 3-D variables (rhs_di.F90:450-476 with the dim3
    terms; rhs.F90:500-547; rhs_lc.F90:519-545): c = I + (c0 - I) exp(-t/lambda) to 1e-9 after
    60 steps, the flow at rest."""
    wl = dataclasses.replace(WORKLOADS["periodic-di-o4-16k"], nside=24)
    Wi = 0.5
    kw = dict(wl.params(), form=form, kolmogorov_forcing=0, Wi=Wi, epsPTT=0.0, Mdiff=0.0)
    O.set_pow_mode(True)
    try:
        layer = O.Oracle(**kw).build_domain(wl.nodes()).setup()
    finally:
        O.set_pow_mode(False)
    r = O.Oracle3(layer, 0.25)
    m = r.nl * r.nz
    c0 = dict(cxx=1.5, cxy=0.2, cyy=1.2, cxz=0.1, cyz=0.05, czz=1.3)
    ident = dict(cxx=1.0, cxy=0.0, cyy=1.0, cxz=0.0, cyz=0.0, czz=1.0)
    one, z = np.ones(m), np.zeros(m)
    r.set_state(one, z, z, z, **{k: c0[k] * one for k in c0})
    dt = 0.3 * min(r.set_tstep())
    r.step(dt, 60)
    st = r.state()
    decay = math.exp(-dt * 60 / Wi)
    assert 1.0 - decay > 0.02
    for k in c0:
        e = float(np.abs(st[k] - (ident[k] + (c0[k] - ident[k]) * decay)).max())
        assert e < 1e-9, (form, k, e)
    for k in ("rou", "rov", "row"):
        assert np.abs(st[k]).max() < 1e-12, k


def test_3d_output_reduces_to_2d():
    """3-D output quantities, known answer: for a state that does not vary in z with w = 0, the
    3-D dump's vorticity magnitude (output.F90:212-216) is |dv/dx - du/dy| of the layer (the z
    stencils see constants), its state columns repeat the layer's on every layer, and the 3-D
    kinetic energy and mass with dV = vol dz (statistics.F90:305-330) are nz dz times the
    layer's."""
    wl = dataclasses.replace(WORKLOADS["periodic-lc-o6-262k"], nside=16)
    ns = wl.nodes()
    o = O.for_workload(wl, ns, kolmogorov_forcing=0).setup()
    o3 = O.Oracle3(o, 0.4)
    nl, nz, dz = o3.nl, o3.nz, o3.dz
    x, y = ns.x, ns.y
    tp = 2.0 * np.pi
    st = dict(ro=1.0 + 0.01 * np.cos(tp * x), u=np.sin(tp * x) * np.cos(tp * y), v=-np.cos(tp * x) * np.sin(tp * y),
              cxx=1.2 + 0.1 * np.sin(tp * x), cxy=0.1 * np.cos(tp * y), cyy=1.1 + 0.05 * np.cos(tp * x), czz=np.ones(nl))
    o.set_state(**st)
    gu, gv = o.gradient(st["u"]), o.gradient(st["v"])
    vort2 = np.abs(gv[:, 0] - gu[:, 1])
    T = lambda a: np.tile(a, nz)
    zero = np.zeros(o3.n)
    o3.set_state(T(st["ro"]), T(st["u"]), T(st["v"]), zero, T(st["cxx"]), T(st["cxy"]), T(st["cyy"]), zero, zero,
                 np.ones(o3.n))
    cols, hd = o3.dump()
    scale = np.abs(vort2).max()
    assert np.abs(cols["vort"].reshape(nz, nl) - vort2[None, :]).max() < 1e-9 * scale
    for k, ref in (("u", st["u"]), ("v", st["v"])):
        assert np.array_equal(cols[k].reshape(nz, nl), np.tile(ref, (nz, 1))), k
    # c passes through psi and back (the 3x3 eigen solution): equal to rounding
    np.testing.assert_allclose(cols["cxx"].reshape(nz, nl), np.tile(st["cxx"], (nz, 1)), rtol=1e-12)
    assert np.all(cols["w"] == 0.0) and np.all(cols["qcrit"] == 0.0)
    np.testing.assert_allclose(o3.kinetic_energy(), nz * dz * o.kinetic_energy(), rtol=1e-12)
    np.testing.assert_allclose(o3.mass(), nz * dz * o.mass(), rtol=1e-12)


def central_first_derivative(m):
    """Weights a_1..a_m of the central difference of 2m + 1 points for d/dz, from Taylor
    matching in exact rationals: sum_j a_j j^(2q-1) = 1/2 for q = 1 and 0 for q = 2..m."""
    A = [[Fraction(j) ** (2 * q - 1) for j in range(1, m + 1)] for q in range(1, m + 1)]
    b = [Fraction(1, 2)] + [Fraction(0)] * (m - 1)
    for c in range(m):  # Gauss-Jordan
        r = next(r for r in range(c, m) if A[r][c] != 0)
        A[c], A[r], b[c], b[r] = A[r], A[c], b[r], b[c]
        for r in range(m):
            if r != c and A[r][c] != 0:
                f = A[r][c] / A[c][c]
                A[r] = [x - f * y for x, y in zip(A[r], A[c])]
                b[r] -= f * b[c]
    return [b[j] / A[j][j] for j in range(m)]


@pytest.mark.parametrize("wlname", ["periodic-di-o4-16k", "periodic-lc-o6-262k", "periodic-chl-o8-1m"])
def test_3d_z_stencils(wlname):
    """calc_fd_weights (fd.F90:27-256): the periodic z derivative is the central difference of
    order + 1 points.  On w = sin(k z) with k = 2 pi / L_z over a uniform periodic column it
    returns exactly cos(k z) * (2 / dz) sum_j a_j sin(j k dz) (the stencil's modified
    wavenumber), with the a_j derived here independently of the restatement's tables.  With
    rho = 1 and u = v = 0 the continuity right-hand side is -dw/dz."""
    wl = dataclasses.replace(WORKLOADS[wlname], nside=12, form="newt")
    ns = wl.nodes()
    o = O.for_workload(wl, ns, kolmogorov_forcing=0).setup()
    o3 = O.Oracle3(o, 1.0)
    nl, nz, dz = o3.nl, o3.nz, o3.dz
    m = wl.order // 2
    assert nz >= 2 * m + 1
    k = 2.0 * np.pi / (nz * dz)
    z = np.repeat(np.arange(nz) * dz, nl)
    o3.set_state(np.ones(o3.n), np.zeros(o3.n), np.zeros(o3.n), np.sin(k * z))
    r = o3.rhs()
    a = central_first_derivative(m)
    kmod = 2.0 / dz * sum(float(aj) * math.sin((j + 1) * k * dz) for j, aj in enumerate(a))
    err = np.abs(r["ro"] + kmod * np.cos(k * z)).max() / k
    assert err < 1e-11, (wlname, err)
    # and the truncation error has the stencil's order: (k dz)^order sized, not zero
    assert 1e-3 * (k * dz) ** wl.order < abs(kmod - k) / k < (k * dz) ** wl.order
    for key in ("rou", "rov", "xx", "xy", "yy"):
        assert np.abs(r[key]).max() < 1e-12, key


def test_conditioning_of_the_moment_matrices():
    """The condition numbers the library reports, from the restatement's SVD: the stated
    order-6 radius (3.2 s) leaves near-singular moment matrices (sigma_max/sigma_min above
    1e12 at some nodes, where the reference still inverts every nonzero sigma,
    svdlib.F90:283-293), the measured radius 4.2 s does not, and order 8 at 5.4 s sits near
    1e10, the reference's own sensitivity at that order."""
    worst = {}
    for order, name, r in [(6, "periodic-lc-o6-262k", 3.2), (6, "periodic-lc-o6-262k", 4.2),
                           (8, "periodic-chl-o8-1m", 5.4)]:
        wl = dataclasses.replace(WORKLOADS[name], nside=48, radius_over_s=r)
        o = O.for_workload(wl).setup()
        cd, cf = o.conditioning()
        assert np.all(cd >= 1.0) and np.all(cf >= 1.0)
        worst[(order, r)] = (max(cd.max(), cf.max()), int(np.sum(np.maximum(cd, cf) > 1e12)))
    print(worst)
    assert worst[(6, 3.2)][1] > 0
    assert worst[(6, 4.2)][0] < 1e8
    assert 1e8 < worst[(8, 5.4)][0] < 1e12


def test_truncated_node_file_is_rejected(tmp_path):
    """A node file that ends before the rows its header announces (setup_domain.F90:93-199
    reads npfb rows) is an error, not a shorter node set."""
    from sunset_viscoelastic_b200.nodesets import read_ipart, write_ipart
    ns = jittered_lattice(12)
    p = tmp_path / "IPART"
    write_ipart(str(p), ns)
    back = read_ipart(str(p))
    assert back.n == ns.n and np.array_equal(back.x, ns.x)
    lines = p.read_text().splitlines()
    (tmp_path / "IPART_short").write_text("\n".join(lines[:-5]) + "\n")
    with pytest.raises(ValueError, match="ends before"):
        read_ipart(str(tmp_path / "IPART_short"))
    cut = lines[:-1] + [" ".join(lines[-1].split()[:4])]
    (tmp_path / "IPART_cut").write_text("\n".join(cut) + "\n")
    with pytest.raises(ValueError, match="7 columns"):
        read_ipart(str(tmp_path / "IPART_cut"))
