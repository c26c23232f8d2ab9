"""Parity of the CUDA path (through the C-ABI) with the CPU restatement of the reference.

Tolerances (from the specification of the FP64 drop-in): weights and single operators
within 1e-10 relative, fields after 100 steps within 1e-8 relative.

The FP64 path reproduces the restatement operation for operation.  The one difference in
the weight build is the Wendland kernel's (1-q/2)**4: the reference calls libm pow, which
glibc rounds wrongly for about one argument in 1200; the device evaluates x^4 correctly
rounded.  With the restatement switched to the same x^4 (oracle.set_pow_mode) the device
weights are bit-identical.  Against the libm restatement the difference is the
reference's own rounding sensitivity, cond(A)*eps: ~1e-14 at order 4, ~1e-11 at order 6,
but ~1e-7 at order 8, where the moment matrices have condition numbers near 1e9 and the
reference's weights are determined only to that level by its own arithmetic.  The tests
therefore check (a) against the restatement with the device's x^4, at the stated
tolerances (mostly bit-exact), and (b) against the libm restatement, at the stated
tolerance or, where larger, twice the reference's own sensitivity measured as the
distance between the two restatements.
"""
import dataclasses

import numpy as np
import pytest

from sunset_viscoelastic_b200 import labfm
from sunset_viscoelastic_b200.nodesets import WORKLOADS, initial_state
import oracle as O

pytestmark = pytest.mark.gpu

W_TOL = 1e-10      # weights, single operators, right-hand sides
F_TOL = 1e-8       # fields after 100 steps


def rel(a, b, scale=None):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    s = max(np.abs(b).max(), 1e-300) if scale is None else scale
    return float(np.abs(a - b).max() / s)


def small(wl_name, nside, **over):
    return dataclasses.replace(WORKLOADS[wl_name], nside=nside, **over)


CASES = {
    "di-o4": small("periodic-di-o4-16k", 48),
    "lc-o6": small("periodic-lc-o6-262k", 40),
    "chl-o8": small("periodic-chl-o8-1m", 32),
}


def oracle(wl, ns, correctly_rounded):
    O.set_pow_mode(correctly_rounded)
    try:
        return O.for_workload(wl, ns).setup()
    finally:
        O.set_pow_mode(False)


@pytest.fixture(scope="module", params=list(CASES))
def trio(request):
    """(name, workload, nodes, libm restatement, restatement with the device's x^4, device)"""
    wl = CASES[request.param]
    ns = wl.nodes()
    return (request.param, wl, ns, oracle(wl, ns, False), oracle(wl, ns, True),
            labfm.for_workload(wl, ns).setup())


def check(name, what, dev, ref, cr, tol, scale=None):
    """dev vs the two restatements; see the module docstring."""
    d_cr = rel(dev, cr, scale)
    d_ref = rel(dev, ref, scale)
    own = rel(cr, ref, scale)
    print(f"{name} {what}: vs restatement(device x^4) {d_cr:.2e}  vs libm restatement {d_ref:.2e}  "
          f"(restatement's own sensitivity {own:.2e})")
    assert d_cr <= tol, (what, d_cr)
    assert d_ref <= max(tol, 2.0 * own), (what, d_ref, own)


def test_neighbours_identical(trio):
    name, wl, ns, ref, cr, gpu = trio
    assert ref.sizes()[:3] == gpu.sizes()[:3]          # np (incl. ghosts), npfb, nb
    rc, rcs, rl = ref.neighbours()
    gc, gcs, gl = gpu.neighbours()
    np.testing.assert_array_equal(rc, gc)
    np.testing.assert_array_equal(rcs, gcs)
    # jittered nodes have no equal distances, so the distance order is unique
    np.testing.assert_array_equal(rl, gl)


def test_weights(trio):
    name, wl, ns, ref, cr, gpu = trio
    wr, wc, wg = ref.weights(), cr.weights(), gpu.weights()
    # the device SVD and weight evaluation reproduce the restatement bit for bit
    for key in ["w_grad", "w_lap", "w_grad_sum", "w_lap_sum"]:
        nbad = int(np.sum(wg[key] != wc[key]))
        print(name, key, "entries differing from the restatement (device x^4):", nbad)
        assert nbad == 0, key
    # the filter coefficient and node volume go through cos/exp (CUDA vs glibc)
    for key in ["w_hyp", "w_hyp_sum", "vol"]:
        assert rel(wg[key], wc[key]) <= 1e-13, key
    for key in ["w_grad", "w_lap", "w_hyp", "w_grad_sum", "w_lap_sum", "w_hyp_sum", "vol"]:
        check(name, key, wg[key], wr[key], wc[key], W_TOL)


def test_operators(trio):
    name, wl, ns, ref, cr, gpu = trio
    smooth = np.sin(2 * np.pi * ns.x) * np.cos(2 * np.pi * ns.y)
    rng = np.random.default_rng(7)
    noisy = smooth + 0.1 * rng.standard_normal(ns.n)
    for op in ["gradient", "laplacian", "filtered", "filter_term"]:
        for tag, phi in [("smooth", smooth), ("noisy", noisy)]:
            # the filter term of a smooth field is tiny against the terms that cancel in it:
            # measure it against the field
            scale = np.abs(phi).max() if op == "filter_term" else None
            check(name, f"{op}({tag})", getattr(gpu, op)(phi), getattr(ref, op)(phi), getattr(cr, op)(phi), W_TOL,
                  scale)
    assert np.array_equal(gpu.gradient(noisy), cr.gradient(noisy))
    assert np.array_equal(gpu.laplacian(noisy), cr.laplacian(noisy))


def test_rhs(trio):
    name, wl, ns, ref, cr, gpu = trio
    st = initial_state(ns)
    rng = np.random.default_rng(3)
    st["cxx"] = 1.0 + 0.2 * np.sin(2 * np.pi * ns.y) ** 2
    st["cxy"] = 0.1 * np.sin(2 * np.pi * ns.x)
    st["cyy"] = 1.0 + 0.1 * rng.random(ns.n)
    for o in (ref, cr, gpu):
        o.set_state(**st)
    sr, sg = cr.state(), gpu.state()
    for k in ["ro", "rou", "rov", "u", "v", "cxx", "cxy", "cyy"]:
        assert rel(sg[k], sr[k]) <= W_TOL, k
    rr, rc, rg = ref.rhs(), cr.rhs(), gpu.rhs()
    # each right-hand side is a sum of terms that nearly cancel for this state (div u ~ 0);
    # measure the difference against the size of the terms, not of the sum
    gu = np.abs(cr.gradient(st["u"])).max()
    cmax = max(np.abs(st["cxx"]).max(), np.abs(st["cyy"]).max())
    scale = {"ro": gu, "rou": max(gu, np.abs(rc["rou"]).max()), "rov": max(gu, np.abs(rc["rov"]).max()),
             "xx": gu * cmax, "xy": gu * cmax, "yy": gu * cmax}
    for k in ["ro", "rou", "rov", "xx", "xy", "yy"]:
        check(name, "rhs_" + k, rg[k], rr[k], rc[k], W_TOL, scale[k])


def test_steps(trio):
    name, wl, ns, ref, cr, gpu = trio
    st = initial_state(ns)
    for o in (ref, cr, gpu):
        o.set_state(**st)
    dtc, dtp = ref.set_tstep()
    assert gpu.set_tstep() == (dtc, dtp)
    dt = wl.cfl * min(dtc, dtp)
    nsteps = 100
    for o in (ref, cr, gpu):
        o.step(dt, nsteps)
    sr, sc, sg = ref.state(), cr.state(), gpu.state()
    for k in ["ro", "rou", "rov", "u", "v", "cxx", "cxy", "cyy"]:
        check(name, f"{k} after {nsteps} steps", sg[k], sr[k], sc[k], F_TOL)
    tr, tg = cr.time(), gpu.time()
    assert tg["itime"] == tr["itime"] == nsteps
    assert abs(tg["time"] - tr["time"]) <= 1e-12 * abs(tr["time"])
    np.testing.assert_allclose(tg["emax"], tr["emax"], rtol=1e-6)
    assert abs(gpu.kinetic_energy() - cr.kinetic_energy()) <= 1e-10 * cr.kinetic_energy()


def test_pid_steps():
    wl = CASES["di-o4"]
    ns = wl.nodes()
    ref = oracle(wl, ns, True)
    gpu = labfm.for_workload(wl, ns).setup()
    st = initial_state(ns)
    ref.set_state(**st)
    gpu.set_state(**st)
    ref.step(0.0, 20, pid=True)
    gpu.step(0.0, 20, pid=True)
    tr, tg = ref.time(), gpu.time()
    assert abs(tg["dt"] - tr["dt"]) <= 1e-12 * tr["dt"]
    sr, sg = ref.state(), gpu.state()
    for k in ["ro", "u", "v", "cxx", "cxy", "cyy"]:
        assert rel(sg[k], sr[k]) <= F_TOL, k


def test_second_lc_step_special_case():
    """rhs_lc.F90:503 switches Omega off in the first stage of the step with itime == 1
    (the second step).  Starting at itime = 0, 1 and 2 must all match the restatement."""
    wl = CASES["lc-o6"]
    ns = wl.nodes()
    ref = oracle(wl, ns, True)
    gpu = labfm.for_workload(wl, ns).setup()
    st = initial_state(ns)
    st["cxx"] = 1.0 + 0.3 * np.sin(2 * np.pi * ns.y) ** 2
    st["cxy"] = 0.2 * np.sin(2 * np.pi * ns.x)
    for it in (0, 1, 2):
        for o in (ref, gpu):
            o.set_state(**st)
            o.set_time(0.0, 1e-6, it, np.array([1e-5, 1e-5, 1e-5]))
        dtc, dtp = ref.set_tstep()
        dt = wl.cfl * min(dtc, dtp)
        ref.step(dt, 2)
        gpu.step(dt, 2)
        sr, sg = ref.state(), gpu.state()
        for k in ["psixx", "psixy", "psiyy", "u", "v"]:
            assert rel(sg[k], sr[k]) <= 1e-12, (it, k)
