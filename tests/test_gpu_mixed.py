"""Mixed precision (SUNSET_MIXED) against the FP64 restatement and the FP64 device path.

The mixed stage streams each weight as a 26-bit fixed-point number scaled per node and
operator (rounding 2^-25 of the node's largest weight), stages the tile's neighbour values
as FP32 offsets from a per-tile FP64 reference, sums the stencils in FP32 difference form
sum_k w_k (phi_j - phi_i), and keeps the RK register as an FP32 increment over the stage's
FP64 state; the state, the pointwise right-hand sides, transforms and reductions stay FP64.
The stated tolerance is 1e-6 relative per field after 100 steps,
with the error of field f measured against the magnitude of the quantity it is a component
of (rho; the momentum or velocity vector; the conformation tensor):

    L_inf = max_i |f_mixed - f_ref| / max_{g in group(f)} max_i |g_ref|,
    L_2   = ||f_mixed - f_ref||_2 / max_{g in group(f)} ||g_ref||_2.

A component that vanishes identically in the exact solution (c_xy of a Taylor-Green flow,
whose shear rate u_y + v_x is zero) has no magnitude of its own to compare with.  For rho
and the diagonal of c, whose values sit near 1, the error is also printed relative to the
deviation from the rest state (f - 1), which is the stricter measure.
"""
import dataclasses

import numpy as np
import pytest

from sunset_viscoelastic_b200 import labfm
from sunset_viscoelastic_b200.nodesets import WORKLOADS, initial_state
import oracle as O

pytestmark = pytest.mark.gpu

M_TOL = 1e-6
FIELDS = ["ro", "rou", "rov", "u", "v", "cxx", "cxy", "cyy"]
GROUP = {"ro": ["ro"], "rou": ["rou", "rov"], "rov": ["rou", "rov"], "u": ["u", "v"], "v": ["u", "v"],
         "cxx": ["cxx", "cxy", "cyy"], "cxy": ["cxx", "cxy", "cyy"], "cyy": ["cxx", "cxy", "cyy"]}
NEAR_ONE = {"ro", "cxx", "cyy"}


def small(wl_name, nside, **over):
    return dataclasses.replace(WORKLOADS[wl_name], nside=nside, **over)


CASES = {
    "di-o4": small("periodic-di-o4-16k", 48),
    "lc-o6": small("periodic-lc-o6-262k", 40),
    "chl-o8": small("periodic-chl-o8-1m", 32),
}


def errors(sa, sb, k):
    """(L_inf, L_2, L_inf against the deviation from 1 or None) of field k, states sa vs sb."""
    a = np.asarray(sa[k], np.float64)
    b = np.asarray(sb[k], np.float64)
    d = a - b
    s_inf = max(np.abs(sb[g]).max() for g in GROUP[k])
    s_2 = max(np.linalg.norm(sb[g]) for g in GROUP[k])
    dev = np.abs(d).max() / max(np.abs(b - 1.0).max(), 1e-300) if k in NEAR_ONE else None
    return np.abs(d).max() / max(s_inf, 1e-300), np.linalg.norm(d) / max(s_2, 1e-300), dev


@pytest.fixture(scope="module", params=list(CASES))
def runs(request):
    """(name, workload, nodes, restatement, FP64 device, mixed device) after 100 steps."""
    wl = CASES[request.param]
    ns = wl.nodes()
    O.set_pow_mode(True)
    try:
        ref = O.for_workload(wl, ns).setup()
    finally:
        O.set_pow_mode(False)
    f64 = labfm.for_workload(wl, ns).setup()
    mx = labfm.for_workload(wl, ns, precision="mixed").setup()
    st = initial_state(ns)
    for o in (ref, f64, mx):
        o.set_state(**st)
    dtc, dtp = ref.set_tstep()
    assert mx.set_tstep() == (dtc, dtp)
    dt = wl.cfl * min(dtc, dtp)
    for o in (ref, f64, mx):
        o.step(dt, 100)
    return request.param, wl, ns, ref, f64, mx


def test_fields_after_100_steps(runs):
    name, wl, ns, ref, f64, mx = runs
    sr, s64, smx = ref.state(), f64.state(), mx.state()
    worst = 0.0
    for k in FIELDS:
        linf, l2, dev = errors(smx, sr, k)
        linf64, _, _ = errors(s64, sr, k)
        extra = f"  (vs deviation from 1: {dev:.2e})" if dev is not None else ""
        print(f"{name} {k}: mixed vs FP64 restatement L_inf {linf:.2e} L_2 {l2:.2e}{extra}; "
              f"FP64 device {linf64:.2e}")
        assert linf <= M_TOL and l2 <= M_TOL, (k, linf, l2)
        worst = max(worst, linf)
    # the mixed step really ran on the rounded weights: it is not the FP64 result
    assert max(np.abs(smx[k] - s64[k]).max() for k in FIELDS) > 0.0
    assert mx.time()["itime"] == 100
    assert abs(mx.kinetic_energy() - ref.kinetic_energy()) <= M_TOL * ref.kinetic_energy()


def test_rhs(runs):
    """calc_all_rhs of the mixed handle uses the mixed stencils: within 1e-4 of the size of
    the FP64 right-hand side's terms.  The viscous term dominates the difference: the FP32
    offsets of the neighbour values round at 2^-24 of their spread over a tile, which the
    Laplacian's O(1/s^2) weights amplify; the field tolerance after 100 steps is the gate."""
    name, wl, ns, ref, f64, mx = runs
    st = initial_state(ns)
    st["cxx"] = 1.0 + 0.3 * np.sin(2 * np.pi * ns.y) ** 2
    st["cxy"] = 0.2 * np.sin(2 * np.pi * ns.x)
    for o in (f64, mx):
        o.set_state(**st)
    r64, rmx = f64.rhs(), mx.rhs()
    # the terms of each right-hand side nearly cancel for this state (div u ~ 0): measure the
    # difference against the size of the terms, not of their sum
    gu = np.abs(f64.gradient(st["u"])).max()
    cmax = max(np.abs(st["cxx"]).max(), np.abs(st["cyy"]).max())
    scale = {"ro": gu, "rou": max(gu, np.abs(r64["rou"]).max()), "rov": max(gu, np.abs(r64["rov"]).max()),
             "xx": gu * cmax, "xy": gu * cmax, "yy": gu * cmax}
    for k in ["ro", "rou", "rov", "xx", "xy", "yy"]:
        e = np.abs(rmx[k] - r64[k]).max() / scale[k]
        print(f"{name} rhs_{k}: mixed vs FP64 {e:.2e} (of the terms' size)")
        assert e <= 1e-4, (k, e)


def test_mixed_pid_steps():
    wl = CASES["di-o4"]
    ns = wl.nodes()
    f64 = labfm.for_workload(wl, ns).setup()
    mx = labfm.for_workload(wl, ns, precision="mixed").setup()
    st = initial_state(ns)
    for o in (f64, mx):
        o.set_state(**st)
        o.step(0.0, 20, pid=True)
    t64, tmx = f64.time(), mx.time()
    assert tmx["itime"] == 20
    assert abs(tmx["dt"] - t64["dt"]) <= 1e-6 * t64["dt"]
    s64, smx = f64.state(), mx.state()
    for k in ["ro", "u", "v", "cxx", "cxy", "cyy"]:
        assert errors(smx, s64, k)[0] <= M_TOL, k


def test_operators_unchanged_by_mixed():
    """The single-operator entry points of a mixed handle keep the FP64 weights."""
    wl = CASES["lc-o6"]
    ns = wl.nodes()
    f64 = labfm.for_workload(wl, ns).setup()
    mx = labfm.for_workload(wl, ns, precision="mixed").setup()
    phi = np.sin(2 * np.pi * ns.x) * np.cos(4 * np.pi * ns.y)
    np.testing.assert_array_equal(mx.gradient(phi), f64.gradient(phi))
    np.testing.assert_array_equal(mx.laplacian(phi), f64.laplacian(phi))
