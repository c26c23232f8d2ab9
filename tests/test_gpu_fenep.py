"""FENE-P on the device against the CPU restatement, in all three forms.

Reference behaviour restated (and followed by the device):
* the FENE-P function f = (L^2 - 3) / (L^2 - tr c) and, in the direct and log-conformation
  forms, its gradient in the polymeric stress divergence (rhs_di.F90:198-245,
  rhs_lc.F90:198-245);
* the relaxation terms (f c - I) / lambda (rhs_di.F90:444-449) and c^-1 (f c - I) / lambda
  (rhs_lc.F90:520-535);
* the Cholesky form's factors of J = f c with an evolving psi_zz (rhs.F90:480-541,
  conf_transforms.F90:39-101), the conversions around its filter (rhs.F90:815-869) and its
  scaled error norm (step.F90:442-452);
* with polymer diffusion, the c_zz Laplacian.

Tolerances as for the sPTT parity tests: right-hand sides within 1e-10 of their terms,
fields after 100 steps within 1e-8, the mixed-precision step within 1e-6 of FP64.
"""
import dataclasses

import numpy as np
import pytest

from sunset_viscoelastic_b200 import labfm
from sunset_viscoelastic_b200.nodesets import WORKLOADS, initial_state
import oracle as O

pytestmark = pytest.mark.gpu

W_TOL = 1e-10
F_TOL = 1e-8
L2 = 100.0

BASE = {"di": ("periodic-di-o4-16k", 40), "lc": ("periodic-lc-o6-262k", 40), "chl": ("periodic-chl-o8-1m", 32)}
CASES = [("di", 0.0), ("lc", 0.0), ("chl", 0.0), ("di", 1e-3), ("chl", 1e-3)]


def rel(a, b, scale=None):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    s = max(np.abs(b).max(), 1e-300) if scale is None else scale
    return float(np.abs(a - b).max() / s)


def fenep_state(ns, form):
    """Taylor-Green flow and a smooth positive-definite conformation with tr c well below L^2.
    c_zz varies where it is evolved (direct and Cholesky forms); the 2-D log-conformation form
    has psi_zz = 0, so c_zz = 1 there (mirror nodes carry psi, not c_zz:
    mirror_boundaries.F90:312-343)."""
    st = initial_state(ns)
    x, y = ns.x, ns.y
    st["cxx"] = 1.5 + 0.4 * np.sin(2 * np.pi * y) ** 2
    st["cxy"] = 0.3 * np.sin(2 * np.pi * x) * np.cos(2 * np.pi * y)
    st["cyy"] = 1.2 + 0.2 * np.cos(2 * np.pi * x)
    st["czz"] = np.ones(ns.n) if form == "lc" else 1.1 + 0.1 * np.sin(2 * np.pi * (x + y))
    return st


@pytest.fixture(scope="module", params=CASES, ids=[f"{f}-Mdiff{m:g}" for f, m in CASES])
def pair(request):
    form, mdiff = request.param
    name, nside = BASE[form]
    wl = dataclasses.replace(WORKLOADS[name], nside=nside)
    ns = wl.nodes()
    over = dict(fenep=True, fenep_l2=L2, Mdiff=mdiff)
    O.set_pow_mode(True)
    try:
        ref = O.for_workload(wl, ns, **over).setup()
    finally:
        O.set_pow_mode(False)
    gpu = labfm.for_workload(wl, ns, **over).setup()
    return form, mdiff, wl, ns, ref, gpu


def test_state_and_rhs(pair):
    form, mdiff, wl, ns, ref, gpu = pair
    st = fenep_state(ns, form)
    for o in (ref, gpu):
        o.set_state(**st)
    sr, sg = ref.state(), gpu.state()
    for k in ["ro", "rou", "rov", "u", "v", "psixx", "psixy", "psiyy", "psizz", "cxx", "cxy", "cyy", "czz"]:
        e = rel(sg[k], sr[k], max(np.abs(sr[k]).max(), 1.0))
        assert e <= W_TOL, (k, e)
    rr, rg = ref.rhs(), gpu.rhs()
    gu = np.abs(ref.gradient(st["u"])).max()
    cmax = max(np.abs(st["cxx"]).max(), np.abs(st["cyy"]).max())
    for k in ["ro", "rou", "rov", "xx", "xy", "yy", "zz"]:
        scale = max(gu * cmax, np.abs(rr[k]).max(), 1e-300)
        e = rel(rg[k], rr[k], scale)
        print(f"{form} Mdiff={mdiff:g} rhs_{k}: {e:.2e} (|rhs| {np.abs(rr[k]).max():.3e})")
        assert e <= W_TOL, (k, e)
    # the zz component evolves in the direct form and in the Cholesky form
    if form in ("di", "chl"):
        assert np.abs(rr["zz"]).max() > 0.0


def test_steps(pair):
    form, mdiff, wl, ns, ref, gpu = pair
    st = fenep_state(ns, form)
    for o in (ref, gpu):
        o.set_state(**st)
    dtc, dtp = ref.set_tstep()
    dt = wl.cfl * min(dtc, dtp)
    for o in (ref, gpu):
        o.step(dt, 100)
    sr, sg = ref.state(), gpu.state()
    for k in ["ro", "rou", "rov", "u", "v", "cxx", "cxy", "cyy", "czz"]:
        e = rel(sg[k], sr[k])
        print(f"{form} Mdiff={mdiff:g} {k} after 100 steps: {e:.2e}")
        assert e <= F_TOL, (k, e)
    tr, tg = ref.time(), gpu.time()
    np.testing.assert_allclose(tg["emax"], tr["emax"], rtol=1e-6)


def test_mixed_precision(pair):
    form, mdiff, wl, ns, ref, gpu = pair
    mx = labfm.for_workload(wl, ns, precision="mixed", fenep=True, fenep_l2=L2, Mdiff=mdiff).setup()
    st = fenep_state(ns, form)
    for o in (gpu, mx):
        o.set_state(**st)
    dtc, dtp = gpu.set_tstep()
    dt = wl.cfl * min(dtc, dtp)
    for o in (gpu, mx):
        o.step(dt, 100)
    a, b = mx.state(), gpu.state()
    for grp in (["ro"], ["rou", "rov"], ["cxx", "cxy", "cyy", "czz"]):
        s = max(np.abs(b[k]).max() for k in grp)
        for k in grp:
            e = float(np.abs(a[k] - b[k]).max() / s)
            print(f"{form} Mdiff={mdiff:g} mixed vs FP64 {k}: {e:.2e}")
            assert e <= 1e-6, (k, e)
    mx.close()
