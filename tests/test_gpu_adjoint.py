"""The adjoint of the time step on the device (sunset_adjoint_run, sunset_adjoint_apply_D).

* Transposed operators: <D phi, psi> = <phi, D^T psi> for d/dx, d/dy, the Laplacian and the
  filter term (dot-product test, 1e-12 relative).
* The full adjoint (log-conformation Oldroyd-B, Wi = 1, beta = 0.5 as in the differentiation
  configuration; J = sum 1/2 rho |u|^2 vol after the run) against central finite differences
  (h = 1e-6 relative) of the device's forward solver and of the CPU restatement, for dJ/dWi,
  dJ/dbeta and the directional derivatives of J along seeded Gaussian perturbations of the
  initial log-conformation field: 1e-5 relative.  The initial psi is non-degenerate (at
  c = I the eigenvalue branch of rhs_lc.F90:465-469 is degenerate and J is not
  differentiable in psi in the usual sense).
* A torch.autograd.Function around the adjoint (test harness only).
"""
import dataclasses

import numpy as np
import pytest

from sunset_viscoelastic_b200 import labfm
from sunset_viscoelastic_b200.nodesets import WORKLOADS
import oracle as O

pytestmark = pytest.mark.gpu

WL = dataclasses.replace(WORKLOADS["periodic-lc-o6-262k"], nside=32, epsPTT=0.0, Wi=1.0, beta=0.5)
NSTEPS, CKPT = 24, 5
FD_TOL = 1e-5


def initial_fields(ns):
    """Taylor-Green velocity, rho = 1, and a non-degenerate smooth log-conformation field."""
    x, y = ns.x, ns.y
    n = ns.n
    return dict(ro=np.ones(n), rou=np.sin(2 * np.pi * x) * np.cos(2 * np.pi * y),
                rov=-np.cos(2 * np.pi * x) * np.sin(2 * np.pi * y),
                psixx=0.2 + 0.1 * np.sin(2 * np.pi * x), psixy=0.1 * np.cos(2 * np.pi * y),
                psiyy=-0.1 + 0.05 * np.sin(2 * np.pi * (x + y)), psizz=np.zeros(n))


KEYS = ["ro", "rou", "rov", "psixx", "psixy", "psiyy", "psizz"]


def make(ns, **over):
    g = labfm.for_workload(WL, ns, **over).setup()
    return g


def set_conservative(g, st):
    """Reset time and itime (sunset_set_state), then load the conservative state as given."""
    n = len(st["ro"])
    one, z = np.ones(n), np.zeros(n)
    g.set_state(ro=one, u=z, v=z, cxx=one, cxy=z, cyy=one)
    import torch
    buf = torch.from_numpy(np.concatenate([st[k] for k in KEYS])).pin_memory()
    out = torch.empty_like(buf).pin_memory()
    g.run_host(buf.data_ptr(), 1e-9, 0, out.data_ptr())


def forward_J(ns, st, dt, **over):
    g = make(ns, **over)
    set_conservative(g, st)
    g.step(dt, NSTEPS)
    return g.kinetic_energy()


def oracle_J(ns, st, dt, **over):
    kw = dict(WL.params())
    kw.update(over)
    o = O.Oracle(**kw).build_domain(ns).setup()
    n = ns.n
    o.set_state(ro=np.ones(n), u=np.zeros(n), v=np.zeros(n), cxx=np.ones(n), cxy=np.zeros(n), cyy=np.ones(n))
    o.set_raw_state(st["ro"], st["rou"], st["rov"], np.concatenate([st[k] for k in KEYS[3:]]))
    o.step(dt, NSTEPS)
    return o.kinetic_energy()


@pytest.fixture(scope="module")
def setup():
    ns = WL.nodes()
    st = initial_fields(ns)
    g = make(ns)
    set_conservative(g, st)
    dtc, dtp = g.set_tstep()
    dt = WL.cfl * min(dtc, dtp)
    J, (dWi, dbeta), grads = g.adjoint_run(dt, NSTEPS, CKPT)
    return ns, st, dt, g, J, dWi, dbeta, grads


def test_transposed_operators_dot_product():
    ns = WL.nodes()
    g = make(ns)
    rng = np.random.default_rng(5)
    phi, psi = rng.standard_normal(ns.n), rng.standard_normal(ns.n)
    ops = [lambda f: g.gradient(f)[:, 0], lambda f: g.gradient(f)[:, 1], g.laplacian, g.filter_term]
    for which, D in enumerate(ops):
        lhs = float(D(phi) @ psi)
        rhs = float(phi @ g.adjoint_apply_D(which, psi))
        print("which", which, "<D phi, psi>", lhs, "<phi, D^T psi>", rhs)
        assert abs(lhs - rhs) <= 1e-12 * max(abs(lhs), np.abs(D(phi)).max() * np.abs(psi).sum()), which


def test_adjoint_J_matches_forward(setup):
    ns, st, dt, g, J, dWi, dbeta, grads = setup
    assert abs(J - forward_J(ns, st, dt)) <= 1e-13 * J


@pytest.mark.parametrize("param", ["Wi", "beta"])
def test_parameter_gradients_against_finite_differences(setup, param):
    ns, st, dt, g, J, dWi, dbeta, grads = setup
    p0 = getattr(WL, param)
    h = 1e-6 * p0
    fd = (forward_J(ns, st, dt, **{param: p0 + h}) - forward_J(ns, st, dt, **{param: p0 - h})) / (2 * h)
    fd_ref = (oracle_J(ns, st, dt, **{param: p0 + h}) - oracle_J(ns, st, dt, **{param: p0 - h})) / (2 * h)
    ad = dWi if param == "Wi" else dbeta
    print(f"dJ/d{param}: adjoint {ad:.12e}  FD device {fd:.12e}  FD restatement {fd_ref:.12e}")
    assert abs(ad - fd) <= FD_TOL * abs(fd)
    assert abs(ad - fd_ref) <= FD_TOL * abs(fd_ref)


def test_initial_psi_gradient_along_gaussian_directions(setup):
    ns, st, dt, g, J, dWi, dbeta, grads = setup
    rng = np.random.default_rng(2024)
    for r in range(4):
        d = {k: rng.standard_normal(ns.n) for k in ("psixx", "psixy", "psiyy")}
        ad = sum(float(grads[k] @ d[k]) for k in d)
        h = 1e-6
        sp = dict(st); sm = dict(st)
        for k in d:
            sp[k] = st[k] + h * d[k]
            sm[k] = st[k] - h * d[k]
        fd = (forward_J(ns, sp, dt) - forward_J(ns, sm, dt)) / (2 * h)
        print(f"direction {r}: adjoint {ad:.12e}  FD {fd:.12e}")
        assert abs(ad - fd) <= FD_TOL * abs(fd)


def test_state_gradient_of_momentum(setup):
    ns, st, dt, g, J, dWi, dbeta, grads = setup
    rng = np.random.default_rng(7)
    d = {k: rng.standard_normal(ns.n) for k in ("ro", "rou", "rov")}
    ad = sum(float(grads[k] @ d[k]) for k in d)
    h = 1e-7
    sp = dict(st); sm = dict(st)
    for k in d:
        sp[k] = st[k] + h * d[k]
        sm[k] = st[k] - h * d[k]
    fd = (forward_J(ns, sp, dt) - forward_J(ns, sm, dt)) / (2 * h)
    print(f"rho / momentum direction: adjoint {ad:.12e}  FD {fd:.12e}")
    assert abs(ad - fd) <= FD_TOL * abs(fd)


def test_torch_autograd_function(setup):
    import torch
    ns, st, dt, g, J0, dWi0, dbeta0, grads0 = setup

    class KineticEnergyAfterSteps(torch.autograd.Function):
        """J(psi0) through the device solver; backward from sunset_adjoint_run."""

        @staticmethod
        def forward(ctx, psi0):
            s = dict(st)
            for c, k in enumerate(("psixx", "psixy", "psiyy")):
                s[k] = psi0[c].detach().cpu().numpy().astype(np.float64)
            h = make(ns)
            set_conservative(h, s)
            J, _, grads = h.adjoint_run(dt, NSTEPS, CKPT)
            ctx.save_for_backward(torch.from_numpy(np.stack([grads[k] for k in ("psixx", "psixy", "psiyy")])))
            return psi0.new_tensor(J)

        @staticmethod
        def backward(ctx, gout):
            (gpsi,) = ctx.saved_tensors
            return gout * gpsi

    psi0 = torch.tensor(np.stack([st["psixx"], st["psixy"], st["psiyy"]]), dtype=torch.float64, requires_grad=True)
    J = KineticEnergyAfterSteps.apply(psi0)
    J.backward()
    assert abs(J.item() - J0) <= 1e-13 * J0
    np.testing.assert_allclose(psi0.grad.numpy()[0], grads0["psixx"], rtol=0, atol=1e-15 * np.abs(grads0["psixx"]).max())
