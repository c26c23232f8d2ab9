"""The hand-written reverse of the pointwise right-hand side (csrc/adjoint.cuh), built for the
host (libsunset_hostcheck.so), against central finite differences of the forward map.

For random nodes (state, stencil sums, parameters; the log-conformation first-step case
included) and random directions d, the adjoint's r_bar . (dP d) must match
r_bar . (P(x + e d) - P(x - e d)) / 2e with e = 1e-6, to 1e-6 of the larger of the derivative
and 1e-2 |r_bar| |P| (the size of the terms it is made of: a small derivative loses digits
to the finite difference's rounding, not to the adjoint).
"""
import ctypes as C
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "..", "sunset_viscoelastic_b200", "lib", "libsunset_hostcheck.so")


@pytest.fixture(scope="module")
def hc():
    if not os.path.exists(LIB):
        from sunset_viscoelastic_b200 import build
        build.build()
    L = C.CDLL(LIB)
    dp = np.ctypeslib.ndpointer(np.float64, flags="C")
    L.sunset_hostcheck_lc.argtypes = [dp, dp, dp, C.c_int, C.c_void_p, dp, dp, dp, dp]
    L.sunset_hostcheck_lc_c.argtypes = [dp, C.c_void_p, dp, dp]
    return L


def forward(L, par, s, g, first):
    r = np.zeros(6)
    L.sunset_hostcheck_lc(par, s, g, first, None, r, np.zeros(6), np.zeros(18), np.zeros(2))
    return r


@pytest.mark.parametrize("seed", range(6))
def test_pointwise_lc_adjoint_matches_finite_differences(hc, seed):
    rng = np.random.default_rng(seed)
    eps = 1e-6
    errs = []
    for trial in range(25):
        par = np.array([1.0, 0.5 + rng.random(), 0.2 + 0.6 * rng.random(), 0.25 * rng.random(), 0.1])
        s = np.concatenate([[1.0 + 0.05 * rng.standard_normal()], rng.standard_normal(2), 0.3 * rng.standard_normal(3)])
        g = rng.standard_normal(18)
        first = int(trial % 5 == 0)
        rb = rng.standard_normal(6)
        r, sb, gb, tb = np.zeros(6), np.zeros(6), np.zeros(18), np.zeros(2)
        hc.sunset_hostcheck_lc(par, s, g, first, rb.ctypes.data, r, sb, gb, tb)
        ds, dg = rng.standard_normal(6), rng.standard_normal(18)
        fd = rb @ (forward(hc, par, s + eps * ds, g + eps * dg, first)
                   - forward(hc, par, s - eps * ds, g - eps * dg, first)) / (2 * eps)
        scale = 1e-2 * np.linalg.norm(rb) * np.linalg.norm(r)
        errs.append(abs(fd - (sb @ ds + gb @ dg)) / max(abs(fd), scale))
        for k, pi in ((0, 1), (1, 2)):  # Wi, beta
            dpar = np.zeros(5)
            dpar[pi] = 1.0
            fdp = rb @ (forward(hc, par + eps * dpar, s, g, first) - forward(hc, par - eps * dpar, s, g, first)) / (2 * eps)
            errs.append(abs(fdp - tb[k]) / max(abs(fdp), scale))
    print("worst relative difference", max(errs), "median", float(np.median(errs)))
    assert max(errs) < 1e-6


def test_c_from_psi_adjoint(hc):
    rng = np.random.default_rng(11)
    eps = 1e-6
    for _ in range(50):
        psi = 0.5 * rng.standard_normal(3)
        cb = rng.standard_normal(3)
        c, pb = np.zeros(3), np.zeros(3)
        hc.sunset_hostcheck_lc_c(psi, cb.ctypes.data, c, pb)
        d = rng.standard_normal(3)
        cp, cm = np.zeros(3), np.zeros(3)
        hc.sunset_hostcheck_lc_c(psi + eps * d, None, cp, np.zeros(3))
        hc.sunset_hostcheck_lc_c(psi - eps * d, None, cm, np.zeros(3))
        fd = cb @ (cp - cm) / (2 * eps)
        assert abs(fd - pb @ d) <= 1e-7 * max(1.0, abs(fd)), (fd, pb @ d)
