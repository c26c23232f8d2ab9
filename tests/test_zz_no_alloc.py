"""The allocation-free kinetic-energy/mass entry point, through the C-ABI.

It serves callers that cannot allocate device memory: they pass device arrays they
already own and receive the sums in a device array they own; the entry point's partial
sums live in a static device array.  Its results must agree with the handle-based
sunset_kinetic_energy / sunset_mass on the same state, on two calls in a row (the second
call reuses the static array the first one left behind).  This file is collected last so
that a failure here leaves every other test already run.
"""
import dataclasses

import numpy as np
import pytest

from sunset_viscoelastic_b200 import labfm
from sunset_viscoelastic_b200.nodesets import WORKLOADS, initial_state

pytestmark = pytest.mark.gpu

TOL = 1e-12  # the two reductions sum in different orders


def test_kinetic_energy_noalloc_matches_handle_reduction():
    import torch
    wl = dataclasses.replace(WORKLOADS["periodic-lc-o6-262k"], nside=64)
    ns = wl.nodes()
    g = labfm.for_workload(wl, ns).setup()
    st = initial_state(ns)
    st["ro"] = 1.0 + 0.05 * np.cos(2 * np.pi * ns.y)
    g.set_state(**st)
    dtc, dtp = g.set_tstep()
    g.step(wl.cfl * min(dtc, dtp), 3)
    ke_ref, mass_ref = g.kinetic_energy(), g.mass()
    s = g.state()
    vol = g.weights()["vol"]
    dev = torch.device("cuda", 0)
    ro, u, v, vo = (torch.tensor(a, dtype=torch.float64, device=dev) for a in (s["ro"], s["u"], s["v"], vol))
    results = []
    for _ in range(2):
        out = torch.full((2,), float("nan"), dtype=torch.float64, device=dev)
        labfm.kinetic_energy_noalloc(0, ns.n, ro.data_ptr(), u.data_ptr(), v.data_ptr(), vo.data_ptr(),
                                     out.data_ptr(), torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        results.append(out.cpu().numpy())
    for ke, mass in results:
        assert abs(ke - ke_ref) <= TOL * abs(ke_ref)
        assert abs(mass - mass_ref) <= TOL * abs(mass_ref)
    assert np.array_equal(results[0], results[1])
    g.close()


def test_kinetic_energy_noalloc_rejects_oversize():
    lib = labfm.load_library()
    rc = lib.sunset_kinetic_energy_noalloc(0, 256 * 16384 + 1, 1, 1, 1, 1, 1, None)
    assert rc == -4
