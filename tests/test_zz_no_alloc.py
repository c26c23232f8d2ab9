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


def test_kinetic_energy_noalloc_many_blocks():
    """Above 65,536 nodes the fold kernel's threads each add several partial pairs: a
    262,144-node state against the handle reduction, and the largest accepted size
    (256 x 16384 nodes) on synthetic arrays against a float64 sum on the device."""
    import torch
    wl = dataclasses.replace(WORKLOADS["periodic-di-o4-16k"], nside=512)
    ns = wl.nodes()
    g = labfm.for_workload(wl, ns).setup()
    st = initial_state(ns)
    st["ro"] = 1.0 + 0.05 * np.sin(2 * np.pi * ns.x)
    g.set_state(**st)
    ke_ref, mass_ref = g.kinetic_energy(), g.mass()
    s = g.state()
    dev = torch.device("cuda", 0)
    ro, u, v, vo = (torch.tensor(a, dtype=torch.float64, device=dev)
                    for a in (s["ro"], s["u"], s["v"], g.weights()["vol"]))
    g.close()
    out = torch.full((2,), float("nan"), dtype=torch.float64, device=dev)
    for _ in range(2):
        labfm.kinetic_energy_noalloc(0, ns.n, ro.data_ptr(), u.data_ptr(), v.data_ptr(), vo.data_ptr(),
                                     out.data_ptr(), torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        ke, mass = out.cpu().numpy()
        assert abs(ke - ke_ref) <= TOL * abs(ke_ref)
        assert abs(mass - mass_ref) <= TOL * abs(mass_ref)
    n = 256 * 16384
    gen = torch.Generator(device=dev).manual_seed(3)
    ro = 1.0 + 0.1 * torch.rand(n, dtype=torch.float64, device=dev, generator=gen)
    u = torch.randn(n, dtype=torch.float64, device=dev, generator=gen)
    v = torch.randn(n, dtype=torch.float64, device=dev, generator=gen)
    vo = torch.rand(n, dtype=torch.float64, device=dev, generator=gen) / n
    labfm.kinetic_energy_noalloc(0, n, ro.data_ptr(), u.data_ptr(), v.data_ptr(), vo.data_ptr(), out.data_ptr(),
                                 torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    ke, mass = out.cpu().numpy()
    ke_t = float(((0.5 * ro) * (u * u + v * v) * vo).sum())
    mass_t = float((ro * vo).sum())
    assert abs(ke - ke_t) <= TOL * abs(ke_t)
    assert abs(mass - mass_t) <= TOL * abs(mass_t)


def test_kinetic_energy_noalloc_leaves_caller_state_alone():
    """The call neither consumes nor reports an error the caller left pending in the CUDA
    runtime, and leaves the calling thread's current device as it was."""
    import ctypes
    import torch
    lib = labfm.load_library()
    rt = ctypes.CDLL("libcudart.so.12")  # the runtime the library is linked against, already loaded
    dev = torch.device("cuda", 0)
    ro = torch.ones(1000, dtype=torch.float64, device=dev)
    out = torch.zeros(2, dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    cur = ctypes.c_int(-1)
    assert rt.cudaGetDevice(ctypes.byref(cur)) == 0
    assert rt.cudaSetDevice(1 << 20) != 0       # a pending, non-sticky error (invalid device)
    rc = lib.sunset_kinetic_energy_noalloc(0, 1000, ro.data_ptr(), ro.data_ptr(), ro.data_ptr(), ro.data_ptr(),
                                           out.data_ptr(), None)
    assert rc == 0
    assert rt.cudaGetLastError() != 0           # still pending for the caller
    assert rt.cudaGetLastError() == 0
    after = ctypes.c_int(-1)
    assert rt.cudaGetDevice(ctypes.byref(after)) == 0 and after.value == cur.value
    rt.cudaDeviceSynchronize()
    assert abs(out.cpu().numpy()[1] - 1000.0) < 1e-9


def test_kinetic_energy_noalloc_rejects_oversize():
    lib = labfm.load_library()
    rc = lib.sunset_kinetic_energy_noalloc(0, 256 * 16384 + 1, 1, 1, 1, 1, 1, None)
    assert rc == -4
