"""Output, restart and checkpoints of a 3-D run on the device.

Reference behaviour restated (and followed by the device):
* output_layer in 3-D with -Dallout (output.F90:184-310): 13 columns for every node-layer,
  layer-major -- rho - rho_char, u, v, w, the vorticity magnitude of the 3-D velocity gradient
  (on walls from the gradients in the wall's frame, :226-235), Q (which the reference never
  sets in 3-D; written as 0), alpha_out (the node-layer's step error, step.F90:456-458) and the
  six c components; output_nodes with z and the layer offset of the global index
  (setup_domain.F90:520-535); time.out with dims 3;
* load_restart_file in 3-D (setup_flow.F90:505-509): rho from rho - rho_char, u, v, w and c,
  the header's flow-control and error history;
* a device checkpoint (binary, between steps) resumes bit for bit.

The dump columns are compared with the restatement's (or3_get_dump) after 20 steps: state
columns and vorticity within 1e-10, alpha_out within 1e-6 (it is the step's error estimate,
like emax).  A restart from the written files on a new handle, and the restatement restarted
from the same columns, agree after 10 more steps within 1e-8.
"""
import dataclasses

import numpy as np
import pytest

from sunset_viscoelastic_b200 import dumpfiles as D
from sunset_viscoelastic_b200 import labfm
from sunset_viscoelastic_b200.nodesets import WORKLOADS, channel, poiseuille_state
import oracle as O

pytestmark = pytest.mark.gpu

G = 8.0


def build(kind):
    if kind == "periodic":
        wl = dataclasses.replace(WORKLOADS["periodic-di-o4-16k"], nside=24)
        ns, kw, Lz = wl.nodes(), dict(wl.params(), kolmogorov_forcing=0), 1.0
    else:
        ns = channel(24)
        kw = dict(form="chl", order=6, Re=1.0, Wi=0.5, beta=0.59, Ma=0.1, grav=(G, 0.0, 0.0), kolmogorov_forcing=0,
                  epsPTT=0.25, Mdiff=1e-3)
        Lz = 0.4
    O.set_pow_mode(True)
    try:
        layer = O.Oracle(**kw).build_domain(ns).setup()
    finally:
        O.set_pow_mode(False)
    ref = O.Oracle3(layer, Lz)
    return ns, kw, Lz, layer, ref


def make_gpu(ns, kw, Lz):
    g = labfm.Sunset(**kw)
    g.build_domain(ns)
    g.set_layers(Lz)
    g.setup()
    return g


def state(layer, ref, kind):
    nd = layer.nodes()
    nl, nz, dz = ref.nl, ref.nz, ref.dz
    x, y = np.tile(nd["x"][:nl], nz), np.tile(nd["y"][:nl], nz)
    kz = 2.0 * np.pi * np.repeat(np.arange(nz) * dz, nl) / (nz * dz)
    tp = 2.0 * np.pi
    if kind == "periodic":
        st = dict(ro=1.0 + 0.01 * np.cos(tp * x) * np.cos(kz), u=np.sin(tp * x) * np.cos(tp * y) * np.cos(kz),
                  v=-np.cos(tp * x) * np.sin(tp * y) * np.cos(kz), w=0.1 * np.sin(kz) * np.cos(tp * x),
                  cxx=1.2 + 0.1 * np.sin(kz), cxy=0.05 * np.sin(tp * x) * np.sin(tp * y), cyy=1.1 + 0.05 * np.cos(tp * y))
    else:
        st = poiseuille_state(type("P", (), {"y": y, "n": len(y)}), G, 1.0, 0.5)
        yy = y * (1.0 - y)
        st["u"] = st["u"] + 0.3 * np.sin(tp * x) * yy * np.cos(kz)
        st["v"] = 0.2 * np.cos(tp * x) * yy
        st["w"] = 0.1 * yy * np.sin(kz)
        st["ro"] = 1.0 + 0.01 * np.sin(tp * x) * np.cos(np.pi * y) * np.cos(kz)
    st.setdefault("czz", 1.05 + 0.02 * np.cos(kz))
    st["cxz"] = 0.03 * np.cos(kz) * np.cos(tp * x)
    st["cyz"] = 0.02 * np.sin(kz) * np.sin(tp * x)
    return st


def set_both(ref, gpu, st):
    c = {k: st[k] for k in ["cxx", "cxy", "cyy", "cxz", "cyz", "czz"]}
    ref.set_state(st["ro"], st["u"], st["v"], st["w"], **c)
    gpu.set_state_3d(st["ro"], st["u"], st["v"], st["w"], **c)


@pytest.mark.parametrize("kind", ["periodic", "walls"])
def test_dump_restart_and_checkpoint(kind, tmp_path):
    ns, kw, Lz, layer, ref = build(kind)
    g = make_gpu(ns, kw, Lz)
    st = state(layer, ref, kind)
    set_both(ref, g, st)
    dc, dp = ref.set_tstep()
    dt = 0.3 * min(dc, dp)
    for o in (ref, g):
        o.step(dt, 20)
    # the dump columns against the restatement's
    cg, hg = g.dump()
    cr, hr = ref.dump()
    assert list(cg) == D.FIELD_COLUMNS_3D
    for k in cr:
        scale = max(np.abs(cr[k]).max(), 1.0)
        tol = 1e-6 if k == "alpha" else 1e-10
        e = float(np.abs(cg[k] - cr[k]).max() / scale)
        print(f"{kind} dump {k}: {e:.2e} (max |{k}| {np.abs(cr[k]).max():.3e})")
        assert e <= tol, (k, e)
    assert np.abs(cr["vort"]).max() > 0 and np.abs(cr["alpha"]).max() > 0 and np.all(cg["qcrit"] == 0.0)
    np.testing.assert_allclose(hg[5:8], hr[5:8], rtol=1e-6)
    assert hg[8] == hr[8]
    # the files: fields, nodes and time.out
    g.write_dump(tmp_path, 1, g.time()["time"])
    hd, cols = D.read_fields(tmp_path / "fields_10000_1")
    nd = D.read_nodes(tmp_path / "nodes_10000")
    for k in cols:
        assert np.array_equal(cols[k], cg[k]), k
    nz, dz = g.layers()
    nl = ref.nl
    assert len(nd["x"]) == nl * nz and np.array_equal(nd["z"], np.repeat(np.arange(nz) * dz, nl))
    assert nd["gi"].tolist() == list(range(1, nl * nz + 1))
    t = open(tmp_path / "time.out").read().split()
    assert t[1] == "3" and int(t[2]) == nl * nz
    # restart from the files on a new handle; the restatement restarted from the same columns
    r = make_gpu(ns, kw, Lz)
    r.set_restart(cols, hd)
    tg = g.time()
    r.set_time(tg["time"], tg["dt"], tg["itime"], tg["emax"])
    ro = cols["ro_minus_rho_char"] + 1.0
    ref.set_state(ro, cols["u"], cols["v"], cols["w"], **{k: cols[k] for k in ["cxx", "cxy", "cyy", "cxz", "cyz", "czz"]})
    a, b = g.state_3d(), r.state_3d()
    for k in ["ro", "u", "v", "w"]:
        assert np.array_equal(a[k], b[k]), k
    for o in (ref, r):
        o.step(dt, 10)
    sr, sg = ref.state(), r.state_3d()
    for k in ["ro", "rou", "rov", "row", "cxx", "cxz", "czz"]:
        e = float(np.abs(sg[k] - sr[k]).max() / max(np.abs(sr[k]).max(), 1e-300))
        assert e <= 1e-8, (k, e)
    # a device checkpoint resumes bit for bit
    ck = g.save_checkpoint()
    g.step(dt, 5)
    a = g.state_3d()
    c = make_gpu(ns, kw, Lz)
    c.load_checkpoint(ck)
    c.step(dt, 5)
    b = c.state_3d()
    for k in a:
        assert np.array_equal(a[k], b[k]), k
    assert c.time()["itime"] == g.time()["itime"]
    with pytest.raises(labfm.SunsetError):  # another layering
        d = labfm.Sunset(**kw)
        d.build_domain(ns)
        d.set_layers(2.0 * Lz)
        d.setup()
        d.load_checkpoint(ck)
    for o in (g, r, c):
        o.close()
