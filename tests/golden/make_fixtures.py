"""Builds tests/golden/ from the reference's own fixtures.

Run with REFERENCE_DIR set to a checkout of the reference (required).  Produces:
  ipart_fixture.npz  -- the reference's IPART node set (4,056 doubly periodic nodes on
                        [-pi,pi]^2, s = 2 pi/64), converted to arrays; together with the
                        parameters of its control.in this is the only fixture the
                        reference ships.
The file is data only; nothing under tests/ reads the reference at run time.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", ".."))
from sunset_viscoelastic_b200.nodesets import read_ipart  # noqa: E402

ref = os.environ.get("REFERENCE_DIR")
if not ref:
    sys.exit("set REFERENCE_DIR to a checkout of the reference (it holds IPART and control.in)")
ns = read_ipart(os.path.join(ref, "IPART"))
# control.in (positional, load_data.F90:53-159)
vals = []
with open(os.path.join(ref, "control.in")) as f:
    for ln in f:
        t = ln.strip()
        if not t or t.startswith("!!"):
            continue
        vals.append([float(v.replace("d", "e").replace("D", "e")) for v in t.split()])
ctrl = dict(L_char=vals[0][0], U_char=vals[1][0], Lz=vals[2][0], t0=vals[3][0], tend=vals[3][1],
            grav=vals[5], Re=vals[6][0], Wi=vals[7][0], beta=vals[8][0], epsPTT=vals[9][0],
            fenep_l2=vals[10][0], Mdiff=vals[11][0], Ma=vals[12][0])
np.savez_compressed(os.path.join(HERE, "ipart_fixture.npz"), gi=ns.gi, x=ns.x, y=ns.y, node_type=ns.node_type,
                    nx=ns.nx, ny=ns.ny, s=ns.s, box=np.array([ns.xmin, ns.xmax, ns.ymin, ns.ymax]),
                    bcond=np.array(ns.bcond, np.int32),
                    control=np.array([ctrl[k] for k in ["L_char", "U_char", "Re", "Wi", "beta", "epsPTT",
                                                        "fenep_l2", "Mdiff", "Ma"]]))
print("wrote ipart_fixture.npz:", ns.n, "nodes", ctrl)
