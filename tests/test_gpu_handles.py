"""Distinct handles are independent: two handles of different configurations (log-conformation
at order 6 and the direct form at order 4, different Wi and epsPTT), stepped at the same time
from two host threads, end bit for bit where each ends when stepped alone.  The library's
calls release the interpreter lock (ctypes), so the two threads' launches interleave on the
device; each kernel takes its run's constants as a launch parameter.
"""
import dataclasses
import threading

import numpy as np
import pytest

from sunset_viscoelastic_b200 import labfm
from sunset_viscoelastic_b200.nodesets import WORKLOADS, initial_state

pytestmark = pytest.mark.gpu


def make(name, **over):
    wl = dataclasses.replace(WORKLOADS[name], nside=48)
    ns = wl.nodes()
    g = labfm.for_workload(wl, ns, **over).setup()
    st = initial_state(ns)
    return g, wl, st


def run(g, st, dt, n, out, key):
    g.set_state(**st)
    for _ in range(n):
        g.step(dt, 5)
    out[key] = g.state()


def test_two_configurations_from_two_threads():
    a, wa, sa = make("periodic-lc-o6-262k", Wi=1.0, epsPTT=0.25)
    b, wb, sb = make("periodic-di-o4-16k", Wi=0.5, epsPTT=0.1)
    for g, st in ((a, sa), (b, sb)):
        g.set_state(**st)
    dta = 0.3 * min(a.set_tstep())
    dtb = 0.3 * min(b.set_tstep())
    alone = {}
    run(a, sa, dta, 8, alone, "a")
    run(b, sb, dtb, 8, alone, "b")
    together = {}
    ta = threading.Thread(target=run, args=(a, sa, dta, 8, together, "a"))
    tb = threading.Thread(target=run, args=(b, sb, dtb, 8, together, "b"))
    ta.start()
    tb.start()
    ta.join(300)
    tb.join(300)
    assert set(together) == {"a", "b"}
    for key in ("a", "b"):
        for f in ("ro", "rou", "rov", "cxx", "cxy", "cyy"):
            assert np.array_equal(together[key][f], alone[key][f]), (key, f)
    a.close()
    b.close()
