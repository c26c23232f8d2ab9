"""The reference's dump and restart files (output.F90:272-310,441-450) read and written on the
host: a file in gfortran's list-directed layout parses, and writing then reading returns the
same numbers bit for bit."""
import numpy as np

from sunset_viscoelastic_b200 import dumpfiles as D

SAMPLE_FIELDS = """ !! header !!
           3
   0.0000000000000000        0.0000000000000000        0.0000000000000000        0.0000000000000000        0.0000000000000000
   1.2345000000000000E-005   1.0000000000000001E-005   9.9999999999999991E-006   2.0000000000000001D-004
 !! end header !!
  -1.0000000000000000E-003  0.50000000000000000      -0.25000000000000000        1.5000000000000000       -0.75000000000000000        3.0000000000000001E-007   1.1000000000000001        2.0000000000000000E-002   1.0000000000000000        1.0000000000000000
   0.0000000000000000        1.0000000000000000        0.0000000000000000        0.0000000000000000        0.0000000000000000        0.0000000000000000        1.0000000000000000        0.0000000000000000        1.0000000000000000        1.0000000000000000
   2.0000000000000000E-003 -0.50000000000000000       0.25000000000000000       -1.5000000000000000        0.75000000000000000        1.0000000000000000E-007   1.2000000000000000       -2.0000000000000000E-002   1.1000000000000001        1.0000000000000000
"""

SAMPLE_NODES = """           2
           1   0.0000000000000000        0.0000000000000000        1.9531250000000000E-003   4.6875000000000003E-003   4.6875000000000003E-003         999
           2   1.9531250000000000E-003   0.0000000000000000        1.9531250000000000E-003   4.6875000000000003E-003   4.0000000000000001E-003          -1
"""


def test_reads_list_directed_layout(tmp_path):
    p = tmp_path / "fields_10000_3"
    p.write_text(SAMPLE_FIELDS)
    hd, cols = D.read_fields(p)
    assert hd.tolist() == [0, 0, 0, 0, 0, 1.2345e-5, 1.0000000000000001e-5, 9.9999999999999991e-6, 2.0000000000000001e-4]
    assert cols["u"].tolist() == [0.5, 1.0, -0.5]
    assert cols["cxy"][0] == 2.0e-2 and cols["czz"].tolist() == [1.0, 1.0, 1.0]
    q = tmp_path / "nodes_10000"
    q.write_text(SAMPLE_NODES)
    nd = D.read_nodes(q)
    assert nd["gi"].tolist() == [1, 2] and nd["node_type"].tolist() == [999, -1]
    assert nd["h_small"][1] == 4.0000000000000001e-3


def test_write_read_round_trip_is_exact(tmp_path):
    rng = np.random.default_rng(4)
    cols = rng.standard_normal((10, 57)) * 10.0 ** rng.integers(-12, 6, (10, 57))
    hd = rng.standard_normal(9)
    D.write_fields(tmp_path / "f", hd, cols)
    hd2, c2 = D.read_fields(tmp_path / "f")
    assert np.array_equal(hd2, hd)
    assert np.array_equal(np.stack([c2[k] for k in D.FIELD_COLUMNS]), cols)
    nodes = dict(gi=np.arange(1, 58), x=rng.random(57), y=rng.random(57), s=rng.random(57), h=rng.random(57),
                 h_small=rng.random(57), node_type=rng.integers(-4, 1000, 57))
    D.write_nodes(tmp_path / "n", nodes)
    n2 = D.read_nodes(tmp_path / "n")
    for k in nodes:
        assert np.array_equal(n2[k], nodes[k]), k
