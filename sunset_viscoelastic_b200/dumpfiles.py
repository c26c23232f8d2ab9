"""The reference's dump files (output.F90:184-370, 421-476) and restart input
(setup_domain.F90:206-242, setup_flow.F90:448-552), read and written from Python.

fields_<10000+rank>_<n>:
    !! header !!
    npfb
    eflow_nm1 sum_eflow driving_force(1:3)
    emax_np1 emax_n emax_nm1 dt
    !! end header !!
    then per node: rho - rho_char, u, v, vorticity, Q criterion, alpha_out, cxx, cxy, cyy, czz
    (-Ddim3 -Dallout: per node-layer, layer-major: rho - rho_char, u, v, w, |vorticity|, Q,
    alpha_out, cxx, cxy, cyy, cxz, cyz, czz)
nodes_<10000+rank>:
    npfb
    then per node: global index, x, y, s, h, h_small, node type (3-D: global index, x, y, z, s, h,
    h_small, node type)

Both are Fortran list-directed output, so numbers are separated by blanks and may carry a
D exponent; the readers accept either.
"""
from __future__ import annotations

import numpy as np

FIELD_COLUMNS = ["ro_minus_rho_char", "u", "v", "vort", "qcrit", "alpha", "cxx", "cxy", "cyy", "czz"]
FIELD_COLUMNS_3D = ["ro_minus_rho_char", "u", "v", "w", "vort", "qcrit", "alpha", "cxx", "cxy", "cyy", "cxz", "cyz",
                    "czz"]
HEADER = ["eflow_nm1", "sum_eflow", "driving_force_x", "driving_force_y", "driving_force_z", "emax_np1", "emax_n",
          "emax_nm1", "dt"]


def _floats(line: str) -> list[float]:
    return [float(t.replace("D", "E").replace("d", "e")) for t in line.split()]


def read_fields(path) -> tuple[np.ndarray, dict]:
    """(header, columns): header the 9 values of HEADER, columns a dict of FIELD_COLUMNS (of
    FIELD_COLUMNS_3D for a 3-D dump's 13 values a row)."""
    with open(path) as f:
        lines = f.read().splitlines()
    if "header" not in lines[0]:
        raise ValueError(f"{path}: no header line")
    n = int(lines[1].split()[0])
    header = np.array(_floats(lines[2]) + _floats(lines[3]))
    if len(header) != 9 or "end header" not in lines[4]:
        raise ValueError(f"{path}: malformed header")
    body = np.array([_floats(l) for l in lines[5:5 + n]])
    if body.ndim != 2 or body.shape[0] != n or body.shape[1] not in (10, 13):
        raise ValueError(f"{path}: expected {n} rows of 10 (or 13) values, got {body.shape}")
    keys = FIELD_COLUMNS if body.shape[1] == 10 else FIELD_COLUMNS_3D
    return header, {k: body[:, c].copy() for c, k in enumerate(keys)}


def read_nodes(path) -> dict:
    """global index, x, y (z in 3-D), s, h, h_small, node type of every node."""
    with open(path) as f:
        lines = f.read().splitlines()
    n = int(lines[0].split()[0])
    rows = [l.split() for l in lines[1:1 + n]]
    w = len(rows[0]) if rows else 7
    if len(rows) != n or w not in (7, 8) or any(len(r) != w for r in rows):
        raise ValueError(f"{path}: expected {n} rows of 7 (or 8) values")
    col = lambda c, t: np.array([t(r[c].replace("D", "E")) for r in rows])
    o = 1 if w == 8 else 0
    out = dict(gi=col(0, int), x=col(1, float), y=col(2, float), s=col(3 + o, float), h=col(4 + o, float),
               h_small=col(5 + o, float), node_type=col(6 + o, int))
    if w == 8:
        out["z"] = col(3, float)
    return out


def write_fields(path, header, columns) -> None:
    """A fields dump in the reference's layout (columns: dict or 10 x npfb)."""
    if isinstance(columns, dict):
        columns = np.stack([columns[k] for k in FIELD_COLUMNS])
    columns = np.asarray(columns, np.float64)
    n = columns.shape[1]
    h = np.asarray(header, np.float64)
    with open(path, "w") as f:
        f.write(" !! header !!\n")
        f.write(f" {n}\n")
        f.write(" " + " ".join(f"{v:.17E}" for v in h[:5]) + "\n")
        f.write(" " + " ".join(f"{v:.17E}" for v in h[5:9]) + "\n")
        f.write(" !! end header !!\n")
        for i in range(n):
            f.write(" " + " ".join(f"{v:.17E}" for v in columns[:, i]) + "\n")


def write_nodes(path, nodes: dict) -> None:
    n = len(nodes["x"])
    with open(path, "w") as f:
        f.write(f" {n}\n")
        for i in range(n):
            f.write(f" {int(nodes['gi'][i])} {nodes['x'][i]:.17E} {nodes['y'][i]:.17E} {nodes['s'][i]:.17E} "
                    f"{nodes['h'][i]:.17E} {nodes['h_small'][i]:.17E} {int(nodes['node_type'][i])}\n")
