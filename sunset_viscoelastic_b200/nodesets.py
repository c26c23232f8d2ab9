"""Node sets for the LABFM path: the IPART format and seeded synthetic workloads.

The reference reads its node set from an ``IPART`` file (setup_domain.F90:93-199):

    line 1: nb npfb smax smin
    line 2: xmin xmax ymin ymax
    line 3: xbcond_L xbcond_U ybcond_L ybcond_U      (0 none, 1 periodic, 2 symmetric, 3 no-slip)
    line 4: nprocsX nprocsY nprocsZ                   (MPI schedule, ignored without MPI)
    line 5: nprocs, then nprocs lines "start end"
    then one row per node: global_index x y node_type nx ny s

``node_type`` is 999 for fluid, 0/1/2 for wall/inflow/outflow boundary nodes (for which
the reader of the reference adds four finite-difference rows along the normal).

The synthetic workloads are seeded jittered lattices on the doubly periodic unit square
(each lattice point offset by a uniform draw in +-0.3 s per axis); they stand in for the
node sets the reference's node generator (source/gen) would make.
"""
from __future__ import annotations

import dataclasses
import math
from typing import Optional

import numpy as np


@dataclasses.dataclass
class NodeSet:
    x: np.ndarray
    y: np.ndarray
    node_type: np.ndarray
    nx: np.ndarray
    ny: np.ndarray
    s: np.ndarray
    xmin: float
    xmax: float
    ymin: float
    ymax: float
    bcond: tuple = (1, 1, 1, 1)
    gi: Optional[np.ndarray] = None

    def __post_init__(self):
        n = len(self.x)
        if self.gi is None:
            self.gi = np.arange(1, n + 1, dtype=np.int32)
        self.x = np.ascontiguousarray(self.x, dtype=np.float64)
        self.y = np.ascontiguousarray(self.y, dtype=np.float64)
        self.node_type = np.ascontiguousarray(self.node_type, dtype=np.int32)
        self.nx = np.ascontiguousarray(self.nx, dtype=np.float64)
        self.ny = np.ascontiguousarray(self.ny, dtype=np.float64)
        self.s = np.ascontiguousarray(self.s, dtype=np.float64)
        self.gi = np.ascontiguousarray(self.gi, dtype=np.int32)

    @property
    def n(self) -> int:
        return len(self.x)

    @property
    def smax(self) -> float:
        return float(self.s.max())

    @property
    def smin(self) -> float:
        return float(self.s.min())


def jittered_lattice(nside: int, jitter: float = 0.3, seed: int = 12345,
                     length: float = 1.0) -> NodeSet:
    """nside x nside lattice on [0,length]^2, spacing s=length/nside, each node moved by
    U(-jitter*s, jitter*s) per axis (numpy default_rng(seed)); doubly periodic."""
    s = length / nside
    rng = np.random.default_rng(seed)
    ii, jj = np.meshgrid(np.arange(nside), np.arange(nside), indexing="xy")
    x = (ii.ravel() + 0.5) * s + rng.uniform(-jitter * s, jitter * s, nside * nside)
    y = (jj.ravel() + 0.5) * s + rng.uniform(-jitter * s, jitter * s, nside * nside)
    n = nside * nside
    return NodeSet(x=x, y=y, node_type=np.full(n, 999, np.int32), nx=np.zeros(n), ny=np.zeros(n),
                   s=np.full(n, s), xmin=0.0, xmax=length, ymin=0.0, ymax=length, bcond=(1, 1, 1, 1))


def reader_nodes(ns: NodeSet):
    """Positions and types of the node list the reference's reader builds from IPART rows:
    each boundary node (node_type 0..2) is followed by four FD rows at j s along its normal,
    node_type -j (setup_domain.F90:177-199)."""
    x, y, t = [], [], []
    for k in range(ns.n):
        x.append(ns.x[k]); y.append(ns.y[k]); t.append(int(ns.node_type[k]))
        if 0 <= ns.node_type[k] <= 2:
            for j in range(1, 5):
                x.append(ns.x[k] + (ns.nx[k] * float(j)) * ns.s[k])
                y.append(ns.y[k] + (ns.ny[k] * float(j)) * ns.s[k])
                t.append(-j)
    return np.array(x), np.array(y), np.array(t, np.int32)


def _with_gaps(types: np.ndarray) -> np.ndarray:
    """Global indices leaving room for the four FD rows the reader adds after each boundary
    node (it numbers them global_index + 1..4, setup_domain.F90:183-190)."""
    step = np.where((types >= 0) & (types <= 2), 5, 1)
    return (np.cumsum(step) - step + 1).astype(np.int32)


def channel(ny_cells: int, lx: float = 1.0, ly: float = 1.0, jitter: float = 0.3,
            seed: int = 12345) -> NodeSet:
    """Walled channel, periodic in x on [0, lx), walls (node_type 0) at y = 0 and y = ly
    with normals into the fluid.  Spacing s = ly / ny_cells.  Wall nodes sit at
    x = (i + 1/2) s; the reader adds their FD rows at 1..4 s along the normal.  The interior
    is the jittered lattice (+-jitter s per axis, default_rng(seed)) on the rows 5..ny_cells-5,
    which keeps it clear of the FD rows."""
    s = ly / ny_cells
    nxc = int(round(lx / s))
    xs = (np.arange(nxc) + 0.5) * s
    rng = np.random.default_rng(seed)
    yj = np.arange(5, ny_cells - 4) * s
    ix, iy = np.meshgrid(xs, yj, indexing="xy")
    n_int = ix.size
    xi = ix.ravel() + rng.uniform(-jitter * s, jitter * s, n_int)
    yi = iy.ravel() + rng.uniform(-jitter * s, jitter * s, n_int)
    x = np.concatenate([xs, xi, xs])
    y = np.concatenate([np.zeros(nxc), yi, np.full(nxc, ly)])
    t = np.concatenate([np.zeros(nxc, np.int32), np.full(n_int, 999, np.int32), np.zeros(nxc, np.int32)])
    nx = np.zeros(len(x))
    ny = np.concatenate([np.ones(nxc), np.zeros(n_int), -np.ones(nxc)])
    return NodeSet(x=x, y=y, node_type=t, nx=nx, ny=ny, s=np.full(len(x), s), xmin=0.0, xmax=lx,
                   ymin=0.0, ymax=ly, bcond=(1, 1, 0, 0), gi=_with_gaps(t))


def inflow_channel(ny_cells: int, lx: float = 2.0, ly: float = 1.0, ybc: int = 1, jitter: float = 0.3,
                   seed: int = 12345) -> NodeSet:
    """Inflow/outflow tube [0, lx] x [0, ly] in the layout of the reference generator's
    in/out cases (gen/datclass.F90 cases 5 and 6): an inflow (node_type 1, normal +x) at
    x = 0, an outflow (node_type 2, normal -x) at x = lx, and periodic (ybc = 1) or symmetric
    (ybc = 2) conditions in y, so no wall meets an inflow.  Spacing s = ly / ny_cells; the
    inflow and outflow nodes sit at y = (j + 1/2) s and the reader adds their FD rows at
    1..4 s along the normal; the interior is a jittered lattice on the x cells 5 .. n - 6."""
    if ybc not in (1, 2):
        raise ValueError("ybc must be 1 (periodic) or 2 (symmetric)")
    s = ly / ny_cells
    nxc = int(round(lx / s))
    ys = (np.arange(ny_cells) + 0.5) * s
    rng = np.random.default_rng(seed)
    xj = (np.arange(5, nxc - 5) + 0.5) * s
    ix, iy = np.meshgrid(xj, ys, indexing="xy")
    n_int = ix.size
    xi = ix.ravel() + rng.uniform(-jitter * s, jitter * s, n_int)
    yi = iy.ravel() + rng.uniform(-jitter * s, jitter * s, n_int)
    ni = len(ys)
    x = np.concatenate([np.zeros(ni), xi, np.full(ni, lx)])
    y = np.concatenate([ys, yi, ys])
    t = np.concatenate([np.ones(ni, np.int32), np.full(n_int, 999, np.int32), np.full(ni, 2, np.int32)])
    nx = np.concatenate([np.ones(ni), np.zeros(n_int), -np.ones(ni)])
    ny = np.zeros(len(x))
    return NodeSet(x=x, y=y, node_type=t, nx=nx, ny=ny, s=np.full(len(x), s), xmin=0.0, xmax=lx,
                   ymin=0.0, ymax=ly, bcond=(0, 0, ybc, ybc), gi=_with_gaps(t))


def inflow_state(ns, u0: float = 1.0, amp: float = 0.05, ly: float = 1.0):
    """Uniform stream u0 in x with a smooth perturbation that respects both y conditions
    (v odd about y = 0 and y = ly, everything else even), and a smooth positive-definite
    conformation: u = u0 (1 + amp cos(2 pi y / ly) cos(pi x)), v = amp u0 sin(2 pi y / ly)
    sin(pi x), rho = 1 + amp/10 cos(pi x).  ns: any object with the reader's x, y."""
    x, y = ns.x, ns.y
    ky = 2.0 * np.pi / ly
    return dict(ro=1.0 + 0.1 * amp * np.cos(np.pi * x), u=u0 * (1.0 + amp * np.cos(ky * y) * np.cos(np.pi * x)),
                v=amp * u0 * np.sin(ky * y) * np.sin(np.pi * x), cxx=1.2 + 0.1 * np.cos(ky * y),
                cxy=0.05 * np.sin(ky * y) * np.cos(np.pi * x), cyy=1.1 + 0.05 * np.cos(np.pi * x), czz=np.ones(len(x)))


def cylinder_channel(R: float = 1.0, half_length: float = 15.0, half_height: float = 2.0, s_min_frac: float = 1 / 64,
                     s_max_frac: float = 1 / 16, growth: float = 0.1, jitter: float = 0.3,
                     seed: int = 12345) -> NodeSet:
    """Channel [-half_length, half_length] x [-half_height, half_height], periodic in x, with
    no-slip walls (node_type 0) at y = +-half_height and a cylinder of radius R at the
    origin.  Local spacing s(r) = s_min + growth (r - R'), capped at s_max, with
    s_min = s_min_frac R, s_max = s_max_frac R and R' = R + 4 s_min: the law is measured from
    the cylinder's last FD row, so the first fluid layers continue the rows' spacing (measured
    from R itself the first ring already sits at 1.4 s_min, and the order-6 stencils of the
    fourth FD row, which then see mostly the regular polar grid of the rows, reach condition
    numbers of 1e9).

    Boundary nodes: the cylinder at spacing ~s_min with outward normals, the walls at s_max
    with normals into the channel; the reader adds their FD rows at 1..4 s along the normal.
    Fluid nodes: rings around the cylinder, from just outside its FD rows, each ring one
    local spacing further out, while the spacing grows; beyond them the jittered lattice at
    s_max, kept clear of the rings and of the walls' FD rows.  Every fluid node is moved by
    U(-jitter s, jitter s) per axis (default_rng(seed))."""
    rng = np.random.default_rng(seed)
    s_min, s_max = s_min_frac * R, s_max_frac * R
    r_fd = R + 4.0 * s_min  # the cylinder's last FD row: the fluid continues at s_min from there
    sfun = lambda r: np.minimum(s_min + growth * np.maximum(r - r_fd, 0.0), s_max)
    xs, ys, ts, nxs, nys, ss = [], [], [], [], [], []

    def add(x, y, t, nx, ny, sp):
        xs.append(np.atleast_1d(x)); ys.append(np.atleast_1d(y)); ts.append(np.atleast_1d(t).astype(np.int32))
        nxs.append(np.atleast_1d(nx)); nys.append(np.atleast_1d(ny)); ss.append(np.atleast_1d(sp))

    # cylinder wall
    nb = int(round(2 * np.pi * R / s_min))
    th = 2 * np.pi * np.arange(nb) / nb
    sb = 2 * np.pi * R / nb
    add(R * np.cos(th), R * np.sin(th), np.zeros(nb), np.cos(th), np.sin(th), np.full(nb, sb))
    # channel walls
    nw = int(round(2 * half_length / s_max))
    sw = 2 * half_length / nw
    xw = -half_length + (np.arange(nw) + 0.5) * sw
    for y0, ny0 in ((-half_height, 1.0), (half_height, -1.0)):
        add(xw, np.full(nw, y0), np.zeros(nw), np.zeros(nw), np.full(nw, ny0), np.full(nw, sw))
    # rings
    r = R + 4.0 * sb + sfun(R + 4.0 * sb)  # = R + 5 s_min
    k = 0
    ring_out = R
    while True:
        sr = float(sfun(r))
        m = int(round(2 * np.pi * r / sr))
        if r + sr > half_height - 4.5 * sw or (sr >= s_max and r > r_fd + (s_max - s_min) / growth + 2 * s_max):
            break
        a = 2 * np.pi * (np.arange(m) + 0.5 * (k % 2)) / m
        sp = 2 * np.pi * r / m
        x = r * np.cos(a) + rng.uniform(-jitter * sp, jitter * sp, m)
        y = r * np.sin(a) + rng.uniform(-jitter * sp, jitter * sp, m)
        add(x, y, np.full(m, 999), np.zeros(m), np.zeros(m), np.full(m, sp))
        ring_out = r
        r = r + sr
        k += 1
    # lattice beyond the rings and clear of the walls' FD rows
    ny_rows = int(round(2 * half_height / sw))
    yj = -half_height + np.arange(5, ny_rows - 4) * sw
    ix, iy = np.meshgrid(xw, yj, indexing="xy")
    keep = np.hypot(ix, iy) > ring_out + 0.75 * s_max
    n = int(keep.sum())
    x = ix[keep] + rng.uniform(-jitter * sw, jitter * sw, n)
    y = iy[keep] + rng.uniform(-jitter * sw, jitter * sw, n)
    add(x, y, np.full(n, 999), np.zeros(n), np.zeros(n), np.full(n, sw))
    cat = lambda v: np.concatenate(v)
    t = cat(ts)
    return NodeSet(x=cat(xs), y=cat(ys), node_type=t, nx=cat(nxs), ny=cat(nys), s=cat(ss), xmin=-half_length,
                   xmax=half_length, ymin=-half_height, ymax=half_height, bcond=(1, 1, 0, 0), gi=_with_gaps(t))


def poiseuille_state(ns: NodeSet, G: float, mu_total: float, lam: float, ly: float = 1.0):
    """Steady Oldroyd-B Poiseuille flow driven by a body force G in x between walls at
    y = 0 and ly: u = G y (ly - y) / (2 mu_total), v = 0, rho = 1, c_xy = lam u',
    c_xx = 1 + 2 (lam u')^2, c_yy = c_zz = 1.  (Values at the FD rows follow from the
    reader's positions, so they are returned for the reader's node list.)"""
    u = G * ns.y * (ly - ns.y) / (2.0 * mu_total)
    du = G * (ly - 2.0 * ns.y) / (2.0 * mu_total)
    n = ns.n
    return dict(ro=np.ones(n), u=u, v=np.zeros(n), cxx=1.0 + 2.0 * (lam * du) ** 2, cxy=lam * du,
                cyy=np.ones(n), czz=np.ones(n))


def read_ipart(path: str) -> NodeSet:
    """Reader following setup_domain.F90:93-199 (non-MPI branch)."""
    with open(path) as f:
        lines = [ln for ln in f.read().splitlines()]
    it = iter(lines)

    def nxt():
        while True:
            try:
                ln = next(it)
            except StopIteration:
                raise ValueError(f"{path}: the file ends before the {npfb} node rows its header announces") from None
            if ln.strip():
                return ln.split()

    npfb = 0
    nb, npfb, smax, smin = nxt()
    npfb = int(npfb)
    xmin, xmax, ymin, ymax = (float(v) for v in nxt())
    bc = tuple(int(v) for v in nxt())
    nxt()  # nprocsX nprocsY nprocsZ
    nproc = int(nxt()[0])
    for _ in range(nproc):
        nxt()
    rows = [nxt() for _ in range(npfb)]
    if any(len(r) < 7 for r in rows):
        raise ValueError(f"{path}: a node row has fewer than the 7 columns gi x y type nx ny s")
    a = np.array([[float(v.replace("D", "E")) for v in r] for r in rows])
    return NodeSet(x=a[:, 1], y=a[:, 2], node_type=a[:, 3].astype(np.int32), nx=a[:, 4], ny=a[:, 5],
                   s=a[:, 6], xmin=xmin, xmax=xmax, ymin=ymin, ymax=ymax, bcond=bc,
                   gi=a[:, 0].astype(np.int32))


def write_ipart(path: str, ns: NodeSet) -> None:
    nb = int(np.sum((ns.node_type >= 0) & (ns.node_type <= 2)))
    with open(path, "w") as f:
        f.write(f"{nb} {ns.n} {ns.smax:.17g} {ns.smin:.17g}\n")
        f.write(f"{ns.xmin:.17g} {ns.xmax:.17g} {ns.ymin:.17g} {ns.ymax:.17g}\n")
        f.write(" ".join(str(int(b)) for b in ns.bcond) + "\n")
        f.write("1 1 1\n1\n1 %d\n" % ns.n)
        for k in range(ns.n):
            f.write(f"{ns.gi[k]} {ns.x[k]:.17g} {ns.y[k]:.17g} {ns.node_type[k]} "
                    f"{ns.nx[k]:.17g} {ns.ny[k]:.17g} {ns.s[k]:.17g}\n")


@dataclasses.dataclass
class Workload:
    """One of the measured configurations: node set, LABFM order, stencil radius,
    formulation and fluid parameters."""
    name: str
    nside: int
    order: int
    radius_over_s: float
    form: str            # "di" | "chl" | "lc"
    Re: float = 1.0
    Wi: float = 1.0
    beta: float = 0.5
    Ma: float = 0.1
    epsPTT: float = 0.0
    steps: int = 100
    cfl: float = 0.3
    geometry: str = "periodic"   # "periodic" (jittered lattice) | "cylinder" (walled channel)
    grav_x: float = 0.0          # body force in x
    kolmogorov_forcing: int = -1  # the reference's default (Cholesky form only)

    @property
    def n(self) -> int:
        return self.nside * self.nside if self.geometry != "cylinder" else self.nodes().n

    @property
    def h_over_s(self) -> float:
        # support radius = ss*h with ss = 2; 0 keeps the reference's own hovs / hovs_bound
        return self.radius_over_s / 2.0

    def nodes(self) -> NodeSet:
        if self.geometry == "cylinder":
            return cylinder_channel()
        return jittered_lattice(self.nside)

    @property
    def periodic(self) -> bool:
        return self.geometry != "cylinder"

    def params(self) -> dict:
        """Keyword arguments of labfm.Sunset / oracle.Oracle for this workload."""
        return dict(form=self.form, order=self.order, Re=self.Re, Wi=self.Wi, beta=self.beta, epsPTT=self.epsPTT,
                    Ma=self.Ma, h_over_s=self.h_over_s, grav=(self.grav_x, 0.0, 0.0),
                    kolmogorov_forcing=self.kolmogorov_forcing)

    def initial(self, ns: NodeSet) -> dict:
        """Initial state on the reader's node list (FD rows included)."""
        if self.geometry == "periodic-psi0":
            return initial_state_psi0(ns)
        if self.geometry == "cylinder":
            x, y, _ = reader_nodes(ns)
            n = len(x)
            z, one = np.zeros(n), np.ones(n)
            return dict(ro=one, u=z, v=z, cxx=one, cxy=z, cyy=one, czz=one)
        return initial_state(ns)


# Radii.  The reference adapts each node's stencil (labf.F90:1079-1721); with one fixed
# radius on jittered nodes the nominal radii are too small: at 2.6 s (order 4), 3.2 s
# (order 6) and 4.2 s (order 8) some nodes get near-singular moment matrices (max
# |w_lap| s^2 ~ 1e4) and the reference algorithm diverges within a few steps.  At order 6
# the 512^2 set still holds a few stencils whose filter row sums exceed 2 at K ~ 45
# (3.78 s) and 4.0 s, and the step diverges within 200 steps, so order 6 uses 4.2 s
# (K ~ 55).  At order 8 the radius from the stated neighbour count, r = s sqrt(K/pi) with
# K ~ 70 (4.72 s), keeps 100 steps finite but grows an unstable mode that overflows before
# step 500 (max |rho - 1| 4e-9 at step 50, 3e-4 at step 400); the reference's own initial
# stencil for order 8, h = 2.7 s (common_parameter.F90:55, radius ss*h = 5.4 s, K ~ 92),
# stays bounded through 500 steps.  Order 4 uses 3.0 s (K ~ 28).
# The walled cylinder channel: Oldroyd-B (direct form) at Re 0.01, Wi 0.5, beta 0.59,
# Ma 0.05, driven by a body force of 50 (a centreline speed near 1 in the empty channel), from
# rest; the reference's own stencil sizes (hovs 2.7, hovs_bound 2.4 at order 8).
WORKLOADS = {
    "periodic-di-o4-16k": Workload("periodic-di-o4-16k", 128, 4, 3.0, "di", steps=100),
    "periodic-lc-o6-262k": Workload("periodic-lc-o6-262k", 512, 6, 4.2, "lc", epsPTT=0.25, steps=200),
    "periodic-chl-o8-1m": Workload("periodic-chl-o8-1m", 1024, 8, 5.4, "chl", Wi=2.0, beta=0.1, steps=500),
    "cylinder-channel-o8": Workload("cylinder-channel-o8", 0, 8, 0.0, "di", Re=0.01, Wi=0.5, beta=0.59, Ma=0.05,
                                    steps=2000, geometry="cylinder", grav_x=50.0, kolmogorov_forcing=0),
    # the differentiation configuration: the order-6 set, Oldroyd-B in log-conformation form,
    # from a non-degenerate log-conformation field (initial_state_psi0)
    "periodic-lc-o6-262k-adjoint": Workload("periodic-lc-o6-262k-adjoint", 512, 6, 4.2, "lc", Wi=1.0, beta=0.5,
                                            steps=200, geometry="periodic-psi0"),
}


def psi0_field(x, y):
    """A smooth, non-degenerate initial log-conformation field psi = log c."""
    return (0.2 + 0.1 * np.sin(2 * np.pi * x), 0.1 * np.cos(2 * np.pi * y),
            -0.1 + 0.05 * np.sin(2 * np.pi * (x + y)))


def initial_state_psi0(ns: NodeSet):
    """Taylor-Green velocity, rho = 1, c = exp(psi0) (psi0_field).  At c = I the eigenvalues
    of psi coincide and the log-conformation right-hand side's omega branch
    (rhs_lc.F90:465-469) is degenerate, so the differentiation runs start from here."""
    st = initial_state(ns)
    a, b, d = psi0_field(ns.x, ns.y)
    # exp of the symmetric 2x2 matrix [[a, b], [b, d]]
    m, r = 0.5 * (a + d), np.sqrt(0.25 * (a - d) ** 2 + b * b)
    e1, e2 = np.exp(m + r), np.exp(m - r)
    sh = np.where(r > 0, (e1 - e2) / np.where(r > 0, 2 * r, 1.0), e1)
    ch = 0.5 * (e1 + e2)
    st["cxx"] = ch + sh * 0.5 * (a - d)
    st["cyy"] = ch - sh * 0.5 * (a - d)
    st["cxy"] = sh * b
    return st


def initial_state(ns: NodeSet):
    """u=sin(2 pi x)cos(2 pi y), v=-cos(2 pi x)sin(2 pi y), rho=1, c=I."""
    u = np.sin(2 * np.pi * ns.x) * np.cos(2 * np.pi * ns.y)
    v = -np.cos(2 * np.pi * ns.x) * np.sin(2 * np.pi * ns.y)
    n = ns.n
    return dict(ro=np.ones(n), u=u, v=v, cxx=np.ones(n), cxy=np.zeros(n), cyy=np.ones(n),
                czz=np.ones(n))
