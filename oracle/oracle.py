"""ctypes front end of the CPU restatement (sunset_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and bench.py's CPU
baseline, never by the product package.  Parity of the restatement with the Fortran
reference is unpinned by reference outputs (see sunset_oracle.h); it is pinned by the
LABFM moment conditions and the reference's analytic checks.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "build", "libsunset_oracle.so")

FORMS = {"di": 0, "chl": 1, "lc": 2, "newt": 3}


class OrConfig(C.Structure):
    _fields_ = [("form", C.c_int), ("fenep", C.c_int), ("morder", C.c_int), ("forder", C.c_int),
                ("mcorr", C.c_int), ("kolmogorov_forcing", C.c_int), ("di_full_gradients", C.c_int),
                ("L_char", C.c_double), ("U_char", C.c_double), ("Re", C.c_double), ("Wi", C.c_double),
                ("beta", C.c_double), ("epsPTT", C.c_double), ("fenep_l2", C.c_double),
                ("Mdiff", C.c_double), ("Ma", C.c_double), ("grav", C.c_double * 3),
                ("h_over_s", C.c_double), ("inflow_type", C.c_int), ("inflow_velocity_control", C.c_int),
                ("u_inflow_start", C.c_double), ("u_inflow_end", C.c_double), ("ramp_time", C.c_double),
                ("vpid", C.c_int)]


def build() -> str:
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        P = C.c_void_p
        dp = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
        ip = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
        L.or_create.restype = P
        L.or_create.argtypes = [C.POINTER(OrConfig)]
        L.or_destroy.argtypes = [P]
        L.or_last_error.restype = C.c_char_p
        L.or_last_error.argtypes = [P]
        L.or_set_threads.argtypes = [C.c_int]
        L.or_build_domain.argtypes = [P, C.c_int, ip, dp, dp, ip, dp, dp, dp, C.c_double, C.c_double,
                                      C.c_double, C.c_double, ip, C.c_double]
        L.or_sizes.argtypes = [P, C.POINTER(C.c_int)] * 1 + [C.POINTER(C.c_int)] * 3
        for name in ["or_find_neighbours", "or_adapt_stencils", "or_calc_labf_weights", "or_calc_boundary_weights",
                     "or_calc_labf_sums", "or_filter_coefficients", "or_setup_all"]:
            getattr(L, name).argtypes = [P]
        L.or_get_nodes.argtypes = [P, dp, dp, dp, dp, dp, ip, ip, ip]
        L.or_get_neighbours.argtypes = [P, ip, ip, ip]
        L.or_get_weights.argtypes = [P, dp, dp, dp, dp, dp, dp, dp]
        L.or_get_conditioning.argtypes = [P, dp, dp]
        L.or_set_neighbours_weights.argtypes = [P, C.c_int, ip, ip, ip, dp, dp, dp, dp, dp, dp, dp]
        for name in ["or_calc_gradient", "or_calc_laplacian", "or_calc_filtered_var", "or_calc_filter_term"]:
            getattr(L, name).argtypes = [P, dp, dp]
        L.or_set_state.argtypes = [P, dp, dp, dp, dp, dp, dp, dp]
        L.or_set_raw_state.argtypes = [P, dp, dp, dp, dp]
        L.or_get_state.argtypes = [P, dp]
        L.or_calc_all_rhs.argtypes = [P, dp]
        L.or_set_tstep.argtypes = [P, C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.or_step.argtypes = [P, C.c_double, C.c_int, C.c_int]
        L.or_get_time.argtypes = [P, C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_int), dp]
        L.or_set_time.argtypes = [P, C.c_double, C.c_double, C.c_int, dp]
        L.or_get_flow_control.argtypes = [P, dp]
        L.or_set_flow_control.argtypes = [P, dp]
        L.or_kinetic_energy.restype = C.c_double
        L.or_kinetic_energy.argtypes = [P]
        L.or_mass.restype = C.c_double
        L.or_mass.argtypes = [P]
        L.or_svd_solve.argtypes = [dp, C.c_int, dp]
        L.or_wab.restype = C.c_double
        L.or_wab.argtypes = [C.c_double, C.c_double]
        L.or_monomials.argtypes = [C.c_int, C.c_double, C.c_double, dp]
        L.or_abfs.argtypes = [C.c_int, C.c_double, C.c_double, dp]
        L.or_pow4_libm.restype = C.c_double
        L.or_pow4_libm.argtypes = [C.c_double]
        L.or_pow4_cr.restype = C.c_double
        L.or_pow4_cr.argtypes = [C.c_double]
        L.or_set_pow_mode.argtypes = [C.c_int]
        L.or3_create.restype = P
        L.or3_create.argtypes = [P, C.c_double]
        L.or3_destroy.argtypes = [P]
        L.or3_sizes.argtypes = [P, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_double)]
        L.or3_set_state.argtypes = [P, dp, dp, dp, dp, C.c_void_p]
        L.or3_get_state.argtypes = [P, dp]
        L.or3_rhs.argtypes = [P, dp]
        L.or3_set_tstep.argtypes = [P, C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.or3_step.argtypes = [P, C.c_double, C.c_int, C.c_int]
        L.or3_get_time.argtypes = [P, C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_int), dp]
        L.or3_kinetic_energy.restype = C.c_double
        L.or3_kinetic_energy.argtypes = [P]
        L.or3_mass.restype = C.c_double
        L.or3_mass.argtypes = [P]
        L.or3_get_dump.argtypes = [P, dp, dp]
        _lib = L
    return _lib


def set_threads(n: int) -> None:
    lib().or_set_threads(int(n))


def set_pow_mode(correctly_rounded: bool) -> None:
    """False (default): libm pow in the Wendland kernel, as the reference; True: the
    correctly rounded x^4 the device path uses."""
    lib().or_set_pow_mode(int(bool(correctly_rounded)))


class OracleError(RuntimeError):
    pass


STATE_FIELDS = ["ro", "rou", "rov", "u", "v", "psixx", "psixy", "psiyy", "psizz", "cxx", "cxy", "cyy", "czz"]
RHS_FIELDS = ["ro", "rou", "rov", "xx", "xy", "yy", "zz"]


class Oracle:
    """One reference 'run': node set + parameters, mirroring the module state of common_vars."""

    def __init__(self, form="di", order=4, forder=None, Re=1.0, Wi=1.0, beta=0.5, epsPTT=0.0, Ma=0.1,
                 fenep=False, fenep_l2=1e30, Mdiff=0.0, grav=(0.0, 0.0, 0.0), mcorr=True,
                 kolmogorov_forcing=-1, di_full_gradients=True, h_over_s=0.0, L_char=1.0, U_char=1.0,
                 inflow_type=1, inflow_velocity_control=0, u_inflow_start=0.0, u_inflow_end=1.0, ramp_time=1.0,
                 vpid=False):
        cfg = OrConfig()
        cfg.form = FORMS[form]
        cfg.fenep = int(fenep)
        cfg.morder = order
        cfg.forder = forder if forder else order
        cfg.mcorr = int(mcorr)
        cfg.kolmogorov_forcing = int(kolmogorov_forcing)
        cfg.di_full_gradients = int(di_full_gradients)
        cfg.L_char, cfg.U_char, cfg.Re, cfg.Wi, cfg.beta = L_char, U_char, Re, Wi, beta
        cfg.epsPTT, cfg.fenep_l2, cfg.Mdiff, cfg.Ma = epsPTT, fenep_l2, Mdiff, Ma
        for k in range(3):
            cfg.grav[k] = grav[k]
        cfg.h_over_s = h_over_s
        cfg.inflow_type, cfg.inflow_velocity_control = int(inflow_type), int(inflow_velocity_control)
        cfg.u_inflow_start, cfg.u_inflow_end, cfg.ramp_time = u_inflow_start, u_inflow_end, ramp_time
        cfg.vpid = int(bool(vpid))
        self.cfg = cfg
        self.L = lib()
        self.h = self.L.or_create(C.byref(cfg))

    def __del__(self):
        try:
            if self.h:
                self.L.or_destroy(self.h)
                self.h = None
        except Exception:
            pass

    def _chk(self, rc):
        if rc != 0:
            raise OracleError(self.L.or_last_error(self.h).decode())

    def build_domain(self, ns):
        bc = np.ascontiguousarray(ns.bcond, dtype=np.int32)
        self._chk(self.L.or_build_domain(self.h, ns.n, ns.gi, ns.x, ns.y, ns.node_type, ns.nx, ns.ny, ns.s,
                                         ns.xmin, ns.xmax, ns.ymin, ns.ymax, bc, ns.smax))
        return self

    def sizes(self):
        a = [C.c_int() for _ in range(4)]
        self.L.or_sizes(self.h, *[C.byref(x) for x in a])
        return tuple(x.value for x in a)  # np, npfb, nb, nplink

    def nodes(self):
        np_, _, _, _ = self.sizes()
        d = {k: np.zeros(np_) for k in ["x", "y", "h", "h_small", "s"]}
        ti = {k: np.zeros(np_, np.int32) for k in ["node_type", "irelation", "vrelation"]}
        self.L.or_get_nodes(self.h, d["x"], d["y"], d["h"], d["h_small"], d["s"], ti["node_type"],
                            ti["irelation"], ti["vrelation"])
        d.update(ti)
        return d

    def find_neighbours(self):
        self._chk(self.L.or_find_neighbours(self.h))

    def adapt_stencils(self):
        """labf.F90:1079-1721 on the current lists, then the neighbour search again."""
        self._chk(self.L.or_adapt_stencils(self.h))

    def calc_labf_weights(self):
        self._chk(self.L.or_calc_labf_weights(self.h))

    def calc_labf_sums(self):
        self._chk(self.L.or_calc_labf_sums(self.h))

    def filter_coefficients(self):
        self._chk(self.L.or_filter_coefficients(self.h))

    def setup(self):
        self._chk(self.L.or_setup_all(self.h))
        return self

    def neighbours(self):
        _, npfb, _, nplink = self.sizes()
        cnt = np.zeros(npfb, np.int32)
        cs = np.zeros(npfb, np.int32)
        lk = np.zeros(npfb * nplink, np.int32)
        self._chk(self.L.or_get_neighbours(self.h, cnt, cs, lk))
        return cnt, cs, lk.reshape(npfb, nplink)

    def weights(self):
        _, npfb, _, nplink = self.sizes()
        wg = np.zeros(npfb * nplink * 2)
        wl = np.zeros(npfb * nplink)
        wh = np.zeros(npfb * nplink)
        gs = np.zeros(npfb * 2)
        ls = np.zeros(npfb)
        hs = np.zeros(npfb)
        vol = np.zeros(npfb)
        self._chk(self.L.or_get_weights(self.h, wg, wl, wh, gs, ls, hs, vol))
        return dict(w_grad=wg.reshape(npfb, nplink, 2), w_lap=wl.reshape(npfb, nplink),
                    w_hyp=wh.reshape(npfb, nplink), w_grad_sum=gs.reshape(npfb, 2), w_lap_sum=ls,
                    w_hyp_sum=hs, vol=vol)

    def conditioning(self):
        """sigma_max / sigma_min of each interior node's derivative and filter moment matrix."""
        _, npfb, _, _ = self.sizes()
        cd, cf = np.zeros(npfb), np.zeros(npfb)
        self._chk(self.L.or_get_conditioning(self.h, cd, cf))
        return cd, cf

    def set_neighbours_weights(self, cnt, cs, links, w):
        npfb, nplink = links.shape
        self._chk(self.L.or_set_neighbours_weights(
            self.h, nplink, np.ascontiguousarray(cnt, np.int32), np.ascontiguousarray(cs, np.int32),
            np.ascontiguousarray(links, np.int32).ravel(), np.ascontiguousarray(w["w_grad"]).ravel(),
            np.ascontiguousarray(w["w_lap"]).ravel(), np.ascontiguousarray(w["w_hyp"]).ravel(),
            np.ascontiguousarray(w["w_grad_sum"]).ravel(), np.ascontiguousarray(w["w_lap_sum"]),
            np.ascontiguousarray(w["w_hyp_sum"]), np.ascontiguousarray(w["vol"])))

    def gradient(self, phi):
        _, npfb, _, _ = self.sizes()
        out = np.zeros(2 * npfb)
        self._chk(self.L.or_calc_gradient(self.h, np.ascontiguousarray(phi, np.float64), out))
        return out.reshape(npfb, 2)

    def laplacian(self, phi):
        _, npfb, _, _ = self.sizes()
        out = np.zeros(npfb)
        self._chk(self.L.or_calc_laplacian(self.h, np.ascontiguousarray(phi, np.float64), out))
        return out

    def filtered(self, phi):
        _, npfb, _, _ = self.sizes()
        out = np.zeros(npfb)
        self._chk(self.L.or_calc_filtered_var(self.h, np.ascontiguousarray(phi, np.float64), out))
        return out

    def filter_term(self, phi):
        _, npfb, _, _ = self.sizes()
        out = np.zeros(npfb)
        self._chk(self.L.or_calc_filter_term(self.h, np.ascontiguousarray(phi, np.float64), out))
        return out

    def set_state(self, ro, u, v, cxx, cxy, cyy, czz=None):
        n = self.sizes()[1]
        f = lambda a: np.ascontiguousarray(a, np.float64)
        czz = np.ones(n) if czz is None else czz
        self._chk(self.L.or_set_state(self.h, f(ro), f(u), f(v), f(cxx), f(cxy), f(cyy), f(czz)))

    def set_raw_state(self, ro, rou, rov, q):
        f = lambda a: np.ascontiguousarray(a, np.float64)
        self._chk(self.L.or_set_raw_state(self.h, f(ro), f(rou), f(rov), f(np.asarray(q).ravel())))

    def state(self):
        n = self.sizes()[1]
        out = np.zeros(13 * n)
        self._chk(self.L.or_get_state(self.h, out))
        out = out.reshape(13, n)
        return {k: out[i].copy() for i, k in enumerate(STATE_FIELDS)}

    def rhs(self):
        n = self.sizes()[1]
        out = np.zeros(7 * n)
        self._chk(self.L.or_calc_all_rhs(self.h, out))
        out = out.reshape(7, n)
        return {k: out[i].copy() for i, k in enumerate(RHS_FIELDS)}

    def set_tstep(self):
        a, b = C.c_double(), C.c_double()
        self._chk(self.L.or_set_tstep(self.h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def step(self, dt, nsteps=1, pid=False):
        self._chk(self.L.or_step(self.h, float(dt), int(nsteps), int(pid)))

    def time(self):
        t, dt, it = C.c_double(), C.c_double(), C.c_int()
        em = np.zeros(3)
        self.L.or_get_time(self.h, C.byref(t), C.byref(dt), C.byref(it), em)
        return dict(time=t.value, dt=dt.value, itime=it.value, emax=em)

    def set_time(self, time, dt, itime, emax):
        self.L.or_set_time(self.h, float(time), float(dt), int(itime), np.ascontiguousarray(emax, np.float64))

    def flow_control(self):
        out = np.zeros(5)
        self.L.or_get_flow_control(self.h, out)
        return dict(eflow_nm1=out[0], sum_eflow=out[1], driving_force=out[2:5].copy())

    def set_flow_control(self, eflow_nm1, sum_eflow, driving_force):
        v = np.array([eflow_nm1, sum_eflow, *np.asarray(driving_force, np.float64)[:3]])
        self.L.or_set_flow_control(self.h, v)

    def kinetic_energy(self):
        return self.L.or_kinetic_energy(self.h)

    def mass(self):
        return self.L.or_mass(self.h)


def for_workload(wl, ns=None, **over):
    """Oracle configured for a nodesets.Workload."""
    kw = wl.params()
    kw.update(over)
    o = Oracle(**kw)
    o.build_domain(ns if ns is not None else wl.nodes())
    return o


STATE3_FIELDS = ["ro", "rou", "rov", "row", "u", "v", "w", "cxx", "cxy", "cyy", "cxz", "cyz", "czz",
                 "psixx", "psixy", "psiyy", "psixz", "psiyz", "psizz"]
RHS3_FIELDS = ["ro", "rou", "rov", "row", "xx", "xy", "yy", "xz", "yz", "zz"]
C3_FIELDS = ["cxx", "cxy", "cyy", "cxz", "cyz", "czz"]


class Oracle3:
    """The 3-D (-Ddim3) run built on a set-up 2-D layer (direct, Cholesky, log-conformation (sPTT)
    and Newtonian forms, FENE-P with the direct and Cholesky forms, node sets without boundary
    nodes or with walls among them).  Arrays are nl*nz, layer-major."""

    def __init__(self, layer: Oracle, Lz: float):
        self.layer = layer
        self.L = layer.L
        self.h = self.L.or3_create(layer.h, float(Lz))
        if not self.h:
            raise OracleError("or3_create: needs weights, walls only among the boundary nodes, "
                              "FENE-P only with the direct and Cholesky forms")
        nl, nz, dz = C.c_int(), C.c_int(), C.c_double()
        self.L.or3_sizes(self.h, C.byref(nl), C.byref(nz), C.byref(dz))
        self.nl, self.nz, self.dz = nl.value, nz.value, dz.value
        self.n = self.nl * self.nz

    def __del__(self):
        if getattr(self, "h", None):
            self.L.or3_destroy(self.h)
            self.h = None

    def set_state(self, ro, u, v, w, cxx=None, cxy=None, cyy=None, cxz=None, cyz=None, czz=None):
        f = lambda a: np.ascontiguousarray(a, np.float64)
        keep = [f(ro), f(u), f(v), f(w)]
        ptr = None
        if cxx is not None:
            cs = [f(a) for a in (cxx, cxy, cyy, cxz, cyz, czz)]
            arr = (C.c_void_p * 6)(*[a.ctypes.data for a in cs])
            keep += cs + [arr]
            ptr = C.cast(arr, C.c_void_p)
        self._keep = keep
        self.L.or3_set_state(self.h, keep[0], keep[1], keep[2], keep[3], ptr)

    def state(self):
        out = np.zeros(19 * self.n)
        self.L.or3_get_state(self.h, out)
        out = out.reshape(19, self.n)
        return {k: out[i].copy() for i, k in enumerate(STATE3_FIELDS)}

    def rhs(self):
        out = np.zeros(10 * self.n)
        self.L.or3_rhs(self.h, out)
        out = out.reshape(10, self.n)
        return {k: out[i].copy() for i, k in enumerate(RHS3_FIELDS)}

    def set_tstep(self):
        a, b = C.c_double(), C.c_double()
        self.L.or3_set_tstep(self.h, C.byref(a), C.byref(b))
        return a.value, b.value

    def step(self, dt, nsteps=1, pid=False):
        self.L.or3_step(self.h, float(dt), int(nsteps), int(pid))

    def time(self):
        t, dt, it = C.c_double(), C.c_double(), C.c_int()
        em = np.zeros(3)
        self.L.or3_get_time(self.h, C.byref(t), C.byref(dt), C.byref(it), em)
        return dict(time=t.value, dt=dt.value, itime=it.value, emax=em)

    def kinetic_energy(self):
        return float(self.L.or3_kinetic_energy(self.h))

    def mass(self):
        return float(self.L.or3_mass(self.h))

    def dump(self):
        """output_layer's 13 columns of every node-layer (layer-major) and the 9 header values."""
        out, hd = np.zeros(13 * self.n), np.zeros(9)
        self.L.or3_get_dump(self.h, out, hd)
        keys = ["ro_minus_rho_char", "u", "v", "w", "vort", "qcrit", "alpha", "cxx", "cxy", "cyy", "cxz", "cyz", "czz"]
        out = out.reshape(13, self.n)
        return {k: out[i].copy() for i, k in enumerate(keys)}, hd
