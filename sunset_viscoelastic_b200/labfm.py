"""Host mirror of the reference's LABFM subroutines over the C-ABI of libsunset_b200.so.

Method names follow the Fortran subroutines they replace (source/base/*.F90 of the
reference); arrays are numpy arrays in the reference's node order.  The class keeps no
numerics of its own: every call goes to the CUDA library, which must be built
(``sunset_viscoelastic_b200.build``) and have a GPU; without either it raises, it does not
fall back to a CPU path.
"""
from __future__ import annotations

import ctypes as C
import os
import warnings

import numpy as np

from . import build as _build

FORMS = {"di": 0, "chl": 1, "lc": 2, "newt": 3}
PRECISION = {"fp64": 0, "mixed": 1}
STATE_FIELDS = ["ro", "rou", "rov", "u", "v", "psixx", "psixy", "psiyy", "psizz", "cxx", "cxy", "cyy", "czz"]
RHS_FIELDS = ["ro", "rou", "rov", "xx", "xy", "yy", "zz"]
# columns of a fields dump (output.F90:299-301)
DUMP_COLUMNS = ["ro_minus_rho_char", "u", "v", "vort", "qcrit", "alpha", "cxx", "cxy", "cyy", "czz"]
# the 3-D dump (output.F90:296-299): every node-layer, layer-major
DUMP_COLUMNS_3D = ["ro_minus_rho_char", "u", "v", "w", "vort", "qcrit", "alpha", "cxx", "cxy", "cyy", "cxz", "cyz",
                   "czz"]
# return codes of include/sunset_gpu.h
ERR_ARG, ERR_CUDA, ERR_SVD, ERR_SCOPE, ERR_NONFINITE, ERR_NOMEM, ERR_ILLCOND = -1, -2, -3, -4, -5, -6, -7

# C-ABI symbols declared in include/sunset_gpu.h
ABI_SYMBOLS = [
    "sunset_version", "sunset_create", "sunset_destroy", "sunset_last_error", "sunset_build_domain",
    "sunset_get_sizes", "sunset_find_neighbours", "sunset_calc_labf_weights", "sunset_calc_boundary_weights",
    "sunset_calc_labf_sums",
    "sunset_filter_coefficients", "sunset_get_neighbours", "sunset_get_weights", "sunset_calc_gradient",
    "sunset_calc_laplacian", "sunset_calc_filtered_var", "sunset_calc_filter_term", "sunset_set_state",
    "sunset_get_state", "sunset_calc_all_rhs", "sunset_set_tstep", "sunset_step", "sunset_get_time",
    "sunset_set_time", "sunset_kinetic_energy", "sunset_mass", "sunset_synchronize", "sunset_run_host",
    "sunset_time_stage_kernel", "sunset_step_timed", "sunset_kinetic_energy_noalloc",
    "sunset_adjoint_run", "sunset_adjoint_apply_D", "sunset_adapt_stencils", "sunset_get_lengths",
    "sunset_set_lengths", "sunset_get_dump", "sunset_write_dump", "sunset_set_restart", "sunset_checkpoint_size",
    "sunset_save_checkpoint", "sunset_load_checkpoint", "sunset_get_flow_control", "sunset_set_flow_control",
    "sunset_set_layers", "sunset_get_layers", "sunset_set_state_3d", "sunset_get_state_3d", "sunset_calc_all_rhs_3d",
    "sunset_get_conditioning", "sunset_kernel_binary_version",
]


class SunsetConfig(C.Structure):
    _fields_ = [("form", C.c_int), ("fenep", C.c_int), ("morder", C.c_int), ("forder", C.c_int),
                ("mcorr", C.c_int), ("kolmogorov_forcing", C.c_int), ("di_full_gradients", C.c_int),
                ("precision", C.c_int), ("L_char", C.c_double), ("U_char", C.c_double), ("Re", C.c_double),
                ("Wi", C.c_double), ("beta", C.c_double), ("epsPTT", C.c_double), ("fenep_l2", C.c_double),
                ("Mdiff", C.c_double), ("Ma", C.c_double), ("grav", C.c_double * 3), ("h_over_s", C.c_double),
                ("device", C.c_int), ("inflow_type", C.c_int), ("inflow_velocity_control", C.c_int),
                ("u_inflow_start", C.c_double), ("u_inflow_end", C.c_double), ("ramp_time", C.c_double),
                ("vpid", C.c_int), ("cond_max", C.c_double), ("svd_max_sweeps", C.c_int)]


class SunsetError(RuntimeError):
    """A negative SUNSET_ERR_* return code; .code holds it (None when not from a call)."""

    def __init__(self, msg, code=None):
        super().__init__(msg)
        self.code = code


_lib = None


def library_path() -> str:
    return _build.LIB


def load_library(build_if_missing: bool = True):
    """Loads libsunset_b200.so (building it first if it is missing and nvcc exists)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(_build.LIB):
        if not build_if_missing:
            raise SunsetError(f"{_build.LIB} is missing; run sunset_viscoelastic_b200.build")
        _build.build()
    L = C.CDLL(_build.LIB)
    P = C.c_void_p
    dp = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
    ip = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
    L.sunset_create.argtypes = [C.POINTER(SunsetConfig), C.POINTER(P)]
    L.sunset_destroy.argtypes = [P]
    L.sunset_last_error.restype = C.c_char_p
    L.sunset_last_error.argtypes = [P]
    L.sunset_build_domain.argtypes = [P, C.c_int, ip, dp, dp, ip, dp, dp, dp, C.c_double, C.c_double, C.c_double,
                                      C.c_double, ip, C.c_double]
    L.sunset_get_sizes.argtypes = [P] + [C.POINTER(C.c_int)] * 4
    for n in ["sunset_find_neighbours", "sunset_calc_labf_weights", "sunset_calc_boundary_weights",
              "sunset_calc_labf_sums", "sunset_filter_coefficients", "sunset_synchronize", "sunset_adapt_stencils"]:
        getattr(L, n).argtypes = [P]
    L.sunset_get_lengths.argtypes = [P, dp, dp]
    L.sunset_set_lengths.argtypes = [P, dp, dp]
    L.sunset_get_dump.argtypes = [P, dp, dp]
    L.sunset_write_dump.argtypes = [P, C.c_char_p, C.c_int, C.c_double]
    L.sunset_set_restart.argtypes = [P, dp, dp]
    L.sunset_get_flow_control.argtypes = [P, dp]
    L.sunset_set_layers.argtypes = [P, C.c_double]
    L.sunset_get_layers.argtypes = [P, C.POINTER(C.c_int), C.POINTER(C.c_double)]
    L.sunset_set_state_3d.argtypes = [P] + [C.c_void_p] * 10
    L.sunset_get_state_3d.argtypes = [P, dp]
    L.sunset_calc_all_rhs_3d.argtypes = [P, dp]
    L.sunset_set_flow_control.argtypes = [P, dp]
    L.sunset_checkpoint_size.argtypes = [P, C.POINTER(C.c_size_t)]
    L.sunset_save_checkpoint.argtypes = [P, C.c_void_p, C.c_size_t]
    L.sunset_load_checkpoint.argtypes = [P, C.c_void_p, C.c_size_t]
    L.sunset_get_neighbours.argtypes = [P, ip, ip, ip]
    L.sunset_get_weights.argtypes = [P, dp, dp, dp, dp, dp, dp, dp]
    L.sunset_get_conditioning.argtypes = [P, C.c_void_p, C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int)]
    L.sunset_kernel_binary_version.argtypes = [C.c_int]
    for n in ["sunset_calc_gradient", "sunset_calc_laplacian", "sunset_calc_filtered_var", "sunset_calc_filter_term"]:
        getattr(L, n).argtypes = [P, dp, dp, C.c_int]
    L.sunset_set_state.argtypes = [P, dp, dp, dp, dp, dp, dp, dp]
    L.sunset_get_state.argtypes = [P, dp]
    L.sunset_calc_all_rhs.argtypes = [P, dp]
    L.sunset_set_tstep.argtypes = [P, C.POINTER(C.c_double), C.POINTER(C.c_double)]
    L.sunset_step.argtypes = [P, C.c_double, C.c_int, C.c_int]
    L.sunset_get_time.argtypes = [P, C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_int), dp]
    L.sunset_set_time.argtypes = [P, C.c_double, C.c_double, C.c_int, dp]
    L.sunset_kinetic_energy.argtypes = [P, C.POINTER(C.c_double)]
    L.sunset_mass.argtypes = [P, C.POINTER(C.c_double)]
    L.sunset_run_host.argtypes = [P, C.c_void_p, C.c_double, C.c_int, C.c_void_p]
    L.sunset_time_stage_kernel.argtypes = [P, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double)]
    L.sunset_adjoint_run.argtypes = [P, C.c_double, C.c_int, C.c_int, C.POINTER(C.c_double), dp, C.c_void_p]
    L.sunset_adjoint_apply_D.argtypes = [P, C.c_int, dp, dp, C.c_int]
    L.sunset_step_timed.argtypes = [P, C.c_double, C.c_int, C.c_int, C.POINTER(C.c_double)]
    L.sunset_kinetic_energy_noalloc.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                                C.c_void_p, C.c_void_p]
    _lib = L
    return L


class Sunset:
    """One LABFM run on one GPU: node set, weights and state, as the reference's module state."""

    def __init__(self, form="di", order=4, forder=None, Re=1.0, Wi=1.0, beta=0.5, epsPTT=0.0, Ma=0.1,
                 fenep=False, fenep_l2=1e30, Mdiff=0.0, grav=(0.0, 0.0, 0.0), mcorr=True, kolmogorov_forcing=-1,
                 di_full_gradients=True, h_over_s=0.0, L_char=1.0, U_char=1.0, precision="fp64", device=0,
                 inflow_type=1, inflow_velocity_control=0, u_inflow_start=0.0, u_inflow_end=1.0, ramp_time=1.0,
                 vpid=False, cond_max=0.0, svd_max_sweeps=0):
        self.L = load_library()
        cfg = SunsetConfig()
        cfg.form = FORMS[form]
        cfg.fenep = int(fenep)
        cfg.morder = order
        cfg.forder = forder if forder else order
        cfg.mcorr = int(mcorr)
        cfg.kolmogorov_forcing = int(kolmogorov_forcing)
        cfg.di_full_gradients = int(di_full_gradients)
        cfg.precision = PRECISION[precision]
        cfg.L_char, cfg.U_char, cfg.Re, cfg.Wi, cfg.beta = L_char, U_char, Re, Wi, beta
        cfg.epsPTT, cfg.fenep_l2, cfg.Mdiff, cfg.Ma = epsPTT, fenep_l2, Mdiff, Ma
        for k in range(3):
            cfg.grav[k] = grav[k]
        cfg.h_over_s = h_over_s
        cfg.device = device
        cfg.inflow_type, cfg.inflow_velocity_control = int(inflow_type), int(inflow_velocity_control)
        cfg.u_inflow_start, cfg.u_inflow_end, cfg.ramp_time = u_inflow_start, u_inflow_end, ramp_time
        cfg.vpid = int(bool(vpid))
        cfg.cond_max, cfg.svd_max_sweeps = float(cond_max), int(svd_max_sweeps)
        self.cfg = cfg
        self.h = C.c_void_p()
        rc = self.L.sunset_create(C.byref(cfg), C.byref(self.h))
        if rc != 0:
            msg = self.L.sunset_last_error(self.h).decode() if self.h else "sunset_create failed"
            self.close()
            raise SunsetError(msg)

    def close(self):
        if getattr(self, "h", None):
            self.L.sunset_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _chk(self, rc):
        if rc != 0:
            raise SunsetError(f"[{rc}] " + self.L.sunset_last_error(self.h).decode(), rc)

    # ---- setup_domain.F90 / neighbours.F90 / labf.F90 ----
    def build_domain(self, ns):
        bc = np.ascontiguousarray(ns.bcond, dtype=np.int32)
        self._chk(self.L.sunset_build_domain(self.h, ns.n, ns.gi, ns.x, ns.y, ns.node_type, ns.nx, ns.ny, ns.s,
                                             ns.xmin, ns.xmax, ns.ymin, ns.ymax, bc, ns.smax))
        return self

    def sizes(self):
        a = [C.c_int() for _ in range(4)]
        self._chk(self.L.sunset_get_sizes(self.h, *[C.byref(x) for x in a]))
        return tuple(x.value for x in a)  # np, npfb, nb, nplink

    def find_neighbours(self):
        self._chk(self.L.sunset_find_neighbours(self.h))

    def calc_labf_weights(self):
        """labf.F90:34-394.  Without a cond_max limit, nodes whose moment matrix is worse
        conditioned than 1e12 are reported by a RuntimeWarning (the reference solves them
        silently); with one, the call fails with SUNSET_ERR_ILLCOND."""
        self._chk(self.L.sunset_calc_labf_weights(self.h))
        _, _, worst, n_ill = self.conditioning(arrays=False)
        if n_ill:
            warnings.warn(f"{n_ill} nodes have moment matrices with condition number above 1e12 "
                          f"(worst {worst:.3g}); their weights carry few correct digits", RuntimeWarning)

    def conditioning(self, arrays=True):
        """(cond_deriv, cond_filter, worst, n_ill): sigma_max/sigma_min of each node's
        derivative and filter moment matrix in reference order (None unless arrays), the
        worst value, and the count above the limit."""
        n = self.sizes()[1]
        cd = np.zeros(n) if arrays else None
        cf = np.zeros(n) if arrays else None
        worst, nill = C.c_double(), C.c_int()
        self._chk(self.L.sunset_get_conditioning(self.h, cd.ctypes.data if arrays else None,
                                                 cf.ctypes.data if arrays else None, C.byref(worst), C.byref(nill)))
        return cd, cf, worst.value, nill.value

    def calc_boundary_weights(self):
        self._chk(self.L.sunset_calc_boundary_weights(self.h))

    def calc_labf_sums(self):
        self._chk(self.L.sunset_calc_labf_sums(self.h))

    def filter_coefficients(self):
        self._chk(self.L.sunset_filter_coefficients(self.h))

    def setup(self):
        """sunset.F90:51-60: find_neighbours, calc_labf_weights, calc_boundary_weights (with
        boundary nodes), calc_labf_sums, filter_coefficients."""
        self.find_neighbours()
        self.calc_labf_weights()
        self.calc_boundary_weights()
        self.calc_labf_sums()
        self.filter_coefficients()
        return self

    def adapt_stencils(self):
        """labf.F90:1079-1721 on the current lists, then the neighbour search again."""
        self._chk(self.L.sunset_adapt_stencils(self.h))

    def lengths(self):
        """(h, h_small) of the npfb nodes in reference order."""
        n = self.sizes()[1]
        h, hs = np.zeros(n), np.zeros(n)
        self._chk(self.L.sunset_get_lengths(self.h, h, hs))
        return h, hs

    def set_lengths(self, h, h_small):
        """Restart: h and h_small of the npfb nodes (reference order), before find_neighbours."""
        f = lambda a: np.ascontiguousarray(a, np.float64)
        self._chk(self.L.sunset_set_lengths(self.h, f(h), f(h_small)))

    def _dump_layout(self):
        nz, _ = self.layers()
        n = self.sizes()[1]
        return (DUMP_COLUMNS_3D, n * nz) if nz > 0 else (DUMP_COLUMNS, n)

    def dump(self):
        """(columns dict of output_layer's columns, header array of 9) in reference order: 10
        columns a node, or on a 3-D handle 13 a node-layer."""
        keys, n = self._dump_layout()
        cols, hd = np.zeros(len(keys) * n), np.zeros(9)
        self._chk(self.L.sunset_get_dump(self.h, cols, hd))
        cols = cols.reshape(len(keys), n)
        return {k: cols[i].copy() for i, k in enumerate(keys)}, hd

    def write_dump(self, directory, n_out, time=0.0):
        self._chk(self.L.sunset_write_dump(self.h, str(directory).encode(), int(n_out), float(time)))

    def set_restart(self, columns, header):
        """load_restart_file from dump columns (dict, or the columns x rows array of dump()) and
        header."""
        if isinstance(columns, dict):
            columns = np.stack([columns[k] for k in self._dump_layout()[0]])
        self._chk(self.L.sunset_set_restart(self.h, np.ascontiguousarray(columns, np.float64).ravel(),
                                            np.ascontiguousarray(header, np.float64)))

    # ---- 3-D (-Ddim3) ----
    def set_layers(self, L_domain_z):
        """build_3rd_dimension: nz layers over L_domain_z; returns (nz, dz)."""
        self._chk(self.L.sunset_set_layers(self.h, float(L_domain_z)))
        return self.layers()

    def layers(self):
        nz, dz = C.c_int(), C.c_double()
        self._chk(self.L.sunset_get_layers(self.h, C.byref(nz), C.byref(dz)))
        return nz.value, dz.value

    def set_state_3d(self, ro, u, v, w, cxx=None, cxy=None, cyy=None, cxz=None, cyz=None, czz=None):
        arrs = [np.ascontiguousarray(a, np.float64) if a is not None else None
                for a in (ro, u, v, w, cxx, cxy, cyy, cxz, cyz, czz)]
        self._keep3 = arrs
        ptrs = [a.ctypes.data if a is not None else None for a in arrs]
        self._chk(self.L.sunset_set_state_3d(self.h, *ptrs))

    def state_3d(self):
        nz, _ = self.layers()
        n = self.sizes()[1] * nz
        out = np.zeros(19 * n)
        self._chk(self.L.sunset_get_state_3d(self.h, out))
        out = out.reshape(19, n)
        keys = ["ro", "rou", "rov", "row", "u", "v", "w", "cxx", "cxy", "cyy", "cxz", "cyz", "czz",
                "psixx", "psixy", "psiyy", "psixz", "psiyz", "psizz"]
        return {k: out[i].copy() for i, k in enumerate(keys)}

    def rhs_3d(self):
        nz, _ = self.layers()
        n = self.sizes()[1] * nz
        out = np.zeros(10 * n)
        self._chk(self.L.sunset_calc_all_rhs_3d(self.h, out))
        out = out.reshape(10, n)
        keys = ["ro", "rou", "rov", "row", "xx", "xy", "yy", "xz", "yz", "zz"]
        return {k: out[i].copy() for i, k in enumerate(keys)}

    def flow_control(self):
        """The flow-rate controller's state: eflow_nm1, sum_eflow, driving_force(1:3)."""
        out = np.zeros(5)
        self._chk(self.L.sunset_get_flow_control(self.h, out))
        return dict(eflow_nm1=out[0], sum_eflow=out[1], driving_force=out[2:5].copy())

    def set_flow_control(self, eflow_nm1, sum_eflow, driving_force):
        v = np.array([eflow_nm1, sum_eflow, *np.asarray(driving_force, np.float64)[:3]])
        self._chk(self.L.sunset_set_flow_control(self.h, v))

    def save_checkpoint(self):
        """The device state between steps, bit for bit, as bytes."""
        nb = C.c_size_t()
        self._chk(self.L.sunset_checkpoint_size(self.h, C.byref(nb)))
        buf = C.create_string_buffer(nb.value)
        self._chk(self.L.sunset_save_checkpoint(self.h, buf, nb.value))
        return buf.raw

    def load_checkpoint(self, data):
        buf = C.create_string_buffer(data, len(data))
        self._chk(self.L.sunset_load_checkpoint(self.h, buf, len(data)))

    def neighbours(self):
        _, npfb, _, nplink = self.sizes()
        cnt = np.zeros(npfb, np.int32)
        cs = np.zeros(npfb, np.int32)
        lk = np.zeros(npfb * nplink, np.int32)
        self._chk(self.L.sunset_get_neighbours(self.h, cnt, cs, lk))
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
        self._chk(self.L.sunset_get_weights(self.h, wg, wl, wh, gs, ls, hs, vol))
        return dict(w_grad=wg.reshape(npfb, nplink, 2), w_lap=wl.reshape(npfb, nplink),
                    w_hyp=wh.reshape(npfb, nplink), w_grad_sum=gs.reshape(npfb, 2), w_lap_sum=ls,
                    w_hyp_sum=hs, vol=vol)

    # ---- derivatives.F90 ----
    def gradient(self, phi):
        n = self.sizes()[1]
        out = np.zeros(2 * n)
        self._chk(self.L.sunset_calc_gradient(self.h, np.ascontiguousarray(phi, np.float64), out, 0))
        return out.reshape(n, 2)

    def laplacian(self, phi):
        out = np.zeros(self.sizes()[1])
        self._chk(self.L.sunset_calc_laplacian(self.h, np.ascontiguousarray(phi, np.float64), out, 0))
        return out

    def filtered(self, phi):
        out = np.zeros(self.sizes()[1])
        self._chk(self.L.sunset_calc_filtered_var(self.h, np.ascontiguousarray(phi, np.float64), out, 0))
        return out

    def filter_term(self, phi):
        out = np.zeros(self.sizes()[1])
        self._chk(self.L.sunset_calc_filter_term(self.h, np.ascontiguousarray(phi, np.float64), out, 0))
        return out

    calc_gradient = gradient
    calc_laplacian = laplacian
    calc_filtered_var = filtered
    calc_filter_term = filter_term

    # ---- setup_flow.F90 / rhs_*.F90 / step.F90 ----
    def set_state(self, ro, u, v, cxx, cxy, cyy, czz=None):
        n = self.sizes()[1]
        f = lambda a: np.ascontiguousarray(a, np.float64)
        czz = np.ones(n) if czz is None else czz
        self._chk(self.L.sunset_set_state(self.h, f(ro), f(u), f(v), f(cxx), f(cxy), f(cyy), f(czz)))

    def state(self):
        n = self.sizes()[1]
        out = np.zeros(13 * n)
        self._chk(self.L.sunset_get_state(self.h, out))
        out = out.reshape(13, n)
        return {k: out[i].copy() for i, k in enumerate(STATE_FIELDS)}

    def rhs(self):
        n = self.sizes()[1]
        out = np.zeros(7 * n)
        self._chk(self.L.sunset_calc_all_rhs(self.h, out))
        out = out.reshape(7, n)
        return {k: out[i].copy() for i, k in enumerate(RHS_FIELDS)}

    calc_all_rhs = rhs

    def set_tstep(self):
        a, b = C.c_double(), C.c_double()
        self._chk(self.L.sunset_set_tstep(self.h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def step(self, dt, nsteps=1, pid=False):
        """step_rk3_4S_2R_EE nsteps times (fixed dt, or set_tstep + set_tstep_PID per step)."""
        self._chk(self.L.sunset_step(self.h, float(dt), int(nsteps), int(pid)))

    step_rk3_4S_2R_EE = step

    def step_timed(self, dt, nsteps=1, pid=False):
        """As step(); returns the device time of the steps in ms (CUDA events on the
        library's stream)."""
        ms = C.c_double()
        self._chk(self.L.sunset_step_timed(self.h, float(dt), int(nsteps), int(pid), C.byref(ms)))
        return ms.value

    def time(self):
        t, dt, it = C.c_double(), C.c_double(), C.c_int()
        em = np.zeros(3)
        self._chk(self.L.sunset_get_time(self.h, C.byref(t), C.byref(dt), C.byref(it), em))
        return dict(time=t.value, dt=dt.value, itime=it.value, emax=em)

    def set_time(self, time, dt, itime, emax):
        self._chk(self.L.sunset_set_time(self.h, float(time), float(dt), int(itime),
                                         np.ascontiguousarray(emax, np.float64)))

    def kinetic_energy(self):
        x = C.c_double()
        self._chk(self.L.sunset_kinetic_energy(self.h, C.byref(x)))
        return x.value

    def mass(self):
        x = C.c_double()
        self._chk(self.L.sunset_mass(self.h, C.byref(x)))
        return x.value

    def synchronize(self):
        self._chk(self.L.sunset_synchronize(self.h))

    def run_host(self, state_in_ptr, dt, nsteps, state_out_ptr):
        """Host-buffer round trip (7*npfb doubles in and out, or 10*npfb*nz on a 3-D handle;
        pointers to pinned memory)."""
        self._chk(self.L.sunset_run_host(self.h, C.c_void_p(state_in_ptr), float(dt), int(nsteps),
                                         C.c_void_p(state_out_ptr)))

    # ---- adjoint (no reference counterpart) ----
    def adjoint_run(self, dt, nsteps, checkpoint_every=20, state_gradient=True):
        """From the current state: J = final kinetic energy after nsteps steps of dt, and
        (dJ/dWi, dJ/dbeta), and dJ/d(initial state) as a dict of 7 fields (ro rou rov
        psixx psixy psiyy psizz), or None."""
        J = C.c_double()
        dp_ = np.zeros(2)
        n = self.sizes()[1]
        ds = np.zeros(7 * n) if state_gradient else None
        self._chk(self.L.sunset_adjoint_run(self.h, float(dt), int(nsteps), int(checkpoint_every), C.byref(J), dp_,
                                            ds.ctypes.data if ds is not None else None))
        grads = None
        if ds is not None:
            grads = {k: ds[f * n:(f + 1) * n].copy() for f, k in
                     enumerate(["ro", "rou", "rov", "psixx", "psixy", "psiyy", "psizz"])}
        return J.value, (dp_[0], dp_[1]), grads

    def adjoint_apply_D(self, which, gbar):
        out = np.zeros(self.sizes()[1])
        self._chk(self.L.sunset_adjoint_apply_D(self.h, int(which), np.ascontiguousarray(gbar, np.float64), out, 0))
        return out

    def time_stage_kernel(self, reps=20):
        """(mean ms per RK stage launch inside `reps` real steps, algorithmic bytes per launch);
        advances the state by reps steps."""
        ms, by = C.c_double(), C.c_double()
        self._chk(self.L.sunset_time_stage_kernel(self.h, int(reps), C.byref(ms), C.byref(by)))
        return ms.value, by.value


def kinetic_energy_noalloc(device, npfb, ro_ptr, u_ptr, v_ptr, vol_ptr, out_ptr, stream_ptr=None):
    """sunset_kinetic_energy_noalloc on device arrays the caller owns (raw device pointers);
    out receives (kinetic energy, mass).  Allocates nothing on the device."""
    rc = load_library().sunset_kinetic_energy_noalloc(int(device), int(npfb), C.c_void_p(ro_ptr), C.c_void_p(u_ptr),
                                                      C.c_void_p(v_ptr), C.c_void_p(vol_ptr), C.c_void_p(out_ptr),
                                                      C.c_void_p(stream_ptr) if stream_ptr else None)
    if rc != 0:
        raise SunsetError(f"sunset_kinetic_energy_noalloc failed with code {rc}", rc)


def for_workload(wl, ns=None, precision="fp64", device=0, **over):
    kw = dict(wl.params(), precision=precision, device=device)
    kw.update(over)
    s = Sunset(**kw)
    s.build_domain(ns if ns is not None else wl.nodes())
    return s
