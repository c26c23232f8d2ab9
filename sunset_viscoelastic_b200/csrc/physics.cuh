// physics.cuh -- pointwise right-hand sides of the viscoelastic equations on one node
// (2-D, interior nodes), restated from rhs_di.F90, rhs.F90 (Cholesky) and rhs_lc.F90,
// and the conformation transforms of conf_transforms.F90.  Expressions keep the
// reference's left-to-right order; zero third components are kept as the literal
// "+ 0.0" terms so signed zeros match the reference's too.
#pragma once

#include "internal.cuh"

namespace sunset {

// Stencil results the right-hand sides read.
struct Grads {
    double ro_x, ro_y, u_x, u_y, v_x, v_y, lapu, lapv;
    double cxx_x, cxx_y, cxy_x, cxy_y, cyy_x, cyy_y;              // DI, LC (momentum)
    double pxx_x, pxx_y, pxy_x, pxy_y, pyy_x, pyy_y;              // LC, CHL
    double lapcxx, lapcxy, lapcyy, lapczz;                        // polymer diffusion
    double f_x, f_y;                                              // FENE-P function (DI, LC)
    double pzz_x, pzz_y;                                          // CHL, FENE-P
};

struct NodeState {
    double ro, u, v, y;                 // y: node ordinate (Kolmogorov forcing)
    double cxx, cxy, cyy, czz;          // conformation tensor
    double pxx, pxy, pyy, pzz;          // psi (LC/CHL)
    double f;                           // FENE-P function (L^2 - 3) / (L^2 - tr c)
    double df;                          // driving_force(1) of the flow-rate controller
};

// The FENE-P function fenepf (rhs_di.F90:201-203, rhs.F90:207-209, rhs_lc.F90:201-203).
__host__ __device__ __forceinline__ double fenep_f(double L2, double cxx, double cyy, double czz) {
    return (L2 - 3.0) / (L2 - ((cxx + cyy) + czz));
}

struct Rhs {
    double ro, rou, rov, xx, xy, yy, zz;
};

// conf_transforms.F90:399-444, 2x2 eigen-decomposition; R column-major.
__host__ __device__ __forceinline__ void eigens2(double a, double b, double d, double *l, double *R) {
    if (fabs(b) <= 1.0e-16) {
        l[0] = a; l[1] = d;
        R[0] = 1.0; R[1] = 0.0; R[2] = 0.0; R[3] = 1.0;
    } else {
        double tr = a + d;
        double det = a * d - b * b;
        double temp = (0.25 * tr) * tr - det;
        if (temp <= 1.0e-16) temp = 0.0;
        temp = sqrt(temp);
        l[0] = 0.5 * tr + temp;
        l[1] = 0.5 * tr - temp;
        R[0] = l[0] - d;
        R[1] = b;
        temp = sqrt(R[0] * R[0] + R[1] * R[1]);
        R[0] = R[0] / temp;
        R[1] = R[1] / temp;
        R[2] = -R[1];
        R[3] = R[0];
    }
}
// gfortran inline matmul order: c(i,j) = a(i,1) b(1,j) + a(i,2) b(2,j)
__host__ __device__ __forceinline__ void mm2(const double *a, const double *b, double *c) {
    double t0 = a[0] * b[0] + a[2] * b[1];
    double t1 = a[1] * b[0] + a[3] * b[1];
    double t2 = a[0] * b[2] + a[2] * b[3];
    double t3 = a[1] * b[2] + a[3] * b[3];
    c[0] = t0; c[1] = t1; c[2] = t2; c[3] = t3;
}
__host__ __device__ __forceinline__ void tr2(const double *a, double *t) { t[0] = a[0]; t[1] = a[2]; t[2] = a[1]; t[3] = a[3]; }

// log_conf_c_from_psi, conf_transforms.F90:133-169
__host__ __device__ __forceinline__ void lc_c_from_psi(double pxx, double pxy, double pyy, double *cxx, double *cxy,
                                              double *cyy) {
    double L[2], R[4], RT[4], Lm[4], C[4];
    eigens2(pxx, pxy, pyy, L, R);
    tr2(R, RT);
    Lm[0] = exp(L[0]); Lm[1] = 0.0; Lm[2] = 0.0; Lm[3] = exp(L[1]);
    mm2(Lm, RT, C);
    mm2(R, C, C);
    *cxx = C[0]; *cxy = C[1]; *cyy = C[3];
}
// log_conf_psi_from_c, conf_transforms.F90:177-215
__host__ __device__ __forceinline__ void lc_psi_from_c(double cxx, double cxy, double cyy, double *pxx, double *pxy,
                                              double *pyy) {
    double L[2], R[4], RT[4], Lm[4], P[4];
    eigens2(cxx, cxy, cyy, L, R);
    tr2(R, RT);
    Lm[0] = log(L[0]); Lm[1] = 0.0; Lm[2] = 0.0; Lm[3] = log(L[1]);
    mm2(Lm, RT, P);
    mm2(R, P, P);
    *pxx = P[0]; *pxy = P[1]; *pyy = P[3];
}
// cholesky_c_from_psi (sPTT), conf_transforms.F90:60-70
__host__ __device__ __forceinline__ void chl_c_from_psi(double pxx, double pxy, double pyy, double *cxx, double *cxy,
                                               double *cyy, double *czz) {
    double e = exp(pxx);
    *cxx = e * e;
    *cxy = exp(pxx) * pxy;
    *cyy = pxy * pxy + exp(2.0 * pyy);
    *czz = 1.0;
}
// cholesky_c_from_psi (FENE-P), conf_transforms.F90:39-55: psi holds the Cholesky factor of
// J = f c, and c = J L^2 / (L^2 - 3 + tr J).
__host__ __device__ __forceinline__ void chl_c_from_psi_fenep(double L2, double pxx, double pxy, double pyy, double pzz,
                                                     double *cxx, double *cxy, double *cyy, double *czz) {
    const double Jxx = exp(2.0 * pxx), Jxy = exp(pxx) * pxy, Jyy = pxy * pxy + exp(2.0 * pyy);
    const double Jzz = exp(2.0 * pzz);
    const double fq = L2 / ((((L2 - 3.0) + Jxx) + Jyy) + Jzz);
    *cxx = Jxx * fq; *cxy = Jxy * fq; *cyy = Jyy * fq; *czz = Jzz * fq;
}
// cholesky_psi_from_c (sPTT), conf_transforms.F90:109-121
__host__ __device__ __forceinline__ void chl_psi_from_c(double cxx, double cxy, double cyy, double czz, double *pxx,
                                               double *pxy, double *pyy, double *pzz) {
    double xx = sqrt(cxx);
    double xy = cxy / (xx);
    double yy = (sqrt(cyy - xy * xy));
    double zz = sqrt(czz);
    *pxx = log(xx); *pxy = xy; *pyy = log(yy); *pzz = log(zz);
}
// cholesky_psi_from_c (FENE-P), conf_transforms.F90:89-101
__host__ __device__ __forceinline__ void chl_psi_from_c_fenep(double L2, double cxx, double cxy, double cyy, double czz,
                                                     double *pxx, double *pxy, double *pyy, double *pzz) {
    const double fr = (L2 - 3.0) / (L2 - ((cxx + cyy) + czz));
    const double Jxx = cxx * fr, Jxy = cxy * fr, Jyy = cyy * fr, Jzz = czz * fr;
    const double xx = sqrt(Jxx);
    const double xy = Jxy / xx;
    const double yy = sqrt(Jyy - xy * xy);
    const double zz = sqrt(Jzz);
    *pxx = log(xx); *pxy = xy; *pyy = log(yy); *pzz = log(zz);
}
// The conversions around the filter of the Cholesky FENE-P form (rhs.F90:815-869): the
// factor of J = f c to the factor of c before filtering, and back after it.
__host__ __device__ __forceinline__ void chl_fenep_to_c_factor(double L2, double &pxx, double &pxy, double &pyy,
                                                      double &pzz) {
    double fr = ((exp(2.0 * pxx) + pxy * pxy) + exp(2.0 * pyy)) + exp(2.0 * pzz);
    fr = (L2 * fr) / ((L2 - 3.0) + fr);
    fr = (L2 - 3.0) / (L2 - fr);
    pxx = pxx - log(sqrt(fr));
    pxy = pxy / sqrt(fr);
    pyy = pyy - log(sqrt(fr));
    pzz = pzz - log(sqrt(fr));
}
__host__ __device__ __forceinline__ void chl_fenep_to_j_factor(double L2, double &pxx, double &pxy, double &pyy,
                                                      double &pzz) {
    const double fr = (L2 - 3.0) / (L2 - (((exp(2.0 * pxx) + pxy * pxy) + exp(2.0 * pyy)) + exp(2.0 * pzz)));
    pxx = pxx + log(sqrt(fr));
    pxy = pxy * sqrt(fr);
    pyy = pyy + log(sqrt(fr));
    pzz = pzz + log(sqrt(fr));
}

// calc_rhs_ro + calc_rhs_rovel, interior branch (rhs_di.F90:126-141,215-275; rhs.F90:220-286;
// rhs_lc.F90:215-275).
// The stress divergence f_visc: solvent Laplacian plus the polymeric term of each form.
__host__ __device__ __forceinline__ void viscous_force(const StepConsts &K, const NodeState &n, const Grads &g,
                                                       double &fvu, double &fvv) {
    fvu = K.coef_solvent * g.lapu;
    fvv = K.coef_solvent * g.lapv;
    if (K.form == SUNSET_FORM_CHL) {
        double gcxx1 = (2.0 * exp(2.0 * n.pxx)) * g.pxx_x;
        double gcxy1 = exp(n.pxx) * g.pxy_x + (n.pxy * exp(n.pxx)) * g.pxx_x;
        double gcxy2 = exp(n.pxx) * g.pxy_y + (n.pxy * exp(n.pxx)) * g.pxx_y;
        double gcyy2 = (2.0 * n.pxy) * g.pxy_y + (2.0 * exp(2.0 * n.pyy)) * g.pyy_y;
        fvu = fvu + K.coef_polymeric * ((gcxx1 + gcxy2) + 0.0);
        fvv = fvv + K.coef_polymeric * ((gcxy1 + gcyy2) + 0.0);
    } else if (K.form != SUNSET_FORM_NEWT && K.fenep) {  // rhs_di.F90:234-245, rhs_lc.F90:234-245
        const double f1 = n.f;
        fvu = fvu + K.coef_polymeric * (((((g.cxx_x * f1 + n.cxx * g.f_x) + g.cxy_y * f1) + n.cxy * g.f_y) + 0.0 * f1) + 0.0 * 0.0);
        fvv = fvv + K.coef_polymeric * (((((g.cxy_x * f1 + n.cxy * g.f_x) + g.cyy_y * f1) + n.cyy * g.f_y) + 0.0 * f1) + 0.0 * 0.0);
    } else if (K.form != SUNSET_FORM_NEWT) {
        fvu = fvu + K.coef_polymeric * ((g.cxx_x + g.cxy_y) + 0.0);
        fvv = fvv + K.coef_polymeric * ((g.cxy_x + g.cyy_y) + 0.0);
    }
}

__host__ __device__ __forceinline__ void rhs_flow(const StepConsts &K, const NodeState &n, const Grads &g, Rhs &r) {
    const double w = 0.0;
    double tmp_scal = (n.u * g.ro_x + n.v * g.ro_y) + w * 0.0;
    double divvel = (g.u_x + g.v_y) + 0.0;
    r.ro = -n.ro * divvel - tmp_scal;
    double tsu = n.ro * ((n.u * g.u_x + n.v * g.u_y) + w * 0.0) - n.u * r.ro;
    double tsv = n.ro * ((n.u * g.v_x + n.v * g.v_y) + w * 0.0) - n.v * r.ro;
    double fvu, fvv;
    viscous_force(K, n, g, fvu, fvv);
    double bfu = n.ro * (K.grav0 + n.df), bfv = n.ro * (K.grav1 + 0.0);
    if (K.kolmo)
        bfu = bfu + (((1.0 / K.Re) * cos(n.y)) * (1.0 + (K.Mdiff * K.beta) * K.Wi)) / (1.0 + K.Mdiff * K.Wi);
    r.rou = ((-tsu - K.csq * g.ro_x) + bfu) + fvu;
    r.rov = ((-tsv - K.csq * g.ro_y) + bfv) + fvv;
}

// Walls (node_type 0).  Wall nodes' first-derivative weights are in the wall's
// normal-tangent frame, so there g.*_x is the normal and g.*_y the tangential derivative.
// wall_velocity_gradient: the rotated velocity gradient the conformation equations use on
// walls (rhs_di.F90:497-512, rhs.F90 and rhs_lc.F90 alike).
__host__ __device__ __forceinline__ Grads wall_velocity_gradient(const Grads &g, double xn, double yn) {
    Grads w = g;
    w.u_x = xn * g.u_x - yn * g.u_y;
    w.v_x = xn * g.v_x - yn * g.v_y;
    w.u_y = yn * g.u_x + xn * g.u_y;
    w.v_y = yn * g.v_x + xn * g.v_y;
    return w;
}

// Mass and momentum on a wall: calc_rhs_ro wall branch (rhs_di.F90:146-158), the
// characteristic amplitudes of calc_rhs_rovel (:291-309; the momentum right-hand side is
// zero), specify_characteristics_isothermal_wall (characteristic_boundaries.F90:27-52,
// acoustic reflection L5 = L1) and calc_rhs_nscbc (rhs_di.F90:601-665).
__host__ __device__ __forceinline__ void rhs_flow_wall(const StepConsts &K, const NodeState &n, const Grads &g, double xn,
                                              double yn, Rhs &r) {
    const double c = K.c_sound;
    const double dutdt = -yn * g.u_y + xn * g.v_y;
    r.ro = -n.ro * dutdt - n.ro * 0.0;
    const double dpdn = K.csq * g.ro_x;
    const double un = n.u * xn + n.v * yn;
    const double dundn = xn * g.u_x + yn * g.v_x;
    const double dutdn = -yn * g.u_x + xn * g.v_x;
    const double L1 = (0.5 * (un - c)) * (dpdn - (n.ro * c) * dundn);
    const double L2 = un * (g.ro_x - (dpdn / c) / c);
    const double L3 = un * dutdn;
    const double L5 = L1;
    const double tmp_scal = ((((c * c) * L2 + L5) + L1) / c) / c;
    r.ro = r.ro - tmp_scal;
    r.rou = (0.0 - n.u * tmp_scal) - (L5 - L1) / c;
    r.rov = (0.0 - n.v * tmp_scal) - n.ro * L3;
}

// Inflow (node_type 1) and outflow (node_type 2) nodes, in the x-y frame (the outflow's
// first-derivative weights are reversed at set-up, labf.F90:986-991, so g.*_x is d/dx on
// both): calc_rhs_ro's in/out branch (rhs_di.F90:155-157), the characteristic amplitudes and
// the transverse, viscous and body-force terms of calc_rhs_rovel (:311-359; no Kolmogorov
// forcing there), the closure of characteristic_boundaries.F90 for the node's type -- soft
// inflow :54-80, hard inflow :82-110, pressure-tracking inflow-outflow :112-150, partially
// non-reflecting outflow :152-189 -- and the update of calc_rhs_nscbc (rhs_di.F90:601-665).
// uin: the node's u_inflow_local.  rhs.F90 and rhs_lc.F90 have the same branches.
__host__ __device__ __forceinline__ void rhs_flow_inout(const StepConsts &K, const NodeState &n, const Grads &g,
                                                        int type, double uin, Rhs &r) {
    const double w = 0.0;
    const double c = K.c_sound, ro = n.ro, u = n.u, v = n.v;
    r.ro = ((-v * g.ro_y - ro * g.v_y) - w * 0.0) - ro * 0.0;
    const double gp_x = K.csq * g.ro_x, gp_y = K.csq * g.ro_y, p = K.csq * ro;
    const double dpdn = gp_x;
    double L1 = (0.5 * (u - c)) * (dpdn - (ro * c) * g.u_x);
    double L2 = u * (g.ro_x - (gp_x / c) / c);
    double L3 = u * g.v_x;
    double L5 = (0.5 * (u + c)) * (dpdn + (ro * c) * g.u_x);
    double fvu, fvv;
    viscous_force(K, n, g, fvu, fvv);
    const double bfu = ro * (K.grav0 + n.df), bfv = ro * (K.grav1 + 0.0);
    const double rou = ((-(v * g.u_y) - w * 0.0) + fvu) + bfu;
    const double rov = (((-(v * g.v_y) - w * 0.0) - gp_y) + fvv) + bfv;
    const double nscbc = K.nscbc, Lx = K.Lx;
    if (type == 1) {
        if (K.inflow_type == 1) {  // hard inflow
            L2 = 0.0; L3 = 0.0; L5 = L1;
        } else if (K.inflow_type == 2) {  // inflow-outflow
            if (u > 0.0) {
                L2 = 0.0;
                L3 = ((v * nscbc) * c) / Lx;
                L5 = ((((((u - uin) * nscbc) * (1.0 - u / c)) * c) * c) * 1.0) / Lx;
            } else {
                L2 = 0.0;
                L5 = (((((p - K.p_in) * nscbc) * c) * 1.0) / 2.0) / Lx;
            }
        } else {  // soft inflow (its L4, of w, has no effect in 2-D)
            L2 = 0.0;
            L3 = (((((v * nscbc) * c) / Lx) - v * g.v_y) - w * 0.0) - gp_y / ro;
            L5 = (((((((u - uin) * nscbc) * (1.0 - u / c)) * c) * c) * 1.0) / Lx -
                  0.5 * (((v * gp_y) + (p * g.v_y)) + (((ro * c) * v) * g.u_y))) -
                 0.5 * (((w * 0.0) + (p * 0.0)) + (((ro * c) * w) * 0.0));
        }
    } else {  // outflow
        if (u < c) L1 = (((((p - K.p_out) * nscbc) * c) * 1.0) / 2.0) / Lx;
        L2 = 0.0;
        if (u <= 0.0) { L2 = 0.0; L3 = 0.0; }
    }
    const double tmp_scal = ((((c * c) * L2 + L5) + L1) / c) / c;
    r.ro = r.ro - tmp_scal;
    r.rou = (rou - u * tmp_scal) - (L5 - L1) / c;
    r.rov = (rov - v * tmp_scal) - ro * L3;
}

// u_inflow_local at time t (update_u_inflow, characteristic_boundaries.F90:262-300): with
// velocity control, the ramp from u_inflow_start to u_inflow_end while t <= ramp_time; the
// value is left as it is after that (and always without control).
__host__ __device__ __forceinline__ double inflow_velocity(const StepConsts &K, double t, double uin) {
    if (K.inflow_control != 1) return uin;
    if (t <= K.ramp_time) return K.u_in_start + ((K.u_in_end - K.u_in_start) * t) / K.ramp_time;
    return uin;
}

// calc_rhs_c, interior branch, rhs_di.F90:415-476 (sPTT / Oldroyd-B, 2-D); on walls
// (rhs_di.F90:490-580) without advection, with the rotated velocity gradient, and rhs_zz
// left at zero.
__host__ __device__ __forceinline__ void rhs_c_di(const StepConsts &K, const NodeState &n, const Grads &g, Rhs &r,
                                         bool wall = false) {
    const double w = 0.0;
    const double cxx = n.cxx, cxy = n.cxy, cyy = n.cyy, czz = n.czz;
    double adxx = -((n.u * g.cxx_x + n.v * g.cxx_y) + w * 0.0);
    double adxy = -((n.u * g.cxy_x + n.v * g.cxy_y) + w * 0.0);
    double adyy = -((n.u * g.cyy_x + n.v * g.cyy_y) + w * 0.0);
    double adzz = -((n.u * 0.0 + n.v * 0.0) + w * 0.0);
    double g11 = g.u_x, g12 = g.u_y, g21 = g.v_x, g22 = g.v_y;
    double ucxx = ((2.0 * g11) * cxx + (2.0 * g12) * cxy) + (2.0 * 0.0) * 0.0;
    double ucxy = (((((g11 * cxy + g12 * cyy) + 0.0 * 0.0) + g21 * cxx) + g22 * cxy) + 0.0 * 0.0);
    double ucyy = ((2.0 * g21) * cxy + (2.0 * g22) * cyy) + (2.0 * 0.0) * 0.0;
    double uczz = ((2.0 * 0.0) * 0.0 + (2.0 * 0.0) * 0.0) + (2.0 * 0.0) * czz;
    double sxx, sxy, syy, szz;
    if (K.fenep) {  // rhs_di.F90:444-449
        const double fr = -n.f;
        sxx = (fr * cxx + 1.0) / K.lambda;
        sxy = (fr * cxy) / K.lambda;
        syy = (fr * cyy + 1.0) / K.lambda;
        szz = (fr * czz + 1.0) / K.lambda;
    } else {
        const double fr = -(((1.0 - K.epsPTT * 2.0) + K.epsPTT * ((cxx + cyy) + czz))) / K.lambda;
        sxx = fr * (cxx - 1.0); sxy = fr * cxy; syy = fr * (cyy - 1.0); szz = fr * (czz - 1.0);
    }
    if (wall) {
        r.xx = (ucxx + sxx) + K.Mdiff * g.lapcxx;
        r.xy = (ucxy + sxy) + K.Mdiff * g.lapcxy;
        r.yy = (ucyy + syy) + K.Mdiff * g.lapcyy;
        r.zz = 0.0;
        return;
    }
    r.xx = ((adxx + ucxx) + sxx) + K.Mdiff * g.lapcxx;
    r.xy = ((adxy + ucxy) + sxy) + K.Mdiff * g.lapcxy;
    r.yy = ((adyy + ucyy) + syy) + K.Mdiff * g.lapcyy;
    r.zz = ((adzz + uczz) + szz) + K.Mdiff * g.lapczz;
}

// calc_rhs_cholesky, interior branch, rhs.F90:424-550 (sPTT, 2-D).
// FAST (the mixed step only): the divisions by the factors' diagonal become products with
// their reciprocals, computed once; the FP64 step keeps the reference's operations.
template <bool FAST = false>
__host__ __device__ __forceinline__ void rhs_c_chl(const StepConsts &K, const NodeState &n, const Grads &g, Rhs &r) {
    const double w = 0.0;
    double adxx = (n.u * g.pxx_x + n.v * g.pxx_y) + w * 0.0;
    double adxy = (n.u * g.pxy_x + n.v * g.pxy_y) + w * 0.0;
    double adyy = (n.u * g.pyy_x + n.v * g.pyy_y) + w * 0.0;
    double lxx = exp(n.pxx), lxy = n.pxy, lyy = exp(n.pyy);
    double g11 = g.u_x, g12 = g.u_y, g21 = g.v_x, g22 = g.v_y;
    double ucxx, ucxy, ucyy;
    const double ilxx = FAST ? 1.0 / lxx : 0.0, ilyy = FAST ? 1.0 / lyy : 0.0;
    if (FAST) {
        const double t = (g12 * lxy) * ilxx;
        ucxx = g11 + t;
        ucxy = (g22 * lxy + ((g12 * lyy) * lyy) * ilxx) + g21 * lxx;
        ucyy = g22 - t;
    } else {
        ucxx = (g11 + (g12 * lxy) / lxx);
        ucxy = ((g22 * lxy + ((g12 * lyy) * lyy) / lxx) + g21 * lxx);
        ucyy = (g22 - (g12 * lxy) / lxx);
    }
    const double cxx = n.cxx, cxy = n.cxy, cyy = n.cyy, czz = n.czz;
    double sxx, sxy, syy, szz = 0.0;
    if (K.fenep) {  // rhs.F90:480-495: psi factors J = f c
        const double fr = n.f, L2 = K.fenep_l2, lam = K.lambda;
        const double srctmp = ((((((2.0 * g11) * cxx + (2.0 * g12) * cxy) + (2.0 * g21) * cxy) + (2.0 * g22) * cyy) -
                                (((fr * cxx + fr * cyy) + fr * czz) - 3.0) / lam) +
                               K.Mdiff * ((g.lapcxx + g.lapcyy) + g.lapczz));
        const double den = ((L2 - cxx) - cyy) - czz;
        sxx = (-(fr / lam) * (fr * cxx - 1.0) + (K.Mdiff * fr) * g.lapcxx) + ((fr * cxx) * srctmp) / den;
        sxy = (-(fr / lam) * (fr * cxy) + (K.Mdiff * fr) * g.lapcxy) + ((fr * cxy) * srctmp) / den;
        syy = (-(fr / lam) * (fr * cyy - 1.0) + (K.Mdiff * fr) * g.lapcyy) + ((fr * cyy) * srctmp) / den;
        szz = (-(fr / lam) * (fr * czz - 1.0) + (K.Mdiff * fr) * g.lapczz) + ((fr * czz) * srctmp) / den;
    } else {
        const double fr = -(((1.0 - K.epsPTT * 3.0) + K.epsPTT * ((cxx + cyy) + czz))) / K.lambda;
        sxx = fr * (cxx - 1.0) + K.Mdiff * g.lapcxx;
        sxy = fr * cxy + K.Mdiff * g.lapcxy;
        syy = fr * (cyy - 1.0) + K.Mdiff * g.lapcyy;
    }
    double csxx, csxy, csyy;
    if (FAST) {
        const double ixx2 = ilxx * ilxx, iyy2 = ilyy * ilyy;
        csxx = (0.5 * sxx) * ixx2;
        csxy = sxy * ilxx - ((0.5 * sxx) * lxy) * ixx2;
        csyy = ((0.5 * syy) * iyy2 - (sxy * lxy) * (ilxx * iyy2)) + (((0.5 * sxx) * lxy) * lxy) * (iyy2 * ixx2);
    } else {
        csxx = ((0.5 * sxx) / lxx) / lxx;
        csxy = sxy / lxx - ((0.5 * sxx) * lxy) / (lxx * lxx);
        csyy = (((0.5 * syy) / lyy) / lyy - (sxy * lxy) / ((lxx * lyy) * lyy)) +
               (((0.5 * sxx) * lxy) * lxy) / ((lyy * lyy) * (lxx * lxx));
    }
    r.xx = (-adxx + ucxx) + csxx;
    r.xy = (-adxy + ucxy) + csxy;
    r.yy = (-adyy + ucyy) + csyy;
    r.zz = 0.0;
    if (K.fenep) {  // rhs.F90:539-541: psi_zz evolves
        const double lzz = exp(n.pzz);
        const double adzz = (n.u * g.pzz_x + n.v * g.pzz_y) + w * 0.0;
        const double cszz = ((0.5 * szz) / lzz) / lzz;
        r.zz = (-adzz + 0.0) + cszz;
    }
}

// calc_rhs_logconf, interior branch, rhs_lc.F90:414-559 (sPTT, 2-D).  `first` is the
// reference's itime==1 .and. iRKstep==1 special case (rhs_lc.F90:503).  On walls (with the
// rotated velocity gradient) there is no advection term.
__host__ __device__ __forceinline__ void rhs_c_lc(const StepConsts &K, const NodeState &n, const Grads &g, bool first,
                                         Rhs &r, bool wall = false) {
    const double w = 0.0;
    double adxx = -((n.u * g.pxx_x + n.v * g.pxx_y) + w * 0.0);
    double adxy = -((n.u * g.pxy_x + n.v * g.pxy_y) + w * 0.0);
    double adyy = -((n.u * g.pyy_x + n.v * g.pyy_y) + w * 0.0);
    double Lv[2], R[4], RT[4], G[4], M[4], B[4], Om[4], P[4], Ci[4], T[4];
    eigens2(n.pxx, n.pxy, n.pyy, Lv, R);
    Lv[0] = exp(Lv[0]);
    Lv[1] = exp(Lv[1]);
    tr2(R, RT);
    double tr_c = Lv[0] + Lv[1];
    G[0] = g.u_x; G[2] = g.u_y; G[1] = g.v_x; G[3] = g.v_y;
    mm2(G, R, T);
    mm2(RT, T, M);
    double om = (Lv[1] * M[2] + Lv[0] * M[1]);
    if (fabs(Lv[1] - Lv[0]) <= 1.0e-30) om = 0.0;
    else om = om / (Lv[1] - Lv[0]);
    M[2] = 0.0; M[1] = 0.0;
    mm2(M, RT, T);
    mm2(R, T, B);
    M[0] = 0.0; M[1] = -om; M[2] = om; M[3] = 0.0;
    mm2(M, RT, T);
    mm2(R, T, Om);
    if (first) {
        Om[0] = Om[1] = Om[2] = Om[3] = 0.0;
        double GT[4];
        tr2(G, GT);
        for (int c = 0; c < 4; c++) B[c] = 0.5 * (G[c] + GT[c]);
    }
    P[0] = n.pxx; P[2] = n.pxy; P[1] = n.pxy; P[3] = n.pyy;
    double OP[4], PO[4], UC[4];
    mm2(Om, P, OP);
    mm2(P, Om, PO);
    for (int c = 0; c < 4; c++) UC[c] = (OP[c] - PO[c]) + 2.0 * B[c];
    double Rx[4];
    if (K.fenep) {  // rhs_lc.F90:520-535: (-1/lambda) c^-1 (f c - I)
        const double cxx = n.cxx, cxy = n.cxy, cyy = n.cyy;
        const double det = cxx * cyy - cxy * cxy;
        Ci[0] = cyy / det; Ci[3] = cxx / det; Ci[2] = -cxy / det; Ci[1] = -cxy / det;
        B[0] = cxx * n.f; B[3] = cyy * n.f; B[2] = cxy * n.f; B[1] = cxy * n.f;
        B[0] = B[0] - 1.0; B[3] = B[3] - 1.0;
        mm2(Ci, B, T);
        for (int c = 0; c < 4; c++) Rx[c] = (-1.0 / K.lambda) * T[c];
    } else {
        double fR = ((1.0 - 2.0 * K.epsPTT) + K.epsPTT * tr_c);
        Ci[0] = fR / Lv[0] - fR; Ci[1] = 0.0; Ci[2] = 0.0; Ci[3] = fR / Lv[1] - fR;
        mm2(Ci, RT, T);
        mm2(R, T, T);
        for (int c = 0; c < 4; c++) Rx[c] = T[c] / K.lambda;
    }
    if (wall) {
        r.xx = UC[0] + Rx[0];
        r.xy = UC[2] + Rx[2];
        r.yy = UC[3] + Rx[3];
        r.zz = 0.0;
        return;
    }
    r.xx = (adxx + UC[0]) + Rx[0];
    r.xy = (adxy + UC[2]) + Rx[2];
    r.yy = (adyy + UC[3]) + Rx[3];
    r.zz = 0.0;
}

}  // namespace sunset
