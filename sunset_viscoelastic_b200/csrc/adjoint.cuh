// adjoint.cuh -- reverse mode of the pointwise part of the time step, written by hand.
//
// The right-hand side of a node is R = P(s, g; theta): s its conservative state, g the
// stencil sums of its neighbourhood (gradients, Laplacians), theta the parameters (Wi, beta).
// Given the adjoint r_bar of R, p_adjoint returns the adjoints of s, g and theta, i.e. the
// vector-Jacobian product r_bar^T dP.  The transposed stencils (step adjoint) carry g_bar on
// to the neighbours.  The code recomputes the forward intermediates of physics.cuh and then
// reverses them statement by statement; it follows the forward functions exactly, including
// their branches (the eigen-decomposition's diagonal case, the clamped discriminant, the
// degenerate-eigenvalue case of omega), so it is the derivative of the code as written.
//
// Layout (log-conformation form, 2-D, interior nodes, Kolmogorov forcing only without
// polymer diffusion):
//   s = (rho, rho u, rho v, psi_xx, psi_xy, psi_yy)
//   g = (ro_x, ro_y, u_x, u_y, lap u, v_x, v_y, lap v, cxx_x, cxy_x, cxy_y, cyy_y,
//        pxx_x, pxx_y, pxy_x, pxy_y, pyy_x, pyy_y)
//   r = (rhs_ro, rhs_rou, rhs_rov, rhs_xx, rhs_xy, rhs_yy)
//   theta = (Wi, beta): coef_solvent = beta mu, coef_polymeric = (1-beta) mu / lambda,
//   lambda = Wi L/U (load_data.F90:131-138).
#pragma once

#include "physics.cuh"

namespace sunset {

constexpr int kAdjS = 6, kAdjG = 18, kAdjR = 6;

enum AdjG { G_RO_X, G_RO_Y, G_U_X, G_U_Y, G_LAPU, G_V_X, G_V_Y, G_LAPV, G_CXX_X, G_CXY_X, G_CXY_Y, G_CYY_Y,
            G_PXX_X, G_PXX_Y, G_PXY_X, G_PXY_Y, G_PYY_X, G_PYY_Y };

__host__ __device__ inline Grads adj_grads(const double *g) {
    Grads G{};
    G.ro_x = g[G_RO_X]; G.ro_y = g[G_RO_Y]; G.u_x = g[G_U_X]; G.u_y = g[G_U_Y]; G.lapu = g[G_LAPU];
    G.v_x = g[G_V_X]; G.v_y = g[G_V_Y]; G.lapv = g[G_LAPV];
    G.cxx_x = g[G_CXX_X]; G.cxx_y = 0.0; G.cxy_x = g[G_CXY_X]; G.cxy_y = g[G_CXY_Y]; G.cyy_x = 0.0;
    G.cyy_y = g[G_CYY_Y];
    G.pxx_x = g[G_PXX_X]; G.pxx_y = g[G_PXX_Y]; G.pxy_x = g[G_PXY_X]; G.pxy_y = g[G_PXY_Y];
    G.pyy_x = g[G_PYY_X]; G.pyy_y = g[G_PYY_Y];
    G.lapcxx = G.lapcxy = G.lapcyy = G.lapczz = 0.0;
    return G;
}

// The forward map as the stage kernel evaluates it (u = rho u * (1/rho), c from psi).
__host__ __device__ inline void p_forward_lc(const StepConsts &K, const double *s, const double *g, bool first,
                                             double yn, double *r) {
    NodeState n;
    n.ro = s[0];
    const double ooro = 1.0 / s[0];
    n.u = s[1] * ooro;
    n.v = s[2] * ooro;
    n.y = yn;
    n.f = 0.0;
    n.df = 0.0;
    n.pxx = s[3]; n.pxy = s[4]; n.pyy = s[5]; n.pzz = 0.0;
    lc_c_from_psi(s[3], s[4], s[5], &n.cxx, &n.cxy, &n.cyy);
    n.czz = 1.0;
    const Grads G = adj_grads(g);
    Rhs q;
    rhs_flow(K, n, G, q);
    rhs_c_lc(K, n, G, first, q);
    r[0] = q.ro; r[1] = q.rou; r[2] = q.rov; r[3] = q.xx; r[4] = q.xy; r[5] = q.yy;
}

// ---- 2x2 helpers (column-major, M(i,j) = M[i + 2 j]) ----
// C = A B:  A_bar += C_bar B^T,  B_bar += A^T C_bar
__host__ __device__ inline void mm2_adj(const double *A, const double *B, const double *Cb, double *Ab, double *Bb) {
    if (Ab) {
        Ab[0] += Cb[0] * B[0] + Cb[2] * B[2];
        Ab[1] += Cb[1] * B[0] + Cb[3] * B[2];
        Ab[2] += Cb[0] * B[1] + Cb[2] * B[3];
        Ab[3] += Cb[1] * B[1] + Cb[3] * B[3];
    }
    if (Bb) {
        Bb[0] += A[0] * Cb[0] + A[1] * Cb[1];
        Bb[1] += A[2] * Cb[0] + A[3] * Cb[1];
        Bb[2] += A[0] * Cb[2] + A[1] * Cb[3];
        Bb[3] += A[2] * Cb[2] + A[3] * Cb[3];
    }
}

// eigens2 (physics.cuh) reversed: given the adjoints of the eigenvalues l and of the
// eigenvector matrix R, accumulate those of (a, b, d).
__host__ __device__ inline void eigens2_adj(double a, double b, double d, const double *lb, const double *Rb,
                                            double *ab, double *bb, double *db) {
    if (fabs(b) <= 1.0e-16) {  // l = (a, d), R = I
        *ab += lb[0];
        *db += lb[1];
        return;
    }
    const double tr = a + d;
    const double det = a * d - b * b;
    double tq = (0.25 * tr) * tr - det;
    const bool clamped = tq <= 1.0e-16;
    if (clamped) tq = 0.0;
    const double sq = sqrt(tq);
    const double l0 = 0.5 * tr + sq;
    const double e0 = l0 - d, e1 = b;
    const double nrm = sqrt(e0 * e0 + e1 * e1);
    // R = [e0, e1; -e1, e0] / nrm (column-major: R0 = e0/n, R1 = e1/n, R2 = -R1, R3 = R0)
    const double R0b = Rb[0] + Rb[3], R1b = Rb[1] - Rb[2];
    double e0b = R0b / nrm, e1b = R1b / nrm;
    const double nb = -(R0b * e0 + R1b * e1) / (nrm * nrm);
    e0b += nb * e0 / nrm;
    e1b += nb * e1 / nrm;
    *bb += e1b;
    double l0b = lb[0] + e0b;
    *db -= e0b;
    const double l1b = lb[1];
    double trb = 0.5 * (l0b + l1b);
    const double sqb = l0b - l1b;
    if (!clamped && tq > 0.0) {
        const double tqb = sqb * 0.5 / sq;
        trb += 0.5 * tr * tqb;
        const double detb = -tqb;
        *ab += d * detb;
        *db += a * detb;
        *bb += -2.0 * b * detb;
    }
    *ab += trb;
    *db += trb;
}

// lc_c_from_psi reversed: (cxx_bar, cxy_bar, cyy_bar) -> psi adjoints (accumulated).
__host__ __device__ inline void lc_c_from_psi_adj(double pxx, double pxy, double pyy, const double *cb,
                                                  double *pb) {
    double L[2], R[4], RT[4], Lm[4], T[4];
    eigens2(pxx, pxy, pyy, L, R);
    tr2(R, RT);
    Lm[0] = exp(L[0]); Lm[1] = 0.0; Lm[2] = 0.0; Lm[3] = exp(L[1]);
    mm2(Lm, RT, T);
    const double Cb[4] = {cb[0], cb[1], 0.0, cb[2]};  // outputs C(0,0), C(1,0), C(1,1)
    double Rb[4] = {0, 0, 0, 0}, Tb[4] = {0, 0, 0, 0}, Lmb[4] = {0, 0, 0, 0}, RTb[4] = {0, 0, 0, 0};
    mm2_adj(R, T, Cb, Rb, Tb);     // C = R T
    mm2_adj(Lm, RT, Tb, Lmb, RTb); // T = Lm RT
    Rb[0] += RTb[0]; Rb[1] += RTb[2]; Rb[2] += RTb[1]; Rb[3] += RTb[3];
    const double lb[2] = {Lmb[0] * Lm[0], Lmb[3] * Lm[3]};
    eigens2_adj(pxx, pxy, pyy, lb, Rb, &pb[0], &pb[1], &pb[2]);
}

// Reverse of p_forward_lc.  sb, gb, tb are accumulated (tb: Wi, beta).
__host__ __device__ inline void p_adjoint_lc(const StepConsts &K, const double *s, const double *g, bool first,
                                             const double *rb, double *sb, double *gb, double *tb) {
    const double ro = s[0], ooro = 1.0 / s[0];
    const double u = s[1] * ooro, v = s[2] * ooro;
    const double pxx = s[3], pxy = s[4], pyy = s[5];
    double ub = 0.0, vb = 0.0, rob = 0.0;

    // ---------------- conformation (rhs_c_lc) ----------------
    double Lv[2], R[4], RT[4], G[4], M[4], T1[4], Md[4], T2[4], W[4], T3[4], Om[4], B[4], P[4], Ci[4], T4[4], T5[4];
    eigens2(pxx, pxy, pyy, Lv, R);
    const double mu0 = Lv[0], mu1 = Lv[1];
    Lv[0] = exp(mu0);
    Lv[1] = exp(mu1);
    tr2(R, RT);
    const double tr_c = Lv[0] + Lv[1];
    G[0] = g[G_U_X]; G[2] = g[G_U_Y]; G[1] = g[G_V_X]; G[3] = g[G_V_Y];
    mm2(G, R, T1);
    mm2(RT, T1, M);
    const double den = Lv[1] - Lv[0];
    const bool degenerate = fabs(den) <= 1.0e-30;
    const double omn = Lv[1] * M[2] + Lv[0] * M[1];
    const double om = degenerate ? 0.0 : omn / den;
    Md[0] = M[0]; Md[1] = 0.0; Md[2] = 0.0; Md[3] = M[3];
    mm2(Md, RT, T2);
    mm2(R, T2, B);
    W[0] = 0.0; W[1] = -om; W[2] = om; W[3] = 0.0;
    mm2(W, RT, T3);
    mm2(R, T3, Om);
    if (first) {
        Om[0] = Om[1] = Om[2] = Om[3] = 0.0;
        B[0] = 0.5 * (G[0] + G[0]); B[1] = 0.5 * (G[1] + G[2]); B[2] = 0.5 * (G[2] + G[1]); B[3] = 0.5 * (G[3] + G[3]);
    }
    P[0] = pxx; P[2] = pxy; P[1] = pxy; P[3] = pyy;
    const double fR = (1.0 - 2.0 * K.epsPTT) + K.epsPTT * tr_c;
    Ci[0] = fR / Lv[0] - fR; Ci[1] = 0.0; Ci[2] = 0.0; Ci[3] = fR / Lv[1] - fR;
    mm2(Ci, RT, T4);
    mm2(R, T4, T5);
    const double lam = K.lambda;

    // outputs r3..r5 = (ad + UC) + T5 / lambda at entries (0,0), (0,1), (1,1)
    double UCb[4] = {rb[3], 0.0, rb[4], rb[5]};
    double T5b[4] = {rb[3] / lam, 0.0, rb[4] / lam, rb[5] / lam};
    double lamb = -(T5[0] * rb[3] + T5[2] * rb[4] + T5[3] * rb[5]) / (lam * lam);
    // advection ad_c = -(u c_x + v c_y)
    ub += -(g[G_PXX_X] * rb[3] + g[G_PXY_X] * rb[4] + g[G_PYY_X] * rb[5]);
    vb += -(g[G_PXX_Y] * rb[3] + g[G_PXY_Y] * rb[4] + g[G_PYY_Y] * rb[5]);
    gb[G_PXX_X] += -u * rb[3]; gb[G_PXX_Y] += -v * rb[3];
    gb[G_PXY_X] += -u * rb[4]; gb[G_PXY_Y] += -v * rb[4];
    gb[G_PYY_X] += -u * rb[5]; gb[G_PYY_Y] += -v * rb[5];

    double Rb[4] = {0, 0, 0, 0}, RTb[4] = {0, 0, 0, 0}, Gb[4] = {0, 0, 0, 0}, Pb[4] = {0, 0, 0, 0};
    double T4b[4] = {0, 0, 0, 0}, Cib[4] = {0, 0, 0, 0}, Omb[4] = {0, 0, 0, 0}, Bb[4] = {0, 0, 0, 0};
    double Lvb[2] = {0.0, 0.0};
    mm2_adj(R, T4, T5b, Rb, T4b);      // T5 = R T4
    mm2_adj(Ci, RT, T4b, Cib, RTb);    // T4 = Ci RT
    double fRb = Cib[0] * (1.0 / Lv[0] - 1.0) + Cib[3] * (1.0 / Lv[1] - 1.0);
    Lvb[0] += -Cib[0] * fR / (Lv[0] * Lv[0]);
    Lvb[1] += -Cib[3] * fR / (Lv[1] * Lv[1]);
    double trb = K.epsPTT * fRb;
    // UC = (Om P - P Om) + 2 B
    mm2_adj(Om, P, UCb, Omb, Pb);
    double mUCb[4] = {-UCb[0], -UCb[1], -UCb[2], -UCb[3]};
    mm2_adj(P, Om, mUCb, Pb, Omb);
    for (int c = 0; c < 4; c++) Bb[c] += 2.0 * UCb[c];
    double pxxb = Pb[0], pxyb = Pb[1] + Pb[2], pyyb = Pb[3];
    if (first) {  // Om = 0, B = (G + G^T)/2
        Gb[0] += Bb[0];
        Gb[1] += 0.5 * (Bb[1] + Bb[2]);
        Gb[2] += 0.5 * (Bb[2] + Bb[1]);
        Gb[3] += Bb[3];
    } else {
        double T3b[4] = {0, 0, 0, 0}, Wb[4] = {0, 0, 0, 0}, T2b[4] = {0, 0, 0, 0}, Mdb[4] = {0, 0, 0, 0};
        double Mb[4] = {0, 0, 0, 0}, T1b[4] = {0, 0, 0, 0};
        mm2_adj(R, T3, Omb, Rb, T3b);   // Om = R T3
        mm2_adj(W, RT, T3b, Wb, RTb);   // T3 = W RT
        const double omb = Wb[2] - Wb[1];
        mm2_adj(R, T2, Bb, Rb, T2b);    // B = R T2
        mm2_adj(Md, RT, T2b, Mdb, RTb); // T2 = Md RT
        Mb[0] += Mdb[0];
        Mb[3] += Mdb[3];
        if (!degenerate) {
            const double omnb = omb / den;
            const double denb = -omb * om / den;
            Lvb[1] += denb;
            Lvb[0] -= denb;
            Lvb[1] += M[2] * omnb;
            Mb[2] += Lv[1] * omnb;
            Lvb[0] += M[1] * omnb;
            Mb[1] += Lv[0] * omnb;
        }
        mm2_adj(RT, T1, Mb, RTb, T1b);  // M = RT T1
        mm2_adj(G, R, T1b, Gb, Rb);     // T1 = G R
    }
    gb[G_U_X] += Gb[0]; gb[G_V_X] += Gb[1]; gb[G_U_Y] += Gb[2]; gb[G_V_Y] += Gb[3];
    Lvb[0] += trb;
    Lvb[1] += trb;
    Rb[0] += RTb[0]; Rb[1] += RTb[2]; Rb[2] += RTb[1]; Rb[3] += RTb[3];
    const double mub[2] = {Lvb[0] * Lv[0], Lvb[1] * Lv[1]};
    eigens2_adj(pxx, pxy, pyy, mub, Rb, &pxxb, &pxyb, &pyyb);

    // ---------------- mass and momentum (rhs_flow) ----------------
    const double ro_x = g[G_RO_X], ro_y = g[G_RO_Y], u_x = g[G_U_X], u_y = g[G_U_Y], v_x = g[G_V_X], v_y = g[G_V_Y];
    const double divvel = (u_x + v_y) + 0.0;
    const double tmp_scal = (u * ro_x + v * ro_y) + 0.0;
    const double rro = -ro * divvel - tmp_scal;
    const double adv_u = (u * u_x + v * u_y) + 0.0, adv_v = (u * v_x + v * v_y) + 0.0;
    const double cs = K.coef_solvent, cp = K.coef_polymeric;
    // r1 = ((-tsu - csq ro_x) + bfu) + fvu, r2 likewise
    const double rrou_b = rb[1], rrov_b = rb[2];
    double tsub = -rrou_b, tsvb = -rrov_b;
    gb[G_RO_X] += -K.csq * rrou_b;
    gb[G_RO_Y] += -K.csq * rrov_b;
    rob += (K.grav0 + 0.0) * rrou_b + (K.grav1 + 0.0) * rrov_b;
    gb[G_LAPU] += cs * rrou_b;
    gb[G_LAPV] += cs * rrov_b;
    double csb = g[G_LAPU] * rrou_b + g[G_LAPV] * rrov_b;
    double cpb = ((g[G_CXX_X] + g[G_CXY_Y]) + 0.0) * rrou_b + ((g[G_CXY_X] + g[G_CYY_Y]) + 0.0) * rrov_b;
    gb[G_CXX_X] += cp * rrou_b;
    gb[G_CXY_Y] += cp * rrou_b;
    gb[G_CXY_X] += cp * rrov_b;
    gb[G_CYY_Y] += cp * rrov_b;
    // tsv = ro adv_v - v rro,  tsu = ro adv_u - u rro
    double rrob = rb[0];
    rob += adv_v * tsvb;
    double adv_vb = ro * tsvb;
    vb += -rro * tsvb;
    rrob += -v * tsvb;
    rob += adv_u * tsub;
    double adv_ub = ro * tsub;
    ub += -rro * tsub;
    rrob += -u * tsub;
    ub += v_x * adv_vb; gb[G_V_X] += u * adv_vb; vb += v_y * adv_vb; gb[G_V_Y] += v * adv_vb;
    ub += u_x * adv_ub; gb[G_U_X] += u * adv_ub; vb += u_y * adv_ub; gb[G_U_Y] += v * adv_ub;
    // rro = -ro divvel - tmp_scal
    rob += -divvel * rrob;
    const double divb = -ro * rrob, tmpb = -rrob;
    gb[G_U_X] += divb;
    gb[G_V_Y] += divb;
    ub += ro_x * tmpb; gb[G_RO_X] += u * tmpb; vb += ro_y * tmpb; gb[G_RO_Y] += v * tmpb;

    // ---------------- state: u = rho u / rho, psi ----------------
    sb[1] += ub * ooro;
    sb[2] += vb * ooro;
    double ooro_b = ub * s[1] + vb * s[2];
    sb[0] += rob - ooro_b * ooro * ooro;
    sb[3] += pxxb; sb[4] += pxyb; sb[5] += pyyb;

    // ---------------- parameters ----------------
    // lambda = Wi L / U; coef_solvent = beta mu; coef_polymeric = (1 - beta) mu / lambda
    const double mu = K.visc_total;
    tb[0] += (lamb - cpb * cp / lam) * (lam / K.Wi);
    tb[1] += mu * csb - (mu / lam) * cpb;
}

}  // namespace sunset
