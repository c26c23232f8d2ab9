// hostcheck.cu -- a host build of the pointwise right-hand side (physics.cuh) and of its
// hand-written adjoint (adjoint.cuh), so the adjoint can be checked against finite
// differences of the forward map without a GPU.  Built into libsunset_hostcheck.so; the time
// step itself never calls it.
#include <vector>

#include "adjoint.cuh"

extern "C" {

// par: Re, Wi, beta, epsPTT, Ma.  s[6], g[18] as in adjoint.cuh; r[6] = P(s, g); with rbar
// given, sbar[6], gbar[18], tbar[2] (Wi, beta) = rbar^T dP.
int sunset_hostcheck_lc(const double *par, const double *s, const double *g, int first, const double *rbar,
                        double *r, double *sbar, double *gbar, double *tbar) {
    SunsetConfig c{};
    c.form = SUNSET_FORM_LC;
    c.morder = c.forder = 6;
    c.kolmogorov_forcing = 0;
    c.L_char = 1.0;
    c.U_char = 1.0;
    c.Re = par[0];
    c.Wi = par[1];
    c.beta = par[2];
    c.epsPTT = par[3];
    c.Ma = par[4];
    c.fenep_l2 = 1e30;
    const sunset::StepConsts K = sunset::step_consts(c, 1, 1, false, false);
    sunset::p_forward_lc(K, s, g, first != 0, 0.0, r);
    if (rbar) {
        for (int k = 0; k < sunset::kAdjS; k++) sbar[k] = 0.0;
        for (int k = 0; k < sunset::kAdjG; k++) gbar[k] = 0.0;
        tbar[0] = tbar[1] = 0.0;
        sunset::p_adjoint_lc(K, s, g, first != 0, rbar, sbar, gbar, tbar);
    }
    return 0;
}

// deal_slice_by_bank (bank_deal.cu) on one slice given as flat lists: lane r's small entries
// are small[soff[r] .. soff[r + 1]), its other entries large[loff[r] .. loff[r + 1]); pos[e] is
// the local position of entry e.  chosen[k * 32 + lane] for k < width (-1: padding).
int sunset_hostcheck_deal(int group, const uint16_t *pos, const int *small, const int *soff, const int *large,
                          const int *loff, int width, int *chosen) {
    std::vector<int> vs[sunset::kSlice], vl[sunset::kSlice];
    int c_s[sunset::kSlice], c[sunset::kSlice];
    for (int r = 0; r < sunset::kSlice; r++) {
        vs[r].assign(small + soff[r], small + soff[r + 1]);
        vl[r].assign(large + loff[r], large + loff[r + 1]);
        c_s[r] = (int)vs[r].size();
        c[r] = c_s[r] + (int)vl[r].size();
    }
    sunset::deal_slice_by_bank(group, pos, vs, vl, c_s, c, width, chosen);
    return 0;
}

// c = lc_c_from_psi(psi) and, with cbar given, psibar = cbar^T dc/dpsi.
int sunset_hostcheck_lc_c(const double *psi, const double *cbar, double *c, double *psibar) {
    sunset::lc_c_from_psi(psi[0], psi[1], psi[2], &c[0], &c[1], &c[2]);
    if (cbar) {
        psibar[0] = psibar[1] = psibar[2] = 0.0;
        sunset::lc_c_from_psi_adj(psi[0], psi[1], psi[2], cbar, psibar);
    }
    return 0;
}
}
