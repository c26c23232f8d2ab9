/*
 * sunset_oracle.c -- CPU restatement (C99 + OpenMP) of SUNSET's LABFM time-step path.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA path and the timed CPU baseline.
 * Parity with the reference is UNPINNED by reference outputs (the reference is Fortran,
 * cannot be compiled here and ships no golden vectors); see sunset_oracle.h.
 *
 * Every routine below restates one reference routine, cited by file:line.  Expressions
 * keep gfortran's left-to-right evaluation order and the file is compiled with
 * -ffp-contract=off, so each operation rounds exactly as the reference's does on x86-64
 * (gfortran -O3 without -march emits no FMA).  Transcendentals call glibc, as the
 * reference does.  OpenMP is used only where the reference loop is parallel and the
 * result does not depend on the thread count; reductions are sequential.
 */
#include "sunset_oracle.h"

#include <float.h>
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ---------------------------------------------------------------------------------------
 * Constants: common_parameter.F90:15-101
 * ------------------------------------------------------------------------------------- */
static const double pi = 3.141592653589793238462643383279502884197;
static const double verysmall = 1.0e-30;
static const double doublesmall = 1.0e-16;
static const double ss = 2.0; /* common_parameter.F90:68 */

/* RK3(2)4[2R+]C, common_parameter.F90:74-94 */
#define RK_A21 (11847461282814.0 / 36547543011857.0)
#define RK_A32 (3943225443063.0 / 7078155732230.0)
#define RK_A43 (-346793006927.0 / 4029903576067.0)
#define RK_B1 (1017324711453.0 / 9774461848756.0)
#define RK_B2 (8237718856693.0 / 13685301971492.0)
#define RK_B3 (57731312506979.0 / 19404895981398.0)
#define RK_B4 (-101169746363290.0 / 37734290219643.0)
#define RK_BH1 (15763415370699.0 / 46270243929542.0)
#define RK_BH2 (514528521746.0 / 5659431552419.0)
#define RK_BH3 (27030193851939.0 / 9429696342944.0)
#define RK_BH4 (-69544964788955.0 / 30262026368149.0)

/* PID, common_parameter.F90:96-101 */
static const double pid_tol = 1.0e-5;
#define PID_A (0.49 / 2.0)
#define PID_B (0.34 / 2.0)
#define PID_C (0.1 / 2.0)
static const double pid_k = 0.9;

static double hovs_for(int forder) { /* common_parameter.F90:44-56 */
    if (forder == 4) return 1.8;
    if (forder == 6) return 2.4;
    if (forder == 10) return 3.1;
    return 2.7;
}
static double hovs_bound_for(int forder) {
    if (forder == 4) return 2.1;
    return 2.4;
}
static int nsize_for(int k) { return (k * k + 3 * k) / 2; } /* labf.F90:56 */

/* ---------------------------------------------------------------------------------------
 * State (common_vars.F90)
 * ------------------------------------------------------------------------------------- */
struct OrSim {
    OrConfig cfg;
    char err[512];
    /* derived parameters, load_data.F90:131-148 */
    double rho_char, visc_total, visc_solvent, visc_polymeric, lambda, csq;
    int kolmo;
    /* nodes */
    int np, npfb, nb, cap;
    double *rx, *ry, *h, *hs, *sp, *rnx, *rny;
    int *type, *fd_parent, *gi, *irel, *vrel;
    double xmin, xmax, ymin, ymax, smax, smin, h0, h2, h3, sup_size;
    int bc[4]; /* xbcond_L, xbcond_U, ybcond_L, ybcond_U */
    int *internal_list, *boundary_list, n_internal;
    /* neighbours */
    int nplink;
    int *ij_count, *ij_count_small, *ij_link; /* link[i*nplink+k], 0-based point index */
    /* weights */
    double *w_grad, *w_lap, *w_hyp, *w_grad_sum, *w_lap_sum, *w_hyp_sum, *vol;
    double *wb_grad2, *wb_grad2_sum; /* boundary second derivatives [jj][k][3] */
    double *cond_d, *cond_f; /* condition numbers of the derivative and filter moment matrices */
    int have_weights;
    /* fields (np) */
    double *ro, *rou, *rov, *row, *u, *v, *w, *p;
    double *psixx, *psixy, *psiyy, *psizz, *cxx, *cxy, *cyy, *czz;
    /* rhs (npfb) */
    double *rhs_ro, *rhs_rou, *rhs_rov, *rhs_row, *rhs_xx, *rhs_xy, *rhs_yy, *rhs_zz;
    /* time */
    double time, dt, dt_cfl, dt_parabolic;
    int itime, iRKstep;
    double emax_nm1, emax_n, emax_np1;
    double ero_norm, erou_norm, exx_norm;
    double driving_force[3];
    double *u_inflow_local; /* nb: inflow velocity of each boundary node (common_vars.F90:111) */
    double eflow_nm1, sum_eflow; /* flow-rate controller (common_vars.F90:82) */
};

static int fail(OrSim *s, const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(s->err, sizeof(s->err), fmt, ap);
    va_end(ap);
    return -1;
}

const char *or_last_error(OrSim *s) { return s ? s->err : "null handle"; }

void or_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

static void *xcalloc(size_t n, size_t sz) {
    void *p = calloc(n ? n : 1, sz);
    if (!p) {
        fprintf(stderr, "sunset_oracle: out of memory\n");
        abort();
    }
    return p;
}

OrSim *or_create(const OrConfig *cfg) {
    OrSim *s = (OrSim *)xcalloc(1, sizeof(OrSim));
    s->cfg = *cfg;
    if (s->cfg.L_char == 0.0) s->cfg.L_char = 1.0;
    if (s->cfg.U_char == 0.0) s->cfg.U_char = 1.0;
    /* load_data.F90:131-148 */
    s->rho_char = 1.0;
    s->visc_total = s->rho_char * s->cfg.U_char * s->cfg.L_char / s->cfg.Re;
    s->visc_solvent = s->cfg.beta * s->visc_total;
    s->visc_polymeric = (1.0 - s->cfg.beta) * s->visc_total;
    s->lambda = s->cfg.Wi * s->cfg.L_char / s->cfg.U_char;
    {
        double t = s->cfg.U_char / s->cfg.Ma;
        s->csq = t * t; /* (u_char/Ma)**two */
    }
    s->kolmo = cfg->kolmogorov_forcing < 0 ? (cfg->form == OR_FORM_CHL) : cfg->kolmogorov_forcing;
    /* setup_flow.F90:147-157 */
    s->dt = 1.0e-6;
    s->emax_np1 = pid_tol;
    s->emax_n = pid_tol;
    s->emax_nm1 = pid_tol;
    s->ero_norm = 1.0 / 1.0;
    s->erou_norm = 1.0 / (1.0 * s->cfg.U_char);
    s->exx_norm = 1.0 / (1.0);
    return s;
}

#define FREE(p) do { free(p); (p) = NULL; } while (0)
static void free_fields(OrSim *s) {
    FREE(s->ro); FREE(s->rou); FREE(s->rov); FREE(s->row); FREE(s->u); FREE(s->v); FREE(s->w);
    FREE(s->p); FREE(s->psixx); FREE(s->psixy); FREE(s->psiyy); FREE(s->psizz);
    FREE(s->cxx); FREE(s->cxy); FREE(s->cyy); FREE(s->czz);
    FREE(s->rhs_ro); FREE(s->rhs_rou); FREE(s->rhs_rov); FREE(s->rhs_row);
    FREE(s->rhs_xx); FREE(s->rhs_xy); FREE(s->rhs_yy); FREE(s->rhs_zz);
}
static void free_links(OrSim *s) {
    FREE(s->ij_count); FREE(s->ij_count_small); FREE(s->ij_link);
    FREE(s->w_grad); FREE(s->w_lap); FREE(s->w_hyp); FREE(s->w_grad_sum); FREE(s->w_lap_sum);
    FREE(s->w_hyp_sum); FREE(s->vol); FREE(s->wb_grad2); FREE(s->wb_grad2_sum);
    FREE(s->cond_d); FREE(s->cond_f);
    s->have_weights = 0;
}
void or_destroy(OrSim *s) {
    if (!s) return;
    free_fields(s);
    free_links(s);
    FREE(s->rx); FREE(s->ry); FREE(s->h); FREE(s->hs); FREE(s->sp); FREE(s->rnx); FREE(s->rny);
    FREE(s->type); FREE(s->fd_parent); FREE(s->gi); FREE(s->irel); FREE(s->vrel);
    FREE(s->internal_list); FREE(s->boundary_list); FREE(s->u_inflow_local);
    free(s);
}

/* ---------------------------------------------------------------------------------------
 * rbfs.F90:48-68 (kernel 1, Wendland C2)
 * ------------------------------------------------------------------------------------- */
double or_pow4_libm(double x) { return pow(x, 4.0); } /* qq4**4.0 -> libm pow */

/* x^4 rounded once from the exact double-double product (Dekker two-product on fma).
   glibc's pow(x,4.0), which the reference calls, is not always correctly rounded (about
   one argument in 1200 in [0,1] differs by one ulp); this variant is the device path's. */
double or_pow4_cr(double x) {
    double a = x * x;
    double ae = fma(x, x, -a);
    double b = a * a;
    double be = fma(a, a, -b);
    double t = fma(2.0 * a, ae, be);
    t = fma(ae, ae, t);
    return b + t;
}

static int g_pow_cr = 0;
void or_set_pow_mode(int correctly_rounded) { g_pow_cr = correctly_rounded; }

double or_wab(double qq, double h2) {
    double qq4 = 1.0 - 0.5 * qq;
    qq4 = g_pow_cr ? or_pow4_cr(qq4) : pow(qq4, 4.0);
    double f = 0.0;
    if (qq <= 2.0 && qq > 0.0) f = ((7.0 / ((4.0 * pi) * h2)) * (2.0 * qq + 1.0)) * qq4;
    return f;
}
static double or_fac(double qq, double h3) {
    double qq2 = qq * qq, qq3 = qq * qq2, qq4 = qq * qq3;
    double f = 0.0;
    if (qq <= 2.0 && qq > 0.0)
        f = (7.0 / ((4.0 * pi) * h3)) * ((((0.625 * qq4) - (3.75 * qq3)) + (7.5 * qq2)) - (5.0 * qq));
    return f;
}

/* ---------------------------------------------------------------------------------------
 * labf.F90:1815-1920 monomials: x^p y^q/(p!q!), degree-graded, x-power descending.
 * Each term is (coef*x^p)*y^q with x^k built as x2=x*x, x3=x2*x, ... as written there.
 * ------------------------------------------------------------------------------------- */
static const double fact[11] = {1, 1, 2, 6, 24, 120, 720, 5040, 40320, 362880, 3628800};

void or_monomials(int order, double x, double y, double *out) {
    double xp[11], yp[11];
    xp[0] = 1.0; yp[0] = 1.0; xp[1] = x; yp[1] = y;
    for (int k = 2; k <= order; k++) { xp[k] = xp[k - 1] * x; yp[k] = yp[k - 1] * y; }
    int idx = 0;
    for (int d = 1; d <= order; d++) {
        for (int p = d; p >= 0; p--) {
            int q = d - p;
            double den = fact[p] * fact[q];
            double t;
            if (den == 1.0) {
                if (p == 0) t = yp[q];
                else if (q == 0) t = xp[p];
                else t = xp[p] * yp[q];
            } else {
                double c = 1.0 / den;
                if (q == 0) t = c * xp[p];
                else if (p == 0) t = c * yp[q];
                else t = (c * xp[p]) * yp[q];
            }
            out[idx++] = t;
        }
    }
}

/* labf.F90:2329-2391: univariate probabilists' Hermite polynomials, as written. */
static double hermite(int n, double z) {
    double z2, z3, z4;
    switch (n) {
    case 0: return 1.0;
    case 1: return z;
    case 2: return z * z - 1.0;
    case 3: return (z * z) * z - 3.0 * z;
    case 4: return ((((z * z) * z) * z) - ((6.0 * z) * z)) + 3.0;
    case 5: z2 = z * z; z3 = z * z2; return ((z2 * z3) - (10.0 * z3)) + (15.0 * z);
    case 6: z2 = z * z; z3 = z * z2; return (((z3 * z3) - ((15.0 * z2) * z2)) + (45.0 * z2)) - 15.0;
    case 7:
        z2 = z * z; z3 = z * z2; z4 = z3 * z;
        return (((z4 * z3) - ((21.0 * z3) * z2)) + (105.0 * z3)) - (105.0 * z);
    case 8:
        z2 = z * z; z4 = z2 * z2;
        return ((((z4 * z4) - ((28.0 * z4) * z2)) + (210.0 * z4)) - (420.0 * z2)) + 105.0;
    case 9:
        z2 = z * z; z3 = z * z2; z4 = z3 * z;
        return (((((z4 * z3) * z2) - ((36.0 * z4) * z3)) + ((378.0 * z3) * z2)) - (1260.0 * z3)) + (945.0 * z);
    case 10:
        z2 = z * z; z4 = z2 * z2;
        return ((((((z4 * z4) * z2) - ((45.0 * z4) * z4)) + ((630.0 * z4) * z2)) - (3150.0 * z4)) + (4725.0 * z2)) - 945.0;
    }
    return 0.0;
}

/* labf.F90:2025-2121 (ABF==2): He_p(x)He_q(y) in the monomials' ordering. */
void or_abfs(int order, double x, double y, double *out) {
    double hx[11], hy[11];
    for (int k = 0; k <= order; k++) { hx[k] = hermite(k, x); hy[k] = hermite(k, y); }
    int idx = 0;
    for (int d = 1; d <= order; d++)
        for (int p = d; p >= 0; p--) {
            int q = d - p;
            if (q == 0) out[idx++] = hx[p];
            else if (p == 0) out[idx++] = hy[q];
            else out[idx++] = hx[p] * hy[q];
        }
}

/* labf.F90:1041-1048, 1-D monomials of the tangential boundary operators, as written */
static void monomials1D(double z, double *out) {
    double z2 = z * z;
    out[0] = z;
    out[1] = 0.5 * z2;
    out[2] = ((1.0 / 6.0) * z) * z2;
    out[3] = (z2 * z2) / 24.0;
    out[4] = ((z2 * z2) * z) / 120.0;
    out[5] = ((z2 * z2) * z2) / 720.0;
}
/* labf.F90:1050-1077 (ABF==2): Hermite ABFs of the 1-D operators */
static void abfs1D(double z, double ff1, double *out) {
    const double oosqrt2 = 1.0 / sqrt(2.0);
    out[0] = ff1 * hermite(1, z);
    out[1] = ff1 * hermite(2, z);
    out[2] = (ff1 * oosqrt2) * hermite(3, z);
    out[3] = ff1 * hermite(4, z);
    out[4] = ff1 * hermite(5, z);
    out[5] = ff1 * hermite(6, z);
}

/* ---------------------------------------------------------------------------------------
 * svdlib.F90:22-327 -- Golub-Kahan-Reinsch SVD and solve, split into factor + apply.
 * labf.F90 solves five right-hand sides with five SVDs of identical copies of one
 * matrix; the factorisation is deterministic, so factoring once and applying it to
 * each right-hand side gives bit-identical results.
 * ------------------------------------------------------------------------------------- */
static double nr_hypot(double a, double b) { /* svdlib.F90:308-327 */
    double absA = fabs(a), absB = fabs(b), t;
    if (absA > absB) {
        t = absB / absA;
        return absA * sqrt(1.0 + t * t);
    }
    if (absB == 0.0) return 0.0;
    t = absA / absB;
    return absB * sqrt(1.0 + t * t);
}

typedef struct {
    int n;
    double *u, *v, *w, *rv1, *tmp;
} SvdWork;

static void svdw_init(SvdWork *sw, int nmax) {
    sw->n = nmax;
    sw->u = (double *)xcalloc((size_t)nmax * nmax, sizeof(double));
    sw->v = (double *)xcalloc((size_t)nmax * nmax, sizeof(double));
    sw->w = (double *)xcalloc(nmax + 2, sizeof(double));
    sw->rv1 = (double *)xcalloc(nmax + 2, sizeof(double));
    sw->tmp = (double *)xcalloc(nmax + 2, sizeof(double));
}
static void svdw_free(SvdWork *sw) { free(sw->u); free(sw->v); free(sw->w); free(sw->rv1); free(sw->tmp); }

#define UM(i, j) umat[((j) - 1) * n + ((i) - 1)]
#define VM(i, j) vmat[((j) - 1) * n + ((i) - 1)]

/* svdlib.F90:37-278. Returns 0, or -1 if the QR iteration does not converge in 30 steps
   (where the reference stops). */
static int svd_factor(const double *amat, int n, SvdWork *sw) {
    double *umat = sw->u, *vmat = sw->v, *W = sw->w - 1, *rv1 = sw->rv1 - 1; /* 1-based */
    double anorm, c, f, g, h, s, scale, x, y, z;
    int i, its, j, jj, k, l = 1, nm;
    memcpy(umat, amat, sizeof(double) * n * n);
    g = 0.0; scale = 0.0; anorm = 0.0;
    for (i = 1; i <= n; i++) {
        l = i + 1;
        rv1[i] = scale * g;
        g = 0.0; s = 0.0; scale = 0.0;
        for (k = i; k <= n; k++) scale = scale + fabs(UM(k, i));
        if (scale != 0.0) {
            for (k = i; k <= n; k++) {
                UM(k, i) = UM(k, i) / scale;
                s = s + UM(k, i) * UM(k, i);
            }
            f = UM(i, i);
            g = -copysign(sqrt(s), f);
            h = f * g - s;
            UM(i, i) = f - g;
            for (j = l; j <= n; j++) {
                s = 0.0;
                for (k = i; k <= n; k++) s = s + UM(k, i) * UM(k, j);
                f = s / h;
                for (k = i; k <= n; k++) UM(k, j) = UM(k, j) + f * UM(k, i);
            }
            for (k = i; k <= n; k++) UM(k, i) = scale * UM(k, i);
        }
        W[i] = scale * g;
        g = 0.0; s = 0.0; scale = 0.0;
        for (k = l; k <= n; k++) scale = scale + fabs(UM(i, k));
        if (scale != 0.0) {
            for (k = l; k <= n; k++) {
                UM(i, k) = UM(i, k) / scale;
                s = s + UM(i, k) * UM(i, k);
            }
            f = UM(i, l);
            g = -copysign(sqrt(s), f);
            h = f * g - s;
            UM(i, l) = f - g;
            for (k = l; k <= n; k++) rv1[k] = UM(i, k) / h;
            for (j = l; j <= n; j++) {
                s = 0.0;
                for (k = l; k <= n; k++) s = s + UM(j, k) * UM(i, k);
                for (k = l; k <= n; k++) UM(j, k) = UM(j, k) + s * rv1[k];
            }
            for (k = l; k <= n; k++) UM(i, k) = scale * UM(i, k);
        }
        {
            double t = fabs(W[i]) + fabs(rv1[i]);
            anorm = (t > anorm) ? t : anorm;
        }
    }
    /* Accumulation of right-hand transformations, svdlib.F90:115-141 */
    for (i = n; i >= 1; i--) {
        if (i < n) {
            if (g != 0.0) {
                for (j = l; j <= n; j++) VM(j, i) = (UM(i, j) / UM(i, l)) / g;
                for (j = l; j <= n; j++) {
                    s = 0.0;
                    for (k = l; k <= n; k++) s = s + UM(i, k) * VM(k, j);
                    for (k = l; k <= n; k++) VM(k, j) = VM(k, j) + s * VM(k, i);
                }
            }
            for (j = l; j <= n; j++) { VM(i, j) = 0.0; VM(j, i) = 0.0; }
        }
        VM(i, i) = 1.0;
        g = rv1[i];
        l = i;
    }
    /* Accumulation of left-hand transformations, svdlib.F90:143-171 */
    for (i = n; i >= 1; i--) {
        l = i + 1;
        g = W[i];
        for (j = l; j <= n; j++) UM(i, j) = 0.0;
        if (g != 0.0) {
            g = 1.0 / g;
            for (j = l; j <= n; j++) {
                s = 0.0;
                for (k = l; k <= n; k++) s = s + UM(k, i) * UM(k, j);
                f = (s / UM(i, i)) * g;
                for (k = i; k <= n; k++) UM(k, j) = UM(k, j) + f * UM(k, i);
            }
            for (j = i; j <= n; j++) UM(j, i) = UM(j, i) * g;
        } else {
            for (j = i; j <= n; j++) UM(j, i) = 0.0;
        }
        UM(i, i) = UM(i, i) + 1.0;
    }
    /* Diagonalisation of the bidiagonal form, svdlib.F90:173-278 */
    nm = 1;
    for (k = n; k >= 1; k--) {
        for (its = 1; its <= 30; its++) {
            for (l = k; l >= 1; l--) {
                nm = l - 1;
                if ((fabs(rv1[l]) + anorm) == anorm) goto L2000;
                if ((fabs(W[nm]) + anorm) == anorm) goto L1000;
            }
        L1000:
            c = 0.0; s = 1.0;
            for (i = l; i <= k; i++) {
                f = s * rv1[i];
                rv1[i] = c * rv1[i];
                if ((fabs(f) + anorm) == anorm) goto L2000;
                g = W[i];
                h = nr_hypot(f, g);
                W[i] = h;
                h = 1.0 / h;
                c = (g * h);
                s = -(f * h);
                for (j = 1; j <= n; j++) {
                    y = UM(j, nm);
                    z = UM(j, i);
                    UM(j, nm) = (y * c) + (z * s);
                    UM(j, i) = -(y * s) + (z * c);
                }
            }
        L2000:
            z = W[k];
            if (l == k) {
                if (z < 0.0) {
                    W[k] = -z;
                    for (j = 1; j <= n; j++) VM(j, k) = -VM(j, k);
                }
                break;
            }
            if (its == 30) return -1;
            x = W[l];
            nm = k - 1;
            y = W[nm];
            g = rv1[nm];
            h = rv1[k];
            f = ((y - z) * (y + z) + (g - h) * (g + h)) / ((2.0 * h) * y);
            g = nr_hypot(f, 1.0);
            f = ((x - z) * (x + z) + h * ((y / (f + copysign(g, f))) - h)) / x;
            c = 1.0; s = 1.0;
            for (j = l; j <= nm; j++) {
                i = j + 1;
                g = rv1[i];
                y = W[i];
                h = s * g;
                g = c * g;
                z = nr_hypot(f, h);
                rv1[j] = z;
                c = f / z;
                s = h / z;
                f = (x * c) + (g * s);
                g = -(x * s) + (g * c);
                h = y * s;
                y = y * c;
                for (jj = 1; jj <= n; jj++) {
                    x = VM(jj, j);
                    z = VM(jj, i);
                    VM(jj, j) = (x * c) + (z * s);
                    VM(jj, i) = -(x * s) + (z * c);
                }
                z = nr_hypot(f, h);
                W[j] = z;
                if (z != 0.0) {
                    z = 1.0 / z;
                    c = f * z;
                    s = h * z;
                }
                f = (c * g) + (s * y);
                x = -(s * g) + (c * y);
                for (jj = 1; jj <= n; jj++) {
                    y = UM(jj, j);
                    z = UM(jj, i);
                    UM(jj, j) = (y * c) + (z * s);
                    UM(jj, i) = -(y * s) + (z * c);
                }
            }
            rv1[l] = 0.0;
            rv1[k] = f;
            W[k] = x;
        }
    }
    return 0;
}

/* svdlib.F90:279-303: x = V diag(1/w) U^T b, skipping exactly-zero singular values. */
/* 2-norm condition number sigma_max / sigma_min of the factored matrix (infinite when a
   singular value is exactly zero).  The reference inverts every nonzero sigma however small
   (svdlib.F90:283-293); this is what the library reports so that a near-singular moment
   matrix does not pass silently. */
static double svd_cond(const SvdWork *sw, int n) {
    double smax = 0.0, smin = INFINITY;
    for (int j = 0; j < n; j++) {
        const double w = fabs(sw->w[j]);
        smax = w > smax ? w : smax;
        smin = w < smin ? w : smin;
    }
    return smin > 0.0 ? smax / smin : INFINITY;
}

static void svd_apply(const SvdWork *sw, int n, double *bvec) {
    const double *umat = sw->u, *vmat = sw->v, *W = sw->w - 1;
    double *tmp = sw->tmp - 1, *b = bvec - 1, s;
    for (int j = 1; j <= n; j++) {
        s = 0.0;
        if (W[j] != 0.0) {
            for (int i = 1; i <= n; i++) s = s + UM(i, j) * b[i];
            s = s / W[j];
        }
        tmp[j] = s;
    }
    for (int j = 1; j <= n; j++) {
        s = 0.0;
        for (int jj = 1; jj <= n; jj++) s = s + VM(j, jj) * tmp[jj];
        b[j] = s;
    }
}
#undef UM
#undef VM

void or_svd_solve(double *amat, int n, double *bvec) {
    SvdWork sw;
    svdw_init(&sw, n);
    if (svd_factor(amat, n, &sw) == 0) svd_apply(&sw, n, bvec);
    else for (int i = 0; i < n; i++) bvec[i] = NAN;
    svdw_free(&sw);
}

/* ---------------------------------------------------------------------------------------
 * setup_domain.F90:80-374 (build_domain, non-MPI) and mirror_boundaries.F90:34-261
 * ------------------------------------------------------------------------------------- */
static void grow_nodes(OrSim *s, int cap) {
#define GROW(p, T) p = (T *)realloc(p, sizeof(T) * (size_t)cap)
    GROW(s->rx, double); GROW(s->ry, double); GROW(s->h, double); GROW(s->hs, double);
    GROW(s->sp, double); GROW(s->rnx, double); GROW(s->rny, double);
    GROW(s->type, int); GROW(s->fd_parent, int); GROW(s->gi, int); GROW(s->irel, int); GROW(s->vrel, int);
#undef GROW
    s->cap = cap;
}

static int add_point(OrSim *s) {
    if (s->np >= s->cap) grow_nodes(s, s->cap * 2 + 64);
    return s->np++;
}

/* create_mirror_particles, mirror_boundaries.F90:34-261 */
static int create_mirror_particles(OrSim *s) {
    const double mlayer_buff = 2.0;
    const int xL = s->bc[0], xU = s->bc[1], yL = s->bc[2], yU = s->bc[3];
    const double xmin = s->xmin, xmax = s->xmax, ymin = s->ymin, ymax = s->ymax;
    if ((xL == 1 && xU != 1) || (xU == 1 && xL != 1) || (yL == 1 && yU != 1) || (yU == 1 && yL != 1))
        return fail(s, "periodic boundary conditions incorrectly specified with bcond");
    int npfb = s->npfb;
    s->np = npfb;
    for (int i = 0; i < npfb; i++) {
        double xi = s->rx[i], yi = s->ry[i], lim = (ss * s->h[i]) * mlayer_buff;
        int k;
#define MIRROR(VREL, XNEW, YNEW)                                                  \
    do {                                                                          \
        double xn_ = (XNEW), yn_ = (YNEW);                                        \
        k = add_point(s);                                                         \
        s->irel[k] = i; s->vrel[k] = (VREL); s->rx[k] = xn_; s->ry[k] = yn_;      \
    } while (0)
        if (xi <= xmin + lim) {
            if (xL == 1) MIRROR(1, (xi + xmax) - xmin, yi);
            else if (xL == 2) MIRROR(2, 2.0 * xmin - xi, yi);
        }
        if (xi >= xmax - lim) {
            if (xU == 1) MIRROR(1, (xi - xmax) + xmin, yi);
            else if (xU == 2) MIRROR(2, 2.0 * xmax - xi, yi);
        }
        if (yi <= ymin + lim) {
            if (yL == 1) MIRROR(1, xi, (yi + ymax) - ymin);
            else if (yL == 2) MIRROR(3, xi, 2.0 * ymin - yi);
            else if (yL == 3) MIRROR(4, xi, 2.0 * ymin - yi);
        }
        if (yi >= ymax - lim) {
            if (yU == 1) MIRROR(1, xi, (yi - ymax) + ymin);
            else if (yU == 2) MIRROR(3, xi, 2.0 * ymax - yi);
            else if (yU == 3) MIRROR(4, xi, 2.0 * ymax - yi);
        }
        /* corners: cdist = sqrt(dot_product(rcorn-rp,rcorn-rp)) with z=0 */
        const double cx[4] = {xmin, xmax, xmin, xmax}, cy[4] = {ymin, ymin, ymax, ymax};
        const int bx[4] = {xL, xU, xL, xU}, by[4] = {yL, yL, yU, yU};
        for (int c = 0; c < 4; c++) {
            double dx = cx[c] - xi, dy = cy[c] - yi, dz = 0.0 - 0.0;
            double cdist = sqrt((dx * dx + dy * dy) + dz * dz);
            if (cdist <= lim && bx[c] != 0 && by[c] != 0) {
                int right = (c == 1 || c == 3), top = (c == 2 || c == 3);
                double xp = right ? (xi - xmax) + xmin : (xi + xmax) - xmin;
                double yp = top ? (yi - ymax) + ymin : (yi + ymax) - ymin;
                double xs = right ? 2.0 * xmax - xi : 2.0 * xmin - xi;
                double ys = top ? 2.0 * ymax - yi : 2.0 * ymin - yi;
                if (bx[c] == 1 && by[c] == 1) MIRROR(1, xp, yp);
                else if (bx[c] == 2 && by[c] == 1) MIRROR(2, xs, yp);
                else if (bx[c] == 1 && by[c] == 2) MIRROR(3, xp, ys);
                else if (bx[c] == 2 && by[c] == 2) MIRROR(4, xs, ys);
                else {
                    /* the reference increments imp and sets irelation but no position or
                       vrelation for other combinations (e.g. periodic x + no-slip y) */
                    return fail(s, "corner mirror for bcond (%d,%d) is undefined in the reference", bx[c], by[c]);
                }
            }
        }
#undef MIRROR
    }
    for (int i = npfb; i < s->np; i++) {
        int par = s->irel[i];
        s->type[i] = s->type[par];
        s->h[i] = s->h[par];
        s->hs[i] = s->hs[par];
        s->sp[i] = s->sp[par];
        s->rnx[i] = s->rnx[par];
        s->rny[i] = s->rny[par];
        s->fd_parent[i] = 0;
        s->gi[i] = s->gi[par];
    }
    return 0;
}

int or_build_domain(OrSim *s, int nrows, const int *gi, const double *x, const double *y,
                    const int *node_type, const double *nx, const double *ny, const double *sp,
                    double xmin, double xmax, double ymin, double ymax, const int *bcond,
                    double smax) {
    const double hovs = hovs_for(s->cfg.forder), hovs_bound = hovs_bound_for(s->cfg.forder);
    const double hos = s->cfg.h_over_s;
    free_fields(s);
    free_links(s);
    s->np = 0;
    s->cap = 0;
    grow_nodes(s, 5 * nrows + 64);
    s->xmin = xmin; s->xmax = xmax; s->ymin = ymin; s->ymax = ymax;
    for (int c = 0; c < 4; c++) s->bc[c] = bcond[c];
    s->smax = smax;
    s->h0 = (hos > 0 ? hos : hovs) * smax; /* setup_domain.F90:105 */
    s->sup_size = ss * s->h0;
    s->h2 = s->h0 * s->h0;
    s->h3 = s->h2 * s->h0;
    int nb = 0;
    for (int r = 0; r < nrows; r++) { /* setup_domain.F90:177-199 */
        int ii = add_point(s);
        s->gi[ii] = gi[r];
        s->rx[ii] = x[r]; s->ry[ii] = y[r];
        s->rnx[ii] = nx[r]; s->rny[ii] = ny[r];
        s->h[ii] = sp[r] * hovs;
        s->sp[ii] = sp[r];
        s->type[ii] = node_type[r];
        s->fd_parent[ii] = -1;
        s->irel[ii] = ii;
        s->vrel[ii] = 1;
        if (node_type[r] >= 0 && node_type[r] <= 2) {
            s->h[ii] = s->sp[ii] * hovs_bound;
            int k = ii;
            nb++;
            for (int j = 1; j <= 4; j++) {
                ii = add_point(s);
                s->gi[ii] = s->gi[k] + j;
                s->rx[ii] = s->rx[k] + (s->rnx[k] * (double)j) * s->sp[k];
                s->ry[ii] = s->ry[k] + (s->rny[k] * (double)j) * s->sp[k];
                s->rnx[ii] = s->rnx[k]; s->rny[ii] = s->rny[k];
                s->h[ii] = s->h[k]; s->sp[ii] = s->sp[k];
                s->type[ii] = -j;
                s->fd_parent[ii] = k;
                s->irel[ii] = ii;
                s->vrel[ii] = 1;
            }
        }
    }
    s->npfb = s->np;
    s->nb = nb;
    for (int i = 0; i < s->npfb; i++) {
        if (hos > 0) s->h[i] = hos * s->sp[i];
        s->hs[i] = s->h[i]; /* h_small = h, setup_domain.F90:202 */
    }
    if (create_mirror_particles(s)) return -1;
    /* internal / boundary lists, setup_domain.F90:314-327 */
    FREE(s->internal_list); FREE(s->boundary_list);
    s->internal_list = (int *)xcalloc(s->npfb, sizeof(int));
    s->boundary_list = (int *)xcalloc(s->nb ? s->nb : 1, sizeof(int));
    int ii = 0, jj = 0;
    for (int i = 0; i < s->npfb; i++) {
        int t = s->type[i];
        if (t < 0 || t == 999 || t == 998) s->internal_list[ii++] = i;
        else s->boundary_list[jj++] = i;
    }
    s->n_internal = ii;
    if (jj != s->nb) return fail(s, "boundary count mismatch (%d vs %d)", jj, s->nb);
    s->smin = 1e300;
    for (int i = 0; i < s->npfb; i++) if (s->sp[i] < s->smin) s->smin = s->sp[i];
    return 0;
}

int or_sizes(OrSim *s, int *np, int *npfb, int *nb, int *nplink) {
    if (np) *np = s->np;
    if (npfb) *npfb = s->npfb;
    if (nb) *nb = s->nb;
    if (nplink) *nplink = s->nplink;
    return 0;
}

int or_get_nodes(OrSim *s, double *x, double *y, double *h, double *h_small, double *sp,
                 int *node_type, int *irelation, int *vrelation) {
    for (int i = 0; i < s->np; i++) {
        if (x) x[i] = s->rx[i];
        if (y) y[i] = s->ry[i];
        if (h) h[i] = s->h[i];
        if (h_small) h_small[i] = s->hs[i];
        if (sp) sp[i] = s->sp[i];
        if (node_type) node_type[i] = s->type[i];
        if (irelation) irelation[i] = s->irel[i] + 1;
        if (vrelation) vrelation[i] = s->vrel[i];
    }
    return 0;
}

/* ---------------------------------------------------------------------------------------
 * neighbours.F90:32-341
 * ------------------------------------------------------------------------------------- */
static void quicksort_neighbours(int *link, double *a, int first, int last) { /* :316-341 (1-based) */
    double x = a[(first + last) / 2], t;
    int i = first, j = last, it;
    for (;;) {
        while (a[i] < x) i++;
        while (x < a[j]) j--;
        if (i >= j) break;
        t = a[i]; a[i] = a[j]; a[j] = t;
        it = link[i]; link[i] = link[j]; link[j] = it;
        i++;
        j--;
    }
    if (first < i - 1) quicksort_neighbours(link, a, first, i - 1);
    if (j + 1 < last) quicksort_neighbours(link, a, j + 1, last);
}

int or_find_neighbours(OrSim *s) {
    const int np = s->np, npfb = s->npfb;
    /* cell_generator, :75-93 */
    double sizeX = s->xmax - s->xmin, sizeY = s->ymax - s->ymin;
    double unoss = 1.0 / (1.0 * s->sup_size);
    double xmaxt = s->xmax + sizeX, xmint = s->xmin - sizeX;
    double ymaxt = s->ymax + sizeY, ymint = s->ymin - sizeY;
    int ncx = (int)((xmaxt - xmint) * unoss) + 1;
    int ncy = (int)((ymaxt - ymint) * unoss) + 1;
    long nct = (long)ncx * ncy;
    /* neighbour_cells, :95-158: 1-based cell ids, order self,E,NE,SE,W,NW,SW,N,S */
    /* divide, :160-206 */
    int *cellpart = (int *)xcalloc(np, sizeof(int));
    int *nc = (int *)xcalloc(nct + 2, sizeof(int));
    int *ist = (int *)xcalloc(nct + 2, sizeof(int));
    int *ip = (int *)xcalloc(np, sizeof(int));
    for (int k = 0; k < np; k++) {
        double ddx = s->rx[k] - xmint, ddy = s->ry[k] - ymint;
        int icell = (int)(ddx * unoss) + 1, jcell = (int)(ddy * unoss) + 1;
        long ii = icell + (long)(jcell - 1) * ncx;
        if (icell < 1 || icell > ncx || jcell < 1 || jcell > ncy) {
            free(cellpart); free(nc); free(ist); free(ip);
            return fail(s, "node %d outside the cell grid", k);
        }
        nc[ii]++;
        cellpart[k] = (int)ii;
    }
    ist[1] = 1;
    for (long ii = 1; ii <= nct; ii++) { ist[ii + 1] = ist[ii] + nc[ii]; nc[ii] = 0; }
    for (int k = 0; k < np; k++) { ip[ist[cellpart[k]] + nc[cellpart[k]] - 1] = k; nc[cellpart[k]]++; }

    /* neighboring_list_parallel, :208-243: count, then fill */
    free_links(s);
    s->ij_count = (int *)xcalloc(npfb, sizeof(int));
    s->ij_count_small = (int *)xcalloc(npfb, sizeof(int));
    int pass, nplink = 0;
    for (pass = 0; pass < 2; pass++) {
        if (pass == 1) s->ij_link = (int *)xcalloc((size_t)npfb * nplink, sizeof(int));
        int maxc = 0;
#pragma omp parallel for schedule(static) reduction(max : maxc)
        for (int i = 0; i < npfb; i++) {
            int ic = cellpart[i];
            int icx = (ic - 1) % ncx + 1, icy = (ic - 1) / ncx + 1;
            long cells[9];
            int ncell = 0;
            cells[ncell++] = ic;
            if (icx + 1 <= ncx) {
                cells[ncell++] = ic + 1;
                if (icy + 1 <= ncy) cells[ncell++] = ic + ncx + 1;
                if (icy - 1 >= 1) cells[ncell++] = ic - ncx + 1;
            }
            if (icx - 1 >= 1) {
                cells[ncell++] = ic - 1;
                if (icy + 1 <= ncy) cells[ncell++] = ic + ncx - 1;
                if (icy - 1 >= 1) cells[ncell++] = ic - ncx - 1;
            }
            if (icy + 1 <= ncy) cells[ncell++] = ic + ncx;
            if (icy - 1 >= 1) cells[ncell++] = ic - ncx;
            double hs2 = (s->h[i] * ss) * (s->h[i] * ss);
            int cnt = 0;
            for (int kc = 0; kc < ncell; kc++) {
                long jc = cells[kc];
                for (int jj = ist[jc]; jj < ist[jc + 1]; jj++) {
                    int j = ip[jj - 1];
                    double rx = s->rx[i] - s->rx[j], ry = s->ry[i] - s->ry[j], rz = 0.0 - 0.0;
                    double rr2 = (rx * rx + ry * ry) + rz * rz;
                    if (rr2 <= hs2) {
                        if (pass == 1) s->ij_link[(size_t)i * nplink + cnt] = j;
                        cnt++;
                    }
                }
            }
            s->ij_count[i] = cnt;
            if (cnt > maxc) maxc = cnt;
        }
        if (pass == 0) nplink = maxc;
    }
    s->nplink = nplink;
    free(cellpart); free(nc); free(ist); free(ip);

    /* order_neighbours, :272-314 */
#pragma omp parallel
    {
        double *rij2 = (double *)xcalloc(nplink + 1, sizeof(double));
#pragma omp for schedule(static)
        for (int i = 0; i < npfb; i++) {
            int *lk = s->ij_link + (size_t)i * nplink;
            int cnt = s->ij_count[i];
            for (int k = 0; k < cnt; k++) {
                int j = lk[k];
                double rx = s->rx[i] - s->rx[j], ry = s->ry[i] - s->ry[j], rz = 0.0 - 0.0;
                rij2[k + 1] = (rx * rx + ry * ry) + rz * rz;
            }
            if (cnt >= 1) quicksort_neighbours(lk - 1, rij2, 1, cnt);
            int small = 0;
            double hs2 = (s->hs[i] * ss) * (s->hs[i] * ss);
            for (int k = 0; k < cnt; k++) {
                int j = lk[k];
                double rx = s->rx[i] - s->rx[j], ry = s->ry[i] - s->ry[j], rz = 0.0 - 0.0;
                double rad2 = (rx * rx + ry * ry) + rz * rz;
                if (rad2 <= hs2) small++;
            }
            s->ij_count_small[i] = small;
        }
        free(rij2);
    }
    return 0;
}

int or_get_neighbours(OrSim *s, int *ij_count, int *ij_count_small, int *ij_link) {
    if (!s->ij_count) return fail(s, "neighbours not built");
    for (int i = 0; i < s->npfb; i++) {
        if (ij_count) ij_count[i] = s->ij_count[i];
        if (ij_count_small) ij_count_small[i] = s->ij_count_small[i];
        if (ij_link)
            for (int k = 0; k < s->nplink; k++) {
                size_t o = (size_t)i * s->nplink + k;
                ij_link[o] = k < s->ij_count[i] ? s->ij_link[o] + 1 : 0;
            }
    }
    return 0;
}

/* ---------------------------------------------------------------------------------------
 * labf.F90:34-231 calc_labf_weights, :233-394 calc_filter_weights, :453-503 volumes
 * ------------------------------------------------------------------------------------- */
static void alloc_weights(OrSim *s) {
    size_t nn = (size_t)s->npfb * s->nplink;
    FREE(s->w_grad); FREE(s->w_lap); FREE(s->w_hyp); FREE(s->vol); FREE(s->cond_d); FREE(s->cond_f);
    s->cond_d = (double *)xcalloc(s->npfb, sizeof(double));
    s->cond_f = (double *)xcalloc(s->npfb, sizeof(double));
    s->w_grad = (double *)xcalloc(2 * nn, sizeof(double));
    s->w_lap = (double *)xcalloc(nn, sizeof(double));
    s->w_hyp = (double *)xcalloc(nn, sizeof(double));
    s->vol = (double *)xcalloc(s->npfb, sizeof(double));
}

/* Assemble A(i1,i2) = sum_k X_i1 G_i2 over links 0..cnt-1 of node i with length hh,
   labf.F90:88-123 (and :268-303 for the filter). A is column-major n x n. */
static void assemble_moments(const OrSim *s, int i, int cnt, double hh, int order_large, int n,
                             double *amat, double *gvec, double *xvec) {
    memset(amat, 0, sizeof(double) * n * n);
    const int *lk = s->ij_link + (size_t)i * s->nplink;
    for (int k = 0; k < cnt; k++) {
        int j = lk[k];
        double rijx = s->rx[i] - s->rx[j], rijy = s->ry[i] - s->ry[j];
        double x = -rijx, y = -rijy;
        double rad = sqrt(x * x + y * y) / hh, qq = rad;
        double ff1 = or_wab(qq, s->h2);
        double xx = x / hh, yy = y / hh;
        or_abfs(order_large, xx, yy, gvec);
        int nl = nsize_for(order_large);
        for (int m = 0; m < nl; m++) gvec[m] = gvec[m] * ff1;
        or_monomials(order_large, x / hh, y / hh, xvec);
        for (int i2 = 0; i2 < n; i2++)
            for (int i1 = 0; i1 < n; i1++) amat[i2 * n + i1] = amat[i2 * n + i1] + xvec[i1] * gvec[i2];
    }
}

/* The order drop near walls: keep the first m unknowns (labf.F90:125-148). */
static void drop_order(double *amat, int n, int m) {
    for (int i1 = 0; i1 < n; i1++)
        for (int i2 = m; i2 < n; i2++) amat[i2 * n + i1] = 0.0;
    for (int i1 = m; i1 < n; i1++) {
        for (int i2 = 0; i2 < n; i2++) amat[i2 * n + i1] = 0.0;
        amat[i1 * n + i1] = 1.0;
    }
}

static double dotn(const double *a, const double *b, int n) {
    double s = 0.0;
    for (int m = 0; m < n; m++) s = s + a[m] * b[m];
    return s;
}

/* hyperviscosity right-hand sides, labf.F90:325-351 */
static void hyp_rhs(int order, double *b, int n) {
    memset(b, 0, sizeof(double) * n);
    if (order <= 5) { b[9] = -1.0; b[11] = -2.0; b[13] = -1.0; }
    else if (order <= 7) { b[20] = 1.0; b[22] = 3.0; b[24] = 3.0; b[26] = 1.0; }
    else if (order <= 9) { b[35] = -1.0; b[37] = -4.0; b[39] = -6.0; b[41] = -4.0; b[43] = -1.0; }
    else { b[54] = 1.0; b[56] = 5.0; b[58] = 10.0; b[60] = 10.0; b[62] = 5.0; b[64] = 1.0; }
}

int or_get_conditioning(OrSim *s, double *cond_deriv, double *cond_filter) {
    if (!s->cond_d) return fail(s, "weights not built");
    if (cond_deriv) memcpy(cond_deriv, s->cond_d, sizeof(double) * s->npfb);
    if (cond_filter) memcpy(cond_filter, s->cond_f, sizeof(double) * s->npfb);
    return 0;
}

int or_calc_labf_weights(OrSim *s) {
    if (!s->ij_count) return fail(s, "neighbours not built");
    const int forder = s->cfg.forder, morder = s->cfg.morder;
    const int nlarge = nsize_for(forder), nG = nsize_for(morder), nF = nsize_for(forder);
    alloc_weights(s);
    int bad = -1;
#pragma omp parallel
    {
        SvdWork sw;
        svdw_init(&sw, nlarge);
        double *amat = (double *)xcalloc((size_t)nlarge * nlarge, sizeof(double));
        double *gvec = (double *)xcalloc(nlarge, sizeof(double));
        double *xvec = (double *)xcalloc(nlarge, sizeof(double));
        double *bx = (double *)xcalloc(nlarge, sizeof(double)), *by = (double *)xcalloc(nlarge, sizeof(double));
        double *bxx = (double *)xcalloc(nlarge, sizeof(double)), *byy = (double *)xcalloc(nlarge, sizeof(double));
        double *blap = (double *)xcalloc(nlarge, sizeof(double)), *bh = (double *)xcalloc(nlarge, sizeof(double));
#pragma omp for schedule(dynamic, 64)
        for (int ii = 0; ii < s->n_internal; ii++) {
            int i = s->internal_list[ii];
            const int *lk = s->ij_link + (size_t)i * s->nplink;
            int t = s->type[i];
            /* ---- derivative weights, :80-215 ---- */
            double hh = s->hs[i];
            assemble_moments(s, i, s->ij_count_small[i], hh, forder, nG, amat, gvec, xvec);
            if (morder >= 7 && (t == 998 || t < 0)) drop_order(amat, nG, 27);
            if (morder >= 5 && (t == -1 || t == -2)) drop_order(amat, nG, 14);
            memset(bx, 0, sizeof(double) * nG); bx[0] = 1.0;
            memset(by, 0, sizeof(double) * nG); by[1] = 1.0;
            memset(bxx, 0, sizeof(double) * nG); bxx[2] = 1.0;
            memset(byy, 0, sizeof(double) * nG); byy[4] = 1.0;
            if (svd_factor(amat, nG, &sw)) {
#pragma omp critical
                bad = i;
                continue;
            }
            s->cond_d[i] = svd_cond(&sw, nG);
            svd_apply(&sw, nG, bx);
            svd_apply(&sw, nG, by);
            svd_apply(&sw, nG, bxx);
            svd_apply(&sw, nG, byy);
            for (int m = 0; m < nG; m++) blap[m] = bxx[m] + byy[m];
            for (int k = 0; k < s->ij_count[i]; k++) {
                int j = lk[k];
                double x = -(s->rx[i] - s->rx[j]), y = -(s->ry[i] - s->ry[j]);
                double rad = sqrt(x * x + y * y) / hh, qq = rad;
                double ff1 = or_wab(qq, s->h2);
                double xx = x / hh, yy = y / hh;
                or_abfs(forder, xx, yy, gvec);
                for (int m = 0; m < nlarge; m++) gvec[m] = gvec[m] * ff1;
                size_t o = (size_t)i * s->nplink + k;
                s->w_grad[2 * o + 0] = dotn(bx, gvec, nG) / hh;
                s->w_grad[2 * o + 1] = dotn(by, gvec, nG) / hh;
                s->w_lap[o] = (dotn(blap, gvec, nG) / hh) / hh;
            }
            /* ---- filter weights, calc_filter_weights :258-388 ---- */
            hh = s->h[i];
            assemble_moments(s, i, s->ij_count[i], hh, forder, nF, amat, gvec, xvec);
            if (forder >= 7 && (t == 998 || t < 0)) drop_order(amat, nF, 27);
            hyp_rhs(forder, bh, nF);
            if (forder >= 7 && (t == 998 || t < 0)) hyp_rhs(6, bh, nF);
            if (forder >= 5 && t == -1) {
                drop_order(amat, nF, 14);
                hyp_rhs(4, bh, nF);
            }
            if (svd_factor(amat, nF, &sw)) {
#pragma omp critical
                bad = i;
                continue;
            }
            s->cond_f[i] = svd_cond(&sw, nF);
            svd_apply(&sw, nF, bh);
            for (int k = 0; k < s->ij_count[i]; k++) {
                int j = lk[k];
                double x = -(s->rx[i] - s->rx[j]), y = -(s->ry[i] - s->ry[j]);
                double rad = sqrt(x * x + y * y) / hh, qq = rad;
                double ff1 = or_wab(qq, s->h2);
                double xx = x / hh, yy = y / hh;
                or_abfs(forder, xx, yy, gvec);
                for (int m = 0; m < nF; m++) gvec[m] = gvec[m] * ff1;
                s->w_hyp[(size_t)i * s->nplink + k] = dotn(bh, gvec, nF);
            }
            /* ---- node volume, calc_node_volumes :460-486 ---- */
            double vsum = 0.0;
            for (int k = 0; k < s->ij_count[i]; k++) {
                int j = lk[k];
                double x = -(s->rx[i] - s->rx[j]), y = -(s->ry[i] - s->ry[j]);
                double rad = sqrt(x * x + y * y) / hh;
                double f1 = ((9.0 / pi) * exp((-9.0 * rad) * rad)) / (hh * hh);
                vsum = vsum + f1;
            }
            s->vol[i] = 1.0 / vsum;
        }
        svdw_free(&sw);
        free(amat); free(gvec); free(xvec); free(bx); free(by); free(bxx); free(byy); free(blap); free(bh);
    }
    if (bad >= 0) return fail(s, "SVD not converging at node %d (svdlib.F90:219-222)", bad);
    for (int jj = 0; jj < s->nb; jj++) { /* :489-493 */
        int i = s->boundary_list[jj];
        s->vol[i] = s->sp[i] * s->sp[i];
    }
    return 0;
}

/* ---------------------------------------------------------------------------------------
 * labf.F90:505-1039 -- calc_boundary_weights.  Boundary node i0 and its four FD rows
 * i1..i4 (the nodes that follow it): normal derivatives by 5-point finite differences,
 * tangential ones by 6th-order 1-D LABFM on the same layer, curvature correction, and the
 * rotation of rows 1-2 into the x-y frame.  Wall first derivatives stay in the
 * normal-tangent frame (the wall equations are solved there).
 * ------------------------------------------------------------------------------------- */
static double dot6(const double *a, const double *b) { /* dot_product, summed in order */
    double t = 0.0;
    for (int k = 0; k < 6; k++) t = t + a[k] * b[k];
    return t;
}

/* 1-D LABFM along the tangent (xt,yt) of node i, over the links on i's own layer:
   assemble the 6x6 moment matrix (labf.F90:696-722 and the row variants). */
static void assemble_1d(const OrSim *s, int i, double xt, double yt, double hh, double *amat) {
    const int *lk = s->ij_link + (size_t)i * s->nplink;
    double xvec[6], gvec[6];
    memset(amat, 0, sizeof(double) * 36);
    for (int k = 0; k < s->ij_count[i]; k++) {
        int j = lk[k];
        if (s->type[j] != s->type[i]) continue;
        double rijx = s->rx[i] - s->rx[j], rijy = s->ry[i] - s->ry[j];
        double x = -(rijx * xt + rijy * yt);
        if (i == j) x = 0.0;
        monomials1D(x / hh, xvec);
        double ff1 = or_fac(fabs(x / hh), s->h3);
        x = x / hh;
        abfs1D(x, ff1, gvec);
        for (int i1 = 0; i1 < 6; i1++)
            for (int i2 = 0; i2 < 6; i2++) amat[i1 + 6 * i2] = amat[i1 + 6 * i2] + xvec[i1] * gvec[i2];
    }
}

/* the 1-D ABF vector of link j of node i (labf.F90:737-748) */
static void abf_1d_link(const OrSim *s, int i, int j, double xt, double yt, double hh, double *gvec) {
    double rijx = s->rx[i] - s->rx[j], rijy = s->ry[i] - s->ry[j];
    double x = -(rijx * xt + rijy * yt);
    if (i == j) x = 0.0;
    double ff1 = or_fac(fabs(x / hh), s->h3);
    x = x / hh;
    abfs1D(x, ff1, gvec);
}

/* ---------------------------------------------------------------------------------------
 * adapt_stencils (labf.F90:1079-1412) and adapt_stencils_main (:1414-1721), 2-D, Hermite ABFs.
 * For every plain interior node (node_type > 2 and not 998) the length scale shrinks by the
 * reference's factor 0.98 -- a default-real (single-precision) literal -- while
 *   1. the residual of the Laplacian system, sqrt(|A b_L - C_L|^2 h^2 / n), stays below
 *      res_tol / h,
 *   2. no wavenumber q = i pi / (32 s), i = 1..33, is amplified by the d/dx, d/dy or
 *      Laplacian stencil beyond 1.0001 (or turned negative, for the Laplacian), and
 *   3. at most log(0.6) / log(0.98) reductions (log(0.6) in single precision) have been made.
 * The first pass reduces h (and h_small with it) over the node's list, keeping the links
 * within 2 h; the second reduces h_small over the small list.  A moment matrix whose SVD does
 * not converge (the reference stops) ends the node's reduction here.  The caller rebuilds the
 * neighbour lists with the new lengths (sunset.F90:43-51).
 * ------------------------------------------------------------------------------------- */
static double adapt_res_tol(int order) {
    const int n = nsize_for(order);
    const double c = order == 4 ? 1.0e-3 : order == 6 ? 5.0e-3 : order == 8 ? 3.0e-2 : 1.0;
    return ((c * (double)(n * n * n * n)) * DBL_EPSILON) / (double)order;
}

typedef struct {
    SvdWork sw;
    double *amat, *gvec, *xvec, *bl, *bx, *by, *res, *dl, *dx, *dy;
    int *tl;
} AdaptWork;

static void adapt_node(OrSim *s, int i, int main_pass, AdaptWork *w) {
    const int order = main_pass ? s->cfg.morder : s->cfg.forder;
    const int n = nsize_for(order), nl = nsize_for(s->cfg.forder);
    const double rf = (double)0.98f, amp_tol = 1.0001;
    const double limit = (double)logf(0.6f) / log(rf);
    const double res_tol = adapt_res_tol(order);
    const int nk = 32;
    int *lk = s->ij_link + (size_t)i * s->nplink;
    for (int ii = 0;; ii++) {
        const double hh = (main_pass ? s->hs[i] : s->h[i]) * rf;
        const int cur = main_pass ? s->ij_count_small[i] : s->ij_count[i];
        int cnt = 0;
        for (int k = 0; k < cur; k++) {
            const int j = lk[k];
            const double rx = s->rx[i] - s->rx[j], ry = s->ry[i] - s->ry[j];
            if (sqrt(rx * rx + ry * ry) <= hh * ss) w->tl[cnt++] = j;
        }
        /* moment matrix over the temporary list, as in calc_labf_weights */
        memset(w->amat, 0, sizeof(double) * n * n);
        for (int k = 0; k < cnt; k++) {
            const int j = w->tl[k];
            const double x = -(s->rx[i] - s->rx[j]), y = -(s->ry[i] - s->ry[j]);
            const double qq = sqrt(x * x + y * y) / hh;
            const double ff1 = or_wab(qq, s->h2);
            or_abfs(s->cfg.forder, x / hh, y / hh, w->gvec);
            for (int m = 0; m < nl; m++) w->gvec[m] = w->gvec[m] * ff1;
            or_monomials(s->cfg.forder, x / hh, y / hh, w->xvec);
            for (int i2 = 0; i2 < n; i2++)
                for (int i1 = 0; i1 < n; i1++) w->amat[i2 * n + i1] = w->amat[i2 * n + i1] + w->xvec[i1] * w->gvec[i2];
        }
        const double thr = res_tol / hh;
        double hc;
        if (svd_factor(w->amat, n, &w->sw)) {
            hc = (2.0 * res_tol) / hh;
        } else {
            memset(w->bl, 0, sizeof(double) * n); w->bl[2] = (1.0 / hh) / hh; w->bl[4] = (1.0 / hh) / hh;
            memset(w->bx, 0, sizeof(double) * n); w->bx[0] = 1.0 / hh;
            memset(w->by, 0, sizeof(double) * n); w->by[1] = 1.0 / hh;
            svd_apply(&w->sw, n, w->bl);
            svd_apply(&w->sw, n, w->bx);
            svd_apply(&w->sw, n, w->by);
            /* residual of the Laplacian system */
            hc = 0.0;
            for (int i1 = 0; i1 < n; i1++) {
                double r = (i1 == 2 || i1 == 4) ? (-1.0 / hh) / hh : 0.0;
                for (int i2 = 0; i2 < n; i2++) r = r + w->amat[i2 * n + i1] * w->bl[i2];
                hc = hc + r * r;
            }
            hc = (hc * hh) * hh;
            hc = sqrt(hc / (double)n);
            if (hc < thr) {
                /* stencil amplification: the dot products of each link do not depend on q */
                for (int k = 0; k < cnt; k++) {
                    const int j = w->tl[k];
                    const double x = -(s->rx[i] - s->rx[j]), y = -(s->ry[i] - s->ry[j]);
                    const double qq = sqrt(x * x + y * y) / hh;
                    const double ff1 = or_wab(qq, s->h2);
                    or_abfs(s->cfg.forder, x / hh, y / hh, w->gvec);
                    for (int m = 0; m < nl; m++) w->gvec[m] = w->gvec[m] * ff1;
                    w->dl[k] = dotn(w->bl, w->gvec, n);
                    w->dx[k] = dotn(w->bx, w->gvec, n);
                    w->dy[k] = dotn(w->by, w->gvec, n);
                }
                for (int i1 = 1; i1 <= nk + 1 && hc < thr; i1++) {
                    const double q = (((double)i1 * pi) / s->sp[i]) / (double)nk;
                    double hl = 0.0, hx = 0.0, hy = 0.0;
                    for (int k = 0; k < cnt; k++) {
                        const int j = w->tl[k];
                        const double x = -(s->rx[i] - s->rx[j]), y = -(s->ry[i] - s->ry[j]);
                        hl = hl + (0.5 - (0.5 * cos(x * q)) * cos(y * q)) * w->dl[k];
                        hx = hx + (cos(y * q) * sin(x * q)) * w->dx[k];
                        hy = hy + (cos(x * q) * sin(y * q)) * w->dy[k];
                    }
                    hl = hl / (q * q);
                    hx = hx / q;
                    hy = hy / q;
                    if (hl > amp_tol || hl < 0.0) hc = (2.0 * res_tol) / hh;
                    if (fabs(hx) > amp_tol) hc = (2.0 * res_tol) / hh;
                    if (fabs(hy) > amp_tol) hc = (2.0 * res_tol) / hh;
                    if (isnan(hc)) hc = (2.0 * res_tol) / hh;
                }
            }
        }
        if ((double)ii > limit) hc = (2.0 * res_tol) / hh;
        if (hc >= thr) break; /* (a NaN residual compares false and is accepted, as there) */
        if (main_pass) {
            s->hs[i] = hh;
            s->ij_count_small[i] = cnt;
        } else {
            s->h[i] = hh;
            s->hs[i] = hh;
            for (int k = 0; k < cnt; k++) lk[k] = w->tl[k];
            s->ij_count[i] = cnt;
            s->ij_count_small[i] = cnt;
        }
    }
}

int or_adapt_stencils(OrSim *s) {
    if (!s->ij_count) return fail(s, "neighbours not built");
    const int nmax = nsize_for(s->cfg.forder > s->cfg.morder ? s->cfg.forder : s->cfg.morder);
#pragma omp parallel
    {
        AdaptWork w;
        svdw_init(&w.sw, nmax);
        w.amat = (double *)xcalloc((size_t)nmax * nmax, sizeof(double));
        w.gvec = (double *)xcalloc(nmax, sizeof(double)); w.xvec = (double *)xcalloc(nmax, sizeof(double));
        w.bl = (double *)xcalloc(nmax, sizeof(double)); w.bx = (double *)xcalloc(nmax, sizeof(double));
        w.by = (double *)xcalloc(nmax, sizeof(double)); w.res = NULL;
        w.dl = (double *)xcalloc(s->nplink + 1, sizeof(double)); w.dx = (double *)xcalloc(s->nplink + 1, sizeof(double));
        w.dy = (double *)xcalloc(s->nplink + 1, sizeof(double)); w.tl = (int *)xcalloc(s->nplink + 1, sizeof(int));
#pragma omp for schedule(dynamic, 16)
        for (int i = 0; i < s->npfb; i++) {
            if (s->type[i] <= 2 || s->type[i] == 998) continue;
            adapt_node(s, i, 0, &w);
            adapt_node(s, i, 1, &w);
        }
        svdw_free(&w.sw);
        free(w.amat); free(w.gvec); free(w.xvec); free(w.bl); free(w.bx); free(w.by);
        free(w.dl); free(w.dx); free(w.dy); free(w.tl);
    }
    return or_find_neighbours(s);
}

int or_calc_boundary_weights(OrSim *s) {
    if (s->nb == 0) return 0;
    const int npfb = s->npfb, nplink = s->nplink, nb = s->nb;
    FREE(s->wb_grad2);
    s->wb_grad2 = (double *)xcalloc((size_t)3 * nplink * nb, sizeof(double));
#define WB(jj, k, c) s->wb_grad2[((size_t)(jj) * nplink + (k)) * 3 + (c)]
#define WG(i, k, c) s->w_grad[2 * ((size_t)(i) * nplink + (k)) + (c)]
#define WL(i, k) s->w_lap[(size_t)(i) * nplink + (k)]
#define WH(i, k) s->w_hyp[(size_t)(i) * nplink + (k)]
    /* preface, :541-565: boundary nodes keep only links on their own layer and their FD
       children */
    int *tmp = (int *)xcalloc(nplink, sizeof(int));
    for (int jj = 0; jj < nb; jj++) {
        int i = s->boundary_list[jj];
        int kk = s->type[i], nsize = s->ij_count[i];
        int *lk = s->ij_link + (size_t)i * nplink;
        memcpy(tmp, lk, sizeof(int) * nsize);
        for (int k = 0; k < nplink; k++) lk[k] = -1;
        s->ij_count[i] = 0;
        for (int k = 0; k < nsize; k++) {
            int j = tmp[k];
            if (s->type[j] == kk) lk[s->ij_count[i]++] = j;
            if (j < npfb && s->fd_parent[j] == i) lk[s->ij_count[i]++] = j;
        }
        s->ij_count_small[i] = s->ij_count[i];
    }
    free(tmp);

    /* boundary node: normal operators, :572-612 */
    for (int jj = 0; jj < nb; jj++) {
        int i = s->boundary_list[jj];
        double dx = s->sp[i], dx2 = dx * dx;
        for (int k = 0; k < nplink; k++) {
            WG(i, k, 0) = 0.0; WG(i, k, 1) = 0.0; WH(i, k) = 0.0;
            WB(jj, k, 0) = 0.0; WB(jj, k, 1) = 0.0; WB(jj, k, 2) = 0.0;
        }
        const int *lk = s->ij_link + (size_t)i * nplink;
        for (int k = 0; k < s->ij_count[i]; k++) {
            int j = lk[k];
            if (j >= npfb) continue;
            if (s->fd_parent[j] != i) continue;
            int t = s->type[j];
            if (j == i) WG(i, k, 0) = 0.0;
            if (t == -1) WG(i, k, 0) = 4.0 / dx;
            if (t == -2) WG(i, k, 0) = -(3.0 / dx);
            if (t == -3) WG(i, k, 0) = (4.0 / 3.0) / dx;
            if (t == -4) WG(i, k, 0) = -(0.25 / dx);
            if (j == i) WB(jj, k, 0) = 0.0;
            if (t == -1) WB(jj, k, 0) = -((104.0 / 12.0) / dx2);
            if (t == -2) WB(jj, k, 0) = (114.0 / 12.0) / dx2;
            if (t == -3) WB(jj, k, 0) = -((56.0 / 12.0) / dx2);
            if (t == -4) WB(jj, k, 0) = (11.0 / 12.0) / dx2;
        }
    }
    /* first row: normal operators, :615-645 */
    for (int jj = 0; jj < nb; jj++) {
        int i = s->boundary_list[jj] + 1;
        double dx = s->sp[i], dx2 = dx * dx; /* dx2 of the boundary node's row: same s */
        for (int k = 0; k < nplink; k++) { WG(i, k, 0) = 0.0; WG(i, k, 1) = 0.0; WL(i, k) = 0.0; }
        const int *lk = s->ij_link + (size_t)i * nplink;
        int par = s->fd_parent[i];
        for (int k = 0; k < s->ij_count[i]; k++) {
            int j = lk[k];
            if (j >= npfb) continue;
            int t = s->type[j], same = s->fd_parent[j] == par;
            if (j == par) WG(i, k, 0) = -(0.25 / dx);
            if (j == i) WG(i, k, 0) = 0.0;
            if (t == -2 && same) WG(i, k, 0) = 1.5 / dx;
            if (t == -3 && same) WG(i, k, 0) = -(0.5 / dx);
            if (t == -4 && same) WG(i, k, 0) = (1.0 / 12.0) / dx;
            if (j == par) WL(i, k) = (11.0 / 12.0) / dx2;
            if (j == i) WL(i, k) = 0.0;
            if (t == -2 && same) WL(i, k) = (6.0 / 12.0) / dx2;
            if (t == -3 && same) WL(i, k) = (4.0 / 12.0) / dx2;
            if (t == -4 && same) WL(i, k) = -((1.0 / 12.0) / dx2);
        }
    }
    /* second row: normal operators, :648-676 */
    for (int jj = 0; jj < nb; jj++) {
        int i = s->boundary_list[jj] + 2;
        double dx = s->sp[i], dx2 = dx * dx;
        for (int k = 0; k < nplink; k++) { WG(i, k, 0) = 0.0; WG(i, k, 1) = 0.0; WL(i, k) = 0.0; }
        const int *lk = s->ij_link + (size_t)i * nplink;
        int par = s->fd_parent[i];
        for (int k = 0; k < s->ij_count[i]; k++) {
            int j = lk[k];
            if (j >= npfb) continue;
            int t = s->type[j], same = s->fd_parent[j] == par;
            if (j == par) WG(i, k, 0) = (1.0 / 12.0) / dx;
            if (t == -1 && same) WG(i, k, 0) = -((8.0 / 12.0) / dx);
            if (j == i) WG(i, k, 0) = (0.0 / 12.0) / dx;
            if (t == -3 && same) WG(i, k, 0) = (8.0 / 12.0) / dx;
            if (t == -4 && same) WG(i, k, 0) = -((1.0 / 12.0) / dx);
            if (j == par) WL(i, k) = -((1.0 / 12.0) / dx2);
            if (t == -1 && same) WL(i, k) = (16.0 / 12.0) / dx2;
            if (j == i) WL(i, k) = (0.0 / 12.0) / dx2;
            if (t == -3 && same) WL(i, k) = (16.0 / 12.0) / dx2;
            if (t == -4 && same) WL(i, k) = -((1.0 / 12.0) / dx2);
        }
    }

    SvdWork sw;
    svdw_init(&sw, 6);
    double amat[36], bvect[6], bvectt[6], bvecthyp[6], gvec[6];
    /* boundary node: transverse operators, :688-755 */
    for (int jj = 0; jj < nb; jj++) {
        int i = s->boundary_list[jj];
        double xt = -s->rny[i], yt = s->rnx[i], hh = s->h[i];
        assemble_1d(s, i, xt, yt, hh, amat);
        memset(bvect, 0, sizeof bvect); bvect[0] = 1.0;
        memset(bvectt, 0, sizeof bvectt); bvectt[1] = 1.0;
        memset(bvecthyp, 0, sizeof bvecthyp); bvecthyp[3] = -1.0;
        if (svd_factor(amat, 6, &sw)) { svdw_free(&sw); return fail(s, "svd_solve: no convergence (boundary node %d)", i); }
        svd_apply(&sw, 6, bvect);
        svd_apply(&sw, 6, bvectt);
        svd_apply(&sw, 6, bvecthyp);
        const int *lk = s->ij_link + (size_t)i * nplink;
        for (int k = 0; k < s->ij_count[i]; k++) {
            int j = lk[k];
            if (s->type[j] != s->type[i]) continue;
            abf_1d_link(s, i, j, xt, yt, hh, gvec);
            WG(i, k, 1) = dot6(bvect, gvec) / hh;
            WB(jj, k, 1) = (dot6(bvectt, gvec) / hh) / hh;
            WH(i, k) = WH(i, k) + dot6(bvecthyp, gvec);
        }
    }
    /* first and second rows: transverse operators on a tangent rotated by the tangential
       gradient of the resolution, :758-955 */
    for (int row = 1; row <= 2; row++) {
        for (int jj = 0; jj < nb; jj++) {
            int i = s->boundary_list[jj] + row;
            double hh = s->h[i];
            int ii = s->fd_parent[i];
            double grads = 0.0;
            const int *lp = s->ij_link + (size_t)ii * nplink;
            for (int k = 0; k < s->ij_count[ii]; k++) {
                int j = lp[k];
                grads = grads + (s->sp[j] - s->sp[ii]) * WG(ii, k, 1);
            }
            grads = -atan(grads);
            double xt = cos(grads) * (-s->rny[i]) - sin(grads) * s->rnx[i];
            double yt = sin(grads) * (-s->rny[i]) + cos(grads) * s->rnx[i];
            assemble_1d(s, i, xt, yt, hh, amat);
            memset(bvect, 0, sizeof bvect); bvect[0] = 1.0;
            memset(bvectt, 0, sizeof bvectt); bvectt[1] = 1.0;
            if (svd_factor(amat, 6, &sw)) { svdw_free(&sw); return fail(s, "svd_solve: no convergence (row node %d)", i); }
            svd_apply(&sw, 6, bvect);
            svd_apply(&sw, 6, bvectt);
            const int *lk = s->ij_link + (size_t)i * nplink;
            for (int k = 0; k < s->ij_count[i]; k++) {
                int j = lk[k];
                if (s->type[j] != s->type[i]) continue;
                abf_1d_link(s, i, j, xt, yt, hh, gvec);
                WG(i, k, 1) = dot6(bvect, gvec) / hh;
                WL(i, k) = WL(i, k) + (dot6(bvectt, gvec) / hh) / hh;
            }
            for (int k = 0; k < s->ij_count[i]; k++)
                WG(i, k, 1) = (1.0 / cos(grads)) * WG(i, k, 1) - tan(grads) * WG(i, k, 0);
        }
    }
    svdw_free(&sw);

    /* wall curvature 1/R, :965-982 */
    double *ooR = (double *)xcalloc(nb, sizeof(double));
    for (int jj = 0; jj < nb; jj++) {
        int i = s->boundary_list[jj];
        if (s->type[i] != 0) continue;
        double tmp_t = 0.0;
        const int *lk = s->ij_link + (size_t)i * nplink;
        for (int k = 0; k < s->ij_count[i]; k++) {
            int j = lk[k];
            if (s->type[j] != s->type[i]) continue;
            double tmp_n = ((s->rnx[j] * s->rnx[i] + s->rny[j] * s->rny[i]) + 0.0 * 0.0) - 1.0;
            tmp_t = tmp_t + WB(jj, k, 1) * tmp_n;
        }
        ooR[jj] = sqrt(fabs(tmp_t));
    }
    /* outflow: reverse the first-derivative weights, :986-991 */
    for (int jj = 0; jj < nb; jj++) {
        int i = s->boundary_list[jj];
        if (s->type[i] == 2)
            for (int k = 0; k < nplink; k++) { WG(i, k, 0) = -WG(i, k, 0); WG(i, k, 1) = -WG(i, k, 1); }
    }
    /* divergence term in the Laplacian of rows 1 and 2, :994-1003 */
    for (int jj = 0; jj < nb; jj++) {
        int i = s->boundary_list[jj] + 1;
        if (s->type[i - 1] == 0)
            for (int k = 0; k < nplink; k++) WL(i, k) = WL(i, k) + (WG(i, k, 0) * ooR[jj]) / (1.0 + ooR[jj] * s->sp[i]);
        i = s->boundary_list[jj] + 2;
        if (s->type[i - 2] == 0)
            for (int k = 0; k < nplink; k++)
                WL(i, k) = WL(i, k) + (WG(i, k, 0) * ooR[jj]) / (1.0 + (2.0 * ooR[jj]) * s->sp[i]);
    }
    /* walls: second normal derivative with the curvature term, Laplacian = sum, :1007-1016 */
    for (int jj = 0; jj < nb; jj++) {
        int i = s->boundary_list[jj];
        if (s->type[i] != 0) continue;
        for (int k = 0; k < s->ij_count[i]; k++) {
            WB(jj, k, 0) = WB(jj, k, 0) + WG(i, k, 0) * ooR[jj];
            WL(i, k) = WB(jj, k, 0) + WB(jj, k, 1);
        }
    }
    /* rows 1 and 2: first derivatives from the normal-tangent frame to x-y, :1019-1035 */
    for (int jj = 0; jj < nb; jj++) {
        int ib = s->boundary_list[jj];
        double xn = s->rnx[ib], yn = s->rny[ib];
        for (int row = 1; row <= 2; row++) {
            int i = ib + row;
            for (int k = 0; k < s->ij_count[i]; k++) {
                double g1 = WG(i, k, 0), g2 = WG(i, k, 1);
                WG(i, k, 0) = (0.0 + xn * g1) + (-yn) * g2;
                WG(i, k, 1) = (0.0 + yn * g1) + xn * g2;
            }
        }
    }
    free(ooR);
#undef WB
#undef WG
#undef WL
#undef WH
    return 0;
}

/* labf.F90:396-451 */
int or_calc_labf_sums(OrSim *s) {
    const int npfb = s->npfb, nplink = s->nplink;
    const double L = s->cfg.L_char;
    FREE(s->w_grad_sum); FREE(s->w_lap_sum); FREE(s->w_hyp_sum);
    s->w_grad_sum = (double *)xcalloc(2 * (size_t)npfb, sizeof(double));
    s->w_lap_sum = (double *)xcalloc(npfb, sizeof(double));
    s->w_hyp_sum = (double *)xcalloc(npfb, sizeof(double));
#pragma omp parallel for schedule(static)
    for (int i = 0; i < npfb; i++) {
        double gx = 0.0, gy = 0.0, lp = 0.0, hy = 0.0;
        for (int k = 0; k < s->ij_count[i]; k++) {
            size_t o = (size_t)i * nplink + k;
            hy = hy + s->w_hyp[o];
            gx = gx + s->w_grad[2 * o];
            gy = gy + s->w_grad[2 * o + 1];
            lp = lp + s->w_lap[o];
        }
        s->w_grad_sum[2 * i] = gx / L;
        s->w_grad_sum[2 * i + 1] = gy / L;
        for (int k = 0; k < nplink; k++) {
            size_t o = (size_t)i * nplink + k;
            s->w_grad[2 * o] = s->w_grad[2 * o] / L;
            s->w_grad[2 * o + 1] = s->w_grad[2 * o + 1] / L;
        }
        s->w_lap_sum[i] = (lp / L) / L;
        for (int k = 0; k < nplink; k++) {
            size_t o = (size_t)i * nplink + k;
            s->w_lap[o] = (s->w_lap[o] / L) / L;
        }
        s->w_hyp_sum[i] = hy;
    }
    /* second derivatives on the boundary, :426-446 */
    if (s->nb != 0) {
        FREE(s->wb_grad2_sum);
        s->wb_grad2_sum = (double *)xcalloc(3 * (size_t)s->nb, sizeof(double));
        for (int jj = 0; jj < s->nb; jj++) {
            int i = s->boundary_list[jj];
            double *sum = s->wb_grad2_sum + 3 * jj;
            for (int k = 0; k < s->ij_count[i]; k++)
                for (int c = 0; c < 3; c++) sum[c] = sum[c] + s->wb_grad2[((size_t)jj * nplink + k) * 3 + c];
            for (int c = 0; c < 3; c++) sum[c] = (sum[c] / L) / L;
            for (int k = 0; k < nplink; k++)
                for (int c = 0; c < 3; c++) {
                    double *w = &s->wb_grad2[((size_t)jj * nplink + k) * 3 + c];
                    *w = (*w / L) / L;
                }
        }
    }
    return 0;
}

/* labf.F90:1723-1811 */
int or_filter_coefficients(OrSim *s) {
    const int npfb = s->npfb, nplink = s->nplink;
    double *fc = (double *)xcalloc(npfb, sizeof(double));
    const double oosqrt2 = 1.0 / sqrt(2.0);
#pragma omp parallel for schedule(static)
    for (int ii = 0; ii < s->n_internal; ii++) {
        int i = s->internal_list[ii];
        double lscal = (2.0 * s->h[i]) * sqrt(pi / (double)s->ij_count[i]);
        double tmp = ((2.0 / 3.0) * pi) / lscal;
        double lsum = 0.0;
        const int *lk = s->ij_link + (size_t)i * nplink;
        for (int k = 0; k < s->ij_count[i]; k++) {
            int j = lk[k];
            double x = s->rx[j] - s->rx[i], y = s->ry[j] - s->ry[i];
            double fji = 1.0 - cos(tmp * x) * cos(tmp * y);
            lsum = lsum + fji * s->w_hyp[(size_t)i * nplink + k];
        }
        fc[i] = (2.0 / 3.0) / lsum;
        int t = s->type[i];
        if (t < 0 && s->type[s->fd_parent[i]] == 0) {
            if (t == -1) fc[i] = (fc[i] * 0.5) * oosqrt2;
            if (t == -2) fc[i] = fc[i] * 0.5;
            if (t == -3) fc[i] = fc[i] * oosqrt2;
            if (t == -4 || t == 998) fc[i] = fc[i] * oosqrt2;
        }
    }
    for (int ii = 0; ii < s->nb; ii++) {
        int i = s->boundary_list[ii];
        double lscal = s->sp[i];
        double tmp = ((2.0 / 3.0) * pi) / lscal;
        double lsum = 0.0;
        const int *lk = s->ij_link + (size_t)i * nplink;
        for (int k = 0; k < s->ij_count[i]; k++) {
            int j = lk[k];
            double x = s->rx[j] - s->rx[i], y = s->ry[j] - s->ry[i];
            double fji = 1.0 - cos(tmp * sqrt(x * x + y * y));
            lsum = lsum + fji * s->w_hyp[(size_t)i * nplink + k];
        }
        fc[i] = (1.0 / 3.0) / lsum;
        fc[i] = fc[i] * 0.5;
    }
#pragma omp parallel for schedule(static)
    for (int i = 0; i < npfb; i++) {
        double sum = 0.0;
        for (int k = 0; k < s->ij_count[i]; k++) {
            size_t o = (size_t)i * nplink + k;
            s->w_hyp[o] = s->w_hyp[o] * fc[i];
            sum = sum + s->w_hyp[o];
        }
        s->w_hyp_sum[i] = sum;
    }
    free(fc);
    s->have_weights = 1;
    return 0;
}

int or_setup_all(OrSim *s) { /* sunset.F90:51-60 */
    if (or_find_neighbours(s)) return -1;
    if (or_calc_labf_weights(s)) return -1;
    if (s->nb != 0 && or_calc_boundary_weights(s)) return -1;
    if (or_calc_labf_sums(s)) return -1;
    if (or_filter_coefficients(s)) return -1;
    return 0;
}

int or_get_weights(OrSim *s, double *w_grad, double *w_lap, double *w_hyp, double *w_grad_sum,
                   double *w_lap_sum, double *w_hyp_sum, double *vol) {
    if (!s->have_weights) return fail(s, "weights not built");
    size_t nn = (size_t)s->npfb * s->nplink;
    if (w_grad) memcpy(w_grad, s->w_grad, 2 * nn * sizeof(double));
    if (w_lap) memcpy(w_lap, s->w_lap, nn * sizeof(double));
    if (w_hyp) memcpy(w_hyp, s->w_hyp, nn * sizeof(double));
    if (w_grad_sum) memcpy(w_grad_sum, s->w_grad_sum, 2 * (size_t)s->npfb * sizeof(double));
    if (w_lap_sum) memcpy(w_lap_sum, s->w_lap_sum, (size_t)s->npfb * sizeof(double));
    if (w_hyp_sum) memcpy(w_hyp_sum, s->w_hyp_sum, (size_t)s->npfb * sizeof(double));
    if (vol) memcpy(vol, s->vol, (size_t)s->npfb * sizeof(double));
    return 0;
}

int or_set_neighbours_weights(OrSim *s, int nplink, const int *ij_count, const int *ij_count_small,
                              const int *ij_link, const double *w_grad, const double *w_lap,
                              const double *w_hyp, const double *w_grad_sum, const double *w_lap_sum,
                              const double *w_hyp_sum, const double *vol) {
    const int npfb = s->npfb;
    free_links(s);
    s->nplink = nplink;
    size_t nn = (size_t)npfb * nplink;
    s->ij_count = (int *)xcalloc(npfb, sizeof(int));
    s->ij_count_small = (int *)xcalloc(npfb, sizeof(int));
    s->ij_link = (int *)xcalloc(nn, sizeof(int));
    memcpy(s->ij_count, ij_count, npfb * sizeof(int));
    memcpy(s->ij_count_small, ij_count_small, npfb * sizeof(int));
    for (size_t o = 0; o < nn; o++) s->ij_link[o] = ij_link[o] - 1;
    alloc_weights(s);
    memcpy(s->w_grad, w_grad, 2 * nn * sizeof(double));
    memcpy(s->w_lap, w_lap, nn * sizeof(double));
    memcpy(s->w_hyp, w_hyp, nn * sizeof(double));
    s->w_grad_sum = (double *)xcalloc(2 * (size_t)npfb, sizeof(double));
    s->w_lap_sum = (double *)xcalloc(npfb, sizeof(double));
    s->w_hyp_sum = (double *)xcalloc(npfb, sizeof(double));
    memcpy(s->w_grad_sum, w_grad_sum, 2 * (size_t)npfb * sizeof(double));
    memcpy(s->w_lap_sum, w_lap_sum, npfb * sizeof(double));
    memcpy(s->w_hyp_sum, w_hyp_sum, npfb * sizeof(double));
    memcpy(s->vol, vol, npfb * sizeof(double));
    for (int i = 0; i < npfb; i++)
        for (int k = 0; k < ij_count[i]; k++)
            if (s->ij_link[(size_t)i * nplink + k] < 0 || s->ij_link[(size_t)i * nplink + k] >= s->np)
                return fail(s, "link out of range at node %d", i);
    s->have_weights = 1;
    return 0;
}

/* ---------------------------------------------------------------------------------------
 * derivatives.F90 (2-D)
 * ------------------------------------------------------------------------------------- */
/* calc_gradient :26-71; comp = 0 both, 1 = x only, 2 = y only (calc_gradient_only :416-464) */
static void calc_gradient(const OrSim *s, const double *phi, double *gx, double *gy, int comp) {
    const int nplink = s->nplink;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < s->npfb; i++) {
        double g1 = 0.0, g2 = 0.0;
        const int *lk = s->ij_link + (size_t)i * nplink;
        const double *wg = s->w_grad + 2 * (size_t)i * nplink;
        for (int k = 0; k < s->ij_count_small[i]; k++) {
            double pj = phi[lk[k]];
            if (comp != 2) g1 = g1 + pj * wg[2 * k];
            if (comp != 1) g2 = g2 + pj * wg[2 * k + 1];
        }
        if (comp != 2) gx[i] = g1 - phi[i] * s->w_grad_sum[2 * i];
        if (comp != 1) gy[i] = g2 - phi[i] * s->w_grad_sum[2 * i + 1];
    }
}
/* calc_laplacian :73-116 */
static void calc_laplacian(const OrSim *s, const double *phi, double *lap) {
    const int nplink = s->nplink;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < s->npfb; i++) {
        double l = 0.0;
        const int *lk = s->ij_link + (size_t)i * nplink;
        const double *wl = s->w_lap + (size_t)i * nplink;
        for (int k = 0; k < s->ij_count_small[i]; k++) l = l + phi[lk[k]] * wl[k];
        lap[i] = l - phi[i] * s->w_lap_sum[i];
    }
}
/* calc_laplacian_transverse_only_on_bound :306-358 */
static void calc_laplacian_transverse(const OrSim *s, const double *phi, double *lap) {
    const int nplink = s->nplink;
#pragma omp parallel for schedule(static)
    for (int ii = 0; ii < s->n_internal; ii++) {
        int i = s->internal_list[ii];
        double l = 0.0;
        const int *lk = s->ij_link + (size_t)i * nplink;
        const double *wl = s->w_lap + (size_t)i * nplink;
        for (int k = 0; k < s->ij_count_small[i]; k++) l = l + phi[lk[k]] * wl[k];
        lap[i] = l - phi[i] * s->w_lap_sum[i];
    }
    for (int ii = 0; ii < s->nb; ii++) {
        int i = s->boundary_list[ii];
        double l = 0.0;
        const int *lk = s->ij_link + (size_t)i * nplink;
        for (int k = 0; k < s->ij_count_small[i]; k++)
            l = l + phi[lk[k]] * s->wb_grad2[((size_t)ii * nplink + k) * 3 + 1];
        lap[i] = l - phi[i] * s->wb_grad2_sum[3 * ii + 1];
    }
}
/* calc_filtered_var :360-414 (in place on phi(1:npfb)) */
static void calc_filtered_var(const OrSim *s, double *phi, double *work) {
    const int nplink = s->nplink;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < s->npfb; i++) {
        double t = 0.0;
        const int *lk = s->ij_link + (size_t)i * nplink;
        const double *wh = s->w_hyp + (size_t)i * nplink;
        for (int k = 0; k < s->ij_count[i]; k++) t = t + phi[lk[k]] * wh[k];
        work[i] = phi[i] + (t - phi[i] * s->w_hyp_sum[i]);
    }
    memcpy(phi, work, sizeof(double) * s->npfb);
}
/* calc_filter_term :466-511 */
static void calc_filter_term(const OrSim *s, const double *phi, double *out) {
    const int nplink = s->nplink;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < s->npfb; i++) {
        double t = 0.0;
        const int *lk = s->ij_link + (size_t)i * nplink;
        const double *wh = s->w_hyp + (size_t)i * nplink;
        for (int k = 0; k < s->ij_count[i]; k++) t = t + phi[lk[k]] * wh[k];
        out[i] = t - phi[i] * s->w_hyp_sum[i];
    }
}

static double *extend_to_np(const OrSim *s, const double *phi) {
    double *e = (double *)xcalloc(s->np, sizeof(double));
    memcpy(e, phi, sizeof(double) * s->npfb);
    for (int j = s->npfb; j < s->np; j++) e[j] = e[s->irel[j]];
    return e;
}

int or_calc_gradient(OrSim *s, const double *phi, double *grad) {
    if (!s->have_weights) return fail(s, "weights not built");
    double *e = extend_to_np(s, phi);
    double *gx = (double *)xcalloc(s->npfb, sizeof(double)), *gy = (double *)xcalloc(s->npfb, sizeof(double));
    calc_gradient(s, e, gx, gy, 0);
    for (int i = 0; i < s->npfb; i++) { grad[2 * i] = gx[i]; grad[2 * i + 1] = gy[i]; }
    free(e); free(gx); free(gy);
    return 0;
}
int or_calc_laplacian(OrSim *s, const double *phi, double *lap) {
    if (!s->have_weights) return fail(s, "weights not built");
    double *e = extend_to_np(s, phi);
    calc_laplacian(s, e, lap);
    free(e);
    return 0;
}
int or_calc_filtered_var(OrSim *s, const double *phi, double *out) {
    if (!s->have_weights) return fail(s, "weights not built");
    double *e = extend_to_np(s, phi);
    double *w = (double *)xcalloc(s->npfb, sizeof(double));
    calc_filtered_var(s, e, w);
    memcpy(out, e, sizeof(double) * s->npfb);
    free(e); free(w);
    return 0;
}
int or_calc_filter_term(OrSim *s, const double *phi, double *out) {
    if (!s->have_weights) return fail(s, "weights not built");
    double *e = extend_to_np(s, phi);
    calc_filter_term(s, e, out);
    free(e);
    return 0;
}

/* ---------------------------------------------------------------------------------------
 * conf_transforms.F90 (2-D parts)
 * ------------------------------------------------------------------------------------- */
/* eigens 2x2, :399-444. R column-major: R[0]=R(1,1), R[1]=R(2,1), R[2]=R(1,2), R[3]=R(2,2) */
static void eigens2(double a, double b, double d, double *l, double *R) {
    if (fabs(b) <= doublesmall) {
        l[0] = a; l[1] = d;
        R[0] = 1.0; R[1] = 0.0; R[2] = 0.0; R[3] = 1.0;
    } else {
        double tr = a + d;
        double det = a * d - b * b;
        double temp = (0.25 * tr) * tr - det;
        if (temp <= doublesmall) temp = 0.0;
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
/* 2x2 column-major matmul, gfortran inline order: c(i,j) = a(i,1)b(1,j) + a(i,2)b(2,j) */
static void mm2(const double *a, const double *b, double *c) {
    double t[4];
    t[0] = a[0] * b[0] + a[2] * b[1];
    t[1] = a[1] * b[0] + a[3] * b[1];
    t[2] = a[0] * b[2] + a[2] * b[3];
    t[3] = a[1] * b[2] + a[3] * b[3];
    memcpy(c, t, sizeof(t));
}
static void tr2(const double *a, double *t) { t[0] = a[0]; t[1] = a[2]; t[2] = a[1]; t[3] = a[3]; }

/* log_conf_c_from_psi :133-169 (2-D leaves c_zz untouched) */
static void log_conf_c_from_psi(double pxx, double pxy, double pyy, double *cxx, double *cxy, double *cyy) {
    double L[2], R[4], RT[4], Lm[4], C[4];
    eigens2(pxx, pxy, pyy, L, R);
    tr2(R, RT);
    Lm[0] = exp(L[0]); Lm[1] = 0.0; Lm[2] = 0.0; Lm[3] = exp(L[1]);
    mm2(Lm, RT, C);
    mm2(R, C, C);
    *cxx = C[0]; *cxy = C[1]; *cyy = C[3];
}
/* log_conf_psi_from_c :177-215 */
static void log_conf_psi_from_c(double cxx, double cxy, double cyy, double *pxx, double *pxy, double *pyy) {
    double L[2], R[4], RT[4], Lm[4], P[4];
    eigens2(cxx, cxy, cyy, L, R);
    tr2(R, RT);
    Lm[0] = log(L[0]); Lm[1] = 0.0; Lm[2] = 0.0; Lm[3] = log(L[1]);
    mm2(Lm, RT, P);
    mm2(R, P, P);
    *pxx = P[0]; *pxy = P[1]; *pyy = P[3];
}
/* cholesky_c_from_psi :33-74 */
static void cholesky_c_from_psi(const OrSim *s, double pxx, double pxy, double pyy, double pzz,
                                double *cxx, double *cxy, double *cyy, double *czz) {
    if (s->cfg.fenep) {
        double L2 = s->cfg.fenep_l2;
        double Jxx = exp(2.0 * pxx), Jxy = exp(pxx) * pxy, Jyy = pxy * pxy + exp(2.0 * pyy);
        double Jzz = exp(2.0 * pzz);
        double fq = L2 / ((((L2 - 3.0) + Jxx) + Jyy) + Jzz);
        *cxx = Jxx * fq; *cxy = Jxy * fq; *cyy = Jyy * fq; *czz = Jzz * fq;
    } else {
        double e = exp(pxx);
        *cxx = e * e;
        *cxy = exp(pxx) * pxy;
        *cyy = pxy * pxy + exp(2.0 * pyy);
        *czz = 1.0;
    }
}
/* cholesky_psi_from_c :82-125 */
static void cholesky_psi_from_c(const OrSim *s, double cxx, double cxy, double cyy, double czz,
                                double *pxx, double *pxy, double *pyy, double *pzz) {
    double xx, xy, yy, zz;
    if (s->cfg.fenep) {
        double L2 = s->cfg.fenep_l2;
        double fr = (L2 - 3.0) / (L2 - ((cxx + cyy) + czz));
        double Jxx = cxx * fr, Jxy = cxy * fr, Jyy = cyy * fr, Jzz = czz * fr;
        xx = sqrt(Jxx);
        xy = Jxy / xx;
        yy = sqrt(Jyy - xy * xy);
        zz = sqrt(Jzz);
    } else {
        xx = sqrt(cxx);
        xy = cxy / (xx);
        yy = (sqrt(cyy - xy * xy));
        zz = sqrt(czz);
    }
    *pxx = log(xx); *pxy = xy; *pyy = log(yy); *pzz = log(zz);
}

/* ---------------------------------------------------------------------------------------
 * Fields: setup_flow.F90:24-173 initial_solution, step.F90:514-567
 * ------------------------------------------------------------------------------------- */
static void alloc_fields(OrSim *s) {
    free_fields(s);
    int np = s->np, npfb = s->npfb;
#define A(p, n) s->p = (double *)xcalloc(n, sizeof(double))
    A(ro, np); A(rou, np); A(rov, np); A(row, np); A(u, np); A(v, np); A(w, np); A(p, np);
    A(psixx, np); A(psixy, np); A(psiyy, np); A(psizz, np); A(cxx, np); A(cxy, np); A(cyy, np); A(czz, np);
    A(rhs_ro, npfb); A(rhs_rou, npfb); A(rhs_rov, npfb); A(rhs_row, npfb);
    A(rhs_xx, npfb); A(rhs_xy, npfb); A(rhs_yy, npfb); A(rhs_zz, npfb);
#undef A
}

/* reapply_mirror_bcs, mirror_boundaries.F90:263-352 (no pgrad) */
static void reapply_mirror_bcs(OrSim *s) {
    const int form = s->cfg.form;
    for (int j = s->npfb; j < s->np; j++) {
        int i = s->irel[j], vr = s->vrel[j];
        s->ro[j] = s->ro[i];
        if (vr == 1) { s->rou[j] = s->rou[i]; s->rov[j] = s->rov[i]; }
        else if (vr == 2) { s->rou[j] = -s->rou[i]; s->rov[j] = s->rov[i]; }
        else if (vr == 3) { s->rou[j] = s->rou[i]; s->rov[j] = -s->rov[i]; }
        else if (vr == 4) { s->rou[j] = -s->rou[i]; s->rov[j] = -s->rov[i]; }
        if (form == OR_FORM_NEWT) continue;
        int flip = (vr == 2 || vr == 3);
        if (form != OR_FORM_DI) {
            s->psixx[j] = s->psixx[i];
            s->psixy[j] = flip ? -s->psixy[i] : s->psixy[i];
            s->psiyy[j] = s->psiyy[i];
            s->psizz[j] = s->psizz[i];
        } else {
            s->cxx[j] = s->cxx[i];
            s->cxy[j] = flip ? -s->cxy[i] : s->cxy[i];
            s->cyy[j] = s->cyy[i];
            s->czz[j] = s->czz[i];
        }
    }
}

static void get_velocity_from_momentum(OrSim *s) { /* step.F90:514-529 */
#pragma omp parallel for schedule(static)
    for (int i = 0; i < s->np; i++) {
        double ooro = 1.0 / s->ro[i];
        s->u[i] = s->rou[i] * ooro;
        s->v[i] = s->rov[i] * ooro;
        s->w[i] = s->row[i] * ooro;
    }
}

static void get_c_from_psi(OrSim *s) { /* step.F90:531-567 */
    if (s->cfg.form == OR_FORM_LC) {
#pragma omp parallel for schedule(static)
        for (int i = 0; i < s->np; i++)
            log_conf_c_from_psi(s->psixx[i], s->psixy[i], s->psiyy[i], &s->cxx[i], &s->cxy[i], &s->cyy[i]);
    } else if (s->cfg.form == OR_FORM_CHL) {
#pragma omp parallel for schedule(static)
        for (int i = 0; i < s->np; i++)
            cholesky_c_from_psi(s, s->psixx[i], s->psixy[i], s->psiyy[i], s->psizz[i], &s->cxx[i],
                                &s->cxy[i], &s->cyy[i], &s->czz[i]);
    }
}

/* update_u_inflow, characteristic_boundaries.F90:262-300: with velocity control the inflow
   velocity ramps linearly to u_inflow_end over ramp_time; it is updated only while
   time <= ramp_time, so it keeps its last ramp value after that */
static void update_u_inflow(OrSim *s) {
    if (s->cfg.inflow_velocity_control != 1) return;
    const double t = s->time, rt = s->cfg.ramp_time;
    double um;
    if (t <= rt) um = s->cfg.u_inflow_start + ((s->cfg.u_inflow_end - s->cfg.u_inflow_start) * t) / rt;
    else um = s->cfg.u_inflow_end;
    if (t <= rt)
        for (int jj = 0; jj < s->nb; jj++)
            if (s->type[s->boundary_list[jj]] == 1) s->u_inflow_local[jj] = um;
}

static void apply_time_dependent_bounds(OrSim *s) { /* characteristic_boundaries.F90:191-257 */
    update_u_inflow(s);
    for (int jj = 0; jj < s->nb; jj++) {
        int i = s->boundary_list[jj];
        if (s->type[i] == 0) { s->rou[i] = 0.0; s->rov[i] = 0.0; s->row[i] = 0.0; }
        else if (s->type[i] == 1 && s->cfg.inflow_type == 1) { /* hard inflow: prescribed velocity */
            s->rou[i] = s->u_inflow_local[jj] * s->ro[i];
            s->rov[i] = 0.0;
            s->row[i] = 0.0;
        }
    }
}

/* initial_solution, setup_flow.F90:48-50,128-138: u_char everywhere, then the initial u of
   each inflow node */
static void init_u_inflow(OrSim *s) {
    free(s->u_inflow_local);
    s->u_inflow_local = (double *)xcalloc(s->nb > 0 ? s->nb : 1, sizeof(double));
    for (int jj = 0; jj < s->nb; jj++) {
        int i = s->boundary_list[jj];
        s->u_inflow_local[jj] = s->type[i] == 1 ? s->u[i] : s->cfg.U_char;
    }
}

int or_set_state(OrSim *s, const double *ro, const double *u, const double *v, const double *cxx,
                 const double *cxy, const double *cyy, const double *czz) {
    if (s->npfb == 0) return fail(s, "domain not built");
    alloc_fields(s);
    const int npfb = s->npfb, np = s->np, form = s->cfg.form;
    for (int i = 0; i < np; i++) { s->ro[i] = 1.0; s->cxx[i] = 1.0; s->cyy[i] = 1.0; s->czz[i] = 1.0; }
    for (int i = 0; i < npfb; i++) { /* hardcode_initial_conditions, :180-260 */
        s->u[i] = u[i]; s->v[i] = v[i]; s->w[i] = 0.0; s->ro[i] = ro[i];
        s->p[i] = s->ro[i] * s->csq;
        s->cxx[i] = cxx[i]; s->cxy[i] = cxy[i]; s->cyy[i] = cyy[i]; s->czz[i] = czz ? czz[i] : 1.0;
        if (form == OR_FORM_LC) {
            log_conf_psi_from_c(s->cxx[i], s->cxy[i], s->cyy[i], &s->psixx[i], &s->psixy[i], &s->psiyy[i]);
        } else if (form == OR_FORM_CHL) {
            cholesky_psi_from_c(s, s->cxx[i], s->cxy[i], s->cyy[i], s->czz[i], &s->psixx[i],
                                &s->psixy[i], &s->psiyy[i], &s->psizz[i]);
        }
    }
    for (int jj = 0; jj < s->nb; jj++) { /* :266-280 walls */
        int i = s->boundary_list[jj];
        if (s->type[i] == 0) { s->u[i] = 0.0; s->v[i] = 0.0; s->w[i] = 0.0; }
    }
    for (int i = 0; i < np; i++) { /* setup_flow.F90:68-74 */
        s->rou[i] = s->ro[i] * s->u[i];
        s->rov[i] = s->ro[i] * s->v[i];
        s->row[i] = s->ro[i] * s->w[i];
    }
    reapply_mirror_bcs(s);
    get_c_from_psi(s);
    for (int i = npfb; i < np; i++) { /* :120-125 */
        s->u[i] = s->rou[i] / s->ro[i];
        s->v[i] = s->rov[i] / s->ro[i];
        s->w[i] = s->row[i] / s->ro[i];
    }
    s->time = 0.0; s->itime = 0; s->dt = 1.0e-6;
    s->emax_np1 = pid_tol; s->emax_n = pid_tol; s->emax_nm1 = pid_tol;
    s->driving_force[0] = s->driving_force[1] = s->driving_force[2] = 0.0;
    s->eflow_nm1 = 1.0; s->sum_eflow = 0.0; /* setup_flow.F90:165-169 */
    init_u_inflow(s);
    return 0;
}

int or_set_raw_state(OrSim *s, const double *ro, const double *rou, const double *rov, const double *q) {
    if (!s->ro) alloc_fields(s);
    const int npfb = s->npfb;
    for (int i = 0; i < npfb; i++) {
        s->ro[i] = ro[i]; s->rou[i] = rou[i]; s->rov[i] = rov[i]; s->row[i] = 0.0;
        if (s->cfg.form == OR_FORM_DI) {
            s->cxx[i] = q[i]; s->cxy[i] = q[npfb + i]; s->cyy[i] = q[2 * npfb + i]; s->czz[i] = q[3 * npfb + i];
        } else {
            s->psixx[i] = q[i]; s->psixy[i] = q[npfb + i]; s->psiyy[i] = q[2 * npfb + i]; s->psizz[i] = q[3 * npfb + i];
            if (s->cfg.form == OR_FORM_LC) s->czz[i] = 1.0;
        }
    }
    reapply_mirror_bcs(s);
    get_velocity_from_momentum(s);
    get_c_from_psi(s);
    if (!s->u_inflow_local) init_u_inflow(s);
    return 0;
}

int or_get_state(OrSim *s, double *out) {
    const int n = s->npfb;
    if (!s->ro) return fail(s, "state not set");
    double *src[13] = {s->ro, s->rou, s->rov, s->u, s->v, s->psixx, s->psixy, s->psiyy, s->psizz,
                       s->cxx, s->cxy, s->cyy, s->czz};
    for (int f = 0; f < 13; f++) memcpy(out + (size_t)f * n, src[f], sizeof(double) * n);
    return 0;
}

/* ---------------------------------------------------------------------------------------
 * rhs_di.F90 / rhs.F90 / rhs_lc.F90 -- calc_all_rhs, 2-D, walls only among boundaries
 * ------------------------------------------------------------------------------------- */
typedef struct {
    double *gro_x, *gro_y, *gu_x, *gu_y, *gv_x, *gv_y, *gp_x, *gp_y;
    double *lapu, *lapv;
    double *gcxx_x, *gcxx_y, *gcxy_x, *gcxy_y, *gcyy_x, *gcyy_y; /* DI, LC momentum */
    double *gpxx_x, *gpxx_y, *gpxy_x, *gpxy_y, *gpyy_x, *gpyy_y, *gpzz_x, *gpzz_y; /* chl, lc */
    double *fenepf, *gf_x, *gf_y;
    double *lapcxx, *lapcxy, *lapcyy, *lapczz;
    double *L; /* nb x 5 */
} RhsWork;

static double *zarr(int n) { return (double *)xcalloc(n, sizeof(double)); }

static void rhs_work_alloc(const OrSim *s, RhsWork *w) {
    int n = s->npfb;
    memset(w, 0, sizeof(*w));
    w->gro_x = zarr(n); w->gro_y = zarr(n); w->gu_x = zarr(n); w->gu_y = zarr(n);
    w->gv_x = zarr(n); w->gv_y = zarr(n); w->gp_x = zarr(n); w->gp_y = zarr(n);
    w->lapu = zarr(n); w->lapv = zarr(n);
    w->gcxx_x = zarr(n); w->gcxx_y = zarr(n); w->gcxy_x = zarr(n); w->gcxy_y = zarr(n);
    w->gcyy_x = zarr(n); w->gcyy_y = zarr(n);
    w->gpxx_x = zarr(n); w->gpxx_y = zarr(n); w->gpxy_x = zarr(n); w->gpxy_y = zarr(n);
    w->gpyy_x = zarr(n); w->gpyy_y = zarr(n); w->gpzz_x = zarr(n); w->gpzz_y = zarr(n);
    w->fenepf = zarr(s->np); w->gf_x = zarr(n); w->gf_y = zarr(n);
    w->lapcxx = zarr(n); w->lapcxy = zarr(n); w->lapcyy = zarr(n); w->lapczz = zarr(n);
    w->L = zarr(5 * (s->nb ? s->nb : 1));
}
static void rhs_work_free(RhsWork *w) {
    double **p = (double **)w;
    for (size_t k = 0; k < sizeof(RhsWork) / sizeof(double *); k++) free(p[k]);
}

/* calc_rhs_ro: rhs_di.F90:119-163 (identical in rhs.F90 and rhs_lc.F90) */
static void calc_rhs_ro(OrSim *s, RhsWork *W) {
#pragma omp parallel for schedule(static)
    for (int jj = 0; jj < s->n_internal; jj++) {
        int i = s->internal_list[jj];
        double tmp_scal = (s->u[i] * W->gro_x[i] + s->v[i] * W->gro_y[i]) + s->w[i] * 0.0;
        double divvel = (W->gu_x[i] + W->gv_y[i]) + 0.0;
        s->rhs_ro[i] = -s->ro[i] * divvel - tmp_scal;
    }
    for (int jj = 0; jj < s->nb; jj++) {
        int i = s->boundary_list[jj];
        if (s->type[i] == 0) {
            double xn = s->rnx[i], yn = s->rny[i];
            double dutdt = -yn * W->gu_y[i] + xn * W->gv_y[i];
            s->rhs_ro[i] = -s->ro[i] * dutdt - s->ro[i] * 0.0;
        } else {
            s->rhs_ro[i] = ((-s->v[i] * W->gro_y[i] - s->ro[i] * W->gv_y[i]) - s->w[i] * 0.0) - s->ro[i] * 0.0;
        }
    }
}

/* polymeric stress divergence for node i: DI/LC read gradients of c (rhs_di.F90:232-250),
   chl builds them from gradients of psi (rhs.F90:238-260). */
static void polymeric_divergence(const OrSim *s, const RhsWork *W, int i, double *fu, double *fv) {
    const int form = s->cfg.form;
    if (form == OR_FORM_NEWT) { *fu = 0.0; *fv = 0.0; return; }
    if (form == OR_FORM_CHL) {
        double pxx = s->psixx[i], pxy = s->psixy[i], pyy = s->psiyy[i];
        double gcxx1 = (2.0 * exp(2.0 * pxx)) * W->gpxx_x[i];
        double gcxy1 = exp(pxx) * W->gpxy_x[i] + (pxy * exp(pxx)) * W->gpxx_x[i];
        double gcxy2 = exp(pxx) * W->gpxy_y[i] + (pxy * exp(pxx)) * W->gpxx_y[i];
        double gcyy2 = (2.0 * pxy) * W->gpxy_y[i] + (2.0 * exp(2.0 * pyy)) * W->gpyy_y[i];
        *fu = (gcxx1 + gcxy2) + 0.0;
        *fv = (gcxy1 + gcyy2) + 0.0;
        return;
    }
    if (s->cfg.fenep) {
        double f1 = W->fenepf[i];
        *fu = (((((W->gcxx_x[i] * f1 + s->cxx[i] * W->gf_x[i]) + W->gcxy_y[i] * f1) + s->cxy[i] * W->gf_y[i]) + 0.0 * f1) + 0.0 * 0.0);
        *fv = (((((W->gcxy_x[i] * f1 + s->cxy[i] * W->gf_x[i]) + W->gcyy_y[i] * f1) + s->cyy[i] * W->gf_y[i]) + 0.0 * f1) + 0.0 * 0.0);
        return;
    }
    *fu = (W->gcxx_x[i] + W->gcxy_y[i]) + 0.0;
    *fv = (W->gcxy_x[i] + W->gcyy_y[i]) + 0.0;
}

/* calc_rhs_rovel: rhs_di.F90:165-382, rhs.F90:165-391, rhs_lc.F90:165-381 */
static void calc_rhs_rovel(OrSim *s, RhsWork *W) {
    const double coef_solvent = s->visc_solvent, coef_polymeric = s->visc_polymeric / s->lambda;
    const double *g = s->cfg.grav, *df = s->driving_force;
    const double kol = (1.0 + (s->cfg.Mdiff * s->cfg.beta) * s->cfg.Wi);
    const double kold = (1.0 + s->cfg.Mdiff * s->cfg.Wi);
#pragma omp parallel for schedule(static)
    for (int jj = 0; jj < s->n_internal; jj++) {
        int i = s->internal_list[jj];
        double u = s->u[i], v = s->v[i], ro = s->ro[i];
        double tsu = ro * ((u * W->gu_x[i] + v * W->gu_y[i]) + s->w[i] * 0.0) - u * s->rhs_ro[i];
        double tsv = ro * ((u * W->gv_x[i] + v * W->gv_y[i]) + s->w[i] * 0.0) - v * s->rhs_ro[i];
        double fvu = coef_solvent * W->lapu[i], fvv = coef_solvent * W->lapv[i];
        double pu, pv;
        polymeric_divergence(s, W, i, &pu, &pv);
        if (s->cfg.form != OR_FORM_NEWT) {
            fvu = fvu + coef_polymeric * pu;
            fvv = fvv + coef_polymeric * pv;
        }
        double bfu = ro * (g[0] + df[0]), bfv = ro * (g[1] + df[1]);
        if (s->kolmo) bfu = bfu + (((1.0 / s->cfg.Re) * cos(s->ry[i])) * kol) / kold;
        s->rhs_rou[i] = ((-tsu - W->gp_x[i]) + bfu) + fvu;
        s->rhs_rov[i] = ((-tsv - W->gp_y[i]) + bfv) + fvv;
        s->rhs_row[i] = 0.0;
    }
    for (int jj = 0; jj < s->nb; jj++) {
        int i = s->boundary_list[jj];
        double ro = s->ro[i], c = sqrt(s->csq), dpdn = W->gp_x[i];
        double *L = W->L + 5 * jj;
        if (s->type[i] == 0) {
            double xn = s->rnx[i], yn = s->rny[i];
            double un = s->u[i] * xn + s->v[i] * yn;
            double dundn = xn * W->gu_x[i] + yn * W->gv_x[i];
            double dutdn = -yn * W->gu_x[i] + xn * W->gv_x[i];
            L[0] = (0.5 * (un - c)) * (dpdn - (ro * c) * dundn);
            L[1] = un * (W->gro_x[i] - (W->gp_x[i] / c) / c);
            L[2] = un * dutdn;
            L[3] = un * (0.0 * xn + 0.0 * yn);
            L[4] = (0.5 * (un + c)) * (dpdn + (ro * c) * dundn);
            s->rhs_rou[i] = 0.0; s->rhs_rov[i] = 0.0; s->rhs_row[i] = 0.0;
        } else { /* inflow/outflow in the x-y frame, rhs_di.F90:311-359 (rhs.F90, rhs_lc.F90 alike;
                    no Kolmogorov forcing there) */
            const double u = s->u[i], v = s->v[i], w = s->w[i];
            L[0] = (0.5 * (u - c)) * (dpdn - (ro * c) * W->gu_x[i]);
            L[1] = u * (W->gro_x[i] - (W->gp_x[i] / c) / c);
            L[2] = u * W->gv_x[i];
            L[3] = u * 0.0;
            L[4] = (0.5 * (u + c)) * (dpdn + (ro * c) * W->gu_x[i]);
            double fvu = coef_solvent * W->lapu[i], fvv = coef_solvent * W->lapv[i];
            if (s->cfg.form != OR_FORM_NEWT) {
                double pu, pv;
                polymeric_divergence(s, W, i, &pu, &pv);
                fvu = fvu + coef_polymeric * pu;
                fvv = fvv + coef_polymeric * pv;
            }
            const double bfu = ro * (g[0] + df[0]), bfv = ro * (g[1] + df[1]), bfw = ro * (g[2] + df[2]);
            s->rhs_rou[i] = ((-(v * W->gu_y[i]) - w * 0.0) + fvu) + bfu;
            s->rhs_rov[i] = (((-(v * W->gv_y[i]) - w * 0.0) - W->gp_y[i]) + fvv) + bfv;
            s->rhs_row[i] = (((-(v * 0.0) - w * 0.0) - 0.0) + coef_solvent * 0.0) + bfw;
        }
    }
}

/* calc_rhs_c, DI: rhs_di.F90:384-599 */
static void calc_rhs_c_di(OrSim *s, RhsWork *W) {
    const double lambda = s->lambda, eps = s->cfg.epsPTT, Mdiff = s->cfg.Mdiff, L = s->cfg.L_char;
#pragma omp parallel for schedule(static)
    for (int jj = 0; jj < s->n_internal + s->nb; jj++) {
        int wall = jj >= s->n_internal;
        int i = wall ? s->boundary_list[jj - s->n_internal] : s->internal_list[jj];
        if (wall && s->type[i] != 0) {
            s->rhs_xx[i] = 0.0; s->rhs_xy[i] = 0.0; s->rhs_yy[i] = 0.0; s->rhs_zz[i] = 0.0;
            continue;
        }
        double u = s->u[i], v = s->v[i];
        double cxx = s->cxx[i], cxy = s->cxy[i], cyy = s->cyy[i], czz = s->czz[i];
        double adxx = -((u * W->gcxx_x[i] + v * W->gcxx_y[i]) + s->w[i] * 0.0);
        double adxy = -((u * W->gcxy_x[i] + v * W->gcxy_y[i]) + s->w[i] * 0.0);
        double adyy = -((u * W->gcyy_x[i] + v * W->gcyy_y[i]) + s->w[i] * 0.0);
        double adzz = -((u * 0.0 + v * 0.0) + s->w[i] * 0.0);
        double g11 = W->gu_x[i], g12 = W->gu_y[i], g21 = W->gv_x[i], g22 = W->gv_y[i];
        if (wall) { /* rotated gradients, rhs_di.F90:497-512 */
            double xn = s->rnx[i], yn = s->rny[i];
            double a11 = xn * W->gu_x[i] - yn * W->gu_y[i], a21 = xn * W->gv_x[i] - yn * W->gv_y[i];
            double a12 = yn * W->gu_x[i] + xn * W->gu_y[i], a22 = yn * W->gv_x[i] + xn * W->gv_y[i];
            g11 = a11; g21 = a21; g12 = a12; g22 = a22;
        }
        double ucxx = ((2.0 * g11) * cxx + (2.0 * g12) * cxy) + (2.0 * 0.0) * 0.0;
        double ucxy = (((((g11 * cxy + g12 * cyy) + 0.0 * 0.0) + g21 * cxx) + g22 * cxy) + 0.0 * 0.0);
        double ucyy = ((2.0 * g21) * cxy + (2.0 * g22) * cyy) + (2.0 * 0.0) * 0.0;
        double uczz = ((2.0 * 0.0) * 0.0 + (2.0 * 0.0) * 0.0) + (2.0 * 0.0) * czz;
        double sxx, sxy, syy, szz;
        if (s->cfg.fenep) {
            double fr = -W->fenepf[i];
            sxx = (fr * cxx + 1.0) / lambda;
            sxy = (fr * cxy) / lambda;
            syy = (fr * cyy + 1.0) / lambda;
            szz = (fr * czz + 1.0) / lambda;
        } else {
            double fr = -(((1.0 - eps * 2.0) + eps * ((cxx + cyy) + czz))) / lambda;
            sxx = fr * (cxx - 1.0);
            sxy = fr * cxy;
            syy = fr * (cyy - 1.0);
            szz = fr * (czz - 1.0); /* undefined in the reference 2-D path; defined here */
        }
        if (!wall) {
            s->rhs_xx[i] = ((adxx + ucxx) + sxx) + Mdiff * W->lapcxx[i];
            s->rhs_xy[i] = ((adxy + ucxy) + sxy) + Mdiff * W->lapcxy[i];
            s->rhs_yy[i] = ((adyy + ucyy) + syy) + Mdiff * W->lapcyy[i];
            s->rhs_zz[i] = ((adzz + uczz) + szz) + Mdiff * W->lapczz[i];
        } else {
            double den = ((72.0 * s->sp[i]) * s->sp[i]) * L * L;
            double *f[3] = {s->cxx, s->cxy, s->cyy};
            double *lp[3] = {W->lapcxx, W->lapcxy, W->lapcyy};
            for (int c = 0; c < 3; c++) {
                double *q = f[c];
                lp[c][i] = lp[c][i] + (((((-415.0 * q[i]) + 576.0 * q[i + 1]) - 216.0 * q[i + 2]) + 64.0 * q[i + 3]) - 9.0 * q[i + 4]) / den;
            }
            s->rhs_xx[i] = (ucxx + sxx) + Mdiff * W->lapcxx[i];
            s->rhs_xy[i] = (ucxy + sxy) + Mdiff * W->lapcxy[i];
            s->rhs_yy[i] = (ucyy + syy) + Mdiff * W->lapcyy[i];
            /* rhs_zz on walls is left untouched in 2-D (rhs_di.F90:573-580) */
        }
    }
}

/* calc_rhs_cholesky, rhs.F90:393-722 (2-D) */
static void calc_rhs_cholesky(OrSim *s, RhsWork *W) {
    const double lambda = s->lambda, eps = s->cfg.epsPTT, Mdiff = s->cfg.Mdiff, L = s->cfg.L_char;
    for (int jj = 0; jj < s->n_internal + s->nb; jj++) {
        int wall = jj >= s->n_internal;
        int i = wall ? s->boundary_list[jj - s->n_internal] : s->internal_list[jj];
        double u = s->u[i], v = s->v[i];
        if (wall && s->type[i] == 1) u = 0.0;
        double adxx = (u * W->gpxx_x[i] + v * W->gpxx_y[i]) + s->w[i] * 0.0;
        double adxy = (u * W->gpxy_x[i] + v * W->gpxy_y[i]) + s->w[i] * 0.0;
        double adyy = (u * W->gpyy_x[i] + v * W->gpyy_y[i]) + s->w[i] * 0.0;
        double adzz = (u * W->gpzz_x[i] + v * W->gpzz_y[i]) + s->w[i] * 0.0;
        double lxx = exp(s->psixx[i]), lxy = s->psixy[i], lyy = exp(s->psiyy[i]), lzz = exp(s->psizz[i]);
        double g11 = W->gu_x[i], g12 = W->gu_y[i], g21 = W->gv_x[i], g22 = W->gv_y[i];
        if (wall && s->type[i] == 0) {
            double xn = s->rnx[i], yn = s->rny[i];
            g11 = xn * W->gu_x[i] - yn * W->gu_y[i];
            g12 = yn * W->gu_x[i] + xn * W->gu_y[i];
            g21 = xn * W->gv_x[i] - yn * W->gv_y[i];
            g22 = yn * W->gv_x[i] + xn * W->gv_y[i];
        }
        double ucxx = (g11 + (g12 * lxy) / lxx);
        double ucxy = ((g22 * lxy + ((g12 * lyy) * lyy) / lxx) + g21 * lxx);
        double ucyy = (g22 - (g12 * lxy) / lxx);
        double uczz = 0.0;
        double cxx = s->cxx[i], cxy = s->cxy[i], cyy = s->cyy[i], czz = s->czz[i];
        if (wall) {
            double den = ((72.0 * s->sp[i]) * s->sp[i]) * L * L;
            double *f[4] = {s->cxx, s->cxy, s->cyy, s->czz};
            double *lp[4] = {W->lapcxx, W->lapcxy, W->lapcyy, W->lapczz};
            for (int c = 0; c < 4; c++) {
                double *q = f[c];
                lp[c][i] = lp[c][i] + (((((-415.0 * q[i]) + 576.0 * q[i + 1]) - 216.0 * q[i + 2]) + 64.0 * q[i + 3]) - 9.0 * q[i + 4]) / den;
            }
        }
        double sxx, sxy, syy, szz = 0.0;
        if (s->cfg.fenep) {
            double fr = W->fenepf[i], L2 = s->cfg.fenep_l2;
            double srctmp = ((((((2.0 * g11) * cxx + (2.0 * g12) * cxy) + (2.0 * g21) * cxy) + (2.0 * g22) * cyy)
                              - (((fr * cxx + fr * cyy) + fr * czz) - 3.0) / lambda)
                             + Mdiff * ((W->lapcxx[i] + W->lapcyy[i]) + W->lapczz[i]));
            double den = ((L2 - cxx) - cyy) - czz;
            sxx = (-(fr / lambda) * (fr * cxx - 1.0) + (Mdiff * fr) * W->lapcxx[i]) + ((fr * cxx) * srctmp) / den;
            sxy = (-(fr / lambda) * (fr * cxy) + (Mdiff * fr) * W->lapcxy[i]) + ((fr * cxy) * srctmp) / den;
            syy = (-(fr / lambda) * (fr * cyy - 1.0) + (Mdiff * fr) * W->lapcyy[i]) + ((fr * cyy) * srctmp) / den;
            szz = (-(fr / lambda) * (fr * czz - 1.0) + (Mdiff * fr) * W->lapczz[i]) + ((fr * czz) * srctmp) / den;
        } else {
            double fr = -(((1.0 - eps * 3.0) + eps * ((cxx + cyy) + czz))) / lambda;
            sxx = fr * (cxx - 1.0) + Mdiff * W->lapcxx[i];
            sxy = fr * cxy + Mdiff * W->lapcxy[i];
            syy = fr * (cyy - 1.0) + Mdiff * W->lapcyy[i];
        }
        double csxx = ((0.5 * sxx) / lxx) / lxx;
        double csxy = sxy / lxx - ((0.5 * sxx) * lxy) / (lxx * lxx);
        double csyy = (((0.5 * syy) / lyy) / lyy - (sxy * lxy) / ((lxx * lyy) * lyy))
                      + (((0.5 * sxx) * lxy) * lxy) / ((lyy * lyy) * (lxx * lxx));
        double cszz = ((0.5 * szz) / lzz) / lzz;
        s->rhs_xx[i] = (-adxx + ucxx) + csxx;
        s->rhs_xy[i] = (-adxy + ucxy) + csxy;
        s->rhs_yy[i] = (-adyy + ucyy) + csyy;
        if (s->cfg.fenep) s->rhs_zz[i] = (-adzz + uczz) + cszz;
    }
}

/* calc_rhs_logconf, rhs_lc.F90:383-750 (2-D) */
static void calc_rhs_logconf(OrSim *s, RhsWork *W) {
    const double lambda = s->lambda, eps = s->cfg.epsPTT;
    const int first = (s->itime == 1 && s->iRKstep == 1); /* :503 */
#pragma omp parallel for schedule(static)
    for (int jj = 0; jj < s->n_internal + s->nb; jj++) {
        int wall = jj >= s->n_internal;
        int i = wall ? s->boundary_list[jj - s->n_internal] : s->internal_list[jj];
        double u = s->u[i], v = s->v[i];
        double adxx = -((u * W->gpxx_x[i] + v * W->gpxx_y[i]) + s->w[i] * 0.0);
        double adxy = -((u * W->gpxy_x[i] + v * W->gpxy_y[i]) + s->w[i] * 0.0);
        double adyy = -((u * W->gpyy_x[i] + v * W->gpyy_y[i]) + s->w[i] * 0.0);
        double Lv[2], R[4], RT[4], G[4], M[4], B[4], Om[4], UC[4], P[4], Ci[4], Rx[4], T[4];
        eigens2(s->psixx[i], s->psixy[i], s->psiyy[i], Lv, R);
        Lv[0] = exp(Lv[0]);
        Lv[1] = exp(Lv[1]);
        tr2(R, RT);
        double tr_c = Lv[0] + Lv[1];
        if (wall && s->type[i] == 0) {
            double xn = s->rnx[i], yn = s->rny[i];
            G[0] = xn * W->gu_x[i] - yn * W->gu_y[i];
            G[2] = yn * W->gu_x[i] + xn * W->gu_y[i];
            G[1] = xn * W->gv_x[i] - yn * W->gv_y[i];
            G[3] = yn * W->gv_x[i] + xn * W->gv_y[i];
        } else {
            G[0] = W->gu_x[i]; G[2] = W->gu_y[i]; G[1] = W->gv_x[i]; G[3] = W->gv_y[i];
        }
        mm2(G, R, T);
        mm2(RT, T, M);
        double om = (Lv[1] * M[2] + Lv[0] * M[1]);
        if (fabs(Lv[1] - Lv[0]) <= verysmall) om = 0.0;
        else om = om / (Lv[1] - Lv[0]);
        M[2] = 0.0; M[1] = 0.0;
        mm2(M, RT, T);
        mm2(R, T, B);
        M[0] = 0.0; M[1] = 0.0; M[2] = 0.0; M[3] = 0.0;
        M[2] = om; M[1] = -om;
        mm2(M, RT, T);
        mm2(R, T, Om);
        if (first) {
            Om[0] = Om[1] = Om[2] = Om[3] = 0.0;
            double GT[4];
            tr2(G, GT);
            for (int c = 0; c < 4; c++) B[c] = 0.5 * (G[c] + GT[c]);
        }
        P[0] = s->psixx[i]; P[2] = s->psixy[i]; P[1] = s->psixy[i]; P[3] = s->psiyy[i];
        double OP[4], PO[4];
        mm2(Om, P, OP);
        mm2(P, Om, PO);
        for (int c = 0; c < 4; c++) UC[c] = (OP[c] - PO[c]) + 2.0 * B[c];
        if (s->cfg.fenep) {
            double fR = W->fenepf[i];
            double cxx = s->cxx[i], cxy = s->cxy[i], cyy = s->cyy[i];
            double det = cxx * cyy - cxy * cxy;
            Ci[0] = cyy / det; Ci[3] = cxx / det; Ci[2] = -cxy / det; Ci[1] = -cxy / det;
            B[0] = cxx; B[3] = cyy; B[2] = cxy; B[1] = cxy;
            for (int c = 0; c < 4; c++) B[c] = B[c] * fR;
            B[0] = B[0] - 1.0; B[3] = B[3] - 1.0;
            mm2(Ci, B, T);
            for (int c = 0; c < 4; c++) Rx[c] = (-1.0 / lambda) * T[c];
        } else {
            double fR = ((1.0 - 2.0 * eps) + eps * tr_c);
            Ci[0] = fR / Lv[0] - fR; Ci[1] = 0.0; Ci[2] = 0.0; Ci[3] = fR / Lv[1] - fR;
            mm2(Ci, RT, T);
            mm2(R, T, T);
            for (int c = 0; c < 4; c++) Rx[c] = T[c] / lambda;
        }
        if (wall && s->type[i] == 0) {
            s->rhs_xx[i] = UC[0] + Rx[0];
            s->rhs_xy[i] = UC[2] + Rx[2];
            s->rhs_yy[i] = UC[3] + Rx[3];
        } else {
            s->rhs_xx[i] = (adxx + UC[0]) + Rx[0];
            s->rhs_xy[i] = (adxy + UC[2]) + Rx[2];
            s->rhs_yy[i] = (adyy + UC[3]) + Rx[3];
        }
    }
}

/* specify_characteristics_isothermal_wall (characteristic_boundaries.F90:27-52) and the
   boundary update of calc_rhs_nscbc (rhs_di.F90:601-665). */
static void calc_rhs_nscbc(OrSim *s, RhsWork *W) {
    const double nscbc = 2.87e-1;                                  /* common_parameter.F90:71 */
    const double Lx = (s->xmax - s->xmin) * s->cfg.L_char;         /* setup_domain.F90:98 */
    const double p_in = s->rho_char * s->csq, p_out = s->rho_char * s->csq; /* load_data.F90:147-148 */
    for (int jj = 0; jj < s->nb; jj++) {
        int i = s->boundary_list[jj];
        double *L = W->L + 5 * jj;
        const double c = sqrt(s->csq), u = s->u[i], v = s->v[i], w = s->w[i], p = s->p[i], ro = s->ro[i];
        const double uin = s->u_inflow_local[jj];
        if (s->type[i] == 0) {
            L[4] = L[0]; /* specify_characteristics_isothermal_wall, :27-52 */
        } else if (s->type[i] == 1) {
            if (s->cfg.inflow_type == 1) { /* specify_characteristics_hard_inflow, :82-110 */
                L[1] = 0.0; L[2] = 0.0; L[3] = 0.0; L[4] = L[0];
            } else if (s->cfg.inflow_type == 2) { /* specify_characteristics_inflow_outflow, :112-150 */
                if (u > 0.0) {
                    L[1] = 0.0;
                    L[2] = ((v * nscbc) * c) / Lx;
                    L[3] = ((w * nscbc) * c) / Lx;
                    L[4] = ((((((u - uin) * nscbc) * (1.0 - u / c)) * c) * c) * 1.0) / Lx;
                } else {
                    L[1] = 0.0;
                    L[4] = (((((p - p_in) * nscbc) * c) * 1.0) / 2.0) / Lx;
                }
            } else { /* specify_characteristics_soft_inflow, :54-80 */
                L[1] = 0.0;
                L[2] = (((((v * nscbc) * c) / Lx) - v * W->gv_y[i]) - w * 0.0) - W->gp_y[i] / ro;
                L[3] = ((w * nscbc) * c) / Lx + s->rhs_row[i];
                L[4] = (((((((u - uin) * nscbc) * (1.0 - u / c)) * c) * c) * 1.0) / Lx -
                        0.5 * (((v * W->gp_y[i]) + (p * W->gv_y[i])) + (((ro * c) * v) * W->gu_y[i]))) -
                       0.5 * (((w * 0.0) + (p * 0.0)) + (((ro * c) * w) * 0.0));
            }
        } else if (s->type[i] == 2) { /* specify_characteristics_outflow, :152-189 */
            if (u < c) L[0] = (((((p - p_out) * nscbc) * c) * 1.0) / 2.0) / Lx;
            L[1] = 0.0;
            if (u <= 0.0) { L[1] = 0.0; L[2] = 0.0; L[3] = 0.0; }
        }
        double tmp_scal = ((((c * c) * L[1] + L[4]) + L[0]) / c) / c;
        s->rhs_ro[i] = s->rhs_ro[i] - tmp_scal;
        s->rhs_rou[i] = (s->rhs_rou[i] - s->u[i] * tmp_scal) - (L[4] - L[0]) / c;
        s->rhs_rov[i] = (s->rhs_rov[i] - s->v[i] * tmp_scal) - s->ro[i] * L[2];
        s->rhs_row[i] = (s->rhs_row[i] - s->w[i] * tmp_scal) - s->ro[i] * L[3];
    }
}

static int calc_all_rhs(OrSim *s) {
    const int form = s->cfg.form, npfb = s->npfb;
    if (!s->u_inflow_local) init_u_inflow(s);
    RhsWork W;
    rhs_work_alloc(s, &W);
    memset(s->rhs_ro, 0, sizeof(double) * npfb); memset(s->rhs_rou, 0, sizeof(double) * npfb);
    memset(s->rhs_rov, 0, sizeof(double) * npfb); memset(s->rhs_row, 0, sizeof(double) * npfb);
    memset(s->rhs_xx, 0, sizeof(double) * npfb); memset(s->rhs_xy, 0, sizeof(double) * npfb);
    memset(s->rhs_yy, 0, sizeof(double) * npfb); memset(s->rhs_zz, 0, sizeof(double) * npfb);
    calc_gradient(s, s->ro, W.gro_x, W.gro_y, 0);
    calc_gradient(s, s->u, W.gu_x, W.gu_y, 0);
    calc_gradient(s, s->v, W.gv_x, W.gv_y, 0);
    for (int i = 0; i < s->np; i++) s->p[i] = s->csq * s->ro[i];
    for (int i = 0; i < npfb; i++) { W.gp_x[i] = s->csq * W.gro_x[i]; W.gp_y[i] = s->csq * W.gro_y[i]; }
    calc_rhs_ro(s, &W);
    /* calc_rhs_rovel derivative calls */
    calc_laplacian(s, s->u, W.lapu);
    calc_laplacian(s, s->v, W.lapv);
    if (form == OR_FORM_DI || form == OR_FORM_LC) {
        int full = (form == OR_FORM_DI && s->cfg.di_full_gradients);
        calc_gradient(s, s->cxx, W.gcxx_x, W.gcxx_y, full ? 0 : 1);
        calc_gradient(s, s->cxy, W.gcxy_x, W.gcxy_y, 0);
        calc_gradient(s, s->cyy, W.gcyy_x, W.gcyy_y, full ? 0 : 2);
        if (s->cfg.fenep) {
            for (int i = 0; i < s->np; i++)
                W.fenepf[i] = (s->cfg.fenep_l2 - 3.0) / (s->cfg.fenep_l2 - ((s->cxx[i] + s->cyy[i]) + s->czz[i]));
            calc_gradient(s, W.fenepf, W.gf_x, W.gf_y, 0);
        }
    } else if (form == OR_FORM_CHL) {
        calc_gradient(s, s->psixx, W.gpxx_x, W.gpxx_y, 0);
        calc_gradient(s, s->psixy, W.gpxy_x, W.gpxy_y, 0);
        calc_gradient(s, s->psiyy, W.gpyy_x, W.gpyy_y, 0);
        if (s->cfg.fenep) {
            calc_gradient(s, s->psizz, W.gpzz_x, W.gpzz_y, 0);
            for (int i = 0; i < s->np; i++)
                W.fenepf[i] = (s->cfg.fenep_l2 - 3.0) / (s->cfg.fenep_l2 - ((s->cxx[i] + s->cyy[i]) + s->czz[i]));
        }
    }
    calc_rhs_rovel(s, &W);
    if (form == OR_FORM_DI) {
        if (s->cfg.Mdiff != 0.0) {
            calc_laplacian_transverse(s, s->cxx, W.lapcxx);
            calc_laplacian_transverse(s, s->cxy, W.lapcxy);
            calc_laplacian_transverse(s, s->cyy, W.lapcyy);
            if (s->cfg.fenep) calc_laplacian_transverse(s, s->czz, W.lapczz);
        }
        calc_rhs_c_di(s, &W);
    } else if (form == OR_FORM_CHL) {
        if (s->cfg.Mdiff != 0.0) {
            calc_laplacian_transverse(s, s->cxx, W.lapcxx);
            calc_laplacian_transverse(s, s->cxy, W.lapcxy);
            calc_laplacian_transverse(s, s->cyy, W.lapcyy);
            calc_laplacian_transverse(s, s->czz, W.lapczz);
        }
        calc_rhs_cholesky(s, &W);
    } else if (form == OR_FORM_LC) {
        calc_gradient(s, s->psixx, W.gpxx_x, W.gpxx_y, 0);
        calc_gradient(s, s->psixy, W.gpxy_x, W.gpxy_y, 0);
        calc_gradient(s, s->psiyy, W.gpyy_x, W.gpyy_y, 0);
        calc_rhs_logconf(s, &W);
    }
    if (s->nb != 0) calc_rhs_nscbc(s, &W);
    rhs_work_free(&W);
    return 0;
}

int or_calc_all_rhs(OrSim *s, double *rhs) {
    if (!s->have_weights || !s->ro) return fail(s, "weights or state missing");
    if (calc_all_rhs(s)) return -1;
    const int n = s->npfb;
    double *src[7] = {s->rhs_ro, s->rhs_rou, s->rhs_rov, s->rhs_xx, s->rhs_xy, s->rhs_yy, s->rhs_zz};
    for (int f = 0; f < 7; f++) memcpy(rhs + (size_t)f * n, src[f], sizeof(double) * n);
    return 0;
}

/* filter_variables: rhs_di.F90:667-720, rhs.F90:792-900, rhs_lc.F90:818-893 */
static void filter_variables(OrSim *s) {
    const int form = s->cfg.form, npfb = s->npfb;
    double *work = zarr(npfb);
    calc_filtered_var(s, s->ro, work);
    calc_filtered_var(s, s->rou, work);
    calc_filtered_var(s, s->rov, work);
    if (form == OR_FORM_DI) {
        calc_filtered_var(s, s->cxx, work);
        calc_filtered_var(s, s->cxy, work);
        calc_filtered_var(s, s->cyy, work);
        calc_filtered_var(s, s->czz, work);
    } else if (form == OR_FORM_CHL) {
        const double L2 = s->cfg.fenep_l2;
        if (s->cfg.fenep) {
            for (int i = 0; i < s->np; i++) {
                double fr = ((exp(2.0 * s->psixx[i]) + s->psixy[i] * s->psixy[i]) + exp(2.0 * s->psiyy[i])) + exp(2.0 * s->psizz[i]);
                fr = (L2 * fr) / ((L2 - 3.0) + fr);
                fr = (L2 - 3.0) / (L2 - fr);
                s->psixx[i] = s->psixx[i] - log(sqrt(fr));
                s->psixy[i] = s->psixy[i] / sqrt(fr);
                s->psiyy[i] = s->psiyy[i] - log(sqrt(fr));
                s->psizz[i] = s->psizz[i] - log(sqrt(fr));
            }
        }
        calc_filtered_var(s, s->psixx, work);
        calc_filtered_var(s, s->psixy, work);
        calc_filtered_var(s, s->psiyy, work);
        if (s->cfg.fenep) {
            calc_filtered_var(s, s->psizz, work);
            for (int i = 0; i < npfb; i++) {
                double fr = (L2 - 3.0) / (L2 - (((exp(2.0 * s->psixx[i]) + s->psixy[i] * s->psixy[i]) + exp(2.0 * s->psiyy[i])) + exp(2.0 * s->psizz[i])));
                s->psixx[i] = s->psixx[i] + log(sqrt(fr));
                s->psixy[i] = s->psixy[i] * sqrt(fr);
                s->psiyy[i] = s->psiyy[i] + log(sqrt(fr));
                s->psizz[i] = s->psizz[i] + log(sqrt(fr));
            }
        }
    } else if (form == OR_FORM_LC) {
        calc_filtered_var(s, s->psixx, work);
        calc_filtered_var(s, s->psixy, work);
        calc_filtered_var(s, s->psiyy, work);
        if (s->cfg.fenep) calc_filtered_var(s, s->psizz, work);
    }
    free(work);
    if (s->cfg.mcorr) {
        double tm = 0.0, tv = 0.0;
        for (int i = 0; i < npfb; i++) {
            tm = tm + (s->ro[i] - s->rho_char) * s->vol[i];
            tv = tv + s->vol[i];
        }
        double dro = tm / tv;
        for (int i = 0; i < npfb; i++) s->ro[i] = s->ro[i] - dro;
    }
}

/* step_rk3_4S_2R_EE, step.F90:218-512 */
static int step_rk3_4s_2r_ee(OrSim *s) {
    const int npfb = s->npfb, form = s->cfg.form;
    const double a[3] = {RK_A21, RK_A32, RK_A43};
    const double b[4] = {RK_B1, RK_B2, RK_B3, RK_B4};
    const double bh[4] = {RK_BH1, RK_BH2, RK_BH3, RK_BH4};
    const double cc[4] = {0.0, RK_A21, RK_A32 + RK_B1, 1.0};
    double RKa[3], RKb[4], RKbmbh[4], RKc[4];
    const double dt = s->dt;
    s->emax_nm1 = s->emax_n;
    s->emax_n = s->emax_np1;
    for (int k = 0; k < 3; k++) RKa[k] = dt * a[k];
    for (int k = 0; k < 4; k++) { RKb[k] = dt * b[k]; RKbmbh[k] = dt * (b[k] - bh[k]); RKc[k] = dt * cc[k]; }
    double *Q[6], *reg[6], *eacc[6], *rhs[6];
    double *xx, *xy, *yy, *zz;
    if (form == OR_FORM_DI) { xx = s->cxx; xy = s->cxy; yy = s->cyy; zz = s->czz; }
    else { xx = s->psixx; xy = s->psixy; yy = s->psiyy; zz = s->psizz; }
    Q[0] = s->ro; Q[1] = s->rou; Q[2] = s->rov; Q[3] = xx; Q[4] = xy; Q[5] = yy;
    double *Qzz = zz, *Qrow = s->row;
    rhs[0] = s->rhs_ro; rhs[1] = s->rhs_rou; rhs[2] = s->rhs_rov; rhs[3] = s->rhs_xx; rhs[4] = s->rhs_xy; rhs[5] = s->rhs_yy;
    for (int f = 0; f < 6; f++) { reg[f] = zarr(npfb); eacc[f] = zarr(npfb); }
    double *reg_row = zarr(npfb), *reg_zz = zarr(npfb), *e_row = zarr(npfb), *e_zz = zarr(npfb);
    for (int i = 0; i < npfb; i++) {
        for (int f = 0; f < 6; f++) reg[f][i] = Q[f][i];
        reg_row[i] = Qrow[i];
        reg_zz[i] = Qzz[i];
    }
    double time0 = s->time;
    s->iRKstep = 0;
    int rc = 0;
    for (int k = 0; k < 3; k++) {
        s->iRKstep++;
        s->time = time0 + RKc[s->iRKstep - 1];
        if (calc_all_rhs(s)) { rc = -1; goto done; }
#pragma omp parallel for schedule(static)
        for (int i = 0; i < npfb; i++) {
            for (int f = 0; f < 6; f++) Q[f][i] = reg[f][i] + RKa[k] * rhs[f][i];
            Qrow[i] = reg_row[i] + RKa[k] * s->rhs_row[i];
            Qzz[i] = reg_zz[i] + RKa[k] * s->rhs_zz[i];
            for (int f = 0; f < 6; f++) reg[f][i] = reg[f][i] + RKb[k] * rhs[f][i];
            reg_row[i] = reg_row[i] + RKb[k] * s->rhs_row[i];
            reg_zz[i] = reg_zz[i] + RKb[k] * s->rhs_zz[i];
            for (int f = 0; f < 6; f++) eacc[f][i] = eacc[f][i] + RKbmbh[k] * rhs[f][i];
            e_row[i] = e_row[i] + RKbmbh[k] * s->rhs_row[i];
            e_zz[i] = e_zz[i] + RKbmbh[k] * s->rhs_zz[i];
        }
        if (s->nb != 0) apply_time_dependent_bounds(s);
        reapply_mirror_bcs(s);
        get_velocity_from_momentum(s);
        if (form != OR_FORM_DI) get_c_from_psi(s);
    }
    s->iRKstep++;
    s->time = time0 + RKc[s->iRKstep - 1];
    if (calc_all_rhs(s)) { rc = -1; goto done; }
    double en[6] = {0, 0, 0, 0, 0, 0}, en_row = 0.0, en_zz = 0.0;
    const double norms[6] = {s->ero_norm, s->erou_norm, s->erou_norm, s->exx_norm, s->exx_norm, s->exx_norm};
    for (int i = 0; i < npfb; i++) {
        for (int f = 0; f < 6; f++) Q[f][i] = reg[f][i] + RKb[3] * rhs[f][i];
        Qrow[i] = reg_row[i] + RKb[3] * s->rhs_row[i];
        Qzz[i] = reg_zz[i] + RKb[3] * s->rhs_zz[i];
        for (int f = 0; f < 6; f++) eacc[f][i] = eacc[f][i] + RKbmbh[3] * rhs[f][i];
        e_row[i] = e_row[i] + RKbmbh[3] * s->rhs_row[i];
        e_zz[i] = e_zz[i] + RKbmbh[3] * s->rhs_zz[i];
        /* Cholesky FENE-P (step.F90:442-452): the conformation errors are scaled by
           1/sqrt(f).  The reference rescales its running maxima by each node's factor in
           turn, which makes the result depend on the node order; here each node's own
           errors are scaled by its own factor before the maximum (decision, order-free). */
        double sc = 1.0;
        if (form == OR_FORM_CHL && s->cfg.fenep) {
            double fr = (s->cfg.fenep_l2 - 3.0) / (((s->cfg.fenep_l2 - s->cxx[i]) - s->cyy[i]) - s->czz[i]);
            sc = 1.0 / sqrt(fr);
        }
        for (int f = 0; f < 6; f++) {
            double t = fabs(eacc[f][i]) * norms[f];
            if (f >= 3) t = t * sc;
            en[f] = (t > en[f]) ? t : en[f];
        }
        {
            double t = fabs(e_row[i]) * s->erou_norm;
            en_row = (t > en_row) ? t : en_row;
            t = (fabs(e_zz[i]) * s->exx_norm) * sc;
            en_zz = (t > en_zz) ? t : en_zz;
        }
    }
#define MAXD(a, b) ((a) > (b) ? (a) : (b))
    /* emax_conf = max(xx, max(xy, max(yy, max(xz, max(yz, zz))))) with xz = yz = 0 */
    double emax_conf = MAXD(en[3], MAXD(en[4], MAXD(en[5], MAXD(0.0, MAXD(0.0, en_zz)))));
    s->emax_np1 = MAXD(emax_conf, MAXD(en[0], MAXD(en[1], MAXD(en[2], MAXD(en_row, doublesmall)))));
#undef MAXD
    if (s->nb != 0) apply_time_dependent_bounds(s);
    reapply_mirror_bcs(s);
    filter_variables(s);
    if (s->nb != 0) apply_time_dependent_bounds(s);
    reapply_mirror_bcs(s);
    get_velocity_from_momentum(s);
    if (form != OR_FORM_DI) get_c_from_psi(s);
done:
    for (int f = 0; f < 6; f++) { free(reg[f]); free(eacc[f]); }
    free(reg_row); free(reg_zz); free(e_row); free(e_zz);
    return rc;
}

/* set_tstep, step.F90:569-622 */
int or_set_tstep(OrSim *s, double *dt_cfl, double *dt_parabolic) {
    double dcfl = 1.0e10, dvisc = 1.0e10;
    for (int i = 0; i < s->npfb; i++) {
        double c = sqrt(s->csq);
        double umax = sqrt((s->u[i] * s->u[i] + s->v[i] * s->v[i]) + s->w[i] * s->w[i]);
        double uplusc = umax + c;
        double t = (s->type[i] == 2) ? (0.8 * s->sp[i]) / uplusc : s->sp[i] / uplusc;
        dcfl = (t < dcfl) ? t : dcfl;
        t = ((s->sp[i] * s->sp[i]) * s->ro[i]) / s->visc_total;
        dvisc = (t < dvisc) ? t : dvisc;
    }
    s->dt_cfl = (1.0 * dcfl) * s->cfg.L_char;
    s->dt_parabolic = (((2.0 / 3.0) * dvisc) * s->cfg.L_char) * s->cfg.L_char;
    if (dt_cfl) *dt_cfl = s->dt_cfl;
    if (dt_parabolic) *dt_parabolic = s->dt_parabolic;
    return 0;
}

/* set_tstep_PID, step.F90:624-682 */
static void set_tstep_pid(OrSim *s) {
    double facA = PID_A * log(pid_tol / s->emax_np1);
    double facB = PID_B * log(s->emax_n / pid_tol);
    double facC = PID_C * log(pid_tol / s->emax_nm1);
    double dtfactor = pid_k * exp((facA + facB) + facC);
    dtfactor = (0.5 > dtfactor) ? 0.5 : dtfactor;
    dtfactor = (1.02 < dtfactor) ? 1.02 : dtfactor;
    s->dt = s->dt * dtfactor;
    double dt_max = (s->dt_cfl < s->dt_parabolic) ? s->dt_cfl : s->dt_parabolic;
    if (s->dt > dt_max) s->dt = dt_max;
}

/* velocity_control with -Dvpid (statistics.F90:214-303), called after every step
   (sunset.F90:104, statistics.F90:80-82): a PID controller drives the volume-mean x velocity
   to L_domain_y L_domain_x / tot_vol through driving_force(1).  The reference sums over the
   nodes in an OpenMP reduction (order unspecified); here in node order. */
static void velocity_control(OrSim *s) {
    double tot_vol = 0.0, tot_u = 0.0;
    for (int i = 0; i < s->npfb; i++) {
        const double dvi = s->vol[i];
        tot_vol = tot_vol + dvi;
        tot_u = tot_u + s->u[i] * dvi;
    }
    tot_u = tot_u / tot_vol;
    const double Lx = (s->xmax - s->xmin) * s->cfg.L_char, Ly = (s->ymax - s->ymin) * s->cfg.L_char;
    const double eflow_n = 1.0 - (tot_u * tot_vol) / (Ly * Lx);
    s->sum_eflow = s->sum_eflow + eflow_n * s->dt;
    const double deflowdt = (eflow_n - s->eflow_nm1) / s->dt;
    const double facA = ((((0.5 * 0.5) * 0.5) * 1.0) * 2.0) * 2.0;
    const double facB = facA / 0.4, facC = facA * 0.02;
    double df = ((facA * eflow_n) + facB * s->sum_eflow) + facC * deflowdt;
    df = (500.0 < df) ? 500.0 : df;
    df = (-500.0 > df) ? -500.0 : df;
    s->driving_force[0] = df;
    s->eflow_nm1 = eflow_n;
}

int or_get_flow_control(OrSim *s, double *out) {
    out[0] = s->eflow_nm1; out[1] = s->sum_eflow;
    out[2] = s->driving_force[0]; out[3] = s->driving_force[1]; out[4] = s->driving_force[2];
    return 0;
}
int or_set_flow_control(OrSim *s, const double *in) {
    s->eflow_nm1 = in[0]; s->sum_eflow = in[1];
    s->driving_force[0] = in[2]; s->driving_force[1] = in[3]; s->driving_force[2] = in[4];
    return 0;
}

int or_step(OrSim *s, double dt, int nsteps, int pid) {
    if (!s->have_weights || !s->ro) return fail(s, "weights or state missing");
    for (int n = 0; n < nsteps; n++) {
        if (pid) {
            or_set_tstep(s, NULL, NULL);
            set_tstep_pid(s);
        } else {
            s->dt = dt;
        }
        if (step_rk3_4s_2r_ee(s)) return -1;
        s->itime++;
        /* statistics_control after the step: the controller with -Dvpid, else the driving
           force zeroed (statistics.F90:80-90,288; a restart may have loaded one) */
        if (s->cfg.vpid) velocity_control(s);
        else s->driving_force[0] = s->driving_force[1] = s->driving_force[2] = 0.0;
    }
    return 0;
}

int or_get_time(OrSim *s, double *time, double *dt, int *itime, double *emax) {
    if (time) *time = s->time;
    if (dt) *dt = s->dt;
    if (itime) *itime = s->itime;
    if (emax) { emax[0] = s->emax_nm1; emax[1] = s->emax_n; emax[2] = s->emax_np1; }
    return 0;
}
int or_set_time(OrSim *s, double time, double dt, int itime, const double *emax) {
    s->time = time; s->dt = dt; s->itime = itime;
    if (emax) { s->emax_nm1 = emax[0]; s->emax_n = emax[1]; s->emax_np1 = emax[2]; }
    return 0;
}

double or_kinetic_energy(OrSim *s) {
    double ke = 0.0;
    for (int i = 0; i < s->npfb; i++)
        ke = ke + ((0.5 * s->ro[i]) * (s->u[i] * s->u[i] + s->v[i] * s->v[i])) * s->vol[i];
    return ke;
}
double or_mass(OrSim *s) {
    double m = 0.0;
    for (int i = 0; i < s->npfb; i++) m = m + s->ro[i] * s->vol[i];
    return m;
}

/* =========================================================================================
 * 3-D (-Ddim3): build_3rd_dimension (setup_domain.F90:435-547), calc_fd_weights
 * (fd.F90:27-256), the z parts of derivatives.F90 (:48-63, :96-108, :145-157, :340-352,
 * :387-405, :441-453) and the dim3 branches of rhs_di.F90, rhs.F90 (Cholesky) and rhs_lc.F90
 * (log-conformation), conf_transforms.F90:27-397 and step.F90, for the direct, Cholesky,
 * log-conformation (sPTT) and Newtonian forms on node sets without boundary nodes or with walls
 * (node_type 0) among them.
 *
 * The 3-D node set is nz copies of the 2-D one, layer-major: node k = iz*nl + i at
 * z = iz*dz.  The reference searches neighbours per layer (neighbours.F90:180-183,223-233,
 * cells of the node's own layer) over identical positions, and the LABFM weights, sums,
 * volumes and filter coefficients depend only on those positions, so every layer's lists and
 * weights are the layer's own (the 2-D OrSim below), used with an offset of iz*nl.  Mirror
 * images take their parent's value in the same layer; u and v flip with the mirror as in 2-D,
 * w and c_xz, c_yz are copied unchanged (mirror_boundaries.F90:302-303,324-341).
 *
 * Walls (build_3rd_dimension copies node_type and rnorm to every layer, :487-532): a wall
 * node's x-y operators are its boundary weights (normal and tangential derivatives), its z
 * operators the same stencils as everywhere; its right-hand sides are the wall branches of
 * calc_rhs_ro / calc_rhs_rovel / calc_rhs_nscbc and of the conformation equations with their
 * dim3 terms, and apply_time_dependent_bounds holds rho u, rho v, rho w at zero there.
 * ========================================================================================= */
struct Or3 {
    OrSim *s;                /* the layer */
    int nl, nz, ncfd;
    size_t n3;
    double dz, fdg[13], fdl[13], fdh[13];
    double *ro, *rou, *rov, *row, *u, *v, *w, *c[6]; /* n3 each; c: xx xy yy xz yz zz */
    double *psi[6];                                  /* Cholesky, log-conf: xx xy yy xz yz zz */
    double time, dt, dt_cfl, dt_par;
    int itime, iRKstep;
    double emax_nm1, emax_n, emax_np1;
    int *bidx;               /* nl: the layer node's index in boundary_list, or -1 */
    double *uin;             /* n3: u_inflow_local of each node-layer (inflow node-layers' in use) */
    double *alpha;           /* n3: the last step's error of each node-layer (alpha_out) */
    char err[256];
};

/* calc_fd_weights, fd.F90:52-172 (ij_count_fd = forder + 1), then the L_char scaling of
   :246-247 */
static int fd_tables(int ncfd, double dz, double L, double *g, double *g2, double *h) {
    const double one = 1.0, two = 2.0;
    if (ncfd == 5) {
        g[0] = (one / 12.0) / dz; g[1] = -((8.0 / 12.0) / dz); g[2] = 0.0; g[3] = (8.0 / 12.0) / dz; g[4] = -((one / 12.0) / dz);
        g2[0] = -(((one / 12.0) / dz) / dz); g2[1] = ((16.0 / 12.0) / dz) / dz; g2[2] = -(((30.0 / 12.0) / dz) / dz);
        g2[3] = ((16.0 / 12.0) / dz) / dz; g2[4] = -(((one / 12.0) / dz) / dz);
        h[0] = -(one / 16.0); h[1] = 4.0 / 16.0; h[2] = -(6.0 / 16.0); h[3] = 4.0 / 16.0; h[4] = -(one / 16.0);
    } else if (ncfd == 7) {
        g[0] = -((one / 60.0) / dz); g[1] = (9.0 / 60.0) / dz; g[2] = -((45.0 / 60.0) / dz); g[3] = 0.0;
        g[4] = (45.0 / 60.0) / dz; g[5] = -((9.0 / 60.0) / dz); g[6] = (one / 60.0) / dz;
        g2[0] = ((two / 180.0) / dz) / dz; g2[1] = -(((27.0 / 180.0) / dz) / dz); g2[2] = ((270.0 / 180.0) / dz) / dz;
        g2[3] = -(((490.0 / 180.0) / dz) / dz); g2[4] = ((270.0 / 180.0) / dz) / dz; g2[5] = -(((27.0 / 180.0) / dz) / dz);
        g2[6] = ((two / 180.0) / dz) / dz;
        h[0] = one / 64.0; h[1] = -(6.0 / 64.0); h[2] = 15.0 / 64.0; h[3] = -(20.0 / 64.0); h[4] = 15.0 / 64.0;
        h[5] = -(6.0 / 64.0); h[6] = one / 64.0;
    } else if (ncfd == 9) {
        g[0] = (3.0 / 840.0) / dz; g[1] = -((32.0 / 840.0) / dz); g[2] = (168.0 / 840.0) / dz; g[3] = -((672.0 / 840.0) / dz);
        g[4] = 0.0; g[5] = (672.0 / 840.0) / dz; g[6] = -((168.0 / 840.0) / dz); g[7] = (32.0 / 840.0) / dz;
        g[8] = -((3.0 / 840.0) / dz);
        g2[0] = -(((9.0 / 5040.0) / dz) / dz); g2[1] = ((128.0 / 5040.0) / dz) / dz; g2[2] = -(((1008.0 / 5040.0) / dz) / dz);
        g2[3] = ((8064.0 / 5040.0) / dz) / dz; g2[4] = -(((14350.0 / 5040.0) / dz) / dz); g2[5] = ((8064.0 / 5040.0) / dz) / dz;
        g2[6] = -(((1008.0 / 5040.0) / dz) / dz); g2[7] = ((128.0 / 5040.0) / dz) / dz; g2[8] = -(((9.0 / 5040.0) / dz) / dz);
        h[0] = -(one / 256.0); h[1] = 8.0 / 256.0; h[2] = -(28.0 / 256.0); h[3] = 56.0 / 256.0; h[4] = -(70.0 / 256.0);
        h[5] = 56.0 / 256.0; h[6] = -(28.0 / 256.0); h[7] = 8.0 / 256.0; h[8] = -(one / 256.0);
    } else if (ncfd == 11) {
        g[0] = -((one / 1260.0) / dz); g[1] = (5.0 / 504.0) / dz; g[2] = -((5.0 / 84.0) / dz); g[3] = (5.0 / 21.0) / dz;
        g[4] = -((5.0 / 6.0) / dz); g[5] = 0.0; g[6] = (5.0 / 6.0) / dz; g[7] = -((5.0 / 21.0) / dz); g[8] = (5.0 / 84.0) / dz;
        g[9] = -((5.0 / 504.0) / dz); g[10] = (one / 1260.0) / dz;
        g2[0] = ((one / 3150.0) / dz) / dz; g2[1] = -(((5.0 / 1008.0) / dz) / dz); g2[2] = ((5.0 / 126.0) / dz) / dz;
        g2[3] = -(((5.0 / 21.0) / dz) / dz); g2[4] = ((5.0 / 3.0) / dz) / dz; g2[5] = -(((1086.0 / 371.0) / dz) / dz);
        g2[6] = ((5.0 / 3.0) / dz) / dz; g2[7] = -(((5.0 / 21.0) / dz) / dz); g2[8] = ((5.0 / 126.0) / dz) / dz;
        g2[9] = -(((5.0 / 1008.0) / dz) / dz); g2[10] = ((one / 3150.0) / dz) / dz;
        h[0] = one / 1024.0; h[1] = -(10.0 / 1024.0); h[2] = 45.0 / 1024.0; h[3] = -(120.0 / 1024.0); h[4] = 210.0 / 1024.0;
        h[5] = -(252.0 / 1024.0); h[6] = 210.0 / 1024.0; h[7] = -(120.0 / 1024.0); h[8] = 45.0 / 1024.0;
        h[9] = -(10.0 / 1024.0); h[10] = one / 1024.0;
    } else {
        return -1;
    }
    for (int k = 0; k < ncfd; k++) { g[k] = g[k] / L; g2[k] = (g2[k] / L) / L; }
    return 0;
}

Or3 *or3_create(OrSim *s, double Lz) {
    if (!s || !s->have_weights || (s->cfg.fenep && s->cfg.form != OR_FORM_DI && s->cfg.form != OR_FORM_CHL) || !(Lz > 0.0))
        return NULL;
    Or3 *o = (Or3 *)xcalloc(1, sizeof(Or3));
    o->s = s;
    o->nl = s->npfb;
    o->bidx = (int *)xcalloc(o->nl, sizeof(int));
    for (int i = 0; i < o->nl; i++) o->bidx[i] = -1;
    for (int jj = 0; jj < s->nb; jj++) o->bidx[s->boundary_list[jj]] = jj;
    o->ncfd = s->cfg.forder + 1;
    /* build_3rd_dimension, :444-483 (mean_alpha = 1, one process in z) */
    double dzl = 0.0, sv = 0.0;
    for (int i = 0; i < s->npfb; i++) {
        sv = sv + s->sp[i] * s->sp[i];
        dzl = dzl + (s->sp[i] * s->sp[i]) * s->sp[i];
    }
    double dz = dzl / sv;
    const double L = s->cfg.L_char, Lzd = (Lz * L) / L;
    int nz = (int)ceil((Lzd / dz) / 1.0);
    dz = (Lzd / (double)nz) / 1.0;
    if (nz < o->ncfd / 2 + 2) {
        nz = o->ncfd / 2 + 2;
        dz = Lzd / (double)(o->ncfd / 2 + 2);
    }
    o->nz = nz;
    o->dz = dz;
    if (fd_tables(o->ncfd, dz, L, o->fdg, o->fdl, o->fdh)) { free(o->bidx); free(o); return NULL; }
    o->n3 = (size_t)o->nl * nz;
    double **a[] = {&o->ro, &o->rou, &o->rov, &o->row, &o->u, &o->v, &o->w, &o->c[0], &o->c[1], &o->c[2], &o->c[3], &o->c[4], &o->c[5],
                    &o->psi[0], &o->psi[1], &o->psi[2], &o->psi[3], &o->psi[4], &o->psi[5]};
    for (size_t k = 0; k < sizeof(a) / sizeof(a[0]); k++) *a[k] = (double *)xcalloc(o->n3, sizeof(double));
    o->uin = (double *)xcalloc(o->n3, sizeof(double));
    o->alpha = (double *)xcalloc(o->n3, sizeof(double));
    return o;
}

void or3_destroy(Or3 *o) {
    if (!o) return;
    double *a[] = {o->ro, o->rou, o->rov, o->row, o->u, o->v, o->w, o->c[0], o->c[1], o->c[2], o->c[3], o->c[4], o->c[5],
                   o->psi[0], o->psi[1], o->psi[2], o->psi[3], o->psi[4], o->psi[5]};
    for (size_t k = 0; k < sizeof(a) / sizeof(a[0]); k++) free(a[k]);
    free(o->bidx);
    free(o->uin);
    free(o->alpha);
    free(o);
}

int or3_sizes(Or3 *o, int *nl, int *nz, double *dz) {
    if (nl) *nl = o->nl;
    if (nz) *nz = o->nz;
    if (dz) *dz = o->dz;
    return 0;
}

/* sign classes of a field at a mirror image: 0 none, 1 like u, 2 like v, 3 like c_xy */
static double val3(const Or3 *o, const double *f, int j, size_t off, int cls) {
    const OrSim *s = o->s;
    if (j < o->nl) return f[off + j];
    const int vr = s->vrel[j];
    const double x = f[off + s->irel[j]];
    const int flip = (cls == 1 && (vr == 2 || vr == 4)) || (cls == 2 && (vr == 3 || vr == 4)) ||
                     (cls == 3 && (vr == 2 || vr == 3));
    return flip ? -x : x;
}
/* layer of the m-th point of the z stencil (fd.F90:62-66, periodic in z) */
static size_t zoff(const Or3 *o, int iz, int m) {
    int l = (iz + m - o->ncfd / 2) % o->nz;
    if (l < 0) l += o->nz;
    return (size_t)l * o->nl;
}

/* calc_gradient / calc_gradient_only in 3-D: comp bits 1 = x, 2 = y, 4 = z */
static void grad3(const Or3 *o, const double *f, int cls, int comp, double *gx, double *gy, double *gz) {
    const OrSim *s = o->s;
    const int nplink = s->nplink;
#pragma omp parallel for schedule(static)
    for (size_t k = 0; k < o->n3; k++) {
        const int iz = (int)(k / o->nl), i = (int)(k % o->nl);
        const size_t off = (size_t)iz * o->nl;
        if (comp & 3) {
            double g1 = 0.0, g2 = 0.0;
            const int *lk = s->ij_link + (size_t)i * nplink;
            const double *wg = s->w_grad + 2 * (size_t)i * nplink;
            for (int q = 0; q < s->ij_count_small[i]; q++) {
                const double pj = val3(o, f, lk[q], off, cls);
                if (comp & 1) g1 = g1 + pj * wg[2 * q];
                if (comp & 2) g2 = g2 + pj * wg[2 * q + 1];
            }
            if (comp & 1) gx[k] = g1 - f[k] * s->w_grad_sum[2 * i];
            if (comp & 2) gy[k] = g2 - f[k] * s->w_grad_sum[2 * i + 1];
        }
        if (comp & 4) {
            double t = 0.0;
            for (int m = 0; m < o->ncfd; m++) t = t + f[zoff(o, iz, m) + i] * o->fdg[m];
            gz[k] = t;
        }
    }
}
/* calc_laplacian in 3-D (:73-108) */
static void lap3(const Or3 *o, const double *f, int cls, double *lap) {
    const OrSim *s = o->s;
    const int nplink = s->nplink;
#pragma omp parallel for schedule(static)
    for (size_t k = 0; k < o->n3; k++) {
        const int iz = (int)(k / o->nl), i = (int)(k % o->nl);
        const size_t off = (size_t)iz * o->nl;
        double l = 0.0;
        const int *lk = s->ij_link + (size_t)i * nplink;
        const double *wl = s->w_lap + (size_t)i * nplink;
        for (int q = 0; q < s->ij_count_small[i]; q++) l = l + val3(o, f, lk[q], off, cls) * wl[q];
        double r = l - f[k] * s->w_lap_sum[i];
        double t = 0.0;
        for (int m = 0; m < o->ncfd; m++) t = t + f[zoff(o, iz, m) + i] * o->fdl[m];
        lap[k] = r + t;
    }
}
/* The conformation Laplacian in 3-D: calc_laplacian_transverse_only_on_bound (:306-358), whose
   x-y part on a wall node takes the tangential second-derivative weights (ij_wb_grad2(2,:,:)),
   then the z stencil; on walls calc_rhs_c adds the one-sided normal second derivative over the
   node's four FD rows, the next nodes of its layer (rhs_di.F90:553-568, rhs.F90:631-643) */
static void lap3_conf(const Or3 *o, const double *f, int cls, double *lap) {
    const OrSim *s = o->s;
    const int nplink = s->nplink;
    const double L = s->cfg.L_char;
#pragma omp parallel for schedule(static)
    for (size_t k = 0; k < o->n3; k++) {
        const int iz = (int)(k / o->nl), i = (int)(k % o->nl);
        const size_t off = (size_t)iz * o->nl;
        const int jb = o->bidx[i];
        const int *lk = s->ij_link + (size_t)i * nplink;
        double l = 0.0, r;
        if (jb < 0) {
            const double *wl = s->w_lap + (size_t)i * nplink;
            for (int q = 0; q < s->ij_count_small[i]; q++) l = l + val3(o, f, lk[q], off, cls) * wl[q];
            r = l - f[k] * s->w_lap_sum[i];
        } else {
            for (int q = 0; q < s->ij_count_small[i]; q++)
                l = l + val3(o, f, lk[q], off, cls) * s->wb_grad2[((size_t)jb * nplink + q) * 3 + 1];
            r = l - f[k] * s->wb_grad2_sum[3 * jb + 1];
        }
        double t = 0.0;
        for (int m = 0; m < o->ncfd; m++) t = t + f[zoff(o, iz, m) + i] * o->fdl[m];
        lap[k] = r + t;
        if (jb >= 0) {
            const double den = ((72.0 * s->sp[i]) * s->sp[i]) * L * L;
            lap[k] = lap[k] + (((((-415.0 * f[k]) + 576.0 * f[k + 1]) - 216.0 * f[k + 2]) + 64.0 * f[k + 3]) - 9.0 * f[k + 4]) / den;
        }
    }
}
/* calc_filtered_var in 3-D (:360-405): the x-y filter, then the z filter of the result */
static void filter3(const Or3 *o, double *f, int cls, double *work) {
    const OrSim *s = o->s;
    const int nplink = s->nplink;
#pragma omp parallel for schedule(static)
    for (size_t k = 0; k < o->n3; k++) {
        const int iz = (int)(k / o->nl), i = (int)(k % o->nl);
        const size_t off = (size_t)iz * o->nl;
        double t = 0.0;
        const int *lk = s->ij_link + (size_t)i * nplink;
        const double *wh = s->w_hyp + (size_t)i * nplink;
        for (int q = 0; q < s->ij_count[i]; q++) t = t + val3(o, f, lk[q], off, cls) * wh[q];
        work[k] = f[k] + (t - f[k] * s->w_hyp_sum[i]);
    }
    memcpy(f, work, sizeof(double) * o->n3);
#pragma omp parallel for schedule(static)
    for (size_t k = 0; k < o->n3; k++) {
        const int iz = (int)(k / o->nl), i = (int)(k % o->nl);
        double t = 0.0;
        for (int m = 0; m < o->ncfd; m++) t = t + f[zoff(o, iz, m) + i] * o->fdh[m];
        work[k] = f[k] + t;
    }
    memcpy(f, work, sizeof(double) * o->n3);
}

/* cholesky_c_from_psi and cholesky_psi_from_c in 3-D, sPTT (conf_transforms.F90:60-71,
   108-121) */
static void chl3_c_from_psi(const double *p, double *c) {
    const double e = exp(p[0]);
    c[0] = e * e;
    c[1] = exp(p[0]) * p[1];
    c[2] = p[1] * p[1] + exp(2.0 * p[2]);
    c[3] = exp(p[0]) * p[3];
    c[4] = p[1] * p[3] + exp(p[2]) * p[4];
    c[5] = (exp(2.0 * p[5]) + p[3] * p[3]) + p[4] * p[4];
}
static void chl3_psi_from_c(const double *c, double *p) {
    const double xx = sqrt(c[0]);
    const double xy = c[1] / (xx);
    const double yy = (sqrt(c[2] - xy * xy));
    const double xz = c[3] / xx;
    const double yz = (c[4] - xy * xz) / yy;
    const double zz = sqrt((c[5] - xz * xz) - yz * yz);
    p[0] = log(xx); p[1] = xy; p[2] = log(yy); p[3] = xz; p[4] = yz; p[5] = log(zz);
}
/* the same with FENE-P (conf_transforms.F90:39-58, 89-106): psi are the Cholesky factors of
   J = f c, f = (L^2 - 3)/(L^2 - tr c), and c = J L^2/(L^2 - 3 + tr J) */
static void chl3_c_from_psi_fenep(double L2, const double *p, double *c) {
    const double Jxx = exp(2.0 * p[0]), Jxy = exp(p[0]) * p[1], Jyy = p[1] * p[1] + exp(2.0 * p[2]);
    const double Jzz = (exp(2.0 * p[5]) + p[3] * p[3]) + p[4] * p[4];
    const double fq = L2 / ((((L2 - 3.0) + Jxx) + Jyy) + Jzz);
    c[0] = Jxx * fq; c[1] = Jxy * fq; c[2] = Jyy * fq; c[5] = Jzz * fq;
    const double Jxz = exp(p[0]) * p[3], Jyz = p[1] * p[3] + exp(p[2]) * p[4];
    c[3] = Jxz * fq; c[4] = Jyz * fq;
}
static void chl3_psi_from_c_fenep(double L2, const double *c, double *p) {
    const double fr = (L2 - 3.0) / (L2 - ((c[0] + c[2]) + c[5]));
    const double Jxx = c[0] * fr, Jxy = c[1] * fr, Jyy = c[2] * fr, Jzz = c[5] * fr;
    const double xx = sqrt(Jxx);
    const double xy = Jxy / xx;
    const double yy = sqrt(Jyy - xy * xy);
    const double Jxz = c[3] * fr, Jyz = c[4] * fr;
    const double xz = Jxz / xx;
    const double yz = (Jyz - xy * xz) / yy;
    const double zz = sqrt((Jzz - xz * xz) - yz * yz);
    p[0] = log(xx); p[1] = xy; p[2] = log(yy); p[3] = xz; p[4] = yz; p[5] = log(zz);
}
/* filter_variables under FENE-P in 3-D (rhs.F90:816-834): the factors of J to those of c,
   and after the filter (:853-868) back */
static void chl3_fenep_to_c_factor(double L2, double *p) {
    double fr = ((((exp(2.0 * p[0]) + p[1] * p[1]) + exp(2.0 * p[2])) + p[3] * p[3]) + p[4] * p[4]) + exp(2.0 * p[5]);
    fr = (L2 * fr) / ((L2 - 3.0) + fr);
    fr = (L2 - 3.0) / (L2 - fr);
    p[0] = p[0] - log(sqrt(fr));
    p[1] = p[1] / sqrt(fr);
    p[2] = p[2] - log(sqrt(fr));
    p[5] = p[5] - log(sqrt(fr));
    p[3] = p[3] / sqrt(fr);
    p[4] = p[4] / sqrt(fr);
}
static void chl3_fenep_to_j_factor(double L2, double *p) {
    const double fr =
        (L2 - 3.0) / (L2 - (((((exp(2.0 * p[0]) + p[1] * p[1]) + exp(2.0 * p[2])) + p[3] * p[3]) + p[4] * p[4]) + exp(2.0 * p[5])));
    p[0] = p[0] + log(sqrt(fr));
    p[1] = p[1] * sqrt(fr);
    p[2] = p[2] + log(sqrt(fr));
    p[5] = p[5] + log(sqrt(fr));
    p[3] = p[3] * sqrt(fr);
    p[4] = p[4] * sqrt(fr);
}
/* eigens (3x3 symmetric), conf_transforms.F90:218-397: closed-form eigenvalues (trigonometric
   solution of the characteristic cubic), eigenvectors by cross products and a 2x2 rotation.
   R column-major, R[i + 3j] = R(i+1, j+1); its columns are the eigenvectors of L[0..2]. */
static void eigens3(double axx, double axy, double ayy, double axz, double ayz, double azz, double *L, double *R) {
    const double onethird = 1.0 / 3.0, twothirds = 2.0 / 3.0, eps = DBL_EPSILON;
    double a[9];
    a[0] = axx; a[3] = axy; a[6] = axz;
    a[1] = axy; a[4] = ayy; a[7] = ayz;
    a[2] = axz; a[5] = ayz; a[8] = azz;
    const double p1 = (axy * axy + axz * axz) + ayz * ayz;
    if (p1 <= doublesmall) {
        L[0] = axx; L[1] = ayy; L[2] = azz;
        for (int k = 0; k < 9; k++) R[k] = 0.0;
        R[0] = 1.0; R[4] = 1.0; R[8] = 1.0;
        return;
    }
    const double q = onethird * ((axx + ayy) + azz);
    const double p2 = (((axx - q) * (axx - q) + (ayy - q) * (ayy - q)) + (azz - q) * (azz - q)) + 2.0 * p1;
    const double p = sqrt(p2 / 6.0);
    const double bxx = (1.0 / p) * (axx - q), bxy = (1.0 / p) * axy, byy = (1.0 / p) * (ayy - q);
    const double bxz = (1.0 / p) * axz, byz = (1.0 / p) * ayz, bzz = (1.0 / p) * (azz - q);
    double detbo2 = (bxx * (byy * bzz - byz * byz) - bxy * (bxy * bzz - byz * bxz)) + bxz * (bxy * byz - byy * bxz);
    detbo2 = 0.5 * detbo2;
    double phi;
    if (detbo2 <= -1.0) phi = onethird * pi;
    else if (detbo2 >= 1.0) phi = 0.0;
    else phi = onethird * acos(detbo2);
    L[2] = q + (2.0 * p) * cos(phi);
    L[0] = q + (2.0 * p) * cos(phi + twothirds * pi);
    L[1] = (3.0 * q - L[0]) - L[2];
#define A_(i, j) a[(i - 1) + 3 * (j - 1)]
#define R_(i, j) R[(i - 1) + 3 * (j - 1)]
    A_(1, 1) = A_(1, 1) - L[0]; A_(2, 2) = A_(2, 2) - L[0]; A_(3, 3) = A_(3, 3) - L[0];
    R_(1, 1) = A_(1, 2) * A_(2, 3) - A_(1, 3) * A_(2, 2);
    R_(2, 1) = A_(1, 3) * A_(1, 2) - A_(1, 1) * A_(2, 3);
    R_(3, 1) = A_(1, 1) * A_(2, 2) - A_(1, 2) * A_(1, 2);
    R_(1, 2) = A_(1, 2) * A_(3, 3) - A_(1, 3) * A_(2, 3);
    R_(2, 2) = A_(1, 3) * A_(1, 3) - A_(1, 1) * A_(3, 3);
    R_(3, 2) = A_(1, 1) * A_(2, 3) - A_(1, 2) * A_(1, 3);
    R_(1, 3) = A_(2, 2) * A_(3, 3) - A_(2, 3) * A_(2, 3);
    R_(2, 3) = A_(2, 3) * A_(1, 3) - A_(1, 2) * A_(3, 3);
    R_(3, 3) = A_(1, 2) * A_(2, 3) - A_(2, 2) * A_(1, 3);
    double n1 = (R_(1, 1) * R_(1, 1) + R_(2, 1) * R_(2, 1)) + R_(3, 1) * R_(3, 1);
    double n2 = (R_(1, 2) * R_(1, 2) + R_(2, 2) * R_(2, 2)) + R_(3, 2) * R_(3, 2);
    double n3 = (R_(1, 3) * R_(1, 3) + R_(2, 3) * R_(2, 3)) + R_(3, 3) * R_(3, 3);
    double norm = n1;
    int ic = 1;
    if (n2 > norm) { ic = 2; norm = n1; } /* (the reference keeps n1 here) */
    if (n3 > norm) ic = 3;
    if (ic == 1) {
        norm = sqrt(1.0 / n1);
        R_(1, 1) = R_(1, 1) * norm; R_(2, 1) = R_(2, 1) * norm; R_(3, 1) = R_(3, 1) * norm;
    } else if (ic == 2) {
        norm = sqrt(1.0 / n2);
        R_(1, 1) = R_(1, 2) * norm; R_(2, 1) = R_(2, 2) * norm; R_(3, 1) = R_(3, 2) * norm;
    } else {
        norm = sqrt(1.0 / n3);
        R_(1, 1) = R_(1, 3) * norm; R_(2, 1) = R_(2, 3) * norm; R_(3, 1) = R_(3, 3) * norm;
    }
    if (fabs(R_(1, 1)) > fabs(R_(2, 1))) {
        norm = sqrt(1.0 / (R_(1, 1) * R_(1, 1) + R_(3, 1) * R_(3, 1)));
        R_(1, 2) = -R_(3, 1) * norm; R_(2, 2) = 0.0; R_(3, 2) = R_(1, 1) * norm;
    } else {
        norm = sqrt(1.0 / (R_(2, 1) * R_(2, 1) + R_(3, 1) * R_(3, 1)));
        R_(1, 2) = 0.0; R_(2, 2) = R_(3, 1) * norm; R_(3, 2) = -R_(2, 1) * norm;
    }
    R_(1, 3) = R_(2, 1) * R_(3, 2) - R_(3, 1) * R_(2, 2);
    R_(2, 3) = R_(3, 1) * R_(1, 2) - R_(1, 1) * R_(3, 2);
    R_(3, 3) = R_(1, 1) * R_(2, 2) - R_(2, 1) * R_(1, 2);
    A_(1, 1) = A_(1, 1) + L[0]; A_(2, 2) = A_(2, 2) + L[0]; A_(3, 3) = A_(3, 3) + L[0];
    n1 = (A_(1, 1) * R_(1, 2) + A_(1, 2) * R_(2, 2)) + A_(1, 3) * R_(3, 2);
    n2 = (A_(1, 2) * R_(1, 2) + A_(2, 2) * R_(2, 2)) + A_(2, 3) * R_(3, 2);
    n3 = (A_(1, 3) * R_(1, 2) + A_(2, 3) * R_(2, 2)) + A_(3, 3) * R_(3, 2);
    A_(3, 3) = (A_(1, 3) * R_(1, 3) + A_(2, 3) * R_(2, 3)) + A_(3, 3) * R_(3, 3);
    A_(1, 3) = (A_(1, 1) * R_(1, 3) + A_(1, 2) * R_(2, 3)) + A_(1, 3) * R_(3, 3);
    A_(2, 3) = (A_(1, 2) * R_(1, 3) + A_(2, 2) * R_(2, 3)) + A_(2, 3) * R_(3, 3);
    n1 = ((R_(1, 2) * n1 + R_(2, 2) * n2) + R_(3, 2) * n3) - L[1];
    n2 = (R_(1, 2) * A_(1, 3) + R_(2, 2) * A_(2, 3)) + R_(3, 2) * A_(3, 3);
    n3 = ((R_(1, 3) * A_(1, 3) + R_(2, 3) * A_(2, 3)) + R_(3, 3) * A_(3, 3)) - L[1];
    if (fabs(n1) >= fabs(n3)) {
        norm = fabs(n1) > fabs(n2) ? fabs(n1) : fabs(n2);
        if (norm > eps) {
            if (fabs(n1) >= fabs(n2)) { n2 = n2 / n1; n1 = sqrt(1.0 / (1.0 + n2 * n2)); n2 = n2 * n1; }
            else { n1 = n1 / n2; n2 = sqrt(1.0 / (1.0 + n1 * n1)); n1 = n1 * n2; }
            R_(1, 2) = n2 * R_(1, 2) - n1 * R_(1, 3);
            R_(2, 2) = n2 * R_(2, 2) - n1 * R_(2, 3);
            R_(3, 2) = n2 * R_(3, 2) - n1 * R_(3, 3);
        }
    } else {
        norm = fabs(n3) > fabs(n2) ? fabs(n3) : fabs(n2);
        if (norm > eps) {
            if (fabs(n3) >= fabs(n2)) { n2 = n2 / n3; n3 = sqrt(1.0 / (1.0 + n2 * n2)); n2 = n2 * n3; }
            else { n3 = n3 / n2; n2 = sqrt(1.0 / (1.0 + n3 * n3)); n3 = n3 * n2; }
            R_(1, 2) = n3 * R_(1, 2) - n2 * R_(1, 3);
            R_(2, 2) = n3 * R_(2, 2) - n2 * R_(2, 3);
            R_(3, 2) = n3 * R_(3, 2) - n2 * R_(3, 3);
        }
    }
    R_(1, 3) = R_(2, 1) * R_(3, 2) - R_(3, 1) * R_(2, 2);
    R_(2, 3) = R_(3, 1) * R_(1, 2) - R_(1, 1) * R_(3, 2);
    R_(3, 3) = R_(1, 1) * R_(2, 2) - R_(2, 1) * R_(1, 2);
#undef A_
#undef R_
}
/* C = A B, 3x3 column-major, matmul's sum in k order */
static void mm3(const double *A, const double *B, double *C) {
    double t[9];
    for (int j = 0; j < 3; j++)
        for (int i = 0; i < 3; i++) t[i + 3 * j] = (A[i] * B[3 * j] + A[i + 3] * B[1 + 3 * j]) + A[i + 6] * B[2 + 3 * j];
    memcpy(C, t, sizeof(t));
}
static void tr3(const double *A, double *T) {
    for (int j = 0; j < 3; j++)
        for (int i = 0; i < 3; i++) T[i + 3 * j] = A[j + 3 * i];
}
/* log_conf_c_from_psi / log_conf_psi_from_c in 3-D (conf_transforms.F90:127-215):
   R f(Lambda) R^T with f = exp or log; out: xx (1,1), xy (2,1), yy (2,2), xz (1,3), yz (2,3), zz */
static void lc3_transform(const double *in, double *out, int to_c) {
    double L[3], R[9], RT[9], Lm[9] = {0}, M[9];
    eigens3(in[0], in[1], in[2], in[3], in[4], in[5], L, R);
    tr3(R, RT);
    for (int k = 0; k < 3; k++) Lm[4 * k] = to_c ? exp(L[k]) : log(L[k]);
    mm3(Lm, RT, M);
    mm3(R, M, M);
    out[0] = M[0]; out[1] = M[1]; out[2] = M[4]; out[3] = M[6]; out[4] = M[7]; out[5] = M[8];
}

static void or3_c_from_psi(Or3 *o) {
    const int form = o->s->cfg.form;
    if (form != OR_FORM_CHL && form != OR_FORM_LC) return;
#pragma omp parallel for schedule(static)
    for (size_t k = 0; k < o->n3; k++) {
        double p[6], c[6];
        for (int q = 0; q < 6; q++) p[q] = o->psi[q][k];
        if (form == OR_FORM_CHL && o->s->cfg.fenep) chl3_c_from_psi_fenep(o->s->cfg.fenep_l2, p, c);
        else if (form == OR_FORM_CHL) chl3_c_from_psi(p, c);
        else lc3_transform(p, c, 1);
        for (int q = 0; q < 6; q++) o->c[q][k] = c[q];
    }
}

/* apply_time_dependent_bounds on every layer (characteristic_boundaries.F90:191-257) at the
   time o->time: update_u_inflow (:262-300, the ramp while time <= ramp_time), then walls at
   rest, and a hard inflow's momentum prescribed (rho u = u_inflow_local rho, rho v = rho w = 0) */
static void bounds3(Or3 *o) {
    const OrSim *s = o->s;
    const int ramp = s->cfg.inflow_velocity_control == 1 && o->time <= s->cfg.ramp_time;
    const double um = s->cfg.u_inflow_start + ((s->cfg.u_inflow_end - s->cfg.u_inflow_start) * o->time) / s->cfg.ramp_time;
    for (int iz = 0; iz < o->nz; iz++)
        for (int jj = 0; jj < s->nb; jj++) {
            const int i = s->boundary_list[jj];
            const size_t k = (size_t)iz * o->nl + i;
            if (s->type[i] == 1 && ramp) o->uin[k] = um;
            if (s->type[i] == 0) { o->rou[k] = 0.0; o->rov[k] = 0.0; o->row[k] = 0.0; }
            else if (s->type[i] == 1 && s->cfg.inflow_type == 1) {
                o->rou[k] = o->uin[k] * o->ro[k]; o->rov[k] = 0.0; o->row[k] = 0.0;
            }
        }
}

/* hardcode_initial_conditions in 3-D: rho, u, v, w and c given (u, v, w zero on walls,
   setup_flow.F90:266-280); rho u = rho * u ... */
int or3_set_state(Or3 *o, const double *ro, const double *u, const double *v, const double *w,
                  const double *const *c6) {
    for (size_t k = 0; k < o->n3; k++) {
        o->ro[k] = ro[k]; o->u[k] = u[k]; o->v[k] = v[k]; o->w[k] = w[k];
        if (o->bidx[k % o->nl] >= 0 && o->s->type[k % o->nl] == 0) { o->u[k] = 0.0; o->v[k] = 0.0; o->w[k] = 0.0; }
        o->rou[k] = o->ro[k] * o->u[k]; o->rov[k] = o->ro[k] * o->v[k]; o->row[k] = o->ro[k] * o->w[k];
        for (int q = 0; q < 6; q++) o->c[q][k] = c6 ? c6[q][k] : ((q == 0 || q == 2 || q == 5) ? 1.0 : 0.0);
        if (o->s->cfg.form == OR_FORM_CHL || o->s->cfg.form == OR_FORM_LC) {
            double c[6], p[6];
            for (int q = 0; q < 6; q++) c[q] = o->c[q][k];
            if (o->s->cfg.form == OR_FORM_CHL && o->s->cfg.fenep) chl3_psi_from_c_fenep(o->s->cfg.fenep_l2, c, p);
            else if (o->s->cfg.form == OR_FORM_CHL) chl3_psi_from_c(c, p);
            else lc3_transform(c, p, 0);
            for (int q = 0; q < 6; q++) o->psi[q][k] = p[q];
        }
    }
    or3_c_from_psi(o);
    /* u_inflow_local (setup_flow.F90:48-50,128-138): u_char, the initial u on inflow nodes */
    for (size_t k = 0; k < o->n3; k++) {
        const int i = (int)(k % o->nl);
        o->uin[k] = (o->bidx[i] >= 0 && o->s->type[i] == 1) ? o->u[k] : o->s->cfg.U_char;
    }
    o->time = 0.0; o->itime = 0; o->dt = 1.0e-6;
    o->emax_np1 = o->emax_n = o->emax_nm1 = pid_tol;
    /* the flow-rate controller's state (setup_flow.F90:165-169) */
    o->s->driving_force[0] = o->s->driving_force[1] = o->s->driving_force[2] = 0.0;
    o->s->eflow_nm1 = 1.0; o->s->sum_eflow = 0.0;
    return 0;
}
int or3_get_state(Or3 *o, double *out /* 19 x n3: ro rou rov row u v w cxx cxy cyy cxz cyz czz, psi x 6 */) {
    const double *a[19] = {o->ro, o->rou, o->rov, o->row, o->u, o->v, o->w, o->c[0], o->c[1], o->c[2], o->c[3], o->c[4], o->c[5],
                           o->psi[0], o->psi[1], o->psi[2], o->psi[3], o->psi[4], o->psi[5]};
    for (int f = 0; f < 19; f++) memcpy(out + (size_t)f * o->n3, a[f], sizeof(double) * o->n3);
    return 0;
}

/* calc_all_rhs in 3-D (rhs_di.F90:45-599, interior branches with the dim3 terms):
   r[10] = ro, rou, rov, row, xx, xy, yy, xz, yz, zz */
static void rhs3(Or3 *o, double *const *r) {
    const OrSim *s = o->s;
    const size_t n = o->n3;
    const int di = s->cfg.form == OR_FORM_DI, chl = s->cfg.form == OR_FORM_CHL, islc = s->cfg.form == OR_FORM_LC;
    const int full = di && s->cfg.di_full_gradients;
    enum { ROX, ROY, ROZ, UX, UY, UZ, VX, VY, VZ, WX, WY, WZ, LU, LV, LW, NG0 };
    double *G[NG0];
    for (int q = 0; q < NG0; q++) G[q] = zarr((int)n);
    grad3(o, o->ro, 0, 7, G[ROX], G[ROY], G[ROZ]);
    grad3(o, o->u, 1, 7, G[UX], G[UY], G[UZ]);
    grad3(o, o->v, 2, 7, G[VX], G[VY], G[VZ]);
    grad3(o, o->w, 0, 7, G[WX], G[WY], G[WZ]);
    lap3(o, o->u, 1, G[LU]);
    lap3(o, o->v, 2, G[LV]);
    lap3(o, o->w, 0, G[LW]);
    /* conformation gradients: c_xx x only, c_xy, c_xz, c_yz full, c_yy y only, c_zz z only
       (rhs_di.F90:186-194), the others computed only with full gradients (else zero) */
    double *gc[6][3], *lc[6], *gp[6][3];
    static const int ccls[6] = {0, 3, 0, 0, 0, 0};
    static const int cmask[6] = {1, 7, 2, 7, 7, 4};
    for (int q = 0; q < 6; q++) {
        for (int d = 0; d < 3; d++) { gc[q][d] = zarr((int)n); gp[q][d] = NULL; }
        lc[q] = zarr((int)n);
        if (islc) { /* rhs_lc.F90:184-193 (c, momentum) and :397-409 (psi, advection) */
            for (int d = 0; d < 3; d++) gp[q][d] = zarr((int)n);
            grad3(o, o->c[q], ccls[q], cmask[q], gc[q][0], gc[q][1], gc[q][2]);
            grad3(o, o->psi[q], ccls[q], 7, gp[q][0], gp[q][1], gp[q][2]);
            continue;
        }
        if (!di && !chl) continue;
        /* Cholesky: full gradients of every psi component (rhs.F90:186-201) */
        if (chl) grad3(o, o->psi[q], ccls[q], 7, gc[q][0], gc[q][1], gc[q][2]);
        else grad3(o, o->c[q], ccls[q], full ? 7 : cmask[q], gc[q][0], gc[q][1], gc[q][2]);
        if (s->cfg.Mdiff != 0.0) lap3_conf(o, o->c[q], ccls[q], lc[q]);
    }
    /* FENE-P (direct form): the function f = (L^2 - 3)/(L^2 - tr c) at every node and its
       gradient, rhs_di.F90:198-205 */
    const int fen = di && s->cfg.fenep;
    double *ff = NULL, *gf[3] = {NULL, NULL, NULL};
    if (fen) {
        const double L2 = s->cfg.fenep_l2;
        ff = zarr((int)n);
        for (size_t k = 0; k < n; k++) ff[k] = (L2 - 3.0) / (L2 - ((o->c[0][k] + o->c[2][k]) + o->c[5][k]));
        for (int d = 0; d < 3; d++) gf[d] = zarr((int)n);
        grad3(o, ff, 0, 7, gf[0], gf[1], gf[2]);
    }
    const double csq = s->csq, cs = s->visc_solvent, cp = s->visc_polymeric / s->lambda;
    const double *g = s->cfg.grav, *df = s->driving_force;
    const double kol = (1.0 + (s->cfg.Mdiff * s->cfg.beta) * s->cfg.Wi), kold = (1.0 + s->cfg.Mdiff * s->cfg.Wi);
    const double lambda = s->lambda, eps = s->cfg.epsPTT, Md = s->cfg.Mdiff;
#pragma omp parallel for schedule(static)
    for (size_t k = 0; k < n; k++) {
        const int i = (int)(k % o->nl);
        const double ro = o->ro[k], u = o->u[k], v = o->v[k], w = o->w[k];
        const double gpx = csq * G[ROX][k], gpy = csq * G[ROY][k], gpz = csq * G[ROZ][k];
        /* calc_rhs_ro, :128-139 */
        const double tmp = ((u * G[ROX][k] + v * G[ROY][k]) + w * G[ROZ][k]);
        const double divv = (G[UX][k] + G[VY][k]) + G[WZ][k];
        const double rr = -ro * divv - tmp;
        /* calc_rhs_rovel, :215-275 */
        const double tsu = ro * ((u * G[UX][k] + v * G[UY][k]) + w * G[UZ][k]) - u * rr;
        const double tsv = ro * ((u * G[VX][k] + v * G[VY][k]) + w * G[VZ][k]) - v * rr;
        const double tsw = ro * ((u * G[WX][k] + v * G[WY][k]) + w * G[WZ][k]) - w * rr;
        double fvu = cs * G[LU][k], fvv = cs * G[LV][k], fvw = cs * G[LW][k];
        if (chl) { /* grad c from grad psi, rhs.F90:245-262 */
            const double pxx = o->psi[0][k], pxy = o->psi[1][k], pyy = o->psi[2][k], pxz = o->psi[3][k], pyz = o->psi[4][k],
                         pzz = o->psi[5][k];
            const double gcxx1 = (2.0 * exp(2.0 * pxx)) * gc[0][0][k];
            const double gcxy1 = exp(pxx) * gc[1][0][k] + (pxy * exp(pxx)) * gc[0][0][k];
            const double gcxy2 = exp(pxx) * gc[1][1][k] + (pxy * exp(pxx)) * gc[0][1][k];
            const double gcyy2 = (2.0 * pxy) * gc[1][1][k] + (2.0 * exp(2.0 * pyy)) * gc[2][1][k];
            const double gcxz1 = exp(pxx) * gc[3][0][k] + (pxz * exp(pxx)) * gc[0][0][k];
            const double gcxz3 = exp(pxx) * gc[3][2][k] + (pxz * exp(pxx)) * gc[0][2][k];
            const double gcyz2 = (pxy * gc[3][1][k] + pxz * gc[1][1][k]) + exp(pyy) * (gc[4][1][k] + pyz * gc[2][1][k]);
            const double gcyz3 = (pxy * gc[3][2][k] + pxz * gc[1][2][k]) + exp(pyy) * (gc[4][2][k] + pyz * gc[2][2][k]);
            const double gczz3 = ((2.0 * exp(2.0 * pzz)) * gc[5][2][k] + (2.0 * pxz) * gc[3][2][k]) + (2.0 * pyz) * gc[4][2][k];
            fvu = fvu + cp * ((gcxx1 + gcxy2) + gcxz3);
            fvv = fvv + cp * ((gcxy1 + gcyy2) + gcyz3);
            fvw = fvw + cp * ((gcxz1 + gcyz2) + gczz3);
        }
        if (fen) { /* the quotient rule, rhs_di.F90:234-245 */
            const double f1 = ff[k], g0 = gf[0][k], g1 = gf[1][k], g2 = gf[2][k];
            const double cxx = o->c[0][k], cxy = o->c[1][k], cyy = o->c[2][k], cxz = o->c[3][k], cyz = o->c[4][k], czz = o->c[5][k];
            fvu = fvu + cp * (((((gc[0][0][k] * f1 + cxx * g0) + gc[1][1][k] * f1) + cxy * g1) + gc[3][2][k] * f1) + cxz * g2);
            fvv = fvv + cp * (((((gc[1][0][k] * f1 + cxy * g0) + gc[2][1][k] * f1) + cyy * g1) + gc[4][2][k] * f1) + cyz * g2);
            fvw = fvw + cp * (((((gc[3][0][k] * f1 + cxz * g0) + gc[4][1][k] * f1) + cyz * g1) + gc[5][2][k] * f1) + czz * g2);
        } else if (di || islc) {
            fvu = fvu + cp * ((gc[0][0][k] + gc[1][1][k]) + gc[3][2][k]);
            fvv = fvv + cp * ((gc[1][0][k] + gc[2][1][k]) + gc[4][2][k]);
            fvw = fvw + cp * ((gc[3][0][k] + gc[4][1][k]) + gc[5][2][k]);
        }
        double bfu = ro * (g[0] + df[0]), bfv = ro * (g[1] + df[1]), bfw = ro * (g[2] + df[2]);
        if (s->kolmo) bfu = bfu + (((1.0 / s->cfg.Re) * cos(s->ry[i])) * kol) / kold;
        r[0][k] = rr;
        r[1][k] = ((-tsu - gpx) + bfu) + fvu;
        r[2][k] = ((-tsv - gpy) + bfv) + fvv;
        r[3][k] = ((-tsw - gpz) + bfw) + fvw;
        for (int q = 4; q < 10; q++) r[q][k] = 0.0;
        /* the x-y velocity gradients; a wall node's are in its normal-tangent frame and turn to
           x-y for the conformation equations (rhs_di.F90:497-517, rhs.F90:586-611,
           rhs_lc.F90:602-627; d/dz is d/dz everywhere) */
        const int ty = o->bidx[i] >= 0 ? s->type[i] : 999, wall = ty == 0, inout = ty == 1 || ty == 2;
        double Gux = G[UX][k], Guy = G[UY][k], Gvx = G[VX][k], Gvy = G[VY][k], Gwx = G[WX][k], Gwy = G[WY][k];
        if (wall) {
            const double xn = s->rnx[i], yn = s->rny[i];
            Gux = xn * G[UX][k] - yn * G[UY][k];
            Guy = yn * G[UX][k] + xn * G[UY][k];
            Gvx = xn * G[VX][k] - yn * G[VY][k];
            Gvy = yn * G[VX][k] + xn * G[VY][k];
            Gwx = xn * G[WX][k] - yn * G[WY][k];
            Gwy = yn * G[WX][k] + xn * G[WY][k];
            /* calc_rhs_ro's wall branch (rhs_di.F90:149-154), the wall amplitudes of
               calc_rhs_rovel (:291-307), the isothermal wall (characteristic_boundaries.F90:27-52:
               L5 = L1) and the update of calc_rhs_nscbc (rhs_di.F90:601-665) */
            const double c = sqrt(csq);
            const double un = u * xn + v * yn;
            const double dutdt = -yn * G[UY][k] + xn * G[VY][k];
            const double dundn = xn * G[UX][k] + yn * G[VX][k];
            const double dutdn = -yn * G[UX][k] + xn * G[VX][k];
            const double L1 = (0.5 * (un - c)) * (gpx - (ro * c) * dundn);
            const double L2 = un * (G[ROX][k] - (gpx / c) / c);
            const double L3 = un * dutdn;
            const double L4 = un * (G[WX][k] * xn + G[WY][k] * yn);
            const double L5 = L1;
            const double ts = ((((c * c) * L2 + L5) + L1) / c) / c;
            r[0][k] = (-ro * dutdt - ro * G[WZ][k]) - ts;
            r[1][k] = (0.0 - u * ts) - (L5 - L1) / c;
            r[2][k] = (0.0 - v * ts) - ro * L3;
            r[3][k] = (0.0 - w * ts) - ro * L4;
        } else if (inout) {
            /* inflow (node_type 1) and outflow (2) in the x-y frame: calc_rhs_ro's in/out branch
               (rhs_di.F90:155-157), the amplitudes and the transverse, viscous and body-force
               terms of calc_rhs_rovel (:311-359; no Kolmogorov forcing), the closure of
               characteristic_boundaries.F90 for the node's type (soft :54-80, hard :82-110,
               inflow-outflow :112-150, outflow :152-189) and calc_rhs_nscbc (:601-665) */
            const double c = sqrt(csq), p = csq * ro, uinf = o->uin[k];
            const double nscbc = 2.87e-1, Lx = (s->xmax - s->xmin) * s->cfg.L_char, pin = s->rho_char * s->csq;
            const double rro = ((-v * G[ROY][k] - ro * G[VY][k]) - w * G[ROZ][k]) - ro * G[WZ][k];
            double L1 = (0.5 * (u - c)) * (gpx - (ro * c) * G[UX][k]);
            double L2 = u * (G[ROX][k] - (gpx / c) / c);
            double L3 = u * G[VX][k];
            double L4 = u * G[WX][k];
            double L5 = (0.5 * (u + c)) * (gpx + (ro * c) * G[UX][k]);
            const double bu = ro * (g[0] + df[0]), bv = ro * (g[1] + df[1]), bw = ro * (g[2] + df[2]);
            const double rou = ((-(v * G[UY][k]) - w * G[UZ][k]) + fvu) + bu;
            const double rov = (((-(v * G[VY][k]) - w * G[VZ][k]) - gpy) + fvv) + bv;
            const double row = (((-(v * G[WY][k]) - w * G[WZ][k]) - gpz) + fvw) + bw;
            if (ty == 1) {
                if (s->cfg.inflow_type == 1) {
                    L2 = 0.0; L3 = 0.0; L4 = 0.0; L5 = L1;
                } else if (s->cfg.inflow_type == 2) {
                    if (u > 0.0) {
                        L2 = 0.0;
                        L3 = ((v * nscbc) * c) / Lx;
                        L4 = ((w * nscbc) * c) / Lx;
                        L5 = ((((((u - uinf) * nscbc) * (1.0 - u / c)) * c) * c) * 1.0) / Lx;
                    } else {
                        L2 = 0.0;
                        L5 = (((((p - pin) * nscbc) * c) * 1.0) / 2.0) / Lx;
                    }
                } else {
                    L2 = 0.0;
                    L3 = (((((v * nscbc) * c) / Lx) - v * G[VY][k]) - w * G[VZ][k]) - gpy / ro;
                    L4 = ((w * nscbc) * c) / Lx + row;
                    L5 = (((((((u - uinf) * nscbc) * (1.0 - u / c)) * c) * c) * 1.0) / Lx -
                          0.5 * (((v * gpy) + (p * G[VY][k])) + (((ro * c) * v) * G[UY][k]))) -
                         0.5 * (((w * gpz) + (p * G[WZ][k])) + (((ro * c) * w) * G[UZ][k]));
                }
            } else {
                if (u < c) L1 = (((((p - pin) * nscbc) * c) * 1.0) / 2.0) / Lx;
                L2 = 0.0;
                if (u <= 0.0) { L2 = 0.0; L3 = 0.0; L4 = 0.0; }
            }
            const double ts = ((((c * c) * L2 + L5) + L1) / c) / c;
            r[0][k] = rro - ts;
            r[1][k] = (rou - u * ts) - (L5 - L1) / c;
            r[2][k] = (rov - v * ts) - ro * L3;
            r[3][k] = (row - w * ts) - ro * L4;
        }
        if (chl) { /* calc_rhs_cholesky, rhs.F90:421-556 (sPTT, 3-D), walls :553-717 */
            const double ux = Gux, uy = Guy, uz = G[UZ][k], vx = Gvx, vy = Gvy, vz = G[VZ][k];
            const double wx = Gwx, wy = Gwy, wz = G[WZ][k];
            double ad[6];
            const double ua = ty == 1 ? 0.0 : u; /* inflow: no streamwise advection (rhs.F90:562-564) */
            for (int q = 0; q < 6; q++) ad[q] = (ua * gc[q][0][k] + v * gc[q][1][k]) + w * gc[q][2][k];
            const double lxx = exp(o->psi[0][k]), lxy = o->psi[1][k], lyy = exp(o->psi[2][k]), lzz = exp(o->psi[5][k]);
            const double lxz = o->psi[3][k], lyz = o->psi[4][k];
            double ucxx = (ux + (uy * lxy) / lxx);
            double ucxy = ((vy * lxy + ((uy * lyy) * lyy) / lxx) + vx * lxx);
            double ucyy = (vy - (uy * lxy) / lxx);
            ucxx = ucxx + (uz * lxz) / lxx;
            ucxy = (ucxy + vz * lxz) + ((uz * lyy) * lyz) / lxx;
            ucyy = (ucyy + vz * lyz) - ((uz * lxy) * lyz) / lxx;
            const double ucxz = (((wx * lxx + wy * lxy) + wz * lxz) + ((uy * lyy) * lyz) / lxx) + (uz * ((lyz * lyz) + (lzz * lzz))) / lxx;
            const double ucyz = (((((wy * lyy + wz * lyz) - ((uy * lxz) * lyy) / lxx) + ((uz * lxz) * lyz) / lxx) +
                                  ((vz * lzz) * lzz) / lyy) - (((uz * lxy) * lzz) * lzz) / (lxx * lyy));
            const double uczz = ((wz - (uz * lxz) / lxx) - (vz * lyz) / lyy) + ((uz * lxy) * lyz) / (lxx * lyy);
            const double cxx = o->c[0][k], cxy = o->c[1][k], cyy = o->c[2][k], cxz = o->c[3][k], cyz = o->c[4][k], czz = o->c[5][k];
            double sxx, sxy, syy, sxz, syz, szz;
            if (s->cfg.fenep) { /* rhs.F90:204-209, 479-500: the factors of J = f c */
                const double L2 = s->cfg.fenep_l2;
                const double fr = (L2 - 3.0) / (L2 - ((cxx + cyy) + czz));
                const double srctmp =
                    ((((((((((((2.0 * ux) * cxx + (2.0 * uy) * cxy) + (2.0 * vx) * cxy) + (2.0 * vy) * cyy) + (2.0 * uz) * cxz) +
                           (2.0 * vz) * cyz) + (2.0 * wx) * cxz) + (2.0 * wy) * cyz) + (2.0 * wz) * czz) -
                       (((fr * cxx + fr * cyy) + fr * czz) - 3.0) / lambda) +
                      Md * ((lc[0][k] + lc[2][k]) + lc[5][k])));
                const double den = ((L2 - cxx) - cyy) - czz;
                sxx = (-(fr / lambda) * (fr * cxx - 1.0) + (Md * fr) * lc[0][k]) + ((fr * cxx) * srctmp) / den;
                sxy = (-(fr / lambda) * (fr * cxy) + (Md * fr) * lc[1][k]) + ((fr * cxy) * srctmp) / den;
                syy = (-(fr / lambda) * (fr * cyy - 1.0) + (Md * fr) * lc[2][k]) + ((fr * cyy) * srctmp) / den;
                szz = (-(fr / lambda) * (fr * czz - 1.0) + (Md * fr) * lc[5][k]) + ((fr * czz) * srctmp) / den;
                sxz = (-(fr / lambda) * (fr * cxz) + (Md * fr) * lc[3][k]) + ((fr * cxz) * srctmp) / den;
                syz = (-(fr / lambda) * (fr * cyz) + (Md * fr) * lc[4][k]) + ((fr * cyz) * srctmp) / den;
            } else {
                const double fr = -(((1.0 - eps * 3.0) + eps * ((cxx + cyy) + czz))) / lambda;
                sxx = fr * (cxx - 1.0) + Md * lc[0][k]; sxy = fr * cxy + Md * lc[1][k];
                syy = fr * (cyy - 1.0) + Md * lc[2][k]; sxz = fr * cxz + Md * lc[3][k];
                syz = fr * cyz + Md * lc[4][k]; szz = fr * (czz - 1.0) + Md * lc[5][k];
            }
            const double csxx = ((0.5 * sxx) / lxx) / lxx;
            const double csxy = sxy / lxx - ((0.5 * sxx) * lxy) / (lxx * lxx);
            const double csyy = (((0.5 * syy) / lyy) / lyy - (sxy * lxy) / ((lxx * lyy) * lyy)) +
                                (((0.5 * sxx) * lxy) * lxy) / ((lyy * lyy) * (lxx * lxx));
            double cszz = ((0.5 * szz) / lzz) / lzz;
            const double csxz = sxz / lxx - ((0.5 * sxx) * lxz) / (lxx * lxx);
            const double csyz = ((((syz / lyy - (sxz * lxy) / (lxx * lyy)) +
                                   (((0.5 * sxx) * lxy) * (((2.0 * lxz) * lyy) - lxy * lyz)) / (((lxx * lxx) * lyy) * lyy)) -
                                  ((0.5 * syy) * lyz) / (lyy * lyy)) +
                                 (sxy * ((lxy * lyz) - (lxz * lyy))) / ((lxx * lyy) * lyy));
            cszz = (cszz - ((csxz * lxz) / lzz) / lzz) - ((csyz * lyz) / lzz) / lzz;
            r[4][k] = (-ad[0] + ucxx) + csxx;
            r[5][k] = (-ad[1] + ucxy) + csxy;
            r[6][k] = (-ad[2] + ucyy) + csyy;
            r[7][k] = (-ad[3] + ucxz) + csxz;
            r[8][k] = (-ad[4] + ucyz) + csyz;
            r[9][k] = (-ad[5] + uczz) + cszz;
            continue;
        }
        if (islc) { /* calc_rhs_logconf, rhs_lc.F90:383-560 (sPTT, 3-D), walls :564-740 */
            const int first = (o->itime == 1 && o->iRKstep == 1);
            double ad[6];
            for (int q = 0; q < 6; q++) ad[q] = -((u * gp[q][0][k] + v * gp[q][1][k]) + w * gp[q][2][k]);
            double Lv[3], R[9], RT[9], Gm[9], T[9], M[9], B[9], Om[9], P[9], OP[9], PO[9], UC[9], Ci[9] = {0}, Rx[9];
            eigens3(o->c[0][k], o->c[1][k], o->c[2][k], o->c[3][k], o->c[4][k], o->c[5][k], Lv, R);
            tr3(R, RT);
            const double tr_c = (Lv[0] + Lv[1]) + Lv[2];
            Gm[0] = Gux; Gm[3] = Guy; Gm[6] = G[UZ][k];
            Gm[1] = Gvx; Gm[4] = Gvy; Gm[7] = G[VZ][k];
            Gm[2] = Gwx; Gm[5] = Gwy; Gm[8] = G[WZ][k];
            mm3(Gm, R, T);
            mm3(RT, T, M);
            double oxy = (Lv[1] * M[3] + Lv[0] * M[1]);
            if (fabs(Lv[1] - Lv[0]) <= verysmall) oxy = 0.0;
            else oxy = oxy / (Lv[1] - Lv[0]);
            double oxz = (Lv[2] * M[6] + Lv[0] * M[2]);
            if (fabs(Lv[2] - Lv[0]) <= verysmall) oxz = 0.0;
            else oxz = oxz / (Lv[2] - Lv[0]);
            double oyz = (Lv[2] * M[7] + Lv[1] * M[5]);
            if (fabs(Lv[2] - Lv[1]) <= verysmall) oyz = 0.0;
            else oyz = oyz / (Lv[2] - Lv[1]);
            M[3] = 0.0; M[1] = 0.0; M[6] = 0.0; M[2] = 0.0; M[7] = 0.0; M[5] = 0.0;
            mm3(M, RT, T);
            mm3(R, T, B);
            for (int q = 0; q < 9; q++) M[q] = 0.0;
            M[3] = oxy; M[1] = -oxy; M[6] = oxz; M[2] = -oxz; M[7] = oyz; M[5] = -oyz;
            mm3(M, RT, T);
            mm3(R, T, Om);
            if (first) {
                double GT[9];
                tr3(Gm, GT);
                for (int q = 0; q < 9; q++) { Om[q] = 0.0; B[q] = 0.5 * (Gm[q] + GT[q]); }
            }
            P[0] = o->psi[0][k]; P[3] = o->psi[1][k]; P[1] = o->psi[1][k]; P[4] = o->psi[2][k];
            P[6] = o->psi[3][k]; P[2] = o->psi[3][k]; P[7] = o->psi[4][k]; P[5] = o->psi[4][k]; P[8] = o->psi[5][k];
            mm3(Om, P, OP);
            mm3(P, Om, PO);
            for (int q = 0; q < 9; q++) UC[q] = (OP[q] - PO[q]) + 2.0 * B[q];
            const double fR = ((1.0 - 2.0 * eps) + eps * tr_c);
            Ci[0] = fR / Lv[0] - fR; Ci[4] = fR / Lv[1] - fR; Ci[8] = fR / Lv[2] - fR;
            mm3(Ci, RT, T);
            mm3(R, T, T);
            for (int q = 0; q < 9; q++) Rx[q] = T[q] / lambda;
            static const int e6[6] = {0, 3, 4, 6, 7, 8};
            for (int q = 0; q < 6; q++) /* walls: without the advection (:717-726) */
                r[4 + q][k] = wall ? UC[e6[q]] + Rx[e6[q]] : (ad[q] + UC[e6[q]]) + Rx[e6[q]];
            continue;
        }
        if (!di) continue;
        /* calc_rhs_c, :415-476, walls :478-590 */
        const double cxx = o->c[0][k], cxy = o->c[1][k], cyy = o->c[2][k], cxz = o->c[3][k], cyz = o->c[4][k], czz = o->c[5][k];
        double ad[6];
        for (int q = 0; q < 6; q++) ad[q] = -((u * gc[q][0][k] + v * gc[q][1][k]) + w * gc[q][2][k]);
        const double ux = Gux, uy = Guy, uz = G[UZ][k], vx = Gvx, vy = Gvy, vz = G[VZ][k];
        const double wx = Gwx, wy = Gwy, wz = G[WZ][k];
        const double ucxx = ((2.0 * ux) * cxx + (2.0 * uy) * cxy) + (2.0 * uz) * cxz;
        const double ucxy = (((((ux * cxy + uy * cyy) + uz * cyz) + vx * cxx) + vy * cxy) + vz * cxz);
        const double ucyy = ((2.0 * vx) * cxy + (2.0 * vy) * cyy) + (2.0 * vz) * cyz;
        const double uczz = ((2.0 * wx) * cxz + (2.0 * wy) * cyz) + (2.0 * wz) * czz;
        const double ucxz = (((((ux * cxz + uy * cyz) + uz * czz) + wx * cxx) + wy * cxy) + wz * cxz);
        const double ucyz = (((((vx * cxz + vy * cyz) + vz * czz) + wx * cxy) + wy * cyy) + wz * cyz);
        double sxx, sxy, syy, sxz, syz, szz;
        if (fen) { /* rhs_di.F90:454-464 */
            const double fr = -ff[k];
            sxx = (fr * cxx + 1.0) / lambda; sxy = (fr * cxy) / lambda; syy = (fr * cyy + 1.0) / lambda;
            szz = (fr * czz + 1.0) / lambda; sxz = (fr * cxz) / lambda; syz = (fr * cyz) / lambda;
        } else {
            const double fr = -(((1.0 - eps * 2.0) + eps * ((cxx + cyy) + czz))) / lambda;
            sxx = fr * (cxx - 1.0); sxy = fr * cxy; syy = fr * (cyy - 1.0);
            sxz = fr * cxz; syz = fr * cyz; szz = fr * (czz - 1.0);
        }
        if (inout) continue; /* :582-590: zero on inflow and outflow nodes (to be completed there) */
        if (wall) { /* :571-580: without the advection */
            r[4][k] = (ucxx + sxx) + Md * lc[0][k];
            r[5][k] = (ucxy + sxy) + Md * lc[1][k];
            r[6][k] = (ucyy + syy) + Md * lc[2][k];
            r[7][k] = (ucxz + sxz) + Md * lc[3][k];
            r[8][k] = (ucyz + syz) + Md * lc[4][k];
            r[9][k] = (uczz + szz) + Md * lc[5][k];
            continue;
        }
        r[4][k] = ((ad[0] + ucxx) + sxx) + Md * lc[0][k];
        r[5][k] = ((ad[1] + ucxy) + sxy) + Md * lc[1][k];
        r[6][k] = ((ad[2] + ucyy) + syy) + Md * lc[2][k];
        r[7][k] = ((ad[3] + ucxz) + sxz) + Md * lc[3][k];
        r[8][k] = ((ad[4] + ucyz) + syz) + Md * lc[4][k];
        r[9][k] = ((ad[5] + uczz) + szz) + Md * lc[5][k];
    }
    for (int q = 0; q < NG0; q++) free(G[q]);
    for (int q = 0; q < 6; q++) { for (int d = 0; d < 3; d++) { free(gc[q][d]); free(gp[q][d]); } free(lc[q]); }
    free(ff);
    for (int d = 0; d < 3; d++) free(gf[d]);
}

int or3_rhs(Or3 *o, double *out /* 10 x n3 */) {
    double *r[10];
    for (int q = 0; q < 10; q++) r[q] = out + (size_t)q * o->n3;
    rhs3(o, r);
    return 0;
}

/* set_tstep (step.F90:569-622) over the 3-D nodes */
int or3_set_tstep(Or3 *o, double *dt_cfl, double *dt_par) {
    const OrSim *s = o->s;
    double dcfl = 1.0e10, dvisc = 1.0e10;
    for (size_t k = 0; k < o->n3; k++) {
        const int i = (int)(k % o->nl);
        const double c = sqrt(s->csq);
        const double um = sqrt((o->u[k] * o->u[k] + o->v[k] * o->v[k]) + o->w[k] * o->w[k]);
        const double t = (o->bidx[i] >= 0 && s->type[i] == 2) ? (0.8 * s->sp[i]) / (um + c) : s->sp[i] / (um + c);
        dcfl = (t < dcfl) ? t : dcfl;
        const double tv = ((s->sp[i] * s->sp[i]) * o->ro[k]) / s->visc_total;
        dvisc = (tv < dvisc) ? tv : dvisc;
    }
    o->dt_cfl = (1.0 * dcfl) * s->cfg.L_char;
    o->dt_par = (((2.0 / 3.0) * dvisc) * s->cfg.L_char) * s->cfg.L_char;
    if (dt_cfl) *dt_cfl = o->dt_cfl;
    if (dt_par) *dt_par = o->dt_par;
    return 0;
}

/* step_rk3_4S_2R_EE (step.F90:218-512) in 3-D, with apply_time_dependent_bounds after each
   stage and around the filter (step.F90:346, 488, 498) where the node set has walls */
static void step3(Or3 *o) {
    const OrSim *s = o->s;
    const size_t n = o->n3;
    const int nf = s->cfg.form == OR_FORM_NEWT ? 4 : 10;
    const double a[3] = {RK_A21, RK_A32, RK_A43}, b[4] = {RK_B1, RK_B2, RK_B3, RK_B4};
    const double bh[4] = {RK_BH1, RK_BH2, RK_BH3, RK_BH4};
    const double cc[4] = {0.0, RK_A21, RK_A32 + RK_B1, 1.0};
    const double dt = o->dt;
    o->emax_nm1 = o->emax_n;
    o->emax_n = o->emax_np1;
    double **cq = s->cfg.form == OR_FORM_DI ? o->c : o->psi; /* evolved: c (direct) or psi */
    double *Q[10] = {o->ro, o->rou, o->rov, o->row, cq[0], cq[1], cq[2], cq[3], cq[4], cq[5]};
    double *reg[10], *eacc[10], *r[10];
    for (int f = 0; f < 10; f++) { reg[f] = zarr((int)n); eacc[f] = zarr((int)n); r[f] = zarr((int)n); }
    for (int f = 0; f < nf; f++) memcpy(reg[f], Q[f], sizeof(double) * n);
    const double time0 = o->time;
    o->iRKstep = 0;
    for (int st = 0; st < 4; st++) {
        o->iRKstep++;
        o->time = time0 + dt * cc[st];
        rhs3(o, r);
        const double RKb = dt * b[st], RKbmbh = dt * (b[st] - bh[st]);
        if (st < 3) {
            const double RKa = dt * a[st];
#pragma omp parallel for schedule(static)
            for (size_t k = 0; k < n; k++)
                for (int f = 0; f < nf; f++) {
                    Q[f][k] = reg[f][k] + RKa * r[f][k];
                    reg[f][k] = reg[f][k] + RKb * r[f][k];
                    eacc[f][k] = eacc[f][k] + RKbmbh * r[f][k];
                }
            bounds3(o);
            for (size_t k = 0; k < n; k++) { /* get_velocity_from_momentum */
                const double oo = 1.0 / o->ro[k];
                o->u[k] = o->rou[k] * oo; o->v[k] = o->rov[k] * oo; o->w[k] = o->row[k] * oo;
            }
            or3_c_from_psi(o); /* get_c_from_psi */
        } else {
            double en[10] = {0};
            const double norms[10] = {1.0, 1.0 / (1.0 * s->cfg.U_char), 1.0 / (1.0 * s->cfg.U_char), 1.0 / (1.0 * s->cfg.U_char),
                                      1.0, 1.0, 1.0, 1.0, 1.0, 1.0};
            /* Cholesky FENE-P (step.F90:442-452): the xx, xy, yy and zz errors scaled by
               1/sqrt(f) of the node's c, each node's own before the maximum (the reference
               rescales its running maxima, which depends on the node order) */
            const int chlf = s->cfg.form == OR_FORM_CHL && s->cfg.fenep;
            for (size_t k = 0; k < n; k++) {
                double sc = 1.0;
                if (chlf) {
                    const double L2 = s->cfg.fenep_l2;
                    sc = 1.0 / sqrt((L2 - 3.0) / (((L2 - o->c[0][k]) - o->c[2][k]) - o->c[5][k]));
                }
                double al = 0.0; /* alpha_out (step.F90:456-458): rho, rho u, rho v, xx, xy, yy */
                for (int f = 0; f < nf; f++) {
                    Q[f][k] = reg[f][k] + RKb * r[f][k];
                    eacc[f][k] = eacc[f][k] + RKbmbh * r[f][k];
                    double t = fabs(eacc[f][k]) * norms[f];
                    if (f != 3 && f < 7) al = (t > al) ? t : al;
                    if (f == 4 || f == 5 || f == 6 || f == 9) t = t * sc;
                    en[f] = (t > en[f]) ? t : en[f];
                }
                o->alpha[k] = al;
            }
#define MAXD(x, y) ((x) > (y) ? (x) : (y))
            /* :475-483 (xx xy yy xz yz zz; ro rou rov row) */
            const double econf = MAXD(en[4], MAXD(en[5], MAXD(en[6], MAXD(en[7], MAXD(en[8], en[9])))));
            o->emax_np1 = MAXD(econf, MAXD(en[0], MAXD(en[1], MAXD(en[2], MAXD(en[3], doublesmall)))));
#undef MAXD
            bounds3(o);
        }
    }
    /* filter_variables (rhs_di.F90:667-720): ro, rou, rov, row, then c; the mass correction */
    static const int cls[10] = {0, 1, 2, 0, 0, 3, 0, 0, 0, 0};
    const int chlf = s->cfg.form == OR_FORM_CHL && s->cfg.fenep;
    if (chlf) /* rhs.F90:816-834: filter the factors of c */
        for (size_t k = 0; k < n; k++) {
            double p[6];
            for (int q = 0; q < 6; q++) p[q] = o->psi[q][k];
            chl3_fenep_to_c_factor(s->cfg.fenep_l2, p);
            for (int q = 0; q < 6; q++) o->psi[q][k] = p[q];
        }
    for (int f = 0; f < nf; f++) filter3(o, Q[f], cls[f], r[0]);
    if (chlf) /* :853-868: back to the factors of J */
        for (size_t k = 0; k < n; k++) {
            double p[6];
            for (int q = 0; q < 6; q++) p[q] = o->psi[q][k];
            chl3_fenep_to_j_factor(s->cfg.fenep_l2, p);
            for (int q = 0; q < 6; q++) o->psi[q][k] = p[q];
        }
    if (s->cfg.mcorr) {
        double tm = 0.0, tv = 0.0;
        for (size_t k = 0; k < n; k++) {
            const int i = (int)(k % o->nl);
            tm = tm + (o->ro[k] - s->rho_char) * s->vol[i];
            tv = tv + s->vol[i];
        }
        const double dro = tm / tv;
        for (size_t k = 0; k < n; k++) o->ro[k] = o->ro[k] - dro;
    }
    bounds3(o);
    for (size_t k = 0; k < n; k++) {
        const double oo = 1.0 / o->ro[k];
        o->u[k] = o->rou[k] * oo; o->v[k] = o->rov[k] * oo; o->w[k] = o->row[k] * oo;
    }
    or3_c_from_psi(o);
    for (int f = 0; f < 10; f++) { free(reg[f]); free(eacc[f]); free(r[f]); }
}

/* velocity_control with -Dvpid in 3-D (statistics.F90:214-303): dV = vol dz, summed over the
   node-layers in order (the reference's OpenMP reduction has no fixed order) */
static void velocity_control3(Or3 *o) {
    OrSim *s = o->s;
    double tot_vol = 0.0, tot_u = 0.0;
    for (size_t k = 0; k < o->n3; k++) {
        const double dvi = s->vol[k % o->nl] * o->dz;
        tot_vol = tot_vol + dvi;
        tot_u = tot_u + o->u[k] * dvi;
    }
    tot_u = tot_u / tot_vol;
    const double Lx = (s->xmax - s->xmin) * s->cfg.L_char, Ly = (s->ymax - s->ymin) * s->cfg.L_char;
    const double eflow_n = 1.0 - (tot_u * tot_vol) / (Ly * Lx);
    s->sum_eflow = s->sum_eflow + eflow_n * o->dt;
    const double deflowdt = (eflow_n - s->eflow_nm1) / o->dt;
    const double facA = ((((0.5 * 0.5) * 0.5) * 1.0) * 2.0) * 2.0;
    const double facB = facA / 0.4, facC = facA * 0.02;
    double df = ((facA * eflow_n) + facB * s->sum_eflow) + facC * deflowdt;
    df = (500.0 < df) ? 500.0 : df;
    df = (-500.0 > df) ? -500.0 : df;
    s->driving_force[0] = df;
    s->eflow_nm1 = eflow_n;
}

int or3_step(Or3 *o, double dt, int nsteps, int pid) {
    for (int q = 0; q < nsteps; q++) {
        if (pid) {
            or3_set_tstep(o, NULL, NULL);
            double facA = PID_A * log(pid_tol / o->emax_np1);
            double facB = PID_B * log(o->emax_n / pid_tol);
            double facC = PID_C * log(pid_tol / o->emax_nm1);
            double f = pid_k * exp((facA + facB) + facC);
            f = (0.5 > f) ? 0.5 : f;
            f = (1.02 < f) ? 1.02 : f;
            o->dt = o->dt * f;
            const double dmax = (o->dt_cfl < o->dt_par) ? o->dt_cfl : o->dt_par;
            if (o->dt > dmax) o->dt = dmax;
        } else {
            o->dt = dt;
        }
        step3(o);
        o->itime++;
        /* statistics_control after the step: the controller with -Dvpid, else the driving force
           zeroed (statistics.F90:80-90,288) */
        if (o->s->cfg.vpid) velocity_control3(o);
        else o->s->driving_force[0] = o->s->driving_force[1] = o->s->driving_force[2] = 0.0;
    }
    return 0;
}

/* output_layer in 3-D with -Dallout (output.F90:184-310): 13 columns a node-layer, layer-major:
   rho - rho_char, u, v, w, |vorticity| (walls: the turned gradients of :226-235), Q (never set
   in 3-D by the reference: 0 here), alpha_out, c xx xy yy xz yz zz; the header's 9 values */
int or3_get_dump(Or3 *o, double *out, double *header) {
    const OrSim *s = o->s;
    const size_t n = o->n3;
    double *G[9];
    for (int q = 0; q < 9; q++) G[q] = zarr((int)n);
    grad3(o, o->u, 1, 7, G[0], G[1], G[2]);
    grad3(o, o->v, 2, 7, G[3], G[4], G[5]);
    grad3(o, o->w, 0, 7, G[6], G[7], G[8]);
    for (size_t k = 0; k < n; k++) {
        const int i = (int)(k % o->nl);
        const double ux = G[0][k], uy = G[1][k], uz = G[2][k], vx = G[3][k], vy = G[4][k], vz = G[5][k];
        const double wx = G[6][k], wy = G[7][k];
        double a, b, c;
        if (o->bidx[i] >= 0 && s->type[i] == 0) {
            const double xn = s->rnx[i], yn = s->rny[i];
            a = wy - (xn * vz - yn * uz);
            b = (xn * uz + yn * vz) - wx;
            c = (((xn * vx) - yn * ux) - xn * uy) - yn * vy;
        } else {
            a = wy - vz;
            b = uz - wx;
            c = vx - uy;
        }
        const double col[13] = {-s->rho_char + o->ro[k], o->u[k], o->v[k], o->w[k], sqrt((a * a + b * b) + c * c), 0.0, o->alpha[k],
                                o->c[0][k], o->c[1][k], o->c[2][k], o->c[3][k], o->c[4][k], o->c[5][k]};
        for (int q = 0; q < 13; q++) out[(size_t)q * n + k] = col[q];
    }
    for (int q = 0; q < 9; q++) free(G[q]);
    const double hd[9] = {s->eflow_nm1, s->sum_eflow, s->driving_force[0], 0.0, 0.0, o->emax_np1, o->emax_n, o->emax_nm1, o->dt};
    for (int q = 0; q < 9; q++) header[q] = hd[q];
    return 0;
}

/* mass_and_energy_check in 3-D (statistics.F90:305-330): dV = vol dz, node-layers in order */
double or3_kinetic_energy(Or3 *o) {
    double ke = 0.0;
    for (size_t k = 0; k < o->n3; k++)
        ke = ke + ((0.5 * o->ro[k]) * ((o->u[k] * o->u[k] + o->v[k] * o->v[k]) + o->w[k] * o->w[k])) *
                      (o->s->vol[k % o->nl] * o->dz);
    return ke;
}
double or3_mass(Or3 *o) {
    double m = 0.0;
    for (size_t k = 0; k < o->n3; k++) m = m + o->ro[k] * (o->s->vol[k % o->nl] * o->dz);
    return m;
}

int or3_get_time(Or3 *o, double *time, double *dt, int *itime, double *emax) {
    if (time) *time = o->time;
    if (dt) *dt = o->dt;
    if (itime) *itime = o->itime;
    if (emax) { emax[0] = o->emax_nm1; emax[1] = o->emax_n; emax[2] = o->emax_np1; }
    return 0;
}
