/*
 * sunset_oracle.h -- CPU restatement of SUNSET's LABFM time-step path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA path and the
 * timed CPU baseline; the product (sunset_viscoelastic_b200/) never links or calls it.
 *
 * Parity status: the reference is Fortran 90 and no Fortran compiler exists on
 * either machine, so it cannot be run to produce golden vectors and it ships none
 * (no tests, no fixtures besides the IPART node set).  Parity of this restatement
 * with the reference is therefore UNPINNED by reference outputs; it is pinned by
 * (i) a line-by-line transcription (every function cites the reference file:line it
 * follows, evaluation order kept left-to-right as gfortran evaluates it, compiled
 * with -ffp-contract=off), (ii) the LABFM moment conditions the reference solves for
 * (labf.F90:153-180), checked on the reference's own IPART fixture, and (iii) the
 * reference's analytic checks (mass conservation under mcorr, rhs_di.F90:697-717).
 *
 * Indices are 0-based internally; ij_link exported through or_get_neighbours is
 * 1-based like common_vars.F90:88.  Arrays of per-node data are node-major.
 */
#ifndef SUNSET_ORACLE_H
#define SUNSET_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Conformation-tensor formulation (Makefile:71-90). */
enum { OR_FORM_DI = 0, OR_FORM_CHL = 1, OR_FORM_LC = 2, OR_FORM_NEWT = 3 };

typedef struct {
    int form;               /* OR_FORM_* */
    int fenep;              /* 1: FENE-P (-Dfenep), 0: sPTT / Oldroyd-B */
    int morder, forder;     /* LABFM order of derivatives / filter: 4,6,8,10 */
    int mcorr;              /* mass correction (-Dmcorr, default on) */
    int kolmogorov_forcing; /* -1: as the reference (on for chl only, rhs.F90:275) */
    int di_full_gradients;  /* DI reads d(cxx)/dy, d(cyy)/dx it never computes
                               (rhs_di.F90:186-190,421-423): 1 = compute them,
                               0 = treat them as zero */
    double L_char, U_char, Re, Wi, beta, epsPTT, fenep_l2, Mdiff, Ma;
    double grav[3];
    double h_over_s;        /* >0: h = h_small = h_over_s*s for every node (fixed-radius
                               harness); 0: reference hovs/hovs_bound (common_parameter.F90:44-66) */
    /* inflow boundaries (control.in, load_data.F90:150-152): inflow_type 0 soft
       (non-reflecting), 1 hard, 2 pressure-tracking inflow-outflow; inflow_velocity_control 1
       ramps the inflow velocity from u_inflow_start to u_inflow_end over ramp_time */
    int inflow_type, inflow_velocity_control;
    double u_inflow_start, u_inflow_end, ramp_time;
    int vpid;               /* -Dvpid: PID control of the mean x velocity through driving_force(1)
                               after every step (statistics.F90:214-303) */
} OrConfig;

typedef struct OrSim OrSim;

OrSim *or_create(const OrConfig *cfg);
void or_destroy(OrSim *s);
const char *or_last_error(OrSim *s);
void or_set_threads(int n);

/* build_domain (setup_domain.F90:80-374, non-MPI): rows as in IPART. */
int or_build_domain(OrSim *s, int nrows, const int *gi, const double *x, const double *y,
                    const int *node_type, const double *nx, const double *ny, const double *sp,
                    double xmin, double xmax, double ymin, double ymax, const int *bcond,
                    double smax);
int or_sizes(OrSim *s, int *np, int *npfb, int *nb, int *nplink);
int or_get_nodes(OrSim *s, double *x, double *y, double *h, double *h_small, double *sp,
                 int *node_type, int *irelation, int *vrelation);

int or_find_neighbours(OrSim *s);
int or_adapt_stencils(OrSim *s);        /* labf.F90:1079-1721, then the neighbour search again */
int or_calc_labf_weights(OrSim *s);      /* + calc_filter_weights + calc_node_volumes */
/* sigma_max / sigma_min of each interior node's derivative and filter moment matrices as the
   weight build factored them (npfb each; 0 for boundary nodes, infinite for a zero sigma). */
int or_get_conditioning(OrSim *s, double *cond_deriv, double *cond_filter);
int or_calc_boundary_weights(OrSim *s);
int or_calc_labf_sums(OrSim *s);
int or_filter_coefficients(OrSim *s);
int or_setup_all(OrSim *s);              /* sunset.F90:51-60 sequence */

int or_get_neighbours(OrSim *s, int *ij_count, int *ij_count_small, int *ij_link /* npfb*nplink, 1-based */);
int or_get_weights(OrSim *s, double *w_grad /* npfb*nplink*2 */, double *w_lap, double *w_hyp,
                   double *w_grad_sum /* npfb*2 */, double *w_lap_sum, double *w_hyp_sum,
                   double *vol);
/* Replace neighbours and weights (e.g. with ones built on the device) so that the
   step can be timed / compared without rebuilding them on the host. */
int or_set_neighbours_weights(OrSim *s, int nplink, const int *ij_count, const int *ij_count_small,
                              const int *ij_link /* 1-based into [1,np] */, const double *w_grad,
                              const double *w_lap, const double *w_hyp, const double *w_grad_sum,
                              const double *w_lap_sum, const double *w_hyp_sum, const double *vol);

/* Operators on a field given on the npfb interior nodes (ghosts copied from parents). */
int or_calc_gradient(OrSim *s, const double *phi, double *grad /* npfb*2 */);
int or_calc_laplacian(OrSim *s, const double *phi, double *lap);
int or_calc_filtered_var(OrSim *s, const double *phi, double *out);
int or_calc_filter_term(OrSim *s, const double *phi, double *out);

/* Fields (npfb arrays); psi/c transforms as initial_solution (setup_flow.F90:24-173). */
int or_set_state(OrSim *s, const double *ro, const double *u, const double *v,
                 const double *cxx, const double *cxy, const double *cyy, const double *czz);
int or_set_raw_state(OrSim *s, const double *ro, const double *rou, const double *rov,
                     const double *q /* 4*npfb: xx,xy,yy,zz of c (DI) or psi */);
int or_get_state(OrSim *s, double *out /* 13*npfb: ro rou rov u v psixx psixy psiyy psizz cxx cxy cyy czz */);
int or_calc_all_rhs(OrSim *s, double *rhs /* 7*npfb: ro rou rov xx xy yy zz */);

int or_set_tstep(OrSim *s, double *dt_cfl, double *dt_parabolic);
/* nsteps of step_rk3_4S_2R_EE.  pid=0: fixed dt; pid=1: set_tstep + set_tstep_PID. */
int or_step(OrSim *s, double dt, int nsteps, int pid);
int or_get_time(OrSim *s, double *time, double *dt, int *itime, double *emax /* 3 */);
int or_set_time(OrSim *s, double time, double dt, int itime, const double *emax /* 3 */);
/* the flow-rate controller's state: eflow_nm1, sum_eflow, driving_force(1:3) */
int or_get_flow_control(OrSim *s, double *out /* 5 */);
int or_set_flow_control(OrSim *s, const double *in /* 5 */);
double or_kinetic_energy(OrSim *s);
double or_mass(OrSim *s);

/* Single building blocks exposed for the known-answer tests. */
void or_svd_solve(double *amat /* n*n col-major, untouched */, int n, double *bvec);
double or_wab(double qq, double h2);
void or_monomials(int order, double x, double y, double *out);
void or_abfs(int order, double x, double y, double *out);
double or_pow4_libm(double x);
double or_pow4_cr(double x);
/* 0 (default): Wendland's (1-q/2)**4 through libm pow, as the reference; 1: correctly
   rounded x^4, as the device path evaluates it. */
void or_set_pow_mode(int correctly_rounded);

/* 3-D (-Ddim3), direct, Cholesky, log-conformation (sPTT) and Newtonian forms, node sets without boundary nodes: nz copies of
   the layer in z (build_3rd_dimension, setup_domain.F90:435-547), z derivatives by the periodic
   central differences of fd.F90.  Create after or_setup_all on the layer; Lz is the control
   file's L_domain_z.  Arrays are nl*nz, layer-major (node iz*nl + i). */
typedef struct Or3 Or3;
Or3 *or3_create(OrSim *layer, double Lz);
void or3_destroy(Or3 *o);
int or3_sizes(Or3 *o, int *nl, int *nz, double *dz);
int or3_set_state(Or3 *o, const double *ro, const double *u, const double *v, const double *w,
                  const double *const *c6 /* cxx cxy cyy cxz cyz czz, or NULL: c = I */);
int or3_get_state(Or3 *o, double *out /* 19 x n: ro rou rov row u v w cxx cxy cyy cxz cyz czz, then psixx psixy psiyy psixz psiyz psizz */);
int or3_rhs(Or3 *o, double *out /* 10 x n: ro rou rov row xx xy yy xz yz zz */);
int or3_set_tstep(Or3 *o, double *dt_cfl, double *dt_parabolic);
int or3_step(Or3 *o, double dt, int nsteps, int pid);
int or3_get_time(Or3 *o, double *time, double *dt, int *itime, double *emax /* 3 */);
double or3_kinetic_energy(Or3 *o);
int or3_get_dump(Or3 *o, double *out /* 13 x n */, double *header /* 9 */);
double or3_mass(Or3 *o);

#ifdef __cplusplus
}
#endif
#endif
