/*
 * sunset_gpu.h -- C-ABI of the B200 LABFM time-step path (libsunset_b200.so).
 *
 * Every entry point replaces one Fortran subroutine of the reference (uom-complexfluids/
 * sunset-viscoelastic, cited as file:line inside source/base) and keeps its meaning: the
 * reference's arrays are passed as plain pointers in the reference's node order and
 * layout (1-based neighbour indices, node-major weights), so a thin ISO_C_BINDING module
 * can forward the reference's module arrays unchanged.  The device keeps its own copies
 * (Morton-ordered, sliced-ELL links); host pointers are only read or written inside the
 * call that receives them.
 *
 * All functions return 0 on success or a negative SUNSET_ERR_* code; the message is
 * available from sunset_last_error().  Nothing aborts the host process.  A handle owns
 * one CUDA stream; calls on one handle must not overlap, distinct handles are independent
 * (every kernel takes its run's constants as a launch parameter).
 */
#ifndef SUNSET_GPU_H
#define SUNSET_GPU_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SUNSET_OK 0
#define SUNSET_ERR_ARG -1          /* bad argument or call order */
#define SUNSET_ERR_CUDA -2         /* CUDA runtime error */
#define SUNSET_ERR_SVD -3          /* SVD did not converge in 30 QR sweeps (svdlib.F90:219-222) */
#define SUNSET_ERR_SCOPE -4        /* configuration outside the implemented path */
#define SUNSET_ERR_NONFINITE -5    /* NaN/Inf in the time-step error norm */
#define SUNSET_ERR_NOMEM -6        /* device allocation failed */
#define SUNSET_ERR_ILLCOND -7      /* a moment matrix's condition number exceeds cond_max */

/* Conformation formulation (reference Makefile:71-90 ceform -> -Ddi/-Dchl/-Dlc). */
#define SUNSET_FORM_DI 0
#define SUNSET_FORM_CHL 1
#define SUNSET_FORM_LC 2
#define SUNSET_FORM_NEWT 3

#define SUNSET_FP64 0   /* FP64 throughout: the drop-in */
#define SUNSET_MIXED 1  /* time step streams FP32-rounded weights and keeps FP32 RK increments;
                           weight solves, fields, stencil arithmetic and reductions stay FP64 */

/* Run parameters: the reference's compile-time flags (Makefile) and control.in values
   (load_data.F90:53-159) in one struct. */
typedef struct {
    int form;               /* SUNSET_FORM_* */
    int fenep;              /* 1: FENE-P, 0: sPTT / Oldroyd-B (epsPTT = 0) */
    int morder, forder;     /* LABFM order of derivatives and filter (4, 6, 8, 10) */
    int mcorr;              /* mass correction, reference default on (Makefile:122-125) */
    int kolmogorov_forcing; /* -1: as the reference (on for chl only, rhs.F90:275) */
    int di_full_gradients;  /* DI: compute d(cxx)/dy and d(cyy)/dx, which rhs_di.F90:421-423
                               reads but never computes (1), or take them as zero (0) */
    int precision;          /* SUNSET_FP64 or SUNSET_MIXED */
    double L_char, U_char, Re, Wi, beta, epsPTT, fenep_l2, Mdiff, Ma;
    double grav[3];
    double h_over_s;        /* >0: h = h_small = h_over_s*s (fixed radius 2h); 0: reference
                               hovs/hovs_bound (common_parameter.F90:44-66) */
    int device;             /* CUDA device ordinal */
    /* inflow boundaries (control.in, load_data.F90:150-152): inflow_type 0 soft
       (non-reflecting), 1 hard (prescribed velocity), 2 pressure-tracking inflow-outflow;
       inflow_velocity_control 1 ramps the inflow velocity linearly from u_inflow_start to
       u_inflow_end over ramp_time (characteristic_boundaries.F90:262-300), 0 keeps each inflow
       node's initial u */
    int inflow_type, inflow_velocity_control;
    double u_inflow_start, u_inflow_end, ramp_time;
    int vpid;               /* -Dvpid: after every step a PID controller drives the volume-mean x
                               velocity through driving_force(1) (statistics.F90:214-303) */
    double cond_max;        /* > 0: sunset_calc_labf_weights fails with SUNSET_ERR_ILLCOND when any
                               node's moment matrix has sigma_max/sigma_min above it; 0: such
                               nodes (above 1e12) are only counted, see sunset_get_conditioning.
                               The reference inverts every nonzero sigma (svdlib.F90:283-293) */
    int svd_max_sweeps;     /* QR sweeps per singular value before SUNSET_ERR_SVD; 0: the
                               reference's 30 (svdlib.F90:219-222) */
} SunsetConfig;

typedef struct SunsetHandle SunsetHandle;

/* flags for the operator calls */
#define SUNSET_PTR_HOST 0    /* arrays are host memory */
#define SUNSET_PTR_DEVICE 1  /* arrays are device memory on the handle's device */

int sunset_create(const SunsetConfig *cfg, SunsetHandle **out);
void sunset_destroy(SunsetHandle *h);
const char *sunset_last_error(const SunsetHandle *h);
int sunset_version(void);
/* The SASS target the library's kernels were built for, as the CUDA runtime reports it for
   one of them on `device` (cudaFuncGetAttributes binaryVersion: 100 for sm_100a), or a
   negative SUNSET_ERR_* code.  No reference counterpart. */
int sunset_kernel_binary_version(int device);

/* setup_domain.F90:80-374 build_domain (IPART rows -> nodes, 4 FD rows per boundary node)
   + mirror_boundaries.F90:34-261 create_mirror_particles, as device-resident ghost points.
   bcond = {xbcond_L, xbcond_U, ybcond_L, ybcond_U}. */
int sunset_build_domain(SunsetHandle *h, int nrows, const int *global_index, const double *x,
                        const double *y, const int *node_type, const double *nx, const double *ny,
                        const double *s, double xmin, double xmax, double ymin, double ymax,
                        const int *bcond, double smax);
/* np (nodes + ghosts), npfb, nb, nplink (max neighbours) */
int sunset_get_sizes(SunsetHandle *h, int *np, int *npfb, int *nb, int *nplink);

/* neighbours.F90:32-341 find_neighbours: cell-list search + per-row distance sort. */
int sunset_find_neighbours(SunsetHandle *h);
/* labf.F90:1079-1721 adapt_stencils + adapt_stencils_main: per interior node (node_type 999)
   the smoothing length h, and then h_small, shrink by 2% steps while the Laplacian system's
   residual, the stencils' amplification of wavenumbers up to Nyquist and the reduction count
   stay within the reference's limits; then the neighbour lists are rebuilt with the new
   lengths (sunset.F90:43-51).  Call after sunset_find_neighbours, before the weights. */
int sunset_adapt_stencils(SunsetHandle *h);
/* The smoothing lengths h and h_small of the npfb nodes (reference order), the module
   arrays of common_vars.F90 that sunset_adapt_stencils changes. */
int sunset_get_lengths(SunsetHandle *h, double *h_out, double *h_small_out);
/* labf.F90:34-231 calc_labf_weights (+ calc_filter_weights :233-394). */
int sunset_calc_labf_weights(SunsetHandle *h);
/* Conditioning of the weight solves of sunset_calc_labf_weights (labf.F90:153-180, 325-388):
   sigma_max/sigma_min of each interior node's derivative and filter moment matrix, npfb each in
   reference order (0 for boundary nodes, which that call does not build; any pointer may be
   NULL), the worst value, and the number of nodes above cond_max (1e12 when cond_max is 0).
   The reference has no such output: it solves whatever it is given. */
int sunset_get_conditioning(SunsetHandle *h, double *cond_deriv, double *cond_filter, double *worst, int *n_ill);
/* labf.F90:505-1039 calc_boundary_weights: prunes the links of boundary nodes to their own
   layer and FD children, then FD normal and 1-D LABFM tangential operators for boundary
   nodes and FD rows 1-2, curvature and frame rotations.  A no-op without boundary nodes;
   required between sunset_calc_labf_weights and sunset_calc_labf_sums when there are. */
int sunset_calc_boundary_weights(SunsetHandle *h);
/* labf.F90:396-451 calc_labf_sums (+ node volumes, labf.F90:453-503). */
int sunset_calc_labf_sums(SunsetHandle *h);
/* labf.F90:1723-1811 filter_coefficients. */
int sunset_filter_coefficients(SunsetHandle *h);

/* ij_count(npfb), ij_count_small(npfb), ij_link(nplink*npfb) 1-based into [1,np] with the
   reference's ghost numbering (common_vars.F90:87-88). */
int sunset_get_neighbours(SunsetHandle *h, int *ij_count, int *ij_count_small, int *ij_link);
/* ij_w_grad(2,nplink,npfb), ij_w_lap(nplink,npfb), ij_w_hyp(nplink,npfb), ij_w_grad_sum(2,npfb),
   ij_w_lap_sum(npfb), ij_w_hyp_sum(npfb), vol(npfb) (common_vars.F90:91-94). Any may be NULL. */
int sunset_get_weights(SunsetHandle *h, double *w_grad, double *w_lap, double *w_hyp,
                       double *w_grad_sum, double *w_lap_sum, double *w_hyp_sum, double *vol);

/* derivatives.F90 operators on a field phi(npfb) in reference order (ghost values follow
   their parents): calc_gradient :26-71 -> grad(npfb,2) node-major; calc_laplacian :73-116;
   calc_filtered_var :360-414 (out-of-place); calc_filter_term :466-511. */
int sunset_calc_gradient(SunsetHandle *h, const double *phi, double *grad, int flags);
int sunset_calc_laplacian(SunsetHandle *h, const double *phi, double *lap, int flags);
int sunset_calc_filtered_var(SunsetHandle *h, const double *phi, double *out, int flags);
int sunset_calc_filter_term(SunsetHandle *h, const double *phi, double *out, int flags);

/* Fields in reference order (npfb each).  setup_flow.F90:24-173 initial_solution: rho, u,
   v and the conformation tensor c; psi is formed from c as the formulation requires. */
int sunset_set_state(SunsetHandle *h, const double *ro, const double *u, const double *v,
                     const double *cxx, const double *cxy, const double *cyy, const double *czz);
/* 13*npfb: ro rou rov u v psixx psixy psiyy psizz cxx cxy cyy czz */
int sunset_get_state(SunsetHandle *h, double *out);
/* rhs_*.F90 calc_all_rhs at the current state: 7*npfb: ro rou rov xx xy yy zz */
int sunset_calc_all_rhs(SunsetHandle *h, double *out);

/* step.F90:569-622 set_tstep: the CFL and viscous limits at the current state. */
int sunset_set_tstep(SunsetHandle *h, double *dt_cfl, double *dt_parabolic);
/* step.F90:218-512 step_rk3_4S_2R_EE, nsteps times.  mode 0: fixed dt; mode 1: set_tstep +
   set_tstep_PID (step.F90:624-682) before every step.  Steps run as a captured CUDA graph. */
int sunset_step(SunsetHandle *h, double dt, int nsteps, int mode);
/* time, dt, itime, emax(3) = {emax_nm1, emax_n, emax_np1} */
int sunset_get_time(SunsetHandle *h, double *time, double *dt, int *itime, double *emax);
int sunset_set_time(SunsetHandle *h, double time, double dt, int itime, const double *emax);
/* sum 0.5 rho |u|^2 dV and sum rho dV over the interior nodes (mass_and_energy_check,
   statistics.F90:305-330): dV = vol in 2-D, vol dz over the node-layers of a 3-D handle */
int sunset_kinetic_energy(SunsetHandle *h, double *ke);
int sunset_mass(SunsetHandle *h, double *mass);
int sunset_synchronize(SunsetHandle *h);

/* Host-buffer round trip, the drop-in use from a host code that owns the fields: copy the
   evolved variables in from host arrays (pinned for full speed), run nsteps, copy them
   back.  7*npfb in reference order: ro rou rov q_xx q_xy q_yy q_zz, q = c (DI) or psi.  On a
   3-D handle 10*npfb*nz, layer-major: ro rou rov row q_xx q_xy q_yy q_xz q_yz q_zz (the first 4
   for the Newtonian form). */
int sunset_run_host(SunsetHandle *h, const double *state_in, double dt, int nsteps, double *state_out);

/* sunset_step with the steps bracketed by CUDA events on the handle's stream: *ms is the
   device time of the nsteps steps. */
int sunset_step_timed(SunsetHandle *h, double dt, int nsteps, int mode, double *ms);

/* ---- 3-D (-Ddim3): direct, Cholesky, log-conformation (sPTT) and Newtonian forms, FENE-P with
   the direct and Cholesky forms, FP64, node sets with or without boundary nodes (walls, inflow,
   outflow), the flow-rate controller ---- */
/* build_3rd_dimension (setup_domain.F90:435-547) and calc_fd_weights (fd.F90:27-256): after
   sunset_build_domain, the node set becomes nz layers in z over L_domain_z (the control file's
   value): dz from the mean spacing, nz = ceiling(L_domain_z/dz), at least ij_count_fd/2 + 2,
   z-derivatives by periodic central differences of forder + 1 points.  The neighbour lists and
   weights are built for the layer (the same calls as in 2-D) and serve every layer.  Then
   sunset_set_state_3d, and sunset_step / sunset_set_tstep / sunset_get_time act on the 3-D
   state.  Arrays are npfb*nz, layer-major (node iz*npfb + i, reference order in the layer).
   Boundary nodes are boundary nodes of every layer (node_type and normals copied, :487-532):
   the wall and inflow/outflow branches of the right-hand sides apply with their dim3 terms,
   u_inflow_local is kept for every inflow node-layer, and sunset_get_flow_control /
   sunset_set_flow_control read and set the controller of a -Dvpid run as in 2-D. */
int sunset_set_layers(SunsetHandle *h, double L_domain_z);
int sunset_get_layers(SunsetHandle *h, int *nz, double *dz);
/* initial_solution in 3-D: rho, u, v, w and the six c components (all NULL: c = I) */
int sunset_set_state_3d(SunsetHandle *h, const double *ro, const double *u, const double *v, const double *w,
                        const double *cxx, const double *cxy, const double *cyy, const double *cxz,
                        const double *cyz, const double *czz);
/* 19*npfb*nz: ro, rou, rov, row, u, v, w, cxx, cxy, cyy, cxz, cyz, czz, psixx, psixy, psiyy,
   psixz, psiyz, psizz (the Cholesky or log-conformation variables; zero otherwise) */
int sunset_get_state_3d(SunsetHandle *h, double *out);
/* calc_all_rhs with the dim3 terms (rhs_di.F90, rhs.F90): 10*npfb*nz: ro, rou, rov, row, xx,
   xy, yy, xz, yz, zz (of c in the direct form, of psi in the Cholesky and log-conformation
   forms) */
int sunset_calc_all_rhs_3d(SunsetHandle *h, double *out);

/* ---- Dumps, restart, checkpoints ---- */
/* output.F90:184-370 output_layer: the columns of a fields dump, 10*npfb in reference order
   (rho - rho_char, u, v, vorticity, Q criterion, alpha_out = the node's error norm of the
   last step, cxx, cxy, cyy, czz; vorticity and Q rotated on walls as :229-241), and the
   header's 9 values (eflow_nm1, sum_eflow, driving_force(3) of the flow-rate controller,
   emax_np1, emax_n, emax_nm1, dt).  On a 3-D handle the -Dallout dump of :296-299, 13*npfb*nz
   over every node-layer, layer-major: rho - rho_char, u, v, w, |vorticity| (3-D gradient;
   on walls as :226-235), Q (never set by the reference in 3-D: 0), alpha_out, cxx, cxy, cyy,
   cxz, cyz, czz. */
int sunset_get_dump(SunsetHandle *h, double *columns, double *header);
/* The same as files in the reference's layout: <directory>/fields_10000_<n_out>, with
   <directory>/nodes_10000 (output_nodes, output.F90:421-476: global index, x, y, s, h,
   h_small, node type) when n_out == 1, and a line "time 2 npfb n_out 1" appended to
   <directory>/time.out.  Readable by the reference's restart loader and vtk_conv.  3-D: the
   13-column rows of every node-layer, nodes with z and the layer offset of the global index
   (setup_domain.F90:520-535), "time 3 npfb*nz n_out 1". */
int sunset_write_dump(SunsetHandle *h, const char *directory, int n_out, double time);
/* Restart (-Drestart): setup_domain.F90:206-242 loads h and h_small from the nodes file
   before the neighbour search (adapt_stencils is skipped); load_restart_file,
   setup_flow.F90:448-552, sets rho, u, v and c (psi formed from c) and the error-norm history
   and dt and the flow-rate controller's state from a fields dump (columns and header as
   sunset_get_dump returns them; driving_force(2:3) must be zero).  Time and step count
   restart at 0, as there.  On a 3-D handle from the 13 columns (:505-509: rho, u, v, w, c). */
int sunset_set_lengths(SunsetHandle *h, const double *h_lengths, const double *h_small);
int sunset_set_restart(SunsetHandle *h, const double *columns, const double *header);
/* The flow-rate controller's state (common_vars.F90:82, statistics.F90:214-303): eflow_nm1,
   sum_eflow, driving_force(1:3), 5 values. */
int sunset_get_flow_control(SunsetHandle *h, double *out);
int sunset_set_flow_control(SunsetHandle *h, const double *in);
/* Binary checkpoint of the device state between steps (no counterpart in the reference):
   the fields, the step's scalars (time, dt, step count, error-norm history) and the per-node
   error, bit for bit, into a caller buffer of sunset_checkpoint_size bytes.  Loading it into
   a handle built on the same node set and configuration resumes the run exactly.  A 3-D
   handle's checkpoint holds the 19 fields of every node-layer, the node-layers' step error and
   u_inflow_local, and loads only into a handle with the same layers. */
int sunset_checkpoint_size(SunsetHandle *h, size_t *bytes);
int sunset_save_checkpoint(SunsetHandle *h, void *buffer, size_t bytes);
int sunset_load_checkpoint(SunsetHandle *h, const void *buffer, size_t bytes);

/* Stage-kernel timing: runs `reps` fixed-dt steps at the current dt, launched kernel by
   kernel (not as a graph) with CUDA events on the handle's stream before the first and after
   the last of each step's four RK stage launches (which run back to back), and returns the
   mean stage-kernel time per launch in ms and its algorithmic bytes per launch.  Advances the
   state by `reps` steps.  On a 3-D handle it times the derivative gather of each stage
   (events around each launch) at the current dt instead. */
int sunset_time_stage_kernel(SunsetHandle *h, int reps, double *ms_per_launch,
                             double *bytes_per_launch);

/* Adjoint of the fixed-dt time step (log-conformation form, FP64, node sets without walls).
   From the current state it runs nsteps steps of size dt (the handle ends at the final
   state), evaluates J = sum_i 1/2 rho_i |u_i|^2 vol_i at the final state, and returns dJ/dWi
   and dJ/dbeta in dJ_dparams[2] and, unless dJ_dstate0 is NULL, dJ with respect to the
   initial state (7*npfb host doubles in reference order: ro rou rov psixx psixy psiyy psizz).
   The reverse sweep recomputes each segment of checkpoint_every steps from its stored state,
   recording the stage inputs and stencil sums (device memory: about
   (124 * checkpoint_every + 7 * nsteps / checkpoint_every) doubles a node, plus the reverse
   link streams).  The adjoint is of the discrete step as computed (step.F90:218-512 with the filter
   and the mass correction); SUNSET_ERR_SCOPE for other forms, mixed precision, walls or
   Mdiff != 0.  No reference counterpart (the reference has no adjoint). */
int sunset_adjoint_run(SunsetHandle *h, double dt, int nsteps, int checkpoint_every, double *J,
                       double *dJ_dparams, double *dJ_dstate0);

/* Transposed single operators: out = D^T gbar with D the operator of sunset_calc_gradient
   (which 0: d/dx, 1: d/dy), sunset_calc_laplacian (2) or sunset_calc_filter_term (3),
   npfb values in reference order, flags as for the operators.  A gather over the reverse
   neighbour lists (deterministic, no atomics).  No reference counterpart. */
int sunset_adjoint_apply_D(SunsetHandle *h, int which, const double *gbar, double *out, int flags);

/* Allocation-free variant of sunset_kinetic_energy/sunset_mass; it has no counterpart in
   the reference.  For callers that cannot allocate device memory (their arrays live in
   their own device pool, and cudaMalloc could synchronise the device or exceed a memory
   cap): they pass device arrays they own, ro, u, v, vol (npfb each, any consistent node
   order) and out (2 doubles, device), and get out[0] = sum 0.5 ro (u^2+v^2) vol and
   out[1] = sum ro vol.  The partial sums use a static device array sized for at most
   4,194,304 nodes (256 KB per GPU, held until the process exits); larger npfb returns
   SUNSET_ERR_SCOPE.  The first call on a device looks the array's address up and should
   come before any stream capture.  Work is enqueued on `stream` (NULL: the default
   stream); the calling thread's current device is left as it was.  All calls share the
   array, so calls that overlap on the GPU race. */
int sunset_kinetic_energy_noalloc(int device, int npfb, const double *ro, const double *u, const double *v,
                                  const double *vol, double *out, void *stream);

#ifdef __cplusplus
}
#endif
#endif
