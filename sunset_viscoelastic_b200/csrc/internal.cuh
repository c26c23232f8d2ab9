// internal.cuh -- shared definitions of the B200 LABFM path (device layout, handle, helpers).
//
// Device layout
//   * Interior nodes are renumbered in Morton (Z-curve) order of their position; perm[i]
//     gives the reference index of internal node i, iperm the inverse.
//   * Ghost points (the reference's mirror nodes, mirror_boundaries.F90:34-261) exist only
//     as positions for the weight build; each link stores the internal index of the
//     parent plus a 2-bit reflection code, so fields are never copied to ghosts.
//   * Links are kept in sliced ELL: slices of 32 consecutive internal nodes, each padded
//     to its own (even) width; links k = 2m, 2m+1 of node i sit next to each other at
//     slice_ptr[i/32] + 64 m + 2 (i%32) (sell_at), so a warp reading link pair m of its 32
//     nodes issues one coalesced 512-byte access.  Padding has weight 0 and points at node 0.
//   * The time step streams its own copy of the links (stream.cu): the same SELL slots with
//     each node's links in a shared-memory-bank-aware order, FP64 or (mixed) FP32 weights.
//   * Fields are structure-of-arrays FP64 in both precisions; the mixed path keeps FP32 RK
//     increments, stages each tile's halo as FP32 offsets from a per-tile FP64 reference
//     and sums the stencils in FP32 difference form.
#pragma once

#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/sunset_gpu.h"

namespace sunset {

constexpr double kPi = 3.141592653589793238462643383279502884197;
constexpr double kSs = 2.0;  // stencil support in units of h, common_parameter.F90:68
constexpr int kSlice = 32;
constexpr int kLinkMask = 0x3fffffff;  // low 30 bits: internal parent index
#ifndef SUNSET_TILE_SLICES
#define SUNSET_TILE_SLICES 8
#endif
constexpr int kTileSlices = SUNSET_TILE_SLICES;  // slices per thread block of the staged stencil kernels
constexpr int kTile = kTileSlices * 32;
// per-tile partial sums live in a buffer of nodes / 128 + 1 entries
static_assert(kTile >= 128 && kTile <= 1024, "tile of 128 to 1024 nodes");
constexpr int kLocMask = 0x3fff;       // low 14 bits of a local link: position in the tile's halo
// Condition number above which a moment matrix is counted as ill-conditioned when the run
// sets no limit of its own (SunsetConfig::cond_max = 0): its weights lose about 12 of
// FP64's 16 digits.
constexpr double kCondWarn = 1.0e12;

// RK3(2)4[2R+]C, common_parameter.F90:74-94
#define SUNSET_RK_A21 (11847461282814.0 / 36547543011857.0)
#define SUNSET_RK_A32 (3943225443063.0 / 7078155732230.0)
#define SUNSET_RK_A43 (-346793006927.0 / 4029903576067.0)
#define SUNSET_RK_B1 (1017324711453.0 / 9774461848756.0)
#define SUNSET_RK_B2 (8237718856693.0 / 13685301971492.0)
#define SUNSET_RK_B3 (57731312506979.0 / 19404895981398.0)
#define SUNSET_RK_B4 (-101169746363290.0 / 37734290219643.0)
#define SUNSET_RK_BH1 (15763415370699.0 / 46270243929542.0)
#define SUNSET_RK_BH2 (514528521746.0 / 5659431552419.0)
#define SUNSET_RK_BH3 (27030193851939.0 / 9429696342944.0)
#define SUNSET_RK_BH4 (-69544964788955.0 / 30262026368149.0)

inline int nsize_for(int k) { return (k * k + 3 * k) / 2; }  // labf.F90:56

// Position of link k of lane `lane` in the slice stored from `base`.  Links are stored in
// pairs, so one 16-byte load brings links 2m and 2m+1 of a node and a warp's pair load is
// 512 contiguous bytes; slice widths are even.
__host__ __device__ __forceinline__ long long sell_at(long long base, int k, int lane) {
    return base + ((long long)(k >> 1) << 6) + (lane << 1) + (k & 1);
}
// The mixed stage's packed links (stream.cu) interleave the three words of a link: pair m of
// lane `lane` holds x, y, l of link 2m then of link 2m+1 in six consecutive words, so a warp's
// pair row is 768 contiguous bytes and a slice's rows follow each other.  Word 0 of link k:
__host__ __device__ __forceinline__ long long pk_at(long long base, int k, int lane) {
    return 3 * (base + ((long long)(k >> 1) << 6)) + 6 * lane + 3 * (k & 1);
}
// The mixed filter's links: per pair and lane three words, the FP32 weights of links 2m and
// 2m+1 and their two 16-bit local indices (low half: link 2m); a warp's pair row is 384
// contiguous bytes.  Word 0 of pair m:
__host__ __device__ __forceinline__ long long wf_at(long long base, int m, int lane) {
    return (3 * (base + ((long long)m << 6))) / 2 + 3 * lane;
}

// Scalars the step kernels share on the device (one per handle).
struct DevScalars {
    double dt, time;
    double emax_nm1, emax_n, emax_np1;
    double dro;            // mass correction of the current step
    double tv;             // sum of node volumes (constant once the weights exist)
    double dt_cfl, dt_par; // set_tstep results of the current state
    unsigned long long emax_bits;  // running max of the step's error norm (bit pattern)
    unsigned long long cfl_bits, par_bits;  // running minima (bit patterns, positive)
    unsigned int done_ctr;  // last-block counter of the mass reduction
    int itime;
    int err;  // 1: non-finite error norm; 2: a bounded wait on the stage's link stream gave up
    // flow-rate controller (statistics.F90:214-303): driving_force(1), eflow_nm1, sum_eflow
    double df, eflow_nm1, sum_eflow;
};

// One buffer of the state: conservative fields, conformation variables and the derived
// fields (velocity and c) the stencils read.
struct Fields {
    double *ro, *rou, *rov;
    double *q[4];   // DI: cxx cxy cyy czz; LC/CHL: psixx psixy psiyy psizz
    double *u, *v;
    double *c[4];   // cxx cxy cyy czz (DI: aliases q)
    double *f;      // FENE-P function (L^2 - 3) / (L^2 - tr c) of DI and LC (its gradient
                    // enters the momentum equation); null otherwise
};

struct StepConsts {
    int npfb, nslices, form, fenep, mcorr, kolmo, di_full, has_mirrors, mdiff_on, has_walls;
    double csq, c_sound, coef_solvent, coef_polymeric, lambda, epsPTT, fenep_l2, Mdiff, Re, Wi, beta;
    double visc_total, rho_char, L_char, grav0, grav1, ero_norm, erou_norm, exx_norm;
    // inflow/outflow closures and the flow-rate controller (load_data.F90:145-152,
    // setup_domain.F90:98-99, common_parameter.F90:71)
    int inflow_type, inflow_control, vpid;
    double u_in_start, u_in_end, ramp_time, nscbc, Lx, Ly, p_in, p_out;
};

// Derived parameters of a run (load_data.F90:131-148) and the switches of the step kernels.
inline StepConsts step_consts(const SunsetConfig &c, int npfb, int nslices, bool has_mirrors, bool has_walls,
                              double xlen = 1.0, double ylen = 1.0) {
    StepConsts K{};
    K.npfb = npfb;
    K.nslices = nslices;
    K.form = c.form;
    K.fenep = c.fenep;
    K.mcorr = c.mcorr;
    K.kolmo = c.kolmogorov_forcing < 0 ? (c.form == SUNSET_FORM_CHL) : c.kolmogorov_forcing;
    K.di_full = c.di_full_gradients;
    K.has_mirrors = has_mirrors;
    K.has_walls = has_walls;
    K.mdiff_on = c.Mdiff != 0.0;
    double t = c.U_char / c.Ma;
    K.csq = t * t;
    K.c_sound = sqrt(K.csq);
    K.rho_char = 1.0;
    K.visc_total = K.rho_char * c.U_char * c.L_char / c.Re;
    K.coef_solvent = c.beta * K.visc_total;
    K.lambda = c.Wi * c.L_char / c.U_char;
    K.coef_polymeric = ((1.0 - c.beta) * K.visc_total) / K.lambda;
    K.epsPTT = c.epsPTT;
    K.fenep_l2 = c.fenep_l2;
    K.Mdiff = c.Mdiff;
    K.Re = c.Re;
    K.Wi = c.Wi;
    K.beta = c.beta;
    K.L_char = c.L_char;
    K.grav0 = c.grav[0];
    K.grav1 = c.grav[1];
    K.ero_norm = 1.0 / 1.0;
    K.erou_norm = 1.0 / (1.0 * c.U_char);
    K.exx_norm = 1.0 / (1.0);
    K.inflow_type = c.inflow_type;
    K.inflow_control = c.inflow_velocity_control;
    K.vpid = c.vpid;
    K.u_in_start = c.u_inflow_start;
    K.u_in_end = c.u_inflow_end;
    K.ramp_time = c.ramp_time;
    K.nscbc = 2.87e-1;
    K.Lx = xlen * c.L_char;
    K.Ly = ylen * c.L_char;
    K.p_in = K.rho_char * K.csq;
    K.p_out = K.rho_char * K.csq;
    return K;
}

struct Handle {
    SunsetConfig cfg{};
    std::string err;
    int device = 0;
    cudaStream_t stream = nullptr;

    // ---- domain (host copies kept for export) ----
    int npfb = 0, np = 0, nb = 0, nghost = 0, nrows = 0;
    double xmin = 0, xmax = 0, ymin = 0, ymax = 0, smax = 0, h0 = 0, h2 = 0, h3 = 0, hmax = 0;
    int bc[4] = {0, 0, 0, 0};
    std::vector<int> h_perm, h_iperm;  // internal <-> reference
    std::vector<int> h_gi;             // global index of each node (reference order; FD rows: parent's + j)
    bool domain_ok = false, nbr_ok = false, w_ok = false, bw_ok = false, sums_ok = false, fc_ok = false;
    bool state_ok = false, state3_ok = false;

    // ---- device: points (internal interior 0..npfb-1, ghosts npfb..np-1) ----
    double *px = nullptr, *py = nullptr;       // np
    double *h = nullptr, *hs = nullptr, *sp = nullptr;  // npfb (internal order)
    int *ntype = nullptr;                      // npfb
    int *gpar = nullptr, *gvrel = nullptr;     // ghosts: parent (internal), vrel 1..4
    int *perm = nullptr, *iperm = nullptr;     // npfb
    // boundary framework: boundary nodes (node_type 0..2) in the reference's order jj
    double *rnx = nullptr, *rny = nullptr;     // npfb: unit normal into the fluid (0 for fluid nodes)
    int *fdpar = nullptr;                      // npfb: FD parent of an FD row, -1 otherwise
    int *blist = nullptr, *brow = nullptr;     // nb: boundary node jj; 4*nb: its FD rows 1..4
    int *bidx = nullptr;                       // npfb: jj of a boundary node, -1 otherwise
    std::vector<int> h_btype;                  // nb: node type of boundary node jj

    // ---- neighbours (sliced ELL) ----
    int nslices = 0, nplink = 0;
    long long nlinks_sell = 0;
    long long *slice_ptr = nullptr;            // nslices+1
    int *slice_w = nullptr, *slice_ws = nullptr;  // widths: all links, small links
    int *cnt = nullptr, *cnt_small = nullptr;  // npfb
    int *lpt = nullptr;                        // SELL: point id (ghost-aware), for setup/export
    int *lidx = nullptr;                       // SELL: parent | vrel code << 30
    bool has_mirrors = false;
    // tiles of kTileSlices slices: the sorted set of nodes their links reach (the halo) and,
    // per link, the position of its parent in that set | reflection code << 14
    int ntiles = 0, halo_max = 0;
    int *halo_ptr = nullptr, *halo = nullptr;
    uint16_t *lloc = nullptr;

    // ---- weights (SELL, FP64) ----
    double *wx = nullptr, *wy = nullptr, *wl = nullptr, *wh = nullptr;
    // condition numbers of each interior node's derivative / filter moment matrix (internal
    // order), the worst one and how many exceed the limit
    double *cond_d = nullptr, *cond_f = nullptr;
    double cond_worst = 0.0;
    int cond_nill = 0;
    bool cond_ok = false;
    double *gsx = nullptr, *gsy = nullptr, *lsum = nullptr, *hsum = nullptr, *vol = nullptr;
    // mixed precision: the stage's links packed as three words (26-bit fixed-point weight of
    // d/dx, d/dy, Laplacian with 6 bits of the local index each, stream.cu), interleaved per
    // link pair and lane, and their per-node scales; the filter's FP32 weights with their
    // local indices, interleaved likewise
    unsigned *pk = nullptr;  // 3 words a SELL slot, interleaved (pk_at)
    float *scx = nullptr, *scy = nullptr, *scl = nullptr;
    unsigned *wf = nullptr;  // 1.5 words a SELL slot (wf_at)
    // the time step's link stream: local links and (FP64 step) weights in the bank-aware
    // order of stream.cu; the arrays above stay in the reference's order
    uint16_t *lloc_s = nullptr;
    double *wx_s = nullptr, *wy_s = nullptr, *wl_s = nullptr, *wh_s = nullptr;
    double *wb2 = nullptr;  // nb x nplink x 2: normal and tangential second derivatives of boundary nodes
    double *wbt = nullptr, *wbt_sum = nullptr;  // nb x nplink, nb: tangential ones scaled by 1/L^2 (reference
                                                // link order) and their sums: the wall Laplacian of c

    // ---- state ----
    Fields buf[2]{};
    int cur = 0;  // buffer holding the current state
    double *reg[7] = {};   // RK register S: ro rou rov q0..q3
    double *eacc[7] = {};  // error accumulators
    double *rhs[7] = {};   // rhs output of sunset_calc_all_rhs
    // mixed precision: RK register as the FP32 increment D = S - U over the stage's state,
    // and the error accumulator in FP32
    float *dreg32[7] = {}, *eacc32[7] = {};
    double *partials = nullptr;
    double *alpha = nullptr;  // per-node step error of the last step (output.F90 alpha_out)
    double *uin = nullptr;    // nb: u_inflow_local of each boundary node (common_vars.F90:111)
    bool uin_set = false;     // uin initialised from a state
    int npart = 0;
    DevScalars *dsc = nullptr;
    double *tmpd = nullptr;  // scratch, 4*npfb doubles
    double *io = nullptr;    // 7*npfb staging block of sunset_run_host

    // ---- 3-D (step3d.cu): nz layers of the node set, z stencils of fd.F90 ----
    int nz = 0, ncfd = 0, cur3 = 0;
    double dz = 0.0, fdg[13] = {}, fdl[13] = {}, fdh[13] = {};
    double *f3[2][19] = {};  // per buffer: ro rou rov row u v w cxx cxy cyy cxz cyz czz psi(6); node (i, iz) at i*nz + iz
    double *reg3[10] = {}, *eacc3[10] = {}, *rhs3[10] = {};
    double *g3 = nullptr, *tmp3 = nullptr, *partials3 = nullptr;
    // boundary nodes in 3-D: the layer's Laplacian weights and sums with each boundary node's
    // replaced by its tangential second-derivative weights (the conformation Laplacian there),
    // and u_inflow_local of every node-layer
    double *wl3 = nullptr, *lsum3 = nullptr, *uin3 = nullptr;
    double *alpha3 = nullptr;  // the last step's error of every node-layer (alpha_out)
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    int graph_mode[2] = {-1, -1};

    // ---- adjoint (step.cu) ----
    long long *rptr = nullptr;                 // reverse links of each node (npfb + 1)
    int *rslot = nullptr, *rnode = nullptr;    // their SELL slots and owning nodes
    unsigned char *rcode = nullptr;            // reflection code | small-link flag << 2
    // the reverse lists as link streams: sliced ELL over the same slices and tiles of nodes
    // as the forward stream; per link the position of its owning node in the tile's reverse
    // halo | reflection code << 14, and the owner's weights.  Two orders: the small links
    // (stage stencils, wx wy wl; bank-aware for 16-byte loads) and all links (filter, wh;
    // for 8-byte loads)
    long long *rv_sptr = nullptr;
    int *rv_sw = nullptr, *rv_sws = nullptr;   // slice widths: all links, small links
    uint16_t *rv_loc_s = nullptr, *rv_loc_f = nullptr;
    int *rv_hptr = nullptr, *rv_halo = nullptr;
    int rv_hmax = 0;
    double *rv_wx = nullptr, *rv_wy = nullptr, *rv_wl = nullptr, *rv_wh = nullptr;
    double *rv_tvol = nullptr;                 // the filter's transpose applied to the volumes
    double *adj_gp[2] = {};                    // g_bar of a stage as 9 arrays of pairs (ping-pong)
    double *adj_sb[6] = {}, *adj_sbar[6] = {}, *adj_ua[7] = {};
    double *adj_tacc = nullptr, *adj_rpart = nullptr, *adj_acc = nullptr, *adj_cp = nullptr;
    double *adj_g = nullptr;                   // stencil sums of the segment's stages (18 arrays each)
    std::vector<Fields> adj_store;             // stage inputs of one checkpoint segment
    int adj_ckpt = 0, adj_nseg = 0;
    bool adj_ready = false;
    int *adj_segd = nullptr;                   // the segment a captured record reads its checkpoint from
    cudaGraphExec_t adj_rec_graph = nullptr;   // record of a full segment (checkpoint *adj_segd)
    cudaGraphExec_t adj_rev_graph = nullptr;   // reverse sweep of a full segment
    double adj_graph_dt = 0.0;                 // dt and checkpoint store the two graphs were captured with
    const double *adj_graph_cp = nullptr;

    std::vector<void *> allocs;
};

// error helpers
int set_err(Handle *H, int code, const char *fmt, ...);
#define SUNSET_CUDA(H, call)                                                                    \
    do {                                                                                        \
        cudaError_t e_ = (call);                                                                \
        if (e_ != cudaSuccess)                                                                  \
            return ::sunset::set_err((H), SUNSET_ERR_CUDA, "%s failed: %s (%s:%d)", #call,      \
                                     cudaGetErrorString(e_), __FILE__, __LINE__);               \
    } while (0)

template <typename T>
int dalloc(Handle *H, T **p, size_t n) {
    void *q = nullptr;
    cudaError_t e = cudaMalloc(&q, (n ? n : 1) * sizeof(T));
    if (e != cudaSuccess) return set_err(H, SUNSET_ERR_NOMEM, "cudaMalloc(%zu) failed: %s", n * sizeof(T), cudaGetErrorString(e));
    H->allocs.push_back(q);
    *p = static_cast<T *>(q);
    return 0;
}
void dfree(Handle *H, void *p);

// stage entry points implemented in the .cu files
int build_domain_device(Handle *H, const std::vector<double> &x, const std::vector<double> &y,
                        const std::vector<double> &h, const std::vector<double> &hs,
                        const std::vector<double> &s, const std::vector<int> &type);
int find_neighbours_device(Handle *H);
int build_halos(Handle *H);
int adapt_stencils_device(Handle *H);  // labf.F90:1079-1721: new h, h_small per node
int labf_weights_device(Handle *H);
int conditioning_check(Handle *H);
int boundary_prune_links(Handle *H);
int boundary_weights_device(Handle *H);
int upload_boundary(Handle *H, const std::vector<double> &nx, const std::vector<double> &ny,
                    const std::vector<int> &fdpar_ref, const std::vector<int> &blist_ref,
                    const std::vector<int> &type);
int labf_sums_device(Handle *H);
int filter_coefficients_device(Handle *H);
int make_stream_links(Handle *H);
// Bank-aware order of one slice's links (stream.cu): lane r's entries small[r] go to slots
// [0, c_s[r]) and large[r] to [c_s[r], c[r]); in each slot the lanes of every group of
// `group` lanes (16: 8-byte shared-memory loads; 8: 16-byte loads) take entries whose local
// positions pos[e] differ mod `group` wherever a matching allows.  chosen[k * 32 + lane]:
// the entry in slot k (-1: padding), for k < width.  The lists are left as they are.
void deal_slice_by_bank(int group, const uint16_t *pos, std::vector<int> *small, std::vector<int> *large,
                        const int *c_s, const int *c, int width, int *chosen);

int state_alloc(Handle *H);
int state_set_device(Handle *H, const double *ro, const double *u, const double *v, const double *cxx,
                     const double *cxy, const double *cyy, const double *czz);  // internal order, device
int state_set_conservative_device(Handle *H, const double *const *f7);  // internal order, device
// 3-D (step3d.cu)
int layers_set(Handle *H, double Lz);
int state3_set(Handle *H, const double *const *fields10);
int state3_get(Handle *H, double *out19);
int rhs3_calc(Handle *H, double *out10);
int tstep3(Handle *H);
// ev (optional, 8 per step): recorded before and after each stage's derivative gather
int step3_run(Handle *H, double dt, int nsteps, int mode, cudaEvent_t *ev = nullptr);
// mean k3_derivs launch time (ms) over reps fixed-dt steps, and its algorithmic bytes
int time3_derivs(Handle *H, int reps, double *ms, double *bytes);
int ke_mass3(Handle *H, double *ke, double *mass);
int dump3_columns(Handle *H, double *out13);
int state3_column_to_host(Handle *H, const double *dev, double *host);
size_t checkpoint3_bytes(const Handle *H);
int checkpoint3_save(Handle *H, void *buf);
int checkpoint3_load(Handle *H, const void *buf, size_t bytes);
int state3_alloc(Handle *H);
int run_host3(Handle *H, const double *state_in, double dt, int nsteps, double *state_out);
int step_run(Handle *H, double dt, int nsteps, int mode);
int rhs_only(Handle *H);
int set_tstep_device(Handle *H);
int op_gradient(Handle *H, const double *phi, double *gx, double *gy);
int op_laplacian(Handle *H, const double *phi, double *lap);
int op_filter(Handle *H, const double *phi, double *out, int term_only);
int reduce_ke_mass(Handle *H, double *ke, double *mass);
// Field dumps and checkpoints (step.cu)
int dump_columns(Handle *H, double *out);  // 10 x npfb, internal order, on the device
size_t checkpoint_bytes(const Handle *H);
int checkpoint_save(Handle *H, void *buf);
int checkpoint_load(Handle *H, const void *buf, size_t bytes);
int time_stage_kernel(Handle *H, int reps, double *ms, double *bytes);
int adjoint_run(Handle *H, double dt, int nsteps, int ckpt, double *J, double *dtheta, double *dU0);
int adjoint_apply_D(Handle *H, int which, const double *gbar, double *out);

}  // namespace sunset

// C-ABI handle
struct SunsetHandle {
    sunset::Handle H;
};
