// abi.cu -- the extern "C" entry points of include/sunset_gpu.h: argument checks, the host
// part of build_domain (IPART rows -> nodes + FD rows, setup_domain.F90:177-202), the
// reference-order <-> Morton-order permutations, and the calls into the device stages.
#include <stdarg.h>
#include <stdio.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "internal.cuh"

namespace sunset {

int set_err(Handle *H, int code, const char *fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    H->err = buf;
    return code;
}

void dfree(Handle *H, void *p) {
    if (!p) return;
    auto it = std::find(H->allocs.begin(), H->allocs.end(), p);
    if (it != H->allocs.end()) {
        cudaFree(p);
        H->allocs.erase(it);
    }
}

namespace {

__global__ void k_gather(const double *in, const int *perm, int n, double *out) {  // out[i] = in[perm[i]]
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = in[perm[i]];
}
__global__ void k_scatter(const double *in, const int *perm, int n, double *out) {  // out[perm[i]] = in[i]
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[perm[i]] = in[i];
}

// The seven evolved fields at once, between the reference-order staging block (7 x n,
// field-major) and the internal-order field arrays.
struct Fields7 {
    double *p[7];
};
__global__ void k_gather7(const double *in, const int *perm, int n, Fields7 out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int r = perm[i];
#pragma unroll
    for (int f = 0; f < 7; f++) out.p[f][i] = in[(size_t)f * n + r];
}
__global__ void k_scatter7(Fields7 in, const int *perm, int n, double *out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int r = perm[i];
#pragma unroll
    for (int f = 0; f < 7; f++) out[(size_t)f * n + r] = in.p[f][i];
}

double hovs_for(int forder) {  // common_parameter.F90:44-56
    if (forder == 4) return 1.8;
    if (forder == 6) return 2.4;
    if (forder == 10) return 3.1;
    return 2.7;
}
double hovs_bound_for(int forder) { return forder == 4 ? 2.1 : 2.4; }

int set_device(Handle *H) {
    SUNSET_CUDA(H, cudaSetDevice(H->device));
    return 0;
}

// Copies a reference-order array (host or device) into internal order on the device.
int to_internal(Handle *H, const double *src, int flags, double *dst) {
    const int n = H->npfb;
    double *ref = H->tmpd + 3 * (size_t)n;
    if (flags == SUNSET_PTR_DEVICE) {
        SUNSET_CUDA(H, cudaMemcpyAsync(ref, src, n * sizeof(double), cudaMemcpyDeviceToDevice, H->stream));
    } else {
        SUNSET_CUDA(H, cudaMemcpyAsync(ref, src, n * sizeof(double), cudaMemcpyHostToDevice, H->stream));
    }
    k_gather<<<(n + 255) / 256, 256, 0, H->stream>>>(ref, H->perm, n, dst);
    SUNSET_CUDA(H, cudaGetLastError());
    return 0;
}
int to_reference(Handle *H, const double *src, int flags, double *dst) {
    const int n = H->npfb;
    double *ref = H->tmpd + 3 * (size_t)n;
    k_scatter<<<(n + 255) / 256, 256, 0, H->stream>>>(src, H->perm, n, ref);
    SUNSET_CUDA(H, cudaGetLastError());
    if (flags == SUNSET_PTR_DEVICE) {
        SUNSET_CUDA(H, cudaMemcpyAsync(dst, ref, n * sizeof(double), cudaMemcpyDeviceToDevice, H->stream));
    } else {
        SUNSET_CUDA(H, cudaMemcpyAsync(dst, ref, n * sizeof(double), cudaMemcpyDeviceToHost, H->stream));
        SUNSET_CUDA(H, cudaStreamSynchronize(H->stream));
    }
    return 0;
}

int need(Handle *H, bool ok, const char *what) {
    if (!ok) return set_err(H, SUNSET_ERR_ARG, "call order: %s first", what);
    return 0;
}

// The device error word of the step kernels: 0 = none, 1 = the time-step error norm of a
// step was NaN or infinite (k_finalize, k3_finalize), 2 = a wait of the mixed stage kernel
// on its link stream gave up (k_stage).  No other value is ever written.
int check_err_flag(Handle *H) {
    int e = 0;
    SUNSET_CUDA(H, cudaMemcpyAsync(&e, &H->dsc->err, sizeof(int), cudaMemcpyDeviceToHost, H->stream));
    SUNSET_CUDA(H, cudaStreamSynchronize(H->stream));
    if (e == 1) return set_err(H, SUNSET_ERR_NONFINITE, "non-finite time-step error norm");
    if (e == 2) return set_err(H, SUNSET_ERR_CUDA, "a bounded wait on the stage kernel's link stream gave up");
    if (e) return set_err(H, SUNSET_ERR_CUDA, "unknown device error word %d", e);
    return 0;
}

// Two CUDA events destroyed with the object, so every return path releases them.
struct EventPair {
    cudaEvent_t e[2] = {nullptr, nullptr};
    ~EventPair() {
        for (cudaEvent_t x : e)
            if (x) cudaEventDestroy(x);
    }
};

}  // namespace
}  // namespace sunset

using namespace sunset;

extern "C" {

int sunset_version(void) { return 1; }

int sunset_kernel_binary_version(int device) {
    int prev = -1;
    if (cudaGetDevice(&prev) != cudaSuccess) return SUNSET_ERR_CUDA;
    if (device != prev && cudaSetDevice(device) != cudaSuccess) return SUNSET_ERR_CUDA;
    cudaFuncAttributes fa{};
    const cudaError_t e = cudaFuncGetAttributes(&fa, (const void *)k_gather);
    if (device != prev) cudaSetDevice(prev);
    return e == cudaSuccess ? fa.binaryVersion : SUNSET_ERR_CUDA;
}

int sunset_create(const SunsetConfig *cfg, SunsetHandle **out) {
    if (!cfg || !out) return SUNSET_ERR_ARG;
    SunsetHandle *sh = new SunsetHandle();
    Handle *H = &sh->H;
    H->cfg = *cfg;
    if (H->cfg.L_char == 0.0) H->cfg.L_char = 1.0;
    if (H->cfg.U_char == 0.0) H->cfg.U_char = 1.0;
    H->device = cfg->device;
    *out = sh;
    const SunsetConfig &c = H->cfg;
    if (!(c.morder == 4 || c.morder == 6 || c.morder == 8 || c.morder == 10) || c.forder != c.morder)
        return set_err(H, SUNSET_ERR_SCOPE, "orders must be equal and one of 4, 6, 8, 10 (got %d, %d)", c.morder, c.forder);
    if (c.form < 0 || c.form > 3) return set_err(H, SUNSET_ERR_ARG, "unknown form %d", c.form);
    if (c.precision != SUNSET_FP64 && c.precision != SUNSET_MIXED) return set_err(H, SUNSET_ERR_ARG, "bad precision");
    if (c.Re <= 0 || c.Ma <= 0 || (c.form != SUNSET_FORM_NEWT && c.Wi <= 0))
        return set_err(H, SUNSET_ERR_ARG, "Re, Ma and Wi must be positive");
    if (c.form == SUNSET_FORM_NEWT) H->cfg.fenep = 0;  // no polymer
    if (H->cfg.fenep && !(c.fenep_l2 > 3.0))
        return set_err(H, SUNSET_ERR_ARG, "FENE-P needs L^2 > 3 (got %g)", c.fenep_l2);
    if (c.inflow_type < 0 || c.inflow_type > 2) return set_err(H, SUNSET_ERR_ARG, "inflow_type must be 0, 1 or 2");
    if (c.inflow_velocity_control == 1 && !(c.ramp_time > 0.0))
        return set_err(H, SUNSET_ERR_ARG, "inflow velocity control needs ramp_time > 0");
    if (c.grav[2] != 0.0) return set_err(H, SUNSET_ERR_SCOPE, "grav(3) must be zero on this 2-D path");
    if (int rc = set_device(H)) return rc;
    SUNSET_CUDA(H, cudaStreamCreateWithFlags(&H->stream, cudaStreamNonBlocking));
    return 0;
}

void sunset_destroy(SunsetHandle *sh) {
    if (!sh) return;
    Handle *H = &sh->H;
    cudaSetDevice(H->device);
    if (H->stream) cudaStreamSynchronize(H->stream);
    for (int b = 0; b < 2; b++)
        if (H->graph[b]) cudaGraphExecDestroy(H->graph[b]);
    for (cudaGraphExec_t g : {H->adj_rec_graph, H->adj_rev_graph})
        if (g) cudaGraphExecDestroy(g);
    for (void *p : H->allocs) cudaFree(p);
    H->allocs.clear();
    if (H->stream) cudaStreamDestroy(H->stream);
    delete sh;
}

const char *sunset_last_error(const SunsetHandle *sh) { return sh ? sh->H.err.c_str() : "null handle"; }

int sunset_build_domain(SunsetHandle *sh, int nrows, const int *gi, const double *x, const double *y,
                        const int *node_type, const double *nx, const double *ny, const double *s, double xmin,
                        double xmax, double ymin, double ymax, const int *bcond, double smax) {
    if (!sh) return SUNSET_ERR_ARG;
    Handle *H = &sh->H;
    if (H->domain_ok) return set_err(H, SUNSET_ERR_ARG, "domain already built; create a new handle");
    if (nrows <= 0 || !x || !y || !node_type || !s || !bcond) return set_err(H, SUNSET_ERR_ARG, "bad arguments");
    if (!(xmax > xmin && ymax > ymin)) return set_err(H, SUNSET_ERR_ARG, "empty domain");
    if (!(smax > 0.0) || !std::isfinite(smax)) return set_err(H, SUNSET_ERR_ARG, "smax must be positive");
    for (int c = 0; c < 4; c++)
        if (bcond[c] < 0 || bcond[c] > 3) return set_err(H, SUNSET_ERR_ARG, "bcond[%d] = %d is not 0..3", c, bcond[c]);
    // the rows of a node file (setup_domain.F90:177-199) as the reference reads them: a row the
    // reader would misplace or a spacing the cell list cannot hold is an error here, where the
    // reference reads on into undefined behaviour.  Positions may lie a little outside the box
    // (the reference's own IPART does), but not outside the tripled domain its search cells
    // cover (neighbours.F90:84-89).
    const double lx = xmax - xmin, ly = ymax - ymin;
    for (int r = 0; r < nrows; r++) {
        const int t = node_type[r];
        if (!(t == 999 || t == 998 || (t >= 0 && t <= 2)))
            return set_err(H, SUNSET_ERR_ARG, "row %d: node type %d is not 0, 1, 2, 998 or 999", r + 1, t);
        if (!std::isfinite(x[r]) || !std::isfinite(y[r]) || x[r] < xmin - lx || x[r] > xmax + lx || y[r] < ymin - ly ||
            y[r] > ymax + ly)
            return set_err(H, SUNSET_ERR_ARG, "row %d: position (%g, %g) outside the search cells", r + 1, x[r], y[r]);
        if (!(s[r] > 0.0) || !(s[r] <= smax))
            return set_err(H, SUNSET_ERR_ARG, "row %d: spacing %g outside (0, smax = %g]", r + 1, s[r], smax);
        if (t <= 2) {
            const double rnx = nx ? nx[r] : 0.0, rny = ny ? ny[r] : 0.0;
            if (!(std::fabs(rnx * rnx + rny * rny - 1.0) < 1e-6))
                return set_err(H, SUNSET_ERR_ARG, "row %d: boundary node without a unit normal", r + 1);
        }
    }
    if (int rc = set_device(H)) return rc;
    const double hovs = hovs_for(H->cfg.forder), hovs_bound = hovs_bound_for(H->cfg.forder);
    const double hos = H->cfg.h_over_s;
    std::vector<double> vx, vy, vh, vs, vnx, vny;
    std::vector<int> vt, vfd, vb;
    int nb = 0;
    for (int r = 0; r < nrows; r++) {  // setup_domain.F90:177-199
        int t = node_type[r];
        const double rnx = nx ? nx[r] : 0.0, rny = ny ? ny[r] : 0.0;
        H->h_gi.push_back(gi ? gi[r] : r + 1);
        vx.push_back(x[r]);
        vy.push_back(y[r]);
        vs.push_back(s[r]);
        vt.push_back(t);
        vh.push_back(s[r] * hovs);
        vnx.push_back(rnx);
        vny.push_back(rny);
        vfd.push_back(-1);
        if (t >= 0 && t <= 2) {
            nb++;
            const int k = (int)vx.size() - 1;
            vb.push_back(k);
            vh.back() = s[r] * hovs_bound;
            for (int j = 1; j <= 4; j++) {
                vx.push_back(x[r] + (rnx * (double)j) * s[r]);
                vy.push_back(y[r] + (rny * (double)j) * s[r]);
                vs.push_back(s[r]);
                vt.push_back(-j);
                vh.push_back(s[r] * hovs_bound);
                vnx.push_back(rnx);
                vny.push_back(rny);
                vfd.push_back(k);
                H->h_gi.push_back(H->h_gi[k] + j);  // setup_domain.F90:190
            }
        }
    }
    const int n = (int)vx.size();
    if (n >= (1 << 30)) return set_err(H, SUNSET_ERR_SCOPE, "too many nodes");
    if (hos > 0)
        for (int i = 0; i < n; i++) vh[i] = hos * vs[i];
    std::vector<double> vhs = vh;  // h_small = h
    H->npfb = n;
    H->nb = nb;
    H->nrows = nrows;
    H->xmin = xmin; H->xmax = xmax; H->ymin = ymin; H->ymax = ymax;
    for (int c = 0; c < 4; c++) H->bc[c] = bcond[c];
    if ((bcond[0] == 1) != (bcond[1] == 1) || (bcond[2] == 1) != (bcond[3] == 1))
        return set_err(H, SUNSET_ERR_ARG, "periodic boundary conditions incorrectly specified with bcond");
    H->smax = smax;
    H->h0 = (hos > 0 ? hos : hovs) * smax;  // setup_domain.F90:105
    H->h2 = H->h0 * H->h0;
    H->h3 = H->h2 * H->h0;
    H->hmax = *std::max_element(vh.begin(), vh.end());
    int rc = build_domain_device(H, vx, vy, vh, vhs, vs, vt);
    if (rc) return rc;
    rc = upload_boundary(H, vnx, vny, vfd, vb, vt);
    if (rc) return rc;
    H->domain_ok = true;
    return 0;
}

int sunset_get_sizes(SunsetHandle *sh, int *np, int *npfb, int *nb, int *nplink) {
    if (!sh) return SUNSET_ERR_ARG;
    Handle *H = &sh->H;
    if (np) *np = H->np;
    if (npfb) *npfb = H->npfb;
    if (nb) *nb = H->nb;
    if (nplink) *nplink = H->nplink;
    return 0;
}

int sunset_find_neighbours(SunsetHandle *sh) {
    if (!sh) return SUNSET_ERR_ARG;
    Handle *H = &sh->H;
    if (int rc = need(H, H->domain_ok, "sunset_build_domain")) return rc;
    if (H->nbr_ok) return set_err(H, SUNSET_ERR_ARG, "neighbours already built");
    if (int rc = set_device(H)) return rc;
    int rc = find_neighbours_device(H);
    if (rc) return rc;
    rc = build_halos(H);
    if (rc) return rc;
    H->nbr_ok = true;
    return 0;
}

int sunset_adapt_stencils(SunsetHandle *sh) {
    if (!sh) return SUNSET_ERR_ARG;
    Handle *H = &sh->H;
    if (int rc = need(H, H->nbr_ok, "sunset_find_neighbours")) return rc;
    if (H->w_ok) return set_err(H, SUNSET_ERR_ARG, "adapt the stencils before building the weights");
    if (int rc = set_device(H)) return rc;
    if (int rc = adapt_stencils_device(H)) return rc;
    // the neighbour lists again with the new lengths (sunset.F90:43-51)
    void **lists[] = {(void **)&H->slice_ptr, (void **)&H->slice_w, (void **)&H->slice_ws, (void **)&H->lpt,
                      (void **)&H->lidx, (void **)&H->halo_ptr, (void **)&H->halo, (void **)&H->lloc};
    for (void **p : lists) {
        dfree(H, *p);
        *p = nullptr;
    }
    H->nbr_ok = false;
    int rc = find_neighbours_device(H);
    if (rc) return rc;
    rc = build_halos(H);
    if (rc) return rc;
    H->nbr_ok = true;
    return 0;
}

int sunset_get_lengths(SunsetHandle *sh, double *h, double *h_small) {
    if (!sh || !h || !h_small) return SUNSET_ERR_ARG;
    Handle *H = &sh->H;
    if (int rc = need(H, H->domain_ok, "sunset_build_domain")) return rc;
    if (int rc = set_device(H)) return rc;
    const int n = H->npfb;
    std::vector<double> hv(n), hsv(n);
    SUNSET_CUDA(H, cudaMemcpy(hv.data(), H->h, n * sizeof(double), cudaMemcpyDeviceToHost));
    SUNSET_CUDA(H, cudaMemcpy(hsv.data(), H->hs, n * sizeof(double), cudaMemcpyDeviceToHost));
    for (int i = 0; i < n; i++) {  // internal node i is reference node perm[i]
        h[H->h_perm[i]] = hv[i];
        h_small[H->h_perm[i]] = hsv[i];
    }
    return 0;
}

int sunset_calc_labf_weights(SunsetHandle *sh) {
    if (!sh) return SUNSET_ERR_ARG;
    Handle *H = &sh->H;
    if (int rc = need(H, H->nbr_ok, "sunset_find_neighbours")) return rc;
    if (int rc = set_device(H)) return rc;
    int rc = labf_weights_device(H);
    if (rc) return rc;
    H->w_ok = true;
    H->bw_ok = H->nb == 0;
    H->sums_ok = H->fc_ok = false;
    return 0;
}

int sunset_get_conditioning(SunsetHandle *sh, double *cond_deriv, double *cond_filter, double *worst, int *n_ill) {
    if (!sh) return SUNSET_ERR_ARG;
    Handle *H = &sh->H;
    if (int rc = need(H, H->cond_ok, "sunset_calc_labf_weights")) return rc;
    if (int rc = set_device(H)) return rc;
    const int n = H->npfb;
    std::vector<double> t(n);
    double *dst[2] = {cond_deriv, cond_filter};
    const double *src[2] = {H->cond_d, H->cond_f};
    for (int a = 0; a < 2; a++) {
        if (!dst[a]) continue;
        SUNSET_CUDA(H, cudaMemcpy(t.data(), src[a], n * sizeof(double), cudaMemcpyDeviceToHost));
        for (int i = 0; i < n; i++) dst[a][H->h_perm[i]] = t[i];  // internal node i is reference node perm[i]
    }
    if (worst) *worst = H->cond_worst;
    if (n_ill) *n_ill = H->cond_nill;
    return 0;
}

int sunset_calc_boundary_weights(SunsetHandle *sh) {
    if (!sh) return SUNSET_ERR_ARG;
    Handle *H = &sh->H;
    if (H->nb == 0) return 0;
    if (int rc = need(H, H->w_ok && !H->bw_ok, "sunset_calc_labf_weights")) return rc;
    if (int rc = set_device(H)) return rc;
    int rc = boundary_prune_links(H);
    if (rc) return rc;
    rc = boundary_weights_device(H);
    if (rc) return rc;
    H->bw_ok = true;
    return 0;
}

int sunset_calc_labf_sums(SunsetHandle *sh) {
    if (!sh) return SUNSET_ERR_ARG;
    Handle *H = &sh->H;
    if (int rc = need(H, H->w_ok && H->bw_ok && !H->sums_ok, H->w_ok ? "sunset_calc_boundary_weights" : "sunset_calc_labf_weights")) return rc;
    if (int rc = set_device(H)) return rc;
    int rc = labf_sums_device(H);
    if (rc) return rc;
    H->sums_ok = true;
    return 0;
}

int sunset_filter_coefficients(SunsetHandle *sh) {
    if (!sh) return SUNSET_ERR_ARG;
    Handle *H = &sh->H;
    if (int rc = need(H, H->sums_ok && !H->fc_ok, "sunset_calc_labf_sums")) return rc;
    if (int rc = set_device(H)) return rc;
    int rc = filter_coefficients_device(H);
    if (rc) return rc;
    rc = state_alloc(H);
    if (rc) return rc;
    rc = make_stream_links(H);
    if (rc) return rc;
    H->fc_ok = true;
    return 0;
}

int sunset_get_neighbours(SunsetHandle *sh, int *ij_count, int *ij_count_small, int *ij_link) {
    if (!sh) return SUNSET_ERR_ARG;
    Handle *H = &sh->H;
    if (int rc = need(H, H->nbr_ok, "sunset_find_neighbours")) return rc;
    if (int rc = set_device(H)) return rc;
    const int n = H->npfb, nplink = H->nplink;
    std::vector<int> cnt(n), cs(n), lpt(H->nlinks_sell);
    std::vector<long long> sptr(H->nslices + 1);
    SUNSET_CUDA(H, cudaMemcpy(cnt.data(), H->cnt, n * sizeof(int), cudaMemcpyDeviceToHost));
    SUNSET_CUDA(H, cudaMemcpy(cs.data(), H->cnt_small, n * sizeof(int), cudaMemcpyDeviceToHost));
    SUNSET_CUDA(H, cudaMemcpy(lpt.data(), H->lpt, lpt.size() * sizeof(int), cudaMemcpyDeviceToHost));
    SUNSET_CUDA(H, cudaMemcpy(sptr.data(), H->slice_ptr, sptr.size() * sizeof(long long), cudaMemcpyDeviceToHost));
    for (int r = 0; r < n; r++) {
        int i = H->h_iperm[r];
        if (ij_count) ij_count[r] = cnt[i];
        if (ij_count_small) ij_count_small[r] = cs[i];
        if (ij_link) {
            for (int k = 0; k < nplink; k++) {
                int v = 0;
                if (k < cnt[i]) {
                    int p = lpt[sell_at(sptr[i >> 5], k, i & 31)];
                    v = (p < n ? H->h_perm[p] : p) + 1;
                }
                ij_link[(size_t)r * nplink + k] = v;
            }
        }
    }
    return 0;
}

int sunset_get_weights(SunsetHandle *sh, double *w_grad, double *w_lap, double *w_hyp, double *w_grad_sum,
                       double *w_lap_sum, double *w_hyp_sum, double *vol) {
    if (!sh) return SUNSET_ERR_ARG;
    Handle *H = &sh->H;
    if (int rc = need(H, H->w_ok, "sunset_calc_labf_weights")) return rc;
    if (int rc = set_device(H)) return rc;
    const int n = H->npfb, nplink = H->nplink;
    const size_t L = H->nlinks_sell;
    std::vector<int> cnt(n);
    std::vector<long long> sptr(H->nslices + 1);
    SUNSET_CUDA(H, cudaMemcpy(cnt.data(), H->cnt, n * sizeof(int), cudaMemcpyDeviceToHost));
    SUNSET_CUDA(H, cudaMemcpy(sptr.data(), H->slice_ptr, sptr.size() * sizeof(long long), cudaMemcpyDeviceToHost));
    auto scatter_links = [&](const double *dsrc, double *dst, int stride, int comp) -> int {
        std::vector<double> tmp(L);
        SUNSET_CUDA(H, cudaMemcpy(tmp.data(), dsrc, L * sizeof(double), cudaMemcpyDeviceToHost));
        for (int r = 0; r < n; r++) {
            int i = H->h_iperm[r];
            for (int k = 0; k < nplink; k++) {
                double v = 0.0;
                if (k < cnt[i]) v = tmp[sell_at(sptr[i >> 5], k, i & 31)];
                dst[((size_t)r * nplink + k) * stride + comp] = v;
            }
        }
        return 0;
    };
    auto scatter_nodes = [&](const double *dsrc, double *dst, int stride, int comp) -> int {
        std::vector<double> tmp(n);
        SUNSET_CUDA(H, cudaMemcpy(tmp.data(), dsrc, n * sizeof(double), cudaMemcpyDeviceToHost));
        for (int r = 0; r < n; r++) dst[(size_t)r * stride + comp] = tmp[H->h_iperm[r]];
        return 0;
    };
    int rc = 0;
    if (w_grad && !rc) rc = scatter_links(H->wx, w_grad, 2, 0);
    if (w_grad && !rc) rc = scatter_links(H->wy, w_grad, 2, 1);
    if (w_lap && !rc) rc = scatter_links(H->wl, w_lap, 1, 0);
    if (w_hyp && !rc) rc = scatter_links(H->wh, w_hyp, 1, 0);
    if (H->sums_ok) {
        if (w_grad_sum && !rc) rc = scatter_nodes(H->gsx, w_grad_sum, 2, 0);
        if (w_grad_sum && !rc) rc = scatter_nodes(H->gsy, w_grad_sum, 2, 1);
        if (w_lap_sum && !rc) rc = scatter_nodes(H->lsum, w_lap_sum, 1, 0);
        if (w_hyp_sum && !rc) rc = scatter_nodes(H->hsum, w_hyp_sum, 1, 0);
        if (vol && !rc) rc = scatter_nodes(H->vol, vol, 1, 0);
    }
    return rc;
}

static int op_common(SunsetHandle *sh, Handle **HH) {
    if (!sh) return SUNSET_ERR_ARG;
    Handle *H = &sh->H;
    *HH = H;
    if (int rc = need(H, H->fc_ok, "sunset_filter_coefficients")) return rc;
    return set_device(H);
}

int sunset_calc_gradient(SunsetHandle *sh, const double *phi, double *grad, int flags) {
    Handle *H;
    if (int rc = op_common(sh, &H)) return rc;
    if (!phi || !grad) return set_err(H, SUNSET_ERR_ARG, "null array");
    const int n = H->npfb;
    double *p = H->tmpd, *gx = H->tmpd + n, *gy = H->tmpd + 2 * (size_t)n;
    if (int rc = to_internal(H, phi, flags, p)) return rc;
    if (int rc = op_gradient(H, p, gx, gy)) return rc;
    std::vector<double> hx(n), hy(n);
    double *ref = H->tmpd + 3 * (size_t)n;
    for (int c = 0; c < 2; c++) {
        const double *src = c == 0 ? gx : gy;
        std::vector<double> &dst = c == 0 ? hx : hy;
        if (int rc = to_reference(H, src, SUNSET_PTR_DEVICE, ref)) return rc;
        SUNSET_CUDA(H, cudaMemcpyAsync(dst.data(), ref, n * sizeof(double), cudaMemcpyDeviceToHost, H->stream));
        SUNSET_CUDA(H, cudaStreamSynchronize(H->stream));
    }
    if (flags == SUNSET_PTR_DEVICE) {
        std::vector<double> inter(2 * (size_t)n);
        for (int r = 0; r < n; r++) { inter[2 * r] = hx[r]; inter[2 * r + 1] = hy[r]; }
        SUNSET_CUDA(H, cudaMemcpy(grad, inter.data(), inter.size() * sizeof(double), cudaMemcpyHostToDevice));
    } else {
        for (int r = 0; r < n; r++) { grad[2 * r] = hx[r]; grad[2 * r + 1] = hy[r]; }
    }
    return 0;
}

int sunset_calc_laplacian(SunsetHandle *sh, const double *phi, double *lap, int flags) {
    Handle *H;
    if (int rc = op_common(sh, &H)) return rc;
    if (!phi || !lap) return set_err(H, SUNSET_ERR_ARG, "null array");
    const int n = H->npfb;
    double *p = H->tmpd, *o = H->tmpd + n;
    if (int rc = to_internal(H, phi, flags, p)) return rc;
    if (int rc = op_laplacian(H, p, o)) return rc;
    return to_reference(H, o, flags, lap);
}

int sunset_calc_filtered_var(SunsetHandle *sh, const double *phi, double *out, int flags) {
    Handle *H;
    if (int rc = op_common(sh, &H)) return rc;
    if (!phi || !out) return set_err(H, SUNSET_ERR_ARG, "null array");
    const int n = H->npfb;
    double *p = H->tmpd, *o = H->tmpd + n;
    if (int rc = to_internal(H, phi, flags, p)) return rc;
    if (int rc = op_filter(H, p, o, 0)) return rc;
    return to_reference(H, o, flags, out);
}

int sunset_calc_filter_term(SunsetHandle *sh, const double *phi, double *out, int flags) {
    Handle *H;
    if (int rc = op_common(sh, &H)) return rc;
    if (!phi || !out) return set_err(H, SUNSET_ERR_ARG, "null array");
    const int n = H->npfb;
    double *p = H->tmpd, *o = H->tmpd + n;
    if (int rc = to_internal(H, phi, flags, p)) return rc;
    if (int rc = op_filter(H, p, o, 1)) return rc;
    return to_reference(H, o, flags, out);
}

int sunset_set_state(SunsetHandle *sh, const double *ro, const double *u, const double *v, const double *cxx,
                     const double *cxy, const double *cyy, const double *czz) {
    Handle *H;
    if (int rc = op_common(sh, &H)) return rc;
    if (!ro || !u || !v || !cxx || !cxy || !cyy) return set_err(H, SUNSET_ERR_ARG, "null array");
    if (H->nz > 0) return set_err(H, SUNSET_ERR_ARG, "a 3-D handle: use sunset_set_state_3d");
    const int n = H->npfb;
    // stage the seven inputs in internal order inside the (not yet used) second buffer and rhs
    double *d[7] = {H->rhs[0], H->rhs[1], H->rhs[2], H->rhs[3], H->rhs[4], H->rhs[5], H->rhs[6]};
    const double *src[7] = {ro, u, v, cxx, cxy, cyy, czz};
    std::vector<double> ones;
    if (!czz) {
        ones.assign(n, 1.0);
        src[6] = ones.data();
    }
    for (int f = 0; f < 7; f++)
        if (int rc = to_internal(H, src[f], SUNSET_PTR_HOST, d[f])) return rc;
    int rc = state_set_device(H, d[0], d[1], d[2], d[3], d[4], d[5], d[6]);
    if (rc) return rc;
    SUNSET_CUDA(H, cudaStreamSynchronize(H->stream));
    H->state_ok = true;
    return 0;
}

int sunset_get_state(SunsetHandle *sh, double *out) {
    Handle *H;
    if (int rc = op_common(sh, &H)) return rc;
    if (int rc = need(H, H->state_ok, "sunset_set_state")) return rc;
    const int n = H->npfb;
    const Fields &F = H->buf[H->cur];
    const double *src[13] = {F.ro, F.rou, F.rov, F.u, F.v, F.q[0], F.q[1], F.q[2], F.q[3], F.c[0], F.c[1], F.c[2], F.c[3]};
    for (int f = 0; f < 13; f++) {
        if (H->cfg.form == SUNSET_FORM_DI && f >= 5 && f <= 8) {
            for (int r = 0; r < n; r++) out[(size_t)f * n + r] = 0.0;
            continue;
        }
        if (int rc = to_reference(H, src[f], SUNSET_PTR_HOST, out + (size_t)f * n)) return rc;
    }
    return 0;
}

int sunset_set_layers(SunsetHandle *sh, double L_domain_z) {
    if (!sh) return SUNSET_ERR_ARG;
    Handle *H = &sh->H;
    if (int rc = need(H, H->domain_ok, "sunset_build_domain")) return rc;
    if (H->state_ok || H->state3_ok || H->nz > 0) return set_err(H, SUNSET_ERR_ARG, "set the layers once, before the state");
    if (int rc = set_device(H)) return rc;
    return layers_set(H, L_domain_z);
}

int sunset_get_layers(SunsetHandle *sh, int *nz, double *dz) {
    if (!sh) return SUNSET_ERR_ARG;
    Handle *H = &sh->H;
    if (nz) *nz = H->nz;
    if (dz) *dz = H->dz;
    return 0;
}

int sunset_set_state_3d(SunsetHandle *sh, const double *ro, const double *u, const double *v, const double *w,
                        const double *cxx, const double *cxy, const double *cyy, const double *cxz, const double *cyz,
                        const double *czz) {
    Handle *H;
    if (int rc = op_common(sh, &H)) return rc;
    if (H->nz == 0) return set_err(H, SUNSET_ERR_ARG, "call order: sunset_set_layers first");
    if (!ro || !u || !v || !w) return set_err(H, SUNSET_ERR_ARG, "null array");
    const bool anyc = cxx || cxy || cyy || cxz || cyz || czz, allc = cxx && cxy && cyy && cxz && cyz && czz;
    if (anyc && !allc) return set_err(H, SUNSET_ERR_ARG, "give all six c components or none");
    const double *f[10] = {ro, u, v, w, cxx, cxy, cyy, cxz, cyz, czz};
    if (int rc = state3_set(H, f)) return rc;
    SUNSET_CUDA(H, cudaStreamSynchronize(H->stream));
    H->state3_ok = true;
    return 0;
}

int sunset_get_state_3d(SunsetHandle *sh, double *out) {
    Handle *H;
    if (int rc = op_common(sh, &H)) return rc;
    if (int rc = need(H, H->state3_ok, "sunset_set_state_3d")) return rc;
    if (!out) return set_err(H, SUNSET_ERR_ARG, "null array");
    return state3_get(H, out);
}

int sunset_calc_all_rhs_3d(SunsetHandle *sh, double *out) {
    Handle *H;
    if (int rc = op_common(sh, &H)) return rc;
    if (int rc = need(H, H->state3_ok, "sunset_set_state_3d")) return rc;
    if (!out) return set_err(H, SUNSET_ERR_ARG, "null array");
    return rhs3_calc(H, out);
}

int sunset_calc_all_rhs(SunsetHandle *sh, double *out) {
    Handle *H;
    if (int rc = op_common(sh, &H)) return rc;
    if (int rc = need(H, H->state_ok, "sunset_set_state")) return rc;
    if (int rc = rhs_only(H)) return rc;
    for (int f = 0; f < 7; f++)
        if (int rc = to_reference(H, H->rhs[f], SUNSET_PTR_HOST, out + (size_t)f * H->npfb)) return rc;
    return 0;
}

int sunset_set_tstep(SunsetHandle *sh, double *dt_cfl, double *dt_parabolic) {
    Handle *H;
    if (int rc = op_common(sh, &H)) return rc;
    if (H->nz > 0) {
        if (int rc = need(H, H->state3_ok, "sunset_set_state_3d")) return rc;
        if (int rc = tstep3(H)) return rc;
    } else {
        if (int rc = need(H, H->state_ok, "sunset_set_state")) return rc;
        if (int rc = set_tstep_device(H)) return rc;
    }
    DevScalars s;
    SUNSET_CUDA(H, cudaMemcpyAsync(&s, H->dsc, sizeof(s), cudaMemcpyDeviceToHost, H->stream));
    SUNSET_CUDA(H, cudaStreamSynchronize(H->stream));
    if (dt_cfl) *dt_cfl = s.dt_cfl;
    if (dt_parabolic) *dt_parabolic = s.dt_par;
    return 0;
}

int sunset_step(SunsetHandle *sh, double dt, int nsteps, int mode) {
    Handle *H;
    if (int rc = op_common(sh, &H)) return rc;
    if (nsteps < 0 || (mode == 0 && !(dt > 0.0)) || mode < 0 || mode > 1)
        return set_err(H, SUNSET_ERR_ARG, "bad dt/nsteps/mode");
    if (H->nz > 0) {
        if (int rc = need(H, H->state3_ok, "sunset_set_state_3d")) return rc;
        if (int rc = step3_run(H, dt, nsteps, mode)) return rc;
        return check_err_flag(H);
    }
    if (int rc = need(H, H->state_ok, "sunset_set_state")) return rc;
    if (int rc = step_run(H, dt, nsteps, mode)) return rc;
    return check_err_flag(H);
}

int sunset_step_timed(SunsetHandle *sh, double dt, int nsteps, int mode, double *ms) {
    Handle *H;
    if (int rc = op_common(sh, &H)) return rc;
    if (int rc = need(H, H->nz > 0 ? H->state3_ok : H->state_ok, H->nz > 0 ? "sunset_set_state_3d" : "sunset_set_state"))
        return rc;
    if (nsteps < 0 || (mode == 0 && !(dt > 0.0)) || mode < 0 || mode > 1 || !ms)
        return set_err(H, SUNSET_ERR_ARG, "bad dt/nsteps/mode");
    EventPair ev;  // destroyed on every return path
    SUNSET_CUDA(H, cudaEventCreate(&ev.e[0]));
    SUNSET_CUDA(H, cudaEventCreate(&ev.e[1]));
    SUNSET_CUDA(H, cudaEventRecord(ev.e[0], H->stream));
    int rc = H->nz > 0 ? step3_run(H, dt, nsteps, mode) : step_run(H, dt, nsteps, mode);
    SUNSET_CUDA(H, cudaEventRecord(ev.e[1], H->stream));
    SUNSET_CUDA(H, cudaEventSynchronize(ev.e[1]));
    float t = 0.f;
    SUNSET_CUDA(H, cudaEventElapsedTime(&t, ev.e[0], ev.e[1]));
    *ms = t;
    if (rc) return rc;
    return check_err_flag(H);
}

int sunset_get_time(SunsetHandle *sh, double *time, double *dt, int *itime, double *emax) {
    Handle *H;
    if (int rc = op_common(sh, &H)) return rc;
    DevScalars s;
    SUNSET_CUDA(H, cudaMemcpyAsync(&s, H->dsc, sizeof(s), cudaMemcpyDeviceToHost, H->stream));
    SUNSET_CUDA(H, cudaStreamSynchronize(H->stream));
    if (time) *time = s.time;
    if (dt) *dt = s.dt;
    if (itime) *itime = s.itime;
    if (emax) { emax[0] = s.emax_nm1; emax[1] = s.emax_n; emax[2] = s.emax_np1; }
    return 0;
}

int sunset_set_time(SunsetHandle *sh, double time, double dt, int itime, const double *emax) {
    Handle *H;
    if (int rc = op_common(sh, &H)) return rc;
    DevScalars s;
    SUNSET_CUDA(H, cudaMemcpyAsync(&s, H->dsc, sizeof(s), cudaMemcpyDeviceToHost, H->stream));
    SUNSET_CUDA(H, cudaStreamSynchronize(H->stream));
    s.time = time; s.dt = dt; s.itime = itime;
    if (emax) { s.emax_nm1 = emax[0]; s.emax_n = emax[1]; s.emax_np1 = emax[2]; }
    SUNSET_CUDA(H, cudaMemcpyAsync(H->dsc, &s, sizeof(s), cudaMemcpyHostToDevice, H->stream));
    SUNSET_CUDA(H, cudaStreamSynchronize(H->stream));
    return 0;
}

// mass_and_energy_check (statistics.F90:305-330): over the 2-D state, or the 3-D one with
// dV = vol dz
int sunset_kinetic_energy(SunsetHandle *sh, double *ke) {
    Handle *H;
    if (int rc = op_common(sh, &H)) return rc;
    if (!ke) return set_err(H, SUNSET_ERR_ARG, "null pointer");
    if (H->nz > 0) {
        if (int rc = need(H, H->state3_ok, "sunset_set_state_3d")) return rc;
        return ke_mass3(H, ke, nullptr);
    }
    if (int rc = need(H, H->state_ok, "sunset_set_state")) return rc;
    return reduce_ke_mass(H, ke, nullptr);
}

int sunset_mass(SunsetHandle *sh, double *mass) {
    Handle *H;
    if (int rc = op_common(sh, &H)) return rc;
    if (!mass) return set_err(H, SUNSET_ERR_ARG, "null pointer");
    if (H->nz > 0) {
        if (int rc = need(H, H->state3_ok, "sunset_set_state_3d")) return rc;
        return ke_mass3(H, nullptr, mass);
    }
    if (int rc = need(H, H->state_ok, "sunset_set_state")) return rc;
    return reduce_ke_mass(H, nullptr, mass);
}

int sunset_synchronize(SunsetHandle *sh) {
    if (!sh) return SUNSET_ERR_ARG;
    Handle *H = &sh->H;
    SUNSET_CUDA(H, cudaStreamSynchronize(H->stream));
    return 0;
}

int sunset_run_host(SunsetHandle *sh, const double *state_in, double dt, int nsteps, double *state_out) {
    Handle *H;
    if (int rc = op_common(sh, &H)) return rc;
    if (!state_in || !state_out) return set_err(H, SUNSET_ERR_ARG, "null array");
    if (nsteps < 0 || !(dt > 0.0)) return set_err(H, SUNSET_ERR_ARG, "bad dt/nsteps");
    if (H->nz > 0) {
        if (int rc = need(H, H->state3_ok, "sunset_set_state_3d")) return rc;
        if (int rc = run_host3(H, state_in, dt, nsteps, state_out)) return rc;
        return check_err_flag(H);
    }
    if (int rc = need(H, H->state_ok, "sunset_set_state")) return rc;
    const int n = H->npfb;
    // one copy each way through a 7 x npfb staging block (allocated on the first call), with
    // the permutation between reference and internal order done on the device
    if (!H->io && dalloc(H, &H->io, 7 * (size_t)n)) return SUNSET_ERR_NOMEM;
    const int nb = (n + 255) / 256;
    Fields7 d{{H->rhs[0], H->rhs[1], H->rhs[2], H->rhs[3], H->rhs[4], H->rhs[5], H->rhs[6]}};
    SUNSET_CUDA(H, cudaMemcpyAsync(H->io, state_in, 7 * (size_t)n * sizeof(double), cudaMemcpyHostToDevice, H->stream));
    k_gather7<<<nb, 256, 0, H->stream>>>(H->io, H->perm, n, d);
    SUNSET_CUDA(H, cudaGetLastError());
    if (int rc = state_set_conservative_device(H, d.p)) return rc;
    if (int rc = step_run(H, dt, nsteps, 0)) return rc;
    const Fields &F = H->buf[H->cur];
    Fields7 src{{F.ro, F.rou, F.rov, F.q[0], F.q[1], F.q[2], F.q[3]}};
    k_scatter7<<<nb, 256, 0, H->stream>>>(src, H->perm, n, H->io);
    SUNSET_CUDA(H, cudaGetLastError());
    SUNSET_CUDA(H, cudaMemcpyAsync(state_out, H->io, 7 * (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, H->stream));
    return check_err_flag(H);
}

int sunset_adjoint_apply_D(SunsetHandle *sh, int which, const double *gbar, double *out, int flags) {
    Handle *H;
    if (int rc = op_common(sh, &H)) return rc;
    if (!gbar || !out) return set_err(H, SUNSET_ERR_ARG, "null array");
    if (which < 0 || which > 3) return set_err(H, SUNSET_ERR_ARG, "which must be 0 (d/dx), 1 (d/dy), 2 (Laplacian) or 3 (filter)");
    const int n = H->npfb;
    double *p = H->tmpd, *o = H->tmpd + n;
    if (int rc = to_internal(H, gbar, flags, p)) return rc;
    if (int rc = adjoint_apply_D(H, which, p, o)) return rc;
    return to_reference(H, o, flags, out);
}

int sunset_adjoint_run(SunsetHandle *sh, double dt, int nsteps, int checkpoint_every, double *J,
                       double *dJ_dparams, double *dJ_dstate0) {
    Handle *H;
    if (int rc = op_common(sh, &H)) return rc;
    if (int rc = need(H, H->state_ok, "sunset_set_state")) return rc;
    if (H->nz > 0) return set_err(H, SUNSET_ERR_SCOPE, "the adjoint is 2-D only");
    if (!J || !dJ_dparams) return set_err(H, SUNSET_ERR_ARG, "null output");
    if (!(dt > 0.0)) return set_err(H, SUNSET_ERR_ARG, "dt must be positive");
    const int n = H->npfb;
    double *du = nullptr;
    if (dalloc(H, &du, 7 * (size_t)n)) return SUNSET_ERR_NOMEM;
    int rc = adjoint_run(H, dt, nsteps, checkpoint_every, J, dJ_dparams, du);
    if (!rc && dJ_dstate0)
        for (int f = 0; f < 7 && !rc; f++)
            rc = to_reference(H, du + (size_t)f * n, SUNSET_PTR_HOST, dJ_dstate0 + (size_t)f * n);
    dfree(H, du);
    return rc;
}

int sunset_set_lengths(SunsetHandle *sh, const double *h, const double *h_small) {
    if (!sh) return SUNSET_ERR_ARG;
    Handle *H = &sh->H;
    if (int rc = need(H, H->domain_ok, "sunset_build_domain")) return rc;
    if (H->nbr_ok) return set_err(H, SUNSET_ERR_ARG, "set the lengths before sunset_find_neighbours");
    if (!h || !h_small) return set_err(H, SUNSET_ERR_ARG, "null array");
    if (int rc = set_device(H)) return rc;
    const int n = H->npfb;
    std::vector<double> hv(n), hsv(n);
    for (int i = 0; i < n; i++) {
        const int r = H->h_perm[i];
        if (!(h[r] > 0.0) || !(h_small[r] > 0.0) || h_small[r] > h[r])
            return set_err(H, SUNSET_ERR_ARG, "node %d: need 0 < h_small <= h", r + 1);
        hv[i] = h[r];
        hsv[i] = h_small[r];
        H->hmax = std::max(H->hmax, h[r]);
    }
    SUNSET_CUDA(H, cudaMemcpy(H->h, hv.data(), n * sizeof(double), cudaMemcpyHostToDevice));
    SUNSET_CUDA(H, cudaMemcpy(H->hs, hsv.data(), n * sizeof(double), cudaMemcpyHostToDevice));
    return 0;
}

int sunset_get_dump(SunsetHandle *sh, double *columns, double *header) {
    Handle *H;
    if (int rc = op_common(sh, &H)) return rc;
    if (!columns || !header) return set_err(H, SUNSET_ERR_ARG, "null array");
    if (H->nz > 0) {  // 13 columns over every node-layer, layer-major (output.F90:296-299, -Dallout)
        if (int rc = need(H, H->state3_ok, "sunset_set_state_3d")) return rc;
        const size_t n = (size_t)H->npfb * H->nz;
        double *cols = nullptr;
        if (dalloc(H, &cols, 13 * n)) return SUNSET_ERR_NOMEM;
        int rc = dump3_columns(H, cols);
        for (int f = 0; f < 13 && !rc; f++) rc = state3_column_to_host(H, cols + (size_t)f * n, columns + (size_t)f * n);
        dfree(H, cols);
        if (rc) return rc;
    } else {
        if (int rc = need(H, H->state_ok, "sunset_set_state")) return rc;
        const int n = H->npfb;
        double *cols = nullptr;
        if (dalloc(H, &cols, 10 * (size_t)n)) return SUNSET_ERR_NOMEM;
        int rc = dump_columns(H, cols);
        for (int f = 0; f < 10 && !rc; f++) rc = to_reference(H, cols + (size_t)f * n, SUNSET_PTR_HOST, columns + (size_t)f * n);
        dfree(H, cols);
        if (rc) return rc;
    }
    DevScalars sc;
    SUNSET_CUDA(H, cudaMemcpy(&sc, H->dsc, sizeof(sc), cudaMemcpyDeviceToHost));
    // eflow_nm1, sum_eflow, driving_force(3) (only its x component is ever set), emax_np1,
    // emax_n, emax_nm1, dt (output.F90:272-276)
    const double hd[9] = {sc.eflow_nm1, sc.sum_eflow, sc.df, 0.0, 0.0, sc.emax_np1, sc.emax_n, sc.emax_nm1, sc.dt};
    for (int k = 0; k < 9; k++) header[k] = hd[k];
    return 0;
}

int sunset_write_dump(SunsetHandle *sh, const char *directory, int n_out, double time) {
    Handle *H;
    if (int rc = op_common(sh, &H)) return rc;
    if (!directory || n_out < 0) return set_err(H, SUNSET_ERR_ARG, "bad arguments");
    const int nz = H->nz > 0 ? H->nz : 1, ncol = H->nz > 0 ? 13 : 10;
    const long long n = (long long)H->npfb * nz;  // rows: the nodes, or every node-layer in 3-D
    std::vector<double> cols(ncol * (size_t)n), hd(9);
    if (int rc = sunset_get_dump(sh, cols.data(), hd.data())) return rc;
    const std::string dir(directory);
    const std::string fname = dir + "/fields_10000_" + std::to_string(n_out);
    FILE *f = fopen(fname.c_str(), "w");
    if (!f) return set_err(H, SUNSET_ERR_ARG, "cannot write %s", fname.c_str());
    // output.F90:272-310, list-directed layout
    fprintf(f, " !! header !!\n %lld\n", n);
    fprintf(f, " %.17E %.17E %.17E %.17E %.17E\n", hd[0], hd[1], hd[2], hd[3], hd[4]);
    fprintf(f, " %.17E %.17E %.17E %.17E\n", hd[5], hd[6], hd[7], hd[8]);
    fprintf(f, " !! end header !!\n");
    for (long long i = 0; i < n; i++) {
        for (int c = 0; c < ncol; c++) fprintf(f, " %.17E", cols[(size_t)c * n + i]);
        fputc('\n', f);
    }
    const bool ok = fclose(f) == 0;
    if (!ok) return set_err(H, SUNSET_ERR_ARG, "cannot write %s", fname.c_str());
    if (n_out == 1 && H->nz > 0) {  // output_nodes in 3-D: gi + layer offset, x, y, z, s, h, h_small, type
        const int nl = H->npfb;
        std::vector<double> x(nl), y(nl), sp(nl), hv(nl), hsv(nl);
        std::vector<int> t(nl);
        SUNSET_CUDA(H, cudaMemcpy(x.data(), H->px, nl * sizeof(double), cudaMemcpyDeviceToHost));
        SUNSET_CUDA(H, cudaMemcpy(y.data(), H->py, nl * sizeof(double), cudaMemcpyDeviceToHost));
        SUNSET_CUDA(H, cudaMemcpy(sp.data(), H->sp, nl * sizeof(double), cudaMemcpyDeviceToHost));
        SUNSET_CUDA(H, cudaMemcpy(hv.data(), H->h, nl * sizeof(double), cudaMemcpyDeviceToHost));
        SUNSET_CUDA(H, cudaMemcpy(hsv.data(), H->hs, nl * sizeof(double), cudaMemcpyDeviceToHost));
        SUNSET_CUDA(H, cudaMemcpy(t.data(), H->ntype, nl * sizeof(int), cudaMemcpyDeviceToHost));
        std::vector<int> at(nl);
        for (int i = 0; i < nl; i++) at[H->h_perm[i]] = i;
        const std::string nname = dir + "/nodes_10000";
        FILE *g = fopen(nname.c_str(), "w");
        if (!g) return set_err(H, SUNSET_ERR_ARG, "cannot write %s", nname.c_str());
        fprintf(g, " %lld\n", n);
        for (int iz = 0; iz < H->nz; iz++)  // setup_domain.F90:520-535
            for (int r = 0; r < nl; r++) {
                const int i = at[r];
                fprintf(g, " %lld %.17E %.17E %.17E %.17E %.17E %.17E %d\n", (long long)H->h_gi[r] + (long long)iz * nl, x[i],
                        y[i], (double)iz * H->dz, sp[i], hv[i], hsv[i], t[i]);
            }
        if (fclose(g) != 0) return set_err(H, SUNSET_ERR_ARG, "cannot write %s", nname.c_str());
    } else if (n_out == 1) {  // output_nodes, output.F90:421-476
        std::vector<double> x(n), y(n), sp(n), hv(n), hsv(n);
        std::vector<int> t(n);
        SUNSET_CUDA(H, cudaMemcpy(x.data(), H->px, n * sizeof(double), cudaMemcpyDeviceToHost));
        SUNSET_CUDA(H, cudaMemcpy(y.data(), H->py, n * sizeof(double), cudaMemcpyDeviceToHost));
        SUNSET_CUDA(H, cudaMemcpy(sp.data(), H->sp, n * sizeof(double), cudaMemcpyDeviceToHost));
        SUNSET_CUDA(H, cudaMemcpy(hv.data(), H->h, n * sizeof(double), cudaMemcpyDeviceToHost));
        SUNSET_CUDA(H, cudaMemcpy(hsv.data(), H->hs, n * sizeof(double), cudaMemcpyDeviceToHost));
        SUNSET_CUDA(H, cudaMemcpy(t.data(), H->ntype, n * sizeof(int), cudaMemcpyDeviceToHost));
        std::vector<int> at(n);  // reference index -> internal
        for (int i = 0; i < n; i++) at[H->h_perm[i]] = i;
        const std::string nname = dir + "/nodes_10000";
        FILE *g = fopen(nname.c_str(), "w");
        if (!g) return set_err(H, SUNSET_ERR_ARG, "cannot write %s", nname.c_str());
        fprintf(g, " %d\n", n);
        for (int r = 0; r < n; r++) {
            const int i = at[r];
            fprintf(g, " %d %.17E %.17E %.17E %.17E %.17E %d\n", H->h_gi[r], x[i], y[i], sp[i], hv[i], hsv[i], t[i]);
        }
        if (fclose(g) != 0) return set_err(H, SUNSET_ERR_ARG, "cannot write %s", nname.c_str());
    }
    const std::string tname = dir + "/time.out";  // unit 21: time, dims, npfb, n_out, nprocs
    FILE *tf = fopen(tname.c_str(), "a");
    if (!tf) return set_err(H, SUNSET_ERR_ARG, "cannot write %s", tname.c_str());
    fprintf(tf, " %.17E %d %lld %d 1\n", time, H->nz > 0 ? 3 : 2, n, n_out);
    if (fclose(tf) != 0) return set_err(H, SUNSET_ERR_ARG, "cannot write %s", tname.c_str());
    return 0;
}

int sunset_set_restart(SunsetHandle *sh, const double *columns, const double *header) {
    Handle *H;
    if (int rc = op_common(sh, &H)) return rc;
    if (!columns || !header) return set_err(H, SUNSET_ERR_ARG, "null array");
    if (header[3] != 0.0 || header[4] != 0.0)
        return set_err(H, SUNSET_ERR_SCOPE, "driving_force(2:3) must be zero (the controller drives x only)");
    const double *c = columns;
    if (H->nz > 0) {  // load_restart_file in 3-D (setup_flow.F90:505-509): 13 columns a node-layer
        const size_t n = (size_t)H->npfb * H->nz;
        std::vector<double> ro(n);
        for (size_t k = 0; k < n; k++) ro[k] = c[k] + 1.0;
        if (int rc = sunset_set_state_3d(sh, ro.data(), c + n, c + 2 * n, c + 3 * n, c + 7 * n, c + 8 * n, c + 9 * n,
                                         c + 10 * n, c + 11 * n, c + 12 * n))
            return rc;
    } else {
        const int n = H->npfb;
        // load_restart_file, setup_flow.F90:448-552: rho = (rho - rho_char) + rho_char, u, v, c
        std::vector<double> ro(n);
        for (int i = 0; i < n; i++) ro[i] = columns[i] + 1.0;
        if (int rc = sunset_set_state(sh, ro.data(), c + n, c + 2 * (size_t)n, c + 6 * (size_t)n, c + 7 * (size_t)n,
                                      c + 8 * (size_t)n, c + 9 * (size_t)n))
            return rc;
    }
    DevScalars sc;
    SUNSET_CUDA(H, cudaMemcpy(&sc, H->dsc, sizeof(sc), cudaMemcpyDeviceToHost));
    sc.eflow_nm1 = header[0];
    sc.sum_eflow = header[1];
    sc.df = header[2];
    sc.emax_np1 = header[5];
    sc.emax_n = header[6];
    sc.emax_nm1 = header[7];
    sc.dt = header[8];
    SUNSET_CUDA(H, cudaMemcpy(H->dsc, &sc, sizeof(sc), cudaMemcpyHostToDevice));
    return 0;
}

int sunset_get_flow_control(SunsetHandle *sh, double *out) {
    Handle *H;
    if (int rc = op_common(sh, &H)) return rc;
    if (int rc = need(H, H->nz > 0 ? H->state3_ok : H->state_ok, H->nz > 0 ? "sunset_set_state_3d" : "sunset_set_state"))
        return rc;
    if (!out) return set_err(H, SUNSET_ERR_ARG, "null array");
    DevScalars sc;
    SUNSET_CUDA(H, cudaMemcpy(&sc, H->dsc, sizeof(sc), cudaMemcpyDeviceToHost));
    out[0] = sc.eflow_nm1;
    out[1] = sc.sum_eflow;
    out[2] = sc.df;
    out[3] = 0.0;
    out[4] = 0.0;
    return 0;
}

int sunset_set_flow_control(SunsetHandle *sh, const double *in) {
    Handle *H;
    if (int rc = op_common(sh, &H)) return rc;
    if (int rc = need(H, H->nz > 0 ? H->state3_ok : H->state_ok, H->nz > 0 ? "sunset_set_state_3d" : "sunset_set_state"))
        return rc;
    if (!in) return set_err(H, SUNSET_ERR_ARG, "null array");
    if (in[3] != 0.0 || in[4] != 0.0) return set_err(H, SUNSET_ERR_SCOPE, "driving_force(2:3) must be zero (the controller drives x only)");
    DevScalars sc;
    SUNSET_CUDA(H, cudaMemcpy(&sc, H->dsc, sizeof(sc), cudaMemcpyDeviceToHost));
    sc.eflow_nm1 = in[0];
    sc.sum_eflow = in[1];
    sc.df = in[2];
    SUNSET_CUDA(H, cudaMemcpy(H->dsc, &sc, sizeof(sc), cudaMemcpyHostToDevice));
    return 0;
}

int sunset_checkpoint_size(SunsetHandle *sh, size_t *bytes) {
    Handle *H;
    if (int rc = op_common(sh, &H)) return rc;
    if (!bytes) return set_err(H, SUNSET_ERR_ARG, "null pointer");
    *bytes = H->nz > 0 ? checkpoint3_bytes(H) : checkpoint_bytes(H);
    return 0;
}

int sunset_save_checkpoint(SunsetHandle *sh, void *buffer, size_t bytes) {
    Handle *H;
    if (int rc = op_common(sh, &H)) return rc;
    if (H->nz > 0) {
        if (int rc = need(H, H->state3_ok, "sunset_set_state_3d")) return rc;
        if (!buffer || bytes < checkpoint3_bytes(H)) return set_err(H, SUNSET_ERR_ARG, "checkpoint buffer too small");
        return checkpoint3_save(H, buffer);
    }
    if (int rc = need(H, H->state_ok, "sunset_set_state")) return rc;
    if (!buffer || bytes < checkpoint_bytes(H)) return set_err(H, SUNSET_ERR_ARG, "checkpoint buffer too small");
    return checkpoint_save(H, buffer);
}

int sunset_load_checkpoint(SunsetHandle *sh, const void *buffer, size_t bytes) {
    Handle *H;
    if (int rc = op_common(sh, &H)) return rc;
    if (!buffer) return set_err(H, SUNSET_ERR_ARG, "null buffer");
    if (H->nz > 0) {
        if (int rc = checkpoint3_load(H, buffer, bytes)) return rc;
        H->state3_ok = true;
        return 0;
    }
    if (int rc = state_alloc(H)) return rc;
    if (int rc = checkpoint_load(H, buffer, bytes)) return rc;
    H->state_ok = true;
    return 0;
}

int sunset_time_stage_kernel(SunsetHandle *sh, int reps, double *ms_per_launch, double *bytes_per_launch) {
    Handle *H;
    if (int rc = op_common(sh, &H)) return rc;
    if (reps <= 0 || !ms_per_launch || !bytes_per_launch) return set_err(H, SUNSET_ERR_ARG, "bad arguments");
    if (H->nz > 0) {  // 3-D: the derivative gather k3_derivs
        if (int rc = need(H, H->state3_ok, "sunset_set_state_3d")) return rc;
        if (int rc = time3_derivs(H, reps, ms_per_launch, bytes_per_launch)) return rc;
        return check_err_flag(H);
    }
    if (int rc = need(H, H->state_ok, "sunset_set_state")) return rc;
    return time_stage_kernel(H, reps, ms_per_launch, bytes_per_launch);
}

}  // extern "C"
