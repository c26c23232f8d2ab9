// setup.cu -- device-resident domain: ghost points, Morton renumbering, cell-list neighbour
// search and per-row distance sort (neighbours.F90, mirror_boundaries.F90).
//
// Compiled with -fmad=false: ghost positions and squared distances are formed with the
// same operations, in the same order, as the reference, so the neighbour sets and the
// distance order match it exactly.
#include <cub/cub.cuh>

#include "internal.cuh"

namespace sunset {

namespace {

// ---------------------------------------------------------------------------------------
// Mirror (ghost) points, mirror_boundaries.F90:34-261.  One pass counts each node's
// mirrors, a scan gives offsets in reference node order, a second pass writes them, so
// the ghost numbering equals the reference's (npfb+1, npfb+2, ... in node order).
// ---------------------------------------------------------------------------------------
struct MirrorArgs {
    const double *x, *y, *h;
    int n;
    double xmin, xmax, ymin, ymax;
    int xL, xU, yL, yU;
};

template <bool WRITE>
__device__ int mirrors_of(const MirrorArgs &a, int i, double *gx, double *gy, int *gpar, int *gvrel) {
    const double xi = a.x[i], yi = a.y[i];
    const double lim = (kSs * a.h[i]) * 2.0;  // ss*h(i)*mlayer_buff
    int m = 0;
    auto emit = [&](int vrel, double xn, double yn) {
        if (WRITE) { gx[m] = xn; gy[m] = yn; gpar[m] = i; gvrel[m] = vrel; }
        m++;
    };
    if (xi <= a.xmin + lim) {
        if (a.xL == 1) emit(1, (xi + a.xmax) - a.xmin, yi);
        else if (a.xL == 2) emit(2, 2.0 * a.xmin - xi, yi);
    }
    if (xi >= a.xmax - lim) {
        if (a.xU == 1) emit(1, (xi - a.xmax) + a.xmin, yi);
        else if (a.xU == 2) emit(2, 2.0 * a.xmax - xi, yi);
    }
    if (yi <= a.ymin + lim) {
        if (a.yL == 1) emit(1, xi, (yi + a.ymax) - a.ymin);
        else if (a.yL == 2) emit(3, xi, 2.0 * a.ymin - yi);
        else if (a.yL == 3) emit(4, xi, 2.0 * a.ymin - yi);
    }
    if (yi >= a.ymax - lim) {
        if (a.yU == 1) emit(1, xi, (yi - a.ymax) + a.ymin);
        else if (a.yU == 2) emit(3, xi, 2.0 * a.ymax - yi);
        else if (a.yU == 3) emit(4, xi, 2.0 * a.ymax - yi);
    }
    const double cx[4] = {a.xmin, a.xmax, a.xmin, a.xmax}, cy[4] = {a.ymin, a.ymin, a.ymax, a.ymax};
    const int bx[4] = {a.xL, a.xU, a.xL, a.xU}, by[4] = {a.yL, a.yL, a.yU, a.yU};
    for (int c = 0; c < 4; c++) {
        double dx = cx[c] - xi, dy = cy[c] - yi, dz = 0.0 - 0.0;
        double cdist = sqrt((dx * dx + dy * dy) + dz * dz);
        if (cdist <= lim && bx[c] != 0 && by[c] != 0) {
            bool right = (c == 1 || c == 3), top = (c == 2 || c == 3);
            double xp = right ? (xi - a.xmax) + a.xmin : (xi + a.xmax) - a.xmin;
            double yp = top ? (yi - a.ymax) + a.ymin : (yi + a.ymax) - a.ymin;
            double xs = right ? 2.0 * a.xmax - xi : 2.0 * a.xmin - xi;
            double ys = top ? 2.0 * a.ymax - yi : 2.0 * a.ymin - yi;
            if (bx[c] == 1 && by[c] == 1) emit(1, xp, yp);
            else if (bx[c] == 2 && by[c] == 1) emit(2, xs, yp);
            else if (bx[c] == 1 && by[c] == 2) emit(3, xp, ys);
            else if (bx[c] == 2 && by[c] == 2) emit(4, xs, ys);
            else emit(-1, xi, yi);  // undefined in the reference (host rejects it)
        }
    }
    return m;
}

__global__ void k_count_mirrors(MirrorArgs a, int *count) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < a.n) count[i] = mirrors_of<false>(a, i, nullptr, nullptr, nullptr, nullptr);
}

__global__ void k_write_mirrors(MirrorArgs a, const int *offset, double *gx, double *gy, int *gpar_ref,
                                int *gvrel) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    int o = offset[i];
    mirrors_of<true>(a, i, gx + o, gy + o, gpar_ref + o, gvrel + o);
}

__device__ __forceinline__ uint32_t spread16(uint32_t v) {
    v &= 0xffff;
    v = (v | (v << 8)) & 0x00ff00ff;
    v = (v | (v << 4)) & 0x0f0f0f0f;
    v = (v | (v << 2)) & 0x33333333;
    v = (v | (v << 1)) & 0x55555555;
    return v;
}

__global__ void k_morton(const double *x, const double *y, int n, double x0, double y0, double inv_dx,
                         double inv_dy, uint32_t *key, int *val) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double fx = (x[i] - x0) * inv_dx, fy = (y[i] - y0) * inv_dy;
    uint32_t qx = (uint32_t)fmin(fmax(fx, 0.0), 65535.0);
    uint32_t qy = (uint32_t)fmin(fmax(fy, 0.0), 65535.0);
    key[i] = spread16(qx) | (spread16(qy) << 1);
    val[i] = i;
}

__global__ void k_gather_nodes(int n, const int *perm, const double *x, const double *y, const double *h,
                               const double *hs, const double *s, const int *type, double *px, double *py,
                               double *ho, double *hso, double *so, int *to, int *iperm) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int r = perm[i];
    px[i] = x[r]; py[i] = y[r]; ho[i] = h[r]; hso[i] = hs[r]; so[i] = s[r]; to[i] = type[r];
    iperm[r] = i;
}

__global__ void k_place_ghosts(int ng, int npfb, const double *gx, const double *gy, const int *gpar_ref,
                               const int *iperm, double *px, double *py, int *gpar) {
    int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= ng) return;
    px[npfb + g] = gx[g];
    py[npfb + g] = gy[g];
    gpar[g] = iperm[gpar_ref[g]];
}

// ---------------------------------------------------------------------------------------
// Cell list over all points (interior + ghosts) and the per-node search,
// neighbours.F90:160-270.  The cell side is ss*max(h), so the 3x3 block of cells around
// a node covers its support.
// ---------------------------------------------------------------------------------------
struct Grid {
    double x0, y0, inv;
    int ncx, ncy;
};

__global__ void k_cell_id(const double *px, const double *py, int np, Grid g, int *cid, int *pid) {
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= np) return;
    int cx = (int)((px[p] - g.x0) * g.inv), cy = (int)((py[p] - g.y0) * g.inv);
    cx = min(max(cx, 0), g.ncx - 1);
    cy = min(max(cy, 0), g.ncy - 1);
    cid[p] = cx + g.ncx * cy;
    pid[p] = p;
}

__global__ void k_cell_bounds(const int *cid_sorted, int np, int *cstart, int *cend) {
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= np) return;
    int c = cid_sorted[p];
    if (p == 0 || cid_sorted[p - 1] != c) cstart[c] = p;
    if (p == np - 1 || cid_sorted[p + 1] != c) cend[c] = p + 1;
}

// The reference's search grid (cell_generator, neighbours.F90:75-93): square cells of side
// ss*h0 over the domain tripled in each direction.
struct RefGrid {
    double xmint, ymint, unoss;
};

struct SearchArgs {
    const double *px, *py, *h;
    const int *cstart, *cend, *pts;
    Grid g;
    RefGrid rg;
    int npfb;
};

template <bool FILL>
__global__ void k_search(SearchArgs a, int *count, const long long *rowptr, int *opt, double *or2) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.npfb) return;
    const double xi = a.px[i], yi = a.py[i];
    const double hh = a.h[i] * kSs, hs2 = hh * hh;
    int cx = min(max((int)((xi - a.g.x0) * a.g.inv), 0), a.g.ncx - 1);
    int cy = min(max((int)((yi - a.g.y0) * a.g.inv), 0), a.g.ncy - 1);
    // the reference scans only the 3x3 block of its own cells around the node
    // (neighbour_cells, neighbours.F90:95-158), so where a node's ss*h exceeds the cell side
    // ss*h0 (boundary nodes at order 4: hovs_bound > hovs) the points further out are not its
    // neighbours even inside the radius
    const int ci = (int)((xi - a.rg.xmint) * a.rg.unoss), cj = (int)((yi - a.rg.ymint) * a.rg.unoss);
    long long o = FILL ? rowptr[i] : 0;
    int cnt = 0;
    for (int dy = -1; dy <= 1; dy++) {
        int yy = cy + dy;
        if (yy < 0 || yy >= a.g.ncy) continue;
        for (int dx = -1; dx <= 1; dx++) {
            int xx = cx + dx;
            if (xx < 0 || xx >= a.g.ncx) continue;
            int c = xx + a.g.ncx * yy;
            int e = a.cend[c];
            for (int q = a.cstart[c]; q < e; q++) {
                int p = a.pts[q];
                double rx = xi - a.px[p], ry = yi - a.py[p], rz = 0.0 - 0.0;
                double rr2 = (rx * rx + ry * ry) + rz * rz;
                if (rr2 <= hs2) {
                    const int dcx = (int)((a.px[p] - a.rg.xmint) * a.rg.unoss) - ci;
                    const int dcy = (int)((a.py[p] - a.rg.ymint) * a.rg.unoss) - cj;
                    if (dcx < -1 || dcx > 1 || dcy < -1 || dcy > 1) continue;
                    if (FILL) { opt[o + cnt] = p; or2[o + cnt] = rr2; }
                    cnt++;
                }
            }
        }
    }
    if (!FILL) count[i] = cnt;
}

// Reference numbering of a point, used to order links at equal distance deterministically.
__device__ __forceinline__ int ref_point(int p, int npfb, const int *perm) { return p < npfb ? perm[p] : p; }

// Position of the cell (dx, dy) relative to a node's own cell in the reference's scan of the
// neighbouring cells (neighbour_cells, neighbours.F90:95-158): self, E, NE, SE, W, NW, SW, N, S.
__device__ __forceinline__ int scan_position(int dx, int dy) {
    if (dx == 0 && dy == 0) return 0;
    if (dx == 1) return dy == 0 ? 1 : dy == 1 ? 2 : 3;
    if (dx == -1) return dy == 0 ? 4 : dy == 1 ? 5 : 6;
    return dy == 1 ? 7 : 8;
}

constexpr int kMaxRowSort = 1024;  // longest row the reference-order sort accepts

// order_neighbours (neighbours.F90:272-341), reproducing where links at exactly equal
// distance end up (straight walls, FD rows and their periodic images give such ties): the
// row is first put in the order in which the reference's cell scan finds the links (scan
// position of the link's cell, then point number within a cell, as divide() fills the
// cells), then sorted by squared distance with the reference's quicksort
// (quicksort_neighbours), run with an explicit stack.  ij_count_small counts the links
// inside ss*h_small.
__global__ void k_sort_rows(int npfb, const long long *rowptr, int *opt, double *or2, const double *hs,
                            const int *perm, const double *px, const double *py, RefGrid rg, int *cnt_small,
                            int *err) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= npfb) return;
    long long b = rowptr[i], e = rowptr[i + 1];
    const int n = (int)(e - b);
    if (n > kMaxRowSort) {
        atomicExch(err, i + 1);
        return;
    }
    const int ci = (int)((px[i] - rg.xmint) * rg.unoss), cj = (int)((py[i] - rg.ymint) * rg.unoss);
    auto scan_key = [&](int p) -> long long {
        int dx = (int)((px[p] - rg.xmint) * rg.unoss) - ci, dy = (int)((py[p] - rg.ymint) * rg.unoss) - cj;
        // (k_search keeps no link beyond the 3x3 cells; such a link would go last)
        int pos = (dx < -1 || dx > 1 || dy < -1 || dy > 1) ? 9 : scan_position(dx, dy);
        return ((long long)pos << 32) | (unsigned)ref_point(p, npfb, perm);
    };
    for (long long a = b + 1; a < e; a++) {  // insertion sort into scan order
        double key = or2[a];
        int p = opt[a];
        long long kp = scan_key(p);
        long long c = a - 1;
        while (c >= b && scan_key(opt[c]) > kp) {
            or2[c + 1] = or2[c];
            opt[c + 1] = opt[c];
            c--;
        }
        or2[c + 1] = key;
        opt[c + 1] = p;
    }
    // quicksort_neighbours on the 1-based range [1, n] of this row
    double *a = or2 + b - 1;
    int *lk = opt + b - 1;
    int stk[2 * 64];
    int top = 0;
    if (n >= 1) { stk[0] = 1; stk[1] = n; top = 1; }
    while (top > 0) {
        top--;
        const int first = stk[2 * top], last = stk[2 * top + 1];
        const double x = a[(first + last) / 2];
        int ii = first, jj = last;
        for (;;) {
            while (a[ii] < x) ii++;
            while (x < a[jj]) jj--;
            if (ii >= jj) break;
            double t = a[ii]; a[ii] = a[jj]; a[jj] = t;
            int it = lk[ii]; lk[ii] = lk[jj]; lk[jj] = it;
            ii++;
            jj--;
        }
        if (top + 2 > 64) {  // deeper than any row of kMaxRowSort links needs in practice
            atomicExch(err, i + 1);
            return;
        }
        if (first < ii - 1) { stk[2 * top] = first; stk[2 * top + 1] = ii - 1; top++; }
        if (jj + 1 < last) { stk[2 * top] = jj + 1; stk[2 * top + 1] = last; top++; }
    }
    double t = hs[i] * kSs, hs2 = t * t;
    int small = 0;
    for (long long q = b; q < e; q++)
        if (or2[q] <= hs2) small++;
    cnt_small[i] = small;
}

__global__ void k_fill_sell(int npfb, int nslices, const long long *rowptr, const int *opt,
                            const long long *slice_ptr, const int *slice_w, const int *gpar,
                            const int *gvrel, int *lpt, int *lidx, int *mirror_flag) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int sl = i >> 5;
    if (sl >= nslices) return;
    int lane = i & 31;
    long long base = slice_ptr[sl];
    int w = slice_w[sl];
    long long b = i < npfb ? rowptr[i] : 0;
    int cnt = i < npfb ? (int)(rowptr[i + 1] - b) : 0;
    for (int k = 0; k < w; k++) {
        long long o = sell_at(base, k, lane);
        if (k < cnt) {
            int p = opt[b + k];
            lpt[o] = p;
            if (p < npfb) {
                lidx[o] = p;
            } else {
                int g = p - npfb;
                int code = gvrel[g] - 1;
                lidx[o] = gpar[g] | (code << 30);
                if (code != 0) *mirror_flag = 1;
            }
        } else {
            lpt[o] = -1;
            lidx[o] = 0;
        }
    }
}

}  // namespace

// ---------------------------------------------------------------------------------------
int build_domain_device(Handle *H, const std::vector<double> &x, const std::vector<double> &y,
                        const std::vector<double> &h, const std::vector<double> &hs,
                        const std::vector<double> &s, const std::vector<int> &type) {
    const int n = H->npfb;
    cudaStream_t st = H->stream;
    double *dx, *dy, *dh, *dhs, *ds;
    int *dt;
    if (dalloc(H, &dx, n) || dalloc(H, &dy, n) || dalloc(H, &dh, n) || dalloc(H, &dhs, n) ||
        dalloc(H, &ds, n) || dalloc(H, &dt, n))
        return SUNSET_ERR_NOMEM;
    SUNSET_CUDA(H, cudaMemcpyAsync(dx, x.data(), n * sizeof(double), cudaMemcpyHostToDevice, st));
    SUNSET_CUDA(H, cudaMemcpyAsync(dy, y.data(), n * sizeof(double), cudaMemcpyHostToDevice, st));
    SUNSET_CUDA(H, cudaMemcpyAsync(dh, h.data(), n * sizeof(double), cudaMemcpyHostToDevice, st));
    SUNSET_CUDA(H, cudaMemcpyAsync(dhs, hs.data(), n * sizeof(double), cudaMemcpyHostToDevice, st));
    SUNSET_CUDA(H, cudaMemcpyAsync(ds, s.data(), n * sizeof(double), cudaMemcpyHostToDevice, st));
    SUNSET_CUDA(H, cudaMemcpyAsync(dt, type.data(), n * sizeof(int), cudaMemcpyHostToDevice, st));

    // mirrors
    MirrorArgs ma{dx, dy, dh, n, H->xmin, H->xmax, H->ymin, H->ymax, H->bc[0], H->bc[1], H->bc[2], H->bc[3]};
    int *mcount, *moff;
    if (dalloc(H, &mcount, n + 1) || dalloc(H, &moff, n + 1)) return SUNSET_ERR_NOMEM;
    const int TB = 256;
    k_count_mirrors<<<(n + TB - 1) / TB, TB, 0, st>>>(ma, mcount);
    SUNSET_CUDA(H, cudaMemsetAsync(mcount + n, 0, sizeof(int), st));
    size_t tmpb = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tmpb, mcount, moff, n + 1, st);
    void *tmp;
    if (dalloc(H, (char **)&tmp, tmpb)) return SUNSET_ERR_NOMEM;
    cub::DeviceScan::ExclusiveSum(tmp, tmpb, mcount, moff, n + 1, st);
    dfree(H, tmp);
    int ng = 0;
    SUNSET_CUDA(H, cudaMemcpyAsync(&ng, moff + n, sizeof(int), cudaMemcpyDeviceToHost, st));
    SUNSET_CUDA(H, cudaStreamSynchronize(st));
    H->nghost = ng;
    H->np = n + ng;
    double *gx, *gy;
    int *gpar_ref;
    if (dalloc(H, &gx, ng) || dalloc(H, &gy, ng) || dalloc(H, &gpar_ref, ng) || dalloc(H, &H->gvrel, ng) ||
        dalloc(H, &H->gpar, ng))
        return SUNSET_ERR_NOMEM;
    k_write_mirrors<<<(n + TB - 1) / TB, TB, 0, st>>>(ma, moff, gx, gy, gpar_ref, H->gvrel);
    {
        std::vector<int> vr(ng);
        SUNSET_CUDA(H, cudaMemcpyAsync(vr.data(), H->gvrel, ng * sizeof(int), cudaMemcpyDeviceToHost, st));
        SUNSET_CUDA(H, cudaStreamSynchronize(st));
        for (int v : vr)
            if (v < 0) return set_err(H, SUNSET_ERR_SCOPE, "corner mirror for this bcond combination is undefined in the reference");
    }

    // Morton renumbering of the interior nodes
    uint32_t *key, *key2;
    int *val, *val2;
    if (dalloc(H, &key, n) || dalloc(H, &key2, n) || dalloc(H, &val, n) || dalloc(H, &val2, n)) return SUNSET_ERR_NOMEM;
    double Lx = H->xmax - H->xmin, Ly = H->ymax - H->ymin;
    k_morton<<<(n + TB - 1) / TB, TB, 0, st>>>(dx, dy, n, H->xmin, H->ymin, 65535.0 / Lx, 65535.0 / Ly, key, val);
    tmpb = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, tmpb, key, key2, val, val2, n, 0, 32, st);
    if (dalloc(H, (char **)&tmp, tmpb)) return SUNSET_ERR_NOMEM;
    cub::DeviceRadixSort::SortPairs(tmp, tmpb, key, key2, val, val2, n, 0, 32, st);
    dfree(H, tmp);
    if (dalloc(H, &H->perm, n) || dalloc(H, &H->iperm, n) || dalloc(H, &H->px, H->np) ||
        dalloc(H, &H->py, H->np) || dalloc(H, &H->h, n) || dalloc(H, &H->hs, n) || dalloc(H, &H->sp, n) ||
        dalloc(H, &H->ntype, n))
        return SUNSET_ERR_NOMEM;
    SUNSET_CUDA(H, cudaMemcpyAsync(H->perm, val2, n * sizeof(int), cudaMemcpyDeviceToDevice, st));
    k_gather_nodes<<<(n + TB - 1) / TB, TB, 0, st>>>(n, H->perm, dx, dy, dh, dhs, ds, dt, H->px, H->py, H->h,
                                                     H->hs, H->sp, H->ntype, H->iperm);
    if (ng > 0)
        k_place_ghosts<<<(ng + TB - 1) / TB, TB, 0, st>>>(ng, n, gx, gy, gpar_ref, H->iperm, H->px, H->py, H->gpar);
    SUNSET_CUDA(H, cudaGetLastError());
    H->h_perm.resize(n);
    H->h_iperm.resize(n);
    SUNSET_CUDA(H, cudaMemcpyAsync(H->h_perm.data(), H->perm, n * sizeof(int), cudaMemcpyDeviceToHost, st));
    SUNSET_CUDA(H, cudaMemcpyAsync(H->h_iperm.data(), H->iperm, n * sizeof(int), cudaMemcpyDeviceToHost, st));
    SUNSET_CUDA(H, cudaStreamSynchronize(st));
    for (void *p : {(void *)dx, (void *)dy, (void *)dh, (void *)dhs, (void *)ds, (void *)dt, (void *)mcount,
                    (void *)moff, (void *)gx, (void *)gy, (void *)gpar_ref, (void *)key, (void *)key2, (void *)val,
                    (void *)val2})
        dfree(H, p);
    return 0;
}

// ---------------------------------------------------------------------------------------
int find_neighbours_device(Handle *H) {
    const int n = H->npfb, np = H->np;
    cudaStream_t st = H->stream;
    const int TB = 256;
    // grid: covers the domain plus the ghost band (ghosts lie within 4 h of an edge)
    double cs = kSs * H->hmax;
    double margin = 2.0 * cs + 4.0 * H->hmax + 1e-12 * (H->xmax - H->xmin);
    Grid g;
    g.x0 = H->xmin - margin;
    g.y0 = H->ymin - margin;
    g.inv = 1.0 / cs;
    g.ncx = (int)((H->xmax - H->xmin + 2 * margin) * g.inv) + 1;
    g.ncy = (int)((H->ymax - H->ymin + 2 * margin) * g.inv) + 1;
    long long ncell = (long long)g.ncx * g.ncy;
    if (ncell > (1LL << 31)) return set_err(H, SUNSET_ERR_SCOPE, "cell grid too large (%lld cells)", ncell);
    int *cid, *cid2, *pid, *pid2, *cstart, *cend;
    if (dalloc(H, &cid, np) || dalloc(H, &cid2, np) || dalloc(H, &pid, np) || dalloc(H, &pid2, np) ||
        dalloc(H, &cstart, ncell) || dalloc(H, &cend, ncell))
        return SUNSET_ERR_NOMEM;
    k_cell_id<<<(np + TB - 1) / TB, TB, 0, st>>>(H->px, H->py, np, g, cid, pid);
    size_t tmpb = 0;
    void *tmp;
    cub::DeviceRadixSort::SortPairs(nullptr, tmpb, cid, cid2, pid, pid2, np, 0, 32, st);
    if (dalloc(H, (char **)&tmp, tmpb)) return SUNSET_ERR_NOMEM;
    cub::DeviceRadixSort::SortPairs(tmp, tmpb, cid, cid2, pid, pid2, np, 0, 32, st);
    dfree(H, tmp);
    SUNSET_CUDA(H, cudaMemsetAsync(cstart, 0, ncell * sizeof(int), st));
    SUNSET_CUDA(H, cudaMemsetAsync(cend, 0, ncell * sizeof(int), st));
    k_cell_bounds<<<(np + TB - 1) / TB, TB, 0, st>>>(cid2, np, cstart, cend);

    const RefGrid rg{H->xmin - (H->xmax - H->xmin), H->ymin - (H->ymax - H->ymin), 1.0 / (1.0 * (kSs * H->h0))};
    SearchArgs sa{H->px, H->py, H->h, cstart, cend, pid2, g, rg, n};
    int *count;
    long long *cnt64, *rowptr;
    if (dalloc(H, &count, n) || dalloc(H, &cnt64, n + 1) || dalloc(H, &rowptr, n + 1)) return SUNSET_ERR_NOMEM;
    k_search<false><<<(n + TB - 1) / TB, TB, 0, st>>>(sa, count, nullptr, nullptr, nullptr);
    std::vector<int> hcount(n);
    SUNSET_CUDA(H, cudaMemcpyAsync(hcount.data(), count, n * sizeof(int), cudaMemcpyDeviceToHost, st));
    SUNSET_CUDA(H, cudaStreamSynchronize(st));
    std::vector<long long> hrow(n + 1);
    hrow[0] = 0;
    int maxc = 0;
    for (int i = 0; i < n; i++) {
        hrow[i + 1] = hrow[i] + hcount[i];
        maxc = hcount[i] > maxc ? hcount[i] : maxc;
    }
    long long nl = hrow[n];
    SUNSET_CUDA(H, cudaMemcpyAsync(rowptr, hrow.data(), (n + 1) * sizeof(long long), cudaMemcpyHostToDevice, st));
    int *opt;
    double *or2;
    if (dalloc(H, &opt, nl) || dalloc(H, &or2, nl)) return SUNSET_ERR_NOMEM;
    k_search<true><<<(n + TB - 1) / TB, TB, 0, st>>>(sa, nullptr, rowptr, opt, or2);
    if (!H->cnt_small && dalloc(H, &H->cnt_small, n)) return SUNSET_ERR_NOMEM;
    int *serr;
    if (dalloc(H, &serr, 1)) return SUNSET_ERR_NOMEM;
    SUNSET_CUDA(H, cudaMemsetAsync(serr, 0, sizeof(int), st));
    k_sort_rows<<<(n + TB - 1) / TB, TB, 0, st>>>(n, rowptr, opt, or2, H->hs, H->perm, H->px, H->py, rg,
                                                  H->cnt_small, serr);
    int hserr = 0;
    SUNSET_CUDA(H, cudaMemcpyAsync(&hserr, serr, sizeof(int), cudaMemcpyDeviceToHost, st));
    SUNSET_CUDA(H, cudaStreamSynchronize(st));
    dfree(H, serr);
    if (hserr) return set_err(H, SUNSET_ERR_SCOPE, "neighbour row of node %d too long to sort", hserr - 1);
    std::vector<int> hsmall(n);
    SUNSET_CUDA(H, cudaMemcpyAsync(hsmall.data(), H->cnt_small, n * sizeof(int), cudaMemcpyDeviceToHost, st));
    SUNSET_CUDA(H, cudaStreamSynchronize(st));

    // sliced ELL layout
    H->nslices = (n + kSlice - 1) / kSlice;
    std::vector<long long> sptr(H->nslices + 1);
    std::vector<int> sw(H->nslices), sws(H->nslices);
    sptr[0] = 0;
    for (int sl = 0; sl < H->nslices; sl++) {
        int w = 0, ws = 0;
        for (int i = sl * kSlice; i < n && i < (sl + 1) * kSlice; i++) {
            w = hcount[i] > w ? hcount[i] : w;
            ws = hsmall[i] > ws ? hsmall[i] : ws;
        }
        w = (w + 1) & ~1;  // even widths: links are stored in pairs (sell_at)
        ws = (ws + 1) & ~1;
        sw[sl] = w;
        sws[sl] = ws;
        sptr[sl + 1] = sptr[sl] + (long long)w * kSlice;
    }
    H->nlinks_sell = sptr[H->nslices];
    H->nplink = maxc;
    if (dalloc(H, &H->slice_ptr, H->nslices + 1) || dalloc(H, &H->slice_w, H->nslices) ||
        dalloc(H, &H->slice_ws, H->nslices) || dalloc(H, &H->lpt, H->nlinks_sell) ||
        dalloc(H, &H->lidx, H->nlinks_sell) || (!H->cnt && dalloc(H, &H->cnt, n)))
        return SUNSET_ERR_NOMEM;
    SUNSET_CUDA(H, cudaMemcpyAsync(H->slice_ptr, sptr.data(), sptr.size() * sizeof(long long), cudaMemcpyHostToDevice, st));
    SUNSET_CUDA(H, cudaMemcpyAsync(H->slice_w, sw.data(), sw.size() * sizeof(int), cudaMemcpyHostToDevice, st));
    SUNSET_CUDA(H, cudaMemcpyAsync(H->slice_ws, sws.data(), sws.size() * sizeof(int), cudaMemcpyHostToDevice, st));
    SUNSET_CUDA(H, cudaMemcpyAsync(H->cnt, hcount.data(), n * sizeof(int), cudaMemcpyHostToDevice, st));
    int *mflag;
    if (dalloc(H, &mflag, 1)) return SUNSET_ERR_NOMEM;
    SUNSET_CUDA(H, cudaMemsetAsync(mflag, 0, sizeof(int), st));
    int nthreads = H->nslices * kSlice;
    k_fill_sell<<<(nthreads + TB - 1) / TB, TB, 0, st>>>(n, H->nslices, rowptr, opt, H->slice_ptr, H->slice_w,
                                                          H->gpar, H->gvrel, H->lpt, H->lidx, mflag);
    int hm = 0;
    SUNSET_CUDA(H, cudaMemcpyAsync(&hm, mflag, sizeof(int), cudaMemcpyDeviceToHost, st));
    SUNSET_CUDA(H, cudaStreamSynchronize(st));
    SUNSET_CUDA(H, cudaGetLastError());
    H->has_mirrors = hm != 0;
    for (void *p : {(void *)cid, (void *)cid2, (void *)pid, (void *)pid2, (void *)cstart, (void *)cend, (void *)count,
                    (void *)cnt64, (void *)rowptr, (void *)opt, (void *)or2, (void *)mflag})
        dfree(H, p);
    return 0;
}

}  // namespace sunset

// ---------------------------------------------------------------------------------------
// Halo lists of the staged stencil kernels.  A thread block owns kTileSlices consecutive
// slices (kTile nodes); its halo is the sorted set of parents its links reach.  The
// kernels load the halo's fields once into shared memory (consecutive halo entries are
// mostly consecutive nodes in Morton order, so these loads coalesce) and every link then
// reads shared memory through a 16-bit position.  Built on the host once per node set.
// ---------------------------------------------------------------------------------------
#include <algorithm>
#include <thread>

namespace sunset {

// Boundary framework data in internal order: normals, FD parents, the boundary list in
// the reference's order (setup_domain.F90:314-327 builds it in node order) with each
// boundary node's four FD rows (the reader places them right after their parent), and the
// boundary index of each node.  Inputs are in the reference's node order.
int upload_boundary(Handle *H, const std::vector<double> &nx, const std::vector<double> &ny,
                    const std::vector<int> &fdpar_ref, const std::vector<int> &blist_ref,
                    const std::vector<int> &type) {
    const int n = H->npfb, nb = (int)blist_ref.size();
    const std::vector<int> &perm = H->h_perm, &iperm = H->h_iperm;
    std::vector<double> inx(n), iny(n);
    std::vector<int> ifd(n), ibidx(n, -1), ibl(nb), ibrow(4 * (size_t)(nb ? nb : 1), 0);
    for (int i = 0; i < n; i++) {
        const int r = perm[i];
        inx[i] = nx[r];
        iny[i] = ny[r];
        ifd[i] = fdpar_ref[r] >= 0 ? iperm[fdpar_ref[r]] : -1;
    }
    H->h_btype.resize(nb);
    for (int jj = 0; jj < nb; jj++) {
        const int r = blist_ref[jj];
        ibl[jj] = iperm[r];
        ibidx[iperm[r]] = jj;
        H->h_btype[jj] = type[r];
        for (int j = 1; j <= 4; j++) ibrow[4 * jj + j - 1] = iperm[r + j];
    }
    if (dalloc(H, &H->rnx, n) || dalloc(H, &H->rny, n) || dalloc(H, &H->fdpar, n) || dalloc(H, &H->bidx, n) ||
        dalloc(H, &H->blist, nb ? nb : 1) || dalloc(H, &H->brow, 4 * (size_t)(nb ? nb : 1)))
        return SUNSET_ERR_NOMEM;
    cudaStream_t st = H->stream;
    SUNSET_CUDA(H, cudaMemcpyAsync(H->rnx, inx.data(), n * sizeof(double), cudaMemcpyHostToDevice, st));
    SUNSET_CUDA(H, cudaMemcpyAsync(H->rny, iny.data(), n * sizeof(double), cudaMemcpyHostToDevice, st));
    SUNSET_CUDA(H, cudaMemcpyAsync(H->fdpar, ifd.data(), n * sizeof(int), cudaMemcpyHostToDevice, st));
    SUNSET_CUDA(H, cudaMemcpyAsync(H->bidx, ibidx.data(), n * sizeof(int), cudaMemcpyHostToDevice, st));
    if (nb) {
        SUNSET_CUDA(H, cudaMemcpyAsync(H->blist, ibl.data(), nb * sizeof(int), cudaMemcpyHostToDevice, st));
        SUNSET_CUDA(H, cudaMemcpyAsync(H->brow, ibrow.data(), 4 * (size_t)nb * sizeof(int), cudaMemcpyHostToDevice, st));
    }
    SUNSET_CUDA(H, cudaStreamSynchronize(st));
    return 0;
}

int build_halos(Handle *H) {
    const int n = H->npfb, nsl = H->nslices;
    const long long L = H->nlinks_sell;
    std::vector<int> lidx(L), cnt(n), sw(nsl);
    std::vector<long long> sptr(nsl + 1);
    SUNSET_CUDA(H, cudaMemcpy(lidx.data(), H->lidx, L * sizeof(int), cudaMemcpyDeviceToHost));
    SUNSET_CUDA(H, cudaMemcpy(cnt.data(), H->cnt, n * sizeof(int), cudaMemcpyDeviceToHost));
    SUNSET_CUDA(H, cudaMemcpy(sw.data(), H->slice_w, nsl * sizeof(int), cudaMemcpyDeviceToHost));
    SUNSET_CUDA(H, cudaMemcpy(sptr.data(), H->slice_ptr, (nsl + 1) * sizeof(long long), cudaMemcpyDeviceToHost));
    const int nt = (nsl + kTileSlices - 1) / kTileSlices;
    std::vector<std::vector<int>> halos(nt);
    std::vector<uint16_t> loc(L, 0);
    unsigned nthr = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
    std::vector<std::thread> pool;
    for (unsigned w = 0; w < nthr; w++) {
        pool.emplace_back([&, w]() {
            for (int t = (int)w; t < nt; t += (int)nthr) {
                std::vector<int> &hv = halos[t];
                for (int sl = t * kTileSlices; sl < std::min(nsl, (t + 1) * kTileSlices); sl++)
                    for (int lane = 0; lane < kSlice; lane++) {
                        int i = sl * kSlice + lane;
                        if (i >= n) break;
                        for (int k = 0; k < cnt[i]; k++) hv.push_back(lidx[sell_at(sptr[sl], k, lane)] & kLinkMask);
                    }
                std::sort(hv.begin(), hv.end());
                hv.erase(std::unique(hv.begin(), hv.end()), hv.end());
                for (int sl = t * kTileSlices; sl < std::min(nsl, (t + 1) * kTileSlices); sl++)
                    for (int lane = 0; lane < kSlice; lane++) {
                        int i = sl * kSlice + lane;
                        int c = i < n ? cnt[i] : 0;
                        for (int k = 0; k < sw[sl]; k++) {
                            long long o = sell_at(sptr[sl], k, lane);
                            if (k >= c) { loc[o] = 0; continue; }
                            int p = lidx[o] & kLinkMask, code = (unsigned)lidx[o] >> 30;
                            int pos = (int)(std::lower_bound(hv.begin(), hv.end(), p) - hv.begin());
                            loc[o] = (uint16_t)(pos | (code << 14));
                        }
                    }
            }
        });
    }
    for (auto &th : pool) th.join();
    std::vector<int> hptr(nt + 1);
    hptr[0] = 0;
    int hmax = 0;
    for (int t = 0; t < nt; t++) {
        hptr[t + 1] = hptr[t] + (int)halos[t].size();
        hmax = std::max(hmax, (int)halos[t].size());
    }
    if (hmax > kLocMask + 1) return set_err(H, SUNSET_ERR_SCOPE, "tile halo of %d nodes exceeds the 14-bit local index", hmax);
    std::vector<int> hall(hptr[nt]);
    for (int t = 0; t < nt; t++) std::copy(halos[t].begin(), halos[t].end(), hall.begin() + hptr[t]);
    if (dalloc(H, &H->halo_ptr, nt + 1) || dalloc(H, &H->halo, hall.size()) || dalloc(H, &H->lloc, L))
        return SUNSET_ERR_NOMEM;
    SUNSET_CUDA(H, cudaMemcpy(H->halo_ptr, hptr.data(), hptr.size() * sizeof(int), cudaMemcpyHostToDevice));
    SUNSET_CUDA(H, cudaMemcpy(H->halo, hall.data(), hall.size() * sizeof(int), cudaMemcpyHostToDevice));
    SUNSET_CUDA(H, cudaMemcpy(H->lloc, loc.data(), L * sizeof(uint16_t), cudaMemcpyHostToDevice));
    H->ntiles = nt;
    H->halo_max = hmax;
    return 0;
}

}  // namespace sunset
