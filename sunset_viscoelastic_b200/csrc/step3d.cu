// step3d.cu -- the 3-D (-Ddim3) time step of the direct, Cholesky, log-conformation (sPTT) and
// Newtonian forms on node sets with or without boundary nodes (walls, inflow, outflow).
//
// The 3-D node set is nz copies of the 2-D one in z (build_3rd_dimension,
// setup_domain.F90:435-547), layer-major in the reference (node iz*nl + i at z = iz*dz).  On the
// device the layers are innermost: node (i, iz) sits at i*nz + iz, so a warp covers the layers of
// one node (or a few): the node's links and weights are the same in every lane (one broadcast
// load a link), its neighbours' values are contiguous (coalesced), and the z stencil reads
// adjacent entries.  The C-ABI converts to and from the reference order.  The reference builds
// the neighbour lists per layer from identical positions (neighbours.F90:180-183,223-233), so
// every layer uses the layer's lists and LABFM weights (built once, 2-D); only the state is
// 3-D.  z-derivatives are the periodic central differences of fd.F90 (ij_count_fd = forder+1
// points) over the same node in the neighbouring layers.  Mirror images take their parent's
// value in the same layer, u and v with the mirror's sign, w, c_xz and c_yz unchanged
// (mirror_boundaries.F90:302-303,324-341).
//
// Structure: one kernel a stage (k3_stage), as calc_all_rhs and the RK update: each node-layer
// gathers every derivative of every field (x-y LABFM sums in the reference's link order, then
// the z stencils) into its block's shared memory, then computes the right-hand side and the RK
// update from there, so the derivatives never cross HBM; the filter as the x-y filter
// followed by the z filter of its result (derivatives.F90:387-405); the mass correction and
// the derived fields; all FP64.
//
// Boundary nodes: build_3rd_dimension copies node_type and the normals to every layer
// (setup_domain.F90:487-532).  A boundary node's x-y operators are its boundary weights (on
// walls d/dn and d/dt; on inflow and outflow nodes d/dx and d/dy), so the gather is unchanged,
// except that the conformation Laplacian there takes the tangential second-derivative weights
// (calc_laplacian_transverse_only_on_bound, derivatives.F90:306-358).  The boundary branches of
// the right-hand sides run in point3_body<FORM, true>, and apply_time_dependent_bounds after
// each stage and after the filter holds rho u, rho v, rho w at zero on walls and prescribes a
// hard inflow's momentum, with u_inflow_local on its ramp.
#include <cstring>

#include "internal.cuh"
#include "physics.cuh"

namespace sunset {

namespace {

constexpr int kMaxFd = 13;
constexpr int kG3 = 57;  // derivative slots, see enum G3

struct Layer3 {
    int nl, nz, ncfd;
    int nzc;  // > 0: blocks of (warps) nodes x 32 layers, nzc chunks of layers a node (zthread)
    const long long *slice_ptr;
    const int *cnt, *cnt_small, *lidx;
    const double *wx, *wy, *wl, *wh, *gsx, *gsy, *lsum, *hsum;
    const double *wlc, *lsumc;  // with boundary nodes: the conformation Laplacian's weights and sums
    double fdg[kMaxFd], fdl[kMaxFd], fdh[kMaxFd];
};

// derivative arrays (each nl*nz)
enum G3 {
    ROX, ROY, ROZ, UX, UY, UZ, VX, VY, VZ, WX, WY, WZ, LU, LV, LW,
    CG0 = 15,  // c grads (Cholesky: psi grads): CG0 + 3*q + d, q = xx xy yy xz yz zz, d = x y z
    LC0 = 33,  // c Laplacians: LC0 + q
    PG0 = 39   // log-conformation: psi grads, PG0 + 3*q + d
};

// sign class of a field at a mirror image: 0 none, 1 like u (x mirrors), 2 like v (y
// mirrors), 3 like c_xy (one of the two); code = vrelation - 1 (1 x, 2 y, 3 both)
__device__ __forceinline__ double mirror_value(double x, int cls, int code) {
    const bool flip = (cls == 1 && (code == 1 || code == 3)) || (cls == 2 && (code == 2 || code == 3)) ||
                      (cls == 3 && (code == 1 || code == 2));
    return flip ? -x : x;
}

// layer l = iz + m - ncfd/2 of the m-th point of the periodic z stencil (fd.F90:62-66); the
// offset is below nz in magnitude (layers_set keeps nz >= ncfd/2 + 2), so one wrap suffices
__device__ __forceinline__ int zwrap(int l, int nz) {
    l += (l < 0) ? nz : 0;
    return (l >= nz) ? l - nz : l;
}

// thread k of the node-major layered arrays: node i, layer iz (n < 2^31, checked in layers_set).
// With 32 layers or more, a block takes one chunk of 32 layers of consecutive nodes, one node a
// warp: the warp keeps its broadcast link loads and coalesced layer reads, and the block's
// nodes, neighbours in the Morton order, share most of their neighbours' values in L1.
// Otherwise the threads run over the node-layers in order.
struct ZThread {
    int k, i, iz;
};
__device__ __forceinline__ bool zthread(const Layer3 &L, ZThread &t) {
    if (L.nzc > 0) {
        const int grp = (int)blockIdx.x / L.nzc, zc = (int)blockIdx.x - grp * L.nzc;
        const int i = grp * (int)(blockDim.x >> 5) + (int)(threadIdx.x >> 5), iz = zc * 32 + (int)(threadIdx.x & 31);
        if (i >= L.nl || iz >= L.nz) return false;
        t.i = i;
        t.iz = iz;
        t.k = i * L.nz + iz;
        return true;
    }
    const unsigned k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= (unsigned)L.nl * (unsigned)L.nz) return false;
    t.k = (int)k;
    t.i = (int)(k / (unsigned)L.nz);
    t.iz = (int)k - t.i * L.nz;
    return true;
}

// the 19 state fields (ro rou rov row u v w cxx cxy cyy cxz cyz czz psi(6)); slot 19 holds the
// FENE-P function of the direct form where the gather reads it
struct Fields3 {
    double *p[20];
};

// What one pass over a node's links gathers: per field, the G slots of its x-y sums (and z
// stencil) and of its Laplacian (-1: not needed).
struct FDesc {
    int f, cls, gx, gy, gl, gz;
};
template <int FORM, bool MD>
__host__ __device__ constexpr int ndesc() {
    return FORM == SUNSET_FORM_NEWT ? 4 : FORM == SUNSET_FORM_DI ? 10 : FORM == SUNSET_FORM_CHL ? (MD ? 16 : 10) : 16;
}
template <int FORM, bool MD, bool FULL>
__host__ __device__ constexpr FDesc desc3(int d) {
    if (d == 0) return FDesc{0, 0, ROX, ROY, -1, ROZ};
    if (d == 1) return FDesc{4, 1, UX, UY, LU, UZ};
    if (d == 2) return FDesc{5, 2, VX, VY, LV, VZ};
    if (d == 3) return FDesc{6, 0, WX, WY, LW, WZ};
    const int q = (d - 4) % 6, cls = q == 1 ? 3 : 0;
    const bool hx = q == 0 || q == 1 || q == 3 || q == 4, hy = q == 1 || q == 2 || q == 3 || q == 4;
    const bool hz = q == 1 || q == 3 || q == 4 || q == 5;
    if (FORM == SUNSET_FORM_DI)  // rhs_di.F90:186-194 (c_xx x, c_yy y, c_zz z only, unless full)
        return FDesc{7 + q, cls, (FULL || hx) ? CG0 + 3 * q : -1, (FULL || hy) ? CG0 + 3 * q + 1 : -1, MD ? LC0 + q : -1,
                     (FULL || hz) ? CG0 + 3 * q + 2 : -1};
    if (FORM == SUNSET_FORM_CHL) {  // rhs.F90:186-201: full psi gradients; Laplacians of c
        if (d < 10) return FDesc{13 + q, cls, CG0 + 3 * q, CG0 + 3 * q + 1, -1, CG0 + 3 * q + 2};
        return FDesc{7 + q, cls, -1, -1, LC0 + q, -1};
    }
    // log-conformation, rhs_lc.F90:184-193 (c, momentum) and :397-409 (psi, advection)
    if (d < 10) return FDesc{7 + q, cls, hx ? CG0 + 3 * q : -1, hy ? CG0 + 3 * q + 1 : -1, -1, hz ? CG0 + 3 * q + 2 : -1};
    return FDesc{13 + q, cls, PG0 + 3 * q, PG0 + 3 * q + 1, -1, PG0 + 3 * q + 2};
}

// the gathered fields of a pass; with FEN (FENE-P, direct form) one more, the function
// f = (L^2 - 3)/(L^2 - tr c) of slot 19, whose gradient goes to the slots PG0.. the direct form
// leaves free (rhs_di.F90:198-205)
template <int FORM, bool MD, bool FEN>
__host__ __device__ constexpr int ndesc3() { return ndesc<FORM, MD>() + (FEN ? 1 : 0); }
template <int FORM, bool MD, bool FULL, bool FEN>
__host__ __device__ constexpr FDesc desc3f(int d) {
    return (FEN && d == ndesc<FORM, MD>()) ? FDesc{19, 0, PG0, PG0 + 1, -1, PG0 + 2} : desc3<FORM, MD, FULL>(d);
}

// Every derivative the right-hand side reads, in one pass over each node's links: the x-y
// LABFM sums of all fields (in the reference's link order, each sum as calc_gradient /
// calc_laplacian forms it), then the z stencils.  The layers of a node share its links, so a
// warp's link and weight loads are one broadcast each.  The links go in pairs whose field
// values are all loaded before either is summed, so that a warp keeps two links' gathers in
// flight (the sums still run in link order).
// Minimum resident blocks a SM asked of the compiler: the direct form's gather runs fastest at
// 5 (96 registers); the forms with 16 gathered fields lose their loads in flight at that size
// and run at 4 (128 registers).
#ifndef SUNSET_3D_BLOCKS_DI
#define SUNSET_3D_BLOCKS_DI 5
#endif
#ifndef SUNSET_3D_BLOCKS
#define SUNSET_3D_BLOCKS 4
#endif
__host__ __device__ constexpr int derivs_min_blocks(int form) {
    return form == SUNSET_FORM_DI ? SUNSET_3D_BLOCKS_DI : SUNSET_3D_BLOCKS;
}

//
// ST(slot, value) receives each derivative: a global array of the standalone gather, or the
// fused stage kernel's shared memory.
// BND: the node set has boundary nodes, whose conformation Laplacians (fields 7-12) take the
// weights wlc and sums lsumc.
template <int FORM, bool MD, bool FULL, bool FEN, bool BND, class ST>
__device__ __forceinline__ void derivs3_body(const Layer3 &L, const Fields3 &F, const ZThread &z, ST store) {
    constexpr int N = ndesc3<FORM, MD, FEN>();
    constexpr int LB = 2;
    constexpr bool kCL = BND && MD;
    const int k = z.k, i = z.i, iz = z.iz, row = i * L.nz, h = L.ncfd / 2;
    double sx[N], sy[N], sl[N];
#pragma unroll
    for (int d = 0; d < N; d++) { sx[d] = 0.0; sy[d] = 0.0; sl[d] = 0.0; }
    const long long base = L.slice_ptr[i >> 5];
    const int cs = L.cnt_small[i];
    int q = 0;
    for (; q + LB <= cs; q += LB) {
        int pj[LB], code[LB];
        double wx[LB], wy[LB], wl[LB], wc[LB], v[LB][N];
#pragma unroll
        for (int b = 0; b < LB; b++) {
            const long long o = sell_at(base, q + b, i & 31);
            const int l = __ldg(L.lidx + o);
            pj[b] = (l & kLinkMask) * L.nz + iz;
            code[b] = (int)((unsigned)l >> 30);
            wx[b] = __ldg(L.wx + o);
            wy[b] = __ldg(L.wy + o);
            wl[b] = __ldg(L.wl + o);
            wc[b] = kCL ? __ldg(L.wlc + o) : 0.0;
        }
#pragma unroll
        for (int b = 0; b < LB; b++)
#pragma unroll
            for (int d = 0; d < N; d++) v[b][d] = F.p[desc3f<FORM, MD, FULL, FEN>(d).f][pj[b]];
#pragma unroll
        for (int b = 0; b < LB; b++)
#pragma unroll
            for (int d = 0; d < N; d++) {
                const FDesc D = desc3f<FORM, MD, FULL, FEN>(d);
                const double x = mirror_value(v[b][d], D.cls, code[b]);
                if (D.gx >= 0) sx[d] = sx[d] + x * wx[b];
                if (D.gy >= 0) sy[d] = sy[d] + x * wy[b];
                if (D.gl >= 0) sl[d] = sl[d] + x * ((kCL && D.f >= 7) ? wc[b] : wl[b]);
            }
    }
    for (; q < cs; q++) {
        const long long o = sell_at(base, q, i & 31);
        const int l = __ldg(L.lidx + o);
        const int pj = (l & kLinkMask) * L.nz + iz;
        const int code = (int)((unsigned)l >> 30);
        const double wx = __ldg(L.wx + o), wy = __ldg(L.wy + o), wl = __ldg(L.wl + o);
        const double wc = kCL ? __ldg(L.wlc + o) : 0.0;
#pragma unroll
        for (int d = 0; d < N; d++) {
            const FDesc D = desc3f<FORM, MD, FULL, FEN>(d);
            const double x = mirror_value(F.p[D.f][pj], D.cls, code);
            if (D.gx >= 0) sx[d] = sx[d] + x * wx;
            if (D.gy >= 0) sy[d] = sy[d] + x * wy;
            if (D.gl >= 0) sl[d] = sl[d] + x * ((kCL && D.f >= 7) ? wc : wl);
        }
    }
    // the x-y sums in sum form; the Laplacians keep theirs for the z part
#pragma unroll
    for (int d = 0; d < N; d++) {
        const FDesc D = desc3f<FORM, MD, FULL, FEN>(d);
        const double p = F.p[D.f][k];
        if (D.gx >= 0) store(D.gx, sx[d] - p * L.gsx[i]);
        if (D.gy >= 0) store(D.gy, sy[d] - p * L.gsy[i]);
        if (D.gl >= 0) sl[d] = sl[d] - p * ((kCL && D.f >= 7) ? L.lsumc[i] : L.lsum[i]);
    }
    // the z stencils, point by point over all fields (each field's sums still run in point
    // order); a fixed trip count with the points past ncfd cut off, so that the loads of several
    // points can be in flight together
    double tg[N], tl[N];
#pragma unroll
    for (int d = 0; d < N; d++) { tg[d] = 0.0; tl[d] = 0.0; }
#pragma unroll
    for (int m = 0; m < kMaxFd; m++) {
        if (m >= L.ncfd) break;
        const int r = row + zwrap(iz + m - h, L.nz);
        const double cg = L.fdg[m], cl = L.fdl[m];
#pragma unroll
        for (int d = 0; d < N; d++) {
            const FDesc D = desc3f<FORM, MD, FULL, FEN>(d);
            if (D.gl < 0 && D.gz < 0) continue;
            const double fm = F.p[D.f][r];
            if (D.gl >= 0) tl[d] = tl[d] + fm * cl;
            if (D.gz >= 0) tg[d] = tg[d] + fm * cg;
        }
    }
#pragma unroll
    for (int d = 0; d < N; d++) {
        const FDesc D = desc3f<FORM, MD, FULL, FEN>(d);
        if (D.gl >= 0) store(D.gl, sl[d] + tl[d]);
        if (D.gz >= 0) store(D.gz, tg[d]);
    }
}

// The derivative slots a form's gather writes, numbered compactly (-1: not written; the
// right-hand side then reads zero, as from the zeroed global arrays).
template <int FORM, bool MD, bool FULL, bool FEN>
__host__ __device__ constexpr int gslot(int slot) {
    int idx = 0;
    for (int s2 = 0; s2 < kG3; s2++) {
        bool used = false;
        for (int d = 0; d < ndesc3<FORM, MD, FEN>(); d++) {
            const FDesc D = desc3f<FORM, MD, FULL, FEN>(d);
            if (D.gx == s2 || D.gy == s2 || D.gl == s2 || D.gz == s2) used = true;
        }
        if (s2 == slot) return used ? idx : -1;
        if (used) idx++;
    }
    return -1;
}
template <int FORM, bool MD, bool FULL, bool FEN>
__host__ __device__ constexpr int ngslots() {
    int c = 0;
    for (int s2 = 0; s2 < kG3; s2++) c += gslot<FORM, MD, FULL, FEN>(s2) >= 0 ? 1 : 0;
    return c;
}
// gslot as a table in constant memory, built at compile time: a slot index the compiler folds
// is an immediate constant operand, one it cannot fold a single constant-bank load instead of
// gslot's loops
struct GTable {
    signed char idx[kG3];
};
template <int FORM, bool MD, bool FULL, bool FEN>
__host__ __device__ constexpr GTable make_gtable() {
    GTable t{};
    for (int a = 0; a < kG3; a++) t.idx[a] = (signed char)gslot<FORM, MD, FULL, FEN>(a);
    return t;
}
template <int FORM, bool MD, bool FULL, bool FEN>
__constant__ GTable kGTable = make_gtable<FORM, MD, FULL, FEN>();

// calc_filtered_var in 3-D for the NF evolved fields (ro, rou, rov, row, then the six c or psi
// variables) in one pass over each node's links: the x-y filter of every field into its
// scratch array ...
struct Filter3 {
    double *f[10];  // the fields, filtered in place
    double *t[10];  // x-y filtered values
};
// sign class at mirrors of the filtered fields: rou like u, rov like v, c_xy / psi_xy like c_xy
__host__ __device__ constexpr int filter_cls(int q) { return q == 1 ? 1 : q == 2 ? 2 : q == 5 ? 3 : 0; }

template <int NF>
__global__ void __launch_bounds__(128) k3_filter_xy(Layer3 L, Filter3 A) {
    ZThread z;
    if (!zthread(L, z)) return;
    const int k = z.k, i = z.i, iz = z.iz;
    const long long base = L.slice_ptr[i >> 5];
    double t[NF];
#pragma unroll
    for (int q = 0; q < NF; q++) t[q] = 0.0;
    const int c = L.cnt[i];
#pragma unroll 4
    for (int m = 0; m < c; m++) {
        const long long o = sell_at(base, m, i & 31);
        const int l = __ldg(L.lidx + o);
        const int pj = (l & kLinkMask) * L.nz + iz;
        const int code = (int)((unsigned)l >> 30);
        const double w = __ldg(L.wh + o);
#pragma unroll
        for (int q = 0; q < NF; q++) t[q] = t[q] + mirror_value(A.f[q][pj], filter_cls(q), code) * w;
    }
    // the own values loaded before the first store (the arrays are not known to be distinct)
    const double hs = L.hsum[i];
    double p[NF];
#pragma unroll
    for (int q = 0; q < NF; q++) p[q] = A.f[q][k];
#pragma unroll
    for (int q = 0; q < NF; q++) A.t[q][k] = p[q] + (t[q] - p[q] * hs);
}
// ... then the z filter of that result (back into the field)
template <int NF>
__global__ void __launch_bounds__(128) k3_filter_z(Layer3 L, Filter3 A) {
    ZThread z;
    if (!zthread(L, z)) return;
    const int k = z.k, iz = z.iz, row = z.i * L.nz, h = L.ncfd / 2;
    double t[NF], own[NF];
#pragma unroll
    for (int q = 0; q < NF; q++) { t[q] = 0.0; own[q] = A.t[q][k]; }
#pragma unroll
    for (int m = 0; m < kMaxFd; m++) {
        if (m >= L.ncfd) break;
        const int r = row + zwrap(iz + m - h, L.nz);
        const double c = L.fdh[m];
#pragma unroll
        for (int q = 0; q < NF; q++) t[q] = t[q] + A.t[q][r] * c;
    }
#pragma unroll
    for (int q = 0; q < NF; q++) A.f[q][k] = own[q] + t[q];
}

struct Point3 {
    StepConsts K;
    int nl, nz, di, full, md;
    const double *py;                     // node ordinate (Kolmogorov forcing)
    // boundary nodes: node types, normals into the fluid, boundary index and FD rows, spacing;
    // u_inflow_local of every node-layer
    const int *ntype, *bidx, *brow;
    const double *rnx, *rny, *sp;
    double *uin;
    double *alpha;  // stage 3: each node-layer's step error (alpha_out, step.F90:456-458)
    const double *fen;                    // FENE-P function of the direct form, or null
    int chl, lc;
    const double *in[19];                 // ro rou rov row u v w cxx cxy cyy cxz cyz czz psi(6)
    double *out[19];
    double *reg[10], *eacc[10], *rhs[10];
    DevScalars *sc;
    int stage;                            // 0..3, 4 = right-hand side only
};

__device__ __forceinline__ unsigned long long dbits(double x) { return (unsigned long long)__double_as_longlong(x); }

// eigens (3x3 symmetric), conf_transforms.F90:218-397: closed-form eigenvalues (trigonometric
// solution of the characteristic cubic), eigenvectors by cross products and a 2x2 rotation.
// R column-major, R[i + 3j] = R(i+1, j+1); its columns are the eigenvectors of L[0..2].
__device__ void eigens3(double axx, double axy, double ayy, double axz, double ayz, double azz, double *L, double *R) {
    const double onethird = 1.0 / 3.0, twothirds = 2.0 / 3.0, eps = 2.220446049250313e-16, pi = 3.141592653589793;
    double a[9];
    a[0] = axx; a[3] = axy; a[6] = axz;
    a[1] = axy; a[4] = ayy; a[7] = ayz;
    a[2] = axz; a[5] = ayz; a[8] = azz;
    const double p1 = (axy * axy + axz * axz) + ayz * ayz;
    if (p1 <= 1.0e-16) {
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
    if (n2 > norm) { ic = 2; norm = n1; }  // (the reference keeps n1 here)
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
// C = A B, 3x3 column-major, matmul's sum in k order
__device__ __forceinline__ void mm3(const double *A, const double *B, double *C) {
    double t[9];
#pragma unroll
    for (int j = 0; j < 3; j++)
#pragma unroll
        for (int i = 0; i < 3; i++) t[i + 3 * j] = (A[i] * B[3 * j] + A[i + 3] * B[1 + 3 * j]) + A[i + 6] * B[2 + 3 * j];
#pragma unroll
    for (int k = 0; k < 9; k++) C[k] = t[k];
}
__device__ __forceinline__ void tr3(const double *A, double *T) {
#pragma unroll
    for (int j = 0; j < 3; j++)
#pragma unroll
        for (int i = 0; i < 3; i++) T[i + 3 * j] = A[j + 3 * i];
}
// log_conf_c_from_psi / log_conf_psi_from_c in 3-D (conf_transforms.F90:127-215): R f(Lambda) R^T
// with f = exp or log; in/out xx xy yy xz yz zz
__device__ void lc3_transform(const double *in, double *out, bool to_c) {
    double L[3], R[9], RT[9], Lm[9], M[9];
    eigens3(in[0], in[1], in[2], in[3], in[4], in[5], L, R);
    tr3(R, RT);
    for (int k = 0; k < 9; k++) Lm[k] = 0.0;
    for (int k = 0; k < 3; k++) Lm[4 * k] = to_c ? exp(L[k]) : log(L[k]);
    mm3(Lm, RT, M);
    mm3(R, M, M);
    out[0] = M[0]; out[1] = M[1]; out[2] = M[4]; out[3] = M[6]; out[4] = M[7]; out[5] = M[8];
}

// cholesky_c_from_psi / cholesky_psi_from_c in 3-D (conf_transforms.F90:28-125): sPTT, or
// with L2 > 0 (FENE-P, :39-58 and :89-106) the factors of J = f c, f = (L^2 - 3)/(L^2 - tr c),
// with c = J L^2 / (L^2 - 3 + tr J)
__device__ __forceinline__ void chl3_c_from_psi(const double *p, double *c, double L2 = 0.0) {
    if (L2 > 0.0) {
        const double Jxx = exp(2.0 * p[0]), Jxy = exp(p[0]) * p[1], Jyy = p[1] * p[1] + exp(2.0 * p[2]);
        const double Jzz = (exp(2.0 * p[5]) + p[3] * p[3]) + p[4] * p[4];
        const double fq = L2 / ((((L2 - 3.0) + Jxx) + Jyy) + Jzz);
        c[0] = Jxx * fq; c[1] = Jxy * fq; c[2] = Jyy * fq; c[5] = Jzz * fq;
        const double Jxz = exp(p[0]) * p[3], Jyz = p[1] * p[3] + exp(p[2]) * p[4];
        c[3] = Jxz * fq; c[4] = Jyz * fq;
        return;
    }
    const double e = exp(p[0]);
    c[0] = e * e;
    c[1] = exp(p[0]) * p[1];
    c[2] = p[1] * p[1] + exp(2.0 * p[2]);
    c[3] = exp(p[0]) * p[3];
    c[4] = p[1] * p[3] + exp(p[2]) * p[4];
    c[5] = (exp(2.0 * p[5]) + p[3] * p[3]) + p[4] * p[4];
}
__device__ __forceinline__ void chl3_psi_from_c(const double *c, double *p, double L2 = 0.0) {
    double J[6];
    const double fr = L2 > 0.0 ? (L2 - 3.0) / (L2 - ((c[0] + c[2]) + c[5])) : 1.0;
    for (int q = 0; q < 6; q++) J[q] = L2 > 0.0 ? c[q] * fr : c[q];
    const double xx = sqrt(J[0]);
    const double xy = J[1] / (xx);
    const double yy = (sqrt(J[2] - xy * xy));
    const double xz = J[3] / xx;
    const double yz = (J[4] - xy * xz) / yy;
    const double zz = sqrt((J[5] - xz * xz) - yz * yz);
    p[0] = log(xx); p[1] = xy; p[2] = log(yy); p[3] = xz; p[4] = yz; p[5] = log(zz);
}
// filter_variables under FENE-P in 3-D, rhs.F90:816-834: the factors of J to those of c for the
// filter; :853-868 back after it (to_c false)
__device__ __forceinline__ void chl3_fenep_factor(double L2, double *p, bool to_c) {
    const double trJ = ((((exp(2.0 * p[0]) + p[1] * p[1]) + exp(2.0 * p[2])) + p[3] * p[3]) + p[4] * p[4]) + exp(2.0 * p[5]);
    double fr;
    if (to_c) {
        fr = (L2 * trJ) / ((L2 - 3.0) + trJ);
        fr = (L2 - 3.0) / (L2 - fr);
        p[0] = p[0] - log(sqrt(fr));
        p[1] = p[1] / sqrt(fr);
        p[2] = p[2] - log(sqrt(fr));
        p[5] = p[5] - log(sqrt(fr));
        p[3] = p[3] / sqrt(fr);
        p[4] = p[4] / sqrt(fr);
    } else {
        fr = (L2 - 3.0) / (L2 - trJ);
        p[0] = p[0] + log(sqrt(fr));
        p[1] = p[1] * sqrt(fr);
        p[2] = p[2] + log(sqrt(fr));
        p[5] = p[5] + log(sqrt(fr));
        p[3] = p[3] * sqrt(fr);
        p[4] = p[4] * sqrt(fr);
    }
}

// calc_rhs_ro, calc_rhs_rovel and calc_rhs_c with the dim3 terms (rhs_di.F90:119-139,
// 215-275, 415-476), then the stage's RK update (step.F90:285-343, 366-483).  BND: the node
// set has boundary nodes, whose node-layers take the wall or inflow/outflow branches.
//
// GET(slot) returns derivative `slot` of node-layer k (global arrays, or the fused kernel's
// shared memory); the bits of the node-layer's step error norm are returned (stage 3).
template <int FORM, bool BND, class GET>
__device__ __forceinline__ unsigned long long point3_body(const Point3 &P, size_t k, GET g) {
    constexpr bool kDi = FORM == SUNSET_FORM_DI, kChl = FORM == SUNSET_FORM_CHL, kLc = FORM == SUNSET_FORM_LC;
    unsigned long long eb = 0;
    {
        const StepConsts &K = P.K;
        const int i = (int)((unsigned)k / (unsigned)P.nz);
        const int ty = BND ? P.ntype[i] : 999;
        const bool wall = ty == 0, inout = ty == 1 || ty == 2;
        double uin = inout ? P.uin[k] : 0.0;
        const double ro = P.in[0][k], u = P.in[4][k], v = P.in[5][k], w = P.in[6][k];
        const double gpx = K.csq * g(ROX), gpy = K.csq * g(ROY), gpz = K.csq * g(ROZ);
        const double tmp = ((u * g(ROX) + v * g(ROY)) + w * g(ROZ));
        const double divv = (g(UX) + g(VY)) + g(WZ);
        const double rr = -ro * divv - tmp;
        const double tsu = ro * ((u * g(UX) + v * g(UY)) + w * g(UZ)) - u * rr;
        const double tsv = ro * ((u * g(VX) + v * g(VY)) + w * g(VZ)) - v * rr;
        const double tsw = ro * ((u * g(WX) + v * g(WY)) + w * g(WZ)) - w * rr;
        double fvu = K.coef_solvent * g(LU), fvv = K.coef_solvent * g(LV), fvw = K.coef_solvent * g(LW);
        auto gp = [&](int q, int d) { return g(CG0 + 3 * q + d); };  // Cholesky: psi gradients
        if (kChl) {  // grad c from grad psi, rhs.F90:245-262
            const double pxx = P.in[13][k], pxy = P.in[14][k], pyy = P.in[15][k], pxz = P.in[16][k], pyz = P.in[17][k],
                         pzz = P.in[18][k];
            const double gcxx1 = (2.0 * exp(2.0 * pxx)) * gp(0, 0);
            const double gcxy1 = exp(pxx) * gp(1, 0) + (pxy * exp(pxx)) * gp(0, 0);
            const double gcxy2 = exp(pxx) * gp(1, 1) + (pxy * exp(pxx)) * gp(0, 1);
            const double gcyy2 = (2.0 * pxy) * gp(1, 1) + (2.0 * exp(2.0 * pyy)) * gp(2, 1);
            const double gcxz1 = exp(pxx) * gp(3, 0) + (pxz * exp(pxx)) * gp(0, 0);
            const double gcxz3 = exp(pxx) * gp(3, 2) + (pxz * exp(pxx)) * gp(0, 2);
            const double gcyz2 = (pxy * gp(3, 1) + pxz * gp(1, 1)) + exp(pyy) * (gp(4, 1) + pyz * gp(2, 1));
            const double gcyz3 = (pxy * gp(3, 2) + pxz * gp(1, 2)) + exp(pyy) * (gp(4, 2) + pyz * gp(2, 2));
            const double gczz3 = ((2.0 * exp(2.0 * pzz)) * gp(5, 2) + (2.0 * pxz) * gp(3, 2)) + (2.0 * pyz) * gp(4, 2);
            fvu = fvu + K.coef_polymeric * ((gcxx1 + gcxy2) + gcxz3);
            fvv = fvv + K.coef_polymeric * ((gcxy1 + gcyy2) + gcyz3);
            fvw = fvw + K.coef_polymeric * ((gcxz1 + gcyz2) + gczz3);
        }
        if (kDi && P.fen) {  // FENE-P, the quotient rule (rhs_di.F90:234-245)
            const double f1 = P.fen[k], g0 = g(PG0), g1 = g(PG0 + 1), g2 = g(PG0 + 2);
            const double cxx = P.in[7][k], cxy = P.in[8][k], cyy = P.in[9][k], cxz = P.in[10][k], cyz = P.in[11][k],
                         czz = P.in[12][k];
            fvu = fvu + K.coef_polymeric * (((((g(CG0 + 0) * f1 + cxx * g0) + g(CG0 + 3 + 1) * f1) + cxy * g1) +
                                             g(CG0 + 9 + 2) * f1) + cxz * g2);
            fvv = fvv + K.coef_polymeric * (((((g(CG0 + 3 + 0) * f1 + cxy * g0) + g(CG0 + 6 + 1) * f1) + cyy * g1) +
                                             g(CG0 + 12 + 2) * f1) + cyz * g2);
            fvw = fvw + K.coef_polymeric * (((((g(CG0 + 9 + 0) * f1 + cxz * g0) + g(CG0 + 12 + 1) * f1) + cyz * g1) +
                                             g(CG0 + 15 + 2) * f1) + czz * g2);
        } else if (kDi || kLc) {
            fvu = fvu + K.coef_polymeric * ((g(CG0 + 0) + g(CG0 + 3 + 1)) + g(CG0 + 9 + 2));
            fvv = fvv + K.coef_polymeric * ((g(CG0 + 3 + 0) + g(CG0 + 6 + 1)) + g(CG0 + 12 + 2));
            fvw = fvw + K.coef_polymeric * ((g(CG0 + 9 + 0) + g(CG0 + 12 + 1)) + g(CG0 + 15 + 2));
        }
        double bfu = ro * (K.grav0 + P.sc->df), bfv = ro * (K.grav1 + 0.0), bfw = ro * (0.0 + 0.0);
        if (K.kolmo)
            bfu = bfu + (((1.0 / K.Re) * cos(P.py[i])) * (1.0 + (K.Mdiff * K.beta) * K.Wi)) / (1.0 + K.Mdiff * K.Wi);
        double r[10];
        r[0] = rr;
        r[1] = ((-tsu - gpx) + bfu) + fvu;
        r[2] = ((-tsv - gpy) + bfv) + fvv;
        r[3] = ((-tsw - gpz) + bfw) + fvw;
        for (int q = 4; q < 10; q++) r[q] = 0.0;
        // the x-y velocity gradients; a wall node's are in its normal-tangent frame and turn to
        // x-y for the conformation equations (rhs_di.F90:497-517, rhs.F90:586-611,
        // rhs_lc.F90:602-627; d/dz is d/dz everywhere)
        double gux = g(UX), guy = g(UY), gvx = g(VX), gvy = g(VY), gwx = g(WX), gwy = g(WY);
        // the conformation Laplacian on a wall (and in the Cholesky form on every boundary
        // node) adds the one-sided normal second derivative over the node's four FD rows, the
        // next nodes of its layer (rhs_di.F90:553-568, rhs.F90:631-643)
        auto fdrows = [&](int q) {
            const int *rw = P.brow + 4 * P.bidx[i];
            const int iz = (int)k - i * P.nz;
            const double *c = P.in[7 + q];
            const double den = (((72.0 * P.sp[i]) * P.sp[i]) * K.L_char) * K.L_char;
            return (((((-415.0 * c[k]) + 576.0 * c[rw[0] * P.nz + iz]) - 216.0 * c[rw[1] * P.nz + iz]) +
                     64.0 * c[rw[2] * P.nz + iz]) - 9.0 * c[rw[3] * P.nz + iz]) / den;
        };
        if (wall) {
            const double xn = P.rnx[i], yn = P.rny[i];
            gux = xn * g(UX) - yn * g(UY);
            guy = yn * g(UX) + xn * g(UY);
            gvx = xn * g(VX) - yn * g(VY);
            gvy = yn * g(VX) + xn * g(VY);
            gwx = xn * g(WX) - yn * g(WY);
            gwy = yn * g(WX) + xn * g(WY);
            // calc_rhs_ro's wall branch (rhs_di.F90:149-154), the wall amplitudes of
            // calc_rhs_rovel (:291-307), the isothermal wall (characteristic_boundaries.F90:27-52:
            // L5 = L1) and the update of calc_rhs_nscbc (rhs_di.F90:601-665)
            const double c = sqrt(K.csq);
            const double un = u * xn + v * yn;
            const double dutdt = -yn * g(UY) + xn * g(VY);
            const double dundn = xn * g(UX) + yn * g(VX);
            const double dutdn = -yn * g(UX) + xn * g(VX);
            const double L1 = (0.5 * (un - c)) * (gpx - (ro * c) * dundn);
            const double L2 = un * (g(ROX) - (gpx / c) / c);
            const double L3 = un * dutdn;
            const double L4 = un * (g(WX) * xn + g(WY) * yn);
            const double L5 = L1;
            const double ts = ((((c * c) * L2 + L5) + L1) / c) / c;
            r[0] = (-ro * dutdt - ro * g(WZ)) - ts;
            r[1] = (0.0 - u * ts) - (L5 - L1) / c;
            r[2] = (0.0 - v * ts) - ro * L3;
            r[3] = (0.0 - w * ts) - ro * L4;
        } else if (inout) {
            // inflow (node_type 1) and outflow (2) in the x-y frame: calc_rhs_ro's in/out branch
            // (rhs_di.F90:155-157), the amplitudes and the transverse, viscous and body-force
            // terms of calc_rhs_rovel (:311-359; no Kolmogorov forcing), the closure of
            // characteristic_boundaries.F90 for the node's type (soft :54-80, hard :82-110,
            // inflow-outflow :112-150, outflow :152-189) and calc_rhs_nscbc (:601-665)
            const double c = sqrt(K.csq), p = K.csq * ro, nscbc = K.nscbc, Lx = K.Lx;
            const double rro = ((-v * g(ROY) - ro * g(VY)) - w * g(ROZ)) - ro * g(WZ);
            double L1 = (0.5 * (u - c)) * (gpx - (ro * c) * g(UX));
            double L2 = u * (g(ROX) - (gpx / c) / c);
            double L3 = u * g(VX);
            double L4 = u * g(WX);
            double L5 = (0.5 * (u + c)) * (gpx + (ro * c) * g(UX));
            const double bu = ro * (K.grav0 + P.sc->df), bv = ro * (K.grav1 + 0.0), bw = ro * (0.0 + 0.0);
            const double rou = ((-(v * g(UY)) - w * g(UZ)) + fvu) + bu;
            const double rov = (((-(v * g(VY)) - w * g(VZ)) - gpy) + fvv) + bv;
            const double row = (((-(v * g(WY)) - w * g(WZ)) - gpz) + fvw) + bw;
            if (ty == 1) {
                if (K.inflow_type == 1) {
                    L2 = 0.0; L3 = 0.0; L4 = 0.0; L5 = L1;
                } else if (K.inflow_type == 2) {
                    if (u > 0.0) {
                        L2 = 0.0;
                        L3 = ((v * nscbc) * c) / Lx;
                        L4 = ((w * nscbc) * c) / Lx;
                        L5 = ((((((u - uin) * nscbc) * (1.0 - u / c)) * c) * c) * 1.0) / Lx;
                    } else {
                        L2 = 0.0;
                        L5 = (((((p - K.p_in) * nscbc) * c) * 1.0) / 2.0) / Lx;
                    }
                } else {
                    L2 = 0.0;
                    L3 = (((((v * nscbc) * c) / Lx) - v * g(VY)) - w * g(VZ)) - gpy / ro;
                    L4 = ((w * nscbc) * c) / Lx + row;
                    L5 = (((((((u - uin) * nscbc) * (1.0 - u / c)) * c) * c) * 1.0) / Lx -
                          0.5 * (((v * gpy) + (p * g(VY))) + (((ro * c) * v) * g(UY)))) -
                         0.5 * (((w * gpz) + (p * g(WZ))) + (((ro * c) * w) * g(UZ)));
                }
            } else {
                if (u < c) L1 = (((((p - K.p_out) * nscbc) * c) * 1.0) / 2.0) / Lx;
                L2 = 0.0;
                if (u <= 0.0) { L2 = 0.0; L3 = 0.0; L4 = 0.0; }
            }
            const double ts = ((((c * c) * L2 + L5) + L1) / c) / c;
            r[0] = rro - ts;
            r[1] = (rou - u * ts) - (L5 - L1) / c;
            r[2] = (rov - v * ts) - ro * L3;
            r[3] = (row - w * ts) - ro * L4;
        }
        if (kChl) {  // calc_rhs_cholesky, rhs.F90:421-556 (sPTT, 3-D), walls :553-717
            const double ux = gux, uy = guy, uz = g(UZ), vx = gvx, vy = gvy, vz = g(VZ);
            const double wx = gwx, wy = gwy, wz = g(WZ);
            double ad[6];
            const double ua = ty == 1 ? 0.0 : u;  // inflow: no streamwise advection (rhs.F90:562-564)
#pragma unroll
            for (int q = 0; q < 6; q++) ad[q] = (ua * gp(q, 0) + v * gp(q, 1)) + w * gp(q, 2);
            const double lxx = exp(P.in[13][k]), lxy = P.in[14][k], lyy = exp(P.in[15][k]), lzz = exp(P.in[18][k]);
            const double lxz = P.in[16][k], lyz = P.in[17][k];
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
            const double cxx = P.in[7][k], cxy = P.in[8][k], cyy = P.in[9][k], cxz = P.in[10][k], cyz = P.in[11][k],
                         czz = P.in[12][k];
            const double Md = K.Mdiff;
            auto lc = [&](int q) {
                if (!P.md) return 0.0;
                const double x = g(LC0 + q);
                return (wall || inout) ? x + fdrows(q) : x;
            };
            double sxx, sxy, syy, sxz, syz, szz;
            if (K.fenep) {  // rhs.F90:204-209, 479-500: the factors of J = f c
                const double L2 = K.fenep_l2, la = K.lambda;
                const double fr = (L2 - 3.0) / (L2 - ((cxx + cyy) + czz));
                const double srctmp =
                    ((((((((((((2.0 * ux) * cxx + (2.0 * uy) * cxy) + (2.0 * vx) * cxy) + (2.0 * vy) * cyy) + (2.0 * uz) * cxz) +
                           (2.0 * vz) * cyz) + (2.0 * wx) * cxz) + (2.0 * wy) * cyz) + (2.0 * wz) * czz) -
                       (((fr * cxx + fr * cyy) + fr * czz) - 3.0) / la) +
                      Md * ((lc(0) + lc(2)) + lc(5))));
                const double den = ((L2 - cxx) - cyy) - czz;
                sxx = (-(fr / la) * (fr * cxx - 1.0) + (Md * fr) * lc(0)) + ((fr * cxx) * srctmp) / den;
                sxy = (-(fr / la) * (fr * cxy) + (Md * fr) * lc(1)) + ((fr * cxy) * srctmp) / den;
                syy = (-(fr / la) * (fr * cyy - 1.0) + (Md * fr) * lc(2)) + ((fr * cyy) * srctmp) / den;
                szz = (-(fr / la) * (fr * czz - 1.0) + (Md * fr) * lc(5)) + ((fr * czz) * srctmp) / den;
                sxz = (-(fr / la) * (fr * cxz) + (Md * fr) * lc(3)) + ((fr * cxz) * srctmp) / den;
                syz = (-(fr / la) * (fr * cyz) + (Md * fr) * lc(4)) + ((fr * cyz) * srctmp) / den;
            } else {
                const double fr = -(((1.0 - K.epsPTT * 3.0) + K.epsPTT * ((cxx + cyy) + czz))) / K.lambda;
                sxx = fr * (cxx - 1.0) + Md * lc(0); sxy = fr * cxy + Md * lc(1);
                syy = fr * (cyy - 1.0) + Md * lc(2); sxz = fr * cxz + Md * lc(3);
                syz = fr * cyz + Md * lc(4); szz = fr * (czz - 1.0) + Md * lc(5);
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
            r[4] = (-ad[0] + ucxx) + csxx;
            r[5] = (-ad[1] + ucxy) + csxy;
            r[6] = (-ad[2] + ucyy) + csyy;
            r[7] = (-ad[3] + ucxz) + csxz;
            r[8] = (-ad[4] + ucyz) + csyz;
            r[9] = (-ad[5] + uczz) + cszz;
        }
        if (kLc) {  // calc_rhs_logconf, rhs_lc.F90:383-560 (sPTT, 3-D), walls :564-740
            const bool first = (P.sc->itime == 1) && (P.stage == 0);
            double ad[6];
#pragma unroll
            for (int q = 0; q < 6; q++) ad[q] = -((u * g(PG0 + 3 * q) + v * g(PG0 + 3 * q + 1)) + w * g(PG0 + 3 * q + 2));
            double Lv[3], R[9], RT[9], Gm[9], T[9], M[9], B[9], Om[9], Ps[9], OP[9], PO[9], Ci[9], Rx[9];
            eigens3(P.in[7][k], P.in[8][k], P.in[9][k], P.in[10][k], P.in[11][k], P.in[12][k], Lv, R);
            tr3(R, RT);
            const double tr_c = (Lv[0] + Lv[1]) + Lv[2];
            Gm[0] = gux; Gm[3] = guy; Gm[6] = g(UZ);
            Gm[1] = gvx; Gm[4] = gvy; Gm[7] = g(VZ);
            Gm[2] = gwx; Gm[5] = gwy; Gm[8] = g(WZ);
            mm3(Gm, R, T);
            mm3(RT, T, M);
            double oxy = (Lv[1] * M[3] + Lv[0] * M[1]);
            if (fabs(Lv[1] - Lv[0]) <= 1.0e-30) oxy = 0.0;
            else oxy = oxy / (Lv[1] - Lv[0]);
            double oxz = (Lv[2] * M[6] + Lv[0] * M[2]);
            if (fabs(Lv[2] - Lv[0]) <= 1.0e-30) oxz = 0.0;
            else oxz = oxz / (Lv[2] - Lv[0]);
            double oyz = (Lv[2] * M[7] + Lv[1] * M[5]);
            if (fabs(Lv[2] - Lv[1]) <= 1.0e-30) oyz = 0.0;
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
            Ps[0] = P.in[13][k]; Ps[3] = P.in[14][k]; Ps[1] = P.in[14][k]; Ps[4] = P.in[15][k];
            Ps[6] = P.in[16][k]; Ps[2] = P.in[16][k]; Ps[7] = P.in[17][k]; Ps[5] = P.in[17][k]; Ps[8] = P.in[18][k];
            mm3(Om, Ps, OP);
            mm3(Ps, Om, PO);
            const double fR = ((1.0 - 2.0 * K.epsPTT) + K.epsPTT * tr_c);
            for (int q = 0; q < 9; q++) Ci[q] = 0.0;
            Ci[0] = fR / Lv[0] - fR; Ci[4] = fR / Lv[1] - fR; Ci[8] = fR / Lv[2] - fR;
            mm3(Ci, RT, T);
            mm3(R, T, T);
            for (int q = 0; q < 9; q++) Rx[q] = T[q] / K.lambda;
            static constexpr int idx[6] = {0, 3, 4, 6, 7, 8};  // (1,1) (1,2) (2,2) (1,3) (2,3) (3,3)
#pragma unroll
            for (int q = 0; q < 6; q++) {
                const int e = idx[q];
                const double uc = (OP[e] - PO[e]) + 2.0 * B[e];
                r[4 + q] = wall ? uc + Rx[e] : (ad[q] + uc) + Rx[e];  // walls: no advection (:717-726)
            }
        }
        if (kDi) {
            const double cxx = P.in[7][k], cxy = P.in[8][k], cyy = P.in[9][k], cxz = P.in[10][k], cyz = P.in[11][k],
                         czz = P.in[12][k];
            double ad[6];
#pragma unroll
            for (int q = 0; q < 6; q++) ad[q] = -((u * g(CG0 + 3 * q) + v * g(CG0 + 3 * q + 1)) + w * g(CG0 + 3 * q + 2));
            const double ux = gux, uy = guy, uz = g(UZ), vx = gvx, vy = gvy, vz = g(VZ);
            const double wx = gwx, wy = gwy, wz = g(WZ);
            const double ucxx = ((2.0 * ux) * cxx + (2.0 * uy) * cxy) + (2.0 * uz) * cxz;
            const double ucxy = (((((ux * cxy + uy * cyy) + uz * cyz) + vx * cxx) + vy * cxy) + vz * cxz);
            const double ucyy = ((2.0 * vx) * cxy + (2.0 * vy) * cyy) + (2.0 * vz) * cyz;
            const double uczz = ((2.0 * wx) * cxz + (2.0 * wy) * cyz) + (2.0 * wz) * czz;
            const double ucxz = (((((ux * cxz + uy * cyz) + uz * czz) + wx * cxx) + wy * cxy) + wz * cxz);
            const double ucyz = (((((vx * cxz + vy * cyz) + vz * czz) + wx * cxy) + wy * cyy) + wz * cyz);
            double sxx, sxy, syy, sxz, syz, szz;
            if (P.fen) {  // FENE-P relaxation, rhs_di.F90:454-464
                const double fr = -P.fen[k], la = K.lambda;
                sxx = (fr * cxx + 1.0) / la; sxy = (fr * cxy) / la; syy = (fr * cyy + 1.0) / la;
                szz = (fr * czz + 1.0) / la; sxz = (fr * cxz) / la; syz = (fr * cyz) / la;
            } else {
                const double fr = -(((1.0 - K.epsPTT * 2.0) + K.epsPTT * ((cxx + cyy) + czz))) / K.lambda;
                sxx = fr * (cxx - 1.0); sxy = fr * cxy; syy = fr * (cyy - 1.0);
                sxz = fr * cxz; syz = fr * cyz; szz = fr * (czz - 1.0);
            }
            const double Md = K.Mdiff;
            auto lc = [&](int q) {
                if (!P.md) return 0.0;
                const double x = g(LC0 + q);
                return wall ? x + fdrows(q) : x;
            };
            if (inout) {  // :582-590: zero on inflow and outflow nodes (to be completed there)
                for (int q = 4; q < 10; q++) r[q] = 0.0;
            } else if (wall) {  // rhs_di.F90:571-580: without the advection
                r[4] = (ucxx + sxx) + Md * lc(0);
                r[5] = (ucxy + sxy) + Md * lc(1);
                r[6] = (ucyy + syy) + Md * lc(2);
                r[7] = (ucxz + sxz) + Md * lc(3);
                r[8] = (ucyz + syz) + Md * lc(4);
                r[9] = (uczz + szz) + Md * lc(5);
            } else {
                r[4] = ((ad[0] + ucxx) + sxx) + Md * lc(0);
                r[5] = ((ad[1] + ucxy) + sxy) + Md * lc(1);
                r[6] = ((ad[2] + ucyy) + syy) + Md * lc(2);
                r[7] = ((ad[3] + ucxz) + sxz) + Md * lc(3);
                r[8] = ((ad[4] + ucyz) + syz) + Md * lc(4);
                r[9] = ((ad[5] + uczz) + szz) + Md * lc(5);
            }
        }
        const int nf = (kDi || kChl || kLc) ? 10 : 4;
        if (P.stage == 4) {
            for (int q = 0; q < 10; q++) P.rhs[q][k] = r[q];
        } else {
            // evolved fields: rho, rho u, rho v, rho w, then c (direct) or psi (Cholesky)
            const int c0 = (kChl || kLc) ? 13 : 7;
            const int src[10] = {0, 1, 2, 3, c0, c0 + 1, c0 + 2, c0 + 3, c0 + 4, c0 + 5};
            const int stage = P.stage;
            const double dt = P.sc->dt;
            const double a = stage == 0 ? SUNSET_RK_A21 : stage == 1 ? SUNSET_RK_A32 : SUNSET_RK_A43;
            const double b = stage == 0 ? SUNSET_RK_B1 : stage == 1 ? SUNSET_RK_B2 : stage == 2 ? SUNSET_RK_B3 : SUNSET_RK_B4;
            const double bh = stage == 0 ? SUNSET_RK_BH1 : stage == 1 ? SUNSET_RK_BH2 : stage == 2 ? SUNSET_RK_BH3 : SUNSET_RK_BH4;
            const double RKb = dt * b, RKbmbh = dt * (b - bh);
            double Un[10];
            double en = 0.0, al = 0.0;
            for (int q = 0; q < 10; q++) Un[q] = P.in[src[q]][k];
            // every register read before the first is written (the compiler cannot tell the
            // arrays apart, and would otherwise wait out each load after a store)
            double Sq[10], Eq[10];
#pragma unroll
            for (int q = 0; q < 10; q++) {
                if (q >= nf) break;
                Sq[q] = stage == 0 ? Un[q] : P.reg[q][k];
                Eq[q] = stage == 0 ? 0.0 : P.eacc[q][k];
            }
#pragma unroll
            for (int q = 0; q < 10; q++) {
                if (q >= nf) break;
                const double S = Sq[q], E = Eq[q];
                if (stage < 3) {
                    Un[q] = S + (dt * a) * r[q];
                    P.reg[q][k] = S + RKb * r[q];
                    P.eacc[q][k] = E + RKbmbh * r[q];
                } else {
                    Un[q] = S + RKb * r[q];
                    const double norm = q == 0 ? K.ero_norm : q < 4 ? K.erou_norm : K.exx_norm;
                    double t = fabs(E + RKbmbh * r[q]) * norm;
                    if (q != 3 && q < 7) al = (t > al) ? t : al;  // alpha_out: rho, momentum x y, xx xy yy
                    // Cholesky FENE-P (step.F90:442-452): the xx, xy, yy and zz errors scaled by
                    // 1/sqrt(f) of the node-layer's c, each node-layer's own before the maximum
                    if (kChl && K.fenep && (q == 4 || q == 5 || q == 6 || q == 9))
                        t = t * (1.0 / sqrt((K.fenep_l2 - 3.0) / (((K.fenep_l2 - P.in[7][k]) - P.in[9][k]) - P.in[12][k])));
                    en = (t > en) ? t : en;
                    if (t != t) en = t;
                }
            }
            if (stage == 3) {
                eb = dbits(en);
                P.alpha[k] = al;
            }
            // apply_time_dependent_bounds (characteristic_boundaries.F90:191-257) at the stage's
            // time time0 + c_s dt: walls at rest; on inflow node-layers u_inflow_local follows
            // its ramp, and a hard inflow prescribes the momentum
            if (wall) { Un[1] = 0.0; Un[2] = 0.0; Un[3] = 0.0; }
            if (ty == 1) {
                const double cs = stage == 0 ? 0.0 : stage == 1 ? SUNSET_RK_A21 : stage == 2 ? (SUNSET_RK_A32 + SUNSET_RK_B1) : 1.0;
                uin = inflow_velocity(K, P.sc->time + dt * cs, uin);
                P.uin[k] = uin;
                if (K.inflow_type == 1) { Un[1] = uin * Un[0]; Un[2] = 0.0; Un[3] = 0.0; }
            }
            for (int q = 0; q < 10; q++) P.out[src[q]][k] = Un[q];
            const double oo = 1.0 / Un[0];  // get_velocity_from_momentum
            P.out[4][k] = Un[1] * oo;
            P.out[5][k] = Un[2] * oo;
            P.out[6][k] = Un[3] * oo;
            if (kChl || kLc) {  // get_c_from_psi
                double c[6];
                if (kChl) chl3_c_from_psi(Un + 4, c, K.fenep ? K.fenep_l2 : 0.0);
                else lc3_transform(Un + 4, c, true);
                for (int q = 0; q < 6; q++) P.out[7 + q][k] = c[q];
            }
        }
    }
    return eb;
}

// block maximum of the step error bits, then one atomic (stage 3; all threads of the block)
__device__ __forceinline__ void block_emax3(unsigned long long eb, DevScalars *sc) {
    __shared__ unsigned long long sm[32];
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long t = __shfl_down_sync(0xffffffffu, eb, o);
        eb = t > eb ? t : eb;
    }
    if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = eb;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long m = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) m = sm[w] > m ? sm[w] : m;
        if (m) atomicMax(&sc->emax_bits, m);
    }
}

// One stage fused: the derivatives of node-layer k (derivs3_body) go to this block's shared
// memory, compact slots of 128 doubles (one per thread), and the pointwise right-hand side
// and RK update (point3_body) read them there, so no derivative array crosses HBM.
template <int FORM, bool MD, bool FULL, bool FEN, bool BND>
__global__ void __launch_bounds__(128, derivs_min_blocks(FORM)) k3_stage(Layer3 L, Fields3 F, Point3 P) {
    constexpr int NS = ngslots<FORM, MD, FULL, FEN>();
    __shared__ double sg[NS * 128];
    ZThread z;
    const bool live = zthread(L, z);
    unsigned long long eb = 0;
    if (live) {
        derivs3_body<FORM, MD, FULL, FEN, BND>(L, F, z, [&](int slot, double v) {
            const int c = kGTable<FORM, MD, FULL, FEN>.idx[slot];
            if (c >= 0) sg[c * 128 + threadIdx.x] = v;
        });
        eb = point3_body<FORM, BND>(P, (size_t)z.k, [&](int a) {
            const int c = kGTable<FORM, MD, FULL, FEN>.idx[a];
            return c >= 0 ? sg[c * 128 + threadIdx.x] : 0.0;
        });
    }
    if (P.stage == 3) block_emax3(eb, P.sc);
}

// Block sums of (rho - rho_char) vol (or of vol), in a fixed tree; folded in block order.
__global__ void k3_mass_partials(int nz, size_t n, const double *ro, const double *vol, double rho_char, int volume_only,
                                 double *partials) {
    __shared__ double red[128];
    const size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    double v = 0.0;
    if (k < n) {
        const double vi = vol[k / nz];
        v = volume_only ? vi : (ro[k] - rho_char) * vi;
    }
    red[threadIdx.x] = v;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) red[threadIdx.x] = red[threadIdx.x] + red[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) partials[blockIdx.x] = red[0];
}
constexpr int kFoldThreads = 1024;
__global__ void __launch_bounds__(kFoldThreads) k3_fold(const double *partials, int nblk, double *out, const double *divisor,
                                                         int enabled) {
    __shared__ double red[kFoldThreads];
    double a = 0.0;
    for (int b = threadIdx.x; b < nblk; b += blockDim.x) a = a + partials[b];
    red[threadIdx.x] = a;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) red[threadIdx.x] = red[threadIdx.x] + red[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = divisor ? (enabled ? red[0] / *divisor : 0.0) : red[0];
}

// velocity_control with -Dvpid in 3-D (statistics.F90:214-303, dV = vol dz): block sums of
// u dV and of dV (a fixed tree), then the fold and the PID update of driving_force(1)
__global__ void k3_flow_partials(int nz, size_t n, const double *u, const double *vol, double dz, double *pu,
                                 double *pv) {
    __shared__ double ru[128], rv[128];
    const size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    double a = 0.0, b = 0.0;
    if (k < n) {
        b = vol[k / nz] * dz;
        a = u[k] * b;
    }
    ru[threadIdx.x] = a;
    rv[threadIdx.x] = b;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) {
            ru[threadIdx.x] = ru[threadIdx.x] + ru[threadIdx.x + s];
            rv[threadIdx.x] = rv[threadIdx.x] + rv[threadIdx.x + s];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        pu[blockIdx.x] = ru[0];
        pv[blockIdx.x] = rv[0];
    }
}
constexpr int kFlowThreads = 1024;
__global__ void __launch_bounds__(kFlowThreads) k3_velocity_control(const double *pu, const double *pv, int nblk, double Lx,
                                                                     double Ly, DevScalars *sc) {
    __shared__ double ru[kFlowThreads], rv[kFlowThreads];
    double a = 0.0, b = 0.0;
    for (int q = threadIdx.x; q < nblk; q += blockDim.x) {
        a = a + pu[q];
        b = b + pv[q];
    }
    ru[threadIdx.x] = a;
    rv[threadIdx.x] = b;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) {
            ru[threadIdx.x] = ru[threadIdx.x] + ru[threadIdx.x + s];
            rv[threadIdx.x] = rv[threadIdx.x] + rv[threadIdx.x + s];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const double tot_vol = rv[0], dt = sc->dt;
        const double tot_u = ru[0] / tot_vol;
        const double eflow_n = 1.0 - (tot_u * tot_vol) / (Ly * Lx);
        sc->sum_eflow = sc->sum_eflow + eflow_n * dt;
        const double deflowdt = (eflow_n - sc->eflow_nm1) / dt;
        const double facA = ((((0.5 * 0.5) * 0.5) * 1.0) * 2.0) * 2.0;
        const double facB = facA / 0.4, facC = facA * 0.02;
        double df = ((facA * eflow_n) + facB * sc->sum_eflow) + facC * deflowdt;
        df = (500.0 < df) ? 500.0 : df;
        df = (-500.0 > df) ? -500.0 : df;
        sc->df = df;
        sc->eflow_nm1 = eflow_n;
    }
}

// End of step: mass correction, apply_time_dependent_bounds (ntype: node types, or null without
// boundary nodes: walls at rest, a hard inflow's momentum from u_inflow_local), u, v, w from the
// momentum, the error-norm history and time.
__global__ void k3_finalize(size_t n, int nz, const int *ntype, const double *uin, int hard_in, Fields3 F, int chl, int lc,
                            double L2, DevScalars *sc, int vpid) {
    const size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) {
        // every load before the first store (the arrays are not known to be distinct)
        const double r = F.p[0][k] - sc->dro;
        double m1 = F.p[1][k], m2 = F.p[2][k], m3 = F.p[3][k];
        double p[6], c[6];
        if (chl || lc)
            for (int q = 0; q < 6; q++) p[q] = F.p[13 + q][k];
        const int ty = ntype ? ntype[(unsigned)k / (unsigned)nz] : 999;
        if (ty == 0) {
            m1 = 0.0; m2 = 0.0; m3 = 0.0;
        } else if (ty == 1 && hard_in) {  // the hard inflow's momentum from the corrected density
            m1 = uin[k] * r; m2 = 0.0; m3 = 0.0;
        }
        if (ty == 0 || (ty == 1 && hard_in)) {
            F.p[1][k] = m1; F.p[2][k] = m2; F.p[3][k] = m3;
        }
        F.p[0][k] = r;
        const double oo = 1.0 / r;
        F.p[4][k] = m1 * oo;
        F.p[5][k] = m2 * oo;
        F.p[6][k] = m3 * oo;
        if (chl || lc) {
            if (chl) chl3_c_from_psi(p, c, L2);
            else lc3_transform(p, c, true);
            for (int q = 0; q < 6; q++) F.p[7 + q][k] = c[q];
        }
    }
    if (k == 0) {
        const double e = __longlong_as_double((long long)sc->emax_bits);
        const double emax = (e > 1.0e-16) ? e : 1.0e-16;
        if (!(e == e) || isinf(e)) sc->err = 1;
        sc->emax_nm1 = sc->emax_n;
        sc->emax_n = sc->emax_np1;
        sc->emax_np1 = emax;
        sc->emax_bits = 0ull;
        sc->time = sc->time + sc->dt;
        sc->itime = sc->itime + 1;
        if (!vpid) sc->df = 0.0;
    }
}

// set_tstep (step.F90:569-622) over the 3-D nodes: block minima as bit patterns
__global__ void k3_tstep(int nz, size_t n, const int *ntype, const double *u, const double *v, const double *w,
                         const double *ro, const double *sp, double csq, double visc_total, DevScalars *sc) {
    const size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    double tc = 1.0e10, tp = 1.0e10;
    if (k < n) {
        const int i = (int)((unsigned)k / (unsigned)nz);
        const double c = sqrt(csq);
        const double um = sqrt((u[k] * u[k] + v[k] * v[k]) + w[k] * w[k]);
        tc = (ntype && ntype[i] == 2) ? (0.8 * sp[i]) / (um + c) : sp[i] / (um + c);  // outflow: 0.8
        tp = ((sp[i] * sp[i]) * ro[k]) / visc_total;
    }
    unsigned long long bc = dbits(tc), bp = dbits(tp);
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long x = __shfl_down_sync(0xffffffffu, bc, o), y = __shfl_down_sync(0xffffffffu, bp, o);
        bc = x < bc ? x : bc;
        bp = y < bp ? y : bp;
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMin(&sc->cfl_bits, bc);
        atomicMin(&sc->par_bits, bp);
    }
}
// fold the minima into dt_cfl, dt_parabolic; with pid, set_tstep_PID (step.F90:624-682)
__global__ void k3_tstep_fold(DevScalars *sc, double L, int pid) {
    const double dcfl = __longlong_as_double((long long)sc->cfl_bits);
    const double dvisc = __longlong_as_double((long long)sc->par_bits);
    sc->dt_cfl = (1.0 * dcfl) * L;
    sc->dt_par = (((2.0 / 3.0) * dvisc) * L) * L;
    sc->cfl_bits = 0x7ff0000000000000ull;
    sc->par_bits = 0x7ff0000000000000ull;
    if (!pid) return;
    const double facA = (0.49 / 2.0) * log(1.0e-5 / sc->emax_np1);
    const double facB = (0.34 / 2.0) * log(sc->emax_n / 1.0e-5);
    const double facC = (0.1 / 2.0) * log(1.0e-5 / sc->emax_nm1);
    double f = 0.9 * exp((facA + facB) + facC);
    f = (0.5 > f) ? 0.5 : f;
    f = (1.02 < f) ? 1.02 : f;
    double dt = sc->dt * f;
    const double dmax = (sc->dt_cfl < sc->dt_par) ? sc->dt_cfl : sc->dt_par;
    if (dt > dmax) dt = dmax;
    sc->dt = dt;
}

// reference arrays (layer-major, reference node order) <-> internal arrays (node-major, layers
// innermost, internal node order)
__global__ void k3_gather(const double *in, const int *perm, int nl, int nz, size_t n, double *out) {
    const size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const size_t i = k / nz, iz = k - i * nz;
    out[k] = in[iz * nl + perm[i]];
}
__global__ void k3_scatter(const double *in, const int *perm, int nl, int nz, size_t n, double *out) {
    const size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const size_t i = k / nz, iz = k - i * nz;
    out[iz * nl + perm[i]] = in[k];
}
__global__ void k3_fill(size_t n, double v, double *out) {
    const size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) out[k] = v;
}
// the Cholesky or log-conformation state from the given c: psi from c, then c from psi
// (setup_flow.F90:86-117)
__global__ void k3_psi_from_c(size_t n, Fields3 F, int lc, double L2) {
    const size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    double c[6], p[6];
    for (int q = 0; q < 6; q++) c[q] = F.p[7 + q][k];
    if (lc) {
        lc3_transform(c, p, false);
        lc3_transform(p, c, true);
    } else {
        chl3_psi_from_c(c, p, L2);
        chl3_c_from_psi(p, c, L2);
    }
    for (int q = 0; q < 6; q++) {
        F.p[13 + q][k] = p[q];
        F.p[7 + q][k] = c[q];
    }
}
// Cholesky FENE-P around the filter: the six psi (fields 4-9 of the filter's list) from the
// factors of J to those of c (to_c), or back
__global__ void k3_fenep_factors(size_t n, Filter3 A, double L2, int to_c) {
    const size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    double p[6];
    for (int q = 0; q < 6; q++) p[q] = A.f[4 + q][k];
    chl3_fenep_factor(L2, p, to_c != 0);
    for (int q = 0; q < 6; q++) A.f[4 + q][k] = p[q];
}
// hardcode_initial_conditions in 3-D: u, v, w zero on walls (setup_flow.F90:266-280; ntype
// null without walls), then rho u = rho * u, rho v, rho w
__global__ void k3_momentum(size_t n, int nz, const int *ntype, const double *ro, double *u, double *v, double *w,
                            double *rou, double *rov, double *row) {
    const size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    if (ntype && ntype[(unsigned)k / (unsigned)nz] == 0) {
        u[k] = 0.0; v[k] = 0.0; w[k] = 0.0;
    }
    rou[k] = ro[k] * u[k];
    rov[k] = ro[k] * v[k];
    row[k] = ro[k] * w[k];
}
// u_inflow_local of the initial state (setup_flow.F90:48-50,128-138): u on inflow node-layers,
// u_char elsewhere
__global__ void k3_init_uin(size_t n, int nz, const int *ntype, const double *u, double uchar, double *uin) {
    const size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    uin[k] = ntype[(unsigned)k / (unsigned)nz] == 1 ? u[k] : uchar;
}
// boundary nodes: the layer's Laplacian weights and sums, each boundary node's replaced by its
// tangential second-derivative weights (reference link order, as the layer's lists) and their
// sum: the conformation Laplacian's
__global__ void k3_boundary_lap_weights(int nl, const int *bidx, const long long *slice_ptr,
                                        const int *cnt_small, int nplink, const double *wbt, const double *wbt_sum,
                                        double *wl3, double *lsum3) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nl) return;
    const int jj = bidx[i];  // -1 off the boundary (FD rows carry negative node types)
    if (jj < 0) return;
    const long long base = slice_ptr[i >> 5];
    for (int q = 0; q < cnt_small[i]; q++) wl3[sell_at(base, q, i & 31)] = wbt[(size_t)jj * nplink + q];
    lsum3[i] = wbt_sum[jj];
}

// calc_fd_weights, fd.F90:52-172, then the L_char scaling of :246-247
int fd_tables(int ncfd, double dz, double L, double *g, double *g2, double *h) {
    const double one = 1.0, two = 2.0;
    if (ncfd == 5) {
        const double G[5] = {(one / 12.0) / dz, -((8.0 / 12.0) / dz), 0.0, (8.0 / 12.0) / dz, -((one / 12.0) / dz)};
        const double G2[5] = {-(((one / 12.0) / dz) / dz), ((16.0 / 12.0) / dz) / dz, -(((30.0 / 12.0) / dz) / dz),
                              ((16.0 / 12.0) / dz) / dz, -(((one / 12.0) / dz) / dz)};
        const double Hh[5] = {-(one / 16.0), 4.0 / 16.0, -(6.0 / 16.0), 4.0 / 16.0, -(one / 16.0)};
        for (int k = 0; k < 5; k++) { g[k] = G[k]; g2[k] = G2[k]; h[k] = Hh[k]; }
    } else if (ncfd == 7) {
        const double G[7] = {-((one / 60.0) / dz), (9.0 / 60.0) / dz, -((45.0 / 60.0) / dz), 0.0,
                             (45.0 / 60.0) / dz, -((9.0 / 60.0) / dz), (one / 60.0) / dz};
        const double G2[7] = {((two / 180.0) / dz) / dz, -(((27.0 / 180.0) / dz) / dz), ((270.0 / 180.0) / dz) / dz,
                              -(((490.0 / 180.0) / dz) / dz), ((270.0 / 180.0) / dz) / dz, -(((27.0 / 180.0) / dz) / dz),
                              ((two / 180.0) / dz) / dz};
        const double Hh[7] = {one / 64.0, -(6.0 / 64.0), 15.0 / 64.0, -(20.0 / 64.0), 15.0 / 64.0, -(6.0 / 64.0), one / 64.0};
        for (int k = 0; k < 7; k++) { g[k] = G[k]; g2[k] = G2[k]; h[k] = Hh[k]; }
    } else if (ncfd == 9) {
        const double G[9] = {(3.0 / 840.0) / dz, -((32.0 / 840.0) / dz), (168.0 / 840.0) / dz, -((672.0 / 840.0) / dz), 0.0,
                             (672.0 / 840.0) / dz, -((168.0 / 840.0) / dz), (32.0 / 840.0) / dz, -((3.0 / 840.0) / dz)};
        const double G2[9] = {-(((9.0 / 5040.0) / dz) / dz), ((128.0 / 5040.0) / dz) / dz, -(((1008.0 / 5040.0) / dz) / dz),
                              ((8064.0 / 5040.0) / dz) / dz, -(((14350.0 / 5040.0) / dz) / dz), ((8064.0 / 5040.0) / dz) / dz,
                              -(((1008.0 / 5040.0) / dz) / dz), ((128.0 / 5040.0) / dz) / dz, -(((9.0 / 5040.0) / dz) / dz)};
        const double Hh[9] = {-(one / 256.0), 8.0 / 256.0, -(28.0 / 256.0), 56.0 / 256.0, -(70.0 / 256.0),
                              56.0 / 256.0, -(28.0 / 256.0), 8.0 / 256.0, -(one / 256.0)};
        for (int k = 0; k < 9; k++) { g[k] = G[k]; g2[k] = G2[k]; h[k] = Hh[k]; }
    } else if (ncfd == 11) {
        const double G[11] = {-((one / 1260.0) / dz), (5.0 / 504.0) / dz, -((5.0 / 84.0) / dz), (5.0 / 21.0) / dz,
                              -((5.0 / 6.0) / dz), 0.0, (5.0 / 6.0) / dz, -((5.0 / 21.0) / dz), (5.0 / 84.0) / dz,
                              -((5.0 / 504.0) / dz), (one / 1260.0) / dz};
        const double G2[11] = {((one / 3150.0) / dz) / dz, -(((5.0 / 1008.0) / dz) / dz), ((5.0 / 126.0) / dz) / dz,
                               -(((5.0 / 21.0) / dz) / dz), ((5.0 / 3.0) / dz) / dz, -(((1086.0 / 371.0) / dz) / dz),
                               ((5.0 / 3.0) / dz) / dz, -(((5.0 / 21.0) / dz) / dz), ((5.0 / 126.0) / dz) / dz,
                               -(((5.0 / 1008.0) / dz) / dz), ((one / 3150.0) / dz) / dz};
        const double Hh[11] = {one / 1024.0, -(10.0 / 1024.0), 45.0 / 1024.0, -(120.0 / 1024.0), 210.0 / 1024.0,
                               -(252.0 / 1024.0), 210.0 / 1024.0, -(120.0 / 1024.0), 45.0 / 1024.0, -(10.0 / 1024.0),
                               one / 1024.0};
        for (int k = 0; k < 11; k++) { g[k] = G[k]; g2[k] = G2[k]; h[k] = Hh[k]; }
    } else {
        return -1;
    }
    for (int k = 0; k < ncfd; k++) {
        g[k] = g[k] / L;
        g2[k] = (g2[k] / L) / L;
    }
    return 0;
}

Layer3 layer3(const Handle *H) {
    Layer3 L{};
    L.nl = H->npfb;
    L.nz = H->nz;
    L.ncfd = H->ncfd;
    L.nzc = H->nz >= 32 ? (H->nz + 31) / 32 : 0;
    L.slice_ptr = H->slice_ptr;
    L.cnt = H->cnt;
    L.cnt_small = H->cnt_small;
    L.lidx = H->lidx;
    L.wx = H->wx; L.wy = H->wy; L.wl = H->wl; L.wh = H->wh;
    L.gsx = H->gsx; L.gsy = H->gsy; L.lsum = H->lsum; L.hsum = H->hsum;
    L.wlc = H->wl3;
    L.lsumc = H->lsum3;
    for (int m = 0; m < kMaxFd; m++) { L.fdg[m] = H->fdg[m]; L.fdl[m] = H->fdl[m]; L.fdh[m] = H->fdh[m]; }
    return L;
}

inline size_t n3(const Handle *H) { return (size_t)H->npfb * H->nz; }
inline unsigned nblk(size_t n) { return (unsigned)((n + 127) / 128); }
// blocks of 128 threads over the node-layers in zthread's order
inline unsigned zblocks(const Handle *H) {
    if (H->nz >= 32) return (unsigned)(((H->npfb + 3) / 4) * ((H->nz + 31) / 32));
    return nblk(n3(H));
}

// FENE-P function of every node-layer (rhs_di.F90:201-203), into the staging array
__global__ void k3_fenep(unsigned n, const double *cxx, const double *cyy, const double *czz, double L2, double *f) {
    const unsigned k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) f[k] = (L2 - 3.0) / (L2 - ((cxx[k] + cyy[k]) + czz[k]));
}

Point3 point3(Handle *H, int b, int stage) {
    Point3 P{};
    P.K = step_consts(H->cfg, H->npfb, H->nslices, H->has_mirrors, false, H->xmax - H->xmin, H->ymax - H->ymin);
    P.nl = H->npfb;
    P.nz = H->nz;
    P.di = H->cfg.form == SUNSET_FORM_DI;
    P.chl = H->cfg.form == SUNSET_FORM_CHL;
    P.lc = H->cfg.form == SUNSET_FORM_LC;
    P.full = H->cfg.di_full_gradients;
    P.md = H->cfg.Mdiff != 0.0;
    P.py = H->py;
    P.ntype = H->ntype;
    P.bidx = H->bidx;
    P.brow = H->brow;
    P.rnx = H->rnx;
    P.rny = H->rny;
    P.sp = H->sp;
    P.uin = H->uin3;
    P.alpha = H->alpha3;
    P.fen = (H->cfg.form == SUNSET_FORM_DI && H->cfg.fenep) ? H->tmp3 : nullptr;
    for (int f = 0; f < 19; f++) {
        P.in[f] = H->f3[b][f];
        P.out[f] = H->f3[b ^ 1][f];
    }
    for (int q = 0; q < 10; q++) { P.reg[q] = H->reg3[q]; P.eacc[q] = H->eacc3[q]; P.rhs[q] = H->rhs3[q]; }
    P.sc = H->dsc;
    P.stage = stage;
    return P;
}

// One fused stage (k3_stage) of buffer b: derivatives, right-hand side and RK update
template <int FORM, bool MD, bool FULL, bool FEN = false>
int stage3_launch(Handle *H, int b, int stage) {
    const size_t n = n3(H);
    Fields3 F{};
    for (int q = 0; q < 19; q++) F.p[q] = H->f3[b][q];
    if (FEN) {
        k3_fenep<<<nblk(n), 128, 0, H->stream>>>((unsigned)n, H->f3[b][7], H->f3[b][9], H->f3[b][12], H->cfg.fenep_l2, H->tmp3);
        F.p[19] = H->tmp3;
    }
    if (H->nb > 0)
        k3_stage<FORM, MD, FULL, FEN, true><<<zblocks(H), 128, 0, H->stream>>>(layer3(H), F, point3(H, b, stage));
    else
        k3_stage<FORM, MD, FULL, FEN, false><<<zblocks(H), 128, 0, H->stream>>>(layer3(H), F, point3(H, b, stage));
    SUNSET_CUDA(H, cudaGetLastError());
    return 0;
}
int stage3(Handle *H, int b, int stage) {
    const bool md = H->cfg.Mdiff != 0.0, full = H->cfg.di_full_gradients != 0;
    switch (H->cfg.form) {
    case SUNSET_FORM_DI:
        if (H->cfg.fenep) {
            if (md)
                return full ? stage3_launch<SUNSET_FORM_DI, true, true, true>(H, b, stage)
                            : stage3_launch<SUNSET_FORM_DI, true, false, true>(H, b, stage);
            return full ? stage3_launch<SUNSET_FORM_DI, false, true, true>(H, b, stage)
                        : stage3_launch<SUNSET_FORM_DI, false, false, true>(H, b, stage);
        }
        if (md) return full ? stage3_launch<SUNSET_FORM_DI, true, true>(H, b, stage) : stage3_launch<SUNSET_FORM_DI, true, false>(H, b, stage);
        return full ? stage3_launch<SUNSET_FORM_DI, false, true>(H, b, stage) : stage3_launch<SUNSET_FORM_DI, false, false>(H, b, stage);
    case SUNSET_FORM_CHL:
        return md ? stage3_launch<SUNSET_FORM_CHL, true, false>(H, b, stage) : stage3_launch<SUNSET_FORM_CHL, false, false>(H, b, stage);
    case SUNSET_FORM_LC: return stage3_launch<SUNSET_FORM_LC, false, false>(H, b, stage);
    default: return stage3_launch<SUNSET_FORM_NEWT, false, false>(H, b, stage);
    }
}

int tstep3_launch(Handle *H, int b, int pid) {
    const size_t n = n3(H);
    const double *const *f = H->f3[b];
    k3_tstep<<<nblk(n), 128, 0, H->stream>>>(H->nz, n, H->nb > 0 ? H->ntype : nullptr, f[4], f[5], f[6], f[0], H->sp, step_consts(H->cfg, 1, 1, false, false).csq,
                                             step_consts(H->cfg, 1, 1, false, false).visc_total, H->dsc);
    k3_tstep_fold<<<1, 1, 0, H->stream>>>(H->dsc, H->cfg.L_char, pid);
    SUNSET_CUDA(H, cudaGetLastError());
    return 0;
}

}  // namespace

// ---------------------------------------------------------------------------------------
int layers_set(Handle *H, double Lz) {
    if (!(Lz > 0.0)) return set_err(H, SUNSET_ERR_ARG, "L_domain_z must be positive");
    if (H->cfg.fenep && H->cfg.form != SUNSET_FORM_DI && H->cfg.form != SUNSET_FORM_CHL)
        return set_err(H, SUNSET_ERR_SCOPE, "the 3-D path covers FENE-P with the direct and Cholesky forms");
    if (H->cfg.precision != SUNSET_FP64) return set_err(H, SUNSET_ERR_SCOPE, "the 3-D path runs in FP64");
    if (H->cfg.grav[2] != 0.0) return set_err(H, SUNSET_ERR_SCOPE, "grav(3) must be zero");
    const int ncfd = H->cfg.forder + 1;
    // build_3rd_dimension, setup_domain.F90:444-483: dz from the mean spacing (s^3 over s^2,
    // summed in the reference's node order), then nz layers over L_domain_z
    std::vector<double> sp(H->npfb);
    SUNSET_CUDA(H, cudaMemcpy(sp.data(), H->sp, H->npfb * sizeof(double), cudaMemcpyDeviceToHost));
    std::vector<double> sref(H->npfb);
    for (int i = 0; i < H->npfb; i++) sref[H->h_perm[i]] = sp[i];
    double dzl = 0.0, sv = 0.0;
    for (int r = 0; r < H->npfb; r++) {
        sv = sv + sref[r] * sref[r];
        dzl = dzl + (sref[r] * sref[r]) * sref[r];
    }
    double dz = dzl / sv;
    const double L = H->cfg.L_char, Lzd = (Lz * L) / L;
    int nz = (int)ceil((Lzd / dz) / 1.0);
    dz = (Lzd / (double)nz) / 1.0;
    if (nz < ncfd / 2 + 2) {
        nz = ncfd / 2 + 2;
        dz = Lzd / (double)(ncfd / 2 + 2);
    }
    if ((double)nz * H->npfb >= 2.0e9) return set_err(H, SUNSET_ERR_SCOPE, "too many 3-D nodes");
    H->nz = nz;
    H->dz = dz;
    H->ncfd = ncfd;
    for (int m = 0; m < 13; m++) H->fdg[m] = H->fdl[m] = H->fdh[m] = 0.0;
    if (fd_tables(ncfd, dz, L, H->fdg, H->fdl, H->fdh)) return set_err(H, SUNSET_ERR_SCOPE, "no z stencil for this order");
    return 0;
}

int state3_alloc(Handle *H) {
    if (H->g3) return 0;
    const size_t n = n3(H);
    if (dalloc(H, &H->alpha3, n)) return SUNSET_ERR_NOMEM;
    SUNSET_CUDA(H, cudaMemsetAsync(H->alpha3, 0, n * sizeof(double), H->stream));
    for (int b = 0; b < 2; b++)
        for (int f = 0; f < 19; f++)
            if (dalloc(H, &H->f3[b][f], n)) return SUNSET_ERR_NOMEM;
    for (int q = 0; q < 10; q++)
        if (dalloc(H, &H->reg3[q], n) || dalloc(H, &H->eacc3[q], n) || dalloc(H, &H->rhs3[q], n)) return SUNSET_ERR_NOMEM;
    // g3: the x-y filtered values of the ten evolved fields (the derivatives stay on chip)
    if (dalloc(H, &H->g3, (size_t)10 * n) || dalloc(H, &H->tmp3, n)) return SUNSET_ERR_NOMEM;
    for (int b = 0; b < 2; b++)
        for (int f = 7; f < 19; f++) SUNSET_CUDA(H, cudaMemsetAsync(H->f3[b][f], 0, n * sizeof(double), H->stream));
    if (H->nb > 0) {  // the boundary nodes' Laplacian weights of the layer (after the set-up's weights)
        if (!H->wbt) return set_err(H, SUNSET_ERR_ARG, "call order: the set-up's weights first");
        if (dalloc(H, &H->wl3, (size_t)H->nlinks_sell) || dalloc(H, &H->lsum3, (size_t)H->npfb) || dalloc(H, &H->uin3, n))
            return SUNSET_ERR_NOMEM;
        SUNSET_CUDA(H, cudaMemcpyAsync(H->wl3, H->wl, (size_t)H->nlinks_sell * sizeof(double), cudaMemcpyDeviceToDevice, H->stream));
        SUNSET_CUDA(H, cudaMemcpyAsync(H->lsum3, H->lsum, (size_t)H->npfb * sizeof(double), cudaMemcpyDeviceToDevice, H->stream));
        k3_boundary_lap_weights<<<(H->npfb + 127) / 128, 128, 0, H->stream>>>(H->npfb, H->bidx, H->slice_ptr, H->cnt_small,
                                                                        H->nplink, H->wbt, H->wbt_sum, H->wl3, H->lsum3);
        SUNSET_CUDA(H, cudaGetLastError());
    }
    const unsigned nb = nblk(n);
    // block partials: the mass sums, and the controller's two sums (from nb + 16 on)
    if (!H->partials3 && dalloc(H, &H->partials3, 3 * ((size_t)nb + 16))) return SUNSET_ERR_NOMEM;
    if (!H->dsc) {
        if (dalloc(H, &H->dsc, 1)) return SUNSET_ERR_NOMEM;
    }
    return 0;
}

// fields10: ro u v w cxx cxy cyy cxz cyz czz, reference layer-major, host memory (c may be null: c = I)
int state3_set(Handle *H, const double *const *fields10) {
    if (int rc = state3_alloc(H)) return rc;
    const size_t n = n3(H);
    cudaStream_t st = H->stream;
    H->cur3 = 0;
    double *const *f = H->f3[0];
    static const int dst[10] = {0, 4, 5, 6, 7, 8, 9, 10, 11, 12};
    for (int q = 0; q < 10; q++) {
        double *d = f[dst[q]];
        if (!fields10[q]) {  // c = I
            k3_fill<<<nblk(n), 128, 0, st>>>(n, (q == 4 || q == 6 || q == 9) ? 1.0 : 0.0, d);
            continue;
        }
        SUNSET_CUDA(H, cudaMemcpyAsync(H->tmp3, fields10[q], n * sizeof(double), cudaMemcpyHostToDevice, st));
        k3_gather<<<nblk(n), 128, 0, st>>>(H->tmp3, H->perm, H->npfb, H->nz, n, d);
    }
    k3_momentum<<<nblk(n), 128, 0, st>>>(n, H->nz, H->nb > 0 ? H->ntype : nullptr, f[0], f[4], f[5], f[6], f[1], f[2], f[3]);
    if (H->nb > 0) k3_init_uin<<<nblk(n), 128, 0, st>>>(n, H->nz, H->ntype, f[4], H->cfg.U_char, H->uin3);
    if (H->cfg.form == SUNSET_FORM_CHL || H->cfg.form == SUNSET_FORM_LC) {
        Fields3 F19;
        for (int q = 0; q < 19; q++) F19.p[q] = f[q];
        k3_psi_from_c<<<nblk(n), 128, 0, st>>>(n, F19, H->cfg.form == SUNSET_FORM_LC, H->cfg.fenep ? H->cfg.fenep_l2 : 0.0);
    }
    SUNSET_CUDA(H, cudaGetLastError());
    DevScalars s{};
    s.dt = 1.0e-6;
    s.emax_nm1 = s.emax_n = s.emax_np1 = 1.0e-5;  // pid_tol
    s.eflow_nm1 = 1.0;
    s.cfl_bits = 0x7ff0000000000000ull;
    s.par_bits = 0x7ff0000000000000ull;
    SUNSET_CUDA(H, cudaMemcpyAsync(H->dsc, &s, sizeof(s), cudaMemcpyHostToDevice, st));
    // sum of the 3-D nodes' volumes, for the mass correction
    k3_mass_partials<<<nblk(n), 128, 0, st>>>(H->nz, n, f[0], H->vol, 1.0, 1, H->partials3);
    k3_fold<<<1, kFoldThreads, 0, st>>>(H->partials3, (int)nblk(n), &H->dsc->tv, nullptr, 1);
    SUNSET_CUDA(H, cudaGetLastError());
    return tstep3_launch(H, 0, 0);
}

// out19: ro rou rov row u v w cxx cxy cyy cxz cyz czz psixx psixy psiyy psixz psiyz psizz,
// reference layer-major, host memory
int state3_get(Handle *H, double *out19) {
    const size_t n = n3(H);
    cudaStream_t st = H->stream;
    for (int f = 0; f < 19; f++) {
        k3_scatter<<<nblk(n), 128, 0, st>>>(H->f3[H->cur3][f], H->perm, H->npfb, H->nz, n, H->tmp3);
        SUNSET_CUDA(H, cudaMemcpyAsync(out19 + (size_t)f * n, H->tmp3, n * sizeof(double), cudaMemcpyDeviceToHost, st));
        SUNSET_CUDA(H, cudaStreamSynchronize(st));
    }
    return 0;
}

// u, v, w from the momentum and c from psi (get_velocity_from_momentum, get_c_from_psi,
// step.F90:514-567) after the evolved fields were set
__global__ void k3_derive(size_t n, Fields3 F, int chl, int lc, double L2) {
    const size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const double oo = 1.0 / F.p[0][k];
    const double m1 = F.p[1][k], m2 = F.p[2][k], m3 = F.p[3][k];
    double p[6], c[6];
    if (chl || lc)
        for (int q = 0; q < 6; q++) p[q] = F.p[13 + q][k];
    F.p[4][k] = m1 * oo;
    F.p[5][k] = m2 * oo;
    F.p[6][k] = m3 * oo;
    if (chl || lc) {
        if (chl) chl3_c_from_psi(p, c, L2);
        else lc3_transform(p, c, true);
        for (int q = 0; q < 6; q++) F.p[7 + q][k] = c[q];
    }
}

// The host-buffer round trip on a 3-D handle: the ten evolved fields (rho, rho u, rho v, rho w,
// then c in the direct form or psi) of every node-layer, layer-major, in from host memory; nsteps
// fixed-dt steps; the same fields back out.
int run_host3(Handle *H, const double *state_in, double dt, int nsteps, double *state_out) {
    const size_t n = n3(H);
    cudaStream_t st = H->stream;
    const bool chl = H->cfg.form == SUNSET_FORM_CHL, lc = H->cfg.form == SUNSET_FORM_LC;
    const int c0 = (chl || lc) ? 13 : 7;
    const int fld[10] = {0, 1, 2, 3, c0, c0 + 1, c0 + 2, c0 + 3, c0 + 4, c0 + 5};
    const int nf = H->cfg.form == SUNSET_FORM_NEWT ? 4 : 10;
    double *const *f = H->f3[H->cur3];
    for (int q = 0; q < nf; q++) {
        SUNSET_CUDA(H, cudaMemcpyAsync(H->tmp3, state_in + (size_t)q * n, n * sizeof(double), cudaMemcpyHostToDevice, st));
        k3_gather<<<nblk(n), 128, 0, st>>>(H->tmp3, H->perm, H->npfb, H->nz, n, f[fld[q]]);
    }
    Fields3 F19;
    for (int q = 0; q < 19; q++) F19.p[q] = f[q];
    k3_derive<<<nblk(n), 128, 0, st>>>(n, F19, chl, lc, H->cfg.fenep ? H->cfg.fenep_l2 : 0.0);
    SUNSET_CUDA(H, cudaGetLastError());
    if (int rc = step3_run(H, dt, nsteps, 0)) return rc;
    for (int q = 0; q < nf; q++)
        if (int rc = state3_column_to_host(H, H->f3[H->cur3][fld[q]], state_out + (size_t)q * n)) return rc;
    return 0;
}

// one internal node-layer array to the reference's layer-major order, in host memory
int state3_column_to_host(Handle *H, const double *dev, double *host) {
    const size_t n = n3(H);
    k3_scatter<<<nblk(n), 128, 0, H->stream>>>(dev, H->perm, H->npfb, H->nz, n, H->tmp3);
    SUNSET_CUDA(H, cudaGetLastError());
    SUNSET_CUDA(H, cudaMemcpyAsync(host, H->tmp3, n * sizeof(double), cudaMemcpyDeviceToHost, H->stream));
    SUNSET_CUDA(H, cudaStreamSynchronize(H->stream));
    return 0;
}

// out10: the right-hand sides ro rou rov row xx xy yy xz yz zz, reference layer-major, host
int rhs3_calc(Handle *H, double *out10) {
    const size_t n = n3(H);
    if (int rc = stage3(H, H->cur3, 4)) return rc;
    for (int q = 0; q < 10; q++) {
        k3_scatter<<<nblk(n), 128, 0, H->stream>>>(H->rhs3[q], H->perm, H->npfb, H->nz, n, H->tmp3);
        SUNSET_CUDA(H, cudaMemcpyAsync(out10 + (size_t)q * n, H->tmp3, n * sizeof(double), cudaMemcpyDeviceToHost, H->stream));
        SUNSET_CUDA(H, cudaStreamSynchronize(H->stream));
    }
    return 0;
}

int tstep3(Handle *H) { return tstep3_launch(H, H->cur3, 0); }

// mode 0: fixed dt; 1: set_tstep + set_tstep_PID before each step (sunset.F90:82-83)
int step3_run(Handle *H, double dt, int nsteps, int mode, cudaEvent_t *ev) {
    const size_t n = n3(H);
    cudaStream_t st = H->stream;
    const Layer3 L = layer3(H);
    const bool chl = H->cfg.form == SUNSET_FORM_CHL, lc = H->cfg.form == SUNSET_FORM_LC;
    const bool evolves_c = H->cfg.form != SUNSET_FORM_NEWT;
    if (mode == 0) SUNSET_CUDA(H, cudaMemcpyAsync(&H->dsc->dt, &dt, sizeof(double), cudaMemcpyHostToDevice, st));
    for (int s = 0; s < nsteps; s++) {
        if (mode == 1) {
            if (int rc = tstep3_launch(H, H->cur3, 1)) return rc;
        }
        int b = H->cur3;
        for (int stage = 0; stage < 4; stage++) {
            if (ev) SUNSET_CUDA(H, cudaEventRecord(ev[8 * s + 2 * stage], st));
            if (int rc = stage3(H, b, stage)) return rc;
            if (ev) SUNSET_CUDA(H, cudaEventRecord(ev[8 * s + 2 * stage + 1], st));
            b ^= 1;
        }
        // filter_variables: ro rou rov row, then c (rhs_di.F90:667-694) or psi (rhs.F90:792-840);
        // the mass correction
        // (the derivative scratch holds the x-y filtered values)
        const int c0 = (chl || lc) ? 13 : 7;
        const int fld[10] = {0, 1, 2, 3, c0, c0 + 1, c0 + 2, c0 + 3, c0 + 4, c0 + 5};
        Filter3 FA{};
        for (int q = 0; q < 10; q++) {
            FA.f[q] = H->f3[b][fld[q]];
            FA.t[q] = H->g3 + (size_t)q * n;
        }
        if (evolves_c) {
            const bool chlf = chl && H->cfg.fenep;  // rhs.F90:816-868: filter the factors of c
            if (chlf) k3_fenep_factors<<<nblk(n), 128, 0, st>>>(n, FA, H->cfg.fenep_l2, 1);
            k3_filter_xy<10><<<zblocks(H), 128, 0, st>>>(L, FA);
            k3_filter_z<10><<<zblocks(H), 128, 0, st>>>(L, FA);
            if (chlf) k3_fenep_factors<<<nblk(n), 128, 0, st>>>(n, FA, H->cfg.fenep_l2, 0);
        } else {
            k3_filter_xy<4><<<zblocks(H), 128, 0, st>>>(L, FA);
            k3_filter_z<4><<<zblocks(H), 128, 0, st>>>(L, FA);
        }
        k3_mass_partials<<<nblk(n), 128, 0, st>>>(H->nz, n, H->f3[b][0], H->vol, 1.0, 0, H->partials3);
        k3_fold<<<1, kFoldThreads, 0, st>>>(H->partials3, (int)nblk(n), &H->dsc->dro, &H->dsc->tv, H->cfg.mcorr);
        Fields3 F19;
        for (int q = 0; q < 19; q++) F19.p[q] = H->f3[b][q];
        k3_finalize<<<nblk(n), 128, 0, st>>>(n, H->nz, H->nb > 0 ? H->ntype : nullptr, H->uin3, H->cfg.inflow_type == 1, F19, chl, lc,
                                             H->cfg.fenep ? H->cfg.fenep_l2 : 0.0, H->dsc, H->cfg.vpid);
        if (H->cfg.vpid) {  // statistics_control after the step (sunset.F90:104)
            const size_t off = nblk(n) + 16;
            k3_flow_partials<<<nblk(n), 128, 0, st>>>(H->nz, n, H->f3[b][4], H->vol, H->dz, H->partials3 + off,
                                                      H->partials3 + 2 * off);
            const double L = H->cfg.L_char;
            k3_velocity_control<<<1, kFlowThreads, 0, st>>>(H->partials3 + off, H->partials3 + 2 * off, (int)nblk(n),
                                                          (H->xmax - H->xmin) * L, (H->ymax - H->ymin) * L, H->dsc);
        }
        SUNSET_CUDA(H, cudaGetLastError());
        H->cur3 = b;
    }
    return tstep3_launch(H, H->cur3, 0);
}


// The 13 columns of the 3-D fields dump (output_layer, output.F90:184-310 with -Dallout, every
// node-layer): rho - rho_char, u, v, w, the vorticity magnitude from the 3-D velocity gradient
// (calc_gradient: the layer's x-y weights, on walls in the normal-tangent frame and turned
// there as :226-235 does, and the z stencil), Q (which the reference never sets in 3-D: 0),
// alpha_out, then c xx xy yy xz yz zz.  Internal order, one column after another.
__global__ void k3_dump(Layer3 L, Fields3 F, const int *ntype, const double *rnx, const double *rny, const double *alpha,
                        double rho_char, double *out) {
    const size_t n = (size_t)L.nl * L.nz;
    const size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int i = (int)((unsigned)k / (unsigned)L.nz), iz = (int)k - i * L.nz, row = i * L.nz, h = L.ncfd / 2;
    const double *fu = F.p[4], *fv = F.p[5], *fw = F.p[6];
    double g[3][3];  // [u v w][x y z]
    const double *ff[3] = {fu, fv, fw};
    const int cls[3] = {1, 2, 0};
    const long long base = L.slice_ptr[i >> 5];
    for (int f = 0; f < 3; f++) {
        double sx = 0.0, sy = 0.0, sz = 0.0;
        for (int q = 0; q < L.cnt_small[i]; q++) {
            const long long o = sell_at(base, q, i & 31);
            const int l = L.lidx[o];
            const double x = mirror_value(ff[f][(l & kLinkMask) * L.nz + iz], cls[f], (int)((unsigned)l >> 30));
            sx = sx + x * L.wx[o];
            sy = sy + x * L.wy[o];
        }
        for (int m = 0; m < L.ncfd; m++) sz = sz + ff[f][row + zwrap(iz + m - h, L.nz)] * L.fdg[m];
        g[f][0] = sx - ff[f][k] * L.gsx[i];
        g[f][1] = sy - ff[f][k] * L.gsy[i];
        g[f][2] = sz;
    }
    double a, b, c;
    if (ntype && ntype[i] == 0) {
        const double xn = rnx[i], yn = rny[i];
        a = g[2][1] - (xn * g[1][2] - yn * g[0][2]);
        b = (xn * g[0][2] + yn * g[1][2]) - g[2][0];
        c = (((xn * g[1][0]) - yn * g[0][0]) - xn * g[0][1]) - yn * g[1][1];
    } else {
        a = g[2][1] - g[1][2];
        b = g[0][2] - g[2][0];
        c = g[1][0] - g[0][1];
    }
    const double vort = sqrt((a * a + b * b) + c * c);
    const double col[13] = {-rho_char + F.p[0][k], fu[k], fv[k], fw[k], vort, 0.0, alpha[k],
                            F.p[7][k], F.p[8][k], F.p[9][k], F.p[10][k], F.p[11][k], F.p[12][k]};
    for (int q = 0; q < 13; q++) out[(size_t)q * n + k] = col[q];
}
int dump3_columns(Handle *H, double *out13) {
    const size_t n = n3(H);
    Fields3 F{};
    for (int q = 0; q < 19; q++) F.p[q] = H->f3[H->cur3][q];
    k3_dump<<<nblk(n), 128, 0, H->stream>>>(layer3(H), F, H->nb > 0 ? H->ntype : nullptr, H->rnx, H->rny, H->alpha3, 1.0,
                                            out13);
    SUNSET_CUDA(H, cudaGetLastError());
    return 0;
}

// Checkpoint of a 3-D handle: the 19 fields of the current buffer, the step's scalars, the
// node-layers' step error and (with boundary nodes) u_inflow_local, in the internal order,
// behind a header that names the configuration, the layers and the node set's fingerprint.
namespace {
struct Checkpoint3Header {
    char magic[8];
    int version, npfb, nz, form, fenep, nb;
    double dz, xsum, ysum;
};
}  // namespace
size_t checkpoint3_bytes(const Handle *H) {
    return sizeof(Checkpoint3Header) + sizeof(DevScalars) + (20 + (H->nb > 0 ? 1 : 0)) * n3(H) * sizeof(double);
}
static int checkpoint3_header(Handle *H, Checkpoint3Header &hd) {
    memset(&hd, 0, sizeof(hd));
    memcpy(hd.magic, "SUNSET3D", 8);
    hd.version = 1;
    hd.npfb = H->npfb;
    hd.nz = H->nz;
    hd.form = H->cfg.form;
    hd.fenep = H->cfg.fenep;
    hd.nb = H->nb;
    hd.dz = H->dz;
    std::vector<double> x(H->npfb), y(H->npfb);
    SUNSET_CUDA(H, cudaMemcpy(x.data(), H->px, H->npfb * sizeof(double), cudaMemcpyDeviceToHost));
    SUNSET_CUDA(H, cudaMemcpy(y.data(), H->py, H->npfb * sizeof(double), cudaMemcpyDeviceToHost));
    for (int i = 0; i < H->npfb; i++) { hd.xsum = hd.xsum + x[i]; hd.ysum = hd.ysum + y[i]; }
    return 0;
}
int checkpoint3_save(Handle *H, void *buf) {
    Checkpoint3Header hd;
    if (int rc = checkpoint3_header(H, hd)) return rc;
    const size_t n = n3(H);
    char *p = static_cast<char *>(buf);
    memcpy(p, &hd, sizeof(hd));
    p += sizeof(hd);
    SUNSET_CUDA(H, cudaMemcpyAsync(p, H->dsc, sizeof(DevScalars), cudaMemcpyDeviceToHost, H->stream));
    p += sizeof(DevScalars);
    for (int f = 0; f < 19; f++, p += n * sizeof(double))
        SUNSET_CUDA(H, cudaMemcpyAsync(p, H->f3[H->cur3][f], n * sizeof(double), cudaMemcpyDeviceToHost, H->stream));
    SUNSET_CUDA(H, cudaMemcpyAsync(p, H->alpha3, n * sizeof(double), cudaMemcpyDeviceToHost, H->stream));
    p += n * sizeof(double);
    if (H->nb > 0) SUNSET_CUDA(H, cudaMemcpyAsync(p, H->uin3, n * sizeof(double), cudaMemcpyDeviceToHost, H->stream));
    SUNSET_CUDA(H, cudaStreamSynchronize(H->stream));
    return 0;
}
int checkpoint3_load(Handle *H, const void *buf, size_t bytes) {
    if (bytes != checkpoint3_bytes(H))
        return set_err(H, SUNSET_ERR_ARG, "checkpoint of %zu bytes, expected %zu", bytes, checkpoint3_bytes(H));
    Checkpoint3Header mine, hd;
    if (int rc = checkpoint3_header(H, mine)) return rc;
    const char *p = static_cast<const char *>(buf);
    memcpy(&hd, p, sizeof(hd));
    if (memcmp(hd.magic, mine.magic, 8) != 0 || hd.version != mine.version || hd.npfb != mine.npfb || hd.nz != mine.nz ||
        hd.form != mine.form || hd.fenep != mine.fenep || hd.nb != mine.nb || hd.dz != mine.dz || hd.xsum != mine.xsum ||
        hd.ysum != mine.ysum)
        return set_err(H, SUNSET_ERR_ARG, "checkpoint written for another configuration, layering or node set");
    if (int rc = state3_alloc(H)) return rc;
    const size_t n = n3(H);
    p += sizeof(hd);
    SUNSET_CUDA(H, cudaMemcpyAsync(H->dsc, p, sizeof(DevScalars), cudaMemcpyHostToDevice, H->stream));
    p += sizeof(DevScalars);
    H->cur3 = 0;
    for (int f = 0; f < 19; f++, p += n * sizeof(double))
        SUNSET_CUDA(H, cudaMemcpyAsync(H->f3[0][f], p, n * sizeof(double), cudaMemcpyHostToDevice, H->stream));
    SUNSET_CUDA(H, cudaMemcpyAsync(H->alpha3, p, n * sizeof(double), cudaMemcpyHostToDevice, H->stream));
    p += n * sizeof(double);
    if (H->nb > 0) SUNSET_CUDA(H, cudaMemcpyAsync(H->uin3, p, n * sizeof(double), cudaMemcpyHostToDevice, H->stream));
    // the mass correction's total volume, as sunset_set_state_3d leaves it
    k3_mass_partials<<<nblk(n), 128, 0, H->stream>>>(H->nz, n, H->f3[0][0], H->vol, 1.0, 1, H->partials3);
    k3_fold<<<1, kFoldThreads, 0, H->stream>>>(H->partials3, (int)nblk(n), &H->dsc->tv, nullptr, 1);
    SUNSET_CUDA(H, cudaGetLastError());
    SUNSET_CUDA(H, cudaStreamSynchronize(H->stream));
    return 0;
}

// Kinetic energy and mass of the 3-D state (mass_and_energy_check, statistics.F90:305-330, with
// dV = vol dz): block sums in a fixed tree, the blocks summed in order on the host.
__global__ void k3_ke_mass(int nz, size_t n, const double *ro, const double *u, const double *v, const double *w,
                           const double *vol, double dz, double *pk, double *pm) {
    __shared__ double s1[128], s2[128];
    const size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    double ke = 0.0, m = 0.0;
    if (k < n) {
        const double dv = vol[k / nz] * dz;
        ke = ((0.5 * ro[k]) * ((u[k] * u[k] + v[k] * v[k]) + w[k] * w[k])) * dv;
        m = ro[k] * dv;
    }
    s1[threadIdx.x] = ke;
    s2[threadIdx.x] = m;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) {
            s1[threadIdx.x] = s1[threadIdx.x] + s1[threadIdx.x + s];
            s2[threadIdx.x] = s2[threadIdx.x] + s2[threadIdx.x + s];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        pk[blockIdx.x] = s1[0];
        pm[blockIdx.x] = s2[0];
    }
}
int ke_mass3(Handle *H, double *ke, double *mass) {
    const size_t n = n3(H);
    const unsigned nb = nblk(n), off = nb + 16;
    const double *const *f = H->f3[H->cur3];
    k3_ke_mass<<<nb, 128, 0, H->stream>>>(H->nz, n, f[0], f[4], f[5], f[6], H->vol, H->dz, H->partials3, H->partials3 + off);
    SUNSET_CUDA(H, cudaGetLastError());
    std::vector<double> pk(nb), pm(nb);
    SUNSET_CUDA(H, cudaMemcpyAsync(pk.data(), H->partials3, nb * sizeof(double), cudaMemcpyDeviceToHost, H->stream));
    SUNSET_CUDA(H, cudaMemcpyAsync(pm.data(), H->partials3 + off, nb * sizeof(double), cudaMemcpyDeviceToHost, H->stream));
    SUNSET_CUDA(H, cudaStreamSynchronize(H->stream));
    double a = 0.0, b = 0.0;
    for (unsigned q = 0; q < nb; q++) { a += pk[q]; b += pm[q]; }
    if (ke) *ke = a;
    if (mass) *mass = b;
    return 0;
}

int time3_derivs(Handle *H, int reps, double *ms, double *bytes) {
    if (reps < 1) reps = 1;
    DevScalars s;
    SUNSET_CUDA(H, cudaMemcpy(&s, H->dsc, sizeof(s), cudaMemcpyDeviceToHost));
    std::vector<cudaEvent_t> ev(8 * (size_t)reps);
    for (auto &e : ev) SUNSET_CUDA(H, cudaEventCreate(&e));
    int rc = step3_run(H, s.dt, reps, 0, ev.data());
    SUNSET_CUDA(H, cudaStreamSynchronize(H->stream));
    double tot = 0.0;
    for (int k = 0; k < 4 * reps && !rc; k++) {
        float t = 0.f;
        SUNSET_CUDA(H, cudaEventElapsedTime(&t, ev[2 * k], ev[2 * k + 1]));
        tot += t;
    }
    for (auto &e : ev) cudaEventDestroy(e);
    if (rc) return rc;
    *ms = tot / (4.0 * reps);
    // Algorithmic bytes of one fused stage launch (k3_stage), averaged over the four stages:
    // the state fields the stage reads (gathered or pointwise, 8 bytes a node-layer each) once,
    // the next state and its derived fields written once, the RK registers S and E of the ten
    // evolved fields read in stages 1-3 and written in stages 0-2, the step error of each
    // node-layer written by the final stage, the FENE-P function of the
    // direct form read once, the layer's small links once (a 4-byte index and three 8-byte
    // weights; all layers share them) with the three stencil sums and the ordinate of each
    // node of the layer.  Neighbours' values re-read through the caches are not counted.
    const int form = H->cfg.form;
    const int nread = form == SUNSET_FORM_DI ? 13 : form == SUNSET_FORM_NEWT ? 7 : 19;
    const int nwrite = form == SUNSET_FORM_DI ? 13 : form == SUNSET_FORM_NEWT ? 7 : 19;
    const int nevo = form == SUNSET_FORM_NEWT ? 4 : 10;
    long long links = 0;
    {
        std::vector<int> cs(H->npfb);
        SUNSET_CUDA(H, cudaMemcpy(cs.data(), H->cnt_small, cs.size() * sizeof(int), cudaMemcpyDeviceToHost));
        for (int c : cs) links += c;
    }
    const double fen = (form == SUNSET_FORM_DI && H->cfg.fenep) ? 8.0 : 0.0;
    *bytes = (double)n3(H) * (8.0 * (nread + nwrite) + 16.0 * nevo * 6.0 / 4.0 + 8.0 / 4.0 + fen) + (double)links * 28.0 +
             (double)H->npfb * 32.0;
    return 0;
}

}  // namespace sunset
