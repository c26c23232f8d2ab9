// weights.cu -- LABFM weight construction on the device (labf.F90, svdlib.F90, rbfs.F90).
//
// One warp builds the weights of one node: it assembles the moment matrix
// A = sum_k X(r_k/h) [W(r_k/h) H(r_k/h)]^T (monomials X, Hermite ABFs H, Wendland C2 W)
// in shared memory, factors it with the reference's Golub-Kahan-Reinsch SVD and applies
// the factorisation to each right-hand side.  The SVD is the reference's algorithm with
// its serial recurrences kept serial: lanes split only loops whose iterations are
// independent (columns of a Householder update, rows of a Givens rotation), and every
// dot product is summed by one lane in the reference's order.  With -fmad=false each
// operation then rounds exactly as the reference's does, so the factorisation - and the
// weights - are those of the CPU restatement bit for bit.
//
// The five SVDs of identical matrix copies in labf.F90:157-180 become one factorisation
// applied to five right-hand sides; the filter matrix (labf.F90:258-303) is the same
// matrix whenever h == h_small, the counts agree and the order drops agree, and is then
// not factored again.
#include <cmath>

#include "internal.cuh"

namespace sunset {

namespace {

__host__ __device__ constexpr int nsz(int k) { return (k * k + 3 * k) / 2; }

// (p, q) exponents of unknown m in the reference's degree-graded ordering
// (labf.F90:1815-1920): degree d, p from d down to 0.
__host__ __device__ constexpr int deg_of(int m) {
    int d = 1, base = 0;
    while (m >= base + d + 1) { base += d + 1; d++; }
    return d;
}
__host__ __device__ constexpr int p_of(int m) {
    int d = 1, base = 0;
    while (m >= base + d + 1) { base += d + 1; d++; }
    return d - (m - base);
}
__host__ __device__ constexpr int q_of(int m) { return deg_of(m) - p_of(m); }

__device__ __forceinline__ double fact(int k) {
    double f = 1.0;
    for (int j = 2; j <= k; j++) f *= (double)j;
    return f;
}

// labf.F90:2329-2391 probabilists' Hermite polynomials, in the reference's operation order.
__device__ __forceinline__ double hermite(int n, double z) {
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

// x^p y^q / (p! q!) as written in labf.F90:1815-1920: x2=x*x, x3=x2*x, ..., then
// (coef*x^p)*y^q.
__device__ __forceinline__ double monomial(int p, int q, double x, double y) {
    double xp = x, yq = y;
    for (int k = 2; k <= p; k++) xp = xp * x;
    for (int k = 2; k <= q; k++) yq = yq * y;
    double den = fact(p) * fact(q);
    if (den == 1.0) {
        if (p == 0) return yq;
        if (q == 0) return xp;
        return xp * yq;
    }
    double c = 1.0 / den;
    if (q == 0) return c * xp;
    if (p == 0) return c * yq;
    return (c * xp) * yq;
}

// x^4 correctly rounded.  The reference evaluates (1-q/2)**4.0 with libm pow; glibc's pow
// returns the correctly rounded power for these arguments, which this reproduces with an
// exact double-double product (Dekker's two-product, built on fma) rounded once.
__device__ __forceinline__ double pow4_cr(double x) {
    double a = x * x;
    double ae = fma(x, x, -a);           // x*x = a + ae exactly
    double b = a * a;                     // (a + ae)^2 = a^2 + 2 a ae + ae^2
    double be = fma(a, a, -b);            // a*a = b + be exactly
    double t = fma(2.0 * a, ae, be);      // small terms
    t = fma(ae, ae, t);
    return b + t;
}

// rbfs.F90:48-57, Wendland C2 (zero at q=0 and q>2).
__device__ __forceinline__ double wab(double qq, double h2) {
    double qq4 = 1.0 - 0.5 * qq;
    qq4 = pow4_cr(qq4);
    double f = 0.0;
    if (qq <= 2.0 && qq > 0.0) f = ((7.0 / ((4.0 * kPi) * h2)) * (2.0 * qq + 1.0)) * qq4;
    return f;
}

__device__ __forceinline__ double nr_hypot(double a, double b) {  // svdlib.F90:308-327
    double absA = fabs(a), absB = fabs(b), t;
    if (absA > absB) {
        t = absB / absA;
        return absA * sqrt(1.0 + t * t);
    }
    if (absB == 0.0) return 0.0;
    t = absA / absB;
    return absB * sqrt(1.0 + t * t);
}

// Shared scalars are written by lane 0 between two warp barriers, so no lane reads a
// half-updated value and every lane sees the new one.
__device__ __forceinline__ void wstore(double *p, double v, int lane) {
    __syncwarp();
    if (lane == 0) *p = v;
    __syncwarp();
}

// svdlib.F90:37-278 on a warp.  U (in: A, out: U) and V are column-major n x n with
// leading dimension ld; W and rv1 are 1-based.  Returns 0 or -1 (no convergence within
// maxits QR sweeps per singular value; the reference's limit is 30).
template <int N>
__device__ int svd_factor_warp(double *U, double *V, double *W, double *rv1, int ld, int lane, int maxits = 30) {
    const int n = N;
#define UM(i, j) U[((j) - 1) * ld + ((i) - 1)]
#define VM(i, j) V[((j) - 1) * ld + ((i) - 1)]
    double anorm = 0.0, c, f, g = 0.0, h, s, scale = 0.0, x, y, z;
    int l = 1, nm;
    for (int i = 1; i <= n; i++) {
        l = i + 1;
        wstore(&rv1[i], scale * g, lane);
        g = 0.0; s = 0.0; scale = 0.0;
        for (int k = i; k <= n; k++) scale = scale + fabs(UM(k, i));
        if (scale != 0.0) {
            __syncwarp();
            for (int k = i + lane; k <= n; k += 32) UM(k, i) = UM(k, i) / scale;
            __syncwarp();
            for (int k = i; k <= n; k++) s = s + UM(k, i) * UM(k, i);
            f = UM(i, i);
            g = -copysign(sqrt(s), f);
            h = f * g - s;
            wstore(&UM(i, i), f - g, lane);
            for (int j = l + lane; j <= n; j += 32) {
                double sj = 0.0;
                for (int k = i; k <= n; k++) sj = sj + UM(k, i) * UM(k, j);
                double fj = sj / h;
                for (int k = i; k <= n; k++) UM(k, j) = UM(k, j) + fj * UM(k, i);
            }
            __syncwarp();
            for (int k = i + lane; k <= n; k += 32) UM(k, i) = scale * UM(k, i);
            __syncwarp();
        }
        wstore(&W[i], scale * g, lane);
        g = 0.0; s = 0.0; scale = 0.0;
        for (int k = l; k <= n; k++) scale = scale + fabs(UM(i, k));
        if (scale != 0.0) {
            __syncwarp();
            for (int k = l + lane; k <= n; k += 32) UM(i, k) = UM(i, k) / scale;
            __syncwarp();
            for (int k = l; k <= n; k++) s = s + UM(i, k) * UM(i, k);
            f = UM(i, l);
            g = -copysign(sqrt(s), f);
            h = f * g - s;
            wstore(&UM(i, l), f - g, lane);
            for (int k = l + lane; k <= n; k += 32) rv1[k] = UM(i, k) / h;
            __syncwarp();
            for (int j = l + lane; j <= n; j += 32) {
                double sj = 0.0;
                for (int k = l; k <= n; k++) sj = sj + UM(j, k) * UM(i, k);
                for (int k = l; k <= n; k++) UM(j, k) = UM(j, k) + sj * rv1[k];
            }
            __syncwarp();
            for (int k = l + lane; k <= n; k += 32) UM(i, k) = scale * UM(i, k);
            __syncwarp();
        }
        double t = fabs(W[i]) + fabs(rv1[i]);
        anorm = (t > anorm) ? t : anorm;
    }
    // right-hand transformations, svdlib.F90:115-141
    for (int i = n; i >= 1; i--) {
        if (i < n) {
            if (g != 0.0) {
                __syncwarp();
                for (int j = l + lane; j <= n; j += 32) VM(j, i) = (UM(i, j) / UM(i, l)) / g;
                __syncwarp();
                for (int j = l + lane; j <= n; j += 32) {
                    double sj = 0.0;
                    for (int k = l; k <= n; k++) sj = sj + UM(i, k) * VM(k, j);
                    for (int k = l; k <= n; k++) VM(k, j) = VM(k, j) + sj * VM(k, i);
                }
                __syncwarp();
            }
            for (int j = l + lane; j <= n; j += 32) { VM(i, j) = 0.0; VM(j, i) = 0.0; }
            __syncwarp();
        }
        wstore(&VM(i, i), 1.0, lane);
        g = rv1[i];
        l = i;
    }
    // left-hand transformations, svdlib.F90:143-171
    for (int i = n; i >= 1; i--) {
        l = i + 1;
        g = W[i];
        __syncwarp();
        for (int j = l + lane; j <= n; j += 32) UM(i, j) = 0.0;
        __syncwarp();
        if (g != 0.0) {
            g = 1.0 / g;
            for (int j = l + lane; j <= n; j += 32) {
                double sj = 0.0;
                for (int k = l; k <= n; k++) sj = sj + UM(k, i) * UM(k, j);
                double fj = (sj / UM(i, i)) * g;
                for (int k = i; k <= n; k++) UM(k, j) = UM(k, j) + fj * UM(k, i);
            }
            __syncwarp();
            for (int j = i + lane; j <= n; j += 32) UM(j, i) = UM(j, i) * g;
            __syncwarp();
        } else {
            for (int j = i + lane; j <= n; j += 32) UM(j, i) = 0.0;
            __syncwarp();
        }
        wstore(&UM(i, i), UM(i, i) + 1.0, lane);
    }
    // diagonalisation, svdlib.F90:173-278
    nm = 1;
    for (int k = n; k >= 1; k--) {
        for (int its = 1; its <= 30; its++) {
            bool to2000 = false;
            for (l = k; l >= 1; l--) {
                nm = l - 1;
                if ((fabs(rv1[l]) + anorm) == anorm) { to2000 = true; break; }
                if ((fabs(W[nm]) + anorm) == anorm) break;
            }
            if (!to2000) {
                c = 0.0; s = 1.0;
                for (int i = l; i <= k; i++) {
                    double r = rv1[i];
                    f = s * r;
                    wstore(&rv1[i], c * r, lane);
                    if ((fabs(f) + anorm) == anorm) break;
                    g = W[i];
                    h = nr_hypot(f, g);
                    wstore(&W[i], h, lane);
                    h = 1.0 / h;
                    c = (g * h);
                    s = -(f * h);
                    for (int j = 1 + lane; j <= n; j += 32) {
                        double yy = UM(j, nm), zz = UM(j, i);
                        UM(j, nm) = (yy * c) + (zz * s);
                        UM(j, i) = -(yy * s) + (zz * c);
                    }
                    __syncwarp();
                }
            }
            z = W[k];
            if (l == k) {
                if (z < 0.0) {
                    wstore(&W[k], -z, lane);
                    for (int j = 1 + lane; j <= n; j += 32) VM(j, k) = -VM(j, k);
                    __syncwarp();
                }
                break;
            }
            if (its >= maxits) return -1;
            x = W[l];
            nm = k - 1;
            y = W[nm];
            g = rv1[nm];
            h = rv1[k];
            f = ((y - z) * (y + z) + (g - h) * (g + h)) / ((2.0 * h) * y);
            g = nr_hypot(f, 1.0);
            f = ((x - z) * (x + z) + h * ((y / (f + copysign(g, f))) - h)) / x;
            c = 1.0; s = 1.0;
            for (int j = l; j <= nm; j++) {
                int i = j + 1;
                g = rv1[i];
                y = W[i];
                h = s * g;
                g = c * g;
                z = nr_hypot(f, h);
                wstore(&rv1[j], z, lane);
                c = f / z;
                s = h / z;
                f = (x * c) + (g * s);
                g = -(x * s) + (g * c);
                h = y * s;
                y = y * c;
                for (int jj = 1 + lane; jj <= n; jj += 32) {
                    double xv = VM(jj, j), zv = VM(jj, i);
                    VM(jj, j) = (xv * c) + (zv * s);
                    VM(jj, i) = -(xv * s) + (zv * c);
                }
                z = nr_hypot(f, h);
                wstore(&W[j], z, lane);
                if (z != 0.0) {
                    z = 1.0 / z;
                    c = f * z;
                    s = h * z;
                }
                f = (c * g) + (s * y);
                x = -(s * g) + (c * y);
                for (int jj = 1 + lane; jj <= n; jj += 32) {
                    double yv = UM(jj, j), zv = UM(jj, i);
                    UM(jj, j) = (yv * c) + (zv * s);
                    UM(jj, i) = -(yv * s) + (zv * c);
                }
                __syncwarp();
            }
            wstore(&rv1[l], 0.0, lane);
            wstore(&rv1[k], f, lane);
            wstore(&W[k], x, lane);
        }
    }
    __syncwarp();
    return 0;
#undef UM
#undef VM
}

// svdlib.F90:279-303: b <- V diag(1/w) U^T b (exactly-zero singular values skipped).
template <int N>
__device__ void svd_apply_warp(const double *U, const double *V, const double *W, double *tmp, double *b, int ld,
                               int lane) {
    __syncwarp();
    for (int j = 1 + lane; j <= N; j += 32) {
        double s = 0.0;
        if (W[j] != 0.0) {
            for (int i = 1; i <= N; i++) s = s + U[(j - 1) * ld + (i - 1)] * b[i - 1];
            s = s / W[j];
        }
        tmp[j] = s;
    }
    __syncwarp();
    for (int j = 1 + lane; j <= N; j += 32) {
        double s = 0.0;
        for (int jj = 1; jj <= N; jj++) s = s + V[(jj - 1) * ld + (j - 1)] * tmp[jj];
        b[j - 1] = s;
    }
    __syncwarp();
}

struct WArgs {
    int npfb, morder, forder;
    double h2;
    const double *px, *py, *h, *hs;
    const int *ntype, *cnt, *cnt_small, *lpt;
    const long long *slice_ptr;
    double *wx, *wy, *wl, *wh;
    int *err;
    int maxits;               // QR sweeps per singular value (<= 0: the reference's 30)
    double *cond_d, *cond_f;  // per node sigma_max / sigma_min of the two moment matrices, or null
};

// 2-norm condition number of a factored matrix, sigma_max / sigma_min over W[1..N]
// (infinite when a singular value is exactly zero).  The reference inverts every nonzero
// sigma however small (svdlib.F90:283-293); the library reports it instead of staying
// silent about a near-singular stencil.
template <int N>
__device__ __forceinline__ double svd_cond(const double *W) {
    double smax = 0.0, smin = INFINITY;
    for (int j = 1; j <= N; j++) {
        const double w = fabs(W[j]);
        smax = w > smax ? w : smax;
        smin = w < smin ? w : smin;
    }
    return smin > 0.0 ? smax / smin : INFINITY;
}

__device__ __forceinline__ long long sell_off(const long long *slice_ptr, int i, int k) {
    return sell_at(slice_ptr[i >> 5], k, i & 31);
}

// Moment matrix over links [0,cnt) of node i with length scale hh (labf.F90:88-123).
template <int ORDER>
__device__ void assemble(const WArgs &a, int i, int cnt, double hh, double *U, int ld, double *X, double *G,
                         int lane) {
    constexpr int n = nsz(ORDER);
    __syncwarp();
    for (int e = lane; e < n * n; e += 32) U[(e / n) * ld + (e % n)] = 0.0;
    const double xi = a.px[i], yi = a.py[i];
    for (int k = 0; k < cnt; k++) {
        int p = a.lpt[sell_off(a.slice_ptr, i, k)];
        double x = -(xi - a.px[p]), y = -(yi - a.py[p]);
        double rad = sqrt(x * x + y * y) / hh;
        double ff1 = wab(rad, a.h2);
        double xx = x / hh, yy = y / hh;
        __syncwarp();
        for (int m = lane; m < n; m += 32) {
            int pm = p_of(m), qm = q_of(m);
            X[m] = monomial(pm, qm, x / hh, y / hh);
            double g = (qm == 0) ? hermite(pm, xx) : (pm == 0) ? hermite(qm, yy) : hermite(pm, xx) * hermite(qm, yy);
            G[m] = g * ff1;
        }
        __syncwarp();
        for (int e = lane; e < n * n; e += 32) {
            int i1 = e % n, i2 = e / n;
            double *u = &U[i2 * ld + i1];
            *u = *u + X[i1] * G[i2];
        }
    }
    __syncwarp();
}

// labf.F90:125-148: keep the first m unknowns.
template <int N>
__device__ void drop_order(double *U, int ld, int m, int lane) {
    __syncwarp();
    for (int e = lane; e < N * N; e += 32) {
        int i1 = e % N, i2 = e / N;
        if (i2 >= m || i1 >= m) U[i2 * ld + i1] = (i1 == i2) ? 1.0 : 0.0;
    }
    __syncwarp();
}

__device__ void hyp_rhs(int order, double *b, int n, int lane) {
    __syncwarp();
    for (int m = lane; m < n; m += 32) b[m] = 0.0;
    __syncwarp();
    if (lane == 0) {
        if (order <= 5) { b[9] = -1.0; b[11] = -2.0; b[13] = -1.0; }
        else if (order <= 7) { b[20] = 1.0; b[22] = 3.0; b[24] = 3.0; b[26] = 1.0; }
        else if (order <= 9) { b[35] = -1.0; b[37] = -4.0; b[39] = -6.0; b[41] = -4.0; b[43] = -1.0; }
        else { b[54] = 1.0; b[56] = 5.0; b[58] = 10.0; b[60] = 10.0; b[62] = 5.0; b[64] = 1.0; }
    }
    __syncwarp();
}

template <int ORDER>
__host__ __device__ constexpr int smem_doubles() {
    return 2 * nsz(ORDER) * (nsz(ORDER) | 1) + 3 * (nsz(ORDER) + 2) + 7 * nsz(ORDER);
}

template <int ORDER>
__global__ void k_labf_weights(WArgs a) {
    constexpr int n = nsz(ORDER);
    constexpr int ld = n | 1;
    extern __shared__ double smem[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, wpb = blockDim.x >> 5;
    double *U = smem + warp * smem_doubles<ORDER>();
    double *V = U + n * ld, *W = V + n * ld, *rv1 = W + (n + 2), *tmp = rv1 + (n + 2);
    double *X = tmp + (n + 2), *G = X + n, *bx = G + n, *by = bx + n, *bxx = by + n, *byy = bxx + n, *bh = byy + n;
    for (int i = blockIdx.x * wpb + warp; i < a.npfb; i += gridDim.x * wpb) {
        const int t = a.ntype[i];
        if (!(t < 0 || t == 999 || t == 998)) continue;  // boundary nodes: labf.F90:505-1039
        const int cnt = a.cnt[i], cs = a.cnt_small[i];
        double hh = a.hs[i];
        // ---- derivative weights, labf.F90:80-215 ----
        assemble<ORDER>(a, i, cs, hh, U, ld, X, G, lane);
        if (a.morder >= 7 && (t == 998 || t < 0)) drop_order<n>(U, ld, 27, lane);
        if (a.morder >= 5 && (t == -1 || t == -2)) drop_order<n>(U, ld, 14, lane);
        if (svd_factor_warp<n>(U, V, W, rv1, ld, lane, a.maxits > 0 ? a.maxits : 30)) {
            if (lane == 0) atomicExch(a.err, i + 1);
            continue;
        }
        double cond_d = 0.0;
        if (lane == 0) cond_d = svd_cond<n>(W);
        if (lane == 0 && a.cond_d) a.cond_d[i] = cond_d;
        for (int m = lane; m < n; m += 32) {
            bx[m] = (m == 0) ? 1.0 : 0.0;
            by[m] = (m == 1) ? 1.0 : 0.0;
            bxx[m] = (m == 2) ? 1.0 : 0.0;
            byy[m] = (m == 4) ? 1.0 : 0.0;
        }
        svd_apply_warp<n>(U, V, W, tmp, bx, ld, lane);
        svd_apply_warp<n>(U, V, W, tmp, by, ld, lane);
        svd_apply_warp<n>(U, V, W, tmp, bxx, ld, lane);
        svd_apply_warp<n>(U, V, W, tmp, byy, ld, lane);
        for (int m = lane; m < n; m += 32) bxx[m] = bxx[m] + byy[m];  // bvecxx + bvecyy
        __syncwarp();
        const double xi = a.px[i], yi = a.py[i];
        for (int k = lane; k < cnt; k += 32) {
            int p = a.lpt[sell_off(a.slice_ptr, i, k)];
            double x = -(xi - a.px[p]), y = -(yi - a.py[p]);
            double rad = sqrt(x * x + y * y) / hh;
            double ff1 = wab(rad, a.h2);
            double xx = x / hh, yy = y / hh;
            double hx[ORDER + 1], hy[ORDER + 1];
#pragma unroll
            for (int d = 0; d <= ORDER; d++) { hx[d] = hermite(d, xx); hy[d] = hermite(d, yy); }
            double sx = 0.0, sy = 0.0, sl = 0.0;
#pragma unroll
            for (int m = 0; m < n; m++) {
                constexpr int dummy = 0;
                (void)dummy;
                const int pm = p_of(m), qm = q_of(m);
                double g = (qm == 0) ? hx[pm] : (pm == 0) ? hy[qm] : hx[pm] * hy[qm];
                g = g * ff1;
                sx = sx + bx[m] * g;
                sy = sy + by[m] * g;
                sl = sl + bxx[m] * g;
            }
            long long o = sell_off(a.slice_ptr, i, k);
            a.wx[o] = sx / hh;
            a.wy[o] = sy / hh;
            a.wl[o] = (sl / hh) / hh;
        }
        // ---- filter weights, calc_filter_weights (labf.F90:258-388) ----
        const double hf = a.h[i];
        const bool same = (hf == hh) && (cnt == cs) && (a.forder == a.morder) && (t != -2);
        if (!same) {
            assemble<ORDER>(a, i, cnt, hf, U, ld, X, G, lane);
            if (a.forder >= 7 && (t == 998 || t < 0)) drop_order<n>(U, ld, 27, lane);
            if (a.forder >= 5 && t == -1) drop_order<n>(U, ld, 14, lane);
            if (svd_factor_warp<n>(U, V, W, rv1, ld, lane, a.maxits > 0 ? a.maxits : 30)) {
                if (lane == 0) atomicExch(a.err, i + 1);
                continue;
            }
            if (lane == 0) cond_d = svd_cond<n>(W);
        }
        if (lane == 0 && a.cond_f) a.cond_f[i] = cond_d;
        int hord = a.forder;
        if (a.forder >= 7 && (t == 998 || t < 0)) hord = 6;
        if (a.forder >= 5 && t == -1) hord = 4;
        hyp_rhs(hord, bh, n, lane);
        svd_apply_warp<n>(U, V, W, tmp, bh, ld, lane);
        for (int k = lane; k < cnt; k += 32) {
            int p = a.lpt[sell_off(a.slice_ptr, i, k)];
            double x = -(xi - a.px[p]), y = -(yi - a.py[p]);
            double rad = sqrt(x * x + y * y) / hf;
            double ff1 = wab(rad, a.h2);
            double xx = x / hf, yy = y / hf;
            double hx[ORDER + 1], hy[ORDER + 1];
#pragma unroll
            for (int d = 0; d <= ORDER; d++) { hx[d] = hermite(d, xx); hy[d] = hermite(d, yy); }
            double sh = 0.0;
#pragma unroll
            for (int m = 0; m < n; m++) {
                const int pm = p_of(m), qm = q_of(m);
                double g = (qm == 0) ? hx[pm] : (pm == 0) ? hy[qm] : hx[pm] * hy[qm];
                g = g * ff1;
                sh = sh + bh[m] * g;
            }
            a.wh[sell_off(a.slice_ptr, i, k)] = sh;
        }
        __syncwarp();
    }
}

// calc_labf_sums (labf.F90:396-451) and calc_node_volumes (:453-503), one thread per node;
// link k of a slice is read by the 32 threads of a warp at once.
struct SumArgs {
    int npfb;
    double L;
    const double *px, *py, *h, *sp;
    const int *ntype, *cnt, *lpt, *fdpar;
    const long long *slice_ptr;
    double *wx, *wy, *wl, *wh, *gsx, *gsy, *lsum, *hsum, *vol;
};

__global__ void k_labf_sums(SumArgs a) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.npfb) return;
    const long long base = a.slice_ptr[i >> 5];
    const int lane = i & 31;
    const int cnt = a.cnt[i];
    double gx = 0.0, gy = 0.0, lp = 0.0, hy = 0.0;
    for (int k = 0; k < cnt; k++) {
        long long o = sell_at(base, k, lane);
        hy = hy + a.wh[o];
        gx = gx + a.wx[o];
        gy = gy + a.wy[o];
        lp = lp + a.wl[o];
    }
    a.gsx[i] = gx / a.L;
    a.gsy[i] = gy / a.L;
    a.lsum[i] = (lp / a.L) / a.L;
    a.hsum[i] = hy;
    for (int k = 0; k < cnt; k++) {
        long long o = sell_at(base, k, lane);
        a.wx[o] = a.wx[o] / a.L;
        a.wy[o] = a.wy[o] / a.L;
        a.wl[o] = (a.wl[o] / a.L) / a.L;
    }
    const int t = a.ntype[i];
    if (t < 0 || t == 999 || t == 998) {
        const double hh = a.h[i], xi = a.px[i], yi = a.py[i];
        double v = 0.0;
        for (int k = 0; k < cnt; k++) {
            int p = a.lpt[sell_at(base, k, lane)];
            double x = -(xi - a.px[p]), y = -(yi - a.py[p]);
            double rad = sqrt(x * x + y * y) / hh;
            double f1 = ((9.0 / kPi) * exp((-9.0 * rad) * rad)) / (hh * hh);
            v = v + f1;
        }
        a.vol[i] = 1.0 / v;
    } else {
        a.vol[i] = a.sp[i] * a.sp[i];
    }
}

// filter_coefficients, labf.F90:1723-1811, with the reduction of the FD rows of walls.
__global__ void k_filter_coeff(SumArgs a) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.npfb) return;
    const long long base = a.slice_ptr[i >> 5];
    const int lane = i & 31;
    const int cnt = a.cnt[i];
    const double xi = a.px[i], yi = a.py[i];
    const int t = a.ntype[i];
    double fc;
    if (t < 0 || t == 999 || t == 998) {
        double lscal = (2.0 * a.h[i]) * sqrt(kPi / (double)cnt);
        double tmp = ((2.0 / 3.0) * kPi) / lscal;
        double lsum = 0.0;
        for (int k = 0; k < cnt; k++) {
            long long o = sell_at(base, k, lane);
            int p = a.lpt[o];
            double x = a.px[p] - xi, y = a.py[p] - yi;
            double fji = 1.0 - cos(tmp * x) * cos(tmp * y);
            lsum = lsum + fji * a.wh[o];
        }
        fc = (2.0 / 3.0) / lsum;
        if (t < 0 && a.ntype[a.fdpar[i]] == 0) {
            const double oosqrt2 = 1.0 / sqrt(2.0);
            if (t == -1) fc = (fc * 0.5) * oosqrt2;
            if (t == -2) fc = fc * 0.5;
            if (t == -3) fc = fc * oosqrt2;
            if (t == -4) fc = fc * oosqrt2;
        }
    } else {
        double tmp = ((2.0 / 3.0) * kPi) / a.sp[i];
        double lsum = 0.0;
        for (int k = 0; k < cnt; k++) {
            long long o = sell_at(base, k, lane);
            int p = a.lpt[o];
            double x = a.px[p] - xi, y = a.py[p] - yi;
            double fji = 1.0 - cos(tmp * sqrt(x * x + y * y));
            lsum = lsum + fji * a.wh[o];
        }
        fc = (1.0 / 3.0) / lsum;
        fc = fc * 0.5;
    }
    double sum = 0.0;
    for (int k = 0; k < cnt; k++) {
        long long o = sell_at(base, k, lane);
        double w = a.wh[o] * fc;
        a.wh[o] = w;
        sum = sum + w;
    }
    a.hsum[i] = sum;
}

// ---------------------------------------------------------------------------------------
// calc_boundary_weights (labf.F90:505-1039): boundary node i0 and its FD rows i1..i4.
// Normal first and second derivatives of i0, i1, i2 are the reference's 5-point finite
// differences; tangential ones come from 6th-order 1-D LABFM on the node's own layer (a
// 6 x 6 moment matrix, factored by the warp SVD above, so bit for bit the restatement's);
// then the wall curvature, the divergence term of rows 1-2 and the rotation of rows 1-2 to
// the x-y frame.  Wall first derivatives stay in the normal-tangent frame: the wall
// equations are written there.
// ---------------------------------------------------------------------------------------
struct BndArgs {
    int npfb, nb, nplink;
    double h3;
    const double *px, *py, *h, *sp, *rnx, *rny;
    const int *ntype, *gpar, *fdpar, *blist, *brow;
    int *cnt, *cnt_small, *lpt, *lidx;
    uint16_t *lloc;
    const long long *slice_ptr;
    const int *slice_w;
    double *wx, *wy, *wl, *wh;
    double *wb2;  // nb x nplink x 2: second derivatives (normal, tangential) of boundary nodes
    int *err;
};

// point p (interior or ghost) -> the interior node whose data it carries
__device__ __forceinline__ int bnd_owner(const BndArgs &a, int p) { return p < a.npfb ? p : a.gpar[p - a.npfb]; }

// rbfs.F90:58-68 (the kernel derivative `fac` of the 1-D operators; it uses the global h3)
__device__ __forceinline__ double fac(double qq, double h3) {
    double qq2 = qq * qq, qq3 = qq * qq2, qq4 = qq * qq3;
    double f = 0.0;
    if (qq <= 2.0 && qq > 0.0)
        f = (7.0 / ((4.0 * kPi) * h3)) * ((((0.625 * qq4) - (3.75 * qq3)) + (7.5 * qq2)) - (5.0 * qq));
    return f;
}

// labf.F90:1041-1048
__device__ __forceinline__ double monomial1d(int m, double z) {
    double z2 = z * z;
    switch (m) {
    case 0: return z;
    case 1: return 0.5 * z2;
    case 2: return ((1.0 / 6.0) * z) * z2;
    case 3: return (z2 * z2) / 24.0;
    case 4: return ((z2 * z2) * z) / 120.0;
    default: return ((z2 * z2) * z2) / 720.0;
    }
}

// labf.F90:1050-1077 (ABF==2)
__device__ __forceinline__ double abf1d(int m, double z, double ff1) {
    if (m == 2) return (ff1 * (1.0 / sqrt(2.0))) * hermite(3, z);
    return ff1 * hermite(m + 1, z);
}

// tangential coordinate (scaled by hh) of point p relative to node i, and its kernel value
__device__ __forceinline__ void tangential(const BndArgs &a, int i, int p, double xt, double yt, double hh,
                                           double &z, double &ff1) {
    double rijx = a.px[i] - a.px[p], rijy = a.py[i] - a.py[p];
    double x = -(rijx * xt + rijy * yt);
    if (i == p) x = 0.0;
    ff1 = fac(fabs(x / hh), a.h3);
    z = x / hh;
}

__device__ __forceinline__ double dot6(const double *b, const double *g) {
    double t = 0.0;
    for (int k = 0; k < 6; k++) t = t + b[k] * g[k];
    return t;
}

constexpr int kBndWarpDoubles = 2 * 6 * 7 + 3 * 8 + 3 * 6;  // U, V, W/rv1/tmp, three right-hand sides

// 1-D moment matrix of node i along (xt, yt) over its links on its own layer, then its
// factorisation; lanes 0..35 each own one matrix entry and sum it over the links in order.
__device__ int bnd_factor_1d(const BndArgs &a, int i, double xt, double yt, double hh, double *U, double *V,
                             double *W, double *rv1, int lane) {
    const long long base = a.slice_ptr[i >> 5];
    const int ti = a.ntype[i], cnt = a.cnt[i];
    for (int e = lane; e < 36; e += 32) {
        const int i1 = e % 6, i2 = e / 6;
        double acc = 0.0;
        for (int k = 0; k < cnt; k++) {
            const int p = a.lpt[sell_at(base, k, i & 31)];
            if (a.ntype[bnd_owner(a, p)] != ti) continue;
            double rijx = a.px[i] - a.px[p], rijy = a.py[i] - a.py[p];
            double x = -(rijx * xt + rijy * yt);
            if (i == p) x = 0.0;
            const double xv = monomial1d(i1, x / hh);
            double z, ff1;
            tangential(a, i, p, xt, yt, hh, z, ff1);
            acc = acc + xv * abf1d(i2, z, ff1);
        }
        U[i2 * 7 + i1] = acc;
    }
    __syncwarp();
    return svd_factor_warp<6>(U, V, W, rv1, 7, lane);
}

// Drop every link of boundary node jj that is neither on its own layer nor one of its FD
// children (labf.F90:541-565), compacting the SELL slots in order; the freed slots become
// padding.
__global__ void k_prune_boundary_links(BndArgs a) {
    const int jj = blockIdx.x * blockDim.x + threadIdx.x;
    if (jj >= a.nb) return;
    const int i = a.blist[jj], kk = a.ntype[i], c = a.cnt[i];
    const long long base = a.slice_ptr[i >> 5];
    const int ln = i & 31;
    int w = 0;
    for (int k = 0; k < c; k++) {
        const long long o = sell_at(base, k, ln);
        const int p = a.lpt[o];
        const bool keep = (a.ntype[bnd_owner(a, p)] == kk) || (p < a.npfb && a.fdpar[p] == i);
        if (!keep) continue;
        const long long o2 = sell_at(base, w, ln);
        a.lpt[o2] = p;
        a.lidx[o2] = a.lidx[o];
        a.lloc[o2] = a.lloc[o];
        w++;
    }
    for (int k = w; k < c; k++) {
        const long long o = sell_at(base, k, ln);
        a.lpt[o] = 0;
        a.lidx[o] = 0;
        a.lloc[o] = 0;
    }
    a.cnt[i] = w;
    a.cnt_small[i] = w;
}

// Boundary nodes: normal FD operators (labf.F90:572-612) and tangential 1-D LABFM
// (:688-755).  One warp per boundary node.
__global__ void k_boundary_node_weights(BndArgs a) {
    __shared__ double sm[4][kBndWarpDoubles];
    const int lane = threadIdx.x & 31, wrp = threadIdx.x >> 5;
    const int jj = blockIdx.x * 4 + wrp;
    if (jj >= a.nb) return;
    double *U = sm[wrp], *V = U + 42, *W = V + 42, *rv1 = W + 8, *tmp = rv1 + 8, *bt = tmp + 8, *btt = bt + 6,
           *bh = btt + 6;
    const int i = a.blist[jj];
    const long long base = a.slice_ptr[i >> 5];
    const int ln = i & 31, cnt = a.cnt[i];
    const double dx = a.sp[i], dx2 = dx * dx;
    double *wb = a.wb2 + (size_t)jj * a.nplink * 2;
    for (int k = lane; k < a.slice_w[i >> 5]; k += 32) {
        const long long o = sell_at(base, k, ln);
        a.wx[o] = 0.0; a.wy[o] = 0.0; a.wl[o] = 0.0; a.wh[o] = 0.0;
    }
    for (int k = lane; k < a.nplink; k += 32) { wb[2 * k] = 0.0; wb[2 * k + 1] = 0.0; }
    __syncwarp();
    for (int k = lane; k < cnt; k += 32) {
        const long long o = sell_at(base, k, ln);
        const int p = a.lpt[o];
        if (p >= a.npfb || a.fdpar[p] != i) continue;
        const int t = a.ntype[p];
        if (t == -1) { a.wx[o] = 4.0 / dx; wb[2 * k] = -((104.0 / 12.0) / dx2); }
        if (t == -2) { a.wx[o] = -(3.0 / dx); wb[2 * k] = (114.0 / 12.0) / dx2; }
        if (t == -3) { a.wx[o] = (4.0 / 3.0) / dx; wb[2 * k] = -((56.0 / 12.0) / dx2); }
        if (t == -4) { a.wx[o] = -(0.25 / dx); wb[2 * k] = (11.0 / 12.0) / dx2; }
    }
    const double xt = -a.rny[i], yt = a.rnx[i], hh = a.h[i];
    __syncwarp();
    if (bnd_factor_1d(a, i, xt, yt, hh, U, V, W, rv1, lane)) {
        if (lane == 0) atomicExch(a.err, i + 1);
        return;
    }
    for (int m = lane; m < 6; m += 32) {
        bt[m] = (m == 0) ? 1.0 : 0.0;
        btt[m] = (m == 1) ? 1.0 : 0.0;
        bh[m] = (m == 3) ? -1.0 : 0.0;
    }
    svd_apply_warp<6>(U, V, W, tmp, bt, 7, lane);
    svd_apply_warp<6>(U, V, W, tmp, btt, 7, lane);
    svd_apply_warp<6>(U, V, W, tmp, bh, 7, lane);
    const int ti = a.ntype[i];
    for (int k = lane; k < cnt; k += 32) {
        const long long o = sell_at(base, k, ln);
        const int p = a.lpt[o];
        if (a.ntype[bnd_owner(a, p)] != ti) continue;
        double z, ff1, g[6];
        tangential(a, i, p, xt, yt, hh, z, ff1);
        for (int m = 0; m < 6; m++) g[m] = abf1d(m, z, ff1);
        a.wy[o] = dot6(bt, g) / hh;
        wb[2 * k + 1] = (dot6(btt, g) / hh) / hh;
        a.wh[o] = a.wh[o] + dot6(bh, g);
    }
}

// FD rows 1 and 2: normal FD operators (labf.F90:615-676) and tangential 1-D LABFM on a
// tangent rotated by the tangential gradient of the resolution (:758-955).  One warp per
// (boundary node, row).
__global__ void k_boundary_row_weights(BndArgs a) {
    __shared__ double sm[4][kBndWarpDoubles];
    const int lane = threadIdx.x & 31, wrp = threadIdx.x >> 5;
    const int w = blockIdx.x * 4 + wrp;
    if (w >= 2 * a.nb) return;
    const int jj = w >> 1, row = 1 + (w & 1);
    double *U = sm[wrp], *V = U + 42, *W = V + 42, *rv1 = W + 8, *tmp = rv1 + 8, *bt = tmp + 8, *btt = bt + 6;
    const int i = a.brow[4 * jj + row - 1], par = a.blist[jj];
    const long long base = a.slice_ptr[i >> 5];
    const int ln = i & 31, cnt = a.cnt[i];
    const double dx = a.sp[i], dx2 = dx * dx;
    for (int k = lane; k < a.slice_w[i >> 5]; k += 32) {
        const long long o = sell_at(base, k, ln);
        a.wx[o] = 0.0; a.wy[o] = 0.0; a.wl[o] = 0.0;
    }
    __syncwarp();
    for (int k = lane; k < cnt; k += 32) {
        const long long o = sell_at(base, k, ln);
        const int p = a.lpt[o];
        if (p >= a.npfb) continue;
        const int t = a.ntype[p];
        const bool same = a.fdpar[p] == par;
        if (row == 1) {
            if (p == par) { a.wx[o] = -(0.25 / dx); a.wl[o] = (11.0 / 12.0) / dx2; }
            if (t == -2 && same) { a.wx[o] = 1.5 / dx; a.wl[o] = (6.0 / 12.0) / dx2; }
            if (t == -3 && same) { a.wx[o] = -(0.5 / dx); a.wl[o] = (4.0 / 12.0) / dx2; }
            if (t == -4 && same) { a.wx[o] = (1.0 / 12.0) / dx; a.wl[o] = -((1.0 / 12.0) / dx2); }
        } else {
            if (p == par) { a.wx[o] = (1.0 / 12.0) / dx; a.wl[o] = -((1.0 / 12.0) / dx2); }
            if (t == -1 && same) { a.wx[o] = -((8.0 / 12.0) / dx); a.wl[o] = (16.0 / 12.0) / dx2; }
            if (t == -3 && same) { a.wx[o] = (8.0 / 12.0) / dx; a.wl[o] = (16.0 / 12.0) / dx2; }
            if (t == -4 && same) { a.wx[o] = -((1.0 / 12.0) / dx); a.wl[o] = -((1.0 / 12.0) / dx2); }
        }
    }
    // tangential gradient of the resolution at the boundary node, in the order of its links
    double grads = 0.0;
    {
        const long long pb = a.slice_ptr[par >> 5];
        for (int k = 0; k < a.cnt[par]; k++) {
            const long long o = sell_at(pb, k, par & 31);
            const int p = a.lpt[o];
            grads = grads + (a.sp[bnd_owner(a, p)] - a.sp[par]) * a.wy[o];
        }
    }
    grads = -atan(grads);
    const double xt = cos(grads) * (-a.rny[i]) - sin(grads) * a.rnx[i];
    const double yt = sin(grads) * (-a.rny[i]) + cos(grads) * a.rnx[i];
    const double hh = a.h[i];
    __syncwarp();
    if (bnd_factor_1d(a, i, xt, yt, hh, U, V, W, rv1, lane)) {
        if (lane == 0) atomicExch(a.err, i + 1);
        return;
    }
    for (int m = lane; m < 6; m += 32) {
        bt[m] = (m == 0) ? 1.0 : 0.0;
        btt[m] = (m == 1) ? 1.0 : 0.0;
    }
    svd_apply_warp<6>(U, V, W, tmp, bt, 7, lane);
    svd_apply_warp<6>(U, V, W, tmp, btt, 7, lane);
    const int ti = a.ntype[i];
    const double sec = 1.0 / cos(grads), tn = tan(grads);
    for (int k = lane; k < cnt; k += 32) {
        const long long o = sell_at(base, k, ln);
        const int p = a.lpt[o];
        if (a.ntype[bnd_owner(a, p)] == ti) {
            double z, ff1, g[6];
            tangential(a, i, p, xt, yt, hh, z, ff1);
            for (int m = 0; m < 6; m++) g[m] = abf1d(m, z, ff1);
            a.wy[o] = dot6(bt, g) / hh;
            a.wl[o] = a.wl[o] + (dot6(btt, g) / hh) / hh;
        }
        a.wy[o] = sec * a.wy[o] - tn * a.wx[o];
    }
}

// Wall curvature, outflow sign, divergence term of rows 1-2, wall Laplacian, rows 1-2 to
// the x-y frame (labf.F90:965-1035).  One thread per boundary node.
__global__ void k_boundary_frame(BndArgs a) {
    const int jj = blockIdx.x * blockDim.x + threadIdx.x;
    if (jj >= a.nb) return;
    const int i = a.blist[jj], ti = a.ntype[i];
    const long long base = a.slice_ptr[i >> 5];
    const int ln = i & 31;
    double *wb = a.wb2 + (size_t)jj * a.nplink * 2;
    double ooR = 0.0;
    if (ti == 0) {
        double tmp_t = 0.0;
        for (int k = 0; k < a.cnt[i]; k++) {
            const int p = a.lpt[sell_at(base, k, ln)];
            const int q = bnd_owner(a, p);
            if (a.ntype[q] != ti) continue;
            const double tmp_n = ((a.rnx[q] * a.rnx[i] + a.rny[q] * a.rny[i]) + 0.0 * 0.0) - 1.0;
            tmp_t = tmp_t + wb[2 * k + 1] * tmp_n;
        }
        ooR = sqrt(fabs(tmp_t));
    }
    if (ti == 2)
        for (int k = 0; k < a.slice_w[i >> 5]; k++) {
            const long long o = sell_at(base, k, ln);
            a.wx[o] = -a.wx[o];
            a.wy[o] = -a.wy[o];
        }
    for (int row = 1; row <= 2; row++) {
        if (ti != 0) break;
        const int r = a.brow[4 * jj + row - 1];
        const long long rb = a.slice_ptr[r >> 5];
        const double den = row == 1 ? 1.0 + ooR * a.sp[r] : 1.0 + (2.0 * ooR) * a.sp[r];
        for (int k = 0; k < a.slice_w[r >> 5]; k++) {
            const long long o = sell_at(rb, k, r & 31);
            a.wl[o] = a.wl[o] + (a.wx[o] * ooR) / den;
        }
    }
    if (ti == 0)
        for (int k = 0; k < a.cnt[i]; k++) {
            const long long o = sell_at(base, k, ln);
            wb[2 * k] = wb[2 * k] + a.wx[o] * ooR;
            a.wl[o] = wb[2 * k] + wb[2 * k + 1];
        }
    const double xn = a.rnx[i], yn = a.rny[i];
    for (int row = 1; row <= 2; row++) {
        const int r = a.brow[4 * jj + row - 1];
        const long long rb = a.slice_ptr[r >> 5];
        for (int k = 0; k < a.cnt[r]; k++) {
            const long long o = sell_at(rb, k, r & 31);
            const double g1 = a.wx[o], g2 = a.wy[o];
            a.wx[o] = (0.0 + xn * g1) + (-yn) * g2;
            a.wy[o] = (0.0 + yn * g1) + xn * g2;
        }
    }
}

// adapt_stencils + adapt_stencils_main (labf.F90:1079-1721), 2-D, Hermite ABFs.  One warp
// per plain interior node (node_type > 2, not 998).  The length scale shrinks by the
// reference's single-precision factor 0.98 while the Laplacian system's residual stays below
// res_tol / h, no wavenumber q = i pi / (32 s), i = 1..33, is amplified beyond 1.0001 by the
// d/dx, d/dy or Laplacian stencil (nor turned negative by the Laplacian), and at most
// `limit` reductions have been made.  Pass 0 reduces h (h_small with it) over the node's
// list, pass 1 h_small over its small list.  The lists are sorted by distance, so the links
// within 2 h are a prefix of each.  The arithmetic follows the CPU restatement operation for
// operation (the same moment matrix, warp SVD and sums in the same order); the amplification
// sums run one wavenumber per lane, each over the links in order.  A moment matrix whose SVD
// does not converge ends the node's reduction (the reference stops).
struct AdaptArgs {
    WArgs w;
    double *h, *hs;
    const double *sp;
    int nplink, per_warp;
    double rf, limit, res_tol[2];
};

template <int ORDER>
__host__ __device__ constexpr int adapt_fixed_doubles() {
    return 2 * nsz(ORDER) * (nsz(ORDER) | 1) + 3 * (nsz(ORDER) + 2) + nsz(ORDER) * (nsz(ORDER) | 1) + 6 * nsz(ORDER);
}

template <int ORDER>
__global__ void k_adapt_stencils(AdaptArgs a) {
    constexpr int n = nsz(ORDER);
    constexpr int ld = n | 1;
    extern __shared__ double smem[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, wpb = blockDim.x >> 5;
    double *U = smem + (size_t)warp * a.per_warp;
    double *V = U + n * ld, *W = V + n * ld, *rv1 = W + (n + 2), *tmp = rv1 + (n + 2), *M = tmp + (n + 2);
    double *X = M + n * ld, *G = X + n, *bl = G + n, *bx = bl + n, *by = bx + n, *R = by + n;
    double *lx = R + n, *ly = lx + a.nplink, *dl = ly + a.nplink, *dxv = dl + a.nplink, *dyv = dxv + a.nplink;
    const WArgs &wa = a.w;
    constexpr double amp_tol = 1.0001;
    constexpr int nk = 32;
    for (int i = blockIdx.x * wpb + warp; i < wa.npfb; i += gridDim.x * wpb) {
        const int t = wa.ntype[i];
        if (t <= 2 || t == 998) continue;
        const double xi = wa.px[i], yi = wa.py[i], si = a.sp[i];
        int c_all = wa.cnt[i], c_small = wa.cnt_small[i];
        double h_i = a.h[i], hs_i = a.hs[i];
        for (int pass = 0; pass < 2; pass++) {
            const double res_tol = a.res_tol[pass];
            for (int ii = 0;; ii++) {
                const double hh = (pass ? hs_i : h_i) * a.rf;
                const int cur = pass ? c_small : c_all;
                int cnt = cur;  // leading links within hh * ss
                for (int b = 0; b < cur; b += 32) {
                    const int k = b + lane;
                    bool out = false;
                    if (k < cur) {
                        const int p = wa.lpt[sell_off(wa.slice_ptr, i, k)];
                        const double rx = xi - wa.px[p], ry = yi - wa.py[p];
                        out = !(sqrt(rx * rx + ry * ry) <= hh * kSs);
                    }
                    const unsigned m = __ballot_sync(0xffffffffu, out);
                    if (m) { cnt = b + __ffs(m) - 1; break; }
                }
                assemble<ORDER>(wa, i, cnt, hh, U, ld, X, G, lane);
                for (int e = lane; e < n * ld; e += 32) M[e] = U[e];
                __syncwarp();
                const double thr = res_tol / hh;
                double hc;
                if (svd_factor_warp<n>(U, V, W, rv1, ld, lane)) {
                    hc = (2.0 * res_tol) / hh;
                } else {
                    for (int m = lane; m < n; m += 32) {
                        bl[m] = (m == 2 || m == 4) ? (1.0 / hh) / hh : 0.0;
                        bx[m] = m == 0 ? 1.0 / hh : 0.0;
                        by[m] = m == 1 ? 1.0 / hh : 0.0;
                    }
                    svd_apply_warp<n>(U, V, W, tmp, bl, ld, lane);
                    svd_apply_warp<n>(U, V, W, tmp, bx, ld, lane);
                    svd_apply_warp<n>(U, V, W, tmp, by, ld, lane);
                    // residual of the Laplacian system, rows in parallel, sums in order
                    for (int r = lane; r < n; r += 32) {
                        double v = (r == 2 || r == 4) ? (-1.0 / hh) / hh : 0.0;
                        for (int c = 0; c < n; c++) v = v + M[c * ld + r] * bl[c];
                        R[r] = v;
                    }
                    __syncwarp();
                    hc = 0.0;
                    if (lane == 0) {
                        for (int r = 0; r < n; r++) hc = hc + R[r] * R[r];
                        hc = (hc * hh) * hh;
                        hc = sqrt(hc / (double)n);
                    }
                    hc = __shfl_sync(0xffffffffu, hc, 0);
                    if (hc < thr) {
                        // each link's dot products with the three solutions (independent of q)
                        for (int k = lane; k < cnt; k += 32) {
                            const int p = wa.lpt[sell_off(wa.slice_ptr, i, k)];
                            const double x = -(xi - wa.px[p]), y = -(yi - wa.py[p]);
                            const double qq = sqrt(x * x + y * y) / hh;
                            const double ff1 = wab(qq, wa.h2);
                            const double xx = x / hh, yy = y / hh;
                            double sl = 0.0, sx = 0.0, sy = 0.0;
                            for (int m = 0; m < n; m++) {
                                const int pm = p_of(m), qm = q_of(m);
                                const double g = ((qm == 0) ? hermite(pm, xx) : (pm == 0) ? hermite(qm, yy)
                                                                                          : hermite(pm, xx) * hermite(qm, yy)) * ff1;
                                sl = sl + bl[m] * g;
                                sx = sx + bx[m] * g;
                                sy = sy + by[m] * g;
                            }
                            lx[k] = x; ly[k] = y; dl[k] = sl; dxv[k] = sx; dyv[k] = sy;
                        }
                        __syncwarp();
                        bool fail = false;
                        for (int i1 = lane + 1; i1 <= nk + 1; i1 += 32) {
                            const double q = (((double)i1 * kPi) / si) / (double)nk;
                            double hl = 0.0, hx = 0.0, hy = 0.0;
                            for (int k = 0; k < cnt; k++) {
                                const double x = lx[k], y = ly[k];
                                hl = hl + (0.5 - (0.5 * cos(x * q)) * cos(y * q)) * dl[k];
                                hx = hx + (cos(y * q) * sin(x * q)) * dxv[k];
                                hy = hy + (cos(x * q) * sin(y * q)) * dyv[k];
                            }
                            hl = hl / (q * q);
                            hx = hx / q;
                            hy = hy / q;
                            if (hl > amp_tol || hl < 0.0 || fabs(hx) > amp_tol || fabs(hy) > amp_tol) fail = true;
                        }
                        if (__any_sync(0xffffffffu, fail)) hc = (2.0 * res_tol) / hh;
                    }
                }
                if ((double)ii > a.limit) hc = (2.0 * res_tol) / hh;
                if (hc >= thr) break;  // a NaN residual compares false and is accepted, as in the reference
                if (pass == 0) {
                    h_i = hh;
                    hs_i = hh;
                    c_all = cnt;
                    c_small = cnt;
                } else {
                    hs_i = hh;
                    c_small = cnt;
                }
                __syncwarp();
            }
        }
        if (lane == 0) {
            a.h[i] = h_i;
            a.hs[i] = hs_i;
        }
    }
}

// The largest dynamic shared memory a block may opt into on the handle's device (227 KB on
// B200): the weight and adaptation kernels are latency-bound, one warp a node, so as many
// warps as their per-warp matrices fit.
int smem_optin(Handle *H, int *bytes) {
    SUNSET_CUDA(H, cudaDeviceGetAttribute(bytes, cudaDevAttrMaxSharedMemoryPerBlockOptin, H->device));
    return 0;
}

template <int ORDER>
int launch_weights(Handle *H, WArgs &a) {
    constexpr int per_warp = smem_doubles<ORDER>() * (int)sizeof(double);
    int optin = 0;
    if (int rc = smem_optin(H, &optin)) return rc;
    int wpb = optin / per_warp;
    if (wpb > 16) wpb = 16;
    if (wpb < 1) wpb = 1;
    size_t smem = (size_t)wpb * per_warp;
    SUNSET_CUDA(H, cudaFuncSetAttribute(k_labf_weights<ORDER>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int nsm = 0;
    SUNSET_CUDA(H, cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, H->device));
    int nb = (a.npfb + wpb - 1) / wpb;
    int cap = nsm * 8;
    if (nb > cap) nb = cap;
    k_labf_weights<ORDER><<<nb, wpb * 32, smem, H->stream>>>(a);
    SUNSET_CUDA(H, cudaGetLastError());
    return 0;
}

}  // namespace

template <int ORDER>
int launch_adapt(Handle *H, AdaptArgs &a) {
    const int per_warp = (adapt_fixed_doubles<ORDER>() + 5 * a.nplink + 1) & ~1;
    const size_t per_warp_bytes = (size_t)per_warp * sizeof(double);
    int optin = 0;
    if (int rc = smem_optin(H, &optin)) return rc;
    int wpb = (int)((size_t)optin / per_warp_bytes);
    if (wpb > 16) wpb = 16;
    if (wpb < 1) return set_err(H, SUNSET_ERR_SCOPE, "neighbour lists too long for the stencil adaptation");
    a.per_warp = per_warp;
    const size_t smem = (size_t)wpb * per_warp_bytes;
    SUNSET_CUDA(H, cudaFuncSetAttribute(k_adapt_stencils<ORDER>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int nsm = 0;
    SUNSET_CUDA(H, cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, H->device));
    int nb = (a.w.npfb + wpb - 1) / wpb;
    if (nb > nsm * 8) nb = nsm * 8;
    k_adapt_stencils<ORDER><<<nb, wpb * 32, smem, H->stream>>>(a);
    SUNSET_CUDA(H, cudaGetLastError());
    return 0;
}

// The residual tolerance of the adaptation, labf.F90:1126-1139 (Hermite ABFs).
static double adapt_res_tol(int order) {
    const int n = (order * order + 3 * order) / 2;
    const double c = order == 4 ? 1.0e-3 : order == 6 ? 5.0e-3 : order == 8 ? 3.0e-2 : 1.0;
    return ((c * (double)(n * n * n * n)) * 2.220446049250313080847e-16) / (double)order;
}

int adapt_stencils_device(Handle *H) {
    if (H->cfg.forder != H->cfg.morder)
        return set_err(H, SUNSET_ERR_SCOPE, "the device stencil adaptation requires forder == morder");
    AdaptArgs a{};
    a.w = WArgs{H->npfb, H->cfg.morder, H->cfg.forder, H->h2, H->px, H->py, H->h, H->hs, H->ntype, H->cnt,
                H->cnt_small, H->lpt, H->slice_ptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    a.h = H->h;
    a.hs = H->hs;
    a.sp = H->sp;
    a.nplink = H->nplink;
    a.rf = (double)0.98f;                          // reduction_factor = 0.98, a default-real literal
    a.limit = (double)logf(0.6f) / log(a.rf);      // log(0.6) of a default-real literal
    a.res_tol[0] = adapt_res_tol(H->cfg.forder);  // adapt_stencils
    a.res_tol[1] = adapt_res_tol(H->cfg.morder);  // adapt_stencils_main
    int rc;
    switch (H->cfg.morder) {
    case 4: rc = launch_adapt<4>(H, a); break;
    case 6: rc = launch_adapt<6>(H, a); break;
    case 8: rc = launch_adapt<8>(H, a); break;
    case 10: rc = launch_adapt<10>(H, a); break;
    default: return set_err(H, SUNSET_ERR_SCOPE, "order %d", H->cfg.morder);
    }
    if (rc) return rc;
    SUNSET_CUDA(H, cudaStreamSynchronize(H->stream));
    return 0;
}

// Condition numbers of the moment matrices the weight build factored: the worst one and the
// number of nodes above the limit (the configured cond_max, else kCondWarn), kept in the
// handle.  With cond_max > 0 such a node is an error; without, it is only counted.
int conditioning_check(Handle *H) {
    const int n = H->npfb;
    std::vector<double> cd(n), cf(n);
    SUNSET_CUDA(H, cudaMemcpyAsync(cd.data(), H->cond_d, n * sizeof(double), cudaMemcpyDeviceToHost, H->stream));
    SUNSET_CUDA(H, cudaMemcpyAsync(cf.data(), H->cond_f, n * sizeof(double), cudaMemcpyDeviceToHost, H->stream));
    SUNSET_CUDA(H, cudaStreamSynchronize(H->stream));
    const double lim = H->cfg.cond_max > 0.0 ? H->cfg.cond_max : kCondWarn;
    double worst = 0.0;
    int nill = 0, iworst = -1;
    for (int i = 0; i < n; i++) {
        const double c = cd[i] > cf[i] ? cd[i] : cf[i];
        if (c > lim) nill++;
        if (c > worst || (std::isinf(c) && iworst < 0)) { worst = c; iworst = i; }
    }
    H->cond_worst = worst;
    H->cond_nill = nill;
    H->cond_ok = true;
    if (H->cfg.cond_max > 0.0 && nill > 0)
        return set_err(H, SUNSET_ERR_ILLCOND,
                       "%d nodes have moment matrices with condition number above %g (worst %.3g at reference node %d)",
                       nill, lim, worst, iworst >= 0 ? H->h_perm[iworst] : -1);
    return 0;
}

int labf_weights_device(Handle *H) {
    const int n = H->npfb;
    if (H->cfg.forder != H->cfg.morder)
        return set_err(H, SUNSET_ERR_SCOPE, "the device weight build requires forder == morder");
    if (!H->wx) {
        if (dalloc(H, &H->wx, H->nlinks_sell) || dalloc(H, &H->wy, H->nlinks_sell) ||
            dalloc(H, &H->wl, H->nlinks_sell) || dalloc(H, &H->wh, H->nlinks_sell) || dalloc(H, &H->gsx, n) ||
            dalloc(H, &H->gsy, n) || dalloc(H, &H->lsum, n) || dalloc(H, &H->hsum, n) || dalloc(H, &H->vol, n))
            return SUNSET_ERR_NOMEM;
    }
    cudaStream_t st = H->stream;
    SUNSET_CUDA(H, cudaMemsetAsync(H->wx, 0, H->nlinks_sell * sizeof(double), st));
    SUNSET_CUDA(H, cudaMemsetAsync(H->wy, 0, H->nlinks_sell * sizeof(double), st));
    SUNSET_CUDA(H, cudaMemsetAsync(H->wl, 0, H->nlinks_sell * sizeof(double), st));
    SUNSET_CUDA(H, cudaMemsetAsync(H->wh, 0, H->nlinks_sell * sizeof(double), st));
    int *derr;
    if (dalloc(H, &derr, 1)) return SUNSET_ERR_NOMEM;
    SUNSET_CUDA(H, cudaMemsetAsync(derr, 0, sizeof(int), st));
    if (!H->cond_d && (dalloc(H, &H->cond_d, n) || dalloc(H, &H->cond_f, n))) return SUNSET_ERR_NOMEM;
    SUNSET_CUDA(H, cudaMemsetAsync(H->cond_d, 0, n * sizeof(double), st));
    SUNSET_CUDA(H, cudaMemsetAsync(H->cond_f, 0, n * sizeof(double), st));
    WArgs a{n, H->cfg.morder, H->cfg.forder, H->h2, H->px, H->py, H->h, H->hs, H->ntype, H->cnt, H->cnt_small,
            H->lpt, H->slice_ptr, H->wx, H->wy, H->wl, H->wh, derr, H->cfg.svd_max_sweeps, H->cond_d, H->cond_f};
    int rc;
    switch (H->cfg.morder) {
    case 4: rc = launch_weights<4>(H, a); break;
    case 6: rc = launch_weights<6>(H, a); break;
    case 8: rc = launch_weights<8>(H, a); break;
    case 10: rc = launch_weights<10>(H, a); break;
    default: return set_err(H, SUNSET_ERR_ARG, "order must be 4, 6, 8 or 10");
    }
    if (rc) return rc;
    int herr = 0;
    SUNSET_CUDA(H, cudaMemcpyAsync(&herr, derr, sizeof(int), cudaMemcpyDeviceToHost, st));
    SUNSET_CUDA(H, cudaStreamSynchronize(st));
    dfree(H, derr);
    if (herr) return set_err(H, SUNSET_ERR_SVD, "SVD not converging at internal node %d (svdlib.F90:219-222)", herr - 1);
    return conditioning_check(H);
}

int boundary_prune_links(Handle *H);

// calc_boundary_weights (labf.F90:505-1039); the links of the boundary nodes are pruned by
// boundary_prune_links() first.
int boundary_weights_device(Handle *H) {
    if (H->nb == 0) return 0;
    const int nb = H->nb;
    if (!H->wb2 && dalloc(H, &H->wb2, (size_t)nb * H->nplink * 2)) return SUNSET_ERR_NOMEM;
    int *derr;
    if (dalloc(H, &derr, 1)) return SUNSET_ERR_NOMEM;
    cudaStream_t st = H->stream;
    SUNSET_CUDA(H, cudaMemsetAsync(derr, 0, sizeof(int), st));
    BndArgs a{H->npfb, nb, H->nplink, H->h3, H->px, H->py, H->h, H->sp, H->rnx, H->rny, H->ntype, H->gpar,
              H->fdpar, H->blist, H->brow, H->cnt, H->cnt_small, H->lpt, H->lidx, H->lloc, H->slice_ptr,
              H->slice_w, H->wx, H->wy, H->wl, H->wh, H->wb2, derr};
    k_boundary_node_weights<<<(nb + 3) / 4, 128, 0, st>>>(a);
    k_boundary_row_weights<<<(2 * nb + 3) / 4, 128, 0, st>>>(a);
    k_boundary_frame<<<(nb + 127) / 128, 128, 0, st>>>(a);
    SUNSET_CUDA(H, cudaGetLastError());
    int herr = 0;
    SUNSET_CUDA(H, cudaMemcpyAsync(&herr, derr, sizeof(int), cudaMemcpyDeviceToHost, st));
    SUNSET_CUDA(H, cudaStreamSynchronize(st));
    dfree(H, derr);
    if (herr) return set_err(H, SUNSET_ERR_SVD, "SVD not converging at boundary node or row %d", herr - 1);
    return 0;
}

int boundary_prune_links(Handle *H) {
    if (H->nb == 0) return 0;
    BndArgs a{H->npfb, H->nb, H->nplink, H->h3, H->px, H->py, H->h, H->sp, H->rnx, H->rny, H->ntype, H->gpar,
              H->fdpar, H->blist, H->brow, H->cnt, H->cnt_small, H->lpt, H->lidx, H->lloc, H->slice_ptr,
              H->slice_w, H->wx, H->wy, H->wl, H->wh, H->wb2, nullptr};
    k_prune_boundary_links<<<(H->nb + 127) / 128, 128, 0, H->stream>>>(a);
    SUNSET_CUDA(H, cudaGetLastError());
    SUNSET_CUDA(H, cudaStreamSynchronize(H->stream));
    return 0;
}

// The tangential second-derivative weights of boundary nodes scaled by 1/L^2 and their sums
// over all links (calc_labf_sums, labf.F90:426-446): the transverse Laplacian of the
// conformation tensor on walls (derivatives.F90:306-358).  One thread per boundary node.
__global__ void k_boundary_tangential_sums(int nb, int nplink, double L, const int *blist, const int *cnt,
                                           const double *wb2, double *wbt, double *wbt_sum) {
    const int jj = blockIdx.x * blockDim.x + threadIdx.x;
    if (jj >= nb) return;
    const double *w = wb2 + (size_t)jj * nplink * 2;
    double sum = 0.0;
    for (int k = 0; k < cnt[blist[jj]]; k++) sum = sum + w[2 * k + 1];
    wbt_sum[jj] = (sum / L) / L;
    for (int k = 0; k < nplink; k++) wbt[(size_t)jj * nplink + k] = (w[2 * k + 1] / L) / L;
}

int labf_sums_device(Handle *H) {
    SumArgs a{H->npfb, H->cfg.L_char, H->px, H->py, H->h, H->sp, H->ntype, H->cnt, H->lpt, H->fdpar, H->slice_ptr,
              H->wx, H->wy, H->wl, H->wh, H->gsx, H->gsy, H->lsum, H->hsum, H->vol};
    k_labf_sums<<<(H->npfb + 255) / 256, 256, 0, H->stream>>>(a);
    if (H->nb > 0) {
        if (!H->wbt && (dalloc(H, &H->wbt, (size_t)H->nb * H->nplink) || dalloc(H, &H->wbt_sum, H->nb)))
            return SUNSET_ERR_NOMEM;
        k_boundary_tangential_sums<<<(H->nb + 127) / 128, 128, 0, H->stream>>>(H->nb, H->nplink, H->cfg.L_char, H->blist,
                                                                             H->cnt, H->wb2, H->wbt, H->wbt_sum);
    }
    SUNSET_CUDA(H, cudaGetLastError());
    SUNSET_CUDA(H, cudaStreamSynchronize(H->stream));
    return 0;
}

int filter_coefficients_device(Handle *H) {
    SumArgs a{H->npfb, H->cfg.L_char, H->px, H->py, H->h, H->sp, H->ntype, H->cnt, H->lpt, H->fdpar, H->slice_ptr,
              H->wx, H->wy, H->wl, H->wh, H->gsx, H->gsy, H->lsum, H->hsum, H->vol};
    k_filter_coeff<<<(H->npfb + 255) / 256, 256, 0, H->stream>>>(a);
    SUNSET_CUDA(H, cudaGetLastError());
    SUNSET_CUDA(H, cudaStreamSynchronize(H->stream));
    return 0;
}

}  // namespace sunset
