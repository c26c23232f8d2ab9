// step.cu -- the time step (FP64 and mixed precision): fused RK stage kernels, filter + mass
// correction, finalisation, PID time-step control, and the single-operator kernels of the
// C-ABI.
//
// One RK stage is one kernel: a block owns a tile of 8 slices (256 nodes), stages the
// fields of every node the tile's links reach (its halo) in shared memory, and streams the
// tile's links through a per-thread cp.async ring.  A thread owns a node: its stencil sums
// feed the right-hand side in registers, which feeds the low-storage RK update
// (step.F90:291-343), which writes the next state and its derived fields (velocity,
// conformation tensor) into the other state buffer.  Ghost links carry the parent's
// index and a reflection code, so no mirror copy (mirror_boundaries.F90:263-352) or
// halo exchange runs between stages.
//
// Sums take the reference's sum form (sum_k w_k phi_j - phi_i sum_k w_k,
// derivatives.F90:36-46) and the file is built with -fmad=false, so each product and sum of
// the FP64 path rounds as in the reference.  The single-operator kernels sum in the
// reference's link order and reproduce it bit for bit; the step sums in the bank-aware
// order of stream.cu, which changes only the rounding (and libm's exp, log, cos may differ
// from glibc in the last bit).
#include <type_traits>

#include "adjoint.cuh"
#include "internal.cuh"
#include "physics.cuh"

namespace sunset {

namespace {

__constant__ StepConsts cK;

struct StageArgs {
    const long long *slice_ptr;
    const int *slice_ws, *slice_w;
    const int *lidx;
    const uint16_t *lloc;
    const int *halo_ptr, *halo;
    int hmax;
    const double *wx, *wy, *wl, *wh;
    const float *wx32, *wy32, *wl32, *wh32;  // mixed precision
    const double *gsx, *gsy, *lsum, *hsum, *vol, *py_node;
    const int *ntype;            // node types (walls: 0)
    const double *rnx, *rny;     // wall normals into the fluid
    Fields in, out;
    double *reg[7], *eacc[7], *rhs[7];
    float *dreg[7], *eacc32[7];  // mixed precision
    DevScalars *sc;
    double *partials;
    int stage;  // 0..3; 4 = rhs only
};

// Reflection codes of a ghost link: 1 -> vrelation 2 (x mirror: u and the xy component
// change sign), 2 -> vrelation 3 (y mirror: v and xy), 3 -> vrelation 4 (u and v).
__device__ __forceinline__ void reflect(int code, double &uj, double &vj, double &xyj) {
    if (code == 1 || code == 3) uj = -uj;
    if (code == 2 || code == 3) vj = -vj;
    if (code == 1 || code == 2) xyj = -xyj;
}

// Fields a stage gathers from its neighbours, in shared-memory order:
//   0 ro, 1 u, 2 v, then DI: cxx cxy cyy; LC: cxx cxy cyy psixx psixy psiyy;
//   CHL: psixx psixy psiyy (+ cxx cxy cyy with polymer diffusion).
__host__ __device__ constexpr int ngather(int form, bool md) {
    return form == SUNSET_FORM_DI ? 6 : form == SUNSET_FORM_LC ? 9 : form == SUNSET_FORM_CHL ? (md ? 9 : 6) : 3;
}

template <int FORM, bool MD>
__device__ __forceinline__ const double *gather_src(const Fields &F, int f) {
    if (f == 0) return F.ro;
    if (f == 1) return F.u;
    if (f == 2) return F.v;
    if (FORM == SUNSET_FORM_DI || FORM == SUNSET_FORM_LC) {
        if (f <= 5) return F.c[f - 3];
        return F.q[f - 6];
    }
    if (f <= 5) return F.q[f - 3];
    return F.c[f - 6];
}


// cp.async (global -> shared, completion tracked per thread in commit groups), with memory
// clobbers so the compiler keeps shared-memory reads after the wait that covers them.
template <int N>
__device__ __forceinline__ void cp_async(void *dst_shared, const void *src_global) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst_shared);
    const size_t g = __cvta_generic_to_global(src_global);
    if constexpr (N == 16)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(g) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(d), "l"(g), "n"(N) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// The block's halo (fields of every node its links reach) into shared memory, laid out
// field-major with stride hmax, by cp.async so all of a thread's copies are in flight at
// once.  All threads of the block take part; the wait also covers any copies the thread
// issued before.
template <int NG, typename SRC>
__device__ __forceinline__ void load_halo(const StageArgs &A, double *sm, SRC src) {
    const int hb = A.halo_ptr[blockIdx.x], hn = A.halo_ptr[blockIdx.x + 1] - hb;
    const int hm = A.hmax;
    for (int h = threadIdx.x; h < hn; h += blockDim.x) {
        const int node = __ldg(A.halo + hb + h);
#pragma unroll
        for (int f = 0; f < NG; f++) cp_async<8>(&sm[f * hm + h], src(f) + node);
    }
    cp_async_commit();
    cp_async_wait<0>();
    __syncthreads();
}

// Per-thread ring of link pairs in shared memory, filled by cp.async (LDGSTS).  Thread t
// copies its own node's link pair m -- NA weight pairs and the pair's two 16-bit local
// indices -- D-1 pairs ahead of the pair it works on, so D-1 pairs per thread are in flight
// without holding registers.  A thread reads back only what it copied itself, so no barrier
// is needed; slots are reused only after the thread has consumed them.
template <bool MX, int NA, int D>
struct LinkRing {
    static_assert((D & (D - 1)) == 0, "ring depth must be a power of two");
    using W2 = typename std::conditional<MX, float2, double2>::type;
    W2 *w;          // [D][NA][kTile]
    unsigned *l;    // [D][kTile]
    const W2 *src[NA];
    const unsigned *lsrc;
    long long pb;   // pair index of this node's pair 0; pair m sits at pb + 32 m
    int npair;

    static constexpr size_t bytes() { return (size_t)D * kTile * (NA * sizeof(W2) + sizeof(unsigned)); }

    __device__ __forceinline__ void init(double *base, const unsigned *lidx2, long long pb_, int npair_) {
        w = reinterpret_cast<W2 *>(base);
        l = reinterpret_cast<unsigned *>(w + (size_t)D * NA * kTile);
        lsrc = lidx2;
        pb = pb_;
        npair = npair_;
    }
    __device__ __forceinline__ void issue(int m) {
        if (m < npair) {
            const int s = m & (D - 1);
            const long long o = pb + ((long long)m << 5);
#pragma unroll
            for (int a = 0; a < NA; a++) cp_async<sizeof(W2)>(w + (s * NA + a) * kTile + threadIdx.x, src[a] + o);
            cp_async<4>(l + s * kTile + threadIdx.x, lsrc + o);
        }
        cp_async_commit();  // empty groups keep the group count uniform
    }
    __device__ __forceinline__ void prologue() {
#pragma unroll
        for (int m = 0; m < D - 1; m++) issue(m);
    }
    // make pair m resident (and start pair m + D - 1)
    __device__ __forceinline__ void next(int m) {
        issue(m + D - 1);
        cp_async_wait<D - 1>();
    }
    __device__ __forceinline__ void weights(int m, int a, double &x0, double &x1) const {
        const W2 v = w[((m & (D - 1)) * NA + a) * kTile + threadIdx.x];
        x0 = (double)v.x;
        x1 = (double)v.y;
    }
    __device__ __forceinline__ unsigned index(int m) const { return l[(m & (D - 1)) * kTile + threadIdx.x]; }
};

// Ring depth: FP64 pairs are 52 bytes a thread, FP32 ones 28.
#ifndef SUNSET_RING_FP64
#define SUNSET_RING_FP64 2
#endif
#ifndef SUNSET_RING_MIXED
#define SUNSET_RING_MIXED 4
#endif
__host__ __device__ constexpr int ring_depth(bool mx) { return mx ? SUNSET_RING_MIXED : SUNSET_RING_FP64; }

// Doubles of the shared-memory halo, rounded up so the ring after it is 16-byte aligned.
__host__ __device__ inline size_t halo_doubles(int ng, int hmax) { return ((size_t)ng * hmax + 1) & ~(size_t)1; }

// Stencil sums of one node over its small links, sum form of derivatives.F90:36-46,
// neighbours read from the block's shared-memory halo.  In the mixed path the weights are
// the FP32-rounded ones and A.gsx.. hold the FP64 sums of those, so the FP64 arithmetic
// below evaluates the difference form sum_k w_k (phi_j - phi_i) of the rounded stencil.
template <int FORM, bool MD, bool MX, class RING>
__device__ __forceinline__ void gather_stage(const StageArgs &A, int i, const double *sm, RING &R, Grads &g) {
    const int hm = A.hmax;
    const int npair = R.npair;
    const Fields &F = A.in;
    double s_ro_x = 0, s_ro_y = 0, s_u_x = 0, s_u_y = 0, s_v_x = 0, s_v_y = 0, s_lu = 0, s_lv = 0;
    double s_cxx_x = 0, s_cxx_y = 0, s_cxy_x = 0, s_cxy_y = 0, s_cyy_x = 0, s_cyy_y = 0;
    double s_pxx_x = 0, s_pxx_y = 0, s_pxy_x = 0, s_pxy_y = 0, s_pyy_x = 0, s_pyy_y = 0;
    double s_lxx = 0, s_lxy = 0, s_lyy = 0;
    const bool mir = cK.has_mirrors;
    const bool full = (FORM == SUNSET_FORM_DI) && cK.di_full;
    // FP64 step: separate multiply and add, as the reference; mixed step: fused
    auto mac = [](double &acc, double x, double w) {
        if constexpr (MX) acc = __fma_rn(x, w, acc);
        else acc = acc + x * w;
    };
    auto link = [&](int lk, double wxk, double wyk, double wlk) {
        const int j = lk & kLocMask;
        double roj = sm[j], uj = sm[hm + j], vj = sm[2 * hm + j];
        double cxxj = 0.0, cxyj = 0.0, cyyj = 0.0, pxxj = 0.0, pxyj = 0.0, pyyj = 0.0;
        if (FORM == SUNSET_FORM_DI || FORM == SUNSET_FORM_LC) {
            cxxj = sm[3 * hm + j]; cxyj = sm[4 * hm + j]; cyyj = sm[5 * hm + j];
        }
        if (FORM == SUNSET_FORM_LC) {
            pxxj = sm[6 * hm + j]; pxyj = sm[7 * hm + j]; pyyj = sm[8 * hm + j];
        }
        if (FORM == SUNSET_FORM_CHL) {
            pxxj = sm[3 * hm + j]; pxyj = sm[4 * hm + j]; pyyj = sm[5 * hm + j];
            if (MD) { cxxj = sm[6 * hm + j]; cxyj = sm[7 * hm + j]; cyyj = sm[8 * hm + j]; }
        }
        if (mir) {
            const int code = lk >> 14;
            reflect(code, uj, vj, cxyj);
            if (code == 1 || code == 2) pxyj = -pxyj;
        }
        mac(s_ro_x, roj, wxk);
        mac(s_ro_y, roj, wyk);
        mac(s_u_x, uj, wxk);
        mac(s_u_y, uj, wyk);
        mac(s_lu, uj, wlk);
        mac(s_v_x, vj, wxk);
        mac(s_v_y, vj, wyk);
        mac(s_lv, vj, wlk);
        if (FORM == SUNSET_FORM_DI || FORM == SUNSET_FORM_LC) {
            mac(s_cxx_x, cxxj, wxk);
            if (full) mac(s_cxx_y, cxxj, wyk);
            mac(s_cxy_x, cxyj, wxk);
            mac(s_cxy_y, cxyj, wyk);
            if (full) mac(s_cyy_x, cyyj, wxk);
            mac(s_cyy_y, cyyj, wyk);
        }
        if (FORM == SUNSET_FORM_LC || FORM == SUNSET_FORM_CHL) {
            mac(s_pxx_x, pxxj, wxk);
            mac(s_pxx_y, pxxj, wyk);
            mac(s_pxy_x, pxyj, wxk);
            mac(s_pxy_y, pxyj, wyk);
            mac(s_pyy_x, pyyj, wxk);
            mac(s_pyy_y, pyyj, wyk);
        }
        if (MD && (FORM == SUNSET_FORM_DI || FORM == SUNSET_FORM_CHL)) {
            mac(s_lxx, cxxj, wlk);
            mac(s_lxy, cxyj, wlk);
            mac(s_lyy, cyyj, wlk);
        }
    };
    // links in order k = 2m, 2m+1: the sums keep the reference's order
    for (int m = 0; m < npair; m++) {
        R.next(m);
        double wx0, wx1, wy0, wy1, wl0, wl1;
        R.weights(m, 0, wx0, wx1);
        R.weights(m, 1, wy0, wy1);
        R.weights(m, 2, wl0, wl1);
        const unsigned l2 = R.index(m);
        link((int)(l2 & 0xffffu), wx0, wy0, wl0);
        link((int)(l2 >> 16), wx1, wy1, wl1);
    }
    if (i >= cK.npfb) return;
    const double gx = A.gsx[i], gy = A.gsy[i], ls = A.lsum[i];
    const double roi = F.ro[i], ui = F.u[i], vi = F.v[i];
    g.ro_x = s_ro_x - roi * gx;
    g.ro_y = s_ro_y - roi * gy;
    g.u_x = s_u_x - ui * gx;
    g.u_y = s_u_y - ui * gy;
    g.lapu = s_lu - ui * ls;
    g.v_x = s_v_x - vi * gx;
    g.v_y = s_v_y - vi * gy;
    g.lapv = s_lv - vi * ls;
    g.cxx_x = g.cxx_y = g.cxy_x = g.cxy_y = g.cyy_x = g.cyy_y = 0.0;
    g.pxx_x = g.pxx_y = g.pxy_x = g.pxy_y = g.pyy_x = g.pyy_y = 0.0;
    g.lapcxx = g.lapcxy = g.lapcyy = g.lapczz = 0.0;
    if (FORM == SUNSET_FORM_DI || FORM == SUNSET_FORM_LC) {
        const double cxx = F.c[0][i], cxy = F.c[1][i], cyy = F.c[2][i];
        g.cxx_x = s_cxx_x - cxx * gx;
        if (full) g.cxx_y = s_cxx_y - cxx * gy;
        g.cxy_x = s_cxy_x - cxy * gx;
        g.cxy_y = s_cxy_y - cxy * gy;
        if (full) g.cyy_x = s_cyy_x - cyy * gx;
        g.cyy_y = s_cyy_y - cyy * gy;
    }
    if (FORM == SUNSET_FORM_LC || FORM == SUNSET_FORM_CHL) {
        const double pxx = F.q[0][i], pxy = F.q[1][i], pyy = F.q[2][i];
        g.pxx_x = s_pxx_x - pxx * gx;
        g.pxx_y = s_pxx_y - pxx * gy;
        g.pxy_x = s_pxy_x - pxy * gx;
        g.pxy_y = s_pxy_y - pxy * gy;
        g.pyy_x = s_pyy_x - pyy * gx;
        g.pyy_y = s_pyy_y - pyy * gy;
    }
    if (MD && (FORM == SUNSET_FORM_DI || FORM == SUNSET_FORM_CHL)) {
        g.lapcxx = s_lxx - F.c[0][i] * ls;
        g.lapcxy = s_lxy - F.c[1][i] * ls;
        g.lapcyy = s_lyy - F.c[2][i] * ls;
    }
}

__device__ __forceinline__ unsigned long long dbits(double x) { return (unsigned long long)__double_as_longlong(x); }

__device__ __forceinline__ void block_max_bits(unsigned long long v, unsigned long long *dst) {
    __shared__ unsigned long long sm[32];
    __syncthreads();
    for (int o = 16; o > 0; o >>= 1) {
        unsigned long long t = __shfl_down_sync(0xffffffffu, v, o);
        v = t > v ? t : v;
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) sm[w] = v;
    __syncthreads();
    if (w == 0) {
        v = lane < (int)(blockDim.x >> 5) ? sm[lane] : 0ull;
        for (int o = 16; o > 0; o >>= 1) {
            unsigned long long t = __shfl_down_sync(0xffffffffu, v, o);
            v = t > v ? t : v;
        }
        if (lane == 0 && v) atomicMax(dst, v);
    }
}
__device__ __forceinline__ void block_min_bits(unsigned long long v, unsigned long long *dst) {
    __shared__ unsigned long long sm2[32];
    __syncthreads();
    for (int o = 16; o > 0; o >>= 1) {
        unsigned long long t = __shfl_down_sync(0xffffffffu, v, o);
        v = t < v ? t : v;
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) sm2[w] = v;
    __syncthreads();
    if (w == 0) {
        v = lane < (int)(blockDim.x >> 5) ? sm2[lane] : ~0ull;
        for (int o = 16; o > 0; o >>= 1) {
            unsigned long long t = __shfl_down_sync(0xffffffffu, v, o);
            v = t < v ? t : v;
        }
        if (lane == 0) atomicMin(dst, v);
    }
}

// Resident blocks per SM the stage kernel is compiled for (up to 85 registers a thread):
// the tile halo plus the link ring take 55-70 KB of shared memory on the order-6 and
// order-8 sets, so a fourth block would not fit anyway.
#ifndef SUNSET_STAGE_BLOCKS
#define SUNSET_STAGE_BLOCKS 3
#endif
__host__ __device__ constexpr int stage_min_blocks(int) { return SUNSET_STAGE_BLOCKS; }

// One RK stage (stage = 0,1,2: intermediate; 3: final; 4: right-hand side only).  One
// block per tile of kTile nodes; the tile's halo is staged in shared memory first.
//
// MX (mixed precision): FP32 weights; the register S is kept as the FP32 increment
// D = S - U over the stage's FP64 state U (so S = U + D loses only FP32 rounding of an
// O(dt rhs) quantity) and the error accumulator E as FP32.
template <int FORM, bool MD, bool MX>
__global__ void __launch_bounds__(kTile, stage_min_blocks(FORM)) k_stage(StageArgs A) {
    extern __shared__ __align__(16) double smem[];
    constexpr int NG = ngather(FORM, MD);
    const int i = blockIdx.x * kTile + threadIdx.x;
    bool active = (i >> 5) < cK.nslices;
    LinkRing<MX, 3, ring_depth(MX)> R;
    if constexpr (MX) {
        R.src[0] = reinterpret_cast<const float2 *>(A.wx32);
        R.src[1] = reinterpret_cast<const float2 *>(A.wy32);
        R.src[2] = reinterpret_cast<const float2 *>(A.wl32);
    } else {
        R.src[0] = reinterpret_cast<const double2 *>(A.wx);
        R.src[1] = reinterpret_cast<const double2 *>(A.wy);
        R.src[2] = reinterpret_cast<const double2 *>(A.wl);
    }
    R.init(smem + halo_doubles(NG, A.hmax), reinterpret_cast<const unsigned *>(A.lloc),
           active ? (A.slice_ptr[i >> 5] >> 1) + (i & 31) : 0, active ? A.slice_ws[i >> 5] >> 1 : 0);
    R.prologue();  // the first link pairs stream in while the halo is staged
    load_halo<NG>(A, smem, [&](int f) { return gather_src<FORM, MD>(A.in, f); });
    const int stage = A.stage;
    if (stage == 0 && i == 0) {
        A.sc->cfl_bits = 0x7ff0000000000000ull;
        A.sc->par_bits = 0x7ff0000000000000ull;
    }
    Grads g;
    if (active) gather_stage<FORM, MD, MX>(A, i, smem, R, g);
    active = active && i < cK.npfb;
    unsigned long long emax_bits = 0;
    if (active) {
        const Fields &F = A.in;
        NodeState n;
        n.ro = F.ro[i]; n.u = F.u[i]; n.v = F.v[i]; n.y = A.py_node[i];
        n.cxx = F.c[0][i]; n.cxy = F.c[1][i]; n.cyy = F.c[2][i]; n.czz = F.c[3][i];
        n.pxx = F.q[0][i]; n.pxy = F.q[1][i]; n.pyy = F.q[2][i]; n.pzz = F.q[3][i];
        Rhs r;
        const bool wall = cK.has_walls && A.ntype[i] == 0;
        if (wall) {  // wall closure; then the conformation with the rotated velocity gradient
            const double xn = A.rnx[i], yn = A.rny[i];
            rhs_flow_wall(cK, n, g, xn, yn, r);
            const double gux = g.u_x, guy = g.u_y, gvx = g.v_x, gvy = g.v_y;
            g.u_x = xn * gux - yn * guy;
            g.v_x = xn * gvx - yn * gvy;
            g.u_y = yn * gux + xn * guy;
            g.v_y = yn * gvx + xn * gvy;
        } else {
            rhs_flow(cK, n, g, r);
        }
        if (FORM == SUNSET_FORM_DI) rhs_c_di(cK, n, g, r, wall);
        else if (FORM == SUNSET_FORM_CHL) rhs_c_chl(cK, n, g, r);
        else if (FORM == SUNSET_FORM_LC) {
            const bool first = (A.sc->itime == 1) && (stage == 0);
            rhs_c_lc(cK, n, g, first, r, wall);
        } else { r.xx = r.xy = r.yy = r.zz = 0.0; }
        const double rr[7] = {r.ro, r.rou, r.rov, r.xx, r.xy, r.yy, r.zz};
        constexpr int nf = (FORM == SUNSET_FORM_DI) ? 7 : (FORM == SUNSET_FORM_NEWT ? 3 : 6);
        if (stage == 4) {
#pragma unroll
            for (int f = 0; f < 7; f++) A.rhs[f][i] = rr[f];
        } else {
            const double U[7] = {F.ro[i], F.rou[i], F.rov[i], F.q[0][i], F.q[1][i], F.q[2][i], F.q[3][i]};
            const double dt = A.sc->dt;
            const double a = stage == 0 ? SUNSET_RK_A21 : stage == 1 ? SUNSET_RK_A32 : SUNSET_RK_A43;
            const double b = stage == 0 ? SUNSET_RK_B1 : stage == 1 ? SUNSET_RK_B2 : stage == 2 ? SUNSET_RK_B3 : SUNSET_RK_B4;
            const double bh = stage == 0 ? SUNSET_RK_BH1 : stage == 1 ? SUNSET_RK_BH2 : stage == 2 ? SUNSET_RK_BH3 : SUNSET_RK_BH4;
            const double RKb = dt * b, RKbmbh = dt * (b - bh);
            double Un[7];
#pragma unroll
            for (int f = 0; f < 7; f++) Un[f] = U[f];
            if (stage < 3) {
                const double RKa = dt * a;
#pragma unroll
                for (int f = 0; f < nf; f++) {
                    if constexpr (MX) {
                        const double S = (stage == 0) ? U[f] : U[f] + (double)A.dreg[f][i];
                        const double E = (stage == 0) ? 0.0 : (double)A.eacc32[f][i];
                        Un[f] = S + RKa * rr[f];
                        A.dreg[f][i] = (float)((S + RKb * rr[f]) - Un[f]);
                        A.eacc32[f][i] = (float)(E + RKbmbh * rr[f]);
                    } else {
                        const double S = (stage == 0) ? U[f] : A.reg[f][i];
                        const double E = (stage == 0) ? 0.0 : A.eacc[f][i];
                        Un[f] = S + RKa * rr[f];
                        A.reg[f][i] = S + RKb * rr[f];
                        A.eacc[f][i] = E + RKbmbh * rr[f];
                    }
                }
            } else {
                double en = 0.0;
#pragma unroll
                for (int f = 0; f < nf; f++) {
                    const double norm = f == 0 ? cK.ero_norm : f < 3 ? cK.erou_norm : cK.exx_norm;
                    double E;
                    if constexpr (MX) {
                        Un[f] = (U[f] + (double)A.dreg[f][i]) + RKb * rr[f];
                        E = (double)A.eacc32[f][i] + RKbmbh * rr[f];
                    } else {
                        Un[f] = A.reg[f][i] + RKb * rr[f];
                        E = A.eacc[f][i] + RKbmbh * rr[f];
                    }
                    const double t = fabs(E) * norm;
                    en = (t > en) ? t : en;
                    if (t != t) en = t;
                }
                emax_bits = dbits(en);
            }
            if (wall) { Un[1] = 0.0; Un[2] = 0.0; }  // apply_time_dependent_bounds, characteristic_boundaries.F90:200-206
            const Fields &O = A.out;
            O.ro[i] = Un[0]; O.rou[i] = Un[1]; O.rov[i] = Un[2];
            if (FORM != SUNSET_FORM_NEWT) {
                O.q[0][i] = Un[3]; O.q[1][i] = Un[4]; O.q[2][i] = Un[5]; O.q[3][i] = Un[6];
            }
            if (stage < 3) {  // get_velocity_from_momentum, get_c_from_psi (step.F90:514-567)
                const double ooro = 1.0 / Un[0];
                O.u[i] = Un[1] * ooro;
                O.v[i] = Un[2] * ooro;
                if (FORM == SUNSET_FORM_LC) {
                    double cxx, cxy, cyy;
                    lc_c_from_psi(Un[3], Un[4], Un[5], &cxx, &cxy, &cyy);
                    O.c[0][i] = cxx; O.c[1][i] = cxy; O.c[2][i] = cyy; O.c[3][i] = F.c[3][i];
                } else if (FORM == SUNSET_FORM_CHL) {
                    double cxx, cxy, cyy, czz;
                    chl_c_from_psi(Un[3], Un[4], Un[5], &cxx, &cxy, &cyy, &czz);
                    O.c[0][i] = cxx; O.c[1][i] = cxy; O.c[2][i] = cyy; O.c[3][i] = czz;
                }
            }
        }
    }
    if (stage == 3) block_max_bits(emax_bits, &A.sc->emax_bits);
}

// filter_variables (rhs_di.F90:667-720; rhs.F90:792-900; rhs_lc.F90:818-893): the
// hyperviscous filter of each evolved field plus the mass-correction partial sums.
template <int FORM, bool MX>
__global__ void __launch_bounds__(kTile, 4) k_filter(StageArgs A) {
    extern __shared__ __align__(16) double smem[];
    constexpr int nf = (FORM == SUNSET_FORM_DI) ? 7 : (FORM == SUNSET_FORM_NEWT ? 3 : 6);
    const Fields &F = A.in;
    const int i = blockIdx.x * kTile + threadIdx.x;
    const bool live = (i >> 5) < cK.nslices;
    LinkRing<MX, 1, ring_depth(MX)> R;
    if constexpr (MX) R.src[0] = reinterpret_cast<const float2 *>(A.wh32);
    else R.src[0] = reinterpret_cast<const double2 *>(A.wh);
    R.init(smem + halo_doubles(nf, A.hmax), reinterpret_cast<const unsigned *>(A.lloc),
           live ? (A.slice_ptr[i >> 5] >> 1) + (i & 31) : 0, live ? A.slice_w[i >> 5] >> 1 : 0);
    R.prologue();
    load_halo<nf>(A, smem, [&](int f) -> const double * {
        return f == 0 ? F.ro : f == 1 ? F.rou : f == 2 ? F.rov : F.q[f - 3];
    });
    const int hm = A.hmax;
    double part = 0.0;
    if (live) {
        const int npair = R.npair;
        double t[7] = {0, 0, 0, 0, 0, 0, 0};
        const bool mir = cK.has_mirrors;
        auto link = [&](int lk, double whk) {
            const int j = lk & kLocMask;
            double v[7];
#pragma unroll
            for (int f = 0; f < nf; f++) v[f] = smem[f * hm + j];
            if (mir) {
                double dummy = 0.0;
                const int code = lk >> 14;
                reflect(code, v[1], v[2], nf > 4 ? v[4] : dummy);
            }
#pragma unroll
            for (int f = 0; f < nf; f++) {
                if constexpr (MX) t[f] = __fma_rn(v[f], whk, t[f]);
                else t[f] = t[f] + v[f] * whk;
            }
        };
        for (int m = 0; m < npair; m++) {
            R.next(m);
            double wh0, wh1;
            R.weights(m, 0, wh0, wh1);
            const unsigned l2 = R.index(m);
            link((int)(l2 & 0xffffu), wh0);
            link((int)(l2 >> 16), wh1);
        }
        if (i < cK.npfb) {
            const double hs = A.hsum[i];
            const double *src[7] = {F.ro, F.rou, F.rov, F.q[0], F.q[1], F.q[2], F.q[3]};
            double *dst[7] = {A.out.ro, A.out.rou, A.out.rov, A.out.q[0], A.out.q[1], A.out.q[2], A.out.q[3]};
            double rof = 0.0;
            const bool wall = cK.has_walls && A.ntype[i] == 0;
#pragma unroll
            for (int f = 0; f < 7; f++) {
                if (f < nf) {
                    const double p = src[f][i];
                    double r = p + (t[f] - p * hs);
                    if (wall && (f == 1 || f == 2)) r = 0.0;  // apply_time_dependent_bounds after the filter
                    dst[f][i] = r;
                    if (f == 0) rof = r;
                } else if (FORM != SUNSET_FORM_NEWT) {
                    dst[f][i] = src[f][i];
                }
            }
            part = (rof - cK.rho_char) * A.vol[i];
        }
    }
    // deterministic two-level sum: fixed tree in the block, fixed order over blocks
    __shared__ double red[kTile];
    red[threadIdx.x] = part;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) red[threadIdx.x] = red[threadIdx.x] + red[threadIdx.x + s];
        __syncthreads();
    }
    __shared__ bool last;
    if (threadIdx.x == 0) {
        A.partials[blockIdx.x] = red[0];
        __threadfence();
        unsigned int prev = atomicAdd(&A.sc->done_ctr, 1u);
        last = (prev == gridDim.x - 1);
    }
    __syncthreads();
    if (last) {
        __threadfence();
        double acc = 0.0;
        for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) acc = acc + ((volatile double *)A.partials)[b];
        red[threadIdx.x] = acc;
        __syncthreads();
        for (int s = blockDim.x / 2; s > 0; s >>= 1) {
            if ((int)threadIdx.x < s) red[threadIdx.x] = red[threadIdx.x] + red[threadIdx.x + s];
            __syncthreads();
        }
        if (threadIdx.x == 0) {
            A.sc->dro = cK.mcorr ? red[0] / A.sc->tv : 0.0;
            A.sc->done_ctr = 0;
        }
    }
}

// End of step: mass correction, velocity and c from the filtered state
// (filter_variables + get_velocity_from_momentum + get_c_from_psi) and the step's scalar
// bookkeeping (error-norm history, time, itime).
template <int FORM>
__global__ void __launch_bounds__(128) k_finalize(StageArgs A, int advance) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const double dro = A.sc->dro;
    if (i < cK.npfb) {
        const Fields &F = A.out;
        double ro = F.ro[i];
        if (cK.mcorr) ro = ro - dro;
        F.ro[i] = ro;
        double ooro = 1.0 / ro;
        F.u[i] = F.rou[i] * ooro;
        F.v[i] = F.rov[i] * ooro;
        if (FORM == SUNSET_FORM_LC) {
            double cxx, cxy, cyy;
            lc_c_from_psi(F.q[0][i], F.q[1][i], F.q[2][i], &cxx, &cxy, &cyy);
            F.c[0][i] = cxx; F.c[1][i] = cxy; F.c[2][i] = cyy;
        } else if (FORM == SUNSET_FORM_CHL) {
            double cxx, cxy, cyy, czz;
            chl_c_from_psi(F.q[0][i], F.q[1][i], F.q[2][i], &cxx, &cxy, &cyy, &czz);
            F.c[0][i] = cxx; F.c[1][i] = cxy; F.c[2][i] = cyy; F.c[3][i] = czz;
        }
    }
    if (advance && i == 0) {
        DevScalars *sc = A.sc;
        double e = __longlong_as_double((long long)sc->emax_bits);
        double emax = (e > 1.0e-16) ? e : 1.0e-16;
        if (!(e == e) || isinf(e)) sc->err = 1;
        sc->emax_nm1 = sc->emax_n;
        sc->emax_n = sc->emax_np1;
        sc->emax_np1 = emax;
        sc->emax_bits = 0ull;
        sc->time = sc->time + sc->dt;
        sc->itime = sc->itime + 1;
    }
}

// set_tstep (step.F90:569-622) over the current state: block minima of s/(|u|+c) and
// s^2 rho/mu, folded into dt_cfl and dt_parabolic by k_pid / the host.
__global__ void __launch_bounds__(128) k_tstep(const double *u, const double *v, const double *ro, const double *sp,
                                                const int *ntype, int npfb, DevScalars *sc) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double tc = 1.0e10, tp = 1.0e10;
    if (i < npfb) {
        double umax = sqrt((u[i] * u[i] + v[i] * v[i]) + 0.0 * 0.0);
        double uplusc = umax + cK.c_sound;
        tc = (ntype[i] == 2) ? (0.8 * sp[i]) / uplusc : sp[i] / uplusc;
        tp = ((sp[i] * sp[i]) * ro[i]) / cK.visc_total;
    }
    block_min_bits(dbits(tc), &sc->cfl_bits);
    block_min_bits(dbits(tp), &sc->par_bits);
}

// set_tstep_PID, step.F90:624-682.
__global__ void k_pid(DevScalars *sc) {
    double dcfl = __longlong_as_double((long long)sc->cfl_bits);
    double dvisc = __longlong_as_double((long long)sc->par_bits);
    sc->dt_cfl = (1.0 * dcfl) * cK.L_char;
    sc->dt_par = (((2.0 / 3.0) * dvisc) * cK.L_char) * cK.L_char;
    double facA = (0.49 / 2.0) * log(1.0e-5 / sc->emax_np1);
    double facB = (0.34 / 2.0) * log(sc->emax_n / 1.0e-5);
    double facC = (0.1 / 2.0) * log(1.0e-5 / sc->emax_nm1);
    double dtfactor = 0.9 * exp((facA + facB) + facC);
    dtfactor = (0.5 > dtfactor) ? 0.5 : dtfactor;
    dtfactor = (1.02 < dtfactor) ? 1.02 : dtfactor;
    double dt = sc->dt * dtfactor;
    double dt_max = (sc->dt_cfl < sc->dt_par) ? sc->dt_cfl : sc->dt_par;
    if (dt > dt_max) dt = dt_max;
    sc->dt = dt;
    sc->cfl_bits = 0x7ff0000000000000ull;
    sc->par_bits = 0x7ff0000000000000ull;
}

__global__ void k_tstep_fold(DevScalars *sc) {
    double dcfl = __longlong_as_double((long long)sc->cfl_bits);
    double dvisc = __longlong_as_double((long long)sc->par_bits);
    sc->dt_cfl = (1.0 * dcfl) * cK.L_char;
    sc->dt_par = (((2.0 / 3.0) * dvisc) * cK.L_char) * cK.L_char;
}

// ---------------------------------------------------------------------------------------
// Single operators of the C-ABI (derivatives.F90), on a field in internal order.
// ---------------------------------------------------------------------------------------
__global__ void k_op_grad_lap(StageArgs A, const double *phi, double *gx, double *gy, double *lap) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if ((i >> 5) >= cK.nslices) return;
    const long long base = A.slice_ptr[i >> 5];
    const int ws = A.slice_ws[i >> 5];
    double sx = 0.0, sy = 0.0, sl = 0.0;
    for (int k = 0; k < ws; k++) {
        const long long o = sell_at(base, k, i & 31);
        const int j = __ldg(A.lidx + o) & kLinkMask;
        const double pj = phi[j];
        sx = sx + pj * __ldg(A.wx + o);
        sy = sy + pj * __ldg(A.wy + o);
        sl = sl + pj * __ldg(A.wl + o);
    }
    if (i >= cK.npfb) return;
    const double p = phi[i];
    if (gx) gx[i] = sx - p * A.gsx[i];
    if (gy) gy[i] = sy - p * A.gsy[i];
    if (lap) lap[i] = sl - p * A.lsum[i];
}

__global__ void k_op_filter(StageArgs A, const double *phi, double *out, int term_only) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if ((i >> 5) >= cK.nslices) return;
    const long long base = A.slice_ptr[i >> 5];
    const int w = A.slice_w[i >> 5];
    double t = 0.0;
    for (int k = 0; k < w; k++) {
        const long long o = sell_at(base, k, i & 31);
        const int j = __ldg(A.lidx + o) & kLinkMask;
        t = t + phi[j] * __ldg(A.wh + o);
    }
    if (i >= cK.npfb) return;
    const double p = phi[i];
    out[i] = term_only ? (t - p * A.hsum[i]) : p + (t - p * A.hsum[i]);
}

// initial_solution (setup_flow.F90:24-173) on internal-order device arrays.
// Wall nodes get zero velocity (setup_flow.F90:266-280).
__global__ void k_set_state(int npfb, int form, const double *ro, const double *u, const double *v,
                            const double *cxx, const double *cxy, const double *cyy, const double *czz,
                            const int *ntype, int has_walls, Fields F) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= npfb) return;
    double r = ro[i];
    double ui = u[i], vi = v[i];
    if (has_walls && ntype[i] == 0) { ui = 0.0; vi = 0.0; }
    F.ro[i] = r;
    F.u[i] = ui;
    F.v[i] = vi;
    F.rou[i] = r * ui;
    F.rov[i] = r * vi;
    double c0 = cxx[i], c1 = cxy[i], c2 = cyy[i], c3 = czz[i];
    if (form == SUNSET_FORM_LC) {
        double p0, p1, p2;
        lc_psi_from_c(c0, c1, c2, &p0, &p1, &p2);
        F.q[0][i] = p0; F.q[1][i] = p1; F.q[2][i] = p2; F.q[3][i] = 0.0;
        lc_c_from_psi(p0, p1, p2, &c0, &c1, &c2);
        F.c[0][i] = c0; F.c[1][i] = c1; F.c[2][i] = c2; F.c[3][i] = c3;
    } else if (form == SUNSET_FORM_CHL) {
        double p0, p1, p2, p3;
        chl_psi_from_c(c0, c1, c2, c3, &p0, &p1, &p2, &p3);
        F.q[0][i] = p0; F.q[1][i] = p1; F.q[2][i] = p2; F.q[3][i] = p3;
        chl_c_from_psi(p0, p1, p2, &c0, &c1, &c2, &c3);
        F.c[0][i] = c0; F.c[1][i] = c1; F.c[2][i] = c2; F.c[3][i] = c3;
    } else {
        F.q[0][i] = c0; F.q[1][i] = c1; F.q[2][i] = c2; F.q[3][i] = c3;
    }
}

// Conservative state given directly (ro, rou, rov, q0..q3), derived fields recomputed
// as get_velocity_from_momentum / get_c_from_psi do.
__global__ void k_set_conservative(int npfb, int form, const double *ro, const double *rou, const double *rov,
                                   const double *q0, const double *q1, const double *q2, const double *q3, Fields F) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= npfb) return;
    F.ro[i] = ro[i]; F.rou[i] = rou[i]; F.rov[i] = rov[i];
    F.q[0][i] = q0[i]; F.q[1][i] = q1[i]; F.q[2][i] = q2[i]; F.q[3][i] = q3[i];
    double ooro = 1.0 / ro[i];
    F.u[i] = rou[i] * ooro;
    F.v[i] = rov[i] * ooro;
    if (form == SUNSET_FORM_LC) {
        double c0, c1, c2;
        lc_c_from_psi(q0[i], q1[i], q2[i], &c0, &c1, &c2);
        F.c[0][i] = c0; F.c[1][i] = c1; F.c[2][i] = c2; F.c[3][i] = 1.0;
    } else if (form == SUNSET_FORM_CHL) {
        double c0, c1, c2, c3;
        chl_c_from_psi(q0[i], q1[i], q2[i], &c0, &c1, &c2, &c3);
        F.c[0][i] = c0; F.c[1][i] = c1; F.c[2][i] = c2; F.c[3][i] = c3;
    }
}

__global__ void k_ke_mass(int npfb, Fields F, const double *vol, double *partials) {
    __shared__ double s1[128], s2[128];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double ke = 0.0, m = 0.0;
    if (i < npfb) {
        ke = ((0.5 * F.ro[i]) * (F.u[i] * F.u[i] + F.v[i] * F.v[i])) * vol[i];
        m = F.ro[i] * vol[i];
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
        partials[2 * blockIdx.x] = s1[0];
        partials[2 * blockIdx.x + 1] = s2[0];
    }
}

__global__ void k_sum_vol(int npfb, const double *vol, double *partials) {
    __shared__ double s1[128];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    s1[threadIdx.x] = i < npfb ? vol[i] : 0.0;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) s1[threadIdx.x] = s1[threadIdx.x] + s1[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) partials[blockIdx.x] = s1[0];
}

__global__ void k_fold_partials(const double *partials, int n, double *out) {
    __shared__ double sm[128];
    double acc = 0.0;
    for (int b = threadIdx.x; b < n; b += blockDim.x) acc = acc + partials[b];
    sm[threadIdx.x] = acc;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) sm[threadIdx.x] = sm[threadIdx.x] + sm[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = sm[0];
}

// Kernel arguments over buffer `from`.  step: the time step's link stream (bank-aware order;
// FP32 weights with their own sums in mixed precision); otherwise the reference-order FP64
// arrays of the single-operator entry points.
StageArgs make_args(Handle *H, int from, int stage, bool step = false) {
    const bool mx = step && H->cfg.precision == SUNSET_MIXED;
    StageArgs A{};
    A.slice_ptr = H->slice_ptr;
    A.slice_ws = H->slice_ws;
    A.slice_w = H->slice_w;
    A.lidx = H->lidx;
    A.lloc = step ? H->lloc_s : H->lloc;
    A.halo_ptr = H->halo_ptr;
    A.halo = H->halo;
    A.hmax = H->halo_max;
    if (step) {
        A.wx = H->wx_s; A.wy = H->wy_s; A.wl = H->wl_s; A.wh = H->wh_s;
    } else {
        A.wx = H->wx; A.wy = H->wy; A.wl = H->wl; A.wh = H->wh;
    }
    A.wx32 = H->wx32; A.wy32 = H->wy32; A.wl32 = H->wl32; A.wh32 = H->wh32;
    if (mx) {
        A.gsx = H->gsx32; A.gsy = H->gsy32; A.lsum = H->lsum32; A.hsum = H->hsum32;
    } else {
        A.gsx = H->gsx; A.gsy = H->gsy; A.lsum = H->lsum; A.hsum = H->hsum;
    }
    A.vol = H->vol;
    A.py_node = H->py;
    A.ntype = H->ntype;
    A.rnx = H->rnx;
    A.rny = H->rny;
    A.in = H->buf[from];
    A.out = H->buf[from ^ 1];
    for (int f = 0; f < 7; f++) {
        A.reg[f] = H->reg[f]; A.eacc[f] = H->eacc[f]; A.rhs[f] = H->rhs[f];
        A.dreg[f] = H->dreg32[f]; A.eacc32[f] = H->eacc32[f];
    }
    A.sc = H->dsc;
    A.partials = H->partials;
    A.stage = stage;
    return A;
}

int upload_consts(Handle *H) {
    const StepConsts K = step_consts(H->cfg, H->npfb, H->nslices, H->has_mirrors, H->nb > 0);
    SUNSET_CUDA(H, cudaMemcpyToSymbolAsync(cK, &K, sizeof(K), 0, cudaMemcpyHostToDevice, H->stream));
    return 0;
}

constexpr size_t kMaxStageSmem = 200 * 1024;

// Opt the staged kernels into large dynamic shared memory on the handle's device.
int set_smem_attributes(Handle *H) {
#define SUNSET_SMEM_ATTR(K) SUNSET_CUDA(H, cudaFuncSetAttribute(K, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kMaxStageSmem))
    SUNSET_SMEM_ATTR((k_stage<SUNSET_FORM_DI, false, false>));
    SUNSET_SMEM_ATTR((k_stage<SUNSET_FORM_DI, true, false>));
    SUNSET_SMEM_ATTR((k_stage<SUNSET_FORM_CHL, false, false>));
    SUNSET_SMEM_ATTR((k_stage<SUNSET_FORM_CHL, true, false>));
    SUNSET_SMEM_ATTR((k_stage<SUNSET_FORM_LC, false, false>));
    SUNSET_SMEM_ATTR((k_stage<SUNSET_FORM_NEWT, false, false>));
    SUNSET_SMEM_ATTR((k_filter<SUNSET_FORM_DI, false>));
    SUNSET_SMEM_ATTR((k_filter<SUNSET_FORM_CHL, false>));
    SUNSET_SMEM_ATTR((k_filter<SUNSET_FORM_LC, false>));
    SUNSET_SMEM_ATTR((k_filter<SUNSET_FORM_NEWT, false>));
    if (H->cfg.precision == SUNSET_MIXED) {
        SUNSET_SMEM_ATTR((k_stage<SUNSET_FORM_DI, false, true>));
        SUNSET_SMEM_ATTR((k_stage<SUNSET_FORM_DI, true, true>));
        SUNSET_SMEM_ATTR((k_stage<SUNSET_FORM_CHL, false, true>));
        SUNSET_SMEM_ATTR((k_stage<SUNSET_FORM_CHL, true, true>));
        SUNSET_SMEM_ATTR((k_stage<SUNSET_FORM_LC, false, true>));
        SUNSET_SMEM_ATTR((k_stage<SUNSET_FORM_NEWT, false, true>));
        SUNSET_SMEM_ATTR((k_filter<SUNSET_FORM_DI, true>));
        SUNSET_SMEM_ATTR((k_filter<SUNSET_FORM_CHL, true>));
        SUNSET_SMEM_ATTR((k_filter<SUNSET_FORM_LC, true>));
        SUNSET_SMEM_ATTR((k_filter<SUNSET_FORM_NEWT, true>));
    }
#undef SUNSET_SMEM_ATTR
    return 0;
}

inline bool is_mx(const Handle *H) { return H->cfg.precision == SUNSET_MIXED; }

template <int FORM, bool MD>
int launch_stage(Handle *H, const StageArgs &A, bool mx) {
    const size_t smem = halo_doubles(ngather(FORM, MD), H->halo_max) * sizeof(double) +
                        (mx ? LinkRing<true, 3, ring_depth(true)>::bytes() : LinkRing<false, 3, ring_depth(false)>::bytes());
    if (smem > kMaxStageSmem) return set_err(H, SUNSET_ERR_SCOPE, "tile halo too large for shared memory");
    if (mx) k_stage<FORM, MD, true><<<H->ntiles, kTile, smem, H->stream>>>(A);
    else k_stage<FORM, MD, false><<<H->ntiles, kTile, smem, H->stream>>>(A);
    return 0;
}

// A must come from make_args(..., step = true); mx is the handle's precision.
int launch_stage_any(Handle *H, const StageArgs &A, bool mx) {
    const bool md = H->cfg.Mdiff != 0.0;
    switch (H->cfg.form) {
    case SUNSET_FORM_DI: return md ? launch_stage<SUNSET_FORM_DI, true>(H, A, mx) : launch_stage<SUNSET_FORM_DI, false>(H, A, mx);
    case SUNSET_FORM_CHL: return md ? launch_stage<SUNSET_FORM_CHL, true>(H, A, mx) : launch_stage<SUNSET_FORM_CHL, false>(H, A, mx);
    case SUNSET_FORM_LC: return launch_stage<SUNSET_FORM_LC, false>(H, A, mx);
    default: return launch_stage<SUNSET_FORM_NEWT, false>(H, A, mx);
    }
}

template <int FORM>
int launch_filter(Handle *H, const StageArgs &A, bool mx) {
    constexpr int nf = (FORM == SUNSET_FORM_DI) ? 7 : (FORM == SUNSET_FORM_NEWT ? 3 : 6);
    const size_t smem = halo_doubles(nf, H->halo_max) * sizeof(double) +
                        (mx ? LinkRing<true, 1, ring_depth(true)>::bytes() : LinkRing<false, 1, ring_depth(false)>::bytes());
    if (smem > kMaxStageSmem) return set_err(H, SUNSET_ERR_SCOPE, "tile halo too large for shared memory");
    if (mx) k_filter<FORM, true><<<H->ntiles, kTile, smem, H->stream>>>(A);
    else k_filter<FORM, false><<<H->ntiles, kTile, smem, H->stream>>>(A);
    return 0;
}

// The kernels of one step.  stage_ev (optional, 8 events): recorded before and after each
// of the four RK stage launches, for timing the stage kernel inside a real step sequence.
template <int FORM>
int launch_step_kernels(Handle *H, int from, int pid, cudaEvent_t *stage_ev) {
    const int TB = 128;
    cudaStream_t st = H->stream;
    const bool mx = is_mx(H);
    if (pid) k_pid<<<1, 1, 0, st>>>(H->dsc);
    int b = from;
    for (int s = 0; s < 4; s++) {
        StageArgs A = make_args(H, b, s, true);
        if (stage_ev) SUNSET_CUDA(H, cudaEventRecord(stage_ev[2 * s], st));
        if (int rc = launch_stage_any(H, A, mx)) return rc;
        if (stage_ev) SUNSET_CUDA(H, cudaEventRecord(stage_ev[2 * s + 1], st));
        b ^= 1;
    }
    StageArgs F = make_args(H, b, 5, true);
    if (int rc = launch_filter<FORM>(H, F, mx)) return rc;
    b ^= 1;
    StageArgs Z = make_args(H, b ^ 1, 5, true);  // in = filter input, out = filtered buffer
    const int fb = (H->npfb + TB - 1) / TB;
    k_finalize<FORM><<<fb, TB, 0, st>>>(Z, 1);
    k_tstep<<<fb, TB, 0, st>>>(H->buf[b].u, H->buf[b].v, H->buf[b].ro, H->sp, H->ntype, H->npfb, H->dsc);
    return 0;
}

int launch_step(Handle *H, int from, int pid, cudaEvent_t *stage_ev = nullptr) {
    switch (H->cfg.form) {
    case SUNSET_FORM_DI: return launch_step_kernels<SUNSET_FORM_DI>(H, from, pid, stage_ev);
    case SUNSET_FORM_CHL: return launch_step_kernels<SUNSET_FORM_CHL>(H, from, pid, stage_ev);
    case SUNSET_FORM_LC: return launch_step_kernels<SUNSET_FORM_LC>(H, from, pid, stage_ev);
    default: return launch_step_kernels<SUNSET_FORM_NEWT>(H, from, pid, stage_ev);
    }
}

}  // namespace

// ---------------------------------------------------------------------------------------
int state_alloc(Handle *H) {
    if (H->dsc) return 0;
    if (int rc = set_smem_attributes(H)) return rc;
    const int n = H->npfb;
    for (int b = 0; b < 2; b++) {
        Fields &F = H->buf[b];
        if (dalloc(H, &F.ro, n) || dalloc(H, &F.rou, n) || dalloc(H, &F.rov, n) || dalloc(H, &F.u, n) ||
            dalloc(H, &F.v, n))
            return SUNSET_ERR_NOMEM;
        for (int k = 0; k < 4; k++)
            if (dalloc(H, &F.q[k], n)) return SUNSET_ERR_NOMEM;
        if (H->cfg.form == SUNSET_FORM_DI) {
            for (int k = 0; k < 4; k++) F.c[k] = F.q[k];
        } else {
            for (int k = 0; k < 4; k++)
                if (dalloc(H, &F.c[k], n)) return SUNSET_ERR_NOMEM;
        }
    }
    for (int f = 0; f < 7; f++) {
        if (dalloc(H, &H->rhs[f], n)) return SUNSET_ERR_NOMEM;
        if (is_mx(H)) {
            if (dalloc(H, &H->dreg32[f], n) || dalloc(H, &H->eacc32[f], n)) return SUNSET_ERR_NOMEM;
        } else {
            if (dalloc(H, &H->reg[f], n) || dalloc(H, &H->eacc[f], n)) return SUNSET_ERR_NOMEM;
        }
    }
    const int nthr = H->nslices * kSlice;
    H->npart = (nthr + 127) / 128 + 1;
    if (dalloc(H, &H->partials, 2 * (size_t)H->npart + 16) || dalloc(H, &H->dsc, 1) || dalloc(H, &H->tmpd, 4 * (size_t)n))
        return SUNSET_ERR_NOMEM;
    SUNSET_CUDA(H, cudaMemsetAsync(H->dsc, 0, sizeof(DevScalars), H->stream));
    return 0;
}

static int init_scalars(Handle *H) {
    DevScalars s{};
    s.dt = 1.0e-6;
    s.time = 0.0;
    s.emax_nm1 = s.emax_n = s.emax_np1 = 1.0e-5;  // pid_tol, setup_flow.F90:149-152
    s.cfl_bits = 0x7ff0000000000000ull;
    s.par_bits = 0x7ff0000000000000ull;
    SUNSET_CUDA(H, cudaMemcpyAsync(H->dsc, &s, sizeof(s), cudaMemcpyHostToDevice, H->stream));
    // sum of volumes (constant), same tree as the mass correction
    const int TB = 128, nb = (H->npfb + TB - 1) / TB;
    k_sum_vol<<<nb, TB, 0, H->stream>>>(H->npfb, H->vol, H->partials);
    k_fold_partials<<<1, 128, 0, H->stream>>>(H->partials, nb, &H->dsc->tv);
    SUNSET_CUDA(H, cudaGetLastError());
    return 0;
}

int state_set_device(Handle *H, const double *ro, const double *u, const double *v, const double *cxx,
                     const double *cxy, const double *cyy, const double *czz) {
    int rc = upload_consts(H);
    if (rc) return rc;
    H->cur = 0;
    k_set_state<<<(H->npfb + 127) / 128, 128, 0, H->stream>>>(H->npfb, H->cfg.form, ro, u, v, cxx, cxy, cyy, czz,
                                                              H->ntype, H->nb > 0, H->buf[0]);
    SUNSET_CUDA(H, cudaGetLastError());
    rc = init_scalars(H);
    if (rc) return rc;
    return set_tstep_device(H);
}

int state_set_conservative_device(Handle *H, const double *const *f7) {
    int rc = upload_consts(H);
    if (rc) return rc;
    k_set_conservative<<<(H->npfb + 127) / 128, 128, 0, H->stream>>>(H->npfb, H->cfg.form, f7[0], f7[1], f7[2],
                                                                     f7[3], f7[4], f7[5], f7[6], H->buf[H->cur]);
    SUNSET_CUDA(H, cudaGetLastError());
    return 0;
}

int set_tstep_device(Handle *H) {
    const Fields &F = H->buf[H->cur];
    DevScalars *sc = H->dsc;
    unsigned long long inf = 0x7ff0000000000000ull;
    SUNSET_CUDA(H, cudaMemcpyAsync(&sc->cfl_bits, &inf, sizeof(inf), cudaMemcpyHostToDevice, H->stream));
    SUNSET_CUDA(H, cudaMemcpyAsync(&sc->par_bits, &inf, sizeof(inf), cudaMemcpyHostToDevice, H->stream));
    k_tstep<<<(H->npfb + 127) / 128, 128, 0, H->stream>>>(F.u, F.v, F.ro, H->sp, H->ntype, H->npfb, sc);
    k_tstep_fold<<<1, 1, 0, H->stream>>>(sc);
    SUNSET_CUDA(H, cudaGetLastError());
    return 0;
}

int rhs_only(Handle *H) {
    int rc = upload_consts(H);
    if (rc) return rc;
    StageArgs A = make_args(H, H->cur, 4, true);
    if ((rc = launch_stage_any(H, A, is_mx(H)))) return rc;
    SUNSET_CUDA(H, cudaGetLastError());
    return 0;
}

int step_run(Handle *H, double dt, int nsteps, int mode) {
    int rc = upload_consts(H);
    if (rc) return rc;
    cudaStream_t st = H->stream;
    if (mode == 0) SUNSET_CUDA(H, cudaMemcpyAsync(&H->dsc->dt, &dt, sizeof(double), cudaMemcpyHostToDevice, st));
    for (int s = 0; s < nsteps; s++) {
        int from = H->cur;
        if (!H->graph[from] || H->graph_mode[from] != mode) {
            if (H->graph[from]) { cudaGraphExecDestroy(H->graph[from]); H->graph[from] = nullptr; }
            cudaGraph_t g;
            SUNSET_CUDA(H, cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
            int lrc = launch_step(H, from, mode);
            cudaError_t ce = cudaStreamEndCapture(st, &g);
            if (lrc) return lrc;
            SUNSET_CUDA(H, ce);
            SUNSET_CUDA(H, cudaGraphInstantiate(&H->graph[from], g, 0));
            cudaGraphDestroy(g);
            H->graph_mode[from] = mode;
        }
        SUNSET_CUDA(H, cudaGraphLaunch(H->graph[from], st));
        H->cur ^= 1;
    }
    return 0;
}

int op_gradient(Handle *H, const double *phi, double *gx, double *gy) {
    int rc = upload_consts(H);
    if (rc) return rc;
    StageArgs A = make_args(H, 0, 5);
    const int TB = 128, nblk = (H->nslices * kSlice + TB - 1) / TB;
    k_op_grad_lap<<<nblk, TB, 0, H->stream>>>(A, phi, gx, gy, nullptr);
    SUNSET_CUDA(H, cudaGetLastError());
    return 0;
}

int op_laplacian(Handle *H, const double *phi, double *lap) {
    int rc = upload_consts(H);
    if (rc) return rc;
    StageArgs A = make_args(H, 0, 5);
    const int TB = 128, nblk = (H->nslices * kSlice + TB - 1) / TB;
    k_op_grad_lap<<<nblk, TB, 0, H->stream>>>(A, phi, nullptr, nullptr, lap);
    SUNSET_CUDA(H, cudaGetLastError());
    return 0;
}

int op_filter(Handle *H, const double *phi, double *out, int term_only) {
    int rc = upload_consts(H);
    if (rc) return rc;
    StageArgs A = make_args(H, 0, 5);
    const int TB = 128, nblk = (H->nslices * kSlice + TB - 1) / TB;
    k_op_filter<<<nblk, TB, 0, H->stream>>>(A, phi, out, term_only);
    SUNSET_CUDA(H, cudaGetLastError());
    return 0;
}

int reduce_ke_mass(Handle *H, double *ke, double *mass) {
    const int TB = 128, nb = (H->npfb + TB - 1) / TB;
    double *p = H->partials;
    k_ke_mass<<<nb, TB, 0, H->stream>>>(H->npfb, H->buf[H->cur], H->vol, p);
    std::vector<double> hp(2 * (size_t)nb);
    SUNSET_CUDA(H, cudaMemcpyAsync(hp.data(), p, hp.size() * sizeof(double), cudaMemcpyDeviceToHost, H->stream));
    SUNSET_CUDA(H, cudaStreamSynchronize(H->stream));
    double k = 0.0, m = 0.0;
    for (int b = 0; b < nb; b++) { k += hp[2 * b]; m += hp[2 * b + 1]; }
    if (ke) *ke = k;
    if (mass) *mass = m;
    return 0;
}

// Average duration of the RK stage kernel inside real steps: `reps` steps at the current dt
// (fixed-dt mode), each launched directly rather than as a graph, with CUDA events on the
// handle's stream around each of the four stage launches.  Advances the state by reps
// steps.  Also returns the stage kernel's algorithmic bytes per launch.
int time_stage_kernel(Handle *H, int reps, double *ms, double *bytes) {
    int rc = upload_consts(H);
    if (rc) return rc;
    if (reps < 1) reps = 1;
    const bool mx = is_mx(H);
    std::vector<cudaEvent_t> ev(8 * (size_t)reps);
    for (auto &e : ev) SUNSET_CUDA(H, cudaEventCreate(&e));
    for (int r = 0; r < reps; r++) {
        if ((rc = launch_step(H, H->cur, 0, ev.data() + 8 * r))) break;
        H->cur ^= 1;
    }
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
    // Algorithmic bytes of one stage launch, averaged over the four stages: each node's
    // small links once (16-bit local index + 3 weights of 8 bytes, 4 in the mixed path;
    // links, not padded SELL slots), its state and derived fields read once (the halo
    // copies of neighbours' values are re-reads), the RK registers S and E read in stages
    // 1-3 and written in stages 0-2 (8 bytes, 4 in the mixed path), the next state with
    // its derived fields written (conservative fields only after stage 3), and the stencil
    // sums and ordinate read.
    long long links = 0;
    {
        std::vector<int> cs(H->npfb);
        SUNSET_CUDA(H, cudaMemcpy(cs.data(), H->cnt_small, cs.size() * sizeof(int), cudaMemcpyDeviceToHost));
        for (int c : cs) links += c;
    }
    const int form = H->cfg.form;
    const int nf = form == SUNSET_FORM_DI ? 7 : 6;      // evolved fields (S and E registers)
    const int nread = form == SUNSET_FORM_DI ? 9 : 13;   // state + derived fields of a node
    const int nwrite = form == SUNSET_FORM_DI ? 9 : 13;  // next state + derived fields (stages 0-2)
    const double wb = mx ? 4.0 : 8.0;
    *bytes = (double)links * (2 + 3 * wb) +
             (double)H->npfb * (8.0 * nread + 3.0 * nf * wb + 8.0 * (3.0 * nwrite + 7.0) / 4.0 + 8.0 * 4);
    return 0;
}


// =======================================================================================
// Adjoint of the fixed-dt time step (log-conformation form, periodic node sets, FP64).
//
// The forward map of one step is U_{n+1} = mcorr(filter(U4)), with the four stages
// U_{s+1} = S_s + alpha_s dt R(U_s), S_{s+1} = S_s + beta_s dt R(U_s), S_0 = U_0
// (alpha = a21, a32, a43, b4; beta = b1, b2, b3; step.F90:291-343).  Its reverse, given the
// adjoint of U_{n+1}: the filter's transpose (with the mass correction's), then for
// s = 3..0: R_bar = dt (alpha_s U_bar_{s+1} + beta_s S_bar_{s+1}), S_bar_s = U_bar_{s+1} +
// S_bar_{s+1}, U_bar_s = dR(U_s)^T R_bar (+ S_bar_0 at s = 0).  dR^T is the pointwise reverse
// of adjoint.cuh followed by the transposed stencils: node j collects w_ij g_bar_i from every
// node i whose links reach it, through a reverse-neighbour list built once (a gather, in a
// fixed order, without atomics), plus its own -sum(w) g_bar_j terms, and the derived fields
// (u = rho u / rho, c from psi) are reversed into the conservative state.
//
// Stage inputs are recomputed per segment of `checkpoint_every` steps from the state stored
// at the segment's start, and kept (13 fields per stage) for that segment's reverse sweep.
// =======================================================================================
namespace {

struct AdjArgs {
    int npfb;
    const long long *rptr;      // reverse links of node j: [rptr[j], rptr[j+1])
    const int *rslot, *rnode;   // SELL slot (reference order) and the node owning it
    const unsigned char *rcode; // bits 0-1: reflection code, bit 2: a small link (stencils of the stage)
    const double *wx, *wy, *wl, *wh;
    const double *gsx, *gsy, *lsum, *hsum, *vol;
    double *gb[kAdjG];
    double *sb[kAdjS];
    double *ub_in[7], *ub_out[7], *sbar[7];
    double *tpart;
    const double *mc_sum, *mc_tv;  // sum of rho_bar and of the volumes (mass correction)
    double dt, alpha, beta;
    int first, add_sbar, mcorr;
};

__device__ __forceinline__ double sgn_u(int c) { return (c == 1 || c == 3) ? -1.0 : 1.0; }
__device__ __forceinline__ double sgn_v(int c) { return (c == 2 || c == 3) ? -1.0 : 1.0; }
__device__ __forceinline__ double sgn_xy(int c) { return (c == 1 || c == 2) ? -1.0 : 1.0; }

// Stage adjoint, part 1: the stage's stencil sums g at its input state (the forward gather),
// R_bar and S_bar of each node, and the pointwise reverse: g_bar, the node's direct state
// adjoint and block sums of the parameter adjoint.
__global__ void __launch_bounds__(kTile, 2) k_adj_point_lc(StageArgs A, AdjArgs B) {
    extern __shared__ __align__(16) double smem[];
    constexpr int NG = ngather(SUNSET_FORM_LC, false);
    const int i = blockIdx.x * kTile + threadIdx.x;
    bool active = (i >> 5) < cK.nslices;
    LinkRing<false, 3, ring_depth(false)> R;
    R.src[0] = reinterpret_cast<const double2 *>(A.wx);
    R.src[1] = reinterpret_cast<const double2 *>(A.wy);
    R.src[2] = reinterpret_cast<const double2 *>(A.wl);
    R.init(smem + halo_doubles(NG, A.hmax), reinterpret_cast<const unsigned *>(A.lloc),
           active ? (A.slice_ptr[i >> 5] >> 1) + (i & 31) : 0, active ? A.slice_ws[i >> 5] >> 1 : 0);
    R.prologue();
    load_halo<NG>(A, smem, [&](int f) { return gather_src<SUNSET_FORM_LC, false>(A.in, f); });
    Grads g;
    if (active) gather_stage<SUNSET_FORM_LC, false, false>(A, i, smem, R, g);
    double t0 = 0.0, t1 = 0.0;
    if (active && i < B.npfb) {
        const Fields &F = A.in;
        const double s[kAdjS] = {F.ro[i], F.rou[i], F.rov[i], F.q[0][i], F.q[1][i], F.q[2][i]};
        const double gv[kAdjG] = {g.ro_x, g.ro_y, g.u_x, g.u_y, g.lapu, g.v_x, g.v_y, g.lapv, g.cxx_x, g.cxy_x,
                                  g.cxy_y, g.cyy_y, g.pxx_x, g.pxx_y, g.pxy_x, g.pxy_y, g.pyy_x, g.pyy_y};
        double rb[kAdjR];
        for (int f = 0; f < kAdjR; f++) {
            const double ui = B.ub_in[f][i], si = B.sbar[f][i];
            rb[f] = B.dt * (B.alpha * ui + B.beta * si);
            B.sbar[f][i] = ui + si;
        }
        double sbv[kAdjS] = {0, 0, 0, 0, 0, 0}, gbv[kAdjG], tb[2] = {0.0, 0.0};
        for (int k = 0; k < kAdjG; k++) gbv[k] = 0.0;
        p_adjoint_lc(cK, s, gv, B.first != 0, rb, sbv, gbv, tb);
        for (int k = 0; k < kAdjG; k++) B.gb[k][i] = gbv[k];
        for (int k = 0; k < kAdjS; k++) B.sb[k][i] = sbv[k];
        t0 = tb[0];
        t1 = tb[1];
    }
    __shared__ double red[2][kTile];
    red[0][threadIdx.x] = t0;
    red[1][threadIdx.x] = t1;
    __syncthreads();
    for (int st = blockDim.x / 2; st > 0; st >>= 1) {
        if ((int)threadIdx.x < st) {
            red[0][threadIdx.x] = red[0][threadIdx.x] + red[0][threadIdx.x + st];
            red[1][threadIdx.x] = red[1][threadIdx.x] + red[1][threadIdx.x + st];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        B.tpart[2 * blockIdx.x] = red[0][0];
        B.tpart[2 * blockIdx.x + 1] = red[1][0];
    }
}

// Stage adjoint, part 2: the transposed stencils and the reverse of the derived fields;
// writes U_bar of the stage's input state (+ S_bar at the first stage).
__global__ void __launch_bounds__(128) k_adj_transpose_lc(StageArgs A, AdjArgs B) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= B.npfb) return;
    double ph[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};  // rho, u, v, cxx, cxy, cyy, psixx, psixy, psiyy
    for (long long e = B.rptr[j]; e < B.rptr[j + 1]; e++) {
        const int code = B.rcode[e];
        if (!(code & 4)) continue;
        const int o = B.rslot[e], i = B.rnode[e], rc = code & 3;
        const double wx = B.wx[o], wy = B.wy[o], wl = B.wl[o];
        ph[0] += wx * B.gb[G_RO_X][i] + wy * B.gb[G_RO_Y][i];
        ph[1] += sgn_u(rc) * (wx * B.gb[G_U_X][i] + wy * B.gb[G_U_Y][i] + wl * B.gb[G_LAPU][i]);
        ph[2] += sgn_v(rc) * (wx * B.gb[G_V_X][i] + wy * B.gb[G_V_Y][i] + wl * B.gb[G_LAPV][i]);
        ph[3] += wx * B.gb[G_CXX_X][i];
        ph[4] += sgn_xy(rc) * (wx * B.gb[G_CXY_X][i] + wy * B.gb[G_CXY_Y][i]);
        ph[5] += wy * B.gb[G_CYY_Y][i];
        ph[6] += wx * B.gb[G_PXX_X][i] + wy * B.gb[G_PXX_Y][i];
        ph[7] += sgn_xy(rc) * (wx * B.gb[G_PXY_X][i] + wy * B.gb[G_PXY_Y][i]);
        ph[8] += wx * B.gb[G_PYY_X][i] + wy * B.gb[G_PYY_Y][i];
    }
    const double gx = B.gsx[j], gy = B.gsy[j], ls = B.lsum[j];
    ph[0] -= gx * B.gb[G_RO_X][j] + gy * B.gb[G_RO_Y][j];
    ph[1] -= gx * B.gb[G_U_X][j] + gy * B.gb[G_U_Y][j] + ls * B.gb[G_LAPU][j];
    ph[2] -= gx * B.gb[G_V_X][j] + gy * B.gb[G_V_Y][j] + ls * B.gb[G_LAPV][j];
    ph[3] -= gx * B.gb[G_CXX_X][j];
    ph[4] -= gx * B.gb[G_CXY_X][j] + gy * B.gb[G_CXY_Y][j];
    ph[5] -= gy * B.gb[G_CYY_Y][j];
    ph[6] -= gx * B.gb[G_PXX_X][j] + gy * B.gb[G_PXX_Y][j];
    ph[7] -= gx * B.gb[G_PXY_X][j] + gy * B.gb[G_PXY_Y][j];
    ph[8] -= gx * B.gb[G_PYY_X][j] + gy * B.gb[G_PYY_Y][j];
    const Fields &F = A.in;
    const double ooro = 1.0 / F.ro[j];
    const double u = F.rou[j] * ooro, v = F.rov[j] * ooro;
    double pb[3] = {0.0, 0.0, 0.0};
    const double cb[3] = {ph[3], ph[4], ph[5]};
    lc_c_from_psi_adj(F.q[0][j], F.q[1][j], F.q[2][j], cb, pb);
    double U[7];
    U[0] = B.sb[0][j] + ph[0] - (ph[1] * u + ph[2] * v) * ooro;
    U[1] = B.sb[1][j] + ph[1] * ooro;
    U[2] = B.sb[2][j] + ph[2] * ooro;
    U[3] = B.sb[3][j] + ph[6] + pb[0];
    U[4] = B.sb[4][j] + ph[7] + pb[1];
    U[5] = B.sb[5][j] + ph[8] + pb[2];
    U[6] = 0.0;
    for (int f = 0; f < 7; f++) B.ub_out[f][j] = B.add_sbar ? U[f] + B.sbar[f][j] : U[f];
}

// Filter and mass correction reversed (rhs_lc.F90:818-893): U4_bar_j = Uf_bar_j (1 - hsum_j)
// + sum over reverse links w_h Uf_bar_i, with Uf_bar = U_bar and, for rho,
// rho_f_bar_i = rho_bar_i - vol_i sum(rho_bar) / sum(vol) when the mass is corrected.
__global__ void __launch_bounds__(128) k_adj_filter_lc(AdjArgs B) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= B.npfb) return;
    const double mc = B.mcorr ? *B.mc_sum / *B.mc_tv : 0.0;
    auto uf = [&](int f, int i) { return f == 0 ? B.ub_in[0][i] - B.vol[i] * mc : B.ub_in[f][i]; };
    double acc[6];
    const double own = 1.0 - B.hsum[j];
    for (int f = 0; f < 6; f++) acc[f] = uf(f, j) * own;
    for (long long e = B.rptr[j]; e < B.rptr[j + 1]; e++) {
        const int o = B.rslot[e], i = B.rnode[e], rc = B.rcode[e] & 3;
        const double w = B.wh[o];
        acc[0] += w * uf(0, i);
        acc[1] += w * sgn_u(rc) * uf(1, i);
        acc[2] += w * sgn_v(rc) * uf(2, i);
        acc[3] += w * uf(3, i);
        acc[4] += w * sgn_xy(rc) * uf(4, i);
        acc[5] += w * uf(5, i);
    }
    for (int f = 0; f < 6; f++) B.ub_out[f][j] = acc[f];
    B.ub_out[6][j] = 0.0;
}

// Adjoint of J = sum 1/2 rho |u|^2 vol at the final state.
__global__ void k_adj_objective(int npfb, Fields F, const double *vol, AdjArgs B) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= npfb) return;
    const double u = F.u[i], v = F.v[i], w = vol[i];
    B.ub_out[0][i] = -0.5 * (u * u + v * v) * w;
    B.ub_out[1][i] = u * w;
    B.ub_out[2][i] = v * w;
    for (int f = 3; f < 7; f++) B.ub_out[f][i] = 0.0;
}

// Sum of rho_bar (block partials) for the mass correction's adjoint.
__global__ void k_adj_sum(int npfb, const double *x, double *partials) {
    __shared__ double sm[128];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    sm[threadIdx.x] = i < npfb ? x[i] : 0.0;
    __syncthreads();
    for (int st = blockDim.x / 2; st > 0; st >>= 1) {
        if ((int)threadIdx.x < st) sm[threadIdx.x] = sm[threadIdx.x] + sm[threadIdx.x + st];
        __syncthreads();
    }
    if (threadIdx.x == 0) partials[blockIdx.x] = sm[0];
}

// acc[c] += sum_b partials[stride b + c] (c < stride), in block order.
__global__ void k_adj_fold(const double *partials, int n, int stride, double *acc, int accumulate) {
    __shared__ double sm[128];
    for (int c = 0; c < stride; c++) {
        double a = 0.0;
        for (int b = threadIdx.x; b < n; b += blockDim.x) a = a + partials[stride * b + c];
        sm[threadIdx.x] = a;
        __syncthreads();
        for (int st = blockDim.x / 2; st > 0; st >>= 1) {
            if ((int)threadIdx.x < st) sm[threadIdx.x] = sm[threadIdx.x] + sm[threadIdx.x + st];
            __syncthreads();
        }
        if (threadIdx.x == 0) acc[c] = accumulate ? acc[c] + sm[0] : sm[0];
        __syncthreads();
    }
}

// Transposed single operators (the adjoint of derivative application): out_j =
// sum over reverse links w_ij gbar_i - sum_k w_jk gbar_j, for d/dx, d/dy, Laplacian or filter.
__global__ void k_adj_apply_D(AdjArgs B, int which, const double *gbar, double *out) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= B.npfb) return;
    const double *w = which == 0 ? B.wx : which == 1 ? B.wy : which == 2 ? B.wl : B.wh;
    const double *sum = which == 0 ? B.gsx : which == 1 ? B.gsy : which == 2 ? B.lsum : B.hsum;
    double acc = 0.0;
    for (long long e = B.rptr[j]; e < B.rptr[j + 1]; e++) {
        if (which < 3 && !(B.rcode[e] & 4)) continue;
        acc += w[B.rslot[e]] * gbar[B.rnode[e]];
    }
    out[j] = acc - sum[j] * gbar[j];
}

StageArgs make_args_io(Handle *H, const Fields &in, const Fields &out, int stage) {
    StageArgs A = make_args(H, 0, stage, true);
    A.in = in;
    A.out = out;
    return A;
}

}  // namespace

// Reverse-neighbour lists (host build): for every node j the SELL slots, in the order of
// (owning node, link), whose link points at j.
static int adjoint_build_reverse(Handle *H) {
    if (H->rptr) return 0;
    const int n = H->npfb, nsl = H->nslices;
    const long long L = H->nlinks_sell;
    std::vector<int> lidx(L), cnt(n), cs(n);
    std::vector<long long> sptr(nsl + 1);
    SUNSET_CUDA(H, cudaMemcpy(lidx.data(), H->lidx, L * sizeof(int), cudaMemcpyDeviceToHost));
    SUNSET_CUDA(H, cudaMemcpy(cnt.data(), H->cnt, n * sizeof(int), cudaMemcpyDeviceToHost));
    SUNSET_CUDA(H, cudaMemcpy(cs.data(), H->cnt_small, n * sizeof(int), cudaMemcpyDeviceToHost));
    SUNSET_CUDA(H, cudaMemcpy(sptr.data(), H->slice_ptr, (nsl + 1) * sizeof(long long), cudaMemcpyDeviceToHost));
    std::vector<long long> rptr(n + 1, 0);
    for (int i = 0; i < n; i++)
        for (int k = 0; k < cnt[i]; k++) rptr[(lidx[sell_at(sptr[i >> 5], k, i & 31)] & kLinkMask) + 1]++;
    for (int j = 0; j < n; j++) rptr[j + 1] += rptr[j];
    const long long ne = rptr[n];
    std::vector<int> rslot(ne), rnode(ne);
    std::vector<unsigned char> rcode(ne);
    std::vector<long long> fill(rptr.begin(), rptr.end() - 1);
    for (int i = 0; i < n; i++)
        for (int k = 0; k < cnt[i]; k++) {
            const long long o = sell_at(sptr[i >> 5], k, i & 31);
            const int p = lidx[o] & kLinkMask, code = (unsigned)lidx[o] >> 30;
            const long long e = fill[p]++;
            rslot[e] = (int)o;
            rnode[e] = i;
            rcode[e] = (unsigned char)(code | (k < cs[i] ? 4 : 0));
        }
    if (dalloc(H, &H->rptr, n + 1) || dalloc(H, &H->rslot, ne ? ne : 1) || dalloc(H, &H->rnode, ne ? ne : 1) ||
        dalloc(H, &H->rcode, ne ? ne : 1))
        return SUNSET_ERR_NOMEM;
    SUNSET_CUDA(H, cudaMemcpy(H->rptr, rptr.data(), (n + 1) * sizeof(long long), cudaMemcpyHostToDevice));
    SUNSET_CUDA(H, cudaMemcpy(H->rslot, rslot.data(), ne * sizeof(int), cudaMemcpyHostToDevice));
    SUNSET_CUDA(H, cudaMemcpy(H->rnode, rnode.data(), ne * sizeof(int), cudaMemcpyHostToDevice));
    SUNSET_CUDA(H, cudaMemcpy(H->rcode, rcode.data(), ne * sizeof(unsigned char), cudaMemcpyHostToDevice));
    return 0;
}

static AdjArgs adj_args(Handle *H) {
    AdjArgs B{};
    B.npfb = H->npfb;
    B.rptr = H->rptr; B.rslot = H->rslot; B.rnode = H->rnode; B.rcode = H->rcode;
    B.wx = H->wx; B.wy = H->wy; B.wl = H->wl; B.wh = H->wh;
    B.gsx = H->gsx; B.gsy = H->gsy; B.lsum = H->lsum; B.hsum = H->hsum; B.vol = H->vol;
    for (int k = 0; k < kAdjG; k++) B.gb[k] = H->adj_gb[k];
    for (int k = 0; k < kAdjS; k++) B.sb[k] = H->adj_sb[k];
    for (int f = 0; f < 7; f++) B.sbar[f] = H->adj_sbar[f];
    B.tpart = H->adj_tpart;
    return B;
}

int adjoint_apply_D(Handle *H, int which, const double *gbar, double *out) {
    if (int rc = adjoint_build_reverse(H)) return rc;
    AdjArgs B = adj_args(H);
    k_adj_apply_D<<<(H->npfb + 127) / 128, 128, 0, H->stream>>>(B, which, gbar, out);
    SUNSET_CUDA(H, cudaGetLastError());
    return 0;
}

static int alloc_fields(Handle *H, Fields &F) {
    const int n = H->npfb;
    if (dalloc(H, &F.ro, n) || dalloc(H, &F.rou, n) || dalloc(H, &F.rov, n) || dalloc(H, &F.u, n) || dalloc(H, &F.v, n))
        return SUNSET_ERR_NOMEM;
    for (int k = 0; k < 4; k++)
        if (dalloc(H, &F.q[k], n) || dalloc(H, &F.c[k], n)) return SUNSET_ERR_NOMEM;
    return 0;
}

int adjoint_run(Handle *H, double dt, int nsteps, int ckpt, double *J, double *dtheta, double *dU0) {
    if (H->cfg.form != SUNSET_FORM_LC)
        return set_err(H, SUNSET_ERR_SCOPE, "the adjoint is built for the log-conformation form");
    if (H->cfg.precision != SUNSET_FP64) return set_err(H, SUNSET_ERR_SCOPE, "the adjoint runs the FP64 step");
    if (H->nb > 0) return set_err(H, SUNSET_ERR_SCOPE, "the adjoint covers node sets without walls");
    if (H->cfg.Mdiff != 0.0) return set_err(H, SUNSET_ERR_SCOPE, "the adjoint assumes Mdiff = 0");
    if (nsteps < 1 || ckpt < 1) return set_err(H, SUNSET_ERR_ARG, "nsteps and checkpoint_every must be positive");
    const int n = H->npfb;
    cudaStream_t st = H->stream;
    if (int rc = adjoint_build_reverse(H)) return rc;
    if (int rc = upload_consts(H)) return rc;
    const int nseg = (nsteps + ckpt - 1) / ckpt;
    // storage: checkpoints (7 conservative fields), the stage inputs of one segment, scratch
    if (H->adj_ready && H->adj_ckpt != ckpt)
        return set_err(H, SUNSET_ERR_ARG, "checkpoint_every must stay the same for a handle (%d)", H->adj_ckpt);
    if (H->adj_nseg < nseg) {  // checkpoint store: grows with the number of segments
        if (H->adj_cp) dfree(H, H->adj_cp);
        H->adj_cp = nullptr;
        if (dalloc(H, &H->adj_cp, (size_t)7 * n * nseg)) return SUNSET_ERR_NOMEM;
        H->adj_nseg = nseg;
    }
    if (!H->adj_ready) {
        H->adj_ckpt = ckpt;
        H->adj_store.resize(4 * (size_t)ckpt + 2);
        for (auto &F : H->adj_store)
            if (int rc = alloc_fields(H, F)) return rc;
        for (int k = 0; k < kAdjG; k++)
            if (dalloc(H, &H->adj_gb[k], n)) return SUNSET_ERR_NOMEM;
        for (int k = 0; k < kAdjS; k++)
            if (dalloc(H, &H->adj_sb[k], n)) return SUNSET_ERR_NOMEM;
        for (int f = 0; f < 7; f++)
            if (dalloc(H, &H->adj_sbar[f], n) || dalloc(H, &H->adj_ua[f], n) || dalloc(H, &H->adj_ub[f], n))
                return SUNSET_ERR_NOMEM;
        if (dalloc(H, &H->adj_tpart, 2 * (size_t)H->ntiles + 2 * (size_t)((n + 127) / 128) + 8) ||
            dalloc(H, &H->adj_acc, 4))
            return SUNSET_ERR_NOMEM;
        H->adj_ready = true;
        SUNSET_CUDA(H, cudaFuncSetAttribute(k_adj_point_lc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kMaxStageSmem));
    }
    DevScalars sc0;
    SUNSET_CUDA(H, cudaMemcpyAsync(&sc0, H->dsc, sizeof(sc0), cudaMemcpyDeviceToHost, st));
    SUNSET_CUDA(H, cudaStreamSynchronize(st));
    SUNSET_CUDA(H, cudaMemcpyAsync(&H->dsc->dt, &dt, sizeof(double), cudaMemcpyHostToDevice, st));
    // ---- forward with checkpoints ----
    for (int sg = 0; sg < nseg; sg++) {
        const Fields &F = H->buf[H->cur];
        double *cp = H->adj_cp + (size_t)7 * n * sg;
        double *src[7] = {F.ro, F.rou, F.rov, F.q[0], F.q[1], F.q[2], F.q[3]};
        for (int f = 0; f < 7; f++)
            SUNSET_CUDA(H, cudaMemcpyAsync(cp + (size_t)f * n, src[f], n * sizeof(double), cudaMemcpyDeviceToDevice, st));
        const int len = std::min(ckpt, nsteps - sg * ckpt);
        if (int rc = step_run(H, dt, len, 0)) return rc;
    }
    if (int rc = reduce_ke_mass(H, J, nullptr)) return rc;
    DevScalars scN;
    SUNSET_CUDA(H, cudaMemcpyAsync(&scN, H->dsc, sizeof(scN), cudaMemcpyDeviceToHost, st));
    SUNSET_CUDA(H, cudaStreamSynchronize(st));
    if (scN.err) return set_err(H, SUNSET_ERR_NONFINITE, "non-finite error norm in the forward run");
    // ---- reverse ----
    const int TB = 128, nb = (n + TB - 1) / TB;
    AdjArgs B = adj_args(H);
    double **ua = H->adj_ua, **ubb = H->adj_ub;
    for (int f = 0; f < 7; f++) B.ub_out[f] = ua[f];
    k_adj_objective<<<nb, TB, 0, st>>>(n, H->buf[H->cur], H->vol, B);
    SUNSET_CUDA(H, cudaMemsetAsync(H->adj_acc, 0, 4 * sizeof(double), st));
    const double alpha[4] = {SUNSET_RK_A21, SUNSET_RK_A32, SUNSET_RK_A43, SUNSET_RK_B4};
    const double beta[4] = {SUNSET_RK_B1, SUNSET_RK_B2, SUNSET_RK_B3, 0.0};
    const size_t smem = halo_doubles(ngather(SUNSET_FORM_LC, false), H->halo_max) * sizeof(double) +
                        LinkRing<false, 3, ring_depth(false)>::bytes();
    double *part2 = H->adj_tpart + 2 * (size_t)H->ntiles;
    for (int sg = nseg - 1; sg >= 0; sg--) {
        const int n0 = sg * ckpt, len = std::min(ckpt, nsteps - n0);
        // recompute the segment, keeping the stage inputs
        {
            Fields &F0 = H->adj_store[0];
            const double *cp = H->adj_cp + (size_t)7 * n * sg;
            k_set_conservative<<<nb, TB, 0, st>>>(n, SUNSET_FORM_LC, cp, cp + n, cp + 2 * (size_t)n, cp + 3 * (size_t)n,
                                                  cp + 4 * (size_t)n, cp + 5 * (size_t)n, cp + 6 * (size_t)n, F0);
            const int it = sc0.itime + n0;
            SUNSET_CUDA(H, cudaMemcpyAsync(&H->dsc->itime, &it, sizeof(int), cudaMemcpyHostToDevice, st));
            Fields &T = H->adj_store[4 * (size_t)ckpt], &X = H->adj_store[4 * (size_t)ckpt + 1];
            for (int k = 0; k < len; k++) {
                for (int s = 0; s < 4; s++) {
                    StageArgs A = make_args_io(H, H->adj_store[4 * k + s], s < 3 ? H->adj_store[4 * k + s + 1] : T, s);
                    if (int rc = launch_stage_any(H, A, false)) return rc;
                }
                Fields &next = k + 1 < len ? H->adj_store[4 * (k + 1)] : X;
                StageArgs Fa = make_args_io(H, T, next, 5);
                if (int rc = launch_filter<SUNSET_FORM_LC>(H, Fa, false)) return rc;
                k_finalize<SUNSET_FORM_LC><<<nb, TB, 0, st>>>(Fa, 1);
            }
        }
        // reverse sweep over the segment
        for (int k = len - 1; k >= 0; k--) {
            // filter and mass correction: ua (adjoint of U_{k+1}) -> ubb
            for (int f = 0; f < 7; f++) { B.ub_in[f] = ua[f]; B.ub_out[f] = ubb[f]; }
            if (H->cfg.mcorr) {
                k_adj_sum<<<nb, TB, 0, st>>>(n, ua[0], part2);
                k_adj_fold<<<1, 128, 0, st>>>(part2, nb, 1, H->adj_acc + 2, 0);
            }
            B.mcorr = H->cfg.mcorr;
            B.mc_sum = H->adj_acc + 2;
            B.mc_tv = &H->dsc->tv;
            k_adj_filter_lc<<<nb, TB, 0, st>>>(B);
            std::swap(ua, ubb);
            for (int f = 0; f < 7; f++) SUNSET_CUDA(H, cudaMemsetAsync(B.sbar[f], 0, n * sizeof(double), st));
            for (int s = 3; s >= 0; s--) {
                StageArgs A = make_args_io(H, H->adj_store[4 * k + s], H->adj_store[4 * k + s], s);
                for (int f = 0; f < 7; f++) { B.ub_in[f] = ua[f]; B.ub_out[f] = ubb[f]; }
                B.dt = dt;
                B.alpha = alpha[s];
                B.beta = beta[s];
                B.first = (s == 0) && (sc0.itime + n0 + k == 1);
                B.add_sbar = s == 0;
                k_adj_point_lc<<<H->ntiles, kTile, smem, st>>>(A, B);
                k_adj_fold<<<1, 128, 0, st>>>(H->adj_tpart, H->ntiles, 2, H->adj_acc, 1);
                k_adj_transpose_lc<<<nb, TB, 0, st>>>(A, B);
                std::swap(ua, ubb);
            }
        }
    }
    SUNSET_CUDA(H, cudaGetLastError());
    double acc[2];
    SUNSET_CUDA(H, cudaMemcpyAsync(acc, H->adj_acc, 2 * sizeof(double), cudaMemcpyDeviceToHost, st));
    for (int f = 0; f < 7; f++)
        SUNSET_CUDA(H, cudaMemcpyAsync(dU0 + (size_t)f * n, ua[f], n * sizeof(double), cudaMemcpyDeviceToDevice, st));
    // the handle keeps the final state and its time
    SUNSET_CUDA(H, cudaMemcpyAsync(H->dsc, &scN, sizeof(scN), cudaMemcpyHostToDevice, st));
    SUNSET_CUDA(H, cudaStreamSynchronize(st));
    dtheta[0] = acc[0];
    dtheta[1] = acc[1];
    return 0;
}

}  // namespace sunset
