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
#include <algorithm>
#include <cstring>
#include <thread>
#include <type_traits>

#include "adjoint.cuh"
#include "internal.cuh"
#include "physics.cuh"

namespace sunset {

namespace {


struct StageArgs {
    StepConsts K;  // the run's constants (load_data.F90:131-148), a kernel parameter of every launch
    const long long *slice_ptr;
    const int *slice_ws, *slice_w;
    const int *lidx;
    const uint16_t *lloc;
    const int *halo_ptr, *halo;
    int hmax;
    const double *wx, *wy, *wl, *wh;
    // mixed precision: the stage's packed links and their per-node scales (stream.cu), the
    // filter's FP32 weights
    const unsigned *pk;
    const float *scx, *scy, *scl;
    const unsigned *wf;
    const double *gsx, *gsy, *lsum, *hsum, *vol, *py_node;
    const int *ntype;            // node types (walls: 0)
    const double *rnx, *rny;     // wall normals into the fluid
    // polymer diffusion on walls: reference-order local links, small-link counts, boundary
    // index and FD rows, tangential second-derivative weights and their sums, spacings
    const uint16_t *lloc_ref;
    const int *cnt_small, *bidx, *brow;
    const double *wbt, *wbt_sum, *sp;
    int nplink;
    Fields in, out;
    double *reg[7], *eacc[7], *rhs[7];
    float *dreg[7], *eacc32[7];  // mixed precision
    DevScalars *sc;
    double *partials;
    double *alpha;  // per-node step error (stage 3), or null
    double *uin;    // nb: u_inflow_local of the boundary nodes (inflow/outflow sets), or null
    double *gsave;  // log-conformation FP64 stages of the adjoint's recording: the 18 stencil
                    // sums of each node (adjoint.cuh order, arrays of npfb), else null
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
// FENE-P (FP) appends the FENE-P function f (DI, LC) or psizz (CHL), and with polymer
// diffusion czz (DI, CHL).
__host__ __device__ constexpr int ngather(int form, bool md, bool fp = false) {
    return form == SUNSET_FORM_DI    ? 6 + (fp ? 1 : 0) + (fp && md ? 1 : 0)
           : form == SUNSET_FORM_LC  ? 9 + (fp ? 1 : 0)
           : form == SUNSET_FORM_CHL ? (md ? 9 : 6) + (fp ? 1 : 0) + (fp && md ? 1 : 0)
                                     : 3;
}
// Positions of the FENE-P fields: f (DI, LC) or psizz (CHL), then czz (polymer diffusion).
__host__ __device__ constexpr int fp_slot(int form, bool md) {
    return form == SUNSET_FORM_DI ? 6 : form == SUNSET_FORM_LC ? 9 : (md ? 9 : 6);
}

template <int FORM, bool MD, bool FP = false>
__device__ __forceinline__ const double *gather_src(const Fields &F, int f) {
    if (f == 0) return F.ro;
    if (f == 1) return F.u;
    if (f == 2) return F.v;
    if (FP && f >= fp_slot(FORM, MD)) {
        if (f == fp_slot(FORM, MD)) return FORM == SUNSET_FORM_CHL ? F.q[3] : F.f;
        return F.c[3];
    }
    if (FORM == SUNSET_FORM_DI || FORM == SUNSET_FORM_LC) {
        if (f <= 5) return F.c[f - 3];
        return F.q[f - 6];
    }
    if (f <= 5) return F.q[f - 3];
    return F.c[f - 6];
}


// The link streams are read once a stage and exceed L2: their copies carry an L2 evict-first
// policy, so that they do not push the tiles' halo fields (read by several tiles) and the
// state out of L2.  Measured on the 1M-node order-8 set: the FP64 step 2.333 -> 2.301 ms, the
// mixed step 1.350 -> 1.285 ms; on the order-6 set 0.498 -> 0.486 and 0.334 -> 0.313 ms.
#ifndef SUNSET_LINK_EVICT_FIRST
#define SUNSET_LINK_EVICT_FIRST 1
#endif
__device__ __forceinline__ unsigned long long l2_evict_first() {
    unsigned long long p;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
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
template <int N>
__device__ __forceinline__ void cp_async_link(void *dst_shared, const void *src_global) {
    if constexpr (SUNSET_LINK_EVICT_FIRST && N == 16) {
        const unsigned d = (unsigned)__cvta_generic_to_shared(dst_shared);
        const size_t g = __cvta_generic_to_global(src_global);
        asm volatile("cp.async.cg.shared.global.L2::cache_hint [%0], [%1], 16, %2;" ::"r"(d), "l"(g),
                     "l"(l2_evict_first())
                     : "memory");
    } else {
        cp_async<N>(dst_shared, src_global);
    }
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
            for (int a = 0; a < NA; a++) cp_async_link<sizeof(W2)>(w + (s * NA + a) * kTile + threadIdx.x, src[a] + o);
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
// The filter streams one weight a link (20 bytes a thread and slot in FP64, 12 in FP32), so its
// ring runs deeper for the same shared memory.
#ifndef SUNSET_FILTER_RING_FP64
#define SUNSET_FILTER_RING_FP64 4
#endif
#ifndef SUNSET_FILTER_RING_MIXED
#define SUNSET_FILTER_RING_MIXED 8
#endif
__host__ __device__ constexpr int filter_ring_depth(bool mx) { return mx ? SUNSET_FILTER_RING_MIXED : SUNSET_FILTER_RING_FP64; }

// Doubles of the shared-memory halo, rounded up so the ring after it is 16-byte aligned.
__host__ __device__ inline size_t halo_doubles(int ng, int hmax) { return ((size_t)ng * hmax + 1) & ~(size_t)1; }

// Stencil sums of one node over its small links, sum form of derivatives.F90:36-46,
// neighbours read from the block's shared-memory halo.  In the mixed path the weights are
// the FP32-rounded ones and A.gsx.. hold the FP64 sums of those, so the FP64 arithmetic
// below evaluates the difference form sum_k w_k (phi_j - phi_i) of the rounded stencil.
template <int FORM, bool MD, bool MX, bool FP, class RING>
__device__ __forceinline__ void gather_stage(const StageArgs &A, int i, const double *sm, RING &R, Grads &g) {
    const StepConsts &cK = A.K;
    const int hm = A.hmax;
    const int npair = R.npair;
    const Fields &F = A.in;
    double s_ro_x = 0, s_ro_y = 0, s_u_x = 0, s_u_y = 0, s_v_x = 0, s_v_y = 0, s_lu = 0, s_lv = 0;
    double s_cxx_x = 0, s_cxx_y = 0, s_cxy_x = 0, s_cxy_y = 0, s_cyy_x = 0, s_cyy_y = 0;
    double s_pxx_x = 0, s_pxx_y = 0, s_pxy_x = 0, s_pxy_y = 0, s_pyy_x = 0, s_pyy_y = 0;
    double s_lxx = 0, s_lxy = 0, s_lyy = 0;
    double s_f_x = 0, s_f_y = 0, s_lzz = 0;  // FENE-P: f or psizz gradient, czz Laplacian
    constexpr int kFp = fp_slot(FORM, MD);
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
        if constexpr (FP && FORM != SUNSET_FORM_NEWT) {  // scalar or zz fields: no reflection sign
            const double fj = sm[kFp * hm + j];
            mac(s_f_x, fj, wxk);
            mac(s_f_y, fj, wyk);
            if (MD && (FORM == SUNSET_FORM_DI || FORM == SUNSET_FORM_CHL)) mac(s_lzz, sm[(kFp + 1) * hm + j], wlk);
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
    g.f_x = g.f_y = g.pzz_x = g.pzz_y = 0.0;
    if constexpr (FP && FORM != SUNSET_FORM_NEWT) {
        const double fi = FORM == SUNSET_FORM_CHL ? F.q[3][i] : F.f[i];
        const double gfx = s_f_x - fi * gx, gfy = s_f_y - fi * gy;
        if (FORM == SUNSET_FORM_CHL) { g.pzz_x = gfx; g.pzz_y = gfy; }
        else { g.f_x = gfx; g.f_y = gfy; }
        if (MD && (FORM == SUNSET_FORM_DI || FORM == SUNSET_FORM_CHL)) g.lapczz = s_lzz - F.c[3][i] * ls;
    }
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

// ---------------------------------------------------------------------------------------
// Mixed-precision stage gather.
//
// The tile's halo is staged as FP32 offsets from a per-tile FP64 reference of each field
// (the field's value at the tile's first halo node; zero, when the node set has mirrors, for
// the fields a mirror link reflects), two fields to an 8-byte word and the words of one halo
// node together (an odd number of words per node, so the bank-aware link order of stream.cu
// keeps a half-warp's 8-byte loads on distinct bank pairs), so one link's neighbour values
// take ceil(NG/2) 8-byte shared loads at one address plus constant offsets.  Each thread differences them with
// its own node's offsets and sums w_k (phi_j - phi_i) in FP32: the offsets keep the bits a
// difference of two nearby values needs, since phi_j - ref spans a tile, not |phi|.  The
// sums are scaled to FP64 once per node (the packed weights are integers in units of the
// node's scale, stream.cu).
//
// The link stream reaches shared memory by bulk copies (the TMA engine, cp.async.bulk, from
// this GPU's memory only, no cluster multicast): lane 0 of each warp keeps kMxDepth chunks of
// kMxChunk link pairs of its slice in flight, each completing on an mbarrier of the warp, so
// the link loads stay off the LSU pipe that the halo gathers keep busy.  Every wait on an
// mbarrier is bounded: when one gives up, the kernel sets the device error word to 2, waits
// (bounded again) for the warp's copies in flight and finishes with the sums it has; the host
// reports the error.
// ---------------------------------------------------------------------------------------
#ifndef SUNSET_MX_CHUNK
#define SUNSET_MX_CHUNK 2
#endif
#ifndef SUNSET_MX_DEPTH
#define SUNSET_MX_DEPTH 2
#endif
constexpr int kMxChunk = SUNSET_MX_CHUNK;  // link pairs per bulk copy
constexpr int kMxDepth = SUNSET_MX_DEPTH;  // bulk copies in flight per warp
constexpr int kMxWaitLimit = 1 << 20;      // try_wait rounds before a wait gives up

// Shared memory of the mixed stage kernel, in order: the warps' link rings (kMxDepth stages
// of three words x kMxChunk pairs x 32 lanes, 8 bytes a lane and pair), their mbarriers, the
// NG field references (FP64) and the halo as ceil(NG/2) arrays of float2 of hmax entries.
__host__ __device__ constexpr size_t mx_ring_bytes() { return (size_t)kTileSlices * kMxDepth * 3 * kMxChunk * 32 * 8; }
__host__ __device__ constexpr size_t mx_bar_bytes() { return (size_t)kTileSlices * kMxDepth * 8; }
// 8-byte words a halo node takes: ceil(NG/2), made odd
__host__ __device__ constexpr int mx_words(int ng) { return ((ng + 1) / 2) | 1; }
__host__ __device__ inline size_t mx_smem_bytes(int ng, int hmax) {
    return mx_ring_bytes() + mx_bar_bytes() + (size_t)ng * 8 + (size_t)mx_words(ng) * hmax * 8;
}
__device__ __forceinline__ double *mx_refs(double *smem) {
    return reinterpret_cast<double *>(reinterpret_cast<char *>(smem) + mx_ring_bytes() + mx_bar_bytes());
}
__device__ __forceinline__ float2 *mx_halo(double *smem, int ng) { return reinterpret_cast<float2 *>(mx_refs(smem) + ng); }

__device__ __forceinline__ unsigned smem_addr(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(unsigned bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
// makes the barriers' initialisation visible to the bulk-copy engine
__device__ __forceinline__ void mbar_init_fence() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(unsigned bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ bool mbar_wait_bounded(unsigned bar, unsigned parity) {
    for (int it = 0; it < kMxWaitLimit; it++)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}
// global -> this CTA's shared memory by the bulk-copy engine, completion counted on `bar`
__device__ __forceinline__ void bulk_load(unsigned dst, const void *src, unsigned bytes, unsigned bar) {
    if constexpr (SUNSET_LINK_EVICT_FIRST) {
        asm volatile("cp.async.bulk.shared::cta.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;"
                     ::"r"(dst), "l"(src), "r"(bytes), "r"(bar), "l"(l2_evict_first())
                     : "memory");
    } else {
        asm volatile("cp.async.bulk.shared::cta.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                     "l"(src), "r"(bytes), "r"(bar)
                     : "memory");
    }
}
// orders this thread's generic-proxy shared accesses before its later bulk copies
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// The xy component among the gathered fields (a mirror link flips its sign with codes 1, 2).
__host__ __device__ constexpr bool is_xy_slot(int form, bool md, int f) {
    return f == 4 || (form == SUNSET_FORM_LC && f == 7) || (form == SUNSET_FORM_CHL && md && f == 7);
}

// One warp's ring of packed link words (its slice's small links, pair by pair).
struct MxRing {
    uint2 *ring;      // kMxDepth stages of [kMxChunk pairs][32 lanes][3 uint2: x0 y0, l0 x1, y1 l1]
    unsigned bar0;    // shared address of the warp's first mbarrier
    long long base;   // SELL slot of the slice's pair 0
    int npair, nchunk;

    // lane 0: one bulk copy of chunk c (its pair rows are 768 contiguous bytes each)
    __device__ __forceinline__ void issue(const StageArgs &A, int c) const {
        const int s = c % kMxDepth;
        const int np = min(kMxChunk, npair - c * kMxChunk);
        const unsigned bytes = (unsigned)np * 768u, bar = bar0 + 8u * s;
        mbar_expect_tx(bar, bytes);
        bulk_load(smem_addr(ring + s * 3 * kMxChunk * 32), A.pk + 3 * (base + (long long)c * kMxChunk * 64), bytes, bar);
    }
    __device__ __forceinline__ bool wait(int c) const {
        return mbar_wait_bounded(bar0 + 8u * (c % kMxDepth), (unsigned)(c / kMxDepth) & 1u);
    }
};

// The halo as FP32 offsets and this thread's own offsets oi (all threads of the block take
// part; ends with a barrier).  The warp's mbarriers are initialised and its first chunks
// started before, so the link stream flows while the halo loads.
template <int FORM, bool MD, bool FP>
__device__ __forceinline__ void load_halo_mx(const StageArgs &A, int i, double *smem, MxRing &R, bool wact,
                                             float *oi) {
    const StepConsts &cK = A.K;
    constexpr int NG = ngather(FORM, MD, FP), NP = (NG + 1) / 2;
    const int lane = threadIdx.x & 31;
    if (wact && lane == 0) {
        for (int s = 0; s < kMxDepth; s++) mbar_init(R.bar0 + 8u * s, 1u);
        mbar_init_fence();
        for (int c = 0; c < kMxDepth && c < R.nchunk; c++) R.issue(A, c);
    }
    const bool mir = cK.has_mirrors;
    const int hb = A.halo_ptr[blockIdx.x], hn = A.halo_ptr[blockIdx.x + 1] - hb;
    const int n0 = __ldg(A.halo + hb);
    double rf[NG];
#pragma unroll
    for (int f = 0; f < NG; f++)
        rf[f] = (mir && (f == 1 || f == 2 || is_xy_slot(FORM, MD, f))) ? 0.0 : __ldg(gather_src<FORM, MD, FP>(A.in, f) + n0);
    if (threadIdx.x == 0) {
        double *ref = mx_refs(smem);
#pragma unroll
        for (int f = 0; f < NG; f++) ref[f] = rf[f];
    }
    float2 *hp = mx_halo(smem, NG);
    constexpr int NW = mx_words(NG);
#pragma unroll 4
    for (int h = threadIdx.x; h < hn; h += blockDim.x) {
        const int node = __ldg(A.halo + hb + h);
#pragma unroll
        for (int p = 0; p < NP; p++) {
            const float a = (float)(__ldg(gather_src<FORM, MD, FP>(A.in, 2 * p) + node) - rf[2 * p]);
            const float b = 2 * p + 1 < NG ? (float)(__ldg(gather_src<FORM, MD, FP>(A.in, 2 * p + 1) + node) - rf[2 * p + 1])
                                           : 0.0f;
            hp[h * NW + p] = make_float2(a, b);
        }
    }
    const int ii = i < cK.npfb ? i : 0;
#pragma unroll
    for (int f = 0; f < NG; f++) oi[f] = (float)(__ldg(gather_src<FORM, MD, FP>(A.in, f) + ii) - rf[f]);
    __syncthreads();
}

// Stencil sums of node i over its small links in difference form, FP32 (see above).  MIR:
// the node set has mirror links (a reflected neighbour value is -phi_parent, and the
// reflected fields have reference 0); without mirrors the signs are compiled out.
//
// A packed link word w (stream.cu) is the 32-bit integer 64 q + b, q the weight in units of
// the node's scale and b six index bits: w & ~63 converted to FP32 is 64 q, w & 63 is b.
template <int FORM, bool MD, bool FP, bool MIR>
__device__ __forceinline__ void gather_stage_mx(const StageArgs &A, int i, const double *smem, const MxRing &R,
                                                bool wact, const float *oi, Grads &g) {
    const StepConsts &cK = A.K;
    constexpr int NG = ngather(FORM, MD, FP), NP = (NG + 1) / 2, NW = mx_words(NG);
    constexpr int kFp = fp_slot(FORM, MD);
    const int lane = threadIdx.x & 31;
    const float2 *hp = mx_halo(const_cast<double *>(smem), NG);
    const bool full = (FORM == SUNSET_FORM_DI) && cK.di_full;
    // the x and y sums of every gathered field, two fields to a float2 (the halo's pairs), so
    // the differences and both sums run as paired FP32 instructions (FADD2, FFMA2); the
    // Laplacians the right-hand side reads as scalars
    float2 ax[NP], ay[NP], noi[NP];
#pragma unroll
    for (int p = 0; p < NP; p++) {
        ax[p] = make_float2(0.0f, 0.0f);
        ay[p] = make_float2(0.0f, 0.0f);
        noi[p] = make_float2(-oi[2 * p], 2 * p + 1 < NG ? -oi[2 * p + 1] : 0.0f);
    }
    float s_lu = 0, s_lv = 0, s_lxx = 0, s_lxy = 0, s_lyy = 0, s_lzz = 0;
    auto comp = [](const float2 *a, int f) { return (f & 1) ? a[f >> 1].y : a[f >> 1].x; };
    auto link = [&](unsigned x, unsigned y, unsigned l) {
        const unsigned loc = (x & 63u) | ((y & 63u) << 6) | ((l & 15u) << 12);
        const float wx = (float)(int)(x & ~63u), wy = (float)(int)(y & ~63u), wl = (float)(int)(l & ~63u);
        const float2 *v = hp + (loc & kLocMask) * NW;
        float2 dp[NP];
        if constexpr (MIR) {  // reflected fields have reference 0: the mirror value is -phi_parent
            const unsigned code = loc >> 14;
            const float su = (code == 1u || code == 3u) ? -1.0f : 1.0f, sv = (code == 2u || code == 3u) ? -1.0f : 1.0f;
            const float sxy = (code == 1u || code == 2u) ? -1.0f : 1.0f;
#pragma unroll
            for (int p = 0; p < NP; p++) {
                const float2 q = v[p];
                const int f0 = 2 * p, f1 = 2 * p + 1;
                const float s0 = f0 == 1 ? su : f0 == 2 ? sv : is_xy_slot(FORM, MD, f0) ? sxy : 1.0f;
                const float s1 = f1 == 1 ? su : f1 == 2 ? sv : is_xy_slot(FORM, MD, f1) ? sxy : 1.0f;
                dp[p] = __ffma2_rn(make_float2(s0, s1), q, noi[p]);
            }
        } else {
#pragma unroll
            for (int p = 0; p < NP; p++) dp[p] = __fadd2_rn(v[p], noi[p]);
        }
        const float2 wx2 = make_float2(wx, wx), wy2 = make_float2(wy, wy);
#pragma unroll
        for (int p = 0; p < NP; p++) {
            ax[p] = __ffma2_rn(wx2, dp[p], ax[p]);
            ay[p] = __ffma2_rn(wy2, dp[p], ay[p]);
        }
        s_lu = __fmaf_rn(wl, comp(dp, 1), s_lu);
        s_lv = __fmaf_rn(wl, comp(dp, 2), s_lv);
        if (MD && (FORM == SUNSET_FORM_DI || FORM == SUNSET_FORM_CHL)) {  // c in slots 3-5 (DI) or 6-8 (CHL)
            constexpr int q = FORM == SUNSET_FORM_DI ? 3 : 6;
            s_lxx = __fmaf_rn(wl, comp(dp, q), s_lxx);
            s_lxy = __fmaf_rn(wl, comp(dp, q + 1), s_lxy);
            s_lyy = __fmaf_rn(wl, comp(dp, q + 2), s_lyy);
            if (FP) s_lzz = __fmaf_rn(wl, comp(dp, kFp + 1), s_lzz);
        }
    };
    if (wact) {
        for (int c = 0; c < R.nchunk; c++) {
            if (!R.wait(c)) {
                if (lane == 0) atomicExch(&A.sc->err, 2);
                for (int c2 = c; c2 < c + kMxDepth && c2 < R.nchunk; c2++) R.wait(c2);
                break;
            }
            const int np = min(kMxChunk, R.npair - c * kMxChunk);
            const uint2 *rs = R.ring + (c % kMxDepth) * 3 * kMxChunk * 32 + 3 * lane;
#pragma unroll
            for (int p = 0; p < kMxChunk; p++) {
                if (p < np) {
                    const uint2 a = rs[p * 96], b = rs[p * 96 + 1], e = rs[p * 96 + 2];
                    link(a.x, a.y, b.x);
                    link(b.y, e.x, e.y);
                }
            }
            __syncwarp();
            if (lane == 0 && c + kMxDepth < R.nchunk) {
                fence_proxy_async();
                R.issue(A, c + kMxDepth);
            }
        }
    }
    if (i >= cK.npfb) return;
    const double cx = (double)A.scx[i], cy = (double)A.scy[i], cl = (double)A.scl[i];
    auto X = [&](int f) { return (double)comp(ax, f) * cx; };
    auto Y = [&](int f) { return (double)comp(ay, f) * cy; };
    g.ro_x = X(0);
    g.ro_y = Y(0);
    g.u_x = X(1);
    g.u_y = Y(1);
    g.lapu = (double)s_lu * cl;
    g.v_x = X(2);
    g.v_y = Y(2);
    g.lapv = (double)s_lv * cl;
    g.cxx_x = g.cxx_y = g.cxy_x = g.cxy_y = g.cyy_x = g.cyy_y = 0.0;
    g.pxx_x = g.pxx_y = g.pxy_x = g.pxy_y = g.pyy_x = g.pyy_y = 0.0;
    if (FORM == SUNSET_FORM_DI || FORM == SUNSET_FORM_LC) {  // c in slots 3, 4, 5
        g.cxx_x = X(3);
        g.cxx_y = full ? Y(3) : 0.0;
        g.cxy_x = X(4);
        g.cxy_y = Y(4);
        g.cyy_x = full ? X(5) : 0.0;
        g.cyy_y = Y(5);
    }
    if (FORM == SUNSET_FORM_LC || FORM == SUNSET_FORM_CHL) {  // psi in slots 6-8 (LC) or 3-5 (CHL)
        constexpr int q = FORM == SUNSET_FORM_LC ? 6 : 3;
        g.pxx_x = X(q);
        g.pxx_y = Y(q);
        g.pxy_x = X(q + 1);
        g.pxy_y = Y(q + 1);
        g.pyy_x = X(q + 2);
        g.pyy_y = Y(q + 2);
    }
    g.lapcxx = (double)s_lxx * cl;
    g.lapcxy = (double)s_lxy * cl;
    g.lapcyy = (double)s_lyy * cl;
    g.lapczz = (double)s_lzz * cl;
    g.f_x = g.f_y = g.pzz_x = g.pzz_y = 0.0;
    if constexpr (FP && FORM != SUNSET_FORM_NEWT) {
        if (FORM == SUNSET_FORM_CHL) { g.pzz_x = X(kFp); g.pzz_y = Y(kFp); }
        else { g.f_x = X(kFp); g.f_y = Y(kFp); }
    }
}

// Polymer diffusion on a wall node: the transverse Laplacian of c over the node's small links
// with the tangential second-derivative weights (calc_laplacian_transverse_only_on_bound,
// derivatives.F90:306-358), plus the one-sided normal second derivative from its four FD rows
// (rhs_di.F90:556-568; rhs.F90 likewise, there for c_zz too).  Links in the reference's
// order, neighbours from the tile's shared-memory halo.
template <int FORM, bool MD, bool FP, class HV>
__device__ __forceinline__ void wall_conformation_laplacian(const StageArgs &A, int i, HV hv, Grads &g) {
    const StepConsts &cK = A.K;
    const int jj = A.bidx[i];
    const long long base = A.slice_ptr[i >> 5];
    const int ln = i & 31, cs = A.cnt_small[i];
    constexpr int c0 = FORM == SUNSET_FORM_DI ? 3 : 6;  // halo slots of cxx, cxy, cyy
    constexpr bool zz = FORM == SUNSET_FORM_CHL && FP;   // c_zz enters the Cholesky FENE-P source
    constexpr int cz = fp_slot(FORM, MD) + 1;
    const double *w = A.wbt + (size_t)jj * A.nplink;
    double l0 = 0.0, l1 = 0.0, l2 = 0.0, l3 = 0.0;
    for (int k = 0; k < cs; k++) {
        const unsigned lk = A.lloc_ref[sell_at(base, k, ln)];
        const int h = lk & kLocMask, code = lk >> 14;
        double cxy = hv(c0 + 1, h);
        if (code == 1 || code == 2) cxy = -cxy;
        const double wk = w[k];
        l0 = l0 + hv(c0, h) * wk;
        l1 = l1 + cxy * wk;
        l2 = l2 + hv(c0 + 2, h) * wk;
        if (zz) l3 = l3 + hv(cz, h) * wk;
    }
    const Fields &F = A.in;
    const double ws = A.wbt_sum[jj], L = cK.L_char;
    const double den = (((72.0 * A.sp[i]) * A.sp[i]) * L) * L;
    const int *r = A.brow + 4 * jj;
    auto fd = [&](const double *q) {
        return (((((-415.0 * q[i]) + 576.0 * q[r[0]]) - 216.0 * q[r[1]]) + 64.0 * q[r[2]]) - 9.0 * q[r[3]]) / den;
    };
    g.lapcxx = (l0 - F.c[0][i] * ws) + fd(F.c[0]);
    g.lapcxy = (l1 - F.c[1][i] * ws) + fd(F.c[1]);
    g.lapcyy = (l2 - F.c[2][i] * ws) + fd(F.c[2]);
    if (zz) g.lapczz = (l3 - F.c[3][i] * ws) + fd(F.c[3]);
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

// Resident blocks per SM the stage kernel is compiled for.  FP64: up to 85 registers a
// thread; the tile halo plus the link ring take 55-70 KB of shared memory on the order-6 and
// order-8 sets, so a fourth block would not fit anyway.  Mixed: the FP32 halo and the
// bulk-copy rings take 40-50 KB, and the FP32 sums fewer registers.
#ifndef SUNSET_STAGE_BLOCKS
#define SUNSET_STAGE_BLOCKS 3
#endif
#ifndef SUNSET_STAGE_BLOCKS_MX
#define SUNSET_STAGE_BLOCKS_MX 4
#endif
__host__ __device__ constexpr int stage_min_blocks(bool mx) { return mx ? SUNSET_STAGE_BLOCKS_MX : SUNSET_STAGE_BLOCKS; }

// One RK stage (stage = 0,1,2: intermediate; 3: final; 4: right-hand side only).  One
// block per tile of kTile nodes; the tile's halo is staged in shared memory first.
//
// MX (mixed precision): packed fixed-point weights, FP32 halo offsets and FP32 sums in
// difference form (gather_stage_mx); the register S is kept as the FP32 increment
// D = S - U over the stage's FP64 state U (so S = U + D loses only FP32 rounding of an
// O(dt rhs) quantity) and the error accumulator E as FP32.
// BND: the node set has boundary nodes (walls, inflows, outflows); without them the
// closures are compiled out, which keeps them from costing the periodic sets registers.
template <int FORM, bool MD, bool MX, bool FP, bool BND>
__global__ void __launch_bounds__(kTile, stage_min_blocks(MX)) k_stage(StageArgs A) {
    const StepConsts &cK = A.K;
    extern __shared__ __align__(16) double smem[];
    constexpr int NG = ngather(FORM, MD, FP);
    const int i = blockIdx.x * kTile + threadIdx.x;
    bool active = (i >> 5) < cK.nslices;
    const int stage = A.stage;
    if (stage == 0 && i == 0) {
        A.sc->cfl_bits = 0x7ff0000000000000ull;
        A.sc->par_bits = 0x7ff0000000000000ull;
    }
    Grads g;
    if constexpr (MX) {
        const int warp = threadIdx.x >> 5, sl = blockIdx.x * kTileSlices + warp;
        MxRing R;
        R.ring = reinterpret_cast<uint2 *>(smem) + (size_t)warp * kMxDepth * 3 * kMxChunk * 32;
        R.bar0 = smem_addr(reinterpret_cast<char *>(smem) + mx_ring_bytes() + (size_t)warp * kMxDepth * 8);
        R.base = active ? A.slice_ptr[sl] : 0;
        R.npair = active ? A.slice_ws[sl] >> 1 : 0;
        R.nchunk = (R.npair + kMxChunk - 1) / kMxChunk;
        float oi[NG];
        load_halo_mx<FORM, MD, FP>(A, i, smem, R, active, oi);
        if (cK.has_mirrors) gather_stage_mx<FORM, MD, FP, true>(A, i, smem, R, active, oi, g);
        else gather_stage_mx<FORM, MD, FP, false>(A, i, smem, R, active, oi, g);
    } else {
        LinkRing<false, 3, ring_depth(false)> R;
        R.src[0] = reinterpret_cast<const double2 *>(A.wx);
        R.src[1] = reinterpret_cast<const double2 *>(A.wy);
        R.src[2] = reinterpret_cast<const double2 *>(A.wl);
        R.init(smem + halo_doubles(NG, A.hmax), reinterpret_cast<const unsigned *>(A.lloc),
               active ? (A.slice_ptr[i >> 5] >> 1) + (i & 31) : 0, active ? A.slice_ws[i >> 5] >> 1 : 0);
        R.prologue();  // the first link pairs stream in while the halo is staged
        load_halo<NG>(A, smem, [&](int f) { return gather_src<FORM, MD, FP>(A.in, f); });
        if (active) gather_stage<FORM, MD, false, FP>(A, i, smem, R, g);
    }
    // a node's own value of gathered field f in the tile's halo slot h (wall Laplacian of c)
    auto hv = [&](int f, int h) -> double {
        if constexpr (MX) {
            const float2 v = mx_halo(smem, NG)[h * mx_words(NG) + (f >> 1)];
            return mx_refs(smem)[f] + (double)((f & 1) ? v.y : v.x);
        } else {
            return smem[f * A.hmax + h];
        }
    };
    active = active && i < cK.npfb;
    unsigned long long emax_bits = 0;
    if constexpr (FORM == SUNSET_FORM_LC && !MX) {
        if (active && A.gsave) {
            const double gv[kAdjG] = {g.ro_x, g.ro_y, g.u_x, g.u_y, g.lapu, g.v_x, g.v_y, g.lapv, g.cxx_x, g.cxy_x,
                                      g.cxy_y, g.cyy_y, g.pxx_x, g.pxx_y, g.pxy_x, g.pxy_y, g.pyy_x, g.pyy_y};
#pragma unroll
            for (int k = 0; k < kAdjG; k++) A.gsave[(size_t)k * cK.npfb + i] = gv[k];
        }
    }
    if (active) {
        const Fields &F = A.in;
        NodeState n;
        n.ro = F.ro[i]; n.u = F.u[i]; n.v = F.v[i]; n.y = A.py_node[i];
        n.cxx = F.c[0][i]; n.cxy = F.c[1][i]; n.cyy = F.c[2][i]; n.czz = F.c[3][i];
        n.pxx = F.q[0][i]; n.pxy = F.q[1][i]; n.pyy = F.q[2][i]; n.pzz = F.q[3][i];
        n.f = 0.0;
        if constexpr (FP) n.f = FORM == SUNSET_FORM_CHL ? fenep_f(cK.fenep_l2, n.cxx, n.cyy, n.czz) : F.f[i];
        n.df = A.sc->df;
        Rhs r;
        const int ty = BND ? A.ntype[i] : 999;
        const bool wall = ty == 0, inout = ty == 1 || ty == 2;
        const int jb = inout ? A.bidx[i] : 0;
        double uin = inout ? A.uin[jb] : 0.0;
        if (inout) {  // inflow/outflow closure in the x-y frame
            if constexpr (MD && FORM == SUNSET_FORM_CHL)  // rhs.F90:624-636: the same one-sided flux closure
                wall_conformation_laplacian<FORM, MD, FP>(A, i, hv, g);
            rhs_flow_inout(cK, n, g, ty, uin, r);
        } else if (wall) {  // wall closure; then the conformation with the rotated velocity gradient
            if constexpr (MD && (FORM == SUNSET_FORM_DI || FORM == SUNSET_FORM_CHL))
                wall_conformation_laplacian<FORM, MD, FP>(A, i, hv, g);
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
        if (FORM == SUNSET_FORM_DI) {
            rhs_c_di(cK, n, g, r, wall);
            if (inout) r.xx = r.xy = r.yy = r.zz = 0.0;  // rhs_di.F90:582-590 (left to be completed there)
        } else if (FORM == SUNSET_FORM_CHL) {
            if (ty == 1) {  // inflow: no streamwise advection of psi (rhs.F90:562-564)
                NodeState m = n;
                m.u = 0.0;
                rhs_c_chl<MX>(cK, m, g, r);
            } else {
                rhs_c_chl<MX>(cK, n, g, r);
            }
        } else if (FORM == SUNSET_FORM_LC) {
            const bool first = (A.sc->itime == 1) && (stage == 0);
            rhs_c_lc(cK, n, g, first, r, wall);
        } else { r.xx = r.xy = r.yy = r.zz = 0.0; }
        const double rr[7] = {r.ro, r.rou, r.rov, r.xx, r.xy, r.yy, r.zz};
        // evolved fields: DI 7 (czz), CHL FENE-P 7 (psizz), otherwise 6 (3 Newtonian)
        constexpr int nf = (FORM == SUNSET_FORM_DI || (FORM == SUNSET_FORM_CHL && FP)) ? 7 : (FORM == SUNSET_FORM_NEWT ? 3 : 6);
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
                // every register read before the first is written: the compiler cannot tell the
                // fields' arrays apart, and would otherwise wait out each load after a store
                double S[7], E[7];
#pragma unroll
                for (int f = 0; f < nf; f++) {
                    if constexpr (MX) {
                        S[f] = (stage == 0) ? U[f] : U[f] + (double)A.dreg[f][i];
                        E[f] = (stage == 0) ? 0.0 : (double)A.eacc32[f][i];
                    } else {
                        S[f] = (stage == 0) ? U[f] : A.reg[f][i];
                        E[f] = (stage == 0) ? 0.0 : A.eacc[f][i];
                    }
                }
#pragma unroll
                for (int f = 0; f < nf; f++) {
                    Un[f] = S[f] + RKa * rr[f];
                    if constexpr (MX) {
                        A.dreg[f][i] = (float)((S[f] + RKb * rr[f]) - Un[f]);
                        A.eacc32[f][i] = (float)(E[f] + RKbmbh * rr[f]);
                    } else {
                        A.reg[f][i] = S[f] + RKb * rr[f];
                        A.eacc[f][i] = E[f] + RKbmbh * rr[f];
                    }
                }
            } else {
                double en = 0.0, al = 0.0;
                // Cholesky FENE-P: the conformation errors scaled by the node's 1/sqrt(f)
                // (step.F90:442-452 scales the running maxima by each node's factor in turn;
                // here each node's own errors are scaled before the maximum, order-free)
                double conf_scale = 1.0;
                if constexpr (FORM == SUNSET_FORM_CHL && FP)
                    conf_scale = 1.0 / sqrt((cK.fenep_l2 - 3.0) / (((cK.fenep_l2 - n.cxx) - n.cyy) - n.czz));
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
                    double t = fabs(E) * norm;
                    if (f < 6) al = (t > al) ? t : al;  // alpha_out: rho, momentum, xx, xy, yy (step.F90:455-457)
                    if (f >= 3) t = t * conf_scale;
                    en = (t > en) ? t : en;
                    if (t != t) en = t;
                }
                emax_bits = dbits(en);
                if (A.alpha) A.alpha[i] = al;
            }
            // apply_time_dependent_bounds (characteristic_boundaries.F90:191-257) at the stage's
            // time time0 + c_s dt (step.F90:285, c = 0, a21, a32 + b1, 1): walls at rest; on
            // inflow nodes u_inflow_local follows its ramp, and a hard inflow prescribes u
            if (wall) { Un[1] = 0.0; Un[2] = 0.0; }
            if (ty == 1) {
                const double cs = stage == 0 ? 0.0 : stage == 1 ? SUNSET_RK_A21 : stage == 2 ? (SUNSET_RK_A32 + SUNSET_RK_B1) : 1.0;
                uin = inflow_velocity(cK, A.sc->time + dt * cs, uin);
                A.uin[jb] = uin;
                if (cK.inflow_type == 1) { Un[1] = uin * Un[0]; Un[2] = 0.0; }
            }
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
                    O.c[0][i] = cxx; O.c[1][i] = cxy; O.c[2][i] = cyy; O.c[3][i] = n.czz;  // carried
                } else if (FORM == SUNSET_FORM_CHL) {
                    double cxx, cxy, cyy, czz;
                    if constexpr (FP) chl_c_from_psi_fenep(cK.fenep_l2, Un[3], Un[4], Un[5], Un[6], &cxx, &cxy, &cyy, &czz);
                    else chl_c_from_psi(Un[3], Un[4], Un[5], &cxx, &cxy, &cyy, &czz);
                    O.c[0][i] = cxx; O.c[1][i] = cxy; O.c[2][i] = cyy; O.c[3][i] = czz;
                }
                if constexpr (FP && (FORM == SUNSET_FORM_DI || FORM == SUNSET_FORM_LC)) {
                    // DI: c is the state itself (czz = Un[6]); LC: czz is carried
                    const double czz = FORM == SUNSET_FORM_DI ? Un[6] : n.czz;
                    O.f[i] = fenep_f(cK.fenep_l2, FORM == SUNSET_FORM_DI ? Un[3] : O.c[0][i],
                                     FORM == SUNSET_FORM_DI ? Un[5] : O.c[2][i], czz);
                }
            }
        }
    }
    if (stage == 3) block_max_bits(emax_bits, &A.sc->emax_bits);
}

// filter_variables (rhs_di.F90:667-720; rhs.F90:792-900; rhs_lc.F90:818-893): the
// hyperviscous filter of each evolved field plus the mass-correction partial sums.
//
// FP (Cholesky FENE-P): psizz is filtered too, and the psi factors of J = f c are converted to
// factors of c before filtering and back after it (rhs.F90:815-869) -- in shared memory for
// the halo, in registers for the node itself.
template <int FORM, bool MX, bool FP = false>
__global__ void __launch_bounds__(kTile, 4) k_filter(StageArgs A) {
    const StepConsts &cK = A.K;
    extern __shared__ __align__(16) double smem[];
    constexpr bool CF = FP && FORM == SUNSET_FORM_CHL;
    constexpr int nf = (FORM == SUNSET_FORM_DI || CF) ? 7 : (FORM == SUNSET_FORM_NEWT ? 3 : 6);
    const Fields &F = A.in;
    const int i = blockIdx.x * kTile + threadIdx.x;
    const bool live = (i >> 5) < cK.nslices;
    LinkRing<MX, 1, filter_ring_depth(MX)> R;
    static_assert(!MX, "the mixed filter is k_filter_mx");
    R.src[0] = reinterpret_cast<const double2 *>(A.wh);
    R.init(smem + halo_doubles(nf, A.hmax), reinterpret_cast<const unsigned *>(A.lloc),
           live ? (A.slice_ptr[i >> 5] >> 1) + (i & 31) : 0, live ? A.slice_w[i >> 5] >> 1 : 0);
    R.prologue();
    load_halo<nf>(A, smem, [&](int f) -> const double * {
        return f == 0 ? F.ro : f == 1 ? F.rou : f == 2 ? F.rov : F.q[f - 3];
    });
    const int hm = A.hmax;
    if constexpr (CF) {
        const int hn = A.halo_ptr[blockIdx.x + 1] - A.halo_ptr[blockIdx.x];
        for (int h = threadIdx.x; h < hn; h += blockDim.x)
            chl_fenep_to_c_factor(cK.fenep_l2, smem[3 * hm + h], smem[4 * hm + h], smem[5 * hm + h], smem[6 * hm + h]);
        __syncthreads();
    }
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
            // all loads before the first store (the arrays are not known to be distinct)
            double own[7], res[7];
#pragma unroll
            for (int f = 0; f < 7; f++) own[f] = (f < nf || FORM != SUNSET_FORM_NEWT) ? src[f][i] : 0.0;
            const double vol = A.vol[i];
            if constexpr (CF) chl_fenep_to_c_factor(cK.fenep_l2, own[3], own[4], own[5], own[6]);
#pragma unroll
            for (int f = 0; f < 7; f++) {
                if (f < nf) {
                    const double p = own[f];
                    double r = p + (t[f] - p * hs);
                    if (wall && (f == 1 || f == 2)) r = 0.0;  // apply_time_dependent_bounds after the filter
                    res[f] = r;
                    if (f == 0) rof = r;
                }
            }
            if constexpr (CF) chl_fenep_to_j_factor(cK.fenep_l2, res[3], res[4], res[5], res[6]);
#pragma unroll
            for (int f = 0; f < 7; f++) {
                if (f < nf) dst[f][i] = res[f];
                else if (FORM != SUNSET_FORM_NEWT) dst[f][i] = own[f];  // carried through (never converted)
            }
            part = (rof - cK.rho_char) * vol;
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

// The mixed-precision filter: the design of the mixed stage kernel applied to
// filter_variables (rhs_*.F90 as above).  The tile's halo of the evolved fields as FP32
// offsets from per-tile FP64 references (AoS words, odd count a node), the link stream (one
// FP32 weight a link and the 16-bit local index, both in the bank-aware order) moved by bulk
// copies, and the filter term sum_k w_k (phi_j - phi_i) summed in FP32, added to the node's
// FP64 value.  Cholesky FENE-P converts the psi factors of J = f c to those of c in FP64
// before the offsets are taken, and back after the filter.
constexpr int kMxfChunk = 4;  // link pairs per bulk copy (two weight words and one index word a pair and lane)
constexpr int kMxfDepth = 2;
__host__ __device__ constexpr size_t mxf_ring_bytes() { return (size_t)kTileSlices * kMxfDepth * kMxfChunk * 32 * 12; }
__host__ __device__ constexpr size_t mxf_bar_bytes() { return (size_t)kTileSlices * kMxfDepth * 8; }
__host__ __device__ inline size_t mxf_smem_bytes(int nf, int hmax) {
    return mxf_ring_bytes() + mxf_bar_bytes() + (size_t)mx_words(nf) * hmax * 8;
}

template <int FORM, bool FP, bool MIR>
__global__ void __launch_bounds__(kTile, 4) k_filter_mx(StageArgs A) {
    const StepConsts &cK = A.K;
    extern __shared__ __align__(16) double smem[];
    constexpr bool CF = FP && FORM == SUNSET_FORM_CHL;
    constexpr int nf = (FORM == SUNSET_FORM_DI || CF) ? 7 : (FORM == SUNSET_FORM_NEWT ? 3 : 6);
    constexpr int NP = (nf + 1) / 2, NW = mx_words(nf);
    const Fields &F = A.in;
    const int i = blockIdx.x * kTile + threadIdx.x;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int sl = blockIdx.x * kTileSlices + warp;
    const bool live = sl < cK.nslices;
    // per warp: kMxfDepth stages of [kMxfChunk pairs][32 lanes][w0 w1 idx0|idx1]
    char *ringb = reinterpret_cast<char *>(smem) + (size_t)warp * kMxfDepth * kMxfChunk * 32 * 12;
    const unsigned bar0 = smem_addr(reinterpret_cast<char *>(smem) + mxf_ring_bytes() + (size_t)warp * kMxfDepth * 8);
    float2 *hp = reinterpret_cast<float2 *>(reinterpret_cast<char *>(smem) + mxf_ring_bytes() + mxf_bar_bytes());
    const long long base = live ? A.slice_ptr[sl] : 0;
    const int npair = live ? A.slice_w[sl] >> 1 : 0, nchunk = (npair + kMxfChunk - 1) / kMxfChunk;
    auto issue = [&](int c) {
        const int s = c % kMxfDepth;
        const int np = min(kMxfChunk, npair - c * kMxfChunk);
        const unsigned bar = bar0 + 8u * s;
        const long long o = base + (long long)c * kMxfChunk * 64;
        char *st = ringb + (size_t)s * kMxfChunk * 32 * 12;
        mbar_expect_tx(bar, (unsigned)np * 384u);
        bulk_load(smem_addr(st), A.wf + (3 * o) / 2, (unsigned)np * 384u, bar);
    };
    auto wait = [&](int c) { return mbar_wait_bounded(bar0 + 8u * (c % kMxfDepth), (unsigned)(c / kMxfDepth) & 1u); };
    if (live && lane == 0) {
        for (int s = 0; s < kMxfDepth; s++) mbar_init(bar0 + 8u * s, 1u);
        mbar_init_fence();
        for (int c = 0; c < kMxfDepth && c < nchunk; c++) issue(c);
    }
    // halo as offsets (FENE-P Cholesky: psi of c, converted in FP64 first); MIR: the node set
    // has mirror links, whose reflected fields have reference 0
    constexpr bool mir = MIR;
    const double *src[7] = {F.ro, F.rou, F.rov, F.q[0], F.q[1], F.q[2], F.q[3]};
    const int hb = A.halo_ptr[blockIdx.x], hn = A.halo_ptr[blockIdx.x + 1] - hb;
    const int n0 = __ldg(A.halo + hb);
    auto values = [&](int node, double *v) {
#pragma unroll
        for (int f = 0; f < nf; f++) v[f] = __ldg(src[f] + node);
        if constexpr (CF) chl_fenep_to_c_factor(cK.fenep_l2, v[3], v[4], v[5], v[6]);
    };
    double rf[nf];
    values(n0, rf);
#pragma unroll
    for (int f = 0; f < nf; f++)
        if (mir && (f == 1 || f == 2 || f == 4)) rf[f] = 0.0;
    for (int h = threadIdx.x; h < hn; h += blockDim.x) {
        double v[nf];
        values(__ldg(A.halo + hb + h), v);
#pragma unroll
        for (int p = 0; p < NP; p++)
            hp[h * NW + p] = make_float2((float)(v[2 * p] - rf[2 * p]), 2 * p + 1 < nf ? (float)(v[2 * p + 1] - rf[2 * p + 1]) : 0.0f);
    }
    double own[7];
    values(i < cK.npfb ? i : 0, own);
    // the filter terms of field pairs (the halo's float2 words), in paired FP32 instructions
    float2 noi[NP], tp[NP];
#pragma unroll
    for (int p = 0; p < NP; p++) {
        noi[p] = make_float2(-(float)(own[2 * p] - rf[2 * p]), 2 * p + 1 < nf ? -(float)(own[2 * p + 1] - rf[2 * p + 1]) : 0.0f);
        tp[p] = make_float2(0.0f, 0.0f);
    }
    __syncthreads();
    auto link = [&](unsigned loc, float w) {
        const float2 *v = hp + (loc & kLocMask) * NW;
        const float2 w2 = make_float2(w, w);
        if (MIR && (loc >> 14)) {  // a mirror image: u, v and the xy component with the mirror's sign
            const unsigned code = loc >> 14;
            const float su = (code == 1u || code == 3u) ? -1.0f : 1.0f, sv = (code == 2u || code == 3u) ? -1.0f : 1.0f;
            const float sxy = (code == 1u || code == 2u) ? -1.0f : 1.0f;
#pragma unroll
            for (int p = 0; p < NP; p++) {
                const int f0 = 2 * p, f1 = 2 * p + 1;
                const float s0 = f0 == 1 ? su : f0 == 2 ? sv : f0 == 4 ? sxy : 1.0f;
                const float s1 = f1 == 1 ? su : f1 == 2 ? sv : f1 == 4 ? sxy : 1.0f;
                tp[p] = __ffma2_rn(w2, __ffma2_rn(make_float2(s0, s1), v[p], noi[p]), tp[p]);
            }
        } else {
#pragma unroll
            for (int p = 0; p < NP; p++) tp[p] = __ffma2_rn(w2, __fadd2_rn(v[p], noi[p]), tp[p]);
        }
    };
    if (live) {
        for (int c = 0; c < nchunk; c++) {
            if (!wait(c)) {
                if (lane == 0) atomicExch(&A.sc->err, 2);
                for (int c2 = c; c2 < c + kMxfDepth && c2 < nchunk; c2++) wait(c2);
                break;
            }
            const int np = min(kMxfChunk, npair - c * kMxfChunk);
            const unsigned *st = reinterpret_cast<const unsigned *>(ringb + (size_t)(c % kMxfDepth) * kMxfChunk * 32 * 12) +
                                 3 * lane;
#pragma unroll
            for (int p = 0; p < kMxfChunk; p++) {
                if (p < np) {
                    const unsigned w0 = st[p * 96], w1 = st[p * 96 + 1], l2 = st[p * 96 + 2];
                    link(l2 & 0xffffu, __uint_as_float(w0));
                    link(l2 >> 16, __uint_as_float(w1));
                }
            }
            __syncwarp();
            if (lane == 0 && c + kMxfDepth < nchunk) {
                fence_proxy_async();
                issue(c + kMxfDepth);
            }
        }
    }
    double part = 0.0;
    if (live && i < cK.npfb) {
        double *dst[7] = {A.out.ro, A.out.rou, A.out.rov, A.out.q[0], A.out.q[1], A.out.q[2], A.out.q[3]};
        const bool wall = cK.has_walls && A.ntype[i] == 0;
        // loads before the first store (the arrays are not known to be distinct)
        const double vol = A.vol[i], carried = nf < 7 && FORM != SUNSET_FORM_NEWT ? src[6][i] : 0.0;
        double res[7];
#pragma unroll
        for (int f = 0; f < 7; f++) {
            if (f < nf) {
                double r = own[f] + (double)((f & 1) ? tp[f >> 1].y : tp[f >> 1].x);
                if (wall && (f == 1 || f == 2)) r = 0.0;  // apply_time_dependent_bounds after the filter
                res[f] = r;
            }
        }
        if constexpr (CF) chl_fenep_to_j_factor(cK.fenep_l2, res[3], res[4], res[5], res[6]);
#pragma unroll
        for (int f = 0; f < 7; f++) {
            if (f < nf) dst[f][i] = res[f];
            else if (FORM != SUNSET_FORM_NEWT) dst[f][i] = carried;  // psi_zz / c_zz, nf = 6
        }
        part = (res[0] - cK.rho_char) * vol;
    }
    // deterministic two-level sum: fixed tree in the block, fixed order over blocks
    __shared__ double red[kTile];
    red[threadIdx.x] = part;
    __syncthreads();
    for (int s2 = blockDim.x / 2; s2 > 0; s2 >>= 1) {
        if ((int)threadIdx.x < s2) red[threadIdx.x] = red[threadIdx.x] + red[threadIdx.x + s2];
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
        for (int s2 = blockDim.x / 2; s2 > 0; s2 >>= 1) {
            if ((int)threadIdx.x < s2) red[threadIdx.x] = red[threadIdx.x] + red[threadIdx.x + s2];
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
    const StepConsts &cK = A.K;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const double dro = A.sc->dro;
    double uvol = 0.0;
    if (i < cK.npfb) {
        const Fields &F = A.out;
        // every load before the first store: the compiler cannot tell the field arrays apart
        // and would otherwise wait out each load after a store
        double ro = F.ro[i], rou = F.rou[i], rov = F.rov[i];
        double q0 = 0.0, q1 = 0.0, q2 = 0.0, q3 = 0.0;
        if (FORM == SUNSET_FORM_LC || FORM == SUNSET_FORM_CHL) { q0 = F.q[0][i]; q1 = F.q[1][i]; q2 = F.q[2][i]; }
        if (FORM == SUNSET_FORM_CHL && cK.fenep) q3 = F.q[3][i];
        // the conformation the FENE-P function reads: c itself (direct form), c_zz (carried,
        // log-conformation); the Cholesky form's comes from psi below
        double c0 = 0.0, c2 = 0.0, c3 = 0.0;
        if (F.f) {
            if (FORM != SUNSET_FORM_LC && FORM != SUNSET_FORM_CHL) { c0 = F.c[0][i]; c2 = F.c[2][i]; }
            if (FORM != SUNSET_FORM_CHL) c3 = F.c[3][i];
        }
        const bool hard_in = cK.has_walls && cK.inflow_type == 1 && A.ntype[i] == 1;
        const double uin = hard_in ? A.uin[A.bidx[i]] : 0.0;
        const double vol = cK.vpid ? A.vol[i] : 0.0;
        if (cK.mcorr) ro = ro - dro;
        F.ro[i] = ro;
        if (hard_in) {
            // the bounds again after the filter (step.F90:498): the hard inflow's momentum
            // from the corrected density, at the step's end time (u_inflow_local unchanged)
            rou = uin * ro;
            rov = 0.0;
            F.rou[i] = rou;
            F.rov[i] = rov;
        }
        double ooro = 1.0 / ro;
        const double u = rou * ooro;
        F.u[i] = u;
        F.v[i] = rov * ooro;
        if (FORM == SUNSET_FORM_LC) {
            double cxx, cxy, cyy;
            lc_c_from_psi(q0, q1, q2, &cxx, &cxy, &cyy);
            F.c[0][i] = cxx; F.c[1][i] = cxy; F.c[2][i] = cyy;
            c0 = cxx; c2 = cyy;
        } else if (FORM == SUNSET_FORM_CHL) {
            double cxx, cxy, cyy, czz;
            if (cK.fenep) chl_c_from_psi_fenep(cK.fenep_l2, q0, q1, q2, q3, &cxx, &cxy, &cyy, &czz);
            else chl_c_from_psi(q0, q1, q2, &cxx, &cxy, &cyy, &czz);
            F.c[0][i] = cxx; F.c[1][i] = cxy; F.c[2][i] = cyy; F.c[3][i] = czz;
            c0 = cxx; c2 = cyy; c3 = czz;
        }
        if (F.f) F.f[i] = fenep_f(cK.fenep_l2, c0, c2, c3);
        if (cK.vpid) uvol = u * vol;
    }
    if (cK.vpid && advance) {
        // velocity_control with -Dvpid (statistics.F90:214-303), after the step: the volume
        // sum of u (fixed tree in the block, blocks in order), then the PID update of
        // driving_force(1) by the last block
        __shared__ double red[128];
        __shared__ bool last;
        red[threadIdx.x] = uvol;
        __syncthreads();
        for (int s = blockDim.x / 2; s > 0; s >>= 1) {
            if ((int)threadIdx.x < s) red[threadIdx.x] = red[threadIdx.x] + red[threadIdx.x + s];
            __syncthreads();
        }
        if (threadIdx.x == 0) {
            A.partials[blockIdx.x] = red[0];
            __threadfence();
            const unsigned int prev = atomicAdd(&A.sc->done_ctr, 1u);
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
                DevScalars *sc = A.sc;
                const double tot_vol = sc->tv, dt = sc->dt;
                const double tot_u = red[0] / tot_vol;
                const double eflow_n = 1.0 - (tot_u * tot_vol) / (cK.Ly * cK.Lx);
                sc->sum_eflow = sc->sum_eflow + eflow_n * dt;
                const double deflowdt = (eflow_n - sc->eflow_nm1) / dt;
                const double facA = ((((0.5 * 0.5) * 0.5) * 1.0) * 2.0) * 2.0;
                const double facB = facA / 0.4, facC = facA * 0.02;
                double df = ((facA * eflow_n) + facB * sc->sum_eflow) + facC * deflowdt;
                df = (500.0 < df) ? 500.0 : df;
                df = (-500.0 > df) ? -500.0 : df;
                sc->df = df;
                sc->eflow_nm1 = eflow_n;
                sc->done_ctr = 0;
            }
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
        // without -Dvpid the statistics call after the step zeroes the driving force
        // (statistics.F90:288; a restart may have loaded one for the first step)
        if (!cK.vpid) sc->df = 0.0;
    }
}

// set_tstep (step.F90:569-622) over the current state: block minima of s/(|u|+c) and
// s^2 rho/mu, folded into dt_cfl and dt_parabolic by k_pid / the host.
__global__ void __launch_bounds__(128) k_tstep(const double *u, const double *v, const double *ro, const double *sp,
                                                const int *ntype, int npfb, DevScalars *sc, StepConsts cK) {
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
__global__ void k_pid(DevScalars *sc, StepConsts cK) {
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

__global__ void k_tstep_fold(DevScalars *sc, StepConsts cK) {
    double dcfl = __longlong_as_double((long long)sc->cfl_bits);
    double dvisc = __longlong_as_double((long long)sc->par_bits);
    sc->dt_cfl = (1.0 * dcfl) * cK.L_char;
    sc->dt_par = (((2.0 / 3.0) * dvisc) * cK.L_char) * cK.L_char;
}

// ---------------------------------------------------------------------------------------
// Single operators of the C-ABI (derivatives.F90), on a field in internal order.
// ---------------------------------------------------------------------------------------
__global__ void k_op_grad_lap(StageArgs A, const double *phi, double *gx, double *gy, double *lap) {
    const StepConsts &cK = A.K;
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
    const StepConsts &cK = A.K;
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
                            const int *ntype, int has_walls, Fields F, StepConsts cK) {
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
        if (cK.fenep) {
            chl_psi_from_c_fenep(cK.fenep_l2, c0, c1, c2, c3, &p0, &p1, &p2, &p3);
            F.q[0][i] = p0; F.q[1][i] = p1; F.q[2][i] = p2; F.q[3][i] = p3;
            chl_c_from_psi_fenep(cK.fenep_l2, p0, p1, p2, p3, &c0, &c1, &c2, &c3);
        } else {
            chl_psi_from_c(c0, c1, c2, c3, &p0, &p1, &p2, &p3);
            F.q[0][i] = p0; F.q[1][i] = p1; F.q[2][i] = p2; F.q[3][i] = p3;
            chl_c_from_psi(p0, p1, p2, &c0, &c1, &c2, &c3);
        }
        F.c[0][i] = c0; F.c[1][i] = c1; F.c[2][i] = c2; F.c[3][i] = c3;
    } else {
        F.q[0][i] = c0; F.q[1][i] = c1; F.q[2][i] = c2; F.q[3][i] = c3;
    }
    if (F.f) F.f[i] = fenep_f(cK.fenep_l2, c0, c2, c3);
}

// Conservative state given directly (ro, rou, rov, q0..q3), derived fields recomputed
// as get_velocity_from_momentum / get_c_from_psi do.
__device__ __forceinline__ void set_conservative_node(int i, int form, double ro, double rou, double rov, double q0,
                                                      double q1, double q2, double q3, const Fields &F,
                                                      const StepConsts &cK) {
    F.ro[i] = ro; F.rou[i] = rou; F.rov[i] = rov;
    F.q[0][i] = q0; F.q[1][i] = q1; F.q[2][i] = q2; F.q[3][i] = q3;
    double ooro = 1.0 / ro;
    F.u[i] = rou * ooro;
    F.v[i] = rov * ooro;
    if (form == SUNSET_FORM_LC) {
        double c0, c1, c2;
        lc_c_from_psi(q0, q1, q2, &c0, &c1, &c2);
        F.c[0][i] = c0; F.c[1][i] = c1; F.c[2][i] = c2; F.c[3][i] = 1.0;
    } else if (form == SUNSET_FORM_CHL) {
        double c0, c1, c2, c3;
        if (cK.fenep) chl_c_from_psi_fenep(cK.fenep_l2, q0, q1, q2, q3, &c0, &c1, &c2, &c3);
        else chl_c_from_psi(q0, q1, q2, &c0, &c1, &c2, &c3);
        F.c[0][i] = c0; F.c[1][i] = c1; F.c[2][i] = c2; F.c[3][i] = c3;
    }
    if (F.f) F.f[i] = fenep_f(cK.fenep_l2, F.c[0][i], F.c[2][i], F.c[3][i]);
}
__global__ void k_set_conservative(int npfb, int form, const double *ro, const double *rou, const double *rov,
                                   const double *q0, const double *q1, const double *q2, const double *q3, Fields F,
                                   StepConsts cK) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= npfb) return;
    set_conservative_node(i, form, ro[i], rou[i], rov[i], q0[i], q1[i], q2[i], q3[i], F, cK);
}
// The state from checkpoint *seg of the adjoint's store (7 fields of npfb doubles each a
// checkpoint): the index is read on the device, so a captured graph serves every segment.
__global__ void k_load_checkpoint(int npfb, int form, const double *store, const int *seg, Fields F, StepConsts cK) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= npfb) return;
    const double *cp = store + (size_t)7 * npfb * (size_t)*seg;
    const size_t n = (size_t)npfb;
    set_conservative_node(i, form, cp[i], cp[n + i], cp[2 * n + i], cp[3 * n + i], cp[4 * n + i], cp[5 * n + i],
                          cp[6 * n + i], F, cK);
}
// Scalars set on the stream by a kernel rather than a copy from pageable host memory (which
// the driver stages, and which can hold the host until the stream reaches it).
__global__ void k_set_dt(DevScalars *sc, double dt) { sc->dt = dt; }
__global__ void k_set_segment(DevScalars *sc, int *seg, int s, int itime) {
    sc->itime = itime;
    *seg = s;
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
// The run's constants, passed to every kernel that reads them as a kernel parameter (so that
// handles of different configurations never share them).
StepConsts consts_of(const Handle *H) {
    return step_consts(H->cfg, H->npfb, H->nslices, H->has_mirrors, H->nb > 0, H->xmax - H->xmin, H->ymax - H->ymin);
}

StageArgs make_args(Handle *H, int from, int stage, bool step = false) {
    const bool mx = step && H->cfg.precision == SUNSET_MIXED;
    StageArgs A{};
    A.K = consts_of(H);
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
    A.pk = H->pk;
    A.scx = H->scx; A.scy = H->scy; A.scl = H->scl;
    A.wf = H->wf;
    A.gsx = H->gsx; A.gsy = H->gsy; A.lsum = H->lsum;
    A.hsum = H->hsum;
    A.vol = H->vol;
    A.py_node = H->py;
    A.ntype = H->ntype;
    A.rnx = H->rnx;
    A.rny = H->rny;
    A.lloc_ref = H->lloc;
    A.cnt_small = H->cnt_small;
    A.bidx = H->bidx;
    A.brow = H->brow;
    A.wbt = H->wbt;
    A.wbt_sum = H->wbt_sum;
    A.sp = H->sp;
    A.nplink = H->nplink;
    A.in = H->buf[from];
    A.out = H->buf[from ^ 1];
    for (int f = 0; f < 7; f++) {
        A.reg[f] = H->reg[f]; A.eacc[f] = H->eacc[f]; A.rhs[f] = H->rhs[f];
        A.dreg[f] = H->dreg32[f]; A.eacc32[f] = H->eacc32[f];
    }
    A.sc = H->dsc;
    A.partials = H->partials;
    A.alpha = H->alpha;
    A.uin = H->uin;
    A.stage = stage;
    return A;
}

int upload_consts(Handle *) { return 0; }

constexpr size_t kMaxStageSmem = 200 * 1024;

#define SUNSET_SMEM_ATTR(K) SUNSET_CUDA(H, cudaFuncSetAttribute(K, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kMaxStageSmem))
template <int FORM, bool MD, bool FP>
int stage_smem_attributes(Handle *H, bool mx) {
    if (H->nb > 0) {
        SUNSET_SMEM_ATTR((k_stage<FORM, MD, false, FP, true>));
        if (mx) SUNSET_SMEM_ATTR((k_stage<FORM, MD, true, FP, true>));
    } else {
        SUNSET_SMEM_ATTR((k_stage<FORM, MD, false, FP, false>));
        if (mx) SUNSET_SMEM_ATTR((k_stage<FORM, MD, true, FP, false>));
    }
    return 0;
}
template <int FORM, bool FP>
int filter_smem_attributes(Handle *H, bool mx) {
    SUNSET_SMEM_ATTR((k_filter<FORM, false, FP>));
    if (mx) SUNSET_SMEM_ATTR((k_filter_mx<FORM, FP, true>));
    if (mx) SUNSET_SMEM_ATTR((k_filter_mx<FORM, FP, false>));
    return 0;
}

// Opt the staged kernels of the handle's configuration into large dynamic shared memory.
int set_smem_attributes(Handle *H) {
    const bool mx = H->cfg.precision == SUNSET_MIXED, md = H->cfg.Mdiff != 0.0, fp = H->cfg.fenep != 0;
    int rc = 0;
    switch (H->cfg.form) {
    case SUNSET_FORM_DI:
        rc = md ? (fp ? stage_smem_attributes<SUNSET_FORM_DI, true, true>(H, mx) : stage_smem_attributes<SUNSET_FORM_DI, true, false>(H, mx))
                : (fp ? stage_smem_attributes<SUNSET_FORM_DI, false, true>(H, mx) : stage_smem_attributes<SUNSET_FORM_DI, false, false>(H, mx));
        if (!rc) rc = filter_smem_attributes<SUNSET_FORM_DI, false>(H, mx);
        break;
    case SUNSET_FORM_CHL:
        rc = md ? (fp ? stage_smem_attributes<SUNSET_FORM_CHL, true, true>(H, mx) : stage_smem_attributes<SUNSET_FORM_CHL, true, false>(H, mx))
                : (fp ? stage_smem_attributes<SUNSET_FORM_CHL, false, true>(H, mx) : stage_smem_attributes<SUNSET_FORM_CHL, false, false>(H, mx));
        if (!rc) rc = fp ? filter_smem_attributes<SUNSET_FORM_CHL, true>(H, mx) : filter_smem_attributes<SUNSET_FORM_CHL, false>(H, mx);
        break;
    case SUNSET_FORM_LC:
        rc = fp ? stage_smem_attributes<SUNSET_FORM_LC, false, true>(H, mx) : stage_smem_attributes<SUNSET_FORM_LC, false, false>(H, mx);
        if (!rc) rc = filter_smem_attributes<SUNSET_FORM_LC, false>(H, mx);
        break;
    default:
        rc = stage_smem_attributes<SUNSET_FORM_NEWT, false, false>(H, mx);
        if (!rc) rc = filter_smem_attributes<SUNSET_FORM_NEWT, false>(H, mx);
    }
    return rc;
}
#undef SUNSET_SMEM_ATTR

inline bool is_mx(const Handle *H) { return H->cfg.precision == SUNSET_MIXED; }

template <int FORM, bool MD, bool FP>
int launch_stage(Handle *H, const StageArgs &A, bool mx) {
    const size_t smem = mx ? mx_smem_bytes(ngather(FORM, MD, FP), H->halo_max)
                           : halo_doubles(ngather(FORM, MD, FP), H->halo_max) * sizeof(double) +
                                 LinkRing<false, 3, ring_depth(false)>::bytes();
    if (smem > kMaxStageSmem) return set_err(H, SUNSET_ERR_SCOPE, "tile halo too large for shared memory");
    if (H->nb > 0) {
        if (mx) k_stage<FORM, MD, true, FP, true><<<H->ntiles, kTile, smem, H->stream>>>(A);
        else k_stage<FORM, MD, false, FP, true><<<H->ntiles, kTile, smem, H->stream>>>(A);
    } else {
        if (mx) k_stage<FORM, MD, true, FP, false><<<H->ntiles, kTile, smem, H->stream>>>(A);
        else k_stage<FORM, MD, false, FP, false><<<H->ntiles, kTile, smem, H->stream>>>(A);
    }
    return 0;
}

// A must come from make_args(..., step = true); mx is the handle's precision.
int launch_stage_any(Handle *H, const StageArgs &A, bool mx) {
    const bool md = H->cfg.Mdiff != 0.0, fp = H->cfg.fenep != 0;
    switch (H->cfg.form) {
    case SUNSET_FORM_DI:
        if (md) return fp ? launch_stage<SUNSET_FORM_DI, true, true>(H, A, mx) : launch_stage<SUNSET_FORM_DI, true, false>(H, A, mx);
        return fp ? launch_stage<SUNSET_FORM_DI, false, true>(H, A, mx) : launch_stage<SUNSET_FORM_DI, false, false>(H, A, mx);
    case SUNSET_FORM_CHL:
        if (md) return fp ? launch_stage<SUNSET_FORM_CHL, true, true>(H, A, mx) : launch_stage<SUNSET_FORM_CHL, true, false>(H, A, mx);
        return fp ? launch_stage<SUNSET_FORM_CHL, false, true>(H, A, mx) : launch_stage<SUNSET_FORM_CHL, false, false>(H, A, mx);
    case SUNSET_FORM_LC:
        return fp ? launch_stage<SUNSET_FORM_LC, false, true>(H, A, mx) : launch_stage<SUNSET_FORM_LC, false, false>(H, A, mx);
    default: return launch_stage<SUNSET_FORM_NEWT, false, false>(H, A, mx);
    }
}

template <int FORM>
int launch_filter(Handle *H, const StageArgs &A, bool mx) {
    const bool cf = FORM == SUNSET_FORM_CHL && H->cfg.fenep;  // Cholesky FENE-P: psizz and the conversions
    const int nf = (FORM == SUNSET_FORM_DI || cf) ? 7 : (FORM == SUNSET_FORM_NEWT ? 3 : 6);
    if (mx) {
        const size_t smem = mxf_smem_bytes(nf, H->halo_max);
        if (smem > kMaxStageSmem) return set_err(H, SUNSET_ERR_SCOPE, "tile halo too large for shared memory");
        if (H->has_mirrors) {
            if (cf) k_filter_mx<FORM, true, true><<<H->ntiles, kTile, smem, H->stream>>>(A);
            else k_filter_mx<FORM, false, true><<<H->ntiles, kTile, smem, H->stream>>>(A);
        } else {
            if (cf) k_filter_mx<FORM, true, false><<<H->ntiles, kTile, smem, H->stream>>>(A);
            else k_filter_mx<FORM, false, false><<<H->ntiles, kTile, smem, H->stream>>>(A);
        }
        return 0;
    }
    const size_t smem = halo_doubles(nf, H->halo_max) * sizeof(double) + LinkRing<false, 1, filter_ring_depth(false)>::bytes();
    if (smem > kMaxStageSmem) return set_err(H, SUNSET_ERR_SCOPE, "tile halo too large for shared memory");
    if (cf) k_filter<FORM, false, true><<<H->ntiles, kTile, smem, H->stream>>>(A);
    else k_filter<FORM, false><<<H->ntiles, kTile, smem, H->stream>>>(A);
    return 0;
}

// The kernels of one step.  stage_ev (optional, 2 events): recorded before the first and
// after the last of the four RK stage launches, which run back to back on the stream, for
// timing the stage kernel inside a real step sequence.
template <int FORM>
int launch_step_kernels(Handle *H, int from, int pid, cudaEvent_t *stage_ev) {
    const int TB = 128;
    cudaStream_t st = H->stream;
    const bool mx = is_mx(H);
    if (pid) k_pid<<<1, 1, 0, st>>>(H->dsc, consts_of(H));
    int b = from;
    for (int s = 0; s < 4; s++) {
        StageArgs A = make_args(H, b, s, true);
        if (stage_ev && s == 0) SUNSET_CUDA(H, cudaEventRecord(stage_ev[0], st));
        if (int rc = launch_stage_any(H, A, mx)) return rc;
        if (stage_ev && s == 3) SUNSET_CUDA(H, cudaEventRecord(stage_ev[1], st));
        b ^= 1;
    }
    StageArgs F = make_args(H, b, 5, true);
    if (int rc = launch_filter<FORM>(H, F, mx)) return rc;
    b ^= 1;
    StageArgs Z = make_args(H, b ^ 1, 5, true);  // in = filter input, out = filtered buffer
    const int fb = (H->npfb + TB - 1) / TB;
    k_finalize<FORM><<<fb, TB, 0, st>>>(Z, 1);
    k_tstep<<<fb, TB, 0, st>>>(H->buf[b].u, H->buf[b].v, H->buf[b].ro, H->sp, H->ntype, H->npfb, H->dsc, consts_of(H));
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

// u_inflow_local of the initial state (setup_flow.F90:48-50,128-138): u of each inflow node,
// U_char elsewhere.
__global__ void k_init_uin(int nb, const int *blist, const int *ntype, const double *u, double uchar, double *uin) {
    const int jj = blockIdx.x * blockDim.x + threadIdx.x;
    if (jj >= nb) return;
    const int i = blist[jj];
    uin[jj] = ntype[i] == 1 ? u[i] : uchar;
}

int init_inflow(Handle *H) {
    if (H->nb == 0) return 0;
    k_init_uin<<<(H->nb + 127) / 128, 128, 0, H->stream>>>(H->nb, H->blist, H->ntype, H->buf[H->cur].u, H->cfg.U_char,
                                                          H->uin);
    SUNSET_CUDA(H, cudaGetLastError());
    H->uin_set = true;
    return 0;
}

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
        if (H->cfg.fenep && (H->cfg.form == SUNSET_FORM_DI || H->cfg.form == SUNSET_FORM_LC) && dalloc(H, &F.f, n))
            return SUNSET_ERR_NOMEM;
    }
    for (int f = 0; f < 7; f++) {
        if (dalloc(H, &H->rhs[f], n)) return SUNSET_ERR_NOMEM;
        if (is_mx(H)) {
            if (dalloc(H, &H->dreg32[f], n) || dalloc(H, &H->eacc32[f], n)) return SUNSET_ERR_NOMEM;
        } else {
            if (dalloc(H, &H->reg[f], n) || dalloc(H, &H->eacc[f], n)) return SUNSET_ERR_NOMEM;
        }
    }
    if (dalloc(H, &H->alpha, n)) return SUNSET_ERR_NOMEM;
    SUNSET_CUDA(H, cudaMemsetAsync(H->alpha, 0, n * sizeof(double), H->stream));
    if (H->nb > 0 && dalloc(H, &H->uin, H->nb)) return SUNSET_ERR_NOMEM;
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
    s.eflow_nm1 = 1.0;  // flow-rate controller, setup_flow.F90:165-169 (sum_eflow, df = 0)
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
                                                              H->ntype, H->nb > 0, H->buf[0], consts_of(H));
    SUNSET_CUDA(H, cudaGetLastError());
    rc = init_scalars(H);
    if (rc) return rc;
    if ((rc = init_inflow(H))) return rc;
    return set_tstep_device(H);
}

int state_set_conservative_device(Handle *H, const double *const *f7) {
    int rc = upload_consts(H);
    if (rc) return rc;
    k_set_conservative<<<(H->npfb + 127) / 128, 128, 0, H->stream>>>(H->npfb, H->cfg.form, f7[0], f7[1], f7[2],
                                                                     f7[3], f7[4], f7[5], f7[6], H->buf[H->cur],
                                                                     consts_of(H));
    SUNSET_CUDA(H, cudaGetLastError());
    if (!H->uin_set) return init_inflow(H);
    return 0;
}

int set_tstep_device(Handle *H) {
    const Fields &F = H->buf[H->cur];
    DevScalars *sc = H->dsc;
    unsigned long long inf = 0x7ff0000000000000ull;
    SUNSET_CUDA(H, cudaMemcpyAsync(&sc->cfl_bits, &inf, sizeof(inf), cudaMemcpyHostToDevice, H->stream));
    SUNSET_CUDA(H, cudaMemcpyAsync(&sc->par_bits, &inf, sizeof(inf), cudaMemcpyHostToDevice, H->stream));
    k_tstep<<<(H->npfb + 127) / 128, 128, 0, H->stream>>>(F.u, F.v, F.ro, H->sp, H->ntype, H->npfb, sc, consts_of(H));
    k_tstep_fold<<<1, 1, 0, H->stream>>>(sc, consts_of(H));
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
    if (mode == 0) {
        k_set_dt<<<1, 1, 0, st>>>(H->dsc, dt);
        SUNSET_CUDA(H, cudaGetLastError());
    }
    for (int s = 0; s < nsteps; s++) {
        int from = H->cur;
        if (!H->graph[from] || H->graph_mode[from] != mode) {
            if (H->graph[from]) { cudaGraphExecDestroy(H->graph[from]); H->graph[from] = nullptr; }
            cudaGraph_t g;
            SUNSET_CUDA(H, cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
            g = nullptr;
            int lrc = launch_step(H, from, mode);
            cudaError_t ce = cudaStreamEndCapture(st, &g);
            if (lrc || ce != cudaSuccess) {  // the capture ended either way: drop what it recorded
                if (g) cudaGraphDestroy(g);
                if (lrc) return lrc;
                SUNSET_CUDA(H, ce);
            }
            const cudaError_t ie = cudaGraphInstantiate(&H->graph[from], g, 0);
            cudaGraphDestroy(g);
            if (ie != cudaSuccess) H->graph[from] = nullptr;
            SUNSET_CUDA(H, ie);
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
    std::vector<cudaEvent_t> ev(2 * (size_t)reps);
    for (auto &e : ev) SUNSET_CUDA(H, cudaEventCreate(&e));
    for (int r = 0; r < reps; r++) {
        if ((rc = launch_step(H, H->cur, 0, ev.data() + 2 * r))) break;
        H->cur ^= 1;
    }
    SUNSET_CUDA(H, cudaStreamSynchronize(H->stream));
    double tot = 0.0;  // the four stage launches of each step, back to back
    for (int r = 0; r < reps && !rc; r++) {
        float t = 0.f;
        SUNSET_CUDA(H, cudaEventElapsedTime(&t, ev[2 * r], ev[2 * r + 1]));
        tot += t;
    }
    for (auto &e : ev) cudaEventDestroy(e);
    if (rc) return rc;
    *ms = tot / (4.0 * reps);
    // Algorithmic bytes of one stage launch, averaged over the four stages: each node's
    // small links once (16-bit local index + 3 weights of 8 bytes = 26 bytes; 12 in the mixed
    // path's packed words; links, not padded SELL slots), its state and derived fields read
    // once (the halo copies of neighbours' values are re-reads), the RK registers S and E
    // read in stages 1-3 and written in stages 0-2 (8 bytes, 4 in the mixed path), the next
    // state with its derived fields written (conservative fields only after stage 3), and
    // the per-node stencil sums (mixed: weight scales) and ordinate read.
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
    *bytes = (double)links * (mx ? 12.0 : 2.0 + 3.0 * wb) +
             (double)H->npfb * (8.0 * nread + 3.0 * nf * wb + 8.0 * (3.0 * nwrite + 7.0) / 4.0 + (mx ? 20.0 : 32.0));
    return 0;
}


// ---------------------------------------------------------------------------------------
// Field dumps (output.F90:184-370): per node rho - rho_char, u, v, vorticity, Q criterion,
// the step error alpha_out, cxx, cxy, cyy, czz.  On wall nodes the velocity gradient is in
// the wall's normal-tangent frame, so vorticity and Q are rotated as output.F90:229-241 does.
// ---------------------------------------------------------------------------------------
namespace {
__global__ void k_dump(int n, Fields F, const double *gux, const double *guy, const double *gvx, const double *gvy,
                       const int *ntype, const double *rnx, const double *rny, int has_walls, const double *alpha,
                       double *out, StepConsts cK) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double ux = gux[i], uy = guy[i], vx = gvx[i], vy = gvy[i];
    double vort = vx - uy;
    double q = (-(0.5 * (ux * ux)) - 0.5 * (vy * vy)) - uy * vx;
    if (has_walls && ntype[i] == 0) {
        const double xn = rnx[i], yn = rny[i];
        vort = xn * (vx - uy) - yn * (ux + vy);
        const double a = xn * ux - yn * uy, b = yn * vx + xn * vy;
        q = (-(0.5 * (a * a)) - 0.5 * (b * b)) - (yn * ux + xn * uy) * (xn * vx - yn * vy);
    }
    const double col[10] = {-cK.rho_char + F.ro[i], F.u[i], F.v[i], vort, q, alpha ? alpha[i] : 0.0,
                            F.c[0][i], F.c[1][i], F.c[2][i], F.c[3][i]};
#pragma unroll
    for (int f = 0; f < 10; f++) out[(size_t)f * n + i] = col[f];
}

struct CheckpointHeader {
    char magic[8];
    int version, npfb, form, precision, fenep, nfields;
    double xsum, ysum;  // fingerprint of the node set
};
}  // namespace

int dump_columns(Handle *H, double *out) {
    const int n = H->npfb;
    const Fields &F = H->buf[H->cur];
    double *g = H->tmpd;  // 4 x npfb scratch
    if (int rc = op_gradient(H, F.u, g, g + n)) return rc;
    if (int rc = op_gradient(H, F.v, g + 2 * (size_t)n, g + 3 * (size_t)n)) return rc;
    k_dump<<<(n + 127) / 128, 128, 0, H->stream>>>(n, F, g, g + n, g + 2 * (size_t)n, g + 3 * (size_t)n, H->ntype,
                                                   H->rnx, H->rny, H->nb > 0, H->alpha, out, consts_of(H));
    SUNSET_CUDA(H, cudaGetLastError());
    return 0;
}

// Checkpoint: the device state between steps, bit for bit -- the 13 fields of the current
// buffer (and the FENE-P function where it is kept), the step's scalars (time, dt, itime,
// error-norm history) and the per-node step error, in the internal node order, behind a
// header that names the configuration and fingerprints the node set.  The RK registers are
// rebuilt by every step, so they are not part of it.
static void checkpoint_arrays(const Handle *H, double *const *&arr, int &na, double *tmp[16]) {
    const Fields &F = H->buf[H->cur];
    na = 0;
    const double *src[14] = {F.ro, F.rou, F.rov, F.u, F.v, F.q[0], F.q[1], F.q[2], F.q[3], F.c[0], F.c[1], F.c[2], F.c[3], F.f};
    for (int k = 0; k < 13; k++) {
        if (H->cfg.form == SUNSET_FORM_DI && k >= 9) break;  // DI: c aliases q
        tmp[na++] = const_cast<double *>(src[k]);
    }
    if (F.f) tmp[na++] = F.f;
    tmp[na++] = H->alpha;
    arr = tmp;
}

size_t checkpoint_bytes(const Handle *H) {
    double *tmp[16];
    double *const *arr;
    int na;
    checkpoint_arrays(H, arr, na, tmp);
    return sizeof(CheckpointHeader) + sizeof(DevScalars) + ((size_t)na * H->npfb + (size_t)H->nb) * sizeof(double);
}

static int node_fingerprint(Handle *H, double *xs, double *ys) {
    std::vector<double> x(H->npfb), y(H->npfb);
    SUNSET_CUDA(H, cudaMemcpy(x.data(), H->px, H->npfb * sizeof(double), cudaMemcpyDeviceToHost));
    SUNSET_CUDA(H, cudaMemcpy(y.data(), H->py, H->npfb * sizeof(double), cudaMemcpyDeviceToHost));
    double a = 0.0, b = 0.0;
    for (int i = 0; i < H->npfb; i++) { a = a + x[i]; b = b + y[i]; }
    *xs = a;
    *ys = b;
    return 0;
}

int checkpoint_save(Handle *H, void *buf) {
    double *tmp[16];
    double *const *arr;
    int na;
    checkpoint_arrays(H, arr, na, tmp);
    CheckpointHeader hd{};
    memcpy(hd.magic, "SUNSETCK", 8);
    hd.version = 2;
    hd.npfb = H->npfb;
    hd.form = H->cfg.form;
    hd.precision = H->cfg.precision;
    hd.fenep = H->cfg.fenep;
    hd.nfields = na;
    if (int rc = node_fingerprint(H, &hd.xsum, &hd.ysum)) return rc;
    char *p = static_cast<char *>(buf);
    memcpy(p, &hd, sizeof(hd));
    p += sizeof(hd);
    SUNSET_CUDA(H, cudaMemcpyAsync(p, H->dsc, sizeof(DevScalars), cudaMemcpyDeviceToHost, H->stream));
    p += sizeof(DevScalars);
    for (int k = 0; k < na; k++) {
        SUNSET_CUDA(H, cudaMemcpyAsync(p, arr[k], H->npfb * sizeof(double), cudaMemcpyDeviceToHost, H->stream));
        p += H->npfb * sizeof(double);
    }
    if (H->nb > 0) SUNSET_CUDA(H, cudaMemcpyAsync(p, H->uin, H->nb * sizeof(double), cudaMemcpyDeviceToHost, H->stream));
    SUNSET_CUDA(H, cudaStreamSynchronize(H->stream));
    return 0;
}

int checkpoint_load(Handle *H, const void *buf, size_t bytes) {
    double *tmp[16];
    double *const *arr;
    int na;
    checkpoint_arrays(H, arr, na, tmp);
    if (bytes != checkpoint_bytes(H)) return set_err(H, SUNSET_ERR_ARG, "checkpoint of %zu bytes, expected %zu", bytes, checkpoint_bytes(H));
    CheckpointHeader hd;
    const char *p = static_cast<const char *>(buf);
    memcpy(&hd, p, sizeof(hd));
    double xs, ys;
    if (int rc = node_fingerprint(H, &xs, &ys)) return rc;
    if (memcmp(hd.magic, "SUNSETCK", 8) != 0 || hd.version != 2 || hd.npfb != H->npfb || hd.form != H->cfg.form ||
        hd.precision != H->cfg.precision || hd.fenep != H->cfg.fenep || hd.nfields != na || hd.xsum != xs || hd.ysum != ys)
        return set_err(H, SUNSET_ERR_ARG, "checkpoint written for another configuration or node set");
    p += sizeof(hd);
    SUNSET_CUDA(H, cudaMemcpyAsync(H->dsc, p, sizeof(DevScalars), cudaMemcpyHostToDevice, H->stream));
    p += sizeof(DevScalars);
    for (int k = 0; k < na; k++) {
        SUNSET_CUDA(H, cudaMemcpyAsync(arr[k], p, H->npfb * sizeof(double), cudaMemcpyHostToDevice, H->stream));
        p += H->npfb * sizeof(double);
    }
    if (H->nb > 0) SUNSET_CUDA(H, cudaMemcpyAsync(H->uin, p, H->nb * sizeof(double), cudaMemcpyHostToDevice, H->stream));
    SUNSET_CUDA(H, cudaStreamSynchronize(H->stream));
    H->uin_set = true;
    return upload_consts(H);
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
// Checkpoints: the state every `checkpoint_every` steps.  A segment's forward stages are
// recorded -- the stage input states (13 fields) and the 18 stencil sums g of every node
// and stage, written by the stage kernel itself -- while it is recomputed from its
// checkpoint (the last segment is recorded during the forward run), so the reverse sweep
// runs no forward gather.  Per step the reverse runs five kernels, each over tiles of 256
// nodes j with a shared-memory halo of the nodes whose links reach the tile and a cp.async
// stream of the reverse links (the owners' weights gathered once into that order):
//   filter:       U4_bar = (filter + mass correction)^T U_bar_{n+1}, then the pointwise
//                 reverse of stage 3 (S_bar_3, g_bar_3 and the state's own s_bar_3);
//   stage 3, 2, 1: U_bar_s = transposed stencils of g_bar_s + s_bar_s + the derived
//                 fields reversed, then the pointwise reverse of stage s - 1;
//   stage 0:      U_bar_0 (+ S_bar_0), the adjoint of the step's input, and its per-tile
//                 sums of rho_bar for the next mass-correction reverse.
// The parameter adjoint accumulates per tile and folds once at the end, so, like the
// gathers, its result does not depend on scheduling.
// =======================================================================================
namespace {

// CSR reverse lists: the single transposed operators and the source of the link stream.
struct AdjArgs {
    int npfb;
    const long long *rptr;      // reverse links of node j: [rptr[j], rptr[j+1])
    const int *rslot, *rnode;   // SELL slot (reference order) and the node owning it
    const unsigned char *rcode; // bits 0-1: reflection code, bit 2: a small link (stencils of the stage)
    const double *wx, *wy, *wl, *wh;
    const double *gsx, *gsy, *lsum, *hsum;
};

// Kernels of the reverse sweep.
struct RevArgs {
    StepConsts K;               // the run's constants
    const long long *sptr;      // reverse link streams: slice starts (links)
    const int *sw, *sws;        // slice widths: all links (filter), small links (stage stencils)
    const uint16_t *locs, *locf;  // halo position | reflection code << 14: stage, filter order
    const int *hptr, *halo;     // tile halos of the reverse stream
    int hmax;
    const double *wx, *wy, *wl, *wh;  // owners' weights: wx wy wl in the stage order, wh in the filter's
    const double *tvol;         // filter transpose of the volumes (mass correction)
    const double *gsx, *gsy, *lsum, *hsum;
    Fields cur;                 // input state of the stage whose stencils are transposed
    Fields prev;                // input state of the stage whose pointwise reverse follows
    const double *gprev;        // that stage's recorded stencil sums (18 arrays of npfb)
    const double2 *gb_in;       // g_bar of the transposed stage (9 pair arrays of npfb)
    double2 *gb_out;            // g_bar of the stage whose pointwise reverse follows
    double *sb[kAdjS];          // the state's own adjoint from the pointwise reverse
    double *sbar[kAdjS];        // S_bar, the adjoint of the RK register
    double *ua[kAdjS];          // U_bar of a step's input state
    double *tacc;               // per-tile sums of the parameter adjoint (Wi, beta)
    double *rpart;              // per-tile sums of rho_bar of ua
    const double *tv;           // sum of the volumes
    double dt, alpha, beta;     // RK coefficients of the stage whose pointwise reverse follows
    int first;                  // that stage is the log-conformation first step (itime 1, stage 0)
    int mcorr;
};

// g_bar as 9 pair arrays, so the transposed gather reads 16 bytes a load:
//   0 (ro_x, ro_y)  1 (u_x, u_y)  2 (v_x, v_y)  3 (lap u, lap v)  4 (cxx_x, cyy_y)
//   5 (cxy_x, cxy_y)  6 (pxx_x, pxx_y)  7 (pxy_x, pxy_y)  8 (pyy_x, pyy_y)
constexpr int kAdjPairs = 9;

__device__ __forceinline__ void store_gbar(double2 *out, int n, int j, const double *gb) {
    out[j] = make_double2(gb[G_RO_X], gb[G_RO_Y]);
    out[(size_t)n + j] = make_double2(gb[G_U_X], gb[G_U_Y]);
    out[2 * (size_t)n + j] = make_double2(gb[G_V_X], gb[G_V_Y]);
    out[3 * (size_t)n + j] = make_double2(gb[G_LAPU], gb[G_LAPV]);
    out[4 * (size_t)n + j] = make_double2(gb[G_CXX_X], gb[G_CYY_Y]);
    out[5 * (size_t)n + j] = make_double2(gb[G_CXY_X], gb[G_CXY_Y]);
    out[6 * (size_t)n + j] = make_double2(gb[G_PXX_X], gb[G_PXX_Y]);
    out[7 * (size_t)n + j] = make_double2(gb[G_PXY_X], gb[G_PXY_Y]);
    out[8 * (size_t)n + j] = make_double2(gb[G_PYY_X], gb[G_PYY_Y]);
}

// Sums over the block's threads in a fixed tree (a, b: two sums at once).
__device__ __forceinline__ void tile_sum2(double &a, double &b) {
    __shared__ double red[2][kTile];
    red[0][threadIdx.x] = a;
    red[1][threadIdx.x] = b;
    __syncthreads();
    for (int st = kTile / 2; st > 0; st >>= 1) {
        if ((int)threadIdx.x < st) {
            red[0][threadIdx.x] = red[0][threadIdx.x] + red[0][threadIdx.x + st];
            red[1][threadIdx.x] = red[1][threadIdx.x] + red[1][threadIdx.x + st];
        }
        __syncthreads();
    }
    a = red[0][0];
    b = red[1][0];
    __syncthreads();
}

// Pointwise reverse of a stage at node j, given U_bar of its output ub: R_bar = dt (alpha
// U_bar + beta S_bar), S_bar <- U_bar + S_bar (sbar_zero: S_bar of the output is zero), then
// adjoint.cuh's reverse of the right-hand side at the recorded state and stencil sums.
__device__ __forceinline__ void point_reverse(const RevArgs &B, int j, const double *ub, bool sbar_zero, double &t0,
                                              double &t1) {
    const StepConsts &cK = B.K;
    const int n = cK.npfb;
    // every load before the first store (the arrays are not known to be distinct, and each
    // load after a store would wait out the one before)
    double si[kAdjR];
#pragma unroll
    for (int f = 0; f < kAdjR; f++) si[f] = sbar_zero ? 0.0 : B.sbar[f][j];
    const Fields &P = B.prev;
    const double s[kAdjS] = {P.ro[j], P.rou[j], P.rov[j], P.q[0][j], P.q[1][j], P.q[2][j]};
    double g[kAdjG], gbv[kAdjG], sbv[kAdjS] = {0, 0, 0, 0, 0, 0}, tb[2] = {0.0, 0.0};
#pragma unroll
    for (int k = 0; k < kAdjG; k++) {
        g[k] = B.gprev[(size_t)k * n + j];
        gbv[k] = 0.0;
    }
    double rb[kAdjR];
#pragma unroll
    for (int f = 0; f < kAdjR; f++) {
        rb[f] = B.dt * (B.alpha * ub[f] + B.beta * si[f]);
        B.sbar[f][j] = ub[f] + si[f];
    }
    p_adjoint_lc(cK, s, g, B.first != 0, rb, sbv, gbv, tb);
    store_gbar(B.gb_out, n, j, gbv);
#pragma unroll
    for (int k = 0; k < kAdjS; k++) B.sb[k][j] = sbv[k];
    t0 += tb[0];
    t1 += tb[1];
}

// Stage a tile's reverse halo: NA arrays of T per node (T = double2: the g_bar pairs).
template <int NA, typename T, typename SRC>
__device__ __forceinline__ void load_rev_halo(const RevArgs &B, T *sm, SRC src) {
    const int hb = B.hptr[blockIdx.x], hn = B.hptr[blockIdx.x + 1] - hb;
    const int hm = B.hmax;
    for (int h = threadIdx.x; h < hn; h += blockDim.x) {
        const int node = __ldg(B.halo + hb + h);
#pragma unroll
        for (int a = 0; a < NA; a++) cp_async<sizeof(T)>(&sm[a * hm + h], src(a) + node);
    }
    cp_async_commit();
    cp_async_wait<0>();
    __syncthreads();
}

__host__ __device__ constexpr size_t rev_stage_smem(int hmax) {
    return (size_t)2 * kAdjPairs * hmax * sizeof(double) + LinkRing<false, 3, ring_depth(false)>::bytes();
}
__host__ __device__ inline size_t rev_filter_smem(int hmax) {
    return halo_doubles(kAdjS, hmax) * sizeof(double) + LinkRing<false, 1, ring_depth(false)>::bytes();
}

// Reverse of the filter and the mass correction (rhs_lc.F90:818-893), fused with the
// pointwise reverse of stage 3.  The filter's output is Uf_j = U4_j (1 - hsum_j) + sum_k
// w_jk U4_k; the mass correction subtracts vol_i (sum_k rho_f,k vol_k - M) / sum(vol) from
// rho, so rho_f_bar_i = rho_bar_i - vol_i sum(rho_bar) / sum(vol), and
// U4_bar_j = Uf_bar_j (1 - hsum_j) + sum over reverse links w_ij Uf_bar_i, whose rho part
// is (filter^T rho_bar)_j - tvol_j sum(rho_bar) / sum(vol).
__global__ void __launch_bounds__(kTile, 2) k_adj_filter_lc(RevArgs B) {
    const StepConsts &cK = B.K;
    extern __shared__ __align__(16) double smem[];
    const int n = cK.npfb;
    const int j = blockIdx.x * kTile + threadIdx.x;
    const bool in_slice = (j >> 5) < cK.nslices;
    LinkRing<false, 1, ring_depth(false)> R;
    R.src[0] = reinterpret_cast<const double2 *>(B.wh);
    R.init(smem + halo_doubles(kAdjS, B.hmax), reinterpret_cast<const unsigned *>(B.locf),
           in_slice ? (B.sptr[j >> 5] >> 1) + (j & 31) : 0, in_slice ? B.sw[j >> 5] >> 1 : 0);
    R.prologue();
    load_rev_halo<kAdjS>(B, smem, [&](int f) { return (const double *)B.ua[f]; });
    // sum of rho_bar over all tiles, in the same order in every block
    double rs = 0.0, dummy = 0.0;
    for (int b = threadIdx.x; b < (int)gridDim.x; b += kTile) rs = rs + B.rpart[b];
    tile_sum2(rs, dummy);
    const double mc = B.mcorr ? rs / *B.tv : 0.0;
    const int hm = B.hmax;
    const bool mir = cK.has_mirrors;
    double acc[kAdjS] = {0, 0, 0, 0, 0, 0};
    auto link = [&](int lk, double w) {
        const int h = lk & kLocMask;
        double a1 = smem[hm + h], a2 = smem[2 * hm + h], a4 = smem[4 * hm + h];
        if (mir) {
            const int code = lk >> 14;
            if (code == 1 || code == 3) a1 = -a1;
            if (code == 2 || code == 3) a2 = -a2;
            if (code == 1 || code == 2) a4 = -a4;
        }
        acc[0] = __fma_rn(w, smem[h], acc[0]);
        acc[1] = __fma_rn(w, a1, acc[1]);
        acc[2] = __fma_rn(w, a2, acc[2]);
        acc[3] = __fma_rn(w, smem[3 * hm + h], acc[3]);
        acc[4] = __fma_rn(w, a4, acc[4]);
        acc[5] = __fma_rn(w, smem[5 * hm + h], acc[5]);
    };
    for (int m = 0; m < R.npair; m++) {
        R.next(m);
        double w0, w1;
        R.weights(m, 0, w0, w1);
        const unsigned l2 = R.index(m);
        link((int)(l2 & 0xffffu), w0);
        link((int)(l2 >> 16), w1);
    }
    double t0 = 0.0, t1 = 0.0;
    if (in_slice && j < n) {
        const double own = 1.0 - B.hsum[j];
#pragma unroll
        for (int f = 0; f < kAdjS; f++) acc[f] = __fma_rn(own, B.ua[f][j], acc[f]);
        acc[0] = acc[0] - mc * B.tvol[j];
        point_reverse(B, j, acc, true, t0, t1);
    }
    tile_sum2(t0, t1);
    if (threadIdx.x == 0) {
        B.tacc[2 * blockIdx.x] += t0;
        B.tacc[2 * blockIdx.x + 1] += t1;
    }
}

// Transposed stencils of stage s (the small links): node j collects w_ij g_bar_i from the
// owners i of its reverse links and -sum_k w_jk g_bar_j from its own, then reverses the
// derived fields (u = rho u / rho, v, c from psi) into the conservative state:
// U_bar_s = s_bar_s + that.  FUSE: the pointwise reverse of stage s - 1 follows (s > 0);
// otherwise (s = 0) U_bar_0 + S_bar_0 is the adjoint of the step's input.
template <bool FUSE>
__global__ void __launch_bounds__(kTile, 2) k_adj_stage_lc(RevArgs B) {
    const StepConsts &cK = B.K;
    extern __shared__ __align__(16) double smem[];
    const int n = cK.npfb;
    const int j = blockIdx.x * kTile + threadIdx.x;
    const bool in_slice = (j >> 5) < cK.nslices;
    double2 *sm = reinterpret_cast<double2 *>(smem);
    LinkRing<false, 3, ring_depth(false)> R;
    R.src[0] = reinterpret_cast<const double2 *>(B.wx);
    R.src[1] = reinterpret_cast<const double2 *>(B.wy);
    R.src[2] = reinterpret_cast<const double2 *>(B.wl);
    R.init(smem + 2 * (size_t)kAdjPairs * B.hmax, reinterpret_cast<const unsigned *>(B.locs),
           in_slice ? (B.sptr[j >> 5] >> 1) + (j & 31) : 0, in_slice ? B.sws[j >> 5] >> 1 : 0);
    R.prologue();
    load_rev_halo<kAdjPairs>(B, sm, [&](int p) { return B.gb_in + (size_t)p * n; });
    const int hm = B.hmax;
    const bool mir = cK.has_mirrors;
    // rho, u, v, cxx, cxy, cyy, psixx, psixy, psiyy
    double ph0 = 0, ph1 = 0, ph2 = 0, ph3 = 0, ph4 = 0, ph5 = 0, ph6 = 0, ph7 = 0, ph8 = 0;
    auto link = [&](int lk, double wx, double wy, double wl) {
        const int h = lk & kLocMask;
        const double2 a = sm[h], gu = sm[hm + h], gv = sm[2 * hm + h], lp = sm[3 * hm + h], c1 = sm[4 * hm + h];
        const double2 c2 = sm[5 * hm + h], p0 = sm[6 * hm + h], p1 = sm[7 * hm + h], p2 = sm[8 * hm + h];
        double tu = __fma_rn(wx, gu.x, __fma_rn(wy, gu.y, wl * lp.x));
        double tv = __fma_rn(wx, gv.x, __fma_rn(wy, gv.y, wl * lp.y));
        double txy = __fma_rn(wx, c2.x, wy * c2.y);
        double tpxy = __fma_rn(wx, p1.x, wy * p1.y);
        if (mir) {
            const int code = lk >> 14;
            if (code == 1 || code == 3) tu = -tu;
            if (code == 2 || code == 3) tv = -tv;
            if (code == 1 || code == 2) { txy = -txy; tpxy = -tpxy; }
        }
        ph0 = __fma_rn(wx, a.x, __fma_rn(wy, a.y, ph0));
        ph1 = ph1 + tu;
        ph2 = ph2 + tv;
        ph3 = __fma_rn(wx, c1.x, ph3);
        ph4 = ph4 + txy;
        ph5 = __fma_rn(wy, c1.y, ph5);
        ph6 = __fma_rn(wx, p0.x, __fma_rn(wy, p0.y, ph6));
        ph7 = ph7 + tpxy;
        ph8 = __fma_rn(wx, p2.x, __fma_rn(wy, p2.y, ph8));
    };
    for (int m = 0; m < R.npair; m++) {
        R.next(m);
        double wx0, wx1, wy0, wy1, wl0, wl1;
        R.weights(m, 0, wx0, wx1);
        R.weights(m, 1, wy0, wy1);
        R.weights(m, 2, wl0, wl1);
        const unsigned l2 = R.index(m);
        link((int)(l2 & 0xffffu), wx0, wy0, wl0);
        link((int)(l2 >> 16), wx1, wy1, wl1);
    }
    double t0 = 0.0, t1 = 0.0;
    if (in_slice && j < n) {
        const double gx = B.gsx[j], gy = B.gsy[j], ls = B.lsum[j];
        const double2 *G = B.gb_in;
        const double2 a = G[j], gu = G[(size_t)n + j], gv = G[2 * (size_t)n + j], lp = G[3 * (size_t)n + j];
        const double2 c1 = G[4 * (size_t)n + j], c2 = G[5 * (size_t)n + j], p0 = G[6 * (size_t)n + j];
        const double2 p1 = G[7 * (size_t)n + j], p2 = G[8 * (size_t)n + j];
        ph0 = ph0 - __fma_rn(gx, a.x, gy * a.y);
        ph1 = ph1 - __fma_rn(gx, gu.x, __fma_rn(gy, gu.y, ls * lp.x));
        ph2 = ph2 - __fma_rn(gx, gv.x, __fma_rn(gy, gv.y, ls * lp.y));
        ph3 = ph3 - gx * c1.x;
        ph4 = ph4 - __fma_rn(gx, c2.x, gy * c2.y);
        ph5 = ph5 - gy * c1.y;
        ph6 = ph6 - __fma_rn(gx, p0.x, gy * p0.y);
        ph7 = ph7 - __fma_rn(gx, p1.x, gy * p1.y);
        ph8 = ph8 - __fma_rn(gx, p2.x, gy * p2.y);
        const Fields &F = B.cur;
        const double ooro = 1.0 / F.ro[j];
        const double u = F.rou[j] * ooro, v = F.rov[j] * ooro;
        double pb[3] = {0.0, 0.0, 0.0};
        const double cb[3] = {ph3, ph4, ph5};
        lc_c_from_psi_adj(F.q[0][j], F.q[1][j], F.q[2][j], cb, pb);
        double U[kAdjS];
        U[0] = B.sb[0][j] + ph0 - (ph1 * u + ph2 * v) * ooro;
        U[1] = B.sb[1][j] + ph1 * ooro;
        U[2] = B.sb[2][j] + ph2 * ooro;
        U[3] = B.sb[3][j] + ph6 + pb[0];
        U[4] = B.sb[4][j] + ph7 + pb[1];
        U[5] = B.sb[5][j] + ph8 + pb[2];
        if constexpr (FUSE) {
            point_reverse(B, j, U, false, t0, t1);
        } else {
            double sb[kAdjS];
#pragma unroll
            for (int f = 0; f < kAdjS; f++) sb[f] = B.sbar[f][j];
#pragma unroll
            for (int f = 0; f < kAdjS; f++) {
                const double x = U[f] + sb[f];
                B.ua[f][j] = x;
                if (f == 0) t0 = x;
            }
        }
    }
    tile_sum2(t0, t1);
    if (threadIdx.x == 0) {
        if constexpr (FUSE) {
            B.tacc[2 * blockIdx.x] += t0;
            B.tacc[2 * blockIdx.x + 1] += t1;
        } else {
            B.rpart[blockIdx.x] = t0;
        }
    }
}

// Adjoint of J = sum 1/2 rho |u|^2 vol at the final state, and its per-tile sums of rho_bar.
__global__ void __launch_bounds__(kTile) k_adj_objective(Fields F, const double *vol, RevArgs B) {
    const StepConsts &cK = B.K;
    const int i = blockIdx.x * kTile + threadIdx.x;
    double r = 0.0, dummy = 0.0;
    if (i < cK.npfb) {
        const double u = F.u[i], v = F.v[i], w = vol[i];
        r = -0.5 * (u * u + v * v) * w;
        B.ua[0][i] = r;
        B.ua[1][i] = u * w;
        B.ua[2][i] = v * w;
        for (int f = 3; f < kAdjS; f++) B.ua[f][i] = 0.0;
    }
    tile_sum2(r, dummy);
    if (threadIdx.x == 0) B.rpart[blockIdx.x] = r;
}

// The filter's transpose applied to the volumes: tvol_j = vol_j (1 - hsum_j) + sum over
// reverse links w_ij vol_i.
__global__ void k_adj_tvol(AdjArgs B, const double *vol, double *tvol) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= B.npfb) return;
    double acc = vol[j] * (1.0 - B.hsum[j]);
    for (long long e = B.rptr[j]; e < B.rptr[j + 1]; e++) acc += B.wh[B.rslot[e]] * vol[B.rnode[e]];
    tvol[j] = acc;
}

// The reverse streams' weights: the owner's weights at its forward SELL slot (-1: padding,
// weight 0), wx wy wl in the stage order, wh in the filter's.
__global__ void k_adj_stream_weights(long long L, const int *slot_s, const int *slot_f, const double *wx,
                                     const double *wy, const double *wl, const double *wh, double *ox,
                                     double *oy, double *ol, double *oh) {
    const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (e >= L) return;
    const int s = slot_s[e], f = slot_f[e];
    ox[e] = s < 0 ? 0.0 : wx[s];
    oy[e] = s < 0 ? 0.0 : wy[s];
    ol[e] = s < 0 ? 0.0 : wl[s];
    oh[e] = f < 0 ? 0.0 : wh[f];
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
    B.gsx = H->gsx; B.gsy = H->gsy; B.lsum = H->lsum; B.hsum = H->hsum;
    return B;
}

// The reverse link streams (host build from the CSR lists): node j's reverse links in sliced
// ELL over the forward's slices, tiles of kTileSlices slices with the sorted set of owners
// as their halo.  Two orders of the links, each dealt slot by slot so that the lanes reading
// the halo together meet distinct shared-memory banks (deal_slice_by_bank): the small links
// for the stage kernel's 16-byte loads (groups of 8 lanes), all links for the filter's
// 8-byte loads (groups of 16).  Then the owners' weights are gathered into those orders on
// the device, and the filter transpose of the volumes is formed.
static int adjoint_build_stream(Handle *H) {
    if (H->rv_sptr) return 0;
    const int n = H->npfb, nsl = H->nslices;
    std::vector<long long> rptr(n + 1);
    SUNSET_CUDA(H, cudaMemcpy(rptr.data(), H->rptr, (n + 1) * sizeof(long long), cudaMemcpyDeviceToHost));
    const long long ne = rptr[n];
    std::vector<int> rslot(ne), rnode(ne);
    std::vector<unsigned char> rcode(ne);
    SUNSET_CUDA(H, cudaMemcpy(rslot.data(), H->rslot, ne * sizeof(int), cudaMemcpyDeviceToHost));
    SUNSET_CUDA(H, cudaMemcpy(rnode.data(), H->rnode, ne * sizeof(int), cudaMemcpyDeviceToHost));
    SUNSET_CUDA(H, cudaMemcpy(rcode.data(), H->rcode, ne * sizeof(unsigned char), cudaMemcpyDeviceToHost));
    std::vector<long long> sptr(nsl + 1, 0);
    std::vector<int> sw(nsl), sws(nsl);
    for (int sl = 0; sl < nsl; sl++) {
        int w = 0, ws = 0;
        for (int j = sl * kSlice; j < std::min(n, (sl + 1) * kSlice); j++) {
            int c = 0;
            for (long long e = rptr[j]; e < rptr[j + 1]; e++) c += (rcode[e] & 4) ? 1 : 0;
            w = std::max(w, (int)(rptr[j + 1] - rptr[j]));
            ws = std::max(ws, c);
        }
        sw[sl] = (w + 1) & ~1;
        sws[sl] = (ws + 1) & ~1;
        sptr[sl + 1] = sptr[sl] + (long long)sw[sl] * kSlice;
    }
    const long long L = sptr[nsl];
    if (ne >= 0x7fffffffLL) return set_err(H, SUNSET_ERR_SCOPE, "too many links for the reverse stream");
    const int nt = (nsl + kTileSlices - 1) / kTileSlices;
    std::vector<int> slot_s(L, -1), slot_f(L, -1);
    std::vector<uint16_t> loc_s(L, 0), loc_f(L, 0), pos(ne);
    std::vector<std::vector<int>> halos(nt);
    unsigned nthr = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
    std::vector<std::thread> pool;
    for (unsigned w = 0; w < nthr; w++) {
        pool.emplace_back([&, w]() {
            std::vector<int> small[kSlice], large[kSlice], chosen;
            for (int t = (int)w; t < nt; t += (int)nthr) {
                std::vector<int> &hv = halos[t];
                const int j0 = t * kTileSlices * kSlice, j1 = std::min(n, (t + 1) * kTileSlices * kSlice);
                for (int j = j0; j < j1; j++)
                    for (long long e = rptr[j]; e < rptr[j + 1]; e++) hv.push_back(rnode[e]);
                std::sort(hv.begin(), hv.end());
                hv.erase(std::unique(hv.begin(), hv.end()), hv.end());
                for (int j = j0; j < j1; j++)
                    for (long long e = rptr[j]; e < rptr[j + 1]; e++) {
                        const int p = (int)(std::lower_bound(hv.begin(), hv.end(), rnode[e]) - hv.begin());
                        pos[e] = (uint16_t)((p & kLocMask) | ((rcode[e] & 3) << 14));
                    }
                for (int sl = t * kTileSlices; sl < std::min(nsl, (t + 1) * kTileSlices); sl++) {
                    int c[kSlice], c_s[kSlice];
                    // stage order: the small links
                    for (int lane = 0; lane < kSlice; lane++) {
                        const int j = sl * kSlice + lane;
                        small[lane].clear();
                        large[lane].clear();
                        if (j < n)
                            for (long long e = rptr[j]; e < rptr[j + 1]; e++)
                                if (rcode[e] & 4) small[lane].push_back((int)e);
                        c[lane] = c_s[lane] = (int)small[lane].size();
                    }
                    chosen.assign((size_t)sws[sl] * kSlice, -1);
                    deal_slice_by_bank(8, pos.data(), small, large, c_s, c, sws[sl], chosen.data());
                    for (int k = 0; k < sws[sl]; k++)
                        for (int lane = 0; lane < kSlice; lane++) {
                            const int e = chosen[k * kSlice + lane];
                            if (e < 0) continue;
                            const long long o = sell_at(sptr[sl], k, lane);
                            slot_s[o] = rslot[e];
                            loc_s[o] = pos[e];
                        }
                    // filter order: all links
                    for (int lane = 0; lane < kSlice; lane++) {
                        const int j = sl * kSlice + lane;
                        small[lane].clear();
                        if (j < n)
                            for (long long e = rptr[j]; e < rptr[j + 1]; e++) small[lane].push_back((int)e);
                        c[lane] = c_s[lane] = (int)small[lane].size();
                    }
                    chosen.assign((size_t)sw[sl] * kSlice, -1);
                    deal_slice_by_bank(16, pos.data(), small, large, c_s, c, sw[sl], chosen.data());
                    for (int k = 0; k < sw[sl]; k++)
                        for (int lane = 0; lane < kSlice; lane++) {
                            const int e = chosen[k * kSlice + lane];
                            if (e < 0) continue;
                            const long long o = sell_at(sptr[sl], k, lane);
                            slot_f[o] = rslot[e];
                            loc_f[o] = pos[e];
                        }
                }
            }
        });
    }
    for (auto &th : pool) th.join();
    std::vector<int> hptr(nt + 1, 0);
    int hmax = 0;
    for (int t = 0; t < nt; t++) {
        hptr[t + 1] = hptr[t] + (int)halos[t].size();
        hmax = std::max(hmax, (int)halos[t].size());
    }
    if (hmax > kLocMask + 1)
        return set_err(H, SUNSET_ERR_SCOPE, "reverse tile halo of %d nodes exceeds the 14-bit local index", hmax);
    std::vector<int> hall(std::max(1, hptr[nt]));
    for (int t = 0; t < nt; t++) std::copy(halos[t].begin(), halos[t].end(), hall.begin() + hptr[t]);
    int *dslot = nullptr;
    const size_t Lz = L ? (size_t)L : 1;
    if (dalloc(H, &H->rv_sptr, nsl + 1) || dalloc(H, &H->rv_sw, nsl) || dalloc(H, &H->rv_sws, nsl) ||
        dalloc(H, &H->rv_loc_s, Lz) || dalloc(H, &H->rv_loc_f, Lz) || dalloc(H, &H->rv_hptr, nt + 1) ||
        dalloc(H, &H->rv_halo, hall.size()) || dalloc(H, &H->rv_wx, Lz) || dalloc(H, &H->rv_wy, Lz) ||
        dalloc(H, &H->rv_wl, Lz) || dalloc(H, &H->rv_wh, Lz) || dalloc(H, &H->rv_tvol, n) || dalloc(H, &dslot, 2 * Lz))
        return SUNSET_ERR_NOMEM;
    SUNSET_CUDA(H, cudaMemcpy(H->rv_sptr, sptr.data(), (nsl + 1) * sizeof(long long), cudaMemcpyHostToDevice));
    SUNSET_CUDA(H, cudaMemcpy(H->rv_sw, sw.data(), nsl * sizeof(int), cudaMemcpyHostToDevice));
    SUNSET_CUDA(H, cudaMemcpy(H->rv_sws, sws.data(), nsl * sizeof(int), cudaMemcpyHostToDevice));
    SUNSET_CUDA(H, cudaMemcpy(H->rv_loc_s, loc_s.data(), L * sizeof(uint16_t), cudaMemcpyHostToDevice));
    SUNSET_CUDA(H, cudaMemcpy(H->rv_loc_f, loc_f.data(), L * sizeof(uint16_t), cudaMemcpyHostToDevice));
    SUNSET_CUDA(H, cudaMemcpy(H->rv_hptr, hptr.data(), (nt + 1) * sizeof(int), cudaMemcpyHostToDevice));
    SUNSET_CUDA(H, cudaMemcpy(H->rv_halo, hall.data(), hall.size() * sizeof(int), cudaMemcpyHostToDevice));
    SUNSET_CUDA(H, cudaMemcpy(dslot, slot_s.data(), L * sizeof(int), cudaMemcpyHostToDevice));
    SUNSET_CUDA(H, cudaMemcpy(dslot + Lz, slot_f.data(), L * sizeof(int), cudaMemcpyHostToDevice));
    H->rv_hmax = hmax;
    if (L)
        k_adj_stream_weights<<<(unsigned)((L + 255) / 256), 256, 0, H->stream>>>(
            L, dslot, dslot + Lz, H->wx, H->wy, H->wl, H->wh, H->rv_wx, H->rv_wy, H->rv_wl, H->rv_wh);
    AdjArgs A = adj_args(H);
    k_adj_tvol<<<(n + 127) / 128, 128, 0, H->stream>>>(A, H->vol, H->rv_tvol);
    SUNSET_CUDA(H, cudaGetLastError());
    SUNSET_CUDA(H, cudaStreamSynchronize(H->stream));
    dfree(H, dslot);
    return 0;
}

static RevArgs rev_args(Handle *H) {
    RevArgs B{};
    B.K = consts_of(H);
    B.sptr = H->rv_sptr; B.sw = H->rv_sw; B.sws = H->rv_sws;
    B.locs = H->rv_loc_s; B.locf = H->rv_loc_f;
    B.hptr = H->rv_hptr; B.halo = H->rv_halo; B.hmax = H->rv_hmax;
    B.wx = H->rv_wx; B.wy = H->rv_wy; B.wl = H->rv_wl; B.wh = H->rv_wh; B.tvol = H->rv_tvol;
    B.gsx = H->gsx; B.gsy = H->gsy; B.lsum = H->lsum; B.hsum = H->hsum;
    for (int k = 0; k < kAdjS; k++) {
        B.sb[k] = H->adj_sb[k];
        B.sbar[k] = H->adj_sbar[k];
        B.ua[k] = H->adj_ua[k];
    }
    B.tacc = H->adj_tacc;
    B.rpart = H->adj_rpart;
    B.tv = &H->dsc->tv;
    B.mcorr = H->cfg.mcorr;
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

// Captures the launches fn() makes on the handle's stream into *exec (replacing it).
template <class FN>
int capture_graph(Handle *H, cudaGraphExec_t *exec, FN fn) {
    if (*exec) { cudaGraphExecDestroy(*exec); *exec = nullptr; }
    cudaGraph_t g = nullptr;
    SUNSET_CUDA(H, cudaStreamBeginCapture(H->stream, cudaStreamCaptureModeThreadLocal));
    const int lrc = fn();
    const cudaError_t ce = cudaStreamEndCapture(H->stream, &g);
    if (lrc || ce != cudaSuccess) {  // the capture ended either way: drop what it recorded
        if (g) cudaGraphDestroy(g);
        if (lrc) return lrc;
        SUNSET_CUDA(H, ce);
    }
    const cudaError_t ie = cudaGraphInstantiate(exec, g, 0);
    cudaGraphDestroy(g);
    if (ie != cudaSuccess) *exec = nullptr;
    SUNSET_CUDA(H, ie);
    return 0;
}

int adjoint_run(Handle *H, double dt, int nsteps, int ckpt, double *J, double *dtheta, double *dU0) {
    if (H->cfg.form != SUNSET_FORM_LC)
        return set_err(H, SUNSET_ERR_SCOPE, "the adjoint is built for the log-conformation form");
    if (H->cfg.precision != SUNSET_FP64) return set_err(H, SUNSET_ERR_SCOPE, "the adjoint runs the FP64 step");
    if (H->nb > 0) return set_err(H, SUNSET_ERR_SCOPE, "the adjoint covers node sets without boundaries");
    if (H->cfg.vpid) return set_err(H, SUNSET_ERR_SCOPE, "the adjoint covers runs without the flow-rate controller");
    if (H->cfg.Mdiff != 0.0) return set_err(H, SUNSET_ERR_SCOPE, "the adjoint assumes Mdiff = 0");
    if (H->cfg.fenep) return set_err(H, SUNSET_ERR_SCOPE, "the adjoint covers Oldroyd-B and sPTT, not FENE-P");
    if (nsteps < 1 || ckpt < 1) return set_err(H, SUNSET_ERR_ARG, "nsteps and checkpoint_every must be positive");
    const int n = H->npfb;
    cudaStream_t st = H->stream;
    if (int rc = adjoint_build_reverse(H)) return rc;
    if (int rc = adjoint_build_stream(H)) return rc;
    if (int rc = upload_consts(H)) return rc;
    const int nseg = (nsteps + ckpt - 1) / ckpt;
    const size_t smem_stage = rev_stage_smem(H->rv_hmax), smem_filter = rev_filter_smem(H->rv_hmax);
    if (smem_stage > kMaxStageSmem || smem_filter > kMaxStageSmem)
        return set_err(H, SUNSET_ERR_SCOPE, "reverse tile halo too large for shared memory");
    // storage: checkpoints (7 conservative fields), the recorded stages of one segment, scratch
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
        if (dalloc(H, &H->adj_g, (size_t)4 * ckpt * kAdjG * n) || dalloc(H, &H->adj_gp[0], (size_t)2 * kAdjPairs * n) ||
            dalloc(H, &H->adj_gp[1], (size_t)2 * kAdjPairs * n))
            return SUNSET_ERR_NOMEM;
        for (int k = 0; k < kAdjS; k++)
            if (dalloc(H, &H->adj_sb[k], n) || dalloc(H, &H->adj_sbar[k], n)) return SUNSET_ERR_NOMEM;
        for (int f = 0; f < 7; f++)
            if (dalloc(H, &H->adj_ua[f], n)) return SUNSET_ERR_NOMEM;
        if (dalloc(H, &H->adj_tacc, 2 * (size_t)H->ntiles) || dalloc(H, &H->adj_rpart, (size_t)H->ntiles) ||
            dalloc(H, &H->adj_acc, 4))
            return SUNSET_ERR_NOMEM;
        SUNSET_CUDA(H, cudaFuncSetAttribute(k_adj_stage_lc<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kMaxStageSmem));
        SUNSET_CUDA(H, cudaFuncSetAttribute(k_adj_stage_lc<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kMaxStageSmem));
        SUNSET_CUDA(H, cudaFuncSetAttribute(k_adj_filter_lc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kMaxStageSmem));
        H->adj_ready = true;
    }
    if (!H->adj_segd && dalloc(H, &H->adj_segd, 1)) return SUNSET_ERR_NOMEM;
    // a full segment's record and reverse sweep run as captured graphs (one launch each, so a
    // host thread that loses its core does not leave the device idle); they hold dt and the
    // checkpoint store, and are captured again when either changes
    if (H->adj_graph_dt != dt || H->adj_graph_cp != H->adj_cp) {
        for (cudaGraphExec_t *g : {&H->adj_rec_graph, &H->adj_rev_graph})
            if (*g) { cudaGraphExecDestroy(*g); *g = nullptr; }
        H->adj_graph_dt = dt;
        H->adj_graph_cp = H->adj_cp;
    }
    DevScalars sc0;
    SUNSET_CUDA(H, cudaMemcpyAsync(&sc0, H->dsc, sizeof(sc0), cudaMemcpyDeviceToHost, st));
    SUNSET_CUDA(H, cudaStreamSynchronize(st));
    k_set_dt<<<1, 1, 0, st>>>(H->dsc, dt);
    const int TB = 128, nb = (n + TB - 1) / TB;
    // Records len steps of the segment whose checkpoint index and start step k_set_segment has
    // set: stage inputs in adj_store[4 k + s], their stencil sums in adj_g, the state after the
    // segment in adj_store[4 ckpt + 1].
    auto record_launch = [&](int len) -> int {
        Fields &F0 = H->adj_store[0];
        k_load_checkpoint<<<nb, TB, 0, st>>>(n, SUNSET_FORM_LC, H->adj_cp, H->adj_segd, F0, consts_of(H));
        Fields &T = H->adj_store[4 * (size_t)ckpt], &X = H->adj_store[4 * (size_t)ckpt + 1];
        for (int k = 0; k < len; k++) {
            for (int s = 0; s < 4; s++) {
                StageArgs A = make_args_io(H, H->adj_store[4 * k + s], s < 3 ? H->adj_store[4 * k + s + 1] : T, s);
                A.gsave = H->adj_g + (size_t)(4 * k + s) * kAdjG * n;
                if (int rc = launch_stage_any(H, A, false)) return rc;
            }
            Fields &next = k + 1 < len ? H->adj_store[4 * (k + 1)] : X;
            StageArgs Fa = make_args_io(H, T, next, 5);
            if (int rc = launch_filter<SUNSET_FORM_LC>(H, Fa, false)) return rc;
            k_finalize<SUNSET_FORM_LC><<<nb, TB, 0, st>>>(Fa, 1);
        }
        SUNSET_CUDA(H, cudaGetLastError());
        return 0;
    };
    auto record = [&](int sg) -> int {
        const int n0 = sg * ckpt, len = std::min(ckpt, nsteps - n0);
        k_set_segment<<<1, 1, 0, st>>>(H->dsc, H->adj_segd, sg, sc0.itime + n0);
        if (len < ckpt) return record_launch(len);
        if (!H->adj_rec_graph)
            if (int rc = capture_graph(H, &H->adj_rec_graph, [&]() { return record_launch(ckpt); })) return rc;
        SUNSET_CUDA(H, cudaGraphLaunch(H->adj_rec_graph, st));
        return 0;
    };
    // ---- forward with checkpoints; the last segment is recorded as it runs ----
    for (int sg = 0; sg < nseg; sg++) {
        const Fields &F = H->buf[H->cur];
        double *cp = H->adj_cp + (size_t)7 * n * sg;
        double *src[7] = {F.ro, F.rou, F.rov, F.q[0], F.q[1], F.q[2], F.q[3]};
        for (int f = 0; f < 7; f++)
            SUNSET_CUDA(H, cudaMemcpyAsync(cp + (size_t)f * n, src[f], n * sizeof(double), cudaMemcpyDeviceToDevice, st));
        const int len = std::min(ckpt, nsteps - sg * ckpt);
        if (sg + 1 < nseg) {
            if (int rc = step_run(H, dt, len, 0)) return rc;
        } else {
            if (int rc = record(sg)) return rc;
            const Fields &X = H->adj_store[4 * (size_t)ckpt + 1];
            const Fields &D = H->buf[H->cur];
            const double *xs[13] = {X.ro, X.rou, X.rov, X.u, X.v, X.q[0], X.q[1], X.q[2], X.q[3],
                                    X.c[0], X.c[1], X.c[2], X.c[3]};
            double *ds[13] = {D.ro, D.rou, D.rov, D.u, D.v, D.q[0], D.q[1], D.q[2], D.q[3], D.c[0], D.c[1], D.c[2], D.c[3]};
            for (int f = 0; f < 13; f++)
                SUNSET_CUDA(H, cudaMemcpyAsync(ds[f], xs[f], n * sizeof(double), cudaMemcpyDeviceToDevice, st));
        }
    }
    if (int rc = set_tstep_device(H)) return rc;
    if (int rc = reduce_ke_mass(H, J, nullptr)) return rc;
    DevScalars scN;
    SUNSET_CUDA(H, cudaMemcpyAsync(&scN, H->dsc, sizeof(scN), cudaMemcpyDeviceToHost, st));
    SUNSET_CUDA(H, cudaStreamSynchronize(st));
    if (scN.err) return set_err(H, SUNSET_ERR_NONFINITE, "non-finite error norm in the forward run");
    // ---- reverse ----
    RevArgs B = rev_args(H);
    B.dt = dt;
    k_adj_objective<<<H->ntiles, kTile, 0, st>>>(H->buf[H->cur], H->vol, B);
    SUNSET_CUDA(H, cudaMemsetAsync(H->adj_tacc, 0, 2 * (size_t)H->ntiles * sizeof(double), st));
    const double alpha[4] = {SUNSET_RK_A21, SUNSET_RK_A32, SUNSET_RK_A43, SUNSET_RK_B4};
    const double beta[4] = {SUNSET_RK_B1, SUNSET_RK_B2, SUNSET_RK_B3, 0.0};
    auto gstage = [&](int k, int s) { return H->adj_g + (size_t)(4 * k + s) * kAdjG * n; };
    auto gpair = [&](int b) { return reinterpret_cast<double2 *>(H->adj_gp[b]); };
    // reverse sweep of len steps of the segment starting at step n0 (first: the itime = 1 case
    // of the log-conformation right-hand side may occur in it)
    auto reverse_launch = [&](int len, int n0, bool first) -> int {
        for (int k = len - 1; k >= 0; k--) {
            // filter + mass correction reversed, then the pointwise reverse of stage 3
            B.prev = H->adj_store[4 * k + 3];
            B.gprev = gstage(k, 3);
            B.gb_out = gpair(0);
            B.alpha = alpha[3];
            B.beta = beta[3];
            B.first = 0;
            k_adj_filter_lc<<<H->ntiles, kTile, smem_filter, st>>>(B);
            int cur = 0;
            for (int s = 3; s >= 1; s--) {  // stencils of stage s, pointwise reverse of stage s - 1
                B.cur = H->adj_store[4 * k + s];
                B.gb_in = gpair(cur);
                B.gb_out = gpair(cur ^ 1);
                B.prev = H->adj_store[4 * k + s - 1];
                B.gprev = gstage(k, s - 1);
                B.alpha = alpha[s - 1];
                B.beta = beta[s - 1];
                B.first = first && (s == 1) && (sc0.itime + n0 + k == 1);
                k_adj_stage_lc<true><<<H->ntiles, kTile, smem_stage, st>>>(B);
                cur ^= 1;
            }
            B.cur = H->adj_store[4 * k];
            B.gb_in = gpair(cur);
            k_adj_stage_lc<false><<<H->ntiles, kTile, smem_stage, st>>>(B);
        }
        SUNSET_CUDA(H, cudaGetLastError());
        return 0;
    };
    for (int sg = nseg - 1; sg >= 0; sg--) {
        const int n0 = sg * ckpt, len = std::min(ckpt, nsteps - n0);
        if (sg + 1 < nseg)
            if (int rc = record(sg)) return rc;
        const int k1 = 1 - sc0.itime - n0;  // the segment's step with itime = 1, if any
        if (len < ckpt || (k1 >= 0 && k1 < len)) {
            if (int rc = reverse_launch(len, n0, true)) return rc;
            continue;
        }
        if (!H->adj_rev_graph)
            if (int rc = capture_graph(H, &H->adj_rev_graph, [&]() { return reverse_launch(ckpt, 0, false); })) return rc;
        SUNSET_CUDA(H, cudaGraphLaunch(H->adj_rev_graph, st));
    }
    SUNSET_CUDA(H, cudaGetLastError());
    k_adj_fold<<<1, 128, 0, st>>>(H->adj_tacc, H->ntiles, 2, H->adj_acc, 0);
    double acc[2];
    SUNSET_CUDA(H, cudaMemcpyAsync(acc, H->adj_acc, 2 * sizeof(double), cudaMemcpyDeviceToHost, st));
    for (int f = 0; f < kAdjS; f++)
        SUNSET_CUDA(H, cudaMemcpyAsync(dU0 + (size_t)f * n, H->adj_ua[f], n * sizeof(double), cudaMemcpyDeviceToDevice, st));
    SUNSET_CUDA(H, cudaMemsetAsync(dU0 + (size_t)6 * n, 0, n * sizeof(double), st));
    // the handle keeps the final state and its time
    SUNSET_CUDA(H, cudaMemcpyAsync(H->dsc, &scN, sizeof(scN), cudaMemcpyHostToDevice, st));
    SUNSET_CUDA(H, cudaStreamSynchronize(st));
    dtheta[0] = acc[0];
    dtheta[1] = acc[1];
    return 0;
}

}  // namespace sunset
