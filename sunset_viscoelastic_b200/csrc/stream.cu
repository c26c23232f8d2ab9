// stream.cu -- the link stream of the time step: bank-aware link order, and the weights the
// stage and filter kernels stream (FP64 copies, or packed fixed-point stage links and FP32
// filter weights for the mixed precision).
//
// The setup, the single-operator entry points and the weight export keep the reference's
// link order (derivatives.F90 sums over ij_link in order).  The time step sums each node's
// links in its own order instead, chosen for the hardware: the stage and filter kernels
// gather the tile halo from shared memory with 8-byte loads, which are served per
// half-warp, one wavefront per bank pair (position mod 16) and distinct position.  In the
// reference order neighbouring lanes often meet in the same bank pair at the same link slot
// (4.9 wavefronts a load on the order-6 set against the ideal 2).  order_links_by_bank()
// re-deals each node's links slot by slot so that the 16 lanes of a half-warp read distinct
// bank pairs wherever a bipartite matching allows it (2.6 on that set).  Only the rounding
// of the sums changes (relative 1e-16 a sum).
//
// Mixed precision: the weight solves stay FP64; the stage kernel streams each link as three
// 32-bit words, one per operator (d/dx, d/dy, Laplacian).  A word is the integer 64 q + b:
// q the weight rounded to a 26-bit integer in units of a power of two per node and operator
// (2^(e-25), e the exponent of the node's largest |w| of that operator), b six bits of the
// link's 16-bit local index (bits 0-5, 6-11 and 12-15 of the index in the x, y and
// Laplacian words).  The stage masks b off and converts 64 q to FP32.  That is 12 bytes a
// link against 26 in FP64 (16-bit index + three doubles), with 25 bits relative to the node's
// largest weight; the stage sums in difference form, sum_k w_k (phi_j - phi_i), so a
// constant field keeps zero derivatives whatever the rounding.  (Converting the whole word,
// index bits included, saves the masks but adds b to 64 q: a perturbation of up to one
// unit of q that is not zero-mean -- the Laplacian word's bits are 0 for halos under 4096
// nodes -- and acts as a small extra Laplacian, 1e-6 of the fields in 100 steps.)
// The filter streams its weight rounded to FP32 with the local index (6 bytes a link).
#include <algorithm>
#include <thread>
#include <vector>

#include "internal.cuh"

namespace sunset {

namespace {

struct StreamArgs {
    int npfb;
    const long long *slice_ptr;
    const int *slice_w;
    const int *src;  // SELL entry -> SELL entry of the reference-order arrays it takes (-1: padding)
    const uint16_t *lloc;
    const double *wx, *wy, *wl, *wh;
    uint16_t *lloc_s;
    double *wx_s, *wy_s, *wl_s, *wh_s;      // FP64 step
    unsigned *pk;                           // mixed step: packed stage links (pk_at)
    float *scx, *scy, *scl;                 // their per-node scales
    unsigned *wf;                           // mixed filter (wf_at)
};

constexpr int kPackBits = 26;  // bits of a packed stage weight (sign included)

// Exponent e with max|w| < 2^e (0 for an all-zero operator row).
__device__ __forceinline__ int pack_exponent(double wmax) {
    int e = 0;
    if (wmax > 0.0) frexp(wmax, &e);
    return e;
}
// A weight as the word 64 q + b: q its kPackBits-bit integer in units of
// 2^(e - kPackBits + 1), b six index bits.
__device__ __forceinline__ unsigned pack_weight(double w, int e, unsigned idx6) {
    const long long lim = (1ll << (kPackBits - 1)) - 1;
    long long q = llrint(ldexp(w, kPackBits - 1 - e));
    q = q > lim ? lim : (q < -lim ? -lim : q);
    return ((unsigned)(int)q << 6) | (idx6 & 63u);
}

// One thread per node: gather its links into the stream order; MX: pack the stage weights
// with the node's scales, round the filter weights to FP32 and sum those.  Padding entries
// keep weight 0 and local index 0.
template <bool MX>
__global__ void k_stream_weights(StreamArgs a) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.npfb) return;
    const long long base = a.slice_ptr[i >> 5];
    const int lane = i & 31;
    const int w = a.slice_w[i >> 5];
    int ex = 0, ey = 0, el = 0;
    if constexpr (MX) {
        double mx = 0.0, my = 0.0, ml = 0.0;
        for (int k = 0; k < w; k++) {
            const int q = a.src[sell_at(base, k, lane)];
            if (q < 0) continue;
            mx = fmax(mx, fabs(a.wx[q]));
            my = fmax(my, fabs(a.wy[q]));
            ml = fmax(ml, fabs(a.wl[q]));
        }
        ex = pack_exponent(mx);
        ey = pack_exponent(my);
        el = pack_exponent(ml);
        a.scx[i] = ldexpf(1.0f, ex - (kPackBits - 1) - 6);  // a word's value is 64 q
        a.scy[i] = ldexpf(1.0f, ey - (kPackBits - 1) - 6);
        a.scl[i] = ldexpf(1.0f, el - (kPackBits - 1) - 6);
    }
    // the packed words of a padding slot point at the node itself (its first link in the
    // reference order, distance 0), so even a nonzero weight there would meet phi_i - phi_i
    const unsigned self_loc = a.lloc[sell_at(base, 0, lane)];
    for (int k = 0; k < w; k++) {
        const long long o = sell_at(base, k, lane);
        const int q = a.src[o];
        const unsigned loc = q < 0 ? 0u : a.lloc[q];
        a.lloc_s[o] = (uint16_t)loc;
        if constexpr (MX) {
            const unsigned ploc = q < 0 ? self_loc : loc;
            unsigned *pw = a.pk + pk_at(base, k, lane);
            pw[0] = pack_weight(q < 0 ? 0.0 : a.wx[q], ex, ploc);
            pw[1] = pack_weight(q < 0 ? 0.0 : a.wy[q], ey, ploc >> 6);
            pw[2] = pack_weight(q < 0 ? 0.0 : a.wl[q], el, ploc >> 12);
            unsigned *fw = a.wf + wf_at(base, k >> 1, lane);
            fw[k & 1] = __float_as_uint(q < 0 ? 0.0f : (float)a.wh[q]);
            fw[2] = (k & 1) ? ((fw[2] & 0xffffu) | (loc << 16)) : ((fw[2] & 0xffff0000u) | loc);
        } else {
            a.wx_s[o] = q < 0 ? 0.0 : a.wx[q];
            a.wy_s[o] = q < 0 ? 0.0 : a.wy[q];
            a.wl_s[o] = q < 0 ? 0.0 : a.wl[q];
            a.wh_s[o] = q < 0 ? 0.0 : a.wh[q];
        }
    }
}

}  // namespace

// New SELL order of the links for the time step: src[o] = the SELL entry (in the reference
// order) whose link goes to entry o, or -1 for padding.  Small links stay in the slots
// [0, cnt_small) and the other links in [cnt_small, cnt), so the stage kernel (small links)
// and the filter (all links) see the same sets as in the reference order.
static int order_links_by_bank(Handle *H, std::vector<int> &src) {
    const int n = H->npfb, nsl = H->nslices;
    const long long L = H->nlinks_sell;
    std::vector<uint16_t> loc(L);
    std::vector<int> cnt(n), cs(n), sw(nsl);
    std::vector<long long> sptr(nsl + 1);
    SUNSET_CUDA(H, cudaMemcpy(loc.data(), H->lloc, L * sizeof(uint16_t), cudaMemcpyDeviceToHost));
    SUNSET_CUDA(H, cudaMemcpy(cnt.data(), H->cnt, n * sizeof(int), cudaMemcpyDeviceToHost));
    SUNSET_CUDA(H, cudaMemcpy(cs.data(), H->cnt_small, n * sizeof(int), cudaMemcpyDeviceToHost));
    SUNSET_CUDA(H, cudaMemcpy(sw.data(), H->slice_w, nsl * sizeof(int), cudaMemcpyDeviceToHost));
    SUNSET_CUDA(H, cudaMemcpy(sptr.data(), H->slice_ptr, (nsl + 1) * sizeof(long long), cudaMemcpyDeviceToHost));
    src.assign(L, -1);
    const unsigned nthr = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
    std::vector<std::thread> pool;
    for (unsigned w = 0; w < nthr; w++) {
        pool.emplace_back([&, w]() {
            std::vector<int> small[kSlice], large[kSlice];
            std::vector<int> chosen;
            for (int sl = (int)w; sl < nsl; sl += (int)nthr) {
                int c[kSlice], c_s[kSlice];
                for (int lane = 0; lane < kSlice; lane++) {
                    const int i = sl * kSlice + lane;
                    c[lane] = i < n ? cnt[i] : 0;
                    c_s[lane] = i < n ? std::min(cs[i], c[lane]) : 0;
                    small[lane].clear();
                    large[lane].clear();
                    for (int k = 0; k < c[lane]; k++)
                        (k < c_s[lane] ? small[lane] : large[lane]).push_back((int)sell_at(sptr[sl], k, lane));
                }
                chosen.assign((size_t)sw[sl] * kSlice, -1);
                deal_slice_by_bank(16, loc.data(), small, large, c_s, c, sw[sl], chosen.data());
                for (int k = 0; k < sw[sl]; k++)
                    for (int lane = 0; lane < kSlice; lane++)
                        if (chosen[k * kSlice + lane] >= 0) src[sell_at(sptr[sl], k, lane)] = chosen[k * kSlice + lane];
            }
        });
    }
    for (auto &th : pool) th.join();
    return 0;
}

// Called once the FP64 weights, their sums and the filter coefficients exist.
int make_stream_links(Handle *H) {
    const long long L = H->nlinks_sell;
    const int n = H->npfb;
    const bool mx = H->cfg.precision == SUNSET_MIXED;
    if (L >= (1ll << 31)) return set_err(H, SUNSET_ERR_SCOPE, "the link stream supports at most 2^31 link slots");
    if (!H->lloc_s) {
        if (dalloc(H, &H->lloc_s, L)) return SUNSET_ERR_NOMEM;
        if (mx) {
            if (dalloc(H, &H->pk, 3 * L) || dalloc(H, &H->wf, 3 * L / 2) || dalloc(H, &H->scx, n) ||
                dalloc(H, &H->scy, n) || dalloc(H, &H->scl, n))
                return SUNSET_ERR_NOMEM;
        } else {
            if (dalloc(H, &H->wx_s, L) || dalloc(H, &H->wy_s, L) || dalloc(H, &H->wl_s, L) || dalloc(H, &H->wh_s, L))
                return SUNSET_ERR_NOMEM;
        }
    }
    std::vector<int> src;
    if (int rc = order_links_by_bank(H, src)) return rc;
    int *d_src = nullptr;
    if (dalloc(H, &d_src, L)) return SUNSET_ERR_NOMEM;
    SUNSET_CUDA(H, cudaMemcpy(d_src, src.data(), L * sizeof(int), cudaMemcpyHostToDevice));
    StreamArgs a{n, H->slice_ptr, H->slice_w, d_src, H->lloc, H->wx, H->wy, H->wl, H->wh, H->lloc_s,
                 H->wx_s, H->wy_s, H->wl_s, H->wh_s, H->pk, H->scx, H->scy, H->scl, H->wf};
    if (mx) k_stream_weights<true><<<(n + 255) / 256, 256, 0, H->stream>>>(a);
    else k_stream_weights<false><<<(n + 255) / 256, 256, 0, H->stream>>>(a);
    SUNSET_CUDA(H, cudaGetLastError());
    SUNSET_CUDA(H, cudaStreamSynchronize(H->stream));
    dfree(H, d_src);
    return 0;
}

}  // namespace sunset
