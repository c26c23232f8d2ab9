// noalloc.cu -- kinetic energy and mass of a state without any device allocation.
//
// sunset_kinetic_energy() reduces the handle's state through per-block partial sums kept
// in a buffer the handle allocated.  Some callers cannot allocate device memory at all:
// host codes whose arrays live in their own device pool (a Fortran code with CUDA
// Fortran/OpenACC-managed arrays) and that must not call cudaMalloc, because it can
// synchronise the whole device and fails outright under a memory cap.  They hand over
// device arrays they already own and get the two sums back in a device array they own.
//
// The partial sums live in a file-scope __device__ array of kNoAllocMaxBlocks pairs
// (256 KB, held by every GPU that loads the library until the process exits).  Host code
// may not use the array's name as an address: it is a host-side stand-in, and a kernel
// given it would fault or, where the GPU can reach host memory, read the wrong memory.
// The device address is looked up once per device with cudaGetSymbolAddress, on the
// first call made on that device (so that first call should come before any stream
// capture), and passed to the kernels.  Every call shares the array: two calls whose
// kernels overlap on the GPU (different streams, or different host threads) race on it.
//
// The call leaves the calling thread's current device as it found it, and reports only
// its own launch errors: each kernel goes through cudaLaunchKernel, whose return value is
// that launch's status, so an error the caller left pending is neither consumed nor
// reported here.
#include <mutex>

#include "internal.cuh"

namespace sunset {
namespace {

constexpr int kNoAllocThreads = 256;
constexpr int kNoAllocMaxBlocks = 16384;  // => at most 256 * 16384 = 4,194,304 nodes
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double g_noalloc_partials[2 * kNoAllocMaxBlocks];

std::mutex g_mutex;
double *g_scratch[kMaxDevices] = {};

// Per block: fixed-tree sums of 0.5 rho |u|^2 vol and rho vol (the expressions of
// sunset_kinetic_energy), written to partials[2b], partials[2b+1].
__global__ void __launch_bounds__(kNoAllocThreads) k_ke_mass_partials(int n, const double *ro, const double *u,
                                                                      const double *v, const double *vol,
                                                                      double *partials) {
    __shared__ double s1[kNoAllocThreads], s2[kNoAllocThreads];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double ke = 0.0, m = 0.0;
    if (i < n) {
        ke = ((0.5 * ro[i]) * (u[i] * u[i] + v[i] * v[i])) * vol[i];
        m = ro[i] * vol[i];
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

// One block folds the nb partial pairs (strided per thread, then a fixed tree).
__global__ void __launch_bounds__(kNoAllocThreads) k_ke_mass_fold(const double *partials, int nb, double *out) {
    __shared__ double s1[kNoAllocThreads], s2[kNoAllocThreads];
    double a = 0.0, b = 0.0;
    for (int k = threadIdx.x; k < nb; k += blockDim.x) {
        a = a + partials[2 * k];
        b = b + partials[2 * k + 1];
    }
    s1[threadIdx.x] = a;
    s2[threadIdx.x] = b;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) {
            s1[threadIdx.x] = s1[threadIdx.x] + s1[threadIdx.x + s];
            s2[threadIdx.x] = s2[threadIdx.x] + s2[threadIdx.x + s];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        out[0] = s1[0];
        out[1] = s2[0];
    }
}

}  // namespace
}  // namespace sunset

using namespace sunset;

extern "C" int sunset_kinetic_energy_noalloc(int device, int npfb, const double *ro, const double *u,
                                             const double *v, const double *vol, double *out, void *stream) {
    if (npfb <= 0 || !ro || !u || !v || !vol || !out) return SUNSET_ERR_ARG;
    if (npfb > kNoAllocThreads * kNoAllocMaxBlocks) return SUNSET_ERR_SCOPE;  // beyond the static scratch
    if (device < 0 || device >= kMaxDevices) return SUNSET_ERR_ARG;
    int prev = -1;
    if (cudaGetDevice(&prev) != cudaSuccess) return SUNSET_ERR_CUDA;
    struct Restore {  // the caller's current device again on every return path
        int dev;
        ~Restore() { cudaSetDevice(dev); }
    } restore{prev};
    if (device != prev && cudaSetDevice(device) != cudaSuccess) return SUNSET_ERR_CUDA;
    double *scratch;
    {
        std::lock_guard<std::mutex> lock(g_mutex);
        if (!g_scratch[device]) {
            void *p = nullptr;
            if (cudaGetSymbolAddress(&p, g_noalloc_partials) != cudaSuccess || !p) return SUNSET_ERR_CUDA;
            g_scratch[device] = static_cast<double *>(p);
        }
        scratch = g_scratch[device];
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    int n = npfb, nb = (npfb + kNoAllocThreads - 1) / kNoAllocThreads;
    // every partial the fold reads is written by this call first: nothing has to start at zero
    void *pa[] = {&n, &ro, &u, &v, &vol, &scratch};
    if (cudaLaunchKernel((const void *)k_ke_mass_partials, dim3(nb), dim3(kNoAllocThreads), pa, 0, st) != cudaSuccess)
        return SUNSET_ERR_CUDA;
    void *fa[] = {&scratch, &nb, &out};
    if (cudaLaunchKernel((const void *)k_ke_mass_fold, dim3(1), dim3(kNoAllocThreads), fa, 0, st) != cudaSuccess)
        return SUNSET_ERR_CUDA;
    return SUNSET_OK;
}
