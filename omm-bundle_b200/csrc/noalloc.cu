// mm_trace without any device allocation.
//
// msw_mm_dtrace / msw_mm_ztrace reduce sum_ij conj(A_ij) B_ij in two passes
// and keep the per-block partial sums in scratch that the library allocates
// (and grows) with cudaMalloc.  Some callers cannot let a library do that:
// applications whose own memory manager owns the device (a pool reserved at
// start-up that leaves nothing for other allocators), and tight loops where
// cudaMalloc's implicit device synchronisation is not acceptable.  This file
// gives them the same reduction with its scratch in a fixed device array
// that is part of the loaded library.
//
// Limits and sharing rules (also stated in include/ommgpu.h):
//   * the partial sums live in g_noalloc_partials, a file-scope __device__
//     array of OMM_NOALLOC_MAX_PARTIALS records; one record per block of
//     OMM_NOALLOC_ELEMS_PER_BLOCK elements, so at most
//     OMM_NOALLOC_MAX_PARTIALS * OMM_NOALLOC_ELEMS_PER_BLOCK elements per
//     call (larger inputs are rejected with OMM_ERR_ARG);
//   * every GPU that loads the library holds the array (1 MiB) until exit;
//   * all calls share it and it keeps the last call's contents; each call
//     writes every record it later reads, so nothing needs clearing, but two
//     calls that overlap on the same GPU (e.g. on two streams at once) race
//     on it.  Calls on different GPUs use different copies of the array;
//   * the host-side name of a __device__ array is not a device address, so
//     its address is taken with cudaGetSymbolAddress on the first call made
//     in a CUDA context (once per device, and again if the device's context
//     is replaced, e.g. after cudaDeviceReset).  That first call must
//     therefore come before any stream capture.
#include <cuda.h>
#include <cuda_runtime.h>

#include <mutex>

#include "ommgpu.h"

namespace {

constexpr int kThreads = 256;
constexpr int kPerThread = 8;
constexpr int kElemsPerBlock = OMM_NOALLOC_ELEMS_PER_BLOCK;
static_assert(kElemsPerBlock == kThreads * kPerThread, "block size and elements per block disagree");
constexpr int kMaxDevices = 64;

// two doubles (re, im) per partial record
static __device__ __align__(256) double g_noalloc_partials[2 * OMM_NOALLOC_MAX_PARTIALS];

// device address of the array per device, valid for the context it was looked up in (context
// ids are unique for the life of the process, so a replaced context is always noticed)
struct AddrCache {
    unsigned long long ctx_id = 0;
    double* addr = nullptr;
};
AddrCache g_partials_addr[kMaxDevices];
std::mutex g_addr_mutex;

typedef CUresult (*CtxGetCurrentFn)(CUcontext*);
typedef CUresult (*CtxGetIdFn)(CUcontext, unsigned long long*);
CtxGetCurrentFn g_ctx_get_current = nullptr;
CtxGetIdFn g_ctx_get_id = nullptr;
std::once_flag g_driver_once;

// the driver entry points that identify the current context (no -lcuda needed)
void load_driver_entry_points() {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
        g_ctx_get_current = (CtxGetCurrentFn)f;
    f = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
        g_ctx_get_id = (CtxGetIdFn)f;
}

// the scratch array's device address in the current context of device dev, looked up with
// cudaGetSymbolAddress the first time this context is seen; nullptr on failure
double* partials_address(int dev) {
    std::call_once(g_driver_once, load_driver_entry_points);
    if (!g_ctx_get_current || !g_ctx_get_id) return nullptr;
    CUcontext ctx = nullptr;
    unsigned long long id = 0;
    void* p = nullptr;
    if (g_ctx_get_current(&ctx) != CUDA_SUCCESS || !ctx) {
        // no context bound to this thread yet: the runtime call binds the device's primary context
        if (cudaGetSymbolAddress(&p, g_noalloc_partials) != cudaSuccess || !p) return nullptr;
        if (g_ctx_get_current(&ctx) != CUDA_SUCCESS || !ctx) return nullptr;
    }
    if (g_ctx_get_id(ctx, &id) != CUDA_SUCCESS) return nullptr;
    std::lock_guard<std::mutex> lock(g_addr_mutex);
    AddrCache& c = g_partials_addr[dev];
    if (c.addr && c.ctx_id == id) return c.addr;
    if (!p && (cudaGetSymbolAddress(&p, g_noalloc_partials) != cudaSuccess || !p)) return nullptr;
    c.ctx_id = id;
    c.addr = (double*)p;
    return c.addr;
}

thread_local const char* g_noalloc_error = "";

template <bool REAL>
__global__ void __launch_bounds__(kThreads) noalloc_dot_kernel(int rows, long long total, const double* __restrict__ A,
                                                             int lda, const double* __restrict__ B, int ldb,
                                                             double* __restrict__ partials) {
    double re = 0.0, im = 0.0;
    long long base = (long long)blockIdx.x * kElemsPerBlock;
#pragma unroll
    for (int q = 0; q < kPerThread; ++q) {
        long long e = base + (long long)q * kThreads + threadIdx.x;
        if (e < total) {
            long long i = e % rows, j = e / rows;
            if (REAL) {
                re += A[i + j * lda] * B[i + j * ldb];
            } else {
                const double* a = A + 2 * (i + j * lda);
                const double* b = B + 2 * (i + j * ldb);
                re += a[0] * b[0] + a[1] * b[1];  // conj(a) * b
                im += a[0] * b[1] - a[1] * b[0];
            }
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        re += __shfl_down_sync(0xffffffffu, re, o);
        im += __shfl_down_sync(0xffffffffu, im, o);
    }
    __shared__ double s_re[kThreads / 32], s_im[kThreads / 32];
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) {
        s_re[w] = re;
        s_im[w] = im;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double r = 0.0, m = 0.0;
        for (int k = 0; k < kThreads / 32; ++k) {
            r += s_re[k];
            m += s_im[k];
        }
        partials[2 * blockIdx.x] = r;  // every record read below is written here first
        partials[2 * blockIdx.x + 1] = m;
    }
}

// one block: Neumaier-compensated sum of nb records -> result[0..1]
__global__ void __launch_bounds__(kThreads) noalloc_final_kernel(const double* __restrict__ partials, int nb,
                                                               double* __restrict__ result) {
    __shared__ double s_sum[2][kThreads], s_cmp[2][kThreads];
    for (int k = 0; k < 2; ++k) {
        double s = 0.0, c = 0.0;
        for (int b = threadIdx.x; b < nb; b += kThreads) {
            double v = partials[2 * b + k], t = s + v;
            c += (fabs(s) >= fabs(v)) ? ((s - t) + v) : ((v - t) + s);
            s = t;
        }
        s_sum[k][threadIdx.x] = s;
        s_cmp[k][threadIdx.x] = c;
    }
    __syncthreads();
    if (threadIdx.x < 2) {
        int k = threadIdx.x;
        double S = 0.0, C = 0.0;
        for (int i = 0; i < kThreads; ++i) {
            double v = s_sum[k][i], t = S + v;
            C += (fabs(S) >= fabs(v)) ? ((S - t) + v) : ((v - t) + S);
            S = t;
            C += s_cmp[k][i];
        }
        result[k] = S + C;
    }
}

}  // namespace

extern "C" {

const char* omm_gpu_noalloc_last_error(void) { return g_noalloc_error; }

int omm_gpu_mm_trace_noalloc(int rows, int cols, const void* A, int lda, const void* B, int ldb, int is_complex,
                             double* result, void* stream) {
    if (rows < 0 || cols < 0 || (rows > 0 && (lda < rows || ldb < rows))) {
        g_noalloc_error = "mm_trace_noalloc: invalid dimensions or leading dimensions";
        return OMM_ERR_ARG;
    }
    if (!result || ((long long)rows * cols > 0 && (!A || !B))) {
        g_noalloc_error = "mm_trace_noalloc: null pointer";
        return OMM_ERR_ARG;
    }
    long long total = (long long)rows * cols;
    long long nb = (total + kElemsPerBlock - 1) / kElemsPerBlock;
    if (nb > OMM_NOALLOC_MAX_PARTIALS) {
        g_noalloc_error = "mm_trace_noalloc: rows*cols exceeds OMM_NOALLOC_MAX_ELEMS (the fixed scratch holds "
                          "OMM_NOALLOC_MAX_PARTIALS block sums)";
        return OMM_ERR_ARG;
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        g_noalloc_error = "mm_trace_noalloc: no usable current CUDA device";
        return OMM_ERR_CUDA;
    }
    // the device address of the scratch array in the current context (looked up on the first call
    // in each context, with that device current)
    double* partials = partials_address(dev);
    if (!partials) {
        g_noalloc_error = "mm_trace_noalloc: cudaGetSymbolAddress of the scratch array failed";
        return OMM_ERR_CUDA;
    }
    cudaStream_t s = (cudaStream_t)stream;
    if (nb > 0) {
        if (is_complex)
            noalloc_dot_kernel<false><<<(unsigned)nb, kThreads, 0, s>>>(rows, total, (const double*)A, lda,
                                                                       (const double*)B, ldb, partials);
        else
            noalloc_dot_kernel<true><<<(unsigned)nb, kThreads, 0, s>>>(rows, total, (const double*)A, lda,
                                                                      (const double*)B, ldb, partials);
    }
    noalloc_final_kernel<<<1, kThreads, 0, s>>>(partials, (int)nb, result);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        g_noalloc_error = "mm_trace_noalloc: kernel launch failed";
        return OMM_ERR_CUDA;
    }
    g_noalloc_error = "";
    return OMM_OK;
}

}  // extern "C"
