// Format conversions of the registration path:
//   * MatrixSwitch m_copy between dense and CSC storages, with the optional
//     hard / soft threshold (MatrixSwitch.F90:630-900, MatrixSwitch_m_copy.F90:
//     sdensdenref_thre :102-147, sdenscscref :495-551, sdenscscref_thre :553-629);
//   * pspBLAS psp_den2sp (pspBasicTool.F90:205-421: nonzeros, or |a| >= thre)
//     and psp_sp2den (:423-533);
//   * COO registration (psp_register_spm with 'coo' + psp_coo2csc,
//     pspMat.F90:87-140, pspBasicTool.F90:907-942).
// Dense -> CSC runs on the device: one CTA per column counts the kept entries,
// the column pointers are the prefix sum of the counts, and a second pass
// compacts each column in row order (warp ballots + a block scan), so the
// result is the reference's column-major scan order.
#include "internal.h"

#include <algorithm>
#include <cstring>
#include <numeric>

namespace ommgpu {

namespace {

constexpr int kConvThreads = 256;

// which entries a conversion keeps
enum KeepMode : int {
    KEEP_ALL = 0,      // m_copy without threshold: every element (MatrixSwitch_m_copy.F90:512-531)
    KEEP_GT = 1,       // |a| >  threshold (m_copy with threshold)
    KEEP_GE = 2,       // |a| >= threshold (psp_den2sp with thre > 0)
    KEEP_NONZERO = 3,  // a /= 0           (psp_den2sp with thre = 0)
};

__device__ __forceinline__ double absval(double a) { return fabs(a); }
__device__ __forceinline__ double absval(zdbl a) { return hypot(a.x, a.y); }
__device__ __forceinline__ bool is_zero(double a) { return a == 0.0; }
__device__ __forceinline__ bool is_zero(zdbl a) { return a.x == 0.0 && a.y == 0.0; }

template <typename T>
__device__ __forceinline__ bool keep(T a, int mode, double thr) {
    switch (mode) {
        case KEEP_ALL: return true;
        case KEEP_GT: return absval(a) > thr;
        case KEEP_GE: return absval(a) >= thr;
        default: return !is_zero(a);
    }
}

// soft thresholding: a - soft * a / |a|  (MatrixSwitch_m_copy.F90:127, :595)
__device__ __forceinline__ double shifted(double a, double soft) { return soft == 0.0 ? a : a - soft * a / fabs(a); }
__device__ __forceinline__ zdbl shifted(zdbl a, double soft) {
    if (soft == 0.0) return a;
    double r = hypot(a.x, a.y);
    return zdbl{a.x - soft * a.x / r, a.y - soft * a.y / r};
}

template <typename T>
__global__ void __launch_bounds__(kConvThreads) count_kernel(int rows, const T* __restrict__ A, int lda, int mode,
                                                             double thr, int* __restrict__ counts) {
    const int j = blockIdx.x;
    const T* col = A + (size_t)j * lda;
    int c = 0;
    for (int i = threadIdx.x; i < rows; i += blockDim.x) c += keep(col[i], mode, thr) ? 1 : 0;
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    __shared__ int part[kConvThreads / 32];
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        int t = 0;
        for (int w = 0; w < kConvThreads / 32; ++w) t += part[w];
        counts[j] = t;
    }
}

// column j's kept entries in row order at colptr[j] ..
template <typename T>
__global__ void __launch_bounds__(kConvThreads) compact_kernel(int rows, const T* __restrict__ A, int lda, int mode,
                                                               double thr, double soft, const int* __restrict__ colptr,
                                                               int* __restrict__ rowind, T* __restrict__ val) {
    const int j = blockIdx.x;
    const T* col = A + (size_t)j * lda;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __shared__ int wsum[kConvThreads / 32];
    int base = colptr[j];
    for (int i0 = 0; i0 < rows; i0 += kConvThreads) {
        const int i = i0 + threadIdx.x;
        T a{};
        bool k = false;
        if (i < rows) {
            a = col[i];
            k = keep(a, mode, thr);
        }
        const unsigned ballot = __ballot_sync(0xffffffffu, k);
        if (lane == 0) wsum[warp] = __popc(ballot);
        __syncthreads();
        int before = 0, total = 0;
        for (int w = 0; w < kConvThreads / 32; ++w) {
            before += (w < warp) ? wsum[w] : 0;
            total += wsum[w];
        }
        if (k) {
            const int pos = base + before + __popc(ballot & ((1u << lane) - 1u));
            rowind[pos] = i;
            val[pos] = shifted(a, soft);
        }
        base += total;
        __syncthreads();  // wsum is rewritten by the next tile
    }
}

template <typename T>
__global__ void threshold_dense_kernel(int rows, int cols, T* __restrict__ A, int lda, double thr, double soft) {
    size_t tot = (size_t)rows * cols;
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < tot; e += (size_t)gridDim.x * blockDim.x) {
        int i = (int)(e % rows), j = (int)(e / rows);
        T& a = A[i + (size_t)j * lda];
        a = keep(a, KEEP_GT, thr) ? shifted(a, soft) : T{};
    }
}

}  // namespace

// Dense (device view) -> CSC in M (host arrays and the device copy).  soft is the shift of kept
// values (0 for hard thresholding).
void dense_to_csc(const DView& A, int mode, double thr, double soft, msw_matrix* M) {
    const int rows = A.rows, cols = A.cols;
    M->h_colptr.assign(cols + 1, 0);
    M->nnz = 0;
    M->h_rowind.clear();
    M->h_val.clear();
    if (rows == 0 || cols == 0) return;
    DevBuf counts;
    counts.alloc((size_t)cols * sizeof(int));
    if (A.is_real)
        count_kernel<double><<<cols, kConvThreads, 0, rt().stream>>>(rows, A.as<double>(), A.ld, mode, thr,
                                                                       counts.as<int>());
    else
        count_kernel<zdbl><<<cols, kConvThreads, 0, rt().stream>>>(rows, A.as<zdbl>(), A.ld, mode, thr,
                                                                     counts.as<int>());
    OMM_KCHECK();
    std::vector<int> cnt(cols);
    OMM_CK(cudaMemcpyAsync(cnt.data(), counts.p, cols * sizeof(int), cudaMemcpyDeviceToHost, rt().stream));
    sync();
    long long total = 0;
    for (int j = 0; j < cols; ++j) {
        M->h_colptr[j] = (int)total;
        total += cnt[j];
        if (total > 0x7fffffffLL) fail(OMM_ERR_ARG, "m_copy: more than 2^31-1 kept entries");
    }
    M->h_colptr[cols] = (int)total;
    M->nnz = (int)total;
    const size_t es = A.is_real ? 8 : 16;
    M->d_colptr.alloc((size_t)(cols + 1) * sizeof(int));
    M->d_rowind.alloc(std::max<size_t>(1, (size_t)total) * sizeof(int));
    M->d_val.alloc(std::max<size_t>(1, (size_t)total) * es);
    OMM_CK(cudaMemcpyAsync(M->d_colptr.p, M->h_colptr.data(), (cols + 1) * sizeof(int), cudaMemcpyHostToDevice,
                           rt().stream));
    if (A.is_real)
        compact_kernel<double><<<cols, kConvThreads, 0, rt().stream>>>(rows, A.as<double>(), A.ld, mode, thr, soft,
                                                                         M->d_colptr.as<int>(), M->d_rowind.as<int>(),
                                                                         M->d_val.as<double>());
    else
        compact_kernel<zdbl><<<cols, kConvThreads, 0, rt().stream>>>(rows, A.as<zdbl>(), A.ld, mode, thr, soft,
                                                                       M->d_colptr.as<int>(), M->d_rowind.as<int>(),
                                                                       M->d_val.as<zdbl>());
    OMM_KCHECK();
    M->h_rowind.resize(total);
    M->h_val.resize((size_t)total * (A.is_real ? 1 : 2));
    if (total) {
        OMM_CK(cudaMemcpyAsync(M->h_rowind.data(), M->d_rowind.p, total * sizeof(int), cudaMemcpyDeviceToHost,
                               rt().stream));
        OMM_CK(cudaMemcpyAsync(M->h_val.data(), M->d_val.p, total * es, cudaMemcpyDeviceToHost, rt().stream));
    }
    sync();
}

void threshold_dense(DView& A, double thr, double soft) {
    size_t tot = (size_t)A.rows * A.cols;
    if (!tot) return;
    int grid = (int)std::min<size_t>((tot + 255) / 256, 148 * 32);
    if (A.is_real)
        threshold_dense_kernel<double><<<grid, 256, 0, rt().stream>>>(A.rows, A.cols, A.as<double>(), A.ld, thr, soft);
    else
        threshold_dense_kernel<zdbl><<<grid, 256, 0, rt().stream>>>(A.rows, A.cols, A.as<zdbl>(), A.ld, thr, soft);
    OMM_KCHECK();
}

}  // namespace ommgpu

using namespace ommgpu;

namespace {

std::unique_ptr<msw_matrix> new_matrix(const char label[5], int dim1, int dim2) {
    Label L = parse_storage(label);
    auto M = std::make_unique<msw_matrix>();
    M->dim1 = dim1;
    M->dim2 = dim2;
    M->is_real = L.real;
    M->fmt = L.fmt;
    M->loc = (L.where == 's') ? Loc::Host : Loc::Device;
    memcpy(M->label, label, 5);
    M->label[5] = 0;
    return M;
}

// src converted to a new matrix with `label`; mode/thr/soft as in dense_to_csc
msw_matrix* convert(const msw_matrix* src, const char label[5], bool thresholded, int mode, double thr, double soft) {
    Label L = parse_storage(label);
    if (L.real != src->is_real) fail(OMM_ERR_ARG, "m_copy: real/complex mismatch");
    auto M = new_matrix(label, src->dim1, src->dim2);
    if (L.fmt == Fmt::CSC && src->fmt == Fmt::CSC) {
        if (thresholded) fail(OMM_ERR_UNSUPPORTED, "m_copy: thresholding not yet implemented");  // MatrixSwitch.F90:840
        M->nnz = src->nnz;
        M->h_colptr = src->h_colptr;
        M->h_rowind = src->h_rowind;
        M->h_val = src->h_val;
        return M.release();
    }
    if (L.fmt == Fmt::CSC) {  // dense -> CSC on the device
        Staged s;
        stage_in(src, s, true);
        dense_to_csc(s.v, mode, thr, soft, M.get());
        return M.release();
    }
    // -> dense: copy (or scatter a CSC), then the threshold
    size_t bytes = M->elems() * M->esize();
    DView out{nullptr, M->dim1, M->dim2, std::max(1, M->dim1), M->is_real};
    DevBuf tmp;
    if (M->loc == Loc::Device) {
        M->dev.alloc_zero(std::max<size_t>(1, bytes));
        out.p = M->dev.p;
    } else {
        M->host_store.assign(M->elems() * (M->is_real ? 1 : 2), 0.0);
        M->host = M->host_store.data();
        tmp.alloc_zero(std::max<size_t>(1, bytes));
        out.p = tmp.p;
    }
    if (src->fmt == Fmt::CSC) {
        csc_to_dense_view(src, out);
    } else if (bytes) {
        OMM_CK(cudaMemcpyAsync(out.p, src->loc == Loc::Device ? src->dev.p : src->host, bytes,
                               src->loc == Loc::Device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                               rt().stream));
    }
    if (thresholded) threshold_dense(out, thr, soft);
    if (M->loc == Loc::Host && bytes)
        OMM_CK(cudaMemcpyAsync(M->host, out.p, bytes, cudaMemcpyDeviceToHost, rt().stream));
    sync();
    return M.release();
}

int finish(const Error& e) {
    set_last_error(e.msg);
    return e.code;
}

}  // namespace

extern "C" {

int msw_copy_thre(msw_matrix** dst, const msw_matrix* src, const char label[5], double threshold,
                  bool threshold_is_soft) {
    try {
        if (!dst || !src) fail(OMM_ERR_ARG, "m_copy: null argument");
        double thr = std::fabs(threshold);  // MatrixSwitch.F90:797-811
        *dst = convert(src, label, true, KEEP_GT, thr, threshold_is_soft ? thr : 0.0);
    } catch (const Error& e) {
        return finish(e);
    }
    set_last_error("");
    return OMM_OK;
}

int psp_gpu_den2sp(const msw_matrix* den, double thre, const char label[5], msw_matrix** sp) {
    try {
        if (!den || !sp) fail(OMM_ERR_ARG, "psp_den2sp: null argument");
        if (den->fmt != Fmt::Dense) fail(OMM_ERR_ARG, "psp_den2sp: the input must be dense");
        if (parse_storage(label).fmt != Fmt::CSC) fail(OMM_ERR_ARG, "psp_den2sp: label must be a csc storage");
        if (thre < 0.0) fail(OMM_ERR_ARG, "psp_den2sp_dm: thre must be non-negative");  // pspBasicTool.F90:256-257
        *sp = convert(den, label, false, thre == 0.0 ? KEEP_NONZERO : KEEP_GE, thre, 0.0);
    } catch (const Error& e) {
        return finish(e);
    }
    set_last_error("");
    return OMM_OK;
}

int psp_gpu_sp2den(const msw_matrix* sp, const char label[5], msw_matrix** den) {
    try {
        if (!den || !sp) fail(OMM_ERR_ARG, "psp_sp2den: null argument");
        if (sp->fmt != Fmt::CSC) fail(OMM_ERR_ARG, "psp_sp2den: the input must be sparse");
        if (parse_storage(label).fmt != Fmt::Dense) fail(OMM_ERR_ARG, "psp_sp2den: label must be a dense storage");
        *den = convert(sp, label, false, KEEP_ALL, 0.0, 0.0);
    } catch (const Error& e) {
        return finish(e);
    }
    set_last_error("");
    return OMM_OK;
}

int msw_csc_arrays(const msw_matrix* A, int* nnz, int* colptr, int* rowind, void* val) {
    try {
        if (!A || !nnz) fail(OMM_ERR_ARG, "msw_csc_arrays: null argument");
        if (A->fmt != Fmt::CSC) fail(OMM_ERR_ARG, "msw_csc_arrays: not a CSC matrix");
        *nnz = A->nnz;
        if (colptr) std::copy(A->h_colptr.begin(), A->h_colptr.end(), colptr);
        if (rowind) std::copy(A->h_rowind.begin(), A->h_rowind.end(), rowind);
        if (val) std::copy(A->h_val.begin(), A->h_val.end(), (double*)val);
    } catch (const Error& e) {
        return finish(e);
    }
    set_last_error("");
    return OMM_OK;
}

int msw_register_coo(msw_matrix** A, const char label[5], int dim1, int dim2, int nnz, const int* rowind,
                     const int* colind, const void* val, int index_base) {
    try {
        if (!A || (nnz > 0 && (!rowind || !colind || !val)) || nnz < 0) fail(OMM_ERR_ARG, "m_register_coo: bad argument");
        if (index_base != 0 && index_base != 1) fail(OMM_ERR_ARG, "m_register_coo: index_base must be 0 or 1");
        if (parse_storage(label).fmt != Fmt::CSC) fail(OMM_ERR_ARG, "m_register_coo: label must be a csc storage");
        auto M = new_matrix(label, dim1, dim2);
        const int w = M->is_real ? 1 : 2;
        const double* v = (const double*)val;
        std::vector<int> order(nnz);
        std::iota(order.begin(), order.end(), 0);
        for (int k = 0; k < nnz; ++k) {
            int r = rowind[k] - index_base, c = colind[k] - index_base;
            if (r < 0 || r >= dim1 || c < 0 || c >= dim2) fail(OMM_ERR_ARG, "m_register_coo: index out of range");
        }
        // column-major order (psp_coo2csc assumes it, pspBasicTool.F90:917); duplicates are summed
        std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
            return colind[a] != colind[b] ? colind[a] < colind[b] : rowind[a] < rowind[b];
        });
        M->h_colptr.assign(dim2 + 1, 0);
        M->h_rowind.reserve(nnz);
        M->h_val.reserve((size_t)nnz * w);
        int prev_r = -1, prev_c = -1;
        for (int k : order) {
            int r = rowind[k] - index_base, c = colind[k] - index_base;
            if (r == prev_r && c == prev_c) {
                for (int q = 0; q < w; ++q) M->h_val[M->h_val.size() - w + q] += v[(size_t)k * w + q];
                continue;
            }
            M->h_rowind.push_back(r);
            for (int q = 0; q < w; ++q) M->h_val.push_back(v[(size_t)k * w + q]);
            M->h_colptr[c + 1]++;
            prev_r = r;
            prev_c = c;
        }
        for (int j = 0; j < dim2; ++j) M->h_colptr[j + 1] += M->h_colptr[j];
        M->nnz = (int)M->h_rowind.size();
        *A = M.release();
    } catch (const Error& e) {
        return finish(e);
    }
    set_last_error("");
    return OMM_OK;
}

}  // extern "C"
