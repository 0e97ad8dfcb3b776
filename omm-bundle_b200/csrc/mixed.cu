// Reduced-precision products of the "gmx" solver.
//
// The CG state (C, D, G, [HC; SC], [HG; SG], the n x n W matrices) stays in
// FP64.  What changes in the reduced-precision stages is how the products of
// a step are computed:
//   * Gram products [HWd; SWd] = X D^T, [HWdd; SWdd] = Y D^T and calc_G
//     G = [4I - 2SW, -2HW] X on the tcgen05 BF16 GEMM (gemm_tc.cu) with FP32
//     accumulation; nseg = 1 is plain BF16, nseg = 3 the hi/lo split
//     (~2^-16 relative);
//   * the SpMM [HG; SG] = D [H, S] on CUDA cores in FP32 (column-group union
//     plan of spmm.cu with FP32 values), written back as FP64.
// The BF16 GEMM wants both operands K-major, so every FP64 matrix that feeds
// one gets a bf16 "shadow" in the layout that GEMM needs:
//   Dt  (n rows x m)   D^T-major: row j = D(j, :)          Gram B operand
//   Xt  (2n rows x m)  row i = X(i, :)                     Gram A operand
//   Yt  (2n rows x m)  row i = Y(i, :)                     Gram A operand
//   Xc  (m rows x 2n)  row j = X(:, j)  (X column-major)   calc_G B operand
//   Lt  (n rows x 2n)  row i = [4I - 2SW, -2HW](i, :)      calc_G A operand
// plus D in FP32 column-major for the SpMM.  Row strides are padded to
// multiples of 8 elements (16-byte rows for TMA).
#include "internal.h"

#include <cmath>

namespace ommgpu {

namespace {

inline int pad8(int x) { return (x + 7) / 8 * 8; }

__device__ __forceinline__ void split_bf16(double x, __nv_bfloat16& hi, __nv_bfloat16& lo) {
    hi = __float2bfloat16_rn((float)x);
    lo = __float2bfloat16_rn((float)(x - (double)__bfloat162float(hi)));
}

// dst (row-major, rows x cols, row stride ldd) = src^T-layout: dst[i*ldd + k] = src(i, k), src column-major.
// i.e. a transposed copy of the memory layout; hi (and lo when given) bf16 parts.
__global__ void shadow_rowmajor_kernel(int rows, int cols, const double* __restrict__ src, int lds,
                                       __nv_bfloat16* __restrict__ hi, __nv_bfloat16* __restrict__ lo, int ldd) {
    __shared__ double tile[32][33];
    int i0 = blockIdx.x * 32, k0 = blockIdx.y * 32;
    int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 32 x 8
    for (int yy = ty; yy < 32; yy += 8) {
        int i = i0 + tx, k = k0 + yy;
        tile[yy][tx] = (i < rows && k < cols) ? src[(size_t)i + (size_t)k * lds] : 0.0;
    }
    __syncthreads();
    for (int yy = ty; yy < 32; yy += 8) {
        int i = i0 + yy, k = k0 + tx;
        if (i < rows && k < cols) {
            __nv_bfloat16 h, l;
            split_bf16(tile[tx][yy], h, l);
            hi[(size_t)i * ldd + k] = h;
            if (lo) lo[(size_t)i * ldd + k] = l;
        }
    }
}

// dst (column-major with leading dimension ldd) = bf16 parts of src (column-major).
__global__ void shadow_colmajor_kernel(int rows, int cols, const double* __restrict__ src, int lds,
                                       __nv_bfloat16* __restrict__ hi, __nv_bfloat16* __restrict__ lo, int ldd) {
    size_t tot = (size_t)rows * cols;
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < tot; e += (size_t)gridDim.x * blockDim.x) {
        int i = (int)(e % rows), j = (int)(e / rows);
        __nv_bfloat16 h, l;
        split_bf16(src[(size_t)i + (size_t)j * lds], h, l);
        hi[(size_t)i + (size_t)j * ldd] = h;
        if (lo) lo[(size_t)i + (size_t)j * ldd] = l;
    }
}

__global__ void to_f32_kernel(int rows, int cols, const double* __restrict__ src, int lds, float* __restrict__ dst,
                              int ldd) {
    size_t tot = (size_t)rows * cols;
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < tot; e += (size_t)gridDim.x * blockDim.x) {
        int i = (int)(e % rows), j = (int)(e / rows);
        dst[(size_t)i + (size_t)j * ldd] = (float)src[(size_t)i + (size_t)j * lds];
    }
}

// Lt (row-major n x 2n, row stride ldl): row i = [4I - 2 SW, -2 HW](i, :)  (calc_G's left factor)
__global__ void calcG_left_bf16_kernel(int n, const double* __restrict__ SW, const double* __restrict__ HW,
                                       __nv_bfloat16* __restrict__ hi, __nv_bfloat16* __restrict__ lo, int ldl) {
    size_t tot = (size_t)n * 2 * n;
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < tot; e += (size_t)gridDim.x * blockDim.x) {
        int k = (int)(e % (2 * n)), i = (int)(e / (2 * n));  // consecutive threads along a row of Lt
        double v;
        if (k < n) v = (i == k ? 4.0 : 0.0) - 2.0 * SW[i + (size_t)k * n];
        else v = -2.0 * HW[i + (size_t)(k - n) * n];
        __nv_bfloat16 h, l;
        split_bf16(v, h, l);
        hi[(size_t)i * ldl + k] = h;
        if (lo) lo[(size_t)i * ldl + k] = l;
    }
}

inline int grid1d(size_t tot) {
    size_t b = (tot + 255) / 256;
    return (int)std::min<size_t>(std::max<size_t>(b, 1), 148 * 32);
}

void ensure(DevBuf& b, size_t bytes) {
    if (!b.p || b.bytes < bytes) b.alloc(bytes);
}

}  // namespace

// ------------------------------------------------------------------ shadows
void mx_shadow_rowmajor(const DView& src, DevBuf& hi, DevBuf& lo, int nseg, int& ldd) {
    ldd = pad8(src.cols);
    size_t bytes = (size_t)src.rows * ldd * sizeof(__nv_bfloat16);
    ensure(hi, bytes);
    if (nseg == 3) ensure(lo, bytes);
    dim3 grid((src.rows + 31) / 32, (src.cols + 31) / 32);
    shadow_rowmajor_kernel<<<grid, 256, 0, rt().stream>>>(src.rows, src.cols, src.as<double>(), src.ld,
                                                          hi.as<__nv_bfloat16>(),
                                                          nseg == 3 ? lo.as<__nv_bfloat16>() : nullptr, ldd);
    OMM_KCHECK();
}

void mx_shadow_colmajor(const DView& src, DevBuf& hi, DevBuf& lo, int nseg, int& ldd) {
    ldd = pad8(src.rows);
    size_t bytes = (size_t)src.cols * ldd * sizeof(__nv_bfloat16);
    ensure(hi, bytes);
    if (nseg == 3) ensure(lo, bytes);
    size_t tot = (size_t)src.rows * src.cols;
    shadow_colmajor_kernel<<<grid1d(tot), 256, 0, rt().stream>>>(src.rows, src.cols, src.as<double>(), src.ld,
                                                                  hi.as<__nv_bfloat16>(),
                                                                  nseg == 3 ? lo.as<__nv_bfloat16>() : nullptr, ldd);
    OMM_KCHECK();
}

void mx_to_f32(const DView& src, DevBuf& dst) {
    ensure(dst, (size_t)src.rows * src.cols * sizeof(float));
    size_t tot = (size_t)src.rows * src.cols;
    to_f32_kernel<<<grid1d(tot), 256, 0, rt().stream>>>(src.rows, src.cols, src.as<double>(), src.ld, dst.as<float>(),
                                                         src.rows);
    OMM_KCHECK();
}

void mx_calcG_left(int n, const DView& SW, const DView& HW, DevBuf& hi, DevBuf& lo, int nseg, int& ldl) {
    ldl = pad8(2 * n);
    size_t bytes = (size_t)n * ldl * sizeof(__nv_bfloat16);
    ensure(hi, bytes);
    if (nseg == 3) ensure(lo, bytes);
    calcG_left_bf16_kernel<<<grid1d((size_t)n * 2 * n), 256, 0, rt().stream>>>(
        n, SW.as<double>(), HW.as<double>(), hi.as<__nv_bfloat16>(), nseg == 3 ? lo.as<__nv_bfloat16>() : nullptr,
        ldl);
    OMM_KCHECK();
}

}  // namespace ommgpu

using namespace ommgpu;

// C = A * B with the reduced-precision SpMM of the "gmx" solver (see include/ommgpu.h).
extern "C" int omm_gpu_spmm_lowp(const msw_matrix* A, const msw_matrix* B, msw_matrix* C, int nseg, int* path) {
    try {
        if (!A || !B || !C || !A->dense() || B->fmt != Fmt::CSC || !C->dense())
            fail(OMM_ERR_ARG, "spmm_lowp: A dense, B csc, C dense required");
        if (!A->is_real || !B->is_real || !C->is_real) fail(OMM_ERR_UNSUPPORTED, "spmm_lowp: real matrices only");
        if (A->loc != Loc::Device || C->loc != Loc::Device) fail(OMM_ERR_ARG, "spmm_lowp: A and C must be 'g' storage");
        if (A->dim2 != B->dim1 || C->dim1 != A->dim1 || C->dim2 != B->dim2)
            fail(OMM_ERR_ARG, "spmm_lowp: dimensions do not match");
        if (nseg != 1 && nseg != 3) fail(OMM_ERR_ARG, "spmm_lowp: nseg must be 1 or 3");
        ensure_csc_device(B);
        DView a{A->dev.p, A->dim1, A->dim2, std::max(1, A->dim1), true};
        DView c{C->dev.p, C->dim1, C->dim2, std::max(1, C->dim1), true};
        int used = 0;
        if (spmm_tc_available(B)) {
            static DevBuf hi, lo;
            int ld = 0;
            mx_shadow_rowmajor(a, hi, lo, nseg, ld);
            SpmmPlanView P = spmm_plan_view(B);
            if (spmm_tc(hi.as<__nv_bfloat16>(), nseg == 3 ? lo.as<__nv_bfloat16>() : nullptr, ld, a.rows, B, P, c,
                        nullptr, nullptr, nullptr, nseg))
                used = 2;
        }
        if (!used && spmm32_available(B)) {
            static DevBuf f32;
            mx_to_f32(a, f32);
            spmm32_dense_csc(f32.as<float>(), a.rows, a.rows, B, c, nullptr, nullptr);
            used = 1;
        }
        if (!used) {
            double one[2] = {1.0, 0.0}, zero[2] = {0.0, 0.0};
            spmm_dense_csc(a, B, c, one, zero);
        }
        if (path) *path = used;
        if (unsigned e = gemm_bf16_errors())
            fail(OMM_ERR_CUDA, "spmm_lowp: a pipeline wait timed out (error bits " + std::to_string(e) + ")");
    } catch (const Error& e) {
        set_last_error(e.msg);
        return e.code;
    }
    set_last_error("");
    return OMM_OK;
}

