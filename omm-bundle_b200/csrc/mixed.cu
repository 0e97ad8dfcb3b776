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
//   Dk  (m/8 planes of n x 8)  k-blocked copy of Dt        tensor-core SpMM A operand
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

// bf16 shadows of src (rows x cols, column-major), from one read of src:
//  * row-major (when hi != nullptr): hi[i*ldd + k] = src(i, k), i.e. a transposed copy of the layout;
//  * k-blocked (when khi != nullptr): khi[kblock_offset(i, k, cols)] = src(i, k), zero for k >= cols:
//    the 8 k-values of a row are one 16-byte vector, the vectors of a 256-row block's rows are
//    contiguous (one 4 KB chunk per 8 k), and the chunks of one row block follow each other, so a
//    run of consecutive chunks is one contiguous bulk copy.
//  * column-major (when chi != nullptr): chi[i + k*ldc] = src(i, k).
// lo / klo / clo (when given) receive the low bf16 parts of the hi/lo split.
// With add != nullptr, src is first updated in place, src = b*src + a*add (the expression of
// axpby_kernel), and the shadows are those of the updated values.
template <typename TA>
__global__ void shadow_rowmajor_kernel(int rows, int cols, double* __restrict__ src, int lds,
                                       const TA* __restrict__ add, int ldadd, double a, double b,
                                       __nv_bfloat16* __restrict__ hi, __nv_bfloat16* __restrict__ lo, int ldd,
                                       __nv_bfloat16* __restrict__ khi, __nv_bfloat16* __restrict__ klo,
                                       __nv_bfloat16* __restrict__ chi, __nv_bfloat16* __restrict__ clo, int ldc) {
    __shared__ double tile[32][33];
    int i0 = blockIdx.x * 32, k0 = blockIdx.y * 32;
    int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 32 x 8
    for (int yy = ty; yy < 32; yy += 8) {
        int i = i0 + tx, k = k0 + yy;
        double v = 0.0;
        if (i < rows && k < cols) {
            v = src[(size_t)i + (size_t)k * lds];
            if (add) {
                const double c = b * v;
                v = c + a * (double)add[(size_t)i + (size_t)k * ldadd];
                src[(size_t)i + (size_t)k * lds] = v;
            }
            if (chi) {
                __nv_bfloat16 h, l;
                split_bf16(v, h, l);
                chi[(size_t)i + (size_t)k * ldc] = h;
                if (clo) clo[(size_t)i + (size_t)k * ldc] = l;
            }
        }
        tile[yy][tx] = v;
    }
    __syncthreads();
    if (hi) {
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
    if (khi && threadIdx.x < 128) {
        const int r = threadIdx.x & 31, q = threadIdx.x >> 5;  // row of the tile, 8-k block of the tile
        const int i = i0 + r, kb = (k0 >> 3) + q;
        if (i < rows && 8 * kb < cols) {
            __align__(16) __nv_bfloat16 h[8], l[8];
#pragma unroll
            for (int e = 0; e < 8; ++e) split_bf16(tile[8 * q + e][r], h[e], l[e]);
            const size_t off = kblock_offset(i, 8 * kb, cols);
            *reinterpret_cast<uint4*>(khi + off) = *reinterpret_cast<const uint4*>(h);
            if (klo) *reinterpret_cast<uint4*>(klo + off) = *reinterpret_cast<const uint4*>(l);
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

// ---- complex products as real GEMMs.  With A' = [Re A | Im A] (K doubled) and, for the
// N x K operand B, B' = [[Re B | -Im B]; [Im B | Re B]] (N and K doubled), A' B'^T holds
// Re(A B^T) in its first N columns and Im(A B^T) in the next N.

// A' rows from a column-major complex src (rows x cols): dst[i*ldd + k] = Re src(i,k),
// dst[i*ldd + cols + k] = Im src(i,k).  With `conj_b`, also the rows rows..2rows-1 of the B'
// of B = conj(src): B' = [[Re | Im]; [-Im | Re]] (the Gram products' D^H).
__global__ void cshadow_rows_kernel(int rows, int cols, const zdbl* __restrict__ src, int lds,
                                    __nv_bfloat16* __restrict__ hi, __nv_bfloat16* __restrict__ lo, int ldd,
                                    int conj_b) {
    size_t tot = (size_t)rows * cols;
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < tot; e += (size_t)gridDim.x * blockDim.x) {
        int k = (int)(e % cols), i = (int)(e / cols);  // consecutive threads along a destination row
        zdbl v = src[(size_t)i + (size_t)k * lds];
        __nv_bfloat16 rh, rl, ih, il;
        split_bf16(v.x, rh, rl);
        split_bf16(v.y, ih, il);
        size_t r0 = (size_t)i * ldd;
        hi[r0 + k] = rh;
        hi[r0 + cols + k] = ih;
        if (lo) {
            lo[r0 + k] = rl;
            lo[r0 + cols + k] = il;
        }
        if (conj_b) {
            size_t r1 = (size_t)(rows + i) * ldd;
            hi[r1 + k] = __hneg(ih);
            hi[r1 + cols + k] = rh;
            if (lo) {
                lo[r1 + k] = __hneg(il);
                lo[r1 + cols + k] = rl;
            }
        }
    }
}

// B' of B = src^T (B row j = src(:, j), no conjugate) from a column-major complex src
// (rows x cols): row j = [Re src(:,j) | -Im src(:,j)], row cols+j = [Im src(:,j) | Re src(:,j)].
__global__ void cshadow_cols_kernel(int rows, int cols, const zdbl* __restrict__ src, int lds,
                                    __nv_bfloat16* __restrict__ hi, __nv_bfloat16* __restrict__ lo, int ldd) {
    size_t tot = (size_t)rows * cols;
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < tot; e += (size_t)gridDim.x * blockDim.x) {
        int i = (int)(e % rows), j = (int)(e / rows);  // consecutive threads down a source column
        zdbl v = src[(size_t)i + (size_t)j * lds];
        __nv_bfloat16 rh, rl, ih, il;
        split_bf16(v.x, rh, rl);
        split_bf16(v.y, ih, il);
        size_t r0 = (size_t)j * ldd, r1 = (size_t)(cols + j) * ldd;
        hi[r0 + i] = rh;
        hi[r0 + rows + i] = __hneg(ih);
        hi[r1 + i] = ih;
        hi[r1 + rows + i] = rh;
        if (lo) {
            lo[r0 + i] = rl;
            lo[r0 + rows + i] = __hneg(il);
            lo[r1 + i] = il;
            lo[r1 + rows + i] = rl;
        }
    }
}

// dst(i, j) = (re(i, j), re(i, N + j)) for the M x 2N real product (column-major, ld M)
__global__ void interleave_kernel(int M, int N, const double* __restrict__ re, zdbl* __restrict__ dst, int ldd) {
    size_t tot = (size_t)M * N;
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < tot; e += (size_t)gridDim.x * blockDim.x) {
        int i = (int)(e % M), j = (int)(e / M);
        dst[(size_t)i + (size_t)j * ldd] = zdbl{re[(size_t)i + (size_t)j * M], re[(size_t)i + (size_t)(N + j) * M]};
    }
}

// complex calc_G left factor L = [4I - 2 SW, -2 HW] (n x 2n) as A' rows: [Re L(i,:) | Im L(i,:)]
__global__ void calcG_left_cplx_kernel(int n, const zdbl* __restrict__ SW, const zdbl* __restrict__ HW,
                                       __nv_bfloat16* __restrict__ hi, __nv_bfloat16* __restrict__ lo, int ldl) {
    size_t tot = (size_t)n * 2 * n;
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < tot; e += (size_t)gridDim.x * blockDim.x) {
        int k = (int)(e % (2 * n)), i = (int)(e / (2 * n));
        zdbl v;
        if (k < n) {
            zdbl w = SW[i + (size_t)k * n];
            v = zdbl{(i == k ? 4.0 : 0.0) - 2.0 * w.x, -2.0 * w.y};
        } else {
            zdbl w = HW[i + (size_t)(k - n) * n];
            v = zdbl{-2.0 * w.x, -2.0 * w.y};
        }
        __nv_bfloat16 rh, rl, ih, il;
        split_bf16(v.x, rh, rl);
        split_bf16(v.y, ih, il);
        hi[(size_t)i * ldl + k] = rh;
        hi[(size_t)i * ldl + 2 * n + k] = ih;
        if (lo) {
            lo[(size_t)i * ldl + k] = rl;
            lo[(size_t)i * ldl + 2 * n + k] = il;
        }
    }
}

// row-major bf16 hi/lo of SW - I (n x n): the small factor of the refinement gradient
__global__ void delta_shadow_kernel(int n, const double* __restrict__ SW, __nv_bfloat16* __restrict__ hi,
                                    __nv_bfloat16* __restrict__ lo, int ldd) {
    size_t tot = (size_t)n * n;
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < tot; e += (size_t)gridDim.x * blockDim.x) {
        int k = (int)(e % n), i = (int)(e / n);  // consecutive threads along a destination row
        double v = SW[i + (size_t)k * n] - (i == k ? 1.0 : 0.0);
        __nv_bfloat16 h, l;
        split_bf16(v, h, l);
        hi[(size_t)i * ldd + k] = h;
        lo[(size_t)i * ldd + k] = l;
    }
}

inline int grid1d(size_t tot) {
    size_t b = (tot + 255) / 256;
    return (int)std::min<size_t>(std::max<size_t>(b, 1), 148 * 32);
}

void ensure(DevBuf& b, size_t bytes) {
    if (!b.p || b.bytes < bytes) b.alloc(bytes);
}

// k-blocked shadows of rows x cols; rows past the last one in the last row block start zeroed
// (the SpMM copies whole row blocks; those rows only feed output rows that are never stored)
void ensure_kblock(DevBuf& b, int rows, int cols) {
    const size_t bytes = kblock_elems(rows, cols) * sizeof(__nv_bfloat16);
    if (!b.p || b.bytes < bytes) b.alloc_zero(bytes);
}

}  // namespace

// ------------------------------------------------------------------ shadows
void mx_shadow_rowmajor(const DView& src, DevBuf& hi, DevBuf& lo, int nseg, int& ldd, DevBuf* khi, DevBuf* klo) {
    ldd = pad8(src.cols);
    size_t bytes = (size_t)src.rows * ldd * sizeof(__nv_bfloat16);
    ensure(hi, bytes);
    if (nseg == 3) ensure(lo, bytes);
    if (khi) {  // k-blocked copy (kblock_offset)
        ensure_kblock(*khi, src.rows, src.cols);
        if (nseg == 3) ensure_kblock(*klo, src.rows, src.cols);
    }
    dim3 grid((src.rows + 31) / 32, (src.cols + 31) / 32);
    shadow_rowmajor_kernel<double><<<grid, 256, 0, rt().stream>>>(
        src.rows, src.cols, src.as<double>(), src.ld, nullptr, 0, 0.0, 1.0, hi.as<__nv_bfloat16>(),
        nseg == 3 ? lo.as<__nv_bfloat16>() : nullptr, ldd, khi ? khi->as<__nv_bfloat16>() : nullptr,
        (khi && nseg == 3) ? klo->as<__nv_bfloat16>() : nullptr, nullptr, nullptr, 0);
    OMM_KCHECK();
}

// D = b*D + a*G (FP64, in place) and the row-major and (when khi is given) k-blocked bf16 shadows
// of the result, in one pass: the real CG step's new direction and the operands of its products.
void mx_update_shadow_rowmajor(DView& D, const DView& G, double a, double b, DevBuf& hi, DevBuf& lo, int nseg,
                               int& ldd, DevBuf* khi, DevBuf* klo) {
    if (!D.is_real || !G.is_real || D.rows != G.rows || D.cols != G.cols)
        fail(OMM_ERR_ARG, "mx_update_shadow_rowmajor: real operands of equal shape");
    ldd = pad8(D.cols);
    const size_t bytes = (size_t)D.rows * ldd * sizeof(__nv_bfloat16);
    ensure(hi, bytes);
    if (nseg == 3) ensure(lo, bytes);
    if (khi) {
        ensure_kblock(*khi, D.rows, D.cols);
        if (nseg == 3) ensure_kblock(*klo, D.rows, D.cols);
    }
    dim3 grid((D.rows + 31) / 32, (D.cols + 31) / 32);
    shadow_rowmajor_kernel<double><<<grid, 256, 0, rt().stream>>>(
        D.rows, D.cols, D.as<double>(), D.ld, G.as<double>(), G.ld, a, b, hi.as<__nv_bfloat16>(),
        nseg == 3 ? lo.as<__nv_bfloat16>() : nullptr, ldd, khi ? khi->as<__nv_bfloat16>() : nullptr,
        (khi && nseg == 3) ? klo->as<__nv_bfloat16>() : nullptr, nullptr, nullptr, 0);
    OMM_KCHECK();
}

// X = X + a*Y (FP64, in place) and the row-major (t) and column-major (c) bf16 shadows of the
// result, in one pass over X and Y: the real CG step's [HC; SC] += x [HG; SG] and the operands
// the next Gram and calc_G products read.
void mx_update_shadows(DView& X, const DView& Y, double a, DevBuf& thi, DevBuf& tlo, int& ldt, DevBuf& chi,
                       DevBuf& clo, int& ldc, int nseg, const float* Y32, int ldy32) {
    if (!X.is_real || (!Y32 && (!Y.is_real || X.rows != Y.rows || X.cols != Y.cols)))
        fail(OMM_ERR_ARG, "mx_update_shadows: real operands of equal shape");
    ldt = pad8(X.cols);
    ldc = pad8(X.rows);
    const size_t tb = (size_t)X.rows * ldt * sizeof(__nv_bfloat16), cb = (size_t)X.cols * ldc * sizeof(__nv_bfloat16);
    ensure(thi, tb);
    ensure(chi, cb);
    if (nseg == 3) {
        ensure(tlo, tb);
        ensure(clo, cb);
    }
    dim3 grid((X.rows + 31) / 32, (X.cols + 31) / 32);
    if (Y32)
        shadow_rowmajor_kernel<float><<<grid, 256, 0, rt().stream>>>(
            X.rows, X.cols, X.as<double>(), X.ld, Y32, ldy32, a, 1.0, thi.as<__nv_bfloat16>(),
            nseg == 3 ? tlo.as<__nv_bfloat16>() : nullptr, ldt, nullptr, nullptr, chi.as<__nv_bfloat16>(),
            nseg == 3 ? clo.as<__nv_bfloat16>() : nullptr, ldc);
    else
        shadow_rowmajor_kernel<double><<<grid, 256, 0, rt().stream>>>(
            X.rows, X.cols, X.as<double>(), X.ld, Y.as<double>(), Y.ld, a, 1.0, thi.as<__nv_bfloat16>(),
            nseg == 3 ? tlo.as<__nv_bfloat16>() : nullptr, ldt, nullptr, nullptr, chi.as<__nv_bfloat16>(),
            nseg == 3 ? clo.as<__nv_bfloat16>() : nullptr, ldc);
    OMM_KCHECK();
}

void mx_shadow_kblock(const DView& src, DevBuf& khi, DevBuf& klo, int nseg) {
    ensure_kblock(khi, src.rows, src.cols);
    if (nseg == 3) ensure_kblock(klo, src.rows, src.cols);
    dim3 grid((src.rows + 31) / 32, (src.cols + 31) / 32);
    shadow_rowmajor_kernel<double><<<grid, 256, 0, rt().stream>>>(src.rows, src.cols, src.as<double>(), src.ld, nullptr, 0,
                                                          0.0, 1.0, nullptr, nullptr, 0, khi.as<__nv_bfloat16>(),
                                                          nseg == 3 ? klo.as<__nv_bfloat16>() : nullptr, nullptr,
                                                          nullptr, 0);
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

void mx_cshadow_rows(const DView& src, DevBuf& hi, DevBuf& lo, int nseg, int& ldd, bool conj_b) {
    ldd = pad8(2 * src.cols);
    size_t bytes = (size_t)src.rows * (conj_b ? 2 : 1) * ldd * sizeof(__nv_bfloat16);
    ensure(hi, bytes);
    if (nseg == 3) ensure(lo, bytes);
    cshadow_rows_kernel<<<grid1d((size_t)src.rows * src.cols), 256, 0, rt().stream>>>(
        src.rows, src.cols, src.as<zdbl>(), src.ld, hi.as<__nv_bfloat16>(),
        nseg == 3 ? lo.as<__nv_bfloat16>() : nullptr, ldd, conj_b ? 1 : 0);
    OMM_KCHECK();
}

void mx_cshadow_cols(const DView& src, DevBuf& hi, DevBuf& lo, int nseg, int& ldd) {
    ldd = pad8(2 * src.rows);
    size_t bytes = (size_t)2 * src.cols * ldd * sizeof(__nv_bfloat16);
    ensure(hi, bytes);
    if (nseg == 3) ensure(lo, bytes);
    cshadow_cols_kernel<<<grid1d((size_t)src.rows * src.cols), 256, 0, rt().stream>>>(
        src.rows, src.cols, src.as<zdbl>(), src.ld, hi.as<__nv_bfloat16>(),
        nseg == 3 ? lo.as<__nv_bfloat16>() : nullptr, ldd);
    OMM_KCHECK();
}

void mx_interleave(int M, int N, const double* re, DView& dst) {
    interleave_kernel<<<grid1d((size_t)M * N), 256, 0, rt().stream>>>(M, N, re, dst.as<zdbl>(), dst.ld);
    OMM_KCHECK();
}

void mx_calcG_left_cplx(int n, const DView& SW, const DView& HW, DevBuf& hi, DevBuf& lo, int nseg, int& ldl) {
    ldl = pad8(4 * n);
    size_t bytes = (size_t)n * ldl * sizeof(__nv_bfloat16);
    ensure(hi, bytes);
    if (nseg == 3) ensure(lo, bytes);
    calcG_left_cplx_kernel<<<grid1d((size_t)n * 2 * n), 256, 0, rt().stream>>>(
        n, SW.as<zdbl>(), HW.as<zdbl>(), hi.as<__nv_bfloat16>(), nseg == 3 ? lo.as<__nv_bfloat16>() : nullptr, ldl);
    OMM_KCHECK();
}

void mx_delta_shadow(int n, const DView& SW, DevBuf& hi, DevBuf& lo, int& ldd) {
    ldd = pad8(n);
    size_t bytes = (size_t)n * ldd * sizeof(__nv_bfloat16);
    ensure(hi, bytes);
    ensure(lo, bytes);
    delta_shadow_kernel<<<grid1d((size_t)n * n), 256, 0, rt().stream>>>(n, SW.as<double>(), hi.as<__nv_bfloat16>(),
                                                                          lo.as<__nv_bfloat16>(), ldd);
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

namespace {

// operand shadow shared by omm_gpu_spmm_lowp_prepare / _apply
struct LowpOperand {
    DevBuf hi, lo;
    int rows = 0, cols = 0, nseg = 0;
};
LowpOperand& lowp_operand() {
    static LowpOperand* op = new LowpOperand();
    return *op;
}

void lowp_check(const msw_matrix* B, const msw_matrix* C, int rows, int cols) {
    if (!B || !C || B->fmt != Fmt::CSC || !C->dense()) fail(OMM_ERR_ARG, "spmm_lowp: B csc and C dense required");
    if (!B->is_real || !C->is_real) fail(OMM_ERR_UNSUPPORTED, "spmm_lowp: real matrices only");
    if (C->loc != Loc::Device) fail(OMM_ERR_ARG, "spmm_lowp: C must be 'g' storage");
    if (cols != B->dim1 || C->dim1 != rows || C->dim2 != B->dim2) fail(OMM_ERR_ARG, "spmm_lowp: dimensions do not match");
}

// the tensor-core product from the prepared shadow; false when B (and B2) cannot take it
bool lowp_apply(const msw_matrix* B, msw_matrix* C, const msw_matrix* B2, msw_matrix* C2, int nseg) {
    LowpOperand& op = lowp_operand();
    ensure_csc_device(B);
    if (B2) ensure_csc_device(B2);
    if (!spmm_tc_available(B) || (B2 && (!spmm_tc_available(B2) || !same_pattern(B, B2)))) return false;
    DView c{C->dev.p, C->dim1, C->dim2, std::max(1, C->dim1), true};
    DView c2{C2 ? C2->dev.p : nullptr, C2 ? C2->dim1 : 0, C2 ? C2->dim2 : 0, C2 ? std::max(1, C2->dim1) : 1, true};
    SpmmPlanView P = spmm_plan_view(B), P2;
    if (B2) P2 = spmm_plan_view(B2);
    return spmm_tc(op.hi.as<__nv_bfloat16>(), nseg == 3 ? op.lo.as<__nv_bfloat16>() : nullptr, op.rows, op.cols, B,
                   P, c, B2, B2 ? &P2 : nullptr, B2 ? &c2 : nullptr, nseg);
}

}  // namespace

// C = A * B (and C2 = A * B2) with the reduced-precision SpMM of the "gmx" solver (include/ommgpu.h).
extern "C" int omm_gpu_spmm_lowp(const msw_matrix* A, const msw_matrix* B, msw_matrix* C, const msw_matrix* B2,
                                 msw_matrix* C2, int nseg, int* path) {
    try {
        if (!A || !A->dense() || A->loc != Loc::Device) fail(OMM_ERR_ARG, "spmm_lowp: A must be dense 'g' storage");
        if (!A->is_real) fail(OMM_ERR_UNSUPPORTED, "spmm_lowp: real matrices only");
        if (nseg != 1 && nseg != 3) fail(OMM_ERR_ARG, "spmm_lowp: nseg must be 1 or 3");
        lowp_check(B, C, A->dim1, A->dim2);
        if ((B2 == nullptr) != (C2 == nullptr)) fail(OMM_ERR_ARG, "spmm_lowp: B2 and C2 go together");
        if (B2) lowp_check(B2, C2, A->dim1, A->dim2);
        ensure_csc_device(B);
        if (B2) ensure_csc_device(B2);
        DView a{A->dev.p, A->dim1, A->dim2, std::max(1, A->dim1), true};
        int used = 0;
        if (spmm_tc_available(B) && (!B2 || spmm_tc_available(B2))) {
            LowpOperand& op = lowp_operand();
            mx_shadow_kblock(a, op.hi, op.lo, nseg);
            op.rows = a.rows;
            op.cols = a.cols;
            op.nseg = nseg;
            if (B2 && !same_pattern(B, B2)) {
                if (lowp_apply(B, C, nullptr, nullptr, nseg) && lowp_apply(B2, C2, nullptr, nullptr, nseg)) used = 2;
            } else if (lowp_apply(B, C, B2, C2, nseg)) {
                used = 2;
            }
        }
        for (int k = 0; k < (B2 ? 2 : 1) && !used; ++k) {
            const msw_matrix* Bk = k ? B2 : B;
            msw_matrix* Ck = k ? C2 : C;
            DView c{Ck->dev.p, Ck->dim1, Ck->dim2, std::max(1, Ck->dim1), true};
            if (spmm32_available(Bk)) {
                static DevBuf f32;
                mx_to_f32(a, f32);
                spmm32_dense_csc(f32.as<float>(), a.rows, a.rows, Bk, c, nullptr, nullptr);
                if (k == (B2 ? 1 : 0)) used = 1;
            } else {
                double one[2] = {1.0, 0.0}, zero[2] = {0.0, 0.0};
                spmm_dense_csc(a, Bk, c, one, zero);
            }
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

extern "C" int omm_gpu_spmm_lowp_prepare(const msw_matrix* A, int nseg) {
    try {
        if (!A || !A->dense() || A->loc != Loc::Device) fail(OMM_ERR_ARG, "spmm_lowp_prepare: A must be dense 'g'");
        if (!A->is_real) fail(OMM_ERR_UNSUPPORTED, "spmm_lowp_prepare: real matrices only");
        if (nseg != 1 && nseg != 3) fail(OMM_ERR_ARG, "spmm_lowp_prepare: nseg must be 1 or 3");
        DView a{A->dev.p, A->dim1, A->dim2, std::max(1, A->dim1), true};
        LowpOperand& op = lowp_operand();
        mx_shadow_kblock(a, op.hi, op.lo, nseg);
        op.rows = a.rows;
        op.cols = a.cols;
        op.nseg = nseg;
    } catch (const Error& e) {
        set_last_error(e.msg);
        return e.code;
    }
    set_last_error("");
    return OMM_OK;
}

extern "C" int omm_gpu_spmm_lowp_apply(const msw_matrix* B, msw_matrix* C, const msw_matrix* B2, msw_matrix* C2,
                                       int nseg) {
    try {
        LowpOperand& op = lowp_operand();
        if (op.rows == 0) fail(OMM_ERR_STATE, "spmm_lowp_apply: no operand prepared");
        if (nseg != op.nseg) fail(OMM_ERR_ARG, "spmm_lowp_apply: nseg differs from the prepared operand");
        lowp_check(B, C, op.rows, op.cols);
        if ((B2 == nullptr) != (C2 == nullptr)) fail(OMM_ERR_ARG, "spmm_lowp_apply: B2 and C2 go together");
        if (B2) lowp_check(B2, C2, op.rows, op.cols);
        if (!lowp_apply(B, C, B2, C2, nseg))
            fail(OMM_ERR_UNSUPPORTED, "spmm_lowp_apply: B (and B2) must take the tensor-core path with one pattern");
    } catch (const Error& e) {
        set_last_error(e.msg);
        return e.code;
    }
    set_last_error("");
    return OMM_OK;
}

extern "C" int omm_gpu_spmm_lowp_apply_f32(const msw_matrix* B, const msw_matrix* B2, float* Y, int ldy, void* t_hi,
                                           void* t_lo, int ldt, int nseg) {
    try {
        LowpOperand& op = lowp_operand();
        if (op.rows == 0) fail(OMM_ERR_STATE, "spmm_lowp_apply_f32: no operand prepared");
        if (nseg != op.nseg) fail(OMM_ERR_ARG, "spmm_lowp_apply_f32: nseg differs from the prepared operand");
        if (!B || B->fmt != Fmt::CSC || !B->is_real || (B2 && (B2->fmt != Fmt::CSC || !B2->is_real)))
            fail(OMM_ERR_ARG, "spmm_lowp_apply_f32: real CSC matrices required");
        if (B->dim1 != op.cols || B->dim2 != op.cols || (B2 && (B2->dim1 != op.cols || B2->dim2 != op.cols)))
            fail(OMM_ERR_ARG, "spmm_lowp_apply_f32: dimensions do not match");
        if (!Y || ldy < (B2 ? 2 : 1) * op.rows) fail(OMM_ERR_ARG, "spmm_lowp_apply_f32: Y too small");
        if (t_lo && !t_hi) fail(OMM_ERR_ARG, "spmm_lowp_apply_f32: t_lo without t_hi");
        if (t_hi && ldt < op.cols) fail(OMM_ERR_ARG, "spmm_lowp_apply_f32: shadow stride too small");
        ensure_csc_device(B);
        if (B2) ensure_csc_device(B2);
        if (!spmm_lowp_f32(op.hi.as<__nv_bfloat16>(), nseg == 3 ? op.lo.as<__nv_bfloat16>() : nullptr, op.rows, op.cols, B,
                      B2, Y, ldy, (__nv_bfloat16*)t_hi, (__nv_bfloat16*)t_lo, ldt, nseg))
            fail(OMM_ERR_UNSUPPORTED, "spmm_lowp_apply_f32: B (and B2, same pattern) must take the tensor-core path");
    } catch (const Error& e) {
        set_last_error(e.msg);
        return e.code;
    }
    set_last_error("");
    return OMM_OK;
}

extern "C" int omm_gpu_tc_errors(unsigned* bits) {
    try {
        unsigned e = gemm_bf16_errors();
        if (bits) *bits = e;
    } catch (const Error& e) {
        set_last_error(e.msg);
        return e.code;
    }
    set_last_error("");
    return OMM_OK;
}
