// Elementwise, reduction and initialisation kernels of the libOMM CG loop, plus
// the cuBLAS wrapper used for the FP64 dense products.
//
// All matrices are column-major views (pointer, rows, cols, leading dimension).
// Real matrices are double, complex ones zdbl (interleaved re, im).
#include "internal.h"

#include <cmath>

namespace ommgpu {

namespace {

constexpr int kThreads = 256;

__host__ __device__ inline zdbl zmul(zdbl a, zdbl b) { return {a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x}; }
__host__ __device__ inline zdbl zadd(zdbl a, zdbl b) { return {a.x + b.x, a.y + b.y}; }
__host__ __device__ inline zdbl zconj(zdbl a) { return {a.x, -a.y}; }

// ---- generic scalar helpers: real matrices use only the .x part of the complex scalars
template <typename T> struct Sc;
template <> struct Sc<double> {
    __device__ static double load(const double* p, size_t i) { return p[i]; }
    __device__ static void store(double* p, size_t i, double v) { p[i] = v; }
    __device__ static double conj(double v) { return v; }
    __device__ static double mul(zdbl a, double v) { return a.x * v; }
    __device__ static double add(double a, double b) { return a + b; }
    __device__ static double from(zdbl a) { return a.x; }
};
template <> struct Sc<zdbl> {
    __device__ static zdbl load(const zdbl* p, size_t i) { return p[i]; }
    __device__ static void store(zdbl* p, size_t i, zdbl v) { p[i] = v; }
    __device__ static zdbl conj(zdbl v) { return zconj(v); }
    __device__ static zdbl mul(zdbl a, zdbl v) { return zmul(a, v); }
    __device__ static zdbl add(zdbl a, zdbl b) { return zadd(a, b); }
    __device__ static zdbl from(zdbl a) { return a; }
};

inline int grid_for(size_t elems, int per_thread = 4) {
    size_t b = (elems + (size_t)kThreads * per_thread - 1) / ((size_t)kThreads * per_thread);
    if (b < 1) b = 1;
    if (b > 148 * 32) b = 148 * 32;
    return (int)b;
}

// C = beta*C + alpha*op(A)  (MatrixSwitch_m_add.F90:95-175: C=beta*C first, then += alpha*op(A))
template <typename T>
__global__ void axpby_kernel(int rows, int cols, const T* __restrict__ A, int lda, int op, T* __restrict__ C, int ldc,
                             zdbl alpha, zdbl beta, int beta_zero) {
    size_t total = (size_t)rows * cols;
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
        int i = (int)(e % rows), j = (int)(e / rows);
        T a;
        if (op == 0) a = A[i + (size_t)j * lda];
        else if (op == 1) a = A[j + (size_t)i * lda];
        else a = Sc<T>::conj(A[j + (size_t)i * lda]);
        T c = beta_zero ? T{} : Sc<T>::mul(beta, C[i + (size_t)j * ldc]);
        C[i + (size_t)j * ldc] = Sc<T>::add(c, Sc<T>::mul(alpha, a));
    }
}

template <typename T>
__global__ void scale_kernel(int rows, int cols, T* C, int ldc, zdbl beta) {
    size_t total = (size_t)rows * cols;
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
        int i = (int)(e % rows), j = (int)(e / rows);
        C[i + (size_t)j * ldc] = Sc<T>::mul(beta, C[i + (size_t)j * ldc]);
    }
}

// m_set (MatrixSwitch_m_set.F90:19-75): lu 0 all, 1 upper (j>=i), 2 lower (j<=i)
template <typename T>
__global__ void set_kernel(int rows, int cols, T* C, int ldc, int lu, zdbl alpha, zdbl beta) {
    size_t total = (size_t)rows * cols;
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
        int i = (int)(e % rows), j = (int)(e / rows);
        if (lu == 1 && j < i) continue;
        if (lu == 2 && j > i) continue;
        C[i + (size_t)j * ldc] = Sc<T>::from(i == j ? beta : alpha);
    }
}

template <typename T>
__global__ void set_element_kernel(T* C, size_t idx, zdbl alpha, zdbl beta) {
    C[idx] = Sc<T>::add(Sc<T>::from(alpha), Sc<T>::mul(beta, C[idx]));
}

// C(j,i) = conj(C(i,j)) for j > i  (omm_ops.F90:483-487 / :590-594).  One 32 x 32 tile of the
// lower triangle per block, its source tile of the upper triangle staged through shared memory
// so that both the reads and the writes run down columns (coalesced).
template <typename T>
__global__ void fill_lower_kernel(int n, T* C, int ldc) {
    const int bi = blockIdx.x, bj = blockIdx.y;  // destination tile: rows 32*bi.., columns 32*bj..
    if (bi < bj) return;
    __shared__ T tile[32][33];
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 32 x 8
    for (int yy = ty; yy < 32; yy += 8) {
        int r = 32 * bj + tx, c = 32 * bi + yy;  // source C(r, c) in the upper triangle
        if (r < n && c < n) tile[yy][tx] = C[r + (size_t)c * ldc];
    }
    __syncthreads();
    for (int yy = ty; yy < 32; yy += 8) {
        int r = 32 * bi + tx, c = 32 * bj + yy;  // destination C(r, c) = conj(C(c, r))
        if (r < n && c < n && r > c) C[r + (size_t)c * ldc] = Sc<T>::conj(tile[tx][yy]);
    }
}

// W += x*(Wd^H + Wd) + x^2*Wdd  (omm.F90:499-501, :514-516, :168-170), applied as the
// reference's three m_add calls in order.
template <typename T>
__global__ void w_update_kernel(int n, T* W, int ldw, const T* Wd, int ldd, const T* Wdd, int lddd, double x) {
    size_t total = (size_t)n * n;
    zdbl xz{x, 0.0}, x2{x * x, 0.0};
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
        int i = (int)(e % n), j = (int)(e / n);
        T w = W[i + (size_t)j * ldw];
        w = Sc<T>::add(w, Sc<T>::mul(xz, Sc<T>::conj(Wd[j + (size_t)i * ldd])));
        w = Sc<T>::add(w, Sc<T>::mul(xz, Wd[i + (size_t)j * ldd]));
        w = Sc<T>::add(w, Sc<T>::mul(x2, Wdd[i + (size_t)j * lddd]));
        W[i + (size_t)j * ldw] = w;
    }
}

// ---- reference C0: BSD LCG under NORAND (omm_rand.F90:19-55), element order of
// omm.F90:331-341: element e = j + i*n (column-major) uses draws 2e+1 and 2e+2.
__device__ inline void lcg_jump(unsigned long long t, unsigned long long& A, unsigned long long& Cc) {
    // affine map x -> a x + c (mod 2^31) raised to the power t
    const unsigned long long M = (1ull << 31) - 1;  // mask
    unsigned long long ra = 1, rc = 0;              // result map
    unsigned long long ba = 1103515245ull, bc = 12345ull;
    while (t) {
        if (t & 1ull) {  // result = base o result
            rc = (ba * rc + bc) & M;
            ra = (ba * ra) & M;
        }
        // base = base o base
        bc = (ba * bc + bc) & M;
        ba = (ba * ba) & M;
        t >>= 1;
    }
    A = ra;
    Cc = rc;
}
template <typename T>
__global__ void lcg_kernel(int n, int m, T* C, int ldc, double scale) {
    size_t total = (size_t)n * m;
    const unsigned long long M = (1ull << 31) - 1;
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
        unsigned long long A, Cc;
        lcg_jump(2ull * e + 1ull, A, Cc);
        unsigned long long x1 = (A * 123456ull + Cc) & M;
        unsigned long long x2 = (1103515245ull * x1 + 12345ull) & M;
        double r1 = (double)x1 / 2147483648.0, r2 = (double)x2 / 2147483648.0;
        double h = 0.5 * r1;
        double el = (r2 - 0.5 >= 0.0) ? fabs(h) : -fabs(h);
        el = el * scale;
        int j = (int)(e % n), i = (int)(e / n);
        zdbl v{el, 0.0};
        C[j + (size_t)i * ldc] = Sc<T>::from(v);
    }
}

// ---- reductions ------------------------------------------------------------------
template <int K>
__device__ inline void block_reduce_store(double (&v)[K], double* out) {
    __shared__ double sm[K][kThreads / 32];
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < K; ++k) {
        double a = v[k];
        for (int o = 16; o > 0; o >>= 1) a += __shfl_down_sync(0xffffffffu, a, o);
        if (lane == 0) sm[k][w] = a;
    }
    __syncthreads();
    if (threadIdx.x < K) {
        double s = 0.0;
        for (int i = 0; i < (int)(blockDim.x / 32); ++i) s += sm[threadIdx.x][i];
        out[(size_t)blockIdx.x * K + threadIdx.x] = s;
    }
}

// (s, c) + (s2, c2) for compensated sums: s + s2 split exactly into t + e (Knuth's TwoSum),
// the rounding errors carried in c
__device__ inline void comp_add(double& s, double& c, double s2, double c2) {
    const double t = s + s2, z = t - s;
    const double e = (s - (t - z)) + (s2 - z);
    s = t;
    c += c2 + e;
}

// Final pass: one block sums nb partial records of K values with compensation, in a fixed order
// (each thread a strided share, then a tree over the warp's lanes, then the warps in turn), so
// the result does not depend on timing.
template <int K>
__global__ void final_reduce_kernel(const double* part, int nb, double* out) {
    __shared__ double s_sum[K][kThreads / 32], s_cmp[K][kThreads / 32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    double s[K], c[K];
#pragma unroll
    for (int k = 0; k < K; ++k) s[k] = c[k] = 0.0;
    for (int b = threadIdx.x; b < nb; b += blockDim.x)
#pragma unroll
        for (int k = 0; k < K; ++k) comp_add(s[k], c[k], part[(size_t)b * K + k], 0.0);
#pragma unroll
    for (int k = 0; k < K; ++k) {
        for (int o = 16; o > 0; o >>= 1) {
            const double s2 = __shfl_down_sync(0xffffffffu, s[k], o), c2 = __shfl_down_sync(0xffffffffu, c[k], o);
            comp_add(s[k], c[k], s2, c2);
        }
        if (lane == 0) {
            s_sum[k][w] = s[k];
            s_cmp[k][w] = c[k];
        }
    }
    __syncthreads();
    if (threadIdx.x < K) {
        const int k = threadIdx.x;
        double S = 0.0, C = 0.0;
        for (int i = 0; i < (int)(blockDim.x / 32); ++i) comp_add(S, C, s_sum[k][i], s_cmp[k][i]);
        out[k] = S + C;
    }
}

template <typename T>
__device__ inline void dot_acc(T a, T b, double& re, double& im);
template <>
__device__ inline void dot_acc<double>(double a, double b, double& re, double&) { re += a * b; }
template <>
__device__ inline void dot_acc<zdbl>(zdbl a, zdbl b, double& re, double& im) {
    re += a.x * b.x + a.y * b.y;  // conj(a)*b
    im += a.x * b.y - a.y * b.x;
}

template <typename T>
__global__ void dot_kernel(int rows, int cols, const T* A, int lda, const T* B, int ldb, double* part) {
    double v[2] = {0.0, 0.0};
    size_t total = (size_t)rows * cols;
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
        int i = (int)(e % rows), j = (int)(e / rows);
        dot_acc<T>(A[i + (size_t)j * lda], B[i + (size_t)j * ldb], v[0], v[1]);
    }
    block_reduce_store<2>(v, part);
}

template <typename T>
__global__ void trace_kernel(int n, const T* A, int lda, double* part) {
    double v[2] = {0.0, 0.0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        T a = A[i + (size_t)i * lda];
        zdbl z;
        if constexpr (sizeof(T) == 8) { z.x = *(const double*)&a; z.y = 0.0; }
        else { z = *(const zdbl*)&a; }
        v[0] += z.x;
        v[1] += z.y;
    }
    block_reduce_store<2>(v, part);
}

// The 13 traces of calc_coeff (omm_ops.F90:194-211) in one pass over the six n x n
// matrices.  TrHdSd needs SWd^H, read through a shared-memory transposed tile.
// Index: 0 TrH 1 TrHS 2 TrHd 3 TrHdS 4 TrHSd 5 TrHdd 6 TrHddS 7 TrHSdd 8 TrHdSd
//        9 TrHdSdH 10 TrHddSd 11 TrHdSdd 12 TrHddSdd
template <typename T>
__device__ inline double re_dot(T a, T b) {
    double re = 0.0, im = 0.0;
    dot_acc<T>(a, b, re, im);
    return re;
}
template <typename T>
__device__ inline double re_of(T a) {
    if constexpr (sizeof(T) == 8) return *(const double*)&a;
    else return ((const zdbl*)&a)->x;
}
template <typename T>
__global__ void coeff_kernel(int n, const T* HW, int l0, const T* SW, int l1, const T* HWd, int l2, const T* SWd,
                             int l3, const T* HWdd, int l4, const T* SWdd, int l5, double* part) {
    __shared__ T tileT[32][33];
    double v[13];
#pragma unroll
    for (int k = 0; k < 13; ++k) v[k] = 0.0;
    int tiles = (n + 31) / 32;
    int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 32 x 8
    for (int t = blockIdx.x; t < tiles * tiles; t += gridDim.x) {
        int bi = t % tiles, bj = t / tiles;
        // load SWd tile (rows bj*32.., cols bi*32..) so that tileT[c][r] = SWd(bj*32+r, bi*32+c)
        __syncthreads();
        for (int yy = ty; yy < 32; yy += 8) {
            int r = bj * 32 + tx, c = bi * 32 + yy;
            T val{};
            if (r < n && c < n) val = SWd[r + (size_t)c * l3];
            tileT[yy][tx] = val;
        }
        __syncthreads();
        for (int yy = ty; yy < 32; yy += 8) {
            int i = bi * 32 + tx, j = bj * 32 + yy;
            if (i >= n || j >= n) continue;
            T hw = HW[i + (size_t)j * l0], sw = SW[i + (size_t)j * l1], hwd = HWd[i + (size_t)j * l2];
            T swd = SWd[i + (size_t)j * l3], hwdd = HWdd[i + (size_t)j * l4], swdd = SWdd[i + (size_t)j * l5];
            T swdT = tileT[tx][yy];  // SWd(j, i)
            if (i == j) {
                v[0] += re_of(hw);
                v[2] += re_of(hwd);
                v[5] += re_of(hwdd);
            }
            v[1] += re_dot(hw, sw);
            v[3] += re_dot(sw, hwd);
            v[4] += re_dot(hw, swd);
            v[6] += re_dot(hwdd, sw);
            v[7] += re_dot(hw, swdd);
            v[8] += re_dot(Sc<T>::conj(swdT), hwd);  // mm_trace(SWd^H, HWd): conj((SWd^H)_ij) = SWd_ji
            v[9] += re_dot(swd, hwd);
            v[10] += re_dot(hwdd, swd);
            v[11] += re_dot(swdd, hwd);
            v[12] += re_dot(hwdd, swdd);
        }
    }
    block_reduce_store<13>(v, part);
}

template <typename T>
__global__ void lambda_kernel(int rows, int cols, const T* PG, int l0, const T* G, int l1, const T* Gp, int l2,
                              const T* PGp, int l3, double* part) {
    double v[2] = {0.0, 0.0};
    size_t total = (size_t)rows * cols;
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
        int i = (int)(e % rows), j = (int)(e / rows);
        T g = G[i + (size_t)j * l1], gp = Gp[i + (size_t)j * l2];
        T w2;
        if constexpr (sizeof(T) == 8) w2 = g - gp;
        else w2 = zdbl{((zdbl*)&g)->x - ((zdbl*)&gp)->x, ((zdbl*)&g)->y - ((zdbl*)&gp)->y};
        v[0] += re_dot(PG[i + (size_t)j * l0], w2);  // mm_trace(PG, work2), work2 = G - G_p
        v[1] += re_dot(PGp[i + (size_t)j * l3], gp); // mm_trace(PG_p, G_p)
    }
    block_reduce_store<2>(v, part);
}

template <typename T>
__global__ void transpose_kernel(int rows, int cols, const T* A, int lda, int conj, T* Tm, int ldt) {
    // Tm (cols x rows) = op(A), A rows x cols
    __shared__ T tile[32][33];
    int bx = blockIdx.x * 32, by = blockIdx.y * 32;
    int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    for (int yy = ty; yy < 32; yy += 8) {
        int r = bx + tx, c = by + yy;
        if (r < rows && c < cols) tile[yy][tx] = A[r + (size_t)c * lda];
    }
    __syncthreads();
    for (int yy = ty; yy < 32; yy += 8) {
        int r = by + tx, c = bx + yy;  // Tm(r, c) = A(c, r)
        if (r < cols && c < rows) {
            T v = tile[tx][yy];
            Tm[r + (size_t)c * ldt] = conj ? Sc<T>::conj(v) : v;
        }
    }
}

inline int op_code(char op) {
    if (op == 'n' || op == 'N') return 0;
    if (op == 't' || op == 'T') return 1;
    if (op == 'c' || op == 'C') return 2;
    fail(OMM_ERR_ARG, std::string("process_opM: invalid opM '") + op + "'");
}

double* scratch_partials(size_t nrec, int K) {
    rt().scratch.ensure((nrec * K + 64) * sizeof(double));
    return rt().scratch.as<double>();
}

template <int K>
void finish_reduce(double* part, int nb, double* out) {
    double* res = part + (size_t)nb * K;  // result slot right after the partials
    final_reduce_kernel<K><<<1, kThreads, 0, rt().stream>>>(part, nb, res);
    OMM_KCHECK();
    OMM_CK(cudaMemcpyAsync(rt().host_pinned, res, K * sizeof(double), cudaMemcpyDeviceToHost, rt().stream));
    sync();
    for (int k = 0; k < K; ++k) out[k] = rt().host_pinned[k];
}

}  // namespace

// ------------------------------------------------------------------ host wrappers
void k_axpby(const DView& A, char op, DView& C, const double alpha[2], const double beta[2]) {
    int oc = op_code(op);
    if (A.is_real && oc == 2) oc = 1;
    size_t tot = (size_t)C.rows * C.cols;
    if (tot == 0) return;
    zdbl a{alpha[0], alpha[1]}, b{beta[0], beta[1]};
    int bz = 0;  // the reference multiplies C by beta even when beta == 0 (NaN propagates); keep that
    if (C.is_real)
        axpby_kernel<double><<<grid_for(tot), kThreads, 0, rt().stream>>>(C.rows, C.cols, A.as<double>(), A.ld, oc,
                                                                            C.as<double>(), C.ld, a, b, bz);
    else
        axpby_kernel<zdbl><<<grid_for(tot), kThreads, 0, rt().stream>>>(C.rows, C.cols, A.as<zdbl>(), A.ld, oc,
                                                                          C.as<zdbl>(), C.ld, a, b, bz);
    OMM_KCHECK();
}

void k_scale(DView& C, const double beta[2]) {
    size_t tot = (size_t)C.rows * C.cols;
    if (tot == 0) return;
    zdbl b{beta[0], beta[1]};
    if (C.is_real) scale_kernel<double><<<grid_for(tot), kThreads, 0, rt().stream>>>(C.rows, C.cols, C.as<double>(), C.ld, b);
    else scale_kernel<zdbl><<<grid_for(tot), kThreads, 0, rt().stream>>>(C.rows, C.cols, C.as<zdbl>(), C.ld, b);
    OMM_KCHECK();
}

void k_set(DView& C, char seC, const double alpha[2], const double beta[2]) {
    int lu = (seC == 'u' || seC == 'U') ? 1 : (seC == 'l' || seC == 'L') ? 2 : 0;  // process_seM
    size_t tot = (size_t)C.rows * C.cols;
    if (tot == 0) return;
    zdbl a{alpha[0], alpha[1]}, b{beta[0], beta[1]};
    if (C.is_real) set_kernel<double><<<grid_for(tot), kThreads, 0, rt().stream>>>(C.rows, C.cols, C.as<double>(), C.ld, lu, a, b);
    else set_kernel<zdbl><<<grid_for(tot), kThreads, 0, rt().stream>>>(C.rows, C.cols, C.as<zdbl>(), C.ld, lu, a, b);
    OMM_KCHECK();
}

void k_set_element(DView& C, int i, int j, const double alpha[2], const double beta[2]) {
    size_t idx = (size_t)i + (size_t)j * C.ld;
    zdbl a{alpha[0], alpha[1]}, b{beta[0], beta[1]};
    if (C.is_real) set_element_kernel<double><<<1, 1, 0, rt().stream>>>(C.as<double>(), idx, a, b);
    else set_element_kernel<zdbl><<<1, 1, 0, rt().stream>>>(C.as<zdbl>(), idx, a, b);
    OMM_KCHECK();
}

void k_fill_lower_from_upper(DView& C) {
    if (C.rows == 0) return;
    int nt = (C.rows + 31) / 32;
    dim3 grid(nt, nt);
    if (C.is_real) fill_lower_kernel<double><<<grid, kThreads, 0, rt().stream>>>(C.rows, C.as<double>(), C.ld);
    else fill_lower_kernel<zdbl><<<grid, kThreads, 0, rt().stream>>>(C.rows, C.as<zdbl>(), C.ld);
    OMM_KCHECK();
}

void k_w_update(DView& W, const DView& Wd, const DView& Wdd, double x) {
    size_t tot = (size_t)W.rows * W.rows;
    if (W.is_real)
        w_update_kernel<double><<<grid_for(tot), kThreads, 0, rt().stream>>>(W.rows, W.as<double>(), W.ld,
                                                                               Wd.as<double>(), Wd.ld,
                                                                               Wdd.as<double>(), Wdd.ld, x);
    else
        w_update_kernel<zdbl><<<grid_for(tot), kThreads, 0, rt().stream>>>(W.rows, W.as<zdbl>(), W.ld, Wd.as<zdbl>(),
                                                                             Wd.ld, Wdd.as<zdbl>(), Wdd.ld, x);
    OMM_KCHECK();
}

void k_lcg_init(DView& C) {
    // the scale 1e-2/sqrt(m) of omm.F90:342 is applied by the caller through m_scale
    size_t tot = (size_t)C.rows * C.cols;
    if (C.is_real) lcg_kernel<double><<<grid_for(tot), kThreads, 0, rt().stream>>>(C.rows, C.cols, C.as<double>(), C.ld, 1.0);
    else lcg_kernel<zdbl><<<grid_for(tot), kThreads, 0, rt().stream>>>(C.rows, C.cols, C.as<zdbl>(), C.ld, 1.0);
    OMM_KCHECK();
}

void r_trace(const DView& A, double out[2]) {
    int nb = 64;
    double* part = scratch_partials(nb + 1, 2);
    if (A.is_real) trace_kernel<double><<<nb, kThreads, 0, rt().stream>>>(A.rows, A.as<double>(), A.ld, part);
    else trace_kernel<zdbl><<<nb, kThreads, 0, rt().stream>>>(A.rows, A.as<zdbl>(), A.ld, part);
    OMM_KCHECK();
    finish_reduce<2>(part, nb, out);
}

void r_dot(const DView& A, const DView& B, double out[2]) {
    size_t tot = (size_t)A.rows * A.cols;
    int nb = grid_for(tot, 8);
    double* part = scratch_partials(nb + 1, 2);
    if (A.is_real)
        dot_kernel<double><<<nb, kThreads, 0, rt().stream>>>(A.rows, A.cols, A.as<double>(), A.ld, B.as<double>(), B.ld, part);
    else
        dot_kernel<zdbl><<<nb, kThreads, 0, rt().stream>>>(A.rows, A.cols, A.as<zdbl>(), A.ld, B.as<zdbl>(), B.ld, part);
    OMM_KCHECK();
    finish_reduce<2>(part, nb, out);
}

void r_coeff(const DView& HW, const DView& SW, const DView& HWd, const DView& SWd, const DView& HWdd, const DView& SWdd,
             double coeff[5]) {
    int n = HW.rows;
    int tiles = (n + 31) / 32;
    int nb = tiles * tiles;
    if (nb > 148 * 8) nb = 148 * 8;
    double* part = scratch_partials(nb + 1, 13);
    if (HW.is_real)
        coeff_kernel<double><<<nb, kThreads, 0, rt().stream>>>(n, HW.as<double>(), HW.ld, SW.as<double>(), SW.ld,
                                                                 HWd.as<double>(), HWd.ld, SWd.as<double>(), SWd.ld,
                                                                 HWdd.as<double>(), HWdd.ld, SWdd.as<double>(),
                                                                 SWdd.ld, part);
    else
        coeff_kernel<zdbl><<<nb, kThreads, 0, rt().stream>>>(n, HW.as<zdbl>(), HW.ld, SW.as<zdbl>(), SW.ld,
                                                               HWd.as<zdbl>(), HWd.ld, SWd.as<zdbl>(), SWd.ld,
                                                               HWdd.as<zdbl>(), HWdd.ld, SWdd.as<zdbl>(), SWdd.ld,
                                                               part);
    OMM_KCHECK();
    double t[13];
    finish_reduce<13>(part, nb, t);
    // omm_ops.F90:213-217
    coeff[0] = 2.0 * t[0] - t[1];
    coeff[1] = 2.0 * (2.0 * t[2] - t[3] - t[4]);
    coeff[2] = 2.0 * (t[5] - t[8] - t[9]) - t[6] - t[7];
    coeff[3] = -2.0 * (t[10] + t[11]);
    coeff[4] = -t[12];
}

void r_lambda(const DView& PG, const DView& G, const DView& Gp, const DView& PGp, double out[2]) {
    size_t tot = (size_t)G.rows * G.cols;
    int nb = grid_for(tot, 8);
    double* part = scratch_partials(nb + 1, 2);
    if (G.is_real)
        lambda_kernel<double><<<nb, kThreads, 0, rt().stream>>>(G.rows, G.cols, PG.as<double>(), PG.ld, G.as<double>(),
                                                                  G.ld, Gp.as<double>(), Gp.ld, PGp.as<double>(),
                                                                  PGp.ld, part);
    else
        lambda_kernel<zdbl><<<nb, kThreads, 0, rt().stream>>>(G.rows, G.cols, PG.as<zdbl>(), PG.ld, G.as<zdbl>(), G.ld,
                                                                Gp.as<zdbl>(), Gp.ld, PGp.as<zdbl>(), PGp.ld, part);
    OMM_KCHECK();
    finish_reduce<2>(part, nb, out);
}

void gemm(char opA, char opB, int M, int N, int K, const double alpha[2], const DView& A, const DView& B,
          const double beta[2], DView& C) {
    auto cop = [&](char o, bool real) {
        int c = op_code(o);
        if (c == 0) return CUBLAS_OP_N;
        if (c == 1 || real) return CUBLAS_OP_T;
        return CUBLAS_OP_C;
    };
    if (M == 0 || N == 0) return;
    if (C.is_real && fp64_emu_enabled() && fp64_emu_worth(M, N, K)) {
        // FP64-accurate product on the int8 tensor cores (ozaki.cu); 'c' is 't' for real data
        gemm_f64_emu(op_code(opA) ? 't' : 'n', op_code(opB) ? 't' : 'n', M, N, K, alpha[0], A, B, beta[0], C);
        return;
    }
    if (!C.is_real && alpha[1] == 0.0 && beta[1] == 0.0 && fp64_emu_enabled() && fp64_emu_worth(M, N, K)) {
        // complex, as four real products of the parts
        const char ops[3] = {'n', 't', 'c'};
        gemm_z_emu(ops[op_code(opA)], ops[op_code(opB)], M, N, K, alpha[0], A, B, beta[0], C);
        return;
    }
    OMM_CKB(cublasSetStream(rt().blas, rt().stream));
    if (C.is_real) {
        OMM_CKB(cublasDgemm(rt().blas, cop(opA, true), cop(opB, true), M, N, K, &alpha[0], A.as<double>(), A.ld,
                            B.as<double>(), B.ld, &beta[0], C.as<double>(), C.ld));
    } else {
        cuDoubleComplex a = make_cuDoubleComplex(alpha[0], alpha[1]), b = make_cuDoubleComplex(beta[0], beta[1]);
        OMM_CKB(cublasZgemm(rt().blas, cop(opA, false), cop(opB, false), M, N, K, &a, A.as<cuDoubleComplex>(), A.ld,
                            B.as<cuDoubleComplex>(), B.ld, &b, C.as<cuDoubleComplex>(), C.ld));
    }
}

void transpose_into(const DView& A, char op, DView& Tm) {
    int oc = op_code(op);
    if (oc == 0) {  // plain copy
        double one[2] = {1.0, 0.0}, zero[2] = {0.0, 0.0};
        k_axpby(A, 'n', Tm, one, zero);
        return;
    }
    dim3 grid((A.rows + 31) / 32, (A.cols + 31) / 32);
    if (A.is_real)
        transpose_kernel<double><<<grid, kThreads, 0, rt().stream>>>(A.rows, A.cols, A.as<double>(), A.ld, 0,
                                                                      Tm.as<double>(), Tm.ld);
    else
        transpose_kernel<zdbl><<<grid, kThreads, 0, rt().stream>>>(A.rows, A.cols, A.as<zdbl>(), A.ld, oc == 2,
                                                                    Tm.as<zdbl>(), Tm.ld);
    OMM_KCHECK();
}

}  // namespace ommgpu
