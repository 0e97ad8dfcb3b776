// Dense x CSC products (pspBLAS psp_gemspm local update, pspMspm_nn.F90:191-198;
// MatrixSwitch serial loop MatrixSwitch_mm_multiply.F90:263-327):
//     C(:, j) = beta*C(:, j) + alpha * sum_{l in column j of B} B_l * A(:, row_l)
// A is n x K column-major, so A(:, row) is a contiguous n-vector: every kernel
// here reads whole contiguous column segments of A (coalesced) and writes
// contiguous column segments of C.
//
// Two kernels:
//  * gather  : one CTA per (row chunk, output column); generic CSC.
//  * cgu     : "column-group union".  Output columns are cut into groups of G
//              consecutive columns; a group's nonzeros live in the union U_g
//              of their row indices, and the group is the dense product
//              A(:, U_g) * B_g with B_g the |U_g| x G block of B (zero filled).
//              For the block-sparse H and S of atom-centred bases (24 x 24
//              atom blocks, all columns of an atom share one pattern) the
//              union adds no fill at G = block size, and the product is a
//              register-tiled dense GEMM with K = |U_g|.  A second value array
//              with the same pattern (S beside H) is multiplied in the same
//              pass, so A is read once for both.
// The plan (groups, union rows, dense blocks) is built once per matrix on the
// host and kept on the device.
#include "internal.h"

#include <algorithm>
#include <atomic>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <numeric>
#include <thread>

namespace ommgpu {

struct SpmmPlan {
    int G = 0;          // group width
    int ngroups = 0;
    double efficiency = 0.0;  // nnz / sum(|U_g| * G)
    bool cgu = false;
    std::vector<int> h_gptr;    // ngroups+1 offsets into union rows
    std::vector<int> h_urows;   // union rows
    int maxK = 0;               // the largest union
    DevBuf gptr, urows;
    DevBuf bvals;               // sum(|U_g|*G) values, row-major per group (k, c)
    const msw_matrix* owner = nullptr;
    DevBuf bvals32;             // FP32 copy of bvals for the reduced-precision solver stages
};

namespace {

constexpr int kGatherThreads = 128;

__device__ inline zdbl zfma(zdbl a, zdbl b, zdbl c) {  // a*b + c
    return {fma(a.x, b.x, fma(-a.y, b.y, c.x)), fma(a.x, b.y, fma(a.y, b.x, c.y))};
}

template <typename T> struct Ar;
template <> struct Ar<double> {
    __device__ static double fmaa(double a, double b, double c) { return fma(a, b, c); }
    __device__ static double mulz(zdbl s, double v) { return s.x * v; }
    __device__ static double add(double a, double b) { return a + b; }
    __device__ static double zero() { return 0.0; }
};
template <> struct Ar<zdbl> {
    __device__ static zdbl fmaa(zdbl a, zdbl b, zdbl c) { return zfma(a, b, c); }
    __device__ static zdbl mulz(zdbl s, zdbl v) { return {s.x * v.x - s.y * v.y, s.x * v.y + s.y * v.x}; }
    __device__ static zdbl add(zdbl a, zdbl b) { return {a.x + b.x, a.y + b.y}; }
    __device__ static zdbl zero() { return {0.0, 0.0}; }
};

// C(r, j) = beta*C(r,j) + alpha*sum_l val_l*A(r, row_l); blockIdx.y = column j.
template <typename T>
__global__ void __launch_bounds__(kGatherThreads) gather_kernel(int n, const T* __restrict__ A, int lda,
                                                                  const int* __restrict__ colptr,
                                                                  const int* __restrict__ rowind,
                                                                  const T* __restrict__ val, T* __restrict__ C,
                                                                  int ldc, zdbl alpha, zdbl beta, int beta_zero) {
    constexpr int R = 4;  // rows per thread
    int j = blockIdx.y;
    int r0 = blockIdx.x * (kGatherThreads * R) + threadIdx.x;
    int s = colptr[j], e = colptr[j + 1];
    T acc[R];
#pragma unroll
    for (int q = 0; q < R; ++q) acc[q] = Ar<T>::zero();
    __shared__ int s_row[kGatherThreads];
    __shared__ T s_val[kGatherThreads];
    for (int base = s; base < e; base += kGatherThreads) {
        int cnt = min(kGatherThreads, e - base);
        __syncthreads();
        if (threadIdx.x < cnt) {
            s_row[threadIdx.x] = rowind[base + threadIdx.x];
            s_val[threadIdx.x] = val[base + threadIdx.x];
        }
        __syncthreads();
        for (int l = 0; l < cnt; ++l) {
            const T* a = A + (size_t)s_row[l] * lda;
            T v = s_val[l];
#pragma unroll
            for (int q = 0; q < R; ++q) {
                int r = r0 + q * kGatherThreads;
                if (r < n) acc[q] = Ar<T>::fmaa(a[r], v, acc[q]);
            }
        }
    }
#pragma unroll
    for (int q = 0; q < R; ++q) {
        int r = r0 + q * kGatherThreads;
        if (r < n) {
            T* c = C + r + (size_t)j * ldc;
            T out = Ar<T>::mulz(alpha, acc[q]);
            if (!beta_zero) out = Ar<T>::add(Ar<T>::mulz(beta, *c), out);
            *c = out;
        }
    }
}

// Column-group union kernel.  CTA = (row tile of BM = 16*TM rows, group g).
// 64 threads: tm in [0,16) covers rows tm + 16*i (i < TM), tn in [0,4) covers
// group columns tn*TN + q (q < TN).  NM = 1 or 2 value sets (fused H and S).
// The next K-chunk (BK union rows) is fetched into registers while the current
// one is multiplied out of shared memory.
template <typename T, int TM, int TN, int NM>
__global__ void __launch_bounds__(64) cgu_kernel(int n, int N, const T* __restrict__ A, int lda,
                                                 const int* __restrict__ gptr, const int* __restrict__ urows,
                                                 const T* __restrict__ B0, const T* __restrict__ B1,
                                                 T* __restrict__ C0, int ldc0, T* __restrict__ C1, int ldc1,
                                                 zdbl alpha, zdbl beta, int beta_zero) {
    constexpr int BM = 16 * TM;
    constexpr int G = 4 * TN;
    constexpr int BK = 8;
    constexpr int A_PER = BK * BM / 64;          // A elements per thread per chunk
    constexpr int B_PER = (BK * G + 63) / 64;    // B elements per thread per chunk and value set
    __shared__ T As[BK][BM];
    __shared__ T Bs[NM][BK][G];
    const int g = blockIdx.y;
    const int r0 = blockIdx.x * BM;
    const int tid = threadIdx.x;
    const int tm = tid & 15, tn = tid >> 4;
    const int k_begin = gptr[g], K = gptr[g + 1] - k_begin;
    const T* Bg[2] = {B0 + (size_t)k_begin * G, (NM == 2) ? B1 + (size_t)k_begin * G : nullptr};

    T acc[NM][TM][TN];
#pragma unroll
    for (int s = 0; s < NM; ++s)
#pragma unroll
        for (int i = 0; i < TM; ++i)
#pragma unroll
            for (int q = 0; q < TN; ++q) acc[s][i][q] = Ar<T>::zero();

    T ra[A_PER];
    T rb[NM][B_PER];
    auto fetch = [&](int k0) {
#pragma unroll
        for (int u = 0; u < A_PER; ++u) {
            int e = tid + 64 * u;
            int kk = e / BM, mm = e % BM;
            int r = r0 + mm;
            ra[u] = Ar<T>::zero();
            if (k0 + kk < K && r < n) ra[u] = A[(size_t)__ldg(urows + k_begin + k0 + kk) * lda + r];
        }
#pragma unroll
        for (int s = 0; s < NM; ++s)
#pragma unroll
            for (int u = 0; u < B_PER; ++u) {
                int e = tid + 64 * u;
                int kk = e / G;
                rb[s][u] = Ar<T>::zero();
                if (e < BK * G && k0 + kk < K) rb[s][u] = Bg[s][(size_t)k0 * G + e];
            }
    };
    auto stash = [&]() {
#pragma unroll
        for (int u = 0; u < A_PER; ++u) {
            int e = tid + 64 * u;
            As[e / BM][e % BM] = ra[u];
        }
#pragma unroll
        for (int s = 0; s < NM; ++s)
#pragma unroll
            for (int u = 0; u < B_PER; ++u) {
                int e = tid + 64 * u;
                if (e < BK * G) Bs[s][e / G][e % G] = rb[s][u];
            }
    };

    const int nk = (K + BK - 1) / BK;
    if (nk > 0) {
        fetch(0);
        stash();
        __syncthreads();
    }
    for (int t = 0; t < nk; ++t) {
        if (t + 1 < nk) fetch((t + 1) * BK);
#pragma unroll
        for (int kk = 0; kk < BK; ++kk) {
            T a[TM];
#pragma unroll
            for (int i = 0; i < TM; ++i) a[i] = As[kk][tm + 16 * i];
#pragma unroll
            for (int s = 0; s < NM; ++s) {
                T b[TN];
#pragma unroll
                for (int q = 0; q < TN; ++q) b[q] = Bs[s][kk][tn * TN + q];
#pragma unroll
                for (int i = 0; i < TM; ++i)
#pragma unroll
                    for (int q = 0; q < TN; ++q) acc[s][i][q] = Ar<T>::fmaa(a[i], b[q], acc[s][i][q]);
            }
        }
        __syncthreads();
        if (t + 1 < nk) {
            stash();
            __syncthreads();
        }
    }
#pragma unroll
    for (int s = 0; s < NM; ++s) {
        T* Cs = (s == 0) ? C0 : C1;
        int ldc = (s == 0) ? ldc0 : ldc1;
#pragma unroll
        for (int q = 0; q < TN; ++q) {
            int col = g * G + tn * TN + q;
            if (col >= N) continue;
#pragma unroll
            for (int i = 0; i < TM; ++i) {
                int r = r0 + tm + 16 * i;
                if (r >= n) continue;
                T* c = Cs + r + (size_t)col * ldc;
                T out = Ar<T>::mulz(alpha, acc[s][i][q]);
                if (!beta_zero) out = Ar<T>::add(Ar<T>::mulz(beta, *c), out);
                *c = out;
            }
        }
    }
}

// ---- FP64 column-group kernel on the FP64 tensor cores (mma.sync m8n8k4 f64; tcgen05 has no
// FP64 kind).  Per CTA 128 rows of A (4 warps x 32) x one column group (G = 8..32 columns, NM
// value sets).  K (the group's union rows) runs in 16-row chunks, double buffered with cp.async
// gathers of the union rows' column segments of A.  Per 4-k step a warp issues
// 4 (row tiles) x G/8 (column tiles) x NM DMMAs; the A fragments serve both value sets.
// Fragment layouts (m8n8k4, f64): A(r, k) at lane 4r + k, B(k, c) at lane 4c + k,
// D(r, 2q + i) at lane 4r + q, element i.
__device__ __forceinline__ void cp_async8(double* dst, const double* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)), "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait1() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait0() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }
__device__ __forceinline__ void dmma(double (&d)[2], double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(d[0]), "+d"(d[1])
                 : "d"(a), "d"(b));
}

constexpr int kDmmaBM = 128, kDmmaBK = 16, kDmmaAS = kDmmaBM + 8;  // A rows padded: fragment loads in 2 wavefronts
template <int G>
constexpr int dmma_gs() {
    return (G % 16 == 8) ? G : G + 8;  // B row stride with 2 * stride = 16 (mod 32) banks
}
template <int G, int NM>
constexpr int dmma_smem() {
    return 2 * (kDmmaBK * kDmmaAS + NM * kDmmaBK * dmma_gs<G>()) * (int)sizeof(double);
}

// stage_k: the group's union rows are staged in shared memory (after the operand buffers) once,
// so the gathers of every chunk index shared memory instead of waiting on global loads.
template <int G, int NM>
__global__ void __launch_bounds__(128) cgu_dmma_kernel(int n, int N, const double* __restrict__ A, int lda,
                                                       const int* __restrict__ gptr, const int* __restrict__ urows,
                                                       const double* __restrict__ B0, const double* __restrict__ B1,
                                                       double* __restrict__ C0, int ldc0, double* __restrict__ C1,
                                                       int ldc1, double alpha, double beta, int beta_zero,
                                                       int stage_k) {
    constexpr int BM = kDmmaBM, BK = kDmmaBK, AS = kDmmaAS, GS = dmma_gs<G>(), NT = G / 8;
    extern __shared__ double dsm[];
    double* As = dsm;                       // [2][BK][AS]
    double* Bs = dsm + 2 * BK * AS;         // [2][NM][BK][GS]
    int* s_ur = (int*)(dsm + dmma_smem<G, NM>() / (int)sizeof(double));  // [K] when stage_k
    const int g = blockIdx.y, r0 = blockIdx.x * BM;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int kb = gptr[g], K = gptr[g + 1] - kb;
    if (stage_k) {
        for (int i = threadIdx.x; i < K; i += blockDim.x) s_ur[i] = urows[kb + i];
        __syncthreads();
    }
    const int* ur = stage_k ? s_ur : urows + kb;
    const double* Bg[2] = {B0 + (size_t)kb * G, NM == 2 ? B1 + (size_t)kb * G : nullptr};

    double acc[NM][4][NT][2];
#pragma unroll
    for (int s = 0; s < NM; ++s)
#pragma unroll
        for (int mt = 0; mt < 4; ++mt)
#pragma unroll
            for (int nt = 0; nt < NT; ++nt) acc[s][mt][nt][0] = acc[s][mt][nt][1] = 0.0;

    auto load = [&](int stage, int k0) {
        double* as = As + stage * BK * AS;
#pragma unroll
        for (int u = 0; u < BK * BM / 128; ++u) {  // 16 column-segment elements per thread
            const int e = threadIdx.x + 128 * u;
            const int kk = e / BM, mm = e % BM;
            const int k = k0 + kk, r = r0 + mm;
            double* dst = as + kk * AS + mm;
            if (k < K && r < n) cp_async8(dst, A + (size_t)ur[k] * lda + r);
            else *dst = 0.0;
        }
        double* bs = Bs + stage * NM * BK * GS;
#pragma unroll
        for (int s = 0; s < NM; ++s)
            for (int e = threadIdx.x; e < BK * G; e += 128) {
                const int kk = e / G, c = e % G;
                double* dst = bs + (s * BK + kk) * GS + c;
                if (k0 + kk < K) cp_async8(dst, Bg[s] + (size_t)(k0 + kk) * G + c);
                else *dst = 0.0;
            }
    };

    const int nk = (K + BK - 1) / BK;
    if (nk > 0) load(0, 0);
    cp_async_commit();
    for (int t = 0; t < nk; ++t) {
        if (t + 1 < nk) load((t + 1) & 1, (t + 1) * BK);
        cp_async_commit();
        cp_async_wait1();  // chunk t has landed
        __syncthreads();
        const double* as = As + (t & 1) * BK * AS;
        const double* bs = Bs + (t & 1) * NM * BK * GS;
#pragma unroll
        for (int k4 = 0; k4 < BK; k4 += 4) {
            const int ka = k4 + (lane & 3);
            double af[4];
#pragma unroll
            for (int mt = 0; mt < 4; ++mt) af[mt] = as[ka * AS + warp * 32 + mt * 8 + (lane >> 2)];
#pragma unroll
            for (int s = 0; s < NM; ++s)
#pragma unroll
                for (int nt = 0; nt < NT; ++nt) {
                    const double bf = bs[(s * BK + ka) * GS + nt * 8 + (lane >> 2)];
#pragma unroll
                    for (int mt = 0; mt < 4; ++mt) dmma(acc[s][mt][nt], af[mt], bf);
                }
        }
        __syncthreads();  // the buffer is refilled by the next iteration's load
    }
    cp_async_wait0();
#pragma unroll
    for (int s = 0; s < NM; ++s) {
        double* Cs = s == 0 ? C0 : C1;
        const int ldc = s == 0 ? ldc0 : ldc1;
#pragma unroll
        for (int mt = 0; mt < 4; ++mt) {
            const int r = r0 + warp * 32 + mt * 8 + (lane >> 2);
            if (r >= n) continue;
#pragma unroll
            for (int nt = 0; nt < NT; ++nt)
#pragma unroll
                for (int i = 0; i < 2; ++i) {
                    const int col = g * G + nt * 8 + (lane & 3) * 2 + i;
                    if (col >= N) continue;
                    double* c = Cs + r + (size_t)col * ldc;
                    double out = alpha * acc[s][mt][nt][i];
                    if (!beta_zero) out += beta * *c;
                    *c = out;
                }
        }
    }
}

template <int G>
void launch_cgu_dmma(const DView& A, const SpmmPlan& P, const SpmmPlan* P2, DView& C, DView* C2, double al,
                     double be, int bz, int N) {
    dim3 grid((A.rows + kDmmaBM - 1) / kDmmaBM, P.ngroups);
    const int stage_k = (P.maxK > 0 && P.maxK <= 4096) ? 1 : 0;  // at most 16 KB of indices beside the buffers
    ktime_begin();
    const int extra = stage_k ? (P.maxK * (int)sizeof(int) + 15) / 16 * 16 : 0;
    if (P2) {
        const int SM = dmma_smem<G, 2>() + extra;
        static int attr = 0;
        if (SM > attr) {
            OMM_CK(cudaFuncSetAttribute(cgu_dmma_kernel<G, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, SM));
            attr = SM;
        }
        cgu_dmma_kernel<G, 2><<<grid, 128, SM, rt().stream>>>(A.rows, N, A.as<double>(), A.ld, P.gptr.as<int>(),
                                                                P.urows.as<int>(), P.bvals.as<double>(),
                                                                P2->bvals.as<double>(), C.as<double>(), C.ld,
                                                                C2->as<double>(), C2->ld, al, be, bz, stage_k);
    } else {
        const int SM = dmma_smem<G, 1>() + extra;
        static int attr = 0;
        if (SM > attr) {
            OMM_CK(cudaFuncSetAttribute(cgu_dmma_kernel<G, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, SM));
            attr = SM;
        }
        cgu_dmma_kernel<G, 1><<<grid, 128, SM, rt().stream>>>(A.rows, N, A.as<double>(), A.ld, P.gptr.as<int>(),
                                                                P.urows.as<int>(), P.bvals.as<double>(), nullptr,
                                                                C.as<double>(), C.ld, nullptr, 0, al, be, bz, stage_k);
    }
    OMM_KCHECK();
    // FP64 flops of the dense group blocks (= 2 nnz n per product for atom-block patterns)
    ktime_end("cgu_dmma_kernel", 2.0 * A.rows * (double)P.h_urows.size() * P.G * (P2 ? 2 : 1));
}

// FP32 variant of the column-group kernel for the reduced-precision solver stages:
// A and the group blocks in FP32, FP32 accumulation, FP64 output (C = A*B).
template <int TM, int TN, int NM>
__global__ void __launch_bounds__(64) cgu32_kernel(int n, int N, const float* __restrict__ A, int lda,
                                                   const int* __restrict__ gptr, const int* __restrict__ urows,
                                                   const float* __restrict__ B0, const float* __restrict__ B1,
                                                   double* __restrict__ C0, int ldc0, double* __restrict__ C1,
                                                   int ldc1) {
    constexpr int BM = 16 * TM;
    constexpr int G = 4 * TN;
    constexpr int BK = 8;
    constexpr int A_PER = BK * BM / 64;
    constexpr int B_PER = (BK * G + 63) / 64;
    __shared__ float As[BK][BM];
    __shared__ float Bs[NM][BK][G];
    const int g = blockIdx.y;
    const int r0 = blockIdx.x * BM;
    const int tid = threadIdx.x;
    const int tm = tid & 15, tn = tid >> 4;
    const int k_begin = gptr[g], K = gptr[g + 1] - k_begin;
    const float* Bg[2] = {B0 + (size_t)k_begin * G, (NM == 2) ? B1 + (size_t)k_begin * G : nullptr};
    float acc[NM][TM][TN];
#pragma unroll
    for (int s = 0; s < NM; ++s)
#pragma unroll
        for (int i = 0; i < TM; ++i)
#pragma unroll
            for (int q = 0; q < TN; ++q) acc[s][i][q] = 0.0f;
    float ra[A_PER];
    float rb[NM][B_PER];
    auto fetch = [&](int k0) {
#pragma unroll
        for (int u = 0; u < A_PER; ++u) {
            int e = tid + 64 * u;
            int kk = e / BM, mm = e % BM;
            int r = r0 + mm;
            ra[u] = 0.0f;
            if (k0 + kk < K && r < n) ra[u] = A[(size_t)__ldg(urows + k_begin + k0 + kk) * lda + r];
        }
#pragma unroll
        for (int s = 0; s < NM; ++s)
#pragma unroll
            for (int u = 0; u < B_PER; ++u) {
                int e = tid + 64 * u;
                rb[s][u] = 0.0f;
                if (e < BK * G && k0 + e / G < K) rb[s][u] = Bg[s][(size_t)k0 * G + e];
            }
    };
    auto stash = [&]() {
#pragma unroll
        for (int u = 0; u < A_PER; ++u) {
            int e = tid + 64 * u;
            As[e / BM][e % BM] = ra[u];
        }
#pragma unroll
        for (int s = 0; s < NM; ++s)
#pragma unroll
            for (int u = 0; u < B_PER; ++u) {
                int e = tid + 64 * u;
                if (e < BK * G) Bs[s][e / G][e % G] = rb[s][u];
            }
    };
    const int nk = (K + BK - 1) / BK;
    if (nk > 0) {
        fetch(0);
        stash();
        __syncthreads();
    }
    for (int t = 0; t < nk; ++t) {
        if (t + 1 < nk) fetch((t + 1) * BK);
#pragma unroll
        for (int kk = 0; kk < BK; ++kk) {
            float a[TM];
#pragma unroll
            for (int i = 0; i < TM; ++i) a[i] = As[kk][tm + 16 * i];
#pragma unroll
            for (int s = 0; s < NM; ++s) {
                float b[TN];
#pragma unroll
                for (int q = 0; q < TN; ++q) b[q] = Bs[s][kk][tn * TN + q];
#pragma unroll
                for (int i = 0; i < TM; ++i)
#pragma unroll
                    for (int q = 0; q < TN; ++q) acc[s][i][q] = fmaf(a[i], b[q], acc[s][i][q]);
            }
        }
        __syncthreads();
        if (t + 1 < nk) {
            stash();
            __syncthreads();
        }
    }
#pragma unroll
    for (int s = 0; s < NM; ++s) {
        double* Cs = (s == 0) ? C0 : C1;
        int ldc = (s == 0) ? ldc0 : ldc1;
#pragma unroll
        for (int q = 0; q < TN; ++q) {
            int col = g * G + tn * TN + q;
            if (col >= N) continue;
#pragma unroll
            for (int i = 0; i < TM; ++i) {
                int r = r0 + tm + 16 * i;
                if (r < n) Cs[r + (size_t)col * ldc] = (double)acc[s][i][q];
            }
        }
    }
}

__global__ void f64_to_f32_kernel(size_t n, const double* __restrict__ a, float* __restrict__ b) {
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x)
        b[e] = (float)a[e];
}

// ----------------------------------------------------------------------- plan
struct Candidate {
    int G;
    long long cells;
    std::vector<int> gptr, urows;
};

Candidate build_groups(const msw_matrix* B, int G) {
    Candidate c;
    c.G = G;
    int N = B->dim2;
    int ng = (N + G - 1) / G;
    c.gptr.assign(ng + 1, 0);
    std::vector<int> mark(B->dim1, -1);
    std::vector<int> rows;
    for (int g = 0; g < ng; ++g) {
        rows.clear();
        for (int j = g * G; j < std::min(N, (g + 1) * G); ++j)
            for (int l = B->h_colptr[j]; l < B->h_colptr[j + 1]; ++l) {
                int r = B->h_rowind[l];
                if (mark[r] != g) { mark[r] = g; rows.push_back(r); }
            }
        std::sort(rows.begin(), rows.end());
        c.urows.insert(c.urows.end(), rows.begin(), rows.end());
        c.gptr[g + 1] = (int)c.urows.size();
    }
    c.cells = (long long)c.urows.size() * G;
    return c;
}

// The plan is built once per matrix, but an SCF caller registers a new H every cycle, so the
// group blocks are filled on the device, from B's CSC arrays: one CTA per group, its union rows in shared
// memory, a warp per column whose lanes find each nonzero's row in the (ascending) union by binary
// search and add the value into its block cell (duplicate entries add up, as the reference's
// loops would sum them).
__device__ __forceinline__ void add_to(double* d, const double* v, long long l) { atomicAdd(d, v[l]); }
__device__ __forceinline__ void add_to(zdbl* d, const zdbl* v, long long l) {
    atomicAdd(&d->x, v[l].x);
    atomicAdd(&d->y, v[l].y);
}
template <typename T>
__global__ void __launch_bounds__(256) fill_blocks_kernel(int G, int N, const int* __restrict__ gptr,
                                                          const int* __restrict__ urows, const int* __restrict__ colptr,
                                                          const int* __restrict__ rowind, const T* __restrict__ val,
                                                          T* __restrict__ out) {
    extern __shared__ int su[];
    const int g = blockIdx.x, kb = gptr[g], nk = gptr[g + 1] - kb;
    for (int i = threadIdx.x; i < nk; i += blockDim.x) su[i] = urows[kb + i];
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int jj = warp; jj < G; jj += 8) {
        const int j = g * G + jj;
        if (j >= N) break;
        for (int l = colptr[j] + lane; l < colptr[j + 1]; l += 32) {
            const int r = rowind[l];
            int lo = 0, hi = nk - 1;
            while (lo < hi) {
                const int mid = (lo + hi) >> 1;
                if (su[mid] < r) lo = mid + 1;
                else hi = mid;
            }
            add_to(out + (size_t)(kb + lo) * G + jj, val, l);
        }
    }
}

void upload_blocks(const msw_matrix* B, SpmmPlan& P, DevBuf& dst) {
    // the group structure on the device (cgu plans upload it in finish_plan; others need it here)
    DevBuf gp, ur;
    const int* d_gptr = P.gptr.as<int>();
    const int* d_urows = P.urows.as<int>();
    if (!P.gptr.p) {
        gp.alloc(P.h_gptr.size() * sizeof(int));
        ur.alloc(std::max<size_t>(1, P.h_urows.size()) * sizeof(int));
        OMM_CK(cudaMemcpyAsync(gp.p, P.h_gptr.data(), P.h_gptr.size() * sizeof(int), cudaMemcpyHostToDevice,
                               rt().stream));
        if (!P.h_urows.empty())
            OMM_CK(cudaMemcpyAsync(ur.p, P.h_urows.data(), P.h_urows.size() * sizeof(int), cudaMemcpyHostToDevice,
                                   rt().stream));
        d_gptr = gp.as<int>();
        d_urows = ur.as<int>();
    }
    ensure_csc_device(B);
    const size_t cells = std::max<size_t>(1, P.h_urows.size() * (size_t)P.G);
    const int smem = std::max(1, P.maxK) * (int)sizeof(int);
    if (smem > 200 * 1024) fail(OMM_ERR_UNSUPPORTED, "spmm plan: a column group's row union is too long");
    if (B->is_real) {
        dst.alloc_zero(cells * sizeof(double));
        if (smem > 48 * 1024)
            OMM_CK(cudaFuncSetAttribute(fill_blocks_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        fill_blocks_kernel<double><<<P.ngroups, 256, smem, rt().stream>>>(
            P.G, B->dim2, d_gptr, d_urows, B->d_colptr.as<int>(), B->d_rowind.as<int>(), B->d_val.as<double>(),
            dst.as<double>());
    } else {
        dst.alloc_zero(cells * sizeof(zdbl));
        if (smem > 48 * 1024)
            OMM_CK(cudaFuncSetAttribute(fill_blocks_kernel<zdbl>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        fill_blocks_kernel<zdbl><<<P.ngroups, 256, smem, rt().stream>>>(P.G, B->dim2, d_gptr, d_urows,
                                                                       B->d_colptr.as<int>(), B->d_rowind.as<int>(),
                                                                       B->d_val.as<zdbl>(), dst.as<zdbl>());
    }
    OMM_KCHECK();
    OMM_CK(cudaStreamSynchronize(rt().stream));  // the temporary group structure goes out of scope
}

// Column groups of recently planned patterns, by content: a caller that registers a matrix
// with a pattern seen before (H and S of the same basis, or H afresh every SCF cycle) skips the
// search over group widths.  A hit needs equal dimensions, column pointers and row indices.
struct GroupsOfPattern {
    int dim1 = 0, dim2 = 0, nnz = 0;
    HostVec<int> colptr, rowind;
    int G = 0;
    double efficiency = 0.0;
    bool cgu = false;
    std::vector<int> gptr, urows;
};
std::mutex g_groups_mu;
std::deque<std::shared_ptr<const GroupsOfPattern>> g_groups;  // most recent first
constexpr size_t kGroupsKept = 2;

bool same_ints(const int* a, const int* b, long long n) {
    std::atomic<int> diff{0};
    host_parallel(n, [&](long long i0, long long i1) {
        if (std::memcmp(a + i0, b + i0, (size_t)(i1 - i0) * sizeof(int)) != 0) diff = 1;
    });
    return !diff;
}

std::shared_ptr<const GroupsOfPattern> find_groups(const msw_matrix* B) {
    std::deque<std::shared_ptr<const GroupsOfPattern>> kept;
    {
        std::lock_guard<std::mutex> lk(g_groups_mu);
        kept = g_groups;
    }
    for (auto& e : kept)
        if (e->dim1 == B->dim1 && e->dim2 == B->dim2 && e->nnz == B->nnz &&
            same_ints(e->colptr.data(), B->h_colptr.data(), (long long)B->dim2 + 1) &&
            same_ints(e->rowind.data(), B->h_rowind.data(), B->nnz))
            return e;
    return nullptr;
}

void keep_groups(const msw_matrix* B, const SpmmPlan& P) {
    auto e = std::make_shared<GroupsOfPattern>();
    e->dim1 = B->dim1;
    e->dim2 = B->dim2;
    e->nnz = B->nnz;
    e->colptr = B->h_colptr;
    e->rowind.resize(B->h_rowind.size());
    const int* src = B->h_rowind.data();
    int* dst = e->rowind.data();
    host_parallel((long long)B->h_rowind.size(), [&](long long i0, long long i1) {
        std::memcpy(dst + i0, src + i0, (size_t)(i1 - i0) * sizeof(int));
    });
    e->G = P.G;
    e->efficiency = P.efficiency;
    e->cgu = P.cgu;
    e->gptr = P.h_gptr;
    e->urows = P.h_urows;
    std::lock_guard<std::mutex> lk(g_groups_mu);
    g_groups.push_front(std::move(e));
    while (g_groups.size() > kGroupsKept) g_groups.pop_back();
}

void finish_plan(const msw_matrix* B, SpmmPlan& P);

SpmmPlan& get_plan(const msw_matrix* B) {
    msw_matrix* Bm = const_cast<msw_matrix*>(B);
    if (Bm->plan) return *Bm->plan;
    auto P = std::make_shared<SpmmPlan>();
    P->owner = B;
    if (auto hit = find_groups(B)) {
        P->G = hit->G;
        P->ngroups = (int)hit->gptr.size() - 1;
        P->efficiency = hit->efficiency;
        P->cgu = hit->cgu;
        P->h_gptr = hit->gptr;
        P->h_urows = hit->urows;
        finish_plan(B, *P);
        Bm->plan = P;
        return *P;
    }
    // choose the widest group width whose fill is within 5 % of the best one
    std::vector<Candidate> cands(4);
    {
        const int widths[4] = {8, 16, 24, 32};
        std::vector<std::thread> th;
        for (int i = 0; i < 4; ++i) th.emplace_back([&, i] { cands[i] = build_groups(B, widths[i]); });
        for (auto& t : th) t.join();
    }
    long long nnz = std::max(1, B->nnz);
    double best = 0.0;
    for (auto& c : cands) best = std::max(best, (double)nnz / std::max<long long>(1, c.cells));
    Candidate* pick = &cands[0];
    for (auto& c : cands) {
        double eff = (double)nnz / std::max<long long>(1, c.cells);
        if (eff >= 0.95 * best) pick = &c;
    }
    P->G = pick->G;
    P->ngroups = (int)pick->gptr.size() - 1;
    P->efficiency = (double)nnz / std::max<long long>(1, pick->cells);
    // the dense-union form pays off when most of its cells are real nonzeros and
    // columns are long enough for the tile loop
    double avg = (double)B->nnz / std::max(1, B->dim2);
    P->cgu = (P->efficiency >= 0.5) && (avg >= 16.0);
    P->h_gptr.swap(pick->gptr);
    P->h_urows.swap(pick->urows);
    finish_plan(B, *P);
    keep_groups(B, *P);
    Bm->plan = P;
    return *P;
}

void clear_kept_groups() {
    std::lock_guard<std::mutex> lk(g_groups_mu);
    g_groups.clear();
}

// device copies of the groups and the dense blocks of the values
void finish_plan(const msw_matrix* B, SpmmPlan& Pl) {
    SpmmPlan* P = &Pl;
    P->maxK = 0;
    for (size_t g = 0; g + 1 < P->h_gptr.size(); ++g) P->maxK = std::max(P->maxK, P->h_gptr[g + 1] - P->h_gptr[g]);
    if (P->cgu) {
        P->gptr.alloc(P->h_gptr.size() * sizeof(int));
        P->urows.alloc(std::max<size_t>(1, P->h_urows.size()) * sizeof(int));
        OMM_CK(cudaMemcpyAsync(P->gptr.p, P->h_gptr.data(), P->h_gptr.size() * sizeof(int), cudaMemcpyHostToDevice,
                               rt().stream));
        if (!P->h_urows.empty())
            OMM_CK(cudaMemcpyAsync(P->urows.p, P->h_urows.data(), P->h_urows.size() * sizeof(int),
                                   cudaMemcpyHostToDevice, rt().stream));
        upload_blocks(B, *P, P->bvals);
    }
}

template <typename T, int TM, int TN>
void launch_cgu(const DView& A, const SpmmPlan& P, const SpmmPlan* P2, DView& C, DView* C2, zdbl al, zdbl be,
                int bz, int N) {
    constexpr int BM = 16 * TM;
    dim3 grid((A.rows + BM - 1) / BM, P.ngroups);
    if (P2)
        cgu_kernel<T, TM, TN, 2><<<grid, 64, 0, rt().stream>>>(A.rows, N, A.as<T>(), A.ld, P.gptr.as<int>(),
                                                               P.urows.as<int>(), P.bvals.as<T>(), P2->bvals.as<T>(),
                                                               C.as<T>(), C.ld, C2->as<T>(), C2->ld, al, be, bz);
    else
        cgu_kernel<T, TM, TN, 1><<<grid, 64, 0, rt().stream>>>(A.rows, N, A.as<T>(), A.ld, P.gptr.as<int>(),
                                                               P.urows.as<int>(), P.bvals.as<T>(), nullptr,
                                                               C.as<T>(), C.ld, nullptr, 0, al, be, bz);
    OMM_KCHECK();
}

template <typename T, int TM>
void dispatch_cgu(int G, const DView& A, const SpmmPlan& P, const SpmmPlan* P2, DView& C, DView* C2, zdbl al,
                  zdbl be, int bz, int N) {
    switch (G) {
        case 8: launch_cgu<T, TM, 2>(A, P, P2, C, C2, al, be, bz, N); break;
        case 16: launch_cgu<T, TM, 4>(A, P, P2, C, C2, al, be, bz, N); break;
        case 24: launch_cgu<T, TM, 6>(A, P, P2, C, C2, al, be, bz, N); break;
        default: launch_cgu<T, TM, 8>(A, P, P2, C, C2, al, be, bz, N); break;
    }
}

}  // namespace

void spmm_plan_cache_clear() { clear_kept_groups(); }

unsigned long long next_pattern_id() {
    static std::atomic<unsigned long long> next{1};
    return next.fetch_add(1);
}

// Comparing two patterns walks nnz row indices (milliseconds at 10^7 nonzeros), and the
// solver asks once per CG step, so results are memoised by the pair of pattern ids.
bool same_pattern(const msw_matrix* A, const msw_matrix* B) {
    if (!A || !B || A->fmt != Fmt::CSC || B->fmt != Fmt::CSC) return false;
    if (A->dim1 != B->dim1 || A->dim2 != B->dim2 || A->nnz != B->nnz || A->is_real != B->is_real) return false;
    if (A == B) return true;
    static std::mutex mu;
    static std::map<std::pair<unsigned long long, unsigned long long>, bool> memo;
    auto key = std::minmax(A->pattern_id, B->pattern_id);
    {
        std::lock_guard<std::mutex> lk(mu);
        auto it = memo.find(key);
        if (it != memo.end()) return it->second;
    }
    const bool eq = A->h_colptr.size() == B->h_colptr.size() && A->h_rowind.size() == B->h_rowind.size() &&
                    same_ints(A->h_colptr.data(), B->h_colptr.data(), (long long)A->h_colptr.size()) &&
                    same_ints(A->h_rowind.data(), B->h_rowind.data(), (long long)A->h_rowind.size());
    std::lock_guard<std::mutex> lk(mu);
    if (memo.size() > 4096) memo.clear();
    memo[key] = eq;
    return eq;
}

void spmm_dense_csc_gather(const DView& A, const msw_matrix* B, DView& C, const double alpha[2],
                           const double beta[2]) {
    ensure_csc_device(B);
    int n = A.rows, N = B->dim2;
    if (n == 0 || N == 0) return;
    zdbl al{alpha[0], alpha[1]}, be{beta[0], beta[1]};
    int bz = (beta[0] == 0.0 && beta[1] == 0.0) ? 1 : 0;
    dim3 grid((n + kGatherThreads * 4 - 1) / (kGatherThreads * 4), N);
    if (A.is_real)
        gather_kernel<double><<<grid, kGatherThreads, 0, rt().stream>>>(n, A.as<double>(), A.ld, B->d_colptr.as<int>(),
                                                                        B->d_rowind.as<int>(), B->d_val.as<double>(),
                                                                        C.as<double>(), C.ld, al, be, bz);
    else
        gather_kernel<zdbl><<<grid, kGatherThreads, 0, rt().stream>>>(n, A.as<zdbl>(), A.ld, B->d_colptr.as<int>(),
                                                                      B->d_rowind.as<int>(), B->d_val.as<zdbl>(),
                                                                      C.as<zdbl>(), C.ld, al, be, bz);
    OMM_KCHECK();
}

void spmm_dense_csc(const DView& A, const msw_matrix* B, DView& C, const double alpha[2], const double beta[2],
                    const msw_matrix* B2, DView* C2) {
    if (A.rows == 0 || B->dim2 == 0) return;
    SpmmPlan& P = get_plan(B);
    bool fuse = B2 && C2 && same_pattern(B, B2);
    if (!P.cgu) {
        spmm_dense_csc_gather(A, B, C, alpha, beta);
        if (B2 && C2) spmm_dense_csc_gather(A, B2, *C2, alpha, beta);
        return;
    }
    SpmmPlan* P2 = nullptr;
    if (fuse) {
        msw_matrix* B2m = const_cast<msw_matrix*>(B2);
        if (!B2m->plan) {
            // same pattern: share the groups, fill the second value set
            auto Q = std::make_shared<SpmmPlan>();
            Q->G = P.G; Q->ngroups = P.ngroups; Q->efficiency = P.efficiency; Q->cgu = true; Q->maxK = P.maxK;
            Q->h_gptr = P.h_gptr; Q->h_urows = P.h_urows; Q->owner = B2;
            upload_blocks(B2, *Q, Q->bvals);
            B2m->plan = Q;
        }
        P2 = B2m->plan.get();
        if (P2->G != P.G || P2->h_gptr != P.h_gptr) fuse = false, P2 = nullptr;
    }
    zdbl al{alpha[0], alpha[1]}, be{beta[0], beta[1]};
    int bz = (beta[0] == 0.0 && beta[1] == 0.0) ? 1 : 0;
    if (A.is_real) {
        // FP64 tensor cores (DMMA)
        const SpmmPlan* Q = fuse ? P2 : nullptr;
        DView* C2f = fuse ? C2 : nullptr;
        switch (P.G) {
            case 8: launch_cgu_dmma<8>(A, P, Q, C, C2f, alpha[0], beta[0], bz, B->dim2); break;
            case 16: launch_cgu_dmma<16>(A, P, Q, C, C2f, alpha[0], beta[0], bz, B->dim2); break;
            case 24: launch_cgu_dmma<24>(A, P, Q, C, C2f, alpha[0], beta[0], bz, B->dim2); break;
            default: launch_cgu_dmma<32>(A, P, Q, C, C2f, alpha[0], beta[0], bz, B->dim2); break;
        }
    } else {
        // rows per thread chosen so that the accumulators of one or two value sets fit in registers
        if (fuse) dispatch_cgu<zdbl, 2>(P.G, A, P, P2, C, C2, al, be, bz, B->dim2);
        else dispatch_cgu<zdbl, 4>(P.G, A, P, nullptr, C, nullptr, al, be, bz, B->dim2);
    }
    if (B2 && C2 && !fuse) spmm_dense_csc(A, B2, *C2, alpha, beta);
}

namespace {
void ensure_f32_values(SpmmPlan& P) {
    if (P.bvals32.p) return;
    size_t cnt = P.bvals.bytes / sizeof(double);
    P.bvals32.alloc(std::max<size_t>(1, cnt) * sizeof(float));
    size_t b = std::min<size_t>((cnt + 255) / 256, 148 * 32);
    f64_to_f32_kernel<<<(int)std::max<size_t>(b, 1), 256, 0, rt().stream>>>(cnt, P.bvals.as<double>(),
                                                                             P.bvals32.as<float>());
    OMM_KCHECK();
}
template <int TM, int TN>
void launch_cgu32(const float* A, int lda, int n, const SpmmPlan& P, const SpmmPlan* P2, DView& C, DView* C2, int N) {
    constexpr int BM = 16 * TM;
    dim3 grid((n + BM - 1) / BM, P.ngroups);
    if (P2)
        cgu32_kernel<TM, TN, 2><<<grid, 64, 0, rt().stream>>>(n, N, A, lda, P.gptr.as<int>(), P.urows.as<int>(),
                                                              P.bvals32.as<float>(), P2->bvals32.as<float>(),
                                                              C.as<double>(), C.ld, C2->as<double>(), C2->ld);
    else
        cgu32_kernel<TM, TN, 1><<<grid, 64, 0, rt().stream>>>(n, N, A, lda, P.gptr.as<int>(), P.urows.as<int>(),
                                                              P.bvals32.as<float>(), nullptr, C.as<double>(), C.ld,
                                                              nullptr, 0);
    OMM_KCHECK();
}
}  // namespace

bool spmm32_available(const msw_matrix* B) { return B && B->fmt == Fmt::CSC && B->is_real && get_plan(B).cgu; }

// C (FP64) = A (FP32, n x K column-major) * B (CSC, FP32 values); fused second matrix when the
// patterns agree (B2 / C2).  Requires a column-group plan (spmm32_available).
void spmm32_dense_csc(const float* A, int lda, int n, const msw_matrix* B, DView& C, const msw_matrix* B2,
                      DView* C2) {
    SpmmPlan& P = get_plan(B);
    if (!P.cgu) fail(OMM_ERR_UNSUPPORTED, "spmm32: matrix has no column-group plan");
    ensure_f32_values(P);
    SpmmPlan* P2 = nullptr;
    if (B2 && C2 && same_pattern(B, B2)) {
        // second value set sharing the groups (built like spmm_dense_csc does)
        msw_matrix* B2m = const_cast<msw_matrix*>(B2);
        if (!B2m->plan) {
            auto Q = std::make_shared<SpmmPlan>();
            Q->G = P.G; Q->ngroups = P.ngroups; Q->efficiency = P.efficiency; Q->cgu = true; Q->maxK = P.maxK;
            Q->h_gptr = P.h_gptr; Q->h_urows = P.h_urows; Q->owner = B2;
            upload_blocks(B2, *Q, Q->bvals);
            B2m->plan = Q;
        }
        P2 = B2m->plan.get();
        if (P2->G != P.G || P2->h_gptr != P.h_gptr) P2 = nullptr;
        else ensure_f32_values(*P2);
    }
    int N = B->dim2;
    switch (P.G) {
        case 8: launch_cgu32<8, 2>(A, lda, n, P, P2, C, P2 ? C2 : nullptr, N); break;
        case 16: launch_cgu32<8, 4>(A, lda, n, P, P2, C, P2 ? C2 : nullptr, N); break;
        case 24: launch_cgu32<8, 6>(A, lda, n, P, P2, C, P2 ? C2 : nullptr, N); break;
        default: launch_cgu32<8, 8>(A, lda, n, P, P2, C, P2 ? C2 : nullptr, N); break;
    }
    if (B2 && C2 && !P2) spmm32_dense_csc(A, lda, n, B2, *C2, nullptr, nullptr);
}

SpmmPlanView spmm_plan_view(const msw_matrix* B) {
    SpmmPlan& P = get_plan(B);
    SpmmPlanView v;
    v.cgu = P.cgu;
    v.G = P.G;
    v.ngroups = P.ngroups;
    v.gptr = P.h_gptr.data();
    v.urows = P.h_urows.data();
    v.d_gptr = P.gptr.as<int>();
    v.d_bvals = P.bvals.as<double>();
    return v;
}

bool spmm_tc_available(const msw_matrix* B) {
    if (!B || B->fmt != Fmt::CSC || !B->is_real) return false;
    return spmm_tc_plan(B, spmm_plan_view(B)) != nullptr;
}

SpmmInfo spmm_info(const msw_matrix* B) {
    SpmmPlan& P = get_plan(B);
    return SpmmInfo{P.G, P.ngroups, P.efficiency, (long long)P.h_urows.size(), P.cgu};
}

}  // namespace ommgpu

extern "C" int omm_gpu_spmm_plan_info(const msw_matrix* B, int* G, int* ngroups, double* fill, int* column_groups) {
    using namespace ommgpu;
    try {
        if (!B || B->fmt != Fmt::CSC) fail(OMM_ERR_ARG, "spmm_plan_info: B must be a CSC matrix");
        SpmmInfo info = spmm_info(B);
        if (G) *G = info.group_width;
        if (ngroups) *ngroups = info.ngroups;
        if (fill) *fill = info.efficiency;
        if (column_groups) *column_groups = info.cgu ? 1 : 0;
    } catch (const Error& e) {
        set_last_error(e.msg);
        return e.code;
    }
    set_last_error("");
    return OMM_OK;
}

namespace ommgpu {

// psp_gemspm with every op combination (pspMspm.F90:58-120 dispatch to _nn/_nt/_tn/_tt):
// C = alpha*op(A)*op(B) + beta*C.  op(A) != 'n' is materialised with a transpose;
// op(B) != 'n' uses the CSC of B^T (conjugated values for 'c').
void gemspm(char opA, const DView& A, char opB, const msw_matrix* B, DView& C, const double alpha[2],
            const double beta[2]) {
    DevBuf tA;
    DView Aop = A;
    bool trA = !(opA == 'n' || opA == 'N');
    if (trA) {
        Aop.rows = A.cols;
        Aop.cols = A.rows;
        Aop.ld = A.cols;
        tA.alloc((size_t)Aop.rows * Aop.cols * (A.is_real ? 8 : 16));
        Aop.p = tA.p;
        transpose_into(A, opA, Aop);
    }
    const msw_matrix* Bop = B;
    if (!(opB == 'n' || opB == 'N')) {
        Bop = csc_transpose(B);
        if (!B->is_real && (opB == 'c' || opB == 'C')) {
            // conjugated copy of the transpose, kept beside it
            msw_matrix* Bm = const_cast<msw_matrix*>(B);
            if (!Bm->conj_transposed) {
                auto Cj = std::make_shared<msw_matrix>();
                Cj->dim1 = Bop->dim1; Cj->dim2 = Bop->dim2; Cj->is_real = false; Cj->fmt = Fmt::CSC;
                Cj->loc = Loc::Device; Cj->nnz = Bop->nnz;
                Cj->h_colptr = Bop->h_colptr; Cj->h_rowind = Bop->h_rowind; Cj->h_val = Bop->h_val;
                for (int l = 0; l < Cj->nnz; ++l) Cj->h_val[2 * l + 1] = -Cj->h_val[2 * l + 1];
                Bm->conj_transposed = Cj;
            }
            Bop = Bm->conj_transposed.get();
        }
    }
    spmm_dense_csc(Aop, Bop, C, alpha, beta);
}

// psp_gespmm (pspSpmm.F90:61-123): C = alpha*op(A)*op(B) + beta*C with A CSC.
// Evaluated as C^T = op(B)^T op(A)^T with the dense x CSC kernel, then transposed back.
void gespmm(char opA, const msw_matrix* A, char opB, const DView& B, DView& C, const double alpha[2],
            const double beta[2]) {
    // X = op(B)^T as a dense (N x K) matrix; for complex the conjugation rule
    // (op(B)^T)_{jk} = op(B)_{kj} is carried into a per-op choice below.
    bool real = B.is_real;
    int M = C.rows, N = C.cols;
    // op(B)^T: 'n' -> B^T, 't' -> B, 'c' -> conj(B)
    DevBuf tX, tY;
    DView X;
    X.is_real = real;
    bool bN = (opB == 'n' || opB == 'N'), bT = (opB == 't' || opB == 'T');
    if (bN) {
        X.rows = B.cols; X.cols = B.rows; X.ld = B.cols;
        tX.alloc((size_t)X.rows * X.cols * (real ? 8 : 16));
        X.p = tX.p;
        transpose_into(B, 't', X);
    } else if (bT || real) {
        X = B;
    } else {
        X.rows = B.rows; X.cols = B.cols; X.ld = B.rows;
        tX.alloc((size_t)X.rows * X.cols * 16);
        X.p = tX.p;
        // conj(B) = (B^H)^T: two transposes keep this on existing kernels
        DevBuf tmp;
        DView Th{nullptr, B.cols, B.rows, B.cols, false};
        tmp.alloc((size_t)B.rows * B.cols * 16);
        Th.p = tmp.p;
        transpose_into(B, 'c', Th);
        transpose_into(Th, 't', X);
    }
    // Y = op(A)^T as CSC: 'n' -> A^T, 't' -> A, 'c' -> conj(A)
    const msw_matrix* Y = A;
    std::shared_ptr<msw_matrix> conjA;
    bool aN = (opA == 'n' || opA == 'N'), aT = (opA == 't' || opA == 'T');
    if (aN) Y = csc_transpose(A);
    else if (!aT && !A->is_real) {
        conjA = std::make_shared<msw_matrix>();
        *conjA = msw_matrix();
        conjA->dim1 = A->dim1; conjA->dim2 = A->dim2; conjA->is_real = false; conjA->fmt = Fmt::CSC;
        conjA->nnz = A->nnz; conjA->h_colptr = A->h_colptr; conjA->h_rowind = A->h_rowind; conjA->h_val = A->h_val;
        for (int l = 0; l < conjA->nnz; ++l) conjA->h_val[2 * l + 1] = -conjA->h_val[2 * l + 1];
        Y = conjA.get();
    }
    // Z = X * Y  (N x M), then C = alpha*Z^T + beta*C
    DView Z{nullptr, N, M, N, real};
    tY.alloc((size_t)N * M * (real ? 8 : 16));
    Z.p = tY.p;
    double one[2] = {1.0, 0.0}, zero[2] = {0.0, 0.0};
    spmm_dense_csc_gather(X, Y, Z, one, zero);
    k_axpby(Z, 't', C, alpha, beta);
}

}  // namespace ommgpu
