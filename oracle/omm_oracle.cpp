// ============================================================================
// TEST INFRASTRUCTURE — NOT PART OF THE PRODUCT.
//
// CPU FP64 restatement of libOMM's omm() conjugate-gradient solver and of the
// MatrixSwitch / pspBLAS operations it drives, used only as the parity checker
// for the GPU library (tests/, __graft_entry__.smoke(), and the cpu_baseline /
// reference arm of bench.py).  The product path never calls this file.
//
// Parity pins (checked by tests/test_oracle_golden.py):
//   * libOMM/examples/example_gamma.F90:51-53   e_min, D_11, ED_11 (tol 1e-4)
//   * libOMM/examples/example_kpoints.F90:66-70 complex, 2 k-points (tol 1e-4)
//   * MatrixSwitch/examples/example_sdden.F90:43-44 traces/products (tol 1e-10)
//
// Dense BLAS/LAPACK calls go to the host OpenBLAS that SciPy bundles
// (symbols scipy_dgemm_, scipy_dpotrf_, ...), resolved with dlopen at
// orc_init().  Every routine cites the reference file:line it restates.
// ============================================================================
#include <complex>
#include <vector>
#include <string>
#include <cmath>
#include <cstring>
#include <cstdio>
#include <cstdint>
#include <dlfcn.h>
#include <atomic>
#include <thread>

typedef std::complex<double> zc;

// ---------------------------------------------------------------------------
// BLAS / LAPACK entry points (Fortran calling convention, LP64).
// Trailing size_t arguments are the hidden Fortran string lengths.
// ---------------------------------------------------------------------------
typedef void (*gemm_d_t)(const char*, const char*, const int*, const int*, const int*, const double*,
                         const double*, const int*, const double*, const int*, const double*, double*,
                         const int*, size_t, size_t);
typedef void (*gemm_z_t)(const char*, const char*, const int*, const int*, const int*, const zc*, const zc*,
                         const int*, const zc*, const int*, const zc*, zc*, const int*, size_t, size_t);
typedef void (*potrf_d_t)(const char*, const int*, double*, const int*, int*, size_t);
typedef void (*potrf_z_t)(const char*, const int*, zc*, const int*, int*, size_t);
typedef void (*sygst_d_t)(const int*, const char*, const int*, double*, const int*, const double*, const int*,
                          int*, size_t);
typedef void (*sygst_z_t)(const int*, const char*, const int*, zc*, const int*, const zc*, const int*, int*,
                          size_t);
typedef void (*trmm_d_t)(const char*, const char*, const char*, const char*, const int*, const int*,
                         const double*, const double*, const int*, double*, const int*, size_t, size_t, size_t,
                         size_t);
typedef void (*trmm_z_t)(const char*, const char*, const char*, const char*, const int*, const int*, const zc*,
                         const zc*, const int*, zc*, const int*, size_t, size_t, size_t, size_t);
typedef double (*dot_d_t)(const int*, const double*, const int*, const double*, const int*);
typedef void (*sytrf_d_t)(const char*, const int*, double*, const int*, int*, double*, const int*, int*, size_t);
typedef void (*sytrf_z_t)(const char*, const int*, zc*, const int*, int*, zc*, const int*, int*, size_t);
typedef void (*sytri_d_t)(const char*, const int*, double*, const int*, const int*, double*, int*, size_t);
typedef void (*sytri_z_t)(const char*, const int*, zc*, const int*, const int*, zc*, int*, size_t);
typedef void (*setnt_t)(int);

static struct {
    void* h = nullptr;
    gemm_d_t dgemm; gemm_z_t zgemm;
    potrf_d_t dpotrf; potrf_z_t zpotrf;
    sygst_d_t dsygst; sygst_z_t zhegst;
    trmm_d_t dtrmm, dtrsm; trmm_z_t ztrmm, ztrsm;
    dot_d_t ddot;
    sytrf_d_t dsytrf; sytrf_z_t zhetrf;
    sytri_d_t dsytri; sytri_z_t zhetri;
    setnt_t set_threads;
} L;

static thread_local std::string g_err;
static int g_threads = 1;

// Split [0, n) over g_threads host threads in interleaved chunks of 16.
template <typename F>
static void parallel_for(int n, F&& f) {
    int nt = g_threads > 1 ? g_threads : 1;
    if (nt == 1 || n < 64) {
        for (int i = 0; i < n; ++i) f(i);
        return;
    }
    std::atomic<int> next(0);
    auto work = [&]() {
        for (;;) {
            int s = next.fetch_add(16);
            if (s >= n) break;
            int e = s + 16 < n ? s + 16 : n;
            for (int i = s; i < e; ++i) f(i);
        }
    };
    std::vector<std::thread> th;
    for (int t = 1; t < nt; ++t) th.emplace_back(work);
    work();
    for (auto& t : th) t.join();
}

struct OrcDie {
    std::string msg;
};
[[noreturn]] static void die(const std::string& m) { throw OrcDie{m}; }

// ---------------------------------------------------------------------------
// Matrix type (restates MatrixSwitch_ops.F90:62-97 for the 'sden'/'scsc'
// storage used here).  Dense data is column-major; CSC indices are 0-based
// column offsets (like MatrixSwitch's iaux4) and 0-based row indices.
// Dense matrices may alias caller memory (m_register_sden semantics,
// MatrixSwitch_m_register.F90:129).
// ---------------------------------------------------------------------------
template <typename T>
struct Mat {
    bool init = false;
    bool csc = false;
    int d1 = 0, d2 = 0;
    std::vector<T> own;
    T* p = nullptr;  // dense values (col-major) or CSC values
    int nnz = 0;
    const int* cp = nullptr;  // CSC column offsets (d2+1)
    const int* ri = nullptr;  // CSC row indices
    std::vector<int> own_cp, own_ri;  // owned pattern (a CSC made here, e.g. the PW preconditioner)
    T& operator()(int i, int j) { return p[(size_t)i + (size_t)j * d1]; }
    const T& operator()(int i, int j) const { return p[(size_t)i + (size_t)j * d1]; }
    size_t size() const { return (size_t)d1 * d2; }
};

template <typename T>
static void m_allocate(Mat<T>& M, int i, int j) {  // MatrixSwitch.F90:312-419 (zero filled)
    M.d1 = i; M.d2 = j; M.csc = false;
    M.own.assign((size_t)i * j, T(0));
    M.p = M.own.data();
    M.init = true;
}
template <typename T>
static void m_deallocate(Mat<T>& M) {
    M.own.clear(); M.own.shrink_to_fit(); M.p = nullptr; M.init = false;
}

static inline double conj_(double x) { return x; }
static inline zc conj_(zc x) { return std::conj(x); }
static inline double re_(double x) { return x; }
static inline double re_(zc x) { return x.real(); }

// op(A)(i,k) accessor for 'n','t','c' (MatrixSwitch_ops.F90:129-185)
template <typename T>
static inline T opel(const Mat<T>& A, char op, int i, int k) {
    if (op == 'n' || op == 'N') return A(i, k);
    if (op == 't' || op == 'T') return A(k, i);
    return conj_(A(k, i));
}
static inline bool is_tr(char op) {
    if (op == 'n' || op == 'N') return false;
    if (op == 't' || op == 'T' || op == 'c' || op == 'C') return true;
    die("process_opM: invalid opM");
}

// ---------------------------------------------------------------------------
// BLAS wrappers
// ---------------------------------------------------------------------------
static void gemm(char ta, char tb, int m, int n, int k, double al, const double* a, int lda, const double* b, int ldb,
                 double be, double* c, int ldc) {
    if (ta == 'c' || ta == 'C') ta = 't';
    if (tb == 'c' || tb == 'C') tb = 't';
    L.dgemm(&ta, &tb, &m, &n, &k, &al, a, &lda, b, &ldb, &be, c, &ldc, 1, 1);
}
static void gemm(char ta, char tb, int m, int n, int k, zc al, const zc* a, int lda, const zc* b, int ldb, zc be,
                 zc* c, int ldc) {
    L.zgemm(&ta, &tb, &m, &n, &k, &al, a, &lda, b, &ldb, &be, c, &ldc, 1, 1);
}

// ---------------------------------------------------------------------------
// mm_multiply  (MatrixSwitch.F90:1046-1390 dispatch)
//   dense x dense : 'lap' -> dgemm/zgemm (MatrixSwitch.F90:1303, :1645)
//   dense x CSC   : MatrixSwitch_mm_multiply.F90:263-327 (psp_gemspm local
//                   update pspMspm_nn.F90:191-198 is the same arithmetic)
//   CSC x dense   : MatrixSwitch_mm_multiply.F90:192-256 (pspSpmm_nn.F90)
// C = alpha*op(A)*op(B) + beta*C
// ---------------------------------------------------------------------------
template <typename T>
static void mm_multiply(const Mat<T>& A, char opA, const Mat<T>& B, char opB, Mat<T>& C, T alpha, T beta) {
    bool trA = is_tr(opA), trB = is_tr(opB);
    int Ar = trA ? A.d2 : A.d1, Ac = trA ? A.d1 : A.d2;
    int Br = trB ? B.d2 : B.d1, Bc = trB ? B.d1 : B.d2;
    if (Ar != C.d1 || Bc != C.d2 || Ac != Br) die("mm_multiply: matrices A, B and C are not compatible");
    if (!A.csc && !B.csc) {
        gemm(opA, opB, C.d1, C.d2, Ac, alpha, A.p, A.d1, B.p, B.d1, beta, C.p, C.d1);
        return;
    }
    // sparse products: C=beta*C, then accumulate nonzero by nonzero
    for (size_t e = 0; e < C.size(); ++e) C.p[e] = beta * C.p[e];
    if (!A.csc && B.csc && !trA && !trB) {
        // the omm() case C*H: column j of C gathers columns of A (pspMspm_nn.F90:191-198);
        // output columns are independent, so they are split over host threads.
        parallel_for(B.d2, [&](int j) {
            T* cj = C.p + (size_t)j * C.d1;
            for (int l = B.cp[j]; l < B.cp[j + 1]; ++l) {
                const T* ak = A.p + (size_t)B.ri[l] * A.d1;
                const T v = B.p[l];
                for (int i = 0; i < C.d1; ++i) cj[i] += alpha * ak[i] * v;
            }
        });
    } else if (!A.csc && B.csc) {
        bool cj = (opB == 'c' || opB == 'C');
        for (int c = 0; c < B.d2; ++c)
            for (int l = B.cp[c]; l < B.cp[c + 1]; ++l) {
                int r = B.ri[l];
                T v = cj ? conj_(B.p[l]) : B.p[l];
                int k = trB ? c : r, j = trB ? r : c;  // op(B)(k,j)
                for (int i = 0; i < C.d1; ++i) C(i, j) += alpha * opel(A, opA, i, k) * v;
            }
    } else if (A.csc && !B.csc) {
        bool cj = (opA == 'c' || opA == 'C');
        for (int c = 0; c < A.d2; ++c)
            for (int l = A.cp[c]; l < A.cp[c + 1]; ++l) {
                int r = A.ri[l];
                T v = cj ? conj_(A.p[l]) : A.p[l];
                int i = trA ? c : r, k = trA ? r : c;  // op(A)(i,k)
                for (int j = 0; j < C.d2; ++j) C(i, j) += alpha * v * opel(B, opB, k, j);
            }
    } else {
        die("mm_multiply: invalid implementation");
    }
}

// m_add: C = beta*C + alpha*op(A)  (MatrixSwitch_m_add.F90:95-175; CSC->dense :182-222)
template <typename T>
static void m_add(const Mat<T>& A, char opA, Mat<T>& C, T alpha, T beta) {
    bool trA = is_tr(opA);
    if (!trA ? (A.d1 != C.d1 || A.d2 != C.d2) : (A.d1 != C.d2 || A.d2 != C.d1))
        die("m_add: matrices A and C are not compatible");
    for (size_t e = 0; e < C.size(); ++e) C.p[e] = beta * C.p[e];
    if (A.csc) {
        bool cj = (opA == 'c' || opA == 'C');
        for (int c = 0; c < A.d2; ++c)
            for (int l = A.cp[c]; l < A.cp[c + 1]; ++l) {
                int r = A.ri[l];
                T v = cj ? conj_(A.p[l]) : A.p[l];
                if (!trA) C(r, c) += alpha * v; else C(c, r) += alpha * v;
            }
        return;
    }
    if (!trA) {
        for (size_t e = 0; e < C.size(); ++e) C.p[e] = C.p[e] + alpha * A.p[e];
    } else {
        for (int i = 0; i < C.d1; ++i)
            for (int j = 0; j < C.d2; ++j) C(i, j) = C(i, j) + alpha * opel(A, opA, i, j);
    }
}

// m_scale: C = beta*C (MatrixSwitch.F90:2496-2621)
template <typename T>
static void m_scale(Mat<T>& C, T beta) {
    for (size_t e = 0; e < C.size(); ++e) C.p[e] = beta * C.p[e];
}

// m_set(C,'a',alpha,beta): off-diagonal alpha, diagonal beta (MatrixSwitch_m_set.F90:19-75)
template <typename T>
static void m_set_all(Mat<T>& C, T alpha, T beta) {
    for (int j = 0; j < C.d2; ++j)
        for (int i = 0; i < C.d1; ++i) C(i, j) = (i == j) ? beta : alpha;
}

// m_trace: real part of sum of the diagonal (MatrixSwitch.F90:2060-2156 + CONV)
template <typename T>
static double m_trace(const Mat<T>& A) {
    if (A.d1 != A.d2) die("m_trace: matrix A is not square");
    T a = T(0);
    for (int i = 0; i < A.d1; ++i) a = a + A(i, i);
    return re_(a);
}

// mm_trace: Re sum_ij conj(A_ij)*B_ij (MatrixSwitch.F90:2336-2356 'lap' ddot; :2466-2471 complex)
static double mm_trace(const Mat<double>& A, const Mat<double>& B) {
    if (A.d1 != B.d1 || A.d2 != B.d2) die("mm_trace: matrices A and B are not compatible");
    int nn = A.d1 * A.d2, one = 1;
    return L.ddot(&nn, A.p, &one, B.p, &one);
}
static double mm_trace(const Mat<zc>& A, const Mat<zc>& B) {
    if (A.d1 != B.d1 || A.d2 != B.d2) die("mm_trace: matrices A and B are not compatible");
    zc a(0, 0);
    for (int i = 0; i < A.d1; ++i)
        for (int j = 0; j < A.d2; ++j) a = a + std::conj(A(i, j)) * B(i, j);
    return a.real();
}

// ---------------------------------------------------------------------------
// libOMM building blocks (libOMM/src/omm_ops.F90)
// ---------------------------------------------------------------------------
// calc_G: G = 4*HC - 2*SW*HC - 2*HW*SC  (omm_ops.F90:17-39)
template <typename T>
static void calc_G(const Mat<T>& HW, const Mat<T>& SW, Mat<T>& G, const Mat<T>& HC, const Mat<T>& SC) {
    m_add(HC, 'n', G, T(4.0), T(0.0));
    mm_multiply(SW, 'n', HC, 'n', G, T(-2.0), T(1.0));
    mm_multiply(HW, 'n', SC, 'n', G, T(-2.0), T(1.0));
}
// calc_AW: AC = C*A ; AW = AC*C^H  (omm_ops.F90:44-64)
template <typename T>
static void calc_AW(const Mat<T>& A, const Mat<T>& C, Mat<T>& AW, Mat<T>& AC) {
    mm_multiply(C, 'n', A, 'n', AC, T(1.0), T(0.0));
    mm_multiply(AC, 'n', C, 'c', AW, T(1.0), T(0.0));
}
// calc_A: CAW = AW*C1 ; A = C1^H*CAW  (omm_ops.F90:104-124)
template <typename T>
static void calc_A(const Mat<T>& AW, const Mat<T>& C1, Mat<T>& A, Mat<T>& CAW) {
    mm_multiply(AW, 'n', C1, 'n', CAW, T(1.0), T(0.0));
    mm_multiply(C1, 'c', CAW, 'n', A, T(1.0), T(0.0));
}
// calc_A2: CAW = AW*C2 ; A = C1^H*CAW  (omm_ops.F90:129-150)
template <typename T>
static void calc_A2(const Mat<T>& AW, const Mat<T>& C1, const Mat<T>& C2, Mat<T>& A, Mat<T>& CAW) {
    mm_multiply(AW, 'n', C2, 'n', CAW, T(1.0), T(0.0));
    mm_multiply(C1, 'c', CAW, 'n', A, T(1.0), T(0.0));
}
// calc_coeff: 13 traces -> quartic coefficients (omm_ops.F90:156-219)
template <typename T>
static void calc_coeff(const Mat<T>& HW, const Mat<T>& SW, const Mat<T>& HWd, const Mat<T>& SWd, const Mat<T>& HWdd,
                       const Mat<T>& SWdd, Mat<T>& SWdH, double coeff[5]) {
    double TrH = m_trace(HW);
    double TrHS = mm_trace(HW, SW);
    double TrHd = m_trace(HWd);
    double TrHdS = mm_trace(SW, HWd);
    double TrHSd = mm_trace(HW, SWd);
    double TrHdd = m_trace(HWdd);
    double TrHddS = mm_trace(HWdd, SW);
    double TrHSdd = mm_trace(HW, SWdd);
    m_add(SWd, 'c', SWdH, T(1.0), T(0.0));
    double TrHdSd = mm_trace(SWdH, HWd);
    double TrHdSdH = mm_trace(SWd, HWd);
    double TrHddSd = mm_trace(HWdd, SWd);
    double TrHdSdd = mm_trace(SWdd, HWd);
    double TrHddSdd = mm_trace(HWdd, SWdd);
    coeff[0] = 2.0 * TrH - TrHS;
    coeff[1] = 2.0 * (2.0 * TrHd - TrHdS - TrHSd);
    coeff[2] = 2.0 * (TrHdd - TrHdSd - TrHdSdH) - TrHddS - TrHSdd;
    coeff[3] = -2.0 * (TrHddSd + TrHdSdd);
    coeff[4] = -TrHddSdd;
}

// m_factorize: S = U^H*U, dpotrf('u') (omm_ops.F90:225-384, :301, :370)
static void m_factorize(Mat<double>& C) {
    if (C.csc) die("m_dfactorize: invalid implementation");
    int n = C.d1, info = 0;
    L.dpotrf("u", &n, C.p, &n, &info, 1);
    if (info != 0) die("m_dfactorize: error in dpotrf");
}
static void m_factorize(Mat<zc>& C) {
    if (C.csc) die("m_zfactorize: invalid implementation");
    int n = C.d1, info = 0;
    L.zpotrf("u", &n, C.p, &n, &info, 1);
    if (info != 0) die("m_zfactorize: error in zpotrf");
}
// m_reduce: C := U^-H*C*U^-1 then fill lower triangle (omm_ops.F90:481-487, :588-594)
static void m_reduce(const Mat<double>& A, Mat<double>& C) {
    if (C.csc || A.csc) die("m_dreduce: invalid implementation");
    int n = C.d1, one = 1, info = 0;
    L.dsygst(&one, "u", &n, C.p, &n, A.p, &n, &info, 1);
    if (info != 0) die("m_dreduce: error in dsygst");
    for (int i = 0; i < n - 1; ++i)
        for (int j = i + 1; j < n; ++j) C(j, i) = C(i, j);
}
static void m_reduce(const Mat<zc>& A, Mat<zc>& C) {
    if (C.csc || A.csc) die("m_zreduce: invalid implementation");
    int n = C.d1, one = 1, info = 0;
    L.zhegst(&one, "u", &n, C.p, &n, A.p, &n, &info, 1);
    if (info != 0) die("m_zreduce: error in zhegst");
    for (int i = 0; i < n - 1; ++i)
        for (int j = i + 1; j < n; ++j) C(j, i) = std::conj(C(i, j));
}
// m_transform: C := C*U^H, dtrmm('r','u','t','n') (omm_ops.F90:718, :786)
static void m_transform(const Mat<double>& A, Mat<double>& C) {
    double one = 1.0;
    L.dtrmm("r", "u", "t", "n", &C.d1, &C.d2, &one, A.p, &A.d1, C.p, &C.d1, 1, 1, 1, 1);
}
static void m_transform(const Mat<zc>& A, Mat<zc>& C) {
    zc one(1.0, 0.0);
    L.ztrmm("r", "u", "c", "n", &C.d1, &C.d2, &one, A.p, &A.d1, C.p, &C.d1, 1, 1, 1, 1);
}
// m_back_transform: C := C*U^-H, dtrsm('r','u','t','n') (omm_ops.F90:885)
static void m_back_transform(const Mat<double>& A, Mat<double>& C) {
    double one = 1.0;
    L.dtrsm("r", "u", "t", "n", &C.d1, &C.d2, &one, A.p, &A.d1, C.p, &C.d1, 1, 1, 1, 1);
}
static void m_back_transform(const Mat<zc>& A, Mat<zc>& C) {
    zc one(1.0, 0.0);
    L.ztrsm("r", "u", "c", "n", &C.d1, &C.d2, &one, A.p, &A.d1, C.p, &C.d1, 1, 1, 1, 1);
}
// m_inverse: dsytrf/dsytri('u') + fill lower (omm_ops.F90:1059-1076; complex zhetrf/zhetri)
static void m_inverse(Mat<double>& C) {
    int n = C.d1, info = 0, lw = -1;
    std::vector<int> ipiv(n);
    double wq;
    L.dsytrf("u", &n, C.p, &n, ipiv.data(), &wq, &lw, &info, 1);
    lw = (int)wq > n ? (int)wq : n;
    std::vector<double> w(lw);
    L.dsytrf("u", &n, C.p, &n, ipiv.data(), w.data(), &lw, &info, 1);
    if (info != 0) die("m_dinverse: error in dsytrf");
    L.dsytri("u", &n, C.p, &n, ipiv.data(), w.data(), &info, 1);
    if (info != 0) die("m_dinverse: error in dsytri");
    for (int i = 0; i < n - 1; ++i)
        for (int j = i + 1; j < n; ++j) C(j, i) = C(i, j);
}
static void m_inverse(Mat<zc>& C) {
    int n = C.d1, info = 0, lw = -1;
    std::vector<int> ipiv(n);
    zc wq;
    L.zhetrf("u", &n, C.p, &n, ipiv.data(), &wq, &lw, &info, 1);
    lw = (int)wq.real() > n ? (int)wq.real() : n;
    std::vector<zc> w(lw);
    L.zhetrf("u", &n, C.p, &n, ipiv.data(), w.data(), &lw, &info, 1);
    if (info != 0) die("m_zinverse: error in zhetrf");
    L.zhetri("u", &n, C.p, &n, ipiv.data(), w.data(), &info, 1);
    if (info != 0) die("m_zinverse: error in zhetri");
    for (int i = 0; i < n - 1; ++i)
        for (int j = i + 1; j < n; ++j) C(j, i) = std::conj(C(i, j));
}

// ---------------------------------------------------------------------------
// omm_solve_quartic (libOMM/src/omm_quartic.F90:60-153)
// ---------------------------------------------------------------------------
static const double OMM_PI = 3.141592653589793238462643383279502884197;
static double fsign(double a, double b) { return b >= 0.0 ? std::fabs(a) : -std::fabs(a); }

static void omm_solve_quartic(const double c[5], double* x_min, bool* fail) {
    *fail = false;
    double a = 3.0 * c[3] / (4.0 * c[4]);
    double b = 2.0 * c[2] / (4.0 * c[4]);
    if ((std::fabs(b) >= 1.0e11) || (std::fabs(c[4]) <= 1.0e-11)) {
        *x_min = -0.5 * c[1] / c[2];
        return;
    }
    double d = c[1] / (4.0 * c[4]);
    double Q = (a * a - 3.0 * b) / 9.0;
    double R = (2.0 * a * a * a - 9.0 * a * b + 27.0 * d) / 54.0;
    if (R * R < Q * Q * Q) {
        double theta = std::acos(R / std::sqrt(Q * Q * Q));
        double t[3], z[3];
        t[0] = -2.0 * std::sqrt(Q) * std::cos(theta / 3.0) - a / 3.0;
        t[1] = -2.0 * std::sqrt(Q) * std::cos((theta + 2.0 * OMM_PI) / 3.0) - a / 3.0;
        t[2] = -2.0 * std::sqrt(Q) * std::cos((theta - 2.0 * OMM_PI) / 3.0) - a / 3.0;
        for (int i = 0; i < 3; ++i) {
            double tt = t[i];
            z[i] = c[4] * (tt * tt) * (tt * tt) + c[3] * tt * tt * tt + c[2] * tt * tt + c[1] * tt + c[0];
        }
        if (c[4] > 0.0) {
            int o[3];
            if (z[0] >= z[1] && z[0] >= z[2]) { o[0] = 0; o[1] = 1; o[2] = 2; }
            else if (z[1] > z[2]) { o[0] = 1; o[1] = 2; o[2] = 0; }
            else { o[0] = 2; o[1] = 0; o[2] = 1; }
            if ((0.0 <= t[o[0]]) && (t[o[1]] <= t[o[0]])) *x_min = t[o[1]];
            else *x_min = t[o[2]];
        } else {
            if (z[0] <= z[1] && z[0] <= z[2]) *x_min = t[0];
            else if (z[1] < z[2]) *x_min = t[1];
            else *x_min = t[2];
        }
    } else {
        double S = -fsign(1.0, R) * std::pow(std::fabs(R) + std::sqrt(R * R - Q * Q * Q), 1.0 / 3.0);
        double U = (S == 0.0) ? 0.0 : Q / S;
        *x_min = (S + U) - (a / 3.0);
        if (c[4] < 0.0) *fail = true;
    }
}

// ---------------------------------------------------------------------------
// C0 initialisation: omm_rand_seed (NORAND, omm_rand.F90:27-28) and the BSD
// LCG (omm_rand.F90:37-55); element order and scaling from omm.F90:329-342.
// ---------------------------------------------------------------------------
static inline double bsd_lcg(int32_t* x) {
    int64_t v = (1103515245LL * (int64_t)(*x) + 12345LL) % (1LL << 31);
    *x = (int32_t)v;
    return (double)(*x) / (double)(1LL << 31);
}
template <typename T>
static void lcg_init(Mat<T>& C, int m, int n) {
    int32_t seed = 123456;
    for (int i = 0; i < m; ++i)
        for (int j = 0; j < n; ++j) {
            double r1 = bsd_lcg(&seed), r2 = bsd_lcg(&seed);
            double el = fsign(0.5 * r1, r2 - 0.5);
            C(j, i) = T(el) + T(0.0) * C(j, i);  // m_set_element(C,j,i,el,0)
        }
    m_scale(C, T(1.0e-2 / std::sqrt((double)m)));
}

// ---------------------------------------------------------------------------
// omm() — libOMM/src/omm.F90:5-672.  Module-SAVEd per-ip state lives in Ctx.
// ---------------------------------------------------------------------------
// calc_PW_precon (omm_ops.F90:1225-1334): P on the CSC pattern of T, value by value.
// Real (dcalc_PW_precon): s = 2 T_i / scale_T, P_i = (27 + 18 s + 12 s^2 + 8 s^3) /
// (27 + 18 s + 12 s^2 + 8 s^3 + 16 s^4).  Complex (zcalc_PW_precon): P_i = 1 / (1 + |T_i| / scale_T).
static double pw_precon_value(double t, double scale_T) {
    double s = 2.0 * t / scale_T;
    double num = 27.0 + 18.0 * s + 12.0 * s * s + 8.0 * s * s * s;
    return num / (num + 16.0 * s * s * s * s);
}
static zc pw_precon_value(zc t, double scale_T) { return zc(1.0 / (1.0 + std::abs(t) / scale_T), 0.0); }

template <typename T>
static void calc_PW_precon(const Mat<T>& Tk, double scale_T, Mat<T>& P) {
    if (!Tk.csc) die("dcalc_PW_precon: invalid implementation");  // omm_ops.F90:1264-1270
    P.init = true;
    P.csc = true;
    P.d1 = Tk.d1;
    P.d2 = Tk.d2;
    P.nnz = Tk.nnz;
    P.own_cp.assign(Tk.cp, Tk.cp + Tk.d2 + 1);
    P.own_ri.assign(Tk.ri, Tk.ri + Tk.nnz);
    P.cp = P.own_cp.data();
    P.ri = P.own_ri.data();
    P.own.resize(Tk.nnz);
    for (int i = 0; i < Tk.nnz; ++i) P.own[i] = pw_precon_value(Tk.p[i], scale_T);
    P.p = P.own.data();
}

template <typename T>
struct IpState {
    Mat<T> HW, HWd, HWdd, SW, SC, SG, C_Chl, P, work2, QW, CD;
};
template <typename T>
struct State {
    bool alloc = false;
    std::vector<char> first_call;
    std::vector<double> x_min;
    std::vector<IpState<T>> ip;
};
struct Ctx {
    State<double> r;
    State<zc> z;
};

extern "C" {
typedef struct {
    int dim1, dim2;
    int is_csc;
    int nnz;
    void* val;        // dense col-major values, or CSC values
    int* colptr;      // CSC 0-based column offsets (dim2+1)
    int* rowind;      // CSC 0-based row indices
} orc_mat;
}

template <typename T>
static Mat<T> wrap(const orc_mat* o) {
    Mat<T> M;
    M.init = true;
    M.d1 = o->dim1; M.d2 = o->dim2;
    M.csc = o->is_csc != 0;
    M.p = (T*)o->val;
    M.nnz = o->nnz; M.cp = o->colptr; M.ri = o->rowind;
    return M;
}

template <typename T>
static void free_state(State<T>& st) {
    st.ip.clear(); st.x_min.clear(); st.first_call.clear(); st.alloc = false;
}

template <typename T>
static int omm_impl(State<T>& st, int m, int n, Mat<T>& H, Mat<T>* S, bool new_S, double* e_min_out, Mat<T>& D_min,
                    bool calc_ED, double eta, Mat<T>& C_min, bool init_C, Mat<T>* Tk, double scale_T, int flavour,
                    int np, int ip1, double cg_tol, bool dealloc, double* e_hist, int e_hist_cap, int* n_hist,
                    int max_steps) {
    const T one(1.0), zero(0.0);
    bool no_S, use_Cholesky, S_is_U, use_precon;
    int ip = ip1 - 1;
    if (S) {  // omm.F90:125-155
        no_S = false;
        if (flavour == 0) { use_Cholesky = false; S_is_U = false; use_precon = false; }
        else if (flavour == 1) { use_Cholesky = true; S_is_U = false; use_precon = false; }
        else if (flavour == 2) { use_Cholesky = true; S_is_U = true; use_precon = false; }
        else if (flavour == 3 || flavour == 4) { use_Cholesky = false; S_is_U = false; use_precon = true; }
        else die("omm: illegal value of flavour");
    } else {
        no_S = true; use_Cholesky = false; S_is_U = false; use_precon = false;
    }
    if (flavour == 4 && S && !Tk) die("omm: flavour 4 needs the kinetic energy matrix T");
    double cg_tol_internal = (cg_tol < 0.0) ? 1.0e-9 : cg_tol;  // omm.F90:157-161

    if (calc_ED) {  // omm.F90:163-251
        if (!st.alloc || st.first_call[ip]) die("omm: cannot calculate ED matrix before D matrix");
        IpState<T>& s = st.ip[ip];
        double x = st.x_min[ip];
        m_add(s.HWd, 'c', s.HW, T(x), one);
        m_add(s.HWd, 'n', s.HW, T(x), one);
        m_add(s.HWdd, 'n', s.HW, T(x * x), one);
        if (eta != 0.0) m_add(s.SW, 'n', s.HW, T(eta), one);
        calc_A2(s.HW, C_min, s.CD, D_min, s.work2);
        if (!dealloc && eta != 0.0) m_add(s.SW, 'n', s.HW, T(-eta), one);
        if (dealloc) free_state(st);
        return 0;
    }

    if (!st.alloc) {  // omm.F90:253-290
        st.first_call.assign(np, 1);
        st.x_min.assign(np, 0.0);
        st.ip.clear();
        st.ip.resize(np);
        st.alloc = true;
    }
    IpState<T>& s = st.ip[ip];
    if (!s.HW.init) m_allocate(s.HW, n, n);
    if (!s.HWd.init) m_allocate(s.HWd, n, n);
    if (!s.HWdd.init) m_allocate(s.HWdd, n, n);
    if (!s.SW.init) m_allocate(s.SW, n, n);
    if (!use_Cholesky || !no_S) {
        if (!s.SC.init) m_allocate(s.SC, n, m);
        if (!s.SG.init) m_allocate(s.SG, n, m);
    }
    if (use_Cholesky && !s.C_Chl.init) m_allocate(s.C_Chl, n, m);
    if (use_precon && flavour != 4 && !s.P.init) m_allocate(s.P, m, m);
    if (!s.work2.init) m_allocate(s.work2, n, m);

    Mat<T> SWd, SWdd, G, G_p, PG, PG_p, D, HC, HG, work1;  // omm.F90:292-303
    m_allocate(SWd, n, n); m_allocate(SWdd, n, n);
    m_allocate(G, n, m); m_allocate(G_p, n, m);
    if (use_precon) { m_allocate(PG, n, m); m_allocate(PG_p, n, m); }
    m_allocate(D, n, m); m_allocate(HC, n, m); m_allocate(HG, n, m); m_allocate(work1, n, n);

    if (use_Cholesky) {  // omm.F90:306-309
        if (new_S && !S_is_U) m_factorize(*S);
        m_reduce(*S, H);
    }
    if (use_precon && new_S && flavour == 4) {  // omm.F90:321-322
        calc_PW_precon(*Tk, scale_T, s.P);
    } else if (use_precon && new_S) {  // omm.F90:312-320 (flavour 3)
        if (Tk) {
            m_add(*Tk, 'n', s.P, one, zero);
            m_add(*S, 'n', s.P, one, T(1.0 / scale_T));
        } else {
            m_add(*S, 'n', s.P, one, zero);
        }
        m_inverse(s.P);
    }
    if (st.first_call[ip] && !init_C) lcg_init(C_min, m, n);  // omm.F90:329-343
    if (use_Cholesky && (init_C || new_S)) {                  // omm.F90:344-348
        m_add(C_min, 'n', s.C_Chl, one, zero);
        m_transform(*S, s.C_Chl);
    }
    Mat<T>& Cw = use_Cholesky ? s.C_Chl : C_min;  // the working coefficients
    // omm.F90:352-377
    calc_AW(H, Cw, s.HW, HC);
    if (use_Cholesky) {
        if (st.first_call[ip] || init_C || new_S) mm_multiply(s.C_Chl, 'n', s.C_Chl, 'c', s.SW, one, zero);
    } else if (no_S) {
        if (st.first_call[ip] || init_C) mm_multiply(C_min, 'n', C_min, 'c', s.SW, one, zero);
    } else {
        if (st.first_call[ip] || init_C || new_S) calc_AW(*S, C_min, s.SW, s.SC);
        else m_add(s.SG, 'n', s.SC, T(st.x_min[ip]), one);
    }
    if (use_Cholesky || no_S) calc_G(s.HW, s.SW, G, HC, Cw);
    else calc_G(s.HW, s.SW, G, HC, s.SC);
    if (use_precon) mm_multiply(G, 'n', s.P, 'n', PG, one, zero);
    // omm.F90:388-413
    if (use_precon) {
        mm_multiply(HC, 'n', PG, 'c', s.HWd, one, zero);
        mm_multiply(s.SC, 'n', PG, 'c', SWd, one, zero);
    } else {
        mm_multiply(HC, 'n', G, 'c', s.HWd, one, zero);
        if (use_Cholesky || no_S) mm_multiply(Cw, 'n', G, 'c', SWd, one, zero);
        else mm_multiply(s.SC, 'n', G, 'c', SWd, one, zero);
    }
    if (use_precon) {
        calc_AW(H, PG, s.HWdd, HG);
        calc_AW(*S, PG, SWdd, s.SG);
    } else {
        calc_AW(H, G, s.HWdd, HG);
        if (use_Cholesky || no_S) mm_multiply(G, 'n', G, 'c', SWdd, one, zero);
        else calc_AW(*S, G, SWdd, s.SG);
    }
    double coeff[5];
    calc_coeff(s.HW, s.SW, s.HWd, SWd, s.HWdd, SWdd, work1, coeff);
    double e_min = coeff[0];

    // CG loop, omm.F90:429-555
    int icg = 0;
    bool conv = false, ls_conv = false, ls_fail = false;
    int n_step_max_outer = 100;
    long n_step_max_inner = (m < 10000) ? (long)m * n - 1 : 10000000L;
    double lambda = 0.0;
    int nh = 0;
    for (int i = 1; i <= n_step_max_outer; ++i) {
        lambda = 0.0;
        for (long j = 1; j <= n_step_max_inner; ++j) {
            if (use_precon) m_add(PG, 'n', D, one, T(lambda));
            else m_add(G, 'n', D, one, T(lambda));
            m_add(G, 'n', G_p, one, zero);
            if (use_precon) m_add(PG, 'n', PG_p, one, zero);
            double e_min_old = e_min;
            if (icg > 0) {
                mm_multiply(HC, 'n', D, 'c', s.HWd, one, zero);
                if (use_Cholesky || no_S) mm_multiply(Cw, 'n', D, 'c', SWd, one, zero);
                else mm_multiply(s.SC, 'n', D, 'c', SWd, one, zero);
                calc_AW(H, D, s.HWdd, HG);
                if (use_Cholesky || no_S) mm_multiply(D, 'n', D, 'c', SWdd, one, zero);
                else calc_AW(*S, D, SWdd, s.SG);
                calc_coeff(s.HW, s.SW, s.HWd, SWd, s.HWdd, SWdd, work1, coeff);
            }
            double x;
            omm_solve_quartic(coeff, &x, &ls_fail);
            st.x_min[ip] = x;
            if (ls_fail) {
                e_min = 3.0 * e_min;
                m_scale(Cw, T(0.5));
                ls_conv = false;
            } else {
                e_min = coeff[4] * (x * x) * (x * x) + coeff[3] * x * x * x + coeff[2] * x * x + coeff[1] * x + coeff[0];
                m_add(D, 'n', Cw, T(x), one);
                ls_conv = true;
            }
            if (ls_fail) {
                m_scale(s.SW, T(0.25));
            } else {
                m_add(SWd, 'c', s.SW, T(x), one);
                m_add(SWd, 'n', s.SW, T(x), one);
                m_add(SWdd, 'n', s.SW, T(x * x), one);
            }
            double e_diff = 2.0 * std::fabs((e_min - e_min_old) / (e_min + e_min_old));
            if (e_hist && nh < e_hist_cap) e_hist[nh] = e_min;
            ++nh;
            ++icg;
            if (e_diff <= cg_tol_internal) { conv = true; break; }
            if (max_steps > 0 && icg >= max_steps) break;  // bounded timing sample (not in the reference)
            if (ls_fail) {
                m_scale(s.HW, T(0.25));
            } else {
                m_add(s.HWd, 'c', s.HW, T(x), one);
                m_add(s.HWd, 'n', s.HW, T(x), one);
                m_add(s.HWdd, 'n', s.HW, T(x * x), one);
            }
            if (ls_fail) {
                m_scale(HC, T(0.5));
                if (!use_Cholesky || !no_S) m_scale(s.SC, T(0.5));
                m_add(G_p, 'n', G, one, zero);
                m_add(HC, 'n', G, T(1.5), one);
            } else {
                m_add(HG, 'n', HC, T(x), one);
                if (use_Cholesky || no_S) {
                    calc_G(s.HW, s.SW, G, HC, Cw);
                } else {
                    m_add(s.SG, 'n', s.SC, T(x), one);
                    calc_G(s.HW, s.SW, G, HC, s.SC);
                }
            }
            if (use_precon) mm_multiply(G, 'n', s.P, 'n', PG, one, zero);
            if (ls_conv) {
                m_add(G, 'n', s.work2, one, zero);
                m_add(G_p, 'n', s.work2, T(-1.0), one);
                double lambda_n, lambda_d;
                if (use_precon) { lambda_n = mm_trace(PG, s.work2); lambda_d = mm_trace(PG_p, G_p); }
                else { lambda_n = mm_trace(G, s.work2); lambda_d = mm_trace(G_p, G_p); }
                lambda = lambda_n / lambda_d;
            } else {
                break;
            }
        }
        if (conv) break;
        if (max_steps > 0 && icg >= max_steps) break;
    }
    if (n_hist) *n_hist = nh;
    // omm.F90:569-593
    if (!s.QW.init) m_allocate(s.QW, n, n);
    if (!s.CD.init) m_allocate(s.CD, n, m);
    m_set_all(s.QW, zero, T(2.0));
    m_add(s.SW, 'n', s.QW, T(-1.0), one);
    if (use_Cholesky) {
        m_add(s.C_Chl, 'n', C_min, one, zero);
        m_back_transform(*S, C_min);
    }
    calc_A(s.QW, C_min, D_min, s.CD);
    double TrQS = mm_trace(s.QW, s.SW);
    e_min = e_min + TrQS * eta;
    *e_min_out = e_min;
    if (dealloc) free_state(st);
    else st.first_call[ip] = 0;
    return conv ? 0 : 1;
}

// ---------------------------------------------------------------------------
// C ABI of the oracle (ctypes from oracle/oracle.py)
// ---------------------------------------------------------------------------
extern "C" {

const char* orc_last_error() { return g_err.c_str(); }

int orc_init(const char* openblas_path, int nthreads) {
    if (!L.h) {
        L.h = dlopen(openblas_path, RTLD_NOW | RTLD_LOCAL);
        if (!L.h) { g_err = dlerror(); return -1; }
#define SYM(field, name)                                        \
    L.field = (decltype(L.field))dlsym(L.h, name);              \
    if (!L.field) { g_err = std::string("missing ") + name; return -2; }
        SYM(dgemm, "scipy_dgemm_") SYM(zgemm, "scipy_zgemm_")
        SYM(dpotrf, "scipy_dpotrf_") SYM(zpotrf, "scipy_zpotrf_")
        SYM(dsygst, "scipy_dsygst_") SYM(zhegst, "scipy_zhegst_")
        SYM(dtrmm, "scipy_dtrmm_") SYM(dtrsm, "scipy_dtrsm_")
        SYM(ztrmm, "scipy_ztrmm_") SYM(ztrsm, "scipy_ztrsm_")
        SYM(ddot, "scipy_ddot_")
        SYM(dsytrf, "scipy_dsytrf_") SYM(zhetrf, "scipy_zhetrf_")
        SYM(dsytri, "scipy_dsytri_") SYM(zhetri, "scipy_zhetri_")
        SYM(set_threads, "scipy_openblas_set_num_threads")
#undef SYM
    }
    if (nthreads > 0) {
        L.set_threads(nthreads);
        g_threads = nthreads;
    }
    return 0;
}

void* orc_ctx_new() { return new Ctx(); }
void orc_ctx_free(void* c) { delete (Ctx*)c; }

// Returns 0 when CG converged, 1 when the iteration caps were reached, <0 on "die".
int orc_omm(void* ctx, int is_real, int m, int n, orc_mat* H, orc_mat* S, int new_S, double* e_min, orc_mat* D_min,
            int calc_ED, double eta, orc_mat* C_min, int init_C, orc_mat* T, double scale_T, int flavour, int np,
            int ip, double cg_tol, int dealloc, double* e_hist, int e_hist_cap, int* n_hist, int max_steps) {
    try {
        Ctx* c = (Ctx*)ctx;
        if (is_real) {
            Mat<double> h = wrap<double>(H), d = wrap<double>(D_min), cm = wrap<double>(C_min), s, t;
            if (S) s = wrap<double>(S);
            if (T) t = wrap<double>(T);
            return omm_impl<double>(c->r, m, n, h, S ? &s : nullptr, new_S, e_min, d, calc_ED, eta, cm, init_C,
                                    T ? &t : nullptr, scale_T, flavour, np, ip, cg_tol, dealloc, e_hist, e_hist_cap,
                                    n_hist, max_steps);
        } else {
            Mat<zc> h = wrap<zc>(H), d = wrap<zc>(D_min), cm = wrap<zc>(C_min), s, t;
            if (S) s = wrap<zc>(S);
            if (T) t = wrap<zc>(T);
            return omm_impl<zc>(c->z, m, n, h, S ? &s : nullptr, new_S, e_min, d, calc_ED, eta, cm, init_C,
                                T ? &t : nullptr, scale_T, flavour, np, ip, cg_tol, dealloc, e_hist, e_hist_cap,
                                n_hist, max_steps);
        }
    } catch (OrcDie& e) {
        g_err = e.msg;
        return -1;
    }
}

// C = alpha*op(A)*op(B) + beta*C for any dense/CSC combination (alpha, beta complex as re,im pairs).
// pspBLAS convention (pspMspm.F90:79-116, pspSpmm.F90): alpha==0 leaves C=beta*C, and C untouched when beta==0 too.
int orc_mm_multiply(int is_real, orc_mat* A, char opA, orc_mat* B, char opB, orc_mat* C, double ar, double ai,
                    double br, double bi, int psp_semantics) {
    try {
        if (is_real) {
            Mat<double> a = wrap<double>(A), b = wrap<double>(B), c = wrap<double>(C);
            if (psp_semantics && ar == 0.0) {
                if (br != 0.0) m_scale(c, br);
                return 0;
            }
            mm_multiply(a, opA, b, opB, c, ar, br);
        } else {
            Mat<zc> a = wrap<zc>(A), b = wrap<zc>(B), c = wrap<zc>(C);
            if (psp_semantics && ar == 0.0 && ai == 0.0) {
                if (br != 0.0 || bi != 0.0) m_scale(c, zc(br, bi));
                return 0;
            }
            mm_multiply(a, opA, b, opB, c, zc(ar, ai), zc(br, bi));
        }
        return 0;
    } catch (OrcDie& e) {
        g_err = e.msg;
        return -1;
    }
}

int orc_calc_coeff(int is_real, int n, void* HW, void* SW, void* HWd, void* SWd, void* HWdd, void* SWdd,
                   double* coeff) {
    try {
        orc_mat o{n, n, 0, 0, nullptr, nullptr, nullptr};
        if (is_real) {
            Mat<double> M[6];
            void* ps[6] = {HW, SW, HWd, SWd, HWdd, SWdd};
            for (int i = 0; i < 6; ++i) { o.val = ps[i]; M[i] = wrap<double>(&o); }
            Mat<double> w; m_allocate(w, n, n);
            calc_coeff(M[0], M[1], M[2], M[3], M[4], M[5], w, coeff);
        } else {
            Mat<zc> M[6];
            void* ps[6] = {HW, SW, HWd, SWd, HWdd, SWdd};
            for (int i = 0; i < 6; ++i) { o.val = ps[i]; M[i] = wrap<zc>(&o); }
            Mat<zc> w; m_allocate(w, n, n);
            calc_coeff(M[0], M[1], M[2], M[3], M[4], M[5], w, coeff);
        }
        return 0;
    } catch (OrcDie& e) {
        g_err = e.msg;
        return -1;
    }
}

double orc_mm_trace(int is_real, int d1, int d2, void* A, void* B) {
    orc_mat oa{d1, d2, 0, 0, A, nullptr, nullptr}, ob{d1, d2, 0, 0, B, nullptr, nullptr};
    if (is_real) return mm_trace(wrap<double>(&oa), wrap<double>(&ob));
    return mm_trace(wrap<zc>(&oa), wrap<zc>(&ob));
}

void orc_solve_quartic(const double* c, double* x_min, int* fail) {
    bool f;
    omm_solve_quartic(c, x_min, &f);
    *fail = f ? 1 : 0;
}

void orc_lcg_init(int is_real, int n, int m, void* C) {
    orc_mat o{n, m, 0, 0, C, nullptr, nullptr};
    if (is_real) { Mat<double> c = wrap<double>(&o); lcg_init(c, m, n); }
    else { Mat<zc> c = wrap<zc>(&o); lcg_init(c, m, n); }
}

// calc_G restated (omm_ops.F90:17-39): G = 4*HC - 2*SW*HC - 2*HW*SC
int orc_calc_G(int is_real, int n, int m, void* HW, void* SW, void* G, void* HC, void* SC) {
    try {
        orc_mat nn{n, n, 0, 0, nullptr, nullptr, nullptr}, nm{n, m, 0, 0, nullptr, nullptr, nullptr};
        if (is_real) {
            nn.val = HW; Mat<double> hw = wrap<double>(&nn);
            nn.val = SW; Mat<double> sw = wrap<double>(&nn);
            nm.val = G; Mat<double> g = wrap<double>(&nm);
            nm.val = HC; Mat<double> hc = wrap<double>(&nm);
            nm.val = SC; Mat<double> sc = wrap<double>(&nm);
            calc_G(hw, sw, g, hc, sc);
        } else {
            nn.val = HW; Mat<zc> hw = wrap<zc>(&nn);
            nn.val = SW; Mat<zc> sw = wrap<zc>(&nn);
            nm.val = G; Mat<zc> g = wrap<zc>(&nm);
            nm.val = HC; Mat<zc> hc = wrap<zc>(&nm);
            nm.val = SC; Mat<zc> sc = wrap<zc>(&nm);
            calc_G(hw, sw, g, hc, sc);
        }
        return 0;
    } catch (OrcDie& e) {
        g_err = e.msg;
        return -1;
    }
}

}  // extern "C"
