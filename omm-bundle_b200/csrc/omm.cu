// omm() — the orbital-minimization CG solver (libOMM/src/omm.F90:5-672) on one GPU.
//
// Control flow, flavours, quirks and the per-ip SAVEd state follow omm.F90
// line by line (citations inline).  What changes is where the data lives and
// how the products are grouped:
//   * all matrices stay in HBM for the whole call; only the five quartic
//     coefficients and the two Polak-Ribiere traces come back to the host
//     each CG step (two 8..104-byte reads);
//   * HC and SC are one stacked 2n x m matrix X = [HC; SC] and HG, SG one
//     Y = [HG; SG] (column-major, leading dimension 2n).  The four Gram
//     products of a step are then two GEMMs, [HWd; SWd] = X D^H and
//     [HWdd; SWdd] = Y D^H, and calc_G (omm_ops.F90:17-39) is one GEMM
//     G = [4I - 2 SW, -2 HW] X with K = 2n;
//   * for sparse H and S with one pattern, HG and SG come from one fused
//     SpMM pass over D;
//   * when S is the identity (no S, or the Cholesky flavour) the S half of X
//     and Y holds copies of C and D, updated with the same operations, so the
//     stacked products stay uniform.
#include "internal.h"

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>

namespace ommgpu {

struct OmmState {
    bool allocated = false;
    std::vector<char> first_call;
    std::vector<double> x_min;
    std::vector<IpState> ip;
};

static OmmState g_state;     // omm's per-ip SAVEd state (omm.F90:62-106)
static OmmState g_state_cb;  // omm_callback's own copy (omm_callback.F90 keeps separate SAVEd variables)
static OmmState* g_cur = &g_state;
static omm_gpu_stats g_stats{};
static std::string g_log_path = "libOMM.log";
static bool g_log_enabled = true;
static bool g_log_start = false;
// end of the BF16 stage, end of the split-BF16 stage, and the convergence threshold of the
// refinement stage as a fraction of cg_tol
static double g_mixed_tol[3] = {1e-5, 1e-8, 0.1};

namespace {

DView view(const DevBuf& b, int rows, int cols, int ld, bool real, size_t off_elems = 0) {
    DView v;
    v.p = (char*)b.p + off_elems * (real ? 8 : 16);
    v.rows = rows;
    v.cols = cols;
    v.ld = ld;
    v.is_real = real;
    return v;
}

const double ONE[2] = {1.0, 0.0}, ZERO[2] = {0.0, 0.0}, MONE[2] = {-1.0, 0.0};

void copy_view(const DView& src, DView& dst) { k_axpby(src, 'n', dst, ONE, ZERO); }

// ---- log file (omm.F90:118-123, :417-428, :504, :553-556, :587-591)
struct Log {
    FILE* f = nullptr;
    Log() {
        if (!g_log_enabled) return;
        f = fopen(g_log_path.c_str(), g_log_start ? "a" : "w");
        g_log_start = true;
    }
    ~Log() {
        if (f) fclose(f);
    }
    void line(const char* s) {
        if (f) fprintf(f, "%s\n", s);
    }
};

// Fortran es15.7e3 (e.g. "-2.4438247E+001")
std::string es15(double v) {
    char b[64];
    if (v == 0.0) {
        snprintf(b, sizeof b, "%15s", "0.0000000E+000");
        return b;
    }
    int e = (int)std::floor(std::log10(std::fabs(v)));
    double mant = v / std::pow(10.0, e);
    if (std::fabs(mant) >= 9.99999995) { mant /= 10.0; e += 1; }
    snprintf(b, sizeof b, "%10.7fE%c%03d", mant, e < 0 ? '-' : '+', std::abs(e));
    char o[64];
    snprintf(o, sizeof o, "%15s", b);
    return o;
}

// ---- dense Cholesky operations (omm_ops.F90:225-965) on cuSOLVER / cuBLAS
void factorize_upper(DView& S) {  // dpotrf('u') / zpotrf('u')
    Runtime& R = rt();
    int lwork = 0;
    int m = S.rows;
    DevBuf info;
    info.alloc_zero(sizeof(int));
    if (S.is_real) {
        OMM_CKS(cusolverDnDpotrf_bufferSize(R.solver, CUBLAS_FILL_MODE_UPPER, m, S.as<double>(), S.ld, &lwork));
        DevBuf w;
        w.alloc(std::max(1, lwork) * sizeof(double));
        OMM_CKS(cusolverDnDpotrf(R.solver, CUBLAS_FILL_MODE_UPPER, m, S.as<double>(), S.ld, w.as<double>(), lwork,
                                 info.as<int>()));
        int h = 0;
        OMM_CK(cudaMemcpyAsync(&h, info.p, sizeof(int), cudaMemcpyDeviceToHost, R.stream));
        sync();
        if (h != 0) fail(OMM_ERR_NOT_SPD, "m_dfactorize: error in dpotrf");
    } else {
        OMM_CKS(cusolverDnZpotrf_bufferSize(R.solver, CUBLAS_FILL_MODE_UPPER, m, S.as<cuDoubleComplex>(), S.ld,
                                            &lwork));
        DevBuf w;
        w.alloc(std::max(1, lwork) * sizeof(cuDoubleComplex));
        OMM_CKS(cusolverDnZpotrf(R.solver, CUBLAS_FILL_MODE_UPPER, m, S.as<cuDoubleComplex>(), S.ld,
                                 w.as<cuDoubleComplex>(), lwork, info.as<int>()));
        int h = 0;
        OMM_CK(cudaMemcpyAsync(&h, info.p, sizeof(int), cudaMemcpyDeviceToHost, R.stream));
        sync();
        if (h != 0) fail(OMM_ERR_NOT_SPD, "m_zfactorize: error in zpotrf");
    }
}

// H := U^-H H U^-1 for large m: the blocked form of LAPACK's sygst (itype 1, upper), which
// updates the upper triangle one block row at a time in m^3 flops (two full triangular solves
// take 2 m^3).  For block row k (A = H, B = U, rows k..k+kb, the rest r..m):
//   A11 <- B11^-H A11 B11^-1;  A12 <- B11^-H A12;  A12 -= A11 B12 / 2;
//   A22 -= A12^H B12 + B12^H A12 (upper triangle);  A12 -= A11 B12 / 2;  A12 <- A12 B22^-1.
void reduce_upper_blocked(const DView& U, DView& H, int nb) {
    Runtime& R = rt();
    OMM_CKB(cublasSetStream(R.blas, R.stream));
    const int m = H.rows;
    const size_t es = H.is_real ? 8 : 16;
    auto at = [&](const DView& A, int i, int j) { return (char*)A.p + ((size_t)i + (size_t)j * A.ld) * es; };
    auto sub = [&](const DView& A, int i, int j, int rows, int cols) {
        DView v = A;
        v.p = at(A, i, j);
        v.rows = rows;
        v.cols = cols;
        return v;
    };
    // the block row's symmetric products on the int8 tensor cores when they are large enough and
    // the trailing block splits into whole 256-row tiles (the Hermitian-tile skip of A22)
    auto emu_update = [&](int kb_, int nr_) {
        return H.is_real && fp64_emu_enabled() && nr_ % 256 == 0 && fp64_emu_worth(nr_, nr_, kb_) &&
               fp64_emu_worth(kb_, nr_, kb_);
    };
    for (int k = 0; k < m; k += nb) {
        const int kb = std::min(nb, m - k), r = k + kb, nr = m - r;
        DView A11 = H;
        A11.p = at(H, k, k);
        A11.rows = A11.cols = kb;
        k_fill_lower_from_upper(A11);  // the diagonal block in full for its two solves
        if (H.is_real) {
            const double one = 1.0, mone = -1.0, mhalf = -0.5;
            double *a11 = (double*)A11.p, *a12 = (double*)at(H, k, r), *a22 = (double*)at(H, r, r);
            const double *b11 = (const double*)at(U, k, k), *b12 = (const double*)at(U, k, r),
                         *b22 = (const double*)at(U, r, r);
            OMM_CKB(cublasDtrsm(R.blas, CUBLAS_SIDE_LEFT, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_T, CUBLAS_DIAG_NON_UNIT, kb,
                                kb, &one, b11, U.ld, a11, H.ld));
            OMM_CKB(cublasDtrsm(R.blas, CUBLAS_SIDE_RIGHT, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_N, CUBLAS_DIAG_NON_UNIT,
                                kb, kb, &one, b11, U.ld, a11, H.ld));
            if (nr == 0) break;
            OMM_CKB(cublasDtrsm(R.blas, CUBLAS_SIDE_LEFT, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_T, CUBLAS_DIAG_NON_UNIT, kb,
                                nr, &one, b11, U.ld, a12, H.ld));
            if (emu_update(kb, nr)) {
                // the symmetric products as FP64-accurate products on the int8 tensor cores: A11 is
                // full (both triangles), and A22's rank-2k update forms only its upper tiles
                DView vA11 = sub(H, k, k, kb, kb), vA12 = sub(H, k, r, kb, nr), vA22 = sub(H, r, r, nr, nr);
                const DView vB12 = sub(U, k, r, kb, nr);
                gemm_f64_emu('n', 'n', kb, nr, kb, -0.5, vA11, vB12, 1.0, vA12);
                gemm_f64_emu('t', 'n', nr, nr, kb, -1.0, vA12, vB12, 1.0, vA22, nr);
                gemm_f64_emu('t', 'n', nr, nr, kb, -1.0, vB12, vA12, 1.0, vA22, nr);
                gemm_f64_emu('n', 'n', kb, nr, kb, -0.5, vA11, vB12, 1.0, vA12);
            } else {
                OMM_CKB(cublasDsymm(R.blas, CUBLAS_SIDE_LEFT, CUBLAS_FILL_MODE_UPPER, kb, nr, &mhalf, a11, H.ld, b12,
                                    U.ld, &one, a12, H.ld));
                OMM_CKB(cublasDsyr2k(R.blas, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_T, nr, kb, &mone, a12, H.ld, b12, U.ld,
                                     &one, a22, H.ld));
                OMM_CKB(cublasDsymm(R.blas, CUBLAS_SIDE_LEFT, CUBLAS_FILL_MODE_UPPER, kb, nr, &mhalf, a11, H.ld, b12,
                                    U.ld, &one, a12, H.ld));
            }
            OMM_CKB(cublasDtrsm(R.blas, CUBLAS_SIDE_RIGHT, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_N, CUBLAS_DIAG_NON_UNIT,
                                kb, nr, &one, b22, U.ld, a12, H.ld));
        } else {
            const cuDoubleComplex one = make_cuDoubleComplex(1.0, 0.0), mone = make_cuDoubleComplex(-1.0, 0.0),
                                  mhalf = make_cuDoubleComplex(-0.5, 0.0);
            const double rone = 1.0;
            auto* a11 = (cuDoubleComplex*)A11.p;
            auto* a12 = (cuDoubleComplex*)at(H, k, r);
            auto* a22 = (cuDoubleComplex*)at(H, r, r);
            auto* b11 = (const cuDoubleComplex*)at(U, k, k);
            auto* b12 = (const cuDoubleComplex*)at(U, k, r);
            auto* b22 = (const cuDoubleComplex*)at(U, r, r);
            OMM_CKB(cublasZtrsm(R.blas, CUBLAS_SIDE_LEFT, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_C, CUBLAS_DIAG_NON_UNIT, kb,
                                kb, &one, b11, U.ld, a11, H.ld));
            OMM_CKB(cublasZtrsm(R.blas, CUBLAS_SIDE_RIGHT, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_N, CUBLAS_DIAG_NON_UNIT,
                                kb, kb, &one, b11, U.ld, a11, H.ld));
            if (nr == 0) break;
            OMM_CKB(cublasZtrsm(R.blas, CUBLAS_SIDE_LEFT, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_C, CUBLAS_DIAG_NON_UNIT, kb,
                                nr, &one, b11, U.ld, a12, H.ld));
            OMM_CKB(cublasZhemm(R.blas, CUBLAS_SIDE_LEFT, CUBLAS_FILL_MODE_UPPER, kb, nr, &mhalf, a11, H.ld, b12, U.ld,
                                &one, a12, H.ld));
            OMM_CKB(cublasZher2k(R.blas, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_C, nr, kb, &mone, a12, H.ld, b12, U.ld,
                                 &rone, a22, H.ld));
            OMM_CKB(cublasZhemm(R.blas, CUBLAS_SIDE_LEFT, CUBLAS_FILL_MODE_UPPER, kb, nr, &mhalf, a11, H.ld, b12, U.ld,
                                &one, a12, H.ld));
            OMM_CKB(cublasZtrsm(R.blas, CUBLAS_SIDE_RIGHT, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_N, CUBLAS_DIAG_NON_UNIT,
                                kb, nr, &one, b22, U.ld, a12, H.ld));
        }
    }
    k_fill_lower_from_upper(H);
}

// H := U^-H H U^-1 from the upper triangle of H, then fill the lower triangle
// (dsygst(1,'u') + omm_ops.F90:483-487).
void reduce_upper(const DView& U, DView& H) {
    Runtime& R = rt();
    int m = H.rows;
    if (m >= 4096) {
        reduce_upper_blocked(U, H, m >= 16384 ? 1024 : 512);
        return;
    }
    k_fill_lower_from_upper(H);  // dsygst reads only the upper triangle
    if (H.is_real) {
        double one = 1.0;
        OMM_CKB(cublasDtrsm(R.blas, CUBLAS_SIDE_LEFT, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_T, CUBLAS_DIAG_NON_UNIT, m, m,
                            &one, U.as<double>(), U.ld, H.as<double>(), H.ld));
        OMM_CKB(cublasDtrsm(R.blas, CUBLAS_SIDE_RIGHT, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_N, CUBLAS_DIAG_NON_UNIT, m, m,
                            &one, U.as<double>(), U.ld, H.as<double>(), H.ld));
    } else {
        cuDoubleComplex one = make_cuDoubleComplex(1.0, 0.0);
        OMM_CKB(cublasZtrsm(R.blas, CUBLAS_SIDE_LEFT, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_C, CUBLAS_DIAG_NON_UNIT, m, m,
                            &one, U.as<cuDoubleComplex>(), U.ld, H.as<cuDoubleComplex>(), H.ld));
        OMM_CKB(cublasZtrsm(R.blas, CUBLAS_SIDE_RIGHT, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_N, CUBLAS_DIAG_NON_UNIT, m, m,
                            &one, U.as<cuDoubleComplex>(), U.ld, H.as<cuDoubleComplex>(), H.ld));
    }
    k_fill_lower_from_upper(H);
}

// C := C U^H (dtrmm('r','u','t','n'), omm_ops.F90:718 / ztrmm 'c' :786)
void transform(const DView& U, DView& C) {
    Runtime& R = rt();
    DevBuf tmp;
    tmp.alloc((size_t)C.rows * C.cols * (C.is_real ? 8 : 16));
    DView T = C;
    T.p = tmp.p;
    T.ld = C.rows;
    if (C.is_real) {
        double one = 1.0;
        OMM_CKB(cublasDtrmm(R.blas, CUBLAS_SIDE_RIGHT, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_T, CUBLAS_DIAG_NON_UNIT,
                            C.rows, C.cols, &one, U.as<double>(), U.ld, C.as<double>(), C.ld, T.as<double>(), T.ld));
    } else {
        cuDoubleComplex one = make_cuDoubleComplex(1.0, 0.0);
        OMM_CKB(cublasZtrmm(R.blas, CUBLAS_SIDE_RIGHT, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_C, CUBLAS_DIAG_NON_UNIT,
                            C.rows, C.cols, &one, U.as<cuDoubleComplex>(), U.ld, C.as<cuDoubleComplex>(), C.ld,
                            T.as<cuDoubleComplex>(), T.ld));
    }
    copy_view(T, C);
    sync();
}

// C := C U^-H (dtrsm('r','u','t','n'), omm_ops.F90:885)
void back_transform(const DView& U, DView& C) {
    Runtime& R = rt();
    if (C.is_real) {
        double one = 1.0;
        OMM_CKB(cublasDtrsm(R.blas, CUBLAS_SIDE_RIGHT, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_T, CUBLAS_DIAG_NON_UNIT,
                            C.rows, C.cols, &one, U.as<double>(), U.ld, C.as<double>(), C.ld));
    } else {
        cuDoubleComplex one = make_cuDoubleComplex(1.0, 0.0);
        OMM_CKB(cublasZtrsm(R.blas, CUBLAS_SIDE_RIGHT, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_C, CUBLAS_DIAG_NON_UNIT,
                            C.rows, C.cols, &one, U.as<cuDoubleComplex>(), U.ld, C.as<cuDoubleComplex>(), C.ld));
    }
}

// P := P^-1, then the lower triangle from the upper (m_inverse, omm_ops.F90:1059-1076).
// The inverse is formed from an LU factorisation (getrf/getrs with an identity
// right-hand side) instead of dsytrf/dsytri; both give the same inverse up to rounding.
void invert(DView& P) {
    Runtime& R = rt();
    int m = P.rows;
    DevBuf ipiv, info, work, rhs;
    ipiv.alloc(std::max(1, m) * sizeof(int));
    info.alloc_zero(sizeof(int));
    rhs.alloc((size_t)m * m * (P.is_real ? 8 : 16));
    DView I = P;
    I.p = rhs.p;
    I.ld = m;
    double zero[2] = {0.0, 0.0}, one[2] = {1.0, 0.0};
    k_set(I, 'a', zero, one);
    int lwork = 0, h = 0;
    if (P.is_real) {
        OMM_CKS(cusolverDnDgetrf_bufferSize(R.solver, m, m, P.as<double>(), P.ld, &lwork));
        work.alloc(std::max(1, lwork) * sizeof(double));
        OMM_CKS(cusolverDnDgetrf(R.solver, m, m, P.as<double>(), P.ld, work.as<double>(), ipiv.as<int>(),
                                 info.as<int>()));
        OMM_CKS(cusolverDnDgetrs(R.solver, CUBLAS_OP_N, m, m, P.as<double>(), P.ld, ipiv.as<int>(), I.as<double>(),
                                 I.ld, info.as<int>()));
    } else {
        OMM_CKS(cusolverDnZgetrf_bufferSize(R.solver, m, m, P.as<cuDoubleComplex>(), P.ld, &lwork));
        work.alloc(std::max(1, lwork) * sizeof(cuDoubleComplex));
        OMM_CKS(cusolverDnZgetrf(R.solver, m, m, P.as<cuDoubleComplex>(), P.ld, work.as<cuDoubleComplex>(),
                                 ipiv.as<int>(), info.as<int>()));
        OMM_CKS(cusolverDnZgetrs(R.solver, CUBLAS_OP_N, m, m, P.as<cuDoubleComplex>(), P.ld, ipiv.as<int>(),
                                 I.as<cuDoubleComplex>(), I.ld, info.as<int>()));
    }
    OMM_CK(cudaMemcpyAsync(&h, info.p, sizeof(int), cudaMemcpyDeviceToHost, R.stream));
    sync();
    if (h != 0) fail(OMM_ERR_NOT_SPD, P.is_real ? "m_dinverse: error in dsytrf" : "m_zinverse: error in zhetrf");
    copy_view(I, P);
    k_fill_lower_from_upper(P);
}

// ---- the products of one CG direction
// A*M for A (n x m) and M = H or S (dense or CSC), into out (n x m view).
// The plane-wave preconditioner of flavour 4 (omm_ops.F90:1225-1334): a CSC matrix with T's
// pattern and values P_i = f(T_i): real (dcalc_PW_precon) s = 2 T_i / scale_T,
// f = (27 + 18 s + 12 s^2 + 8 s^3) / (27 + 18 s + 12 s^2 + 8 s^3 + 16 s^4); complex
// (zcalc_PW_precon) f = 1 / (1 + |T_i| / scale_T).  Built on the host from T's CSC (once per new S).
std::shared_ptr<msw_matrix> pw_precon(const msw_matrix* T, double scale_T) {
    auto P = std::make_shared<msw_matrix>();
    P->dim1 = T->dim1;
    P->dim2 = T->dim2;
    P->is_real = T->is_real;
    P->fmt = Fmt::CSC;
    P->loc = Loc::Device;
    memcpy(P->label, T->is_real ? "gdcsc" : "gzcsc", 6);
    P->nnz = T->nnz;
    P->h_colptr = T->h_colptr;
    P->h_rowind = T->h_rowind;
    P->h_val.resize(T->h_val.size());
    if (T->is_real) {
        for (int i = 0; i < T->nnz; ++i) {
            double sv = 2.0 * T->h_val[i] / scale_T;
            double num = 27.0 + 18.0 * sv + 12.0 * sv * sv + 8.0 * sv * sv * sv;
            P->h_val[i] = num / (num + 16.0 * sv * sv * sv * sv);
        }
    } else {
        for (int i = 0; i < T->nnz; ++i) {
            P->h_val[2 * i] = 1.0 / (1.0 + std::hypot(T->h_val[2 * i], T->h_val[2 * i + 1]) / scale_T);
            P->h_val[2 * i + 1] = 0.0;
        }
    }
    ensure_csc_device(P.get());
    return P;
}

// PG = G * P (omm.F90:379, :535): dense P (flavour 3) or the CSC P of flavour 4
void apply_precon(OmmCall& c, const DView& G, DView& PG) {
    if (c.pw_precon) {
        spmm_dense_csc(G, c.s->Pcsc.get(), PG, ONE, ZERO);
        return;
    }
    DView P = view(c.s->P, c.m, c.m, c.m, c.real);
    gemm('n', 'n', c.n, c.m, c.m, ONE, G, P, ZERO, PG);
}

// H applied through the caller's routine (omm_callback's H(C, HC), omm_ops.F90:69-99): the
// library's operand and a contiguous n x m result are handed over as 'g' matrices aliasing its
// device buffers; the result is copied into `out` (which may be a half of a stacked buffer).
void apply_callback(OmmCall& c, const DView& A, DView& out) {
    if (A.ld != A.rows) fail(OMM_ERR_ARG, "omm_callback: internal operand is not contiguous");
    msw_matrix Cm, HCm;
    for (msw_matrix* M : {&Cm, &HCm}) {
        M->dim1 = c.n;
        M->dim2 = c.m;
        M->is_real = c.real;
        M->loc = Loc::Device;
        M->fmt = Fmt::Dense;
        memcpy(M->label, c.real ? "gdden" : "gzden", 6);
        M->dev.owns = false;
        M->dev.bytes = (size_t)c.n * c.m * c.es;
    }
    Cm.dev.p = A.p;
    HCm.dev.p = out.ld == out.rows ? out.p : c.s->cb_out.p;
    if (out.ld != out.rows) {
        c.s->cb_out.ensure((size_t)c.n * c.m * c.es);
        HCm.dev.p = c.s->cb_out.p;
    }
    sync();  // the operand is complete before the caller's routine runs
    int rc = c.hcb(&Cm, &HCm, c.hcb_user);
    Cm.dev.p = HCm.dev.p = nullptr;  // aliases: nothing to free
    if (rc != 0) fail(OMM_ERR_CALLBACK, "omm_callback: the H routine returned " + std::to_string(rc));
    if (out.ld != out.rows) copy_view(view(c.s->cb_out, c.n, c.m, c.n, c.real), out);
}

void apply_op(OmmCall& c, const DView& A, bool isH, DView& out) {
    if (isH && c.hcb) {
        apply_callback(c, A, out);
        return;
    }
    const msw_matrix* Mm = isH ? c.Hm : c.Sm;
    if (!Mm->dense()) {
        spmm_dense_csc(A, Mm, out, ONE, ZERO);
    } else {
        const DView& Md = isH ? c.H : c.S;
        gemm('n', 'n', c.n, c.m, c.m, ONE, A, Md, ZERO, out);
    }
}

// [HA; SA] = A*[H, S] into a stacked 2n x m buffer (SA = A when S is the identity)
void apply_HS(OmmCall& c, const DView& A, DevBuf& stack) {
    int n = c.n, m = c.m;
    DView top = view(stack, n, m, 2 * n, c.real, 0);
    DView bot = view(stack, n, m, 2 * n, c.real, n);
    if (c.s_identity) {
        apply_op(c, A, true, top);
        copy_view(A, bot);
        return;
    }
    if (c.H_csc && c.S_csc && same_pattern(c.Hm, c.Sm)) {
        spmm_dense_csc(A, c.Hm, top, ONE, ZERO, c.Sm, &bot);
        return;
    }
    apply_op(c, A, true, top);
    apply_op(c, A, false, bot);
}

// [HWdd; SWdd] = Y Dir^H with Y = [HG; SG] = Dir [H, S] (2n x m, ld 2n).  Both halves are
// Hermitian (Dir H Dir^H, Dir S Dir^H), so only their upper triangles are formed: row block i
// of each half against rows i*bs.. of Dir, the two halves in one strided-batched call, then the
// lower triangles are mirrored.  nb row blocks cost (nb + 1) / (2 nb) of the full product's flops.
// Device pointer arrays of the batched block products below, kept by the buffers they address
// (their addresses are stable across the CG steps of a solve, so each set is uploaded once).
struct BlockPtrs {
    const void *a = nullptr, *b = nullptr, *w = nullptr;
    int lda = 0, ldb = 0, ldw = 0, n = 0, halves = 0, nb = 0, device = -1;
    bool cplx = false;
    DevBuf arrays;  // [count] A pointers, [count] B pointers, [count] W pointers
};
std::mutex g_block_ptrs_mu;
std::vector<std::shared_ptr<BlockPtrs>> g_block_ptrs;  // most recent last, at most 8

std::shared_ptr<BlockPtrs> block_ptrs(const DView& A, const DView& B, DView& W, int n, int halves, int nb) {
    int dev = 0;
    OMM_CK(cudaGetDevice(&dev));
    {
        std::lock_guard<std::mutex> lk(g_block_ptrs_mu);
        for (auto& e : g_block_ptrs)
            if (e->a == A.p && e->b == B.p && e->w == W.p && e->lda == A.ld && e->ldb == B.ld && e->ldw == W.ld &&
                e->n == n && e->halves == halves && e->nb == nb && e->device == dev && e->cplx == !A.is_real)
                return e;
    }
    auto e = std::make_shared<BlockPtrs>();
    e->a = A.p; e->b = B.p; e->w = W.p;
    e->lda = A.ld; e->ldb = B.ld; e->ldw = W.ld;
    e->n = n; e->halves = halves; e->nb = nb; e->device = dev; e->cplx = !A.is_real;
    const size_t es = A.is_real ? 8 : 16;
    const int bs = n / nb, count = halves * nb * (nb + 1) / 2;
    std::vector<const void*> h(3 * (size_t)count);
    int q = 0;
    for (int hf = 0; hf < halves; ++hf)
        for (int bi = 0; bi < nb; ++bi)
            for (int bj = bi; bj < nb; ++bj, ++q) {
                const size_t row = (size_t)hf * n + (size_t)bi * bs;
                h[q] = (const char*)A.p + row * es;
                h[count + q] = (const char*)B.p + (size_t)bj * bs * es;
                h[2 * count + q] = (const char*)W.p + (row + (size_t)bj * bs * W.ld) * es;
            }
    e->arrays.alloc(h.size() * sizeof(void*));
    OMM_CK(cudaMemcpyAsync(e->arrays.p, h.data(), h.size() * sizeof(void*), cudaMemcpyHostToDevice, rt().stream));
    OMM_CK(cudaStreamSynchronize(rt().stream));
    std::lock_guard<std::mutex> lk(g_block_ptrs_mu);
    g_block_ptrs.push_back(e);
    if (g_block_ptrs.size() > 8) g_block_ptrs.erase(g_block_ptrs.begin());
    return e;
}

// W_h = A_h B^H for `halves` stacked Hermitian n x n products (A_h = rows h*n .. of A, n x k; W_h
// = rows h*n .. of W): the bs x bs blocks on and above each diagonal in ONE batched GEMM (nb
// blocks per side cost (nb + 1) / (2 nb) of the flops, and a single launch keeps the SMs full
// where a staircase of shrinking row blocks does not), then the lower triangles mirrored.
// False when n does not split into equal blocks of at least 128.
bool hermitian_blocks_batched(const DView& A, const DView& B, DView& W, int n, int k, int halves) {
    if (A.is_real && n % 128 == 0 && fp64_emu_enabled() && fp64_emu_worth(halves * n, n, k)) {
        // one FP64 product on the int8 tensor cores over the stacked halves, forming only the
        // tiles that reach each half's upper triangle, then the mirror
        gemm_f64_emu('n', 't', halves * n, n, k, 1.0, A, B, 0.0, W, n);
        for (int hf = 0; hf < halves; ++hf) {
            DView Wh = W;
            Wh.rows = Wh.cols = n;
            Wh.p = (char*)W.p + (size_t)hf * n * 8;
            k_fill_lower_from_upper(Wh);
        }
        return true;
    }
    int nb = 0;
    for (int c : {8, 4, 2})
        if (n % c == 0 && n / c >= 128) {
            nb = c;
            break;
        }
    if (!nb) return false;
    const std::shared_ptr<BlockPtrs> keep = block_ptrs(A, B, W, n, halves, nb);
    const BlockPtrs& P = *keep;
    const int bs = n / nb, count = halves * nb * (nb + 1) / 2;
    Runtime& R = rt();
    OMM_CKB(cublasSetStream(R.blas, R.stream));
    if (A.is_real) {
        const double one = 1.0, zero = 0.0;
        const double* const* pa = (const double* const*)P.arrays.p;
        OMM_CKB(cublasDgemmBatched(R.blas, CUBLAS_OP_N, CUBLAS_OP_T, bs, bs, k, &one, pa, A.ld, pa + count, B.ld,
                                   &zero, (double* const*)(pa + 2 * count), W.ld, count));
    } else {
        const cuDoubleComplex one = make_cuDoubleComplex(1.0, 0.0), zero = make_cuDoubleComplex(0.0, 0.0);
        const cuDoubleComplex* const* pa = (const cuDoubleComplex* const*)P.arrays.p;
        OMM_CKB(cublasZgemmBatched(R.blas, CUBLAS_OP_N, CUBLAS_OP_C, bs, bs, k, &one, pa, A.ld, pa + count, B.ld,
                                   &zero, (cuDoubleComplex* const*)(pa + 2 * count), W.ld, count));
    }
    for (int hf = 0; hf < halves; ++hf) {
        DView Wh = W;
        Wh.rows = Wh.cols = n;
        Wh.p = (char*)W.p + (size_t)hf * n * (W.is_real ? 8 : 16);
        k_fill_lower_from_upper(Wh);
    }
    return true;
}

void hermitian_pair_nt(const DView& Y, const DView& Dir, DView& Wdd, int n, int m) {
    if (hermitian_blocks_batched(Y, Dir, Wdd, n, m, 2)) return;
    const int nb = n >= 2048 ? 8 : (n >= 768 ? 4 : (n >= 256 ? 2 : 1));
    if (nb == 1) {
        gemm('n', 'c', 2 * n, n, m, ONE, Y, Dir, ZERO, Wdd);
        return;
    }
    Runtime& R = rt();
    OMM_CKB(cublasSetStream(R.blas, R.stream));
    const int bs = (n + nb - 1) / nb;
    for (int i = 0; i < nb; ++i) {
        const int r0 = i * bs, nr = std::min(bs, n - r0), nc = n - r0;
        if (nr <= 0) break;
        const size_t ya = (size_t)r0, da = (size_t)r0, wa = (size_t)r0 + (size_t)r0 * Wdd.ld;
        if (Y.is_real) {
            const double one = 1.0, zero = 0.0;
            OMM_CKB(cublasDgemmStridedBatched(R.blas, CUBLAS_OP_N, CUBLAS_OP_T, nr, nc, m, &one, Y.as<double>() + ya,
                                              Y.ld, n, Dir.as<double>() + da, Dir.ld, 0, &zero,
                                              Wdd.as<double>() + wa, Wdd.ld, n, 2));
        } else {
            const cuDoubleComplex one = make_cuDoubleComplex(1.0, 0.0), zero = make_cuDoubleComplex(0.0, 0.0);
            OMM_CKB(cublasZgemmStridedBatched(R.blas, CUBLAS_OP_N, CUBLAS_OP_C, nr, nc, m, &one,
                                              Y.as<cuDoubleComplex>() + ya, Y.ld, n, Dir.as<cuDoubleComplex>() + da,
                                              Dir.ld, 0, &zero, Wdd.as<cuDoubleComplex>() + wa, Wdd.ld, n, 2));
        }
    }
    DView top = Wdd, bot = Wdd;
    top.rows = bot.rows = n;
    bot.p = (char*)Wdd.p + (size_t)n * (Wdd.is_real ? 8 : 16);
    k_fill_lower_from_upper(top);
    k_fill_lower_from_upper(bot);
}

// the FP64 step's products of a real problem run on the int8 tensor cores (eval_direction's
// Gram products and SpMM from shared residues, calc_G through gemm_f64_emu)
bool fp64_step_emu(const OmmCall& c) {
    return c.real && c.n % 128 == 0 && fp64_emu_enabled() && fp64_emu_worth(2 * c.n, c.n, c.m);
}

// D = G + lambda D (omm.F90:444-446) for the FP64 step; on the int8 path the same pass forms the
// exponents of D's rows for eval_direction's residues of D
void fp64_dir_update(OmmCall& c, const DView& G, DView& D, double lambda) {
    IpState& s = *c.s;
    if (fp64_step_emu(c)) {
        s.De.ensure((size_t)c.n * sizeof(int));
        oz_axpby_exps(c.n, c.m, 1.0, G, lambda, D, s.De.as<int>(), nullptr);
        s.de_ok = true;
        s.de_src = D.p;
    } else {
        double lam[2] = {lambda, 0.0};
        k_axpby(G, 'n', D, ONE, lam);
        s.de_ok = false;
    }
}

// [HC; SC] += x [HG; SG] (omm.F90:503-504, both halves at once) for the FP64 step; on the int8
// path the same pass forms the exponents of X's rows (eval_direction's Gram products) and columns
// (calc_G's product)
void fp64_x_update(OmmCall& c, double x) {
    IpState& s = *c.s;
    const int n = c.n, m = c.m;
    DView X2 = view(s.X, 2 * n, m, 2 * n, c.real), Y2 = view(s.Y, 2 * n, m, 2 * n, c.real);
    if (fp64_step_emu(c) && fp64_emu_worth(n, m, 2 * n)) {
        s.Xe_r.ensure((size_t)2 * n * sizeof(int));
        s.Xe_c.ensure((size_t)m * sizeof(int));
        oz_axpby_exps(2 * n, m, x, Y2, 1.0, X2, s.Xe_r.as<int>(), s.Xe_c.as<int>());
        s.xr_ok = s.xc_ok = true;
    } else {
        double xz[2] = {x, 0.0};
        k_axpby(Y2, 'n', X2, xz, ONE);
        s.xr_ok = s.xc_ok = false;
    }
}

// HWd/SWd, HG/SG, HWdd/SWdd for direction Dir and the quartic coefficients
// (omm.F90:388-412 before the loop with Dir = G or PG, :448-463 inside it).
void eval_direction(OmmCall& c, const DView& Dir, double coeff[5]) {
    IpState& s = *c.s;
    int n = c.n, m = c.m;
    DView X = view(s.X, 2 * n, m, 2 * n, c.real);
    DView Wd = view(s.Wd, 2 * n, n, 2 * n, c.real);
    DView Y = view(s.Y, 2 * n, m, 2 * n, c.real);
    DView Wdd = view(s.Wdd, 2 * n, n, 2 * n, c.real);
    if (fp64_step_emu(c)) {
        // both Gram products on the int8 tensor cores, sharing the residues of Dir, and -- for
        // atom-block CSC H (and S) -- the SpMM too, from the same residues
        OzOperand* od = &oz_scratch(OZS_DIR);
        OzOperand* oa = &oz_scratch(OZS_X);
        const int bits = oz_bits(m, OZ_NMOD);
        const msw_matrix* S2 = c.s_identity ? nullptr : c.Sm;
        const bool sp = c.H_csc && !c.hcb && (c.s_identity || (c.S_csc && same_pattern(c.Hm, c.Sm))) &&
                        oz_spmm_available(c.Hm, S2);
        // the exponents the last D / X update formed, when Dir is that D and X is unchanged since
        const int* de = (s.de_ok && s.de_src == Dir.p) ? s.De.as<int>() : nullptr;
        const int* xe = s.xr_ok ? s.Xe_r.as<int>() : nullptr;
        s.de_ok = s.xr_ok = false;
        oz_prepare(Dir, false, n, m, OZ_NMOD, bits, *od, sp, -1, de, sp && oz_spmm_kb_halves(S2 != nullptr));
        oz_prepare(X, false, 2 * n, m, OZ_NMOD, bits, *oa, false, -1, xe);
        oz_gemm(*oa, *od, 1.0, 0.0, Wd);                   // [HWd; SWd] = [HC; SC] Dir^T
        DView Yv = view(s.Y, S2 ? 2 * n : n, m, 2 * n, true);
        if (sp && oz_spmm(c.Hm, S2, *od, Yv)) {            // [HG; SG] = Dir [H, S]
            if (!S2) {
                DView bot = view(s.Y, n, m, 2 * n, true, n);
                copy_view(Dir, bot);
            }
        } else {
            apply_HS(c, Dir, s.Y);
        }
        oz_prepare(Y, false, 2 * n, m, OZ_NMOD, bits, *oa);
        oz_gemm(*oa, *od, 1.0, 0.0, Wdd, n);               // [HWdd; SWdd]: upper tiles of each half
        DView top = view(s.Wdd, n, n, 2 * n, true), bot = view(s.Wdd, n, n, 2 * n, true, n);
        k_fill_lower_from_upper(top);
        k_fill_lower_from_upper(bot);
    } else {
        s.de_ok = s.xr_ok = false;
        gemm('n', 'c', 2 * n, n, m, ONE, X, Dir, ZERO, Wd);  // [HWd; SWd] = [HC; SC] Dir^H
        apply_HS(c, Dir, s.Y);                                 // [HG; SG] = Dir [H, S]
        hermitian_pair_nt(Y, Dir, Wdd, n, m);                 // [HWdd; SWdd] = [HG; SG] Dir^H
    }
    r_coeff(view(s.HW, n, n, n, c.real), view(s.SW, n, n, n, c.real), view(s.Wd, n, n, 2 * n, c.real),
            view(s.Wd, n, n, 2 * n, c.real, n), view(s.Wdd, n, n, 2 * n, c.real),
            view(s.Wdd, n, n, 2 * n, c.real, n), coeff);
}

__global__ void calcG_left_real(int n, const double* SW, const double* HW, double* L) {
    size_t tot = (size_t)n * 2 * n;
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < tot; e += (size_t)gridDim.x * blockDim.x) {
        int i = (int)(e % n), j = (int)(e / n);
        double v;
        if (j < n) v = (i == j ? 4.0 : 0.0) - 2.0 * SW[i + (size_t)j * n];
        else v = -2.0 * HW[i + (size_t)(j - n) * n];
        L[e] = v;
    }
}
__global__ void calcG_left_cplx(int n, const zdbl* SW, const zdbl* HW, zdbl* L) {
    size_t tot = (size_t)n * 2 * n;
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < tot; e += (size_t)gridDim.x * blockDim.x) {
        int i = (int)(e % n), j = (int)(e / n);
        zdbl v;
        if (j < n) {
            zdbl s = SW[i + (size_t)j * n];
            v = {(i == j ? 4.0 : 0.0) - 2.0 * s.x, -2.0 * s.y};
        } else {
            zdbl h = HW[i + (size_t)(j - n) * n];
            v = {-2.0 * h.x, -2.0 * h.y};
        }
        L[e] = v;
    }
}

// calc_G (omm_ops.F90:17-39): G = 4 HC - 2 SW HC - 2 HW SC = [4I - 2SW, -2HW] [HC; SC]
void calc_G(OmmCall& c, DView& G) {
    IpState& s = *c.s;
    int n = c.n, m = c.m;
    size_t tot = (size_t)n * 2 * n;
    int grid = (int)std::min<size_t>((tot + 255) / 256, 148 * 16);
    if (c.real) calcG_left_real<<<grid, 256, 0, rt().stream>>>(n, s.SW.as<double>(), s.HW.as<double>(), s.Lg.as<double>());
    else calcG_left_cplx<<<grid, 256, 0, rt().stream>>>(n, s.SW.as<zdbl>(), s.HW.as<zdbl>(), s.Lg.as<zdbl>());
    OMM_KCHECK();
    DView L = view(s.Lg, n, 2 * n, n, c.real);
    DView X = view(s.X, 2 * n, m, 2 * n, c.real);
    if (s.xc_ok && c.real && fp64_emu_enabled() && fp64_emu_worth(n, m, 2 * n)) {
        // X's column exponents from the update that just wrote X (fp64_x_update)
        s.xc_ok = false;
        gemm_f64_emu('n', 'n', n, m, 2 * n, 1.0, L, X, 0.0, G, 0, s.Xe_c.as<int>());
        return;
    }
    s.xc_ok = false;
    gemm('n', 'n', n, m, 2 * n, ONE, L, X, ZERO, G);
}

// ---- reduced-precision stages of the "gmx" solver (products only; the state stays FP64)
struct MixedCtx {
    int ldDt = 0, ldDg = 0, ldXt = 0, ldYt = 0, ldXc = 0, ldLt = 0, ldHc = 0, ldSc = 0;
    bool dense_ready = false;
    // s.Dt / s.Dk hold the nseg-part shadows of the matrix at dir_src, written by the CG step's
    // direction update (mx_update_dir); any other write of those shadows clears it
    const void* dir_src = nullptr;
    int dir_nseg = 0;
    // the last [HG; SG] came from the group-block tensor-core SpMM: FP32 in s.Y32 (ld 2n), with
    // its row-major shadows already in s.Yt (s.Y is stale)
    bool y32 = false;
};

bool dir_kblock(const OmmCall& c) {
    return (c.H_csc && spmm_tc_available(c.Hm)) || (!c.s_identity && c.S_csc && spmm_tc_available(c.Sm));
}

// row-major bf16 shadow of A (n x m) into s.Dt (used as the A operand of A*H and the B operand of the Gram)
void mx_shadow_dir(OmmCall& c, MixedCtx& mc, const DView& A, int nseg) {
    IpState& s = *c.s;
    mc.dir_src = nullptr;
    if (!c.real) {
        // A' = [Re | Im] rows (A operand of A*H), plus the B' of conj(A) (Gram products' A^H)
        mx_cshadow_rows(A, s.Dt_h, s.Dt_l, nseg, mc.ldDt, false);
        mx_cshadow_rows(A, s.Dg_h, s.Dg_l, nseg, mc.ldDg, true);
        return;
    }
    // the k-blocked copy feeds the tensor-core SpMM of CSC operators
    bool kblock = dir_kblock(c);
    mx_shadow_rowmajor(A, s.Dt_h, s.Dt_l, nseg, mc.ldDt, kblock ? &s.Dk_h : nullptr, kblock ? &s.Dk_l : nullptr);
}

// D = lambda D + G (the CG direction, omm.F90:437-441) and, for a real problem, D's shadows in the
// same pass, for the mx_eval_direction of D that follows
void mx_update_dir(OmmCall& c, MixedCtx& mc, DView& D, const DView& G, double lambda, int nseg) {
    IpState& s = *c.s;
    if (!c.real) {
        double lam[2] = {lambda, 0.0};
        k_axpby(G, 'n', D, ONE, lam);
        return;
    }
    const bool kblock = dir_kblock(c);
    mx_update_shadow_rowmajor(D, G, 1.0, lambda, s.Dt_h, s.Dt_l, nseg, mc.ldDt, kblock ? &s.Dk_h : nullptr,
                              kblock ? &s.Dk_l : nullptr);
    mc.dir_src = D.p;
    mc.dir_nseg = nseg;
}

// out (M x N, FP64 or complex view) = A_op * B_op^T on the bf16 GEMM; for complex operands the
// shadows are the A' (M x 2K) and B' (2N x 2K) layouts and the [Re | Im] result is interleaved.
void mx_gemm(OmmCall& c, int M, int N, int K, DevBuf& ah, DevBuf& al, int lda, DevBuf& bh, DevBuf& bl, int ldb,
             int nseg, DView& out) {
    const __nv_bfloat16* Al = nseg == 3 ? al.as<__nv_bfloat16>() : nullptr;
    const __nv_bfloat16* Bl = nseg == 3 ? bl.as<__nv_bfloat16>() : nullptr;
    if (c.real) {
        gemm_bf16_tn(M, N, K, ah.as<__nv_bfloat16>(), Al, lda, bh.as<__nv_bfloat16>(), Bl, ldb, nseg, 1.0, 0.0,
                     out.as<double>(), out.ld);
        return;
    }
    c.s->cx_out.ensure((size_t)M * 2 * N * sizeof(double));
    gemm_bf16_tn(M, 2 * N, 2 * K, ah.as<__nv_bfloat16>(), Al, lda, bh.as<__nv_bfloat16>(), Bl, ldb, nseg, 1.0, 0.0,
                 c.s->cx_out.as<double>(), M);
    mx_interleave(M, N, c.s->cx_out.as<double>(), out);
}

// stacked [A H; A S] into `stack` (2n x m); requires the row-major shadow of A in s.Dt (mx_shadow_dir)
void mx_products(OmmCall& c, MixedCtx& mc, const DView& A, DevBuf& stack, int nseg) {
    IpState& s = *c.s;
    int n = c.n, m = c.m;
    DView top = view(stack, n, m, 2 * n, c.real, 0), bot = view(stack, n, m, 2 * n, c.real, n);
    auto csc_prod = [&](const msw_matrix* M, DView& out, const msw_matrix* M2, DView* out2) {
        if (spmm_tc_available(M) && (!M2 || spmm_tc_available(M2))) {
            // tensor cores, A from the k-blocked bf16 shadow of A in s.Dk
            SpmmPlanView P = spmm_plan_view(M), P2;
            if (M2) P2 = spmm_plan_view(M2);
            if (spmm_tc(s.Dk_h.as<__nv_bfloat16>(), nseg == 3 ? s.Dk_l.as<__nv_bfloat16>() : nullptr, n, m, M, P,
                        out, M2, M2 ? &P2 : nullptr, out2, nseg))
                return;
        }
        if (spmm32_available(M)) {
            mx_to_f32(A, s.D32);
            spmm32_dense_csc(s.D32.as<float>(), n, n, M, out, M2, out2);
        } else {
            spmm_dense_csc(A, M, out, ONE, ZERO, M2, out2);  // generic pattern: FP64 gather kernel
        }
    };
    auto dense_prod = [&](DevBuf& hi, DevBuf& lo, int ld, DView& out) {
        mx_gemm(c, n, m, m, s.Dt_h, s.Dt_l, mc.ldDt, hi, lo, ld, nseg, out);
    };
    if (!c.H_csc || (!c.s_identity && !c.S_csc)) {
        // dense operators: their column-major bf16 shadows are the K-major B operands of A*H, A*S
        // (complex: the B' layout of H^T, S^T)
        if (!mc.dense_ready) {
            if (c.real) {
                if (!c.H_csc) mx_shadow_colmajor(c.H, s.Hc_h, s.Hc_l, 3, mc.ldHc);
                if (!c.s_identity && !c.S_csc) mx_shadow_colmajor(c.S, s.Sc_h, s.Sc_l, 3, mc.ldSc);
            } else {
                if (!c.H_csc) mx_cshadow_cols(c.H, s.Hc_h, s.Hc_l, 3, mc.ldHc);
                if (!c.s_identity && !c.S_csc) mx_cshadow_cols(c.S, s.Sc_h, s.Sc_l, 3, mc.ldSc);
            }
            mc.dense_ready = true;
        }
    }
    if (c.H_csc && !c.s_identity && c.S_csc && same_pattern(c.Hm, c.Sm)) {
        csc_prod(c.Hm, top, c.Sm, &bot);
        return;
    }
    if (c.H_csc) csc_prod(c.Hm, top, nullptr, nullptr);
    else dense_prod(s.Hc_h, s.Hc_l, mc.ldHc, top);
    if (c.s_identity) copy_view(A, bot);
    else if (c.S_csc) csc_prod(c.Sm, bot, nullptr, nullptr);
    else dense_prod(s.Sc_h, s.Sc_l, mc.ldSc, bot);
}

// bf16 shadows of X = [HC; SC]: row-major (Gram A operand) and column-major (calc_G B operand)
void mx_X_shadows(OmmCall& c, MixedCtx& mc, int nseg) {
    IpState& s = *c.s;
    DView X = view(s.X, 2 * c.n, c.m, 2 * c.n, c.real);
    if (c.real) {
        mx_shadow_rowmajor(X, s.Xt_h, s.Xt_l, nseg, mc.ldXt);
        mx_shadow_colmajor(X, s.Xc_h, s.Xc_l, nseg, mc.ldXc);
    } else {
        mx_cshadow_rows(X, s.Xt_h, s.Xt_l, nseg, mc.ldXt, false);
        mx_cshadow_cols(X, s.Xc_h, s.Xc_l, nseg, mc.ldXc);
    }
}

// [out] (2n x n) = (stack as row-major shadow) * Dir^H  (real: Dir^T from s.Dt; complex: B' of conj(Dir))
// hermitian: both n x n halves of the product are Hermitian ([HWdd; SWdd] = Y Dir^T with
// Y = Dir [H, S]); the real GEMM then forms only the tiles that reach their upper triangles
// (n a multiple of 128) and the lower triangles are mirrored.
void mx_gram(OmmCall& c, MixedCtx& mc, DevBuf& hi, DevBuf& lo, int ld, DevBuf& out, int nseg,
             bool hermitian = false) {
    int n = c.n, m = c.m;
    DView o = view(out, 2 * n, n, 2 * n, c.real);
    if (c.real && hermitian && n % 128 == 0) {
        gemm_bf16_tn(2 * n, n, m, hi.as<__nv_bfloat16>(), nseg == 3 ? lo.as<__nv_bfloat16>() : nullptr, ld,
                     c.s->Dt_h.as<__nv_bfloat16>(), nseg == 3 ? c.s->Dt_l.as<__nv_bfloat16>() : nullptr, mc.ldDt,
                     nseg, 1.0, 0.0, o.as<double>(), o.ld, n);
        DView top = view(out, n, n, 2 * n, true), bot = view(out, n, n, 2 * n, true, n);
        k_fill_lower_from_upper(top);
        k_fill_lower_from_upper(bot);
        return;
    }
    if (c.real) mx_gemm(c, 2 * n, n, m, hi, lo, ld, c.s->Dt_h, c.s->Dt_l, mc.ldDt, nseg, o);
    else mx_gemm(c, 2 * n, n, m, hi, lo, ld, c.s->Dg_h, c.s->Dg_l, mc.ldDg, nseg, o);
}

// eval_direction with reduced-precision products (requires current X shadows)
void mx_eval_direction(OmmCall& c, MixedCtx& mc, const DView& Dir, int nseg, double coeff[5]) {
    IpState& s = *c.s;
    int n = c.n, m = c.m;
    if (mc.dir_src == Dir.p && mc.dir_nseg == nseg) mc.dir_src = nullptr;  // made by mx_update_dir
    else mx_shadow_dir(c, mc, Dir, nseg);
    mx_gram(c, mc, s.Xt_h, s.Xt_l, mc.ldXt, s.Wd, nseg);        // [HWd; SWd] = X Dir^T
    mc.y32 = false;
    if (c.real && c.H_csc && c.S_csc && !c.s_identity && same_pattern(c.Hm, c.Sm)) {
        // [HG; SG] = Dir [H, S] in FP32 on tcgen05, the Gram's row-major shadows written by the
        // same kernel
        const int ldt = (m + 7) / 8 * 8;
        const size_t tb = (size_t)2 * n * ldt * sizeof(__nv_bfloat16);
        s.Yt_h.ensure(tb);
        if (nseg == 3) s.Yt_l.ensure(tb);
        s.Y32.ensure((size_t)2 * n * m * sizeof(float));
        if (spmm_lowp_f32(s.Dk_h.as<__nv_bfloat16>(), nseg == 3 ? s.Dk_l.as<__nv_bfloat16>() : nullptr, n, m, c.Hm, c.Sm,
                     s.Y32.as<float>(), 2 * n, s.Yt_h.as<__nv_bfloat16>(),
                     nseg == 3 ? s.Yt_l.as<__nv_bfloat16>() : nullptr, ldt, nseg)) {
            mc.ldYt = ldt;
            mc.y32 = true;
        }
    }
    if (!mc.y32) {
        mx_products(c, mc, Dir, s.Y, nseg);                      // [HG; SG] = Dir [H, S]
        DView Y = view(s.Y, 2 * n, m, 2 * n, c.real);
        if (c.real) mx_shadow_rowmajor(Y, s.Yt_h, s.Yt_l, nseg, mc.ldYt);
        else mx_cshadow_rows(Y, s.Yt_h, s.Yt_l, nseg, mc.ldYt, false);
    }
    mx_gram(c, mc, s.Yt_h, s.Yt_l, mc.ldYt, s.Wdd, nseg, true);  // [HWdd; SWdd] = Y Dir^H
    const bool r = c.real;
    r_coeff(view(s.HW, n, n, n, r), view(s.SW, n, n, n, r), view(s.Wd, n, n, 2 * n, r), view(s.Wd, n, n, 2 * n, r, n),
            view(s.Wdd, n, n, 2 * n, r), view(s.Wdd, n, n, 2 * n, r, n), coeff);
}

// calc_G with the reduced-precision GEMM (requires current X shadows)
void mx_calc_G(OmmCall& c, MixedCtx& mc, DView& G, int nseg) {
    IpState& s = *c.s;
    int n = c.n, m = c.m;
    if (c.real)
        mx_calcG_left(n, view(s.SW, n, n, n, true), view(s.HW, n, n, n, true), s.Lt_h, s.Lt_l, nseg, mc.ldLt);
    else
        mx_calcG_left_cplx(n, view(s.SW, n, n, n, false), view(s.HW, n, n, n, false), s.Lt_h, s.Lt_l, nseg, mc.ldLt);
    mx_gemm(c, n, m, 2 * n, s.Lt_h, s.Lt_l, mc.ldLt, s.Xc_h, s.Xc_l, mc.ldXc, nseg, G);
}

// energy of the current W matrices: 2 tr(HW) - tr(HW SW)  (calc_coeff's coeff(0), omm_ops.F90:213)
double energy_c0(OmmCall& c) {
    int n = c.n;
    double t[2], d[2];
    r_trace(view(c.s->HW, n, n, n, c.real), t);
    r_dot(view(c.s->HW, n, n, n, c.real), view(c.s->SW, n, n, n, c.real), d);
    return 2.0 * t[0] - d[0];
}

// D = C^H * CD for a Hermitian result (CD = QW C with QW Hermitian): only the blocks on and
// above the diagonal are computed, then the lower triangle is mirrored.  For large m the blocks
// are nb x nb plain GEMMs (cuBLAS's GEMM runs about 1.4x faster per flop than its syrkx at these
// shapes; the diagonal blocks cost 1/nb extra flops); small m take syrkx / herkx.
void density_product(const DView& C, const DView& CD, DView& D) {
    Runtime& R = rt();
    int m = C.cols, n = C.rows;
    if (C.is_real && fp64_emu_enabled() && fp64_emu_worth(m, m, n)) {
        // FP64-accurate D = C^T CD on the int8 tensor cores: only the tiles reaching the upper
        // triangle when m splits into 128-row tiles, then the mirror
        gemm_f64_emu('t', 'n', m, m, n, 1.0, C, CD, 0.0, D, m % 128 == 0 ? m : 0);
        k_fill_lower_from_upper(D);
        return;
    }
    const int nb = m >= 8192 ? 8 : (m >= 2048 ? 4 : 1);
    if (nb > 1) {
        const size_t es = C.is_real ? 8 : 16;
        auto cols = [&](const DView& A, int c0, int nc) {
            DView v = A;
            v.p = (char*)A.p + (size_t)c0 * A.ld * es;
            v.cols = nc;
            return v;
        };
        const double one[2] = {1.0, 0.0}, zero[2] = {0.0, 0.0};
        const int bs = (m + nb - 1) / nb;
        for (int bi = 0; bi < nb; ++bi) {
            const int r0 = bi * bs, nr = std::min(bs, m - r0);
            if (nr <= 0) break;
            for (int bj = bi; bj < nb; ++bj) {
                const int c0 = bj * bs, nc = std::min(bs, m - c0);
                if (nc <= 0) break;
                DView Dij = D;
                Dij.p = (char*)D.p + ((size_t)r0 + (size_t)c0 * D.ld) * es;
                Dij.rows = nr;
                Dij.cols = nc;
                gemm('c', 'n', nr, nc, n, one, cols(C, r0, nr), cols(CD, c0, nc), zero, Dij);
            }
        }
        k_fill_lower_from_upper(D);
        return;
    }
    OMM_CKB(cublasSetStream(R.blas, R.stream));
    if (C.is_real) {
        double one = 1.0, zero = 0.0;
        OMM_CKB(cublasDsyrkx(R.blas, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_T, m, n, &one, C.as<double>(), C.ld,
                             CD.as<double>(), CD.ld, &zero, D.as<double>(), D.ld));
    } else {
        cuDoubleComplex one = make_cuDoubleComplex(1.0, 0.0);
        double zero = 0.0;
        OMM_CKB(cublasZherkx(R.blas, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_C, m, n, &one, C.as<cuDoubleComplex>(), C.ld,
                             CD.as<cuDoubleComplex>(), CD.ld, &zero, D.as<cuDoubleComplex>(), D.ld));
    }
    k_fill_lower_from_upper(D);
}

// W (n x n) = A B^H for a Hermitian result (A = HC or SC, B = C: C H C^H, C S C^H): the upper
// triangle as a staircase of row blocks (block i of A against rows i*bs.. of B, plain GEMMs,
// which run faster per flop than syrkx at these shapes), or syrkx / herkx for small n; the lower
// triangle is mirrored.
void hermitian_product_nt(const DView& A, const DView& B, DView& W) {
    Runtime& R = rt();
    int n = A.rows, k = A.cols;
    if (n >= 256 && hermitian_blocks_batched(A, B, W, n, k, 1)) return;
    const int nb = n >= 2048 ? 8 : (n >= 768 ? 4 : (n >= 256 ? 2 : 1));
    if (nb > 1) {
        const size_t es = A.is_real ? 8 : 16;
        const int bs = (n + nb - 1) / nb;
        const double one[2] = {1.0, 0.0}, zero[2] = {0.0, 0.0};
        for (int i = 0; i < nb; ++i) {
            const int r0 = i * bs, nr = std::min(bs, n - r0);
            if (nr <= 0) break;
            DView Ai = A, Bi = B, Wi = W;
            Ai.p = (char*)A.p + (size_t)r0 * es;
            Ai.rows = nr;
            Bi.p = (char*)B.p + (size_t)r0 * es;
            Bi.rows = n - r0;
            Wi.p = (char*)W.p + ((size_t)r0 + (size_t)r0 * W.ld) * es;
            Wi.rows = nr;
            Wi.cols = n - r0;
            gemm('n', 'c', nr, n - r0, k, one, Ai, Bi, zero, Wi);
        }
        k_fill_lower_from_upper(W);
        return;
    }
    OMM_CKB(cublasSetStream(R.blas, R.stream));
    if (A.is_real) {
        double one = 1.0, zero = 0.0;
        OMM_CKB(cublasDsyrkx(R.blas, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_N, n, k, &one, A.as<double>(), A.ld,
                             B.as<double>(), B.ld, &zero, W.as<double>(), W.ld));
    } else {
        cuDoubleComplex one = make_cuDoubleComplex(1.0, 0.0);
        double zero = 0.0;
        OMM_CKB(cublasZherkx(R.blas, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_N, n, k, &one, A.as<cuDoubleComplex>(), A.ld,
                             B.as<cuDoubleComplex>(), B.ld, &zero, W.as<cuDoubleComplex>(), W.ld));
    }
    k_fill_lower_from_upper(W);
}

// HC, SC, HW, SW recomputed from C in FP64; returns the energy 2 tr(HW) - tr(HW SW) of C.
// Ends every solve that used reduced-precision products: the energy those stages carry
// from step to step is built from their line-search coefficients, while this one is the
// functional of the returned C (and the SW the density is formed with is that of C).
double fp64_state_from_C(OmmCall& c, const DView& Cw) {
    IpState& s = *c.s;
    int n = c.n, m = c.m;
    DView HW = view(s.HW, n, n, n, c.real), SW = view(s.SW, n, n, n, c.real);
    DView HC = view(s.X, n, m, 2 * n, c.real), SC = view(s.X, n, m, 2 * n, c.real, n);
    apply_HS(c, Cw, s.X);
    hermitian_product_nt(HC, Cw, HW);
    hermitian_product_nt(SC, Cw, SW);
    return energy_c0(c);
}

// The refinement stage's gradient.  With SW = I + Delta (Delta -> 0 at the minimum):
//   G = 4 HC - 2 SW HC - 2 HW SC = 2 HC - 2 HW SC - 2 Delta HC,
// the first two terms in FP64 (one DGEMM with K = n: half of calc_G's flops) and the small
// Delta HC on the split-bf16 GEMM (error ~2^-16 |Delta| |HC|, far below the step's needs).
// Requires the current split X shadows (the HC half of Xc is the B operand).  Complex
// problems take the FP64 calc_G.
void calc_G_refine(OmmCall& c, MixedCtx& mc, DView& G) {
    if (!c.real) {
        calc_G(c, G);
        return;
    }
    IpState& s = *c.s;
    int n = c.n, m = c.m;
    DView HW = view(s.HW, n, n, n, true), SW = view(s.SW, n, n, n, true);
    DView HC = view(s.X, n, m, 2 * n, true), SC = view(s.X, n, m, 2 * n, true, n);
    const double two[2] = {2.0, 0.0}, zero[2] = {0.0, 0.0}, mtwo[2] = {-2.0, 0.0};
    k_axpby(HC, 'n', G, two, zero);                       // G = 2 HC
    gemm('n', 'n', n, m, n, mtwo, HW, SC, ONE, G);        // G -= 2 HW SC
    mx_delta_shadow(n, SW, s.Lt_h, s.Lt_l, mc.ldLt);
    gemm_bf16_tn(n, m, n, s.Lt_h.as<__nv_bfloat16>(), s.Lt_l.as<__nv_bfloat16>(), mc.ldLt,
                 s.Xc_h.as<__nv_bfloat16>(), s.Xc_l.as<__nv_bfloat16>(), mc.ldXc, 3, -2.0, 1.0, G.as<double>(),
                 G.ld);                                    // G -= 2 (SW - I) HC
}

// Recompute HC, SC, HW, SW and G from the coefficients C (CG restart at a precision switch).
// fp64_state: HC, SC, HW, SW in FP64 (energies from them are FP64-accurate); G then uses
// nseg (0 = FP64, 3 = split BF16, -1 = the refinement gradient with split X shadows).
// Otherwise all products use nseg (1 or 3).
void refresh_from_C(OmmCall& c, MixedCtx& mc, const DView& Cw, DView& G, int nseg, bool fp64_state) {
    IpState& s = *c.s;
    s.de_ok = s.xr_ok = s.xc_ok = false;  // X and the direction are rewritten here
    int n = c.n, m = c.m;
    DView HW = view(s.HW, n, n, n, c.real), SW = view(s.SW, n, n, n, c.real);
    DView HC = view(s.X, n, m, 2 * n, c.real), SC = view(s.X, n, m, 2 * n, c.real, n);
    if (fp64_state) {
        fp64_state_from_C(c, Cw);
        if (nseg == 0) {
            calc_G(c, G);
        } else if (nseg < 0) {
            mx_X_shadows(c, mc, 3);
            calc_G_refine(c, mc, G);
        } else {
            mx_X_shadows(c, mc, nseg);
            mx_calc_G(c, mc, G, nseg);
        }
        return;
    }
    mx_shadow_dir(c, mc, Cw, nseg);            // C^T shadow in the Dt slot
    mx_products(c, mc, Cw, s.X, nseg);          // [HC; SC] = C [H, S]
    mx_X_shadows(c, mc, nseg);
    mx_gram(c, mc, s.Xt_h, s.Xt_l, mc.ldXt, s.Wd, nseg);   // [HW; SW] = X C^H into the Wd slot
    copy_view(view(s.Wd, n, n, 2 * n, c.real), HW);
    copy_view(view(s.Wd, n, n, 2 * n, c.real, n), SW);
    mx_calc_G(c, mc, G, nseg);
}

// quartic line search (omm_quartic.F90:60-153)
void solve_quartic(const double c[5], double* x_min, bool* fail) {
    const double Pi = 3.141592653589793238462643383279502884197;
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
        t[1] = -2.0 * std::sqrt(Q) * std::cos((theta + 2.0 * Pi) / 3.0) - a / 3.0;
        t[2] = -2.0 * std::sqrt(Q) * std::cos((theta - 2.0 * Pi) / 3.0) - a / 3.0;
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
        double S = -(R >= 0.0 ? 1.0 : -1.0) * std::pow(std::fabs(R) + std::sqrt(R * R - Q * Q * Q), 1.0 / 3.0);
        double U = (S == 0.0) ? 0.0 : Q / S;
        *x_min = (S + U) - (a / 3.0);
        if (c[4] < 0.0) *fail = true;
    }
}

void alloc_nm(DevBuf& b, int rows, int cols, size_t es) {
    if (!b.p) b.alloc_zero(std::max<size_t>(1, (size_t)rows * cols) * es);
}

void free_state() {
    sync();
    *g_cur = OmmState();
}

}  // namespace

void solve_quartic_host(const double c[5], double* x, bool* f) { solve_quartic(c, x, f); }

int omm_run(int m, int n, msw_matrix* H, msw_matrix* S, bool new_S, double* e_min_out, msw_matrix* D_min,
            bool calc_ED, double eta, msw_matrix* C_min, bool init_C, msw_matrix* T, double scale_T, int flavour,
            int np, int ip1, double cg_tol, bool long_out, bool dealloc, const char* m_storage,
            const char* m_operation, omm_gpu_H_fn hcb = nullptr, void* hcb_user = nullptr) {
    auto t_start = std::chrono::steady_clock::now();
    g_stats = omm_gpu_stats{};
    OmmCall c;
    c.opk = parse_op(m_operation);
    Label ls = parse_storage(m_storage);
    if (ls.fmt != Fmt::Dense) fail(OMM_ERR_UNSUPPORTED, "omm: m_storage must be a dense storage label");
    c.real = ls.real;
    c.es = c.real ? 8 : 16;
    c.m = m;
    c.n = n;
    c.hcb = hcb;
    c.hcb_user = hcb_user;
    if ((!H && !hcb) || !C_min || !D_min) fail(OMM_ERR_ARG, "omm: H, D_min and C_min are required");
    if (np < 1 || ip1 < 1 || ip1 > np) fail(OMM_ERR_ARG, "omm: ip must be in 1..np");
    if (n < 1 || m < 1 || n > m) fail(OMM_ERR_ARG, "omm: need 1 <= n <= m");
    auto chk = [&](const msw_matrix* A, int r, int cc, const char* nm) {
        if (A->dim1 != r || A->dim2 != cc) fail(OMM_ERR_ARG, std::string("omm: matrix ") + nm + " has wrong dimensions");
        if (A->is_real != c.real) fail(OMM_ERR_ARG, std::string("omm: matrix ") + nm + " real/complex mismatch");
    };
    if (!hcb) chk(H, m, m, "H");
    chk(C_min, n, m, "C_min");
    chk(D_min, m, m, "D_min");
    bool have_S = (S != nullptr);
    if (have_S) chk(S, m, m, "S");
    // flavour (omm.F90:125-155)
    if (have_S && hcb) {
        // omm_callback accepts flavours 0 and 3 only (omm_callback.F90:136-155)
        c.no_S = false;
        if (flavour == 0) {}
        else if (flavour == 3) c.use_precon = true;
        else fail(OMM_ERR_ARG, "omm: illegal value of flavour");
    } else if (have_S) {
        c.no_S = false;
        if (flavour == 0) {}
        else if (flavour == 1) c.use_Cholesky = true;
        else if (flavour == 2) { c.use_Cholesky = true; c.S_is_U = true; }
        else if (flavour == 3) c.use_precon = true;
        else if (flavour == 4) { c.use_precon = true; c.pw_precon = true; }
        else fail(OMM_ERR_ARG, "omm: illegal value of flavour");
    } else {
        c.no_S = true;
    }
    c.s_identity = c.no_S || c.use_Cholesky;
    if (c.pw_precon && !calc_ED) {  // checked before any state changes
        if (!T) fail(OMM_ERR_ARG, "omm: flavour 4 needs the kinetic energy matrix T");
        if (T->dim1 != m || T->dim2 != m || T->is_real != c.real) fail(OMM_ERR_ARG, "omm: matrix T has wrong dimensions");
        if (T->dense()) fail(OMM_ERR_ARG, std::string(c.real ? "d" : "z") + "calc_PW_precon: invalid implementation");
    }
    double cg_tol_internal = (cg_tol < 0.0) ? 1.0e-9 : cg_tol;  // omm.F90:157-161
    int ip = ip1 - 1;
    Log log;

    // -------------------------------------------------------------- calc_ED (omm.F90:163-251)
    if (calc_ED) {
        if (!g_cur->allocated || g_cur->first_call[ip])
            fail(OMM_ERR_STATE, "omm: cannot calculate ED matrix before D matrix");
        IpState& s = g_cur->ip[ip];
        double x = g_cur->x_min[ip];
        DView HW = view(s.HW, n, n, n, c.real), SW = view(s.SW, n, n, n, c.real);
        DView HWd = view(s.Wd, n, n, 2 * n, c.real), HWdd = view(s.Wdd, n, n, 2 * n, c.real);
        k_w_update(HW, HWd, HWdd, x);
        double et[2] = {eta, 0.0}, met[2] = {-eta, 0.0};
        if (eta != 0.0) k_axpby(SW, 'n', HW, et, ONE);
        Staged sc, sd;
        stage_in(C_min, sc, true);
        stage_in(D_min, sd, false);
        DView CD = view(s.CD, n, m, n, c.real), W2 = view(s.work2, n, m, n, c.real);
        gemm('n', 'n', n, m, n, ONE, HW, CD, ZERO, W2);              // calc_A2: CAW = AW*C2
        gemm('c', 'n', m, m, n, ONE, sc.v, W2, ZERO, sd.v);          // A = C1^H*CAW
        if (!dealloc && eta != 0.0) k_axpby(SW, 'n', HW, met, ONE);
        stage_out(D_min, sd);
        sync();
        if (dealloc) free_state();
        return OMM_OK;
    }

    // -------------------------------------------------------------- state (omm.F90:253-303)
    if (!g_cur->allocated) {
        g_cur->first_call.assign(np, 1);
        g_cur->x_min.assign(np, 0.0);
        g_cur->ip.clear();
        g_cur->ip.resize(np);
        g_cur->allocated = true;
    }
    if ((int)g_cur->ip.size() < np) {
        g_cur->ip.resize(np);
        g_cur->first_call.resize(np, 1);
        g_cur->x_min.resize(np, 0.0);
    }
    IpState& s = g_cur->ip[ip];
    if (s.init && (s.n != n || s.m != m || s.is_real != c.real))
        fail(OMM_ERR_ARG, "omm: dimensions changed for this ip without dealloc");
    // A call that fails from here on leaves no half-updated state for this ip behind (the
    // reference stops the program in die(); here the next call starts this ip afresh).
    struct ResetOnError {
        OmmState* st;
        int ip;
        bool armed = true;
        ~ResetOnError() {
            if (!armed || ip >= (int)st->ip.size()) return;
            st->ip[ip] = IpState();
            st->first_call[ip] = 1;
        }
    } reset_on_error{g_cur, ip};
    c.s = &s;
    s.n = n; s.m = m; s.is_real = c.real;
    size_t es = c.es;
    alloc_nm(s.HW, n, n, es);
    alloc_nm(s.SW, n, n, es);
    alloc_nm(s.Wd, 2 * n, n, es);
    alloc_nm(s.Wdd, 2 * n, n, es);
    alloc_nm(s.X, 2 * n, m, es);
    alloc_nm(s.Y, 2 * n, m, es);
    alloc_nm(s.Lg, n, 2 * n, es);
    if (c.use_Cholesky) alloc_nm(s.C_Chl, n, m, es);
    if (c.use_precon && !c.pw_precon) alloc_nm(s.P, m, m, es);
    alloc_nm(s.work2, n, m, es);
    s.init = true;
    DevBuf Gb, Gpb, Db, PGb, PGpb;  // per-call work matrices, zero-filled (m_allocate)
    Gb.alloc_zero((size_t)n * m * es);
    Gpb.alloc_zero((size_t)n * m * es);
    Db.alloc_zero((size_t)n * m * es);
    if (c.use_precon) {
        PGb.alloc_zero((size_t)n * m * es);
        PGpb.alloc_zero((size_t)n * m * es);
    }

    // -------------------------------------------------------------- operands on the device
    Staged sH, sS, sT, sC;
    c.Hm = H;
    c.Sm = S;
    c.H_csc = !hcb && !H->dense();
    c.S_csc = have_S && !S->dense();
    if (hcb) {}
    // CSC operands reach the device through their column-group plans; the raw CSC arrays are
    // uploaded only by the kernels that read them (gather, scatter)
    else if (!c.H_csc) { stage_in(H, sH, true); c.H = sH.v; }
    if (have_S) {
        if (!c.S_csc) { stage_in(S, sS, true); c.S = sS.v; }
    }
    stage_in(C_min, sC, true);
    DView Cmin = sC.v;

    // -------------------------------------------------------------- Cholesky reduction (omm.F90:306-309)
    if (c.use_Cholesky) {
        if (c.H_csc || c.S_csc) fail(OMM_ERR_UNSUPPORTED, "m_dreduce: invalid implementation (Cholesky flavour needs dense H and S)");
        if (new_S && !c.S_is_U) factorize_upper(c.S);
        reduce_upper(c.S, c.H);
    }
    // -------------------------------------------------------------- preconditioner (omm.F90:312-324)
    if (c.pw_precon && new_S) {
        // calc_PW_precon (omm_ops.F90:1225-1334): P on the CSC pattern of T, value by value
        s.Pcsc = pw_precon(T, scale_T);
    } else if (c.use_precon && new_S) {
        DView P = view(s.P, m, m, m, c.real);
        DView Sd = c.S;
        DevBuf Sdense;
        if (c.S_csc) {
            Sdense.alloc_zero((size_t)m * m * es);
            Sd = view(Sdense, m, m, m, c.real);
            csc_to_dense_view(S, Sd);  // scatter S into a dense buffer
        }
        if (T) {
            if (T->dim1 != m || T->dim2 != m || T->is_real != c.real) fail(OMM_ERR_ARG, "omm: matrix T has wrong dimensions");
            if (!T->dense()) fail(OMM_ERR_UNSUPPORTED, "omm: T must be dense for the GPU preconditioner");
            stage_in(T, sT, true);
            copy_view(sT.v, P);
            double invs[2] = {1.0 / scale_T, 0.0};
            k_axpby(Sd, 'n', P, ONE, invs);
        } else {
            copy_view(Sd, P);
        }
        invert(P);
    }
    // -------------------------------------------------------------- C0 (omm.F90:329-343)
    if (g_cur->first_call[ip] && !init_C) {
        k_lcg_init(Cmin);
        double sc[2] = {1.0e-2 / std::sqrt((double)m), 0.0};
        k_scale(Cmin, sc);
    }
    if (c.use_Cholesky && (init_C || new_S)) {  // omm.F90:344-348
        DView Cc = view(s.C_Chl, n, m, n, c.real);
        copy_view(Cmin, Cc);
        transform(c.S, Cc);
    }
    DView Cw = c.use_Cholesky ? view(s.C_Chl, n, m, n, c.real) : Cmin;
    DView HW = view(s.HW, n, n, n, c.real), SW = view(s.SW, n, n, n, c.real);
    DView HC = view(s.X, n, m, 2 * n, c.real), SC = view(s.X, n, m, 2 * n, c.real, n);
    DView HG = view(s.Y, n, m, 2 * n, c.real), SG = view(s.Y, n, m, 2 * n, c.real, n);
    DView G = view(Gb, n, m, n, c.real), Gp = view(Gpb, n, m, n, c.real), D = view(Db, n, m, n, c.real);
    DView PG = view(PGb, n, m, n, c.real), PGp = view(PGpb, n, m, n, c.real);
    bool first = g_cur->first_call[ip] != 0;

    // -------------------------------------------------------------- precision stages ("gmx")
    // stage 0: BF16 products; 1: split BF16 (hi/lo); 2: HC, SC, HW, SW recomputed from C
    // in FP64 (so energies are FP64-accurate), then split-BF16 products for the last CG
    // steps -- the FP64 refinement; 3: FP64 products (the "gpu" label, and the escape
    // if stage 2 does not converge).  Each switch is a CG restart from C.  Convergence
    // is tested (e_diff <= cg_tol, omm.F90:506) only in stages 2 and 3.
    MixedCtx mc;
    s.de_ok = s.xr_ok = s.xc_ok = false;  // no exponents carried over from an earlier call
    // complex problems take the reduced-precision stages with dense H and S (the tensor-core
    // SpMM is real only)
    const bool lowp_ok = c.real || (!c.H_csc && (c.s_identity || !c.S_csc));
    int stage = (c.opk == OpKind::Mixed && lowp_ok && !c.use_precon && !c.hcb) ? 0 : 3;
    const bool used_lowp = stage < 3;
    const double stage_tol[2] = {g_mixed_tol[0], g_mixed_tol[1]};
    // The refinement starts with a steepest-descent step from a point the reduced-precision
    // stages left O(split_tol) from the minimum, so one small energy change there says less
    // than it does deep in an FP64 run: stage 2 converges at a tighter e_diff.
    const double refine_tol = g_mixed_tol[2] * cg_tol_internal;
    int stage_steps = 0;
    auto nseg_of = [](int st) { return st == 0 ? 1 : 3; };
    // grad = the FP64 gradient at the current C.  In stage 2 the slope of the line search is
    // taken from it: c1 = 4 TrHd - 2 TrHdS - 2 TrHSd (omm_ops.F90:214) equals sum(G o D), and near
    // convergence the split-BF16 traces lose it to cancellation.
    auto eval_dir = [&](const DView& Dir, double* cf, const DView& grad) {
        if (stage < 3) {
            mx_eval_direction(c, mc, Dir, nseg_of(stage), cf);
            if (stage == 2) {
                double t[2];
                r_dot(grad, Dir, t);
                cf[1] = t[0];
            }
        } else {
            eval_direction(c, Dir, cf);
        }
    };

    // -------------------------------------------------------------- initial energy and gradient (omm.F90:352-413)
    if (stage < 3) {
        refresh_from_C(c, mc, Cw, G, nseg_of(stage), false);
    } else {
    apply_op(c, Cw, true, HC);                              // calc_AW(H, C, HW, HC)
    hermitian_product_nt(HC, Cw, HW);                      // C H C^H
    if (c.s_identity) {
        bool recompute = c.use_Cholesky ? (first || init_C || new_S) : (first || init_C);
        if (recompute) hermitian_product_nt(Cw, Cw, SW);
        copy_view(Cw, SC);                                  // S = I: the S half holds C
    } else {
        if (first || init_C || new_S) {                     // calc_AW(S, C, SW, SC)
            apply_op(c, Cw, false, SC);
            hermitian_product_nt(SC, Cw, SW);
        } else {
            double xm[2] = {g_cur->x_min[ip], 0.0};
            k_axpby(SG, 'n', SC, xm, ONE);                  // SC += x_min*SG (omm.F90:366)
        }
    }
    calc_G(c, G);
    }
    if (c.use_precon) apply_precon(c, G, PG);  // omm.F90:379
    double coeff[5];
    eval_dir(c.use_precon ? PG : G, coeff, G);
    double e_min = coeff[0];

    if (log.f) {
        log.line("+---------------------------------------------+");
        if (c.use_Cholesky) log.line("| libOMM (Cholesky factorization)             |");
        else if (c.use_precon) log.line("| libOMM (preconditioning)                    |");
        else log.line("| libOMM                                      |");
        log.line("+---------------------------------------------+");
        if (long_out) log.line("|             e_min            e_diff         |");
    }

    sync();
    auto t_loop = std::chrono::steady_clock::now();
    const double wait0 = sync_wait_seconds();
    g_stats.t_setup = std::chrono::duration<double>(t_loop - t_start).count();
    // -------------------------------------------------------------- CG loop (omm.F90:429-555)
    int icg = 0;
    bool conv = false, ls_conv = false, ls_fail = false;
    const int n_step_max_outer = 100;
    long n_step_max_inner = (m < 10000) ? (long)m * n - 1 : 10000000L;
    double e_diff = 0.0;
    int outer_i = 0;
    for (outer_i = 1; outer_i <= n_step_max_outer; ++outer_i) {
        double lambda = 0.0;
        for (long j = 1; j <= n_step_max_inner; ++j) {
            double lam[2] = {lambda, 0.0};
            s.de_ok = false;
            if (c.use_precon) k_axpby(PG, 'n', D, ONE, lam);
            else if (stage < 3) mx_update_dir(c, mc, D, G, lambda, nseg_of(stage));
            else fp64_dir_update(c, G, D, lambda);
            std::swap(G, Gp);  // G_p = G; G is recomputed before it is read again
            if (c.use_precon) std::swap(PG, PGp);
            double e_min_old = e_min;
            if (icg > 0) eval_dir(D, coeff, Gp);  // G_p holds the gradient at the current C
            if (!std::isfinite(coeff[0]) || !std::isfinite(coeff[1]) || !std::isfinite(coeff[2]) ||
                !std::isfinite(coeff[3]) || !std::isfinite(coeff[4]))
                fail(OMM_ERR_NONFINITE, "omm: non-finite line-search coefficients");
            double x;
            solve_quartic(coeff, &x, &ls_fail);
            g_cur->x_min[ip] = x;
            double xz[2] = {x, 0.0}, x2[2] = {x * x, 0.0};
            if (ls_fail) {
                if (log.f) log.line("| WARNING: Rescaling coefficients!            |");
                e_min = 3.0 * e_min;
                double h[2] = {0.5, 0.0};
                k_scale(Cw, h);
                if (c.s_identity) k_scale(SC, h);  // the S half mirrors C
                s.xr_ok = s.xc_ok = false;
                ls_conv = false;
                g_stats.ls_fail++;
            } else {
                e_min = coeff[4] * (x * x) * (x * x) + coeff[3] * x * x * x + coeff[2] * x * x + coeff[1] * x + coeff[0];
                k_axpby(D, 'n', Cw, xz, ONE);
                ls_conv = true;
            }
            if (ls_fail) {
                double q[2] = {0.25, 0.0};
                k_scale(SW, q);
            } else {
                k_w_update(SW, view(s.Wd, n, n, 2 * n, c.real, n), view(s.Wdd, n, n, 2 * n, c.real, n), x);
            }
            e_diff = 2.0 * std::fabs((e_min - e_min_old) / (e_min + e_min_old));
            if (log.f && long_out) {
                char b[128];
                snprintf(b, sizeof b, "| %5d %5ld %s %s |", outer_i, j, es15(e_min).c_str(), es15(e_diff).c_str());
                log.line(b);
            }
            ++icg;
            if (stage < 3) {
                if (stage < 2) g_stats.icg_low++;
                else g_stats.icg_fp64++;
                ++stage_steps;
                // end of a stage: converged to its tolerance, reached its noise floor (the
                // energy rose), a failed line search, or a step cap
                bool rose = (e_min > e_min_old) && !ls_fail;
                bool done2 = (stage == 2) && e_diff <= refine_tol;
                bool next = (stage < 2) ? (e_diff <= stage_tol[stage] || rose || ls_fail || stage_steps >= 400)
                                        : (!done2 && (rose || ls_fail || stage_steps >= 8));
                if (next) {
                    stage = ls_fail ? 3 : stage + 1;
                    stage_steps = 0;
                    if (stage == 2) {
                        // FP64 state, the refinement gradient, and the split X shadows for the
                        // split-bf16 Gram products
                        refresh_from_C(c, mc, Cw, G, -1, true);
                    }
                    else if (stage == 3) refresh_from_C(c, mc, Cw, G, 0, true);
                    else refresh_from_C(c, mc, Cw, G, nseg_of(stage), false);
                    e_min = energy_c0(c);
                    if (log.f) {
                        char b[128];
                        snprintf(b, sizeof b, "| precision stage %d from step %5d, e_min %s |", stage, icg,
                                 es15(e_min).c_str());
                        log.line(b);
                    }
                    lambda = 0.0;  // CG restarts from the refreshed gradient
                    continue;
                }
            } else {
                g_stats.icg_fp64++;
            }
            if (stage == 2 ? e_diff <= refine_tol : (stage == 3 && e_diff <= cg_tol_internal)) {
                conv = true;
                break;
            }
            if (ls_fail) {
                double q[2] = {0.25, 0.0};
                k_scale(HW, q);
            } else {
                k_w_update(HW, view(s.Wd, n, n, 2 * n, c.real), view(s.Wdd, n, n, 2 * n, c.real), x);
            }
            if (ls_fail) {
                double h[2] = {0.5, 0.0}, f15[2] = {1.5, 0.0};
                k_scale(HC, h);
                if (!c.s_identity) k_scale(SC, h);  // with S = I the S half was halved with C
                s.xr_ok = s.xc_ok = false;
                copy_view(Gp, G);
                k_axpby(HC, 'n', G, f15, ONE);
            } else {
                // HC += x HG and SC += x SG as one update of the stacked 2n x m matrix; in the
                // reduced-precision stages of a real problem the same pass writes X's shadows
                DView X2 = view(s.X, 2 * n, m, 2 * n, c.real), Y2 = view(s.Y, 2 * n, m, 2 * n, c.real);
                if (stage < 3) {
                    s.xr_ok = s.xc_ok = false;
                    const int ns = stage < 2 ? nseg_of(stage) : 3;
                    if (c.real) {
                        mx_update_shadows(X2, Y2, x, s.Xt_h, s.Xt_l, mc.ldXt, s.Xc_h, s.Xc_l, mc.ldXc, ns,
                                          mc.y32 ? s.Y32.as<float>() : nullptr, 2 * n);
                    } else {
                        k_axpby(Y2, 'n', X2, xz, ONE);
                        mx_X_shadows(c, mc, ns);
                    }
                    // stage 2, the refinement: the gradient from the FP64 state (calc_G_refine),
                    // products of the direction in split BF16 (their errors only scale the tiny
                    // last steps)
                    if (stage < 2) mx_calc_G(c, mc, G, ns);
                    else calc_G_refine(c, mc, G);
                } else {
                    fp64_x_update(c, x);  // with the exponents of X's rows and columns
                    calc_G(c, G);
                }
            }
            if (c.use_precon) apply_precon(c, G, PG);  // omm.F90:535
            if (ls_conv) {
                double tr[2];
                if (c.use_precon) r_lambda(PG, G, Gp, PGp, tr);
                else r_lambda(G, G, Gp, Gp, tr);
                lambda = tr[0] / tr[1];
            } else {
                break;
            }
        }
        if (conv) break;
    }
    if (outer_i > n_step_max_outer && log.f) log.line("| WARNING: OMM failed to converge!            |");
    if (log.f && long_out) log.line("+---------------------------------------------+");

    if (used_lowp) {
        e_min = fp64_state_from_C(c, Cw);
        if (log.f) {
            char b[128];
            snprintf(b, sizeof b, "| FP64 energy of C:   %s          |", es15(e_min).c_str());
            log.line(b);
        }
    }
    if (unsigned eb = gemm_bf16_errors())
        fail(OMM_ERR_CUDA, "omm: a tensor-core pipeline wait timed out (error bits " + std::to_string(eb) + ")");
    sync();
    auto t_dens = std::chrono::steady_clock::now();
    g_stats.t_loop = std::chrono::duration<double>(t_dens - t_loop).count();
    g_stats.t_loop_sync = sync_wait_seconds() - wait0;
    // -------------------------------------------------------------- density (omm.F90:569-593)
    alloc_nm(s.QW, n, n, es);
    alloc_nm(s.CD, n, m, es);
    DView QW = view(s.QW, n, n, n, c.real), CD = view(s.CD, n, m, n, c.real);
    double two[2] = {2.0, 0.0};
    k_set(QW, 'a', ZERO, two);
    k_axpby(SW, 'n', QW, MONE, ONE);
    if (c.use_Cholesky) {
        copy_view(view(s.C_Chl, n, m, n, c.real), Cmin);
        back_transform(c.S, Cmin);
    }
    Staged sD;
    stage_in(D_min, sD, false);
    gemm('n', 'n', n, m, n, ONE, QW, Cmin, ZERO, CD);     // calc_A: CAW = QW*C
    density_product(Cmin, CD, sD.v);                      // D = C^H*CAW (Hermitian: one triangle, then mirrored)
    double trqs[2];
    r_dot(QW, SW, trqs);
    double TrQS = trqs[0];
    if (log.f) {
        char b[128];
        snprintf(b, sizeof b, "| minim: icg           = %5d                |", icg);
        log.line(b);
        snprintf(b, sizeof b, "| minim: Tr[(2*I-S)*S] = %13.7f        |", TrQS);
        log.line(b);
        log.line("+---------------------------------------------+");
    }
    e_min = e_min + TrQS * eta;
    *e_min_out = e_min;

    // outputs back to host storages
    stage_out(C_min, sC);
    stage_out(D_min, sD);
    if (c.use_Cholesky) {
        if (!c.H_csc) stage_out(H, sH);
        if (!c.S_csc) stage_out(S, sS);
    }
    sync();
    g_stats.icg = icg;
    g_stats.converged = conv ? 1 : 0;
    g_stats.e_min = e_min;
    g_stats.e_diff = e_diff;
    g_stats.trqs = TrQS;
    reset_on_error.armed = false;
    if (dealloc) free_state();
    else g_cur->first_call[ip] = 0;
    auto t_end = std::chrono::steady_clock::now();
    g_stats.t_final = std::chrono::duration<double>(t_end - t_dens).count();
    g_stats.seconds = std::chrono::duration<double>(t_end - t_start).count();
    return conv ? OMM_OK : OMM_NOT_CONVERGED;
}

}  // namespace ommgpu

using namespace ommgpu;

extern "C" {

int omm_gpu_callback(int m, int n, omm_gpu_H_fn H, void* user, msw_matrix* S, bool new_S, double* e_min,
                     msw_matrix* D_min, bool calc_ED, double eta, msw_matrix* C_min, bool init_C, msw_matrix* T,
                     double scale_T, int flavour, int np, int ip, double cg_tol, bool long_out, bool dealloc,
                     const char m_storage[5], const char m_operation[3]) {
    try {
        if (!H) fail(OMM_ERR_ARG, "omm_callback: H routine is required");
        g_cur = &g_state_cb;
        int rc = omm_run(m, n, nullptr, S, new_S, e_min, D_min, calc_ED, eta, C_min, init_C, T, scale_T, flavour, np,
                         ip, cg_tol, long_out, dealloc, m_storage, m_operation, H, user);
        g_cur = &g_state;
        set_last_error(rc == OMM_NOT_CONVERGED ? "omm: OMM failed to converge" : "");
        return rc;
    } catch (const Error& e) {
        g_cur = &g_state;
        set_last_error(e.msg);
        return e.code;
    } catch (const std::exception& e) {
        g_cur = &g_state;
        set_last_error(e.what());
        return OMM_ERR_ARG;
    }
}

int omm_gpu(int m, int n, msw_matrix* H, msw_matrix* S, bool new_S, double* e_min, msw_matrix* D_min, bool calc_ED,
            double eta, msw_matrix* C_min, bool init_C, msw_matrix* T, double scale_T, int flavour, int np, int ip,
            double cg_tol, bool long_out, bool dealloc, const char m_storage[5], const char m_operation[3]) {
    try {
        g_cur = &g_state;
        int rc = omm_run(m, n, H, S, new_S, e_min, D_min, calc_ED, eta, C_min, init_C, T, scale_T, flavour, np, ip,
                         cg_tol, long_out, dealloc, m_storage, m_operation);
        set_last_error(rc == OMM_NOT_CONVERGED ? "omm: OMM failed to converge" : "");
        return rc;
    } catch (const Error& e) {
        set_last_error(e.msg);
        return e.code;
    } catch (const std::exception& e) {
        set_last_error(e.what());
        return OMM_ERR_ARG;
    }
}

int omm_gpu_get_stats(omm_gpu_stats* st) {
    if (!st) return OMM_ERR_ARG;
    *st = g_stats;
    return OMM_OK;
}

int omm_gpu_set_log(const char* path) {
    if (!path) {
        g_log_enabled = false;
    } else {
        g_log_enabled = true;
        g_log_path = path;
        g_log_start = false;
    }
    return OMM_OK;
}

int omm_gpu_set_mixed(double bf16_tol, double split_tol, double refine_factor) {
    if (!(bf16_tol > 0.0) || !(split_tol > 0.0) || !(refine_factor > 0.0) || refine_factor > 1.0) return OMM_ERR_ARG;
    g_mixed_tol[0] = bf16_tol;
    g_mixed_tol[1] = split_tol;
    g_mixed_tol[2] = refine_factor;
    return OMM_OK;
}

int omm_gpu_finalize(void) {
    try {
        g_state = OmmState();
        g_state_cb = OmmState();
        if (rt().stream) sync();
        rt().scratch.release();
        rt().scratch2.release();
        oz_release_scratch();
        pool_trim();
        spmm_plan_cache_clear();
        host_pool_release();
        {
            std::lock_guard<std::mutex> lk(g_block_ptrs_mu);
            g_block_ptrs.clear();
        }
    } catch (const Error& e) {
        set_last_error(e.msg);
        return e.code;
    }
    return OMM_OK;
}

}  // extern "C"
