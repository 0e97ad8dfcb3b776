// Internal declarations of the B200 libOMM library (not part of the C ABI).
#pragma once

#include <cuda_runtime.h>
#include <cublas_v2.h>
#include <cusolverDn.h>
#include <cuda_bf16.h>

#include <functional>
#include <memory>
#include <string>
#include <utility>
#include <vector>

#include "ommgpu.h"

namespace ommgpu {

// ----------------------------------------------------------------- errors
struct Error {
    int code;
    std::string msg;
};
[[noreturn]] void fail(int code, const std::string& msg);
void set_last_error(const std::string& msg);

#define OMM_CK(x)                                                                                     \
    do {                                                                                              \
        cudaError_t e_ = (x);                                                                         \
        if (e_ != cudaSuccess)                                                                        \
            ::ommgpu::fail(e_ == cudaErrorMemoryAllocation ? OMM_ERR_ALLOC : OMM_ERR_CUDA,            \
                           std::string(#x) + ": " + cudaGetErrorString(e_));                          \
    } while (0)
#define OMM_CKB(x)                                                                                    \
    do {                                                                                              \
        cublasStatus_t s_ = (x);                                                                      \
        if (s_ != CUBLAS_STATUS_SUCCESS)                                                              \
            ::ommgpu::fail(OMM_ERR_CUDA, std::string(#x) + ": cublas status " + std::to_string((int)s_)); \
    } while (0)
#define OMM_CKS(x)                                                                                    \
    do {                                                                                              \
        cusolverStatus_t s_ = (x);                                                                    \
        if (s_ != CUSOLVER_STATUS_SUCCESS)                                                            \
            ::ommgpu::fail(OMM_ERR_CUDA, std::string(#x) + ": cusolver status " + std::to_string((int)s_)); \
    } while (0)
// Every launch of a kernel of this library is followed by OMM_KCHECK(), which
// also counts it (omm_gpu_kernel_launches()).
long long count_launch();
#define OMM_KCHECK()                   \
    do {                               \
        ::ommgpu::count_launch();      \
        OMM_CK(cudaGetLastError());    \
    } while (0)

// Per-kernel timing with CUDA events on the library stream around selected launches (the
// dominant kernels of the solvers), off unless omm_gpu_kernel_timing(1) turned it on.
// ktime_begin() before the launch, ktime_end(name, work) after it with the launch's
// algorithmic work (flops, int8 ops or bytes, as the kernel's roofline counts it).
bool ktime_on();
void ktime_begin();
void ktime_end(const char* name, double work);

// ----------------------------------------------------------------- complex
struct __align__(16) zdbl {
    double x, y;
};

// ----------------------------------------------------------------- device memory
struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    bool owns = true;  // false when aliasing caller memory (msw_register_gden)
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    DevBuf(DevBuf&& o) noexcept : p(o.p), bytes(o.bytes), owns(o.owns) { o.p = nullptr; o.bytes = 0; }
    DevBuf& operator=(DevBuf&& o) noexcept {
        if (this != &o) { release(); p = o.p; bytes = o.bytes; owns = o.owns; o.p = nullptr; o.bytes = 0; }
        return *this;
    }
    ~DevBuf() { release(); }
    void alloc(size_t b);         // uninitialised
    void alloc_zero(size_t b);    // zero-filled (on the library stream)
    void ensure(size_t b);        // grow-only
    void release();
    template <typename T> T* as() const { return (T*)p; }
};

// ----------------------------------------------------------------- runtime
struct Runtime {
    int device = -1;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    cublasHandle_t blas = nullptr;
    cusolverDnHandle_t solver = nullptr;
    DevBuf scratch;   // reduction partials and small temporaries
    DevBuf scratch2;  // transposes / staging
    double* host_pinned = nullptr;  // small pinned host buffer for scalar read-back
};
Runtime& rt();
bool runtime_bound();  // rt() has been set up on a device (no CUDA call is made to find out)
void sync();
double sync_wait_seconds();  // host time spent in sync() so far
void pool_trim();  // return cached device blocks to the driver

// ----------------------------------------------------------------- host memory
// Large host arrays (CSC copies of registered matrices, column-group blocks) come from a
// pool: a freed block is kept and handed to the next request of the same size, so an SCF
// caller that registers H and S afresh every cycle pays no page faults for their copies.
// Blocks below 1 MiB go straight to malloc; the pool keeps at most 4 GiB, oldest freed first.
void* host_pool_get(size_t bytes);
void host_pool_put(void* p, size_t bytes);
void host_pool_release();  // free every cached block
size_t host_pool_cached_bytes();

// std::vector allocator over the pool.  Elements are default-initialised (resize() does not
// zero-fill), so every user writes what it resizes.
template <typename T>
struct HostAlloc {
    using value_type = T;
    HostAlloc() = default;
    template <typename U>
    HostAlloc(const HostAlloc<U>&) {}
    T* allocate(size_t n) { return static_cast<T*>(host_pool_get(n * sizeof(T))); }
    void deallocate(T* p, size_t n) { host_pool_put(p, n * sizeof(T)); }
    template <typename U>
    void construct(U* p) { ::new ((void*)p) U; }
    template <typename U, typename... A>
    void construct(U* p, A&&... a) { ::new ((void*)p) U(std::forward<A>(a)...); }
    template <typename U>
    bool operator==(const HostAlloc<U>&) const { return true; }
    template <typename U>
    bool operator!=(const HostAlloc<U>&) const { return false; }
};
template <typename T>
using HostVec = std::vector<T, HostAlloc<T>>;

// f(begin, end) over [0, count) split across up to 16 host threads (one thread below
// 64 items per thread).  f must not throw: record failures and report them after the call.
void host_parallel(long long count, const std::function<void(long long, long long)>& f);
void spmm_plan_cache_clear();  // drop the column-group plans kept by pattern (spmm.cu)

// ----------------------------------------------------------------- matrix handle
enum class Loc { Host, Device };
enum class Fmt { Dense, CSC };

struct SpmmPlan;    // column-group plan of a CSC matrix (spmm.cu)
struct SpmmTcPlan;  // its tensor-core form (spmm_tc.cu)
struct SpmmTc2Plan; // its tensor-core form over blocks of groups (spmm_tc2.cu)
struct OzSpmmPlan;  // its int8 form for the FP64 products (ozaki.cu)

// A fresh identifier for a CSC pattern (never reused): given to every matrix at creation and
// again whenever its pattern or values change, so comparisons of patterns can be memoised.
unsigned long long next_pattern_id();

}  // namespace ommgpu

struct msw_matrix {
    int dim1 = 0, dim2 = 0;
    bool is_real = true;
    ommgpu::Loc loc = ommgpu::Loc::Device;
    ommgpu::Fmt fmt = ommgpu::Fmt::Dense;
    char label[6] = "gdden";
    // dense
    void* host = nullptr;              // host data (aliased caller array or host_store)
    std::vector<double> host_store;    // owned host data of 's' matrices made by msw_allocate
    ommgpu::DevBuf dev;                // device data of 'g' dense matrices (ld = dim1)
    // CSC (host copy always kept, 0-based)
    int nnz = 0;
    ommgpu::HostVec<int> h_colptr, h_rowind;
    ommgpu::HostVec<double> h_val;     // nnz reals or 2*nnz interleaved complex
    ommgpu::DevBuf d_colptr, d_rowind, d_val;
    unsigned long long pattern_id = ommgpu::next_pattern_id();
    std::shared_ptr<ommgpu::SpmmPlan> plan;       // lazily built
    std::shared_ptr<ommgpu::SpmmTcPlan> tc_plan;  // lazily built (empty plan = not eligible)
    std::shared_ptr<ommgpu::SpmmTc2Plan> tc2_plan, tc2_plan_split;  // group-block forms (bf16, split)
    std::shared_ptr<ommgpu::OzSpmmPlan> oz_plan;  // int8 form (with the S of the same pattern), lazily built
    std::shared_ptr<msw_matrix> transposed;       // CSC of the (conjugate-free) transpose, lazily built
    std::shared_ptr<msw_matrix> conj_transposed;  // CSC of the conjugate transpose (complex), lazily built
    size_t esize() const { return is_real ? 8 : 16; }
    size_t elems() const { return (size_t)dim1 * dim2; }
    bool dense() const { return fmt == ommgpu::Fmt::Dense; }
};

namespace ommgpu {

// A device view of a dense matrix: pointer + leading dimension + element type.
struct DView {
    void* p = nullptr;
    int rows = 0, cols = 0, ld = 0;
    bool is_real = true;
    template <typename T> T* as() const { return (T*)p; }
};

// Parse/validate labels
struct Label {
    char where;   // 's', 'p', 'g'
    bool real;    // 'd' vs 'z'
    Fmt fmt;
};
Label parse_storage(const char* label);
enum class OpKind { FP64, Mixed };
OpKind parse_op(const char* label);

// host <-> device staging of a matrix handle for one operation
struct Staged {
    DView v;
    DevBuf tmp;
    const msw_matrix* src = nullptr;
};
void stage_in(const msw_matrix* A, Staged& s, bool copy_data = true);
void stage_out(msw_matrix* A, const Staged& s);
void ensure_csc_device(const msw_matrix* A);
const msw_matrix* csc_transpose(const msw_matrix* A);

// ----------------------------------------------------------------- kernels (kernels.cu)
// Elementwise on column-major views; 'op' in {'n','t','c'} applies to A.
void k_axpby(const DView& A, char op, DView& C, const double alpha[2], const double beta[2]);
void k_scale(DView& C, const double beta[2]);
void k_set(DView& C, char seC, const double alpha[2], const double beta[2]);
void k_set_element(DView& C, int i, int j, const double alpha[2], const double beta[2]);
void k_fill_lower_from_upper(DView& C);      // C(j,i) = conj(C(i,j)) for j > i
void k_w_update(DView& W, const DView& Wd, const DView& Wdd, double x);  // W += x (Wd^H + Wd) + x^2 Wdd
void k_lcg_init(DView& C);                   // reference C0 (NORAND LCG), unscaled
// reductions (deterministic two-pass); results copied to host
void r_trace(const DView& A, double out[2]);                          // sum of diagonal
void r_dot(const DView& A, const DView& B, double out[2]);            // sum conj(A) B
void r_coeff(const DView& HW, const DView& SW, const DView& HWd, const DView& SWd, const DView& HWdd,
             const DView& SWdd, double coeff[5]);                     // calc_coeff traces
void r_lambda(const DView& PG, const DView& G, const DView& Gp, const DView& PGp, double out[2]);
// dense products on cuBLAS (FP64 / complex FP64)
void gemm(char opA, char opB, int M, int N, int K, const double alpha[2], const DView& A, const DView& B,
          const double beta[2], DView& C);
void transpose_into(const DView& A, char op, DView& T);  // T = op(A)

// ----------------------------------------------------------------- SpMM (spmm.cu)
// C = alpha * A * B + beta * C with A dense (op 'n'), B CSC (op 'n').
// B2/C2 optional second matrix with the same sparsity pattern (fused H and S).
void spmm_dense_csc(const DView& A, const msw_matrix* B, DView& C, const double alpha[2], const double beta[2],
                    const msw_matrix* B2 = nullptr, DView* C2 = nullptr);
void spmm_dense_csc_gather(const DView& A, const msw_matrix* B, DView& C, const double alpha[2],
                           const double beta[2]);
bool same_pattern(const msw_matrix* A, const msw_matrix* B);
// general psp_gemspm / psp_gespmm with all op combinations
void gemspm(char opA, const DView& A, char opB, const msw_matrix* B, DView& C, const double alpha[2],
            const double beta[2]);
void gespmm(char opA, const msw_matrix* A, char opB, const DView& B, DView& C, const double alpha[2],
            const double beta[2]);
// statistics of the plan (for benches/tests)
struct SpmmInfo {
    int group_width;
    int ngroups;
    double efficiency;
    long long union_rows;
    bool cgu;
};
SpmmInfo spmm_info(const msw_matrix* B);

void csc_to_dense_view(const msw_matrix* A, DView& out);

// ----------------------------------------------------------------- tensor-core GEMM (gemm_tc.cu)
// out (FP64, M x N, col-major) = alpha * sum_seg A_seg B_seg^T + beta * out; bf16 K-major operands.
// herm > 0 (a multiple of 128 dividing M): out is a stack of Hermitian herm x herm blocks, of which
// only the tiles reaching the upper triangles are formed; the caller mirrors the lower ones.
void gemm_bf16_tn(int M, int N, int K, const __nv_bfloat16* A_hi, const __nv_bfloat16* A_lo, int lda,
                  const __nv_bfloat16* B_hi, const __nv_bfloat16* B_lo, int ldb, int nseg, double alpha, double beta,
                  double* out, int ldo, int herm = 0);
unsigned gemm_bf16_errors();

// ----------------------------------------------------------------- FP64 GEMM on the int8 tensor cores (ozaki.cu)
// Residues of one operand (rows x K, K-major int8 planes, one per modulus) and its row exponents.
struct OzOperand {
    DevBuf planes, exps;
    int rows = 0, K = 0, ldk = 0, nmod = 0, bits = 0;
    size_t plane = 0;
    // optional k-blocked copy (the int8 SpMM's A operand): per modulus, blocks of 256 rows, each
    // ldk / 16 chunks of 256 rows x 16 B
    DevBuf kb;
    size_t kb_plane = 0;
    bool kb_halves = false;  // kb per 128-row half of each block (the SM-pair SpMM's layout)
};
constexpr int OZ_NMOD = 16;    // moduli of the FP64-accurate products (53-bit operands for K < 2^17)
// the residues kept between products (grow-only device buffers, released by oz_release_scratch,
// which omm_gpu_finalize calls): the CG step's direction and [HC; SC], the two operands of
// gemm_f64_emu, the operand of omm_gpu_spmm_f64
enum { OZS_DIR = 0, OZS_X, OZS_GEMM_A, OZS_GEMM_B, OZS_GEMM_AI, OZS_GEMM_BI, OZS_SPMM_A, OZS_COUNT };
OzOperand& oz_scratch(int slot);
void oz_release_scratch();
int oz_bits(int K, int nmod);  // bits each operand keeps for inner dimension K
// src: FP64 column-major; kcontig: element (r, k) at src[k + r ld] (else at src[r + k ld])
// part: -1 for a real source; 0 / 1 for the real / imaginary part of a complex one
// exps_in: the operand's row exponents already formed (oz_axpby_exps), copied instead of recomputed
// kb_halves: the k-blocked copy in the SM-pair SpMM's half-major layout (oz_spmm_kb_halves)
void oz_prepare(const DView& src, bool kcontig, int rows, int K, int nmod, int bits, OzOperand& op,
                bool with_kb = false, int part = -1, const int* exps_in = nullptr, bool kb_halves = false);
// the SpMM's form wants A's k-blocked copy half-major (the SM-pair form, for products with S)
bool oz_spmm_kb_halves(bool with_s);
// Y = beta Y + alpha X (real, R x K, rows contiguous) with the exponents oz_prepare would form of
// Y's rows (erow, R ints) and of its columns (ecol, K ints: the rows of Y^T); either may be null
void oz_axpby_exps(int R, int K, double alpha, const DView& X, double beta, DView& Y, int* erow, int* ecol);
// out (A.rows x B.rows) = alpha * A B^T + beta * out; herm as for gemm_bf16_tn
// out_part 0 / 1: C is complex and the product goes to its real / imaginary part
void oz_gemm(const OzOperand& A, const OzOperand& B, double alpha, double beta, DView& C, int herm = 0,
             int out_part = -1);
// Y = A [H, S] in FP64 on the int8 tensor cores (S's product n rows below H's; H's only when S is
// null) for real CSC H (and S of H's pattern) with a column-group plan; A's residues must carry
// the k-blocked copy.  False (nothing done) when the matrices do not fit.
bool oz_spmm_available(const msw_matrix* H, const msw_matrix* S);
bool oz_spmm(const msw_matrix* H, const msw_matrix* S, const OzOperand& A, DView& Y);
// real op(A) op(B) (ops 'n'/'t') through oz_prepare + oz_gemm
// b_exps: the exponents of op(B)'s columns already formed (oz_axpby_exps)
void gemm_f64_emu(char opA, char opB, int M, int N, int K, double alpha, const DView& A, const DView& B, double beta,
                  DView& C, int herm = 0, const int* b_exps = nullptr);
// complex op(A) op(B) (ops 'n', 't', 'c'; real alpha, beta) as four real FP64-accurate products
void gemm_z_emu(char opA, char opB, int M, int N, int K, double alpha, const DView& A, const DView& B, double beta,
                DView& C);
bool fp64_emu_enabled();  // real FP64 GEMMs of the solver on the int8 tensor cores (default on)
void set_fp64_emu(int mode, long long panel_bytes);
size_t oz_panel_bytes();
bool fp64_emu_worth(int M, int N, int K);  // large enough for the emulation to pay

// ----------------------------------------------------------------- tensor-core SpMM (spmm_tc.cu)
struct SpmmPlanView {
    bool cgu = false;
    int G = 0, ngroups = 0;
    const int* gptr = nullptr;   // host, ngroups + 1
    const int* urows = nullptr;  // host
    const int* d_gptr = nullptr;
    const double* d_bvals = nullptr;
};
SpmmPlanView spmm_plan_view(const msw_matrix* B);
SpmmTcPlan* spmm_tc_plan(const msw_matrix* B, const SpmmPlanView& P);
// k-blocked bf16 shadow of an n x K matrix (the tensor-core SpMM's A operand), tile-major: for each
// block of KBLOCK_ROWS rows, the ceil(K/8) planes of KBLOCK_ROWS x 8 values one after another, so a
// run of consecutive 8-k chunks of one row block is one contiguous range
constexpr int KBLOCK_ROWS = 256;
__host__ __device__ inline size_t kblock_offset(int i, int k, int K) {  // element (i, k)
    const size_t planes = (size_t)(K + 7) / 8;
    return (((size_t)(i / KBLOCK_ROWS) * planes + (size_t)(k / 8)) * KBLOCK_ROWS + (size_t)(i % KBLOCK_ROWS)) * 8 +
           (size_t)(k % 8);
}
inline size_t kblock_elems(int n, int K) {
    return (size_t)((n + KBLOCK_ROWS - 1) / KBLOCK_ROWS) * KBLOCK_ROWS * (size_t)((K + 7) / 8) * 8;
}
bool spmm_tc(const __nv_bfloat16* Dk_hi, const __nv_bfloat16* Dk_lo, int n, int K, const msw_matrix* B,
             const SpmmPlanView& P, DView& C, const msw_matrix* B2, const SpmmPlanView* P2, DView* C2, int nseg);
bool spmm_tc_available(const msw_matrix* B);
// Y (FP32; with S, S's product at rows n..2n-1) = A [H, S] over blocks of column groups, with the
// row-major bf16 shadows of Y when t_hi is given (spmm_tc2.cu); false when not eligible
bool spmm_tc2(const __nv_bfloat16* Dk_hi, const __nv_bfloat16* Dk_lo, int n, int m, const msw_matrix* H,
              const msw_matrix* S, float* y, int ldy, __nv_bfloat16* t_hi, __nv_bfloat16* t_lo, int ldt, int nseg);
// the same with one column group per CTA (spmm_tc.cu)
bool spmm_tc_f32(const __nv_bfloat16* Dk_hi, const __nv_bfloat16* Dk_lo, int n, int m, const msw_matrix* H,
                 const msw_matrix* S, float* y, int ldy, __nv_bfloat16* t_hi, __nv_bfloat16* t_lo, int ldt, int nseg);
// whichever of the two omm_gpu_set_spmm_groups selects (default: one group per CTA)
bool spmm_lowp_f32(const __nv_bfloat16* Dk_hi, const __nv_bfloat16* Dk_lo, int n, int m, const msw_matrix* H,
                   const msw_matrix* S, float* y, int ldy, __nv_bfloat16* t_hi, __nv_bfloat16* t_lo, int ldt, int nseg);

// ----------------------------------------------------------------- reduced-precision helpers (mixed.cu, spmm.cu)
bool spmm32_available(const msw_matrix* B);
void spmm32_dense_csc(const float* A, int lda, int n, const msw_matrix* B, DView& C, const msw_matrix* B2,
                      DView* C2);
void mx_shadow_rowmajor(const DView& src, DevBuf& hi, DevBuf& lo, int nseg, int& ldd, DevBuf* khi = nullptr,
                        DevBuf* klo = nullptr);
void mx_shadow_kblock(const DView& src, DevBuf& khi, DevBuf& klo, int nseg);

// ----------------------------------------------------------------- format conversions (convert.cu)
// Dense device view -> CSC (host arrays + device copy) keeping, per `mode`, all entries (0),
// |a| > thr (1), |a| >= thr (2) or the nonzeros (3); kept values are shifted by soft (soft threshold).
void dense_to_csc(const DView& A, int mode, double thr, double soft, msw_matrix* M);
void threshold_dense(DView& A, double thr, double soft);
void mx_shadow_colmajor(const DView& src, DevBuf& hi, DevBuf& lo, int nseg, int& ldd);
// D = b*D + a*G in place, with the row-major (and k-blocked) shadows of the result (one pass; real)
void mx_update_shadow_rowmajor(DView& D, const DView& G, double a, double b, DevBuf& hi, DevBuf& lo, int nseg,
                               int& ldd, DevBuf* khi, DevBuf* klo);
// X += a*Y in place, with the row-major and column-major shadows of the result (one pass; real)
void mx_update_shadows(DView& X, const DView& Y, double a, DevBuf& thi, DevBuf& tlo, int& ldt, DevBuf& chi,
                       DevBuf& clo, int& ldc, int nseg, const float* Y32 = nullptr, int ldy32 = 0);
void mx_to_f32(const DView& src, DevBuf& dst);
void mx_calcG_left(int n, const DView& SW, const DView& HW, DevBuf& hi, DevBuf& lo, int nseg, int& ldl);
void mx_delta_shadow(int n, const DView& SW, DevBuf& hi, DevBuf& lo, int& ldd);
// complex products as real GEMMs (mixed.cu): A' rows [Re | Im]; with conj_b also the B' rows of
// conj(src); B' of src^T from columns; the [Re | Im] product interleaved into a complex view
void mx_cshadow_rows(const DView& src, DevBuf& hi, DevBuf& lo, int nseg, int& ldd, bool conj_b);
void mx_cshadow_cols(const DView& src, DevBuf& hi, DevBuf& lo, int nseg, int& ldd);
void mx_interleave(int M, int N, const double* re, DView& dst);
void mx_calcG_left_cplx(int n, const DView& SW, const DView& HW, DevBuf& hi, DevBuf& lo, int nseg, int& ldl);

// ----------------------------------------------------------------- omm per-ip state (omm.cu)
struct IpState {
    bool init = false;
    int n = 0, m = 0;
    bool is_real = true;
    DevBuf HW, SW;      // n x n
    DevBuf Wd, Wdd;     // [HWd; SWd], [HWdd; SWdd]: 2n x n, leading dimension 2n
    DevBuf X, Y;        // [HC; SC], [HG; SG]: 2n x m, leading dimension 2n
    DevBuf C_Chl;       // n x m
    DevBuf P;           // m x m
    DevBuf work2, CD;   // n x m
    DevBuf QW;          // n x n
    DevBuf Lg;          // n x 2n left factor of calc_G
    // bf16 / FP32 shadows of the reduced-precision stages (mixed.cu)
    DevBuf cb_out;  // contiguous n x m result of omm_callback's H routine
    DevBuf Dg_h, Dg_l;  // complex mixed solver: the B' shadow of conj(D) for the Gram products
    DevBuf cx_out;      // complex mixed solver: [Re | Im] results of the real GEMMs
    std::shared_ptr<msw_matrix> Pcsc;  // flavour 4's preconditioner (CSC, T's pattern)
    DevBuf Dt_h, Dt_l, Dk_h, Dk_l, Xt_h, Xt_l, Yt_h, Yt_l, Xc_h, Xc_l, Lt_h, Lt_l, Hc_h, Hc_l, Sc_h, Sc_l;
    DevBuf D32;         // FP32 copy of the direction for the SpMM
    DevBuf Y32;         // [HG; SG] in FP32 from the group-block tensor-core SpMM (2n x m, ld 2n)
    // exponents formed by the FP64 step's D and X updates (oz_axpby_exps) for the next products
    // of the unchanged matrices: D's rows, X's rows and X's columns.  Each flag is set by its
    // update and cleared by the product that uses it or by any other write of the matrix.
    DevBuf De, Xe_r, Xe_c;
    bool de_ok = false, xr_ok = false, xc_ok = false;
    const void* de_src = nullptr;  // the direction matrix De belongs to
};

struct OmmCall {
    int m = 0, n = 0;
    bool real = true;
    size_t es = 8;
    IpState* s = nullptr;
    DView H, S;                 // dense views when dense
    const msw_matrix* Hm = nullptr;
    const msw_matrix* Sm = nullptr;
    bool H_csc = false, S_csc = false;
    bool no_S = false, use_Cholesky = false, S_is_U = false, use_precon = false;
    bool s_identity = false;    // S == I inside the CG loop (no S, or Cholesky flavour)
    OpKind opk = OpKind::FP64;
    bool pw_precon = false;      // flavour 4: P on T's CSC pattern
    omm_gpu_H_fn hcb = nullptr;  // omm_callback's H routine (H applied by the caller)
    void* hcb_user = nullptr;
};

}  // namespace ommgpu
