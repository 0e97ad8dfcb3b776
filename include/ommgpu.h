/*
 * ommgpu.h — C ABI of the B200 (sm_100a) libOMM / MatrixSwitch / pspBLAS library.
 *
 * Every entry point replaces one routine of the reference's Fortran API; the
 * comment above each declaration names the reference routine it replaces
 * (file:line inside the reference project).  A Fortran caller reaches these
 * through the ISO_C_BINDING shim in omm-bundle_b200/fortran/; C, C++ and
 * Python (ctypes) call them directly.
 *
 * Conventions
 *   - Matrices are opaque handles (msw_matrix*), the counterpart of
 *     MatrixSwitch's type(matrix) (MatrixSwitch/src/MatrixSwitch_ops.F90:62-97).
 *   - Storage labels are the reference's 5-character labels
 *     [s|p][d|z][den|csc] plus a new first letter 'g' for GPU-resident storage:
 *       gdden / gzden   dense FP64 / complex FP64 in HBM, column-major
 *       gdcsc / gzcsc   CSC in HBM (0-based internally; 1-based accepted at registration)
 *     's' labels keep the data in host memory (sdden aliases the caller's array
 *     like m_register_sden); 'p' labels collapse to one process and are
 *     treated as their 's' counterparts (the BLACS descriptor is accepted, only
 *     the global sizes are used).
 *   - Operation labels ('label' / m_operation) are the reference's 3-character
 *     labels.  New labels select the GPU implementations:
 *       "gpu"   FP64 everywhere (complex FP64 for z matrices)
 *       "gmx"   mixed precision: BF16/FP32 bulk products with FP32
 *               accumulation, FP64 refinement of the final CG iterations
 *               (omm only; MatrixSwitch products treat it as "gpu").
 *     The reference labels "ref", "lap", "psp" are accepted and run the FP64
 *     GPU implementation.
 *   - Matrix element indices (i, j) are 1-based like the Fortran API.
 *   - Complex scalars are passed as double[2] = {re, im}; complex arrays are
 *     interleaved (re, im) pairs, i.e. Fortran complex(dp) / C double _Complex.
 *   - Every function returns an int status: 0 on success, OMM_NOT_CONVERGED
 *     (positive) when omm() hit its iteration caps (the reference only logs a
 *     warning then), and a negative code on error.  Errors that the reference
 *     reports through die() (file + stop 1) return a negative code and keep the
 *     message for omm_gpu_last_error(); the Fortran shim turns them back into
 *     die() so existing callers see the same behaviour.
 *   - All device work of one library instance runs on one CUDA stream
 *     (omm_gpu_set_stream); calls return after that work completed unless a
 *     function says otherwise.
 */
#ifndef OMMGPU_H
#define OMMGPU_H

#include <stdbool.h>
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct msw_matrix msw_matrix;

#define OMM_OK 0
#define OMM_NOT_CONVERGED 1
#define OMM_ERR_ARG (-1)         /* invalid argument (die() in the reference) */
#define OMM_ERR_CUDA (-2)        /* CUDA / cuBLAS / cuSOLVER failure */
#define OMM_ERR_ALLOC (-3)       /* device allocation failed */
#define OMM_ERR_NOT_SPD (-4)     /* Cholesky factor of S failed (dpotrf info != 0) */
#define OMM_ERR_STATE (-5)       /* calc_ED before a density was computed */
#define OMM_ERR_UNSUPPORTED (-6) /* combination the reference also rejects */
#define OMM_ERR_NONFINITE (-7)   /* NaN/Inf in the line-search coefficients */
#define OMM_ERR_CALLBACK (-8)    /* omm_callback's H routine returned non-zero */

/* Message of the last error of the calling thread ("" when none). */
const char* omm_gpu_last_error(void);

/* Select the CUDA device (default: the current device at first call) and the
 * stream used by all subsequent work (NULL = a stream owned by the library). */
int omm_gpu_set_device(int device);
int omm_gpu_set_stream(void* cuda_stream);
/* Number of kernels of this library launched so far in the process (library
 * kernels such as cuBLAS/cuSOLVER are not counted).  No reference counterpart. */
long long omm_gpu_kernel_launches(void);
/* Device pool counters (no reference counterpart): out[0] cudaMalloc calls made by the
 * library since start-up, out[1] their bytes, out[2] blocks given back with cudaFree,
 * out[3] bytes held for reuse now.  Work buffers released by one call are reused by the
 * next up to 48 GB; the rest is freed. */
int omm_gpu_pool_stats(long long out[4]);
/* Per-kernel timing for measurement (no reference counterpart).  While on,
 * the library records CUDA events on its stream around each launch of its
 * dominant kernels ("cgu_dmma_kernel": FP64 SpMM, work = FP64 flops;
 * "oz_gemm_pair_kernel" / "oz_gemm_kernel": the int8 GEMMs of the FP64
 * products on SM pairs / single SMs, work = int8 ops; "oz_spmm_kernel": the
 * FP64 SpMM on the int8 tensor cores, work = the FP64 flops it stands for;
 * "oz_exp_kernel", "oz_res_rows_kernel", "oz_res_kc_kernel",
 * "oz_reconstruct_kernel", "oz_axpby_exps_kernel": the passes around the int8 products, work =
 * algorithmic bytes; "spmm_tc_kernel" / "spmm_tc2_kernel": the mixed step's
 * SpMM, work = algorithmic bytes; "gemm_bf16_pair_kernel" /
 * "gemm_bf16_kernel": work = flops).  _get returns the launches, their summed
 * event time and summed work since timing was turned on (it synchronises);
 * turning it off releases the events. */
int omm_gpu_kernel_timing(int on);
int omm_gpu_kernel_timing_get(const char* kernel, long long* launches, double* total_ms, double* work);
/* Free every device buffer, the per-ip omm state, the host memory kept for reuse by
 * CSC registrations and the column-group plans kept by pattern (library stays usable). */
int omm_gpu_finalize(void);

/* ---------------------------------------------------------------- MatrixSwitch */

/* m_allocate — MatrixSwitch/src/MatrixSwitch.F90:312-419 (zero-filled). */
int msw_allocate(msw_matrix** A, int dim1, int dim2, const char label[5]);
/* m_deallocate — MatrixSwitch.F90:527-601.  *A is set to NULL. */
int msw_deallocate(msw_matrix** A);
/* m_register_sden — MatrixSwitch/src/MatrixSwitch_m_register.F90:99-133 (real)
 * and :139-173 (complex, is_complex != 0).  The handle aliases the caller's
 * column-major array; nothing is copied. */
int msw_register_sden(msw_matrix** A, int dim1, int dim2, void* host, int is_complex);
/* Device-memory counterpart of m_register_sden: the handle aliases a
 * column-major dim1 x dim2 array that already lives in this GPU's memory
 * (e.g. a torch tensor); nothing is copied and the memory stays the caller's.
 * No reference counterpart (the reference has no device memory). */
int msw_register_gden(msw_matrix** A, int dim1, int dim2, void* device_ptr, int is_complex);
/* m_register_pcsc — MatrixSwitch_m_register.F90:394-443 (real) and :451-500
 * (complex) / pspBLAS psp_register_spm (pspBLAS/src/pspVariable/pspMat.F90:87-140).
 * Copies the CSC arrays.  label is "gdcsc"/"gzcsc" (device), "sdcsc"/"szcsc"
 * (host) or "pdcsc"/"pzcsc" (collapsed to one process, stored on the device).
 * index_base is 0 or 1 and applies to both colptr and rowind. */
int msw_register_csc(msw_matrix** A, const char label[5], int dim1, int dim2, int nnz, const int* colptr,
                     const int* rowind, const void* val, int index_base);
/* m_copy — MatrixSwitch.F90:630-963 without thresholding: a new matrix in the
 * storage given by label holding the same elements (host <-> device, CSC -> dense,
 * and dense -> CSC keeping every element like m_copy_sdenscscref,
 * MatrixSwitch_m_copy.F90:495-551). */
int msw_copy(msw_matrix** dst, const msw_matrix* src, const char label[5]);
/* m_copy with threshold (MatrixSwitch.F90:630-900): entries with |a| > |threshold|
 * are kept (shifted down by |threshold| * a/|a| when threshold_is_soft), the others
 * are omitted (sparse label) or zeroed (dense label); dense -> CSC is compacted on
 * the device in column-major order (MatrixSwitch_m_copy.F90:553-629).  CSC -> CSC
 * with a threshold returns OMM_ERR_UNSUPPORTED like the reference's die()
 * ("thresholding not yet implemented", MatrixSwitch.F90:840). */
int msw_copy_thre(msw_matrix** dst, const msw_matrix* src, const char label[5], double threshold,
                  bool threshold_is_soft);
/* COO registration — psp_register_spm with 'coo' then psp_coo2csc
 * (pspBLAS/src/pspVariable/pspMat.F90:87-140, pspUtility/pspBasicTool.F90:907-942):
 * a CSC matrix from (row, column, value) triplets in any order; the reference
 * assumes column-major order and no repeats, here entries are sorted and
 * repeated (row, column) pairs are summed.  index_base 0 or 1. */
int msw_register_coo(msw_matrix** A, const char label[5], int dim1, int dim2, int nnz, const int* rowind,
                     const int* colind, const void* val, int index_base);
/* psp_den2sp / psp_sp2den — pspUtility/pspBasicTool.F90:205-533: dense -> CSC
 * keeping the nonzeros (thre == 0) or the entries with |a| >= thre (thre > 0;
 * thre < 0 is OMM_ERR_ARG), compacted on the device; CSC -> dense. */
int psp_gpu_den2sp(const msw_matrix* den, double thre, const char label[5], msw_matrix** sp);
/* The CSC arrays of a sparse matrix (the reference's iaux4 / iaux3 / dval, 0-based):
 * *nnz always; colptr (dim2+1), rowind (nnz) and val (nnz reals or 2*nnz interleaved
 * complex) when not NULL.  No reference counterpart (the Fortran type exposes them). */
int msw_csc_arrays(const msw_matrix* A, int* nnz, int* colptr, int* rowind, void* val);
int psp_gpu_sp2den(const msw_matrix* sp, const char label[5], msw_matrix** den);
/* Bulk transfers of a dense matrix between a device handle and a host array
 * (column-major, dim1 x dim2).  No reference counterpart: the reference keeps
 * data in host memory, so these are the explicit boundary of 'g' storage. */
int msw_upload(msw_matrix* A, const void* host);
int msw_download(const msw_matrix* A, void* host);
/* Raw device pointer of a dense 'g' matrix (column-major, leading dimension = dim1),
 * for zero-copy interoperation (e.g. DLPack).  NULL for other storages. */
void* msw_device_ptr(const msw_matrix* A);
int msw_dims(const msw_matrix* A, int* dim1, int* dim2, int* is_complex, int* is_csc);

/* mm_multiply — MatrixSwitch.F90:1046-1390 (real) / :1395-1726 (complex):
 * C = alpha*op(A)*op(B) + beta*C, op in {'n','t','c'}. */
int msw_mm_dmultiply(const msw_matrix* A, char opA, const msw_matrix* B, char opB, msw_matrix* C, double alpha,
                     double beta, const char label[3]);
int msw_mm_zmultiply(const msw_matrix* A, char opA, const msw_matrix* B, char opB, msw_matrix* C,
                     const double alpha[2], const double beta[2], const char label[3]);
/* m_add — MatrixSwitch.F90:1731-1902 / :1907-2055: C = alpha*op(A) + beta*C. */
int msw_m_dadd(const msw_matrix* A, char opA, msw_matrix* C, double alpha, double beta, const char label[3]);
int msw_m_zadd(const msw_matrix* A, char opA, msw_matrix* C, const double alpha[2], const double beta[2],
               const char label[3]);
/* m_trace — MatrixSwitch.F90:2060-2156 / :2161-2248 (complex result as {re, im}). */
int msw_m_dtrace(const msw_matrix* A, double* alpha, const char label[3]);
int msw_m_ztrace(const msw_matrix* A, double alpha[2], const char label[3]);
/* mm_trace — MatrixSwitch.F90:2253-2377 / :2382-2491: sum_ij conj(A_ij)*B_ij. */
int msw_mm_dtrace(const msw_matrix* A, const msw_matrix* B, double* alpha, const char label[3]);
int msw_mm_ztrace(const msw_matrix* A, const msw_matrix* B, double alpha[2], const char label[3]);
/* mm_trace that allocates nothing.  No counterpart in the reference.
 * For callers that must not let the library allocate device memory:
 * applications whose own memory manager owns the GPU (a pool reserved at
 * start-up that leaves no room for other allocators), and loops that cannot
 * afford the device synchronisation a cudaMalloc implies.  msw_mm_[dz]trace
 * keep their block partial sums in scratch the library allocates on demand;
 * this variant keeps them in a fixed 1 MiB __device__ array inside the library
 * (held by every GPU that loads it until the process exits) and touches no
 * handle, stream or allocator of the library.
 *   A, B    device pointers, column-major rows x cols with leading dimensions
 *           lda, ldb >= rows; doubles, or interleaved (re, im) pairs when
 *           is_complex != 0.
 *   result  device pointer to 2 doubles: {Re, Im} of sum_ij conj(A_ij)*B_ij
 *           (Im = 0 for real input; {0, 0} when rows*cols == 0), written by
 *           the last kernel of the call.
 *   stream  CUDA stream the two kernels are queued on (NULL = legacy default);
 *           the call does not synchronise.
 * Limit: rows*cols <= OMM_NOALLOC_MAX_ELEMS, else OMM_ERR_ARG and nothing runs.
 * All calls share the scratch array, which keeps the last call's contents;
 * each call writes every record it reads, so nothing needs clearing, but
 * calls that overlap on the same GPU (e.g. on two streams at once) race on it.
 * The first call in a CUDA context (made with that device current) looks up
 * the array's device address with cudaGetSymbolAddress; it is looked up again
 * when the device's context changes (e.g. after cudaDeviceReset).  Make that
 * first call before any stream capture.  Errors: omm_gpu_noalloc_last_error(). */
#define OMM_NOALLOC_ELEMS_PER_BLOCK 2048
#define OMM_NOALLOC_MAX_PARTIALS 65536
#define OMM_NOALLOC_MAX_ELEMS ((long long)OMM_NOALLOC_MAX_PARTIALS * OMM_NOALLOC_ELEMS_PER_BLOCK)
int omm_gpu_mm_trace_noalloc(int rows, int cols, const void* A, int lda, const void* B, int ldb, int is_complex,
                             double* result, void* stream);
const char* omm_gpu_noalloc_last_error(void);
/* m_scale — MatrixSwitch.F90:2496-2621 / :2626-2742: C = beta*C. */
int msw_m_dscale(msw_matrix* C, double beta, const char label[3]);
int msw_m_zscale(msw_matrix* C, const double beta[2], const char label[3]);
/* m_set — MatrixSwitch.F90:2747-2827 / :2832-2912: off-diagonal <- alpha,
 * diagonal <- beta, restricted to the 'u'/'l' triangle when seC says so. */
int msw_m_dset(msw_matrix* C, char seC, double alpha, double beta, const char label[3]);
int msw_m_zset(msw_matrix* C, char seC, const double alpha[2], const double beta[2], const char label[3]);
/* m_set_element — MatrixSwitch.F90:2917-3086 / :3091-3260: C(i,j) = alpha + beta*C(i,j), 1-based. */
int msw_m_dset_element(msw_matrix* C, int i, int j, double alpha, double beta, const char label[3]);
int msw_m_zset_element(msw_matrix* C, int i, int j, const double alpha[2], const double beta[2],
                       const char label[3]);
/* m_get_element — MatrixSwitch.F90:3309-3417 / :3422-3530, 1-based. */
int msw_m_dget_element(const msw_matrix* C, int i, int j, double* alpha, const char label[3]);
int msw_m_zget_element(const msw_matrix* C, int i, int j, double alpha[2], const char label[3]);

/* ---------------------------------------------- MatrixSwitch wrapper (string keys)
 * The reference's key-based layer for callers that name matrices by string
 * instead of holding handles (MatrixSwitch/src/MatrixSwitch_wrapper.F90,
 * MatrixSwitch_wrapper_params.F90).  Keys are NUL-terminated C strings, stored
 * cut to 10 characters with trailing blanks insignificant (Fortran semantics,
 * MatrixSwitch_wrapper_params.F90:19); an unknown key is OMM_ERR_ARG
 * ("ms_lookup: key not found", :47-71).  A slot that holds no matrix is the
 * reference's uninitialised type(matrix).  Optional Fortran arguments are
 * pointers (NULL = absent); labels as above (NULL label in ms_m_allocate =
 * "sdden", MatrixSwitch.F90:344-347). */
/* ms_wrapper_open — MatrixSwitch_wrapper.F90:219-236 (replaces any open table). */
int ms_wrapper_open(int num_matrices, const char* const* keys);
/* ms_wrapper_close — MatrixSwitch_wrapper.F90:244-261: deallocates every slot. */
int ms_wrapper_close(void);
/* The handle bound to key (NULL when its slot holds no matrix): ms_lookup +
 * ms_matrices, MatrixSwitch_wrapper_params.F90:47-71. */
int ms_lookup(const char* key, msw_matrix** A);
/* ms_is_initialized / _serial / _real / _square / _sparse, ms_dim1 / ms_dim2 —
 * MatrixSwitch_wrapper.F90:269-394. */
int ms_is_initialized(const char* key, bool* out);
int ms_is_serial(const char* key, bool* out);
int ms_is_real(const char* key, bool* out);
int ms_is_square(const char* key, bool* out);
int ms_is_sparse(const char* key, bool* out);
int ms_dim1(const char* key, int* out);
int ms_dim2(const char* key, int* out);
/* m_allocate / m_deallocate / m_copy / m_convert — MatrixSwitch_wrapper.F90:399-475. */
int ms_m_allocate(const char* key, int i, int j, const char label[5]);
int ms_m_deallocate(const char* key);
int ms_m_copy(const char* key, const char* A, const char label[5], const double* threshold,
              const bool* threshold_is_soft);
int ms_m_convert(const char* key, const char label[5], const double* threshold, const bool* threshold_is_soft);
/* mm_multiply, m_add, m_trace, mm_trace, m_scale, m_set, m_set_element,
 * m_get_element by key — MatrixSwitch_wrapper.F90:480-849. */
int ms_mm_dmultiply(const char* A, char opA, const char* B, char opB, const char* C, double alpha, double beta,
                    const char label[3]);
int ms_mm_zmultiply(const char* A, char opA, const char* B, char opB, const char* C, const double alpha[2],
                    const double beta[2], const char label[3]);
int ms_m_dadd(const char* A, char opA, const char* C, double alpha, double beta, const char label[3]);
int ms_m_zadd(const char* A, char opA, const char* C, const double alpha[2], const double beta[2],
              const char label[3]);
int ms_m_dtrace(const char* A, double* alpha, const char label[3]);
int ms_m_ztrace(const char* A, double alpha[2], const char label[3]);
int ms_mm_dtrace(const char* A, const char* B, double* alpha, const char label[3]);
int ms_mm_ztrace(const char* A, const char* B, double alpha[2], const char label[3]);
int ms_m_dscale(const char* C, double beta, const char label[3]);
int ms_m_zscale(const char* C, const double beta[2], const char label[3]);
int ms_m_dset(const char* C, char seC, double alpha, double beta, const char label[3]);
int ms_m_zset(const char* C, char seC, const double alpha[2], const double beta[2], const char label[3]);
int ms_m_dset_element(const char* C, int i, int j, double alpha, double beta, const char label[3]);
int ms_m_zset_element(const char* C, int i, int j, const double alpha[2], const double beta[2],
                      const char label[3]);
int ms_m_dget_element(const char* C, int i, int j, double* alpha, const char label[3]);
int ms_m_zget_element(const char* C, int i, int j, double alpha[2], const char label[3]);
/* m_register_sdden / m_register_szden — MatrixSwitch_wrapper.F90:855-887: the
 * slot aliases the caller's column-major dim1 x dim2 array. */
int ms_m_register_sdden(const char* key, int dim1, int dim2, double* A);
int ms_m_register_szden(const char* key, int dim1, int dim2, void* A);
/* m_register_pddbc / m_register_pzdbc — MatrixSwitch_wrapper.F90:894-932,
 * one process: A is the whole desc[2] x desc[3] matrix (aliased). */
int ms_m_register_pddbc(const char* key, double* A, const int desc[9]);
int ms_m_register_pzdbc(const char* key, void* A, const int desc[9]);
/* m_register_pdcsc / m_register_pzcsc — MatrixSwitch_wrapper.F90:1090-1132:
 * idx1 = 1-based row index per nonzero, idx2 = desc[3] + 1 one-based column
 * pointers (psp_register_spm, pspMat.F90:87-136); copied. */
int ms_m_register_pdcsc(const char* key, const int* idx1, const int* idx2, const double* val, const int desc[9]);
int ms_m_register_pzcsc(const char* key, const int* idx1, const int* idx2, const void* val, const int desc[9]);
/* m_register_pdcoo / m_register_pzcoo — MatrixSwitch_wrapper.F90:1039-1082:
 * nnz 1-based (row idx1, column idx2, value) triplets, stored as CSC. */
int ms_m_register_pdcoo(const char* key, int nnz, const int* idx1, const int* idx2, const double* val,
                        const int desc[9]);
int ms_m_register_pzcoo(const char* key, int nnz, const int* idx1, const int* idx2, const void* val,
                        const int desc[9]);
/* m_copy_external_pdbcpcsc — MatrixSwitch_wrapper.F90:989-1030: CSC of the
 * entries of the dense array with |a| > |threshold| (every entry when NULL). */
int ms_m_copy_external_pddbcpdcsc(const char* key, const double* A, const int desc[9], const double* threshold);
int ms_m_copy_external_pzdbcpzcsc(const char* key, const void* A, const int desc[9], const double* threshold);

/* -------------------------------------------------------------------- pspBLAS */

/* psp_gemspm — pspBLAS/src/pspLevel3/pspMspm.F90:58-120 (real), :123-183 (complex):
 * C = alpha*op(A)*op(B) + beta*C with A dense (M x K after op), B CSC.
 * As in the reference, alpha == 0 only scales C by beta, and leaves C
 * untouched when beta == 0 as well. */
int psp_gpu_dgemspm(int M, int N, int K, const msw_matrix* A, char opA, const msw_matrix* B, char opB,
                    msw_matrix* C, double alpha, double beta);
int psp_gpu_zgemspm(int M, int N, int K, const msw_matrix* A, char opA, const msw_matrix* B, char opB,
                    msw_matrix* C, const double alpha[2], const double beta[2]);
/* psp_gespmm — pspBLAS/src/pspLevel3/pspSpmm.F90:61-123 (real), :128-190 (complex):
 * C = alpha*op(A)*op(B) + beta*C with A CSC, B dense; same alpha == 0 rule. */
int psp_gpu_dgespmm(int M, int N, int K, const msw_matrix* A, char opA, const msw_matrix* B, char opB,
                    msw_matrix* C, double alpha, double beta);
int psp_gpu_zgespmm(int M, int N, int K, const msw_matrix* A, char opA, const msw_matrix* B, char opB,
                    msw_matrix* C, const double alpha[2], const double beta[2]);

/* ---------------------------------------------------------------------- libOMM */

/* omm — libOMM/src/omm.F90:5-51 (argument meaning and order kept).
 * S == NULL (or an unallocated handle) means "no S" like an uninitialized
 * type(matrix); T may be NULL.  H, S, D_min, C_min may use any storage label
 * above; host storages are staged to the device for the call and the outputs
 * (C_min, D_min, and H/S when the Cholesky flavour modifies them) are written
 * back.  m_storage is the label of the internal work matrices ('g' labels;
 * 's'/'p' labels are mapped to their 'g' counterpart) and m_operation one of
 * the operation labels above.  The per-ip state (the reference's SAVEd
 * matrices) stays on the device until a call with dealloc = true.
 * Returns OMM_OK, OMM_NOT_CONVERGED (the reference only logs a warning then)
 * or a negative error code. */
int omm_gpu(int m, int n, msw_matrix* H, msw_matrix* S, bool new_S, double* e_min, msw_matrix* D_min, bool calc_ED,
            double eta, msw_matrix* C_min, bool init_C, msw_matrix* T, double scale_T, int flavour, int np, int ip,
            double cg_tol, bool long_out, bool dealloc, const char m_storage[5], const char m_operation[3]);

/* omm_wrapper — libOMM/src/omm_wrapper.F90:5-96 as built with -DCBIND (the
 * logicals are C bool): omm with its five matrices named by keys of the
 * MatrixSwitch wrapper's table; a key whose slot holds no matrix passes an
 * absent S or T, as in the reference.  Same status codes as omm_gpu. */
int omm_wrapper(int m, int n, const char* H, const char* S, bool new_S, double* e_min, const char* D_min,
                bool calc_ED, double eta, const char* C_min, bool init_C, const char* T, double scale_T, int flavour,
                int np, int ip, double cg_tol, bool long_out, bool dealloc, const char m_storage[5],
                const char m_operation[3]);

/* omm_callback — libOMM/src/omm_callback.F90:5-673: the same minimisation with H
 * supplied as a routine instead of a matrix: H(C, HC) must set HC = C * H for
 * the n x m coefficient matrix C (omm_ops.F90:69-99 calc_HW_callback).  The
 * library calls it with 'g' dense matrices aliasing its device buffers (do not
 * deallocate them), after its stream is idle; HC must be complete when the
 * routine returns, or its work enqueued on the library stream (every msw_* /
 * psp_* call made from inside does that).  A non-zero return aborts the solve
 * with OMM_ERR_CALLBACK.  As in the reference only flavours 0 and 3 are legal
 * (others give OMM_ERR_ARG), and the per-ip state is separate from omm's.  The
 * "gmx" label runs FP64 here (the products of H are the caller's). */
typedef int (*omm_gpu_H_fn)(const msw_matrix* C, msw_matrix* HC, void* user);
int omm_gpu_callback(int m, int n, omm_gpu_H_fn H, void* user, msw_matrix* S, bool new_S, double* e_min,
                     msw_matrix* D_min, bool calc_ED, double eta, msw_matrix* C_min, bool init_C, msw_matrix* T,
                     double scale_T, int flavour, int np, int ip, double cg_tol, bool long_out, bool dealloc,
                     const char m_storage[5], const char m_operation[3]);

/* Statistics of the last omm_gpu call (no reference counterpart). */
typedef struct {
    int icg;               /* CG steps taken (the reference's icg) */
    int icg_low;           /* of which in the reduced-precision stage ("gmx") */
    int icg_fp64;          /* of which in the FP64-refined stages */
    int ls_fail;           /* line-search failures (coefficient rescalings) */
    int converged;         /* 1 if e_diff <= cg_tol was reached */
    double e_min;          /* returned energy */
    double e_diff;         /* last relative energy change */
    double trqs;           /* Tr[(2I - SW) SW] */
    double seconds;        /* wall time of the call (host clock) */
    double t_setup;        /* of which: allocation, staging, initial products */
    double t_loop;         /* CG iterations */
    double t_final;        /* density matrix and write-back */
    double t_loop_sync;    /* part of t_loop the host spent waiting for the GPU */
} omm_gpu_stats;
int omm_gpu_get_stats(omm_gpu_stats* st);

/* Logging: the reference writes libOMM.log in the working directory
 * (omm.F90:118-123, replace on the first call, append after).  Pass NULL to
 * disable the file, or a path to redirect it.  Default: "libOMM.log". */
int omm_gpu_set_log(const char* path);

/* Stage tolerances of the "gmx" solver (no reference counterpart).  It runs CG
 * steps with BF16 products until the relative energy change falls below
 * bf16_tol (default 1e-5), then with split-BF16 (hi/lo) products until it falls
 * below split_tol (default 1e-8), then recomputes HC, SC, HW, SW and the
 * gradient from C in FP64 and refines (FP64 gradient and line-search slope,
 * split-BF16 curvature terms) until e_diff <= refine_factor * cg_tol
 * (default 0.1, in (0, 1]).  A stage also ends early when its energy stops
 * decreasing or a line search fails; a refinement that does not converge in
 * 8 steps hands over to FP64 products with the reference's test
 * e_diff <= cg_tol (omm.F90:506). */
int omm_gpu_set_mixed(double bf16_tol, double split_tol, double refine_factor);

/* ------------------------------------------------------- tensor-core kernels */

/* BF16 tensor-core GEMM (tcgen05 + TMA) used by the "gmx" solver, exposed for
 * testing and reuse; no reference counterpart.
 *   out (FP64, M x N, column-major, ldo) = alpha * sum_seg A_seg * B_seg^T + beta * out
 * A_hi/A_lo (M x K) and B_hi/B_lo (N x K) are device bf16 arrays, K-major
 * (row stride lda/ldb elements, multiples of 8, 16-byte aligned).
 * nseg = 1: A_hi B_hi^T.  nseg = 3: A_hi B_hi^T + A_hi B_lo^T + A_lo B_hi^T
 * (hi/lo bf16 splits of higher-precision operands).  Synchronous. */
int omm_gpu_gemm_bf16(int M, int N, int K, const void* A_hi, const void* A_lo, int lda, const void* B_hi,
                      const void* B_lo, int ldb, int nseg, double alpha, double beta, double* out, int ldo);
/* The same product enqueued on the library stream without waiting for it (for
 * timing); its pipeline errors are read with omm_gpu_tc_errors. */
int omm_gpu_gemm_bf16_async(int M, int N, int K, const void* A_hi, const void* A_lo, int lda, const void* B_hi,
                            const void* B_lo, int ldb, int nseg, double alpha, double beta, double* out, int ldo);

/* The reduced-precision form of psp_gemspm's product used by the "gmx" solver,
 * exposed for testing and measurement; no reference counterpart.
 *   C = A * B, A and C dense FP64 'g' matrices, B a real CSC matrix; with B2
 *   and C2 (both NULL or both given) also C2 = A * B2, in the same pass over A
 *   when B and B2 share one pattern (the solver's [HC; SC] = C [H, S]).
 * nseg = 1: bf16 operands with FP32 accumulation; nseg = 3: hi/lo bf16 split
 * products (~2^-16 relative).  *path (may be NULL) reports the kernel used:
 * 2 = tcgen05 tensor cores (B is a union of 8-row aligned blocks per column
 * group), 1 = FP32 CUDA cores, 0 = FP64 gather.  Synchronous. */
int omm_gpu_spmm_lowp(const msw_matrix* A, const msw_matrix* B, msw_matrix* C, const msw_matrix* B2, msw_matrix* C2,
                      int nseg, int* path);
/* The two halves of omm_gpu_spmm_lowp's tensor-core path, for timing the
 * kernel alone (no reference counterpart).  _prepare converts A to the
 * library's bf16 operand buffer (one per process; asynchronous on the library
 * stream); _apply runs the tcgen05 SpMM on it (asynchronous, no host sync;
 * OMM_ERR_UNSUPPORTED when B, B2 cannot take the tensor-core path or differ
 * in pattern).  A later _prepare replaces the operand; calls that overlap on
 * the GPU race on it.  omm_gpu_tc_errors synchronises the stream and returns
 * (and clears) the error bits of timed-out pipeline waits (0 = none). */
int omm_gpu_spmm_lowp_prepare(const msw_matrix* A, int nseg);
/* The column-group plan the SpMM kernels use for a CSC matrix (built on first
 * use): group width G (8, 16, 24 or 32 columns), number of groups, fill (nonzeros
 * / cells of the dense union blocks) and whether the column-group kernels take it
 * (1) or the generic gather kernel does (0).  No reference counterpart. */
int omm_gpu_spmm_plan_info(const msw_matrix* B, int* G, int* ngroups, double* fill, int* column_groups);
int omm_gpu_spmm_lowp_apply(const msw_matrix* B, msw_matrix* C, const msw_matrix* B2, msw_matrix* C2, int nseg);
/* The mixed solver's per-step form of the same product (no reference counterpart):
 * Y = A * B in FP32 (column-major, leading dimension ldy), with B2's product n rows
 * below (ldy >= 2n) when B2 is given (same pattern as B); with t_hi (and t_lo for
 * nseg = 3) also the row-major bf16 hi/lo parts of Y (rows of B's product, then
 * B2's; row stride ldt, a multiple of 8).  A is the operand of the last _prepare;
 * asynchronous.  omm_gpu_set_spmm_groups picks the kernel, for this call and for
 * the mixed CG step: 1 (default) = one column group per CTA, 4 = CTAs of four
 * neighbouring column groups that fetch every plane of A in the union of their
 * rows once (fewer bytes from L2, one CTA per SM). */
int omm_gpu_set_spmm_groups(int groups_per_cta);
int omm_gpu_spmm_lowp_apply_f32(const msw_matrix* B, const msw_matrix* B2, float* Y, int ldy, void* t_hi, void* t_lo,
                                int ldt, int nseg);
int omm_gpu_tc_errors(unsigned* bits);
/* Limit of every pipeline wait of the tensor-core kernels (default 2e9 ns = 2 s)
 * and a test switch: with withhold_copies != 0 their copy producers issue
 * nothing, so each CTA's first wait runs out after wait_ns, its TMEM is freed
 * and the call reports OMM_ERR_CUDA with the error bits (omm_gpu_tc_errors;
 * GEMM: 4 = operand wait, 8 = accumulator wait; SpMM: 64, 128).  Used by the
 * tests of the timed-out-wait path; no copy is in flight while it runs.
 * wait_ns == 0 is OMM_ERR_ARG.  No reference counterpart. */
int omm_gpu_tc_set_wait(unsigned long long wait_ns, int withhold_copies);
/* Whether the tensor-core GEMMs (the bf16 GEMM and the int8 GEMMs of the FP64
 * products) form 256 x 256 tiles on pairs of SMs (clusters of two CTAs,
 * tcgen05 cta_group::2) where the shape allows: on != 0 (default), or 128 x 256
 * tiles on single SMs.  The FP64 products are identical either way (their
 * int8 products are exact); bf16 products agree to the FP32 accumulation's
 * rounding.  No reference counterpart. */
int omm_gpu_tc_set_pairs(int on);

/* FP64 GEMM on the int8 tensor cores, as the solver's FP64 products use it; no
 * reference counterpart (the reference calls BLAS dgemm, e.g. omm_ops.F90:62,
 * MatrixSwitch.F90:1303).  C = alpha*op(A)*op(B) + beta*C, op 'n' or 't',
 * device FP64 column-major arrays.  Each row of op(A) and column of op(B) is
 * scaled by a power of two and rounded to a 53-bit integer; their exact
 * integer product is formed modulo 16 coprime moduli <= 256 by int8 tcgen05
 * GEMMs and rebuilt by the Chinese remainder theorem, then rounded once to
 * FP64 (the accuracy of an FP64 GEMM relative to the rows' and columns'
 * largest entries).  K < 2^17.  NaN/Inf in a row or column give NaN in the
 * row or column of C.  Synchronous. */
int omm_gpu_gemm_f64(char opA, char opB, int M, int N, int K, double alpha, const double* A, int lda, const double* B,
                     int ldb, double beta, double* C, int ldc);
/* The same product enqueued on the library stream without waiting (for timing);
 * its pipeline errors are read with omm_gpu_tc_errors. */
int omm_gpu_gemm_f64_async(char opA, char opB, int M, int N, int K, double alpha, const double* A, int lda,
                           const double* B, int ldb, double beta, double* C, int ldc);
/* FP64 SpMM on the int8 tensor cores, as the FP64 CG step forms [HG; SG] = D [H, S]
 * (psp_gemspm's local product, pspBLAS/src/pspLevel3/pspMspm_nn.F90:191-198, with
 * both matrices at once): Y(0:n-1, :) = A H and, when S is given (same pattern as H),
 * Y(n:2n-1, :) = A S.  A (n x m) and Y (ldy >= n, or 2n with S) are device FP64
 * column-major arrays; H and S real CSC of order m < 2^17 whose columns form groups
 * of at most 32 (atom-block matrices), n a multiple of 4.  Rows of A and columns of
 * H and S are rounded to 53 bits relative to their largest entry and multiplied
 * exactly (16 moduli, as omm_gpu_gemm_f64).  OMM_ERR_UNSUPPORTED when the matrices
 * do not fit.  Synchronous.  No reference counterpart. */
int omm_gpu_spmm_f64(const double* A, int lda, int n, const msw_matrix* H, const msw_matrix* S, double* Y, int ldy);
/* Form of that int8 SpMM kernel (and of the FP64 CG step's): 0 = one column group per CTA,
 * four pipeline stages of one chunk pair; 1 (default) = one group per CTA, two stages of three
 * chunk pairs, chunks adjacent in memory fetched as one copy of up to 24 KB; 2 = two
 * consecutive column groups per CTA walking the union of their rows once, with two-pair
 * stages; 3 = the groups of form 2 on SM pairs (clusters of two CTAs, each holding 128 of
 * the 256 rows; products without S take form 1).  All give the same bits.  OMM_ERR_ARG
 * otherwise.  No reference counterpart. */
int omm_gpu_set_oz_spmm_form(int form);
/* Which engine the real FP64 products of omm()/MatrixSwitch use: mode 1 = the
 * int8 tensor-core GEMM above (default), 0 = cuBLAS DGEMM.  panel_bytes caps
 * the scratch of one int8 product's residues (0 = default 4 GiB; larger
 * products run in column panels).  No reference counterpart. */
int omm_gpu_set_fp64_gemm(int mode, long long panel_bytes);

/* ------------------------------------------------------- gradients / adjoint */

/* Functional gradient dOmega/dC = G = 4 HC - 2 SW HC - 2 HW SC of the Kim
 * functional Omega(C) = tr[(2I - S_W) H_W] at the given C (calc_G,
 * libOMM/src/omm_ops.F90:17-39).  Writes G (n x m, same storage kind as C)
 * and Omega.  S may be NULL (S = I). */
int omm_gpu_functional_grad(int m, int n, const msw_matrix* H, const msw_matrix* S, const msw_matrix* C,
                            msw_matrix* G, double* omega);
/* Adjoint of the converged energy with respect to Hamiltonian parameters,
 * H(theta) = H0 + sum_k theta_k V_k:  dE/dtheta_k = Re sum_ij conj(D_ij) (V_k)_ij
 * with D = C^H (2I - S_W) C, evaluated as tr[(2I - S_W) C V_k C^H] without
 * forming the m x m density.  C is the converged C_min; V are nv sparse (CSC)
 * or dense matrices.  grad has nv entries.  No reference counterpart (the
 * reference has no derivatives). */
int omm_gpu_energy_adjoint(int m, int n, const msw_matrix* S, const msw_matrix* C, int nv, const msw_matrix* const* V,
                           double* grad);

/* tomato_TB — tomato/src/tomato_TB.F90:1-636: the tight-binding H (and S, when the
 * template has an overlap) of a periodic supercell, replicated from the element list of
 * <template_basedir>/<system_label>_<cutoff>_<size>.template.  Same arguments, in/out
 * meaning and selection rules as the reference: switch1 picks the basis size by frac_occ
 * (else by num_orbs_per_atom), switch2 the supercell by num_orbs (else num_cells_dir),
 * switch3 the orbital cutoff by sparsity (else orb_r_cut); all of them, num_occ_states and
 * the k point (zeroed in non-periodic directions) are written back.  With build_matrix
 * false only those scalars are returned (sparsity estimated from the element count) and
 * *H, *S are set to NULL.  Otherwise *H and *S are new matrices in m_storage ("sdden",
 * "sdcsc", "pdcsc", "gdden", ...; real for gamma_point, complex otherwise), *S is NULL
 * without an overlap, and sparsity is the reference's sampled estimate (num_orbs elements
 * drawn with the omm LCG from the NORAND seed 123456).  Values are the reference's sums in
 * its own order: bit-identical at the Gamma point; k-point phases come from the device
 * sincos.  The replication and the summation run on the GPU. */
int tomato_gpu_TB(const char* template_basedir, const char* system_label, bool switch1, double* frac_occ,
                  int* num_orbs_per_atom, bool switch2, int* num_orbs, int num_cells_dir[3], bool switch3,
                  double* sparsity, double* orb_r_cut, int* num_occ_states, bool gamma_point, double k_point[3],
                  bool defect, double defect_perturbation, msw_matrix** H, msw_matrix** S, const char m_storage[5],
                  bool build_matrix);

#ifdef __cplusplus
}
#endif

#endif /* OMMGPU_H */
