// The reference's string-key boundary, for callers that name matrices by key instead of
// holding handles: MatrixSwitch's wrapper layer (a table of matrices, each bound to a key of
// at most 10 characters: MatrixSwitch/src/MatrixSwitch_wrapper.F90,
// MatrixSwitch_wrapper_params.F90) and libOMM's omm_wrapper (libOMM/src/omm_wrapper.F90),
// which resolves its five matrix keys in that table and calls omm.  These are the entry
// points a C caller of the reference binds when it is built with -DCBIND (logicals as C bool).
//
// Key semantics follow Fortran character assignment and comparison: keys are stored cut to
// 10 characters, and trailing blanks are not significant.  A key whose slot holds no
// matrix is the reference's uninitialised type(matrix): omm_wrapper passes it to omm as an
// absent S or T.  Every slot's matrix is a handle of the C ABI (ms_lookup returns it), so the
// two interfaces can be mixed.  Host code only: the work is done by the handle API.
#include "internal.h"

#include <cstring>
#include <mutex>
#include <string>
#include <vector>

namespace ommgpu {
namespace {

constexpr size_t kMaxKeyLength = 10;  // MatrixSwitch_wrapper_params.F90:19

struct Slot {
    std::string key;
    msw_matrix* m = nullptr;
};
std::vector<Slot> g_slots;
bool g_open = false;
std::recursive_mutex g_mu;

std::string norm_key(const char* k, size_t cap) {
    if (!k) fail(OMM_ERR_ARG, "ms_lookup: null key");
    std::string s(k, strnlen(k, 4096));
    if (s.size() > cap) s.resize(cap);
    while (!s.empty() && s.back() == ' ') s.pop_back();
    return s;
}

// ms_lookup (MatrixSwitch_wrapper_params.F90:47-71): the slot bound to key, or die
Slot& slot(const char* key) {
    if (!g_open) fail(OMM_ERR_STATE, "ms_lookup: the wrapper is not open (ms_wrapper_open)");
    std::string k = norm_key(key, 4096);
    for (Slot& s : g_slots)
        if (s.key == k) return s;
    fail(OMM_ERR_ARG, "ms_lookup: key not found");
}

msw_matrix* need(const char* key) {
    Slot& s = slot(key);
    if (!s.m) fail(OMM_ERR_ARG, std::string("matrix '") + key + "' is not allocated");
    return s.m;
}

void check(int rc) {
    if (rc < 0) throw Error{rc, omm_gpu_last_error()};
}

// replace the slot's matrix by a newly made one
void rebind(Slot& s, msw_matrix* m) {
    if (s.m) msw_deallocate(&s.m);
    s.m = m;
}

template <typename F>
int guarded(F&& f) {
    std::lock_guard<std::recursive_mutex> lock(g_mu);
    try {
        f();
    } catch (const Error& e) {
        set_last_error(e.msg);
        return e.code;
    }
    set_last_error("");
    return OMM_OK;
}

// the global sizes of a one-process BLACS descriptor (desc(3), desc(4))
void desc_dims(const int* desc, int& d1, int& d2) {
    if (!desc) fail(OMM_ERR_ARG, "m_register: null descriptor");
    d1 = desc[2];
    d2 = desc[3];
    if (d1 < 0 || d2 < 0) fail(OMM_ERR_ARG, "m_register: negative global size in the descriptor");
}

}  // namespace
}  // namespace ommgpu

using namespace ommgpu;

extern "C" {

// ms_wrapper_open — MatrixSwitch_wrapper.F90:219-236
int ms_wrapper_open(int num_matrices, const char* const* keys) {
    return guarded([&] {
        if (num_matrices < 0 || (num_matrices > 0 && !keys)) fail(OMM_ERR_ARG, "ms_wrapper_open: bad arguments");
        for (Slot& s : g_slots) rebind(s, nullptr);
        g_slots.assign(num_matrices, Slot{});
        for (int i = 0; i < num_matrices; ++i) g_slots[i].key = norm_key(keys[i], kMaxKeyLength);
        g_open = true;
    });
}

// ms_wrapper_close — MatrixSwitch_wrapper.F90:244-261
int ms_wrapper_close(void) {
    return guarded([&] {
        for (Slot& s : g_slots) rebind(s, nullptr);
        g_slots.clear();
        g_open = false;
    });
}

int ms_lookup(const char* key, msw_matrix** A) {
    return guarded([&] {
        if (!A) fail(OMM_ERR_ARG, "ms_lookup: null result");
        *A = slot(key).m;
    });
}

// ms_is_initialized / ms_is_serial / ms_is_real / ms_is_square / ms_is_sparse / ms_dim1 /
// ms_dim2 — MatrixSwitch_wrapper.F90:269-394
int ms_is_initialized(const char* key, bool* out) {
    return guarded([&] { *out = slot(key).m != nullptr; });
}
int ms_is_serial(const char* key, bool* out) {
    return guarded([&] { *out = need(key)->label[0] == 's'; });
}
int ms_is_real(const char* key, bool* out) {
    return guarded([&] { *out = need(key)->is_real; });
}
int ms_is_square(const char* key, bool* out) {
    return guarded([&] {
        const msw_matrix* m = need(key);
        *out = m->dim1 == m->dim2;
    });
}
int ms_is_sparse(const char* key, bool* out) {
    return guarded([&] { *out = !need(key)->dense(); });
}
int ms_dim1(const char* key, int* out) {
    return guarded([&] { *out = need(key)->dim1; });
}
int ms_dim2(const char* key, int* out) {
    return guarded([&] { *out = need(key)->dim2; });
}

// m_allocate / m_deallocate / m_copy / m_convert — MatrixSwitch_wrapper.F90:399-475
int ms_m_allocate(const char* key, int i, int j, const char label[5]) {
    return guarded([&] {
        Slot& s = slot(key);
        msw_matrix* m = nullptr;
        check(msw_allocate(&m, i, j, label ? label : "sdden"));  // default label: MatrixSwitch.F90:344-347
        rebind(s, m);
    });
}
int ms_m_deallocate(const char* key) {
    return guarded([&] { rebind(slot(key), nullptr); });
}
int ms_m_copy(const char* key, const char* A, const char label[5], const double* threshold,
              const bool* threshold_is_soft) {
    return guarded([&] {
        const msw_matrix* src = need(A);
        Slot& s = slot(key);
        msw_matrix* m = nullptr;
        const char* lab = label ? label : src->label;
        if (threshold) check(msw_copy_thre(&m, src, lab, *threshold, threshold_is_soft ? *threshold_is_soft : false));
        else check(msw_copy(&m, src, lab));
        rebind(s, m);
    });
}
int ms_m_convert(const char* key, const char label[5], const double* threshold, const bool* threshold_is_soft) {
    return guarded([&] {
        Slot& s = slot(key);
        if (!s.m) fail(OMM_ERR_ARG, "m_convert: matrix not allocated");
        msw_matrix* m = nullptr;
        const char* lab = label ? label : s.m->label;
        if (threshold) check(msw_copy_thre(&m, s.m, lab, *threshold, threshold_is_soft ? *threshold_is_soft : false));
        else check(msw_copy(&m, s.m, lab));
        rebind(s, m);
    });
}

// mm_multiply, m_add, m_trace, mm_trace, m_scale, m_set, m_set_element, m_get_element by key —
// MatrixSwitch_wrapper.F90:480-849
int ms_mm_dmultiply(const char* A, char opA, const char* B, char opB, const char* C, double alpha, double beta,
                    const char label[3]) {
    return guarded([&] { check(msw_mm_dmultiply(need(A), opA, need(B), opB, need(C), alpha, beta, label)); });
}
int ms_mm_zmultiply(const char* A, char opA, const char* B, char opB, const char* C, const double alpha[2],
                    const double beta[2], const char label[3]) {
    return guarded([&] { check(msw_mm_zmultiply(need(A), opA, need(B), opB, need(C), alpha, beta, label)); });
}
int ms_m_dadd(const char* A, char opA, const char* C, double alpha, double beta, const char label[3]) {
    return guarded([&] { check(msw_m_dadd(need(A), opA, need(C), alpha, beta, label)); });
}
int ms_m_zadd(const char* A, char opA, const char* C, const double alpha[2], const double beta[2],
              const char label[3]) {
    return guarded([&] { check(msw_m_zadd(need(A), opA, need(C), alpha, beta, label)); });
}
int ms_m_dtrace(const char* A, double* alpha, const char label[3]) {
    return guarded([&] { check(msw_m_dtrace(need(A), alpha, label)); });
}
int ms_m_ztrace(const char* A, double alpha[2], const char label[3]) {
    return guarded([&] { check(msw_m_ztrace(need(A), alpha, label)); });
}
int ms_mm_dtrace(const char* A, const char* B, double* alpha, const char label[3]) {
    return guarded([&] { check(msw_mm_dtrace(need(A), need(B), alpha, label)); });
}
int ms_mm_ztrace(const char* A, const char* B, double alpha[2], const char label[3]) {
    return guarded([&] { check(msw_mm_ztrace(need(A), need(B), alpha, label)); });
}
int ms_m_dscale(const char* C, double beta, const char label[3]) {
    return guarded([&] { check(msw_m_dscale(need(C), beta, label)); });
}
int ms_m_zscale(const char* C, const double beta[2], const char label[3]) {
    return guarded([&] { check(msw_m_zscale(need(C), beta, label)); });
}
int ms_m_dset(const char* C, char seC, double alpha, double beta, const char label[3]) {
    return guarded([&] { check(msw_m_dset(need(C), seC, alpha, beta, label)); });
}
int ms_m_zset(const char* C, char seC, const double alpha[2], const double beta[2], const char label[3]) {
    return guarded([&] { check(msw_m_zset(need(C), seC, alpha, beta, label)); });
}
int ms_m_dset_element(const char* C, int i, int j, double alpha, double beta, const char label[3]) {
    return guarded([&] { check(msw_m_dset_element(need(C), i, j, alpha, beta, label)); });
}
int ms_m_zset_element(const char* C, int i, int j, const double alpha[2], const double beta[2],
                      const char label[3]) {
    return guarded([&] { check(msw_m_zset_element(need(C), i, j, alpha, beta, label)); });
}
int ms_m_dget_element(const char* C, int i, int j, double* alpha, const char label[3]) {
    return guarded([&] { check(msw_m_dget_element(need(C), i, j, alpha, label)); });
}
int ms_m_zget_element(const char* C, int i, int j, double alpha[2], const char label[3]) {
    return guarded([&] { check(msw_m_zget_element(need(C), i, j, alpha, label)); });
}

// m_register_sdden / m_register_szden — MatrixSwitch_wrapper.F90:855-887: the slot's matrix
// aliases the caller's column-major array (MatrixSwitch_m_register.F90:129)
int ms_m_register_sdden(const char* key, int dim1, int dim2, double* A) {
    return guarded([&] {
        Slot& s = slot(key);
        msw_matrix* m = nullptr;
        check(msw_register_sden(&m, dim1, dim2, A, 0));
        rebind(s, m);
    });
}
int ms_m_register_szden(const char* key, int dim1, int dim2, void* A) {
    return guarded([&] {
        Slot& s = slot(key);
        msw_matrix* m = nullptr;
        check(msw_register_sden(&m, dim1, dim2, A, 1));
        rebind(s, m);
    });
}
// m_register_pddbc / m_register_pzdbc — MatrixSwitch_wrapper.F90:894-932, collapsed to one
// process: the local array is the whole desc(3) x desc(4) matrix
int ms_m_register_pddbc(const char* key, double* A, const int desc[9]) {
    return guarded([&] {
        int d1, d2;
        desc_dims(desc, d1, d2);
        Slot& s = slot(key);
        msw_matrix* m = nullptr;
        check(msw_register_sden(&m, d1, d2, A, 0));
        rebind(s, m);
    });
}
int ms_m_register_pzdbc(const char* key, void* A, const int desc[9]) {
    return guarded([&] {
        int d1, d2;
        desc_dims(desc, d1, d2);
        Slot& s = slot(key);
        msw_matrix* m = nullptr;
        check(msw_register_sden(&m, d1, d2, A, 1));
        rebind(s, m);
    });
}
// m_register_pdcsc / m_register_pzcsc — MatrixSwitch_wrapper.F90:1090-1132 (MatrixSwitch_m_register
// .F90:394-500 through psp_register_spm, pspMat.F90:87-136): idx1 holds the 1-based row index of
// each nonzero, idx2 the desc(4) + 1 one-based column pointers; nnz = idx2[desc(4)] - 1
int ms_m_register_pdcsc(const char* key, const int* idx1, const int* idx2, const double* val, const int desc[9]) {
    return guarded([&] {
        int d1, d2;
        desc_dims(desc, d1, d2);
        if (!idx2) fail(OMM_ERR_ARG, "m_register_pcsc: null column pointers");
        Slot& s = slot(key);
        msw_matrix* m = nullptr;
        check(msw_register_csc(&m, "pdcsc", d1, d2, idx2[d2] - 1, idx2, idx1, val, 1));
        rebind(s, m);
    });
}
int ms_m_register_pzcsc(const char* key, const int* idx1, const int* idx2, const void* val, const int desc[9]) {
    return guarded([&] {
        int d1, d2;
        desc_dims(desc, d1, d2);
        if (!idx2) fail(OMM_ERR_ARG, "m_register_pcsc: null column pointers");
        Slot& s = slot(key);
        msw_matrix* m = nullptr;
        check(msw_register_csc(&m, "pzcsc", d1, d2, idx2[d2] - 1, idx2, idx1, val, 1));
        rebind(s, m);
    });
}
// m_register_pdcoo / m_register_pzcoo — MatrixSwitch_wrapper.F90:1039-1082: nnz 1-based
// (row, column, value) triplets, kept as CSC (repeats summed)
int ms_m_register_pdcoo(const char* key, int nnz, const int* idx1, const int* idx2, const double* val,
                        const int desc[9]) {
    return guarded([&] {
        int d1, d2;
        desc_dims(desc, d1, d2);
        Slot& s = slot(key);
        msw_matrix* m = nullptr;
        check(msw_register_coo(&m, "pdcsc", d1, d2, nnz, idx1, idx2, val, 1));
        rebind(s, m);
    });
}
int ms_m_register_pzcoo(const char* key, int nnz, const int* idx1, const int* idx2, const void* val,
                        const int desc[9]) {
    return guarded([&] {
        int d1, d2;
        desc_dims(desc, d1, d2);
        Slot& s = slot(key);
        msw_matrix* m = nullptr;
        check(msw_register_coo(&m, "pzcsc", d1, d2, nnz, idx1, idx2, val, 1));
        rebind(s, m);
    });
}
// m_copy_external_pdbcpcsc — MatrixSwitch_wrapper.F90:989-1030: a CSC matrix of the entries of
// the (one-process) dense array whose magnitude exceeds |threshold| (all entries when NULL)
int ms_m_copy_external_pddbcpdcsc(const char* key, const double* A, const int desc[9], const double* threshold) {
    return guarded([&] {
        int d1, d2;
        desc_dims(desc, d1, d2);
        Slot& s = slot(key);
        msw_matrix* dense = nullptr;
        check(msw_register_sden(&dense, d1, d2, const_cast<double*>(A), 0));
        msw_matrix* m = nullptr;
        int rc = threshold ? msw_copy_thre(&m, dense, "pdcsc", *threshold, false) : msw_copy(&m, dense, "pdcsc");
        msw_deallocate(&dense);
        check(rc);
        rebind(s, m);
    });
}
int ms_m_copy_external_pzdbcpzcsc(const char* key, const void* A, const int desc[9], const double* threshold) {
    return guarded([&] {
        int d1, d2;
        desc_dims(desc, d1, d2);
        Slot& s = slot(key);
        msw_matrix* dense = nullptr;
        check(msw_register_sden(&dense, d1, d2, const_cast<void*>(A), 1));
        msw_matrix* m = nullptr;
        int rc = threshold ? msw_copy_thre(&m, dense, "pzcsc", *threshold, false) : msw_copy(&m, dense, "pzcsc");
        msw_deallocate(&dense);
        check(rc);
        rebind(s, m);
    });
}

// omm_wrapper — libOMM/src/omm_wrapper.F90:5-96 (CBIND: the logicals are C bool): the five
// matrix keys are resolved in the wrapper's table and omm runs on them; a key whose slot holds
// no matrix is an uninitialised S or T (absent), as in the reference
int omm_wrapper(int m, int n, const char* H, const char* S, bool new_S, double* e_min, const char* D_min,
                bool calc_ED, double eta, const char* C_min, bool init_C, const char* T, double scale_T, int flavour,
                int np, int ip, double cg_tol, bool long_out, bool dealloc, const char m_storage[5],
                const char m_operation[3]) {
    msw_matrix *h = nullptr, *s = nullptr, *d = nullptr, *c = nullptr, *t = nullptr;
    int rc = guarded([&] {
        h = need(H);
        s = slot(S).m;
        d = need(D_min);
        c = need(C_min);
        t = slot(T).m;
    });
    if (rc != OMM_OK) return rc;
    // the solve runs outside the table's lock (its status and message are omm's own)
    return omm_gpu(m, n, h, s, new_S, e_min, d, calc_ED, eta, c, init_C, t, scale_T, flavour, np, ip, cg_tol,
                   long_out, dealloc, m_storage, m_operation);
}

}  // extern "C"
