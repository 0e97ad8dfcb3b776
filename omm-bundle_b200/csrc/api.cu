// Runtime, matrix handles, and the MatrixSwitch / pspBLAS entry points of the C ABI.
//
// MatrixSwitch's per-operation dispatch tables (MatrixSwitch.F90:1096-1351 and
// siblings) choose an implementation from (storage format, serial, label).
// Here every storage is served by the GPU: dense products go to cuBLAS
// (FP64/complex FP64), dense x CSC and CSC x dense products to the SpMM kernels
// of spmm.cu, and elementwise/trace operations to kernels.cu.  Host ('s')
// matrices are staged to the device for the duration of one call.
#include "internal.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <atomic>
#include <chrono>
#include <map>
#include <mutex>

namespace ommgpu {

static thread_local std::string g_last_error;
static std::atomic<long long> g_launches{0};
long long count_launch() { return ++g_launches; }

// ---- per-kernel timing: events recorded around selected launches while enabled
namespace {
struct KTimes {
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev;
    std::vector<double> work;
};
bool g_ktime = false;
std::map<std::string, KTimes> g_ktimes;
cudaEvent_t g_kstart = nullptr;
cudaEvent_t new_event() {
    cudaEvent_t e = nullptr;
    OMM_CK(cudaEventCreate(&e));
    return e;
}
}  // namespace
bool ktime_on() { return g_ktime; }
void ktime_begin() {
    if (!g_ktime) return;
    g_kstart = new_event();
    OMM_CK(cudaEventRecord(g_kstart, rt().stream));
}
void ktime_end(const char* name, double work) {
    if (!g_ktime || !g_kstart) return;
    cudaEvent_t stop = new_event();
    OMM_CK(cudaEventRecord(stop, rt().stream));
    KTimes& k = g_ktimes[name];
    k.ev.push_back({g_kstart, stop});
    k.work.push_back(work);
    g_kstart = nullptr;
}
void set_last_error(const std::string& m) { g_last_error = m; }
[[noreturn]] void fail(int code, const std::string& msg) { throw Error{code, msg}; }

// ------------------------------------------------------------------ DevBuf
// Device buffers come from a size-keyed cache of earlier allocations: omm() is
// called once per SCF step with the same sizes, and fresh cudaMalloc/cudaFree
// of ~10 GB of work matrices per call cost more than the solve at large m.
// All work is ordered on the library's one stream, so a block released while
// kernels still read it is only written again by work queued after them.
// omm_gpu_finalize() returns the cached blocks to the driver.
namespace {
struct Pool {
    std::mutex mu;
    std::multimap<size_t, void*> blocks;
    size_t cached = 0;
    long long mallocs = 0;      // cudaMalloc calls made by the pool since start-up
    long long malloc_bytes = 0;
    long long frees = 0;        // blocks given back to the driver (cap reached, trim)
};
Pool& pool() {
    static Pool* p = new Pool();  // never destroyed: outlives static DevBufs at exit
    return *p;
}
// Bytes kept for reuse at most (the rest is freed).  A solve whose work buffers exceed the
// cap reallocates the excess on every call (omm_gpu_pool_stats counts the cudaMalloc calls).
// A caller that needs the memory for its own tensors between solves calls omm_gpu_finalize().
constexpr size_t kPoolCap = size_t(48) << 30;
size_t pool_round(size_t b) {
    if (b < (size_t(1) << 20)) return (b + 255) & ~size_t(255);
    return (b + (size_t(2) << 20) - 1) & ~((size_t(2) << 20) - 1);
}
}  // namespace

void pool_trim() {
    Pool& P = pool();
    std::lock_guard<std::mutex> lk(P.mu);
    for (auto& kv : P.blocks) cudaFree(kv.second);
    P.frees += (long long)P.blocks.size();
    P.blocks.clear();
    P.cached = 0;
}

void DevBuf::alloc(size_t b) {
    release();
    owns = true;
    if (b == 0) b = 16;
    b = pool_round(b);
    {
        Pool& P = pool();
        std::lock_guard<std::mutex> lk(P.mu);
        auto it = P.blocks.lower_bound(b);
        if (it != P.blocks.end() && it->first <= b + b / 8) {
            p = it->second;
            bytes = it->first;
            P.cached -= bytes;
            P.blocks.erase(it);
            return;
        }
    }
    cudaError_t e = cudaMalloc(&p, b);
    if (e != cudaSuccess) {
        (void)cudaGetLastError();
        pool_trim();  // give cached blocks back and retry once
        e = cudaMalloc(&p, b);
    }
    if (e == cudaSuccess) {
        Pool& P = pool();
        std::lock_guard<std::mutex> lk(P.mu);
        P.mallocs += 1;
        P.malloc_bytes += (long long)b;
    }
    if (e != cudaSuccess) {
        p = nullptr;
        (void)cudaGetLastError();
        fail(OMM_ERR_ALLOC, "cudaMalloc of " + std::to_string(b) + " bytes failed: " + cudaGetErrorString(e));
    }
    bytes = b;
}
void DevBuf::alloc_zero(size_t b) {
    alloc(b);
    OMM_CK(cudaMemsetAsync(p, 0, bytes, rt().stream));
}
void DevBuf::ensure(size_t b) {
    if (bytes >= b && p) return;
    if (p) OMM_CK(cudaStreamSynchronize(rt().stream));
    alloc(b);
}
void DevBuf::release() {
    if (p && owns) {
        Pool& P = pool();
        std::lock_guard<std::mutex> lk(P.mu);
        if (P.cached + bytes <= kPoolCap) {
            P.blocks.emplace(bytes, p);
            P.cached += bytes;
        } else {
            cudaFree(p);
            P.frees += 1;
        }
    }
    owns = true;
    p = nullptr;
    bytes = 0;
}

// ------------------------------------------------------------------ runtime
static Runtime* g_rt = nullptr;
static std::mutex g_rt_mu;

Runtime& rt() {
    if (g_rt && g_rt->device >= 0) return *g_rt;
    std::lock_guard<std::mutex> lk(g_rt_mu);
    if (!g_rt) g_rt = new Runtime();
    if (g_rt->device < 0) {
        int dev = 0;
        OMM_CK(cudaGetDevice(&dev));
        OMM_CK(cudaSetDevice(dev));
        g_rt->device = dev;
        OMM_CK(cudaStreamCreateWithFlags(&g_rt->stream, cudaStreamNonBlocking));
        g_rt->own_stream = true;
        OMM_CKB(cublasCreate(&g_rt->blas));
        OMM_CKB(cublasSetStream(g_rt->blas, g_rt->stream));
        OMM_CKS(cusolverDnCreate(&g_rt->solver));
        OMM_CKS(cusolverDnSetStream(g_rt->solver, g_rt->stream));
        OMM_CK(cudaMallocHost((void**)&g_rt->host_pinned, 64 * sizeof(double)));
    }
    return *g_rt;
}
bool runtime_bound() {
    std::lock_guard<std::mutex> lk(g_rt_mu);
    return g_rt && g_rt->device >= 0;
}
static double g_sync_wait = 0.0;
double sync_wait_seconds() { return g_sync_wait; }
void sync() {
    auto t0 = std::chrono::steady_clock::now();
    OMM_CK(cudaStreamSynchronize(rt().stream));
    g_sync_wait += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

// ------------------------------------------------------------------ labels
Label parse_storage(const char* label) {
    if (!label) fail(OMM_ERR_ARG, "m_allocate_elements: invalid label");
    Label L{};
    char c1 = label[0], c2 = label[1];
    std::string f(label + 2, label + 5);
    if (c1 != 's' && c1 != 'p' && c1 != 'g') fail(OMM_ERR_ARG, "m_allocate_elements: invalid label");
    if (c2 != 'd' && c2 != 'z') fail(OMM_ERR_ARG, "m_allocate_elements: invalid label");
    L.where = c1;
    L.real = (c2 == 'd');
    if (f == "den" || f == "dbc") L.fmt = Fmt::Dense;
    else if (f == "csc") L.fmt = Fmt::CSC;
    else fail(OMM_ERR_UNSUPPORTED, std::string("storage format '") + f + "' is not provided by the GPU library");
    return L;
}

OpKind parse_op(const char* label) {
    if (!label) return OpKind::FP64;
    std::string s(label, label + 3);
    if (s == "gmx") return OpKind::Mixed;
    if (s == "gpu" || s == "ref" || s == "lap" || s == "psp" || s == "t1D") return OpKind::FP64;
    fail(OMM_ERR_ARG, "invalid implementation label '" + s + "'");
}

// ------------------------------------------------------------------ staging
void stage_in(const msw_matrix* A, Staged& s, bool copy_data) {
    if (!A->dense()) fail(OMM_ERR_UNSUPPORTED, "dense operand expected");
    s.src = A;
    s.v.rows = A->dim1;
    s.v.cols = A->dim2;
    s.v.ld = std::max(1, A->dim1);
    s.v.is_real = A->is_real;
    if (A->loc == Loc::Device) {
        s.v.p = A->dev.p;
        return;
    }
    s.tmp.alloc(A->elems() * A->esize());
    s.v.p = s.tmp.p;
    if (copy_data && A->elems())
        OMM_CK(cudaMemcpyAsync(s.tmp.p, A->host, A->elems() * A->esize(), cudaMemcpyHostToDevice, rt().stream));
}
void stage_out(msw_matrix* A, const Staged& s) {
    if (A->loc == Loc::Device || A->elems() == 0) return;
    OMM_CK(cudaMemcpyAsync(A->host, s.v.p, A->elems() * A->esize(), cudaMemcpyDeviceToHost, rt().stream));
    OMM_CK(cudaStreamSynchronize(rt().stream));
}

void ensure_csc_device(const msw_matrix* A) {
    msw_matrix* M = const_cast<msw_matrix*>(A);
    if (M->d_colptr.p) return;
    M->d_colptr.alloc((M->dim2 + 1) * sizeof(int));
    M->d_rowind.alloc(std::max(1, M->nnz) * sizeof(int));
    M->d_val.alloc(std::max<size_t>(1, (size_t)M->nnz) * M->esize());
    OMM_CK(cudaMemcpyAsync(M->d_colptr.p, M->h_colptr.data(), (M->dim2 + 1) * sizeof(int), cudaMemcpyHostToDevice,
                           rt().stream));
    if (M->nnz) {
        OMM_CK(cudaMemcpyAsync(M->d_rowind.p, M->h_rowind.data(), M->nnz * sizeof(int), cudaMemcpyHostToDevice,
                               rt().stream));
        OMM_CK(cudaMemcpyAsync(M->d_val.p, M->h_val.data(), M->nnz * M->esize(), cudaMemcpyHostToDevice, rt().stream));
    }
    OMM_CK(cudaStreamSynchronize(rt().stream));
}

static void invalidate_csc(msw_matrix* M) {
    M->d_colptr.release();
    M->d_rowind.release();
    M->d_val.release();
    M->plan.reset();
    M->tc_plan.reset();
    M->tc2_plan.reset();
    M->tc2_plan_split.reset();
    M->oz_plan.reset();
    M->transposed.reset();
    M->conj_transposed.reset();
    M->pattern_id = next_pattern_id();
}

const msw_matrix* csc_transpose(const msw_matrix* A) {
    msw_matrix* M = const_cast<msw_matrix*>(A);
    if (M->transposed) return M->transposed.get();
    auto T = std::make_shared<msw_matrix>();
    T->dim1 = A->dim2;
    T->dim2 = A->dim1;
    T->is_real = A->is_real;
    T->fmt = Fmt::CSC;
    T->loc = Loc::Device;
    T->nnz = A->nnz;
    T->h_colptr.assign(T->dim2 + 1, 0);
    for (int l = 0; l < A->nnz; ++l) T->h_colptr[A->h_rowind[l] + 1]++;
    for (int j = 0; j < T->dim2; ++j) T->h_colptr[j + 1] += T->h_colptr[j];
    std::vector<int> pos(T->h_colptr.begin(), T->h_colptr.end() - 1);
    T->h_rowind.assign(A->nnz, 0);
    int w = A->is_real ? 1 : 2;
    T->h_val.assign((size_t)A->nnz * w, 0.0);
    for (int c = 0; c < A->dim2; ++c)
        for (int l = A->h_colptr[c]; l < A->h_colptr[c + 1]; ++l) {
            int r = A->h_rowind[l];
            int d = pos[r]++;
            T->h_rowind[d] = c;
            for (int q = 0; q < w; ++q) T->h_val[(size_t)d * w + q] = A->h_val[(size_t)l * w + q];
        }
    M->transposed = T;
    return T.get();
}

// CSC -> dense scatter (for m_add with a CSC source and msw_copy)
template <typename T>
__global__ void csc_scatter_kernel(int ncol, const int* colptr, const int* rowind, const T* val, T* C, int ldc) {
    int j = blockIdx.x;
    if (j >= ncol) return;
    for (int l = colptr[j] + threadIdx.x; l < colptr[j + 1]; l += blockDim.x) C[rowind[l] + (size_t)j * ldc] = val[l];
}
static void csc_to_dense(const msw_matrix* A, DView& out) {
    ensure_csc_device(A);
    OMM_CK(cudaMemsetAsync(out.p, 0, (size_t)out.ld * out.cols * A->esize(), rt().stream));
    if (A->dim2 == 0) return;
    if (A->is_real)
        csc_scatter_kernel<double><<<A->dim2, 128, 0, rt().stream>>>(A->dim2, A->d_colptr.as<int>(),
                                                                      A->d_rowind.as<int>(), A->d_val.as<double>(),
                                                                      out.as<double>(), out.ld);
    else
        csc_scatter_kernel<zdbl><<<A->dim2, 128, 0, rt().stream>>>(A->dim2, A->d_colptr.as<int>(),
                                                                    A->d_rowind.as<int>(), A->d_val.as<zdbl>(),
                                                                    out.as<zdbl>(), out.ld);
    OMM_KCHECK();
}

void csc_to_dense_view(const msw_matrix* A, DView& out) { csc_to_dense(A, out); }

static bool is_tr(char op) {
    if (op == 'n' || op == 'N') return false;
    if (op == 't' || op == 'T' || op == 'c' || op == 'C') return true;
    fail(OMM_ERR_ARG, "process_opM: invalid opM");
}

}  // namespace ommgpu

using namespace ommgpu;

// ==================================================================== C ABI
#define API_BEGIN try {
#define API_END                                         \
    }                                                   \
    catch (const ommgpu::Error& e) {                    \
        set_last_error(e.msg);                          \
        return e.code;                                  \
    }                                                   \
    catch (const std::bad_alloc&) {                     \
        set_last_error("host allocation failed");       \
        return OMM_ERR_ALLOC;                           \
    }                                                   \
    catch (const std::exception& e) {                   \
        set_last_error(e.what());                       \
        return OMM_ERR_ARG;                             \
    }                                                   \
    set_last_error("");                                 \
    return OMM_OK;

extern "C" {

const char* omm_gpu_last_error(void) { return g_last_error.c_str(); }

long long omm_gpu_kernel_launches(void) { return g_launches.load(); }
int omm_gpu_pool_stats(long long* out) {
    if (!out) return OMM_ERR_ARG;
    Pool& P = pool();
    std::lock_guard<std::mutex> lk(P.mu);
    out[0] = P.mallocs;
    out[1] = P.malloc_bytes;
    out[2] = P.frees;
    out[3] = (long long)P.cached;
    return OMM_OK;
}

int omm_gpu_kernel_timing(int on) {
    API_BEGIN
    if (!on && g_ktime) {
        sync();
        for (auto& kv : g_ktimes)
            for (auto& pr : kv.second.ev) {
                cudaEventDestroy(pr.first);
                cudaEventDestroy(pr.second);
            }
        g_ktimes.clear();
    }
    g_ktime = on != 0;
    API_END
}

int omm_gpu_kernel_timing_get(const char* kernel, long long* launches, double* total_ms, double* work) {
    API_BEGIN
    if (!kernel || !launches || !total_ms || !work) fail(OMM_ERR_ARG, "kernel_timing_get: null argument");
    *launches = 0;
    *total_ms = 0.0;
    *work = 0.0;
    auto it = g_ktimes.find(kernel);
    if (it != g_ktimes.end()) {
        sync();
        for (size_t i = 0; i < it->second.ev.size(); ++i) {
            float ms = 0.f;
            OMM_CK(cudaEventElapsedTime(&ms, it->second.ev[i].first, it->second.ev[i].second));
            *total_ms += ms;
            *work += it->second.work[i];
        }
        *launches = (long long)it->second.ev.size();
    }
    API_END
}

int omm_gpu_set_device(int device) {
    API_BEGIN
    if (g_rt && g_rt->device >= 0 && g_rt->device != device)
        fail(OMM_ERR_ARG, "omm_gpu_set_device: the library is already bound to device " +
                              std::to_string(g_rt->device) + "; call omm_gpu_finalize first");
    OMM_CK(cudaSetDevice(device));
    rt();
    API_END
}

int omm_gpu_set_stream(void* s) {
    API_BEGIN
    Runtime& r = rt();
    OMM_CK(cudaStreamSynchronize(r.stream));
    if (r.own_stream) OMM_CK(cudaStreamDestroy(r.stream));
    if (s) {
        r.stream = (cudaStream_t)s;
        r.own_stream = false;
    } else {
        OMM_CK(cudaStreamCreateWithFlags(&r.stream, cudaStreamNonBlocking));
        r.own_stream = true;
    }
    OMM_CKB(cublasSetStream(r.blas, r.stream));
    OMM_CKS(cusolverDnSetStream(r.solver, r.stream));
    API_END
}

int msw_allocate(msw_matrix** A, int dim1, int dim2, const char label[5]) {
    API_BEGIN
    if (!A) fail(OMM_ERR_ARG, "m_allocate: null handle");
    if (dim1 < 0 || dim2 < 0) fail(OMM_ERR_ARG, "m_allocate: negative dimension");
    Label L = parse_storage(label);
    auto* M = new msw_matrix();
    M->dim1 = dim1;
    M->dim2 = dim2;
    M->is_real = L.real;
    M->fmt = L.fmt;
    memcpy(M->label, label, 5);
    M->label[5] = 0;
    M->loc = (L.where == 's') ? Loc::Host : Loc::Device;
    if (L.fmt == Fmt::Dense) {
        if (M->loc == Loc::Host) {
            M->host_store.assign(M->elems() * (L.real ? 1 : 2), 0.0);
            M->host = M->host_store.data();
        } else {
            M->dev.alloc_zero(std::max<size_t>(1, M->elems()) * M->esize());
        }
    } else {
        // empty sparse matrix (MatrixSwitch.F90:409-412: iaux2(1)=0)
        M->h_colptr.assign(dim2 + 1, 0);
    }
    *A = M;
    API_END
}

int msw_deallocate(msw_matrix** A) {
    API_BEGIN
    if (A && *A) {
        if ((*A)->loc == Loc::Device && (*A)->dev.p) OMM_CK(cudaStreamSynchronize(rt().stream));
        delete *A;
        *A = nullptr;
    }
    API_END
}

int msw_register_sden(msw_matrix** A, int dim1, int dim2, void* host, int is_complex) {
    API_BEGIN
    if (!A || (!host && dim1 * dim2 > 0)) fail(OMM_ERR_ARG, "m_register_sden: null argument");
    auto* M = new msw_matrix();
    M->dim1 = dim1;
    M->dim2 = dim2;
    M->is_real = !is_complex;
    M->fmt = Fmt::Dense;
    M->loc = Loc::Host;
    memcpy(M->label, is_complex ? "szden" : "sdden", 6);
    M->host = host;
    *A = M;
    API_END
}

int msw_register_gden(msw_matrix** A, int dim1, int dim2, void* device_ptr, int is_complex) {
    API_BEGIN
    if (!A || (!device_ptr && dim1 * dim2 > 0)) fail(OMM_ERR_ARG, "msw_register_gden: null argument");
    auto* M = new msw_matrix();
    M->dim1 = dim1;
    M->dim2 = dim2;
    M->is_real = !is_complex;
    M->fmt = Fmt::Dense;
    M->loc = Loc::Device;
    memcpy(M->label, is_complex ? "gzden" : "gdden", 6);
    M->dev.p = device_ptr;
    M->dev.bytes = M->elems() * M->esize();
    M->dev.owns = false;
    *A = M;
    API_END
}

int msw_register_csc(msw_matrix** A, const char label[5], int dim1, int dim2, int nnz, const int* colptr,
                     const int* rowind, const void* val, int index_base) {
    API_BEGIN
    if (!A || !colptr || (nnz > 0 && (!rowind || !val))) fail(OMM_ERR_ARG, "m_register_csc: null argument");
    Label L = parse_storage(label);
    if (L.fmt != Fmt::CSC) fail(OMM_ERR_ARG, "m_register_csc: label must be a csc storage");
    if (index_base != 0 && index_base != 1) fail(OMM_ERR_ARG, "m_register_csc: index_base must be 0 or 1");
    auto M = std::make_unique<msw_matrix>();
    M->dim1 = dim1;
    M->dim2 = dim2;
    M->is_real = L.real;
    M->fmt = Fmt::CSC;
    M->loc = (L.where == 's') ? Loc::Host : Loc::Device;
    memcpy(M->label, label, 5);
    M->label[5] = 0;
    M->nnz = nnz;
    M->h_colptr.assign(colptr, colptr + dim2 + 1);
    for (auto& v : M->h_colptr) v -= index_base;
    if (M->h_colptr[0] != 0 || M->h_colptr[dim2] != nnz)
        fail(OMM_ERR_ARG, "m_register_csc: column pointers do not span nnz");
    for (int j = 0; j < dim2; ++j)
        if (M->h_colptr[j + 1] < M->h_colptr[j]) fail(OMM_ERR_ARG, "m_register_csc: column pointers decrease");
    // the copies (m_register_pcsc copies, MatrixSwitch_m_register.F90:394-443) run on host threads
    const int w = L.real ? 1 : 2;
    M->h_rowind.resize(nnz);
    M->h_val.resize((size_t)nnz * w);
    std::atomic<int> bad{0};
    int* ri = M->h_rowind.data();
    host_parallel(nnz, [&](long long b, long long e) {
        int out = 0;
        for (long long k = b; k < e; ++k) {
            const int v = rowind[k] - index_base;
            out |= (v < 0 || v >= dim1);
            ri[k] = v;
        }
        if (out) bad = 1;
    });
    if (bad) fail(OMM_ERR_ARG, "m_register_csc: row index out of range");
    const double* vs = (const double*)val;
    double* vd = M->h_val.data();
    host_parallel((long long)nnz * w, [&](long long b, long long e) {
        std::memcpy(vd + b, vs + b, (size_t)(e - b) * sizeof(double));
    });
    *A = M.release();
    API_END
}

int msw_copy(msw_matrix** dst, const msw_matrix* src, const char label[5]) {
    API_BEGIN
    if (!dst || !src) fail(OMM_ERR_ARG, "m_copy: null argument");
    Label L = parse_storage(label);
    if (L.real != src->is_real) fail(OMM_ERR_ARG, "m_copy: real/complex mismatch");
    auto M = std::make_unique<msw_matrix>();
    M->dim1 = src->dim1;
    M->dim2 = src->dim2;
    M->is_real = src->is_real;
    M->fmt = L.fmt;
    M->loc = (L.where == 's') ? Loc::Host : Loc::Device;
    memcpy(M->label, label, 5);
    M->label[5] = 0;
    if (L.fmt == Fmt::CSC) {
        if (src->fmt != Fmt::CSC) {
            // m_copy_sdenscscref (MatrixSwitch_m_copy.F90:495-551): every element, column by column
            Staged s;
            stage_in(src, s, true);
            dense_to_csc(s.v, 0, 0.0, 0.0, M.get());
        } else {
            M->nnz = src->nnz;
            M->h_colptr = src->h_colptr;
            M->h_rowind = src->h_rowind;
            M->h_val = src->h_val;
        }
    } else {
        size_t bytes = M->elems() * M->esize();
        DView out{nullptr, M->dim1, M->dim2, std::max(1, M->dim1), M->is_real};
        DevBuf tmp;
        if (M->loc == Loc::Device) {
            M->dev.alloc_zero(std::max<size_t>(1, bytes));
            out.p = M->dev.p;
        } else {
            M->host_store.assign(M->elems() * (M->is_real ? 1 : 2), 0.0);
            M->host = M->host_store.data();
            tmp.alloc(std::max<size_t>(1, bytes));
            out.p = tmp.p;
        }
        if (src->fmt == Fmt::CSC) {
            csc_to_dense(src, out);
        } else if (src->loc == Loc::Device) {
            if (bytes) OMM_CK(cudaMemcpyAsync(out.p, src->dev.p, bytes, cudaMemcpyDeviceToDevice, rt().stream));
        } else {
            if (bytes) OMM_CK(cudaMemcpyAsync(out.p, src->host, bytes, cudaMemcpyHostToDevice, rt().stream));
        }
        if (M->loc == Loc::Host && bytes)
            OMM_CK(cudaMemcpyAsync(M->host, out.p, bytes, cudaMemcpyDeviceToHost, rt().stream));
        sync();
    }
    *dst = M.release();
    API_END
}

int msw_upload(msw_matrix* A, const void* host) {
    API_BEGIN
    if (!A || !host || !A->dense()) fail(OMM_ERR_ARG, "msw_upload: dense matrix and host array required");
    size_t bytes = A->elems() * A->esize();
    if (A->loc == Loc::Device) {
        if (bytes) OMM_CK(cudaMemcpyAsync(A->dev.p, host, bytes, cudaMemcpyHostToDevice, rt().stream));
        sync();
    } else if (bytes) {
        memcpy(A->host, host, bytes);
    }
    API_END
}

int msw_download(const msw_matrix* A, void* host) {
    API_BEGIN
    if (!A || !host || !A->dense()) fail(OMM_ERR_ARG, "msw_download: dense matrix and host array required");
    size_t bytes = A->elems() * A->esize();
    if (A->loc == Loc::Device) {
        if (bytes) OMM_CK(cudaMemcpyAsync(host, A->dev.p, bytes, cudaMemcpyDeviceToHost, rt().stream));
        sync();
    } else if (bytes) {
        memcpy(host, A->host, bytes);
    }
    API_END
}

void* msw_device_ptr(const msw_matrix* A) {
    if (!A || !A->dense() || A->loc != Loc::Device) return nullptr;
    return A->dev.p;
}

int msw_dims(const msw_matrix* A, int* d1, int* d2, int* is_complex, int* is_csc) {
    API_BEGIN
    if (!A) fail(OMM_ERR_ARG, "msw_dims: null handle");
    if (d1) *d1 = A->dim1;
    if (d2) *d2 = A->dim2;
    if (is_complex) *is_complex = A->is_real ? 0 : 1;
    if (is_csc) *is_csc = A->fmt == Fmt::CSC ? 1 : 0;
    API_END
}

// ------------------------------------------------------------------ mm_multiply
static void mm_multiply_impl(const msw_matrix* A, char opA, const msw_matrix* B, char opB, msw_matrix* C,
                             const double al[2], const double be[2], const char* label) {
    if (!A || !B || !C) fail(OMM_ERR_ARG, "mm_multiply: null matrix");
    parse_op(label);
    bool trA = is_tr(opA), trB = is_tr(opB);
    if (A->is_real != C->is_real || B->is_real != C->is_real)
        fail(OMM_ERR_ARG, "mm_multiply: matrices A, B and C must all be real or all complex");
    int Ar = trA ? A->dim2 : A->dim1, Ac = trA ? A->dim1 : A->dim2;
    int Br = trB ? B->dim2 : B->dim1, Bc = trB ? B->dim1 : B->dim2;
    if (Ar != C->dim1 || Bc != C->dim2 || Ac != Br)
        fail(OMM_ERR_ARG, "mm_multiply: matrices A, B and C are not compatible");
    if (!C->dense()) fail(OMM_ERR_UNSUPPORTED, "mm_multiply: sparse output is not provided by the GPU library");
    Staged sc;
    stage_in(C, sc, true);
    if (A->dense() && B->dense()) {
        Staged sa, sb;
        stage_in(A, sa);
        stage_in(B, sb);
        gemm(opA, opB, C->dim1, C->dim2, Ac, al, sa.v, sb.v, be, sc.v);
    } else if (A->dense() && !B->dense()) {
        Staged sa;
        stage_in(A, sa);
        gemspm(opA, sa.v, opB, B, sc.v, al, be);
    } else if (!A->dense() && B->dense()) {
        Staged sb;
        stage_in(B, sb);
        gespmm(opA, A, opB, sb.v, sc.v, al, be);
    } else {
        fail(OMM_ERR_UNSUPPORTED, "mm_multiply: sparse x sparse products are not provided by the GPU library");
    }
    stage_out(C, sc);
    sync();
}

int msw_mm_dmultiply(const msw_matrix* A, char opA, const msw_matrix* B, char opB, msw_matrix* C, double alpha,
                     double beta, const char label[3]) {
    API_BEGIN
    double al[2] = {alpha, 0.0}, be[2] = {beta, 0.0};  // CONV: real scalars promote for complex matrices
    mm_multiply_impl(A, opA, B, opB, C, al, be, label);
    API_END
}
int msw_mm_zmultiply(const msw_matrix* A, char opA, const msw_matrix* B, char opB, msw_matrix* C,
                     const double alpha[2], const double beta[2], const char label[3]) {
    API_BEGIN
    if (C && C->is_real) fail(OMM_ERR_ARG, "mm_zmultiply: matrix C is real");
    mm_multiply_impl(A, opA, B, opB, C, alpha, beta, label);
    API_END
}

// ------------------------------------------------------------------ m_add
static void m_add_impl(const msw_matrix* A, char opA, msw_matrix* C, const double al[2], const double be[2],
                       const char* label) {
    if (!A || !C) fail(OMM_ERR_ARG, "m_add: null matrix");
    parse_op(label);
    bool trA = is_tr(opA);
    if (A->is_real != C->is_real) fail(OMM_ERR_ARG, "m_add: real/complex mismatch");
    if (!trA ? (A->dim1 != C->dim1 || A->dim2 != C->dim2) : (A->dim1 != C->dim2 || A->dim2 != C->dim1))
        fail(OMM_ERR_ARG, "m_add: matrices A and C are not compatible");
    if (!C->dense()) fail(OMM_ERR_UNSUPPORTED, "m_add: sparse destination is not provided by the GPU library");
    Staged sc;
    stage_in(C, sc, true);
    if (A->dense()) {
        Staged sa;
        stage_in(A, sa);
        k_axpby(sa.v, opA, sc.v, al, be);
    } else {
        DevBuf tmp;
        DView d{nullptr, A->dim1, A->dim2, std::max(1, A->dim1), A->is_real};
        tmp.alloc(std::max<size_t>(1, A->elems()) * A->esize());
        d.p = tmp.p;
        csc_to_dense(A, d);
        k_axpby(d, opA, sc.v, al, be);
        sync();
    }
    stage_out(C, sc);
    sync();
}
int msw_m_dadd(const msw_matrix* A, char opA, msw_matrix* C, double alpha, double beta, const char label[3]) {
    API_BEGIN
    double al[2] = {alpha, 0.0}, be[2] = {beta, 0.0};
    m_add_impl(A, opA, C, al, be, label);
    API_END
}
int msw_m_zadd(const msw_matrix* A, char opA, msw_matrix* C, const double alpha[2], const double beta[2],
               const char label[3]) {
    API_BEGIN
    m_add_impl(A, opA, C, alpha, beta, label);
    API_END
}

// ------------------------------------------------------------------ traces
static void m_trace_impl(const msw_matrix* A, double out[2], const char* label) {
    if (!A) fail(OMM_ERR_ARG, "m_trace: null matrix");
    parse_op(label);
    if (A->dim1 != A->dim2) fail(OMM_ERR_ARG, "m_trace: matrix A is not square");
    if (A->dense()) {
        Staged s;
        stage_in(A, s);
        r_trace(s.v, out);
    } else {
        out[0] = out[1] = 0.0;
        int w = A->is_real ? 1 : 2;
        for (int j = 0; j < A->dim2; ++j)
            for (int l = A->h_colptr[j]; l < A->h_colptr[j + 1]; ++l)
                if (A->h_rowind[l] == j) {
                    out[0] += A->h_val[(size_t)l * w];
                    if (w == 2) out[1] += A->h_val[(size_t)l * w + 1];
                }
    }
}
int msw_m_dtrace(const msw_matrix* A, double* alpha, const char label[3]) {
    API_BEGIN
    double o[2];
    m_trace_impl(A, o, label);
    *alpha = o[0];  // CONV: real part of a complex trace
    API_END
}
int msw_m_ztrace(const msw_matrix* A, double alpha[2], const char label[3]) {
    API_BEGIN
    m_trace_impl(A, alpha, label);
    API_END
}
static void mm_trace_impl(const msw_matrix* A, const msw_matrix* B, double out[2], const char* label) {
    if (!A || !B) fail(OMM_ERR_ARG, "mm_trace: null matrix");
    parse_op(label);
    if (A->dim1 != B->dim1 || A->dim2 != B->dim2) fail(OMM_ERR_ARG, "mm_trace: matrices A and B are not compatible");
    if (A->is_real != B->is_real) fail(OMM_ERR_ARG, "mm_trace: real/complex mismatch");
    if (!A->dense() || !B->dense()) fail(OMM_ERR_UNSUPPORTED, "mm_trace: invalid implementation");
    Staged sa, sb;
    stage_in(A, sa);
    stage_in(B, sb);
    r_dot(sa.v, sb.v, out);
}
int msw_mm_dtrace(const msw_matrix* A, const msw_matrix* B, double* alpha, const char label[3]) {
    API_BEGIN
    double o[2];
    mm_trace_impl(A, B, o, label);
    *alpha = o[0];
    API_END
}
int msw_mm_ztrace(const msw_matrix* A, const msw_matrix* B, double alpha[2], const char label[3]) {
    API_BEGIN
    mm_trace_impl(A, B, alpha, label);
    API_END
}

// ------------------------------------------------------------------ scale / set
static void m_scale_impl(msw_matrix* C, const double be[2], const char* label) {
    if (!C) fail(OMM_ERR_ARG, "m_scale: null matrix");
    parse_op(label);
    if (C->dense()) {
        Staged s;
        stage_in(C, s);
        k_scale(s.v, be);
        stage_out(C, s);
        sync();
    } else {
        if (C->is_real) {
            for (auto& v : C->h_val) v *= be[0];
        } else {
            for (int l = 0; l < C->nnz; ++l) {
                double x = C->h_val[2 * l], y = C->h_val[2 * l + 1];
                C->h_val[2 * l] = be[0] * x - be[1] * y;
                C->h_val[2 * l + 1] = be[0] * y + be[1] * x;
            }
        }
        invalidate_csc(C);
    }
}
int msw_m_dscale(msw_matrix* C, double beta, const char label[3]) {
    API_BEGIN
    double be[2] = {beta, 0.0};
    m_scale_impl(C, be, label);
    API_END
}
int msw_m_zscale(msw_matrix* C, const double beta[2], const char label[3]) {
    API_BEGIN
    m_scale_impl(C, beta, label);
    API_END
}

static void m_set_impl(msw_matrix* C, char seC, const double al[2], const double be[2], const char* label) {
    if (!C) fail(OMM_ERR_ARG, "m_set: null matrix");
    parse_op(label);
    if (!C->dense()) fail(OMM_ERR_UNSUPPORTED, "m_set: invalid implementation");
    Staged s;
    stage_in(C, s);
    k_set(s.v, seC, al, be);
    stage_out(C, s);
    sync();
}
int msw_m_dset(msw_matrix* C, char seC, double alpha, double beta, const char label[3]) {
    API_BEGIN
    double al[2] = {alpha, 0.0}, be[2] = {beta, 0.0};
    m_set_impl(C, seC, al, be, label);
    API_END
}
int msw_m_zset(msw_matrix* C, char seC, const double alpha[2], const double beta[2], const char label[3]) {
    API_BEGIN
    m_set_impl(C, seC, alpha, beta, label);
    API_END
}

// ------------------------------------------------------------------ elements
static void set_element_impl(msw_matrix* C, int i, int j, const double al[2], const double be[2], const char* label) {
    if (!C) fail(OMM_ERR_ARG, "m_set_element: null matrix");
    parse_op(label);
    if (i < 1 || i > C->dim1 || j < 1 || j > C->dim2) fail(OMM_ERR_ARG, "m_set_element: element out of range");
    int w = C->is_real ? 1 : 2;
    if (C->dense()) {
        if (C->loc == Loc::Host) {
            double* p = (double*)C->host + ((size_t)(i - 1) + (size_t)(j - 1) * C->dim1) * w;
            if (w == 1) p[0] = al[0] + be[0] * p[0];
            else {
                double x = p[0], y = p[1];
                p[0] = al[0] + (be[0] * x - be[1] * y);
                p[1] = al[1] + (be[0] * y + be[1] * x);
            }
        } else {
            DView v{C->dev.p, C->dim1, C->dim2, std::max(1, C->dim1), C->is_real};
            k_set_element(v, i - 1, j - 1, al, be);
        }
        return;
    }
    // CSC: update in place, or insert a new entry (MatrixSwitch.F90:2917-3086 sdcsc branch)
    for (int l = C->h_colptr[j - 1]; l < C->h_colptr[j]; ++l)
        if (C->h_rowind[l] == i - 1) {
            double* p = &C->h_val[(size_t)l * w];
            if (w == 1) p[0] = al[0] + be[0] * p[0];
            else {
                double x = p[0], y = p[1];
                p[0] = al[0] + (be[0] * x - be[1] * y);
                p[1] = al[1] + (be[0] * y + be[1] * x);
            }
            invalidate_csc(C);
            return;
        }
    int pos = C->h_colptr[j];
    for (int l = C->h_colptr[j - 1]; l < C->h_colptr[j]; ++l)
        if (C->h_rowind[l] > i - 1) { pos = l; break; }
    C->h_rowind.insert(C->h_rowind.begin() + pos, i - 1);
    C->h_val.insert(C->h_val.begin() + (size_t)pos * w, al, al + w);
    for (int c = j; c <= C->dim2; ++c) C->h_colptr[c]++;
    C->nnz++;
    invalidate_csc(C);
}
int msw_m_dset_element(msw_matrix* C, int i, int j, double alpha, double beta, const char label[3]) {
    API_BEGIN
    double al[2] = {alpha, 0.0}, be[2] = {beta, 0.0};
    set_element_impl(C, i, j, al, be, label);
    API_END
}
int msw_m_zset_element(msw_matrix* C, int i, int j, const double alpha[2], const double beta[2],
                       const char label[3]) {
    API_BEGIN
    set_element_impl(C, i, j, alpha, beta, label);
    API_END
}

static void get_element_impl(const msw_matrix* C, int i, int j, double out[2], const char* label) {
    if (!C) fail(OMM_ERR_ARG, "m_get_element: null matrix");
    parse_op(label);
    if (i < 1 || i > C->dim1 || j < 1 || j > C->dim2) fail(OMM_ERR_ARG, "m_get_element: element out of range");
    int w = C->is_real ? 1 : 2;
    out[0] = out[1] = 0.0;
    if (C->dense()) {
        size_t off = ((size_t)(i - 1) + (size_t)(j - 1) * C->dim1) * w;
        if (C->loc == Loc::Host) {
            const double* p = (const double*)C->host + off;
            out[0] = p[0];
            if (w == 2) out[1] = p[1];
        } else {
            OMM_CK(cudaMemcpyAsync(rt().host_pinned, (const double*)C->dev.p + off, w * sizeof(double),
                                   cudaMemcpyDeviceToHost, rt().stream));
            sync();
            out[0] = rt().host_pinned[0];
            if (w == 2) out[1] = rt().host_pinned[1];
        }
        return;
    }
    for (int l = C->h_colptr[j - 1]; l < C->h_colptr[j]; ++l)
        if (C->h_rowind[l] == i - 1) {
            out[0] = C->h_val[(size_t)l * w];
            if (w == 2) out[1] = C->h_val[(size_t)l * w + 1];
        }
}
int msw_m_dget_element(const msw_matrix* C, int i, int j, double* alpha, const char label[3]) {
    API_BEGIN
    double o[2];
    get_element_impl(C, i, j, o, label);
    *alpha = o[0];
    API_END
}
int msw_m_zget_element(const msw_matrix* C, int i, int j, double alpha[2], const char label[3]) {
    API_BEGIN
    get_element_impl(C, i, j, alpha, label);
    API_END
}

// ------------------------------------------------------------------ pspBLAS
static void psp_impl(bool sparse_left, int M, int N, int K, const msw_matrix* A, char opA, const msw_matrix* B,
                     char opB, msw_matrix* C, const double al[2], const double be[2]) {
    if (!A || !B || !C) fail(OMM_ERR_ARG, "psp: null matrix");
    bool trA = is_tr(opA), trB = is_tr(opB);
    if (sparse_left ? (A->fmt != Fmt::CSC || !B->dense()) : (!A->dense() || B->fmt != Fmt::CSC))
        fail(OMM_ERR_ARG, sparse_left ? "psp_gespmm: A must be sparse (csc) and B dense"
                                      : "psp_gemspm: A must be dense and B sparse (csc)");
    int Ar = trA ? A->dim2 : A->dim1, Ac = trA ? A->dim1 : A->dim2;
    int Br = trB ? B->dim2 : B->dim1, Bc = trB ? B->dim1 : B->dim2;
    if (Ar != M || Bc != N || Ac != K || Br != K || C->dim1 != M || C->dim2 != N)
        fail(OMM_ERR_ARG, "psp: dimensions M, N, K do not match the matrices");
    if (A->is_real != C->is_real || B->is_real != C->is_real) fail(OMM_ERR_ARG, "psp: real/complex mismatch");
    Staged sc;
    stage_in(C, sc, true);
    if (al[0] == 0.0 && al[1] == 0.0) {
        // pspMspm.F90:114-116 / pspSpmm.F90: only C = beta*C, and nothing when beta == 0
        if (be[0] != 0.0 || be[1] != 0.0) k_scale(sc.v, be);
    } else if (sparse_left) {
        Staged sb;
        stage_in(B, sb);
        gespmm(opA, A, opB, sb.v, sc.v, al, be);
    } else {
        Staged sa;
        stage_in(A, sa);
        gemspm(opA, sa.v, opB, B, sc.v, al, be);
    }
    stage_out(C, sc);
    sync();
}

int psp_gpu_dgemspm(int M, int N, int K, const msw_matrix* A, char opA, const msw_matrix* B, char opB,
                    msw_matrix* C, double alpha, double beta) {
    API_BEGIN
    double al[2] = {alpha, 0.0}, be[2] = {beta, 0.0};
    psp_impl(false, M, N, K, A, opA, B, opB, C, al, be);
    API_END
}
int psp_gpu_zgemspm(int M, int N, int K, const msw_matrix* A, char opA, const msw_matrix* B, char opB,
                    msw_matrix* C, const double alpha[2], const double beta[2]) {
    API_BEGIN
    psp_impl(false, M, N, K, A, opA, B, opB, C, alpha, beta);
    API_END
}
int psp_gpu_dgespmm(int M, int N, int K, const msw_matrix* A, char opA, const msw_matrix* B, char opB,
                    msw_matrix* C, double alpha, double beta) {
    API_BEGIN
    double al[2] = {alpha, 0.0}, be[2] = {beta, 0.0};
    psp_impl(true, M, N, K, A, opA, B, opB, C, al, be);
    API_END
}
int psp_gpu_zgespmm(int M, int N, int K, const msw_matrix* A, char opA, const msw_matrix* B, char opB,
                    msw_matrix* C, const double alpha[2], const double beta[2]) {
    API_BEGIN
    psp_impl(true, M, N, K, A, opA, B, opB, C, alpha, beta);
    API_END
}

}  // extern "C"
