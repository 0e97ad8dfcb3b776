// Tensor-core SpMM for atom-block sparse matrices: [HG, SG] = D [H, S] with tcgen05.
//
// Uses the column-group union plan of spmm.cu: output columns are cut into
// groups of G <= 32 columns whose nonzero rows form a union U_g, and
//     Y(:, group g) = D(:, U_g) * B_g        (B_g = |U_g| x G dense block).
// For atom-centred bases U_g is a union of whole atom blocks, i.e. of runs of
// 8 consecutive, 8-aligned rows ("chunks").  That makes the gather a set of
// TMA tile loads from Dk, the k-blocked bf16 shadow of D (plane k/8 holds
// D(:, k..k+7) as one 16-byte vector per row): the chunk D(r0:r0+256, x:x+8)
// is one contiguous 4 KB block that lands exactly in the K-major no-swizzle
// layout tcgen05 reads (core matrices of 8 rows x 16 B, 128 B apart along M).
// Contiguous boxes matter: with 16-byte pieces strided by a row pitch, the
// L1-to-crossbar request path saturates long before bytes or tensor pipes do,
// and a tiled TMA box issues one request per 16-byte line whatever the layout,
// so both operands are fetched with the untiled bulk copy (one 4 KB / 1 KB
// transfer each).  Dk carries a 4 KB tail so that the 256-row copy of the last
// plane stays inside the allocation (rows past n only feed output rows that
// are never stored).
// B_g^T (the group's columns padded to 32, x K) is stored once per matrix in
// bf16 (hi, and lo for the split products), laid out [g][k/8][32][8] so the
// two chunks of one 16-k step are one contiguous 1 KB block.  Per CTA: one
// group x 256 rows of D; two M=128 x N=32 x K=16 MMAs per 16 k, per value set
// (H and S share the A tiles: NM = 2), accumulators in TMEM (32 columns each),
// FP64 column-major output.
// NSEG = 3 adds the hi*lo and lo*hi products of hi/lo bf16 splits (~2^-16).
#include "internal.h"

#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cstdint>

#include "tc_ptx.h"

namespace ommgpu {

struct SpmmTcPlan {
    int G = 0, ngroups = 0, maxsteps = 0, kpad = 0;
    DevBuf cx;            // int [ngroups][2*maxsteps]: first row of each 8-row chunk (padding repeats the last)
    DevBuf nsteps;        // int [ngroups]
    DevBuf bt_hi, bt_lo;  // bf16 [ngroups][kpad/8][32][8]: B_g^T in 8-k chunks, zero padded
};

namespace {

using namespace tc;

constexpr int BMT = 256;                  // rows of D per CTA
constexpr int A_CHUNK = BMT * 16;         // one 8-k chunk of A: 256 rows x 16 B
constexpr int B_CHUNK = 32 * 16;          // one 8-k chunk of B^T: 32 rows x 16 B
constexpr int kSlack = 0;                  // no shared memory beyond the stages

struct SpParams {
    int n, N, G;
    const __nv_bfloat16* a_hi;  // Dk planes of n x 8 (hi, lo)
    const __nv_bfloat16* a_lo;
    const __nv_bfloat16* b_hi[2];  // B^T chunks of value set 0 and 1 (hi, lo)
    const __nv_bfloat16* b_lo[2];
    const int* cx;
    const int* nsteps;
    int cstride;  // 2*maxsteps
    double* out0;
    int ld0;
    double* out1;
    int ld1;
    unsigned* err;
};

// K-major, no swizzle: core matrices of 8 rows x 16 B; lbo = next core matrix along K, sbo = along M/N
__device__ __forceinline__ uint64_t desc_noswz(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFF);
    d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
    d |= (uint64_t)1 << 46;  // version
    return d;                // layout type 0 = no swizzle
}
// kind::f16, bf16 x bf16 -> FP32, K-major A and B, M = 128, N = 32
constexpr uint32_t IDESC_SP = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(32 >> 3) << 17) |
                              ((uint32_t)(128 >> 4) << 24);

__device__ __forceinline__ void mma_sp(uint32_t tmem, uint64_t a, uint64_t b, uint32_t acc) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(
            tmem),
        "l"(a), "l"(b), "r"(IDESC_SP), "r"(acc)
        : "memory");
}

template <int NM, int NSEG, int STAGES>
__global__ void __launch_bounds__(128) spmm_tc_kernel(const __grid_constant__ SpParams p) {
    constexpr int PARTS = (NSEG == 3) ? 2 : 1;
    constexpr int A_BYTES = 2 * A_CHUNK * PARTS;
    constexpr int B_BYTES = 2 * B_CHUNK * PARTS;
    constexpr int STAGE = A_BYTES + NM * B_BYTES;
    constexpr uint32_t TMEM_COLS = (NM == 2) ? 128 : 64;  // 2 row halves x NM x 32 columns

    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    uint64_t* bars = (uint64_t*)(smem + STAGES * STAGE);
    uint64_t* full = bars;
    uint64_t* empty = bars + STAGES;
    uint64_t* accb = bars + 2 * STAGES;
    uint32_t* tmem_slot = (uint32_t*)(bars + 2 * STAGES + 1);
    volatile int* abort_flag = (volatile int*)(tmem_slot + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = blockIdx.x, row0 = blockIdx.y * BMT;
    const int T = p.nsteps[g];
    const int* cx = p.cx + (size_t)g * p.cstride;

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(smem_u32(&full[s]), 1);
            mbar_init(smem_u32(&empty[s]), 1);
        }
        mbar_init(smem_u32(accb), 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 2) tmem_alloc(smem_u32(tmem_slot), TMEM_COLS);
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp == 0 && lane == 0) {
        // ---------------- TMA producer: per step two 8-k chunks of A (hi[, lo]) and of each B^T
        int issued = 0;
        for (int t = 0; t < T; ++t) {
            const int s = t % STAGES, r = t / STAGES;
            if (r > 0 && !mbar_wait(smem_u32(&empty[s]), (r - 1) & 1)) {
                atomicOr(p.err, 16u);
                *abort_flag = 1;
                break;
            }
            if (*abort_flag) break;
            uint8_t* st = smem + s * STAGE;
            const uint32_t fb = smem_u32(&full[s]);
            mbar_expect_tx(fb, STAGE);
            const int x0 = __ldg(cx + 2 * t), x1 = __ldg(cx + 2 * t + 1);
            // A: rows row0..row0+255 of planes x0/8 and x1/8 of Dk (x0, x1 are multiples of 8)
            const size_t a0 = ((size_t)(x0 >> 3) * p.n + row0) * 8, a1 = ((size_t)(x1 >> 3) * p.n + row0) * 8;
            bulk_load(smem_u32(st), p.a_hi + a0, A_CHUNK, fb);
            bulk_load(smem_u32(st + A_CHUNK), p.a_hi + a1, A_CHUNK, fb);
            if (NSEG == 3) {
                bulk_load(smem_u32(st + 2 * A_CHUNK), p.a_lo + a0, A_CHUNK, fb);
                bulk_load(smem_u32(st + 3 * A_CHUNK), p.a_lo + a1, A_CHUNK, fb);
            }
            // B^T: chunks 2t and 2t+1 of group g (32 rows of 16 B each, adjacent)
            const size_t b0 = (size_t)(g * p.cstride + 2 * t) * 32 * 8;
#pragma unroll
            for (int mm = 0; mm < NM; ++mm) {
                uint8_t* sb = st + A_BYTES + mm * B_BYTES;
                bulk_load(smem_u32(sb), p.b_hi[mm] + b0, 2 * B_CHUNK, fb);
                if (NSEG == 3) bulk_load(smem_u32(sb + 2 * B_CHUNK), p.b_lo[mm] + b0, 2 * B_CHUNK, fb);
            }
            issued = t + 1;
        }
        for (int t = (issued > STAGES ? issued - STAGES : 0); t < issued; ++t) {
            if (!mbar_wait(smem_u32(&full[t % STAGES]), (t / STAGES) & 1)) {
                atomicOr(p.err, 32u);
                break;
            }
        }
    } else if (warp == 1 && lane == 0) {
        // ---------------- MMA issuer
        for (int t = 0; t < T; ++t) {
            const int s = t % STAGES, r = t / STAGES;
            if (!mbar_wait(smem_u32(&full[s]), r & 1)) {
                atomicOr(p.err, 64u);
                *abort_flag = 1;
                break;
            }
            if (*abort_flag) break;
            fence_after();
            const uint32_t sa = smem_u32(smem + s * STAGE);
#pragma unroll
            for (int mm = 0; mm < NM; ++mm) {
                const uint32_t sb = sa + A_BYTES + mm * B_BYTES;
#pragma unroll
                for (int h = 0; h < 2; ++h) {  // rows 0-127 and 128-255 of the tile
                    const uint32_t acc_cols = tmem + (uint32_t)(32 * (2 * mm + h));
                    const uint32_t ah = sa + h * 128 * 16, al = sa + 2 * A_CHUNK + h * 128 * 16;
                    // A: next core matrix along K is the next chunk (A_CHUNK bytes); along M 128 B
                    mma_sp(acc_cols, desc_noswz(ah, A_CHUNK, 128), desc_noswz(sb, B_CHUNK, 128), t > 0 ? 1u : 0u);
                    if (NSEG == 3) {
                        mma_sp(acc_cols, desc_noswz(ah, A_CHUNK, 128), desc_noswz(sb + 2 * B_CHUNK, B_CHUNK, 128), 1u);
                        mma_sp(acc_cols, desc_noswz(al, A_CHUNK, 128), desc_noswz(sb, B_CHUNK, 128), 1u);
                    }
                }
            }
            mma_commit(smem_u32(&empty[s]));
        }
        mma_commit(smem_u32(accb));
    }
    __syncwarp();

    // ---------------- epilogue
    const bool ok = mbar_wait(smem_u32(accb), 0);
    if (!ok) atomicOr(p.err, 128u);
    const bool go = __all_sync(0xffffffffu, ok && !*abort_flag && T > 0);
    fence_after();
    if (go) {
#pragma unroll
        for (int mm = 0; mm < NM; ++mm) {
            double* out = (mm == 0) ? p.out0 : p.out1;
            const int ld = (mm == 0) ? p.ld0 : p.ld1;
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                uint32_t v[32];
                tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(32 * (2 * mm + h)), v);
                const int row = row0 + h * 128 + warp * 32 + lane;
                if (row < p.n) {
#pragma unroll
                    for (int c = 0; c < 32; ++c) {
                        const int col = g * p.G + c;
                        if (c < p.G && col < p.N) out[(size_t)row + (size_t)col * ld] = (double)__uint_as_float(v[c]);
                    }
                }
            }
        }
    }
    fence_before();
    __syncthreads();
    if (warp == 2) tmem_dealloc(tmem, TMEM_COLS);
}

// B^T of every group in bf16 (hi, lo), in 8-k chunks:
// bt[((g * kpad/8 + k/8) * 32 + c) * 8 + k%8] = B_g(k, c)
__global__ void build_bt_kernel(int ngroups, int G, const int* __restrict__ gptr, const double* __restrict__ bvals,
                                __nv_bfloat16* __restrict__ hi, __nv_bfloat16* __restrict__ lo, int kpad) {
    int g = blockIdx.x;
    int kb = gptr[g], K = gptr[g + 1] - kb;
    for (int e = threadIdx.x; e < K * G; e += blockDim.x) {
        int k = e / G, c = e % G;
        double v = bvals[((size_t)kb + k) * G + c];
        __nv_bfloat16 h = __float2bfloat16_rn((float)v);
        __nv_bfloat16 l = __float2bfloat16_rn((float)(v - (double)__bfloat162float(h)));
        size_t off = (((size_t)g * (kpad / 8) + k / 8) * 32 + c) * 8 + k % 8;
        hi[off] = h;
        lo[off] = l;
    }
}

template <int NM, int NSEG>
constexpr int stages_for() {
    return NSEG == 3 ? 4 : 6;
}
template <int NM, int NSEG>
constexpr int smem_for() {
    return stages_for<NM, NSEG>() * (2 * A_CHUNK * (NSEG == 3 ? 2 : 1) + NM * 2 * B_CHUNK * (NSEG == 3 ? 2 : 1)) +
           1024 + 256 + kSlack;
}

template <int NM, int NSEG>
void launch(const SpParams& p, int ngroups) {
    constexpr int ST = stages_for<NM, NSEG>();
    constexpr int SM = smem_for<NM, NSEG>();
    static bool attr = false;
    if (!attr) {
        OMM_CK(cudaFuncSetAttribute(spmm_tc_kernel<NM, NSEG, ST>, cudaFuncAttributeMaxDynamicSharedMemorySize, SM));
        attr = true;
    }
    dim3 grid(ngroups, (p.n + BMT - 1) / BMT);
    spmm_tc_kernel<NM, NSEG, ST><<<grid, 128, SM, rt().stream>>>(p);
    OMM_KCHECK();
}

}  // namespace

unsigned* tc_error_flag();

// Build (once per matrix) the tensor-core plan; false when the matrix's groups are not unions of
// aligned 8-row runs or are wider than 32 columns.
SpmmTcPlan* spmm_tc_plan(const msw_matrix* B, const SpmmPlanView& P) {
    msw_matrix* Bm = const_cast<msw_matrix*>(B);
    if (Bm->tc_plan) return Bm->tc_plan->ngroups ? Bm->tc_plan.get() : nullptr;
    auto T = std::make_shared<SpmmTcPlan>();
    Bm->tc_plan = T;
    if (!P.cgu || P.G > 32 || !B->is_real) return nullptr;
    int maxchunks = 0;
    std::vector<int> nst(P.ngroups);
    for (int g = 0; g < P.ngroups; ++g) {
        int kb = P.gptr[g], K = P.gptr[g + 1] - kb;
        if (K == 0 || K % 8) return nullptr;
        for (int c = 0; c < K / 8; ++c) {
            int x = P.urows[kb + 8 * c];
            if (x % 8) return nullptr;
            for (int q = 1; q < 8; ++q)
                if (P.urows[kb + 8 * c + q] != x + q) return nullptr;
        }
        nst[g] = (K / 8 + 1) / 2;
        maxchunks = std::max(maxchunks, 2 * nst[g]);
    }
    if (maxchunks == 0) return nullptr;
    std::vector<int> cx((size_t)P.ngroups * maxchunks, 0);
    for (int g = 0; g < P.ngroups; ++g) {
        int kb = P.gptr[g], nch = (P.gptr[g + 1] - kb) / 8;
        for (int c = 0; c < maxchunks; ++c) cx[(size_t)g * maxchunks + c] = P.urows[kb + 8 * std::min(c, nch - 1)];
    }
    T->G = P.G;
    T->maxsteps = maxchunks / 2;
    T->kpad = 16 * T->maxsteps;
    T->cx.alloc(cx.size() * sizeof(int));
    T->nsteps.alloc(nst.size() * sizeof(int));
    OMM_CK(cudaMemcpyAsync(T->cx.p, cx.data(), cx.size() * sizeof(int), cudaMemcpyHostToDevice, rt().stream));
    OMM_CK(cudaMemcpyAsync(T->nsteps.p, nst.data(), nst.size() * sizeof(int), cudaMemcpyHostToDevice, rt().stream));
    size_t bt = (size_t)32 * P.ngroups * T->kpad * sizeof(__nv_bfloat16);
    T->bt_hi.alloc_zero(bt);
    T->bt_lo.alloc_zero(bt);
    build_bt_kernel<<<P.ngroups, 256, 0, rt().stream>>>(P.ngroups, P.G, P.d_gptr, P.d_bvals,
                                                        T->bt_hi.as<__nv_bfloat16>(), T->bt_lo.as<__nv_bfloat16>(),
                                                        T->kpad);
    OMM_KCHECK();
    OMM_CK(cudaStreamSynchronize(rt().stream));
    T->ngroups = P.ngroups;
    return T.get();
}

// C (FP64, n x B->dim2 view) = A * B with A (n x K) given by its k-blocked bf16 shadow Dk (hi[, lo];
// ceil(K/8) planes of n x 8, followed by at least SPMM_TC_TAIL readable bytes);
// optional second matrix B2 with the same groups into C2.
bool spmm_tc(const __nv_bfloat16* Dk_hi, const __nv_bfloat16* Dk_lo, int n, int K, const msw_matrix* B,
             const SpmmPlanView& P, DView& C, const msw_matrix* B2, const SpmmPlanView* P2, DView* C2, int nseg) {
    SpmmTcPlan* T = spmm_tc_plan(B, P);
    if (!T) return false;
    SpmmTcPlan* T2 = nullptr;
    if (B2) {
        T2 = spmm_tc_plan(B2, *P2);
        if (!T2 || T2->G != T->G || T2->maxsteps != T->maxsteps || T2->ngroups != T->ngroups) return false;
    }
    if (K != B->dim1) fail(OMM_ERR_ARG, "spmm_tc: inner dimensions differ");
    if (((uintptr_t)Dk_hi | (uintptr_t)Dk_lo) & 15) fail(OMM_ERR_ARG, "spmm_tc: shadow not 16-byte aligned");
    SpParams p{};
    p.n = n;
    p.N = B->dim2;
    p.G = T->G;
    p.a_hi = Dk_hi;
    p.a_lo = nseg == 3 ? Dk_lo : Dk_hi;
    p.b_hi[0] = T->bt_hi.as<__nv_bfloat16>();
    p.b_lo[0] = T->bt_lo.as<__nv_bfloat16>();
    p.b_hi[1] = T2 ? T2->bt_hi.as<__nv_bfloat16>() : p.b_hi[0];
    p.b_lo[1] = T2 ? T2->bt_lo.as<__nv_bfloat16>() : p.b_lo[0];
    p.cx = T->cx.as<int>();
    p.nsteps = T->nsteps.as<int>();
    p.cstride = 2 * T->maxsteps;
    p.out0 = C.as<double>();
    p.ld0 = C.ld;
    p.out1 = T2 ? C2->as<double>() : nullptr;
    p.ld1 = T2 ? C2->ld : 0;
    p.err = tc_error_flag();
    if (T2) {
        if (nseg == 3) launch<2, 3>(p, T->ngroups);
        else launch<2, 1>(p, T->ngroups);
    } else {
        if (nseg == 3) launch<1, 3>(p, T->ngroups);
        else launch<1, 1>(p, T->ngroups);
    }
    return true;
}

}  // namespace ommgpu
