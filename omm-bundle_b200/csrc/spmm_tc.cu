// Tensor-core SpMM for atom-block sparse matrices: [HG, SG] = D [H, S] with tcgen05.
//
// Uses the column-group union plan of spmm.cu: output columns are cut into
// groups of G <= 32 columns whose nonzero rows form a union U_g, and
//     Y(:, group g) = D(:, U_g) * B_g        (B_g = |U_g| x G dense block).
// For atom-centred bases U_g is a union of whole atom blocks, i.e. of runs of
// 8 consecutive, 8-aligned rows ("chunks").  That makes the gather a set of
// bulk copies from Dk, the k-blocked bf16 shadow of D (kblock_offset: per
// 256-row block, chunk k/8 holds D(:, k..k+7) as one 16-byte vector per row):
// the chunk D(r0:r0+256, x:x+8) is one contiguous 4 KB block that lands exactly
// in the K-major no-swizzle layout tcgen05 reads (core matrices of 8 rows x
// 16 B, 128 B apart along M), and the chunks of one row block follow each
// other, so a run of consecutive chunks is one copy.  Contiguous boxes matter:
// with 16-byte pieces strided by a row pitch, the L1-to-crossbar request path
// saturates long before bytes or tensor pipes do, and a tiled TMA box issues
// one request per 16-byte line whatever the layout, so both operands are
// fetched with the untiled bulk copy, and a step whose two chunks are adjacent
// planes takes one 8 KB copy.
// B_g^T (the group's G columns, x K) is stored once per matrix in bf16 (hi, and lo
// for the split products) in 8-k chunks of NB = round16(G) rows, laid out
// [g][k/8][NB][8] so the two chunks of one 16-k step are one contiguous block.
// When S shares H's pattern, one B^T of round16(2G) rows holds H's group columns
// then S's, so a single M = 128 x N = round16(2G) x K = 16 MMA per 128-row block
// produces HG and SG together (for 24-wide atom groups N = 48 instead of two
// padded N = 32 MMAs: half the MMA issues and about half the operand reads from
// shared memory).  Per CTA: one group x 256 rows of D, accumulators in TMEM,
// FP64 column-major output split at column G between the two products.
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
    int NB = 0;           // rows of B^T per 8-k chunk: G rounded up to 16 (the MMA's N)
    DevBuf cx;            // int [ngroups][2*maxsteps]: first row of each 8-row chunk (padding repeats the last)
    DevBuf nsteps;        // int [ngroups]
    DevBuf bt_hi, bt_lo;  // bf16 [ngroups][kpad/8][NB][8]: B_g^T in 8-k chunks, zero padded
    // the pair with a second matrix of the same pattern (S beside H): its columns follow this
    // matrix's in one B^T of pair_NB = 2G rounded to 16 rows, so one MMA serves both
    unsigned long long pair_id = 0;  // pattern id of the partner the pair arrays were built for
    int pair_NB = 0;
    DevBuf pair_hi, pair_lo;
};

namespace {

using namespace tc;

constexpr int BMT = 256;                  // rows of D per CTA
constexpr int HALVES = BMT / 128;         // M = 128 MMA row blocks per CTA
constexpr int A_CHUNK = BMT * 16;         // one 8-k chunk of A: BMT rows x 16 B
constexpr int NB_MAX = 64;                // B^T rows per chunk (2G <= 64)
constexpr int B_CHUNK_MAX = NB_MAX * 16;  // one 8-k chunk of B^T at most
constexpr int ACC_STRIDE = 64;            // TMEM columns between the row blocks' accumulators

struct SpParams {
    int n, N, G;
    int nplanes;                // 8-k chunks of the k-blocked A shadow per row block
    int NB;                     // MMA N: B^T rows per chunk
    uint32_t idesc;             // instruction descriptor for N = NB
    const __nv_bfloat16* a_hi;  // Dk planes of n x 8 (hi, lo)
    const __nv_bfloat16* a_lo;
    const __nv_bfloat16* b_hi;  // B^T chunks (hi, lo): one matrix, or the pair
    const __nv_bfloat16* b_lo;
    const int* cx;
    const int* nsteps;
    int cstride;  // 2*maxsteps
    double* out0;  // columns 0 .. G-1 of the product
    int ld0;
    double* out1;  // columns G .. 2G-1 (the pair's second matrix), or null
    int ld1;
    // FP32 form (y32 set, out0/out1 unused): the products in FP32, column-major, the pair's
    // second one n rows below the first; with t_hi, the row-major bf16 shadows (hi, and lo) of
    // those values (rows 0 .. n-1 the first product, n .. 2n-1 the second)
    float* y32;
    int ldy32;
    bool pair;
    __nv_bfloat16* t_hi;
    __nv_bfloat16* t_lo;
    int ldt;
    unsigned* err;
    WaitCfg wc;
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
// kind::f16, bf16 x bf16 -> FP32, K-major A and B, M = 128, N = nb (a multiple of 16, <= 256)
inline uint32_t idesc_for(int nb) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(nb >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}

__device__ __forceinline__ void mma_sp(uint32_t tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(
            tmem),
        "l"(a), "l"(b), "r"(idesc), "r"(acc)
        : "memory");
}

// SPS 16-k steps per pipeline stage (CH = 2 SPS chunks): a stage's A chunks are fetched as runs
// of consecutive planes of the tile's row block (one bulk copy per run; atom-aligned unions are
// mostly such runs) and its B^T chunks as one copy, so wider stages mean fewer, larger copies.
template <int NSEG, int STAGES, int SPS>
__global__ void __launch_bounds__(128) spmm_tc_kernel(const __grid_constant__ SpParams p) {
    constexpr int PARTS = (NSEG == 3) ? 2 : 1;
    constexpr int CH = 2 * SPS;
    constexpr int A_BYTES = CH * A_CHUNK * PARTS;     // hi chunks, then lo chunks
    constexpr int B_BYTES = CH * B_CHUNK_MAX * PARTS;  // room for the widest B^T
    constexpr int STAGE = A_BYTES + B_BYTES;
    constexpr uint32_t TMEM_COLS = HALVES * ACC_STRIDE <= 64 ? 64 : (HALVES * ACC_STRIDE <= 128 ? 128 : 256);

    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    uint64_t* bars = (uint64_t*)(smem + STAGES * STAGE);
    uint64_t* full = bars;
    uint64_t* empty = bars + STAGES;
    uint64_t* accb = bars + 2 * STAGES;
    uint32_t* tmem_slot = (uint32_t*)(bars + 2 * STAGES + 1);
    volatile int* abort_flag = (volatile int*)(tmem_slot + 1);
    int* s_cx = (int*)(bars + 2 * STAGES + 2);  // the group's chunk starts, CH * S ints

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = blockIdx.x, row0 = blockIdx.y * BMT;
    const int S = (p.nsteps[g] + SPS - 1) / SPS;  // stages (a last odd step pairs with a zero one)
    const int* cx = p.cx + (size_t)g * p.cstride;
    const int b_chunk = p.NB * 16;  // bytes of one 8-k chunk of B^T
    const uint32_t stage_tx = (uint32_t)(CH * A_CHUNK * PARTS + CH * b_chunk * PARTS);
    const size_t rb_base = (size_t)(row0 / BMT) * p.nplanes;  // first chunk of this row block

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(smem_u32(&full[s]), 1);
            mbar_init(smem_u32(&empty[s]), 1);
        }
        mbar_init(smem_u32(accb), 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    // the producer reads a chunk start every step: staged once, they stay off its critical path
    for (int i = threadIdx.x; i < CH * S; i += blockDim.x) s_cx[i] = cx[i];
    if (warp == 2) tmem_alloc(smem_u32(tmem_slot), TMEM_COLS);
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp == 0 && lane == 0) {
        // ---------------- bulk-copy producer: per stage CH 8-k chunks of A (hi[, lo]) and of B^T
        // (nothing under the withholding test switch)
        int issued = 0;
        const int S_issue = p.wc.withhold ? 0 : S;
        for (int t = 0; t < S_issue; ++t) {
            const int s = t % STAGES, r = t / STAGES;
            if (r > 0 && !mbar_wait(smem_u32(&empty[s]), (r - 1) & 1, p.wc.ns)) {
                atomicOr(p.err, 16u);
                *abort_flag = 1;
                break;
            }
            if (*abort_flag) break;
            uint8_t* st = smem + s * STAGE;
            const uint32_t fb = smem_u32(&full[s]);
            mbar_expect_tx(fb, stage_tx);
            // A: the tile's row block of the stage's chunks (chunk starts are multiples of 8), one copy
            // per run of consecutive planes
            const int* xs = s_cx + CH * t;
            for (int c = 0; c < CH;) {
                const int p0 = xs[c] >> 3;
                int len = 1;
                while (c + len < CH && (xs[c + len] >> 3) == p0 + len) ++len;
                const size_t a = (rb_base + (size_t)p0) * (size_t)(BMT * 8);
                bulk_load(smem_u32(st + c * A_CHUNK), p.a_hi + a, (uint32_t)(len * A_CHUNK), fb);
                if (NSEG == 3) bulk_load(smem_u32(st + (CH + c) * A_CHUNK), p.a_lo + a, (uint32_t)(len * A_CHUNK), fb);
                c += len;
            }
            // B^T: chunks CH t .. CH t + CH - 1 of group g (NB rows of 16 B each, adjacent)
            const size_t b0 = (size_t)(g * p.cstride + CH * t) * p.NB * 8;
            uint8_t* sb = st + A_BYTES;
            bulk_load(smem_u32(sb), p.b_hi + b0, (uint32_t)(CH * b_chunk), fb);
            if (NSEG == 3) bulk_load(smem_u32(sb + CH * b_chunk), p.b_lo + b0, (uint32_t)(CH * b_chunk), fb);
            issued = t + 1;
        }
        for (int t = (issued > STAGES ? issued - STAGES : 0); t < issued; ++t) {
            if (!mbar_wait(smem_u32(&full[t % STAGES]), (t / STAGES) & 1, p.wc.ns)) {
                atomicOr(p.err, 32u);
                break;
            }
        }
    } else if (warp == 1 && lane == 0) {
        // ---------------- MMA issuer: one M = 128 x N = NB x K = 16 MMA per row block and step
        for (int t = 0; t < S; ++t) {
            const int s = t % STAGES, r = t / STAGES;
            if (!mbar_wait(smem_u32(&full[s]), r & 1, p.wc.ns)) {
                atomicOr(p.err, 64u);
                *abort_flag = 1;
                break;
            }
            if (*abort_flag) break;
            fence_after();
            const uint32_t sa = smem_u32(smem + s * STAGE);
            const uint32_t sb = sa + A_BYTES;
#pragma unroll
            for (int j = 0; j < SPS; ++j) {  // chunks 2j, 2j + 1 of the stage
                // B: next core matrix along K is the next chunk (b_chunk bytes); along N 128 B
                const uint32_t bj = sb + 2 * j * b_chunk;
                const uint64_t bh = desc_noswz(bj, b_chunk, 128);
                const uint32_t first = (t > 0 || j > 0) ? 1u : 0u;
#pragma unroll
                for (int h = 0; h < HALVES; ++h) {  // rows 128h .. 128h+127 of the tile
                    const uint32_t acc_cols = tmem + (uint32_t)(ACC_STRIDE * h);
                    const uint32_t ah = sa + 2 * j * A_CHUNK + h * 128 * 16;
                    const uint32_t al = sa + (CH + 2 * j) * A_CHUNK + h * 128 * 16;
                    // A: next core matrix along K is the next chunk (A_CHUNK bytes); along M 128 B
                    mma_sp(acc_cols, desc_noswz(ah, A_CHUNK, 128), bh, p.idesc, first);
                    if (NSEG == 3) {
                        mma_sp(acc_cols, desc_noswz(ah, A_CHUNK, 128),
                               desc_noswz(bj + CH * b_chunk, b_chunk, 128), p.idesc, 1u);
                        mma_sp(acc_cols, desc_noswz(al, A_CHUNK, 128), bh, p.idesc, 1u);
                    }
                }
            }
            mma_commit(smem_u32(&empty[s]));
        }
        mma_commit(smem_u32(accb));
    }
    __syncwarp();

    // ---------------- epilogue: TMEM -> FP64, columns < G to out0, G .. 2G-1 to out1
    const bool ok = mbar_wait(smem_u32(accb), 0, p.wc.ns);
    if (!ok) atomicOr(p.err, 128u);
    const bool go = __all_sync(0xffffffffu, ok && !*abort_flag && S > 0);
    fence_after();
    if (go && p.y32) {
        const int ncols = p.pair ? 2 * p.G : p.G;
#pragma unroll
        for (int h = 0; h < HALVES; ++h) {
            const int row = row0 + h * 128 + warp * 32 + lane;
            for (int q = 0; q * 32 < ncols; ++q) {
                uint32_t v[32];
                tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(ACC_STRIDE * h + 32 * q), v);
                if (row < p.n) {
                    // accumulator column c: the first product's group column c (c < G), the
                    // second's c - G; G is a multiple of 8, so no 8-column block straddles them
#pragma unroll
                    for (int cb = 0; cb < 32; cb += 8) {
                        const int c0 = 32 * q + cb;
                        if (c0 >= ncols) break;
                        const bool second = c0 >= p.G;
                        const int col0 = g * p.G + (second ? c0 - p.G : c0);
                        const size_t r = (size_t)row + (second ? (size_t)p.n : 0);
                        __align__(16) __nv_bfloat16 hi8[8], lo8[8];
#pragma unroll
                        for (int e = 0; e < 8; ++e) {
                            const float f = __uint_as_float(v[cb + e]);
                            if (col0 + e < p.N) p.y32[r + (size_t)(col0 + e) * p.ldy32] = f;
                            hi8[e] = __float2bfloat16_rn(f);
                            lo8[e] = __float2bfloat16_rn(f - __bfloat162float(hi8[e]));
                        }
                        if (p.t_hi && col0 + 8 <= p.N) {
                            *reinterpret_cast<uint4*>(p.t_hi + r * p.ldt + col0) = *reinterpret_cast<const uint4*>(hi8);
                            if (p.t_lo)
                                *reinterpret_cast<uint4*>(p.t_lo + r * p.ldt + col0) = *reinterpret_cast<const uint4*>(lo8);
                        }
                    }
                }
            }
        }
    } else if (go) {
        const int ncols = p.out1 ? 2 * p.G : p.G;
#pragma unroll
        for (int h = 0; h < HALVES; ++h) {
            const int row = row0 + h * 128 + warp * 32 + lane;
            for (int q = 0; q * 32 < ncols; ++q) {
                uint32_t v[32];
                tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(ACC_STRIDE * h + 32 * q), v);
                if (row < p.n) {
#pragma unroll
                    for (int c = 0; c < 32; ++c) {
                        const int cc = 32 * q + c;
                        if (cc >= ncols) break;
                        const bool second = cc >= p.G;
                        const int col = g * p.G + (second ? cc - p.G : cc);
                        if (col < p.N) {
                            double* out = second ? p.out1 : p.out0;
                            const int ld = second ? p.ld1 : p.ld0;
                            out[(size_t)row + (size_t)col * ld] = (double)__uint_as_float(v[c]);
                        }
                    }
                }
            }
        }
    }
    fence_before();
    __syncthreads();
    if (warp == 2) tmem_dealloc(tmem, TMEM_COLS);
}

// B^T of every group in bf16 (hi, lo), in 8-k chunks of NB rows:
// bt[((g * kpad/8 + k/8) * NB + c0 + c) * 8 + k%8] = B_g(k, c) with c0 = 0, or G for the second
// matrix of a pair (rows not written stay zero)
__global__ void build_bt_kernel(int ngroups, int G, int NB, int c0, const int* __restrict__ gptr,
                                const double* __restrict__ bvals, __nv_bfloat16* __restrict__ hi,
                                __nv_bfloat16* __restrict__ lo, int kpad) {
    int g = blockIdx.x;
    int kb = gptr[g], K = gptr[g + 1] - kb;
    for (int e = threadIdx.x; e < K * G; e += blockDim.x) {
        int k = e / G, c = e % G;
        double v = bvals[((size_t)kb + k) * G + c];
        __nv_bfloat16 h = __float2bfloat16_rn((float)v);
        __nv_bfloat16 l = __float2bfloat16_rn((float)(v - (double)__bfloat162float(h)));
        size_t off = (((size_t)g * (kpad / 8) + k / 8) * NB + c0 + c) * 8 + k % 8;
        hi[off] = h;
        lo[off] = l;
    }
}

// Four steps in flight per tile: TMEM caps the tiles per SM at 4 (128 columns each), and
// deeper pipelines only cost CTAs (measured: 6 single-step stages 16-24 % slower than 4).  One
// step per stage: 2 stages of 2 steps (half the copies, each larger) measured 0.178 ms against
// 0.165 ms for the bf16 product at lattice_8x8x8, the coarser hand-off between copies and MMAs
// costing more than the copies it saves; 2 stages of 3 steps (three CTAs per SM) measured 0.143 ms
// against 0.134 ms with FP32 output.
template <int NSEG>
constexpr int steps_per_stage() {
    return 1;
}
template <int NSEG>
constexpr int stages_for() {
    return 4 / steps_per_stage<NSEG>();
}
// stages, alignment slack, barriers, then the chunk list (cstride ints)
template <int NSEG>
int smem_for(int cstride) {
    constexpr int CH = 2 * steps_per_stage<NSEG>(), PARTS = NSEG == 3 ? 2 : 1;
    return stages_for<NSEG>() * (CH * A_CHUNK * PARTS + CH * B_CHUNK_MAX * PARTS) + 1024 + 256 +
           cstride * (int)sizeof(int);
}
static_assert(BMT == KBLOCK_ROWS, "the k-blocked shadow's row blocks are the tiles' rows");

template <int NSEG>
void launch(const SpParams& p, int ngroups) {
    constexpr int ST = stages_for<NSEG>(), SPS = steps_per_stage<NSEG>();
    const int SM = smem_for<NSEG>(p.cstride);
    if (SM > 227 * 1024) fail(OMM_ERR_UNSUPPORTED, "spmm_tc: column groups with too many row chunks");
    static int attr = 0;
    if (SM > attr) {
        OMM_CK(cudaFuncSetAttribute(spmm_tc_kernel<NSEG, ST, SPS>, cudaFuncAttributeMaxDynamicSharedMemorySize, SM));
        attr = SM;
    }
    dim3 grid(ngroups, (p.n + BMT - 1) / BMT);
    spmm_tc_kernel<NSEG, ST, SPS><<<grid, 128, SM, rt().stream>>>(p);
    OMM_KCHECK();
}

inline int round16(int x) { return (x + 15) / 16 * 16; }

}  // namespace

unsigned* tc_error_flag();
tc::WaitCfg tc_wait_cfg();

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
    maxchunks = (maxchunks + 3) / 4 * 4;  // whole two-step stages (padding chunks meet zero B^T rows)
    if (maxchunks == 0) return nullptr;
    std::vector<int> cx((size_t)P.ngroups * maxchunks, 0);
    for (int g = 0; g < P.ngroups; ++g) {
        int kb = P.gptr[g], nch = (P.gptr[g + 1] - kb) / 8;
        for (int c = 0; c < maxchunks; ++c) cx[(size_t)g * maxchunks + c] = P.urows[kb + 8 * std::min(c, nch - 1)];
    }
    T->G = P.G;
    T->NB = round16(P.G);
    T->maxsteps = maxchunks / 2;
    T->kpad = 16 * T->maxsteps;
    T->cx.alloc(cx.size() * sizeof(int));
    T->nsteps.alloc(nst.size() * sizeof(int));
    OMM_CK(cudaMemcpyAsync(T->cx.p, cx.data(), cx.size() * sizeof(int), cudaMemcpyHostToDevice, rt().stream));
    OMM_CK(cudaMemcpyAsync(T->nsteps.p, nst.data(), nst.size() * sizeof(int), cudaMemcpyHostToDevice, rt().stream));
    size_t bt = (size_t)T->NB * P.ngroups * T->kpad * sizeof(__nv_bfloat16);
    T->bt_hi.alloc_zero(bt);
    T->bt_lo.alloc_zero(bt);
    build_bt_kernel<<<P.ngroups, 256, 0, rt().stream>>>(P.ngroups, P.G, T->NB, 0, P.d_gptr, P.d_bvals,
                                                        T->bt_hi.as<__nv_bfloat16>(), T->bt_lo.as<__nv_bfloat16>(),
                                                        T->kpad);
    OMM_KCHECK();
    OMM_CK(cudaStreamSynchronize(rt().stream));
    T->ngroups = P.ngroups;
    return T.get();
}

// C (FP64, n x B->dim2 view) = A * B with A (n x K) given by its k-blocked bf16 shadow Dk (hi[, lo];
// kblock_elems(n, K) elements laid out by kblock_offset);
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
    if (T2 && T->pair_id != B2->pattern_id) {
        // one B^T for the pair: this matrix's group columns, then B2's (same groups and chunks)
        T->pair_NB = round16(2 * T->G);
        size_t bt = (size_t)T->pair_NB * T->ngroups * T->kpad * sizeof(__nv_bfloat16);
        T->pair_hi.alloc_zero(bt);
        T->pair_lo.alloc_zero(bt);
        build_bt_kernel<<<T->ngroups, 256, 0, rt().stream>>>(T->ngroups, T->G, T->pair_NB, 0, P.d_gptr, P.d_bvals,
                                                             T->pair_hi.as<__nv_bfloat16>(),
                                                             T->pair_lo.as<__nv_bfloat16>(), T->kpad);
        OMM_KCHECK();
        build_bt_kernel<<<T->ngroups, 256, 0, rt().stream>>>(T->ngroups, T->G, T->pair_NB, T->G, P2->d_gptr,
                                                             P2->d_bvals, T->pair_hi.as<__nv_bfloat16>(),
                                                             T->pair_lo.as<__nv_bfloat16>(), T->kpad);
        OMM_KCHECK();
        T->pair_id = B2->pattern_id;
    }
    SpParams p{};
    p.n = n;
    p.N = B->dim2;
    p.G = T->G;
    p.nplanes = (K + 7) / 8;
    p.NB = T2 ? T->pair_NB : T->NB;
    p.idesc = idesc_for(p.NB);
    p.a_hi = Dk_hi;
    p.a_lo = nseg == 3 ? Dk_lo : Dk_hi;
    p.b_hi = (T2 ? T->pair_hi : T->bt_hi).as<__nv_bfloat16>();
    p.b_lo = (T2 ? T->pair_lo : T->bt_lo).as<__nv_bfloat16>();
    p.cx = T->cx.as<int>();
    p.nsteps = T->nsteps.as<int>();
    p.cstride = 2 * T->maxsteps;
    p.out0 = C.as<double>();
    p.ld0 = C.ld;
    p.out1 = T2 ? C2->as<double>() : nullptr;
    p.ld1 = T2 ? C2->ld : 0;
    p.err = tc_error_flag();
    p.wc = tc_wait_cfg();
    if (p.NB > NB_MAX) fail(OMM_ERR_ARG, "spmm_tc: group too wide");
    if (nseg == 3) launch<3>(p, T->ngroups);
    else launch<1>(p, T->ngroups);
    return true;
}

// The FP32 form of the product for the mixed CG step, with the same interface as the group-block
// kernel (spmm_tc2): y (FP32, column-major, ld ldy) = A [H, S] (S's product n rows below H's) and
// the row-major bf16 shadows of y (t_lo for nseg = 3), one column group per CTA.
bool spmm_tc_f32(const __nv_bfloat16* Dk_hi, const __nv_bfloat16* Dk_lo, int n, int m, const msw_matrix* H,
                 const msw_matrix* S, float* y, int ldy, __nv_bfloat16* t_hi, __nv_bfloat16* t_lo, int ldt, int nseg) {
    SpmmPlanView P = spmm_plan_view(H), PS;
    SpmmTcPlan* T = spmm_tc_plan(H, P);
    if (!T) return false;
    SpmmTcPlan* T2 = nullptr;
    if (S) {
        if (!same_pattern(H, S)) return false;
        PS = spmm_plan_view(S);
        T2 = spmm_tc_plan(S, PS);
        if (!T2 || T2->G != T->G || T2->maxsteps != T->maxsteps || T2->ngroups != T->ngroups) return false;
    }
    if (m != H->dim1 || H->dim2 != m) fail(OMM_ERR_ARG, "spmm_tc_f32: dimensions differ");
    if (((uintptr_t)Dk_hi | (uintptr_t)Dk_lo | (uintptr_t)t_hi | (uintptr_t)t_lo) & 15)
        fail(OMM_ERR_ARG, "spmm_tc_f32: operands not 16-byte aligned");
    if (t_hi && ldt % 8) fail(OMM_ERR_ARG, "spmm_tc_f32: shadow row stride must be a multiple of 8");
    if (T->G % 8) return false;
    if (T2 && T->pair_id != S->pattern_id) {
        T->pair_NB = round16(2 * T->G);
        size_t bt = (size_t)T->pair_NB * T->ngroups * T->kpad * sizeof(__nv_bfloat16);
        T->pair_hi.alloc_zero(bt);
        T->pair_lo.alloc_zero(bt);
        build_bt_kernel<<<T->ngroups, 256, 0, rt().stream>>>(T->ngroups, T->G, T->pair_NB, 0, P.d_gptr, P.d_bvals,
                                                             T->pair_hi.as<__nv_bfloat16>(),
                                                             T->pair_lo.as<__nv_bfloat16>(), T->kpad);
        OMM_KCHECK();
        build_bt_kernel<<<T->ngroups, 256, 0, rt().stream>>>(T->ngroups, T->G, T->pair_NB, T->G, PS.d_gptr,
                                                             PS.d_bvals, T->pair_hi.as<__nv_bfloat16>(),
                                                             T->pair_lo.as<__nv_bfloat16>(), T->kpad);
        OMM_KCHECK();
        T->pair_id = S->pattern_id;
    }
    SpParams p{};
    p.n = n;
    p.N = m;
    p.G = T->G;
    p.nplanes = (m + 7) / 8;
    p.NB = T2 ? T->pair_NB : T->NB;
    p.idesc = idesc_for(p.NB);
    p.a_hi = Dk_hi;
    p.a_lo = nseg == 3 ? Dk_lo : Dk_hi;
    p.b_hi = (T2 ? T->pair_hi : T->bt_hi).as<__nv_bfloat16>();
    p.b_lo = (T2 ? T->pair_lo : T->bt_lo).as<__nv_bfloat16>();
    p.cx = T->cx.as<int>();
    p.nsteps = T->nsteps.as<int>();
    p.cstride = 2 * T->maxsteps;
    p.y32 = y;
    p.ldy32 = ldy;
    p.pair = T2 != nullptr;
    p.t_hi = t_hi;
    p.t_lo = t_lo;
    p.ldt = ldt;
    p.err = tc_error_flag();
    p.wc = tc_wait_cfg();
    if (p.NB > NB_MAX) fail(OMM_ERR_ARG, "spmm_tc_f32: group too wide");
    ktime_begin();
    if (nseg == 3) launch<3>(p, T->ngroups);
    else launch<1>(p, T->ngroups);
    const double nnz = (double)H->nnz, np_ = S ? 2.0 : 1.0;
    ktime_end("spmm_tc_kernel", np_ * (nnz * (2 * (nseg == 3 ? 2 : 1) + 4) + (m + 1) * 4.0) +
                                    (double)n * m * 2 * (nseg == 3 ? 2 : 1) + np_ * (double)n * m * 4);
    return true;
}

}  // namespace ommgpu
