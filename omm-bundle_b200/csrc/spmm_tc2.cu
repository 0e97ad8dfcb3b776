// Tensor-core SpMM over blocks of column groups: [HG, SG] = D [H, S] in FP32, with the bf16
// shadows the next products read, for atom-block CSC matrices (the mixed solver's per-step
// product, psp_gemspm's local update pspMspm_nn.F90:191-198 in reduced precision).
//
// The column-group plan of spmm.cu cuts the output columns into groups of G columns whose
// nonzero rows form a union U_g, a list of 8-row chunks; the k-blocked bf16 shadow Dk of D
// holds chunk x of a 256-row block as one contiguous 4 KB plane.  spmm_tc.cu gives every group
// its own CTA, so each plane of D is fetched once per group whose union holds it (33 times on
// a radius-2 cubic lattice).  Here a CTA takes GB consecutive groups (neighbouring atoms):
// it walks the union W of their chunk lists, CW chunks per pipeline stage, fetching each
// plane of W once (consecutive planes as one bulk copy), and for every group of the block
// pairs up the group's chunks inside the stage (an odd one with a zero chunk) into
// M128 x N x K16 MMAs accumulating in that group's TMEM tile.  On a cubic lattice four
// atoms along x share 72 shell atoms where one atom has 33: 0.55 of the plane fetches.
// The B^T values of every (stage, group, chunk pair) are laid out in MMA order, so a stage's
// B operand is one contiguous bulk copy.  When S shares H's pattern one B^T of N = 2G rounded
// to 16 holds H's group columns then S's (one MMA serves both products).
//
// Output: Y (FP32, column-major, leading dimension ldy; S's product n rows below H's) and,
// optionally, the row-major bf16 shadows of Y (hi, and lo for the split products) that the
// Gram product reads, written from the same registers (each thread one row, G contiguous
// values per group).  NSEG = 3 adds the hi*lo and lo*hi products of hi/lo bf16 splits.
#include "internal.h"

#include <cuda.h>

#include <algorithm>
#include <cstdint>
#include <vector>

#include "tc_ptx.h"

namespace ommgpu {

unsigned* tc_error_flag();
tc::WaitCfg tc_wait_cfg();

struct SpmmTc2Plan {
    int G = 0, NB = 0, ngroups = 0, nblocks = 0, GB = 0, CW = 0;
    int maxstages = 0, maxprog = 0;
    DevBuf planes;  // int [nblocks][maxstages * CW]: the block's union chunks (planes), -1 past the end
    DevBuf nchunks; // int [nblocks]
    DevBuf prog;    // uint16 [nblocks][maxstages][maxprog]: slot << 12 | x << 6 | y (y == CW: zero chunk)
    DevBuf nprog;   // int [nblocks][maxstages]
    DevBuf bofs;    // int [nblocks][maxstages]: first pair of the stage in the B^T array
    DevBuf pairs;   // int4 [npairs]: (group, chunk of the pair's first half, of its second or -1, 0)
    int npairs = 0;
    DevBuf bt_hi, bt_lo;  // bf16 [npairs][2][NB][8]
    unsigned long long h_id = 0, s_id = 0;  // the matrices the B^T arrays were built from
};

namespace {

using namespace tc;

constexpr int BMT = 256;           // rows of D per CTA (two M = 128 MMA row blocks)
constexpr int A_CHUNK = BMT * 16;  // one 8-k plane of a 256-row block
constexpr int GB_MAX = 4;          // groups per block: GB x 2 row blocks x 64 TMEM columns = 512
constexpr int STAGES2 = 3;

struct Tc2Params {
    int n, G, NB, GB, ngroups, nplanes, maxstages, maxprog;
    uint32_t idesc;
    const __nv_bfloat16* a_hi;  // Dk (hi, lo)
    const __nv_bfloat16* a_lo;
    const __nv_bfloat16* b_hi;  // B^T pairs (hi, lo)
    const __nv_bfloat16* b_lo;
    const int* planes;
    const int* nchunks;
    const uint16_t* prog;
    const int* nprog;
    const int* bofs;
    float* y;  // H's product; S's at y + n (same columns)
    int ldy;
    bool pair;
    __nv_bfloat16* t_hi;  // row-major shadows of Y (rows 0..n-1 H, n..2n-1 S), or null
    __nv_bfloat16* t_lo;
    int ldt;
    unsigned* err;
    WaitCfg wc;
};

__device__ __forceinline__ uint64_t desc_noswz2(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFF);
    d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
    d |= (uint64_t)1 << 46;
    return d;
}
__device__ __forceinline__ void mma_bf16(uint32_t tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(
            tmem),
        "l"(a), "l"(b), "r"(idesc), "r"(acc)
        : "memory");
}

template <int CW, int PARTS>
struct Tc2Layout {
    static constexpr int A_BYTES = CW * A_CHUNK * PARTS;            // hi planes, then lo planes
    static constexpr int PAIR_BYTES = 2 * 64 * 16;                  // the largest pair (NB = 64)
    static constexpr int B_BYTES = GB_MAX * (CW / 2) * PAIR_BYTES * PARTS;
    static constexpr int STAGE = A_BYTES + B_BYTES;
    static constexpr int ZERO = STAGES2 * STAGE;                    // one zero plane after the stages
    static constexpr int BARS = ZERO + A_CHUNK;
    static constexpr int TABLES = BARS + 128;
};

// one CTA: block blockIdx.x of GB groups x rows 256 blockIdx.y .. + 255
template <int NSEG, int CW>
__global__ void __launch_bounds__(192, 1) spmm_tc2_kernel(const __grid_constant__ Tc2Params p) {
    constexpr int PARTS = NSEG == 3 ? 2 : 1;
    using LY = Tc2Layout<CW, PARTS>;
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    uint64_t* bars = (uint64_t*)(smem + LY::BARS);
    uint64_t* full = bars;
    uint64_t* empty = bars + STAGES2;
    uint64_t* accb = bars + 2 * STAGES2;
    uint32_t* tmem_slot = (uint32_t*)(bars + 2 * STAGES2 + 1);
    volatile int* abort_flag = (volatile int*)(tmem_slot + 1);
    int* s_planes = (int*)(smem + LY::TABLES);                  // maxstages * CW
    int* s_nprog = s_planes + p.maxstages * CW;                 // maxstages
    int* s_bofs = s_nprog + p.maxstages;                        // maxstages
    uint16_t* s_prog = (uint16_t*)(s_bofs + p.maxstages);       // maxstages * maxprog

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int b = blockIdx.x, rb = blockIdx.y, row0 = rb * BMT;
    const int L = p.nchunks[b];
    const int S = (L + CW - 1) / CW;
    const uint32_t pair_bytes = (uint32_t)(2 * p.NB * 16);
    const uint32_t zero_addr = smem_u32(smem + LY::ZERO);

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES2; ++s) {
            mbar_init(smem_u32(&full[s]), 1);
            mbar_init(smem_u32(&empty[s]), GB_MAX);  // one commit per issuing warp
        }
        mbar_init(smem_u32(accb), GB_MAX);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    // the block's tables and the zero plane, once
    for (int i = threadIdx.x; i < S * CW; i += blockDim.x) s_planes[i] = p.planes[(size_t)b * p.maxstages * CW + i];
    for (int i = threadIdx.x; i < S; i += blockDim.x) {
        s_nprog[i] = p.nprog[(size_t)b * p.maxstages + i];
        s_bofs[i] = p.bofs[(size_t)b * p.maxstages + i];
    }
    for (int i = threadIdx.x; i < S * p.maxprog; i += blockDim.x)
        s_prog[i] = p.prog[(size_t)b * p.maxstages * p.maxprog + i];
    for (int i = threadIdx.x; i < A_CHUNK / 16; i += blockDim.x)
        reinterpret_cast<uint4*>(smem + LY::ZERO)[i] = make_uint4(0, 0, 0, 0);
    if (warp == 2) tmem_alloc(smem_u32(tmem_slot), 512);
    // the zero plane is read by the tensor core (async proxy): order the generic-proxy stores
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = *tmem_slot;
    const size_t rb_base = (size_t)rb * p.nplanes;

    if (warp == 0 && lane == 0) {
        // ---------------- producer: the stage's planes (runs of consecutive planes as one copy), its B^T pairs
        int issued = 0;
        const int S_issue = p.wc.withhold ? 0 : S;
        for (int t = 0; t < S_issue; ++t) {
            const int s = t % STAGES2, r = t / STAGES2;
            if (r > 0 && !mbar_wait(smem_u32(&empty[s]), (r - 1) & 1, p.wc.ns)) {
                atomicOr(p.err, 16u);
                *abort_flag = 1;
                break;
            }
            if (*abort_flag) break;
            uint8_t* st = smem + s * LY::STAGE;
            const int nch = min(CW, L - t * CW), np = s_nprog[t];
            const uint32_t fb = smem_u32(&full[s]);
            mbar_expect_tx(fb, (uint32_t)(nch * A_CHUNK * PARTS) + (uint32_t)np * pair_bytes * PARTS);
            const int* xs = s_planes + t * CW;
            for (int c = 0; c < nch;) {
                const int p0 = xs[c];
                int len = 1;
                while (c + len < nch && xs[c + len] == p0 + len) ++len;
                const size_t a = (rb_base + (size_t)p0) * (size_t)(BMT * 8);
                bulk_load(smem_u32(st + c * A_CHUNK), p.a_hi + a, (uint32_t)(len * A_CHUNK), fb);
                if (NSEG == 3)
                    bulk_load(smem_u32(st + (CW + c) * A_CHUNK), p.a_lo + a, (uint32_t)(len * A_CHUNK), fb);
                c += len;
            }
            const size_t b0 = (size_t)s_bofs[t] * (size_t)(2 * p.NB * 8);
            uint8_t* sb = st + LY::A_BYTES;
            bulk_load(smem_u32(sb), p.b_hi + b0, (uint32_t)np * pair_bytes, fb);
            if (NSEG == 3) bulk_load(smem_u32(sb + np * pair_bytes), p.b_lo + b0, (uint32_t)np * pair_bytes, fb);
            issued = t + 1;
        }
        for (int t = (issued > STAGES2 ? issued - STAGES2 : 0); t < issued; ++t) {
            if (!mbar_wait(smem_u32(&full[t % STAGES2]), (t / STAGES2) & 1, p.wc.ns)) {
                atomicOr(p.err, 32u);
                break;
            }
        }
    } else if (warp >= 1 && warp <= GB_MAX && lane == 0) {
        // ---------------- MMA issuers: warp 1 + a issues the MMAs of slot a's program entries
        // (planes x, y; one MMA per row block).  The four issuers are separate warps, so their
        // descriptor work and issue run side by side on the SM's four sub-partitions; each
        // commits its own MMAs
        const int a = warp - 1;
        uint32_t used = 0;  // this slot's accumulators (row block 0, 1) already written
        for (int t = 0; t < S; ++t) {
            const int s = t % STAGES2, r = t / STAGES2;
            if (!mbar_wait(smem_u32(&full[s]), r & 1, p.wc.ns)) {
                atomicOr(p.err, 64u);
                *abort_flag = 1;
                break;
            }
            if (*abort_flag) break;
            fence_after();
            const uint32_t sa = smem_u32(smem + s * LY::STAGE);
            const uint32_t sb = sa + LY::A_BYTES;
            const int np = s_nprog[t];
            const uint16_t* pr = s_prog + t * p.maxprog;
            // entries are ordered by slot: this slot's run starts after the entries of slots < a
            int i = 0;
            while (i < np && (pr[i] >> 12) < a) ++i;
            for (; i < np && (pr[i] >> 12) == a; ++i) {
                const int e = pr[i], x = (e >> 6) & 63, y = e & 63;
                const uint32_t bh = sb + (uint32_t)i * pair_bytes;
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const uint32_t acc = tmem + (uint32_t)((a * 2 + h) * 64);
                    const uint32_t bit = 1u << h;
                    const uint32_t ax = sa + (uint32_t)(x * A_CHUNK + h * 128 * 16);
                    const uint32_t lbo = y == CW ? zero_addr - (sa + (uint32_t)(x * A_CHUNK)) : (uint32_t)((y - x) * A_CHUNK);
                    mma_bf16(acc, desc_noswz2(ax, lbo, 128), desc_noswz2(bh, p.NB * 16, 128), p.idesc,
                             (used & bit) ? 1u : 0u);
                    used |= bit;
                    if (NSEG == 3) {
                        const uint32_t bl = sb + (uint32_t)np * pair_bytes + (uint32_t)i * pair_bytes;
                        const uint32_t sal = sa + (uint32_t)(CW * A_CHUNK);
                        const uint32_t axl = sal + (uint32_t)(x * A_CHUNK + h * 128 * 16);
                        const uint32_t lbol =
                            y == CW ? zero_addr - (sal + (uint32_t)(x * A_CHUNK)) : (uint32_t)((y - x) * A_CHUNK);
                        mma_bf16(acc, desc_noswz2(ax, lbo, 128), desc_noswz2(bl, p.NB * 16, 128), p.idesc, 1u);
                        mma_bf16(acc, desc_noswz2(axl, lbol, 128), desc_noswz2(bh, p.NB * 16, 128), p.idesc, 1u);
                    }
                }
            }
            mma_commit(smem_u32(&empty[s]));
        }
        mma_commit(smem_u32(accb));
    }
    __syncwarp();

    // ---------------- epilogue: warps 2-5, warp w holds TMEM lanes 32 (w % 4) .. + 31 of both row blocks
    const bool ok = mbar_wait(smem_u32(accb), 0, p.wc.ns);
    if (!ok) atomicOr(p.err, 128u);
    const bool go = __all_sync(0xffffffffu, ok && !*abort_flag && S > 0);
    fence_after();
    const int quarter = warp & 3;
    if (go && warp >= 2) {
        for (int a = 0; a < p.GB; ++a) {
            const int g = b * p.GB + a;
            if (g >= p.ngroups) break;
#pragma unroll 1
            for (int h = 0; h < 2; ++h) {
                const int row = row0 + h * 128 + quarter * 32 + lane;
                uint32_t v[64];
                const uint32_t base = tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)((a * 2 + h) * 64);
                tmem_ld32(base, *reinterpret_cast<uint32_t(*)[32]>(v));
                tmem_ld32(base + 32, *reinterpret_cast<uint32_t(*)[32]>(v + 32));
                if (row < p.n) {
                    // accumulator column c: H's group column c (c < G), S's column c - G (c < 2G);
                    // constant indices keep v[] in registers
                    const int c0 = g * p.G, nc = p.pair ? 2 * p.G : p.G;
#pragma unroll
                    for (int c = 0; c < 64; ++c) {
                        if (c < nc) {
                            const bool sp = c >= p.G;
                            p.y[(size_t)(sp ? p.n : 0) + (size_t)row + (size_t)(c0 + (sp ? c - p.G : c)) * p.ldy] =
                                __uint_as_float(v[c]);
                        }
                    }
                    if (p.t_hi) {
#pragma unroll
                        for (int cb = 0; cb < 64; cb += 8) {
                            if (cb < nc) {
                                const bool sp = cb >= p.G;
                                const size_t to = (size_t)(row + (sp ? p.n : 0)) * p.ldt + c0 + (sp ? cb - p.G : cb);
                                __align__(16) __nv_bfloat16 hi8[8], lo8[8];
#pragma unroll
                                for (int e = 0; e < 8; ++e) {
                                    const float f = __uint_as_float(v[cb + e]);
                                    hi8[e] = __float2bfloat16_rn(f);
                                    lo8[e] = __float2bfloat16_rn(f - __bfloat162float(hi8[e]));
                                }
                                *reinterpret_cast<uint4*>(p.t_hi + to) = *reinterpret_cast<const uint4*>(hi8);
                                if (p.t_lo) *reinterpret_cast<uint4*>(p.t_lo + to) = *reinterpret_cast<const uint4*>(lo8);
                            }
                        }
                    }
                }
            }
        }
    }
    fence_before();
    __syncthreads();
    if (warp == 2) tmem_dealloc(tmem, 512);
}

// B^T of every pair: bt[((q * 2 + half) * NB + c) * 8 + kk] = B_g(8 chunk + kk, c) for the pair's
// chunk of that half (zero for a missing one), c < G from H, G <= c < 2G from S (when given)
__global__ void build_pairs_kernel(int npairs, int G, int NB, const int4* __restrict__ pairs,
                                   const int* __restrict__ gptr, const double* __restrict__ bh,
                                   const double* __restrict__ bs, __nv_bfloat16* __restrict__ hi,
                                   __nv_bfloat16* __restrict__ lo) {
    const size_t per = (size_t)2 * NB * 8;
    const size_t tot = per * npairs;
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < tot; e += (size_t)gridDim.x * blockDim.x) {
        const int q = (int)(e / per);
        const int rem = (int)(e % per);
        const int half = rem / (NB * 8), c = (rem / 8) % NB, kk = rem % 8;
        const int4 pr = pairs[q];
        const int ch = half ? pr.z : pr.y;
        double v = 0.0;
        if (ch >= 0) {
            const size_t k = (size_t)gptr[pr.x] + (size_t)(8 * ch + kk);
            if (c < G) v = bh[k * G + c];
            else if (bs && c < 2 * G) v = bs[k * G + (c - G)];
        }
        const __nv_bfloat16 h = __float2bfloat16_rn((float)v);
        hi[e] = h;
        lo[e] = __float2bfloat16_rn((float)(v - (double)__bfloat162float(h)));
    }
}

inline int round16(int x) { return (x + 15) / 16 * 16; }
inline uint32_t idesc_n(int nb) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(nb >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}

template <int NSEG, int CW>
void launch2(const Tc2Params& p, int nblocks, int nrb) {
    using LY = Tc2Layout<CW, NSEG == 3 ? 2 : 1>;
    const int sm = LY::TABLES + 1024 + p.maxstages * (CW + 2) * 4 + p.maxstages * p.maxprog * 2 + 64;
    if (sm > 227 * 1024) fail(OMM_ERR_UNSUPPORTED, "spmm_tc2: block tables exceed shared memory");
    static int attr = 0;
    if (sm > attr) {
        OMM_CK(cudaFuncSetAttribute(spmm_tc2_kernel<NSEG, CW>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
        attr = sm;
    }
    spmm_tc2_kernel<NSEG, CW><<<dim3(nblocks, nrb), 192, sm, rt().stream>>>(p);
    OMM_KCHECK();
}

}  // namespace

// CW of the stage windows: 8 planes for plain bf16, 4 for the split products (twice the bytes)
constexpr int cw_for(int nseg) { return nseg == 3 ? 4 : 8; }

// The block plan of H (with S beside it when given; same pattern), built on first use and
// when either matrix changed; nullptr when the pattern cannot take the tensor cores.
SpmmTc2Plan* spmm_tc2_plan(const msw_matrix* H, const SpmmPlanView& P, const msw_matrix* S,
                           const SpmmPlanView* PS, int nseg) {
    if (!spmm_tc_available(H)) return nullptr;
    msw_matrix* Hm = const_cast<msw_matrix*>(H);
    const int CW = cw_for(nseg);
    const unsigned long long sid = S ? S->pattern_id : 0;
    SpmmTc2Plan* T = (nseg == 3 ? Hm->tc2_plan_split : Hm->tc2_plan).get();
    if (T && T->h_id == H->pattern_id && T->s_id == sid) return T;
    auto Tn = std::make_shared<SpmmTc2Plan>();
    T = Tn.get();
    T->G = P.G;
    T->NB = S ? round16(2 * P.G) : round16(P.G);
    if (T->NB > 64) return nullptr;
    T->ngroups = P.ngroups;
    T->GB = GB_MAX;
    T->CW = CW;
    T->nblocks = (P.ngroups + T->GB - 1) / T->GB;
    T->maxprog = T->GB * CW / 2;
    // chunk lists per group, union per block, stage programs
    std::vector<std::vector<int>> W(T->nblocks);
    for (int bl = 0; bl < T->nblocks; ++bl) {
        std::vector<int>& w = W[bl];
        for (int a = 0; a < T->GB; ++a) {
            const int g = bl * T->GB + a;
            if (g >= P.ngroups) break;
            for (int k = P.gptr[g]; k < P.gptr[g + 1]; k += 8) w.push_back(P.urows[k] / 8);
        }
        std::sort(w.begin(), w.end());
        w.erase(std::unique(w.begin(), w.end()), w.end());
        T->maxstages = std::max(T->maxstages, (int)((w.size() + CW - 1) / CW));
    }
    const int MS = T->maxstages;
    std::vector<int> planes((size_t)T->nblocks * MS * CW, -1), nch(T->nblocks), nprog((size_t)T->nblocks * MS, 0),
        bofs((size_t)T->nblocks * MS, 0);
    std::vector<uint16_t> prog((size_t)T->nblocks * MS * T->maxprog, 0);
    std::vector<int4> pairs;
    for (int bl = 0; bl < T->nblocks; ++bl) {
        const std::vector<int>& w = W[bl];
        nch[bl] = (int)w.size();
        for (size_t i = 0; i < w.size(); ++i) planes[(size_t)bl * MS * CW + i] = w[i];
        const int S_b = (int)((w.size() + CW - 1) / CW);
        for (int t = 0; t < S_b; ++t) {
            const size_t pt = (size_t)bl * MS + t;
            bofs[pt] = (int)pairs.size();
            const int lo_ = t * CW, hi_ = std::min((int)w.size(), lo_ + CW);
            int cnt = 0;
            for (int a = 0; a < T->GB; ++a) {
                const int g = bl * T->GB + a;
                if (g >= P.ngroups) break;
                // the group's chunks (index c in its union) that fall in this window, in order
                std::vector<std::pair<int, int>> in;  // (window position, chunk index)
                const int nchk = (P.gptr[g + 1] - P.gptr[g]) / 8;
                for (int c = 0; c < nchk; ++c) {
                    const int pl = P.urows[P.gptr[g] + 8 * c] / 8;
                    auto it = std::lower_bound(w.begin() + lo_, w.begin() + hi_, pl);
                    if (it != w.begin() + hi_ && *it == pl) in.push_back({(int)(it - w.begin()) - lo_, c});
                }
                for (size_t q = 0; q < in.size(); q += 2) {
                    const int x = in[q].first, cx = in[q].second;
                    const int y = q + 1 < in.size() ? in[q + 1].first : CW;
                    const int cy = q + 1 < in.size() ? in[q + 1].second : -1;
                    if (cnt >= T->maxprog) fail(OMM_ERR_UNSUPPORTED, "spmm_tc2: stage program overflow");
                    prog[pt * T->maxprog + cnt++] = (uint16_t)((a << 12) | (x << 6) | y);
                    pairs.push_back(make_int4(g, cx, cy, 0));
                }
            }
            nprog[pt] = cnt;
        }
    }
    T->npairs = (int)pairs.size();
    auto up = [&](DevBuf& d, const void* src, size_t bytes) {
        d.alloc(std::max<size_t>(bytes, 16));
        OMM_CK(cudaMemcpyAsync(d.p, src, bytes, cudaMemcpyHostToDevice, rt().stream));
    };
    up(T->planes, planes.data(), planes.size() * sizeof(int));
    up(T->nchunks, nch.data(), nch.size() * sizeof(int));
    up(T->prog, prog.data(), prog.size() * sizeof(uint16_t));
    up(T->nprog, nprog.data(), nprog.size() * sizeof(int));
    up(T->bofs, bofs.data(), bofs.size() * sizeof(int));
    up(T->pairs, pairs.data(), pairs.size() * sizeof(int4));
    const size_t bt = (size_t)T->npairs * 2 * T->NB * 8 * sizeof(__nv_bfloat16);
    T->bt_hi.alloc(std::max<size_t>(bt, 16));
    T->bt_lo.alloc(std::max<size_t>(bt, 16));
    build_pairs_kernel<<<148 * 8, 256, 0, rt().stream>>>(T->npairs, T->G, T->NB, T->pairs.as<int4>(), P.d_gptr,
                                                         P.d_bvals, S ? PS->d_bvals : nullptr,
                                                         T->bt_hi.as<__nv_bfloat16>(), T->bt_lo.as<__nv_bfloat16>());
    OMM_KCHECK();
    OMM_CK(cudaStreamSynchronize(rt().stream));
    T->h_id = H->pattern_id;
    T->s_id = sid;
    if (nseg == 3) Hm->tc2_plan_split = Tn;
    else Hm->tc2_plan = Tn;
    return T;
}

// Y (FP32, n x m column-major, ld ldy; S's product at rows n..2n-1 when S given) = A [H, S]
// with A (n x m) given by its k-blocked bf16 shadow (hi[, lo]); optionally the row-major bf16
// shadows of Y (t_hi[, t_lo], row stride ldt).  false when the pattern cannot take it.
bool spmm_tc2(const __nv_bfloat16* Dk_hi, const __nv_bfloat16* Dk_lo, int n, int m, const msw_matrix* H,
              const msw_matrix* S, float* y, int ldy, __nv_bfloat16* t_hi, __nv_bfloat16* t_lo, int ldt, int nseg) {
    SpmmPlanView P = spmm_plan_view(H), PS;
    if (S) {
        if (!same_pattern(H, S)) return false;
        PS = spmm_plan_view(S);
    }
    SpmmTc2Plan* T = spmm_tc2_plan(H, P, S, S ? &PS : nullptr, nseg);
    if (!T) return false;
    if (m != H->dim1 || H->dim2 != m) fail(OMM_ERR_ARG, "spmm_tc2: dimensions differ");
    if (((uintptr_t)Dk_hi | (uintptr_t)Dk_lo | (uintptr_t)t_hi | (uintptr_t)t_lo) & 15)
        fail(OMM_ERR_ARG, "spmm_tc2: operands not 16-byte aligned");
    if (t_hi && ldt % 8) fail(OMM_ERR_ARG, "spmm_tc2: shadow row stride must be a multiple of 8");
    Tc2Params p{};
    p.n = n;
    p.G = T->G;
    p.NB = T->NB;
    p.GB = T->GB;
    p.ngroups = T->ngroups;
    p.nplanes = (m + 7) / 8;
    p.maxstages = T->maxstages;
    p.maxprog = T->maxprog;
    p.idesc = idesc_n(T->NB);
    p.a_hi = Dk_hi;
    p.a_lo = nseg == 3 ? Dk_lo : Dk_hi;
    p.b_hi = T->bt_hi.as<__nv_bfloat16>();
    p.b_lo = T->bt_lo.as<__nv_bfloat16>();
    p.planes = T->planes.as<int>();
    p.nchunks = T->nchunks.as<int>();
    p.prog = T->prog.as<uint16_t>();
    p.nprog = T->nprog.as<int>();
    p.bofs = T->bofs.as<int>();
    p.y = y;
    p.ldy = ldy;
    p.pair = S != nullptr;
    p.t_hi = t_hi;
    p.t_lo = t_lo;
    p.ldt = ldt;
    p.err = tc_error_flag();
    p.wc = tc_wait_cfg();
    const int nrb = (n + BMT - 1) / BMT;
    ktime_begin();
    if (nseg == 3) launch2<3, 4>(p, T->nblocks, nrb);
    else launch2<1, 8>(p, T->nblocks, nrb);
    // algorithmic bytes: the CSC operands (bf16 values, row indices, column pointers), A once,
    // the FP32 outputs
    const double nnz = (double)H->nnz, np_ = S ? 2.0 : 1.0;
    ktime_end("spmm_tc2_kernel", np_ * (nnz * (2 * (nseg == 3 ? 2 : 1) + 4) + (m + 1) * 4.0) +
                                     (double)n * m * 2 * (nseg == 3 ? 2 : 1) + np_ * (double)n * m * 4);
    return true;
}

namespace {
int g_spmm_groups = 1;  // column groups per CTA of the mixed step's SpMM: 1 (spmm_tc.cu) or 4 (here)
}

bool spmm_lowp_f32(const __nv_bfloat16* Dk_hi, const __nv_bfloat16* Dk_lo, int n, int m, const msw_matrix* H,
                   const msw_matrix* S, float* y, int ldy, __nv_bfloat16* t_hi, __nv_bfloat16* t_lo, int ldt, int nseg) {
    if (g_spmm_groups == 1) return spmm_tc_f32(Dk_hi, Dk_lo, n, m, H, S, y, ldy, t_hi, t_lo, ldt, nseg);
    return spmm_tc2(Dk_hi, Dk_lo, n, m, H, S, y, ldy, t_hi, t_lo, ldt, nseg);
}

}  // namespace ommgpu

extern "C" int omm_gpu_set_spmm_groups(int groups_per_cta) {
    if (groups_per_cta != 1 && groups_per_cta != 4) {
        ommgpu::set_last_error("omm_gpu_set_spmm_groups: 1 or 4 column groups per CTA");
        return OMM_ERR_ARG;
    }
    ommgpu::g_spmm_groups = groups_per_cta;
    ommgpu::set_last_error("");
    return OMM_OK;
}
