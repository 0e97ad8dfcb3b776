// BF16 tensor-core GEMM for sm_100a: tcgen05.mma with TMEM accumulators, fed by TMA.
//
//   out(M x N, FP64, column-major, ld) = alpha * sum_seg A_seg(M x K) * B_seg(N x K)^T + beta * out
//
// A and B are bf16, K-major (each row of M or N holds K contiguous values,
// row stride lda/ldb elements, a multiple of 8).  One segment is a plain BF16
// product; three segments (hi*hi, hi*lo, lo*hi of hi/lo bf16 splits of the
// operands) give a product accurate to ~2^-16 relative at three times the cost,
// accumulated in the same TMEM tile.
//
// CTA = one 128 x 256 output tile, 4 warps:
//   warp 0 lane 0   TMA producer: 64-wide K chunks of A (128 rows) and B (256
//                   rows) into a 4-stage ring of 128B-swizzled shared buffers,
//                   completion counted on full[s]
//   warp 1 lane 0   MMA issuer: 4 x tcgen05.mma (M128 N256 K16) per chunk into
//                   TMEM, tcgen05.commit frees the stage (empty[s]); a last
//                   commit signals the accumulator (acc)
//   warp 2          allocates / frees the 256 TMEM columns
//   warps 0-3       epilogue: tcgen05.ld 32 lanes x 32 columns at a time, each
//                   thread one row, coalesced column-major FP64 stores
// Every mbarrier wait gives up after ~2 s of global time, sets the error flag
// and lets the CTA drain (waits for its issued copies and MMAs, frees TMEM).
// gemm_bf16_pair_kernel below forms 256 x 256 tiles on pairs of SMs instead.
#include "internal.h"

#include <cuda.h>
#include <cudaTypedefs.h>

#include <cstdint>

#include "tc_ptx.h"

namespace ommgpu {

// rows x cols bf16 array (cols contiguous, row stride ld elements) as a 2D TMA tensor with a
// box of box_cols x box_rows; 128-byte swizzle or none.
CUtensorMap tma_map_bf16(const void* base, int rows, int cols, int ld, int box_cols, int box_rows, bool swizzle128);

// wait limit and test switch handed to every tcgen05 kernel (omm_gpu_tc_set_wait)
static tc::WaitCfg g_wait_cfg;
tc::WaitCfg tc_wait_cfg() { return g_wait_cfg; }

// whether the GEMMs run 256 x 256 tiles on SM pairs where the shape allows (omm_gpu_tc_set_pairs)
static bool g_pairs = true;
bool tc_pairs_enabled() { return g_pairs; }

// device word collecting the error bits of the bounded waits of every tcgen05 kernel
unsigned* tc_error_flag() {
    static DevBuf* flag = nullptr;
    if (!flag) {
        flag = new DevBuf();
        flag->alloc_zero(sizeof(unsigned));
    }
    return flag->as<unsigned>();
}

namespace tc {

constexpr int BM = 128, BN = 256, BK = 64, STAGES = 4;
constexpr int A_BYTES = BM * BK * 2;  // 16 KB
constexpr int B_BYTES = BN * BK * 2;  // 32 KB
constexpr int STAGE_BYTES = A_BYTES + B_BYTES;
constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + 1024 /*alignment slack*/ + 256 /*barriers*/;
constexpr uint32_t TMEM_COLS = 256;


struct Params {
    int M, N, K;  // K: columns per segment
    int nseg;     // 1 or 3
    double alpha, beta;
    double* out;
    int ldo;
    unsigned* err;
    int herm;  // > 0: the rows are Hermitian blocks of herm rows (herm % BM == 0); tiles wholly
               // below a block's diagonal are skipped (the caller mirrors the lower triangles)
    WaitCfg wc;
};

// The tile (mt, nt) of the launch's linear index L (x fastest): L walks groups of 8 tile rows
// column by column, so that the tiles in flight at one time share their A rows and B columns
// through L2 (a plain x-fastest order pairs each wave with one or two B columns only and reads
// every A row from memory once per column).
__device__ __forceinline__ void tile_of(int L, int nM, int nN, int& mt, int& nt) {
    constexpr int GROUP = 8;
    const int per = GROUP * nN, g = L / per, first = g * GROUP, size = min(GROUP, nM - first), r = L - g * per;
    mt = first + r % size;
    nt = r / size;
}

// shared memory matrix descriptor: K-major, 128B swizzle, 8-row groups 1024 B apart
__device__ __forceinline__ uint64_t make_desc(uint32_t saddr) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFF);          // start address
    d |= (uint64_t)(16 >> 4) << 16;                    // leading byte offset (unused for swizzled K-major)
    d |= (uint64_t)(1024 >> 4) << 32;                  // stride byte offset
    d |= (uint64_t)1 << 46;                            // descriptor version (sm_100)
    d |= (uint64_t)2 << 61;                            // SWIZZLE_128B
    return d;
}
// instruction descriptor: kind::f16, A/B bf16, FP32 accumulate, both K-major, M=128, N=256
constexpr uint32_t IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);

__device__ __forceinline__ void mma_f16(uint32_t tmem, uint64_t a, uint64_t b, uint32_t accumulate) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(
            tmem),
        "l"(a), "l"(b), "r"(IDESC), "r"(accumulate)
        : "memory");
}

__global__ void __launch_bounds__(128, 1) gemm_bf16_kernel(const __grid_constant__ CUtensorMap tA0,
                                                           const __grid_constant__ CUtensorMap tA1,
                                                           const __grid_constant__ CUtensorMap tB0,
                                                           const __grid_constant__ CUtensorMap tB1, Params p) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    uint8_t* sA = smem;
    uint8_t* sB = smem + STAGES * A_BYTES;
    uint64_t* bars = (uint64_t*)(smem + STAGES * STAGE_BYTES);
    uint64_t* full = bars;
    uint64_t* empty = bars + STAGES;
    uint64_t* accb = bars + 2 * STAGES;
    uint32_t* tmem_slot = (uint32_t*)(bars + 2 * STAGES + 1);
    volatile int* abort_flag = (volatile int*)(tmem_slot + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    int mt, nt;
    tile_of(blockIdx.y * gridDim.x + blockIdx.x, gridDim.x, gridDim.y, mt, nt);
    const int m0 = mt * BM, n0 = nt * BN;
    // every row of the tile below every column of it, in its Hermitian block: nothing to form
    // (uniform over the CTA, before any barrier or TMEM allocation)
    if (p.herm > 0 && m0 % p.herm > n0 + BN - 1) return;
    const int KT = (p.K + BK - 1) / BK;
    const int T = KT * p.nseg;

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(smem_u32(&full[s]), 1);
            mbar_init(smem_u32(&empty[s]), 1);
        }
        mbar_init(smem_u32(accb), 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tA0)) : "memory");
        asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tB0)) : "memory");
    }
    if (warp == 2) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;

    if (warp == 0 && lane == 0) {
        // ---------------- TMA producer (issues nothing under the withholding test switch)
        int issued = 0;
        const int T_issue = p.wc.withhold ? 0 : T;
        for (int t = 0; t < T_issue; ++t) {
            const int s = t % STAGES, r = t / STAGES;
            if (r > 0 && !mbar_wait(smem_u32(&empty[s]), (r - 1) & 1, p.wc.ns)) {
                atomicOr(p.err, 1u);
                *abort_flag = 1;
                break;
            }
            if (*abort_flag) break;
            const int seg = t / KT, kt = t % KT;
            const CUtensorMap* ma = (seg == 2) ? &tA1 : &tA0;
            const CUtensorMap* mb = (seg == 1) ? &tB1 : &tB0;
            const uint32_t fb = smem_u32(&full[s]);
            mbar_expect_tx(fb, STAGE_BYTES);
            tma_load_2d(smem_u32(sA + s * A_BYTES), ma, kt * BK, m0, fb);
            tma_load_2d(smem_u32(sB + s * B_BYTES), mb, kt * BK, n0, fb);
            issued = t + 1;
        }
        // drain: every issued copy must have landed before the CTA may exit
        for (int t = (issued > STAGES ? issued - STAGES : 0); t < issued; ++t) {
            if (!mbar_wait(smem_u32(&full[t % STAGES]), (t / STAGES) & 1, p.wc.ns)) {
                atomicOr(p.err, 2u);
                break;
            }
        }
    } else if (warp == 1 && lane == 0) {
        // ---------------- MMA issuer
        for (int t = 0; t < T; ++t) {
            const int s = t % STAGES, r = t / STAGES;
            if (!mbar_wait(smem_u32(&full[s]), r & 1, p.wc.ns)) {
                atomicOr(p.err, 4u);
                *abort_flag = 1;
                break;
            }
            if (*abort_flag) break;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t a0 = smem_u32(sA + s * A_BYTES), b0 = smem_u32(sB + s * B_BYTES);
#pragma unroll
            for (int kk = 0; kk < BK / 16; ++kk)
                mma_f16(tmem, make_desc(a0 + kk * 32), make_desc(b0 + kk * 32), (t > 0 || kk > 0) ? 1u : 0u);
            mma_commit(smem_u32(&empty[s]));
        }
        mma_commit(smem_u32(accb));  // arrives once every MMA issued above has completed
    }
    __syncwarp();

    // ---------------- epilogue: TMEM -> registers -> FP64 global
    const bool ok = mbar_wait(smem_u32(accb), 0, p.wc.ns);
    if (!ok) atomicOr(p.err, 8u);
    // the tcgen05.ld below is warp-collective: decide per warp
    const bool go = __all_sync(0xffffffffu, ok && !*abort_flag && T > 0);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (go) {
        const int row = m0 + warp * 32 + lane;
#pragma unroll 1
        for (int c0 = 0; c0 < BN; c0 += 32) {
            uint32_t v[32];
            const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0;
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
                "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
                : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                  "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]),
                  "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]),
                  "=r"(v[22]), "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]),
                  "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
                : "r"(taddr));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (row < p.M) {
#pragma unroll
                for (int q = 0; q < 32; ++q) {
                    const int col = n0 + c0 + q;
                    if (col < p.N) {
                        double* o = p.out + (size_t)row + (size_t)col * p.ldo;
                        double val = p.alpha * (double)__uint_as_float(v[q]);
                        if (p.beta != 0.0) val += p.beta * *o;
                        *o = val;
                    }
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 2) {
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
    }
}

// ---- the same product on SM pairs: a cluster of two CTAs forms one 256 x 256 tile with
// M256 N256 K16 MMAs (cta_group::2).  CTA r stages rows 128 r .. 128 r + 127 of the tile's A and
// of its B per 64-wide K chunk (16 KB + 16 KB, six stages), so each SM loads half the B bytes per
// MMA of the one-CTA kernel; its TMEM holds rows 128 r .. + 127 of the tile, all 256 columns.
// Rank 0 (the leader) posts the expected bytes of both halves on its full[s], issues the MMAs and
// commits to empty[s] and acc of both CTAs; both CTAs copy their halves (completion counted on
// the leader's full[s]) and run the epilogue of their own rows.  Waits are bounded as above; the
// pair meets at a cluster barrier before TMEM is freed.
constexpr int BM2 = 256, BN2 = 256, STAGES2 = 6;
constexpr int HALF_BYTES = 128 * BK * 2;            // 16 KB: 128 rows of a 64-wide bf16 K chunk
constexpr int STAGE2_BYTES = 2 * HALF_BYTES;        // this CTA's A half + B half
constexpr int SMEM2_BYTES = STAGES2 * STAGE2_BYTES + 1024 + 256;
constexpr uint32_t IDESC_PAIR =
    (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN2 >> 3) << 17) | ((uint32_t)(BM2 >> 4) << 24);

__device__ __forceinline__ void mma_f16_pair(uint32_t tmem, uint64_t a, uint64_t b, uint32_t accumulate) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n tcgen05.mma.cta_group::2.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(
            tmem),
        "l"(a), "l"(b), "r"(IDESC_PAIR), "r"(accumulate)
        : "memory");
}

__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(128, 1)
    gemm_bf16_pair_kernel(const __grid_constant__ CUtensorMap tA0, const __grid_constant__ CUtensorMap tA1,
                          const __grid_constant__ CUtensorMap tB0, const __grid_constant__ CUtensorMap tB1, Params p) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    uint8_t* sA = smem;
    uint8_t* sB = smem + STAGES2 * HALF_BYTES;
    uint64_t* bars = (uint64_t*)(smem + STAGES2 * STAGE2_BYTES);
    uint64_t* full = bars;               // [STAGES2] both halves landed (the leader's counts)
    uint64_t* empty = bars + STAGES2;    // [STAGES2] chunk consumed (each CTA's own)
    uint64_t* accb = bars + 2 * STAGES2; // every MMA of the tile completed (each CTA's own)
    uint32_t* tmem_slot = (uint32_t*)(bars + 2 * STAGES2 + 1);
    volatile int* abort_flag = (volatile int*)(tmem_slot + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t rank = cluster_rank();
    const bool leader = rank == 0;
    int mt, nt;  // the pair's tile: both CTAs of the cluster compute the same one
    tile_of(blockIdx.y * (gridDim.x >> 1) + (blockIdx.x >> 1), gridDim.x >> 1, gridDim.y, mt, nt);
    const int m0 = mt * BM2, n0 = nt * BN2;
    // the whole pair tile below its Hermitian block's diagonal: both CTAs leave before any barrier
    if (p.herm > 0 && m0 % p.herm > n0 + BN2 - 1) return;
    const int KT = (p.K + BK - 1) / BK;
    const int T = KT * p.nseg;

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES2; ++s) {
            mbar_init(smem_u32(&full[s]), 1);
            mbar_init(smem_u32(&empty[s]), 1);
        }
        mbar_init(smem_u32(accb), 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tA0)) : "memory");
        asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tB0)) : "memory");
    }
    if (warp == 2) tmem_alloc_pair(smem_u32(tmem_slot), TMEM_COLS);
    fence_before();
    cluster_sync();
    fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp == 0 && lane == 0) {
        // ---------------- TMA producer of this CTA's halves (nothing under the withholding switch)
        const uint32_t lead_full0 = peer_addr(smem_u32(&full[0]), 0);
        int issued = 0;
        const int T_issue = p.wc.withhold ? 0 : T;
        for (int t = 0; t < T_issue; ++t) {
            const int s = t % STAGES2, r = t / STAGES2;
            if (r > 0 && !mbar_wait_cl(smem_u32(&empty[s]), (r - 1) & 1, p.wc.ns)) {
                atomicOr(p.err, 1u);
                *abort_flag = 1;
                break;
            }
            if (*abort_flag) break;
            const int seg = t / KT, kt = t % KT;
            const CUtensorMap* ma = (seg == 2) ? &tA1 : &tA0;
            const CUtensorMap* mb = (seg == 1) ? &tB1 : &tB0;
            const uint32_t fb = lead_full0 + (uint32_t)(s * sizeof(uint64_t));
            if (leader) mbar_expect_tx(smem_u32(&full[s]), 2 * STAGE2_BYTES);
            tma_load_2d_pair(smem_u32(sA + s * HALF_BYTES), ma, kt * BK, m0 + 128 * (int)rank, fb);
            tma_load_2d_pair(smem_u32(sB + s * HALF_BYTES), mb, kt * BK, n0 + 128 * (int)rank, fb);
            issued = t + 1;
        }
        // the last chunks issued: landed (leader's full[s]) or consumed (the follower's empty[s])
        for (int t = (issued > STAGES2 ? issued - STAGES2 : 0); t < issued; ++t) {
            const bool ok = leader ? mbar_wait_cl(smem_u32(&full[t % STAGES2]), (t / STAGES2) & 1, p.wc.ns)
                                   : mbar_wait_cl(smem_u32(&empty[t % STAGES2]), (t / STAGES2) & 1, p.wc.ns);
            if (!ok) {
                atomicOr(p.err, 2u);
                break;
            }
        }
    } else if (warp == 1 && lane == 0 && leader) {
        // ---------------- MMA issuer (leader only)
        for (int t = 0; t < T; ++t) {
            const int s = t % STAGES2, r = t / STAGES2;
            if (!mbar_wait_cl(smem_u32(&full[s]), r & 1, p.wc.ns)) {
                atomicOr(p.err, 4u);
                *abort_flag = 1;
                break;
            }
            if (*abort_flag) break;
            fence_after();
            const uint32_t a0 = smem_u32(sA + s * HALF_BYTES), b0 = smem_u32(sB + s * HALF_BYTES);
#pragma unroll
            for (int kk = 0; kk < BK / 16; ++kk)
                mma_f16_pair(tmem, make_desc(a0 + kk * 32), make_desc(b0 + kk * 32), (t > 0 || kk > 0) ? 1u : 0u);
            mma_commit_pair(smem_u32(&empty[s]), 3);
        }
        mma_commit_pair(smem_u32(accb), 3);  // arrives in both CTAs once every MMA above completed
    }
    __syncwarp();

    // ---------------- epilogue: this CTA's 128 rows, TMEM -> registers -> FP64 global
    const bool ok = mbar_wait_cl(smem_u32(accb), 0, p.wc.ns);
    if (!ok) {
        atomicOr(p.err, 8u);
        *abort_flag = 1;
    }
    // the leader commits acc even after giving up (its MMAs must be known complete before TMEM
    // is freed), so each CTA takes the other's abort state too, across a cluster barrier
    fence_before();
    cluster_sync();
    fence_after();
    const bool peer_abort = ld_cluster_u32(peer_addr(smem_u32((const void*)abort_flag), rank ^ 1u)) != 0;
    const bool go = __all_sync(0xffffffffu, ok && !*abort_flag && !peer_abort && T > 0);
    if (go) {
        const int row = m0 + 128 * (int)rank + warp * 32 + lane;
#pragma unroll 1
        for (int c0 = 0; c0 < BN2; c0 += 32) {
            uint32_t v[32];
            tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
            if (row < p.M) {
#pragma unroll
                for (int q = 0; q < 32; ++q) {
                    const int col = n0 + c0 + q;
                    if (col < p.N) {
                        double* o = p.out + (size_t)row + (size_t)col * p.ldo;
                        double val = p.alpha * (double)__uint_as_float(v[q]);
                        if (p.beta != 0.0) val += p.beta * *o;
                        *o = val;
                    }
                }
            }
        }
    }
    fence_before();
    __syncthreads();
    cluster_sync();  // no MMA, copy or arrival of either CTA still targets the other
    fence_after();
    if (warp == 2) tmem_dealloc_pair(tmem, TMEM_COLS);
}

// ------------------------------------------------------------------ host side
PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        OMM_CK(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q));
        if (q != cudaDriverEntryPointSuccess || !p) fail(OMM_ERR_CUDA, "cuTensorMapEncodeTiled is not available");
        fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
    }
    return fn;
}

// rows x cols bf16, K-major (cols contiguous, row stride ld elements), box = box_rows x 64, 128B swizzle
CUtensorMap make_map(const void* base, int rows, int cols, int ld, int box_rows) {
    return tma_map_bf16(base, rows, cols, ld, BK, box_rows, true);
}

unsigned* err_flag() { return tc_error_flag(); }

}  // namespace tc

CUtensorMap tma_map_bf16(const void* base, int rows, int cols, int ld, int box_cols, int box_rows, bool swizzle128) {
    CUtensorMap m;
    cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)ld * 2};
    cuuint32_t box[2] = {(cuuint32_t)box_cols, (cuuint32_t)box_rows};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = tc::encode_fn()(&m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims, strides, box,
                                 estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                                 swizzle128 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_NONE,
                                 CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) fail(OMM_ERR_CUDA, "cuTensorMapEncodeTiled failed with " + std::to_string((int)r));
    return m;
}

// out (FP64, M x N, column-major, ldo) = alpha * sum_seg A_seg B_seg^T + beta * out.
// nseg = 1: A_hi B_hi^T.  nseg = 3: A_hi B_hi^T + A_hi B_lo^T + A_lo B_hi^T.
void gemm_bf16_tn(int M, int N, int K, const __nv_bfloat16* A_hi, const __nv_bfloat16* A_lo, int lda,
                  const __nv_bfloat16* B_hi, const __nv_bfloat16* B_lo, int ldb, int nseg, double alpha, double beta,
                  double* out, int ldo, int herm) {
    using namespace tc;
    if (M <= 0 || N <= 0) return;
    if (herm < 0 || (herm > 0 && (herm % BM || M % herm))) fail(OMM_ERR_ARG, "gemm_bf16: bad Hermitian block size");
    if (K <= 0) fail(OMM_ERR_ARG, "gemm_bf16: K must be positive");
    if (lda % 8 || ldb % 8 || lda < K || ldb < K) fail(OMM_ERR_ARG, "gemm_bf16: lda/ldb must be >= K and multiples of 8");
    if (((uintptr_t)A_hi | (uintptr_t)B_hi) & 15) fail(OMM_ERR_ARG, "gemm_bf16: operands must be 16-byte aligned");
    if (nseg != 1 && nseg != 3) fail(OMM_ERR_ARG, "gemm_bf16: nseg must be 1 or 3");
    if (nseg == 3 && (!A_lo || !B_lo || (((uintptr_t)A_lo | (uintptr_t)B_lo) & 15)))
        fail(OMM_ERR_ARG, "gemm_bf16: split operands missing or misaligned");
    // SM pairs (256 x 256 tiles) unless a Hermitian block would split a pair's rows
    const bool pairs = tc_pairs_enabled() && M > BM && (herm == 0 || herm % BM2 == 0);
    const int brows = pairs ? 128 : BN;
    CUtensorMap a0 = make_map(A_hi, M, K, lda, BM), b0 = make_map(B_hi, N, K, ldb, brows);
    CUtensorMap a1 = nseg == 3 ? make_map(A_lo, M, K, lda, BM) : a0;
    CUtensorMap b1 = nseg == 3 ? make_map(B_lo, N, K, ldb, brows) : b0;
    static bool attr = false;
    if (!attr) {
        OMM_CK(cudaFuncSetAttribute(gemm_bf16_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES));
        OMM_CK(cudaFuncSetAttribute(gemm_bf16_pair_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM2_BYTES));
        attr = true;
    }
    Params p{M, N, K, nseg, alpha, beta, out, ldo, err_flag(), herm, tc_wait_cfg()};
    ktime_begin();
    if (pairs) {
        dim3 grid(2 * ((M + BM2 - 1) / BM2), (N + BN2 - 1) / BN2);
        gemm_bf16_pair_kernel<<<grid, 128, SMEM2_BYTES, rt().stream>>>(a0, a1, b0, b1, p);
    } else {
        dim3 grid((M + BM - 1) / BM, (N + BN - 1) / BN);
        gemm_bf16_kernel<<<grid, 128, SMEM_BYTES, rt().stream>>>(a0, a1, b0, b1, p);
    }
    OMM_KCHECK();
    ktime_end(pairs ? "gemm_bf16_pair_kernel" : "gemm_bf16_kernel",
              2.0 * M * N * (double)K * nseg / (herm > 0 ? 2.0 : 1.0));
}

// error bits of the bounded waits since the last call (and clears them)
unsigned gemm_bf16_errors() {
    unsigned h = 0;
    OMM_CK(cudaMemcpyAsync(&h, tc::err_flag(), sizeof(unsigned), cudaMemcpyDeviceToHost, rt().stream));
    OMM_CK(cudaStreamSynchronize(rt().stream));
    if (h) OMM_CK(cudaMemsetAsync(tc::err_flag(), 0, sizeof(unsigned), rt().stream));
    return h;
}

}  // namespace ommgpu

using namespace ommgpu;

extern "C" int omm_gpu_tc_set_wait(unsigned long long wait_ns, int withhold_copies) {
    if (wait_ns == 0) {
        set_last_error("omm_gpu_tc_set_wait: the wait limit must be positive");
        return OMM_ERR_ARG;
    }
    g_wait_cfg.ns = wait_ns;
    g_wait_cfg.withhold = withhold_copies ? 1 : 0;
    set_last_error("");
    return OMM_OK;
}

extern "C" int omm_gpu_tc_set_pairs(int on) {
    g_pairs = on != 0;
    set_last_error("");
    return OMM_OK;
}

extern "C" int omm_gpu_gemm_bf16_async(int M, int N, int K, const void* A_hi, const void* A_lo, int lda,
                                       const void* B_hi, const void* B_lo, int ldb, int nseg, double alpha,
                                       double beta, double* out, int ldo) {
    try {
        gemm_bf16_tn(M, N, K, (const __nv_bfloat16*)A_hi, (const __nv_bfloat16*)A_lo, lda, (const __nv_bfloat16*)B_hi,
                     (const __nv_bfloat16*)B_lo, ldb, nseg, alpha, beta, out, ldo);
    } catch (const Error& e) {
        set_last_error(e.msg);
        return e.code;
    }
    set_last_error("");
    return OMM_OK;
}

extern "C" int omm_gpu_gemm_bf16(int M, int N, int K, const void* A_hi, const void* A_lo, int lda, const void* B_hi,
                                 const void* B_lo, int ldb, int nseg, double alpha, double beta, double* out, int ldo) {
    try {
        gemm_bf16_tn(M, N, K, (const __nv_bfloat16*)A_hi, (const __nv_bfloat16*)A_lo, lda, (const __nv_bfloat16*)B_hi,
                     (const __nv_bfloat16*)B_lo, ldb, nseg, alpha, beta, out, ldo);
        unsigned e = gemm_bf16_errors();
        if (e) fail(OMM_ERR_CUDA, "gemm_bf16: a pipeline wait timed out (error bits " + std::to_string(e) + ")");
    } catch (const Error& e) {
        set_last_error(e.msg);
        return e.code;
    }
    set_last_error("");
    return OMM_OK;
}
