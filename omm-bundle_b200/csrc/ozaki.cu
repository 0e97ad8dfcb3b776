// FP64 matrix products on the int8 tensor cores (tcgen05 .kind::i8) by modular arithmetic.
//
//   out (M x N, FP64, column-major) = alpha * A_op(M x K) * B_op(N x K)^T + beta * out
//
// Method: the integer-modular emulation of floating-point GEMM (Ozaki, Uchino and Imamura,
// "Ozaki Scheme II: A GEMM-oriented emulation of floating-point matrix multiplication using
// an integer modular technique", 2024/2025), written here from its mathematics:
//   1. every row r of A_op is scaled by a power of two so that its largest entry has `bits`
//      significant bits, and rounded to integers: A'(r, k) = rint(A(r, k) 2^(bits-1-e_r)) with
//      e_r = floor(log2 max_k |A(r, k)|); likewise B'.  |A'| <= 2^bits, |B'| <= 2^bits.
//   2. The integer product C' = A' B'^T is exact in Z and |C'| <= K 2^(bitsA+bitsB).  It is
//      computed modulo nmod pairwise coprime moduli p_l <= 256 (their product P exceeding
//      4 |C'|): the residues A' mod p_l, B' mod p_l, in the symmetric range [-128, 127], are
//      int8 operands, and one int8 GEMM per modulus accumulates exactly in int32
//      (K * 128^2 < 2^31 for K < 2^17); its epilogue reduces the result mod p_l to a byte.
//   3. The Chinese remainder theorem rebuilds C' from its residues r_l:
//          C' = sum_l r_l W_l - q P,   W_l = (P/p_l) ((P/p_l)^-1 mod p_l),
//      with q = round(sum_l r_l W_l / P) taken from FP64 sums of r_l (W_l / P) (exact, since
//      C'/P is at most 1/4 away from an integer), and the sum formed modulo 2^128 in 32-bit
//      limbs; C' (|C'| < 2^126) is converted to FP64 and scaled back by 2^(e_r + e_c - ...).
// With 16 moduli (P ~ 2^125.4) both operands keep 53 bits for any K < 2^17: the result is
// the exact product of the operands rounded to 53 bits relative to their row maxima, rounded
// once to FP64 -- the accuracy class of an FP64 GEMM.  The int8 GEMMs run at the tensor
// cores' int8 rate (twice the bf16 rate), i.e. 16 of them cost about 8 bf16 GEMMs.
//
// Layouts: the int8 residue operands are K-major planes (plane l = rows x ldk bytes), read by
// 3D TMA boxes of 128 x 128 B into the 128-byte-swizzled shared layout tcgen05 reads; the
// product's residues are column-major byte planes.  Operand sources are FP64 column-major
// matrices read either with the rows contiguous (a transposing pass) or with K contiguous.
#include "internal.h"

#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <memory>
#include <tuple>
#include <vector>

#include "tc_ptx.h"

namespace ommgpu {

unsigned* tc_error_flag();
tc::WaitCfg tc_wait_cfg();
bool tc_pairs_enabled();
namespace tc {
PFN_cuTensorMapEncodeTiled_v12000 encode_fn();
}

namespace oz {

constexpr int MAXMOD = 16;
// pairwise coprime moduli <= 256 (256 = 2^8, 255 = 3*5*17, 253 = 11*23, 247 = 13*19,
// 217 = 7*31, the rest prime), largest first
constexpr int kMods[MAXMOD] = {256, 255, 253, 251, 247, 241, 239, 233, 229, 227, 223, 217, 211, 199, 197, 193};
constexpr int ZERO_EXP = -2139062144;  // 0x80808080: the exponent of an all-zero row (memset 0x80)
constexpr int BAD_EXP = 1 << 30;       // a row holding NaN or Inf
constexpr int MAX_K = (1 << 17) - 1;   // K * 128^2 < 2^31: exact int32 accumulation

struct Table {
    int nmod = 0;
    int p[MAXMOD];
    double inv_p[MAXMOD];
    uint32_t W[MAXMOD][4];  // W_l in 32-bit limbs, least significant first
    double w[MAXMOD];       // W_l / P
    uint32_t P[4];          // P = prod p_l in limbs
    double log2P = 0;
};

typedef unsigned __int128 u128;

Table make_table(int nmod) {
    Table t{};
    t.nmod = nmod;
    u128 P = 1;
    for (int l = 0; l < nmod; ++l) P *= (u128)kMods[l];
    for (int l = 0; l < nmod; ++l) {
        const int p = kMods[l];
        t.p[l] = p;
        t.inv_p[l] = 1.0 / p;
        const u128 Pl = P / (u128)p;
        const int a = (int)(Pl % (u128)p);
        int inv = 0;
        for (int x = 1; x < p; ++x)
            if ((a * x) % p == 1) {
                inv = x;
                break;
            }
        const u128 W = Pl * (u128)inv;  // < P since inv < p
        for (int q = 0; q < 4; ++q) t.W[l][q] = (uint32_t)(W >> (32 * q));
        t.w[l] = (double)((long double)W / (long double)P);
    }
    for (int q = 0; q < 4; ++q) t.P[q] = (uint32_t)(P >> (32 * q));
    t.log2P = (double)log2l((long double)P);
    return t;
}

const Table& table(int nmod) {
    static Table t[MAXMOD + 1];
    static bool init = false;
    if (!init) {
        for (int n = 1; n <= MAXMOD; ++n) t[n] = make_table(n);
        init = true;
    }
    return t[nmod];
}

struct ModParams {
    int nmod;
    int p[MAXMOD];
    uint32_t c18[MAXMOD], c36[MAXMOD];  // 2^18 mod p, 2^36 mod p
    uint32_t off[MAXMOD];               // a multiple of p >= 2^25
    uint32_t half[MAXMOD];              // (p - 1) / 2: the symmetric residues lie in [-half, p - 1 - half]
    uint32_t magic[MAXMOD];             // ceil(2^39 / p): u / p = umulhi(u, magic) >> 7 for u < 2^28
};

// The residue kernels' constants: x (|x| <= 2^53) is taken as x + 2^53 = hi 2^32 + lo (seven bytes),
// and for p_l != 256
struct ModB {
    uint32_t wlo[MAXMOD], whi[MAXMOD];  // the bytes 256^k mod p_l for k = 0..3 and k = 4..6
    uint32_t e[MAXMOD];                 // p_l - (2^53 mod p_l)
    uint32_t negp[MAXMOD];              // -p_l (two's complement)
    uint32_t magic[MAXMOD];             // ceil(2^39 / p_l)
    unsigned long long mh[MAXMOD];      // magic * (p_l - 1) / 2
};

// ------------------------------------------------------------------ row exponents
// rows contiguous in the source (element (r, k) at A[r + k lda]): one thread per row over a
// 256-column slab, combined across slabs with atomicMax; the loads go out 16 at a time so that
// enough bytes are in flight to cover the memory latency
__global__ void __launch_bounds__(256) oz_exp_rows_kernel(int R, int K, const double* __restrict__ A, int rs,
                                                          int lda, int* __restrict__ e) {
    const int r = blockIdx.x * 256 + threadIdx.x;
    const int k0 = blockIdx.y * 256, k1 = min(K, k0 + 256);
    if (r >= R) return;
    double mx = 0.0;
    bool bad = false;
    for (int kb = k0; kb < k1; kb += 16) {
        double v[16];
#pragma unroll
        for (int u = 0; u < 16; ++u) {
            const int k = kb + u;
            v[u] = k < k1 ? A[(size_t)r * rs + (size_t)k * lda] : 0.0;
        }
#pragma unroll
        for (int u = 0; u < 16; ++u) {
            const double a = fabs(v[u]);
            bad |= !(a <= 1.7976931348623157e308);
            mx = fmax(mx, a);
        }
    }
    if (bad) atomicMax(&e[r], BAD_EXP);
    else if (mx > 0.0) atomicMax(&e[r], ilogb(mx));
}

// K contiguous in the source (element (r, k) at A[k + r lda]): one warp per row
__global__ void __launch_bounds__(256) oz_exp_kc_kernel(int R, int K, const double* __restrict__ A, int rs, int lda,
                                                        int* __restrict__ e) {
    const int r = blockIdx.x * 8 + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    if (r >= R) return;
    const double* a = A + (size_t)r * lda;
    double mx = 0.0;
    bool bad = false;
    for (int k = lane; k < K; k += 32) {
        const double v = fabs(a[(size_t)k * rs]);
        bad |= !(v <= 1.7976931348623157e308);
        mx = fmax(mx, v);
    }
    for (int o = 16; o > 0; o >>= 1) {
        mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        bad |= __shfl_xor_sync(0xffffffffu, (int)bad, o) != 0;
    }
    if (lane == 0) e[r] = bad ? BAD_EXP : (mx > 0.0 ? ilogb(mx) : ZERO_EXP);
}

// y = beta y + alpha x over R x K (rows contiguous: element (r, k) at y[r + k ldy], x likewise;
// the same arithmetic as the library's axpby) with the exponents that oz_prepare would form of the
// result's rows (erow, the row-contiguous operand) and columns (ecol, the K-contiguous operand of
// its transpose), atomicMax'ed into arrays preset to ZERO_EXP.  The matrix is walked in memory
// order, as a plain axpby would: warp gw of W takes the 128-row column chunks q = gw, gw + W, ...
// (q = k nrb + rb; W a multiple of nrb, so a warp keeps one row block rb and the warps at work
// cover a compact window of the matrix), lane l the rows 128 rb + l + 32 u.  The largest |y| of a
// chunk is the largest IEEE bit pattern (NaN and Inf above every finite value), reduced exactly over
// the warp in two 32-bit halves (the low half only when no normal value decides it); the rows'
// largest bit patterns are kept over the warp's chunks and go out once at its end.
constexpr int AX_WR = 128;
__device__ __forceinline__ int oz_exp_of_bits(unsigned long long b) {
    const double c = __longlong_as_double((long long)b);
    if (!(c <= 1.7976931348623157e308)) return BAD_EXP;
    return c > 0.0 ? ilogb(c) : ZERO_EXP;
}
__global__ void __launch_bounds__(256) oz_axpby_exps_kernel(int R, int K, double alpha, const double* __restrict__ x,
                                                            int ldx, double beta, double* __restrict__ y, int ldy,
                                                            int W, int* __restrict__ erow, int* __restrict__ ecol) {
    const int lane = threadIdx.x & 31;
    const int gw = blockIdx.x * 8 + (threadIdx.x >> 5);
    if (gw >= W) return;
    const int nrb = (R + AX_WR - 1) / AX_WR;
    const long long nch = (long long)nrb * K;
    const int rb = gw % nrb;
    unsigned long long rk[4] = {0, 0, 0, 0};
    for (long long q = gw; q < nch; q += W) {
        const int k = (int)(q / nrb);
        double v[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int r = rb * AX_WR + lane + 32 * u;
            if (r < R) {
                const double a = x[(size_t)r + (size_t)k * ldx];
                const double c = beta * y[(size_t)r + (size_t)k * ldy];
                v[u] = c + alpha * a;
            } else {
                v[u] = 0.0;
            }
        }
        unsigned long long ck = 0;
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int r = rb * AX_WR + lane + 32 * u;
            if (r < R) y[(size_t)r + (size_t)k * ldy] = v[u];
            const unsigned long long key = (unsigned long long)__double_as_longlong(fabs(v[u]));
            rk[u] = max(rk[u], key);
            ck = max(ck, key);
        }
        if (ecol) {
            const unsigned hi = __reduce_max_sync(0xffffffffu, (unsigned)(ck >> 32));
            unsigned lo = 0;
            if (hi < 0x00100000u)  // no normal value in the chunk: the low half decides
                lo = __reduce_max_sync(0xffffffffu, (unsigned)(ck >> 32) == hi ? (unsigned)ck : 0u);
            const unsigned long long m = ((unsigned long long)hi << 32) | lo;
            if (lane == 0 && m != 0) atomicMax(&ecol[k], oz_exp_of_bits(m));
        }
    }
    if (erow) {
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int r = rb * AX_WR + lane + 32 * u;
            if (r < R && rk[u] != 0) atomicMax(&erow[r], oz_exp_of_bits(rk[u]));
        }
    }
}

// ------------------------------------------------------------------ residues
// 2^s as a double for -1022 <= s <= 1023 (built from its exponent field)
__device__ __forceinline__ double pow2(int s) { return __hiloint2double((s + 1023) << 20, 0); }
// the two power-of-two factors whose product scales a row with largest-entry exponent e to
// `bits` significant bits (split so that each stays a normal double for any FP64 row)
__device__ __forceinline__ void oz_scales(int e, int bits, double& f1, double& f2) {
    if (e == ZERO_EXP || e == BAD_EXP) {
        f1 = f2 = 0.0;
        return;
    }
    const int s = bits - 1 - e, s1 = s / 2;
    f1 = pow2(s1);
    f2 = pow2(s - s1);
}
// an entry scaled by two exact powers of two; rounding it to the integer A'(r, k) is left to the
// conversion in oz_limbs (round to nearest even, like rint)
__device__ __forceinline__ double oz_integer(double v, double f1, double f2) { return (v * f1) * f2; }
// A'(r, k) = rint(x) (|x| <= 2^53) as three limbs a 2^36 + b 2^18 + c, b and c in [0, 2^18)
struct Limbs {
    int a, b, c;
};
__device__ __forceinline__ Limbs oz_limbs(double x) {
    const long long v = __double2ll_rn(x);
    return {(int)(v >> 36), (int)((v >> 18) & 0x3FFFF), (int)(v & 0x3FFFF)};
}
// x mod p in [-128, 127] in exact integer arithmetic: t = a (2^36 mod p) + b (2^18 mod p) + c is
// congruent to x with -2^25 < t < 2^26.6, so u = t + off is in [0, 2^27.1); with
// q = floor((u + half) / p), u - q p is the residue in [-half, p - 1 - half].  The quotient of
// v < 2^28 by p is umulhi(v, ceil(2^39 / p)) >> 7 exactly (its error is below 2^-11 < 1/p).
// For p = 256 (the first modulus) the residue is the low byte of x, i.e. of c.
__device__ __forceinline__ int oz_residue(const Limbs& x, const ModParams& mp, int l) {
    const uint32_t u = (uint32_t)(x.a * (int)mp.c36[l] + x.b * (int)mp.c18[l] + x.c) + mp.off[l];
    const uint32_t q = __umulhi(u + mp.half[l], mp.magic[l]) >> 7;
    return (int)(u - q * (uint32_t)mp.p[l]);
}
// The same residue from x + 2^53 = hi 2^32 + lo, in fewer operations: s = sum_k b_k (256^k mod p)
// over its seven bytes b_k is two byte dot products (s < 7 * 255^2 < 2^19), u = s + e == x (mod p)
// with u >= 0, q = floor((u + half) / p) = (u magic + half magic) >> 39 exactly (one 32 x 32 + 64
// multiply-add; the quotient rule above, applied to u + half < 2^20), and r = u - q p in
// [-half, p - 1 - half] -- the residue oz_residue gives.  p = 256 takes the low byte of x.
__device__ __forceinline__ uint32_t oz_resb(uint32_t lo, uint32_t hi, const ModB& mb, int l) {
    if (l == 0) return lo;
    const uint32_t u = __dp4a(hi, mb.whi[l], __dp4a(lo, mb.wlo[l], mb.e[l]));
    const uint32_t q = (uint32_t)(((unsigned long long)u * mb.magic[l] + mb.mh[l]) >> 39);
    return u + q * mb.negp[l];
}
// the 16 moduli's words of four consecutive entries (x + 2^53 as lo / hi words), stored one plane
// apart at dst and, when d2 is set, one kb plane apart at d2
__device__ __forceinline__ void oz_store_planes_b(uint32_t* dst, size_t plane_words, uint32_t* d2, size_t kb_words,
                                                  const uint32_t (&lo)[4], const uint32_t (&hi)[4], const ModB& mb) {
#pragma unroll
    for (int l = 0; l < MAXMOD; ++l) {
        uint32_t r[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) r[u] = oz_resb(lo[u], hi[u], mb, l);
        const uint32_t w = __byte_perm(__byte_perm(r[0], r[1], 0x0040), __byte_perm(r[2], r[3], 0x0040), 0x5410);
        *dst = w;
        dst += plane_words;
        if (d2) {
            *d2 = w;
            d2 += kb_words;
        }
    }
}

// Both residue kernels give every lane four consecutive k of one row, so that each store of a
// warp covers whole 32-byte sectors of a plane (the K-major planes are the GEMM's operands).  They
// form all 16 moduli (the only count the products use).
//
// Rows contiguous in the source (element (r, k) at A[r + k lda]): a CTA transposes a tile of
// 32 rows x 128 k through shared memory.  Loading, warp w reads k0 + 16 w .. + 15 for the 32 rows
// (each read coalesced over the rows; all sixteen loads of a lane first) and stores x + 2^53 of
// the rounded integers.  The tile keeps entry (row, k) at row * RT_LD + k + k / 4, so that the
// loads' stores (one k, 32 rows: RT_LD odd) and the lanes' reads (one row, k = 4 j + u:
// 5 j + u) fall in distinct banks.  Computing, without the k-blocked copy warp w takes rows
// 4 w .. 4 w + 3 and lane j the k 4 j .. 4 j + 3 of each (a 128-byte line of a plane per store).
// With it (KB), warp w takes rows 8 (w / 2) .. + 7 and k 64 (w % 2) .. + 63, lane j the row
// parity j / 16 and the k 4 (j % 16) .. + 3: each store then covers two adjacent rows of four
// 16-k chunks, i.e. whole 32-byte sectors of the k-blocked planes too (the other mapping wrote
// them half at a time, which cost partial-sector writes and re-reads).
constexpr int RT_ROWS = 32, RT_K = 128, RT_LD = RT_K + RT_K / 4 + 1;  // 161
// The k-blocked copy (the int8 SpMM's A operand): plane l at kb + l kb_plane holds, per block of
// 256 rows, its nch16 chunks of 16 k, each 256 rows x 16 B.
template <bool KB>
__global__ void __launch_bounds__(256) oz_res_rows_kernel(int R, int K, const double* __restrict__ A, int rs, int lda,
                                                          const int* __restrict__ e, int bits, int8_t* __restrict__ out,
                                                          int ldk, size_t plane, const __grid_constant__ ModB mb,
                                                          uint8_t* __restrict__ kb, size_t kb_plane, int nch16,
                                                          int kbh) {
    __shared__ long long tile[RT_ROWS * RT_LD];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int r0 = blockIdx.x * RT_ROWS, k0 = blockIdx.y * RT_K;
    {
        const int r = r0 + lane;
        double v[16];
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            const int k = k0 + 16 * warp + j;
            v[j] = (r < R && k < K) ? A[(size_t)r * rs + (size_t)k * lda] : 0.0;
        }
        double f1 = 0.0, f2 = 0.0;
        if (r < R) oz_scales(e[r], bits, f1, f2);
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            const int kk = 16 * warp + j;
            tile[lane * RT_LD + kk + kk / 4] = __double2ll_rn(oz_integer(v[j], f1, f2)) + (1ll << 53);
        }
    }
    __syncthreads();
    const int kk = KB ? 64 * (warp & 1) + 4 * (lane & 15) : 4 * lane, k = k0 + kk;
    if (k >= ldk) return;  // past the padded row (ldk is a multiple of 16)
#pragma unroll 1
    for (int i = 0; i < 4; ++i) {
        const int rr = KB ? 8 * (warp >> 1) + (lane >> 4) + 2 * i : 4 * warp + i, r = r0 + rr;
        if (r >= R) break;
        uint32_t lo[4], hi[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const unsigned long long v = (unsigned long long)tile[rr * RT_LD + kk + kk / 4 + u];
            lo[u] = (uint32_t)v;
            hi[u] = (uint32_t)(v >> 32);
        }
        uint32_t* dst = reinterpret_cast<uint32_t*>(out + (size_t)r * ldk + k);
        // chunk (k / 16) of the 256-row block r / 256: 256 rows x 16 B, or (kbh, the SM-pair form's
        // half-major layout) per 128-row half of the block its chunks of 128 rows x 16 B
        const size_t kbo = kbh ? ((((size_t)(r / 256) * 2 + (r % 256) / 128) * nch16 + (k >> 4)) * 128 + (r % 128)) * 16
                               : (((size_t)(r / 256) * nch16 + (k >> 4)) * 256 + (r % 256)) * 16;
        uint32_t* d2 = KB ? reinterpret_cast<uint32_t*>(kb + kbo + (k & 15)) : nullptr;
        oz_store_planes_b(dst, plane / 4, d2, kb_plane / 4, lo, hi, mb);
    }
}

// K contiguous in the source (element (r, k) at A[k + r lda]): warp w of a CTA takes row
// 8 blockIdx.x + w, lane j the k 4 j .. 4 j + 3 of each 128-k slab of the CTA's 512
__global__ void __launch_bounds__(256) oz_res_kc_kernel(int R, int K, const double* __restrict__ A, int rs, int lda,
                                                        const int* __restrict__ e, int bits, int8_t* __restrict__ out,
                                                        int ldk, size_t plane, const __grid_constant__ ModB mb) {
    const int r = blockIdx.x * 8 + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    if (r >= R) return;
    double f1, f2;
    oz_scales(e[r], bits, f1, f2);
    const double* a = A + (size_t)r * lda;
    const int kb = blockIdx.y * 512 + 4 * lane;
    // all sixteen loads first (four slabs of 128 k), then the residues slab by slab; a lane's four
    // consecutive k are two 16-byte loads where the row is contiguous and 16-byte aligned
    double v[4][4];
    const bool vec = rs == 1 && ((reinterpret_cast<uintptr_t>(a) & 15) == 0);
#pragma unroll
    for (int s = 0; s < 4; ++s) {
        const int k = kb + 128 * s;
        if (vec && k + 3 < K) {
            const double2 x0 = *reinterpret_cast<const double2*>(a + k);
            const double2 x1 = *reinterpret_cast<const double2*>(a + k + 2);
            v[s][0] = x0.x;
            v[s][1] = x0.y;
            v[s][2] = x1.x;
            v[s][3] = x1.y;
        } else {
#pragma unroll
            for (int u = 0; u < 4; ++u) v[s][u] = k + u < K ? a[(size_t)(k + u) * rs] : 0.0;
        }
    }
#pragma unroll
    for (int s = 0; s < 4; ++s) {
        const int k = kb + 128 * s;
        if (k >= ldk) break;
        uint32_t lo[4], hi[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const unsigned long long x = (unsigned long long)(__double2ll_rn(oz_integer(v[s][u], f1, f2)) + (1ll << 53));
            lo[u] = (uint32_t)x;
            hi[u] = (uint32_t)(x >> 32);
        }
        uint32_t* dst = reinterpret_cast<uint32_t*>(out + (size_t)r * ldk + k);
        oz_store_planes_b(dst, plane / 4, nullptr, 0, lo, hi, mb);
    }
}

// ------------------------------------------------------------------ int8 tensor-core GEMM per modulus
using namespace tc;

constexpr int BM = 128, BN = 256, BK = 128, STAGES = 4;  // BK in bytes = int8 elements
constexpr int A_BYTES = BM * BK;                         // 16 KB
constexpr int B_BYTES = BN * BK;                         // 32 KB
constexpr int STAGE_BYTES = A_BYTES + B_BYTES;
constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + 1024 + 256;
constexpr uint32_t TMEM_COLS = 512;  // two 256-column accumulators
constexpr int GEMM_THREADS = 192;   // warp 0 copies, warp 1 MMAs and TMEM, warps 2-5 epilogue
// kind::i8: s32 accumulator (dtype 2), s8 A and B (1), K-major both, N = 256, M = 128
constexpr uint32_t IDESC_I8 = (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);

struct GemmParams {
    int M, N, K, nmod;
    int p[MAXMOD];
    uint32_t magic[MAXMOD];  // ceil(2^39 / p): u / p = umulhi(u, magic) >> 7, at most one too high
    uint32_t off[MAXMOD];    // a multiple of p >= 2^31: a + off is non-negative for any int32 a
    uint8_t* R;  // residue planes of the product: (i, j) of plane l at R[l rplane + i + j ldr]
    size_t rplane;
    int ldr;
    int b_row0;         // first row of the B operand this launch reads (column panels)
    const int2* tiles;  // (m0, n0) of the output tiles to form (tiles below a Hermitian block's
    int ntiles;         // diagonal are left out); work item w = tile w % ntiles, modulus w / ntiles
    unsigned* err;
    WaitCfg wc;
};

__device__ __forceinline__ uint64_t make_desc_sw128(uint32_t saddr) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFF);
    d |= (uint64_t)(16 >> 4) << 16;
    d |= (uint64_t)(1024 >> 4) << 32;
    d |= (uint64_t)1 << 46;
    d |= (uint64_t)2 << 61;
    return d;
}
__device__ __forceinline__ void mma_i8(uint32_t tmem, uint64_t a, uint64_t b, uint32_t accumulate) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n}\n" ::"r"(
            tmem),
        "l"(a), "l"(b), "r"(IDESC_I8), "r"(accumulate)
        : "memory");
}
__device__ __forceinline__ void tma_load_3d(uint32_t dst, const CUtensorMap* map, int x, int y, int z, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(
            dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(bar)
        : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

// Persistent: each CTA walks the work items blockIdx.x, blockIdx.x + gridDim.x, ... (an item is one
// 128 x 256 output tile modulo one p_l; items are modulus-major, so the CTAs running at the same
// time share one modulus' residue planes in L2).  Warp 0 lane 0 issues the TMA loads of 128-byte K
// slabs of both operands into a 4-stage ring, continuing from one item straight into the next;
// warp 1 lane 0 issues the M128 N256 K32 int8 MMAs (4 per slab) into one of two TMEM accumulators,
// alternating per item, so that warps 2-5 reduce the previous item's accumulator mod p to bytes
// (each thread one row, 32 columns at a time) while the next item's MMAs run.
__global__ void __launch_bounds__(GEMM_THREADS, 1) oz_gemm_kernel(const __grid_constant__ CUtensorMap tA,
                                                                  const __grid_constant__ CUtensorMap tB,
                                                                  const __grid_constant__ GemmParams p) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    uint8_t* sA = smem;
    uint8_t* sB = smem + STAGES * A_BYTES;
    uint64_t* bars = (uint64_t*)(smem + STAGES * STAGE_BYTES);
    uint64_t* full = bars;                  // [STAGES] copies landed
    uint64_t* empty = bars + STAGES;        // [STAGES] slab consumed by the MMAs
    uint64_t* accf = bars + 2 * STAGES;     // [2] accumulator complete (MMA -> epilogue)
    uint64_t* acce = bars + 2 * STAGES + 2; // [2] accumulator drained (epilogue -> MMA)
    uint64_t* doneb = bars + 2 * STAGES + 4;  // every MMA issued by the CTA has completed
    uint32_t* tmem_slot = (uint32_t*)(bars + 2 * STAGES + 5);
    volatile int* abort_flag = (volatile int*)(tmem_slot + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int KT = (p.K + BK - 1) / BK;
    const int items = p.ntiles * p.nmod;

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(smem_u32(&full[s]), 1);
            mbar_init(smem_u32(&empty[s]), 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(smem_u32(&accf[b]), 1);
            mbar_init(smem_u32(&acce[b]), 4);  // one arrival per epilogue warp
        }
        mbar_init(smem_u32(doneb), 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tA)) : "memory");
        asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tB)) : "memory");
    }
    if (warp == 1) tmem_alloc(smem_u32(tmem_slot), TMEM_COLS);
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp == 0) {
        if (lane == 0) {
            // ---------------- TMA producer (issues nothing under the withholding test switch)
            int it = 0;
            bool stop = false;
            for (int w = blockIdx.x; w < items && !stop && !p.wc.withhold; w += gridDim.x) {
                const int2 t = p.tiles[w % p.ntiles];
                const int l = w / p.ntiles;
                for (int kt = 0; kt < KT; ++kt, ++it) {
                    const int s = it % STAGES, r = it / STAGES;
                    if (r > 0 && !mbar_wait(smem_u32(&empty[s]), (r - 1) & 1, p.wc.ns)) {
                        atomicOr(p.err, 256u);
                        *abort_flag = 1;
                    }
                    if (*abort_flag) {
                        stop = true;
                        break;
                    }
                    const uint32_t fb = smem_u32(&full[s]);
                    mbar_expect_tx(fb, STAGE_BYTES);
                    tma_load_3d(smem_u32(sA + s * A_BYTES), &tA, kt * BK, t.x, l, fb);
                    tma_load_3d(smem_u32(sB + s * B_BYTES), &tB, kt * BK, p.b_row0 + t.y, l, fb);
                }
            }
            // every issued copy must have landed before the CTA may exit
            for (int j = (it > STAGES ? it - STAGES : 0); j < it; ++j) {
                if (!mbar_wait(smem_u32(&full[j % STAGES]), (j / STAGES) & 1, p.wc.ns)) {
                    atomicOr(p.err, 512u);
                    break;
                }
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            // ---------------- MMA issuer
            int it = 0, tc = 0;
            bool stop = false;
            for (int w = blockIdx.x; w < items && !stop; w += gridDim.x, ++tc) {
                const int b = tc & 1, use = tc >> 1;
                if (use > 0 && !mbar_wait(smem_u32(&acce[b]), (use - 1) & 1, p.wc.ns)) {
                    atomicOr(p.err, 4096u);
                    *abort_flag = 1;
                }
                if (*abort_flag) break;
                fence_after();
                const uint32_t acc = tmem + (uint32_t)(b * BN);
                for (int kt = 0; kt < KT; ++kt, ++it) {
                    const int s = it % STAGES, r = it / STAGES;
                    if (!mbar_wait(smem_u32(&full[s]), r & 1, p.wc.ns)) {
                        atomicOr(p.err, 1024u);
                        *abort_flag = 1;
                    }
                    if (*abort_flag) {
                        stop = true;
                        break;
                    }
                    fence_after();
                    const uint32_t a0 = smem_u32(sA + s * A_BYTES), b0 = smem_u32(sB + s * B_BYTES);
#pragma unroll
                    for (int kk = 0; kk < BK / 32; ++kk)
                        mma_i8(acc, make_desc_sw128(a0 + kk * 32), make_desc_sw128(b0 + kk * 32),
                               (kt > 0 || kk > 0) ? 1u : 0u);
                    mma_commit(smem_u32(&empty[s]));
                }
                if (stop) break;
                mma_commit(smem_u32(&accf[b]));
            }
            mma_commit(smem_u32(doneb));  // arrives once every MMA issued above has completed
        }
    } else {
        // ---------------- epilogue: warp w reads TMEM lanes 32 (w % 4) .. + 31, one row per thread
        const int quarter = warp & 3;
        int tc = 0;
        for (int w = blockIdx.x; w < items; w += gridDim.x, ++tc) {
            const int b = tc & 1, use = tc >> 1;
            const bool ok = mbar_wait(smem_u32(&accf[b]), use & 1, p.wc.ns);
            if (!ok) atomicOr(p.err, 2048u);
            if (!__all_sync(0xffffffffu, ok && !*abort_flag)) {
                if (lane == 0) *abort_flag = 1;
                break;
            }
            fence_after();
            const int2 t = p.tiles[w % p.ntiles];
            const int l = w / p.ntiles;
            const int row = t.x + quarter * 32 + lane;
            const int pm = p.p[l];
            const uint32_t mg = p.magic[l], off = p.off[l];
            uint8_t* R = p.R + (size_t)l * p.rplane + row;
#pragma unroll 1
            for (int c0 = 0; c0 < BN; c0 += 32) {
                uint32_t v[32];
                tmem_ld32(tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(b * BN + c0), v);
                if (row < p.M) {
#pragma unroll
                    for (int q = 0; q < 32; ++q) {
                        const int col = t.y + c0 + q;
                        if (col < p.N) {
                            // (int32 accumulator) mod p in [0, p), integer operations only
                            const uint32_t u = v[q] + off;
                            int r = (int)(u - (__umulhi(u, mg) >> 7) * (uint32_t)pm);
                            if (r < 0) r += pm;
                            R[(size_t)col * p.ldr] = (uint8_t)r;
                        }
                    }
                }
            }
            fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(smem_u32(&acce[b]));
        }
    }
    __syncthreads();
    if (warp == 1) {
        // TMEM is released only after every MMA of this CTA has completed
        if (!mbar_wait(smem_u32(doneb), 0, p.wc.ns) && lane == 0) atomicOr(p.err, 8192u);
        __syncwarp();
        fence_after();
        tmem_dealloc(tmem, TMEM_COLS);
    }
}

// ---- the same GEMM on SM pairs: a cluster of two CTAs forms 256 x 256 tiles with M256 N256 K32
// MMAs (cta_group::2).  Each CTA stages its own 128 rows of A and 128 rows of B per slab (32 KB, so
// six stages fit), which halves the B bytes each SM loads per MMA against the one-CTA kernel; the
// accumulator of CTA r holds rows 128 r .. 128 r + 127 of the tile, all 256 columns.
//   rank 0 (leader) warp 1 lane 0: waits for both CTAs' slabs on its full[s] (which counts the
//       copies of both), issues the MMAs, and commits to empty[s] / accf[b] / doneb of BOTH CTAs
//   both CTAs warp 0 lane 0: wait on their own empty[s], copy their half of the slab; the
//       completion goes to the leader's full[s] (the leader also posts the expected bytes)
//   both CTAs warps 2-5: epilogue of their own TMEM rows, then arrive on the leader's acce[b]
//       (8 arrivals: four warps in each CTA)
// Every wait is bounded as in the one-CTA kernel; both CTAs meet at a cluster barrier before TMEM
// is freed, so neither leaves while the other can still touch its shared memory.
constexpr int BM2 = 256, BN2 = 256, STAGES2 = 6;
constexpr int A2_BYTES = 128 * BK, B2_BYTES = 128 * BK;  // each CTA's half of a slab: 16 KB + 16 KB
constexpr int STAGE2_BYTES = A2_BYTES + B2_BYTES;
constexpr int SMEM2_BYTES = STAGES2 * STAGE2_BYTES + 1024 + 256;
constexpr uint32_t IDESC_I8_PAIR =
    (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN2 >> 3) << 17) | ((uint32_t)(BM2 >> 4) << 24);

__device__ __forceinline__ void mma_i8_pair(uint32_t tmem, uint64_t a, uint64_t b, uint32_t accumulate) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n tcgen05.mma.cta_group::2.kind::i8 [%0], %1, %2, %3, p;\n}\n" ::"r"(
            tmem),
        "l"(a), "l"(b), "r"(IDESC_I8_PAIR), "r"(accumulate)
        : "memory");
}

__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(GEMM_THREADS, 1)
    oz_gemm_pair_kernel(const __grid_constant__ CUtensorMap tA, const __grid_constant__ CUtensorMap tB,
                        const __grid_constant__ GemmParams p) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    uint8_t* sA = smem;
    uint8_t* sB = smem + STAGES2 * A2_BYTES;
    uint64_t* bars = (uint64_t*)(smem + STAGES2 * STAGE2_BYTES);
    uint64_t* full = bars;                     // [STAGES2] both halves of the slab landed (leader's)
    uint64_t* empty = bars + STAGES2;          // [STAGES2] slab consumed (each CTA's own)
    uint64_t* accf = bars + 2 * STAGES2;       // [2] accumulator complete (each CTA's own)
    uint64_t* acce = bars + 2 * STAGES2 + 2;   // [2] accumulator drained in both CTAs (leader's)
    uint64_t* doneb = bars + 2 * STAGES2 + 4;  // every MMA of the pair has completed (each CTA's own)
    uint32_t* tmem_slot = (uint32_t*)(bars + 2 * STAGES2 + 5);
    volatile int* abort_flag = (volatile int*)(tmem_slot + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t rank = cluster_rank();
    const bool leader = rank == 0;
    const int pair = blockIdx.x >> 1, npairs = gridDim.x >> 1;
    const int KT = (p.K + BK - 1) / BK;
    const int items = p.ntiles * p.nmod;

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES2; ++s) {
            mbar_init(smem_u32(&full[s]), 1);
            mbar_init(smem_u32(&empty[s]), 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(smem_u32(&accf[b]), 1);
            mbar_init(smem_u32(&acce[b]), 8);  // four epilogue warps in each CTA
        }
        mbar_init(smem_u32(doneb), 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tA)) : "memory");
        asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tB)) : "memory");
    }
    if (warp == 1) tmem_alloc_pair(smem_u32(tmem_slot), TMEM_COLS);
    fence_before();
    cluster_sync();  // both CTAs' barriers exist before either arrives on the other's
    fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp == 0) {
        if (lane == 0) {
            // ---------------- TMA producer of this CTA's half (nothing under the withholding switch)
            const uint32_t lead_full0 = peer_addr(smem_u32(&full[0]), 0);
            int it = 0;
            bool stop = false;
            for (int w = pair; w < items && !stop && !p.wc.withhold; w += npairs) {
                const int2 t = p.tiles[w % p.ntiles];
                const int l = w / p.ntiles;
                for (int kt = 0; kt < KT; ++kt, ++it) {
                    const int s = it % STAGES2, r = it / STAGES2;
                    if (r > 0 && !mbar_wait_cl(smem_u32(&empty[s]), (r - 1) & 1, p.wc.ns)) {
                        atomicOr(p.err, 256u);
                        *abort_flag = 1;
                    }
                    if (*abort_flag) {
                        stop = true;
                        break;
                    }
                    const uint32_t fb = lead_full0 + (uint32_t)(s * sizeof(uint64_t));
                    if (leader) mbar_expect_tx(smem_u32(&full[s]), 2 * STAGE2_BYTES);
                    tma_load_3d_pair(smem_u32(sA + s * A2_BYTES), &tA, kt * BK, t.x + 128 * (int)rank, l, fb);
                    tma_load_3d_pair(smem_u32(sB + s * B2_BYTES), &tB, kt * BK, p.b_row0 + t.y + 128 * (int)rank, l,
                                     fb);
                }
            }
            // the last slabs issued: the leader sees both halves land on its full[s]; either CTA
            // sees its slab consumed on its own empty[s] (the MMAs read only landed slabs)
            for (int j = (it > STAGES2 ? it - STAGES2 : 0); j < it; ++j) {
                const bool ok = leader ? mbar_wait_cl(smem_u32(&full[j % STAGES2]), (j / STAGES2) & 1, p.wc.ns)
                                       : mbar_wait_cl(smem_u32(&empty[j % STAGES2]), (j / STAGES2) & 1, p.wc.ns);
                if (!ok) {
                    atomicOr(p.err, 512u);
                    break;
                }
            }
        }
    } else if (warp == 1) {
        if (lane == 0 && leader) {
            // ---------------- MMA issuer (leader only)
            int it = 0, tc = 0;
            bool stop = false;
            for (int w = pair; w < items && !stop; w += npairs, ++tc) {
                const int b = tc & 1, use = tc >> 1;
                if (use > 0 && !mbar_wait_cl(smem_u32(&acce[b]), (use - 1) & 1, p.wc.ns)) {
                    atomicOr(p.err, 4096u);
                    *abort_flag = 1;
                }
                if (*abort_flag) break;
                fence_after();
                const uint32_t acc = tmem + (uint32_t)(b * BN2);
                for (int kt = 0; kt < KT; ++kt, ++it) {
                    const int s = it % STAGES2, r = it / STAGES2;
                    if (!mbar_wait_cl(smem_u32(&full[s]), r & 1, p.wc.ns)) {
                        atomicOr(p.err, 1024u);
                        *abort_flag = 1;
                    }
                    if (*abort_flag) {
                        stop = true;
                        break;
                    }
                    fence_after();
                    const uint32_t a0 = smem_u32(sA + s * A2_BYTES), b0 = smem_u32(sB + s * B2_BYTES);
#pragma unroll
                    for (int kk = 0; kk < BK / 32; ++kk)
                        mma_i8_pair(acc, make_desc_sw128(a0 + kk * 32), make_desc_sw128(b0 + kk * 32),
                                    (kt > 0 || kk > 0) ? 1u : 0u);
                    mma_commit_pair(smem_u32(&empty[s]), 3);
                }
                if (stop) break;
                mma_commit_pair(smem_u32(&accf[b]), 3);
            }
            mma_commit_pair(smem_u32(doneb), 3);  // arrives in both CTAs once every MMA above completed
        }
    } else {
        // ---------------- epilogue: this CTA's 128 rows of the tile, one row per thread
        const int quarter = warp & 3;
        const uint32_t lead_acce0 = peer_addr(smem_u32(&acce[0]), 0);
        int tc = 0;
        for (int w = pair; w < items; w += npairs, ++tc) {
            const int b = tc & 1, use = tc >> 1;
            const bool ok = mbar_wait_cl(smem_u32(&accf[b]), use & 1, p.wc.ns);
            if (!ok) atomicOr(p.err, 2048u);
            if (!__all_sync(0xffffffffu, ok && !*abort_flag)) {
                if (lane == 0) *abort_flag = 1;
                break;
            }
            fence_after();
            const int2 t = p.tiles[w % p.ntiles];
            const int l = w / p.ntiles;
            const int row = t.x + 128 * (int)rank + quarter * 32 + lane;
            const int pm = p.p[l];
            const uint32_t mg = p.magic[l], off = p.off[l];
            uint8_t* R = p.R + (size_t)l * p.rplane + row;
#pragma unroll 1
            for (int c0 = 0; c0 < BN2; c0 += 32) {
                uint32_t v[32];
                tmem_ld32(tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(b * BN2 + c0), v);
                if (row < p.M) {
#pragma unroll
                    for (int q = 0; q < 32; ++q) {
                        const int col = t.y + c0 + q;
                        if (col < p.N) {
                            const uint32_t u = v[q] + off;
                            int r = (int)(u - (__umulhi(u, mg) >> 7) * (uint32_t)pm);
                            if (r < 0) r += pm;
                            R[(size_t)col * p.ldr] = (uint8_t)r;
                        }
                    }
                }
            }
            fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive_cl(lead_acce0 + (uint32_t)(b * sizeof(uint64_t)));
        }
    }
    __syncthreads();
    if (warp == 1) {
        if (!mbar_wait_cl(smem_u32(doneb), 0, p.wc.ns) && lane == 0) atomicOr(p.err, 8192u);
        __syncwarp();
    }
    fence_before();
    cluster_sync();  // no MMA, copy or arrival of either CTA still targets the other
    fence_after();
    if (warp == 1) tmem_dealloc_pair(tmem, TMEM_COLS);
}

// ------------------------------------------------------------------ reconstruction
struct RecParams {
    int M, N, nmod;
    const uint8_t* R;
    size_t rplane;
    int ldr;
    const int* eA;
    const int* eB;
    int shift;  // (bitsA - 1) + (bitsB - 1)
    double alpha, beta;
    double* out;  // out(i, j) at out[i os + j ldo]: os = 1, or 2 for a part of a complex matrix
    int ldo, os;
    int herm, n_off;
    uint32_t W[MAXMOD][4];
    float w[MAXMOD];  // W_l / P
    uint32_t P[4];
    // the same constants as bytes for the dot-product form: Wq[g][i] holds byte i of W_l for the
    // moduli l = 4 g .. 4 g + 3 (one per byte), Fq[g][k] byte k of round(2^16 W_l / P), Pb[i] byte i of P
    uint32_t Wq[MAXMOD / 4][16];
    uint32_t Fq[MAXMOD / 4][2];
    uint32_t Pb[16];
};

// one thread per row, 8 columns per CTA row: out(i, j) = alpha * C'(i, j) 2^(eA_i + eB_j - shift)
// + beta * out(i, j), C' from its residues by the CRT
// One output from its residues: rp[g] holds r_l for l = 4 g .. 4 g + 3 as bytes.  With W_l and P
// in bytes, byte sums S_i = sum_l r_l W_l[i] are four-way byte dot products (each < 2^20), and
// q = round(sum_l r_l W_l / P) comes from the 16-bit fixed-point weights round(2^16 W_l / P)
// (their error, below 16 * 255 * 2^-17, is far inside the 1/4 by which T / P stays off the
// half-integers).  C' = T - q P = sum_i (S_i - q P[i]) 256^i is formed from i = 4 on: the bytes
// below 2^32 change C' by less than 2^44, under 2^-60 of the bound 2^-52 max|A'| sum|B'| >= 2^52
// that a 53-bit product is held to.  Each d_i = S_i - q P[i] is below 2^20 in magnitude (S_i and
// q P[i] both lie in [0, 2^20)), so pairs d_i + 256 d_(i+1) stay below 2^29 in 32-bit integers;
// the bytes 4..9 and 10..15 are summed exactly from three pairs each in two 64-bit integers and
// joined by one fma, then scaled by 2^(ea + eb - shift + 32).
__device__ __forceinline__ double oz_value(const RecParams& p, const uint32_t (&rp)[MAXMOD / 4], int ea, int eb) {
    if (ea == BAD_EXP || eb == BAD_EXP) return __longlong_as_double(0x7ff8000000000000ll);  // NaN in, NaN out
    if (ea == ZERO_EXP || eb == ZERO_EXP) return 0.0;
    uint32_t q0 = 0, q1 = 0;
#pragma unroll
    for (int g = 0; g < MAXMOD / 4; ++g) {
        q0 = __dp4a(rp[g], p.Fq[g][0], q0);
        q1 = __dp4a(rp[g], p.Fq[g][1], q1);
    }
    const int q = (int)((q0 + (q1 << 8) + 32768u) >> 16);
    int pr[6];  // pr[k] = d_(4+2k) + 256 d_(5+2k)
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        int d[2];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int i = 4 + 2 * k + h;
            uint32_t si = 0;
#pragma unroll
            for (int g = 0; g < MAXMOD / 4; ++g) si = __dp4a(rp[g], p.Wq[g][i], si);
            d[h] = (int)si - q * (int)p.Pb[i];
        }
        pr[k] = d[0] + 256 * d[1];
    }
    const long long lo = (long long)pr[0] + (long long)pr[1] * 65536 + (long long)pr[2] * 4294967296ll;
    const long long hi = (long long)pr[3] + (long long)pr[4] * 65536 + (long long)pr[5] * 4294967296ll;
    const double x = fma((double)hi, 281474976710656.0, (double)lo);  // hi 2^48 + lo, in units of 2^32
    // x 2^(ea + eb - shift + 32) as two exact products by normal powers of two (a shift below
    // -2044 underflows to zero either way)
    const int sh = ea + eb - p.shift + 32, s1 = max(-1022, sh / 2), s2 = max(-1022, sh - s1);
    return (x * pow2(s1)) * pow2(s2);
}

// the 4 x 4 byte transpose: word l of w holds rows 0..3 of modulus base + l (byte u = row u); out[u]
// holds the four moduli of row u
__device__ __forceinline__ void oz_transpose4(uint32_t a, uint32_t b, uint32_t c, uint32_t d, uint32_t (&o)[4]) {
    const uint32_t t0 = __byte_perm(a, b, 0x5140), t1 = __byte_perm(a, b, 0x7362);
    const uint32_t t2 = __byte_perm(c, d, 0x5140), t3 = __byte_perm(c, d, 0x7362);
    o[0] = __byte_perm(t0, t2, 0x5410);
    o[1] = __byte_perm(t0, t2, 0x7632);
    o[2] = __byte_perm(t1, t3, 0x5410);
    o[3] = __byte_perm(t1, t3, 0x7632);
}

// thread: rows 4 t .. 4 t + 3 of 8 columns; one 4-byte load per plane gives the four rows'
// residues (the planes' leading dimension ldr is a multiple of 128)
__global__ void __launch_bounds__(256) oz_reconstruct_kernel(const __grid_constant__ RecParams p) {
    const int i0 = 4 * (blockIdx.x * 256 + threadIdx.x);
    if (i0 >= p.M) return;
    int ea[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) ea[u] = i0 + u < p.M ? p.eA[i0 + u] : ZERO_EXP;
    for (int jj = 0; jj < 8; ++jj) {
        const int j = blockIdx.y * 8 + jj;
        if (j >= p.N) return;
        if (p.herm > 0 && ((i0 / BM) * BM) % p.herm > ((p.n_off + j) / BN) * BN + BN - 1) continue;
        const int eb = p.eB[j];
        const uint8_t* r = p.R + (size_t)i0 + (size_t)j * p.ldr;
        uint32_t res[MAXMOD];
#pragma unroll
        for (int l = 0; l < MAXMOD; ++l)
            res[l] = l < p.nmod ? *reinterpret_cast<const uint32_t*>(r + (size_t)l * p.rplane) : 0u;
        uint32_t rows[MAXMOD / 4][4];  // rows[g][u]: row u's residues of moduli 4 g .. 4 g + 3
#pragma unroll
        for (int g = 0; g < MAXMOD / 4; ++g) oz_transpose4(res[4 * g], res[4 * g + 1], res[4 * g + 2], res[4 * g + 3], rows[g]);
        double* o = p.out + (size_t)i0 * p.os + (size_t)j * p.ldo;
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            if (i0 + u >= p.M) break;
            const uint32_t rp[MAXMOD / 4] = {rows[0][u], rows[1][u], rows[2][u], rows[3][u]};
            double val = oz_value(p, rp, ea[u], eb) * p.alpha;
            if (p.beta != 0.0) val = fma(p.beta, o[u * p.os], val);
            o[u * p.os] = val;
        }
    }
}

// ------------------------------------------------------------------ FP64 SpMM on the int8 tensor cores
// Y = A [H, S] for atom-block CSC H and S (the FP64 CG step's [HG; SG] = D [H, S]) by the same
// modular method: A's rows and H's / S's columns are rounded to 53-bit integers, and every modulus
// is one int8 SpMM over the column-group plan of spmm.cu -- output columns in groups of G whose
// nonzero rows form a union U_g -- with U_g covered by 16-row chunks.  A's residues come
// k-blocked (per block of 256 rows, chunk c holds A(:, 16 c .. 16 c + 15) as 256 rows x 16 B,
// contiguous), so a chunk is one 4 KB bulk copy that lands in the K-major no-swizzle layout
// tcgen05 reads; two chunks make the K = 32 of one int8 MMA.  B_g^T (H's group columns, then
// S's) is stored per modulus in the same chunk order, 16 B per column and chunk, zero where a
// chunk row is not in U_g.  A CTA takes one group and 256 rows and walks all moduli: warp 0
// copies (STG stages of PPS chunk pairs; chunks adjacent in memory go in one copy, and the
// stage's B^T in one), warp 1 issues two M128 N(2G) K32 MMAs per chunk pair into TMEM, warps 2-5
// reduce each modulus' int32 accumulator mod p to bytes in the product's residue planes while the
// next modulus' copies are in flight; the CRT reconstruction then forms the FP64 result.
constexpr int SP_A_CHUNK = 256 * 16;
// a stage: PPS chunk pairs of A and their B^T (NB <= HS columns: 2 chunks x HS x 16 B per pair)
template <int PPS, int HS>
constexpr int sp_stage_bytes() {
    return PPS * (2 * SP_A_CHUNK + 2 * HS * 16);
}

struct OzSpParams {
    int n, G, NB, ngroups, nch16, cstride, nmod;
    int ncol;          // columns of the product (a CTA's last group may reach past them)
    uint32_t idesc;
    const uint8_t* a;  // A's k-blocked residues, plane l at a + l a_plane
    size_t a_plane;
    const int8_t* bt;  // B^T residues [l][g][cstride][NB][16]
    const int* cx;     // [g][cstride]: first row of each 16-row chunk (the last repeated past the end)
    const int* nsteps; // [g]: chunk pairs
    uint8_t* R;        // product residues: (row, column) of plane l at R + l rplane + row + column ldr;
    size_t rplane;     // S's product n rows below H's
    int ldr;
    bool pair;         // B^T holds S's columns after H's
    int p[MAXMOD];
    uint32_t magic[MAXMOD], off[MAXMOD];
    unsigned* err;
    WaitCfg wc;
};

__device__ __forceinline__ uint64_t desc_kmajor(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFF);
    d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
    d |= (uint64_t)1 << 46;  // version; layout type 0 = no swizzle
    return d;
}
__device__ __forceinline__ void mma_i8_n(uint32_t tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accumulate) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n}\n" ::"r"(
            tmem),
        "l"(a), "l"(b), "r"(idesc), "r"(accumulate)
        : "memory");
}

template <int STG, int PPS, int MINB, int HS>
__global__ void __launch_bounds__(192, MINB) oz_spmm_kernel(const __grid_constant__ OzSpParams p) {
    constexpr int STAGE = sp_stage_bytes<PPS, HS>();
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    uint64_t* bars = (uint64_t*)(smem + STG * STAGE);
    uint64_t* full = bars;            // [STG]
    uint64_t* empty = bars + STG;     // [STG]
    uint64_t* accf = bars + 2 * STG;  // a modulus' accumulator complete
    uint64_t* acce = accf + 1;        // ... and drained by the epilogue
    uint64_t* doneb = accf + 2;       // every MMA of the CTA completed
    uint32_t* tmem_slot = (uint32_t*)(accf + 3);
    volatile int* abort_flag = (volatile int*)(tmem_slot + 1);
    int* s_cx = (int*)(tmem_slot + 2);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // the row blocks of one group are consecutive CTAs: its B^T is fetched from memory once
    const int g = blockIdx.y, rb = blockIdx.x, row0 = rb * 256;
    const int S = p.nsteps[g];                 // chunk pairs per modulus
    const int SS = (S + PPS - 1) / PPS;        // stages per modulus
    const int T = SS * p.nmod;
    const uint32_t b_bytes = (uint32_t)(2 * p.NB * 16);

    if (threadIdx.x == 0) {
        for (int s = 0; s < STG; ++s) {
            mbar_init(smem_u32(&full[s]), 1);
            mbar_init(smem_u32(&empty[s]), 1);
        }
        mbar_init(smem_u32(accf), 1);
        mbar_init(smem_u32(acce), 4);  // one arrival per epilogue warp
        mbar_init(smem_u32(doneb), 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    for (int i = threadIdx.x; i < 2 * S; i += blockDim.x) s_cx[i] = p.cx[(size_t)g * p.cstride + i];
    if (warp == 1) tmem_alloc(smem_u32(tmem_slot), 2 * HS);  // one M128 x NB accumulator per 128-row half
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp == 0) {
        if (lane == 0) {
            // ---------------- copies: per stage the A chunks of up to PPS pairs (a run of chunks
            // adjacent in memory as one copy) and their B^T (one copy; nothing under the
            // withholding test switch)
            int issued = 0;
            const int T_issue = p.wc.withhold ? 0 : T;
            for (int it = 0; it < T_issue; ++it) {
                const int s = it % STG, r = it / STG;
                if (r > 0 && !mbar_wait(smem_u32(&empty[s]), (r - 1) & 1, p.wc.ns)) {
                    atomicOr(p.err, 16384u);
                    *abort_flag = 1;
                    break;
                }
                if (*abort_flag) break;
                const int l = it / SS, t0 = (it % SS) * PPS, np = min(PPS, S - t0);
                uint8_t* st = smem + s * STAGE;
                const uint32_t fb = smem_u32(&full[s]);
                mbar_expect_tx(fb, (uint32_t)np * ((uint32_t)(2 * SP_A_CHUNK) + b_bytes));
                const uint8_t* ab = p.a + (size_t)l * p.a_plane + (size_t)rb * p.nch16 * SP_A_CHUNK;
                int j = 0;
                while (j < 2 * np) {
                    const int c = s_cx[2 * t0 + j] >> 4;
                    int len = 1;
                    while (j + len < 2 * np && (s_cx[2 * t0 + j + len] >> 4) == c + len) ++len;
                    bulk_load(smem_u32(st + j * SP_A_CHUNK), ab + (size_t)c * SP_A_CHUNK, (uint32_t)len * SP_A_CHUNK,
                              fb);
                    j += len;
                }
                const int8_t* bb = p.bt + (((size_t)l * p.ngroups + g) * p.cstride + 2 * t0) * p.NB * 16;
                bulk_load(smem_u32(st + 2 * PPS * SP_A_CHUNK), bb, (uint32_t)np * b_bytes, fb);
                issued = it + 1;
            }
            for (int it = (issued > STG ? issued - STG : 0); it < issued; ++it) {
                if (!mbar_wait(smem_u32(&full[it % STG]), (it / STG) & 1, p.wc.ns)) {
                    atomicOr(p.err, 32768u);
                    break;
                }
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            // ---------------- MMAs: per chunk pair one M128 x NB x K32 MMA per 128-row half
            int it = 0;
            bool stop = false;
            for (int l = 0; l < p.nmod && !stop; ++l) {
                if (l > 0 && !mbar_wait(smem_u32(acce), (l - 1) & 1, p.wc.ns)) {
                    atomicOr(p.err, 65536u);
                    *abort_flag = 1;
                }
                if (*abort_flag) break;
                fence_after();
                for (int ss = 0; ss < SS; ++ss, ++it) {
                    const int s = it % STG, r = it / STG;
                    if (!mbar_wait(smem_u32(&full[s]), r & 1, p.wc.ns)) {
                        atomicOr(p.err, 131072u);
                        *abort_flag = 1;
                    }
                    if (*abort_flag) {
                        stop = true;
                        break;
                    }
                    fence_after();
                    const int t0 = ss * PPS, np = min(PPS, S - t0);
                    const uint32_t sa = smem_u32(smem + s * STAGE), sb = sa + 2 * PPS * SP_A_CHUNK;
                    for (int q = 0; q < np; ++q) {
                        const uint64_t db = desc_kmajor(sb + (uint32_t)q * b_bytes, (uint32_t)(p.NB * 16), 128);
#pragma unroll
                        for (int h = 0; h < 2; ++h)
                            mma_i8_n(tmem + (uint32_t)(HS * h),
                                     desc_kmajor(sa + (uint32_t)(2 * q * SP_A_CHUNK + h * 128 * 16), SP_A_CHUNK, 128),
                                     db, p.idesc, t0 + q > 0 ? 1u : 0u);
                    }
                    mma_commit(smem_u32(&empty[s]));
                }
                if (stop) break;
                mma_commit(smem_u32(accf));
            }
            mma_commit(smem_u32(doneb));
        }
    } else {
        // ---------------- epilogue: warp w reads TMEM lanes 32 (w % 4) .. + 31 of both halves
        const int quarter = warp & 3;
        const int ncols = p.pair ? 2 * p.G : p.G;
        for (int l = 0; l < p.nmod; ++l) {
            const bool ok = mbar_wait(smem_u32(accf), l & 1, p.wc.ns);
            if (!ok) atomicOr(p.err, 262144u);
            if (!__all_sync(0xffffffffu, ok && !*abort_flag)) {
                if (lane == 0) *abort_flag = 1;
                break;
            }
            fence_after();
            const int pm = p.p[l];
            const uint32_t mg = p.magic[l], off = p.off[l];
            uint8_t* Rl = p.R + (size_t)l * p.rplane;
#pragma unroll 1
            for (int h = 0; h < 2; ++h) {
                const int row = row0 + 128 * h + 32 * quarter + lane;
#pragma unroll 1
                for (int cb = 0; cb < ncols; cb += 32) {
                    uint32_t v[32];
                    tmem_ld32(tmem + ((uint32_t)(32 * quarter) << 16) + (uint32_t)(HS * h + cb), v);
                    if (row < p.n) {
#pragma unroll
                        for (int q = 0; q < 32; ++q) {
                            const int c = cb + q;
                            const bool sp = c >= p.G;
                            const int col = g * p.G + (sp ? c - p.G : c);
                            if (c < ncols && col < p.ncol) {
                                const uint32_t u = v[q] + off;
                                int r = (int)(u - (__umulhi(u, mg) >> 7) * (uint32_t)pm);
                                if (r < 0) r += pm;
                                Rl[(size_t)(sp ? p.n + row : row) + (size_t)col * p.ldr] = (uint8_t)r;
                            }
                        }
                    }
                }
            }
            fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(smem_u32(acce));
        }
    }
    __syncthreads();
    if (warp == 1) {
        if (!mbar_wait(smem_u32(doneb), 0, p.wc.ns) && lane == 0) atomicOr(p.err, 524288u);
        __syncwarp();
        fence_after();
        tmem_dealloc(tmem, 2 * HS);
    }
}

// The SpMM on SM pairs (form 3): a cluster of two CTAs takes 256 rows of the product and a group set
// of two consecutive column groups (their joint union walked once); CTA rank r holds rows 128 r ..
// 128 r + 127 of each A chunk and half r of the set's B^T columns (H's columns in half 0, S's in
// half 1), both stored half-major so that a run of chunks is one copy.  The leader (rank 0) issues
// one M256 x N(2 * 2G) x K32 `cta_group::2` MMA per chunk pair, which reads both CTAs' halves; each
// CTA's TMEM holds its 128 rows x all columns.  An untiled bulk copy completes on a barrier of its
// own CTA, so the other CTA's MMA warp forwards each of its stages' completion to the leader
// (pfull); the leader's commits arrive in both CTAs (empty, accf, doneb), and both CTAs' epilogue
// warps arrive on the leader's acce before it reuses the accumulator.
constexpr int SPP_A = 128 * 16;  // one CTA's half of a 16-row chunk of A
template <int PPS>
__host__ __device__ constexpr int spp_stage_bytes(int nbh) {
    return PPS * 2 * (SPP_A + nbh * 16);
}
__device__ __forceinline__ void mma_i8_pair_n(uint32_t tmem, uint64_t a, uint64_t b, uint32_t idesc,
                                              uint32_t accumulate) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n tcgen05.mma.cta_group::2.kind::i8 [%0], %1, %2, %3, p;\n}\n" ::"r"(
            tmem),
        "l"(a), "l"(b), "r"(idesc), "r"(accumulate)
        : "memory");
}

template <int STG, int PPS>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(192, 4)
    oz_spmm_pair_kernel(const __grid_constant__ OzSpParams p) {
    const int nbh = p.NB / 2;  // B^T columns per CTA: half r holds H's (r = 0) or S's (r = 1) columns
    const int STAGE = spp_stage_bytes<PPS>(nbh);
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    uint64_t* bars = (uint64_t*)(smem + STG * STAGE);
    uint64_t* full = bars;             // [STG] this CTA's copies of the stage landed (own)
    uint64_t* pfull = bars + STG;      // [STG] the other CTA's copies landed (leader's)
    uint64_t* empty = bars + 2 * STG;  // [STG] stage consumed by the MMAs (own)
    uint64_t* accf = bars + 3 * STG;   // a modulus' accumulator complete (own)
    uint64_t* acce = accf + 1;         // ... and drained in both CTAs (leader's)
    uint64_t* doneb = accf + 2;        // every MMA of the pair completed (own)
    uint32_t* tmem_slot = (uint32_t*)(accf + 3);
    volatile int* abort_flag = (volatile int*)(tmem_slot + 1);
    int* s_cx = (int*)(tmem_slot + 2);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t rank = cluster_rank();
    const bool leader = rank == 0;
    const int g = blockIdx.y, rb = blockIdx.x >> 1, row0 = rb * 256;
    const int S = p.nsteps[g];
    const int SS = (S + PPS - 1) / PPS;
    const int T = SS * p.nmod;
    const uint32_t b_bytes = (uint32_t)(2 * nbh * 16);  // one CTA's B^T of a chunk pair

    if (threadIdx.x == 0) {
        for (int s = 0; s < STG; ++s) {
            mbar_init(smem_u32(&full[s]), 1);
            mbar_init(smem_u32(&pfull[s]), 1);
            mbar_init(smem_u32(&empty[s]), 1);
        }
        mbar_init(smem_u32(accf), 1);
        mbar_init(smem_u32(acce), 8);  // four epilogue warps in each CTA
        mbar_init(smem_u32(doneb), 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    for (int i = threadIdx.x; i < 2 * S; i += blockDim.x) s_cx[i] = p.cx[(size_t)g * p.cstride + i];
    if (warp == 1) tmem_alloc_pair(smem_u32(tmem_slot), 128);
    fence_before();
    cluster_sync();  // both CTAs' barriers exist before either arrives on the other's
    fence_after();
    const uint32_t tmem = *tmem_slot;
    const int T_issue = p.wc.withhold ? 0 : T;

    if (warp == 0) {
        if (lane == 0) {
            // ---------------- copies of this CTA's halves: per stage the A chunks of up to PPS pairs
            // (a run of adjacent chunks as one copy) and their B^T (one copy)
            int issued = 0;
            for (int it = 0; it < T_issue; ++it) {
                const int s = it % STG, r = it / STG;
                if (r > 0 && !mbar_wait_cl(smem_u32(&empty[s]), (r - 1) & 1, p.wc.ns)) {
                    atomicOr(p.err, 16384u);
                    *abort_flag = 1;
                    break;
                }
                if (*abort_flag) break;
                const int l = it / SS, t0 = (it % SS) * PPS, np = min(PPS, S - t0);
                uint8_t* st = smem + s * STAGE;
                const uint32_t fb = smem_u32(&full[s]);
                mbar_expect_tx(fb, (uint32_t)np * ((uint32_t)(2 * SPP_A) + b_bytes));
                const uint8_t* ab = p.a + (size_t)l * p.a_plane + ((size_t)rb * 2 + rank) * p.nch16 * SPP_A;
                int j = 0;
                while (j < 2 * np) {
                    const int c = s_cx[2 * t0 + j] >> 4;
                    int len = 1;
                    while (j + len < 2 * np && (s_cx[2 * t0 + j + len] >> 4) == c + len) ++len;
                    bulk_load(smem_u32(st + j * SPP_A), ab + (size_t)c * SPP_A, (uint32_t)len * SPP_A, fb);
                    j += len;
                }
                const int8_t* bb =
                    p.bt + ((((size_t)l * p.ngroups + g) * 2 + rank) * p.cstride + 2 * t0) * nbh * 16;
                bulk_load(smem_u32(st + 2 * PPS * SPP_A), bb, (uint32_t)np * b_bytes, fb);
                issued = it + 1;
            }
            for (int it = (issued > STG ? issued - STG : 0); it < issued; ++it) {
                if (!mbar_wait_cl(smem_u32(&full[it % STG]), (it / STG) & 1, p.wc.ns)) {
                    atomicOr(p.err, 32768u);
                    break;
                }
            }
        }
    } else if (warp == 1) {
        if (lane == 0 && !leader) {
            // ---------------- forwarder: each stage of this CTA landed -> the leader's pfull
            const uint32_t lead_pfull0 = peer_addr(smem_u32(&pfull[0]), 0);
            for (int it = 0; it < T_issue; ++it) {
                const int s = it % STG, r = it / STG;
                if (!mbar_wait_cl(smem_u32(&full[s]), r & 1, p.wc.ns)) {
                    atomicOr(p.err, 1048576u);
                    break;
                }
                mbar_arrive_cl(lead_pfull0 + (uint32_t)(s * sizeof(uint64_t)));
            }
        } else if (lane == 0) {
            // ---------------- MMAs (leader): per chunk pair one M256 x NB x K32 MMA over both CTAs
            int it = 0;
            bool stop = false;
            for (int l = 0; l < p.nmod && !stop; ++l) {
                if (l > 0 && !mbar_wait_cl(smem_u32(acce), (l - 1) & 1, p.wc.ns)) {
                    atomicOr(p.err, 65536u);
                    *abort_flag = 1;
                }
                if (*abort_flag) break;
                fence_after();
                for (int ss = 0; ss < SS; ++ss, ++it) {
                    const int s = it % STG, r = it / STG;
                    if (!mbar_wait_cl(smem_u32(&full[s]), r & 1, p.wc.ns) ||
                        !mbar_wait_cl(smem_u32(&pfull[s]), r & 1, p.wc.ns)) {
                        atomicOr(p.err, 131072u);
                        *abort_flag = 1;
                    }
                    if (*abort_flag) {
                        stop = true;
                        break;
                    }
                    fence_after();
                    const int t0 = ss * PPS, np = min(PPS, S - t0);
                    const uint32_t sa = smem_u32(smem + s * STAGE), sb = sa + 2 * PPS * SPP_A;
                    for (int q = 0; q < np; ++q)
                        mma_i8_pair_n(tmem, desc_kmajor(sa + (uint32_t)(2 * q * SPP_A), SPP_A, 128),
                                      desc_kmajor(sb + (uint32_t)q * b_bytes, (uint32_t)(nbh * 16), 128), p.idesc,
                                      t0 + q > 0 ? 1u : 0u);
                    mma_commit_pair(smem_u32(&empty[s]), 3);
                }
                if (stop) break;
                mma_commit_pair(smem_u32(accf), 3);
            }
            mma_commit_pair(smem_u32(doneb), 3);
        }
    } else {
        // ---------------- epilogue: this CTA's 128 rows, warp w's TMEM lanes 32 (w % 4) .. + 31
        const int quarter = warp & 3;
        const int ncols = 2 * p.G;
        const uint32_t lead_acce = peer_addr(smem_u32(acce), 0);
        const int row = row0 + 128 * (int)rank + 32 * quarter + lane;
        for (int l = 0; l < p.nmod; ++l) {
            const bool ok = mbar_wait_cl(smem_u32(accf), l & 1, p.wc.ns);
            if (!ok) atomicOr(p.err, 262144u);
            if (!__all_sync(0xffffffffu, ok && !*abort_flag)) {
                if (lane == 0) *abort_flag = 1;
                break;
            }
            fence_after();
            const int pm = p.p[l];
            const uint32_t mg = p.magic[l], off = p.off[l];
            uint8_t* Rl = p.R + (size_t)l * p.rplane;
#pragma unroll 1
            for (int cb = 0; cb < ncols; cb += 32) {
                uint32_t v[32];
                tmem_ld32(tmem + ((uint32_t)(32 * quarter) << 16) + (uint32_t)cb, v);
                if (row < p.n) {
#pragma unroll
                    for (int q = 0; q < 32; ++q) {
                        const int c = cb + q;
                        const bool sp = c >= p.G;
                        const int col = g * p.G + (sp ? c - p.G : c);
                        if (c < ncols && col < p.ncol) {
                            const uint32_t u = v[q] + off;
                            int r = (int)(u - (__umulhi(u, mg) >> 7) * (uint32_t)pm);
                            if (r < 0) r += pm;
                            Rl[(size_t)(sp ? p.n + row : row) + (size_t)col * p.ldr] = (uint8_t)r;
                        }
                    }
                }
            }
            fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive_cl(lead_acce);
        }
    }
    __syncthreads();
    if (warp == 1) {
        if (!mbar_wait_cl(smem_u32(doneb), 0, p.wc.ns) && lane == 0) atomicOr(p.err, 524288u);
        __syncwarp();
    }
    fence_before();
    cluster_sync();  // no MMA, copy or arrival of either CTA still targets the other
    fence_after();
    if (warp == 1) tmem_dealloc_pair(tmem, 128);
}

// column exponents of the group blocks: e[g G + j] for the columns j < G of group g below N
__global__ void oz_colexp_kernel(int ngroups, int G, int N, const int* __restrict__ gptr,
                                 const double* __restrict__ bvals, int* __restrict__ e) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ngroups * G) return;
    const int g = i / G, j = i % G;
    if (g * G + j >= N) return;
    double mx = 0.0;
    bool bad = false;
    for (int k = gptr[g]; k < gptr[g + 1]; ++k) {
        const double v = fabs(bvals[(size_t)k * G + j]);
        bad |= !(v <= 1.7976931348623157e308);
        mx = fmax(mx, v);
    }
    e[g * G + j] = bad ? BAD_EXP : (mx > 0.0 ? ilogb(mx) : ZERO_EXP);
}

// B^T residues: for union entry k of group g (row urows[k]) and column j, the residue of the
// column-scaled integer of B_g(k, j) in every modulus, at bt[((l nsg + s') cstride + cidx) NB + c0 +
// coff + j][krow]: s' = sgk[k] smul + sadd with sgk[k] the CTA's group set holding g (smul = 2 and
// sadd = the half for the half-major layout of the SM-pair form), cidx[k] the 16-row chunk of the
// row in the set's chunk list, krow[k] the row in the chunk, coff[k] the group's first column in
// the set
__global__ void oz_bt_kernel(int nentries, int G, int NB, int c0, int nsg, int cstride, int smul, int sadd,
                             const int* __restrict__ gofk, const int* __restrict__ sgk, const int* __restrict__ coff,
                             const int* __restrict__ cidx, const int* __restrict__ krow,
                             const double* __restrict__ bvals, const int* __restrict__ e, int bits,
                             const __grid_constant__ ModParams mp, int8_t* __restrict__ bt) {
    const long long tot = (long long)nentries * G;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < tot;
         i += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(i / G), j = (int)(i % G);
        const int g = gofk[k];
        double f1, f2;
        oz_scales(e[g * G + j], bits, f1, f2);
        const Limbs x = oz_limbs(oz_integer(bvals[i], f1, f2));
        const size_t o =
            (((size_t)sgk[k] * smul + sadd) * cstride + cidx[k]) * NB * 16 + (size_t)(c0 + coff[k] + j) * 16 + krow[k];
        const size_t lplane = (size_t)nsg * cstride * NB * 16;
#pragma unroll
        for (int l = 0; l < MAXMOD; ++l)
            if (l < mp.nmod) bt[(size_t)l * lplane + o] = (int8_t)(l == 0 ? (x.c & 0xFF) : oz_residue(x, mp, l));
    }
}

// the reconstruction's constants: W_l and P in 32-bit limbs and as bytes, the fixed-point weights
void fill_rec_tables(RecParams& rp, const Table& tb, int nmod) {
    for (int l = 0; l < MAXMOD; ++l) {
        for (int q = 0; q < 4; ++q) rp.W[l][q] = l < nmod ? tb.W[l][q] : 0u;
        rp.w[l] = l < nmod ? (float)tb.w[l] : 0.0f;
    }
    for (int q = 0; q < 4; ++q) rp.P[q] = tb.P[q];
    for (int g = 0; g < MAXMOD / 4; ++g) {
        for (int i = 0; i < 16; ++i) {
            uint32_t v = 0;
            for (int u = 0; u < 4; ++u) {
                const int l = 4 * g + u;
                const uint32_t byte = l < nmod ? (tb.W[l][i / 4] >> (8 * (i % 4))) & 0xFFu : 0u;
                v |= byte << (8 * u);
            }
            rp.Wq[g][i] = v;
        }
        for (int k = 0; k < 2; ++k) {
            uint32_t v = 0;
            for (int u = 0; u < 4; ++u) {
                const int l = 4 * g + u;
                const uint32_t F = l < nmod ? (uint32_t)std::min(65535.0, std::nearbyint(tb.w[l] * 65536.0)) : 0u;
                v |= ((F >> (8 * k)) & 0xFFu) << (8 * u);
            }
            rp.Fq[g][k] = v;
        }
    }
    for (int i = 0; i < 16; ++i) rp.Pb[i] = (tb.P[i / 4] >> (8 * (i % 4))) & 0xFFu;
}

// ------------------------------------------------------------------ host side
CUtensorMap map_planes(const void* base, int rows, int K, int ldk, int nmod, int box_rows) {
    CUtensorMap m;
    cuuint64_t dims[3] = {(cuuint64_t)K, (cuuint64_t)rows, (cuuint64_t)nmod};
    cuuint64_t strides[2] = {(cuuint64_t)ldk, (cuuint64_t)ldk * (cuuint64_t)rows};
    cuuint32_t box[3] = {(cuuint32_t)BK, (cuuint32_t)box_rows, 1};
    cuuint32_t estr[3] = {1, 1, 1};
    CUresult r = tc::encode_fn()(&m, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, const_cast<void*>(base), dims, strides, box, estr,
                                 CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                                 CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) fail(OMM_ERR_CUDA, "oz: cuTensorMapEncodeTiled failed with " + std::to_string((int)r));
    return m;
}

ModB mod_b() {
    ModB m{};
    for (int l = 0; l < MAXMOD; ++l) {
        const uint64_t p = (uint64_t)kMods[l];
        uint64_t w[7], v = 1 % p;
        for (int k = 0; k < 7; ++k) {
            w[k] = v;
            v = (v * 256) % p;
        }
        m.wlo[l] = (uint32_t)(w[0] | (w[1] << 8) | (w[2] << 16) | (w[3] << 24));
        m.whi[l] = (uint32_t)(w[4] | (w[5] << 8) | (w[6] << 16));
        m.e[l] = (uint32_t)(p - (1ull << 53) % p);
        m.negp[l] = (uint32_t)(0u - (uint32_t)p);
        const uint64_t mg = ((1ull << 39) + p - 1) / p;
        m.magic[l] = (uint32_t)mg;
        m.mh[l] = (p - 1) / 2 * mg;
    }
    return m;
}

ModParams mod_params(int nmod) {
    const Table& t = table(nmod);
    ModParams mp{};
    mp.nmod = nmod;
    for (int l = 0; l < nmod; ++l) {
        const uint32_t p = (uint32_t)t.p[l];
        mp.p[l] = t.p[l];
        mp.c18[l] = (uint32_t)((1ull << 18) % p);
        mp.c36[l] = (uint32_t)((1ull << 36) % p);
        mp.off[l] = (uint32_t)(((1ull << 25) + p - 1) / p * p);
        mp.half[l] = (p - 1) / 2;
        mp.magic[l] = (uint32_t)(((1ull << 39) + p - 1) / p);
    }
    return mp;
}

}  // namespace oz

void oz_axpby_exps(int R, int K, double alpha, const DView& X, double beta, DView& Y, int* erow, int* ecol) {
    using namespace oz;
    if (!X.is_real || !Y.is_real) fail(OMM_ERR_ARG, "oz_axpby_exps: real operands only");
    if (R == 0 || K == 0) return;
    cudaStream_t st = rt().stream;
    if (erow) OMM_CK(cudaMemsetAsync(erow, 0x80, (size_t)R * sizeof(int), st));
    if (ecol) OMM_CK(cudaMemsetAsync(ecol, 0x80, (size_t)K * sizeof(int), st));
    static int sms = 0;
    if (!sms) OMM_CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, rt().device));
    // 64 warps per SM, rounded down to a multiple of the row blocks
    const int nrb = (R + AX_WR - 1) / AX_WR;
    const int W = std::max(nrb, sms * 64 / nrb * nrb);
    ktime_begin();
    oz_axpby_exps_kernel<<<(W + 7) / 8, 256, 0, st>>>(R, K, alpha, X.as<double>(), X.ld, beta, Y.as<double>(), Y.ld,
                                                      W, erow, ecol);
    OMM_KCHECK();
    ktime_end("oz_axpby_exps_kernel", 24.0 * R * (double)K);
}

// residues of one operand (rows x K of A_op, K-major int8 planes) and its row exponents (exps_in:
// exponents already formed, e.g. by oz_axpby_exps, copied instead of recomputed)
void oz_prepare(const DView& src, bool kcontig, int rows, int K, int nmod, int bits, OzOperand& op, bool with_kb,
                int part, const int* exps_in, bool kb_halves) {
    using namespace oz;
    if (with_kb && kcontig) fail(OMM_ERR_ARG, "oz_prepare: k-blocked residues need a row-contiguous source");
    op.rows = rows;
    op.K = K;
    op.ldk = (K + 15) / 16 * 16;
    op.nmod = nmod;
    op.bits = bits;
    op.plane = (size_t)op.ldk * rows;
    op.planes.ensure(op.plane * nmod);
    op.kb_plane = with_kb ? (size_t)(rows + 255) / 256 * 256 * op.ldk : 0;
    op.kb_halves = with_kb && kb_halves;
    if (with_kb) op.kb.ensure(op.kb_plane * nmod);
    op.exps.ensure((size_t)rows * sizeof(int));
    cudaStream_t st = rt().stream;
    // a real matrix, or the real (part 0) / imaginary (part 1) part of a complex one: element
    // (i, k) at a[i rs + k ld] with rs = 2 and ld twice the complex leading dimension
    if ((part >= 0) == src.is_real) fail(OMM_ERR_ARG, "oz_prepare: part given for a real source or missing");
    const double* a = src.as<double>() + (part > 0 ? 1 : 0);
    const int rs = part >= 0 ? 2 : 1, ld = part >= 0 ? 2 * src.ld : src.ld;
    // algorithmic bytes: the FP64 operand read once per pass, the residue planes written once
    const double src_bytes = 8.0 * rows * (double)K;
    if (exps_in) {
        OMM_CK(cudaMemcpyAsync(op.exps.p, exps_in, (size_t)rows * sizeof(int), cudaMemcpyDeviceToDevice, st));
    } else {
        OMM_CK(cudaMemsetAsync(op.exps.p, 0x80, (size_t)rows * sizeof(int), st));
        ktime_begin();
        if (kcontig) {
            oz_exp_kc_kernel<<<(rows + 7) / 8, 256, 0, st>>>(rows, K, a, rs, ld, op.exps.as<int>());
        } else {
            dim3 g((rows + 255) / 256, (K + 255) / 256);
            oz_exp_rows_kernel<<<g, 256, 0, st>>>(rows, K, a, rs, ld, op.exps.as<int>());
        }
        OMM_KCHECK();
        ktime_end("oz_exp_kernel", src_bytes);
    }
    if (nmod != MAXMOD) fail(OMM_ERR_ARG, "oz_prepare: the residue kernels form all 16 moduli");
    static const ModB mb = mod_b();
    ktime_begin();
    if (kcontig) {
        dim3 g((rows + 7) / 8, (K + 511) / 512);
        oz_res_kc_kernel<<<g, 256, 0, st>>>(rows, K, a, rs, ld, op.exps.as<int>(), bits, op.planes.as<int8_t>(),
                                            op.ldk, op.plane, mb);
    } else {
        dim3 g((rows + 31) / 32, (K + 127) / 128);
        if (with_kb)
            oz_res_rows_kernel<true><<<g, 256, 0, st>>>(rows, K, a, rs, ld, op.exps.as<int>(), bits,
                                                        op.planes.as<int8_t>(), op.ldk, op.plane, mb,
                                                        op.kb.as<uint8_t>(), op.kb_plane, op.ldk / 16,
                                                        op.kb_halves ? 1 : 0);
        else
            oz_res_rows_kernel<false><<<g, 256, 0, st>>>(rows, K, a, rs, ld, op.exps.as<int>(), bits,
                                                         op.planes.as<int8_t>(), op.ldk, op.plane, mb, nullptr, 0,
                                                         op.ldk / 16, 0);
    }
    OMM_KCHECK();
    ktime_end(kcontig ? "oz_res_kc_kernel" : "oz_res_rows_kernel",
              src_bytes + (double)nmod * rows * K * (with_kb ? 2.0 : 1.0));
}

namespace {
size_t g_panel_bytes = (size_t)4 << 30;  // cap on the product's residue planes per launch

// algorithmic bytes of one reconstruction over M x nc outputs: the residue planes read, each
// output written (and read when beta != 0); a Hermitian product (herm > 0) forms the upper
// tiles only, about half
double recon_bytes(const oz::RecParams& rp, int M, int nc) {
    const double per = rp.nmod + 8.0 + (rp.beta != 0.0 ? 8.0 : 0.0);
    return per * M * (double)nc * (rp.herm > 0 ? 0.5 : 1.0);
}
}
size_t oz_panel_bytes() { return g_panel_bytes; }

namespace {
DevBuf& product_planes() {
    static DevBuf* b = new DevBuf();
    return *b;
}
}  // namespace

OzOperand& oz_scratch(int slot) {
    static OzOperand* ops = new OzOperand[OZS_COUNT];
    if (slot < 0 || slot >= OZS_COUNT) fail(OMM_ERR_ARG, "oz_scratch: no such operand");
    return ops[slot];
}

void oz_release_patterns();
void oz_release_scratch() {
    oz_release_patterns();
    product_planes().release();
    for (int i = 0; i < OZS_COUNT; ++i) {
        OzOperand& o = oz_scratch(i);
        o.planes.release();
        o.exps.release();
        o.kb.release();
        o.rows = o.K = 0;
    }
}

// (m0, n0) of the bm x bn tiles of an M x nc panel starting at global column c0 that reach the
// upper triangle of their Hermitian block (all tiles when herm == 0); kept per shape
const DevBuf& tile_list(int M, int nc, int herm, int c0, int bm, int bn) {
    static std::map<std::tuple<int, int, int, int, int, int>, std::unique_ptr<DevBuf>>* cache =
        new std::map<std::tuple<int, int, int, int, int, int>, std::unique_ptr<DevBuf>>();
    auto key = std::make_tuple(M, nc, herm, c0, bm, bn);
    auto it = cache->find(key);
    if (it != cache->end()) return *it->second;
    // in groups of 8 tile rows walked column by column, so that the tiles in flight at one time
    // share their operand rows through L2
    std::vector<int2> v;
    const int nM = (M + bm - 1) / bm, nN = (nc + bn - 1) / bn, GROUP = 8;
    for (int L = 0; L < nM * nN; ++L) {
        const int per = GROUP * nN, g = L / per, first = g * GROUP, size = std::min(GROUP, nM - first), r = L - g * per;
        const int m0 = (first + r % size) * bm, n0 = (r / size) * bn;
        if (herm == 0 || m0 % herm <= c0 + n0 + bn - 1) v.push_back(make_int2(m0, n0));
    }
    auto b = std::make_unique<DevBuf>();
    b->alloc(std::max<size_t>(1, v.size()) * sizeof(int2));
    if (!v.empty())
        OMM_CK(cudaMemcpyAsync(b->p, v.data(), v.size() * sizeof(int2), cudaMemcpyHostToDevice, rt().stream));
    OMM_CK(cudaStreamSynchronize(rt().stream));
    b->bytes = v.size() * sizeof(int2);
    const DevBuf& ref = *b;
    (*cache)[key] = std::move(b);
    return ref;
}

int oz_bits(int K, int nmod) {
    const double room = oz::table(nmod).log2P - 2.0 - std::log2((double)std::max(K, 1));
    return std::min(53, (int)std::floor(room / 2.0));
}

// out (M x N FP64, column-major, ldo) = alpha * A B^T + beta * out from prepared operands
void oz_gemm(const OzOperand& A, const OzOperand& B, double alpha, double beta, DView& C, int herm, int out_part) {
    using namespace oz;
    const int M = A.rows, N = B.rows, K = A.K;
    if (B.K != K || A.nmod != B.nmod) fail(OMM_ERR_ARG, "oz_gemm: operands differ in K or moduli");
    if (K > MAX_K) fail(OMM_ERR_ARG, "oz_gemm: K must be below 2^17");
    if (herm < 0 || (herm > 0 && (herm % BM || M % herm))) fail(OMM_ERR_ARG, "oz_gemm: bad Hermitian block size");
    const Table& tb = table(A.nmod);
    if ((double)(A.bits + B.bits) > tb.log2P - 2.0 - std::log2((double)std::max(K, 1)))
        fail(OMM_ERR_ARG, "oz_gemm: operand bits exceed the moduli's range");
    if (M == 0 || N == 0) return;
    if (K == 0) {
        if (out_part >= 0) fail(OMM_ERR_ARG, "oz_gemm: empty inner dimension for a complex part");
        const double b2[2] = {beta, 0.0};
        if (beta != 1.0) k_scale(C, b2);
        return;
    }
    static bool attr = false;
    if (!attr) {
        OMM_CK(cudaFuncSetAttribute(oz_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES));
        OMM_CK(cudaFuncSetAttribute(oz_gemm_pair_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM2_BYTES));
        attr = true;
    }
    // SM pairs (256 x 256 tiles) unless a Hermitian block would split a pair's rows
    const bool pairs = tc_pairs_enabled() && M > BM && (herm == 0 || herm % BM2 == 0);
    const int tbm_ = pairs ? BM2 : BM, tbn_ = pairs ? BN2 : BN;
    const CUtensorMap ta = map_planes(A.planes.p, M, K, A.ldk, A.nmod, BM);
    const CUtensorMap tbm = map_planes(B.planes.p, N, K, B.ldk, B.nmod, pairs ? 128 : BN);
    // the product's residue planes, for at most ~4 GB of them at a time: panels of columns
    const int ldr = (M + 127) / 128 * 128;
    const size_t cap = oz_panel_bytes();
    int np = (int)std::min<size_t>((size_t)N, std::max<size_t>(BN, cap / ((size_t)A.nmod * ldr) / BN * BN));
    DevBuf& Rb = product_planes();
    const size_t rplane = (size_t)ldr * np;
    Rb.ensure(rplane * A.nmod);
    GemmParams gp{};
    gp.M = M;
    gp.K = K;
    gp.nmod = A.nmod;
    for (int l = 0; l < A.nmod; ++l) {
        const uint32_t pl = (uint32_t)tb.p[l];
        gp.p[l] = tb.p[l];
        gp.magic[l] = (uint32_t)(((1ull << 39) + pl - 1) / pl);
        gp.off[l] = (uint32_t)(((1ull << 31) + pl - 1) / pl * pl);
    }
    gp.R = Rb.as<uint8_t>();
    gp.rplane = rplane;
    gp.ldr = ldr;
    gp.err = tc_error_flag();
    gp.wc = tc_wait_cfg();
    static int sms = 0;
    if (!sms) OMM_CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, rt().device));
    RecParams rp{};
    rp.M = M;
    rp.nmod = A.nmod;
    rp.R = Rb.as<uint8_t>();
    rp.rplane = rplane;
    rp.ldr = ldr;
    rp.eA = A.exps.as<int>();
    rp.shift = (A.bits - 1) + (B.bits - 1);
    rp.alpha = alpha;
    rp.beta = beta;
    if ((out_part >= 0) == C.is_real) fail(OMM_ERR_ARG, "oz_gemm: output part given for a real result or missing");
    rp.ldo = out_part >= 0 ? 2 * C.ld : C.ld;
    rp.os = out_part >= 0 ? 2 : 1;
    rp.herm = herm;
    fill_rec_tables(rp, tb, A.nmod);
    for (int c0 = 0; c0 < N; c0 += np) {
        const int nc = std::min(np, N - c0);
        // the panel's columns are rows c0 .. c0 + nc - 1 of the B operand
        const DevBuf& tl = tile_list(M, nc, herm, c0, tbm_, tbn_);
        gp.N = nc;
        gp.b_row0 = c0;
        gp.tiles = tl.as<int2>();
        gp.ntiles = (int)(tl.bytes / sizeof(int2));
        const int items = gp.ntiles * A.nmod;
        if (items > 0) {
            ktime_begin();
            if (pairs) {
                oz_gemm_pair_kernel<<<2 * std::min(items, sms / 2), GEMM_THREADS, SMEM2_BYTES, rt().stream>>>(ta, tbm,
                                                                                                             gp);
            } else {
                oz_gemm_kernel<<<std::min(items, sms), GEMM_THREADS, SMEM_BYTES, rt().stream>>>(ta, tbm, gp);
            }
            OMM_KCHECK();
            // int8 ops of the tiles formed (the useful rows x columns of each, all moduli)
            double cells = 0.0;
            for (int m0 = 0; m0 < M; m0 += tbm_)
                for (int n0 = 0; n0 < nc; n0 += tbn_)
                    if (herm == 0 || m0 % herm <= c0 + n0 + tbn_ - 1)
                        cells += (double)std::min(tbm_, M - m0) * std::min(tbn_, nc - n0);
            ktime_end(pairs ? "oz_gemm_pair_kernel" : "oz_gemm_kernel", 2.0 * K * cells * A.nmod);
        }
        rp.N = nc;
        rp.n_off = c0;
        rp.eB = B.exps.as<int>() + c0;
        rp.out = C.as<double>() + (size_t)c0 * rp.ldo + (out_part > 0 ? 1 : 0);
        dim3 rg((M + 1023) / 1024, (nc + 7) / 8);
        ktime_begin();
        oz_reconstruct_kernel<<<rg, 256, 0, rt().stream>>>(rp);
        OMM_KCHECK();
        ktime_end("oz_reconstruct_kernel", recon_bytes(rp, M, nc));
    }
}

// ------------------------------------------------------------------ FP64 SpMM on the int8 tensor cores (host)
// The plan of an H (and S of the same pattern): the groups' 16-row chunk lists, the B^T residues of
// the column-scaled integers of H's and S's group blocks, and their column exponents.  Built
// once per pair of matrices (their pattern ids change with their values).
namespace {
// Form of the int8 SpMM: 0 = one column group per CTA, four stages of one chunk pair (four CTAs
// per SM); 1 = one group, two stages of three chunk pairs (a third of the copies, each up to six
// chunks long; three CTAs per SM); 2 = two consecutive groups per CTA sharing the walk of their
// joint union (N = 4G MMAs, 256 TMEM columns, two CTAs per SM, four stages of two pairs).  At
// m = 12,288, n = 1,536 form 1 took 1.71 ms, form 0 2.06 ms; three stages of two pairs 1.85 ms,
// four of two (two CTAs per SM) 2.43 ms, five of one 2.02 ms, two of two at four CTAs per SM
// 1.69 ms.  Form 2 moves 19 % fewer operand
// bytes from L2 on a cubic lattice but took 2.06 ms: with two CTAs per SM a CTA's MMAs wait out
// its epilogue, which is twice as long.  3 = the two groups of form 2 on an SM pair (clusters of
// two CTAs, `cta_group::2` MMAs over both CTAs' halves of the operands): the same 19 % fewer bytes
// at four CTAs per SM; products without S take form 1.  It took 1.77 ms against form 1's 1.71 ms:
// each CTA's copies are half as large, and the other CTA's stages reach the leader one hop later.
int g_oz_spmm_form = 1;
int oz_spmm_sg() { return g_oz_spmm_form >= 2 ? 2 : 1; }

}  // namespace

// The part of a plan that depends on the pattern only (the column groups' unions as chunk lists
// and the index arrays of the B^T layout), kept by content for the patterns planned last: an SCF
// caller registers H afresh every cycle with the pattern of the cycle before.
struct OzPatternPlan {
    int G = 0, ngroups = 0, sg = 1, nsg = 0, maxch = 0, nent = 0;
    std::vector<int> gptr, urows;  // the key, with G and sg
    DevBuf cx, nsteps, gofk, sgk, coff, cidx, krow;
};
namespace {
std::mutex g_ozpp_mu;
std::deque<std::shared_ptr<OzPatternPlan>> g_ozpp;  // most recent first
constexpr size_t kOzPatternsKept = 2;
}  // namespace
bool oz_spmm_kb_halves(bool with_s) { return with_s && g_oz_spmm_form == 3; }
// drops the kept pattern plans (plans still held by matrices keep theirs)
void oz_release_patterns() {
    std::lock_guard<std::mutex> lk(g_ozpp_mu);
    g_ozpp.clear();
}

struct OzSpmmPlan {
    int G = 0, NB = 0, ngroups = 0, cstride = 0, nmod = 0, bits = 0, m = 0;
    int sg = 1;  // column groups per CTA; G and ngroups count the CTAs' group sets
    double nnz = 0;  // nonzeros of H (and S): the FP64 flops of a product are 2 nnz n
    bool pair = false;
    bool halves = false;  // B^T half-major (H's columns, then S's, per group set): the SM-pair form
    std::shared_ptr<OzPatternPlan> pat;
    DevBuf bt, eH, eS;
    unsigned long long h_id = 0, s_id = 0;
};

// null when the matrices do not fit the kernel (no column-group plan, groups wider than 32
// columns, or S of another pattern)
static OzSpmmPlan* oz_spmm_plan(const msw_matrix* H, const msw_matrix* S, int bits, int sg, bool halves) {
    using namespace oz;
    msw_matrix* Hm = const_cast<msw_matrix*>(H);
    if (halves && (!S || sg != 2)) return nullptr;
    if (Hm->oz_plan && Hm->oz_plan->h_id == H->pattern_id && Hm->oz_plan->s_id == (S ? S->pattern_id : 0) &&
        Hm->oz_plan->bits == bits && Hm->oz_plan->sg == sg && Hm->oz_plan->halves == halves)
        return Hm->oz_plan->ngroups ? Hm->oz_plan.get() : nullptr;
    auto T = std::make_shared<OzSpmmPlan>();
    T->h_id = H->pattern_id;
    T->s_id = S ? S->pattern_id : 0;
    T->bits = bits;
    T->sg = sg;
    T->halves = halves;
    Hm->oz_plan = T;
    const SpmmPlanView P = spmm_plan_view(H);
    if (!P.cgu || P.G > 32 || P.ngroups == 0) return nullptr;
    SpmmPlanView PS{};
    if (S) {
        PS = spmm_plan_view(S);
        if (!PS.cgu || PS.G != P.G || PS.ngroups != P.ngroups) return nullptr;
        for (int g = 0; g <= P.ngroups; ++g)
            if (PS.gptr[g] != P.gptr[g]) return nullptr;
        if (!std::equal(P.urows, P.urows + P.gptr[P.ngroups], PS.urows)) return nullptr;
    }
    // a CTA takes sg consecutive groups (a group set): the union of their unions covered by
    // 16-row chunks, ascending -- from the pattern cache when this pattern was planned before
    const int nent = P.gptr[P.ngroups];
    std::shared_ptr<OzPatternPlan> pp;
    {
        std::lock_guard<std::mutex> lk(g_ozpp_mu);
        for (auto& e : g_ozpp)
            if (e->sg == sg && e->G == P.G && e->ngroups == P.ngroups && e->nent == nent &&
                std::equal(e->gptr.begin(), e->gptr.end(), P.gptr) &&
                std::memcmp(e->urows.data(), P.urows, (size_t)nent * sizeof(int)) == 0) {
                pp = e;
                break;
            }
    }
    cudaStream_t st = rt().stream;
    if (!pp) {
        pp = std::make_shared<OzPatternPlan>();
        pp->G = P.G;
        pp->ngroups = P.ngroups;
        pp->sg = sg;
        pp->nent = nent;
        pp->gptr.assign(P.gptr, P.gptr + P.ngroups + 1);
        pp->urows.assign(P.urows, P.urows + nent);
        const int nsg = (P.ngroups + sg - 1) / sg;
        std::vector<int> gofk(nent), sgk(nent), coff(nent), cidx(nent), krow(nent), nst(nsg);
        std::vector<std::vector<int>> chunks(nsg);
        int maxch = 0;
        for (int s2 = 0; s2 < nsg; ++s2) {
            auto& ch = chunks[s2];
            const int g0 = s2 * sg, g1 = std::min(P.ngroups, g0 + sg);
            for (int k = P.gptr[g0]; k < P.gptr[g1]; ++k) ch.push_back(P.urows[k] & ~15);
            std::sort(ch.begin(), ch.end());
            ch.erase(std::unique(ch.begin(), ch.end()), ch.end());
            if (ch.empty()) return nullptr;
            for (int g = g0; g < g1; ++g)
                for (int k = P.gptr[g]; k < P.gptr[g + 1]; ++k) {
                    const int r = P.urows[k];
                    gofk[k] = g;
                    sgk[k] = s2;
                    coff[k] = (g - g0) * P.G;
                    cidx[k] = (int)(std::lower_bound(ch.begin(), ch.end(), r & ~15) - ch.begin());
                    krow[k] = r & 15;
                }
            nst[s2] = ((int)ch.size() + 1) / 2;
            maxch = std::max(maxch, 2 * nst[s2]);
        }
        pp->nsg = nsg;
        pp->maxch = maxch;
        std::vector<int> cx((size_t)nsg * maxch);
        for (int s2 = 0; s2 < nsg; ++s2)
            for (int c = 0; c < maxch; ++c)
                cx[(size_t)s2 * maxch + c] = chunks[s2][std::min<size_t>(c, chunks[s2].size() - 1)];
        pp->cx.alloc(cx.size() * sizeof(int));
        pp->nsteps.alloc(nst.size() * sizeof(int));
        OMM_CK(cudaMemcpyAsync(pp->cx.p, cx.data(), cx.size() * sizeof(int), cudaMemcpyHostToDevice, st));
        OMM_CK(cudaMemcpyAsync(pp->nsteps.p, nst.data(), nst.size() * sizeof(int), cudaMemcpyHostToDevice, st));
        const std::pair<DevBuf*, const std::vector<int>*> idx[] = {
            {&pp->gofk, &gofk}, {&pp->sgk, &sgk}, {&pp->coff, &coff}, {&pp->cidx, &cidx}, {&pp->krow, &krow}};
        for (const auto& pr : idx) {
            pr.first->alloc(std::max(1, nent) * sizeof(int));
            OMM_CK(cudaMemcpyAsync(pr.first->p, pr.second->data(), nent * sizeof(int), cudaMemcpyHostToDevice, st));
        }
        OMM_CK(cudaStreamSynchronize(st));  // the host index vectors go out of scope
        std::lock_guard<std::mutex> lk(g_ozpp_mu);
        g_ozpp.push_front(pp);
        while (g_ozpp.size() > kOzPatternsKept) g_ozpp.pop_back();
    }
    const int nsg = pp->nsg, maxch = pp->maxch;
    const int Gs = sg * P.G;  // columns of a group set
    T->pat = pp;
    T->G = Gs;
    T->pair = S != nullptr;
    T->NB = ((S ? 2 * Gs : Gs) + 15) / 16 * 16;
    if (T->NB > (sg == 1 ? 64 : 128)) return nullptr;
    // the SM-pair form: each CTA's half of B^T is one matrix's Gs columns, whole 8-row core matrices
    if (halves && (Gs % 8 != 0 || 2 * Gs > 128)) return nullptr;
    if (halves) T->NB = 2 * Gs;
    T->ngroups = 0;  // not usable until built
    T->cstride = maxch;
    T->nmod = OZ_NMOD;
    T->m = H->dim2;
    T->nnz = (double)H->nnz + (S ? (double)S->nnz : 0.0);
    const int ncol = P.ngroups * P.G;
    T->eH.alloc(std::max(ncol, H->dim2) * sizeof(int));
    oz_colexp_kernel<<<(ncol + 255) / 256, 256, 0, st>>>(P.ngroups, P.G, H->dim2, P.d_gptr, P.d_bvals, T->eH.as<int>());
    OMM_KCHECK();
    if (S) {
        T->eS.alloc(std::max(ncol, S->dim2) * sizeof(int));
        oz_colexp_kernel<<<(ncol + 255) / 256, 256, 0, st>>>(P.ngroups, P.G, S->dim2, PS.d_gptr, PS.d_bvals,
                                                             T->eS.as<int>());
        OMM_KCHECK();
    }
    const ModParams mp = mod_params(OZ_NMOD);
    T->bt.alloc_zero((size_t)OZ_NMOD * nsg * maxch * T->NB * 16);
    const int grid = (int)std::min<long long>(((long long)nent * P.G + 255) / 256, 148LL * 16);
    for (int half = 0; half < (S ? 2 : 1); ++half) {
        // standard layout: S's columns after H's in one NB-wide row; half-major: a Gs-wide row per half
        const int nb = halves ? Gs : T->NB, c0 = halves ? 0 : (half ? Gs : 0);
        oz_bt_kernel<<<grid, 256, 0, st>>>(nent, P.G, nb, c0, halves ? 2 * nsg : nsg, maxch, halves ? 2 : 1,
                                           halves ? half : 0, pp->gofk.as<int>(),
                                           pp->sgk.as<int>(), pp->coff.as<int>(), pp->cidx.as<int>(), pp->krow.as<int>(),
                                           half ? PS.d_bvals : P.d_bvals, (half ? T->eS : T->eH).as<int>(), bits, mp,
                                           T->bt.as<int8_t>());
        OMM_KCHECK();
    }
    T->ngroups = nsg;
    return T.get();
}

bool oz_spmm_available(const msw_matrix* H, const msw_matrix* S) {
    if (!H || H->fmt != Fmt::CSC || !H->is_real) return false;
    if (S && (S->fmt != Fmt::CSC || !S->is_real)) return false;
    if (H->dim1 >= (1 << 17) || H->dim1 != H->dim2) return false;
    if (g_oz_spmm_form == 3 && S && oz_spmm_plan(H, S, oz_bits(H->dim1, OZ_NMOD), 2, true)) return true;
    return oz_spmm_plan(H, S, oz_bits(H->dim1, OZ_NMOD), g_oz_spmm_form == 3 ? 1 : oz_spmm_sg(), false) != nullptr;
}

// Y (FP64, column-major, ld Y.ld) = A [H, S]: A's product with H in rows 0 .. n-1, with S in rows
// n .. 2n-1 (only H's when S is null); A given by its residues with the k-blocked copy.
namespace {
template <int STG, int PPS, int MINB, int HS>
void launch_oz_spmm(dim3 grid, const oz::OzSpParams& p, int cstride) {
    using namespace oz;
    const int smem = STG * sp_stage_bytes<PPS, HS>() + 1024 + 256 + cstride * (int)sizeof(int);
    static int attr = 0;
    if (smem > attr) {
        OMM_CK(cudaFuncSetAttribute(oz_spmm_kernel<STG, PPS, MINB, HS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    smem));
        attr = smem;
    }
    oz_spmm_kernel<STG, PPS, MINB, HS><<<grid, 192, smem, rt().stream>>>(p);
}
}  // namespace

bool oz_spmm(const msw_matrix* H, const msw_matrix* S, const OzOperand& A, DView& Y) {
    using namespace oz;
    const int n = A.rows, m = H->dim2;
    if (!A.kb.p || A.K != H->dim1 || A.nmod != OZ_NMOD) return false;
    if (!oz_spmm_available(H, S)) return false;
    // the layout of A's k-blocked copy decides: half-major goes to the SM-pair kernel
    const bool halves = A.kb_halves;
    if (halves && !S) return false;
    OzSpmmPlan* T = oz_spmm_plan(H, S, oz_bits(H->dim1, OZ_NMOD), halves ? 2 : (g_oz_spmm_form == 3 ? 1 : oz_spmm_sg()),
                                 halves);
    if (!T || T->bits != A.bits) return false;
    if (n % 4) return false;  // the reconstruction reads four rows' residues at a time
    const Table& tb = table(OZ_NMOD);
    const int ldr = (2 * n + 127) / 128 * 128;
    DevBuf& Rb = product_planes();
    const size_t rplane = (size_t)ldr * m;
    Rb.ensure(rplane * OZ_NMOD);
    OzSpParams p{};
    p.n = n;
    p.G = T->G;
    p.NB = T->NB;
    p.ngroups = T->ngroups;
    p.nch16 = A.ldk / 16;
    p.cstride = T->cstride;
    p.nmod = OZ_NMOD;
    p.ncol = m;
    p.idesc = (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(T->NB >> 3) << 17) |
              ((uint32_t)((halves ? 256 : 128) >> 4) << 24);
    p.a = A.kb.as<uint8_t>();
    p.a_plane = A.kb_plane;
    p.bt = T->bt.as<int8_t>();
    p.cx = T->pat->cx.as<int>();
    p.nsteps = T->pat->nsteps.as<int>();
    p.R = Rb.as<uint8_t>();
    p.rplane = rplane;
    p.ldr = ldr;
    p.pair = T->pair;
    for (int l = 0; l < OZ_NMOD; ++l) {
        const uint32_t pl = (uint32_t)tb.p[l];
        p.p[l] = tb.p[l];
        p.magic[l] = (uint32_t)(((1ull << 39) + pl - 1) / pl);
        p.off[l] = (uint32_t)(((1ull << 31) + pl - 1) / pl * pl);
    }
    p.err = tc_error_flag();
    p.wc = tc_wait_cfg();
    dim3 grid((n + 255) / 256, T->ngroups);
    ktime_begin();
    if (halves) {
        // at most four CTAs per SM, so that the four 128-column TMEM allocations always fit: a CTA
        // blocked in its allocation while its cluster peer waits at the cluster barrier could
        // otherwise wait on CTAs that wait on it.  228 KB of shared memory per SM, 1 KB reserved per
        // CTA: 48 KB or more per CTA leaves room for four.
        const int smem =
            std::max(48 * 1024, 3 * spp_stage_bytes<3>(T->NB / 2) + 1024 + 256 + T->cstride * (int)sizeof(int));
        static int attr = 0;
        if (smem > attr) {
            OMM_CK(cudaFuncSetAttribute(oz_spmm_pair_kernel<3, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
            attr = smem;
        }
        oz_spmm_pair_kernel<3, 3><<<dim3(2 * grid.x, grid.y), 192, smem, rt().stream>>>(p);
    } else if (T->sg == 2) launch_oz_spmm<4, 2, 2, 128>(grid, p, T->cstride);
    else if (g_oz_spmm_form == 1 || g_oz_spmm_form == 3) launch_oz_spmm<2, 3, 3, 64>(grid, p, T->cstride);
    else launch_oz_spmm<4, 1, 4, 64>(grid, p, T->cstride);
    OMM_KCHECK();
    // work: the FP64 flops of the product (2 nnz n), to compare with the FP64 SpMM it replaces
    ktime_end("oz_spmm_kernel", 2.0 * T->nnz * n);
    // the CRT reconstruction of each half
    RecParams rp{};
    rp.N = m;
    rp.nmod = OZ_NMOD;
    rp.rplane = rplane;
    rp.ldr = ldr;
    rp.eA = A.exps.as<int>();
    rp.shift = (A.bits - 1) + (T->bits - 1);
    rp.alpha = 1.0;
    rp.beta = 0.0;
    rp.ldo = Y.ld;
    rp.os = 1;
    rp.herm = 0;
    rp.n_off = 0;
    fill_rec_tables(rp, tb, OZ_NMOD);
    dim3 rg((n + 1023) / 1024, (m + 7) / 8);
    for (int half = 0; half < (S ? 2 : 1); ++half) {
        rp.M = n;
        rp.R = Rb.as<uint8_t>() + (size_t)half * n;
        rp.eB = (half ? T->eS : T->eH).as<int>();
        rp.out = Y.as<double>() + (size_t)half * n;
        ktime_begin();
        oz_reconstruct_kernel<<<rg, 256, 0, rt().stream>>>(rp);
        OMM_KCHECK();
        ktime_end("oz_reconstruct_kernel", recon_bytes(rp, n, m));
    }
    return true;
}

}  // namespace ommgpu

namespace ommgpu {

namespace {
int g_emu = -1;  // -1: not decided yet
}

void set_fp64_emu(int mode, long long panel_bytes) {
    g_emu = mode ? 1 : 0;
    g_panel_bytes = panel_bytes > 0 ? (size_t)panel_bytes : ((size_t)4 << 30);
}

bool fp64_emu_enabled() {
    if (g_emu < 0) {
        const char* v = std::getenv("OMM_GPU_FP64_GEMM");
        g_emu = (v && std::strcmp(v, "cublas") == 0) ? 0 : 1;
    }
    return g_emu == 1;
}

bool fp64_emu_worth(int M, int N, int K) {
    return K >= 64 && K < (1 << 17) && M >= 128 && N >= 128 && (double)M * N * K >= (double)(1 << 27);
}

void gemm_f64_emu(char opA, char opB, int M, int N, int K, double alpha, const DView& A, const DView& B, double beta,
                  DView& C, int herm, const int* b_exps) {
    OzOperand* oa = &oz_scratch(OZS_GEMM_A);
    OzOperand* ob = &oz_scratch(OZS_GEMM_B);
    const int bits = oz_bits(K, OZ_NMOD);
    // A_op (M x K): A itself ('n', rows contiguous) or A^T ('t', K contiguous)
    oz_prepare(A, opA != 'n', M, K, OZ_NMOD, bits, *oa);
    // B_op (N x K) = op(B)^T: B^T when op(B) = B ('n': K contiguous), B when op(B) = B^T ('t')
    oz_prepare(B, opB == 'n', N, K, OZ_NMOD, bits, *ob, false, -1, b_exps);
    oz_gemm(*oa, *ob, alpha, beta, C, herm);
}

// complex C = alpha op(A) op(B) + beta C (alpha, beta real; ops 'n', 't', 'c') as four real
// FP64-accurate products of the parts: with op(A) = Ar + i sA Ai and op(B) = Br + i sB Bi
// (s = -1 for 'c'),  Re C = Ar Br - sA sB Ai Bi,  Im C = sB Ar Bi + sA Ai Br
void gemm_z_emu(char opA, char opB, int M, int N, int K, double alpha, const DView& A, const DView& B, double beta,
                DView& C) {
    const int bits = oz_bits(K, OZ_NMOD);
    const double sA = opA == 'c' ? -1.0 : 1.0, sB = opB == 'c' ? -1.0 : 1.0;
    OzOperand& ar = oz_scratch(OZS_GEMM_A);
    OzOperand& ai = oz_scratch(OZS_GEMM_AI);
    OzOperand& br = oz_scratch(OZS_GEMM_B);
    OzOperand& bi = oz_scratch(OZS_GEMM_BI);
    oz_prepare(A, opA != 'n', M, K, OZ_NMOD, bits, ar, false, 0);
    oz_prepare(A, opA != 'n', M, K, OZ_NMOD, bits, ai, false, 1);
    oz_prepare(B, opB == 'n', N, K, OZ_NMOD, bits, br, false, 0);
    oz_prepare(B, opB == 'n', N, K, OZ_NMOD, bits, bi, false, 1);
    oz_gemm(ar, br, alpha, beta, C, 0, 0);
    oz_gemm(ai, bi, -sA * sB * alpha, 1.0, C, 0, 0);
    oz_gemm(ar, bi, sB * alpha, beta, C, 0, 1);
    oz_gemm(ai, br, sA * alpha, 1.0, C, 0, 1);
}

}  // namespace ommgpu

using namespace ommgpu;

extern "C" int omm_gpu_set_fp64_gemm(int mode, long long panel_bytes) {
    if (mode != 0 && mode != 1) {
        set_last_error("omm_gpu_set_fp64_gemm: mode must be 0 (cuBLAS) or 1 (int8 tensor cores)");
        return OMM_ERR_ARG;
    }
    set_fp64_emu(mode, panel_bytes);
    set_last_error("");
    return OMM_OK;
}

namespace {
// the argument checks and views shared by the two entry points below
void gemm_f64_entry(char opA, char opB, int M, int N, int K, double alpha, const double* A, int lda, const double* B,
                    int ldb, double beta, double* C, int ldc) {
    if (M < 0 || N < 0 || K < 0) fail(OMM_ERR_ARG, "gemm_f64: negative dimension");
    if ((opA != 'n' && opA != 't') || (opB != 'n' && opB != 't')) fail(OMM_ERR_ARG, "gemm_f64: ops are 'n' or 't'");
    const int ra = opA == 'n' ? M : K, rb = opB == 'n' ? K : N;
    if (lda < std::max(1, ra) || ldb < std::max(1, rb) || ldc < std::max(1, M))
        fail(OMM_ERR_ARG, "gemm_f64: leading dimension too small");
    if (K >= (1 << 17)) fail(OMM_ERR_ARG, "gemm_f64: K must be below 2^17");
    DView a, b, c;
    a.p = (void*)A;
    a.rows = ra;
    a.cols = opA == 'n' ? K : M;
    a.ld = lda;
    b.p = (void*)B;
    b.rows = rb;
    b.cols = opB == 'n' ? N : K;
    b.ld = ldb;
    c.p = C;
    c.rows = M;
    c.cols = N;
    c.ld = ldc;
    gemm_f64_emu(opA, opB, M, N, K, alpha, a, b, beta, c);
}
}  // namespace

extern "C" int omm_gpu_gemm_f64(char opA, char opB, int M, int N, int K, double alpha, const double* A, int lda,
                                const double* B, int ldb, double beta, double* C, int ldc) {
    try {
        gemm_f64_entry(opA, opB, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc);
        sync();
        unsigned e = gemm_bf16_errors();
        if (e) fail(OMM_ERR_CUDA, "gemm_f64: a pipeline wait timed out (error bits " + std::to_string(e) + ")");
    } catch (const Error& e) {
        set_last_error(e.msg);
        return e.code;
    }
    set_last_error("");
    return OMM_OK;
}

extern "C" int omm_gpu_gemm_f64_async(char opA, char opB, int M, int N, int K, double alpha, const double* A, int lda,
                                      const double* B, int ldb, double beta, double* C, int ldc) {
    try {
        gemm_f64_entry(opA, opB, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc);
    } catch (const Error& e) {
        set_last_error(e.msg);
        return e.code;
    }
    set_last_error("");
    return OMM_OK;
}

extern "C" int omm_gpu_spmm_f64(const double* A, int lda, int n, const msw_matrix* H, const msw_matrix* S, double* Y,
                                int ldy) {
    try {
        if (!A || !H || !Y || n <= 0) fail(OMM_ERR_ARG, "spmm_f64: null argument or empty A");
        if (H->fmt != Fmt::CSC || !H->is_real || (S && (S->fmt != Fmt::CSC || !S->is_real)))
            fail(OMM_ERR_ARG, "spmm_f64: real CSC matrices required");
        const int m = H->dim1;
        if (H->dim2 != m || (S && (S->dim1 != m || S->dim2 != m))) fail(OMM_ERR_ARG, "spmm_f64: square H, S of one order");
        if (lda < n || ldy < (S ? 2 : 1) * n) fail(OMM_ERR_ARG, "spmm_f64: leading dimension too small");
        if (m >= (1 << 17)) fail(OMM_ERR_ARG, "spmm_f64: the order must be below 2^17");
        ensure_csc_device(H);
        if (S) ensure_csc_device(S);
        if (!oz_spmm_available(H, S))
            fail(OMM_ERR_UNSUPPORTED, "spmm_f64: H (and S, same pattern) need column groups of at most 32 columns");
        DView a, y;
        a.p = (void*)A;
        a.rows = n;
        a.cols = m;
        a.ld = lda;
        y.p = Y;
        y.rows = (S ? 2 : 1) * n;
        y.cols = m;
        y.ld = ldy;
        OzOperand* op = &oz_scratch(OZS_SPMM_A);
        oz_prepare(a, false, n, m, OZ_NMOD, oz_bits(m, OZ_NMOD), *op, true, -1, nullptr, oz_spmm_kb_halves(S != nullptr));
        if (!oz_spmm(H, S, *op, y)) fail(OMM_ERR_UNSUPPORTED, "spmm_f64: n must be a multiple of 4");
        sync();
        unsigned e = gemm_bf16_errors();
        if (e) fail(OMM_ERR_CUDA, "spmm_f64: a pipeline wait timed out (error bits " + std::to_string(e) + ")");
    } catch (const Error& e) {
        set_last_error(e.msg);
        return e.code;
    }
    set_last_error("");
    return OMM_OK;
}

extern "C" int omm_gpu_set_oz_spmm_form(int form) {
    if (form < 0 || form > 3) {
        ommgpu::set_last_error("omm_gpu_set_oz_spmm_form: form 0, 1, 2 or 3");
        return OMM_ERR_ARG;
    }
    ommgpu::g_oz_spmm_form = form;
    return OMM_OK;
}
