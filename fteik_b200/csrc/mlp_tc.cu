/*
 * mlp_tc.cu -- the surrogate network's GEMMs on the tensor cores (tcgen05,
 * BF16 operands, FP32 accumulators in tensor memory).  No counterpart in the
 * reference.
 *
 * C[M][N] = sum_k A(m,k) B(k,n) (+ bias[n]) with the operand accessors of
 * the CUDA-core kernel (mlp.cu): A(m,k) = A[m lda + k] (ta = 0) or
 * A[k lda + m] (ta = 1); B(k,n) = B[k ldb + n] (tb = 0) or B[n ldb + k]
 * (tb = 1).  A CTA computes one 128 x 256 tile (M x N; N up to 256) over a
 * range of K (split K: partial tiles go to a workspace that a second kernel
 * adds in a fixed order).
 *
 * Each K block of 64 reaches shared memory as BF16 in the 128-byte-swizzled
 * K-major layout the MMA reads: FP32 values rounded to BF16 (PROD = 1) or
 * split into BF16 hi + lo parts (PROD = 3: products hi hi + hi lo + lo hi,
 * about FP32 accuracy).  With 16-byte aligned operands the FP32 values
 * arrive by cp.async copies into a ring of half-stages several blocks
 * ahead and are converted from shared memory (ASYNC); otherwise every
 * thread loads and converts each block directly (two stages).  One thread
 * issues the MMAs (kind::f16, 128 x 256 x 16 each) and commits them to an
 * mbarrier.  The epilogue reads the accumulators from tensor memory with
 * tcgen05.ld into a shared-memory tile and writes C row by row, with the
 * bias, the previous contents and the SiLU activation (or its derivative)
 * applied as asked.  Every mbarrier wait is bounded; on a timeout the CTA
 * sets the error word, lets its MMAs drain and frees its tensor memory.
 */
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "fteik_dev.h"

namespace fkmtc {

constexpr int BM = 128, BN = 256, BK = 64;
constexpr int NT = 256;
static_assert(NT == BN && NT == 2 * BM, "the staging maps a thread to one B row and half an A row");
constexpr int A_TILE = BM * BK * 2;   /* 16 KB of BF16 */
constexpr int B_TILE = BN * BK * 2;   /* 32 KB */
constexpr uint32_t TMEM_COLS = 256;
constexpr long long WAIT_LIMIT = 1ll << 24;

/* kind::f16 instruction descriptor: D FP32, A and B BF16, both K-major,
 * N >> 3 at bit 17, M >> 4 at bit 24 */
constexpr uint32_t IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) |
                           ((uint32_t)(BM >> 4) << 24);

/* FP32 half-stages of the asynchronous staging: 32 k of A (128 rows) and
 * B (256 columns) as copied from global memory */
constexpr int HK = 32;
constexpr int FA_BYTES = BM * HK * 4;   /* 16 KB */
constexpr int FB_BYTES = BN * HK * 4;   /* 32 KB */
constexpr int FSTAGE = FA_BYTES + FB_BYTES;

template <int PROD>
struct Cfg {
    static constexpr int NP = PROD == 3 ? 2 : 1;          /* hi (+ lo) copies */
    static constexpr int STAGE = NP * (A_TILE + B_TILE);
    static constexpr int SMEM = 2 * STAGE + 1024;         /* + alignment slack */
    /* asynchronous staging: a ring of NS FP32 half-stages and one BF16 stage */
    static constexpr int NS = PROD == 3 ? 2 : 3;
    static constexpr int SMEM_ASYNC = NS * FSTAGE + STAGE + 1024;
};

/* byte offset of element (row, k) in a swizzled K-major tile (rows of 128 B) */
__device__ __forceinline__ uint32_t swz(int row, int k)
{
    return (uint32_t)row * 128u + ((uint32_t)(((k >> 3) ^ (row & 7))) << 4) + (uint32_t)(k & 7) * 2u;
}

__device__ __forceinline__ uint64_t sdesc_sw128(uint32_t saddr)
{
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) |
           ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity)
{
    for (long long i = 0; i < WAIT_LIMIT; ++i)
        if (mbar_try(bar, parity)) return true;
    return false;
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void mma_bf16(uint32_t d, uint64_t a, uint64_t b, uint32_t acc)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d),
        "l"(a), "l"(b), "r"(IDESC), "r"(acc)
        : "memory");
}

__device__ __forceinline__ void mma_commit(uint32_t bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}

#define FKM_R8(i) "=r"(r[i]), "=r"(r[i + 1]), "=r"(r[i + 2]), "=r"(r[i + 3]), "=r"(r[i + 4]), \
                  "=r"(r[i + 5]), "=r"(r[i + 6]), "=r"(r[i + 7])

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t *r)
{
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : FKM_R8(0), FKM_R8(8), FKM_R8(16), FKM_R8(24)
        : "r"(taddr)
        : "memory");
}

__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

/* one value into the hi (and lo) tiles */
template <int PROD>
__device__ __forceinline__ void put(uint8_t *hi, uint8_t *lo, uint32_t off, float v)
{
    const __nv_bfloat16 h = __float2bfloat16_rn(v);
    *reinterpret_cast<__nv_bfloat16 *>(hi + off) = h;
    if (PROD == 3) *reinterpret_cast<__nv_bfloat16 *>(lo + off) = __float2bfloat16_rn(v - __bfloat162float(h));
}

/* 8 consecutive-k values (two float4) as one 16-byte swizzle unit of the hi
 * (and lo) tiles */
template <int PROD>
__device__ __forceinline__ void put8(uint8_t *hi, uint8_t *lo, uint32_t off, float4 a, float4 b)
{
    const float v[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
    uint32_t h[4], l[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const __nv_bfloat162 p = __floats2bfloat162_rn(v[2 * i], v[2 * i + 1]);
        h[i] = *reinterpret_cast<const uint32_t *>(&p);
        if (PROD == 3) {
            const __nv_bfloat162 q = __floats2bfloat162_rn(v[2 * i] - __low2float(p), v[2 * i + 1] - __high2float(p));
            l[i] = *reinterpret_cast<const uint32_t *>(&q);
        }
    }
    *reinterpret_cast<uint4 *>(hi + off) = make_uint4(h[0], h[1], h[2], h[3]);
    if (PROD == 3) *reinterpret_cast<uint4 *>(lo + off) = make_uint4(l[0], l[1], l[2], l[3]);
}

/* Stage the K block [k0, k0 + 64) of A (rows m0 ..) and B (columns n0 ..);
 * out-of-range elements are zero.  Rows with k contiguous in memory move in
 * 16-byte loads when the whole block is in range and aligned.  Operands
 * with m (n) contiguous move, when the whole block is in range, in units
 * of one row and 8 consecutive k: a warp's 32 units are 32 consecutive
 * rows, so each of a unit's 8 loads is one coalesced 128-byte segment and
 * the 8 values fill one 16-byte swizzle unit.  cs (A with m contiguous and
 * a full block only): the thread's A values are added to *cs, k in order
 * (the thread's row is t mod 128 in every block). */
template <int PROD>
__device__ __forceinline__ void stage(uint8_t *sA, uint8_t *sB, int M, int N, int K, const float *__restrict__ A,
                                      int lda, int ta, const float *__restrict__ B, int ldb, int tb, int m0, int n0,
                                      int k0, int k1, float *cs)
{
    uint8_t *aLo = sA + A_TILE, *bLo = sB + B_TILE;
    const int t = threadIdx.x;
    const bool kfull = k0 + BK <= k1;
    if (!ta && kfull && (lda & 3) == 0 && ((uintptr_t)A & 15) == 0) {
        const int row = t >> 1, kb = (t & 1) * 32, m = m0 + row;
        const float4 *src = reinterpret_cast<const float4 *>(A + (size_t)m * lda + k0 + kb);
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            float4 a = make_float4(0.f, 0.f, 0.f, 0.f), b = a;
            if (m < M) { a = src[2 * c]; b = src[2 * c + 1]; }
            put8<PROD>(sA, aLo, swz(row, kb + 8 * c), a, b);
        }
    } else if (ta && kfull) {
        const int row = t & (BM - 1), m = m0 + row;
#pragma unroll
        for (int j = 0; j < BM * (BK / 8) / NT; ++j) {
            const int g = (t >> 7) + 2 * j;
            const float *src = A + (size_t)(k0 + 8 * g) * lda + m;
            float v[8];
#pragma unroll
            for (int i = 0; i < 8; ++i) v[i] = m < M ? src[(size_t)i * lda] : 0.0f;
            if (cs)
#pragma unroll
                for (int i = 0; i < 8; ++i) *cs += v[i];
            put8<PROD>(sA, aLo, swz(row, 8 * g), make_float4(v[0], v[1], v[2], v[3]),
                       make_float4(v[4], v[5], v[6], v[7]));
        }
    } else if (!ta) {
        /* A[m][k], k contiguous: thread -> row t / 2, 32 consecutive k */
        const int row = t >> 1, kb = (t & 1) * 32, m = m0 + row;
#pragma unroll 8
        for (int i = 0; i < 32; ++i) {
            const int k = k0 + kb + i;
            const float v = (m < M && k < k1) ? A[(size_t)m * lda + k] : 0.0f;
            put<PROD>(sA, aLo, swz(row, kb + i), v);
        }
    } else {
        /* A[k][m], m contiguous: thread -> k = t / 4, 32 consecutive m */
        const int kk = t >> 2, mb = (t & 3) * 32, k = k0 + kk;
#pragma unroll 8
        for (int i = 0; i < 32; ++i) {
            const int m = m0 + mb + i;
            const float v = (m < M && k < k1) ? A[(size_t)k * lda + m] : 0.0f;
            put<PROD>(sA, aLo, swz(mb + i, kk), v);
        }
    }
    if (tb && kfull && (ldb & 3) == 0 && ((uintptr_t)B & 15) == 0) {
        const int n = n0 + t;
        const float4 *src = reinterpret_cast<const float4 *>(B + (size_t)n * ldb + k0);
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            float4 a = make_float4(0.f, 0.f, 0.f, 0.f), b = a;
            if (n < N) { a = src[2 * c]; b = src[2 * c + 1]; }
            put8<PROD>(sB, bLo, swz(t, 8 * c), a, b);
        }
    } else if (!tb && kfull) {
        const int n = n0 + t;
#pragma unroll 2
        for (int g = 0; g < BK / 8; ++g) {
            const float *src = B + (size_t)(k0 + 8 * g) * ldb + n;
            float v[8];
#pragma unroll
            for (int i = 0; i < 8; ++i) v[i] = n < N ? src[(size_t)i * ldb] : 0.0f;
            put8<PROD>(sB, bLo, swz(t, 8 * g), make_float4(v[0], v[1], v[2], v[3]),
                       make_float4(v[4], v[5], v[6], v[7]));
        }
    } else if (tb) {
        /* B[n][k], k contiguous: thread -> row n = t, 64 consecutive k */
        const int n = n0 + t;
#pragma unroll 8
        for (int i = 0; i < 64; ++i) {
            const int k = k0 + i;
            const float v = (n < N && k < k1) ? B[(size_t)n * ldb + k] : 0.0f;
            put<PROD>(sB, bLo, swz(t, i), v);
        }
    } else {
        /* B[k][n], n contiguous: thread -> k = t / 4, 64 consecutive n */
        const int kk = t >> 2, nb = (t & 3) * 64, k = k0 + kk;
#pragma unroll 8
        for (int i = 0; i < 64; ++i) {
            const int n = n0 + nb + i;
            const float v = (n < N && k < k1) ? B[(size_t)k * ldb + n] : 0.0f;
            put<PROD>(sB, bLo, swz(nb + i, kk), v);
        }
    }
    /* the generic-proxy writes become visible to the tensor cores' reads */
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

/* ---- asynchronous staging ---------------------------------------------
 * The FP32 operands come in by 16-byte cp.async copies (zero-filled outside
 * the matrices) into a ring of NS half-stages of 32 k, NS - 1 of them in
 * flight ahead of the one being converted, so global-memory latency is
 * hidden behind the conversion and the MMAs; every thread then converts a
 * landed half-stage into the BF16 stage exactly as stage() would (same
 * roundings, same swizzled layout, same order of the column sums).
 * Layouts of a half-stage: a k-contiguous operand as rows of 32 values
 * (128 B), chunk c of row r at chunk c ^ (r mod 8) (conflict-free 16-byte
 * reads of 8 consecutive rows); an m- (n-) contiguous operand as 32 rows of
 * k, 128 (256) values each.  Needs 16-byte aligned operands, leading
 * dimensions and contiguous extents that are multiples of 4. */
__device__ __forceinline__ void cp16(uint32_t dst, const float *src, bool ok)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(ok ? 16 : 0) : "memory");
}

__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }

template <int N_>
__device__ __forceinline__ void cp_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N_) : "memory"); }

/* The copies of one thread: 4 chunks of A and 8 of B per half-stage.
 * Pointers run along k (advance() moves them one half-stage on); the
 * destinations and the in-range tests follow from the thread index. */
template <int TA, int TB>
struct Copier {
    const float *pa[FA_BYTES / 16 / NT], *pb[FB_BYTES / 16 / NT];
    size_t sa, sb;   /* pointer step per half-stage */

    __device__ __forceinline__ Copier(const float *A, int lda, const float *B, int ldb, int m0, int n0, int k0)
    {
        const int t = threadIdx.x;
#pragma unroll
        for (int j = 0; j < FA_BYTES / 16 / NT; ++j) {
            const int q = t + NT * j;
            pa[j] = TA ? A + (size_t)(k0 + (q >> 5)) * lda + m0 + 4 * (q & 31)
                       : A + (size_t)(m0 + (q >> 3)) * lda + k0 + 4 * (q & 7);
        }
#pragma unroll
        for (int j = 0; j < FB_BYTES / 16 / NT; ++j) {
            const int q = t + NT * j;
            pb[j] = TB ? B + (size_t)(n0 + (q >> 3)) * ldb + k0 + 4 * (q & 7)
                       : B + (size_t)(k0 + (q >> 6)) * ldb + n0 + 4 * (q & 63);
        }
        sa = TA ? (size_t)HK * lda : HK;
        sb = TB ? HK : (size_t)HK * ldb;
    }

    /* the half-stage k in [k0, k0 + 32) into the ring slot at f (zero
     * outside the matrices, k1 = the end of this CTA's K range) */
    __device__ __forceinline__ void issue(uint32_t f, const float *A, const float *B, int M, int N, int m0, int n0,
                                          int k0, int k1) const
    {
        const int t = threadIdx.x;
#pragma unroll
        for (int j = 0; j < FA_BYTES / 16 / NT; ++j) {
            const int q = t + NT * j;
            if (!TA) {
                const int r = q >> 3, c = q & 7;
                const bool ok = m0 + r < M && k0 + 4 * c < k1;
                cp16(f + r * 128 + ((c ^ (r & 7)) << 4), ok ? pa[j] : A, ok);
            } else {
                const int r = q >> 5, c = q & 31;
                const bool ok = m0 + 4 * c < M && k0 + r < k1;
                cp16(f + r * 512 + c * 16, ok ? pa[j] : A, ok);
            }
        }
        f += FA_BYTES;
#pragma unroll
        for (int j = 0; j < FB_BYTES / 16 / NT; ++j) {
            const int q = t + NT * j;
            if (TB) {
                const int r = q >> 3, c = q & 7;
                const bool ok = n0 + r < N && k0 + 4 * c < k1;
                cp16(f + r * 128 + ((c ^ (r & 7)) << 4), ok ? pb[j] : B, ok);
            } else {
                const int r = q >> 6, c = q & 63;
                const bool ok = n0 + 4 * c < N && k0 + r < k1;
                cp16(f + r * 1024 + c * 16, ok ? pb[j] : B, ok);
            }
        }
    }

    __device__ __forceinline__ void advance()
    {
#pragma unroll
        for (int j = 0; j < FA_BYTES / 16 / NT; ++j) pa[j] += sa;
#pragma unroll
        for (int j = 0; j < FB_BYTES / 16 / NT; ++j) pb[j] += sb;
    }
};

/* a landed half-stage (slot f) into half hh (k 32 hh ..) of the BF16 stage */
template <int PROD>
__device__ __forceinline__ void convert_half(const uint8_t *f, uint8_t *sA, uint8_t *sB, int ta, int tb, int hh,
                                             float *cs)
{
    uint8_t *aLo = sA + A_TILE, *bLo = sB + B_TILE;
    const float *fA = reinterpret_cast<const float *>(f), *fB = reinterpret_cast<const float *>(f + FA_BYTES);
    const int t = threadIdx.x, row = t & (BM - 1);
#pragma unroll
    for (int j = 0; j < BM * (HK / 8) / NT; ++j) {
        const int g = (t >> 7) + 2 * j;
        float v[8];
        if (!ta) {
            const float4 a = *reinterpret_cast<const float4 *>(fA + row * 32 + (((2 * g) ^ (row & 7)) << 2));
            const float4 b = *reinterpret_cast<const float4 *>(fA + row * 32 + (((2 * g + 1) ^ (row & 7)) << 2));
            v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w; v[4] = b.x; v[5] = b.y; v[6] = b.z; v[7] = b.w;
        } else {
#pragma unroll
            for (int i = 0; i < 8; ++i) v[i] = fA[(8 * g + i) * BM + row];
            if (cs)
#pragma unroll
                for (int i = 0; i < 8; ++i) *cs += v[i];
        }
        put8<PROD>(sA, aLo, swz(row, HK * hh + 8 * g), make_float4(v[0], v[1], v[2], v[3]),
                   make_float4(v[4], v[5], v[6], v[7]));
    }
#pragma unroll
    for (int g = 0; g < HK / 8; ++g) {
        float v[8];
        if (tb) {
            const float4 a = *reinterpret_cast<const float4 *>(fB + t * 32 + (((2 * g) ^ (t & 7)) << 2));
            const float4 b = *reinterpret_cast<const float4 *>(fB + t * 32 + (((2 * g + 1) ^ (t & 7)) << 2));
            v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w; v[4] = b.x; v[5] = b.y; v[6] = b.z; v[7] = b.w;
        } else {
#pragma unroll
            for (int i = 0; i < 8; ++i) v[i] = fB[(8 * g + i) * BN + t];
        }
        put8<PROD>(sB, bLo, swz(t, HK * hh + 8 * g), make_float4(v[0], v[1], v[2], v[3]),
                   make_float4(v[4], v[5], v[6], v[7]));
    }
}

/* the MMAs of one BF16 stage (K 64), accumulating unless first */
template <int PROD>
__device__ __forceinline__ void issue_mmas(uint32_t tmem, const uint8_t *sA, const uint8_t *sB, bool first)
{
    const uint32_t a_hi = (uint32_t)__cvta_generic_to_shared(sA), a_lo = a_hi + A_TILE;
    const uint32_t b_hi = (uint32_t)__cvta_generic_to_shared(sB), b_lo = b_hi + B_TILE;
#pragma unroll
    for (int kk = 0; kk < BK / 16; ++kk) {
        const uint32_t ko = (uint32_t)kk * 32u;
        mma_bf16(tmem, sdesc_sw128(a_hi + ko), sdesc_sw128(b_hi + ko), (!first || kk > 0) ? 1u : 0u);
        if (PROD == 3) {
            mma_bf16(tmem, sdesc_sw128(a_hi + ko), sdesc_sw128(b_lo + ko), 1u);
            mma_bf16(tmem, sdesc_sw128(a_lo + ko), sdesc_sw128(b_hi + ko), 1u);
        }
    }
}

/* ---- epilogue ----------------------------------------------------------
 * The accumulators go through a [128][TS] FP32 tile in shared memory (row
 * stride 132: 16-byte rows; the float4 writes of 8 consecutive rows and
 * the float4 reads of one row are both conflict-free), one 128-column half
 * at a time, then out by rows: lane l of a warp holds columns 4 l .. 4 l + 3
 * of the half, so a row is one 512-byte store.  MODE: 0 C = v; 1 C = v and
 * C2 = silu(v); 2 C = silu(v); 3 C = v silu'(z), z = C2; 4 split-K partial
 * tile (C = the workspace slice, no bias).  The bias and the previous
 * contents are added first where asked (modes 0-3). */
constexpr int TS = 132;
static_assert(BM * TS * 4 <= 2 * FSTAGE && BM * TS * 4 <= 2 * Cfg<1>::STAGE, "the epilogue tile fits the stages");

__device__ __forceinline__ float silu_bwd1(float v, float z)
{
    const float sg = fk_sigmoid(z);
    return v * sg * (1.0f + z * (1.0f - sg));
}

template <int MODE>
__device__ __forceinline__ void epi_rows_vec(const float *tile, int warp, int lane, int m0, int M, int N, int nc0,
                                             float *__restrict__ C, size_t ldc, const float *__restrict__ bias,
                                             int accumulate, float *__restrict__ C2)
{
    const int n = nc0 + 4 * lane;
    if (n >= N) return;   /* N is a multiple of 4: a lane's columns are all in or all out */
    float4 bv = make_float4(0.f, 0.f, 0.f, 0.f);
    if (MODE != 4 && bias) bv = make_float4(bias[n], bias[n + 1], bias[n + 2], bias[n + 3]);
    for (int r0 = warp; r0 < BM; r0 += 4 * (NT / 32)) {
        float4 zv[4];
        if (MODE == 3) {
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int m = m0 + r0 + j * (NT / 32);
                zv[j] = m < M ? *reinterpret_cast<const float4 *>(C2 + (size_t)m * ldc + n) : make_float4(0.f, 0.f, 0.f, 0.f);
            }
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int rr = r0 + j * (NT / 32), m = m0 + rr;
            if (m >= M) break;
            float4 v = *reinterpret_cast<const float4 *>(tile + rr * TS + 4 * lane);
            float4 *c = reinterpret_cast<float4 *>(C + (size_t)m * ldc + n);
            if (MODE == 4) { *c = v; continue; }
            if (bias) { v.x += bv.x; v.y += bv.y; v.z += bv.z; v.w += bv.w; }
            if (accumulate) {
                const float4 o = *c;
                v.x = o.x + v.x; v.y = o.y + v.y; v.z = o.z + v.z; v.w = o.w + v.w;
            }
            if (MODE == 0) *c = v;
            if (MODE == 1) {
                *c = v;
                *reinterpret_cast<float4 *>(C2 + (size_t)m * ldc + n) =
                    make_float4(fk_silu(v.x), fk_silu(v.y), fk_silu(v.z), fk_silu(v.w));
            }
            if (MODE == 2) *c = make_float4(fk_silu(v.x), fk_silu(v.y), fk_silu(v.z), fk_silu(v.w));
            if (MODE == 3)
                *c = make_float4(silu_bwd1(v.x, zv[j].x), silu_bwd1(v.y, zv[j].y), silu_bwd1(v.z, zv[j].z),
                                 silu_bwd1(v.w, zv[j].w));
        }
    }
}

/* the same for any alignment: lane l holds columns l, l + 32, l + 64, l + 96 */
__device__ __forceinline__ void epi_rows_scalar(const float *tile, int warp, int lane, int m0, int M, int N, int nc0,
                                                float *__restrict__ C, size_t ldc, const float *__restrict__ bias,
                                                int accumulate, float *__restrict__ C2, int mode)
{
    for (int rr = warp; rr < BM; rr += NT / 32) {
        const int m = m0 + rr;
        if (m >= M) break;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int n = nc0 + i * 32 + lane;
            if (n >= N) continue;
            float v = tile[rr * TS + i * 32 + lane];
            float *c = C + (size_t)m * ldc + n;
            if (mode == 4) { *c = v; continue; }
            if (bias) v += bias[n];
            if (accumulate) v = *c + v;
            if (mode == 3) *c = silu_bwd1(v, C2[(size_t)m * ldc + n]);
            else if (mode == 2) *c = fk_silu(v);
            else {
                *c = v;
                if (mode == 1) C2[(size_t)m * ldc + n] = fk_silu(v);
            }
        }
    }
}

template <int PROD, bool ASYNC, int TA, int TB>
__global__ void __launch_bounds__(NT, 1) gemm_tc_kernel(int M, int N, int K, const float *__restrict__ A, int lda,
                                                        const float *__restrict__ B, int ldb,
                                                        float *__restrict__ C, int ldc,
                                                        const float *__restrict__ bias, int accumulate,
                                                        float *__restrict__ C2, int act, int kchunk,
                                                        float *__restrict__ colsum, int *error)
{
    constexpr int ta = TA, tb = TB;
    using G = Cfg<PROD>;
    extern __shared__ uint8_t smem_raw[];
    __shared__ __align__(8) uint64_t bars[2];
    __shared__ uint32_t s_tmem;
    __shared__ int s_fail;
    __shared__ float s_cs[BM];
    uint8_t *base = reinterpret_cast<uint8_t *>(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
    const int kb = blockIdx.z * kchunk, ke = min(K, kb + kchunk);
    const int nkb = (ke - kb + BK - 1) / BK;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t bar0 = (uint32_t)__cvta_generic_to_shared(&bars[0]);
    if (threadIdx.x == 0) {
        mbar_init(bar0, 1);
        mbar_init(bar0 + 8, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        s_fail = 0;
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         (uint32_t)__cvta_generic_to_shared(&s_tmem)),
                     "r"(TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = s_tmem;
    int committed = 0;
    uint32_t last_bar = bar0, last_par = 0;   /* the barrier and parity of the last commit */
    float cs = 0.0f;   /* colsum: this thread's A values (row t mod 128) */
    if constexpr (ASYNC) {
        const uint32_t ring = (uint32_t)__cvta_generic_to_shared(base);
        uint8_t *sA = base + G::NS * FSTAGE, *sB = sA + G::NP * A_TILE;
        const int nh = 2 * nkb;
        Copier<TA, TB> cp(A, lda, B, ldb, m0, n0, kb);
#pragma unroll
        for (int h = 0; h < G::NS - 1; ++h) {
            if (h < nh) {
                cp.issue(ring + h * FSTAGE, A, B, M, N, m0, n0, kb + h * HK, ke);
                cp.advance();
            }
            cp_commit();
        }
        for (int h = 0; h < nh; ++h) {
            const int b = h >> 1, hh = h & 1;
            cp_wait<G::NS - 2>();   /* this thread's copies of half-stage h have landed */
            __syncthreads();        /* everyone's have; slot (h - 1) mod NS is converted */
            if (s_fail) break;
            {
                const int hn = h + G::NS - 1;
                if (hn < nh) {
                    cp.issue(ring + (hn % G::NS) * FSTAGE, A, B, M, N, m0, n0, kb + hn * HK, ke);
                    cp.advance();
                }
                cp_commit();
            }
            /* the MMAs of stage b - 1 read the BF16 stage */
            if (hh == 0 && b > 0 && !mbar_wait(bar0, (b - 1) & 1)) {
                atomicCAS(error, 0, 1);
                s_fail = 1;
                continue;
            }
            convert_half<PROD>(base + (h % G::NS) * FSTAGE, sA, sB, ta, tb, hh, colsum ? &cs : nullptr);
            if (hh == 1) {
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                __syncthreads();
                if (s_fail) break;
                if (threadIdx.x == 0) {
                    tc_fence_after();
                    issue_mmas<PROD>(tmem, sA, sB, b == 0);
                    mma_commit(bar0);
                }
                committed = b + 1;
                last_par = (uint32_t)(b & 1);
            }
        }
        cp_wait<0>();
    } else {
        for (int b = 0; b < nkb; ++b) {
            const int buf = b & 1;
            uint8_t *sA = base + buf * G::STAGE;
            uint8_t *sB = sA + G::NP * A_TILE;
            if (b >= 2 && !mbar_wait(bar0 + 8u * buf, ((b - 2) >> 1) & 1)) {   /* the MMAs of b - 2 read this stage */
                if (threadIdx.x == 0) { atomicCAS(error, 0, 1); s_fail = 1; }
            }
            __syncthreads();
            if (s_fail) break;
            stage<PROD>(sA, sB, M, N, K, A, lda, ta, B, ldb, tb, m0, n0, kb + b * BK, ke, colsum ? &cs : nullptr);
            __syncthreads();
            if (threadIdx.x == 0) {
                tc_fence_after();
                issue_mmas<PROD>(tmem, sA, sB, b == 0);
                mma_commit(bar0 + 8u * buf);
            }
            committed = b + 1;
            last_bar = bar0 + 8u * buf;
            last_par = (uint32_t)((b >> 1) & 1);
        }
    }
    /* every MMA of this CTA has completed: the last commit covers them all */
    bool ok = !s_fail;
    if (committed > 0 && !mbar_wait(last_bar, last_par)) {
        ok = false;
        atomicCAS(error, 0, 2);
    }
    if (colsum && threadIdx.x >= BM) s_cs[threadIdx.x - BM] = cs;
    ok = __syncthreads_and(ok) != 0;   /* the epilogue's barriers need every thread on one path */
    tc_fence_after();
    if (colsum && threadIdx.x < BM && m0 + (int)threadIdx.x < M)
        colsum[(size_t)blockIdx.z * M + m0 + threadIdx.x] = cs + s_cs[threadIdx.x];
    if (ok && committed == 0 && gridDim.z > 1) {
        /* a split-K slice past the end of K: its partial tile is zero */
        for (int e = threadIdx.x; e < BM * BN; e += NT) {
            const int m = m0 + e / BN, n = n0 + e % BN;
            if (m < M && n < N) C[((size_t)blockIdx.z * M + m) * N + n] = 0.0f;
        }
    }
    if (ok && committed > 0) {
        /* the operand stages are free (every MMA has completed): the warps
         * holding a 128-column half read their 32 TMEM lanes into the tile,
         * then every warp stores rows */
        float *tile = reinterpret_cast<float *>(base);
        const int q = warp & 3, half = warp >> 2;
        const int mode = gridDim.z > 1 ? 4 : act;
        float *Cb = gridDim.z > 1 ? C + (size_t)blockIdx.z * M * N : C;
        const size_t ldo = gridDim.z > 1 ? (size_t)N : (size_t)ldc;
        const bool vec = (N & 3) == 0 && (ldo & 3) == 0 && ((uintptr_t)Cb & 15) == 0 &&
                         (!(mode == 1 || mode == 3) || ((uintptr_t)C2 & 15) == 0);
        for (int p = 0; p < 2; ++p) {
            if (half == p) {
#pragma unroll 1
                for (int c = 0; c < 128; c += 32) {
                    uint32_t r[32];
                    tmem_ld32(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(p * 128 + c), r);
                    tmem_wait_ld();
                    float4 *trow = reinterpret_cast<float4 *>(tile + (q * 32 + lane) * TS + c);
#pragma unroll
                    for (int j = 0; j < 8; ++j)
                        trow[j] = make_float4(__uint_as_float(r[4 * j]), __uint_as_float(r[4 * j + 1]),
                                              __uint_as_float(r[4 * j + 2]), __uint_as_float(r[4 * j + 3]));
                }
            }
            __syncthreads();
            const int nc0 = n0 + p * 128;
            if (!vec)
                epi_rows_scalar(tile, warp, lane, m0, M, N, nc0, Cb, ldo, bias, accumulate, C2, mode);
            else if (mode == 4)
                epi_rows_vec<4>(tile, warp, lane, m0, M, N, nc0, Cb, ldo, nullptr, 0, nullptr);
            else if (mode == 1)
                epi_rows_vec<1>(tile, warp, lane, m0, M, N, nc0, Cb, ldo, bias, accumulate, C2);
            else if (mode == 2)
                epi_rows_vec<2>(tile, warp, lane, m0, M, N, nc0, Cb, ldo, bias, accumulate, C2);
            else if (mode == 3)
                epi_rows_vec<3>(tile, warp, lane, m0, M, N, nc0, Cb, ldo, bias, accumulate, C2);
            else
                epi_rows_vec<0>(tile, warp, lane, m0, M, N, nc0, Cb, ldo, bias, accumulate, C2);
            __syncthreads();
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
    }
}

/* ---- fused forward pass ----------------------------------------------------
 * The whole network for 128 rows in one CTA, BF16 operands (products mode
 * 1), the activations never leaving the SM: layer 0 (6 inputs) on the CUDA
 * cores into a BF16 A tile in shared memory (128 rows x 256, four 64-wide
 * K blocks in the MMA's swizzled layout), each hidden layer as 16 MMAs
 * (128 x 256 x 16) into tensor memory with the layer's BF16 weights
 * (packed once per call, 128 KB) brought into shared memory by four bulk
 * copies while the previous layer's epilogue runs, the epilogue adding the
 * bias, applying SiLU and writing the next A tile, and the last hidden
 * layer's epilogue forming the output row by row.  Every rounding and sum
 * is the layer-by-layer path's: the same MMAs in the same K order, the
 * same BF16 roundings of the FP32 activations, the first and last layers'
 * multiply-add chains in the same k order (the last one split between the
 * four warps holding a row's column quarters, each continuing the previous
 * one's chain), so tau is the same bits.  CTAs loop over row tiles; waits are
 * bounded. */
constexpr int FW = 256;                   /* hidden width */
constexpr int F_ABLK = BM * 64 * 2;       /* 16 KB: one 64-wide K block of the A tile */
constexpr int F_WBLK = FW * 64 * 2;       /* 32 KB: one K block of a layer's weights */
/* layer 0's weights and biases in shared memory, [6 + 1][4 column quarters][66]
 * (a quarter's 64 columns padded to 66 floats: the four quarters a warp
 * reads fall in different banks) */
constexpr int F_L0Q = 66;
constexpr int F_L0 = 7 * 4 * F_L0Q * 4;
constexpr int F_SMEM = 4 * F_ABLK + 4 * F_WBLK + F_L0 + 1024;
constexpr int F_MAXH = 8;
constexpr int F_NT = 512;                 /* 16 warps: 4 per TMEM lane quarter, 64 columns each */

struct FusedNet {
    const float *w;                       /* all weights and biases, FP32 */
    int nh;                               /* hidden 256 x 256 layers (1 .. F_MAXH) */
    long long woff[F_MAXH + 2], boff[F_MAXH + 2];   /* layer 0, hidden 1 .. nh, last nh + 1 */
};

/* wq[l - 1][kb][swz(n, k)]: hidden layer l's W[n][64 kb + k] in BF16 */
__global__ void fused_pack_kernel(FusedNet net, uint8_t *__restrict__ wq)
{
    const long long total = (long long)net.nh * FW * FW;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const int l = (int)(e / (FW * FW)), n = (int)((e / FW) % FW), k = (int)(e % FW);
        const float v = net.w[net.woff[l + 1] + (long long)n * FW + k];
        uint8_t *blk = wq + ((size_t)l * 4 + (k >> 6)) * F_WBLK;
        *reinterpret_cast<__nv_bfloat16 *>(blk + swz(n, k & 63)) = __float2bfloat16_rn(v);
    }
}

__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void *src, uint32_t bytes, uint32_t bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ float silu_f(float v) { return fk_silu(v); }

/* 8 activations of one row as one 16-byte unit of the A tile (k = n0 .. n0 + 7) */
__device__ __forceinline__ void put_a8(uint8_t *A, int row, int n0, const float (&a)[8])
{
    uint32_t h[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const __nv_bfloat162 p = __floats2bfloat162_rn(a[2 * i], a[2 * i + 1]);
        h[i] = *reinterpret_cast<const uint32_t *>(&p);
    }
    *reinterpret_cast<uint4 *>(A + (n0 >> 6) * F_ABLK + swz(row, n0 & 63)) = make_uint4(h[0], h[1], h[2], h[3]);
}

__global__ void __launch_bounds__(F_NT, 1) mlp_fused_fwd_kernel(FusedNet net, const uint8_t *__restrict__ wq,
                                                              long long n, const float *__restrict__ x,
                                                              float *__restrict__ tau, int *error)
{
    extern __shared__ uint8_t smem_raw[];
    __shared__ __align__(8) uint64_t bars[2];   /* 0: weights landed, 1: MMAs done */
    __shared__ uint32_t s_tmem;
    __shared__ float s_part[BM];
    uint8_t *A = reinterpret_cast<uint8_t *>(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    uint8_t *W = A + 4 * F_ABLK;
    float *l0 = reinterpret_cast<float *>(W + 4 * F_WBLK);   /* [k (6 weights, then the bias)][quarter][66] */
    const uint32_t a_s = (uint32_t)__cvta_generic_to_shared(A), w_s = (uint32_t)__cvta_generic_to_shared(W);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t bar_w = (uint32_t)__cvta_generic_to_shared(&bars[0]), bar_m = bar_w + 8;
    if (tid == 0) {
        mbar_init(bar_w, 1);
        mbar_init(bar_m, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         (uint32_t)__cvta_generic_to_shared(&s_tmem)),
                     "r"(TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    {
        const float *w0 = net.w + net.woff[0], *b0 = net.w + net.boff[0];
        for (int e = tid; e < 7 * FW; e += F_NT) {
            const int k = e / FW, col = e % FW;
            l0[(k * 4 + (col >> 6)) * F_L0Q + (col & 63)] = k < 6 ? w0[col * 6 + k] : b0[col];
        }
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = s_tmem;
    const long long ntile = (n + BM - 1) / BM;
    int nw_done = 0, nm_done = 0;
    bool w_pending = false;   /* thread 0: a weight load not yet waited for */
    auto load_w = [&](int l) {   /* hidden layer l's weights (thread 0) */
        mbar_expect_tx(bar_w, 4 * F_WBLK);
        const uint8_t *src = wq + (size_t)(l - 1) * 4 * F_WBLK;
#pragma unroll
        for (int kb = 0; kb < 4; ++kb) bulk_g2s(w_s + kb * F_WBLK, src + (size_t)kb * F_WBLK, F_WBLK, bar_w);
    };
    if (tid == 0 && blockIdx.x < ntile) { load_w(1); w_pending = true; }
    bool ok = true;
    for (long long tile = blockIdx.x; tile < ntile && ok; tile += gridDim.x) {
        const long long row0 = tile * BM;
        /* layer 0: row tid / 4, columns 64 (tid % 4) .. + 63 */
        {
            const int r = tid >> 2, h = tid & 3;
            const long long m = row0 + r;
            float xi[6];
#pragma unroll
            for (int k = 0; k < 6; ++k) xi[k] = m < n ? x[m * 6 + k] : 0.0f;
            /* two columns per packed multiply-add: each lane of the pair is the
             * scalar chain fmaf(x_k, w_k, acc) over k = 0 .. 5, as in the
             * layer-by-layer GEMM */
            const float *lq = l0 + h * F_L0Q;
#pragma unroll 1
            for (int c = 0; c < 64; c += 8) {
                float a[8];
#pragma unroll
                for (int j = 0; j < 8; j += 2) {
                    float2 acc = make_float2(0.0f, 0.0f);
#pragma unroll
                    for (int k = 0; k < 6; ++k)
                        acc = __ffma2_rn(make_float2(xi[k], xi[k]),
                                         *reinterpret_cast<const float2 *>(lq + k * 4 * F_L0Q + c + j), acc);
                    const float2 b = *reinterpret_cast<const float2 *>(lq + 6 * 4 * F_L0Q + c + j);
                    a[j] = silu_f(acc.x + b.x);
                    a[j + 1] = silu_f(acc.y + b.y);
                }
                put_a8(A, r, h * 64 + c, a);
            }
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        for (int l = 1; l <= net.nh && ok; ++l) {
            if (tid == 0) {
                if (!mbar_wait(bar_w, nw_done & 1)) { atomicCAS(error, 0, 3); ok = false; }
                else w_pending = false;
                if (ok) {
                    tc_fence_after();
#pragma unroll
                    for (int kb = 0; kb < 4; ++kb)
#pragma unroll
                        for (int kk = 0; kk < 4; ++kk)
                            mma_bf16(tmem, sdesc_sw128(a_s + kb * F_ABLK + kk * 32),
                                     sdesc_sw128(w_s + kb * F_WBLK + kk * 32), (kb | kk) ? 1u : 0u);
                    mma_commit(bar_m);
                }
            }
            ++nw_done;
            ok = __syncthreads_and(ok) != 0;
            if (!ok) break;
            if (!mbar_wait(bar_m, nm_done & 1)) { atomicCAS(error, 0, 4); ok = false; }
            ++nm_done;
            ok = __syncthreads_and(ok) != 0;
            if (!ok) break;
            tc_fence_after();
            /* the MMAs are done with A and W: the next weights come in during the epilogue */
            const bool more = l < net.nh || tile + gridDim.x < ntile;
            if (more && tid == 0) { load_w(l < net.nh ? l + 1 : 1); w_pending = true; }
            /* warp w: TMEM lanes 32 (w mod 4) .. + 31 (rows), columns 64 (w / 4) .. + 63 */
            const int q = warp & 3, cq = warp >> 2, row = q * 32 + lane;
            const float *bl = net.w + net.boff[l];
            if (l < net.nh) {
#pragma unroll 1
                for (int c = 0; c < 64; c += 32) {
                    uint32_t r[32];
                    tmem_ld32(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(cq * 64 + c), r);
                    tmem_wait_ld();
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        float a[8];
#pragma unroll
                        for (int j = 0; j < 8; ++j) {
                            const int col = cq * 64 + c + 8 * u + j;
                            a[j] = silu_f(__uint_as_float(r[8 * u + j]) + __ldg(bl + col));
                        }
                        put_a8(A, row, cq * 64 + c + 8 * u, a);
                    }
                }
            } else {
                /* last hidden layer: the output's multiply-add chain over the 256
                 * activations in order, each column quarter's warp continuing
                 * the previous quarter's chain */
                const float *wl = net.w + net.woff[l + 1];
                for (int p = 0; p < 4; ++p) {
                    if (cq == p) {
                        float acc = p ? s_part[row] : 0.0f;
#pragma unroll 1
                        for (int c = 0; c < 64; c += 32) {
                            uint32_t r[32];
                            tmem_ld32(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(p * 64 + c), r);
                            tmem_wait_ld();
#pragma unroll
                            for (int j = 0; j < 32; ++j) {
                                const int col = p * 64 + c + j;
                                const float a = silu_f(__uint_as_float(r[j]) + __ldg(bl + col));
                                acc = fmaf(a, __ldg(wl + col), acc);
                            }
                        }
                        if (p < 3) s_part[row] = acc;
                        else if (row0 + row < n) tau[row0 + row] = acc + __ldg(net.w + net.boff[l + 1]);
                    }
                    __syncthreads();
                }
            }
            tc_fence_before();
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            __syncthreads();
        }
    }
    /* a weight load still in flight ends before the CTA does */
    if (tid == 0 && w_pending && !mbar_wait(bar_w, nw_done & 1)) atomicCAS(error, 0, 5);
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
    }
}

} // namespace fkmtc

/* 1: stage the operands asynchronously where their alignment allows (the
 * default); 0: always synchronously.  Both give the same bits. */
static int g_async = 1;
extern "C" void fk_mlp_set_async_staging(int on) { g_async = on != 0; }

template <int PROD, bool ASYNC, int TA, int TB>
static cudaError_t launch_tc(dim3 grid, cudaStream_t s, int M, int N, int K, const float *A, int lda,
                             const float *B, int ldb, float *C, int ldc, const float *bias, int accumulate,
                             float *C2, int act, int kchunk, float *colsum, int *error)
{
    using namespace fkmtc;
    const int smem = ASYNC ? Cfg<PROD>::SMEM_ASYNC : Cfg<PROD>::SMEM;
    cudaError_t e = cudaFuncSetAttribute(gemm_tc_kernel<PROD, ASYNC, TA, TB>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    gemm_tc_kernel<PROD, ASYNC, TA, TB><<<grid, NT, smem, s>>>(M, N, K, A, lda, B, ldb, C, ldc, bias, accumulate,
                                                               C2, act, kchunk, colsum, error);
    return cudaGetLastError();
}

template <int PROD, bool ASYNC>
static cudaError_t launch_tc_layout(int ta, int tb, dim3 grid, cudaStream_t s, int M, int N, int K, const float *A,
                                    int lda, const float *B, int ldb, float *C, int ldc, const float *bias,
                                    int accumulate, float *C2, int act, int kchunk, float *colsum, int *error)
{
    if (!ta && tb)
        return launch_tc<PROD, ASYNC, 0, 1>(grid, s, M, N, K, A, lda, B, ldb, C, ldc, bias, accumulate, C2, act,
                                            kchunk, colsum, error);
    if (!ta && !tb)
        return launch_tc<PROD, ASYNC, 0, 0>(grid, s, M, N, K, A, lda, B, ldb, C, ldc, bias, accumulate, C2, act,
                                            kchunk, colsum, error);
    if (ta && !tb)
        return launch_tc<PROD, ASYNC, 1, 0>(grid, s, M, N, K, A, lda, B, ldb, C, ldc, bias, accumulate, C2, act,
                                            kchunk, colsum, error);
    return launch_tc<PROD, ASYNC, 1, 1>(grid, s, M, N, K, A, lda, B, ldb, C, ldc, bias, accumulate, C2, act, kchunk,
                                        colsum, error);
}

/* Launch one tensor-core GEMM (PROD 1 or 3); ws: split-K workspace of split
 * M N floats, or NULL for split = 1; colsum (A[k][m] with K a multiple of
 * 64, or NULL): [split][M] sums over each slice's k of A(m, k); error:
 * device word set on a wait timeout.  Returns a cudaError_t. */
extern "C" int fk_mlp_gemm_tc(int prod, int M, int N, int K, const float *A, int lda, int ta, const float *B,
                              int ldb, int tb, float *C, int ldc, const float *bias, int accumulate, float *C2,
                              int act, int split, float *ws, float *colsum, int *error, cudaStream_t s)
{
    using namespace fkmtc;
    if (M <= 0 || N <= 0 || K <= 0) return 0;
    if (N > BN || (prod != 1 && prod != 3) || (split > 1 && !ws)) return (int)cudaErrorInvalidValue;
    if (colsum && (!ta || K % BK)) return (int)cudaErrorInvalidValue;   /* only full blocks of A[k][m] */
    const int kchunk = ((K + split * BK - 1) / (split * BK)) * BK;
    const dim3 grid(1, (M + BM - 1) / BM, split);
    float *Cw = split > 1 ? ws : C;
    const int ldw = split > 1 ? N : ldc, accw = split > 1 ? 0 : accumulate, actw = split > 1 ? 0 : act;
    const float *bw = split > 1 ? nullptr : bias;
    /* 16-byte copies: aligned operands, leading dimensions and contiguous extents in fours */
    const bool async = g_async && ((uintptr_t)A & 15) == 0 && ((uintptr_t)B & 15) == 0 && lda % 4 == 0 &&
                       ldb % 4 == 0 && K % 4 == 0 && (!ta || M % 4 == 0) && (tb || N % 4 == 0);
    cudaError_t e;
    if (prod == 3)
        e = async ? launch_tc_layout<3, true>(ta, tb, grid, s, M, N, K, A, lda, B, ldb, Cw, ldw, bw, accw, C2, actw,
                                              kchunk, colsum, error)
                  : launch_tc_layout<3, false>(ta, tb, grid, s, M, N, K, A, lda, B, ldb, Cw, ldw, bw, accw, C2, actw,
                                               kchunk, colsum, error);
    else
        e = async ? launch_tc_layout<1, true>(ta, tb, grid, s, M, N, K, A, lda, B, ldb, Cw, ldw, bw, accw, C2, actw,
                                              kchunk, colsum, error)
                  : launch_tc_layout<1, false>(ta, tb, grid, s, M, N, K, A, lda, B, ldb, Cw, ldw, bw, accw, C2, actw,
                                               kchunk, colsum, error);
    return (int)e;
}

/* The fused forward pass of n rows (x [n][6] device, tau [n] device) of a
 * network with nh hidden 256 x 256 layers; wq: 128 KB per hidden layer of
 * scratch for the packed weights.  Returns a cudaError_t. */
extern "C" int fk_mlp_forward_fused(const float *w, int nh, const long long *woff, const long long *boff,
                                    long long n, const float *x, float *tau, unsigned char *wq, int *error,
                                    cudaStream_t s)
{
    using namespace fkmtc;
    if (n <= 0) return 0;
    if (nh < 1 || nh > F_MAXH) return (int)cudaErrorInvalidValue;
    FusedNet net;
    net.w = w;
    net.nh = nh;
    for (int l = 0; l < nh + 2; ++l) { net.woff[l] = woff[l]; net.boff[l] = boff[l]; }
    fused_pack_kernel<<<256, 256, 0, s>>>(net, wq);
    cudaError_t e = cudaFuncSetAttribute(mlp_fused_fwd_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, F_SMEM);
    if (e != cudaSuccess) return (int)e;
    int dev = 0, nsm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    const long long ntile = (n + BM - 1) / BM;
    const int grid = (int)(ntile < nsm ? ntile : nsm);
    mlp_fused_fwd_kernel<<<grid, F_NT, F_SMEM, s>>>(net, wq, n, x, tau, error);
    return (int)cudaGetLastError();
}
