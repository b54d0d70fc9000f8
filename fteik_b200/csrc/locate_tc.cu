/*
 * locate_tc.cu -- the batched L2 grid search (locate.F90:620-744) as a
 * tensor-core contraction.
 *
 * For an event whose picks cover every table with one common weight w, the
 * reference's misfit at grid point g,
 *     t0(g)  = sum_i w (o_i - T_i(g)) / sum_i w
 *     obj(g) = sum_i (sqrt(1/2) w (o_i - T_i(g) - t0(g)))^2,
 * equals (1/2) w^2 sum_i (o'_i - T'_i(g))^2, where o' is the picks minus their
 * mean and T'(g) the tables at g minus their mean over tables.  Because
 * sum_i o'_i = 0 this is
 *     obj(g) = (1/2) w^2 ( p + s(g) ),   s(g) = q(g) - 2 sum_i o'_i T'_i(g),
 *     p = sum o'^2 (per event),  q(g) = sum T'(g)^2 (per grid point),
 * so ranking grid points by s needs one events x stations by stations x points
 * product.  It runs on tcgen05 in BF16 with FP32 accumulation:
 *   - each operand is split as x = hi + lo (hi = bf16(x), lo = bf16(x - hi));
 *     the product is hi*hi + hi*lo (the default: the event side's rounding,
 *     o_lo . T(g), varies smoothly over the grid and the FP64 re-score
 *     decides) or hi*hi + hi*lo + lo*hi (relative error about 2^-16);
 *   - the event operand carries -2 o' (an exact scaling of the split);
 *   - q(g) enters as one more K step: the event side holds 1, 1, 1 and the
 *     table side q's three-way bf16 split (about 2^-24 relative), so the
 *     accumulator is s(g) itself.
 * Every thread of the epilogue owns one event row; it reduces each run of 32
 * grid points to its minimum and keeps the four best runs of its partition.
 * A second kernel takes each event's best runs over all partitions and
 * evaluates every point of them with the reference's misfit in FP64 on the
 * FP32 tables (one lane per point, coalesced), returning the minimum (first
 * index among equal misfits).
 *
 * Operand layout (all K-major, prepacked in global memory so that one untiled
 * bulk copy moves a tile into shared memory):
 *   main tile: 128 rows x 64 stations of bf16 = 16 KB in the 128-byte
 *     swizzled canonical form: row r at r * 128 bytes, 16-byte chunk c of row
 *     r at chunk position c ^ (r % 8);
 *   extra tile (the q step): 128 rows x 16 k of bf16 = 4 KB, no swizzle:
 *     8-row groups 256 bytes apart, k 0-7 and 8-15 in two 128-byte halves,
 *     row r of a group at 16 r;
 *   table tile = [hi][lo][extra] = 36 KB per 128 grid points;
 *   event tile = [hi][lo] = 32 KB per 128 events; the event side of the extra
 *     step is the same for all rows and is built once in shared memory.
 * Grid points of the padded last table tile get q = 1e30 and T' = 0.
 *
 * Kernel roles (320 threads, one CTA per SM):
 *   warp 0, one lane   bulk copies: two event tiles per work item, then a
 *                      4-stage ring of table tiles
 *   warp 1, one lane   tcgen05.mma: per table tile, 2 event tiles x (4 k-steps
 *                      x 2 or 3 products + the q step) into a 128 x 128 FP32
 *                      accumulator each; two accumulator sets (512 TMEM
 *                      columns) alternate
 *   warps 2-9          tcgen05.ld of the accumulators, run minima, top 4 runs
 * A work item is (event group of 256, grid partition).  Items are ordered
 * partition-major so the CTAs running at one time read the same table tiles
 * (L2 reuse).  Every wait is bounded; on timeout the CTA records an error,
 * stops issuing, waits (bounded) for its copies and MMAs, frees TMEM and
 * returns.
 */
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <stdint.h>
#include <stdio.h>
#include "fteik_dev.h"

namespace fktc {

constexpr int BM = 128;                    /* events per tile (TMEM lanes) */
constexpr int BN = 128;                    /* grid points per tile */
constexpr int BK = 64;                     /* stations: one 128-byte row of bf16 */
constexpr int RUN = 32;                    /* grid points per candidate run */
constexpr int TILE_BYTES = BM * BK * 2;    /* 16 KB */
constexpr int PAIR_BYTES = 2 * TILE_BYTES; /* hi + lo */
constexpr int XTRA_BYTES = BN * 16 * 2;    /* 4 KB: the q step */
constexpr int BTILE_BYTES = PAIR_BYTES + XTRA_BYTES;
constexpr int NSTAGE = 4;
constexpr int TOPK = FK_TC_TOPK;
constexpr int NTHREADS = 320;
constexpr int SMEM_A = 2 * PAIR_BYTES;
constexpr int SMEM_AX = XTRA_BYTES;
constexpr int SMEM_B = NSTAGE * BTILE_BYTES;
constexpr int NBAR = 2 * NSTAGE + 7;
constexpr int SMEM_BYTES = SMEM_A + SMEM_AX + SMEM_B + NBAR * 8 + 1024;
constexpr uint32_t TMEM_COLS = 512;
constexpr float PAD_Q = 1.0e30f;

/* instruction descriptor, kind::f16: D F32 (bits 4-5 = 1), A BF16 (7-9 = 1),
 * B BF16 (10-12 = 1), both K-major, N >> 3 at bit 17, M >> 4 at bit 24 */
constexpr uint32_t IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) |
                           ((uint32_t)(BM >> 4) << 24);

/* byte offset of element (row, k) inside one swizzled 16 KB main tile */
__host__ __device__ __forceinline__ uint32_t swz(int row, int k)
{
    return (uint32_t)row * 128u + ((uint32_t)(((k >> 3) ^ (row & 7))) << 4) + (uint32_t)(k & 7) * 2u;
}

/* byte offset of element (row, k), k < 16, inside one 4 KB extra tile */
__host__ __device__ __forceinline__ uint32_t xoff(int row, int k)
{
    return (uint32_t)(row >> 3) * 256u + (uint32_t)(k >> 3) * 128u + (uint32_t)(row & 7) * 16u +
           (uint32_t)(k & 7) * 2u;
}

__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

/* shared-memory matrix descriptors (descriptor version 1 at bit 46):
 * 128-byte swizzle, K-major: leading offset 16 B (unused), 8-row groups
 * 1024 B apart; no swizzle, K-major: k halves 128 B apart (leading offset),
 * 8-row groups 256 B apart (stride offset) */
__device__ __forceinline__ uint64_t sdesc_sw128(uint32_t saddr)
{
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) |
           ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}

__device__ __forceinline__ uint64_t sdesc_plain(uint32_t saddr)
{
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)(128 >> 4) << 16) |
           ((uint64_t)(256 >> 4) << 32) | ((uint64_t)1 << 46);
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
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

/* Bounded wait for the phase of the given parity.  False on timeout or when
 * another role has aborted. */
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, volatile int *abort,
                                          long long limit)
{
    for (long long i = 0; i < limit; ++i) {
        if (mbar_try(bar, parity)) return true;
        if (*abort) return false;
    }
    return false;
}

__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void *src, uint32_t bytes, uint32_t bar)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
        "l"(src), "r"(bytes), "r"(bar)
        : "memory");
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

#define FKTC_R8(i) "=r"(r[i]), "=r"(r[i + 1]), "=r"(r[i + 2]), "=r"(r[i + 3]), "=r"(r[i + 4]), \
                   "=r"(r[i + 5]), "=r"(r[i + 6]), "=r"(r[i + 7])

/* 32 consecutive columns of this warp's 32 TMEM lanes; no wait */
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t *r)
{
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : FKTC_R8(0), FKTC_R8(8), FKTC_R8(16), FKTC_R8(24)
        : "r"(taddr)
        : "memory");
}

__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

struct Params {
    const uint8_t *apack;   /* [2 * nmg][hi, lo] event tiles */
    const uint8_t *bpack;   /* [ntile][hi, lo, extra] table tiles */
    int nev, ntile, nmg, npart, nitems;
    float *cand_v;          /* [nev][npart][TOPK]: run minima */
    int *cand_i;            /*                     run numbers (first point / RUN) */
    int *error;
    float *dbg;             /* optional: CTA 0's first accumulators, [256][128] */
    long long spin_limit;
};

__device__ __forceinline__ void part_range(const Params &P, int p, int &tb, int &te)
{
    tb = (int)((long long)p * P.ntile / P.npart);
    te = (int)((long long)(p + 1) * P.ntile / P.npart);
}

__device__ __forceinline__ void set_abort(volatile int *abort, int *error, int code)
{
    *abort = 1;
    atomicCAS(error, 0, code);
}

/* NPROD: 3 = hi*hi + hi*lo + lo*hi; 2 = hi*hi + hi*lo (the event operand
 * rounded to BF16 once: its rounding error o_lo . T(g) varies smoothly over
 * the grid, unlike the tables' rounding, which both forms keep) */
template <int NPROD>
__global__ void __launch_bounds__(NTHREADS, 1) l2_tc_kernel(Params P)
{
    extern __shared__ uint8_t smem_raw[];
    __shared__ uint32_t s_tmem;
    __shared__ int s_abort;
    const uint32_t raw = smem_u32(smem_raw);
    const uint32_t sA = (raw + 1023u) & ~1023u;
    const uint32_t sAX = sA + SMEM_A;
    const uint32_t sB = sAX + SMEM_AX;
    const uint32_t bar0 = sB + SMEM_B;
    /* barriers: full[s], empty[s], a_full, a_empty, tfull[2], tempty[2], drain */
    auto FULL = [&](int s) { return bar0 + 8u * (uint32_t)s; };
    auto EMPTY = [&](int s) { return bar0 + 8u * (uint32_t)(NSTAGE + s); };
    const uint32_t A_FULL = bar0 + 8u * (2 * NSTAGE);
    const uint32_t A_EMPTY = A_FULL + 8u;
    auto TFULL = [&](int b) { return A_EMPTY + 8u + 8u * (uint32_t)b; };
    auto TEMPTY = [&](int b) { return A_EMPTY + 24u + 8u * (uint32_t)b; };
    const uint32_t DRAIN = A_EMPTY + 40u;
    volatile int *abort = &s_abort;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    /* event side of the q step: k = 0, 1, 2 hold 1.0, the rest 0 */
    {
        uint8_t *ax = smem_raw + (sAX - raw);
        for (int i = threadIdx.x; i < XTRA_BYTES / 16; i += NTHREADS) {
            const int row = i >> 1, khalf = i & 1;
            uint4 v = make_uint4(0u, 0u, 0u, 0u);
            if (khalf == 0) { v.x = 0x3F803F80u; v.y = 0x00003F80u; }
            *reinterpret_cast<uint4 *>(ax + xoff(row, khalf * 8)) = v;
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    if (threadIdx.x == 0) {
        for (int s = 0; s < NSTAGE; ++s) { mbar_init(FULL(s), 1); mbar_init(EMPTY(s), 1); }
        mbar_init(A_FULL, 1);
        mbar_init(A_EMPTY, 1);
        for (int b = 0; b < 2; ++b) { mbar_init(TFULL(b), 1); mbar_init(TEMPTY(b), 8); }
        mbar_init(DRAIN, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        s_abort = 0;
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_tmem)),
                     "r"(TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = s_tmem;
    const long long lim = P.spin_limit;

    if (warp == 0 && lane == 0) {
        /* ---- producer ---- */
        int stage = 0;
        uint32_t ph = 0, a_ph = 0;
        bool issued[NSTAGE] = {false, false, false, false};
        uint32_t iss_ph[NSTAGE] = {0, 0, 0, 0};
        bool a_issued = false;
        uint32_t a_iss_ph = 0;
        for (int item = blockIdx.x; item < P.nitems && !*abort; item += gridDim.x) {
            const int p = item / P.nmg, mg = item % P.nmg;
            if (!mbar_wait(A_EMPTY, a_ph ^ 1u, abort, lim)) { set_abort(abort, P.error, 1); break; }
            mbar_expect_tx(A_FULL, (uint32_t)SMEM_A);
            bulk_g2s(sA, P.apack + (size_t)(2 * mg) * PAIR_BYTES, (uint32_t)PAIR_BYTES, A_FULL);
            bulk_g2s(sA + PAIR_BYTES, P.apack + (size_t)(2 * mg + 1) * PAIR_BYTES, (uint32_t)PAIR_BYTES,
                     A_FULL);
            a_issued = true;
            a_iss_ph = a_ph;
            a_ph ^= 1u;
            int tb, te;
            part_range(P, p, tb, te);
            for (int t = tb; t < te; ++t) {
                if (!mbar_wait(EMPTY(stage), ph ^ 1u, abort, lim)) { set_abort(abort, P.error, 2); break; }
                mbar_expect_tx(FULL(stage), (uint32_t)BTILE_BYTES);
                bulk_g2s(sB + (uint32_t)stage * BTILE_BYTES, P.bpack + (size_t)t * BTILE_BYTES,
                         (uint32_t)BTILE_BYTES, FULL(stage));
                issued[stage] = true;
                iss_ph[stage] = ph;
                if (++stage == NSTAGE) { stage = 0; ph ^= 1u; }
            }
        }
        /* every copy this thread issued has landed before the CTA exits */
        for (int s = 0; s < NSTAGE; ++s)
            if (issued[s])
                for (long long i = 0; i < lim && !mbar_try(FULL(s), iss_ph[s]); ++i) {}
        if (a_issued)
            for (long long i = 0; i < lim && !mbar_try(A_FULL, a_iss_ph); ++i) {}
    } else if (warp == 1 && lane == 0) {
        /* ---- MMA issuer ---- */
        int stage = 0, buf = 0;
        uint32_t ph = 0, a_ph = 0;
        uint32_t tph[2] = {0, 0};
        const uint64_t ax_desc = sdesc_plain(sAX);
        for (int item = blockIdx.x; item < P.nitems && !*abort; item += gridDim.x) {
            const int p = item / P.nmg;
            if (!mbar_wait(A_FULL, a_ph, abort, lim)) { set_abort(abort, P.error, 3); break; }
            a_ph ^= 1u;
            tc_fence_after();
            int tb, te;
            part_range(P, p, tb, te);
            bool ok = true;
            for (int t = tb; t < te; ++t) {
                if (!mbar_wait(TEMPTY(buf), tph[buf] ^ 1u, abort, lim)) { ok = false; set_abort(abort, P.error, 4); break; }
                if (!mbar_wait(FULL(stage), ph, abort, lim)) { ok = false; set_abort(abort, P.error, 5); break; }
                tc_fence_after();
                const uint32_t b_hi = sB + (uint32_t)stage * BTILE_BYTES, b_lo = b_hi + TILE_BYTES;
                const uint64_t bx_desc = sdesc_plain(b_hi + PAIR_BYTES);
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const uint32_t d = tmem + (uint32_t)buf * 256u + (uint32_t)h * 128u;
                    const uint32_t a_hi = sA + (uint32_t)h * PAIR_BYTES, a_lo = a_hi + TILE_BYTES;
                    mma_bf16(d, ax_desc, bx_desc, 0u);      /* q(g) */
#pragma unroll
                    for (int k = 0; k < BK / 16; ++k) {
                        const uint32_t ko = (uint32_t)k * 32u;
                        mma_bf16(d, sdesc_sw128(a_hi + ko), sdesc_sw128(b_hi + ko), 1u);
                        mma_bf16(d, sdesc_sw128(a_hi + ko), sdesc_sw128(b_lo + ko), 1u);
                        if (NPROD == 3) mma_bf16(d, sdesc_sw128(a_lo + ko), sdesc_sw128(b_hi + ko), 1u);
                    }
                }
                mma_commit(EMPTY(stage));
                mma_commit(TFULL(buf));
                if (++stage == NSTAGE) { stage = 0; ph ^= 1u; }
                tph[buf] ^= 1u;
                buf ^= 1;
            }
            mma_commit(A_EMPTY);
            if (!ok) break;
        }
        /* no MMA of this CTA is in flight when TMEM is freed */
        mma_commit(DRAIN);
        for (long long i = 0; i < lim && !mbar_try(DRAIN, 0); ++i) {}
    } else if (warp >= 2) {
        /* ---- epilogue: thread = one event row of one event tile ---- */
        const int quad = warp & 3;            /* TMEM lane quarter this warp may read */
        const int h = (warp - 2) >> 2;        /* event tile 0 or 1 of the group */
        const int row = quad * 32 + lane;
        int buf = 0;
        uint32_t tph[2] = {0, 0};
        bool first_tile = true;
        /* control flow stays warp-uniform: tcgen05.ld is .sync.aligned */
        for (int item = blockIdx.x; item < P.nitems; item += gridDim.x) {
            if (__any_sync(0xffffffffu, *abort != 0)) break;
            const int p = item / P.nmg, mg = item % P.nmg;
            float bv[TOPK];
            int bi[TOPK];
#pragma unroll
            for (int k = 0; k < TOPK; ++k) { bv[k] = __int_as_float(0x7f800000); bi[k] = -1; }
            int tb, te;
            part_range(P, p, tb, te);
            bool ok = true;
            for (int t = tb; t < te; ++t) {
                const bool got = mbar_wait(TFULL(buf), tph[buf], abort, lim);
                if (!__all_sync(0xffffffffu, got)) {
                    ok = false;
                    if (lane == 0) set_abort(abort, P.error, 6);
                    break;
                }
                tc_fence_after();
                const uint32_t taddr = tmem + ((uint32_t)(quad * 32) << 16) + (uint32_t)buf * 256u +
                                       (uint32_t)h * 128u;
                uint32_t r[BN];
#pragma unroll
                for (int c = 0; c < BN / 32; ++c) tmem_ld32(taddr + (uint32_t)c * 32u, r + c * 32);
                tmem_wait_ld();
                tc_fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive(TEMPTY(buf));   /* accumulators are in registers */
                if (P.dbg && first_tile && blockIdx.x == 0) {
                    for (int j = 0; j < BN; ++j)
                        P.dbg[(size_t)(h * BM + row) * BN + j] = __uint_as_float(r[j]);
                }
#pragma unroll
                for (int c = 0; c < BN / RUN; ++c) {
                    float m[16];
#pragma unroll
                    for (int j = 0; j < 16; ++j)
                        m[j] = fminf(__uint_as_float(r[c * 32 + j]), __uint_as_float(r[c * 32 + 16 + j]));
#pragma unroll
                    for (int w = 8; w > 0; w >>= 1)
#pragma unroll
                        for (int j = 0; j < w; ++j) m[j] = fminf(m[j], m[j + w]);
                    float cv = m[0];
                    if (cv < bv[TOPK - 1]) {
                        int ci = (t * BN) / RUN + c;
#pragma unroll
                        for (int k = 0; k < TOPK; ++k) {
                            if (cv < bv[k]) {
                                const float tv = bv[k];
                                const int ti = bi[k];
                                bv[k] = cv; bi[k] = ci;
                                cv = tv; ci = ti;
                            }
                        }
                    }
                }
                first_tile = false;
                tph[buf] ^= 1u;
                buf ^= 1;
            }
            if (!ok) break;
            const int e = (2 * mg + h) * BM + row;
            if (e < P.nev) {
                const size_t o = ((size_t)e * P.npart + p) * TOPK;
#pragma unroll
                for (int k = 0; k < TOPK; ++k) { P.cand_v[o + k] = bv[k]; P.cand_i[o + k] = bi[k]; }
            }
        }
    }
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS)
                     : "memory");
    }
}

/* ---- packing ------------------------------------------------------------ */

__device__ __forceinline__ void split_bf16(double x, __nv_bfloat16 &hi, __nv_bfloat16 &lo)
{
    hi = __float2bfloat16_rn((float)x);
    lo = __float2bfloat16_rn((float)(x - (double)__bfloat162float(hi)));
}

/* One thread per grid point (rows of the padded last tile included). */
__global__ void pack_tables_kernel(int ngrd, int ldgrd, int ntf, int ntile,
                                   const float *__restrict__ tables, uint8_t *__restrict__ bpack)
{
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= ntile * BN) return;
    const int tile = g / BN, r = g % BN;
    uint8_t *hi = bpack + (size_t)tile * BTILE_BYTES, *lo = hi + TILE_BYTES, *xt = hi + PAIR_BYTES;
    const bool real = g < ngrd;
    double mean = 0.0;
    if (real) {
        for (int i = 0; i < ntf; ++i) mean += (double)__ldg(tables + (size_t)i * ldgrd + g);
        mean /= (double)ntf;
    }
    double q = 0.0;
    for (int c = 0; c < BK / 8; ++c) {
        __align__(16) __nv_bfloat16 vh[8], vl[8];
        for (int j = 0; j < 8; ++j) {
            const int k = c * 8 + j;
            double d = 0.0;
            if (real && k < ntf) {
                d = (double)__ldg(tables + (size_t)k * ldgrd + g) - mean;
                q += d * d;
            }
            split_bf16(d, vh[j], vl[j]);
        }
        const uint32_t off = swz(r, c * 8);
        *reinterpret_cast<uint4 *>(hi + off) = *reinterpret_cast<const uint4 *>(vh);
        *reinterpret_cast<uint4 *>(lo + off) = *reinterpret_cast<const uint4 *>(vl);
    }
    if (!real) q = (double)PAD_Q;
    /* q = q1 + q2 + q3, three bf16 terms */
    __align__(16) __nv_bfloat16 vx[8];
    const __nv_bfloat16 z = __float2bfloat16_rn(0.0f);
    for (int j = 0; j < 8; ++j) vx[j] = z;
    vx[0] = __float2bfloat16_rn((float)q);
    const double r1 = q - (double)__bfloat162float(vx[0]);
    vx[1] = __float2bfloat16_rn((float)r1);
    vx[2] = __float2bfloat16_rn((float)(r1 - (double)__bfloat162float(vx[1])));
    *reinterpret_cast<uint4 *>(xt + xoff(r, 0)) = *reinterpret_cast<const uint4 *>(vx);
    *reinterpret_cast<uint4 *>(xt + xoff(r, 8)) = make_uint4(0u, 0u, 0u, 0u);
}

/* One thread per event row slot: -2 (o - mean o), split.  Rows of
 * ineligible or padding events are zero (their scores are not used). */
__global__ void pack_events_kernel(int nev, int nrows, int ntf, const double *__restrict__ obs,
                                   const unsigned char *__restrict__ elig, uint8_t *__restrict__ apack)
{
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nrows) return;
    const int tile = e / BM, r = e % BM;
    uint8_t *hi = apack + (size_t)tile * PAIR_BYTES, *lo = hi + TILE_BYTES;
    const bool use = e < nev && elig[e];
    double mean = 0.0;
    if (use) {
        for (int i = 0; i < ntf; ++i) mean += obs[(size_t)e * ntf + i];
        mean /= (double)ntf;
    }
    for (int c = 0; c < BK / 8; ++c) {
        __align__(16) __nv_bfloat16 vh[8], vl[8];
        for (int j = 0; j < 8; ++j) {
            const int k = c * 8 + j;
            const double d = (use && k < ntf) ? -2.0 * (obs[(size_t)e * ntf + k] - mean) : 0.0;
            split_bf16(d, vh[j], vl[j]);
        }
        const uint32_t off = swz(r, c * 8);
        *reinterpret_cast<uint4 *>(hi + off) = *reinterpret_cast<const uint4 *>(vh);
        *reinterpret_cast<uint4 *>(lo + off) = *reinterpret_cast<const uint4 *>(vl);
    }
}

/* ---- FP64 re-score -------------------------------------------------------- */

__device__ __forceinline__ bool lex_lt(float v, int i, float w, int j)
{
    return v < w || (v == w && i < j);
}

__device__ __forceinline__ bool lex_lt_d(double v, int i, double w, int j)
{
    return v < w || (v == w && i < j);
}

/* FP64 misfit of one grid point, locate.F90:675-708 evaluated in one pass:
 * with d_i = o_i - T_i(g) and t0 = sum w d / sum w,
 *   obj = 1/2 sum (w (d - t0))^2 = 1/2 (sum w^2 d^2 - 2 t0 sum w^2 d + t0^2 sum w^2).
 * Reduced picks keep |d| within tens of seconds, so the cancellation costs
 * about 1e-12 absolute in FP64.  Picks and weights come from shared memory. */
__device__ __forceinline__ double misfit64(const float *__restrict__ tab, size_t ld, long long g, int ntf,
                                           const double *o, const double *w, double sw, double sw2,
                                           double &t0)
{
    double a = 0.0, b = 0.0, c = 0.0;
#pragma unroll 16
    for (int i = 0; i < ntf; ++i) {
        const double wi = w[i];
        const double d = o[i] - (double)__ldg(tab + (size_t)i * ld + g);
        const double w2d = wi * wi * d;
        a += wi * d;
        b += w2d;
        c += w2d * d;
    }
    t0 = a / sw;
    return 0.5 * (c - 2.0 * t0 * b + t0 * t0 * sw2);
}

/* misfit64 for NP grid points at once (independent loads in flight);
 * g[j] < 0 skips point j (result 1e300). */
template <int NP>
__device__ __forceinline__ void misfit64_n(const float *__restrict__ tab, size_t ld, const long long (&g)[NP],
                                           int ntf, const double *o, const double *w, double sw, double sw2,
                                           double (&ob)[NP], double (&t0)[NP])
{
    double a[NP], b[NP], c[NP];
    long long gg[NP];
#pragma unroll
    for (int j = 0; j < NP; ++j) { a[j] = b[j] = c[j] = 0.0; gg[j] = g[j] < 0 ? 0 : g[j]; }
#pragma unroll 8
    for (int i = 0; i < ntf; ++i) {
        const double wi = w[i], oi = o[i];
        const float *row = tab + (size_t)i * ld;
#pragma unroll
        for (int j = 0; j < NP; ++j) {
            const double d = oi - (double)__ldg(row + gg[j]);
            const double w2d = wi * wi * d;
            a[j] += wi * d;
            b[j] += w2d;
            c[j] += w2d * d;
        }
    }
#pragma unroll
    for (int j = 0; j < NP; ++j) {
        t0[j] = a[j] / sw;
        ob[j] = g[j] < 0 ? 1.0e300 : 0.5 * (c[j] - 2.0 * t0[j] * b[j] + t0[j] * t0[j] * sw2);
    }
}

/* One warp per event: take the R best runs by approximate score (ties by run
 * number), evaluate the reference's misfit in FP64 at every point of each run
 * (lane = point), keep the minimum (first index among equal misfits). */
__global__ void rescore_kernel(int nev, int npart, int ngrd, int ntf, int ldgrd, int R,
                               const float *__restrict__ tables, const double *__restrict__ obs,
                               const double *__restrict__ wts, const unsigned char *__restrict__ elig,
                               const float *__restrict__ cand_v, const int *__restrict__ cand_i,
                               int *__restrict__ out_idx, double *__restrict__ out_t0,
                               double *__restrict__ out_obj)
{
    __shared__ double s_o[8][BK], s_w[8][BK];
    const int wib = threadIdx.x >> 5;
    const int e = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (e >= nev || !elig[e]) return;
    const int C = npart * TOPK;
    const float *cv = cand_v + (size_t)e * C;
    const int *ci = cand_i + (size_t)e * C;
    for (int i = lane; i < BK; i += 32) {
        s_o[wib][i] = i < ntf ? obs[(size_t)e * ntf + i] : 0.0;
        s_w[wib][i] = i < ntf ? wts[(size_t)e * ntf + i] : 0.0;
    }
    __syncwarp();
    const double *o = s_o[wib], *w = s_w[wib];
    double sw = 0.0, sw2 = 0.0;
    for (int i = 0; i < ntf; ++i) { sw += w[i]; sw2 += w[i] * w[i]; }
    float pv = -3.0e38f;
    int pi = -1;
    double best_obj = 1.0e300, best_t0 = 0.0;
    int best_g = 0x7fffffff;
    for (int r = 0; r < R; ++r) {
        float mv = 3.0e38f;
        int mi = 0x7fffffff;
        for (int c = lane; c < C; c += 32) {
            const int i = ci[c];
            const float v = cv[c];
            if (i >= 0 && (long long)i * RUN < ngrd && lex_lt(pv, pi, v, i) && lex_lt(v, i, mv, mi)) {
                mv = v;
                mi = i;
            }
        }
#pragma unroll
        for (int s = 16; s > 0; s >>= 1) {
            const float ov = __shfl_xor_sync(0xffffffffu, mv, s);
            const int oi = __shfl_xor_sync(0xffffffffu, mi, s);
            if (lex_lt(ov, oi, mv, mi)) { mv = ov; mi = oi; }
        }
        if (mi == 0x7fffffff) break;
        pv = mv;
        pi = mi;
        const int g = mi * RUN + lane;
        double ob = 1.0e300, t0 = 0.0;
        if (g < ngrd) ob = misfit64(tables, (size_t)ldgrd, g, ntf, o, w, sw, sw2, t0);
        int gg = g < ngrd ? g : 0x7fffffff;
#pragma unroll
        for (int s = 16; s > 0; s >>= 1) {
            const double oo = __shfl_xor_sync(0xffffffffu, ob, s);
            const int og = __shfl_xor_sync(0xffffffffu, gg, s);
            const double ot = __shfl_xor_sync(0xffffffffu, t0, s);
            if (lex_lt_d(oo, og, ob, gg)) { ob = oo; gg = og; t0 = ot; }
        }
        if (lex_lt_d(ob, gg, best_obj, best_g)) { best_obj = ob; best_g = gg; best_t0 = t0; }
    }
    if (lane == 0) {
        out_idx[e] = best_g;
        out_t0[e] = best_t0;
        out_obj[e] = best_obj;
    }
}


/* a node's stations rounded up to 4 in the node-major block copy */
__host__ __device__ __forceinline__ int ntf_pad(int ntf) { return (ntf + 3) & ~3; }

/* misfit64 of NP nodes whose tables are 16-byte aligned runs (node-major
 * block copy): the same operations in the same station order as
 * misfit64_n, four stations per load; row[j] == nullptr skips node j. */
template <int NP>
__device__ __forceinline__ void misfit64_rows(const float *const (&row)[NP], const float *dummy, int ntf,
                                              const double *o, const double *w, double sw, double sw2,
                                              double (&ob)[NP], double (&t0)[NP])
{
    double a[NP], b[NP], c[NP];
    const float4 *r4[NP];
#pragma unroll
    for (int j = 0; j < NP; ++j) {
        a[j] = b[j] = c[j] = 0.0;
        r4[j] = reinterpret_cast<const float4 *>(row[j] ? row[j] : dummy);
    }
    const int nq = ntf_pad(ntf) / 4;
#pragma unroll 4
    for (int q = 0; q < nq; ++q) {
        float4 v[NP];
#pragma unroll
        for (int j = 0; j < NP; ++j) v[j] = __ldg(r4[j] + q);
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int i = 4 * q + u;
            if (i < ntf) {
                const double wi = w[i], oi = o[i];
#pragma unroll
                for (int j = 0; j < NP; ++j) {
                    const float tv = u == 0 ? v[j].x : u == 1 ? v[j].y : u == 2 ? v[j].z : v[j].w;
                    const double d = oi - (double)tv;
                    const double w2d = wi * wi * d;
                    a[j] += wi * d;
                    b[j] += w2d;
                    c[j] += w2d * d;
                }
            }
        }
    }
#pragma unroll
    for (int j = 0; j < NP; ++j) {
        t0[j] = a[j] / sw;
        ob[j] = row[j] ? 0.5 * (c[j] - 2.0 * t0[j] * b[j] + t0[j] * t0[j] * sw2) : 1.0e300;
    }
}

/* ---- pruned search (surrogate coarse lattice) ---------------------------- */

struct PruneGeom {
    int nz, nx, ny;           /* fine grid */
    int bz, bx, by;           /* block of fine nodes per coarse node */
    int ncz, ncx, ncy;
    int ldgrd, ldc, ntf;
};

/* One warp per event.
 *  1. the RC best coarse runs of the tensor-core ranking on the coarse
 *     (surrogate) tables; every coarse node of them scored in FP64 on those
 *     tables; the K best coarse nodes kept;
 *  2. every fine node of the K coarse nodes' blocks (coarse node c owns the
 *     fine nodes f with floor(f / b) = c on every axis: bz bx by per block,
 *     bz bx by K in all) scored in FP64 on the exact tables, read from their
 *     node-major block copy (each node's tables one 16-byte aligned run,
 *     read four stations per load); the minimum
 *     returned (first index among equal misfits);
 *  3. while a node next to that minimum (26-neighbourhood) lies in a block
 *     not yet examined, that block is examined too (a descent over blocks on
 *     the exact misfit, 32 blocks at most); flag[e] = 1 when the limit stops
 *     it, and the caller searches the event exhaustively.
 * flag[e]: 0xFF for a fall-back event, else the number of blocks examined. */
__global__ void __launch_bounds__(256, 3) prune_kernel(int nev, int npart, int RC, int K, PruneGeom G,
                             const float *__restrict__ coarse, const float *__restrict__ fine,
                             const double *__restrict__ obs, const double *__restrict__ wts,
                             const unsigned char *__restrict__ elig, const float *__restrict__ cand_v,
                             const int *__restrict__ cand_i, int *__restrict__ out_idx,
                             double *__restrict__ out_t0, double *__restrict__ out_obj,
                             unsigned char *__restrict__ flag)
{
    __shared__ int s_sel[8][32];   /* examined coarse nodes per warp */
    __shared__ double s_o[8][BK], s_w[8][BK];
    const int wib = threadIdx.x >> 5;
    const int e = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (e >= nev || !elig[e]) return;
    const long long ncoarse = (long long)G.ncz * G.ncx * G.ncy;
    const int C = npart * TOPK;
    const float *cv = cand_v + (size_t)e * C;
    const int *ci = cand_i + (size_t)e * C;
    for (int i = lane; i < BK; i += 32) {
        s_o[wib][i] = i < G.ntf ? obs[(size_t)e * G.ntf + i] : 0.0;
        s_w[wib][i] = i < G.ntf ? wts[(size_t)e * G.ntf + i] : 0.0;
    }
    __syncwarp();
    const double *o = s_o[wib], *w = s_w[wib];
    double sw = 0.0, sw2 = 0.0;
    for (int i = 0; i < G.ntf; ++i) { sw += w[i]; sw2 += w[i] * w[i]; }
    /* 1a. best coarse runs; each lane scores its point of every run */
    double cval[4];
    int cidx[4];
    long long cg[4];
    float pv = -3.0e38f;
    int pi = -1;
    for (int r = 0; r < 4; ++r) {
        cg[r] = -1;
        cidx[r] = 0x7fffffff;
        if (r >= RC) continue;
        float mv = 3.0e38f;
        int mi = 0x7fffffff;
        for (int c = lane; c < C; c += 32) {
            const int i = ci[c];
            const float v = cv[c];
            if (i >= 0 && (long long)i * RUN < ncoarse && lex_lt(pv, pi, v, i) && lex_lt(v, i, mv, mi)) {
                mv = v;
                mi = i;
            }
        }
#pragma unroll
        for (int s = 16; s > 0; s >>= 1) {
            const float ov = __shfl_xor_sync(0xffffffffu, mv, s);
            const int oi = __shfl_xor_sync(0xffffffffu, mi, s);
            if (lex_lt(ov, oi, mv, mi)) { mv = ov; mi = oi; }
        }
        if (mi == 0x7fffffff) continue;
        pv = mv;
        pi = mi;
        const long long c = (long long)mi * RUN + lane;
        if (c < ncoarse) { cg[r] = c; cidx[r] = (int)c; }
    }
    {
        double ct0[4];
        misfit64_n<4>(coarse, (size_t)G.ldc, cg, G.ntf, o, w, sw, sw2, cval, ct0);
    }
    /* 1b. the K best coarse nodes */
    double pvd = -1.0e300;
    int pid = -1;
    int nsel = 0;
    for (int k = 0; k < K; ++k) {
        double mv = 1.0e300;
        int mi = 0x7fffffff;
#pragma unroll
        for (int r = 0; r < 4; ++r)
            if (lex_lt_d(pvd, pid, cval[r], cidx[r]) && lex_lt_d(cval[r], cidx[r], mv, mi)) {
                mv = cval[r];
                mi = cidx[r];
            }
#pragma unroll
        for (int s = 16; s > 0; s >>= 1) {
            const double ov = __shfl_xor_sync(0xffffffffu, mv, s);
            const int oi = __shfl_xor_sync(0xffffffffu, mi, s);
            if (lex_lt_d(ov, oi, mv, mi)) { mv = ov; mi = oi; }
        }
        if (mi == 0x7fffffff) break;
        pvd = mv;
        pid = mi;
        if (lane == 0) s_sel[wib][k] = mi;
        nsel = k + 1;
    }
    __syncwarp();
    /* 2. fine nodes of the selected blocks */
    const int nb = G.bz * G.bx * G.by, ntp = ntf_pad(G.ntf);
    double best = 1.0e300, bt0 = 0.0;
    int bg = 0x7fffffff, bk = -1;
    auto scan_block = [&](int k) {
        const int c = s_sel[wib][k];
        const int cz = c % G.ncz, cx = (c / G.ncz) % G.ncx, cy = c / (G.ncz * G.ncx);
        for (int p0 = lane; p0 < nb; p0 += 64) {
            long long g2[2];
#pragma unroll
            for (int j = 0; j < 2; ++j) {
                const int p = p0 + 32 * j;
                const int fz = G.bz * cz + p % G.bz, fx = G.bx * cx + (p / G.bz) % G.bx,
                          fy = G.by * cy + p / (G.bz * G.bx);
                g2[j] = (p < nb && fz < G.nz && fx < G.nx && fy < G.ny)
                            ? fz + (long long)G.nz * (fx + (long long)G.nx * fy) : -1;
            }
            /* each node's tables are one 16-byte aligned run in the node-major block copy */
            long long q2[2];
#pragma unroll
            for (int j = 0; j < 2; ++j) q2[j] = g2[j] >= 0 ? p0 + 32 * j : -1;
            double ob[2], t0[2];
            const float *rows[2];
#pragma unroll
            for (int j = 0; j < 2; ++j) rows[j] = q2[j] >= 0 ? fine + ((size_t)c * nb + q2[j]) * ntp : nullptr;
            misfit64_rows<2>(rows, fine, G.ntf, o, w, sw, sw2, ob, t0);
#pragma unroll
            for (int j = 0; j < 2; ++j)
                if (g2[j] >= 0 && lex_lt_d(ob[j], (int)g2[j], best, bg)) {
                    best = ob[j]; bg = (int)g2[j]; bt0 = t0[j]; bk = k;
                }
        }
#pragma unroll
        for (int s = 16; s > 0; s >>= 1) {
            const double ob = __shfl_xor_sync(0xffffffffu, best, s);
            const int og = __shfl_xor_sync(0xffffffffu, bg, s);
            const double ot = __shfl_xor_sync(0xffffffffu, bt0, s);
            const int ok = __shfl_xor_sync(0xffffffffu, bk, s);
            if (lex_lt_d(ob, og, best, bg)) { best = ob; bg = og; bt0 = ot; bk = ok; }
        }
    };
    for (int k = 0; k < nsel; ++k) scan_block(k);
    /* 3. while a neighbour of the minimum lies in a block not yet examined,
     * examine that block (a descent over blocks on the exact misfit); give
     * up after MAXB blocks in all */
    constexpr int MAXB = 32;
    unsigned char fb = 0;
    for (;;) {
        /* every node of the 26-neighbourhood of the best node must lie in
         * an examined block: a minimum over face neighbours alone can sit
         * next to a lower diagonal node in an oblique valley (lane q checks
         * neighbour q; the first missing block in lane order is added) */
        int add = -1;
        if (bk >= 0 && lane < 27 && lane != 13) {
            const int f0 = bg % G.nz, f1 = (bg / G.nz) % G.nx, f2 = bg / (G.nz * G.nx);
            const int gz = f0 + lane % 3 - 1, gx = f1 + (lane / 3) % 3 - 1, gy = f2 + lane / 9 - 1;
            if (gz >= 0 && gx >= 0 && gy >= 0 && gz < G.nz && gx < G.nx && gy < G.ny) {
                const int cn = gz / G.bz + G.ncz * (gx / G.bx + G.ncx * (gy / G.by));
                bool have = false;
                for (int k = 0; k < nsel; ++k) have |= s_sel[wib][k] == cn;
                if (!have) add = cn;
            }
        }
        const unsigned miss = __ballot_sync(0xffffffffu, add >= 0);
        add = miss ? __shfl_sync(0xffffffffu, add, __ffs(miss) - 1) : -1;
        if (add < 0) break;
        if (nsel >= MAXB) { fb = 1; break; }
        if (lane == 0) s_sel[wib][nsel] = add;
        __syncwarp();
        scan_block(nsel);
        ++nsel;
    }
    if (bk < 0) fb = 1;
    if (lane != 0) return;
    out_idx[e] = bg;
    out_t0[e] = bt0;
    out_obj[e] = best;
    flag[e] = fb ? (unsigned char)0xFF : (unsigned char)nsel;
}

/* Block-major, node-major copy of the exact tables for the pruned search:
 * out[(c nb + p) ntp + i] = T_i(node p of block c), p = pz + bz (px + bx py),
 * ntp = ntf rounded up to 4 (a node's tables are one 16-byte aligned run);
 * padding and nodes outside the grid hold 0 (never read). */
__global__ void block_tables_kernel(int nz, int nx, int ny, int bz, int bx, int by, int ncz, int ncx, int ntf,
                                    int ldgrd, long long nblk, const float *__restrict__ tables,
                                    float *__restrict__ out)
{
    const int nb = bz * bx * by, ntp = ntf_pad(ntf);
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= nblk * nb) return;
    const long long c = t / nb;
    const int p = (int)(t % nb);
    const int cz = (int)(c % ncz), cx = (int)((c / ncz) % ncx), cy = (int)(c / ((long long)ncz * ncx));
    const int fz = bz * cz + p % bz, fx = bx * cx + (p / bz) % bx, fy = by * cy + p / (bz * bx);
    const bool in = fz < nz && fx < nx && fy < ny;
    const long long g = in ? fz + (long long)nz * (fx + (long long)nx * fy) : 0;
    float4 *dst = reinterpret_cast<float4 *>(out + (size_t)t * ntp);
    for (int q = 0; q < ntp / 4; ++q) {
        float v[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int i = 4 * q + u;
            v[u] = (in && i < ntf) ? __ldg(tables + (size_t)i * ldgrd + g) : 0.0f;
        }
        dst[q] = make_float4(v[0], v[1], v[2], v[3]);
    }
}

} // namespace fktc

using namespace fktc;

extern "C" size_t fk_locate_tc_table_bytes(int ngrd)
{
    const size_t ntile = ((size_t)ngrd + BN - 1) / BN;
    return ntile * BTILE_BYTES;
}

extern "C" size_t fk_locate_tc_event_bytes(int nev)
{
    const size_t nmg = ((size_t)nev + 2 * BM - 1) / (2 * BM);
    return nmg * 2 * PAIR_BYTES;
}

extern "C" int fk_locate_tc_pack_tables(int ngrd, int ldgrd, int ntf, const float *tables,
                                        void *bpack, cudaStream_t s)
{
    if (ntf < 1 || ntf > BK) return (int)cudaErrorInvalidValue;
    const int ntile = (ngrd + BN - 1) / BN;
    const int n = ntile * BN;
    pack_tables_kernel<<<(n + 255) / 256, 256, 0, s>>>(ngrd, ldgrd, ntf, ntile, tables,
                                                       (uint8_t *)bpack);
    return (int)cudaGetLastError();
}

/* Partitions of the grid: enough work items to fill whole waves of CTAs. */
static int pick_npart(int nmg, int ntile, int nsm)
{
    int best = 1;
    double best_eff = -1.0;
    for (int waves = 1; waves <= 16; ++waves) {
        int P = (waves * nsm + nmg - 1) / nmg;
        if (P > ntile) P = ntile;
        if (P < 1) P = 1;
        const long long items = (long long)P * nmg;
        const long long slots = (items + nsm - 1) / nsm * nsm;
        const double eff = (double)items / (double)slots;
        if (eff > best_eff + 1e-9) { best_eff = eff; best = P; }
        if (eff > 0.97) break;
    }
    return best;
}

/* products of the ranking, 2 (the default) or 3 (l2_tc_kernel<NPROD>) */
static int g_nprod = 2;
extern "C" void fk_locate_tc_set_products(int n) { g_nprod = n == 2 ? 2 : 3; }
extern "C" int fk_locate_tc_get_products(void) { return g_nprod; }

extern "C" int fk_locate_tc_npart(int nev, int ngrd)
{
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    const int nmg = (nev + 2 * BM - 1) / (2 * BM);
    const int ntile = (ngrd + BN - 1) / BN;
    return pick_npart(nmg, ntile, nsm);
}

extern "C" int fk_locate_tc(int ngrd, int ldgrd, int ntf, const float *tables, const void *bpack,
                            int nev, const double *obs, const double *wts,
                            const unsigned char *elig, void *apack, int npart, float *cand_v,
                            int *cand_i, int rescore, int *out_idx, double *out_t0,
                            double *out_obj, int *error, float *dbg, cudaStream_t s)
{
    if (nev <= 0) return 0;
    if (ntf < 1 || ntf > BK || npart < 1) return (int)cudaErrorInvalidValue;
    const int nmg = (nev + 2 * BM - 1) / (2 * BM);
    const int ntile = (ngrd + BN - 1) / BN;
    if (npart > ntile) return (int)cudaErrorInvalidValue;
    pack_events_kernel<<<(nmg * 2 * BM + 127) / 128, 128, 0, s>>>(nev, nmg * 2 * BM, ntf, obs, elig,
                                                                  (uint8_t *)apack);
    static int attr_done = 0;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaStreamIsCapturing(s, &cs);
    if (!attr_done && cs == cudaStreamCaptureStatusNone) {
        cudaError_t e = cudaFuncSetAttribute(l2_tc_kernel<3>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             SMEM_BYTES);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(l2_tc_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES);
        if (e != cudaSuccess) return (int)e;
        attr_done = 1;
    }
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    Params P;
    P.apack = (const uint8_t *)apack;
    P.bpack = (const uint8_t *)bpack;
    P.nev = nev;
    P.ntile = ntile;
    P.nmg = nmg;
    P.npart = npart;
    P.nitems = nmg * npart;
    P.cand_v = cand_v;
    P.cand_i = cand_i;
    P.error = error;
    P.dbg = dbg;
    P.spin_limit = 1ll << 22;
    const int grid = P.nitems < nsm ? P.nitems : nsm;
    if (g_nprod == 2)
        l2_tc_kernel<2><<<grid, NTHREADS, SMEM_BYTES, s>>>(P);
    else
        l2_tc_kernel<3><<<grid, NTHREADS, SMEM_BYTES, s>>>(P);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return (int)e;
    if (rescore > 0) {
        rescore_kernel<<<(nev * 32 + 255) / 256, 256, 0, s>>>(nev, npart, ngrd, ntf, ldgrd, rescore,
                                                              tables, obs, wts, elig, cand_v, cand_i,
                                                              out_idx, out_t0, out_obj);
        e = cudaGetLastError();
    }
    return (int)e;
}

extern "C" int fk_locate_prune(int nev, int npart, int rc, int k, int nz, int nx, int ny, int bz, int bx,
                               int by, int ldgrd, int ldc, int ntf, const float *coarse, const float *fine,
                               const double *obs, const double *wts, const unsigned char *elig,
                               const float *cand_v, const int *cand_i, int *out_idx, double *out_t0,
                               double *out_obj, unsigned char *flag, cudaStream_t s)
{
    if (nev <= 0) return 0;
    if (rc < 1 || rc > 4 || k < 1 || k > 32 || bz < 1 || bx < 1 || by < 1) return (int)cudaErrorInvalidValue;
    PruneGeom G;
    G.nz = nz; G.nx = nx; G.ny = ny;
    G.bz = bz; G.bx = bx; G.by = by;
    G.ncz = (nz + bz - 1) / bz;
    G.ncx = (nx + bx - 1) / bx;
    G.ncy = (ny + by - 1) / by;
    G.ldgrd = ldgrd; G.ldc = ldc; G.ntf = ntf;
    prune_kernel<<<(nev * 32 + 255) / 256, 256, 0, s>>>(nev, npart, rc, k, G, coarse, fine, obs, wts, elig,
                                                        cand_v, cand_i, out_idx, out_t0, out_obj, flag);
    return (int)cudaGetLastError();
}

extern "C" int fk_locate_block_tables(int nz, int nx, int ny, int bz, int bx, int by, int ntf, int ldgrd,
                                      const float *tables, float *out, cudaStream_t s)
{
    const int ncz = (nz + bz - 1) / bz, ncx = (nx + bx - 1) / bx, ncy = (ny + by - 1) / by;
    const long long nblk = (long long)ncz * ncx * ncy;
    const long long n = nblk * bz * bx * by;
    block_tables_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(nz, nx, ny, bz, bx, by, ncz, ncx, ntf, ldgrd,
                                                                    nblk, tables, out);
    return (int)cudaGetLastError();
}
