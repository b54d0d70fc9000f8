/*
 * locate.cu -- grid-search event location (locate.F90:620-744, :112-126).
 *
 * fk_locate_l2_exact reproduces the reference's FP32 objective bit for bit:
 * for every grid point g and event e, in the reference's order,
 *   t0[g]  += w_i * (xnorm * (o_i - T_i[g]))            over used tables i
 *   obj[g] += ((sqrt(1/2) * w_i) * (o_i - (T_i[g] + t0[g])))^2
 * with no fused multiply-add, then MINLOC (first minimum).  A thread keeps
 * the tables of its grid point in registers and evaluates a block of events
 * against them, so the tables stream from HBM once per event block rather
 * than once per event.  The argmin is a 64-bit atomicMin on
 * (float bits of obj) << 32 | g, which for non-negative objectives orders by
 * value and then by the smaller index, as MINLOC does.
 */
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include "fteik_dev.h"

namespace {

constexpr int kThreads = 256;
constexpr int kEvBlock = 32;  /* events per CTA */
constexpr int kMaxTf = 64;    /* tables held in registers */

__device__ __forceinline__ unsigned long long pack_key(float obj, int g)
{
    return ((unsigned long long)__float_as_uint(obj) << 32) | (unsigned)g;
}

template <int NTF>
__global__ void __launch_bounds__(kThreads)
l2_exact_kernel(int ngrd, int ldgrd, int ntf, const float *__restrict__ tables, int nev,
                const float *__restrict__ obs, const float *__restrict__ wts,
                const float *__restrict__ xnorm, unsigned long long *__restrict__ best)
{
    __shared__ float s_obs[kEvBlock][NTF];
    __shared__ float s_w[kEvBlock][NTF];
    __shared__ float s_xn[kEvBlock];
    __shared__ unsigned long long s_best[kThreads / 32];
    const int g = blockIdx.x * kThreads + threadIdx.x;
    const int e0 = blockIdx.y * kEvBlock;
    const int nev_blk = min(kEvBlock, nev - e0);
    for (int t = threadIdx.x; t < kEvBlock * NTF; t += kThreads) {
        const int e = t / NTF, i = t % NTF;
        const bool ok = e < nev_blk && i < ntf;
        s_obs[e][i] = ok ? obs[(size_t)(e0 + e) * ntf + i] : 0.0f;
        s_w[e][i] = ok ? wts[(size_t)(e0 + e) * ntf + i] : 0.0f;
    }
    if (threadIdx.x < kEvBlock) s_xn[threadIdx.x] = (threadIdx.x < nev_blk) ? xnorm[e0 + threadIdx.x] : 0.0f;
    float T[NTF];
#pragma unroll
    for (int i = 0; i < NTF; ++i)
        T[i] = (g < ngrd && i < ntf) ? __ldg(tables + (size_t)i * ldgrd + g) : 0.0f;
    __syncthreads();
    const float sqrtHalf = 0.70710677f; /* SQRT(0.5) in FP32 (constants.F90) */
    for (int e = 0; e < nev_blk; ++e) {
        const float xn = s_xn[e];
        float t0 = 0.0f;
#pragma unroll
        for (int i = 0; i < NTF; ++i) {
            const float w = s_w[e][i];
            if (i < ntf && w > 0.0f) {
                const float res = __fmul_rn(xn, __fsub_rn(s_obs[e][i], __fadd_rn(T[i], 0.0f)));
                t0 = __fadd_rn(t0, __fmul_rn(w, res));
            }
        }
        float obj = 0.0f;
#pragma unroll
        for (int i = 0; i < NTF; ++i) {
            const float w = s_w[e][i];
            if (i < ntf && w > 0.0f) {
                const float wt = __fmul_rn(sqrtHalf, w);
                const float est = __fadd_rn(__fadd_rn(T[i], t0), 0.0f);
                const float res = __fmul_rn(wt, __fsub_rn(s_obs[e][i], est));
                obj = __fadd_rn(obj, __fmul_rn(res, res));
            }
        }
        unsigned long long key = (g < ngrd) ? pack_key(obj, g) : ~0ull;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            unsigned long long k2 = __shfl_xor_sync(0xffffffffu, key, o);
            key = k2 < key ? k2 : key;
        }
        if ((threadIdx.x & 31) == 0) s_best[threadIdx.x >> 5] = key;
        __syncthreads();
        if (threadIdx.x == 0) {
            unsigned long long k = s_best[0];
            for (int w2 = 1; w2 < kThreads / 32; ++w2) k = s_best[w2] < k ? s_best[w2] : k;
            atomicMin(best + e0 + e, k);
        }
        __syncthreads();
    }
}

/* t0 and obj at the optimum, same arithmetic. */
__global__ void l2_at_opt_kernel(int ngrd, int ldgrd, int ntf, const float *__restrict__ tables,
                                 int nev, const float *__restrict__ obs,
                                 const float *__restrict__ wts, const float *__restrict__ xnorm,
                                 const unsigned long long *__restrict__ best, int *out_idx,
                                 float *out_t0, float *out_obj)
{
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nev) return;
    const int g = (int)(best[e] & 0xffffffffu);
    const float xn = xnorm[e];
    const float *o = obs + (size_t)e * ntf, *w = wts + (size_t)e * ntf;
    float t0 = 0.0f;
    for (int i = 0; i < ntf; ++i)
        if (w[i] > 0.0f)
            t0 = __fadd_rn(t0, __fmul_rn(w[i], __fmul_rn(xn, __fsub_rn(o[i], tables[(size_t)i * ldgrd + g]))));
    float obj = 0.0f;
    for (int i = 0; i < ntf; ++i)
        if (w[i] > 0.0f) {
            const float res = __fmul_rn(__fmul_rn(0.70710677f, w[i]),
                                        __fsub_rn(o[i], __fadd_rn(tables[(size_t)i * ldgrd + g], t0)));
            obj = __fadd_rn(obj, __fmul_rn(res, res));
        }
    out_idx[e] = g;
    out_t0[e] = t0;
    out_obj[e] = obj;
}

__global__ void xnorm_kernel(int nev, int ntf, const float *__restrict__ wts, float *xnorm,
                             unsigned long long *best)
{
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nev) return;
    float s = 0.0f; /* SUM over the padded weight row, in order */
    for (int i = 0; i < ntf; ++i) s = __fadd_rn(s, wts[(size_t)e * ntf + i]);
    xnorm[e] = __fdiv_rn(1.0f, s);
    best[e] = ~0ull;
}

} // namespace

extern "C" size_t fk_locate_l2_exact_scratch(int ngrd, int nev)
{
    (void)ngrd;
    return (size_t)nev * (sizeof(unsigned long long) + sizeof(float)) + 256;
}

extern "C" int fk_locate_l2_exact(int ngrd, int ldgrd, int ntf, const float *tables, int nev,
                                  const float *obs, const float *wts, int *out_idx,
                                  float *out_t0, float *out_obj, void *scratch,
                                  size_t scratch_bytes, cudaStream_t s)
{
    if (nev <= 0) return 0;
    if (ntf > kMaxTf || ntf < 1) return (int)cudaErrorInvalidValue;
    if (scratch_bytes < fk_locate_l2_exact_scratch(ngrd, nev)) return (int)cudaErrorInvalidValue;
    unsigned long long *best = (unsigned long long *)scratch;
    float *xn = (float *)(best + nev);
    xnorm_kernel<<<(nev + 127) / 128, 128, 0, s>>>(nev, ntf, wts, xn, best);
    dim3 grid((ngrd + kThreads - 1) / kThreads, (nev + kEvBlock - 1) / kEvBlock);
    if (ntf <= 16)
        l2_exact_kernel<16><<<grid, kThreads, 0, s>>>(ngrd, ldgrd, ntf, tables, nev, obs, wts, xn, best);
    else if (ntf <= 32)
        l2_exact_kernel<32><<<grid, kThreads, 0, s>>>(ngrd, ldgrd, ntf, tables, nev, obs, wts, xn, best);
    else
        l2_exact_kernel<64><<<grid, kThreads, 0, s>>>(ngrd, ldgrd, ntf, tables, nev, obs, wts, xn, best);
    l2_at_opt_kernel<<<(nev + 127) / 128, 128, 0, s>>>(ngrd, ldgrd, ntf, tables, nev, obs, wts, xn,
                                                       best, out_idx, out_t0, out_obj);
    return (int)cudaGetLastError();
}

/* ------------------------------------------------------------------------ */
/* Allocation-free variant.                                                 */
/*                                                                          */
/* Some callers cannot let a library call cudaMalloc: a host that hands out */
/* all device memory from its own pool (a framework's caching allocator, a  */
/* real-time service with a fixed memory budget) or that must not trigger   */
/* the device-wide synchronisation cudaMalloc/cudaFree can cause.  For them */
/* fteik_b200_locate_l2_noalloc runs the same grid search on buffers the    */
/* caller owns, keeping its per-event scratch (the best (misfit, index) key */
/* and the weight normaliser, 12 bytes per event) in the fixed array below. */
/* ------------------------------------------------------------------------ */

#define FK_NOALLOC_MAX_EVENTS 65536
/* Lives on every device that loads this library until the process exits. */
static __device__ __align__(256) unsigned char g_noalloc_scratch[FK_NOALLOC_MAX_EVENTS * 12 + 256];

extern "C" void fteik_b200_locate_l2_noalloc(int ngrd, int ldgrd, int ntf, const float *tables,
                                             int nev, const float *obs, const float *wts,
                                             int *opt_index, float *t0, float *obj, void *stream,
                                             int *ierr)
{
    *ierr = 1;
    if (nev < 1 || nev > FK_NOALLOC_MAX_EVENTS) {
        fprintf(stderr, "fteik_b200_locate_l2_noalloc: nev=%d must be in [1,%d]\n", nev,
                FK_NOALLOC_MAX_EVENTS);
        return;
    }
    if (ntf < 1 || ntf > kMaxTf || ngrd < 1 || ldgrd < ngrd) {
        fprintf(stderr, "fteik_b200_locate_l2_noalloc: need 1 <= ntf <= %d and 1 <= ngrd <= ldgrd\n",
                kMaxTf);
        return;
    }
    if (!tables || !obs || !wts || !opt_index || !t0 || !obj) {
        fprintf(stderr, "fteik_b200_locate_l2_noalloc: null buffer\n");
        return;
    }
    /* the device address of the array, looked up on every call with the
     * caller's current device (the host-side name of the array is not a
     * device address); nothing is cached, so concurrent first calls from
     * several host threads and a reset device leave no stale address */
    void *scratch = NULL;
    cudaError_t e = cudaGetSymbolAddress(&scratch, g_noalloc_scratch);
    if (e != cudaSuccess) {
        fprintf(stderr, "fteik_b200_locate_l2_noalloc: cudaGetSymbolAddress failed (%s)\n",
                cudaGetErrorString(e));
        return;
    }
    const int rc = fk_locate_l2_exact(ngrd, ldgrd, ntf, tables, nev, obs, wts, opt_index, t0, obj,
                                      scratch, sizeof(g_noalloc_scratch),
                                      (cudaStream_t)stream);
    if (rc != 0) {
        fprintf(stderr, "fteik_b200_locate_l2_noalloc: launch failed (%s)\n",
                cudaGetErrorString((cudaError_t)rc));
        return;
    }
    *ierr = 0;
}

/* ------------------------------------------------------------------------ */
/* L1 grid search (no counterpart in the reference, which has L2 only).     */
/*                                                                          */
/* For the picks of an event (positive weights, all equal to w) and a grid  */
/* point g the residuals r_i = o_i - T_i(g) give                            */
/*   t0(g)  = median of r  (any point between the two middle values when   */
/*            the count is even; the midpoint is reported)                  */
/*   obj(g) = w sum_i |r_i - t0| = w (sum of the upper half - sum of the    */
/*            lower half of the sorted residuals).                          */
/* A thread holds the 64 residuals of one grid point in registers and sorts */
/* them with a fully unrolled bitonic network (skipped picks sort last as   */
/* +inf); the half sums use compile-time indices.  The argmin is the        */
/* first-index minimum (64-bit atomicMin on (bits << 32) | g); t0 and obj   */
/* at the optimum are recomputed in FP64.                                   */
/* ------------------------------------------------------------------------ */

namespace {

template <int N>
__device__ __forceinline__ void bitonic_sort(float (&v)[N])
{
#pragma unroll
    for (int k = 2; k <= N; k <<= 1)
#pragma unroll
        for (int j = k >> 1; j > 0; j >>= 1)
#pragma unroll
            for (int i = 0; i < N; ++i) {
                const int l = i ^ j;
                if (l > i) {
                    const float a = v[i], b = v[l];
                    const bool up = (i & k) == 0;
                    v[i] = up ? fminf(a, b) : fmaxf(a, b);
                    v[l] = up ? fmaxf(a, b) : fminf(a, b);
                }
            }
}

template <int N>
__global__ void __launch_bounds__(128) l1_exact_kernel(int ngrd, int ldgrd, int ntf, const float *__restrict__ tables,
                                                       int nev, const float *__restrict__ obs,
                                                       const float *__restrict__ wts, unsigned long long *__restrict__ best)
{
    constexpr int EVB = 16;
    __shared__ float s_obs[EVB][N];
    __shared__ float s_w[EVB][N];
    __shared__ int s_n[EVB];
    __shared__ float s_wv[EVB];
    __shared__ unsigned long long s_best[EVB][4];
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    const int e0 = blockIdx.y * EVB;
    const int nb = min(EVB, nev - e0);
    for (int t = threadIdx.x; t < EVB * N; t += blockDim.x) {
        const int e = t / N, i = t % N;
        const bool ok = e < nb && i < ntf;
        s_obs[e][i] = ok ? obs[(size_t)(e0 + e) * ntf + i] : 0.0f;
        s_w[e][i] = ok ? wts[(size_t)(e0 + e) * ntf + i] : 0.0f;
    }
    __syncthreads();
    if (threadIdx.x < EVB) {
        int n = 0;
        float wv = 0.0f;
        for (int i = 0; i < N; ++i)
            if (s_w[threadIdx.x][i] > 0.0f) { ++n; wv = s_w[threadIdx.x][i]; }
        s_n[threadIdx.x] = n;
        s_wv[threadIdx.x] = wv;
    }
    float T[N];
#pragma unroll
    for (int i = 0; i < N; ++i) T[i] = (g < ngrd && i < ntf) ? __ldg(tables + (size_t)i * ldgrd + g) : 0.0f;
    __syncthreads();
    const float INF = __int_as_float(0x7f800000);
    for (int e = 0; e < nb; ++e) {
        float r[N];
#pragma unroll
        for (int i = 0; i < N; ++i) r[i] = s_w[e][i] > 0.0f ? s_obs[e][i] - T[i] : INF;
        bitonic_sort<N>(r);
        const int n = s_n[e], h = n / 2;
        float obj = 0.0f;
#pragma unroll
        for (int i = 0; i < N; ++i) {
            /* lower half: i < h; upper half: n - h <= i < n (the middle one of
             * an odd count drops out) */
            const float c = i < h ? -1.0f : ((i >= n - h && i < n) ? 1.0f : 0.0f);
            obj = fmaf(c, (i < n) ? r[i] : 0.0f, obj);
        }
        obj *= s_wv[e];
        unsigned long long key = (g < ngrd && n > 0) ? pack_key(obj, g) : ~0ull;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const unsigned long long k2 = __shfl_xor_sync(0xffffffffu, key, o);
            key = k2 < key ? k2 : key;
        }
        if ((threadIdx.x & 31) == 0) s_best[e][threadIdx.x >> 5] = key;
    }
    __syncthreads();
    if (threadIdx.x < nb) {
        unsigned long long k = s_best[threadIdx.x][0];
        for (int w2 = 1; w2 < 4; ++w2) k = s_best[threadIdx.x][w2] < k ? s_best[threadIdx.x][w2] : k;
        atomicMin(best + e0 + threadIdx.x, k);
    }
}

/* FP64 median and misfit at the chosen point from the FP64 picks
 * (insertion sort, one thread per event). */
__global__ void l1_at_opt_kernel(int ldgrd, int ntf, const float *__restrict__ tables, int nev,
                                 const double *__restrict__ obs, const double *__restrict__ wts,
                                 const unsigned long long *__restrict__ best, int *out_idx, double *out_t0,
                                 double *out_obj)
{
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nev) return;
    const int g = (int)(best[e] & 0xffffffffu);
    double r[64];
    int n = 0;
    double wv = 0.0;
    for (int i = 0; i < ntf; ++i) {
        const double w = wts[(size_t)e * ntf + i];
        if (w > 0.0) {
            const double v = obs[(size_t)e * ntf + i] - (double)tables[(size_t)i * ldgrd + g];
            int j = n++;
            while (j > 0 && r[j - 1] > v) { r[j] = r[j - 1]; --j; }
            r[j] = v;
            wv = w;
        }
    }
    double t0 = 0.0, obj = 0.0;
    if (n > 0) {
        t0 = (n % 2) ? r[n / 2] : 0.5 * (r[n / 2 - 1] + r[n / 2]);
        for (int i = 0; i < n; ++i) obj += fabs(r[i] - t0);
        obj *= wv;
    }
    out_idx[e] = g;
    out_t0[e] = t0;
    out_obj[e] = obj;
}

__global__ void l1_init_kernel(int nev, unsigned long long *best)
{
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e < nev) best[e] = ~0ull;
}

} // namespace

extern "C" int fk_locate_l1_exact(int ngrd, int ldgrd, int ntf, const float *tables, int nev, const float *obs,
                                  const float *wts, const double *obs64, const double *wts64, int *out_idx,
                                  double *out_t0, double *out_obj, unsigned long long *scratch, cudaStream_t s)
{
    if (nev <= 0) return 0;
    if (ntf < 1 || ntf > kMaxTf) return (int)cudaErrorInvalidValue;
    l1_init_kernel<<<(nev + 255) / 256, 256, 0, s>>>(nev, scratch);
    dim3 grid((ngrd + 127) / 128, (nev + 15) / 16);
    if (ntf <= 16)
        l1_exact_kernel<16><<<grid, 128, 0, s>>>(ngrd, ldgrd, ntf, tables, nev, obs, wts, scratch);
    else if (ntf <= 32)
        l1_exact_kernel<32><<<grid, 128, 0, s>>>(ngrd, ldgrd, ntf, tables, nev, obs, wts, scratch);
    else
        l1_exact_kernel<64><<<grid, 128, 0, s>>>(ngrd, ldgrd, ntf, tables, nev, obs, wts, scratch);
    l1_at_opt_kernel<<<(nev + 127) / 128, 128, 0, s>>>(ldgrd, ntf, tables, nev, obs64, wts64, scratch, out_idx,
                                                       out_t0, out_obj);
    return (int)cudaGetLastError();
}
