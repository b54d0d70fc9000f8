/*
 * mlp.cu -- kernels of the travel-time surrogate: a fully connected network
 * 6 -> W -> ... -> W -> 1 with SiLU activations, trained and evaluated on
 * the GPU by these kernels (no library GEMM).
 *
 * The network has no counterpart in the reference; it ranks grid points for
 * the pruned grid search and is checked against the exhaustive search.
 *
 * Products C[M][N] = sum_k A(m,k) B(k,n) (+ bias[n]), A(m,k) = A[m*lda + k]
 * (ta = 0) or A[k*lda + m] (ta = 1); B(k,n) = B[k*ldb + n] (tb = 0) or
 * B[n*ldb + k] (tb = 1).  Forward Z = X W^T + b is (ta, tb) = (0, 1); the
 * input gradient dZ W is (0, 1) on the transposed weights; the weight
 * gradient dZ^T X is (1, 0).  fk_mlp_gemm sends each product to:
 *   - the thin-layer kernels (FP32): K <= 8 (the 6-input first layer, the
 *     1-output layer's input gradient), N = 1 (the output layer), and the
 *     weight gradients with M or N <= 8 (first and last layers), the bias
 *     gradient from the same pass;
 *   - the tensor cores (mlp_tc.cu) for the hidden layers (N, K >= 64);
 *   - otherwise the FP32 tiled GEMM below (128 x 64 output tiles, K in
 *     steps of 16 through shared memory, 8 x 4 outputs per thread).
 * K is split over CTAs only for long K (the weight gradients); slices are
 * added in a fixed order, and every reduction here (slices, column sums,
 * the loss) has a fixed order, so training is reproducible run to run.
 */
#include <cuda_runtime.h>
#include <stdint.h>
#include "fteik_dev.h"

namespace fkmlp {

constexpr int TM = 128, TN = 64, TK = 16;
constexpr int NT = 256;  /* 16 x 16 threads, 8 x 4 outputs each */

__global__ void __launch_bounds__(NT) gemm_kernel(int M, int N, int K, const float *__restrict__ A,
                                                  int lda, int ta, const float *__restrict__ B,
                                                  int ldb, int tb, float *__restrict__ C, int ldc,
                                                  const float *__restrict__ bias, int accumulate)
{
    __shared__ float As[TK][TM + 4];
    __shared__ float Bs[TK][TN + 4];
    const int m0 = blockIdx.y * TM, n0 = blockIdx.x * TN;
    /* split-K: slice blockIdx.z of gridDim.z writes its partial tile to the
     * workspace C + z M N (C is then the workspace, ldc = N); a second kernel
     * adds the slices in a fixed order, so training is reproducible */
    const int kchunk = ((K + gridDim.z * TK - 1) / (gridDim.z * TK)) * TK;
    const int kb = blockIdx.z * kchunk, ke = min(K, kb + kchunk);
    const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
    float acc[8][4];
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = 0.0f;
    for (int k0 = kb; k0 < ke; k0 += TK) {
        /* A tile: TM x TK = 2048 values, 8 per thread */
        for (int t = threadIdx.x; t < TM * TK; t += NT) {
            int mm, kk;
            if (ta) { kk = t / TM; mm = t % TM; }     /* consecutive m: contiguous */
            else { mm = t / TK; kk = t % TK; }        /* consecutive k: contiguous */
            const int m = m0 + mm, k = k0 + kk;
            float v = 0.0f;
            if (m < M && k < ke) v = ta ? A[(size_t)k * lda + m] : A[(size_t)m * lda + k];
            As[kk][mm] = v;
        }
        for (int t = threadIdx.x; t < TN * TK; t += NT) {
            int nn, kk;
            if (tb) { nn = t / TK; kk = t % TK; }
            else { kk = t / TN; nn = t % TN; }
            const int n = n0 + nn, k = k0 + kk;
            float v = 0.0f;
            if (n < N && k < ke) v = tb ? B[(size_t)n * ldb + k] : B[(size_t)k * ldb + n];
            Bs[kk][nn] = v;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < TK; ++kk) {
            float a[8], b[4];
#pragma unroll
            for (int i = 0; i < 8; ++i) a[i] = As[kk][ty + 16 * i];
#pragma unroll
            for (int j = 0; j < 4; ++j) b[j] = Bs[kk][tx + 16 * j];
#pragma unroll
            for (int i = 0; i < 8; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const int m = m0 + ty + 16 * i;
        if (m >= M) continue;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int n = n0 + tx + 16 * j;
            if (n >= N) continue;
            float *c = C + (size_t)m * ldc + n;
            if (gridDim.z > 1) {
                C[((size_t)blockIdx.z * M + m) * N + n] = acc[i][j];
            } else {
                const float v = acc[i][j] + (bias ? bias[n] : 0.0f);
                *c = accumulate ? *c + v : v;
            }
        }
    }
}

/* The output value v of element (m, n) of C, the activation applied as asked:
 * act 0: C = v; act 1: C = v and C2 = silu(v) (the forward pass keeping the
 * pre-activation); act 2: C = silu(v); act 3: C = v silu'(z) with z = C2
 * (the backward pass: dz = da s (1 + z (1 - s)), s = sigmoid(z), as
 * silu_bwd_kernel). */
__device__ __forceinline__ void store_act(float *__restrict__ C, float *__restrict__ C2, size_t off, float v,
                                          int act)
{
    if (act == 3) {
        const float z = C2[off], s = fk_sigmoid(z);
        C[off] = v * s * (1.0f + z * (1.0f - s));
        return;
    }
    const float a = act ? fk_silu(v) : v;
    C[off] = act == 2 ? a : v;
    if (act == 1) C2[off] = a;
}

/* C[m][n] (+)= sum over the split slices in order + bias[n], activation as
 * store_act; with db, also db[m] = sum over the slices in order of the
 * column sums cs[z][m]. */
__global__ void splitk_reduce_kernel(int M, int N, int split, const float *__restrict__ ws, float *__restrict__ C,
                                     int ldc, const float *__restrict__ bias, int accumulate, float *__restrict__ C2,
                                     int act, const float *__restrict__ cs, float *__restrict__ db)
{
    const size_t n_el = (size_t)M * N, n_all = n_el + (db ? (size_t)M : 0);
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n_all; e += (size_t)gridDim.x * blockDim.x) {
        if (e >= n_el) {
            const int m = (int)(e - n_el);
            float v = 0.0f;
#pragma unroll 16
            for (int z = 0; z < split; ++z) v += cs[(size_t)z * M + m];
            db[m] = v;
            continue;
        }
        const int m = (int)(e / N), n = (int)(e % N);
        float v = 0.0f;
#pragma unroll 16
        for (int z = 0; z < split; ++z) v += ws[(size_t)z * n_el + e];
        if (bias) v += bias[n];
        const size_t off = (size_t)m * ldc + n;
        if (accumulate) v = C[off] + v;
        store_act(C, C2, off, v, act);
    }
}

/* The same plain sums (no bias, accumulation or activation) four outputs
 * per group of 4 threads with 16-byte loads and stores (N and ldc
 * multiples of 4, 16-byte aligned buffers): thread u of a group adds
 * slices u, u + 4, ... in order, and the group's 4 sums are added in
 * thread order (a fixed order).  The column sums as splitk_reduce_kernel. */
__global__ void splitk_reduce_vec_kernel(int M, int N, int split, const float *__restrict__ ws, float *__restrict__ C,
                                         int ldc, const float *__restrict__ cs, float *__restrict__ db)
{
    const size_t n4 = (size_t)M * N / 4, n_all = n4 + (db ? (size_t)M : 0);
    const size_t e = (blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 2;
    const int u = threadIdx.x & 3;
    /* every lane reaches the shuffles below (no early exit) */
    float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
    if (e < n4) {
#pragma unroll 4
        for (int z = u; z < split; z += 4) {
            const float4 w = reinterpret_cast<const float4 *>(ws)[(size_t)z * n4 + e];
            v.x += w.x; v.y += w.y; v.z += w.z; v.w += w.w;
        }
    }
    /* lanes 4 g .. 4 g + 3 hold one output's partial sums: ((s0 + s1) + s2) + s3 */
    float4 r;
    r.x = __shfl_sync(0xffffffffu, v.x, 0, 4); r.y = __shfl_sync(0xffffffffu, v.y, 0, 4);
    r.z = __shfl_sync(0xffffffffu, v.z, 0, 4); r.w = __shfl_sync(0xffffffffu, v.w, 0, 4);
#pragma unroll
    for (int i = 1; i < 4; ++i) {
        r.x += __shfl_sync(0xffffffffu, v.x, i, 4); r.y += __shfl_sync(0xffffffffu, v.y, i, 4);
        r.z += __shfl_sync(0xffffffffu, v.z, i, 4); r.w += __shfl_sync(0xffffffffu, v.w, i, 4);
    }
    if (u != 0 || e >= n_all) return;
    if (e < n4) {
        const int m = (int)(4 * e / N), n = (int)(4 * e % N);
        *reinterpret_cast<float4 *>(C + (size_t)m * ldc + n) = r;
    } else {
        const int m = (int)(e - n4);
        float t = 0.0f;
#pragma unroll 16
        for (int z = 0; z < split; ++z) t += cs[(size_t)z * M + m];
        db[m] = t;
    }
}

/* The same sums for few outputs and many slices (the thin layers' weight
 * gradients): one warp per output, lane l adding slices l, l + 32, ... in
 * order, then a fixed butterfly over the lanes (the same order on every
 * run).  No bias, accumulation or activation. */
__global__ void splitk_reduce_warp_kernel(int M, int N, int split, const float *__restrict__ ws,
                                          float *__restrict__ C, int ldc, const float *__restrict__ cs,
                                          float *__restrict__ db)
{
    const size_t n_el = (size_t)M * N, n_all = n_el + (db ? (size_t)M : 0);
    const size_t e = (blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (e >= n_all) return;
    const bool is_db = e >= n_el;
    const float *src = is_db ? cs + (e - n_el) : ws + e;
    const size_t stride = is_db ? (size_t)M : n_el;
    float v = 0.0f;
#pragma unroll 4
    for (int z = lane; z < split; z += 32) v += src[(size_t)z * stride];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) {
        if (is_db) db[e - n_el] = v;
        else C[(e / N) * ldc + e % N] = v;
    }
}

/* Products with K <= 8 (the first layer, 6 inputs; the output layer's
 * input gradient, K = 1), A[m][k]: thread n of a block of SK_N columns
 * keeps B(., n) in registers and runs over SK_R rows, the multiply-adds in
 * k order from zero as gemm_kernel, then the bias and the activation
 * (store_act); stores are coalesced along n. */
constexpr int SK_N = 128, SK_R = 32, SK_KMAX = 8;
__global__ void __launch_bounds__(SK_N, 4) smallk_kernel(int M, int N, int K, const float *__restrict__ A, int lda,
                                                      const float *__restrict__ B, int ldb, int tb,
                                                      float *__restrict__ C, int ldc, const float *__restrict__ bias,
                                                      int accumulate, float *__restrict__ C2, int act)
{
    const int n = blockIdx.x * SK_N + threadIdx.x;
    if (n >= N) return;
    float b[SK_KMAX];
#pragma unroll
    for (int k = 0; k < SK_KMAX; ++k) b[k] = k < K ? (tb ? B[(size_t)n * ldb + k] : B[(size_t)k * ldb + n]) : 0.0f;
    const float bn = bias ? bias[n] : 0.0f;
    for (int m0 = blockIdx.y * SK_R; m0 < M; m0 += gridDim.y * SK_R) {
        const int m1 = min(M, m0 + SK_R);
#pragma unroll 4
        for (int m = m0; m < m1; ++m) {
            float acc = 0.0f;
#pragma unroll
            for (int k = 0; k < SK_KMAX; ++k)
                if (k < K) acc = fmaf(A[(size_t)m * lda + k], b[k], acc);
            float v = acc + bn;
            const size_t off = (size_t)m * ldc + n;
            if (accumulate) v = C[off] + v;
            store_act(C, C2, off, v, act);
        }
    }
}

/* The same products four columns per thread (N, ldc multiples of 4,
 * 16-byte aligned C and C2): 64 column quads x 4 row groups per block,
 * float4 stores (and float4 loads of z for act 3); the same arithmetic per
 * element as smallk_kernel. */
constexpr int SKQ_R = 32;
__global__ void __launch_bounds__(256) smallk_quad_kernel(int M, int N, int K, const float *__restrict__ A, int lda,
                                                          const float *__restrict__ B, int ldb, int tb,
                                                          float *__restrict__ C, int ldc,
                                                          const float *__restrict__ bias, int accumulate,
                                                          float *__restrict__ C2, int act)
{
    const int t = threadIdx.x, n = blockIdx.x * 256 + 4 * (t & 63), rs = t >> 6;
    if (n >= N) return;
    float b[SK_KMAX][4];
#pragma unroll
    for (int k = 0; k < SK_KMAX; ++k)
#pragma unroll
        for (int c = 0; c < 4; ++c)
            b[k][c] = k < K ? (tb ? B[(size_t)(n + c) * ldb + k] : B[(size_t)k * ldb + n + c]) : 0.0f;
    float bn[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) bn[c] = bias ? bias[n + c] : 0.0f;
    for (int m0 = blockIdx.y * SKQ_R; m0 < M; m0 += gridDim.y * SKQ_R) {
#pragma unroll 2
        for (int i = rs; i < SKQ_R; i += 4) {
            const int m = m0 + i;
            if (m >= M) break;
            float v[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
            for (int k = 0; k < SK_KMAX; ++k)
                if (k < K) {
                    const float a = A[(size_t)m * lda + k];
#pragma unroll
                    for (int c = 0; c < 4; ++c) v[c] = fmaf(a, b[k][c], v[c]);
                }
#pragma unroll
            for (int c = 0; c < 4; ++c) v[c] = v[c] + bn[c];
            const size_t off = (size_t)m * ldc + n;
            float4 *cp = reinterpret_cast<float4 *>(C + off);
            if (accumulate) {
                const float4 o = *cp;
                v[0] = o.x + v[0]; v[1] = o.y + v[1]; v[2] = o.z + v[2]; v[3] = o.w + v[3];
            }
            if (act == 3) {
                const float4 z = *reinterpret_cast<const float4 *>(C2 + off);
                const float zs[4] = {z.x, z.y, z.z, z.w};
#pragma unroll
                for (int c = 0; c < 4; ++c) {
                    const float sg = fk_sigmoid(zs[c]);
                    v[c] = v[c] * sg * (1.0f + zs[c] * (1.0f - sg));
                }
                *cp = make_float4(v[0], v[1], v[2], v[3]);
            } else if (act == 2) {
                *cp = make_float4(fk_silu(v[0]), fk_silu(v[1]), fk_silu(v[2]), fk_silu(v[3]));
            } else {
                *cp = make_float4(v[0], v[1], v[2], v[3]);
                if (act == 1)
                    *reinterpret_cast<float4 *>(C2 + off) =
                        make_float4(fk_silu(v[0]), fk_silu(v[1]), fk_silu(v[2]), fk_silu(v[3]));
            }
        }
    }
}

/* Products with N = 1 (the output layer), A[m][k]: one thread per row, the
 * multiply-adds in k order from zero as gemm_kernel; a block of 256
 * threads brings 64 rows x 64 k of A into a [64][65] tile by coalesced
 * loads (16 per thread, all in flight), then 64 of them run the rows'
 * chains; B(k, 0) = B[k bs]. */
constexpr int GV_R = 64, GV_K = 64, GV_NT = 256;
__global__ void __launch_bounds__(GV_NT) gemv_kernel(int M, int K, const float *__restrict__ A, int lda,
                                                     const float *__restrict__ B, int bs, float *__restrict__ C,
                                                     int ldc, const float *__restrict__ bias, int accumulate)
{
    __shared__ float tile[GV_R][GV_K + 1];
    __shared__ float sb[GV_K];
    const int m0 = blockIdx.x * GV_R, t = threadIdx.x, c = t & (GV_K - 1), r0 = t / GV_K;
    float acc = 0.0f;
    for (int k0 = 0; k0 < K; k0 += GV_K) {
        const int kn = min(GV_K, K - k0);
        float v[GV_R * GV_K / GV_NT];
#pragma unroll
        for (int i = 0; i < GV_R * GV_K / GV_NT; ++i) {
            const int m = m0 + r0 + i * (GV_NT / GV_K);
            v[i] = (m < M && c < kn) ? A[(size_t)m * lda + k0 + c] : 0.0f;
        }
#pragma unroll
        for (int i = 0; i < GV_R * GV_K / GV_NT; ++i) tile[r0 + i * (GV_NT / GV_K)][c] = v[i];
        if (t < kn) sb[t] = B[(size_t)(k0 + t) * bs];
        __syncthreads();
        if (t < GV_R)
            for (int k = 0; k < kn; ++k) acc = fmaf(tile[t][k], sb[k], acc);
        __syncthreads();
    }
    const int m = m0 + t;
    if (t < GV_R && m < M) {
        const float v = acc + (bias ? bias[0] : 0.0f);
        float *cp = C + (size_t)m * ldc;
        *cp = accumulate ? *cp + v : v;
    }
}

/* Weight gradients of the thin layers: C[m][n] = sum_k A[k lda + m]
 * B[k ldb + n] with N <= 8 (BIG_M: one thread per m, B's row broadcast) or
 * M <= 8 (one thread per n, A's row broadcast), K in slices of kchunk (one
 * per blockIdx.y): the partial products go to ws[slice][M][N] and the
 * column sums of A over the slice to cs[slice][M] (the bias gradient),
 * each in k order; a reduction adds the slices in order.  SC: the small
 * dimension when known at compile time (the surrogate's 6 inputs and 1
 * output), else 0 (read from M or N). */
constexpr int TS_MAX = 8;

/* The same products with 16-byte loads along the wide dimension D (M when
 * BIG_M, else N; D and its leading dimension multiples of 4, 16-byte
 * aligned): a block covers 256 of D (64 quads) and one K slice; its 4
 * row groups (threads t / 64) take rows kb + g, kb + g + 4, ... of the
 * slice, the narrow operand's rows of the slice (S values each) staged in
 * shared memory; the groups' sums are added in group order.  Same outputs
 * and layout as tn_small_kernel; the order of the k sums differs, fixed. */
constexpr int TQ_K = 64;   /* rows per slice */
template <bool BIG_M, int S>
__global__ void __launch_bounds__(256) tn_quad_kernel(int M, int N, int K, const float *__restrict__ A, int lda,
                                                      const float *__restrict__ B, int ldb, float *__restrict__ ws,
                                                      float *__restrict__ cs)
{
    static_assert(BIG_M || S <= 4, "narrow A: its column sums ride in the first 4 sums");
    __shared__ float nar[TQ_K * S];
    __shared__ float red[4][256][S + 1];
    const int t = threadIdx.x, g = t >> 6, dq = t & 63;
    const int D = BIG_M ? M : N;
    const int d = blockIdx.x * 256 + 4 * dq;
    const int kb = blockIdx.y * TQ_K, ke = min(K, kb + TQ_K);
    for (int i = t; i < (ke - kb) * S; i += 256) {
        const int k = kb + i / S, j = i % S;
        nar[i] = BIG_M ? B[(size_t)k * ldb + j] : A[(size_t)k * lda + j];
    }
    __syncthreads();
    float acc[4][S], sum[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        sum[c] = 0.0f;
#pragma unroll
        for (int j = 0; j < S; ++j) acc[c][j] = 0.0f;
    }
    if (d < D) {
        const float *wide = BIG_M ? A + d : B + d;
        const size_t ld = BIG_M ? (size_t)lda : (size_t)ldb;
#pragma unroll 4
        for (int k = kb + g; k < ke; k += 4) {
            const float4 w = *reinterpret_cast<const float4 *>(wide + (size_t)k * ld);
            const float wv[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
            for (int j = 0; j < S; ++j) {
                const float nv = nar[(k - kb) * S + j];
#pragma unroll
                for (int c = 0; c < 4; ++c) acc[c][j] = fmaf(wv[c], nv, acc[c][j]);
                if (!BIG_M) sum[j < 4 ? j : 0] += (j < 4) ? nv : 0.0f;
            }
            if (BIG_M)
#pragma unroll
                for (int c = 0; c < 4; ++c) sum[c] += wv[c];
        }
    }
#pragma unroll
    for (int c = 0; c < 4; ++c) {
#pragma unroll
        for (int j = 0; j < S; ++j) red[g][4 * dq + c][j] = acc[c][j];
        red[g][4 * dq + c][S] = sum[c];
    }
    __syncthreads();
    const int dl = blockIdx.x * 256 + t;
    if (dl >= D) return;
    float *w = ws + (size_t)blockIdx.y * M * N;
#pragma unroll
    for (int j = 0; j < S; ++j) {
        const float v = ((red[0][t][j] + red[1][t][j]) + red[2][t][j]) + red[3][t][j];
        if (BIG_M) w[(size_t)dl * N + j] = v;
        else w[(size_t)j * N + dl] = v;
    }
    if (!cs) return;
    if (BIG_M) {
        cs[(size_t)blockIdx.y * M + dl] = ((red[0][t][S] + red[1][t][S]) + red[2][t][S]) + red[3][t][S];
    } else if (dl == 0) {
        /* the narrow operand's column sums: thread 4 dq + c of group g kept
         * sum[c] = its group's sum of A(c, k) (c < S <= 4) */
#pragma unroll
        for (int j = 0; j < S; ++j)
            cs[(size_t)blockIdx.y * M + j] = ((red[0][j][S] + red[1][j][S]) + red[2][j][S]) + red[3][j][S];
    }
}

template <bool BIG_M, int SC>
__global__ void __launch_bounds__(256) tn_small_kernel(int M, int N, int K, int kchunk, const float *__restrict__ A,
                                                       int lda, const float *__restrict__ B, int ldb,
                                                       float *__restrict__ ws, float *__restrict__ cs)
{
    constexpr int SM_ = SC ? SC : TS_MAX;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;   /* m (BIG_M) or n */
    const int S = SC ? SC : (BIG_M ? N : M);
    if (i >= (BIG_M ? M : N)) return;
    const int kb = blockIdx.y * kchunk, ke = min(K, kb + kchunk);
    float acc[SM_], sum[SM_];
#pragma unroll
    for (int j = 0; j < SM_; ++j) acc[j] = sum[j] = 0.0f;
#pragma unroll 8
    for (int k = kb; k < ke; ++k) {
        if (BIG_M) {
            const float a = A[(size_t)k * lda + i];
            sum[0] += a;
#pragma unroll
            for (int j = 0; j < SM_; ++j)
                if (j < S) acc[j] = fmaf(a, B[(size_t)k * ldb + j], acc[j]);
        } else {
            const float b = B[(size_t)k * ldb + i];
#pragma unroll
            for (int j = 0; j < SM_; ++j)
                if (j < S) {
                    const float a = A[(size_t)k * lda + j];
                    acc[j] = fmaf(a, b, acc[j]);
                    sum[j] += a;
                }
        }
    }
    float *w = ws + (size_t)blockIdx.y * M * N;
#pragma unroll
    for (int j = 0; j < SM_; ++j)
        if (j < S) {
            if (BIG_M) w[(size_t)i * N + j] = acc[j];
            else w[(size_t)j * N + i] = acc[j];
        }
    if (cs) {
        if (BIG_M) cs[(size_t)blockIdx.y * M + i] = sum[0];
        else if (i == 0)
#pragma unroll
            for (int j = 0; j < SM_; ++j)
                if (j < S) cs[(size_t)blockIdx.y * M + j] = sum[j];
    }
}

__device__ __forceinline__ float sigmoid(float z) { return fk_sigmoid(z); }

__global__ void silu_kernel(size_t n, const float *__restrict__ z, float *__restrict__ a)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const float v = z[i];
        a[i] = fk_silu(v);
    }
}

__global__ void silu_inplace_kernel(size_t n, float *a)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const float v = a[i];
        a[i] = fk_silu(v);
    }
}

/* dz = da * d/dz silu(z) = da * s (1 + z (1 - s)), s = sigmoid(z) */
__global__ void silu_bwd_kernel(size_t n, const float *__restrict__ z, const float *__restrict__ da,
                                float *__restrict__ dz)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const float v = z[i], s = sigmoid(v);
        dz[i] = da[i] * s * (1.0f + v * (1.0f - s));
    }
}

__global__ void silu_bwd_inplace_kernel(size_t n, const float *__restrict__ z, float *d)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const float v = z[i], s = sigmoid(v);
        d[i] = d[i] * s * (1.0f + v * (1.0f - s));
    }
}

/* db[n] = sum_m dz[m][n] in a fixed order: block (column group of 32, row
 * chunk r) sums rows r CR .. r CR + CR - 1, warp w every 8th of them, the
 * 8 warps' sums added in order into part[r][n]; colsum_final adds the
 * chunks in order. */
constexpr int CS_CR = 256;
__global__ void colsum_kernel(int M, int N, const float *__restrict__ dz, float *__restrict__ part)
{
    __shared__ float red[8][32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int n = blockIdx.x * 32 + lane;
    const int m0 = blockIdx.y * CS_CR, m1 = min(M, m0 + CS_CR);
    float s = 0.0f;
    if (n < N)
        for (int m = m0 + w; m < m1; m += 8) s += dz[(size_t)m * N + n];
    red[w][lane] = s;
    __syncthreads();
    if (w == 0 && n < N) {
        float t = red[0][lane];
        for (int k = 1; k < 8; ++k) t += red[k][lane];
        part[(size_t)blockIdx.y * N + n] = t;
    }
}

__global__ void colsum_final_kernel(int N, int nchunk, const float *__restrict__ part, float *__restrict__ db)
{
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N) return;
    float s = 0.0f;
    for (int r = 0; r < nchunk; ++r) s += part[(size_t)r * N + n];
    db[n] = s;
}

/* mean squared error over n outputs: dpred = 2 (pred - y) / n; the loss in
 * a fixed order: block sums into part[], and the block that finishes last
 * (a counter, reset by it) adds them in a fixed order into *loss */
__global__ void mse_kernel(int n, const float *__restrict__ pred, const float *__restrict__ y,
                           float *__restrict__ dpred, double *__restrict__ loss, double *part, unsigned *count)
{
    __shared__ double red[256];
    __shared__ bool last;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double l = 0.0;
    if (i < n) {
        const float d = pred[i] - y[i];
        dpred[i] = 2.0f * d / (float)n;
        l = (double)d * (double)d / (double)n;
    }
    red[threadIdx.x] = l;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        part[blockIdx.x] = red[0];
        __threadfence();
        last = atomicAdd(count, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;   /* block-uniform: read after the barrier */
    /* the last block adds the block sums in a fixed order: thread i the
     * sums i, i + 256, ... in order, then a fixed tree */
    __threadfence();
    double t = 0.0;
    for (unsigned b = threadIdx.x; b < gridDim.x; b += blockDim.x)
        t += reinterpret_cast<volatile double *>(part)[b];
    red[threadIdx.x] = t;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        *loss = red[0];
        *count = 0;
    }
}

__global__ void adam_kernel(size_t n, float *__restrict__ w, const float *__restrict__ g,
                            float *__restrict__ m, float *__restrict__ v, float lr, float b1,
                            float b2, float eps, float c1, float c2)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.0f - b1) * gi;
        const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    }
}

/* Adam with the step's learning rate and bias corrections read from the
 * device (sched[3 t .. 3 t + 2] = lr_t, 1 - b1^t, 1 - b2^t, t = *tdev), so
 * that a captured training step replays with the schedule moving on. */
__global__ void adam_sched_kernel(size_t n, float *__restrict__ w, const float *__restrict__ g,
                                  float *__restrict__ m, float *__restrict__ v, const float *__restrict__ sched,
                                  const long long *__restrict__ tdev, float b1, float b2, float eps)
{
    const long long t = *tdev;
    const float lr = sched[3 * t], c1 = sched[3 * t + 1], c2 = sched[3 * t + 2];
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.0f - b1) * gi;
        const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    }
}

__global__ void step_inc_kernel(long long *tdev) { *tdev += 1; }

/* wt = the transposes of the listed layers' weights: W [out][in] at off
 * becomes W^T [in][out] at the same offset (the input-gradient products
 * then read k-contiguous rows); blockIdx.y = the layer */
constexpr int TL_MAX = 16;
struct TLayers {
    int n;
    long long off[TL_MAX];
    int in[TL_MAX], out[TL_MAX];
};

__global__ void transpose_layers_kernel(TLayers L, const float *__restrict__ w, float *__restrict__ wt)
{
    const int l = blockIdx.y;
    if (l >= L.n) return;
    const int in = L.in[l], out = L.out[l];
    const long long off = L.off[l];
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < (size_t)in * out;
         e += (size_t)gridDim.x * blockDim.x) {
        const int j = (int)(e / out), o = (int)(e % out);
        wt[off + e] = w[off + (size_t)o * in + j];
    }
}

/* counter-based hash (splitmix64 finaliser) */
__device__ __forceinline__ uint64_t mix64(uint64_t x)
{
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

struct Geom {
    int nz, nx, ny, ntf, ldgrd;
    float dz, dx, dy;
    float vref;
};

__device__ __forceinline__ void norm_inputs(const Geom &G, float zg, float xg, float yg, float zs,
                                            float xs, float ys, float *x)
{
    const float ez = fmaxf((G.nz - 1) * G.dz, 1e-30f), ex = fmaxf((G.nx - 1) * G.dx, 1e-30f),
                ey = fmaxf((G.ny - 1) * G.dy, 1e-30f);
    x[0] = 2.0f * zg / ez - 1.0f;
    x[1] = 2.0f * xg / ex - 1.0f;
    x[2] = 2.0f * yg / ey - 1.0f;
    x[3] = 2.0f * zs / ez - 1.0f;
    x[4] = 2.0f * xs / ex - 1.0f;
    x[5] = 2.0f * ys / ey - 1.0f;
}

/* One training batch from the tables: sample b of step t draws sample id
 * j in [0, nsamp) and from it a table i and a grid node g; input = the
 * normalised node and station positions, target tau = T v_ref / distance
 * (distance floored at half a cell). */
__global__ void sample_kernel(Geom G, const float *__restrict__ tables, const float *__restrict__ sta,
                              uint64_t seed, long long nsamp, long long t, const long long *__restrict__ tdev,
                              int B, float *__restrict__ x, float *__restrict__ y)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= B) return;
    if (tdev) t = *tdev;   /* a captured step: the step number from the device */
    const long long ngrd = (long long)G.nz * G.nx * G.ny;
    const uint64_t j = mix64(seed ^ mix64((uint64_t)t * 0x100000001B3ull + (uint64_t)b)) % (uint64_t)nsamp;
    const uint64_t h = mix64(seed * 0x2545F4914F6CDD1Dull + j);
    const int i = (int)(h % (uint64_t)G.ntf);
    const long long g = (long long)(mix64(h) % (uint64_t)ngrd);
    const int iz = (int)(g % G.nz), ix = (int)((g / G.nz) % G.nx), iy = (int)(g / ((long long)G.nz * G.nx));
    const float zg = iz * G.dz, xg = ix * G.dx, yg = iy * G.dy;
    const float zs = sta[3 * i], xs = sta[3 * i + 1], ys = sta[3 * i + 2];
    norm_inputs(G, zg, xg, yg, zs, xs, ys, x + (size_t)b * 6);
    const float hmin = fminf(G.dz, fminf(G.dx, G.dy));
    const float d = fmaxf(sqrtf((zg - zs) * (zg - zs) + (xg - xs) * (xg - xs) + (yg - ys) * (yg - ys)), 0.5f * hmin);
    y[b] = tables[(size_t)i * G.ldgrd + g] * G.vref / d;
}

/* Inputs of the coarse lattice: row r = table i, coarse node c (z fastest);
 * the node sits at the centre of its fine block (bz x bx x by nodes, the
 * part inside the grid), in general between grid nodes. */
__device__ __forceinline__ float block_centre(int c, int b, int n, float h)
{
    const int lo = b * c, hi = min(b * c + b, n) - 1;
    return 0.5f * (float)(lo + hi) * h;
}

__global__ void coarse_inputs_kernel(Geom G, const float *__restrict__ sta, int bz, int bx, int by, int ncz,
                                     int ncx, int ncy, long long r0, long long nrow, float *__restrict__ x,
                                     float *__restrict__ dist)
{
    const long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (r >= nrow) return;
    const long long row = r0 + r;
    const long long nc = (long long)ncz * ncx * ncy;
    const int i = (int)(row / nc);
    const long long c = row % nc;
    const int cz = (int)(c % ncz), cx = (int)((c / ncz) % ncx), cy = (int)(c / ((long long)ncz * ncx));
    const float zg = block_centre(cz, bz, G.nz, G.dz), xg = block_centre(cx, bx, G.nx, G.dx),
                yg = block_centre(cy, by, G.ny, G.dy);
    const float zs = sta[3 * i], xs = sta[3 * i + 1], ys = sta[3 * i + 2];
    norm_inputs(G, zg, xg, yg, zs, xs, ys, x + (size_t)r * 6);
    dist[r] = sqrtf((zg - zs) * (zg - zs) + (xg - xs) * (xg - xs) + (yg - ys) * (yg - ys)) / G.vref;
}

/* T = tau * distance / v_ref into the coarse table layout [ntf][ldc] */
__global__ void coarse_store_kernel(long long r0, long long nrow, long long nc, int ldc,
                                    const float *__restrict__ tau, const float *__restrict__ dist,
                                    float *__restrict__ out)
{
    const long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (r >= nrow) return;
    const long long row = r0 + r;
    out[(row / nc) * ldc + row % nc] = tau[r] * dist[r];
}

} // namespace fkmlp

using namespace fkmlp;

static int grid1d(size_t n) { size_t b = (n + 255) / 256; return (int)(b < 4096 ? (b ? b : 1) : 4096); }

extern "C" int fk_mlp_gemm_tc(int prod, int M, int N, int K, const float *A, int lda, int ta, const float *B,
                              int ldb, int tb, float *C, int ldc, const float *bias, int accumulate, float *C2,
                              int act, int split, float *ws, float *colsum, int *error, cudaStream_t s);

/* 0: every GEMM on the CUDA cores in FP32; 1 or 3: GEMMs with N and K of at
 * least 64 (the hidden layers) on the tensor cores with that many BF16
 * products (mlp_tc.cu) */
static int g_tensor = 1;
static int *g_tc_error = nullptr;

extern "C" void fk_mlp_set_tensor(int products) { g_tensor = products; }
extern "C" int fk_mlp_get_tensor(void) { return g_tensor; }

/* the tensor-core kernels' error word (allocated on first use, outside any capture) */
extern "C" int *fk_mlp_tc_error_word(cudaStream_t s)
{
    if (!g_tc_error) {
        cudaError_t e = cudaMalloc((void **)&g_tc_error, sizeof(int));
        if (e == cudaSuccess) e = cudaMemsetAsync(g_tc_error, 0, sizeof(int), s);
        if (e != cudaSuccess) { g_tc_error = nullptr; return nullptr; }
    }
    return g_tc_error;
}

/* the tensor-core kernels' error word (a wait that timed out), read and cleared */
extern "C" int fk_mlp_tc_status(cudaStream_t s)
{
    if (!g_tc_error) return 0;
    int v = 0;
    cudaError_t e = cudaMemcpyAsync(&v, g_tc_error, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e == cudaSuccess && v) e = cudaMemsetAsync(g_tc_error, 0, sizeof(int), s);
    return e != cudaSuccess ? (int)e : v;
}

static float *g_ws = nullptr;
static size_t g_ws_cap = 0;

/* split-K / slice workspace; grows on a training run's first (eager) step,
 * never during a capture */
static int workspace(size_t need, cudaStream_t s)
{
    if (need <= g_ws_cap) return 0;
    cudaError_t e = cudaStreamSynchronize(s);   /* the old workspace may still be read */
    if (e == cudaSuccess && g_ws) e = cudaFree(g_ws);
    g_ws = nullptr;
    g_ws_cap = 0;
    if (e == cudaSuccess) e = cudaMalloc((void **)&g_ws, sizeof(float) * need);
    if (e != cudaSuccess) return (int)e;
    g_ws_cap = need;
    return 0;
}

extern "C" int fk_mlp_colsum(int M, int N, const float *dz, float *db, cudaStream_t s);

/* C = A B (+ bias) with the activation act (store_act) and, with colsum
 * (weight gradients, ta = 1 and lda = M only), colsum[m] = sum_k A(m, k)
 * (the bias gradient).  Thin products go to their own CUDA-core kernels
 * (K <= 8; N = 1; weight gradients with M or N <= 8), the hidden layers'
 * to the tensor cores (g_tensor), the rest to gemm_kernel; K is split
 * over CTAs only when it is long (the weight gradients, K = the batch),
 * the slices added in a fixed order, so every result is reproducible. */
extern "C" int fk_mlp_gemm(int M, int N, int K, const float *A, int lda, int ta, const float *B, int ldb,
                           int tb, float *C, int ldc, const float *bias, int accumulate, float *C2, int act,
                           float *colsum, cudaStream_t s)
{
    if (M <= 0 || N <= 0) return 0;
    if ((colsum && (!ta || lda != M)) || (act && !C2 && act != 2) || act < 0 || act > 3)
        return (int)cudaErrorInvalidValue;
    if (!ta && N == 1 && act == 0) {
        gemv_kernel<<<(M + GV_R - 1) / GV_R, GV_NT, 0, s>>>(M, K, A, lda, B, tb ? 1 : ldb, C, ldc, bias,
                                                            accumulate);
        return (int)cudaGetLastError();
    }
    const bool al16 = ((uintptr_t)C & 15) == 0 && (!C2 || ((uintptr_t)C2 & 15) == 0);
    if (!ta && K <= SK_KMAX && N % 4 == 0 && ldc % 4 == 0 && al16) {
        const int rb = (M + SKQ_R - 1) / SKQ_R;
        smallk_quad_kernel<<<dim3((N + 255) / 256, rb < 65535 ? rb : 65535), 256, 0, s>>>(
            M, N, K, A, lda, B, ldb, tb, C, ldc, bias, accumulate, C2, act);
        return (int)cudaGetLastError();
    }
    if (!ta && K <= SK_KMAX) {
        const int rb = (M + SK_R - 1) / SK_R;
        smallk_kernel<<<dim3((N + SK_N - 1) / SK_N, rb < 65535 ? rb : 65535), SK_N, 0, s>>>(
            M, N, K, A, lda, B, ldb, tb, C, ldc, bias, accumulate, C2, act);
        return (int)cudaGetLastError();
    }
    if (ta && !tb && ((N == 6 && M % 4 == 0 && lda % 4 == 0 && ((uintptr_t)A & 15) == 0) ||
                      (M == 1 && N % 4 == 0 && ldb % 4 == 0 && ((uintptr_t)B & 15) == 0))) {
        /* the surrogate's first and last layers: 16-byte loads along the wide side */
        const bool big_m = N == 6;
        const int nchunk = (K + TQ_K - 1) / TQ_K;
        const int e = workspace((size_t)nchunk * M * N + (size_t)nchunk * M, s);
        if (e) return e;
        float *cs = g_ws + (size_t)nchunk * M * N;
        const dim3 grid(((big_m ? M : N) + 255) / 256, nchunk);
        if (big_m)
            tn_quad_kernel<true, 6><<<grid, 256, 0, s>>>(M, N, K, A, lda, B, ldb, g_ws, cs);
        else
            tn_quad_kernel<false, 1><<<grid, 256, 0, s>>>(M, N, K, A, lda, B, ldb, g_ws, cs);
        const size_t nout = (size_t)M * N + M;
        if (!bias && !accumulate && !act && ldc >= N)
            splitk_reduce_warp_kernel<<<(unsigned)((nout * 32 + 255) / 256), 256, 0, s>>>(M, N, nchunk, g_ws, C, ldc,
                                                                                          cs, colsum);
        else
            splitk_reduce_kernel<<<grid1d(nout), 256, 0, s>>>(M, N, nchunk, g_ws, C, ldc, bias, accumulate, C2, act,
                                                              cs, colsum);
        return (int)cudaGetLastError();
    }
    if (ta && !tb && (N <= TS_MAX || M <= TS_MAX)) {
        const bool big_m = N <= TS_MAX;
        const int nb = ((big_m ? M : N) + 255) / 256;
        int nchunk = 1;
        while (nb * nchunk < 148 && K / (nchunk * 2) >= 64) nchunk *= 2;
        const int kchunk = (K + nchunk - 1) / nchunk;
        const int e = workspace((size_t)nchunk * M * N + (size_t)nchunk * M, s);
        if (e) return e;
        float *cs = g_ws + (size_t)nchunk * M * N;
        const dim3 grid(nb, nchunk);
        if (big_m && N == 6)
            tn_small_kernel<true, 6><<<grid, 256, 0, s>>>(M, N, K, kchunk, A, lda, B, ldb, g_ws, cs);
        else if (big_m)
            tn_small_kernel<true, 0><<<grid, 256, 0, s>>>(M, N, K, kchunk, A, lda, B, ldb, g_ws, cs);
        else if (M == 1)
            tn_small_kernel<false, 1><<<grid, 256, 0, s>>>(M, N, K, kchunk, A, lda, B, ldb, g_ws, cs);
        else
            tn_small_kernel<false, 0><<<grid, 256, 0, s>>>(M, N, K, kchunk, A, lda, B, ldb, g_ws, cs);
        const size_t nout = (size_t)M * N + M;
        if (!bias && !accumulate && !act && ldc >= N)
            splitk_reduce_warp_kernel<<<(unsigned)((nout * 32 + 255) / 256), 256, 0, s>>>(M, N, nchunk, g_ws, C, ldc,
                                                                                          cs, colsum);
        else
            splitk_reduce_kernel<<<grid1d(nout), 256, 0, s>>>(M, N, nchunk, g_ws, C, ldc, bias, accumulate, C2, act,
                                                              cs, colsum);
        return (int)cudaGetLastError();
    }
    if (g_tensor && N >= 64 && N <= 256 && K >= 64 && M >= 64) {
        if (!fk_mlp_tc_error_word(s)) return (int)cudaErrorMemoryAllocation;
        /* long K with few 128-row tiles for the 148 SMs (the weight
         * gradients, K = the batch): split K, each slice 256 or more */
        const int mt = (M + 127) / 128;
        int split = 1;
        while (mt * split < 148 && K / (split * 2) >= 256) split *= 2;
        const bool cs_fused = colsum && K % 64 == 0;
        float *cs = nullptr;
        if (split > 1) {
            const int e = workspace((size_t)split * M * N + (cs_fused ? (size_t)split * M : 0), s);
            if (e) return e;
            if (cs_fused) cs = g_ws + (size_t)split * M * N;
        } else if (cs_fused) {
            cs = colsum;
        }
        int e = fk_mlp_gemm_tc(g_tensor, M, N, K, A, lda, ta, B, ldb, tb, C, ldc, bias, accumulate, C2, act, split,
                               g_ws, cs, g_tc_error, s);
        if (!e && split > 1) {
            const size_t nout = (size_t)M * N + (cs_fused ? M : 0);
            if (!bias && !accumulate && !act && N % 4 == 0 && ldc % 4 == 0 && ((uintptr_t)C & 15) == 0)
                splitk_reduce_vec_kernel<<<(unsigned)((4 * ((size_t)M * N / 4 + (cs_fused ? M : 0)) + 255) / 256), 256, 0,
                                           s>>>(M, N, split, g_ws, C, ldc, cs, cs_fused ? colsum : nullptr);
            else
                splitk_reduce_kernel<<<grid1d(nout), 256, 0, s>>>(M, N, split, g_ws, C, ldc, bias, accumulate, C2, act,
                                                                  cs, cs_fused ? colsum : nullptr);
            e = (int)cudaGetLastError();
        }
        if (!e && colsum && !cs_fused) e = fk_mlp_colsum(K, M, A, colsum, s);
        return e;
    }
    if (act && ldc != N) return (int)cudaErrorInvalidValue;   /* the activation pass needs a contiguous C */
    const int tiles = ((N + TN - 1) / TN) * ((M + TM - 1) / TM);
    /* long K with few output tiles (weight gradients): split K over CTAs */
    int split = 1;
    while (tiles * split < 128 && K / (split * 2) >= 256) split *= 2;
    dim3 grid((N + TN - 1) / TN, (M + TM - 1) / TM, split);
    cudaError_t e;
    if (split == 1) {
        gemm_kernel<<<grid, NT, 0, s>>>(M, N, K, A, lda, ta, B, ldb, tb, C, ldc, bias, accumulate);
        /* the activation as a second pass over the contiguous C */
        if (act == 1)
            silu_kernel<<<grid1d((size_t)M * N), 256, 0, s>>>((size_t)M * N, C, C2);
        else if (act == 2)
            silu_inplace_kernel<<<grid1d((size_t)M * N), 256, 0, s>>>((size_t)M * N, C);
        else if (act == 3)
            silu_bwd_inplace_kernel<<<grid1d((size_t)M * N), 256, 0, s>>>((size_t)M * N, C2, C);
        e = cudaGetLastError();
    } else {
        /* partial tiles into the workspace, then an ordered reduction */
        const int ew = workspace((size_t)split * M * N, s);
        if (ew) return ew;
        gemm_kernel<<<grid, NT, 0, s>>>(M, N, K, A, lda, ta, B, ldb, tb, g_ws, N, nullptr, 0);
        e = cudaGetLastError();
        if (e == cudaSuccess)
            splitk_reduce_kernel<<<grid1d((size_t)M * N), 256, 0, s>>>(M, N, split, g_ws, C, ldc, bias, accumulate,
                                                                       C2, act, nullptr, nullptr);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess && colsum) return fk_mlp_colsum(K, M, A, colsum, s);
    return (int)e;
}

extern "C" int fk_mlp_silu(size_t n, const float *z, float *a, cudaStream_t s)
{
    silu_kernel<<<grid1d(n), 256, 0, s>>>(n, z, a);
    return (int)cudaGetLastError();
}

extern "C" int fk_mlp_silu_bwd(size_t n, const float *z, const float *da, float *dz, cudaStream_t s)
{
    silu_bwd_kernel<<<grid1d(n), 256, 0, s>>>(n, z, da, dz);
    return (int)cudaGetLastError();
}

static float *g_colsum = nullptr;
static size_t g_colsum_cap = 0;

extern "C" int fk_mlp_colsum(int M, int N, const float *dz, float *db, cudaStream_t s)
{
    const int nchunk = (M + CS_CR - 1) / CS_CR;
    const size_t need = (size_t)nchunk * N;
    if (need > g_colsum_cap) {   /* grows on the first (eager) step, never during a capture */
        cudaError_t e = cudaStreamSynchronize(s);
        if (e == cudaSuccess && g_colsum) e = cudaFree(g_colsum);
        g_colsum = nullptr;
        g_colsum_cap = 0;
        if (e == cudaSuccess) e = cudaMalloc((void **)&g_colsum, sizeof(float) * need);
        if (e != cudaSuccess) return (int)e;
        g_colsum_cap = need;
    }
    colsum_kernel<<<dim3((N + 31) / 32, nchunk), 256, 0, s>>>(M, N, dz, g_colsum);
    colsum_final_kernel<<<(N + 127) / 128, 128, 0, s>>>(N, nchunk, g_colsum, db);
    return (int)cudaGetLastError();
}

static double *g_mse_part = nullptr;
static unsigned *g_mse_count = nullptr;
static int g_mse_cap = 0;

/* *loss = the mean squared error (written, not added) */
extern "C" int fk_mlp_mse(int n, const float *pred, const float *y, float *dpred, double *loss, cudaStream_t s)
{
    const int nb = (n + 255) / 256;
    if (nb > g_mse_cap) {   /* grows on a training run's first (eager) step, never during a capture */
        cudaError_t e = cudaStreamSynchronize(s);
        if (e == cudaSuccess && g_mse_part) e = cudaFree(g_mse_part);
        g_mse_part = nullptr;
        g_mse_cap = 0;
        if (e == cudaSuccess) e = cudaMalloc((void **)&g_mse_part, sizeof(double) * nb);
        if (e == cudaSuccess && !g_mse_count) {
            e = cudaMalloc((void **)&g_mse_count, sizeof(unsigned));
            if (e == cudaSuccess) e = cudaMemsetAsync(g_mse_count, 0, sizeof(unsigned), s);
        }
        if (e != cudaSuccess) return (int)e;
        g_mse_cap = nb;
    }
    mse_kernel<<<nb, 256, 0, s>>>(n, pred, y, dpred, loss, g_mse_part, g_mse_count);
    return (int)cudaGetLastError();
}

extern "C" int fk_mlp_adam(size_t n, float *w, const float *g, float *m, float *v, float lr, float b1,
                           float b2, float eps, float c1, float c2, cudaStream_t s)
{
    adam_kernel<<<grid1d(n), 256, 0, s>>>(n, w, g, m, v, lr, b1, b2, eps, c1, c2);
    return (int)cudaGetLastError();
}

extern "C" int fk_mlp_adam_sched(size_t n, float *w, const float *g, float *m, float *v, const float *sched,
                                 const long long *tdev, float b1, float b2, float eps, cudaStream_t s)
{
    adam_sched_kernel<<<grid1d(n), 256, 0, s>>>(n, w, g, m, v, sched, tdev, b1, b2, eps);
    return (int)cudaGetLastError();
}

extern "C" int fk_mlp_transpose_layers(int n, const long long *off, const int *in, const int *out, const float *w,
                                       float *wt, cudaStream_t s)
{
    if (n <= 0) return 0;
    if (n > TL_MAX) return (int)cudaErrorInvalidValue;
    TLayers L;
    L.n = n;
    for (int i = 0; i < n; ++i) { L.off[i] = off[i]; L.in[i] = in[i]; L.out[i] = out[i]; }
    transpose_layers_kernel<<<dim3(64, n), 256, 0, s>>>(L, w, wt);
    return (int)cudaGetLastError();
}

extern "C" int fk_mlp_step_inc(long long *tdev, cudaStream_t s)
{
    step_inc_kernel<<<1, 1, 0, s>>>(tdev);
    return (int)cudaGetLastError();
}

extern "C" int fk_mlp_sample(int nz, int nx, int ny, double dz, double dx, double dy, int ntf, int ldgrd,
                             double vref, const float *tables, const float *sta, unsigned long long seed,
                             long long nsamp, long long step, const long long *step_dev, int B, float *x,
                             float *y, cudaStream_t s)
{
    Geom G{nz, nx, ny, ntf, ldgrd, (float)dz, (float)dx, (float)dy, (float)vref};
    sample_kernel<<<(B + 255) / 256, 256, 0, s>>>(G, tables, sta, (uint64_t)seed, nsamp, step, step_dev, B, x,
                                                  y);
    return (int)cudaGetLastError();
}

extern "C" int fk_mlp_coarse_inputs(int nz, int nx, int ny, double dz, double dx, double dy, int ntf,
                                    double vref, const float *sta, int bz, int bx, int by, int ncz, int ncx,
                                    int ncy, long long r0, long long nrow, float *x, float *dist, cudaStream_t s)
{
    Geom G{nz, nx, ny, ntf, 0, (float)dz, (float)dx, (float)dy, (float)vref};
    coarse_inputs_kernel<<<(unsigned)((nrow + 255) / 256), 256, 0, s>>>(G, sta, bz, bx, by, ncz, ncx, ncy, r0,
                                                                      nrow, x, dist);
    return (int)cudaGetLastError();
}

extern "C" int fk_mlp_coarse_store(long long r0, long long nrow, long long nc, int ldc, const float *tau,
                                   const float *dist, float *out, cudaStream_t s)
{
    coarse_store_kernel<<<(unsigned)((nrow + 255) / 256), 256, 0, s>>>(r0, nrow, nc, ldc, tau, dist, out);
    return (int)cudaGetLastError();
}
