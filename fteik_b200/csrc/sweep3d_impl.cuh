/*
 * sweep3d_impl.cuh -- column-walk schedule of the 3D sweeps (one CTA per
 * (grid, source) pair; kept as the single-CTA path).
 *
 * Schedule.  A sweep in direction (sz,sx,sy) updates node (i,j,k) from its
 * seven upwind neighbours only, so any topological order of that dependency
 * graph gives the level-set result bit for bit.  Each lane owns one logical
 * x column and walks the (z, y) plane in z-fastest order, lane x running one
 * step behind lane x-1 (register carries, warp shuffles, a smem ring for the
 * previous y-row).
 */
#pragma once
#include "stencil3d.cuh"

namespace fk3 {

/* ------------------------------------------------------------------------ */
/* Schedule and data movement                                               */
/* ------------------------------------------------------------------------ */

constexpr int kD = 6;          /* prefetch distance, walk positions */
constexpr int kSlots = kD + 1; /* slot ring: the slot refilled is never the one just read */

__device__ __forceinline__ void named_barrier(int nthreads)
{
    asm volatile("bar.sync 1, %0;" ::"r"(nthreads) : "memory");
}

template <int BYTES>
__device__ __forceinline__ void cp_async(void *smem, const void *gmem)
{
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(sa), "l"(gmem), "n"(BYTES)
                 : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(kD - 1) : "memory"); }

__device__ __forceinline__ int ring_pitch(int nz) { return (nz + 1) & ~1; }

/* Shared header of one CTA; S sources walk together. */
template <typename R, int S>
struct Hdr {
    Mesh<R> mesh;
    Mesh<double> mesh64;
    R xres[2][S][kMaxWarps]; /* lane-31 hand-off: result, tn, slowness */
    R xtn[2][S][kMaxWarps];
    R xsl[2][2][kMaxWarps];
    double wmax[kMaxWarps];
};

template <typename R, int S>
__host__ __device__ inline size_t hdr_bytes() { return (sizeof(Hdr<R, S>) + 127) & ~size_t(127); }

template <typename R, int S>
__host__ __device__ inline size_t slot_bytes(int nthreads)
{
    return ((size_t)kSlots * (S + 2) * nthreads * sizeof(R) + 127) & ~size_t(127);
}

template <typename R, int S>
__host__ __device__ inline size_t smem_need(int nthreads, int nz)
{
    return hdr_bytes<R, S>() + slot_bytes<R, S>(nthreads) +
           (size_t)S * nthreads * ((nz + 1) & ~1) * sizeof(R);
}

/* Source set of a CTA. */
template <int S>
struct Srcs {
    Src q[S];
    int nv; /* valid sources (1..S) */
};

/* One sweep of S work items sharing a grid; returns this thread's FP64
 * max |dt| over its nodes and sources.
 *
 * Per step lane x needs, for walk position p (node (i', x', k')):
 *   own        r_last, te_last, tn_last, ten_last               (registers)
 *   lane x-1   r_last, tn_last and its two newest slowness cells (shuffle)
 *   ring       this lane's results of row k'-1                   (smem)
 *   slot       old time(s) and the two slowness cells of node p that are
 *              new to this lane, cp.async'd kD positions ahead     (smem)
 * The 8 cells around a node: x-upwind column = lane x-1's cells, z-upwind
 * layer = this lane's cells of the previous position. */
template <typename R, bool INIT, int S>
__device__ double sweep(Hdr<R, S> &sm, R *slots, R *rings, const Srcs<S> &src,
                        const fk_grid3d_t &g, R *const *tt, const R *__restrict__ slow,
                        int sweep_no, int nthreads)
{
    const int nz = g.nz, nx = g.nx, ny = g.ny, zp = g.zp, zcp = g.zcp;
    const int s0 = sweep_no - 1;
    const int sz = (s0 < 4) ? 1 : -1;
    const int sx = (s0 % 2 == 0) ? 1 : -1;
    const int sy = ((s0 / 2) % 2 == 0) ? 1 : -1;
    int loz = 1, lox = 1, loy = 1;
    if (INIT) { /* solver3D.F90:493-565 source-limited boxes (S == 1) */
        const Src &q = src.q[0];
        loz = (sz > 0) ? max(1, q.zsi - 1) : max(1, nz - q.zsi - 1);
        lox = (sx > 0) ? max(1, q.xsi - 1) : max(1, nx - q.xsi - 1);
        loy = (sy > 0) ? max(1, q.ysi - 1) : max(1, ny - q.ysi - 1);
    }
    const int ky0 = loy - 1;
    const long P = (long)(ny - ky0) * nz;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int xl = tid;
    const bool xin = xl < nx;
    const int ix = (sx > 0) ? xl : nx - 1 - xl;
    const int cxD = min(max((sx > 0) ? ix : ix - 1, 0), nx - 2);
    const int rp = ring_pitch(nz);
    const long nsteps = P + (long)nthreads - 1;
    const R HUGEV = (R)FK_HUGE;
    const unsigned FULL = 0xffffffffu;
    const int nv = src.nv;

    /* slot layout: [kSlots][S+2][nthreads] */
    auto slot = [&](int sl, int k) -> R * { return slots + ((size_t)sl * (S + 2) + k) * nthreads + tid; };

    /* physical position of walk position (il, kl) and its prefetch */
    auto issue = [&](int il_, int kl_, int sl) {
        const int iz = (sz > 0) ? il_ : nz - 1 - il_;
        const int iy = (sy > 0) ? kl_ : ny - 1 - kl_;
        const size_t idx = ((size_t)iy * nx + ix) * zp + iz;
#pragma unroll
        for (int k = 0; k < S; ++k)
            if (k < nv) cp_async<sizeof(R)>(slot(sl, k), tt[k] + idx);
        const int czD = min(max((sz > 0) ? iz : iz - 1, 0), nz - 2);
        const int cyU = min(max((sy > 0) ? iy - 1 : iy, 0), ny - 2);
        const int cyD = min(max((sy > 0) ? iy : iy - 1, 0), ny - 2);
        cp_async<sizeof(R)>(slot(sl, S), slow + ((size_t)cyU * (nx - 1) + cxD) * zcp + czD);
        cp_async<sizeof(R)>(slot(sl, S + 1), slow + ((size_t)cyD * (nx - 1) + cxD) * zcp + czD);
    };

    int il = 0, kl = ky0;                 /* walk position of the next node */
    int ilf = kD % nz, klf = ky0 + kD / nz; /* and of its prefetch */
    long pf = 0;
    if (xin) { /* prologue: positions 0 .. kD-1 */
        int a = 0, b = ky0;
        for (int d = 0; d < kD; ++d) {
            if (d < P) issue(a, b, d % kSlots);
            cp_commit();
            if (++a == nz) { a = 0; ++b; }
        }
    }

    R r_last[S], te_last[S], tn_last[S], ten_last[S];
#pragma unroll
    for (int k = 0; k < S; ++k) r_last[k] = te_last[k] = tn_last[k] = ten_last[k] = HUGEV;
    R dDU_last = 0, dDD_last = 0, uDU_last = 0, uDD_last = 0;
    double dmax = 0.0;

    for (long s = 0; s < nsteps; ++s) {
        R te[S], ten[S];
#pragma unroll
        for (int k = 0; k < S; ++k) {
            te[k] = __shfl_up_sync(FULL, r_last[k], 1);
            ten[k] = __shfl_up_sync(FULL, tn_last[k], 1);
        }
        R uDU = __shfl_up_sync(FULL, dDU_last, 1);
        R uDD = __shfl_up_sync(FULL, dDD_last, 1);
        if (lane == 0 && warp > 0) {
            const int b = (int)((s + 1) & 1);
#pragma unroll
            for (int k = 0; k < S; ++k) {
                te[k] = sm.xres[b][k][warp - 1];
                ten[k] = sm.xtn[b][k][warp - 1];
            }
            uDU = sm.xsl[b][0][warp - 1];
            uDD = sm.xsl[b][1][warp - 1];
        }
        const long p = s - xl;
        R result[S], tn[S];
#pragma unroll
        for (int k = 0; k < S; ++k) { result[k] = r_last[k]; tn[k] = tn_last[k]; }
        R dDU = dDU_last, dDD = dDD_last;
        if (xin && p >= 0 && p < P) {
            cp_wait();
            const int sl = (int)(p % kSlots);
            R told[S];
#pragma unroll
            for (int k = 0; k < S; ++k) told[k] = (k < nv) ? *slot(sl, k) : HUGEV;
            dDU = *slot(sl, S);
            dDD = *slot(sl, S + 1);
            if (pf + kD < P) issue(ilf, klf, (int)((p + kD) % kSlots));
            cp_commit();
            ++pf;
            if (++ilf == nz) { ilf = 0; ++klf; }
#pragma unroll
            for (int k = 0; k < S; ++k) {
                tn[k] = (kl > ky0) ? rings[((size_t)k * nthreads + xl) * rp + il] : HUGEV;
                result[k] = told[k];
            }
            if (il >= loz && xl >= lox && kl >= loy) {
                /* s<z><x><y>: U upwind, D other (clamped) */
                const R sUUU = uDU_last, sUUD = uDD_last, sDUU = uDU, sDUD = uDD;
                const R sUDU = dDU_last, sUDD = dDD_last, sDDU = dDU;
                const R s1 = rmin(rmin(sUUU, sUUD), rmin(sUDU, sUDD));
                const R s2 = rmin(rmin(sUUU, sUUD), rmin(sDUU, sDUD));
                const R s3 = rmin(rmin(sUUU, sUDU), rmin(sDUU, sDDU));
                const R s4 = rmin(sUUU, sUUD);
                const R s5 = rmin(sUUU, sUDU);
                const R s6 = rmin(sUUU, sDUU);
                const R s7 = sUUU;
                const int iz = (sz > 0) ? il : nz - 1 - il;
                const int iy = (sy > 0) ? kl : ny - 1 - kl;
                const size_t idx = ((size_t)iy * nx + ix) * zp + iz;
#pragma unroll
                for (int k = 0; k < S; ++k) {
                    if (k >= nv) break;
                    const R tv = r_last[k], tev = te_last[k], tnv = tn_last[k], tnve = ten_last[k];
                    R r;
                    if (!INIT) {
                        r = noinit(sm.mesh, tv, te[k], tn[k], tev, ten[k], tnv, tnve, s1, s2, s3,
                                   s4, s5, s6, s7, told[k]);
                    } else {
                        const Src &q = src.q[k];
                        const double tmin = (double)rmin(rmin(tv, te[k]), tn[k]);
                        const bool lcart = tmin > q.eps_t;
                        if (lcart || sizeof(R) == 8)
                            r = init_node<R>(q, sm.mesh, lcart, tv, te[k], tn[k], tev, ten[k], tnv,
                                             tnve, told[k], s1, s2, s3, s4, s5, s6, s7, iz + 1,
                                             ix + 1, iy + 1, sz, sx, sy);
                        else /* near-source spherical stencil in FP64 */
                            r = (R)init_node<double>(
                                q, sm.mesh64, lcart, (double)tv, (double)te[k], (double)tn[k],
                                (double)tev, (double)ten[k], (double)tnv, (double)tnve,
                                (double)told[k], (double)s1, (double)s2, (double)s3, (double)s4,
                                (double)s5, (double)s6, (double)s7, iz + 1, ix + 1, iy + 1, sz, sx,
                                sy);
                    }
                    if (r != told[k]) {
                        tt[k][idx] = r;
                        const double d = fabs((double)r - (double)told[k]);
                        dmax = d > dmax ? d : dmax;
                    }
                    result[k] = r;
                }
            }
#pragma unroll
            for (int k = 0; k < S; ++k) rings[((size_t)k * nthreads + xl) * rp + il] = result[k];
            if (++il == nz) { il = 0; ++kl; }
        }
#pragma unroll
        for (int k = 0; k < S; ++k) {
            te_last[k] = te[k];
            ten_last[k] = ten[k];
            r_last[k] = result[k];
            tn_last[k] = tn[k];
        }
        uDU_last = uDU; uDD_last = uDD;
        dDU_last = dDU; dDD_last = dDD;
        if (lane == 31) {
            const int b = (int)(s & 1);
#pragma unroll
            for (int k = 0; k < S; ++k) {
                sm.xres[b][k][warp] = result[k];
                sm.xtn[b][k][warp] = tn[k];
            }
            sm.xsl[b][0][warp] = dDU;
            sm.xsl[b][1][warp] = dDD;
        }
        named_barrier(nthreads);
    }
    return dmax;
}

template <typename R, int S>
__device__ __forceinline__ double block_max(Hdr<R, S> &sm, double v, int nthreads)
{
    for (int o = 16; o > 0; o >>= 1) {
        double w = __shfl_xor_sync(0xffffffffu, v, o);
        v = w > v ? w : v;
    }
    const int warp = threadIdx.x >> 5, nw = nthreads >> 5;
    if ((threadIdx.x & 31) == 0) sm.wmax[warp] = v;
    named_barrier(nthreads);
    double m = 0.0;
    for (int w = 0; w < nw; ++w) m = sm.wmax[w] > m ? sm.wmax[w] : m;
    named_barrier(nthreads);
    return m;
}

__device__ __forceinline__ void setup_src(Src &q, const fk_work3d_t &w, const fk_grid3d_t &g,
                                          double eps)
{
    q.zsi = w.zsi; q.xsi = w.xsi; q.ysi = w.ysi;
    q.zsa = w.zsa; q.xsa = w.xsa; q.ysa = w.ysa;
    q.szero = w.szero; q.szero2 = w.szero * w.szero;
    double hmin = g.dz < g.dx ? g.dz : g.dx;
    hmin = g.dy < hmin ? g.dy : hmin;
    q.eps_t = eps * hmin * w.szero; /* localSolver.F90:906 */
}

template <typename R, int S>
__device__ void init_hdr(Hdr<R, S> &sm, const fk_grid3d_t &g)
{
    if (threadIdx.x == 0) {
        make_mesh<R>(sm.mesh, g.dz, g.dx, g.dy);
        make_mesh<double>(sm.mesh64, g.dz, g.dx, g.dy);
    }
    const int nthreads = ((g.nx + 31) / 32) * 32; /* the threads still running */
    for (int t = threadIdx.x; t < 2 * S * kMaxWarps; t += nthreads) {
        (&sm.xres[0][0][0])[t] = (R)FK_HUGE;
        (&sm.xtn[0][0][0])[t] = (R)FK_HUGE;
    }
    for (int t = threadIdx.x; t < 4 * kMaxWarps; t += nthreads) (&sm.xsl[0][0][0])[t] = (R)0;
}

/* Field initialisation + the 8 initialisation sweeps, one work item per CTA
 * (solver3D.F90:1201-1211). */
template <typename R, int MAXT>
__global__ void __launch_bounds__(MAXT, 1)
init_kernel(const fk_grid3d_t *__restrict__ grids, const fk_work3d_t *__restrict__ work,
            double eps)
{
    extern __shared__ __align__(128) unsigned char smem_raw[];
    Hdr<R, 1> &sm = *reinterpret_cast<Hdr<R, 1> *>(smem_raw);
    const fk_work3d_t w = work[blockIdx.x];
    const fk_grid3d_t g = grids[w.grid];
    const int nthreads = ((g.nx + 31) / 32) * 32;
    if ((int)threadIdx.x >= nthreads) return;
    R *slots = reinterpret_cast<R *>(smem_raw + hdr_bytes<R, 1>());
    R *rings = reinterpret_cast<R *>(smem_raw + hdr_bytes<R, 1>() + slot_bytes<R, 1>(nthreads));
    R *tt = reinterpret_cast<R *>(w.tt);
    Srcs<1> src;
    setup_src(src.q[0], w, g, eps);
    src.nv = 1;
    init_hdr(sm, g);
    const size_t nfield = (size_t)g.ny * g.nx * g.zp;
    for (size_t e = threadIdx.x; e < nfield; e += nthreads) tt[e] = (R)FK_HUGE;
    named_barrier(nthreads);
    if (threadIdx.x < 8) { /* localSolver.F90:933-956, FP64 */
        const Src &q = src.q[0];
        const int di = threadIdx.x & 1, dj = (threadIdx.x >> 1) & 1, dk = (threadIdx.x >> 2) & 1;
        const double t = tana<double>(q, sm.mesh64, q.zsi + di, q.xsi + dj, q.ysi + dk);
        tt[((size_t)(q.ysi - 1 + dk) * g.nx + (q.xsi - 1 + dj)) * g.zp + (q.zsi - 1 + di)] = (R)t;
    }
    __threadfence_block();
    named_barrier(nthreads);
    R *ttp[1] = {tt};
    for (int s = 1; s <= 8; ++s)
        sweep<R, true, 1>(sm, slots, rings, src, g, ttp, reinterpret_cast<const R *>(g.slow), s,
                          nthreads);
}

/* Gauss-Seidel passes: S work items of one grid per CTA
 * (solver3D.F90:1213-1222; with conv_tol >= 0 and max_pass > 0 the passes
 * repeat until no node moves by more than conv_tol). */
template <typename R, int S, int MAXT>
__global__ void __launch_bounds__(MAXT, 1)
pass_kernel(const fk_grid3d_t *__restrict__ grids, const fk_work3d_t *__restrict__ work,
            const int *__restrict__ groups, fk_result3d_t *__restrict__ results, double eps,
            int nsweep, double conv_tol, int max_pass)
{
    extern __shared__ __align__(128) unsigned char smem_raw[];
    Hdr<R, S> &sm = *reinterpret_cast<Hdr<R, S> *>(smem_raw);
    int wi[S];
    int nv = 0;
#pragma unroll
    for (int k = 0; k < S; ++k) {
        wi[k] = groups[blockIdx.x * S + k];
        if (wi[k] >= 0) nv = k + 1;
    }
    const fk_grid3d_t g = grids[work[wi[0]].grid];
    const int nthreads = ((g.nx + 31) / 32) * 32;
    if ((int)threadIdx.x >= nthreads) return;
    R *slots = reinterpret_cast<R *>(smem_raw + hdr_bytes<R, S>());
    R *rings = reinterpret_cast<R *>(smem_raw + hdr_bytes<R, S>() + slot_bytes<R, S>(nthreads));
    Srcs<S> src;
    src.nv = nv;
    R *ttp[S];
#pragma unroll
    for (int k = 0; k < S; ++k) {
        const fk_work3d_t w = work[wi[k] >= 0 ? wi[k] : wi[0]];
        setup_src(src.q[k], w, g, eps);
        ttp[k] = reinterpret_cast<R *>(w.tt);
    }
    init_hdr(sm, g);
    named_barrier(nthreads);
    const bool converge = conv_tol >= 0.0 && max_pass > 0;
    const int npasses = converge ? max_pass : nsweep;
    double res = 0.0;
    int ran = 0;
    for (int it = 0; it < npasses; ++it) {
        double d = 0.0;
        for (int s = 1; s <= 8; ++s) {
            const double ds = sweep<R, false, S>(sm, slots, rings, src, g, ttp,
                                                 reinterpret_cast<const R *>(g.slow), s, nthreads);
            d = ds > d ? ds : d;
        }
        res = block_max(sm, d, nthreads);
        ++ran;
        if (converge && res <= conv_tol) break;
    }
    if (threadIdx.x < nv) {
        results[wi[threadIdx.x]].residual = res;
        results[wi[threadIdx.x]].npass = ran;
        results[wi[threadIdx.x]].status = 0;
    }
}

template <typename R>
inline int pick_s(int max_nx, int max_nz, int nwork, int nsm)
{
    const int nthreads = ((max_nx + 31) / 32) * 32;
    if (smem_need<R, 2>(nthreads, max_nz) <= 227 * 1024 && nwork >= nsm) return 2;
    return 1;
}

template <typename R, int S>
inline auto pass_fn(int nthreads)
{
    return (nthreads <= 256) ? pass_kernel<R, S, 256> : pass_kernel<R, S, 1024>;
}

template <typename R>
inline auto init_fn(int nthreads)
{
    return (nthreads <= 256) ? init_kernel<R, 256> : init_kernel<R, 1024>;
}

template <typename R>
inline int prepare_solve(int max_nx, int max_nz, int S)
{
    const int nthreads = ((max_nx + 31) / 32) * 32;
    cudaError_t e = cudaFuncSetAttribute(init_fn<R>(nthreads), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem_need<R, 1>(nthreads, max_nz));
    if (e != cudaSuccess) return (int)e;
    if (S == 2)
        e = cudaFuncSetAttribute(pass_fn<R, 2>(nthreads), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem_need<R, 2>(nthreads, max_nz));
    else
        e = cudaFuncSetAttribute(pass_fn<R, 1>(nthreads), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem_need<R, 1>(nthreads, max_nz));
    return (int)e;
}

/* groups: device [ngroups][S] work indices (-1 = empty slot). */
template <typename R>
inline int launch_solve(const fk_grid3d_t *grids, const fk_work3d_t *work, const int *groups,
                        int ngroups, int S, fk_result3d_t *results, int nwork, int max_nx,
                        int max_nz, double eps, int nsweep, double conv_tol, int max_pass,
                        cudaStream_t stream)
{
    if (nwork <= 0) return 0;
    if (max_nx > kMaxWarps * 32) return (int)cudaErrorInvalidValue;
    const int nthreads = ((max_nx + 31) / 32) * 32;
    if (smem_need<R, 1>(nthreads, max_nz) > 227 * 1024) return (int)cudaErrorInvalidValue;
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    cudaError_t e = cudaStreamIsCapturing(stream, &cap);
    if (e != cudaSuccess) return (int)e;
    if (cap == cudaStreamCaptureStatusNone) { /* under capture prepare_solve ran already */
        int pe = prepare_solve<R>(max_nx, max_nz, S);
        if (pe) return pe;
    }
    init_fn<R>(nthreads)<<<nwork, nthreads, smem_need<R, 1>(nthreads, max_nz), stream>>>(grids, work, eps);
    if (S == 2)
        pass_fn<R, 2>(nthreads)<<<ngroups, nthreads, smem_need<R, 2>(nthreads, max_nz), stream>>>(
            grids, work, groups, results, eps, nsweep, conv_tol, max_pass);
    else
        pass_fn<R, 1>(nthreads)<<<ngroups, nthreads, smem_need<R, 1>(nthreads, max_nz), stream>>>(
            grids, work, groups, results, eps, nsweep, conv_tol, max_pass);
    return (int)cudaGetLastError();
}

} // namespace fk3
