/*
 * sweep2d.cu -- the reference's 2D level-set solve (solver2D.F90:782-978,
 * node updates localSolver.F90:123-289) and its natural-order twin
 * solveSourceFSM (solver2D.F90:1042-1280), in FP64.
 *
 * One CTA owns one (grid, source).  Thread t owns the logical x columns
 * b NT + t (b = 0, 1, ...: column blocks of NT <= 512 threads) and walks
 * their z positions, block after block, thread t one step behind thread t-1,
 * so tv is the thread's previous result, te the previous result of thread
 * t-1 (warp shuffle, the two-slot hand-off between warps, or for thread 0 of
 * block b > 0 the last thread's result of block b-1 through a ring indexed
 * by z, Zb >= NT steps old) and tev the thread's previous te.  Both reference
 * schedules are topological orders of the same dependency graph, so LSM and
 * FSM give identical fields here (the FSM's initialisation box clamp is
 * applied to both).  Compiled without multiply-add contraction.
 */
#include <cuda_runtime.h>
#include "fteik_dev.h"

namespace {

constexpr int kMaxWarps = 16;
constexpr int kMaxThreads = kMaxWarps * 32;   /* 512: 128 registers per thread, no spills */

struct Mesh2 {
    double dz, dx, dzi, dxi, dz2i, dx2i, dz2i_dx2i, dz2i_p_dx2i, dz2i_p_dx2i_inv;
};

struct Src2 {
    int zsi, xsi;
    double zsa, xsa, szero, eps;
};

__device__ __forceinline__ double dmin(double a, double b) { return (b < a) ? b : a; }

/* localSolver.F90:36-50 */
__device__ __forceinline__ double tana2(const Src2 &q, const Mesh2 &c, int i, int j)
{
    double dz_ = ((double)i - q.zsa) * c.dz;
    double dx_ = ((double)j - q.xsa) * c.dx;
    return q.szero * hypot(dx_, dz_);
}

/* localSolver.F90:123-158 */
__device__ __forceinline__ double noinit2(const Mesh2 &c, double tv, double te,
                                          double tev, double s1, double s2, double s3)
{
    double temtv = te - tv;
    double t12min = dmin(tv + c.dz * s1, te + c.dx * s2);
    double t1_2d = FK_HUGE;
    if (temtv < c.dz * s3 && -temtv < c.dx * s3) {
        double ta = tev + temtv, tb = tev - temtv, tab = ta - tb;
        t1_2d = ((tb * c.dz2i + ta * c.dx2i) +
                 sqrt((4.0 * (s3 * s3)) * c.dz2i_p_dx2i - c.dz2i_dx2i * (tab * tab))) *
                c.dz2i_p_dx2i_inv;
    }
    return dmin(t12min, t1_2d);
}

/* localSolver.F90:195-289, node (iz, ix) 1-based. */
__device__ double init2(const Src2 &q, const Mesh2 &c, int sz, int sx, double tv,
                        double te, double tev, double t, double sref1, double sref2,
                        double sref3, int iz, int ix)
{
    const double sgnrz = (double)sz, sgnrx = (double)sx;
    double t1d = dmin(tv + c.dz * sref1, te + c.dx * sref2);
    double t1 = FK_HUGE, t2 = FK_HUGE, t3 = FK_HUGE;
    if (abs(iz - q.zsi) > q.eps || abs(ix - q.xsi) > q.eps) {
        if (tv <= te + c.dx * sref3 && te <= tv + c.dz * sref3 && te >= tev && tv >= tev) {
            double ta = tev + te - tv, tb = tev - te + tv;
            t1 = ((tb * c.dz2i + ta * c.dx2i) +
                  sqrt(4.0 * sref3 * sref3 * (c.dz2i + c.dx2i) -
                       c.dz2i * c.dx2i * (ta - tb) * (ta - tb))) /
                 (c.dz2i + c.dx2i);
        } else if ((te - tev) <= c.dz * c.dz * sref3 / sqrt(c.dx * c.dx + c.dz * c.dz) &&
                   te > tev) {
            double r = (te - tev) / c.dz;
            t2 = te + c.dx * sqrt(sref3 * sref3 - r * r);
        } else if ((tv - tev) <= c.dx * c.dx * sref3 / sqrt(c.dx * c.dx + c.dz * c.dz) &&
                   tv > tev) {
            double r = (tv - tev) / c.dx;
            t3 = tv + c.dz * sqrt(sref3 * sref3 - r * r);
        }
    } else {
        /* tAnaD (localSolver.F90:74-112) and the perturbations, used only by
         * the spherical operator near the source */
        double dz_ = ((double)iz - q.zsa) * c.dz, dx_ = ((double)ix - q.xsa) * c.dx;
        double d0 = dz_ * dz_ + dx_ * dx_;
        double t0c = 0.0, d0i_szero = 0.0;
        if (d0 > 0.0) {
            double sq = sqrt(d0);
            t0c = q.szero * sq;
            d0i_szero = q.szero / sq;
        }
        double tzc = d0i_szero * dz_, txc = d0i_szero * dx_;
        double tauv = tv - tana2(q, c, iz - sz, ix);
        double taue = te - tana2(q, c, iz, ix - sx);
        double tauev = tev - tana2(q, c, iz - sz, ix - sx);
        if (tv < te + c.dx * sref3 && te < tv + c.dz * sref3 && te >= tev && tv >= tev) {
            double ta = tauev + taue - tauv, tb = tauev - taue + tauv;
            double apoly = c.dz2i + c.dx2i;
            double bpoly = 4.0 * (sgnrx * txc * c.dxi + sgnrz * tzc * c.dzi) -
                           2.0 * (ta * c.dx2i + tb * c.dz2i);
            double cpoly = (ta * ta * c.dx2i) + (tb * tb * c.dz2i) -
                           4.0 * (sgnrx * txc * c.dxi * ta + sgnrz * tzc * c.dzi * tb) +
                           4.0 * (q.szero * q.szero - sref3 * sref3);
            double dpoly = bpoly * bpoly - 4.0 * apoly * cpoly;
            if (dpoly >= 0.0) t1 = 0.5 * (sqrt(dpoly) - bpoly) / apoly + t0c;
            if (t1 < tv || t1 < te) t1 = FK_HUGE;
        }
    }
    double t2d = dmin(dmin(t1, t2), t3);
    return dmin(dmin(t, t1d), t2d);
}

__device__ __forceinline__ void bar(int n)
{
    asm volatile("bar.sync 1, %0;" ::"r"(n) : "memory");
}

struct Smem2 {
    Mesh2 mesh;
    double xres[2][kMaxWarps];
    double wmax[kMaxWarps];
};

template <bool INIT>
__device__ double sweep2(Smem2 &sm, double *ring, const Src2 &q, const fk_grid2d_t &g,
                         double *__restrict__ tt, const double *__restrict__ slow,
                         int sweep, int nthreads)
{
    const int nz = g.nz, nx = g.nx, zp = g.zp, zcp = g.zcp;
    const int sz = (sweep <= 2) ? 1 : -1;            /* localSolver.F90:160-193 */
    const int sx = (sweep == 1 || sweep == 3) ? 1 : -1;
    int loz = 1, lox = 1;
    if (INIT) {
        loz = (sz > 0) ? max(1, q.zsi - 1) : max(1, nz - q.zsi - 1);
        lox = (sx > 0) ? max(1, q.xsi - 1) : max(1, nx - q.xsi - 1);
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int t = threadIdx.x;
    const int nblk = (nx + nthreads - 1) / nthreads;   /* column blocks */
    /* steps per block: the ring between blocks needs >= nthreads; one block needs no ring */
    const int zb = (nblk > 1 && nthreads > nz) ? nthreads : nz;
    const int nsteps = nblk * zb + nthreads - 1;
    /* The node and slowness loads of a thread's next item are issued one
     * step ahead: within a sweep only this thread writes its columns. */
    struct Item {
        double told, sUU, sUD, sDU;
        size_t idx;
        int iz, ix, b, il;
        bool valid, upd;
    };
    auto fetch = [&](int j, Item &f) {
        f.b = j >= 0 ? j / zb : -1;
        f.il = j - f.b * zb;
        const int xl = f.b * nthreads + t;
        f.valid = j >= 0 && f.b < nblk && xl < nx && f.il < nz;
        f.upd = f.valid && f.il >= loz && xl >= lox;
        if (!f.valid) return;
        f.ix = (sx > 0) ? xl : nx - 1 - xl;
        f.iz = (sz > 0) ? f.il : nz - 1 - f.il;
        f.idx = (size_t)f.ix * zp + f.iz;
        f.told = tt[f.idx];
        if (f.upd) {
            const int cxU = (sx > 0) ? f.ix - 1 : f.ix;
            const int cxD = min(max((sx > 0) ? f.ix : f.ix - 1, 0), nx - 2);
            const int czU = (sz > 0) ? f.iz - 1 : f.iz;
            const int czD = min(max((sz > 0) ? f.iz : f.iz - 1, 0), nz - 2);
            f.sUU = slow[(size_t)cxU * zcp + czU];
            f.sUD = slow[(size_t)cxD * zcp + czU]; /* z U, x D */
            f.sDU = slow[(size_t)cxU * zcp + czD]; /* z D, x U */
        }
    };
    Item nxt;
    fetch(-t, nxt);
    double r_last = FK_HUGE, te_last = FK_HUGE, dmax = 0.0;
    for (int s = 0; s < nsteps; ++s) {
        const Item cur = nxt;
        fetch(s + 1 - t, nxt);
        double te = __shfl_up_sync(0xffffffffu, r_last, 1);
        if (lane == 0 && warp > 0) te = sm.xres[(s + 1) & 1][warp - 1];
        if (t == 0) te = (cur.b > 0 && cur.il < nz) ? ring[cur.il] : FK_HUGE;
        double result = r_last;
        if (cur.valid) {
            const double told = cur.told;
            result = told;
            if (cur.upd) {
                const double s1 = dmin(cur.sUU, cur.sUD), s2 = dmin(cur.sUU, cur.sDU), s3 = cur.sUU;
                double tu;
                if (INIT)
                    tu = init2(q, sm.mesh, sz, sx, r_last, te, te_last, told, s1, s2, s3,
                               cur.iz + 1, cur.ix + 1);
                else
                    tu = noinit2(sm.mesh, r_last, te, te_last, s1, s2, s3);
                result = dmin(told, tu);
                if (result != told) {
                    tt[cur.idx] = result;
                    double d = fabs(result - told);
                    dmax = d > dmax ? d : dmax;
                }
            }
        }
        te_last = te;
        r_last = result;
        if (lane == 31) sm.xres[s & 1][warp] = result;
        if (t == nthreads - 1 && cur.b >= 0 && cur.b < nblk && cur.il < nz) ring[cur.il] = result;
        bar(nthreads);
    }
    return dmax;
}

__global__ void __launch_bounds__(kMaxThreads, 1)
solve2d_kernel(const fk_grid2d_t *__restrict__ grids, const fk_work2d_t *__restrict__ work,
               fk_result3d_t *__restrict__ results, double eps, int nsweep,
               double conv_tol, int max_pass)
{
    __shared__ Smem2 sm;
    extern __shared__ double ring2[];                 /* [nz]: last thread -> thread 0 of the next block */
    const fk_work2d_t w = work[blockIdx.x];
    const fk_grid2d_t g = grids[w.grid];
    const int nthreads = min(((g.nx + 31) / 32) * 32, (int)blockDim.x);
    if ((int)threadIdx.x >= nthreads) return;
    Src2 q;
    q.zsi = w.zsi; q.xsi = w.xsi; q.zsa = w.zsa; q.xsa = w.xsa; q.szero = w.szero;
    q.eps = eps; /* grid points, localSolver.F90:327 */
    if (threadIdx.x == 0) {
        Mesh2 &m = sm.mesh;
        m.dz = g.dz; m.dx = g.dx;
        m.dzi = 1.0 / g.dz; m.dxi = 1.0 / g.dx;
        m.dz2i = 1.0 / (g.dz * g.dz); m.dx2i = 1.0 / (g.dx * g.dx);
        m.dz2i_dx2i = m.dz2i * m.dx2i;
        m.dz2i_p_dx2i = m.dz2i + m.dx2i;
        m.dz2i_p_dx2i_inv = 1.0 / (m.dz2i + m.dx2i);
    }
    if (threadIdx.x < 2 * kMaxWarps) sm.xres[threadIdx.x / kMaxWarps][threadIdx.x % kMaxWarps] = FK_HUGE;
    double *tt = w.tt;
    const size_t nfield = (size_t)g.nx * g.zp;
    for (size_t e = threadIdx.x; e < nfield; e += nthreads) tt[e] = FK_HUGE;
    bar(nthreads);
    if (threadIdx.x < 4) { /* localSolver.F90:342-349 */
        const int di = threadIdx.x & 1, dj = threadIdx.x >> 1;
        tt[(size_t)(q.xsi - 1 + dj) * g.zp + (q.zsi - 1 + di)] =
            tana2(q, sm.mesh, q.zsi + di, q.xsi + dj);
    }
    __threadfence_block();
    bar(nthreads);
    for (int s = 1; s <= 4; ++s) sweep2<true>(sm, ring2, q, g, tt, g.slow, s, nthreads);
    const bool converge = conv_tol >= 0.0 && max_pass > 0;
    const int npasses = converge ? max_pass : nsweep;
    double res = 0.0;
    int ran = 0;
    for (int it = 0; it < npasses; ++it) {
        double d = 0.0;
        for (int s = 1; s <= 4; ++s) {
            double ds = sweep2<false>(sm, ring2, q, g, tt, g.slow, s, nthreads);
            d = ds > d ? ds : d;
        }
        for (int o = 16; o > 0; o >>= 1) {
            double v = __shfl_xor_sync(0xffffffffu, d, o);
            d = v > d ? v : d;
        }
        if ((threadIdx.x & 31) == 0) sm.wmax[threadIdx.x >> 5] = d;
        bar(nthreads);
        res = 0.0;
        for (int ww = 0; ww < (nthreads >> 5); ++ww) res = sm.wmax[ww] > res ? sm.wmax[ww] : res;
        bar(nthreads);
        ++ran;
        if (converge && res <= conv_tol) break;
    }
    if (threadIdx.x == 0) {
        results[blockIdx.x].residual = res;
        results[blockIdx.x].npass = ran;
        results[blockIdx.x].status = 0;
    }
}

} // namespace

extern "C" int fk2d_solve(int fsm, const fk_grid2d_t *grids, const fk_work2d_t *work,
                          fk_result3d_t *results, int nwork, int max_nx, int max_nz, double eps,
                          int nsweep, double conv_tol, int max_pass, cudaStream_t stream)
{
    (void)fsm; /* same dependency graph, same result: see the file comment */
    if (nwork <= 0) return 0;
    const int nthreads = min(((max_nx + 31) / 32) * 32, kMaxThreads);
    const size_t smem = sizeof(double) * (size_t)(max_nz > 1 ? max_nz : 1);
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(solve2d_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return (int)e;
    }
    solve2d_kernel<<<nwork, nthreads, smem, stream>>>(grids, work, results, eps, nsweep,
                                                      conv_tol, max_pass);
    return (int)cudaGetLastError();
}
