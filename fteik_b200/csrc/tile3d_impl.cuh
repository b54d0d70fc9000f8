/*
 * tile3d_impl.cuh -- tile-wavefront schedule of the 3D sweeps (the batched
 * and single-source product path).
 *
 * The (x, y) plane of every (grid, source) work item is cut into fixed
 * physical tiles of TX x TY columns; a tile task is one sweep over one tile,
 * every column walked over its whole z extent.  Inside a task thread
 * (lane tx, warp ty) owns one column and walks z with a skew of ox + oy
 * steps (ox, oy = its offsets from the tile's upwind corner in the sweep's
 * direction), so the seven upwind neighbours of a node come from:
 *   tv, tev, tnv, tnve   this thread's previous step            (registers)
 *   te, ten              the x-upwind lane's previous step      (shuffle)
 *   tn, ten              the y-upwind warp's previous step      (shared memory)
 *   tile faces           the neighbour tiles' final values      (global, L2)
 * A sweep over a tile reads only upwind nodes, so the result equals the
 * reference's level-set sweep (autoCode.f90) bit for bit in FP64.
 *
 * Tasks are ordered sweep-major, and within a sweep by tile level
 * bx' + by' in that sweep's logical coordinates; CTAs claim them through one
 * atomic ticket.  A task waits only on tasks with smaller tickets:
 *   - its own tile and its eight neighbours done with the previous sweep
 *     (the neighbours may still be reading this tile's faces),
 *   - its two upwind face neighbours done with this sweep.
 * Every waited-on task is already claimed by a running CTA that itself waits
 * only on earlier tickets, so the waits cannot cycle.  Every wait is bounded:
 * past the limit the CTA sets the error word and stops; the host reports it.
 */
#pragma once
#include "stencil3d.cuh"

namespace fk3tw {
using fk3::Mesh;
using fk3::Src;
using fk3::rmin;
using fk3::rmax;

constexpr int TX = 32;
constexpr int TY = 8;
constexpr int NT = TX * TY;

struct Params {
    const fk_grid3d_t *grids;
    const fk_work3d_t *work;
    const int2 *tasks;          /* one sweep's tasks: {work, by' * ntx + bx'} in level order */
    const int *done_base;       /* per work item: first tile's index in done[] */
    int ntask_sweep;
    int s_begin, s_end;         /* global sweep numbers: 0..7 init, 8.. Gauss-Seidel */
    int *done;                  /* per tile: sweeps completed */
    unsigned long long *ticket;
    int *error;                 /* 0 ok; else the first failure */
    unsigned long long *resid;  /* [nwork][npass]: FP64 max |dt| bits */
    int *pass_tiles;            /* [nwork][npass]: tiles done with the pass's last sweep */
    int *conv_pass;             /* [nwork]: first converged pass, or a large value */
    int npass;
    int converge;
    double eps, conv_tol;
    long long spin_limit;
};

__device__ __forceinline__ int ld_acquire(const int *p)
{
    int v;
    asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_release(int *p, int v)
{
    asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

template <typename R>
__device__ __forceinline__ R ldcg(const R *p) { return __ldcg(p); }

__device__ __forceinline__ void tw_setup_src(Src &q, const fk_work3d_t &w, const fk_grid3d_t &g,
                                          double eps)
{
    q.zsi = w.zsi; q.xsi = w.xsi; q.ysi = w.ysi;
    q.zsa = w.zsa; q.xsa = w.xsa; q.ysa = w.ysa;
    q.szero = w.szero; q.szero2 = w.szero * w.szero;
    double hmin = g.dz < g.dx ? g.dz : g.dx;
    hmin = g.dy < hmin ? g.dy : hmin;
    q.eps_t = eps * hmin * w.szero; /* localSolver.F90:906 */
}

/* Sweep one tile.  Returns this thread's FP64 max |dt|. */
template <typename R, bool INIT>
__device__ double tile_sweep(const fk_grid3d_t &g, R *__restrict__ tt, const R *__restrict__ slow,
                             const Src &q, const Mesh<R> &mesh, const Mesh<double> &mesh64,
                             int sweep_no, int bx, int by, R (*xr)[TY][TX], R (*xte)[TY][TX])
{
    const int nz = g.nz, nx = g.nx, ny = g.ny, zp = g.zp, zcp = g.zcp;
    const int s0 = sweep_no - 1;
    const int sz = (s0 < 4) ? 1 : -1;
    const int sx = (s0 % 2 == 0) ? 1 : -1;
    const int sy = ((s0 / 2) % 2 == 0) ? 1 : -1;
    int loz = 1, lox = 1, loy = 1;
    if (INIT) { /* solver3D.F90:493-565, flipped bound clamped to the grid */
        loz = (sz > 0) ? max(1, q.zsi - 1) : max(1, nz - q.zsi - 1);
        lox = (sx > 0) ? max(1, q.xsi - 1) : max(1, nx - q.xsi - 1);
        loy = (sy > 0) ? max(1, q.ysi - 1) : max(1, ny - q.ysi - 1);
    }
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    const int tw = min(TX, nx - bx * TX), th = min(TY, ny - by * TY);
    const int x = bx * TX + tx, y = by * TY + ty;
    const bool col = tx < tw && ty < th;
    const int ox = (sx > 0) ? tx : tw - 1 - tx;
    const int oy = (sy > 0) ? ty : th - 1 - ty;
    const int xlog = (sx > 0) ? x : nx - 1 - x; /* logical x, y */
    const int ylog = (sy > 0) ? y : ny - 1 - y;
    const bool colupd = col && xlog >= lox && ylog >= loy;
    const int srcx = tx - sx;                    /* x-upwind lane */
    const int wy = ty - sy;                      /* y-upwind warp */
    /* column offsets (32-bit: a field and a slowness grid hold < 2^31 entries) */
    const int cbase = (y * nx + x) * zp;
    const int cbase_x = (y * nx + (x - sx)) * zp;        /* used when the neighbour exists */
    const int cbase_y = ((y - sy) * nx + x) * zp;
    const int cbase_xy = ((y - sy) * nx + (x - sx)) * zp;
    /* slowness columns: U upwind cell, D other (clamped) */
    const int cxU = (sx > 0) ? x - 1 : x, cxD = min(max((sx > 0) ? x : x - 1, 0), nx - 2);
    const int cyU = (sy > 0) ? y - 1 : y, cyD = min(max((sy > 0) ? y : y - 1, 0), ny - 2);
    const int sUU = (cyU * (nx - 1) + cxU) * zcp; /* x U, y U */
    const int sUD = (cyD * (nx - 1) + cxU) * zcp; /* x U, y D */
    const int sDU = (cyU * (nx - 1) + cxD) * zcp; /* x D, y U */
    const int sDD = (cyD * (nx - 1) + cxD) * zcp; /* x D, y D */
    const R HUGEV = (R)FK_HUGE;
    const unsigned FULL = 0xffffffffu;
    const int zoff = (sz > 0) ? 0 : zp - nz; /* padded walk: dummy positions */
    /* walk only positions a node of this sweep can need: from the z-upwind
     * neighbour of the first updated level to the last real level */
    const int qs = zoff + loz - 1, qe = zoff + nz - 1;
    const int nsteps = (qe - qs + 1) + (TX - 1) + (TY - 1);
    const bool edge_x = ox == 0, edge_y = oy == 0;
    const bool has_x = xlog >= 1, has_y = ylog >= 1;

    /* Global operands of a walk position, loaded one step ahead: the old
     * time, the tile-face values and the 4 slowness cells of the z-downwind
     * layer (the z-upwind layer is the previous position's). */
    struct Pre {
        R told, te, tn, ten;
        R duu, dud, ddu, ddd; /* slowness s<z><x><y>, z = D */
    };
    auto fetch = [&](int qpos, Pre &f) {
        if (!(col && qpos >= qs && qpos <= qe)) return;
        const int iz = (sz > 0) ? qpos : zp - 1 - qpos;
        f.told = ldcg(tt + (cbase + iz));
        if (edge_x) f.te = has_x ? ldcg(tt + (cbase_x + iz)) : HUGEV;
        if (edge_y) f.tn = has_y ? ldcg(tt + (cbase_y + iz)) : HUGEV;
        if (edge_x && edge_y) f.ten = (has_x && has_y) ? ldcg(tt + (cbase_xy + iz)) : HUGEV;
        if (colupd) {
            const int czD = min(max((sz > 0) ? iz : iz - 1, 0), nz - 2);
            f.duu = __ldg(slow + (sUU + czD));
            f.dud = __ldg(slow + (sUD + czD));
            f.ddu = __ldg(slow + (sDU + czD));
            f.ddd = __ldg(slow + (sDD + czD));
        }
    };
    Pre cur, nxt;
    fetch(qs - ox - oy, nxt);
    R zu_uu = 0, zu_ud = 0, zu_du = 0, zu_dd = 0; /* z-upwind layer (previous position) */

    R r_last = HUGEV, te_last = HUGEV, tn_last = HUGEV, ten_last = HUGEV;
    double dmax = 0.0;
    for (int st = 0; st < nsteps; ++st) {
        const int pp = (st + 1) & 1, cp = st & 1;
        const R sh_r = __shfl_sync(FULL, r_last, srcx & 31);
        const R sh_tn = __shfl_sync(FULL, tn_last, srcx & 31);
        const int qpos = qs + st - ox - oy;
        cur = nxt;
        fetch(qpos + 1, nxt);
        R te = HUGEV, tn = HUGEV, ten = HUGEV, result = r_last;
        const int iz = (sz > 0) ? qpos : zp - 1 - qpos;
        if (col && qpos >= qs && qpos <= qe) {
            const int il = qpos - zoff; /* logical unpadded z */
            const R told = cur.told;
            result = told;
            /* every real node gathers its upwind values: downstream lanes
             * and warps take them over even where this node is not updated */
            te = edge_x ? cur.te : sh_r;
            tn = edge_y ? cur.tn : xr[pp][wy][tx];
            ten = !edge_y ? xte[pp][wy][tx] : (!edge_x ? sh_tn : cur.ten);
            if (colupd && il >= loz) {
                const R uuu = zu_uu, uud = zu_ud, udu = zu_du, udd = zu_dd;
                const R s1 = rmin(rmin(uuu, uud), rmin(udu, udd));
                const R s2 = rmin(rmin(uuu, uud), rmin(cur.duu, cur.dud));
                const R s3 = rmin(rmin(uuu, udu), rmin(cur.duu, cur.ddu));
                const R s4 = rmin(uuu, uud);
                const R s5 = rmin(uuu, udu);
                const R s6 = rmin(uuu, cur.duu);
                const R s7 = uuu;
                const R tv = r_last, tev = te_last, tnv = tn_last, tnve = ten_last;
                R r;
                if (!INIT) {
                    r = fk3::noinit(mesh, tv, te, tn, tev, ten, tnv, tnve, s1, s2, s3, s4, s5, s6, s7,
                                    told);
                } else {
                    const double tmin = (double)rmin(rmin(tv, te), tn);
                    const bool lcart = tmin > q.eps_t;
                    if (lcart || sizeof(R) == 8)
                        r = fk3::init_node<R>(q, mesh, lcart, tv, te, tn, tev, ten, tnv, tnve, told, s1,
                                              s2, s3, s4, s5, s6, s7, iz + 1, x + 1, y + 1, sz, sx, sy);
                    else /* near-source spherical stencil in FP64 */
                        r = (R)fk3::init_node<double>(
                            q, mesh64, lcart, (double)tv, (double)te, (double)tn, (double)tev,
                            (double)ten, (double)tnv, (double)tnve, (double)told, (double)s1,
                            (double)s2, (double)s3, (double)s4, (double)s5, (double)s6, (double)s7,
                            iz + 1, x + 1, y + 1, sz, sx, sy);
                }
                if (r != told) {
                    tt[cbase + iz] = r;
                    const double d = fabs((double)r - (double)told);
                    dmax = d > dmax ? d : dmax;
                }
                result = r;
            }
        }
        if (colupd) { zu_uu = cur.duu; zu_ud = cur.dud; zu_du = cur.ddu; zu_dd = cur.ddd; }
        xr[cp][ty][tx] = result;
        xte[cp][ty][tx] = te;
        r_last = result;
        te_last = te;
        tn_last = tn;
        ten_last = ten;
        __syncthreads();
    }
    return dmax;
}

/* Persistent tile-task kernel over sweeps [s_begin, s_end). */
template <typename R, bool INIT>
__global__ void __launch_bounds__(NT, INIT ? 2 : 3) tile_kernel(Params P)
{
    __shared__ R xr[2][TY][TX];
    __shared__ R xte[2][TY][TX];
    __shared__ long long s_task;
    __shared__ int s_fail;
    __shared__ double s_max[TY];
    const int tid = threadIdx.x;
    const long long total = (long long)(P.s_end - P.s_begin) * P.ntask_sweep;
    for (;;) {
        if (tid == 0) {
            long long t = (long long)atomicAdd(P.ticket, 1ull);
            if (t >= total || *((volatile int *)P.error) != 0) t = -1;
            s_task = t;
            s_fail = 0;
        }
        __syncthreads();
        const long long t = s_task;
        if (t < 0) break;
        const int s = P.s_begin + (int)(t / P.ntask_sweep);
        const int2 tk = P.tasks[t % P.ntask_sweep];
        const fk_work3d_t w = P.work[tk.x];
        const fk_grid3d_t g = P.grids[w.grid];
        const int ntx = (g.nx + TX - 1) / TX, nty = (g.ny + TY - 1) / TY;
        const int bxl = tk.y % ntx, byl = tk.y / ntx;
        const int sweep_no = s % 8 + 1;
        const int s0 = sweep_no - 1;
        const int sx = (s0 % 2 == 0) ? 1 : -1;
        const int sy = ((s0 / 2) % 2 == 0) ? 1 : -1;
        const int bx = (sx > 0) ? bxl : ntx - 1 - bxl;
        const int by = (sy > 0) ? byl : nty - 1 - byl;
        int *done = P.done + P.done_base[tk.x];
        const int me = by * ntx + bx;
        /* dependencies: threads 0..10 each watch one tile */
        if (tid < 11) {
            int need = -1, idx = -1;
            if (tid < 9) { /* self and the 8 neighbours: done with sweep s-1 */
                const int dx = tid % 3 - 1, dy = tid / 3 - 1;
                const int nbx = bx + dx, nby = by + dy;
                if (nbx >= 0 && nbx < ntx && nby >= 0 && nby < nty) { idx = nby * ntx + nbx; need = s; }
            } else if (tid == 9) { /* x-upwind face: done with sweep s */
                if (bxl > 0) { idx = by * ntx + (bx - sx); need = s + 1; }
            } else { /* y-upwind face */
                if (byl > 0) { idx = (by - sy) * ntx + bx; need = s + 1; }
            }
            if (idx >= 0) {
                long long it = 0;
                while (ld_acquire(done + idx) < need) {
                    if (++it > P.spin_limit) {
                        atomicCAS(P.error, 0, 1000 + tid);
                        s_fail = 1;
                        break;
                    }
                    __nanosleep(64);
                }
            }
        }
        __syncthreads();
        if (s_fail) break;
        __threadfence();
        const int pass = INIT ? -1 : (s - 8) / 8;
        bool skip = false;
        if (!INIT && P.converge) skip = *((volatile int *)(P.conv_pass + tk.x)) < pass;
        Src q;
        tw_setup_src(q, w, g, P.eps);
        double dmax = 0.0;
        if (INIT) {
            /* tiles outside this sweep's source-limited box keep their values */
            const int s0i = sweep_no - 1;
            const int szi = (s0i < 4) ? 1 : -1;
            (void)szi;
            const int lox = (sx > 0) ? max(1, q.xsi - 1) : max(1, g.nx - q.xsi - 1);
            const int loy = (sy > 0) ? max(1, q.ysi - 1) : max(1, g.ny - q.ysi - 1);
            const int xmax_log = (sx > 0) ? min(g.nx, (bx + 1) * TX) - 1 : g.nx - 1 - bx * TX;
            const int ymax_log = (sy > 0) ? min(g.ny, (by + 1) * TY) - 1 : g.ny - 1 - by * TY;
            skip = xmax_log < lox || ymax_log < loy;
        }
        if (!skip) {
            Mesh<R> mesh;
            Mesh<double> mesh64;
            fk3::make_mesh<R>(mesh, g.dz, g.dx, g.dy);
            if (INIT) fk3::make_mesh<double>(mesh64, g.dz, g.dx, g.dy);
            dmax = tile_sweep<R, INIT>(g, reinterpret_cast<R *>(w.tt),
                                       reinterpret_cast<const R *>(g.slow), q, mesh, mesh64,
                                       sweep_no, bx, by, xr, xte);
        }
        /* publish: results visible before the completion count */
        __threadfence();
        if (!INIT) {
            for (int o = 16; o > 0; o >>= 1) {
                const double v = __shfl_xor_sync(0xffffffffu, dmax, o);
                dmax = v > dmax ? v : dmax;
            }
            if ((tid & 31) == 0) s_max[tid >> 5] = dmax;
        }
        __syncthreads();
        if (tid == 0) {
            if (!INIT) {
                double m = 0.0;
                for (int k = 0; k < TY; ++k) m = s_max[k] > m ? s_max[k] : m;
                if (pass < P.npass) {
                    unsigned long long *rp = P.resid + (size_t)tk.x * P.npass + pass;
                    atomicMax(rp, (unsigned long long)__double_as_longlong(m));
                    if (sweep_no == 8) {
                        __threadfence();
                        const int c = atomicAdd(P.pass_tiles + (size_t)tk.x * P.npass + pass, 1);
                        if (c == ntx * nty - 1) {
                            const double r = __longlong_as_double((long long)atomicAdd(rp, 0ull));
                            if (P.converge && r <= P.conv_tol) atomicMin(P.conv_pass + tk.x, pass);
                        }
                    }
                }
            }
            st_release(done + me, s + 1);
        }
    }
}

/* Field initialisation of every work item (solver3D.F90:1201-1202) and the
 * analytic source corners (localSolver.F90:933-956, FP64). */
template <typename R>
__global__ void field_init_kernel(const fk_grid3d_t *__restrict__ grids,
                                  const fk_work3d_t *__restrict__ work, double eps)
{
    const fk_work3d_t w = work[blockIdx.y];
    const fk_grid3d_t g = grids[w.grid];
    R *tt = reinterpret_cast<R *>(w.tt);
    const size_t n = (size_t)g.ny * g.nx * g.zp;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n;
         e += (size_t)gridDim.x * blockDim.x)
        tt[e] = (R)FK_HUGE;
}

template <typename R>
__global__ void corners_kernel(const fk_grid3d_t *__restrict__ grids,
                               const fk_work3d_t *__restrict__ work, int nwork, double eps)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nwork * 8) return;
    const fk_work3d_t w = work[i / 8];
    const fk_grid3d_t g = grids[w.grid];
    Src q;
    tw_setup_src(q, w, g, eps);
    Mesh<double> m64;
    fk3::make_mesh<double>(m64, g.dz, g.dx, g.dy);
    const int c = i % 8, di = c & 1, dj = (c >> 1) & 1, dk = (c >> 2) & 1;
    const double t = fk3::tana<double>(q, m64, q.zsi + di, q.xsi + dj, q.ysi + dk);
    R *tt = reinterpret_cast<R *>(w.tt);
    tt[((size_t)(q.ysi - 1 + dk) * g.nx + (q.xsi - 1 + dj)) * g.zp + (q.zsi - 1 + di)] = (R)t;
}

/* Per-work-item results from the pass bookkeeping. */
static __global__ void finalize_kernel(int nwork, int npass, int converge, int nsweep,
                                const unsigned long long *__restrict__ resid,
                                const int *__restrict__ conv_pass, const int *__restrict__ error,
                                fk_result3d_t *__restrict__ results)
{
    const int w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= nwork) return;
    int ran = converge ? min(conv_pass[w] + 1, npass) : nsweep;
    if (ran < 0) ran = 0;
    results[w].npass = ran;
    results[w].residual = (ran > 0) ? __longlong_as_double((long long)resid[(size_t)w * npass + ran - 1]) : 0.0;
    results[w].status = *error;
}

inline int occupancy_ctas(const void *fn, int threads)
{
    int dev = 0, nsm = 0, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fn, threads, 0);
    if (per < 1) per = 1;
    return nsm * per;
}

extern cudaEvent_t *g_tile_events; /* sweep3d_f32.cu */

template <typename R>
inline int launch_tiles(const fk_grid3d_t *grids, const fk_work3d_t *work, int nwork,
                        const fk_tiles3d_t *pl, fk_result3d_t *results, double eps, int nsweep,
                        double conv_tol, int max_pass, cudaStream_t st)
{
    if (nwork <= 0) return 0;
    const int converge = conv_tol >= 0.0 && max_pass > 0;
    const int npass = converge ? max_pass : nsweep;
    const int npr = npass > 0 ? npass : 1;
    cudaError_t e = cudaSuccess;
    e = cudaMemsetAsync(pl->done, 0, sizeof(int) * (size_t)pl->ntiles_total, st);
    if (!e) e = cudaMemsetAsync(pl->tickets, 0, 2 * sizeof(unsigned long long), st);
    if (!e) e = cudaMemsetAsync(pl->error, 0, sizeof(int), st);
    if (!e) e = cudaMemsetAsync(pl->resid, 0, sizeof(unsigned long long) * (size_t)nwork * npr, st);
    if (!e) e = cudaMemsetAsync(pl->pass_tiles, 0, sizeof(int) * (size_t)nwork * npr, st);
    if (!e) e = cudaMemsetAsync(pl->conv_pass, 0x3f, sizeof(int) * (size_t)nwork, st);
    if (e) return (int)e;
    field_init_kernel<R><<<dim3(64, nwork), 256, 0, st>>>(grids, work, eps);
    corners_kernel<R><<<(nwork * 8 + 127) / 128, 128, 0, st>>>(grids, work, nwork, eps);
    Params P;
    P.grids = grids;
    P.work = work;
    P.tasks = reinterpret_cast<const int2 *>(pl->tasks);
    P.done_base = pl->done_base;
    P.ntask_sweep = pl->ntask_sweep;
    P.done = pl->done;
    P.error = pl->error;
    P.resid = pl->resid;
    P.pass_tiles = pl->pass_tiles;
    P.conv_pass = pl->conv_pass;
    P.npass = npr;
    P.converge = converge;
    P.eps = eps;
    P.conv_tol = conv_tol;
    P.spin_limit = pl->spin_limit;
    P.s_begin = 0;
    P.s_end = 8;
    P.ticket = pl->tickets;
    const int gi = occupancy_ctas((const void *)tile_kernel<R, true>, NT);
    if (g_tile_events) cudaEventRecord(g_tile_events[0], st);
    tile_kernel<R, true><<<gi, NT, 0, st>>>(P);
    if (g_tile_events) cudaEventRecord(g_tile_events[1], st);
    if (npass > 0) {
        P.s_begin = 8;
        P.s_end = 8 + 8 * npass;
        P.ticket = pl->tickets + 1;
        const int gp = occupancy_ctas((const void *)tile_kernel<R, false>, NT);
        tile_kernel<R, false><<<gp, NT, 0, st>>>(P);
    }
    if (g_tile_events) cudaEventRecord(g_tile_events[2], st);
    finalize_kernel<<<(nwork + 127) / 128, 128, 0, st>>>(nwork, npr, converge, npass, pl->resid,
                                                          pl->conv_pass, pl->error, results);
    return (int)cudaGetLastError();
}

} // namespace fk3tw
