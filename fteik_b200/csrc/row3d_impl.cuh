/*
 * row3d_impl.cuh -- slab-pipelined schedule of the 3D sweeps (the product
 * path for batched and single-source solves).
 *
 * A task is one sweep over one slab of TY = FK_SLAB_Y (4) physical y-rows of
 * one (grid, source) work item, over the whole x extent, run by one block of
 * TY warps: warp ty owns row TY P + ty; lane l walks the columns x' = 32 k + l
 * (k = 0, 1, ... in the sweep's logical x order) one after the other, each
 * over its z positions.  At block step t the thread works on item
 * j = t - l - DL oy (column block k = j / Zp, z position j % Zp), oy being
 * its row's offset from the slab's upwind edge, so its seven upwind values
 * come from:
 *   tv, tev, tnv, tnve   its own previous step                    (registers)
 *   te                   lane l-1's previous step                 (shuffle)
 *                        or, for lane 0, lane 31 of block k-1 through a
 *                        per-warp ring in shared memory (Zp - 31 >= 1 steps old)
 * (the initialisation sweeps start at the block holding x' = lox - 1)
 *   tn                   the y-upwind warp's step t - DL           (shared memory)
 *                        or, for the slab's first row, the upwind slab's
 *                        last row, final for this sweep            (global, L2)
 *   ten                  lane l-1's tn of the previous step        (shuffle)
 *                        or, for lane 0, lane 31's through the ring
 * Rows lag DL steps behind their upwind row, so the block synchronises
 * once per DL steps (the upwind row's values of the previous window are then
 * visible) instead of every step: DL = 2, except DLP = 4 in the staged
 * FP32 pass step.  A longer lag lengthens the chain of upwind slabs and the
 * skew ramp (31 + DL (TY - 1) steps, paid once per slab); a shorter one
 * costs barriers.  Measured on 64 sources x 4 grids: the staged FP32 pass
 * step 57.1 ms at DL = 2, 53.3 ms at 4, 60.0 ms at 8; the direct one 64.0 ms
 * at 2, 67.0 ms at 4; the initialisation sweeps 14.4, 14.9 and 16.5 ms at
 * 2, 4 and 8.
 *
 * Slabs publish their progress as (sweep << 20) | steps done every CH steps
 * (8 in the initialisation sweeps; in the passes 8 when a sweep has few
 * slab tasks for the resident blocks, whose chains of upwind slabs are then
 * the critical path, else 32, fewer polls) and (sweep + 1) << 20
 * when done (one thread, release store after a block
 * barrier).  A slab waits (one thread, acquire loads, bounded) for the
 * upwind slab to be ahead of what it prefetches, and before it starts, for
 * slabs P-1, P, P+1 to be done with the previous sweep (they read this
 * slab's old values).  Tasks are claimed through one atomic ticket,
 * sweep-major and in the sweep's y order, so a slab only waits on slabs with
 * smaller tickets: the waits cannot cycle.  As in the level-set sweep
 * (autoCode.f90), each node reads only upwind nodes, so the result equals
 * the reference's sweep bit for bit in FP64.
 */
#pragma once
#include "slab3d_common.cuh"

namespace fk3rw {
using fk3::Mesh;
using fk3::Src;
using fk3::rmin;
using fk3::rmax;

constexpr int TY = FK_SLAB_Y;        /* rows (warps) per slab */
constexpr int NT = TY * 32;
constexpr int CH_INIT = 8;           /* progress granularity of the initialisation sweeps, steps */
constexpr int CH_INIT_STG = 16;      /* the same on the staged walk (11.4 against 11.6 ms at 8, 11.6 at 32) */
constexpr int CH_FEW = 8, CH_MANY = 32; /* passes: few tasks per sweep want a short lag, many few polls */
constexpr int DL = 2;                /* row-to-row lag inside a slab = block barrier interval */
constexpr int NB = 2 * DL;           /* row exchange buffer depth */
constexpr int DLP = 4, NBP = 2 * DLP; /* the same for the staged FP32 pass step */
constexpr int SHIFT = 20;            /* counter = (sweep << SHIFT) | steps */

template <typename R, int S>
struct Pre {
    R told[S], tn[S];                /* per source */
    R duu, dud, ddu, ddd;            /* z-downwind slowness layer, s<z><x><y> with z = D */
    int addr;                        /* node offset in the fields */
};

/* Sleep between polls, doubling from 64 ns to 1 us: a waiting block's polls
 * take issue slots and L2 requests from the working ones, and a wait ends
 * at most ~1 us after its condition holds. */
__device__ __forceinline__ void poll_backoff(unsigned &ns)
{
    __nanosleep(ns);
    ns = ns < 1024u ? 2u * ns : 1024u;
}

/* Bounded acquire wait by one thread until *p >= need; false on timeout. */
__device__ __forceinline__ bool wait_ge1(const int *p, int need, long long limit, int *error, int code)
{
    long long it = 0;
    unsigned ns = 64;
    while (fk3tw::ld_acquire(p) < need) {
        if (++it > limit) {
            atomicCAS(error, 0, code);
            return false;
        }
        poll_backoff(ns);
    }
    return true;
}

/* One sweep over physical slab P.  Returns false on a wait timeout (the
 * whole block returns false). */
/* One sweep over physical slab P.  In the initialisation sweeps each source
 * updates only its own box (solver3D.F90:493-565); with two sources per
 * thread the walk covers the union of the two boxes and a source's nodes
 * outside its own box keep their values, which is what that source's own
 * walk would read there. */
template <typename R, bool INIT, bool RESID, int S, int CHP>
__device__ __forceinline__ bool slab_sweep(const fk3tw::Params &P_, const fk_grid3d_t &g, R *const (&ttp)[S],
                                           const R *__restrict__ slow, const Src (&qs)[S], int s, int sweep_no,
                                           int P, int nslab, int *const (&prog)[S], R (*xr)[S][TY][32],
                                           R *ring, int zring, int *s_flag,
                                           double (&dmax)[S])
{
    constexpr int CH = INIT ? CH_INIT : CHP;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    const unsigned FULL = 0xffffffffu;
    const int nz = g.nz, nx = g.nx, ny = g.ny, zp = g.zp, zcp = g.zcp;
    const int s0 = sweep_no - 1;
    const int sz = (s0 < 4) ? 1 : -1;
    const int sx = (s0 % 2 == 0) ? 1 : -1;
    const int sy = ((s0 / 2) % 2 == 0) ? 1 : -1;
    int loz = 1, lox = 1, loy = 1;            /* the walk's box: the union of the sources' boxes */
    int lozi[S], loxi[S], loyi[S];
    R eps_r[S];
#pragma unroll
    for (int i = 0; i < S; ++i) {
        lozi[i] = loxi[i] = loyi[i] = 1;
        eps_r[i] = (R)qs[i].eps_t;
        if (INIT) { /* solver3D.F90:493-565, flipped bound clamped to the grid */
            lozi[i] = (sz > 0) ? max(1, qs[i].zsi - 1) : max(1, nz - qs[i].zsi - 1);
            loxi[i] = (sx > 0) ? max(1, qs[i].xsi - 1) : max(1, nx - qs[i].xsi - 1);
            loyi[i] = (sy > 0) ? max(1, qs[i].ysi - 1) : max(1, ny - qs[i].ysi - 1);
        }
    }
    if (INIT) {
        loz = lozi[0]; lox = loxi[0]; loy = loyi[0];
#pragma unroll
        for (int i = 1; i < S; ++i)
            if (ttp[i]) { loz = min(loz, lozi[i]); lox = min(lox, loxi[i]); loy = min(loy, loyi[i]); }
    }
    Mesh<R> mesh;
    fk3::make_mesh<R>(mesh, g.dz, g.dx, g.dy);
    const R HUGEV = (R)FK_HUGE;
    const int th = min(TY, ny - TY * P);             /* rows in this slab */
    const bool row = ty < th;
    const int y = TY * P + ty;
    const int oy = (sy > 0) ? ty : th - 1 - ty;      /* offset from the upwind edge */
    const int yl = (sy > 0) ? y : ny - 1 - y;        /* logical row */
    const bool rowupd = row && yl >= loy;
    const int wy = ty - sy;                          /* y-upwind warp (oy >= 1) */
    const int Z = nz - loz + 1;                      /* walk positions: il = loz-1 .. nz-1 */
    const int Zp = Z > 32 ? Z : 32;
    const int K = (nx + 31) / 32;
    /* column blocks wholly before x' = lox - 1 are neither updated nor read */
    const int k0 = (lox - 1) / 32;
    const int T = (K - k0) * Zp + 31 + DL * (TY - 1);
    const int Pu = P - sy;                           /* upwind slab */
    const bool has_up = Pu >= 0 && Pu < nslab;
    /* the upwind slab changes in this sweep when its last logical row does */
    const int ylast_up = has_up ? ((sy > 0) ? TY * Pu + min(TY, ny - TY * Pu) - 1 : TY * Pu) : 0;
    const bool wait_up = has_up && (((sy > 0) ? ylast_up : ny - 1 - ylast_up) >= loy);
    const int yu = y - sy;
    const bool has_yu = row && yu >= 0 && yu < ny;
    const int cyU = (sy > 0) ? y - 1 : y;
    const int cyD = min(max((sy > 0) ? y : y - 1, 0), ny - 2);
    const int rowU = cyU * (nx - 1), rowD = cyD * (nx - 1);
    const int ybase = y * nx, yubase = yu * nx;

    auto fetch = [&](int kk, int zz, Pre<R, S> &f) {
        const int xl = 32 * kk + tx;
        if (!(row && zz >= 0 && zz < Z && kk < K && xl < nx)) return;
        const int x = (sx > 0) ? xl : nx - 1 - xl;
        const int il = loz - 1 + zz;
        const int iz = (sz > 0) ? il : nz - 1 - il;
        f.addr = (ybase + x) * zp + iz;
        const int au = (yubase + x) * zp + iz;
#pragma unroll
        for (int i = 0; i < S; ++i) {
            if (ttp[i]) {
                f.told[i] = fk3tw::ldcg(ttp[i] + f.addr);
                if (oy == 0) f.tn[i] = has_yu ? fk3tw::ldcg(ttp[i] + au) : HUGEV;
            }
        }
        if (rowupd && xl >= lox) {
            const int cxU = (sx > 0) ? x - 1 : x;
            const int cxD = min(max((sx > 0) ? x : x - 1, 0), nx - 2);
            const int czD = min(max((sz > 0) ? iz : iz - 1, 0), nz - 2);
            f.duu = __ldg(slow + ((rowU + cxU) * zcp + czD));
            f.dud = __ldg(slow + ((rowD + cxU) * zcp + czD));
            f.ddu = __ldg(slow + ((rowU + cxD) * zcp + czD));
            f.ddd = __ldg(slow + ((rowD + cxD) * zcp + czD));
        }
    };

    /* the first row's prefetches reach item t + 1 - tx at step t; the upwind
     * slab's last row works on that item at its step t + 1 + DL (th_up - 1) */
    const int *prog_up = prog[0] + (has_up ? Pu : P);
    if (threadIdx.x == 0) {
        s_flag[0] = 1;
        if (wait_up && !wait_ge1(prog_up, (s << SHIFT) | min(T, CH + DL * (TY - 1) + 2), P_.spin_limit, P_.error,
                                 3000))
            s_flag[0] = 0;
    }
    __syncthreads();
    if (!s_flag[0]) return false;

    int kn = k0, zqn = -tx - DL * oy;    /* item of the next step */
    Pre<R, S> cur, nxt;
#pragma unroll
    for (int i = 0; i < S; ++i) nxt.told[i] = nxt.tn[i] = HUGEV;
    nxt.duu = nxt.dud = nxt.ddu = nxt.ddd = (R)0;
    nxt.addr = 0;
    fetch(kn, zqn, nxt);
    R zu_uu = 0, zu_ud = 0, zu_du = 0, zu_dd = 0;   /* z-upwind layer (previous step) */
    R r_last[S], te_last[S], tn_last[S], ten_last[S];
#pragma unroll
    for (int i = 0; i < S; ++i) r_last[i] = te_last[i] = tn_last[i] = ten_last[i] = HUGEV;
    R *ring_r = ring, *ring_tn = ring + S * zring;   /* [S][zring] each */
    for (int t = 0; t < T; ++t) {
        if (wait_up && t > 0 && t % CH == 0) {
            if (threadIdx.x == 0 &&
                !wait_ge1(prog_up, (s << SHIFT) | min(T, t + CH + DL * (TY - 1) + 2), P_.spin_limit, P_.error,
                          3001))
                s_flag[0] = 0;
            __syncthreads();
            if (!s_flag[0]) return false;
        }
        const int pp = (t + NB - DL) % NB, cp = t % NB;   /* read the upwind row's step t - DL */
        R sh_r[S], sh_tn[S];
#pragma unroll
        for (int i = 0; i < S; ++i) {
            sh_r[i] = __shfl_up_sync(FULL, r_last[i], 1);
            sh_tn[i] = __shfl_up_sync(FULL, tn_last[i], 1);
        }
        const int k = kn, zq = zqn;
        cur = nxt;
        if (++zqn == Zp) { zqn = 0; ++kn; }
        fetch(kn, zqn, nxt);
        const int xl = 32 * k + tx;
        const bool valid = row && zq >= 0 && zq < Z && k < K && xl < nx;
        const bool from_ring = k > k0 && zq >= 0 && zq < Zp;
        const bool upd = valid && rowupd && xl >= lox && zq >= 1; /* il = loz - 1 + zq >= loz */
        R s1, s2, s3, s4, s5, s6, s7;
        {
            const R uuu = zu_uu, uud = zu_ud, udu = zu_du, udd = zu_dd;
            s1 = rmin(rmin(uuu, uud), rmin(udu, udd));
            s2 = rmin(rmin(uuu, uud), rmin(cur.duu, cur.dud));
            s3 = rmin(rmin(uuu, udu), rmin(cur.duu, cur.ddu));
            s4 = rmin(uuu, uud);
            s5 = rmin(uuu, udu);
            s6 = rmin(uuu, cur.duu);
            s7 = uuu;
        }
#pragma unroll
        for (int i = 0; i < S; ++i) {
            const R te = (tx == 0) ? (from_ring ? ring_r[i * zring + zq] : HUGEV) : sh_r[i];
            R tn = HUGEV, ten = HUGEV, result = HUGEV;
            if (valid) {
                tn = (oy == 0) ? cur.tn[i] : xr[pp][i][wy][tx];
                /* lane l-1's y-upwind value one step ago is this node's ten */
                ten = (tx == 0) ? (from_ring ? ring_tn[i * zring + zq] : HUGEV) : sh_tn[i];
                const R told = cur.told[i];
                result = told;
                /* a source updates only inside its own box (the walk's box for S = 1) */
                const bool updi = S == 1 || !INIT ||
                                  (yl >= loyi[i] && xl >= loxi[i] && loz - 1 + zq >= lozi[i]);
                if (upd && updi && ttp[i]) {
                    const Src &q = qs[i];
                    const R tv = r_last[i], tev = te_last[i], tnv = tn_last[i], tnve = ten_last[i];
                    R r;
                    if (!INIT) {
                        r = fk3::noinit(mesh, tv, te, tn, tev, ten, tnv, tnve, s1, s2, s3, s4, s5, s6, s7, told);
                    } else {
                        const int x = (sx > 0) ? xl : nx - 1 - xl;
                        const int il = loz - 1 + zq;
                        const int iz = (sz > 0) ? il : nz - 1 - il;
                        /* the Cartesian / spherical switch (localSolver.F90:572-575)
                         * compares in the field's precision: in FP32 both the upwind
                         * time and the threshold are rounded to FP32, so a time that
                         * equals the threshold in FP64 (a node eps cells from a
                         * node-centred source along a grid line of a uniform medium)
                         * stays spherical, as in FP64, instead of being pushed past the
                         * threshold by its own rounding */
                        const bool lcart = rmin(rmin(tv, te), tn) > eps_r[i];
                        if (lcart && sizeof(R) == 4)
                            /* away from the source the initialisation stencil is the
                             * plane-wave one (localSolver.F90:715-732) */
                            r = fk3::noinit(mesh, tv, te, tn, tev, ten, tnv, tnve, s1, s2, s3, s4, s5, s6, s7,
                                            told);
                        else if (lcart || sizeof(R) == 8)
                            r = fk3::init_node<R>(q, mesh, lcart, tv, te, tn, tev, ten, tnv, tnve, told, s1, s2,
                                                  s3, s4, s5, s6, s7, iz + 1, x + 1, y + 1, sz, sx, sy);
                        else { /* near-source spherical stencil in FP64 (constants built here: few nodes) */
                            Mesh<double> mesh64;
                            fk3::make_mesh<double>(mesh64, g.dz, g.dx, g.dy);
                            r = (R)fk3::init_node<double>(
                                q, mesh64, lcart, (double)tv, (double)te, (double)tn, (double)tev, (double)ten,
                                (double)tnv, (double)tnve, (double)told, (double)s1, (double)s2, (double)s3,
                                (double)s4, (double)s5, (double)s6, (double)s7, iz + 1, x + 1, y + 1, sz, sx,
                                sy);
                        }
                    }
                    if (r != told) {
                        ttp[i][cur.addr] = r;
                        if (RESID) {
                            const double d = fabs((double)r - (double)told);
                            dmax[i] = d > dmax[i] ? d : dmax[i];
                        }
                    }
                    result = r;
                }
            }
            if (tx == 31 && zq >= 0 && zq < Zp) {
                ring_r[i * zring + zq] = result;
                ring_tn[i * zring + zq] = tn;
            }
            xr[cp][i][ty][tx] = result;
            r_last[i] = result;
            te_last[i] = te;
            tn_last[i] = tn;
            ten_last[i] = ten;
        }
        if (valid && rowupd && xl >= lox) { zu_uu = cur.duu; zu_ud = cur.dud; zu_du = cur.ddu; zu_dd = cur.ddd; }
        if ((t + 1) % DL == 0) __syncthreads();   /* the window's row values become visible */
        else __syncwarp();                        /* lane 31 -> lane 0 ring */
        if (threadIdx.x == 0 && (t + 1) % CH == 0 && t + 1 < T) {
            __threadfence();
#pragma unroll
            for (int i = 0; i < S; ++i)
                if (prog[i]) fk3tw::st_release(prog[i] + P, (s << SHIFT) | (t + 1));
        }
    }
    return true;
}

/* Logical z positions of the box of initialisation sweep `sweep_no` of
 * source q (solver3D.F90:493-565): the read-only layer loz - 1 and the
 * updated layers loz .. nz - 1. */
__device__ __forceinline__ int init_box_depth(const Src &q, int nz, int sweep_no)
{
    const int loz = (sweep_no <= 4) ? max(1, q.zsi - 1) : max(1, nz - q.zsi - 1);
    return nz - loz + 1;
}

/* One initialisation sweep of one source over a box at most TY z positions
 * deep (a source within two cells of the surface in the upward sweeps, of
 * the bottom in the downward ones), walked with the axes turned: warp ty is
 * the box's logical z layer loz - 1 + ty, lanes walk x as in slab_sweep,
 * and the walk runs along y, so one task covers the whole box.  slab_sweep
 * walks such a box with at least 32 z steps per column block for its 2 or 3
 * layers; here a column block takes as many steps as the box has rows.  A
 * node's seven upwind values arrive through the same channels in other
 * roles -- its own previous step is the y-upwind node, the row above the
 * z-upwind one, lane l-1 the x-upwind one -- and go to the stencil in their
 * physical roles with the same slowness cells, so every node gets the bits
 * slab_sweep gives it.  No other task reads the box while it runs: no
 * progress counters, no waits. */
template <typename R>
__device__ __forceinline__ void slab_sweep_zrows(const fk_grid3d_t &g, R *tt, const R *__restrict__ slow,
                                                 const Src &q, int sweep_no, R (*xr)[1][TY][32], R *ring,
                                                 int zring)
{
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    const unsigned FULL = 0xffffffffu;
    const int nz = g.nz, nx = g.nx, ny = g.ny, zp = g.zp, zcp = g.zcp;
    const int s0 = sweep_no - 1;
    const int sz = (s0 < 4) ? 1 : -1;
    const int sx = (s0 % 2 == 0) ? 1 : -1;
    const int sy = ((s0 / 2) % 2 == 0) ? 1 : -1;
    /* solver3D.F90:493-565, flipped bounds clamped to the grid */
    const int loz = (sz > 0) ? max(1, q.zsi - 1) : max(1, nz - q.zsi - 1);
    const int lox = (sx > 0) ? max(1, q.xsi - 1) : max(1, nx - q.xsi - 1);
    const int loy = (sy > 0) ? max(1, q.ysi - 1) : max(1, ny - q.ysi - 1);
    Mesh<R> mesh;
    fk3::make_mesh<R>(mesh, g.dz, g.dx, g.dy);
    const R HUGEV = (R)FK_HUGE;
    const R eps_r = (R)q.eps_t;
    const int Zr = nz - loz + 1;                     /* rows: logical z loz - 1 .. nz - 1 */
    const bool row = ty < Zr;
    const int iz = (sz > 0) ? loz - 1 + ty : nz - loz - ty;
    const bool rowupd = row && ty >= 1;              /* logical z >= loz */
    const int Y = ny - loy + 1;                      /* walk positions: logical y loy - 1 .. ny - 1 */
    const int Yp = Y > 32 ? Y : 32;
    const int K = (nx + 31) / 32;
    const int k0 = (lox - 1) / 32;
    const int T = (K - k0) * Yp + 31 + DL * (TY - 1);
    /* slowness cells: z fixed by the row (U: the layer above, D: this one,
     * clamped), x by the lane's column, y by the step: each step fetches its
     * y-downwind layer, the previous step's is its y-upwind one */
    const int czU = (sz > 0) ? iz - 1 : iz;
    const int czD = min(max((sz > 0) ? iz : iz - 1, 0), nz - 2);

    struct Item {
        R told;
        R uud, udd, dud, ddd;   /* y-downwind layer, s<z><x><y> with y = D */
        int addr;
    };
    auto fetch = [&](int kk, int jj, Item &f) {
        const int xl = 32 * kk + tx;
        if (!(row && jj >= 0 && jj < Y && kk < K && xl < nx)) return;
        const int x = (sx > 0) ? xl : nx - 1 - xl;
        const int yl = loy - 1 + jj;
        const int y = (sy > 0) ? yl : ny - 1 - yl;
        f.addr = (y * nx + x) * zp + iz;
        f.told = fk3tw::ldcg(tt + f.addr);
        if (rowupd && xl >= lox) {
            const int cxU = (sx > 0) ? x - 1 : x;
            const int cxD = min(max((sx > 0) ? x : x - 1, 0), nx - 2);
            const int rD = min(max((sy > 0) ? y : y - 1, 0), ny - 2) * (nx - 1);
            f.uud = __ldg(slow + ((rD + cxU) * zcp + czU));
            f.udd = __ldg(slow + ((rD + cxD) * zcp + czU));
            f.dud = __ldg(slow + ((rD + cxU) * zcp + czD));
            f.ddd = __ldg(slow + ((rD + cxD) * zcp + czD));
        }
    };

    int kn = k0, jn = -tx - DL * ty;     /* item of the next step */
    Item cur, nxt;
    nxt.told = HUGEV;
    nxt.uud = nxt.udd = nxt.dud = nxt.ddd = (R)0;
    nxt.addr = 0;
    fetch(kn, jn, nxt);
    R yu_uu = 0, yu_ud = 0, yu_du = 0, yu_dd = 0;   /* y-upwind layer (previous step) */
    /* previous step's: own result (y-upwind node), x-upwind value, z-upwind
     * value, and x-upwind's z-upwind value */
    R r_last = HUGEV, te_last = HUGEV, tv_last = HUGEV, tev_last = HUGEV;
    R *ring_r = ring, *ring_tv = ring + zring;
    for (int t = 0; t < T; ++t) {
        const int pp = (t + NB - DL) % NB, cp = t % NB;   /* the row above's step t - DL */
        const R sh_r = __shfl_up_sync(FULL, r_last, 1);
        const R sh_tv = __shfl_up_sync(FULL, tv_last, 1);
        const int k = kn, j = jn;
        cur = nxt;
        if (++jn == Yp) { jn = 0; ++kn; }
        fetch(kn, jn, nxt);
        const int xl = 32 * k + tx;
        const bool valid = row && j >= 0 && j < Y && k < K && xl < nx;
        const bool from_ring = k > k0 && j >= 0 && j < Yp;
        const bool upd = valid && rowupd && xl >= lox && j >= 1;   /* logical y >= loy */
        /* the seven cells in the names of slab_sweep: uuu = (zU, xU, yU) ... */
        const R uuu = yu_uu, udu = yu_ud, duu = yu_du, ddu = yu_dd;
        const R uud = cur.uud, udd = cur.udd, dud = cur.dud;
        const R s4 = rmin(uuu, uud), s5 = rmin(uuu, udu), s6 = rmin(uuu, duu);
        const R s1 = rmin(s4, rmin(udu, udd));
        const R s2 = rmin(s4, rmin(duu, dud));
        const R s3 = rmin(s5, rmin(duu, ddu));
        const R s7 = uuu;
        const R te = (tx == 0) ? (from_ring ? ring_r[j] : HUGEV) : sh_r;
        R tv = HUGEV, tev = HUGEV, result = HUGEV;
        if (valid) {
            tv = (ty == 0) ? HUGEV : xr[pp][0][ty - 1][tx];
            tev = (tx == 0) ? (from_ring ? ring_tv[j] : HUGEV) : sh_tv;
            const R told = cur.told;
            result = told;
            if (upd) {
                const R tn = r_last, ten = te_last, tnv = tv_last, tnve = tev_last;
                const int x = (sx > 0) ? xl : nx - 1 - xl;
                const int yl = loy - 1 + j;
                const int y = (sy > 0) ? yl : ny - 1 - yl;
                /* as in slab_sweep: the switch compares in the field's precision */
                const bool lcart = rmin(rmin(tv, te), tn) > eps_r;
                R r;
                if (lcart && sizeof(R) == 4)
                    r = fk3::noinit(mesh, tv, te, tn, tev, ten, tnv, tnve, s1, s2, s3, s4, s5, s6, s7, told);
                else if (lcart || sizeof(R) == 8)
                    r = fk3::init_node<R>(q, mesh, lcart, tv, te, tn, tev, ten, tnv, tnve, told, s1, s2, s3, s4, s5,
                                          s6, s7, iz + 1, x + 1, y + 1, sz, sx, sy);
                else {   /* near-source spherical stencil in FP64 (constants built here: few nodes) */
                    Mesh<double> mesh64;
                    fk3::make_mesh<double>(mesh64, g.dz, g.dx, g.dy);
                    r = (R)fk3::init_node<double>(q, mesh64, lcart, (double)tv, (double)te, (double)tn, (double)tev,
                                                  (double)ten, (double)tnv, (double)tnve, (double)told, (double)s1,
                                                  (double)s2, (double)s3, (double)s4, (double)s5, (double)s6,
                                                  (double)s7, iz + 1, x + 1, y + 1, sz, sx, sy);
                }
                if (r != told) tt[cur.addr] = r;
                result = r;
            }
        }
        if (tx == 31 && j >= 0 && j < Yp) {
            ring_r[j] = result;
            ring_tv[j] = tv;
        }
        xr[cp][0][ty][tx] = result;
        r_last = result;
        te_last = te;
        tv_last = tv;
        tev_last = tev;
        if (valid && rowupd && xl >= lox) { yu_uu = cur.uud; yu_ud = cur.udd; yu_du = cur.dud; yu_dd = cur.ddd; }
        if ((t + 1) % DL == 0) __syncthreads();   /* the window's row values become visible */
        else __syncwarp();                        /* lane 31 -> lane 0 ring */
    }
}

/* The Gauss-Seidel stencil of the FP32 pass steps for the S sources of a
 * thread (they share the slowness): with PACKED the two sources in packed
 * float2 instructions (noinit_v<float2>; 5 % faster in the staged step,
 * 14 % slower in the direct one), else noinit_f32 per source.  Both forms
 * perform the same roundings in the same order, so every configuration
 * gives the same bits. */
template <int S, bool PACKED>
__device__ __forceinline__ void pass_stencil(const Mesh<float> &mesh, const float (&tv)[S], const float (&te)[S],
                                             const float (&tn)[S], const float (&tev)[S], const float (&ten)[S],
                                             const float (&tnv)[S], const float (&tnve)[S], float s1, float s2,
                                             float s3, float s4, float s5, float s6, float s7,
                                             const float (&told)[S], float (&r)[S])
{
    if constexpr (PACKED && S == 2) {
        const float2 o = fk3::noinit_v<float2>(
            mesh, make_float2(tv[0], tv[1]), make_float2(te[0], te[1]), make_float2(tn[0], tn[1]),
            make_float2(tev[0], tev[1]), make_float2(ten[0], ten[1]), make_float2(tnv[0], tnv[1]),
            make_float2(tnve[0], tnve[1]), s1, s2, s3, s4, s5, s6, s7, make_float2(told[0], told[1]));
        r[0] = o.x;
        r[S - 1] = o.y;
    } else {
#pragma unroll
        for (int i = 0; i < S; ++i)
            r[i] = fk3::noinit_f32(mesh, tv[i], te[i], tn[i], tev[i], ten[i], tnv[i], tnve[i], s1, s2, s3, s4, s5,
                                   s6, s7, told[i]);
    }
}

/* One Gauss-Seidel sweep over physical slab P in FP32: the walk of
 * slab_sweep without the bookkeeping of the initialisation sweeps.  A pass
 * has no source-limited box, so a lane's items are (column block k, z
 * position zq) with zq wrapping at Zp and k = 0, 1, ...; the field and
 * slowness indices are linear in both (the edge clamps are per-lane
 * constants: x' = 0 is never updated and x' = nx - 1 has a zero x offset),
 * and the steps run in windows of DL so the exchange-buffer slots are
 * compile-time constants.  (Moving the two sources' row values as one 64-bit
 * shared-memory word instead measured 14 % slower.)  A missing second source
 * (odd number of sources on a grid) walks source 0's field without storing.
 * The nodes updated, their order and the waits are those of slab_sweep; the
 * stencil is noinit_f32 per source, so a source gives the same bits whether
 * it walks alone or paired. */
template <bool RESID, int S, int CHP>
__device__ __forceinline__ bool slab_pass_f32(const fk3tw::Params &P_, const fk_grid3d_t &g,
                                              float *const (&ttp)[S], const float *__restrict__ slow, int s,
                                              int sweep_no, int P, int nslab, int *const (&prog)[S],
                                              float (*xr)[S][TY][32], float *ring, int zring, int *s_flag,
                                              double (&dmax)[S])
{
    constexpr int CH = CHP;
    static_assert(CH % DL == 0 && NB == 2 * DL, "progress and buffer slots follow the DL windows");
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    const unsigned FULL = 0xffffffffu;
    const int nz = g.nz, nx = g.nx, ny = g.ny, zp = g.zp, zcp = g.zcp;
    const int s0 = sweep_no - 1;
    const int sz = (s0 < 4) ? 1 : -1;
    const int sx = (s0 % 2 == 0) ? 1 : -1;
    const int sy = ((s0 / 2) % 2 == 0) ? 1 : -1;
    Mesh<float> mesh;
    fk3::make_mesh<float>(mesh, g.dz, g.dx, g.dy);
    const float HUGEV = (float)FK_HUGE;
    const int th = min(TY, ny - TY * P);
    const bool row = ty < th;
    const int y = TY * P + ty;
    const int oy = (sy > 0) ? ty : th - 1 - ty;
    const int yl = (sy > 0) ? y : ny - 1 - y;
    const bool rowupd = row && yl >= 1;
    const int wy = ty - sy;
    const int Z = nz;
    const int Zp = Z > 32 ? Z : 32;
    const int K = (nx + 31) / 32;
    const int T = K * Zp + 31 + DL * (TY - 1);
    const int Pu = P - sy;
    const bool has_up = Pu >= 0 && Pu < nslab;
    const int ylast_up = has_up ? ((sy > 0) ? TY * Pu + min(TY, ny - TY * Pu) - 1 : TY * Pu) : 0;
    const bool wait_up = has_up && (((sy > 0) ? ylast_up : ny - 1 - ylast_up) >= 1);
    const int yu = y - sy;
    const bool has_yu = row && yu >= 0 && yu < ny;
    const bool has2 = S == 2 && ttp[S - 1] != nullptr;
    const float *const tt0 = ttp[0];
    const float *const tt1 = has2 ? ttp[S - 1] : ttp[0];

    /* item (k, zq) of this lane: node x = x0 + 32 sx k, z = iz0 + sz zq */
    const int x0 = (sx > 0) ? tx : nx - 1 - tx;
    const int iz0 = (sz > 0) ? 0 : nz - 1;
    const int kl = row ? (nx - tx + 31) / 32 : 0;                  /* blocks with x' < nx */
    const int kmin = rowupd ? (tx == 0 ? 1 : 0) : 0x7fffffff;       /* updated: x' >= 1, y' >= 1 */
    const int kxl = (nx - 1 >= tx && (nx - 1 - tx) % 32 == 0) ? (nx - 1 - tx) / 32 : -1; /* x' = nx - 1 */
    const int baseT = (y * nx + x0) * zp + iz0;
    const int dkT = 32 * sx * zp;
    const int dyT = sy * nx * zp;                                   /* to the y-upwind row */
    /* slowness: cells (cxU | cxD, cyU | cyD, czD), czD = iz - (sz < 0) clamped to the grid */
    const int cyU = (sy > 0) ? y - 1 : y;
    const int cyD = min(max((sy > 0) ? y : y - 1, 0), ny - 2);
    const int baseS = (cyU * (nx - 1) + x0 - (sx > 0 ? 1 : 0)) * zcp + ((sz > 0) ? 0 : nz - 2);
    const int dkS = 32 * sx * zcp;
    const int offY = (cyD - cyU) * (nx - 1) * zcp;
    const int offX = sx * zcp;

    struct Item {
        float told[S], tn[S];
        float duu, dud, ddu, ddd;   /* z-downwind slowness layer, s<z><x><y> with z = D */
        int it, k, zq;
    };
    auto fetch = [&](Item &f, int kk, int zz) {
        f.k = kk;
        f.zq = zz;
        f.it = baseT + kk * dkT + sz * zz;
        const bool v = (unsigned)zz < (unsigned)Z && kk < kl;
        if (v) {
            f.told[0] = fk3tw::ldcg(tt0 + f.it);
            if (S == 2) f.told[S - 1] = fk3tw::ldcg(tt1 + f.it);
            if (oy == 0) {
                f.tn[0] = has_yu ? fk3tw::ldcg(tt0 + (f.it - dyT)) : HUGEV;
                if (S == 2) f.tn[S - 1] = has_yu ? fk3tw::ldcg(tt1 + (f.it - dyT)) : HUGEV;
            }
        }
        if (v && kk >= kmin) {
            const int is = baseS + kk * dkS + sz * min(zz, nz - 2);
            const int ox = (kk == kxl) ? 0 : offX;
            f.duu = __ldg(slow + is);
            f.dud = __ldg(slow + (is + offY));
            f.ddu = __ldg(slow + (is + ox));
            f.ddd = __ldg(slow + (is + ox + offY));
        }
    };

    const int *prog_up = prog[0] + (has_up ? Pu : P);
    if (threadIdx.x == 0) {
        s_flag[0] = 1;
        if (wait_up && !wait_ge1(prog_up, (s << SHIFT) | min(T, CH + DL * (TY - 1) + 2), P_.spin_limit, P_.error,
                                 3000))
            s_flag[0] = 0;
    }
    __syncthreads();
    if (!s_flag[0]) return false;

    int nk = 0, nzq = -tx - DL * oy;     /* item of the next step */
    Item nxt;
#pragma unroll
    for (int i = 0; i < S; ++i) nxt.told[i] = nxt.tn[i] = HUGEV;
    nxt.duu = nxt.dud = nxt.ddu = nxt.ddd = 0.0f;
    fetch(nxt, nk, nzq);
    if (++nzq == Zp) { nzq = 0; ++nk; }
    float zu_uu = 0.0f, zu_ud = 0.0f, zu_du = 0.0f, zu_dd = 0.0f;   /* z-upwind layer (previous step) */
    float r_last[S], te_last[S], tn_last[S], ten_last[S];
#pragma unroll
    for (int i = 0; i < S; ++i) r_last[i] = te_last[i] = tn_last[i] = ten_last[i] = HUGEV;
    float *ring_r = ring, *ring_tn = ring + S * zring;   /* [S][zring] each */
    for (int t0 = 0; t0 < T; t0 += DL) {
        if (wait_up && t0 > 0 && t0 % CH == 0) {
            if (threadIdx.x == 0 &&
                !wait_ge1(prog_up, (s << SHIFT) | min(T, t0 + CH + DL * (TY - 1) + 2), P_.spin_limit, P_.error,
                          3001))
                s_flag[0] = 0;
            __syncthreads();
            if (!s_flag[0]) return false;
        }
        const int half = (t0 / DL) & 1;   /* this window writes slots half DL + u, reads the other half */
        float (*const xw)[S][TY][32] = xr + half * DL;
        float (*const xrd)[S][TY][32] = xr + (1 - half) * DL;
#pragma unroll
        for (int u = 0; u < DL; ++u) {
            float sh_r[S], sh_tn[S];
#pragma unroll
            for (int i = 0; i < S; ++i) {
                sh_r[i] = __shfl_up_sync(FULL, r_last[i], 1);
                sh_tn[i] = __shfl_up_sync(FULL, tn_last[i], 1);
            }
            const Item cur = nxt;
            fetch(nxt, nk, nzq);
            if (++nzq == Zp) { nzq = 0; ++nk; }
            const bool valid = (unsigned)cur.zq < (unsigned)Z && cur.k < kl;
            const bool upd = valid && cur.zq >= 1 && cur.k >= kmin;
            const bool from_ring = tx == 0 && cur.k > 0;   /* then 0 <= zq < Zp */
            float rte[S], rten[S];
#pragma unroll
            for (int i = 0; i < S; ++i) rte[i] = rten[i] = HUGEV;
            if (from_ring) {
#pragma unroll
                for (int i = 0; i < S; ++i) { rte[i] = ring_r[i * zring + cur.zq]; rten[i] = ring_tn[i * zring + cur.zq]; }
            }
            float tnw[S];
            if (oy != 0) {
#pragma unroll
                for (int i = 0; i < S; ++i) tnw[i] = xrd[u][i][wy][tx];
            }
            const float s4 = fminf(zu_uu, zu_ud), s5 = fminf(zu_uu, zu_du), s6 = fminf(zu_uu, cur.duu);
            const float s1 = fminf(s4, fminf(zu_du, zu_dd));
            const float s2 = fminf(s4, fminf(cur.duu, cur.dud));
            const float s3 = fminf(s5, fminf(cur.duu, cur.ddu));
            const float s7 = zu_uu;
            float res[S], tnv_[S], te[S], ten[S];
#pragma unroll
            for (int i = 0; i < S; ++i) {
                te[i] = (tx == 0) ? rte[i] : sh_r[i];
                ten[i] = (tx == 0) ? rten[i] : sh_tn[i];
                tnv_[i] = (oy == 0) ? cur.tn[i] : tnw[i];
                res[i] = cur.told[i];
            }
            if (upd) {
                pass_stencil<S, false>(mesh, r_last, te, tnv_, te_last, ten, tn_last, ten_last, s1, s2, s3, s4, s5, s6,
                                s7, cur.told, res);
#pragma unroll
                for (int i = 0; i < S; ++i) {
                    const float r = res[i], told = cur.told[i];
                    if (r != told && (i == 0 || has2)) {
                        (i == 0 ? ttp[0] : ttp[S - 1])[cur.it] = r;
                        if (RESID) {
                            const double d = fabs((double)r - (double)told);
                            dmax[i] = d > dmax[i] ? d : dmax[i];
                        }
                    }
                }
            }
#pragma unroll
            for (int i = 0; i < S; ++i) {
                te_last[i] = te[i];
                ten_last[i] = ten[i];
            }
#pragma unroll
            for (int i = 0; i < S; ++i) {
                xw[u][i][ty][tx] = res[i];
                if (tx == 31 && cur.zq >= 0) { ring_r[i * zring + cur.zq] = res[i]; ring_tn[i * zring + cur.zq] = tnv_[i]; }
            }
#pragma unroll
            for (int i = 0; i < S; ++i) {
                r_last[i] = res[i];
                tn_last[i] = tnv_[i];
            }
            zu_uu = cur.duu; zu_ud = cur.dud; zu_du = cur.ddu; zu_dd = cur.ddd;
            if (u < DL - 1) __syncwarp();   /* lane 31 -> lane 0 ring */
        }
        __syncthreads();                    /* the window's row values become visible */
        if (threadIdx.x == 0 && (t0 + DL) % CH == 0 && t0 + DL < T) {
            __threadfence();
#pragma unroll
            for (int i = 0; i < S; ++i)
                if (prog[i]) fk3tw::st_release(prog[i] + P, (s << SHIFT) | (t0 + DL));
        }
    }
    return true;
}

/* ---- staged FP32 pass step ---------------------------------------------
 * The walk of slab_pass_f32 with the lane's own node values and slowness
 * moved in 16-byte groups of 4 consecutive z positions by cp.async into a
 * per-warp shared-memory stage, instead of one 4-byte L2 load per value and
 * step (each of which fetches a whole 32-byte sector).
 *
 * Groups follow the walk: items 4 G .. 4 G + 3 of the lane's linear walk
 * j = k Zp + zq.  Zp is a multiple of 4, and descending sweeps start with
 * zoff = (-nz) mod 4 dummy items, so a group is always 4 consecutive nodes
 * iz = 4 m .. 4 m + 3 of one column: a 16-byte aligned block of the field
 * ([ny][nx][zp], zp a multiple of 8) and of the node-indexed slowness copies
 * (fk_grid3d_t.slowz).  The dummy items and the walk positions past nz are
 * invalid items, as in slab_pass_f32.
 *
 * Loads are warp-uniform: every 4 steps all 32 lanes issue one group each,
 * two groups ahead of the one they read next (the lanes' walks are skewed by
 * one item, so their groups start at different steps), after waiting for
 * the batch issued 4 steps before; a lane reads an item from the stage one
 * step before using it.  A group lives in buffer G mod 3: the two groups a
 * lane reads in the next 4 steps and the one in flight.  Stage per warp:
 * [3 buffers][4 arrays: told per source, the x-upwind slowness cells of
 * the two y sides][32 slots][4 floats] (6 KB); lane l's slot is
 * (l >> 2) | ((l & 3) << 3), so the 32 lanes read 32 different banks in
 * every step.  The x-downwind slowness cells of a lane are lane l + 1's
 * x-upwind ones (its next item is this lane's current one): only lane 31
 * stages its own, in a small area after the arrays.  The slab's first row stages
 * its y-upwind values (the upwind slab's last row, final for this sweep)
 * the same way, in a per-block stage [3 buffers][S][32 slots][4 floats];
 * its groups reach SG_AHEAD steps past the batch's step, so the first row
 * waits for the upwind slab to be that much further ahead than a direct
 * load one step ahead would need. */
constexpr int SG_NARR = 4;             /* told per source, the x-upwind slowness cells (y U, D) */
constexpr int SG_NBUF = 3;
constexpr int SG_ARR_BYTES = 32 * 16;
/* lane 31's x-downwind cells (y U, D): [3 buffers][2][4 floats] after the arrays */
constexpr int SG_X31_OFF = SG_NBUF * SG_NARR * SG_ARR_BYTES;
/* 6.1 KB: with the rings and the first row's stage, five blocks of the
 * two-source staged step fit an SM (registers capped at 102 by the launch
 * bounds; 95 used): 46.9 ms on 64 sources x 4 grids against 47.4 ms with
 * the 9 KB stage (six arrays, lane 31's cells among them) at four */
constexpr int SG_WARP_BYTES = SG_X31_OFF + 128;
/* the slab's first row also stages its y-upwind values (the upwind slab's
 * last row): [3 buffers][S sources][32 slots][4 floats] per block */
template <int S> constexpr int sg_tn_bytes() { return SG_NBUF * S * SG_ARR_BYTES; }
/* items a load batch reaches past its step: the upwind slab must be this
 * far ahead of the first row (wait target t0 + CH + DLP (TY - 1) + SG_AHEAD) */
constexpr int SG_AHEAD = 11;

__device__ __forceinline__ void cpa16(uint32_t saddr, const void *gptr)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(saddr), "l"(gptr) : "memory");
}
__device__ __forceinline__ void cpa_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cpa_wait0() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

template <bool INIT, bool RESID, int S, int CHP>
__device__ __forceinline__ bool slab_pass_f32_staged(const fk3tw::Params &P_, const fk_grid3d_t &g,
                                                     float *const (&ttp)[S], int s, int sweep_no, int P,
                                                     int nslab, int *const (&prog)[S], float (*xr)[S][TY][32],
                                                     float *ring, int zring, int *s_flag, double (&dmax)[S],
                                                     uint32_t stage, const float *stage_f, uint32_t stage_tn,
                                                     const float *stage_tn_f, const Src &q0)
{
    static_assert(!INIT || (S == 1 && !RESID), "initialisation sweeps: one source per thread");
    constexpr int CH = INIT ? CH_INIT_STG : CHP;
    static_assert(CH % DLP == 0 && NBP == 2 * DLP, "windows and progress align");
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    const unsigned FULL = 0xffffffffu;
    const int nz = g.nz, nx = g.nx, ny = g.ny, zp = g.zp;
    const int s0 = sweep_no - 1;
    const int sz = (s0 < 4) ? 1 : -1;
    const int sx = (s0 % 2 == 0) ? 1 : -1;
    const int sy = ((s0 / 2) % 2 == 0) ? 1 : -1;
    /* the walk's box (solver3D.F90:493-565 in the initialisation sweeps,
     * logical positions from 1 in the passes) */
    const int lozb = INIT ? ((sz > 0) ? max(1, q0.zsi - 1) : max(1, nz - q0.zsi - 1)) : 1;
    const int loxb = INIT ? ((sx > 0) ? max(1, q0.xsi - 1) : max(1, nx - q0.xsi - 1)) : 1;
    const int loyb = INIT ? ((sy > 0) ? max(1, q0.ysi - 1) : max(1, ny - q0.ysi - 1)) : 1;
    Mesh<float> mesh;
    fk3::make_mesh<float>(mesh, g.dz, g.dx, g.dy);
    const float eps_r = (float)q0.eps_t;
    const float HUGEV = (float)FK_HUGE;
    const int th = min(TY, ny - TY * P);
    const bool row = ty < th;
    const int y = TY * P + ty;
    const int oy = (sy > 0) ? ty : th - 1 - ty;
    const int yl = (sy > 0) ? y : ny - 1 - y;
    const bool rowupd = row && yl >= loyb;
    const int wy = ty - sy;
    const int zoff = (sz > 0) ? 0 : ((4 - (nz & 3)) & 3);   /* leading dummy items */
    const int Zn = nz + zoff;                               /* items zoff .. Zn - 1 are the nodes */
    const int Zp = ((max(Zn, 32) + 3) >> 2) << 2;
    const int K = (nx + 31) / 32;
    const int k0 = (loxb - 1) / 32;                         /* blocks before x' = lox - 1: not walked */
    const int T = (K - k0) * Zp + 31 + DLP * (TY - 1);
    const int Pu = P - sy;
    const bool has_up = Pu >= 0 && Pu < nslab;
    const int ylast_up = has_up ? ((sy > 0) ? TY * Pu + min(TY, ny - TY * Pu) - 1 : TY * Pu) : 0;
    const bool wait_up = has_up && (((sy > 0) ? ylast_up : ny - 1 - ylast_up) >= loyb);
    const int yu = y - sy;
    const bool has_yu = row && yu >= 0 && yu < ny;
    const bool has2 = S == 2 && ttp[S - 1] != nullptr;
    float *const tt0 = ttp[0];
    float *const tt1 = has2 ? ttp[S - 1] : ttp[0];

    const int x0 = (sx > 0) ? tx : nx - 1 - tx;
    const int kl = row ? (nx - tx + 31) / 32 : 0;                  /* blocks with x' < nx */
    /* updated: x' >= lox (1 in the passes), y' >= loy */
    const int kmin = rowupd ? (loxb > tx ? (loxb - tx + 31) >> 5 : 0) : 0x7fffffff;
    const int kxl = (nx - 1 >= tx && (nx - 1 - tx) % 32 == 0) ? (nx - 1 - tx) / 32 : -1; /* x' = nx - 1 */
    /* node iz of walk position zq: sz > 0: zq; sz < 0: nz - 1 + zoff - zq */
    const int colT = (y * nx + x0) * zp;
    const int dkT = 32 * sx * zp;
    const int dyT = sy * nx * zp;
    const int izw = (sz > 0) ? 0 : nz - 1 + zoff;                  /* iz = izw + sz zq */
    const int cyU = (sy > 0) ? y - 1 : y;
    const int cyD = min(max((sy > 0) ? y : y - 1, 0), ny - 2);
    const float *const sl = g.slowz + ((sz > 0) ? (size_t)0 : (size_t)(ny - 1) * (nx - 1) * zp);
    const int colS = (cyU * (nx - 1) + x0 - (sx > 0 ? 1 : 0)) * zp;
    const int dkS = 32 * sx * zp;
    const int offY = (cyD - cyU) * (nx - 1) * zp;
    const int offX = sx * zp;
    const int slot = (tx >> 2) | ((tx & 3) << 3);
    const uint32_t my = stage + (uint32_t)(slot * 16);   /* cp.async destination */
    const float *const myf = stage_f + slot * 4;          /* the same bytes, for reading */
    const bool load_tn = oy == 0 && has_yu;               /* first row: stage the upwind slab's last row */
    const uint32_t myt = stage_tn + (uint32_t)(slot * 16);
    const float *const mytf = stage_tn_f + slot * 4;
    const uint32_t x31 = stage + (uint32_t)SG_X31_OFF;
    const float *const x31f = stage_f + SG_X31_OFF / 4;
    constexpr int A = SG_ARR_BYTES / 4;                   /* floats per array */
    constexpr int BUFF = SG_NARR * A;                     /* floats per buffer */
    static_assert(BUFF == 512 && S * A * 4 == S * BUFF, "the cursor's shifts below assume 4 arrays of 128 floats");
    const bool loads_slow = rowupd;                       /* a row that updates reads slowness */

    const int c = tx + DLP * oy;                 /* the lane's item at step t is t - c */
    /* group loads: batch b (step 4 b) issues group G_b = ((4 b + 1 - c) >> 2) + 2, i.e. two groups
     * past the one holding item 4 b + 1 - c, the first read after the batch; G_{b+1} = G_b + 1.
     * Cursor (lk, lzq) = (column block, walk position) of the group's first item. */
    int gl = ((1 - 8 - c) >> 2) + 2;            /* G_{-2}: the prologue issues G_{-2}, G_{-1} */
    int lk = k0, lzq = 4 * gl;
    while (lzq >= Zp) { lzq -= Zp; ++lk; }
    auto issue = [&]() {
        const int buf = (gl + 3 * 0x2000000) % 3;
        const uint32_t d = my + (uint32_t)(buf * (SG_NARR * SG_ARR_BYTES));
        if (lzq >= 0 && lzq < Zn && lk < kl) {
            const int izb = (sz > 0) ? lzq : nz + zoff - 4 - lzq;
            const int it = colT + lk * dkT + izb;
            cpa16(d, tt0 + it);
            if (S == 2) cpa16(d + SG_ARR_BYTES, tt1 + it);
            if (load_tn) {
                const uint32_t dt = myt + (uint32_t)(buf * (S * SG_ARR_BYTES));
                cpa16(dt, tt0 + (it - dyT));
                if (S == 2) cpa16(dt + SG_ARR_BYTES, tt1 + (it - dyT));
            }
            if (loads_slow && lk >= kmin) {
                const int is = colS + lk * dkS + izb;
                const int ox = (lk == kxl) ? 0 : offX;
                cpa16(d + 2 * SG_ARR_BYTES, sl + is);
                cpa16(d + 3 * SG_ARR_BYTES, sl + (is + offY));
                if (tx == 31) {   /* the other lanes take their x-downwind cells from lane l + 1 */
                    cpa16(x31 + (uint32_t)(buf * 32), sl + (is + ox));
                    cpa16(x31 + (uint32_t)(buf * 32 + 16), sl + (is + ox + offY));
                }
            }
        }
        cpa_commit();
        ++gl;
        lzq += 4;
        if (lzq >= Zp) { lzq -= Zp; ++lk; }
    };

    struct Item {
        float told[S], tn[S];
        float duu, dud, ddu, ddd;
        int k, zq;
    };
    /* read cursor: the next item jr of the walk, its group's buffer (as a
     * float offset rb = (jr / 4 mod 3) BUFF) and its place eo in the group,
     * advanced one item per step */
    int jr = -c;
    int rb = (((jr >> 2) + 3 * 0x2000000) % 3) * BUFF;
    int eo = (sz > 0) ? (jr & 3) : 3 - (jr & 3);
    auto advance = [&]() {
        ++jr;
        if ((jr & 3) == 0) {
            rb = (rb == 2 * BUFF) ? 0 : rb + BUFF;
            eo = (sz > 0) ? 0 : 3;
        } else {
            eo += sz;
        }
    };
    /* item jr = (kk, zz) of the walk from the stage (its group is resident) */
    auto fetch = [&](Item &f, int kk, int zz) {
        f.k = kk;
        f.zq = zz;
        if (jr >= 0) {
            const float *a = myf + rb + eo;
            f.told[0] = a[0];
            if (S == 2) f.told[S - 1] = a[A];
            f.duu = a[2 * A];
            f.dud = a[3 * A];
            f.ddu = x31f[(rb >> 6) + eo];       /* lane 31's (the others' are not used) */
            f.ddd = x31f[(rb >> 6) + 4 + eo];
            if (oy == 0) {   /* the upwind slab's last row, final for this sweep (invalid items: any value) */
                const float *b = mytf + ((rb * S) >> 2) + eo;
                f.tn[0] = has_yu ? b[0] : HUGEV;
                if (S == 2) f.tn[S - 1] = has_yu ? b[A] : HUGEV;
            }
        }
        advance();
    };

    const int *prog_up = prog[0] + (has_up ? Pu : P);
    if (threadIdx.x == 0) {
        s_flag[0] = 1;
        if (wait_up && !wait_ge1(prog_up, (s << SHIFT) | min(T, CH + DLP * (TY - 1) + SG_AHEAD), P_.spin_limit, P_.error,
                                 3000))
            s_flag[0] = 0;
    }
    __syncthreads();
    if (!s_flag[0]) return false;

    issue();                                    /* G_{-2} */
    issue();                                    /* G_{-1} */
    cpa_wait0();
    int nk = k0, nzq = -c;                      /* item of the next step */
    Item nxt;
#pragma unroll
    for (int i = 0; i < S; ++i) nxt.told[i] = nxt.tn[i] = HUGEV;
    nxt.duu = nxt.dud = nxt.ddu = nxt.ddd = 0.0f;
    fetch(nxt, nk, nzq);
    if (++nzq == Zp) { nzq = 0; ++nk; }
    float zu_uu = 0.0f, zu_ud = 0.0f, zu_du = 0.0f, zu_dd = 0.0f;
    float r_last[S], te_last[S], tn_last[S], ten_last[S];
#pragma unroll
    for (int i = 0; i < S; ++i) r_last[i] = te_last[i] = tn_last[i] = ten_last[i] = HUGEV;
    float *ring_r = ring, *ring_tn = ring + S * zring;
    bool ok = true;
    for (int t0 = 0; t0 < T; t0 += DLP) {
        if (wait_up && t0 > 0 && t0 % CH == 0) {
            if (threadIdx.x == 0 &&
                !wait_ge1(prog_up, (s << SHIFT) | min(T, t0 + CH + DLP * (TY - 1) + SG_AHEAD), P_.spin_limit,
                          P_.error, 3001))
                s_flag[0] = 0;
            __syncthreads();
            if (!s_flag[0]) { ok = false; break; }
        }
        const int half = (t0 / DLP) & 1;
        float (*const xw)[S][TY][32] = xr + half * DLP;
        float (*const xrd)[S][TY][32] = xr + (1 - half) * DLP;
#pragma unroll
        for (int u = 0; u < DLP; ++u) {
            if (((t0 + u) & 3) == 0) {          /* load batch every 4 steps: warp-uniform */
                cpa_wait0();                    /* the batch of 4 steps ago has landed */
                issue();
            }
            float sh_r[S], sh_tn[S];
#pragma unroll
            for (int i = 0; i < S; ++i) {
                sh_r[i] = __shfl_up_sync(FULL, r_last[i], 1);
                sh_tn[i] = __shfl_up_sync(FULL, tn_last[i], 1);
            }
            const Item cur = nxt;
            fetch(nxt, nk, nzq);
            if (++nzq == Zp) { nzq = 0; ++nk; }
            /* x-downwind cells: lane l + 1's x-upwind ones, its next item being
             * this lane's current one; lane 31 stages its own, and the last
             * column (zero x offset) repeats its x-upwind cells */
            const float dn_uu = __shfl_down_sync(FULL, nxt.duu, 1), dn_ud = __shfl_down_sync(FULL, nxt.dud, 1);
            const float c_ddu = (tx == 31) ? cur.ddu : (cur.k == kxl) ? cur.duu : dn_uu;
            const float c_ddd = (tx == 31) ? cur.ddd : (cur.k == kxl) ? cur.dud : dn_ud;
            const bool valid = (unsigned)(cur.zq - zoff) < (unsigned)nz && cur.k < kl;
            const bool upd = valid && cur.zq >= zoff + lozb && cur.k >= kmin;
            const bool from_ring = tx == 0 && cur.k > k0;   /* then 0 <= zq < Zp */
            float rte[S], rten[S];
#pragma unroll
            for (int i = 0; i < S; ++i) rte[i] = rten[i] = HUGEV;
            if (from_ring) {
#pragma unroll
                for (int i = 0; i < S; ++i) { rte[i] = ring_r[i * zring + cur.zq]; rten[i] = ring_tn[i * zring + cur.zq]; }
            }
            float tnw[S];
            if (oy != 0) {
#pragma unroll
                for (int i = 0; i < S; ++i) tnw[i] = xrd[u][i][wy][tx];
            }
            const float s4 = fminf(zu_uu, zu_ud), s5 = fminf(zu_uu, zu_du), s6 = fminf(zu_uu, cur.duu);
            const float s1 = fminf(s4, fminf(zu_du, zu_dd));
            const float s2 = fminf(s4, fminf(cur.duu, cur.dud));
            const float s3 = fminf(s5, fminf(cur.duu, c_ddu));
            const float s7 = zu_uu;
            float res[S], tnv_[S], te[S], ten[S];
#pragma unroll
            for (int i = 0; i < S; ++i) {
                te[i] = (tx == 0) ? rte[i] : sh_r[i];
                ten[i] = (tx == 0) ? rten[i] : sh_tn[i];
                tnv_[i] = (oy == 0) ? cur.tn[i] : tnw[i];
                res[i] = cur.told[i];
            }
            if (upd) {
                if constexpr (INIT) {
                    /* as in slab_sweep: the plane-wave stencil where the switch
                     * (compared in FP32) says Cartesian, else the FP64
                     * spherical one near the source */
                    const float tv = r_last[0], tn = tnv_[0];
                    if (rmin(rmin(tv, te[0]), tn) > eps_r) {
                        res[0] = fk3::noinit_f32(mesh, tv, te[0], tn, te_last[0], ten[0], tn_last[0], ten_last[0], s1,
                                                 s2, s3, s4, s5, s6, s7, cur.told[0]);
                    } else {
                        const int xl = 32 * cur.k + tx;
                        const int x = (sx > 0) ? xl : nx - 1 - xl;
                        const int iz = izw + sz * cur.zq;
                        Mesh<double> mesh64;   /* built here: few nodes take this branch */
                        fk3::make_mesh<double>(mesh64, g.dz, g.dx, g.dy);
                        res[0] = (float)fk3::init_node<double>(
                            q0, mesh64, false, (double)tv, (double)te[0], (double)tn, (double)te_last[0],
                            (double)ten[0], (double)tn_last[0], (double)ten_last[0], (double)cur.told[0], (double)s1,
                            (double)s2, (double)s3, (double)s4, (double)s5, (double)s6, (double)s7, iz + 1, x + 1,
                            y + 1, sz, sx, sy);
                    }
                } else {
                    pass_stencil<S, true>(mesh, r_last, te, tnv_, te_last, ten, tn_last, ten_last, s1, s2, s3, s4, s5,
                                          s6, s7, cur.told, res);
                }
                const int it = colT + cur.k * dkT + izw + sz * cur.zq;
#pragma unroll
                for (int i = 0; i < S; ++i) {
                    const float r = res[i], told = cur.told[i];
                    if (r != told && (i == 0 || has2)) {
                        (i == 0 ? tt0 : tt1)[it] = r;
                        if (RESID) {
                            const double d = fabs((double)r - (double)told);
                            dmax[i] = d > dmax[i] ? d : dmax[i];
                        }
                    }
                }
            }
#pragma unroll
            for (int i = 0; i < S; ++i) {
                te_last[i] = te[i];
                ten_last[i] = ten[i];
            }
#pragma unroll
            for (int i = 0; i < S; ++i) {
                xw[u][i][ty][tx] = res[i];
                if (tx == 31 && cur.zq >= 0) { ring_r[i * zring + cur.zq] = res[i]; ring_tn[i * zring + cur.zq] = tnv_[i]; }
            }
#pragma unroll
            for (int i = 0; i < S; ++i) {
                r_last[i] = res[i];
                tn_last[i] = tnv_[i];
            }
            zu_uu = cur.duu; zu_ud = cur.dud; zu_du = c_ddu; zu_dd = c_ddd;
            if (u < DLP - 1) __syncwarp();
        }
        /* (row-pair named barriers instead of the block barrier measured 2 %
         * slower: fewer barrier stalls, more dependency stalls) */
        __syncthreads();
        if (threadIdx.x == 0 && (t0 + DLP) % CH == 0 && t0 + DLP < T) {
            __threadfence();
#pragma unroll
            for (int i = 0; i < S; ++i)
                if (prog[i]) fk3tw::st_release(prog[i] + P, (s << SHIFT) | (t0 + DLP));
        }
    }
    cpa_wait0();   /* no copy into the stage outlives the task */
    return ok;
}

/* Persistent slab-task kernel over sweeps [s_begin, s_end).  S = 2 runs
 * two sources of one grid in the same threads (the Gauss-Seidel passes,
 * whose walk does not depend on the source): the slowness, the indices and
 * the barriers are shared and the two stencils give each thread two
 * independent dependency chains.  tasks = {pair, j'} with pairs[2 pair + i]
 * the work items (-1: none) when S = 2, {work, j'} when S = 1. */
template <typename R, bool INIT, bool RESID, int S, int CHP, bool STG = false>
__global__ void __launch_bounds__(NT, INIT ? 4 : (S == 1 ? 6 : (STG ? 5 : 4))) slab_kernel(fk3tw::Params P, const int *pairs,
                                                                             int zring)
{
    __shared__ R xr[(sizeof(R) == 4 && STG) ? NBP : NB][S][TY][32];
    __shared__ long long s_task;
    __shared__ int s_flag[2];
    __shared__ double s_max[S][TY];
    extern __shared__ __align__(16) unsigned char slab_smem[];
    R *ring = reinterpret_cast<R *>(slab_smem) + (size_t)(threadIdx.x >> 5) * 2 * S * zring;
    /* staged pass step: the per-warp stages follow the rings (16-byte aligned: zring is a multiple of 4) */
    const size_t stage_off = (size_t)TY * 2 * S * zring * sizeof(R) + (size_t)(threadIdx.x >> 5) * SG_WARP_BYTES;
    const uint32_t stage = (uint32_t)__cvta_generic_to_shared(slab_smem) + (uint32_t)stage_off;
    const float *const stage_f = reinterpret_cast<const float *>(slab_smem + stage_off);
    const size_t stage_tn_off = (size_t)TY * 2 * S * zring * sizeof(R) + (size_t)TY * SG_WARP_BYTES;
    const uint32_t stage_tn = (uint32_t)__cvta_generic_to_shared(slab_smem) + (uint32_t)stage_tn_off;
    const float *const stage_tn_f = reinterpret_cast<const float *>(slab_smem + stage_tn_off);
    const int tid = threadIdx.x;
    const long long total = (long long)(P.s_end - P.s_begin) * P.ntask_sweep;
    for (;;) {
        if (tid == 0) {
            long long t = (long long)atomicAdd(P.ticket, 1ull);
            if (t >= total || *((volatile int *)P.error) != 0) t = -1;
            s_task = t;
            s_flag[1] = 1;
        }
        __syncthreads();
        const long long t = s_task;
        if (t < 0) break;
        const int s = P.s_begin + (int)(t / P.ntask_sweep);
        const int2 tk = P.tasks[t % P.ntask_sweep];
        int wi[S];
        if (S == 1) wi[0] = tk.x;
        else {
#pragma unroll
            for (int i = 0; i < S; ++i) wi[i] = pairs[S * tk.x + i];
        }
        const fk_work3d_t w0 = P.work[wi[0]];
        const fk_grid3d_t g = P.grids[w0.grid];
        const int nslab = (g.ny + TY - 1) / TY;
        const int sweep_no = s % 8 + 1;
        const int s0 = sweep_no - 1;
        const int sy = ((s0 / 2) % 2 == 0) ? 1 : -1;
        /* initialisation, one source per thread (P.done_t set): task {w, -1}
         * walks the sweep of a box at most TY z positions deep with the axes
         * turned, and then the slab tasks of that sweep have nothing to do */
        const bool turned_task = INIT && S == 1 && P.done_t != nullptr && tk.y < 0;
        const int Pp = turned_task ? 0 : (sy > 0) ? tk.y : nslab - 1 - tk.y;   /* physical slab */
        int *prog[S];
        R *ttp[S];
#pragma unroll
        for (int i = 0; i < S; ++i) {
            prog[i] = wi[i] >= 0 ? P.done + P.done_base[wi[i]] : nullptr;
            ttp[i] = wi[i] >= 0 ? reinterpret_cast<R *>(i == 0 ? w0.tt : P.work[wi[i]].tt) : nullptr;
        }
        /* done with the previous sweep: slabs P-1, P, P+1 of every source,
         * and the turned-axes task of the source; a turned-axes task waits for
         * every slab of its source and its own previous task (all of them
         * hold smaller tickets, so the waits cannot cycle) */
        {
            auto wait_done = [&](const int *c) {   /* bounded acquire wait for (sweep s - 1) done */
                long long it = 0;
                unsigned ns = 64;
                while (fk3tw::ld_acquire(c) < (s << SHIFT)) {
                    if (++it > P.spin_limit) {
                        atomicCAS(P.error, 0, 2000 + tid);
                        s_flag[1] = 0;
                        return false;
                    }
                    poll_backoff(ns);
                }
                return true;
            };
            if (!turned_task) {
                if (tid < 3 * S) {
                    const int i = tid / 3, pq = Pp + tid % 3 - 1;
                    if (prog[i] && pq >= 0 && pq < nslab) wait_done(prog[i] + pq);
                } else if (tid == 3 * S && INIT && S == 1 && P.done_t != nullptr) {
                    wait_done(P.done_t + wi[0]);
                }
            } else {
                /* every slab q of the source (q = tid, tid + NT, ...), and q = nslab its previous turned task */
                for (int q = tid; q <= nslab; q += NT)
                    if (!wait_done(q < nslab ? prog[0] + q : P.done_t + wi[0])) break;
            }
        }
        __syncthreads();
        if (!s_flag[1]) break;
        __threadfence();
        const int pass = INIT ? -1 : (s - 8) / 8;
        bool skip = false;
        if (!INIT && P.converge) {
            skip = true;
#pragma unroll
            for (int i = 0; i < S; ++i)
                if (wi[i] >= 0) skip = skip && *((volatile int *)(P.conv_pass + wi[i])) < pass;
        }
        Src qs[S];
#pragma unroll
        for (int i = 0; i < S; ++i) fk3tw::tw_setup_src(qs[i], i == 0 ? w0 : P.work[wi[i] >= 0 ? wi[i] : wi[0]], g, P.eps);
        const bool thin = INIT && S == 1 && P.done_t != nullptr && init_box_depth(qs[0], g.nz, sweep_no) <= TY;
        if (INIT) {
            /* slabs wholly before every source's rows of this sweep keep their values */
            const int ylast = (sy > 0) ? min(g.ny, TY * (Pp + 1)) - 1 : TY * Pp;
            const int yl_max = (sy > 0) ? ylast : g.ny - 1 - ylast;
            skip = true;
#pragma unroll
            for (int i = 0; i < S; ++i) {
                const int loy = (sy > 0) ? max(1, qs[i].ysi - 1) : max(1, g.ny - qs[i].ysi - 1);
                if (wi[i] >= 0 && yl_max >= loy) skip = false;
            }
            /* a thin box is the turned-axes task's alone */
            if (turned_task) skip = !thin;
            else if (thin) skip = true;
        }
        double dmax[S];
#pragma unroll
        for (int i = 0; i < S; ++i) dmax[i] = 0.0;
        if (!skip && turned_task) {
            if constexpr (INIT && S == 1)
                slab_sweep_zrows<R>(g, ttp[0], reinterpret_cast<const R *>(g.slow), qs[0], sweep_no,
                                    reinterpret_cast<R (*)[1][TY][32]>(xr), ring, zring);
        } else if (!skip) {
            bool ok;
            if constexpr (sizeof(R) == 4 && STG && (!INIT || S == 1))
                ok = slab_pass_f32_staged<INIT, RESID, S, CHP>(P, g, ttp, s, sweep_no, Pp, nslab, prog, xr, ring,
                                                               zring, s_flag, dmax, stage, stage_f, stage_tn,
                                                               stage_tn_f, qs[0]);
            else if constexpr (!INIT && sizeof(R) == 4)
                ok = slab_pass_f32<RESID, S, CHP>(P, g, ttp, reinterpret_cast<const float *>(g.slow), s, sweep_no,
                                                  Pp, nslab, prog, xr, ring, zring, s_flag, dmax);
            else
                ok = slab_sweep<R, INIT, RESID, S, CHP>(P, g, ttp, reinterpret_cast<const R *>(g.slow), qs, s,
                                                        sweep_no, Pp, nslab, prog, xr, ring, zring, s_flag, dmax);
            if (!ok) break;
        }
        __syncthreads();
        if (RESID && !INIT) {
#pragma unroll
            for (int i = 0; i < S; ++i) {
                double d = dmax[i];
                for (int o = 16; o > 0; o >>= 1) {
                    const double v = __shfl_xor_sync(0xffffffffu, d, o);
                    d = v > d ? v : d;
                }
                if ((tid & 31) == 0) s_max[i][tid >> 5] = d;
            }
            __syncthreads();
        }
        if (tid == 0) {
            __threadfence();
#pragma unroll
            for (int i = 0; i < S; ++i) {
                if (wi[i] < 0) continue;
                if (RESID && !INIT && pass < P.npass) {
                    double m = 0.0;
                    for (int k = 0; k < TY; ++k) m = s_max[i][k] > m ? s_max[i][k] : m;
                    unsigned long long *rp = P.resid + (size_t)wi[i] * P.npass + pass;
                    atomicMax(rp, (unsigned long long)__double_as_longlong(m));
                    if (sweep_no == 8) {
                        __threadfence();
                        const int c = atomicAdd(P.pass_slabs + (size_t)wi[i] * P.npass + pass, 1);
                        if (c == nslab - 1) {
                            const double r = __longlong_as_double((long long)atomicAdd(rp, 0ull));
                            if (P.converge && r <= P.conv_tol) atomicMin(P.conv_pass + wi[i], pass);
                        }
                    }
                }
                fk3tw::st_release(turned_task ? P.done_t + wi[i] : prog[i] + Pp, (s + 1) << SHIFT);
            }
        }
    }
}

template <typename R, bool INIT, bool RESID, int S, bool STG = false>
inline int launch_slab_kernel(const fk3tw::Params &P, const int *pairs, int zring, cudaStream_t st,
                              int progress = 0, int blocks_per_sm = 0)
{
    const size_t smem = (size_t)TY * 2 * S * zring * sizeof(R) +
                        (STG ? (size_t)TY * SG_WARP_BYTES + (size_t)sg_tn_bytes<S>() : 0);
    int dev = 0, nsm = 0, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    /* deep grids: the per-warp rings (and the stage) need the opt-in shared
     * memory once they and the kernel's static arrays pass the default 48 KB */
    cudaFuncAttributes fa;
    if (cudaFuncGetAttributes(&fa, slab_kernel<R, INIT, RESID, S, CH_MANY, STG>) != cudaSuccess)
        return (int)cudaGetLastError();
    if (smem + fa.sharedSizeBytes > 48 * 1024) {
        cudaError_t ea = cudaFuncSetAttribute(slab_kernel<R, INIT, RESID, S, CH_MANY, STG>,
                                              cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (ea == cudaSuccess && !INIT)
            ea = cudaFuncSetAttribute(slab_kernel<R, INIT, RESID, S, CH_FEW, STG>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (ea != cudaSuccess) return (int)ea;
    }
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, slab_kernel<R, INIT, RESID, S, CH_MANY, STG>, NT, smem);
    if (per < 1) per = 1;
    if (blocks_per_sm > 0 && blocks_per_sm < per) per = blocks_per_sm;
    /* fewer than 4 slab tasks per resident block and sweep: the upwind chains bound the time */
    const bool few = progress == CH_FEW || (progress == 0 && P.ntask_sweep < 4 * nsm * per);
    if (!INIT && few)
        slab_kernel<R, INIT, RESID, S, CH_FEW, STG><<<nsm * per, NT, smem, st>>>(P, pairs, zring);
    else
        slab_kernel<R, INIT, RESID, S, CH_MANY, STG><<<nsm * per, NT, smem, st>>>(P, pairs, zring);
    return (int)cudaGetLastError();
}

/* The FP32 initialisation kernel lives in its own unit (slab_init_f32.cu),
 * compiled without multiply-add contraction: its near-source spherical
 * stencil is FP64 and so rounds as the FP64 CPU algorithm does. */
int launch_init_f32(const fk3tw::Params &P, int zring, cudaStream_t st, int blocks_per_sm, const int *pairs,
                    bool staged);

template <typename R>
inline int launch_rows(const fk_grid3d_t *grids, const fk_work3d_t *work, int nwork, const fk_slabs3d_t *pl,
                       fk_result3d_t *results, double eps, int nsweep, double conv_tol, int max_pass,
                       cudaStream_t st)
{
    if (nwork <= 0) return 0;
    const int converge = conv_tol >= 0.0 && max_pass > 0;
    const int npass = converge ? max_pass : nsweep;
    const int npr = npass > 0 ? npass : 1;
    /* walk positions per column: nz, plus up to 3 leading items in the staged
     * step's descending sweeps, at least 32, a multiple of 4 */
    const int zring = ((pl->max_nz + 3 > 32 ? pl->max_nz + 3 : 32) + 3) / 4 * 4;
    /* counters hold (sweep << SHIFT) | steps: steps of a slab and sweep numbers must fit */
    const int zr = zring > pl->max_ny ? zring : pl->max_ny;   /* the turned-axes walk runs along y */
    const long long steps = (long long)((pl->max_nx + 31) / 32) * (zr + 3) + 31 + (DL > DLP ? DL : DLP) * TY;
    if (steps >= (1LL << SHIFT) || 8 + 8 * (long long)npr + 1 >= (1LL << (31 - SHIFT)))
        return (int)cudaErrorInvalidValue;
    cudaError_t e = cudaSuccess;
    e = cudaMemsetAsync(pl->done, 0, sizeof(int) * (size_t)pl->nslab_total, st);
    if (!e) e = cudaMemsetAsync(pl->tickets, 0, 2 * sizeof(unsigned long long), st);
    if (!e) e = cudaMemsetAsync(pl->error, 0, sizeof(int), st);
    if (!e) e = cudaMemsetAsync(pl->resid, 0, sizeof(unsigned long long) * (size_t)nwork * npr, st);
    if (!e) e = cudaMemsetAsync(pl->pass_slabs, 0, sizeof(int) * (size_t)nwork * npr, st);
    if (!e) e = cudaMemsetAsync(pl->conv_pass, 0x3f, sizeof(int) * (size_t)nwork, st);
    if (!e) e = cudaMemsetAsync(pl->done_t, 0, sizeof(int) * (size_t)nwork, st);
    if (e) return (int)e;
    fk3tw::field_init_kernel<R><<<dim3(64, nwork), 256, 0, st>>>(grids, work, eps);
    fk3tw::corners_kernel<R><<<(nwork * 8 + 127) / 128, 128, 0, st>>>(grids, work, nwork, eps);
    fk3tw::Params P;
    P.grids = grids;
    P.work = work;
    P.tasks = reinterpret_cast<const int2 *>(pl->tasks);
    P.done_base = pl->done_base;
    P.ntask_sweep = pl->ntask_sweep;
    P.done = pl->done;
    P.done_t = nullptr;
    P.error = pl->error;
    P.resid = pl->resid;
    P.pass_slabs = pl->pass_slabs;
    P.conv_pass = pl->conv_pass;
    P.npass = npr;
    P.converge = converge;
    P.eps = eps;
    P.conv_tol = conv_tol;
    P.spin_limit = pl->spin_limit;
    P.s_begin = 0;
    P.s_end = 8;
    P.ticket = pl->tickets;
    if (fk3tw::g_slab_events) cudaEventRecord(fk3tw::g_slab_events[0], st);
    /* initialisation with one source per thread: the turned-axes tasks ahead
     * of the slab tasks; their rings hold a y walk, so they are sized for
     * the deepest or widest grid */
    fk3tw::Params Pt = P;
    Pt.tasks = reinterpret_cast<const int2 *>(pl->tasks_init);
    Pt.ntask_sweep = pl->ntask_init_sweep;
    Pt.done_t = pl->done_t;
    const int zring_t = ((zring > pl->max_ny ? zring : pl->max_ny) + 3) / 4 * 4;
    int rc;
    if constexpr (sizeof(R) == 4) {
        if (pl->init_pairs) { /* two sources per thread over the union of their boxes */
            fk3tw::Params Pi = P;
            Pi.tasks = reinterpret_cast<const int2 *>(pl->tasks2);
            Pi.ntask_sweep = pl->ntask2_sweep;
            rc = launch_init_f32(Pi, zring, st, pl->init_blocks_per_sm, pl->init_pairs, false);
        } else {
            /* with the staged pass step (the node-indexed slowness built) the
             * slab tasks take the staged walk too */
            rc = launch_init_f32(Pt, zring_t, st, pl->init_blocks_per_sm, nullptr, pl->staged != 0);
        }
    }
    else
        rc = launch_slab_kernel<R, true, false, 1>(Pt, nullptr, zring_t, st, 0, pl->init_blocks_per_sm);
    if (rc) return rc;
    if (fk3tw::g_slab_events) cudaEventRecord(fk3tw::g_slab_events[1], st);
    if (npass > 0) {
        P.s_begin = 8;
        P.s_end = 8 + 8 * npass;
        P.ticket = pl->tickets + 1;
        const bool stg = sizeof(R) == 4 && pl->staged;
        if (pl->pairs) { /* two sources per thread */
            P.tasks = reinterpret_cast<const int2 *>(pl->tasks2);
            P.ntask_sweep = pl->ntask2_sweep;
            const int *pr = pl->pairs;
            const int ch = pl->progress, bps = pl->blocks_per_sm;
            if (stg)
                rc = converge ? launch_slab_kernel<R, false, true, 2, true>(P, pr, zring, st, ch, bps)
                              : launch_slab_kernel<R, false, false, 2, true>(P, pr, zring, st, ch, bps);
            else
                rc = converge ? launch_slab_kernel<R, false, true, 2>(P, pr, zring, st, ch, bps)
                              : launch_slab_kernel<R, false, false, 2>(P, pr, zring, st, ch, bps);
        } else {
            const int ch = pl->progress, bps = pl->blocks_per_sm;
            if (stg)
                rc = converge ? launch_slab_kernel<R, false, true, 1, true>(P, nullptr, zring, st, ch, bps)
                              : launch_slab_kernel<R, false, false, 1, true>(P, nullptr, zring, st, ch, bps);
            else
                rc = converge ? launch_slab_kernel<R, false, true, 1>(P, nullptr, zring, st, ch, bps)
                              : launch_slab_kernel<R, false, false, 1>(P, nullptr, zring, st, ch, bps);
        }
        if (rc) return rc;
    }
    if (fk3tw::g_slab_events) cudaEventRecord(fk3tw::g_slab_events[2], st);
    fk3tw::finalize_kernel<<<(nwork + 127) / 128, 128, 0, st>>>(nwork, npr, converge, npass, pl->resid,
                                                                 pl->conv_pass, pl->error, results);
    return (int)cudaGetLastError();
}

} // namespace fk3rw
