/*
 * rays2d.cu -- 2D ray paths in the current travel-time field, one thread per
 * ray (rays.F90:449-825).  Compiled without multiply-add contraction: the
 * FP64 arithmetic follows the reference's operation order.
 *
 * A ray is traced backwards from its end point to the source grid point
 * (source.F90:180-181) by integrating dx/ds = -grad T / u with steps of
 * ds = min(dx, dz) / 2 (rays.F90:489): Euler, midpoint or the reference's
 * RK4 (rays.F90:671-712; its k2 is evaluated at x_n + k1 and then halved),
 * the gradient bilinearly interpolated from the nodal finite differences of
 * solver2D.F90:984-1032 and divided by the slowness of the cell holding the
 * point (evalf2d, rays.F90:857-894), positions clamped into the model
 * (updatePosition2D, :813-825).  The ray stops when a step ends within
 * sqrt((dx^2 + dz^2) / 2) of the source grid point, which then becomes its
 * last point (:522-527), or fails after nx nz steps.  Along the way:
 *   tn  = sum of step length x slowness of the step's starting cell (:537);
 *   tne = the travel-time field's bilinear drop over each step (:533-535);
 *   the path split exactly at the cell boundaries each step crosses, pieces
 *   in one cell merged: the (cell, length) list that the reference's
 *   segmentation (:560-640) builds.
 * Pass 1 counts points and pieces per ray; pass 2 writes them at offsets
 * the host computed from the counts.
 */
#include <cuda_runtime.h>
#include <math.h>

#include "fteik_dev.h"

namespace fkray {

constexpr double EPS = 2.220446049250313e-16; /* EPSILON(1.d0) */

struct Grid {
    int nz, nx, zp, zcp;
    double dz, dx;
    const double *slow; /* [nx-1][zcp] */
    const double *tt;   /* [nx][zp] */
    const double *gx;   /* [nx][nz] */
    const double *gz;
};

__device__ __forceinline__ int cell_ix(double x, double d, int n)
{
    int i = (int)(x / d + 1.0);
    return i < 1 ? 1 : (i > n - 1 ? n - 1 : i);
}

/* rays.F90:969-999 */
__device__ __forceinline__ double bilinear(double x, double z, double x1, double z1, double x2, double z2,
                                           double c11, double c12, double c21, double c22)
{
    const double den = (x1 - x2) * (z1 - z2);
    const double a0 = (c11 * x2 * z2 - c12 * x2 * z1 - c21 * x1 * z2 + c22 * x1 * z1) / den;
    const double a1 = (-c11 * z2 + c12 * z1 + c21 * z2 - c22 * z1) / den;
    const double a2 = (-c11 * x2 + c12 * x2 + c21 * x1 - c22 * x1) / den;
    const double a3 = (c11 - c12 - c21 + c22) / den;
    return a0 + a1 * x + a2 * z + a3 * x * z;
}

__device__ __forceinline__ void evalf(const Grid &g, double xn, double zn, double &d1, double &d3)
{
    const int ix = cell_ix(xn, g.dx, g.nx), iz = cell_ix(zn, g.dz, g.nz);
    const double u = g.slow[(size_t)(ix - 1) * g.zcp + (iz - 1)];
    const double x1 = (double)(ix - 1) * g.dx, x2 = (double)ix * g.dx;
    const double z1 = (double)(iz - 1) * g.dz, z2 = (double)iz * g.dz;
    const size_t n11 = (size_t)(ix - 1) * g.nz + (iz - 1), n21 = (size_t)ix * g.nz + (iz - 1);
    const double dtdx = bilinear(xn, zn, x1, z1, x2, z2, g.gx[n11], g.gx[n11 + 1], g.gx[n21], g.gx[n21 + 1]);
    const double dtdz = bilinear(xn, zn, x1, z1, x2, z2, g.gz[n11], g.gz[n11 + 1], g.gz[n21], g.gz[n21 + 1]);
    d1 = -dtdx / u;
    d3 = -dtdz / u;
}

__device__ __forceinline__ void update(const Grid &g, double xn, double zn, double ds, double d1, double d3,
                                       double &x1, double &z1)
{
    double a = xn + ds * d1, b = zn + ds * d3;
    const double xmax = (double)(g.nx - 1) * g.dx - EPS, zmax = (double)(g.nz - 1) * g.dz - EPS;
    a = a > EPS ? a : EPS;
    x1 = a < xmax ? a : xmax;
    b = b > EPS ? b : EPS;
    z1 = b < zmax ? b : zmax;
}

__device__ void step(const Grid &g, int integrator, double ds, double xn, double zn, double &x1, double &z1)
{
    double d1, d3;
    if (integrator == 2) {
        double xm, zm;
        evalf(g, xn, zn, d1, d3);
        update(g, xn, zn, 0.5 * ds, d1, d3, xm, zm);
        evalf(g, xm, zm, d1, d3);
        update(g, xn, zn, ds, d1, d3, x1, z1);
    } else if (integrator == 3) {
        const double dsscal[3] = {0.5, 0.5, 1.0};
        double k[4][2], xk, zk;
        evalf(g, xn, zn, k[0][0], k[0][1]);
        k[0][0] = ds * k[0][0];
        k[0][1] = ds * k[0][1];
        update(g, xn, zn, 1.0, k[0][0], k[0][1], xk, zk);
#pragma unroll
        for (int i = 1; i < 4; i++) {
            evalf(g, xk, zk, k[i][0], k[i][1]);
            k[i][0] = ds * dsscal[i - 1] * k[i][0];
            k[i][1] = ds * dsscal[i - 1] * k[i][1];
            update(g, xn, zn, 1.0, k[i][0], k[i][1], xk, zk);
        }
        d1 = 1.0 / 6.0 * (k[0][0] + 2.0 * (k[1][0] + k[2][0]) + k[3][0]);
        d3 = 1.0 / 6.0 * (k[0][1] + 2.0 * (k[1][1] + k[2][1]) + k[3][1]);
        update(g, xn, zn, 1.0, d1, d3, x1, z1);
    } else {
        evalf(g, xn, zn, d1, d3);
        update(g, xn, zn, ds, d1, d3, x1, z1);
    }
}

/* The step (xa, za) -> (xb, zb) cut at the grid lines it crosses; each
 * piece appended to the (cell, length) list or merged into its last entry. */
template <bool STORE>
__device__ void split(const Grid &g, double xa, double za, double xb, double zb, int &ns, int &last, int *cells,
                      double *lens)
{
    const double ddx = xb - xa, ddz = zb - za;
    const double L = sqrt(ddx * ddx + ddz * ddz);
    if (!(L > 0.0)) return;
    double tx[8], tz[8];
    int nxc = 0, nzc = 0;
    if (ddx != 0.0) {
        const double lo = xa < xb ? xa : xb, hi = xa < xb ? xb : xa;
        const int m0 = (int)floor(lo / g.dx) + 1, m1 = (int)ceil(hi / g.dx) - 1;
        for (int m = m0; m <= m1 && nxc < 8; m++) tx[nxc++] = ((double)m * g.dx - xa) / ddx;
        if (ddx < 0.0)
            for (int i = 0; i < nxc / 2; i++) { const double t = tx[i]; tx[i] = tx[nxc - 1 - i]; tx[nxc - 1 - i] = t; }
    }
    if (ddz != 0.0) {
        const double lo = za < zb ? za : zb, hi = za < zb ? zb : za;
        const int m0 = (int)floor(lo / g.dz) + 1, m1 = (int)ceil(hi / g.dz) - 1;
        for (int m = m0; m <= m1 && nzc < 8; m++) tz[nzc++] = ((double)m * g.dz - za) / ddz;
        if (ddz < 0.0)
            for (int i = 0; i < nzc / 2; i++) { const double t = tz[i]; tz[i] = tz[nzc - 1 - i]; tz[nzc - 1 - i] = t; }
    }
    double tprev = 0.0;
    int i = 0, j = 0;
    for (;;) {
        double tnext;
        if (i < nxc && (j >= nzc || tx[i] <= tz[j])) tnext = tx[i++];
        else if (j < nzc) tnext = tz[j++];
        else tnext = 1.0;
        if (tnext > tprev) {
            const double tm = 0.5 * (tprev + tnext);
            const double xm = xa + tm * ddx, zm = za + tm * ddz;
            const int c = (cell_ix(xm, g.dx, g.nx) - 1) * (g.nz - 1) + cell_ix(zm, g.dz, g.nz);
            const double len = (tnext - tprev) * L;
            if (ns > 0 && last == c) {
                if (STORE) lens[ns - 1] += len;
            } else {
                if (STORE) {
                    cells[ns] = c;
                    lens[ns] = len;
                }
                last = c;
                ns++;
            }
            tprev = tnext;
        }
        if (tnext >= 1.0) break;
    }
}

/* One thread per ray.  Pass 1 (STORE = false) writes npts / nseg / status;
 * pass 2 writes the points from pts_off[r] and the pieces from seg_off[r]. */
template <bool STORE>
__global__ void trace_kernel(Grid g, int integrator, double xs, double zs, int nray, const double *__restrict__ xr,
                             const double *__restrict__ zr, int *npts, int *nseg, int *status, double *tn,
                             double *tne, const long long *pts_off, const long long *seg_off, double *px,
                             double *pz, int *cells, double *lens)
{
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= nray) return;
    const double ds = (g.dx < g.dz ? g.dx : g.dz) / 2.0;
    const double rad2 = (g.dx * g.dx + g.dz * g.dz) / 2.0;
    double *qx = STORE ? px + pts_off[r] : nullptr, *qz = STORE ? pz + pts_off[r] : nullptr;
    int *qc = STORE ? cells + seg_off[r] : nullptr;
    double *ql = STORE ? lens + seg_off[r] : nullptr;
    double xn = xr[r], zn = zr[r], t_n = 0.0, t_e = 0.0;
    int np = 0, ns = 0, last = -1;
    bool done = false;
    if (STORE) { qx[np] = xn; qz[np] = zn; }
    np++;
    const long long maxk = (long long)g.nx * g.nz;
    for (long long k = 1; k <= maxk; k++) {
        const int ix = cell_ix(xn, g.dx, g.nx), iz = cell_ix(zn, g.dz, g.nz);
        const double x1 = (double)(ix - 1) * g.dx, x2 = (double)ix * g.dx;
        const double z1 = (double)(iz - 1) * g.dz, z2 = (double)iz * g.dz;
        const size_t m11 = (size_t)(ix - 1) * g.zp + (iz - 1), m21 = (size_t)ix * g.zp + (iz - 1);
        const double c11 = g.tt[m11], c12 = g.tt[m11 + 1], c21 = g.tt[m21], c22 = g.tt[m21 + 1];
        double xn1, zn1;
        step(g, integrator, ds, xn, zn, xn1, zn1);
        if ((xn1 - xs) * (xn1 - xs) + (zn1 - zs) * (zn1 - zs) < rad2) {
            done = true;
            xn1 = xs;
            zn1 = zs;
        }
        const double u = g.slow[(size_t)(ix - 1) * g.zcp + (iz - 1)];
        t_e = t_e - (bilinear(xn1, zn1, x1, z1, x2, z2, c11, c12, c21, c22) -
                     bilinear(xn, zn, x1, z1, x2, z2, c11, c12, c21, c22));
        t_n = t_n + sqrt((xn1 - xn) * (xn1 - xn) + (zn1 - zn) * (zn1 - zn)) * u;
        split<STORE>(g, xn, zn, xn1, zn1, ns, last, qc, ql);
        xn = xn1;
        zn = zn1;
        if (STORE) { qx[np] = xn; qz[np] = zn; }
        np++;
        if (done) break;
    }
    if (!STORE) {
        npts[r] = np;
        nseg[r] = ns;
        status[r] = done ? 0 : 1;
        tn[r] = t_n;
        tne[r] = t_e;
    }
}

} // namespace fkray

extern "C" int fk_rays2d(int pass, int nz, int nx, int zp, int zcp, double dz, double dx, const double *slow,
                         const double *tt, const double *gx, const double *gz, int integrator, double xs, double zs,
                         int nray, const double *xr, const double *zr, int *npts, int *nseg, int *status,
                         double *tn, double *tne, const long long *pts_off, const long long *seg_off, double *px,
                         double *pz, int *cells, double *lens, cudaStream_t s)
{
    if (nray <= 0) return 0;
    const fkray::Grid g = {nz, nx, zp, zcp, dz, dx, slow, tt, gx, gz};
    const int nb = (nray + 63) / 64;
    if (pass == 1)
        fkray::trace_kernel<false><<<nb, 64, 0, s>>>(g, integrator, xs, zs, nray, xr, zr, npts, nseg, status, tn,
                                                     tne, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr);
    else
        fkray::trace_kernel<true><<<nb, 64, 0, s>>>(g, integrator, xs, zs, nray, xr, zr, npts, nseg, status, tn,
                                                    tne, pts_off, seg_off, px, pz, cells, lens);
    return (int)cudaGetLastError();
}
