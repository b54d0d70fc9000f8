/*
 * fteik_oracle.c -- TEST INFRASTRUCTURE ONLY (see fteik_oracle.h).
 *
 * A plain-C restatement of the reference fteik algorithms for the eikonal
 * solver and the grid-search locator.  Every function cites the reference
 * file:line it follows.  It is the oracle the CUDA product is tested
 * against and the CPU baseline timed beside it; the product never calls it.
 */
#include "fteik_oracle.h"

#include <math.h>
#include <stdbool.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define HUGEV ORC_HUGE
#define CHUNK 32 /* constants.F90:23 chunkSize */

static inline double dmin2(double a, double b) { return (b < a) ? b : a; }
static inline double dmax2(double a, double b) { return (b > a) ? b : a; }
static inline int imin(int a, int b) { return a < b ? a : b; }
static inline int imax(int a, int b) { return a > b ? a : b; }

/* ===================================================================== */
/* source.F90:82-236                                                     */
/* ===================================================================== */
int orc_source_snap(int is3d, int nz, int nx, int ny, double z0, double x0,
                    double y0, double dz, double dx, double dy, double zsrc,
                    double xsrc, double ysrc, int *zsi, int *xsi, int *ysi,
                    double *zsa, double *xsa, double *ysa)
{
    const double eps = 2.220446049250313e-16; /* EPSILON(1.d0) */
    const double perturb = 0.0001;            /* constants.F90:21 */
    if (!is3d) { ny = 1; dy = 1.0; y0 = 0.0; ysrc = 0.0; }
    double zmax = (double)(nz - 1) * dz;
    double xmax = (double)(nx - 1) * dx;
    double ymax = (double)(ny - 1) * dy;
    double zl = zsrc - z0, xl = xsrc - x0, yl = ysrc - y0;
    if (zl < 0.0 || zl > zmax || xl < 0.0 || xl > xmax ||
        yl < 0.0 || yl > ymax) return 1;
    double za = zl / dz + 1.0, xa = xl / dx + 1.0, ya = yl / dy + 1.0;
    if (fabs(za - 1.0) < eps) za = za + perturb;
    if (za >= (double)nz) za = za - perturb;
    if (fabs(xa - 1.0) < eps) xa = xa + perturb;
    if (xa >= (double)nx) xa = xa - perturb;
    if (fabs(ya - 1.0) < eps) ya = ya + perturb;
    if (ya >= (double)ny) ya = ya - perturb;
    int zi = (int)za, xi = (int)xa, yi = (int)ya;
    if (!is3d) { yi = 1; ya = 1.0; }
    if (zi < 1 || zi > nz || xi < 1 || xi > nx ||
        (is3d && (yi < 1 || yi > ny))) return 1;
    *zsi = zi; *xsi = xi; *ysi = yi;
    *zsa = za; *xsa = xa; *ysa = ya;
    return 0;
}

/* ===================================================================== */
/* model.F90:311-607                                                     */
/* ===================================================================== */
int orc_cell_velocity_to_slowness(int is3d, int nz, int nx, int ny, int order,
                                  const double *vel, double *slow)
{
    /* model.F90:505-607 (fteik_model_setCellVelocityModel64f) */
    if (!is3d) ny = 2;
    const int nzm1 = nz - 1, nxm1 = nx - 1, nym1 = ny - 1;
    const long ncell = (long)nzm1 * nxm1 * nym1;
    for (long i = 0; i < ncell; i++) if (!(vel[i] > 0.0)) return 1;
    if (order == 1) {
        if (is3d) {
            for (int iy = 0; iy < nym1; iy++)
                for (int ix = 0; ix < nxm1; ix++)
                    for (int iz = 0; iz < nzm1; iz++) {
                        long j = (long)iz * nxm1 * nym1 + (long)iy * nxm1 + ix;
                        long c = ((long)iy * nxm1 + ix) * nzm1 + iz;
                        slow[c] = 1.0 / vel[j];
                    }
        } else {
            for (int ix = 0; ix < nxm1; ix++)
                for (int iz = 0; iz < nzm1; iz++)
                    slow[(long)ix * nzm1 + iz] = 1.0 / vel[(long)iz * nxm1 + ix];
        }
    } else if (order == 2 && is3d) {
        for (int iy = 0; iy < nym1; iy++)
            for (int ix = 0; ix < nxm1; ix++)
                for (int iz = 0; iz < nzm1; iz++) {
                    long j = (long)ix * nzm1 * nym1 + (long)iy * nzm1 + iz;
                    long c = ((long)iy * nxm1 + ix) * nzm1 + iz;
                    slow[c] = 1.0 / vel[j];
                }
    } else {
        for (long i = 0; i < ncell; i++) slow[i] = 1.0 / vel[i];
    }
    return 0;
}

int orc_nodal_velocity_to_slowness(int is3d, int nz, int nx, int ny, int order,
                                   int keep_defects, const double *vel,
                                   double *slow)
{
    /* model.F90:311-449 (fteik_model_setNodalVelocityModel64f) */
    if (!is3d) ny = 1;
    const long ngrd = (long)nz * nx * ny;
    for (long i = 0; i < ngrd; i++) if (!(vel[i] > 0.0)) return 1;
    const int nzm1 = nz - 1, nxm1 = nx - 1;
    if (is3d) {
        const int nym1 = ny - 1;
        for (int iy = 1; iy <= nym1; iy++)
            for (int ix = 1; ix <= nxm1; ix++)
                for (int iz = 1; iz <= nzm1; iz++) {
                    long id[8];
                    double scale = 0.125;
                    if (order == 1) {
                        long b = (long)nx * ny;
                        id[0] = (iz - 1) * b + (long)(iy - 1) * nx + ix;
                        id[1] = id[0] + 1;
                        id[2] = (iz - 1) * b + (long)iy * nx + ix;
                        id[3] = id[2] + 1;
                        id[4] = (long)iz * b + (long)(iy - 1) * nx + ix;
                        id[5] = id[4] + 1;
                        id[6] = (long)iz * b + (long)iy * nx + ix;
                        id[7] = id[6] + 1;
                        if (keep_defects) scale = 1.0; /* model.F90:353 */
                    } else if (order == 2) {
                        long b = (long)ny * nz;
                        id[0] = (long)(ix - 1) * b + (long)(iy - 1) * nz + iz;
                        id[1] = id[0] + 1;
                        id[2] = (long)(ix - 1) * b + (long)iy * nz + iz;
                        id[3] = id[2] + 1;
                        id[4] = (long)ix * b + (long)(iy - 1) * nz + iz;
                        id[5] = id[4] + 1;
                        id[6] = (long)ix * b + (long)iy * nz + iz;
                        id[7] = id[6] + 1;
                    } else {
                        long nzx = (long)nz * nx;
                        int iy2 = keep_defects ? iy : iy + 1; /* model.F90:386-389 */
                        id[0] = (iy - 1) * nzx + (long)(ix - 1) * nz + iz;
                        id[1] = id[0] + 1;
                        id[2] = (iy - 1) * nzx + (long)ix * nz + iz;
                        id[3] = id[2] + 1;
                        id[4] = (iy2 - 1) * nzx + (long)(ix - 1) * nz + iz;
                        id[5] = id[4] + 1;
                        id[6] = (iy2 - 1) * nzx + (long)ix * nz + iz;
                        id[7] = id[6] + 1;
                    }
                    double s = 0.0;
                    for (int m = 0; m < 8; m++) s += vel[id[m] - 1];
                    long c = ((long)(iy - 1) * nxm1 + (ix - 1)) * nzm1 + (iz - 1);
                    slow[c] = (scale == 1.0) ? s : s * scale;
                }
        const long ncell = (long)nzm1 * nxm1 * nym1;
        for (long i = 0; i < ncell; i++) slow[i] = 1.0 / slow[i];
    } else {
        for (int ix = 1; ix <= nxm1; ix++)
            for (int iz = 1; iz <= nzm1; iz++) {
                long id[4];
                if (order == 1) {
                    id[0] = (long)(iz - 1) * nx + ix; id[1] = id[0] + 1;
                    id[2] = (long)iz * nx + ix;       id[3] = id[2] + 1;
                } else {
                    id[0] = (long)(ix - 1) * nz + iz; id[1] = id[0] + 1;
                    id[2] = (long)ix * nz + iz;       id[3] = id[2] + 1;
                }
                double s = 0.0;
                for (int m = 0; m < 4; m++) s += vel[id[m] - 1];
                slow[(long)(ix - 1) * nzm1 + (iz - 1)] = s * 0.25;
            }
        const long ncell = (long)nzm1 * nxm1;
        for (long i = 0; i < ncell; i++) slow[i] = 1.0 / slow[i];
    }
    return 0;
}

/* ===================================================================== */
/* 3D local solver: localSolver.F90:359-969                              */
/* ===================================================================== */
typedef struct {
    double dz, dx, dy;
    double dzi, dxi, dyi, dz2i, dx2i, dy2i;
    double dsum, dsum_nine, dsumi;
    double dz2dx2, dz2dy2, dx2dy2;
    double dz2i_dx2i, dz2i_dy2i, dx2i_dy2i;
    double dz2i_p_dx2i, dz2i_p_dy2i, dx2i_p_dy2i;
    double dz2i_p_dx2i_inv, dz2i_p_dy2i_inv, dx2i_p_dy2i_inv;
    /* source terms */
    int zsi, xsi, ysi;
    double zsa, xsa, ysa, szero, szero2, epsSolver;
} ls3d_t;

/* localSolver.F90:878-931 (fteik_localSolver_initialize64fF constants) */
static void ls3d_setup(ls3d_t *c, double dz, double dx, double dy, int zsi,
                       int xsi, int ysi, double zsa, double xsa, double ysa,
                       double szero, double eps)
{
    c->dz = dz; c->dx = dx; c->dy = dy;
    c->zsi = zsi; c->xsi = xsi; c->ysi = ysi;
    c->zsa = zsa; c->xsa = xsa; c->ysa = ysa;
    c->szero = szero; c->szero2 = szero * szero;
    c->epsSolver = eps * dmin2(dmin2(dz, dx), dy) * szero;
    double dz2 = dz * dz, dx2 = dx * dx, dy2 = dy * dy;
    c->dzi = 1.0 / dz; c->dxi = 1.0 / dx; c->dyi = 1.0 / dy;
    c->dz2i = 1.0 / dz2; c->dx2i = 1.0 / dx2; c->dy2i = 1.0 / dy2;
    c->dsum = c->dz2i + c->dx2i + c->dy2i;
    c->dsum_nine = c->dsum * 9.0;
    c->dsumi = 1.0 / c->dsum;
    c->dz2dx2 = 1.0 / (dz2 * dx2);
    c->dz2dy2 = 1.0 / (dz2 * dy2);
    c->dx2dy2 = 1.0 / (dx2 * dy2);
    c->dz2i_dx2i = c->dz2i * c->dx2i;
    c->dz2i_dy2i = c->dz2i * c->dy2i;
    c->dx2i_dy2i = c->dx2i * c->dy2i;
    c->dz2i_p_dy2i_inv = 1.0 / (c->dz2i + c->dy2i);
    c->dz2i_p_dx2i_inv = 1.0 / (c->dz2i + c->dx2i);
    c->dx2i_p_dy2i_inv = 1.0 / (c->dx2i + c->dy2i);
    c->dz2i_p_dx2i = c->dz2i + c->dx2i;
    c->dz2i_p_dy2i = c->dz2i + c->dy2i;
    c->dx2i_p_dy2i = c->dx2i + c->dy2i;
}

/* localSolver.F90:775-792 */
static inline double tana3d(const ls3d_t *c, int i, int j, int k)
{
    double diffz = ((double)i - c->zsa) * c->dz;
    double diffx = ((double)j - c->xsa) * c->dx;
    double diffy = ((double)k - c->ysa) * c->dy;
    double d0 = diffz * diffz + diffx * diffx + diffy * diffy;
    return c->szero * sqrt(d0);
}

/* localSolver.F90:819-851 */
static inline void tanad3d(const ls3d_t *c, int i, int j, int k, double *t_anad,
                           double *tzc, double *txc, double *tyc)
{
    double diffz = ((double)i - c->zsa) * c->dz;
    double diffx = ((double)j - c->xsa) * c->dx;
    double diffy = ((double)k - c->ysa) * c->dy;
    double d0 = diffz * diffz + diffx * diffx + diffy * diffy;
    double d0i_szero = 0.0;
    *t_anad = 0.0;
    if (d0 > 0.0) {
        double sqrtd0 = sqrt(d0);
        *t_anad = c->szero * sqrtd0;
        d0i_szero = c->szero / sqrtd0;
    }
    *tzc = d0i_szero * diffz;
    *txc = d0i_szero * diffx;
    *tyc = d0i_szero * diffy;
}

/* localSolver.F90:384-534 (fteik_localSolver_noInit64fF), one node.  tupd
 * enters holding the node's current time. */
static inline double ls3d_noinit(const ls3d_t *c, double tv, double te,
                                 double tn, double tev, double ten, double tnv,
                                 double tnve, double s1, double s2, double s3,
                                 double s4, double s5, double s6, double s7,
                                 double tupd)
{
    double t12min = tv + c->dz * s1;
    t12min = dmin2(t12min, te + c->dx * s2);
    t12min = dmin2(t12min, tn + c->dy * s3);
    /* ZX plane */
    double t1_2d = HUGEV;
    double temtv = te - tv;
    if (temtv < c->dz * s4 && -temtv < c->dx * s4) {
        double sref2 = s4 * s4;
        double ta = tev + temtv, tb = tev - temtv;
        double tab = ta - tb, tab2 = tab * tab;
        double four_sref2 = 4.0 * sref2;
        t1_2d = ((tb * c->dz2i + ta * c->dx2i) +
                 sqrt(four_sref2 * c->dz2i_p_dx2i - c->dz2i_dx2i * tab2)) *
                c->dz2i_p_dx2i_inv;
    }
    t12min = dmin2(t12min, t1_2d);
    /* ZY plane */
    double t2_2d = HUGEV;
    double tvmtn = tv - tn;
    if (tvmtn < c->dy * s5 && -tvmtn < c->dz * s5) {
        double sref2 = s5 * s5;
        double ta = tvmtn + tnv, tb = -tvmtn + tnv;
        double tab = ta - tb, tab2 = tab * tab;
        double four_sref2 = 4.0 * sref2;
        t2_2d = ((ta * c->dz2i + tb * c->dy2i) +
                 sqrt(four_sref2 * c->dz2i_p_dy2i - c->dz2i_dy2i * tab2)) *
                c->dz2i_p_dy2i_inv;
    }
    t12min = dmin2(t12min, t2_2d);
    /* XY plane */
    double t3_2d = HUGEV;
    double temtn = te - tn;
    if (temtn < c->dy * s6 && -temtn < c->dx * s6) {
        double sref2 = s6 * s6;
        double ta = temtn + ten, tb = -temtn + ten;
        double tab = ta - tb, tab2 = tab * tab;
        double four_sref2 = 4.0 * sref2;
        t3_2d = ((ta * c->dx2i + tb * c->dy2i) +
                 sqrt(four_sref2 * c->dx2i_p_dy2i - c->dx2i_dy2i * tab2)) *
                c->dx2i_p_dy2i_inv;
    }
    t12min = dmin2(t12min, t3_2d);
    /* 3D operator */
    double t3d = HUGEV;
    double tmax = dmax2(dmax2(tv, te), tn);
    if (t12min > tmax) {
        double sref2 = s7 * s7;
        double ta = te + 0.5 * (-tn + ten - tv + tev) - tnv + tnve;
        double tb = tv + 0.5 * (-tn + tnv - te + tev) - ten + tnve;
        double tc = tn + 0.5 * (-te + ten - tv + tnv) - tev + tnve;
        double tab = ta - tb, tbc = tb - tc, tac = ta - tc;
        double t2 = sref2 * c->dsum_nine;
        double tab2 = tab * tab, tbc2 = tbc * tbc, tac2 = tac * tac;
        double t3 = c->dz2dx2 * tab2 + c->dz2dy2 * tbc2 + c->dx2dy2 * tac2;
        if (t2 >= t3) {
            double t1 = tb * c->dz2i + ta * c->dx2i + tc * c->dy2i;
            t3d = (t1 + sqrt(t2 - t3)) * c->dsumi;
        }
    }
    t3d = dmin2(t3d, t12min);
    return dmin2(tupd, t3d);
}

/* localSolver.F90:538-751 (fteik_localSolver_init64fF), one node. */
static double ls3d_init(const ls3d_t *c, double tv, double te, double tn,
                        double tev, double ten, double tnv, double tnve,
                        double tt0, double slow1, double slow2, double slow3,
                        double slow4, double slow5, double slow6, double slow7,
                        int i, int j, int k, int sgntz, int sgntx, int sgnty,
                        double sgnrz_dzi, double sgnrx_dxi, double sgnry_dyi)
{
    double t1d = tv + c->dz * slow1;
    t1d = dmin2(t1d, te + c->dx * slow2);
    t1d = dmin2(t1d, tn + c->dy * slow3);
    double tmin = dmin2(dmin2(tv, te), tn);
    double tmax = dmax2(dmax2(tv, te), tn);
    bool lcart = (tmin > c->epsSolver);
    double t0c = 0.0, tzc = 0.0, txc = 0.0, tyc = 0.0;
    double tauv = HUGEV, taue = HUGEV, taun = HUGEV, tauev = HUGEV,
           tauen = HUGEV, taunv = HUGEV, taunve = HUGEV;
    if (!lcart) {
        tanad3d(c, i, j, k, &t0c, &tzc, &txc, &tyc);
        tauv = tv - tana3d(c, i - sgntz, j, k);
        taue = te - tana3d(c, i, j - sgntx, k);
        taun = tn - tana3d(c, i, j, k - sgnty);
        tauev = tev - tana3d(c, i - sgntz, j - sgntx, k);
        tauen = ten - tana3d(c, i, j - sgntx, k - sgnty);
        taunv = tnv - tana3d(c, i - sgntz, j, k - sgnty);
        taunve = tnve - tana3d(c, i - sgntz, j - sgntx, k - sgnty);
    }
    bool ldoZX = (tv < te + c->dx * slow4) && (te < tv + c->dz * slow4);
    bool ldoZY = (tv < tn + c->dy * slow5) && (tn < tv + c->dz * slow5);
    bool ldoXY = (te < tn + c->dy * slow6) && (tn < te + c->dx * slow6);
    bool ldoZXCart = ldoZX && (lcart || k != c->ysi);
    bool ldoZYCart = ldoZY && (lcart || j != c->xsi);
    bool ldoXYCart = ldoXY && (lcart || i != c->zsi);
    bool ldoZXSphere = ldoZX && !ldoZXCart;
    bool ldoZYSphere = ldoZY && !ldoZYCart;
    bool ldoXYSphere = ldoXY && !ldoXYCart;
    /* ZX plane */
    double t1_2d = HUGEV;
    if (ldoZXCart) {
        double sref2 = slow4 * slow4;
        double ta = tev + te - tv, tb = tev - te + tv;
        double tab = ta - tb, tab2 = tab * tab, four_sref2 = 4.0 * sref2;
        t1_2d = ((tb * c->dz2i + ta * c->dx2i) +
                 sqrt(four_sref2 * c->dz2i_p_dx2i - c->dz2i_dx2i * tab2)) *
                c->dz2i_p_dx2i_inv;
    }
    if (ldoZXSphere) {
        double sref2 = slow4 * slow4;
        double ta = tauev + taue - tauv, tb = tauev - taue + tauv;
        double apoly = c->dz2i_p_dx2i;
        double bpoly = 4.0 * (sgnrx_dxi * txc + sgnrz_dzi * tzc) -
                       2.0 * (ta * c->dx2i + tb * c->dz2i);
        double cpoly = ((ta * ta) * c->dx2i) + ((tb * tb) * c->dz2i) -
                       4.0 * (sgnrx_dxi * txc * ta + sgnrz_dzi * tzc * tb) +
                       4.0 * (c->szero2 - sref2 + tyc * tyc);
        double dpoly = bpoly * bpoly - 4.0 * apoly * cpoly;
        if (dpoly >= 0.0) t1_2d = (sqrt(dpoly) - bpoly) / (2.0 * apoly) + t0c;
        if (t1_2d < tv || t1_2d < te) t1_2d = HUGEV;
    }
    double t1d_t2d_min = dmin2(t1d, t1_2d);
    /* ZY plane */
    double t2_2d = HUGEV;
    if (ldoZYCart) {
        double sref2 = slow5 * slow5;
        double ta = tv - tn + tnv, tb = tn - tv + tnv;
        double tab = ta - tb, tab2 = tab * tab, four_sref2 = 4.0 * sref2;
        t2_2d = ((ta * c->dz2i + tb * c->dy2i) +
                 sqrt(four_sref2 * c->dz2i_p_dy2i - c->dz2i_dy2i * tab2)) *
                c->dz2i_p_dy2i_inv;
    }
    if (ldoZYSphere) {
        double sref2 = slow5 * slow5;
        double ta = tauv - taun + taunv, tb = taun - tauv + taunv;
        double apoly = c->dz2i_p_dy2i;
        double bpoly = 4.0 * (sgnry_dyi * tyc + sgnrz_dzi * tzc) -
                       2.0 * (ta * c->dz2i + tb * c->dy2i);
        double cpoly = ((ta * ta) * c->dz2i) + ((tb * tb) * c->dy2i) -
                       4.0 * (sgnrz_dzi * tzc * ta + sgnry_dyi * tyc * tb) +
                       4.0 * (c->szero2 - sref2 + txc * txc);
        double dpoly = bpoly * bpoly - 4.0 * apoly * cpoly;
        if (dpoly >= 0.0) t2_2d = (sqrt(dpoly) - bpoly) / (2.0 * apoly) + t0c;
        if (t2_2d < tv || t2_2d < tn) t2_2d = HUGEV;
    }
    t1d_t2d_min = dmin2(t1d_t2d_min, t2_2d);
    /* XY plane */
    double t3_2d = HUGEV;
    if (ldoXYCart) {
        double sref2 = slow6 * slow6;
        double ta = te - tn + ten, tb = tn - te + ten;
        double tab = ta - tb, tab2 = tab * tab, four_sref2 = 4.0 * sref2;
        t3_2d = ((ta * c->dx2i + tb * c->dy2i) +
                 sqrt(four_sref2 * c->dx2i_p_dy2i - c->dx2i_dy2i * tab2)) *
                c->dx2i_p_dy2i_inv;
    }
    if (ldoXYSphere) {
        double sref2 = slow6 * slow6;
        double ta = taue - taun + tauen, tb = taun - taue + tauen;
        double apoly = c->dx2i_p_dy2i;
        double bpoly = 4.0 * (sgnry_dyi * tyc + sgnrx_dxi * txc) -
                       2.0 * (ta * c->dx2i + tb * c->dy2i);
        double cpoly = ((ta * ta) * c->dx2i) + ((tb * tb) * c->dy2i) -
                       4.0 * (sgnrx_dxi * txc * ta + sgnry_dyi * tyc * tb) +
                       4.0 * (c->szero2 - sref2 + tzc * tzc);
        double dpoly = bpoly * bpoly - 4.0 * apoly * cpoly;
        if (dpoly >= 0.0) t3_2d = (sqrt(dpoly) - bpoly) / (2.0 * apoly) + t0c;
        if (t3_2d < te || t3_2d < tn) t3_2d = HUGEV;
    }
    t1d_t2d_min = dmin2(t1d_t2d_min, t3_2d);
    /* 3D operators */
    double t3d = HUGEV;
    bool ldo3D = (t1d_t2d_min > tmax);
    if (ldo3D && lcart) {
        double sref2 = slow7 * slow7;
        double ta = te + 0.5 * (-tn + ten - tv + tev) - tnv + tnve;
        double tb = tv + 0.5 * (-tn + tnv - te + tev) - ten + tnve;
        double tc = tn + 0.5 * (-te + ten - tv + tnv) - tev + tnve;
        double tab = ta - tb, tbc = tb - tc, tac = ta - tc;
        double t2 = sref2 * c->dsum_nine;
        double tab2 = tab * tab, tbc2 = tbc * tbc, tac2 = tac * tac;
        double t3 = c->dz2dx2 * tab2 + c->dz2dy2 * tbc2 + c->dx2dy2 * tac2;
        if (t2 >= t3) {
            double t1 = tb * c->dz2i + ta * c->dx2i + tc * c->dy2i;
            t3d = (t1 + sqrt(t2 - t3)) * c->dsumi;
        }
    }
    if (ldo3D && !lcart) {
        double sref2 = slow7 * slow7;
        double ta = taue + 0.5 * (-taun + tauen - tauv + tauev) - taunv + taunve;
        double tb = tauv + 0.5 * (-taun + taunv - taue + tauev) - tauen + taunve;
        double tc = taun + 0.5 * (-taue + tauen - tauv + taunv) - tauev + taunve;
        double apoly = c->dx2i + c->dz2i + c->dy2i;
        double bpoly = 6.0 * (sgnrz_dzi * tzc + sgnry_dyi * tyc + sgnrx_dxi * txc) -
                       2.0 * (ta * c->dx2i + tb * c->dz2i + tc * c->dy2i);
        double cpoly = ((ta * ta) * c->dx2i) + ((tb * tb) * c->dz2i) +
                       ((tc * tc) * c->dy2i) -
                       6.0 * (sgnrx_dxi * txc * ta + sgnrz_dzi * tzc * tb +
                              sgnry_dyi * tyc * tc) +
                       9.0 * (c->szero2 - sref2);
        double dpoly = bpoly * bpoly - 4.0 * apoly * cpoly;
        if (dpoly >= 0.0) t3d = (sqrt(dpoly) - bpoly) / (2.0 * apoly) + t0c;
        if (t3d < te || t3d < tn || t3d < tv) t3d = HUGEV;
    }
    double tupd = dmin2(t1d_t2d_min, t3d);
    return dmin2(tt0, tupd);
}

/* Sweep sign tables: autoCode.f90 parameter lines (sgnt*: 34-36 ... 356-358;
 * sgnv*: 407-409 ... 960-962) and python/prefetch.py:4-8,50-52. */
static void sweep_signs(int sweep, int *sgntz, int *sgntx, int *sgnty)
{
    int s = sweep - 1;
    *sgntz = (s < 4) ? 1 : -1;
    *sgntx = (s % 2 == 0) ? 1 : -1;
    *sgnty = ((s / 2) % 2 == 0) ? 1 : -1;
}

/* solver3D.F90:493-565 (getSweepLimits) -> inclusive 1-based box.
 * The flipped-axis initialisation bound si+1 is clamped to n-1: at si = n-1
 * the reference reads one node past the end of the grid (only its own 2D
 * FSM clamps, solver2D.F90:1086-1130); everywhere else the box is the
 * reference's. */
static void sweep_box(int sgnt, int linit, int n, int si, int *lo, int *hi)
{
    if (sgnt > 0) {
        *lo = linit ? imax(2, si) : 2;
        *hi = n;
    } else {
        *lo = 1;
        *hi = linit ? imin(si + 1, n - 1) : n - 1;
    }
}

/* autoCode.f90:389-447 (prefetchSweep<s>Slowness64fF), generalised over the
 * sweep's slowness signs. */
static inline void fetch_slow7(const double *slow, int nz, int nx, int ny,
                               int i, int j, int k, int sgnvz, int sgnvx,
                               int sgnvy, double *s)
{
    const long nzm1 = nz - 1, nzm1_nxm1 = (long)(nz - 1) * (nx - 1);
#define VG(a, b, c) slow[((long)(c) - 1) * nzm1_nxm1 + ((long)(b) - 1) * nzm1 + (a) - 1]
    int i1 = i - sgnvz, j1 = j - sgnvx, k1 = k - sgnvy;
    int im = imax(i - 1, 1), jm = imax(j - 1, 1), km = imax(k - 1, 1);
    int ip = imin(i, nz - 1), jp = imin(j, nx - 1), kp = imin(k, ny - 1);
    double sl[19];
    sl[0] = VG(i1, jm, km);  sl[4] = VG(im, j1, km);  sl[8] = VG(im, jm, k1);
    sl[12] = VG(i1, j1, km); sl[14] = VG(i1, jm, k1); sl[16] = VG(im, j1, k1);
    sl[18] = VG(i1, j1, k1); sl[5] = VG(ip, j1, km);  sl[10] = VG(ip, jm, k1);
    sl[17] = VG(ip, j1, k1); sl[2] = VG(i1, jp, km);  sl[9] = VG(im, jp, k1);
    sl[15] = VG(i1, jp, k1); sl[11] = VG(ip, jp, k1); sl[1] = VG(i1, jm, kp);
    sl[6] = VG(im, j1, kp);  sl[13] = VG(i1, j1, kp); sl[7] = VG(ip, j1, kp);
    sl[3] = VG(i1, jp, kp);
#undef VG
    s[0] = dmin2(dmin2(dmin2(sl[0], sl[1]), sl[2]), sl[3]);
    s[1] = dmin2(dmin2(dmin2(sl[4], sl[5]), sl[6]), sl[7]);
    s[2] = dmin2(dmin2(dmin2(sl[8], sl[9]), sl[10]), sl[11]);
    s[3] = dmin2(sl[12], sl[13]);
    s[4] = dmin2(sl[14], sl[15]);
    s[5] = dmin2(sl[16], sl[17]);
    s[6] = sl[18];
}

/* autoCode.f90:23-46 (prefetchSweep<s>TravelTimes64fF) generalised. */
static inline void fetch_tt8(const double *tt, int nz, int nx, int i, int j,
                             int k, int sz, int sx, int sy, double *t)
{
    const long nzx = (long)nz * nx;
#define G(a, b, c) tt[((long)(c) - 1) * nzx + ((long)(b) - 1) * nz + (a) - 1]
    t[0] = G(i - sz, j, k);           /* tv   */
    t[1] = G(i, j - sx, k);           /* te   */
    t[2] = G(i, j, k - sy);           /* tn   */
    t[3] = G(i - sz, j - sx, k);      /* tev  */
    t[4] = G(i, j - sx, k - sy);      /* ten  */
    t[5] = G(i - sz, j, k - sy);      /* tnv  */
    t[6] = G(i - sz, j - sx, k - sy); /* tnve */
    t[7] = G(i, j, k);                /* t    */
#undef G
}

/* One node update of sweep `sweep` at (i,j,k), 1-based. */
static inline double update_node3d(const ls3d_t *c, const double *slow,
                                   const double *tt, int nz, int nx, int ny,
                                   int i, int j, int k, int sz, int sx, int sy,
                                   int linit)
{
    double s[7], t[8];
    fetch_slow7(slow, nz, nx, ny, i, j, k, sz > 0, sx > 0, sy > 0, s);
    fetch_tt8(tt, nz, nx, i, j, k, sz, sx, sy, t);
    if (!linit)
        return ls3d_noinit(c, t[0], t[1], t[2], t[3], t[4], t[5], t[6], s[0],
                           s[1], s[2], s[3], s[4], s[5], s[6], t[7]);
    return ls3d_init(c, t[0], t[1], t[2], t[3], t[4], t[5], t[6], t[7], s[0],
                     s[1], s[2], s[3], s[4], s[5], s[6], i, j, k, sz, sx, sy,
                     (double)sz / c->dz, (double)sx / c->dx, (double)sy / c->dy);
}

/* Natural-order sweep: a valid topological order of the sweep's dependency
 * graph, hence the same result as the level order of autoCode.f90 (a node
 * reads only upwind nodes of earlier levels). */
static double sweep3d_natural(const ls3d_t *c, const double *slow, double *tt,
                              int nz, int nx, int ny, int sweep, int linit)
{
    int sz, sx, sy;
    sweep_signs(sweep, &sz, &sx, &sy);
    int zlo, zhi, xlo, xhi, ylo, yhi;
    sweep_box(sz, linit, nz, c->zsi, &zlo, &zhi);
    sweep_box(sx, linit, nx, c->xsi, &xlo, &xhi);
    sweep_box(sy, linit, ny, c->ysi, &ylo, &yhi);
    const long nzx = (long)nz * nx;
    double dmax = 0.0;
    for (int kk = 0; kk <= yhi - ylo; kk++) {
        int k = (sy > 0) ? ylo + kk : yhi - kk;
        for (int jj = 0; jj <= xhi - xlo; jj++) {
            int j = (sx > 0) ? xlo + jj : xhi - jj;
            for (int ii = 0; ii <= zhi - zlo; ii++) {
                int i = (sz > 0) ? zlo + ii : zhi - ii;
                long idx = (long)(k - 1) * nzx + (long)(j - 1) * nz + (i - 1);
                double told = tt[idx];
                double tnew = update_node3d(c, slow, tt, nz, nx, ny, i, j, k,
                                            sz, sx, sy, linit);
                tt[idx] = tnew;
                double d = fabs(tnew - told);
                if (d > dmax) dmax = d;
            }
        }
    }
    return dmax;
}

/* ------------------------------------------------------------------------- */
/* Level-set schedule: graph3d.F90:122-353 (levels i+j+k in sweep-permuted   */
/* coordinates, nodes inside a level sorted by grid index) and the masks of  */
/* solver3D.F90:289-320,340-387.                                             */
/* ------------------------------------------------------------------------- */
typedef struct {
    int nz, nx, ny, nlevels;
    long ngrd;
    long *levelPtr;   /* nlevels+1 */
    int32_t *ijkv[8]; /* 4*ngrd per sweep: iz, ix, iy (1-based), index (0-based) */
    unsigned char *lupd[8];
} lvl_t;

static void lvl_free(lvl_t *g)
{
    if (!g) return;
    free(g->levelPtr);
    for (int s = 0; s < 8; s++) { free(g->ijkv[s]); free(g->lupd[s]); }
    free(g);
}

static lvl_t *lvl_create(int nz, int nx, int ny)
{
    lvl_t *g = (lvl_t *)calloc(1, sizeof(lvl_t));
    g->nz = nz; g->nx = nx; g->ny = ny;
    g->ngrd = (long)nz * nx * ny;
    g->nlevels = nx + ny + nz - 2;
    g->levelPtr = (long *)calloc((size_t)g->nlevels + 1, sizeof(long));
    /* level sizes are the same for every sweep */
    long *cnt = (long *)calloc((size_t)g->nlevels, sizeof(long));
    for (int k = 0; k < ny; k++)
        for (int j = 0; j < nx; j++)
            for (int i = 0; i < nz; i++) cnt[i + j + k]++;
    g->levelPtr[0] = 0;
    for (int l = 0; l < g->nlevels; l++) g->levelPtr[l + 1] = g->levelPtr[l] + cnt[l];
    free(cnt);
    for (int s = 0; s < 8; s++) {
        int sz, sx, sy;
        sweep_signs(s + 1, &sz, &sx, &sy);
        g->ijkv[s] = (int32_t *)malloc(sizeof(int32_t) * 4 * (size_t)g->ngrd);
        g->lupd[s] = (unsigned char *)calloc((size_t)g->ngrd, 1);
        int zlo, zhi, xlo, xhi, ylo, yhi;
        sweep_box(sz, 0, nz, 0, &zlo, &zhi);
        sweep_box(sx, 0, nx, 0, &xlo, &xhi);
        sweep_box(sy, 0, ny, 0, &ylo, &yhi);
#pragma omp parallel for schedule(dynamic, 4)
        for (int l = 0; l < g->nlevels; l++) {
            long pos = g->levelPtr[l];
            /* sorted by grid index: iterate physical (k, j) ascending; each
             * (j,k) pair owns a disjoint index range. */
            for (int k = 0; k < ny; k++) {
                int kp = (sy > 0) ? k : ny - 1 - k;
                for (int j = 0; j < nx; j++) {
                    int jp = (sx > 0) ? j : nx - 1 - j;
                    int ip = l - kp - jp;
                    if (ip < 0 || ip >= nz) continue;
                    int i = (sz > 0) ? ip : nz - 1 - ip;
                    int32_t *e = g->ijkv[s] + 4 * pos;
                    e[0] = i + 1; e[1] = j + 1; e[2] = k + 1;
                    e[3] = (int32_t)((long)k * nz * nx + (long)j * nz + i);
                    g->lupd[s][pos] = (e[0] >= zlo && e[0] <= zhi &&
                                       e[1] >= xlo && e[1] <= xhi &&
                                       e[2] >= ylo && e[2] <= yhi);
                    pos++;
                }
            }
        }
    }
    return g;
}

/* One sweep in the reference's schedule: autoCode.f90:1052-1316.  Runs
 * inside an OpenMP parallel region; returns this thread's max |dt|. */
static double sweep3d_levels(const ls3d_t *c, const double *slow, double *tt,
                             const lvl_t *g, int sweep, int linit,
                             const unsigned char *lupdInit)
{
    int sz, sx, sy;
    sweep_signs(sweep, &sz, &sx, &sy);
    const int s = sweep - 1;
    const int32_t *ijkv = g->ijkv[s];
    const unsigned char *mask = linit ? lupdInit : g->lupd[s];
    const int nz = g->nz, nx = g->nx, ny = g->ny;
    double t1[CHUNK], t2[CHUNK], t3[CHUNK], t4[CHUNK], t5[CHUNK], t6[CHUNK],
        t7[CHUNK], tt1[CHUNK], sv[7][CHUNK];
    double dmax = 0.0;
    for (int l = 0; l < g->nlevels; l++) {
        long l1 = g->levelPtr[l], l2 = g->levelPtr[l + 1];
#pragma omp for schedule(static)
        for (long kn = l1; kn < l2; kn += CHUNK) {
            long n2 = (l2 - kn < CHUNK) ? (l2 - kn) : CHUNK;
            for (long q = 0; q < n2; q++) {
                long node = kn + q;
                if (!mask[node]) continue;
                const int32_t *e = ijkv + 4 * node;
                double sl[7], tq[8];
                fetch_slow7(slow, nz, nx, ny, e[0], e[1], e[2], sz > 0, sx > 0,
                            sy > 0, sl);
                for (int m = 0; m < 7; m++) sv[m][q] = sl[m];
                fetch_tt8(tt, nz, nx, e[0], e[1], e[2], sz, sx, sy, tq);
                t1[q] = tq[0]; t2[q] = tq[1]; t3[q] = tq[2]; t4[q] = tq[3];
                t5[q] = tq[4]; t6[q] = tq[5]; t7[q] = tq[6]; tt1[q] = tq[7];
            }
            for (long q = 0; q < n2; q++) {
                long node = kn + q;
                if (!mask[node]) continue;
                const int32_t *e = ijkv + 4 * node;
                double told = tt1[q];
                if (!linit)
                    tt1[q] = ls3d_noinit(c, t1[q], t2[q], t3[q], t4[q], t5[q],
                                         t6[q], t7[q], sv[0][q], sv[1][q],
                                         sv[2][q], sv[3][q], sv[4][q], sv[5][q],
                                         sv[6][q], tt1[q]);
                else
                    tt1[q] = ls3d_init(c, t1[q], t2[q], t3[q], t4[q], t5[q],
                                       t6[q], t7[q], tt1[q], sv[0][q], sv[1][q],
                                       sv[2][q], sv[3][q], sv[4][q], sv[5][q],
                                       sv[6][q], e[0], e[1], e[2], sz, sx, sy,
                                       (double)sz / c->dz, (double)sx / c->dx,
                                       (double)sy / c->dy);
                double d = fabs(tt1[q] - told);
                if (d > dmax) dmax = d;
            }
            for (long q = 0; q < n2; q++) {
                long node = kn + q;
                if (mask[node]) tt[ijkv[4 * node + 3]] = tt1[q];
            }
        }
        /* implicit barrier of the omp for, then the reference's BARRIER */
#pragma omp barrier
    }
    return dmax;
}

static int solve3d_impl(int nz, int nx, int ny, double dz, double dx, double dy,
                        const double *slow, int zsi, int xsi, int ysi,
                        double zsa, double xsa, double ysa, double eps,
                        int nsweep, double conv_tol, int max_pass,
                        int level_set, int nthreads, double *tt, int *npass)
{
    if (nz < 3 || nx < 3 || ny < 3) return 1;
    if (zsi < 1 || zsi > nz - 1 || xsi < 1 || xsi > nx - 1 || ysi < 1 ||
        ysi > ny - 1) return 1;
    const long nzx = (long)nz * nx, ngrd = nzx * ny;
    const long nzm1_nxm1 = (long)(nz - 1) * (nx - 1);
    /* source.F90:429-464 szero = slow at the source cell */
    double szero = slow[(long)(ysi - 1) * nzm1_nxm1 + (long)(xsi - 1) * (nz - 1) + zsi - 1];
    ls3d_t c;
    ls3d_setup(&c, dz, dx, dy, zsi, xsi, ysi, zsa, xsa, ysa, szero, eps);
    /* solver3D.F90:1201-1202 + localSolver.F90:933-956 */
    for (long i = 0; i < ngrd; i++) tt[i] = HUGEV;
    for (int m = 0; m < 8; m++) {
        int di = m & 1, dj = (m >> 1) & 1, dk = (m >> 2) & 1;
        tt[(long)(ysi - 1 + dk) * nzx + (long)(xsi - 1 + dj) * nz + (zsi - 1 + di)] =
            tana3d(&c, zsi + di, xsi + dj, ysi + dk);
    }
    int converge = (conv_tol >= 0.0 && max_pass > 0);
    int npasses = converge ? max_pass : nsweep;
    int ran = 0;
    if (!level_set) {
        for (int s = 1; s <= 8; s++) sweep3d_natural(&c, slow, tt, nz, nx, ny, s, 1);
        for (int it = 0; it < npasses; it++) {
            double dmax = 0.0;
            for (int s = 1; s <= 8; s++) {
                double d = sweep3d_natural(&c, slow, tt, nz, nx, ny, s, 0);
                if (d > dmax) dmax = d;
            }
            ran++;
            if (converge && dmax <= conv_tol) break;
        }
    } else {
        lvl_t *g = lvl_create(nz, nx, ny);
        unsigned char *lupdInit[8];
        for (int s = 0; s < 8; s++) {
            /* solver3D.F90:340-387 setInitialUpdateNodes, O(8 ngrd) per solve */
            int sz, sx, sy, zlo, zhi, xlo, xhi, ylo, yhi;
            sweep_signs(s + 1, &sz, &sx, &sy);
            sweep_box(sz, 1, nz, zsi, &zlo, &zhi);
            sweep_box(sx, 1, nx, xsi, &xlo, &xhi);
            sweep_box(sy, 1, ny, ysi, &ylo, &yhi);
            lupdInit[s] = (unsigned char *)malloc((size_t)ngrd);
            const int32_t *ijkv = g->ijkv[s];
#pragma omp parallel for schedule(static)
            for (long n = 0; n < ngrd; n++) {
                const int32_t *e = ijkv + 4 * n;
                lupdInit[s][n] = (e[0] >= zlo && e[0] <= zhi && e[1] >= xlo &&
                                  e[1] <= xhi && e[2] >= ylo && e[2] <= yhi);
            }
        }
        int nth = nthreads;
#ifdef _OPENMP
        if (nth <= 0) nth = omp_get_max_threads();
#else
        nth = 1;
#endif
        double pass_max = 0.0;
        int stop = 0;
#pragma omp parallel num_threads(nth)
        {
            for (int s = 1; s <= 8; s++)
                sweep3d_levels(&c, slow, tt, g, s, 1, lupdInit[s - 1]);
            for (int it = 0; it < npasses; it++) {
                double dmax = 0.0;
                for (int s = 1; s <= 8; s++) {
                    double d = sweep3d_levels(&c, slow, tt, g, s, 0, NULL);
                    if (d > dmax) dmax = d;
                }
#pragma omp single
                { pass_max = 0.0; }
#pragma omp critical
                { if (dmax > pass_max) pass_max = dmax; }
#pragma omp barrier
#pragma omp single
                {
                    ran++;
                    if (converge && pass_max <= conv_tol) stop = 1;
                }
                if (stop) break;
            }
        }
        for (int s = 0; s < 8; s++) free(lupdInit[s]);
        lvl_free(g);
    }
    if (npass) *npass = ran;
    return 0;
}

int orc_solve3d(int nz, int nx, int ny, double dz, double dx, double dy,
                const double *slow, int zsi, int xsi, int ysi, double zsa,
                double xsa, double ysa, double eps, int nsweep,
                double conv_tol, int max_pass, int level_set, int nthreads,
                double *tt, int *npass)
{
    return solve3d_impl(nz, nx, ny, dz, dx, dy, slow, zsi, xsi, ysi, zsa, xsa,
                        ysa, eps, nsweep, conv_tol, max_pass, level_set,
                        nthreads, tt, npass);
}

int orc_sweep3d(int sweep, int linit, int nz, int nx, int ny, double dz,
                double dx, double dy, const double *slow, int zsi, int xsi,
                int ysi, double zsa, double xsa, double ysa, double eps,
                double *tt)
{
    if (sweep < 1 || sweep > 8) return 1;
    const long nzm1_nxm1 = (long)(nz - 1) * (nx - 1);
    double szero = slow[(long)(ysi - 1) * nzm1_nxm1 + (long)(xsi - 1) * (nz - 1) + zsi - 1];
    ls3d_t c;
    ls3d_setup(&c, dz, dx, dy, zsi, xsi, ysi, zsa, xsa, ysa, szero, eps);
    sweep3d_natural(&c, slow, tt, nz, nx, ny, sweep, linit);
    return 0;
}

void orc_count_updates3d(int nz, int nx, int ny, int zsi, int xsi, int ysi,
                         int64_t *n_init, int64_t *n_pass)
{
    int64_t a = 0, b = 0;
    for (int s = 1; s <= 8; s++) {
        int sz, sx, sy, zlo, zhi, xlo, xhi, ylo, yhi;
        sweep_signs(s, &sz, &sx, &sy);
        sweep_box(sz, 1, nz, zsi, &zlo, &zhi);
        sweep_box(sx, 1, nx, xsi, &xlo, &xhi);
        sweep_box(sy, 1, ny, ysi, &ylo, &yhi);
        a += (int64_t)imax(0, zhi - zlo + 1) * imax(0, xhi - xlo + 1) * imax(0, yhi - ylo + 1);
        sweep_box(sz, 0, nz, zsi, &zlo, &zhi);
        sweep_box(sx, 0, nx, xsi, &xlo, &xhi);
        sweep_box(sy, 0, ny, ysi, &ylo, &yhi);
        b += (int64_t)(zhi - zlo + 1) * (xhi - xlo + 1) * (yhi - ylo + 1);
    }
    if (n_init) *n_init = a;
    if (n_pass) *n_pass = b;
}

/* ===================================================================== */
/* 2D: localSolver.F90:1-352, solver2D.F90:377-978, :1042-1280           */
/* ===================================================================== */
typedef struct {
    double dz, dx, dzi, dxi, dz2i, dx2i, dz2i_dx2i, dz2i_p_dx2i,
        dz2i_p_dx2i_inv, epsSolver;
    double szero, szero2, zsa, xsa;
    int zsi, xsi;
} ls2d_t;

/* localSolver.F90:36-50 */
static inline double tana2d(const ls2d_t *c, int i, int j)
{
    double diffz = ((double)i - c->zsa) * c->dz;
    double diffx = ((double)j - c->xsa) * c->dx;
    return c->szero * hypot(diffx, diffz);
}

/* localSolver.F90:74-112 */
static inline void tanad2d(const ls2d_t *c, int i, int j, double *t_anad,
                           double *tzc, double *txc)
{
    double diffz = ((double)i - c->zsa) * c->dz;
    double diffx = ((double)j - c->xsa) * c->dx;
    double d0 = diffz * diffz + diffx * diffx;
    double d0i_szero = 0.0;
    *t_anad = 0.0;
    if (d0 > 0.0) {
        double sqrtd0 = sqrt(d0);
        *t_anad = c->szero * sqrtd0;
        d0i_szero = c->szero / sqrtd0;
    }
    *tzc = d0i_szero * diffz;
    *txc = d0i_szero * diffx;
}

/* localSolver.F90:123-158 (one node) */
static inline double ls2d_noinit(const ls2d_t *c, double tv, double te,
                                 double tev, double s1, double s2, double s3)
{
    double temtv = te - tv;
    double t12min = dmin2(tv + c->dz * s1, te + c->dx * s2);
    double t1_2d = HUGEV;
    if (temtv < c->dz * s3 && -temtv < c->dx * s3) {
        double sref2 = s3 * s3;
        double ta = tev + temtv, tb = tev - temtv;
        double tab = ta - tb, tab2 = tab * tab, four_sref2 = 4.0 * sref2;
        t1_2d = ((tb * c->dz2i + ta * c->dx2i) +
                 sqrt(four_sref2 * c->dz2i_p_dx2i - c->dz2i_dx2i * tab2)) *
                c->dz2i_p_dx2i_inv;
    }
    return dmin2(t12min, t1_2d);
}

/* 2D slowness stencil: solver2D.F90:474-585 / localSolver.F90:222-231 */
static inline void fetch_slow2d(const double *slow, int nz, int nx, int iz,
                                int ix, int sgnvz, int sgnvx, double *s1,
                                double *s2, double *s3)
{
    int i1 = iz - sgnvz, j1 = ix - sgnvx;
    long n = nz - 1;
    long indx1 = (long)(imax(ix - 1, 1) - 1) * n + i1;
    long indx2 = (long)(imin(ix, nx - 1) - 1) * n + i1;
    long indx3 = (long)(j1 - 1) * n + imax(iz - 1, 1);
    long indx4 = (long)(j1 - 1) * n + imin(iz, nz - 1);
    long indx5 = (long)(j1 - 1) * n + i1;
    *s1 = dmin2(slow[indx1 - 1], slow[indx2 - 1]);
    *s2 = dmin2(slow[indx3 - 1], slow[indx4 - 1]);
    *s3 = slow[indx5 - 1];
}

/* localSolver.F90:195-289 (fteik_localSolver2d_init64f) */
static double ls2d_init(const ls2d_t *c, int sgntz, int sgntx, int sgnvz,
                        int sgnvx, int nz, int nx, int iz, int ix,
                        const double *slow, const double *tt)
{
    double sgnrz = (double)sgntz, sgnrx = (double)sgntx;
    long indxv = (long)(ix - 1) * nz + iz - sgntz;
    long indxe = (long)(ix - sgntx - 1) * nz + iz;
    long indxev = (long)(ix - sgntx - 1) * nz + iz - sgntz;
    long indx = (long)(ix - 1) * nz + iz;
    double tv = tt[indxv - 1], te = tt[indxe - 1], tev = tt[indxev - 1],
           t = tt[indx - 1];
    double sref1, sref2, sref3;
    fetch_slow2d(slow, nz, nx, iz, ix, sgnvz, sgnvx, &sref1, &sref2, &sref3);
    double t1d = dmin2(tv + c->dz * sref1, te + c->dx * sref2);
    double t0c, tzc, txc;
    tanad2d(c, iz, ix, &t0c, &tzc, &txc);
    double tauv = tv - tana2d(c, iz - sgntz, ix);
    double taue = te - tana2d(c, iz, ix - sgntx);
    double tauev = tev - tana2d(c, iz - sgntz, ix - sgntx);
    double t1 = HUGEV, t2 = HUGEV, t3 = HUGEV;
    if (abs(iz - c->zsi) > c->epsSolver || abs(ix - c->xsi) > c->epsSolver) {
        if (tv <= te + c->dx * sref3 && te <= tv + c->dz * sref3 && te >= tev &&
            tv >= tev) {
            double ta = tev + te - tv, tb = tev - te + tv;
            t1 = ((tb * c->dz2i + ta * c->dx2i) +
                  sqrt(4.0 * sref3 * sref3 * (c->dz2i + c->dx2i) -
                       c->dz2i * c->dx2i * (ta - tb) * (ta - tb))) /
                 (c->dz2i + c->dx2i);
        } else if ((te - tev) <= c->dz * c->dz * sref3 / sqrt(c->dx * c->dx + c->dz * c->dz) &&
                   te > tev) {
            double q = (te - tev) / c->dz;
            t2 = te + c->dx * sqrt(sref3 * sref3 - q * q);
        } else if ((tv - tev) <= c->dx * c->dx * sref3 / sqrt(c->dx * c->dx + c->dz * c->dz) &&
                   tv > tev) {
            double q = (tv - tev) / c->dx;
            t3 = tv + c->dz * sqrt(sref3 * sref3 - q * q);
        }
    } else {
        if (tv < te + c->dx * sref3 && te < tv + c->dz * sref3 && te >= tev &&
            tv >= tev) {
            double ta = tauev + taue - tauv, tb = tauev - taue + tauv;
            double apoly = c->dz2i + c->dx2i;
            double bpoly = 4.0 * (sgnrx * txc * c->dxi + sgnrz * tzc * c->dzi) -
                           2.0 * (ta * c->dx2i + tb * c->dz2i);
            double cpoly = (ta * ta * c->dx2i) + (tb * tb * c->dz2i) -
                           4.0 * (sgnrx * txc * c->dxi * ta + sgnrz * tzc * c->dzi * tb) +
                           4.0 * (c->szero * c->szero - sref3 * sref3);
            double dpoly = bpoly * bpoly - 4.0 * apoly * cpoly;
            if (dpoly >= 0.0) t1 = 0.5 * (sqrt(dpoly) - bpoly) / apoly + t0c;
            if (t1 < tv || t1 < te) t1 = HUGEV;
        }
    }
    double t2d = dmin2(dmin2(t1, t2), t3);
    return dmin2(dmin2(t, t1d), t2d);
}

static void sweep2d_signs(int sweep, int *sgntz, int *sgntx, int *sgnvz,
                          int *sgnvx)
{
    /* localSolver.F90:160-193 */
    *sgntz = (sweep <= 2) ? 1 : -1;
    *sgntx = (sweep == 1 || sweep == 3) ? 1 : -1;
    *sgnvz = (*sgntz > 0);
    *sgnvx = (*sgntx > 0);
}

int orc_solve2d(int fsm, int nz, int nx, double dz, double dx,
                const double *slow, int zsi, int xsi, double zsa, double xsa,
                double eps, int nsweep, double conv_tol, int max_pass,
                double *tt, int *npass)
{
    if (nz < 3 || nx < 3) return 1;
    if (zsi < 1 || zsi > nz - 1 || xsi < 1 || xsi > nx - 1) return 1;
    ls2d_t c;
    memset(&c, 0, sizeof(c));
    c.dz = dz; c.dx = dx;
    c.zsi = zsi; c.xsi = xsi; c.zsa = zsa; c.xsa = xsa;
    c.szero = slow[(long)(xsi - 1) * (nz - 1) + zsi - 1];
    c.szero2 = c.szero * c.szero;
    c.epsSolver = eps; /* grid points, localSolver.F90:327 */
    c.dzi = 1.0 / dz; c.dxi = 1.0 / dx;
    c.dz2i = 1.0 / (dz * dz); c.dx2i = 1.0 / (dx * dx);
    c.dz2i_dx2i = c.dz2i * c.dx2i;
    c.dz2i_p_dx2i = c.dz2i + c.dx2i;
    c.dz2i_p_dx2i_inv = 1.0 / (c.dz2i + c.dx2i);
    const long ngrd = (long)nz * nx;
    for (long i = 0; i < ngrd; i++) tt[i] = HUGEV;
    /* localSolver.F90:342-349 */
    tt[(long)(xsi - 1) * nz + zsi - 1] = tana2d(&c, zsi, xsi);
    tt[(long)(xsi - 1) * nz + zsi] = tana2d(&c, zsi + 1, xsi);
    tt[(long)xsi * nz + zsi - 1] = tana2d(&c, zsi, xsi + 1);
    tt[(long)xsi * nz + zsi] = tana2d(&c, zsi + 1, xsi + 1);
    /* initialisation: solver2D.F90:825-867 (LSM) and :1080-1130 (FSM).  The
     * upper bound xsi+1 / zsi+1 of the flipped sweeps is clamped to n-1 as
     * the FSM does; the LSM reads past the grid when the source sits in the
     * last cell. */
    int xhi = imin(nx - 1, xsi + 1), zhi = imin(nz - 1, zsi + 1);
    for (int sweep = 1; sweep <= 4; sweep++) {
        int sgntz, sgntx, sgnvz, sgnvx;
        sweep2d_signs(sweep, &sgntz, &sgntx, &sgnvz, &sgnvx);
        int xa = (sgntx > 0) ? imax(2, xsi) : xhi, xb = (sgntx > 0) ? nx : 1;
        int za = (sgntz > 0) ? imax(2, zsi) : zhi, zb = (sgntz > 0) ? nz : 1;
        for (int ix = xa; (sgntx > 0) ? ix <= xb : ix >= xb; ix += sgntx)
            for (int iz = za; (sgntz > 0) ? iz <= zb : iz >= zb; iz += sgntz) {
                double tu = ls2d_init(&c, sgntz, sgntx, sgnvz, sgnvx, nz, nx,
                                      iz, ix, slow, tt);
                long id = (long)(ix - 1) * nz + iz - 1;
                tt[id] = dmin2(tt[id], tu);
            }
    }
    int converge = (conv_tol >= 0.0 && max_pass > 0);
    int npasses = converge ? max_pass : nsweep;
    int ran = 0;
    for (int it = 0; it < npasses; it++) {
        double dmax = 0.0;
        for (int sweep = 1; sweep <= 4; sweep++) {
            int sgntz, sgntx, sgnvz, sgnvx;
            sweep2d_signs(sweep, &sgntz, &sgntx, &sgnvz, &sgnvx);
            if (!fsm) {
                /* solver2D.F90:899-925: levels 2..nx+nz, i in
                 * [max(1,l-nz), min(nx,l-1)] */
                for (int level = 2; level <= nx + nz; level++) {
                    int i1 = imax(1, level - nz), i2 = imin(nx, level - 1);
                    for (int i = i1; i <= i2; i++) {
                        int ix = (sgntx > 0) ? i : nx + 1 - i;
                        int iz = (sgntz > 0) ? level - i : nz + 1 - (level - i);
                        /* solver2D.F90:377-434 isUpdateNode */
                        int upd = ((sgntx > 0) ? ix > 1 : ix < nx) &&
                                  ((sgntz > 0) ? iz > 1 : iz < nz);
                        if (!upd) continue;
                        double s1, s2, s3;
                        fetch_slow2d(slow, nz, nx, iz, ix, sgnvz, sgnvx, &s1, &s2, &s3);
                        double tv = tt[(long)(ix - 1) * nz + iz - sgntz - 1];
                        double te = tt[(long)(ix - sgntx - 1) * nz + iz - 1];
                        double tev = tt[(long)(ix - sgntx - 1) * nz + iz - sgntz - 1];
                        long id = (long)(ix - 1) * nz + iz - 1;
                        double tu = ls2d_noinit(&c, tv, te, tev, s1, s2, s3);
                        double tn = dmin2(tt[id], tu);
                        double d = fabs(tn - tt[id]);
                        if (d > dmax) dmax = d;
                        tt[id] = tn;
                    }
                }
            } else {
                /* solver2D.F90:1134-1268: natural loops */
                int ja = (sgntx > 0) ? 2 : nx - 1, jb = (sgntx > 0) ? nx : 1;
                int ia = (sgntz > 0) ? 2 : nz - 1, ib = (sgntz > 0) ? nz : 1;
                for (int j = ja; (sgntx > 0) ? j <= jb : j >= jb; j += sgntx)
                    for (int i = ia; (sgntz > 0) ? i <= ib : i >= ib; i += sgntz) {
                        double s1, s2, s3;
                        fetch_slow2d(slow, nz, nx, i, j, sgnvz, sgnvx, &s1, &s2, &s3);
                        double tv = tt[(long)(j - 1) * nz + i - sgntz - 1];
                        double te = tt[(long)(j - sgntx - 1) * nz + i - 1];
                        double tev = tt[(long)(j - sgntx - 1) * nz + i - sgntz - 1];
                        long id = (long)(j - 1) * nz + i - 1;
                        double tu = ls2d_noinit(&c, tv, te, tev, s1, s2, s3);
                        double tn = dmin2(tt[id], tu);
                        double d = fabs(tn - tt[id]);
                        if (d > dmax) dmax = d;
                        tt[id] = tn;
                    }
            }
        }
        ran++;
        if (converge && dmax <= conv_tol) break;
    }
    if (npass) *npass = ran;
    return 0;
}

/* ===================================================================== */
/* receiver.F90:62-164 / :217-313                                        */
/* ===================================================================== */
void orc_receiver_setup(int is3d, int nz, int nx, int ny, double z0, double x0,
                        double y0, double dz, double dx, double dy, int nrec,
                        const double *z, const double *x, const double *y,
                        int *zri, int *xri, int *yri, double *zdr, double *xdr,
                        double *ydr, int *ierr)
{
    int e = 0;
    if (!is3d) { ny = 1; dy = 1.0; y0 = 0.0; }
    for (int r = 0; r < nrec; r++) {
        double yr_in = is3d ? y[r] : y0;
        if (z[r] < z0 || z[r] > z0 + dz * (double)(nz - 1)) e++;
        if (x[r] < x0 || x[r] > x0 + dx * (double)(nx - 1)) e++;
        if (yr_in < y0 || yr_in > y0 + dy * (double)(ny - 1)) e++;
        double zr = (z[r] - z0) / dz, xr = (x[r] - x0) / dx, yr = (yr_in - y0) / dy;
        int iz = (int)(zr + 1.0), ix = (int)(xr + 1.0), iy = (int)(yr + 1.0);
        if (!is3d) iy = 1;
        zri[r] = imax(1, imin(nz - 1, iz));
        xri[r] = imax(1, imin(nx - 1, ix));
        yri[r] = imax(1, imin(ny - 1, iy));
        zdr[r] = z[r] - (z0 + dz * (double)(zri[r] - 1));
        xdr[r] = x[r] - (x0 + dx * (double)(xri[r] - 1));
        ydr[r] = yr_in - (y0 + dy * (double)(yri[r] - 1));
        if (!is3d) ydr[r] = 0.0;
    }
    *ierr = e;
}

void orc_receiver_interp(int is3d, int nz, int nx, int ny, double dz,
                         double dx, double dy, const double *tt, int nrec,
                         const int *zri, const int *xri, const int *yri,
                         const double *zdr, const double *xdr,
                         const double *ydr, double *ttr)
{
    const long nzx = (long)nz * nx;
    (void)ny;
    for (int r = 0; r < nrec; r++) {
#define G3(a, b, c) tt[((long)(c) - 1) * nzx + ((long)(b) - 1) * nz + (a) - 1]
        if (is3d) {
            int i = zri[r], j = xri[r], k = yri[r];
            double tt000 = G3(i, j, k), tt100 = G3(i + 1, j, k);
            double tt010 = G3(i, j + 1, k), tt110 = G3(i + 1, j + 1, k);
            double tt001 = G3(i, j, k + 1), tt101 = G3(i + 1, j, k + 1);
            double tt011 = G3(i, j + 1, k + 1), tt111 = G3(i + 1, j + 1, k + 1);
            double zd = zdr[r] / dz, xd = xdr[r] / dx, yd = ydr[r] / dy;
            double omz = 1.0 - zd;
            double c00 = tt000 * omz + tt100 * zd;
            double c01 = tt001 * omz + tt101 * zd;
            double c10 = tt010 * omz + tt110 * zd;
            double c11 = tt011 * omz + tt111 * zd;
            double omx = 1.0 - xd;
            double c0 = c00 * omx + c10 * xd;
            double c1 = c01 * omx + c11 * xd;
            ttr[r] = c0 * (1.0 - yd) + c1 * yd;
        } else {
            int i = zri[r], j = xri[r];
            double tt00 = G3(i, j, 1), tt10 = G3(i + 1, j, 1);
            double tt01 = G3(i, j + 1, 1), tt11 = G3(i + 1, j + 1, 1);
            double zd = zdr[r] / dz, xd = xdr[r] / dx;
            double omz = 1.0 - zd, omx = 1.0 - xd;
            ttr[r] = tt00 * omz * omx + tt10 * zd * omx + tt01 * omz * xd +
                     tt11 * zd * xd;
        }
#undef G3
    }
}

/* ===================================================================== */
/* analytic.F90                                                          */
/* ===================================================================== */
void orc_analytic_constant(int nz, int nx, int ny, double z0, double x0,
                           double y0, double dz, double dx, double dy,
                           double vconst, double zs, double xs, double ys,
                           double *tt)
{
    /* analytic.F90:618-662, 844-851 */
    for (int k = 0; k < ny; k++)
        for (int j = 0; j < nx; j++)
            for (int i = 0; i < nz; i++) {
                double x = x0 + (double)(float)j * dx;
                double y = y0 + (double)(float)k * dy;
                double z = z0 + (double)(float)i * dz;
                double dist = sqrt((x - xs) * (x - xs) + (y - ys) * (y - ys) +
                                   (z - zs) * (z - zs));
                tt[((long)k * nx + j) * nz + i] = dist / vconst;
            }
}

void orc_analytic_linear(int nz, int nx, int ny, double z0, double x0,
                         double y0, double dz, double dx, double dy,
                         double vtop, double vbottom, double zs, double xs,
                         double ys, double *tt)
{
    /* analytic.F90:871-890 initializeGradientVars */
    double ztop = z0, zbot = z0 + (double)(nz - 1) * dz;
    double vel0 = vtop + (vbottom - vtop) / (zbot - ztop) * zs;
    double slow0 = 1.0 / vel0;
    double gz = (vbottom - vel0) / (zbot - zs);
    double absG2 = gz * gz;
    double absG = sqrt(absG2);
    /* analytic.F90:456-528 (job 1) + acoshArg :853-869 */
    for (int k = 0; k < ny; k++)
        for (int j = 0; j < nx; j++)
            for (int i = 0; i < nz; i++) {
                double x = x0 + (double)(float)j * dx;
                double y = y0 + (double)(float)k * dy;
                double z = z0 + (double)(float)i * dz;
                double ddx = x - xs, ddy = y - ys, ddz = z - zs;
                double dist2 = ddx * ddx + ddy * ddy + ddz * ddz;
                double vel = vel0 + 0.0 * ddx + 0.0 * ddy + gz * ddz;
                double arg = 1.0 + 0.5 / vel * slow0 * absG2 * dist2;
                tt[((long)k * nx + j) * nz + i] = acosh(arg) / dmax2(1.0e-10, absG);
            }
}

/* ===================================================================== */
/* locate.F90:620-744 (FP32 L2 objective) and :112-126 (MINLOC)          */
/* ===================================================================== */
static void l2_block(int g1, int g2, int ldgrd, int ntf, const float *tables,
                     const float *obs, const float *wts,
                     const unsigned char *skip, float xnorm, float *obj,
                     float *t0)
{
    const float sqrtHalf = 0.70710677f; /* SQRT(0.5) in FP32, constants.F90 */
    for (int g = g1; g < g2; g++) { obj[g] = 0.0f; t0[g] = 0.0f; }
    for (int i = 0; i < ntf; i++) {
        if (skip[i]) continue;
        float wt = wts[i], toff = 0.0f, ob = obs[i];
        const float *tp = tables + (size_t)i * ldgrd;
        for (int g = g1; g < g2; g++) {
            float est = tp[g] + toff;
            float res = xnorm * (ob - est);
            t0[g] = t0[g] + wt * res;
        }
    }
    for (int i = 0; i < ntf; i++) {
        if (skip[i]) continue;
        float wt = sqrtHalf * wts[i], toff = 0.0f, ob = obs[i];
        const float *tp = tables + (size_t)i * ldgrd;
        for (int g = g1; g < g2; g++) {
            float est = tp[g] + t0[g] + toff;
            float res = wt * (ob - est);
            obj[g] = obj[g] + res * res;
        }
    }
}

static float wsum(int ntf, const float *wts)
{
    float s = 0.0f;
    for (int i = 0; i < ntf; i++) s = s + wts[i];
    return s;
}

void orc_locate_l2_field(int ngrd, int ldgrd, int ntf, const float *tables,
                         const float *obs, const float *wts,
                         const unsigned char *skip, int nthreads, float *obj,
                         float *t0)
{
    float xnorm = 1.0f / wsum(ntf, wts);
    int nth = nthreads;
#ifdef _OPENMP
    if (nth <= 0) nth = omp_get_max_threads();
#endif
#pragma omp parallel for schedule(static) num_threads(nth)
    for (int b = 0; b < ngrd; b += 512) {
        int g2 = (b + 512 < ngrd) ? b + 512 : ngrd;
        l2_block(b, g2, ldgrd, ntf, tables, obs, wts, skip, xnorm, obj, t0);
    }
}

void orc_locate_l2(int ngrd, int ldgrd, int ntf, const float *tables,
                   const float *obs, const float *wts,
                   const unsigned char *skip, int nthreads, int *optIndx,
                   float *t0Opt, float *objOpt)
{
    float *obj = (float *)malloc(sizeof(float) * (size_t)ngrd);
    float *t0 = (float *)malloc(sizeof(float) * (size_t)ngrd);
    orc_locate_l2_field(ngrd, ldgrd, ntf, tables, obs, wts, skip, nthreads,
                        obj, t0);
    int best = 0;
    for (int g = 1; g < ngrd; g++) if (obj[g] < obj[best]) best = g;
    *optIndx = best + 1;
    *t0Opt = t0[best];
    *objOpt = obj[best];
    free(obj);
    free(t0);
}

void orc_locate_l2_points64(int ngrd, int ldgrd, int ntf, const float *tables,
                            const float *obs, const float *wts,
                            const unsigned char *skip, int npts,
                            const int *pts, double *obj, double *t0)
{
    (void)ngrd;
    double sw = 0.0;
    for (int i = 0; i < ntf; i++) if (!skip[i]) sw += (double)wts[i];
    for (int p = 0; p < npts; p++) {
        int g = pts[p];
        double a = 0.0;
        for (int i = 0; i < ntf; i++) {
            if (skip[i]) continue;
            a += (double)wts[i] * ((double)obs[i] - (double)tables[(size_t)i * ldgrd + g]);
        }
        a /= sw;
        double o = 0.0;
        for (int i = 0; i < ntf; i++) {
            if (skip[i]) continue;
            double r = (double)wts[i] * ((double)obs[i] - (double)tables[(size_t)i * ldgrd + g] - a);
            o += 0.5 * r * r;
        }
        obj[p] = o;
        t0[p] = a;
    }
}

void orc_locate_l2_best64(int ngrd, int ldgrd, int ntf, const float *tables,
                          const double *obs, const double *wts, int nthreads,
                          int *idx, double *t0Opt, double *objOpt)
{
    /* locate.F90:675-708 evaluated in FP64 at every grid point; MINLOC
     * (first minimum) as locate.F90:122 */
    double sw = 0.0;
    for (int i = 0; i < ntf; i++) if (wts[i] > 0.0) sw += wts[i];
    int nth = nthreads > 0 ? nthreads : 1;
    double *bo = (double *)malloc(sizeof(double) * (size_t)nth);
    double *bt = (double *)malloc(sizeof(double) * (size_t)nth);
    int *bg = (int *)malloc(sizeof(int) * (size_t)nth);
    for (int t = 0; t < nth; t++) { bo[t] = HUGE_VAL; bt[t] = 0.0; bg[t] = -1; }
#pragma omp parallel num_threads(nth)
    {
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
        /* static contiguous chunks: each thread's first minimum is the
         * first within its chunk, chunks are merged in order below */
        long long lo = (long long)ngrd * tid / nth, hi = (long long)ngrd * (tid + 1) / nth;
        for (long long g = lo; g < hi; g++) {
            double a = 0.0;
            for (int i = 0; i < ntf; i++)
                if (wts[i] > 0.0) a += wts[i] * (obs[i] - (double)tables[(size_t)i * ldgrd + g]);
            a /= sw;
            double o = 0.0;
            for (int i = 0; i < ntf; i++)
                if (wts[i] > 0.0) {
                    double r = wts[i] * (obs[i] - (double)tables[(size_t)i * ldgrd + g] - a);
                    o += 0.5 * r * r;
                }
            if (o < bo[tid]) { bo[tid] = o; bt[tid] = a; bg[tid] = (int)g; }
        }
    }
    int best = 0;
    for (int t = 1; t < nth; t++)
        if (bo[t] < bo[best]) best = t;
    *idx = bg[best];
    *t0Opt = bt[best];
    *objOpt = bo[best];
    free(bo); free(bt); free(bg);
}

static int cmp_dbl(const void *a, const void *b)
{
    double x = *(const double *)a, y = *(const double *)b;
    return (x > y) - (x < y);
}

void orc_locate_l1_best64(int ngrd, int ldgrd, int ntf, const float *tables,
                          const double *obs, const double *wts, int nthreads,
                          int *idx, double *t0Opt, double *objOpt)
{
    double wv = 0.0;
    for (int i = 0; i < ntf; i++) if (wts[i] > 0.0) wv = wts[i];
    int nth = nthreads > 0 ? nthreads : 1;
    double *bo = (double *)malloc(sizeof(double) * (size_t)nth);
    double *bt = (double *)malloc(sizeof(double) * (size_t)nth);
    int *bg = (int *)malloc(sizeof(int) * (size_t)nth);
    for (int t = 0; t < nth; t++) { bo[t] = HUGE_VAL; bt[t] = 0.0; bg[t] = -1; }
#pragma omp parallel num_threads(nth)
    {
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
        double r[256];
        long long lo = (long long)ngrd * tid / nth, hi = (long long)ngrd * (tid + 1) / nth;
        for (long long g = lo; g < hi; g++) {
            int n = 0;
            for (int i = 0; i < ntf; i++)
                if (wts[i] > 0.0) r[n++] = obs[i] - (double)tables[(size_t)i * ldgrd + g];
            if (n == 0) continue;
            qsort(r, (size_t)n, sizeof(double), cmp_dbl);
            double t0 = (n % 2) ? r[n / 2] : 0.5 * (r[n / 2 - 1] + r[n / 2]);
            double o = 0.0;
            for (int i = 0; i < n; i++) o += fabs(r[i] - t0);
            o *= wv;
            if (o < bo[tid]) { bo[tid] = o; bt[tid] = t0; bg[tid] = (int)g; }
        }
    }
    int best = 0;
    for (int t = 1; t < nth; t++)
        if (bo[t] < bo[best]) best = t;
    *idx = bg[best];
    *t0Opt = bt[best];
    *objOpt = bo[best];
    free(bo); free(bt); free(bg);
}

/* ============================================================ gradient == */
/* solver3D.F90:1249-1321, loop by loop: interior forward differences along
 * z, x and y, then the last node of each axis backward. */
void orc_gradient3d(int nz, int nx, int ny, double dz, double dx, double dy,
                    const double *tt, double *g)
{
    const long nzx = (long)nz * nx;
    const long n = nzx * ny;
    for (long m = 0; m < 3 * n; m++) g[m] = 0.0;
    for (int iy = 0; iy < ny; iy++)
        for (int ix = 0; ix < nx; ix++)
            for (int iz = 0; iz < nz - 1; iz++) {
                const long m1 = iy * nzx + (long)ix * nz + iz, m2 = m1 + 1;
                g[3 * m1 + 2] = (tt[m2] - tt[m1]) / dz;
            }
    for (int iy = 0; iy < ny; iy++)
        for (int ix = 0; ix < nx - 1; ix++)
            for (int iz = 0; iz < nz; iz++) {
                const long m1 = iy * nzx + (long)ix * nz + iz, m2 = m1 + nz;
                g[3 * m1 + 0] = (tt[m2] - tt[m1]) / dx;
            }
    for (int iy = 0; iy < ny - 1; iy++)
        for (int ix = 0; ix < nx; ix++)
            for (int iz = 0; iz < nz; iz++) {
                const long m1 = iy * nzx + (long)ix * nz + iz, m2 = m1 + nzx;
                g[3 * m1 + 1] = (tt[m2] - tt[m1]) / dy;
            }
    if (nz > 1)
        for (int iy = 0; iy < ny; iy++)
            for (int ix = 0; ix < nx; ix++) {
                const long m2 = iy * nzx + (long)ix * nz + nz - 1, m1 = m2 - 1;
                g[3 * m2 + 2] = (tt[m2] - tt[m1]) / dz;
            }
    if (nx > 1)
        for (int iy = 0; iy < ny; iy++)
            for (int iz = 0; iz < nz; iz++) {
                const long m2 = iy * nzx + (long)(nx - 1) * nz + iz, m1 = m2 - nz;
                g[3 * m2 + 0] = (tt[m2] - tt[m1]) / dx;
            }
    if (ny > 1)
        for (int ix = 0; ix < nx; ix++)
            for (int iz = 0; iz < nz; iz++) {
                const long m2 = (long)(ny - 1) * nzx + (long)ix * nz + iz, m1 = m2 - nzx;
                g[3 * m2 + 1] = (tt[m2] - tt[m1]) / dy;
            }
}

/* solver2D.F90:984-1032, loop by loop: interior backward differences, then
 * the first node of each axis forward and the last backward. */
void orc_gradient2d(int nz, int nx, double dz, double dx, const double *tt,
                    double *gx, double *gz)
{
    for (long m = 0; m < (long)nz * nx; m++) gx[m] = gz[m] = 0.0;
    for (int ix = 0; ix < nx; ix++)
        for (int iz = 1; iz < nz - 1; iz++) {
            const long m2 = (long)ix * nz + iz, m1 = m2 - 1;
            gz[m2] = (tt[m2] - tt[m1]) / dz;
        }
    for (int ix = 1; ix < nx - 1; ix++)
        for (int iz = 0; iz < nz; iz++) {
            const long m2 = (long)ix * nz + iz, m1 = m2 - nz;
            gx[m2] = (tt[m2] - tt[m1]) / dx;
        }
    if (nz > 1)
        for (int ix = 0; ix < nx; ix++) {
            long m1 = (long)ix * nz, m2 = m1 + 1;
            gz[m1] = (tt[m2] - tt[m1]) / dz;
            m1 = (long)ix * nz + nz - 2; m2 = m1 + 1;
            gz[m2] = (tt[m2] - tt[m1]) / dz;
        }
    if (nx > 1)
        for (int iz = 0; iz < nz; iz++) {
            long m1 = iz, m2 = (long)nz + iz;
            gx[m1] = (tt[m2] - tt[m1]) / dx;
            m1 = (long)(nx - 2) * nz + iz; m2 = (long)(nx - 1) * nz + iz;
            gx[m2] = (tt[m2] - tt[m1]) / dx;
        }
}

/* ============================================================== rays 2D == */
/* rays.F90:449-670 (fteik_rays_trace2d), the integrators of :671-825
 * (Euler, midpoint and the reference's RK4, whose k2 is evaluated at
 * x_n + k1 and then halved) and evalf2d / bilinear (:843-999), for one ray
 * traced from its end point (xr, zr) to the source grid point (xs, zs), all
 * relative to the model origin.  Cell (ix, iz) of a position: 1-based,
 * INT(x/dx + 1) clamped to [1, n-1].  The reference's segmentation of the
 * path into cells (:560-640) overwrites its x coordinates and stops after
 * the first ray (a debugging PAUSE); here every integration step is split
 * exactly at the cell boundaries it crosses, consecutive pieces in one cell
 * merged, which is the (cell, length) list those lines intend.  Returns 0,
 * 1 when the ray does not reach the source within nx*nz steps (the
 * reference's limit), 2 when a capacity is too small. */
#define RAY_EPS 2.220446049250313e-16

static inline int ray_cell_ix(double x, double d, int n)
{
    int i = (int)(x / d + 1.0);
    return i < 1 ? 1 : (i > n - 1 ? n - 1 : i);
}

static inline double ray_bilinear(double x, double z, double x1, double z1, double x2, double z2,
                                  double c11, double c12, double c21, double c22)
{
    /* rays.F90:969-999 */
    double den = (x1 - x2) * (z1 - z2);
    double a0 = (c11 * x2 * z2 - c12 * x2 * z1 - c21 * x1 * z2 + c22 * x1 * z1) / den;
    double a1 = (-c11 * z2 + c12 * z1 + c21 * z2 - c22 * z1) / den;
    double a2 = (-c11 * x2 + c12 * x2 + c21 * x1 - c22 * x1) / den;
    double a3 = (c11 - c12 - c21 + c22) / den;
    return a0 + a1 * x + a2 * z + a3 * x * z;
}

typedef struct {
    int nz, nx;
    double dz, dx;
    const double *slow, *gx, *gz;
} ray_grid_t;

/* rays.F90:857-894 (evalf2d) */
static void ray_evalf(const ray_grid_t *g, double xn, double zn, double *d1, double *d3)
{
    const int ix = ray_cell_ix(xn, g->dx, g->nx), iz = ray_cell_ix(zn, g->dz, g->nz);
    const long icell = (long)(ix - 1) * (g->nz - 1) + iz;
    const double x1 = (double)(ix - 1) * g->dx, x2 = (double)ix * g->dx;
    const double z1 = (double)(iz - 1) * g->dz, z2 = (double)iz * g->dz;
    const long i11 = (long)(ix - 1) * g->nz + iz, i12 = i11 + 1, i21 = (long)ix * g->nz + iz, i22 = i21 + 1;
    double dtdx = ray_bilinear(xn, zn, x1, z1, x2, z2, g->gx[i11 - 1], g->gx[i12 - 1], g->gx[i21 - 1],
                               g->gx[i22 - 1]);
    double dtdz = ray_bilinear(xn, zn, x1, z1, x2, z2, g->gz[i11 - 1], g->gz[i12 - 1], g->gz[i21 - 1],
                               g->gz[i22 - 1]);
    *d1 = -dtdx / g->slow[icell - 1];
    *d3 = -dtdz / g->slow[icell - 1];
}

/* rays.F90:813-825 (updatePosition2D) */
static void ray_update(const ray_grid_t *g, double xn, double zn, double ds, double d1, double d3,
                       double *x1, double *z1)
{
    double a = xn + ds * d1, b = zn + ds * d3;
    double xmax = (double)(g->nx - 1) * g->dx - RAY_EPS, zmax = (double)(g->nz - 1) * g->dz - RAY_EPS;
    a = a > RAY_EPS ? a : RAY_EPS;
    *x1 = a < xmax ? a : xmax;
    b = b > RAY_EPS ? b : RAY_EPS;
    *z1 = b < zmax ? b : zmax;
}

static void ray_step(const ray_grid_t *g, int integrator, double ds, double xn, double zn, double *x1,
                     double *z1)
{
    double d1, d3;
    if (integrator == 2) {
        /* rays.F90:765-787 (updateMidpoint2D) */
        double xm, zm;
        ray_evalf(g, xn, zn, &d1, &d3);
        ray_update(g, xn, zn, 0.5 * ds, d1, d3, &xm, &zm);
        ray_evalf(g, xm, zm, &d1, &d3);
        ray_update(g, xn, zn, ds, d1, d3, x1, z1);
    } else if (integrator == 3) {
        /* rays.F90:671-712 (updateRK42D) */
        static const double dsscal[3] = {0.5, 0.5, 1.0};
        double k[4][2], xk, zk;
        ray_evalf(g, xn, zn, &k[0][0], &k[0][1]);
        k[0][0] = ds * k[0][0];
        k[0][1] = ds * k[0][1];
        ray_update(g, xn, zn, 1.0, k[0][0], k[0][1], &xk, &zk);
        for (int i = 1; i < 4; i++) {
            ray_evalf(g, xk, zk, &k[i][0], &k[i][1]);
            k[i][0] = ds * dsscal[i - 1] * k[i][0];
            k[i][1] = ds * dsscal[i - 1] * k[i][1];
            ray_update(g, xn, zn, 1.0, k[i][0], k[i][1], &xk, &zk);
        }
        d1 = 1.0 / 6.0 * (k[0][0] + 2.0 * (k[1][0] + k[2][0]) + k[3][0]);
        d3 = 1.0 / 6.0 * (k[0][1] + 2.0 * (k[1][1] + k[2][1]) + k[3][1]);
        ray_update(g, xn, zn, 1.0, d1, d3, x1, z1);
    } else {
        /* rays.F90:735-748 (updateEuler2D) */
        ray_evalf(g, xn, zn, &d1, &d3);
        ray_update(g, xn, zn, ds, d1, d3, x1, z1);
    }
}

/* Split the straight step (xa, za) -> (xb, zb) at the cell boundaries it
 * crosses; append (cell, length) pieces, merging a piece into the last entry
 * when it lies in the same cell. */
static int ray_split(const ray_grid_t *g, double xa, double za, double xb, double zb, int maxseg, int *cells,
                     double *lens, int *nseg)
{
    const double ddx = xb - xa, ddz = zb - za;
    const double L = sqrt(ddx * ddx + ddz * ddz);
    if (!(L > 0.0)) return 0;
    double tx[8], tz[8];
    int nxc = 0, nzc = 0;
    if (ddx != 0.0) {
        const double lo = xa < xb ? xa : xb, hi = xa < xb ? xb : xa;
        const int m0 = (int)floor(lo / g->dx) + 1, m1 = (int)ceil(hi / g->dx) - 1;
        for (int m = m0; m <= m1 && nxc < 8; m++) tx[nxc++] = ((double)m * g->dx - xa) / ddx;
        if (ddx < 0.0)
            for (int i = 0; i < nxc / 2; i++) { double t = tx[i]; tx[i] = tx[nxc - 1 - i]; tx[nxc - 1 - i] = t; }
    }
    if (ddz != 0.0) {
        const double lo = za < zb ? za : zb, hi = za < zb ? zb : za;
        const int m0 = (int)floor(lo / g->dz) + 1, m1 = (int)ceil(hi / g->dz) - 1;
        for (int m = m0; m <= m1 && nzc < 8; m++) tz[nzc++] = ((double)m * g->dz - za) / ddz;
        if (ddz < 0.0)
            for (int i = 0; i < nzc / 2; i++) { double t = tz[i]; tz[i] = tz[nzc - 1 - i]; tz[nzc - 1 - i] = t; }
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
            const int ix = ray_cell_ix(xm, g->dx, g->nx), iz = ray_cell_ix(zm, g->dz, g->nz);
            const int c = (ix - 1) * (g->nz - 1) + iz;
            const double len = (tnext - tprev) * L;
            if (*nseg > 0 && cells[*nseg - 1] == c) {
                lens[*nseg - 1] += len;
            } else {
                if (*nseg >= maxseg) return 2;
                cells[*nseg] = c;
                lens[*nseg] = len;
                (*nseg)++;
            }
            tprev = tnext;
        }
        if (tnext >= 1.0) break;
    }
    return 0;
}

int orc_ray2d(int nz, int nx, double dz, double dx, const double *slow, const double *tt, const double *gx,
              const double *gz, double xs, double zs, int integrator, double xr, double zr, int maxpts,
              double *px, double *pz, int *npts, int maxseg, int *cells, double *lens, int *nseg, double *tn,
              double *tne)
{
    const ray_grid_t g = {nz, nx, dz, dx, slow, gx, gz};
    const double ds = (dx < dz ? dx : dz) / 2.0;
    const double rad2 = (dx * dx + dz * dz) / 2.0;
    double xn = xr, zn = zr, t_n = 0.0, t_e = 0.0;
    int np = 0, ns = 0, done = 0;
    if (maxpts < 1) return 2;
    px[np] = xn; pz[np] = zn; np++;
    const long maxk = (long)nx * nz;
    for (long k = 1; k <= maxk; k++) {
        const int ix = ray_cell_ix(xn, dx, nx), iz = ray_cell_ix(zn, dz, nz);
        const double x1 = (double)(ix - 1) * dx, x2 = (double)ix * dx;
        const double z1 = (double)(iz - 1) * dz, z2 = (double)iz * dz;
        const long i11 = (long)(ix - 1) * nz + iz, i12 = i11 + 1, i21 = (long)ix * nz + iz, i22 = i21 + 1;
        const double c11 = tt[i11 - 1], c12 = tt[i12 - 1], c21 = tt[i21 - 1], c22 = tt[i22 - 1];
        double xn1, zn1;
        ray_step(&g, integrator, ds, xn, zn, &xn1, &zn1);
        if ((xn1 - xs) * (xn1 - xs) + (zn1 - zs) * (zn1 - zs) < rad2) {
            done = 1;
            xn1 = xs;
            zn1 = zs;
        }
        const long icell = (long)(ix - 1) * (nz - 1) + iz;
        t_e = t_e - (ray_bilinear(xn1, zn1, x1, z1, x2, z2, c11, c12, c21, c22) -
                     ray_bilinear(xn, zn, x1, z1, x2, z2, c11, c12, c21, c22));
        t_n = t_n + sqrt((xn1 - xn) * (xn1 - xn) + (zn1 - zn) * (zn1 - zn)) * slow[icell - 1];
        if (ray_split(&g, xn, zn, xn1, zn1, maxseg, cells, lens, &ns)) return 2;
        xn = xn1;
        zn = zn1;
        if (np >= maxpts) return 2;
        px[np] = xn; pz[np] = zn; np++;
        if (done) break;
    }
    *npts = np;
    *nseg = ns;
    *tn = t_n;
    *tne = t_e;
    return done ? 0 : 1;
}
