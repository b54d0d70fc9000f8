/*
 * fields.cu -- device-side data movement around the solver: slowness packing,
 * field export in the reference's three orderings (solver3D.F90:844-980,
 * solver2D.F90:1295-1420), receiver interpolation (receiver.F90:217-313) and
 * the analytic reference fields (analytic.F90:456-528,618-662,844-890).
 */
#include <cuda_runtime.h>
#include "fteik_dev.h"

namespace {

template <typename R>
__global__ void pack_slow_kernel(int nzc, int nxc, int nyc, int zcp,
                                 const double *__restrict__ in, R *__restrict__ out)
{
    const size_t n = (size_t)nzc * nxc * nyc;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n;
         e += (size_t)gridDim.x * blockDim.x) {
        const int iz = (int)(e % nzc);
        const size_t col = e / nzc;
        out[col * zcp + iz] = (R)in[e];
    }
}

/* Cell velocities (FP64, natural order) to padded slowness 1/v in the
 * working precision; *bad = 1 if a velocity is not positive. */
template <typename R>
__global__ void pack_vel_kernel(int nzc, int nxc, int nyc, int zcp, const double *__restrict__ vel,
                                R *__restrict__ out, int *__restrict__ bad)
{
    const size_t n = (size_t)nzc * nxc * nyc;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n;
         e += (size_t)gridDim.x * blockDim.x) {
        const int iz = (int)(e % nzc);
        const size_t col = e / nzc;
        const double v = vel[e];
        if (!(v > 0.0)) *bad = 1;
        out[col * zcp + iz] = (R)(1.0 / v);
    }
}

__global__ void gather64_kernel(const double *__restrict__ v, const long long *__restrict__ idx, int n,
                                double *__restrict__ out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = v[idx[i]];
}

/* order 0: natural, z fastest; 1: x fastest then y then z (XYZ, or XZ in 2D);
 * 2: z fastest, y, then x (ZYX). */
template <typename R>
__global__ void field_export_kernel(int nz, int nx, int ny, int zp, const R *__restrict__ tt,
                                    int order, double *__restrict__ out)
{
    const size_t n = (size_t)nz * nx * ny;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n;
         e += (size_t)gridDim.x * blockDim.x) {
        /* e enumerates the source layout [iy][ix][iz] */
        const int iz = (int)(e % nz);
        const size_t r = e / nz;
        const int ix = (int)(r % nx);
        const int iy = (int)(r / nx);
        size_t j;
        if (order == 1)
            j = ((size_t)iz * ny + iy) * nx + ix;
        else if (order == 2)
            j = ((size_t)ix * ny + iy) * nz + iz;
        else
            j = e;
        out[j] = (double)tt[((size_t)iy * nx + ix) * zp + iz];
    }
}

template <typename R>
__global__ void field_cell_kernel(int is3d, int nz, int nx, int ny, int zp,
                                  const R *__restrict__ tt, int order,
                                  double *__restrict__ out)
{
    const int nzc = nz - 1, nxc = nx - 1, nyc = is3d ? ny - 1 : 1;
    const size_t n = (size_t)nzc * nxc * nyc;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n;
         e += (size_t)gridDim.x * blockDim.x) {
        const int iz = (int)(e % nzc);
        const size_t r = e / nzc;
        const int ix = (int)(r % nxc);
        const int iy = (int)(r / nxc);
        size_t j;
        double v;
        if (is3d) {
            const R *b = tt + ((size_t)iy * nx + ix) * zp + iz;
            const size_t sx = zp, sy = (size_t)nx * zp;
            /* solver3D.F90:937-948: 0.125*SUM of the 8 corner nodes */
            double s = (double)b[0];
            s += (double)b[1];
            s += (double)b[sx];
            s += (double)b[sx + 1];
            s += (double)b[sy];
            s += (double)b[sy + 1];
            s += (double)b[sy + sx];
            s += (double)b[sy + sx + 1];
            v = 0.125 * s;
            j = (order == 1) ? ((size_t)iz * nyc + iy) * nxc + ix
                : (order == 2) ? ((size_t)ix * nyc + iy) * nzc + iz : e;
        } else {
            const R *b = tt + (size_t)ix * zp + iz;
            double s = (double)b[0];
            s += (double)b[1];
            s += (double)b[zp];
            s += (double)b[zp + 1];
            v = 0.25 * s;
            j = (order == 1) ? (size_t)iz * nxc + ix : e;
        }
        out[j] = v;
    }
}

/* receiver.F90:246-306 */
template <typename R>
__device__ double interp_one(int is3d, int nx, int zp, double dz, double dx, double dy,
                             const R *__restrict__ tt, int zri, int xri, int yri, double zdr,
                             double xdr, double ydr)
{
    const size_t sx = zp, sy = (size_t)nx * zp;
    if (is3d) {
        const R *b = tt + ((size_t)(yri - 1) * nx + (xri - 1)) * zp + (zri - 1);
        double tt000 = b[0], tt100 = b[1], tt010 = b[sx], tt110 = b[sx + 1];
        double tt001 = b[sy], tt101 = b[sy + 1], tt011 = b[sy + sx], tt111 = b[sy + sx + 1];
        double zd = zdr / dz, xd = xdr / dx, yd = ydr / dy;
        double omz = 1.0 - zd;
        double c00 = tt000 * omz + tt100 * zd;
        double c01 = tt001 * omz + tt101 * zd;
        double c10 = tt010 * omz + tt110 * zd;
        double c11 = tt011 * omz + tt111 * zd;
        double omx = 1.0 - xd;
        double c0 = c00 * omx + c10 * xd;
        double c1 = c01 * omx + c11 * xd;
        return c0 * (1.0 - yd) + c1 * yd;
    }
    const R *b = tt + (size_t)(xri - 1) * zp + (zri - 1);
    double tt00 = b[0], tt10 = b[1], tt01 = b[sx], tt11 = b[sx + 1];
    double zd = zdr / dz, xd = xdr / dx;
    double omz = 1.0 - zd, omx = 1.0 - xd;
    return tt00 * omz * omx + tt10 * zd * omx + tt01 * omz * xd + tt11 * zd * xd;
}

template <typename R>
__global__ void receivers_kernel(int is3d, int nx, int zp, double dz, double dx, double dy,
                                 const R *__restrict__ tt, int nrec, const int *__restrict__ ri,
                                 const double *__restrict__ rd, double *__restrict__ ttr)
{
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= nrec) return;
    ttr[r] = interp_one<R>(is3d, nx, zp, dz, dx, dy, tt, ri[r], ri[nrec + r], ri[2 * nrec + r],
                           rd[r], rd[nrec + r], rd[2 * nrec + r]);
}

template <typename R>
__global__ void receivers_batch_kernel(int is3d, int nx, int zp, double dz, double dx, double dy,
                                       void *const *__restrict__ fields, int nfield, int nrec,
                                       const int *__restrict__ ri, const double *__restrict__ rd,
                                       double *__restrict__ ttr)
{
    const size_t n = (size_t)nfield * nrec;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n;
         e += (size_t)gridDim.x * blockDim.x) {
        const int f = (int)(e / nrec), r = (int)(e % nrec);
        const R *tt = reinterpret_cast<const R *>(fields[f]);
        ttr[e] = interp_one<R>(is3d, nx, zp, dz, dx, dy, tt, ri[r], ri[nrec + r], ri[2 * nrec + r],
                               rd[r], rd[nrec + r], rd[2 * nrec + r]);
    }
}

/* solver3D.F90:1249-1321: forward differences along each axis, backward on
 * the axis' last node; g[3 m + 0, 1, 2] = dT/dx, dT/dy, dT/dz at node m
 * (natural order, z fastest), computed in FP64 from the field's values. */
template <typename R>
__global__ void gradient3d_kernel(int nz, int nx, int ny, int zp, double dz, double dx, double dy,
                                  const R *__restrict__ tt, double *__restrict__ g)
{
    const size_t n = (size_t)nz * nx * ny;
    const size_t sx = zp, sy = (size_t)nx * zp;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n;
         e += (size_t)gridDim.x * blockDim.x) {
        const int iz = (int)(e % nz);
        const size_t r = e / nz;
        const int ix = (int)(r % nx), iy = (int)(r / nx);
        const size_t b = (size_t)iy * sy + (size_t)ix * sx + iz;
        const double t = (double)tt[b];
        double gx = 0.0, gy = 0.0, gz = 0.0;
        if (nx > 1) gx = (ix < nx - 1) ? ((double)tt[b + sx] - t) / dx : (t - (double)tt[b - sx]) / dx;
        if (ny > 1) gy = (iy < ny - 1) ? ((double)tt[b + sy] - t) / dy : (t - (double)tt[b - sy]) / dy;
        if (nz > 1) gz = (iz < nz - 1) ? ((double)tt[b + 1] - t) / dz : (t - (double)tt[b - 1]) / dz;
        g[3 * e] = gx;
        g[3 * e + 1] = gy;
        g[3 * e + 2] = gz;
    }
}

/* solver2D.F90:984-1032: backward differences, forward on the axis' first
 * node; gx, gz at node m = ix nz + iz. */
__global__ void gradient2d_kernel(int nz, int nx, int zp, double dz, double dx, const double *__restrict__ tt,
                                  double *__restrict__ gx, double *__restrict__ gz)
{
    const size_t n = (size_t)nz * nx;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n;
         e += (size_t)gridDim.x * blockDim.x) {
        const int iz = (int)(e % nz), ix = (int)(e / nz);
        const size_t b = (size_t)ix * zp + iz;
        const double t = tt[b];
        double vz = 0.0, vx = 0.0;
        if (nz > 1) vz = (iz == 0) ? (tt[b + 1] - t) / dz : (t - tt[b - 1]) / dz;
        if (nx > 1) vx = (ix == 0) ? (tt[b + zp] - t) / dx : (t - tt[b - zp]) / dx;
        gz[e] = vz;
        gx[e] = vx;
    }
}

/* analytic.F90:618-662,844-851 (constant) and :456-528,853-890 (linear
 * vertical gradient, vel0 the velocity at the source depth measured from z0). */
struct AnaParams {
    int kind;
    double v0, vel0, slow0, gz, absG2, absG;
};

__device__ __forceinline__ AnaParams ana_params(int kind, int nz, double z0, double dz,
                                                double v0, double v1, double zs)
{
    AnaParams a;
    a.kind = kind;
    a.v0 = v0;
    const double zbot = z0 + (double)(nz - 1) * dz;
    a.vel0 = v0 + (v1 - v0) / (zbot - z0) * zs;
    a.slow0 = 1.0 / a.vel0;
    a.gz = (v1 - a.vel0) / (zbot - zs);
    a.absG2 = a.gz * a.gz;
    a.absG = sqrt(a.absG2);
    return a;
}

__device__ __forceinline__ double ana_time(const AnaParams &a, double x, double y, double z,
                                           double xs, double ys, double zs)
{
    const double ddx = x - xs, ddy = y - ys, ddz = z - zs;
    if (a.kind == 0) return sqrt(ddx * ddx + ddy * ddy + ddz * ddz) / a.v0;
    const double dist2 = ddx * ddx + ddy * ddy + ddz * ddz;
    const double vel = a.vel0 + 0.0 * ddx + 0.0 * ddy + a.gz * ddz;
    const double arg = 1.0 + 0.5 / vel * a.slow0 * a.absG2 * dist2;
    return acosh(arg) / (a.absG > 1.0e-10 ? a.absG : 1.0e-10);
}

__global__ void analytic_points_kernel(int kind, int nz, double z0, double dz, double v0,
                                       double v1, int npts, const double *__restrict__ z,
                                       const double *__restrict__ x, const double *__restrict__ y,
                                       int nsrc, const double *__restrict__ zs,
                                       const double *__restrict__ xs,
                                       const double *__restrict__ ys, int ldr,
                                       double *__restrict__ out)
{
    const size_t n = (size_t)nsrc * npts;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n;
         e += (size_t)gridDim.x * blockDim.x) {
        const int s = (int)(e / npts), p = (int)(e % npts);
        const AnaParams a = ana_params(kind, nz, z0, dz, v0, v1, zs[s]);
        out[(size_t)s * ldr + p] = ana_time(a, x[p], y[p], z[p], xs[s], ys[s], zs[s]);
    }
}

__global__ void f64_to_f32_kernel(size_t n, const double *__restrict__ in, float *__restrict__ out)
{
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n;
         e += (size_t)gridDim.x * blockDim.x)
        out[e] = (float)in[e];
}

/* analytic.F90: constant (kind 0) and linear vertical gradient (kind 1). */
__global__ void analytic_kernel(int kind, int nz, int nx, int ny, double z0, double x0,
                                double y0, double dz, double dx, double dy, double v0,
                                double v1, double zs, double xs, double ys,
                                double *__restrict__ out)
{
    const size_t n = (size_t)nz * nx * ny;
    const AnaParams a = ana_params(kind, nz, z0, dz, v0, v1, zs);
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n;
         e += (size_t)gridDim.x * blockDim.x) {
        const int iz = (int)(e % nz);
        const size_t r = e / nz;
        const int ix = (int)(r % nx), iy = (int)(r / nx);
        /* analytic.F90:470-472: REAL(i-1) is a single-precision conversion */
        const double x = x0 + (double)(float)ix * dx;
        const double y = y0 + (double)(float)iy * dy;
        const double z = z0 + (double)(float)iz * dz;
        out[e] = ana_time(a, x, y, z, xs, ys, zs);
    }
}

inline int nblocks(size_t n)
{
    size_t b = (n + 255) / 256;
    return (int)(b < 148 * 16 ? (b > 0 ? b : 1) : 148 * 16);
}

} // namespace

extern "C" int fk_pack_slowness(int precision, int is3d, int nz, int nx, int ny, int zcp,
                                const double *slow_nat, void *slow_dev, cudaStream_t s)
{
    const int nyc = is3d ? ny - 1 : 1;
    const size_t n = (size_t)(nz - 1) * (nx - 1) * nyc;
    if (precision == 8)
        pack_slow_kernel<double><<<nblocks(n), 256, 0, s>>>(nz - 1, nx - 1, nyc, zcp, slow_nat,
                                                           (double *)slow_dev);
    else
        pack_slow_kernel<float><<<nblocks(n), 256, 0, s>>>(nz - 1, nx - 1, nyc, zcp, slow_nat,
                                                          (float *)slow_dev);
    return (int)cudaGetLastError();
}

/* Cell slowness re-indexed by node z: out[c][iz] = slow[c][min(iz, nz-2)]
 * (copy 0) and slow[c][max(iz-1, 0)] (copy 1) for iz < zp (the padding
 * repeats the last cell), columns c over (ny-1)(nx-1). */
__global__ void node_slowness_kernel(int nz, int ncol, int zcp, int zp, const float *__restrict__ slow,
                                     float *__restrict__ out)
{
    const size_t n = (size_t)ncol * zp;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n;
         e += (size_t)gridDim.x * blockDim.x) {
        const int iz = (int)(e % zp);
        const size_t c = e / zp;
        const int up = min(iz, nz - 2), dn = min(max(iz - 1, 0), nz - 2);
        out[e] = slow[c * zcp + up];
        out[n + e] = slow[c * zcp + dn];
    }
}

extern "C" int fk_node_slowness_f32(int nz, int nx, int ny, int zcp, int zp, const float *slow_dev,
                                    float *slowz_dev, cudaStream_t s)
{
    const int ncol = (nx - 1) * (ny - 1);
    const size_t n = (size_t)ncol * zp;
    node_slowness_kernel<<<nblocks(n), 256, 0, s>>>(nz, ncol, zcp, zp, slow_dev, slowz_dev);
    return (int)cudaGetLastError();
}

extern "C" int fk_pack_velocity(int precision, int nz, int nx, int ny, int zcp, const double *vel_nat,
                                void *slow_dev, int *bad_dev, cudaStream_t s)
{
    const size_t n = (size_t)(nz - 1) * (nx - 1) * (ny - 1);
    if (precision == 8)
        pack_vel_kernel<double><<<nblocks(n), 256, 0, s>>>(nz - 1, nx - 1, ny - 1, zcp, vel_nat,
                                                          (double *)slow_dev, bad_dev);
    else
        pack_vel_kernel<float><<<nblocks(n), 256, 0, s>>>(nz - 1, nx - 1, ny - 1, zcp, vel_nat,
                                                         (float *)slow_dev, bad_dev);
    return (int)cudaGetLastError();
}

extern "C" int fk_gather64(const double *v, const long long *idx, int n, double *out, cudaStream_t s)
{
    if (n <= 0) return 0;
    gather64_kernel<<<(n + 255) / 256, 256, 0, s>>>(v, idx, n, out);
    return (int)cudaGetLastError();
}

extern "C" int fk_field_to_f64(int precision, int is3d, int nz, int nx, int ny, int zp,
                               const void *tt, int order, double *out, cudaStream_t s)
{
    /* 2D: XZ (order 1) is XYZ with ny = 1; ZYX does not exist */
    if (!is3d) { ny = 1; if (order != 1) order = 0; }
    const size_t n = (size_t)nz * nx * ny;
    if (precision == 8)
        field_export_kernel<double><<<nblocks(n), 256, 0, s>>>(nz, nx, ny, zp,
                                                              (const double *)tt, order, out);
    else
        field_export_kernel<float><<<nblocks(n), 256, 0, s>>>(nz, nx, ny, zp,
                                                             (const float *)tt, order, out);
    return (int)cudaGetLastError();
}

extern "C" int fk_field_cell_to_f64(int precision, int is3d, int nz, int nx, int ny, int zp,
                                    const void *tt, int order, double *out, cudaStream_t s)
{
    const size_t n = (size_t)(nz - 1) * (nx - 1) * (is3d ? ny - 1 : 1);
    if (precision == 8)
        field_cell_kernel<double><<<nblocks(n), 256, 0, s>>>(is3d, nz, nx, ny, zp,
                                                            (const double *)tt, order, out);
    else
        field_cell_kernel<float><<<nblocks(n), 256, 0, s>>>(is3d, nz, nx, ny, zp,
                                                           (const float *)tt, order, out);
    return (int)cudaGetLastError();
}

extern "C" int fk_receivers(int precision, int is3d, int nz, int nx, int ny, int zp,
                            double dz, double dx, double dy, const void *tt, int nrec,
                            const int *ri, const double *rd, double *ttr, cudaStream_t s)
{
    (void)nz; (void)ny;
    if (nrec <= 0) return 0;
    const int nb = (nrec + 127) / 128;
    if (precision == 8)
        receivers_kernel<double><<<nb, 128, 0, s>>>(is3d, nx, zp, dz, dx, dy,
                                                    (const double *)tt, nrec, ri, rd, ttr);
    else
        receivers_kernel<float><<<nb, 128, 0, s>>>(is3d, nx, zp, dz, dx, dy,
                                                   (const float *)tt, nrec, ri, rd, ttr);
    return (int)cudaGetLastError();
}

static int receivers_batch(int precision, int is3d, int nx, int zp, double dz, double dx, double dy,
                           void *const *fields, int nfield, int nrec, const int *ri, const double *rd,
                           double *ttr, cudaStream_t s)
{
    const size_t n = (size_t)nfield * nrec;
    if (n == 0) return 0;
    if (precision == 8)
        receivers_batch_kernel<double><<<nblocks(n), 256, 0, s>>>(is3d, nx, zp, dz, dx, dy, fields,
                                                                  nfield, nrec, ri, rd, ttr);
    else
        receivers_batch_kernel<float><<<nblocks(n), 256, 0, s>>>(is3d, nx, zp, dz, dx, dy, fields,
                                                                 nfield, nrec, ri, rd, ttr);
    return (int)cudaGetLastError();
}

extern "C" int fk_receivers_batch(int precision, int nz, int nx, int ny, int zp, double dz,
                                  double dx, double dy, void *const *fields, int nfield,
                                  int nrec, const int *ri, const double *rd, double *ttr,
                                  cudaStream_t s)
{
    (void)nz; (void)ny;
    return receivers_batch(precision, 1, nx, zp, dz, dx, dy, fields, nfield, nrec, ri, rd, ttr, s);
}

extern "C" int fk_receivers_batch2d(int nx, int zp, double dz, double dx, void *const *fields, int nfield,
                                    int nrec, const int *ri, const double *rd, double *ttr, cudaStream_t s)
{
    return receivers_batch(8, 0, nx, zp, dz, dx, 1.0, fields, nfield, nrec, ri, rd, ttr, s);
}

extern "C" int fk_analytic_field(int kind, int nz, int nx, int ny, double z0, double x0,
                                 double y0, double dz, double dx, double dy, double v0,
                                 double v1, double zs, double xs, double ys, double *out,
                                 cudaStream_t s)
{
    const size_t n = (size_t)nz * nx * ny;
    analytic_kernel<<<nblocks(n), 256, 0, s>>>(kind, nz, nx, ny, z0, x0, y0, dz, dx, dy, v0, v1,
                                               zs, xs, ys, out);
    return (int)cudaGetLastError();
}

extern "C" int fk_analytic_points(int kind, int nz, double z0, double dz, double v0, double v1,
                                  int npts, const double *z, const double *x, const double *y,
                                  int nsrc, const double *zs, const double *xs, const double *ys,
                                  int ldr, double *out, cudaStream_t s)
{
    const size_t n = (size_t)nsrc * npts;
    if (n == 0) return 0;
    analytic_points_kernel<<<nblocks(n), 256, 0, s>>>(kind, nz, z0, dz, v0, v1, npts, z, x, y,
                                                      nsrc, zs, xs, ys, ldr, out);
    return (int)cudaGetLastError();
}

extern "C" int fk_f64_to_f32(size_t n, const double *in, float *out, cudaStream_t s)
{
    if (n == 0) return 0;
    f64_to_f32_kernel<<<nblocks(n), 256, 0, s>>>(n, in, out);
    return (int)cudaGetLastError();
}

namespace {
/* Copy nfield padded FP32 fields ([nyx rows][zp]) into a dense [nyx][nz]
 * buffer, 16-byte vectors where the pitch allows. */
__global__ void unpad_kernel(const float *__restrict__ src, float *__restrict__ dst, size_t rows,
                             int nz, int zp)
{
    const size_t n = rows * (size_t)nz;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n;
         e += (size_t)gridDim.x * blockDim.x) {
        const size_t r = e / nz;
        const int z = (int)(e - r * nz);
        dst[e] = src[r * zp + z];
    }
}
} // namespace

extern "C" int fk_unpad_f32(const float *src, float *dst, size_t rows, int nz, int zp, cudaStream_t s)
{
    if (rows == 0) return 0;
    unpad_kernel<<<148 * 8, 256, 0, s>>>(src, dst, rows, nz, zp);
    return (int)cudaGetLastError();
}

extern "C" int fk_gradient3d(int precision, int nz, int nx, int ny, int zp, double dz, double dx, double dy,
                             const void *tt, double *g, cudaStream_t s)
{
    const size_t n = (size_t)nz * nx * ny;
    if (n == 0) return 0;
    if (precision == 8)
        gradient3d_kernel<double><<<nblocks(n), 256, 0, s>>>(nz, nx, ny, zp, dz, dx, dy,
                                                             (const double *)tt, g);
    else
        gradient3d_kernel<float><<<nblocks(n), 256, 0, s>>>(nz, nx, ny, zp, dz, dx, dy,
                                                            (const float *)tt, g);
    return (int)cudaGetLastError();
}

extern "C" int fk_gradient2d(int nz, int nx, int zp, double dz, double dx, const double *tt, double *gx,
                             double *gz, cudaStream_t s)
{
    const size_t n = (size_t)nz * nx;
    if (n == 0) return 0;
    gradient2d_kernel<<<nblocks(n), 256, 0, s>>>(nz, nx, zp, dz, dx, tt, gx, gz);
    return (int)cudaGetLastError();
}
