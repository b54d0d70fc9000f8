/*
 * host_model.c -- the reference's model, source and receiver modules
 * (model.F90, source.F90, receiver.F90): geometry, velocity-to-slowness
 * conversion, source snapping and receiver cell lookup.  These run once per
 * set-up call on the host in FP64, exactly as the reference does; the
 * device copy of the slowness is made lazily in the solver's precision.
 */
#include "host_common.h"
#include "fteik_b200.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

fk_model_t fk_model;
fk_source_t fk_source;
fk_receiver_t fk_receiver;

static int imin(int a, int b) { return a < b ? a : b; }
static int imax(int a, int b) { return a > b ? a : b; }

/* ------------------------------------------------------------ geometry -- */
void fk_model_invalidate_dev(void)
{
    fk_model.dev32_ok = false;
    fk_model.dev64_ok = false;
    fk_model.devz_ok = false;
}

void fteik_model_free(void)
{
    free(fk_model.slow);
    fk_dfree(fk_model.slow_dev32);
    fk_dfree(fk_model.slow_dev64);
    fk_dfree(fk_model.slowz_dev);
    memset(&fk_model, 0, sizeof(fk_model));
    fk_model.lis3d = true;
}

void fteik_model_setGridSize(bool lis3d, int nz, int nx, int ny, int *ierr)
{
    /* model.F90:181-216 */
    *ierr = 0;
    fk_model.nz = fk_model.nx = fk_model.ny = 0;
    fk_model.ngrd = fk_model.ncell = 0;
    if (nz < 3 || nx < 3 || (lis3d && ny < 3)) {
        if (nz < 3) FK_ERR("fteik_model_setGridSize: nz=%d must be at least 3", nz);
        if (nx < 3) FK_ERR("fteik_model_setGridSize: nx=%d must be at least 3", nx);
        if (lis3d && ny < 3) FK_ERR("fteik_model_setGridSize: ny=%d must be at least 3", ny);
        *ierr = 1;
        return;
    }
    if (!lis3d) ny = 1;
    long long ngrd = (long long)nz * nx * ny;
    if (ngrd > 2147483647LL) {
        FK_ERR("fteik_model_setGridSize: grid of %lld nodes exceeds the int index range", ngrd);
        *ierr = 1;
        return;
    }
    fk_model.nz = nz; fk_model.nx = nx; fk_model.ny = ny;
    fk_model.ncell = (nz - 1) * (nx - 1) * imax(1, ny - 1);
    fk_model.ngrd = (int)ngrd;
    free(fk_model.slow);
    fk_model.slow = (double *)calloc((size_t)fk_model.ncell, sizeof(double));
    fk_dfree(fk_model.slow_dev32); fk_model.slow_dev32 = NULL;
    fk_dfree(fk_model.slow_dev64); fk_model.slow_dev64 = NULL;
    fk_dfree(fk_model.slowz_dev); fk_model.slowz_dev = NULL;
    fk_model_invalidate_dev();
    fk_model.have_model = false;
}

void fteik_model_setGridSpacing(bool lis3d, double dz, double dx, double dy, int *ierr)
{
    /* model.F90:134-172 */
    *ierr = 0;
    fk_model.dz = fk_model.dx = fk_model.dy = 0.0;
    if (dz <= 0.0 || dx <= 0.0 || (lis3d && dy <= 0.0)) {
        FK_ERR("fteik_model_setGridSpacing: grid spacing must be positive");
        *ierr = 1;
        return;
    }
    fk_model.dz = dz;
    fk_model.dx = dx;
    fk_model.dy = lis3d ? dy : 1.0;
}

void fteik_model_setOrigin3D(double z0, double x0, double y0)
{
    fk_model.z0 = z0; fk_model.x0 = x0; fk_model.y0 = y0;
}

void fteik_model_setOrigin2D(double z0, double x0)
{
    fk_model.z0 = z0; fk_model.x0 = x0; fk_model.y0 = 0.0;
}

void fteik_model_initializeGeometry(bool lis3d, int nz, int nx, int ny, double z0,
                                    double x0, double y0, double dz, double dx,
                                    double dy, int *ierr)
{
    /* model.F90:88-129 */
    fk_model.lis3d = lis3d;
    fk_model.have_geom = false;
    fteik_model_setGridSize(lis3d, nz, nx, ny, ierr);
    if (*ierr) { FK_ERR("fteik_model_initializeGeometry: Error setting grid size"); return; }
    fteik_model_setGridSpacing(lis3d, dz, dx, dy, ierr);
    if (*ierr) { FK_ERR("fteik_model_initializeGeometry: Error setting grid spacing"); return; }
    if (lis3d) fteik_model_setOrigin3D(z0, x0, y0);
    else fteik_model_setOrigin2D(z0, x0);
    fk_model.have_geom = true;
}

void fteik_model_getGridSize(int *nz, int *nx, int *ny, int *ngrd, int *ncell, int *ierr)
{
    *ierr = 0;
    *nz = *nx = *ny = *ngrd = *ncell = 0;
    if (fk_model.nx < 1 || fk_model.nz < 1) {
        FK_ERR("fteik_model_getGridSize: Grid not yet set");
        *ierr = 1;
        return;
    }
    *nz = fk_model.nz; *nx = fk_model.nx; *ny = fk_model.ny;
    *ngrd = fk_model.ngrd; *ncell = fk_model.ncell;
}

int fteik_model_grid2indexF(int i, int j, int k, int nz, int nzx)
{
    return (k - 1) * nzx + (j - 1) * nz + i;
}

int fteik_model_grid2index(int iz, int ix, int iy, int nz, int nzx)
{
    return fteik_model_grid2indexF(iz + 1, ix + 1, iy + 1, nz, nzx) - 1;
}

void fteik_model_index2gridF(int igrd, int *i, int *j, int *k, int *ierr)
{
    /* model.F90:790-810 */
    const int nz = fk_model.nz, nx = fk_model.nx, ny = fk_model.ny;
    const int nzx = nz * nx;
    int g = igrd - 1;
    *k = nzx > 0 ? g / nzx : 0;
    *j = nz > 0 ? (g - *k * nzx) / nz : 0;
    *i = g - *k * nzx - *j * nz;
    *k += 1; *j += 1; *i += 1;
    *ierr = 0;
    if (*i < 1 || *i > nz) *ierr += 1;
    if (*j < 1 || *j > nx) *ierr += 1;
    if (*k < 1 || *k > ny) *ierr += 1;
}

int fteik_model_velGrid2indexF(int i, int j, int k, int nzm1, int nzm1_nxm1)
{
    return (k - 1) * nzm1_nxm1 + (j - 1) * nzm1 + i;
}

/* --------------------------------------------------------- velocities -- */
static int check_positive(const double *v, long n, const char *who)
{
    double vmin = v[0];
    for (long i = 1; i < n; i++) if (v[i] < vmin) vmin = v[i];
    if (!(vmin > 0.0)) {
        FK_ERR("%s: velocities must be positive (min %g)", who, vmin);
        return 1;
    }
    return 0;
}

void fteik_model_setVelocityModel64f(int nv, const double vel[], int *ierr)
{
    /* model.F90:719-754 */
    *ierr = 0;
    fk_model.have_model = false;
    if (nv != fk_model.ncell || nv < 1) {
        FK_ERR("fteik_model_setVelocityModel64f: ncell=%d but nv=%d", fk_model.ncell, nv);
        *ierr = 1;
        return;
    }
    if (check_positive(vel, nv, "fteik_model_setVelocityModel64f")) { *ierr = 1; return; }
    for (int i = 0; i < nv; i++) fk_model.slow[i] = 1.0 / vel[i];
    fk_model_invalidate_dev();
    fk_model.have_model = true;
}

void fteik_model_setVelocityModel32f(int nv, const float vel4[], int *ierr)
{
    /* model.F90:719-754: slow = 1 / DBLE(vel4) */
    *ierr = 0;
    fk_model.have_model = false;
    if (nv != fk_model.ncell || nv < 1) {
        FK_ERR("fteik_model_setVelocityModel32f: ncell=%d but nv=%d", fk_model.ncell, nv);
        *ierr = 1;
        return;
    }
    float vmin = vel4[0];
    for (int i = 1; i < nv; i++) if (vel4[i] < vmin) vmin = vel4[i];
    if (!(vmin > 0.0f)) {
        FK_ERR("fteik_model_setVelocityModel32f: All velocities must be positive");
        *ierr = 1;
        return;
    }
    for (int i = 0; i < nv; i++) fk_model.slow[i] = 1.0 / (double)vel4[i];
    fk_model_invalidate_dev();
    fk_model.have_model = true;
}

void fteik_model_getVelocityModel64f(int nwork, int *nv, double vel[], int *ierr)
{
    /* model.F90:651-688 */
    *ierr = 0;
    *nv = 0;
    if (nwork == -1) {
        *nv = fk_model.ncell;
        return;
    }
    if (nwork < fk_model.ncell) {
        FK_ERR("fteik_model_getVelocityModel64f: nv < ncell");
        *ierr = 1;
        return;
    }
    if (!fk_model.have_model) {
        FK_ERR("fteik_model_getVelocityModel64f: Velocity model not yet set");
        for (int i = 0; i < nwork; i++) vel[i] = 0.0;
        *ierr = 1;
        return;
    }
    for (int i = 0; i < fk_model.ncell; i++) vel[i] = 1.0 / fk_model.slow[i];
    for (int i = fk_model.ncell; i < nwork; i++) vel[i] = 0.0;
    *nv = fk_model.ncell;
}

void fteik_model_isModel3D(bool *lis3d, int *ierr)
{
    /* model.F90:692-706 */
    *ierr = 0;
    *lis3d = fk_model.lis3d;
    if (!fk_model.have_geom || fk_model.nx < 1 || fk_model.nz < 1) {
        FK_ERR("fteik_model_isModel3D: Model not yet initialized");
        *ierr = 1;
    }
}

void fteik_model_setCellVelocityModel64f(int nc, int order, const double vel[], int *ierr)
{
    /* model.F90:505-607 */
    *ierr = 0;
    fk_model.have_model = false;
    const int ncell = fk_model.ncell;
    if (nc < ncell || nc < 1) {
        FK_ERR("fteik_model_setCellVelocityModel64f: nc must be at least %d", ncell);
        *ierr = 1;
        return;
    }
    if (check_positive(vel, nc, "fteik_model_setCellVelocityModel64f")) { *ierr = 1; return; }
    const int nzm1 = fk_model.nz - 1, nxm1 = fk_model.nx - 1;
    if (fk_model.lis3d && order == FTEIK_XYZ_ORDERING) {
        const int nym1 = fk_model.ny - 1;
        for (int iy = 0; iy < nym1; iy++)
            for (int ix = 0; ix < nxm1; ix++)
                for (int iz = 0; iz < nzm1; iz++)
                    fk_model.slow[((long)iy * nxm1 + ix) * nzm1 + iz] =
                        1.0 / vel[(long)iz * nxm1 * nym1 + (long)iy * nxm1 + ix];
    } else if (fk_model.lis3d && order == FTEIK_ZYX_ORDERING) {
        const int nym1 = fk_model.ny - 1;
        for (int iy = 0; iy < nym1; iy++)
            for (int ix = 0; ix < nxm1; ix++)
                for (int iz = 0; iz < nzm1; iz++)
                    fk_model.slow[((long)iy * nxm1 + ix) * nzm1 + iz] =
                        1.0 / vel[(long)ix * nzm1 * nym1 + (long)iy * nzm1 + iz];
    } else if (!fk_model.lis3d && order == FTEIK_XZ_ORDERING) {
        for (int ix = 0; ix < nxm1; ix++)
            for (int iz = 0; iz < nzm1; iz++)
                fk_model.slow[(long)ix * nzm1 + iz] = 1.0 / vel[(long)iz * nxm1 + ix];
    } else {
        if (order != FTEIK_NATURAL_ORDERING && fk_model.verbose > 0)
            fprintf(stdout, "fteik_model_setCellVelocityModel64f: Defaulting to natural order\n");
        for (int i = 0; i < ncell; i++) fk_model.slow[i] = 1.0 / vel[i];
    }
    fk_model_invalidate_dev();
    fk_model.have_model = true;
}

void fteik_model_setNodalVelocityModel64f(int ng, int order, const double vel[], int *ierr)
{
    /* model.F90:311-449.  Nodal velocities are averaged over the 8 (3D) or 4
     * (2D) corners of each cell.  The reference's XYZ branch omits the 1/8
     * factor (model.F90:353) and its natural branch reuses one y-plane
     * (model.F90:386-389); both are treated as defects and the average is
     * taken over the cell's true corners. */
    *ierr = 0;
    fk_model.have_model = false;
    const int nz = fk_model.nz, nx = fk_model.nx, ny = fk_model.ny;
    if (ng < fk_model.ngrd || ng < 1) {
        FK_ERR("fteik_model_setNodalVelocityModel64f: ng must be at least %d", fk_model.ngrd);
        *ierr = 1;
        return;
    }
    if (check_positive(vel, ng, "fteik_model_setNodalVelocityModel64f")) { *ierr = 1; return; }
    const int nzm1 = nz - 1, nxm1 = nx - 1;
    if (fk_model.lis3d) {
        const int nym1 = ny - 1;
        for (int iy = 1; iy <= nym1; iy++)
            for (int ix = 1; ix <= nxm1; ix++)
                for (int iz = 1; iz <= nzm1; iz++) {
                    long id[8];
                    if (order == FTEIK_XYZ_ORDERING) {
                        long b = (long)nx * ny;
                        id[0] = (iz - 1) * b + (long)(iy - 1) * nx + ix;
                        id[2] = (iz - 1) * b + (long)iy * nx + ix;
                        id[4] = (long)iz * b + (long)(iy - 1) * nx + ix;
                        id[6] = (long)iz * b + (long)iy * nx + ix;
                    } else if (order == FTEIK_ZYX_ORDERING) {
                        long b = (long)ny * nz;
                        id[0] = (long)(ix - 1) * b + (long)(iy - 1) * nz + iz;
                        id[2] = (long)(ix - 1) * b + (long)iy * nz + iz;
                        id[4] = (long)ix * b + (long)(iy - 1) * nz + iz;
                        id[6] = (long)ix * b + (long)iy * nz + iz;
                    } else {
                        long nzx = (long)nz * nx;
                        id[0] = (iy - 1) * nzx + (long)(ix - 1) * nz + iz;
                        id[2] = (iy - 1) * nzx + (long)ix * nz + iz;
                        id[4] = (long)iy * nzx + (long)(ix - 1) * nz + iz;
                        id[6] = (long)iy * nzx + (long)ix * nz + iz;
                    }
                    id[1] = id[0] + 1; id[3] = id[2] + 1; id[5] = id[4] + 1; id[7] = id[6] + 1;
                    double s = 0.0;
                    for (int m = 0; m < 8; m++) s += vel[id[m] - 1];
                    fk_model.slow[((long)(iy - 1) * nxm1 + (ix - 1)) * nzm1 + (iz - 1)] =
                        1.0 / (s * 0.125);
                }
    } else {
        for (int ix = 1; ix <= nxm1; ix++)
            for (int iz = 1; iz <= nzm1; iz++) {
                long id[4];
                if (order == FTEIK_XZ_ORDERING) {
                    id[0] = (long)(iz - 1) * nx + ix; id[2] = (long)iz * nx + ix;
                } else {
                    id[0] = (long)(ix - 1) * nz + iz; id[2] = (long)ix * nz + iz;
                }
                id[1] = id[0] + 1; id[3] = id[2] + 1;
                double s = 0.0;
                for (int m = 0; m < 4; m++) s += vel[id[m] - 1];
                fk_model.slow[(long)(ix - 1) * nzm1 + (iz - 1)] = 1.0 / (s * 0.25);
            }
    }
    fk_model_invalidate_dev();
    fk_model.have_model = true;
}

const void *fk_model_slow_dev(int precision)
{
    /* Upload the slowness once per model in the solve's precision. */
    const int nz = fk_model.nz, nx = fk_model.nx, ny = fk_model.ny;
    const int zcp = FK_PITCH(nz - 1);
    const int nyc = fk_model.lis3d ? ny - 1 : 1;
    const size_t nelem = (size_t)zcp * (nx - 1) * nyc;
    void **slot = precision == 8 ? &fk_model.slow_dev64 : &fk_model.slow_dev32;
    bool *ok = precision == 8 ? &fk_model.dev64_ok : &fk_model.dev32_ok;
    if (*ok) return *slot;
    if (!*slot) {
        *slot = fk_dalloc(nelem * (size_t)precision, "fteik_model");
        if (!*slot) return NULL;
    }
    double *tmp = (double *)fk_dalloc(sizeof(double) * (size_t)fk_model.ncell, "fteik_model");
    if (!tmp) return NULL;
    int e = (int)cudaMemsetAsync(*slot, 0, nelem * (size_t)precision, fk_stream());
    if (!e) e = (int)cudaMemcpyAsync(tmp, fk_model.slow, sizeof(double) * (size_t)fk_model.ncell,
                                    cudaMemcpyHostToDevice, fk_stream());
    if (!e) e = fk_pack_slowness(precision, fk_model.lis3d, nz, nx, ny, zcp, tmp, *slot, fk_stream());
    if (!e) e = (int)cudaStreamSynchronize(fk_stream());
    fk_dfree(tmp);
    if (fk_check(e, "fteik_model: slowness upload")) return NULL;
    *ok = true;
    return *slot;
}

const float *fk_model_slowz_dev(void)
{
    /* the FP32 node-indexed slowness copies of the staged pass step, from
     * the padded FP32 cell slowness */
    if (fk_model.devz_ok) return fk_model.slowz_dev;
    if (!fk_model.lis3d) return NULL;
    const float *slow = (const float *)fk_model_slow_dev(4);
    if (!slow) return NULL;
    const int nz = fk_model.nz, nx = fk_model.nx, ny = fk_model.ny;
    const size_t n = (size_t)2 * (nx - 1) * (ny - 1) * FK_PITCH(nz);
    if (!fk_model.slowz_dev) {
        fk_model.slowz_dev = (float *)fk_dalloc(sizeof(float) * n, "fteik_model");
        if (!fk_model.slowz_dev) return NULL;
    }
    int e = fk_node_slowness_f32(nz, nx, ny, FK_PITCH(nz - 1), FK_PITCH(nz), slow, fk_model.slowz_dev,
                                 fk_stream());
    if (!e) e = (int)cudaStreamSynchronize(fk_stream());
    if (fk_check(e, "fteik_model: node-indexed slowness")) return NULL;
    fk_model.devz_ok = true;
    return fk_model.slowz_dev;
}

/* -------------------------------------------------------------- source -- */
int fk_snap_source(bool is3d, int nz, int nx, int ny, double z0, double x0, double y0,
                   double dz, double dx, double dy, double zsrc, double xsrc, double ysrc,
                   int isrc, int *zsi, int *xsi, int *ysi, double *zsa, double *xsa,
                   double *ysa)
{
    /* source.F90:133-179 */
    const double eps = 2.220446049250313e-16, perturb = 0.0001;
    if (!is3d) { ny = 1; dy = 1.0; y0 = 0.0; ysrc = 0.0; }
    double zmax = (double)(nz - 1) * dz, xmax = (double)(nx - 1) * dx, ymax = (double)(ny - 1) * dy;
    double zl = zsrc - z0, xl = xsrc - x0, yl = ysrc - y0;
    if (zl < 0.0 || zl > zmax || xl < 0.0 || xl > xmax || yl < 0.0 || yl > ymax) {
        if (zl < 0.0 || zl > zmax)
            FK_ERR("fteik_source_initialize64f: src=%d zsrc=%12.5e must be in range [%12.5e,%12.5e]",
                   isrc, zsrc, z0, zmax + z0);
        if (xl < 0.0 || xl > xmax)
            FK_ERR("fteik_source_initialize64f: src=%d xsrc=%12.5e must be in range [%12.5e,%12.5e]",
                   isrc, xsrc, x0, xmax + x0);
        if (yl < 0.0 || yl > ymax)
            FK_ERR("fteik_source_initialize64f: src=%d ysrc=%12.5e must be in range [%12.5e,%12.5e]",
                   isrc, ysrc, y0, ymax + y0);
        return 1;
    }
    double za = zl / dz + 1.0, xa = xl / dx + 1.0, ya = yl / dy + 1.0;
    if (fabs(za - 1.0) < eps) za = za + perturb;
    if (za >= (double)nz) za = za - perturb;
    if (fabs(xa - 1.0) < eps) xa = xa + perturb;
    if (xa >= (double)nx) xa = xa - perturb;
    if (fabs(ya - 1.0) < eps) ya = ya + perturb;
    if (ya >= (double)ny) ya = ya - perturb;
    int zi = (int)za, xi = (int)xa, yi = (int)ya;
    if (!is3d) { yi = 1; ya = 1.0; }
    if (zi < 1 || zi > nz || xi < 1 || xi > nx || (is3d && (yi < 1 || yi > ny))) {
        FK_ERR("fteik_source_initialize64f: Point (%d%d%d) out of bounds", zi, xi, yi);
        return 1;
    }
    *zsi = zi; *xsi = xi; *ysi = yi;
    *zsa = za; *xsa = xa; *ysa = ya;
    return 0;
}

void fteik_source_setVerbosity(int verbose) { fk_source.verbose = verbose; }

void fteik_source_free(void)
{
    free(fk_source.zsi); free(fk_source.xsi); free(fk_source.ysi);
    free(fk_source.zsa); free(fk_source.xsa); free(fk_source.ysa);
    free(fk_source.zs_true); free(fk_source.xs_true); free(fk_source.ys_true);
    memset(&fk_source, 0, sizeof(fk_source));
}

void fteik_source_initialize64f(int nsrc, const double zsrc[], const double xsrc[],
                                const double ysrc[], int verbose, int *ierr)
{
    /* source.F90:82-236 */
    *ierr = 0;
    fteik_source_free();
    fk_source.verbose = verbose;
    if (nsrc < 1) { FK_ERR("fteik_source_initialize64fF: No sources"); *ierr = 1; return; }
    if (fk_model.nz < 1 || fk_model.nx < 1 || fk_model.ny < 1 || fk_model.dz <= 0.0 ||
        fk_model.dx <= 0.0 || fk_model.dy <= 0.0) {
        FK_ERR("fteik_source_initialize64fF: Model not yet set");
        *ierr = 1;
        return;
    }
    fk_source.nsrc = nsrc;
    fk_source.zsi = (int *)calloc((size_t)nsrc, sizeof(int));
    fk_source.xsi = (int *)calloc((size_t)nsrc, sizeof(int));
    fk_source.ysi = (int *)calloc((size_t)nsrc, sizeof(int));
    fk_source.zsa = (double *)calloc((size_t)nsrc, sizeof(double));
    fk_source.xsa = (double *)calloc((size_t)nsrc, sizeof(double));
    fk_source.ysa = (double *)calloc((size_t)nsrc, sizeof(double));
    fk_source.zs_true = (double *)calloc((size_t)nsrc, sizeof(double));
    fk_source.xs_true = (double *)calloc((size_t)nsrc, sizeof(double));
    fk_source.ys_true = (double *)calloc((size_t)nsrc, sizeof(double));
    for (int i = 0; i < nsrc; i++) {
        double ys = ysrc ? ysrc[i] : 0.0;
        fk_source.zs_true[i] = zsrc[i];
        fk_source.xs_true[i] = xsrc[i];
        fk_source.ys_true[i] = ys;
        if (fk_snap_source(fk_model.lis3d, fk_model.nz, fk_model.nx, fk_model.ny, fk_model.z0,
                           fk_model.x0, fk_model.y0, fk_model.dz, fk_model.dx, fk_model.dy,
                           zsrc[i], xsrc[i], ys, i + 1, &fk_source.zsi[i], &fk_source.xsi[i],
                           &fk_source.ysi[i], &fk_source.zsa[i], &fk_source.xsa[i],
                           &fk_source.ysa[i])) {
            *ierr = 1;
            return;
        }
        if (fk_source.zsi[i] > fk_model.nz - 1 || fk_source.xsi[i] > fk_model.nx - 1 ||
            (fk_model.lis3d && fk_source.ysi[i] > fk_model.ny - 1))
            FK_ERR("fteik_source_initialize64f: Warning solver may segfault for source = %d", i + 1);
        if (verbose > 0)
            fprintf(stdout, "fteik_source_initialize64f: Source grid point: (iz,ix,iy)=%6d%6d%6d\n",
                    fk_source.zsi[i], fk_source.xsi[i], fk_source.ysi[i]);
    }
    fk_source.have = true;
}

static int src_check(int isrc, const char *who)
{
    if (!fk_source.have) { FK_ERR("%s: Source not initialized", who); return 1; }
    if (isrc < 1 || isrc > fk_source.nsrc) {
        FK_ERR("%s: Source = %d must be in range [1,%d]", who, isrc, fk_source.nsrc);
        return 1;
    }
    return 0;
}

void fteik_source_getSourceIndices32iF(int isrc, int *zsi, int *xsi, int *ysi, int *ierr)
{
    *zsi = *xsi = *ysi = 0;
    *ierr = src_check(isrc, "fteik_source_getSourceIndices32iF");
    if (*ierr) return;
    *zsi = fk_source.zsi[isrc - 1]; *xsi = fk_source.xsi[isrc - 1]; *ysi = fk_source.ysi[isrc - 1];
}

void fteik_source_getSourceIndices64fF(int isrc, double *zsa, double *xsa, double *ysa, int *ierr)
{
    *zsa = *xsa = *ysa = 0.0;
    *ierr = src_check(isrc, "fteik_source_getSourceIndices64fF");
    if (*ierr) return;
    *zsa = fk_source.zsa[isrc - 1]; *xsa = fk_source.xsa[isrc - 1]; *ysa = fk_source.ysa[isrc - 1];
}

double fk_source_szero(int isrc)
{
    /* source.F90:429-464 */
    const int nzm1 = fk_model.nz - 1, nxm1 = fk_model.nx - 1;
    long c = ((long)(fk_source.ysi[isrc - 1] - 1) * nxm1 + (fk_source.xsi[isrc - 1] - 1)) * nzm1 +
             (fk_source.zsi[isrc - 1] - 1);
    return fk_model.slow[c];
}

void fteik_source_getSzero64fF(int isrc, double *szero, double *szero2, int *ierr)
{
    *szero = *szero2 = 0.0;
    *ierr = 1;
    if (!fk_source.have) { FK_ERR("fteik_source_getSzero64fF: Source not yet initialized"); return; }
    if (!fk_model.have_model) { FK_ERR("fteik_source_getSzero64fF: Slowness model not yet set"); return; }
    if (src_check(isrc, "fteik_source_getSzero64fF")) return;
    *ierr = 0;
    *szero = fk_source_szero(isrc);
    *szero2 = *szero * *szero;
}

void fteik_source_getSolverInfo64fF(int isrc, int *zsi, int *xsi, int *ysi, double *zsa,
                                    double *xsa, double *ysa, double *szero, double *szero2,
                                    int *ierr)
{
    fteik_source_getSourceIndices32iF(isrc, zsi, xsi, ysi, ierr);
    if (*ierr) return;
    fteik_source_getSourceIndices64fF(isrc, zsa, xsa, ysa, ierr);
    if (*ierr) return;
    fteik_source_getSzero64fF(isrc, szero, szero2, ierr);
}

void fteik_source_getNumberOfSources(int *nsrc, int *ierr)
{
    *nsrc = 0;
    *ierr = 0;
    if (!fk_source.have) { FK_ERR("fteik_source_getNumberOfSources: No sources initialized"); *ierr = 1; return; }
    *nsrc = fk_source.nsrc;
}

/* ------------------------------------------------------------ receivers -- */
int fk_receiver_geometry(bool is3d, int nz, int nx, int ny, double z0, double x0, double y0,
                         double dz, double dx, double dy, int nrec, const double *z,
                         const double *x, const double *y, int *ri, double *rd)
{
    /* receiver.F90:95-150 */
    int e = 0;
    if (!is3d) { ny = 1; dy = 1.0; }
    for (int r = 0; r < nrec; r++) {
        double yr_in = (is3d && y) ? y[r] : y0;
        if (z[r] < z0 || z[r] > z0 + dz * (double)(nz - 1)) {
            FK_ERR("fteik_receiver_initialize64f: z=%12.5e out of range [%12.5e,%12.5e]", z[r], z0,
                   z0 + dz * (double)(nz - 1));
            e++;
        }
        if (x[r] < x0 || x[r] > x0 + dx * (double)(nx - 1)) {
            FK_ERR("fteik_receiver_initialize64f: x=%12.5e out of range [%12.5e,%12.5e]", x[r], x0,
                   x0 + dx * (double)(nx - 1));
            e++;
        }
        if (yr_in < y0 || yr_in > y0 + dy * (double)(ny - 1)) {
            FK_ERR("fteik_receiver_initialize64f: y=%12.5e out of range [%12.5e,%12.5e]", yr_in, y0,
                   y0 + dy * (double)(ny - 1));
            e++;
        }
        double zr = (z[r] - z0) / dz, xr = (x[r] - x0) / dx, yr = (yr_in - y0) / dy;
        int iz = (int)(zr + 1.0), ix = (int)(xr + 1.0), iy = (int)(yr + 1.0);
        if (!is3d) iy = 1;
        int zri = imax(1, imin(nz - 1, iz)), xri = imax(1, imin(nx - 1, ix));
        int yri = imax(1, imin(ny - 1, iy));
        ri[r] = zri; ri[nrec + r] = xri; ri[2 * nrec + r] = yri;
        rd[r] = z[r] - (z0 + dz * (double)(zri - 1));
        rd[nrec + r] = x[r] - (x0 + dx * (double)(xri - 1));
        rd[2 * nrec + r] = is3d ? yr_in - (y0 + dy * (double)(yri - 1)) : 0.0;
    }
    return e;
}

void fteik_receiver_setVerbosity(int verbose) { fk_receiver.verbose = verbose; }

void fteik_receiver_free(void)
{
    free(fk_receiver.ri); free(fk_receiver.rd);
    free(fk_receiver.zrec); free(fk_receiver.xrec); free(fk_receiver.yrec);
    fk_dfree(fk_receiver.ri_dev); fk_dfree(fk_receiver.rd_dev);
    memset(&fk_receiver, 0, sizeof(fk_receiver));
}

int fk_receiver_setup(int nrec, const double *z, const double *x, const double *y, int verbose)
{
    fteik_receiver_free();
    fk_receiver.verbose = verbose;
    if (fk_model.nx < 1 || fk_model.ny < 1 || fk_model.nz < 1) {
        FK_ERR("fteik_receiver_initialize64f: Grid not yet set");
        return 1;
    }
    if (nrec < 1) { FK_ERR("fteik_receiver_initialize64f: No receivers"); return 1; }
    fk_receiver.nrec = nrec;
    fk_receiver.ri = (int *)calloc(3 * (size_t)nrec, sizeof(int));
    fk_receiver.rd = (double *)calloc(3 * (size_t)nrec, sizeof(double));
    fk_receiver.zrec = (double *)malloc(sizeof(double) * (size_t)nrec);
    fk_receiver.xrec = (double *)malloc(sizeof(double) * (size_t)nrec);
    fk_receiver.yrec = (double *)malloc(sizeof(double) * (size_t)nrec);
    for (int r = 0; r < nrec; r++) {
        fk_receiver.zrec[r] = z[r];
        fk_receiver.xrec[r] = x[r];
        fk_receiver.yrec[r] = y ? y[r] : fk_model.y0;
    }
    int e = fk_receiver_geometry(fk_model.lis3d, fk_model.nz, fk_model.nx, fk_model.ny,
                                 fk_model.z0, fk_model.x0, fk_model.y0, fk_model.dz,
                                 fk_model.dx, fk_model.dy, nrec, z, x, fk_receiver.yrec,
                                 fk_receiver.ri, fk_receiver.rd);
    fk_receiver.have = true; /* receiver.F90:151: initialised even if out of range */
    return e;
}

int fk_receiver_upload(void)
{
    if (fk_receiver.ri_dev) return 0;
    const int n = fk_receiver.nrec;
    fk_receiver.ri_dev = (int *)fk_dalloc(3 * sizeof(int) * (size_t)n, "fteik_receiver");
    fk_receiver.rd_dev = (double *)fk_dalloc(3 * sizeof(double) * (size_t)n, "fteik_receiver");
    if (!fk_receiver.ri_dev || !fk_receiver.rd_dev) return 1;
    int e = (int)cudaMemcpyAsync(fk_receiver.ri_dev, fk_receiver.ri, 3 * sizeof(int) * (size_t)n,
                                 cudaMemcpyHostToDevice, fk_stream());
    if (!e) e = (int)cudaMemcpyAsync(fk_receiver.rd_dev, fk_receiver.rd, 3 * sizeof(double) * (size_t)n,
                                    cudaMemcpyHostToDevice, fk_stream());
    return fk_check(e, "fteik_receiver: upload");
}

void fteik_receiver_initialize64f(int nrec, const double z[], const double x[], const double y[],
                                  int verbose, int *ierr)
{
    *ierr = fk_receiver_setup(nrec, z, x, y, verbose);
}

void fteik_receiver_getNumberOfReceivers(int *nrec, int *ierr)
{
    *nrec = 0;
    *ierr = 0;
    if (!fk_receiver.have) { FK_ERR("fteik_receiver_getNumberOfReceivers: Receivers not set"); *ierr = 1; return; }
    *nrec = fk_receiver.nrec;
}

void fteik_receiver_getTravelTimes64f(int nrec, int ngrd, const double ttimes[], double ttr[],
                                      int *ierr)
{
    /* receiver.F90:217-313 on a caller field: upload, interpolate on the
     * device, copy back. */
    *ierr = 0;
    if (!fk_receiver.have) { FK_ERR("fteik_receiver_getTravelTimes64f: Receivers not initialized"); *ierr = 1; return; }
    if (nrec < 1) return;
    if (ngrd < fk_model.ngrd) { FK_ERR("fteik_receiver_getTravelTimes64f: ngrd too small"); *ierr = 1; return; }
    if (fk_receiver_upload()) { *ierr = 1; return; }
    const int nz = fk_model.nz, nx = fk_model.nx, ny = fk_model.ny;
    const int n = nrec < fk_receiver.nrec ? nrec : fk_receiver.nrec;
    for (int r = n; r < nrec; r++) ttr[r] = FK_HUGE;
    double *dtt = (double *)fk_dalloc(sizeof(double) * (size_t)fk_model.ngrd, "fteik_receiver");
    double *dtr = (double *)fk_dalloc(sizeof(double) * (size_t)(n > 0 ? n : 1), "fteik_receiver");
    if (!dtt || !dtr) { fk_dfree(dtt); fk_dfree(dtr); *ierr = 1; return; }
    int e = (int)cudaMemcpyAsync(dtt, ttimes, sizeof(double) * (size_t)fk_model.ngrd,
                                 cudaMemcpyHostToDevice, fk_stream());
    /* a caller field is unpadded: pitch nz */
    if (!e) e = fk_receivers(8, fk_model.lis3d, nz, nx, ny, nz, fk_model.dz, fk_model.dx,
                            fk_model.dy, dtt, n, fk_receiver.ri_dev, fk_receiver.rd_dev, dtr,
                            fk_stream());
    if (!e) e = (int)cudaMemcpyAsync(ttr, dtr, sizeof(double) * (size_t)n, cudaMemcpyDeviceToHost,
                                    fk_stream());
    if (!e) e = (int)cudaStreamSynchronize(fk_stream());
    fk_dfree(dtt);
    fk_dfree(dtr);
    *ierr = fk_check(e, "fteik_receiver_getTravelTimes64f");
}
