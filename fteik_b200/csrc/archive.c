/*
 * archive.c -- the reference's archive entry points (h5io.F90:104-420,
 * h5io.c:59-345) without the HDF5 library, which this image lacks.
 *
 * The archive named by fteik_h5io_initializeF("path/name.h5") is the
 * directory "path/name.h5.d/" laid out like the reference's HDF5 groups:
 *   Geometry.txt                       nz nx ny dz dx dy z0 x0 y0
 *   TravelTimeFields/<name>.npy        FP32, the reference's order: x fastest,
 *                                      then y, then z (2D: z flipped)
 *   VelocityModels/<name>.npy          INT16 m/s per cell, same order
 *   LevelSchedules/Sweep_<s>.npy       INT16 level of every node, sweeps 1-8
 * Each dataset is a NumPy .npy file (format 1.0), readable with numpy.load.
 * Return codes follow the reference: 0 success, -1 misuse (no model, no
 * archive, no times, a name already used), 1 an I/O failure.
 */
#define _POSIX_C_SOURCE 200809L
#include "host_common.h"
#include "fteik_b200.h"

#include <errno.h>
#include <limits.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <sys/stat.h>
#include <sys/types.h>

#ifndef PATH_MAX
#define PATH_MAX 4096
#endif

static struct {
    bool open;
    char dir[PATH_MAX];
} AR;

static int make_dir(const char *path)
{
    if (mkdir(path, 0755) == 0 || errno == EEXIST) return 0;
    FK_ERR("archive: cannot create directory %s (%s)", path, strerror(errno));
    return 1;
}

static int make_dirs(const char *path)
{
    char tmp[PATH_MAX];
    size_t n = strlen(path);
    if (n == 0 || n >= sizeof(tmp)) return 1;
    memcpy(tmp, path, n + 1);
    for (size_t i = 1; i < n; i++)
        if (tmp[i] == '/') {
            tmp[i] = '\0';
            if (make_dir(tmp)) return 1;
            tmp[i] = '/';
        }
    return make_dir(tmp);
}

static bool file_exists(const char *path)
{
    struct stat st;
    return stat(path, &st) == 0;
}

/* NumPy format 1.0: magic, version, little-endian header length, a Python
 * dict literal padded with spaces to a 64-byte boundary, the raw data. */
static int write_npy(const char *path, const char *descr, const int *shape, int ndim, const void *data,
                     size_t elem)
{
    char hdr[256];
    int k = snprintf(hdr, sizeof(hdr), "{'descr': '%s', 'fortran_order': False, 'shape': (", descr);
    size_t count = 1;
    for (int d = 0; d < ndim; d++) {
        k += snprintf(hdr + k, sizeof(hdr) - (size_t)k, "%d,%s", shape[d], d + 1 < ndim ? " " : "");
        count *= (size_t)shape[d];
    }
    k += snprintf(hdr + k, sizeof(hdr) - (size_t)k, "), }");
    size_t total = 10 + (size_t)k + 1;
    size_t pad = (64 - total % 64) % 64;
    if ((size_t)k + pad + 1 >= sizeof(hdr)) return 1;
    memset(hdr + k, ' ', pad);
    hdr[k + pad] = '\n';
    const uint16_t hlen = (uint16_t)(k + pad + 1);
    FILE *f = fopen(path, "wb");
    if (!f) { FK_ERR("archive: cannot open %s (%s)", path, strerror(errno)); return 1; }
    const unsigned char magic[8] = {0x93, 'N', 'U', 'M', 'P', 'Y', 1, 0};
    const unsigned char hl[2] = {(unsigned char)(hlen & 0xff), (unsigned char)(hlen >> 8)};
    int bad = fwrite(magic, 1, 8, f) != 8 || fwrite(hl, 1, 2, f) != 2 || fwrite(hdr, 1, hlen, f) != hlen ||
              fwrite(data, elem, count, f) != count;
    bad |= fclose(f) != 0;
    if (bad) FK_ERR("archive: failed writing %s", path);
    return bad;
}

static int dataset_path(char *out, const char *group, const char *name)
{
    if (!name || !*name || strchr(name, '/')) { FK_ERR("archive: invalid dataset name"); return -1; }
    if (snprintf(out, PATH_MAX, "%s/%s/%s.npy", AR.dir, group, name) >= PATH_MAX) return -1;
    if (file_exists(out)) { FK_ERR("archive: %s already exists", out); return -1; }
    return 0;
}

int fteik_h5io_initializeF(const char *fileName)
{
    /* h5io.F90:104-131, h5io.c:59-160 */
    if (!fk_model.have_geom) { fprintf(stdout, "fteik_h5io_initializeF: File not initialized\n"); return -1; }
    AR.open = false;
    if (!fileName || !*fileName) { FK_ERR("fteik_h5io_initialize: Error file name is blank"); return -1; }
    const size_t n = strlen(fileName);
    const bool h5 = (n > 3 && strcmp(fileName + n - 3, ".h5") == 0) ||
                    (n > 5 && strcmp(fileName + n - 5, ".hdf5") == 0);
    if (!h5) { FK_ERR("fteik_h5io_initialize: Couldn't create xdmf file name"); return -1; }
    if (snprintf(AR.dir, sizeof(AR.dir), "%s.d", fileName) >= (int)sizeof(AR.dir)) return -1;
    char sub[PATH_MAX];
    if (make_dirs(AR.dir)) return 1;
    const char *groups[3] = {"TravelTimeFields", "VelocityModels", "LevelSchedules"};
    for (int g = 0; g < 3; g++) {
        snprintf(sub, sizeof(sub), "%s/%s", AR.dir, groups[g]);
        if (make_dir(sub)) return 1;
    }
    snprintf(sub, sizeof(sub), "%s/Geometry.txt", AR.dir);
    FILE *f = fopen(sub, "w");
    if (!f) { FK_ERR("archive: cannot write %s", sub); return 1; }
    fprintf(f, "%d %d %d %.17g %.17g %.17g %.17g %.17g %.17g\n", fk_model.nz, fk_model.nx,
            fk_model.lis3d ? fk_model.ny : 1, fk_model.dz, fk_model.dx, fk_model.dy, fk_model.z0, fk_model.x0,
            fk_model.y0);
    if (fclose(f) != 0) return 1;
    AR.open = true;
    return 0;
}

int fteik_h5io_finalizeF(void)
{
    /* h5io.F90:133-138 */
    AR.open = false;
    return 0;
}

int fteik_h5io_writeTravelTimesF(const char *ttName)
{
    /* h5io.F90:263-347: the current field in FP32, x fastest; 2D flipped in z */
    if (!AR.open) { fprintf(stdout, "fteik_h5io_writeTravelTimesF: File not initialized\n"); return -1; }
    char path[PATH_MAX];
    if (dataset_path(path, "TravelTimeFields", ttName)) return -1;
    const int nz = fk_model.nz, nx = fk_model.nx, ny = fk_model.lis3d ? fk_model.ny : 1;
    const size_t ngrd = (size_t)nz * nx * ny;
    double *t = (double *)malloc(sizeof(double) * ngrd);
    float *o = (float *)malloc(sizeof(float) * ngrd);
    int ierr = (t && o) ? 0 : 1;
    if (!ierr) {
        if (fk_model.lis3d)
            fteik_solver3d_getTravelTimeField64f((int)ngrd, FTEIK_XYZ_ORDERING, t, &ierr);
        else
            fteik_solver2d_getTravelTimeField64f((int)ngrd, FTEIK_XYZ_ORDERING, t, &ierr);
        if (ierr) {
            fprintf(stdout, "fteik_h5io_writeTravelTimesF: %dD travel times not yet computed\n",
                    fk_model.lis3d ? 3 : 2);
            ierr = -1;
        }
    }
    if (!ierr) {
        if (fk_model.lis3d) {
            for (size_t i = 0; i < ngrd; i++) o[i] = (float)t[i];
        } else { /* row iz of the output is depth nz + 1 - iz */
            for (int iz = 0; iz < nz; iz++)
                for (int ix = 0; ix < nx; ix++)
                    o[(size_t)iz * nx + ix] = (float)t[(size_t)(nz - 1 - iz) * nx + ix];
        }
        int shape3[3] = {nz, ny, nx}, shape2[2] = {nz, nx};
        ierr = fk_model.lis3d ? write_npy(path, "<f4", shape3, 3, o, sizeof(float))
                              : write_npy(path, "<f4", shape2, 2, o, sizeof(float));
    }
    free(t);
    free(o);
    return ierr;
}

int fteik_h5io_writeVelocityModelF(const char *velName)
{
    /* h5io.F90:348-420: INT2(INT(1/slow + 0.5)) per cell, x fastest; 2D flipped in z */
    if (!AR.open) { fprintf(stdout, "fteik_h5io_writeVelocityModelF: File not initialized\n"); return -1; }
    if (!fk_model.have_model) { fprintf(stdout, "fteik_h5io_writeVelocityModelF: Velocity model not set\n"); return -1; }
    char path[PATH_MAX];
    if (dataset_path(path, "VelocityModels", velName)) return -1;
    const int nzc = fk_model.nz - 1, nxc = fk_model.nx - 1, nyc = fk_model.lis3d ? fk_model.ny - 1 : 1;
    const size_t ncell = (size_t)nzc * nxc * nyc;
    int16_t *v = (int16_t *)malloc(sizeof(int16_t) * ncell);
    if (!v) return 1;
    for (int iz = 0; iz < nzc; iz++)
        for (int iy = 0; iy < nyc; iy++)
            for (int ix = 0; ix < nxc; ix++) {
                const int jz = fk_model.lis3d ? iz : nzc - 1 - iz;
                const double sl = fk_model.slow[((size_t)iy * nxc + ix) * nzc + jz];
                v[((size_t)iz * nyc + iy) * nxc + ix] = (int16_t)(int)(1.0 / sl + 0.5);
            }
    int shape3[3] = {nzc, nyc, nxc}, shape2[2] = {nzc, nxc};
    int ierr = fk_model.lis3d ? write_npy(path, "<i2", shape3, 3, v, sizeof(int16_t))
                              : write_npy(path, "<i2", shape2, 2, v, sizeof(int16_t));
    free(v);
    return ierr;
}

int fteik_h5io_writeLevelSchedulesF(void)
{
    /* h5io.F90:140-262: for sweep s the level of every node (1-based; the
     * nodes whose sweep-permuted coordinates sum to level + 2, graph3d.F90),
     * x fastest; 3D only, as the reference */
    if (!AR.open) { fprintf(stdout, "fteik_h5io_writeLevelSchedulesF: File not initialized\n"); return -1; }
    if (!fk_model.have_geom) { fprintf(stdout, "fteik_h5io_writeLevelSchedulesF: Grid not set\n"); return -1; }
    if (!fk_model.lis3d) { fprintf(stdout, "fteik_h5io_writeLevelSchedulesF: Not yet done for 2D\n"); return -1; }
    const int nz = fk_model.nz, nx = fk_model.nx, ny = fk_model.ny;
    int16_t *lv = (int16_t *)malloc(sizeof(int16_t) * (size_t)nz * nx * ny);
    if (!lv) return 1;
    int nerr = 0;
    for (int s = 0; s < 8; s++) {
        const bool fz = s >= 4, fx = s % 2 == 1, fy = (s / 2) % 2 == 1;
        for (int iz = 0; iz < nz; iz++)
            for (int iy = 0; iy < ny; iy++)
                for (int ix = 0; ix < nx; ix++) {
                    const int pz = fz ? nz - 1 - iz : iz, px = fx ? nx - 1 - ix : ix, py = fy ? ny - 1 - iy : iy;
                    lv[((size_t)iz * ny + iy) * nx + ix] = (int16_t)(pz + px + py + 1);
                }
        char name[32], path[PATH_MAX];
        snprintf(name, sizeof(name), "Sweep_%d", s + 1);
        int shape[3] = {nz, ny, nx};
        if (snprintf(path, sizeof(path), "%s/LevelSchedules/%s.npy", AR.dir, name) >= (int)sizeof(path) ||
            write_npy(path, "<i2", shape, 3, lv, sizeof(int16_t))) {
            fprintf(stdout, "fteik_h5io_writeLevelSchedulesF: Error sweep schedule: %d\n", s + 1);
            nerr++;
        }
    }
    free(lv);
    return nerr;
}
