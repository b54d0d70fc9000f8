/*
 * host_common.h -- process-wide state of the C host layer (the counterpart
 * of the reference's Fortran SAVE module variables) and small helpers.
 */
#ifndef FTEIK_HOST_COMMON_H
#define FTEIK_HOST_COMMON_H

#include <stdbool.h>
#include <stddef.h>
#include <stdio.h>
#include <cuda_runtime.h>

#include "fteik_dev.h"

#define FK_ERR(...) do { fprintf(stderr, __VA_ARGS__); fputc('\n', stderr); } while (0)

/* ---- device, stream, allocation ---- */
int fk_dev_ready(const char *who);           /* 0 if a CUDA device is usable */
cudaStream_t fk_stream(void);
/* Poll limit of the bounded device-side waits (fteik_b200_setSpinLimit), and
 * a counter bumped by every change of it (captured graphs that baked the old
 * limit in are rebuilt when it moves). */
long long fk_spin_limit(void);
int fk_spin_epoch(void);

/* Launch configuration of the 3D slab sweeps (fteik_b200_setSlabConfig):
 * each knob a value, or -1 for the library's choice. */
typedef struct {
    int staged;          /* FP32 passes: staged pass step (1) or direct loads (0) */
    int pairs;           /* passes: two sources of one grid per thread (1) or one (0) */
    int progress;        /* passes: progress every 8 or 32 steps, 0 = by the number of slab tasks */
    int blocks_per_sm;   /* resident blocks per SM of the persistent kernels, 1..4, 0 = all that fit */
} fk_slabcfg_t;
fk_slabcfg_t fk_slabcfg(void);
int fk_slabcfg_epoch(void);

/* ---- ray paths (rays.F90) ---- */
#define FK_RAYS_EULER 1
#define FK_RAYS_MIDPOINT 2
#define FK_RAYS_RK4 3
int fk_rays_integrator(void);
void fk_rays_reset(void);
void *fk_dalloc(size_t bytes, const char *who);
void fk_dfree(void *p);
int fk_check(int cuda_err, const char *who);  /* 0 on success, prints otherwise */
int fk_sync(const char *who);
/* Copies and zero fills on the library stream, complete on return (a
 * cudaError_t).  The library stream is non-blocking: plain cudaMemcpy /
 * cudaMemset run on the legacy stream, unordered with its kernels. */
int fk_h2d(void *dst, const void *src, size_t bytes);
int fk_d2h(void *dst, const void *src, size_t bytes);
int fk_zero(void *dst, size_t bytes);

/* ---- model (model.F90) ---- */
typedef struct {
    bool lis3d, have_geom, have_model;
    int nz, nx, ny, ngrd, ncell, verbose;
    double dz, dx, dy, z0, x0, y0;
    double *slow;          /* host FP64, natural cell order */
    void *slow_dev32;      /* device FP32 padded */
    void *slow_dev64;      /* device FP64 padded */
    float *slowz_dev;      /* device FP32 node-indexed copies (3D; fk_grid3d_t.slowz) */
    bool dev32_ok, dev64_ok, devz_ok;
} fk_model_t;
extern fk_model_t fk_model;
const void *fk_model_slow_dev(int precision); /* uploads lazily */
const float *fk_model_slowz_dev(void);        /* 3D FP32 node-indexed copies, built lazily */
void fk_model_invalidate_dev(void);

/* ---- sources (source.F90) ---- */
typedef struct {
    int nsrc, verbose;
    bool have;
    int *zsi, *xsi, *ysi;
    double *zsa, *xsa, *ysa, *zs_true, *xs_true, *ys_true;
} fk_source_t;
extern fk_source_t fk_source;
/* source.F90:82-236 for one source; 0 on success */
int fk_snap_source(bool is3d, int nz, int nx, int ny, double z0, double x0,
                   double y0, double dz, double dx, double dy, double zsrc,
                   double xsrc, double ysrc, int isrc, int *zsi, int *xsi,
                   int *ysi, double *zsa, double *xsa, double *ysa);
double fk_source_szero(int isrc); /* slowness of the source cell */

/* ---- receivers (receiver.F90) ---- */
typedef struct {
    int nrec, verbose;
    bool have;
    int *ri;          /* host 3*nrec: zri, xri, yri */
    double *rd;       /* host 3*nrec: zdr, xdr, ydr */
    double *zrec, *xrec, *yrec;
    int *ri_dev;
    double *rd_dev;
} fk_receiver_t;
extern fk_receiver_t fk_receiver;
/* rays.F90:271-347 (setRayDestinations): at least one point, every point
 * inside the model; messages as the reference's.  Returns ierr. */
int fk_check_ray_points(bool is3d, int np, const double *z, const double *x, const double *y);
int fk_receiver_setup(int nrec, const double *z, const double *x,
                      const double *y, int verbose); /* returns ierr */
int fk_receiver_upload(void);
/* receiver.F90:62-164 for an arbitrary geometry */
int fk_receiver_geometry(bool is3d, int nz, int nx, int ny, double z0,
                         double x0, double y0, double dz, double dx, double dy,
                         int nrec, const double *z, const double *x,
                         const double *y, int *ri, double *rd);

#endif
