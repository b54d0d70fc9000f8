/*
 * host_common.c -- device context, stream and allocation helpers of the C
 * host layer.
 */
#include "host_common.h"

#include <stdlib.h>

static int g_dev_state = 0; /* 0 unknown, 1 ready, -1 unusable */
static cudaStream_t g_stream = NULL;
static int g_device = -1;

int fk_dev_ready(const char *who)
{
    if (g_dev_state == 1) return 0;
    if (g_dev_state == -1) {
        FK_ERR("%s: no usable CUDA device; this library has no CPU path", who);
        return 1;
    }
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n < 1) {
        g_dev_state = -1;
        FK_ERR("%s: no usable CUDA device (%s); this library has no CPU path", who,
               e != cudaSuccess ? cudaGetErrorString(e) : "device count 0");
        return 1;
    }
    int dev = 0;
    cudaGetDevice(&dev);
    e = cudaStreamCreateWithFlags(&g_stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        g_dev_state = -1;
        FK_ERR("%s: cannot create a CUDA stream (%s)", who, cudaGetErrorString(e));
        return 1;
    }
    g_device = dev;
    g_dev_state = 1;
    return 0;
}

int fteik_b200_device(void) { return g_dev_state == 1 ? g_device : -1; }

const char *fteik_b200_version(void) { return "fteik-b200 0.1 (sm_100a)"; }

cudaStream_t fk_stream(void) { return g_stream; }

/* Polls a bounded device-side wait of the 3D sweeps (a slab waiting on its
 * upwind slab) makes before it gives up and raises the kernel's error word:
 * by default 2^22 polls of at most 1 us each, seconds, far longer than any
 * wait of a correct run. */
#define FK_SPIN_LIMIT_DEFAULT (1LL << 22)
static long long g_spin_limit = FK_SPIN_LIMIT_DEFAULT;
static int g_spin_epoch = 0;

long long fk_spin_limit(void) { return g_spin_limit; }
int fk_spin_epoch(void) { return g_spin_epoch; }

void fteik_b200_setSpinLimit(long long polls, int *ierr)
{
    *ierr = 0;
    if (polls < 0) {
        g_spin_limit = FK_SPIN_LIMIT_DEFAULT;
    } else {
        g_spin_limit = polls;
    }
    g_spin_epoch++;
}

void fteik_b200_getSpinLimit(long long *polls) { *polls = g_spin_limit; }

static fk_slabcfg_t g_slabcfg = {-1, -1, -1, -1};
static int g_slabcfg_epoch = 0;

fk_slabcfg_t fk_slabcfg(void) { return g_slabcfg; }
int fk_slabcfg_epoch(void) { return g_slabcfg_epoch; }

void fteik_b200_setSlabConfig(int staged, int pairs, int progress, int blocksPerSM, int *ierr)
{
    *ierr = 0;
    if (staged < -1 || staged > 1 || pairs < -1 || pairs > 1 ||
        !(progress == -1 || progress == 0 || progress == 8 || progress == 32) || blocksPerSM < -1 ||
        blocksPerSM > 4) {
        FK_ERR("fteik_b200_setSlabConfig: staged and pairs must be -1, 0 or 1, progress -1, 0, 8 or 32, "
               "blocksPerSM -1, 0 or 1..4");
        *ierr = 1;
        return;
    }
    g_slabcfg.staged = staged;
    g_slabcfg.pairs = pairs;
    g_slabcfg.progress = progress;
    g_slabcfg.blocks_per_sm = blocksPerSM;
    g_slabcfg_epoch++;
}

void fteik_b200_getSlabConfig(int *staged, int *pairs, int *progress, int *blocksPerSM)
{
    *staged = g_slabcfg.staged;
    *pairs = g_slabcfg.pairs;
    *progress = g_slabcfg.progress;
    *blocksPerSM = g_slabcfg.blocks_per_sm;
}

void *fteik_b200_stream(void)
{
    if (fk_dev_ready("fteik_b200_stream")) return NULL;
    return (void *)g_stream;
}

void *fk_dalloc(size_t bytes, const char *who)
{
    if (fk_dev_ready(who)) return NULL;
    void *p = NULL;
    cudaError_t e = cudaMalloc(&p, bytes ? bytes : 16);
    if (e != cudaSuccess) {
        FK_ERR("%s: cudaMalloc of %zu bytes failed (%s)", who, bytes, cudaGetErrorString(e));
        return NULL;
    }
    return p;
}

void fk_dfree(void *p)
{
    if (p && g_dev_state == 1) cudaFree(p);
}

int fk_check(int err, const char *who)
{
    if (err == 0) return 0;
    FK_ERR("%s: CUDA error %d (%s)", who, err, cudaGetErrorString((cudaError_t)err));
    return 1;
}

int fk_sync(const char *who)
{
    cudaError_t e = cudaStreamSynchronize(g_stream);
    if (e != cudaSuccess) {
        FK_ERR("%s: CUDA error (%s)", who, cudaGetErrorString(e));
        return 1;
    }
    return 0;
}

int fk_h2d(void *dst, const void *src, size_t bytes)
{
    cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, g_stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(g_stream);
    return (int)e;
}

int fk_d2h(void *dst, const void *src, size_t bytes)
{
    cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, g_stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(g_stream);
    return (int)e;
}

int fk_zero(void *dst, size_t bytes)
{
    cudaError_t e = cudaMemsetAsync(dst, 0, bytes, g_stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(g_stream);
    return (int)e;
}

int fk_check_ray_points(bool is3d, int np, const double *z, const double *x, const double *y)
{
    if (np < 1) {
        FK_ERR("fteik_rays_setRayDestinations: No origins!");
        return 1;
    }
    const double zmax = fk_model.z0 + (double)(fk_model.nz - 1) * fk_model.dz;
    const double xmax = fk_model.x0 + (double)(fk_model.nx - 1) * fk_model.dx;
    const double ymax = is3d ? fk_model.y0 + (double)(fk_model.ny - 1) * fk_model.dy : fk_model.y0;
    int ierr = 0;
    for (int i = 0; i < np; i++) {
        if (z[i] < fk_model.z0 || z[i] > zmax) {
            FK_ERR("fteik_rays_setRayDestinations: zr(%d)=%g must be in range [%g, %g]", i + 1, z[i], fk_model.z0, zmax);
            ierr = 1;
        }
        if (x[i] < fk_model.x0 || x[i] > xmax) {
            FK_ERR("fteik_rays_setRayDestinations: xr(%d)=%g must be in range [%g, %g]", i + 1, x[i], fk_model.x0, xmax);
            ierr = 1;
        }
        if (is3d && (y[i] < fk_model.y0 || y[i] > ymax)) {
            FK_ERR("fteik_rays_setRayDestinations: yr(%d)=%g must be in range [%g, %g]", i + 1, y[i], fk_model.y0, ymax);
            ierr = 1;
        }
    }
    return ierr;
}

/* rays.F90:93-104, :215-229: the ray-path integrator, reset to Euler when a
 * solver is initialised or freed (fteik_rays_initialize calls
 * fteik_rays_free, rays.F90:143,176-199). */
static int g_ray_integrator = FK_RAYS_EULER;

int fk_rays_integrator(void) { return g_ray_integrator; }
void fk_rays_reset(void) { g_ray_integrator = FK_RAYS_EULER; }

void fteik_rays_setODEIntegrator(int integrator, int *ierr)
{
    *ierr = 0;
    g_ray_integrator = FK_RAYS_EULER;
    if (integrator < FK_RAYS_EULER || integrator > FK_RAYS_RK4) {
        FK_ERR("fteik_rays_setODEIntegrator: Invalid integrator = %d using Euler", integrator);
        *ierr = 1;
        return;
    }
    g_ray_integrator = integrator;
}
