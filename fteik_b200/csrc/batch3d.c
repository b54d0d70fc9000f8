/*
 * batch3d.c -- batched multi-source, multi-grid 3D solve (no reference
 * counterpart; the reference solves one source at a time,
 * solver3D.F90:1156-1243, and callers loop over sources,
 * python/fteik3d.py:258-263).
 *
 * Every (grid, source) pair becomes one work item; one persistent kernel
 * launch runs the initialisation sweeps of them all and one more runs their
 * Gauss-Seidel passes, slab tasks of every item interleaved (row3d_impl.cuh).
 * The launches are captured once into a CUDA graph and replayed while the
 * work list is unchanged.
 * Fields stay on the device until exported.
 */
#include "host_common.h"
#include "fteik_b200.h"
#include "slabplan.h"

#include <stdio.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
    int nz, nx, ny, ngrd, ncell, zp, zcp;
    double dz, dx, dy;
    double *vel_dev;        /* device FP64 cell velocities, natural order */
    double *szero;          /* host [nsrc]: slowness of each source's cell */
    void *slow_dev;         /* device padded, batch precision */
    float *slowz_dev;       /* FP32: node-indexed slowness copies (fk_grid3d_t.slowz) */
    bool have_model;
    int nsrc;
    int *zsi, *xsi, *ysi;
    double *zsa, *xsa, *ysa;
    void *fields;           /* device [nsrc][ny][nx][zp] */
    int nrec;
    int *ri_dev;
    double *rd_dev;
    int work0;              /* index of this grid's first work item */
    float *dl_buf;          /* device dense FP32 tables being downloaded */
    size_t dl_cap;
    cudaEvent_t dl_ready, dl_done;  /* unpacked (library stream), copied (copy stream) */
    bool have_dl_ev;
} bgrid_t;

static struct {
    bool init, solved;
    int ngrid, precision, nsweep, max_pass;
    double eps, conv_tol;
    bgrid_t *g;
    fk_grid3d_t *grids_dev;
    fk_work3d_t *work_dev;
    fk_result3d_t *res_dev;
    fk_result3d_t *res_host;
    int nwork, max_nx, max_nz;
    int *work_order;        /* work item -> (grid, src) packed as grid<<20|src */
    fk_slabplan_t plan;     /* slab-pipelined schedule */
    int spin_epoch;         /* poll limit the plan (and graph) was built with */
    int cfg_epoch;          /* slab configuration the plan (and graph) was built with */
    int tuned[6];           /* configuration in use: staged, pairs, progress, blocks/SM passes, init, init pairs */
    float tune_ms[2];       /* its init / pass kernel times when tuned (0: not timed) */
    int tune_runs;          /* candidate solves the last tuning ran (0: cache hit or nothing to tune) */
    bool work_dirty;        /* source positions changed, shape unchanged */
    cudaGraphExec_t graph;
    bool graph_ok;
    double *export_buf;
    size_t export_cap;
    void *stage;            /* device staging: slowness upload, dense field export */
    size_t stage_cap;
    cudaEvent_t ev[3];      /* in the graph: before init, after init, after passes */
    bool have_ev;
    cudaStream_t copy_stream; /* asynchronous table downloads */
    void *hmap, *hmap_dev;    /* mapped pinned host memory: small results kernels write */
    size_t hmap_cap;
} SB;

/* Mapped pinned host memory for the small results the host waits for (the
 * velocity check, the source-cell velocities): kernels write them straight
 * to the host, so no copy queues behind table downloads still running on
 * the copy stream.  *dev receives the device address. */
static void *hmap_buf(size_t bytes, void **dev, const char *who)
{
    if (!SB.hmap || SB.hmap_cap < bytes) {
        if (SB.hmap) {
            cudaStreamSynchronize(fk_stream());
            cudaFreeHost(SB.hmap);
        }
        SB.hmap = SB.hmap_dev = NULL;
        SB.hmap_cap = 0;
        void *p = NULL, *d = NULL;
        cudaError_t e = cudaHostAlloc(&p, bytes, cudaHostAllocMapped);
        if (e == cudaSuccess) e = cudaHostGetDevicePointer(&d, p, 0);
        if (e != cudaSuccess) {
            if (p) cudaFreeHost(p);
            FK_ERR("%s: mapped host allocation of %zu bytes failed (%s)", who, bytes, cudaGetErrorString(e));
            return NULL;
        }
        SB.hmap = p;
        SB.hmap_dev = d;
        SB.hmap_cap = bytes;
    }
    *dev = SB.hmap_dev;
    return SB.hmap;
}

static void *stage_buf(size_t bytes, const char *who)
{
    if (SB.stage && SB.stage_cap >= bytes) return SB.stage;
    fk_dfree(SB.stage);
    SB.stage = fk_dalloc(bytes, who);
    SB.stage_cap = SB.stage ? bytes : 0;
    return SB.stage;
}

static void free_grid(bgrid_t *g)
{
    free(g->szero); free(g->zsi); free(g->xsi); free(g->ysi);
    free(g->zsa); free(g->xsa); free(g->ysa);
    fk_dfree(g->vel_dev); fk_dfree(g->slow_dev); fk_dfree(g->slowz_dev); fk_dfree(g->fields);
    fk_dfree(g->ri_dev); fk_dfree(g->rd_dev);
    fk_dfree(g->dl_buf);
    if (g->have_dl_ev) { cudaEventDestroy(g->dl_ready); cudaEventDestroy(g->dl_done); }
    memset(g, 0, sizeof(*g));
}

static void invalidate(void)
{
    if (SB.graph_ok) cudaGraphExecDestroy(SB.graph);
    SB.graph_ok = false;
    SB.solved = false;
}

void fteik_b200_batch3d_finalize(void)
{
    if (SB.copy_stream) cudaStreamSynchronize(SB.copy_stream);
    invalidate();
    for (int i = 0; i < SB.ngrid; i++) free_grid(&SB.g[i]);
    free(SB.g);
    fk_dfree(SB.grids_dev); fk_dfree(SB.work_dev); fk_dfree(SB.res_dev); fk_dfree(SB.export_buf);
    fk_dfree(SB.stage);
    fk_slabplan_free(&SB.plan);
    if (SB.have_ev) for (int i = 0; i < 3; i++) cudaEventDestroy(SB.ev[i]);
    free(SB.res_host); free(SB.work_order);
    if (SB.hmap) cudaFreeHost(SB.hmap);
    cudaStream_t cs = SB.copy_stream;   /* kept for the process's next batch */
    memset(&SB, 0, sizeof(SB));
    SB.copy_stream = cs;
}

void fteik_b200_batch3d_initialize(int ngrid, const int nz[], const int nx[], const int ny[],
                                   const double dz[], const double dx[], const double dy[],
                                   int nsweep, double eps, double convTol, int maxPass,
                                   int precision, int *ierr)
{
    *ierr = 0;
    fteik_b200_batch3d_finalize();
    if (ngrid < 1) { FK_ERR("fteik_b200_batch3d_initialize: ngrid must be positive"); *ierr = 1; return; }
    if (precision != 4 && precision != 8) { FK_ERR("fteik_b200_batch3d_initialize: precision must be 4 or 8"); *ierr = 1; return; }
    if (nsweep < 0) { FK_ERR("fteik_b200_batch3d_initialize: nsweep must be non-negative"); *ierr = 1; return; }
    if (fk_dev_ready("fteik_b200_batch3d_initialize")) { *ierr = 1; return; }
    SB.g = (bgrid_t *)calloc((size_t)ngrid, sizeof(bgrid_t));
    SB.ngrid = ngrid;
    for (int i = 0; i < ngrid; i++) {
        bgrid_t *g = &SB.g[i];
        if (nz[i] < 3 || nx[i] < 3 || ny[i] < 3 || dz[i] <= 0 || dx[i] <= 0 || dy[i] <= 0) {
            FK_ERR("fteik_b200_batch3d_initialize: grid %d needs n >= 3 and h > 0", i + 1);
            *ierr = 1;
            return;
        }
        if ((int)eps > nz[i] || (int)eps > nx[i] || (int)eps > ny[i]) {
            FK_ERR("fteik_b200_batch3d_initialize: eps=%d bigger than grid %d", (int)eps, i + 1);
            *ierr = 1;
            return;
        }
        g->nz = nz[i]; g->nx = nx[i]; g->ny = ny[i];
        g->ngrd = nz[i] * nx[i] * ny[i];
        g->ncell = (nz[i] - 1) * (nx[i] - 1) * (ny[i] - 1);
        g->zp = FK_PITCH(nz[i]); g->zcp = FK_PITCH(nz[i] - 1);
        g->dz = dz[i]; g->dx = dx[i]; g->dy = dy[i];
    }
    SB.precision = precision;
    SB.nsweep = nsweep;
    SB.eps = eps;
    SB.conv_tol = convTol;
    SB.max_pass = maxPass;
    SB.init = true;
}

static bgrid_t *grid_of(int igrid, const char *who)
{
    if (!SB.init) { FK_ERR("%s: batch not initialized", who); return NULL; }
    if (igrid < 1 || igrid > SB.ngrid) { FK_ERR("%s: grid %d out of range [1,%d]", who, igrid, SB.ngrid); return NULL; }
    return &SB.g[igrid - 1];
}

void fteik_b200_batch3d_setVelocityModel64f(int igrid, int ncell, const double vel[], int *ierr)
{
    const char *who = "fteik_b200_batch3d_setVelocityModel64f";
    *ierr = 1;
    bgrid_t *g = grid_of(igrid, who);
    if (!g) return;
    if (ncell != g->ncell) { FK_ERR("%s: ncell=%d, grid has %d cells", who, ncell, g->ncell); return; }
    /* the velocities go up as given (pinned caller memory: one DMA) and are
     * checked and inverted on the device */
    const size_t nelem = (size_t)g->zcp * (g->nx - 1) * (g->ny - 1);
    if (!g->slow_dev) g->slow_dev = fk_dalloc(nelem * (size_t)SB.precision, who);
    if (!g->vel_dev) g->vel_dev = (double *)fk_dalloc(sizeof(double) * (size_t)ncell, who);
    void *bad_dev = NULL;
    volatile int *bad = (volatile int *)hmap_buf(sizeof(int), &bad_dev, who);
    if (!g->slow_dev || !g->vel_dev || !bad) return;
    g->have_model = false;
    cudaStream_t s = fk_stream();
    int e = (int)cudaStreamSynchronize(s);   /* no kernel of the stream uses the flag */
    *bad = 0;
    if (!e) e = (int)cudaMemsetAsync(g->slow_dev, 0, nelem * (size_t)SB.precision, s);
    if (!e) e = (int)cudaMemcpyAsync(g->vel_dev, vel, sizeof(double) * (size_t)ncell, cudaMemcpyHostToDevice, s);
    if (!e) e = fk_pack_velocity(SB.precision, g->nz, g->nx, g->ny, g->zcp, g->vel_dev, g->slow_dev,
                                 (int *)bad_dev, s);
    if (!e && SB.precision == 4) {
        /* node-indexed copies for the staged pass step */
        if (!g->slowz_dev)
            g->slowz_dev = (float *)fk_dalloc(sizeof(float) * 2 * (size_t)g->zp * (g->nx - 1) * (g->ny - 1), who);
        e = g->slowz_dev ? fk_node_slowness_f32(g->nz, g->nx, g->ny, g->zcp, g->zp, (const float *)g->slow_dev,
                                                g->slowz_dev, s)
                         : 1;
    }
    if (!e) e = (int)cudaStreamSynchronize(s);
    if (fk_check(e, who)) return;
    if (*bad) { FK_ERR("%s: velocities must be positive", who); return; }
    g->have_model = true;
    SB.solved = false;
    SB.work_dirty = true; /* szero of this grid's sources */
    *ierr = 0;
}

void fteik_b200_batch3d_setSources64f(int igrid, int nsrc, const double zsrc[],
                                      const double xsrc[], const double ysrc[], int *ierr)
{
    const char *who = "fteik_b200_batch3d_setSources64f";
    *ierr = 1;
    bgrid_t *g = grid_of(igrid, who);
    if (!g) return;
    if (nsrc < 1) { FK_ERR("%s: No sources", who); return; }
    const bool same_shape = g->fields != NULL && nsrc == g->nsrc;
    free(g->zsi); free(g->xsi); free(g->ysi); free(g->zsa); free(g->xsa); free(g->ysa);
    if (!same_shape) { fk_dfree(g->fields); g->fields = NULL; }
    g->nsrc = 0;
    g->zsi = (int *)malloc(sizeof(int) * (size_t)nsrc);
    g->xsi = (int *)malloc(sizeof(int) * (size_t)nsrc);
    g->ysi = (int *)malloc(sizeof(int) * (size_t)nsrc);
    g->zsa = (double *)malloc(sizeof(double) * (size_t)nsrc);
    g->xsa = (double *)malloc(sizeof(double) * (size_t)nsrc);
    g->ysa = (double *)malloc(sizeof(double) * (size_t)nsrc);
    for (int i = 0; i < nsrc; i++)
        if (fk_snap_source(true, g->nz, g->nx, g->ny, 0.0, 0.0, 0.0, g->dz, g->dx, g->dy, zsrc[i],
                           xsrc[i], ysrc[i], i + 1, &g->zsi[i], &g->xsi[i], &g->ysi[i], &g->zsa[i],
                           &g->xsa[i], &g->ysa[i]))
            return;
    const size_t fbytes = (size_t)g->zp * g->nx * g->ny * (size_t)SB.precision;
    if (!g->fields) g->fields = fk_dalloc(fbytes * (size_t)nsrc, who);
    if (!g->fields) return;
    g->nsrc = nsrc;
    if (same_shape) {
        /* same work list: the captured graph stays valid, only the work
         * descriptors it reads change */
        SB.work_dirty = true;
        SB.solved = false;
    } else {
        invalidate();
    }
    *ierr = 0;
}

void fteik_b200_batch3d_setReceivers64f(int igrid, int nrec, const double zrec[],
                                        const double xrec[], const double yrec[], int *ierr)
{
    const char *who = "fteik_b200_batch3d_setReceivers64f";
    *ierr = 1;
    bgrid_t *g = grid_of(igrid, who);
    if (!g) return;
    if (nrec < 1) { FK_ERR("%s: No receivers", who); return; }
    int *ri = (int *)malloc(3 * sizeof(int) * (size_t)nrec);
    double *rd = (double *)malloc(3 * sizeof(double) * (size_t)nrec);
    int bad = fk_receiver_geometry(true, g->nz, g->nx, g->ny, 0.0, 0.0, 0.0, g->dz, g->dx, g->dy,
                                   nrec, zrec, xrec, yrec, ri, rd);
    fk_dfree(g->ri_dev); fk_dfree(g->rd_dev);
    g->ri_dev = (int *)fk_dalloc(3 * sizeof(int) * (size_t)nrec, who);
    g->rd_dev = (double *)fk_dalloc(3 * sizeof(double) * (size_t)nrec, who);
    int e = 1;
    if (g->ri_dev && g->rd_dev) {
        e = (int)fk_h2d(g->ri_dev, ri, 3 * sizeof(int) * (size_t)nrec);
        if (!e) e = (int)fk_h2d(g->rd_dev, rd, 3 * sizeof(double) * (size_t)nrec);
        e = fk_check(e, who);
    }
    free(ri); free(rd);
    g->nrec = e ? 0 : nrec;
    *ierr = (e || bad) ? 1 : 0;
}

static int cmp_work(const void *a, const void *b)
{
    /* largest grids (most CTA steps) first */
    const int ga = (*(const int *)a) >> 20, gb = (*(const int *)b) >> 20;
    const long wa = (long)SB.g[ga].nz * SB.g[ga].ny * ((SB.g[ga].nx + 31) / 32);
    const long wb = (long)SB.g[gb].nz * SB.g[gb].ny * ((SB.g[gb].nx + 31) / 32);
    if (wa != wb) return wa < wb ? 1 : -1;
    return (*(const int *)a) - (*(const int *)b);
}

static void fill_work(fk_work3d_t *wh)
{
    for (int w = 0; w < SB.nwork; w++) {
        const int i = SB.work_order[w] >> 20, s = SB.work_order[w] & ((1 << 20) - 1);
        bgrid_t *g = &SB.g[i];
        const size_t fbytes = (size_t)g->zp * g->nx * g->ny * (size_t)SB.precision;
        wh[w].grid = i;
        wh[w].zsi = g->zsi[s]; wh[w].xsi = g->xsi[s]; wh[w].ysi = g->ysi[s];
        wh[w].zsa = g->zsa[s]; wh[w].xsa = g->xsa[s]; wh[w].ysa = g->ysa[s];
        wh[w].szero = g->szero[s];
        wh[w].tt = (char *)g->fields + fbytes * (size_t)s;
    }
}

/* szero of every source: 1 / v of its cell (source.F90:429-464), the
 * velocities gathered from the device copy of each grid's model. */
static int update_szero(const char *who)
{
    cudaStream_t s = fk_stream();
    int e = 0;
    for (int i = 0; i < SB.ngrid && !e; i++) {
        bgrid_t *g = &SB.g[i];
        if (g->nsrc < 1) continue;
        const int n = g->nsrc;
        free(g->szero);
        g->szero = (double *)malloc(sizeof(double) * (size_t)n);
        void *hdev = NULL;
        e = (int)cudaStreamSynchronize(s);       /* no kernel of the stream uses the buffer */
        char *hbuf = (char *)hmap_buf((sizeof(long long) + sizeof(double)) * (size_t)n, &hdev, who);
        if (!g->szero || !hbuf) return 1;
        /* cell indices in, velocities out, both in mapped host memory */
        long long *idx = (long long *)hbuf;
        volatile double *v = (volatile double *)(hbuf + sizeof(long long) * (size_t)n);
        for (int k = 0; k < n; k++)
            idx[k] = ((long long)(g->ysi[k] - 1) * (g->nx - 1) + (g->xsi[k] - 1)) * (g->nz - 1) + (g->zsi[k] - 1);
        if (!e) e = fk_gather64(g->vel_dev, (const long long *)hdev, n,
                                (double *)((char *)hdev + sizeof(long long) * (size_t)n), s);
        if (!e) e = (int)cudaStreamSynchronize(s);
        for (int k = 0; !e && k < n; k++) g->szero[k] = 1.0 / v[k];
    }
    return fk_check(e, who);
}

static int upload_work(const char *who)
{
    if (update_szero(who)) return 1;
    fk_work3d_t *wh = (fk_work3d_t *)malloc(sizeof(fk_work3d_t) * (size_t)SB.nwork);
    fill_work(wh);
    int e = (int)fk_h2d(SB.work_dev, wh, sizeof(fk_work3d_t) * (size_t)SB.nwork);
    free(wh);
    SB.work_dirty = false;
    return fk_check(e, who);
}

static int build_work(const char *who)
{
    int nwork = 0, max_nx = 0, max_nz = 0;
    for (int i = 0; i < SB.ngrid; i++) {
        bgrid_t *g = &SB.g[i];
        if (!g->have_model) { FK_ERR("%s: grid %d has no velocity model", who, i + 1); return 1; }
        if (g->nsrc < 1) continue;
        if (g->nsrc >= (1 << 20)) { FK_ERR("%s: too many sources", who); return 1; }
        nwork += g->nsrc;
        if (g->nx > max_nx) max_nx = g->nx;
        if (g->nz > max_nz) max_nz = g->nz;
    }
    if (nwork == 0) { FK_ERR("%s: no sources", who); return 1; }
    if (update_szero(who)) return 1;
    fk_dfree(SB.grids_dev); fk_dfree(SB.work_dev); fk_dfree(SB.res_dev);
    free(SB.res_host); free(SB.work_order);
    SB.grids_dev = (fk_grid3d_t *)fk_dalloc(sizeof(fk_grid3d_t) * (size_t)SB.ngrid, who);
    SB.work_dev = (fk_work3d_t *)fk_dalloc(sizeof(fk_work3d_t) * (size_t)nwork, who);
    SB.res_dev = (fk_result3d_t *)fk_dalloc(sizeof(fk_result3d_t) * (size_t)nwork, who);
    SB.res_host = (fk_result3d_t *)calloc((size_t)nwork, sizeof(fk_result3d_t));
    SB.work_order = (int *)malloc(sizeof(int) * (size_t)nwork);
    if (!SB.grids_dev || !SB.work_dev || !SB.res_dev) return 1;
    fk_grid3d_t *gh = (fk_grid3d_t *)malloc(sizeof(fk_grid3d_t) * (size_t)SB.ngrid);
    fk_work3d_t *wh = (fk_work3d_t *)malloc(sizeof(fk_work3d_t) * (size_t)nwork);
    int k = 0;
    for (int i = 0; i < SB.ngrid; i++) {
        bgrid_t *g = &SB.g[i];
        gh[i].nz = g->nz; gh[i].nx = g->nx; gh[i].ny = g->ny;
        gh[i].zp = g->zp; gh[i].zcp = g->zcp;
        gh[i].dz = g->dz; gh[i].dx = g->dx; gh[i].dy = g->dy;
        gh[i].slow = g->slow_dev;
        gh[i].slowz = g->slowz_dev;
        for (int s = 0; s < g->nsrc; s++) SB.work_order[k++] = (i << 20) | s;
    }
    qsort(SB.work_order, (size_t)nwork, sizeof(int), cmp_work);
    SB.nwork = nwork;
    fill_work(wh);
    int e = (int)fk_h2d(SB.grids_dev, gh, sizeof(fk_grid3d_t) * (size_t)SB.ngrid);
    if (!e) e = (int)fk_h2d(SB.work_dev, wh, sizeof(fk_work3d_t) * (size_t)nwork);
    if (!e) {
        int *wnx = (int *)malloc(sizeof(int) * (size_t)nwork);
        int *wny = (int *)malloc(sizeof(int) * (size_t)nwork);
        int *wnz = (int *)malloc(sizeof(int) * (size_t)nwork);
        int *wg = (int *)malloc(sizeof(int) * (size_t)nwork);
        for (int w = 0; w < nwork; w++) {
            wnx[w] = gh[wh[w].grid].nx;
            wny[w] = gh[wh[w].grid].ny;
            wnz[w] = gh[wh[w].grid].nz;
            wg[w] = wh[w].grid;
        }
        const int np = (SB.conv_tol >= 0.0 && SB.max_pass > 0) ? SB.max_pass : SB.nsweep;
        const fk_slabcfg_t cfg = fk_slabcfg();
        e = fk_slabplan_build(&SB.plan, nwork, wnx, wny, wnz, wg, np, cfg.pairs != 0, who);
        SB.spin_epoch = fk_spin_epoch();
        SB.cfg_epoch = fk_slabcfg_epoch();
        free(wnx);
        free(wny);
        free(wnz);
        free(wg);
    }
    free(gh);
    free(wh);
    SB.nwork = nwork;
    SB.max_nx = max_nx;
    SB.max_nz = max_nz;
    return fk_check(e, who);
}

/* ------------------------------------------------------------------ tuner --
 * Launch configuration of the two persistent sweep kernels, chosen per work
 * list by timing (no counterpart in the reference, whose OpenMP loops have a
 * fixed chunk size, constants.F90:23).  The knobs (fteik_b200_setSlabConfig)
 * the caller left at -1 are searched on the first solve of a new work list,
 * eagerly, with CUDA events around each kernel:
 *   1. staged x pairs x progress (8 | 32), all resident blocks;
 *   2. the best of 1 at 3 and 2 resident blocks per SM;
 * the pass kernel takes the fastest pass time, the initialisation kernel the
 * blocks per SM of the fastest initialisation time.  Every candidate is run
 * twice and timed by its faster run.  Every configuration gives the same
 * fields bit for bit, so the search changes only the time.  The choice is
 * kept per work list (grid shapes, sources per grid, precision, passes) in
 * memory and, when FTEIK_B200_TUNE_CACHE names a file, in that file, so
 * later processes skip the search. */
static void tune_apply(const int t[6])
{
    SB.plan.dev.staged = SB.precision == 4 && t[0] == 1;
    SB.plan.dev.pairs = t[1] ? SB.plan.pairs_all : NULL;
    SB.plan.dev.progress = t[2];
    SB.plan.dev.blocks_per_sm = t[3];
    SB.plan.dev.init_blocks_per_sm = t[4];
    SB.plan.dev.init_pairs = (SB.precision == 4 && t[5]) ? SB.plan.pairs_all : NULL;
    memcpy(SB.tuned, t, sizeof(SB.tuned));
}

static void tune_key(char *key, size_t cap)
{
    struct cudaDeviceProp prop;
    int dev = 0;
    cudaGetDevice(&dev);
    if (cudaGetDeviceProperties(&prop, dev) != cudaSuccess) {
        prop.name[0] = 0;
        prop.multiProcessorCount = 0;
    }
    size_t o = (size_t)snprintf(key, cap, "%s|sm%d|p%d|n%d|c%d:%d|", prop.name, prop.multiProcessorCount,
                                SB.precision, SB.nsweep, SB.conv_tol >= 0.0, SB.max_pass);
    for (int i = 0; i < SB.ngrid && o < cap; i++)
        o += (size_t)snprintf(key + o, cap - o, "%dx%dx%dx%d;", SB.g[i].nz, SB.g[i].nx, SB.g[i].ny, SB.g[i].nsrc);
    for (char *c = key; *c; c++)
        if (*c == ' ' || *c == '\t' || *c == '\n') *c = '_';
}

#define TUNE_MEM 16
static char g_tune_key[TUNE_MEM][512];
static int g_tune_val[TUNE_MEM][6];
static int g_tune_n = 0;

static int tune_lookup(const char *key, int t[6])
{
    for (int i = 0; i < g_tune_n; i++)
        if (strcmp(g_tune_key[i], key) == 0) { memcpy(t, g_tune_val[i], 6 * sizeof(int)); return 1; }
    const char *path = getenv("FTEIK_B200_TUNE_CACHE");
    if (!path || !*path) return 0;
    FILE *f = fopen(path, "r");
    if (!f) return 0;
    char line[700], k[600];
    int found = 0;
    while (fgets(line, sizeof(line), f))
        if (sscanf(line, "%599s %d %d %d %d %d %d", k, &t[0], &t[1], &t[2], &t[3], &t[4], &t[5]) == 7 &&
            strcmp(k, key) == 0)
            found = 1;   /* the last line for a key wins */
    fclose(f);
    return found;
}

static void tune_store(const char *key, const int t[6])
{
    const int i = g_tune_n < TUNE_MEM ? g_tune_n++ : TUNE_MEM - 1;
    snprintf(g_tune_key[i], sizeof(g_tune_key[i]), "%s", key);
    memcpy(g_tune_val[i], t, 6 * sizeof(int));
    const char *path = getenv("FTEIK_B200_TUNE_CACHE");
    if (!path || !*path) return;
    FILE *f = fopen(path, "a");
    if (!f) return;
    fprintf(f, "%s %d %d %d %d %d %d\n", key, t[0], t[1], t[2], t[3], t[4], t[5]);
    fclose(f);
}

/* One eager solve of the current plan with events around both kernels. */
static int tune_time(float *init_ms, float *pass_ms)
{
    cudaStream_t s = fk_stream();
    fk3d_slabs_set_events(SB.ev);
    int e = fk3d_solve_slabs(SB.precision, SB.grids_dev, SB.work_dev, SB.nwork, &SB.plan.dev, SB.res_dev,
                             SB.eps, SB.nsweep, SB.conv_tol, SB.max_pass, s);
    fk3d_slabs_set_events(NULL);
    if (!e) e = (int)cudaEventSynchronize(SB.ev[2]);
    if (!e) e = (int)cudaEventElapsedTime(init_ms, SB.ev[0], SB.ev[1]);
    if (!e) e = (int)cudaEventElapsedTime(pass_ms, SB.ev[1], SB.ev[2]);
    if (!e) e = (int)cudaMemcpyAsync(SB.res_host, SB.res_dev, sizeof(fk_result3d_t) * (size_t)SB.nwork,
                                    cudaMemcpyDeviceToHost, s);
    if (!e) e = (int)cudaStreamSynchronize(s);
    for (int w = 0; !e && w < SB.nwork; w++)
        if (SB.res_host[w].status) e = (int)cudaErrorLaunchFailure;
    return e;
}

static int ensure_events(void)
{
    if (SB.have_ev) return 0;
    bool ok = true;
    for (int i = 0; i < 3; i++) ok = ok && cudaEventCreate(&SB.ev[i]) == cudaSuccess;
    SB.have_ev = ok;
    return ok ? 0 : 1;
}

static int tune(const char *who)
{
    const fk_slabcfg_t cfg = fk_slabcfg();
    /* a knob at 0 is explicit: progress by task count, all resident blocks */
    int t[6] = {SB.precision == 4 && cfg.staged == 1, cfg.pairs != 0, cfg.progress > 0 ? cfg.progress : 0,
                cfg.blocks_per_sm > 0 ? cfg.blocks_per_sm : 0, cfg.blocks_per_sm > 0 ? cfg.blocks_per_sm : 0,
                SB.precision == 4 && cfg.pairs != 0};
    SB.tune_ms[0] = SB.tune_ms[1] = 0.0f;
    SB.tune_runs = 0;
    const bool search = (cfg.staged < 0 && SB.precision == 4) || cfg.pairs < 0 || cfg.progress < 0 ||
                        cfg.blocks_per_sm < 0;
    if (!search) { tune_apply(t); return 0; }
    char key[512];
    tune_key(key, sizeof(key));
    if (tune_lookup(key, t)) { tune_apply(t); return 0; }
    if (ensure_events()) { FK_ERR("%s: cannot create events", who); return 1; }
    const int st_n = (cfg.staged < 0 && SB.precision == 4) ? 2 : 1;
    const int pr_n = cfg.pairs < 0 ? 2 : 1;
    const int ch_n = cfg.progress < 0 ? 2 : 1;
    /* the two kernels are chosen apart: the passes by their time, the
     * initialisation sweeps (pairs, blocks per SM) by theirs */
    float best_pass = 3.4e38f, best_init = 3.4e38f;
    int best[6], best_i[2] = {t[4], t[5]};
    memcpy(best, t, sizeof(best));
    for (int a = 0; a < st_n * pr_n * ch_n; a++) {
        const int pr = pr_n == 2 ? 1 - (a / st_n) % 2 : t[1];
        int c[6] = {st_n == 2 ? a % 2 : t[0], pr, ch_n == 2 ? ((a / (st_n * pr_n)) % 2 ? 32 : 8) : t[2], t[3], t[4],
                    SB.precision == 4 && pr};
        tune_apply(c);
        float im = 3.4e38f, pm = 3.4e38f;
        for (int r = 0; r < 2; r++) {
            float i1, p1;
            if (fk_check(tune_time(&i1, &p1), who)) return 1;
            im = i1 < im ? i1 : im;
            pm = p1 < pm ? p1 : pm;
            SB.tune_runs++;
        }
        if (im < best_init) { best_init = im; best_i[0] = c[4]; best_i[1] = c[5]; }
        if (pm < best_pass) { best_pass = pm; memcpy(best, c, sizeof(best)); }
    }
    if (cfg.blocks_per_sm < 0) {
        for (int bps = 3; bps >= 2; bps--) {
            int c[6] = {best[0], best[1], best[2], bps, bps, best_i[1]};
            tune_apply(c);
            float im = 3.4e38f, pm = 3.4e38f;
            for (int r = 0; r < 2; r++) {
                float i1, p1;
                if (fk_check(tune_time(&i1, &p1), who)) return 1;
                im = i1 < im ? i1 : im;
                pm = p1 < pm ? p1 : pm;
                SB.tune_runs++;
            }
            if (im < best_init) { best_init = im; best_i[0] = bps; best_i[1] = c[5]; }
            if (pm < best_pass) { best_pass = pm; memcpy(best, c, sizeof(best)); }
        }
    }
    best[4] = best_i[0];
    best[5] = best_i[1];
    tune_apply(best);
    SB.tune_ms[0] = best_init;
    SB.tune_ms[1] = best_pass;
    tune_store(key, best);
    return 0;
}

void fteik_b200_batch3d_getSlabConfig(int *staged, int *pairs, int *progress, int *blocksPerSM,
                                      int *initBlocksPerSM, int *initPairs, float *initMs, float *passMs,
                                      int *tuneRuns, int *ierr)
{
    *initPairs = SB.tuned[5];
    *ierr = SB.graph_ok ? 0 : 1;
    if (!SB.graph_ok) FK_ERR("fteik_b200_batch3d_getSlabConfig: solve once first");
    *staged = SB.tuned[0];
    *pairs = SB.tuned[1];
    *progress = SB.tuned[2];
    *blocksPerSM = SB.tuned[3];
    *initBlocksPerSM = SB.tuned[4];
    *initMs = SB.tune_ms[0];
    *passMs = SB.tune_ms[1];
    *tuneRuns = SB.tune_runs;
}

void fteik_b200_batch3d_solve(int *ierr)
{
    const char *who = "fteik_b200_batch3d_solve";
    *ierr = 1;
    if (!SB.init) { FK_ERR("%s: batch not initialized", who); return; }
    cudaStream_t s = fk_stream();
    if (SB.graph_ok && SB.work_dirty) {
        if (upload_work(who)) return;
    }
    if (SB.graph_ok && (SB.spin_epoch != fk_spin_epoch() || SB.cfg_epoch != fk_slabcfg_epoch()))
        invalidate();   /* new poll limit or launch configuration */
    if (!SB.graph_ok) {
        if (build_work(who)) return;
        SB.work_dirty = false;
        if (tune(who)) return;
        cudaGraph_t graph;
        int e = (int)cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
        if (!e) {
            const int le = fk3d_solve_slabs(SB.precision, SB.grids_dev, SB.work_dev, SB.nwork, &SB.plan.dev,
                                            SB.res_dev, SB.eps, SB.nsweep, SB.conv_tol, SB.max_pass, s);
            e = (int)cudaStreamEndCapture(s, &graph);
            if (!e) e = le;
        }
        if (!e) e = (int)cudaGraphInstantiate(&SB.graph, graph, 0);
        if (!e) cudaGraphDestroy(graph);
        if (fk_check(e, who)) return;
        SB.graph_ok = true;
    }
    int e = (int)cudaGraphLaunch(SB.graph, s);
    if (!e) e = (int)cudaMemcpyAsync(SB.res_host, SB.res_dev, sizeof(fk_result3d_t) * (size_t)SB.nwork,
                                    cudaMemcpyDeviceToHost, s);
    if (!e) e = (int)cudaStreamSynchronize(s);
    if (fk_check(e, who)) return;
    for (int w = 0; w < SB.nwork; w++)
        if (SB.res_host[w].status) { FK_ERR("%s: work item %d failed", who, w); return; }
    SB.solved = true;
    *ierr = 0;
}

/* Launch the solve without waiting (the caller synchronises); used for
 * timing back-to-back solves. */
int fteik_b200_batch3d_solveAsync(void)
{
    if (!SB.graph_ok) return 1;
    return (int)cudaGraphLaunch(SB.graph, fk_stream());
}

static const fk_result3d_t *result_of(int igrid, int isrc, const char *who)
{
    bgrid_t *g = grid_of(igrid, who);
    if (!g) return NULL;
    if (!SB.solved) { FK_ERR("%s: not solved", who); return NULL; }
    if (isrc < 1 || isrc > g->nsrc) { FK_ERR("%s: source %d out of range", who, isrc); return NULL; }
    for (int w = 0; w < SB.nwork; w++)
        if (SB.work_order[w] == (((igrid - 1) << 20) | (isrc - 1))) return &SB.res_host[w];
    return NULL;
}

void fteik_b200_batch3d_getSolveInfo(int igrid, int isrc, double *residual, int *npass, int *ierr)
{
    const fk_result3d_t *r = result_of(igrid, isrc, "fteik_b200_batch3d_getSolveInfo");
    *ierr = r ? 0 : 1;
    *residual = r ? r->residual : 0.0;
    *npass = r ? r->npass : 0;
}

static int ensure_export(size_t n)
{
    if (SB.export_buf && SB.export_cap >= n) return 0;
    fk_dfree(SB.export_buf);
    SB.export_buf = (double *)fk_dalloc(sizeof(double) * n, "fteik_b200_batch3d");
    SB.export_cap = SB.export_buf ? n : 0;
    return SB.export_buf == NULL;
}

void fteik_b200_batch3d_getTravelTimeField64f(int igrid, int isrc, int ngrd, int order, double tt[],
                                              int *ierr)
{
    const char *who = "fteik_b200_batch3d_getTravelTimeField64f";
    *ierr = 1;
    if (!result_of(igrid, isrc, who)) return;
    bgrid_t *g = &SB.g[igrid - 1];
    if (ngrd != g->ngrd) { FK_ERR("%s: ngrd=%d, grid has %d", who, ngrd, g->ngrd); return; }
    if (ensure_export((size_t)ngrd)) return;
    const size_t fbytes = (size_t)g->zp * g->nx * g->ny * (size_t)SB.precision;
    cudaStream_t s = fk_stream();
    int e = fk_field_to_f64(SB.precision, 1, g->nz, g->nx, g->ny, g->zp,
                            (char *)g->fields + fbytes * (size_t)(isrc - 1), order, SB.export_buf, s);
    if (!e) e = (int)cudaMemcpyAsync(tt, SB.export_buf, sizeof(double) * (size_t)ngrd, cudaMemcpyDeviceToHost, s);
    if (!e) e = (int)cudaStreamSynchronize(s);
    *ierr = fk_check(e, who);
}

void fteik_b200_batch3d_getTravelTimeFields32f(int igrid, long long nval, float tt[], int *ierr)
{
    /* Unpadding copy of every source's FP32 field: one 2D memcpy per grid
     * (rows of nz floats with pitch zp). */
    const char *who = "fteik_b200_batch3d_getTravelTimeFields32f";
    *ierr = 1;
    bgrid_t *g = grid_of(igrid, who);
    if (!g) return;
    if (!SB.solved) { FK_ERR("%s: not solved", who); return; }
    if (SB.precision != 4) { FK_ERR("%s: the batch was solved in FP64", who); return; }
    if (nval < (long long)g->nsrc * g->ngrd) { FK_ERR("%s: nval too small", who); return; }
    /* unpad on the device in chunks of sources, one contiguous copy each */
    const size_t per_src = (size_t)g->ngrd * sizeof(float);
    int chunk = (int)((256u << 20) / per_src);
    if (chunk < 1) chunk = 1;
    if (chunk > g->nsrc) chunk = g->nsrc;
    float *st = (float *)stage_buf(per_src * (size_t)chunk, who);
    if (!st) return;
    cudaStream_t s = fk_stream();
    int e = 0;
    for (int s0 = 0; s0 < g->nsrc && !e; s0 += chunk) {
        const int ns = (g->nsrc - s0) < chunk ? (g->nsrc - s0) : chunk;
        const float *src = (const float *)g->fields + (size_t)s0 * g->zp * g->nx * g->ny;
        e = fk_unpad_f32(src, st, (size_t)ns * g->nx * g->ny, g->nz, g->zp, s);
        if (!e) e = (int)cudaMemcpyAsync(tt + (size_t)s0 * g->ngrd, st, per_src * (size_t)ns,
                                        cudaMemcpyDeviceToHost, s);
    }
    if (!e) e = (int)cudaStreamSynchronize(s);
    *ierr = fk_check(e, who);
}

void fteik_b200_batch3d_getTravelTimeFields32fAsync(int igrid, long long nval, float tt[], int *ierr)
{
    /* The tables unpacked into a per-grid device buffer on the library
     * stream (after this grid's previous download has left that buffer),
     * then copied to tt on a copy stream: the copy overlaps whatever the
     * caller enqueues next, a new solve included, which may overwrite the
     * fields as soon as the unpacking has run. */
    const char *who = "fteik_b200_batch3d_getTravelTimeFields32fAsync";
    *ierr = 1;
    bgrid_t *g = grid_of(igrid, who);
    if (!g) return;
    if (!SB.solved) { FK_ERR("%s: not solved", who); return; }
    if (SB.precision != 4) { FK_ERR("%s: the batch was solved in FP64", who); return; }
    if (nval < (long long)g->nsrc * g->ngrd) { FK_ERR("%s: nval too small", who); return; }
    const size_t bytes = (size_t)g->nsrc * g->ngrd * sizeof(float);
    int e = 0;
    if (!SB.copy_stream) e = (int)cudaStreamCreateWithFlags(&SB.copy_stream, cudaStreamNonBlocking);
    if (!e && !g->have_dl_ev) {
        e = (int)cudaEventCreateWithFlags(&g->dl_ready, cudaEventDisableTiming);
        if (!e) e = (int)cudaEventCreateWithFlags(&g->dl_done, cudaEventDisableTiming);
        g->have_dl_ev = !e;
    }
    if (fk_check(e, who)) return;
    cudaStream_t s = fk_stream();
    if (g->dl_cap < bytes) {
        e = (int)cudaStreamSynchronize(SB.copy_stream);   /* the old buffer may still be read */
        fk_dfree(g->dl_buf);
        g->dl_buf = (float *)fk_dalloc(bytes, who);
        g->dl_cap = g->dl_buf ? bytes : 0;
        if (!g->dl_buf) return;
    }
    if (!e) e = (int)cudaStreamWaitEvent(s, g->dl_done, 0);
    if (!e) e = fk_unpad_f32((const float *)g->fields, g->dl_buf, (size_t)g->nsrc * g->nx * g->ny, g->nz, g->zp, s);
    if (!e) e = (int)cudaEventRecord(g->dl_ready, s);
    if (!e) e = (int)cudaStreamWaitEvent(SB.copy_stream, g->dl_ready, 0);
    if (!e) e = (int)cudaMemcpyAsync(tt, g->dl_buf, bytes, cudaMemcpyDeviceToHost, SB.copy_stream);
    if (!e) e = (int)cudaEventRecord(g->dl_done, SB.copy_stream);
    *ierr = fk_check(e, who);
}

void fteik_b200_batch3d_waitDownloads(int *ierr)
{
    *ierr = 0;
    if (SB.copy_stream) *ierr = fk_check((int)cudaStreamSynchronize(SB.copy_stream), "fteik_b200_batch3d_waitDownloads");
}

void fteik_b200_batch3d_getTravelTimes64f(int igrid, int nval, double ttr[], int *ierr)
{
    const char *who = "fteik_b200_batch3d_getTravelTimes64f";
    *ierr = 1;
    bgrid_t *g = grid_of(igrid, who);
    if (!g) return;
    if (!SB.solved) { FK_ERR("%s: not solved", who); return; }
    if (g->nrec < 1) { FK_ERR("%s: no receivers", who); return; }
    if (nval < g->nsrc * g->nrec) { FK_ERR("%s: nval too small", who); return; }
    const size_t n = (size_t)g->nsrc * g->nrec;
    const size_t fbytes = (size_t)g->zp * g->nx * g->ny * (size_t)SB.precision;
    void **ptrs = (void **)malloc(sizeof(void *) * (size_t)g->nsrc);
    for (int s2 = 0; s2 < g->nsrc; s2++) ptrs[s2] = (char *)g->fields + fbytes * (size_t)s2;
    void **ptrs_dev = (void **)fk_dalloc(sizeof(void *) * (size_t)g->nsrc, who);
    if (!ptrs_dev || ensure_export(n)) { free(ptrs); fk_dfree(ptrs_dev); return; }
    cudaStream_t s = fk_stream();
    int e = (int)cudaMemcpyAsync(ptrs_dev, ptrs, sizeof(void *) * (size_t)g->nsrc, cudaMemcpyHostToDevice, s);
    if (!e) e = fk_receivers_batch(SB.precision, g->nz, g->nx, g->ny, g->zp, g->dz, g->dx, g->dy,
                                  ptrs_dev, g->nsrc, g->nrec, g->ri_dev, g->rd_dev, SB.export_buf, s);
    if (!e) e = (int)cudaMemcpyAsync(ttr, SB.export_buf, sizeof(double) * n, cudaMemcpyDeviceToHost, s);
    if (!e) e = (int)cudaStreamSynchronize(s);
    free(ptrs);
    fk_dfree(ptrs_dev);
    *ierr = fk_check(e, who);
}

float *fk_locate_table_row(int itf, int ngrd);

void fteik_b200_batch3d_exportToLocator(int igrid, int itf0, int *ierr)
{
    const char *who = "fteik_b200_batch3d_exportToLocator";
    *ierr = 1;
    bgrid_t *g = grid_of(igrid, who);
    if (!g) return;
    if (!SB.solved) { FK_ERR("%s: not solved", who); return; }
    if (SB.precision != 4) { FK_ERR("%s: the batch was solved in FP64", who); return; }
    float *dst0 = fk_locate_table_row(itf0, g->ngrd);
    float *dst1 = fk_locate_table_row(itf0 + g->nsrc - 1, g->ngrd);
    if (!dst0 || !dst1) { FK_ERR("%s: locator tables %d..%d unavailable for ngrd=%d", who, itf0, itf0 + g->nsrc - 1, g->ngrd); return; }
    const size_t fbytes = (size_t)g->zp * g->nx * g->ny * sizeof(float);
    int e = 0;
    for (int s2 = 0; s2 < g->nsrc && !e; s2++) {
        float *dst = fk_locate_table_row(itf0 + s2, g->ngrd);
        e = (int)cudaMemcpy2DAsync(dst, sizeof(float) * (size_t)g->nz,
                                   (char *)g->fields + fbytes * (size_t)s2, sizeof(float) * (size_t)g->zp,
                                   sizeof(float) * (size_t)g->nz, (size_t)g->nx * g->ny,
                                   cudaMemcpyDeviceToDevice, fk_stream());
    }
    if (!e) e = (int)cudaStreamSynchronize(fk_stream());
    *ierr = fk_check(e, who);
}

/* Run one solve outside the graph with CUDA events around its
 * initialisation kernel and its Gauss-Seidel kernel; returns their device
 * times.  The fields end as after fteik_b200_batch3d_solve. */
void fteik_b200_batch3d_timeSolve(float *init_ms, float *pass_ms, int *ierr)
{
    const char *who = "fteik_b200_batch3d_timeSolve";
    *init_ms = *pass_ms = 0.0f;
    *ierr = 1;
    if (!SB.graph_ok) { FK_ERR("%s: solve once first", who); return; }
    if (SB.work_dirty && upload_work(who)) return;
    if (ensure_events()) { FK_ERR("%s: cannot create events", who); return; }
    cudaStream_t s = fk_stream();
    fk3d_slabs_set_events(SB.ev);
    int e = fk3d_solve_slabs(SB.precision, SB.grids_dev, SB.work_dev, SB.nwork, &SB.plan.dev,
                             SB.res_dev, SB.eps, SB.nsweep, SB.conv_tol, SB.max_pass, s);
    fk3d_slabs_set_events(NULL);
    if (!e) e = (int)cudaEventSynchronize(SB.ev[2]);
    if (!e) e = (int)cudaEventElapsedTime(init_ms, SB.ev[0], SB.ev[1]);
    if (!e) e = (int)cudaEventElapsedTime(pass_ms, SB.ev[1], SB.ev[2]);
    *ierr = fk_check(e, who);
}
