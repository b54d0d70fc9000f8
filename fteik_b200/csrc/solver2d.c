/*
 * solver2d.c -- the reference's 2D solver module (solver2D.F90) over the
 * CUDA solve (FP64 on the device).
 */
#include "host_common.h"
#include "fteik_b200.h"

#include <stdint.h>
#include <stdlib.h>
#include <string.h>

static struct {
    bool init, have_times;
    int nsweep, verbose, src;
    double eps, conv_tol;
    double *tt;           /* device field [nx][zp] */
    double *export_buf;
    size_t export_cap;
    double *tt_rec;       /* host [nsrc][nrec] receiver times */
    fk_grid2d_t *grid_dev;
    fk_work2d_t *work_dev;
    fk_result3d_t *res_dev;
    /* solveLSM: all sources of a chunk in one launch */
    int cap;              /* sources per chunk the buffers hold */
    double *tt_all;       /* device [cap][nx][zp] */
    fk_work2d_t *work_all;
    fk_result3d_t *res_all;
    void **fptr_dev;      /* device [cap] field pointers (receiver gather) */
    double *rec_all;      /* device [cap][nrec] */
    int rec_cap;
    double *gx, *gz;      /* device [ngrd] gradient of the current field */
    bool have_grad;
} S2;

/* Ray paths of the last traceRaysTo* (host copies). */
static struct {
    int nray;
    int *npts, *nseg, *status;
    double *tn, *tne, *tcell;
    long long *pts_off, *seg_off;
    double *px, *pz, *lens;   /* positions relative to the model origin */
    int *cells;               /* 1-based natural cell index */
} R2;

static void rays_free(void)
{
    free(R2.npts); free(R2.nseg); free(R2.status); free(R2.tn); free(R2.tne); free(R2.tcell);
    free(R2.pts_off); free(R2.seg_off); free(R2.px); free(R2.pz); free(R2.lens); free(R2.cells);
    memset(&R2, 0, sizeof(R2));
}

void fteik_solver2d_free(void)
{
    fk_dfree(S2.tt); fk_dfree(S2.export_buf);
    fk_dfree(S2.grid_dev); fk_dfree(S2.work_dev); fk_dfree(S2.res_dev);
    fk_dfree(S2.tt_all); fk_dfree(S2.work_all); fk_dfree(S2.res_all); fk_dfree(S2.fptr_dev);
    fk_dfree(S2.rec_all); fk_dfree(S2.gx); fk_dfree(S2.gz);
    free(S2.tt_rec);
    memset(&S2, 0, sizeof(S2));
    S2.src = -1;
    rays_free();
    fk_rays_reset();
    fteik_receiver_free();
    fteik_source_free();
    fteik_model_free();
}

void fteik_solver2d_setVerbosity(int verbose) { S2.verbose = verbose; }
void fteik_solver2d_setConvergenceTolerance(double convTol) { S2.conv_tol = convTol; }

void fteik_solver2d_setNumberOfSweeps(int nsweep, int *ierr)
{
    *ierr = 0;
    S2.nsweep = 1;
    if (nsweep < 0) {
        FK_ERR("fteik_solver2d_setNumberOfSweeps: nsweep = %d must be positive", nsweep);
        *ierr = 1;
        return;
    }
    S2.nsweep = nsweep;
}

void fteik_solver2d_setSphereToCartEpsilon(double eps, int *ierr)
{
    *ierr = 0;
    S2.eps = 0.0;
    if (fk_model.nx < 1 || fk_model.nz < 1) {
        FK_ERR("fteik_solver2d_setSphereToCartEpsilon: Grid not yet set");
        *ierr = 1;
        return;
    }
    if ((int)eps > fk_model.nz || (int)eps > fk_model.nx) {
        FK_ERR("fteik_solver2d_setSphereToCartEpsilon: eps=%d bigger than the grid", (int)eps);
        *ierr = 1;
        return;
    }
    S2.eps = eps;
}

void fteik_solver2d_initialize(int nz, int nx, double z0, double x0, double dz, double dx,
                               int nsweep, double eps, double convTol, int verbose, int *ierr)
{
    /* solver2D.F90:124-198 */
    if (verbose > 0) fprintf(stdout, "fteik_solver2d_initialize64f: Initializing...\n");
    fteik_solver2d_free();
    S2.verbose = verbose;
    S2.conv_tol = convTol;
    fteik_model_initializeGeometry(false, nz, nx, 1, z0, x0, 0.0, dz, dx, 1.0, ierr);
    if (*ierr) { FK_ERR("fteik_solver2d_initialize64f: Error setting grid geometry"); return; }
    fteik_solver2d_setNumberOfSweeps(nsweep, ierr);
    if (*ierr) { FK_ERR("fteik_solver2d_initialize64f: Failed to set max number of sweeps"); return; }
    fteik_solver2d_setSphereToCartEpsilon(eps, ierr);
    if (*ierr) { FK_ERR("fteik_solver2d_initialize64f: Failed to set epsilon"); return; }
    if (fk_dev_ready("fteik_solver2d_initialize")) { *ierr = 1; return; }
    S2.init = true;
    S2.src = -1;
}

void fteik_solver2d_setVelocityModel64f(int ncell, const double vel[], int *ierr)
{
    fteik_model_setVelocityModel64f(ncell, vel, ierr);
}

void fteik_solver2d_setCellVelocityModel64f(int nc, int order, const double vel[], int *ierr)
{
    fteik_model_setCellVelocityModel64f(nc, order, vel, ierr);
}

void fteik_solver2d_setNodalVelocityModel64f(int ng, int order, const double vel[], int *ierr)
{
    fteik_model_setNodalVelocityModel64f(ng, order, vel, ierr);
}

static void alloc_rec(void)
{
    free(S2.tt_rec);
    S2.tt_rec = NULL;
    if (fk_source.have && fk_receiver.have) {
        size_t n = (size_t)fk_source.nsrc * fk_receiver.nrec;
        S2.tt_rec = (double *)malloc(sizeof(double) * n);
        for (size_t i = 0; i < n; i++) S2.tt_rec[i] = FK_HUGE;
    }
}

void fteik_solver2d_setSources64f(int nsrc, const double zsrc[], const double xsrc[], int *ierr)
{
    fteik_source_initialize64f(nsrc, zsrc, xsrc, NULL, S2.verbose, ierr);
    if (*ierr) { FK_ERR("fteik_solver2d_setSources64f: Failed to set source"); return; }
    alloc_rec();
}

void fteik_solver2d_setReceivers64f(int nrec, const double zrec[], const double xrec[], int *ierr)
{
    /* solver2D.F90:1560-1600 */
    *ierr = 0;
    if (nrec < 1) { fprintf(stdout, "fteik_solver2d_setReceivers64f: No receivers to set\n"); return; }
    double *y = (double *)malloc(sizeof(double) * (size_t)nrec);
    for (int i = 0; i < nrec; i++) y[i] = fk_model.y0;
    *ierr = fk_receiver_setup(nrec, zrec, xrec, y, S2.verbose);
    free(y);
    if (*ierr) FK_ERR("fteik_solver2d_setReceivers64f: Failed to set receivers");
    alloc_rec();
}

void fteik_solver2d_getNumberOfReceivers(int *nrec, int *ierr)
{
    fteik_receiver_getNumberOfReceivers(nrec, ierr);
}

static void set_work(fk_work2d_t *w, int isrc, double *tt)
{
    w->grid = 0;
    w->zsi = fk_source.zsi[isrc - 1]; w->xsi = fk_source.xsi[isrc - 1];
    w->zsa = fk_source.zsa[isrc - 1]; w->xsa = fk_source.xsa[isrc - 1];
    w->szero = fk_source_szero(isrc);
    w->tt = tt;
}

static int solve_one(int isrc, int fsm, const char *who)
{
    S2.have_times = false;
    S2.src = -1;
    if (!fk_model.have_model) { FK_ERR("%s: Model not yet set", who); return 1; }
    if (!fk_source.have || isrc < 1 || isrc > fk_source.nsrc) {
        FK_ERR("%s: Source number = %d must be in range [1,%d]", who, isrc,
               fk_source.have ? fk_source.nsrc : 0);
        return 1;
    }
    if (!S2.init || fk_dev_ready(who)) return 1;
    const int nz = fk_model.nz, nx = fk_model.nx, zp = FK_PITCH(nz);
    if (!S2.tt) S2.tt = (double *)fk_dalloc(sizeof(double) * (size_t)zp * nx, who);
    if (!S2.grid_dev) S2.grid_dev = (fk_grid2d_t *)fk_dalloc(sizeof(fk_grid2d_t), who);
    if (!S2.work_dev) S2.work_dev = (fk_work2d_t *)fk_dalloc(sizeof(fk_work2d_t), who);
    if (!S2.res_dev) S2.res_dev = (fk_result3d_t *)fk_dalloc(sizeof(fk_result3d_t), who);
    const double *slow = (const double *)fk_model_slow_dev(8);
    if (!S2.tt || !S2.grid_dev || !S2.work_dev || !S2.res_dev || !slow) return 1;
    fk_grid2d_t g = {nz, nx, zp, FK_PITCH(nz - 1), fk_model.dz, fk_model.dx, slow};
    fk_work2d_t w;
    set_work(&w, isrc, S2.tt);
    cudaStream_t s = fk_stream();
    fk_result3d_t res;
    int e = (int)cudaMemcpyAsync(S2.grid_dev, &g, sizeof(g), cudaMemcpyHostToDevice, s);
    if (!e) e = (int)cudaMemcpyAsync(S2.work_dev, &w, sizeof(w), cudaMemcpyHostToDevice, s);
    /* solver2D.F90:935-946: the reference's test never stops early */
    if (!e) e = fk2d_solve(fsm, S2.grid_dev, S2.work_dev, S2.res_dev, 1, nx, nz, S2.eps, S2.nsweep,
                          -1.0, 0, s);
    if (!e) e = (int)cudaMemcpyAsync(&res, S2.res_dev, sizeof(res), cudaMemcpyDeviceToHost, s);
    if (!e) e = (int)cudaStreamSynchronize(s);
    if (fk_check(e, who) || res.status) return 1;
    S2.have_times = true;
    S2.have_grad = false;
    return 0;
}

static int ensure_export2(size_t n)
{
    if (S2.export_buf && S2.export_cap >= n) return 0;
    fk_dfree(S2.export_buf);
    S2.export_buf = (double *)fk_dalloc(sizeof(double) * n, "fteik_solver2d");
    S2.export_cap = S2.export_buf ? n : 0;
    return S2.export_buf == NULL;
}

static int extract_receivers(int isrc)
{
    /* solver2D.F90:1449-1475 */
    if (!fk_receiver.have || !fk_source.have) return 0;
    if (!S2.tt_rec) alloc_rec();
    const int nrec = fk_receiver.nrec;
    if (fk_receiver_upload() || ensure_export2((size_t)nrec)) return 1;
    cudaStream_t s = fk_stream();
    int e = fk_receivers(8, 0, fk_model.nz, fk_model.nx, 1, FK_PITCH(fk_model.nz), fk_model.dz,
                         fk_model.dx, 1.0, S2.tt, nrec, fk_receiver.ri_dev, fk_receiver.rd_dev,
                         S2.export_buf, s);
    if (!e) e = (int)cudaMemcpyAsync(S2.tt_rec + (size_t)(isrc - 1) * nrec, S2.export_buf,
                                    sizeof(double) * (size_t)nrec, cudaMemcpyDeviceToHost, s);
    if (!e) e = (int)cudaStreamSynchronize(s);
    return fk_check(e, "fteik_solver2d: receiver extraction");
}

void fteik_solver2d_solveSourceLSM(int isrc, int *ierr)
{
    *ierr = solve_one(isrc, 0, "fteik_solver2d_solveSourceLSM");
    if (*ierr) return;
    S2.src = isrc;
    *ierr = extract_receivers(isrc);
}

void fteik_solver2d_solveSourceFSM(int isrc, int *ierr)
{
    /* solver2D.F90:1042-1280: the FSM leaves the receiver times alone */
    *ierr = solve_one(isrc, 1, "fteik_solver2d_solveSourceFSM");
}

/* All sources of a chunk solved by one launch (one CTA per source, each
 * with its own field), then the receiver times of the chunk gathered by one
 * launch.  Each CTA runs the single-source solve, so the fields equal
 * solveSourceLSM's bit for bit. */
static int solve_chunks(const char *who)
{
    const int nz = fk_model.nz, nx = fk_model.nx, zp = FK_PITCH(nz), nsrc = fk_source.nsrc;
    const size_t fsz = (size_t)zp * nx;
    /* chunk: up to 4096 sources and 1 GiB of fields */
    int cap = nsrc < 4096 ? nsrc : 4096;
    while (cap > 1 && (size_t)cap * fsz * sizeof(double) > ((size_t)1 << 30)) cap /= 2;
    if (cap > S2.cap) {
        fk_dfree(S2.tt_all); fk_dfree(S2.work_all); fk_dfree(S2.res_all); fk_dfree(S2.fptr_dev);
        S2.tt_all = (double *)fk_dalloc(sizeof(double) * fsz * (size_t)cap, who);
        S2.work_all = (fk_work2d_t *)fk_dalloc(sizeof(fk_work2d_t) * (size_t)cap, who);
        S2.res_all = (fk_result3d_t *)fk_dalloc(sizeof(fk_result3d_t) * (size_t)cap, who);
        S2.fptr_dev = (void **)fk_dalloc(sizeof(void *) * (size_t)cap, who);
        S2.cap = (S2.tt_all && S2.work_all && S2.res_all && S2.fptr_dev) ? cap : 0;
        if (!S2.cap) return 1;
    }
    const int nrec = (fk_receiver.have && S2.tt_rec) ? fk_receiver.nrec : 0;
    if (nrec > 0) {
        if (fk_receiver_upload()) return 1;
        if ((size_t)cap * nrec > (size_t)S2.rec_cap) {
            fk_dfree(S2.rec_all);
            S2.rec_all = (double *)fk_dalloc(sizeof(double) * (size_t)cap * nrec, who);
            S2.rec_cap = S2.rec_all ? cap * nrec : 0;
            if (!S2.rec_all) return 1;
        }
    }
    if (!S2.tt) S2.tt = (double *)fk_dalloc(sizeof(double) * fsz, who);
    if (!S2.grid_dev) S2.grid_dev = (fk_grid2d_t *)fk_dalloc(sizeof(fk_grid2d_t), who);
    const double *slow = (const double *)fk_model_slow_dev(8);
    if (!S2.tt || !S2.grid_dev || !slow) return 1;
    fk_grid2d_t g = {nz, nx, zp, FK_PITCH(nz - 1), fk_model.dz, fk_model.dx, slow};
    fk_work2d_t *w = (fk_work2d_t *)malloc(sizeof(fk_work2d_t) * (size_t)cap);
    void **fp = (void **)malloc(sizeof(void *) * (size_t)cap);
    fk_result3d_t *res = (fk_result3d_t *)malloc(sizeof(fk_result3d_t) * (size_t)cap);
    cudaStream_t s = fk_stream();
    int e = (w && fp && res) ? 0 : 1;
    if (!e) e = (int)cudaMemcpyAsync(S2.grid_dev, &g, sizeof(g), cudaMemcpyHostToDevice, s);
    for (int c0 = 0; !e && c0 < nsrc; c0 += cap) {
        const int n = nsrc - c0 < cap ? nsrc - c0 : cap;
        for (int i = 0; i < n; i++) {
            set_work(&w[i], c0 + i + 1, S2.tt_all + fsz * (size_t)i);
            fp[i] = S2.tt_all + fsz * (size_t)i;
        }
        e = (int)cudaMemcpyAsync(S2.work_all, w, sizeof(fk_work2d_t) * (size_t)n, cudaMemcpyHostToDevice, s);
        if (!e) e = (int)cudaMemcpyAsync(S2.fptr_dev, fp, sizeof(void *) * (size_t)n, cudaMemcpyHostToDevice, s);
        /* solver2D.F90:935-946: the reference's test never stops early */
        if (!e) e = fk2d_solve(0, S2.grid_dev, S2.work_all, S2.res_all, n, nx, nz, S2.eps, S2.nsweep, -1.0, 0, s);
        if (!e && nrec > 0)
            e = fk_receivers_batch2d(nx, zp, fk_model.dz, fk_model.dx, S2.fptr_dev, n, nrec, fk_receiver.ri_dev,
                                     fk_receiver.rd_dev, S2.rec_all, s);
        if (!e && nrec > 0)
            e = (int)cudaMemcpyAsync(S2.tt_rec + (size_t)c0 * nrec, S2.rec_all, sizeof(double) * (size_t)n * nrec,
                                     cudaMemcpyDeviceToHost, s);
        if (!e) e = (int)cudaMemcpyAsync(res, S2.res_all, sizeof(fk_result3d_t) * (size_t)n, cudaMemcpyDeviceToHost, s);
        /* the last source's field stays the current one, as after the reference's loop */
        if (!e && c0 + n == nsrc)
            e = (int)cudaMemcpyAsync(S2.tt, S2.tt_all + fsz * (size_t)(n - 1), sizeof(double) * fsz,
                                     cudaMemcpyDeviceToDevice, s);
        if (!e) e = (int)cudaStreamSynchronize(s);
        for (int i = 0; !e && i < n; i++)
            if (res[i].status) {
                FK_ERR("fteik_solver2d_solveLSM: Error solving source %d", c0 + i + 1);
                e = 1;
            }
    }
    free(w);
    free(fp);
    free(res);
    if (fk_check(e, who)) return 1;
    S2.have_times = true;
    S2.have_grad = false;
    S2.src = nsrc;
    return 0;
}

void fteik_solver2d_solveLSM(int *ierr)
{
    /* solver2D.F90:740-773 */
    *ierr = 0;
    S2.have_times = false;
    if (!fk_model.have_model) { FK_ERR("fteik_solver2d_solveLSM: Model not yet set"); *ierr = 1; return; }
    if (!fk_source.have || fk_source.nsrc < 1) {
        if (S2.verbose > 0) FK_ERR("fteik_solver2d_solveLSM: No sources");
        return;
    }
    if (!S2.init || fk_dev_ready("fteik_solver2d_solveLSM")) { *ierr = 1; return; }
    alloc_rec();
    *ierr = solve_chunks("fteik_solver2d_solveLSM");
}

void fteik_solver2d_getTravelTimeField64f(int ngrd, int order, double tt[], int *ierr)
{
    *ierr = 0;
    if (!S2.have_times) { FK_ERR("fteik_solver2d_getTravelTimeField64f: Travel times not yet computed"); *ierr = 1; return; }
    if (ngrd != fk_model.ngrd) {
        FK_ERR("fteik_solver2d_getTravelTimeField64f: ngin=%d /= ngrd =%d", ngrd, fk_model.ngrd);
        *ierr = 1;
        return;
    }
    if (order != FTEIK_XZ_ORDERING && order != FTEIK_NATURAL_ORDERING)
        fprintf(stdout, "fteik_solver2d_getTravelTimeField64f: Defaulting to natural order\n");
    if (ensure_export2((size_t)ngrd)) { *ierr = 1; return; }
    cudaStream_t s = fk_stream();
    int e = fk_field_to_f64(8, 0, fk_model.nz, fk_model.nx, 1, FK_PITCH(fk_model.nz), S2.tt,
                            order == FTEIK_XZ_ORDERING ? 1 : 0, S2.export_buf, s);
    if (!e) e = (int)cudaMemcpyAsync(tt, S2.export_buf, sizeof(double) * (size_t)ngrd,
                                    cudaMemcpyDeviceToHost, s);
    if (!e) e = (int)cudaStreamSynchronize(s);
    *ierr = fk_check(e, "fteik_solver2d_getTravelTimeField64f");
}

void fteik_solver2d_getTravelTimeFieldCell64f(int ncell, int order, double tt[], int *ierr)
{
    *ierr = 0;
    if (!S2.have_times) { FK_ERR("fteik_solver2d_getTravelTimeFieldCell64f: Travel times not yet computed"); *ierr = 1; return; }
    if (ncell != fk_model.ncell) {
        FK_ERR("fteik_solver2d_getTravelTimeFieldCell64f: ncin=%d /= ncell =%d", ncell, fk_model.ncell);
        *ierr = 1;
        return;
    }
    if (ensure_export2((size_t)ncell)) { *ierr = 1; return; }
    cudaStream_t s = fk_stream();
    int e = fk_field_cell_to_f64(8, 0, fk_model.nz, fk_model.nx, 1, FK_PITCH(fk_model.nz), S2.tt,
                                 order == FTEIK_XZ_ORDERING ? 1 : 0, S2.export_buf, s);
    if (!e) e = (int)cudaMemcpyAsync(tt, S2.export_buf, sizeof(double) * (size_t)ncell,
                                    cudaMemcpyDeviceToHost, s);
    if (!e) e = (int)cudaStreamSynchronize(s);
    *ierr = fk_check(e, "fteik_solver2d_getTravelTimeFieldCell64f");
}

void fteik_solver2d_getTravelTimes64f(int ldr, double ttr[], int *ierr)
{
    /* solver2D.F90:1410-1447 */
    *ierr = 0;
    if (!fk_receiver.have || fk_receiver.nrec < 1) {
        fprintf(stdout, "fteik_solver2d_getTravelTimes64f: No receivers\n");
        return;
    }
    if (!fk_source.have || fk_source.nsrc < 1) { FK_ERR("fteik_solver2d_getTravelTimes64f: No sources"); *ierr = 1; return; }
    if (!S2.have_times) { FK_ERR("fteik_solver2d_getTravelTimes64f: Travel times not yet computed"); *ierr = 1; return; }
    const int nrec = fk_receiver.nrec;
    if (ldr < nrec) {
        FK_ERR("fteik_solver2d_getTravelTimes64f: ldr=%d must be at least nrec=%d", ldr, nrec);
        *ierr = 1;
        return;
    }
    if (!S2.tt_rec) alloc_rec();
    if (ldr > nrec) memset(ttr, 0, sizeof(double) * (size_t)ldr * fk_source.nsrc);
    for (int i = 0; i < fk_source.nsrc; i++)
        memcpy(ttr + (size_t)i * ldr, S2.tt_rec + (size_t)i * nrec, sizeof(double) * (size_t)nrec);
}

/* solver2D.F90:984-1032 on the device, once per solved field. */
static int gradient2(const char *who)
{
    if (S2.have_grad) return 0;
    const size_t n = (size_t)fk_model.nz * fk_model.nx;
    if (!S2.gx) S2.gx = (double *)fk_dalloc(sizeof(double) * n, who);
    if (!S2.gz) S2.gz = (double *)fk_dalloc(sizeof(double) * n, who);
    if (!S2.gx || !S2.gz) return 1;
    int e = fk_gradient2d(fk_model.nz, fk_model.nx, FK_PITCH(fk_model.nz), fk_model.dz, fk_model.dx, S2.tt,
                          S2.gx, S2.gz, fk_stream());
    if (fk_check(e, who)) return 1;
    S2.have_grad = true;
    return 0;
}

void fteik_b200_solver2d_getTravelTimeGradient64f(int ngrd, double gradx[], double gradz[], int *ierr)
{
    const char *who = "fteik_b200_solver2d_getTravelTimeGradient64f";
    *ierr = 1;
    if (!S2.have_times) { FK_ERR("%s: Travel times not yet computed", who); return; }
    if (ngrd != fk_model.nz * fk_model.nx) { FK_ERR("%s: ngrd=%d must be %d", who, ngrd, fk_model.nz * fk_model.nx); return; }
    if (gradient2(who)) return;
    cudaStream_t s = fk_stream();
    int e = (int)cudaMemcpyAsync(gradx, S2.gx, sizeof(double) * (size_t)ngrd, cudaMemcpyDeviceToHost, s);
    if (!e) e = (int)cudaMemcpyAsync(gradz, S2.gz, sizeof(double) * (size_t)ngrd, cudaMemcpyDeviceToHost, s);
    if (!e) e = (int)cudaStreamSynchronize(s);
    if (fk_check(e, who)) return;
    *ierr = 0;
}

void fteik_solver2d_traceRaysToReceivers(int *ierr)
{
    /* solver2D.F90:283-306 */
    *ierr = 0;
    if (!fk_receiver.have || fk_receiver.nrec < 1) {
        FK_ERR("fteik_solver2d_traceRaysToReceivers: No receivers set");
        *ierr = 1;
        return;
    }
    fteik_solver2d_traceRaysToPoints(fk_receiver.nrec, fk_receiver.xrec, fk_receiver.zrec, ierr);
    if (*ierr) { FK_ERR("fteik_solver2d_traceRaysToReceivers: Failed to compute rays"); *ierr = 1; }
}

/* rays.F90:449-670 on the device: every ray of the points at once, one
 * thread each (rays2d.cu), counted then written; results kept on the host. */
static int trace2d(int np, const double *xp, const double *zp, const char *who)
{
    rays_free();
    const int nz = fk_model.nz, nx = fk_model.nx, zp_ = FK_PITCH(nz), zcp = FK_PITCH(nz - 1);
    const double *slow = (const double *)fk_model_slow_dev(8);
    if (!slow) return 1;
    const double xs = (double)(fk_source.xsi[S2.src - 1] - 1) * fk_model.dx;   /* source.F90:180-181 */
    const double zs = (double)(fk_source.zsi[S2.src - 1] - 1) * fk_model.dz;
    const int integ = fk_rays_integrator();
    R2.nray = np;
    R2.npts = (int *)malloc(sizeof(int) * (size_t)np);
    R2.nseg = (int *)malloc(sizeof(int) * (size_t)np);
    R2.status = (int *)malloc(sizeof(int) * (size_t)np);
    R2.tn = (double *)malloc(sizeof(double) * (size_t)np);
    R2.tne = (double *)malloc(sizeof(double) * (size_t)np);
    R2.tcell = (double *)malloc(sizeof(double) * (size_t)np);
    R2.pts_off = (long long *)malloc(sizeof(long long) * (size_t)np);
    R2.seg_off = (long long *)malloc(sizeof(long long) * (size_t)np);
    double *rel = (double *)malloc(sizeof(double) * 2 * (size_t)np);
    for (int i = 0; i < np; i++) {
        rel[i] = xp[i] - fk_model.x0;
        rel[np + i] = zp[i] - fk_model.z0;
    }
    /* device: [xr zr tn tne] doubles, [npts nseg status] ints, then the two offset arrays */
    const size_t nd = 4 * (size_t)np, ni = 3 * (size_t)np;
    char *d = (char *)fk_dalloc(sizeof(double) * nd + sizeof(int) * ni + sizeof(long long) * 2 * (size_t)np + 64, who);
    if (!d) { free(rel); return 1; }
    double *d_xr = (double *)d, *d_zr = d_xr + np, *d_tn = d_zr + np, *d_tne = d_tn + np;
    int *d_npts = (int *)(d_tne + np), *d_nseg = d_npts + np, *d_st = d_nseg + np;
    long long *d_po = (long long *)(((uintptr_t)(d_st + np) + 15) & ~(uintptr_t)15), *d_so = d_po + np;
    cudaStream_t st = fk_stream();
    int e = (int)cudaMemcpyAsync(d_xr, rel, sizeof(double) * 2 * (size_t)np, cudaMemcpyHostToDevice, st);
    if (!e) e = fk_rays2d(1, nz, nx, zp_, zcp, fk_model.dz, fk_model.dx, slow, S2.tt, S2.gx, S2.gz, integ, xs, zs,
                          np, d_xr, d_zr, d_npts, d_nseg, d_st, d_tn, d_tne, NULL, NULL, NULL, NULL, NULL, NULL, st);
    if (!e) e = (int)cudaMemcpyAsync(R2.npts, d_npts, sizeof(int) * (size_t)np, cudaMemcpyDeviceToHost, st);
    if (!e) e = (int)cudaMemcpyAsync(R2.nseg, d_nseg, sizeof(int) * (size_t)np, cudaMemcpyDeviceToHost, st);
    if (!e) e = (int)cudaMemcpyAsync(R2.status, d_st, sizeof(int) * (size_t)np, cudaMemcpyDeviceToHost, st);
    if (!e) e = (int)cudaMemcpyAsync(R2.tn, d_tn, sizeof(double) * (size_t)np, cudaMemcpyDeviceToHost, st);
    if (!e) e = (int)cudaMemcpyAsync(R2.tne, d_tne, sizeof(double) * (size_t)np, cudaMemcpyDeviceToHost, st);
    if (!e) e = (int)cudaStreamSynchronize(st);
    free(rel);
    if (fk_check(e, who)) { fk_dfree(d); return 1; }
    long long tp = 0, ts = 0;
    for (int i = 0; i < np; i++) {
        R2.pts_off[i] = tp;
        R2.seg_off[i] = ts;
        tp += R2.npts[i];
        ts += R2.nseg[i];
    }
    R2.px = (double *)malloc(sizeof(double) * (size_t)(tp ? tp : 1));
    R2.pz = (double *)malloc(sizeof(double) * (size_t)(tp ? tp : 1));
    R2.lens = (double *)malloc(sizeof(double) * (size_t)(ts ? ts : 1));
    R2.cells = (int *)malloc(sizeof(int) * (size_t)(ts ? ts : 1));
    char *o = (char *)fk_dalloc(sizeof(double) * (size_t)(2 * tp + ts) + sizeof(int) * (size_t)ts + 64, who);
    if (!o) { fk_dfree(d); return 1; }
    double *d_px = (double *)o, *d_pz = d_px + tp, *d_len = d_pz + tp;
    int *d_cells = (int *)(d_len + ts);
    e = (int)cudaMemcpyAsync(d_po, R2.pts_off, sizeof(long long) * (size_t)np, cudaMemcpyHostToDevice, st);
    if (!e) e = (int)cudaMemcpyAsync(d_so, R2.seg_off, sizeof(long long) * (size_t)np, cudaMemcpyHostToDevice, st);
    if (!e) e = fk_rays2d(2, nz, nx, zp_, zcp, fk_model.dz, fk_model.dx, slow, S2.tt, S2.gx, S2.gz, integ, xs, zs,
                          np, d_xr, d_zr, d_npts, d_nseg, d_st, d_tn, d_tne, d_po, d_so, d_px, d_pz, d_cells,
                          d_len, st);
    if (!e && tp) e = (int)cudaMemcpyAsync(R2.px, d_px, sizeof(double) * (size_t)tp, cudaMemcpyDeviceToHost, st);
    if (!e && tp) e = (int)cudaMemcpyAsync(R2.pz, d_pz, sizeof(double) * (size_t)tp, cudaMemcpyDeviceToHost, st);
    if (!e && ts) e = (int)cudaMemcpyAsync(R2.lens, d_len, sizeof(double) * (size_t)ts, cudaMemcpyDeviceToHost, st);
    if (!e && ts) e = (int)cudaMemcpyAsync(R2.cells, d_cells, sizeof(int) * (size_t)ts, cudaMemcpyDeviceToHost, st);
    if (!e) e = (int)cudaStreamSynchronize(st);
    fk_dfree(o);
    fk_dfree(d);
    if (fk_check(e, who)) return 1;
    /* the time of each ray from its (cell, length) pieces (rays.F90:650) */
    int bad = 0;
    for (int i = 0; i < np; i++) {
        double t = 0.0;
        for (int k = 0; k < R2.nseg[i]; k++) t += R2.lens[R2.seg_off[i] + k] * fk_model.slow[R2.cells[R2.seg_off[i] + k] - 1];
        R2.tcell[i] = t;
        if (R2.status[i]) {
            FK_ERR("fteik_rays_trace2d: Ray path %d failed to terminate", i + 1);
            bad = 1;
        }
    }
    return bad;
}

void fteik_solver2d_traceRaysToPoints(int np, const double xp[], const double zp[], int *ierr)
{
    /* solver2D.F90:310-350: the gradient of the current field, the ray end
     * points, then the ray paths (rays.F90:406-670), which the reference
     * keeps in module variables and this library returns through
     * fteik_b200_solver2d_getRay*. */
    *ierr = 0;
    if (!S2.have_times) {
        FK_ERR("fteik_solver2d_traceRaysToPoints: Travel time field not yet computed");
        *ierr = 1;
        return;
    }
    if (gradient2("fteik_solver2d_traceRaysToPoints")) { *ierr = 1; return; }
    if (fk_check_ray_points(false, np, zp, xp, NULL)) {
        FK_ERR("fteik_solver2d_traceRaysToPoints: Failed to set ray origins");
        *ierr = 1;
        return;
    }
    if (trace2d(np, xp, zp, "fteik_solver2d_traceRaysToPoints")) {
        FK_ERR("fteik_solver2d_traceRaysToPoints: Failed to compute rays");
        *ierr = 1;
    }
}

void fteik_b200_solver2d_getNumberOfRays(int *nray, int *ierr)
{
    *nray = R2.nray;
    *ierr = 0;
}

void fteik_b200_solver2d_getRayTimes(int nray, double tstep[], double tfield[], double tcell[], int status[],
                                     int *ierr)
{
    *ierr = 1;
    if (nray != R2.nray || R2.nray < 1) {
        FK_ERR("fteik_b200_solver2d_getRayTimes: nray=%d but %d rays are traced", nray, R2.nray);
        return;
    }
    for (int i = 0; i < nray; i++) {
        tstep[i] = R2.tn[i];
        tfield[i] = R2.tne[i];
        tcell[i] = R2.tcell[i];
        status[i] = R2.status[i];
    }
    *ierr = 0;
}

void fteik_b200_solver2d_getRayPath(int ir, int maxpts, double x[], double z[], int *npts, int *ierr)
{
    *ierr = 1;
    *npts = 0;
    if (ir < 1 || ir > R2.nray) { FK_ERR("fteik_b200_solver2d_getRayPath: ray %d not traced", ir); return; }
    *npts = R2.npts[ir - 1];
    if (maxpts == 0) { *ierr = 0; return; }          /* size query */
    if (maxpts < *npts) { FK_ERR("fteik_b200_solver2d_getRayPath: maxpts=%d < %d", maxpts, *npts); return; }
    for (int k = 0; k < *npts; k++) {
        x[k] = R2.px[R2.pts_off[ir - 1] + k] + fk_model.x0;
        z[k] = R2.pz[R2.pts_off[ir - 1] + k] + fk_model.z0;
    }
    *ierr = 0;
}

void fteik_b200_solver2d_getRayCells(int ir, int maxseg, int cells[], double lengths[], int *nseg, int *ierr)
{
    *ierr = 1;
    *nseg = 0;
    if (ir < 1 || ir > R2.nray) { FK_ERR("fteik_b200_solver2d_getRayCells: ray %d not traced", ir); return; }
    *nseg = R2.nseg[ir - 1];
    if (maxseg == 0) { *ierr = 0; return; }          /* size query */
    if (maxseg < *nseg) { FK_ERR("fteik_b200_solver2d_getRayCells: maxseg=%d < %d", maxseg, *nseg); return; }
    for (int k = 0; k < *nseg; k++) {
        cells[k] = R2.cells[R2.seg_off[ir - 1] + k];
        lengths[k] = R2.lens[R2.seg_off[ir - 1] + k];
    }
    *ierr = 0;
}
