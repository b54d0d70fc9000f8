/*
 * solver2d.c -- the reference's 2D solver module (solver2D.F90) over the
 * CUDA solve (FP64 on the device).
 */
#include "host_common.h"
#include "fteik_b200.h"

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
} S2;

void fteik_solver2d_free(void)
{
    fk_dfree(S2.tt); fk_dfree(S2.export_buf);
    fk_dfree(S2.grid_dev); fk_dfree(S2.work_dev); fk_dfree(S2.res_dev);
    free(S2.tt_rec);
    memset(&S2, 0, sizeof(S2));
    S2.src = -1;
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
    if (nx > 1024) {
        FK_ERR("fteik_solver2d_initialize: nx=%d exceeds the 1024 columns one CTA walks", nx);
        *ierr = 1;
        return;
    }
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
    w.grid = 0;
    w.zsi = fk_source.zsi[isrc - 1]; w.xsi = fk_source.xsi[isrc - 1];
    w.zsa = fk_source.zsa[isrc - 1]; w.xsa = fk_source.xsa[isrc - 1];
    w.szero = fk_source_szero(isrc);
    w.tt = S2.tt;
    cudaStream_t s = fk_stream();
    fk_result3d_t res;
    int e = (int)cudaMemcpyAsync(S2.grid_dev, &g, sizeof(g), cudaMemcpyHostToDevice, s);
    if (!e) e = (int)cudaMemcpyAsync(S2.work_dev, &w, sizeof(w), cudaMemcpyHostToDevice, s);
    /* solver2D.F90:935-946: the reference's test never stops early */
    if (!e) e = fk2d_solve(fsm, S2.grid_dev, S2.work_dev, S2.res_dev, 1, nx, S2.eps, S2.nsweep,
                          -1.0, 0, s);
    if (!e) e = (int)cudaMemcpyAsync(&res, S2.res_dev, sizeof(res), cudaMemcpyDeviceToHost, s);
    if (!e) e = (int)cudaStreamSynchronize(s);
    if (fk_check(e, who) || res.status) return 1;
    S2.have_times = true;
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

void fteik_solver2d_solveLSM(int *ierr)
{
    /* solver2D.F90:740-773 */
    *ierr = 0;
    if (!fk_model.have_model) { FK_ERR("fteik_solver2d_solveLSM: Model not yet set"); *ierr = 1; return; }
    if (!fk_source.have || fk_source.nsrc < 1) {
        if (S2.verbose > 0) FK_ERR("fteik_solver2d_solveLSM: No sources");
        return;
    }
    alloc_rec();
    for (int i = 1; i <= fk_source.nsrc; i++) {
        fteik_solver2d_solveSourceLSM(i, ierr);
        if (*ierr) { FK_ERR("fteik_solver2d_solveLSM: Error solving source %d", i); return; }
    }
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

void fteik_solver2d_traceRaysToReceivers(int *ierr)
{
    FK_ERR("fteik_solver2d_traceRaysToReceivers: ray tracing is not part of this library");
    *ierr = 1;
}

void fteik_solver2d_traceRaysToPoints(int np, const double xp[], const double zp[], int *ierr)
{
    (void)np; (void)xp; (void)zp;
    FK_ERR("fteik_solver2d_traceRaysToPoints: ray tracing is not part of this library");
    *ierr = 1;
}
