/*
 * solver3d.c -- the reference's 3D solver module (solver3D.F90) over the
 * CUDA solve: state and argument checks in C, every sweep on the device.
 */
#include "host_common.h"
#include "fteik_b200.h"
#include "slabplan.h"

#include <stdlib.h>
#include <string.h>

static struct {
    bool init, have_times;
    int nsweep, verbose, src, precision;
    double eps, conv_tol;
    void *tt;               /* device field, padded, FP32 or FP64 */
    double *export_buf;     /* device FP64 staging for exports */
    fk_grid3d_t *grid_dev;
    fk_work3d_t *work_dev;
    fk_result3d_t *res_dev;
    fk_slabplan_t plan;
    int plan_npass;
    int plan_cfg;           /* slab configuration epoch the plan was built with */
    fk_result3d_t last;
    double *grad;           /* device [3 ngrd] gradient of the current field */
    bool have_grad;
} S3 = {.precision = 4};

static void free_buffers(void)
{
    fk_dfree(S3.tt); S3.tt = NULL;
    fk_dfree(S3.export_buf); S3.export_buf = NULL;
    fk_dfree(S3.grid_dev); S3.grid_dev = NULL;
    fk_dfree(S3.work_dev); S3.work_dev = NULL;
    fk_dfree(S3.res_dev); S3.res_dev = NULL;
    fk_dfree(S3.grad); S3.grad = NULL;
    S3.have_grad = false;
    fk_slabplan_free(&S3.plan);
    S3.plan_npass = 0;
}

void fteik_solver3d_free(void)
{
    /* solver3D.F90:575-610 */
    free_buffers();
    int prec = S3.precision;
    memset(&S3, 0, sizeof(S3));
    S3.precision = prec;
    S3.src = -1;
    fk_rays_reset();
    fteik_receiver_free();
    fteik_source_free();
    fteik_model_free();
}

void fteik_solver3d_setVerbosity(int verbose) { S3.verbose = verbose; }
void fteik_solver3d_setConvergenceTolerance(double convTol) { S3.conv_tol = convTol; }

void fteik_solver3d_setNumberOfSweeps(int nsweep, int *ierr)
{
    *ierr = 0;
    S3.nsweep = 0;
    if (nsweep < 0) {
        FK_ERR("fteik_solver3d_setNumberOfSweeps: nsweep = %d must be positive", nsweep);
        *ierr = 1;
        return;
    }
    S3.nsweep = nsweep;
}

void fteik_solver3d_setSphereToCartEpsilon(double eps, int *ierr)
{
    /* solver3D.F90:640-673 */
    *ierr = 0;
    S3.eps = 0.0;
    if (fk_model.nx < 1 || fk_model.ny < 1 || fk_model.nz < 1) {
        FK_ERR("fteik_solver3d_setSphereToCartEpsilon: Grid not yet set");
        *ierr = 1;
        return;
    }
    if ((int)eps > fk_model.nz || (int)eps > fk_model.nx || (int)eps > fk_model.ny) {
        FK_ERR("fteik_solver3d_setSphereToCartEpsilon: eps=%d bigger than the grid", (int)eps);
        *ierr = 1;
        return;
    }
    S3.eps = eps;
}

/* Solve precision of the drop-in entry points: 4 (default, FP32 fields) or
 * 8 (FP64 fields, the CPU algorithm's rounding). */
void fteik_b200_solver3d_setPrecision(int precision, int *ierr)
{
    *ierr = 0;
    if (precision != 4 && precision != 8) { FK_ERR("fteik_b200_solver3d_setPrecision: 4 or 8"); *ierr = 1; return; }
    if (precision != S3.precision) {
        fk_dfree(S3.tt); S3.tt = NULL;
        S3.have_times = false;
    }
    S3.precision = precision;
}

void fteik_solver3d_initialize(int nz, int nx, int ny, double z0, double x0, double y0,
                               double dz, double dx, double dy, int nsweep, double eps,
                               double convTol, int verbose, int *ierr)
{
    /* solver3D.F90:126-184 */
    if (verbose > 0) fprintf(stdout, "fteik_solver3d_initialize: Initializing...\n");
    fteik_solver3d_free();
    S3.verbose = verbose;
    S3.conv_tol = convTol;
    fteik_model_initializeGeometry(true, nz, nx, ny, z0, x0, y0, dz, dx, dy, ierr);
    if (*ierr) { FK_ERR("fteik_solver3d_initialize: Error setting grid geometry"); return; }
    fk_model.verbose = verbose;
    fteik_solver3d_setNumberOfSweeps(nsweep, ierr);
    if (*ierr) { FK_ERR("fteik_solver3d_initialize: Failed to set max number of sweeps"); return; }
    fteik_solver3d_setSphereToCartEpsilon(eps, ierr);
    if (*ierr) { FK_ERR("fteik_solver3d_initialize: Failed to set epsilon"); return; }
    if (fk_dev_ready("fteik_solver3d_initialize")) { *ierr = 1; return; }
    S3.init = true;
    S3.src = -1;
}

void fteik_solver3d_setVelocityModel64f(int ncell, const double vel[], int *ierr)
{
    fteik_model_setVelocityModel64f(ncell, vel, ierr);
    if (*ierr) FK_ERR("fteik_solver3d_setVelocityModel64f: Error setting velocity model");
}

void fteik_solver3d_setCellVelocityModel64f(int nc, int order, const double vel[], int *ierr)
{
    fteik_model_setCellVelocityModel64f(nc, order, vel, ierr);
    if (*ierr) FK_ERR("fteik_solver3d_setCellVelocityModel64f: Error setting velocity model");
}

void fteik_solver3d_setNodalVelocityModel64f(int ng, int order, const double vel[], int *ierr)
{
    fteik_model_setNodalVelocityModel64f(ng, order, vel, ierr);
    if (*ierr) FK_ERR("fteik_solver3d_setNodalVelocityModel64f: Error setting velocity model");
}

void fteik_solver3d_setSources64f(int nsrc, const double zsrc[], const double xsrc[],
                                  const double ysrc[], int *ierr)
{
    fteik_source_initialize64f(nsrc, zsrc, xsrc, ysrc, S3.verbose, ierr);
    if (*ierr) FK_ERR("fteik_solver3d_setSources64f: Failed to set source");
}

void fteik_solver3d_getNumberOfSources(int *nsrc, int *ierr)
{
    fteik_source_getNumberOfSources(nsrc, ierr);
    if (*ierr) FK_ERR("fteik_solver3d_getNumberOfSources: No sources initialized!");
}

void fteik_solver3d_setReceivers64f(int nrec, const double zrec[], const double xrec[],
                                    const double yrec[], int *ierr)
{
    *ierr = 0;
    if (nrec < 1) { fprintf(stdout, "fteik_solver3d_setReceivers64f: No receivers to set\n"); return; }
    *ierr = fk_receiver_setup(nrec, zrec, xrec, yrec, S3.verbose);
    if (*ierr) FK_ERR("fteik_solver3d_setReceivers64f: Failed to set receivers");
}

void fteik_solver3d_getNumberOfReceivers(int *nrec, int *ierr)
{
    fteik_receiver_getNumberOfReceivers(nrec, ierr);
}

static int ensure_buffers(void)
{
    const int nz = fk_model.nz, nx = fk_model.nx, ny = fk_model.ny;
    const size_t nfield = (size_t)FK_PITCH(nz) * nx * ny;
    if (!S3.tt) S3.tt = fk_dalloc(nfield * (size_t)S3.precision, "fteik_solver3d");
    if (!S3.grid_dev) S3.grid_dev = (fk_grid3d_t *)fk_dalloc(sizeof(fk_grid3d_t), "fteik_solver3d");
    if (!S3.work_dev) S3.work_dev = (fk_work3d_t *)fk_dalloc(sizeof(fk_work3d_t), "fteik_solver3d");
    if (!S3.res_dev) S3.res_dev = (fk_result3d_t *)fk_dalloc(sizeof(fk_result3d_t), "fteik_solver3d");
    return !(S3.tt && S3.grid_dev && S3.work_dev && S3.res_dev);
}

void fteik_solver3d_solveSourceLSM(int isrc, int *ierr)
{
    /* solver3D.F90:1156-1243 */
    *ierr = 0;
    S3.have_times = false;
    S3.src = -1;
    if (!fk_model.have_model) {
        FK_ERR("fteik_solver3d_solveSourceLSM: Model not yet set");
        *ierr = 1;
        return;
    }
    if (!fk_source.have || isrc < 1 || isrc > fk_source.nsrc) {
        FK_ERR("fteik_solver3d_solveSourceLSM: Source number = %d must be in range [1,%d]", isrc,
               fk_source.have ? fk_source.nsrc : 0);
        *ierr = 1;
        return;
    }
    if (!S3.init || fk_dev_ready("fteik_solver3d_solveSourceLSM") || ensure_buffers()) {
        *ierr = 1;
        return;
    }
    const void *slow = fk_model_slow_dev(S3.precision);
    if (!slow) { *ierr = 1; return; }
    fk_grid3d_t g;
    g.nz = fk_model.nz; g.nx = fk_model.nx; g.ny = fk_model.ny;
    g.zp = FK_PITCH(g.nz); g.zcp = FK_PITCH(g.nz - 1);
    g.dz = fk_model.dz; g.dx = fk_model.dx; g.dy = fk_model.dy;
    g.slow = slow;
    g.slowz = NULL;
    const fk_slabcfg_t cfg = fk_slabcfg();
    const bool staged = S3.precision == 4 && cfg.staged == 1;
    if (staged) {
        g.slowz = fk_model_slowz_dev();
        if (!g.slowz) { *ierr = 1; return; }
    }
    fk_work3d_t w;
    w.grid = 0;
    w.zsi = fk_source.zsi[isrc - 1]; w.xsi = fk_source.xsi[isrc - 1]; w.ysi = fk_source.ysi[isrc - 1];
    w.zsa = fk_source.zsa[isrc - 1]; w.xsa = fk_source.xsa[isrc - 1]; w.ysa = fk_source.ysa[isrc - 1];
    w.szero = fk_source_szero(isrc);
    w.tt = S3.tt;
    cudaStream_t s = fk_stream();
    int e = (int)cudaMemcpyAsync(S3.grid_dev, &g, sizeof(g), cudaMemcpyHostToDevice, s);
    if (!e) e = (int)cudaMemcpyAsync(S3.work_dev, &w, sizeof(w), cudaMemcpyHostToDevice, s);
    /* the reference's 3D solver has no convergence test: nsweep passes */
    if (!e) {
        if (!S3.plan.mem || S3.plan_npass < S3.nsweep || S3.plan.dev.spin_limit != fk_spin_limit() ||
            S3.plan_cfg != fk_slabcfg_epoch()) {
            const int gid0 = 0;
            if (fk_slabplan_build(&S3.plan, 1, &g.nx, &g.ny, &g.nz, &gid0, S3.nsweep, cfg.pairs != 0,
                                  "fteik_solver3d")) {
                *ierr = 1;
                return;
            }
            S3.plan_npass = S3.nsweep;
            S3.plan_cfg = fk_slabcfg_epoch();
        }
        S3.plan.dev.staged = staged;
        S3.plan.dev.progress = cfg.progress > 0 ? cfg.progress : 0;
        S3.plan.dev.blocks_per_sm = cfg.blocks_per_sm > 0 ? cfg.blocks_per_sm : 0;
        S3.plan.dev.init_blocks_per_sm = S3.plan.dev.blocks_per_sm;
        e = fk3d_solve_slabs(S3.precision, S3.grid_dev, S3.work_dev, 1, &S3.plan.dev, S3.res_dev,
                             S3.eps, S3.nsweep, -1.0, 0, s);
    }
    if (!e) e = (int)cudaMemcpyAsync(&S3.last, S3.res_dev, sizeof(S3.last), cudaMemcpyDeviceToHost, s);
    if (!e) e = (int)cudaStreamSynchronize(s);
    if (fk_check(e, "fteik_solver3d_solveSourceLSM") || S3.last.status != 0) {
        *ierr = 1;
        return;
    }
    S3.have_times = true;
    S3.have_grad = false;
    S3.src = isrc;
}

static int ensure_export(size_t n)
{
    static size_t cap = 0;
    if (S3.export_buf && cap >= n) return 0;
    fk_dfree(S3.export_buf);
    S3.export_buf = (double *)fk_dalloc(sizeof(double) * n, "fteik_solver3d");
    cap = S3.export_buf ? n : 0;
    return S3.export_buf == NULL;
}

void fteik_solver3d_getTravelTimeField64f(int ngrd, int order, double tt[], int *ierr)
{
    /* solver3D.F90:844-897 */
    *ierr = 0;
    if (!S3.have_times) { FK_ERR("fteik_solver3d_getTravelTimeField64f: Travel times not yet computed"); *ierr = 1; return; }
    if (ngrd != fk_model.ngrd) {
        FK_ERR("fteik_solver3d_getTravelTimeField64f: ngin=%d /= ngrd =%d", ngrd, fk_model.ngrd);
        *ierr = 1;
        return;
    }
    if (order != FTEIK_NATURAL_ORDERING && order != FTEIK_XYZ_ORDERING && order != FTEIK_ZYX_ORDERING) {
        fprintf(stderr, "fteik_solver3d_getTravelTimeField64f: Defaulting to natural order\n");
        order = FTEIK_NATURAL_ORDERING;
    }
    if (ensure_export((size_t)ngrd)) { *ierr = 1; return; }
    cudaStream_t s = fk_stream();
    int e = fk_field_to_f64(S3.precision, 1, fk_model.nz, fk_model.nx, fk_model.ny,
                            FK_PITCH(fk_model.nz), S3.tt, order, S3.export_buf, s);
    if (!e) e = (int)cudaMemcpyAsync(tt, S3.export_buf, sizeof(double) * (size_t)ngrd,
                                    cudaMemcpyDeviceToHost, s);
    if (!e) e = (int)cudaStreamSynchronize(s);
    *ierr = fk_check(e, "fteik_solver3d_getTravelTimeField64f");
}

void fteik_solver3d_getTravelTimeFieldCell64f(int ncell, int order, double tt[], int *ierr)
{
    /* solver3D.F90:915-980.  The natural ordering returns cell averages in
     * cell order; the reference copies node values there (solver3D.F90:974). */
    *ierr = 0;
    if (!S3.have_times) { FK_ERR("fteik_solver3d_getTravelTimeFieldCell64f: Travel times not yet computed"); *ierr = 1; return; }
    if (ncell != fk_model.ncell) {
        FK_ERR("fteik_solver3d_getTravelTimeFieldCell64f: ncin=%d /= ncell =%d", ncell, fk_model.ncell);
        *ierr = 1;
        return;
    }
    if (ensure_export((size_t)ncell)) { *ierr = 1; return; }
    cudaStream_t s = fk_stream();
    int e = fk_field_cell_to_f64(S3.precision, 1, fk_model.nz, fk_model.nx, fk_model.ny,
                                 FK_PITCH(fk_model.nz), S3.tt, order, S3.export_buf, s);
    if (!e) e = (int)cudaMemcpyAsync(tt, S3.export_buf, sizeof(double) * (size_t)ncell,
                                    cudaMemcpyDeviceToHost, s);
    if (!e) e = (int)cudaStreamSynchronize(s);
    *ierr = fk_check(e, "fteik_solver3d_getTravelTimeFieldCell64f");
}

void fteik_solver3d_getTravelTimes64f(int nrec, double ttr[], int *ierr)
{
    /* solver3D.F90:990-1016 -> receiver.F90:217-313 on the device field */
    *ierr = 0;
    if (nrec <= 0) { fprintf(stdout, "fteik_solver3d_getTravelTimes64f: No receivers\n"); return; }
    if (!S3.have_times) { FK_ERR("fteik_solver3d_getTravelTimes64f: Travel times not yet computed"); *ierr = 1; return; }
    if (!fk_receiver.have) { FK_ERR("fteik_solver3d_getTravelTimes64f: Error getting travel times"); *ierr = 1; return; }
    const int n = nrec < fk_receiver.nrec ? nrec : fk_receiver.nrec;
    for (int r = n; r < nrec; r++) ttr[r] = FK_HUGE;
    if (fk_receiver_upload() || ensure_export((size_t)(n > 0 ? n : 1))) { *ierr = 1; return; }
    cudaStream_t s = fk_stream();
    int e = fk_receivers(S3.precision, 1, fk_model.nz, fk_model.nx, fk_model.ny,
                         FK_PITCH(fk_model.nz), fk_model.dz, fk_model.dx, fk_model.dy, S3.tt, n,
                         fk_receiver.ri_dev, fk_receiver.rd_dev, S3.export_buf, s);
    if (!e) e = (int)cudaMemcpyAsync(ttr, S3.export_buf, sizeof(double) * (size_t)n,
                                    cudaMemcpyDeviceToHost, s);
    if (!e) e = (int)cudaStreamSynchronize(s);
    *ierr = fk_check(e, "fteik_solver3d_getTravelTimes64f");
}

/* Residual and passes of the last drop-in solve. */
void fteik_b200_solver3d_getSolveInfo(double *residual, int *npass, int *ierr)
{
    *ierr = S3.have_times ? 0 : 1;
    *residual = S3.last.residual;
    *npass = S3.last.npass;
}

/* Device pointer of the current FP32/FP64 field (for in-process callers). */
const void *fk_solver3d_field(int *precision)
{
    if (precision) *precision = S3.precision;
    return S3.have_times ? S3.tt : NULL;
}

/* solver3D.F90:1249-1321 on the device, once per solved field. */
static int gradient(const char *who)
{
    if (S3.have_grad) return 0;
    const size_t n = (size_t)fk_model.nz * fk_model.nx * fk_model.ny;
    if (!S3.grad) S3.grad = (double *)fk_dalloc(sizeof(double) * 3 * n, who);
    if (!S3.grad) return 1;
    int e = fk_gradient3d(S3.precision, fk_model.nz, fk_model.nx, fk_model.ny, FK_PITCH(fk_model.nz),
                          fk_model.dz, fk_model.dx, fk_model.dy, S3.tt, S3.grad, fk_stream());
    if (fk_check(e, who)) return 1;
    S3.have_grad = true;
    return 0;
}

void fteik_b200_solver3d_getTravelTimeGradient64f(int ngrd, double grad[], int *ierr)
{
    const char *who = "fteik_b200_solver3d_getTravelTimeGradient64f";
    *ierr = 1;
    if (!S3.have_times) { FK_ERR("%s: Travel times not yet computed", who); return; }
    if (ngrd != fk_model.ngrd) { FK_ERR("%s: ngrd=%d must be %d", who, ngrd, fk_model.ngrd); return; }
    if (gradient(who)) return;
    cudaStream_t s = fk_stream();
    int e = (int)cudaMemcpyAsync(grad, S3.grad, sizeof(double) * 3 * (size_t)ngrd, cudaMemcpyDeviceToHost, s);
    if (!e) e = (int)cudaStreamSynchronize(s);
    if (fk_check(e, who)) return;
    *ierr = 0;
}

void fteik_solver3d_traceRaysToReceivers(int *ierr)
{
    /* solver3D.F90:756-782 */
    *ierr = 0;
    if (!fk_receiver.have || fk_receiver.nrec < 1) {
        FK_ERR("fteik_solver3d_traceRaysToReceivers: No receivers set");
        *ierr = 1;
        return;
    }
    fteik_solver3d_traceRaysToPoints(fk_receiver.nrec, fk_receiver.zrec, fk_receiver.xrec, fk_receiver.yrec, ierr);
    if (*ierr) { FK_ERR("fteik_solver3d_traceRaysToReceivers: Failed to compute rays"); *ierr = 1; }
}

void fteik_solver3d_traceRaysToPoints(int np, const double zp[], const double xp[],
                                      const double yp[], int *ierr)
{
    /* solver3D.F90:784-823: the gradient of the current field and the ray
     * end points; the reference's 3D tracer (rays.F90:442-447) is a stub and
     * its ray paths have no C accessor, so nothing more is observable. */
    *ierr = 0;
    if (!S3.have_times) {
        FK_ERR("fteik_solver3d_traceRaysToPoints: Travel time field not yet computed");
        *ierr = 1;
        return;
    }
    if (gradient("fteik_solver3d_traceRaysToPoints")) { *ierr = 1; return; }
    if (fk_check_ray_points(true, np, zp, xp, yp)) {
        FK_ERR("fteik_solver3d_traceRaysToPoints: Failed to set ray origins");
        *ierr = 1;
    }
}
