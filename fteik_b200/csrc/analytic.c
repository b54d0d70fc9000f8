/*
 * analytic.c -- the reference's analytic module (analytic.F90): closed-form
 * travel times for a constant velocity and a linear vertical gradient,
 * evaluated on the device.  The module shares the model, source and receiver
 * state as in the reference (analytic.F90:100-160).
 */
#include "host_common.h"
#include "fteik_b200.h"

#include <stdlib.h>
#include <string.h>

static struct {
    bool init, have;
    int nz, nx, ny, ngrd, verbose;
    double z0, x0, y0, dz, dx, dy;
    double vconst, vtop, vbottom;
    double *tt;        /* device, natural order */
} SA = {.vconst = 5.0e3, .vtop = 5.0e3, .vbottom = 5.0e3};

void fteik_analytic_setVerbosity(int verbose) { SA.verbose = verbose; }

void fteik_analytic_free(void)
{
    fk_dfree(SA.tt);
    memset(&SA, 0, sizeof(SA));
    SA.vconst = SA.vtop = SA.vbottom = 5.0e3; /* analytic.F90:224-226 */
}

void fteik_analytic_initialize64f(int nz, int nx, int ny, double z0, double x0, double y0,
                                  double dz, double dx, double dy, int verbose, int *ierr)
{
    /* analytic.F90:100-155 */
    *ierr = 0;
    fteik_analytic_free();
    SA.verbose = verbose;
    if (nx < 1 || ny < 1 || nz < 1) {
        FK_ERR("fteik_analytic_initialize64f: Invalid number of grid points %d %d %d", nx, ny, nz);
        *ierr = 1;
        return;
    }
    if (dx <= 0.0 || dy <= 0.0 || dz <= 0.0) {
        FK_ERR("fteik_analytic_initialize64f: Grid spacing must be positive");
        *ierr = 1;
        return;
    }
    SA.nz = nz; SA.nx = nx; SA.ny = ny; SA.ngrd = nz * nx * ny;
    SA.dz = dz; SA.dx = dx; SA.dy = dy;
    /* the shared model gets a zero origin (analytic.F90:136-141); the
     * analytic fields use the caller's origin (setOrigin, :282-289) */
    fteik_model_initializeGeometry(ny >= 2, nz, nx, ny, 0.0, 0.0, 0.0, dz, dx, dy, ierr);
    SA.z0 = z0; SA.x0 = x0; SA.y0 = y0;
    if (fk_dev_ready("fteik_analytic_initialize64f")) { *ierr = 1; return; }
    SA.tt = (double *)fk_dalloc(sizeof(double) * (size_t)SA.ngrd, "fteik_analytic");
    if (!SA.tt) { *ierr = 1; return; }
    SA.init = true;
}

void fteik_analytic_setSources64f(int nsrc, const double zsrc[], const double xsrc[],
                                  const double ysrc[], int *ierr)
{
    fteik_source_initialize64f(nsrc, zsrc, xsrc, ysrc, SA.verbose, ierr);
    if (*ierr) FK_ERR("fteik_analytic_setSources64f: Failed to set source");
}

void fteik_analytic_setReceivers64f(int nrec, const double zrec[], const double xrec[],
                                    const double yrec[], int *ierr)
{
    *ierr = fk_receiver_setup(nrec, zrec, xrec, yrec, SA.verbose);
}

void fteik_analytic_setConstantVelocity64f(double vconst, int *ierr)
{
    *ierr = 0;
    if (vconst <= 0.0) {
        FK_ERR("fteik_analytic_setConstantVelocity64f: Velocity must be positive %g", vconst);
        *ierr = 1;
        return;
    }
    SA.vconst = vconst;
}

void fteik_analytic_setLinearVelocityGradient64f(double v0, double v1, int *ierr)
{
    /* analytic.F90:289-318 */
    *ierr = 0;
    SA.vtop = SA.vconst;
    SA.vbottom = SA.vconst;
    if (v0 <= 0.0) { FK_ERR("fteik_analytic_setLinearVelocityGradient64f: v0 must be positive"); *ierr = 1; return; }
    if (v1 <= 0.0) { FK_ERR("fteik_analytic_setLinearVelocityGradient64f: v1 must be positive"); *ierr = 1; return; }
    if (SA.nz < 2) { FK_ERR("fteik_analytic_setLinearVelocityGradient64f: 2 points required in z"); *ierr = 1; return; }
    SA.vtop = v0;
    SA.vbottom = v1;
}

static void solve_src(int kind, int isrc, int *ierr, const char *who)
{
    *ierr = 0;
    if (!SA.init) { FK_ERR("%s: Not initialized", who); *ierr = 1; return; }
    if (!fk_source.have || isrc < 1 || isrc > fk_source.nsrc) {
        FK_ERR("%s: Source = %d must be in range [1,%d]", who, isrc, fk_source.have ? fk_source.nsrc : 0);
        *ierr = 1;
        return;
    }
    double v0 = kind == 0 ? SA.vconst : SA.vtop, v1 = kind == 0 ? SA.vconst : SA.vbottom;
    int e = fk_analytic_field(kind, SA.nz, SA.nx, SA.ny, SA.z0, SA.x0, SA.y0, SA.dz, SA.dx, SA.dy,
                              v0, v1, fk_source.zs_true[isrc - 1], fk_source.xs_true[isrc - 1],
                              fk_source.ys_true[isrc - 1], SA.tt, fk_stream());
    if (!e) e = (int)cudaStreamSynchronize(fk_stream());
    *ierr = fk_check(e, who);
    SA.have = *ierr == 0;
}

void fteik_analytic_solveSourceConstantVelocity64f(int isrc, int *ierr)
{
    solve_src(0, isrc, ierr, "fteik_analytic_solveSourceConstantVelocity64f");
}

void fteik_analytic_solveSourceLinearVelocityGradient64f(int isrc, int *ierr)
{
    solve_src(1, isrc, ierr, "fteik_analytic_solveLinearVelocityGradient64f");
}

void fteik_analytic_getTravelTimeField64f(int ngrd, int order, double tt[], int *ierr)
{
    /* analytic.F90:686-735 */
    *ierr = 0;
    if (!SA.init || !SA.have) { FK_ERR("fteik_analytic_getTravelTimeField64f: ttimes not initialized"); *ierr = 1; return; }
    if (ngrd < SA.ngrd) { FK_ERR("fteik_analytic_getTravelTimeField64f: Insufficient space"); *ierr = 1; return; }
    double *buf = (double *)fk_dalloc(sizeof(double) * (size_t)SA.ngrd, "fteik_analytic");
    if (!buf) { *ierr = 1; return; }
    if (order != FTEIK_XYZ_ORDERING && order != FTEIK_ZYX_ORDERING) order = FTEIK_NATURAL_ORDERING;
    int e = fk_field_to_f64(8, 1, SA.nz, SA.nx, SA.ny, SA.nz, SA.tt, order, buf, fk_stream());
    if (!e) e = (int)cudaMemcpyAsync(tt, buf, sizeof(double) * (size_t)SA.ngrd,
                                    cudaMemcpyDeviceToHost, fk_stream());
    if (!e) e = (int)cudaStreamSynchronize(fk_stream());
    fk_dfree(buf);
    for (int i = SA.ngrd; i < ngrd; i++) tt[i] = 0.0;
    *ierr = fk_check(e, "fteik_analytic_getTravelTimeField64f");
}

static void rec_times(int kind, int ldr, double ttr[], int *ierr, const char *who)
{
    /* analytic.F90:747-842: exact times at every receiver for every source */
    *ierr = 0;
    if (!SA.init) { FK_ERR("%s: Not initialized", who); *ierr = 1; return; }
    if (!fk_source.have || fk_source.nsrc < 1) { FK_ERR("%s: No sources", who); *ierr = 1; return; }
    const int nrec = fk_receiver.have ? fk_receiver.nrec : 0;
    const int nsrc = fk_source.nsrc;
    if (ldr < nrec) { FK_ERR("%s: ldr < nrec %d %d", who, ldr, nrec); *ierr = 1; return; }
    if (nrec < 1) return;
    if (ldr > nrec) memset(ttr, 0, sizeof(double) * (size_t)ldr * nsrc);
    size_t npt = 3 * (size_t)nrec + 3 * (size_t)nsrc;
    double *d = (double *)fk_dalloc(sizeof(double) * (npt + (size_t)ldr * nsrc), who);
    if (!d) { *ierr = 1; return; }
    double *h = (double *)malloc(sizeof(double) * npt);
    memcpy(h, fk_receiver.zrec, sizeof(double) * nrec);
    memcpy(h + nrec, fk_receiver.xrec, sizeof(double) * nrec);
    memcpy(h + 2 * nrec, fk_receiver.yrec, sizeof(double) * nrec);
    memcpy(h + 3 * nrec, fk_source.zs_true, sizeof(double) * nsrc);
    memcpy(h + 3 * nrec + nsrc, fk_source.xs_true, sizeof(double) * nsrc);
    memcpy(h + 3 * nrec + 2 * nsrc, fk_source.ys_true, sizeof(double) * nsrc);
    cudaStream_t s = fk_stream();
    double *out = d + npt;
    int e = (int)cudaMemcpyAsync(d, h, sizeof(double) * npt, cudaMemcpyHostToDevice, s);
    if (!e) e = (int)cudaMemsetAsync(out, 0, sizeof(double) * (size_t)ldr * nsrc, s);
    double v0 = kind == 0 ? SA.vconst : SA.vtop, v1 = kind == 0 ? SA.vconst : SA.vbottom;
    if (!e) e = fk_analytic_points(kind, SA.nz, SA.z0, SA.dz, v0, v1, nrec, d, d + nrec, d + 2 * nrec,
                                  nsrc, d + 3 * nrec, d + 3 * nrec + nsrc, d + 3 * nrec + 2 * nsrc,
                                  ldr, out, s);
    if (!e) e = (int)cudaMemcpyAsync(ttr, out, sizeof(double) * (size_t)ldr * nsrc,
                                    cudaMemcpyDeviceToHost, s);
    if (!e) e = (int)cudaStreamSynchronize(s);
    free(h);
    fk_dfree(d);
    *ierr = fk_check(e, who);
}

void fteik_analytic_getTravelTimesConstantVel64f(int ldr, double ttr[], int *ierr)
{
    rec_times(0, ldr, ttr, ierr, "fteik_analytic_getTravelTimesConstantVel64f");
}

void fteik_analytic_getTravelTimesGradientVel64f(int ldr, double ttr[], int *ierr)
{
    rec_times(1, ldr, ttr, ierr, "fteik_analytic_getTravelTimesGradientVel64f");
}
