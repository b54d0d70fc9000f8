/*
 * fteik_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement of the reference fteik hot path (bakerb845/fteik), used as
 * the oracle the CUDA product is tested against and as the timed CPU
 * baseline.  Nothing in the product library links or calls this code: only
 * tests/, the smoke check in __graft_entry__.py and the cpu_baseline /
 * reference legs of bench.py load it (through ctypes).
 *
 * Precision follows the reference: the eikonal solvers are FP64, the locator
 * objective is FP32 with the reference's accumulation order.  The file is
 * compiled with -ffp-contract=off so no multiply-add is fused, as on the
 * reference's default x86-64 build.
 *
 * Conventions (as in the reference):
 *   - grids are column major, z fastest: node (iz,ix,iy) 1-based lives at
 *     (iy-1)*nz*nx + (ix-1)*nz + iz - 1 (0-based C offset);
 *   - cells likewise with (nz-1),(nx-1),(ny-1);
 *   - source/receiver indices are Fortran 1-based where noted.
 *
 * Parity status: the Fortran reference cannot be compiled in this
 * environment (no Fortran compiler), so the restatement is pinned through the
 * reference's own known-answer relations (analytic constant and linear
 * gradient media, the locator's known true index, the index round trip) and
 * through an independent literal transcription of the level-set sweep
 * (tests/test_oracle_levelset.py) rather than against bit-level golden output
 * of the reference binary.  The reference's own 2D check against a third-party
 * 2D solver (testing/test2d.F90:25-87, within 1e-10) needs Fortran and that
 * solver, neither of which is here, so it is not reproduced; the 2D solve is
 * held to the analytic linear-gradient time (first-order convergence) and to
 * the transcription instead.
 */
#ifndef FTEIK_ORACLE_H
#define FTEIK_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_HUGE 99999.0

/* ---------------------------------------------------------------- source -- */
/* source.F90:82-236 (fteik_source_initialize64f), one source.
 * Returns 0 on success, 1 if the source lies outside the model. */
int orc_source_snap(int is3d, int nz, int nx, int ny,
                    double z0, double x0, double y0,
                    double dz, double dx, double dy,
                    double zsrc, double xsrc, double ysrc,
                    int *zsi, int *xsi, int *ysi,
                    double *zsa, double *xsa, double *ysa);

/* ----------------------------------------------------------------- model -- */
/* model.F90:311-607.  order: 0 natural (ZXY/ZX), 1 XYZ/XZ, 2 ZYX.
 * keep_defects != 0 reproduces the reference's nodal-averaging defects
 * (model.F90:353 missing 1/8 for XYZ; model.F90:386-389 y-plane reuse).
 * Returns 0 on success. */
int orc_cell_velocity_to_slowness(int is3d, int nz, int nx, int ny, int order,
                                  const double *vel, double *slow);
int orc_nodal_velocity_to_slowness(int is3d, int nz, int nx, int ny, int order,
                                   int keep_defects,
                                   const double *vel, double *slow);

/* -------------------------------------------------------------- solver3d -- */
/* solver3D.F90:1156-1243 (solveSourceLSM) + autoCode.f90 sweeps +
 * localSolver.F90:384-959.  Runs the 8 initialisation sweeps and then
 * nsweep Gauss-Seidel passes of 8 sweeps.  If conv_tol >= 0 and max_pass > 0
 * the passes continue until the FP64 max |dt| of a whole pass is <= conv_tol
 * or max_pass passes ran (nsweep is then ignored).  nthreads <= 0 uses
 * OpenMP's default.  level_set != 0 runs the reference's schedule (levels,
 * 32-node chunks, a barrier per level, precomputed node lists); 0 runs the
 * equivalent natural-order loops (single thread).  tt has ngrd entries.
 * Returns 0 on success.  *npass (if not NULL) receives the passes run. */
int orc_solve3d(int nz, int nx, int ny, double dz, double dx, double dy,
                const double *slow,
                int zsi, int xsi, int ysi, double zsa, double xsa, double ysa,
                double eps, int nsweep, double conv_tol, int max_pass,
                int level_set, int nthreads, double *tt, int *npass);

/* One sweep (1..8) of the 3D solver on an existing field.  linit selects the
 * initialisation stencil and the source-limited update box. */
int orc_sweep3d(int sweep, int linit, int nz, int nx, int ny,
                double dz, double dx, double dy, const double *slow,
                int zsi, int xsi, int ysi, double zsa, double xsa, double ysa,
                double eps, double *tt);

/* Counts of node updates the reference evaluates: the init pass (8 masked
 * sweeps for the given source) and one full pass (8 sweeps). */
void orc_count_updates3d(int nz, int nx, int ny, int zsi, int xsi, int ysi,
                         int64_t *n_init, int64_t *n_pass);

/* -------------------------------------------------------------- solver2d -- */
/* solver2D.F90:782-978 (solveSourceLSM) and :1042-1280 (solveSourceFSM).
 * nsweep passes of 4 sweeps (the reference's convergence test never fires);
 * conv_tol / max_pass as for 3D.  Returns 0 on success. */
int orc_solve2d(int fsm, int nz, int nx, double dz, double dx,
                const double *slow, int zsi, int xsi, double zsa, double xsa,
                double eps, int nsweep, double conv_tol, int max_pass,
                double *tt, int *npass);

/* ------------------------------------------------------------- receivers -- */
/* receiver.F90:62-164 and :217-313. */
void orc_receiver_setup(int is3d, int nz, int nx, int ny,
                        double z0, double x0, double y0,
                        double dz, double dx, double dy,
                        int nrec, const double *z, const double *x,
                        const double *y, int *zri, int *xri, int *yri,
                        double *zdr, double *xdr, double *ydr, int *ierr);
void orc_receiver_interp(int is3d, int nz, int nx, int ny,
                         double dz, double dx, double dy, const double *tt,
                         int nrec, const int *zri, const int *xri,
                         const int *yri, const double *zdr, const double *xdr,
                         const double *ydr, double *ttr);

/* -------------------------------------------------------------- analytic -- */
/* analytic.F90:618-662 (constant) and :456-528,844-890 (linear gradient).
 * Output in the solver's natural order (z fastest). */
/* ------------------------------------------------------------- gradient -- */
/* solver3D.F90:1249-1321: g[3 m + 0, 1, 2] = dT/dx, dT/dy, dT/dz at node m
 * (natural order), forward differences, backward on each axis' last node. */
void orc_gradient3d(int nz, int nx, int ny, double dz, double dx, double dy,
                    const double *tt, double *g);
/* solver2D.F90:984-1032: backward differences, forward on each axis' first
 * node; gx[m], gz[m] with m = ix nz + iz. */
void orc_gradient2d(int nz, int nx, double dz, double dx, const double *tt,
                    double *gx, double *gz);

/* rays.F90:449-825: one 2D ray from (xr, zr) to the source grid point (xs,
 * zs), positions relative to the model origin; slow [(nx-1)(nz-1)], tt, gx,
 * gz [nx nz] z fastest; integrator 1 Euler, 2 midpoint, 3 RK4.  Outputs the
 * integration points, the (cell, length) pieces (1-based natural cell
 * index), the time along the steps (tn) and from the field (tne).  Returns
 * 0, 1 (did not reach the source in nx nz steps) or 2 (capacity). */
int orc_ray2d(int nz, int nx, double dz, double dx, const double *slow, const double *tt, const double *gx,
              const double *gz, double xs, double zs, int integrator, double xr, double zr, int maxpts,
              double *px, double *pz, int *npts, int maxseg, int *cells, double *lens, int *nseg, double *tn,
              double *tne);

void orc_analytic_constant(int nz, int nx, int ny, double z0, double x0,
                           double y0, double dz, double dx, double dy,
                           double vconst, double zs, double xs, double ys,
                           double *tt);
void orc_analytic_linear(int nz, int nx, int ny, double z0, double x0,
                         double y0, double dz, double dx, double dy,
                         double vtop, double vbottom,
                         double zs, double xs, double ys, double *tt);

/* ---------------------------------------------------------------- locate -- */
/* locate.F90:620-744 + :112-126 for one event, FP32 in the reference's
 * accumulation order (two passes over 512-point blocks), with the origin-time
 * work array reset per event (the documented maths; the reference keeps
 * accumulating it across events, locate.F90:641-690).
 * tables: ntf x ldgrd floats (row itf holds table itf).  obs/wts/skip are
 * per table (ntf entries), already reduced by tepoch as locate.F90:475-495
 * does.  Returns optIndx 1-based; t0Opt excludes tepoch. */
void orc_locate_l2(int ngrd, int ldgrd, int ntf, const float *tables,
                   const float *obs, const float *wts,
                   const unsigned char *skip, int nthreads,
                   int *optIndx, float *t0Opt, float *objOpt);
/* Per-grid-point FP32 objective and origin time for one event. */
void orc_locate_l2_field(int ngrd, int ldgrd, int ntf, const float *tables,
                         const float *obs, const float *wts,
                         const unsigned char *skip, int nthreads,
                         float *obj, float *t0);
/* The same misfit evaluated in FP64 at selected grid points (0-based). */
void orc_locate_l2_points64(int ngrd, int ldgrd, int ntf, const float *tables,
                            const float *obs, const float *wts,
                            const unsigned char *skip, int npts,
                            const int *pts, double *obj, double *t0);

/* Exhaustive FP64 search with the same misfit: picks and weights in FP64
 * (reduced picks, weight 0 = skipped), tables FP32.  Returns the 0-based
 * index of the first minimum and the FP64 t0 / misfit there. */
void orc_locate_l2_best64(int ngrd, int ldgrd, int ntf, const float *tables,
                          const double *obs, const double *wts, int nthreads,
                          int *idx, double *t0Opt, double *objOpt);

/* Exhaustive FP64 L1 search (no reference counterpart): t0 = median of the
 * residuals of the picks with positive weight (midpoint for an even count),
 * obj = w sum |r - t0| with w the common weight; first minimum. */
void orc_locate_l1_best64(int ngrd, int ldgrd, int ntf, const float *tables,
                          const double *obs, const double *wts, int nthreads,
                          int *idx, double *t0Opt, double *objOpt);

#ifdef __cplusplus
}
#endif
#endif
