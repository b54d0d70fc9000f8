/*
 * fteik_b200.h -- C ABI of libfteik_shared.so, the B200 implementation of
 * fteik's eikonal solver and grid-search locator.
 *
 * Part 1 declares the reference's own entry points with the reference's
 * exact symbol names, argument passing (scalars by value, arrays and outputs
 * by pointer, bool = C _Bool) and conventions (1-based source, event and
 * table numbers; ierr = 0 on success; travel times in FP64 with 99999 for
 * unreached nodes).  Each cites the Fortran BIND(C) routine it replaces
 * (paths relative to the reference repository).  Where the reference's own
 * header include/fteik/fteik_fortran.h disagrees with its Fortran, the
 * Fortran is followed.
 *
 * Part 2 declares additions with no reference counterpart (prefix
 * fteik_b200_): a batched multi-source, multi-grid 3D solve, device-resident
 * hand-off and batched location.
 *
 * The library owns one CUDA stream and uses the current CUDA device (device
 * 0 unless the caller selected another); callers need no CUDA context.  It
 * has no CPU fallback: without a usable CUDA device every compute entry
 * point fails with ierr = 1 and a message on stderr.  Like the reference,
 * the state is a process-wide singleton and the API is not re-entrant.
 */
#ifndef FTEIK_B200_H
#define FTEIK_B200_H

#include <stdbool.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Orderings, constants.F90:29-39 */
enum fteikOrder_enum {
    FTEIK_NATURAL_ORDERING = 0,
    FTEIK_ZXY_ORDERING = 0,
    FTEIK_ZX_ORDERING = 0,
    FTEIK_XYZ_ORDERING = 1,
    FTEIK_XZ_ORDERING = 1,
    FTEIK_ZYX_ORDERING = 2
};

/* =====================  Part 1: reference entry points  ================== */

/* ---- model: model.F90 ---- */
/* model.F90:88-129 */
void fteik_model_initializeGeometry(bool lis3d, int nz, int nx, int ny,
                                    double z0, double x0, double y0,
                                    double dz, double dx, double dy, int *ierr);
/* model.F90:181-216 */
void fteik_model_setGridSize(bool lis3d, int nz, int nx, int ny, int *ierr);
/* model.F90:134-172 */
void fteik_model_setGridSpacing(bool lis3d, double dz, double dx, double dy,
                                int *ierr);
/* model.F90:225-240 / :245-258 */
void fteik_model_setOrigin3D(double z0, double x0, double y0);
void fteik_model_setOrigin2D(double z0, double x0);
/* model.F90:264-296 */
void fteik_model_getGridSize(int *nz, int *nx, int *ny, int *ngrd, int *ncell,
                             int *ierr);
/* model.F90:574-607 (cells in natural order) */
void fteik_model_setVelocityModel64f(int nv, const double vel[], int *ierr);
/* model.F90:719-754: FP32 cell velocities, widened to FP64 before 1/v */
void fteik_model_setVelocityModel32f(int nv, const float vel4[], int *ierr);
/* model.F90:651-688: nwork = -1 queries nv = ncell; else vel[0..ncell) = 1/slowness */
void fteik_model_getVelocityModel64f(int nwork, int *nv, double vel[], int *ierr);
/* model.F90:692-706 */
void fteik_model_isModel3D(bool *lis3d, int *ierr);
/* model.F90:311-449 (order 0 natural, 1 XYZ, 2 ZYX) */
void fteik_model_setNodalVelocityModel64f(int ng, int order,
                                          const double vel[], int *ierr);
/* model.F90:505-607 */
void fteik_model_setCellVelocityModel64f(int nc, int order,
                                         const double vel[], int *ierr);
/* model.F90:760-780 (1-based) and fwrapper.c:8-14 (0-based) */
int fteik_model_grid2indexF(int i, int j, int k, int nz, int nzx);
int fteik_model_grid2index(int iz, int ix, int iy, int nz, int nzx);
/* model.F90:790-810 */
void fteik_model_index2gridF(int igrd, int *i, int *j, int *k, int *ierr);
/* model.F90:827-836 */
int fteik_model_velGrid2indexF(int i, int j, int k, int nzm1, int nzm1_nxm1);
/* model.F90:612-640 */
void fteik_model_free(void);

/* ---- source: source.F90 ---- */
/* source.F90:82-236 */
void fteik_source_initialize64f(int nsrc, const double zsrc[],
                                const double xsrc[], const double ysrc[],
                                int verbose, int *ierr);
/* source.F90:290-330 */
void fteik_source_getSolverInfo64fF(int isrc, int *zsi, int *xsi, int *ysi,
                                    double *zsa, double *xsa, double *ysa,
                                    double *szero, double *szero2, int *ierr);
/* source.F90:341-370 / :381-410 / :429-464 */
void fteik_source_getSourceIndices64fF(int isrc, double *zsa, double *xsa,
                                       double *ysa, int *ierr);
void fteik_source_getSourceIndices32iF(int isrc, int *zsi, int *xsi, int *ysi,
                                       int *ierr);
void fteik_source_getSzero64fF(int isrc, double *szero, double *szero2,
                               int *ierr);
void fteik_source_getNumberOfSources(int *nsrc, int *ierr);
void fteik_source_free(void);
/* source.F90:243-249 */
void fteik_source_setVerbosity(int verbose);

/* ---- receivers: receiver.F90 ---- */
/* receiver.F90:62-164 */
void fteik_receiver_initialize64f(int nrec, const double z[], const double x[],
                                  const double y[], int verbose, int *ierr);
/* receiver.F90:217-313: interpolates a caller-supplied FP64 field */
void fteik_receiver_getTravelTimes64f(int nrec, int ngrd, const double ttimes[],
                                      double ttr[], int *ierr);
void fteik_receiver_getNumberOfReceivers(int *nrec, int *ierr);
void fteik_receiver_free(void);
/* receiver.F90:171-177 */
void fteik_receiver_setVerbosity(int verbose);

/* ---- 3D solver: solver3D.F90 ---- */
/* solver3D.F90:126-184 */
void fteik_solver3d_initialize(int nz, int nx, int ny, double z0, double x0,
                               double y0, double dz, double dx, double dy,
                               int nsweep, double eps, double convTol,
                               int verbose, int *ierr);
/* solver3D.F90:575-610 */
void fteik_solver3d_free(void);
/* solver3D.F90:191-196 / :206-211 */
void fteik_solver3d_setVerbosity(int verbose);
void fteik_solver3d_setConvergenceTolerance(double convTol);
/* solver3D.F90:683-698 / :640-673 */
void fteik_solver3d_setNumberOfSweeps(int nsweep, int *ierr);
void fteik_solver3d_setSphereToCartEpsilon(double eps, int *ierr);
/* solver3D.F90:1138-1148 / :1115-1125 / :1083-1093 */
void fteik_solver3d_setVelocityModel64f(int ncell, const double vel[], int *ierr);
void fteik_solver3d_setCellVelocityModel64f(int nc, int order,
                                            const double vel[], int *ierr);
void fteik_solver3d_setNodalVelocityModel64f(int ng, int order,
                                             const double vel[], int *ierr);
/* solver3D.F90:717-727 / :737-748 */
void fteik_solver3d_setSources64f(int nsrc, const double zsrc[],
                                  const double xsrc[], const double ysrc[],
                                  int *ierr);
void fteik_solver3d_getNumberOfSources(int *nsrc, int *ierr);
/* solver3D.F90:1045-1062 / :1024-1032 */
void fteik_solver3d_setReceivers64f(int nrec, const double zrec[],
                                    const double xrec[], const double yrec[],
                                    int *ierr);
void fteik_solver3d_getNumberOfReceivers(int *nrec, int *ierr);
/* solver3D.F90:1156-1243 */
void fteik_solver3d_solveSourceLSM(int isrc, int *ierr);
/* solver3D.F90:844-897 */
void fteik_solver3d_getTravelTimeField64f(int ngrd, int order, double tt[],
                                          int *ierr);
/* solver3D.F90:915-980 */
void fteik_solver3d_getTravelTimeFieldCell64f(int ncell, int order,
                                              double tt[], int *ierr);
/* solver3D.F90:990-1016 */
void fteik_solver3d_getTravelTimes64f(int nrec, double ttr[], int *ierr);
/* solver3D.F90:756-823: as the reference, computes the travel-time gradient
 * of the current field and checks the ray end points (ierr = 1 with no
 * solved field, no points or a point outside the model); the reference's
 * 3D tracer is a stub (rays.F90:442-447) and its rays have no C accessor. */
void fteik_solver3d_traceRaysToReceivers(int *ierr);
void fteik_solver3d_traceRaysToPoints(int np, const double zp[],
                                      const double xp[], const double yp[],
                                      int *ierr);
/* The travel-time gradient of the current field, solver3D.F90:1249-1321
 * (forward differences, backward on each axis' last node), in the layout of
 * the reference's module array tgrad, which C callers cannot reach there:
 * grad[3 m + 0, 1, 2] = dT/dx, dT/dy, dT/dz at node m (natural order, z
 * fastest); ngrd = nz nx ny. */
void fteik_b200_solver3d_getTravelTimeGradient64f(int ngrd, double grad[], int *ierr);

/* ---- 2D solver: solver2D.F90 ---- */
/* solver2D.F90:124-198 */
void fteik_solver2d_initialize(int nz, int nx, double z0, double x0, double dz,
                               double dx, int nsweep, double eps,
                               double convTol, int verbose, int *ierr);
void fteik_solver2d_free(void);
void fteik_solver2d_setVerbosity(int verbose);
void fteik_solver2d_setConvergenceTolerance(double convTol);
void fteik_solver2d_setNumberOfSweeps(int nsweep, int *ierr);
void fteik_solver2d_setSphereToCartEpsilon(double eps, int *ierr);
void fteik_solver2d_setVelocityModel64f(int ncell, const double vel[], int *ierr);
void fteik_solver2d_setCellVelocityModel64f(int nc, int order,
                                            const double vel[], int *ierr);
void fteik_solver2d_setNodalVelocityModel64f(int ng, int order,
                                             const double vel[], int *ierr);
void fteik_solver2d_setSources64f(int nsrc, const double zsrc[],
                                  const double xsrc[], int *ierr);
void fteik_solver2d_setReceivers64f(int nrec, const double zrec[],
                                    const double xrec[], int *ierr);
void fteik_solver2d_getNumberOfReceivers(int *nrec, int *ierr);
/* solver2D.F90:782-978 */
void fteik_solver2d_solveSourceLSM(int isrc, int *ierr);
/* solver2D.F90:1042-1280 */
void fteik_solver2d_solveSourceFSM(int isrc, int *ierr);
/* solver2D.F90:740-773: every source */
void fteik_solver2d_solveLSM(int *ierr);
/* solver2D.F90:1295-1340 / :1350-1400 */
void fteik_solver2d_getTravelTimeField64f(int ngrd, int order, double tt[],
                                          int *ierr);
void fteik_solver2d_getTravelTimeFieldCell64f(int ncell, int order,
                                              double tt[], int *ierr);
/* solver2D.F90:1410-1447: ttr[ldr*nsrc], receiver times of every source */
void fteik_solver2d_getTravelTimes64f(int ldr, double ttr[], int *ierr);
/* solver2D.F90:283-350: the travel-time gradient of the current field and a
 * check of the ray end points, as the reference (its 2D rays have no C
 * accessor) */
void fteik_solver2d_traceRaysToReceivers(int *ierr);
void fteik_solver2d_traceRaysToPoints(int np, const double xp[],
                                      const double zp[], int *ierr);
/* The gradient of the current 2D field, solver2D.F90:984-1032 (backward
 * differences, forward on each axis' first node): the reference's module
 * arrays tgradx, tgradz (read by testing/test2d.F90 through USE), which C
 * callers cannot reach there; node m = ix nz + iz, ngrd = nz nx. */
void fteik_b200_solver2d_getTravelTimeGradient64f(int ngrd, double gradx[], double gradz[],
                                                  int *ierr);

/* ---- analytic solutions: analytic.F90 ---- */
void fteik_analytic_initialize64f(int nz, int nx, int ny, double z0, double x0,
                                  double y0, double dz, double dx, double dy,
                                  int verbose, int *ierr);
void fteik_analytic_setSources64f(int nsrc, const double zsrc[],
                                  const double xsrc[], const double ysrc[],
                                  int *ierr);
void fteik_analytic_setReceivers64f(int nrec, const double zrec[],
                                    const double xrec[], const double yrec[],
                                    int *ierr);
void fteik_analytic_setConstantVelocity64f(double vconst, int *ierr);
void fteik_analytic_setLinearVelocityGradient64f(double v0, double v1,
                                                 int *ierr);
void fteik_analytic_solveSourceConstantVelocity64f(int isrc, int *ierr);
void fteik_analytic_solveSourceLinearVelocityGradient64f(int isrc, int *ierr);
void fteik_analytic_getTravelTimeField64f(int ngrd, int order, double tt[],
                                          int *ierr);
/* analytic.F90:747-842: ttr[ldr*nsrc], exact times at every receiver */
void fteik_analytic_getTravelTimesConstantVel64f(int ldr, double ttr[],
                                                 int *ierr);
void fteik_analytic_getTravelTimesGradientVel64f(int ldr, double ttr[],
                                                 int *ierr);
void fteik_analytic_free(void);
/* analytic.F90:194-200 */
void fteik_analytic_setVerbosity(int verbose);

/* ---- locator: locate.F90 ---- */
/* locate.F90:142-223 */
void locate_initialize(int nEvents, int ntf, int ngrd, int *ierr);
/* locate.F90:233-270 */
void locate_finalize(void);
/* locate.F90:287-343 (itf 1-based) */
void locate_setTravelTimeField64f(int ngrd, int itf, const double tt[],
                                  int *ierr);
/* locate.F90:361-396 (the Fortran takes float[]) */
void locate_setTravelTimeField32f(int ngrd, int itf, const float tt[],
                                  int *ierr);
/* locate.F90:431-497 (evnmbr and obs2tf 1-based) */
void locate_setObservation64f(int evnmbr, int nttimes, bool lhaveOT,
                              double t0, const int obs2tf[],
                              const double pickTimes[], const double wts[],
                              int *ierr);
/* fwrapper.c:42-55 (0-based event and table numbers) */
void locate_setObservation64fC(int evnmbr, int nttimes, bool lhaveOT,
                               double t0, const int obs2tf[],
                               const double pickTimes[], const double wts[],
                               int *ierr);
/* locate.F90:112-126 (optIndx 1-based grid index) */
void locate_locateEvent(int evnmbr, int *optIndx, double *t0Opt,
                        double *objOpt);
/* locate.F90:511-531 / :541-560 / :573-592 */
void locate_setNumberOfEvents(int nEvents, int *ierr);
void locate_setNumberOfTravelTimeFields(int ntf, int *ierr);
void locate_setNumberOfGridPointsF(int ngrd, int *ierr);

/* ---- archive (h5io.F90:104-420) without HDF5: "name.h5" is written as the
 * directory "name.h5.d/" with the reference's groups, each dataset a NumPy
 * .npy file in the reference's layout (travel times FP32 x fastest, 2D
 * flipped in z; velocities INT16 per cell; level schedules INT16 per node).
 * Returns 0, -1 on misuse (as the reference), 1 on an I/O failure. ---- */
int fteik_h5io_initializeF(const char *fileName);
int fteik_h5io_finalizeF(void);
int fteik_h5io_writeLevelSchedulesF(void);
int fteik_h5io_writeVelocityModelF(const char *velName);
int fteik_h5io_writeTravelTimesF(const char *ttName);

/* ---- ray paths: rays.F90 ---- */
/* rays.F90:215-229: integrator of the ray-path equation for the next
 * traceRaysTo* call: 1 Euler (default), 2 midpoint, 3 the reference's RK4;
 * an invalid value sets Euler and ierr = 1.  Initialising or freeing a
 * solver resets it to Euler, as in the reference. */
void fteik_rays_setODEIntegrator(int integrator, int *ierr);

/* =====================  Part 2: additions (fteik_b200_)  ================= */

/* Library version string and the CUDA device in use (-1 if none). */
const char *fteik_b200_version(void);
int fteik_b200_device(void);
/* The library's CUDA stream (a cudaStream_t), for callers that time or
 * order their own work against the library's; NULL without a device. */
void *fteik_b200_stream(void);

/* Poll limit of the bounded device-side waits of the 3D sweeps (a slab
 * waiting on its upwind slab or on its neighbours' previous sweep).  A wait
 * that runs out of polls stops its kernel, which returns normally with an
 * error word set; the solve reports it as ierr = 1 and the library stays
 * usable.  polls < 0 restores the default (2^22 polls of at most 1 us,
 * seconds of waiting).  Takes effect at the next solve (a captured batch
 * graph is rebuilt).  No counterpart in the reference, whose OpenMP
 * barriers wait without a limit. */
void fteik_b200_setSpinLimit(long long polls, int *ierr);
void fteik_b200_getSpinLimit(long long *polls);

/* Launch configuration of the persistent 3D sweep kernels, for the
 * single-source solver and the batch.  Each knob takes a value or -1 for
 * the library's choice (the default; the batch then picks by timing, see
 * fteik_b200_batch3d_getSlabConfig):
 *   staged      FP32 passes: 1 = each lane's node values, upwind-row values
 *               and slowness move in 16-byte groups through shared memory
 *               (cp.async), 0 = one 4-byte load per value and step;
 *   pairs       passes: 1 = two sources of one grid share each thread, 0 = one;
 *   progress    passes: slabs publish progress every 8 or 32 steps, or 0 =
 *               8 when a sweep has fewer than 4 slab tasks per resident
 *               block, else 32;
 *   blocksPerSM resident blocks per SM, 1..4, or 0 = as many as fit.
 * Results are the same bits whichever configuration runs.  Takes effect at
 * the next solve (a captured batch graph is rebuilt).  No counterpart in the
 * reference. */
void fteik_b200_setSlabConfig(int staged, int pairs, int progress, int blocksPerSM, int *ierr);
void fteik_b200_getSlabConfig(int *staged, int *pairs, int *progress, int *blocksPerSM);

/* Precision of fteik_solver3d_solveSourceLSM: 4 (default; FP32 fields with
 * FP64 source corners, near-source stencil and residual) or 8 (FP64 fields,
 * the reference's precision).  Applies from the next solve. */
void fteik_b200_solver3d_setPrecision(int precision, int *ierr);
/* FP64 max |dt| of the last Gauss-Seidel pass and passes run, for the last
 * fteik_solver3d_solveSourceLSM. */
void fteik_b200_solver3d_getSolveInfo(double *residual, int *npass, int *ierr);

/* Batched 3D solve: ngrid grids of any size, each with its own sources, all
 * solved by one kernel launch (one CTA per grid x source), replayed from a
 * CUDA graph.  precision 4 = FP32 fields (near-source stencil, source
 * corners and residual in FP64), 8 = FP64 fields.  nsweep / convTol /
 * maxPass as for fteik_solver3d_initialize, except that convTol >= 0 with
 * maxPass > 0 iterates every source to convergence.  Grid and source
 * numbers are 1-based. */
void fteik_b200_batch3d_initialize(int ngrid, const int nz[], const int nx[],
                                   const int ny[], const double dz[],
                                   const double dx[], const double dy[],
                                   int nsweep, double eps, double convTol,
                                   int maxPass, int precision, int *ierr);
/* Cell velocities of grid igrid in the natural (z fastest) order. */
void fteik_b200_batch3d_setVelocityModel64f(int igrid, int ncell,
                                            const double vel[], int *ierr);
/* Sources of grid igrid, coordinates relative to the grid origin (0,0,0). */
void fteik_b200_batch3d_setSources64f(int igrid, int nsrc, const double zsrc[],
                                      const double xsrc[], const double ysrc[],
                                      int *ierr);
void fteik_b200_batch3d_setReceivers64f(int igrid, int nrec,
                                        const double zrec[], const double xrec[],
                                        const double yrec[], int *ierr);
/* Solve every (grid, source) pair. */
void fteik_b200_batch3d_solve(int *ierr);
/* Replay the last solve's CUDA graph on the library stream without waiting;
 * returns a cudaError_t (non-zero also when no solve was captured yet). */
int fteik_b200_batch3d_solveAsync(void);
/* Field of one source, FP64 in a reference ordering. */
void fteik_b200_batch3d_getTravelTimeField64f(int igrid, int isrc, int ngrd,
                                              int order, double tt[], int *ierr);
/* Fields of every source of a grid as FP32, natural order, [nsrc][ngrd]. */
void fteik_b200_batch3d_getTravelTimeFields32f(int igrid, long long nval,
                                               float tt[], int *ierr);
/* The same, returning once the copy is queued: the tables are unpacked on
 * the library stream and copied to tt on a copy stream, so the copy runs
 * while the caller uploads the next models and solves again.  tt should be
 * pinned host memory and must stay untouched until
 * fteik_b200_batch3d_waitDownloads returns. */
void fteik_b200_batch3d_getTravelTimeFields32fAsync(int igrid, long long nval,
                                                    float tt[], int *ierr);
/* Wait for every queued table download. */
void fteik_b200_batch3d_waitDownloads(int *ierr);
/* Receiver times of every source of a grid: ttr[isrc*nrec + irec]. */
void fteik_b200_batch3d_getTravelTimes64f(int igrid, int nval, double ttr[],
                                          int *ierr);
/* The launch configuration the batch runs (see fteik_b200_setSlabConfig):
 * knobs left at -1 are chosen by timing the candidates on the first solve of
 * a new work list (grid shapes, sources per grid, precision, passes); the
 * initialisation kernel takes its own blocks per SM and source pairing
 * (initPairs: two sources per thread over the union of their boxes).  The
 * choice is remembered in the process and, when the environment variable
 * FTEIK_B200_TUNE_CACHE names a file, appended to that file for later
 * processes.  initMs / passMs: the chosen kernels' times during the search
 * (0 when nothing was searched), tuneRuns the candidate solves it ran (0 on
 * a cache hit).  No counterpart in the reference. */
void fteik_b200_batch3d_getSlabConfig(int *staged, int *pairs, int *progress, int *blocksPerSM,
                                      int *initBlocksPerSM, int *initPairs, float *initMs, float *passMs,
                                      int *tuneRuns, int *ierr);
/* Run one solve outside its CUDA graph with events around the
 * initialisation kernel and the Gauss-Seidel kernel and return their device
 * times (ms); the fields end as after fteik_b200_batch3d_solve. */
void fteik_b200_batch3d_timeSolve(float *init_ms, float *pass_ms, int *ierr);
/* Residual (FP64 max |dt| of the last pass) and passes run. */
void fteik_b200_batch3d_getSolveInfo(int igrid, int isrc, double *residual,
                                     int *npass, int *ierr);
/* Copy the FP32 tables of every source of grid igrid into the locator's
 * device table store (tables itf0 .. itf0+nsrc-1, 1-based) without leaving
 * the device.  The locator must have been initialised with ngrd equal to
 * that grid's node count. */
void fteik_b200_batch3d_exportToLocator(int igrid, int itf0, int *ierr);
void fteik_b200_batch3d_finalize(void);

/* Locate events ev[0..n-1] (1-based) in one batch with the reference's FP32
 * objective (bit-identical optimum); outputs as locate_locateEvent. */
void fteik_b200_locate_locateEvents(int n, const int ev[], int optIndx[],
                                    double t0Opt[], double objOpt[], int *ierr);

/* Search method of locate_locateEvent and fteik_b200_locate_locateEvents
 * (the reference has one method, locate.F90:620-744):
 *   0  exact FP32 search, the reference's arithmetic and optimum (default);
 *   1  tensor-core search: the L2 misfit ranked by a BF16 hi+lo contraction
 *      with FP32 accumulation, the best candidates re-scored with the
 *      reference's formula in FP64 (t0Opt and objOpt are those FP64 values).
 *      Events whose picks do not cover every table with one common weight
 *      fall back to method 0. */
void fteik_b200_locate_setMethod(int method, int *ierr);
/* BF16 products of the tensor-core ranking (methods 1 and 2): 2 (default)
 * = hi*hi + hi*lo, the event operand rounded to BF16 once (its rounding
 * error varies smoothly over the grid, and the FP64 re-score of the best
 * candidates decides); 3 = hi*hi + hi*lo + lo*hi of both split operands. */
void fteik_b200_locate_setRankingProducts(int nprod, int *ierr);
void fteik_b200_locate_getRankingProducts(int *nprod);
/* Misfit norm of every method (no counterpart in the reference, which has
 * L2 only): 2 (default) = locate.F90:620-744; 1 = L1 with origin-time
 * removal, obj(g) = w sum_i |o_i - T_i(g) - t0(g)|, t0(g) = the median of the
 * residuals (midpoint of the two middle values for an even count), for
 * events whose positive pick weights are all equal to w; searched
 * exhaustively on the GPU, the optimum's t0 and misfit in FP64. */
void fteik_b200_locate_setNorm(int norm, int *ierr);
/* Candidates per event re-scored in FP64 by method 1 (default 8). */
void fteik_b200_locate_setRescoreCandidates(int ncand, int *ierr);
/* Diagnostic for method 1: enable = 1 records, at the next search, the first
 * two accumulator tiles (events 1..256 x grid points 1..128, FP32, row-major
 * by event); enable = 0 copies them to out (32768 floats, may be NULL). */
void fteik_b200_locate_debugAccumulators(int enable, float *out, int *ierr);

/* ---- surrogate-pruned search (method 2; no counterpart in the reference) --
 * A small network (fteik_b200_mlp_*) learns tau = T v_ref / distance from
 * the locator's own tables.  The grid is cut into blocks of bz x bx x by
 * fine nodes (aligned to the grid: block c holds the nodes f with
 * floor(f / b) = c on each axis); the network's travel times at the block
 * centres are ranked by the tensor-core search, the best blocks are
 * re-scored node by node on the exact tables in FP64, and while the best
 * node lies on a face of the examined set the neighbouring block is examined
 * too; events that exceed 32 blocks are searched exhaustively (method 1).
 * Grid geometry: the tables' nodes are (iz, ix, iy) on a z-fastest grid with
 * origin 0; station positions in the same frame, one per table. */
void fteik_b200_locate_setGeometry(int nz, int nx, int ny, double dz, double dx, double dy,
                                   int ntf, const double zsta[], const double xsta[],
                                   const double ysta[], int *ierr);
void fteik_b200_locate_trainSurrogate(long long nsamples, int steps, int batch, double lr,
                                      double vref, unsigned long long seed, double *loss,
                                      int *ierr);
void fteik_b200_locate_buildSurrogate(int bz, int bx, int by, int *ierr);
/* coarse runs of 32 examined (1-4, default 4) and blocks kept (1-32,
 * default 8: 8 x 64 = 512 fine nodes with 4 x 4 x 4 blocks) */
void fteik_b200_locate_setPruning(int ncoarse_runs, int ncoarse_nodes, int *ierr);
/* last method-2 call: events searched exhaustively, coarse nodes, blocks of
 * fine nodes examined over the other events, and the most for one event */
void fteik_b200_locate_getPruneInfo(int *nfallback, int *ncoarse, long long *nblocks, int *maxblocks,
                                    int *ierr);
void fteik_b200_locate_getSurrogateTable(int itf, int n, float out[], int *ierr);
/* Device time of the stages of the last method-2 call (CUDA events on the
 * library stream, recorded while enabled): coarse ranking, pruned re-score,
 * results to the host. */
void fteik_b200_locate_setStageTiming(int enable, int *ierr);
void fteik_b200_locate_getStageTimes(float *coarse_ms, float *prune_ms, float *copy_ms, int *ierr);

/* ---- surrogate network (no counterpart in the reference) ----------------
 * 6 normalised inputs (grid node z, x, y and station z, x, y, each mapped to
 * [-1, 1] over the grid) -> depth hidden layers of width SiLU units -> tau.
 * FP32 on the GPU, trained by Adam on mean squared error. */
void fteik_b200_mlp_initialize(int width, int depth, unsigned long long seed, int *ierr);
void fteik_b200_mlp_finalize(void);
void fteik_b200_mlp_getNumberOfWeights(int *n, int *ierr);
/* weights: per linear layer W [out][in] then b [out] */
void fteik_b200_mlp_getWeights(int n, float w[], int *ierr);
void fteik_b200_mlp_setWeights(int n, const float w[], int *ierr);
void fteik_b200_mlp_forward(int n, const float x[], float tau[], int *ierr);
/* mean squared error of n rows (x [n][6], y [n]) and its gradient (n weights) */
void fteik_b200_mlp_gradient(int n, const float x[], const float y[], double *loss, float grad[],
                             int *ierr);
void fteik_b200_mlp_train(int n, const float x[], const float y[], int steps, int batch, double lr,
                          double *loss, int *ierr);
/* Arithmetic of the network's hidden-layer products (forward, input and
 * weight gradients, inference): 1 (default) = tensor cores (tcgen05), BF16
 * operands, FP32 accumulation; 3 = tensor cores, each FP32 operand split
 * into BF16 hi + lo and the products hi hi + hi lo + lo hi (about FP32
 * accuracy, three times the tensor work); 0 = FP32 on the CUDA cores.  The
 * first and last layers (6 inputs, 1 output) always run on the CUDA cores;
 * weights, Adam and losses stay FP32. */
void fteik_b200_mlp_setTensorProducts(int products, int *ierr);
void fteik_b200_mlp_getTensorProducts(int *products);
/* Training on the locator's tables (fteik_b200_locate_trainSurrogate)
 * captures one step in a CUDA graph and replays it (on = 1, the default);
 * 0 launches every kernel of every step.  Both give the same weights bit
 * for bit. */
void fteik_b200_mlp_setTrainGraph(int on);
void fteik_b200_mlp_getTrainGraph(int *on);
/* Inference (fteik_b200_mlp_forward, the surrogate's coarse tables) with
 * BF16 products and 256 hidden units runs the whole network in one
 * tensor-core kernel per 128 rows (on = 1, the default); 0 runs it layer by
 * layer.  Both give the same bits. */
void fteik_b200_mlp_setFusedForward(int on);
void fteik_b200_mlp_getFusedForward(int *on);
/* The tensor-core products stage their FP32 operands into shared memory by
 * asynchronous copies, several K blocks ahead, where the operands are
 * 16-byte aligned (on = 1, the default); 0 stages every K block with plain
 * loads.  Both give the same bits. */
void fteik_b200_mlp_setAsyncStaging(int on);
void fteik_b200_mlp_getAsyncStaging(int *on);

/* The 2D ray paths of the last fteik_solver2d_traceRaysToPoints /
 * ToReceivers (rays.F90:449-670, which keeps them in module variables no C
 * caller can read).  Ray ir (1-based) runs from its end point to the
 * source's grid point: its integration points (x, z, model coordinates,
 * getRayPath), and the cells it crosses with the length inside each (cells:
 * 1-based natural cell index (ix - 1)(nz - 1) + iz, getRayCells).
 * maxpts / maxseg = 0 only returns the count.  getRayTimes: per ray the
 * time along the steps (step length x slowness of its starting cell), the
 * drop of the travel-time field along the path, the time from the cell
 * pieces (length x cell slowness), and status 1 when the ray did not reach
 * the source in nx nz steps.  No counterpart in the reference's C API. */
void fteik_b200_solver2d_getNumberOfRays(int *nray, int *ierr);
void fteik_b200_solver2d_getRayTimes(int nray, double tstep[], double tfield[], double tcell[], int status[],
                                     int *ierr);
void fteik_b200_solver2d_getRayPath(int ir, int maxpts, double x[], double z[], int *npts, int *ierr);
void fteik_b200_solver2d_getRayCells(int ir, int maxseg, int cells[], double lengths[], int *nseg, int *ierr);

/* Allocation-free grid search (no counterpart in the reference).  For
 * callers that cannot let a library allocate device memory -- a host that
 * hands out every device buffer from its own pool, or a service that must
 * avoid the device-wide synchronisation cudaMalloc/cudaFree can cause.  All
 * buffers are device pointers the caller owns: tables[ntf][ldgrd] FP32,
 * obs/wts[nev][ntf] FP32 (picks already reduced by the event's largest pick,
 * weight 0 = skipped pick), and the outputs opt_index (0-based grid index;
 * add 1 for locate_locateEvent's optIndx), t0 and obj in FP32 -- the same
 * objective and optimum as locate_locateEvent.  stream is a cudaStream_t
 * (NULL: the legacy default stream); the call returns after launching.
 * Limits: 1 <= nev <= 65536, 1 <= ntf <= 64.  Its scratch (12 bytes per
 * event) is a fixed array that every device loading the library keeps until
 * exit; every call looks up that array's device address on the current
 * device (the first lookup on a device may load the library's device code,
 * so make the first call on a device before any stream capture).  Every call reuses the
 * same array, so calls whose work overlaps on the GPU race: order them on
 * one stream.  It allocates nothing (no cudaMalloc, cudaFree or stream
 * creation). */
void fteik_b200_locate_l2_noalloc(int ngrd, int ldgrd, int ntf, const float *tables,
                                  int nev, const float *obs, const float *wts,
                                  int *opt_index, float *t0, float *obj, void *stream,
                                  int *ierr);

#ifdef __cplusplus
}
#endif
#endif
