/*
 * fteik_dev.h -- internal C interface between the C host layer and the CUDA
 * kernels of libfteik_shared.so.  Plain C types and device pointers only.
 *
 * Device data layout (all grids column major, z fastest, like the reference):
 *   travel-time field of one source : [ny][nx][zp]   zp  = pitch >= nz
 *   cell slowness of one grid       : [ny-1][nx-1][zcp] zcp = pitch >= nz-1
 * Pitches are multiples of 8 elements so every z column starts on a 32-byte
 * boundary.
 */
#ifndef FTEIK_DEV_H
#define FTEIK_DEV_H

#include <stdint.h>
#include <cuda_runtime.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FK_HUGE 99999.0
#define FK_PITCH(n) ((((n) + 7) / 8) * 8)

/* One 3D grid of a (possibly batched) solve. */
typedef struct {
    int nz, nx, ny;
    int zp, zcp;          /* field / slowness z pitches (elements) */
    double dz, dx, dy;
    const void *slow;     /* device: float (FP32 solve) or double (FP64 solve) */
    /* FP32 solve, optional: the cell slowness re-indexed by node z for the
     * staged pass step, [2][ny-1][nx-1][zp]: copy 0 holds at node iz the
     * cell min(iz, nz-2) (the z-downwind cell of ascending sweeps), copy 1
     * the cell max(iz-1, 0) (descending sweeps); NULL when not built */
    const float *slowz;
} fk_grid3d_t;

/* One (grid, source) work item. */
typedef struct {
    int grid;             /* index into the grid table */
    int zsi, xsi, ysi;    /* 1-based source cell (source.F90 conventions) */
    double zsa, xsa, ysa; /* 1-based fractional source position */
    double szero;         /* slowness of the source cell */
    void *tt;             /* device field, [ny][nx][zp] */
} fk_work3d_t;

/* Per-work-item outputs of a solve. */
typedef struct {
    double residual;      /* FP64 max |dt| of the last pass */
    int npass;            /* Gauss-Seidel passes run after the init pass */
    int status;           /* 0 ok */
} fk_result3d_t;

/* Plan of a slab-pipelined 3D solve (device buffers; see row3d_impl.cuh):
 * tasks are slabs of FK_SLAB_Y y-rows, {work, j'} ordered by the logical
 * slab j', done[] one progress counter per slab, done_base each work item's
 * first counter; the other buffers are scratch sized as noted. */
typedef struct {
    const int *tasks;              /* 2 * ntask_sweep ints */
    const int *done_base;          /* nwork */
    int ntask_sweep, nslab_total;
    int *done;                     /* nslab_total */
    unsigned long long *tickets;   /* 2: initialisation and pass launches */
    int *error;                    /* 1 */
    unsigned long long *resid;     /* nwork * max(npass, 1) */
    int *pass_slabs;               /* nwork * max(npass, 1) */
    int *conv_pass;                /* nwork */
    long long spin_limit;          /* bounded waits: polls before giving up */
    int max_nx, max_ny, max_nz;    /* largest grid of the plan */
    /* the Gauss-Seidel passes run sources of one grid in pairs
     * (NULL: one source per task); pairs[2 p + i] work items (-1: none),
     * tasks2 {pair, j'} ordered by j' */
    const int *pairs;
    const int *tasks2;
    int ntask2_sweep;
    /* launch configuration: FP32 passes in the staged pass step (every
     * grid's slowz built); progress step of the passes (8, 32 or 0 = by the
     * number of slab tasks); resident blocks per SM of the pass and of the
     * initialisation kernel (0 = as many as fit) */
    int staged, progress, blocks_per_sm, init_blocks_per_sm;
    /* FP32 initialisation sweeps: the source pairs walked together (the
     * union of their boxes), or NULL for one source per thread */
    const int *init_pairs;
    /* initialisation sweeps with one source per thread: tasks_init = one
     * {work, -1} task per work item (the whole sweep of a box at most
     * FK_SLAB_Y z positions deep, walked with the axes turned) followed by
     * the slab tasks; done_t one counter per work item for those tasks */
    const int *tasks_init;
    int ntask_init_sweep;
    int *done_t;                   /* nwork */
} fk_slabs3d_t;

#define FK_SLAB_Y 4

/* Slab-pipelined solve of every work item: field initialisation, 8
 * initialisation sweeps, then nsweep passes of 8 sweeps (or, when conv_tol
 * >= 0 and max_pass > 0, passes until a pass changes no node by more than
 * conv_tol).  precision: 4 (FP32 field, FP64 near-source stencil) or 8 (FP64
 * field).  grids/work/results are device arrays.  Returns a cudaError_t. */
int fk3d_solve_slabs(int precision, const fk_grid3d_t *grids, const fk_work3d_t *work,
                     int nwork, const fk_slabs3d_t *plan, fk_result3d_t *results, double eps,
                     int nsweep, double conv_tol, int max_pass, cudaStream_t stream);
/* Optional timing: events recorded before the initialisation kernel, after
 * it and after the Gauss-Seidel kernel of every later fk3d_solve_slabs on
 * this host thread (NULL to stop). */
void fk3d_slabs_set_events(cudaEvent_t *ev3);

/* ---- 2D ---------------------------------------------------------------- */
typedef struct {
    int nz, nx, zp, zcp;
    double dz, dx;
    const double *slow;   /* device, [nx-1][zcp] */
} fk_grid2d_t;

typedef struct {
    int grid;
    int zsi, xsi;
    double zsa, xsa, szero;
    double *tt;           /* device, [nx][zp] FP64 */
} fk_work2d_t;

/* 2D LSM (fsm = 0) or FSM (fsm = 1) solve of every work item in FP64. */
int fk2d_solve(int fsm, const fk_grid2d_t *grids, const fk_work2d_t *work,
               fk_result3d_t *results, int nwork, int max_nx, int max_nz, double eps,
               int nsweep, double conv_tol, int max_pass, cudaStream_t stream);

/* 2D ray paths (rays2d.cu): pass 1 counts points and (cell, length) pieces
 * and writes npts / nseg / status / tn / tne per ray; pass 2 writes the
 * points and pieces at pts_off / seg_off.  Positions relative to the model
 * origin; slow [nx-1][zcp], tt [nx][zp], gx / gz [nx][nz] device arrays. */
int fk_rays2d(int pass, int nz, int nx, int zp, int zcp, double dz, double dx, const double *slow,
              const double *tt, const double *gx, const double *gz, int integrator, double xs, double zs,
              int nray, const double *xr, const double *zr, int *npts, int *nseg, int *status,
              double *tn, double *tne, const long long *pts_off, const long long *seg_off, double *px,
              double *pz, int *cells, double *lens, cudaStream_t s);

/* ---- field utilities --------------------------------------------------- */
/* Fill a padded slowness array (precision 4 or 8) from FP64 cell slowness in
 * the reference's natural layout. */
int fk_pack_slowness(int precision, int is3d, int nz, int nx, int ny, int zcp,
                     const double *slow_nat, void *slow_dev, cudaStream_t s);
/* 3D cell velocities (device, FP64 natural) -> padded slowness 1/v;
 * *bad_dev = 1 when a velocity is not positive (bad_dev zeroed by the caller). */
/* The node-indexed FP32 slowness copies of fk_grid3d_t.slowz from the
 * padded FP32 cell slowness (3D). */
int fk_node_slowness_f32(int nz, int nx, int ny, int zcp, int zp, const float *slow_dev,
                         float *slowz_dev, cudaStream_t s);
int fk_pack_velocity(int precision, int nz, int nx, int ny, int zcp, const double *vel_nat,
                     void *slow_dev, int *bad_dev, cudaStream_t s);
/* out[i] = v[idx[i]] on the device. */
int fk_gather64(const double *v, const long long *idx, int n, double *out, cudaStream_t s);
/* Copy a padded field (precision 4 or 8) to FP64 in the requested ordering:
 * 0 natural (z fastest), 1 XYZ / XZ (x fastest, z slowest), 2 ZYX. */
int fk_field_to_f64(int precision, int is3d, int nz, int nx, int ny, int zp,
                    const void *tt, int order, double *out, cudaStream_t s);
/* Cell-averaged field (getTravelTimeFieldCell64f). */
int fk_field_cell_to_f64(int precision, int is3d, int nz, int nx, int ny,
                         int zp, const void *tt, int order, double *out,
                         cudaStream_t s);
/* Trilinear (3D) / bilinear (2D) receiver interpolation, receiver.F90. */
int fk_receivers(int precision, int is3d, int nz, int nx, int ny, int zp,
                 double dz, double dx, double dy, const void *tt, int nrec,
                 const int *ri /* 3*nrec: zri,xri,yri 1-based */,
                 const double *rd /* 3*nrec: zdr,xdr,ydr */, double *ttr,
                 cudaStream_t s);
/* Batched receiver extraction for many fields sharing one geometry:
 * fields[f] -> ttr[f*nrec + r]. */
int fk_receivers_batch(int precision, int nz, int nx, int ny, int zp,
                       double dz, double dx, double dy, void *const *fields,
                       int nfield, int nrec, const int *ri, const double *rd,
                       double *ttr, cudaStream_t s);
/* The same for FP64 2D fields (bilinear, receiver.F90:246-285 in 2D). */
int fk_receivers_batch2d(int nx, int zp, double dz, double dx, void *const *fields, int nfield,
                         int nrec, const int *ri, const double *rd, double *ttr, cudaStream_t s);
/* Finite-difference travel-time gradients (solver3D.F90:1249-1321,
 * solver2D.F90:984-1032), FP64 out: 3D g[3 m + {x, y, z}], 2D gx[m], gz[m]. */
int fk_gradient3d(int precision, int nz, int nx, int ny, int zp, double dz, double dx, double dy,
                  const void *tt, double *g, cudaStream_t s);
int fk_gradient2d(int nz, int nx, int zp, double dz, double dx, const double *tt, double *gx,
                  double *gz, cudaStream_t s);
/* Analytic fields (analytic.F90) in the solver's natural order. */
int fk_analytic_field(int kind /*0 const, 1 linear*/, int nz, int nx, int ny,
                      double z0, double x0, double y0, double dz, double dx,
                      double dy, double v0, double v1, double zs, double xs,
                      double ys, double *out, cudaStream_t s);

/* Analytic times at arbitrary points for nsrc sources: out[s*ldr + p]. */
int fk_analytic_points(int kind, int nz, double z0, double dz, double v0, double v1,
                       int npts, const double *z, const double *x, const double *y,
                       int nsrc, const double *zs, const double *xs, const double *ys,
                       int ldr, double *out, cudaStream_t s);
int fk_f64_to_f32(size_t n, const double *in, float *out, cudaStream_t s);
/* Dense copy of padded FP32 rows: src [rows][zp] -> dst [rows][nz]. */
int fk_unpad_f32(const float *src, float *dst, size_t rows, int nz, int zp, cudaStream_t s);

/* ---- locate ------------------------------------------------------------- */
/* Exact FP32 L2 grid search (locate.F90:620-744) for nev events:
 * tables [ntf][ldgrd] FP32; obs/wts [nev][ntf] FP32 (0 weight = skipped);
 * out_idx 0-based, out_t0 / out_obj FP32 values at the optimum. */
int fk_locate_l2_exact(int ngrd, int ldgrd, int ntf, const float *tables,
                       int nev, const float *obs, const float *wts,
                       int *out_idx, float *out_t0, float *out_obj,
                       void *scratch, size_t scratch_bytes, cudaStream_t s);
size_t fk_locate_l2_exact_scratch(int ngrd, int nev);
/* Exhaustive L1 search: picks of one common weight per event (0 = skipped);
 * FP32 obs / wts rank, FP64 obs64 / wts64 give out_t0 (median residual) and
 * out_obj at the optimum; out_idx 0-based; scratch holds nev 64-bit keys. */
int fk_locate_l1_exact(int ngrd, int ldgrd, int ntf, const float *tables, int nev, const float *obs,
                       const float *wts, const double *obs64, const double *wts64, int *out_idx,
                       double *out_t0, double *out_obj, unsigned long long *scratch, cudaStream_t s);

/* Tensor-core L2 search (locate_tc.cu).  Events with every table picked at
 * one common weight (elig[e] = 1) are ranked by a BF16 hi+lo contraction in
 * runs of 32 grid points; the best runs are re-scored point by point in FP64.
 *   pack_tables: tables [ntf][ldgrd] -> bpack (fk_locate_tc_table_bytes).
 *   fk_locate_tc: obs / wts [nev][ntf] FP64 picks (reduced) and weights;
 *                apack scratch (fk_locate_tc_event_bytes); cand_v / cand_i
 *                [nev][npart][FK_TC_TOPK] (run minima / run numbers);
 *                rescore = runs re-scored per event (0: ranking only);
 *                out_idx 0-based, out_t0 / out_obj FP64; error: device int,
 *                0 on success; dbg optional [256][128] floats of the first
 *                accumulators. */
#define FK_TC_TOPK 4
size_t fk_locate_tc_table_bytes(int ngrd);
size_t fk_locate_tc_event_bytes(int nev);
int fk_locate_tc_npart(int nev, int ngrd);
int fk_locate_tc_pack_tables(int ngrd, int ldgrd, int ntf, const float *tables, void *bpack,
                             cudaStream_t s);
int fk_locate_tc(int ngrd, int ldgrd, int ntf, const float *tables, const void *bpack,
                 int nev, const double *obs, const double *wts, const unsigned char *elig,
                 void *apack, int npart, float *cand_v, int *cand_i, int rescore, int *out_idx,
                 double *out_t0, double *out_obj, int *error, float *dbg, cudaStream_t s);

/* Pruned search: coarse runs (cand_* from fk_locate_tc on the coarse
 * surrogate tables [ntf][ldc], coarse node c = cz + ncz (cx + ncx cy) owning
 * the fine block [bz cz, bz cz + bz) x [bx cx, ..) x [by cy, ..)) -> the k best
 * coarse nodes (rc runs examined, rc <= 4, k <= 32) -> FP64 misfit on the
 * exact tables (block-major copy, fk_locate_block_tables) at every fine
 * node of their blocks, then a
 * descent over neighbouring blocks.  flag[e]: 0xFF when the event needs the
 * exhaustive search, else the number of blocks examined. */
int fk_locate_prune(int nev, int npart, int rc, int k, int nz, int nx, int ny, int bz, int bx, int by,
                    int ldgrd, int ldc, int ntf, const float *coarse, const float *fine,
                    const double *obs, const double *wts, const unsigned char *elig,
                    const float *cand_v, const int *cand_i, int *out_idx, double *out_t0,
                    double *out_obj, unsigned char *flag, cudaStream_t s);
/* Block-major copy of tables [ntf][ldgrd] for fk_locate_prune's fine
 * stage: out [nblocks][ntf][bz bx by] (ncz ncx ncy blocks, z fastest). */
int fk_locate_block_tables(int nz, int nx, int ny, int bz, int bx, int by, int ntf, int ldgrd,
                           const float *tables, float *out, cudaStream_t s);

/* ---- surrogate network (mlp.c / mlp.cu) ----------------------------------- */
/* A training batch for step `step`, or, when step_dev is not NULL, for the
 * step number the device holds there (a batch function that can read it
 * lets the trainer capture one step in a CUDA graph and replay it). */
typedef int (*fk_batch_fn)(void *ctx, long long step, const long long *step_dev, int B, float *x, float *y,
                           cudaStream_t s);
int fk_mlp_ready(void);
size_t fk_mlp_flops_per_row(void);
int fk_mlp_train_device(fk_batch_fn next_batch, void *ctx, int capturable, long long steps, int B, double lr,
                        double *last_loss);
int fk_mlp_forward_device(long long n, const float *x, float *tau, cudaStream_t s);
/* Training batch from tables [ntf][ldgrd] on a z-fastest grid and station
 * positions sta [ntf][3] (z, x, y): inputs x [B][6], targets tau [B]. */
int fk_mlp_sample(int nz, int nx, int ny, double dz, double dx, double dy, int ntf, int ldgrd,
                  double vref, const float *tables, const float *sta, unsigned long long seed,
                  long long nsamp, long long step, const long long *step_dev, int B, float *x, float *y,
                  cudaStream_t s);
/* Rows r0 .. r0+nrow-1 of the coarse lattice (row = table * ncoarse + node,
 * node = the centre of its fine block bz x bx x by, clipped to the grid):
 * network inputs and distance / v_ref. */
int fk_mlp_coarse_inputs(int nz, int nx, int ny, double dz, double dx, double dy, int ntf,
                         double vref, const float *sta, int bz, int bx, int by, int ncz, int ncx,
                         int ncy, long long r0, long long nrow, float *x, float *dist, cudaStream_t s);
int fk_mlp_coarse_store(long long r0, long long nrow, long long nc, int ldc, const float *tau,
                        const float *dist, float *out, cudaStream_t s);

#ifdef __cplusplus
}
#endif
#ifdef __CUDACC__
/* The surrogate's SiLU, z / (1 + e^-z), with the fast exponential and
 * division (relative error of order 1e-7): one definition for every kernel
 * that applies it, so the fused and layer-by-layer passes round alike. */
static __device__ __forceinline__ float fk_sigmoid(float z) { return __fdividef(1.0f, 1.0f + __expf(-z)); }
static __device__ __forceinline__ float fk_silu(float z) { return z * fk_sigmoid(z); }
#endif

#endif
