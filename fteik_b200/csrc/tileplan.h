/* tileplan.h -- host-side plan of the tile-wavefront 3D solve. */
#ifndef FTEIK_TILEPLAN_H
#define FTEIK_TILEPLAN_H
#include "fteik_dev.h"

typedef struct {
    fk_tiles3d_t dev; /* device pointers passed to fk3d_solve_tiles */
    void *mem;        /* the one device allocation behind them */
    int nwork, npass;
} fk_tileplan_t;

/* Build the plan for nwork work items with the given grid sizes and grid
 * numbers (gid); npass is the most Gauss-Seidel passes a solve will run.  The schedule is the row
 * pipeline unless FTEIK_B200_SCHEDULE=tiles.  Returns 0 on success. */
int fk_tileplan_build(fk_tileplan_t *pl, int nwork, const int *nx, const int *ny, const int *nz,
                      const int *gid, int npass, const char *who);
void fk_tileplan_free(fk_tileplan_t *pl);
/* FTEIK_B200_SCHEDULE=walker selects the column-walk kernels instead. */
int fk_schedule_walker(void);
/* FK_PLAN_ROWS, or FK_PLAN_TILES with FTEIK_B200_SCHEDULE=tiles. */
int fk_schedule_kind(void);
#endif
