/* slabplan.h -- host-side plan of the slab-pipelined 3D solve. */
#ifndef FTEIK_SLABPLAN_H
#define FTEIK_SLABPLAN_H
#include "fteik_dev.h"

typedef struct {
    fk_slabs3d_t dev; /* device pointers passed to fk3d_solve_slabs */
    void *mem;        /* the one device allocation behind them */
    int nwork, npass;
    const int *pairs_all; /* the source pairs (dev.pairs is this or NULL) */
} fk_slabplan_t;

/* Build the plan for nwork work items with the given grid sizes and grid
 * numbers (gid); npass is the most Gauss-Seidel passes a solve will run;
 * pairing (0 or 1) lets consecutive work items of one grid walk the passes
 * together (the pairs are built either way: pairs_all).  The plan's bounded waits take the library's current poll limit
 * (fteik_b200_setSpinLimit).  Returns 0 on success. */
int fk_slabplan_build(fk_slabplan_t *pl, int nwork, const int *nx, const int *ny, const int *nz,
                      const int *gid, int npass, int pairing, const char *who);
void fk_slabplan_free(fk_slabplan_t *pl);
#endif
