/*
 * slabplan.c -- host side of the slab-pipelined 3D sweeps: the per-sweep
 * task table (the slabs of every work item in logical slab order, and the
 * source pairs of the Gauss-Seidel passes) and the device bookkeeping
 * buffers, in one device allocation.
 */
#include "host_common.h"
#include "slabplan.h"

#include <stdlib.h>
#include <string.h>

void fk_slabplan_free(fk_slabplan_t *pl)
{
    fk_dfree(pl->mem);
    memset(pl, 0, sizeof(*pl));
}

static size_t al(size_t b) { return (b + 255) & ~(size_t)255; }

/* Slab plan: tasks {work, j'} for logical slabs j' = 0.. (FK_SLAB_Y rows
 * each) in order, all work items interleaved; one progress counter per
 * slab.  With pairing, consecutive work items of one grid walk the
 * Gauss-Seidel passes together (tasks2 {pair, j'}). */
int fk_slabplan_build(fk_slabplan_t *pl, int nwork, const int *nx, const int *ny, const int *nz,
                      const int *gid, int npass, int pairing, const char *who)
{
    fk_slabplan_free(pl);
    int *base = (int *)malloc(sizeof(int) * (size_t)nwork);
    int *nsl = (int *)malloc(sizeof(int) * (size_t)nwork);
    long nslab = 0;
    int maxsl = 0, maxny = 0, maxnx = 0, maxnz = 0;
    for (int w = 0; w < nwork; w++) {
        nsl[w] = (ny[w] + FK_SLAB_Y - 1) / FK_SLAB_Y;
        base[w] = (int)nslab;
        nslab += nsl[w];
        if (nsl[w] > maxsl) maxsl = nsl[w];
        if (ny[w] > maxny) maxny = ny[w];
        if (nx[w] > maxnx) maxnx = nx[w];
        if (nz[w] > maxnz) maxnz = nz[w];
    }
    if (nslab > (1L << 30)) { FK_ERR("%s: too many slabs", who); free(base); free(nsl); return 1; }
    int *tasks = (int *)malloc(sizeof(int) * 2 * (size_t)nslab);
    long k = 0;
    for (int j = 0; j < maxsl; j++)
        for (int w = 0; w < nwork; w++)
            if (j < nsl[w]) {
                tasks[2 * k] = w;
                tasks[2 * k + 1] = j;
                k++;
            }
    /* pairs of work items of one grid */
    int *pairs = (int *)malloc(sizeof(int) * 2 * (size_t)nwork);
    int npair = 0;
    for (int w = 0; w < nwork; w++) {
        pairs[2 * npair] = w;
        pairs[2 * npair + 1] = -1;
        if (w + 1 < nwork && gid[w + 1] == gid[w]) pairs[2 * npair + 1] = ++w;
        npair++;
    }
    long ntask2 = 0;
    for (int p = 0; p < npair; p++) ntask2 += nsl[pairs[2 * p]];
    int *tasks2 = (int *)malloc(sizeof(int) * 2 * (size_t)ntask2);
    k = 0;
    for (int j = 0; j < maxsl; j++)
        for (int p = 0; p < npair; p++)
            if (j < nsl[pairs[2 * p]]) {
                tasks2[2 * k] = p;
                tasks2[2 * k + 1] = j;
                k++;
            }
    /* initialisation sweeps, one source per thread: a turned-axes task per
     * work item ahead of the slab tasks of each sweep */
    const long ntask_i = nslab + nwork;
    int *tasks_i = (int *)malloc(sizeof(int) * 2 * (size_t)ntask_i);
    for (int w = 0; w < nwork; w++) {
        tasks_i[2 * w] = w;
        tasks_i[2 * w + 1] = -1;
    }
    memcpy(tasks_i + 2 * (size_t)nwork, tasks, sizeof(int) * 2 * (size_t)nslab);
    const int np = npass > 0 ? npass : 1;
    size_t off_tasks = 0;
    size_t off_base = off_tasks + al(sizeof(int) * 2 * (size_t)nslab);
    size_t off_done = off_base + al(sizeof(int) * (size_t)nwork);
    size_t off_tick = off_done + al(sizeof(int) * (size_t)nslab);
    size_t off_err = off_tick + al(2 * sizeof(unsigned long long));
    size_t off_res = off_err + al(sizeof(int));
    size_t off_pt = off_res + al(sizeof(unsigned long long) * (size_t)nwork * np);
    size_t off_cp = off_pt + al(sizeof(int) * (size_t)nwork * np);
    size_t off_pairs = off_cp + al(sizeof(int) * (size_t)nwork);
    size_t off_t2 = off_pairs + al(sizeof(int) * 2 * (size_t)npair);
    size_t off_ti = off_t2 + al(sizeof(int) * 2 * (size_t)ntask2);
    size_t off_dt = off_ti + al(sizeof(int) * 2 * (size_t)ntask_i);
    size_t total = off_dt + al(sizeof(int) * (size_t)nwork);
    char *m = (char *)fk_dalloc(total, who);
    int e = m ? 0 : 1;
    if (!e) e = fk_check((int)fk_h2d(m + off_tasks, tasks, sizeof(int) * 2 * (size_t)nslab), who);
    if (!e) e = fk_check((int)fk_h2d(m + off_base, base, sizeof(int) * (size_t)nwork), who);
    if (!e) e = fk_check((int)fk_h2d(m + off_pairs, pairs, sizeof(int) * 2 * (size_t)npair), who);
    if (!e) e = fk_check((int)fk_h2d(m + off_t2, tasks2, sizeof(int) * 2 * (size_t)ntask2), who);
    if (!e) e = fk_check((int)fk_h2d(m + off_ti, tasks_i, sizeof(int) * 2 * (size_t)ntask_i), who);
    free(tasks_i);
    free(tasks);
    free(tasks2);
    free(pairs);
    free(base);
    free(nsl);
    if (e) { fk_dfree(m); return 1; }
    pl->mem = m;
    pl->nwork = nwork;
    pl->npass = np;
    pl->dev.tasks = (const int *)(m + off_tasks);
    pl->dev.done_base = (const int *)(m + off_base);
    pl->dev.ntask_sweep = (int)nslab;
    pl->dev.nslab_total = (int)nslab;
    pl->dev.done = (int *)(m + off_done);
    pl->dev.tickets = (unsigned long long *)(m + off_tick);
    pl->dev.error = (int *)(m + off_err);
    pl->dev.resid = (unsigned long long *)(m + off_res);
    pl->dev.pass_slabs = (int *)(m + off_pt);
    pl->dev.conv_pass = (int *)(m + off_cp);
    pl->dev.spin_limit = fk_spin_limit();
    pl->dev.max_nx = maxnx;
    pl->dev.max_ny = maxny;
    pl->dev.max_nz = maxnz;
    pl->pairs_all = (const int *)(m + off_pairs);
    pl->dev.pairs = pairing ? pl->pairs_all : NULL;
    pl->dev.tasks2 = (const int *)(m + off_t2);
    pl->dev.ntask2_sweep = (int)ntask2;
    pl->dev.tasks_init = (const int *)(m + off_ti);
    pl->dev.ntask_init_sweep = (int)ntask_i;
    pl->dev.done_t = (int *)(m + off_dt);
    return 0;
}
