/*
 * tileplan.c -- host side of the 3D schedules: the per-sweep task table
 * (row tasks ordered by row, or tile tasks ordered by tile level, of every
 * work item) and the device bookkeeping buffers, in one device allocation.
 */
#include "host_common.h"
#include "tileplan.h"

#include <stdlib.h>
#include <string.h>

void fk_tileplan_free(fk_tileplan_t *pl)
{
    fk_dfree(pl->mem);
    memset(pl, 0, sizeof(*pl));
}

static size_t al(size_t b) { return (b + 255) & ~(size_t)255; }

static int rowplan_build(fk_tileplan_t *pl, int nwork, const int *nx, const int *ny, const int *nz,
                         const int *gid, int npass, const char *who);

int fk_tileplan_build(fk_tileplan_t *pl, int nwork, const int *nx, const int *ny, const int *nz,
                      const int *gid, int npass, const char *who)
{
    if (fk_schedule_kind() == FK_PLAN_ROWS) return rowplan_build(pl, nwork, nx, ny, nz, gid, npass, who);
    fk_tileplan_free(pl);
    int *ntx = (int *)malloc(sizeof(int) * (size_t)nwork);
    int *nty = (int *)malloc(sizeof(int) * (size_t)nwork);
    int *base = (int *)malloc(sizeof(int) * (size_t)nwork);
    long ntiles = 0;
    int maxL = 0;
    for (int w = 0; w < nwork; w++) {
        ntx[w] = (nx[w] + FK_TILE_X - 1) / FK_TILE_X;
        nty[w] = (ny[w] + FK_TILE_Y - 1) / FK_TILE_Y;
        base[w] = (int)ntiles;
        ntiles += (long)ntx[w] * nty[w];
        if (ntx[w] + nty[w] - 2 > maxL) maxL = ntx[w] + nty[w] - 2;
    }
    if (ntiles > (1L << 30)) { FK_ERR("%s: too many tiles", who); free(ntx); free(nty); free(base); return 1; }
    int *tasks = (int *)malloc(sizeof(int) * 2 * (size_t)ntiles);
    long k = 0;
    for (int L = 0; L <= maxL; L++)
        for (int w = 0; w < nwork; w++) {
            int b0 = L - (nty[w] - 1);
            if (b0 < 0) b0 = 0;
            int b1 = L < ntx[w] - 1 ? L : ntx[w] - 1;
            for (int bxl = b0; bxl <= b1; bxl++) {
                tasks[2 * k] = w;
                tasks[2 * k + 1] = (L - bxl) * ntx[w] + bxl;
                k++;
            }
        }
    const int np = npass > 0 ? npass : 1;
    size_t off_tasks = 0;
    size_t off_base = off_tasks + al(sizeof(int) * 2 * (size_t)ntiles);
    size_t off_done = off_base + al(sizeof(int) * (size_t)nwork);
    size_t off_tick = off_done + al(sizeof(int) * (size_t)ntiles);
    size_t off_err = off_tick + al(2 * sizeof(unsigned long long));
    size_t off_res = off_err + al(sizeof(int));
    size_t off_pt = off_res + al(sizeof(unsigned long long) * (size_t)nwork * np);
    size_t off_cp = off_pt + al(sizeof(int) * (size_t)nwork * np);
    size_t total = off_cp + al(sizeof(int) * (size_t)nwork);
    char *m = (char *)fk_dalloc(total, who);
    int e = m ? 0 : 1;
    if (!e) e = fk_check((int)fk_h2d(m + off_tasks, tasks, sizeof(int) * 2 * (size_t)ntiles), who);
    if (!e) e = fk_check((int)fk_h2d(m + off_base, base, sizeof(int) * (size_t)nwork), who);
    free(tasks); free(ntx); free(nty); free(base);
    if (e) { fk_dfree(m); return 1; }
    pl->mem = m;
    pl->nwork = nwork;
    pl->npass = np;
    pl->dev.tasks = (const int *)(m + off_tasks);
    pl->dev.done_base = (const int *)(m + off_base);
    pl->dev.ntask_sweep = (int)ntiles;
    pl->dev.ntiles_total = (int)ntiles;
    pl->dev.done = (int *)(m + off_done);
    pl->dev.tickets = (unsigned long long *)(m + off_tick);
    pl->dev.error = (int *)(m + off_err);
    pl->dev.resid = (unsigned long long *)(m + off_res);
    pl->dev.pass_tiles = (int *)(m + off_pt);
    pl->dev.conv_pass = (int *)(m + off_cp);
    /* a bounded wait gives up after 2^22 polls (a few seconds), far longer than
     * any tile takes */
    pl->dev.spin_limit = 1LL << 22;
    pl->dev.kind = FK_PLAN_TILES;
    for (int w = 0; w < nwork; w++) {
        if (nx[w] > pl->dev.max_nx) pl->dev.max_nx = nx[w];
        if (ny[w] > pl->dev.max_ny) pl->dev.max_ny = ny[w];
        if (nz[w] > pl->dev.max_nz) pl->dev.max_nz = nz[w];
    }
    return 0;
}

/* Slab plan: tasks {work, j'} for logical slabs j' = 0.. (FK_SLAB_Y rows
 * each) in order, all work items interleaved; one progress counter per
 * slab.  For the Gauss-Seidel passes, consecutive work items of one grid are
 * paired (tasks2 {pair, j'}), unless FTEIK_B200_PAIRS=0. */
static int rowplan_build(fk_tileplan_t *pl, int nwork, const int *nx, const int *ny, const int *nz,
                         const int *gid, int npass, const char *who)
{
    fk_tileplan_free(pl);
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
    const char *pv = getenv("FTEIK_B200_PAIRS");
    const int pairing = !(pv && strcmp(pv, "0") == 0);
    int *pairs = (int *)malloc(sizeof(int) * 2 * (size_t)nwork);
    int npair = 0;
    for (int w = 0; w < nwork; w++) {
        pairs[2 * npair] = w;
        pairs[2 * npair + 1] = -1;
        if (pairing && w + 1 < nwork && gid[w + 1] == gid[w]) pairs[2 * npair + 1] = ++w;
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
    size_t total = off_t2 + al(sizeof(int) * 2 * (size_t)ntask2);
    char *m = (char *)fk_dalloc(total, who);
    int e = m ? 0 : 1;
    if (!e) e = fk_check((int)fk_h2d(m + off_tasks, tasks, sizeof(int) * 2 * (size_t)nslab), who);
    if (!e) e = fk_check((int)fk_h2d(m + off_base, base, sizeof(int) * (size_t)nwork), who);
    if (!e) e = fk_check((int)fk_h2d(m + off_pairs, pairs, sizeof(int) * 2 * (size_t)npair), who);
    if (!e) e = fk_check((int)fk_h2d(m + off_t2, tasks2, sizeof(int) * 2 * (size_t)ntask2), who);
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
    pl->dev.ntiles_total = (int)nslab;
    pl->dev.done = (int *)(m + off_done);
    pl->dev.tickets = (unsigned long long *)(m + off_tick);
    pl->dev.error = (int *)(m + off_err);
    pl->dev.resid = (unsigned long long *)(m + off_res);
    pl->dev.pass_tiles = (int *)(m + off_pt);
    pl->dev.conv_pass = (int *)(m + off_cp);
    pl->dev.spin_limit = 1LL << 22;
    pl->dev.kind = FK_PLAN_ROWS;
    pl->dev.max_nx = maxnx;
    pl->dev.max_ny = maxny;
    pl->dev.max_nz = maxnz;
    pl->dev.pairs = pairing ? (const int *)(m + off_pairs) : NULL;
    pl->dev.tasks2 = (const int *)(m + off_t2);
    pl->dev.ntask2_sweep = (int)ntask2;
    return 0;
}

int fk_schedule_walker(void)
{
    const char *v = getenv("FTEIK_B200_SCHEDULE");
    return v && strcmp(v, "walker") == 0;
}

int fk_schedule_kind(void)
{
    const char *v = getenv("FTEIK_B200_SCHEDULE");
    return (v && strcmp(v, "tiles") == 0) ? FK_PLAN_TILES : FK_PLAN_ROWS;
}
