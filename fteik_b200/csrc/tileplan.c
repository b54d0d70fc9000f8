/*
 * tileplan.c -- host side of the tile-wavefront schedule: the per-sweep
 * task table (tile tasks of every work item ordered by tile level) and the
 * device bookkeeping buffers, in one device allocation.
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

int fk_tileplan_build(fk_tileplan_t *pl, int nwork, const int *nx, const int *ny, int npass,
                      const char *who)
{
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
    if (!e) e = fk_check((int)cudaMemcpy(m + off_tasks, tasks, sizeof(int) * 2 * (size_t)ntiles,
                                         cudaMemcpyHostToDevice), who);
    if (!e) e = fk_check((int)cudaMemcpy(m + off_base, base, sizeof(int) * (size_t)nwork,
                                         cudaMemcpyHostToDevice), who);
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
    return 0;
}

int fk_schedule_walker(void)
{
    const char *v = getenv("FTEIK_B200_SCHEDULE");
    return v && strcmp(v, "walker") == 0;
}
