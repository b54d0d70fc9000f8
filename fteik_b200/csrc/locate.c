/*
 * locate.c -- the reference's locator module (locate.F90) over the device
 * grid search.  Travel-time tables live on the device as FP32 rows of
 * ldgrd entries (ldgrd = ngrd padded to 64 bytes, locate.F90:181-186).
 */
#include "host_common.h"
#include "fteik_b200.h"

#include <stdlib.h>
#include <string.h>

static struct {
    bool init, dirty;
    int nev, ntf, ngrd, ldgrd;
    double *tepoch;
    float *origin;
    bool *have_ot;
    float *obs, *wts;      /* host [nev][ntf]; weight 0 = skipped */
    float *tables;         /* device [ntf][ldgrd] */
    float *obs_dev, *wts_dev;
    int *idx_dev;
    float *t0_dev, *obj_dev;
    void *scratch;
    size_t scratch_bytes;
    int cap_ev;
    /* tensor-core search (locate_tc.cu) */
    int method;              /* 0: exact FP32 (reference arithmetic), 1: tensor core */
    int norm;                /* 2 (the reference's misfit) or 1 */
    unsigned char *l1ok;     /* host [nev]: positive weights all equal */
    int *l1_idx;             /* device outputs of the L1 search */
    double *l1_t0, *l1_obj;
    unsigned long long *l1_best;
    int l1_cap;
    int rescore;             /* candidates re-scored in FP64 per event */
    bool dirty64, tables_dirty;
    long long table_gen;     /* counts table writes */
    double *obs64, *w64;     /* host [nev][ntf], reduced picks and weights */
    unsigned char *elig;     /* host [nev]: every table picked at one weight */
    double *obs64_dev, *w64_dev;
    unsigned char *elig_dev;
    void *bpack;
    void *apack;
    size_t apack_bytes;
    float *cand_v;
    int *cand_i;
    size_t cand_n;
    int *tc_idx;
    double *tc_t0, *tc_obj;
    int tc_cap;
    int *err_dev;
    float *dbg_dev;
} SL;

/* Surrogate-pruned search state: grid geometry of the tables, station
 * positions, the coarse lattice and its surrogate tables. */
static struct {
    bool have_geom, ready;
    int nz, nx, ny;
    double dz, dx, dy, vref;
    float *sta_dev;          /* [ntf][3] z, x, y */
    int bz, bx, by, ncz, ncx, ncy, ngrd_c, ldc;
    float *coarse;           /* device [ntf][ldc] surrogate travel times */
    float *fine_blk;         /* device block-major copy of the exact tables */
    size_t fine_cap;         /* its size in floats */
    size_t coarse_cap, bpack_cap;   /* sizes of coarse / bpack_c (floats / bytes) */
    float *bx_in, *bx_dist, *bx_tau; /* build scratch: inputs, distances, outputs of a chunk */
    long long blk_gen;       /* table generation fine_blk was built from */
    int blk_shape[3];        /* and its block shape (bz, bx, by) */
    void *bpack_c;
    int rc, k;
    unsigned char *flag_dev;
    int flag_cap;
    int last_fallback;
    long long last_blocks;   /* blocks of fine nodes examined in the last call */
    int last_max_blocks;
    bool timing;             /* record stage events in method-2 calls */
    cudaEvent_t ev[4];
    float stage_ms[3];       /* coarse ranking, pruned re-score, results to host */
    double *sub_obs, *sub_w;
    unsigned char *sub_elig;
    int sub_cap;
} SP;

static void surrogate_free(void)
{
    for (int k = 0; k < 4; k++)
        if (SP.ev[k]) cudaEventDestroy(SP.ev[k]);
    fk_dfree(SP.sta_dev); fk_dfree(SP.coarse); fk_dfree(SP.bpack_c); fk_dfree(SP.flag_dev);
    fk_dfree(SP.fine_blk);
    fk_dfree(SP.bx_in); fk_dfree(SP.bx_dist); fk_dfree(SP.bx_tau);
    fk_dfree(SP.sub_obs); fk_dfree(SP.sub_w); fk_dfree(SP.sub_elig);
    memset(&SP, 0, sizeof(SP));
}

void locate_finalize(void)
{
    surrogate_free();
    free(SL.tepoch); free(SL.origin); free(SL.have_ot); free(SL.obs); free(SL.wts);
    fk_dfree(SL.tables); fk_dfree(SL.obs_dev); fk_dfree(SL.wts_dev);
    fk_dfree(SL.idx_dev); fk_dfree(SL.t0_dev); fk_dfree(SL.obj_dev); fk_dfree(SL.scratch);
    free(SL.obs64); free(SL.w64); free(SL.elig); free(SL.l1ok);
    fk_dfree(SL.l1_idx); fk_dfree(SL.l1_t0); fk_dfree(SL.l1_obj); fk_dfree(SL.l1_best);
    fk_dfree(SL.obs64_dev); fk_dfree(SL.w64_dev); fk_dfree(SL.elig_dev); fk_dfree(SL.bpack);
    fk_dfree(SL.apack); fk_dfree(SL.cand_v); fk_dfree(SL.cand_i);
    fk_dfree(SL.tc_idx); fk_dfree(SL.tc_t0); fk_dfree(SL.tc_obj); fk_dfree(SL.err_dev);
    fk_dfree(SL.dbg_dev);
    memset(&SL, 0, sizeof(SL));
}

void locate_setNumberOfEvents(int nEvents, int *ierr)
{
    *ierr = 0;
    SL.nev = 0;
    if (nEvents < 1) { FK_ERR("locate_setNumberOfEvents: nEvents=%d must be positive", nEvents); *ierr = 1; return; }
    SL.nev = nEvents;
}

void locate_setNumberOfTravelTimeFields(int ntf, int *ierr)
{
    *ierr = 0;
    SL.ntf = 0;
    if (ntf < 1) { FK_ERR("locate_setNumberOfTravelTimeFields: ntf=%d must be positive", ntf); *ierr = 1; return; }
    SL.ntf = ntf;
}

void locate_setNumberOfGridPointsF(int ngrd, int *ierr)
{
    *ierr = 0;
    SL.ngrd = 0;
    if (ngrd < 1) { FK_ERR("locate_setNumberOfGridPointsF: ngrd=%d must be positive", ngrd); *ierr = 1; return; }
    SL.ngrd = ngrd;
}

void locate_initialize(int nEvents, int ntf, int ngrd, int *ierr)
{
    /* locate.F90:142-223 */
    locate_finalize();
    locate_setNumberOfEvents(nEvents, ierr);
    if (*ierr) { FK_ERR("locate_initializeF: Failed to set number of events"); return; }
    locate_setNumberOfTravelTimeFields(ntf, ierr);
    if (*ierr) { FK_ERR("locate_initializeF: Failed to set number of travel time fields"); return; }
    locate_setNumberOfGridPointsF(ngrd, ierr);
    if (*ierr) { FK_ERR("locate_initializeF: Failed to set number of grid points"); return; }
    if (ntf > 64) {
        FK_ERR("locate_initialize: ntf=%d; the device search holds at most 64 tables per grid point", ntf);
        *ierr = 1;
        return;
    }
    if (fk_dev_ready("locate_initialize")) { *ierr = 1; return; }
    SL.ldgrd = (ngrd + 15) / 16 * 16;
    SL.tepoch = (double *)calloc((size_t)nEvents, sizeof(double));
    SL.origin = (float *)calloc((size_t)nEvents, sizeof(float));
    SL.have_ot = (bool *)calloc((size_t)nEvents, sizeof(bool));
    SL.obs = (float *)calloc((size_t)nEvents * ntf, sizeof(float));
    SL.wts = (float *)calloc((size_t)nEvents * ntf, sizeof(float));
    SL.tables = (float *)fk_dalloc(sizeof(float) * (size_t)ntf * SL.ldgrd, "locate_initialize");
    SL.obs_dev = (float *)fk_dalloc(sizeof(float) * (size_t)nEvents * ntf, "locate_initialize");
    SL.wts_dev = (float *)fk_dalloc(sizeof(float) * (size_t)nEvents * ntf, "locate_initialize");
    SL.obs64 = (double *)calloc((size_t)nEvents * ntf, sizeof(double));
    SL.w64 = (double *)calloc((size_t)nEvents * ntf, sizeof(double));
    SL.elig = (unsigned char *)calloc((size_t)nEvents, 1);
    SL.l1ok = (unsigned char *)calloc((size_t)nEvents, 1);
    SL.norm = 2;
    if (!SL.tables || !SL.obs_dev || !SL.wts_dev) { *ierr = 1; return; }
    if (fk_check((int)fk_zero(SL.tables, sizeof(float) * (size_t)ntf * SL.ldgrd),
                 "locate_initialize")) { *ierr = 1; return; }
    SL.init = true;
    SL.dirty = true;
    SL.dirty64 = true;
    SL.tables_dirty = true;
    SL.table_gen++;
    SL.rescore = 8;
}

static int table_check(int ngrd, int itf, const char *who)
{
    if (!SL.init) { FK_ERR("%s: Locator not initialized", who); return 1; }
    /* locate.F90:302 accepts itf = 0 and then writes before the table
     * store; here table numbers must be in [1, ntf] */
    if (itf < 1 || itf > SL.ntf) { FK_ERR("%s: itf=%d out of range [1,%d]", who, itf, SL.ntf); return 1; }
    if (ngrd != SL.ngrd) { FK_ERR("%s: ngrdIn=%d /= ngrd=%d", who, ngrd, SL.ngrd); return 1; }
    return 0;
}

void locate_setTravelTimeField64f(int ngrd, int itf, const double tt[], int *ierr)
{
    /* locate.F90:287-343: FP64 -> FP32 (REAL()) on the device */
    *ierr = table_check(ngrd, itf, "locate_setTravelTimeField64f");
    if (*ierr) return;
    double *d = (double *)fk_dalloc(sizeof(double) * (size_t)ngrd, "locate_setTravelTimeField64f");
    if (!d) { *ierr = 1; return; }
    cudaStream_t s = fk_stream();
    int e = (int)cudaMemcpyAsync(d, tt, sizeof(double) * (size_t)ngrd, cudaMemcpyHostToDevice, s);
    if (!e) e = fk_f64_to_f32((size_t)ngrd, d, SL.tables + (size_t)(itf - 1) * SL.ldgrd, s);
    if (!e) e = (int)cudaStreamSynchronize(s);
    fk_dfree(d);
    SL.tables_dirty = true;
    SL.table_gen++;
    *ierr = fk_check(e, "locate_setTravelTimeField64f");
}

void locate_setTravelTimeField32f(int ngrd, int itf, const float tt[], int *ierr)
{
    /* locate.F90:361-396 */
    *ierr = table_check(ngrd, itf, "locate_setTravelTimeField32f");
    if (*ierr) return;
    int e = (int)cudaMemcpyAsync(SL.tables + (size_t)(itf - 1) * SL.ldgrd, tt,
                                 sizeof(float) * (size_t)ngrd, cudaMemcpyHostToDevice, fk_stream());
    if (!e) e = (int)cudaStreamSynchronize(fk_stream());
    SL.tables_dirty = true;
    SL.table_gen++;
    *ierr = fk_check(e, "locate_setTravelTimeField32f");
}

/* Device table row of table itf (1-based), for the in-library hand-off. */
float *fk_locate_table_row(int itf, int ngrd)
{
    if (!SL.init || itf < 1 || itf > SL.ntf || ngrd != SL.ngrd) return NULL;
    SL.tables_dirty = true;
    SL.table_gen++; /* the caller writes the row */
    return SL.tables + (size_t)(itf - 1) * SL.ldgrd;
}

void locate_setObservation64f(int evnmbr, int nttimes, bool lhaveOT, double t0,
                              const int obs2tf[], const double pickTimes[], const double wts[],
                              int *ierr)
{
    /* locate.F90:431-497 */
    *ierr = 0;
    if (!SL.init) { FK_ERR("locate_setObservation64f: Locator not initialized"); *ierr = 1; return; }
    if (nttimes < 1 || nttimes > SL.ntf) {
        FK_ERR("locate_setObservation64f: nttimes=%d must be in [1,%d]", nttimes, SL.ntf);
        *ierr = 1;
        return;
    }
    int mn = obs2tf[0], mx = obs2tf[0];
    for (int i = 1; i < nttimes; i++) {
        if (obs2tf[i] < mn) mn = obs2tf[i];
        if (obs2tf[i] > mx) mx = obs2tf[i];
    }
    if (mn < 1) { FK_ERR("locate_setObservation64f: All values in obs2tf must be positive"); *ierr = 1; return; }
    if (mx > SL.ntf) { FK_ERR("locate_setObservation64f: obs2tf exceeds ntf=%d", SL.ntf); *ierr = 1; return; }
    if (evnmbr < 1 || evnmbr > SL.nev) {
        FK_ERR("locate_setObservation64f: evnmbr=%d must be in [1,%d]", evnmbr, SL.nev);
        *ierr = 1;
        return;
    }
    double tep = pickTimes[0];
    for (int i = 1; i < nttimes; i++) if (pickTimes[i] > tep) tep = pickTimes[i];
    SL.tepoch[evnmbr - 1] = tep;
    SL.origin[evnmbr - 1] = 0.0f;
    if (lhaveOT) {
        SL.have_ot[evnmbr - 1] = true;
        SL.origin[evnmbr - 1] = (float)(t0 - tep);
    }
    float *o = SL.obs + (size_t)(evnmbr - 1) * SL.ntf, *w = SL.wts + (size_t)(evnmbr - 1) * SL.ntf;
    double *o64 = SL.obs64 + (size_t)(evnmbr - 1) * SL.ntf, *w64 = SL.w64 + (size_t)(evnmbr - 1) * SL.ntf;
    memset(o, 0, sizeof(float) * SL.ntf);
    memset(w, 0, sizeof(float) * SL.ntf);
    memset(o64, 0, sizeof(double) * SL.ntf);
    memset(w64, 0, sizeof(double) * SL.ntf);
    for (int i = 0; i < nttimes; i++) {
        int k = obs2tf[i] - 1;
        if (wts[i] > 0.0) {
            o[k] = (float)(pickTimes[i] - tep); /* reduced time */
            w[k] = (float)wts[i];
            o64[k] = pickTimes[i] - tep;
            w64[k] = wts[i];
        }
    }
    /* the tensor-core search takes events whose picks cover every table
     * with one common weight; others go through the exact search */
    bool el = true;
    for (int k = 0; k < SL.ntf && el; k++) el = w64[k] > 0.0 && w64[k] == w64[0];
    SL.elig[evnmbr - 1] = el ? 1 : 0;
    /* the L1 misfit takes picks of one common weight */
    double wref = 0.0;
    bool l1 = true;
    for (int k = 0; k < SL.ntf && l1; k++)
        if (w64[k] > 0.0) {
            if (wref == 0.0) wref = w64[k];
            l1 = w64[k] == wref;
        }
    SL.l1ok[evnmbr - 1] = (l1 && wref > 0.0) ? 1 : 0;
    SL.dirty = true;
    SL.dirty64 = true;
}

void locate_setObservation64fC(int evnmbr, int nttimes, bool lhaveOT, double t0,
                               const int obs2tf[], const double pickTimes[], const double wts[],
                               int *ierr)
{
    /* fwrapper.c:42-55 */
    int *f = (int *)malloc(sizeof(int) * (size_t)(nttimes > 0 ? nttimes : 1));
    for (int i = 0; i < nttimes; i++) f[i] = obs2tf[i] + 1;
    locate_setObservation64f(evnmbr + 1, nttimes, lhaveOT, t0, f, pickTimes, wts, ierr);
    free(f);
}

static int ensure_out(int n)
{
    if (SL.cap_ev >= n && SL.idx_dev) return 0;
    fk_dfree(SL.idx_dev); fk_dfree(SL.t0_dev); fk_dfree(SL.obj_dev); fk_dfree(SL.scratch);
    SL.idx_dev = (int *)fk_dalloc(sizeof(int) * (size_t)n, "locate");
    SL.t0_dev = (float *)fk_dalloc(sizeof(float) * (size_t)n, "locate");
    SL.obj_dev = (float *)fk_dalloc(sizeof(float) * (size_t)n, "locate");
    SL.scratch_bytes = fk_locate_l2_exact_scratch(SL.ngrd, n);
    SL.scratch = fk_dalloc(SL.scratch_bytes, "locate");
    SL.cap_ev = (SL.idx_dev && SL.t0_dev && SL.obj_dev && SL.scratch) ? n : 0;
    return SL.cap_ev == 0;
}

static int upload_obs(void)
{
    if (!SL.dirty) return 0;
    cudaStream_t s = fk_stream();
    size_t n = (size_t)SL.nev * SL.ntf;
    int e = (int)cudaMemcpyAsync(SL.obs_dev, SL.obs, sizeof(float) * n, cudaMemcpyHostToDevice, s);
    if (!e) e = (int)cudaMemcpyAsync(SL.wts_dev, SL.wts, sizeof(float) * n, cudaMemcpyHostToDevice, s);
    if (fk_check(e, "locate: observation upload")) return 1;
    SL.dirty = false;
    return 0;
}

/* Locate events [e0, e0+n) (0-based, contiguous). */
static int locate_range(int e0, int n, int *idx, float *t0, float *obj)
{
    if (upload_obs() || ensure_out(n)) return 1;
    cudaStream_t s = fk_stream();
    int e = fk_locate_l2_exact(SL.ngrd, SL.ldgrd, SL.ntf, SL.tables, n,
                               SL.obs_dev + (size_t)e0 * SL.ntf, SL.wts_dev + (size_t)e0 * SL.ntf,
                               SL.idx_dev, SL.t0_dev, SL.obj_dev, SL.scratch, SL.scratch_bytes, s);
    if (!e) e = (int)cudaMemcpyAsync(idx, SL.idx_dev, sizeof(int) * (size_t)n, cudaMemcpyDeviceToHost, s);
    if (!e) e = (int)cudaMemcpyAsync(t0, SL.t0_dev, sizeof(float) * (size_t)n, cudaMemcpyDeviceToHost, s);
    if (!e) e = (int)cudaMemcpyAsync(obj, SL.obj_dev, sizeof(float) * (size_t)n, cudaMemcpyDeviceToHost, s);
    if (!e) e = (int)cudaStreamSynchronize(s);
    return fk_check(e, "locate");
}

static int upload_obs64(void)
{
    if (!SL.dirty64) return 0;
    const size_t n = (size_t)SL.nev * SL.ntf;
    if (!SL.obs64_dev) {
        SL.obs64_dev = (double *)fk_dalloc(sizeof(double) * n, "locate");
        SL.w64_dev = (double *)fk_dalloc(sizeof(double) * n, "locate");
        SL.elig_dev = (unsigned char *)fk_dalloc((size_t)SL.nev, "locate");
        if (!SL.obs64_dev || !SL.w64_dev || !SL.elig_dev) return 1;
    }
    cudaStream_t s = fk_stream();
    int e = (int)cudaMemcpyAsync(SL.obs64_dev, SL.obs64, sizeof(double) * n, cudaMemcpyHostToDevice, s);
    if (!e) e = (int)cudaMemcpyAsync(SL.w64_dev, SL.w64, sizeof(double) * n, cudaMemcpyHostToDevice, s);
    if (!e) e = (int)cudaMemcpyAsync(SL.elig_dev, SL.elig, (size_t)SL.nev, cudaMemcpyHostToDevice, s);
    if (fk_check(e, "locate: FP64 observation upload")) return 1;
    SL.dirty64 = false;
    return 0;
}

static int pack_tables(void)
{
    if (!SL.tables_dirty && SL.bpack) return 0;
    if (!SL.bpack) {
        SL.bpack = fk_dalloc(fk_locate_tc_table_bytes(SL.ngrd), "locate: table pack");
        if (!SL.bpack) return 1;
    }
    int e = fk_locate_tc_pack_tables(SL.ngrd, SL.ldgrd, SL.ntf, SL.tables, SL.bpack, fk_stream());
    if (fk_check(e, "locate: table pack")) return 1;
    SL.tables_dirty = false;
    return 0;
}

static int ensure_tc(int n, int npart)
{
    if (!SL.err_dev) {
        SL.err_dev = (int *)fk_dalloc(sizeof(int), "locate");
        if (!SL.err_dev) return 1;
    }
    const size_t ab = fk_locate_tc_event_bytes(n);
    if (ab > SL.apack_bytes) {
        fk_dfree(SL.apack);
        SL.apack = fk_dalloc(ab, "locate: event pack");
        SL.apack_bytes = SL.apack ? ab : 0;
        if (!SL.apack) return 1;
    }
    const size_t nc = (size_t)n * npart * FK_TC_TOPK;
    if (nc > SL.cand_n) {
        fk_dfree(SL.cand_v); fk_dfree(SL.cand_i);
        SL.cand_v = (float *)fk_dalloc(sizeof(float) * nc, "locate: candidates");
        SL.cand_i = (int *)fk_dalloc(sizeof(int) * nc, "locate: candidates");
        SL.cand_n = (SL.cand_v && SL.cand_i) ? nc : 0;
        if (!SL.cand_n) return 1;
    }
    if (n > SL.tc_cap) {
        fk_dfree(SL.tc_idx); fk_dfree(SL.tc_t0); fk_dfree(SL.tc_obj);
        SL.tc_idx = (int *)fk_dalloc(sizeof(int) * (size_t)n, "locate");
        SL.tc_t0 = (double *)fk_dalloc(sizeof(double) * (size_t)n, "locate");
        SL.tc_obj = (double *)fk_dalloc(sizeof(double) * (size_t)n, "locate");
        SL.tc_cap = (SL.tc_idx && SL.tc_t0 && SL.tc_obj) ? n : 0;
        if (!SL.tc_cap) return 1;
    }
    return 0;
}

/* Tensor-core search of events [e0, e0+n); ineligible events of the range
 * go through the exact search.  t0 excludes tepoch. */
static int locate_range_tc(int e0, int n, int *idx, double *t0, double *obj)
{
    const int npart = fk_locate_tc_npart(n, SL.ngrd);
    if (pack_tables() || upload_obs64() || ensure_tc(n, npart)) return 1;
    cudaStream_t s = fk_stream();
    int e = (int)cudaMemsetAsync(SL.err_dev, 0, sizeof(int), s);
    if (!e)
        e = fk_locate_tc(SL.ngrd, SL.ldgrd, SL.ntf, SL.tables, SL.bpack, n,
                         SL.obs64_dev + (size_t)e0 * SL.ntf, SL.w64_dev + (size_t)e0 * SL.ntf,
                         SL.elig_dev + e0, SL.apack, npart, SL.cand_v, SL.cand_i, SL.rescore,
                         SL.tc_idx, SL.tc_t0, SL.tc_obj, SL.err_dev, SL.dbg_dev, s);
    int kerr = 0;
    if (!e) e = (int)cudaMemcpyAsync(idx, SL.tc_idx, sizeof(int) * (size_t)n, cudaMemcpyDeviceToHost, s);
    if (!e) e = (int)cudaMemcpyAsync(t0, SL.tc_t0, sizeof(double) * (size_t)n, cudaMemcpyDeviceToHost, s);
    if (!e) e = (int)cudaMemcpyAsync(obj, SL.tc_obj, sizeof(double) * (size_t)n, cudaMemcpyDeviceToHost, s);
    if (!e) e = (int)cudaMemcpyAsync(&kerr, SL.err_dev, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (!e) e = (int)cudaStreamSynchronize(s);
    if (fk_check(e, "locate (tensor core)")) return 1;
    if (kerr) {
        FK_ERR("locate (tensor core): pipeline wait timed out (code %d)", kerr);
        return 1;
    }
    for (int i = 0; i < n; i++) {
        if (SL.elig[e0 + i]) continue;
        int ix;
        float ft0, fobj;
        if (locate_range(e0 + i, 1, &ix, &ft0, &fobj)) return 1;
        idx[i] = ix;
        t0[i] = (double)ft0;
        obj[i] = (double)fobj;
    }
    return 0;
}

void fteik_b200_locate_setMethod(int method, int *ierr)
{
    *ierr = 0;
    if (method < 0 || method > 2) {
        FK_ERR("fteik_b200_locate_setMethod: method=%d must be 0 (exact FP32), 1 (tensor core) or 2 (surrogate-pruned)", method);
        *ierr = 1;
        return;
    }
    SL.method = method;
}

void fk_locate_tc_set_products(int n);
int fk_locate_tc_get_products(void);

void fteik_b200_locate_setRankingProducts(int nprod, int *ierr)
{
    *ierr = 0;
    if (nprod != 2 && nprod != 3) {
        FK_ERR("fteik_b200_locate_setRankingProducts: nprod=%d must be 2 or 3", nprod);
        *ierr = 1;
        return;
    }
    fk_locate_tc_set_products(nprod);
}

void fteik_b200_locate_getRankingProducts(int *nprod) { *nprod = fk_locate_tc_get_products(); }

void fteik_b200_locate_setRescoreCandidates(int ncand, int *ierr)
{
    *ierr = 0;
    if (ncand < 1 || ncand > 256) {
        FK_ERR("fteik_b200_locate_setRescoreCandidates: ncand=%d must be in [1,256] (runs of 32 grid points)", ncand);
        *ierr = 1;
        return;
    }
    if (!SL.init) { FK_ERR("fteik_b200_locate_setRescoreCandidates: Locator not initialized"); *ierr = 1; return; }
    SL.rescore = ncand;
}

void fteik_b200_locate_debugAccumulators(int enable, float *out, int *ierr)
{
    /* enable = 1 before a tensor-core locate makes its CTA 0 record the first
     * accumulator tile pair (256 events x 128 grid points); enable = 0 copies
     * it to out (32768 floats, may be NULL) and stops recording */
    *ierr = 0;
    if (!SL.init) { FK_ERR("fteik_b200_locate_debugAccumulators: Locator not initialized"); *ierr = 1; return; }
    if (enable) {
        if (!SL.dbg_dev) SL.dbg_dev = (float *)fk_dalloc(sizeof(float) * 256 * 128, "locate: debug");
        if (!SL.dbg_dev) { *ierr = 1; return; }
        return;
    }
    if (SL.dbg_dev && out) {
        int e = (int)fk_d2h(out, SL.dbg_dev, sizeof(float) * 256 * 128);
        if (fk_check(e, "fteik_b200_locate_debugAccumulators")) *ierr = 1;
    }
    fk_dfree(SL.dbg_dev);
    SL.dbg_dev = NULL;
}

/* Events [e0, e0+n) with the selected method; t0 excludes tepoch. */
static int locate_range_pruned(int e0, int n, int *idx, double *t0, double *obj);

/* L1 search of events [e0, e0+n); t0 excludes tepoch. */
static int locate_range_l1(int e0, int n, int *idx, double *t0, double *obj)
{
    for (int i = 0; i < n; i++)
        if (!SL.l1ok[e0 + i]) {
            FK_ERR("locate (L1): event %d has picks of different weights", e0 + i + 1);
            return 1;
        }
    if (upload_obs() || upload_obs64()) return 1;
    if (n > SL.l1_cap) {
        fk_dfree(SL.l1_idx); fk_dfree(SL.l1_t0); fk_dfree(SL.l1_obj); fk_dfree(SL.l1_best);
        SL.l1_idx = (int *)fk_dalloc(sizeof(int) * (size_t)n, "locate");
        SL.l1_t0 = (double *)fk_dalloc(sizeof(double) * (size_t)n, "locate");
        SL.l1_obj = (double *)fk_dalloc(sizeof(double) * (size_t)n, "locate");
        SL.l1_best = (unsigned long long *)fk_dalloc(sizeof(unsigned long long) * (size_t)n, "locate");
        SL.l1_cap = (SL.l1_idx && SL.l1_t0 && SL.l1_obj && SL.l1_best) ? n : 0;
        if (!SL.l1_cap) return 1;
    }
    cudaStream_t s = fk_stream();
    int e = fk_locate_l1_exact(SL.ngrd, SL.ldgrd, SL.ntf, SL.tables, n, SL.obs_dev + (size_t)e0 * SL.ntf,
                               SL.wts_dev + (size_t)e0 * SL.ntf, SL.obs64_dev + (size_t)e0 * SL.ntf,
                               SL.w64_dev + (size_t)e0 * SL.ntf, SL.l1_idx, SL.l1_t0, SL.l1_obj, SL.l1_best, s);
    if (!e) e = (int)cudaMemcpyAsync(idx, SL.l1_idx, sizeof(int) * (size_t)n, cudaMemcpyDeviceToHost, s);
    if (!e) e = (int)cudaMemcpyAsync(t0, SL.l1_t0, sizeof(double) * (size_t)n, cudaMemcpyDeviceToHost, s);
    if (!e) e = (int)cudaMemcpyAsync(obj, SL.l1_obj, sizeof(double) * (size_t)n, cudaMemcpyDeviceToHost, s);
    if (!e) e = (int)cudaStreamSynchronize(s);
    return fk_check(e, "locate (L1)");
}

void fteik_b200_locate_setNorm(int norm, int *ierr)
{
    *ierr = 0;
    if (norm != 1 && norm != 2) {
        FK_ERR("fteik_b200_locate_setNorm: norm=%d must be 1 or 2", norm);
        *ierr = 1;
        return;
    }
    SL.norm = norm;
}

static int locate_any(int e0, int n, int *idx, double *t0, double *obj)
{
    if (SL.norm == 1) return locate_range_l1(e0, n, idx, t0, obj);
    if (SL.method == 1) return locate_range_tc(e0, n, idx, t0, obj);
    if (SL.method == 2) return locate_range_pruned(e0, n, idx, t0, obj);
    float *ft0 = (float *)malloc(sizeof(float) * (size_t)n);
    float *fobj = (float *)malloc(sizeof(float) * (size_t)n);
    int rc = locate_range(e0, n, idx, ft0, fobj);
    for (int i = 0; i < n && !rc; i++) { t0[i] = (double)ft0[i]; obj[i] = (double)fobj[i]; }
    free(ft0);
    free(fobj);
    return rc;
}

void locate_locateEvent(int evnmbr, int *optIndx, double *t0Opt, double *objOpt)
{
    /* locate.F90:112-126.  The origin-time work array is reset for every
     * event (the reference keeps accumulating it, locate.F90:641-690). */
    *optIndx = 0;
    *t0Opt = 0.0;
    *objOpt = 0.0;
    if (!SL.init || evnmbr < 1 || evnmbr > SL.nev) {
        FK_ERR("locate_locateEvent: invalid event %d or locator not initialized", evnmbr);
        return;
    }
    int idx;
    double t0, obj;
    if (locate_any(evnmbr - 1, 1, &idx, &t0, &obj)) return;
    *optIndx = idx + 1;
    *t0Opt = t0 + SL.tepoch[evnmbr - 1];
    *objOpt = obj;
}

void fteik_b200_locate_locateEvents(int n, const int ev[], int optIndx[], double t0Opt[],
                                    double objOpt[], int *ierr)
{
    *ierr = 0;
    if (!SL.init) { FK_ERR("fteik_b200_locate_locateEvents: Locator not initialized"); *ierr = 1; return; }
    if (n < 1) return;
    /* contiguous runs of events go to the device in one launch each */
    int *idx = (int *)malloc(sizeof(int) * (size_t)n);
    int i = 0;
    while (i < n && !*ierr) {
        if (ev[i] < 1 || ev[i] > SL.nev) { FK_ERR("fteik_b200_locate_locateEvents: event %d out of range", ev[i]); *ierr = 1; break; }
        int j = i + 1;
        while (j < n && ev[j] == ev[j - 1] + 1) j++;
        if (locate_any(ev[i] - 1, j - i, idx + i, t0Opt + i, objOpt + i)) { *ierr = 1; break; }
        i = j;
    }
    if (!*ierr)
        for (int k = 0; k < n; k++) {
            optIndx[k] = idx[k] + 1;
            t0Opt[k] += SL.tepoch[ev[k] - 1];
        }
    free(idx);
}

/* ------------------------------------------------------------------------ */
/* Surrogate-pruned search (method 2).                                      */
/* ------------------------------------------------------------------------ */

void fteik_b200_locate_setGeometry(int nz, int nx, int ny, double dz, double dx, double dy, int ntf,
                                   const double zsta[], const double xsta[], const double ysta[],
                                   int *ierr)
{
    const char *who = "fteik_b200_locate_setGeometry";
    *ierr = 1;
    if (!SL.init) { FK_ERR("%s: Locator not initialized", who); return; }
    if (nz < 2 || nx < 2 || ny < 2 || (long long)nz * nx * ny != SL.ngrd) {
        FK_ERR("%s: nz*nx*ny must equal ngrd=%d", who, SL.ngrd);
        return;
    }
    if (ntf != SL.ntf || dz <= 0.0 || dx <= 0.0 || dy <= 0.0) { FK_ERR("%s: need ntf=%d and positive spacing", who, SL.ntf); return; }
    float *h = (float *)malloc(sizeof(float) * 3 * (size_t)ntf);
    for (int i = 0; i < ntf; i++) {
        h[3 * i] = (float)zsta[i];
        h[3 * i + 1] = (float)xsta[i];
        h[3 * i + 2] = (float)ysta[i];
    }
    fk_dfree(SP.sta_dev);
    SP.sta_dev = (float *)fk_dalloc(sizeof(float) * 3 * (size_t)ntf, who);
    int e = SP.sta_dev ? (int)fk_h2d(SP.sta_dev, h, sizeof(float) * 3 * (size_t)ntf) : 1;
    free(h);
    if (fk_check(e, who)) return;
    SP.nz = nz; SP.nx = nx; SP.ny = ny;
    SP.dz = dz; SP.dx = dx; SP.dy = dy;
    SP.have_geom = true;
    SP.ready = false;
    if (SP.rc == 0) { SP.rc = 4; SP.k = 8; }
    *ierr = 0;
}

typedef struct {
    unsigned long long seed;
    long long nsamp;
} table_batch_t;

static int table_batch(void *ctx, long long step, const long long *step_dev, int B, float *x, float *y,
                       cudaStream_t s)
{
    table_batch_t *c = (table_batch_t *)ctx;
    return fk_mlp_sample(SP.nz, SP.nx, SP.ny, SP.dz, SP.dx, SP.dy, SL.ntf, SL.ldgrd, SP.vref, SL.tables,
                         SP.sta_dev, c->seed, c->nsamp, step, step_dev, B, x, y, s);
}

void fteik_b200_locate_trainSurrogate(long long nsamples, int steps, int batch, double lr, double vref,
                                      unsigned long long seed, double *loss, int *ierr)
{
    /* Trains the surrogate network (fteik_b200_mlp_*; initialised here with
     * 5 x 256 units when absent) on nsamples (table, grid node) pairs of the
     * locator's tables, target tau = T v_ref / distance. */
    const char *who = "fteik_b200_locate_trainSurrogate";
    *ierr = 1;
    *loss = 0.0;
    if (!SL.init || !SP.have_geom) { FK_ERR("%s: set the locator geometry first", who); return; }
    if (nsamples < 1 || steps < 1 || batch < 1 || lr <= 0.0 || vref <= 0.0) { FK_ERR("%s: bad arguments", who); return; }
    if (!fk_mlp_ready()) {
        int e2;
        fteik_b200_mlp_initialize(256, 5, seed, &e2);
        if (e2) return;
    }
    SP.vref = vref;
    table_batch_t c;
    c.seed = seed;
    c.nsamp = nsamples;
    if (fk_mlp_train_device(table_batch, &c, 1, steps, batch, lr, loss)) return;
    SP.ready = false;
    *ierr = 0;
}

void fteik_b200_locate_buildSurrogate(int bz, int bx, int by, int *ierr)
{
    /* Surrogate travel times at the centres of the coarse blocks (bz x bx x
     * by fine nodes each), ranked by the tensor-core search in method 2. */
    const char *who = "fteik_b200_locate_buildSurrogate";
    *ierr = 1;
    if (!SL.init || !SP.have_geom || !fk_mlp_ready() || SP.vref <= 0.0) {
        FK_ERR("%s: needs the locator geometry and a trained surrogate", who);
        return;
    }
    if (bz < 1 || bx < 1 || by < 1 || bz > 32 || bx > 32 || by > 32 || bz * bx * by > 1024 ||
        bz * bx * by < 2) {
        FK_ERR("%s: block %dx%dx%d: each side in [1,32], 2 to 1024 nodes", who, bz, bx, by);
        return;
    }
    SP.bz = bz;
    SP.bx = bx;
    SP.by = by;
    SP.ncz = (SP.nz + bz - 1) / bz;
    SP.ncx = (SP.nx + bx - 1) / bx;
    SP.ncy = (SP.ny + by - 1) / by;
    SP.ngrd_c = SP.ncz * SP.ncx * SP.ncy;
    SP.ldc = (SP.ngrd_c + 15) / 16 * 16;
    /* a rebuild of the same shape reuses every buffer */
    const size_t ncoarse = (size_t)SL.ntf * SP.ldc, nbpack = fk_locate_tc_table_bytes(SP.ngrd_c);
    if (ncoarse != SP.coarse_cap || !SP.coarse) {
        fk_dfree(SP.coarse);
        SP.coarse = (float *)fk_dalloc(sizeof(float) * ncoarse, who);
        SP.coarse_cap = SP.coarse ? ncoarse : 0;
    }
    if (nbpack != SP.bpack_cap || !SP.bpack_c) {
        fk_dfree(SP.bpack_c);
        SP.bpack_c = fk_dalloc(nbpack, who);
        SP.bpack_cap = SP.bpack_c ? nbpack : 0;
    }
    const long long nrow = (long long)SL.ntf * SP.ngrd_c;
    const long long chunk = 1 << 18;
    if (!SP.bx_in) SP.bx_in = (float *)fk_dalloc(sizeof(float) * 6 * (size_t)chunk, who);
    if (!SP.bx_dist) SP.bx_dist = (float *)fk_dalloc(sizeof(float) * (size_t)chunk, who);
    if (!SP.bx_tau) SP.bx_tau = (float *)fk_dalloc(sizeof(float) * (size_t)chunk, who);
    float *x = SP.bx_in, *dist = SP.bx_dist, *tau = SP.bx_tau;
    int e = (SP.coarse && SP.bpack_c && x && dist && tau) ? 0 : 1;
    cudaStream_t s = fk_stream();
    if (!e) e = (int)cudaMemsetAsync(SP.coarse, 0, sizeof(float) * (size_t)SL.ntf * SP.ldc, s);
    for (long long r0 = 0; r0 < nrow && !e; r0 += chunk) {
        const long long m = nrow - r0 < chunk ? nrow - r0 : chunk;
        e = fk_mlp_coarse_inputs(SP.nz, SP.nx, SP.ny, SP.dz, SP.dx, SP.dy, SL.ntf, SP.vref, SP.sta_dev, bz, bx,
                                 by, SP.ncz, SP.ncx, SP.ncy, r0, m, x, dist, s);
        if (!e) e = fk_mlp_forward_device(m, x, tau, s);
        if (!e) e = fk_mlp_coarse_store(r0, m, SP.ngrd_c, SP.ldc, tau, dist, SP.coarse, s);
    }
    if (!e) e = fk_locate_tc_pack_tables(SP.ngrd_c, SP.ldc, SL.ntf, SP.coarse, SP.bpack_c, s);
    /* node-major block copy: each node's tables padded to a multiple of 4 */
    const size_t nfine = (size_t)SP.ngrd_c * (size_t)((SL.ntf + 3) & ~3) * (size_t)(bz * bx * by);
    if (nfine != SP.fine_cap) {   /* a rebuild of the same blocks reuses the copy's memory */
        fk_dfree(SP.fine_blk);
        SP.fine_blk = (float *)fk_dalloc(sizeof(float) * nfine, who);
        SP.fine_cap = SP.fine_blk ? nfine : 0;
    }
    if (!SP.fine_blk) e = 1;
    /* the block copy depends on the exact tables and the block shape only:
     * a rebuild for a retrained network keeps it */
    const bool blk_fresh = SP.blk_gen == SL.table_gen && SP.blk_shape[0] == bz && SP.blk_shape[1] == bx &&
                           SP.blk_shape[2] == by;
    if (!e && !blk_fresh)
        e = fk_locate_block_tables(SP.nz, SP.nx, SP.ny, bz, bx, by, SL.ntf, SL.ldgrd, SL.tables, SP.fine_blk, s);
    if (!e) e = (int)cudaStreamSynchronize(s);
    if (!e) {
        SP.blk_shape[0] = bz;
        SP.blk_shape[1] = bx;
        SP.blk_shape[2] = by;
        SP.blk_gen = SL.table_gen;
    } else {
        SP.blk_shape[0] = 0;   /* the copy is not known to be complete */
    }
    if (fk_check(e, who)) return;
    SP.ready = true;
    *ierr = 0;
}

void fteik_b200_locate_setPruning(int ncoarse_runs, int ncoarse_nodes, int *ierr)
{
    *ierr = 1;
    if (ncoarse_runs < 1 || ncoarse_runs > 4 || ncoarse_nodes < 1 || ncoarse_nodes > 32) {
        FK_ERR("fteik_b200_locate_setPruning: need 1 <= runs <= 4 and 1 <= nodes <= 32");
        return;
    }
    SP.rc = ncoarse_runs;
    SP.k = ncoarse_nodes;
    *ierr = 0;
}

void fteik_b200_locate_getPruneInfo(int *nfallback, int *ncoarse, long long *nblocks, int *maxblocks, int *ierr)
{
    *maxblocks = SP.last_max_blocks;
    *nfallback = SP.last_fallback;
    *ncoarse = SP.ready ? SP.ngrd_c : 0;
    *nblocks = SP.last_blocks;
    *ierr = 0;
}

void fteik_b200_locate_getSurrogateTable(int itf, int n, float out[], int *ierr)
{
    /* coarse surrogate travel times of table itf (coarse nodes z fastest) */
    *ierr = 1;
    if (!SP.ready || itf < 1 || itf > SL.ntf || n < SP.ngrd_c) { FK_ERR("fteik_b200_locate_getSurrogateTable: not built or bad arguments"); return; }
    *ierr = fk_check(fk_d2h(out, SP.coarse + (size_t)(itf - 1) * SP.ldc, sizeof(float) * (size_t)SP.ngrd_c),
                     "fteik_b200_locate_getSurrogateTable");
}

/* Exhaustive tensor-core search of the events evs[0..m-1] (0-based). */
static int locate_tc_subset(const int *evs, int m, int *idx, double *t0, double *obj)
{
    if (m > SP.sub_cap) {
        fk_dfree(SP.sub_obs); fk_dfree(SP.sub_w); fk_dfree(SP.sub_elig);
        SP.sub_obs = (double *)fk_dalloc(sizeof(double) * (size_t)m * SL.ntf, "locate");
        SP.sub_w = (double *)fk_dalloc(sizeof(double) * (size_t)m * SL.ntf, "locate");
        SP.sub_elig = (unsigned char *)fk_dalloc((size_t)m, "locate");
        SP.sub_cap = (SP.sub_obs && SP.sub_w && SP.sub_elig) ? m : 0;
        if (!SP.sub_cap) return 1;
    }
    const size_t nt = (size_t)SL.ntf;
    double *ho = (double *)malloc(sizeof(double) * (size_t)m * nt);
    double *hw = (double *)malloc(sizeof(double) * (size_t)m * nt);
    unsigned char *he = (unsigned char *)malloc((size_t)m);
    for (int i = 0; i < m; i++) {
        memcpy(ho + i * nt, SL.obs64 + (size_t)evs[i] * nt, sizeof(double) * nt);
        memcpy(hw + i * nt, SL.w64 + (size_t)evs[i] * nt, sizeof(double) * nt);
        he[i] = 1;
    }
    const int npart = fk_locate_tc_npart(m, SL.ngrd);
    int e = pack_tables() || ensure_tc(m, npart);
    cudaStream_t s = fk_stream();
    int kerr = 0;
    if (!e) e = (int)cudaMemcpyAsync(SP.sub_obs, ho, sizeof(double) * (size_t)m * nt, cudaMemcpyHostToDevice, s);
    if (!e) e = (int)cudaMemcpyAsync(SP.sub_w, hw, sizeof(double) * (size_t)m * nt, cudaMemcpyHostToDevice, s);
    if (!e) e = (int)cudaMemcpyAsync(SP.sub_elig, he, (size_t)m, cudaMemcpyHostToDevice, s);
    if (!e) e = (int)cudaMemsetAsync(SL.err_dev, 0, sizeof(int), s);
    if (!e)
        e = fk_locate_tc(SL.ngrd, SL.ldgrd, SL.ntf, SL.tables, SL.bpack, m, SP.sub_obs, SP.sub_w, SP.sub_elig,
                         SL.apack, npart, SL.cand_v, SL.cand_i, SL.rescore, SL.tc_idx, SL.tc_t0, SL.tc_obj,
                         SL.err_dev, NULL, s);
    if (!e) e = (int)cudaMemcpyAsync(idx, SL.tc_idx, sizeof(int) * (size_t)m, cudaMemcpyDeviceToHost, s);
    if (!e) e = (int)cudaMemcpyAsync(t0, SL.tc_t0, sizeof(double) * (size_t)m, cudaMemcpyDeviceToHost, s);
    if (!e) e = (int)cudaMemcpyAsync(obj, SL.tc_obj, sizeof(double) * (size_t)m, cudaMemcpyDeviceToHost, s);
    if (!e) e = (int)cudaMemcpyAsync(&kerr, SL.err_dev, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (!e) e = (int)cudaStreamSynchronize(s);
    free(ho); free(hw); free(he);
    if (fk_check(e, "locate (fallback search)")) return 1;
    if (kerr) { FK_ERR("locate (fallback search): pipeline wait timed out (code %d)", kerr); return 1; }
    return 0;
}

static int locate_range_pruned(int e0, int n, int *idx, double *t0, double *obj)
{
    if (!SP.ready) { FK_ERR("locate (surrogate-pruned): build the surrogate first"); return 1; }
    if (SP.blk_gen != SL.table_gen) {
        /* the exact tables changed since the block-major copy was made */
        int eb = fk_locate_block_tables(SP.nz, SP.nx, SP.ny, SP.bz, SP.bx, SP.by, SL.ntf, SL.ldgrd, SL.tables,
                                        SP.fine_blk, fk_stream());
        if (fk_check(eb, "locate (surrogate-pruned): block copy")) return 1;
        SP.blk_gen = SL.table_gen;
        SP.blk_shape[0] = SP.bz;
        SP.blk_shape[1] = SP.bx;
        SP.blk_shape[2] = SP.by;
    }
    const int npart = fk_locate_tc_npart(n, SP.ngrd_c);
    if (upload_obs64() || ensure_tc(n, npart)) return 1;
    if (n > SP.flag_cap) {
        fk_dfree(SP.flag_dev);
        SP.flag_dev = (unsigned char *)fk_dalloc((size_t)n, "locate");
        SP.flag_cap = SP.flag_dev ? n : 0;
        if (!SP.flag_dev) return 1;
    }
    cudaStream_t s = fk_stream();
    unsigned char *flag = (unsigned char *)malloc((size_t)n);
    int kerr = 0;
    if (SP.timing && !SP.ev[0])
        for (int k = 0; k < 4; k++) cudaEventCreate(&SP.ev[k]);
    int e = (int)cudaMemsetAsync(SL.err_dev, 0, sizeof(int), s);
    if (!e && SP.timing) e = (int)cudaEventRecord(SP.ev[0], s);
    if (!e)
        e = fk_locate_tc(SP.ngrd_c, SP.ldc, SL.ntf, SP.coarse, SP.bpack_c, n, SL.obs64_dev + (size_t)e0 * SL.ntf,
                         SL.w64_dev + (size_t)e0 * SL.ntf, SL.elig_dev + e0, SL.apack, npart, SL.cand_v,
                         SL.cand_i, 0, NULL, NULL, NULL, SL.err_dev, NULL, s);
    if (!e && SP.timing) e = (int)cudaEventRecord(SP.ev[1], s);
    if (!e)
        e = fk_locate_prune(n, npart, SP.rc, SP.k, SP.nz, SP.nx, SP.ny, SP.bz, SP.bx, SP.by, SL.ldgrd, SP.ldc, SL.ntf,
                            SP.coarse, SP.fine_blk, SL.obs64_dev + (size_t)e0 * SL.ntf,
                            SL.w64_dev + (size_t)e0 * SL.ntf, SL.elig_dev + e0, SL.cand_v, SL.cand_i,
                            SL.tc_idx, SL.tc_t0, SL.tc_obj, SP.flag_dev, s);
    if (!e && SP.timing) e = (int)cudaEventRecord(SP.ev[2], s);
    if (!e) e = (int)cudaMemcpyAsync(idx, SL.tc_idx, sizeof(int) * (size_t)n, cudaMemcpyDeviceToHost, s);
    if (!e) e = (int)cudaMemcpyAsync(t0, SL.tc_t0, sizeof(double) * (size_t)n, cudaMemcpyDeviceToHost, s);
    if (!e) e = (int)cudaMemcpyAsync(obj, SL.tc_obj, sizeof(double) * (size_t)n, cudaMemcpyDeviceToHost, s);
    if (!e) e = (int)cudaMemcpyAsync(flag, SP.flag_dev, (size_t)n, cudaMemcpyDeviceToHost, s);
    if (!e) e = (int)cudaMemcpyAsync(&kerr, SL.err_dev, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (!e && SP.timing) e = (int)cudaEventRecord(SP.ev[3], s);
    if (!e) e = (int)cudaStreamSynchronize(s);
    if (!e && SP.timing)
        for (int k = 0; k < 3; k++) cudaEventElapsedTime(&SP.stage_ms[k], SP.ev[k], SP.ev[k + 1]);
    if (fk_check(e, "locate (surrogate-pruned)") || kerr) {
        if (kerr) FK_ERR("locate (surrogate-pruned): pipeline wait timed out (code %d)", kerr);
        free(flag);
        return 1;
    }
    /* events whose pruned optimum lies on an unexamined block face: the
     * exhaustive tensor-core search decides them */
    int *fb = (int *)malloc(sizeof(int) * (size_t)n);
    int m = 0;
    SP.last_blocks = 0;
    SP.last_max_blocks = 0;
    for (int i = 0; i < n; i++) {
        if (!SL.elig[e0 + i]) continue;
        if (flag[i] == 0xFF) fb[m++] = e0 + i;
        else {
            SP.last_blocks += flag[i];
            if (flag[i] > SP.last_max_blocks) SP.last_max_blocks = flag[i];
        }
    }
    int rc = 0;
    SP.last_fallback = m;
    if (m > 0) {
        int *fi = (int *)malloc(sizeof(int) * (size_t)m);
        double *ft = (double *)malloc(sizeof(double) * (size_t)m);
        double *fo = (double *)malloc(sizeof(double) * (size_t)m);
        rc = locate_tc_subset(fb, m, fi, ft, fo);
        for (int j = 0; j < m && !rc; j++) {
            idx[fb[j] - e0] = fi[j];
            t0[fb[j] - e0] = ft[j];
            obj[fb[j] - e0] = fo[j];
        }
        free(fi); free(ft); free(fo);
    }
    free(fb);
    free(flag);
    for (int i = 0; i < n && !rc; i++) {
        if (SL.elig[e0 + i]) continue;
        int ix;
        float ft0, fobj;
        if (locate_range(e0 + i, 1, &ix, &ft0, &fobj)) return 1;
        idx[i] = ix;
        t0[i] = (double)ft0;
        obj[i] = (double)fobj;
    }
    return rc;
}

void fteik_b200_locate_setStageTiming(int enable, int *ierr)
{
    SP.timing = enable != 0;
    *ierr = 0;
}

void fteik_b200_locate_getStageTimes(float *coarse_ms, float *prune_ms, float *copy_ms, int *ierr)
{
    *coarse_ms = SP.stage_ms[0];
    *prune_ms = SP.stage_ms[1];
    *copy_ms = SP.stage_ms[2];
    *ierr = SP.timing ? 0 : 1;
}
