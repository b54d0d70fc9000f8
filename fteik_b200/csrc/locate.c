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
    int rescore;             /* candidates re-scored in FP64 per event */
    bool dirty64, tables_dirty;
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

void locate_finalize(void)
{
    free(SL.tepoch); free(SL.origin); free(SL.have_ot); free(SL.obs); free(SL.wts);
    fk_dfree(SL.tables); fk_dfree(SL.obs_dev); fk_dfree(SL.wts_dev);
    fk_dfree(SL.idx_dev); fk_dfree(SL.t0_dev); fk_dfree(SL.obj_dev); fk_dfree(SL.scratch);
    free(SL.obs64); free(SL.w64); free(SL.elig);
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
    if (!SL.tables || !SL.obs_dev || !SL.wts_dev) { *ierr = 1; return; }
    if (fk_check((int)cudaMemset(SL.tables, 0, sizeof(float) * (size_t)ntf * SL.ldgrd),
                 "locate_initialize")) { *ierr = 1; return; }
    SL.init = true;
    SL.dirty = true;
    SL.dirty64 = true;
    SL.tables_dirty = true;
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
    *ierr = fk_check(e, "locate_setTravelTimeField32f");
}

/* Device table row of table itf (1-based), for the in-library hand-off. */
float *fk_locate_table_row(int itf, int ngrd)
{
    if (!SL.init || itf < 1 || itf > SL.ntf || ngrd != SL.ngrd) return NULL;
    SL.tables_dirty = true; /* the caller writes the row */
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
        SL.err_dev = (int *)fk_dalloc(sizeof(int), "locate: table pack");
        if (!SL.bpack || !SL.err_dev) return 1;
    }
    int e = fk_locate_tc_pack_tables(SL.ngrd, SL.ldgrd, SL.ntf, SL.tables, SL.bpack, fk_stream());
    if (fk_check(e, "locate: table pack")) return 1;
    SL.tables_dirty = false;
    return 0;
}

static int ensure_tc(int n, int npart)
{
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
    if (method != 0 && method != 1) {
        FK_ERR("fteik_b200_locate_setMethod: method=%d must be 0 (exact FP32) or 1 (tensor core)", method);
        *ierr = 1;
        return;
    }
    SL.method = method;
}

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
        int e = (int)cudaMemcpy(out, SL.dbg_dev, sizeof(float) * 256 * 128, cudaMemcpyDeviceToHost);
        if (fk_check(e, "fteik_b200_locate_debugAccumulators")) *ierr = 1;
    }
    fk_dfree(SL.dbg_dev);
    SL.dbg_dev = NULL;
}

/* Events [e0, e0+n) with the selected method; t0 excludes tepoch. */
static int locate_any(int e0, int n, int *idx, double *t0, double *obj)
{
    if (SL.method == 1) return locate_range_tc(e0, n, idx, t0, obj);
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
