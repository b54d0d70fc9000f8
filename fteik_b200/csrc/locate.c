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
} SL;

void locate_finalize(void)
{
    free(SL.tepoch); free(SL.origin); free(SL.have_ot); free(SL.obs); free(SL.wts);
    fk_dfree(SL.tables); fk_dfree(SL.obs_dev); fk_dfree(SL.wts_dev);
    fk_dfree(SL.idx_dev); fk_dfree(SL.t0_dev); fk_dfree(SL.obj_dev); fk_dfree(SL.scratch);
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
    if (!SL.tables || !SL.obs_dev || !SL.wts_dev) { *ierr = 1; return; }
    if (fk_check((int)cudaMemset(SL.tables, 0, sizeof(float) * (size_t)ntf * SL.ldgrd),
                 "locate_initialize")) { *ierr = 1; return; }
    SL.init = true;
    SL.dirty = true;
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
    *ierr = fk_check(e, "locate_setTravelTimeField32f");
}

/* Device table row of table itf (1-based), for the in-library hand-off. */
float *fk_locate_table_row(int itf, int ngrd)
{
    if (!SL.init || itf < 1 || itf > SL.ntf || ngrd != SL.ngrd) return NULL;
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
    memset(o, 0, sizeof(float) * SL.ntf);
    memset(w, 0, sizeof(float) * SL.ntf);
    for (int i = 0; i < nttimes; i++) {
        int k = obs2tf[i] - 1;
        if (wts[i] > 0.0) {
            o[k] = (float)(pickTimes[i] - tep); /* reduced time */
            w[k] = (float)wts[i];
        }
    }
    SL.dirty = true;
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
    float t0, obj;
    if (locate_range(evnmbr - 1, 1, &idx, &t0, &obj)) return;
    *optIndx = idx + 1;
    *t0Opt = (double)t0 + SL.tepoch[evnmbr - 1];
    *objOpt = (double)obj;
}

void fteik_b200_locate_locateEvents(int n, const int ev[], int optIndx[], double t0Opt[],
                                    double objOpt[], int *ierr)
{
    *ierr = 0;
    if (!SL.init) { FK_ERR("fteik_b200_locate_locateEvents: Locator not initialized"); *ierr = 1; return; }
    if (n < 1) return;
    /* contiguous runs of events go to the device in one launch each */
    int *idx = (int *)malloc(sizeof(int) * (size_t)n);
    float *t0 = (float *)malloc(sizeof(float) * (size_t)n);
    float *obj = (float *)malloc(sizeof(float) * (size_t)n);
    int i = 0;
    while (i < n && !*ierr) {
        if (ev[i] < 1 || ev[i] > SL.nev) { FK_ERR("fteik_b200_locate_locateEvents: event %d out of range", ev[i]); *ierr = 1; break; }
        int j = i + 1;
        while (j < n && ev[j] == ev[j - 1] + 1) j++;
        if (locate_range(ev[i] - 1, j - i, idx + i, t0 + i, obj + i)) { *ierr = 1; break; }
        i = j;
    }
    if (!*ierr)
        for (int k = 0; k < n; k++) {
            optIndx[k] = idx[k] + 1;
            t0Opt[k] = (double)t0[k] + SL.tepoch[ev[k] - 1];
            objOpt[k] = (double)obj[k];
        }
    free(idx); free(t0); free(obj);
}
