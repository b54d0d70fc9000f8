/*
 * mlp.c -- the travel-time surrogate network (host side): parameters,
 * forward / backward passes and Adam on the device through the kernels of
 * mlp.cu.  No counterpart in the reference.
 *
 * Network: 6 inputs -> depth hidden layers of width units (SiLU) -> 1 output
 * tau; the travel time it predicts is tau * distance / v_ref.  Parameters are
 * one FP32 vector: for each linear layer l, W_l [out][in] then b_l [out].
 */
#include "host_common.h"
#include "fteik_b200.h"

#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

int fk_mlp_gemm(int M, int N, int K, const float *A, int lda, int ta, const float *B, int ldb,
                int tb, float *C, int ldc, const float *bias, int accumulate, float *C2, int act, float *colsum,
                cudaStream_t s);
int fk_mlp_mse(int n, const float *pred, const float *y, float *dpred, double *loss, cudaStream_t s);
int fk_mlp_adam_sched(size_t n, float *w, const float *g, float *m, float *v, const float *sched,
                      const long long *tdev, float b1, float b2, float eps, cudaStream_t s);
int fk_mlp_step_inc(long long *tdev, cudaStream_t s);
int fk_mlp_transpose_layers(int n, const long long *off, const int *in, const int *out, const float *w, float *wt,
                            cudaStream_t s);
int fk_mlp_adam(size_t n, float *w, const float *g, float *m, float *v, float lr, float b1,
                float b2, float eps, float c1, float c2, cudaStream_t s);
void fk_mlp_set_tensor(int products);
int fk_mlp_get_tensor(void);
int fk_mlp_tc_status(cudaStream_t s);
int *fk_mlp_tc_error_word(cudaStream_t s);
void fk_mlp_set_async_staging(int on);
int fk_mlp_forward_fused(const float *w, int nh, const long long *woff, const long long *boff, long long n,
                         const float *x, float *tau, unsigned char *wq, int *error, cudaStream_t s);

void fteik_b200_mlp_setTensorProducts(int products, int *ierr)
{
    *ierr = 0;
    if (products != 0 && products != 1 && products != 3) {
        FK_ERR("fteik_b200_mlp_setTensorProducts: products must be 0, 1 or 3");
        *ierr = 1;
        return;
    }
    fk_mlp_set_tensor(products);
}

void fteik_b200_mlp_getTensorProducts(int *products) { *products = fk_mlp_get_tensor(); }

/* 0, or the CUDA error / tensor-core wait timeout of the work queued so far */
static int tc_check(int e, const char *who)
{
    if (!e) {
        const int st = fk_mlp_tc_status(fk_stream());
        if (st) {
            FK_ERR("%s: a tensor-core GEMM gave up waiting (%d)", who, st);
            return 1;
        }
    }
    return fk_check(e, who);
}

#define MLP_IN 6
#define MLP_MAXL 16

static struct {
    bool init;
    int width, depth, nlayer;          /* nlayer = depth + 1 linear maps */
    int din[MLP_MAXL], dout[MLP_MAXL];
    size_t woff[MLP_MAXL], boff[MLP_MAXL], nparam;
    float *w, *g, *m, *v;              /* device [nparam] */
    float *wt;                         /* device [nparam]: transposed hidden weights (backward pass) */
    long long adam_t;
    int cap;                           /* batch rows the buffers hold */
    float *x[MLP_MAXL + 1];            /* layer inputs; x[nlayer] = output */
    float *z[MLP_MAXL];                /* pre-activations */
    float *dz, *dtmp;                  /* backward scratch [cap][width] */
    double *loss_dev;
} NN;

static void mlp_free_buffers(void)
{
    for (int l = 0; l <= MLP_MAXL; l++) { fk_dfree(NN.x[l]); NN.x[l] = NULL; }
    for (int l = 0; l < MLP_MAXL; l++) { fk_dfree(NN.z[l]); NN.z[l] = NULL; }
    fk_dfree(NN.dz); fk_dfree(NN.dtmp);
    NN.dz = NN.dtmp = NULL;
    NN.cap = 0;
}

static int g_fused = 1;
static unsigned char *g_wq = NULL;   /* packed BF16 weights of the fused forward pass */
static size_t g_wq_cap = 0;

void fteik_b200_mlp_finalize(void)
{
    mlp_free_buffers();
    fk_dfree(g_wq);
    g_wq = NULL;
    g_wq_cap = 0;
    fk_dfree(NN.w); fk_dfree(NN.g); fk_dfree(NN.m); fk_dfree(NN.v); fk_dfree(NN.wt); fk_dfree(NN.loss_dev);
    memset(&NN, 0, sizeof(NN));
}

static uint64_t splitmix(uint64_t *s)
{
    uint64_t z = (*s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

static double uniform01(uint64_t *s) { return (double)(splitmix(s) >> 11) * (1.0 / 9007199254740992.0); }

void fteik_b200_mlp_initialize(int width, int depth, unsigned long long seed, int *ierr)
{
    *ierr = 1;
    fteik_b200_mlp_finalize();
    if (width < 1 || width > 4096 || depth < 1 || depth > MLP_MAXL - 1) {
        FK_ERR("fteik_b200_mlp_initialize: width=%d depth=%d out of range", width, depth);
        return;
    }
    if (fk_dev_ready("fteik_b200_mlp_initialize")) return;
    NN.width = width;
    NN.depth = depth;
    NN.nlayer = depth + 1;
    size_t off = 0;
    for (int l = 0; l < NN.nlayer; l++) {
        NN.din[l] = l == 0 ? MLP_IN : width;
        NN.dout[l] = l == NN.nlayer - 1 ? 1 : width;
        NN.woff[l] = off;
        off += (size_t)NN.din[l] * NN.dout[l];
        NN.boff[l] = off;
        off += (size_t)NN.dout[l];
    }
    NN.nparam = off;
    /* uniform(-a, a) with a = sqrt(3 / fan_in) (unit-variance preactivations
     * for unit-variance inputs); output layer small, bias 1 (tau ~ 1) */
    float *h = (float *)calloc(off, sizeof(float));
    uint64_t st = (uint64_t)seed;
    for (int l = 0; l < NN.nlayer; l++) {
        double a = sqrt(3.0 / NN.din[l]);
        if (l == NN.nlayer - 1) a *= 0.1;
        for (size_t k = 0; k < (size_t)NN.din[l] * NN.dout[l]; k++)
            h[NN.woff[l] + k] = (float)((2.0 * uniform01(&st) - 1.0) * a);
        for (int k = 0; k < NN.dout[l]; k++) h[NN.boff[l] + k] = l == NN.nlayer - 1 ? 1.0f : 0.0f;
    }
    NN.w = (float *)fk_dalloc(sizeof(float) * off, "mlp");
    NN.g = (float *)fk_dalloc(sizeof(float) * off, "mlp");
    NN.m = (float *)fk_dalloc(sizeof(float) * off, "mlp");
    NN.v = (float *)fk_dalloc(sizeof(float) * off, "mlp");
    NN.wt = (float *)fk_dalloc(sizeof(float) * off, "mlp");
    NN.loss_dev = (double *)fk_dalloc(sizeof(double), "mlp");
    int e = (NN.w && NN.g && NN.m && NN.v && NN.wt && NN.loss_dev) ? 0 : 1;
    if (!e) e = (int)fk_h2d(NN.w, h, sizeof(float) * off);
    if (!e) e = (int)fk_zero(NN.m, sizeof(float) * off);
    if (!e) e = (int)fk_zero(NN.v, sizeof(float) * off);
    free(h);
    if (fk_check(e, "fteik_b200_mlp_initialize")) return;
    NN.init = true;
    *ierr = 0;
}

void fteik_b200_mlp_getNumberOfWeights(int *n, int *ierr)
{
    *n = NN.init ? (int)NN.nparam : 0;
    *ierr = NN.init ? 0 : 1;
}

void fteik_b200_mlp_getWeights(int n, float w[], int *ierr)
{
    *ierr = 1;
    if (!NN.init || n < (int)NN.nparam) { FK_ERR("fteik_b200_mlp_getWeights: not initialized or n too small"); return; }
    *ierr = fk_check((int)fk_d2h(w, NN.w, sizeof(float) * NN.nparam),
                     "fteik_b200_mlp_getWeights");
}

void fteik_b200_mlp_setWeights(int n, const float w[], int *ierr)
{
    *ierr = 1;
    if (!NN.init || n != (int)NN.nparam) { FK_ERR("fteik_b200_mlp_setWeights: not initialized or n /= %zu", NN.nparam); return; }
    *ierr = fk_check((int)fk_h2d(NN.w, w, sizeof(float) * NN.nparam),
                     "fteik_b200_mlp_setWeights");
    NN.adam_t = 0;
    fk_zero(NN.m, sizeof(float) * NN.nparam);
    fk_zero(NN.v, sizeof(float) * NN.nparam);
}

static int ensure_batch(int B)
{
    if (B <= NN.cap) return 0;
    mlp_free_buffers();
    int ok = 1;
    for (int l = 0; l <= NN.nlayer; l++) {
        const int d = l < NN.nlayer ? NN.din[l] : 1;
        NN.x[l] = (float *)fk_dalloc(sizeof(float) * (size_t)B * d, "mlp");
        ok &= NN.x[l] != NULL;
    }
    for (int l = 0; l < NN.nlayer; l++) {
        NN.z[l] = (float *)fk_dalloc(sizeof(float) * (size_t)B * NN.dout[l], "mlp");
        ok &= NN.z[l] != NULL;
    }
    const size_t wd = (size_t)B * (NN.width > MLP_IN ? NN.width : MLP_IN);
    NN.dz = (float *)fk_dalloc(sizeof(float) * wd, "mlp");
    NN.dtmp = (float *)fk_dalloc(sizeof(float) * wd, "mlp");
    ok &= NN.dz && NN.dtmp;
    if (!ok) { mlp_free_buffers(); return 1; }
    NN.cap = B;
    return 0;
}

/* Forward pass of B rows already in NN.x[0]; the output lands in
 * NN.x[nlayer] (B values).  The SiLU is applied in the GEMM's epilogue;
 * training (keep_z) also keeps the pre-activations NN.z for the backward
 * pass. */
static int forward(int B, bool keep_z, cudaStream_t s)
{
    int e = 0;
    for (int l = 0; l < NN.nlayer && !e; l++) {
        const int in = NN.din[l], out = NN.dout[l];
        const bool last = l == NN.nlayer - 1;
        if (last)
            e = fk_mlp_gemm(B, out, in, NN.x[l], in, 0, NN.w + NN.woff[l], in, 1, NN.x[l + 1], out,
                            NN.w + NN.boff[l], 0, NULL, 0, NULL, s);
        else if (keep_z)
            e = fk_mlp_gemm(B, out, in, NN.x[l], in, 0, NN.w + NN.woff[l], in, 1, NN.z[l], out,
                            NN.w + NN.boff[l], 0, NN.x[l + 1], 1, NULL, s);
        else
            e = fk_mlp_gemm(B, out, in, NN.x[l], in, 0, NN.w + NN.woff[l], in, 1, NN.x[l + 1], out,
                            NN.w + NN.boff[l], 0, NULL, 2, NULL, s);
    }
    return e;
}

/* Loss and gradient (into NN.g) of B rows with targets y (device). */
static int forward_backward(int B, const float *y, cudaStream_t s)
{
    int e = forward(B, true, s);
    const int L = NN.nlayer;
    /* the input-gradient products of the layers with more than 8 outputs
     * read W^T (k-contiguous rows), transposed once per pass */
    long long toff[MLP_MAXL];
    int tin[MLP_MAXL], tout[MLP_MAXL], nt = 0;
    bool trans[MLP_MAXL] = {false};
    for (int l = 1; l < L; l++)
        if (NN.dout[l] > 8) {
            toff[nt] = (long long)NN.woff[l];
            tin[nt] = NN.din[l];
            tout[nt] = NN.dout[l];
            trans[l] = true;
            nt++;
        }
    if (!e) e = fk_mlp_transpose_layers(nt, toff, tin, tout, NN.w, NN.wt, s);
    /* d loss / d output */
    if (!e) e = fk_mlp_mse(B, NN.x[L], y, NN.dz, NN.loss_dev, s);
    for (int l = L - 1; l >= 0 && !e; l--) {
        const int in = NN.din[l], out = NN.dout[l];
        /* NN.dz holds d loss / d z_l  [B][out]: dW_l = dz^T x_l, and the
         * bias gradient (the column sums of dz) from the same pass */
        e = fk_mlp_gemm(out, in, B, NN.dz, out, 1, NN.x[l], in, 0, NN.g + NN.woff[l], in, NULL, 0, NULL, 0,
                        NN.g + NN.boff[l], s);
        if (!e && l > 0) {
            /* d loss / d z_{l-1} = (dz W_l) silu'(z_{l-1}), the derivative
             * applied in the product's epilogue */
            if (trans[l])
                e = fk_mlp_gemm(B, in, out, NN.dz, out, 0, NN.wt + NN.woff[l], out, 1, NN.dtmp, in, NULL, 0,
                                NN.z[l - 1], 3, NULL, s);
            else
                e = fk_mlp_gemm(B, in, out, NN.dz, out, 0, NN.w + NN.woff[l], in, 0, NN.dtmp, in, NULL, 0,
                                NN.z[l - 1], 3, NULL, s);
            if (!e) { float *t = NN.dz; NN.dz = NN.dtmp; NN.dtmp = t; }
        }
    }
    return e;
}

static int fused_ok(long long n);
static int forward_fused(long long n, const float *x, float *tau, cudaStream_t s);

void fteik_b200_mlp_forward(int n, const float x[], float tau[], int *ierr)
{
    /* x [n][6] normalised inputs, host; tau [n] host */
    *ierr = 1;
    if (!NN.init || n < 1) { FK_ERR("fteik_b200_mlp_forward: not initialized or n < 1"); return; }
    cudaStream_t s = fk_stream();
    const int chunk = 65536;
    for (int r0 = 0; r0 < n; r0 += chunk) {
        const int B = n - r0 < chunk ? n - r0 : chunk;
        if (ensure_batch(B)) return;
        int e = (int)cudaMemcpyAsync(NN.x[0], x + (size_t)r0 * MLP_IN, sizeof(float) * (size_t)B * MLP_IN,
                                     cudaMemcpyHostToDevice, s);
        if (!e) e = fused_ok(B) ? forward_fused(B, NN.x[0], NN.x[NN.nlayer], s) : forward(B, false, s);
        if (!e) e = (int)cudaMemcpyAsync(tau + r0, NN.x[NN.nlayer], sizeof(float) * (size_t)B,
                                         cudaMemcpyDeviceToHost, s);
        if (!e) e = (int)cudaStreamSynchronize(s);
        if (tc_check(e, "fteik_b200_mlp_forward")) return;
    }
    *ierr = 0;
}

void fteik_b200_mlp_gradient(int n, const float x[], const float y[], double *loss, float grad[],
                             int *ierr)
{
    /* mean squared error of n rows and its gradient (nparam floats) */
    *ierr = 1;
    *loss = 0.0;
    if (!NN.init || n < 1) { FK_ERR("fteik_b200_mlp_gradient: not initialized or n < 1"); return; }
    if (ensure_batch(n)) return;
    cudaStream_t s = fk_stream();
    float *ydev = (float *)fk_dalloc(sizeof(float) * (size_t)n, "mlp");
    if (!ydev) return;
    int e = (int)cudaMemcpyAsync(NN.x[0], x, sizeof(float) * (size_t)n * MLP_IN, cudaMemcpyHostToDevice, s);
    if (!e) e = (int)cudaMemcpyAsync(ydev, y, sizeof(float) * (size_t)n, cudaMemcpyHostToDevice, s);
    if (!e) e = forward_backward(n, ydev, s);
    if (!e) e = (int)cudaMemcpyAsync(grad, NN.g, sizeof(float) * NN.nparam, cudaMemcpyDeviceToHost, s);
    if (!e) e = (int)cudaMemcpyAsync(loss, NN.loss_dev, sizeof(double), cudaMemcpyDeviceToHost, s);
    if (!e) e = (int)cudaStreamSynchronize(s);
    fk_dfree(ydev);
    *ierr = tc_check(e, "fteik_b200_mlp_gradient");
}

/* Adam steps over batches produced by next_batch (device x / y).  The
 * learning rate decays by a cosine from lr to lr / 100.
 *
 * With a capturable batch function one training step (batch, forward,
 * backward, Adam, step counter) is captured in a CUDA graph after one eager
 * step and replayed: the step number, learning rate and bias corrections
 * come from device memory (the schedule computed on the host as the eager
 * loop does), so the replayed steps are the eager loop's, bit for bit, at a
 * graph launch per step instead of ~40 kernel launches.  The last 20 steps
 * read the loss back. */
static int adam_constants(long long t_adam, long long t, long long steps, double lr, float *lrt, float *c1,
                          float *c2)
{
    const float b1 = 0.9f, b2 = 0.999f;
    const double frac = (double)t / (double)steps;
    *lrt = (float)(lr * (0.01 + 0.99 * 0.5 * (1.0 + cos(3.141592653589793 * frac))));
    *c1 = (float)(1.0 - pow(b1, (double)t_adam));
    *c2 = (float)(1.0 - pow(b2, (double)t_adam));
    return 0;
}

static int train_step_dev(fk_batch_fn next_batch, void *ctx, int B, float *ydev, const float *sched,
                          long long *tdev, cudaStream_t s)
{
    int e = next_batch(ctx, 0, tdev, B, NN.x[0], ydev, s);
    if (!e) e = forward_backward(B, ydev, s);
    if (!e) e = fk_mlp_adam_sched(NN.nparam, NN.w, NN.g, NN.m, NN.v, sched, tdev, 0.9f, 0.999f, 1e-8f, s);
    if (!e) e = fk_mlp_step_inc(tdev, s);
    return e;
}

static int train_graph(fk_batch_fn next_batch, void *ctx, long long steps, int B, double lr, float *ydev,
                       double *lsum, long long *lcount)
{
    cudaStream_t s = fk_stream();
    float *sched_h = (float *)malloc(sizeof(float) * 3 * (size_t)steps);
    float *sched = (float *)fk_dalloc(sizeof(float) * 3 * (size_t)steps, "mlp");
    long long *tdev = (long long *)fk_dalloc(sizeof(long long), "mlp");
    int e = (sched_h && sched && tdev) ? 0 : 1;
    for (long long t = 0; t < steps && !e; t++)
        adam_constants(NN.adam_t + 1 + t, t, steps, lr, sched_h + 3 * t, sched_h + 3 * t + 1, sched_h + 3 * t + 2);
    if (!e) e = (int)fk_h2d(sched, sched_h, sizeof(float) * 3 * (size_t)steps);
    if (!e) e = (int)cudaMemsetAsync(tdev, 0, sizeof(long long), s);
    /* step 0 eagerly: every buffer a step uses exists before the capture */
    if (!e) e = train_step_dev(next_batch, ctx, B, ydev, sched, tdev, s);
    cudaGraph_t graph = NULL;
    cudaGraphExec_t exec = NULL;
    if (!e) e = (int)cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
    if (!e) {
        const int le = train_step_dev(next_batch, ctx, B, ydev, sched, tdev, s);
        e = (int)cudaStreamEndCapture(s, &graph);
        if (!e) e = le;
    }
    if (!e) e = (int)cudaGraphInstantiate(&exec, graph, 0);
    for (long long t = 1; t < steps && !e; t++) {
        e = (int)cudaGraphLaunch(exec, s);
        if (!e && t >= steps - 20) {
            double l = 0.0;
            e = (int)cudaMemcpyAsync(&l, NN.loss_dev, sizeof(double), cudaMemcpyDeviceToHost, s);
            if (!e) e = (int)cudaStreamSynchronize(s);
            *lsum += l;
            (*lcount)++;
        }
    }
    if (!e) e = (int)cudaStreamSynchronize(s);
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    NN.adam_t += steps;
    fk_dfree(tdev);
    fk_dfree(sched);
    free(sched_h);
    return e;
}

static int g_train_graph = 1;

void fteik_b200_mlp_setTrainGraph(int on) { g_train_graph = on != 0; }
void fteik_b200_mlp_getTrainGraph(int *on) { *on = g_train_graph; }

int fk_mlp_train_device(fk_batch_fn next_batch, void *ctx, int capturable, long long steps, int B, double lr,
                        double *last_loss)
{
    if (!NN.init || steps < 1 || B < 1) return 1;
    if (ensure_batch(B)) return 1;
    cudaStream_t s = fk_stream();
    float *ydev = (float *)fk_dalloc(sizeof(float) * (size_t)B, "mlp");
    if (!ydev) return 1;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    int e = 0;
    double lsum = 0.0;
    long long lcount = 0;
    if (capturable && g_train_graph && steps > 21) {
        e = train_graph(next_batch, ctx, steps, B, lr, ydev, &lsum, &lcount);
    } else {
        for (long long t = 0; t < steps && !e; t++) {
            e = next_batch(ctx, t, NULL, B, NN.x[0], ydev, s);
            if (!e) e = forward_backward(B, ydev, s);
            NN.adam_t++;
            float lrt, c1, c2;
            adam_constants(NN.adam_t, t, steps, lr, &lrt, &c1, &c2);
            if (!e) e = fk_mlp_adam(NN.nparam, NN.w, NN.g, NN.m, NN.v, lrt, b1, b2, eps, c1, c2, s);
            if (!e && t >= steps - 20) {
                double l = 0.0;
                e = (int)cudaMemcpyAsync(&l, NN.loss_dev, sizeof(double), cudaMemcpyDeviceToHost, s);
                if (!e) e = (int)cudaStreamSynchronize(s);
                lsum += l;
                lcount++;
            }
        }
    }
    fk_dfree(ydev);
    if (last_loss) *last_loss = lcount ? lsum / (double)lcount : 0.0;
    return tc_check(e, "mlp training");
}

typedef struct {
    const float *x, *y;   /* device [n][6], [n] */
    long long n;
    unsigned long long seed;
} host_data_t;

static int host_batch(void *ctx, long long step, const long long *step_dev, int B, float *x, float *y,
                      cudaStream_t s)
{
    (void)step_dev;   /* not capturable: the windows are placed by the host */
    /* contiguous windows of a fixed permutation-free ring over the rows */
    host_data_t *d = (host_data_t *)ctx;
    long long start = (step * (long long)B) % d->n;
    int e = 0;
    int done = 0;
    while (done < B && !e) {
        long long take = d->n - start;
        if (take > B - done) take = B - done;
        e = (int)cudaMemcpyAsync(x + (size_t)done * MLP_IN, d->x + (size_t)start * MLP_IN,
                                 sizeof(float) * (size_t)take * MLP_IN, cudaMemcpyDeviceToDevice, s);
        if (!e) e = (int)cudaMemcpyAsync(y + done, d->y + start, sizeof(float) * (size_t)take,
                                         cudaMemcpyDeviceToDevice, s);
        done += (int)take;
        start = 0;
    }
    return e;
}

void fteik_b200_mlp_train(int n, const float x[], const float y[], int steps, int batch, double lr,
                          double *loss, int *ierr)
{
    /* Adam on host data (x [n][6] normalised inputs, y [n] targets tau),
     * batches taken in order around the data */
    *ierr = 1;
    *loss = 0.0;
    if (!NN.init || n < 1 || steps < 1 || batch < 1) { FK_ERR("fteik_b200_mlp_train: bad arguments or not initialized"); return; }
    host_data_t d;
    d.n = n;
    d.seed = 0;
    float *xd = (float *)fk_dalloc(sizeof(float) * (size_t)n * MLP_IN, "mlp");
    float *yd = (float *)fk_dalloc(sizeof(float) * (size_t)n, "mlp");
    if (!xd || !yd) { fk_dfree(xd); fk_dfree(yd); return; }
    int e = (int)fk_h2d(xd, x, sizeof(float) * (size_t)n * MLP_IN);
    if (!e) e = (int)fk_h2d(yd, y, sizeof(float) * (size_t)n);
    d.x = xd;
    d.y = yd;
    if (!fk_check(e, "fteik_b200_mlp_train"))
        *ierr = fk_mlp_train_device(host_batch, &d, 0, steps, batch, lr, loss);
    fk_dfree(xd);
    fk_dfree(yd);
}

/* Inference on device rows (x [n][6] device) into tau (device). */
void fteik_b200_mlp_setFusedForward(int on) { g_fused = on != 0; }
void fteik_b200_mlp_getFusedForward(int *on) { *on = g_fused; }

static int g_async_staging = 1;
void fteik_b200_mlp_setAsyncStaging(int on)
{
    g_async_staging = on != 0;
    fk_mlp_set_async_staging(g_async_staging);
}
void fteik_b200_mlp_getAsyncStaging(int *on) { *on = g_async_staging; }

/* The fused forward pass applies: BF16 products, width 256, 1 to 8 hidden
 * layers, at least one full 128-row tile. */
static int fused_ok(long long n)
{
    const int nh = NN.nlayer - 2;
    return g_fused && fk_mlp_get_tensor() == 1 && NN.width == 256 && nh >= 1 && nh <= 8 && n >= 128;
}

static int forward_fused(long long n, const float *x, float *tau, cudaStream_t s)
{
    const int nh = NN.nlayer - 2;
    const size_t need = (size_t)nh * 256 * 256 * 2;
    if (need > g_wq_cap) {
        fk_dfree(g_wq);
        g_wq = (unsigned char *)fk_dalloc(need, "mlp");
        g_wq_cap = g_wq ? need : 0;
        if (!g_wq) return 1;
    }
    int *err = fk_mlp_tc_error_word(s);
    if (!err) return 1;
    long long woff[10], boff[10];
    for (int l = 0; l < nh + 2; l++) { woff[l] = (long long)NN.woff[l]; boff[l] = (long long)NN.boff[l]; }
    return fk_mlp_forward_fused(NN.w, nh, woff, boff, n, x, tau, g_wq, err, s);
}

int fk_mlp_forward_device(long long n, const float *x, float *tau, cudaStream_t s)
{
    if (!NN.init) return 1;
    if (fused_ok(n)) return forward_fused(n, x, tau, s);
    const int chunk = 65536;
    int e = 0;
    for (long long r0 = 0; r0 < n && !e; r0 += chunk) {
        const int B = (int)(n - r0 < chunk ? n - r0 : chunk);
        if (ensure_batch(B)) return 1;
        e = (int)cudaMemcpyAsync(NN.x[0], x + (size_t)r0 * MLP_IN, sizeof(float) * (size_t)B * MLP_IN,
                                 cudaMemcpyDeviceToDevice, s);
        if (!e) e = forward(B, false, s);
        if (!e) e = (int)cudaMemcpyAsync(tau + r0, NN.x[NN.nlayer], sizeof(float) * (size_t)B,
                                         cudaMemcpyDeviceToDevice, s);
    }
    return e;
}

int fk_mlp_ready(void) { return NN.init ? 1 : 0; }
size_t fk_mlp_flops_per_row(void)
{
    size_t f = 0;
    for (int l = 0; l < NN.nlayer; l++) f += 2 * (size_t)NN.din[l] * NN.dout[l];
    return f;
}
