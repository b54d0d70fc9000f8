/*
 * slab3d_common.cuh -- launch parameters and small kernels shared by the
 * slab-pipelined 3D sweeps (row3d_impl.cuh): the field initialisation, the
 * analytic source corners, the per-work-item results, and the acquire /
 * release accessors of the slab progress counters.
 */
#pragma once
#include "stencil3d.cuh"

namespace fk3tw {
using fk3::Mesh;
using fk3::Src;

struct Params {
    const fk_grid3d_t *grids;
    const fk_work3d_t *work;
    const int2 *tasks;          /* one sweep's tasks: {work or pair, logical slab j'} in j' order */
    const int *done_base;       /* per work item: first slab's index in done[] */
    int ntask_sweep;
    int s_begin, s_end;         /* global sweep numbers: 0..7 init, 8.. Gauss-Seidel */
    int *done;                  /* per slab: (sweep << 20) | steps done */
    int *done_t;                /* per work item, turned-axes initialisation tasks (or NULL) */
    unsigned long long *ticket;
    int *error;                 /* 0 ok; else the first failure */
    unsigned long long *resid;  /* [nwork][npass]: FP64 max |dt| bits */
    int *pass_slabs;            /* [nwork][npass]: slabs done with the pass's last sweep */
    int *conv_pass;             /* [nwork]: first converged pass, or a large value */
    int npass;
    int converge;
    double eps, conv_tol;
    long long spin_limit;
};

__device__ __forceinline__ int ld_acquire(const int *p)
{
    int v;
    asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_release(int *p, int v)
{
    asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

template <typename R>
__device__ __forceinline__ R ldcg(const R *p) { return __ldcg(p); }

__device__ __forceinline__ void tw_setup_src(Src &q, const fk_work3d_t &w, const fk_grid3d_t &g,
                                          double eps)
{
    q.zsi = w.zsi; q.xsi = w.xsi; q.ysi = w.ysi;
    q.zsa = w.zsa; q.xsa = w.xsa; q.ysa = w.ysa;
    q.szero = w.szero; q.szero2 = w.szero * w.szero;
    double hmin = g.dz < g.dx ? g.dz : g.dx;
    hmin = g.dy < hmin ? g.dy : hmin;
    q.eps_t = eps * hmin * w.szero; /* localSolver.F90:906 */
}

/* Field initialisation of every work item (solver3D.F90:1201-1202) and the
 * analytic source corners (localSolver.F90:933-956, FP64). */
template <typename R>
__global__ void field_init_kernel(const fk_grid3d_t *__restrict__ grids,
                                  const fk_work3d_t *__restrict__ work, double eps)
{
    const fk_work3d_t w = work[blockIdx.y];
    const fk_grid3d_t g = grids[w.grid];
    R *tt = reinterpret_cast<R *>(w.tt);
    const size_t n = (size_t)g.ny * g.nx * g.zp;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n;
         e += (size_t)gridDim.x * blockDim.x)
        tt[e] = (R)FK_HUGE;
}

template <typename R>
__global__ void corners_kernel(const fk_grid3d_t *__restrict__ grids,
                               const fk_work3d_t *__restrict__ work, int nwork, double eps)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nwork * 8) return;
    const fk_work3d_t w = work[i / 8];
    const fk_grid3d_t g = grids[w.grid];
    Src q;
    tw_setup_src(q, w, g, eps);
    Mesh<double> m64;
    fk3::make_mesh<double>(m64, g.dz, g.dx, g.dy);
    const int c = i % 8, di = c & 1, dj = (c >> 1) & 1, dk = (c >> 2) & 1;
    const double t = fk3::tana<double>(q, m64, q.zsi + di, q.xsi + dj, q.ysi + dk);
    R *tt = reinterpret_cast<R *>(w.tt);
    tt[((size_t)(q.ysi - 1 + dk) * g.nx + (q.xsi - 1 + dj)) * g.zp + (q.zsi - 1 + di)] = (R)t;
}

/* Per-work-item results from the pass bookkeeping. */
static __global__ void finalize_kernel(int nwork, int npass, int converge, int nsweep,
                                       const unsigned long long *__restrict__ resid,
                                       const int *__restrict__ conv_pass, const int *__restrict__ error,
                                       fk_result3d_t *__restrict__ results)
{
    const int w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= nwork) return;
    int ran = converge ? min(conv_pass[w] + 1, npass) : nsweep;
    if (ran < 0) ran = 0;
    results[w].npass = ran;
    results[w].residual = (ran > 0) ? __longlong_as_double((long long)resid[(size_t)w * npass + ran - 1]) : 0.0;
    results[w].status = *error;
}

extern cudaEvent_t *g_slab_events; /* sweep3d_f32.cu */

} // namespace fk3tw
