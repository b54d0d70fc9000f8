/*
 * stencil3d.cuh -- the 3D node updates of the reference's local solver
 * (localSolver.F90:384-959) for the CUDA sweep kernels, templated on the
 * working precision.  Every expression keeps the reference's operand order.
 */
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "fteik_dev.h"

namespace fk3 {

constexpr int kMaxWarps = 32;

template <typename R>
struct Mesh {
    R dz, dx, dy;
    R dz2i, dx2i, dy2i, dsum_nine, dsumi, dz2dx2, dz2dy2, dx2dy2;
    R dz2i_dx2i, dz2i_dy2i, dx2i_dy2i;
    R dz2i_p_dx2i, dz2i_p_dy2i, dx2i_p_dy2i;
    R dz2i_p_dx2i_inv, dz2i_p_dy2i_inv, dx2i_p_dy2i_inv;
};

/* localSolver.F90:905-931: the mesh constants, derived in FP64 and rounded
 * once to the working precision. */
template <typename R>
__device__ void make_mesh(Mesh<R> &m, double dz, double dx, double dy)
{
    double dz2 = dz * dz, dx2 = dx * dx, dy2 = dy * dy;
    double dz2i = 1.0 / dz2, dx2i = 1.0 / dx2, dy2i = 1.0 / dy2;
    double dsum = dz2i + dx2i + dy2i;
    m.dz = (R)dz; m.dx = (R)dx; m.dy = (R)dy;
    m.dz2i = (R)dz2i; m.dx2i = (R)dx2i; m.dy2i = (R)dy2i;
    m.dsum_nine = (R)(dsum * 9.0);
    m.dsumi = (R)(1.0 / dsum);
    m.dz2dx2 = (R)(1.0 / (dz2 * dx2));
    m.dz2dy2 = (R)(1.0 / (dz2 * dy2));
    m.dx2dy2 = (R)(1.0 / (dx2 * dy2));
    m.dz2i_dx2i = (R)(dz2i * dx2i);
    m.dz2i_dy2i = (R)(dz2i * dy2i);
    m.dx2i_dy2i = (R)(dx2i * dy2i);
    m.dz2i_p_dx2i = (R)(dz2i + dx2i);
    m.dz2i_p_dy2i = (R)(dz2i + dy2i);
    m.dx2i_p_dy2i = (R)(dx2i + dy2i);
    m.dz2i_p_dx2i_inv = (R)(1.0 / (dz2i + dx2i));
    m.dz2i_p_dy2i_inv = (R)(1.0 / (dz2i + dy2i));
    m.dx2i_p_dy2i_inv = (R)(1.0 / (dx2i + dy2i));
}

/* FP32 square root: the hardware approximation (relative error of order
 * 2^-23), far inside the FP32 path's 1e-4 tolerance; FP64 stays IEEE. */
__device__ __forceinline__ float rsqrt_(float x)
{
    float r;
    asm("sqrt.approx.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ double rsqrt_(double x) { return sqrt(x); }
template <typename R> __device__ __forceinline__ R rmin(R a, R b) { return (b < a) ? b : a; }
template <typename R> __device__ __forceinline__ R rmax(R a, R b) { return (b > a) ? b : a; }

/* localSolver.F90:384-534, one node; tupd enters as the node's time.
 * Evaluated without branches: every candidate is computed and the ones the
 * reference's conditions admit are selected, so the result is the
 * reference's (a candidate whose condition fails may be NaN from the root
 * of a negative number; the selects never take it). */
template <typename R>
__device__ __forceinline__ R noinit(const Mesh<R> &c, R tv, R te, R tn, R tev,
                                    R ten, R tnv, R tnve, R s1, R s2, R s3,
                                    R s4, R s5, R s6, R s7, R tupd);

/* Lane-wise arithmetic on one value (float) or on the values of two sources
 * of one grid (float2, one sm_100 instruction for both).  Every operation is
 * rounded once, so the float and float2 forms give identical bits. */
__device__ __forceinline__ float vadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float vsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float vmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float vfma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
template <typename V> __device__ __forceinline__ V vbc(float a);
template <> __device__ __forceinline__ float vbc<float>(float a) { return a; }
__device__ __forceinline__ float vget(float v, int) { return v; }
__device__ __forceinline__ void vset(float &v, int, float x) { v = x; }
__device__ __forceinline__ float2 vadd(float2 a, float2 b) { return __fadd2_rn(a, b); }
/* a - b as (-1) b + a: the product is exact, the sum rounded once */
__device__ __forceinline__ float2 vsub(float2 a, float2 b) { return __ffma2_rn(b, make_float2(-1.0f, -1.0f), a); }
__device__ __forceinline__ float2 vmul(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 vfma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
template <> __device__ __forceinline__ float2 vbc<float2>(float a) { return make_float2(a, a); }
__device__ __forceinline__ float vget(float2 v, int i) { return i ? v.y : v.x; }
__device__ __forceinline__ void vset(float2 &v, int i, float x) { if (i) v.y = x; else v.x = x; }

/* FP32 form of localSolver.F90:384-534 for V = float (one source) or float2
 * (two sources of one grid, which share the slowness s1..s7), held to the
 * FP64 result within 1e-4 rather than bit for bit, in fewer operations:
 * with d = te - tv etc. the plane operator is
 *   t = tev + d (dx2i - dz2i)/B + (2/B) sqrt(s^2 B - C d^2),
 *   B = dz2i + dx2i, C = dz2i dx2i,
 * and the 3D operator's differences are ta - tb = 1.5 (te - tv + ten - tnv),
 * tb - tc = 1.5 (tv - tn + tev - ten), t1 / dsum = tb + ((ta - tb) dx2i -
 * (tb - tc) dy2i) / dsum.  Every candidate is computed and the ones the
 * reference's conditions admit are selected (a rejected one may be NaN). */
template <typename V>
__device__ __forceinline__ V noinit_v(const Mesh<float> &c, V tv, V te, V tn, V tev, V ten, V tnv, V tnve,
                                      float s1, float s2, float s3, float s4, float s5, float s6, float s7, V tupd)
{
    constexpr int N = sizeof(V) / sizeof(float);
    const float HUGEV = (float)FK_HUGE;
    const V t1z = vfma(vbc<V>(c.dz), vbc<V>(s1), tv), t1x = vfma(vbc<V>(c.dx), vbc<V>(s2), te),
            t1y = vfma(vbc<V>(c.dy), vbc<V>(s3), tn);
    const V temtv = vsub(te, tv), tvmtn = vsub(tv, tn), temtn = vsub(te, tn);
    /* plane operators: q = s^2 B - C d^2, t = 2/B sqrt(q) + (d k + t_corner) */
    const V q_zx = vfma(vbc<V>(s4 * s4), vbc<V>(c.dz2i_p_dx2i), vmul(vbc<V>(-c.dz2i_dx2i), vmul(temtv, temtv)));
    const V q_zy = vfma(vbc<V>(s5 * s5), vbc<V>(c.dz2i_p_dy2i), vmul(vbc<V>(-c.dz2i_dy2i), vmul(tvmtn, tvmtn)));
    const V q_xy = vfma(vbc<V>(s6 * s6), vbc<V>(c.dx2i_p_dy2i), vmul(vbc<V>(-c.dx2i_dy2i), vmul(temtn, temtn)));
    const V b_zx = vfma(temtv, vbc<V>((c.dx2i - c.dz2i) * c.dz2i_p_dx2i_inv), tev);
    const V b_zy = vfma(tvmtn, vbc<V>((c.dz2i - c.dy2i) * c.dz2i_p_dy2i_inv), tnv);
    const V b_xy = vfma(temtn, vbc<V>((c.dx2i - c.dy2i) * c.dx2i_p_dy2i_inv), ten);
    V r_zx, r_zy, r_xy;
#pragma unroll
    for (int i = 0; i < N; ++i) {
        vset(r_zx, i, rsqrt_(vget(q_zx, i)));
        vset(r_zy, i, rsqrt_(vget(q_zy, i)));
        vset(r_xy, i, rsqrt_(vget(q_xy, i)));
    }
    const V t_zx = vfma(vbc<V>(2.0f * c.dz2i_p_dx2i_inv), r_zx, b_zx);
    const V t_zy = vfma(vbc<V>(2.0f * c.dz2i_p_dy2i_inv), r_zy, b_zy);
    const V t_xy = vfma(vbc<V>(2.0f * c.dx2i_p_dy2i_inv), r_xy, b_xy);
    /* 3D operator: ta - tb = 1.5 (te - tv + ten - tnv), tb - tc = 1.5 (tv - tn + tev - ten) */
    const V tab = vmul(vadd(temtv, vsub(ten, tnv)), vbc<V>(1.5f));
    const V tbc = vmul(vadd(tvmtn, vsub(tev, ten)), vbc<V>(1.5f));
    const V tac = vadd(tab, tbc);
    const V tb = vadd(vsub(vfma(vadd(vsub(tnv, tn), vsub(tev, te)), vbc<V>(0.5f), tv), ten), tnve);
    const float t2 = (s7 * s7) * c.dsum_nine;
    const V t3 = vfma(vbc<V>(c.dz2dx2), vmul(tab, tab),
                      vfma(vbc<V>(c.dz2dy2), vmul(tbc, tbc), vmul(vbc<V>(c.dx2dy2), vmul(tac, tac))));
    const V d3 = vsub(vbc<V>(t2), t3);
    const V b3 = vfma(vbc<V>(c.dsumi), vfma(tab, vbc<V>(c.dx2i), vmul(tbc, vbc<V>(-c.dy2i))), tb);
    V r3;
#pragma unroll
    for (int i = 0; i < N; ++i) vset(r3, i, rsqrt_(vget(d3, i)));
    const V t3c = vfma(vbc<V>(c.dsumi), r3, b3);
    const float cz4 = c.dz * s4, cx4 = c.dx * s4, cy5 = c.dy * s5, cz5 = c.dz * s5, cy6 = c.dy * s6,
                cx6 = c.dx * s6;
    V out;
#pragma unroll
    for (int i = 0; i < N; ++i) {
        float m = fminf(fminf(vget(t1z, i), vget(t1x, i)), vget(t1y, i));
        const float a = vget(temtv, i), b = vget(tvmtn, i), d = vget(temtn, i);
        if (a < cz4 && -a < cx4) m = fminf(m, vget(t_zx, i));
        if (b < cy5 && -b < cz5) m = fminf(m, vget(t_zy, i));
        if (d < cy6 && -d < cx6) m = fminf(m, vget(t_xy, i));
        const float tmax = fmaxf(fmaxf(vget(tv, i), vget(te, i)), vget(tn, i));
        const float t3d = (m > tmax && t2 >= vget(t3, i)) ? vget(t3c, i) : HUGEV;
        vset(out, i, fminf(vget(tupd, i), fminf(t3d, m)));
    }
    return out;
}

/* noinit_v<float> written with scalar operations: the same roundings in
 * the same order (every multiply-add explicit), so both give the same bits.
 * The direct Gauss-Seidel pass step uses this form (14 % faster there than
 * noinit_v<float2>).  With d = te - tv etc. the
 * plane operator is  t = tev + d (dx2i - dz2i)/B + (2/B) sqrt(s^2 B - C d^2),
 * B = dz2i + dx2i, C = dz2i dx2i, and the 3D operator's differences are
 * ta - tb = 1.5 (te - tv + ten - tnv), tb - tc = 1.5 (tv - tn + tev - ten),
 * t1 / dsum = tb + ((ta - tb) dx2i - (tb - tc) dy2i) / dsum. */
__device__ __forceinline__ float noinit_f32(const Mesh<float> &c, float tv, float te, float tn, float tev,
                                            float ten, float tnv, float tnve, float s1, float s2, float s3,
                                            float s4, float s5, float s6, float s7, float tupd)
{
    const float HUGEV = (float)FK_HUGE;
    float t12min = fminf(fminf(fmaf(c.dz, s1, tv), fmaf(c.dx, s2, te)), fmaf(c.dy, s3, tn));
    const float temtv = te - tv, tvmtn = tv - tn, temtn = te - tn;
    /* zx plane: ta - tb = 2 temtv, tb dz2i + ta dx2i = tev B + temtv (dx2i - dz2i) */
    const float q_zx = fmaf(s4 * s4, c.dz2i_p_dx2i, -c.dz2i_dx2i * (temtv * temtv));
    const float t_zx = fmaf(2.0f * c.dz2i_p_dx2i_inv, rsqrt_(q_zx),
                            fmaf(temtv, (c.dx2i - c.dz2i) * c.dz2i_p_dx2i_inv, tev));
    /* zy plane: ta = tvmtn + tnv, tb = -tvmtn + tnv; ta dz2i + tb dy2i */
    const float q_zy = fmaf(s5 * s5, c.dz2i_p_dy2i, -c.dz2i_dy2i * (tvmtn * tvmtn));
    const float t_zy = fmaf(2.0f * c.dz2i_p_dy2i_inv, rsqrt_(q_zy),
                            fmaf(tvmtn, (c.dz2i - c.dy2i) * c.dz2i_p_dy2i_inv, tnv));
    /* xy plane: ta = temtn + ten, tb = -temtn + ten; ta dx2i + tb dy2i */
    const float q_xy = fmaf(s6 * s6, c.dx2i_p_dy2i, -c.dx2i_dy2i * (temtn * temtn));
    const float t_xy = fmaf(2.0f * c.dx2i_p_dy2i_inv, rsqrt_(q_xy),
                            fmaf(temtn, (c.dx2i - c.dy2i) * c.dx2i_p_dy2i_inv, ten));
    if (temtv < c.dz * s4 && -temtv < c.dx * s4) t12min = fminf(t12min, t_zx);
    if (tvmtn < c.dy * s5 && -tvmtn < c.dz * s5) t12min = fminf(t12min, t_zy);
    if (temtn < c.dy * s6 && -temtn < c.dx * s6) t12min = fminf(t12min, t_xy);
    const float tmax = fmaxf(fmaxf(tv, te), tn);
    const float tab = 1.5f * (temtv + (ten - tnv));
    const float tbc = 1.5f * (tvmtn + (tev - ten));
    const float tac = tab + tbc;
    const float tb = fmaf((tnv - tn) + (tev - te), 0.5f, tv) - ten + tnve;
    const float t2 = (s7 * s7) * c.dsum_nine;
    const float t3 = fmaf(c.dz2dx2, tab * tab, fmaf(c.dz2dy2, tbc * tbc, c.dx2dy2 * (tac * tac)));
    const float t3c = fmaf(c.dsumi, rsqrt_(t2 - t3), fmaf(c.dsumi, fmaf(tab, c.dx2i, -tbc * c.dy2i), tb));
    const float t3d = (t12min > tmax && t2 >= t3) ? t3c : HUGEV;
    return fminf(tupd, fminf(t3d, t12min));
}

template <typename R>
__device__ __forceinline__ R noinit(const Mesh<R> &c, R tv, R te, R tn, R tev,
                                    R ten, R tnv, R tnve, R s1, R s2, R s3,
                                    R s4, R s5, R s6, R s7, R tupd)
{
    if constexpr (sizeof(R) == 4)
        return noinit_v<float>(c, tv, te, tn, tev, ten, tnv, tnve, s1, s2, s3, s4, s5, s6, s7, tupd);
    const R HUGEV = (R)FK_HUGE;
    R t12min = tv + c.dz * s1;
    t12min = rmin(t12min, te + c.dx * s2);
    t12min = rmin(t12min, tn + c.dy * s3);
    const R temtv = te - tv;
    const R tvmtn = tv - tn;
    const R temtn = te - tn;
    R t_zx, t_zy, t_xy;
    {
        R ta = tev + temtv, tb = tev - temtv, tab = ta - tb;
        t_zx = ((tb * c.dz2i + ta * c.dx2i) +
                rsqrt_((R)4 * (s4 * s4) * c.dz2i_p_dx2i - c.dz2i_dx2i * (tab * tab))) *
               c.dz2i_p_dx2i_inv;
    }
    {
        R ta = tvmtn + tnv, tb = -tvmtn + tnv, tab = ta - tb;
        t_zy = ((ta * c.dz2i + tb * c.dy2i) +
                rsqrt_((R)4 * (s5 * s5) * c.dz2i_p_dy2i - c.dz2i_dy2i * (tab * tab))) *
               c.dz2i_p_dy2i_inv;
    }
    {
        R ta = temtn + ten, tb = -temtn + ten, tab = ta - tb;
        t_xy = ((ta * c.dx2i + tb * c.dy2i) +
                rsqrt_((R)4 * (s6 * s6) * c.dx2i_p_dy2i - c.dx2i_dy2i * (tab * tab))) *
               c.dx2i_p_dy2i_inv;
    }
    if (temtv < c.dz * s4 && -temtv < c.dx * s4) t12min = rmin(t12min, t_zx);
    if (tvmtn < c.dy * s5 && -tvmtn < c.dz * s5) t12min = rmin(t12min, t_zy);
    if (temtn < c.dy * s6 && -temtn < c.dx * s6) t12min = rmin(t12min, t_xy);
    const R tmax = rmax(rmax(tv, te), tn);
    const R ta = te + (R)0.5 * (-tn + ten - tv + tev) - tnv + tnve;
    const R tb = tv + (R)0.5 * (-tn + tnv - te + tev) - ten + tnve;
    const R tc = tn + (R)0.5 * (-te + ten - tv + tnv) - tev + tnve;
    const R tab = ta - tb, tbc = tb - tc, tac = ta - tc;
    const R t2 = (s7 * s7) * c.dsum_nine;
    const R t3 = c.dz2dx2 * (tab * tab) + c.dz2dy2 * (tbc * tbc) + c.dx2dy2 * (tac * tac);
    const R t1 = tb * c.dz2i + ta * c.dx2i + tc * c.dy2i;
    const R t3c = (t1 + rsqrt_(t2 - t3)) * c.dsumi;
    const R t3d = (t12min > tmax && t2 >= t3) ? t3c : HUGEV;
    return rmin(tupd, rmin(t3d, t12min));
}

/* Source description used by the initialisation stencil. */
struct Src {
    int zsi, xsi, ysi;
    double zsa, xsa, ysa, szero, szero2, eps_t;
};

/* localSolver.F90:775-792 */
template <typename R>
__device__ __forceinline__ R tana(const Src &q, const Mesh<R> &c, int i, int j, int k)
{
    R dz_ = ((R)i - (R)q.zsa) * c.dz;
    R dx_ = ((R)j - (R)q.xsa) * c.dx;
    R dy_ = ((R)k - (R)q.ysa) * c.dy;
    return (R)q.szero * rsqrt_(dz_ * dz_ + dx_ * dx_ + dy_ * dy_);
}

/* localSolver.F90:538-751, one node.  lcart is the Cartesian/spherical
 * switch (tmin > epsSolver), evaluated by the caller in FP64. */
template <typename R>
__device__ R init_node(const Src &q, const Mesh<R> &c, bool lcart, R tv, R te,
                       R tn, R tev, R ten, R tnv, R tnve, R tt0, R slow1,
                       R slow2, R slow3, R slow4, R slow5, R slow6, R slow7,
                       int i, int j, int k, int sz, int sx, int sy)
{
    const R HUGEV = (R)FK_HUGE;
    const R szero2 = (R)q.szero2;
    R sgnrz_dzi = (R)sz / c.dz, sgnrx_dxi = (R)sx / c.dx, sgnry_dyi = (R)sy / c.dy;
    R t1d = tv + c.dz * slow1;
    t1d = rmin(t1d, te + c.dx * slow2);
    t1d = rmin(t1d, tn + c.dy * slow3);
    R tmax = rmax(rmax(tv, te), tn);
    R t0c = 0, tzc = 0, txc = 0, tyc = 0;
    R tauv = HUGEV, taue = HUGEV, taun = HUGEV, tauev = HUGEV, tauen = HUGEV,
      taunv = HUGEV, taunve = HUGEV;
    if (!lcart) {
        /* localSolver.F90:819-851 (tAnaD) */
        R dz_ = ((R)i - (R)q.zsa) * c.dz;
        R dx_ = ((R)j - (R)q.xsa) * c.dx;
        R dy_ = ((R)k - (R)q.ysa) * c.dy;
        R d0 = dz_ * dz_ + dx_ * dx_ + dy_ * dy_;
        R d0i_szero = 0;
        if (d0 > (R)0) {
            R sq = rsqrt_(d0);
            t0c = (R)q.szero * sq;
            d0i_szero = (R)q.szero / sq;
        }
        tzc = d0i_szero * dz_;
        txc = d0i_szero * dx_;
        tyc = d0i_szero * dy_;
        tauv = tv - tana(q, c, i - sz, j, k);
        taue = te - tana(q, c, i, j - sx, k);
        taun = tn - tana(q, c, i, j, k - sy);
        tauev = tev - tana(q, c, i - sz, j - sx, k);
        tauen = ten - tana(q, c, i, j - sx, k - sy);
        taunv = tnv - tana(q, c, i - sz, j, k - sy);
        taunve = tnve - tana(q, c, i - sz, j - sx, k - sy);
    }
    bool ldoZX = (tv < te + c.dx * slow4) && (te < tv + c.dz * slow4);
    bool ldoZY = (tv < tn + c.dy * slow5) && (tn < tv + c.dz * slow5);
    bool ldoXY = (te < tn + c.dy * slow6) && (tn < te + c.dx * slow6);
    bool zxc = ldoZX && (lcart || k != q.ysi);
    bool zyc = ldoZY && (lcart || j != q.xsi);
    bool xyc = ldoXY && (lcart || i != q.zsi);
    bool zxs = ldoZX && !zxc, zys = ldoZY && !zyc, xys = ldoXY && !xyc;
    R t1_2d = HUGEV;
    if (zxc) {
        R ta = tev + te - tv, tb = tev - te + tv, tab = ta - tb;
        t1_2d = ((tb * c.dz2i + ta * c.dx2i) +
                 rsqrt_((R)4 * (slow4 * slow4) * c.dz2i_p_dx2i - c.dz2i_dx2i * (tab * tab))) *
                c.dz2i_p_dx2i_inv;
    }
    if (zxs) {
        R sref2 = slow4 * slow4;
        R ta = tauev + taue - tauv, tb = tauev - taue + tauv;
        R apoly = c.dz2i_p_dx2i;
        R bpoly = (R)4 * (sgnrx_dxi * txc + sgnrz_dzi * tzc) - (R)2 * (ta * c.dx2i + tb * c.dz2i);
        R cpoly = ((ta * ta) * c.dx2i) + ((tb * tb) * c.dz2i) -
                  (R)4 * (sgnrx_dxi * txc * ta + sgnrz_dzi * tzc * tb) +
                  (R)4 * (szero2 - sref2 + tyc * tyc);
        R dpoly = bpoly * bpoly - (R)4 * apoly * cpoly;
        if (dpoly >= (R)0) t1_2d = (rsqrt_(dpoly) - bpoly) / ((R)2 * apoly) + t0c;
        if (t1_2d < tv || t1_2d < te) t1_2d = HUGEV;
    }
    R tmin12 = rmin(t1d, t1_2d);
    R t2_2d = HUGEV;
    if (zyc) {
        R ta = tv - tn + tnv, tb = tn - tv + tnv, tab = ta - tb;
        t2_2d = ((ta * c.dz2i + tb * c.dy2i) +
                 rsqrt_((R)4 * (slow5 * slow5) * c.dz2i_p_dy2i - c.dz2i_dy2i * (tab * tab))) *
                c.dz2i_p_dy2i_inv;
    }
    if (zys) {
        R sref2 = slow5 * slow5;
        R ta = tauv - taun + taunv, tb = taun - tauv + taunv;
        R apoly = c.dz2i_p_dy2i;
        R bpoly = (R)4 * (sgnry_dyi * tyc + sgnrz_dzi * tzc) - (R)2 * (ta * c.dz2i + tb * c.dy2i);
        R cpoly = ((ta * ta) * c.dz2i) + ((tb * tb) * c.dy2i) -
                  (R)4 * (sgnrz_dzi * tzc * ta + sgnry_dyi * tyc * tb) +
                  (R)4 * (szero2 - sref2 + txc * txc);
        R dpoly = bpoly * bpoly - (R)4 * apoly * cpoly;
        if (dpoly >= (R)0) t2_2d = (rsqrt_(dpoly) - bpoly) / ((R)2 * apoly) + t0c;
        if (t2_2d < tv || t2_2d < tn) t2_2d = HUGEV;
    }
    tmin12 = rmin(tmin12, t2_2d);
    R t3_2d = HUGEV;
    if (xyc) {
        R ta = te - tn + ten, tb = tn - te + ten, tab = ta - tb;
        t3_2d = ((ta * c.dx2i + tb * c.dy2i) +
                 rsqrt_((R)4 * (slow6 * slow6) * c.dx2i_p_dy2i - c.dx2i_dy2i * (tab * tab))) *
                c.dx2i_p_dy2i_inv;
    }
    if (xys) {
        R sref2 = slow6 * slow6;
        R ta = taue - taun + tauen, tb = taun - taue + tauen;
        R apoly = c.dx2i_p_dy2i;
        R bpoly = (R)4 * (sgnry_dyi * tyc + sgnrx_dxi * txc) - (R)2 * (ta * c.dx2i + tb * c.dy2i);
        R cpoly = ((ta * ta) * c.dx2i) + ((tb * tb) * c.dy2i) -
                  (R)4 * (sgnrx_dxi * txc * ta + sgnry_dyi * tyc * tb) +
                  (R)4 * (szero2 - sref2 + tzc * tzc);
        R dpoly = bpoly * bpoly - (R)4 * apoly * cpoly;
        if (dpoly >= (R)0) t3_2d = (rsqrt_(dpoly) - bpoly) / ((R)2 * apoly) + t0c;
        if (t3_2d < te || t3_2d < tn) t3_2d = HUGEV;
    }
    tmin12 = rmin(tmin12, t3_2d);
    R t3d = HUGEV;
    bool ldo3D = tmin12 > tmax;
    if (ldo3D && lcart) {
        R ta = te + (R)0.5 * (-tn + ten - tv + tev) - tnv + tnve;
        R tb = tv + (R)0.5 * (-tn + tnv - te + tev) - ten + tnve;
        R tc = tn + (R)0.5 * (-te + ten - tv + tnv) - tev + tnve;
        R tab = ta - tb, tbc = tb - tc, tac = ta - tc;
        R t2 = (slow7 * slow7) * c.dsum_nine;
        R t3 = c.dz2dx2 * (tab * tab) + c.dz2dy2 * (tbc * tbc) + c.dx2dy2 * (tac * tac);
        if (t2 >= t3) {
            R t1 = tb * c.dz2i + ta * c.dx2i + tc * c.dy2i;
            t3d = (t1 + rsqrt_(t2 - t3)) * c.dsumi;
        }
    }
    if (ldo3D && !lcart) {
        R sref2 = slow7 * slow7;
        R ta = taue + (R)0.5 * (-taun + tauen - tauv + tauev) - taunv + taunve;
        R tb = tauv + (R)0.5 * (-taun + taunv - taue + tauev) - tauen + taunve;
        R tc = taun + (R)0.5 * (-taue + tauen - tauv + taunv) - tauev + taunve;
        R apoly = c.dx2i + c.dz2i + c.dy2i;
        R bpoly = (R)6 * (sgnrz_dzi * tzc + sgnry_dyi * tyc + sgnrx_dxi * txc) -
                  (R)2 * (ta * c.dx2i + tb * c.dz2i + tc * c.dy2i);
        R cpoly = ((ta * ta) * c.dx2i) + ((tb * tb) * c.dz2i) + ((tc * tc) * c.dy2i) -
                  (R)6 * (sgnrx_dxi * txc * ta + sgnrz_dzi * tzc * tb + sgnry_dyi * tyc * tc) +
                  (R)9 * (szero2 - sref2);
        R dpoly = bpoly * bpoly - (R)4 * apoly * cpoly;
        if (dpoly >= (R)0) t3d = (rsqrt_(dpoly) - bpoly) / ((R)2 * apoly) + t0c;
        if (t3d < te || t3d < tn || t3d < tv) t3d = HUGEV;
    }
    R tupd = rmin(tmin12, t3d);
    return rmin(tt0, tupd);
}

} // namespace fk3
