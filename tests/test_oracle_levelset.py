"""Second, independent restatement of the reference's solvers, checked bit for
bit against the C oracle.

The C oracle (oracle/fteik_oracle.c) is organised for speed (flattened sweep
tables, OpenMP over levels).  This file transcribes the reference's Fortran
again, statement by statement, as scalar Python on IEEE doubles, keeping the
reference's structure: the level lists of graph3d.F90, the update masks of
solver3D.F90, the per-sweep prefetch routines of autoCode.f90 and the local
solvers of localSolver.F90.  Python floats never fuse a multiply-add and
math.sqrt is correctly rounded, so with the reference's operation order both
restatements must agree to the last bit; any transcription slip in either
one shows up as a mismatch.  Pure Python, so the grids are small (a few
thousand nodes).

Cited reference files (paths within the fteik project):
  source.F90:82-236, 429-464   source snap, szero
  localSolver.F90:36-100       2D analytic time and derivative
  localSolver.F90:123-158      2D plane-wave update
  localSolver.F90:195-289      2D initialisation update
  localSolver.F90:300-352      2D mesh constants
  localSolver.F90:384-534      3D plane-wave update (noInit)
  localSolver.F90:538-751      3D initialisation update (init)
  localSolver.F90:775-851      3D analytic time and derivative
  localSolver.F90:878-959      3D mesh constants and source corner times
  autoCode.f90:23-368          travel-time prefetch per sweep (signs sgnt)
  autoCode.f90:389-1000        slowness prefetch per sweep (signs sgnv)
  autoCode.f90:1001-1316       sweep driver (level loop, masks, scatter)
  graph3d.F90:122-353          level structure in sweep-permuted coordinates
  solver3D.F90:411-565         update masks and sweep limits
  solver3D.F90:1156-1243       3D solveSourceLSM
  solver2D.F90:377-732         2D level helpers (masks, prefetch, update)
  solver2D.F90:782-978         2D solveSourceLSM
"""
import ctypes
import ctypes.util
import math

import numpy as np
import pytest

import oracle_lib as O
from models import layered_grf_cells, linear_vz_cells

HUGE = 99999.0                      # constants.F90:5
DBL_EPSILON = 2.220446049250313e-16  # constants.F90:19, EPSILON(1.d0)
PERTURB = 0.0001                    # constants.F90:21

_libm = ctypes.CDLL(ctypes.util.find_library("m"))
_libm.hypot.restype = ctypes.c_double
_libm.hypot.argtypes = [ctypes.c_double, ctypes.c_double]


def _hypot(a, b):
    """Fortran HYPOT, which the reference's compiler lowers to libm hypot."""
    return _libm.hypot(a, b)


def _sqrt(x):
    """DSQRT; a negative argument would give NaN in the Fortran."""
    return math.sqrt(x) if x >= 0.0 else float("nan")


# ----------------------------------------------------------- source snap --
def snap(n, h, src, is3d=True):
    """source.F90:82-236 with a zero origin: 1-based (zsi, xsi, ysi) and the
    fractional grid coordinates (zsa, xsa, ysa)."""
    out_i, out_a = [], []
    for ax in range(3 if is3d else 2):
        loc = src[ax] - 0.0
        a = (loc / h[ax]) + 1.0
        if abs(a - 1.0) < DBL_EPSILON:
            a = a + PERTURB
        if a >= float(n[ax]):
            a = a - PERTURB
        out_i.append(int(a))
        out_a.append(a)
    return tuple(out_i), tuple(out_a)


# ------------------------------------------------------------------- 3D --
# (sgntz, sgntx, sgnty) of sweeps 1..8, autoCode.f90 parameter lines 34-36,
# 80-82, 126-128, 172-174, 218-220, 264-266, 310-312, 356-358; the slowness
# signs sgnv are 1 where sgnt = 1 and 0 where sgnt = -1 (lines 407-962).
SIGNS3 = {1: (1, 1, 1), 2: (1, -1, 1), 3: (1, 1, -1), 4: (1, -1, -1),
          5: (-1, 1, 1), 6: (-1, -1, 1), 7: (-1, 1, -1), 8: (-1, -1, -1)}


class Mesh3:
    """localSolver.F90:878-931: the mesh constants in the reference's order."""

    def __init__(self, h, src_i, src_a, szero, eps):
        dz, dx, dy = h
        self.dz, self.dx, self.dy = dz, dx, dy
        self.zsi, self.xsi, self.ysi = src_i
        self.zsa, self.xsa, self.ysa = src_a
        self.szero = szero
        self.szero2 = szero * szero                      # source.F90:459
        self.epsSolver = eps * min(dz, dx, dy) * szero
        dz2, dx2, dy2 = dz * dz, dx * dx, dy * dy
        self.dzi, self.dxi, self.dyi = 1.0 / dz, 1.0 / dx, 1.0 / dy
        self.dz2i, self.dx2i, self.dy2i = 1.0 / dz2, 1.0 / dx2, 1.0 / dy2
        self.dsum = self.dz2i + self.dx2i + self.dy2i
        self.dsum_nine = self.dsum * 9.0
        self.dsumi = 1.0 / self.dsum
        self.dz2dx2 = 1.0 / (dz2 * dx2)
        self.dz2dy2 = 1.0 / (dz2 * dy2)
        self.dx2dy2 = 1.0 / (dx2 * dy2)
        self.dz2i_dx2i = self.dz2i * self.dx2i
        self.dz2i_dy2i = self.dz2i * self.dy2i
        self.dx2i_dy2i = self.dx2i * self.dy2i
        self.dz2i_p_dy2i_inv = 1.0 / (self.dz2i + self.dy2i)
        self.dz2i_p_dx2i_inv = 1.0 / (self.dz2i + self.dx2i)
        self.dx2i_p_dy2i_inv = 1.0 / (self.dx2i + self.dy2i)
        self.dz2i_p_dx2i = self.dz2i + self.dx2i
        self.dz2i_p_dy2i = self.dz2i + self.dy2i
        self.dx2i_p_dy2i = self.dx2i + self.dy2i

    def tana(self, i, j, k):
        """localSolver.F90:775-792."""
        diffz = (float(i) - self.zsa) * self.dz
        diffx = (float(j) - self.xsa) * self.dx
        diffy = (float(k) - self.ysa) * self.dy
        d0 = diffz * diffz + diffx * diffx + diffy * diffy
        return self.szero * math.sqrt(d0)

    def tanad(self, i, j, k):
        """localSolver.F90:819-851 -> (t_anad, tzc, txc, tyc)."""
        diffz = (float(i) - self.zsa) * self.dz
        diffx = (float(j) - self.xsa) * self.dx
        diffy = (float(k) - self.ysa) * self.dy
        d0 = diffz * diffz + diffx * diffx + diffy * diffy
        d0i_szero = 0.0
        t_anad = 0.0
        if d0 > 0.0:
            sqrtd0 = math.sqrt(d0)
            t_anad = self.szero * sqrtd0
            d0i_szero = self.szero / sqrtd0
        return t_anad, d0i_szero * diffz, d0i_szero * diffx, d0i_szero * diffy


def noinit3(m, tv, te, tn, tev, ten, tnv, tnve, s1, s2, s3, s4, s5, s6, s7, tupd):
    """fteik_localSolver_noInit64fF, localSolver.F90:384-534, one node."""
    t12 = tv + m.dz * s1
    t12 = min(t12, te + m.dx * s2)
    t12 = min(t12, tn + m.dy * s3)
    # ZX plane
    t1_2d = HUGE
    temtv = te - tv
    if temtv < m.dz * s4 and -temtv < m.dx * s4:
        sref2 = s4 * s4
        ta = tev + temtv
        tb = tev - temtv
        tab = ta - tb
        tab2 = tab * tab
        four_sref2 = 4.0 * sref2
        t1_2d = ((tb * m.dz2i + ta * m.dx2i)
                 + _sqrt(four_sref2 * m.dz2i_p_dx2i - m.dz2i_dx2i * tab2)) * m.dz2i_p_dx2i_inv
    t12 = min(t12, t1_2d)
    # ZY plane
    t2_2d = HUGE
    tvmtn = tv - tn
    if tvmtn < m.dy * s5 and -tvmtn < m.dz * s5:
        sref2 = s5 * s5
        ta = tvmtn + tnv
        tb = -tvmtn + tnv
        tab = ta - tb
        tab2 = tab * tab
        four_sref2 = 4.0 * sref2
        t2_2d = ((ta * m.dz2i + tb * m.dy2i)
                 + _sqrt(four_sref2 * m.dz2i_p_dy2i - m.dz2i_dy2i * tab2)) * m.dz2i_p_dy2i_inv
    t12 = min(t12, t2_2d)
    # XY plane
    t3_2d = HUGE
    temtn = te - tn
    if temtn < m.dy * s6 and -temtn < m.dx * s6:
        sref2 = s6 * s6
        ta = temtn + ten
        tb = -temtn + ten
        tab = ta - tb
        tab2 = tab * tab
        four_sref2 = 4.0 * sref2
        t3_2d = ((ta * m.dx2i + tb * m.dy2i)
                 + _sqrt(four_sref2 * m.dx2i_p_dy2i - m.dx2i_dy2i * tab2)) * m.dx2i_p_dy2i_inv
    t12 = min(t12, t3_2d)
    # 3D operator
    t3d = HUGE
    tmax = max(tv, te, tn)
    if t12 > tmax:
        sref2 = s7 * s7
        ta = te + 0.5 * (-tn + ten - tv + tev) - tnv + tnve
        tb = tv + 0.5 * (-tn + tnv - te + tev) - ten + tnve
        tc = tn + 0.5 * (-te + ten - tv + tnv) - tev + tnve
        tab = ta - tb
        tbc = tb - tc
        tac = ta - tc
        t2 = sref2 * m.dsum_nine
        tab2 = tab * tab
        tbc2 = tbc * tbc
        tac2 = tac * tac
        t3 = m.dz2dx2 * tab2 + m.dz2dy2 * tbc2 + m.dx2dy2 * tac2
        if t2 >= t3:
            t1 = tb * m.dz2i + ta * m.dx2i + tc * m.dy2i
            t3d = (t1 + math.sqrt(t2 - t3)) * m.dsumi
    t3d = min(t3d, t12)
    return min(tupd, t3d)


def init3(m, tv, te, tn, tev, ten, tnv, tnve, tt0, s1, s2, s3, s4, s5, s6, s7,
          i, j, k, sgntz, sgntx, sgnty, sgnrz_dzi, sgnrx_dxi, sgnry_dyi):
    """fteik_localSolver_init64fF, localSolver.F90:538-751, one node."""
    t1d = tv + m.dz * s1
    t1d = min(t1d, te + m.dx * s2)
    t1d = min(t1d, tn + m.dy * s3)
    tmin = min(tv, te, tn)
    tmax = max(tv, te, tn)
    lcart = tmin > m.epsSolver
    t0c = tzc = txc = tyc = 0.0
    tauv = taue = taun = tauev = tauen = taunv = taunve = HUGE
    if not lcart:
        t0c, tzc, txc, tyc = m.tanad(i, j, k)
        tauv = tv - m.tana(i - sgntz, j, k)
        taue = te - m.tana(i, j - sgntx, k)
        taun = tn - m.tana(i, j, k - sgnty)
        tauev = tev - m.tana(i - sgntz, j - sgntx, k)
        tauen = ten - m.tana(i, j - sgntx, k - sgnty)
        taunv = tnv - m.tana(i - sgntz, j, k - sgnty)
        taunve = tnve - m.tana(i - sgntz, j - sgntx, k - sgnty)
    ldoZX = (tv < te + m.dx * s4) and (te < tv + m.dz * s4)
    ldoZY = (tv < tn + m.dy * s5) and (tn < tv + m.dz * s5)
    ldoXY = (te < tn + m.dy * s6) and (tn < te + m.dx * s6)
    ldoZXCart = ldoZX and (lcart or k != m.ysi)
    ldoZYCart = ldoZY and (lcart or j != m.xsi)
    ldoXYCart = ldoXY and (lcart or i != m.zsi)
    ldoZXSphere = ldoZX and not ldoZXCart
    ldoZYSphere = ldoZY and not ldoZYCart
    ldoXYSphere = ldoXY and not ldoXYCart
    # ZX plane
    t1_2d = HUGE
    if ldoZXCart:
        sref2 = s4 * s4
        ta = tev + te - tv
        tb = tev - te + tv
        tab = ta - tb
        tab2 = tab * tab
        four_sref2 = 4.0 * sref2
        t1_2d = ((tb * m.dz2i + ta * m.dx2i)
                 + _sqrt(four_sref2 * m.dz2i_p_dx2i - m.dz2i_dx2i * tab2)) * m.dz2i_p_dx2i_inv
    if ldoZXSphere:
        sref2 = s4 * s4
        ta = tauev + taue - tauv
        tb = tauev - taue + tauv
        apoly = m.dz2i_p_dx2i
        bpoly = 4.0 * (sgnrx_dxi * txc + sgnrz_dzi * tzc) - 2.0 * (ta * m.dx2i + tb * m.dz2i)
        cpoly = (((ta * ta) * m.dx2i) + ((tb * tb) * m.dz2i)
                 - 4.0 * (sgnrx_dxi * txc * ta + sgnrz_dzi * tzc * tb)
                 + 4.0 * (m.szero2 - sref2 + tyc * tyc))
        dpoly = bpoly * bpoly - 4.0 * apoly * cpoly
        if dpoly >= 0.0:
            t1_2d = (math.sqrt(dpoly) - bpoly) / (2.0 * apoly) + t0c
        if t1_2d < tv or t1_2d < te:
            t1_2d = HUGE
    tmin12 = min(t1d, t1_2d)
    # ZY plane
    t2_2d = HUGE
    if ldoZYCart:
        sref2 = s5 * s5
        ta = tv - tn + tnv
        tb = tn - tv + tnv
        tab = ta - tb
        tab2 = tab * tab
        four_sref2 = 4.0 * sref2
        t2_2d = ((ta * m.dz2i + tb * m.dy2i)
                 + _sqrt(four_sref2 * m.dz2i_p_dy2i - m.dz2i_dy2i * tab2)) * m.dz2i_p_dy2i_inv
    if ldoZYSphere:
        sref2 = s5 * s5
        ta = tauv - taun + taunv
        tb = taun - tauv + taunv
        apoly = m.dz2i_p_dy2i
        bpoly = 4.0 * (sgnry_dyi * tyc + sgnrz_dzi * tzc) - 2.0 * (ta * m.dz2i + tb * m.dy2i)
        cpoly = (((ta * ta) * m.dz2i) + ((tb * tb) * m.dy2i)
                 - 4.0 * (sgnrz_dzi * tzc * ta + sgnry_dyi * tyc * tb)
                 + 4.0 * (m.szero2 - sref2 + txc * txc))
        dpoly = bpoly * bpoly - 4.0 * apoly * cpoly
        if dpoly >= 0.0:
            t2_2d = (math.sqrt(dpoly) - bpoly) / (2.0 * apoly) + t0c
        if t2_2d < tv or t2_2d < tn:
            t2_2d = HUGE
    tmin12 = min(tmin12, t2_2d)
    # XY plane
    t3_2d = HUGE
    if ldoXYCart:
        sref2 = s6 * s6
        ta = te - tn + ten
        tb = tn - te + ten
        tab = ta - tb
        tab2 = tab * tab
        four_sref2 = 4.0 * sref2
        t3_2d = ((ta * m.dx2i + tb * m.dy2i)
                 + _sqrt(four_sref2 * m.dx2i_p_dy2i - m.dx2i_dy2i * tab2)) * m.dx2i_p_dy2i_inv
    if ldoXYSphere:
        sref2 = s6 * s6
        ta = taue - taun + tauen
        tb = taun - taue + tauen
        apoly = m.dx2i_p_dy2i
        bpoly = 4.0 * (sgnry_dyi * tyc + sgnrx_dxi * txc) - 2.0 * (ta * m.dx2i + tb * m.dy2i)
        cpoly = (((ta * ta) * m.dx2i) + ((tb * tb) * m.dy2i)
                 - 4.0 * (sgnrx_dxi * txc * ta + sgnry_dyi * tyc * tb)
                 + 4.0 * (m.szero2 - sref2 + tzc * tzc))
        dpoly = bpoly * bpoly - 4.0 * apoly * cpoly
        if dpoly >= 0.0:
            t3_2d = (math.sqrt(dpoly) - bpoly) / (2.0 * apoly) + t0c
        if t3_2d < te or t3_2d < tn:
            t3_2d = HUGE
    tmin12 = min(tmin12, t3_2d)
    # 3D operators
    t3d = HUGE
    ldo3d = tmin12 > tmax
    if ldo3d and lcart:
        sref2 = s7 * s7
        ta = te + 0.5 * (-tn + ten - tv + tev) - tnv + tnve
        tb = tv + 0.5 * (-tn + tnv - te + tev) - ten + tnve
        tc = tn + 0.5 * (-te + ten - tv + tnv) - tev + tnve
        tab = ta - tb
        tbc = tb - tc
        tac = ta - tc
        t2 = sref2 * m.dsum_nine
        tab2 = tab * tab
        tbc2 = tbc * tbc
        tac2 = tac * tac
        t3 = m.dz2dx2 * tab2 + m.dz2dy2 * tbc2 + m.dx2dy2 * tac2
        if t2 >= t3:
            t1 = tb * m.dz2i + ta * m.dx2i + tc * m.dy2i
            t3d = (t1 + math.sqrt(t2 - t3)) * m.dsumi
    if ldo3d and not lcart:
        sref2 = s7 * s7
        ta = taue + 0.5 * (-taun + tauen - tauv + tauev) - taunv + taunve
        tb = tauv + 0.5 * (-taun + taunv - taue + tauev) - tauen + taunve
        tc = taun + 0.5 * (-taue + tauen - tauv + taunv) - tauev + taunve
        apoly = m.dx2i + m.dz2i + m.dy2i
        bpoly = (6.0 * (sgnrz_dzi * tzc + sgnry_dyi * tyc + sgnrx_dxi * txc)
                 - 2.0 * (ta * m.dx2i + tb * m.dz2i + tc * m.dy2i))
        cpoly = (((ta * ta) * m.dx2i) + ((tb * tb) * m.dz2i) + ((tc * tc) * m.dy2i)
                 - 6.0 * (sgnrx_dxi * txc * ta + sgnrz_dzi * tzc * tb + sgnry_dyi * tyc * tc)
                 + 9.0 * (m.szero2 - sref2))
        dpoly = bpoly * bpoly - 4.0 * apoly * cpoly
        if dpoly >= 0.0:
            t3d = (math.sqrt(dpoly) - bpoly) / (2.0 * apoly) + t0c
        if t3d < te or t3d < tn or t3d < tv:
            t3d = HUGE
    tupd = min(tmin12, t3d)
    return min(tt0, tupd)


def slowness7(slow, n, i, j, k, sgnvz, sgnvx, sgnvy):
    """fteik_prefetchSweep{s}Slowness64fF, autoCode.f90:389-447 (sweep 1;
    the other sweeps differ only in sgnv)."""
    nz, nx, ny = n
    nzm1, nzm1_nxm1 = nz - 1, (nz - 1) * (nx - 1)

    def S(a, b, c):                 # velGrid2indexF, 1-based -> 0-based
        return slow[(c - 1) * nzm1_nxm1 + (b - 1) * nzm1 + a - 1]

    i1, j1, k1 = i - sgnvz, j - sgnvx, k - sgnvy
    mi, mj, mk = max(i - 1, 1), max(j - 1, 1), max(k - 1, 1)
    Mi, Mj, Mk = min(i, nz - 1), min(j, nx - 1), min(k, ny - 1)
    s1 = min(S(i1, mj, mk), S(i1, mj, Mk), S(i1, Mj, mk), S(i1, Mj, Mk))
    s2 = min(S(mi, j1, mk), S(Mi, j1, mk), S(mi, j1, Mk), S(Mi, j1, Mk))
    s3 = min(S(mi, mj, k1), S(mi, Mj, k1), S(Mi, mj, k1), S(Mi, Mj, k1))
    s4 = min(S(i1, j1, mk), S(i1, j1, Mk))
    s5 = min(S(i1, mj, k1), S(i1, Mj, k1))
    s6 = min(S(mi, j1, k1), S(Mi, j1, k1))
    s7 = S(i1, j1, k1)
    return s1, s2, s3, s4, s5, s6, s7


def sweep_limits(sweep, linit, n, src_i):
    """fteik_solver3d_getSweepLimits, solver3D.F90:493-565, as the inclusive
    box (zmin, zmax, xmin, xmax, ymin, ymax) of setUpdateNodes (:411-466).

    Deviation shared with the oracle and the GPU: for a flipped axis the
    initialisation box starts at min(si + 1, n - 1); the reference's si + 1
    reaches n for a source in the last cell, whose upwind neighbour lies
    outside the grid."""
    nz, nx, ny = n
    zsi, xsi, ysi = src_i
    sz, sx, sy = SIGNS3[sweep]
    box = []
    for sgn, nn, si in ((sz, nz, zsi), (sx, nx, xsi), (sy, ny, ysi)):
        if sgn == 1:
            lo, hi = (max(2, si), nn) if linit else (2, nn)
        else:
            lo, hi = (1, min(si + 1, nn - 1)) if linit else (1, nn - 1)
        box += [lo, hi]
    return tuple(box)


_LEVELS = {}


def levels3(n, sweep):
    """graph3d.F90:122-353: level l holds the nodes whose sweep-permuted
    1-based coordinates sum to l + 2; inside a level, by linear index."""
    key = (n, sweep)
    if key not in _LEVELS:
        nz, nx, ny = n
        sz, sx, sy = SIGNS3[sweep]
        lev = {}
        for iy in range(1, ny + 1):
            for ix in range(1, nx + 1):
                for iz in range(1, nz + 1):
                    pz = iz if sz == 1 else nz + 1 - iz
                    px = ix if sx == 1 else nx + 1 - ix
                    py = iy if sy == 1 else ny + 1 - iy
                    lev.setdefault(pz + px + py - 2, []).append((iz, ix, iy))
        _LEVELS[key] = [lev[l] for l in range(1, nx + ny + nz - 1)]
    return _LEVELS[key]


def solve3(n, h, slow, src, eps, nsweep):
    """fteik_solver3d_solveSourceLSM, solver3D.F90:1156-1243."""
    nz, nx, ny = n
    src_i, src_a = snap(n, h, src)
    zsi, xsi, ysi = src_i
    szero = slow[(ysi - 1) * (nz - 1) * (nx - 1) + (xsi - 1) * (nz - 1) + zsi - 1]
    m = Mesh3(h, src_i, src_a, szero, eps)
    nzx = nz * nx

    def G(i, j, k):                 # grid2indexF, 1-based -> 0-based
        return (k - 1) * nzx + (j - 1) * nz + i - 1

    tt = [HUGE] * (nz * nx * ny)
    for dk in (0, 1):               # ts8 / dest, localSolver.F90:933-956
        for dj in (0, 1):
            for di in (0, 1):
                tt[G(zsi + di, xsi + dj, ysi + dk)] = m.tana(zsi + di, xsi + dj, ysi + dk)
    for linit in [True] + [False] * nsweep:
        for sweep in range(1, 9):
            sgntz, sgntx, sgnty = SIGNS3[sweep]
            sgnvz, sgnvx, sgnvy = (1 if s == 1 else 0 for s in (sgntz, sgntx, sgnty))
            sgnrz_dzi = float(sgntz) / m.dz
            sgnrx_dxi = float(sgntx) / m.dx
            sgnry_dyi = float(sgnty) / m.dy
            z1, z2, x1, x2, y1, y2 = sweep_limits(sweep, linit, n, src_i)
            for level in levels3(n, sweep):
                out = []
                for (i, j, k) in level:
                    if not (z1 <= i <= z2 and x1 <= j <= x2 and y1 <= k <= y2):
                        continue
                    s = slowness7(slow, n, i, j, k, sgnvz, sgnvx, sgnvy)
                    tv = tt[G(i - sgntz, j, k)]
                    te = tt[G(i, j - sgntx, k)]
                    tn = tt[G(i, j, k - sgnty)]
                    tev = tt[G(i - sgntz, j - sgntx, k)]
                    ten = tt[G(i, j - sgntx, k - sgnty)]
                    tnv = tt[G(i - sgntz, j, k - sgnty)]
                    tnve = tt[G(i - sgntz, j - sgntx, k - sgnty)]
                    t0 = tt[G(i, j, k)]
                    if linit:
                        v = init3(m, tv, te, tn, tev, ten, tnv, tnve, t0, *s, i, j, k,
                                  sgntz, sgntx, sgnty, sgnrz_dzi, sgnrx_dxi, sgnry_dyi)
                    else:
                        v = noinit3(m, tv, te, tn, tev, ten, tnv, tnve, *s, t0)
                    out.append((G(i, j, k), v))
                for g, v in out:    # nodes of one level are independent
                    tt[g] = v
    return np.array(tt), src_i, src_a


# ------------------------------------------------------------------- 2D --
# (sgntz, sgntx, sgnvz, sgnvx), localSolver.F90 getSweepSigns
SIGNS2 = {1: (1, 1, 1, 1), 2: (1, -1, 1, 0), 3: (-1, 1, 0, 1), 4: (-1, -1, 0, 0)}


class Mesh2:
    """localSolver.F90:300-352: 2D constants; epsSolver is in grid points."""

    def __init__(self, h, src_i, src_a, szero, eps):
        self.dz, self.dx = h
        self.zsi, self.xsi = src_i
        self.zsa, self.xsa = src_a
        self.szero = szero
        self.epsSolver = eps
        dz2, dx2 = self.dz * self.dz, self.dx * self.dx
        self.dzi, self.dxi = 1.0 / self.dz, 1.0 / self.dx
        self.dz2i, self.dx2i = 1.0 / dz2, 1.0 / dx2
        self.dz2i_dx2i = self.dz2i * self.dx2i
        self.dz2i_p_dx2i = self.dz2i + self.dx2i
        self.dz2i_p_dx2i_inv = 1.0 / (self.dz2i + self.dx2i)

    def tana(self, i, j):
        """localSolver.F90:36-45."""
        diffz = (float(i) - self.zsa) * self.dz
        diffx = (float(j) - self.xsa) * self.dx
        return self.szero * _hypot(diffx, diffz)

    def tanad(self, i, j):
        """localSolver.F90:46-100 -> (t_anad, tzc, txc)."""
        diffz = (float(i) - self.zsa) * self.dz
        diffx = (float(j) - self.xsa) * self.dx
        d0 = diffz * diffz + diffx * diffx
        d0i_szero = 0.0
        t_anad = 0.0
        if d0 > 0.0:
            sqrtd0 = math.sqrt(d0)
            t_anad = self.szero * sqrtd0
            d0i_szero = self.szero / sqrtd0
        return t_anad, d0i_szero * diffz, d0i_szero * diffx


def init2(m, n, slow, tt, sweep, iz, ix):
    """fteik_localSolver2d_init64f, localSolver.F90:195-289."""
    nz, nx = n
    dz, dx = m.dz, m.dx
    dz2i, dx2i, dzi, dxi = m.dz2i, m.dx2i, m.dzi, m.dxi
    sgntz, sgntx, sgnvz, sgnvx = SIGNS2[sweep]
    sgnrz, sgnrx = float(sgntz), float(sgntx)
    tv = tt[(ix - 1) * nz + iz - sgntz - 1]
    te = tt[(ix - sgntx - 1) * nz + iz - 1]
    tev = tt[(ix - sgntx - 1) * nz + iz - sgntz - 1]
    t = tt[(ix - 1) * nz + iz - 1]
    i1, j1 = iz - sgnvz, ix - sgnvx
    sref1 = min(slow[(max(ix - 1, 1) - 1) * (nz - 1) + i1 - 1],
                slow[(min(ix, nx - 1) - 1) * (nz - 1) + i1 - 1])
    sref2 = min(slow[(j1 - 1) * (nz - 1) + max(iz - 1, 1) - 1],
                slow[(j1 - 1) * (nz - 1) + min(iz, nz - 1) - 1])
    sref3 = slow[(j1 - 1) * (nz - 1) + i1 - 1]
    t1d = min(tv + dz * sref1, te + dx * sref2)
    t0c, tzc, txc = m.tanad(iz, ix)
    tauv = tv - m.tana(iz - sgntz, ix)
    taue = te - m.tana(iz, ix - sgntx)
    tauev = tev - m.tana(iz - sgntz, ix - sgntx)
    t1 = t2 = t3 = HUGE
    if abs(iz - m.zsi) > m.epsSolver or abs(ix - m.xsi) > m.epsSolver:
        if tv <= te + dx * sref3 and te <= tv + dz * sref3 and te >= tev and tv >= tev:
            ta = tev + te - tv
            tb = tev - te + tv
            t1 = ((tb * dz2i + ta * dx2i)
                  + _sqrt(4.0 * sref3 * sref3 * (dz2i + dx2i)
                          - dz2i * dx2i * (ta - tb) * (ta - tb))) / (dz2i + dx2i)
        elif (te - tev) <= dz * dz * sref3 / math.sqrt(dx * dx + dz * dz) and te > tev:
            r = (te - tev) / dz
            t2 = te + dx * _sqrt(sref3 * sref3 - r * r)
        elif (tv - tev) <= dx * dx * sref3 / math.sqrt(dx * dx + dz * dz) and tv > tev:
            r = (tv - tev) / dx
            t3 = tv + dz * _sqrt(sref3 * sref3 - r * r)
    else:
        if tv < te + dx * sref3 and te < tv + dz * sref3 and te >= tev and tv >= tev:
            ta = tauev + taue - tauv
            tb = tauev - taue + tauv
            apoly = dz2i + dx2i
            bpoly = (4.0 * (sgnrx * txc * dxi + sgnrz * tzc * dzi)
                     - 2.0 * (ta * dx2i + tb * dz2i))
            cpoly = ((ta * ta * dx2i) + (tb * tb * dz2i)
                     - 4.0 * (sgnrx * txc * dxi * ta + sgnrz * tzc * dzi * tb)
                     + 4.0 * (m.szero * m.szero - sref3 * sref3))
            dpoly = bpoly * bpoly - 4.0 * apoly * cpoly
            if dpoly >= 0.0:
                t1 = 0.5 * (math.sqrt(dpoly) - bpoly) / apoly + t0c
            if t1 < tv or t1 < te:
                t1 = HUGE
    t2d = min(t1, t2, t3)
    return min(t, t1d, t2d)


def noinit2(m, tv, te, tev, s1, s2, s3):
    """fteik_localSolver2d_noInit64f, localSolver.F90:123-158, one node."""
    temtv = te - tv
    t12min = min(tv + m.dz * s1, te + m.dx * s2)
    t1_2d = HUGE
    if temtv < m.dz * s3 and -temtv < m.dx * s3:
        sref2 = s3 * s3
        ta = tev + temtv
        tb = tev - temtv
        tab = ta - tb
        tab2 = tab * tab
        four_sref2 = 4.0 * sref2
        t1_2d = ((tb * m.dz2i + ta * m.dx2i)
                 + _sqrt(four_sref2 * m.dz2i_p_dx2i - m.dz2i_dx2i * tab2)) * m.dz2i_p_dx2i_inv
    return min(t12min, t1_2d)


def solve2(n, h, slow, src, eps, nsweep):
    """fteik_solver2d_solveSourceLSM, solver2D.F90:782-978 (the convergence
    test there never fires, so nsweep passes always run)."""
    nz, nx = n
    src_i, src_a = snap(n, h, src, is3d=False)
    zsi, xsi = src_i
    szero = slow[(xsi - 1) * (nz - 1) + zsi - 1]
    m = Mesh2(h, src_i, src_a, szero, eps)
    tt = [HUGE] * (nz * nx)
    for dj in (0, 1):               # ts4 / dest, localSolver.F90:338-345
        for di in (0, 1):
            tt[(xsi + dj - 1) * nz + zsi + di - 1] = m.tana(zsi + di, xsi + dj)
    # four natural-order initialisation sweeps (solver2D.F90:825-867); the
    # flipped ranges start at min(si + 1, n - 1), as in 3D
    xs_up, zs_up = range(max(2, xsi), nx + 1), range(max(2, zsi), nz + 1)
    xs_dn = range(min(xsi + 1, nx - 1), 0, -1)
    zs_dn = range(min(zsi + 1, nz - 1), 0, -1)
    for sweep, xs, zs in ((1, xs_up, zs_up), (2, xs_dn, zs_up), (3, xs_up, zs_dn),
                          (4, xs_dn, zs_dn)):
        for ix in xs:
            for iz in zs:
                v = init2(m, n, slow, tt, sweep, iz, ix)
                g = (ix - 1) * nz + iz - 1
                tt[g] = min(tt[g], v)
    for _ in range(nsweep):
        for sweep in range(1, 5):
            sgntz, sgntx, sgnvz, sgnvx = SIGNS2[sweep]
            for level in range(2, nx + nz + 1):
                out = []
                for i in range(max(1, level - nz), min(nx, level - 1) + 1):
                    ix = i if sgntx == 1 else nx + 1 - i
                    iz = level - i if sgntz == 1 else nz + 1 - (level - i)
                    # isUpdateNode (solver2D.F90:377-430, linit false)
                    okx = ix > 1 if sgntx == 1 else ix < nx
                    okz = iz > 1 if sgntz == 1 else iz < nz
                    if not (okx and okz):
                        continue
                    # prefetchSlowness64f (:431-520): cells upwind of the node
                    izc = iz - 1 if sgntz == 1 else iz
                    ixc = ix - 1 if sgntx == 1 else ix
                    s1 = min(slow[(max(ix - 1, 1) - 1) * (nz - 1) + izc - 1],
                             slow[(min(ix, nx - 1) - 1) * (nz - 1) + izc - 1])
                    s2 = min(slow[(ixc - 1) * (nz - 1) + max(iz - 1, 1) - 1],
                             slow[(ixc - 1) * (nz - 1) + min(iz, nz - 1) - 1])
                    s3 = slow[(ixc - 1) * (nz - 1) + izc - 1]
                    # prefetchTravelTimes64f (:521-610)
                    tv = tt[(ix - 1) * nz + iz - sgntz - 1]
                    te = tt[(ix - sgntx - 1) * nz + iz - 1]
                    tev = tt[(ix - sgntx - 1) * nz + iz - sgntz - 1]
                    out.append(((ix - 1) * nz + iz - 1, noinit2(m, tv, te, tev, s1, s2, s3)))
                for g, v in out:    # updateTravelTimes64f (:611-650)
                    tt[g] = min(tt[g], v)
    return np.array(tt), src_i, src_a


# ---------------------------------------------------------------- tests --
CASES3 = [
    # (n = (nz, nx, ny), h = (dz, dx, dy), source (z, x, y), eps, nsweep, model)
    ((9, 10, 11), (25.0, 25.0, 25.0), (97.3, 121.9, 150.2), 5.0, 2, "grf"),
    ((8, 9, 7), (20.0, 30.0, 25.0), (61.0, 117.5, 70.1), 2.0, 2, "grf"),
    ((7, 8, 9), (50.0, 50.0, 50.0), (0.0, 180.0, 200.0), 5.0, 1, "linear"),   # surface nudge
    ((7, 7, 7), (40.0, 40.0, 40.0), (239.0, 10.0, 230.0), 3.0, 2, "grf"),    # last cells
    ((6, 7, 8), (30.0, 30.0, 30.0), (60.0, 90.0, 120.0), 5.0, 2, "grf"),     # on a node
    ((9, 8, 7), (25.0, 25.0, 25.0), (100.0, 80.0, 70.0), 0.5, 3, "grf"),     # small eps
]


def _cells3(n, h, model, seed):
    """Cell slowness, z fastest (the models are shaped (ny-1, nx-1, nz-1))."""
    nz, nx, ny = n
    if model == "linear":
        v = linear_vz_cells(nz, nx, ny, h[0])
    else:
        v = layered_grf_cells(nz, nx, ny, seed=seed, min_cells=1, corr=2.0)
    return np.ascontiguousarray(1.0 / v, dtype=np.float64).ravel()


@pytest.mark.parametrize("case", range(len(CASES3)))
def test_3d_transcription_matches_oracle_bitwise(case):
    n, h, src, eps, nsweep, model = CASES3[case]
    slow = _cells3(n, h, model, seed=30 + case)
    si_o, sa_o = O.source_snap(True, n, (0.0, 0.0, 0.0), h, src)
    tt_o, _ = O.solve3d(n, h, slow, si_o, sa_o, eps=eps, nsweep=nsweep, level_set=True,
                        nthreads=2)
    tt_p, si_p, sa_p = solve3(n, h, list(slow), src, eps, nsweep)
    assert si_p == tuple(si_o) and sa_p == tuple(sa_o)
    assert np.all(tt_p < HUGE)
    np.testing.assert_array_equal(tt_p, tt_o)


CASES2 = [
    ((15, 17), (10.0, 10.0), (61.3, 83.7), 5.0, 2),
    ((12, 14), (20.0, 15.0), (0.0, 100.0), 3.0, 2),      # surface nudge
    ((11, 13), (10.0, 10.0), (100.0, 120.0), 2.0, 3),    # last cells
    ((13, 11), (25.0, 25.0), (150.0, 125.0), 1.0, 2),    # on a node, small eps
]


@pytest.mark.parametrize("case", range(len(CASES2)))
def test_2d_transcription_matches_oracle_bitwise(case):
    n, h, src, eps, nsweep = CASES2[case]
    nz, nx = n
    rng = np.random.default_rng(40 + case)
    zc = (np.arange(nz - 1) + 0.5) * h[0]
    v = (3000.0 + 2.0 * zc)[:, None] * (1.0 + 0.05 * rng.standard_normal((nz - 1, nx - 1)))
    slow = np.ascontiguousarray((1.0 / v).ravel(order="F"), dtype=np.float64)
    si_o, sa_o = O.source_snap(False, (nz, nx, 1), (0.0, 0.0, 0.0), (h[0], h[1], 1.0),
                               (src[0], src[1], 0.0))
    tt_o, _ = O.solve2d(n, h, slow, si_o[:2], sa_o[:2], eps=eps, nsweep=nsweep)
    tt_p, si_p, sa_p = solve2(n, h, list(slow), src, eps, nsweep)
    assert si_p == tuple(si_o[:2]) and sa_p == tuple(sa_o[:2])
    assert np.all(tt_p < HUGE)
    np.testing.assert_array_equal(tt_p, tt_o)
