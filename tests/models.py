"""Seeded synthetic velocity models and source sets used by the tests and the
benchmark (the reference publishes no data sets; shapes follow the
configurations the benchmark names)."""
import numpy as np


def linear_vz_cells(nz, nx, ny, h, v0=3000.0, grad=0.5):
    """Cell velocities v(z) = v0 + grad*z_c at the cell centre, natural order
    (z fastest), shape (ny-1, nx-1, nz-1)."""
    zc = (np.arange(nz - 1) + 0.5) * h
    v = v0 + grad * zc
    return np.broadcast_to(v, (max(ny - 1, 1), nx - 1, nz - 1)).copy()


def gaussian_field(shape, corr_cells, seed):
    """Unit-variance Gaussian random field with a Gaussian correlation of
    corr_cells cells (FFT-filtered white noise), clipped to +-3 sigma."""
    rng = np.random.default_rng(seed)
    w = rng.standard_normal(shape)
    k = [np.fft.fftfreq(n) for n in shape]
    kk = np.meshgrid(*k, indexing="ij")
    k2 = sum(q * q for q in kk)
    filt = np.exp(-0.5 * k2 * (2.0 * np.pi * corr_cells) ** 2)
    f = np.real(np.fft.ifftn(np.fft.fftn(w) * filt))
    f = (f - f.mean()) / f.std()
    return np.clip(f, -3.0, 3.0)


def layered_grf_cells(nz, nx, ny, seed=2, vels=(3000.0, 4000.0, 5000.0, 6000.0),
                      min_cells=5, amp=0.05, corr=10.0):
    """4 layers with seeded interface depths (>= min_cells cells each) times
    (1 + amp * GRF); shape (ny-1, nx-1, nz-1), natural order."""
    nzc = nz - 1
    rng = np.random.default_rng(seed)
    nl = len(vels)
    mc = max(1, min(min_cells, nzc // nl))
    # each layer gets mc cells plus a seeded share of the rest
    extra = rng.multinomial(nzc - nl * mc, np.ones(nl) / nl)
    th = mc + extra
    edges = np.concatenate([[0], np.cumsum(th)])
    vz = np.empty(nzc)
    for i in range(nl):
        vz[edges[i]:edges[i + 1]] = vels[i]
    g = gaussian_field((ny - 1, nx - 1, nzc), corr, seed)
    return vz[None, None, :] * (1.0 + amp * g)


def interior_source(n, h, seed):
    rng = np.random.default_rng(seed)
    nz, nx, ny = n
    return (rng.uniform(0.1, 0.9) * (nz - 1) * h[0], rng.uniform(0.1, 0.9) * (nx - 1) * h[1],
            rng.uniform(0.1, 0.9) * (ny - 1) * h[2])


def station_tables(nz, nx, ny, h, nsta, v=3000.0, seed=11):
    """Constant-velocity travel-time tables from nsta surface stations to every
    grid node, FP32, shape (nsta, nz*nx*ny), node index z fastest."""
    rng = np.random.default_rng(seed)
    sx = rng.uniform(0, (nx - 1) * h, nsta)
    sy = rng.uniform(0, (ny - 1) * h, nsta)
    z = np.arange(nz) * h
    x = np.arange(nx) * h
    y = np.arange(ny) * h
    Y, X, Z = np.meshgrid(y, x, z, indexing="ij")      # [ny][nx][nz] -> z fastest
    Z, X, Y = Z.ravel(), X.ravel(), Y.ravel()
    t = np.empty((nsta, Z.size), np.float32)
    for i in range(nsta):
        t[i] = (np.sqrt(Z ** 2 + (X - sx[i]) ** 2 + (Y - sy[i]) ** 2) / v).astype(np.float32)
    return t


def synthetic_events(tables, nev, seed=5, noise=0.02, outlier_frac=0.05):
    """Events at random grid nodes: picks = table times + origin time U[0,60]
    + N(0, noise), a fraction of picks replaced by exact + U[-1, 1] s.
    Returns (true node indices, picks [nev][ntf] FP64)."""
    rng = np.random.default_rng(seed)
    ntf, ngrd = tables.shape
    true = rng.integers(0, ngrd, nev)
    exact = tables[:, true].T.astype(np.float64) + rng.uniform(0, 60, (nev, 1))
    picks = exact + rng.normal(0, noise, exact.shape)
    out = rng.random(exact.shape) < outlier_frac
    picks[out] = exact[out] + rng.uniform(-1, 1, out.sum())
    return true, picks


def linear_gradient_tables(nz, nx, ny, h, nsta, v0=3000.0, grad=0.5, seed=11):
    """Analytic travel times in v(z) = v0 + grad z (analytic.F90:853-890 form,
    T = acosh(1 + grad^2 r^2 / (2 v(zs) v(z))) / grad) from nsta surface
    stations to every node; FP32 tables (nsta, nz*nx*ny), z fastest, and the
    station positions (z, x, y)."""
    rng = np.random.default_rng(seed)
    sx = rng.uniform(0, (nx - 1) * h, nsta)
    sy = rng.uniform(0, (ny - 1) * h, nsta)
    sz = np.zeros(nsta)
    z = np.arange(nz) * h
    x = np.arange(nx) * h
    y = np.arange(ny) * h
    Y, X, Z = np.meshgrid(y, x, z, indexing="ij")
    Z, X, Y = Z.ravel(), X.ravel(), Y.ravel()
    t = np.empty((nsta, Z.size), np.float32)
    for i in range(nsta):
        r2 = (Z - sz[i]) ** 2 + (X - sx[i]) ** 2 + (Y - sy[i]) ** 2
        t[i] = (np.arccosh(1.0 + grad ** 2 * r2 / (2.0 * (v0 + grad * sz[i]) * (v0 + grad * Z))) / grad
                ).astype(np.float32)
    return t, (sz, sx, sy)
