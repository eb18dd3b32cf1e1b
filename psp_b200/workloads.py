"""Seeded synthetic Helmholtz workloads.

The reference's own drivers build analytic velocity models and Gaussian
point sources on the unit cube (tests/UnitCube.cpp:74-542).  The workloads
here follow the same construction with seeded parameters:

* the grid size ``n`` includes the PML points (discretization.hpp:44), so an
  ``interior`` grid with ``pml`` points per face has ``n = interior + 2*pml``,
  spacing ``h = 1/(interior+1)`` and box width ``w = (n+1) h``;
* grid index ``i`` sits at the physical coordinate ``(i - pml + 1) h``, so the
  interior points cover (0, 1);
* sources are Gaussians of width 2h with the reference's negative sign
  (UnitCube.cpp:531), centred at seeded interior points at least PML+2 points
  from every face;
* seeds come from ``numpy.random.Generator(PCG64(seed))``.
"""
import math

import numpy as np

from . import PML, Discretization, DistUniformGrid

SIGMA = 1.5  # UnitCube default --sigma (tests/UnitCube.cpp:28), for velocities near 1
# PML amplitude of the velocity models in km/s: the reference's Overthrust
# example (velocities of a few km/s) runs with --sigma 7.5
# (doc/source/examples.rst:35; its default is 30, examples/Overthrust.cpp:33).
# The stretch 1 + i (sigma/eta)(x/b)^2 (2 pi/omega) attenuates a wave of
# speed c by exp(-2 pi sigma / (3 c)) across the layer, so the amplitude has
# to grow with the velocities for the fast layers to be absorbed.
SIGMA_KM = 7.5


class Workload:
    """A velocity model and its right-hand sides.  ``rhs`` is either the
    dense (nz, ny, nx, k) complex128 array or a :class:`SeparableSources`,
    in which case the dense array is built on first use (``rhs``) and can be
    built directly on a CUDA device (``rhs_torch``) without a host copy."""

    def __init__(self, name, disc, velocity, rhs, pml, interior, meta):
        self.name = name
        self.disc = disc
        self.velocity = velocity      # (nz, ny, nx) float64
        self._rhs = rhs
        self.pml = pml
        self.interior = interior
        self.meta = meta

    @property
    def rhs(self):
        """(nz, ny, nx, k) complex128."""
        if isinstance(self._rhs, SeparableSources):
            self._rhs = self._rhs.dense()
        return self._rhs

    @property
    def k(self):
        return self._rhs.k if isinstance(self._rhs, SeparableSources) else self._rhs.shape[-1]

    def rhs_torch(self, device, out=None, cols=None):
        """The right-hand sides (or the sources ``cols``, a range) as a CUDA
        complex128 tensor of nx*ny*nz*len(cols) entries (natural order,
        interleaved per point), written into ``out`` when given."""
        import torch
        if isinstance(self._rhs, SeparableSources):
            return self._rhs.torch(device, out, cols)
        a = self._rhs if cols is None else self._rhs[..., cols]
        t = torch.from_numpy(np.ascontiguousarray(a).reshape(-1)).to(device)
        if out is None:
            return t
        out.copy_(t)
        return out

    def rhs_host(self, cols=None):
        """The right-hand sides (or the sources ``cols``) as a C-contiguous
        (nz, ny, nx, len(cols)) complex128 array."""
        if isinstance(self._rhs, SeparableSources):
            return self._rhs.dense(cols)
        return np.ascontiguousarray(self._rhs if cols is None else self._rhs[..., cols])

    def velocity_grid(self):
        return DistUniformGrid(self.disc.nx, self.disc.ny, self.disc.nz, 1, np.float64, self.velocity)

    def rhs_grid(self):
        return DistUniformGrid(self.disc.nx, self.disc.ny, self.disc.nz, self.k, np.complex128, self.rhs.copy())


class SeparableSources:
    """k point sources whose fields are products gz(z) gy(y) gx(x) (the
    Gaussians of width 2h the reference's drivers use, UnitCube.cpp:485-542),
    kept as their 1-D factors: g[axis][r] is source r's factor along that
    axis, the field is -gz gy gx."""

    def __init__(self, gx, gy, gz):
        self.gx, self.gy, self.gz = (np.asarray(a, dtype=np.float64) for a in (gx, gy, gz))
        self.k = self.gx.shape[0]

    def dense(self, cols=None):
        cols = range(self.k) if cols is None else cols
        out = np.empty((self.gz.shape[1], self.gy.shape[1], self.gx.shape[1], len(cols)), dtype=np.complex128)
        for j, r in enumerate(cols):
            out[..., j] = -(self.gz[r][:, None, None] * self.gy[r][None, :, None] * self.gx[r][None, None, :])
        return out

    def torch(self, device, out=None, cols=None):
        import torch
        cols = list(range(self.k) if cols is None else cols)
        gx, gy, gz = (torch.from_numpy(a[cols].T.copy()).to(device) for a in (self.gx, self.gy, self.gz))
        nz, ny, nx, kk = gz.shape[0], gy.shape[0], gx.shape[0], len(cols)
        if out is None:
            out = torch.empty(nz * ny * nx * kk, dtype=torch.complex128, device=device)
        view = torch.view_as_real(out.view(nz, ny, nx, kk))
        view[..., 1].zero_()
        for z in range(nz):  # -(gz gy) gx, the rounding order of dense()
            torch.mul((gz[z][None, :] * gy)[:, None, :], gx[None, :, :], out=view[z, ..., 0])
            view[z, ..., 0].neg_()
        return out


def _axes(interior, pml):
    """Physical coordinates of the grid points along each axis."""
    out = []
    for m in interior:
        h = 1.0 / (m + 1)
        out.append((np.arange(m + 2 * pml) - pml + 1) * h)
    return out


def make_disc(interior, pml, omega, sigma=SIGMA, top_pml=True):
    ix, iy, iz = interior
    n = [m + 2 * pml for m in interior]
    w = [(nn + 1) / (m + 1.0) for nn, m in zip(n, interior)]
    bcs = (PML, PML, PML, PML, PML if top_pml else 1)
    return Discretization(omega, n[0], n[1], n[2], w[0], w[1], w[2], bcs=bcs, pml=(pml, pml, pml), sigma=sigma)


def gaussian_sources(interior, pml, k, rng):
    X, Y, Z = _axes(interior, pml)
    h = 1.0 / (max(interior) + 1)
    sig = 2.0 * h
    rhs = np.zeros((len(Z), len(Y), len(X), k), dtype=np.complex128)
    centres = []
    for r in range(k):
        c = []
        for m, ax in zip(interior, (X, Y, Z)):
            lo, hi = pml + 2, m + pml - 3
            i = rng.integers(lo, hi + 1)
            c.append(ax[i])
        centres.append(c)
        gx = np.exp(-((X - c[0]) ** 2) / (2 * sig ** 2))
        gy = np.exp(-((Y - c[1]) ** 2) / (2 * sig ** 2))
        gz = np.exp(-((Z - c[2]) ** 2) / (2 * sig ** 2))
        rhs[..., r] = -(gz[:, None, None] * gy[None, :, None] * gx[None, None, :])
    return rhs, centres


def _grid(interior, pml):
    X, Y, Z = _axes(interior, pml)
    return np.meshgrid(Z, Y, X, indexing="ij")


def plain_bump(interior=(40, 40, 40), pml=5, freq=4.0, k=4, seed=1001):
    """FP64 reference case: c = 1 + 0.3 exp(-|x-x0|^2/0.02), omega = 2 pi freq."""
    rng = np.random.Generator(np.random.PCG64(seed))
    Zc, Yc, Xc = _grid(interior, pml)
    x0 = rng.uniform(0.2, 0.8, size=3)
    r2 = (Xc - x0[0]) ** 2 + (Yc - x0[1]) ** 2 + (Zc - x0[2]) ** 2
    vel = 1.0 + 0.3 * np.exp(-r2 / 0.02)
    rhs, centres = gaussian_sources(interior, pml, k, rng)
    disc = make_disc(interior, pml, 2 * math.pi * freq)
    return Workload("plain_bump", disc, np.ascontiguousarray(vel), rhs, pml, interior,
                    dict(x0=x0.tolist(), sources=centres, freq=freq))


def smooth_anomalies(interior=(100, 100, 100), pml=8, freq=10.0, k=16, seed=1002, n_anom=6):
    """Background 1.0 plus seeded Gaussian anomalies (amplitude +-0.4, width
    0.05-0.15), clipped to [0.6, 1.8]; omega = 2 pi freq."""
    rng = np.random.Generator(np.random.PCG64(seed))
    Zc, Yc, Xc = _grid(interior, pml)
    vel = np.ones_like(Xc)
    anoms = []
    for _ in range(n_anom):
        c = rng.uniform(0.1, 0.9, size=3)
        amp = rng.uniform(-0.4, 0.4)
        wid = rng.uniform(0.05, 0.15)
        anoms.append((c.tolist(), amp, wid))
        r2 = (Xc - c[0]) ** 2 + (Yc - c[1]) ** 2 + (Zc - c[2]) ** 2
        vel += amp * np.exp(-r2 / (2 * wid ** 2))
    vel = np.clip(vel, 0.6, 1.8)
    rhs, centres = gaussian_sources(interior, pml, k, rng)
    disc = make_disc(interior, pml, 2 * math.pi * freq)
    return Workload("smooth_anomalies", disc, np.ascontiguousarray(vel), rhs, pml, interior,
                    dict(anomalies=anoms, sources=centres, freq=freq))


def small_case(interior=(12, 13, 14), pml=5, freq=2.0, k=3, seed=7, top_pml=True):
    """A few-second case for parity tests (uneven sides, leftover panel)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    Zc, Yc, Xc = _grid(interior, pml)
    x0 = rng.uniform(0.3, 0.7, size=3)
    r2 = (Xc - x0[0]) ** 2 + (Yc - x0[1]) ** 2 + (Zc - x0[2]) ** 2
    vel = 1.0 + 0.3 * np.exp(-r2 / 0.02)
    rhs, centres = gaussian_sources(interior, pml, k, rng)
    rhs += 0.1 * (rng.standard_normal(rhs.shape) + 1j * rng.standard_normal(rhs.shape))
    disc = make_disc(interior, pml, 2 * math.pi * freq, top_pml=top_pml)
    return Workload("small_case", disc, np.ascontiguousarray(vel), rhs, pml, interior,
                    dict(x0=x0.tolist(), sources=centres, freq=freq))


def layered_faults(interior=(80, 80, 60), pml=8, k=32, seed=1004, n_layers=8, ppw=10.0, perturb=0.03,
                   sigma=SIGMA_KM):
    """Differentiation case: 8 layers of 1.5-5.5 (km/s) whose interface
    depths jitter by +-15 % of the layer thickness, offset across two dipping
    planar faults; uniform spacing h = 1/(max interior + 1) (km), and omega
    chosen so the slowest layer has ``ppw`` points per wavelength; k point
    sources (Gaussians of width 2h) on the first plane below the top PML and
    receivers at every interior point of that plane.  ``meta`` holds the
    receiver indices (natural order) and the model the observed data come
    from (velocity perturbed by +-3 % with a seeded smooth pattern)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    n = [m + 2 * pml for m in interior]
    h = 1.0 / (max(interior) + 1)
    X, Y, Z = [(np.arange(nn) - pml + 1) * h for nn in n]
    Zc, Yc, Xc = np.meshgrid(Z, Y, X, indexing="ij")
    depth = Z[-1] - Z[0]
    speeds = np.linspace(1.5, 5.5, n_layers)
    thick = depth / n_layers
    tops = np.array([Z[0] + thick * (i + rng.uniform(-0.15, 0.15)) for i in range(1, n_layers)])
    shift = np.zeros_like(Zc)
    faults = []
    for _ in range(2):
        normal = np.array([rng.uniform(-1, 1), rng.uniform(-1, 1), rng.uniform(0.3, 0.8)])
        normal /= np.linalg.norm(normal)
        point = np.array([rng.uniform(0.3, 0.7), rng.uniform(0.3, 0.7), 0.5 * depth + Z[0]])
        throw = rng.uniform(0.5, 1.0) * 0.3 * thick
        side = (Xc - point[0]) * normal[0] + (Yc - point[1]) * normal[1] + (Zc - point[2]) * normal[2] > 0
        shift = shift + np.where(side, throw, 0.0)
        faults.append((normal.tolist(), point.tolist(), float(throw)))
    # the solver's z index 0 is the top face (sweep coordinate v = nz-1-z), so
    # depth grows with z and the slow layer sits at the surface
    layer = np.searchsorted(tops, Zc - shift)
    vel = np.ascontiguousarray(speeds[np.clip(layer, 0, n_layers - 1)])
    omega = 2 * math.pi * speeds[0] / (ppw * h)
    w = [(nn + 1) * h for nn in n]
    disc = Discretization(omega, n[0], n[1], n[2], w[0], w[1], w[2], bcs=(PML,) * 5, pml=(pml,) * 3, sigma=sigma)
    # sources and receivers on the first plane below the top PML (solver z index pml)
    zs = pml
    sig = 2.0 * h
    rhs = np.zeros((n[2], n[1], n[0], k), dtype=np.complex128)
    centres = []
    for r in range(k):
        ix = rng.integers(pml + 2, n[0] - pml - 2)
        iy = rng.integers(pml + 2, n[1] - pml - 2)
        centres.append((int(ix), int(iy), zs))
        gx = np.exp(-((X - X[ix]) ** 2) / (2 * sig ** 2))
        gy = np.exp(-((Y - Y[iy]) ** 2) / (2 * sig ** 2))
        gz = np.exp(-((np.arange(n[2]) - zs) * h) ** 2 / (2 * sig ** 2))
        rhs[..., r] = -(gz[:, None, None] * gy[None, :, None] * gx[None, None, :])
    yy, xx = np.meshgrid(np.arange(pml, n[1] - pml), np.arange(pml, n[0] - pml), indexing="ij")
    receivers = (xx + yy * n[0] + zs * n[0] * n[1]).reshape(-1)
    pattern = np.sin(3.1 * Xc / Xc.max() + 1.7) * np.cos(2.3 * Yc / Yc.max()) * np.sin(4.1 * Zc / Zc.max() + 0.4)
    observed_model = np.ascontiguousarray(vel * (1.0 + perturb * pattern))
    return Workload("layered_faults", disc, vel, rhs, pml, interior,
                    dict(receivers=receivers, observed_model=observed_model, faults=faults, h=h,
                         omega=omega, sources=centres, layer_tops=tops.tolist()))


def large_layered(interior=(200, 200, 100), pml=10, k=64, seed=1005, n_layers=12, ppw=10.0, n_faults=3,
                  sigma=SIGMA_KM):
    """Large case: 12 layers of 1.5-6.0 (km/s) whose interface depths jitter
    by +-15 % of the layer thickness, offset across three dipping planar
    faults and arched by one anticline (interfaces raised by a Gaussian
    ridge about a seeded horizontal fold axis); spacing h = 1/(max interior
    + 1) (km), omega for ``ppw`` points per wavelength in the slowest layer,
    and k Gaussian point sources (width 2h) at seeded interior points at
    least PML+2 points from every face.  The sources are kept separable, so
    the (nz, ny, nx, k) array (6 GB at k = 64) is only built when asked for."""
    rng = np.random.Generator(np.random.PCG64(seed))
    n = [m + 2 * pml for m in interior]
    h = 1.0 / (max(interior) + 1)
    X, Y, Z = [(np.arange(nn) - pml + 1) * h for nn in n]
    Zc, Yc, Xc = np.meshgrid(Z, Y, X, indexing="ij")
    depth = Z[-1] - Z[0]
    speeds = np.linspace(1.5, 6.0, n_layers)
    thick = depth / n_layers
    tops = np.array([Z[0] + thick * (i + rng.uniform(-0.15, 0.15)) for i in range(1, n_layers)])
    shift = np.zeros_like(Zc)
    faults = []
    width = [X[-1] - X[0], Y[-1] - Y[0]]
    for _ in range(n_faults):
        normal = np.array([rng.uniform(-1, 1), rng.uniform(-1, 1), rng.uniform(0.3, 0.8)])
        normal /= np.linalg.norm(normal)
        point = np.array([X[0] + rng.uniform(0.25, 0.75) * width[0], Y[0] + rng.uniform(0.25, 0.75) * width[1],
                          0.5 * depth + Z[0]])
        throw = rng.uniform(0.5, 1.0) * 0.3 * thick
        side = (Xc - point[0]) * normal[0] + (Yc - point[1]) * normal[1] + (Zc - point[2]) * normal[2] > 0
        shift = shift + np.where(side, throw, 0.0)
        faults.append((normal.tolist(), point.tolist(), float(throw)))
    # anticline: interfaces raised by amp * exp(-d^2 / (2 w^2)), d the
    # horizontal distance to the fold axis through `axis_point` at `azimuth`
    azimuth = rng.uniform(0, math.pi)
    axis_point = (X[0] + rng.uniform(0.3, 0.7) * width[0], Y[0] + rng.uniform(0.3, 0.7) * width[1])
    fold_amp = rng.uniform(1.0, 2.0) * thick
    fold_w = rng.uniform(0.1, 0.2) * max(width)
    dist = -(Xc - axis_point[0]) * math.sin(azimuth) + (Yc - axis_point[1]) * math.cos(azimuth)
    fold = fold_amp * np.exp(-dist ** 2 / (2 * fold_w ** 2))
    del dist
    # z index 0 is the top face (sweep coordinate v = nz-1-z): depth grows
    # with z and the slow layer sits at the surface
    layer = np.searchsorted(tops, Zc - shift + fold)
    vel = np.ascontiguousarray(speeds[np.clip(layer, 0, n_layers - 1)])
    del Xc, Yc, Zc, shift, fold, layer
    omega = 2 * math.pi * speeds[0] / (ppw * h)
    w = [(nn + 1) * h for nn in n]
    disc = Discretization(omega, n[0], n[1], n[2], w[0], w[1], w[2], bcs=(PML,) * 5, pml=(pml,) * 3, sigma=sigma)
    sig = 2.0 * h
    g = [np.zeros((k, nn)) for nn in n]
    centres = []
    for r in range(k):
        idx = [int(rng.integers(pml + 2, nn - pml - 2)) for nn in n]
        centres.append(idx)
        for a, (ax, i) in enumerate(zip((X, Y, Z), idx)):
            g[a][r] = np.exp(-((ax - ax[i]) ** 2) / (2 * sig ** 2))
    return Workload("large_layered", disc, vel, SeparableSources(*g), pml, interior,
                    dict(h=h, omega=omega, sources=centres, layer_tops=tops.tolist(), faults=faults,
                         anticline=dict(azimuth=azimuth, axis_point=list(axis_point), amplitude=fold_amp,
                                        width=fold_w)))


def batch_problems(count=48, seed=1003, sides=tuple(range(32, 97, 4)), pml=5, ppw_range=(8.0, 12.0),
                   k_range=(1, 8), n_anom=3):
    """Batching case: ``count`` independent problems, every side drawn from
    ``sides`` (points including a ``pml``-point PML per face), a smooth
    velocity in [0.6, 1.8] (background 1 plus seeded Gaussian anomalies),
    omega giving U[8, 12] points per wavelength at the slowest velocity on
    the coarsest axis, and k ~ U{1..8} Gaussian sources.  Returns
    batch.Problem objects (natural order: velocity nx*ny*nz, rhs
    nx*ny*nz x k)."""
    from .batch import Problem
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for i in range(count):
        n = [int(rng.choice(sides)) for _ in range(3)]
        interior = tuple(m - 2 * pml for m in n)
        Zc, Yc, Xc = _grid(interior, pml)
        vel = np.ones_like(Xc)
        for _ in range(n_anom):
            c = rng.uniform(0.15, 0.85, size=3)
            amp = rng.uniform(-0.4, 0.6)
            wid = rng.uniform(0.08, 0.2)
            vel += amp * np.exp(-((Xc - c[0]) ** 2 + (Yc - c[1]) ** 2 + (Zc - c[2]) ** 2) / (2 * wid ** 2))
        vel = np.clip(vel, 0.6, 1.8)
        h = 1.0 / (min(interior) + 1)
        ppw = rng.uniform(*ppw_range)
        omega = 2 * math.pi * float(vel.min()) / (ppw * h)
        k = int(rng.integers(k_range[0], k_range[1] + 1))
        rhs, _ = gaussian_sources(interior, pml, k, rng)
        disc = make_disc(interior, pml, omega)
        out.append(Problem(disc, np.ascontiguousarray(vel).reshape(-1),
                           np.ascontiguousarray(rhs).reshape(-1, k), "batch_%02d" % i,
                           dict(sides=n, ppw=ppw, k=k)))
    return out


CONFIGS = {
    "plain_bump_50": plain_bump,
    "smooth_anomalies_116": smooth_anomalies,
    # profiling-sized member of the same family (factors ~0.5 GB, above L2)
    "smooth_anomalies_56": lambda: smooth_anomalies(interior=(40, 40, 40), pml=8, freq=4.0, k=16),
    "layered_faults_96": layered_faults,
    # test-sized member of the same family
    "layered_faults_24": lambda: layered_faults(interior=(20, 20, 16), pml=5, k=4, ppw=12.0),
    # the large configuration: 200 x 200 x 100 interior + 10 PML points per face
    "large_220": large_layered,
    # a small member of the large family (same generator, same ppw and PML)
    "large_60": lambda: large_layered(interior=(40, 40, 20), pml=10, k=16),
}
