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

SIGMA = 1.5  # UnitCube default --sigma (tests/UnitCube.cpp:28)


class Workload:
    def __init__(self, name, disc, velocity, rhs, pml, interior, meta):
        self.name = name
        self.disc = disc
        self.velocity = velocity      # (nz, ny, nx) float64
        self.rhs = rhs                # (nz, ny, nx, k) complex128
        self.pml = pml
        self.interior = interior
        self.meta = meta

    @property
    def k(self):
        return self.rhs.shape[-1]

    def velocity_grid(self):
        return DistUniformGrid(self.disc.nx, self.disc.ny, self.disc.nz, 1, np.float64, self.velocity)

    def rhs_grid(self):
        return DistUniformGrid(self.disc.nx, self.disc.ny, self.disc.nz, self.k, np.complex128, self.rhs.copy())


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


CONFIGS = {
    "plain_bump_50": plain_bump,
    "smooth_anomalies_116": smooth_anomalies,
    # profiling-sized member of the same family (factors ~0.5 GB, above L2)
    "smooth_anomalies_56": lambda: smooth_anomalies(interior=(40, 40, 40), pml=8, freq=4.0, k=16),
}
