"""Seeded synthetic inputs for the pressure-Poisson workloads.

The reference publishes no benchmark or dataset; its Poisson coefficient is the face
value of 1/rho (DENF_ZI, 1d.f:2987-2994) and its right-hand side the velocity
divergence (DIVGS, 1d.f:3180).  The 2-D workload is a 1/rho field with rho = 1 in
the liquid and rho = rho_bubble inside seeded circular bubbles, and an i.i.d.
Gaussian right-hand side with its mean removed.  Random numbers come from numpy's
PCG64 generator with a fixed seed per workload.
"""
from dataclasses import dataclass

import numpy as np


@dataclass
class PoissonCase:
    nx: int
    ny: int
    hx: float
    hy: float
    rho: np.ndarray     # (ny, nx) cell densities
    f: np.ndarray       # (ny, nx) right-hand side
    bx: np.ndarray      # (ny, nx)   beta on the face left of cell i (periodic)
    by: np.ndarray      # (ny+1, nx) beta on the face below row j; row ny is the top wall


def face_beta(rho):
    """Face coefficients beta = 1/rho_face with rho_face the mean of the two cells
    (the reference interpolates density to faces and inverts it, 1d.f:2987-2994).
    Wall faces take the adjacent cell's value (the reference copies DENF_ZI(N3M) to
    the top face, 1d.f:2991-2992)."""
    ny, nx = rho.shape
    bx = 2.0 / (rho + np.roll(rho, 1, axis=1))
    by = np.empty((ny + 1, nx))
    by[1:ny] = 2.0 / (rho[1:] + rho[:-1])
    by[0] = 1.0 / rho[0]
    by[ny] = 1.0 / rho[ny - 1]
    return bx, by


def bubble_density(nx, ny, *, nbubbles=64, rmin=8.0, rmax=48.0, rho_in=1000.0, rho_out=1.0, seed=2024):
    """rho_out everywhere, rho_in inside nbubbles circles with centres uniform in the
    domain and radii uniform in [rmin, rmax] cells (x periodic)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    cx = rng.uniform(0.0, nx, nbubbles)
    cy = rng.uniform(0.0, ny, nbubbles)
    rr = rng.uniform(rmin, rmax, nbubbles)
    xs = np.arange(nx) + 0.5
    ys = np.arange(ny) + 0.5
    rho = np.full((ny, nx), rho_out)
    for k in range(nbubbles):
        dx = np.abs(xs - cx[k])
        dx = np.minimum(dx, nx - dx)
        dy = ys - cy[k]
        inside = (dy[:, None] ** 2 + dx[None, :] ** 2) <= rr[k] ** 2
        rho[inside] = rho_in
    return rho


def gaussian_rhs(nx, ny, seed=7):
    rng = np.random.Generator(np.random.PCG64(seed))
    f = rng.standard_normal((ny, nx))
    return f - f.mean()


def bubble_poisson_case(n=1024, *, ny=None, nbubbles=64, rmin=None, rmax=None, rho_in=1000.0,
                        seed=2024, rhs_seed=7):
    """The 2-D workload: unit-width domain of n x ny cells (h = 1/n), 64 seeded
    bubbles of density ratio 1000 with radii 8-48 cells at n = 1024; at other n the
    radii scale with n (the same bubbles in the unit domain)."""
    nx = n
    ny = n if ny is None else ny
    h = 1.0 / nx
    rmin = 8.0 * nx / 1024.0 if rmin is None else rmin
    rmax = 48.0 * nx / 1024.0 if rmax is None else rmax
    rho = bubble_density(nx, ny, nbubbles=nbubbles, rmin=rmin, rmax=rmax, rho_in=rho_in, seed=seed)
    bx, by = face_beta(rho)
    f = gaussian_rhs(nx, ny, rhs_seed)
    return PoissonCase(nx=nx, ny=ny, hx=h, hy=h, rho=rho, f=f, bx=bx, by=by)
