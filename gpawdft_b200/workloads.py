"""Seeded synthetic inputs for the grid hot path's benchmark workloads.

Lengths are in Bohr (1 Angstrom = 1 / 0.52917721 Bohr), as in the reference.
Densities are sums of normalised 3D Gaussians
``q (2 pi s^2)^(-3/2) exp(-|r - c|^2 / (2 s^2))`` on the grid points of a
zero-boundary cell (grid point coordinates as in
gpaw/grid_descriptor.py:629-636: index + beg_c times h), re-centred by a
uniform shift so that ``sum(rho) * dv == 0`` exactly, which keeps the Poisson
solver on its neutral branch (gpaw/poisson.py:234-236).
"""
import numpy as np

BOHR_PER_ANGSTROM = 1.0 / 0.52917721


def gaussian_density(N, h_ang, n_gauss, seed, sigma_range=(0.5, 1.5),
                     log_sigma=False, charges='pm1', pbc=False):
    """Neutral Gaussian-sum density on an N^3 grid (extent N-1 when zero-BC).

    Returns (rho, cell_length_bohr).  ``charges='pm1'``: half +1, half -1;
    ``'normal'``: N(0, 1) charges.  Widths uniform (or log-uniform) in
    ``sigma_range`` Angstrom; centres uniform in the cell.
    """
    rng = np.random.default_rng(seed)
    h = h_ang * BOHR_PER_ANGSTROM
    L = N * h
    n = N if pbc else N - 1
    beg = 0 if pbc else 1
    x = (np.arange(n) + beg) * h
    s_lo, s_hi = (v * BOHR_PER_ANGSTROM for v in sigma_range)
    if log_sigma:
        sig = np.exp(rng.uniform(np.log(s_lo), np.log(s_hi), n_gauss))
    else:
        sig = rng.uniform(s_lo, s_hi, n_gauss)
    cen = rng.uniform(0.0, L, (n_gauss, 3))
    if charges == 'pm1':
        q = np.array([1.0, -1.0] * ((n_gauss + 1) // 2))[:n_gauss]
    else:
        q = rng.standard_normal(n_gauss)
    rho = np.zeros((n, n, n))
    for i in range(n_gauss):
        s2 = sig[i] ** 2
        gx = np.exp(-(x - cen[i, 0]) ** 2 / (2 * s2))
        gy = np.exp(-(x - cen[i, 1]) ** 2 / (2 * s2))
        gz = np.exp(-(x - cen[i, 2]) ** 2 / (2 * s2))
        norm = q[i] * (2 * np.pi * s2) ** -1.5
        rho += norm * gx[:, None, None] * gy[None, :, None] * gz[None, None, :]
    rho -= rho.mean()
    return rho, L


def random_grids(shape, dtype, seed):
    """i.i.d. N(0, 1) grids (complex: independent real and imaginary parts)."""
    rng = np.random.default_rng(seed)
    a = rng.standard_normal(shape)
    if np.dtype(dtype).kind == 'c':
        a = a + 1j * rng.standard_normal(shape)
    return a.astype(dtype)
