"""Generalised Gaussians for the Poisson solvers' compensation charges.

Mirrors ``Gaussian(gd, a=19, center)`` of gpaw/utilities/gauss.py:193-260 for
L = 0 .. 8 (l <= 2), with coordinates as in gpaw/utilities/tools.py:106-125:

    g_L(r) = 1/sqrt(4 pi) l! / (2l + 1)! (4a)^(l + 3/2) exp(-a r^2) r^l Y_L

with the real spherical harmonics Y_L in GPAW's order (1; y, z, x; xy, yz,
3z^2 - r^2, xz, x^2 - y^2), and its potential (the solution of
Laplace v = -4 pi g_L vanishing at infinity), in closed form

    v_L(r) = 4 sqrt(pi) / (2l + 1) r^l Y_L
             [sqrt(pi) erf(sqrt(a) r) - S_l(r)] / r^(2l + 1),
    S_0 = 0,  S_1 = 2 sqrt(a) r e^(-a r^2),
    S_2 = (2 sqrt(a) r + 4/3 a^(3/2) r^3) e^(-a r^2),

which follows from the multipole expansion of the Gaussian's potential.
The monopole neutralises charged zero-boundary densities (gpaw/poisson.py:
249-299); the moments up to L = 8 serve the moment corrections of the
extended solver (gpaw/poisson_extended.py).  Built once per centre on the
host (setup, like the stencil tables) and uploaded; every per-solve use is
device arithmetic.
"""
from math import factorial, pi, sqrt

import numpy as np
from scipy.special import erf

# r^l Y_L as (normalisation, polynomial) of the Cartesian components
_NORM = [sqrt(1 / (4 * pi))] + [sqrt(3 / (4 * pi))] * 3 + \
    [sqrt(15 / (4 * pi)), sqrt(15 / (4 * pi)), sqrt(5 / (16 * pi)),
     sqrt(15 / (4 * pi)), sqrt(15 / (16 * pi))]


def rlY_L(L, x, y, z, r2):
    """r^l Y_L(x, y, z) for L <= 8 (gpaw/spherical_harmonics.py order)."""
    poly = [lambda: 1.0, lambda: y, lambda: z, lambda: x, lambda: x * y,
            lambda: y * z, lambda: 3 * z * z - r2, lambda: x * z,
            lambda: x * x - y * y]
    if not 0 <= L < len(poly):
        raise NotImplementedError('moments up to L = 8 (l <= 2)')
    return _NORM[L] * poly[L]()


def l_of(L):
    return 0 if L == 0 else (1 if L < 4 else 2)


class Gaussian:
    def __init__(self, gd, a=19., center=None):
        self.gd = gd
        origin = 0.5 * gd.cell_cv.sum(0) if center is None else center
        r_vG = gd.get_grid_point_distance_vectors(np.array(origin))
        r2 = np.sum(r_vG ** 2, axis=0)
        self.r2 = np.where(r2 < 1e-12, 1e-12, r2)
        self.xyz = r_vG
        self.r = np.sqrt(self.r2)
        if center is None:
            self.a = 4 * a * (gd.icell_cv ** 2).sum(1).max()
        else:
            cell_center = gd.cell_cv.sum(1) / 2
            r_min = (cell_center - np.abs(center - cell_center)).min()
            self.a = a / r_min ** 2
        self.exp_ar2 = np.exp(-self.a * self.r2)
        self.erf_sar = erf(sqrt(self.a) * self.r)

    def Y_L(self, L):
        """r^l Y_L on the grid: the weight of the L-th moment
        (gpaw/utilities/gauss.py:128-160, 245-248)."""
        x, y, z = self.xyz
        return rlY_L(L, x, y, z, self.r2)

    def get_gauss(self, L):
        a = self.a
        if L == 0:   # the monopole in the reference's own arrangement
            return sqrt(a ** 3 * 4) / pi * self.exp_ar2
        l = l_of(L)
        c = (1 / sqrt(4 * pi) * factorial(l) / factorial(2 * l + 1) *
             (4 * a) ** (l + 1.5))
        return c * self.exp_ar2 * self.Y_L(L)

    def get_gauss_pot(self, L):
        if L == 0:
            return 2.0 * 1.7724538509055159 * self.erf_sar / self.r
        a = self.a
        l = l_of(L)
        r = self.r
        sa = sqrt(a)
        if l == 0:
            s = 0.0
        elif l == 1:
            s = 2 * sa * r * self.exp_ar2
        else:
            s = (2 * sa * r + 4.0 / 3.0 * a * sa * r ** 3) * self.exp_ar2
        return (4 * sqrt(pi) / (2 * l + 1) * self.Y_L(L) *
                (sqrt(pi) * self.erf_sar - s) / r ** (2 * l + 1))

    def get_moment(self, n, L):
        """gpaw/utilities/gauss.py:245-248: integrate(n r^l Y_L)."""
        return float((n * self.Y_L(L)).sum() * self.gd.dv)

    def remove_moment(self, n, L, q=None):
        """gpaw/utilities/gauss.py:250-263 (host arrays)."""
        if q is None:
            q = self.get_moment(n, L)
        if abs(q) < 1e-7:
            return 0.
        n -= q * self.get_gauss(L)
        return q * self.get_gauss_pot(L)
