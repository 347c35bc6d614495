"""Generalised Gaussians, L = 0 .. 8 (oracle restatement).

Restates gpaw/utilities/gauss.py:193-263 (``Gaussian``): the monopole that
FDPoissonSolver uses to neutralise charged zero-boundary systems
(gpaw/poisson.py:249-299), and the moments up to l = 2 with their potentials
that the extended solver's moment corrections remove (remove_moment), with
coordinates from gpaw/utilities/tools.py:106-125.  The potentials are the
closed forms of the Gaussians' multipole potentials,
v_L = 4 sqrt(pi) / (2l + 1) r^l Y_L [sqrt(pi) erf(sqrt(a) r) - S_l] / r^(2l+1)
with S_0 = 0, S_1 = 2 sqrt(a) r e^(-a r^2), S_2 = (2 sqrt(a) r +
4/3 a^(3/2) r^3) e^(-a r^2).  Test infrastructure only.
"""
from math import factorial, pi, sqrt

import numpy as np
from scipy.special import erf


def coordinates(gd, origin=None, tiny=1e-12):
    """gpaw/utilities/tools.py:106-125."""
    if origin is None:
        origin = 0.5 * gd.cell_cv.sum(0)
    r_vG = gd.get_grid_point_distance_vectors(np.array(origin))
    r2_G = np.sum(r_vG ** 2, axis=0)
    r2_G = np.where(r2_G < tiny, tiny, r2_G)
    return r_vG, r2_G


class Gaussian:
    def __init__(self, gd, a=19., center=None):
        self.gd = gd
        self.xyz, self.r2 = coordinates(gd, center)
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
        """r^l Y_L (gpaw/spherical_harmonics.py order) on the grid."""
        x, y, z = self.xyz
        r2 = self.r2
        n1, n2a, n2b, n2c = (sqrt(3 / (4 * pi)), sqrt(15 / (4 * pi)),
                             sqrt(5 / (16 * pi)), sqrt(15 / (16 * pi)))
        return [lambda: sqrt(1 / (4 * pi)) + 0 * r2, lambda: n1 * y,
                lambda: n1 * z, lambda: n1 * x, lambda: n2a * x * y,
                lambda: n2a * y * z, lambda: n2b * (3 * z * z - r2),
                lambda: n2a * x * z, lambda: n2c * (x * x - y * y)][L]()

    def get_gauss(self, L):
        if L == 0:
            return sqrt(self.a ** 3 * 4) / pi * self.exp_ar2
        l = 1 if L < 4 else 2
        return (1 / sqrt(4 * pi) * factorial(l) / factorial(2 * l + 1) *
                (4 * self.a) ** (l + 1.5)) * self.exp_ar2 * self.Y_L(L)

    def get_gauss_pot(self, L):
        if L == 0:
            return 2.0 * 1.7724538509055159 * self.erf_sar / self.r
        l = 1 if L < 4 else 2
        r, sa = self.r, sqrt(self.a)
        s = (2 * sa * r if l == 1 else
             2 * sa * r + 4.0 / 3.0 * self.a * sa * r ** 3) * self.exp_ar2
        return (4 * sqrt(pi) / (2 * l + 1) * self.Y_L(L) *
                (sqrt(pi) * self.erf_sar - s) / r ** (2 * l + 1))

    def get_moment(self, n, L):
        """gpaw/utilities/gauss.py:245-248."""
        return self.gd.integrate(n * self.Y_L(L))

    def remove_moment(self, n, L, q=None):
        """gpaw/utilities/gauss.py:250-263."""
        if q is None:
            q = self.get_moment(n, L)
        if abs(q) < 1e-7:
            return 0.
        n -= q * self.get_gauss(L)
        return q * self.get_gauss_pot(L)
