"""Monopole Gaussian used to neutralise charged zero-boundary densities.

Mirrors ``Gaussian(gd, a=19, center)`` of gpaw/utilities/gauss.py:193-240 for
L = 0 (``get_gauss(0)`` = sqrt(4 a^3)/pi exp(-a r^2) and ``get_gauss_pot(0)``
= 2 sqrt(pi) erf(sqrt(a) r)/r), with coordinates as in
gpaw/utilities/tools.py:106-125.  Built once per centre on the host (setup,
like the stencil tables) and uploaded; every per-solve use is a device axpy.
"""
from math import pi, sqrt

import numpy as np
from scipy.special import erf


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

    def get_gauss(self, L):
        if L != 0:
            raise NotImplementedError('only the monopole (L=0) is used by '
                                      'the Poisson solver')
        return sqrt(self.a ** 3 * 4) / pi * self.exp_ar2

    def get_gauss_pot(self, L):
        if L != 0:
            raise NotImplementedError('only the monopole (L=0) is used by '
                                      'the Poisson solver')
        return 2.0 * 1.7724538509055159 * self.erf_sar / self.r
