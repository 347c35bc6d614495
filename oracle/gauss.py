"""Generalised Gaussians, L = 0 (oracle restatement).

Restates gpaw/utilities/gauss.py:193-240 (``Gaussian``) for the monopole that
FDPoissonSolver uses to neutralise charged zero-boundary systems
(gpaw/poisson.py:249-299), with coordinates from gpaw/utilities/tools.py:106-125.
Test infrastructure only.
"""
from math import pi, sqrt

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

    def get_gauss(self, L):
        assert L == 0
        return sqrt(self.a ** 3 * 4) / pi * self.exp_ar2

    def get_gauss_pot(self, L):
        assert L == 0
        return 2.0 * 1.7724538509055159 * self.erf_sar / self.r
