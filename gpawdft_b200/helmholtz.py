"""Helmholtz / screened-Poisson multigrid solver on the GPU (drop-in for
gpaw.helmholtz).

``HelmholtzSolver(k2=0.0, nn='M', relax='GS', eps=2e-10,
use_charge_center=True)`` solves (Laplace + k2) phi = -4 pi rho with k2 <= 0
(the screened Poisson equation, mu^2 = -k2), gpaw/helmholtz.py:101-182:

* ``HelmholtzOperator`` (:55-99) is the general-cell Laplacian of
  gpaw/fd_operators.py with ``k2 * scale`` added to its centre coefficient;
* the hierarchy has at most five levels (four coarsenings, :152-168), nn=1
  Helmholtz operators and nn=1 transformers below level 0;
* charged zero-boundary densities are neutralised with the screened
  potential of a Gaussian (``ScreenedPoissonGaussian``, :34-52).

Everything else -- the charge branches, the V-cycles, their convergence loop
on the device, the float32 defect-correction option -- is the plain solver's
(gpawdft_b200.poisson), whose engine takes any star operators.
"""
from math import pi, sqrt

import numpy as np
from scipy.special import erf

from . import arrays
from .fd_operators import FDOperator, laplace
from .gauss import Gaussian
from .poisson import FDPoissonSolver
from .transformers import Transformer


class ScreenedPoissonGaussian(Gaussian):
    def get_phi(self, mu2):
        """Solution of the screened Poisson equation for the Gaussian
        (gpaw/helmholtz.py:34-52)."""
        r = np.sqrt(self.r2)
        mu = sqrt(mu2)
        sigma = 1. / sqrt(2 * self.a)
        sig2 = sigma ** 2
        mrho = (sig2 * mu - r) / (sqrt(2) * sigma)
        prho = (sig2 * mu + r) / (sqrt(2) * sigma)

        def erfc(values):
            return 1. - erf(values)

        # the Gaussian here is sqrt(4 pi) times a normalised 3D Gaussian
        return sqrt(4 * pi) * np.exp(sig2 * mu2 / 2.0) / (2 * r) * (
            np.exp(-mu * r) * erfc(mrho) - np.exp(mu * r) * erfc(prho))


def helmholtz_coefficients(gd, scale=1.0, n=1, k2=0.0):
    """Coefficient / offset table of HelmholtzOperator (gpaw/helmholtz.py:
    55-99): the general-cell Laplacian's directions and weights, the centre
    coefficient shifted by k2 * scale."""
    M_ic = np.indices((3, 3, 3)).reshape((3, -3)).T[-13:] - 1
    u_cv = gd.h_cv / (gd.h_cv ** 2).sum(1)[:, np.newaxis] ** 0.5
    u2_i = (np.dot(M_ic, u_cv) ** 2).sum(1)
    i_d = u2_i.argsort()
    m_mv = np.array([(2, 0, 0), (0, 2, 0), (0, 0, 2),
                     (0, 1, 1), (1, 0, 1), (1, 1, 0)])
    for D in range(3, 7):
        h_dv = np.dot(M_ic[i_d[:D]], gd.h_cv)
        A_md = (h_dv ** m_mv[:, np.newaxis, :]).prod(2)
        a_d, residual, rank, s = np.linalg.lstsq(A_md, [1, 1, 1, 0, 0, 0],
                                                 rcond=-1)
        if residual.sum() < 1e-14:
            if rank != D:
                raise ValueError('You have a weird unit cell!')
            break
    a_d *= scale
    offsets = [(0, 0, 0)]
    coefs = [laplace[n][0] * a_d.sum()]
    coefs[0] += k2 * scale
    for d in range(D):
        M_c = M_ic[i_d[d]]
        offsets.extend(np.arange(1, n + 1)[:, np.newaxis] * M_c)
        coefs.extend(a_d[d] * np.array(laplace[n][1:]))
        offsets.extend(np.arange(-1, -n - 1, -1)[:, np.newaxis] * M_c)
        coefs.extend(a_d[d] * np.array(laplace[n][1:]))
    return coefs, offsets


class HelmholtzOperator(FDOperator):
    def __init__(self, gd, scale=1.0, n=1, dtype=float, k2=0.0):
        coefs, offsets = helmholtz_coefficients(gd, scale, n, k2)
        FDOperator.__init__(self, coefs, offsets, gd, dtype)
        self.description = (
            '%d*%d+1=%d point O(h^%d) finite-difference Helmholtz' %
            ((self.npoints - 1) // n, n, self.npoints, 2 * n))


class HelmholtzSolver(FDPoissonSolver):
    """(Laplace + k2) phi = -4 pi rho for k2 <= 0 (the screened Poisson
    equation); gpaw/helmholtz.py:101-182."""

    def __init__(self, k2=0.0, nn='M', relax='GS', eps=2e-10,
                 use_charge_center=True, **kwargs):
        assert k2 <= 0, 'Currently only defined for k^2<=0'
        FDPoissonSolver.__init__(self, nn, relax, eps,
                                 use_charge_center=use_charge_center,
                                 **kwargs)
        self.k2 = k2

    def set_grid_descriptor(self, gd):
        """gpaw/helmholtz.py:130-175."""
        self.gd = gd
        self.dv = gd.dv
        scale = -0.25 / pi
        if self.nn == 'M':
            raise ValueError('Helmholtz not defined for Mehrstellen stencil')
        self.operators = [HelmholtzOperator(gd, scale, self.nn, k2=self.k2)]
        self.B = None
        self.interpolators = []
        self.restrictors = []
        level = 0
        self.presmooths = [2]
        self.postsmooths = [1]
        self.weights = [2.0 / 3.0]
        while level < 4 and (self.max_levels is None or
                             level + 1 < self.max_levels):
            try:
                gd2 = gd.coarsen()
            except ValueError:
                break
            self.operators.append(HelmholtzOperator(gd2, scale, 1,
                                                    k2=self.k2))
            self.interpolators.append(Transformer(gd2, gd))
            self.restrictors.append(Transformer(gd, gd2))
            self.presmooths.append(4)
            self.postsmooths.append(4)
            self.weights.append(1.0)
            level += 1
            gd = gd2
        self.levels = level
        self._engine = None
        if self.relax_method == 1:
            self.description = 'Gauss-Seidel'
        else:
            self.description = 'Jacobi'
        self.description += ' solver with %d multi-grid levels' % (level + 1)
        self.description += '\nStencil: ' + self.operators[0].description

    def load_gauss(self, center=None):
        """gpaw/helmholtz.py:177-186 (k2 <= 0: the screened potential)."""
        if not hasattr(self, 'rho_gauss') or center is not None:
            gauss = ScreenedPoissonGaussian(self.gd, center=center)
            self.rho_gauss = arrays.to_device(gauss.get_gauss(0))
            self.phi_gauss = arrays.to_device(gauss.get_phi(abs(self.k2)))
