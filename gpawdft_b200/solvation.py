"""Poisson solver with a spatially varying dielectric on the GPU (drop-in for
gpaw.solvation.poisson's SolvationPoissonSolver and WeightedFDPoissonSolver).

The equation div(eps(r) grad phi(r)) = -4 pi rho(r) is discretised by the
weighted operator A = -1/4pi (eps Laplace + grad eps . grad)
(gpawdft_b200.wfd_operators, c/woperators.c) and solved by the reference's
multigrid (gpaw/solvation/poisson.py:62-150): the weights are restricted to
every coarse level before each solve (``restrict_op_weights``), the coarse
levels use nn=1 stencils, the V-cycle and schedule are FDPoissonSolver's.

Because A's coefficients vary from point to point, the V-cycle does not run
in the constant-coefficient device-loop engine of gpawdft_b200.poisson; it is
driven from the host, one device launch per relax / apply / transfer / axpy
as gpaw/poisson.py:331-366 orders them, with every array on the device.  The
charge branches of ``solve`` (background shift, the dielectric-aware
compensation charge of ``load_gauss``) are the plain solver's.

``dielectric`` is any object with ``eps_gradeps`` = [eps, d eps/dx,
d eps/dy, d eps/dz] (grids of the solver's shape; NumPy arrays or device
tensors), as gpaw.solvation's dielectric classes provide; the cavity and
dielectric models themselves are outside this path.
"""
from math import pi

import numpy as np
from scipy.special import erf

from . import _lib, arrays, blas
from .fd_operators import Gradient, Laplace
from .gauss import Gaussian
from .poisson import FDPoissonSolver, PoissonConvergenceError
from .transformers import Transformer
from .wfd_operators import WeightedFDOperator


class SolvationPoissonSolver(FDPoissonSolver):
    """Base class of the dielectric solvers (gpaw/solvation/poisson.py:
    11-59)."""

    def __init__(self, nn=3, relax='J', eps=2e-10, maxiter=1000,
                 remove_moment=None, use_charge_center=True):
        if remove_moment is not None:
            raise NotImplementedError(
                'Removing arbitrary multipole moments '
                'is not implemented for SolvationPoissonSolver!')
        FDPoissonSolver.__init__(self, nn, relax, eps, maxiter, remove_moment,
                                 use_charge_center=use_charge_center)

    def set_dielectric(self, dielectric):
        self.dielectric = dielectric

    def _eps_gradeps_host(self):
        return [a.cpu().numpy() if arrays.is_device(a) else np.asarray(a)
                for a in self.dielectric.eps_gradeps]

    def load_gauss(self, center=None):
        """Compensation charge of charged systems in the dielectric
        (gpaw/solvation/poisson.py:36-59; Held and Walter, J. Chem. Phys.
        141, 174108 (2014), appendix B)."""
        epsr, dx_epsr, dy_epsr, dz_epsr = self._eps_gradeps_host()
        gauss = Gaussian(self.gd, center=center)
        rho_g = gauss.get_gauss(0)
        phi_g = gauss.get_gauss_pot(0)
        x, y, z = gauss.xyz
        fac = 2. * np.sqrt(gauss.a) * np.exp(-gauss.a * gauss.r2)
        fac /= np.sqrt(np.pi) * gauss.r2
        fac -= erf(np.sqrt(gauss.a) * gauss.r) / (gauss.r2 * gauss.r)
        fac *= 2.0 * 1.7724538509055159
        dx_phi_g = fac * x
        dy_phi_g = fac * y
        dz_phi_g = fac * z
        sp = dx_phi_g * dx_epsr + dy_phi_g * dy_epsr + dz_phi_g * dz_epsr
        rho = epsr * rho_g - 1. / (4. * np.pi) * sp
        invnorm = np.sqrt(4. * np.pi) / (rho.sum() * self.gd.dv)
        self.phi_gauss = arrays.to_device(phi_g * invnorm)
        self.rho_gauss = arrays.to_device(rho * invnorm)


class WeightedFDPoissonSolver(SolvationPoissonSolver):
    """Weighted finite-difference Poisson solver with a dielectric
    (gpaw/solvation/poisson.py:62-150; V. M. Sanchez, M. Sued and D. A.
    Scherlis, J. Chem. Phys. 131, 174108 (2009))."""

    def solve(self, phi, rho, charge=None, eps=None, maxcharge=1e-6,
              zero_initial_phi=False):
        if self.gd.pbc_c.all():
            actual_charge = self.gd.integrate(rho)
            if abs(actual_charge) > maxcharge:
                raise NotImplementedError(
                    'charged periodic systems are not implemented')
        self.restrict_op_weights()
        return FDPoissonSolver.solve(self, phi, rho, charge, eps, maxcharge,
                                     zero_initial_phi)

    def restrict_op_weights(self):
        """Level-0 weights from the dielectric, restricted to every coarse
        level (gpaw/solvation/poisson.py:79-85)."""
        for w, src in zip(self.level0_weights, self.dielectric.eps_gradeps):
            w.copy_(arrays.to_device(np.ascontiguousarray(src)
                                     if not arrays.is_device(src) else src))
        weights = [self.level0_weights] + self.op_coarse_weights
        for i, res in enumerate(self.restrictors):
            for j in range(4):
                res.apply(weights[i][j], weights[i + 1][j])
        self.step = 0.66666666 / self.operators[0].get_diagonal_element()

    def set_grid_descriptor(self, gd):
        """gpaw/solvation/poisson.py:87-110."""
        self.gd = gd
        self.gds = [gd]
        self.dv = gd.dv
        self.B = None
        self.interpolators = []
        self.restrictors = []
        self.operators = []
        level = 0
        self.presmooths = [2]
        self.postsmooths = [1]
        self.weights = [2. / 3.]
        while level < 8 and (self.max_levels is None or
                             level + 1 < self.max_levels):
            try:
                gd2 = gd.coarsen()
            except ValueError:
                break
            self.gds.append(gd2)
            self.interpolators.append(Transformer(gd2, gd))
            self.restrictors.append(Transformer(gd, gd2))
            self.presmooths.append(4)
            self.postsmooths.append(4)
            self.weights.append(1.0)
            level += 1
            gd = gd2
        self.levels = level
        self._engine = None

    def get_description(self):
        if len(getattr(self, 'operators', [])) == 0:
            return 'uninitialized WeightedFDPoissonSolver'
        name = {1: 'Gauss-Seidel', 2: 'Jacobi'}[self.relax_method]
        return ('%s weighted FD solver with dielectric and %d multi-grid '
                'levels' % (name, self.levels + 1))

    def initialize(self, load_gauss=False):
        """gpaw/solvation/poisson.py:119-140 (arrays on the device)."""
        self.presmooths[self.levels] = 8
        self.postsmooths[self.levels] = 8
        self.phis = [None] + [gd.zeros_device() for gd in self.gds[1:]]
        self.residuals = [gd.zeros_device() for gd in self.gds]
        self.rhos = [gd.zeros_device() for gd in self.gds]
        self.level0_weights = [self.gds[0].zeros_device() for _ in range(4)]
        self.op_coarse_weights = [[gd.empty_device() for _ in range(4)]
                                  for gd in self.gds[1:]]
        scale = -0.25 / np.pi
        self.operators = []
        for i, gd in enumerate(self.gds):
            if i == 0:
                nn = self.nn
                weights = self.level0_weights
            else:
                nn = 1
                weights = self.op_coarse_weights[i - 1]
            operators = [Laplace(gd, scale, nn)] + \
                [Gradient(gd, j, scale, nn) for j in (0, 1, 2)]
            self.operators.append(WeightedFDOperator(weights, operators))
        self._lib = _lib.load()
        self._engine = (None, 1)   # no device-loop engine: host-driven V-cycle
        if load_gauss:
            self.load_gauss()

    def _make_engine(self, nbatch):
        if nbatch != 1:
            raise NotImplementedError('the weighted solver solves one grid '
                                      'at a time')

    def _free_engine(self):
        self._engine = None

    def _run(self, phi_d, rho_d, nb, eps_list, maxiter=None, exact=False):
        """solve_neutral (gpaw/poisson.py:306-329) with the host-driven
        V-cycle; returns the iteration count as a one-element array."""
        if nb != 1:
            raise NotImplementedError('the weighted solver solves one grid '
                                      'at a time')
        phi = phi_d[0] if phi_d.dim() == 4 else phi_d
        rho = rho_d[0] if rho_d.dim() == 4 else rho_d
        self.phis[0] = phi
        self.rhos[0].copy_(rho)
        eps = float(eps_list[0])
        maxiter = int(maxiter or self.maxiter)
        self.errors = []
        niter = 1
        while self.iterate2(self.step) > eps and niter < maxiter:
            niter += 1
        if niter == maxiter and not exact:
            raise PoissonConvergenceError(
                'Poisson solver did not converge in %d iterations!' % maxiter)
        if self.gd.pbc_c.all():
            npts = int(np.prod(self.gd.get_size_of_global_array()))
            s = blas.vector_sums(phi, 1)[0]
            blas.add_scalar(phi, -s / npts)
        self.last_errors = np.array([self.errors[-1]])
        return np.array([niter], np.int32)

    def iterate2(self, step, level=0):
        """gpaw/poisson.py:331-366, one device launch per step."""
        residual = self.residuals[level]
        op = self.operators[level]
        if level < self.levels:
            op.relax(self.relax_method, self.phis[level], self.rhos[level],
                     self.presmooths[level], self.weights[level])
            op.apply(self.phis[level], residual)
            blas.axpy(-1.0, self.rhos[level], residual)
            self.restrictors[level].apply(residual, self.rhos[level + 1])
            self.phis[level + 1].zero_()
            self.iterate2(4.0 * step, level + 1)
            self.interpolators[level].apply(self.phis[level + 1], residual)
            blas.axpy(-1.0, residual, self.phis[level])
        op.relax(self.relax_method, self.phis[level], self.rhos[level],
                 self.postsmooths[level], self.weights[level])
        if level == 0:
            op.apply(self.phis[level], residual)
            blas.axpy(-1.0, self.rhos[level], residual)
            error = float(blas.vector_dots(residual, residual, 1)[0]) * \
                self.gd.dv
            self.errors.append(error)
            return error

    def estimate_memory(self, mem=None):
        return int(np.prod(self.gd.n_c)) * 8 * 8
