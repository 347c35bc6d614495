"""Restated Python layer of the grid hot path over a CPU backend (oracle).

Restates gpaw/fd_operators.py (FDOperator, Laplace, Gradient, LaplaceA/B),
gpaw/transformers.py (Transformer), gpaw/poisson.py (FDPoissonSolver) and
gpaw/preconditioner.py (Preconditioner).  ``backend`` is either
``oracle.kernels`` (NumPy restatement) or the compiled reference module from
``oracle.ref.load()``; both expose ``Operator`` and ``Transformer`` with the
reference's constructor signatures.  Test infrastructure only.
"""
from math import pi

import numpy as np

from . import kernels as _np_backend
from . import stencils
from .gauss import Gaussian


class PoissonConvergenceError(ArithmeticError):
    """gpaw/__init__.py:37."""


def get_backend(name):
    if name == 'numpy':
        return _np_backend
    if name in ('ref', 'ref-omp'):
        from . import ref
        return ref.load(omp=(name == 'ref-omp'))
    raise ValueError(name)


class FDOperator:
    """gpaw/fd_operators.py:31-96."""

    def __init__(self, coef_p, offset_pc, gd, dtype=float, backend='numpy'):
        n_c = gd.n_c
        mp, offset_p, cfd = stencils.operator_layout(offset_pc, n_c)
        coef_p = np.ascontiguousarray(coef_p, float)
        self.dtype = dtype
        self.shape = tuple(n_c)
        self.mp = mp
        self.gd = gd
        self.npoints = len(coef_p)
        self.coef_p = coef_p
        self.offset_p = offset_p
        self.offset_pc = np.asarray(offset_pc, int).reshape(-1, 3)
        self.cfd = cfd
        self.operator = get_backend(backend).Operator(
            coef_p, offset_p, np.ascontiguousarray(n_c, np.int64), mp,
            np.ascontiguousarray(gd.neighbor_cd, np.int64), dtype == float,
            None, cfd)

    def apply(self, in_xg, out_xg, phase_cd=None):
        self.operator.apply(in_xg, out_xg, phase_cd)

    def relax(self, relax_method, f_g, s_g, n, w=None):
        self.operator.relax(relax_method, f_g, s_g, n, w)

    def get_diagonal_element(self):
        return self.operator.get_diagonal_element()


def Laplace(gd, scale=1.0, n=1, dtype=float, backend='numpy'):
    """gpaw/fd_operators.py:151-155 (GUC Laplacian; n=9 FFT form not restated)."""
    coef_p, offset_pc = stencils.guc_laplace(gd, scale, n)
    return FDOperator(coef_p, offset_pc, gd, dtype, backend)


def Gradient(gd, v, scale=1.0, n=1, dtype=float, backend='numpy'):
    """gpaw/fd_operators.py:126-148."""
    coef_p, offset_pc = stencils.gradient(gd, v, scale, n)
    return FDOperator(coef_p, offset_pc, gd, dtype, backend)


def transformer_tables(gdin, gdout, nn):
    """Pad / neighbour-pad / skip tables, gpaw/transformers.py:19-58."""
    pad_cd = np.empty((3, 2), np.int64)
    neighborpad_cd = np.empty((3, 2), np.int64)
    skip_cd = np.zeros((3, 2), np.int64)
    if (gdin.N_c == 2 * gdout.N_c).all():
        pad_cd[:, 0] = 2 * nn - 1 - 2 * gdout.beg_c + gdin.beg_c
        pad_cd[:, 1] = 2 * nn - 2 + 2 * gdout.end_c - gdin.end_c
        neighborpad_cd[:, 0] = 2 * nn - 2 + 2 * gdout.beg_c - gdin.beg_c
        neighborpad_cd[:, 1] = 2 * nn - 1 - 2 * gdout.end_c + gdin.end_c
        interpolate = False
    else:
        assert (gdout.N_c == 2 * gdin.N_c).all()
        pad_cd[:, 0] = nn - 1 - gdout.beg_c // 2 + gdin.beg_c
        pad_cd[:, 1] = nn + gdout.end_c // 2 - gdin.end_c
        neighborpad_cd[:, 0] = nn + gdout.beg_c // 2 - gdin.beg_c
        neighborpad_cd[:, 1] = nn - 1 - gdout.end_c // 2 + gdin.end_c
        skip_cd[:, 0] = gdout.beg_c % 2
        skip_cd[:, 1] = gdout.end_c % 2
        interpolate = True
        inpoints = (gdin.n_c[0] + 2 * nn - 1) * (gdin.n_c[1] + 2 * nn - 1)
        outpoints = gdout.n_c[0] * gdout.n_c[1]
        if inpoints > outpoints:
            raise ValueError('Cannot construct interpolator.  Grid %s '
                             'may be too small' % ' x '.join(map(str, gdin.N_c)))
    assert (pad_cd >= 0).all()
    return pad_cd, neighborpad_cd, skip_cd, interpolate


class Transformer:
    """gpaw/transformers.py:17-86 (``_Transformer``) + factory :112-125."""

    def __init__(self, gdin, gdout, nn=1, dtype=float, backend='numpy'):
        assert 1 <= nn <= 4
        self.gdin, self.gdout, self.nn, self.dtype = gdin, gdout, nn, dtype
        pad, npad, skip, self.interpolate = transformer_tables(gdin, gdout, nn)
        self.pad_cd, self.neighborpad_cd, self.skip_cd = pad, npad, skip
        self.transformer = get_backend(backend).Transformer(
            np.ascontiguousarray(gdin.n_c, np.int64),
            np.ascontiguousarray(gdout.n_c, np.int64), 2 * nn, pad, npad,
            skip, np.ascontiguousarray(gdin.neighbor_cd, np.int64),
            dtype == float, None, self.interpolate)

    def apply(self, input, output=None, phases=None):
        if output is None:
            output = self.gdout.empty(input.shape[:-3], dtype=self.dtype)
        self.transformer.apply(input, output, phases)
        return output


class PoissonSolver:
    """FDPoissonSolver, gpaw/poisson.py:61-366 (Jacobi or Gauss-Seidel)."""

    def __init__(self, nn=3, relax='J', eps=2e-10, maxiter=1000,
                 remove_moment=None, use_charge_center=False,
                 backend='numpy'):
        self.relax = relax
        self.nn = nn
        self.eps = eps
        self.maxiter = maxiter
        self.remove_moment = remove_moment
        self.use_charge_center = use_charge_center
        self.backend = backend
        self.relax_method = {'GS': 1, 'J': 2}[relax]
        self.errors = []

    def set_grid_descriptor(self, gd):
        """gpaw/poisson.py:91-132 (multigrid hierarchy and schedule)."""
        self.gd = gd
        scale = -0.25 / pi
        if self.nn == 'M':
            cA, oA = stencils.laplace_A(gd, -scale)
            cB, oB = stencils.laplace_B(gd)
            self.operators = [FDOperator(cA, oA, gd, float, self.backend)]
            self.B = FDOperator(cB, oB, gd, float, self.backend)
        else:
            self.operators = [Laplace(gd, scale, self.nn,
                                      backend=self.backend)]
            self.B = None
        self.interpolators = []
        self.restrictors = []
        level = 0
        self.presmooths = [2]
        self.postsmooths = [1]
        self.weights = [2.0 / 3.0]
        while level < 8:
            try:
                gd2 = gd.coarsen()
            except ValueError:
                break
            self.operators.append(Laplace(gd2, scale, 1,
                                          backend=self.backend))
            self.interpolators.append(Transformer(gd2, gd,
                                                  backend=self.backend))
            self.restrictors.append(Transformer(gd, gd2,
                                                backend=self.backend))
            self.presmooths.append(4)
            self.postsmooths.append(4)
            self.weights.append(1.0)
            level += 1
            gd = gd2
        self.levels = level

    def initialize(self):
        """gpaw/poisson.py:174-195."""
        gd = self.gd
        self.rhos = [gd.empty()]
        self.phis = [None]
        self.residuals = [gd.empty()]
        for level in range(self.levels):
            gd2 = gd.coarsen()
            self.phis.append(gd2.empty())
            self.rhos.append(gd2.empty())
            self.residuals.append(gd2.empty())
            gd = gd2
        level = self.levels
        self.step = 0.66666666 / self.operators[0].get_diagonal_element()
        self.presmooths[level] = 8
        self.postsmooths[level] = 8

    def load_gauss(self, center=None):
        """gpaw/poisson.py:197-201."""
        if not hasattr(self, 'rho_gauss') or center is not None:
            gauss = Gaussian(self.gd, center=center)
            self.rho_gauss = gauss.get_gauss(0)
            self.phi_gauss = gauss.get_gauss_pot(0)

    def solve(self, phi, rho, charge=None, eps=None, maxcharge=1e-6,
              zero_initial_phi=False):
        """gpaw/poisson.py:203-304 (remove_moment branch not restated)."""
        assert np.all(phi.shape == self.gd.n_c)
        assert np.all(rho.shape == self.gd.n_c)
        if eps is None:
            eps = self.eps
        actual_charge = self.gd.integrate(rho)
        background = (actual_charge / self.gd.dv /
                      self.gd.get_size_of_global_array().prod())
        if charge is None:
            charge = actual_charge
        if abs(charge) <= maxcharge:
            return self.solve_neutral(phi, rho - background, eps=eps)
        elif abs(charge) > maxcharge and self.gd.pbc_c.all():
            if zero_initial_phi:
                phi[:] = 0.0
            return self.solve_neutral(phi, rho - background, eps=eps)
        elif abs(charge) > maxcharge and not self.gd.pbc_c.any():
            if self.use_charge_center:
                charge_sign = actual_charge / abs(actual_charge)
                rho_sign = rho * charge_sign
                rho_sign[np.where(rho_sign < 0)] = 0
                absolute_charge = self.gd.integrate(rho_sign)
                center = -self.gd.calculate_dipole_moment(rho_sign) / \
                    absolute_charge
                border_offset = np.inner(self.gd.h_cv, np.array((7, 7, 7)))
                borders = np.inner(self.gd.h_cv, self.gd.N_c)
                borders -= border_offset
                if np.any(center > borders) or np.any(center < border_offset):
                    raise RuntimeError('Poisson solver: center of charge '
                                       'outside borders - please increase box')
                self.load_gauss(center=center)
            else:
                self.load_gauss()
            q = actual_charge / np.sqrt(4 * pi)
            rho_neutral = rho - q * self.rho_gauss
            if zero_initial_phi:
                phi[:] = 0.0
            else:
                phi -= q * self.phi_gauss
            niter = self.solve_neutral(phi, rho_neutral, eps=eps)
            phi += q * self.phi_gauss
            return niter
        else:
            raise NotImplementedError('Charged systems with mixed '
                                      'periodic/zero boundary conditions')

    def solve_neutral(self, phi, rho, eps=2e-10):
        """gpaw/poisson.py:306-329."""
        self.phis[0] = phi
        if self.B is None:
            self.rhos[0][:] = rho
        else:
            self.B.apply(rho, self.rhos[0])
        niter = 1
        maxiter = self.maxiter
        self.errors = []
        while self.iterate2(self.step) > eps and niter < maxiter:
            niter += 1
        if niter == maxiter:
            raise PoissonConvergenceError(
                'Poisson solver did not converge in %d iterations!' % maxiter)
        if self.gd.pbc_c.all():
            phi_ave = np.sum(phi.ravel())
            phi_ave /= np.prod(self.gd.get_size_of_global_array())
            phi -= phi_ave
        return niter

    def iterate2(self, step, level=0):
        """gpaw/poisson.py:331-366 (recursive V-cycle)."""
        residual = self.residuals[level]
        if level < self.levels:
            self.operators[level].relax(self.relax_method, self.phis[level],
                                        self.rhos[level],
                                        self.presmooths[level],
                                        self.weights[level])
            self.operators[level].apply(self.phis[level], residual)
            residual -= self.rhos[level]
            self.restrictors[level].apply(residual, self.rhos[level + 1])
            self.phis[level + 1][:] = 0.0
            self.iterate2(4.0 * step, level + 1)
            self.interpolators[level].apply(self.phis[level + 1], residual)
            self.phis[level] -= residual
        self.operators[level].relax(self.relax_method, self.phis[level],
                                    self.rhos[level], self.postsmooths[level],
                                    self.weights[level])
        if level == 0:
            self.operators[level].apply(self.phis[level], residual)
            residual -= self.rhos[level]
            error = np.dot(residual.ravel(), residual.ravel()) * self.gd.dv
            self.errors.append(error)
            return error


class Preconditioner:
    """gpaw/preconditioner.py:10-60."""

    def __init__(self, gd0, kin0, dtype=float, block=1, backend='numpy'):
        gd1 = gd0.coarsen()
        gd2 = gd1.coarsen()
        self.kin0 = kin0
        self.kin1 = Laplace(gd1, -0.5, 1, dtype, backend)
        self.kin2 = Laplace(gd2, -0.5, 1, dtype, backend)
        self.scratch0 = gd0.zeros((2, block), dtype)
        self.scratch1 = gd1.zeros((3, block), dtype)
        self.scratch2 = gd2.zeros((3, block), dtype)
        self.step = 0.66666666 / kin0.get_diagonal_element()
        self.restrictor0 = Transformer(gd0, gd1, 1, dtype, backend).apply
        self.restrictor1 = Transformer(gd1, gd2, 1, dtype, backend).apply
        self.interpolator2 = Transformer(gd2, gd1, 1, dtype, backend).apply
        self.interpolator1 = Transformer(gd1, gd0, 1, dtype, backend).apply

    def __call__(self, residuals, phases, ekin=None):
        """gpaw/preconditioner.py:34-60 (``kpt`` reduced to its phase_cd)."""
        nb = len(residuals)
        step = self.step
        d0, q0 = self.scratch0[:, :nb]
        r1, d1, q1 = self.scratch1[:, :nb]
        r2, d2, q2 = self.scratch2[:, :nb]
        self.restrictor0(-residuals, r1, phases)
        d1[:] = 4 * step * r1
        self.kin1.apply(d1, q1, phases)
        q1 -= r1
        self.restrictor1(q1, r2, phases)
        d2 = 16 * step * r2
        self.kin2.apply(d2, q2, phases)
        q2 -= r2
        d2 -= 16 * step * q2
        self.interpolator2(d2, q1, phases)
        d1 -= q1
        self.kin1.apply(d1, q1, phases)
        q1 -= r1
        d1 -= 4 * step * q1
        self.interpolator1(-d1, d0, phases)
        self.kin0.apply(d0, q0, phases)
        q0 -= residuals
        d0 -= step * q0   # axpy(-step, q0, d0)
        d0 *= -1.0
        return d0
