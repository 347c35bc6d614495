"""Restated Poisson solver variants over a CPU backend (oracle).

Test infrastructure only.  Restates, over the backends of oracle/layer.py
(the compiled reference C in oracle/_ref, or the NumPy restatement):

* gpaw/helmholtz.py:34-186  -- ScreenedPoissonGaussian, HelmholtzOperator
  (coefficients), HelmholtzSolver;
* gpaw/dipole_correction.py:8-154 -- dipole_correction, DipoleCorrection
  (finite-difference form);
* gpaw/wfd_operators.py:8-76 with c/woperators.c, c/bmgs/wfd.c and
  c/bmgs/wrelax.c -- WeightedFDOperator (``ref`` backend: the reference's own
  WOperator; ``numpy`` backend: a restatement of its apply and relax);
* gpaw/solvation/poisson.py:11-150 -- SolvationPoissonSolver.load_gauss,
  WeightedFDPoissonSolver.
"""
from math import pi, sqrt

import numpy as np
from scipy.special import erf

from . import layer, stencils
from .gauss import Gaussian


# ------------------------------------------------------------ Helmholtz
class ScreenedPoissonGaussian(Gaussian):
    def get_phi(self, mu2):
        """gpaw/helmholtz.py:34-52."""
        r = np.sqrt(self.r2)
        mu = sqrt(mu2)
        sigma = 1. / sqrt(2 * self.a)
        sig2 = sigma ** 2
        mrho = (sig2 * mu - r) / (sqrt(2) * sigma)
        prho = (sig2 * mu + r) / (sqrt(2) * sigma)
        return sqrt(4 * pi) * np.exp(sig2 * mu2 / 2.0) / (2 * r) * (
            np.exp(-mu * r) * (1. - erf(mrho)) -
            np.exp(mu * r) * (1. - erf(prho)))


def helmholtz(gd, scale, n, k2):
    """gpaw/helmholtz.py:55-99: the GUC Laplacian with k2 * scale added to
    the centre coefficient."""
    coefs, offsets = stencils.guc_laplace(gd, scale, n)
    coefs = coefs.copy()
    coefs[0] += k2 * scale
    return coefs, offsets


class HelmholtzSolver(layer.PoissonSolver):
    """gpaw/helmholtz.py:101-186."""

    def __init__(self, k2=0.0, nn='M', relax='GS', eps=2e-10,
                 use_charge_center=True, backend='numpy'):
        assert k2 <= 0
        layer.PoissonSolver.__init__(self, nn, relax, eps,
                                     use_charge_center=use_charge_center,
                                     backend=backend)
        self.k2 = k2

    def set_grid_descriptor(self, gd):
        self.gd = gd
        scale = -0.25 / pi
        if self.nn == 'M':
            raise ValueError('Helmholtz not defined for Mehrstellen stencil')
        c, o = helmholtz(gd, scale, self.nn, self.k2)
        self.operators = [layer.FDOperator(c, o, gd, float, self.backend)]
        self.B = None
        self.interpolators = []
        self.restrictors = []
        level = 0
        self.presmooths = [2]
        self.postsmooths = [1]
        self.weights = [2.0 / 3.0]
        while level < 4:
            try:
                gd2 = gd.coarsen()
            except ValueError:
                break
            c, o = helmholtz(gd2, scale, 1, self.k2)
            self.operators.append(layer.FDOperator(c, o, gd2, float,
                                                   self.backend))
            self.interpolators.append(layer.Transformer(
                gd2, gd, backend=self.backend))
            self.restrictors.append(layer.Transformer(
                gd, gd2, backend=self.backend))
            self.presmooths.append(4)
            self.postsmooths.append(4)
            self.weights.append(1.0)
            level += 1
            gd = gd2
        self.levels = level

    def load_gauss(self, center=None):
        if not hasattr(self, 'rho_gauss') or center is not None:
            gauss = ScreenedPoissonGaussian(self.gd, center=center)
            self.rho_gauss = gauss.get_gauss(0)
            self.phi_gauss = gauss.get_phi(abs(self.k2))


# ------------------------------------------------------------ dipole layer
def dipole_correction(c, gd, rhot_g):
    """gpaw/dipole_correction.py:123-154."""
    moment = gd.calculate_dipole_moment(rhot_g)[c]
    if abs(moment) < 1e-12:
        return gd.zeros(), gd.zeros(), 0.0
    r_g = gd.get_grid_point_coordinates()[c]
    cellsize = abs(gd.cell_cv[c, c])
    sr_g = 2.0 / cellsize * r_g - 1.0
    alpha = 12.0
    drho_g = sr_g * np.exp(-alpha * sr_g ** 2)
    moment2 = gd.calculate_dipole_moment(drho_g)[c]
    factor = -moment / moment2
    drho_g *= factor
    phifactor = factor * (np.pi / alpha) ** 1.5 * cellsize ** 2 / 4.0
    dphi_g = -phifactor * erf(sr_g * np.sqrt(alpha))
    return drho_g, dphi_g, phifactor


class DipoleCorrection:
    """gpaw/dipole_correction.py:8-91 (finite-difference form)."""

    def __init__(self, poissonsolver, direction):
        self.c = direction
        self.poissonsolver = poissonsolver
        self.correction = None

    def set_grid_descriptor(self, gd):
        self.poissonsolver.set_grid_descriptor(gd)

    def initialize(self):
        self.poissonsolver.initialize()

    def solve(self, vHt_g, rhot_g, **kwargs):
        gd = self.poissonsolver.gd
        drhot_g, dvHt_g, self.correction = dipole_correction(self.c, gd,
                                                             rhot_g)
        vHt_g -= dvHt_g
        iters = self.poissonsolver.solve(vHt_g, rhot_g + drhot_g, **kwargs)
        vHt_g += dvHt_g
        return iters


# ------------------------------------------------------------ weighted
class _NumpyWOperator:
    """c/woperators.c with c/bmgs/wfd.c / wrelax.c restated in NumPy for
    float64 grids: the per-stencil tap sums in tap order, scaled by the
    weight and summed in stencil order, unfused."""

    def __init__(self, weights, coef_ps, offset_pcs, gd, mp):
        self.weights = weights
        self.coef_ps = coef_ps
        self.offset_pcs = offset_pcs
        self.gd = gd
        self.mp = mp

    def _pad(self, a):
        mp = self.mp
        pads = []
        out = a
        for c in range(3):
            mode = 'wrap' if self.gd.pbc_c[c] else 'constant'
            w = [(0, 0)] * 3
            w[c] = (mp, mp)
            out = np.pad(out, w, mode=mode)
            pads.append(mode)
        return out

    def _sums(self, b, start):
        mp = self.mp
        n0, n1, n2 = b.shape[0] - 2 * mp, b.shape[1] - 2 * mp, \
            b.shape[2] - 2 * mp
        x = np.zeros((n0, n1, n2))
        coef = np.zeros((n0, n1, n2))
        for w, cp, opc in zip(self.weights, self.coef_ps, self.offset_pcs):
            tmp = np.zeros((n0, n1, n2))
            for c in range(start, len(cp)):
                o = opc[c]
                tmp = tmp + b[mp + o[0]:mp + o[0] + n0,
                              mp + o[1]:mp + o[1] + n1,
                              mp + o[2]:mp + o[2] + n2] * cp[c]
            tmp = tmp * w
            x = x + tmp
            coef = coef + w * cp[0]
        return x, coef

    def apply(self, a, out, phases=None):
        for i in range(a.shape[0] if a.ndim == 4 else 1):
            src = a[i] if a.ndim == 4 else a
            dst = out[i] if a.ndim == 4 else out
            x, _ = self._sums(self._pad(src), 0)
            dst[...] = x

    def relax(self, method, f, s, n, w=1.0):
        assert method == 2, 'the NumPy restatement covers weighted Jacobi'
        for _ in range(n):
            x, coef = self._sums(self._pad(f), 1)
            f[...] = (1.0 - w) * f + w * (s - x) / coef

    def get_diagonal_element(self):
        coef = 0.0
        for w, cp in zip(self.weights, self.coef_ps):
            coef = coef + w * cp[0]
        return float(np.abs(coef).max())


class WeightedFDOperator:
    """gpaw/wfd_operators.py:8-76 over a backend."""

    def __init__(self, weights, operators, backend='numpy'):
        assert len(weights) == len(operators)
        self.gd = operators[0].gd
        self.coef_ps, self.offset_ps, offset_pcs = [], [], []
        for op in operators:
            if 0 in op.offset_p:
                assert op.offset_p[0] == 0
                self.offset_ps.append(np.ascontiguousarray(op.offset_p,
                                                           np.int64).copy())
                self.coef_ps.append(np.ascontiguousarray(op.coef_p,
                                                         float).copy())
                offset_pcs.append(np.asarray(op.offset_pc, int))
            else:
                self.offset_ps.append(np.ascontiguousarray(
                    np.hstack(([0], op.offset_p)).astype(np.int64)))
                self.coef_ps.append(np.ascontiguousarray(
                    np.hstack(([.0], op.coef_p))))
                offset_pcs.append(np.vstack(([[0, 0, 0]],
                                             np.asarray(op.offset_pc, int))))
        self.weights = weights
        self.mp = max(op.mp for op in operators)
        self.cfd = all(op.cfd for op in operators)
        if backend == 'numpy':
            self.operator = _NumpyWOperator(weights, self.coef_ps,
                                            offset_pcs, self.gd, self.mp)
        else:
            self.operator = layer.get_backend(backend).WOperator(
                len(operators), list(weights), self.coef_ps, self.offset_ps,
                np.ascontiguousarray(self.gd.n_c, np.int64), self.mp,
                np.ascontiguousarray(self.gd.neighbor_cd, np.int64),
                operators[0].dtype == float, None, self.cfd)

    def apply(self, in_xg, out_xg, phase_cd=None):
        self.operator.apply(in_xg, out_xg, phase_cd)

    def relax(self, relax_method, f_g, s_g, n, w=None):
        self.operator.relax(relax_method, f_g, s_g, n, 1.0 if w is None
                            else w)

    def get_diagonal_element(self):
        return self.operator.get_diagonal_element()


class WeightedFDPoissonSolver(layer.PoissonSolver):
    """gpaw/solvation/poisson.py:11-150 (WeightedFDPoissonSolver and the
    load_gauss of SolvationPoissonSolver)."""

    def __init__(self, nn=3, relax='J', eps=2e-10, maxiter=1000,
                 use_charge_center=True, backend='numpy'):
        layer.PoissonSolver.__init__(self, nn, relax, eps, maxiter,
                                     use_charge_center=use_charge_center,
                                     backend=backend)

    def set_dielectric(self, dielectric):
        self.dielectric = dielectric

    def load_gauss(self, center=None):
        epsr, dx_epsr, dy_epsr, dz_epsr = self.dielectric.eps_gradeps
        gauss = Gaussian(self.gd, center=center)
        rho_g = gauss.get_gauss(0)
        phi_g = gauss.get_gauss_pot(0)
        x, y, z = gauss.xyz
        fac = 2. * np.sqrt(gauss.a) * np.exp(-gauss.a * gauss.r2)
        fac /= np.sqrt(np.pi) * gauss.r2
        fac -= erf(np.sqrt(gauss.a) * gauss.r) / (gauss.r2 * gauss.r)
        fac *= 2.0 * 1.7724538509055159
        sp = fac * x * dx_epsr + fac * y * dy_epsr + fac * z * dz_epsr
        rho = epsr * rho_g - 1. / (4. * np.pi) * sp
        invnorm = np.sqrt(4. * np.pi) / self.gd.integrate(rho)
        self.phi_gauss = phi_g * invnorm
        self.rho_gauss = rho * invnorm

    def solve(self, phi, rho, charge=None, eps=None, maxcharge=1e-6,
              zero_initial_phi=False):
        if self.gd.pbc_c.all():
            if abs(self.gd.integrate(rho)) > maxcharge:
                raise NotImplementedError(
                    'charged periodic systems are not implemented')
        self.restrict_op_weights()
        return layer.PoissonSolver.solve(self, phi, rho, charge, eps,
                                         maxcharge, zero_initial_phi)

    def restrict_op_weights(self):
        weights = [self.dielectric.eps_gradeps] + self.op_coarse_weights
        for i, res in enumerate(self.restrictors):
            for j in range(4):
                res.apply(weights[i][j], weights[i + 1][j])
        self.step = 0.66666666 / self.operators[0].get_diagonal_element()

    def set_grid_descriptor(self, gd):
        self.gd = gd
        self.gds = [gd]
        self.B = None
        self.interpolators = []
        self.restrictors = []
        self.operators = []
        level = 0
        self.presmooths = [2]
        self.postsmooths = [1]
        self.weights = [2. / 3.]
        while level < 8:
            try:
                gd2 = gd.coarsen()
            except ValueError:
                break
            self.gds.append(gd2)
            self.interpolators.append(layer.Transformer(
                gd2, gd, backend=self.backend))
            self.restrictors.append(layer.Transformer(
                gd, gd2, backend=self.backend))
            self.presmooths.append(4)
            self.postsmooths.append(4)
            self.weights.append(1.0)
            level += 1
            gd = gd2
        self.levels = level

    def initialize(self):
        self.presmooths[self.levels] = 8
        self.postsmooths[self.levels] = 8
        self.phis = [None] + [gd.zeros() for gd in self.gds[1:]]
        self.residuals = [gd.zeros() for gd in self.gds]
        self.rhos = [gd.zeros() for gd in self.gds]
        self.op_coarse_weights = [[gd.empty() for _ in range(4)]
                                  for gd in self.gds[1:]]
        scale = -0.25 / np.pi
        for i, gd in enumerate(self.gds):
            if i == 0:
                nn = self.nn
                weights = self.dielectric.eps_gradeps
            else:
                nn = 1
                weights = self.op_coarse_weights[i - 1]
            operators = [layer.Laplace(gd, scale, nn, backend=self.backend)] \
                + [layer.Gradient(gd, j, scale, nn, backend=self.backend)
                   for j in (0, 1, 2)]
            self.operators.append(WeightedFDOperator(weights, operators,
                                                     self.backend))


# ------------------------------------------------------------ extended grid
def extended_grid_descriptor(gd, N_c):
    """gpaw/utilities/extend_grid.py:7-43 (serial, N_c form)."""
    from .geometry import GridDescriptor
    N_c = np.array(N_c, dtype=int)
    extend_N_cd = np.tile((N_c - gd.N_c) // 2, (2, 1)).T
    egd = GridDescriptor(N_c, gd.h_cv * N_c, gd.pbc_c)
    egd.extend_N_cd = extend_N_cd
    return egd


def extend_array(gd, egd, a_g, aext_g):
    """gpaw/utilities/extend_grid.py:46-49 (grid2grid with an offset)."""
    o = egd.extend_N_cd[:, 0]
    n = gd.n_c
    aext_g[o[0]:o[0] + n[0], o[1]:o[1] + n[1], o[2]:o[2] + n[2]] = a_g


def deextend_array(gd, egd, a_g, aext_g):
    """gpaw/utilities/extend_grid.py:52-56."""
    o = egd.extend_N_cd[:, 0]
    n = gd.n_c
    a_g[:] = aext_g[o[0]:o[0] + n[0], o[1]:o[1] + n[1], o[2]:o[2] + n[2]]


class ExtendedPoissonSolver(layer.PoissonSolver):
    """gpaw/poisson_extended.py:13-241 (serial)."""

    def __init__(self, nn=3, relax='J', eps=2e-10, maxiter=1000,
                 moment_corrections=None, extended=None, backend='numpy'):
        layer.PoissonSolver.__init__(self, nn=nn, relax=relax, eps=eps,
                                     maxiter=maxiter, backend=backend)
        if moment_corrections is None:
            self.moment_corrections = None
        elif isinstance(moment_corrections, int):
            self.moment_corrections = [{'moms': range(moment_corrections),
                                        'center': None}]
        else:
            self.moment_corrections = moment_corrections
        self.is_extended = extended is not None
        if self.is_extended:
            self.extended = dict(extended)
            self.extended['finegpts'] = np.array(self.extended['gpts']) * 2

    def set_grid_descriptor(self, gd):
        if self.is_extended:
            self.gd_original = gd
            gd = extended_grid_descriptor(gd, self.extended['finegpts'])
        layer.PoissonSolver.set_grid_descriptor(self, gd)

    def initialize(self):
        layer.PoissonSolver.initialize(self)
        if self.is_extended:
            self.rho_g = self.gd.zeros()
            self.phi_g = self.gd.zeros()
        if self.moment_corrections is not None:
            self.gauss_i, self.mom_ij, r_ir = [], [], []
            for rmom in self.moment_corrections:
                center = None if rmom['center'] is None else \
                    np.array(rmom['center'])
                g = Gaussian(self.gd, center=center)
                self.gauss_i.append(g)
                r_ir.append(g.r.ravel())
                self.mom_ij.append(rmom['moms'])
            r_ir = np.array(r_ir)
            mask_ir = np.zeros(r_ir.shape, dtype=int)
            for r in range(r_ir.shape[1]):
                mask_ir[np.argmin(r_ir[:, r]), r] = 1
            self.mask_ig = [m.reshape(self.gd.n_c) for m in mask_ir]

    def solve(self, phi, rho, charge=None, eps=None, maxcharge=1e-6,
              zero_initial_phi=False):
        if self.is_extended:
            self.rho_g[:] = 0
            if not self.extended['useprev']:
                self.phi_g[:] = 0
            extend_array(self.gd_original, self.gd, rho, self.rho_g)
            retval = self._solve(self.phi_g, self.rho_g, charge, eps,
                                 maxcharge, zero_initial_phi)
            deextend_array(self.gd_original, self.gd, phi, self.phi_g)
            return retval
        return self._solve(phi, rho, charge, eps, maxcharge, zero_initial_phi)

    def _solve(self, phi, rho, charge=None, eps=None, maxcharge=1e-6,
               zero_initial_phi=False):
        if eps is None:
            eps = self.eps
        if self.moment_corrections:
            rho_neutral = rho * 0.0
            phi_cor_k = []
            for gauss, mask_g, mom_j in zip(self.gauss_i, self.mask_ig,
                                            self.mom_ij):
                rho_masked = rho * mask_g
                for mom in mom_j:
                    phi_cor_k.append(gauss.remove_moment(rho_masked, mom))
                rho_neutral += rho_masked
            for phi_cor in phi_cor_k:
                phi -= phi_cor
            niter = self.solve_neutral(phi, rho_neutral, eps=eps)
            for phi_cor in phi_cor_k:
                phi += phi_cor
            return niter
        return layer.PoissonSolver.solve(self, phi, rho, charge, eps,
                                         maxcharge, zero_initial_phi)
