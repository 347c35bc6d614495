"""Dipole-layer correction around a Poisson solver (drop-in for
gpaw.dipole_correction, finite-difference form).

``DipoleCorrection(poissonsolver, direction, width=1.0)`` with
``set_grid_descriptor``, ``initialize``, ``solve(pot, dens, **kwargs)`` as in
gpaw/dipole_correction.py:8-120: before the solve, the density's dipole
moment along the (non-periodic) ``direction`` is cancelled by a charge of
shape s exp(-12 s^2) (s the scaled coordinate along that axis, -1 .. 1) whose
potential is the matching error function; the potential is corrected back
after the solve (``dipole_correction``, :123-154).

The shape arrays depend only on the grid, so they are built once on the host
and kept on the device; per solve the dipole moment is a device reduction
(the index-weighted sums of gpaw/grid_descriptor.py:576-585) and the rest is
device axpy work around the wrapped solver's solve.  The plane-wave form
(``pwsolve``) is outside the finite-difference hot path.
"""
import numpy as np
from scipy.special import erf

from . import arrays, blas

BOHR = 0.52917721


def dipole_moment_device(gd, rho_d, index_grids):
    """gd.calculate_dipole_moment(rho) (gpaw/grid_descriptor.py:576-585) on
    the device: -dv sum_c (sum_g i_c(g) rho(g)) h_cv[c]."""
    s = blas.pair_dots(index_grids, 3, rho_d, 1)[:, 0]
    return -np.dot(s, gd.h_cv) * gd.dv


class DipoleCorrection:
    """Dipole-correcting wrapper around another Poisson solver."""

    def __init__(self, poissonsolver, direction, width=1.0):
        self.c = direction
        self.poissonsolver = poissonsolver
        self.width = width / BOHR
        self.correction = None   # shift in potential
        self._shapes = None

    def todict(self):
        dct = self.poissonsolver.todict()
        dct['dipolelayer'] = self.c
        if self.width != 1.0 / BOHR:
            dct['width'] = self.width * BOHR
        return dct

    def get_stencil(self):
        return self.poissonsolver.get_stencil()

    def set_grid_descriptor(self, gd):
        self.poissonsolver.set_grid_descriptor(gd)
        self.check_direction(gd, gd.pbc_c)
        self._shapes = None

    def check_direction(self, gd, pbc_c):
        """gpaw/dipole_correction.py:45-70."""
        if isinstance(self.c, str):
            axes = ['xyz'.index(d) for d in self.c]
            for c in range(3):
                if abs(gd.cell_cv[c, axes]).max() < 1e-12:
                    break
            else:
                raise ValueError('No axis perpendicular to {0}-plane!'
                                 .format(self.c))
            self.c = c
        if pbc_c[self.c]:
            raise ValueError('System must be non-periodic perpendicular '
                             'to dipole-layer.')
        for c1 in range(3):
            if c1 != self.c:
                if abs(np.dot(gd.cell_cv[self.c], gd.cell_cv[c1])) > 1e-12:
                    raise ValueError('Dipole correction axis must be '
                                     'orthogonal to the two other axes.')

    def get_description(self):
        poissondesc = self.poissonsolver.get_description()
        desc = 'Dipole correction along %s-axis' % 'xyz'[self.c]
        return '\n'.join([poissondesc, desc])

    def initialize(self):
        self.poissonsolver.initialize()

    def _setup(self):
        """The grid-only parts of gpaw/dipole_correction.py:123-154, built
        once: the shape s exp(-alpha s^2), its dipole moment, erf(s
        sqrt(alpha)) and the index grids of the moment reduction."""
        import torch
        gd = self.poissonsolver.gd
        c = self.c
        r_g = gd.get_grid_point_coordinates()[c]
        cellsize = abs(gd.cell_cv[c, c])
        sr_g = 2.0 / cellsize * r_g - 1.0
        alpha = 12.0
        drho_g = sr_g * np.exp(-alpha * sr_g ** 2)
        moment2 = gd.calculate_dipole_moment(drho_g)[c]
        idx = np.indices(tuple(gd.n_c), float) + \
            np.asarray(gd.beg_c, float)[:, None, None, None]
        self._shapes = dict(
            alpha=alpha, cellsize=cellsize, moment2=moment2,
            drho=arrays.to_device(np.ascontiguousarray(drho_g)),
            erf=arrays.to_device(np.ascontiguousarray(
                erf(sr_g * np.sqrt(alpha)))),
            index=torch.from_numpy(np.ascontiguousarray(idx)).cuda())

    def solve(self, pot, dens, **kwargs):
        return self.fdsolve(pot, dens, **kwargs)

    def fdsolve(self, vHt_g, rhot_g, **kwargs):
        """gpaw/dipole_correction.py:84-91 on the device."""
        if self._shapes is None:
            self._setup()
        sh = self._shapes
        gd = self.poissonsolver.gd
        v_d = arrays.to_device(vHt_g)
        r_d = arrays.to_device(rhot_g)
        moment = dipole_moment_device(gd, r_d, sh['index'])[self.c]
        if abs(moment) < 1e-12:
            self.correction = 0.0
            iters = self.poissonsolver.solve(v_d, r_d, **kwargs)
        else:
            factor = -moment / sh['moment2']
            phifactor = (factor * (np.pi / sh['alpha']) ** 1.5 *
                         sh['cellsize'] ** 2 / 4.0)
            self.correction = phifactor
            # dphi = -phifactor erf(...): vHt -= dphi, solve, vHt += dphi
            blas.axpy(phifactor, sh['erf'], v_d)
            rho2 = r_d.clone()
            blas.axpy(factor, sh['drho'], rho2)
            iters = self.poissonsolver.solve(v_d, rho2, **kwargs)
            blas.axpy(-phifactor, sh['erf'], v_d)
        if not arrays.is_device(vHt_g):
            arrays.writeback(vHt_g, v_d)
        return iters

    def estimate_memory(self, mem=None):
        return self.poissonsolver.estimate_memory(mem)
