"""Extended-grid Poisson solver with multipole moment corrections on the GPU
(drop-in for gpaw.poisson_extended).

``ExtendedPoissonSolver(nn=3, relax='J', eps=2e-10, maxiter=1000,
moment_corrections=None, extended=None)`` as in gpaw/poisson_extended.py:13-
241:

* ``extended={'gpts': N_c, 'useprev': bool}``: the density is copied into a
  larger zero-boundary grid (N_c given in coarse-grid points, the solve runs
  on 2 N_c, centred: gpaw/utilities/extend_grid.py:7-56), solved there and
  the potential copied back; ``useprev`` keeps the previous extended
  potential as the next start;
* ``moment_corrections=k`` (the moments L < k about the cell centre) or a
  list of ``{'moms': [L...], 'center': r}``: every grid point belongs to its
  nearest centre; per centre the density's moments are removed with
  generalised Gaussians (gpaw/utilities/gauss.py:250-263) before a neutral
  solve and their analytic potentials added back after it.

The grid copies, the masks, the moment integrals and the Gaussian
subtractions are device work (the Gaussians and masks are built once, on
the host, like the stencil tables); the solve itself is the plain solver's
device-loop engine on the (extended) grid.
"""
import numpy as np

from . import _lib, arrays, blas
from .gauss import Gaussian
from .grid_descriptor import GridDescriptor
from .poisson import FDPoissonSolver


def extended_grid_descriptor(gd, extend_N_cd=None, N_c=None):
    """gpaw/utilities/extend_grid.py:7-43 (serial)."""
    if extend_N_cd is None:
        assert N_c is not None, 'give only extend_N_cd or N_c'
        N_c = np.array(N_c, dtype=int)
        extend_N_cd = np.tile((N_c - gd.N_c) // 2, (2, 1)).T
    else:
        assert N_c is None, 'give only extend_N_cd or N_c'
        extend_N_cd = np.array(extend_N_cd, dtype=int)
        N_c = gd.N_c + extend_N_cd.sum(axis=1)
    cell_cv = gd.h_cv * N_c
    move_c = gd.get_grid_spacings() * extend_N_cd[:, 0]
    egd = GridDescriptor(N_c, cell_cv, gd.pbc_c)
    egd.extend_N_cd = extend_N_cd
    return egd, cell_cv * 0.52917721, move_c * 0.52917721


def _copy_box(src, src_shape, src_off, dst, dst_shape, dst_off, box):
    lib = _lib.load()
    arr = [np.ascontiguousarray(v, np.int64) for v in
           (src_shape, src_off, dst_shape, dst_off, box)]
    _lib.check(lib.gpw_copy_box(arrays.code_of(src), arrays.ptr(src),
                                arr[0].ctypes.data, arr[1].ctypes.data,
                                arrays.ptr(dst), arr[2].ctypes.data,
                                arr[3].ctypes.data, arr[4].ctypes.data,
                                arrays.stream()))


def extend_array(gd, ext_gd, a_g, aext_g):
    """gpaw/utilities/extend_grid.py:46-49: a_g into aext_g at the offset."""
    off = ext_gd.extend_N_cd[:, 0]
    _copy_box(a_g, gd.n_c, (0, 0, 0), aext_g, ext_gd.n_c, off, gd.n_c)


def deextend_array(gd, ext_gd, a_g, aext_g):
    """gpaw/utilities/extend_grid.py:52-56: the inner box of aext_g into a_g."""
    off = ext_gd.extend_N_cd[:, 0]
    _copy_box(aext_g, ext_gd.n_c, off, a_g, gd.n_c, (0, 0, 0), gd.n_c)


class ExtendedPoissonSolver(FDPoissonSolver):
    def __init__(self, nn=3, relax='J', eps=2e-10, maxiter=1000,
                 moment_corrections=None, extended=None, timer=None,
                 **kwargs):
        FDPoissonSolver.__init__(self, nn=nn, relax=relax, eps=eps,
                                 maxiter=maxiter, remove_moment=None,
                                 **kwargs)
        if moment_corrections is None:
            self.moment_corrections = None
        elif isinstance(moment_corrections, int):
            self.moment_corrections = [{'moms': range(moment_corrections),
                                        'center': None}]
        else:
            self.moment_corrections = moment_corrections
        self.is_extended = False
        if extended is not None:
            self.is_extended = True
            self.extended = dict(extended)
            assert 'gpts' in self.extended, 'gpts parameter is missing'
            self.extended['gpts'] = np.array(self.extended['gpts'])
            self.extended['finegpts'] = self.extended['gpts'] * 2
            assert 'useprev' in self.extended, 'useprev parameter is missing'

    def set_grid_descriptor(self, gd):
        """gpaw/poisson_extended.py:69-78."""
        if self.is_extended:
            self.gd_original = gd
            assert np.all(self.gd_original.N_c < self.extended['finegpts']), \
                'extended grid has to be larger than the original one'
            gd, _, _ = extended_grid_descriptor(
                gd, N_c=self.extended['finegpts'])
        FDPoissonSolver.set_grid_descriptor(self, gd)

    def get_description(self):
        lines = [FDPoissonSolver.get_description(self)]
        if self.is_extended:
            lines.append('    Extended %d*%d*%d grid' % tuple(self.gd.N_c))
            lines.append('    Use previous is %s' % self.extended['useprev'])
        if self.moment_corrections:
            lines.append('    %d moment corrections:' %
                         len(self.moment_corrections))
        return '\n'.join(lines)

    def initialize(self, load_gauss=False):
        """gpaw/poisson_extended.py:105-123."""
        FDPoissonSolver.initialize(self, load_gauss=load_gauss)
        if self.is_extended:
            if not self.gd.orthogonal or self.gd.pbc_c.any():
                raise NotImplementedError('Only orthogonal unit cells' +
                                          'and non-periodic boundary' +
                                          'conditions are tested')
            self.rho_g = self.gd.zeros_device()
            self.phi_g = self.gd.zeros_device()
        if self.moment_corrections is not None:
            if not self.gd.orthogonal or self.gd.pbc_c.any():
                raise NotImplementedError('Only orthogonal unit cells' +
                                          'and non-periodic boundary' +
                                          'conditions are tested')
            self.load_moment_corrections_gauss()

    def load_moment_corrections_gauss(self):
        """gpaw/poisson_extended.py:125-163: Gaussians per centre and the
        nearest-centre masks (host set-up, then device copies)."""
        if hasattr(self, 'gauss_i'):
            return
        self.gauss_i = []
        self.mom_ij = []
        r_ir = []
        for rmom in self.moment_corrections:
            center = None if rmom['center'] is None else \
                np.array(rmom['center'])
            gauss = Gaussian(self.gd, center=center)
            self.gauss_i.append(gauss)
            r_ir.append(gauss.r.ravel())
            self.mom_ij.append(list(rmom['moms']))
        r_ir = np.array(r_ir)
        owner = np.argmin(r_ir, axis=0)
        self.mask_ig = []
        self.dev_i = []
        for i, gauss in enumerate(self.gauss_i):
            mask_g = (owner == i).astype(float).reshape(self.gd.n_c)
            self.mask_ig.append(mask_g)
            per_L = {L: (arrays.to_device(np.ascontiguousarray(
                gauss.Y_L(L) * np.ones(tuple(self.gd.n_c)))),
                arrays.to_device(np.ascontiguousarray(gauss.get_gauss(L))),
                arrays.to_device(np.ascontiguousarray(
                    gauss.get_gauss_pot(L))))
                for L in self.mom_ij[i]}
            self.dev_i.append((arrays.to_device(mask_g), per_L))

    def solve(self, phi, rho, charge=None, eps=None, maxcharge=1e-6,
              zero_initial_phi=False):
        """gpaw/poisson_extended.py:165-187."""
        if self._engine is None:
            self.initialize()
        if self.is_extended:
            self.rho_g.zero_()
            if not self.extended['useprev']:
                self.phi_g.zero_()
            rho_d = arrays.to_device(rho)
            extend_array(self.gd_original, self.gd, rho_d, self.rho_g)
            retval = self._solve(self.phi_g, self.rho_g, charge, eps,
                                 maxcharge, zero_initial_phi)
            phi_d = arrays.to_device(phi)
            deextend_array(self.gd_original, self.gd, phi_d, self.phi_g)
            if not arrays.is_device(phi):
                arrays.writeback(phi, phi_d)
            return retval
        return self._solve(phi, rho, charge, eps, maxcharge, zero_initial_phi)

    def _solve(self, phi, rho, charge=None, eps=None, maxcharge=1e-6,
               zero_initial_phi=False):
        """gpaw/poisson_extended.py:189-225."""
        if eps is None:
            eps = self.eps
        if not self.moment_corrections:
            return FDPoissonSolver.solve(self, phi, rho, charge, eps,
                                         maxcharge, zero_initial_phi)
        assert not self.gd.pbc_c.any()
        lib = _lib.load()
        phi_d = arrays.to_device(phi)
        rho_d = arrays.to_device(rho)
        n = int(np.prod(self.gd.n_c))
        rho_neutral = self.gd.zeros_device()
        rho_masked = self.gd.empty_device()
        phi_cor = []
        for gauss, (mask_d, per_L), mom_j in zip(self.gauss_i, self.dev_i,
                                                 self.mom_ij):
            _lib.check(lib.gpw_mul(n, arrays.ptr(rho_d), arrays.ptr(mask_d),
                                   arrays.ptr(rho_masked), arrays.stream()))
            for L in mom_j:
                Y, g, v = per_L[L]
                q = float(blas.vector_dots(rho_masked, Y, 1)[0]) * self.gd.dv
                if abs(q) < 1e-7:
                    continue
                blas.axpy(-q, g, rho_masked)
                phi_cor.append((q, v))
            blas.axpy(1.0, rho_masked, rho_neutral)
        for q, v in phi_cor:
            blas.axpy(-q, v, phi_d)
        niter = self.solve_neutral(phi_d, rho_neutral, eps=eps)
        for q, v in phi_cor:
            blas.axpy(q, v, phi_d)
        if not arrays.is_device(phi):
            arrays.writeback(phi, phi_d)
        return niter

    def estimate_memory(self, mem=None):
        nbytes = FDPoissonSolver.estimate_memory(self)
        gdbytes = int(np.prod(self.gd.n_c)) * 8
        if self.is_extended:
            nbytes += 2 * gdbytes
        if self.moment_corrections is not None:
            nbytes += len(self.moment_corrections) * gdbytes
        return nbytes

    def __repr__(self):
        return 'ExtendedPoissonSolver(relax=\'%s\', nn=%s, eps=%e)' % (
            self.relax, repr(self.nn), self.eps)

