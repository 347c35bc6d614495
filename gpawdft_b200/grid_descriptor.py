"""Serial grid geometry (host-side mirror of gpaw.grid_descriptor / domain).

Mirrors the single-domain subset of gpaw/grid_descriptor.py:71-343 and
gpaw/domain.py:21-139 that the grid hot path reads: ``N_c``, ``n_c``,
``beg_c``/``end_c``, ``h_cv``, ``dv``, ``pbc_c``, ``neighbor_cd``,
``sdisp_cd``, ``coarsen``/``refine``, ``integrate``, coordinates.  There is no
domain decomposition: ``comm`` must be None or of size 1.
"""
import numbers

import numpy as np

from . import arrays


class GridDescriptor:
    ndim = 3

    def __init__(self, N_c, cell_cv=(1, 1, 1), pbc_c=True, comm=None,
                 parsize_c=None):
        if comm is not None and getattr(comm, 'size', 1) != 1:
            raise NotImplementedError('domain decomposition is not supported '
                                      '(single GPU)')
        if isinstance(pbc_c, (bool, int, np.bool_)):
            pbc_c = (pbc_c,) * 3
        self.N_c = np.array(N_c, int)
        if (self.N_c != N_c).any():
            raise ValueError('Non-int number of grid points %s' % N_c)
        cell_c = np.array(cell_cv, float)
        if cell_c.ndim == 1:
            self.cell_cv = np.diag(cell_c)
        else:
            self.cell_cv = cell_c
            cell_c = (self.cell_cv ** 2).sum(1) ** 0.5
        self.icell_cv = np.linalg.inv(self.cell_cv).T
        self.xxxucell_cv = np.array([self.cell_cv[x] / cell_c[x]
                                     for x in range(3)])
        self.xxxiucell_cv = np.linalg.inv(self.xxxucell_cv.T)
        self.pbc_c = np.asarray(pbc_c, bool)
        # serial neighbours (gpaw/domain.py:111-139): self on periodic axes,
        # -1 (zero boundary) otherwise; sdisp +-1 on periodic wraps.
        self.neighbor_cd = np.zeros((3, 2), int)
        self.sdisp_cd = np.zeros((3, 2), int)
        for c in range(3):
            for d in range(2):
                if self.pbc_c[c]:
                    self.sdisp_cd[c, d] = 1 - 2 * d
                else:
                    self.neighbor_cd[c, d] = -1
        self.beg_c = np.where(self.pbc_c, 0, 1)
        self.end_c = self.N_c.copy()
        if (self.end_c - self.beg_c <= 0).any():
            raise ValueError('Grid too small!')
        self.n_c = self.end_c - self.beg_c
        self.h_cv = self.cell_cv / self.N_c[:, np.newaxis]
        self.volume = abs(np.linalg.det(self.cell_cv))
        self.dv = self.volume / self.N_c.prod()
        self.orthogonal = not (self.cell_cv -
                               np.diag(self.cell_cv.diagonal())).any()
        h_c = self.get_grid_spacings()
        if max(h_c) / min(h_c) > 1.3:
            raise ValueError('Very anisotropic grid spacings: %s' % h_c)

    def __repr__(self):
        return 'GridDescriptor(%s, pbc_c=%s)' % (self.N_c.tolist(),
                                                 self.pbc_c.astype(int).tolist())

    def new_descriptor(self, N_c=None, cell_cv=None, pbc_c=None):
        return self.__class__(self.N_c if N_c is None else N_c,
                              self.cell_cv if cell_cv is None else cell_cv,
                              self.pbc_c if pbc_c is None else pbc_c)

    def get_grid_spacings(self):
        L_c = (np.linalg.inv(self.cell_cv) ** 2).sum(0) ** -0.5
        return L_c / self.N_c

    def get_size_of_global_array(self, pad=False):
        return self.N_c if pad else self.N_c - 1 + self.pbc_c

    def coarsen(self):
        if (self.N_c % 2).any():
            raise ValueError('Grid %s not divisible by 2!' % self.N_c)
        return self.new_descriptor(self.N_c // 2)

    def refine(self):
        return self.new_descriptor(self.N_c * 2)

    def _shape(self, n):
        if isinstance(n, numbers.Integral):
            n = (n,)
        return tuple(n) + tuple(self.n_c)

    def zeros(self, n=(), dtype=float, global_array=False, pad=False):
        return np.zeros(self._shape(n), dtype)

    def empty(self, n=(), dtype=float, global_array=False, pad=False):
        return np.empty(self._shape(n), dtype)

    def zeros_device(self, n=(), dtype=float):
        a = arrays.empty_like_device(self._shape(n), dtype)
        a.zero_()
        return a

    def empty_device(self, n=(), dtype=float):
        return arrays.empty_like_device(self._shape(n), dtype)

    def integrate(self, a_xg, b_yg=None, global_integral=True):
        """gpaw/grid_descriptor.py:263-319: sum(a) dv, or sum(conj(a_x) b_y) dv.

        Reduced on the device by the library's deterministic kernels (NumPy
        inputs are copied there first).
        """
        from .blas import integrate_device
        return integrate_device(self, a_xg, b_yg)

    def get_grid_point_coordinates(self, dtype=float):
        return np.dot(np.indices(self.n_c, dtype).T + self.beg_c,
                      self.h_cv).T.copy()

    def get_grid_point_distance_vectors(self, r_v, mic=True):
        s_Gc = (np.indices(self.n_c, float).T + self.beg_c) / self.N_c
        cell_cv = self.N_c * self.h_cv
        s_Gc -= np.linalg.solve(cell_cv.T, r_v)
        if mic:
            s_Gc -= self.pbc_c * (2 * s_Gc).astype(int)
            s_Gc -= self.pbc_c * (2 * s_Gc).astype(int)
        return np.dot(s_Gc, cell_cv).T.copy()

    def calculate_dipole_moment(self, rho_g):
        rho_01 = rho_g.sum(axis=2)
        rho_02 = rho_g.sum(axis=1)
        rho_cg = [rho_01.sum(axis=1), rho_01.sum(axis=0), rho_02.sum(axis=0)]
        rhog_c = [np.dot(np.arange(self.beg_c[c], self.end_c[c]), rho_cg[c])
                  for c in range(3)]
        return -np.dot(rhog_c, self.h_cv) * self.dv
