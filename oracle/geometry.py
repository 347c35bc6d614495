"""Serial grid geometry (oracle restatement).

Restates the single-domain subset of gpaw/grid_descriptor.py and
gpaw/domain.py that the grid hot path reads: N_c, n_c, beg_c/end_c, h_cv, dv,
pbc_c, neighbor_cd, sdisp_cd, coarsen/refine, integrate, coordinates.
Test infrastructure only.
"""
import numpy as np


class GridDescriptor:
    """gpaw/grid_descriptor.py:71-149 (serial: parsize_c = (1, 1, 1))."""

    def __init__(self, N_c, cell_cv=(1, 1, 1), pbc_c=True):
        if isinstance(pbc_c, (int, bool, np.bool_)):
            pbc_c = (pbc_c,) * 3
        self.N_c = np.array(N_c, int)
        cell_c = np.array(cell_cv, float)
        # gpaw/domain.py:39-48
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
        # gpaw/domain.py:111-139 with parsize 1: neighbour is self (rank 0)
        # on periodic axes and -1 on zero-boundary axes.
        self.neighbor_cd = np.zeros((3, 2), int)
        self.sdisp_cd = np.zeros((3, 2), int)
        for c in range(3):
            for d in range(2):
                sdisp = 2 * d - 1
                if self.pbc_c[c]:
                    self.sdisp_cd[c, d] = -sdisp
                else:
                    self.neighbor_cd[c, d] = -1
        # gpaw/grid_descriptor.py:118-137
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

    def new_descriptor(self, N_c):
        return GridDescriptor(N_c, self.cell_cv, self.pbc_c)

    def coarsen(self):
        """gpaw/grid_descriptor.py:329-337."""
        if (self.N_c % 2).any():
            raise ValueError('Grid %s not divisible by 2!' % self.N_c)
        return self.new_descriptor(self.N_c // 2)

    def refine(self):
        """gpaw/grid_descriptor.py:339-343."""
        return self.new_descriptor(self.N_c * 2)

    def get_size_of_global_array(self, pad=False):
        """gpaw/grid_descriptor.py:203-207."""
        return self.N_c if pad else self.N_c - 1 + self.pbc_c

    def zeros(self, n=(), dtype=float):
        if isinstance(n, int):
            n = (n,)
        return np.zeros(tuple(n) + tuple(self.n_c), dtype)

    def empty(self, n=(), dtype=float):
        if isinstance(n, int):
            n = (n,)
        return np.empty(tuple(n) + tuple(self.n_c), dtype)

    def integrate(self, a_xg, b_yg=None):
        """gpaw/grid_descriptor.py:263-319 (serial).

        One array: ``sum(a) dv`` per leading index.  Two arrays: the matrix
        ``dv * B_y . conj(A_x)`` that the gemm call at :306 forms, returned
        transposed to ``xshape + yshape`` (:312-319), a scalar for two grids.
        """
        xshape = a_xg.shape[:-3]
        if b_yg is None:
            r = a_xg.reshape(xshape + (-1,)).sum(axis=-1) * self.dv
            return r
        A_xg = np.ascontiguousarray(a_xg.reshape((-1,) + a_xg.shape[-3:]))
        B_yg = np.ascontiguousarray(b_yg.reshape((-1,) + b_yg.shape[-3:]))
        A = A_xg.reshape(len(A_xg), -1)
        B = B_yg.reshape(len(B_yg), -1)
        result_yx = self.dv * np.dot(B, A.conj().T)
        yshape = b_yg.shape[:-3]
        result = result_yx.T.reshape(xshape + yshape)
        if result.ndim == 0:
            return result.item()
        return result

    def get_grid_point_coordinates(self):
        """gpaw/grid_descriptor.py:629-636."""
        return np.dot(np.indices(self.n_c, float).T + self.beg_c,
                      self.h_cv).T.copy()

    def get_grid_point_distance_vectors(self, r_v, mic=True):
        """gpaw/grid_descriptor.py:638-659."""
        s_Gc = (np.indices(self.n_c, float).T + self.beg_c) / self.N_c
        cell_cv = self.N_c * self.h_cv
        s_Gc -= np.linalg.solve(cell_cv.T, r_v)
        if mic:
            s_Gc -= self.pbc_c * (2 * s_Gc).astype(int)
            s_Gc -= self.pbc_c * (2 * s_Gc).astype(int)
        return np.dot(s_Gc, cell_cv).T.copy()

    def calculate_dipole_moment(self, rho_g):
        """gpaw/grid_descriptor.py:576-585."""
        rho_01 = rho_g.sum(axis=2)
        rho_02 = rho_g.sum(axis=1)
        rho_cg = [rho_01.sum(axis=1), rho_01.sum(axis=0), rho_02.sum(axis=0)]
        rhog_c = [np.dot(np.arange(self.beg_c[c], self.end_c[c]), rho_cg[c])
                  for c in range(3)]
        return -np.dot(rhog_c, self.h_cv) * self.dv


def phase_cd_for_k(gd, k_c):
    """Bloch phases, gpaw/kpt_descriptor.py:308-313."""
    return np.exp(2j * np.pi * gd.sdisp_cd * np.asarray(k_c)[:, np.newaxis])
