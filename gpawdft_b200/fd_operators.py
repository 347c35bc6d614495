"""Finite-difference operators on the GPU (drop-in for gpaw.fd_operators).

Same classes, constructor arguments and methods as gpaw/fd_operators.py:
``FDOperator`` (:31-96), ``Gradient`` (:126-148), ``Laplace`` (:151-155),
``GUCLaplace`` (:158-208), ``LaplaceA`` / ``LaplaceB`` (:211-251).  The
coefficient and offset tables are built on the host exactly as the reference
builds them; ``apply`` / ``relax`` run in libgpwgrid.so
(``gpw_operator_apply`` / ``gpw_operator_relax``), which replaces
``_gpaw.Operator`` (c/operators.c).

Arrays may be NumPy arrays (copied to and from the device) or CUDA
``torch.Tensor`` objects (device-resident).  Besides float64 / complex128
(the reference's types) float32 / complex64 are accepted.
"""
import ctypes
from math import factorial as fact

import numpy as np

from . import _lib, arrays

# Chelikowsky et al., Phys. Rev. B 50, 11355 (1994) expansion coefficients of
# the second derivative (the table of gpaw/fd_operators.py:21-28).
laplace = [[0],
           [-2, 1],
           [-5 / 2, 4 / 3, -1 / 12],
           [-49 / 18, 3 / 2, -3 / 20, 1 / 90],
           [-205 / 72, 8 / 5, -1 / 5, 8 / 315, -1 / 560],
           [-5269 / 1800, 5 / 3, -5 / 21, 5 / 126, -5 / 1008, 1 / 3150],
           [-5369 / 1800, 12 / 7, -15 / 56, 10 / 189, -1 / 112, 2 / 1925,
            -1 / 16632]]

_REAL = (float, np.float64, np.float32)


def _is_real(dtype):
    return np.dtype(dtype).kind == 'f'


class FDOperator:
    def __init__(self, coef_p, offset_pc, gd, dtype=float, description=None):
        """FDOperator(coefs, offsets, gd, dtype) -> FDOperator object."""
        offset_pc = np.asarray(offset_pc, int).reshape(-1, 3)
        # central (star) stencil iff every offset lies on one axis
        cfd = all(int((o != 0).sum()) < 2 for o in offset_pc)
        maxoffset_c = [max(int(o[c]) for o in offset_pc) for c in range(3)]
        mp = maxoffset_c[0]
        if maxoffset_c[1] != mp or maxoffset_c[2] != mp:
            mp = max(maxoffset_c)
        n_c = gd.n_c
        M_c = n_c + 2 * mp
        stride_c = np.array([M_c[1] * M_c[2], M_c[2], 1])
        offset_p = np.ascontiguousarray(np.dot(offset_pc, stride_c), np.int64)
        coef_p = np.ascontiguousarray(coef_p, float)
        assert coef_p.ndim == 1 and coef_p.shape == offset_p.shape
        if np.dtype(dtype) not in (np.dtype(float), np.dtype(complex),
                                   np.dtype(np.float32),
                                   np.dtype(np.complex64)):
            raise ValueError('dtype must be float, complex, float32 or '
                             'complex64')
        self.dtype = dtype
        self.shape = tuple(int(x) for x in n_c)
        self.mp = mp
        self.gd = gd
        self.npoints = len(coef_p)
        self.coef_p = coef_p
        self.offset_p = offset_p
        self.offset_pc = offset_pc
        self.cfd = cfd
        self.comm = None
        lib = _lib.load()
        size = np.ascontiguousarray(n_c, np.int64)
        nb = np.ascontiguousarray(gd.neighbor_cd, np.int64)
        h = ctypes.c_void_p()
        _lib.check(lib.gpw_operator_new(
            coef_p.ctypes.data, offset_p.ctypes.data, len(coef_p),
            size.ctypes.data, mp, nb.ctypes.data, int(_is_real(dtype)),
            int(cfd), ctypes.byref(h)))
        self._h = h
        self._lib = lib
        if description is None:
            description = '%d point finite-difference stencil' % self.npoints
        self.description = description

    def __del__(self):
        h = getattr(self, '_h', None)
        if h is not None and h.value:
            self._lib.gpw_operator_free(h)
            self._h = None

    def __str__(self):
        return '<' + self.description + '>'

    @property
    def handle(self):
        return self._h

    def _check_grid(self, a):
        if tuple(a.shape[-3:]) != self.shape:
            raise ValueError('grid shape %s does not match operator %s' %
                             (tuple(a.shape[-3:]), self.shape))

    def apply(self, in_xg, out_xg, phase_cd=None):
        """out_xg = A in_xg for every leading grid (c/operators.c:316-405)."""
        self._check_grid(in_xg)
        if tuple(in_xg.shape) != tuple(out_xg.shape):
            raise ValueError('input and output shapes differ')
        if arrays.np_dtype_of(in_xg) != arrays.np_dtype_of(out_xg):
            raise ValueError('input and output dtypes differ')
        code = arrays.code_of(in_xg)
        if code in (_lib.GPW_C128, _lib.GPW_C64) and phase_cd is not None:
            if np.asarray(phase_cd).shape != (3, 2):
                raise ValueError('phase_cd must have shape (3, 2)')
        nin = int(np.prod(in_xg.shape[:-3])) if len(in_xg.shape) > 3 else 1
        src = arrays.to_device(in_xg)
        dst = out_xg if arrays.is_device(out_xg) else None
        if dst is None:
            dst = arrays.empty_like_device(out_xg.shape, out_xg.dtype)
        pbuf, pptr = arrays.phases_arg(phase_cd)
        _lib.check(self._lib.gpw_operator_apply(
            self._h, code, arrays.ptr(src), arrays.ptr(dst), nin, pptr,
            arrays.stream()))
        if not arrays.is_device(out_xg):
            arrays.writeback(out_xg, dst)

    def apply_potential(self, in_xg, out_xg, vt_g, phase_cd=None):
        """out_xg = A in_xg + vt_g in_xg in one pass (new API).

        The kinetic apply and the local potential of
        gpaw/wavefunctions/fd.py:77-80 (``kin.apply`` then
        ``ham.apply_local_potential``, gpaw/hamiltonian.py:397-424) fused:
        every band is read once and written once.  ``vt_g`` is one real grid
        of the operator's shape; float64 for float64 / complex128 bands,
        float32 for float32 / complex64.
        """
        self._check_grid(in_xg)
        self._check_grid(vt_g)
        if tuple(in_xg.shape) != tuple(out_xg.shape):
            raise ValueError('input and output shapes differ')
        if arrays.np_dtype_of(in_xg) != arrays.np_dtype_of(out_xg):
            raise ValueError('input and output dtypes differ')
        code = arrays.code_of(in_xg)
        want = np.float64 if code in (_lib.GPW_F64, _lib.GPW_C128) \
            else np.float32
        if tuple(vt_g.shape) != self.shape or \
                arrays.np_dtype_of(vt_g) != np.dtype(want):
            raise TypeError('vt_g must be one %s grid of shape %s'
                            % (np.dtype(want).name, self.shape))
        if code in (_lib.GPW_C128, _lib.GPW_C64) and phase_cd is not None:
            if np.asarray(phase_cd).shape != (3, 2):
                raise ValueError('phase_cd must have shape (3, 2)')
        nin = int(np.prod(in_xg.shape[:-3])) if len(in_xg.shape) > 3 else 1
        src = arrays.to_device(in_xg)
        pot = arrays.to_device(vt_g)
        dst = out_xg if arrays.is_device(out_xg) else None
        if dst is None:
            dst = arrays.empty_like_device(out_xg.shape, out_xg.dtype)
        pbuf, pptr = arrays.phases_arg(phase_cd)
        _lib.check(self._lib.gpw_operator_apply_potential(
            self._h, code, arrays.ptr(src), arrays.ptr(dst), nin, pptr,
            arrays.ptr(pot), arrays.stream()))
        if not arrays.is_device(out_xg):
            arrays.writeback(out_xg, dst)

    def scaled(self, alpha, beta=0.0):
        """The operator alpha A + beta I: coefficients scaled by alpha on the
        host, beta added to the centre (new API; lets the glue around an
        apply fold into it, see ``apply_fused``)."""
        coef = np.array(self.coef_p, float) * alpha
        centre = [i for i, o in enumerate(self.offset_pc) if not np.any(o)]
        if centre:
            coef[centre[0]] += beta
            op = FDOperator(coef, self.offset_pc, self.gd, self.dtype)
        else:
            op = FDOperator(np.hstack(([beta], coef)),
                            np.vstack(([[0, 0, 0]], self.offset_pc)),
                            self.gd, self.dtype)
        op.description = '%s scaled' % self.description
        return op

    def apply_fused(self, in_xg, out_xg, phase_cd=None, vt_g=None, aux=None,
                    aux_scale=1.0):
        """out = A in + vt in + aux_scale aux in one pass (new API;
        gpw_operator_apply_fused).  Device tensors."""
        self._check_grid(in_xg)
        code = arrays.code_of(in_xg)
        nin = int(np.prod(in_xg.shape[:-3])) if len(in_xg.shape) > 3 else 1
        src = arrays.to_device(in_xg)
        dst = arrays.to_device(out_xg)
        pot = None if vt_g is None else arrays.to_device(vt_g)
        ax = None if aux is None else arrays.to_device(aux)
        if ax is not None and (tuple(ax.shape) != tuple(dst.shape) or
                               arrays.code_of(ax) != code):
            raise ValueError('aux must have the output\'s shape and dtype')
        pbuf, pptr = arrays.phases_arg(phase_cd)
        _lib.check(self._lib.gpw_operator_apply_fused(
            self._h, code, arrays.ptr(src), arrays.ptr(dst), nin, pptr,
            None if pot is None else arrays.ptr(pot),
            None if ax is None else arrays.ptr(ax), float(aux_scale),
            arrays.stream()))

    def relax(self, relax_method, f_g, s_g, n, w=None):
        """n relaxation sweeps of A f = s (c/operators.c:49-91), in place.

        As in the reference one grid of shape n_c; a leading batch axis
        (nin, *n_c) relaxes nin independent grids in one call.
        """
        if w is None:
            w = 1.0
        self._check_grid(f_g)
        self._check_grid(s_g)
        if tuple(f_g.shape) != tuple(s_g.shape) or len(f_g.shape) > 4:
            raise ValueError('func and source must have the same shape')
        nin = int(f_g.shape[0]) if len(f_g.shape) == 4 else 1
        code = arrays.code_of(f_g)
        if code not in (_lib.GPW_F64, _lib.GPW_F32):
            raise TypeError('relax is defined for real grids only')
        if arrays.code_of(s_g) != code:
            raise TypeError('func and source dtypes differ')
        f = arrays.to_device(f_g)
        s = arrays.to_device(s_g)
        _lib.check(self._lib.gpw_operator_relax(
            self._h, code, int(relax_method), arrays.ptr(f), arrays.ptr(s),
            nin, int(n), float(w), arrays.stream()))
        if not arrays.is_device(f_g):
            arrays.writeback(f_g, f)

    def residual(self, f_g, s_g, r_g=None):
        """r = A f - s and sum |r|^2 per grid (device tensors; new API)."""
        import torch
        code = arrays.code_of(f_g)
        nin = int(np.prod(f_g.shape[:-3])) if len(f_g.shape) > 3 else 1
        f = arrays.to_device(f_g)
        s = arrays.to_device(s_g)
        out = torch.empty(nin, dtype=torch.float64, device='cuda')
        _lib.check(self._lib.gpw_operator_residual(
            self._h, code, arrays.ptr(f), arrays.ptr(s),
            arrays.ptr(r_g) if r_g is not None else None, nin,
            arrays.ptr(out), arrays.stream()))
        return out

    def get_diagonal_element(self):
        d = ctypes.c_double()
        _lib.check(self._lib.gpw_operator_get_diagonal_element(
            self._h, ctypes.byref(d)))
        return d.value

    def get_async_sizes(self):
        # (async-MPI flag, GPAW_ASYNC2, GPAW_ASYNC3) of c/operators.c:423-433
        return (0, 1, 1)


class Gradient(FDOperator):
    def __init__(self, gd, v, scale=1.0, n=1, dtype=float):
        h = (gd.h_cv ** 2).sum(1) ** 0.5
        d = gd.xxxiucell_cv[:, v]
        A = np.zeros((2 * n + 1, 2 * n + 1))
        for i, io in enumerate(range(-n, n + 1)):
            for j in range(2 * n + 1):
                A[i, j] = io ** j / float(fact(j))
        A[n, 0] = 1.0
        coefs = np.linalg.inv(A)[1]
        coefs = np.delete(coefs, len(coefs) // 2)
        offs = np.delete(np.arange(-n, n + 1), n)
        coef_p = []
        offset_pc = []
        for i in range(3):
            if abs(d[i]) > 1e-11:
                coef_p.extend(list(coefs * d[i] / h[i] * scale))
                offset = np.zeros((2 * n, 3), int)
                offset[:, i] = offs
                offset_pc.extend(offset)
        FDOperator.__init__(self, coef_p, offset_pc, gd, dtype,
                            'O(h^%d) %s-gradient stencil' % (2 * n, 'xyz'[v]))


def Laplace(gd, scale=1.0, n=1, dtype=float):
    if n == 9:
        raise NotImplementedError('FTLaplace (n=9, FFT) is outside the '
                                  'finite-difference hot path')
    return GUCLaplace(gd, scale, n, dtype)


class GUCLaplace(FDOperator):
    def __init__(self, gd, scale=1.0, n=1, dtype=float):
        """Laplacian for general (non-orthorhombic) cells, O(h^2n)."""
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
                    raise ValueError(
                        'You have a weird unit cell!  '
                        'Try to use the maximally reduced Niggli cell.  '
                        'See the ase.build.niggli_reduce() function.')
                break
        a_d *= scale
        offsets = [(0, 0, 0)]
        coefs = [laplace[n][0] * a_d.sum()]
        for d in range(D):
            M_c = M_ic[i_d[d]]
            offsets.extend(np.arange(1, n + 1)[:, np.newaxis] * M_c)
            coefs.extend(a_d[d] * np.array(laplace[n][1:]))
            offsets.extend(np.arange(-1, -n - 1, -1)[:, np.newaxis] * M_c)
            coefs.extend(a_d[d] * np.array(laplace[n][1:]))
        FDOperator.__init__(self, coefs, offsets, gd, dtype)
        self.description = (
            '%d*%d+1=%d point O(h^%d) finite-difference Laplacian' %
            ((self.npoints - 1) // n, n, self.npoints, 2 * n))


class LaplaceA(FDOperator):
    def __init__(self, gd, scale, dtype=float):
        assert gd.orthogonal
        c = np.divide(-1 / 12, gd.h_cv.diagonal() ** 2) * scale
        c0 = c[1] + c[2]
        c1 = c[0] + c[2]
        c2 = c[1] + c[0]
        a = -16.0 * np.sum(c)
        b = 10.0 * c + 0.125 * a
        FDOperator.__init__(self,
                            [a, b[0], b[0], b[1], b[1], b[2], b[2],
                             c0, c0, c0, c0, c1, c1, c1, c1, c2, c2, c2, c2],
                            [(0, 0, 0),
                             (-1, 0, 0), (1, 0, 0),
                             (0, -1, 0), (0, 1, 0),
                             (0, 0, -1), (0, 0, 1),
                             (0, -1, -1), (0, -1, 1), (0, 1, -1), (0, 1, 1),
                             (-1, 0, -1), (-1, 0, 1), (1, 0, -1), (1, 0, 1),
                             (-1, -1, 0), (-1, 1, 0), (1, -1, 0), (1, 1, 0)],
                            gd, dtype, 'O(h^4) Mehrstellen Laplacian (A)')


class LaplaceB(FDOperator):
    def __init__(self, gd, dtype=float):
        a = 0.5
        b = 1.0 / 12.0
        FDOperator.__init__(self, [a, b, b, b, b, b, b],
                            [(0, 0, 0), (-1, 0, 0), (1, 0, 0),
                             (0, -1, 0), (0, 1, 0), (0, 0, -1), (0, 0, 1)],
                            gd, dtype, 'O(h^4) Mehrstellen Laplacian (B)')


def apply_pseudo_hamiltonian(kin, psit_xG, Htpsit_xG, vt_G, phase_cd=None):
    """The grid part of gpaw/wavefunctions/fd.py:77-80 in one pass:
    ``kin.apply(psit_xG, Htpsit_xG, phase_cd)`` then
    ``Htpsit_xG += psit_xG * vt_G`` (gpaw/hamiltonian.py:397-424), fused in
    the kinetic stencil kernel.  The atomic (projector) and orbital-dependent
    XC terms that follow in the reference are not part of this path."""
    kin.apply_potential(psit_xG, Htpsit_xG, vt_G, phase_cd)
