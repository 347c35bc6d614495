"""Weighted finite-difference operator on the GPU (drop-in for
gpaw.wfd_operators).

``WeightedFDOperator(weights, operators)`` is the compound operator
A = sum_i weights[i](r) operators[i] of gpaw/wfd_operators.py:8-76 -- for the
dielectric Poisson solver a Laplacian and three gradients weighted by the
permittivity and its gradient.  The stencil tables are taken from the given
operators exactly as the reference takes them (a zero-offset tap prepended
where a stencil has none) and handed to ``gpw_woperator_new``, which
replaces ``_gpaw.WOperator`` (c/woperators.c).

The reference keeps pointers to the NumPy weight arrays, so changing them in
place changes the operator.  Here the weights are device tensors held by
reference (NumPy weights are copied to the device once, at construction);
every apply / relax passes their current device addresses, so updating the
tensors in place -- as the solver restricts them to the coarse levels before
each solve -- changes the operator the same way.
"""
import ctypes

import numpy as np

from . import _lib, arrays


class WeightedFDOperator:
    def __init__(self, weights, operators):
        assert len(weights) == len(operators)
        self.gd = operators[0].gd
        self.shape = tuple(int(x) for x in self.gd.n_c)
        self.coef_ps = []
        self.offset_ps = []
        for op in operators:
            assert op.gd is self.gd or tuple(op.gd.n_c) == self.shape
            assert np.dtype(operators[0].dtype) == np.dtype(op.dtype)
            offs = np.asarray(op.offset_p, np.int64)
            coefs = np.asarray(op.coef_p, float)
            if 0 in offs:
                assert offs[0] == 0
                self.offset_ps.append(np.ascontiguousarray(offs.copy()))
                self.coef_ps.append(np.ascontiguousarray(coefs.copy()))
            else:
                self.offset_ps.append(np.ascontiguousarray(
                    np.hstack(([0], offs)).astype(np.int64)))
                self.coef_ps.append(np.ascontiguousarray(
                    np.hstack(([0.0], coefs))))
        for weight in weights:
            assert tuple(weight.shape) == self.shape
            assert arrays.np_dtype_of(weight) == np.dtype(float)
        self.nweights = len(operators)
        self.cfd = all(op.cfd for op in operators)
        self.mp = max(op.mp for op in operators)
        self.dtype = operators[0].dtype
        self.npoints = max(op.npoints for op in operators)
        self.weights = [arrays.to_device(w) for w in weights]
        lib = _lib.load()
        n = self.nweights
        VP = ctypes.c_void_p
        cp = (VP * n)(*[c.ctypes.data for c in self.coef_ps])
        op_ = (VP * n)(*[o.ctypes.data for o in self.offset_ps])
        nc = (ctypes.c_int * n)(*[len(c) for c in self.coef_ps])
        size = np.ascontiguousarray(self.gd.n_c, np.int64)
        nb = np.ascontiguousarray(self.gd.neighbor_cd, np.int64)
        h = VP()
        _lib.check(lib.gpw_woperator_new(
            n, cp, op_, nc, size.ctypes.data, int(self.mp), nb.ctypes.data,
            int(np.dtype(self.dtype).kind == 'f'), int(self.cfd),
            ctypes.byref(h)))
        self._h = h
        self._lib = lib
        self.description = 'Weighted Finite Difference Operator\n  '
        self.description += '\n  '.join([op.description for op in operators])

    def __del__(self):
        h = getattr(self, '_h', None)
        if h is not None and h.value:
            self._lib.gpw_woperator_free(h)
            self._h = None

    def _wptrs(self):
        return (ctypes.c_void_p * self.nweights)(
            *[w.data_ptr() for w in self.weights])

    def _check_grid(self, a):
        if tuple(a.shape[-3:]) != self.shape:
            raise ValueError('grid shape %s does not match operator %s' %
                             (tuple(a.shape[-3:]), self.shape))

    def apply(self, in_xg, out_xg, phase_cd=None):
        """c/woperators.c:362-465 (the same weights for every leading grid)."""
        self._check_grid(in_xg)
        if tuple(in_xg.shape) != tuple(out_xg.shape):
            raise ValueError('input and output shapes differ')
        code = arrays.code_of(in_xg)
        if arrays.code_of(out_xg) != code:
            raise ValueError('input and output dtypes differ')
        nin = int(np.prod(in_xg.shape[:-3])) if len(in_xg.shape) > 3 else 1
        src = arrays.to_device(in_xg)
        dst = out_xg if arrays.is_device(out_xg) else \
            arrays.empty_like_device(out_xg.shape, out_xg.dtype)
        pbuf, pptr = arrays.phases_arg(phase_cd)
        _lib.check(self._lib.gpw_woperator_apply(
            self._h, code, self._wptrs(), arrays.ptr(src), arrays.ptr(dst),
            nin, pptr, arrays.stream()))
        if not arrays.is_device(out_xg):
            arrays.writeback(out_xg, dst)

    def relax(self, relax_method, f_g, s_g, n, w=None):
        """c/woperators.c:61-108: n weighted Gauss-Seidel (1) or Jacobi (2)
        sweeps of A f = s on one float64 grid, in place."""
        if w is None:
            w = 1.0
        self._check_grid(f_g)
        self._check_grid(s_g)
        if arrays.code_of(f_g) != _lib.GPW_F64 or \
                arrays.code_of(s_g) != _lib.GPW_F64:
            raise TypeError('weighted relax is defined for float64 grids')
        f = arrays.to_device(f_g)
        s = arrays.to_device(s_g)
        _lib.check(self._lib.gpw_woperator_relax(
            self._h, int(relax_method), self._wptrs(), arrays.ptr(f),
            arrays.ptr(s), int(n), float(w), arrays.stream()))
        if not arrays.is_device(f_g):
            arrays.writeback(f_g, f)

    def get_diagonal_element(self):
        """c/woperators.c:466-496: the largest |sum_i w_i c_i0|."""
        d = ctypes.c_double()
        _lib.check(self._lib.gpw_woperator_get_diagonal_element(
            self._h, self._wptrs(), ctypes.byref(d), arrays.stream()))
        return d.value

    def get_async_sizes(self):
        return (0, 1, 1)
