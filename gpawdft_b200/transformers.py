"""Restriction / interpolation on the GPU (drop-in for gpaw.transformers).

``Transformer(gdin, gdout, nn=1, dtype=float)`` with
``apply(input, output=None, phases=None) -> output`` as in
gpaw/transformers.py:17-125.  The pad / neighbour-pad / skip tables are
computed on the host exactly as the reference computes them (:31-58) and
passed to ``gpw_transformer_new``, which replaces ``_gpaw.Transformer``
(c/transformers.c:219-262).
"""
import ctypes

import numpy as np

from . import _lib, arrays


class _Transformer:
    def __init__(self, gdin, gdout, nn=1, dtype=float):
        self.gdin = gdin
        self.gdout = gdout
        self.nn = nn
        assert 1 <= nn <= 4
        self.dtype = dtype
        pad_cd = np.empty((3, 2), np.int64)
        neighborpad_cd = np.empty((3, 2), np.int64)
        skip_cd = np.zeros((3, 2), np.int64)
        if (gdin.N_c == 2 * gdout.N_c).all():
            # restriction
            pad_cd[:, 0] = 2 * nn - 1 - 2 * gdout.beg_c + gdin.beg_c
            pad_cd[:, 1] = 2 * nn - 2 + 2 * gdout.end_c - gdin.end_c
            neighborpad_cd[:, 0] = 2 * nn - 2 + 2 * gdout.beg_c - gdin.beg_c
            neighborpad_cd[:, 1] = 2 * nn - 1 - 2 * gdout.end_c + gdin.end_c
            self.interpolate = False
        else:
            assert (gdout.N_c == 2 * gdin.N_c).all()
            # interpolation
            pad_cd[:, 0] = nn - 1 - gdout.beg_c // 2 + gdin.beg_c
            pad_cd[:, 1] = nn + gdout.end_c // 2 - gdin.end_c
            neighborpad_cd[:, 0] = nn + gdout.beg_c // 2 - gdin.beg_c
            neighborpad_cd[:, 1] = nn - 1 - gdout.end_c // 2 + gdin.end_c
            skip_cd[:, 0] = gdout.beg_c % 2
            skip_cd[:, 1] = gdout.end_c % 2
            self.interpolate = True
            inpoints = (gdin.n_c[0] + 2 * nn - 1) * (gdin.n_c[1] + 2 * nn - 1)
            outpoints = gdout.n_c[0] * gdout.n_c[1]
            if inpoints > outpoints:
                points = ' x '.join([str(N) for N in gdin.N_c])
                raise ValueError('Cannot construct interpolator.  Grid %s '
                                 'may be too small' % points)
        assert (pad_cd.ravel() >= 0).all()
        self.ngpin = tuple(int(x) for x in gdin.n_c)
        self.ngpout = tuple(int(x) for x in gdout.n_c)
        self.pad_cd = pad_cd
        self.neighborpad_cd = neighborpad_cd
        self.skip_cd = skip_cd
        lib = _lib.load()
        si = np.ascontiguousarray(gdin.n_c, np.int64)
        so = np.ascontiguousarray(gdout.n_c, np.int64)
        nb = np.ascontiguousarray(gdin.neighbor_cd, np.int64)
        h = ctypes.c_void_p()
        _lib.check(lib.gpw_transformer_new(
            si.ctypes.data, so.ctypes.data, 2 * nn, pad_cd.ctypes.data,
            neighborpad_cd.ctypes.data, skip_cd.ctypes.data, nb.ctypes.data,
            int(np.dtype(dtype).kind == 'f'), int(self.interpolate),
            ctypes.byref(h)))
        self._h = h
        self._lib = lib

    def __del__(self):
        h = getattr(self, '_h', None)
        if h is not None and h.value:
            self._lib.gpw_transformer_free(h)
            self._h = None

    @property
    def handle(self):
        return self._h

    def apply(self, input, output=None, phases=None):
        if tuple(input.shape[-3:]) != self.ngpin:
            raise ValueError('input grid %s does not match %s' %
                             (tuple(input.shape[-3:]), self.ngpin))
        xshape = tuple(input.shape[:-3])
        dev_out = output is None and arrays.is_device(input)
        if output is None:
            if arrays.is_device(input):
                output = arrays.empty_like_device(
                    xshape + self.ngpout, arrays.np_dtype_of(input))
            else:
                output = self.gdout.empty(xshape, dtype=input.dtype)
        if tuple(output.shape[-3:]) != self.ngpout:
            raise ValueError('output grid does not match')
        code = arrays.code_of(input)
        if arrays.code_of(output) != code:
            raise ValueError('input and output dtypes differ')
        nin = int(np.prod(xshape)) if xshape else 1
        src = arrays.to_device(input)
        dst = output if arrays.is_device(output) else \
            arrays.empty_like_device(output.shape, output.dtype)
        pbuf, pptr = arrays.phases_arg(phases)
        _lib.check(self._lib.gpw_transformer_apply(
            self._h, code, arrays.ptr(src), arrays.ptr(dst), nin, pptr,
            arrays.stream()))
        if not arrays.is_device(output):
            arrays.writeback(output, dst)
        del dev_out
        return output

    def apply_subtract(self, input, base, output, phases=None):
        """output = base - I(input) in one pass (interpolation only; device
        tensors; gpw_transformer_apply_subtract)."""
        code = arrays.code_of(input)
        nin = int(np.prod(input.shape[:-3])) if len(input.shape) > 3 else 1
        pbuf, pptr = arrays.phases_arg(phases)
        _lib.check(self._lib.gpw_transformer_apply_subtract(
            self._h, code, arrays.ptr(input), arrays.ptr(base),
            arrays.ptr(output), nin, pptr, arrays.stream()))
        return output

    def get_async_sizes(self):
        return (0, 1)


def Transformer(gdin, gdout, nn=1, dtype=float):
    """gpaw/transformers.py:112-125 (nn=9: identity copy)."""
    if nn != 9:
        return _Transformer(gdin, gdout, nn, dtype)

    class T:
        nn = 1

        def apply(self, input, output, phases=None):
            output[:] = input
            return output

    return T()
