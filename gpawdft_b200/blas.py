"""Device replacements of the NumPy / BLAS glue around the grid hot path.

``axpy`` / ``scal`` of gpaw/utilities/blas.py and ``integrate`` of
gpaw/grid_descriptor.py:263-292, on device tensors through libgpwgrid.so.
"""
import numpy as np

from . import _lib, arrays


def axpy(alpha, x, y):
    """y += alpha * x (device tensors of equal dtype and size)."""
    lib = _lib.load()
    a = complex(alpha)
    _lib.check(lib.gpw_axpy(arrays.code_of(y), y.numel(), a.real, a.imag,
                            arrays.ptr(x), arrays.ptr(y), arrays.stream()))


def scal(alpha, x):
    """x *= alpha."""
    lib = _lib.load()
    a = complex(alpha)
    _lib.check(lib.gpw_scal(arrays.code_of(x), x.numel(), a.real, a.imag,
                            arrays.ptr(x), arrays.stream()))


def add_scalar(x, c, out=None):
    """out = x + c (real tensors); in place when ``out`` is None."""
    lib = _lib.load()
    out = x if out is None else out
    _lib.check(lib.gpw_add_scalar(arrays.code_of(x), x.numel(), float(c),
                                  arrays.ptr(x), arrays.ptr(out),
                                  arrays.stream()))
    return out


def vector_sums(x, nvec):
    """Deterministic per-vector sums of a device tensor viewed as (nvec, n)."""
    import torch
    lib = _lib.load()
    code = arrays.code_of(x)
    ncomp = 2 if code in (_lib.GPW_C128, _lib.GPW_C64) else 1
    out = torch.empty(nvec * ncomp, dtype=torch.float64, device='cuda')
    _lib.check(lib.gpw_sum(code, nvec, x.numel() // nvec, arrays.ptr(x),
                           arrays.ptr(out), arrays.stream()))
    out = out.cpu().numpy()
    if ncomp == 2:
        return out[0::2] + 1j * out[1::2]
    return out


def vector_dots(x, y, nvec):
    import torch
    lib = _lib.load()
    out = torch.empty(nvec, dtype=torch.float64, device='cuda')
    _lib.check(lib.gpw_dot(arrays.code_of(x), nvec, x.numel() // nvec,
                           arrays.ptr(x), arrays.ptr(y), arrays.ptr(out),
                           arrays.stream()))
    return out.cpu().numpy()


def integrate_device(gd, a_xg, b_yg=None):
    a = arrays.to_device(a_xg)
    xshape = tuple(a.shape[:-3])
    nvec = int(np.prod(xshape)) if xshape else 1
    if b_yg is None:
        r = vector_sums(a, nvec) * gd.dv
    else:
        b = arrays.to_device(b_yg)
        r = vector_dots(a, b, nvec) * gd.dv
    if not xshape:
        return r[0].item()
    return r.reshape(xshape)
