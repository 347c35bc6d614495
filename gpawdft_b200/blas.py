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


def pair_dots(x, nx, y, ny):
    """out[ix, iy] = sum(conj(x[ix]) y[iy]) over (nx, n) / (ny, n) views."""
    import torch
    lib = _lib.load()
    code = arrays.code_of(x)
    if arrays.code_of(y) != code:
        raise TypeError('integrate: both arrays need the same dtype')
    cplx = code in (_lib.GPW_C128, _lib.GPW_C64)
    ncomp = 2 if cplx else 1
    n = x.numel() // nx
    if y.numel() != ny * n:
        raise ValueError('integrate: grid shapes differ')
    out = torch.empty(nx * ny * ncomp, dtype=torch.float64, device='cuda')
    _lib.check(lib.gpw_dotc_pairs(code, nx, ny, n, arrays.ptr(x),
                                  arrays.ptr(y), arrays.ptr(out),
                                  arrays.stream()))
    out = out.cpu().numpy()
    if cplx:
        out = out[0::2] + 1j * out[1::2]
    return out.reshape(nx, ny)


def integrate_device(gd, a_xg, b_yg=None):
    """gpaw/grid_descriptor.py:263-319 on the device.

    ``integrate(a)`` is ``sum(a) dv`` per leading index; ``integrate(a, b)``
    is the matrix ``sum(conj(a_x) b_y) dv`` over every pair of leading indices
    (shape ``xshape + yshape``), a Python scalar when both are single grids.
    When ``a is b`` the reference's rank-k update fills only one triangle; the
    full Hermitian matrix returned here agrees with it there.
    """
    a = arrays.to_device(a_xg)
    xshape = tuple(a.shape[:-3])
    nx = int(np.prod(xshape)) if xshape else 1
    if b_yg is None:
        r = vector_sums(a, nx) * gd.dv
        if not xshape:
            return r[0].item()
        return r.reshape(xshape)
    b = a if b_yg is a_xg else arrays.to_device(b_yg)
    yshape = tuple(b.shape[:-3])
    ny = int(np.prod(yshape)) if yshape else 1
    r = pair_dots(a, nx, b, ny) * gd.dv
    r = r.reshape(xshape + yshape)
    if r.ndim == 0:
        return r.item()
    return r
