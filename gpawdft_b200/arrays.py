"""Device-array plumbing for the reference-facing API.

The reference's API works on NumPy arrays.  Here every call accepts either a
NumPy array (host; copied to the device, computed there, copied back -- the
end-to-end form) or a CUDA ``torch.Tensor`` (device-resident; zero copies).
PyTorch is used only for device memory and the current CUDA stream; all
arithmetic runs in libgpwgrid.so.
"""
import numpy as np

try:
    import torch
except ImportError:  # pragma: no cover - torch is part of the image
    torch = None

from . import _lib

_NP_TO_CODE = {np.dtype(np.float64): _lib.GPW_F64,
               np.dtype(np.complex128): _lib.GPW_C128,
               np.dtype(np.float32): _lib.GPW_F32,
               np.dtype(np.complex64): _lib.GPW_C64}


def _torch_maps():
    return ({torch.float64: _lib.GPW_F64, torch.complex128: _lib.GPW_C128,
             torch.float32: _lib.GPW_F32, torch.complex64: _lib.GPW_C64},
            {np.dtype(np.float64): torch.float64,
             np.dtype(np.complex128): torch.complex128,
             np.dtype(np.float32): torch.float32,
             np.dtype(np.complex64): torch.complex64})


def require_cuda():
    if torch is None or not torch.cuda.is_available():
        raise RuntimeError('gpawdft_b200 runs on a CUDA device (sm_100a); '
                           'no CPU fallback exists')
    _lib.load()


def is_device(a):
    return torch is not None and isinstance(a, torch.Tensor)


def stream():
    return ctypes_stream(torch.cuda.current_stream())


def ctypes_stream(s):
    return s.cuda_stream


def code_of(a):
    if is_device(a):
        t2c, _ = _torch_maps()
        return t2c[a.dtype]
    return _NP_TO_CODE[np.dtype(a.dtype)]


def np_dtype_of(a):
    if is_device(a):
        return np.dtype({torch.float64: np.float64,
                         torch.complex128: np.complex128,
                         torch.float32: np.float32,
                         torch.complex64: np.complex64}[a.dtype])
    return np.dtype(a.dtype)


def to_device(a):
    """CUDA tensor view of ``a`` (copied from the host for NumPy input)."""
    require_cuda()
    if is_device(a):
        if not a.is_cuda:
            raise ValueError('tensor must be on a CUDA device')
        if not a.is_contiguous():
            raise ValueError('array must be C-contiguous (as in the reference)')
        return a
    a = np.asarray(a)
    if not a.flags.c_contiguous:
        a = np.ascontiguousarray(a)
    _, np2t = _torch_maps()
    if np.dtype(a.dtype) not in np2t:
        raise TypeError('unsupported dtype %s' % a.dtype)
    return torch.from_numpy(a).to('cuda', non_blocking=False)


def empty_like_device(shape, dtype):
    _, np2t = _torch_maps()
    return torch.empty(tuple(shape), dtype=np2t[np.dtype(dtype)], device='cuda')


def writeback(dst, src_dev):
    """Copy a device result into ``dst`` (NumPy) or nothing if it is ``dst``."""
    if is_device(dst):
        if dst.data_ptr() != src_dev.data_ptr():
            dst.copy_(src_dev)
        return
    dst[...] = src_dev.cpu().numpy().reshape(dst.shape)


def ptr(t):
    return t.data_ptr()


def phases_arg(phase_cd):
    """(3, 2) complex phase table -> 12 interleaved doubles (host), or None."""
    if phase_cd is None:
        return None, None
    p = np.ascontiguousarray(np.asarray(phase_cd, complex).reshape(3, 2))
    buf = np.ascontiguousarray(p.view(np.float64).reshape(12))
    return buf, buf.ctypes.data
