"""gpw_operator_residual_noalloc against gpw_operator_residual (C ABI, GPU).

The allocation-free variant exists for callers that must not allocate device
memory while they run (code inside another framework's memory pool or
allocator hook, processes that reserve all device memory up front): it keeps
the partial sums of the residual-norm reduction in a fixed array compiled
into the library.  Here both entry points run on the same inputs, twice in a
row (the second call must not see state left by the first), and must agree
within the tolerance of the other parity tests: 1e-12 relative for float64
residuals and norms, 2e-6 for float32.  Both are also checked against the
oracle's residual ``A f - s`` and its squared norm (so a fault shared by the
two entry points' kernels cannot pass), and the norm-only form (``r`` NULL)
runs at a valid size.  Requests beyond either limit of the fixed array (grids
per call, reduction blocks per call) are rejected with a clear error before
anything is launched.

This file is collected last on purpose, and passes alone in a fresh process
as well as after the other tests.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GPW_F64, GPW_F32 = 0, 2


def make_op(lib, gd, nn, general=False, tables=False):
    from oracle import stencils
    if general:
        c, o = stencils.guc_laplace(gd, 1.0, nn)
    else:
        c, o = stencils.guc_laplace(gd, -0.25 / np.pi, nn)
    mp, off, cfd = stencils.operator_layout(o, gd.n_c)
    size = np.ascontiguousarray(gd.n_c, np.int64)
    nb = np.ascontiguousarray(gd.neighbor_cd, np.int64)
    h = ctypes.c_void_p()
    rc = lib.gpw_operator_new(c.ctypes.data, off.ctypes.data, len(c),
                              size.ctypes.data, mp, nb.ctypes.data, 1, int(cfd),
                              ctypes.byref(h))
    assert rc == 0, lib.gpw_last_error()
    return (h, c, o) if tables else h


def oracle_residual(c, o, gd, f, s):
    """r = A f - s and per-grid sum(r^2), in float64 on the CPU."""
    from oracle import layer as ol
    op = ol.FDOperator(c, o, gd, float, 'numpy')
    f = f.astype(np.float64)
    r = np.empty_like(f)
    op.apply(f, r)
    r -= s.astype(np.float64)
    return r, (r.reshape(len(r), -1) ** 2).sum(axis=1)


CASES = [
    # (N_c, cell, pbc, nn, general offsets, nin, dtype)
    ((33, 29, 37), (6.6, 5.8, 7.4), 0, 3, False, 3, 'f64'),
    ((24, 24, 24), (4.8, 4.8, 4.8), 1, 1, False, 2, 'f32'),
    ((10, 10, 10), [(0, 1.7, 1.7), (1.7, 0, 1.7), (1.7, 1.7, 0)], 1, 2, True,
     2, 'f64'),
]


@pytest.mark.parametrize('case', CASES, ids=['star-f64', 'star-f32', 'general'])
def test_noalloc_matches_allocating_entry_point(case):
    import torch
    from gpawdft_b200 import _lib
    from oracle.geometry import GridDescriptor
    N, cell, pbc, nn, general, nin, dt = case
    lib = _lib.load()
    gd = GridDescriptor(N, cell, pbc)
    h, c, o = make_op(lib, gd, nn, general, tables=True)
    tdt = torch.float64 if dt == 'f64' else torch.float32
    code = GPW_F64 if dt == 'f64' else GPW_F32
    tol = 1e-12 if dt == 'f64' else 2e-6
    shape = (nin,) + tuple(int(x) for x in gd.n_c)
    g = torch.Generator(device='cuda').manual_seed(7)
    f = torch.randn(shape, dtype=tdt, device='cuda', generator=g)
    s = torch.randn(shape, dtype=tdt, device='cuda', generator=g)
    stream = torch.cuda.current_stream().cuda_stream
    r_ref = torch.empty_like(f)
    n_ref = torch.empty(nin, dtype=torch.float64, device='cuda')
    rc = lib.gpw_operator_residual(h, code, f.data_ptr(), s.data_ptr(),
                                   r_ref.data_ptr(), nin, n_ref.data_ptr(),
                                   stream)
    assert rc == 0, lib.gpw_last_error()
    for call in range(2):
        r = torch.full_like(f, float('nan'))
        n = torch.full((nin,), float('nan'), dtype=torch.float64, device='cuda')
        rc = lib.gpw_operator_residual_noalloc(h, code, f.data_ptr(),
                                               s.data_ptr(), r.data_ptr(), nin,
                                               n.data_ptr(), stream)
        assert rc == 0, lib.gpw_last_error()
        torch.cuda.synchronize()
        rr, rn = r.cpu().double().numpy(), r_ref.cpu().double().numpy()
        assert np.abs(rr - rn).max() <= tol * np.abs(rn).max(), call
        assert np.allclose(n.cpu().numpy(), n_ref.cpu().numpy(), rtol=tol,
                           atol=0), call
    # against the oracle (float32 residuals carry the inputs' rounding)
    ro, no = oracle_residual(c, o, gd, f.cpu().numpy(), s.cpu().numpy())
    assert np.abs(rr - ro).max() <= tol * np.abs(ro).max()
    assert np.allclose(n.cpu().numpy(), no, rtol=5 * tol, atol=0)
    # norm only (r NULL), twice: the same norms
    for call in range(2):
        n2 = torch.full((nin,), float('nan'), dtype=torch.float64,
                        device='cuda')
        rc = lib.gpw_operator_residual_noalloc(h, code, f.data_ptr(),
                                               s.data_ptr(), None, nin,
                                               n2.data_ptr(), stream)
        assert rc == 0, lib.gpw_last_error()
        torch.cuda.synchronize()
        assert np.allclose(n2.cpu().numpy(), n.cpu().numpy(), rtol=tol,
                           atol=0), call
    lib.gpw_operator_free(h)


def test_noalloc_rejects_oversize():
    import torch
    from gpawdft_b200 import _lib
    from oracle.geometry import GridDescriptor
    lib = _lib.load()
    gd = GridDescriptor((8, 8, 8), (2.0, 2.0, 2.0), 0)
    h = make_op(lib, gd, 1)
    x = torch.zeros((1,) + tuple(int(v) for v in gd.n_c), dtype=torch.float64,
                    device='cuda')
    n = torch.zeros(1, dtype=torch.float64, device='cuda')
    stream = torch.cuda.current_stream().cuda_stream
    # more grids than the fixed scratch has counters for: rejected up front
    rc = lib.gpw_operator_residual_noalloc(h, GPW_F64, x.data_ptr(),
                                           x.data_ptr(), None, 5000,
                                           n.data_ptr(), stream)
    assert rc == _lib.GPW_EINVAL
    assert b'4096' in lib.gpw_last_error()
    lib.gpw_operator_free(h)


def test_noalloc_rejects_too_many_reduction_blocks():
    """257 grids of 2 x 512 x 512 points need 256 tiles (32 x 32) each:
    65,792 reduction blocks, more than the 65,536 partial sums of the fixed
    array.  The inputs are real, correctly sized buffers, so the call would be
    valid apart from the limit; it must be refused before any launch."""
    import torch
    from gpawdft_b200 import _lib
    from oracle.geometry import GridDescriptor
    lib = _lib.load()
    gd = GridDescriptor((3, 513, 513), (0.6, 102.6, 102.6), 0)
    assert tuple(gd.n_c) == (2, 512, 512)
    h = make_op(lib, gd, 1)
    nin = 257
    x = torch.zeros((nin,) + tuple(int(v) for v in gd.n_c),
                    dtype=torch.float32, device='cuda')
    n = torch.zeros(nin, dtype=torch.float64, device='cuda')
    stream = torch.cuda.current_stream().cuda_stream
    rc = lib.gpw_operator_residual_noalloc(h, GPW_F32, x.data_ptr(),
                                           x.data_ptr(), None, nin,
                                           n.data_ptr(), stream)
    assert rc == _lib.GPW_EINVAL
    assert b'65536' in lib.gpw_last_error()
    # the same request within the limit (fewer grids) runs
    rc = lib.gpw_operator_residual_noalloc(h, GPW_F32, x.data_ptr(),
                                           x.data_ptr(), None, 255,
                                           n.data_ptr(), stream)
    assert rc == 0, lib.gpw_last_error()
    torch.cuda.synchronize()
    assert (n[:255].cpu().numpy() == 0).all()
    lib.gpw_operator_free(h)
