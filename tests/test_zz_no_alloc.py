"""gpw_operator_residual_noalloc against gpw_operator_residual (C ABI, GPU).

The allocation-free variant exists for callers that must not allocate device
memory while they run (code inside another framework's memory pool or
allocator hook, processes that reserve all device memory up front): it keeps
the partial sums of the residual-norm reduction in a fixed array compiled
into the library.  Here both entry points run on the same inputs, twice in a
row (the second call must not see state left by the first), and must agree
within the tolerance of the other parity tests: 1e-12 relative for float64
residuals and norms, 2e-6 for float32.  The oversize case is rejected with a
clear error before anything is launched.

This file is collected last on purpose, and passes alone in a fresh process
as well as after the other tests.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GPW_F64, GPW_F32 = 0, 2


def make_op(lib, gd, nn, general=False):
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
    return h


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
    h = make_op(lib, gd, nn, general)
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
