"""GPU parity of the FD operators against the oracle (c/operators.c path).

Covers Laplace (nn=1..3, star kernel) and Gradient on zero, periodic and
Bloch-phase boundaries, float64 / complex128 (reference types, 1e-12
relative) and float32 / complex64 (new forms), batched grids, in-place
apply, general-cell GUC and Mehrstellen stencils (general kernel, float64
bit-identical), Jacobi and Gauss-Seidel relaxation, the fused residual.
"""
import numpy as np
import pytest

from helpers import TOL, oracle_dtype, rand, relerr
from oracle import layer as ol
from oracle.geometry import GridDescriptor as OGD, phase_cd_for_k

pytestmark = pytest.mark.gpu

DTYPES = [np.float64, np.complex128, np.float32, np.complex64]


def gds(N, cell, pbc):
    from gpawdft_b200.grid_descriptor import GridDescriptor
    return GridDescriptor(N, cell, pbc), OGD(N, cell, pbc)


def phases_for(ogd, dtype, seed=11):
    if np.dtype(dtype).kind != 'c':
        return None
    rng = np.random.default_rng(seed)
    return phase_cd_for_k(ogd, rng.uniform(-0.5, 0.5, 3))


@pytest.mark.parametrize('pbc', [0, 1])
@pytest.mark.parametrize('dtype', DTYPES)
@pytest.mark.parametrize('nn', [1, 2, 3])
def test_laplace_apply(cuda, pbc, dtype, nn):
    from gpawdft_b200.fd_operators import Laplace
    N = (18, 14, 22)
    gd, ogd = gds(N, (3.4, 2.7, 4.1), pbc)
    a = rand((3,) + tuple(gd.n_c), dtype, 1)
    ph = phases_for(ogd, dtype)
    op = Laplace(gd, -0.5, nn, dtype)
    out = np.zeros_like(a)
    op.apply(a, out, ph)
    oop = ol.Laplace(ogd, -0.5, nn, oracle_dtype(dtype))
    ref = np.zeros(a.shape, oracle_dtype(dtype))
    oop.apply(a.astype(oracle_dtype(dtype)), ref, ph)
    assert relerr(out, ref) < TOL[np.dtype(dtype)]


@pytest.mark.parametrize('pbc', [0, 1])
@pytest.mark.parametrize('dtype', [np.float64, np.complex128])
@pytest.mark.parametrize('v', [0, 1, 2])
def test_gradient_apply(cuda, pbc, dtype, v):
    from gpawdft_b200.fd_operators import Gradient
    gd, ogd = gds((16, 20, 12), (3.0, 3.5, 2.4), pbc)
    a = rand(tuple(gd.n_c), dtype, 2)
    ph = phases_for(ogd, dtype)
    op = Gradient(gd, v, 1.0, 3, dtype)
    out = np.zeros_like(a)
    op.apply(a, out, ph)
    ref = np.zeros_like(a)
    ol.Gradient(ogd, v, 1.0, 3, dtype).apply(a, ref, ph)
    assert relerr(out, ref) < 1e-12


@pytest.mark.parametrize('cell', ['fcc', 'hex', 'bcc'])
@pytest.mark.parametrize('dtype', [np.float64, np.complex128])
def test_guc_laplace_bit_identical(cuda, cell, dtype):
    """Non-star stencils run the general kernel in the reference's order."""
    from gpawdft_b200.fd_operators import Laplace
    cells = {'fcc': [(0, 1.7, 1.7), (1.7, 0, 1.7), (1.7, 1.7, 0)],
             'hex': [(2.0, 0, 0), (1.0, 3 ** 0.5, 0), (0, 0, 2.2)],
             'bcc': [(-1.5, 1.5, 1.5), (1.5, -1.5, 1.5), (1.5, 1.5, -1.5)]}
    gd, ogd = gds((10, 10, 10), cells[cell], 1)
    a = rand((2,) + tuple(gd.n_c), dtype, 3)
    ph = phases_for(ogd, dtype)
    op = Laplace(gd, 1.0, 2, dtype)
    assert not op.cfd
    out = np.zeros_like(a)
    op.apply(a, out, ph)
    ref = np.zeros_like(a)
    ol.Laplace(ogd, 1.0, 2, dtype).apply(a, ref, ph)
    if np.dtype(dtype) == np.float64:
        assert np.array_equal(out, ref)
    else:
        assert relerr(out, ref) < 1e-14


def test_mehrstellen(cuda):
    """LaplaceA (edge offsets: general kernel, bit-identical) and LaplaceB
    (7-point star: fused star kernel, 1e-14)."""
    from gpawdft_b200.fd_operators import LaplaceA, LaplaceB
    from oracle import stencils
    gd, ogd = gds((20, 16, 18), (4.0, 3.2, 3.6), 0)
    a = rand(tuple(gd.n_c), np.float64, 4)
    for op, (c, o) in ((LaplaceA(gd, 0.7), stencils.laplace_A(ogd, 0.7)),
                       (LaplaceB(gd), stencils.laplace_B(ogd))):
        out = np.zeros_like(a)
        op.apply(a, out)
        ref = np.zeros_like(a)
        ol.FDOperator(c, o, ogd).apply(a, ref)
        if op.cfd:
            assert relerr(out, ref) < 1e-14
        else:
            assert np.array_equal(out, ref)


@pytest.mark.parametrize('N', [(3, 3, 3), (20, 16, 18), (21, 35, 70), (21, 35, 65)])
@pytest.mark.parametrize('pbc', [0, 1])
def test_mehrstellen_a_modes(cuda, N, pbc):
    """LaplaceA through its own kernels (compile-time offsets, register-held
    row segments; planes staged by TMA where the grid has zero boundaries
    and 16-byte rows, as the 64-point rows of (21, 35, 65) with zero
    boundaries, else by cp.async) on zero and periodic grids with partial
    tiles in both in-plane axes, batched: apply, residual and weighted
    Jacobi bit-identical to the reference's order (c/bmgs/fd.c, relax.c);
    float32 within 2e-6."""
    import torch
    from gpawdft_b200.fd_operators import LaplaceA
    from oracle import stencils
    gd, ogd = gds(N, tuple(0.21 * n for n in N), pbc)
    op = LaplaceA(gd, 0.7)
    c, o = stencils.laplace_A(ogd, 0.7)
    oop = ol.FDOperator(c, o, ogd)
    a = rand((3,) + tuple(gd.n_c), np.float64, 40)
    s = rand((3,) + tuple(gd.n_c), np.float64, 41)
    ref = np.zeros_like(a)
    oop.apply(a, ref)
    out = np.zeros_like(a)
    op.apply(a, out)
    assert np.array_equal(out, ref)
    r = torch.empty(a.shape, dtype=torch.float64, device='cuda')
    ss = op.residual(torch.from_numpy(a).cuda(), torch.from_numpy(s).cuda(), r)
    assert np.array_equal(r.cpu().numpy(), ref - s)
    assert np.allclose(ss.cpu().numpy(), ((ref - s).reshape(3, -1) ** 2).sum(1), rtol=1e-12)
    g = a[0].copy()
    og = a[0].copy()
    op.relax(2, g, s[0], 2, 2.0 / 3.0)
    oop.relax(2, og, s[0], 2, 2.0 / 3.0)
    assert np.array_equal(g, og)
    op32 = LaplaceA(gd, 0.7, np.float32)
    out32 = np.zeros(a.shape, np.float32)
    op32.apply(a.astype(np.float32), out32)
    assert relerr(out32, ref) < 2e-6


@pytest.mark.parametrize('N', [(2, 2, 2), (3, 5, 7), (8, 2, 9), (40, 33, 65)])
@pytest.mark.parametrize('pbc', [0, 1])
def test_odd_and_tiny_sizes(cuda, N, pbc):
    from gpawdft_b200.fd_operators import Laplace
    if pbc:
        N = tuple(max(n, 3) for n in N)
    gd, ogd = gds(N, tuple(0.3 * n for n in N), pbc)
    nn = 1 if min(gd.n_c) < 3 else 3
    a = rand(tuple(gd.n_c), np.float64, 5)
    out = np.zeros_like(a)
    Laplace(gd, 1.0, nn).apply(a, out)
    ref = np.zeros_like(a)
    ol.Laplace(ogd, 1.0, nn).apply(a, ref)
    assert relerr(out, ref) < 1e-12


def test_inplace_and_device_tensors(cuda):
    import torch
    from gpawdft_b200.fd_operators import Laplace
    gd, ogd = gds((24, 24, 24), (4.8, 4.8, 4.8), 1)
    a = rand((2,) + tuple(gd.n_c), np.float64, 6)
    ref = np.zeros_like(a)
    ol.Laplace(ogd, -0.5, 3).apply(a, ref)
    t = torch.from_numpy(a.copy()).cuda()
    Laplace(gd, -0.5, 3).apply(t, t)
    torch.cuda.synchronize()
    assert relerr(t.cpu().numpy(), ref) < 1e-12


def test_config_a_batch(cuda):
    """32 grids of 48^3, zero boundary, nn=3, h=0.2 A (benchmark config a)."""
    import torch
    from gpawdft_b200.fd_operators import Laplace
    h = 0.2 / 0.52917721
    gd, ogd = gds((49, 49, 49), (49 * h,) * 3, 0)
    a = rand((32, 48, 48, 48), np.float64, 0)
    t = torch.from_numpy(a).cuda()
    o = torch.empty_like(t)
    Laplace(gd, 1.0, 3).apply(t, o)
    ref = np.zeros((4, 48, 48, 48))
    ol.Laplace(ogd, 1.0, 3).apply(a[:4], ref)
    assert relerr(o[:4].cpu().numpy(), ref) < 1e-12


@pytest.mark.parametrize('pbc', [0, 1])
@pytest.mark.parametrize('nn', [1, 3])
@pytest.mark.parametrize('nrelax', [1, 2, 3])
def test_jacobi_relax(cuda, pbc, nn, nrelax):
    from gpawdft_b200.fd_operators import Laplace
    gd, ogd = gds((20, 18, 22), (4.0, 3.6, 4.4), pbc)
    f = rand(tuple(gd.n_c), np.float64, 7)
    s = rand(tuple(gd.n_c), np.float64, 8)
    g = f.copy()
    Laplace(gd, -0.25 / np.pi, nn).relax(2, g, s, nrelax, 2.0 / 3.0)
    r = f.copy()
    ol.Laplace(ogd, -0.25 / np.pi, nn).relax(2, r, s, nrelax, 2.0 / 3.0)
    assert relerr(g, r) < 1e-12


@pytest.mark.parametrize('pbc', [0, 1])
@pytest.mark.parametrize('nn', [1, 2])
def test_gauss_seidel_bit_identical(cuda, pbc, nn):
    from gpawdft_b200.fd_operators import Laplace
    gd, ogd = gds((8, 6, 10), (1.6, 1.2, 2.0), pbc)
    f = rand(tuple(gd.n_c), np.float64, 9)
    s = rand(tuple(gd.n_c), np.float64, 10)
    g = f.copy()
    Laplace(gd, -0.25 / np.pi, nn).relax(1, g, s, 2)
    r = f.copy()
    ol.Laplace(ogd, -0.25 / np.pi, nn).relax(1, r, s, 2)
    assert np.array_equal(g, r)


def test_float32_relax(cuda):
    from gpawdft_b200.fd_operators import Laplace
    gd, ogd = gds((20, 20, 20), (4.0, 4.0, 4.0), 0)
    f = rand(tuple(gd.n_c), np.float64, 7)
    s = rand(tuple(gd.n_c), np.float64, 8)
    g = f.astype(np.float32)
    Laplace(gd, -0.25 / np.pi, 3, np.float32).relax(2, g, s.astype(np.float32),
                                                     2, 2.0 / 3.0)
    r = f.copy()
    ol.Laplace(ogd, -0.25 / np.pi, 3).relax(2, r, s, 2, 2.0 / 3.0)
    assert relerr(g, r) < 2e-6


def test_residual_general_stencil(cuda):
    """Residual epilogue on the general-offset kernel (GUC fcc, periodic)."""
    import torch
    from gpawdft_b200.fd_operators import Laplace
    cell = [(0, 1.7, 1.7), (1.7, 0, 1.7), (1.7, 1.7, 0)]
    gd, ogd = gds((10, 10, 10), cell, 1)
    f = rand((2,) + tuple(gd.n_c), np.float64, 14)
    s = rand((2,) + tuple(gd.n_c), np.float64, 15)
    op = Laplace(gd, 1.0, 2)
    assert not op.cfd
    r = torch.empty(f.shape, dtype=torch.float64, device='cuda')
    ss = op.residual(torch.from_numpy(f).cuda(), torch.from_numpy(s).cuda(), r)
    ref = np.zeros_like(f)
    ol.Laplace(ogd, 1.0, 2).apply(f, ref)
    ref -= s
    assert np.array_equal(r.cpu().numpy(), ref)
    assert np.allclose(ss.cpu().numpy(), (ref.reshape(2, -1) ** 2).sum(1),
                       rtol=1e-12)


def test_residual_and_norm(cuda):
    import torch
    from gpawdft_b200.fd_operators import Laplace
    gd, ogd = gds((30, 26, 34), (6.0, 5.2, 6.8), 0)
    f = rand((2,) + tuple(gd.n_c), np.float64, 12)
    s = rand((2,) + tuple(gd.n_c), np.float64, 13)
    op = Laplace(gd, -0.25 / np.pi, 3)
    r = torch.empty(f.shape, dtype=torch.float64, device='cuda')
    ss = op.residual(torch.from_numpy(f).cuda(), torch.from_numpy(s).cuda(), r)
    ref = np.zeros_like(f)
    ol.Laplace(ogd, -0.25 / np.pi, 3).apply(f, ref)
    ref -= s
    assert relerr(r.cpu().numpy(), ref) < 1e-12
    exp = (ref.reshape(2, -1) ** 2).sum(1)
    assert np.allclose(ss.cpu().numpy(), exp, rtol=1e-12)


@pytest.mark.parametrize('pbc', [(1, 1, 1), (1, 0, 1), (0, 1, 0), (0, 0, 0)])
@pytest.mark.parametrize('dtype', [np.complex128, np.complex64])
@pytest.mark.parametrize('nn', [1, 2, 3])
def test_complex_tma_apply(cuda, pbc, dtype, nn):
    """Complex Bloch-phase Laplace and gradients (radius 1-3) on mixed
    zero / periodic boundaries, batched: wrapped halos on every axis with
    their phases."""
    from gpawdft_b200.fd_operators import Gradient, Laplace
    N = (12, 16, 20)
    gd, ogd = gds(N, (2.4, 3.1, 3.9), pbc)
    a = rand((2,) + tuple(gd.n_c), dtype, 5 + nn)
    ph = phases_for(ogd, dtype, seed=13)
    for make, omake in ((lambda: Laplace(gd, -0.5, nn, dtype),
                         lambda: ol.Laplace(ogd, -0.5, nn, complex)),
                        (lambda: Gradient(gd, 1, 1.0, nn, dtype),
                         lambda: ol.Gradient(ogd, 1, 1.0, nn, complex)),
                        (lambda: Gradient(gd, 0, 1.0, nn, dtype),
                         lambda: ol.Gradient(ogd, 0, 1.0, nn, complex))):
        out = np.zeros_like(a)
        make().apply(a, out, ph)
        ref = np.zeros(a.shape, complex)
        omake().apply(a.astype(complex), ref, ph)
        assert relerr(out, ref) < TOL[np.dtype(dtype)]
