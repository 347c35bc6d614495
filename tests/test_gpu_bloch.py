"""The periodic / Bloch TMA row kernel (gpw_bloch_tma.cuh) against the oracle
(c/operators.c apply over the c/bc.c halo, restated).

Shapes are chosen so the kernel serves them (rows whose staged boxes start
128-byte aligned; axis 1 a multiple of the tile rows), each with every
candidate tile layout pinned in turn (a warp per row, 4 or 8 warps; one
point a lane with several warps per row): lanes of 1-4 points, a last
lane with part
of its points (88 = 29 x 3 + 1), every mix of periodic and zero axes, Bloch
phases on every axis, Laplace radius 1-3 and gradients along each axis.
Tolerances as for the other stencils: 1e-12 (float64 / complex128) and
2e-6 (float32 / complex64) relative to the oracle's max norm.
"""
import numpy as np
import pytest

from helpers import TOL, oracle_dtype, rand, relerr
from oracle import layer as ol
from oracle.geometry import GridDescriptor as OGD, phase_cd_for_k

pytestmark = pytest.mark.gpu

DTYPES = [np.complex128, np.complex64, np.float64, np.float32]
PBCS = [(1, 1, 1), (1, 0, 1), (0, 1, 0), (0, 0, 1), (0, 0, 0)]


@pytest.fixture
def lib():
    from gpawdft_b200 import _lib
    lib = _lib.load()
    yield lib
    _lib.check(lib.gpw_set_bloch_layout(0))


def gds(N, cell, pbc):
    from gpawdft_b200.grid_descriptor import GridDescriptor
    return GridDescriptor(N, cell, pbc), OGD(N, cell, pbc)


def gpts_for(n, pbc):
    return tuple(m if p else m + 1 for m, p in zip(n, pbc))


def check(lib, dtype, gd, ogd, ops, nbatch, seed):
    from gpawdft_b200 import _lib
    a = rand((nbatch,) + tuple(gd.n_c), dtype, seed)
    ph = None
    if np.dtype(dtype).kind == 'c':
        rng = np.random.default_rng(seed + 100)
        ph = phase_cd_for_k(ogd, rng.uniform(-0.5, 0.5, 3))
    for layout in (1, 2, 3, 4):
        _lib.check(lib.gpw_set_bloch_layout(layout))
        for make, omake in ops:
            before = lib.gpw_bloch_launch_count()
            out = np.zeros_like(a)
            make().apply(a, out, ph)
            # every shape has a first layout; a shape with fewer layouts
            # than the index keeps its tuned kernel
            if layout == 1:
                assert lib.gpw_bloch_launch_count() > before, 'not served'
            ref = np.zeros(a.shape, oracle_dtype(dtype))
            omake().apply(a.astype(oracle_dtype(dtype)), ref, ph)
            assert relerr(out, ref) < TOL[np.dtype(dtype)], layout


@pytest.mark.parametrize('pbc', PBCS)
@pytest.mark.parametrize('dtype', DTYPES)
@pytest.mark.parametrize('nn', [1, 2, 3])
def test_bloch_laplace(cuda, lib, pbc, dtype, nn):
    if pbc == (0, 0, 0) and np.dtype(dtype).kind == 'f':
        pytest.skip('real zero-boundary grids take the zero-boundary TMA kernel')
    n = (10, 16, 32)
    gd, ogd = gds(gpts_for(n, pbc), (2.0, 3.2, 6.4), pbc)
    assert tuple(gd.n_c) == n
    from gpawdft_b200.fd_operators import Laplace
    od = oracle_dtype(dtype)
    check(lib, dtype, gd, ogd,
          [(lambda: Laplace(gd, -0.5, nn, dtype),
            lambda: ol.Laplace(ogd, -0.5, nn, od))], 2, 7 + nn)


@pytest.mark.parametrize('n2', [64, 88, 96, 128])
@pytest.mark.parametrize('dtype', [np.complex128, np.complex64])
def test_bloch_row_widths(cuda, lib, n2, dtype):
    """2-4 points per lane, and a partly filled last lane (88)."""
    from gpawdft_b200.fd_operators import Gradient, Laplace
    if np.dtype(dtype) == np.complex64 and (n2 * 8 * 3) % 128:
        pytest.skip('row not 128-byte aligned for a 3-row halo box')
    pbc = (1, 1, 1)
    n = (8, 16, n2)
    gd, ogd = gds(n, (1.6, 3.2, 0.2 * n2), pbc)
    od = oracle_dtype(dtype)
    ops = [(lambda: Laplace(gd, -0.5, 3, dtype),
            lambda: ol.Laplace(ogd, -0.5, 3, od))]
    for v in range(3):
        ops.append((lambda v=v: Gradient(gd, v, 1.0, 3, dtype),
                    lambda v=v: ol.Gradient(ogd, v, 1.0, 3, od)))
    check(lib, dtype, gd, ogd, ops, 2, n2)


def test_bloch_band_block(cuda, lib):
    """The band-stencil shape at reduced band count: 6 bands of 96^3
    complex128 with Bloch phases, Laplace nn=3 (the eigensolver's kinetic
    operator at scale -0.5)."""
    from gpawdft_b200.fd_operators import Laplace
    pbc = (1, 1, 1)
    n = (96, 96, 96)
    gd, ogd = gds(n, (17.28, 17.28, 17.28), pbc)
    check(lib, np.complex128, gd, ogd,
          [(lambda: Laplace(gd, -0.5, 3, np.complex128),
            lambda: ol.Laplace(ogd, -0.5, 3, complex))], 6, 3)
