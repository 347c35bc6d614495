"""GPU parity of restriction / interpolation (c/transformers.c path).

Every 1D pass evaluates the reference's expression in the reference's order
without fused multiply-add, so float64 / complex128 results are expected to
be bit-identical; float32 / complex64 are compared at 2e-6 relative.
"""
import numpy as np
import pytest

from helpers import TOL, oracle_dtype, rand, relerr
from oracle import layer as ol
from oracle.geometry import GridDescriptor as OGD, phase_cd_for_k

pytestmark = pytest.mark.gpu


def pair(N, pbc):
    from gpawdft_b200.grid_descriptor import GridDescriptor
    cell = tuple(0.25 * n for n in N)
    return GridDescriptor(N, cell, pbc), OGD(N, cell, pbc)


@pytest.mark.parametrize('pbc', [0, 1])
@pytest.mark.parametrize('nn', [1, 2, 3, 4])
@pytest.mark.parametrize('dtype', [np.float64, np.complex128, np.float32,
                                   np.complex64])
@pytest.mark.parametrize('direction', ['restrict', 'interpolate'])
def test_transformer(cuda, pbc, nn, dtype, direction):
    from gpawdft_b200.transformers import Transformer
    fine, ofine = pair((36, 28, 44), pbc)
    coarse, ocoarse = fine.coarsen(), ofine.coarsen()
    if direction == 'restrict':
        gi, go, ogi, ogo = fine, coarse, ofine, ocoarse
    else:
        gi, go, ogi, ogo = coarse, fine, ocoarse, ofine
    a = rand((2,) + tuple(gi.n_c), dtype, 21)
    ph = None
    if np.dtype(dtype).kind == 'c':
        ph = phase_cd_for_k(ogi, np.random.default_rng(5).uniform(-.5, .5, 3))
    out = Transformer(gi, go, nn, dtype).apply(a, None, ph)
    ref = ol.Transformer(ogi, ogo, nn, oracle_dtype(dtype)).apply(
        a.astype(oracle_dtype(dtype)), None, ph)
    if np.dtype(dtype) in (np.dtype(np.float64), np.dtype(np.complex128)):
        assert np.array_equal(out, ref), relerr(out, ref)
    else:
        assert relerr(out, ref) < TOL[np.dtype(dtype)]


@pytest.mark.parametrize('pbc', [0, 1])
@pytest.mark.parametrize('N', [(4, 4, 4), (6, 10, 8), (18, 4, 34)])
def test_small_grids(cuda, pbc, N):
    from gpawdft_b200.transformers import Transformer
    fine, ofine = pair(N, pbc)
    coarse, ocoarse = fine.coarsen(), ofine.coarsen()
    a = rand(tuple(fine.n_c), np.float64, 22)
    out = Transformer(fine, coarse, 1).apply(a)
    ref = ol.Transformer(ofine, ocoarse, 1).apply(a)
    assert np.array_equal(out, ref)
    b = rand(tuple(coarse.n_c), np.float64, 23)
    try:
        ref = ol.Transformer(ocoarse, ofine, 1).apply(b)
    except ValueError:
        with pytest.raises(ValueError):
            Transformer(coarse, fine, 1)
        return
    out = Transformer(coarse, fine, 1).apply(b)
    assert np.array_equal(out, ref)


def test_band_config_shapes(cuda):
    """96^3 <-> 48^3 periodic complex128, K=6 (benchmark config 2 shapes)."""
    import torch
    from gpawdft_b200.transformers import Transformer
    h = 0.18 / 0.52917721
    fine, ofine = pair((96, 96, 96), 1)
    from gpawdft_b200.grid_descriptor import GridDescriptor
    fine = GridDescriptor((96,) * 3, (96 * h,) * 3, 1)
    ofine = OGD((96,) * 3, (96 * h,) * 3, 1)
    coarse, ocoarse = fine.coarsen(), ofine.coarsen()
    ph = phase_cd_for_k(ofine, [0.13, -0.31, 0.27])
    a = rand((2, 96, 96, 96), np.complex128, 24)
    t = torch.from_numpy(a).cuda()
    r = Transformer(fine, coarse, 3, complex).apply(t, None, ph)
    back = Transformer(coarse, fine, 3, complex).apply(r, None, ph)
    rr = ol.Transformer(ofine, ocoarse, 3, complex).apply(a[:1], None, ph)
    bb = ol.Transformer(ocoarse, ofine, 3, complex).apply(rr, None, ph)
    assert np.array_equal(r[:1].cpu().numpy(), rr)
    assert np.array_equal(back[:1].cpu().numpy(), bb)


@pytest.fixture
def restrict_layout():
    from gpawdft_b200 import _lib
    lib = _lib.load()

    def pin(k):
        _lib.check(lib.gpw_set_restrict_layout(k))
    yield pin, lib
    _lib.check(lib.gpw_set_restrict_layout(0))


@pytest.mark.parametrize('layout', [1, 2, 3])
@pytest.mark.parametrize('pbc', [0, 1])
@pytest.mark.parametrize('nn', [1, 3, 4])
@pytest.mark.parametrize('dtype', [np.float64, np.complex128, np.complex64])
def test_restrict_layouts(cuda, restrict_layout, layout, pbc, nn, dtype):
    """Each restriction kernel pinned in turn (the tile kernel; the row
    kernel with 384 and with 192 threads) against the oracle: bit-identical
    for float64 / complex128.  Rows of 44 points (pbc) take the row kernel;
    rows of 43 complex64 / float64 points are not whole 16-byte units and
    keep the tile kernel, as real K = 2 restrictions keep theirs.  36 rows:
    the last tile of 8 coarse rows wraps 18 of its fine rows when periodic
    (nn = 4)."""
    from gpawdft_b200.transformers import Transformer
    pin, lib = restrict_layout
    pin(layout)
    fine, ofine = pair((36, 36, 44), pbc)
    coarse, ocoarse = fine.coarsen(), ofine.coarsen()
    a = rand((3,) + tuple(fine.n_c), dtype, 31)
    ph = None
    if np.dtype(dtype).kind == 'c':
        ph = phase_cd_for_k(ofine, np.random.default_rng(6).uniform(-.5, .5, 3))
    n0 = lib.gpw_restrict_rows_launch_count()
    out = Transformer(fine, coarse, nn, dtype).apply(a, None, ph)
    rows = lib.gpw_restrict_rows_launch_count() - n0
    ref = ol.Transformer(ofine, ocoarse, nn, oracle_dtype(dtype)).apply(
        a.astype(oracle_dtype(dtype)), None, ph)
    if np.dtype(dtype) == np.dtype(np.complex64):
        assert relerr(out, ref) < TOL[np.dtype(dtype)]
    else:
        assert np.array_equal(out, ref), relerr(out, ref)
    whole = fine.n_c[2] * np.dtype(dtype).itemsize % 16 == 0
    # real K = 2 restrictions keep their own kernels
    served = whole and (np.dtype(dtype).kind == 'c' or nn > 1)
    assert rows == (1 if layout > 1 and served else 0)


def test_restrict_rows_bands_equal_tile(cuda, restrict_layout):
    """96^3 -> 48^3 complex128 / complex64 Bloch bands, K = 6: both row
    layouts equal the tile kernel bit for bit (same operations, same order)."""
    import torch
    from gpawdft_b200.grid_descriptor import GridDescriptor
    from gpawdft_b200.transformers import Transformer
    pin, lib = restrict_layout
    h = 0.18 / 0.52917721
    fine = GridDescriptor((96,) * 3, (96 * h,) * 3, 1)
    ofine = OGD((96,) * 3, (96 * h,) * 3, 1)
    ph = phase_cd_for_k(ofine, [0.21, -0.44, 0.05])
    for dt, tdt in ((complex, torch.complex128), (np.complex64, torch.complex64)):
        g = torch.Generator(device='cuda').manual_seed(7)
        a = torch.randn((5, 96, 96, 96), dtype=tdt, device='cuda', generator=g)
        R = Transformer(fine, fine.coarsen(), 3, dt)
        outs = []
        for layout in (1, 2, 3):
            pin(layout)
            outs.append(R.apply(a, None, ph).cpu().numpy())
        assert np.array_equal(outs[0], outs[1])
        assert np.array_equal(outs[0], outs[2])
