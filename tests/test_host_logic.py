"""Host-side mirror of the reference interface, checked against the oracle.

The product's geometry, stencil tables, transformer pad tables and multigrid
schedule are built on the host (no GPU needed) and must equal the oracle's
restatement of gpaw/grid_descriptor.py, fd_operators.py, transformers.py and
poisson.py.
"""
import numpy as np
import pytest

from gpawdft_b200.grid_descriptor import GridDescriptor
from oracle import layer, stencils
from oracle.geometry import GridDescriptor as OGD

CELLS = [((12, 10, 14), (3.0, 2.5, 3.5)),
         ((8, 8, 8), [(0, 1.7, 1.7), (1.7, 0, 1.7), (1.7, 1.7, 0)]),
         ((10, 10, 12), [(2.0, 0, 0), (1.0, 3 ** 0.5, 0), (0, 0, 2.4)])]


@pytest.mark.parametrize('pbc', [0, 1])
@pytest.mark.parametrize('N,cell', CELLS)
def test_geometry(N, cell, pbc):
    gd, ogd = GridDescriptor(N, cell, pbc), OGD(N, cell, pbc)
    for attr in ('N_c', 'n_c', 'beg_c', 'end_c', 'h_cv', 'neighbor_cd',
                 'sdisp_cd', 'icell_cv', 'xxxiucell_cv'):
        assert np.array_equal(getattr(gd, attr), getattr(ogd, attr)), attr
    assert gd.dv == ogd.dv
    assert np.array_equal(gd.get_grid_point_coordinates(),
                          ogd.get_grid_point_coordinates())


@pytest.mark.parametrize('nn', [1, 2, 3, 4, 5])
@pytest.mark.parametrize('N,cell', CELLS)
def test_stencil_tables(N, cell, nn):
    from gpawdft_b200.fd_operators import Gradient, Laplace
    gd, ogd = GridDescriptor(N, cell, 1), OGD(N, cell, 1)
    op = Laplace(gd, -0.5, nn)
    c, o = stencils.guc_laplace(ogd, -0.5, nn)
    mp, off, cfd = stencils.operator_layout(o, ogd.n_c)
    assert np.array_equal(op.coef_p, c)
    assert np.array_equal(op.offset_p, off)
    assert (op.mp, op.cfd) == (mp, cfd)
    assert op.get_diagonal_element() == c[0]
    for v in range(3):
        g = Gradient(gd, v, 1.0, nn)
        cg, og = stencils.gradient(ogd, v, 1.0, nn)
        assert np.array_equal(g.coef_p, cg)
        assert np.array_equal(g.offset_pc, og)


@pytest.mark.parametrize('pbc', [0, 1])
@pytest.mark.parametrize('nn', [1, 2, 3, 4])
def test_transformer_tables(pbc, nn):
    from gpawdft_b200.transformers import Transformer
    gd, ogd = GridDescriptor((32, 24, 40), (8, 6, 10), pbc), \
        OGD((32, 24, 40), (8, 6, 10), pbc)
    for gi, go, ogi, ogo in ((gd, gd.coarsen(), ogd, ogd.coarsen()),
                             (gd.coarsen(), gd, ogd.coarsen(), ogd)):
        t = Transformer(gi, go, nn)
        pad, npad, skip, interp = layer.transformer_tables(ogi, ogo, nn)
        assert np.array_equal(t.pad_cd, pad)
        assert np.array_equal(t.neighborpad_cd, npad)
        assert np.array_equal(t.skip_cd, skip)
        assert t.interpolate == interp


@pytest.mark.parametrize('N', [32, 48, 64, 128, 192])
def test_poisson_hierarchy(N):
    from gpawdft_b200.poisson import PoissonSolver
    gd, ogd = GridDescriptor((N,) * 3, (N * 0.4,) * 3, 0), \
        OGD((N,) * 3, (N * 0.4,) * 3, 0)
    ps = PoissonSolver(nn=3)
    ps.set_grid_descriptor(gd)
    ops = layer.PoissonSolver(nn=3)
    ops.set_grid_descriptor(ogd)
    assert ps.levels == ops.levels
    assert ps.presmooths == ops.presmooths
    assert ps.postsmooths == ops.postsmooths
    assert ps.weights == ops.weights
    for a, b in zip(ps.operators, ops.operators):
        assert np.array_equal(a.coef_p, b.coef_p)
        assert a.shape == b.shape
    assert 'Jacobi solver with %d multi-grid levels' % (ps.levels + 1) in \
        ps.get_description()


def test_interpolator_too_small_raises():
    from gpawdft_b200.transformers import Transformer
    gd = GridDescriptor((12, 8, 16), (3, 2, 4), 0)
    with pytest.raises(ValueError):
        Transformer(gd.coarsen(), gd, 3)


def test_inner_schedule_layout():
    """Float32 inner schedule: Chebyshev-weighted Jacobi sweeps whose error
    polynomial prod(1 - w_i lambda) equals 1 / T_k on the damped range."""
    from gpawdft_b200.poisson import (PoissonSolver, chebyshev_weights,
                                      inner_schedule, jacobi_spectrum)
    N = 64
    gd = GridDescriptor((N,) * 3, (N * 0.4,) * 3, 0)
    ps = PoissonSolver(nn=3, precision='fp32')
    ps.set_grid_descriptor(gd)
    npre, npost, ws = inner_schedule(ps.operators)
    L = len(ps.operators)
    assert npre == [2] + [3] * (L - 2) + [0]
    assert npost == [2] + [3] * (L - 2) + [8]
    assert len(ws) == sum(npre) + sum(npost)
    assert all(w > 0 for w in ws)
    # level 0: 19-point sixth-order Laplacian, lambda_max(D^-1 A) -> 2.2204
    hi = jacobi_spectrum(ps.operators[0])
    assert 2.21 < hi < 2.2205
    # pre-sweeps smallest weight first, post-sweeps reversed
    assert ws[:2] == sorted(ws[:2]) and ws[2:4] == ws[:2][::-1]
    for k, ratio in ((2, 6.0), (3, 4.0)):
        lo = hi / ratio
        w = chebyshev_weights(k, lo, hi)
        lam = np.linspace(lo, hi, 2001)
        p = np.prod([1 - wi * lam for wi in w], axis=0)
        x0 = (hi + lo) / (hi - lo)
        tk = np.cosh(k * np.arccosh(x0))
        assert np.abs(p).max() <= 1 / tk * (1 + 1e-9)
    # the 1^3 coarsest grid: one exact sweep (D^-1 A = 1)
    assert jacobi_spectrum(ps.operators[-1]) == pytest.approx(1.0)
