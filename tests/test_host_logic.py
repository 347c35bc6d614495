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
