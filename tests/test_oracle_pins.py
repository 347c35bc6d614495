"""Pins of the NumPy restatement against the compiled reference C (oracle/_ref).

Random inputs beyond the committed fixtures: every operator family, both
boundary kinds, real and complex, must agree bit for bit.  Skipped where the
reference's C could not be built (the fixtures in test_oracle_golden.py still
pin the restatement there).
"""
import numpy as np
import pytest

from oracle import layer, ref
from oracle.geometry import GridDescriptor, phase_cd_for_k

pytestmark = pytest.mark.skipif(not ref.available(),
                                reason='reference C (oracle/_ref) not built')


def rnd(shape, dtype, seed):
    rng = np.random.default_rng(seed)
    a = rng.standard_normal(shape)
    return a + 1j * rng.standard_normal(shape) if dtype == complex else a


@pytest.mark.parametrize('pbc', [0, 1])
@pytest.mark.parametrize('dtype', [float, complex])
def test_operators_and_transformers(pbc, dtype):
    gd = GridDescriptor((24, 20, 28), (6.0, 5.0, 7.0), pbc)
    ph = phase_cd_for_k(gd, [0.3, -0.1, 0.45]) if dtype == complex else None
    a = rnd((2,) + tuple(gd.n_c), dtype, 1)
    for nn in (1, 2, 3, 4):
        outs = []
        for be in ('numpy', 'ref'):
            o = np.zeros_like(a)
            layer.Laplace(gd, -0.5, nn, dtype, be).apply(a, o, ph)
            outs.append(o)
        assert np.array_equal(*outs)
    for nn in (1, 2, 3, 4):
        for gi, go in ((gd, gd.coarsen()), (gd.coarsen(), gd)):
            x = rnd(tuple(gi.n_c), dtype, 2)
            outs = [layer.Transformer(gi, go, nn, dtype, be).apply(x, None, ph)
                    for be in ('numpy', 'ref')]
            assert np.array_equal(*outs)


@pytest.mark.parametrize('method', [1, 2])
def test_relax(method):
    gd = GridDescriptor((10, 8, 12), (2.5, 2.0, 3.0), 0)
    f = rnd(tuple(gd.n_c), float, 3)
    s = rnd(tuple(gd.n_c), float, 4)
    outs = []
    for be in ('numpy', 'ref'):
        g = f.copy()
        layer.Laplace(gd, -0.25 / np.pi, 2, float, be).relax(method, g, s, 2,
                                                              2.0 / 3.0)
        outs.append(g)
    assert np.array_equal(*outs)


def test_poisson_solve():
    from gpawdft_b200.workloads import gaussian_density
    rho, L = gaussian_density(32, 0.2, 8, 1)
    gd = GridDescriptor((32,) * 3, (L,) * 3, 0)
    res = []
    for be in ('numpy', 'ref'):
        ps = layer.PoissonSolver(nn=3, backend=be)
        ps.set_grid_descriptor(gd)
        ps.initialize()
        phi = gd.zeros()
        n = ps.solve(phi, rho)
        res.append((n, phi, ps.errors))
    assert res[0][0] == res[1][0]
    assert np.array_equal(res[0][1], res[1][1])
    assert res[0][2] == res[1][2]
