"""The GPU product replays the golden fixtures of the reference C.

Each case of tests/golden/golden.npz (made from the reference's compiled C by
tests/golden/make_golden.py) runs through the product's drop-in API.
Transformers, Gauss-Seidel and general-offset stencils are expected to be
bit-identical; fused-multiply-add star stencils within 1e-12 relative;
the Poisson solve to the same V-cycle count and a potential within 1e-10
relative (both stop at the same tight tolerance).
"""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, 'golden'))

from make_golden import cases  # noqa: E402

pytestmark = pytest.mark.gpu
GOLD = np.load(os.path.join(HERE, 'golden', 'golden.npz'))
CASES = cases()


def g(name, key):
    return GOLD['%s/%s' % (name, key)]


def relerr(a, b):
    d = np.abs(b).max()
    return np.abs(a - b).max() / (d if d else 1.0)


@pytest.mark.parametrize('name,kind,p', CASES, ids=[c[0] for c in CASES])
def test_product_matches_reference_c(cuda, name, kind, p):
    from gpawdft_b200 import fd_operators as fd
    from gpawdft_b200.grid_descriptor import GridDescriptor
    from gpawdft_b200.poisson import PoissonSolver
    from gpawdft_b200.transformers import Transformer
    dtype = complex if p.get('dtype') == 'complex' else float
    if kind == 'poisson':
        gd = GridDescriptor((p['N'],) * 3, (p['L'],) * 3, 0)
    else:
        gd = GridDescriptor(p['N'], p['cell'], p['pbc'])
    ref = g(name, 'out')
    ph = g(name, 'phase') if dtype == complex else None
    if kind in ('laplace', 'gradient', 'guc'):
        a = g(name, 'a')
        if kind == 'gradient':
            op = fd.Gradient(gd, p['v'], 1.0, p['nn'], dtype)
        elif kind == 'guc':
            op = fd.Laplace(gd, 1.0, p['nn'], dtype)
        else:
            op = fd.Laplace(gd, p['scale'], p['nn'], dtype)
        out = np.zeros_like(a)
        op.apply(a, out, ph)
        if op.cfd:
            assert relerr(out, ref) < 1e-12
        else:
            assert np.array_equal(out, ref)
    elif kind in ('restrict', 'interpolate'):
        gdc = gd.coarsen()
        gi, go = (gd, gdc) if kind == 'restrict' else (gdc, gd)
        out = Transformer(gi, go, p['nn'], dtype).apply(g(name, 'a'), None, ph)
        assert np.array_equal(out, ref)
    elif kind in ('jacobi', 'gs'):
        f = g(name, 'f').copy()
        op = fd.Laplace(gd, -0.25 / np.pi, p['nn'])
        op.relax(2 if kind == 'jacobi' else 1, f, g(name, 's'), p['nrelax'],
                 p.get('w', 1.0))
        if kind == 'gs':
            assert np.array_equal(f, ref)
        else:
            assert relerr(f, ref) < 1e-12
    else:
        ps = PoissonSolver(nn=p['nn'], eps=1e-18)
        ps.set_grid_descriptor(gd)
        ps.initialize()
        phi = gd.zeros()
        n = ps.solve(phi, g(name, 'rho'))
        assert n == int(g(name, 'niter'))
        assert relerr(phi, ref) < 1e-10
