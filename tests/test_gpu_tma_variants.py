"""Every tile variant of the TMA star-stencil kernel, pinned one at a time
(gpw_set_tma_variant), against the oracle (c/bmgs/fd.c, c/bmgs/relax.c
restated) and against the autotuned choice.

The autotuner keeps whichever variant ran fastest, so without pinning a
variant can go untested.  Every variant computes each point with the same
operations in the same order, so pinned results equal the tuned ones
exactly; the float64 kernels stay within 1e-12 of the oracle and the
float32 ones within 2e-6 (relative, max norm).
"""
import numpy as np
import pytest

from helpers import rand, relerr
from oracle import layer as ol
from oracle.geometry import GridDescriptor as OGD
from gpawdft_b200.workloads import gaussian_density

pytestmark = pytest.mark.gpu

NVARIANT = 11           # 0-4 and 10 both element types, 5-9 float32 only
# wave model, one chunk, twice the model's count, balanced split over the
# resident slots (CTAs whose work spans several tile columns)
CHUNKS = [0, 1, -2, -1]


@pytest.fixture
def pin():
    from gpawdft_b200 import _lib
    lib = _lib.load()

    def set_variant(v, nc=0):
        _lib.check(lib.gpw_set_tma_variant(v, nc))
    yield set_variant
    _lib.check(lib.gpw_set_tma_variant(-1, 0))


def gds(N, cell):
    from gpawdft_b200.grid_descriptor import GridDescriptor
    return GridDescriptor(N, cell, 0), OGD(N, cell, 0)


@pytest.mark.parametrize('var', range(NVARIANT))
@pytest.mark.parametrize('dtype', [np.float64, np.float32])
@pytest.mark.parametrize('nn', [1, 3])
def test_variant_apply_relax_residual(cuda, pin, var, dtype, nn):
    import torch
    from gpawdft_b200.fd_operators import Laplace
    tol = 1e-12 if dtype == np.float64 else 2e-6
    # rows of 36 points: a partial 64-wide tile; 26 rows: partial tiles in y
    gd, ogd = gds((22, 26, 36), (4.4, 5.2, 7.2))
    f = rand((2,) + tuple(gd.n_c), np.float64, 21)
    s = rand((2,) + tuple(gd.n_c), np.float64, 22)
    op = Laplace(gd, -0.25 / np.pi, nn, dtype)
    oop = ol.Laplace(ogd, -0.25 / np.pi, nn)
    ref_apply = np.zeros_like(f)
    oop.apply(f, ref_apply)
    ref_relax = f[0].copy()
    oop.relax(2, ref_relax, s[0], 2, 2.0 / 3.0)
    ref_res = ref_apply - s
    for nc in CHUNKS:
        pin(var, nc)
        out = np.zeros(f.shape, dtype)
        op.apply(f.astype(dtype), out)
        assert relerr(out, ref_apply) < tol, (var, nc)
        g = f[0].astype(dtype)
        op.relax(2, g, s[0].astype(dtype), 2, 2.0 / 3.0)
        assert relerr(g, ref_relax) < tol, (var, nc)
        if dtype == np.float64:
            r = torch.empty(f.shape, dtype=torch.float64, device='cuda')
            ss = op.residual(torch.from_numpy(f).cuda(),
                             torch.from_numpy(s).cuda(), r)
            assert relerr(r.cpu().numpy(), ref_res) < tol
            assert np.allclose(ss.cpu().numpy(),
                               (ref_res.reshape(2, -1) ** 2).sum(1),
                               rtol=1e-12)


@pytest.mark.parametrize('N', [32, 48])
@pytest.mark.parametrize('precision', ['fp64', 'fp32'])
def test_variant_poisson_equals_tuned(cuda, pin, N, precision):
    """Batched Poisson solves on the engine's pitched grids (31^3 / 47^3
    rows: the last thread of a row holds 1-3 of its 4 points) with each
    variant pinned, chunked by the wave model and split over the resident
    slots: the same iteration counts and bit-identical potentials as the
    autotuned solve."""
    from gpawdft_b200.grid_descriptor import GridDescriptor
    from gpawdft_b200.poisson import PoissonSolver
    rhos = []
    for s in range(2):
        rho, L = gaussian_density(N, 0.2, 5 + s, 80 + s)
        rhos.append(rho)
    rhos = np.array(rhos)
    gd = GridDescriptor((N,) * 3, (L,) * 3, 0)
    eps = 1e-20 * max(float(np.dot(r.ravel(), r.ravel())) for r in rhos)

    def solve():
        ps = PoissonSolver(nn=3, batch=2, precision=precision, maxiter=200)
        ps.set_grid_descriptor(gd)
        ps.initialize()
        phi = np.zeros_like(rhos)
        n = ps.solve_batch(phi, rhos, eps=eps)
        return phi, n

    want, want_n = solve()
    for var in range(NVARIANT):
        for nc in (0, -1):
            pin(var, nc)
            phi, n = solve()
            assert np.array_equal(n, want_n), (var, nc)
            assert np.array_equal(phi, want), (var, nc)
