"""The mixed-precision Poisson configuration at full size against the
reference's own C.

N_c = 192 zero boundary (191^3 unknowns), h = 0.15 Angstrom, 64 Gaussians
(log-uniform widths 0.3-2.0 Angstrom, N(0, 1) charges re-centred to neutral,
seed 4), solved to relative residual 1e-10.  tests/golden/mixed192.npz holds
what the compiled reference C (oracle/_ref) gives for it (made by
tests/golden/make_mixed192.py): the Hartree energy, the V-cycle count, the
potential at 4096 seeded points and its per-plane sums.  Three GPU plans are
checked against it: the reference's float64 method, the float32 inner
V-cycles with the tuned Chebyshev schedule inside float64 defect
correction, and the configuration as written -- float32 V-cycles of 4
levels with 2 pre- and 2 post-smoothing weighted-Jacobi sweeps.  Bars:
E_H within 1e-8 Ha; the potential within 1e-6 of its largest magnitude
(both solvers stop at the same residual, not at the same iterate).
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FIX = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'golden',
                   'mixed192.npz')


@pytest.fixture(scope='module')
def case():
    from gpawdft_b200.workloads import gaussian_density
    g = np.load(FIX)
    rho, L = gaussian_density(192, 0.15, 64, 4, sigma_range=(0.3, 2.0),
                              log_sigma=True, charges='normal')
    assert L == float(g['L'])
    assert float(rho.sum()) == float(g['rho_sum'])
    assert float(np.abs(rho).sum()) == float(g['rho_abs_sum'])
    return g, rho, L


PLANS = [('fp64', 'reference', None), ('fp32', 'chebyshev', None),
         ('fp32', 'jacobi22', 4)]


@pytest.mark.parametrize('plan', PLANS,
                         ids=['fp64-reference', 'fp32-chebyshev',
                              'fp32-4-levels-2+2-jacobi'])
def test_mixed192_against_reference_c(cuda, case, plan):
    from gpawdft_b200.grid_descriptor import GridDescriptor
    from gpawdft_b200.poisson import PoissonSolver
    g, rho, L = case
    prec, inner, levels = plan
    gd = GridDescriptor((192,) * 3, (L,) * 3, 0)
    ps = PoissonSolver(nn=3, relax='J', maxiter=1000, precision=prec,
                       inner=inner, max_levels=levels)
    ps.set_grid_descriptor(gd)
    ps.initialize()
    if levels is not None:
        assert ps.levels + 1 == levels
    eps = float(g['eps'])
    phi = gd.zeros()
    n = ps.solve(phi, rho, eps=eps)
    assert ps.last_errors[0] <= eps
    eh = 0.5 * gd.dv * float(np.dot(phi.ravel(), rho.ravel()))
    scale = float(g['phi_absmax'])
    err_pts = np.abs(phi.ravel()[g['idx']] - g['phi_samples']).max() / scale
    err_planes = np.abs(phi.sum(axis=(1, 2)) - g['phi_plane_sums']).max() / (
        scale * phi.shape[1] * phi.shape[2])
    print('%s/%s levels=%s: %d outer iterations (reference C %d), '
          'E_H error %.2e Ha, potential error %.2e (points) %.2e (planes)'
          % (prec, inner, levels, n, int(g['niter']), abs(eh - float(g['eh'])),
             err_pts, err_planes))
    assert abs(eh - float(g['eh'])) < 1e-8
    assert err_pts < 1e-6
    assert err_planes < 1e-6
    if prec == 'fp64':
        assert n == int(g['niter'])
