"""The oracle of the Poisson solver variants, pinned on the CPU.

* The NumPy restatement of the weighted operator (c/bmgs/wfd.c, wrelax.c)
  against the reference's own WOperator compiled in oracle/_ref: apply and
  weighted Jacobi bit-identical, on zero and periodic grids, nn = 1..3.
* The Helmholtz coefficient table of the product (host-side, like the
  Laplacian's) equals the oracle's restatement of gpaw/helmholtz.py:55-99.
* The oracle's dipole correction (gpaw/dipole_correction.py:123-154)
  cancels the density's dipole moment along the chosen axis.
* The float32 inner schedule written for the mixed-precision configuration
  ('4 levels, 2 pre- and 2 post-smoothing weighted-Jacobi sweeps').
"""
import numpy as np
import pytest

from oracle import layer as ol
from oracle import ref as oref
from oracle import variants as ov
from oracle.geometry import GridDescriptor as OGD


@pytest.mark.skipif(not oref.available(), reason='needs oracle/_ref')
@pytest.mark.parametrize('pbc', [0, 1])
@pytest.mark.parametrize('nn', [1, 2, 3])
def test_numpy_woperator_equals_reference_c(pbc, nn):
    gd = OGD((12, 10, 14), (3.0, 2.5, 3.5), pbc)
    rng = np.random.default_rng(nn + 10 * pbc)
    W = [1.0 + 0.3 * rng.random(tuple(gd.n_c))] + \
        [rng.standard_normal(tuple(gd.n_c)) for _ in range(3)]
    s = -0.25 / np.pi
    ops = {b: [ol.Laplace(gd, s, nn, backend=b)] +
           [ol.Gradient(gd, j, s, nn, backend=b) for j in range(3)]
           for b in ('ref', 'numpy')}
    A = ov.WeightedFDOperator(W, ops['ref'], 'ref')
    B = ov.WeightedFDOperator(W, ops['numpy'], 'numpy')
    a = rng.standard_normal(tuple(gd.n_c))
    o1, o2 = np.empty_like(a), np.empty_like(a)
    A.apply(a, o1)
    B.apply(a, o2)
    assert np.array_equal(o1, o2)
    src = rng.standard_normal(tuple(gd.n_c))
    f1, f2 = a.copy(), a.copy()
    A.relax(2, f1, src, 3, 0.7)
    B.relax(2, f2, src, 3, 0.7)
    assert np.array_equal(f1, f2)
    assert A.get_diagonal_element() == B.get_diagonal_element()


@pytest.mark.parametrize('cell', [(4.0, 4.4, 5.0),
                                  [(0, 2.55, 2.55), (2.55, 0, 2.55),
                                   (2.55, 2.55, 0)]])
def test_helmholtz_table(cell):
    from gpawdft_b200.helmholtz import helmholtz_coefficients
    gd = OGD((16, 16, 16), cell, 1)
    for n in (1, 2, 3):
        c, o = helmholtz_coefficients(gd, -0.25 / np.pi, n, -0.4)
        oc, oo = ov.helmholtz(gd, -0.25 / np.pi, n, -0.4)
        assert np.array_equal(np.array(c), oc)
        assert np.array_equal(np.array(o).reshape(-1, 3), oo)
        # the shift sits on the centre only
        lc, _ = ov.stencils.guc_laplace(gd, -0.25 / np.pi, n)
        assert np.array_equal(np.array(c)[1:], lc[1:])


def test_oracle_dipole_correction_cancels_moment():
    gd = OGD((16, 16, 40), (5.0, 5.0, 12.0), (1, 1, 0))
    z = gd.get_grid_point_coordinates()[2]
    rho = np.exp(-(z - 5.0) ** 2) - np.exp(-(z - 7.0) ** 2)
    drho, dphi, corr = ov.dipole_correction(2, gd, rho)
    assert abs(gd.calculate_dipole_moment(rho)[2]) > 1e-3
    assert abs(gd.calculate_dipole_moment(rho + drho)[2]) < 1e-10
    assert abs(gd.integrate(drho)) < 1e-10
    assert corr != 0.0


def test_jacobi22_schedule():
    from gpawdft_b200.poisson import jacobi22_schedule
    npre, npost, w = jacobi22_schedule(4)
    assert npre == [2, 2, 2, 0] and npost == [2, 2, 2, 8]
    assert len(w) == 2 * 3 * 2 + 8 and all(x == 2.0 / 3.0 for x in w)


# ------------------------------------------------------------ extended
EXT_GOLDEN = [
    # (solver options, max |phi - phi_default|) from the reference's own
    # gpaw/test/poisson/poisson_extended.py (its tolerance: 1e-10)
    (dict(), 0.0),
    (dict(moment_corrections=4), 4.1182101206e-02),
    (dict(moment_corrections=[{'moms': range(4), 'center': [.5, .5, 1]},
                              {'moms': range(4), 'center': [.5, .5, 2]}]),
     2.7569628594e-02),
    (dict(extended={'gpts': (24, 24, 72), 'useprev': False}),
     2.5351851105e-02),
    (dict(extended={'gpts': (24, 24, 72), 'useprev': False},
          moment_corrections=[{'moms': range(4), 'center': [.5, .5, 1]},
                              {'moms': range(4), 'center': [.5, .5, 2]}]),
     2.75205170866e-02)]


def extended_case():
    """The model of gpaw/test/poisson/poisson_extended.py: two dipolar
    Gaussian blobs in a 1 x 1 x 3 Bohr zero-boundary cell, 16 x 16 x 48."""
    gd = OGD((16, 16, 48), (1, 1, 3), False)
    c = gd.get_grid_point_coordinates()
    rho = gd.zeros()
    for z0 in [1, 2]:
        rho += 10 * (c[2] - z0) * np.exp(
            -20 * np.sum((c.T - np.array([.5, .5, z0])).T ** 2, axis=0))
    return gd, rho


@pytest.mark.skipif(not oref.available(), reason='needs oracle/_ref')
def test_oracle_extended_solver_golden_values():
    gd, rho = extended_case()

    def run(ps):
        ps.set_grid_descriptor(gd)
        ps.initialize()
        phi = gd.zeros()
        ps.solve(phi, rho)
        return phi

    ref = run(ol.PoissonSolver(eps=1e-20, backend='ref'))
    for kw, val in EXT_GOLDEN:
        phi = run(ov.ExtendedPoissonSolver(eps=1e-20, backend='ref', **kw))
        assert abs(np.abs(phi - ref).max() - val) < 1e-10, kw


@pytest.mark.parametrize('impl', ['oracle', 'product'])
def test_gaussian_moments(impl):
    """gpaw/test/gauss_func.py: the L-th generalised Gaussian has unit L-th
    moment and no other (L, L' <= 8), the hydrogen 1s density's moments, and
    remove_moment removes the monopole."""
    from math import pi, sqrt
    gd = OGD((48,) * 3, (20,) * 3, 0)
    if impl == 'oracle':
        from oracle.gauss import Gaussian
    else:
        from gpawdft_b200.gauss import Gaussian
    gauss = Gaussian(gd)
    for gL in range(9):
        g = gauss.get_gauss(gL)
        for mL in range(9):
            assert abs(gauss.get_moment(g, mL) - (gL == mL)) < 1e-4
    from oracle.gauss import coordinates
    r = np.sqrt(coordinates(gd)[1])
    nH = np.exp(-2 * r) / pi
    for L in range(4):
        assert abs(gauss.get_moment(nH, L) - (L == 0) / sqrt(4 * pi)) < 1.5e-3
    gauss.remove_moment(nH, 0)
    assert abs(gauss.get_moment(nH, 0)) < 1e-7


def test_gaussian_potentials_oracle_equals_product():
    from gpawdft_b200.gauss import Gaussian as PG
    from oracle.gauss import Gaussian as OG
    gd = OGD((24, 20, 28), (8.0, 7.0, 9.0), 0)
    for center in (None, np.array([3.0, 3.5, 4.0])):
        p, o = PG(gd, center=center), OG(gd, center=center)
        for L in range(9):
            assert np.allclose(p.get_gauss(L), o.get_gauss(L), rtol=1e-13,
                               atol=0)
            assert np.allclose(p.get_gauss_pot(L), o.get_gauss_pot(L),
                               rtol=1e-12, atol=1e-14)
