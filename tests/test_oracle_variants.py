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
