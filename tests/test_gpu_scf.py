"""GPU parity of the SCF loop's grid steps around the Poisson solve.

``HartreeGridStep.step`` interpolates the spin densities to the fine grid
with the nn=3 (K=6) transformer (gpaw/density.py:632-648), solves the
Poisson equation there warm-started from the previous step's potential
(gpaw/hamiltonian.py:611-619), integrates the Hartree energy, adds the
Hartree potential to the fine-grid effective potential and restricts that
back to the coarse grid (gpaw/hamiltonian.py:552-567).  The oracle runs the
same sequence with the restated layer over the compiled reference C, for
two consecutive SCF steps.  Bars: the interpolated density bit-identical
(the transformers keep the reference's expression order); E_H within 1e-8
Ha; the potentials within 1e-7 of their largest magnitude (both solves stop
at the same residual, not at the same iterate).
"""
import numpy as np
import pytest

from oracle import layer as ol
from oracle import ref as oref
from oracle.geometry import GridDescriptor as OGD

pytestmark = pytest.mark.gpu

BACKEND = 'ref' if oref.available() else 'numpy'


def _gauss(gd, centres, widths, charges):
    """Normalised Gaussians; centres in grid-index units of ``gd``."""
    r = np.indices(tuple(gd.n_c)).astype(float)
    r = np.moveaxis(r, 0, -1) + gd.beg_c
    h = gd.cell_cv.diagonal() / gd.N_c
    out = np.zeros(tuple(gd.n_c))
    for c, w, q in zip(centres, widths, charges):
        d2 = (((r - np.asarray(c)) * h) ** 2).sum(-1)
        out += q * (2 * np.pi * w * w) ** -1.5 * np.exp(-d2 / (2 * w * w))
    return out


@pytest.mark.parametrize('nspins', [1, 2])
def test_two_scf_steps_against_oracle(cuda, nspins):
    from gpawdft_b200.grid_descriptor import GridDescriptor
    from gpawdft_b200.scf import HartreeGridStep
    N, a = 32, 10.0
    gd = GridDescriptor((N,) * 3, (a,) * 3, 0)
    fgd = GridDescriptor((2 * N,) * 3, (a,) * 3, 0)
    ogd = OGD((N,) * 3, (a,) * 3, 0)
    ofgd = OGD((2 * N,) * 3, (a,) * 3, 0)
    rng = np.random.default_rng(21)
    # spin densities on the coarse grid (positive Gaussians) and, on the
    # fine grid, the compensation-like negative charge that neutralises them
    nt_sG = np.array([_gauss(ogd, rng.uniform(10, 22, (3, 3)),
                             rng.uniform(0.8, 1.4, 3), [1.0, 0.7, 0.5])
                      for _ in range(nspins)])
    extra_g = -_gauss(ofgd, rng.uniform(20, 44, (2, 3)), [1.0, 1.2],
                      [1.0, 1.2]) * nspins
    vt0_sg = 0.1 * np.array([_gauss(ofgd, [(32.0, 32.0, 32.0)], [2.0], [1.0])
                             for _ in range(nspins)])

    step = HartreeGridStep(gd, fgd, stencil=3, nspins=nspins)
    interp = ol.Transformer(ogd, ofgd, 3, float, BACKEND)
    restr = ol.Transformer(ofgd, ogd, 3, float, BACKEND)
    ops = ol.PoissonSolver(nn=3, backend=BACKEND)
    ops.set_grid_descriptor(ofgd)
    ops.initialize()
    ovHt = ofgd.zeros()
    first = None
    for it in range(2):
        if it == 1:   # the next SCF step: the density moves a little
            nt_sG = nt_sG * 1.01 + 1e-3 * np.roll(nt_sG, 1, axis=-1)
            extra_g = extra_g * 1.01 + 1e-3 * np.roll(extra_g, 2, axis=-1)
        vt_sg = vt0_sg.copy()
        e, vt_sG, n = step.step(nt_sG, vt_sg, charge=0.0,
                                rhot_extra_g=extra_g)
        # the oracle's sequence
        ont = interp.apply(nt_sG)
        assert np.array_equal(step.nt_sg.cpu().numpy(), ont)
        orhot = ont.sum(axis=0) + extra_g
        on = ops.solve(ovHt, orhot, charge=0.0)
        oe = 0.5 * ofgd.integrate(ovHt, orhot)
        ovt = vt0_sg + ovHt
        ovt_sG = restr.apply(ovt)
        assert abs(n - on) <= 1
        assert abs(e - oe) < 1e-8
        assert np.abs(vt_sG - ovt_sG).max() < 1e-7 * np.abs(ovt_sG).max()
        assert np.abs(vt_sg - ovt).max() < 1e-7 * np.abs(ovt).max()
        if it == 1:
            # the warm start pays: fewer V-cycles than the first solve
            assert n < first
        first = n
