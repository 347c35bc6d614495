"""Device-resident grid steps of the SCF loop around the Poisson solve.

One SCF iteration of GPAW's real-space mode moves the density from the
coarse to the fine grid, solves for the Hartree potential there, and moves
the effective potential back.  Restated here for the grids only:

  gpaw/density.py:632-648    RealSpaceDensity.interpolate: nt_sG (coarse)
                             -> nt_sg (fine), Transformer(gd, finegd, stencil)
  gpaw/hamiltonian.py:611-619  vHt_g = solve(rhot_g, charge=-charge), warm-
                             started from the previous step's vHt_g;
                             e_coulomb = 1/2 integrate(vHt_g, rhot_g);
                             vt_sg += vHt_g
  gpaw/hamiltonian.py:552-567  restrict_and_collect: vt_sg -> vt_sG,
                             Transformer(finegd, gd, stencil)

``HartreeGridStep`` keeps the fine-grid arrays (nt_sg, rhot_g, vHt_g) on the
device across SCF steps, so a step moves no grid between host and device
when its inputs are device tensors.  The parts of those reference functions
that are not grid work -- compensation charges and the pseudo-core density
(LFC), XC, vbar, external potentials -- stay with the caller: their
contributions enter as ``rhot_extra_g`` (added to the interpolated density)
and as the fine-grid ``vt_sg`` that the Hartree potential is added to.
"""
import numpy as np

from . import arrays, blas
from .poisson import PoissonSolver
from .transformers import Transformer


class HartreeGridStep:
    def __init__(self, gd, finegd, poisson=None, stencil=3, nspins=1):
        self.gd = gd
        self.finegd = finegd
        self.nspins = int(nspins)
        self.interpolator = Transformer(gd, finegd, stencil)
        self.restrictor = Transformer(finegd, gd, stencil)
        if poisson is None:
            poisson = PoissonSolver(nn=3)
        self.poisson = poisson
        self.poisson.set_grid_descriptor(finegd)
        self.poisson.initialize()
        self.nt_sg = finegd.zeros_device(self.nspins)
        self.rhot_g = finegd.zeros_device()
        self.vHt_g = finegd.zeros_device()   # the warm start of every solve
        self.npoisson = None

    def interpolate(self, in_xR, out_xR=None):
        """gpaw/density.py:632-648: every leading grid coarse -> fine (one
        batched launch where the reference loops over them)."""
        return self.interpolator.apply(in_xR, out_xR)

    def restrict(self, a_xg, b_xg=None):
        """gpaw/hamiltonian.py:560-567 (no redistribution: one domain)."""
        return self.restrictor.apply(a_xg, b_xg)

    def step(self, nt_sG, vt_sg, charge=0.0, rhot_extra_g=None):
        """One SCF step's grid work.

        nt_sG: (nspins, *gd.n_c) pseudo density on the coarse grid.
        vt_sg: (nspins, *finegd.n_c) fine-grid effective potential without
               the Hartree term; vHt_g is added to it in place.
        Returns (e_coulomb, vt_sG, npoisson) with vt_sG the restricted
        potential -- device tensors, or NumPy arrays when vt_sg is NumPy (it
        is then written back as well).
        """
        if tuple(nt_sG.shape[:1]) != (self.nspins,):
            raise ValueError('nt_sG must have one grid per spin')
        self.interpolate(arrays.to_device(nt_sG), self.nt_sg)
        self.rhot_g.copy_(self.nt_sg[0])
        for s in range(1, self.nspins):
            blas.axpy(1.0, self.nt_sg[s], self.rhot_g)
        if rhot_extra_g is not None:
            blas.axpy(1.0, arrays.to_device(rhot_extra_g), self.rhot_g)
        self.npoisson = self.poisson.solve(self.vHt_g, self.rhot_g,
                                           charge=-charge)
        e_coulomb = 0.5 * self.finegd.integrate(self.vHt_g, self.rhot_g)
        vt_d = arrays.to_device(vt_sg)
        for s in range(self.nspins):
            blas.axpy(1.0, self.vHt_g, vt_d[s])
        vt_sG = self.restrict(vt_d)
        if not arrays.is_device(vt_sg):
            arrays.writeback(vt_sg, vt_d)
            vt_sG = vt_sG.cpu().numpy()
        return e_coulomb, vt_sG, self.npoisson

    def hartree_potential(self):
        """The fine-grid Hartree potential of the last step (device)."""
        return self.vHt_g

    def estimate_memory(self):
        return int(np.prod(self.finegd.n_c)) * 8 * (self.nspins + 2)
