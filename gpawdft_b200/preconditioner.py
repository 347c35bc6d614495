"""Eigensolver preconditioner on the GPU (drop-in for gpaw.preconditioner).

``Preconditioner(gd0, kin0, dtype=float, block=1)(residuals, kpt, ekin=None)``
runs the fixed three-grid smoothing sequence of gpaw/preconditioner.py:34-60
on a block of residuals: restrictions / interpolations (nn=1 Transformers
with the k-point's Bloch phases), the caller's kinetic operator on the fine
grid and nn=1 Laplacians (scale -1/2) on the two coarse grids, with the
array arithmetic as device axpy / scal kernels.  Returns a device view of
internal scratch (as the reference returns a view of its scratch arrays) --
or a NumPy array when the residuals were NumPy.
"""
import numpy as np

from . import arrays, blas
from .fd_operators import Laplace
from .transformers import Transformer


class Preconditioner:
    def __init__(self, gd0, kin0, dtype=float, block=1):
        gd1 = gd0.coarsen()
        gd2 = gd1.coarsen()
        self.gd0, self.gd1, self.gd2 = gd0, gd1, gd2
        self.kin0 = kin0
        self.kin1 = Laplace(gd1, -0.5, 1, dtype)
        self.kin2 = Laplace(gd2, -0.5, 1, dtype)
        self.dtype = dtype
        self.block = block
        self.scratch0 = gd0.zeros_device((2, block), dtype)
        self.scratch1 = gd1.zeros_device((3, block), dtype)
        self.scratch2 = gd2.zeros_device((3, block), dtype)
        self.step = 0.66666666 / kin0.get_diagonal_element()
        self.restrictor_object0 = Transformer(gd0, gd1, 1, dtype)
        self.restrictor_object1 = Transformer(gd1, gd2, 1, dtype)
        self.interpolator_object2 = Transformer(gd2, gd1, 1, dtype)
        self.interpolator_object1 = Transformer(gd1, gd0, 1, dtype)
        self.restrictor0 = self.restrictor_object0.apply
        self.restrictor1 = self.restrictor_object1.apply
        self.interpolator2 = self.interpolator_object2.apply
        self.interpolator1 = self.interpolator_object1.apply

    def calculate_kinetic_energy(self, psit_xG, kpt):
        return None

    def __call__(self, residuals, kpt, ekin=None):
        phases = getattr(kpt, 'phase_cd', kpt)
        host = not arrays.is_device(residuals)
        res = arrays.to_device(residuals)
        single = res.dim() == 3
        if single:
            res = res.unsqueeze(0)
        nb = res.shape[0]
        if nb > self.block:
            raise ValueError('more residuals than the preconditioner block')
        step = self.step
        d0, q0 = self.scratch0[:, :nb]
        r1, d1, q1 = self.scratch1[:, :nb]
        r2, d2, q2 = self.scratch2[:, :nb]
        # r1 = R0(-residuals): restriction is linear and exact under negation
        self.restrictor0(res, r1, phases)
        blas.scal(-1.0, r1)
        d1.copy_(r1)
        blas.scal(4 * step, d1)                      # d1 = 4 step r1
        self.kin1.apply(d1, q1, phases)
        blas.axpy(-1.0, r1, q1)                      # q1 -= r1
        self.restrictor1(q1, r2, phases)
        d2.copy_(r2)
        blas.scal(16 * step, d2)                     # d2 = 16 step r2
        self.kin2.apply(d2, q2, phases)
        blas.axpy(-1.0, r2, q2)                      # q2 -= r2
        blas.axpy(-16 * step, q2, d2)                # d2 -= 16 step q2
        self.interpolator2(d2, q1, phases)
        blas.axpy(-1.0, q1, d1)                      # d1 -= q1
        self.kin1.apply(d1, q1, phases)
        blas.axpy(-1.0, r1, q1)                      # q1 -= r1
        blas.axpy(-4 * step, q1, d1)                 # d1 -= 4 step q1
        self.interpolator1(d1, d0, phases)
        blas.scal(-1.0, d0)                          # d0 = I1(-d1)
        self.kin0.apply(d0, q0, phases)
        blas.axpy(-1.0, res, q0)                     # q0 -= residuals
        blas.axpy(-step, q0, d0)                     # d0 -= step q0
        blas.scal(-1.0, d0)                          # d0 *= -1
        out = d0[0] if single else d0
        if host:
            return out.cpu().numpy()
        return out
