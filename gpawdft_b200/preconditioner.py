"""Eigensolver preconditioner on the GPU (drop-in for gpaw.preconditioner).

``Preconditioner(gd0, kin0, dtype=float, block=1)(residuals, kpt, ekin=None)``
runs the fixed three-grid smoothing sequence of gpaw/preconditioner.py:34-60
on a block of residuals: restrictions / interpolations (nn=1 Transformers
with the k-point's Bloch phases), the caller's kinetic operator on the fine
grid and nn=1 Laplacians (scale -1/2) on the two coarse grids, with the
array arithmetic folded into those launches (see ``__call__``).  Returns a device view of
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

    def _fused_operators(self):
        """The scaled operators that fold the sequence's array arithmetic
        into the applies (built once, on the host)."""
        if getattr(self, '_ops', None) is None:
            step = self.step
            self._ops = (self.kin1.scaled(-4 * step, 1.0),       # q1 from s1
                         self.kin2.scaled(-256 * step * step, 32 * step),
                         self.kin1.scaled(4 * step, -1.0),       # -d1''
                         self.kin0.scaled(step, -1.0))           # the result
        return self._ops

    def __call__(self, residuals, kpt, ekin=None):
        """gpaw/preconditioner.py:34-60 in eight fused launches.

        With s1 = R0(residuals) (so the reference's r1 = R0(-residuals) is
        -s1) the reference's sequence is, exactly in real arithmetic,
          q1  = (I - 4 step A1) s1                      (d1 = -4 step s1)
          r2  = R1(q1)
          d2  = (32 step I - 256 step^2 A2) r2          (its d2 after the update)
          d1  = -4 step s1 - I2(d2)
          -d1 = (4 step A1 - I) d1 + 4 step s1          (its d1 after the update)
          d0  = I1(-d1)
          out = (step A0 - I) d0 - step residuals       (its -(d0 - step q0))
        Every line is one launch: a transfer, or an apply of an operator whose
        coefficients were scaled on the host, its additive term folded into
        the apply's output stage (gpw_operator_apply_fused) or the
        interpolation's (gpw_transformer_apply_subtract).  Rounding differs
        from the reference's step-by-step NumPy arithmetic only in the last
        bits.
        """
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
        op1a, op2, op1b, op0 = self._fused_operators()
        out, d0 = self.scratch0[:, :nb]
        s1, t1, u1 = self.scratch1[:, :nb]
        r2, d2, _ = self.scratch2[:, :nb]
        self.restrictor0(res, s1, phases)                   # s1 = R0(res)
        op1a.apply(s1, u1, phases)                           # q1
        self.restrictor1(u1, r2, phases)                     # r2
        op2.apply(r2, d2, phases)                            # d2
        t1.copy_(s1)
        blas.scal(-4 * step, t1)                             # d1 = -4 step s1
        self.interpolator_object2.apply_subtract(d2, t1, u1, phases)
        op1b.apply_fused(u1, t1, phases, aux=s1, aux_scale=4 * step)
        self.interpolator1(t1, d0, phases)                   # d0 = I1(-d1)
        op0.apply_fused(d0, out, phases, aux=res, aux_scale=-step)
        result = out[0] if single else out
        if host:
            return result.cpu().numpy()
        return result
