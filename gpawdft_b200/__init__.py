"""gpawdft_b200 -- GPAW's real-space grid hot path on NVIDIA B200 (sm_100a).

Drop-in replacements for the reference's grid numerics API:

  gpawdft_b200.grid_descriptor.GridDescriptor   (gpaw.grid_descriptor, serial)
  gpawdft_b200.fd_operators.{FDOperator, Laplace, GUCLaplace, Gradient,
                              LaplaceA, LaplaceB}  (gpaw.fd_operators)
  gpawdft_b200.transformers.Transformer          (gpaw.transformers)
  gpawdft_b200.poisson.{PoissonSolver, FDPoissonSolver,
                        PoissonConvergenceError}  (gpaw.poisson)
  gpawdft_b200.preconditioner.Preconditioner     (gpaw.preconditioner)

All arithmetic runs in the in-tree CUDA library ``libgpwgrid.so`` (C ABI in
include/gpwgrid.h); importing an API class on a machine without that
library or without a CUDA device fails loudly.
"""
__version__ = '0.1.0'


def library_path():
    from ._lib import LIB_PATH
    return LIB_PATH
