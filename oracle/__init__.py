"""Oracle for GPAW's real-space grid hot path.

TEST INFRASTRUCTURE ONLY.  Nothing in the product package imports this; only
``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline / reference legs of
``bench.py`` use it, and only as the checker or as the timed CPU baseline.

Two interchangeable CPU backends stand behind the same restated Python layer:

* ``oracle.kernels`` -- a NumPy restatement of the reference C kernels
  (c/bmgs/fd.c, relax.c, restrict.c, interpolate.c and the halo fill of
  c/bc.c), written so that every floating-point operation happens in the same
  order as in the C code (no FMA contraction), i.e. bit-identical results.
* ``oracle.ref`` -- the reference's own C implementation (c/bmgs/bmgs.c,
  c/bc.c, c/operators.c, c/transformers.c) compiled in place by
  ``oracle/Makefile`` into ``oracle/_ref/`` with a project-written module
  init.  It pins the NumPy restatement (tests/test_oracle_pins.py).

The restated Python layer follows gpaw/grid_descriptor.py, gpaw/domain.py,
gpaw/fd_operators.py, gpaw/transformers.py, gpaw/poisson.py,
gpaw/preconditioner.py and gpaw/utilities/gauss.py; every function cites the
file:line it restates.  The reference's Python package itself cannot be
imported here (it needs the full _gpaw extension with BLAS/LAPACK/libxc and
ASE, and uses NumPy APIs removed in NumPy 2), hence the restatement.
"""
