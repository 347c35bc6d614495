// TMA star-stencil launches for float32 grids (apply, residual, Jacobi, the
// Jacobi sweep that adds its result into float64 phi, and the residual
// restricted into the next level).
#include "gpw_mehr_tma.cuh"
#include "gpw_tma_launch.cuh"

namespace gpw {

cudaError_t tma_stencil_f32(int mode, int R, int var, const StencilArgs& a, int nbatch, const StarCoefs& sc,
                            int nchunk, cudaStream_t st) {
  switch (mode) {
    case MODE_APPLY: return tma_run_radius<float, MODE_APPLY>(R, var, a, nbatch, sc, nchunk, st);
    case MODE_APPLY_EPI: return tma_run_radius<float, MODE_APPLY_EPI>(R, var, a, nbatch, sc, nchunk, st);
    case MODE_RESIDUAL: return tma_run_radius<float, MODE_RESIDUAL>(R, var, a, nbatch, sc, nchunk, st);
    case MODE_JACOBI: return tma_run_radius<float, MODE_JACOBI>(R, var, a, nbatch, sc, nchunk, st);
    case MODE_JACOBI_ADD64: return tma_run_radius<float, MODE_JACOBI_ADD64>(R, var, a, nbatch, sc, nchunk, st);
    case MODE_JACOBI_SCALED_IN:
      return tma_run_radius<float, MODE_JACOBI_SCALED_IN>(R, var, a, nbatch, sc, nchunk, st);
    case MODE_RESID_RESTRICT:  // the float32 form's level 0 (nn = 3) and coarse levels (nn = 1)
      if (R == 3) return tma_run_variant<float, 3, MODE_RESID_RESTRICT>(var, a, nbatch, sc, nchunk, st);
      if (R == 1) return tma_run_variant<float, 1, MODE_RESID_RESTRICT>(var, a, nbatch, sc, nchunk, st);
      return cudaErrorInvalidValue;
  }
  return cudaErrorInvalidValue;
}

cudaError_t mehr_tma_f32(int mode, const StencilArgs& a, int nbatch, const GeneralCoefs& gc, cudaStream_t st) {
  return mehr_tma_mode<float>(mode, a, nbatch, gc, st);
}

}  // namespace gpw
