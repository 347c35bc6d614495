// TMA star-stencil launches for float64 grids (apply, residual, Jacobi and
// the float64 defect of the float32 defect-correction form).
#include "gpw_mehr_tma.cuh"
#include "gpw_tma_launch.cuh"

namespace gpw {

cudaError_t tma_stencil_f64(int mode, int R, int var, const StencilArgs& a, int nbatch, const StarCoefs& sc,
                            int nchunk, cudaStream_t st) {
  switch (mode) {
    case MODE_APPLY: return tma_run_radius<double, MODE_APPLY>(R, var, a, nbatch, sc, nchunk, st);
    case MODE_APPLY_EPI: return tma_run_radius<double, MODE_APPLY_EPI>(R, var, a, nbatch, sc, nchunk, st);
    case MODE_RESIDUAL: return tma_run_radius<double, MODE_RESIDUAL>(R, var, a, nbatch, sc, nchunk, st);
    case MODE_JACOBI: return tma_run_radius<double, MODE_JACOBI>(R, var, a, nbatch, sc, nchunk, st);
    case MODE_RESID_DC: return tma_run_radius<double, MODE_RESID_DC>(R, var, a, nbatch, sc, nchunk, st);
  }
  return cudaErrorInvalidValue;
}

cudaError_t mehr_tma_f64(int mode, const StencilArgs& a, int nbatch, const GeneralCoefs& gc, cudaStream_t st) {
  return mehr_tma_mode<double>(mode, a, nbatch, gc, st);
}

}  // namespace gpw
