// Host-side internal interfaces shared by the C ABI (gpw_api.cu), the kernel
// launchers (gpw_launch.cu) and the multigrid engine (gpw_poisson.cu).
#pragma once
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "gpw_common.cuh"
#include "gpw_reduce.cuh"
#include "gpw_stencil.cuh"

namespace gpw {

// Thread-local error message behind gpw_last_error().
void set_error(const std::string& msg);
int fail(int code, const std::string& msg);
int cuda_fail(cudaError_t e, const char* what);

inline size_t elt_size(int dtype) {
  switch (dtype) {
    case GPW_F64: return 8;
    case GPW_C128: return 16;
    case GPW_F32: return 4;
    case GPW_C64: return 8;
  }
  return 0;
}
inline bool is_complex(int dtype) { return dtype == GPW_C128 || dtype == GPW_C64; }
inline bool valid_dtype(int dtype) { return dtype >= 0 && dtype <= 3; }

inline GridView contiguous_view(const int n[3]) {
  GridView v;
  v.n[0] = n[0];
  v.n[1] = n[1];
  v.n[2] = n[2];
  v.s1 = n[2];
  v.s0 = (int64_t)n[1] * n[2];
  v.sb = (int64_t)n[0] * n[1] * n[2];
  return v;
}
inline int64_t view_points(const GridView& v) { return (int64_t)v.n[0] * v.n[1] * v.n[2]; }

// Engine-owned grids: rows padded to a multiple of 8 elements (64 bytes for
// float64), so every row, plane and batch member starts 16-byte aligned as
// the TMA tile loads and the 2-point vector stores require.
inline GridView pitched_view(const int n[3]) {
  GridView v;
  v.n[0] = n[0];
  v.n[1] = n[1];
  v.n[2] = n[2];
  v.s1 = ((int64_t)n[2] + 7) / 8 * 8;
  v.s0 = (int64_t)n[1] * v.s1;
  v.sb = (int64_t)n[0] * v.s0;
  return v;
}

// ---------------------------------------------------------------- operator
struct OpDesc {
  int n[3];
  int mp;
  int periodic[3];
  int real, cfd;
  int ncoef;
  std::vector<double> coefs;
  std::vector<int> off;  // ncoef * 3
  bool star;             // star kernel eligible for APPLY / RESIDUAL
  bool star_jacobi;      // star kernel eligible for JACOBI (centre first, unique)
  int R;                 // star radius
  StarCoefs sc;
  GeneralCoefs gc;
  double diag;           // get_diagonal_element
};

int build_opdesc(OpDesc& d, const double* coefs, const int64_t* offsets, int ncoef, const int64_t size[3],
                 int range, const int64_t neighbors[6], int real, int cfd);

// Fill the boundary description for an op / transformer input grid.
Boundary make_boundary(const int periodic[3], int dtype, const double* phases);

// Number of CTAs per batch member the stencil launch will use (for sizing the
// residual partial buffer) and the launch itself.
int stencil_blocks_per_member(const OpDesc& d, int mode, const GridView& vout, int nbatch);
cudaError_t launch_stencil(const OpDesc& d, int dtype, int mode, const void* in, const GridView& vin, void* out,
                           const GridView& vout, const void* rho, const GridView& vrho, int nbatch,
                           const Boundary& bc, double w, const unsigned char* active, const GridSum& gs,
                           cudaStream_t st, const void* pot = nullptr, const void* aux = nullptr,
                           double aux_scale = 0.0);

// Fused defect-correction steps (TMA kernel; zero boundaries, 16-byte-pitched
// engine buffers).  mode MODE_RESID_DC: in/rho float64, out (rhs) and out2
// (first inner iterate) float32.  mode MODE_JACOBI_ADD64: in/rho float32,
// out2 = float64 phi that receives the sweep's result.  Returns
// cudaErrorNotSupported when the TMA path does not apply.
bool dc_fusable(const OpDesc& d);
cudaError_t launch_stencil_dc(const OpDesc& d, int mode, const void* in, const GridView& v, void* out, void* out2,
                              const void* rho, int nbatch, double w, double w2, const unsigned char* active,
                              const GridSum& gs, cudaStream_t st);

// ---------------------------------------------------------------- transformer
struct TrDesc {
  int nin[3], nout[3];
  int k;
  int pad[3][2], npad[3][2], skip[3][2];
  int periodic[3];
  int real, interpolate;
};

// subtract != 0 (interpolation only): out = base - I(in); base may alias out.
// sweep (K=2 real restriction only, see restrict_sweep_ok): also write the
// first weighted-Jacobi sweep of the coarse level from phi = 0,
// sweep->phi = (w / c0) out.
struct RestrictSweep {
  void* phi;
  double w, c0;
};
bool restrict_sweep_ok(const TrDesc& d, int dtype);
cudaError_t launch_transfer(const TrDesc& d, int dtype, const void* in, const GridView& vin, void* out,
                            const GridView& vout, int nbatch, const Boundary& bc, int subtract,
                            const void* base, const GridView* vbase, const unsigned char* active,
                            cudaStream_t st, const RestrictSweep* sweep = nullptr);

// ---------------------------------------------------------------- TMA stencils
// The TMA star-stencil path (gpw_star_tma.cuh): real zero-boundary star
// stencils on 16-byte aligned, 16-byte pitched grids.  Launches pick a tile
// variant and an axis-0 chunk count from the autotuner's cache (defaults
// when the shape was never tuned).
struct TmaChoice {
  int var;     // tile variant (gpw_star_tma.cuh)
  int nchunk;  // axis-0 chunks; <= 0: wave model
};
cudaError_t tma_stencil_f64(int mode, int R, int var, const StencilArgs& a, int nbatch, const StarCoefs& sc,
                            int nchunk, cudaStream_t st);
cudaError_t tma_stencil_f32(int mode, int R, int var, const StencilArgs& a, int nbatch, const StarCoefs& sc,
                            int nchunk, cudaStream_t st);
// Time the candidate (variant, chunking) choices of one stencil launch on
// the given buffers (their contents are overwritten) and keep the fastest
// for every later launch of the same shape.  Not allowed during capture.
// mode MODE_RESID_DC / MODE_JACOBI_ADD64 take the launch_stencil_dc arguments.
cudaError_t tune_stencil(const OpDesc& d, int dtype, int mode, const void* in, const GridView& vin, void* out,
                         const GridView& vout, const void* rho, const GridView& vrho, void* out2, int nbatch,
                         double w, const GridSum& gs, cudaStream_t st);
// Number of stencil choices tuned so far (the cache size).
int tuned_stencil_count();

PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder();

// Dynamic shared memory above 48 KB needs a one-time opt-in per kernel.
template <typename F>
inline cudaError_t smem_optin_bytes(F* kernel, size_t bytes) {
  if (bytes <= 48 * 1024) return cudaSuccess;
  return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

// ---------------------------------------------------------------- coarse levels
// The coarse end of a V-cycle in one CTA per batch member (gpw_coarse.cuh);
// smem = the levels' buffer bytes.
struct CoarseArgs;
cudaError_t launch_coarse(int dtype, const CoarseArgs& a, size_t smem, int nbatch, cudaStream_t st);
// The level above the coarse kernel's first level in a cluster of CTAs per
// solve, then the coarse kernel's levels (float32 only; gpw_coarse.cuh).
struct ClusterArgs;
cudaError_t launch_cluster_vcycle(const ClusterArgs& a, size_t smem, int nbatch, cudaStream_t st);

// ---------------------------------------------------------------- blas
cudaError_t launch_axpy(int dtype, int64_t n, double ar, double ai, const void* x, void* y, cudaStream_t st);
cudaError_t launch_scal(int dtype, int64_t n, double ar, double ai, void* x, cudaStream_t st);
cudaError_t launch_reduce(int dtype, int op, int64_t nvec, int64_t n, const void* x, const void* y,
                          const GridSum& gs, int nblk, cudaStream_t st, int ny = 1);
int reduce_blocks(int64_t n);
cudaError_t launch_charge_prepare(int64_t nb, int64_t n, const double* rho, double* rho_out, double* phi,
                                  const double* rho_g, const double* phi_g, const double* sums, double dv,
                                  double npts, double maxcharge, int all_periodic, int any_periodic, int zero_phi,
                                  double* q_out, cudaStream_t st);
cudaError_t launch_charge_finish(int64_t nb, int64_t n, double* phi, const double* phi_g, const double* q,
                                 cudaStream_t st);
cudaError_t launch_copy_box(int dtype, const void* src, const int sn[3], const int so[3], void* dst,
                            const int dn[3], const int dof[3], const int box[3], cudaStream_t st);
cudaError_t launch_mul(int64_t n, const double* x, const double* y, double* out, cudaStream_t st);
cudaError_t launch_add_scalar(int dtype, int64_t n, double c, const void* x, void* y, cudaStream_t st);
cudaError_t launch_zero(int dtype, const GridView& v, void* x, int nbatch, const unsigned char* active,
                        cudaStream_t st);

// Device workspace that grows on demand (stream-ordered frees are avoided:
// growth synchronises the device first).
struct Workspace {
  void* ptr = nullptr;
  size_t bytes = 0;
  int ensure(size_t need);
  Workspace() = default;
  Workspace(const Workspace&) = delete;
  Workspace& operator=(const Workspace&) = delete;
  Workspace(Workspace&& o) noexcept : ptr(o.ptr), bytes(o.bytes) {
    o.ptr = nullptr;
    o.bytes = 0;
  }
  ~Workspace();
};

// Per-reduction scratch: partials + counters + results.
struct SumScratch {
  Workspace partial, counter, result;
  int ensure(int64_t nseg, int64_t nblk_seg);
  GridSum gs() const {
    GridSum g;
    g.partial = (double*)partial.ptr;
    g.counter = (unsigned*)counter.ptr;
    g.result = (double*)result.ptr;
    return g;
  }
};

int num_sms();

// Programmatic dependent launch of the V-cycle's kernels (gpw_set_pdl; on by
// default): the kernel is launched with programmatic stream serialization
// and must call pdl_wait() before touching global memory.
bool pdl_enabled();
template <typename... KArgs, typename... Args>
inline cudaError_t launch_pdl(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                              Args&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = pdl_enabled() ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, kern, static_cast<KArgs>(args)...);
}

// The Mehrstellen Laplacian A on a real zero-boundary grid staged by TMA
// (gpw_mehr_tma.cuh), for arguments chunked for 64 x 16 tiles.
cudaError_t mehr_tma_f64(int mode, const StencilArgs& a, int nbatch, const GeneralCoefs& gc, cudaStream_t st);
cudaError_t mehr_tma_f32(int mode, const StencilArgs& a, int nbatch, const GeneralCoefs& gc, cudaStream_t st);

// The float32 level-0 residual restricted (K = 2, zero boundaries) into the
// next level's rho and first Jacobi iterate in one TMA launch
// (MODE_RESID_RESTRICT); `tune` times its tile variants instead.
bool resid_restrict_ok(const OpDesc& d, const void* in, const void* rho, const GridView& v, const void* out,
                       const void* out2, const GridView& vco, int nbatch);
cudaError_t launch_resid_restrict(const OpDesc& d, const void* in, const void* rho, const GridView& v, void* out,
                                  void* out2, const GridView& vco, int nbatch, double w2, double c02,
                                  const unsigned char* active, bool tune, cudaStream_t st);

// Periodic / Bloch (or mixed-boundary) star applies on the TMA row kernel
// (gpw_bloch.cu): eligibility and launch.
bool bloch_path_ok(const OpDesc& d, int dtype, const void* in, const GridView& vin, const void* out,
                   const GridView& vout, int nbatch);
struct StencilArgs;
cudaError_t launch_bloch(const OpDesc& d, int dtype, const StencilArgs& a, int nbatch, cudaStream_t st);
// The cp.async star / general kernel for an apply.
cudaError_t launch_apply_cpasync(const OpDesc& d, int dtype, const StencilArgs& a, int nbatch, cudaStream_t st);

// Device status word written by kernels whose bounded waits expire
// (GPW_ETIMEDOUT); allocated on first use, which must not happen inside a
// stream capture (handle constructors call it).
int* device_status_word();

// Autotuner records (gpw_tune_export / gpw_tune_import).
void tune_export_tma(std::string& out);
bool tune_import_tma(const int* fields);
void tune_export_bloch(std::string& out);
bool tune_import_bloch(const int* fields);

}  // namespace gpw
