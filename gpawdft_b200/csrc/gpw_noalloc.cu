// Allocation-free variant of the fused residual + norm entry point.
//
// Who needs it: host code that must not (or cannot) allocate device memory
// while it runs -- code executing inside another framework's memory pool or
// allocator callback, real-time / signal-safe paths, processes that reserve
// and lock all device memory up front, or embedders whose allocator is not
// the CUDA runtime.  gpw_operator_residual() grows a device workspace for the
// partial sums of its deterministic reduction on first use (cudaMalloc); this
// variant keeps those partial sums in a fixed array compiled into the
// library instead, so a call allocates nothing.
//
// The array (g_noalloc_scratch, NOALLOC_BYTES = 540,672 bytes, about 528 KB:
// 65,536 double partial sums plus 4,096 unsigned counters) exists once per
// GPU that loads the library and stays resident until the process exits.
// Its device address is looked up with cudaGetSymbolAddress the first time
// the entry point runs on a device (with that device current); that first
// call should therefore come before any stream capture.  All calls share the
// one array: the reduction counters are cleared at the start of every call,
// and two calls that overlap on the GPU (different streams, no ordering
// between them) race on it.
#include <algorithm>
#include <cstring>
#include <mutex>
#include <string>

#include "gpw_internal.h"
#include "gpw_stencil.cuh"

namespace gpw {
const OpDesc* operator_desc(const gpw_operator* op);
}

using namespace gpw;

namespace {

// Limits of one call: CTAs of the reduction over all `nin` grids, and nin.
constexpr int64_t NOALLOC_MAX_PARTIALS = 1 << 16;  // doubles: 512 KiB of partial sums (blocks x grids)
constexpr int64_t NOALLOC_MAX_NIN = 4096;          // grids per call (one counter each)
constexpr size_t NOALLOC_BYTES =
    (size_t)NOALLOC_MAX_PARTIALS * sizeof(double) + (size_t)NOALLOC_MAX_NIN * sizeof(unsigned);
static_assert(NOALLOC_BYTES == 540672, "the documented size of the fixed scratch is 540,672 bytes");

static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_BYTES];

constexpr int kMaxDevices = 64;
void* g_scratch_dev[kMaxDevices] = {};
std::mutex g_setup_mutex;

// Device address of the scratch array for the current device (set-up once per
// device, with that device current).
int scratch_for_current_device(void** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail(e, "residual_noalloc: cudaGetDevice");
  if (dev < 0 || dev >= kMaxDevices) return fail(GPW_ENOTSUP, "residual_noalloc: device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch_dev[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) return cuda_fail(e, "residual_noalloc: cudaGetSymbolAddress");
    g_scratch_dev[dev] = p;
  }
  *out = g_scratch_dev[dev];
  return GPW_OK;
}

void noalloc_chunks(int n0, int64_t tiles, int minz, int& zchunk, int& nchunk) {
  const int64_t want = 4LL * num_sms();
  int64_t nc = (want + tiles - 1) / std::max<int64_t>(tiles, 1);
  const int64_t maxc = std::max(1, (n0 + minz - 1) / minz);
  nc = std::max<int64_t>(1, std::min<int64_t>(nc, maxc));
  zchunk = (int)((n0 + nc - 1) / nc);
  nchunk = (n0 + zchunk - 1) / zchunk;
}

// Launch geometry + launch of the residual kernel on a star (cp.async) or
// general-offset stencil; returns the CTAs per grid through `nblk`.
template <typename T, int R>
cudaError_t star_residual(StencilArgs a, const OpDesc& d, int nbatch, bool launch, int64_t& nblk,
                          cudaStream_t st) {
  using C = StarCfg<R, T>;
  dim3 grid((a.vout.n[2] + C::TZ - 1) / C::TZ, (a.vout.n[1] + C::TY - 1) / C::TY, 1);
  noalloc_chunks(a.vout.n[0], (int64_t)grid.x * grid.y * nbatch, 2 * R + 2, a.zchunk, a.nchunk);
  grid.z = a.nchunk * nbatch;
  a.nblk_seg = grid.x * grid.y * a.nchunk;
  nblk = a.nblk_seg;
  if (!launch) return cudaSuccess;
  const size_t smem = (size_t)C::NSTAGE * C::PS * sizeof(T);
  auto kern = star_stencil_kernel<T, R, MODE_RESIDUAL>;
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  kern<<<grid, dim3(C::TZ, C::NTY), smem, st>>>(a, star_coefs_typed<typename EltTraits<T>::S>(d.sc));
  return cudaGetLastError();
}

template <typename T>
cudaError_t general_residual(StencilArgs a, const OpDesc& d, int nbatch, bool launch, int64_t& nblk,
                             cudaStream_t st) {
  const int mp = d.mp;
  dim3 grid((a.vout.n[2] + GEN_TZ - 1) / GEN_TZ, (a.vout.n[1] + GEN_TY - 1) / GEN_TY, 1);
  noalloc_chunks(a.vout.n[0], (int64_t)grid.x * grid.y * nbatch, 2 * mp + 2, a.zchunk, a.nchunk);
  grid.z = a.nchunk * nbatch;
  a.nblk_seg = grid.x * grid.y * a.nchunk;
  nblk = a.nblk_seg;
  if (!launch) return cudaSuccess;
  const size_t smem = (size_t)(2 * mp + 2) * (GEN_TY + 2 * mp) * (GEN_TZ + 2 * mp) * sizeof(T);
  if (smem > 227 * 1024) return cudaErrorInvalidValue;
  auto kern = general_stencil_kernel<T, MODE_RESIDUAL>;
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  kern<<<grid, dim3(GEN_TZ, GEN_TY), smem, st>>>(a, d.gc);
  return cudaGetLastError();
}

template <typename T>
cudaError_t residual_dispatch(const StencilArgs& a, const OpDesc& d, int nbatch, bool launch, int64_t& nblk,
                              cudaStream_t st) {
  if (d.star) {
    switch (d.R) {
      case 1: return star_residual<T, 1>(a, d, nbatch, launch, nblk, st);
      case 2: return star_residual<T, 2>(a, d, nbatch, launch, nblk, st);
      case 3: return star_residual<T, 3>(a, d, nbatch, launch, nblk, st);
      case 4: return star_residual<T, 4>(a, d, nbatch, launch, nblk, st);
    }
  }
  return general_residual<T>(a, d, nbatch, launch, nblk, st);
}

}  // namespace

extern "C" int gpw_operator_residual_noalloc(gpw_operator* op, int dtype, const void* func, const void* source,
                                             void* r, int64_t nin, double* sumsq_dev, gpw_stream stream) {
  if (!op || !func || !source || !sumsq_dev) return fail(GPW_EINVAL, "residual_noalloc: null argument");
  if (dtype != GPW_F64 && dtype != GPW_F32) return fail(GPW_EINVAL, "residual_noalloc: real dtypes only");
  if (nin <= 0) return fail(GPW_EINVAL, "residual_noalloc: nin must be positive");
  if (nin > NOALLOC_MAX_NIN)
    return fail(GPW_EINVAL, "residual_noalloc: nin exceeds the fixed scratch limit of " +
                                std::to_string(NOALLOC_MAX_NIN) + " grids per call");
  if (r == func) return fail(GPW_EINVAL, "residual_noalloc: r must not alias func");
  const OpDesc& d = *operator_desc(op);
  cudaStream_t st = (cudaStream_t)stream;
  StencilArgs a{};
  a.in = func;
  a.out = r;
  a.rho = source;
  a.vin = a.vout = a.vrho = contiguous_view(d.n);
  a.bc = make_boundary(d.periodic, dtype, nullptr);
  a.w = 1.0;
  a.c0 = d.coefs[0];
  const bool star = d.star && d.R >= 1 && d.R <= 4;
  OpDesc dd = d;
  dd.star = star;
  // size check before touching the device
  int64_t nblk = 0;
  cudaError_t e = (dtype == GPW_F64) ? residual_dispatch<double>(a, dd, (int)nin, false, nblk, st)
                                     : residual_dispatch<float>(a, dd, (int)nin, false, nblk, st);
  if (e != cudaSuccess) return cuda_fail(e, "residual_noalloc: geometry");
  if (nblk * nin > NOALLOC_MAX_PARTIALS)
    return fail(GPW_EINVAL, "residual_noalloc: grid too large for the fixed scratch (" +
                                std::to_string(nblk * nin) + " reduction blocks > " +
                                std::to_string(NOALLOC_MAX_PARTIALS) + ")");
  void* scratch = nullptr;
  int rc = scratch_for_current_device(&scratch);
  if (rc) return rc;
  double* partial = static_cast<double*>(scratch);
  unsigned* counter = reinterpret_cast<unsigned*>(static_cast<unsigned char*>(scratch) +
                                                  (size_t)NOALLOC_MAX_PARTIALS * sizeof(double));
  // the reduction's completion counters must start at zero
  e = cudaMemsetAsync(counter, 0, (size_t)nin * sizeof(unsigned), st);
  if (e != cudaSuccess) return cuda_fail(e, "residual_noalloc: clear counters");
  a.gsum.partial = partial;
  a.gsum.counter = counter;
  a.gsum.result = sumsq_dev;
  e = (dtype == GPW_F64) ? residual_dispatch<double>(a, dd, (int)nin, true, nblk, st)
                         : residual_dispatch<float>(a, dd, (int)nin, true, nblk, st);
  if (e != cudaSuccess) return cuda_fail(e, "residual_noalloc: launch");
  return GPW_OK;
}
