// Kernel launchers: dtype / radius / tap-count dispatch, launch geometry and
// shared-memory opt-in for every device kernel of the library.
#include <algorithm>
#include <cstdio>
#include <initializer_list>
#include <atomic>
#include <map>
#include <mutex>

#include <cudaTypedefs.h>

#include "gpw_blas.cuh"
#include "gpw_coarse.cuh"
#include "gpw_internal.h"
#include "gpw_stencil.cuh"
#include "gpw_transfer.cuh"
#include "gpw_transfer_k2.cuh"
#include "gpw_transfer_rows.cuh"

namespace gpw {

static std::atomic<int> g_pdl{1};
bool pdl_enabled() { return g_pdl.load() != 0; }

int num_sms() {
  static int sms = 0;
  if (!sms) {
    int dev = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0) sms = 148;
  }
  return sms;
}

// Dynamic shared memory above 48 KB needs a one-time opt-in per kernel.
template <typename F>
static cudaError_t smem_optin(F* kernel, size_t bytes) {
  if (bytes <= 48 * 1024) return cudaSuccess;
  return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

// Chunking of axis 0: enough CTAs for ~4 per SM, but never chunks shorter
// than `minz` planes (each chunk re-reads a 2R-plane warm-up).
static void choose_chunks(int n0, int64_t tiles, int minz, int& zchunk, int& nchunk) {
  const int64_t want = 4LL * num_sms();
  int64_t nc = (want + tiles - 1) / std::max<int64_t>(tiles, 1);
  const int64_t maxc = std::max(1, (n0 + minz - 1) / minz);
  nc = std::max<int64_t>(1, std::min<int64_t>(nc, maxc));
  zchunk = (int)((n0 + nc - 1) / nc);
  nchunk = (n0 + zchunk - 1) / zchunk;
}

// ------------------------------------------------------------------ stencils
template <typename T, int R, int MODE, bool EPI>
static cudaError_t run_star_epi(const StencilArgs& a0, const OpDesc& d, int nbatch, cudaStream_t st) {
  using C = StarCfg<R, T>;
  StencilArgs a = a0;
  const GridView& v = a.vout;
  dim3 grid((v.n[2] + C::TZ - 1) / C::TZ, (v.n[1] + C::TY - 1) / C::TY, 1);
  choose_chunks(v.n[0], (int64_t)grid.x * grid.y * nbatch, 2 * R + 2, a.zchunk, a.nchunk);
  grid.z = a.nchunk * nbatch;
  a.nblk_seg = grid.x * grid.y * a.nchunk;
  const size_t smem = (size_t)C::NSTAGE * C::PS * sizeof(T);
  using S = typename EltTraits<T>::S;
  void (*kern)(StencilArgs, StarCoefsT<S>);
  if constexpr (sizeof(T) >= 16)
    kern = star_stencil_kernel_2cta<T, R, MODE, EPI>;
  else
    kern = star_stencil_kernel<T, R, MODE, EPI>;
  static std::once_flag once;
  cudaError_t e = cudaSuccess;
  std::call_once(once, [&] { e = smem_optin(kern, smem); });
  if (e != cudaSuccess) return e;
  kern<<<grid, dim3(C::TZ, C::NTY), smem, st>>>(a, star_coefs_typed<S>(d.sc));  // NT threads
  return cudaGetLastError();
}

template <typename T, int R, int MODE>
static cudaError_t run_star(const StencilArgs& a, const OpDesc& d, int nbatch, cudaStream_t st) {
  if constexpr (MODE == MODE_APPLY) {
    if (a.pot || a.aux) return run_star_epi<T, R, MODE, true>(a, d, nbatch, st);
  }
  return run_star_epi<T, R, MODE, false>(a, d, nbatch, st);
}

// Tile of a general-offset launch for element size es and radius mp: the
// register-blocked kernel's where its ring of planes fits in shared memory
// (next to its static tables), else the plain kernel's.
static void general_tile(int mp, size_t es, int& tz, int& ty, bool& blocked) {
  const int btz = es >= 16 ? 32 : 64, bty = 16;  // GenBlk's TZ x TY
  blocked = mp >= 1 && mp <= GEN_BLK_MAXMP && general_block_smem(mp, es, btz, bty, PMAX) <= 220 * 1024;
  tz = blocked ? btz : GEN_TZ;
  ty = blocked ? bty : GEN_TY;
}

// Opt kernel `kern` in to `smem` bytes of dynamic shared memory (the
// largest so far; the static part counts against the same per-CTA limit).
template <typename K>
static cudaError_t general_optin(K kern, size_t smem, std::mutex& mu, size_t& opted) {
  std::lock_guard<std::mutex> lock(mu);
  if (smem > opted) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    opted = smem;
  }
  return cudaSuccess;
}

// The operator is the Mehrstellen Laplacian A: 19 coefficients at exactly
// the offsets of MEHR_OFF, in that order.
static bool is_mehrstellen_a(const GeneralCoefs& gc) {
  if (gc.ncoef != MEHR_NC || gc.mp != 1) return false;
  for (int c = 0; c < MEHR_NC; ++c)
    for (int e = 0; e < 3; ++e)
      if (gc.off[c][e] != MEHR_OFF[c][e]) return false;
  return true;
}

static bool aligned16(const void* p);
static bool view_tma_ok(const GridView& v, size_t es, int nbatch);

template <typename T, int MODE>
static cudaError_t run_mehrstellen(const StencilArgs& a0, const OpDesc& d, int nbatch, cudaStream_t st) {
  using C = MehrCfg;
  StencilArgs a = a0;
  const GridView& v = a.vout;
  dim3 grid((v.n[2] + C::TZ - 1) / C::TZ, (v.n[1] + C::TY - 1) / C::TY, 1);
  choose_chunks(v.n[0], (int64_t)grid.x * grid.y * nbatch, 4, a.zchunk, a.nchunk);
  grid.z = a.nchunk * nbatch;
  a.nblk_seg = grid.x * grid.y * a.nchunk;
  // zero boundaries on 16-byte-pitched grids: planes staged by TMA
  if (!d.periodic[0] && !d.periodic[1] && !d.periodic[2] && a.in != a.out && aligned16(a.in) &&
      view_tma_ok(a.vin, sizeof(T), nbatch) && tensor_map_encoder()) {
    if constexpr (sizeof(T) == 8) return mehr_tma_f64(MODE, a, nbatch, d.gc, st);
    else return mehr_tma_f32(MODE, a, nbatch, d.gc, st);
  }
  a.gdepth = 4;  // planes loaded ahead (7 planes of 9.5 KB for float64)
  const size_t smem = (size_t)(3 + a.gdepth) * C::PS * sizeof(T);
  auto kern = mehrstellen_kernel<T, MODE>;
  static std::once_flag once;
  cudaError_t e = cudaSuccess;
  std::call_once(once, [&] { e = smem_optin(kern, smem); });
  if (e != cudaSuccess) return e;
  kern<<<grid, dim3(C::NTX, C::NTY), smem, st>>>(a, d.gc);
  return cudaGetLastError();
}

template <typename T, int MODE>
static cudaError_t run_general(const StencilArgs& a0, const OpDesc& d, int nbatch, cudaStream_t st) {
  if constexpr (!EltTraits<T>::cpx && (MODE == MODE_APPLY || MODE == MODE_RESIDUAL || MODE == MODE_JACOBI)) {
    if (is_mehrstellen_a(d.gc)) return run_mehrstellen<T, MODE>(a0, d, nbatch, st);
  }
  StencilArgs a = a0;
  const GridView& v = a.vout;
  const int mp = d.mp;
  int tz, ty;
  bool blocked;
  general_tile(mp, sizeof(T), tz, ty, blocked);
  if (blocked && (tz != GenBlk<T, 1>::TZ || ty != GenBlk<T, 1>::TY)) return cudaErrorInvalidConfiguration;
  dim3 grid((v.n[2] + tz - 1) / tz, (v.n[1] + ty - 1) / ty, 1);
  choose_chunks(v.n[0], (int64_t)grid.x * grid.y * nbatch, 2 * mp + 2, a.zchunk, a.nchunk);
  grid.z = a.nchunk * nbatch;
  a.nblk_seg = grid.x * grid.y * a.nchunk;
  // planes loaded ahead: as many (up to 4) as keep two CTAs per SM
  int depth = 1;
  while (blocked && depth < 4 && general_block_smem(mp, sizeof(T), tz, ty, d.gc.ncoef, depth + 1) <= 110 * 1024)
    ++depth;
  a.gdepth = depth;
  const size_t smem = blocked ? general_block_smem(mp, sizeof(T), tz, ty, d.gc.ncoef, depth)
                              : (size_t)(2 * mp + 2) * (ty + 2 * mp) * (tz + 2 * mp) * sizeof(T);
  if (smem > 227 * 1024) return cudaErrorInvalidValue;
  if (blocked) {
    auto go = [&](auto kern, std::mutex& mu, size_t& opted) -> cudaError_t {
      cudaError_t e = general_optin(kern, smem, mu, opted);
      if (e != cudaSuccess) return e;
      kern<<<grid, dim3(32, GenBlk<T, 1>::NTY), smem, st>>>(a, d.gc);
      return cudaGetLastError();
    };
    static std::mutex mu[GEN_BLK_MAXMP];
    static size_t opted[GEN_BLK_MAXMP] = {48 * 1024, 48 * 1024, 48 * 1024};
    switch (mp) {
      case 1: return go(general_block_kernel<T, MODE, 1>, mu[0], opted[0]);
      case 2: return go(general_block_kernel<T, MODE, 2>, mu[1], opted[1]);
      case 3: return go(general_block_kernel<T, MODE, 3>, mu[2], opted[2]);
    }
    return cudaErrorInvalidValue;
  }
  auto kern = general_stencil_kernel<T, MODE>;
  static std::mutex mu;
  static size_t opted = 48 * 1024;
  cudaError_t e = general_optin(kern, smem, mu, opted);
  if (e != cudaSuccess) return e;
  kern<<<grid, dim3(GEN_TZ, GEN_TY), smem, st>>>(a, d.gc);
  return cudaGetLastError();
}

template <typename T, int MODE>
static cudaError_t dispatch_star(const StencilArgs& a, const OpDesc& d, int nbatch, cudaStream_t st) {
  switch (d.R) {
    case 1: return run_star<T, 1, MODE>(a, d, nbatch, st);
    case 2: return run_star<T, 2, MODE>(a, d, nbatch, st);
    case 3: return run_star<T, 3, MODE>(a, d, nbatch, st);
    case 4: return run_star<T, 4, MODE>(a, d, nbatch, st);
  }
  return cudaErrorInvalidValue;
}

template <typename T, int MODE>
static cudaError_t dispatch_mode(const StencilArgs& a, const OpDesc& d, int nbatch, cudaStream_t st) {
  const bool use_star = (MODE == MODE_JACOBI) ? d.star_jacobi : d.star;
  if (use_star) return dispatch_star<T, MODE>(a, d, nbatch, st);
  return run_general<T, MODE>(a, d, nbatch, st);
}

static bool star_radius_ok(int R) { return R >= 1 && R <= 4; }

// The cp.async star / general kernel for an apply (the periodic TMA row
// kernel's tuner times it beside its own layouts).
cudaError_t launch_apply_cpasync(const OpDesc& d, int dtype, const StencilArgs& a, int nbatch, cudaStream_t st) {
  OpDesc dd = d;
  if (!star_radius_ok(dd.R)) {
    dd.star = false;
    dd.star_jacobi = false;
  }
  switch (dtype) {
    case GPW_F64: return dispatch_mode<double, MODE_APPLY>(a, dd, nbatch, st);
    case GPW_C128: return dispatch_mode<double2, MODE_APPLY>(a, dd, nbatch, st);
    case GPW_F32: return dispatch_mode<float, MODE_APPLY>(a, dd, nbatch, st);
    case GPW_C64: return dispatch_mode<float2, MODE_APPLY>(a, dd, nbatch, st);
  }
  return cudaErrorInvalidValue;
}

int stencil_blocks_per_member(const OpDesc& d, int mode, const GridView& v, int nbatch) {
  const bool use_star = ((mode == MODE_JACOBI) ? d.star_jacobi : d.star) && star_radius_ok(d.R);
  auto blocks = [&](int tz, int ty, int minz) {
    const int gx = (v.n[2] + tz - 1) / tz, gy = (v.n[1] + ty - 1) / ty;
    int zc, nc;
    choose_chunks(v.n[0], (int64_t)gx * gy * nbatch, minz, zc, nc);
    return gx * gy * nc;
  };
  int nblk;
  if (use_star) {
    nblk = blocks(32, d.real ? GPW_STAR_TY : GPW_STAR_TY / 2, 2 * d.R + 2);  // complex128: half-height tiles
  } else {
    // the tile depends on the element size: the most CTAs over the op's types
    nblk = 0;
    for (size_t es : d.real ? std::initializer_list<size_t>{4, 8} : std::initializer_list<size_t>{8, 16}) {
      int tz, ty;
      bool blocked;
      general_tile(d.mp, es, tz, ty, blocked);
      nblk = std::max(nblk, blocks(tz, ty, 2 * d.mp + 2));
    }
  }
  if (use_star) {  // a TMA tile variant may be chosen instead: bound its CTA count
    // (tiles at least 48 points wide and 8 rows high, at most n0 / (2R + 2)
    // axis-0 chunks)
    const int tx2 = (v.n[2] + 47) / 48, ty2 = (v.n[1] + 7) / 8;
    nblk = std::max(nblk, tx2 * ty2 * std::max(1, v.n[0] / (2 * d.R + 2)));
  }
  return nblk;
}

// ------------------------------------------------------------------ TMA path
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  return fn;
}

static int* g_status_dev = nullptr;  // device status word of TMA kernels

int* device_status_word() {
  static std::once_flag once;
  std::call_once(once, [] {
    if (cudaMalloc(&g_status_dev, sizeof(int)) == cudaSuccess) cudaMemset(g_status_dev, 0, sizeof(int));
    tensor_map_encoder();  // resolve the driver entry point outside any capture too
  });
  return g_status_dev;
}

static bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

static bool view_tma_ok(const GridView& v, size_t es, int nbatch) {
  // strides (bytes) multiples of 16 and even element strides (2-point stores)
  if ((v.s1 * es) % 16 || (v.s0 * es) % 16) return false;
  if (nbatch > 1 && (v.sb * es) % 16) return false;
  if (v.s1 % 2 || v.s0 % 2 || (nbatch > 1 && v.sb % 2)) return false;
  return true;
}

// ------------------------------------------------------------------ TMA autotuner
// Per launch shape (dtype, radius, epilogue, grid extent, batch) the tile
// variant and axis-0 chunking that ran fastest when the shape was tuned;
// untuned shapes use variant 2 and the wave model.
namespace {
struct TuneKey {
  int dtype, R, mode, n0, n1, n2, nbatch;
  bool operator<(const TuneKey& o) const {
    const int a[7] = {dtype, R, mode, n0, n1, n2, nbatch}, b[7] = {o.dtype, o.R, o.mode, o.n0, o.n1, o.n2, o.nbatch};
    for (int i = 0; i < 7; ++i)
      if (a[i] != b[i]) return a[i] < b[i];
    return false;
  }
};
std::mutex g_tune_mu;
std::map<TuneKey, TmaChoice> g_tune;
}  // namespace

// Pinned choice (variant >= 0): every TMA stencil launch whose dtype and
// radius have that variant uses it with this chunking, instead of the
// tuned one (set through gpw_set_tma_variant).
static std::atomic<int> g_force_var{-1};
static std::atomic<int> g_force_nc{0};

static bool tma_variant_available(int dtype, int R, int var) {
  if (var < 0 || var >= TMA_NVARIANT) return false;
  if (var >= 5 && var <= 9 && dtype != GPW_F32) return false;  // 4-point variants: float32 only
  return (R == 1 || R == 3) || var == (R == 4 ? 1 : 2);
}

static TmaChoice tma_choice(int dtype, int R, int mode, const GridView& v, int nbatch) {
  const int fv = g_force_var.load();
  if (fv >= 0 && tma_variant_available(dtype, R, fv)) return TmaChoice{fv, g_force_nc.load()};
  std::lock_guard<std::mutex> lock(g_tune_mu);
  auto it = g_tune.find(TuneKey{dtype, R, mode, v.n[0], v.n[1], v.n[2], nbatch});
  if (it != g_tune.end()) return it->second;
  return TmaChoice{R == 4 ? 1 : 2, 0};
}

static bool tma_tuned(int dtype, int R, int mode, const GridView& v, int nbatch) {
  std::lock_guard<std::mutex> lock(g_tune_mu);
  return g_tune.count(TuneKey{dtype, R, mode, v.n[0], v.n[1], v.n[2], nbatch}) != 0;
}

static cudaError_t tma_launch(int dtype, int mode, int R, const TmaChoice& ch, const StencilArgs& a, int nbatch,
                              const StarCoefs& sc, cudaStream_t st) {
  if (dtype == GPW_F64) return tma_stencil_f64(mode, R, ch.var, a, nbatch, sc, ch.nchunk, st);
  return tma_stencil_f32(mode, R, ch.var, a, nbatch, sc, ch.nchunk, st);
}

extern "C" int gpw_set_pdl(int on) {
  g_pdl.store(on ? 1 : 0);
  return GPW_OK;
}

extern "C" int gpw_set_tma_variant(int variant, int nchunk) {
  if (variant < -1 || variant >= TMA_NVARIANT) return fail(GPW_EINVAL, "tma variant out of range");
  g_force_nc.store(nchunk);
  g_force_var.store(variant);
  return GPW_OK;
}

int tuned_stencil_count() {
  std::lock_guard<std::mutex> lock(g_tune_mu);
  return (int)g_tune.size();
}

// The TMA tuner's choices as text records "tma dtype R mode n0 n1 n2 nbatch
// var nchunk", one a line (gpw_tune_export).
void tune_export_tma(std::string& out) {
  std::lock_guard<std::mutex> lock(g_tune_mu);
  char line[160];
  for (const auto& kv : g_tune) {
    const TuneKey& k = kv.first;
    snprintf(line, sizeof line, "tma %d %d %d %d %d %d %d %d %d\n", k.dtype, k.R, k.mode, k.n0, k.n1, k.n2,
             k.nbatch, kv.second.var, kv.second.nchunk);
    out += line;
  }
}

// One "tma ..." record back into the tuner (gpw_tune_import); records whose
// variant is not compiled for that element type and radius are refused.
bool tune_import_tma(const int* f) {
  const int dtype = f[0], R = f[1], mode = f[2];
  if ((dtype != GPW_F64 && dtype != GPW_F32) || R < 1 || R > 4 || mode < 0 || mode > 6) return false;
  if (f[3] <= 0 || f[4] <= 0 || f[5] <= 0 || f[6] <= 0 || f[8] < -8 || f[8] > 64) return false;
  if (!tma_variant_available(dtype, R, f[7])) return false;
  std::lock_guard<std::mutex> lock(g_tune_mu);
  g_tune[TuneKey{dtype, R, mode, f[3], f[4], f[5], f[6]}] = TmaChoice{f[7], f[8]};
  return true;
}

// The TMA path serves real zero-boundary star stencils whose arrays are
// 16-byte aligned with 16-byte (and even-element) strides.
static bool tma_path_ok(const OpDesc& d, int dtype, int mode, const void* in, const GridView& vin, const void* out,
                        const GridView& vout, const void* rho, const GridView& vrho, int nbatch) {
  if (dtype != GPW_F64 && dtype != GPW_F32) return false;
  if (d.periodic[0] || d.periodic[1] || d.periodic[2]) return false;
  const bool star = (mode == MODE_JACOBI) ? d.star_jacobi : d.star;
  if (!star || !star_radius_ok(d.R)) return false;
  if (in == out) return false;
  if (!tensor_map_encoder()) return false;
  const size_t es = elt_size(dtype);
  if (!aligned16(in) || !view_tma_ok(vin, es, nbatch)) return false;
  if (out && (!aligned16(out) || !view_tma_ok(vout, es, nbatch))) return false;
  if (mode != MODE_APPLY && (!aligned16(rho) || !view_tma_ok(vrho, es, nbatch))) return false;
  return true;
}

cudaError_t launch_stencil(const OpDesc& d, int dtype, int mode, const void* in, const GridView& vin, void* out,
                           const GridView& vout, const void* rho, const GridView& vrho, int nbatch,
                           const Boundary& bc, double w, const unsigned char* active, const GridSum& gs,
                           cudaStream_t st, const void* pot, const void* aux, double aux_scale) {
  StencilArgs a{};
  a.pot = mode == MODE_APPLY ? pot : nullptr;
  a.aux = mode == MODE_APPLY ? aux : nullptr;
  a.aux_scale = aux_scale;
  a.in = in;
  a.out = out;
  a.rho = rho;
  a.vin = vin;
  a.vout = vout;
  a.vrho = vrho;
  a.bc = bc;
  a.w = w;
  a.c0 = d.coefs.empty() ? 1.0 : d.coefs[0];
  a.active = active;
  a.gsum = gs;
  if (tma_path_ok(d, dtype, mode, in, vin, out, vout, rho, vrho, nbatch)) {
    // first launch of an untuned shape outside stream capture: tune it now
    // (apply / residual / Jacobi recompute their output from inputs they do
    // not overwrite, so the timed repetitions leave the same result; an aux
    // term read from the output itself is such an input, so that call runs
    // on the default tiles untuned)
    if (!active && out != rho && (!aux || aux != out) && g_force_var.load() < 0 &&
        !tma_tuned(dtype, d.R, mode, vout, nbatch)) {
      cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
      if (cudaStreamIsCapturing(st, &cs) == cudaSuccess && cs == cudaStreamCaptureStatusNone) {
        cudaError_t te = tune_stencil(d, dtype, mode, in, vin, out, vout, rho, vrho, nullptr, nbatch, w, gs, st);
        if (te != cudaSuccess) return te;
      }
    }
    const TmaChoice ch = tma_choice(dtype, d.R, mode, vout, nbatch);
    // an apply with a potential or aux term runs its own kernel instance, on
    // the plain apply's tuned tiles
    const int lmode = (mode == MODE_APPLY && (a.pot || a.aux)) ? MODE_APPLY_EPI : mode;
    return tma_launch(dtype, lmode, d.R, ch, a, nbatch, d.sc, st);
  }
  if (mode == MODE_APPLY && !active && bloch_path_ok(d, dtype, in, vin, out, vout, nbatch))
    return launch_bloch(d, dtype, a, nbatch, st);
  OpDesc dd = d;
  if (!star_radius_ok(dd.R)) {
    dd.star = false;
    dd.star_jacobi = false;
  }
  switch (mode) {
    case MODE_APPLY:
      switch (dtype) {
        case GPW_F64: return dispatch_mode<double, MODE_APPLY>(a, dd, nbatch, st);
        case GPW_C128: return dispatch_mode<double2, MODE_APPLY>(a, dd, nbatch, st);
        case GPW_F32: return dispatch_mode<float, MODE_APPLY>(a, dd, nbatch, st);
        case GPW_C64: return dispatch_mode<float2, MODE_APPLY>(a, dd, nbatch, st);
      }
      break;
    case MODE_RESIDUAL:
      switch (dtype) {
        case GPW_F64: return dispatch_mode<double, MODE_RESIDUAL>(a, dd, nbatch, st);
        case GPW_F32: return dispatch_mode<float, MODE_RESIDUAL>(a, dd, nbatch, st);
      }
      break;
    case MODE_JACOBI:
      switch (dtype) {
        case GPW_F64: return dispatch_mode<double, MODE_JACOBI>(a, dd, nbatch, st);
        case GPW_F32: return dispatch_mode<float, MODE_JACOBI>(a, dd, nbatch, st);
      }
      break;
  }
  return cudaErrorInvalidValue;
}

bool dc_fusable(const OpDesc& d) {
  return !d.periodic[0] && !d.periodic[1] && !d.periodic[2] && d.star_jacobi && star_radius_ok(d.R) &&
         tensor_map_encoder() != nullptr;
}

cudaError_t launch_stencil_dc(const OpDesc& d, int mode, const void* in, const GridView& v, void* out, void* out2,
                              const void* rho, int nbatch, double w, double w2, const unsigned char* active,
                              const GridSum& gs, cudaStream_t st) {
  if (!dc_fusable(d)) return cudaErrorNotSupported;
  const size_t es_in = (mode == MODE_RESID_DC) ? 8 : 4;
  if (!aligned16(in) || !aligned16(rho) || !aligned16(out2) || (out && !aligned16(out)) ||
      !view_tma_ok(v, es_in, nbatch) || !view_tma_ok(v, 4, nbatch))
    return cudaErrorNotSupported;
  StencilArgs a{};
  a.in = in;
  a.out = out;
  a.out2 = out2;
  a.rho = rho;
  a.vin = a.vout = a.vrho = v;
  a.w = w;
  a.w2 = w2;
  a.c0 = d.coefs[0];
  a.active = active;
  a.gsum = gs;
  if (mode != MODE_RESID_DC && mode != MODE_JACOBI_ADD64 && mode != MODE_JACOBI_SCALED_IN) return cudaErrorInvalidValue;
  const int dtype = (mode == MODE_RESID_DC) ? GPW_F64 : GPW_F32;
  const TmaChoice ch = tma_choice(dtype, d.R, mode, v, nbatch);
  return tma_launch(dtype, mode, d.R, ch, a, nbatch, d.sc, st);
}

static cudaError_t tune_stencil_args(const OpDesc& d, int ldtype, int mode, const StencilArgs& a, int nbatch,
                                     cudaStream_t st);

bool resid_restrict_ok(const OpDesc& d, const void* in, const void* rho, const GridView& v, const void* out,
                       const void* out2, const GridView& vco, int nbatch) {
  if (!dc_fusable(d) || (d.R != 1 && d.R != 3) || !tensor_map_encoder()) return false;
  if (!aligned16(in) || !aligned16(rho) || !aligned16(out) || !aligned16(out2)) return false;
  if (!view_tma_ok(v, 4, nbatch)) return false;
  for (int c = 0; c < 3; ++c)
    if (v.n[c] != 2 * vco.n[c] + 1) return false;  // zero boundaries, fine centre 2I + 1
  return true;
}

cudaError_t launch_resid_restrict(const OpDesc& d, const void* in, const void* rho, const GridView& v, void* out,
                                  void* out2, const GridView& vco, int nbatch, double w2, double c02,
                                  const unsigned char* active, bool tune, cudaStream_t st) {
  if (!resid_restrict_ok(d, in, rho, v, out, out2, vco, nbatch)) return cudaErrorNotSupported;
  StencilArgs a{};
  a.in = in;
  a.out = out;
  a.out2 = out2;
  a.rho = rho;
  a.vin = a.vout = a.vrho = v;
  a.vco = vco;
  a.w = 1.0;
  a.w2 = w2;
  a.c0 = c02;  // the next level's diagonal: the first coarse sweep's w2 / c0
  a.active = active;
  // the tuning pass runs on the engine's buffers before any solve, when the
  // mask may mark every member inactive (the timed launches would then do no
  // work): it times every member, like the other stencils' tuning
  if (tune) {
    a.active = nullptr;
    return tune_stencil_args(d, GPW_F32, MODE_RESID_RESTRICT, a, nbatch, st);
  }
  const TmaChoice ch = tma_choice(GPW_F32, d.R, MODE_RESID_RESTRICT, v, nbatch);
  return tma_launch(GPW_F32, MODE_RESID_RESTRICT, d.R, ch, a, nbatch, d.sc, st);
}

cudaError_t tune_stencil(const OpDesc& d, int dtype, int mode, const void* in, const GridView& vin, void* out,
                         const GridView& vout, const void* rho, const GridView& vrho, void* out2, int nbatch,
                         double w, const GridSum& gs, cudaStream_t st) {
  StencilArgs a{};
  a.in = in;
  a.out = out;
  a.out2 = out2;
  a.rho = rho;
  a.vin = vin;
  a.vout = vout;
  a.vrho = vrho;
  a.w = w;
  a.w2 = w;
  a.c0 = d.coefs.empty() ? 1.0 : d.coefs[0];
  a.gsum = gs;
  int ldtype = dtype;
  if (mode == MODE_RESID_DC || mode == MODE_JACOBI_ADD64 || mode == MODE_JACOBI_SCALED_IN) {
    const size_t es_in = (mode == MODE_RESID_DC) ? 8 : 4;
    if (!dc_fusable(d) || !aligned16(in) || !aligned16(rho) || !aligned16(out2) || (out && !aligned16(out)) ||
        !view_tma_ok(vout, es_in, nbatch) || !view_tma_ok(vout, 4, nbatch))
      return cudaSuccess;
    ldtype = (mode == MODE_RESID_DC) ? GPW_F64 : GPW_F32;
    a.vin = a.vrho = vout;
  } else if (!tma_path_ok(d, dtype, mode, in, vin, out, vout, rho, vrho, nbatch)) {
    return cudaSuccess;  // not the TMA path: nothing to tune
  }
  return tune_stencil_args(d, ldtype, mode, a, nbatch, st);
}

// The tuning loop proper, on prepared arguments (element type ldtype).
static cudaError_t tune_stencil_args(const OpDesc& d, int ldtype, int mode, const StencilArgs& a, int nbatch,
                                     cudaStream_t st) {
  const GridView& vout = a.vout;
  const TuneKey key{ldtype, d.R, mode, vout.n[0], vout.n[1], vout.n[2], nbatch};
  {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    if (g_tune.count(key)) return cudaSuccess;
  }
  cudaEvent_t e0, e1;
  if (cudaEventCreate(&e0) != cudaSuccess) return cudaGetLastError();
  if (cudaEventCreate(&e1) != cudaSuccess) {
    cudaEventDestroy(e0);
    return cudaGetLastError();
  }
  TmaChoice best{d.R == 4 ? 1 : 2, 0};
  float best_ms = 1e30f;
  for (int var = 0; var < TMA_NVARIANT; ++var) {
    for (int nc : {0, -2, TMA_SPLIT}) {
      const TmaChoice ch{var, nc};
      cudaError_t e = tma_launch(ldtype, mode, d.R, ch, a, nbatch, d.sc, st);
      if (e != cudaSuccess) {
        cudaGetLastError();  // a variant this shape cannot launch: skip it
        continue;
      }
      // the faster of two rounds of eight launches (one round of three let
      // run-to-run noise pick tiles up to 1.4x slower than the steady state)
      const int reps = 8;
      float ms = 1e30f;
      for (int round = 0; round < 2; ++round) {
        cudaEventRecord(e0, st);
        for (int i = 0; i < reps && e == cudaSuccess; ++i) e = tma_launch(ldtype, mode, d.R, ch, a, nbatch, d.sc, st);
        cudaEventRecord(e1, st);
        if (cudaEventSynchronize(e1) != cudaSuccess || e != cudaSuccess) {
          cudaEventDestroy(e0);
          cudaEventDestroy(e1);
          return e != cudaSuccess ? e : cudaGetLastError();
        }
        float r = 0.f;
        cudaEventElapsedTime(&r, e0, e1);
        ms = std::min(ms, r);
      }
      if (ms < best_ms) {
        best_ms = ms;
        best = ch;
      }
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  std::lock_guard<std::mutex> lock(g_tune_mu);
  g_tune[key] = best;
  return cudaSuccess;
}

// ------------------------------------------------------------------ transfers
template <typename T, int K>
static cudaError_t run_restrict(TransferArgs a, int nbatch, cudaStream_t st) {
  using C = RestrictCfg<T, K>;
  dim3 grid((a.vout.n[2] + RS_OZ - 1) / RS_OZ, (a.vout.n[1] + RS_OY - 1) / RS_OY, 1);
  choose_chunks(a.vout.n[0], (int64_t)grid.x * grid.y * nbatch, K, a.zchunk, a.nchunk);
  grid.z = a.nchunk * nbatch;
  auto kern = restrict_kernel<T, K>;
  static std::once_flag once;
  cudaError_t e = cudaSuccess;
  std::call_once(once, [&] { e = smem_optin(kern, C::smem); });
  if (e != cudaSuccess) return e;
  kern<<<grid, dim3(RS_OZ, RS_OY), C::smem, st>>>(a);
  return cudaGetLastError();
}

template <typename T, int K>
static cudaError_t run_interp(TransferArgs a, int nbatch, cudaStream_t st) {
  using C = InterpCfg<T, K>;
  dim3 grid((a.vout.n[2] + IP_OZ - 1) / IP_OZ, (a.vout.n[1] + IP_OY - 1) / IP_OY, 1);
  choose_chunks(a.vout.n[0], (int64_t)grid.x * grid.y * nbatch, 2 * K, a.zchunk, a.nchunk);
  grid.z = a.nchunk * nbatch;
  auto kern = interpolate_kernel<T, K>;
  static std::once_flag once;
  cudaError_t e = cudaSuccess;
  std::call_once(once, [&] { e = smem_optin(kern, C::smem); });
  if (e != cudaSuccess) return e;
  kern<<<grid, dim3(IP_OZ, IP_OY), C::smem, st>>>(a);
  return cudaGetLastError();
}

// Restriction layout: 0 = the launcher's choice, 1 = the tile kernel
// (restrict_kernel), 2 / 3 = the row kernel with 384 / 192 threads (up to
// 8 / 4 coarse rows per CTA).  Process-wide; for tests and tuning studies.
static std::atomic<int> g_restrict_force{0};
static std::atomic<long long> g_restrict_rows_launches{0};

struct RowsPlan {
  RowRestrictArgs ra;
  size_t smem;
};

// Launch plan of restrict_rows_kernel with `nt` threads, or false where the
// kernel does not apply: 8- or 16-byte elements, rows and strides in whole
// 16-byte units (TMA and bulk copies), at most 32 staged rows (no more than
// the rows of a periodic axis 1) and one axis-1 item a thread, a tensor box
// row of at most 256 scalars, stages that fit in shared memory.
static bool rows_plan(const TransferArgs& a, int k, size_t es, bool cpx, int nt, int mo, RowsPlan& p) {
  const int n1 = a.vin.n[1], n2 = a.vin.n[2], nout2 = a.vout.n[2];
  if (es < 8 || k < 2 || k > 8 || !tensor_map_encoder()) return false;
  if ((n2 * es) % 16 || (a.vin.s1 * (int64_t)es) % 16 || (a.vin.s0 * (int64_t)es) % 16 ||
      (a.vin.sb * (int64_t)es) % 16 || !aligned16(a.in))
    return false;
  RowRestrictArgs& r = p.ra;
  r.t = a;
  r.ty = std::min(std::min(8, nt / std::max(nout2, 1)), a.vout.n[1]);
  if (r.ty < 1) return false;
  r.h = 2 * r.ty + 2 * k - 3;
  if (r.h > 32 || (a.bc.periodic[1] && n1 < r.h)) return false;
  // halo columns: at least K - 1, in whole 16-byte units
  const int unit = (int)(16 / es);
  r.L = (k - 1 + unit - 1) / unit * unit;
  if (n2 < r.L) return false;
  // every tap inside the staged row: fine columns -pad .. -pad + 2 (nout2 - 1) + 2K - 2
  const int lo = -a.pad0[2], hi = -a.pad0[2] + 2 * (nout2 - 1) + 2 * k - 2;
  if (lo < -r.L || hi >= n2 + r.L) return false;
  // row pitches 16 bytes past a multiple of 128: lanes on consecutive rows
  // read distinct banks
  auto pitch_for = [&](int n) {
    int q = n;
    while ((q * (int64_t)es) % 128 != 16) ++q;
    return q;
  };
  r.pitch = pitch_for(n2 + 2 * r.L);
  if (r.pitch * (cpx ? 2 : 1) > 256) return false;
  r.pitchz = pitch_for(nout2);
  r.nseg = (nout2 + mo - 1) / mo;
  const int per128 = (int)(128 / es);
  r.stage_elems = (r.h * r.pitch + per128 - 1) / per128 * per128;
  // the most rows any tile wraps along a periodic axis 1
  int wmax = 0;
  if (a.bc.periodic[1]) {
    const int ntile = (a.vout.n[1] + r.ty - 1) / r.ty;
    for (int t = 0; t < ntile; ++t) {
      const int y0 = 2 * t * r.ty - a.pad0[1];
      const int w = std::min(r.h, std::max(0, -y0) + std::max(0, y0 + r.h - n1));
      wmax = std::max(wmax, w);
    }
  }
  r.wrap_elems = (wmax * n2 + per128 - 1) / per128 * per128;
  r.status = device_status_word();
  p.smem = 128 + (size_t)RR_NS * (r.stage_elems + r.wrap_elems) * es + 2 * (size_t)r.h * r.pitchz * es +
           RR_NS * 8 + 33 * 4;
  return p.smem <= 227 * 1024 && r.status != nullptr;
}

// 4D tensor map of the restriction's input (scalars of complex elements
// counted separately): box = one staged plane, `pitch` elements by h rows.
static bool encode_plane_box(CUtensorMap* map, size_t es, bool cpx, const void* base, const GridView& v, int nbatch,
                             int pitch, int rows) {
  auto enc = tensor_map_encoder();
  if (!enc) return false;
  const size_t ses = cpx ? es / 2 : es;
  const int m = cpx ? 2 : 1;
  cuuint64_t dims[4] = {(cuuint64_t)(v.n[2] * m), (cuuint64_t)v.n[1], (cuuint64_t)v.n[0], (cuuint64_t)nbatch};
  cuuint64_t strides[3] = {(cuuint64_t)(v.s1 * es), (cuuint64_t)(v.s0 * es),
                           (cuuint64_t)(std::max<int64_t>(v.sb, v.s0 * v.n[0]) * es)};
  cuuint32_t box[4] = {(cuuint32_t)(pitch * m), (cuuint32_t)rows, 1, 1};
  cuuint32_t estr[4] = {1, 1, 1, 1};
  CUresult r = enc(map, ses == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4,
                   const_cast<void*>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                   CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

template <typename T, int K, int NT>
static cudaError_t run_restrict_rows(RowsPlan p, int nbatch, cudaStream_t st) {
  TransferArgs& a = p.ra.t;
  CUtensorMap map;
  if (!encode_plane_box(&map, sizeof(T), EltTraits<T>::cpx, a.in, a.vin, nbatch, p.ra.pitch, p.ra.h))
    return cudaErrorInvalidValue;
  dim3 grid(1, (a.vout.n[1] + p.ra.ty - 1) / p.ra.ty, 1);
  choose_chunks(a.vout.n[0], (int64_t)grid.y * nbatch, 2 * K, a.zchunk, a.nchunk);
  grid.z = a.nchunk * nbatch;
  auto kern = restrict_rows_kernel<T, K, NT>;
  static std::once_flag once;
  cudaError_t e = cudaSuccess;
  std::call_once(once, [&] { e = smem_optin(kern, 227 * 1024); });
  if (e != cudaSuccess) return e;
  kern<<<grid, NT, p.smem, st>>>(map, p.ra);
  g_restrict_rows_launches.fetch_add(1);
  return cudaGetLastError();
}

// The row kernel where it applies (complex and float64 data), else false.
template <typename T, int K>
static bool try_restrict_rows(const TransferArgs& a, int nbatch, cudaStream_t st, cudaError_t& e) {
  if constexpr (sizeof(T) < 8) {
    return false;
  } else {
    const int force = g_restrict_force.load();
    if (force == 1) return false;
    RowsPlan p;
    if (force == 3) {
      if (!rows_plan(a, K, sizeof(T), EltTraits<T>::cpx, 192, RowRestrictCfg<192>::MO, p)) return false;
      e = run_restrict_rows<T, K, 192>(p, nbatch, st);
      return true;
    }
    if (!rows_plan(a, K, sizeof(T), EltTraits<T>::cpx, 384, RowRestrictCfg<384>::MO, p)) return false;
    e = run_restrict_rows<T, K, 384>(p, nbatch, st);
    return true;
  }
}

extern "C" int gpw_set_restrict_layout(int k) {
  if (k < 0 || k > 3) return fail(GPW_EINVAL, "restriction layout must be 0-3");
  g_restrict_force.store(k);
  return GPW_OK;
}

// Launches of the row restriction kernel so far in this process.
extern "C" int64_t gpw_restrict_rows_launch_count(void) { return (int64_t)g_restrict_rows_launches.load(); }

template <typename T>
static cudaError_t dispatch_transfer(const TransferArgs& a, int k, bool interp, int nbatch, cudaStream_t st) {
  if (!interp && a.out2 == nullptr) {
    cudaError_t e = cudaSuccess;
    bool done = false;
    switch (k) {
      case 2: done = try_restrict_rows<T, 2>(a, nbatch, st, e); break;
      case 4: done = try_restrict_rows<T, 4>(a, nbatch, st, e); break;
      case 6: done = try_restrict_rows<T, 6>(a, nbatch, st, e); break;
      case 8: done = try_restrict_rows<T, 8>(a, nbatch, st, e); break;
    }
    if (done) return e;
  }
  if (interp) {
    switch (k) {
      case 2: return run_interp<T, 2>(a, nbatch, st);
      case 4: return run_interp<T, 4>(a, nbatch, st);
      case 6: return run_interp<T, 6>(a, nbatch, st);
      case 8: return run_interp<T, 8>(a, nbatch, st);
    }
  } else {
    switch (k) {
      case 2: return run_restrict<T, 2>(a, nbatch, st);
      case 4: return run_restrict<T, 4>(a, nbatch, st);
      case 6: return run_restrict<T, 6>(a, nbatch, st);
      case 8: return run_restrict<T, 8>(a, nbatch, st);
    }
  }
  return cudaErrorInvalidValue;
}

// ------------------------------------------------------------------ coarse levels
// The cluster V-cycle (float32): CG_NCL CTAs per solve in one cluster.
cudaError_t launch_cluster_vcycle(const ClusterArgs& a, size_t smem, int nbatch, cudaStream_t st) {
  // dynamic shared memory up to the per-CTA limit less the kernel's static part
  static std::once_flag once;
  static cudaError_t oe = cudaSuccess;
  static size_t max_dyn = 0;
  std::call_once(once, [] {
    cudaFuncAttributes fa{};
    oe = cudaFuncGetAttributes(&fa, cluster_vcycle_kernel<float>);
    if (oe != cudaSuccess) return;
    max_dyn = 227 * 1024 - fa.sharedSizeBytes;
    oe = cudaFuncSetAttribute(cluster_vcycle_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)max_dyn);
  });
  if (oe != cudaSuccess) return oe;
  if (nbatch < 1 || smem > max_dyn) return cudaErrorInvalidValue;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(nbatch * CG_NCL);
  cfg.blockDim = dim3(CG_CLUSTER_THREADS);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[2];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = CG_NCL;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  attr[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[1].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = pdl_enabled() ? 2 : 1;
  return cudaLaunchKernelEx(&cfg, cluster_vcycle_kernel<float>, a);
}

cudaError_t launch_coarse(int dtype, const CoarseArgs& a, size_t smem, int nbatch, cudaStream_t st) {
  if (a.nl < 1 || a.nl > CG_MAXL || nbatch < 1 || smem > 200 * 1024) return cudaErrorInvalidValue;
  if (dtype == GPW_F64) {
    static std::once_flag once;
    static cudaError_t oe = cudaSuccess;
    std::call_once(once, [] {
      oe = cudaFuncSetAttribute(coarse_vcycle_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                200 * 1024);
    });
    if (oe != cudaSuccess) return oe;
    return launch_pdl(coarse_vcycle_kernel<double>, dim3(nbatch), dim3(CG_THREADS), smem, st, a);
  } else if (dtype == GPW_F32) {
    static std::once_flag once;
    static cudaError_t oe = cudaSuccess;
    std::call_once(once, [] {
      oe = cudaFuncSetAttribute(coarse_vcycle_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                200 * 1024);
    });
    if (oe != cudaSuccess) return oe;
    return launch_pdl(coarse_vcycle_kernel<float>, dim3(nbatch), dim3(CG_THREADS), smem, st, a);
  }
  return cudaErrorInvalidValue;
}

// The vector interpolation needs 16-byte aligned rows / planes / batch
// members of `out` (and `base`) and grids wide enough to fill the vectors.
static bool k2_vec_ok(const TransferArgs& a) {
  auto aligned = [](const void* p) { return ((uintptr_t)p & 15u) == 0; };
  auto view_ok = [](const GridView& v) { return v.s1 % 4 == 0 && v.s0 % 4 == 0 && v.sb % 4 == 0; };
  // a warp covers 128 outputs; rows down to ~32 points still run faster
  // than the scalar kernel's one-point-per-thread form
  if (a.vout.n[2] < 32) return false;
  if (!aligned(a.out) || !view_ok(a.vout)) return false;
  if (a.subtract && (!aligned(a.base) || !view_ok(a.vbase))) return false;
  return true;
}

bool restrict_sweep_ok(const TrDesc& d, int dtype) {
  return d.k == 2 && !d.interpolate && (dtype == GPW_F64 || dtype == GPW_F32);
}

// TMA restriction (restrict_k2_tma_kernel): zero boundaries with pad 0 on
// every axis, 16-byte aligned input with 16-byte strides.
static bool k2r_tma_ok(const TransferArgs& a, size_t es, int nbatch) {
  if (!tensor_map_encoder()) return false;
  for (int c = 0; c < 3; ++c)
    if (a.bc.periodic[c] || a.pad0[c] != 0) return false;
  if (((uintptr_t)a.in & 15u) || (a.vin.s1 * es) % 16 || (a.vin.s0 * es) % 16 ||
      (nbatch > 1 && (a.vin.sb * es) % 16))
    return false;
  return a.vout.n[2] >= 16;
}

// Chunks of a march of n steps over `tiles` tiles: CTAs run in waves of
// `slots`, each chunk pays `warm` extra steps; the count (at most maxc) with
// the least modelled time, waves x steps per chunk.
static int wave_chunks(int n, int64_t tiles, int warm, int64_t slots, int maxc) {
  int best = 1;
  double bestc = 1e300;
  for (int nc = 1; nc <= std::max(1, maxc); ++nc) {
    const int64_t waves = (tiles * nc + slots - 1) / slots;
    const double cost = (double)waves * ((n + nc - 1) / nc + warm);
    if (cost < bestc * (1 - 1e-9)) {
      best = nc;
      bestc = cost;
    }
  }
  return best;
}

template <typename S>
static cudaError_t run_restrict_tma(TransferArgs a, int nbatch, cudaStream_t st) {
  using C = RkCfg<S>;
  static std::once_flag once;
  static cudaError_t oe = cudaSuccess;
  static int per_sm = 1;
  std::call_once(once, [] {
    oe = smem_optin(restrict_k2_tma_kernel<S>, C::smem);
    if (oe == cudaSuccess &&
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, restrict_k2_tma_kernel<S>, RK_TX * RK_TY, C::smem) !=
            cudaSuccess)
      per_sm = 1;
  });
  if (oe != cudaSuccess) return oe;
  auto enc = tensor_map_encoder();
  CUtensorMap map;
  const GridView& v = a.vin;
  const size_t es = sizeof(S);
  cuuint64_t dims[4] = {(cuuint64_t)v.n[2], (cuuint64_t)v.n[1], (cuuint64_t)v.n[0], (cuuint64_t)nbatch};
  cuuint64_t strides[3] = {(cuuint64_t)(v.s1 * es), (cuuint64_t)(v.s0 * es),
                           (cuuint64_t)(std::max<int64_t>(v.sb, v.s0 * v.n[0]) * es)};
  cuuint32_t box[4] = {(cuuint32_t)RK_W, (cuuint32_t)RK_H, 1, 1};
  cuuint32_t estr[4] = {1, 1, 1, 1};
  if (enc(&map, es == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4,
          const_cast<void*>(a.in), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
          CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
    return cudaErrorInvalidValue;
  dim3 grid((a.vout.n[2] + RK_TX - 1) / RK_TX, (a.vout.n[1] + RK_TY - 1) / RK_TY, 1);
  const int64_t tiles = (int64_t)grid.x * grid.y * nbatch;
  const int64_t slots = (int64_t)std::max(1, per_sm) * num_sms();
  a.nchunk = wave_chunks(a.vout.n[0], tiles, 1, slots, a.vout.n[0] / 2);
  a.zchunk = (a.vout.n[0] + a.nchunk - 1) / a.nchunk;
  grid.z = a.nchunk * nbatch;
  cudaError_t le = launch_pdl(restrict_k2_tma_kernel<S>, grid, dim3(RK_TX, RK_TY), C::smem, st, map, a,
                              device_status_word());
  if (le != cudaSuccess) return le;
  return cudaGetLastError();
}

// TMA interpolation-subtraction (interpolate_k2_tma_kernel): zero
// boundaries with pad 1 and skip 1 on every axis, 16-byte aligned coarse
// input, base and output with 16-byte strides.
static bool k2i_tma_ok(const TransferArgs& a, size_t es, int nbatch) {
  if (!tensor_map_encoder() || !a.subtract || !a.base) return false;
  for (int c = 0; c < 3; ++c)
    if (a.bc.periodic[c] || a.pad0[c] != 1 || a.skip0[c] != 1) return false;
  auto ok = [&](const void* p, const GridView& v) {
    return !((uintptr_t)p & 15u) && (v.s1 * es) % 16 == 0 && (v.s0 * es) % 16 == 0 &&
           (nbatch == 1 || (v.sb * es) % 16 == 0);
  };
  if (!ok(a.in, a.vin) || !ok(a.base, a.vbase) || !ok(a.out, a.vout)) return false;
  for (int c = 0; c < 3; ++c)
    if (a.vbase.n[c] != a.vout.n[c]) return false;
  return a.vout.n[2] >= 32;
}

template <typename S>
static cudaError_t run_interp_tma(TransferArgs a, int nbatch, cudaStream_t st) {
  using C = IkCfg<S>;
  static std::once_flag once;
  static cudaError_t oe = cudaSuccess;
  static int per_sm = 1;
  std::call_once(once, [] {
    oe = smem_optin(interpolate_k2_tma_kernel<S>, C::smem);
    if (oe == cudaSuccess && cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                                 &per_sm, interpolate_k2_tma_kernel<S>, IK_TX * IK_NTY, C::smem) != cudaSuccess)
      per_sm = 1;
  });
  if (oe != cudaSuccess) return oe;
  auto enc = tensor_map_encoder();
  const size_t es = sizeof(S);
  auto encode = [&](CUtensorMap* m, const void* base, const GridView& v, int bw, int bh) {
    cuuint64_t dims[4] = {(cuuint64_t)v.n[2], (cuuint64_t)v.n[1], (cuuint64_t)v.n[0], (cuuint64_t)nbatch};
    cuuint64_t strides[3] = {(cuuint64_t)(v.s1 * es), (cuuint64_t)(v.s0 * es),
                             (cuuint64_t)(std::max<int64_t>(v.sb, v.s0 * v.n[0]) * es)};
    cuuint32_t box[4] = {(cuuint32_t)bw, (cuuint32_t)bh, 1, 1};
    cuuint32_t estr[4] = {1, 1, 1, 1};
    return enc(m, es == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4,
               const_cast<void*>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
               CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
  };
  CUtensorMap cmap, bmap;
  if (!encode(&cmap, a.in, a.vin, IK_CW, IK_CH) || !encode(&bmap, a.base, a.vbase, IK_FW, IK_FH))
    return cudaErrorInvalidValue;
  dim3 grid((a.vout.n[2] + IK_FW - 1) / IK_FW, (a.vout.n[1] + IK_FH - 1) / IK_FH, 1);
  const int nm = a.vout.n[0] / 2 + 1;
  const int64_t tiles = (int64_t)grid.x * grid.y * nbatch;
  const int64_t slots = (int64_t)std::max(1, per_sm) * num_sms();
  a.nchunk = wave_chunks(nm, tiles, 1, slots, nm / 2);
  a.zchunk = (nm + a.nchunk - 1) / a.nchunk;
  grid.z = a.nchunk * nbatch;
  cudaError_t le = launch_pdl(interpolate_k2_tma_kernel<S>, grid, dim3(IK_TX, IK_NTY), C::smem, st, cmap, bmap, a,
                              device_status_word());
  if (le != cudaSuccess) return le;
  return cudaGetLastError();
}

// The vector restriction needs zero boundaries and pad 0 along axis 2 (fine
// taps 2 I2 .. 2 I2 + 8 start 16-byte aligned) and aligned input rows.
static bool k2r_vec_ok(const TransferArgs& a) {
  auto aligned = [](const void* p) { return ((uintptr_t)p & 15u) == 0; };
  auto view_ok = [](const GridView& v) { return v.s1 % 4 == 0 && v.s0 % 4 == 0 && v.sb % 4 == 0; };
  // a warp covers 64 outputs: narrower rows leave lanes idle (the scalar
  // kernel's 32-wide rows serve them better)
  if (a.bc.periodic[2] || a.pad0[2] != 0 || a.vout.n[2] < 48) return false;
  if (!aligned(a.in) || !view_ok(a.vin)) return false;
  if (!aligned(a.out) || !view_ok(a.vout)) return false;
  if (a.out2 && !aligned(a.out2)) return false;
  return true;
}

cudaError_t launch_transfer(const TrDesc& d, int dtype, const void* in, const GridView& vin, void* out,
                            const GridView& vout, int nbatch, const Boundary& bc, int subtract,
                            const void* base, const GridView* vbase, const unsigned char* active,
                            cudaStream_t st, const RestrictSweep* sweep) {
  TransferArgs a{};
  a.in = in;
  a.out = out;
  a.vin = vin;
  a.vout = vout;
  a.bc = bc;
  for (int c = 0; c < 3; ++c) {
    a.pad0[c] = d.pad[c][0];
    a.skip0[c] = d.skip[c][0];
  }
  a.active = active;
  a.subtract = subtract;
  a.base = base;
  if (vbase) a.vbase = *vbase;
  const bool interp = d.interpolate != 0;
  if (sweep) {
    if (!restrict_sweep_ok(d, dtype)) return cudaErrorInvalidValue;
    a.out2 = sweep->phi;
    a.w2 = sweep->w;
    a.c02 = sweep->c0;
  }
  if (d.k == 2 && (dtype == GPW_F64 || dtype == GPW_F32) && !interp && k2r_tma_ok(a, elt_size(dtype), nbatch))
    return dtype == GPW_F64 ? run_restrict_tma<double>(a, nbatch, st) : run_restrict_tma<float>(a, nbatch, st);
  if (d.k == 2 && (dtype == GPW_F64 || dtype == GPW_F32) && !interp && k2r_vec_ok(a)) {
    dim3 grid((vout.n[2] + 2 * K2V_TX - 1) / (2 * K2V_TX), (vout.n[1] + K2V_TY - 1) / K2V_TY, 1);
    // ~8 CTAs of 256 threads per SM; chunks of at least 4 output planes
    const int64_t tiles = (int64_t)grid.x * grid.y * nbatch;
    const int64_t want = 8LL * num_sms();
    int64_t nc = std::max<int64_t>(1, (want + tiles - 1) / tiles);
    nc = std::min<int64_t>(nc, std::max(1, vout.n[0] / 4));
    a.zchunk = (int)((vout.n[0] + nc - 1) / nc);
    a.nchunk = (vout.n[0] + a.zchunk - 1) / a.zchunk;
    grid.z = a.nchunk * nbatch;
    const dim3 blk(K2V_TX, K2V_TY);
    if (dtype == GPW_F64) return launch_pdl(restrict_k2_vec_kernel<double>, grid, blk, 0, st, a);
    return launch_pdl(restrict_k2_vec_kernel<float>, grid, blk, 0, st, a);
  }
  if (d.k == 2 && (dtype == GPW_F64 || dtype == GPW_F32) && interp && k2i_tma_ok(a, elt_size(dtype), nbatch))
    return dtype == GPW_F64 ? run_interp_tma<double>(a, nbatch, st) : run_interp_tma<float>(a, nbatch, st);
  if (d.k == 2 && (dtype == GPW_F64 || dtype == GPW_F32) && interp && k2_vec_ok(a)) {
    dim3 grid((vout.n[2] + 4 * K2V_TX - 1) / (4 * K2V_TX), (vout.n[1] + K2V_TY - 1) / K2V_TY, 1);
    // ~8 CTAs of 256 threads per SM; chunks of at least 8 output planes
    const int64_t tiles = (int64_t)grid.x * grid.y * nbatch;
    const int64_t want = 8LL * num_sms();
    int64_t nc = std::max<int64_t>(1, (want + tiles - 1) / tiles);
    nc = std::min<int64_t>(nc, std::max(1, vout.n[0] / 8));
    a.zchunk = (int)((vout.n[0] + nc - 1) / nc);
    a.nchunk = (vout.n[0] + a.zchunk - 1) / a.zchunk;
    grid.z = a.nchunk * nbatch;
    const dim3 blk(K2V_TX, K2V_TY);
    if (dtype == GPW_F64) return launch_pdl(interpolate_k2_vec_kernel<double>, grid, blk, 0, st, a);
    return launch_pdl(interpolate_k2_vec_kernel<float>, grid, blk, 0, st, a);
  }
  if (d.k == 2 && (dtype == GPW_F64 || dtype == GPW_F32)) {
    dim3 grid((vout.n[2] + K2_TX - 1) / K2_TX, (vout.n[1] + K2_TY - 1) / K2_TY, 1);
    choose_chunks(vout.n[0], (int64_t)grid.x * grid.y * nbatch, 4, a.zchunk, a.nchunk);
    grid.z = a.nchunk * nbatch;
    const dim3 blk(K2_TX, K2_TY);
    if (dtype == GPW_F64) {
      if (interp)
        return launch_pdl(interpolate_k2_kernel<double>, grid, blk, 0, st, a);
      else
        return launch_pdl(restrict_k2_kernel<double>, grid, blk, 0, st, a);
    } else {
      if (interp)
        return launch_pdl(interpolate_k2_kernel<float>, grid, blk, 0, st, a);
      else
        return launch_pdl(restrict_k2_kernel<float>, grid, blk, 0, st, a);
    }
    return cudaGetLastError();
  }
  switch (dtype) {
    case GPW_F64: return dispatch_transfer<double>(a, d.k, interp, nbatch, st);
    case GPW_C128: return dispatch_transfer<double2>(a, d.k, interp, nbatch, st);
    case GPW_F32: return dispatch_transfer<float>(a, d.k, interp, nbatch, st);
    case GPW_C64: return dispatch_transfer<float2>(a, d.k, interp, nbatch, st);
  }
  return cudaErrorInvalidValue;
}

// ------------------------------------------------------------------ blas
static dim3 ew_grid(int64_t n) {
  int64_t b = (n + 255) / 256;
  b = std::min<int64_t>(b, 8LL * num_sms());
  return dim3((unsigned)std::max<int64_t>(b, 1));
}

cudaError_t launch_axpy(int dtype, int64_t n, double ar, double ai, const void* x, void* y, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  switch (dtype) {
    case GPW_F64: axpy_real_kernel<double><<<ew_grid(n), 256, 0, st>>>(n, ar, (const double*)x, (double*)y); break;
    case GPW_F32: axpy_real_kernel<float><<<ew_grid(n), 256, 0, st>>>(n, (float)ar, (const float*)x, (float*)y); break;
    case GPW_C128: axpy_cplx_kernel<double2><<<ew_grid(n), 256, 0, st>>>(n, ar, ai, (const double2*)x, (double2*)y); break;
    case GPW_C64: axpy_cplx_kernel<float2><<<ew_grid(n), 256, 0, st>>>(n, ar, ai, (const float2*)x, (float2*)y); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t launch_scal(int dtype, int64_t n, double ar, double ai, void* x, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  switch (dtype) {
    case GPW_F64: scal_real_kernel<double><<<ew_grid(n), 256, 0, st>>>(n, ar, (double*)x); break;
    case GPW_F32: scal_real_kernel<float><<<ew_grid(n), 256, 0, st>>>(n, (float)ar, (float*)x); break;
    case GPW_C128: scal_cplx_kernel<double2><<<ew_grid(n), 256, 0, st>>>(n, ar, ai, (double2*)x); break;
    case GPW_C64: scal_cplx_kernel<float2><<<ew_grid(n), 256, 0, st>>>(n, ar, ai, (float2*)x); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t launch_add_scalar(int dtype, int64_t n, double c, const void* x, void* y, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  switch (dtype) {
    case GPW_F64: add_scalar_kernel<double><<<ew_grid(n), 256, 0, st>>>(n, c, (const double*)x, (double*)y); break;
    case GPW_F32: add_scalar_kernel<float><<<ew_grid(n), 256, 0, st>>>(n, c, (const float*)x, (float*)y); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

int reduce_blocks(int64_t n) {
  int64_t b = (n + 4095) / 4096;
  return (int)std::max<int64_t>(1, std::min<int64_t>(b, 2LL * num_sms()));
}

cudaError_t launch_reduce(int dtype, int op, int64_t nvec, int64_t n, const void* x, const void* y,
                          const GridSum& gs, int nblk, cudaStream_t st, int ny) {
  dim3 grid(nblk, (unsigned)nvec);
  const int ncomp = (op != 1 && is_complex(dtype)) ? 2 : 1;
#define GPW_REDUCE_CASE(T)                                                                              \
  if (op == 0) reduce_kernel<T, 0><<<grid, 256, 0, st>>>(n, (const T*)x, nullptr, gs, ncomp, ny);       \
  else if (op == 1) reduce_kernel<T, 1><<<grid, 256, 0, st>>>(n, (const T*)x, (const T*)y, gs, ncomp, ny); \
  else reduce_kernel<T, 2><<<grid, 256, 0, st>>>(n, (const T*)x, (const T*)y, gs, ncomp, ny);
  switch (dtype) {
    case GPW_F64: GPW_REDUCE_CASE(double) break;
    case GPW_F32: GPW_REDUCE_CASE(float) break;
    case GPW_C128: GPW_REDUCE_CASE(double2) break;
    case GPW_C64: GPW_REDUCE_CASE(float2) break;
    default: return cudaErrorInvalidValue;
  }
#undef GPW_REDUCE_CASE
  return cudaGetLastError();
}

cudaError_t launch_charge_prepare(int64_t nb, int64_t n, const double* rho, double* rho_out, double* phi,
                                  const double* rho_g, const double* phi_g, const double* sums, double dv,
                                  double npts, double maxcharge, int all_periodic, int any_periodic, int zero_phi,
                                  double* q_out, cudaStream_t st) {
  const unsigned gx = (unsigned)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 2LL * num_sms()));
  charge_prepare_kernel<<<dim3(gx, (unsigned)nb), 256, 0, st>>>(n, rho, rho_out, phi, rho_g, phi_g, sums, dv, npts,
                                                                 maxcharge, all_periodic, any_periodic, zero_phi,
                                                                 q_out);
  return cudaGetLastError();
}

cudaError_t launch_charge_finish(int64_t nb, int64_t n, double* phi, const double* phi_g, const double* q,
                                 cudaStream_t st) {
  const unsigned gx = (unsigned)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 2LL * num_sms()));
  charge_finish_kernel<<<dim3(gx, (unsigned)nb), 256, 0, st>>>(n, phi, phi_g, q);
  return cudaGetLastError();
}

cudaError_t launch_copy_box(int dtype, const void* src, const int sn[3], const int so[3], void* dst,
                            const int dn[3], const int dof[3], const int box[3], cudaStream_t st) {
  const int64_t tot = (int64_t)box[0] * box[1] * box[2];
  if (tot <= 0) return cudaSuccess;
  const unsigned g = (unsigned)std::max<int64_t>(1, std::min<int64_t>((tot + 255) / 256, 4LL * num_sms()));
#define GPW_BOX_CASE(T)                                                                                   \
  copy_box_kernel<T><<<g, 256, 0, st>>>((const T*)src, sn[1], sn[2], so[0], so[1], so[2], (T*)dst, dn[1], dn[2], \
                                        dof[0], dof[1], dof[2], box[0], box[1], box[2]);
  switch (dtype) {
    case GPW_F64: GPW_BOX_CASE(double) break;
    case GPW_F32: GPW_BOX_CASE(float) break;
    case GPW_C128: GPW_BOX_CASE(double2) break;
    case GPW_C64: GPW_BOX_CASE(float2) break;
    default: return cudaErrorInvalidValue;
  }
#undef GPW_BOX_CASE
  return cudaGetLastError();
}

cudaError_t launch_mul(int64_t n, const double* x, const double* y, double* out, cudaStream_t st) {
  const unsigned g = (unsigned)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 4LL * num_sms()));
  mul_kernel<<<g, 256, 0, st>>>(n, x, y, out);
  return cudaGetLastError();
}

cudaError_t launch_zero(int dtype, const GridView& v, void* x, int nbatch, const unsigned char* active,
                        cudaStream_t st) {
  const int64_t tot = view_points(v);
  dim3 grid((unsigned)std::max<int64_t>(1, std::min<int64_t>((tot + 255) / 256, 4LL * num_sms())), nbatch);
  switch (dtype) {
    case GPW_F64: zero_kernel<double><<<grid, 256, 0, st>>>(v, (double*)x, active); break;
    case GPW_F32: zero_kernel<float><<<grid, 256, 0, st>>>(v, (float*)x, active); break;
    case GPW_C128: zero_kernel<double2><<<grid, 256, 0, st>>>(v, (double2*)x, active); break;
    case GPW_C64: zero_kernel<float2><<<grid, 256, 0, st>>>(v, (float2*)x, active); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

}  // namespace gpw
