// Launch of the TMA star-stencil kernel (gpw_star_tma.cuh) for one element
// type: tensor maps, axis-0 chunking and the (radius, epilogue, tile
// variant) dispatch.  Included by gpw_tma_f64.cu and gpw_tma_f32.cu, which
// compile the two element types in parallel.
#pragma once
#include <cudaTypedefs.h>

#include <algorithm>
#include <cstring>
#include <mutex>

#include "gpw_internal.h"
#include "gpw_star_tma.cuh"

namespace gpw {

// Every variant is compiled for radius 1 (coarse multigrid levels) and 3
// (the nn=3 Laplacian of level 0); radius 2 uses variant 2 only and radius 4
// variant 1 (128 threads: its float64 accumulators do not fit the register
// share of two 256-thread CTAs per SM).  The 4-point variants (5 - 9) are
// float32 only; variant 10 (48-wide tiles) exists for both.
__host__ __device__ constexpr int tma_default_variant(int R) { return R == 4 ? 1 : 2; }
template <typename S>
__host__ __device__ constexpr bool tma_variant_compiled(int R, int v) {
  if (v >= 5 && v <= 9 && sizeof(S) != 4) return false;
  return (R == 1 || R == 3) ? (v >= 0 && v < TMA_NVARIANT) : v == tma_default_variant(R);
}

// 4D tensor map (axis 2, axis 1, axis 0, batch) over a grid view with a
// box of bw x bh elements of one plane.
inline bool encode_grid_map(CUtensorMap* map, size_t es, const void* base, const GridView& v, int nbatch, int bw,
                            int bh) {
  auto enc = tensor_map_encoder();
  if (!enc) return false;
  cuuint64_t dims[4] = {(cuuint64_t)v.n[2], (cuuint64_t)v.n[1], (cuuint64_t)v.n[0], (cuuint64_t)nbatch};
  cuuint64_t strides[3] = {(cuuint64_t)(v.s1 * es), (cuuint64_t)(v.s0 * es),
                           (cuuint64_t)(std::max<int64_t>(v.sb, v.s0 * v.n[0]) * es)};
  cuuint32_t box[4] = {(cuuint32_t)bw, (cuuint32_t)bh, 1, 1};
  cuuint32_t estr[4] = {1, 1, 1, 1};
  CUresult r = enc(map, es == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4,
                   const_cast<void*>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                   CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

// Axis-0 chunk count from a wave model: CTAs run in waves of `slots`
// (CTAs per SM x SMs); a wave costs its CTAs' planes, each chunk re-reading
// a 2R-plane warm-up.  Chunks keep at least 2R + 2 planes.
inline int tma_model_chunks(int n0, int64_t tiles, int R, int64_t slots) {
  const int maxc = std::max(1, n0 / (2 * R + 2));
  int best = 1;
  double bestc = 1e300;
  for (int nc = 1; nc <= maxc; ++nc) {
    const int64_t ctas = tiles * nc;
    const int64_t waves = (ctas + slots - 1) / slots;
    const double cost = (double)waves * ((n0 + nc - 1) / nc + 2 * R);
    if (cost < bestc * (1 - 1e-9)) {
      best = nc;
      bestc = cost;
    }
  }
  return best;
}

inline int tma_max_chunks(int n0, int R) { return std::max(1, n0 / (2 * R + 2)); }

template <typename S, int R, int MODE, int VAR>
struct TmaKernel {
  using C = TmaCfg<S, R, MODE, VAR>;
  static int slots_per_sm() {
    static int n = -1;
    static std::once_flag once;
    std::call_once(once, [] {
      if (smem_optin_bytes(star_tma_kernel<S, R, MODE, VAR>, C::smem) != cudaSuccess) {
        n = 0;
        return;
      }
      int b = 0;
      if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, star_tma_kernel<S, R, MODE, VAR>, C::NT, C::smem) !=
          cudaSuccess)
        b = 0;
      n = b;
    });
    return n;
  }
  // nchunk == 0: from the wave model; nchunk == TMA_SPLIT: the balanced
  // split over one CTA per resident slot (the model where a norm is
  // summed); other nchunk < 0: the model's count times -nchunk
  static cudaError_t run(const StencilArgs& a0, int nbatch, const StarCoefs& sc, int nchunk, cudaStream_t st) {
    const int spm = slots_per_sm();
    if (spm <= 0) return cudaErrorInvalidConfiguration;
    StencilArgs a = a0;
    CUtensorMap map_in, map_rho, map_aux;
    std::memset(&map_rho, 0, sizeof(map_rho));
    std::memset(&map_aux, 0, sizeof(map_aux));
    if (!encode_grid_map(&map_in, sizeof(S), a.in, a.vin, nbatch, C::W, C::H)) return cudaErrorInvalidValue;
    if (C::HAS_RHO && !encode_grid_map(&map_rho, sizeof(S), a.rho, a.vrho, nbatch, C::TZ, C::TY))
      return cudaErrorInvalidValue;
    if (C::HAS_AUX && !encode_grid_map(&map_aux, 8, a.out2, a.vout, nbatch, C::TZ, C::TY))
      return cudaErrorInvalidValue;
    const GridView& v = a.vout;
    dim3 grid((v.n[2] + C::TZ - 1) / C::TZ, (v.n[1] + C::TY - 1) / C::TY, 1);
    if (C::RR) {  // tiles of CX x CY coarse points
      if (C::CY < 1) return cudaErrorInvalidValue;
      grid = dim3((a.vco.n[2] + C::CX - 1) / C::CX, (a.vco.n[1] + C::CY - 1) / C::CY, 1);
    }
    const int64_t tiles = (int64_t)grid.x * grid.y * nbatch;
    // per-CTA norm partials need whole chunks: the split falls back to the model
    if (nchunk == TMA_SPLIT && a.gsum.partial) nchunk = 0;
    if (nchunk == TMA_SPLIT) {
      // units: planes of a tile column (RESID_RESTRICT: coarse planes); CTAs:
      // the resident slots, but no fewer than 2R + 2 planes of work each
      const int npl = C::RR ? a.vco.n[0] : v.n[0];
      const int64_t units = tiles * npl;
      const int64_t minu = C::RR ? 2 : 2 * R + 2;
      const int64_t nblk = std::max<int64_t>(1, std::min<int64_t>((int64_t)spm * num_sms(), units / minu));
      a.split_gx = (int)grid.x;
      a.split_gy = (int)grid.y;
      a.split_nb = nbatch;
      a.split_npl = npl;
      a.nchunk = 1;
      a.zchunk = v.n[0];
      a.nblk_seg = 0;
      TmaArgs ta{a, device_status_word()};
      const TmaCoefs<S> kc = tma_coefs<S>(sc, R, a.w, a.c0, a.w2);
      return launch_pdl(star_tma_kernel<S, R, MODE, VAR>, dim3((unsigned)nblk, 1, 1), dim3(C::NTX, C::NTY), C::smem,
                        st, map_in, map_rho, map_aux, ta, kc);
    }
    a.split_npl = 0;
    int nc = nchunk > 0 ? nchunk
                        : tma_model_chunks(v.n[0], tiles, R, (int64_t)spm * num_sms()) * std::max(1, -nchunk);
    nc = std::max(1, std::min(nc, tma_max_chunks(v.n[0], R)));
    if (C::RR) nc = std::max(1, std::min(nc, a.vco.n[0] / 2));  // chunks of at least two coarse planes
    a.nchunk = nc;
    a.zchunk = (v.n[0] + nc - 1) / nc;
    grid.z = nc * nbatch;
    a.nblk_seg = grid.x * grid.y * nc;
    TmaArgs ta{a, device_status_word()};
    const TmaCoefs<S> kc = tma_coefs<S>(sc, R, a.w, a.c0, a.w2);
    return launch_pdl(star_tma_kernel<S, R, MODE, VAR>, grid, dim3(C::NTX, C::NTY), C::smem, st, map_in, map_rho,
                      map_aux, ta, kc);
  }
};

template <typename S, int R, int MODE>
cudaError_t tma_run_variant(int var, const StencilArgs& a, int nbatch, const StarCoefs& sc, int nchunk,
                            cudaStream_t st) {
  if (!tma_variant_compiled<S>(R, var)) return cudaErrorInvalidValue;
  if constexpr (R == 1 || R == 3) {
    switch (var) {
      case 0: return TmaKernel<S, R, MODE, 0>::run(a, nbatch, sc, nchunk, st);
      case 1: return TmaKernel<S, R, MODE, 1>::run(a, nbatch, sc, nchunk, st);
      case 2: return TmaKernel<S, R, MODE, 2>::run(a, nbatch, sc, nchunk, st);
      case 3: return TmaKernel<S, R, MODE, 3>::run(a, nbatch, sc, nchunk, st);
      case 4: return TmaKernel<S, R, MODE, 4>::run(a, nbatch, sc, nchunk, st);
      case 10: return TmaKernel<S, R, MODE, 10>::run(a, nbatch, sc, nchunk, st);
    }
    if constexpr (sizeof(S) == 4) {
      switch (var) {
        case 5: return TmaKernel<S, R, MODE, 5>::run(a, nbatch, sc, nchunk, st);
        case 6: return TmaKernel<S, R, MODE, 6>::run(a, nbatch, sc, nchunk, st);
        case 7: return TmaKernel<S, R, MODE, 7>::run(a, nbatch, sc, nchunk, st);
        case 8: return TmaKernel<S, R, MODE, 8>::run(a, nbatch, sc, nchunk, st);
        case 9: return TmaKernel<S, R, MODE, 9>::run(a, nbatch, sc, nchunk, st);
      }
    }
    return cudaErrorInvalidValue;
  } else {
    return TmaKernel<S, R, MODE, tma_default_variant(R)>::run(a, nbatch, sc, nchunk, st);
  }
}

template <typename S, int MODE>
cudaError_t tma_run_radius(int R, int var, const StencilArgs& a, int nbatch, const StarCoefs& sc, int nchunk,
                           cudaStream_t st) {
  switch (R) {
    case 1: return tma_run_variant<S, 1, MODE>(var, a, nbatch, sc, nchunk, st);
    case 2: return tma_run_variant<S, 2, MODE>(var, a, nbatch, sc, nchunk, st);
    case 3: return tma_run_variant<S, 3, MODE>(var, a, nbatch, sc, nchunk, st);
    case 4: return tma_run_variant<S, 4, MODE>(var, a, nbatch, sc, nchunk, st);
  }
  return cudaErrorInvalidValue;
}

}  // namespace gpw
