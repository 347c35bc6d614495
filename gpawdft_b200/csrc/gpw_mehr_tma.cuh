// The Mehrstellen Laplacian A (mehrstellen_kernel's arithmetic and thread
// layout) on real zero-boundary grids, with its planes staged by TMA: one 4D
// box per plane (the tile's 64 x 16 outputs with a one-point halo, from the
// 16-byte aligned column x0 - XL) into a ring of shared-memory stages that
// complete on mbarriers, the tensor map's out-of-bounds zero fill being the
// zero boundary.  Per-cell cp.async staging held the kernel at ~1.5 TB/s;
// the bulk copy frees the load pipe for the stencil's shared-memory reads.
// Every wait is bounded (GPW_ETIMEDOUT in the status word).  Included by
// gpw_tma_f64.cu and gpw_tma_f32.cu.
#pragma once
#include "gpw_star_tma.cuh"
#include "gpw_tma_launch.cuh"

namespace gpw {

template <typename S>
struct MehrTmaCfg {
  static constexpr int NTX = MehrCfg::NTX, NTY = MehrCfg::NTY, NT = MehrCfg::NT;
  static constexpr int TZ = MehrCfg::TZ, TY = MehrCfg::TY;
  static constexpr int XL = 16 / (int)sizeof(S);  // left halo: the box starts 16-byte aligned
  static constexpr int W = TZ + 2 * XL, H = TY + 2;
  static constexpr int D = 2;                      // planes in flight beyond the three in use
  static constexpr int NS = 3 + D;
  static constexpr int STAGE_BYTES = tma_align128(H * W * (int)sizeof(S));
  static constexpr size_t smem = (size_t)NS * STAGE_BYTES + (size_t)NS * 8 + 128;
};

template <typename S>
struct MehrCoefs {
  S cf[MEHR_NC];  // the table's coefficients in its order, rounded once on the host
};

template <typename S, int MODE>
__global__ void __launch_bounds__(MehrCfg::NT, 2)
    mehr_tma_kernel(const __grid_constant__ CUtensorMap tmap, const TmaArgs ta, const MehrCoefs<S> k) {
  using C = MehrTmaCfg<S>;
  constexpr int W = C::W, NS = C::NS;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  unsigned char* ring = smem_raw + ((128u - (smem_u32(smem_raw) & 127u)) & 127u);
  uint64_t* bars = reinterpret_cast<uint64_t*>(ring + NS * C::STAGE_BYTES);
  __shared__ double red[32];
  const StencilArgs& a = ta.s;
  pdl_wait();
  const int b = blockIdx.z / a.nchunk, chunk = blockIdx.z - b * a.nchunk;
  if (a.active && !a.active[b]) return;
  const int x0 = blockIdx.x * C::TZ, y0 = blockIdx.y * C::TY;
  const int n0 = a.vout.n[0];
  const int z0 = chunk * a.zchunk;
  const int z1 = min(n0, z0 + a.zchunk);
  const int tx = threadIdx.x, ty = threadIdx.y, tid = tx + C::NTX * ty;
  double sumsq = 0.0;
  bool timed_out = false;
  if (tid == 0) {
    for (int i = 0; i < NS; ++i) mbar_init(mbar_u32(&bars[i]), 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  __syncthreads();
  // outputs (rows y0 + 2 ty + i, columns x0 + 2 tx + j)
  int64_t obase[2][2], rbase[2][2];
  unsigned omask = 0;
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      const int y = y0 + 2 * ty + i, x = x0 + 2 * tx + j;
      if (y < a.vout.n[1] && x < a.vout.n[2]) omask |= 1u << (2 * i + j);
      obase[i][j] = (int64_t)b * a.vout.sb + (int64_t)y * a.vout.s1 + x;
      rbase[i][j] = (int64_t)b * a.vrho.sb + (int64_t)y * a.vrho.s1 + x;
    }
  if (z0 < z1) {
    // step s stages plane z0 - 1 + s; at s >= 2 it completes output plane
    // z0 + s - 2 from the stages of steps s - 2, s - 1, s
    const int nsteps = z1 - z0 + 2;
    auto issue = [&](int s) {
      const unsigned bar = mbar_u32(&bars[s % NS]);
      mbar_expect_tx(bar, (unsigned)(C::H * W * (int)sizeof(S)));
      tma_load_4d(smem_u32(ring + (s % NS) * C::STAGE_BYTES), &tmap, x0 - C::XL, y0 - 1, z0 - 1 + s, b, bar);
    };
    if (tid == 0)
      for (int s = 0; s < NS && s < nsteps; ++s) issue(s);
    const int cell = (2 * ty + 1) * W + 2 * tx + C::XL;  // output (0, 0) within a stage
    for (int s = 0; s < nsteps; ++s) {
      if (!mbar_wait_bounded(mbar_u32(&bars[s % NS]), (unsigned)((s / NS) & 1))) timed_out = true;
      if (s >= 2) {
        const int o = z0 + s - 2;
        const S* pm = reinterpret_cast<const S*>(ring + ((s - 2) % NS) * C::STAGE_BYTES) + cell;
        const S* pc = reinterpret_cast<const S*>(ring + ((s - 1) % NS) * C::STAGE_BYTES) + cell;
        const S* pp = reinterpret_cast<const S*>(ring + (s % NS) * C::STAGE_BYTES) + cell;
        S c0[4][4], cm[2][4], cp[2][4], cmr[2][2], cpr[2][2];
#pragma unroll
        for (int r = 0; r < 4; ++r)
#pragma unroll
          for (int e = 0; e < 4; ++e) c0[r][e] = pc[(r - 1) * W + e - 1];
#pragma unroll
        for (int r = 0; r < 2; ++r)
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            cm[r][e] = pm[r * W + e - 1];
            cp[r][e] = pp[r * W + e - 1];
          }
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          cmr[0][e] = pm[-W + e];
          cmr[1][e] = pm[2 * W + e];
          cpr[0][e] = pp[-W + e];
          cpr[1][e] = pp[2 * W + e];
        }
#pragma unroll
        for (int i = 0; i < 2; ++i) {
#pragma unroll
          for (int j = 0; j < 2; ++j) {
            const S v[MEHR_NC] = {c0[i + 1][j + 1],
                                  cm[i][j + 1],     cp[i][j + 1],
                                  c0[i][j + 1],     c0[i + 2][j + 1],
                                  c0[i + 1][j],     c0[i + 1][j + 2],
                                  c0[i][j],         c0[i][j + 2],     c0[i + 2][j],     c0[i + 2][j + 2],
                                  cm[i][j],         cm[i][j + 2],     cp[i][j],         cp[i][j + 2],
                                  i == 0 ? cmr[0][j] : cm[0][j + 1], i == 0 ? cm[1][j + 1] : cmr[1][j],
                                  i == 0 ? cpr[0][j] : cp[0][j + 1], i == 0 ? cp[1][j + 1] : cpr[1][j]};
            S acc = S(0);
#pragma unroll
            for (int c = (MODE == MODE_JACOBI) ? 1 : 0; c < MEHR_NC; ++c) acc = mac_rn(k.cf[c], v[c], acc);
            if (!((omask >> (2 * i + j)) & 1u)) continue;
            const S cur = v[0];
            const int64_t oi = obase[i][j] + (int64_t)o * a.vout.s0;
            if constexpr (MODE == MODE_APPLY) {
              if (a.pot) acc = fmac(static_cast<const S*>(a.pot)[oi - (int64_t)b * a.vout.sb], cur, acc);
              if (a.aux) acc = fmac((S)a.aux_scale, static_cast<const S*>(a.aux)[oi], acc);
              static_cast<S*>(a.out)[oi] = acc;
            } else {
              const S rho = static_cast<const S*>(a.rho)[rbase[i][j] + (int64_t)o * a.vrho.s0];
              if constexpr (MODE == MODE_RESIDUAL) {
                const S d = acc - rho;
                if (a.out) static_cast<S*>(a.out)[oi] = d;
                sumsq += norm2(d);
              } else {
                static_cast<S*>(a.out)[oi] = jacobi_rn((S)a.w, cur, rho, acc, (S)a.c0);
              }
            }
          }
        }
      }
      __syncthreads();  // every thread is done with the stage of step s - 2 (refilled next)
      if (tid == 0 && s >= 2 && s - 2 + NS < nsteps) issue(s - 2 + NS);
    }
  }
  pdl_trigger();
  if (timed_out && ta.status) atomicExch(ta.status, GPW_ETIMEDOUT);
  if constexpr (MODE == MODE_RESIDUAL) {
    if (a.gsum.partial) {
      double tot = block_sum(sumsq, red);
      const int blk = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * chunk);
      grid_sum_finish(a.gsum, b, blk, a.nblk_seg, tot, red);
    }
  }
}

// Launch on arguments whose chunking (nchunk, zchunk, nblk_seg) the caller set
// for a 64 x 16 tile grid.
template <typename S, int MODE>
cudaError_t mehr_tma_run(const StencilArgs& a, int nbatch, const GeneralCoefs& gc, cudaStream_t st) {
  using C = MehrTmaCfg<S>;
  static std::once_flag once;
  static cudaError_t oe = cudaSuccess;
  std::call_once(once, [] { oe = smem_optin_bytes(mehr_tma_kernel<S, MODE>, C::smem); });
  if (oe != cudaSuccess) return oe;
  CUtensorMap map;
  if (!encode_grid_map(&map, sizeof(S), a.in, a.vin, nbatch, C::W, C::H)) return cudaErrorInvalidValue;
  MehrCoefs<S> k;
  for (int c = 0; c < MEHR_NC; ++c) k.cf[c] = (S)gc.coef[c];
  const GridView& v = a.vout;
  const dim3 grid((v.n[2] + C::TZ - 1) / C::TZ, (v.n[1] + C::TY - 1) / C::TY, a.nchunk * nbatch);
  TmaArgs ta{a, device_status_word()};
  return launch_pdl(mehr_tma_kernel<S, MODE>, grid, dim3(C::NTX, C::NTY), C::smem, st, map, ta, k);
}

template <typename S>
cudaError_t mehr_tma_mode(int mode, const StencilArgs& a, int nbatch, const GeneralCoefs& gc, cudaStream_t st) {
  switch (mode) {
    case MODE_APPLY: return mehr_tma_run<S, MODE_APPLY>(a, nbatch, gc, st);
    case MODE_RESIDUAL: return mehr_tma_run<S, MODE_RESIDUAL>(a, nbatch, gc, st);
    case MODE_JACOBI: return mehr_tma_run<S, MODE_JACOBI>(a, nbatch, gc, st);
  }
  return cudaErrorInvalidValue;
}

}  // namespace gpw
