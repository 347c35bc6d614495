// TMA-fed star stencil for real grids with zero boundaries (sm_100a).
//
// The fast path of the Poisson V-cycle (every relax sweep and residual) and
// of FD applies on 16-byte-pitched real grids.  Compared with the cp.async
// kernel in gpw_stencil.cuh:
//  * one thread issues one 4D TMA tile load (cp.async.bulk.tensor) per plane
//    into a ring of shared-memory stages, completing on an mbarrier; the
//    tensor map's out-of-bounds zero fill *is* the zero boundary condition
//    (neighbour -1 of c/bc.c), so no thread computes a halo address;
//  * each thread owns 2 adjacent axis-2 points x PY axis-1 rows and reads
//    shared memory with 16-byte vector loads;
//  * the axis-0 accumulators rotate by compile-time renaming (the plane loop
//    is unrolled by 2R+1), so no register moves are spent on the march;
//  * the Jacobi centre value is re-read from the ring (R planes behind),
//    instead of a register queue.
// Every mbarrier wait is bounded; on expiry the kernel records
// GPW_ETIMEDOUT in a device status word and finishes without hanging.
#pragma once
#include <cuda.h>

#include "gpw_common.cuh"
#include "gpw_reduce.cuh"
#include "gpw_stencil.cuh"

namespace gpw {

// Tile-shape variants (the launcher's autotuner times them per grid, dtype,
// radius and epilogue and keeps the fastest): NTY thread rows of 32 threads,
// PY axis-1 rows per thread, D planes of TMA prefetch beyond the current one,
// MINB CTAs per SM the register allocation must allow.
template <int NTY_, int PY_, int D_, int MINB_>
struct TmaShape {
  static constexpr int NTY = NTY_, PY = PY_, D = D_, MINB = MINB_;
};
template <int V> struct TmaVariant;
template <> struct TmaVariant<0> { using T = TmaShape<8, 2, 1, 2>; };  // 64 x 16 tile, 1 plane ahead
template <> struct TmaVariant<1> { using T = TmaShape<4, 2, 2, 1>; };  // 64 x 8 tile, 2 planes ahead
template <> struct TmaVariant<2> { using T = TmaShape<8, 2, 2, 2>; };  // 64 x 16 tile, 2 planes ahead
template <> struct TmaVariant<3> { using T = TmaShape<4, 4, 2, 2>; };  // 64 x 16 tile, 4 rows per thread
template <> struct TmaVariant<4> { using T = TmaShape<8, 2, 3, 2>; };  // 64 x 16 tile, 3 planes ahead

constexpr int tma_align128(int b) { return (b + 127) / 128 * 128; }

template <typename S, int R, int MODE, int V = 0>
struct TmaCfg {
  using Sh = typename TmaVariant<V>::T;
  static constexpr int VEC = 2;                        // points per thread along axis 2
  static constexpr int NTX = 32;                       // threads along axis 2
  static constexpr int TZ = NTX * VEC;                 // tile width (points)
  static constexpr int PY = Sh::PY;                    // axis-1 rows per thread
  static constexpr int NTY = Sh::NTY;                  // threads along axis 1
  static constexpr int MINB = Sh::MINB;                // CTAs per SM the registers must allow
  static constexpr int TY = NTY * PY;                  // tile height
  static constexpr int NT = NTX * NTY;                 // threads per CTA
  static constexpr int ALIGN = 16 / (int)sizeof(S);    // elements per 16 bytes
  static constexpr int XL = ((R + ALIGN - 1) / ALIGN) * ALIGN;  // left halo, 16-byte aligned start
  static constexpr int W = TZ + 2 * XL;                // box width (elements)
  static constexpr int H = TY + 2 * R;                 // box height
  static constexpr int D = Sh::D;                      // planes prefetched beyond the current one
  static constexpr int NS = R + D + 1;                 // ring stages
  // per stage: the input plane (with halo), the rho plane of the output
  // completed at that step, and (JACOBI_ADD64) the float64 phi plane
  static constexpr bool HAS_RHO = MODE != MODE_APPLY;
  static constexpr bool HAS_AUX = MODE == MODE_JACOBI_ADD64;
  static constexpr int IN_BYTES = H * W * (int)sizeof(S);
  static constexpr int RHO_BYTES = HAS_RHO ? TY * TZ * (int)sizeof(S) : 0;
  static constexpr int AUX_BYTES = HAS_AUX ? TY * TZ * 8 : 0;
  static constexpr int STAGE_BYTES = tma_align128(IN_BYTES) + tma_align128(RHO_BYTES) + tma_align128(AUX_BYTES);
  static constexpr int RHO_OFF = tma_align128(IN_BYTES);
  static constexpr int AUX_OFF = RHO_OFF + tma_align128(RHO_BYTES);
  static constexpr int NR = 2 * R + 1;
  static constexpr size_t smem = (size_t)NS * STAGE_BYTES + (size_t)NS * 8 + 128;
};

struct TmaArgs {
  StencilArgs s;          // views, rho, w, c0, active, gsum, chunking
  int* status;            // device status word (GPW_ETIMEDOUT on a stuck wait)
};

__device__ __forceinline__ unsigned mbar_u32(const void* p) { return smem_u32(p); }

__device__ __forceinline__ void mbar_init(unsigned bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned bar, unsigned parity) {
  unsigned done;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(done)
      : "r"(bar), "r"(parity)
      : "memory");
  return done != 0;
}
// Bounded wait: ~2^22 polls (each try_wait itself suspends for a while).
__device__ __forceinline__ bool mbar_wait_bounded(unsigned bar, unsigned parity) {
  for (int it = 0; it < (1 << 22); ++it)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}
__device__ __forceinline__ void tma_load_4d(unsigned dst, const CUtensorMap* map, int c0, int c1, int c2, int c3,
                                            unsigned bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4, %5}], [%6];\n" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(bar)
      : "memory");
}

template <typename S> struct Vec2;
template <> struct Vec2<double> { using T = double2; };
template <> struct Vec2<float> { using T = float2; };

template <typename S, int R, int MODE, int VAR>
__global__ void __launch_bounds__(TmaCfg<S, R, MODE, VAR>::NT, TmaCfg<S, R, MODE, VAR>::MINB)
    star_tma_kernel(const __grid_constant__ CUtensorMap tmap, const __grid_constant__ CUtensorMap tmap_rho,
                    const __grid_constant__ CUtensorMap tmap_aux, const TmaArgs ta, const StarCoefs k) {
  using C = TmaCfg<S, R, MODE, VAR>;
  using V = typename Vec2<S>::T;
  constexpr int W = C::W, NS = C::NS, NR = C::NR, PY = C::PY, D = C::D;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  // 128-byte aligned ring of stages (TMA destinations), then the mbarriers;
  // the launch reserves 128 bytes for the alignment shift
  unsigned char* ring = smem_raw + ((128u - (smem_u32(smem_raw) & 127u)) & 127u);
  uint64_t* bars = reinterpret_cast<uint64_t*>(ring + NS * C::STAGE_BYTES);
  __shared__ double red[32];
  const StencilArgs& a = ta.s;

  const int b = blockIdx.z / a.nchunk, chunk = blockIdx.z - b * a.nchunk;
  if (a.active && !a.active[b]) return;
  const int x0 = blockIdx.x * C::TZ, y0 = blockIdx.y * C::TY;
  const int n0 = a.vout.n[0];
  // balanced chunks of axis 0 (lengths differ by at most one plane)
  const int z0 = (int)((int64_t)chunk * n0 / a.nchunk);
  const int z1 = (int)((int64_t)(chunk + 1) * n0 / a.nchunk);
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int tid = tx + C::NTX * ty;
  const int xl = C::XL + C::VEC * tx;     // local column of this thread's first point
  const int x = x0 + C::VEC * tx;         // global axis-2 index of the first point
  const int yb = ty * PY;                 // first local output row
  const bool xin0 = x < a.vout.n[2], xin1 = x + 1 < a.vout.n[2];
  double sumsq = 0.0;
  bool timed_out = false;

  if (tid == 0) {
    for (int i = 0; i < NS; ++i) mbar_init(mbar_u32(&bars[i]), 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  __syncthreads();

  if (z0 < z1) {
    const int pfirst = z0 - R;
    const int nsteps = z1 - z0 + 2 * R;
    // step i brings input plane pfirst + i and, once it completes an output
    // plane o = z0 - 2R + i of this chunk, that plane's rho (and float64 phi)
    auto issue = [&](int i) {
      unsigned char* st = ring + (i % NS) * C::STAGE_BYTES;
      const unsigned bar = mbar_u32(&bars[i % NS]);
      const int o = z0 - 2 * R + i;
      const bool with_out = C::HAS_RHO && o >= z0;
      const unsigned bytes = C::IN_BYTES + (with_out ? C::RHO_BYTES + C::AUX_BYTES : 0);
      mbar_expect_tx(bar, bytes);
      tma_load_4d(smem_u32(st), &tmap, x0 - C::XL, y0 - R, pfirst + i, b, bar);
      if (with_out) {
        tma_load_4d(smem_u32(st + C::RHO_OFF), &tmap_rho, x0, y0, o, b, bar);
        if constexpr (C::HAS_AUX) tma_load_4d(smem_u32(st + C::AUX_OFF), &tmap_aux, x0, y0, o, b, bar);
      }
    };
    if (tid == 0)
      for (int i = 0; i <= D && i < nsteps; ++i) issue(i);
    V acc[PY][NR];
#pragma unroll
    for (int j = 0; j < PY; ++j)
#pragma unroll
      for (int m = 0; m < NR; ++m) acc[j][m] = V{S(0), S(0)};

    for (int sb = 0; sb < nsteps; sb += NR) {
#pragma unroll
      for (int ph = 0; ph < NR; ++ph) {
        const int s = sb + ph;
        if (s >= nsteps) break;
        const int slot = s % NS;
        const unsigned char* stg = ring + slot * C::STAGE_BYTES;
        const S* sl = reinterpret_cast<const S*>(stg);
        const int o = pfirst + s - R;  // output plane completed by this step
        if (!mbar_wait_bounded(mbar_u32(&bars[slot]), (unsigned)((s / NS) & 1))) timed_out = true;

        // column of PY + 2R rows (2 points each) at this thread's columns
        V col[PY + 2 * R];
#pragma unroll
        for (int i = 0; i < PY + 2 * R; ++i) col[i] = *reinterpret_cast<const V*>(sl + (yb + i) * W + xl);
#pragma unroll
        for (int j = 0; j < PY; ++j) {
          const S* row = sl + (yb + j + R) * W + xl;
          // axis-2 neighbours of the two points: row[-XL .. 1 + XL]
          S nb[2 * C::XL + 2];
#pragma unroll
          for (int q = 0; q < C::XL; q += 2) {
            const V lo = *reinterpret_cast<const V*>(row - C::XL + q);
            const V hi = *reinterpret_cast<const V*>(row + 2 + q);
            nb[q] = lo.x;
            nb[q + 1] = lo.y;
            nb[C::XL + 2 + q] = hi.x;
            nb[C::XL + 2 + q + 1] = hi.y;
          }
          const V c = col[j + R];
          nb[C::XL] = c.x;
          nb[C::XL + 1] = c.y;
          constexpr bool sweep = (MODE == MODE_JACOBI || MODE == MODE_JACOBI_ADD64);
          S p0 = sweep ? S(0) : (S)k.cc * c.x;
          S p1 = sweep ? S(0) : (S)k.cc * c.y;
#pragma unroll
          for (int q = 1; q <= R; ++q) {
            p0 = fma((S)k.cy[R + q], col[j + R + q].x, p0);
            p1 = fma((S)k.cy[R + q], col[j + R + q].y, p1);
            p0 = fma((S)k.cy[R - q], col[j + R - q].x, p0);
            p1 = fma((S)k.cy[R - q], col[j + R - q].y, p1);
            p0 = fma((S)k.cz[R + q], nb[C::XL + q], p0);
            p1 = fma((S)k.cz[R + q], nb[C::XL + 1 + q], p1);
            p0 = fma((S)k.cz[R - q], nb[C::XL - q], p0);
            p1 = fma((S)k.cz[R - q], nb[C::XL + 1 - q], p1);
          }
          // scatter along axis 0 (logical slot m receives offset R - m)
#pragma unroll
          for (int m = 0; m < NR; ++m) {
            const int pm = (m + ph) % NR;
            if (m == R) {
              acc[j][pm].x += p0;
              acc[j][pm].y += p1;
            } else {
              acc[j][pm].x = fma((S)k.cx[2 * R - m], c.x, acc[j][pm].x);
              acc[j][pm].y = fma((S)k.cx[2 * R - m], c.y, acc[j][pm].y);
            }
          }
        }
        // output plane o is complete: logical slot 0 = physical ph
        if (o >= z0) {
          const S* osl = reinterpret_cast<const S*>(ring + ((s + NS - R) % NS) * C::STAGE_BYTES);
          const S* rsl = reinterpret_cast<const S*>(stg + C::RHO_OFF);
          const double* asl = reinterpret_cast<const double*>(stg + C::AUX_OFF);
#pragma unroll
          for (int j = 0; j < PY; ++j) {
            const int y = y0 + yb + j;
            if (y < a.vout.n[1] && xin0) {
              V av = acc[j][ph];
              V res;
              V rho = V{S(0), S(0)};
              if constexpr (C::HAS_RHO) rho = *reinterpret_cast<const V*>(rsl + (yb + j) * C::TZ + C::VEC * tx);
              const int64_t oidx =
                  (int64_t)b * a.vout.sb + (int64_t)o * a.vout.s0 + (int64_t)y * a.vout.s1 + x;
              if constexpr (MODE == MODE_APPLY) {
                res = av;
              } else if constexpr (MODE == MODE_RESIDUAL || MODE == MODE_RESID_DC) {
                res.x = av.x - rho.x;
                res.y = av.y - rho.y;
                sumsq += (double)res.x * res.x + (xin1 ? (double)res.y * res.y : 0.0);
              } else {
                const V cur = *reinterpret_cast<const V*>(osl + (yb + j + R) * W + xl);
                const S w = (S)a.w, wc = w / (S)a.c0;
                res.x = (S(1) - w) * cur.x + wc * (rho.x - av.x);
                res.y = (S(1) - w) * cur.y + wc * (rho.y - av.y);
              }
              if constexpr (MODE == MODE_RESID_DC) {
                // float32 defect and first inner Jacobi iterate from zero
                const float2 rhs = make_float2((float)(-res.x), (float)(-res.y));
                const float wc = (float)a.w2 / (float)a.c0;
                const float2 e1 = make_float2(wc * rhs.x, wc * rhs.y);
                float* rp = static_cast<float*>(a.out) + oidx;
                float* ep = static_cast<float*>(a.out2) + oidx;
                if (xin1) {
                  *reinterpret_cast<float2*>(rp) = rhs;
                  *reinterpret_cast<float2*>(ep) = e1;
                } else {
                  rp[0] = rhs.x;
                  ep[0] = e1.x;
                }
              } else if constexpr (MODE == MODE_JACOBI_ADD64) {
                // phi64 += e (the inner correction), e never stored
                double* pp = static_cast<double*>(a.out2) + oidx;
                double2 pv = *reinterpret_cast<const double2*>(asl + (yb + j) * C::TZ + C::VEC * tx);
                pv.x += (double)res.x;
                pv.y += (double)res.y;
                if (xin1)
                  *reinterpret_cast<double2*>(pp) = pv;
                else
                  pp[0] = pv.x;
              } else if (MODE != MODE_RESIDUAL || a.out) {
                S* op = static_cast<S*>(a.out) + oidx;
                if (xin1)
                  *reinterpret_cast<V*>(op) = res;
                else
                  op[0] = res.x;
              }
            }
          }
        }
#pragma unroll
        for (int j = 0; j < PY; ++j) acc[j][ph] = V{S(0), S(0)};
        __syncthreads();  // every thread is done with plane s - R (its slot is refilled next)
        if (tid == 0 && s + D + 1 < nsteps) issue(s + D + 1);
      }
    }
  }
  if (timed_out && ta.status) atomicExch(ta.status, GPW_ETIMEDOUT);
  if constexpr (MODE == MODE_RESIDUAL || MODE == MODE_RESID_DC) {
    if (a.gsum.partial) {
      double tot = block_sum(sumsq, red);
      const int blk = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * chunk);
      grid_sum_finish(a.gsum, b, blk, a.nblk_seg, tot, red);
    }
  }
}

}  // namespace gpw
