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
#include "gpw_transfer.cuh"

namespace gpw {

// Tile-shape variants (the launcher's autotuner times them per grid, dtype,
// radius and epilogue and keeps the fastest): NTX threads along axis 2 with
// VEC adjacent points each, NTY thread rows, PY axis-1 rows per thread, D
// planes of TMA prefetch beyond the current one, MINB CTAs per SM the
// register allocation must allow.
template <int NTX_, int VEC_, int NTY_, int PY_, int D_, int MINB_>
struct TmaShape {
  static constexpr int NTX = NTX_, VEC = VEC_, NTY = NTY_, PY = PY_, D = D_, MINB = MINB_;
};
template <int V> struct TmaVariant;
template <> struct TmaVariant<0> { using T = TmaShape<32, 2, 8, 2, 1, 2>; };  // 64 x 16 tile, 1 plane ahead
template <> struct TmaVariant<1> { using T = TmaShape<32, 2, 4, 2, 2, 1>; };  // 64 x 8 tile, 2 planes ahead
template <> struct TmaVariant<2> { using T = TmaShape<32, 2, 8, 2, 2, 2>; };  // 64 x 16 tile, 2 planes ahead
template <> struct TmaVariant<3> { using T = TmaShape<32, 2, 4, 4, 2, 2>; };  // 64 x 16 tile, 4 rows per thread
template <> struct TmaVariant<4> { using T = TmaShape<32, 2, 8, 2, 3, 2>; };  // 64 x 16 tile, 3 planes ahead
// float32 only: 4 points per thread (16-byte shared-memory reads)
template <> struct TmaVariant<5> { using T = TmaShape<16, 4, 8, 2, 2, 3>; };  // 64 x 16 tile, 128 threads
template <> struct TmaVariant<6> { using T = TmaShape<16, 4, 8, 1, 2, 4>; };  // 64 x 8 tile, 128 threads
template <> struct TmaVariant<7> { using T = TmaShape<16, 4, 8, 2, 3, 3>; };  // 64 x 16 tile, 3 planes ahead
template <> struct TmaVariant<8> { using T = TmaShape<16, 4, 16, 1, 2, 2>; };  // 64 x 16 tile, 256 threads
// 68 x 16 tile: with the residual restricted in-kernel, 32 coarse columns a
// tile at a 64-column stride
template <> struct TmaVariant<9> { using T = TmaShape<17, 4, 8, 2, 2, 3>; };
// both element types: 48 x 16 tile (192 threads), whole rows of 48-point
// grids with no idle columns
template <> struct TmaVariant<10> { using T = TmaShape<24, 2, 8, 2, 2, 2>; };

// VEC elements of S moved as one vector load / store
template <typename S, int N> struct VecT;
template <> struct VecT<float, 2> { using T = float2; };
template <> struct VecT<float, 4> { using T = float4; };
template <> struct VecT<double, 2> { using T = double2; };
template <typename S, int N>
struct Pack {
  S v[N];
};
template <typename S, int N>
__device__ __forceinline__ Pack<S, N> ldv(const S* p) {
  const typename VecT<S, N>::T t = *reinterpret_cast<const typename VecT<S, N>::T*>(p);
  Pack<S, N> r;
  if constexpr (N == 2) {
    r.v[0] = t.x;
    r.v[1] = t.y;
  } else {
    r.v[0] = t.x;
    r.v[1] = t.y;
    r.v[2] = t.z;
    r.v[3] = t.w;
  }
  return r;
}
template <typename S, int N>
__device__ __forceinline__ void stv(S* p, const Pack<S, N>& r) {
  typename VecT<S, N>::T t;
  if constexpr (N == 2) {
    t.x = r.v[0];
    t.y = r.v[1];
  } else {
    t.x = r.v[0];
    t.y = r.v[1];
    t.z = r.v[2];
    t.w = r.v[3];
  }
  *reinterpret_cast<typename VecT<S, N>::T*>(p) = t;
}
// the first `n` of N elements (n < N): scalar stores
template <typename S, int N>
__device__ __forceinline__ void stv_part(S* p, const Pack<S, N>& r, int n) {
#pragma unroll
  for (int e = 0; e < N; ++e)
    if (e < n) p[e] = r.v[e];
}

constexpr int tma_align128(int b) { return (b + 127) / 128 * 128; }

template <typename S, int R, int MODE, int V = 0>
struct TmaCfg {
  using Sh = typename TmaVariant<V>::T;
  static constexpr int VEC = Sh::VEC;                  // points per thread along axis 2
  static constexpr int NTX = Sh::NTX;                  // threads along axis 2
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
  // ring stages: a Jacobi sweep re-reads its centre value R planes behind;
  // the other epilogues read each plane once, at arrival
  static constexpr bool KEEP_CENTRE = MODE == MODE_JACOBI || MODE == MODE_JACOBI_ADD64 || MODE == MODE_JACOBI_SCALED_IN;
  static constexpr int NS = KEEP_CENTRE ? R + D + 1 : D + 1;
  // per stage: the input plane (with halo), the rho plane of the output
  // completed at that step, and (JACOBI_ADD64) the float64 phi plane
  static constexpr bool HAS_RHO =
      MODE != MODE_APPLY && MODE != MODE_APPLY_EPI && MODE != MODE_JACOBI_SCALED_IN;  // (scaled: rho is the input)
  static constexpr bool HAS_AUX = MODE == MODE_JACOBI_ADD64;
  static constexpr int IN_BYTES = H * W * (int)sizeof(S);
  static constexpr int RHO_BYTES = HAS_RHO ? TY * TZ * (int)sizeof(S) : 0;
  static constexpr int AUX_BYTES = HAS_AUX ? TY * TZ * 8 : 0;
  static constexpr int STAGE_BYTES = tma_align128(IN_BYTES) + tma_align128(RHO_BYTES) + tma_align128(AUX_BYTES);
  static constexpr int RHO_OFF = tma_align128(IN_BYTES);
  static constexpr int AUX_OFF = RHO_OFF + tma_align128(RHO_BYTES);
  static constexpr int NR = 2 * R + 1;
  // RESID_RESTRICT: the residual plane of the tile, and the coarse points a
  // tile restricts (centres 2I + 1 in the tile's first TZ - 4 columns and
  // TY - 2 rows; tiles advance by those and overlap by the rest)
  static constexpr bool RR = MODE == MODE_RESID_RESTRICT;
  static constexpr int CX = (TZ - 4) / 2, CY = (TY - 2) / 2;
  static constexpr int RT_BYTES = RR ? TY * TZ * (int)sizeof(S) : 0;
  static constexpr size_t smem = (size_t)NS * STAGE_BYTES + (size_t)NS * 8 + (size_t)RT_BYTES + 128;
};

// Coefficients and relaxation weights in the kernel's element type, rounded
// once on the host with the same roundings a per-use conversion would make
// (the kernel reads them as constant-bank operands).
template <typename S>
struct TmaCoefs {
  S cx[9], cy[9], cz[9];  // per-axis coefficients indexed offset + R (R <= 4)
  S cc;                   // total centre coefficient
  S w1, wc;               // Jacobi: 1 - w and w / c0
  float wc2;              // RESID_DC: the float32 first sweep's w2 / c0
};

template <typename S>
inline TmaCoefs<S> tma_coefs(const StarCoefs& sc, int R, double w, double c0, double w2) {
  TmaCoefs<S> t{};
  for (int i = 0; i <= 2 * R && i < 9; ++i) {
    t.cx[i] = (S)sc.cx[i];
    t.cy[i] = (S)sc.cy[i];
    t.cz[i] = (S)sc.cz[i];
  }
  t.cc = (S)sc.cc;
  const S ws = (S)w;
  t.w1 = S(1) - ws;
  t.wc = c0 != 0.0 ? ws / (S)c0 : S(0);
  t.wc2 = c0 != 0.0 ? (float)w2 / (float)c0 : 0.0f;
  return t;
}

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

template <typename S, int R, int MODE, int VAR>
__global__ void __launch_bounds__(TmaCfg<S, R, MODE, VAR>::NT, TmaCfg<S, R, MODE, VAR>::MINB)
    star_tma_kernel(const __grid_constant__ CUtensorMap tmap, const __grid_constant__ CUtensorMap tmap_rho,
                    const __grid_constant__ CUtensorMap tmap_aux, const TmaArgs ta, const TmaCoefs<S> k) {
  using C = TmaCfg<S, R, MODE, VAR>;
  constexpr int W = C::W, NS = C::NS, NR = C::NR, PY = C::PY, D = C::D, VEC = C::VEC, XL = C::XL;
  using P = Pack<S, VEC>;
  static_assert(XL % VEC == 0, "halo loads are whole vectors");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  // 128-byte aligned ring of stages (TMA destinations), then the mbarriers;
  // the launch reserves 128 bytes for the alignment shift
  unsigned char* ring = smem_raw + ((128u - (smem_u32(smem_raw) & 127u)) & 127u);
  S* rtile = reinterpret_cast<S*>(ring + NS * C::STAGE_BYTES);  // RESID_RESTRICT (128-byte aligned)
  uint64_t* bars = reinterpret_cast<uint64_t*>(ring + NS * C::STAGE_BYTES + C::RT_BYTES);
  __shared__ double red[32];
  const StencilArgs& a = ta.s;
  pdl_wait();  // the predecessor's results (and the active mask) are visible from here

  const int n0 = a.vout.n[0];
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int tid = tx + C::NTX * ty;
  const int xl = XL + VEC * tx;       // local column of this thread's first point
  const int yb = ty * PY;             // first local output row
  double sumsq = 0.0;
  bool timed_out = false;

  if (tid == 0) {
    for (int i = 0; i < NS; ++i) mbar_init(mbar_u32(&bars[i]), 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  __syncthreads();

  // Work: the CTA's chunk (one segment), or under the balanced split a
  // contiguous range of (tile column, plane) units that may span several
  // columns, each column's part one segment.  The ring's stage and phase
  // run on across segments (gbase: steps of the earlier segments).
  const bool split = a.split_npl > 0;
  const int chunk = split ? 0 : (int)(blockIdx.z % a.nchunk);
  const int bchunk = split ? 0 : (int)(blockIdx.z / a.nchunk);  // the chunk's batch member
  if (!split && a.active && !a.active[bchunk]) return;
  int64_t wu = 0, wend = 1;
  if (split) {
    const int64_t T = (int64_t)a.split_gx * a.split_gy * (int64_t)a.split_nb * a.split_npl;
    wu = (int64_t)blockIdx.x * T / gridDim.x;
    wend = (int64_t)(blockIdx.x + 1) * T / gridDim.x;
  }
  int gbase = 0;
  while (wu < wend) {
    int b, bx, by, z0, z1;
    if (split) {
      const int64_t col = wu / a.split_npl;
      const int c0 = (int)(wu - col * a.split_npl);
      const int64_t rest = (int64_t)c0 + (wend - wu);
      const int c1 = rest < a.split_npl ? (int)rest : a.split_npl;
      wu += c1 - c0;
      const int ntile = a.split_gx * a.split_gy;
      b = (int)(col / ntile);
      const int tile = (int)(col - (int64_t)b * ntile);
      by = tile / a.split_gx;
      bx = tile - by * a.split_gx;
      if constexpr (C::RR) {
        z0 = 2 * c0;
        z1 = min(n0, 2 * c1 + 1);
      } else {
        z0 = c0;
        z1 = c1;
      }
    } else {
      wu = wend;
      b = bchunk;
      bx = blockIdx.x;
      by = blockIdx.y;
      // balanced chunks of axis 0 (lengths differ by at most one plane); for
      // RESID_RESTRICT chunks of coarse planes [C0, C1), i.e. fine planes
      // 2 C0 .. 2 C1 (consecutive chunks share one fine plane)
      if constexpr (C::RR) {
        const int nc0 = a.vco.n[0];
        z0 = 2 * (int)((int64_t)chunk * nc0 / a.nchunk);
        z1 = min(n0, 2 * (int)((int64_t)(chunk + 1) * nc0 / a.nchunk) + 1);
      } else {
        z0 = (int)((int64_t)chunk * n0 / a.nchunk);
        z1 = (int)((int64_t)(chunk + 1) * n0 / a.nchunk);
      }
    }
    if (a.active && !a.active[b]) continue;
    const int x0 = bx * (C::RR ? 2 * C::CX : C::TZ), y0 = by * (C::RR ? 2 * C::CY : C::TY);
    const int x = x0 + VEC * tx;        // global axis-2 index of the first point
    const int nx = min(VEC, a.vout.n[2] - x);  // this thread's points inside the grid (<= 0: none)

    if (z0 < z1) {
      const int pfirst = z0 - R;
      const int nsteps = z1 - z0 + 2 * R;
      // step i brings input plane pfirst + i and, once it completes an output
      // plane o = z0 - 2R + i of this chunk, that plane's rho (and float64 phi)
      auto issue = [&](int i) {
        unsigned char* st = ring + ((gbase + i) % NS) * C::STAGE_BYTES;
        const unsigned bar = mbar_u32(&bars[(gbase + i) % NS]);
        const int o = z0 - 2 * R + i;
        const bool with_out = C::HAS_RHO && o >= z0;
        const unsigned bytes = C::IN_BYTES + (with_out ? C::RHO_BYTES + C::AUX_BYTES : 0);
        mbar_expect_tx(bar, bytes);
        tma_load_4d(smem_u32(st), &tmap, x0 - XL, y0 - R, pfirst + i, b, bar);
        if (with_out) {
          tma_load_4d(smem_u32(st + C::RHO_OFF), &tmap_rho, x0, y0, o, b, bar);
          if constexpr (C::HAS_AUX) tma_load_4d(smem_u32(st + C::AUX_OFF), &tmap_aux, x0, y0, o, b, bar);
        }
      };
      if (tid == 0)
        for (int i = 0; i <= D && i < nsteps; ++i) issue(i);
      P acc[PY][NR];
#pragma unroll
      for (int j = 0; j < PY; ++j)
#pragma unroll
        for (int m = 0; m < NR; ++m)
#pragma unroll
          for (int e = 0; e < VEC; ++e) acc[j][m].v[e] = S(0);
      // RESID_RESTRICT: this thread's coarse points of the tile (tid + u NT)
      // and the in-plane restricted values of their last two fine planes
      constexpr int RK = C::RR ? (C::CX * C::CY + C::NT - 1) / C::NT : 1;
      S rq0[RK], rq1[RK];
#pragma unroll
      for (int u = 0; u < RK; ++u) rq0[u] = rq1[u] = S(0);

      for (int sb = 0; sb < nsteps; sb += NR) {
#pragma unroll
        for (int ph = 0; ph < NR; ++ph) {
          const int s = sb + ph;
          if (s >= nsteps) break;
          const int slot = (gbase + s) % NS;
          const unsigned char* stg = ring + slot * C::STAGE_BYTES;
          const S* sl = reinterpret_cast<const S*>(stg);
          const int o = pfirst + s - R;  // output plane completed by this step
          if (!mbar_wait_bounded(mbar_u32(&bars[slot]), (unsigned)(((gbase + s) / NS) & 1))) timed_out = true;

          // column of PY + 2R rows (VEC points each) at this thread's columns
          P col[PY + 2 * R];
#pragma unroll
          for (int i = 0; i < PY + 2 * R; ++i) col[i] = ldv<S, VEC>(sl + (yb + i) * W + xl);
#pragma unroll
          for (int j = 0; j < PY; ++j) {
            const S* row = sl + (yb + j + R) * W + xl;
            // axis-2 neighbours of the VEC points: row[-XL .. VEC - 1 + XL]
            S nb[2 * XL + VEC];
#pragma unroll
            for (int q = 0; q < XL; q += VEC) {
              const P lo = ldv<S, VEC>(row - XL + q);
              const P hi = ldv<S, VEC>(row + VEC + q);
#pragma unroll
              for (int e = 0; e < VEC; ++e) {
                nb[q + e] = lo.v[e];
                nb[XL + VEC + q + e] = hi.v[e];
              }
            }
            const P c = col[j + R];
#pragma unroll
            for (int e = 0; e < VEC; ++e) nb[XL + e] = c.v[e];
            constexpr bool sweep = (MODE == MODE_JACOBI || MODE == MODE_JACOBI_ADD64 || MODE == MODE_JACOBI_SCALED_IN);
            // the in-plane sum in two independent chains (centre + axis 1,
            // axis 2) joined at the end: half the dependent-FMA latency
            S p[VEC], pz[VEC];
#pragma unroll
            for (int e = 0; e < VEC; ++e) {
              p[e] = sweep ? S(0) : k.cc * c.v[e];
              pz[e] = S(0);
            }
#pragma unroll
            for (int q = 1; q <= R; ++q) {
#pragma unroll
              for (int e = 0; e < VEC; ++e) {
                p[e] = fma(k.cy[R + q], col[j + R + q].v[e], p[e]);
                p[e] = fma(k.cy[R - q], col[j + R - q].v[e], p[e]);
                pz[e] = fma(k.cz[R + q], nb[XL + e + q], pz[e]);
                pz[e] = fma(k.cz[R - q], nb[XL + e - q], pz[e]);
              }
            }
#pragma unroll
            for (int e = 0; e < VEC; ++e) p[e] += pz[e];
            if constexpr (MODE == MODE_APPLY_EPI) {
              // local potential of this (in-range) plane: its part is output
              // plane pfirst + s's
              const int pp = pfirst + s, y = y0 + yb + j;
              if (a.pot && pp >= z0 && pp < z1 && y < a.vout.n[1]) {
                const S* pr = static_cast<const S*>(a.pot) + (int64_t)pp * a.vout.s0 + (int64_t)y * a.vout.s1 + x;
#pragma unroll
                for (int e = 0; e < VEC; ++e)
                  if (e < nx) p[e] = fma(pr[e], c.v[e], p[e]);
              }
            }
            // scatter along axis 0 (logical slot m receives offset R - m)
#pragma unroll
            for (int m = 0; m < NR; ++m) {
              const int pm = (m + ph) % NR;
#pragma unroll
              for (int e = 0; e < VEC; ++e) {
                if (m == R)
                  acc[j][pm].v[e] += p[e];
                else
                  acc[j][pm].v[e] = fma(k.cx[2 * R - m], c.v[e], acc[j][pm].v[e]);
              }
            }
          }
          // output plane o is complete: logical slot 0 = physical ph
          if (o >= z0) {
            const S* rsl = reinterpret_cast<const S*>(stg + C::RHO_OFF);
            const double* asl = reinterpret_cast<const double*>(stg + C::AUX_OFF);
#pragma unroll
            for (int j = 0; j < PY; ++j) {
              const int y = y0 + yb + j;
              if (y < a.vout.n[1] && nx > 0) {
                const P av = acc[j][ph];
                P res;
                P rho{};
                if constexpr (C::HAS_RHO) rho = ldv<S, VEC>(rsl + (yb + j) * C::TZ + VEC * tx);
                const int64_t oidx =
                    (int64_t)b * a.vout.sb + (int64_t)o * a.vout.s0 + (int64_t)y * a.vout.s1 + x;
                if constexpr (MODE == MODE_APPLY || MODE == MODE_APPLY_EPI) {
                  res = av;
                  if (MODE == MODE_APPLY_EPI && a.aux) {
                    const S* xp = static_cast<const S*>(a.aux) + oidx;
                    const S g = (S)a.aux_scale;
#pragma unroll
                    for (int e = 0; e < VEC; ++e)
                      if (e < nx) res.v[e] = fma(g, xp[e], res.v[e]);
                  }
                } else if constexpr (C::RR) {
#pragma unroll
                  for (int e = 0; e < VEC; ++e) res.v[e] = av.v[e] - rho.v[e];
                } else if constexpr (MODE == MODE_RESIDUAL || MODE == MODE_RESID_DC) {
#pragma unroll
                  for (int e = 0; e < VEC; ++e) res.v[e] = av.v[e] - rho.v[e];
                  if (a.gsum.partial) {
                    if constexpr (VEC == 2) {
                      sumsq += (double)res.v[0] * res.v[0] + (nx > 1 ? (double)res.v[1] * res.v[1] : 0.0);
                    } else {
                      double t = (double)res.v[0] * res.v[0];
#pragma unroll
                      for (int e = 1; e < VEC; ++e) t += e < nx ? (double)res.v[e] * res.v[e] : 0.0;
                      sumsq += t;
                    }
                  }
                } else {
                  // the centre value, R planes behind in the ring
                  const S* osl = reinterpret_cast<const S*>(ring + ((gbase + s + NS - R) % NS) * C::STAGE_BYTES);
                  P cur = ldv<S, VEC>(osl + (yb + j + R) * W + xl);
                  P avs = av;
                  if constexpr (MODE == MODE_JACOBI_SCALED_IN) {
                    // the ring holds rhs: rho = rhs, phi = (w2 / c0) rhs, and
                    // A phi = (w2 / c0) A rhs (one scaling per output point)
#pragma unroll
                    for (int e = 0; e < VEC; ++e) {
                      rho.v[e] = cur.v[e];
                      cur.v[e] = k.wc2 * cur.v[e];
                      avs.v[e] = k.wc2 * av.v[e];
                    }
                  }
#pragma unroll
                  for (int e = 0; e < VEC; ++e) res.v[e] = k.w1 * cur.v[e] + k.wc * (rho.v[e] - avs.v[e]);
                }
                if constexpr (MODE == MODE_RESID_DC) {
                  // float32 defect and first inner Jacobi iterate from zero
                  Pack<float, VEC> rhs, e1;
#pragma unroll
                  for (int e = 0; e < VEC; ++e) {
                    rhs.v[e] = (float)(-res.v[e]);
                    e1.v[e] = k.wc2 * rhs.v[e];
                  }
                  float* rp = static_cast<float*>(a.out) + oidx;
                  float* ep = static_cast<float*>(a.out2) + oidx;  // null: the next sweep forms e1 itself
                  if (nx == VEC) {
                    stv<float, VEC>(rp, rhs);
                    if (a.out2) stv<float, VEC>(ep, e1);
                  } else {
                    stv_part<float, VEC>(rp, rhs, nx);
                    if (a.out2) stv_part<float, VEC>(ep, e1, nx);
                  }
                } else if constexpr (MODE == MODE_JACOBI_ADD64) {
                  // phi64 += e (the inner correction), e never stored
                  double* pp = static_cast<double*>(a.out2) + oidx;
                  const double* ap = asl + (yb + j) * C::TZ + VEC * tx;
#pragma unroll
                  for (int h = 0; h < VEC; h += 2) {
                    Pack<double, 2> pv = ldv<double, 2>(ap + h);
                    pv.v[0] += (double)res.v[h];
                    pv.v[1] += (double)res.v[h + 1];
                    if (h + 2 <= nx)
                      stv<double, 2>(pp + h, pv);
                    else
                      stv_part<double, 2>(pp + h, pv, nx - h);
                  }
                } else if constexpr (C::RR) {
                  stv<S, VEC>(rtile + (yb + j) * C::TZ + VEC * tx, res);
                } else if (MODE != MODE_RESIDUAL || a.out) {
                  S* op = static_cast<S*>(a.out) + oidx;
                  if (nx == VEC)
                    stv<S, VEC>(op, res);
                  else
                    stv_part<S, VEC>(op, res, nx);
                }
              }
            }
            if constexpr (C::RR) {
              // restriction of the residual plane o (c/bmgs/restrict.c: axis 2,
              // then axis 1, then axis 0 over fine planes 2 I0, 2 I0 + 1, 2 I0 + 2)
              __syncthreads();  // the tile's residual plane is complete in rtile
#pragma unroll
              for (int u = 0; u < RK; ++u) {
                const int t = tid + u * C::NT;
                const int rci1 = t / C::CX, rci2 = t - (t / C::CX) * C::CX;
                const int rI1 = by * C::CY + rci1, rI2 = bx * C::CX + rci2;
                if (t < C::CX * C::CY && rI1 < a.vco.n[1] && rI2 < a.vco.n[2]) {
                  const S* rr = rtile + (2 * rci1) * C::TZ + 2 * rci2;
                  S zr[3];
#pragma unroll
                  for (int d1 = 0; d1 < 3; ++d1)
                    zr[d1] = r2(rr[d1 * C::TZ], rr[d1 * C::TZ + 1], rr[d1 * C::TZ + 2]);
                  const S yv = r2(zr[0], zr[1], zr[2]);
                  const int ol = o - z0;  // z0 is even
                  if ((ol & 1) == 0) {
                    if (ol >= 2) {
                      const S v = r2(rq0[u], rq1[u], yv);
                      const int64_t ci = (int64_t)b * a.vco.sb + (int64_t)((o - 2) / 2) * a.vco.s0 +
                                         (int64_t)rI1 * a.vco.s1 + rI2;
                      static_cast<S*>(a.out)[ci] = v;
                      static_cast<S*>(a.out2)[ci] = (S)k.wc2 * v;
                    }
                    rq0[u] = yv;
                  } else {
                    rq1[u] = yv;
                  }
                }
              }
            }
          }
#pragma unroll
          for (int j = 0; j < PY; ++j)
#pragma unroll
            for (int e = 0; e < VEC; ++e) acc[j][ph].v[e] = S(0);
          __syncthreads();  // every thread is done with plane s - R (its slot is refilled next)
          if (tid == 0 && s + D + 1 < nsteps) issue(s + D + 1);
        }
      }
      gbase += nsteps;  // every load of the segment has been waited for
    }
  }
  pdl_trigger();
  if (timed_out && ta.status) atomicExch(ta.status, GPW_ETIMEDOUT);
  if constexpr (MODE == MODE_RESIDUAL || MODE == MODE_RESID_DC) {
    if (a.gsum.partial) {
      double tot = block_sum(sumsq, red);
      const int blk = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * chunk);
      grid_sum_finish(a.gsum, bchunk, blk, a.nblk_seg, tot, red);
    }
  }
}

}  // namespace gpw
