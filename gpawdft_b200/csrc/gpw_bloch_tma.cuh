// TMA-fed star stencil (apply) for grids with periodic / Bloch boundaries, or
// any mix of periodic and zero axes, real or complex (sm_100a).
//
// The band stencils of the eigensolver (Laplace / kinetic nn=3 and the
// gradients on periodic cells, c/operators.c:316-405 with the Bloch halo of
// c/bc.c:138-250) run here.  Compared with the cp.async kernel of
// gpw_stencil.cuh:
//  * a CTA owns whole rows (axis 2) of TY axis-1 rows and marches along
//    axis 0; per plane one thread issues three 4D TMA box loads into a ring
//    stage -- the R halo rows above, the TY rows, the R halo rows below --
//    whose coordinates are wrapped on periodic axes and left out of range on
//    zero axes (the tensor map's zero fill is the zero boundary);
//  * the axis-2 halo never exists: a row is staged whole, and the R columns
//    beyond either end are read from the other end of the same row;
//  * Bloch phases are applied in registers as values are read (a wrapped
//    halo row, a wrapped axis-2 neighbour, a wrapped axis-0 plane), each
//    neighbour of a star stencil lying across at most one boundary, so no
//    fix-up pass touches shared memory;
//  * one warp spans a row, each lane VEC adjacent points; the axis-0
//    accumulators rotate by compile-time renaming as in gpw_star_tma.cuh,
//    but only the small scatter-and-store step is instantiated per rotation
//    (a switch on the step), so the in-plane body exists once;
//  * the warps never meet at a CTA barrier: a warp releases a stage through
//    an "empty" mbarrier once its values are in registers, and the stage is
//    refilled when every warp has left it (a ring of D + 3 stages, D planes
//    in flight, refills waiting on the plane read two steps earlier).
// Every mbarrier wait is bounded (GPW_ETIMEDOUT in the status word).
#pragma once
#include <cuda.h>

#include "gpw_common.cuh"
#include "gpw_star_tma.cuh"

namespace gpw {

template <typename T, int R, int VEC, int NW, int D, int WPR>
struct BlochCfg {
  static constexpr int PY = (sizeof(T) >= 16) ? 1 : 2;  // axis-1 rows per thread
  static constexpr int NT = 32 * NW;
  static constexpr int TY = (NW / WPR) * PY;            // output rows per tile (WPR warps span a row)
  static constexpr int ROWS = TY + 2 * R;               // staged rows per plane
  // ring stages: D planes in flight ahead of the one being read, and two
  // more so the refill of a stage waits for the warps to leave the plane
  // read two steps earlier, not the current one
  static constexpr int NS = D + 3;
  static constexpr int NR = 2 * R + 1;
  static constexpr int MINB = NW <= 6 ? 2 : 1;          // CTAs per SM the registers must allow
};

// Real coefficients in the element's scalar type.
template <typename S>
struct BlochCoefs {
  S cx[7], cy[7], cz[7];  // offset + R (R <= 3)
  S cc;
  bool has_y, has_z;      // axis-1 / axis-2 terms present (false for a gradient along another axis)
};

struct BlochArgs {
  void* out;
  GridView vout;          // the input's extents are the same
  Boundary bc;
  int nchunk;             // chunks of axis 0 (gridDim.z = nchunk * nbatch)
  int rowbytes;           // n2 * sizeof(T)
  int stage_bytes;        // ROWS * rowbytes (a multiple of 128)
  int* status;
  const void* pot;        // optional local potential (scalar type, the output's
                          // layout without batch): out = A in + pot in
  const void* aux;        // optional grids in the output's layout and type:
  double aux_scale;       //   out += aux_scale aux
};

__device__ __forceinline__ void mbar_arrive(unsigned bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(bar) : "memory");
}

// EPI: a potential or aux term is present (a.pot / a.aux); the plain apply
// is compiled without their loads and branches.
template <typename T, int R, int VEC, int NW, int D, int WPR, bool EPI>
__global__ void __launch_bounds__(32 * NW, (BlochCfg<T, R, VEC, NW, D, WPR>::MINB))
    bloch_star_kernel(const __grid_constant__ CUtensorMap tmain, const __grid_constant__ CUtensorMap thalo,
                      const BlochArgs a, const BlochCoefs<typename EltTraits<T>::S> k) {
  using C = BlochCfg<T, R, VEC, NW, D, WPR>;
  constexpr int NS = C::NS, NR = C::NR, PY = C::PY, TY = C::TY;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  unsigned char* ring = smem_raw + ((128u - (smem_u32(smem_raw) & 127u)) & 127u);
  uint64_t* full = reinterpret_cast<uint64_t*>(ring + NS * a.stage_bytes);
  uint64_t* empty = full + NS;

  const int n0 = a.vout.n[0], n1 = a.vout.n[1], n2 = a.vout.n[2];
  const int b = blockIdx.z / a.nchunk, chunk = blockIdx.z - b * a.nchunk;
  const int y0 = blockIdx.y * TY;
  const int z0 = (int)((int64_t)chunk * n0 / a.nchunk);
  const int z1 = (int)((int64_t)(chunk + 1) * n0 / a.nchunk);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const Boundary& bc = a.bc;
  bool timed_out = false;

  if (threadIdx.x == 0) {
    for (int i = 0; i < NS; ++i) {
      mbar_init(mbar_u32(&full[i]), 1);
      mbar_init(mbar_u32(&empty[i]), NW);
    }
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  __syncthreads();
  if (z0 >= z1) return;
  const int pfirst = z0 - R;
  const int nsteps = z1 - z0 + 2 * R;
  // thread 0 streams the planes into the ring: step i's plane (wrapped on
  // a periodic axis 0; out of range, i.e. zeros, on a zero axis) with its
  // halo rows; a stage is refilled once every warp has released it
  const int yt = bc.periodic[1] ? (y0 - R + n1) % n1 : y0 - R;
  const int ybot = bc.periodic[1] ? (y0 + TY) % n1 : y0 + TY;
  auto issue = [&](int i) {
    const int slot = i % NS;
    if (i >= NS && !mbar_wait_bounded(mbar_u32(&empty[slot]), (unsigned)((i / NS - 1) & 1))) timed_out = true;
    unsigned char* st = ring + slot * a.stage_bytes;
    const unsigned bar = mbar_u32(&full[slot]);
    int p = pfirst + i;
    if (bc.periodic[0]) p = (p % n0 + n0) % n0;
    mbar_expect_tx(bar, (unsigned)(C::ROWS * a.rowbytes));
    tma_load_4d(smem_u32(st), &thalo, 0, yt, p, b, bar);
    tma_load_4d(smem_u32(st + R * a.rowbytes), &tmain, 0, y0, p, b, bar);
    tma_load_4d(smem_u32(st + (R + TY) * a.rowbytes), &thalo, 0, ybot, p, b, bar);
  };
  if (threadIdx.x == 0)
    for (int i = 0; i <= D && i < nsteps; ++i) issue(i);

  // ---- this lane's columns
  const int wr = w / WPR;                         // warp row of the tile
  const int xb = ((w % WPR) * 32 + lane) * VEC;   // first point of this lane
  const int nx = min(VEC, n2 - xb);   // points inside the row (<= 0: idle lane)
  const bool cpx_phase = EltTraits<T>::cpx && bc.use_phase;
  // Columns of positions xb - R .. xb + VEC - 1 + R along the row, wrapped
  // on a periodic axis (a position below 0 takes the Bloch phase of side 1,
  // one past n2 - 1 that of side 0) or zero on a zero axis.  Right-hand
  // positions start at the lane's own points, so a lane whose last points
  // lie past the row end reads them as the wrapped neighbours of its valid
  // ones; idle lanes read valid columns whose results are never stored.
  int lidx[R], xr[VEC + R];
  unsigned lwrap = 0, lzero = 0;  // bit q-1: position xb - q
  unsigned rwrap = 0, rzero = 0;  // bit t: position xb + t
#pragma unroll
  for (int q = 1; q <= R; ++q) {
    int j, s;
    const bool ok = wrap_axis(xb - q, n2, bc.periodic[2], j, s);
    lidx[q - 1] = ok ? j : 0;
    if (!ok) lzero |= 1u << (q - 1);
    else if (s >= 0) lwrap |= 1u << (q - 1);
  }
#pragma unroll
  for (int t = 0; t < VEC + R; ++t) {
    int j, s;
    const bool ok = wrap_axis(xb + t, n2, bc.periodic[2], j, s);
    xr[t] = ok ? j : 0;
    if (!ok) rzero |= 1u << t;
    else if (s >= 0) rwrap |= 1u << t;
  }
  // halo rows wrapped across the axis-1 boundary carry a Bloch phase
  const bool top_wrap = bc.periodic[1] && y0 == 0;
  const bool bot_wrap = bc.periodic[1] && y0 + TY >= n1;
  const int ylo = y0 + wr * PY;                    // this warp's first output row
  const int nrows_ok = min(PY, n1 - ylo);
  T* const outb = static_cast<T*>(a.out) + (int64_t)b * a.vout.sb + (int64_t)ylo * a.vout.s1 + xb;

  T acc[PY][NR][VEC];
#pragma unroll
  for (int j = 0; j < PY; ++j)
#pragma unroll
    for (int m = 0; m < NR; ++m)
#pragma unroll
      for (int e = 0; e < VEC; ++e) acc[j][m][e] = zero<T>();

  for (int sb = 0; sb < nsteps; sb += NR) {
#pragma unroll
    for (int ph = 0; ph < NR; ++ph) {
      const int s = sb + ph;
      if (s >= nsteps) break;
      const int slot = s % NS;
      const unsigned char* stg = ring + slot * a.stage_bytes;
      const int p = pfirst + s;
      const int o = p - R;  // output plane completed by this step
      if (!mbar_wait_bounded(mbar_u32(&full[slot]), (unsigned)((s / NS) & 1))) timed_out = true;
      // axis-0 image: the scatter value of a wrapped plane carries its
      // phase (side 1 below 0, side 0 past n0 - 1)
      const bool p_wrap = bc.periodic[0] && (p < 0 || p >= n0);

      T c[PY][VEC], part[PY][VEC];
#pragma unroll
      for (int j = 0; j < PY; ++j) {
        const int sr = wr * PY + j + R;  // stage row of this output row
        const T* row = reinterpret_cast<const T*>(stg + sr * a.rowbytes);
#pragma unroll
        for (int e = 0; e < VEC; ++e) {
          T v = row[xr[e]];
          if ((rzero >> e) & 1u) v = zero<T>();
          else if (cpx_phase && ((rwrap >> e) & 1u)) v = phase_mul(bc.ph[2][0], v);
          c[j][e] = v;
        }
        // the in-plane sum in two chains (axis 1, axis 2) joined at the end
        T py[VEC], pz[VEC];
#pragma unroll
        for (int e = 0; e < VEC; ++e) {
          py[e] = zero<T>();
          pz[e] = zero<T>();
        }
        if (k.has_y) {
#pragma unroll
          for (int q = 1; q <= R; ++q) {
            const T* up = reinterpret_cast<const T*>(stg + (sr + q) * a.rowbytes);
            const T* dn = reinterpret_cast<const T*>(stg + (sr - q) * a.rowbytes);
            const bool up_wr = bot_wrap && sr + q >= R + TY, dn_wr = top_wrap && sr - q < R;
#pragma unroll
            for (int e = 0; e < VEC; ++e) {
              T vu = up[xr[e]], vd = dn[xr[e]];
              if (cpx_phase && up_wr) vu = phase_mul(bc.ph[1][0], vu);
              if (cpx_phase && dn_wr) vd = phase_mul(bc.ph[1][1], vd);
              py[e] = fmac(k.cy[R + q], vu, py[e]);
              py[e] = fmac(k.cy[R - q], vd, py[e]);
            }
          }
        }
        if (k.has_z) {
          // the row's values from xb - R to xb + VEC - 1 + R
          T nb[VEC + 2 * R];
#pragma unroll
          for (int e = 0; e < VEC; ++e) nb[R + e] = c[j][e];
#pragma unroll
          for (int q = 1; q <= R; ++q) {
            constexpr int t = VEC - 1;  // the right neighbour q sits at position VEC - 1 + q
            T vl = row[lidx[q - 1]], vr = row[xr[t + q]];
            if ((lzero >> (q - 1)) & 1u) vl = zero<T>();
            else if (cpx_phase && ((lwrap >> (q - 1)) & 1u)) vl = phase_mul(bc.ph[2][1], vl);
            if ((rzero >> (t + q)) & 1u) vr = zero<T>();
            else if (cpx_phase && ((rwrap >> (t + q)) & 1u)) vr = phase_mul(bc.ph[2][0], vr);
            nb[R - q] = vl;
            nb[R + VEC - 1 + q] = vr;
          }
#pragma unroll
          for (int q = 1; q <= R; ++q) {
#pragma unroll
            for (int e = 0; e < VEC; ++e) {
              pz[e] = fmac(k.cz[R + q], nb[R + e + q], pz[e]);
              pz[e] = fmac(k.cz[R - q], nb[R + e - q], pz[e]);
            }
          }
        }
#pragma unroll
        for (int e = 0; e < VEC; ++e) part[j][e] = add(fmac(k.cc, c[j][e], py[e]), pz[e]);
        if (EPI && a.pot && p >= z0 && p < z1 && j < nrows_ok) {
          // local potential of this (in-range) plane: its part is output p's
          using S = typename EltTraits<T>::S;
          const S* pr = static_cast<const S*>(a.pot) + (int64_t)p * a.vout.s0 + (int64_t)(ylo + j) * a.vout.s1 + xb;
#pragma unroll
          for (int e = 0; e < VEC; ++e)
            if (e < nx) part[j][e] = fmac(pr[e], c[j][e], part[j][e]);
        }
        if (cpx_phase && p_wrap) {
          const double2 pp = p < 0 ? bc.ph[0][1] : bc.ph[0][0];
#pragma unroll
          for (int e = 0; e < VEC; ++e) c[j][e] = phase_mul(pp, c[j][e]);
        }
      }
      // every value of the stage is in registers: release it, and refill
      // the stage of step s + D + 1 (last read at step s - 2)
      __syncwarp();
      if (lane == 0) mbar_arrive(mbar_u32(&empty[slot]));
      if (threadIdx.x == 0 && s + D + 1 < nsteps) issue(s + D + 1);

      // scatter along axis 0 (logical slot m receives offset R - m)
#pragma unroll
      for (int j = 0; j < PY; ++j) {
#pragma unroll
        for (int m = 0; m < NR; ++m) {
          const int pm = (m + ph) % NR;
#pragma unroll
          for (int e = 0; e < VEC; ++e) {
            if (m == R)
              acc[j][pm][e] = add(acc[j][pm][e], part[j][e]);
            else
              acc[j][pm][e] = fmac(k.cx[2 * R - m], c[j][e], acc[j][pm][e]);
          }
        }
      }
      // output plane o is complete: logical slot 0 = physical ph
      if (o >= z0 && nx > 0) {
        T* op0 = outb + (int64_t)o * a.vout.s0;
        const T* ax0 = (EPI && a.aux) ? static_cast<const T*>(a.aux) + (op0 - static_cast<T*>(a.out)) : nullptr;
        using S = typename EltTraits<T>::S;
#pragma unroll
        for (int j = 0; j < PY; ++j) {
          if (j < nrows_ok) {
            T* op = op0 + j * a.vout.s1;
#pragma unroll
            for (int e = 0; e < VEC; ++e)
              if (e < nx)
                op[e] = (EPI && ax0) ? fmac((S)a.aux_scale, ax0[j * a.vout.s1 + e], acc[j][ph][e]) : acc[j][ph][e];
          }
        }
      }
#pragma unroll
      for (int j = 0; j < PY; ++j)
#pragma unroll
        for (int e = 0; e < VEC; ++e) acc[j][ph][e] = zero<T>();
    }
  }
  if (timed_out && a.status) atomicExch(a.status, GPW_ETIMEDOUT);
}

}  // namespace gpw
