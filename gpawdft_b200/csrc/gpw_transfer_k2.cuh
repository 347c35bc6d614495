// Direct-evaluation restriction and interpolation for K = 2 (nn = 1) on real
// grids -- the transfers of every multigrid level of the Poisson solver and of
// the eigensolver preconditioner.
//
// The K = 2 operators touch 3 (restriction) or 2 (interpolation) input points
// per axis, so instead of staging tiles in shared memory each thread reads
// its few input values straight through L1 and evaluates the three
// separable 1D passes in the reference's order and expression form
// (axis 2, then axis 1, then axis 0; c/bmgs/restrict.c:37-39,
// c/bmgs/interpolate.c:31-33), unfused -- bit-identical to the reference.
// A thread owns one (axis-1, axis-2) output column and marches along axis 0,
// carrying the axis-0 partial results of the previous plane.  The in-plane
// addresses and boundary handling of a column are resolved once per thread
// (zero boundary: a zero weight on an out-of-grid input; periodic: the
// wrapped index; real data carries no Bloch phase), so the march itself is
// loads and arithmetic only.
#pragma once
#include <climits>

#include "gpw_common.cuh"
#include "gpw_star_tma.cuh"
#include "gpw_transfer.cuh"

namespace gpw {

constexpr int K2_TX = 32, K2_TY = 8;

// Resolve index i along an axis: element offset (times stride) and a
// validity flag (false: zero-boundary halo, value 0).
__device__ __forceinline__ bool k2_axis(int i, int n, int periodic, int64_t stride, int64_t& off) {
  int j, s;
  if (!wrap_axis(i, n, periodic, j, s)) {
    off = 0;
    return false;
  }
  off = (int64_t)j * stride;
  return true;
}

template <typename S>
__device__ __forceinline__ S k2_ld(const S* __restrict__ p, bool ok) {
  return ok ? __ldg(p) : S(0);
}

template <typename S>
__global__ void __launch_bounds__(K2_TX* K2_TY) restrict_k2_kernel(const TransferArgs a) {
  pdl_wait();
  const int b = blockIdx.z / a.nchunk, chunk = blockIdx.z - b * a.nchunk;
  if (a.active && !a.active[b]) return;
  const int I2 = blockIdx.x * K2_TX + threadIdx.x, I1 = blockIdx.y * K2_TY + threadIdx.y;
  if (I1 >= a.vout.n[1] || I2 >= a.vout.n[2]) return;
  const int I0s = chunk * a.zchunk, I0e = min(a.vout.n[0], I0s + a.zchunk);
  const S* __restrict__ in = static_cast<const S*>(a.in) + (int64_t)b * a.vin.sb;
  S* __restrict__ out = static_cast<S*>(a.out) + (int64_t)b * a.vout.sb + (int64_t)I1 * a.vout.s1 + I2;
  // fine centres (unpadded): c = 1 + 2 I - pad0; taps c-1, c, c+1
  const int c1 = 1 + 2 * I1 - a.pad0[1], c2 = 1 + 2 * I2 - a.pad0[2];
  int64_t off[3][3];  // [axis-1 tap][axis-2 tap] in-plane element offsets
  bool ok[3][3];
#pragma unroll
  for (int d1 = 0; d1 < 3; ++d1) {
    int64_t o1, o2;
    const bool v1 = k2_axis(c1 - 1 + d1, a.vin.n[1], a.bc.periodic[1], a.vin.s1, o1);
#pragma unroll
    for (int d2 = 0; d2 < 3; ++d2) {
      const bool v2 = k2_axis(c2 - 1 + d2, a.vin.n[2], a.bc.periodic[2], 1, o2);
      off[d1][d2] = o1 + o2;
      ok[d1][d2] = v1 && v2;
    }
  }
  auto Y = [&](int f0) -> S {
    int64_t o0;
    const bool v0 = k2_axis(f0, a.vin.n[0], a.bc.periodic[0], a.vin.s0, o0);
    const S* pl = in + o0;
    S z[3];
#pragma unroll
    for (int d1 = 0; d1 < 3; ++d1)
      z[d1] = r2(k2_ld(pl + off[d1][0], v0 && ok[d1][0]), k2_ld(pl + off[d1][1], v0 && ok[d1][1]),
                 k2_ld(pl + off[d1][2], v0 && ok[d1][2]));
    return r2(z[0], z[1], z[2]);
  };
  S* __restrict__ out2 =
      a.out2 ? static_cast<S*>(a.out2) + (int64_t)b * a.vout.sb + (int64_t)I1 * a.vout.s1 + I2 : nullptr;
  const S wc = (S)a.w2 / (S)a.c02;
  S ylo = Y(1 + 2 * I0s - a.pad0[0] - 1);
#pragma unroll 2
  for (int I0 = I0s; I0 < I0e; ++I0) {
    const int c0 = 1 + 2 * I0 - a.pad0[0];
    const S ym = Y(c0), yp = Y(c0 + 1);
    const S v = r2(ylo, ym, yp);
    out[(int64_t)I0 * a.vout.s0] = v;
    if (out2) out2[(int64_t)I0 * a.vout.s0] = wc * v;
    ylo = yp;
  }
}

template <typename S>
__global__ void __launch_bounds__(K2_TX* K2_TY) interpolate_k2_kernel(const TransferArgs a) {
  pdl_wait();
  const int b = blockIdx.z / a.nchunk, chunk = blockIdx.z - b * a.nchunk;
  if (a.active && !a.active[b]) return;
  const int o2 = blockIdx.x * K2_TX + threadIdx.x, o1 = blockIdx.y * K2_TY + threadIdx.y;
  if (o1 >= a.vout.n[1] || o2 >= a.vout.n[2]) return;
  const int O0s = chunk * a.zchunk, O0e = min(a.vout.n[0], O0s + a.zchunk);
  const S* __restrict__ in = static_cast<const S*>(a.in) + (int64_t)b * a.vin.sb;
  S* __restrict__ out = static_cast<S*>(a.out) + (int64_t)b * a.vout.sb + (int64_t)o1 * a.vout.s1 + o2;
  const S* __restrict__ base =
      a.subtract ? static_cast<const S*>(a.base) + (int64_t)b * a.vbase.sb + (int64_t)o1 * a.vbase.s1 + o2
                 : nullptr;
  // per axis: o + skip0 = 2 i + e; coarse (unpadded) index u = i - pad0
  const int t1 = o1 + a.skip0[1], t2 = o2 + a.skip0[2];
  const int u1 = (t1 >> 1) - a.pad0[1], e1 = t1 & 1;
  const int u2 = (t2 >> 1) - a.pad0[2], e2 = t2 & 1;
  int64_t off[2][2];
  bool ok[2][2];
#pragma unroll
  for (int d1 = 0; d1 < 2; ++d1) {
    int64_t q1, q2;
    const bool v1 = k2_axis(u1 + d1, a.vin.n[1], a.bc.periodic[1], a.vin.s1, q1);
#pragma unroll
    for (int d2 = 0; d2 < 2; ++d2) {
      const bool v2 = k2_axis(u2 + d2, a.vin.n[2], a.bc.periodic[2], 1, q2);
      off[d1][d2] = q1 + q2;
      ok[d1][d2] = v1 && v2;
    }
  }
  auto Y = [&](int u0) -> S {
    int64_t q0;
    const bool v0 = k2_axis(u0, a.vin.n[0], a.bc.periodic[0], a.vin.s0, q0);
    const S* pl = in + q0;
    S z0 = k2_ld(pl + off[0][0], v0 && ok[0][0]);
    if (e2) z0 = i2h(z0, k2_ld(pl + off[0][1], v0 && ok[0][1]));
    if (!e1) return z0;
    S z1 = k2_ld(pl + off[1][0], v0 && ok[1][0]);
    if (e2) z1 = i2h(z1, k2_ld(pl + off[1][1], v0 && ok[1][1]));
    return i2h(z0, z1);
  };
  // march over coarse planes u: fine outputs o = 2 (u + pad0) + e0 - skip0
  // (e0 = 0: Y(u); e0 = 1: the midpoint of Y(u) and Y(u+1)); the loads of
  // the next plane do not depend on this plane's stores, so they run ahead
  const int us = ((O0s + a.skip0[0]) >> 1) - a.pad0[0];
  const int ue = ((O0e - 1 + a.skip0[0]) >> 1) - a.pad0[0];
  S ya = Y(us);
#pragma unroll 2
  for (int u = us; u <= ue; ++u) {
    const S yb = Y(u + 1);
    const int oe = 2 * (u + a.pad0[0]) - a.skip0[0];
    if (oe >= O0s && oe < O0e) {
      const int64_t q = (int64_t)oe * a.vout.s0;
      out[q] = a.subtract ? base[(int64_t)oe * a.vbase.s0] - ya : ya;
    }
    if (oe + 1 >= O0s && oe + 1 < O0e) {
      const S mid = i2h(ya, yb);
      out[(int64_t)(oe + 1) * a.vout.s0] = a.subtract ? base[(int64_t)(oe + 1) * a.vbase.s0] - mid : mid;
    }
    ya = yb;
  }
}

// ------------------------------------------------------------------ vector form
// Interpolation with each thread owning 4 adjacent axis-2 outputs (16-byte
// loads of `base` and stores of `out` for float32; two 16-byte accesses for
// float64) and axis 0 split into chunks: the scalar kernel above keeps too
// few bytes in flight per thread to reach HBM bandwidth on 127^3 grids.
// Same expressions per output as interpolate_k2_kernel (bit-identical).
// Needs out / base rows, planes and batch members 16-byte aligned; outputs
// past the row end are never written.
constexpr int K2V_TX = 32, K2V_TY = 8;

template <typename S>
__device__ __forceinline__ void ld4(const S* p, S (&v)[4], int nvalid) {
  if (nvalid == 4) {
    if constexpr (sizeof(S) == 4) {
      const float4 t = *reinterpret_cast<const float4*>(p);
      v[0] = t.x; v[1] = t.y; v[2] = t.z; v[3] = t.w;
    } else {
      const double2 t0 = reinterpret_cast<const double2*>(p)[0];
      const double2 t1 = reinterpret_cast<const double2*>(p)[1];
      v[0] = t0.x; v[1] = t0.y; v[2] = t1.x; v[3] = t1.y;
    }
  } else {
#pragma unroll
    for (int k = 0; k < 4; ++k) v[k] = (k < nvalid) ? p[k] : S(0);
  }
}

template <typename S>
__device__ __forceinline__ void st4(S* p, const S (&v)[4], int nvalid) {
  if (nvalid == 4) {
    if constexpr (sizeof(S) == 4) {
      *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
    } else {
      reinterpret_cast<double2*>(p)[0] = make_double2(v[0], v[1]);
      reinterpret_cast<double2*>(p)[1] = make_double2(v[2], v[3]);
    }
  } else {
#pragma unroll
    for (int k = 0; k < 4; ++k)
      if (k < nvalid) p[k] = v[k];
  }
}

template <typename S>
__global__ void __launch_bounds__(K2V_TX* K2V_TY) interpolate_k2_vec_kernel(const TransferArgs a) {
  pdl_wait();
  const int b = blockIdx.z / a.nchunk, chunk = blockIdx.z - b * a.nchunk;
  if (a.active && !a.active[b]) return;
  const int o2 = 4 * (blockIdx.x * K2V_TX + threadIdx.x), o1 = blockIdx.y * K2V_TY + threadIdx.y;
  if (o1 >= a.vout.n[1] || o2 >= a.vout.n[2]) return;
  const int nvalid = min(4, a.vout.n[2] - o2);
  const int O0s = chunk * a.zchunk, O0e = min(a.vout.n[0], O0s + a.zchunk);
  const S* __restrict__ in = static_cast<const S*>(a.in) + (int64_t)b * a.vin.sb;
  S* __restrict__ out = static_cast<S*>(a.out) + (int64_t)b * a.vout.sb + (int64_t)o1 * a.vout.s1 + o2;
  const S* __restrict__ base =
      a.subtract ? static_cast<const S*>(a.base) + (int64_t)b * a.vbase.sb + (int64_t)o1 * a.vbase.s1 + o2
                 : nullptr;
  const int t1 = o1 + a.skip0[1], t2 = o2 + a.skip0[2];
  const int u1 = (t1 >> 1) - a.pad0[1], e1 = t1 & 1;
  const int u2 = (t2 >> 1) - a.pad0[2], e2 = t2 & 1;
  // the 4 outputs need coarse axis-2 points u2 .. u2+2 on rows u1 (and u1+1)
  int64_t off[2][3];
  bool ok[2][3];
#pragma unroll
  for (int d1 = 0; d1 < 2; ++d1) {
    int64_t q1, q2;
    const bool v1 = k2_axis(u1 + d1, a.vin.n[1], a.bc.periodic[1], a.vin.s1, q1);
#pragma unroll
    for (int d2 = 0; d2 < 3; ++d2) {
      const bool v2 = k2_axis(u2 + d2, a.vin.n[2], a.bc.periodic[2], 1, q2);
      off[d1][d2] = q1 + q2;
      ok[d1][d2] = v1 && v2;
    }
  }
  auto Y = [&](int u0, S (&y)[4]) {
    int64_t q0;
    const bool v0 = k2_axis(u0, a.vin.n[0], a.bc.periodic[0], a.vin.s0, q0);
    const S* pl = in + q0;
    S c[2][3];
#pragma unroll
    for (int d2 = 0; d2 < 3; ++d2) {
      c[0][d2] = k2_ld(pl + off[0][d2], v0 && ok[0][d2]);
      c[1][d2] = e1 ? k2_ld(pl + off[1][d2], v0 && ok[1][d2]) : S(0);
    }
    // axis-2 pass per row: output k takes coarse point (e2 + k) / 2, or the
    // midpoint with the next one when e2 + k is odd
    S z[2][4];
#pragma unroll
    for (int d1 = 0; d1 < 2; ++d1) {
      const S m01 = i2h(c[d1][0], c[d1][1]), m12 = i2h(c[d1][1], c[d1][2]);
      z[d1][0] = e2 ? m01 : c[d1][0];
      z[d1][1] = e2 ? c[d1][1] : m01;
      z[d1][2] = e2 ? m12 : c[d1][1];
      z[d1][3] = e2 ? c[d1][2] : m12;
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) y[k] = e1 ? i2h(z[0][k], z[1][k]) : z[0][k];
  };
  const int us = ((O0s + a.skip0[0]) >> 1) - a.pad0[0];
  const int ue = ((O0e - 1 + a.skip0[0]) >> 1) - a.pad0[0];
  S ya[4], yb[4], v[4], bv[4];
  Y(us, ya);
#pragma unroll 2
  for (int u = us; u <= ue; ++u) {
    Y(u + 1, yb);
    const int oe = 2 * (u + a.pad0[0]) - a.skip0[0];
    if (oe >= O0s && oe < O0e) {
      if (a.subtract) {
        ld4(base + (int64_t)oe * a.vbase.s0, bv, nvalid);
#pragma unroll
        for (int k = 0; k < 4; ++k) v[k] = bv[k] - ya[k];
      } else {
#pragma unroll
        for (int k = 0; k < 4; ++k) v[k] = ya[k];
      }
      st4(out + (int64_t)oe * a.vout.s0, v, nvalid);
    }
    if (oe + 1 >= O0s && oe + 1 < O0e) {
      if (a.subtract) {
        ld4(base + (int64_t)(oe + 1) * a.vbase.s0, bv, nvalid);
#pragma unroll
        for (int k = 0; k < 4; ++k) v[k] = bv[k] - i2h(ya[k], yb[k]);
      } else {
#pragma unroll
        for (int k = 0; k < 4; ++k) v[k] = i2h(ya[k], yb[k]);
      }
      st4(out + (int64_t)(oe + 1) * a.vout.s0, v, nvalid);
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) ya[k] = yb[k];
  }
}

// ------------------------------------------------------------------ vector restriction
// Restriction with each thread owning 2 adjacent axis-2 outputs I2, I2+1
// (a warp covers a 64-point output row): per (axis-0, axis-1) tap row the 5
// fine inputs 2 I2 .. 2 I2 + 4 come from one 16-byte load (two for float64)
// plus one scalar.  Zero-boundary grids with pad 0 on axis 2 (fine centre
// 2I + 1), 16-byte aligned rows; a thread whose taps would pass the row end
// falls back to checked scalar loads.  Same expressions per output as
// restrict_k2_kernel (bit-identical).
template <typename S>
__device__ __forceinline__ void ld5(const S* p, S (&v)[5]) {
  if constexpr (sizeof(S) == 4) {
    const float4 a = *reinterpret_cast<const float4*>(p);
    v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
  } else {
    const double2 a = reinterpret_cast<const double2*>(p)[0];
    const double2 b = reinterpret_cast<const double2*>(p)[1];
    v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
  }
  v[4] = p[4];
}

template <typename S>
__device__ __forceinline__ void st2(S* p, S v0, S v1, int nvalid) {
  if (nvalid == 2) {
    if constexpr (sizeof(S) == 4)
      *reinterpret_cast<float2*>(p) = make_float2(v0, v1);
    else
      *reinterpret_cast<double2*>(p) = make_double2(v0, v1);
  } else {
    p[0] = v0;
  }
}

template <typename S>
__global__ void __launch_bounds__(K2V_TX* K2V_TY) restrict_k2_vec_kernel(const TransferArgs a) {
  pdl_wait();
  const int b = blockIdx.z / a.nchunk, chunk = blockIdx.z - b * a.nchunk;
  if (a.active && !a.active[b]) return;
  const int I2 = 2 * (blockIdx.x * K2V_TX + threadIdx.x), I1 = blockIdx.y * K2V_TY + threadIdx.y;
  if (I1 >= a.vout.n[1] || I2 >= a.vout.n[2]) return;
  const int nvalid = min(2, a.vout.n[2] - I2);
  const int I0s = chunk * a.zchunk, I0e = min(a.vout.n[0], I0s + a.zchunk);
  const S* __restrict__ in = static_cast<const S*>(a.in) + (int64_t)b * a.vin.sb;
  S* __restrict__ out = static_cast<S*>(a.out) + (int64_t)b * a.vout.sb + (int64_t)I1 * a.vout.s1 + I2;
  S* __restrict__ out2 =
      a.out2 ? static_cast<S*>(a.out2) + (int64_t)b * a.vout.sb + (int64_t)I1 * a.vout.s1 + I2 : nullptr;
  const S wc = (S)a.w2 / (S)a.c02;
  const int c1 = 1 + 2 * I1 - a.pad0[1];
  const int f2 = 2 * I2 - a.pad0[2];  // first fine tap along axis 2 (c2 - 1 of output I2)
  const bool full = f2 >= 0 && f2 + 4 < a.vin.n[2];
  int64_t o1[3];
  bool v1[3];
#pragma unroll
  for (int d1 = 0; d1 < 3; ++d1) v1[d1] = k2_axis(c1 - 1 + d1, a.vin.n[1], a.bc.periodic[1], a.vin.s1, o1[d1]);
  // the axis-2 and axis-1 passes of both outputs on fine plane f0
  auto Y = [&](int f0, S& y0, S& y1) {
    int64_t o0;
    const bool v0 = k2_axis(f0, a.vin.n[0], a.bc.periodic[0], a.vin.s0, o0);
    S z0[3], z1[3];
#pragma unroll
    for (int d1 = 0; d1 < 3; ++d1) {
      S r[5];
      if (v0 && v1[d1]) {
        const S* row = in + o0 + o1[d1];
        if (full) {
          ld5(row + f2, r);
        } else {
#pragma unroll
          for (int q = 0; q < 5; ++q) {
            const int f = f2 + q;
            r[q] = (f >= 0 && f < a.vin.n[2]) ? row[f] : S(0);
          }
        }
      } else {
#pragma unroll
        for (int q = 0; q < 5; ++q) r[q] = S(0);
      }
      z0[d1] = r2(r[0], r[1], r[2]);
      z1[d1] = r2(r[2], r[3], r[4]);
    }
    y0 = r2(z0[0], z0[1], z0[2]);
    y1 = r2(z1[0], z1[1], z1[2]);
  };
  S l0, l1, m0, m1, p0, p1;
  Y(1 + 2 * I0s - a.pad0[0] - 1, l0, l1);
#pragma unroll 2
  for (int I0 = I0s; I0 < I0e; ++I0) {
    const int c0 = 1 + 2 * I0 - a.pad0[0];
    Y(c0, m0, m1);
    Y(c0 + 1, p0, p1);
    const S v0 = r2(l0, m0, p0), v1v = r2(l1, m1, p1);
    l0 = p0;
    l1 = p1;
    st2(out + (int64_t)I0 * a.vout.s0, v0, v1v, nvalid);
    if (out2) st2(out2 + (int64_t)I0 * a.vout.s0, wc * v0, wc * v1v, nvalid);
  }
}

// ------------------------------------------------------------------ TMA restriction
// K = 2 restriction of zero-boundary real grids (fine centre 2I + 1) fed by
// TMA: a CTA owns a 32 (axis 2) x 8 (axis 1) tile of coarse points and a
// chunk of coarse planes; each fine plane of the tile's footprint (68 x 17
// points from (2 X0, 2 Y0), the last columns / rows past the grid
// zero-filled) arrives as one tensor-map box on its own mbarrier, RK_D coarse
// planes ahead.  Each thread evaluates its coarse point from the three
// staged fine planes with the expressions of restrict_k2_kernel
// (bit-identical) and writes it, and the level's first Jacobi sweep from
// zero if requested.  Every wait is bounded.
constexpr int RK_TX = 32, RK_TY = 8;          // coarse tile
constexpr int RK_W = 2 * RK_TX + 4;           // fine box width (16-byte multiple for f32 / f64)
constexpr int RK_H = 2 * RK_TY + 1;           // fine box height
constexpr int RK_D = 2;                        // coarse planes of prefetch
constexpr int RK_NS = 3 + 2 * RK_D;            // fine-plane stages

template <typename S>
struct RkCfg {
  static constexpr int STAGE = (RK_W * RK_H * (int)sizeof(S) + 127) / 128 * 128;
  static constexpr size_t smem = (size_t)RK_NS * STAGE + RK_NS * 8 + 128;
};

template <typename S>
__global__ void __launch_bounds__(RK_TX* RK_TY) restrict_k2_tma_kernel(const __grid_constant__ CUtensorMap map,
                                                                       const TransferArgs a, int* status) {
  using C = RkCfg<S>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  unsigned char* ring = smem_raw + ((128u - (smem_u32(smem_raw) & 127u)) & 127u);
  uint64_t* bars = reinterpret_cast<uint64_t*>(ring + RK_NS * C::STAGE);
  pdl_wait();
  const int b = blockIdx.z / a.nchunk, chunk = blockIdx.z - b * a.nchunk;
  if (a.active && !a.active[b]) return;
  const int nc0 = a.vout.n[0];
  const int C0 = (int)((int64_t)chunk * nc0 / a.nchunk), C1 = (int)((int64_t)(chunk + 1) * nc0 / a.nchunk);
  const int X0 = blockIdx.x * RK_TX, Y0 = blockIdx.y * RK_TY;
  const int tx = threadIdx.x, ty = threadIdx.y, tid = tx + RK_TX * ty;
  const int I2 = X0 + tx, I1 = Y0 + ty;
  const bool inside = I1 < a.vout.n[1] && I2 < a.vout.n[2];
  bool timed_out = false;
  if (tid == 0) {
    for (int i = 0; i < RK_NS; ++i) mbar_init(mbar_u32(&bars[i]), 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  __syncthreads();
  if (C0 >= C1) return;
  // fine planes 2 C0 .. 2 C1 (step i = fine plane 2 C0 + i)
  const int nsteps = 2 * (C1 - C0) + 1;
  auto issue = [&](int i) {
    const unsigned bar = mbar_u32(&bars[i % RK_NS]);
    mbar_expect_tx(bar, (unsigned)(RK_W * RK_H * sizeof(S)));
    tma_load_4d(smem_u32(ring + (i % RK_NS) * C::STAGE), &map, 2 * X0, 2 * Y0, 2 * C0 + i, b, bar);
  };
  if (tid == 0)
    for (int i = 0; i < 3 + 2 * RK_D && i < nsteps; ++i) issue(i);
  S* __restrict__ out = static_cast<S*>(a.out) + (int64_t)b * a.vout.sb + (int64_t)I1 * a.vout.s1 + I2;
  S* __restrict__ out2 =
      a.out2 ? static_cast<S*>(a.out2) + (int64_t)b * a.vout.sb + (int64_t)I1 * a.vout.s1 + I2 : nullptr;
  const S wc = (S)a.w2 / (S)a.c02;
  for (int c = 0; c < C1 - C0; ++c) {
    // coarse plane C0 + c: fine steps 2c, 2c + 1, 2c + 2
    for (int d = (c == 0 ? 0 : 1); d <= 2; ++d) {
      const int i = 2 * c + d;
      if (!mbar_wait_bounded(mbar_u32(&bars[i % RK_NS]), (unsigned)((i / RK_NS) & 1))) timed_out = true;
    }
    if (inside) {
      S y[3];
#pragma unroll
      for (int d0 = 0; d0 < 3; ++d0) {
        const S* pl = reinterpret_cast<const S*>(ring + ((2 * c + d0) % RK_NS) * C::STAGE);
        S z[3];
#pragma unroll
        for (int d1 = 0; d1 < 3; ++d1) {
          const S* row = pl + (2 * ty + d1) * RK_W + 2 * tx;
          z[d1] = r2(row[0], row[1], row[2]);
        }
        y[d0] = r2(z[0], z[1], z[2]);
      }
      const S v = r2(y[0], y[1], y[2]);
      out[(int64_t)(C0 + c) * a.vout.s0] = v;
      if (out2) out2[(int64_t)(C0 + c) * a.vout.s0] = wc * v;
    }
    __syncthreads();  // fine steps 2c, 2c + 1 are consumed (their slots are refilled next)
    if (tid == 0) {
      const int n1 = 2 * c + 3 + 2 * RK_D;  // next steps to issue: two per coarse plane
      if (n1 < nsteps) issue(n1);
      if (n1 + 1 < nsteps) issue(n1 + 1);
    }
  }
  pdl_trigger();
  if (timed_out && status) atomicExch(status, GPW_ETIMEDOUT);
}

// ------------------------------------------------------------------ TMA interpolation
// K = 2 interpolation with subtraction, out = base - I(e), on zero-boundary
// real grids (pad 1, skip 1 per axis: fine o takes coarse u = (o+1)/2 - 1,
// midpoint with u + 1 when o is even) fed by TMA.  A CTA owns a 64 (axis 2)
// x 16 (axis 1) fine tile and a chunk of coarse planes m; per m one
// mbarrier covers the coarse plane m (a 40 x 10 box from the 16-byte aligned
// column 32 bx - 4 and row 8 by - 1) and the base planes 2m and 2m + 1
// (64 x 16 boxes).  Fine planes 2m, 2m + 1 need coarse planes m - 1 and m.
// Each thread owns 2 adjacent axis-2 points x 2 rows and evaluates them with
// the expressions of interpolate_k2_kernel (bit-identical).  Bounded waits.
constexpr int IK_TX = 32, IK_NTY = 8;              // threads
constexpr int IK_FW = 64, IK_FH = 16;              // fine tile
constexpr int IK_CW = 40, IK_CH = 10;              // coarse box
constexpr int IK_D = 2;                             // coarse planes of prefetch
constexpr int IK_NS = IK_D + 2;                     // stages (plane m - 1 stays resident)

template <typename S>
struct IkCfg {
  static constexpr int CB = (IK_CW * IK_CH * (int)sizeof(S) + 127) / 128 * 128;
  static constexpr int FB = (IK_FW * IK_FH * (int)sizeof(S) + 127) / 128 * 128;
  static constexpr int STAGE = CB + 2 * FB;
  static constexpr size_t smem = (size_t)IK_NS * STAGE + IK_NS * 8 + 128;
};

template <typename S>
__global__ void __launch_bounds__(IK_TX* IK_NTY) interpolate_k2_tma_kernel(const __grid_constant__ CUtensorMap cmap,
                                                                           const __grid_constant__ CUtensorMap bmap,
                                                                           const TransferArgs a, int* status) {
  using C = IkCfg<S>;
  using V = typename VecT<S, 2>::T;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  unsigned char* ring = smem_raw + ((128u - (smem_u32(smem_raw) & 127u)) & 127u);
  uint64_t* bars = reinterpret_cast<uint64_t*>(ring + IK_NS * C::STAGE);
  pdl_wait();
  const int b = blockIdx.z / a.nchunk, chunk = blockIdx.z - b * a.nchunk;
  if (a.active && !a.active[b]) return;
  const int nf0 = a.vout.n[0];
  const int nm = nf0 / 2 + 1;  // coarse planes m whose fine planes 2m, 2m+1 start inside the grid
  const int M0 = (int)((int64_t)chunk * nm / a.nchunk), M1 = (int)((int64_t)(chunk + 1) * nm / a.nchunk);
  const int x0 = blockIdx.x * IK_FW, y0 = blockIdx.y * IK_FH;
  const int cx0 = x0 / 2 - 4, cy0 = y0 / 2 - 1;  // coarse box origin
  const int tx = threadIdx.x, ty = threadIdx.y, tid = tx + IK_TX * ty;
  bool timed_out = false;
  if (tid == 0) {
    for (int i = 0; i < IK_NS; ++i) mbar_init(mbar_u32(&bars[i]), 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  __syncthreads();
  if (M0 >= M1) return;
  // steps: coarse planes M0 - 1 .. M1 - 1 (step i = plane M0 - 1 + i); the
  // first carries no base planes
  const int nsteps = M1 - M0 + 1;
  auto issue = [&](int i) {
    unsigned char* st = ring + (i % IK_NS) * C::STAGE;
    const unsigned bar = mbar_u32(&bars[i % IK_NS]);
    const int m = M0 - 1 + i;
    const bool base = i > 0;
    mbar_expect_tx(bar, (unsigned)(IK_CW * IK_CH * sizeof(S) + (base ? 2 * IK_FW * IK_FH * sizeof(S) : 0)));
    tma_load_4d(smem_u32(st), &cmap, cx0, cy0, m, b, bar);
    if (base) {
      tma_load_4d(smem_u32(st + C::CB), &bmap, x0, y0, 2 * m, b, bar);
      tma_load_4d(smem_u32(st + C::CB + C::FB), &bmap, x0, y0, 2 * m + 1, b, bar);
    }
  };
  if (tid == 0)
    for (int i = 0; i <= IK_D && i < nsteps; ++i) issue(i);
  // this thread's fine points: x = x0 + 2 tx + {0, 1}, y = y0 + 2 ty + {0, 1}
  const int lx = 2 * tx, ly = 2 * ty;
  const bool xin0 = x0 + lx < a.vout.n[2], xin1 = x0 + lx + 1 < a.vout.n[2];
  // per axis: o + 1 = 2 u' + e with u' the padded coarse index, i.e. coarse
  // u = u' - 1; local coarse column u - cx0 = u' + 3 - x0/2
  int cu2[2], ce2[2], cu1[2], ce1[2];
#pragma unroll
  for (int k = 0; k < 2; ++k) {
    const int t2 = x0 + lx + k + 1, t1 = y0 + ly + k + 1;
    cu2[k] = (t2 >> 1) - 1 - cx0;
    ce2[k] = t2 & 1;
    cu1[k] = (t1 >> 1) - 1 - cy0;
    ce1[k] = t1 & 1;
  }
  // Y(u0)[j][k]: the axis-2 and axis-1 passes on coarse plane stage `cp`
  auto Y = [&](const S* cp, int j, int k) -> S {
    const S* r0 = cp + cu1[j] * IK_CW;
    S z0 = r0[cu2[k]];
    if (ce2[k]) z0 = i2h(z0, r0[cu2[k] + 1]);
    if (!ce1[j]) return z0;
    const S* r1 = r0 + IK_CW;
    S z1 = r1[cu2[k]];
    if (ce2[k]) z1 = i2h(z1, r1[cu2[k] + 1]);
    return i2h(z0, z1);
  };
  for (int i = 0; i < nsteps; ++i) {
    if (!mbar_wait_bounded(mbar_u32(&bars[i % IK_NS]), (unsigned)((i / IK_NS) & 1))) timed_out = true;
    if (i > 0) {
      const int m = M0 - 1 + i;
      const S* cm1 = reinterpret_cast<const S*>(ring + ((i - 1) % IK_NS) * C::STAGE);  // plane m - 1
      const S* cm = reinterpret_cast<const S*>(ring + (i % IK_NS) * C::STAGE);         // plane m
#pragma unroll
      for (int f = 0; f < 2; ++f) {  // fine plane 2m + f: even -> midpoint of m-1, m; odd -> m
        const int o = 2 * m + f;
        if (o >= nf0) break;
        const S* base = reinterpret_cast<const S*>(ring + (i % IK_NS) * C::STAGE + C::CB + f * C::FB);
#pragma unroll
        for (int j = 0; j < 2; ++j) {
          const int y = y0 + ly + j;
          if (y >= a.vout.n[1] || !xin0) continue;
          S v[2];
#pragma unroll
          for (int k = 0; k < 2; ++k) {
            const S ya = Y(f == 0 ? cm1 : cm, j, k);
            v[k] = (f == 0) ? i2h(ya, Y(cm, j, k)) : ya;
          }
          const V bv = *reinterpret_cast<const V*>(base + (ly + j) * IK_FW + lx);
          S* op = static_cast<S*>(a.out) + (int64_t)b * a.vout.sb + (int64_t)o * a.vout.s0 + (int64_t)y * a.vout.s1 +
                  x0 + lx;
          if (xin1)
            *reinterpret_cast<V*>(op) = V{bv.x - v[0], bv.y - v[1]};
          else
            op[0] = bv.x - v[0];
        }
      }
    }
    __syncthreads();  // plane step i - 1 is consumed
    if (tid == 0 && i + IK_D + 1 < nsteps) issue(i + IK_D + 1);
  }
  pdl_trigger();
  if (timed_out && status) atomicExch(status, GPW_ETIMEDOUT);
}

}  // namespace gpw
