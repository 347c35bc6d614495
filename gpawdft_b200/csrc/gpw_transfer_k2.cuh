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
#include "gpw_transfer.cuh"

namespace gpw {

constexpr int K2_TX = 32, K2_TY = 8;

// 0.5 * (a0 + 0.5 * (a1 + a_1))   (c/bmgs/restrict.c:38-39)
template <typename S>
__device__ __forceinline__ S r2(S am, S a0, S ap) {
  return rmul(S(0.5), radd(a0, rmul(S(0.5), radd(ap, am))));
}
// 0.5 * (a0 + a1)                 (c/bmgs/interpolate.c:33)
template <typename S>
__device__ __forceinline__ S i2h(S a0, S a1) {
  return rmul(S(0.5), radd(a0, a1));
}

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

}  // namespace gpw
