// Restriction and interpolation between a grid and its 2x coarser grid.
//
// Reference: c/transformers.c:54-123 fills a padded copy (c/bc.c, cfd = 0, so
// halo edges and corners are filled too) and then runs three separable 1D
// passes -- axis 2, then axis 1, then axis 0 -- each writing a transposed
// temporary (c/bmgs/restrict.c:137-154, c/bmgs/interpolate.c:141-168).
//
// Here one kernel does all three passes without temporaries in HBM: a CTA owns
// an (axis-1, axis-2) output tile and marches along axis 0.  Each input plane
// of the tile (with halo) is staged in shared memory by cp.async; the axis-2
// pass and the axis-1 pass run in shared memory; the axis-0 pass gathers from
// a per-thread register queue of the last planes' partial results.  Every 1D
// pass evaluates the reference's expression in the reference's order with
// unfused multiply / add, so results are bit-identical to the reference C.
//
// 1D rules (K = 2 nn taps; w = the reference's weight table):
//   restrict  out[i] = 0.5 * (a[c] + w1 (a[c+1] + a[c-1]) + w3 (a[c+3] + a[c-3]) + ...)
//             c = K - 1 + 2 i in padded coordinates   (c/bmgs/restrict.c:37-57)
//   interpolate, o = 2 i + e - skip0 (e = 0 or 1), c = K/2 - 1 + i:
//             e = 0: out[o] = a[c]
//             e = 1: out[o] = w1 (a[c] + a[c+1]) + w3 (a[c-1] + a[c+2]) + ...
//                                                     (c/bmgs/interpolate.c:31-64)
#pragma once
#include "gpw_common.cuh"

namespace gpw {

struct TransferArgs {
  const void* in;
  void* out;
  GridView vin, vout;
  Boundary bc;        // boundary of the input grid
  int pad0[3];        // low padding of the input (padded -> unpadded shift)
  int skip0[3];       // interpolation: skip of the first output per axis
  int zchunk, nchunk; // output planes of axis 0 per CTA
  const unsigned char* active;
  int subtract;       // interpolation: out = base - I(in) instead of out = I(in)
  const void* base;   // (the reference's phi -= I(e) into another buffer; must not alias out)
  GridView vbase;
  // K=2 restriction into a multigrid level: also write the level's first
  // weighted-Jacobi sweep from phi = 0, out2 = (w2 / c02) out (same view)
  void* out2;
  double w2, c02;
};

// Per-thread descriptors of a box's cells (H x W, NT threads, cell k of a
// thread = tid + k NT): the box origin in (axis 1, axis 2) is fixed for the
// CTA, so each cell's in-plane source offset, validity and wrap sides are
// computed once; loading a plane is then one cp.async per cell and the
// Bloch fix-up touches only wrapped cells.
template <typename T, int H, int W, int NT>
struct BoxLoader {
  static constexpr int NLD = (H * W + NT - 1) / NT;
  int off[NLD];            // j1 * s1 + j2
  unsigned valid = 0;      // bit k: cell k is inside the grid or a periodic image
  unsigned wrapped = 0;    // bit k: cell k is a periodic image along axis 1 or 2
  unsigned char side[NLD]; // wrap sides: bits 0-1 axis 1 (+1), bits 2-3 axis 2 (+1)

  __device__ __forceinline__ void init(const GridView& v, const Boundary& bc, int ys, int xs) {
    const int tid = threadIdx.x + blockDim.x * threadIdx.y;
#pragma unroll
    for (int k = 0; k < NLD; ++k) {
      const int idx = tid + k * NT;
      const int r = idx / W, c = idx - r * W;
      int j1 = 0, j2 = 0, s1 = -1, s2 = -1;
      const bool ok = idx < H * W && wrap_axis(ys + r, v.n[1], bc.periodic[1], j1, s1) &&
                      wrap_axis(xs + c, v.n[2], bc.periodic[2], j2, s2);
      off[k] = ok ? (int)((int64_t)j1 * v.s1 + j2) : 0;
      if (ok) valid |= 1u << k;
      if (ok && (s1 >= 0 || s2 >= 0)) wrapped |= 1u << k;
      side[k] = (unsigned char)((s1 + 1) | ((s2 + 1) << 2));
    }
  }

  // plane p into `slot` (row pitch W); zero-boundary cells read zeros
  __device__ __forceinline__ void load(T* slot, const T* in, const GridView& v, const Boundary& bc, int p) const {
    const int tid = threadIdx.x + blockDim.x * threadIdx.y;
    int j0, s0;
    const bool ok0 = wrap_axis(p, v.n[0], bc.periodic[0], j0, s0);
    const T* base = in + (int64_t)j0 * v.s0;
#pragma unroll
    for (int k = 0; k < NLD; ++k) {
      const int idx = tid + k * NT;
      if ((H * W) % NT == 0 || idx < H * W) {
        const bool ok = ok0 && ((valid >> k) & 1u);
        cp_async<sizeof(T)>(slot + idx, ok ? base + off[k] : in, ok);
      }
    }
  }

  // Bloch phases of the periodic images, axis by axis as the reference's
  // chained halo copies apply them (each thread fixes its own copies)
  __device__ __forceinline__ void fix(T* slot, const GridView& v, const Boundary& bc, int p) const {
    if constexpr (EltTraits<T>::cpx) {
      const int tid = threadIdx.x + blockDim.x * threadIdx.y;
      int j0, s0;
      if (!wrap_axis(p, v.n[0], bc.periodic[0], j0, s0)) return;
      const unsigned todo = s0 >= 0 ? valid : wrapped;
#pragma unroll
      for (int k = 0; k < NLD; ++k) {
        if (!((todo >> k) & 1u)) continue;
        const int idx = tid + k * NT;
        const int s1 = (side[k] & 3) - 1, s2 = ((side[k] >> 2) & 3) - 1;
        T val = slot[idx];
        if (s0 >= 0) val = phase_mul(bc.ph[0][s0], val);
        if (s1 >= 0) val = phase_mul(bc.ph[1][s1], val);
        if (s2 >= 0) val = phase_mul(bc.ph[2][s2], val);
        slot[idx] = val;
      }
    }
  }
};

// unfused helpers for exact reference arithmetic
__device__ __forceinline__ double radd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float radd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double2 radd(double2 a, double2 b) {
  return make_double2(__dadd_rn(a.x, b.x), __dadd_rn(a.y, b.y));
}
__device__ __forceinline__ float2 radd(float2 a, float2 b) {
  return make_float2(__fadd_rn(a.x, b.x), __fadd_rn(a.y, b.y));
}
__device__ __forceinline__ double rmul(double c, double a) { return __dmul_rn(c, a); }
__device__ __forceinline__ float rmul(float c, float a) { return __fmul_rn(c, a); }
__device__ __forceinline__ double2 rmul(double c, double2 a) {
  return make_double2(__dmul_rn(c, a.x), __dmul_rn(c, a.y));
}
__device__ __forceinline__ float2 rmul(float c, float2 a) {
  return make_float2(__fmul_rn(c, a.x), __fmul_rn(c, a.y));
}

// K = 2 rules: 0.5 * (a0 + 0.5 * (a1 + a_1))   (c/bmgs/restrict.c:38-39)
template <typename S>
__device__ __forceinline__ S r2(S am, S a0, S ap) {
  return rmul(S(0.5), radd(a0, rmul(S(0.5), radd(ap, am))));
}
// 0.5 * (a0 + a1)                 (c/bmgs/interpolate.c:33)
template <typename S>
__device__ __forceinline__ S i2h(S a0, S a1) {
  return rmul(S(0.5), radd(a0, a1));
}

template <int K> struct TW;
template <> struct TW<2> { static __device__ __forceinline__ double w(int) { return 0.5; } };
template <> struct TW<4> {
  static __device__ __forceinline__ double w(int j) { return j == 0 ? 0.5625 : -0.0625; }
};
template <> struct TW<6> {
  static __device__ __forceinline__ double w(int j) {
    return j == 0 ? 0.58593750 : (j == 1 ? -0.09765625 : 0.01171875);
  }
};
template <> struct TW<8> {
  static __device__ __forceinline__ double w(int j) {
    return j == 0 ? 0.59814453125 : (j == 1 ? -0.11962890625 : (j == 2 ? 0.02392578125 : -0.00244140625));
  }
};

// restriction tap sum around a[c] with stride `st` (in elements)
template <int K, typename T>
__device__ __forceinline__ T restrict_1d(const T* a, int st) {
  using S = typename EltTraits<T>::S;
  if constexpr (K == 2) {
    // 0.5 * (aa[0] + 0.5 * (aa[1] + aa[-1]))
    return rmul(S(0.5), radd(a[0], rmul(S(0.5), radd(a[st], a[-st]))));
  } else {
    T s = a[0];
#pragma unroll
    for (int j = 0; j < K / 2; ++j) s = radd(s, rmul((S)TW<K>::w(j), radd(a[(2 * j + 1) * st], a[-(2 * j + 1) * st])));
    return rmul(S(0.5), s);
  }
}

// interpolation midpoint value between a[0] and a[st]
template <int K, typename T>
__device__ __forceinline__ T interp_mid(const T* a, int st) {
  using S = typename EltTraits<T>::S;
  if constexpr (K == 2) {
    return rmul(S(0.5), radd(a[0], a[st]));
  } else {
    T s = rmul((S)TW<K>::w(0), radd(a[0], a[st]));
#pragma unroll
    for (int j = 1; j < K / 2; ++j) s = radd(s, rmul((S)TW<K>::w(j), radd(a[-j * st], a[(1 + j) * st])));
    return s;
  }
}

// ------------------------------------------------------------------ restrict
constexpr int RS_OZ = 32, RS_OY = 8;

template <typename T, int K>
struct RestrictCfg {
  static constexpr int H = 2 * RS_OY + 2 * K - 3;  // fine rows per plane tile
  static constexpr int W = 2 * RS_OZ + 2 * K - 3;  // fine cols
  static constexpr int NQ = 2 * K - 1;             // axis-0 taps span
  static constexpr int NS = 3;                     // cp.async stages
  static constexpr size_t smem = (size_t)NS * H * W * sizeof(T) + (size_t)H * RS_OZ * sizeof(T);
};

template <typename T, int K>
__global__ void __launch_bounds__(RS_OZ* RS_OY) restrict_kernel(const TransferArgs a) {
  using C = RestrictCfg<T, K>;
  constexpr int H = C::H, W = C::W, NQ = C::NQ, NS = C::NS;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* ring = reinterpret_cast<T*>(smem_raw);
  T* zb = ring + NS * H * W;  // axis-2 pass result, H x RS_OZ

  const int b = blockIdx.z / a.nchunk, chunk = blockIdx.z - b * a.nchunk;
  if (a.active && !a.active[b]) return;
  const int X0 = blockIdx.x * RS_OZ, Y0 = blockIdx.y * RS_OY;
  const int I0 = chunk * a.zchunk, I1 = min(a.vout.n[0], I0 + a.zchunk);
  if (I0 >= I1) return;
  const T* in = static_cast<const T*>(a.in) + (int64_t)b * a.vin.sb;
  const int tx = threadIdx.x, ty = threadIdx.y, tid = tx + RS_OZ * ty;
  // unpadded origin of the fine tile
  const int ys = 2 * Y0 - a.pad0[1], xs = 2 * X0 - a.pad0[2];
  // fine planes feeding outputs I0 .. I1-1: centre u(I) = K-1 + 2I - pad0
  const int pfirst = K - 1 + 2 * I0 - a.pad0[0] - (K - 1);
  const int plast = K - 1 + 2 * (I1 - 1) - a.pad0[0] + (K - 1);
  const int nsteps = plast - pfirst + 1;
  const int Y = Y0 + ty, X = X0 + tx;
  const bool inside = Y < a.vout.n[1] && X < a.vout.n[2];

  T q[NQ];
#pragma unroll
  for (int i = 0; i < NQ; ++i) q[i] = zero<T>();

  BoxLoader<T, H, W, RS_OZ * RS_OY> ld;
  ld.init(a.vin, a.bc, ys, xs);
#pragma unroll
  for (int st = 0; st < NS - 1; ++st) {
    if (st < nsteps) ld.load(ring + st * H * W, in, a.vin, a.bc, pfirst + st);
    cp_async_commit();
  }
  for (int s = 0; s < nsteps; ++s) {
    const int p = pfirst + s;
    {
      const int sn = s + NS - 1;
      if (sn < nsteps) ld.load(ring + (sn % NS) * H * W, in, a.vin, a.bc, pfirst + sn);
      cp_async_commit();
    }
    cp_async_wait<NS - 1>();
    T* sl = ring + (s % NS) * H * W;
    if (a.bc.use_phase) ld.fix(sl, a.vin, a.bc, p);
    __syncthreads();
    // axis-2 pass: zb[r][J] for all H rows
    for (int idx = tid; idx < H * RS_OZ; idx += RS_OZ * RS_OY) {
      const int r = idx / RS_OZ, J = idx - r * RS_OZ;
      zb[idx] = restrict_1d<K>(sl + r * W + 2 * J + K - 1, 1);
    }
    __syncthreads();
    // axis-1 pass for this thread's output column
    const T v = restrict_1d<K>(zb + (2 * ty + K - 1) * RS_OZ + tx, RS_OZ);
#pragma unroll
    for (int i = 0; i < NQ - 1; ++i) q[i] = q[i + 1];
    q[NQ - 1] = v;
    // plane p completes output I with u(I) + K - 1 == p
    const int t = p - (K - 1) - (K - 1) + a.pad0[0];
    if (s >= NQ - 1 && (t & 1) == 0) {
      const int I = t >> 1;
      if (I >= I0 && I < I1 && inside) {
        const T o = restrict_1d<K>(q + (K - 1), 1);
        static_cast<T*>(a.out)[(int64_t)b * a.vout.sb + (int64_t)I * a.vout.s0 + (int64_t)Y * a.vout.s1 + X] = o;
      }
    }
    __syncthreads();
  }
}

// ------------------------------------------------------------------ interpolate
constexpr int IP_OZ = 32, IP_OY = 8;

template <typename T, int K>
struct InterpCfg {
  static constexpr int H = IP_OY / 2 + 1 + K;  // coarse rows per plane tile
  static constexpr int W = IP_OZ / 2 + 1 + K;  // coarse cols
  static constexpr int NQ = K;                 // axis-0 queue
  static constexpr int NS = 3;
  static constexpr size_t smem = (size_t)NS * H * W * sizeof(T) + (size_t)H * IP_OZ * sizeof(T);
};

template <typename T, int K>
__global__ void __launch_bounds__(IP_OZ* IP_OY) interpolate_kernel(const TransferArgs a) {
  using C = InterpCfg<T, K>;
  constexpr int H = C::H, W = C::W, NQ = C::NQ, NS = C::NS;
  constexpr int base = K / 2 - 1;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* ring = reinterpret_cast<T*>(smem_raw);
  T* zb = ring + NS * H * W;  // axis-2 pass result, H x IP_OZ

  const int b = blockIdx.z / a.nchunk, chunk = blockIdx.z - b * a.nchunk;
  if (a.active && !a.active[b]) return;
  const int X0 = blockIdx.x * IP_OZ, Y0 = blockIdx.y * IP_OY;
  const int O0 = chunk * a.zchunk, O1 = min(a.vout.n[0], O0 + a.zchunk);
  if (O0 >= O1) return;
  const T* in = static_cast<const T*>(a.in) + (int64_t)b * a.vin.sb;
  const int tx = threadIdx.x, ty = threadIdx.y, tid = tx + IP_OZ * ty;
  // coarse index i of a fine output o: o + skip0 = 2 i + e; centre c = base + i (padded)
  // unpadded coarse coordinate of the centre: base + i - pad0.  Tile origin
  // (unpadded) = centre of the first output minus (K/2 - 1).
  const int iy0 = (Y0 + a.skip0[1]) >> 1, ix0 = (X0 + a.skip0[2]) >> 1;
  const int ys = base + iy0 - a.pad0[1] - (K / 2 - 1);
  const int xs = base + ix0 - a.pad0[2] - (K / 2 - 1);
  const int i0f = (O0 + a.skip0[0]) >> 1, i0l = (O1 - 1 + a.skip0[0]) >> 1;
  const int pfirst = base + i0f - a.pad0[0] - (K / 2 - 1);
  const int plast = base + i0l - a.pad0[0] + K / 2;
  const int nsteps = plast - pfirst + 1;
  const int oy = Y0 + ty, ox = X0 + tx;
  const bool inside = oy < a.vout.n[1] && ox < a.vout.n[2];
  // this thread's axis-1 position inside the coarse tile
  const int ey = (oy + a.skip0[1]) & 1, ly = ((oy + a.skip0[1]) >> 1) - iy0 + (K / 2 - 1);

  T q[NQ];
#pragma unroll
  for (int i = 0; i < NQ; ++i) q[i] = zero<T>();

  BoxLoader<T, H, W, IP_OZ * IP_OY> ld;
  ld.init(a.vin, a.bc, ys, xs);
#pragma unroll
  for (int st = 0; st < NS - 1; ++st) {
    if (st < nsteps) ld.load(ring + st * H * W, in, a.vin, a.bc, pfirst + st);
    cp_async_commit();
  }
  for (int s = 0; s < nsteps; ++s) {
    const int p = pfirst + s;
    {
      const int sn = s + NS - 1;
      if (sn < nsteps) ld.load(ring + (sn % NS) * H * W, in, a.vin, a.bc, pfirst + sn);
      cp_async_commit();
    }
    cp_async_wait<NS - 1>();
    T* sl = ring + (s % NS) * H * W;
    if (a.bc.use_phase) ld.fix(sl, a.vin, a.bc, p);
    __syncthreads();
    // axis-2 pass: zb[r][x] for each fine output column x of the tile
    for (int idx = tid; idx < H * IP_OZ; idx += IP_OZ * IP_OY) {
      const int r = idx / IP_OZ, xl = idx - r * IP_OZ;
      const int o = X0 + xl;
      const int e = (o + a.skip0[2]) & 1, lx = ((o + a.skip0[2]) >> 1) - ix0 + (K / 2 - 1);
      const T* rp = sl + r * W + lx;
      zb[idx] = e ? interp_mid<K>(rp, 1) : rp[0];
    }
    __syncthreads();
    // axis-1 pass for this thread's (oy, ox)
    const T* cp = zb + ly * IP_OZ + tx;
    const T v = ey ? interp_mid<K>(cp, IP_OZ) : cp[0];
#pragma unroll
    for (int i = 0; i < NQ - 1; ++i) q[i] = q[i + 1];
    q[NQ - 1] = v;
    // plane p (unpadded) = base + i - pad0 + d; outputs completed at this plane:
    //  even o (e = 0) with centre plane == p          -> q[NQ-1]
    //  odd  o (e = 1) with centre plane == p - K/2    -> taps q[NQ-1-K/2 - j .. ]
    const int ic = p - base + a.pad0[0];  // i with centre at p
    if (inside) {
      T* outp = static_cast<T*>(a.out) + (int64_t)b * a.vout.sb + (int64_t)oy * a.vout.s1 + ox;
      const T* basep = a.subtract ? static_cast<const T*>(a.base) + (int64_t)b * a.vbase.sb +
                                        (int64_t)oy * a.vbase.s1 + ox
                                  : nullptr;
      {
        const int o = 2 * ic - a.skip0[0];
        if (o >= O0 && o < O1) {
          const T val = q[NQ - 1];
          outp[(int64_t)o * a.vout.s0] = a.subtract ? sub(basep[(int64_t)o * a.vbase.s0], val) : val;
        }
      }
      {
        const int i = ic - K / 2;
        const int o = 2 * i + 1 - a.skip0[0];
        if (o >= O0 && o < O1 && s >= K - 1) {
          const T val = interp_mid<K>(q + (NQ - 1 - K / 2), 1);
          outp[(int64_t)o * a.vout.s0] = a.subtract ? sub(basep[(int64_t)o * a.vbase.s0], val) : val;
        }
      }
    }
    __syncthreads();
  }
}

}  // namespace gpw
