// Lexicographic Gauss-Seidel relaxation (c/bmgs/relax.c:11-45) on the GPU.
//
// The reference sweeps the grid in C order, updating in place, so every point
// sees the new values of its lexicographically earlier neighbours and the old
// values of the later ones; periodic halo values are the copies made before
// the sweep (c/operators.c:75-85), i.e. old values.  The same update order is
// reproduced without a sequential loop by processing hyperplanes
//   t = a0 * i0 + a1 * i1 + i2
// in increasing t, with weights chosen so that every lexicographically
// negative offset lies on an earlier hyperplane and every positive one on a
// later hyperplane (a0 = a1 = 1 for star stencils; a1 = mp + 1,
// a0 = (mp + 2) mp + 1 for offsets anywhere in [-mp, mp]^3).  Points of one
// hyperplane are independent and are updated in parallel by one CTA, with a
// barrier between hyperplanes; each update uses the reference's unfused
// arithmetic, so float64 results are bit-identical.
#pragma once
#include "gpw_internal.h"

namespace gpw {

struct GsArgs {
  void* func;
  const void* src;
  void* old;  // snapshot of func at the start of each sweep (periodic halo values)
  GridView v, vs;
  Boundary bc;
  int nsweeps;
  int a0, a1;
  double cinv;  // 1 / coefs[0]
  const unsigned char* active;  // optional: skip when *active == 0
};

template <typename T>
__global__ void __launch_bounds__(1024) gs_relax_kernel(const GsArgs a, const GeneralCoefs k) {
  if (a.active && !*a.active) return;
  T* f = static_cast<T*>(a.func);
  const T* src = static_cast<const T*>(a.src);
  T* old = static_cast<T*>(a.old);
  const int n0 = a.v.n[0], n1 = a.v.n[1], n2 = a.v.n[2];
  const bool anyper = a.bc.periodic[0] || a.bc.periodic[1] || a.bc.periodic[2];
  const int tmax = a.a0 * (n0 - 1) + a.a1 * (n1 - 1) + (n2 - 1);
  for (int sw = 0; sw < a.nsweeps; ++sw) {
    if (anyper) {
      for (int64_t i = threadIdx.x; i < (int64_t)n0 * n1 * n2; i += blockDim.x) {
        const int i2 = (int)(i % n2);
        const int64_t r = i / n2;
        old[i] = f[(r / n1) * a.v.s0 + (r % n1) * a.v.s1 + i2];
      }
      __syncthreads();
    }
    for (int t = 0; t <= tmax; ++t) {
      for (int pq = threadIdx.x; pq < n0 * n1; pq += blockDim.x) {
        const int i0 = pq / n1, i1 = pq - i0 * n1;
        const int i2 = t - a.a0 * i0 - a.a1 * i1;
        if (i2 < 0 || i2 >= n2) continue;
        T x = zero<T>();
        for (int c = 1; c < k.ncoef; ++c) {
          const int g0 = i0 + k.off[c][0], g1 = i1 + k.off[c][1], g2 = i2 + k.off[c][2];
          T val;
          if (g0 >= 0 && g0 < n0 && g1 >= 0 && g1 < n1 && g2 >= 0 && g2 < n2) {
            val = f[(int64_t)g0 * a.v.s0 + (int64_t)g1 * a.v.s1 + g2];
          } else {
            int j0, j1, j2, s0, s1, s2;
            if (wrap_axis(g0, n0, a.bc.periodic[0], j0, s0) && wrap_axis(g1, n1, a.bc.periodic[1], j1, s1) &&
                wrap_axis(g2, n2, a.bc.periodic[2], j2, s2))
              val = old[((int64_t)j0 * n1 + j1) * n2 + j2];
            else
              val = zero<T>();
          }
          x = mac_rn((typename EltTraits<T>::S)k.coef[c], val, x);
        }
        const int64_t gi = (int64_t)i0 * a.v.s0 + (int64_t)i1 * a.v.s1 + i2;
        const T s = src[(int64_t)i0 * a.vs.s0 + (int64_t)i1 * a.vs.s1 + i2];
        f[gi] = (s - x) * (typename EltTraits<T>::S)a.cinv;
      }
      __syncthreads();
    }
  }
}

inline cudaError_t launch_relax_gs_ws(const OpDesc& d, int dtype, void* func, const GridView& v, const void* src,
                                      const GridView& vs, int nsweeps, const Boundary& bc, void* old,
                                      const unsigned char* active, cudaStream_t st) {
  GsArgs a{};
  a.func = func;
  a.src = src;
  a.old = old;
  a.v = v;
  a.vs = vs;
  a.bc = bc;
  a.nsweeps = nsweeps;
  if (d.star) {
    a.a0 = 1;
    a.a1 = 1;
  } else {
    a.a1 = d.mp + 1;
    a.a0 = (d.mp + 2) * d.mp + 1;
  }
  a.cinv = 1.0 / d.coefs[0];
  a.active = active;
  if (dtype == GPW_F64)
    gs_relax_kernel<double><<<1, 1024, 0, st>>>(a, d.gc);
  else if (dtype == GPW_F32)
    gs_relax_kernel<float><<<1, 1024, 0, st>>>(a, d.gc);
  else
    return cudaErrorInvalidValue;
  return cudaGetLastError();
}

// Convenience for the C ABI: snapshot buffer from a lazily grown workspace.
inline cudaError_t launch_relax_gs(const OpDesc& d, int dtype, void* func, const GridView& v, const void* src,
                                   const GridView& vs, int nsweeps, const Boundary& bc, cudaStream_t st) {
  static thread_local Workspace ws;
  const size_t bytes = elt_size(dtype) * (size_t)view_points(v);
  if (ws.ensure(bytes) != GPW_OK) return cudaErrorMemoryAllocation;
  return launch_relax_gs_ws(d, dtype, func, v, src, vs, nsweeps, bc, ws.ptr, nullptr, st);
}

}  // namespace gpw
