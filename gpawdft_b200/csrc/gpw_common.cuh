// Common device/host definitions for the B200 grid hot path.
//
// Grids are C-ordered 3D arrays (axis 0 slowest, axis 2 contiguous) with an
// optional leading batch axis, exactly as the reference stores them
// (gpaw/grid_descriptor.py:237-252).  Device kernels address a grid through
// a GridView: extent n[3], element strides s0, s1 (s2 == 1) and a batch stride,
// so that internally pitched buffers and the caller's contiguous arrays share
// one code path.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/gpwgrid.h"

namespace gpw {

// Programmatic dependent launch: a kernel launched with programmatic stream
// serialization may be dispatched while its predecessor in the stream still
// runs.  It calls pdl_wait() before its first access to global memory (the
// wait returns once the predecessor has finished and its writes are
// visible; without the launch attribute it returns at once), and
// pdl_trigger() once its own main loop is done, letting its successor's CTAs
// take SM slots as this grid drains.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;\n" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory"); }

// ------------------------------------------------------------------ scalars
// Element types: double (f64), float (f32), double2 (c128), float2 (c64).
// Coefficients are always real, as in the reference (bmgsstencil.coefs is
// double* for both the real and the complex instantiation, c/bmgs/bmgs.h:33).
template <typename T> struct EltTraits;
template <> struct EltTraits<double> {
  using S = double;
  static constexpr bool cpx = false;
};
template <> struct EltTraits<float> {
  using S = float;
  static constexpr bool cpx = false;
};
template <> struct EltTraits<double2> {
  using S = double;
  static constexpr bool cpx = true;
};
template <> struct EltTraits<float2> {
  using S = float;
  static constexpr bool cpx = true;
};

__host__ __device__ __forceinline__ double zero_of(double) { return 0.0; }
__host__ __device__ __forceinline__ float zero_of(float) { return 0.0f; }
__host__ __device__ __forceinline__ double2 zero_of(double2) { return make_double2(0.0, 0.0); }
__host__ __device__ __forceinline__ float2 zero_of(float2) { return make_float2(0.0f, 0.0f); }
template <typename T> __device__ __forceinline__ T zero() { return zero_of(T()); }

// acc + c * v  (fused)
__device__ __forceinline__ double fmac(double c, double v, double a) { return fma(c, v, a); }
__device__ __forceinline__ float fmac(float c, float v, float a) { return fmaf(c, v, a); }
__device__ __forceinline__ double2 fmac(double c, double2 v, double2 a) {
  return make_double2(fma(c, v.x, a.x), fma(c, v.y, a.y));
}
__device__ __forceinline__ float2 fmac(float c, float2 v, float2 a) {
  return make_float2(fmaf(c, v.x, a.x), fmaf(c, v.y, a.y));
}
// round-to-nearest multiply then add, never contracted: x + (a * c) exactly as
// the reference's `x += aa[offsets[c]] * coefs[c]` (c/bmgs/fd.c:42-43).
__device__ __forceinline__ double mac_rn(double c, double v, double a) {
  return __dadd_rn(a, __dmul_rn(v, c));
}
__device__ __forceinline__ float mac_rn(float c, float v, float a) {
  return __fadd_rn(a, __fmul_rn(v, c));
}
__device__ __forceinline__ double2 mac_rn(double c, double2 v, double2 a) {
  return make_double2(__dadd_rn(a.x, __dmul_rn(v.x, c)), __dadd_rn(a.y, __dmul_rn(v.y, c)));
}
__device__ __forceinline__ float2 mac_rn(float c, float2 v, float2 a) {
  return make_float2(__fadd_rn(a.x, __fmul_rn(v.x, c)), __fadd_rn(a.y, __fmul_rn(v.y, c)));
}

__device__ __forceinline__ double add(double a, double b) { return a + b; }
__device__ __forceinline__ float add(float a, float b) { return a + b; }
__device__ __forceinline__ double2 add(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 add(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double sub(double a, double b) { return a - b; }
__device__ __forceinline__ float sub(float a, float b) { return a - b; }
__device__ __forceinline__ double2 sub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 sub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double scale(double c, double a) { return c * a; }
__device__ __forceinline__ float scale(float c, float a) { return c * a; }
__device__ __forceinline__ double2 scale(double c, double2 a) { return make_double2(c * a.x, c * a.y); }
__device__ __forceinline__ float2 scale(float c, float2 a) { return make_float2(c * a.x, c * a.y); }
__device__ __forceinline__ double norm2(double a) { return a * a; }
__device__ __forceinline__ double norm2(float a) { return (double)a * (double)a; }
__device__ __forceinline__ double norm2(double2 a) { return a.x * a.x + a.y * a.y; }
__device__ __forceinline__ double norm2(float2 a) { return (double)a.x * a.x + (double)a.y * a.y; }

// Complex phase product p * v with the reference's C99 formula
// (re = pr vr - pi vi, im = pr vi + pi vr; c/bmgs/translate.c:40).
__device__ __forceinline__ double phase_mul(double2, double v) { return v; }
__device__ __forceinline__ float phase_mul(double2, float v) { return v; }
__device__ __forceinline__ double2 phase_mul(double2 p, double2 v) {
  return make_double2(__dsub_rn(__dmul_rn(p.x, v.x), __dmul_rn(p.y, v.y)),
                      __dadd_rn(__dmul_rn(p.x, v.y), __dmul_rn(p.y, v.x)));
}
// (complex64: the same formula in float, rounded after every operation, so
// that every kernel computes the same bits whatever the compiler contracts)
__device__ __forceinline__ float2 phase_mul(double2 p, float2 v) {
  const float px = (float)p.x, py = (float)p.y;
  return make_float2(__fsub_rn(__fmul_rn(px, v.x), __fmul_rn(py, v.y)),
                     __fadd_rn(__fmul_rn(px, v.y), __fmul_rn(py, v.x)));
}
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(__dsub_rn(__dmul_rn(a.x, b.x), __dmul_rn(a.y, b.y)),
                      __dadd_rn(__dmul_rn(a.x, b.y), __dmul_rn(a.y, b.x)));
}

// ------------------------------------------------------------------ boundary
// Serial boundary description of one grid (c/bc.c restated for one domain):
// per axis either a zero boundary (neighbour -1: the halo stays zero,
// c/bc.c:156) or a periodic wrap onto this same domain (neighbour == rank:
// bmgs_translate[mz], c/bc.c:234-249).  A value fetched from below the grid
// (index < 0) is the interior value n above it times ph[c][1]; above the grid
// (index >= n) it is the value n below times ph[c][0].  Corners take the
// product over the wrapped axes (the cfd == 0 chaining, c/bc.c:108-112).
struct Boundary {
  int periodic[3];
  int use_phase;  // complex data with non-trivial Bloch phases
  double2 ph[3][2];
};

// Map an index along one axis; returns false when the value is a zero halo.
__device__ __forceinline__ bool wrap_axis(int i, int n, int periodic, int& j, int& side) {
  side = -1;
  if (i >= 0 && i < n) {
    j = i;
    return true;
  }
  j = 0;
  if (!periodic) return false;
  if (i < 0) {
    j = i % n;
    if (j < 0) j += n;
    side = 1;
  } else {
    j = i % n;
    side = 0;
  }
  return true;
}

// ------------------------------------------------------------------ grid view
struct GridView {
  int n[3];
  int64_t s0, s1;      // element strides of axes 0 and 1 (axis 2 stride 1)
  int64_t sb;          // element stride between batch members
};

// ------------------------------------------------------------------ cp.async
__device__ __forceinline__ unsigned smem_u32(const void* p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
template <int BYTES>
__device__ __forceinline__ void cp_async(void* sdst, const void* gsrc, bool valid) {
  unsigned s = smem_u32(sdst);
  int src_size = valid ? BYTES : 0;
  if constexpr (BYTES == 16) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gsrc), "r"(src_size));
  } else {
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;\n" ::"r"(s), "l"(gsrc), "n"(BYTES),
                 "r"(src_size));
  }
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

}  // namespace gpw
