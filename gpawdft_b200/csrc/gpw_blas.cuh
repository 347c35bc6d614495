// Elementwise and reduction kernels for the NumPy / BLAS glue around the
// grid hot path (axpy / scal of gpaw/utilities/blas.py, integrate of
// gpaw/grid_descriptor.py:263-292, the in-place array arithmetic of
// gpaw/poisson.py and gpaw/preconditioner.py).  Vectorised grid-stride loops;
// reductions are deterministic (fixed per-thread order, fixed tree, partials
// summed in block order).
#pragma once
#include "gpw_common.cuh"
#include "gpw_reduce.cuh"

namespace gpw {

template <typename S>
__global__ void axpy_real_kernel(int64_t n, S alpha, const S* __restrict__ x, S* __restrict__ y) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (; i < n; i += stride) y[i] = fma(alpha, x[i], y[i]);
}

template <typename S2>
__global__ void axpy_cplx_kernel(int64_t n, double ar, double ai, const S2* __restrict__ x, S2* __restrict__ y) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (; i < n; i += stride) {
    S2 v = x[i], w = y[i];
    w.x = w.x + (ar * v.x - ai * v.y);
    w.y = w.y + (ar * v.y + ai * v.x);
    y[i] = w;
  }
}

template <typename S>
__global__ void scal_real_kernel(int64_t n, S alpha, S* __restrict__ x) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (; i < n; i += stride) x[i] = alpha * x[i];
}

template <typename S2>
__global__ void scal_cplx_kernel(int64_t n, double ar, double ai, S2* __restrict__ x) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (; i < n; i += stride) {
    S2 v = x[i];
    S2 w;
    w.x = ar * v.x - ai * v.y;
    w.y = ar * v.y + ai * v.x;
    x[i] = w;
  }
}

template <typename S>
__global__ void add_scalar_kernel(int64_t n, double c, const S* __restrict__ x, S* __restrict__ y) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (; i < n; i += stride) y[i] = x[i] + (S)c;
}

// Segmented sum / dot: vector m = blockIdx.y, CTAs of one vector = gridDim.x.
// OP 0: sum(x) (real; complex -> real and imaginary in two segments),
// OP 1: sum(conj(x) y) real part.
template <typename T, int OP>
__global__ void __launch_bounds__(256) reduce_kernel(int64_t n, const T* __restrict__ x,
                                                     const T* __restrict__ y, GridSum gs, int ncomp) {
  __shared__ double red[32];
  const int m = blockIdx.y;
  const T* xv = x + (int64_t)m * n;
  const T* yv = y ? y + (int64_t)m * n : nullptr;
  double s0 = 0.0, s1 = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    if constexpr (OP == 0) {
      if constexpr (EltTraits<T>::cpx) {
        s0 += (double)xv[i].x;
        s1 += (double)xv[i].y;
      } else {
        s0 += (double)xv[i];
      }
    } else {
      if constexpr (EltTraits<T>::cpx) {
        s0 += (double)xv[i].x * yv[i].x + (double)xv[i].y * yv[i].y;
      } else {
        s0 += (double)xv[i] * (double)yv[i];
      }
    }
  }
  double t0 = block_sum(s0, red);
  grid_sum_finish(gs, m * ncomp, blockIdx.x, gridDim.x, t0, red);
  if (ncomp == 2) {
    __syncthreads();
    double t1 = block_sum(s1, red);
    grid_sum_finish(gs, m * ncomp + 1, blockIdx.x, gridDim.x, t1, red);
  }
}

// Fill `n` elements with zero (used for phi_{l+1} = 0 inside captured graphs
// where a memset node would also do; a kernel keeps the batch mask).
template <typename T>
__global__ void zero_kernel(GridView v, T* __restrict__ x, const unsigned char* active) {
  const int b = blockIdx.y;
  if (active && !active[b]) return;
  const int64_t tot = (int64_t)v.n[0] * v.n[1] * v.n[2];
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < tot; i += (int64_t)gridDim.x * blockDim.x) {
    const int i2 = (int)(i % v.n[2]);
    const int64_t r = i / v.n[2];
    const int i1 = (int)(r % v.n[1]);
    const int i0 = (int)(r / v.n[1]);
    x[(int64_t)b * v.sb + i0 * v.s0 + i1 * v.s1 + i2] = zero<T>();
  }
}

}  // namespace gpw
