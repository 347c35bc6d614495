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

// Segmented sum / dot: segment m = blockIdx.y, CTAs of one segment = gridDim.x.
// OP 0: sum(x[m]) (real; complex -> real and imaginary in two segments),
// OP 1: real part of sum(conj(x[m]) y[m]),
// OP 2: sum(conj(x[m / ny]) y[m % ny]) over every (x, y) vector pair; complex
//       results take two segments (real, imaginary).
template <typename T, int OP>
__global__ void __launch_bounds__(256) reduce_kernel(int64_t n, const T* __restrict__ x,
                                                     const T* __restrict__ y, GridSum gs, int ncomp,
                                                     int ny) {
  __shared__ double red[32];
  const int m = blockIdx.y;
  const T* xv = x + (int64_t)(OP == 2 ? m / ny : m) * n;
  const T* yv = y ? y + (int64_t)(OP == 2 ? m % ny : m) * n : nullptr;
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
        const double xr = xv[i].x, xi = xv[i].y, yr = yv[i].x, yi = yv[i].y;
        s0 += xr * yr + xi * yi;
        if constexpr (OP == 2) s1 += xr * yi - xi * yr;
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

// The charge branches of PoissonSolver.solve (gpaw/poisson.py:209-299) for
// a batch of float64 densities, member b = blockIdx.y, after its sum(rho) is
// in sums[b]:
//   |charge| <= maxcharge, or every axis periodic:
//        rho_out = rho - charge / dv / npts            (the background shift)
//        (charged periodic with zero_phi: phi = 0)
//   charged, no periodic axis, Gaussians given:
//        q = charge / sqrt(4 pi); rho_out = rho - q rho_gauss;
//        phi = 0 (zero_phi) or phi - q phi_gauss       (poisson.py:286-293)
//   charged with mixed boundaries: q = NaN, rho_out = rho (the caller raises).
// charge = sums[b] dv; q_out[b] receives q (0 outside the Gaussian branch).
// The NumPy expressions are rounded as NumPy rounds them (no contraction);
// the axpy on phi fuses, as the BLAS axpy it replaces may.
__global__ void charge_prepare_kernel(int64_t n, const double* __restrict__ rho, double* __restrict__ rho_out,
                                      double* __restrict__ phi, const double* __restrict__ rho_g,
                                      const double* __restrict__ phi_g, const double* __restrict__ sums,
                                      double dv, double npts, double maxcharge, int all_periodic,
                                      int any_periodic, int zero_phi, double* __restrict__ q_out) {
  const int b = blockIdx.y;
  const double charge = __dmul_rn(sums[b], dv);
  int mode;  // 0 background shift, 1 Gaussian, 2 unsupported
  if (fabs(charge) <= maxcharge || all_periodic) mode = 0;
  else if (!any_periodic && rho_g && phi_g) mode = 1;
  else mode = 2;
  const double bg = __ddiv_rn(__ddiv_rn(charge, dv), npts);
  const double q = __ddiv_rn(charge, sqrt(4.0 * 3.14159265358979323846));
  const bool clear_phi = zero_phi && fabs(charge) > maxcharge && mode != 2;
  if (blockIdx.x == 0 && threadIdx.x == 0)
    q_out[b] = mode == 1 ? q : (mode == 2 ? __longlong_as_double(0x7ff8000000000000LL) : 0.0);
  const double* r = rho + (int64_t)b * n;
  double* ro = rho_out + (int64_t)b * n;
  double* ph = phi + (int64_t)b * n;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    if (mode == 0) {
      ro[i] = __dsub_rn(r[i], bg);
      if (clear_phi) ph[i] = 0.0;
    } else if (mode == 1) {
      ro[i] = __dsub_rn(r[i], __dmul_rn(q, rho_g[i]));
      ph[i] = clear_phi ? 0.0 : fma(-q, phi_g[i], ph[i]);
    } else {
      ro[i] = r[i];
    }
  }
}

// phi[b] += q[b] phi_gauss for the members of the Gaussian branch
// (gpaw/poisson.py:298-299).
__global__ void charge_finish_kernel(int64_t n, double* __restrict__ phi, const double* __restrict__ phi_g,
                                     const double* __restrict__ q_in) {
  const int b = blockIdx.y;
  const double q = q_in[b];
  if (!(q != 0.0) || isnan(q)) return;
  double* ph = phi + (int64_t)b * n;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    ph[i] = fma(q, phi_g[i], ph[i]);
}

// dst[dst_off + i] = src[src_off + i] for every index i of the box (grid
// extension / de-extension of the extended Poisson solver); element type T,
// contiguous (n0, n1, n2) grids.
template <typename T>
__global__ void copy_box_kernel(const T* __restrict__ src, int sn1, int sn2, int so0, int so1, int so2,
                                T* __restrict__ dst, int dn1, int dn2, int do0, int do1, int do2, int b0, int b1,
                                int b2) {
  const int64_t tot = (int64_t)b0 * b1 * b2;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < tot; i += (int64_t)gridDim.x * blockDim.x) {
    const int i2 = (int)(i % b2);
    const int64_t r = i / b2;
    const int i1 = (int)(r % b1), i0 = (int)(r / b1);
    dst[((int64_t)(i0 + do0) * dn1 + (i1 + do1)) * dn2 + (i2 + do2)] =
        src[((int64_t)(i0 + so0) * sn1 + (i1 + so1)) * sn2 + (i2 + so2)];
  }
}

// out = x * y elementwise (float64; rounded once, as NumPy's product).
__global__ void mul_kernel(int64_t n, const double* __restrict__ x, const double* __restrict__ y,
                           double* __restrict__ out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = __dmul_rn(x[i], y[i]);
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
