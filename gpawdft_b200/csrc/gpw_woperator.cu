// Weighted finite-difference operator on the GPU: the operator of the
// dielectric Poisson solver (gpaw/solvation/poisson.py), A = sum_i w_i(r) S_i
// with per-point weight grids w_i and stencils S_i (a Laplacian and three
// gradients scaled by -1/4pi: A phi = -div(eps grad phi) / 4pi).  Replaces
// _gpaw.WOperator (c/woperators.c) with its kernels c/bmgs/wfd.c (apply) and
// c/bmgs/wrelax.c (weighted Jacobi and Gauss-Seidel).
//
// Apply and Jacobi: tiles of GEN_TZ x GEN_TY points march along axis 0 over
// a ring of 2 mp + 2 input planes staged by cp.async with their halo (zero,
// periodic or Bloch, as the plain operator's general kernel stages them).
// Every output point forms, per stencil, its tap sum, scales it by that
// stencil's weight at the point and adds it -- the reference's order, with
// unfused multiplies and adds, so float64 results are bit-identical.
// Gauss-Seidel: lexicographic order reproduced by hyperplanes (as the plain
// operator's Gauss-Seidel kernel), one CTA.
#include <algorithm>
#include <cstring>
#include <string>

#include "gpw_internal.h"
#include "gpw_stencil.cuh"

namespace gpw {

constexpr int WMAX = 4;    // stencils (weights) per operator
constexpr int WPMAX = 40;  // taps per stencil

struct WStencils {
  int nw, mp;
  int ncoef[WMAX];
  double coef[WMAX][WPMAX];
  signed char off[WMAX][WPMAX][3];
};

struct WArgs {
  const void* in;
  void* out;
  const double* src;        // Jacobi / Gauss-Seidel right-hand side
  const double* w[WMAX];    // weight grids (one grid each, contiguous)
  GridView v;               // contiguous (nin, n0, n1, n2)
  Boundary bc;
  int zchunk, nchunk;
  double relax_w;           // Jacobi weight
};

__device__ __forceinline__ double scale_rn(double w, double t) { return __dmul_rn(t, w); }
__device__ __forceinline__ double2 scale_rn(double w, double2 t) {
  return make_double2(__dmul_rn(t.x, w), __dmul_rn(t.y, w));
}
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double2 add_rn(double2 a, double2 b) {
  return make_double2(__dadd_rn(a.x, b.x), __dadd_rn(a.y, b.y));
}

// MODE 0: out = A in; MODE 1: one weighted Jacobi sweep of A f = src
// (c/bmgs/wrelax.c:63-95), in = the iterate before the sweep.
template <typename T, int MODE>
__global__ void __launch_bounds__(GEN_TZ* GEN_TY) wstencil_kernel(const WArgs a, const WStencils k) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* ring = reinterpret_cast<T*>(smem_raw);
  const int mp = k.mp;
  const int H = GEN_TY + 2 * mp, W = GEN_TZ + 2 * mp, PS = H * W, NP = 2 * mp + 2;
  const int b = blockIdx.z / a.nchunk, chunk = blockIdx.z - b * a.nchunk;
  const int x0 = blockIdx.x * GEN_TZ, y0 = blockIdx.y * GEN_TY;
  const int n0 = a.v.n[0];
  const int z0 = chunk * a.zchunk;
  const int z1 = min(n0, z0 + a.zchunk);
  const T* in = static_cast<const T*>(a.in) + (int64_t)b * a.v.sb;
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int y = y0 + ty, x = x0 + tx;
  const bool inside = (y < a.v.n[1]) && (x < a.v.n[2]);
  if (z0 >= z1) return;
  for (int p = z0 - mp; p <= z0 + mp; ++p)
    load_plane<T>(ring + ((p - z0 + mp) % NP) * PS, in, a.v, a.bc, p, y0, x0, mp, H, W);
  cp_async_commit();
  for (int o = z0; o < z1; ++o) {
    const int pn = o + mp + 1;
    if (o + 1 < z1) load_plane<T>(ring + ((pn - z0 + mp) % NP) * PS, in, a.v, a.bc, pn, y0, x0, mp, H, W);
    cp_async_commit();
    cp_async_wait<1>();
    if (a.bc.use_phase) {
      if (o == z0) {
        for (int p = z0 - mp; p <= z0 + mp; ++p)
          fix_plane<T>(ring + ((p - z0 + mp) % NP) * PS, a.v, a.bc, p, y0, x0, mp, H, W);
      } else {
        fix_plane<T>(ring + ((o + mp - z0 + mp) % NP) * PS, a.v, a.bc, o + mp, y0, x0, mp, H, W);
      }
    }
    __syncthreads();
    if (inside) {
      const int64_t gi = (int64_t)o * a.v.s0 + (int64_t)y * a.v.s1 + x;  // within one grid
      T acc = zero<T>();
      double cdiag = 0.0;
      for (int iw = 0; iw < k.nw; ++iw) {
        T tmp = zero<T>();
        for (int c = (MODE == 1) ? 1 : 0; c < k.ncoef[iw]; ++c) {
          const int p = o + k.off[iw][c][0];
          const T* sl = ring + ((p - z0 + mp) % NP) * PS;
          tmp = mac_rn(k.coef[iw][c], sl[(ty + mp + k.off[iw][c][1]) * W + tx + mp + k.off[iw][c][2]], tmp);
        }
        const double wv = a.w[iw][gi];
        acc = add_rn(acc, scale_rn(wv, tmp));
        if (MODE == 1) cdiag = __dadd_rn(cdiag, __dmul_rn(wv, k.coef[iw][0]));
      }
      T* outp = static_cast<T*>(a.out) + (int64_t)b * a.v.sb + gi;
      if constexpr (MODE == 0) {
        *outp = acc;
      } else if constexpr (!EltTraits<T>::cpx) {
        // (1 - w) b + w (src - x) / coef, evaluated as the reference does
        const T* sl = ring + ((o - z0 + mp) % NP) * PS;
        const double cur = sl[(ty + mp) * W + tx + mp];
        const double w = a.relax_w;
        const double s = a.src[(int64_t)b * a.v.sb + gi];
        *outp = __dadd_rn(__dmul_rn(__dsub_rn(1.0, w), cur), __ddiv_rn(__dmul_rn(w, __dsub_rn(s, acc)), cdiag));
      }
    }
    __syncthreads();
  }
}

// Weighted lexicographic Gauss-Seidel (c/bmgs/wrelax.c:24-57) over
// hyperplanes t = a0 i0 + a1 i1 + i2, one CTA; periodic halo values are the
// snapshot `old` taken before each sweep.
struct WgsArgs {
  double* func;
  const double* src;
  double* old;
  const double* w[WMAX];
  GridView v;
  Boundary bc;
  int nsweeps, a0, a1;
};

__global__ void __launch_bounds__(1024) wgs_relax_kernel(const WgsArgs a, const WStencils k) {
  double* f = a.func;
  const int n0 = a.v.n[0], n1 = a.v.n[1], n2 = a.v.n[2];
  const bool anyper = a.bc.periodic[0] || a.bc.periodic[1] || a.bc.periodic[2];
  const int tmax = a.a0 * (n0 - 1) + a.a1 * (n1 - 1) + (n2 - 1);
  for (int sw = 0; sw < a.nsweeps; ++sw) {
    if (anyper) {
      for (int64_t i = threadIdx.x; i < (int64_t)n0 * n1 * n2; i += blockDim.x) a.old[i] = f[i];
      __syncthreads();
    }
    for (int t = 0; t <= tmax; ++t) {
      for (int pq = threadIdx.x; pq < n0 * n1; pq += blockDim.x) {
        const int i0 = pq / n1, i1 = pq - i0 * n1;
        const int i2 = t - a.a0 * i0 - a.a1 * i1;
        if (i2 < 0 || i2 >= n2) continue;
        const int64_t gi = ((int64_t)i0 * n1 + i1) * n2 + i2;
        double x = 0.0, cdiag = 0.0;
        for (int iw = 0; iw < k.nw; ++iw) {
          double tmp = 0.0;
          for (int c = 1; c < k.ncoef[iw]; ++c) {
            const int g0 = i0 + k.off[iw][c][0], g1 = i1 + k.off[iw][c][1], g2 = i2 + k.off[iw][c][2];
            double val;
            if (g0 >= 0 && g0 < n0 && g1 >= 0 && g1 < n1 && g2 >= 0 && g2 < n2) {
              val = f[((int64_t)g0 * n1 + g1) * n2 + g2];
            } else {
              int j0, j1, j2, s0, s1, s2;
              if (wrap_axis(g0, n0, a.bc.periodic[0], j0, s0) && wrap_axis(g1, n1, a.bc.periodic[1], j1, s1) &&
                  wrap_axis(g2, n2, a.bc.periodic[2], j2, s2))
                val = a.old[((int64_t)j0 * n1 + j1) * n2 + j2];
              else
                val = 0.0;
            }
            tmp = mac_rn(k.coef[iw][c], val, tmp);
          }
          const double wv = a.w[iw][gi];
          x = __dadd_rn(x, __dmul_rn(tmp, wv));
          cdiag = __dadd_rn(cdiag, __dmul_rn(wv, k.coef[iw][0]));
        }
        f[gi] = __ddiv_rn(__dsub_rn(a.src[gi], x), cdiag);
      }
      __syncthreads();
    }
  }
}

// max over the grid of |sum_i w_i c_i0| (WOperator_get_diagonal_element,
// c/woperators.c:466-496); non-negative doubles order as their bit patterns.
__global__ void wdiag_kernel(int64_t n, WArgs a, WStencils k, unsigned long long* out) {
  double m = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double c = 0.0;
    for (int iw = 0; iw < k.nw; ++iw) c = __dadd_rn(c, __dmul_rn(a.w[iw][i], k.coef[iw][0]));
    m = fmax(m, fabs(c));
  }
  atomicMax(out, (unsigned long long)__double_as_longlong(m));
}

}  // namespace gpw

using namespace gpw;

struct gpw_woperator {
  int n[3], periodic[3], mp, real;
  bool star;
  WStencils k;
  Workspace scratch, dmax;
};

namespace {

void chunks(int n0, int64_t tiles, int mp, int& zchunk, int& nchunk) {
  const int64_t want = 4LL * num_sms();
  int64_t nc = (want + tiles - 1) / std::max<int64_t>(tiles, 1);
  const int minz = 2 * mp + 2;
  nc = std::max<int64_t>(1, std::min<int64_t>(nc, std::max(1, (n0 + minz - 1) / minz)));
  zchunk = (int)((n0 + nc - 1) / nc);
  nchunk = (n0 + zchunk - 1) / zchunk;
}

int fill_weights(const gpw_woperator* op, const double* const* weights, WArgs& a) {
  if (!weights) return fail(GPW_EINVAL, "woperator: null weights");
  for (int i = 0; i < op->k.nw; ++i) {
    if (!weights[i]) return fail(GPW_EINVAL, "woperator: null weight grid");
    a.w[i] = weights[i];
  }
  return GPW_OK;
}

template <typename T, int MODE>
cudaError_t run_wstencil(const gpw_woperator* op, WArgs a, int nbatch, cudaStream_t st) {
  const int mp = op->k.mp;
  dim3 grid((a.v.n[2] + GEN_TZ - 1) / GEN_TZ, (a.v.n[1] + GEN_TY - 1) / GEN_TY, 1);
  chunks(a.v.n[0], (int64_t)grid.x * grid.y * nbatch, mp, a.zchunk, a.nchunk);
  grid.z = a.nchunk * nbatch;
  const size_t smem = (size_t)(2 * mp + 2) * (GEN_TY + 2 * mp) * (GEN_TZ + 2 * mp) * sizeof(T);
  if (smem > 200 * 1024) return cudaErrorInvalidValue;
  auto kern = wstencil_kernel<T, MODE>;
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  kern<<<grid, dim3(GEN_TZ, GEN_TY), smem, st>>>(a, op->k);
  return cudaGetLastError();
}

}  // namespace

extern "C" {

int gpw_woperator_new(int nweights, const double* const* coefs, const int64_t* const* offsets, const int* ncoefs,
                      const int64_t size[3], int range, const int64_t neighbors[6], int real, int cfd,
                      gpw_woperator** out) {
  if (!coefs || !offsets || !ncoefs || !size || !neighbors || !out) return fail(GPW_EINVAL, "null argument");
  if (nweights < 1 || nweights > WMAX)
    return fail(GPW_EINVAL, "woperator: 1.." + std::to_string(WMAX) + " weights");
  gpw_woperator* op = new gpw_woperator();
  std::memset(&op->k, 0, sizeof(op->k));
  op->k.nw = nweights;
  op->k.mp = range;
  op->star = true;
  device_status_word();
  for (int i = 0; i < nweights; ++i) {
    OpDesc d;
    int rc = (ncoefs[i] > WPMAX)
                 ? fail(GPW_EINVAL, "woperator: at most " + std::to_string(WPMAX) + " taps per stencil")
                 : build_opdesc(d, coefs[i], offsets[i], ncoefs[i], size, range, neighbors, real, cfd);
    if (!rc && offsets[i][0] != 0) rc = fail(GPW_EINVAL, "woperator: every stencil's first offset must be 0");
    if (rc) {
      delete op;
      return rc;
    }
    if (i == 0) {
      for (int c = 0; c < 3; ++c) {
        op->n[c] = d.n[c];
        op->periodic[c] = d.periodic[c];
      }
    }
    op->star = op->star && d.star;
    op->k.ncoef[i] = ncoefs[i];
    for (int c = 0; c < ncoefs[i]; ++c) {
      op->k.coef[i][c] = coefs[i][c];
      for (int a = 0; a < 3; ++a) op->k.off[i][c][a] = (signed char)d.off[3 * c + a];
    }
  }
  op->mp = range;
  op->real = real;
  *out = op;
  return GPW_OK;
}

void gpw_woperator_free(gpw_woperator* op) { delete op; }

int gpw_woperator_apply(gpw_woperator* op, int dtype, const double* const* weights, const void* in, void* out,
                        int64_t nin, const double* phases, gpw_stream stream) {
  if (!op || !in || !out) return fail(GPW_EINVAL, "null argument");
  if (dtype != GPW_F64 && dtype != GPW_C128) return fail(GPW_EINVAL, "woperator: float64 or complex128 grids");
  if (nin < 0 || nin > 4096) return fail(GPW_EINVAL, "woperator: nin out of range");
  if (nin == 0) return GPW_OK;
  WArgs a{};
  int rc = fill_weights(op, weights, a);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  a.v = contiguous_view(op->n);
  const size_t bytes = elt_size(dtype) * (size_t)view_points(a.v) * (size_t)nin;
  a.in = in;
  if (in == out) {
    if ((rc = op->scratch.ensure(bytes))) return rc;
    cudaError_t e = cudaMemcpyAsync(op->scratch.ptr, in, bytes, cudaMemcpyDeviceToDevice, st);
    if (e != cudaSuccess) return cuda_fail(e, "woperator apply copy");
    a.in = op->scratch.ptr;
  }
  a.out = out;
  a.bc = make_boundary(op->periodic, dtype, phases);
  cudaError_t e = dtype == GPW_F64 ? run_wstencil<double, 0>(op, a, (int)nin, st)
                                   : run_wstencil<double2, 0>(op, a, (int)nin, st);
  return e == cudaSuccess ? GPW_OK : cuda_fail(e, "woperator apply launch");
}

int gpw_woperator_relax(gpw_woperator* op, int relax_method, const double* const* weights, double* func,
                        const double* source, int nrelax, double w, gpw_stream stream) {
  if (!op || !func || !source) return fail(GPW_EINVAL, "null argument");
  if (relax_method != 1 && relax_method != 2) return fail(GPW_EINVAL, "relax_method must be 1 (GS) or 2 (J)");
  if (nrelax <= 0) return GPW_OK;
  WArgs a{};
  int rc = fill_weights(op, weights, a);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  a.v = contiguous_view(op->n);
  const size_t bytes = sizeof(double) * (size_t)view_points(a.v);
  if ((rc = op->scratch.ensure(bytes))) return rc;
  a.bc = make_boundary(op->periodic, GPW_F64, nullptr);
  if (relax_method == 1) {
    WgsArgs g{};
    g.func = func;
    g.src = source;
    g.old = static_cast<double*>(op->scratch.ptr);
    for (int i = 0; i < op->k.nw; ++i) g.w[i] = a.w[i];
    g.v = a.v;
    g.bc = a.bc;
    g.nsweeps = nrelax;
    if (op->star) {
      g.a0 = g.a1 = 1;
    } else {
      g.a1 = op->mp + 1;
      g.a0 = (op->mp + 2) * op->mp + 1;
    }
    wgs_relax_kernel<<<1, 1024, 0, st>>>(g, op->k);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? GPW_OK : cuda_fail(e, "woperator Gauss-Seidel launch");
  }
  a.src = source;
  a.relax_w = w;
  for (int s = 0; s < nrelax; ++s) {
    // each sweep reads the iterate as it stood before the sweep
    cudaError_t e = cudaMemcpyAsync(op->scratch.ptr, func, bytes, cudaMemcpyDeviceToDevice, st);
    if (e != cudaSuccess) return cuda_fail(e, "woperator relax copy");
    a.in = op->scratch.ptr;
    a.out = func;
    e = run_wstencil<double, 1>(op, a, 1, st);
    if (e != cudaSuccess) return cuda_fail(e, "woperator Jacobi launch");
  }
  return GPW_OK;
}

int gpw_woperator_get_diagonal_element(gpw_woperator* op, const double* const* weights, double* out,
                                       gpw_stream stream) {
  if (!op || !out) return fail(GPW_EINVAL, "null argument");
  WArgs a{};
  int rc = fill_weights(op, weights, a);
  if (rc) return rc;
  if ((rc = op->dmax.ensure(sizeof(unsigned long long)))) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  cudaError_t e = cudaMemsetAsync(op->dmax.ptr, 0, sizeof(unsigned long long), st);
  if (e != cudaSuccess) return cuda_fail(e, "woperator diagonal clear");
  const int64_t n = (int64_t)op->n[0] * op->n[1] * op->n[2];
  const unsigned blocks = (unsigned)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 4LL * num_sms()));
  wdiag_kernel<<<blocks, 256, 0, st>>>(n, a, op->k, static_cast<unsigned long long*>(op->dmax.ptr));
  if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "woperator diagonal launch");
  unsigned long long bits = 0;
  e = cudaMemcpyAsync(&bits, op->dmax.ptr, sizeof(bits), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_fail(e, "woperator diagonal readback");
  std::memcpy(out, &bits, sizeof(double));
  return GPW_OK;
}

}  // extern "C"
