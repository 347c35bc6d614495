// C ABI (include/gpwgrid.h): operator and transformer handles, argument
// validation, in-place handling and the grid BLAS entry points.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <sstream>
#include <string>

#include "gpw_internal.h"
#include "gpw_relax_gs.cuh"

namespace gpw {

static thread_local std::string g_err;
void set_error(const std::string& msg) { g_err = msg; }
int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}
int cuda_fail(cudaError_t e, const char* what) {
  g_err = std::string(what) + ": " + cudaGetErrorString(e);
  return (e == cudaErrorMemoryAllocation) ? GPW_ENOMEM : GPW_ECUDA;
}

int Workspace::ensure(size_t need) {
  if (need <= bytes) return GPW_OK;
  if (ptr) {
    cudaDeviceSynchronize();
    cudaFree(ptr);
    ptr = nullptr;
    bytes = 0;
  }
  size_t nb = std::max(need, (size_t)256);
  cudaError_t e = cudaMalloc(&ptr, nb);
  if (e != cudaSuccess) {
    ptr = nullptr;
    return cuda_fail(e, "workspace allocation");
  }
  bytes = nb;
  return GPW_OK;
}
Workspace::~Workspace() {
  if (ptr) cudaFree(ptr);
}

int SumScratch::ensure(int64_t nseg, int64_t nblk_seg) {
  const bool grow_counter = (size_t)nseg * sizeof(unsigned) > counter.bytes;
  int rc = partial.ensure((size_t)(nseg * nblk_seg) * sizeof(double));
  if (rc) return rc;
  rc = counter.ensure((size_t)nseg * sizeof(unsigned));
  if (rc) return rc;
  if (grow_counter) {
    cudaError_t e = cudaMemset(counter.ptr, 0, counter.bytes);
    if (e != cudaSuccess) return cuda_fail(e, "counter init");
  }
  return result.ensure((size_t)nseg * sizeof(double));
}

Boundary make_boundary(const int periodic[3], int dtype, const double* phases) {
  Boundary b{};
  bool nontrivial = false;
  for (int c = 0; c < 3; ++c) {
    b.periodic[c] = periodic[c];
    for (int d = 0; d < 2; ++d) {
      double re = 1.0, im = 0.0;
      if (phases && is_complex(dtype)) {
        re = phases[(c * 2 + d) * 2];
        im = phases[(c * 2 + d) * 2 + 1];
      }
      b.ph[c][d] = make_double2(re, im);
      if (periodic[c] && (re != 1.0 || im != 0.0)) nontrivial = true;
    }
  }
  b.use_phase = (is_complex(dtype) && nontrivial) ? 1 : 0;
  return b;
}

static int parse_neighbors(const int64_t nb[6], int periodic[3]) {
  for (int c = 0; c < 3; ++c) {
    const int64_t a = nb[2 * c], b = nb[2 * c + 1];
    if (a == 0 && b == 0)
      periodic[c] = 1;
    else if (a == -1 && b == -1)
      periodic[c] = 0;
    else
      return fail(GPW_EINVAL, "neighbors: each axis must be (0, 0) periodic or (-1, -1) zero boundary "
                              "(serial domain; MPI neighbours are not supported)");
  }
  return GPW_OK;
}

int build_opdesc(OpDesc& d, const double* coefs, const int64_t* offsets, int ncoef, const int64_t size[3],
                 int range, const int64_t neighbors[6], int real, int cfd) {
  if (ncoef <= 0 || ncoef > PMAX) return fail(GPW_EINVAL, "ncoefs out of range (1.." + std::to_string(PMAX) + ")");
  if (range < 0 || range > 6) return fail(GPW_EINVAL, "range (padding) must be in 0..6");
  for (int c = 0; c < 3; ++c) {
    if (size[c] <= 0 || size[c] > (1 << 20)) return fail(GPW_EINVAL, "size must be positive");
    d.n[c] = (int)size[c];
  }
  int rc = parse_neighbors(neighbors, d.periodic);
  if (rc) return rc;
  for (int c = 0; c < 3; ++c)
    if (d.periodic[c] && d.n[c] < range)
      return fail(GPW_EINVAL, "periodic axis shorter than the stencil range");
  d.mp = range;
  d.real = real;
  d.cfd = cfd;
  d.ncoef = ncoef;
  d.coefs.assign(coefs, coefs + ncoef);
  d.off.resize(3 * ncoef);
  // decode linear offsets in the array padded by `range` (gpaw/fd_operators.py:50-52)
  const int64_t M1 = size[1] + 2 * range, M2 = size[2] + 2 * range;
  for (int p = 0; p < ncoef; ++p) {
    const int64_t o = offsets[p];
    int64_t o2 = ((o + range) % M2 + M2) % M2 - range;
    int64_t r = (o - o2) / M2;
    int64_t o1 = ((r + range) % M1 + M1) % M1 - range;
    int64_t o0 = (r - o1) / M1;
    if (std::llabs(o0) > range || std::llabs(o1) > range || std::llabs(o2) > range)
      return fail(GPW_EINVAL, "offset outside the padded range");
    d.off[3 * p] = (int)o0;
    d.off[3 * p + 1] = (int)o1;
    d.off[3 * p + 2] = (int)o2;
  }
  // get_diagonal_element: last coefficient with offset 0 (c/operators.c:414-418)
  d.diag = 0.0;
  for (int p = 0; p < ncoef; ++p)
    if (offsets[p] == 0) d.diag = coefs[p];
  // general kernel tables
  d.gc.ncoef = ncoef;
  d.gc.mp = range;
  for (int p = 0; p < ncoef; ++p) {
    d.gc.coef[p] = coefs[p];
    for (int k = 0; k < 3; ++k) d.gc.off[p][k] = (signed char)d.off[3 * p + k];
  }
  // star form: every offset on one axis
  bool star = true;
  int R = 0;
  for (int p = 0; p < ncoef; ++p) {
    int nz = 0;
    for (int k = 0; k < 3; ++k) {
      nz += d.off[3 * p + k] != 0;
      R = std::max(R, std::abs(d.off[3 * p + k]));
    }
    if (nz > 1) star = false;
  }
  R = std::max(R, 1);
  d.star = star && R <= 6;
  d.R = R;
  std::memset(&d.sc, 0, sizeof(d.sc));
  if (d.star) {
    for (int p = 0; p < ncoef; ++p) {
      const int* o = &d.off[3 * p];
      if (o[0] == 0 && o[1] == 0 && o[2] == 0)
        d.sc.cc += coefs[p];
      else if (o[0] != 0)
        d.sc.cx[o[0] + R] += coefs[p];
      else if (o[1] != 0)
        d.sc.cy[o[1] + R] += coefs[p];
      else
        d.sc.cz[o[2] + R] += coefs[p];
    }
  }
  // Jacobi on the star kernel: coefs[0] must be the (unique) centre, which the
  // reference assumes (c/bmgs/relax.c sums c = 1 .. ncoefs-1 and divides by c_0)
  int ncentre = 0;
  for (int p = 0; p < ncoef; ++p) ncentre += (offsets[p] == 0);
  d.star_jacobi = d.star && offsets[0] == 0 && ncentre == 1;
  return GPW_OK;
}

}  // namespace gpw

using namespace gpw;

struct gpw_operator {
  OpDesc d;
  Workspace scratch;
  SumScratch sums;
};

struct gpw_transformer {
  TrDesc d;
};

namespace gpw {
const OpDesc* operator_desc(const gpw_operator* op) { return &op->d; }
const TrDesc* transformer_desc(const gpw_transformer* tr) { return &tr->d; }
}  // namespace gpw

extern "C" {

const char* gpw_last_error(void) { return g_err.c_str(); }
const char* gpw_version(void) { return "gpwgrid 0.1 (sm_100a)"; }

int gpw_operator_new(const double* coefs, const int64_t* offsets, int ncoefs, const int64_t size[3], int range,
                     const int64_t neighbors[6], int real, int cfd, gpw_operator** out) {
  if (!coefs || !offsets || !size || !neighbors || !out) return fail(GPW_EINVAL, "null argument");
  gpw_operator* op = new gpw_operator();
  device_status_word();  // allocate outside any stream capture
  int rc = build_opdesc(op->d, coefs, offsets, ncoefs, size, range, neighbors, real, cfd);
  if (rc) {
    delete op;
    return rc;
  }
  *out = op;
  return GPW_OK;
}

void gpw_operator_free(gpw_operator* op) { delete op; }

int gpw_operator_get_diagonal_element(const gpw_operator* op, double* out) {
  if (!op || !out) return fail(GPW_EINVAL, "null argument");
  *out = op->d.diag;
  return GPW_OK;
}

static int operator_apply(gpw_operator* op, int dtype, const void* in, void* out, int64_t nin, const double* phases,
                          const void* pot, gpw_stream stream, const void* aux = nullptr, double aux_scale = 0.0) {
  if (!op || !in || !out) return fail(GPW_EINVAL, "null argument");
  if (!valid_dtype(dtype)) return fail(GPW_EINVAL, "bad dtype");
  if (nin < 0) return fail(GPW_EINVAL, "nin < 0");
  if (nin == 0) return GPW_OK;
  if (nin > 32768) {
    // grid.z = nchunk * nbatch; split very large batches
    const int64_t half = nin / 2;
    const size_t es = elt_size(dtype) * (size_t)op->d.n[0] * op->d.n[1] * op->d.n[2];
    int rc = operator_apply(op, dtype, in, out, half, phases, pot, stream, aux, aux_scale);
    if (rc) return rc;
    return operator_apply(op, dtype, (const char*)in + half * es, (char*)out + half * es, nin - half, phases, pot,
                          stream, aux ? (const char*)aux + half * es : nullptr, aux_scale);
  }
  cudaStream_t st = (cudaStream_t)stream;
  const OpDesc& d = op->d;
  GridView v = contiguous_view(d.n);
  const size_t bytes = elt_size(dtype) * (size_t)view_points(v) * (size_t)nin;
  const void* src = in;
  if (in == out) {  // the reference pastes into a private padded buffer first
    int rc = op->scratch.ensure(bytes);
    if (rc) return rc;
    cudaError_t e = cudaMemcpyAsync(op->scratch.ptr, in, bytes, cudaMemcpyDeviceToDevice, st);
    if (e != cudaSuccess) return cuda_fail(e, "operator apply copy");
    src = op->scratch.ptr;
  }
  Boundary bc = make_boundary(d.periodic, dtype, phases);
  GridSum gs{};
  cudaError_t e =
      launch_stencil(d, dtype, MODE_APPLY, src, v, out, v, nullptr, v, (int)nin, bc, 1.0, nullptr, gs, st, pot, aux,
                     aux_scale);
  if (e != cudaSuccess) return cuda_fail(e, "operator apply launch");
  return GPW_OK;
}

int gpw_operator_apply(gpw_operator* op, int dtype, const void* in, void* out, int64_t nin, const double* phases,
                       gpw_stream stream) {
  return operator_apply(op, dtype, in, out, nin, phases, nullptr, stream);
}

int gpw_operator_apply_fused(gpw_operator* op, int dtype, const void* in, void* out, int64_t nin,
                             const double* phases, const void* pot, const void* aux, double aux_scale,
                             gpw_stream stream) {
  if (pot && pot == out) return fail(GPW_EINVAL, "apply_fused: the potential must not alias the output");
  return operator_apply(op, dtype, in, out, nin, phases, pot, stream, aux, aux ? aux_scale : 0.0);
}

int gpw_operator_apply_potential(gpw_operator* op, int dtype, const void* in, void* out, int64_t nin,
                                 const double* phases, const void* pot, gpw_stream stream) {
  if (!pot) return fail(GPW_EINVAL, "apply_potential: null potential");
  if (pot == out) return fail(GPW_EINVAL, "apply_potential: the potential must not alias the output");
  return operator_apply(op, dtype, in, out, nin, phases, pot, stream);
}

int gpw_operator_residual(gpw_operator* op, int dtype, const void* func, const void* source, void* r, int64_t nin,
                          double* sumsq_dev, gpw_stream stream) {
  if (!op || !func || !source || !sumsq_dev) return fail(GPW_EINVAL, "null argument");
  if (dtype != GPW_F64 && dtype != GPW_F32) return fail(GPW_EINVAL, "residual: real dtypes only");
  if (nin <= 0 || nin > 4096) return fail(GPW_EINVAL, "residual: nin out of range");
  if (r == func) return fail(GPW_EINVAL, "residual: r must not alias func");
  cudaStream_t st = (cudaStream_t)stream;
  const OpDesc& d = op->d;
  GridView v = contiguous_view(d.n);
  const int nblk = stencil_blocks_per_member(d, MODE_RESIDUAL, v, (int)nin);
  int rc = op->sums.ensure(nin, nblk);
  if (rc) return rc;
  Boundary bc = make_boundary(d.periodic, dtype, nullptr);
  GridSum gs = op->sums.gs();
  cudaError_t e =
      launch_stencil(d, dtype, MODE_RESIDUAL, func, v, r, v, source, v, (int)nin, bc, 1.0, nullptr, gs, st);
  if (e != cudaSuccess) return cuda_fail(e, "residual launch");
  e = cudaMemcpyAsync(sumsq_dev, gs.result, sizeof(double) * nin, cudaMemcpyDeviceToDevice, st);
  if (e != cudaSuccess) return cuda_fail(e, "residual copy");
  return GPW_OK;
}

int gpw_operator_relax(gpw_operator* op, int dtype, int relax_method, void* func, const void* source, int64_t nin,
                       int nrelax, double w, gpw_stream stream) {
  if (!op || !func || !source) return fail(GPW_EINVAL, "null argument");
  if (dtype != GPW_F64 && dtype != GPW_F32) return fail(GPW_EINVAL, "relax: real dtypes only (c/operators.c:63)");
  if (relax_method != 1 && relax_method != 2) return fail(GPW_EINVAL, "relax_method must be 1 (GS) or 2 (J)");
  if (nin < 1 || nin > 32768) return fail(GPW_EINVAL, "relax: nin out of range");
  if (nrelax <= 0) return GPW_OK;
  cudaStream_t st = (cudaStream_t)stream;
  const OpDesc& d = op->d;
  GridView v = contiguous_view(d.n);
  const size_t bytes = elt_size(dtype) * (size_t)view_points(v);
  Boundary bc = make_boundary(d.periodic, dtype, nullptr);
  if (relax_method == 1) {
    for (int64_t m = 0; m < nin; ++m) {
      cudaError_t e = launch_relax_gs(d, dtype, (char*)func + m * bytes, v, (const char*)source + m * bytes, v,
                                      nrelax, bc, st);
      if (e != cudaSuccess) return cuda_fail(e, "Gauss-Seidel launch");
    }
    return GPW_OK;
  }
  int rc = op->scratch.ensure(bytes * nin);
  if (rc) return rc;
  GridSum gs{};
  void* a = func;
  void* b = op->scratch.ptr;
  for (int s = 0; s < nrelax; ++s) {
    cudaError_t e = launch_stencil(d, dtype, MODE_JACOBI, a, v, b, v, source, v, (int)nin, bc, w, nullptr, gs, st);
    if (e != cudaSuccess) return cuda_fail(e, "Jacobi launch");
    std::swap(a, b);
  }
  if (a != func) {
    cudaError_t e = cudaMemcpyAsync(func, a, bytes * nin, cudaMemcpyDeviceToDevice, st);
    if (e != cudaSuccess) return cuda_fail(e, "relax copy");
  }
  return GPW_OK;
}

int gpw_transformer_new(const int64_t size_in[3], const int64_t size_out[3], int k, const int64_t paddings[6],
                        const int64_t npaddings[6], const int64_t skip[6], const int64_t neighbors[6], int real,
                        int interpolate, gpw_transformer** out) {
  if (!size_in || !size_out || !paddings || !npaddings || !skip || !neighbors || !out)
    return fail(GPW_EINVAL, "null argument");
  if (k != 2 && k != 4 && k != 6 && k != 8) return fail(GPW_EINVAL, "k must be 2, 4, 6 or 8");
  gpw_transformer* t = new gpw_transformer();
  TrDesc& d = t->d;
  d.k = k;
  d.real = real;
  d.interpolate = interpolate ? 1 : 0;
  int rc = parse_neighbors(neighbors, d.periodic);
  if (rc) {
    delete t;
    return rc;
  }
  for (int c = 0; c < 3; ++c) {
    d.nin[c] = (int)size_in[c];
    d.nout[c] = (int)size_out[c];
    for (int s = 0; s < 2; ++s) {
      d.pad[c][s] = (int)paddings[2 * c + s];
      d.npad[c][s] = (int)npaddings[2 * c + s];
      d.skip[c][s] = (int)skip[2 * c + s];
    }
    if (d.nin[c] <= 0 || d.nout[c] <= 0 || d.pad[c][0] < 0 || d.pad[c][1] < 0) {
      delete t;
      return fail(GPW_EINVAL, "bad transformer sizes / paddings");
    }
    if (d.periodic[c] && (d.nin[c] < d.pad[c][0] || d.nin[c] < d.pad[c][1])) {
      delete t;
      return fail(GPW_EINVAL, "periodic axis shorter than the transformer halo");
    }
    // output extent implied by the reference's 1D loops
    const int L = d.nin[c] + d.pad[c][0] + d.pad[c][1];
    int expect;
    if (d.interpolate) {
      const int n = L - (k - 1) + d.skip[c][1];
      expect = 2 * n - d.skip[c][0] - d.skip[c][1];
    } else {
      expect = (L - (2 * k - 3)) / 2;
    }
    if (expect != d.nout[c]) {
      delete t;
      return fail(GPW_EINVAL, "size_out inconsistent with size_in, k and paddings");
    }
  }
  *out = t;
  return GPW_OK;
}

void gpw_transformer_free(gpw_transformer* t) { delete t; }

int gpw_transformer_apply(gpw_transformer* t, int dtype, const void* in, void* out, int64_t nin,
                          const double* phases, gpw_stream stream) {
  if (!t || !in || !out) return fail(GPW_EINVAL, "null argument");
  if (!valid_dtype(dtype)) return fail(GPW_EINVAL, "bad dtype");
  if (nin < 0) return fail(GPW_EINVAL, "nin < 0");
  if (nin == 0) return GPW_OK;
  if (in == out) return fail(GPW_EINVAL, "transformer input and output must differ");
  if (nin > 8192) {
    const int64_t half = nin / 2;
    const size_t ei = elt_size(dtype) * (size_t)t->d.nin[0] * t->d.nin[1] * t->d.nin[2];
    const size_t eo = elt_size(dtype) * (size_t)t->d.nout[0] * t->d.nout[1] * t->d.nout[2];
    int rc = gpw_transformer_apply(t, dtype, in, out, half, phases, stream);
    if (rc) return rc;
    return gpw_transformer_apply(t, dtype, (const char*)in + half * ei, (char*)out + half * eo, nin - half, phases,
                                 stream);
  }
  GridView vi = contiguous_view(t->d.nin), vo = contiguous_view(t->d.nout);
  Boundary bc = make_boundary(t->d.periodic, dtype, phases);
  cudaError_t e =
      launch_transfer(t->d, dtype, in, vi, out, vo, (int)nin, bc, 0, nullptr, nullptr, nullptr, (cudaStream_t)stream);
  if (e != cudaSuccess) return cuda_fail(e, "transformer launch");
  return GPW_OK;
}

int gpw_transformer_apply_subtract(gpw_transformer* t, int dtype, const void* in, const void* base, void* out,
                                   int64_t nin, const double* phases, gpw_stream stream) {
  if (!t || !in || !out || !base) return fail(GPW_EINVAL, "null argument");
  if (!valid_dtype(dtype)) return fail(GPW_EINVAL, "bad dtype");
  if (!t->d.interpolate) return fail(GPW_EINVAL, "apply_subtract: interpolating transformers only");
  if (nin <= 0 || nin > 8192) return fail(GPW_EINVAL, "apply_subtract: 1 <= nin <= 8192");
  if (in == out || base == out) return fail(GPW_EINVAL, "apply_subtract: out must differ from in and base");
  GridView vi = contiguous_view(t->d.nin), vo = contiguous_view(t->d.nout);
  Boundary bc = make_boundary(t->d.periodic, dtype, phases);
  cudaError_t e =
      launch_transfer(t->d, dtype, in, vi, out, vo, (int)nin, bc, 1, base, &vo, nullptr, (cudaStream_t)stream);
  if (e != cudaSuccess) return cuda_fail(e, "transformer launch");
  return GPW_OK;
}

int gpw_axpy(int dtype, int64_t n, double ar, double ai, const void* x, void* y, gpw_stream stream) {
  if (!valid_dtype(dtype) || n < 0) return fail(GPW_EINVAL, "axpy: bad arguments");
  if (n && (!x || !y)) return fail(GPW_EINVAL, "null argument");
  cudaError_t e = launch_axpy(dtype, n, ar, ai, x, y, (cudaStream_t)stream);
  return e == cudaSuccess ? GPW_OK : cuda_fail(e, "axpy");
}

int gpw_scal(int dtype, int64_t n, double ar, double ai, void* x, gpw_stream stream) {
  if (!valid_dtype(dtype) || n < 0) return fail(GPW_EINVAL, "scal: bad arguments");
  if (n && !x) return fail(GPW_EINVAL, "null argument");
  cudaError_t e = launch_scal(dtype, n, ar, ai, x, (cudaStream_t)stream);
  return e == cudaSuccess ? GPW_OK : cuda_fail(e, "scal");
}

int gpw_add_scalar(int dtype, int64_t n, double c, const void* x, void* y, gpw_stream stream) {
  if ((dtype != GPW_F64 && dtype != GPW_F32) || n < 0) return fail(GPW_EINVAL, "add_scalar: bad arguments");
  cudaError_t e = launch_add_scalar(dtype, n, c, x, y, (cudaStream_t)stream);
  return e == cudaSuccess ? GPW_OK : cuda_fail(e, "add_scalar");
}

static int reduce_common(int dtype, int op, int64_t nvec, int64_t n, const void* x, const void* y, double* out,
                         gpw_stream stream, int ny = 1) {
  if (!valid_dtype(dtype) || nvec <= 0 || n <= 0 || !x || !out || nvec > 65535)
    return fail(GPW_EINVAL, "reduction: bad arguments");
  static thread_local SumScratch scratch;
  const int nblk = reduce_blocks(n);
  const int ncomp = (op != 1 && is_complex(dtype)) ? 2 : 1;
  int rc = scratch.ensure(nvec * ncomp, nblk);
  if (rc) return rc;
  GridSum gs = scratch.gs();
  cudaStream_t st = (cudaStream_t)stream;
  cudaError_t e = launch_reduce(dtype, op, nvec, n, x, y, gs, nblk, st, ny);
  if (e != cudaSuccess) return cuda_fail(e, "reduction launch");
  e = cudaMemcpyAsync(out, gs.result, sizeof(double) * nvec * ncomp, cudaMemcpyDeviceToDevice, st);
  return e == cudaSuccess ? GPW_OK : cuda_fail(e, "reduction copy");
}

int gpw_sum(int dtype, int64_t nvec, int64_t n, const void* x, double* out_dev, gpw_stream stream) {
  return reduce_common(dtype, 0, nvec, n, x, nullptr, out_dev, stream);
}

int gpw_dot(int dtype, int64_t nvec, int64_t n, const void* x, const void* y, double* out_dev, gpw_stream stream) {
  if (!y) return fail(GPW_EINVAL, "null argument");
  return reduce_common(dtype, 1, nvec, n, x, y, out_dev, stream);
}

int gpw_poisson_charge_prepare(int64_t nb, int64_t n, const double* rho, double* rho_out, double* phi,
                               const double* rho_gauss, const double* phi_gauss, double dv, double npts_global,
                               double maxcharge, int pbc_mask, int zero_initial_phi, double* q_dev,
                               gpw_stream stream) {
  if (nb <= 0 || nb > 65535 || n <= 0 || !rho || !rho_out || !phi || !q_dev || !(dv > 0) || !(npts_global > 0))
    return fail(GPW_EINVAL, "charge_prepare: bad arguments");
  if (rho_out == rho) return fail(GPW_EINVAL, "charge_prepare: rho_out must not alias rho");
  if ((rho_gauss == nullptr) != (phi_gauss == nullptr))
    return fail(GPW_EINVAL, "charge_prepare: give both Gaussian arrays or neither");
  static thread_local SumScratch scratch;
  const int nblk = reduce_blocks(n);
  int rc = scratch.ensure(nb, nblk);
  if (rc) return rc;
  GridSum gs = scratch.gs();
  cudaStream_t st = (cudaStream_t)stream;
  cudaError_t e = launch_reduce(GPW_F64, 0, nb, n, rho, nullptr, gs, nblk, st);
  if (e != cudaSuccess) return cuda_fail(e, "charge_prepare: reduction");
  const int all_p = (pbc_mask & 7) == 7, any_p = (pbc_mask & 7) != 0;
  e = launch_charge_prepare(nb, n, rho, rho_out, phi, rho_gauss, phi_gauss, gs.result, dv, npts_global, maxcharge,
                            all_p, any_p, zero_initial_phi, q_dev, st);
  return e == cudaSuccess ? GPW_OK : cuda_fail(e, "charge_prepare");
}

int gpw_poisson_charge_finish(int64_t nb, int64_t n, double* phi, const double* phi_gauss, const double* q_dev,
                              gpw_stream stream) {
  if (nb <= 0 || nb > 65535 || n <= 0 || !phi || !q_dev) return fail(GPW_EINVAL, "charge_finish: bad arguments");
  if (!phi_gauss) return GPW_OK;
  cudaError_t e = launch_charge_finish(nb, n, phi, phi_gauss, q_dev, (cudaStream_t)stream);
  return e == cudaSuccess ? GPW_OK : cuda_fail(e, "charge_finish");
}

int gpw_copy_box(int dtype, const void* src, const int64_t src_n[3], const int64_t src_off[3], void* dst,
                 const int64_t dst_n[3], const int64_t dst_off[3], const int64_t box[3], gpw_stream stream) {
  if (!valid_dtype(dtype) || !src || !dst || !src_n || !src_off || !dst_n || !dst_off || !box)
    return fail(GPW_EINVAL, "copy_box: bad arguments");
  int sn[3], so[3], dn[3], dof[3], b[3];
  for (int c = 0; c < 3; ++c) {
    if (box[c] < 0 || src_off[c] < 0 || dst_off[c] < 0 || src_off[c] + box[c] > src_n[c] ||
        dst_off[c] + box[c] > dst_n[c] || src_n[c] > (1 << 20) || dst_n[c] > (1 << 20))
      return fail(GPW_EINVAL, "copy_box: the box leaves a grid");
    sn[c] = (int)src_n[c];
    so[c] = (int)src_off[c];
    dn[c] = (int)dst_n[c];
    dof[c] = (int)dst_off[c];
    b[c] = (int)box[c];
  }
  cudaError_t e = launch_copy_box(dtype, src, sn, so, dst, dn, dof, b, (cudaStream_t)stream);
  return e == cudaSuccess ? GPW_OK : cuda_fail(e, "copy_box");
}

int gpw_mul(int64_t n, const double* x, const double* y, double* out, gpw_stream stream) {
  if (n < 0 || (n && (!x || !y || !out))) return fail(GPW_EINVAL, "mul: bad arguments");
  if (!n) return GPW_OK;
  cudaError_t e = launch_mul(n, x, y, out, (cudaStream_t)stream);
  return e == cudaSuccess ? GPW_OK : cuda_fail(e, "mul");
}

static std::string tune_header() {
  int dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceProp p{};
  cudaGetDeviceProperties(&p, dev);
  std::string name(p.name);
  for (char& ch : name)
    if (ch == ' ') ch = '_';
  return "gpwgrid-tune 1 sms " + std::to_string(num_sms()) + " device " + name + "\n";
}

int gpw_tune_export(char* buf, int64_t cap, int64_t* needed) {
  if (!needed) return fail(GPW_EINVAL, "tune_export: null argument");
  std::string text = tune_header();
  tune_export_tma(text);
  tune_export_bloch(text);
  *needed = (int64_t)text.size() + 1;
  if (!buf || cap < *needed) return buf ? fail(GPW_EINVAL, "tune_export: buffer too small") : GPW_OK;
  std::memcpy(buf, text.c_str(), text.size() + 1);
  return GPW_OK;
}

int gpw_tune_import(const char* text, int* imported) {
  if (!text) return fail(GPW_EINVAL, "tune_import: null argument");
  std::istringstream in(text);
  std::string line;
  if (!std::getline(in, line) || line + "\n" != tune_header())
    return fail(GPW_EINVAL, "tune_import: records of another device or SM count (header mismatch)");
  int n = 0;
  while (std::getline(in, line)) {
    std::istringstream ls(line);
    std::string kind;
    ls >> kind;
    int f[11];
    const int want = kind == "tma" ? 9 : (kind == "bloch" ? 11 : 0);
    int got = 0;
    while (got < want && (ls >> f[got])) ++got;
    if (!want || got != want) continue;
    if (kind == "tma" ? tune_import_tma(f) : tune_import_bloch(f)) ++n;
  }
  if (imported) *imported = n;
  return GPW_OK;
}

int gpw_dotc_pairs(int dtype, int64_t nx, int64_t ny, int64_t n, const void* x, const void* y, double* out_dev,
                   gpw_stream stream) {
  if (!y) return fail(GPW_EINVAL, "null argument");
  if (nx <= 0 || ny <= 0 || nx * ny > 65535) return fail(GPW_EINVAL, "dotc_pairs: 1 <= nx * ny <= 65535");
  return reduce_common(dtype, 2, nx * ny, n, x, y, out_dev, stream, (int)ny);
}

}  // extern "C"
