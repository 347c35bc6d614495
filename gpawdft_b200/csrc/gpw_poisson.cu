// Multigrid Poisson engine: the V-cycle of FDPoissonSolver.iterate2 and the
// convergence loop of solve_neutral (gpaw/poisson.py:306-366) on the device.
//
// One V-cycle for level l < L (L = coarsest):
//   relax(l, presmooths[l])            Jacobi sweeps, ping-pong buffers
//   r_l = A_l phi_l - rho_l            fused residual kernel
//   rho_{l+1} = R r_l ; phi_{l+1} = 0
//   V-cycle(l+1)
//   phi_l = phi_l - I phi_{l+1}        interpolation with fused subtraction
// then for every level relax(l, postsmooths[l]) and at level 0 the fused
// residual + deterministic sum(r^2) that gives error = sum(r^2) dv.
//
// The whole V-cycle (plus the per-solve convergence update) is captured once
// per batch size into a CUDA graph whose buffers are all engine-owned; a
// solve copies phi / rho in, replays the graph until every solve of the batch
// has converged, and copies phi out.  Independent same-grid solves are
// batched through every kernel (grid z = chunks x batch); a per-solve
// `active` mask freezes solves that have converged, so each solve's result
// and iteration count equal those of solving it alone.
#include <algorithm>
#include <cstring>
#include <string>
#include <map>
#include <memory>
#include <mutex>
#include <vector>

#include "gpw_coarse.cuh"
#include "gpw_internal.h"
#include "gpw_relax_gs.cuh"

namespace gpw {

struct Level {
  const OpDesc* op = nullptr;
  const TrDesc* restr = nullptr;   // level l -> l+1
  const TrDesc* interp = nullptr;  // level l+1 -> l
  GridView v;
  int pre = 0, post = 0;
  double w = 1.0;
  // per-sweep Jacobi weights, [0] float64 method, [1] float32 inner cycles
  std::vector<double> wpre[2], wpost[2];
  // float64 buffers (nbatch_max grids each)
  Workspace phi[2], rho, res;
  // float32 buffers for the defect-correction form
  Workspace phi32[2], rho32, res32;
};

__device__ __forceinline__ int64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return (int64_t)t;
}

// The convergence test of solve_neutral after each iteration.  A solve that
// stops records the device clock in tdone[b]; with a conditional handle the
// kernel also sets the condition of the graph's device-side while loop.
__global__ void converge_update_kernel(int nbatch, const double* __restrict__ sumsq, double dv,
                                       const double* __restrict__ eps, const int* __restrict__ maxiter_p,
                                       double* __restrict__ err,
                                       int* __restrict__ niter, unsigned char* __restrict__ active,
                                       int* __restrict__ any_active, int64_t* __restrict__ tdone,
                                       cudaGraphConditionalHandle cond, int use_cond) {
  __shared__ int any;
  const int maxiter = *maxiter_p;
  if (threadIdx.x == 0) any = 0;
  __syncthreads();
  for (int b = threadIdx.x; b < nbatch; b += blockDim.x) {
    if (!active[b]) continue;
    const double e = sumsq[b] * dv;
    err[b] = e;
    // while iterate2(step) > eps and niter < maxiter: niter += 1
    if (e > eps[b] && niter[b] < maxiter) {
      niter[b] += 1;
      atomicOr(&any, 1);
    } else {
      active[b] = 0;
      if (tdone) tdone[b] = global_ns();
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    *any_active = any;
    if (use_cond) cudaGraphSetConditional(cond, any ? 1u : 0u);
  }
}

__global__ void stamp_kernel(int64_t* t) { *t = global_ns(); }

// Per-solve state at the start of a solve; eps is read from the engine's
// mapped pinned mailbox, so no copy engine is involved.
__global__ void solve_setup_kernel(int nb, const double* __restrict__ h_eps, int maxiter, double* __restrict__ eps,
                                   int* __restrict__ niter, unsigned char* __restrict__ active, int* maxiter_out) {
  for (int b = threadIdx.x; b < nb; b += blockDim.x) {
    eps[b] = h_eps[b];
    niter[b] = 1;
    active[b] = 1;
  }
  if (threadIdx.x == 0) *maxiter_out = maxiter;
}

// Per-solve results into the mapped pinned mailbox.
__global__ void solve_readback_kernel(int nb, const int* __restrict__ niter, const double* __restrict__ err,
                                      int* __restrict__ h_niter, double* __restrict__ h_err) {
  for (int b = threadIdx.x; b < nb; b += blockDim.x) {
    h_niter[b] = niter[b];
    h_err[b] = err[b];
  }
}

// rows of `len` doubles between two row pitches (elements); one warp a row
__global__ void pitch_copy_kernel(int64_t rows, int len, const double* __restrict__ src, int64_t src_pitch,
                                  double* __restrict__ dst, int64_t dst_pitch) {
  const int64_t r = blockIdx.x * (int64_t)(blockDim.x >> 5) + (threadIdx.x >> 5);
  if (r >= rows) return;
  const double* s = src + r * src_pitch;
  double* d = dst + r * dst_pitch;
  for (int c = threadIdx.x & 31; c < len; c += 32) d[c] = s[c];
}

template <typename T>
__global__ void copy_kernel(int64_t n, const T* __restrict__ x, T* __restrict__ y) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    y[i] = x[i];
}

__global__ void to_f32_neg_kernel(int64_t n, const double* __restrict__ x, float* __restrict__ y,
                                  const unsigned char* active, int64_t per) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    if (active && !active[i / per]) continue;
    y[i] = (float)(-x[i]);
  }
}

__global__ void add_f32_kernel(int64_t n, const float* __restrict__ e, double* __restrict__ phi,
                               const unsigned char* active, int64_t per) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    if (active && !active[i / per]) continue;
    phi[i] += (double)e[i];
  }
}

}  // namespace gpw

using namespace gpw;

struct gpw_poisson {
  std::vector<Level> lv;
  int relax_method = 2;
  double dv = 1.0;
  int64_t nbmax = 1;
  // coarse end of the V-cycle in one CTA per solve (gpw_coarse.cuh): first
  // level handled there per form ([0] float64, [1] float32; nlevels = off)
  int lc[2] = {0, 0};
  CoarseArgs cargs[2];
  size_t csmem[2] = {0, 0};
  // the two levels lc - 1 and lc in a cluster of CTAs per solve, the coarse
  // kernel's levels from lc + 1 in its CTA 0 (float32 form; lt = -1: none)
  int lt = -1;
  ClusterTop ctop;
  CoarseArgs ccl;          // the coarse kernel's levels from lc + 1
  size_t ctsmem = 0;
  bool use_cluster = true;
  bool use_rr = true;  // float32 form: level-0 residual restricted in the same launch
  bool use_rr_coarse = true;  // ... and the coarser levels' residuals
  Workspace d_err, d_eps, d_niter, d_active, d_any, d_r64, d_gs_old, d_maxiter, d_tdone, d_t0;
  SumScratch sums;
  int* h_any = nullptr;  // pinned
  // mapped pinned mailbox: eps in, niter / error out (nbmax each)
  // two slots, so an asynchronous solve can be enqueued while the previous
  // one's results are still to be collected
  void* h_io = nullptr;
  double* h_eps[2] = {nullptr, nullptr};
  double* h_err[2] = {nullptr, nullptr};
  int* h_niter[2] = {nullptr, nullptr};
  double* m_eps[2] = {nullptr, nullptr};  // the same, as device pointers
  double* m_err[2] = {nullptr, nullptr};
  int* m_niter[2] = {nullptr, nullptr};
  struct GraphKey {
    int64_t nb;
    int prec;
    bool operator<(const GraphKey& o) const { return nb != o.nb ? nb < o.nb : prec < o.prec; }
  };
  std::map<GraphKey, cudaGraphExec_t> graphs;
  std::map<GraphKey, int64_t> graph_kernels;  // kernel nodes per graph
  // the whole convergence loop as one graph: a conditional while node whose
  // body is one iteration (null where conditional nodes are unavailable)
  std::map<GraphKey, cudaGraphExec_t> loops;
  int64_t last_kernels = 0, last_graphs = 0;
  bool device_loop = true;  // use the device-side loop when it can be built
  ~gpw_poisson() {
    for (auto& kv : graphs) cudaGraphExecDestroy(kv.second);
    for (auto& kv : loops)
      if (kv.second) cudaGraphExecDestroy(kv.second);
    if (h_any) cudaFreeHost(h_any);
    if (h_io) cudaFreeHost(h_io);
  }
};

namespace {

struct Rec {
  gpw_poisson* ps;
  int nb;
  cudaStream_t st;
  const unsigned char* active;
  bool tune = false;  // tuning pass: time the stencil launches' variants, launch nothing else
  // profiling pass (eager launches): an event after every launch, labelled
  std::vector<std::pair<std::string, cudaEvent_t>>* prof = nullptr;
  cudaError_t err = cudaSuccess;
  void ok(cudaError_t e) {
    if (err == cudaSuccess && e != cudaSuccess) err = e;
  }
  void tick(const std::string& label) {
    if (!prof || tune) return;
    cudaEvent_t ev;
    if (cudaEventCreate(&ev) != cudaSuccess) return;
    cudaEventRecord(ev, st);
    prof->emplace_back(label, ev);
  }
  // one star / general stencil launch (or, in the tuning pass, its tuning)
  void stencil(const OpDesc& d, int dt, int mode, const void* in, void* out, const void* rho, const GridView& v,
               double w, const GridSum& gs) {
    if (tune)
      ok(tune_stencil(d, dt, mode, in, v, out, v, rho, v, nullptr, nb, w, gs, st));
    else
      ok(launch_stencil(d, dt, mode, in, v, out, v, rho, v, nb, make_boundary(d.periodic, dt, nullptr), w, active,
                        gs, st));
  }
  // one fused defect-correction stencil launch (or its tuning)
  void stencil_dc(const OpDesc& d, int mode, const void* in, const GridView& v, void* out, void* out2,
                  const void* rho, double w, double w2, const GridSum& gs) {
    if (tune)
      ok(tune_stencil(d, mode == MODE_RESID_DC ? GPW_F64 : GPW_F32, mode, in, v, out, v, rho, v, out2, nb,
                      mode == MODE_RESID_DC ? w2 : w, gs, st));
    else
      ok(launch_stencil_dc(d, mode, in, v, out, out2, rho, nb, w, w2, active, gs, st));
  }
};

// The float32 residual of level l >= 1 restricted in the same launch
// (MODE_RESID_RESTRICT) into rho_{l+1} and its first weighted-Jacobi sweep:
// K = 2 zero-boundary restriction, Jacobi relaxation, and a level l+1 that
// the cluster kernel or the recursive V-cycle takes from there (the one-CTA
// coarse kernel starts from rho alone).
bool level_rr_ok(const gpw_poisson* ps, int l, const void* in, int nb) {
  const int nl = (int)ps->lv.size();
  if (!ps->use_rr_coarse || ps->relax_method != 2 || l < 1 || l + 1 >= nl || l + 1 == ps->lc[1]) return false;
  const Level& L = ps->lv[l];
  const Level& C = ps->lv[l + 1];
  const std::vector<double>& first = (l + 2 == nl) ? C.wpost[1] : C.wpre[1];
  if (first.empty() || C.op->coefs.empty() || L.restr->k != 2) return false;
  for (int c = 0; c < 3; ++c)
    if (L.restr->pad[c][0] != 0) return false;
  return resid_restrict_ok(*L.op, in, L.rho32.ptr, L.v, C.rho32.ptr, C.phi32[0].ptr, C.v, nb);
}

// Relax `n` sweeps on level l (dtype f64 or f32); returns the index of the
// phi buffer holding the result.
int rec_relax(Rec& r, int l, int cur, const double* ws, int nsweeps, bool f32) {
  Level& L = r.ps->lv[l];
  const int dt = f32 ? GPW_F32 : GPW_F64;
  Workspace* phi = f32 ? L.phi32 : L.phi;
  const void* rho = f32 ? L.rho32.ptr : L.rho.ptr;
  if (r.ps->relax_method == 1) {
    if (r.tune) return cur;
    Boundary bc = make_boundary(L.op->periodic, dt, nullptr);
    for (int b = 0; b < r.nb; ++b) {
      const size_t es = elt_size(dt) * (size_t)L.v.sb;
      r.ok(launch_relax_gs_ws(*L.op, dt, (char*)phi[cur].ptr + b * es, L.v, (const char*)rho + b * es, L.v,
                              nsweeps, bc, r.ps->d_gs_old.ptr, r.active ? r.active + b : nullptr, r.st));
    }
    return cur;
  }
  for (int s = 0; s < nsweeps; ++s) {
    r.stencil(*L.op, dt, MODE_JACOBI, phi[cur].ptr, phi[1 - cur].ptr, rho, L.v, ws[s], GridSum{});
    r.tick("L" + std::to_string(l) + (f32 ? " f32" : " f64") + " jacobi");
    cur = 1 - cur;
  }
  return cur;
}

// Levels l+1 .. L of form p, from the level-l residual `res`: restriction
// into rho_{l+1}, then the coarse one-CTA kernel when l+1 is its first level,
// else the recursive V-cycle from phi_{l+1} = 0, whose first weighted-Jacobi
// sweep ((w / c0) rho_{l+1}, exactly) the restriction writes alongside.
// Returns the buffer holding phi_{l+1}.
// restricted: rho_{l+1} and its first sweep were written by the fused
// residual-restriction launch (float32, not into the one-CTA kernel).
int rec_vcycle(Rec& r, int l, int cur, bool f32, bool first_done = false);
int rec_lower(Rec& r, int l, const void* res, bool f32, bool restricted = false) {
  gpw_poisson* ps = r.ps;
  const int nl = (int)ps->lv.size();
  const int p = f32 ? 1 : 0;
  const int dt = f32 ? GPW_F32 : GPW_F64;
  Level& L = ps->lv[l];
  Level& C = ps->lv[l + 1];
  Workspace* cphi = f32 ? C.phi32 : C.phi;
  Workspace& crho = f32 ? C.rho32 : C.rho;
  Boundary bc = make_boundary(L.op->periodic, dt, nullptr);
  if (l + 1 == ps->lc[p]) {
    // levels l+1 .. L in one CTA per solve: rho_{l+1} in, phi_{l+1} out
    if (!r.tune) {
      r.ok(launch_transfer(*L.restr, dt, res, L.v, crho.ptr, C.v, r.nb, bc, 0, nullptr, nullptr, r.active, r.st));
      r.tick("L" + std::to_string(l) + " restrict");
      CoarseArgs ca = ps->cargs[p];
      ca.rho = crho.ptr;
      ca.vrho = C.v;
      ca.phi = cphi[0].ptr;
      ca.vphi = C.v;
      ca.active = r.active;
      r.ok(launch_coarse(dt, ca, ps->csmem[p], r.nb, r.st));
      r.tick("L" + std::to_string(l + 1) + "+ coarse kernel");
    }
    return 0;
  }
  const bool coarsest = (l + 2 == nl);
  const std::vector<double>& first = coarsest ? C.wpost[p] : C.wpre[p];
  const bool fuse = restricted || (ps->relax_method == 2 && !first.empty() && restrict_sweep_ok(*L.restr, dt) &&
                                   !C.op->coefs.empty());
  if (!r.tune && !restricted) {
    if (fuse) {
      const RestrictSweep sw{cphi[0].ptr, first[0], C.op->coefs[0]};
      r.ok(launch_transfer(*L.restr, dt, res, L.v, crho.ptr, C.v, r.nb, bc, 0, nullptr, nullptr, r.active, r.st,
                           &sw));
      r.tick("L" + std::to_string(l) + " restrict+sweep");
    } else {
      r.ok(launch_transfer(*L.restr, dt, res, L.v, crho.ptr, C.v, r.nb, bc, 0, nullptr, nullptr, r.active, r.st));
      r.ok(launch_zero(dt, C.v, cphi[0].ptr, r.nb, r.active, r.st));
      r.tick("L" + std::to_string(l) + " restrict+zero");
    }
  }
  if (f32 && l + 1 == ps->lt) {
    // level l+1 and below in one cluster launch: rho_{l+1} (and its first
    // sweep) in, phi_{l+1} out in buffer 0
    if (!r.tune) {
      ClusterArgs ca;
      ca.ca = ps->ccl;
      Level& N = ps->lv[ps->lc[1] + 1];
      ca.ca.rho = N.rho32.ptr;
      ca.ca.vrho = N.v;
      ca.ca.phi = N.phi32[0].ptr;
      ca.ca.vphi = N.v;
      ca.ca.active = r.active;
      ca.t = ps->ctop;
      ca.t.rho = crho.ptr;
      ca.t.phi = cphi[0].ptr;
      ca.t.v = C.v;
      ca.t.first_done = fuse ? 1 : 0;
      r.ok(launch_cluster_vcycle(ca, ps->ctsmem, r.nb, r.st));
      r.tick("L" + std::to_string(l + 1) + "+ cluster kernel");
    }
    return 0;
  }
  // the fused first sweep wrote buffer 0 as the result of sweep 1: the
  // V-cycle continues from there (ping-pong parity counts that sweep)
  if (fuse) return rec_vcycle(r, l + 1, 0, f32, true);
  return rec_vcycle(r, l + 1, 0, f32);
}

// Records iterate2(level l) starting from phi buffer `cur`; returns the buffer
// holding phi_l afterwards.  first_done: the first sweep of this level (its
// first pre-sweep, or on the coarsest level its first post-sweep) has already
// been written into buffer `cur`.
int rec_vcycle(Rec& r, int l, int cur, bool f32, bool first_done) {
  gpw_poisson* ps = r.ps;
  const int nl = (int)ps->lv.size();
  Level& L = ps->lv[l];
  const int dt = f32 ? GPW_F32 : GPW_F64;
  Workspace* phi = f32 ? L.phi32 : L.phi;
  Workspace& rho = f32 ? L.rho32 : L.rho;
  Workspace& res = f32 ? L.res32 : L.res;
  const int p = f32 ? 1 : 0;
  if (l < nl - 1) {
    Level& C = ps->lv[l + 1];
    Workspace* cphi = f32 ? C.phi32 : C.phi;
    const int skip = first_done ? 1 : 0;
    cur = rec_relax(r, l, cur, L.wpre[p].data() + skip, (int)L.wpre[p].size() - skip, f32);
    // the residual's norm is not needed below level 0's convergence test
    int ccur;
    if (f32 && level_rr_ok(ps, l, phi[cur].ptr, r.nb)) {
      // float32: the residual restricted straight into rho_{l+1} and its first sweep
      const std::vector<double>& first = (l + 2 == nl) ? C.wpost[1] : C.wpre[1];
      r.ok(launch_resid_restrict(*L.op, phi[cur].ptr, rho.ptr, L.v, C.rho32.ptr, C.phi32[0].ptr, C.v, r.nb,
                                 first[0], C.op->coefs[0], r.active, r.tune, r.st));
      r.tick("L" + std::to_string(l) + " f32 residual + restriction");
      ccur = rec_lower(r, l, nullptr, f32, true);
    } else {
      r.stencil(*L.op, dt, MODE_RESIDUAL, phi[cur].ptr, res.ptr, rho.ptr, L.v, 1.0, GridSum{});
      r.tick("L" + std::to_string(l) + (f32 ? " f32" : " f64") + " residual");
      ccur = rec_lower(r, l, res.ptr, f32);
    }
    Boundary cbc = make_boundary(C.op->periodic, dt, nullptr);
    if (!r.tune) {
      r.ok(launch_transfer(*L.interp, dt, cphi[ccur].ptr, C.v, phi[1 - cur].ptr, L.v, r.nb, cbc, 1, phi[cur].ptr,
                           &L.v, r.active, r.st));
      r.tick("L" + std::to_string(l) + " interpolate-subtract");
    }
    cur = 1 - cur;
    return rec_relax(r, l, cur, L.wpost[p].data(), (int)L.wpost[p].size(), f32);
  }
  const int skip = first_done ? 1 : 0;
  return rec_relax(r, l, cur, L.wpost[p].data() + skip, (int)L.wpost[p].size() - skip, f32);
}

}  // namespace

extern "C" {

int gpw_poisson_new(int nlevels, gpw_operator* const* operators, gpw_transformer* const* restrictors,
                    gpw_transformer* const* interpolators, const int* presmooths, const int* postsmooths,
                    const double* weights, int relax_method, double dv, int64_t nbatch_max, gpw_poisson** out);
int gpw_poisson_solve(gpw_poisson* ps, double* phi, const double* rho, int64_t nbatch, const double* eps, int maxiter,
                      int precision, int* niter, double* error, gpw_stream stream);
void gpw_poisson_free(gpw_poisson* ps);

}  // extern "C"

// The opaque handle types are defined in gpw_api.cu; the engine only needs
// their descriptors, exported through these accessors.
namespace gpw {
const OpDesc* operator_desc(const gpw_operator* op);
const TrDesc* transformer_desc(const gpw_transformer* tr);
}  // namespace gpw

// Choose the first level of the coarse one-CTA kernel for form p (0 float64,
// 1 float32) and fill its arguments: the deepest suffix of levels (never
// level 0) that are real 7-point star Laplacians relaxed by Jacobi and whose
// buffers (two phi + rho per level) fit the shared-memory budget.
// The float32 levels lc - 1 and lc (the level above the coarse kernel's
// first level, and that level) in a cluster of CG_NCL CTAs per solve
// (gpw_coarse.cuh), the coarse kernel's levels from lc + 1 in its CTA 0:
// zero boundaries (padded form), 7-point Jacobi, every CTA owning planes of
// both levels, and everything within one CTA's shared memory at two CTAs per
// SM (so that all of a batch's clusters are resident together).
static void setup_cluster_top(gpw_poisson* ps, bool padded, size_t es) {
  ps->lt = -1;
  const int lc = ps->lc[1], nl = (int)ps->lv.size();
  if (!ps->use_cluster || !padded || lc < 2 || lc + 1 >= nl || ps->relax_method != 2 || es != 4) return;
  const CoarseArgs& ca = ps->cargs[1];
  if (ca.nl < 2) return;
  const int lt = lc - 1;
  const Level& L = ps->lv[lt];
  const OpDesc& d = *L.op;
  if (!d.real || !d.star_jacobi || d.R != 1) return;
  if ((int)(L.wpre[1].size() + L.wpost[1].size()) > CG_MAXW || L.wpre[1].empty()) return;
  const int n0 = L.v.n[0], m0 = ca.lv[0].n[0];
  int maxp = 0, maxq = 0;
  for (int r = 0; r < CG_NCL; ++r) {
    const int z0 = r * n0 / CG_NCL, z1 = (r + 1) * n0 / CG_NCL;
    const int y0 = std::min(m0, z0 / 2), y1 = (r + 1 == CG_NCL) ? m0 : std::min(m0, z1 / 2);
    if (z1 - z0 < 1 || y1 - y0 < 1) return;
    maxp = std::max(maxp, z1 - z0);
    maxq = std::max(maxq, y1 - y0);
  }
  const CoarseLevel& U = ca.lv[0];
  const CoarseLevel& N = ca.lv[1];
  const size_t slab = (size_t)(maxp + 2) * (L.v.n[1] + 2) * (L.v.n[2] + 2);
  const size_t slab2 = (size_t)(maxq + 2) * (U.n[1] + 2) * (U.n[2] + 2);
  const size_t next = (size_t)(N.n[0] + 2) * (N.n[1] + 2) * (N.n[2] + 2);
  // the coarse kernel's levels without its first: bases shifted down
  CoarseArgs cs = ca;
  cs.nl = ca.nl - 1;
  for (int k = 0; k < cs.nl; ++k) {
    cs.lv[k] = ca.lv[k + 1];
    cs.lv[k].base -= ca.lv[1].base;
  }
  const size_t cbytes = ps->csmem[1] - (size_t)ca.lv[1].base * es;
  const size_t bytes = (3 * slab + 3 * slab2 + next) * es + cbytes;
  if (bytes > 110 * 1024) return;
  ClusterTop& t = ps->ctop;
  t = ClusterTop{};
  CoarseLevel& c = t.L;
  for (int a = 0; a < 3; ++a) {
    c.n[a] = L.v.n[a];
    c.periodic[a] = 0;
    c.rpad0[a] = L.restr->pad[a][0];
    c.ipad0[a] = L.interp->pad[a][0];
    c.iskip0[a] = L.interp->skip[a][0];
  }
  c.pts = (int)slab;
  c.cc = d.sc.cc;
  c.cm[0] = d.sc.cx[0];
  c.cp[0] = d.sc.cx[2];
  c.cm[1] = d.sc.cy[0];
  c.cp[1] = d.sc.cy[2];
  c.cm[2] = d.sc.cz[0];
  c.cp[2] = d.sc.cz[2];
  c.npre = (int)L.wpre[1].size();
  c.npost = (int)L.wpost[1].size();
  for (int i = 0; i < c.npre; ++i) c.w[i] = L.wpre[1][i];
  for (int i = 0; i < c.npost; ++i) c.w[c.npre + i] = L.wpost[1][i];
  t.L2 = U;
  t.slab_pts = (int)slab;
  t.slab2_pts = (int)slab2;
  t.next_pts = (int)next;
  ps->ccl = cs;
  ps->ctsmem = bytes;
  ps->lt = lt;
}

static void setup_coarse(gpw_poisson* ps, int p) {
  const int nl = (int)ps->lv.size();
  const size_t es = p ? 4 : 8;
  const size_t budget = 160 * 1024;
  ps->lc[p] = nl;
  ps->csmem[p] = 0;
  if (ps->relax_method != 2) return;
  // padded layout (zero halo) when no level of the hierarchy is periodic
  // and the transfers have the zero-boundary K=2 tables
  bool padded = true;
  for (int l = 0; l < nl; ++l) {
    const Level& L = ps->lv[l];
    for (int a = 0; a < 3; ++a) {
      if (L.op->periodic[a]) padded = false;
      if (l + 1 < nl && (L.restr->k != 2 || L.restr->pad[a][0] != 0 || L.interp->k != 2 ||
                         L.interp->pad[a][0] != 1 || L.interp->skip[a][0] != 1))
        padded = false;
    }
  }
  auto buf_pts = [&](const Level& L) -> size_t {
    return padded ? (size_t)(L.v.n[0] + 2) * (L.v.n[1] + 2) * (L.v.n[2] + 2) : (size_t)view_points(L.v);
  };
  size_t bytes = 0;
  int lc = nl;
  for (int l = nl - 1; l >= 1 && nl - l <= CG_MAXL; --l) {
    const Level& L = ps->lv[l];
    const OpDesc& d = *L.op;
    if (!d.real || !d.star_jacobi || d.R != 1) break;
    if ((int)(L.wpre[p].size() + L.wpost[p].size()) > CG_MAXW) break;
    const size_t b = 3 * buf_pts(L) * es;
    if (bytes + b > budget) break;
    bytes += b;
    lc = l;
  }
  if (lc >= nl) return;
  CoarseArgs& ca = ps->cargs[p];
  ca = CoarseArgs{};
  ca.nl = nl - lc;
  ca.padded = padded ? 1 : 0;
  int base = 0;
  for (int k = 0; k < ca.nl; ++k) {
    const Level& L = ps->lv[lc + k];
    const OpDesc& d = *L.op;
    CoarseLevel& c = ca.lv[k];
    for (int a = 0; a < 3; ++a) {
      c.n[a] = L.v.n[a];
      c.periodic[a] = d.periodic[a];
    }
    c.pts = (int)buf_pts(L);
    c.base = base;
    base += 3 * c.pts;
    c.cc = d.sc.cc;
    c.cm[0] = d.sc.cx[0];
    c.cp[0] = d.sc.cx[2];
    c.cm[1] = d.sc.cy[0];
    c.cp[1] = d.sc.cy[2];
    c.cm[2] = d.sc.cz[0];
    c.cp[2] = d.sc.cz[2];
    c.npre = (int)L.wpre[p].size();
    c.npost = (int)L.wpost[p].size();
    for (int i = 0; i < c.npre; ++i) c.w[i] = L.wpre[p][i];
    for (int i = 0; i < c.npost; ++i) c.w[c.npre + i] = L.wpost[p][i];
    if (lc + k + 1 < nl) {
      for (int a = 0; a < 3; ++a) {
        c.rpad0[a] = L.restr->pad[a][0];
        c.ipad0[a] = L.interp->pad[a][0];
        c.iskip0[a] = L.interp->skip[a][0];
      }
    }
  }
  ps->lc[p] = lc;
  ps->csmem[p] = bytes;
  if (p == 1) setup_cluster_top(ps, padded, es);
}

int gpw_poisson_new(int nlevels, gpw_operator* const* operators, gpw_transformer* const* restrictors,
                    gpw_transformer* const* interpolators, const int* presmooths, const int* postsmooths,
                    const double* weights, int relax_method, double dv, int64_t nbatch_max, gpw_poisson** out) {
  if (nlevels < 1 || nlevels > 16 || !operators || !presmooths || !postsmooths || !weights || !out)
    return fail(GPW_EINVAL, "poisson: bad arguments");
  if (nlevels > 1 && (!restrictors || !interpolators)) return fail(GPW_EINVAL, "poisson: missing transformers");
  if (relax_method != 1 && relax_method != 2) return fail(GPW_EINVAL, "poisson: relax_method must be 1 or 2");
  if (nbatch_max < 1 || nbatch_max > 4096) return fail(GPW_EINVAL, "poisson: nbatch_max out of range");
  std::unique_ptr<gpw_poisson> ps(new gpw_poisson());
  ps->relax_method = relax_method;
  ps->dv = dv;
  ps->nbmax = nbatch_max;
  ps->lv.resize(nlevels);
  for (int l = 0; l < nlevels; ++l) {
    Level& L = ps->lv[l];
    if (!operators[l]) return fail(GPW_EINVAL, "poisson: null operator");
    L.op = operator_desc(operators[l]);
    L.v = pitched_view(L.op->n);
    L.pre = presmooths[l];
    L.post = postsmooths[l];
    L.w = weights[l];
    if (L.pre < 0 || L.post < 0 || L.pre > CG_MAXW || L.post > CG_MAXW || L.pre + L.post > CG_MAXW)
      return fail(GPW_EINVAL, "poisson: smoothing counts out of range");
    for (int p = 0; p < 2; ++p) {
      L.wpre[p].assign(l + 1 < nlevels ? L.pre : 0, L.w);
      L.wpost[p].assign(L.post, L.w);
    }
    if (l < nlevels - 1) {
      if (!restrictors[l] || !interpolators[l]) return fail(GPW_EINVAL, "poisson: null transformer");
      L.restr = transformer_desc(restrictors[l]);
      L.interp = transformer_desc(interpolators[l]);
      if (L.restr->interpolate || !L.interp->interpolate) return fail(GPW_EINVAL, "poisson: transformer kinds");
    }
    const size_t pts = (size_t)L.v.sb * nbatch_max;
    int rc;
    if ((rc = L.phi[0].ensure(pts * 8)) || (rc = L.phi[1].ensure(pts * 8)) || (rc = L.rho.ensure(pts * 8)) ||
        (rc = L.res.ensure(pts * 8)))
      return rc;
    // row padding is never read as data; keep it finite
    for (Workspace* w : {&L.phi[0], &L.phi[1], &L.rho, &L.res}) cudaMemset(w->ptr, 0, w->bytes);
  }
  // level shapes must chain through the transformers
  for (int l = 0; l + 1 < nlevels; ++l) {
    const Level &A = ps->lv[l], &B = ps->lv[l + 1];
    for (int c = 0; c < 3; ++c)
      if (A.restr->nin[c] != A.v.n[c] || A.restr->nout[c] != B.v.n[c] || A.interp->nin[c] != B.v.n[c] ||
          A.interp->nout[c] != A.v.n[c])
        return fail(GPW_EINVAL, "poisson: level shapes do not chain");
  }
  setup_coarse(ps.get(), 0);
  setup_coarse(ps.get(), 1);
  int rc;
  if ((rc = ps->d_err.ensure(nbatch_max * 8)) || (rc = ps->d_eps.ensure(nbatch_max * 8)) ||
      (rc = ps->d_niter.ensure(nbatch_max * 4)) || (rc = ps->d_active.ensure(nbatch_max)) ||
      (rc = ps->d_tdone.ensure(nbatch_max * 8)) || (rc = ps->d_t0.ensure(8)) ||
      (rc = ps->d_any.ensure(16)) || (rc = ps->d_maxiter.ensure(16)) || (rc = ps->d_r64.ensure((size_t)ps->lv[0].v.sb * nbatch_max * 8)))
    return rc;
  if (relax_method == 1) {
    size_t mx = 0;
    for (auto& L : ps->lv) mx = std::max(mx, (size_t)view_points(L.v));
    if ((rc = ps->d_gs_old.ensure(mx * 8))) return rc;
  }
  const int nblk = stencil_blocks_per_member(*ps->lv[0].op, MODE_RESIDUAL, ps->lv[0].v, 1);
  // residual partial slots: enough for any level / batch size (blocks per member shrink with batch)
  int64_t maxblk = 0;
  for (auto& L : ps->lv) maxblk = std::max<int64_t>(maxblk, stencil_blocks_per_member(*L.op, MODE_RESIDUAL, L.v, 1));
  (void)nblk;
  if ((rc = ps->sums.ensure(nbatch_max, maxblk))) return rc;
  if (!device_status_word()) return fail(GPW_ENOMEM, "status word allocation");
  cudaError_t e = cudaMallocHost(&ps->h_any, sizeof(int));
  if (e != cudaSuccess) return cuda_fail(e, "pinned alloc");
  const size_t slot_bytes = ((size_t)nbatch_max * 20 + 15) / 16 * 16;
  e = cudaHostAlloc(&ps->h_io, 2 * slot_bytes + 64, cudaHostAllocMapped | cudaHostAllocPortable);
  if (e != cudaSuccess) return cuda_fail(e, "pinned mailbox");
  void* dio = nullptr;
  e = cudaHostGetDevicePointer(&dio, ps->h_io, 0);
  if (e != cudaSuccess) return cuda_fail(e, "pinned mailbox mapping");
  for (int k = 0; k < 2; ++k) {
    ps->h_eps[k] = (double*)((char*)ps->h_io + k * slot_bytes);
    ps->h_err[k] = ps->h_eps[k] + nbatch_max;
    ps->h_niter[k] = (int*)(ps->h_err[k] + nbatch_max);
    ps->m_eps[k] = (double*)((char*)dio + k * slot_bytes);
    ps->m_err[k] = ps->m_eps[k] + nbatch_max;
    ps->m_niter[k] = (int*)(ps->m_err[k] + nbatch_max);
  }
  *out = ps.release();
  return GPW_OK;
}

void gpw_poisson_free(gpw_poisson* ps) { delete ps; }

static int ensure_f32(gpw_poisson* ps);
static bool fused_dc(const gpw_poisson* ps);
static bool scaled_first(const gpw_poisson* ps);

extern "C" int gpw_poisson_time_level0(gpw_poisson* ps, int64_t nbatch, int which, int reps, double* ms_per_launch,
                                       double* bytes_per_launch, gpw_stream stream) {
  if (!ps || !ms_per_launch || !bytes_per_launch) return fail(GPW_EINVAL, "null argument");
  if (nbatch < 1 || nbatch > ps->nbmax || reps < 1 || which < 0 || which > 7)
    return fail(GPW_EINVAL, "time_level0: bad arguments");
  if (which >= 2) {
    int rc = ensure_f32(ps);
    if (rc) return rc;
  }
  if ((which == 3 || which == 4) && !fused_dc(ps)) return fail(GPW_ENOTSUP, "time_level0: no fused path here");
  if (which == 7 && !scaled_first(ps)) return fail(GPW_ENOTSUP, "time_level0: no scaled first sweep here");
  const bool scaled = scaled_first(ps);
  cudaStream_t st = (cudaStream_t)stream;
  Level& L0 = ps->lv[0];
  const int nb = (int)nbatch;
  const double pts = (double)view_points(L0.v) * nb;
  if (which == 6 && (ps->lv.size() < 2 || ps->lv[1].wpre[1].empty() ||
                     !resid_restrict_ok(*L0.op, L0.phi32[0].ptr, L0.rho32.ptr, L0.v, ps->lv[1].rho32.ptr,
                                        ps->lv[1].phi32[0].ptr, ps->lv[1].v, nb)))
    return fail(GPW_ENOTSUP, "time_level0: no fused residual-restriction here");
  const unsigned char* act = nullptr;
  auto launch = [&]() -> cudaError_t {
    switch (which) {
      case 0:
        return launch_stencil(*L0.op, GPW_F64, MODE_JACOBI, L0.phi[0].ptr, L0.v, L0.phi[1].ptr, L0.v, L0.rho.ptr,
                              L0.v, nb, make_boundary(L0.op->periodic, GPW_F64, nullptr), L0.w, act, GridSum{}, st);
      case 1:
        return launch_stencil(*L0.op, GPW_F64, MODE_RESIDUAL, L0.phi[0].ptr, L0.v, nullptr, L0.v, L0.rho.ptr, L0.v,
                              nb, make_boundary(L0.op->periodic, GPW_F64, nullptr), 1.0, act, ps->sums.gs(), st);
      case 2:
        return launch_stencil(*L0.op, GPW_F32, MODE_JACOBI, L0.phi32[0].ptr, L0.v, L0.phi32[1].ptr, L0.v,
                              L0.rho32.ptr, L0.v, nb, make_boundary(L0.op->periodic, GPW_F32, nullptr), L0.w, act,
                              GridSum{}, st);
      case 3:
        return launch_stencil_dc(*L0.op, MODE_JACOBI_ADD64, L0.phi32[0].ptr, L0.v, nullptr, L0.phi[1].ptr,
                                 L0.rho32.ptr, nb, L0.w, 0.0, act, GridSum{}, st);
      case 4:  // as the iteration launches it (no stored iterate when the next sweep forms it)
        return launch_stencil_dc(*L0.op, MODE_RESID_DC, L0.phi[0].ptr, L0.v, L0.rho32.ptr,
                                 scaled ? nullptr : L0.phi32[1].ptr, L0.rho.ptr, nb, 1.0, L0.w, act, ps->sums.gs(), st);
      case 7:
        return launch_stencil_dc(*L0.op, MODE_JACOBI_SCALED_IN, L0.rho32.ptr, L0.v, L0.phi32[1].ptr, nullptr,
                                 nullptr, nb, L0.wpre[1][1], L0.wpre[1][0], act, GridSum{}, st);
      case 6: {
        Level& C = ps->lv[1];
        return launch_resid_restrict(*L0.op, L0.phi32[0].ptr, L0.rho32.ptr, L0.v, C.rho32.ptr, C.phi32[0].ptr, C.v,
                                     nb, C.wpre[1][0], C.op->coefs[0], act, false, st);
      }
      default:
        return launch_stencil(*L0.op, GPW_F32, MODE_RESIDUAL, L0.phi32[0].ptr, L0.v, L0.res32.ptr, L0.v,
                              L0.rho32.ptr, L0.v, nb, make_boundary(L0.op->periodic, GPW_F32, nullptr), 1.0, act,
                              GridSum{}, st);
    }
  };
  // which 6: reads phi and rho (8 B per fine point), writes the next level's
  // rho and first sweep (8 B per coarse point); 4 without the stored iterate:
  // 20 B; 7: reads rhs, writes phi (8 B)
  static const double bytes_pp[8] = {24.0, 16.0, 12.0, 24.0, 24.0, 12.0, 8.0, 8.0};
  cudaError_t e = launch();  // warm-up (and lazy kernel setup)
  if (e != cudaSuccess) return cuda_fail(e, "time_level0 launch");
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, st);
  for (int i = 0; i < reps && e == cudaSuccess; ++i) e = launch();
  cudaEventRecord(e1, st);
  cudaError_t se = cudaEventSynchronize(e1);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (e != cudaSuccess) return cuda_fail(e, "time_level0 launch");
  if (se != cudaSuccess) return cuda_fail(se, "time_level0 sync");
  *ms_per_launch = ms / reps;
  *bytes_per_launch = (which == 4 && scaled ? 20.0 : bytes_pp[which]) * pts +
                      (which == 6 ? 8.0 * (double)view_points(ps->lv[1].v) * nb : 0.0);
  return GPW_OK;
}

extern "C" int gpw_poisson_last_stats(const gpw_poisson* ps, int64_t* kernel_launches, int64_t* graph_launches) {
  if (!ps) return fail(GPW_EINVAL, "null argument");
  if (kernel_launches) *kernel_launches = ps->last_kernels;
  if (graph_launches) *graph_launches = ps->last_graphs;
  return GPW_OK;
}

static int ensure_f32(gpw_poisson* ps) {
  for (auto& L : ps->lv) {
    const size_t pts = (size_t)L.v.sb * ps->nbmax;
    int rc;
    if ((rc = L.phi32[0].ensure(pts * 4)) || (rc = L.phi32[1].ensure(pts * 4)) || (rc = L.rho32.ensure(pts * 4)) ||
        (rc = L.res32.ensure(pts * 4)))
      return rc;
    for (Workspace* w : {&L.phi32[0], &L.phi32[1], &L.rho32, &L.res32}) cudaMemset(w->ptr, 0, w->bytes);
  }
  return GPW_OK;
}

// Record one outer iteration (one V-cycle, or one defect-correction step)
// plus the convergence update for batch size nb.
// The fused float32 defect-correction iteration applies to zero-boundary star
// Laplacians with at least one pre- and one post-sweep on level 0.
static bool fused_dc(const gpw_poisson* ps) {
  const Level& L0 = ps->lv[0];
  return ps->relax_method == 2 && ps->lv.size() >= 2 && !L0.wpre[1].empty() && !L0.wpost[1].empty() &&
         dc_fusable(*L0.op);
}

// The float32 form's second level-0 pre-sweep reads the defect alone and
// forms the first sweep's iterate itself (MODE_JACOBI_SCALED_IN), so the
// float64 defect stores no iterate: with the fusions on and at least two
// level-0 pre-sweeps.
static bool scaled_first(const gpw_poisson* ps) { return fused_dc(ps) && ps->use_rr && ps->lv[0].wpre[1].size() >= 2; }

// tune = true: the autotuner's pass over the same stencil launches (before
// capture, on the engine's buffers); nothing else is launched.
static cudaError_t record_iteration(gpw_poisson* ps, int nb, int prec, cudaStream_t st, bool tune = false,
                                    const cudaGraphConditionalHandle* cond = nullptr,
                                    std::vector<std::pair<std::string, cudaEvent_t>>* prof = nullptr) {
  Rec r{ps, nb, st, (const unsigned char*)ps->d_active.ptr};
  r.tune = tune;
  r.prof = prof;
  Level& L0 = ps->lv[0];
  const int64_t per = L0.v.sb;
  const int64_t n = per * nb;
  const int thr = 256;
  const int blocks = (int)std::min<int64_t>((n + thr - 1) / thr, 4LL * num_sms());
  auto converge = [&]() {
    if (tune) return;
    converge_update_kernel<<<1, 256, 0, st>>>(nb, ps->sums.gs().result, ps->dv, (const double*)ps->d_eps.ptr,
                                              (const int*)ps->d_maxiter.ptr, (double*)ps->d_err.ptr,
                                              (int*)ps->d_niter.ptr, (unsigned char*)ps->d_active.ptr,
                                              (int*)ps->d_any.ptr, (int64_t*)ps->d_tdone.ptr,
                                              cond ? *cond : cudaGraphConditionalHandle{}, cond ? 1 : 0);
    r.ok(cudaGetLastError());
    r.tick("convergence update");
  };
  if (prec == 0) {
    const int cur = rec_vcycle(r, 0, 0, false);
    if (cur != 0 && !tune) {  // odd ping-pong parity: the iterate goes back to buffer 0
      copy_kernel<double><<<blocks, thr, 0, st>>>(n, (const double*)L0.phi[1].ptr, (double*)L0.phi[0].ptr);
      r.ok(cudaGetLastError());
    }
  } else if (fused_dc(ps)) {
    // Fused defect correction.  On entry L0.rho32 holds rhs = -(A phi - rho)
    // and L0.phi32[0] the first level-0 sweep from zero (both written by the
    // previous MODE_RESID_DC launch).  Finish the float32 V-cycle; its last
    // level-0 post-sweep adds e into float64 phi; then the fused residual
    // writes the next rhs / first sweep and the norm.
    Level& C = ps->lv[1];
    const std::vector<double>& wpre = L0.wpre[1];
    const std::vector<double>& wpost = L0.wpost[1];
    int cur;
    if (scaled_first(ps)) {
      // the second pre-sweep reads rhs alone and forms the first sweep's
      // iterate (w2 / c0) rhs itself, so RESID_DC stores no iterate
      r.stencil_dc(*L0.op, MODE_JACOBI_SCALED_IN, L0.rho32.ptr, L0.v, L0.phi32[1].ptr, nullptr, nullptr, wpre[1],
                   wpre[0], GridSum{});
      r.tick("L0 f32 jacobi from rhs");
      cur = rec_relax(r, 0, 1, wpre.data() + 2, (int)wpre.size() - 2, true);
    } else {
      cur = rec_relax(r, 0, 0, wpre.data() + 1, (int)wpre.size() - 1, true);
    }
    int ccur;
    const int nl = (int)ps->lv.size();
    const bool rr = ps->use_rr && nl > 2 && ps->lc[1] > 1 && ps->lt != 1 && L0.restr->k == 2 &&
                    L0.restr->pad[0][0] == 0 && L0.restr->pad[1][0] == 0 && L0.restr->pad[2][0] == 0 &&
                    !C.wpre[1].empty() && !C.op->coefs.empty() &&
                    resid_restrict_ok(*L0.op, L0.phi32[cur].ptr, L0.rho32.ptr, L0.v, C.rho32.ptr, C.phi32[0].ptr,
                                      C.v, nb);
    if (rr) {
      // the residual restricted straight into level 1's rho and first sweep
      r.ok(launch_resid_restrict(*L0.op, L0.phi32[cur].ptr, L0.rho32.ptr, L0.v, C.rho32.ptr, C.phi32[0].ptr, C.v,
                                 nb, C.wpre[1][0], C.op->coefs[0], r.active, tune, st));
      r.tick("L0 f32 residual + restriction");
      ccur = rec_vcycle(r, 1, 0, true, true);
    } else {
      r.stencil(*L0.op, GPW_F32, MODE_RESIDUAL, L0.phi32[cur].ptr, L0.res32.ptr, L0.rho32.ptr, L0.v, 1.0,
                GridSum{});
      r.tick("L0 f32 residual");
      ccur = rec_lower(r, 0, L0.res32.ptr, true);
    }
    Boundary cbc = make_boundary(C.op->periodic, GPW_F32, nullptr);
    if (!tune) {
      r.ok(launch_transfer(*L0.interp, GPW_F32, C.phi32[ccur].ptr, C.v, L0.phi32[1 - cur].ptr, L0.v, nb, cbc, 1,
                           L0.phi32[cur].ptr, &L0.v, r.active, st));
      r.tick("L0 interpolate-subtract");
    }
    cur = 1 - cur;
    cur = rec_relax(r, 0, cur, wpost.data(), (int)wpost.size() - 1, true);
    r.stencil_dc(*L0.op, MODE_JACOBI_ADD64, L0.phi32[cur].ptr, L0.v, nullptr, L0.phi[0].ptr, L0.rho32.ptr,
                 wpost.back(), 0.0, GridSum{});
    r.tick("L0 f32 jacobi + phi64 update");
    r.stencil_dc(*L0.op, MODE_RESID_DC, L0.phi[0].ptr, L0.v, L0.rho32.ptr,
                 scaled_first(ps) ? nullptr : L0.phi32[0].ptr, L0.rho.ptr, 1.0, wpre[0], ps->sums.gs());
    r.tick(scaled_first(ps) ? "L0 f64 defect" : "L0 f64 defect + first sweep");
    converge();
    return r.err;
  } else {
    // defect correction: rhs32 = -(A phi - rho) (residual computed at the end
    // of the previous iteration into d_r64), e = FP32 V-cycle(rhs32), phi += e
    if (!tune) {
      to_f32_neg_kernel<<<blocks, thr, 0, st>>>(n, (const double*)ps->d_r64.ptr, (float*)L0.rho32.ptr, r.active,
                                                per);
      r.ok(cudaGetLastError());
      r.ok(launch_zero(GPW_F32, L0.v, L0.phi32[0].ptr, nb, r.active, st));
    }
    const int cur = rec_vcycle(r, 0, 0, true);
    if (!tune) {
      add_f32_kernel<<<blocks, thr, 0, st>>>(n, (const float*)L0.phi32[cur].ptr, (double*)L0.phi[0].ptr, r.active,
                                             per);
      r.ok(cudaGetLastError());
    }
  }
  // error = sum(r^2) dv on level 0 after post-smoothing (gpaw/poisson.py:357-361)
  // (the float64 residual itself is kept only as the next defect-correction right-hand side)
  r.stencil(*L0.op, GPW_F64, MODE_RESIDUAL, L0.phi[0].ptr, prec == 1 ? ps->d_r64.ptr : nullptr, L0.rho.ptr, L0.v,
            1.0, ps->sums.gs());
  r.tick("L0 f64 residual + norm");
  converge();
  return r.err;
}

static int64_t count_kernel_nodes(cudaGraph_t g) {
  size_t nnodes = 0;
  int64_t nkern = 0;
  if (cudaGraphGetNodes(g, nullptr, &nnodes) == cudaSuccess && nnodes) {
    std::vector<cudaGraphNode_t> nodes(nnodes);
    if (cudaGraphGetNodes(g, nodes.data(), &nnodes) == cudaSuccess)
      for (auto n : nodes) {
        cudaGraphNodeType t;
        if (cudaGraphNodeGetType(n, &t) == cudaSuccess && t == cudaGraphNodeTypeKernel) ++nkern;
      }
  }
  return nkern;
}

// The graph of one iteration for (batch size, form), captured on first use
// after the autotuning pass over its stencil launches.
static int iteration_graph(gpw_poisson* ps, int nb, int prec, cudaStream_t st, cudaGraphExec_t* out) {
  gpw_poisson::GraphKey key{nb, prec};
  auto it = ps->graphs.find(key);
  if (it != ps->graphs.end()) {
    *out = it->second;
    return GPW_OK;
  }
  // autotune the stencil launches of the iteration on the engine's own
  // buffers (before the inputs are copied in), then capture it
  cudaError_t e = record_iteration(ps, nb, prec, st, true);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_fail(e, "stencil autotuning");
  cudaGraph_t g;
  cudaStream_t cs;
  if ((e = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking)) != cudaSuccess) return cuda_fail(e, "stream");
  if ((e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal)) != cudaSuccess) {
    cudaStreamDestroy(cs);
    return cuda_fail(e, "begin capture");
  }
  cudaError_t re = record_iteration(ps, nb, prec, cs);
  e = cudaStreamEndCapture(cs, &g);
  cudaStreamDestroy(cs);
  if (re != cudaSuccess) return cuda_fail(re, "record V-cycle");
  if (e != cudaSuccess) return cuda_fail(e, "end capture");
  const int64_t nkern = count_kernel_nodes(g);
  cudaGraphExec_t ge;
  e = cudaGraphInstantiate(&ge, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) return cuda_fail(e, "graph instantiate");
  ps->graphs.emplace(key, ge);
  ps->graph_kernels[key] = nkern;
  *out = ge;
  return GPW_OK;
}

// Capture one iteration of engine `ps` into `body`, the child graph of a
// conditional while node whose condition the iteration's convergence kernel
// sets (loop while any solve of the batch is active).
static cudaError_t capture_loop_body(gpw_poisson* ps, int nb, int prec, cudaGraph_t body,
                                     cudaGraphConditionalHandle h) {
  cudaStream_t cs;
  cudaError_t e = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking);
  if (e != cudaSuccess) return e;
  e = cudaStreamBeginCaptureToGraph(cs, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) {
    cudaStreamDestroy(cs);
    return e;
  }
  cudaError_t re = record_iteration(ps, nb, prec, cs, false, &h);
  cudaGraph_t g = nullptr;
  e = cudaStreamEndCapture(cs, &g);
  cudaStreamDestroy(cs);
  return re != cudaSuccess ? re : e;
}

// Add a while node running engine ps's iterations to `parent` (after `dep`
// when given); returns the node.
static cudaError_t add_loop_node(gpw_poisson* ps, int nb, int prec, cudaGraph_t parent, const cudaGraphNode_t* dep,
                                 cudaGraphNode_t* node) {
  cudaGraphConditionalHandle h;
  cudaError_t e = cudaGraphConditionalHandleCreate(&h, parent, 1, cudaGraphCondAssignDefault);
  if (e != cudaSuccess) return e;
  cudaGraphNodeParams np{};
  np.type = cudaGraphNodeTypeConditional;
  np.conditional.handle = h;
  np.conditional.type = cudaGraphCondTypeWhile;
  np.conditional.size = 1;
  e = cudaGraphAddNode(node, parent, dep, dep ? 1 : 0, &np);
  if (e != cudaSuccess) return e;
  return capture_loop_body(ps, nb, prec, np.conditional.phGraph_out[0], h);
}

// The device-side convergence loop for (batch size, form): null when
// conditional graph nodes are not available (the host then replays the
// iteration graph).
static cudaGraphExec_t loop_graph(gpw_poisson* ps, int nb, int prec) {
  gpw_poisson::GraphKey key{nb, prec};
  auto it = ps->loops.find(key);
  if (it != ps->loops.end()) return it->second;
  cudaGraphExec_t ge = nullptr;
  cudaGraph_t parent;
  if (cudaGraphCreate(&parent, 0) == cudaSuccess) {
    cudaGraphNode_t node;
    if (add_loop_node(ps, nb, prec, parent, nullptr, &node) != cudaSuccess ||
        cudaGraphInstantiate(&ge, parent, 0) != cudaSuccess)
      ge = nullptr;
    cudaGraphDestroy(parent);
  }
  cudaGetLastError();  // a failed attempt leaves no sticky state
  ps->loops[key] = ge;
  return ge;
}

// Copies between a caller's C-contiguous (nb, n0, n1, n2) array and the
// engine's row-pitched level-0 layout, as a kernel (no copy engine: the
// caller's own host<->device transfers of other batches may be in flight).
static cudaError_t pitch_copy(const GridView& v, int nb, const double* src, int64_t src_pitch, double* dst,
                              int64_t dst_pitch, cudaStream_t st) {
  const int64_t rows = (int64_t)v.n[0] * v.n[1] * nb;
  const int thr = 256;
  const int64_t blocks = (rows + thr / 32 - 1) / (thr / 32);
  pitch_copy_kernel<<<(unsigned)blocks, thr, 0, st>>>(rows, (int)v.n[2], src, src_pitch, dst, dst_pitch);
  return cudaGetLastError();
}

// Solve-state set-up and inputs: eps, niter = 1, active = 1, phi / rho
// copied into the engine layout, and (float32 form) the initial defect.
// Everything is a kernel on `st`; eps travels through the mapped mailbox,
// which the previous solve on this engine has finished with (solves end in
// a stream synchronisation).
static int solve_prologue(gpw_poisson* ps, double* phi, const double* rho, int nb, const double* eps, int maxiter,
                          int precision, cudaStream_t st, int slot = 0) {
  Level& L0 = ps->lv[0];
  std::memcpy(ps->h_eps[slot], eps, (size_t)nb * 8);
  solve_setup_kernel<<<1, 128, 0, st>>>(nb, ps->m_eps[slot], maxiter, (double*)ps->d_eps.ptr, (int*)ps->d_niter.ptr,
                                        (unsigned char*)ps->d_active.ptr, (int*)ps->d_maxiter.ptr);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = pitch_copy(L0.v, nb, phi, L0.v.n[2], (double*)L0.phi[0].ptr, L0.v.s1, st);
  if (e == cudaSuccess) e = pitch_copy(L0.v, nb, rho, L0.v.n[2], (double*)L0.rho.ptr, L0.v.s1, st);
  if (e != cudaSuccess) return cuda_fail(e, "poisson setup");
  if (precision == 1 && fused_dc(ps)) {
    // initial defect: float32 rhs and first level-0 sweep, fused
    e = launch_stencil_dc(*L0.op, MODE_RESID_DC, L0.phi[0].ptr, L0.v, L0.rho32.ptr, L0.phi32[0].ptr, L0.rho.ptr, nb,
                          1.0, L0.wpre[1][0], (const unsigned char*)ps->d_active.ptr, ps->sums.gs(), st);
    if (e != cudaSuccess) return cuda_fail(e, "poisson initial defect");
  } else if (precision == 1) {
    // initial residual for the first defect-correction step
    Boundary bc = make_boundary(L0.op->periodic, GPW_F64, nullptr);
    e = launch_stencil(*L0.op, GPW_F64, MODE_RESIDUAL, L0.phi[0].ptr, L0.v, ps->d_r64.ptr, L0.v, L0.rho.ptr, L0.v, nb,
                       bc, 1.0, (const unsigned char*)ps->d_active.ptr, ps->sums.gs(), st);
    if (e != cudaSuccess) return cuda_fail(e, "poisson initial residual");
  }
  stamp_kernel<<<1, 1, 0, st>>>((int64_t*)ps->d_t0.ptr);
  if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "stamp");
  return GPW_OK;
}

// Result copy and per-solve statistics into mailbox `slot` (kernels on
// `st`, nothing waited for).
static cudaError_t solve_finish(gpw_poisson* ps, double* phi, int nb, cudaStream_t st, int slot) {
  Level& L0 = ps->lv[0];
  cudaError_t e = pitch_copy(L0.v, nb, (const double*)L0.phi[0].ptr, L0.v.s1, phi, L0.v.n[2], st);
  if (e == cudaSuccess) {
    solve_readback_kernel<<<1, 128, 0, st>>>(nb, (const int*)ps->d_niter.ptr, (const double*)ps->d_err.ptr,
                                             ps->m_niter[slot], ps->m_err[slot]);
    e = cudaGetLastError();
  }
  return e;
}

// The per-solve statistics of a finished solve from mailbox `slot`.
static int solve_collect(gpw_poisson* ps, int nb, int maxiter, int* niter, double* error, int slot) {
  std::memcpy(niter, ps->h_niter[slot], (size_t)nb * 4);
  std::memcpy(error, ps->h_err[slot], (size_t)nb * 8);
  for (int b = 0; b < nb; ++b)
    if (niter[b] >= maxiter) return fail(GPW_ECONV, "Poisson solver did not converge in maxiter iterations");
  return GPW_OK;
}

// Result copy and per-solve statistics, then the one stream synchronisation
// of a synchronous solve.
static int solve_epilogue(gpw_poisson* ps, double* phi, int nb, int maxiter, int* niter, double* error,
                          cudaStream_t st) {
  cudaError_t e = solve_finish(ps, phi, nb, st, 0);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_fail(e, "poisson result copies");
  return solve_collect(ps, nb, maxiter, niter, error, 0);
}

static int check_solve_args(gpw_poisson* ps, int64_t nbatch, int precision, int maxiter) {
  if (nbatch < 1 || nbatch > ps->nbmax) return fail(GPW_EINVAL, "poisson: nbatch out of range");
  if (precision != 0 && precision != 1) return fail(GPW_EINVAL, "poisson: precision must be 0 or 1");
  if (precision == 1 && ps->relax_method != 2) return fail(GPW_ENOTSUP, "poisson: float32 form needs Jacobi");
  if (maxiter < 1) return fail(GPW_EINVAL, "poisson: maxiter < 1");
  int rc;
  if (precision == 1 && (rc = ensure_f32(ps))) return rc;
  return GPW_OK;
}

int gpw_poisson_solve(gpw_poisson* ps, double* phi, const double* rho, int64_t nbatch, const double* eps, int maxiter,
                      int precision, int* niter, double* error, gpw_stream stream) {
  if (!ps || !phi || !rho || !eps || !niter || !error) return fail(GPW_EINVAL, "null argument");
  int rc = check_solve_args(ps, nbatch, precision, maxiter);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  const int nb = (int)nbatch;
  gpw_poisson::GraphKey key{nbatch, precision};
  cudaGraphExec_t iter = nullptr;
  if ((rc = iteration_graph(ps, nb, precision, st, &iter))) return rc;
  cudaGraphExec_t loop = ps->device_loop ? loop_graph(ps, nb, precision) : nullptr;
  if ((rc = solve_prologue(ps, phi, rho, nb, eps, maxiter, precision, st))) return rc;
  ps->last_kernels = (precision == 1) ? 2 : 1;
  ps->last_graphs = 0;
  cudaError_t e;
  if (loop) {
    // the whole convergence loop on the device: one graph launch
    if ((e = cudaGraphLaunch(loop, st)) != cudaSuccess) return cuda_fail(e, "loop graph launch");
  } else {
    // replay until no solve of the batch is active
    for (int it = 0; it < maxiter + 1; ++it) {
      if ((e = cudaGraphLaunch(iter, st)) != cudaSuccess) return cuda_fail(e, "graph launch");
      ps->last_graphs += 1;
      ps->last_kernels += ps->graph_kernels[key];
      if ((e = cudaMemcpyAsync(ps->h_any, ps->d_any.ptr, sizeof(int), cudaMemcpyDeviceToHost, st)) != cudaSuccess)
        return cuda_fail(e, "flag copy");
      if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return cuda_fail(e, "V-cycle");
      if (!*ps->h_any) break;
    }
  }
  rc = solve_epilogue(ps, phi, nb, maxiter, niter, error, st);
  if (loop) {
    // iterations run = the largest iteration count of the batch
    int64_t mx = 0;
    for (int b = 0; b < nb; ++b) mx = std::max<int64_t>(mx, niter[b]);
    ps->last_graphs = mx;
    ps->last_kernels += mx * ps->graph_kernels[key];
  }
  return rc;
}

// Convergence loop driver: on (default) the device-side loop (a conditional
// graph node); off the host replays the iteration graph, one graph launch
// per outer iteration (the same kernels; profilers that cannot see inside
// conditional graph nodes time each kernel this way).
extern "C" int gpw_poisson_set_device_loop(gpw_poisson* ps, int on) {
  if (!ps) return fail(GPW_EINVAL, "null argument");
  ps->device_loop = on != 0;
  return GPW_OK;
}

// A solve enqueued on `stream` without waiting for it (the device-side
// loop only): results go to mailbox `slot` (0 or 1) and are read by
// gpw_poisson_collect once the caller has seen the stream's work finish.  A
// slot is not reused before its solve has been collected.
int gpw_poisson_solve_async(gpw_poisson* ps, double* phi, const double* rho, int64_t nbatch, const double* eps,
                            int maxiter, int precision, int slot, gpw_stream stream) {
  if (!ps || !phi || !rho || !eps) return fail(GPW_EINVAL, "null argument");
  if (slot < 0 || slot > 1) return fail(GPW_EINVAL, "poisson: slot must be 0 or 1");
  int rc = check_solve_args(ps, nbatch, precision, maxiter);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  const int nb = (int)nbatch;
  cudaGraphExec_t iter = nullptr;
  if ((rc = iteration_graph(ps, nb, precision, st, &iter))) return rc;
  cudaGraphExec_t loop = ps->device_loop ? loop_graph(ps, nb, precision) : nullptr;
  if (!loop) return fail(GPW_ENOTSUP, "poisson: asynchronous solves need the device-side loop");
  if ((rc = solve_prologue(ps, phi, rho, nb, eps, maxiter, precision, st, slot))) return rc;
  cudaError_t e = cudaGraphLaunch(loop, st);
  if (e != cudaSuccess) return cuda_fail(e, "loop graph launch");
  if ((e = solve_finish(ps, phi, nb, st, slot)) != cudaSuccess) return cuda_fail(e, "poisson result copies");
  return GPW_OK;
}

int gpw_poisson_collect(gpw_poisson* ps, int64_t nbatch, int maxiter, int precision, int slot, int* niter,
                        double* error) {
  if (!ps || !niter || !error) return fail(GPW_EINVAL, "null argument");
  if (slot < 0 || slot > 1 || nbatch < 1 || nbatch > ps->nbmax) return fail(GPW_EINVAL, "poisson: bad arguments");
  const int rc = solve_collect(ps, (int)nbatch, maxiter, niter, error, slot);
  int64_t mx = 0;
  for (int b = 0; b < nbatch; ++b) mx = std::max<int64_t>(mx, niter[b]);
  ps->last_graphs = mx;
  ps->last_kernels = (precision == 1 ? 2 : 1) + mx * ps->graph_kernels[gpw_poisson::GraphKey{nbatch, precision}];
  return rc;
}

// Per-solve latency of the last solve: device time from the start of the
// iterations to the end of the iteration in which each solve converged.
extern "C" int gpw_poisson_last_latency(gpw_poisson* ps, int64_t nbatch, double* ms, gpw_stream stream) {
  if (!ps || !ms) return fail(GPW_EINVAL, "null argument");
  if (nbatch < 1 || nbatch > ps->nbmax) return fail(GPW_EINVAL, "poisson: nbatch out of range");
  std::vector<int64_t> t(nbatch + 1);
  cudaStream_t st = (cudaStream_t)stream;
  cudaError_t e;
  if ((e = cudaMemcpyAsync(t.data(), ps->d_tdone.ptr, nbatch * 8, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
      (e = cudaMemcpyAsync(t.data() + nbatch, ps->d_t0.ptr, 8, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
      (e = cudaStreamSynchronize(st)) != cudaSuccess)
    return cuda_fail(e, "latency copies");
  for (int64_t b = 0; b < nbatch; ++b) ms[b] = (double)(t[b] - t[nbatch]) * 1e-6;
  return GPW_OK;
}

// Several engines (e.g. one per grid size) solved by ONE graph launch: a
// parent graph with one device-side while loop per engine; the loops are
// independent branches and run concurrently.  Arguments are per engine as
// in gpw_poisson_solve.  Cached per (engines, batch sizes, form).
struct MultiKey {
  std::vector<const void*> eng;
  std::vector<int> nb;
  int prec;
  bool operator<(const MultiKey& o) const {
    if (prec != o.prec) return prec < o.prec;
    if (eng != o.eng) return eng < o.eng;
    return nb < o.nb;
  }
};
static std::mutex g_multi_mu;
static std::map<MultiKey, cudaGraphExec_t> g_multi;

extern "C" int gpw_poisson_solve_many(int nengines, gpw_poisson* const* engines, double* const* phis,
                                      const double* const* rhos, const int64_t* nbatch,
                                      const double* const* eps, int maxiter, int precision, int* const* niters,
                                      double* const* errors, gpw_stream stream) {
  if (nengines < 1 || !engines || !phis || !rhos || !nbatch || !eps || !niters || !errors)
    return fail(GPW_EINVAL, "null argument");
  cudaStream_t st = (cudaStream_t)stream;
  MultiKey key;
  key.prec = precision;
  int rc;
  for (int i = 0; i < nengines; ++i) {
    gpw_poisson* ps = engines[i];
    if (!ps || !phis[i] || !rhos[i] || !eps[i] || !niters[i] || !errors[i]) return fail(GPW_EINVAL, "null argument");
    for (int j = 0; j < i; ++j)
      if (engines[j] == ps) return fail(GPW_EINVAL, "solve_many: an engine appears twice");
    if ((rc = check_solve_args(ps, nbatch[i], precision, maxiter))) return rc;
    cudaGraphExec_t iter;
    if ((rc = iteration_graph(ps, (int)nbatch[i], precision, st, &iter))) return rc;  // tunes the stencils
    key.eng.push_back(ps);
    key.nb.push_back((int)nbatch[i]);
  }
  cudaGraphExec_t ge = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_multi_mu);
    auto it = g_multi.find(key);
    if (it != g_multi.end()) ge = it->second;
  }
  if (!ge) {
    cudaGraph_t parent;
    cudaError_t e = cudaGraphCreate(&parent, 0);
    if (e != cudaSuccess) return cuda_fail(e, "graph create");
    for (int i = 0; i < nengines && e == cudaSuccess; ++i) {
      cudaGraphNode_t node;
      e = add_loop_node(engines[i], (int)nbatch[i], precision, parent, nullptr, &node);
    }
    if (e == cudaSuccess) e = cudaGraphInstantiate(&ge, parent, 0);
    cudaGraphDestroy(parent);
    if (e != cudaSuccess) return cuda_fail(e, "solve_many: device-side loop graph");
    std::lock_guard<std::mutex> lock(g_multi_mu);
    g_multi[key] = ge;
  }
  for (int i = 0; i < nengines; ++i)
    if ((rc = solve_prologue(engines[i], phis[i], rhos[i], (int)nbatch[i], eps[i], maxiter, precision, st)))
      return rc;
  // one clock origin for every engine's latencies: just before the launch
  stamp_kernel<<<1, 1, 0, st>>>((int64_t*)engines[0]->d_t0.ptr);
  for (int i = 1; i < nengines; ++i) {
    copy_kernel<int64_t><<<1, 32, 0, st>>>(1, (const int64_t*)engines[0]->d_t0.ptr, (int64_t*)engines[i]->d_t0.ptr);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "clock origin");
  }
  cudaError_t e = cudaGraphLaunch(ge, st);
  if (e != cudaSuccess) return cuda_fail(e, "solve_many launch");
  int first_rc = GPW_OK;
  for (int i = 0; i < nengines; ++i) {
    gpw_poisson* ps = engines[i];
    rc = solve_epilogue(ps, phis[i], (int)nbatch[i], maxiter, niters[i], errors[i], st);
    if (rc && !first_rc) first_rc = rc;
    int64_t mx = 0;
    for (int b = 0; b < nbatch[i]; ++b) mx = std::max<int64_t>(mx, niters[i][b]);
    ps->last_graphs = mx;
    ps->last_kernels = mx * ps->graph_kernels[gpw_poisson::GraphKey{nbatch[i], precision}] + (precision ? 2 : 1);
  }
  return first_rc;
}

// Float32 inner V-cycle schedule of the defect-correction form (precision 1):
// per level npre[l] / npost[l] Jacobi sweeps with their own weights, listed
// level by level in `weights` (npre[l] pre-sweep weights, then npost[l]
// post-sweep weights; nweights = the total).  The coarsest level runs only
// its post-sweeps (its pre-sweep weights are skipped).  The float64 method
// keeps the reference schedule.  Captured graphs of the float32 form are
// discarded.
// Drop the captured graphs of the float32 form (its schedule or launch plan changed).
static void discard_f32_graphs(gpw_poisson* ps) {
  for (auto it = ps->graphs.begin(); it != ps->graphs.end();) {
    if (it->first.prec == 1) {
      cudaGraphExecDestroy(it->second);
      ps->graph_kernels.erase(it->first);
      it = ps->graphs.erase(it);
    } else {
      ++it;
    }
  }
  for (auto it = ps->loops.begin(); it != ps->loops.end();) {
    if (it->first.prec == 1) {
      if (it->second) cudaGraphExecDestroy(it->second);
      it = ps->loops.erase(it);
    } else {
      ++it;
    }
  }
}

extern "C" int gpw_poisson_set_inner_schedule(gpw_poisson* ps, const int* npre, const int* npost,
                                              const double* weights, int nweights) {
  if (!ps || !npre || !npost || !weights) return fail(GPW_EINVAL, "null argument");
  const int nl = (int)ps->lv.size();
  int total = 0;
  for (int l = 0; l < nl; ++l) {
    const int pre = (l + 1 < nl) ? npre[l] : 0;
    if (npre[l] < 0 || npost[l] < 0 || pre + npost[l] > CG_MAXW)
      return fail(GPW_EINVAL, "inner schedule: sweep counts out of range");
    if (l == 0 && nl > 1 && (pre < 1 || npost[l] < 1))
      return fail(GPW_EINVAL, "inner schedule: level 0 needs at least one pre- and one post-sweep");
    total += npre[l] + npost[l];
  }
  if (total != nweights) return fail(GPW_EINVAL, "inner schedule: weight count does not match the sweep counts");
  int k = 0;
  for (int l = 0; l < nl; ++l) {
    Level& L = ps->lv[l];
    const int pre = (l + 1 < nl) ? npre[l] : 0;
    L.wpre[1].assign(weights + k, weights + k + pre);
    k += npre[l];
    L.wpost[1].assign(weights + k, weights + k + npost[l]);
    k += npost[l];
  }
  setup_coarse(ps, 1);
  discard_f32_graphs(ps);
  return GPW_OK;
}

// Level-0 residual and restriction in one launch (float32 form; on by
// default where it applies): on = 0 launches them separately.  Both plans
// compute the same values.  Captured float32 graphs are discarded.
extern "C" int gpw_poisson_set_fusion(gpw_poisson* ps, int on) {
  if (!ps) return fail(GPW_EINVAL, "null argument");
  if (on < 0 || on > 2) return fail(GPW_EINVAL, "set_fusion: on must be 0, 1 or 2");
  ps->use_rr = on != 0;
  ps->use_rr_coarse = on == 1;
  discard_f32_graphs(ps);
  return GPW_OK;
}

// Cluster launch of the level above the coarse kernel's first level (float32
// form; on by default where it applies): on = 0 runs that level as separate
// stencil and transfer launches again.  Captured float32 graphs are discarded.
extern "C" int gpw_poisson_set_cluster(gpw_poisson* ps, int on) {
  if (!ps) return fail(GPW_EINVAL, "null argument");
  ps->use_cluster = on != 0;
  setup_coarse(ps, 1);
  discard_f32_graphs(ps);
  return GPW_OK;
}

// Live per-launch breakdown of one iteration: the iteration's launches run
// eagerly on the engine's buffers (contents overwritten; call between
// solves, after a solve of this batch size and form tuned the stencils),
// each followed by an event.  Writes up to `cap` entries: labels
// (NUL-separated into `labels`, `labels_len` bytes) and milliseconds.
extern "C" int gpw_poisson_profile_iteration(gpw_poisson* ps, int64_t nbatch, int precision, int reps, char* labels,
                                             int labels_len, double* ms, int cap, int* count, gpw_stream stream) {
  if (!ps || !labels || !ms || !count || cap < 1 || reps < 1) return fail(GPW_EINVAL, "null argument");
  int rc = check_solve_args(ps, nbatch, precision, 1);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  const int nb = (int)nbatch;
  std::vector<unsigned char> act(nb, 1);
  std::vector<std::string> names;
  std::vector<double> acc;
  cudaError_t e;
  for (int rep = 0; rep <= reps; ++rep) {
    // every solve active (the state of a first iteration)
    e = cudaMemcpyAsync(ps->d_active.ptr, act.data(), nb, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_fail(e, "profile setup");
    std::vector<std::pair<std::string, cudaEvent_t>> ev;
    cudaEvent_t e0;
    cudaEventCreate(&e0);
    cudaEventRecord(e0, st);
    cudaError_t re = record_iteration(ps, nb, precision, st, false, nullptr, &ev);
    e = cudaStreamSynchronize(st);
    if (re == cudaSuccess && e == cudaSuccess && rep > 0) {  // rep 0 warms up
      cudaEvent_t prev = e0;
      for (size_t i = 0; i < ev.size(); ++i) {
        float t = 0.f;
        cudaEventElapsedTime(&t, prev, ev[i].second);
        prev = ev[i].second;
        if (rep == 1) {
          names.push_back(ev[i].first);
          acc.push_back(0.0);
        }
        if (i < acc.size()) acc[i] += t;
      }
    }
    cudaEventDestroy(e0);
    for (auto& x : ev) cudaEventDestroy(x.second);
    if (re != cudaSuccess) return cuda_fail(re, "profile iteration");
    if (e != cudaSuccess) return cuda_fail(e, "profile sync");
  }
  int n = 0, off = 0;
  for (size_t i = 0; i < names.size() && n < cap; ++i) {
    const int len = (int)names[i].size() + 1;
    if (off + len > labels_len) break;
    std::memcpy(labels + off, names[i].c_str(), len);
    off += len;
    ms[n++] = acc[i] / reps;
  }
  *count = n;
  return GPW_OK;
}
