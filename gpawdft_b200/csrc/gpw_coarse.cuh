// The coarse end of the multigrid V-cycle in one CTA per solve.
//
// Below ~15^3 points a level is too small to fill the GPU: at 127^3 the
// levels 15^3, 7^3, 3^3 and 1^3 of gpaw/poisson.py's hierarchy cost ~35
// launches per V-cycle, each bound by launch latency.  This kernel runs the
// recursive part of iterate2 (gpaw/poisson.py:331-356) from a level `lc`
// down to the coarsest level and back for one batch member per CTA, with
// every level's phi (two ping-pong buffers) and rho resident in shared
// memory:
//   for l = lc .. L-1:  pre-sweeps, r = A phi - rho, rho_{l+1} = R r,
//                       phi_{l+1} = 0
//   coarsest:           post-sweeps
//   for l = L-1 .. lc:  phi_l -= I phi_{l+1}, post-sweeps
// The input is rho_lc (written by the restriction from level lc-1), the
// output phi_lc (read by the interpolation to level lc-1).
//
// Operators are the 7-point (nn=1) Laplacians of the coarse levels
// (gpaw/poisson.py:118-130) with weighted-Jacobi sweeps, one weight per
// sweep.  Restriction and interpolation are the K=2 transformers
// (c/bmgs/restrict.c:37-39, c/bmgs/interpolate.c:31-33) evaluated with the
// same expressions as gpw_transfer_k2.cuh; boundaries are zero or periodic
// (real data, no Bloch phase).
#pragma once
#include <cooperative_groups.h>

#include "gpw_common.cuh"
#include "gpw_transfer.cuh"
#include "gpw_transfer_k2.cuh"

namespace gpw {

constexpr int CG_MAXL = 8;       // levels handled inside the kernel
constexpr int CG_MAXW = 16;      // sweep weights per level (pre then post)
constexpr int CG_THREADS = 512;  // threads per CTA

struct CoarseLevel {
  int n[3];
  int periodic[3];
  int pts;                // elements per buffer: n0 n1 n2 (padded form: (n0+2)(n1+2)(n2+2))
  int base;               // element offset of the level's buffers: phi0, phi1, rho
  double cc;              // centre coefficient
  double cm[3], cp[3];    // neighbour coefficients at offsets -1 / +1 per axis
  int npre, npost;
  double w[CG_MAXW];      // pre-sweep weights, then post-sweep weights
  int rpad0[3];           // restriction to the next level: low padding
  int ipad0[3], iskip0[3];  // interpolation from the next level
};

struct CoarseArgs {
  int nl;                 // levels in the kernel (lc .. L)
  int padded;             // zero boundaries everywhere: padded layout (see below)
  CoarseLevel lv[CG_MAXL];
  const void* rho;        // rho of level lc, engine layout
  GridView vrho;
  void* phi;              // phi of level lc (result)
  GridView vphi;
  const unsigned char* active;
};

__device__ __forceinline__ int cg_wrap(int i, int n, int periodic, bool& ok) {
  ok = true;
  if (i >= 0 && i < n) return i;
  if (!periodic) {
    ok = false;
    return 0;
  }
  i %= n;
  return i < 0 ? i + n : i;
}

template <typename S>
__device__ __forceinline__ S cg_at(const S* buf, const CoarseLevel& L, int i0, int i1, int i2) {
  bool o0, o1, o2;
  i0 = cg_wrap(i0, L.n[0], L.periodic[0], o0);
  i1 = cg_wrap(i1, L.n[1], L.periodic[1], o1);
  i2 = cg_wrap(i2, L.n[2], L.periodic[2], o2);
  return (o0 && o1 && o2) ? buf[(i0 * L.n[1] + i1) * L.n[2] + i2] : S(0);
}

__device__ __forceinline__ void cg_index(const CoarseLevel& L, int i, int& i0, int& i1, int& i2) {
  i2 = i % L.n[2];
  const int t = i / L.n[2];
  i1 = t % L.n[1];
  i0 = t / L.n[1];
}

// sum_{p != 0} c_p phi[x + o_p]
template <typename S>
__device__ __forceinline__ S cg_offdiag(const S* phi, const CoarseLevel& L, int i0, int i1, int i2) {
  S av = (S)L.cm[2] * cg_at(phi, L, i0, i1, i2 - 1);
  av = fmac((S)L.cp[2], cg_at(phi, L, i0, i1, i2 + 1), av);
  av = fmac((S)L.cm[1], cg_at(phi, L, i0, i1 - 1, i2), av);
  av = fmac((S)L.cp[1], cg_at(phi, L, i0, i1 + 1, i2), av);
  av = fmac((S)L.cm[0], cg_at(phi, L, i0 - 1, i1, i2), av);
  av = fmac((S)L.cp[0], cg_at(phi, L, i0 + 1, i1, i2), av);
  return av;
}

// dst = (1 - w) src + (w / c0) (rho - sum_{p != 0} c_p src[x + o_p])   (c/bmgs/relax.c:62)
template <typename S>
__device__ __forceinline__ void cg_jacobi(const CoarseLevel& L, const S* src, S* dst, const S* rho, double wd) {
  const S w = (S)wd, wc = w / (S)L.cc;
  for (int i = threadIdx.x; i < L.pts; i += blockDim.x) {
    int i0, i1, i2;
    cg_index(L, i, i0, i1, i2);
    const S av = cg_offdiag(src, L, i0, i1, i2);
    dst[i] = (S(1) - w) * src[i] + wc * (rho[i] - av);
  }
  __syncthreads();
}

// r = A phi - rho
template <typename S>
__device__ __forceinline__ void cg_residual(const CoarseLevel& L, const S* phi, S* r, const S* rho) {
  for (int i = threadIdx.x; i < L.pts; i += blockDim.x) {
    int i0, i1, i2;
    cg_index(L, i, i0, i1, i2);
    const S av = cg_offdiag(phi, L, i0, i1, i2);
    r[i] = fmac((S)L.cc, phi[i], av) - rho[i];
  }
  __syncthreads();
}

// rho_C = R r_F (K = 2) and phi_C = 0
template <typename S>
__device__ __forceinline__ void cg_restrict(const CoarseLevel& F, const S* r, const CoarseLevel& C, S* rho_c,
                                            S* phi_c) {
  for (int i = threadIdx.x; i < C.pts; i += blockDim.x) {
    int I0, I1, I2;
    cg_index(C, i, I0, I1, I2);
    const int c0 = 1 + 2 * I0 - F.rpad0[0], c1 = 1 + 2 * I1 - F.rpad0[1], c2 = 1 + 2 * I2 - F.rpad0[2];
    S y[3];
#pragma unroll
    for (int d0 = 0; d0 < 3; ++d0) {
      S z[3];
#pragma unroll
      for (int d1 = 0; d1 < 3; ++d1)
        z[d1] = r2(cg_at(r, F, c0 - 1 + d0, c1 - 1 + d1, c2 - 1), cg_at(r, F, c0 - 1 + d0, c1 - 1 + d1, c2),
                   cg_at(r, F, c0 - 1 + d0, c1 - 1 + d1, c2 + 1));
      y[d0] = r2(z[0], z[1], z[2]);
    }
    rho_c[i] = r2(y[0], y[1], y[2]);
    phi_c[i] = S(0);
  }
  __syncthreads();
}

// dst = base - I e_C (K = 2)
template <typename S>
__device__ __forceinline__ S cg_interp_plane(const S* e, const CoarseLevel& C, int u0, int u1, int u2, int e1,
                                             int e2) {
  S z0 = cg_at(e, C, u0, u1, u2);
  if (e2) z0 = i2h(z0, cg_at(e, C, u0, u1, u2 + 1));
  if (!e1) return z0;
  S z1 = cg_at(e, C, u0, u1 + 1, u2);
  if (e2) z1 = i2h(z1, cg_at(e, C, u0, u1 + 1, u2 + 1));
  return i2h(z0, z1);
}

template <typename S>
__device__ __forceinline__ void cg_interp_sub(const CoarseLevel& F, const S* base, S* dst, const CoarseLevel& C,
                                              const S* e) {
  for (int i = threadIdx.x; i < F.pts; i += blockDim.x) {
    int o0, o1, o2;
    cg_index(F, i, o0, o1, o2);
    const int t0 = o0 + F.iskip0[0], t1 = o1 + F.iskip0[1], t2 = o2 + F.iskip0[2];
    const int u0 = (t0 >> 1) - F.ipad0[0], u1 = (t1 >> 1) - F.ipad0[1], u2 = (t2 >> 1) - F.ipad0[2];
    S v = cg_interp_plane(e, C, u0, u1, u2, t1 & 1, t2 & 1);
    if (t0 & 1) v = i2h(v, cg_interp_plane(e, C, u0 + 1, u1, u2, t1 & 1, t2 & 1));
    dst[i] = base[i] - v;
  }
  __syncthreads();
}

// ---------------------------------------------------------------- padded form
// When every level has zero boundaries, each level buffer is stored with a
// one-point zero halo ((n0+2)(n1+2)(n2+2) elements, the halo never written):
// neighbours sit at fixed offsets and need no bounds checks, and each thread
// walks whole axis-0 columns by adding the plane stride, so no point pays an
// index division.  `pts` then counts the padded elements.  The transfers
// assume the zero-boundary K=2 tables: restriction pad 0 (fine centre
// 2I + 1), interpolation pad 1 and skip 1 on every axis.
struct PadGeom {
  int n0, n1, n2;
  int sy, sz;  // padded row and plane strides
  __device__ __forceinline__ explicit PadGeom(const CoarseLevel& L)
      : n0(L.n[0]), n1(L.n[1]), n2(L.n[2]), sy(L.n[2] + 2), sz((L.n[1] + 2) * (L.n[2] + 2)) {}
  __device__ __forceinline__ int at(int i0, int i1, int i2) const { return (i0 + 1) * sz + (i1 + 1) * sy + i2 + 1; }
};

// Walk the points of a padded level: each thread takes whole axis-0 columns
// (neighbours at fixed strides, no index divisions) when the level has at
// least as many columns as the CTA has threads; on smaller levels, where that
// would leave most threads idle and the rest walking long columns, the
// threads take single points.  body(i0, i1, i2, k), k the padded index.
template <typename F>
__device__ __forceinline__ void pg_points(const PadGeom& g, F body) {
  const int ncol = g.n1 * g.n2;
  if (ncol >= (int)blockDim.x) {
    for (int c = threadIdx.x; c < ncol; c += blockDim.x) {
      const int i1 = c / g.n2, i2 = c - i1 * g.n2;
      int k = g.at(0, i1, i2);
#pragma unroll 4
      for (int i0 = 0; i0 < g.n0; ++i0, k += g.sz) body(i0, i1, i2, k);
    }
  } else {
    for (int i = threadIdx.x; i < ncol * g.n0; i += blockDim.x) {
      const int i0 = i / ncol, c = i - i0 * ncol;
      const int i1 = c / g.n2, i2 = c - i1 * g.n2;
      body(i0, i1, i2, g.at(i0, i1, i2));
    }
  }
}

template <typename S>
__device__ __forceinline__ void pg_jacobi(const CoarseLevel& L, const S* __restrict__ src, S* __restrict__ dst,
                                          const S* __restrict__ rho, double wd) {
  const PadGeom g(L);
  const S w = (S)wd, wc = w / (S)L.cc;
  const S c0m = (S)L.cm[0], c0p = (S)L.cp[0], c1m = (S)L.cm[1], c1p = (S)L.cp[1], c2m = (S)L.cm[2],
          c2p = (S)L.cp[2];
  pg_points(g, [&](int, int, int, int k) {
    S av = c2m * src[k - 1];
    av = fmac(c2p, src[k + 1], av);
    av = fmac(c1m, src[k - g.sy], av);
    av = fmac(c1p, src[k + g.sy], av);
    av = fmac(c0m, src[k - g.sz], av);
    av = fmac(c0p, src[k + g.sz], av);
    dst[k] = (S(1) - w) * src[k] + wc * (rho[k] - av);
  });
  __syncthreads();
}

template <typename S>
__device__ __forceinline__ void pg_residual(const CoarseLevel& L, const S* __restrict__ phi, S* __restrict__ r,
                                            const S* __restrict__ rho) {
  const PadGeom g(L);
  const S c0m = (S)L.cm[0], c0p = (S)L.cp[0], c1m = (S)L.cm[1], c1p = (S)L.cp[1], c2m = (S)L.cm[2],
          c2p = (S)L.cp[2], cc = (S)L.cc;
  pg_points(g, [&](int, int, int, int k) {
    S av = c2m * phi[k - 1];
    av = fmac(c2p, phi[k + 1], av);
    av = fmac(c1m, phi[k - g.sy], av);
    av = fmac(c1p, phi[k + g.sy], av);
    av = fmac(c0m, phi[k - g.sz], av);
    av = fmac(c0p, phi[k + g.sz], av);
    r[k] = fmac(cc, phi[k], av) - rho[k];
  });
  __syncthreads();
}

// rho_C = R r_F and phi_C = 0 (zero boundaries: fine centre 2I + 1)
template <typename S>
__device__ __forceinline__ void pg_restrict(const CoarseLevel& F, const S* __restrict__ r, const CoarseLevel& C,
                                            S* __restrict__ rho_c, S* __restrict__ phi_c) {
  const PadGeom f(F), g(C);
  pg_points(g, [&](int I0, int I1, int I2, int k) {
    const int kf = f.at(2 * I0 + 1, 2 * I1 + 1, 2 * I2 + 1);  // fine centre
    S y[3];
#pragma unroll
    for (int d0 = 0; d0 < 3; ++d0) {
      S z[3];
#pragma unroll
      for (int d1 = 0; d1 < 3; ++d1) {
        const int q = kf + (d0 - 1) * f.sz + (d1 - 1) * f.sy;
        z[d1] = r2(r[q - 1], r[q], r[q + 1]);
      }
      y[d0] = r2(z[0], z[1], z[2]);
    }
    rho_c[k] = r2(y[0], y[1], y[2]);
    phi_c[k] = S(0);
  });
  __syncthreads();
}

// dst = base - I e_C (zero boundaries: skip0 = 1, pad0 = 1 on every axis)
template <typename S>
__device__ __forceinline__ S pg_interp_plane(const S* e, const PadGeom& g, int q, int e1, int e2) {
  S z0 = e[q];
  if (e2) z0 = i2h(z0, e[q + 1]);
  if (!e1) return z0;
  S z1 = e[q + g.sy];
  if (e2) z1 = i2h(z1, e[q + g.sy + 1]);
  return i2h(z0, z1);
}

template <typename S>
__device__ __forceinline__ void pg_interp_sub(const CoarseLevel& F, const S* __restrict__ base, S* __restrict__ dst,
                                              const CoarseLevel& C, const S* __restrict__ e) {
  const PadGeom f(F), g(C);
  pg_points(f, [&](int o0, int o1, int o2, int k) {
    // t = o + 1; coarse u = t / 2 - 1 (padded index u + 1 = t / 2), e = t & 1
    const int t0 = o0 + 1, t1 = o1 + 1, t2 = o2 + 1;
    const int e1 = t1 & 1, e2 = t2 & 1;
    const int q = (t0 >> 1) * g.sz + (t1 >> 1) * g.sy + (t2 >> 1);  // padded coarse index
    S v = pg_interp_plane(e, g, q, e1, e2);
    if (t0 & 1) v = i2h(v, pg_interp_plane(e, g, q + g.sz, e1, e2));
    dst[k] = base[k] - v;
  });
  __syncthreads();
}

template <typename S>
__device__ void coarse_vcycle_padded(const CoarseArgs& a, S* sm, int b) {
  const int nl = a.nl;
  int cur[CG_MAXL];
  // zero every buffer once (the halos stay zero), then load rho of level 0
  int total = 0;
  for (int l = 0; l < nl; ++l) total = max(total, a.lv[l].base + 3 * a.lv[l].pts);
  for (int i = threadIdx.x; i < total; i += blockDim.x) sm[i] = S(0);
  __syncthreads();
  {
    const CoarseLevel& L = a.lv[0];
    const PadGeom g(L);
    S* rho = sm + L.base + 2 * L.pts;
    const S* gr = static_cast<const S*>(a.rho) + (int64_t)b * a.vrho.sb;
    for (int c = threadIdx.x; c < g.n1 * g.n2; c += blockDim.x) {
      const int i1 = c / g.n2, i2 = c - i1 * g.n2;
      int k = g.at(0, i1, i2);
#pragma unroll 4
      for (int i0 = 0; i0 < g.n0; ++i0, k += g.sz) rho[k] = gr[(int64_t)i0 * a.vrho.s0 + (int64_t)i1 * a.vrho.s1 + i2];
    }
    __syncthreads();
  }
  for (int l = 0; l < nl; ++l) {
    const CoarseLevel& L = a.lv[l];
    S* P[2] = {sm + L.base, sm + L.base + L.pts};
    const S* rho = sm + L.base + 2 * L.pts;
    int c = 0;
    if (l == nl - 1) {
      for (int s = 0; s < L.npost; ++s, c = 1 - c) pg_jacobi(L, P[c], P[1 - c], rho, L.w[L.npre + s]);
      cur[l] = c;
      break;
    }
    for (int s = 0; s < L.npre; ++s, c = 1 - c) pg_jacobi(L, P[c], P[1 - c], rho, L.w[s]);
    cur[l] = c;
    pg_residual(L, P[c], P[1 - c], rho);
    const CoarseLevel& C = a.lv[l + 1];
    pg_restrict(L, P[1 - c], C, sm + C.base + 2 * C.pts, sm + C.base);
  }
  for (int l = nl - 2; l >= 0; --l) {
    const CoarseLevel& L = a.lv[l];
    const CoarseLevel& C = a.lv[l + 1];
    S* P[2] = {sm + L.base, sm + L.base + L.pts};
    const S* rho = sm + L.base + 2 * L.pts;
    int c = cur[l];
    pg_interp_sub(L, P[c], P[1 - c], C, sm + C.base + cur[l + 1] * C.pts);
    c = 1 - c;
    for (int s = 0; s < L.npost; ++s, c = 1 - c) pg_jacobi(L, P[c], P[1 - c], rho, L.w[L.npre + s]);
    cur[l] = c;
  }
  {
    const CoarseLevel& L = a.lv[0];
    const PadGeom g(L);
    const S* phi = sm + L.base + cur[0] * L.pts;
    S* gp = static_cast<S*>(a.phi) + (int64_t)b * a.vphi.sb;
    for (int c = threadIdx.x; c < g.n1 * g.n2; c += blockDim.x) {
      const int i1 = c / g.n2, i2 = c - i1 * g.n2;
      int k = g.at(0, i1, i2);
      for (int i0 = 0; i0 < g.n0; ++i0, k += g.sz) gp[(int64_t)i0 * a.vphi.s0 + (int64_t)i1 * a.vphi.s1 + i2] = phi[k];
    }
  }
}

template <typename S>
__global__ void __launch_bounds__(CG_THREADS, 1) coarse_vcycle_kernel(const CoarseArgs a) {
  pdl_wait();
  const int b = blockIdx.x;
  if (a.active && !a.active[b]) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  S* sm = reinterpret_cast<S*>(smem_raw);
  if (a.padded) {
    coarse_vcycle_padded(a, sm, b);
    return;
  }
  const int nl = a.nl;
  int cur[CG_MAXL];
  {
    const CoarseLevel& L = a.lv[0];
    S* phi = sm + L.base;
    S* rho = sm + L.base + 2 * L.pts;
    const S* g = static_cast<const S*>(a.rho) + (int64_t)b * a.vrho.sb;
    for (int i = threadIdx.x; i < L.pts; i += blockDim.x) {
      int i0, i1, i2;
      cg_index(L, i, i0, i1, i2);
      rho[i] = g[(int64_t)i0 * a.vrho.s0 + (int64_t)i1 * a.vrho.s1 + i2];
      phi[i] = S(0);
    }
    __syncthreads();
  }
  // descend
  for (int l = 0; l < nl; ++l) {
    const CoarseLevel& L = a.lv[l];
    S* P[2] = {sm + L.base, sm + L.base + L.pts};
    const S* rho = sm + L.base + 2 * L.pts;
    int c = 0;
    if (l == nl - 1) {
      for (int s = 0; s < L.npost; ++s, c = 1 - c) cg_jacobi(L, P[c], P[1 - c], rho, L.w[L.npre + s]);
      cur[l] = c;
      break;
    }
    for (int s = 0; s < L.npre; ++s, c = 1 - c) cg_jacobi(L, P[c], P[1 - c], rho, L.w[s]);
    cur[l] = c;
    cg_residual(L, P[c], P[1 - c], rho);
    const CoarseLevel& C = a.lv[l + 1];
    cg_restrict(L, P[1 - c], C, sm + C.base + 2 * C.pts, sm + C.base);
  }
  // ascend
  for (int l = nl - 2; l >= 0; --l) {
    const CoarseLevel& L = a.lv[l];
    const CoarseLevel& C = a.lv[l + 1];
    S* P[2] = {sm + L.base, sm + L.base + L.pts};
    const S* rho = sm + L.base + 2 * L.pts;
    int c = cur[l];
    cg_interp_sub(L, P[c], P[1 - c], C, sm + C.base + cur[l + 1] * C.pts);
    c = 1 - c;
    for (int s = 0; s < L.npost; ++s, c = 1 - c) cg_jacobi(L, P[c], P[1 - c], rho, L.w[L.npre + s]);
    cur[l] = c;
  }
  {
    const CoarseLevel& L = a.lv[0];
    const S* phi = sm + L.base + cur[0] * L.pts;
    S* g = static_cast<S*>(a.phi) + (int64_t)b * a.vphi.sb;
    for (int i = threadIdx.x; i < L.pts; i += blockDim.x) {
      int i0, i1, i2;
      cg_index(L, i, i0, i1, i2);
      g[(int64_t)i0 * a.vphi.s0 + (int64_t)i1 * a.vphi.s1 + i2] = phi[i];
    }
  }
}

// ---------------------------------------------------------------- cluster top levels
// The two levels above the one-CTA coarse levels (31^3 and 15^3 at
// N_c = 128, float32 inner cycles) in a thread-block cluster of CG_NCL CTAs
// per solve.  CTA r owns a slab of each: the top level's axis-0 planes
// [r n0 / CG_NCL, (r + 1) n0 / CG_NCL), and of the second level the planes
// whose restriction centres 2I + 1 lie in that range, each slab padded as
// above with one halo plane per side.  After every pass the cluster
// synchronises and each CTA copies its neighbours' boundary planes into its
// halo planes through distributed shared memory.  Both levels run their
// pre-sweeps and residual; the second level's residual is restricted into
// the third level's rho (global memory), CTA 0 runs the coarse kernel's
// V-cycle from there, and every CTA interpolates back up through its slabs
// and runs the post-sweeps.  One launch replaces ~18.  Every pass uses the
// padded functions above on a slab (a level of the CTA's own planes), so
// the arithmetic is that of the coarse kernel.
constexpr int CG_NCL = 8;            // CTAs per cluster (one solve)
constexpr int CG_CLUSTER_THREADS = 256;  // threads per CTA: two CTAs per SM (registers and shared memory)

struct ClusterTop {
  CoarseLevel L;     // the top level (padded form)
  CoarseLevel L2;    // the second level (padded form)
  const void* rho;   // top-level rho, engine layout
  void* phi;         // top-level phi: in, the first pre-sweep's iterate when first_done; out, the result
  GridView v;        // engine view of the top level
  int first_done;
  int slab_pts;      // padded elements of one top-level slab buffer: (maxp + 2)(n1 + 2)(n2 + 2)
  int slab2_pts;     // the same for the second level
  int next_pts;      // padded elements of the third level
};

struct ClusterArgs {
  CoarseArgs ca;     // third level .. coarsest (ca.rho: written here; ca.phi: read back)
  ClusterTop t;
};

// slab boundaries: the top level's plane r n0 / CG_NCL, the second level's
// half of it (capped at its extent)
__device__ __forceinline__ int slab_begin(int rank, int n0) { return rank * n0 / CG_NCL; }
__device__ __forceinline__ int slab2_begin(int rank, int n0, int m0) {
  return rank >= CG_NCL ? m0 : min(m0, slab_begin(rank, n0) / 2);
}

// Fill the halo planes of slab buffer `buf` (np own planes, plane size sz)
// from the neighbours' boundary planes; npm = the lower neighbour's planes.
// All of a thread's remote loads (up to 8 per plane and pass) are issued
// before its stores, so the copy pays the distributed-shared-memory latency
// about once.
template <typename S>
__device__ __forceinline__ void slab_exchange(cooperative_groups::cluster_group& cl, S* buf, int rank, int np,
                                              int npm, int sz) {
  constexpr int U = 8;
  cl.sync();
  const S* lo = rank > 0 ? cl.map_shared_rank(buf, rank - 1) + npm * sz : nullptr;
  const S* hi = rank < CG_NCL - 1 ? cl.map_shared_rank(buf, rank + 1) + sz : nullptr;
  S* dlo = buf;
  S* dhi = buf + (np + 1) * sz;
  for (int j0 = 0; j0 < sz; j0 += U * (int)blockDim.x) {
    S vl[U], vh[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int j = j0 + u * blockDim.x + threadIdx.x;
      if (j < sz) {
        if (lo) vl[u] = lo[j];
        if (hi) vh[u] = hi[j];
      }
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int j = j0 + u * blockDim.x + threadIdx.x;
      if (j < sz) {
        if (lo) dlo[j] = vl[u];
        if (hi) dhi[j] = vh[u];
      }
    }
  }
  __syncthreads();
}

// rho_C(I) = R r for the coarse planes I in [Ia, Ib) (centres 2I + 1 in the
// fine slab starting at plane z0), zero boundaries; written to `out` with
// plane stride os0, row stride os1 at plane index I - oI0 (padded or engine
// layout: `padded` adds the halo offset)
template <typename S>
__device__ __forceinline__ void slab_restrict(const CoarseLevel& F, const S* __restrict__ r, int z0, int Ia, int Ib,
                                              const CoarseLevel& C, S* __restrict__ out, int64_t os0, int64_t os1,
                                              int oI0, bool padded) {
  const PadGeom f(F);
  const int cn1 = C.n[1], cn2 = C.n[2];
  for (int c = threadIdx.x; c < cn1 * cn2; c += blockDim.x) {
    const int I1 = c / cn2, I2 = c - I1 * cn2;
    for (int I0 = Ia; I0 < Ib; ++I0) {
      const int kf = f.at(2 * I0 + 1 - z0, 2 * I1 + 1, 2 * I2 + 1);
      S y[3];
#pragma unroll
      for (int d0 = 0; d0 < 3; ++d0) {
        S z[3];
#pragma unroll
        for (int d1 = 0; d1 < 3; ++d1) {
          const int q = kf + (d0 - 1) * f.sz + (d1 - 1) * f.sy;
          z[d1] = r2(r[q - 1], r[q], r[q + 1]);
        }
        y[d0] = r2(z[0], z[1], z[2]);
      }
      const int p = padded ? 1 : 0;
      out[(int64_t)(I0 - oI0 + p) * os0 + (int64_t)(I1 + p) * os1 + I2 + p] = r2(y[0], y[1], y[2]);
    }
  }
  __syncthreads();
}

// dst = base - I e on the fine slab's planes (global planes [z0, z0 + F.n[0]));
// e holds coarse padded planes from global coarse plane c0 - 1 on (a coarse
// slab buffer, or the whole padded coarse level with c0 = 0)
template <typename S>
__device__ __forceinline__ void slab_interp_sub(const CoarseLevel& F, int z0, const S* __restrict__ base,
                                                S* __restrict__ dst, const CoarseLevel& C, const S* __restrict__ e,
                                                int c0) {
  const PadGeom f(F), g(C);
  for (int c = threadIdx.x; c < f.n1 * f.n2; c += blockDim.x) {
    const int o1 = c / f.n2, o2 = c - o1 * f.n2;
    const int t1 = o1 + 1, t2 = o2 + 1;
    const int e1 = t1 & 1, e2 = t2 & 1;
    const int qc = (t1 >> 1) * g.sy + (t2 >> 1);
    int k = f.at(0, o1, o2);
    for (int l0 = 0; l0 < f.n0; ++l0, k += f.sz) {
      const int t0 = z0 + l0 + 1;
      const int q = ((t0 >> 1) - c0) * g.sz + qc;
      S v = pg_interp_plane(e, g, q, e1, e2);
      if (t0 & 1) v = i2h(v, pg_interp_plane(e, g, q + g.sz, e1, e2));
      dst[k] = base[k] - v;
    }
  }
  __syncthreads();
}

template <typename S>
__global__ void __launch_bounds__(CG_CLUSTER_THREADS, 2) cluster_vcycle_kernel(const ClusterArgs a) {
  namespace cg = cooperative_groups;
  pdl_wait();
  cg::cluster_group cl = cg::this_cluster();
  const int rank = (int)cl.block_rank();
  const int b = blockIdx.x / CG_NCL;
  // the mask is read by every CTA of the cluster alike: all return, or none
  if (a.ca.active && !a.ca.active[b]) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  S* sm = reinterpret_cast<S*>(smem_raw);
  const ClusterTop& t = a.t;
  const CoarseLevel& T = t.L;
  const CoarseLevel& U = t.L2;
  const int n0 = T.n[0], m0 = U.n[0];
  // top-level slab
  const int z0 = slab_begin(rank, n0), z1 = slab_begin(rank + 1, n0), np = z1 - z0;
  const int npm = rank > 0 ? z0 - slab_begin(rank - 1, n0) : 0;
  CoarseLevel Ls = T;
  Ls.n[0] = np;
  const PadGeom gs(Ls);
  // second-level slab
  const int y0 = slab2_begin(rank, n0, m0), y1 = slab2_begin(rank + 1, n0, m0), mp = y1 - y0;
  const int mpm = rank > 0 ? y0 - slab2_begin(rank - 1, n0, m0) : 0;
  CoarseLevel Us = U;
  Us.n[0] = mp;
  const PadGeom gu(Us);
  S* P[2] = {sm, sm + t.slab_pts};
  S* rho = sm + 2 * t.slab_pts;
  S* Q[2] = {sm + 3 * t.slab_pts, sm + 3 * t.slab_pts + t.slab2_pts};
  S* rho2 = sm + 3 * t.slab_pts + 2 * t.slab2_pts;
  S* e = rho2 + t.slab2_pts;        // the third level's phi, padded
  S* csm = e + t.next_pts;          // CTA 0: the coarse kernel's levels
  for (int i = threadIdx.x; i < 3 * t.slab_pts + 3 * t.slab2_pts + t.next_pts; i += blockDim.x) sm[i] = S(0);
  __syncthreads();
  {
    const S* gr = static_cast<const S*>(t.rho) + (int64_t)b * t.v.sb;
    const S* gp = static_cast<const S*>(t.phi) + (int64_t)b * t.v.sb;
    for (int c = threadIdx.x; c < gs.n1 * gs.n2; c += blockDim.x) {
      const int i1 = c / gs.n2, i2 = c - i1 * gs.n2;
      int k = gs.at(0, i1, i2);
      // (unrolled: the loads of several planes are in flight together)
#pragma unroll 4
      for (int i0 = 0; i0 < np; ++i0, k += gs.sz) {
        const int64_t gi = (int64_t)(z0 + i0) * t.v.s0 + (int64_t)i1 * t.v.s1 + i2;
        rho[k] = gr[gi];
        if (t.first_done) P[0][k] = gp[gi];
      }
    }
  }
  // ---- top level: pre-sweeps, residual, restriction into the second level's slab
  int c = 0;
  slab_exchange(cl, P[0], rank, np, npm, gs.sz);
  for (int s = t.first_done; s < T.npre; ++s, c = 1 - c) {
    pg_jacobi(Ls, P[c], P[1 - c], rho, T.w[s]);
    slab_exchange(cl, P[1 - c], rank, np, npm, gs.sz);
  }
  pg_residual(Ls, P[c], P[1 - c], rho);
  slab_exchange(cl, P[1 - c], rank, np, npm, gs.sz);
  slab_restrict(Ls, P[1 - c], z0, y0, y1, U, rho2, gu.sz, gu.sy, y0, true);
  // ---- second level (phi = 0): pre-sweeps, residual, restriction into the third level (global)
  int d = 0;
  slab_exchange(cl, Q[0], rank, mp, mpm, gu.sz);  // (zeros: keeps the barrier sequence uniform)
  for (int s = 0; s < U.npre; ++s, d = 1 - d) {
    pg_jacobi(Us, Q[d], Q[1 - d], rho2, U.w[s]);
    slab_exchange(cl, Q[1 - d], rank, mp, mpm, gu.sz);
  }
  pg_residual(Us, Q[d], Q[1 - d], rho2);
  slab_exchange(cl, Q[1 - d], rank, mp, mpm, gu.sz);
  const CoarseLevel& C = a.ca.lv[0];
  slab_restrict(Us, Q[1 - d], y0, y0 / 2, min(C.n[0], y1 / 2), C,
                static_cast<S*>(const_cast<void*>(a.ca.rho)) + (int64_t)b * a.ca.vrho.sb, a.ca.vrho.s0, a.ca.vrho.s1,
                0, false);
  __threadfence();
  cl.sync();
  if (rank == 0) coarse_vcycle_padded(a.ca, csm, b);
  __threadfence();
  cl.sync();
  {
    const PadGeom g(C);
    const S* gp = static_cast<const S*>(a.ca.phi) + (int64_t)b * a.ca.vphi.sb;
    for (int q = threadIdx.x; q < g.n1 * g.n2; q += blockDim.x) {
      const int i1 = q / g.n2, i2 = q - i1 * g.n2;
      int k = g.at(0, i1, i2);
#pragma unroll 4
      for (int i0 = 0; i0 < g.n0; ++i0, k += g.sz)
        e[k] = __ldcg(gp + (int64_t)i0 * a.ca.vphi.s0 + (int64_t)i1 * a.ca.vphi.s1 + i2);
    }
    __syncthreads();
  }
  // ---- second level: interpolation, post-sweeps
  slab_interp_sub(Us, y0, Q[d], Q[1 - d], C, e, 0);
  d = 1 - d;
  slab_exchange(cl, Q[d], rank, mp, mpm, gu.sz);
  for (int s = 0; s < U.npost; ++s, d = 1 - d) {
    pg_jacobi(Us, Q[d], Q[1 - d], rho2, U.w[U.npre + s]);
    slab_exchange(cl, Q[1 - d], rank, mp, mpm, gu.sz);
  }
  // ---- top level: interpolation from the second level's slab (its halo planes included), post-sweeps
  slab_interp_sub(Ls, z0, P[c], P[1 - c], Us, Q[d], y0);
  c = 1 - c;
  slab_exchange(cl, P[c], rank, np, npm, gs.sz);
  for (int s = 0; s < T.npost; ++s, c = 1 - c) {
    pg_jacobi(Ls, P[c], P[1 - c], rho, T.w[T.npre + s]);
    if (s + 1 < T.npost) slab_exchange(cl, P[1 - c], rank, np, npm, gs.sz);
  }
  {
    S* gp = static_cast<S*>(t.phi) + (int64_t)b * t.v.sb;
    for (int q = threadIdx.x; q < gs.n1 * gs.n2; q += blockDim.x) {
      const int i1 = q / gs.n2, i2 = q - i1 * gs.n2;
      int k = gs.at(0, i1, i2);
      for (int i0 = 0; i0 < np; ++i0, k += gs.sz)
        gp[(int64_t)(z0 + i0) * t.v.s0 + (int64_t)i1 * t.v.s1 + i2] = P[c][k];
    }
  }
  cl.sync();  // no CTA leaves while a neighbour may still read its shared memory
}

}  // namespace gpw
