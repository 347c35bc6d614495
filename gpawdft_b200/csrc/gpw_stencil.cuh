// Finite-difference stencil kernels with fused halo fill.
//
// Reference semantics (c/operators.c:109-157 + c/bc.c:138-250 +
// c/bmgs/fd.c:16-51 / relax.c:46-71): every apply / relax sweep first builds
// a zero-filled padded copy of the grid, pastes the interior and copies
// periodic slabs (times Bloch phases) into the halo, then runs the stencil
// over the padded copy.  Here the padded copy never exists: each CTA streams
// the planes it needs through shared memory (cp.async, zero-fill for zero
// boundaries, wrapped addresses plus a phase fix-up for periodic ones) and
// the halo is produced on the fly.
//
// Two kernels:
//  * general_stencil_kernel -- any offsets within [-mp, mp]^3 (GUC Laplacians
//    with diagonal directions, Mehrstellen, gradients of skew cells).  A ring
//    of 2mp+2 planes lives in shared memory; every output gathers its
//    coefficients in the reference's order with unfused multiply / add, so
//    float64 results are bit-identical to c/bmgs/fd.c.
//  * star_stencil_kernel -- star (cfd) stencils of radius R: register-blocked
//    march along axis 0.  Each arriving plane contributes its in-plane part
//    (axes 1, 2 from shared memory, PY rows per thread held in registers) and
//    its axis-0 terms to 2R+1 running accumulators; an output plane is
//    complete R planes after its centre arrives.  Fused multiply-adds; float64
//    results agree with the reference to ~1e-16 relative.
// Both support three epilogues: APPLY (out = A in), RESIDUAL (out = A in -
// rho and a deterministic sum of |out|^2) and JACOBI (one weighted-Jacobi
// sweep, out = (1-w) in + w (rho - sum_{p!=0} c_p in[x+o_p]) / c_0).
#pragma once
#include "gpw_common.cuh"
#include "gpw_reduce.cuh"

namespace gpw {

// MODE_RESID_DC and MODE_JACOBI_ADD64 are the fused steps of the float32
// defect-correction form (TMA kernel only): RESID_DC reads float64 phi / rho
// and writes the float32 defect rhs = -(A phi - rho) to `out` and the first
// inner Jacobi iterate from zero, (w2 / c0) rhs, to `out2`, plus sum r^2;
// JACOBI_ADD64 is a float32 Jacobi sweep whose result is added to the float64
// array `out2` (phi += e) instead of being stored.  RESID_RESTRICT is a
// float32 residual that is not stored but restricted (K = 2, zero
// boundaries) into the next level: rho_c to `out` and that level's first
// Jacobi iterate from zero, (w2 / c0) rho_c with c0 the next level's
// diagonal, to `out2`, both in the coarse view `vco`.  JACOBI_SCALED_IN is a
// float32 Jacobi sweep whose iterate is never stored: it reads only the
// defect rhs (`in`) and takes phi = (w2 / c0) rhs -- the first inner sweep
// from zero -- with rho = rhs; A phi is formed as (w2 / c0) (A rhs), one
// scaling per output point (it rounds differently from a stencil of the
// stored iterate, within float32 rounding).
enum StencilMode {
  MODE_APPLY = 0,
  MODE_RESIDUAL = 1,
  MODE_JACOBI = 2,
  MODE_RESID_DC = 3,
  MODE_JACOBI_ADD64 = 4,
  MODE_RESID_RESTRICT = 5,
  MODE_JACOBI_SCALED_IN = 6,
  // the TMA star kernel's apply with a potential or aux term (a plain
  // MODE_APPLY instance is compiled without their loads and branches)
  MODE_APPLY_EPI = 7
};

// Number of tile-shape variants of the TMA star kernel (gpw_star_tma.cuh).
constexpr int TMA_NVARIANT = 11;  // 5 - 9: float32 only
// Axis-0 chunk count meaning "balanced split over the resident CTA slots"
// (the other counts: > 0 explicit, 0 the wave model, < 0 the model's count
// times its magnitude).
constexpr int TMA_SPLIT = -1;

constexpr int PMAX = 80;  // GUC n<=6 with 6 directions needs 73

struct StencilArgs {
  const void* in;
  void* out;        // may be null in RESIDUAL mode (norm only)
  const void* rho;  // RESIDUAL / JACOBI
  GridView vin, vout, vrho;
  Boundary bc;
  int zchunk;       // output planes of axis 0 per CTA
  int nchunk;       // chunks along axis 0 (gridDim.z = nchunk * nbatch)
  double w;         // Jacobi weight
  double c0;        // Jacobi diagonal coefficient
  const unsigned char* active;  // optional per-batch-member mask (null: all)
  GridSum gsum;     // RESIDUAL: per-batch-member segmented sum
  int nblk_seg;     // CTAs per batch member
  void* out2;       // RESID_DC: first inner iterate (float); JACOBI_ADD64: float64 phi
  double w2;        // RESID_DC: Jacobi weight of that first inner sweep
  GridView vco;     // RESID_RESTRICT: the next level's view (out, out2)
  const void* pot;  // APPLY: optional local potential, one grid in the output's
                    // layout and the element's scalar type: out = A in + pot in
  const void* aux;  // APPLY: optional grids in the output's layout and type:
  double aux_scale; //   out += aux_scale aux
  // TMA star kernel, balanced split (split_npl > 0): a 1D grid whose CTA i
  // takes units [i T / G, (i + 1) T / G) of T = split_gx split_gy split_nb
  // split_npl units, a unit being one plane (RESID_RESTRICT: one coarse
  // plane) of one tile column (split_gx x split_gy tiles per batch member,
  // split_nb members); a CTA's range may span several columns
  int split_gx, split_gy, split_nb, split_npl;
  int gdepth;       // general_block_kernel: planes loaded ahead of the one completed (1 - 4)
};

struct GeneralCoefs {
  int ncoef, mp;
  double coef[PMAX];
  signed char off[PMAX][3];
};

// ------------------------------------------------------------------ loaders
// Issue cp.async copies of plane p (tile rows y0-mp .. y0+TY+mp, columns
// x0-mp .. x0+TZ+mp) into `slot`.  Cells that fall in a zero halo are
// zero-filled by the copy engine.
template <typename T>
__device__ __forceinline__ void load_plane(T* slot, const T* in, const GridView& v, const Boundary& bc,
                                           int p, int y0, int x0, int mp, int H, int W) {
  const int tid = threadIdx.x + blockDim.x * threadIdx.y;
  const int nthr = blockDim.x * blockDim.y;
  int j0, s0;
  bool ok0 = wrap_axis(p, v.n[0], bc.periodic[0], j0, s0);
  for (int idx = tid; idx < H * W; idx += nthr) {
    int r = idx / W, c = idx - r * W;
    int j1, j2, s1, s2;
    bool ok = ok0 && wrap_axis(y0 - mp + r, v.n[1], bc.periodic[1], j1, s1) &&
              wrap_axis(x0 - mp + c, v.n[2], bc.periodic[2], j2, s2);
    const T* src = ok ? in + (int64_t)j0 * v.s0 + (int64_t)j1 * v.s1 + j2 : in;
    cp_async<sizeof(T)>(slot + idx, src, ok);
  }
}

// Multiply the periodic-halo cells of a landed plane by their Bloch phase
// product (same cell walk as load_plane, so each thread fixes its own copies).
template <typename T>
__device__ __forceinline__ void fix_plane(T* slot, const GridView& v, const Boundary& bc, int p, int y0,
                                          int x0, int mp, int H, int W) {
  if constexpr (EltTraits<T>::cpx) {
    const int tid = threadIdx.x + blockDim.x * threadIdx.y;
    const int nthr = blockDim.x * blockDim.y;
    int j0, s0;
    bool ok0 = wrap_axis(p, v.n[0], bc.periodic[0], j0, s0);
    if (!ok0) return;
    for (int idx = tid; idx < H * W; idx += nthr) {
      int r = idx / W, c = idx - r * W;
      int j1, j2, s1, s2;
      bool ok = wrap_axis(y0 - mp + r, v.n[1], bc.periodic[1], j1, s1) &&
                wrap_axis(x0 - mp + c, v.n[2], bc.periodic[2], j2, s2);
      if (!ok || (s0 < 0 && s1 < 0 && s2 < 0)) continue;
      // axis by axis, as the reference's chained halo copies apply them
      T val = slot[idx];
      if (s0 >= 0) val = phase_mul(bc.ph[0][s0], val);
      if (s1 >= 0) val = phase_mul(bc.ph[1][s1], val);
      if (s2 >= 0) val = phase_mul(bc.ph[2][s2], val);
      slot[idx] = val;
    }
  }
}

// ------------------------------------------------------------------ general
constexpr int GEN_TZ = 32, GEN_TY = 8;

// The weighted-Jacobi update of c/bmgs/relax.c:62, (1 - w) b + w (src - x) / c0,
// with every operation rounded on its own (no contraction into a fused
// multiply-add), as the reference's C evaluates it.
__device__ __forceinline__ double jacobi_rn(double w, double cur, double rho, double x, double c0) {
  return __dadd_rn(__dmul_rn(1.0 - w, cur), __ddiv_rn(__dmul_rn(w, __dsub_rn(rho, x)), c0));
}
__device__ __forceinline__ float jacobi_rn(float w, float cur, float rho, float x, float c0) {
  return __fadd_rn(__fmul_rn(1.0f - w, cur), __fdiv_rn(__fmul_rn(w, __fsub_rn(rho, x)), c0));
}

template <typename T, int MODE>
__global__ void __launch_bounds__(GEN_TZ* GEN_TY)
    general_stencil_kernel(const StencilArgs a, const GeneralCoefs k) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* ring = reinterpret_cast<T*>(smem_raw);
  __shared__ double red[32];
  using S = typename EltTraits<T>::S;

  const int mp = k.mp;
  const int H = GEN_TY + 2 * mp, W = GEN_TZ + 2 * mp, PS = H * W, NP = 2 * mp + 2;
  const int b = blockIdx.z / a.nchunk, chunk = blockIdx.z - b * a.nchunk;
  if (a.active && !a.active[b]) return;
  const int x0 = blockIdx.x * GEN_TZ, y0 = blockIdx.y * GEN_TY;
  const int n0 = a.vout.n[0];
  const int z0 = chunk * a.zchunk;
  const int z1 = min(n0, z0 + a.zchunk);
  const T* in = static_cast<const T*>(a.in) + (int64_t)b * a.vin.sb;
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int y = y0 + ty, x = x0 + tx;
  const bool inside = (y < a.vout.n[1]) && (x < a.vout.n[2]);
  double sumsq = 0.0;

  if (z0 < z1) {
    // prologue: planes z0-mp .. z0+mp
    for (int p = z0 - mp; p <= z0 + mp; ++p)
      load_plane<T>(ring + ((p - z0 + mp) % NP) * PS, in, a.vin, a.bc, p, y0, x0, mp, H, W);
    cp_async_commit();
    for (int o = z0; o < z1; ++o) {
      const int pn = o + mp + 1;
      if (o + 1 < z1) load_plane<T>(ring + ((pn - z0 + mp) % NP) * PS, in, a.vin, a.bc, pn, y0, x0, mp, H, W);
      cp_async_commit();
      cp_async_wait<1>();
      if (a.bc.use_phase) {
        if (o == z0) {
          for (int p = z0 - mp; p <= z0 + mp; ++p)
            fix_plane<T>(ring + ((p - z0 + mp) % NP) * PS, a.vin, a.bc, p, y0, x0, mp, H, W);
        } else {
          fix_plane<T>(ring + ((o + mp - z0 + mp) % NP) * PS, a.vin, a.bc, o + mp, y0, x0, mp, H, W);
        }
      }
      __syncthreads();
      if (inside) {
        T acc = zero<T>();
        const int cstart = (MODE == MODE_JACOBI) ? 1 : 0;
        for (int c = cstart; c < k.ncoef; ++c) {
          const int p = o + k.off[c][0];
          const T* sl = ring + ((p - z0 + mp) % NP) * PS;
          const T v = sl[(ty + mp + k.off[c][1]) * W + tx + mp + k.off[c][2]];
          acc = mac_rn((S)k.coef[c], v, acc);
        }
        const int64_t oi = (int64_t)b * a.vout.sb + (int64_t)o * a.vout.s0 + (int64_t)y * a.vout.s1 + x;
        if constexpr (MODE == MODE_APPLY) {
          if (a.pot) {
            const T* sl = ring + ((o - z0 + mp) % NP) * PS;
            const S pv = static_cast<const S*>(a.pot)[(int64_t)o * a.vout.s0 + (int64_t)y * a.vout.s1 + x];
            acc = fmac(pv, sl[(ty + mp) * W + tx + mp], acc);
          }
          if (a.aux) acc = fmac((S)a.aux_scale, static_cast<const T*>(a.aux)[oi], acc);
          static_cast<T*>(a.out)[oi] = acc;
        } else {
          const int64_t ri = (int64_t)b * a.vrho.sb + (int64_t)o * a.vrho.s0 + (int64_t)y * a.vrho.s1 + x;
          const T rho = static_cast<const T*>(a.rho)[ri];
          if constexpr (MODE == MODE_RESIDUAL) {
            const T r = sub(acc, rho);
            if (a.out) static_cast<T*>(a.out)[oi] = r;
            sumsq += norm2(r);
          } else {
            // (1 - w) * b + w * (src - x) / c0   (c/bmgs/relax.c:62)
            const T* sl = ring + ((o - z0 + mp) % NP) * PS;
            const T cur = sl[(ty + mp) * W + tx + mp];
            if constexpr (EltTraits<T>::cpx) {
              static_cast<T*>(a.out)[oi] = cur;  // relax is real-only (asserted on host)
            } else {
              const S w = (S)a.w, c0 = (S)a.c0;
              static_cast<T*>(a.out)[oi] = jacobi_rn(w, cur, rho, acc, c0);
            }
          }
        }
      }
      __syncthreads();
    }
  }
  if constexpr (MODE == MODE_RESIDUAL) {
    if (!a.gsum.partial) return;  // residual without its norm
    double tot = block_sum(sumsq, red);
    const int blk = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * chunk);
    grid_sum_finish(a.gsum, b, blk, a.nblk_seg, tot, red);
  }
}

// ------------------------------------------------------------------ general, register-blocked
// The same stencil, outputs and arithmetic as general_stencil_kernel, laid
// out for throughput: a CTA owns a TY x TZ tile (16 x 64 points with 128
// threads; 16 x 32 with 256 threads for 16-byte elements) and each thread
// PY x VX outputs (4 x 2; 2 x 1) in rows NTY apart and columns 32 apart, so
// a warp's shared-memory reads for one coefficient are consecutive.  Per coefficient the ring slot and in-plane
// offset come from shared-memory tables, so each output costs one
// shared-memory load and the reference's unfused multiply-add, in the
// reference's coefficient order (float64 results bit-identical to
// c/bmgs/fd.c).  Planes are staged row by row with cp.async, up to four
// planes ahead of the one completed: the wrapped axis-2 source index of a
// lane's columns is computed once per CTA, the axis-1 one once per row.
// What bounds it is that one shared-memory load per output and coefficient:
// at 19 - 37 coefficients the L1 / shared-memory pipe runs at ~70% (ncu).
// Taken where a ring of 2mp + 2 planes fits in shared memory, for radii
// mp <= 3 (compiled per radius, so the staged plane's shape and every
// in-plane offset of a thread's outputs are constants).
// (4 rows a thread for 4- and 8-byte elements, 128 threads: measured ~8%
// faster than 2 rows and 256 threads at 16 x 127^3 float64)
template <typename T, int MP, int PY_ = (sizeof(T) >= 16 ? 2 : 4), int NTY_ = (sizeof(T) >= 16 ? 8 : 4)>
struct GenBlk {
  static constexpr int VX = sizeof(T) >= 16 ? 1 : 2;  // outputs per thread along axis 2
  static constexpr int PY = PY_, NTY = NTY_;          // along axis 1, and thread rows
  static constexpr int TZ = 32 * VX, TY = NTY * PY, NT = 32 * NTY;
  static constexpr int H = TY + 2 * MP, W = TZ + 2 * MP, PS = H * W;  // staged plane
  static constexpr int NCOL = (W + 31) / 32;          // staged columns per lane
  static constexpr int NROW = (H + NTY - 1) / NTY;    // staged rows per thread row
};
constexpr int GEN_BLK_MAXMP = 3;  // radii with a register-blocked instance

// One coefficient as the inner loop reads it (one shared-memory load): its
// value and the byte offset of its neighbour from the output cell, for one
// ring position of the output plane.
template <typename S>
struct alignas(2 * sizeof(S)) GenTab {
  S coef;
  int off;
};

// Dynamic shared memory of general_block_kernel with `depth` planes loaded
// ahead: the ring of 2mp + 1 + depth planes, then a table of ncoef entries
// per ring position of the output plane.
inline size_t general_block_smem(int mp, size_t es, int tz, int ty, int ncoef, int depth = 1) {
  const int np = 2 * mp + 1 + depth;
  const size_t ring = (size_t)np * (ty + 2 * mp) * (tz + 2 * mp) * es;
  const size_t tab = (size_t)np * ncoef * (es >= 8 ? 16 : 8);
  return (ring + 15) / 16 * 16 + tab;
}

template <typename T, int MODE, int MP, int PY_ = GenBlk<T, MP>::PY, int NTY_ = GenBlk<T, MP>::NTY>
__global__ void __launch_bounds__(GenBlk<T, MP, PY_, NTY_>::NT, 2)
    general_block_kernel(const StencilArgs a, const GeneralCoefs k) {
  using G = GenBlk<T, MP, PY_, NTY_>;
  using S = typename EltTraits<T>::S;
  constexpr int VX = G::VX, PY = G::PY, NTY = G::NTY, W = G::W, H = G::H, PS = G::PS;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* ring = reinterpret_cast<T*>(smem_raw);
  __shared__ double red[32];

  const int ncoef = k.ncoef, D = a.gdepth, NP = 2 * MP + 1 + D;
  GenTab<S>* tab = reinterpret_cast<GenTab<S>*>(smem_raw + ((size_t)NP * PS * sizeof(T) + 15) / 16 * 16);
  const int b = blockIdx.z / a.nchunk, chunk = blockIdx.z - b * a.nchunk;
  if (a.active && !a.active[b]) return;
  const int x0 = blockIdx.x * G::TZ, y0 = blockIdx.y * G::TY;
  const int n0 = a.vout.n[0];
  const int z0 = chunk * a.zchunk;
  const int z1 = min(n0, z0 + a.zchunk);
  const T* in = static_cast<const T*>(a.in) + (int64_t)b * a.vin.sb;
  const int tx = threadIdx.x, ty = threadIdx.y, tid = tx + 32 * ty;
  const Boundary& bc = a.bc;
  // tab[cs * ncoef + c]: coefficient c with plane o in ring slot cs
  for (int e = tid; e < NP * ncoef; e += G::NT) {
    const int cs = e / ncoef, c = e - cs * ncoef;
    int sl = cs + k.off[c][0];
    sl = sl < 0 ? sl + NP : (sl >= NP ? sl - NP : sl);
    tab[e].coef = (S)k.coef[c];
    tab[e].off = ((sl - cs) * PS + k.off[c][1] * W + k.off[c][2]) * (int)sizeof(T);
  }
  // this thread's staged cells (rows ty + NTY q, columns tx + 32 m): source
  // offsets within a plane and periodic-image sides, computed once
  int64_t roff[G::NROW];
  int jx[G::NCOL];
  unsigned rowok = 0, colok = 0, fixmask = 0;  // fixmask bit q * NCOL + m: an in-plane periodic image
  signed char sy[G::NROW], sx[G::NCOL];
#pragma unroll
  for (int m = 0; m < G::NCOL; ++m) {
    const int c = tx + 32 * m;
    int s = -1;
    if (c < W && wrap_axis(x0 - MP + c, a.vin.n[2], bc.periodic[2], jx[m], s)) colok |= 1u << m;
    sx[m] = (signed char)s;
  }
#pragma unroll
  for (int q = 0; q < G::NROW; ++q) {
    const int r = ty + NTY * q;
    int j1 = 0, s = -1;
    if (r < H && wrap_axis(y0 - MP + r, a.vin.n[1], bc.periodic[1], j1, s)) rowok |= 1u << q;
    roff[q] = (int64_t)j1 * a.vin.s1;
    sy[q] = (signed char)s;
#pragma unroll
    for (int m = 0; m < G::NCOL; ++m)
      if (((rowok >> q) & (colok >> m) & 1u) && (s >= 0 || sx[m] >= 0)) fixmask |= 1u << (q * G::NCOL + m);
  }
  double sumsq = 0.0;
  __syncthreads();

  if (z0 < z1) {
    // plane p into its ring slot
    auto load = [&](int p) {
      int j0, s0;
      const bool ok0 = wrap_axis(p, a.vin.n[0], bc.periodic[0], j0, s0);
      T* slot = ring + ((p - z0 + MP) % NP) * PS;
      const T* base = in + (int64_t)j0 * a.vin.s0;
#pragma unroll
      for (int q = 0; q < G::NROW; ++q) {
        const int r = ty + NTY * q;
#pragma unroll
        for (int m = 0; m < G::NCOL; ++m) {
          const int c = tx + 32 * m;
          if (r < H && c < W) {
            const bool ok = ok0 && ((rowok >> q) & (colok >> m) & 1u);
            cp_async<sizeof(T)>(slot + r * W + c, ok ? base + roff[q] + jx[m] : in, ok);
          }
        }
      }
    };
    // Bloch phases of this thread's periodic-image cells of plane p, axis by
    // axis as the reference's chained halo copies apply them
    auto fix = [&](int p) {
      if constexpr (EltTraits<T>::cpx) {
        int j0, s0;
        if (!wrap_axis(p, a.vin.n[0], bc.periodic[0], j0, s0)) return;
        if (s0 < 0 && !fixmask) return;
        T* slot = ring + ((p - z0 + MP) % NP) * PS;
#pragma unroll
        for (int q = 0; q < G::NROW; ++q) {
#pragma unroll
          for (int m = 0; m < G::NCOL; ++m) {
            const int r = ty + NTY * q, c = tx + 32 * m;
            if (!((rowok >> q) & (colok >> m) & 1u)) continue;
            if (s0 < 0 && !((fixmask >> (q * G::NCOL + m)) & 1u)) continue;
            T val = slot[r * W + c];
            if (s0 >= 0) val = phase_mul(bc.ph[0][s0], val);
            if (sy[q] >= 0) val = phase_mul(bc.ph[1][sy[q]], val);
            if (sx[m] >= 0) val = phase_mul(bc.ph[2][sx[m]], val);
            slot[r * W + c] = val;
          }
        }
      }
    };
    // one commit group for the first 2mp + 1 planes, then one per plane: at
    // output plane o the groups of planes o + mp + 1 .. o + mp + D may still
    // be in flight
    for (int p = z0 - MP; p <= z0 + MP; ++p) load(p);
    cp_async_commit();
    for (int d = 1; d < D; ++d) {
      if (z0 + d < z1) load(z0 + MP + d);
      cp_async_commit();
    }
    // this thread's first output cell within slot 0
    const unsigned char* cen = reinterpret_cast<const unsigned char*>(ring + (ty + MP) * W + tx + MP);
    // its outputs (rows NTY apart, columns 32 apart): inside the grid, and
    // their element offsets less the plane's (the potential's drops the batch's)
    const int64_t ob = (int64_t)b * a.vout.sb;
    int64_t obase[PY][VX], rbase[PY][VX];
    unsigned omask = 0;
#pragma unroll
    for (int i = 0; i < PY; ++i)
#pragma unroll
      for (int j = 0; j < VX; ++j) {
        const int y = y0 + ty + NTY * i, x = x0 + tx + 32 * j;
        if (y < a.vout.n[1] && x < a.vout.n[2]) omask |= 1u << (i * VX + j);
        obase[i][j] = ob + (int64_t)y * a.vout.s1 + x;
        rbase[i][j] = (int64_t)b * a.vrho.sb + (int64_t)y * a.vrho.s1 + x;
      }
    for (int o = z0; o < z1; ++o) {
      if (o + D < z1) load(o + MP + D);
      cp_async_commit();
      switch (D) {
        case 1: cp_async_wait<1>(); break;
        case 2: cp_async_wait<2>(); break;
        case 3: cp_async_wait<3>(); break;
        default: cp_async_wait<4>(); break;
      }
      if (bc.use_phase) {
        if (o == z0) {
          for (int p = z0 - MP; p <= z0 + MP; ++p) fix(p);
        } else {
          fix(o + MP);
        }
      }
      __syncthreads();
      const int cs = (o - z0 + MP) % NP;  // slot of plane o
      const GenTab<S>* tc = tab + cs * ncoef;
      const unsigned char* co = cen + cs * PS * (int)sizeof(T);
      T acc[PY][VX];
#pragma unroll
      for (int i = 0; i < PY; ++i)
#pragma unroll
        for (int j = 0; j < VX; ++j) acc[i][j] = zero<T>();
#pragma unroll 4
      for (int c = (MODE == MODE_JACOBI) ? 1 : 0; c < ncoef; ++c) {
        const GenTab<S> e = tc[c];
        const T* src = reinterpret_cast<const T*>(co + e.off);
#pragma unroll
        for (int i = 0; i < PY; ++i)
#pragma unroll
          for (int j = 0; j < VX; ++j) acc[i][j] = mac_rn(e.coef, src[i * NTY * W + 32 * j], acc[i][j]);
      }
      const T* cp = reinterpret_cast<const T*>(co);  // plane o's centre cells
      const int64_t oz = (int64_t)o * a.vout.s0, rz = (int64_t)o * a.vrho.s0;
#pragma unroll
      for (int i = 0; i < PY; ++i) {
#pragma unroll
        for (int j = 0; j < VX; ++j) {
          if (!((omask >> (i * VX + j)) & 1u)) continue;
          T r = acc[i][j];
          const T cur = cp[i * NTY * W + 32 * j];
          const int64_t oi = obase[i][j] + oz;
          if constexpr (MODE == MODE_APPLY) {
            if (a.pot) {
              const S pv = static_cast<const S*>(a.pot)[oi - ob];
              r = fmac(pv, cur, r);
            }
            if (a.aux) r = fmac((S)a.aux_scale, static_cast<const T*>(a.aux)[oi], r);
            static_cast<T*>(a.out)[oi] = r;
          } else {
            const T rho = static_cast<const T*>(a.rho)[rbase[i][j] + rz];
            if constexpr (MODE == MODE_RESIDUAL) {
              const T d = sub(r, rho);
              if (a.out) static_cast<T*>(a.out)[oi] = d;
              sumsq += norm2(d);
            } else {
              // (1 - w) * b + w * (src - x) / c0   (c/bmgs/relax.c:62)
              if constexpr (EltTraits<T>::cpx) {
                static_cast<T*>(a.out)[oi] = cur;  // relax is real-only (asserted on host)
              } else {
                const S w = (S)a.w, c0 = (S)a.c0;
                static_cast<T*>(a.out)[oi] = jacobi_rn(w, cur, rho, r, c0);
              }
            }
          }
        }
      }
      __syncthreads();
    }
  }
  if constexpr (MODE == MODE_RESIDUAL) {
    if (!a.gsum.partial) return;  // residual without its norm
    double tot = block_sum(sumsq, red);
    const int blk = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * chunk);
    grid_sum_finish(a.gsum, b, blk, a.nblk_seg, tot, red);
  }
}

// ------------------------------------------------------------------ Mehrstellen A
// The O(h^4) Mehrstellen Laplacian A (gpaw/fd_operators.py LaplaceA: 19
// points, the centre, the 6 faces and the 12 edges of [-1, 1]^3, in that
// table order) on real grids, with the general kernel's arithmetic (each
// output sums its coefficients in table order with unfused multiply and add:
// bit-identical to c/bmgs/fd.c) but with the offsets known at compile time:
// each thread computes 2 x 2 adjacent outputs and holds the row segments they
// share in registers, 10 shared-memory values per output instead of 19.
// MEHR_OFF is the table order the launcher checks the operator against.
constexpr int MEHR_NC = 19;
constexpr signed char MEHR_OFF[MEHR_NC][3] = {
    {0, 0, 0},   {-1, 0, 0},  {1, 0, 0},   {0, -1, 0},  {0, 1, 0},  {0, 0, -1}, {0, 0, 1},
    {0, -1, -1}, {0, -1, 1},  {0, 1, -1},  {0, 1, 1},   {-1, 0, -1}, {-1, 0, 1}, {1, 0, -1},
    {1, 0, 1},   {-1, -1, 0}, {-1, 1, 0},  {1, -1, 0},  {1, 1, 0}};
struct MehrCfg {
  static constexpr int NTX = 32, NTY = 8;  // threads; each 2 (axis 2) x 2 (axis 1) outputs
  static constexpr int TZ = 2 * NTX, TY = 2 * NTY, NT = NTX * NTY;
  static constexpr int H = TY + 2, W = TZ + 2, PS = H * W;
  static constexpr int NCOL = (W + NT - 1) / NT;
};

template <typename T, int MODE>
__global__ void __launch_bounds__(MehrCfg::NT, 2) mehrstellen_kernel(const StencilArgs a, const GeneralCoefs k) {
  static_assert(!EltTraits<T>::cpx, "real grids");
  using C = MehrCfg;
  constexpr int W = C::W, H = C::H, PS = C::PS;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* ring = reinterpret_cast<T*>(smem_raw);
  __shared__ double red[32];
  const int D = a.gdepth, NP = 3 + D;
  const int b = blockIdx.z / a.nchunk, chunk = blockIdx.z - b * a.nchunk;
  if (a.active && !a.active[b]) return;
  const int x0 = blockIdx.x * C::TZ, y0 = blockIdx.y * C::TY;
  const int n0 = a.vout.n[0];
  const int z0 = chunk * a.zchunk;
  const int z1 = min(n0, z0 + a.zchunk);
  const T* in = static_cast<const T*>(a.in) + (int64_t)b * a.vin.sb;
  const int tx = threadIdx.x, ty = threadIdx.y;
  const Boundary& bc = a.bc;
  double sumsq = 0.0;
  // this thread's staged cells: rows ty + NTY q, columns tx + 32 m (W = 66:
  // three column slots, the third for two lanes)
  constexpr int NROW = (H + C::NTY - 1) / C::NTY, NCOLS = (W + 31) / 32;
  int64_t roff[NROW];
  int jx[NCOLS];
  unsigned rowok = 0, colok = 0;
#pragma unroll
  for (int m = 0; m < NCOLS; ++m) {
    const int c = tx + 32 * m;
    int s;
    if (c < W && wrap_axis(x0 - 1 + c, a.vin.n[2], bc.periodic[2], jx[m], s)) colok |= 1u << m;
  }
#pragma unroll
  for (int q = 0; q < NROW; ++q) {
    const int r = ty + C::NTY * q;
    int j1 = 0, s;
    if (r < H && wrap_axis(y0 - 1 + r, a.vin.n[1], bc.periodic[1], j1, s)) rowok |= 1u << q;
    roff[q] = (int64_t)j1 * a.vin.s1;
  }
  // outputs (rows y0 + 2 ty + i, columns x0 + 2 tx + j): inside the grid, offsets
  int64_t obase[2][2], rbase[2][2];
  unsigned omask = 0;
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      const int y = y0 + 2 * ty + i, x = x0 + 2 * tx + j;
      if (y < a.vout.n[1] && x < a.vout.n[2]) omask |= 1u << (2 * i + j);
      obase[i][j] = (int64_t)b * a.vout.sb + (int64_t)y * a.vout.s1 + x;
      rbase[i][j] = (int64_t)b * a.vrho.sb + (int64_t)y * a.vrho.s1 + x;
    }
  // the coefficients, in table order
  T cf[MEHR_NC];
#pragma unroll
  for (int c = 0; c < MEHR_NC; ++c) cf[c] = (T)k.coef[c];

  if (z0 < z1) {
    auto load = [&](int p) {
      int j0, s0;
      const bool ok0 = wrap_axis(p, a.vin.n[0], bc.periodic[0], j0, s0);
      T* slot = ring + ((p - z0 + 1) % NP) * PS;
      const T* base = in + (int64_t)j0 * a.vin.s0;
#pragma unroll
      for (int q = 0; q < NROW; ++q) {
        const int r = ty + C::NTY * q;
#pragma unroll
        for (int m = 0; m < NCOLS; ++m) {
          const int c = tx + 32 * m;
          if (r < H && c < W) {
            const bool ok = ok0 && ((rowok >> q) & (colok >> m) & 1u);
            cp_async<sizeof(T)>(slot + r * W + c, ok ? base + roff[q] + jx[m] : in, ok);
          }
        }
      }
    };
    for (int p = z0 - 1; p <= z0 + 1; ++p) load(p);
    cp_async_commit();
    for (int d = 1; d < D; ++d) {
      if (z0 + d < z1) load(z0 + 1 + d);
      cp_async_commit();
    }
    // this thread's first output cell (row 2 ty + 1, column 2 tx + 1 of a slot)
    const int cell = (2 * ty + 1) * W + 2 * tx + 1;
    for (int o = z0; o < z1; ++o) {
      if (o + D < z1) load(o + 1 + D);
      cp_async_commit();
      switch (D) {
        case 1: cp_async_wait<1>(); break;
        case 2: cp_async_wait<2>(); break;
        case 3: cp_async_wait<3>(); break;
        default: cp_async_wait<4>(); break;
      }
      __syncthreads();
      const int cs = (o - z0 + 1) % NP;
      const T* pm = ring + ((cs + NP - 1) % NP) * PS + cell;  // plane o - 1
      const T* pc = ring + cs * PS + cell;                    // plane o
      const T* pp = ring + ((cs + 1) % NP) * PS + cell;       // plane o + 1
      // row segments: columns -1 .. 2 around the first output column;
      // plane o: rows -1 .. 2; planes o -+ 1: rows 0, 1 (and rows -1, 2 at
      // the output columns only)
      T c0[4][4], cm[2][4], cp[2][4], cmr[2][2], cpr[2][2];
#pragma unroll
      for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int e = 0; e < 4; ++e) c0[r][e] = pc[(r - 1) * W + e - 1];
#pragma unroll
      for (int r = 0; r < 2; ++r)
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          cm[r][e] = pm[r * W + e - 1];
          cp[r][e] = pp[r * W + e - 1];
        }
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        cmr[0][e] = pm[-W + e];
        cmr[1][e] = pm[2 * W + e];
        cpr[0][e] = pp[-W + e];
        cpr[1][e] = pp[2 * W + e];
      }
#pragma unroll
      for (int i = 0; i < 2; ++i) {
#pragma unroll
        for (int j = 0; j < 2; ++j) {
          // the value of coefficient c at output (i, j), table order
          const T v[MEHR_NC] = {c0[i + 1][j + 1],
                                cm[i][j + 1],     cp[i][j + 1],
                                c0[i][j + 1],     c0[i + 2][j + 1],
                                c0[i + 1][j],     c0[i + 1][j + 2],
                                c0[i][j],         c0[i][j + 2],     c0[i + 2][j],     c0[i + 2][j + 2],
                                cm[i][j],         cm[i][j + 2],     cp[i][j],         cp[i][j + 2],
                                i == 0 ? cmr[0][j] : cm[0][j + 1], i == 0 ? cm[1][j + 1] : cmr[1][j],
                                i == 0 ? cpr[0][j] : cp[0][j + 1], i == 0 ? cp[1][j + 1] : cpr[1][j]};
          T acc = T(0);
#pragma unroll
          for (int c = (MODE == MODE_JACOBI) ? 1 : 0; c < MEHR_NC; ++c) acc = mac_rn(cf[c], v[c], acc);
          if (!((omask >> (2 * i + j)) & 1u)) continue;
          const T cur = v[0];
          const int64_t oi = obase[i][j] + (int64_t)o * a.vout.s0;
          if constexpr (MODE == MODE_APPLY) {
            using S = typename EltTraits<T>::S;
            if (a.pot) acc = fmac(static_cast<const S*>(a.pot)[oi - (int64_t)b * a.vout.sb], cur, acc);
            if (a.aux) acc = fmac((S)a.aux_scale, static_cast<const T*>(a.aux)[oi], acc);
            static_cast<T*>(a.out)[oi] = acc;
          } else {
            const T rho = static_cast<const T*>(a.rho)[rbase[i][j] + (int64_t)o * a.vrho.s0];
            if constexpr (MODE == MODE_RESIDUAL) {
              const T d = acc - rho;
              if (a.out) static_cast<T*>(a.out)[oi] = d;
              sumsq += norm2(d);
            } else {
              // (1 - w) * b + w * (src - x) / c0   (c/bmgs/relax.c:62)
              const T w = (T)a.w, cc = (T)a.c0;
              static_cast<T*>(a.out)[oi] = jacobi_rn(w, cur, rho, acc, cc);
            }
          }
        }
      }
      __syncthreads();
    }
  }
  if constexpr (MODE == MODE_RESIDUAL) {
    if (!a.gsum.partial) return;  // residual without its norm
    double tot = block_sum(sumsq, red);
    const int blk = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * chunk);
    grid_sum_finish(a.gsum, b, blk, a.nblk_seg, tot, red);
  }
}

// ------------------------------------------------------------------ star
// Tile TZ (axis 2) x TY (axis 1); PY consecutive axis-1 rows per thread.
#ifndef GPW_STAR_TY
#define GPW_STAR_TY 32
#endif
#ifndef GPW_STAR_PY
#define GPW_STAR_PY 4
#endif
#ifndef GPW_STAR_NS
#define GPW_STAR_NS 3
#endif
// 16-byte elements (complex128) take half-height tiles: two CTAs of 256
// threads per SM (star_stencil_kernel_2cta) instead of one of 512, so one
// CTA's plane barrier overlaps the other's work.
template <int R, typename T>
struct StarCfg {
  static constexpr int TZ = 32;
  static constexpr int PY = (sizeof(T) >= 16) ? (GPW_STAR_PY > 2 ? 2 : GPW_STAR_PY) : GPW_STAR_PY;
  static constexpr int TY = (sizeof(T) >= 16) ? GPW_STAR_TY / 2 : GPW_STAR_TY;
  static constexpr int NTY = TY / PY;
  static constexpr int NT = TZ * NTY;
  static constexpr int H = TY + 2 * R, W = TZ + 2 * R, PS = H * W;
  static constexpr int NLD = (PS + NT - 1) / NT;  // plane cells loaded per thread
  static constexpr int NSTAGE = GPW_STAR_NS;
};

struct StarCoefs {
  double cx[13], cy[13], cz[13];  // per-axis coefficients indexed offset + R (centres zero)
  double cc;                      // total centre (diagonal) coefficient
};

// The same coefficients in the kernel's scalar type, rounded once on the host
// (the rounding a per-use conversion makes): a float32 / complex64 kernel
// then holds no float64 constants to convert inside its plane loop.
template <typename S>
struct StarCoefsT {
  S cx[13], cy[13], cz[13];
  S cc;
};
template <typename S>
inline StarCoefsT<S> star_coefs_typed(const StarCoefs& sc) {
  StarCoefsT<S> t{};
  for (int i = 0; i < 13; ++i) {
    t.cx[i] = (S)sc.cx[i];
    t.cy[i] = (S)sc.cy[i];
    t.cz[i] = (S)sc.cz[i];
  }
  t.cc = (S)sc.cc;
  return t;
}

// Per-thread plane-load descriptors: the tile position in (axis 1, axis 2) is
// fixed for the CTA, so each cell's in-plane source offset, validity and
// wrap sides are computed once; a plane load is then one cp.async per cell.
template <typename T, int R>
struct StarLoader {
  using C = StarCfg<R, T>;
  int off[C::NLD];      // j1 * s1 + j2 (element offset inside a plane)
  unsigned valid = 0;   // bit k: cell k is inside the grid or a periodic image
  unsigned wrapped = 0; // bit k: cell k is a periodic image along axis 1 or 2
  unsigned char side[C::NLD];  // wrap sides: bits 0-1 axis 1 (+1), bits 2-3 axis 2 (+1)

  __device__ __forceinline__ void init(const GridView& v, const Boundary& bc, int y0, int x0) {
    const int tid = threadIdx.x + blockDim.x * threadIdx.y;
#pragma unroll
    for (int k = 0; k < C::NLD; ++k) {
      const int idx = tid + k * C::NT;
      const int r = idx / C::W, c = idx - r * C::W;
      int j1 = 0, j2 = 0, s1 = -1, s2 = -1;
      const bool ok = idx < C::PS && wrap_axis(y0 - R + r, v.n[1], bc.periodic[1], j1, s1) &&
                      wrap_axis(x0 - R + c, v.n[2], bc.periodic[2], j2, s2);
      off[k] = ok ? (int)((int64_t)j1 * v.s1 + j2) : 0;
      if (ok) valid |= 1u << k;
      if (ok && (s1 >= 0 || s2 >= 0)) wrapped |= 1u << k;
      side[k] = (unsigned char)((s1 + 1) | ((s2 + 1) << 2));
    }
  }

  __device__ __forceinline__ void load(T* slot, const T* in, const GridView& v, const Boundary& bc, int p) const {
    const int tid = threadIdx.x + blockDim.x * threadIdx.y;
    int j0, s0;
    const bool ok0 = wrap_axis(p, v.n[0], bc.periodic[0], j0, s0);
    const T* base = in + (int64_t)j0 * v.s0;
#pragma unroll
    for (int k = 0; k < C::NLD; ++k) {
      const int idx = tid + k * C::NT;
      if (C::PS % C::NT == 0 || idx < C::PS) {
        const bool ok = ok0 && ((valid >> k) & 1u);
        cp_async<sizeof(T)>(slot + idx, ok ? base + off[k] : in, ok);
      }
    }
  }

  // Bloch phases of the periodic images, axis by axis as the reference's
  // chained halo copies apply them (each thread fixes its own copies).
  __device__ __forceinline__ void fix(T* slot, const GridView& v, const Boundary& bc, int p) const {
    if constexpr (EltTraits<T>::cpx) {
      const int tid = threadIdx.x + blockDim.x * threadIdx.y;
      int j0, s0;
      if (!wrap_axis(p, v.n[0], bc.periodic[0], j0, s0)) return;
      // on a plane inside the grid only the in-plane periodic images change
      const unsigned todo = s0 < 0 ? wrapped : valid;
      if (!todo) return;
#pragma unroll
      for (int k = 0; k < C::NLD; ++k) {
        const int idx = tid + k * C::NT;
        if (idx >= C::PS || !((todo >> k) & 1u)) continue;
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

// EPI: an apply with a potential or aux term (a.pot / a.aux); the plain
// apply is compiled without their loads and branches.
template <typename T, int R, int MODE, bool EPI>
__device__ __forceinline__ void star_stencil_body(const StencilArgs& a, const StarCoefsT<typename EltTraits<T>::S>& k) {
  using C = StarCfg<R, T>;
  using S = typename EltTraits<T>::S;
  constexpr int PY = C::PY, W = C::W, PS = C::PS, NS = C::NSTAGE;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* ring = reinterpret_cast<T*>(smem_raw);
  __shared__ double red[32];

  const int b = blockIdx.z / a.nchunk, chunk = blockIdx.z - b * a.nchunk;
  if (a.active && !a.active[b]) return;
  const int x0 = blockIdx.x * C::TZ, y0 = blockIdx.y * C::TY;
  const int n0 = a.vout.n[0];
  const int z0 = chunk * a.zchunk;
  const int z1 = min(n0, z0 + a.zchunk);
  const T* in = static_cast<const T*>(a.in) + (int64_t)b * a.vin.sb;
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int x = x0 + tx;
  const int yb = ty * PY;  // first local row of this thread
  const bool xin = x < a.vout.n[2];
  double sumsq = 0.0;

  StarLoader<T, R> ld;
  ld.init(a.vin, a.bc, y0, x0);

  T acc[PY][2 * R + 1];
  T cur[PY][R + 1];  // JACOBI: centre values of the last R+1 planes
#pragma unroll
  for (int j = 0; j < PY; ++j) {
#pragma unroll
    for (int m = 0; m < 2 * R + 1; ++m) acc[j][m] = zero<T>();
#pragma unroll
    for (int m = 0; m < R + 1; ++m) cur[j][m] = zero<T>();
  }

  if (z0 < z1) {
    const int pfirst = z0 - R, plast = z1 - 1 + R;
    const int nsteps = plast - pfirst + 1;
#pragma unroll
    for (int st = 0; st < NS - 1; ++st) {
      if (st < nsteps) ld.load(ring + st * PS, in, a.vin, a.bc, pfirst + st);
      cp_async_commit();
    }
    for (int s = 0; s < nsteps; ++s) {
      const int p = pfirst + s;
      {
        const int sn = s + NS - 1;
        if (sn < nsteps) ld.load(ring + (sn % NS) * PS, in, a.vin, a.bc, pfirst + sn);
        cp_async_commit();
      }
      // prefetch rho for the output plane that completes at this step
      const int o = p - R;
      T rho[PY];
      if constexpr (MODE != MODE_APPLY) {
#pragma unroll
        for (int j = 0; j < PY; ++j) {
          const int y = y0 + yb + j;
          rho[j] = zero<T>();
          if (o >= z0 && xin && y < a.vout.n[1])
            rho[j] = static_cast<const T*>(a.rho)[(int64_t)b * a.vrho.sb + (int64_t)o * a.vrho.s0 +
                                                  (int64_t)y * a.vrho.s1 + x];
        }
      }
      cp_async_wait<NS - 1>();
      T* sl = ring + (s % NS) * PS;
      if (EltTraits<T>::cpx && a.bc.use_phase) ld.fix(sl, a.vin, a.bc, p);
      __syncthreads();

      // column of PY + 2R values along axis 1 at this thread's x
      T col[PY + 2 * R];
#pragma unroll
      for (int i = 0; i < PY + 2 * R; ++i) col[i] = sl[(yb + i) * W + tx + R];
#pragma unroll
      for (int j = 0; j < PY; ++j) {
        const T v = col[j + R];
        // in-plane part: centre + axis-1 + axis-2 neighbours (coefficients
        // are read from the kernel-parameter bank)
        T part = scale((MODE == MODE_JACOBI) ? S(0) : (S)k.cc, v);
#pragma unroll
        for (int q = 1; q <= R; ++q) {
          part = fmac((S)k.cy[R + q], col[j + R + q], part);
          part = fmac((S)k.cy[R - q], col[j + R - q], part);
        }
        const T* row = sl + (yb + j + R) * W + tx + R;
#pragma unroll
        for (int q = 1; q <= R; ++q) {
          part = fmac((S)k.cz[R + q], row[q], part);
          part = fmac((S)k.cz[R - q], row[-q], part);
        }
        if constexpr (MODE == MODE_APPLY && EPI) {
          // local potential of this (in-range) plane: its part is output p's
          const int y = y0 + yb + j;
          if (a.pot && p >= z0 && p < z1 && xin && y < a.vout.n[1])
            part = fmac(static_cast<const S*>(a.pot)[(int64_t)p * a.vout.s0 + (int64_t)y * a.vout.s1 + x], v, part);
        }
        // scatter along axis 0: output plane p-R+m receives offset R-m
#pragma unroll
        for (int m = 0; m < 2 * R + 1; ++m) {
          if (m == R)
            acc[j][m] = add(acc[j][m], part);
          else
            acc[j][m] = fmac((S)k.cx[2 * R - m], v, acc[j][m]);
        }
        if constexpr (MODE == MODE_JACOBI) {
#pragma unroll
          for (int m = 0; m < R; ++m) cur[j][m] = cur[j][m + 1];
          cur[j][R] = v;
        }
      }
      // output plane o = p - R is complete
      if (o >= z0) {
#pragma unroll
        for (int j = 0; j < PY; ++j) {
          const int y = y0 + yb + j;
          if (xin && y < a.vout.n[1]) {
            const int64_t oi = (int64_t)b * a.vout.sb + (int64_t)o * a.vout.s0 + (int64_t)y * a.vout.s1 + x;
            const T av = acc[j][0];
            if constexpr (MODE == MODE_APPLY) {
              static_cast<T*>(a.out)[oi] =
                  (EPI && a.aux) ? fmac((S)a.aux_scale, static_cast<const T*>(a.aux)[oi], av) : av;
            } else if constexpr (MODE == MODE_RESIDUAL) {
              const T r = sub(av, rho[j]);
              if (a.out) static_cast<T*>(a.out)[oi] = r;
              sumsq += norm2(r);
            } else {
              if constexpr (!EltTraits<T>::cpx) {
                const S w = (S)a.w;
                const S wc = w / (S)a.c0;
                static_cast<T*>(a.out)[oi] = (S(1) - w) * cur[j][0] + wc * (rho[j] - av);
              }
            }
          }
        }
      }
#pragma unroll
      for (int j = 0; j < PY; ++j) {
#pragma unroll
        for (int m = 0; m < 2 * R; ++m) acc[j][m] = acc[j][m + 1];
        acc[j][2 * R] = zero<T>();
      }
      __syncthreads();
    }
  }
  if constexpr (MODE == MODE_RESIDUAL) {
    if (!a.gsum.partial) return;  // residual without its norm
    double tot = block_sum(sumsq, red);
    const int blk = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * chunk);
    grid_sum_finish(a.gsum, b, blk, a.nblk_seg, tot, red);
  }
}

template <typename T, int R, int MODE, bool EPI = false>
__global__ void __launch_bounds__(StarCfg<R, T>::NT)
    star_stencil_kernel(const StencilArgs a, const StarCoefsT<typename EltTraits<T>::S> k) {
  star_stencil_body<T, R, MODE, EPI>(a, k);
}

// 16-byte elements: the same kernel with registers capped for two CTAs per SM
template <typename T, int R, int MODE, bool EPI = false>
__global__ void __launch_bounds__(StarCfg<R, T>::NT, 2)
    star_stencil_kernel_2cta(const StencilArgs a, const StarCoefsT<typename EltTraits<T>::S> k) {
  star_stencil_body<T, R, MODE, EPI>(a, k);
}

}  // namespace gpw
