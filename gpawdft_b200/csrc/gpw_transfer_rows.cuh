// Restriction of grids whose fine rows (axis 2) fit in shared memory whole:
// the band transformers of the eigensolver (complex Bloch data, K = 2..8;
// c/transformers.c:54-123 with the halo of c/bc.c:138-250 and the three 1D
// passes of c/bmgs/restrict.c:37-57,137-154).
//
// Compared with restrict_kernel (gpw_transfer.cuh), which stages a 2D tile
// with its halo on both in-plane axes:
//  * a CTA owns TY coarse rows across the whole of axis 2 and marches along
//    axis 0; per fine plane ONE 4D TMA box brings the 2 TY + 2K - 3 fine
//    rows it needs, taken from column -L with the padded row pitch as the
//    box's row length, so the tensor map's zero fill supplies the empty halo
//    columns, the zero boundary of a zero axis and rows / planes out of
//    range; only rows that wrap along a periodic axis 1 (edge tiles) take
//    one bulk copy each into a wrap area (every copy request costs the SM
//    ~80 cycles, so a request per row -- 25 a plane -- was the bottleneck);
//  * Bloch phases, periodic halo columns and wrapped rows are written into
//    the stage of the next plane while the current one is computed
//    (normally the 2L halo values of each row: one value a thread), so the
//    passes themselves hold no branch;
//  * the axis-2 pass is an unrolled window: an item is one row and MO
//    adjacent outputs, which read the MO centre columns and the MO + K - 1
//    odd-offset columns between them once each; consecutive lanes take
//    consecutive rows, and the row pitch is 16 bytes past a multiple of 128,
//    so a warp's loads meet no bank conflict (complex128);
//  * the axis-1 pass of plane p - 1 runs in the same step as the axis-2 pass
//    of plane p (two axis-2 buffers), so a plane costs one CTA barrier;
//  * the axis-0 pass keeps the last 2K - 1 axis-1 results of its output in
//    registers, as restrict_kernel does.
// Every 1D pass evaluates the reference's expression in the reference's
// order without fused multiply-add, and a wrapped value takes the Bloch
// phases of its axes in the order 0, 1, 2 (the reference's chained halo
// copies), so results are bit-identical to restrict_kernel and to the
// reference C.  Every mbarrier wait is bounded (GPW_ETIMEDOUT in the status
// word).
#pragma once
#include "gpw_star_tma.cuh"
#include "gpw_transfer.cuh"

namespace gpw {

struct RowRestrictArgs {
  TransferArgs t;
  int ty;           // coarse rows (axis 1) per CTA
  int h;            // fine rows staged per plane: 2 ty + 2K - 3 (<= 32)
  int L;            // halo columns on each side of a staged row (>= K - 1; L x element a multiple of 16 bytes)
  int pitch;        // stage row pitch = the tensor box's row length, elements (>= n2 + 2 L)
  int pitchz;       // axis-2 pass row pitch, elements
  int nseg;         // axis-2 items per row: ceil(nout2 / MO)
  int stage_elems;  // h * pitch, rounded to 128 bytes
  int wrap_elems;   // per stage: the rows of a tile wrapped along a periodic axis 1, n2 each (rounded to 128 bytes)
  int* status;
};

constexpr int RR_NS = 3;  // ring stages: two planes in flight while one is read

// Bulk copy of `bytes` (a multiple of 16; both addresses 16-byte aligned)
// from global memory into this CTA's shared memory, completing on `bar`.
__device__ __forceinline__ void bulk_load(unsigned dst, const void* src, unsigned bytes, unsigned bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                   dst),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}

template <int NT>
struct RowRestrictCfg {
  static constexpr int MO = NT >= 384 ? 4 : 6;  // axis-2 outputs per item
};

// Axis-0 restriction over a ring of the last 2K - 1 axis-1 results whose
// newest entry is q[NEW]: the centre is K - 1 entries back; the sums run in
// restrict_1d's order.  Compile-time indices keep the ring in registers.
template <int K, int NEW, typename T>
__device__ __forceinline__ T restrict_ring(const T (&q)[2 * K - 1]) {
  using S = typename EltTraits<T>::S;
  constexpr int NQ = 2 * K - 1;
  constexpr int C = (NEW - (K - 1) + NQ) % NQ;
  if constexpr (K == 2) {
    return rmul(S(0.5), radd(q[C], rmul(S(0.5), radd(q[(C + 1) % NQ], q[(C + NQ - 1) % NQ]))));
  } else {
    T s = q[C];
#pragma unroll
    for (int j = 0; j < K / 2; ++j)
      s = radd(s, rmul((S)TW<K>::w(j), radd(q[(C + 2 * j + 1) % NQ], q[(C + NQ - 2 * j - 1) % NQ])));
    return rmul(S(0.5), s);
  }
}

// Write v into ring slot k (runtime) and, when `emit`, return the output it
// completes; one case per slot.
template <int K, int I = 0, typename T>
__device__ __forceinline__ T ring_push(T (&q)[2 * K - 1], int k, const T& v, bool emit) {
  if constexpr (I == 2 * K - 1) {
    return v;
  } else {
    if (k == I) {
      q[I] = v;
      return emit ? restrict_ring<K, I>(q) : v;
    }
    return ring_push<K, I + 1>(q, k, v, emit);
  }
}

// Stage layout: the tensor box of a plane, h rows of `pitch` elements taken
// from fine column -L on: L halo columns (out of range, zero-filled; on a
// periodic axis 2 the fix-up writes the row's last L values there), the n2
// values of the row, then zeros again -- the first L of them the right-hand
// halo (the row's first L values on a periodic axis).  Fine column c of the
// grid is stage column c + L.  Rows out of range along axis 1 arrive as
// zeros; on a periodic axis 1 the fix-up fills them from the wrap area,
// which per-row bulk copies fill with the rows they wrap to.
template <typename T, int K, int NT>
__global__ void __launch_bounds__(NT, NT >= 384 ? 1 : 2)
    restrict_rows_kernel(const __grid_constant__ CUtensorMap tmap, const RowRestrictArgs ra) {
  using S = typename EltTraits<T>::S;
  constexpr int NS = RR_NS, NQ = 2 * K - 1, KH = K / 2, MO = RowRestrictCfg<NT>::MO;
  constexpr int CPX = EltTraits<T>::cpx ? 2 : 1;  // tensor-map scalars per element
  const TransferArgs& a = ra.t;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* ring = reinterpret_cast<T*>(smem_raw + ((128u - (smem_u32(smem_raw) & 127u)) & 127u));
  T* wrap = ring + NS * ra.stage_elems;  // NS areas of wrap_elems
  T* zb = wrap + NS * ra.wrap_elems;     // two buffers of h rows x pitchz
  uint64_t* full = reinterpret_cast<uint64_t*>(zb + 2 * ra.h * ra.pitchz);
  int* frows = reinterpret_cast<int*>(full + NS);  // wrapped rows (stage row index), in order
  int* nfix = frows + 32;

  const int b = blockIdx.z / a.nchunk, chunk = blockIdx.z - b * a.nchunk;
  if (a.active && !a.active[b]) return;
  const int I0 = chunk * a.zchunk, I1 = min(a.vout.n[0], I0 + a.zchunk);
  if (I0 >= I1) return;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int n0 = a.vin.n[0], n1 = a.vin.n[1], n2 = a.vin.n[2];
  const int nout2 = a.vout.n[2];
  const int h = ra.h, pitch = ra.pitch, pitchz = ra.pitchz, L = ra.L;
  const Boundary& bc = a.bc;
  const bool per2 = bc.periodic[2] != 0;
  const bool cpx_phase = EltTraits<T>::cpx && bc.use_phase;
  const int Y0 = blockIdx.y * ra.ty;
  // fine plane of step 0 (the first tap of output I0) and the step count
  const int pfirst = 2 * I0 - a.pad0[0];
  const int nsteps = 2 * (I1 - I0 - 1) + NQ;
  const int yfirst = 2 * Y0 - a.pad0[1];  // fine row of stage row 0
  const T* in = static_cast<const T*>(a.in) + (int64_t)b * a.vin.sb;
  bool timed_out = false;

  // warp 0, lane r: stage row r; wrapped rows (periodic axis 1) also come
  // through the wrap area, in the order of frows
  int rj = 0, rs1 = -1;
  bool rin = false;
  if (warp == 0 && lane < h) rin = wrap_axis(yfirst + lane, n1, bc.periodic[1], rj, rs1);
  const bool rwrapped = rin && rs1 >= 0;
  int widx = 0;
  if (tid == 0) {
    for (int i = 0; i < NS; ++i) mbar_init(mbar_u32(&full[i]), 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  if (warp == 0) {
    const unsigned m = __ballot_sync(0xffffffffu, rwrapped);
    widx = __popc(m & ((1u << lane) - 1u));
    if (rwrapped) frows[widx] = lane;
    if (lane == 0) *nfix = __popc(m);
  }
  __syncthreads();
  const int nwrap = *nfix;

  const unsigned rowbytes = (unsigned)(n2 * sizeof(T));
  const unsigned boxbytes = (unsigned)(h * pitch * sizeof(T));
  // this thread's first halo value of a periodic axis 2 (stage offsets)
  int hsrc = -1, hdst = 0, hside = 0;
  if (per2 && tid < h * 2 * L) {
    const int r = tid / (2 * L), k = tid - r * (2 * L);
    int j1, s1;
    if (!(wrap_axis(yfirst + r, n1, bc.periodic[1], j1, s1) && s1 >= 0)) {
      hsrc = r * pitch + (k < L ? L + n2 - L + k : L + (k - L));
      hdst = r * pitch + (k < L ? k : L + n2 + (k - L));
      hside = k < L ? 1 : 0;
    }
  }
  // warp 0 streams the planes: lane 0 the tensor box, the lanes of wrapped
  // rows their bulk copies
  auto issue = [&](int i) {
    const int slot = i % NS;
    int j0, s0;
    const bool pok = wrap_axis(pfirst + i, n0, bc.periodic[0], j0, s0);
    const unsigned bar = mbar_u32(&full[slot]);
    if (lane == 0) {
      mbar_expect_tx(bar, boxbytes + (pok ? (unsigned)nwrap * rowbytes : 0u));
      // a zero plane: an out-of-range plane coordinate (all zeros)
      tma_load_4d(smem_u32(ring + slot * ra.stage_elems), &tmap, -L * CPX, yfirst, pok ? j0 : pfirst + i, b, bar);
    }
    if (pok && rwrapped)
      bulk_load(smem_u32(wrap + slot * ra.wrap_elems + widx * n2), in + (int64_t)j0 * a.vin.s0 + (int64_t)rj * a.vin.s1,
                rowbytes, bar);
  };
  // Wait for plane i, then complete its stage: wrapped rows from the wrap
  // area, halo columns of a periodic axis 2 from the row's ends, and the
  // Bloch phases of the wrapped axes (0, then 1, then 2, the reference's
  // chained halo order).
  auto land = [&](int i) {
    const int slot = i % NS;
    if (!mbar_wait_bounded(mbar_u32(&full[slot]), (unsigned)((i / NS) & 1))) timed_out = true;
    int j0, s0;
    const bool pok = wrap_axis(pfirst + i, n0, bc.periodic[0], j0, s0);
    const bool ph0 = cpx_phase && pok && s0 >= 0;
    T* st = ring + slot * ra.stage_elems;
    // a value v at column c of row r, with every phase except axis 2's
    // applied: store it, and its halo copy on a periodic axis 2
    auto put = [&](T* row, int c, T v) {
      row[L + c] = v;
      if (per2) {
        if (c >= n2 - L) row[c - (n2 - L)] = cpx_phase ? phase_mul(bc.ph[2][1], v) : v;
        if (c < L) row[L + n2 + c] = cpx_phase ? phase_mul(bc.ph[2][0], v) : v;
      }
    };
    // wrapped rows
    if (nwrap > 0) {
      const T* wa = wrap + slot * ra.wrap_elems;
      for (int idx = tid; idx < nwrap * n2; idx += NT) {
        const int q = idx / n2, c = idx - q * n2;
        const int r = frows[q];
        int j1, s1;
        wrap_axis(yfirst + r, n1, 1, j1, s1);
        T v = pok ? wa[q * n2 + c] : zero<T>();
        if (ph0) v = phase_mul(bc.ph[0][s0], v);
        if (cpx_phase) v = phase_mul(bc.ph[1][s1], v);
        put(st + r * pitch, c, v);
      }
    }
    // the other rows: the axis-0 phase on every value of a wrapped plane,
    // else only the halo columns
    if (ph0) {
      for (int idx = tid; idx < h * n2; idx += NT) {
        const int r = idx / n2, c = idx - r * n2;
        int j1, s1;
        if (wrap_axis(yfirst + r, n1, bc.periodic[1], j1, s1) && s1 >= 0) continue;  // wrapped: done above
        T* row = st + r * pitch;
        put(row, c, phase_mul(bc.ph[0][s0], row[L + c]));
      }
    } else if (per2) {
      // this thread's first halo value is precomputed (hsrc < 0: none)
      if (hsrc >= 0) {
        const T v = st[hsrc];
        st[hdst] = cpx_phase ? phase_mul(bc.ph[2][hside], v) : v;
      }
      for (int idx = tid + NT; idx < h * 2 * L; idx += NT) {
        const int r = idx / (2 * L), k = idx - r * (2 * L);
        int j1, s1;
        if (wrap_axis(yfirst + r, n1, bc.periodic[1], j1, s1) && s1 >= 0) continue;  // wrapped: done above
        T* row = st + r * pitch;
        if (k < L) {
          const T v = row[L + n2 - L + k];
          row[k] = cpx_phase ? phase_mul(bc.ph[2][1], v) : v;
        } else {
          const T v = row[L + (k - L)];
          row[L + n2 + (k - L)] = cpx_phase ? phase_mul(bc.ph[2][0], v) : v;
        }
      }
    }
    // order these writes before the copies that refill the stage
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
  };
  if (warp == 0)
    for (int i = 0; i < NS && i < nsteps; ++i) issue(i);
  land(0);
  __syncthreads();

  // axis-1 / axis-0 item of this thread: coarse (Y, J)
  const int yitems = ra.ty * nout2;
  const int Yl = tid / nout2, J = tid - Yl * nout2;
  const bool yitem = tid < yitems;
  const bool ystore = yitem && Y0 + Yl < a.vout.n[1];
  T q[NQ];  // ring of the last NQ axis-1 results; the next goes to q[qk]
#pragma unroll
  for (int i = 0; i < NQ; ++i) q[i] = zero<T>();
  int qk = 0;
  // stage column of the first odd-offset tap of output 0
  const int cx0 = L + (K - 1 - a.pad0[2]) - (K - 1);
  const int xitems = h * ra.nseg;
  const int xr = tid % h, xJa = (tid / h) * MO;  // this thread's first axis-2 item

  for (int s = 0; s <= nsteps; ++s) {
    if (s < nsteps) {
      // ---- axis-2 pass of plane s into zb[s & 1]: item = row r, outputs
      // Ja .. Ja + MO - 1; odd-offset tap t of the item at rp[2 t], the
      // centre of output i at rp[2 i + K - 1]
      const T* stg = ring + (s % NS) * ra.stage_elems;
      T* zbuf = zb + (s & 1) * h * pitchz;
      for (int it = tid; it < xitems; it += NT) {
        int r = xr, Ja = xJa;
        if (it != tid) {
          const int seg = it / h;
          r = it - seg * h;
          Ja = seg * MO;
        }
        const int nJ = min(MO, nout2 - Ja);
        const T* rp = stg + r * pitch + cx0 + 2 * Ja;
        T* zrow = zbuf + r * pitchz + Ja;
        T w[MO + K - 1];
#pragma unroll
        for (int t = 0; t < MO + K - 1; ++t) w[t] = (t < nJ + K - 1) ? rp[2 * t] : zero<T>();
#pragma unroll
        for (int i = 0; i < MO; ++i) {
          if (i < nJ) {
            T sum = rp[2 * i + K - 1];
#pragma unroll
            for (int j = 0; j < KH; ++j)
              sum = radd(sum, rmul((S)TW<K>::w(j), radd(w[i + KH + j], w[i + KH - 1 - j])));
            zrow[i] = rmul(S(0.5), sum);
          }
        }
      }
    }
    if (s >= 1 && yitem) {
      // ---- axis-1 pass of plane s - 1, axis-0 queue, output
      const T* zbuf = zb + ((s - 1) & 1) * h * pitchz;
      const T v = restrict_1d<K>(zbuf + (K - 1 + 2 * Yl) * pitchz + J, pitchz);
      // step s - 1 completes output I0 + (s - 1 - (NQ - 1)) / 2 when even
      const int t = s - 1 - (NQ - 1);
      const bool emit = t >= 0 && (t & 1) == 0 && ystore;
      const T o = ring_push<K>(q, qk, v, emit);
      qk = qk + 1 == NQ ? 0 : qk + 1;
      if (emit) {
        const int I = I0 + (t >> 1);
        static_cast<T*>(a.out)[(int64_t)b * a.vout.sb + (int64_t)I * a.vout.s0 + (int64_t)(Y0 + Yl) * a.vout.s1 +
                               J] = o;
      }
    }
    if (s + 1 < nsteps) land(s + 1);
    __syncthreads();
    // the stage of plane s is free: refill it with plane s + NS
    if (warp == 0 && s < nsteps && s + NS < nsteps) issue(s + NS);
  }
  if (timed_out && ra.status) atomicExch(ra.status, GPW_ETIMEDOUT);
}

}  // namespace gpw
