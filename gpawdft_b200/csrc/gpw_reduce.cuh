// Deterministic block and grid reductions (warp shuffles + one partial per
// block, summed in block order by the last block to finish).
#pragma once
#include "gpw_common.cuh"

namespace gpw {

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// Sum `v` over the block; result valid in thread 0.  `red` holds >= 32 doubles.
__device__ __forceinline__ double block_sum(double v, double* red) {
  const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  const int nthr = blockDim.x * blockDim.y * blockDim.z;
  const int lane = tid & 31, wid = tid >> 5;
  v = warp_sum(v);
  __syncthreads();
  if (lane == 0) red[wid] = v;
  __syncthreads();
  double s = 0.0;
  if (tid < 32) {
    s = (tid < (nthr + 31) / 32) ? red[tid] : 0.0;
    s = warp_sum(s);
  }
  return s;
}

// Grid-level deterministic sum.  Each block calls with its block sum in thread
// 0; partial[] has one slot per block of the grid (row `seg` of a segmented
// reduction uses slots [seg*nblk_seg, (seg+1)*nblk_seg)).  The last block of
// the segment (ticket counter) adds the partials in block order and writes
// *result, then re-arms the counter.  Safe for repeated launches / graph replay.
struct GridSum {
  double* partial;       // [nseg * nblk_seg]
  unsigned* counter;     // [nseg], zero-initialised once
  double* result;        // [nseg]
};

__device__ __forceinline__ void grid_sum_finish(const GridSum& gs, int seg, int blk_in_seg,
                                                int nblk_seg, double block_total, double* red) {
  __shared__ unsigned s_last;
  const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  if (tid == 0) {
    gs.partial[(int64_t)seg * nblk_seg + blk_in_seg] = block_total;
    __threadfence();
    unsigned t = atomicAdd(&gs.counter[seg], 1u);
    s_last = (t == (unsigned)nblk_seg - 1u);
  }
  __syncthreads();
  if (s_last) {
    __threadfence();
    const int nthr = blockDim.x * blockDim.y * blockDim.z;
    // fixed-order strided sums per thread, then a fixed-shape tree
    double s = 0.0;
    const double* p = gs.partial + (int64_t)seg * nblk_seg;
    for (int i = tid; i < nblk_seg; i += nthr) s += __ldcg(p + i);
    s = block_sum(s, red);
    if (tid == 0) {
      gs.result[seg] = s;
      gs.counter[seg] = 0u;
      __threadfence();
    }
  }
}

}  // namespace gpw
