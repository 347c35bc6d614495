// Kernels of the learned warm start: a small 3D convolutional U-Net that
// maps a (normalised) density to an initial potential for the multigrid
// solver.  No counterpart in the reference.
//
// Activations are bf16 in NDHWC layout ([batch][d][h][w][c], channels
// contiguous); weights bf16 [27 taps][cout][cin] (tap = (kd*3 + kh)*3 + kw)
// with fp32 master copies; every contraction accumulates in fp32.
//
// conv3_kernel<CIN, COUT_CTA, EPI>: 3x3x3, stride 1, zero padding 1, as an
// implicit GEMM on the tensor cores (mma.sync m16n8k16 bf16 -> fp32).  A CTA
// owns a 16 (w) x 8 (h) x 2 (d) block of 256 output points and COUT_CTA
// output channels; the input block with its one-point halo (18 x 10 x 4
// points x CIN) and the CTA's weights for all 27 taps sit in shared memory
// (rows padded by 8 bf16 so ldmatrix rows fall in distinct banks).  Each of
// the 8 warps computes 2 rows of 16 points: per tap and 16-channel slice it
// loads the A fragments (points x cin) with ldmatrix from the tap-shifted
// rows of the input block -- no im2col buffer -- and the B fragments
// (cin x cout) from the weight block.  The data-gradient of a convolution is
// the same kernel on the output gradient with spatially flipped, transposed
// weights (nn_flip_weights).
//
// conv3_wgrad_kernel<CIN, COUT, TG>: dW[tap][co][ci] = sum_p dz[p][co]
// in[p + tap][ci] for a group of TG taps, each CTA reducing a contiguous
// range of 256-point blocks into registers (A = dz^T and B = shifted input
// via ldmatrix.trans), then one fp32 partial per CTA; nn_wgrad_reduce sums
// the partials in a fixed order (deterministic).
#pragma once
#include <cuda_bf16.h>
#include <stdint.h>

namespace gpw {
namespace nn {

constexpr int TW = 16, TH = 8, TD = 2;                  // output block (w, h, d)
constexpr int BW = TW + 2, BH = TH + 2, BD = TD + 2;    // input block with halo
constexpr int BPTS = BW * BH * BD;                      // 720 input points
constexpr int OPTS = TW * TH * TD;                      // 256 output points
constexpr int NWARP = 8;

enum Epilogue {
  EPI_LINEAR = 0,     // out = acc (+ bias)
  EPI_GELU = 1,       // z = acc + bias (stored if z != null), out = gelu(z)
};

struct ConvArgs {
  const __nv_bfloat16* x;   // input [B][D][H][W][CIN]
  const __nv_bfloat16* w;   // weights [27][COUT][CIN]
  const float* bias;        // [COUT] or null
  __nv_bfloat16* z;         // pre-activation out (EPI_GELU, optional)
  __nv_bfloat16* out;       // [B][D][H][W][COUT]
  const __nv_bfloat16* add; // optional tensor added to the result before the epilogue ([..][COUT])
  int B, D, H, W;
  int cout;                 // total output channels (COUT_CTA x gridDim.y)
};

__device__ __forceinline__ unsigned s_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void ldsm_x4(unsigned addr, unsigned& r0, unsigned& r1, unsigned& r2, unsigned& r3) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0, %1, %2, %3}, [%4];\n"
               : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
               : "r"(addr));
}
__device__ __forceinline__ void ldsm_x2(unsigned addr, unsigned& r0, unsigned& r1) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x2.shared.b16 {%0, %1}, [%2];\n" : "=r"(r0), "=r"(r1) : "r"(addr));
}
__device__ __forceinline__ void ldsm_x4_t(unsigned addr, unsigned& r0, unsigned& r1, unsigned& r2, unsigned& r3) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0, %1, %2, %3}, [%4];\n"
               : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
               : "r"(addr));
}
__device__ __forceinline__ void ldsm_x2_t(unsigned addr, unsigned& r0, unsigned& r1) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x2.trans.shared.b16 {%0, %1}, [%2];\n"
               : "=r"(r0), "=r"(r1)
               : "r"(addr));
}
__device__ __forceinline__ void mma_bf16(float (&c)[4], unsigned a0, unsigned a1, unsigned a2, unsigned a3,
                                         unsigned b0, unsigned b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
      "{%0, %1, %2, %3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// GELU(x) = x Phi(x) (the erf form)
__device__ __forceinline__ float gelu(float x) { return 0.5f * x * (1.0f + erff(x * 0.70710678118654752f)); }
// GELU'(x) = Phi(x) + x phi(x)
__device__ __forceinline__ float gelu_grad(float x) {
  return 0.5f * (1.0f + erff(x * 0.70710678118654752f)) + x * 0.39894228040143268f * expf(-0.5f * x * x);
}

// Copy the input block (with zero halo) of output block (bd, bh, bw) of batch
// member b into shared memory rows of CINP = CIN + 8 bf16.
template <int CIN>
__device__ __forceinline__ void load_block(__nv_bfloat16* sx, const __nv_bfloat16* x, int b, int d0, int h0, int w0,
                                           int D, int H, int W) {
  constexpr int CINP = CIN + 8;
  constexpr int V = CIN / 8;  // 16-byte vectors per point
  for (int i = threadIdx.x; i < BPTS * V; i += blockDim.x) {
    const int pt = i / V, v = i - pt * V;
    const int bw = pt % BW, t = pt / BW, bh = t % BH, bd = t / BH;
    const int d = d0 + bd - 1, h = h0 + bh - 1, w = w0 + bw - 1;
    uint4 val = make_uint4(0u, 0u, 0u, 0u);
    if (d >= 0 && d < D && h >= 0 && h < H && w >= 0 && w < W)
      val = *reinterpret_cast<const uint4*>(x + ((((int64_t)b * D + d) * H + h) * W + w) * CIN + v * 8);
    *reinterpret_cast<uint4*>(sx + pt * CINP + v * 8) = val;
  }
}

template <int CIN, int COUT_CTA, int EPI>
__global__ void __launch_bounds__(NWARP * 32, 1) conv3_kernel(const ConvArgs a) {
  constexpr int CINP = CIN + 8;
  constexpr int NT = COUT_CTA / 8;  // n8 tiles
  extern __shared__ __align__(16) unsigned char smem[];
  __nv_bfloat16* sx = reinterpret_cast<__nv_bfloat16*>(smem);
  __nv_bfloat16* sw = sx + BPTS * CINP;  // [27][COUT_CTA][CINP]
  const int nbw = (a.W + TW - 1) / TW, nbh = (a.H + TH - 1) / TH, nbd = (a.D + TD - 1) / TD;
  int blk = blockIdx.x;
  const int ibw = blk % nbw;
  blk /= nbw;
  const int ibh = blk % nbh;
  blk /= nbh;
  const int ibd = blk % nbd;
  const int b = blk / nbd;
  const int w0 = ibw * TW, h0 = ibh * TH, d0 = ibd * TD;
  const int co0 = blockIdx.y * COUT_CTA;

  load_block<CIN>(sx, a.x, b, d0, h0, w0, a.D, a.H, a.W);
  {
    constexpr int V = CIN / 8;
    for (int i = threadIdx.x; i < 27 * COUT_CTA * V; i += blockDim.x) {
      const int v = i % V, t = i / V, co = t % COUT_CTA, tap = t / COUT_CTA;
      *reinterpret_cast<uint4*>(sw + (tap * COUT_CTA + co) * CINP + v * 8) =
          *reinterpret_cast<const uint4*>(a.w + ((int64_t)tap * a.cout + co0 + co) * CIN + v * 8);
    }
  }
  __syncthreads();

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // this warp's 2 output rows: row r = (od, oh), 16 points along w each
  float acc[2][NT][4];
#pragma unroll
  for (int m = 0; m < 2; ++m)
#pragma unroll
    for (int n = 0; n < NT; ++n)
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[m][n][q] = 0.f;

  // ldmatrix row of this lane: matrix mi = lane / 8 (A: rows 0-7 / 8-15 x
  // k 0-7 / 8-15), row lane % 8
  const int mi = lane >> 3, mr = lane & 7;
  const int a_pt = mr + 8 * (mi & 1), a_k = 8 * (mi >> 1);
  // B (x2 per n8 tile): lanes 0-7 rows co, k 0-7; lanes 8-15 k 8-15
  const int b_row = lane & 7, b_k = 8 * ((lane >> 3) & 1);
#pragma unroll 1
  for (int tap = 0; tap < 27; ++tap) {
    const int kd = tap / 9, kh = (tap / 3) % 3, kw = tap % 3;
#pragma unroll
    for (int kc = 0; kc < CIN / 16; ++kc) {
      unsigned af[2][4];
#pragma unroll
      for (int m = 0; m < 2; ++m) {
        const int row = 2 * warp + m;  // 0..15 = od * TH + oh
        const int od = row / TH, oh = row % TH;
        const int pt = ((od + kd) * BH + (oh + kh)) * BW + (a_pt + kw);
        ldsm_x4(s_u32(sx + pt * CINP + kc * 16 + a_k), af[m][0], af[m][1], af[m][2], af[m][3]);
      }
#pragma unroll
      for (int n = 0; n < NT; ++n) {
        unsigned b0, b1;
        ldsm_x2(s_u32(sw + (tap * COUT_CTA + n * 8 + b_row) * CINP + kc * 16 + b_k), b0, b1);
#pragma unroll
        for (int m = 0; m < 2; ++m) mma_bf16(acc[m][n], af[m][0], af[m][1], af[m][2], af[m][3], b0, b1);
      }
    }
  }

  // epilogue: C fragment rows g / g+8 (points), cols 2t, 2t+1 (channels)
  const int g = lane >> 2, t4 = lane & 3;
#pragma unroll
  for (int m = 0; m < 2; ++m) {
    const int row = 2 * warp + m;
    const int od = row / TH, oh = row % TH;
    const int d = d0 + od, h = h0 + oh;
    if (d >= a.D || h >= a.H) continue;
#pragma unroll
    for (int half = 0; half < 2; ++half) {
      const int w = w0 + g + 8 * half;
      if (w >= a.W) continue;
      const int64_t base = ((((int64_t)b * a.D + d) * a.H + h) * a.W + w) * a.cout;
#pragma unroll
      for (int n = 0; n < NT; ++n) {
        const int co = co0 + n * 8 + 2 * t4;
        float v0 = acc[m][n][2 * half], v1 = acc[m][n][2 * half + 1];
        if (a.bias) {
          v0 += a.bias[co];
          v1 += a.bias[co + 1];
        }
        if (a.add) {
          const __nv_bfloat162 ad = *reinterpret_cast<const __nv_bfloat162*>(a.add + base + co);
          v0 += __bfloat162float(ad.x);
          v1 += __bfloat162float(ad.y);
        }
        if constexpr (EPI == EPI_GELU) {
          if (a.z) *reinterpret_cast<__nv_bfloat162*>(a.z + base + co) = __floats2bfloat162_rn(v0, v1);
          v0 = gelu(v0);
          v1 = gelu(v1);
        }
        *reinterpret_cast<__nv_bfloat162*>(a.out + base + co) = __floats2bfloat162_rn(v0, v1);
      }
    }
  }
}

template <int CIN, int COUT_CTA>
constexpr size_t conv3_smem() {
  return (size_t)(BPTS * (CIN + 8) + 27 * COUT_CTA * (CIN + 8)) * 2;
}

// ---------------------------------------------------------------- weight gradient
struct WgradArgs {
  const __nv_bfloat16* x;   // layer input [B][D][H][W][CIN]
  const __nv_bfloat16* dz;  // gradient of the pre-activation [B][D][H][W][COUT]
  float* partial;           // [gridDim.x][27][COUT][CIN]
  int B, D, H, W;
  int nblocks;              // 256-point output blocks in the batch
};

// One CTA: taps [tg*TG, tg*TG + TG) (blockIdx.y = tg), blocks
// [blockIdx.x * nb / gridDim.x, ...).  Warp tiles: (m16 co) x (n8 ci).
template <int CIN, int COUT, int TG>
__global__ void __launch_bounds__(NWARP * 32, 1) conv3_wgrad_kernel(const WgradArgs a) {
  constexpr int CINP = CIN + 8, COUTP = COUT + 8;
  constexpr int MT = COUT / 16, NTL = CIN / 8;         // m16 / n8 tiles per tap
  constexpr int TILES = TG * MT * NTL;                  // per CTA
  constexpr int TPW = (TILES + NWARP - 1) / NWARP;      // tiles per warp
  extern __shared__ __align__(16) unsigned char smem[];
  __nv_bfloat16* sx = reinterpret_cast<__nv_bfloat16*>(smem);
  __nv_bfloat16* sdz = sx + BPTS * CINP;  // [256][COUTP]
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int tg0 = blockIdx.y * TG;
  float acc[TPW][4];
#pragma unroll
  for (int i = 0; i < TPW; ++i)
#pragma unroll
    for (int q = 0; q < 4; ++q) acc[i][q] = 0.f;
  const int nbw = (a.W + TW - 1) / TW, nbh = (a.H + TH - 1) / TH, nbd = (a.D + TD - 1) / TD;
  const int kb0 = (int)((int64_t)blockIdx.x * a.nblocks / gridDim.x);
  const int kb1 = (int)((int64_t)(blockIdx.x + 1) * a.nblocks / gridDim.x);
  // ldmatrix.trans lanes: matrix mi = lane / 8, row lane % 8
  const int mi = lane >> 3, mr = lane & 7;
  for (int kb = kb0; kb < kb1; ++kb) {
    int blk = kb;
    const int ibw = blk % nbw;
    blk /= nbw;
    const int ibh = blk % nbh;
    blk /= nbh;
    const int ibd = blk % nbd;
    const int b = blk / nbd;
    const int w0 = ibw * TW, h0 = ibh * TH, d0 = ibd * TD;
    __syncthreads();  // previous block's tiles fully consumed
    load_block<CIN>(sx, a.x, b, d0, h0, w0, a.D, a.H, a.W);
    {
      constexpr int V = COUT / 8;
      for (int i = threadIdx.x; i < OPTS * V; i += blockDim.x) {
        const int p = i / V, v = i - p * V;
        const int ow = p % TW, t = p / TW, oh = t % TH, od = t / TH;
        const int d = d0 + od, h = h0 + oh, w = w0 + ow;
        uint4 val = make_uint4(0u, 0u, 0u, 0u);
        if (d < a.D && h < a.H && w < a.W)
          val = *reinterpret_cast<const uint4*>(a.dz + ((((int64_t)b * a.D + d) * a.H + h) * a.W + w) * COUT + v * 8);
        *reinterpret_cast<uint4*>(sdz + p * COUTP + v * 8) = val;
      }
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < TPW; ++i) {
      const int tile = warp + NWARP * i;
      if (tile >= TILES) break;
      const int nt = tile % NTL, t2 = tile / NTL, mt = t2 % MT, tl = t2 / MT;
      const int tap = tg0 + tl;
      if (tap >= 27) continue;
      const int kd = tap / 9, kh = (tap / 3) % 3, kw = tap % 3;
      // K = the 256 points of the block, 16 at a time (one output row of 16 w)
#pragma unroll 2
      for (int ks = 0; ks < OPTS / 16; ++ks) {
        const int od = ks / TH, oh = ks % TH;
        // A = dz^T (co x p): smem rows p, cols co; x4.trans matrices
        // (p 0-7, co 0-7), (p 0-7, co 8-15), (p 8-15, co 0-7), (p 8-15, co 8-15)
        const int ap = ks * 16 + mr + 8 * (mi >> 1);
        const int ac = mt * 16 + 8 * (mi & 1);
        unsigned a0, a1, a2, a3;
        ldsm_x4_t(s_u32(sdz + ap * COUTP + ac), a0, a1, a2, a3);
        // B = shifted input (p x ci): rows p, cols ci; x2.trans matrices
        // (p 0-7, ci 0-7), (p 8-15, ci 0-7)
        const int bp = mr + 8 * (mi & 1);
        const int spt = ((od + kd) * BH + (oh + kh)) * BW + (bp + kw);
        unsigned b0, b1;
        ldsm_x2_t(s_u32(sx + spt * CINP + nt * 8), b0, b1);
        mma_bf16(acc[i], a0, a1, a2, a3, b0, b1);
      }
    }
  }
  // write the CTA's partial: C rows g / g+8 (co), cols 2t, 2t+1 (ci)
  const int g = lane >> 2, t4 = lane & 3;
  float* part = a.partial + (int64_t)blockIdx.x * 27 * COUT * CIN;
#pragma unroll
  for (int i = 0; i < TPW; ++i) {
    const int tile = warp + NWARP * i;
    if (tile >= TILES) break;
    const int nt = tile % NTL, t2 = tile / NTL, mt = t2 % MT, tl = t2 / MT;
    const int tap = tg0 + tl;
    if (tap >= 27) continue;
    const int co = mt * 16 + g, ci = nt * 8 + 2 * t4;
    float* p = part + ((int64_t)tap * COUT + co) * CIN + ci;
    p[0] = acc[i][0];
    p[1] = acc[i][1];
    p[8 * CIN] = acc[i][2];
    p[8 * CIN + 1] = acc[i][3];
  }
}

template <int CIN, int COUT>
constexpr size_t wgrad_smem() {
  return (size_t)(BPTS * (CIN + 8) + OPTS * (COUT + 8)) * 2;
}

}  // namespace nn
}  // namespace gpw
