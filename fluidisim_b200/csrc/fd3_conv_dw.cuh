// The weight gradient of a 3x3x3 convolution of the learned preconditioner, all 27 taps per CTA.
//
// gW[tap][co][ci] += sum over cells of gOut[cell][co] * In[cell + tap][ci] (zero outside the sample).
// A CTA takes blocks of BY rows (y) of one z-layer, all X cells of each row, in turn (a persistent
// grid).  For each 16-channel chunk of the input it stages, per block:
//   - the input's halo block (rows z-1..z+1, y0-1..y0+BY) in the flat layout of k_conv_tc,
//     f = (zz (BY+2) + yy)(X+1) + xx, one zero pad cell ending every row, zero rows outside the
//     sample, one 16-channel row of 48 bytes per cell (32 bytes of data, padded against bank
//     conflicts);
//   - the block's output gradient, one row of COUT channels per flat output position, zero at the
//     pad positions.
// Every tap is then the staged input seen from another start row: position m of the block meets
// input row m0 + m + dz (BY+2)(X+1) + dy (X+1) + dx.  The products are mma.sync m16n8k16 (BF16 in,
// FP32 accumulate) with M = output channels, N = 8 input channels, K = 16 positions, the operands
// read transposed from the staged rows by ldmatrix.  Warp w keeps the tiles of taps w, w + 8, ...
// in registers across every block of the chunk and adds them to gW with one atomic per element at
// the end of the chunk.  The arithmetic is the GEMM of k_conv_dw; only the order of the sum over
// cells differs.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "fd3_unet.cuh"

namespace fd3u {

constexpr int DW2_THREADS = 256;
constexpr int DW2_LEAD = 8;   // zero rows before the block (the lowest tap reads row -1)
constexpr int DW2_TAIL = 32;  // zero rows after it (the last K step's positions past the block)
constexpr int DW2_IS = 24;    // bf16 per staged input row (16 channels + 8 of padding)

__host__ __device__ inline int dw2_rows(int X, int Y) {
  int by = 520 / (X + 1);
  if (by < 1) by = 1;
  return by < Y ? by : Y;
}
__host__ __device__ inline int dw2_positions(int X, int BY) { return (BY * (X + 1) + 15) / 16 * 16; }
__host__ __device__ inline int dw2_in_rows(int X, int BY) { return DW2_LEAD + 3 * (BY + 2) * (X + 1) + DW2_TAIL; }
__host__ __device__ inline size_t dw2_smem_bytes(int X, int BY, int cout) {
  return (size_t)dw2_in_rows(X, BY) * DW2_IS * 2 + (size_t)dw2_positions(X, BY) * (cout + 8) * 2;
}

template <int CIN, int COUT>
__global__ void __launch_bounds__(DW2_THREADS, 1) k_conv_dw2(Dims d, int BY, const __nv_bfloat16* __restrict__ in,
                                                            const __nv_bfloat16* __restrict__ gout,
                                                            float* __restrict__ gw) {
  static_assert(CIN % 16 == 0 && (COUT == 16 || COUT == 32), "channel padding");
  constexpr int GS = COUT + 8;           // bf16 per staged gradient row
  constexpr int MT = COUT / 16;          // m16 tiles of output channels
  constexpr int TPW = 4;                 // taps per warp (27 taps over 8 warps)
  extern __shared__ __align__(16) unsigned char smem_dw[];
  const int X = d.X, Y = d.Y, Z = d.Z;
  const int PX = X + 1, PYX = (BY + 2) * PX;
  const int nrows_in = dw2_in_rows(X, BY), npos = dw2_positions(X, BY);
  __nv_bfloat16* sI = reinterpret_cast<__nv_bfloat16*>(smem_dw);
  __nv_bfloat16* sG = sI + (size_t)nrows_in * DW2_IS;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int yblocks = (Y + BY - 1) / BY;
  const long long nblk = (long long)d.B * Z * yblocks;
  const int m0 = PYX + PX;
  const uint4 zero4 = make_uint4(0, 0, 0, 0);

  // rows no block writes: the lead and tail rows and every row's pad cell
  for (int r = tid; r < DW2_LEAD + DW2_TAIL; r += DW2_THREADS) {
    const int q = r < DW2_LEAD ? r : DW2_LEAD + 3 * PYX + (r - DW2_LEAD);
    *reinterpret_cast<uint4*>(sI + q * DW2_IS) = zero4;
    *reinterpret_cast<uint4*>(sI + q * DW2_IS + 8) = zero4;
  }
  for (int r = tid; r < 3 * (BY + 2); r += DW2_THREADS) {
    const int q = DW2_LEAD + r * PX + X;
    *reinterpret_cast<uint4*>(sI + q * DW2_IS) = zero4;
    *reinterpret_cast<uint4*>(sI + q * DW2_IS + 8) = zero4;
  }

  int taps[TPW];
#pragma unroll
  for (int u = 0; u < TPW; ++u) taps[u] = warp + 8 * u;  // >= 27: no tap

  for (int ck = 0; ck < CIN / 16; ++ck) {
    float acc[TPW][MT][2][4];
#pragma unroll
    for (int u = 0; u < TPW; ++u)
#pragma unroll
      for (int mt = 0; mt < MT; ++mt)
#pragma unroll
        for (int nt = 0; nt < 2; ++nt)
#pragma unroll
          for (int e = 0; e < 4; ++e) acc[u][mt][nt][e] = 0.f;

    for (long long blk = blockIdx.x; blk < nblk; blk += gridDim.x) {
      const int yb = (int)(blk % yblocks);
      const int z = (int)((blk / yblocks) % Z);
      const long long b = blk / yblocks / Z;
      const int y0 = yb * BY;
      __syncthreads();  // the previous block's reads are done
      // input rows of the halo block: one warp per row, two 16-byte halves per cell
      for (int r = warp; r < 3 * (BY + 2); r += DW2_THREADS / 32) {
        const int zi = z - 1 + r / (BY + 2), yi = y0 - 1 + r % (BY + 2);
        __nv_bfloat16* dst = sI + (size_t)(DW2_LEAD + r * PX) * DW2_IS;
        if (zi < 0 || zi >= Z || yi < 0 || yi >= Y) {
          for (int e = lane; e < 2 * X; e += 32) *reinterpret_cast<uint4*>(dst + (e >> 1) * DW2_IS + (e & 1) * 8) = zero4;
          continue;
        }
        const __nv_bfloat16* src = in + (((b * Z + zi) * Y + yi) * (long long)X) * CIN + ck * 16;
        for (int e = lane; e < 2 * X; e += 32) {
          const int xx = e >> 1, h = e & 1;
          *reinterpret_cast<uint4*>(dst + xx * DW2_IS + h * 8) =
              *reinterpret_cast<const uint4*>(src + (long long)xx * CIN + h * 8);
        }
      }
      // output-gradient rows of the block's positions (zero at pad positions and past the block)
      for (int e = tid; e < npos * (COUT / 8); e += DW2_THREADS) {
        const int m = e / (COUT / 8), g8 = e % (COUT / 8);
        const int yl = m / PX, x = m % PX;
        uint4 v = zero4;
        if (x < X && yl < BY && y0 + yl < Y)
          v = *reinterpret_cast<const uint4*>(gout + ((((b * Z + z) * Y + y0 + yl) * (long long)X) + x) * COUT + g8 * 8);
        *reinterpret_cast<uint4*>(sG + m * GS + g8 * 8) = v;
      }
      __syncthreads();
      for (int ks = 0; ks < npos / 16; ++ks) {
        uint32_t a[MT][4];
#pragma unroll
        for (int mt = 0; mt < MT; ++mt) {
          const int j = lane >> 3, rr = lane & 7;
          ldsm_x4_trans(a[mt], sG + (ks * 16 + rr + 8 * (j >> 1)) * GS + mt * 16 + 8 * (j & 1));
        }
#pragma unroll
        for (int u = 0; u < TPW; ++u) {
          const int t = taps[u];
          if (t < 27) {
            const int off = (t / 9 - 1) * PYX + ((t / 3) % 3 - 1) * PX + (t % 3 - 1);
            const int row = DW2_LEAD + m0 + ks * 16 + (lane & 15) + off;
#pragma unroll
            for (int nt = 0; nt < 2; ++nt) {
              uint32_t b0, b1;
              ldsm_x2_trans(b0, b1, sI + (size_t)row * DW2_IS + nt * 8);
#pragma unroll
              for (int mt = 0; mt < MT; ++mt) mma_bf16(acc[u][mt][nt], a[mt], b0, b1);
            }
          }
        }
      }
    }
    // this CTA's share of gW for the chunk: tile (mt, nt) element e is co = 16 mt + g + 8 (e >> 1),
    // ci = 16 ck + 8 nt + 2 t4 + (e & 1)
    const int g = lane >> 2, t4 = lane & 3;
#pragma unroll
    for (int u = 0; u < TPW; ++u) {
      const int t = taps[u];
      if (t >= 27) continue;
      float* base = gw + (size_t)t * COUT * CIN;
#pragma unroll
      for (int mt = 0; mt < MT; ++mt)
#pragma unroll
        for (int nt = 0; nt < 2; ++nt) {
          const int co = mt * 16 + g, ci = ck * 16 + nt * 8 + 2 * t4;
          atomicAdd(base + (size_t)co * CIN + ci, acc[u][mt][nt][0]);
          atomicAdd(base + (size_t)co * CIN + ci + 1, acc[u][mt][nt][1]);
          atomicAdd(base + (size_t)(co + 8) * CIN + ci, acc[u][mt][nt][2]);
          atomicAdd(base + (size_t)(co + 8) * CIN + ci + 1, acc[u][mt][nt][3]);
        }
    }
  }
}

}  // namespace fd3u
