// Kernels of the learned preconditioner: a small 3-D U-Net (3 levels, 16/32/64 channels, 3x3x3
// convolutions), BF16 activations and weights with FP32 accumulation on the tensor cores.
//
// Tensors are channels-last, [sample][z][y][x][channel], channel counts padded to multiples of 16.
// A 3x3x3 convolution is an implicit GEMM: for each of the 27 taps, Out[cell][co] +=
// In[cell + tap][ci] * W[tap][co][ci], with zero padding at the sample's faces.  The forward kernel
// and the data-gradient kernel are the same GEMM (the data gradient uses the weights transposed
// and the taps mirrored); the weight gradient is a GEMM over cells, staged through shared memory.
// The tensor-core instruction is mma.sync m16n8k16 (bf16 in, f32 accumulate).
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace fd3u {

constexpr int CONV_THREADS = 256;          // 8 warps, 32 cells each
constexpr int CONV_CELLS = CONV_THREADS;   // cells per CTA
constexpr int DW_THREADS = 256;
constexpr int DW_ROWS = 128;               // cells staged per step of the weight-gradient GEMM

struct Dims {
  int B, Z, Y, X;  // samples and grid of this level
  __host__ __device__ long long cells() const { return (long long)B * Z * Y * X; }
};

__device__ __forceinline__ uint32_t ld32(const __nv_bfloat16* p) { return *reinterpret_cast<const uint32_t*>(p); }

__device__ __forceinline__ void mma_bf16(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// Neighbour of cell q (global index over the batch) at tap (dz, dy, dx); -1 outside the sample.
struct CellPos {
  long long q;
  int z, y, x;
  bool ok;
};
__device__ __forceinline__ CellPos cell_pos(const Dims& d, long long q) {
  CellPos c;
  c.q = q;
  c.ok = q < d.cells();
  long long t = c.ok ? q : 0;
  c.x = (int)(t % d.X); t /= d.X;
  c.y = (int)(t % d.Y); t /= d.Y;
  c.z = (int)(t % d.Z);
  return c;
}
__device__ __forceinline__ long long neighbour(const Dims& d, const CellPos& c, int dz, int dy, int dx) {
  if (!c.ok) return -1;
  const int z = c.z + dz, y = c.y + dy, x = c.x + dx;
  if (z < 0 || z >= d.Z || y < 0 || y >= d.Y || x < 0 || x >= d.X) return -1;
  return c.q + ((long long)dz * d.Y + dy) * d.X + dx;
}

// Epilogues of the convolution GEMM.
enum ConvEpi { EPI_BIAS_RELU = 0, EPI_PLAIN = 1, EPI_BIAS_F32_CH0 = 2 };

// Out[cell][0..COUT) = sum_tap In[cell + tap][0..CIN) . W[tap][co][0..CIN)  (+ bias, ReLU).
// Each warp owns 32 consecutive cells (two m16 tiles) and all COUT channels (COUT/8 n8 tiles).
template <int CIN, int COUT, int EPI>
__global__ void __launch_bounds__(CONV_THREADS) k_conv(Dims d, const __nv_bfloat16* __restrict__ in,
                                                       const __nv_bfloat16* __restrict__ w,
                                                       const float* __restrict__ bias,
                                                       __nv_bfloat16* __restrict__ out, float* __restrict__ out32) {
  static_assert(CIN % 16 == 0 && COUT % 8 == 0, "channel padding");
  constexpr int NT = COUT / 8;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g = lane >> 2, t = lane & 3;
  const long long base = (long long)blockIdx.x * CONV_CELLS + warp * 32;
  CellPos rows[4];
#pragma unroll
  for (int r = 0; r < 4; ++r) rows[r] = cell_pos(d, base + g + 8 * r);  // rows g, g+8 (tile 0), g+16, g+24 (tile 1)
  float acc[2][NT][4];
#pragma unroll
  for (int m = 0; m < 2; ++m)
#pragma unroll
    for (int n = 0; n < NT; ++n)
#pragma unroll
      for (int e = 0; e < 4; ++e) acc[m][n][e] = 0.f;

  for (int tap = 0; tap < 27; ++tap) {
    const int dz = tap / 9 - 1, dy = (tap / 3) % 3 - 1, dx = tap % 3 - 1;
    long long nb[4];
#pragma unroll
    for (int r = 0; r < 4; ++r) nb[r] = neighbour(d, rows[r], dz, dy, dx);
    const __nv_bfloat16* wt = w + (size_t)tap * COUT * CIN;
#pragma unroll
    for (int kc = 0; kc < CIN / 16; ++kc) {
      const int k0 = kc * 16 + 2 * t;
      uint32_t a[2][4];
#pragma unroll
      for (int m = 0; m < 2; ++m) {
        const long long r0 = nb[2 * m], r1 = nb[2 * m + 1];
        a[m][0] = r0 >= 0 ? ld32(in + r0 * CIN + k0) : 0u;
        a[m][1] = r1 >= 0 ? ld32(in + r1 * CIN + k0) : 0u;
        a[m][2] = r0 >= 0 ? ld32(in + r0 * CIN + k0 + 8) : 0u;
        a[m][3] = r1 >= 0 ? ld32(in + r1 * CIN + k0 + 8) : 0u;
      }
#pragma unroll
      for (int n = 0; n < NT; ++n) {
        const __nv_bfloat16* wr = wt + (size_t)(n * 8 + g) * CIN + k0;
        const uint32_t b0 = ld32(wr), b1 = ld32(wr + 8);
        mma_bf16(acc[0][n], a[0], b0, b1);
        mma_bf16(acc[1][n], a[1], b0, b1);
      }
    }
  }
  // accumulator (m, n, e): cell row g + 8*(e >> 1) + 16*m, channel n*8 + 2t + (e & 1)
#pragma unroll
  for (int m = 0; m < 2; ++m) {
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const CellPos& c = rows[2 * m + h];
      if (!c.ok) continue;
#pragma unroll
      for (int n = 0; n < NT; ++n) {
        const int co = n * 8 + 2 * t;
        float v0 = acc[m][n][2 * h], v1 = acc[m][n][2 * h + 1];
        if (EPI == EPI_BIAS_RELU) {
          v0 = fmaxf(v0 + bias[co], 0.f);
          v1 = fmaxf(v1 + bias[co + 1], 0.f);
        }
        if (EPI == EPI_BIAS_F32_CH0) {
          if (co == 0) out32[c.q] = v0 + bias[0];
        } else {
          __nv_bfloat162 p = __floats2bfloat162_rn(v0, v1);
          *reinterpret_cast<__nv_bfloat162*>(out + c.q * COUT + co) = p;
        }
      }
    }
  }
}

__device__ __forceinline__ void ldsm_x4_trans(uint32_t (&r)[4], const void* p) {
  const unsigned a = (unsigned)__cvta_generic_to_shared(p);
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];\n"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(a));
}
__device__ __forceinline__ void ldsm_x2_trans(uint32_t& r0, uint32_t& r1, const void* p) {
  const unsigned a = (unsigned)__cvta_generic_to_shared(p);
  asm volatile("ldmatrix.sync.aligned.m8n8.x2.trans.shared.b16 {%0,%1}, [%2];\n" : "=r"(r0), "=r"(r1) : "r"(a));
}

// Weight gradient of one tap: gW[tap][co][ci] += sum_cells gOut[cell][co] * In[cell + tap][ci],
// over the cells [chunk0, chunk1) of blockIdx.y's range.  M = COUT, N = CIN, K = cells: the two
// operands are staged DW_ROWS cells at a time in shared memory and read transposed by ldmatrix.
template <int CIN, int COUT>
__global__ void __launch_bounds__(DW_THREADS) k_conv_dw(Dims d, const __nv_bfloat16* __restrict__ in,
                                                        const __nv_bfloat16* __restrict__ gout,
                                                        float* __restrict__ gw, long long chunk) {
  static_assert(CIN % 16 == 0 && COUT % 16 == 0, "channel padding");
  constexpr int GS = COUT + 8, IS = CIN + 8;  // padded rows (16-byte aligned, fewer bank conflicts)
  constexpr int MT = COUT / 16, NTT = CIN / 8, TILES = MT * NTT;
  constexpr int TPW = (TILES + 7) / 8;  // tiles per warp
  __shared__ __align__(16) __nv_bfloat16 sG[DW_ROWS * GS];
  __shared__ __align__(16) __nv_bfloat16 sI[DW_ROWS * IS];
  __shared__ long long snb[DW_ROWS];  // the tap's neighbour of each staged row (-1: outside)
  const int tap = blockIdx.x;
  const int dz = tap / 9 - 1, dy = (tap / 3) % 3 - 1, dx = tap % 3 - 1;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const long long c0 = (long long)blockIdx.y * chunk;
  const long long c1 = c0 + chunk < d.cells() ? c0 + chunk : d.cells();
  float acc[TPW][4];
#pragma unroll
  for (int q = 0; q < TPW; ++q)
#pragma unroll
    for (int e = 0; e < 4; ++e) acc[q][e] = 0.f;

  for (long long s = c0; s < c1; s += DW_ROWS) {
    // the neighbour of each row once (one cell position per row, not per 16-byte piece)
    for (int r = threadIdx.x; r < DW_ROWS; r += DW_THREADS)
      snb[r] = s + r < c1 ? neighbour(d, cell_pos(d, s + r), dz, dy, dx) : -1;
    __syncthreads();
    // stage: 16-byte pieces (8 channels) of DW_ROWS rows
    for (int p = threadIdx.x; p < DW_ROWS * (COUT / 8); p += DW_THREADS) {
      const int r = p / (COUT / 8), k = p % (COUT / 8);
      const long long q = s + r;
      uint4 v = make_uint4(0, 0, 0, 0);
      if (q < c1) v = *reinterpret_cast<const uint4*>(gout + q * COUT + k * 8);
      *reinterpret_cast<uint4*>(sG + r * GS + k * 8) = v;
    }
    for (int p = threadIdx.x; p < DW_ROWS * (CIN / 8); p += DW_THREADS) {
      const int r = p / (CIN / 8), k = p % (CIN / 8);
      const long long q = s + r;
      uint4 v = make_uint4(0, 0, 0, 0);
      const long long nb = snb[r];
      if (q < c1 && nb >= 0) v = *reinterpret_cast<const uint4*>(in + nb * CIN + k * 8);
      *reinterpret_cast<uint4*>(sI + r * IS + k * 8) = v;
    }
    __syncthreads();
#pragma unroll
    for (int ks = 0; ks < DW_ROWS / 16; ++ks) {
#pragma unroll
      for (int q = 0; q < TPW; ++q) {
        const int tile = warp + 8 * q;
        if (tile < TILES) {
          const int mt = tile / NTT, nt = tile % NTT;
          uint32_t a[4];
          {
            const int j = lane >> 3, rr = lane & 7;
            ldsm_x4_trans(a, sG + (ks * 16 + rr + 8 * (j >> 1)) * GS + mt * 16 + 8 * (j & 1));
          }
          uint32_t b0, b1;
          {
            const int rr = lane & 15;
            ldsm_x2_trans(b0, b1, sI + (ks * 16 + rr) * IS + nt * 8);
          }
          mma_bf16(acc[q], a, b0, b1);
        }
      }
    }
    __syncthreads();
  }
  const int g = lane >> 2, t = lane & 3;
#pragma unroll
  for (int q = 0; q < TPW; ++q) {
    const int tile = warp + 8 * q;
    if (tile < TILES) {
      const int mt = tile / NTT, nt = tile % NTT;
      float* base = gw + (size_t)tap * COUT * CIN;
      const int co = mt * 16 + g, ci = nt * 8 + 2 * t;
      atomicAdd(base + (size_t)co * CIN + ci, acc[q][0]);
      atomicAdd(base + (size_t)co * CIN + ci + 1, acc[q][1]);
      atomicAdd(base + (size_t)(co + 8) * CIN + ci, acc[q][2]);
      atomicAdd(base + (size_t)(co + 8) * CIN + ci + 1, acc[q][3]);
    }
  }
}

// Bias gradient: gb[co] += sum over cells of gOut[cell][co].  blockIdx.y picks an 8-channel group;
// each thread sums the 16-byte group of its cells (grid-stride), then one atomic per warp and channel.
__global__ void k_bias_grad(long long cells, int C, const __nv_bfloat16* __restrict__ g, float* __restrict__ gb) {
  const int grp = blockIdx.y;
  float s[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < cells; q += (long long)gridDim.x * blockDim.x) {
    const uint4 v = *reinterpret_cast<const uint4*>(g + q * C + grp * 8);
    const __nv_bfloat162* h = reinterpret_cast<const __nv_bfloat162*>(&v);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const float2 t = __bfloat1622float2(h[k]);
      s[2 * k] += t.x;
      s[2 * k + 1] += t.y;
    }
  }
#pragma unroll
  for (int e = 0; e < 8; ++e) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s[e] += __shfl_down_sync(0xffffffffu, s[e], o);
  }
  if ((threadIdx.x & 31) == 0) {
#pragma unroll
    for (int e = 0; e < 8; ++e) atomicAdd(gb + grp * 8 + e, s[e]);
  }
}

// Mean of the 8 children: fine [B][2Z][2Y][2X][C] -> coarse [B][Z][Y][X][C] (d = coarse dims).
// One thread per (coarse cell, 8-channel group): 16-byte loads and stores, the children summed in
// f32 in the order e = 0..7.
__global__ void k_pool(Dims d, int C, const __nv_bfloat16* __restrict__ fine, __nv_bfloat16* __restrict__ coarse) {
  const int G = C / 8;
  const long long n = d.cells() * G;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
    const int g = (int)(q % G);
    long long c = q / G;
    const long long cell = c;
    const int x = (int)(c % d.X); c /= d.X;
    const int y = (int)(c % d.Y); c /= d.Y;
    const int z = (int)(c % d.Z);
    const long long b = c / d.Z;
    const int FX = 2 * d.X, FY = 2 * d.Y, FZ = 2 * d.Z;
    float s[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
#pragma unroll
    for (int e = 0; e < 8; ++e) {
      const long long f = ((b * FZ + 2 * z + (e >> 2)) * FY + 2 * y + ((e >> 1) & 1)) * FX + 2 * x + (e & 1);
      const uint4 v = *reinterpret_cast<const uint4*>(fine + f * C + g * 8);
      const __nv_bfloat162* h = reinterpret_cast<const __nv_bfloat162*>(&v);
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const float2 t = __bfloat1622float2(h[k]);
        s[2 * k] += t.x;
        s[2 * k + 1] += t.y;
      }
    }
    __align__(16) __nv_bfloat162 o[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) o[k] = __floats2bfloat162_rn(0.125f * s[2 * k], 0.125f * s[2 * k + 1]);
    *reinterpret_cast<uint4*>(coarse + cell * C + g * 8) = *reinterpret_cast<const uint4*>(o);
  }
}

// cat(up(coarse), skip): out[fine cell][0..C1) = coarse[parent][..], out[..][C1..C1+C2) = skip.
// One thread per (fine cell, 8-channel group of the C1 + C2 outputs): 16-byte copies.
__global__ void k_up_cat(Dims fd, int C1, int C2, const __nv_bfloat16* __restrict__ coarse,
                         const __nv_bfloat16* __restrict__ skip, __nv_bfloat16* __restrict__ out) {
  const int C = C1 + C2, G = C / 8, G1 = C1 / 8;
  const long long n = fd.cells() * G;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
    const int g = (int)(q % G);
    long long c = q / G;
    const long long cell = c;
    uint4 v;
    if (g >= G1) {
      v = *reinterpret_cast<const uint4*>(skip + cell * C2 + (g - G1) * 8);
    } else {
      const int x = (int)(c % fd.X); c /= fd.X;
      const int y = (int)(c % fd.Y); c /= fd.Y;
      const int z = (int)(c % fd.Z);
      const long long b = c / fd.Z;
      const long long p = ((b * (fd.Z / 2) + z / 2) * (fd.Y / 2) + y / 2) * (fd.X / 2) + x / 2;
      v = *reinterpret_cast<const uint4*>(coarse + p * C1 + g * 8);
    }
    *reinterpret_cast<uint4*>(out + cell * C + g * 8) = v;
  }
}

// Gradient through cat(up(.), skip) into the coarse part: gc[parent][ch] = sum over the 8
// children of g[child][ch] (ch < C1 of the C-wide gradient), times the ReLU mask of act.  One thread
// per (coarse cell, 8-channel group); the children are summed in f32 in the order e = 0..7.
__global__ void k_up_bwd(Dims cd, int C, int C1, const __nv_bfloat16* __restrict__ g,
                         const __nv_bfloat16* __restrict__ act, __nv_bfloat16* __restrict__ gc) {
  const int G1 = C1 / 8;
  const long long n = cd.cells() * G1;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
    const int grp = (int)(q % G1);
    long long c = q / G1;
    const long long cell = c;
    const int x = (int)(c % cd.X); c /= cd.X;
    const int y = (int)(c % cd.Y); c /= cd.Y;
    const int z = (int)(c % cd.Z);
    const long long b = c / cd.Z;
    const int FX = 2 * cd.X, FY = 2 * cd.Y, FZ = 2 * cd.Z;
    float s[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
#pragma unroll
    for (int e = 0; e < 8; ++e) {
      const long long f = ((b * FZ + 2 * z + (e >> 2)) * FY + 2 * y + ((e >> 1) & 1)) * FX + 2 * x + (e & 1);
      const uint4 v = *reinterpret_cast<const uint4*>(g + f * C + grp * 8);
      const __nv_bfloat162* h = reinterpret_cast<const __nv_bfloat162*>(&v);
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const float2 t = __bfloat1622float2(h[k]);
        s[2 * k] += t.x;
        s[2 * k + 1] += t.y;
      }
    }
    const uint4 av = *reinterpret_cast<const uint4*>(act + cell * C1 + grp * 8);
    const __nv_bfloat16* a = reinterpret_cast<const __nv_bfloat16*>(&av);
    __align__(16) __nv_bfloat16 o[8];
#pragma unroll
    for (int e = 0; e < 8; ++e) o[e] = __float2bfloat16(__bfloat162float(a[e]) > 0.f ? s[e] : 0.f);
    *reinterpret_cast<uint4*>(gc + cell * C1 + grp * 8) = *reinterpret_cast<const uint4*>(o);
  }
}

// Gradient of an encoder activation: (skip part of the concat gradient + pool backward of the next
// level's input gradient) times its ReLU mask.  g: [fine][C] slice at channel offset off of a
// Cg-wide tensor; gp: [coarse][C]; act, out: [fine][C].  One thread per (fine cell, 8-channel group).
__global__ void k_enc_grad(Dims fd, int C, const __nv_bfloat16* __restrict__ g, int Cg, int off,
                           const __nv_bfloat16* __restrict__ gp, const __nv_bfloat16* __restrict__ act,
                           __nv_bfloat16* __restrict__ out) {
  const int G = C / 8;
  const long long n = fd.cells() * G;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
    const int grp = (int)(q % G);
    long long c = q / G;
    const long long cell = c;
    const int x = (int)(c % fd.X); c /= fd.X;
    const int y = (int)(c % fd.Y); c /= fd.Y;
    const int z = (int)(c % fd.Z);
    const long long b = c / fd.Z;
    const long long p = ((b * (fd.Z / 2) + z / 2) * (fd.Y / 2) + y / 2) * (fd.X / 2) + x / 2;
    const uint4 gv = *reinterpret_cast<const uint4*>(g + cell * Cg + off + grp * 8);
    const uint4 pv = *reinterpret_cast<const uint4*>(gp + p * C + grp * 8);
    const uint4 av = *reinterpret_cast<const uint4*>(act + cell * C + grp * 8);
    const __nv_bfloat16* ge = reinterpret_cast<const __nv_bfloat16*>(&gv);
    const __nv_bfloat16* pe = reinterpret_cast<const __nv_bfloat16*>(&pv);
    const __nv_bfloat16* ae = reinterpret_cast<const __nv_bfloat16*>(&av);
    __align__(16) __nv_bfloat16 o[8];
#pragma unroll
    for (int e = 0; e < 8; ++e) {
      const float v = __bfloat162float(ge[e]) + 0.125f * __bfloat162float(pe[e]);
      o[e] = __float2bfloat16(__bfloat162float(ae[e]) > 0.f ? v : 0.f);
    }
    *reinterpret_cast<uint4*>(out + cell * C + grp * 8) = *reinterpret_cast<const uint4*>(o);
  }
}

// In-place ReLU mask: g *= (act > 0).
__global__ void k_relu_mask(long long n, __nv_bfloat16* __restrict__ g, const __nv_bfloat16* __restrict__ act) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
    if (!(__bfloat162float(act[q]) > 0.f)) g[q] = __float2bfloat16(0.f);
}

// The network input: [cell][16] with channels (x0 * s, x1, x2) and zeros, from [cell][3] f32.
__global__ void k_input(long long cells, const float* __restrict__ x, float s, __nv_bfloat16* __restrict__ out) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < cells; q += (long long)gridDim.x * blockDim.x) {
    __align__(16) __nv_bfloat16 v[16];
#pragma unroll
    for (int c = 0; c < 16; ++c) v[c] = __float2bfloat16(0.f);
    v[0] = __float2bfloat16(x[3 * q] * s);
    v[1] = __float2bfloat16(x[3 * q + 1]);
    v[2] = __float2bfloat16(x[3 * q + 2]);
    uint4* o = reinterpret_cast<uint4*>(out + q * 16);
    o[0] = reinterpret_cast<const uint4*>(v)[0];
    o[1] = reinterpret_cast<const uint4*>(v)[1];
  }
}

// The head's output gradient: [cell][16] with channel 0 = g * s, the rest 0.
__global__ void k_out_grad(long long cells, const float* __restrict__ g, float s, __nv_bfloat16* __restrict__ out) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < cells; q += (long long)gridDim.x * blockDim.x) {
    __align__(16) __nv_bfloat16 v[16];
#pragma unroll
    for (int c = 0; c < 16; ++c) v[c] = __float2bfloat16(0.f);
    v[0] = __float2bfloat16(g[q] * s);
    uint4* o = reinterpret_cast<uint4*>(out + q * 16);
    o[0] = reinterpret_cast<const uint4*>(v)[0];
    o[1] = reinterpret_cast<const uint4*>(v)[1];
  }
}

// Working copies of one layer's weights from the f32 master [27][cout][cin]: the forward layout
// W[tap][coutp][cinp] and the data-gradient layout Wt[tap][cinp][coutp] with the tap mirrored
// (tap' = 26 - tap), both zero-padded.
__global__ void k_pack(int cin, int cout, int cinp, int coutp, const float* __restrict__ master,
                       __nv_bfloat16* __restrict__ w, __nv_bfloat16* __restrict__ wt) {
  const int n = 27 * coutp * cinp;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
    const int ci = q % cinp, co = (q / cinp) % coutp, tap = q / (cinp * coutp);
    const float v = (ci < cin && co < cout) ? master[((size_t)tap * cout + co) * cin + ci] : 0.f;
    const __nv_bfloat16 b = __float2bfloat16(v);
    w[q] = b;
    wt[((size_t)(26 - tap) * cinp + ci) * coutp + co] = b;
  }
}

// Padded f32 gradient [27][coutp][cinp] back to the master layout [27][cout][cin] (accumulated).
__global__ void k_unpack_grad(int cin, int cout, int cinp, int coutp, const float* __restrict__ gp,
                              float* __restrict__ g) {
  const int n = 27 * cout * cin;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
    const int ci = q % cin, co = (q / cin) % cout, tap = q / (cin * cout);
    g[q] += gp[((size_t)tap * coutp + co) * cinp + ci];
  }
}

__global__ void k_unpack_grad_bias(int cout, const float* __restrict__ gb, float* __restrict__ g) {
  for (int q = threadIdx.x; q < cout; q += blockDim.x) g[q] += gb[q];
}

// Adam (Kingma & Ba, 2015) on the f32 master parameters; the gradient is consumed (zeroed).
__global__ void k_adam(int n, float* __restrict__ p, float* __restrict__ g, float* __restrict__ m,
                       float* __restrict__ v, float lr, float b1, float b2, float eps, float c1, float c2) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
    const float gq = g[q];
    const float mq = b1 * m[q] + (1.f - b1) * gq;
    const float vq = b2 * v[q] + (1.f - b2) * gq * gq;
    m[q] = mq;
    v[q] = vq;
    p[q] -= lr * (mq / c1) / (sqrtf(vq / c2) + eps);
    g[q] = 0.f;
  }
}

}  // namespace fd3u
