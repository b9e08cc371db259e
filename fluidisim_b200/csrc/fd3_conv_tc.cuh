// The 3x3x3 convolution of the learned preconditioner on the 5th-generation tensor cores
// (tcgen05.mma, accumulators in tensor memory), BF16 operands, FP32 accumulation.
//
// The GEMM view is the one of k_conv (fd3_unet.cuh): Out[cell][co] = sum over 27 taps and CIN
// channels of In[cell + tap][ci] * W[tap][co][ci].  M = output cells, N = COUT, K = 27 * CIN.
//
// Tiling.  A CTA owns BY consecutive rows (y) of one z-layer, all X cells of each row.  For each
// 16-channel chunk of the input it stages the halo block of rows z-1..z+1, y0-1..y0+BY, every x,
// in shared memory, and the chunk's weights of all 27 taps.  The staged layout makes every tap a
// plain shifted view of the same block, so no im2col copy is formed:
//   - cells are laid out flat, f = (zz * (BY + 2) + yy) * (X + 1) + xx, one zero pad cell at
//     xx = X ending every row, whole zero rows outside the sample, and zero cells before and after;
//   - each cell's 16 channels are split into two 8-channel halves held in two planes, cell f of
//     plane h at byte 16 f of that plane.
// That is the K-major, no-swizzle canonical operand layout of tcgen05.mma with the 8-row core
// matrices 128 B apart (SBO) and the two K halves one plane apart (LBO), for ANY starting cell.
// An M tile is 128 consecutive flat positions of the output rows (pad positions included and
// discarded at the epilogue); for tap (dz, dy, dx) its A operand starts dz (BY+2)(X+1) + dy (X+1)
// + dx cells further.  A shift of dx = -1 at x = 0 or of dx = +1 at x = X - 1 lands on a pad
// cell, which is the zero padding of the convolution.  The B operand of tap t is the N x 16 weight
// block in the same two-plane layout.
//
// One thread issues the 27 x NTM MMAs of a chunk (NTM <= TC_MAX_TILES M tiles of 128 rows, each
// accumulating into its own N columns of tensor memory) and commits them to an mbarrier; all
// threads wait on it (a bounded wait) before the shared memory is refilled and before the
// epilogue reads tensor memory with tcgen05.ld (warp w reads lanes 32 (w % 4) .. + 31).
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "fd3_unet.cuh"

namespace fd3u {

constexpr int TC_THREADS = 256;
constexpr int TC_MAX_TILES = 5;  // M tiles of 128 rows per CTA
constexpr int TC_LEAD = 8;       // zero cells before the block (the lowest tap reads cell -1)
constexpr int TC_TAIL = 128;     // zero cells after it (the last tile's rows past the block)
constexpr unsigned TC_SPIN_LIMIT = 1u << 26;

// Rows per CTA for rows of X cells: as many as keep BY (X + 1) <= 128 * tiles, where tiles is the
// requested budget of M tiles, raised to what one row needs.
__host__ __device__ inline int tc_rows(int X, int Y, int tiles = TC_MAX_TILES) {
  const int need = (X + 1 + 127) / 128;
  if (tiles < need) tiles = need;
  int by = (128 * tiles) / (X + 1);
  if (by < 1) by = 1;
  return by < Y ? by : Y;
}
__host__ __device__ inline int tc_tiles(int X, int BY) { return (BY * (X + 1) + 127) / 128; }
// Cells of one plane (multiple of 8: 128-byte aligned planes).
__host__ __device__ inline int tc_plane_cells(int X, int BY) {
  return (TC_LEAD + 3 * (BY + 2) * (X + 1) + TC_TAIL + 7) & ~7;
}
// Dynamic shared memory: 128 B of control words, the two input planes, the weights of one chunk.
__host__ __device__ inline size_t tc_smem_bytes(int X, int BY, int cout) {
  return 128 + (size_t)2 * tc_plane_cells(X, BY) * 16 + (size_t)27 * 2 * cout * 16;
}
// Tensor-memory columns: a power of two >= 32 holding NTM tiles of COUT f32 columns.
__host__ __device__ inline uint32_t tc_tmem_cols(int ntm, int cout) {
  uint32_t need = (uint32_t)(ntm * cout), c = 32;
  while (c < need) c <<= 1;
  return c;
}

// Shared-memory matrix descriptor (tcgen05), K-major, no swizzle: start address, leading-dimension
// byte offset (between the two K halves), stride-dimension byte offset (between 8-row groups),
// descriptor version 1.
__device__ __forceinline__ uint64_t tc_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1u << 46;
  return d;
}
// Instruction descriptor of kind::f16: D f32, A and B bf16, both K-major, M = 128, N.
__host__ __device__ constexpr uint32_t tc_idesc(int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void tc_mma(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  const uint32_t z = 0;
  asm volatile(
      "{\n\t"
      ".reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t"
      "}\n"
      :
      : "r"(tmem_d), "l"(a), "l"(b), "r"(idesc), "r"(acc), "r"(z), "r"(z), "r"(z), "r"(z));
}

__device__ __forceinline__ void tc_commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar) : "memory");
}

// Bounded wait for the mbarrier phase `parity`; false when the limit ran out.
__device__ __forceinline__ bool tc_wait(uint32_t mbar, uint32_t parity) {
  for (unsigned it = 0; it < TC_SPIN_LIMIT; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t"
        ".reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t"
        "}\n"
        : "=r"(done)
        : "r"(mbar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

__device__ __forceinline__ void cp_async16(uint32_t saddr, const void* g) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(saddr), "l"(g) : "memory");
}

// 16 columns of 32-bit accumulators of this thread's lane.
__device__ __forceinline__ void tc_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, "
      "[%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

template <int CIN, int COUT, int EPI>
__global__ void __launch_bounds__(TC_THREADS) k_conv_tc(Dims d, int BY, int NTM, const __nv_bfloat16* __restrict__ in,
                                                        const __nv_bfloat16* __restrict__ w,
                                                        const float* __restrict__ bias,
                                                        __nv_bfloat16* __restrict__ out, float* __restrict__ out32,
                                                        int* __restrict__ err) {
  static_assert(CIN % 16 == 0 && COUT % 16 == 0 && COUT >= 16 && COUT <= 256, "channel padding");
  extern __shared__ __align__(128) unsigned char smem[];
  uint64_t* mbar = reinterpret_cast<uint64_t*>(smem);
  uint32_t* taddr_slot = reinterpret_cast<uint32_t*>(smem + 8);
  const int X = d.X, Y = d.Y, Z = d.Z;
  const int PX = X + 1, PYX = (BY + 2) * PX;
  const int plane_cells = tc_plane_cells(X, BY);
  unsigned char* planeA = smem + 128;                          // two planes of plane_cells x 16 B
  unsigned char* planeB = planeA + (size_t)2 * plane_cells * 16;  // 27 taps x 2 planes x COUT x 16 B
  const uint32_t sA = smem_u32(planeA), sB = smem_u32(planeB), sbar = smem_u32(mbar);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  // CTA -> (sample, z, first row)
  const int yblocks = (Y + BY - 1) / BY;
  int bi = blockIdx.x;
  const int yb = bi % yblocks; bi /= yblocks;
  const int z = bi % Z;
  const int b = bi / Z;
  const int y0 = yb * BY;

  const uint32_t ncols = tc_tmem_cols(NTM, COUT);
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(sbar) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(taddr_slot)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  }
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *taddr_slot;

  const int block_cells = 3 * PYX;
  const int m0 = PYX + PX;  // flat position of (zz = 1, yy = 1, x = 0)
  constexpr uint32_t IDESC = tc_idesc(COUT);
  const uint32_t lboA = (uint32_t)plane_cells * 16, lboB = (uint32_t)COUT * 16;
  bool ok = true;

  // Zero once what no chunk overwrites: the lead and tail cells, every row's pad cell, and the rows
  // outside the sample.  Warp-per-row loops below need one division per row, not per element.
  const int nrows = 3 * (BY + 2);
  auto zero16 = [&](int h, int q) {
    asm volatile("st.shared.v4.u32 [%0], {%1, %1, %1, %1};" ::"r"(sA + (uint32_t)(h * plane_cells + q) * 16), "r"(0)
                 : "memory");
  };
  const int tail_cells = plane_cells - TC_LEAD - block_cells;
  for (int e = tid; e < 2 * (TC_LEAD + tail_cells); e += TC_THREADS) {
    const int h = e & 1, k = e >> 1;
    zero16(h, k < TC_LEAD ? k : TC_LEAD + block_cells + (k - TC_LEAD));
  }
  for (int r = warp; r < nrows; r += TC_THREADS / 32) {
    const int zi = z - 1 + r / (BY + 2), yi = y0 - 1 + r % (BY + 2);
    const bool outside = zi < 0 || zi >= Z || yi < 0 || yi >= Y;
    const int q0 = TC_LEAD + r * PX;
    if (outside) {
      for (int e = lane; e < 2 * PX; e += 32) zero16(e & 1, q0 + (e >> 1));
    } else if (lane < 2) {
      zero16(lane, q0 + X);  // the row's pad cell
    }
  }

  for (int ck = 0; ck < CIN / 16; ++ck) {
    if (ck > 0) ok = tc_wait(sbar, (uint32_t)(ck - 1) & 1u) && ok;  // the previous chunk's MMAs are done
    // input planes: one warp per block row; lane pairs take one cell's two halves, so a warp reads
    // 16 consecutive cells' 32-byte chunk slices
    for (int r = warp; r < nrows; r += TC_THREADS / 32) {
      const int zi = z - 1 + r / (BY + 2), yi = y0 - 1 + r % (BY + 2);
      if (zi < 0 || zi >= Z || yi < 0 || yi >= Y) continue;
      const __nv_bfloat16* src = in + ((((long long)b * Z + zi) * Y + yi) * X) * CIN + ck * 16;
      const uint32_t dst = sA + (uint32_t)(TC_LEAD + r * PX) * 16;
      for (int e = lane; e < 2 * X; e += 32) {
        const int xx = e >> 1, h = e & 1;
        cp_async16(dst + (uint32_t)(h * plane_cells + xx) * 16, src + (long long)xx * CIN + h * 8);
      }
    }
    // weights of the chunk: tap t, half h, row n <- W[t][n][ck*16 + 8h .. + 8)
    for (int e = tid; e < 27 * 2 * COUT; e += TC_THREADS) {
      const int n = e % COUT, h = (e / COUT) & 1, t = e / (2 * COUT);
      cp_async16(sB + (uint32_t)e * 16, w + ((size_t)t * COUT + n) * CIN + ck * 16 + h * 8);
    }
    asm volatile("cp.async.wait_all;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      for (int t = 0; t < 27; ++t) {
        const int off = (t / 9 - 1) * PYX + ((t / 3) % 3 - 1) * PX + (t % 3 - 1);
        const uint64_t bdesc = tc_desc(sB + (uint32_t)t * 2 * COUT * 16, lboB, 128);
        for (int j = 0; j < NTM; ++j) {
          const int row0 = TC_LEAD + m0 + 128 * j + off;  // >= TC_LEAD - 1 >= 0
          const uint64_t adesc = tc_desc(sA + (uint32_t)row0 * 16, lboA, 128);
          tc_mma(tmem + (uint32_t)(j * COUT), adesc, bdesc, IDESC, (ck > 0 || t > 0) ? 1u : 0u);
        }
      }
      tc_commit(sbar);
    }
    __syncthreads();
  }
  ok = tc_wait(sbar, (uint32_t)(CIN / 16 - 1) & 1u) && ok;
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (!ok && tid == 0) atomicExch(err, 1);

  // epilogue: warp w reads lanes 32 (w % 4) + lane of tiles j = w / 4, w / 4 + 2, ...
  const int lane_base = 32 * (warp & 3);
  for (int j = warp >> 2; j < NTM; j += TC_THREADS / 128) {
    const int qpos = 128 * j + lane_base + lane;  // flat position relative to m0
    const int yl = qpos / PX, x = qpos % PX;
    const bool valid = ok && x < X && yl < BY && y0 + yl < Y;
    const long long cell = (((long long)b * Z + z) * Y + y0 + yl) * X + x;
#pragma unroll
    for (int c0 = 0; c0 < COUT; c0 += 16) {
      float v[16];
      tc_ld16(tmem + ((uint32_t)lane_base << 16) + (uint32_t)(j * COUT + c0), v);
      if (!valid) continue;
      if constexpr (EPI == EPI_BIAS_F32_CH0) {
        if (c0 == 0) out32[cell] = v[0] + bias[0];
      } else {
        __align__(16) __nv_bfloat16 o[16];
#pragma unroll
        for (int i = 0; i < 16; ++i) {
          float a = v[i];
          if (EPI == EPI_BIAS_RELU) a = fmaxf(a + bias[c0 + i], 0.f);
          o[i] = __float2bfloat16(a);
        }
        uint4* dst = reinterpret_cast<uint4*>(out + cell * COUT + c0);
        dst[0] = reinterpret_cast<const uint4*>(o)[0];
        dst[1] = reinterpret_cast<const uint4*>(o)[1];
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols) : "memory");
  }
}

}  // namespace fd3u
