// The 3x3x3 convolution on the 5th-generation tensor cores as a warp-specialised pipeline.
//
// The GEMM view, the staged layout (the K-major, no-swizzle canonical operand layout, every tap a
// shifted view of one staged halo block) and the MMA sequence of a work tile are those of k_conv_tc
// (fd3_conv_tc.cuh): for each 16-channel chunk, 27 taps x NTM M tiles of 128 rows, accumulated in
// tensor memory in the same order, so the two kernels give the same bits.  What changes is that the
// phases of consecutive work tiles overlap instead of running one after the other:
//
//   warps 4-7   producers: stage (chunk, work tile) units into a ring of S shared-memory slots
//               (cp.async of the input rows, zeros for rows outside the sample, the chunk's
//               weights), each thread then waits for its own copies, fences them for the tensor
//               core's async proxy and arrives on the slot's `full` barrier;
//   warp 8      one thread issues the unit's 27 x NTM tcgen05.mma into one of two accumulators in
//               tensor memory and commits them to the slot's `empty` barrier (the slot can be
//               refilled) and, after a work tile's last chunk, to the accumulator's `full` barrier;
//   warps 0-3   the epilogue: tcgen05.ld of the accumulator (warp w reads lanes 32 w .. 32 w + 31),
//               bias, ReLU, BF16 stores, then an arrive on the accumulator's `empty` barrier.
//
// The CTA is persistent: it takes work tiles blockIdx.x, blockIdx.x + gridDim.x, ...  While the
// epilogue drains one accumulator the MMAs of the next tile fill the other, and the producers run
// up to S units ahead.  Every wait is bounded (TC_SPIN_LIMIT polls); after a wait runs out, the thread
// waits no more, so each role runs through its loop at once, and the kernel sets *err, frees its
// tensor memory and returns.
#pragma once

#include "fd3_conv_tc.cuh"

namespace fd3u {

constexpr int TP_EPI_WARPS = 4, TP_PROD_WARPS = 4;
constexpr int TP_THREADS = 32 * (TP_EPI_WARPS + TP_PROD_WARPS + 1);
constexpr int TP_PRODUCERS = 32 * TP_PROD_WARPS;
constexpr int TP_EPILOGUE = 32 * TP_EPI_WARPS;
constexpr int TP_MAX_STAGES = 4;
constexpr int TP_CTRL_BYTES = 256;  // the barriers and the tensor-memory address slot

// Bytes of one stage slot: the two input planes of a chunk and its weights for all 27 taps.
__host__ __device__ inline size_t tp_stage_bytes(int X, int BY, int cout) {
  return (size_t)2 * tc_plane_cells(X, BY) * 16 + (size_t)27 * 2 * cout * 16;
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile(
      "{\n\t.reg .b64 st;\n\t"
      "mbarrier.arrive.shared::cta.b64 st, [%0];\n\t}" ::"r"(bar)
      : "memory");
}

template <int CIN, int COUT, int EPI>
__global__ void __launch_bounds__(TP_THREADS, 1) k_conv_tp(Dims d, int BY, int NTM, int S, int W,
                                                           const __nv_bfloat16* __restrict__ in,
                                                           const __nv_bfloat16* __restrict__ w,
                                                           const float* __restrict__ bias,
                                                           __nv_bfloat16* __restrict__ out, float* __restrict__ out32,
                                                           int* __restrict__ err) {
  static_assert(CIN % 16 == 0 && COUT % 16 == 0 && COUT >= 16 && COUT <= 256, "channel padding");
  constexpr int NCH = CIN / 16;
  extern __shared__ __align__(128) unsigned char smem[];
  // barriers: full[0..3], empty[4..7], acc_full[8..9], acc_empty[10..11]; the TMEM slot after them
  const uint32_t sbar = smem_u32(smem);
  auto full = [&](int s) { return sbar + 8u * (uint32_t)s; };
  auto empty = [&](int s) { return sbar + 8u * (uint32_t)(4 + s); };
  auto accf = [&](int a) { return sbar + 8u * (uint32_t)(8 + a); };
  auto acce = [&](int a) { return sbar + 8u * (uint32_t)(10 + a); };
  uint32_t* taddr_slot = reinterpret_cast<uint32_t*>(smem + 96);
  const int X = d.X, Y = d.Y, Z = d.Z;
  const int PX = X + 1, PYX = (BY + 2) * PX;
  const int plane_cells = tc_plane_cells(X, BY);
  const size_t stage_bytes = tp_stage_bytes(X, BY, COUT);
  const uint32_t sStage0 = smem_u32(smem + TP_CTRL_BYTES);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int yblocks = (Y + BY - 1) / BY;
  const int nrows = 3 * (BY + 2);
  const int block_cells = 3 * PYX;
  const int m0 = PYX + PX;  // flat position of (zz = 1, yy = 1, x = 0)
  const uint32_t ncols = tc_tmem_cols(2 * NTM, COUT);

  if (tid == 0) {
    for (int s = 0; s < TP_MAX_STAGES; ++s) {
      mbar_init(full(s), TP_PRODUCERS);
      mbar_init(empty(s), 1);
    }
    for (int a = 0; a < 2; ++a) {
      mbar_init(accf(a), 1);
      mbar_init(acce(a), TP_EPILOGUE);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(taddr_slot)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  }
  // zero, in every slot, what no unit writes: the lead and tail cells and every row's pad cell
  const int tail_cells = plane_cells - TC_LEAD - block_cells;
  for (int s = 0; s < S; ++s) {
    const uint32_t sA = sStage0 + (uint32_t)(s * stage_bytes);
    auto zero16 = [&](int h, int q) {
      asm volatile("st.shared.v4.u32 [%0], {%1, %1, %1, %1};" ::"r"(sA + (uint32_t)(h * plane_cells + q) * 16), "r"(0)
                   : "memory");
    };
    for (int e = tid; e < 2 * (TC_LEAD + tail_cells); e += TP_THREADS) {
      const int h = e & 1, k = e >> 1;
      zero16(h, k < TC_LEAD ? k : TC_LEAD + block_cells + (k - TC_LEAD));
    }
    for (int e = tid; e < 2 * nrows; e += TP_THREADS) zero16(e & 1, TC_LEAD + (e >> 1) * PX + X);
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *taddr_slot;
  bool ok = true;

  if (warp >= TP_EPI_WARPS && warp < TP_EPI_WARPS + TP_PROD_WARPS) {
    // ------------------------------------------------------------------------------ producers
    const int ptid = tid - TP_EPILOGUE, pwarp = ptid >> 5;
    int u = 0;
    for (int wi = blockIdx.x; wi < W; wi += gridDim.x) {
      int bi = wi;
      const int yb = bi % yblocks; bi /= yblocks;
      const int z = bi % Z;
      const int b = bi / Z;
      const int y0 = yb * BY;
      for (int ck = 0; ck < NCH; ++ck, ++u) {
        const int s = u % S, k = u / S;
        if (k > 0 && ok) ok = tc_wait(empty(s), (uint32_t)(k - 1) & 1u);
        const uint32_t sA = sStage0 + (uint32_t)(s * stage_bytes);
        const uint32_t sB = sA + (uint32_t)plane_cells * 32u;
        for (int r = pwarp; r < nrows; r += TP_PROD_WARPS) {
          const int zi = z - 1 + r / (BY + 2), yi = y0 - 1 + r % (BY + 2);
          const uint32_t dst = sA + (uint32_t)(TC_LEAD + r * PX) * 16;
          if (zi < 0 || zi >= Z || yi < 0 || yi >= Y) {
            for (int e = lane; e < 2 * X; e += 32) {
              const int xx = e >> 1, h = e & 1;
              asm volatile("st.shared.v4.u32 [%0], {%1, %1, %1, %1};" ::"r"(dst + (uint32_t)(h * plane_cells + xx) * 16),
                           "r"(0)
                           : "memory");
            }
            continue;
          }
          const __nv_bfloat16* src = in + ((((long long)b * Z + zi) * Y + yi) * X) * CIN + ck * 16;
          for (int e = lane; e < 2 * X; e += 32) {
            const int xx = e >> 1, h = e & 1;
            cp_async16(dst + (uint32_t)(h * plane_cells + xx) * 16, src + (long long)xx * CIN + h * 8);
          }
        }
        for (int e = ptid; e < 27 * 2 * COUT; e += TP_PRODUCERS) {
          const int n = e % COUT, h = (e / COUT) & 1, t = e / (2 * COUT);
          cp_async16(sB + (uint32_t)e * 16, w + ((size_t)t * COUT + n) * CIN + ck * 16 + h * 8);
        }
        asm volatile("cp.async.wait_all;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        mbar_arrive(full(s));
      }
    }
  } else if (warp == TP_EPI_WARPS + TP_PROD_WARPS) {
    // ------------------------------------------------------------------------------ the MMA issuer
    if (lane == 0) {
      constexpr uint32_t IDESC = tc_idesc(COUT);
      const uint32_t lboA = (uint32_t)plane_cells * 16, lboB = (uint32_t)COUT * 16;
      int u = 0, i = 0;
      for (int wi = blockIdx.x; wi < W; wi += gridDim.x, ++i) {
        const int a = i & 1;
        if (i >= 2 && ok) ok = tc_wait(acce(a), (uint32_t)((i >> 1) - 1) & 1u);  // the epilogue freed it
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t acc = tmem + (uint32_t)(a * NTM * COUT);
        for (int ck = 0; ck < NCH; ++ck, ++u) {
          const int s = u % S, k = u / S;
          if (ok) ok = tc_wait(full(s), (uint32_t)k & 1u);
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          const uint32_t sA = sStage0 + (uint32_t)(s * stage_bytes);
          const uint32_t sB = sA + (uint32_t)plane_cells * 32u;
          for (int t = 0; t < 27; ++t) {
            const int off = (t / 9 - 1) * PYX + ((t / 3) % 3 - 1) * PX + (t % 3 - 1);
            const uint64_t bdesc = tc_desc(sB + (uint32_t)t * 2 * COUT * 16, lboB, 128);
            for (int j = 0; j < NTM; ++j) {
              const int row0 = TC_LEAD + m0 + 128 * j + off;
              const uint64_t adesc = tc_desc(sA + (uint32_t)row0 * 16, lboA, 128);
              tc_mma(acc + (uint32_t)(j * COUT), adesc, bdesc, IDESC, (ck > 0 || t > 0) ? 1u : 0u);
            }
          }
          tc_commit(empty(s));
          if (ck == NCH - 1) tc_commit(accf(a));
        }
      }
      if (u > 0 && ok) ok = tc_wait(empty((u - 1) % S), (uint32_t)((u - 1) / S) & 1u);  // the last MMAs are done
    }
  } else {
    // ------------------------------------------------------------------------------ the epilogue
    const int lane_base = 32 * warp;
    int i = 0;
    for (int wi = blockIdx.x; wi < W; wi += gridDim.x, ++i) {
      int bi = wi;
      const int yb = bi % yblocks; bi /= yblocks;
      const int z = bi % Z;
      const int b = bi / Z;
      const int y0 = yb * BY;
      const int a = i & 1;
      const bool ready = ok && tc_wait(accf(a), (uint32_t)(i >> 1) & 1u);
      ok = ready;
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      for (int j = 0; j < NTM; ++j) {
        const int qpos = 128 * j + lane_base + lane;  // flat position relative to m0
        const int yl = qpos / PX, x = qpos % PX;
        const bool valid = ready && x < X && yl < BY && y0 + yl < Y;
        const long long cell = (((long long)b * Z + z) * Y + y0 + yl) * X + x;
#pragma unroll
        for (int c0 = 0; c0 < COUT; c0 += 16) {
          float v[16];
          tc_ld16(tmem + ((uint32_t)lane_base << 16) + (uint32_t)(a * NTM * COUT + j * COUT + c0), v);
          if (!valid) continue;
          if constexpr (EPI == EPI_BIAS_F32_CH0) {
            if (c0 == 0) out32[cell] = v[0] + bias[0];
          } else {
            __align__(16) __nv_bfloat16 o[16];
#pragma unroll
            for (int e = 0; e < 16; ++e) {
              float x_ = v[e];
              if (EPI == EPI_BIAS_RELU) x_ = fmaxf(x_ + bias[c0 + e], 0.f);
              o[e] = __float2bfloat16(x_);
            }
            uint4* dst = reinterpret_cast<uint4*>(out + cell * COUT + c0);
            dst[0] = reinterpret_cast<const uint4*>(o)[0];
            dst[1] = reinterpret_cast<const uint4*>(o)[1];
          }
        }
      }
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      mbar_arrive(acce(a));
    }
  }
  if (!ok) atomicExch(err, 1);
  // the MMA issuer's last commits: every accumulator's MMAs are done before tensor memory is freed
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols) : "memory");
  }
}

}  // namespace fd3u
