// The 2.5-D blocked fine-level kernels on TMA-staged layers (fd3_options.kernels = 5).
//
// Each CTA owns a 64 x 8 tile of columns (a warp per row, each lane a pair of adjacent cells; the
// kernel is written for Q cells per lane, Q = 2 or 4) and marches up K layers.  The loads that the paired march (fd3_zmarch2.cuh) issues per thread, with
// their address arithmetic, bounds tests and the divergent halo lanes, become one elected thread's
// cp.async.bulk.tensor copies per layer into a ring of shared-memory stages, each completing on its
// own mbarrier (complete_tx):
//   - a stream whose neighbours the stencil needs (the operand's inputs) as a halo box: x from
//     x0 - 4 (the 16-byte-aligned start left of the tile) over 72 cells, y from y0 - 1 over 10 rows;
//     the tensor map's out-of-bounds fill gives zeros outside the volume;
//   - a stream read at the tile's own cells as a 64 x 8 box, the row codes as a 64 x 8 box of u16;
//   - the prolongation's parent values of level 0 (post1) as a 40 x 6 box of that level's layer k/2.
// Layers outside the volume in z are clamped to the nearest layer: the row codes close every face at
// the volume's edge, and a closed face's term is never added (apply_code_nb), so what sits there does
// not matter.  The operand of a pass that computes one (d = z + beta d, the first pre-sweep, the
// prolonged z) is formed once per layer over the halo box into a ring of four operand planes; the
// other passes read the staged stream itself.  The stencil then reads its seven operands, its codes
// and its epilogue's streams from shared memory only.
//
// One barrier per layer.  At layer k the ring holds layers k - 1 .. k + D + 1 (operand passes, D + 2
// stages: the stage of layer k - 1 is refilled with layer k + D + 1 once the barrier shows every thread
// done with it) or k - 2 .. k + D + 1 (the others, D + 3 stages); D = 2, or deeper where the layers
// stream from HBM.  Every mbarrier wait is bounded (TM_SPIN_LIMIT polls):
// on expiry the CTA stops marching, waits (bounded again) for the copies it has in flight, marks the
// projection not finite (Scalars::status 2) and hands a NaN to its reduction, so the loop stops and
// the host reports an error.
//
// The per-cell arithmetic is that of the other families (apply_code_nb, the same expressions in the
// same order): bit-identical cell values; only the order of the f64 reduction partials differs.
// Needs f32 storage and nx % 8 == 0 (the tensor maps' row strides are multiples of 16 bytes), and,
// with coarse levels, level 0 of exactly half the fine size.
#pragma once

#include <cuda.h>

#include <type_traits>

#include "fd3_zmarch2.cuh"

namespace fd3 {

constexpr int TMX = 64, TMY = 8;
constexpr int TMW = TMX + 8, TMH = TMY + 2;            // halo box
constexpr int TMPW = TMX / 2 + 8, TMPH = TMY / 2 + 2;  // parent box
constexpr unsigned TM_HALO_BYTES = TMW * TMH * 4;
constexpr unsigned TM_OWN_BYTES = TMX * TMY * 4;
constexpr unsigned TM_CODE_BYTES = TMX * TMY * 2;
constexpr unsigned TM_PAR_BYTES = TMPW * TMPH * 4;
__host__ __device__ constexpr unsigned tm_al(unsigned b) { return (b + 127u) & ~127u; }
constexpr unsigned TM_CTRL_BYTES = 128;  // the stages' mbarriers and the abort word
constexpr unsigned TM_SPIN_LIMIT = 1u << 24;

// Resident CTAs per SM the register budget is cut for (the ring's shared memory allows five for every
// pass but post1, which fits four).
#ifndef FD3_TMINB
#define FD3_TMINB 5
#endif

inline int zblocks_t(int nx, int ny, int nz, int k) {
  return ((nx + TMX - 1) / TMX) * ((ny + TMY - 1) / TMY) * ((nz + k - 1) / k);
}

// The tensor maps of one launch: halo streams, tile streams, the codes, the parent (in that order).
struct TMaps {
  CUtensorMap m[5];
};

enum { TP_DIR = 0, TP_PRE, TP_RESTRICT, TP_POST1, TP_POST2, TP_RESID };

// Streams of each pass: NH halo boxes, NO tile boxes, the parent box (PAR), an operand plane (OPP);
// D layers are in flight ahead of the one whose operand is formed (the ring holds S stages).
template <int PASS, int D = 2>
struct TPass {
  static constexpr int NH = (PASS == TP_DIR || PASS == TP_PRE || PASS == TP_POST1) ? 2 : 1;
  static constexpr int NO = PASS == TP_POST2 ? 2 : ((PASS == TP_DIR || PASS == TP_PRE) ? 0 : 1);
  static constexpr int PAR = PASS == TP_POST1 ? 1 : 0;
  static constexpr int OPP = (PASS == TP_DIR || PASS == TP_PRE || PASS == TP_POST1) ? 1 : 0;
  static constexpr int S = OPP ? D + 2 : D + 3;
  static constexpr unsigned OFF_O = NH * tm_al(TM_HALO_BYTES);
  static constexpr unsigned OFF_C = OFF_O + NO * tm_al(TM_OWN_BYTES);
  static constexpr unsigned OFF_P = OFF_C + tm_al(TM_CODE_BYTES);
  static constexpr unsigned STAGE = OFF_P + PAR * tm_al(TM_PAR_BYTES);
  static constexpr unsigned OFF_OP = TM_CTRL_BYTES + S * STAGE;
  static constexpr unsigned OFF_TR = OFF_OP + (OPP ? 4 * tm_al(TM_HALO_BYTES) : 0u);
  static constexpr unsigned SMEM = OFF_TR + (PASS == TP_RESTRICT ? 2u * TMY * TMX * 4u : 0u);
  static constexpr unsigned SMEM_LAUNCH = SMEM + 128;  // the base is aligned to 128 bytes in the kernel
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void tm_expect(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ void tm_load3(uint32_t dst, const CUtensorMap* map, int x, int y, int z, uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(
          dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(bar)
      : "memory");
}
// Bounded wait for phase `parity` of an mbarrier; false when the limit ran out.
__device__ __forceinline__ bool tm_wait(uint32_t bar, uint32_t parity) {
  for (unsigned it = 0; it < TM_SPIN_LIMIT; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// Per-pass runtime inputs beside the tensor maps.
struct TArgs {
  float* out0;        // dout (DIR), z2 (PRE), zout (POST1/POST2), res (RESID)
  float* out1;        // q (DIR)
  Lev L;              // level 0 (RESTRICT: its r; POST1: prolongation on)
  int prolong;        // POST1: 1 = add the parent (coarse levels exist)
  int gate;           // return at once when the inner loop has stopped
  int op;             // the reduction's finishing step (POST2, RESID)
};

// A.P at a pair of cells (0 at a dry cell).  When both rows are plain or dry (no surface ghost, every
// live face of aperture 1: the bulk, the walls and the air) each cell takes the masked sum of its six
// differences, which for a dry cell (code 0) is +0, without a branch per cell; otherwise
// apply_code_nb per wet cell.  The same bits either way (rc_plain).
__device__ __forceinline__ bool rc_plain_or_dry(unsigned code) {
  return (code & RC_GHOSTS) == 0u && (code & (RC_UNIT | RC_WET)) != RC_WET;
}
__device__ __forceinline__ float masked_row(const Geo& g, unsigned code, float pc, float xm, float xp, float ym,
                                            float yp, float zm, float zp) {
  float acc = 0.f;
  acc += (code & (1u << 1)) ? pc - xm : 0.f;
  acc += (code & (1u << 3)) ? pc - xp : 0.f;
  acc += (code & (1u << 5)) ? pc - ym : 0.f;
  acc += (code & (1u << 7)) ? pc - yp : 0.f;
  acc += (code & (1u << 9)) ? pc - zm : 0.f;
  acc += (code & (1u << 11)) ? pc - zp : 0.f;
  return acc * g.inv;
}

// The end of a pass's f64 reduction for any block size (the blocks of the four-cell kernels have 128
// threads): warp shuffles, the warps' sums in order, one partial per block, and the last block to
// arrive merges the partials in a fixed order and applies the PCG step (as reduce_finish).
__device__ __forceinline__ void kt_reduce_finish(double v, Red red, Scalars* S, int op) {
  __shared__ double sw[TPB / 32];
  __shared__ bool last;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) sw[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {  // the block's partial, visible before the block counts in
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += sw[w];
    red.p64[blockIdx.x] = t;
    __threadfence();
    last = atomicAdd(red.count, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  finish_block<RED_F64>(red, (int)gridDim.x, S, op);
  if (threadIdx.x == 0) *red.count = 0u;
}

// Q cells per thread along x (2: 32 lanes per row of the tile, 256 threads; 4: 16 lanes, 128 threads).
template <int Q>
struct TQ {
  static constexpr int LANES = TMX / Q, NT = TMX * TMY / Q;
};
template <int Q>
using QV = typename std::conditional<Q == 4, float4, float2>::type;
__device__ __forceinline__ float qe(const float2& v, int e) { return e == 0 ? v.x : v.y; }
__device__ __forceinline__ float qe(const float4& v, int e) { return e == 0 ? v.x : (e == 1 ? v.y : (e == 2 ? v.z : v.w)); }
__device__ __forceinline__ void qs(float2& v, int e, float x) { if (e == 0) v.x = x; else v.y = x; }
__device__ __forceinline__ void qs(float4& v, int e, float x) {
  if (e == 0) v.x = x; else if (e == 1) v.y = x; else if (e == 2) v.z = x; else v.w = x;
}

template <int PASS, int K, int D, int Q, int MINB>
__global__ void __launch_bounds__(TQ<Q>::NT, MINB)
    kt_pass(const __grid_constant__ TMaps M, Geo g, TArgs a, Red red, Scalars* S) {
  typedef TPass<PASS, D> P;
  typedef QV<Q> V;
  constexpr int NS = P::S, NT = TQ<Q>::NT, LANES = TQ<Q>::LANES;
  constexpr int HF = tm_al(TM_HALO_BYTES) / 4;  // floats between two halo planes (stage or operand ring)
  KSTART();
  if (PASS == TP_DIR) { if (!S->active) return; }
  else if (a.gate && !S->active) return;
  extern __shared__ __align__(128) unsigned char tm_raw[];
  unsigned char* sm = tm_raw + ((128u - (smem_u32(tm_raw) & 127u)) & 127u);  // 128-byte aligned, still shared
  const int tid = threadIdx.x, tx = tid % LANES, ty = tid / LANES;
  const int ntx = (g.nx + TMX - 1) / TMX, nty = (g.ny + TMY - 1) / TMY;
  int b = blockIdx.x;
  const int bx = b % ntx; b /= ntx;
  const int by = b % nty; b /= nty;
  const int x0 = bx * TMX, y0 = by * TMY, k0 = b * K, k1 = min(k0 + K, g.nz);
  const int i0 = x0 + Q * tx, j = y0 + ty;
  const bool inside = i0 < g.nx && j < g.ny;  // nx % 8 == 0: the thread's Q cells are all inside or all out
  double acc = 0.0;
  bool skip = false;
  if (g.tiles) {  // a 64 x 8 tile is two 32 x 8 tiles of the set's tile flags
    const int ntt = (g.nx + TILE_X - 1) / TILE_X, row = (y0 / TILE_Y) * ntt, t0 = x0 / TILE_X;
    skip = !g.tiles[row + t0] && (t0 + 1 >= ntt || !g.tiles[row + t0 + 1]);  // no column of the set
  }
  if (!skip) {
    const int dmode = PASS == TP_DIR ? S->dir_mode : 0;
    const float beta = PASS == TP_DIR ? S->beta : 0.f;
    const bool h1_on = PASS != TP_DIR || dmode != 0;  // d is read only for d = z + beta d
    const bool par_on = P::PAR && a.prolong;
    const uint32_t bar0 = smem_u32(sm);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(sm + 64);
    unsigned char* const stages = sm + TM_CTRL_BYTES;
    // Layers take the stages in turn (layer k0 - 1 the first), both in issue and in wait order.  One
    // thread of the last warp issues the copies: the operand planes are formed by the first warps.
    constexpr int ISSUER = NT - 32;
    int s_issue = 0, issued = k0 - 2;  // the issuer: the next stage to fill, the last layer issued
    auto issue = [&](int L) {
      const int zc = min(max(L, 0), g.nz - 1);
      const uint32_t st = smem_u32(stages + s_issue * P::STAGE), bar = bar0 + 8u * s_issue;
      const uint32_t bytes = (P::NH - (h1_on ? 0 : 1)) * TM_HALO_BYTES + P::NO * TM_OWN_BYTES + TM_CODE_BYTES +
                             (par_on ? TM_PAR_BYTES : 0u);
      tm_expect(bar, bytes);
      tm_load3(st, &M.m[0], x0 - 4, y0 - 1, zc, bar);
      if (P::NH > 1 && h1_on) tm_load3(st + tm_al(TM_HALO_BYTES), &M.m[1], x0 - 4, y0 - 1, zc, bar);
#pragma unroll
      for (int o = 0; o < P::NO; ++o) tm_load3(st + P::OFF_O + o * tm_al(TM_OWN_BYTES), &M.m[P::NH + o], x0, y0, zc, bar);
      tm_load3(st + P::OFF_C, &M.m[P::NH + P::NO], x0, y0, zc, bar);
      if (par_on) tm_load3(st + P::OFF_P, &M.m[P::NH + P::NO + 1], x0 / 2 - 4, y0 / 2 - 1, zc >> 1, bar);
      s_issue = s_issue + 1 == NS ? 0 : s_issue + 1;
      issued = L;
    };
    if (tid == ISSUER) {
      for (int s = 0; s < NS; ++s) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar0 + 8u * s) : "memory");
      *abort_flag = 0;
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
      for (int L = k0 - 1; L <= min(k0 + D, k1); ++L) issue(L);  // layers k - 1 .. k + D of the first k = k0
    }
    __syncthreads();
    int s_wait = 0, waited = k0 - 2;  // the next stage to wait for, the last layer waited for
    uint32_t par = 0u;                 // bit s: the parity of stage s's next phase
    auto wait_next = [&]() {  // a wait that runs out leaves the state, so the drain waits for it again
      const bool ok = tm_wait(bar0 + 8u * s_wait, (par >> s_wait) & 1u);
      if (ok) {
        par ^= 1u << s_wait;
        s_wait = s_wait + 1 == NS ? 0 : s_wait + 1;
        ++waited;
      }
      return ok;
    };

    // The operand plane of a layer over the halo box (operand passes), from its stage: slot t holds the
    // four floats 4t .. 4t + 3 of the box (row t / 18), with their parents from the parent box (post1).
    float* const opl = reinterpret_cast<float*>(sm + P::OFF_OP);
    auto op_slot = [&](const unsigned char* st, float* o, int t) {
      const float4 h0 = reinterpret_cast<const float4*>(st)[t];
      float4 v;
      if (PASS == TP_DIR) {
        if (dmode) {
          const float4 d = reinterpret_cast<const float4*>(st + tm_al(TM_HALO_BYTES))[t];
          v = make_float4(h0.x + beta * d.x, h0.y + beta * d.y, h0.z + beta * d.z, h0.w + beta * d.w);
        } else {
          v = h0;
        }
      } else if (PASS == TP_PRE) {  // the first pre-sweep from zero: prec, r
        const float4 r = reinterpret_cast<const float4*>(st + tm_al(TM_HALO_BYTES))[t];
        v.x = h0.x > 0.f ? 0.f + OMEGA * h0.x * (r.x - 0.f) : 0.f;
        v.y = h0.y > 0.f ? 0.f + OMEGA * h0.y * (r.y - 0.f) : 0.f;
        v.z = h0.z > 0.f ? 0.f + OMEGA * h0.z * (r.z - 0.f) : 0.f;
        v.w = h0.w > 0.f ? 0.f + OMEGA * h0.w * (r.w - 0.f) : 0.f;
      } else {  // post1: z + parent x, zero where prec == 0 (or z alone without coarse levels)
        if (par_on) {
          const float4 m = reinterpret_cast<const float4*>(st + tm_al(TM_HALO_BYTES))[t];
          const int prow = t / (TMW / 4), px = 4 * (t - prow * (TMW / 4));
          const float* pp = reinterpret_cast<const float*>(st + P::OFF_P) + (((prow - 1) >> 1) + 1) * TMPW + (px >> 1) + 2;
          const float pa = pp[0], pb = pp[1];
          float u;
          u = h0.x + pa; v.x = m.x == 0.f ? 0.f : u;
          u = h0.y + pa; v.y = m.y == 0.f ? 0.f : u;
          u = h0.z + pb; v.z = m.z == 0.f ? 0.f : u;
          u = h0.w + pb; v.w = m.w == 0.f ? 0.f : u;
        } else {
          v = h0;
        }
      }
      reinterpret_cast<float4*>(o)[t] = v;
    };
    auto make_op = [&](const unsigned char* st, int slot) {
      if (!P::OPP) return;
      float* o = opl + slot * HF;
#pragma unroll
      for (int t = tid; t < TMW * TMH / 4; t += NT) op_slot(st, o, t);
    };

    // layers k0 - 1 and k0
    bool ok = wait_next();
    make_op(stages, (k0 - 1) & 3);
    ok = wait_next() && ok;
    make_op(stages + P::STAGE, k0 & 3);
    if (!ok) *abort_flag = 1;

    float* const tr = reinterpret_cast<float*>(sm + P::OFF_TR);
    const int hc = (ty + 1) * TMW + 4 + Q * tx;  // the thread's first cell in a halo-box plane
    const int oc = ty * TMX + Q * tx;            // ... in a tile-box plane
    const int nxny = g.nx * g.ny;
    int c = j * g.nx + i0 + k0 * nxny;
    int sk = 1;  // the stage of layer k
    for (int k = k0; k < k1; ++k, c += nxny) {
      const int skn = sk + 1 == NS ? 0 : sk + 1, skp = sk == 0 ? NS - 1 : sk - 1;
      const unsigned char* st = stages + sk * P::STAGE;
      if (!wait_next()) *abort_flag = 1;  // layer k + 1
      make_op(stages + skn * P::STAGE, (k + 1) & 3);
      __syncthreads();
      if (*abort_flag) break;
      if (tid == ISSUER && k + D + 1 <= k1) {
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // the generic reads of the stage before its refill
        issue(k + D + 1);
      }
      const float* O = P::OPP ? opl + (k & 3) * HF : reinterpret_cast<const float*>(st);
      const float* Om = P::OPP ? opl + ((k - 1) & 3) * HF : reinterpret_cast<const float*>(stages + skp * P::STAGE);
      const float* Op = P::OPP ? opl + ((k + 1) & 3) * HF : reinterpret_cast<const float*>(stages + skn * P::STAGE);
      sk = skn;
      if (inside) {
        const V pc = *reinterpret_cast<const V*>(O + hc);
        const float xl = O[hc - 1], xr = O[hc + Q];
        const V ym = *reinterpret_cast<const V*>(O + hc - TMW);
        const V yp = *reinterpret_cast<const V*>(O + hc + TMW);
        const V zm = *reinterpret_cast<const V*>(Om + hc);
        const V zp = *reinterpret_cast<const V*>(Op + hc);
        unsigned cd[Q];
        if constexpr (Q == 4) {
          const uint2 w = *reinterpret_cast<const uint2*>(st + P::OFF_C + 2 * oc);
          cd[0] = w.x & 0xffffu; cd[1] = w.x >> 16; cd[2] = w.y & 0xffffu; cd[3] = w.y >> 16;
        } else {
          const unsigned w = *reinterpret_cast<const unsigned*>(st + P::OFF_C + 2 * oc);
          cd[0] = w & 0xffffu; cd[1] = w >> 16;
        }
        bool fast = true;
#pragma unroll
        for (int e = 0; e < Q; ++e) fast = fast && rc_plain_or_dry(cd[e]);
        unsigned any = 0u;
#pragma unroll
        for (int e = 0; e < Q; ++e) any |= cd[e];
        V av;
        if (any == 0u) {  // every cell dry: the masked sums are +0 (a warp of air skips them)
#pragma unroll
          for (int e = 0; e < Q; ++e) qs(av, e, 0.f);
        } else if (fast) {
#pragma unroll
          for (int e = 0; e < Q; ++e) {
            const float pe = qe(pc, e), xm = e == 0 ? xl : qe(pc, e - 1), xp = e == Q - 1 ? xr : qe(pc, e + 1);
            qs(av, e, masked_row(g, cd[e], pe, xm, xp, qe(ym, e), qe(yp, e), qe(zm, e), qe(zp, e)));
          }
        } else {
#pragma unroll
          for (int e = 0; e < Q; ++e) {
            const float pe = qe(pc, e), xm = e == 0 ? xl : qe(pc, e - 1), xp = e == Q - 1 ? xr : qe(pc, e + 1);
            qs(av, e, (cd[e] & RC_WET) ? apply_code_nb(g, cd[e], i0 + e, j, k, pe, xm, xp, qe(ym, e), qe(yp, e),
                                                       qe(zm, e), qe(zp, e))
                                       : 0.f);
          }
        }
        if (PASS == TP_DIR) {
          *reinterpret_cast<V*>(a.out0 + c) = pc;
          *reinterpret_cast<V*>(a.out1 + c) = av;
#pragma unroll
          for (int e = 0; e < Q; ++e) acc += (double)qe(pc, e) * (double)qe(av, e);
        } else if (PASS == TP_PRE || PASS == TP_POST1 || PASS == TP_POST2) {
          V m, r;
          if (PASS == TP_PRE) {
            m = *reinterpret_cast<const V*>(reinterpret_cast<const float*>(st) + hc);
            r = *reinterpret_cast<const V*>(reinterpret_cast<const float*>(st + tm_al(TM_HALO_BYTES)) + hc);
          } else if (PASS == TP_POST1) {
            m = *reinterpret_cast<const V*>(reinterpret_cast<const float*>(st + tm_al(TM_HALO_BYTES)) + hc);
            r = *reinterpret_cast<const V*>(reinterpret_cast<const float*>(st + P::OFF_O) + oc);
          } else {
            m = *reinterpret_cast<const V*>(reinterpret_cast<const float*>(st + P::OFF_O) + oc);
            r = *reinterpret_cast<const V*>(reinterpret_cast<const float*>(st + P::OFF_O + tm_al(TM_OWN_BYTES)) + oc);
          }
          V z;
#pragma unroll
          for (int e = 0; e < Q; ++e) {  // z + w m (r - A z) where m > 0 (the smoother's update, as a select)
            const float t = qe(pc, e) + OMEGA * qe(m, e) * (qe(r, e) - qe(av, e));
            qs(z, e, qe(m, e) > 0.f ? t : qe(pc, e));
          }
          *reinterpret_cast<V*>(a.out0 + c) = z;
          if (PASS == TP_POST2) {
#pragma unroll
            for (int e = 0; e < Q; ++e) acc += (double)qe(r, e) * (double)qe(z, e);
          }
        } else if (PASS == TP_RESID) {
          const V rh = *reinterpret_cast<const V*>(reinterpret_cast<const float*>(st + P::OFF_O) + oc);
          V rr;
#pragma unroll
          for (int e = 0; e < Q; ++e) {
            qs(rr, e, qe(rh, e) - qe(av, e));
            acc += (double)qe(rr, e) * (double)qe(rr, e);
          }
          *reinterpret_cast<V*>(a.out0 + c) = rr;
        } else {  // TP_RESTRICT: the residual at the thread's cells, into the layer's plane
          const V r = *reinterpret_cast<const V*>(reinterpret_cast<const float*>(st + P::OFF_O) + oc);
          V rr;
#pragma unroll
          for (int e = 0; e < Q; ++e) qs(rr, e, qe(r, e) - qe(av, e));
          *reinterpret_cast<V*>(tr + (k & 1) * TMY * TMX + oc) = rr;
        }
      }  // inside
      if (PASS == TP_RESTRICT && (k & 1)) {
        __syncthreads();  // both layers' residuals before the eight-child means (restrict3, CHILDREN order)
        if (inside && !(ty & 1)) {
#pragma unroll
          for (int h = 0; h < Q / 2; ++h) {  // the coarse cells (i0 / 2 + h, j / 2, k / 2)
            const float* t0 = tr + oc + 2 * h;
            const float* t1 = tr + TMY * TMX + oc + 2 * h;
            float sum = 0.f;
            sum += t0[0];
            sum += t0[1];
            sum += t0[TMX];
            sum += t0[TMX + 1];
            sum += t1[0];
            sum += t1[1];
            sum += t1[TMX];
            sum += t1[TMX + 1];
            a.L.r[((k >> 1) * a.L.ny + (j >> 1)) * a.L.nx + (i0 >> 1) + h] = 0.125f * sum;
          }
        }
      }
    }
    if (*abort_flag) {  // a wait ran out: drain this CTA's copies in flight, then fail the projection
      if (tid == ISSUER) {
        while (waited < issued && wait_next()) {
        }
        S->status = 2;
      }
      acc = __longlong_as_double(0x7ff8000000000000LL);  // and the reduction reports a non-finite value
    }
  }  // !skip
  if (PASS == TP_DIR) kt_reduce_finish(acc, red, S, FIN_DQ);
  if (PASS == TP_POST2 || PASS == TP_RESID) kt_reduce_finish(acc, red, S, a.op);
}

}  // namespace fd3
