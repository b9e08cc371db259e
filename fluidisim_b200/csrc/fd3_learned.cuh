// The learned preconditioner on the host side: the U-Net object (parameters, Adam state,
// activation buffers), its forward and backward passes over a batch, the device-side problem
// hooks a training loop needs (assembly, operator, residual loss), and the flexible conjugate
// gradient that uses the network as its preconditioner (fd3_project_learned).
//
// Included by fd3_volume.cu after the volume host code: it uses its launch helpers.
#pragma once

#include "fd3_conv_dw.cuh"
#include "fd3_conv_tc.cuh"
#include "fd3_conv_tp.cuh"
#include "fd3_unet.cuh"

using namespace fd3u;

// ------------------------------------------------------------------------------------ the network
struct UnetLayer {
  int cin, cout, cinp, coutp;  // logical and padded channel counts
  size_t w_off, b_off;         // offsets of w [27][cout][cin] and b [cout] in the master vector
  __nv_bfloat16 *w = nullptr, *wt = nullptr;  // forward and data-gradient working copies
  float *gw = nullptr, *gb = nullptr;         // padded gradient accumulators
  float* bias = nullptr;                      // padded f32 bias
};

enum { L_E0 = 0, L_E1, L_B, L_D1, L_D0, L_HEAD, L_COUNT };

struct fd3_unet {
  int device = 0;
  cudaStream_t stream = nullptr, own_stream = nullptr;
  long long cap = 0;  // full-resolution cells (batch included) the buffers hold
  UnetLayer layer[L_COUNT];
  size_t nparams = 0;
  float *master = nullptr, *grad = nullptr, *m = nullptr, *v = nullptr;
  float *in_scale = nullptr, *out_scale = nullptr;  // per-sample scales (device)
  int scale_cap = 0;
  long long adam_t = 0;
  // activations (bf16, channels-last)
  __nv_bfloat16 *x0, *e0, *p0, *e1, *p1, *bq, *c1, *d1, *c0, *d0;
  // gradients
  __nv_bfloat16 *gy, *gd0, *gc0, *gd1, *gc1, *gbq, *gp1, *ge1, *gp0, *ge0;
  Dims last{0, 0, 0, 0};
  std::vector<void*> allocations;
  unsigned long long launches = 0;
  int conv_tc = 1;        // 1: convolutions on tcgen05 (k_conv_tc), 0: on mma.sync (k_conv)
  int conv_tiles = TC_MAX_TILES;  // budget of 128-row M tiles per CTA of k_conv_tc (fewer: smaller CTAs)
  // how FCG uses the network: 0 = M(r) = the network's approximation of A^-1 r; 1 = M(r) = V(r) plus
  // the network's approximation of A^-1 (r - A V(r)), V the multigrid V-cycle
  int mode = 0;
  int* dflag = nullptr;   // set by k_conv_tc when a bounded wait ran out
};

namespace {

const int kLayerShape[L_COUNT][2] = {{3, 16}, {16, 32}, {32, 64}, {96, 32}, {48, 16}, {16, 1}};

inline int pad16(int c) { return (c + 15) / 16 * 16; }

template <class T>
int ualloc(fd3_unet* N, T** p, size_t count) {
  void* q = nullptr;
  CK(cudaMalloc(&q, std::max<size_t>(count, 1) * sizeof(T)));
  N->allocations.push_back(q);
  CK(cudaMemsetAsync(q, 0, std::max<size_t>(count, 1) * sizeof(T), N->stream));
  *p = (T*)q;
  return FD3_OK;
}

void unet_release(fd3_unet* N) {
  for (void* q : N->allocations) cudaFree(q);
  N->allocations.clear();
  if (N->own_stream) cudaStreamDestroy(N->own_stream);
}

inline int grid_for(long long n, int block = 256) {
  long long b = (n + block - 1) / block;
  return (int)std::max<long long>(1, std::min<long long>(b, 148LL * 32));
}

template <class K, class... A>
int ulaunch(fd3_unet* N, dim3 grid, int block, K kernel, A... args) {
  kernel<<<grid, block, 0, N->stream>>>(args...);
  N->launches++;
  CK(cudaGetLastError());
  return FD3_OK;
}

// k_conv_tc with its dynamic shared memory (the opt-in limit is raised once per instantiation).
template <int CI, int CO, int E>
int conv_tc_launch(fd3_unet* N, Dims d, const __nv_bfloat16* in, const __nv_bfloat16* w, const float* bias,
                   __nv_bfloat16* out, float* out32) {
  static unsigned attr_set = 0;  // devices on which the limit was raised
  const int BY = tc_rows(d.X, d.Y, N->conv_tiles), NTM = tc_tiles(d.X, BY);
  if (NTM > TC_MAX_TILES) return FD3_ERR_SHAPE;
  const size_t smem = tc_smem_bytes(d.X, BY, CO);
  if (smem > 227 * 1024) return FD3_ERR_SHAPE;
  if (N->device < 32 && !(attr_set & (1u << N->device))) {
    CK(cudaFuncSetAttribute(k_conv_tc<CI, CO, E>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024));
    attr_set |= 1u << N->device;
  }
  const long long grid = (long long)d.B * d.Z * ((d.Y + BY - 1) / BY);
  k_conv_tc<CI, CO, E><<<dim3((unsigned)grid), TC_THREADS, smem, N->stream>>>(d, BY, NTM, in, w, bias, out, out32,
                                                                             N->dflag);
  N->launches++;
  CK(cudaGetLastError());
  return FD3_OK;
}

// k_conv_tp: the pipelined tcgen05 convolution, persistent over the work tiles, one CTA per SM.
// The M-tile budget keeps two accumulators within the 512 columns of tensor memory and at least
// two stage slots within the shared memory; FD3_ERR_SHAPE, before anything is launched, when no
// budget does (the caller then runs k_conv_tc).
template <int CI, int CO, int E>
int conv_tp_launch(fd3_unet* N, Dims d, const __nv_bfloat16* in, const __nv_bfloat16* w, const float* bias,
                   __nv_bfloat16* out, float* out32) {
  static unsigned attr_set = 0;
  static int sms = 0;
  if (!sms) CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, N->device));
  const size_t budget = 227 * 1024 - TP_CTRL_BYTES;
  int tiles = std::min(N->conv_tiles, 256 / CO);
  int BY = 0, NTM = 0, S = 0;
  for (; tiles >= 1; --tiles) {
    BY = tc_rows(d.X, d.Y, tiles);
    NTM = tc_tiles(d.X, BY);
    if (NTM > TC_MAX_TILES || 2 * NTM * CO > 512) continue;
    S = (int)std::min<size_t>(TP_MAX_STAGES, budget / tp_stage_bytes(d.X, BY, CO));
    if (S >= 2) break;
  }
  if (tiles < 1) return FD3_ERR_SHAPE;
  if (N->device < 32 && !(attr_set & (1u << N->device))) {
    CK(cudaFuncSetAttribute(k_conv_tp<CI, CO, E>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024));
    attr_set |= 1u << N->device;
  }
  const long long W = (long long)d.B * d.Z * ((d.Y + BY - 1) / BY);
  const int grid = (int)std::min<long long>(W, sms);
  const size_t smem = TP_CTRL_BYTES + (size_t)S * tp_stage_bytes(d.X, BY, CO);
  k_conv_tp<CI, CO, E><<<dim3((unsigned)grid), TP_THREADS, smem, N->stream>>>(d, BY, NTM, S, (int)W, in, w, bias, out,
                                                                            out32, N->dflag);
  N->launches++;
  CK(cudaGetLastError());
  return FD3_OK;
}

// The convolution for the (CIN, COUT, epilogue) triples the network uses: k_conv_tp (tcgen05,
// pipelined; N->conv_tc 2), k_conv_tc (tcgen05, one phase at a time; 1) or k_conv (mma.sync; 0).
int conv_fwd(fd3_unet* N, Dims d, int cin, int cout, int epi, const __nv_bfloat16* in, const __nv_bfloat16* w,
             const float* bias, __nv_bfloat16* out, float* out32) {
  if (N->conv_tc) {
#define FD3_CONV_TC(CI, CO, E)                                                                          \
  if (cin == CI && cout == CO && epi == E) {                                                           \
    if (N->conv_tc == 2) {                                                                             \
      const int e_ = conv_tp_launch<CI, CO, E>(N, d, in, w, bias, out, out32);                         \
      if (e_ != FD3_ERR_SHAPE) return e_;                                                              \
    }                                                                                                  \
    return conv_tc_launch<CI, CO, E>(N, d, in, w, bias, out, out32);                                   \
  }
    FD3_CONV_TC(16, 16, EPI_BIAS_RELU)
    FD3_CONV_TC(16, 32, EPI_BIAS_RELU)
    FD3_CONV_TC(32, 64, EPI_BIAS_RELU)
    FD3_CONV_TC(96, 32, EPI_BIAS_RELU)
    FD3_CONV_TC(48, 16, EPI_BIAS_RELU)
    FD3_CONV_TC(16, 16, EPI_BIAS_F32_CH0)
    FD3_CONV_TC(16, 16, EPI_PLAIN)
    FD3_CONV_TC(16, 48, EPI_PLAIN)
    FD3_CONV_TC(32, 96, EPI_PLAIN)
    FD3_CONV_TC(64, 32, EPI_PLAIN)
    FD3_CONV_TC(32, 16, EPI_PLAIN)
#undef FD3_CONV_TC
    return FD3_ERR_INVALID_ARGUMENT;
  }
  const int grid = (int)((d.cells() + CONV_CELLS - 1) / CONV_CELLS);
#define FD3_CONV(CI, CO, E)                                                              \
  if (cin == CI && cout == CO && epi == E)                                               \
    return ulaunch(N, dim3(grid), CONV_THREADS, k_conv<CI, CO, E>, d, in, w, bias, out, out32);
  FD3_CONV(16, 16, EPI_BIAS_RELU)
  FD3_CONV(16, 32, EPI_BIAS_RELU)
  FD3_CONV(32, 64, EPI_BIAS_RELU)
  FD3_CONV(96, 32, EPI_BIAS_RELU)
  FD3_CONV(48, 16, EPI_BIAS_RELU)
  FD3_CONV(16, 16, EPI_BIAS_F32_CH0)
  FD3_CONV(16, 16, EPI_PLAIN)
  FD3_CONV(16, 48, EPI_PLAIN)
  FD3_CONV(32, 96, EPI_PLAIN)
  FD3_CONV(64, 32, EPI_PLAIN)
  FD3_CONV(32, 16, EPI_PLAIN)
#undef FD3_CONV
  return FD3_ERR_INVALID_ARGUMENT;
}

// k_conv_dw2 (all taps per CTA, persistent grid) with its dynamic shared memory.
template <int CI, int CO>
int conv_dw2_launch(fd3_unet* N, Dims d, const __nv_bfloat16* in, const __nv_bfloat16* gout, float* gw) {
  static unsigned attr_set = 0;  // devices on which the limit was raised
  const int BY = dw2_rows(d.X, d.Y);
  const size_t smem = dw2_smem_bytes(d.X, BY, CO);
  if (N->device < 32 && !(attr_set & (1u << N->device))) {
    CK(cudaFuncSetAttribute(k_conv_dw2<CI, CO>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024));
    attr_set |= 1u << N->device;
  }
  int sms = 148;
  CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, N->device));
  const long long nblk = (long long)d.B * d.Z * ((d.Y + BY - 1) / BY);
  const int grid = (int)std::min<long long>(nblk, sms);
  k_conv_dw2<CI, CO><<<grid, DW2_THREADS, smem, N->stream>>>(d, BY, in, gout, gw);
  N->launches++;
  CK(cudaGetLastError());
  return FD3_OK;
}

int conv_dw(fd3_unet* N, Dims d, int cin, int cout, const __nv_bfloat16* in, const __nv_bfloat16* gout, float* gw) {
  // the all-taps kernel where its staging fits shared memory (output channels 16 or 32)
  if (d.X <= 256 && (cout == 16 || cout == 32) && dw2_smem_bytes(d.X, dw2_rows(d.X, d.Y), cout) <= 227 * 1024) {
    if (cin == 16 && cout == 16) return conv_dw2_launch<16, 16>(N, d, in, gout, gw);
    if (cin == 48 && cout == 16) return conv_dw2_launch<48, 16>(N, d, in, gout, gw);
    if (cin == 96 && cout == 32) return conv_dw2_launch<96, 32>(N, d, in, gout, gw);
    if (cin == 16 && cout == 32) return conv_dw2_launch<16, 32>(N, d, in, gout, gw);
  }
  const long long cells = d.cells();
  long long slices = std::max<long long>(1, std::min<long long>(44, (cells + DW_ROWS - 1) / DW_ROWS));
  long long chunk = (cells + slices - 1) / slices;
  chunk = (chunk + DW_ROWS - 1) / DW_ROWS * DW_ROWS;
  slices = (cells + chunk - 1) / chunk;
#define FD3_DW(CI, CO) \
  if (cin == CI && cout == CO) return ulaunch(N, dim3(27, (unsigned)slices), DW_THREADS, k_conv_dw<CI, CO>, d, in, gout, gw, chunk);
  FD3_DW(16, 16)
  FD3_DW(16, 32)
  FD3_DW(32, 64)
  FD3_DW(96, 32)
  FD3_DW(48, 16)
#undef FD3_DW
  return FD3_ERR_INVALID_ARGUMENT;
}

int unet_pack(fd3_unet* N) {
  for (int l = 0; l < L_COUNT; ++l) {
    UnetLayer& L = N->layer[l];
    TRY(ulaunch(N, dim3(grid_for(27LL * L.coutp * L.cinp)), 256, k_pack, L.cin, L.cout, L.cinp, L.coutp,
                (const float*)(N->master + L.w_off), L.w, L.wt));
    CK(cudaMemsetAsync(L.bias, 0, L.coutp * sizeof(float), N->stream));
    CK(cudaMemcpyAsync(L.bias, N->master + L.b_off, L.cout * sizeof(float), cudaMemcpyDeviceToDevice, N->stream));
  }
  return FD3_OK;
}

// The error word of the tensor-core convolution (a bounded wait that ran out); read after a
// synchronisation of the network's stream, then cleared.
int unet_check_flag(fd3_unet* N) {
  int h = 0;
  CK(cudaMemcpy(&h, N->dflag, sizeof h, cudaMemcpyDeviceToHost));
  if (h) {
    CK(cudaMemset(N->dflag, 0, sizeof h));
    g_last_cuda_error = "k_conv_tc: a wait for the tensor-core MMAs ran out";
    return FD3_ERR_CUDA;
  }
  return FD3_OK;
}

int unet_check_dims(const fd3_unet* N, int B, int Z, int Y, int X) {
  if (B <= 0 || Z <= 0 || Y <= 0 || X <= 0 || Z % 4 || Y % 4 || X % 4 || X > 512) return FD3_ERR_SHAPE;
  if ((long long)B * Z * Y * X > N->cap || B > N->scale_cap) return FD3_ERR_SCRATCH_LIMIT;
  return FD3_OK;
}

// k_input / k_out_grad with a per-sample scale.
__global__ void k_input_scaled(long long cells, long long per, const float* __restrict__ x, const float* __restrict__ s,
                               __nv_bfloat16* __restrict__ out) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < cells; q += (long long)gridDim.x * blockDim.x) {
    __align__(16) __nv_bfloat16 v[16];
#pragma unroll
    for (int c = 0; c < 16; ++c) v[c] = __float2bfloat16(0.f);
    v[0] = __float2bfloat16(x[3 * q] * s[q / per]);
    v[1] = __float2bfloat16(x[3 * q + 1]);
    v[2] = __float2bfloat16(x[3 * q + 2]);
    uint4* o = reinterpret_cast<uint4*>(out + q * 16);
    o[0] = reinterpret_cast<const uint4*>(v)[0];
    o[1] = reinterpret_cast<const uint4*>(v)[1];
  }
}
__global__ void k_out_grad_scaled(long long cells, long long per, const float* __restrict__ g,
                                  const float* __restrict__ s, __nv_bfloat16* __restrict__ out) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < cells; q += (long long)gridDim.x * blockDim.x) {
    __align__(16) __nv_bfloat16 v[16];
#pragma unroll
    for (int c = 0; c < 16; ++c) v[c] = __float2bfloat16(0.f);
    v[0] = __float2bfloat16(g[q] * s[q / per]);
    uint4* o = reinterpret_cast<uint4*>(out + q * 16);
    o[0] = reinterpret_cast<const uint4*>(v)[0];
    o[1] = reinterpret_cast<const uint4*>(v)[1];
  }
}
__global__ void k_scale_out(long long cells, long long per, float* __restrict__ y, const float* __restrict__ s) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < cells; q += (long long)gridDim.x * blockDim.x)
    y[q] *= s[q / per];
}

int unet_forward(fd3_unet* N, int B, int Z, int Y, int X, const float* in3, float* out) {
  TRY(unet_check_dims(N, B, Z, Y, X));
  Dims d0{B, Z, Y, X}, d1{B, Z / 2, Y / 2, X / 2}, d2{B, Z / 4, Y / 4, X / 4};
  N->last = d0;
  const long long n0 = d0.cells(), n1 = d1.cells(), n2 = d2.cells();
  const long long per = (long long)Z * Y * X;
  UnetLayer* L = N->layer;
  TRY(ulaunch(N, dim3(grid_for(n0)), 256, k_input_scaled, n0, per, in3, (const float*)N->in_scale, N->x0));
  TRY(conv_fwd(N, d0, 16, 16, EPI_BIAS_RELU, N->x0, L[L_E0].w, L[L_E0].bias, N->e0, nullptr));
  TRY(ulaunch(N, dim3(grid_for(n1 * 2)), 256, k_pool, d1, 16, (const __nv_bfloat16*)N->e0, N->p0));
  TRY(conv_fwd(N, d1, 16, 32, EPI_BIAS_RELU, N->p0, L[L_E1].w, L[L_E1].bias, N->e1, nullptr));
  TRY(ulaunch(N, dim3(grid_for(n2 * 4)), 256, k_pool, d2, 32, (const __nv_bfloat16*)N->e1, N->p1));
  TRY(conv_fwd(N, d2, 32, 64, EPI_BIAS_RELU, N->p1, L[L_B].w, L[L_B].bias, N->bq, nullptr));
  TRY(ulaunch(N, dim3(grid_for(n1 * 12)), 256, k_up_cat, d1, 64, 32, (const __nv_bfloat16*)N->bq,
              (const __nv_bfloat16*)N->e1, N->c1));
  TRY(conv_fwd(N, d1, 96, 32, EPI_BIAS_RELU, N->c1, L[L_D1].w, L[L_D1].bias, N->d1, nullptr));
  TRY(ulaunch(N, dim3(grid_for(n0 * 6)), 256, k_up_cat, d0, 32, 16, (const __nv_bfloat16*)N->d1,
              (const __nv_bfloat16*)N->e0, N->c0));
  TRY(conv_fwd(N, d0, 48, 16, EPI_BIAS_RELU, N->c0, L[L_D0].w, L[L_D0].bias, N->d0, nullptr));
  TRY(conv_fwd(N, d0, 16, 16, EPI_BIAS_F32_CH0, N->d0, L[L_HEAD].w, L[L_HEAD].bias, nullptr, out));
  TRY(ulaunch(N, dim3(grid_for(n0)), 256, k_scale_out, n0, per, out, (const float*)N->out_scale));
  return FD3_OK;
}

int unet_backward(fd3_unet* N, const float* gout) {
  const Dims d0 = N->last;
  if (d0.B == 0) return FD3_ERR_DOMAIN;
  Dims d1{d0.B, d0.Z / 2, d0.Y / 2, d0.X / 2}, d2{d0.B, d0.Z / 4, d0.Y / 4, d0.X / 4};
  const long long n0 = d0.cells(), n1 = d1.cells(), n2 = d2.cells();
  const long long per = (long long)d0.Z * d0.Y * d0.X;
  UnetLayer* L = N->layer;
  auto bias_grad = [&](long long cells, int C, const __nv_bfloat16* g, float* gb) {
    return ulaunch(N, dim3(std::min<long long>(256, (cells + 255) / 256), C / 8), 256, k_bias_grad, cells, C, g, gb);
  };
  // head
  TRY(ulaunch(N, dim3(grid_for(n0)), 256, k_out_grad_scaled, n0, per, gout, (const float*)N->out_scale, N->gy));
  TRY(conv_dw(N, d0, 16, 16, N->d0, N->gy, L[L_HEAD].gw));
  TRY(bias_grad(n0, 16, N->gy, L[L_HEAD].gb));
  TRY(conv_fwd(N, d0, 16, 16, EPI_PLAIN, N->gy, L[L_HEAD].wt, nullptr, N->gd0, nullptr));
  TRY(ulaunch(N, dim3(grid_for(n0 * 16)), 256, k_relu_mask, n0 * 16, N->gd0, (const __nv_bfloat16*)N->d0));
  // d0: input c0 = cat(up(d1), e0)
  TRY(conv_dw(N, d0, 48, 16, N->c0, N->gd0, L[L_D0].gw));
  TRY(bias_grad(n0, 16, N->gd0, L[L_D0].gb));
  TRY(conv_fwd(N, d0, 16, 48, EPI_PLAIN, N->gd0, L[L_D0].wt, nullptr, N->gc0, nullptr));
  TRY(ulaunch(N, dim3(grid_for(n1 * 4)), 256, k_up_bwd, d1, 48, 32, (const __nv_bfloat16*)N->gc0,
              (const __nv_bfloat16*)N->d1, N->gd1));
  // d1: input c1 = cat(up(b), e1)
  TRY(conv_dw(N, d1, 96, 32, N->c1, N->gd1, L[L_D1].gw));
  TRY(bias_grad(n1, 32, N->gd1, L[L_D1].gb));
  TRY(conv_fwd(N, d1, 32, 96, EPI_PLAIN, N->gd1, L[L_D1].wt, nullptr, N->gc1, nullptr));
  TRY(ulaunch(N, dim3(grid_for(n2 * 8)), 256, k_up_bwd, d2, 96, 64, (const __nv_bfloat16*)N->gc1,
              (const __nv_bfloat16*)N->bq, N->gbq));
  // b: input p1 = pool(e1)
  TRY(conv_dw(N, d2, 32, 64, N->p1, N->gbq, L[L_B].gw));
  TRY(bias_grad(n2, 64, N->gbq, L[L_B].gb));
  TRY(conv_fwd(N, d2, 64, 32, EPI_PLAIN, N->gbq, L[L_B].wt, nullptr, N->gp1, nullptr));
  TRY(ulaunch(N, dim3(grid_for(n1 * 4)), 256, k_enc_grad, d1, 32, (const __nv_bfloat16*)N->gc1, 96, 64,
              (const __nv_bfloat16*)N->gp1, (const __nv_bfloat16*)N->e1, N->ge1));
  // e1: input p0 = pool(e0)
  TRY(conv_dw(N, d1, 16, 32, N->p0, N->ge1, L[L_E1].gw));
  TRY(bias_grad(n1, 32, N->ge1, L[L_E1].gb));
  TRY(conv_fwd(N, d1, 32, 16, EPI_PLAIN, N->ge1, L[L_E1].wt, nullptr, N->gp0, nullptr));
  TRY(ulaunch(N, dim3(grid_for(n0 * 2)), 256, k_enc_grad, d0, 16, (const __nv_bfloat16*)N->gc0, 48, 32,
              (const __nv_bfloat16*)N->gp0, (const __nv_bfloat16*)N->e0, N->ge0));
  // e0: input x0
  TRY(conv_dw(N, d0, 16, 16, N->x0, N->ge0, L[L_E0].gw));
  TRY(bias_grad(n0, 16, N->ge0, L[L_E0].gb));
  return FD3_OK;
}

// The padded accumulators into the master-layout gradient (then cleared).
int unet_collect(fd3_unet* N) {
  for (int l = 0; l < L_COUNT; ++l) {
    UnetLayer& L = N->layer[l];
    TRY(ulaunch(N, dim3(grid_for(27LL * L.cout * L.cin)), 256, k_unpack_grad, L.cin, L.cout, L.cinp, L.coutp,
                (const float*)L.gw, N->grad + L.w_off));
    TRY(ulaunch(N, dim3(1), 64, k_unpack_grad_bias, L.cout, (const float*)L.gb, N->grad + L.b_off));
    CK(cudaMemsetAsync(L.gw, 0, 27ULL * L.coutp * L.cinp * sizeof(float), N->stream));
    CK(cudaMemsetAsync(L.gb, 0, L.coutp * sizeof(float), N->stream));
  }
  return FD3_OK;
}

}  // namespace

// ------------------------------------------------------------------------ FCG with the network
namespace {

// Block sum of a double, one atomicAdd per block.
// Called by every thread of the block; may be called several times in a row.
__device__ __forceinline__ void block_add(double v, double* out) {
  __shared__ double sh[32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  __syncthreads();  // the previous call's readers are done with sh
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x < 32) {
    v = threadIdx.x < (blockDim.x >> 5) ? sh[threadIdx.x] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (threadIdx.x == 0) atomicAdd(out, v);
  }
}

// q = A d (row codes), with d.q and d.r.
__global__ void k_fcg_apply(Geo g, const unsigned short* __restrict__ codes, const float* __restrict__ d,
                            const float* __restrict__ r, float* __restrict__ q, double* dots) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  double dq = 0.0, dr = 0.0;
  if (c < g.n) {
    const unsigned code = codes[c];
    float a = 0.f;
    if (code & RC_WET) { int i, j, k; cell_ijk(g, c, i, j, k); a = apply_code(g, code, i, j, k, c, Load{d}); }
    q[c] = a;
    dq = (double)d[c] * (double)a;
    dr = (double)d[c] * (double)r[c];
  }
  block_add(dq, dots + 0);
  block_add(dr, dots + 1);
}

// p += alpha d, r -= alpha q, r.r
__global__ void k_fcg_update(int n, float alpha, const float* __restrict__ d, const float* __restrict__ q,
                             float* __restrict__ p, float* __restrict__ r, double* dots) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  double rr = 0.0;
  if (c < n) {
    p[c] += alpha * d[c];
    const float rn = r[c] - alpha * q[c];
    r[c] = rn;
    rr = (double)rn * (double)rn;
  }
  block_add(rr, dots + 2);
}

// The network input from a residual: (r, solid, liquid) per cell; solid = cut fraction 0,
// liquid = a wet row; and r.r for the input scale.
__global__ void k_fcg_input(Geo g, const unsigned short* __restrict__ codes, const float* __restrict__ r,
                            float* __restrict__ in3, double* dots) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  double rr = 0.0;
  if (c < g.n) {
    const float rc = r[c];
    in3[3 * c] = rc;
    in3[3 * c + 1] = solid3(g, c) ? 1.f : 0.f;
    in3[3 * c + 2] = (codes[c] & RC_WET) ? 1.f : 0.f;
    rr = (double)rc * (double)rc;
  }
  block_add(rr, dots + 3);
}

// z = 0 on dry rows, then z.q (the flexible beta's numerator) and z.r.
__global__ void k_fcg_zdots(int n, const unsigned short* __restrict__ codes, float* __restrict__ z,
                            const float* __restrict__ q, const float* __restrict__ r, double* dots) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  double zq = 0.0, zr = 0.0;
  if (c < n) {
    float zc = (codes[c] & RC_WET) ? z[c] : 0.f;
    z[c] = zc;
    zq = (double)zc * (double)q[c];
    zr = (double)zc * (double)r[c];
  }
  block_add(zq, dots + 4);
  block_add(zr, dots + 5);
}

// rho = r - A z on the wet rows (the residual a V-cycle z = V(r) leaves), |rho|^2 into dots[3].
__global__ void k_vres(Geo g, const unsigned short* __restrict__ codes, const float* __restrict__ r,
                       const float* __restrict__ z, float* __restrict__ rho, double* dots) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  double rr = 0.0;
  if (c < g.n) {
    const unsigned code = codes[c];
    float v = 0.f;
    if (code & RC_WET) {
      int i, j, k;
      cell_ijk(g, c, i, j, k);
      v = r[c] - apply_code(g, code, i, j, k, c, Load{z});
    }
    rho[c] = v;
    rr = (double)v * (double)v;
  }
  block_add(rr, dots + 3);
}

// The hybrid preconditioner's output: z = y + z_mg on the wet rows (0 elsewhere), then z.q and z.r.
__global__ void k_fcg_zdots_add(int n, const unsigned short* __restrict__ codes, float* __restrict__ z,
                                const float* __restrict__ zmg, const float* __restrict__ q,
                                const float* __restrict__ r, double* dots) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  double zq = 0.0, zr = 0.0;
  if (c < n) {
    float zc = (codes[c] & RC_WET) ? z[c] + zmg[c] : 0.f;
    z[c] = zc;
    zq = (double)zc * (double)q[c];
    zr = (double)zc * (double)r[c];
  }
  block_add(zq, dots + 4);
  block_add(zr, dots + 5);
}

// d = z + beta d
__global__ void k_fcg_dir(int n, float beta, const float* __restrict__ z, float* __restrict__ d) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c < n) d[c] = beta == 0.f ? z[c] : z[c] + beta * d[c];
}

}  // namespace

// ---------------------------------------------------------------------------------- C ABI
extern "C" {

int fd3_unet_create(int max_batch, int nz, int ny, int nx, fd3_unet** out) {
  if (!out || max_batch <= 0 || nz <= 0 || ny <= 0 || nx <= 0 || nz % 4 || ny % 4 || nx % 4)
    return FD3_ERR_INVALID_ARGUMENT;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return FD3_ERR_NO_DEVICE;
  fd3_unet* N = new (std::nothrow) fd3_unet();
  if (!N) return FD3_ERR_OUT_OF_MEMORY;
  cudaGetDevice(&N->device);
  if (cudaStreamCreateWithFlags(&N->own_stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete N;
    return cuda_fail(cudaGetLastError(), "cudaStreamCreateWithFlags", __LINE__);
  }
  N->stream = N->own_stream;
  N->cap = (long long)max_batch * nz * ny * nx;
  N->scale_cap = max_batch;
  size_t off = 0;
  for (int l = 0; l < L_COUNT; ++l) {
    UnetLayer& L = N->layer[l];
    L.cin = kLayerShape[l][0];
    L.cout = kLayerShape[l][1];
    L.cinp = pad16(L.cin);
    L.coutp = pad16(L.cout);
    L.w_off = off;
    off += 27ULL * L.cout * L.cin;
    L.b_off = off;
    off += L.cout;
  }
  N->nparams = off;
  auto fail = [&](int e) { unet_release(N); delete N; return e; };
  int e;
#define UA(p, n) if ((e = ualloc(N, &(p), (n)))) return fail(e)
  UA(N->master, off); UA(N->grad, off); UA(N->m, off); UA(N->v, off);
  UA(N->in_scale, max_batch); UA(N->out_scale, max_batch);
  for (int l = 0; l < L_COUNT; ++l) {
    UnetLayer& L = N->layer[l];
    const size_t nw = 27ULL * L.coutp * L.cinp;
    UA(L.w, nw); UA(L.wt, nw); UA(L.gw, nw); UA(L.gb, L.coutp); UA(L.bias, L.coutp);
  }
  const long long n0 = N->cap, n1 = n0 / 8, n2 = n0 / 64;
  UA(N->x0, n0 * 16); UA(N->e0, n0 * 16); UA(N->p0, n1 * 16); UA(N->e1, n1 * 32); UA(N->p1, n2 * 32);
  UA(N->bq, n2 * 64); UA(N->c1, n1 * 96); UA(N->d1, n1 * 32); UA(N->c0, n0 * 48); UA(N->d0, n0 * 16);
  UA(N->gy, n0 * 16); UA(N->gd0, n0 * 16); UA(N->gc0, n0 * 48); UA(N->gd1, n1 * 32); UA(N->gc1, n1 * 96);
  UA(N->gbq, n2 * 64); UA(N->gp1, n2 * 32); UA(N->ge1, n1 * 32); UA(N->gp0, n1 * 16); UA(N->ge0, n0 * 16);
  UA(N->dflag, 1);
#undef UA
  if (cudaStreamSynchronize(N->stream) != cudaSuccess) return fail(cuda_fail(cudaGetLastError(), "create", __LINE__));
  *out = N;
  return FD3_OK;
}

void fd3_unet_destroy(fd3_unet* N) {
  if (!N) return;
  cudaStreamSynchronize(N->stream);
  unet_release(N);
  delete N;
}

int fd3_unet_set_stream(fd3_unet* N, void* stream) {
  if (!N) return FD3_ERR_INVALID_ARGUMENT;
  N->stream = stream ? (cudaStream_t)stream : N->own_stream;
  return FD3_OK;
}

uint64_t fd3_unet_param_count(const fd3_unet* N) { return N ? N->nparams : 0; }

int fd3_unet_set_params(fd3_unet* N, const float* params, size_t len) {
  if (!N || !params) return FD3_ERR_INVALID_ARGUMENT;
  if (len != N->nparams) return FD3_ERR_SHAPE;
  for (size_t q = 0; q < len; ++q)
    if (!std::isfinite(params[q])) return FD3_ERR_NOT_FINITE;
  CK(cudaMemcpyAsync(N->master, params, len * sizeof(float), cudaMemcpyHostToDevice, N->stream));
  CK(cudaMemsetAsync(N->m, 0, len * sizeof(float), N->stream));
  CK(cudaMemsetAsync(N->v, 0, len * sizeof(float), N->stream));
  N->adam_t = 0;
  TRY(unet_pack(N));
  CK(cudaStreamSynchronize(N->stream));
  return FD3_OK;
}

int fd3_unet_get_params(const fd3_unet* N, float* params, size_t len) {
  if (!N || !params) return FD3_ERR_INVALID_ARGUMENT;
  if (len != N->nparams) return FD3_ERR_SHAPE;
  CK(cudaMemcpyAsync(params, N->master, len * sizeof(float), cudaMemcpyDeviceToHost, N->stream));
  CK(cudaStreamSynchronize(N->stream));
  return FD3_OK;
}

int fd3_unet_get_grads(fd3_unet* N, float* grads, size_t len) {
  if (!N || !grads) return FD3_ERR_INVALID_ARGUMENT;
  if (len != N->nparams) return FD3_ERR_SHAPE;
  TRY(unet_collect(N));
  CK(cudaMemcpyAsync(grads, N->grad, len * sizeof(float), cudaMemcpyDeviceToHost, N->stream));
  CK(cudaMemsetAsync(N->grad, 0, len * sizeof(float), N->stream));
  CK(cudaStreamSynchronize(N->stream));
  return FD3_OK;
}

// y[b] = out_scale[b] * net(x with channel 0 times in_scale[b]); device pointers, x [B*cells][3],
// y [B*cells]; the scales are host arrays of B values.  Stream-ordered (no synchronisation).
int fd3_unet_forward(fd3_unet* N, int B, int nz, int ny, int nx, const float* d_in, const float* in_scale,
                     const float* out_scale, float* d_out) {
  if (!N || !d_in || !d_out || !in_scale || !out_scale) return FD3_ERR_INVALID_ARGUMENT;
  TRY(unet_check_dims(N, B, nz, ny, nx));
  CK(cudaMemcpyAsync(N->in_scale, in_scale, B * sizeof(float), cudaMemcpyHostToDevice, N->stream));
  CK(cudaMemcpyAsync(N->out_scale, out_scale, B * sizeof(float), cudaMemcpyHostToDevice, N->stream));
  return unet_forward(N, B, nz, ny, nx, d_in, d_out);
}

// Accumulates the parameter gradients of the last forward for dL/dy = d_gout (device, [B*cells]).
int fd3_unet_backward(fd3_unet* N, const float* d_gout) {
  if (!N || !d_gout) return FD3_ERR_INVALID_ARGUMENT;
  return unet_backward(N, d_gout);
}

// Adam step on the accumulated gradient (which it consumes), then the working copies.
int fd3_unet_adam(fd3_unet* N, float lr, float beta1, float beta2, float eps) {
  if (!N) return FD3_ERR_INVALID_ARGUMENT;
  TRY(unet_collect(N));
  N->adam_t += 1;
  const float c1 = 1.f - std::pow(beta1, (float)N->adam_t), c2 = 1.f - std::pow(beta2, (float)N->adam_t);
  TRY(ulaunch(N, dim3(grid_for((long long)N->nparams)), 256, k_adam, (int)N->nparams, N->master, N->grad, N->m, N->v,
              lr, beta1, beta2, eps, c1, c2));
  return unet_pack(N);
}

int fd3_unet_sync(fd3_unet* N) {
  if (!N) return FD3_ERR_INVALID_ARGUMENT;
  CK(cudaStreamSynchronize(N->stream));
  return unet_check_flag(N);
}

int fd3_unet_set_conv_kernels(fd3_unet* N, int tc) {
  if (!N || tc < 0 || tc > 2) return FD3_ERR_INVALID_ARGUMENT;
  N->conv_tc = tc;
  return FD3_OK;
}

int fd3_unet_set_conv_tiles(fd3_unet* N, int tiles) {
  if (!N || tiles < 1 || tiles > TC_MAX_TILES) return FD3_ERR_INVALID_ARGUMENT;
  N->conv_tiles = tiles;
  return FD3_OK;
}

uint64_t fd3_unet_kernel_launches(const fd3_unet* N) { return N ? N->launches : 0; }

}  // extern "C"

// --------------------------------------------------- problem hooks and the learned projection
namespace {

// out = A x from the row codes of the last assembly.
__global__ void k_apply_codes(Geo g, const unsigned short* __restrict__ codes, const float* __restrict__ x,
                              float* __restrict__ out, float scale) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= g.n) return;
  const unsigned code = codes[c];
  float a = 0.f;
  if (code & RC_WET) { int i, j, k; cell_ijk(g, c, i, j, k); a = apply_code(g, code, i, j, k, c, Load{x}); }
  out[c] = scale * a;
}

// t = A z - b and t.t
__global__ void k_residual_t(Geo g, const unsigned short* __restrict__ codes, const float* __restrict__ z,
                             const float* __restrict__ b, float* __restrict__ t, double* dots) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  double tt = 0.0;
  if (c < g.n) {
    const unsigned code = codes[c];
    float a = 0.f;
    if (code & RC_WET) { int i, j, k; cell_ijk(g, c, i, j, k); a = apply_code(g, code, i, j, k, c, Load{z}); }
    const float tv = a - b[c];
    t[c] = tv;
    tt = (double)tv * (double)tv;
  }
  block_add(tt, dots + 6);
}

int pull_dots(fd3_volume* V) {
  CK(cudaMemcpyAsync(V->hfsc, V->fsc, 8 * sizeof(double), cudaMemcpyDeviceToHost, V->stream));
  return sync(V);
}

// The rhs (with b.b in S->b2) and row codes of project_mobile3 for the current velocity (us = u),
// without solving.
int assemble_device(fd3_volume* V, float scale) {
  Geo G = V->geo();
  CK(cudaMemcpyAsync(V->us, V->u, (size_t)V->nu * 4, cudaMemcpyDeviceToDevice, V->stream));
  CK(cudaMemcpyAsync(V->vs, V->v, (size_t)V->nv * 4, cudaMemcpyDeviceToDevice, V->stream));
  CK(cudaMemcpyAsync(V->ws, V->w, (size_t)V->nw * 4, cudaMemcpyDeviceToDevice, V->stream));
  LAUNCH_G(V, k_reset_scalars, 1, 1, V->dS, vscale_k(V));
  LAUNCH(V, k_divergence, V->n, G, (const float*)V->us, (const float*)V->vs, (const float*)V->ws, V->rhs);
  DISPATCH(V, k_rhs_b2, V->n, G, scale, V->rhs, V->prec, V->red(), V->dS, 1, V->codes, (float*)nullptr);
  return FD3_OK;
}

// FCG(1) (Notay, "Flexible conjugate gradients", SIAM J. Sci. Comput. 22, 2000) from the current
// p, the network as the preconditioner: alpha = d.r / d.q, beta = -z.q / d.q.  Stops at the
// reference's tolerance (|r|^2 <= 1e-12 |b|^2), after max_fcg iterations, or when the residual
// stalls (|r_k|^2 > stall * |r_(k-4)|^2); the caller's project_mobile3 then finishes (or takes
// over) from the p it leaves.
int fcg(fd3_volume* V, fd3_unet* N, uint32_t max_fcg, double stall, uint32_t* iters, int* stalled) {
  Geo G = V->geo();
  const unsigned short* codes = V->codes;
  TRY(pull(V));
  const double b2 = V->hS->b2;
  double rr = V->hS->rr;
  *iters = 0;
  *stalled = 0;
  if (!(b2 > 0) || rr <= 1e-12 * b2) return FD3_OK;
  const float dx2 = V->dx * V->dx;
  std::vector<double> hist;
  double dq_prev = 0;
  cudaStream_t net_stream = N->stream;
  N->stream = V->stream;
  const bool hybrid = N->mode == 1;
  auto precondition = [&](double rnorm2) -> int {
    CK(cudaMemsetAsync(V->fsc, 0, 8 * sizeof(double), V->stream));
    const float* net_in = V->res;
    if (hybrid) {  // z_mg = V(r) in V->z, then the network sees the residual it leaves
      vcycle(V, 0, FIN_RZ_PRIME);
      LAUNCH(V, k_vres, V->n, G, codes, (const float*)V->res, (const float*)V->z, V->fz, V->fsc);
      TRY(pull_dots(V));
      rnorm2 = V->hfsc[3];
      CK(cudaMemsetAsync(V->fsc, 0, 8 * sizeof(double), V->stream));
      net_in = V->fz;
    }
    LAUNCH(V, k_fcg_input, V->n, G, codes, net_in, V->fin, V->fsc);
    const float s = (float)std::sqrt(std::max(rnorm2, 1e-300) / (double)V->n);
    const float inv = 1.f / s, outs = s * dx2;
    TRY(fd3_unet_forward(N, 1, V->nz, V->ny, V->nx, V->fin, &inv, &outs, V->fz));
    if (hybrid)
      LAUNCH(V, k_fcg_zdots_add, V->n, V->n, codes, V->fz, (const float*)V->z, (const float*)V->tmp,
             (const float*)V->res, V->fsc);
    else
      LAUNCH(V, k_fcg_zdots, V->n, V->n, codes, V->fz, (const float*)V->tmp, (const float*)V->res, V->fsc);
    return FD3_OK;
  };
  int e = [&]() -> int {
    TRY(precondition(rr));
    LAUNCH(V, k_fcg_dir, V->n, V->n, 0.f, (const float*)V->fz, V->dir);
    for (;;) {
      CK(cudaMemsetAsync(V->fsc, 0, 8 * sizeof(double), V->stream));
      LAUNCH(V, k_fcg_apply, V->n, G, codes, (const float*)V->dir, (const float*)V->res, V->tmp, V->fsc);
      TRY(pull_dots(V));
      const double dq = V->hfsc[0], dr = V->hfsc[1];
      if (!(dq > 0) || !std::isfinite(dr)) { *stalled = 1; return FD3_OK; }
      const float alpha = (float)(dr / dq);
      CK(cudaMemsetAsync(V->fsc, 0, 8 * sizeof(double), V->stream));
      LAUNCH(V, k_fcg_update, V->n, V->n, alpha, (const float*)V->dir, (const float*)V->tmp, V->p, V->res, V->fsc);
      TRY(pull_dots(V));
      rr = V->hfsc[2];
      *iters += 1;
      hist.push_back(rr);
      if (!std::isfinite(rr)) { *stalled = 1; return FD3_OK; }
      if (rr <= 1e-12 * b2) return FD3_OK;
      if (hist.size() > 4 && rr > stall * hist[hist.size() - 5]) { *stalled = 1; return FD3_OK; }
      if (*iters >= max_fcg) { *stalled = 1; return FD3_OK; }
      dq_prev = dq;
      TRY(precondition(rr));
      TRY(pull_dots(V));
      const double zq = V->hfsc[4];
      const float beta = (float)(-zq / dq_prev);
      LAUNCH(V, k_fcg_dir, V->n, V->n, beta, (const float*)V->fz, V->dir);
    }
  }();
  N->stream = net_stream;
  return e;
}

int attach_learned(fd3_volume* V) {
  if (V->fz) return FD3_OK;
  TRY(dalloc(V, &V->fz, V->n));
  TRY(dalloc(V, &V->fin, (size_t)V->n * 3));
  return FD3_OK;
}

}  // namespace

extern "C" {

int fd3_assemble_device(fd3_volume* V, float scale) {
  if (!V) return FD3_ERR_INVALID_ARGUMENT;
  TRY(assemble_device(V, scale));
  return sync(V);
}

int fd3_problem_device(fd3_volume* V, float** d_rhs, const unsigned short** d_codes) {
  if (!V) return FD3_ERR_INVALID_ARGUMENT;
  if (d_rhs) *d_rhs = V->rhs;
  if (d_codes) *d_codes = V->codes;
  return FD3_OK;
}

int fd3_apply_device(fd3_volume* V, const float* d_x, float* d_out) {
  if (!V || !d_x || !d_out) return FD3_ERR_INVALID_ARGUMENT;
  LAUNCH(V, k_apply_codes, V->n, V->geo(), (const unsigned short*)V->codes, d_x, d_out, 1.f);
  return sync(V);
}

int fd3_unet_set_mode(fd3_unet* N, int mode) {
  if (!N || mode < 0 || mode > 1) return FD3_ERR_INVALID_ARGUMENT;
  N->mode = mode;
  return FD3_OK;
}

int fd3_vcycle_residual_device(fd3_volume* V, const float* d_r, float* d_rho, double* rho2) {
  if (!V || !d_r || !d_rho) return FD3_ERR_INVALID_ARGUMENT;
  if (!V->has_mg || V->levels.empty()) return FD3_ERR_DOMAIN;
  prepare_multigrid(V);
  CK(cudaMemcpyAsync(V->res, d_r, (size_t)V->n * 4, cudaMemcpyDeviceToDevice, V->stream));
  vcycle(V, 0, FIN_RZ_PRIME);
  CK(cudaMemsetAsync(V->fsc, 0, 8 * sizeof(double), V->stream));
  LAUNCH(V, k_vres, V->n, V->geo(), (const unsigned short*)V->codes, (const float*)V->res, (const float*)V->z, d_rho,
         V->fsc);
  TRY(pull_dots(V));
  if (rho2) *rho2 = V->hfsc[3];
  return FD3_OK;
}

int fd3_learned_input(fd3_volume* V, const float* d_r, float* d_in3, double* rr) {
  if (!V || !d_r || !d_in3) return FD3_ERR_INVALID_ARGUMENT;
  CK(cudaMemsetAsync(V->fsc, 0, 8 * sizeof(double), V->stream));
  LAUNCH(V, k_fcg_input, V->n, V->geo(), (const unsigned short*)V->codes, d_r, d_in3, V->fsc);
  TRY(pull_dots(V));
  if (rr) *rr = V->hfsc[3];
  return FD3_OK;
}

// loss = weight |A z - b|^2 and d_grad = 2 weight A (A z - b), from the last assembly's rows.
int fd3_residual_loss(fd3_volume* V, const float* d_z, const float* d_b, float weight, float* d_grad, double* loss) {
  if (!V || !d_z || !d_b || !d_grad) return FD3_ERR_INVALID_ARGUMENT;
  Geo G = V->geo();
  CK(cudaMemsetAsync(V->fsc, 0, 8 * sizeof(double), V->stream));
  LAUNCH(V, k_residual_t, V->n, G, (const unsigned short*)V->codes, d_z, d_b, V->tmp, V->fsc);
  LAUNCH(V, k_apply_codes, V->n, G, (const unsigned short*)V->codes, (const float*)V->tmp, d_grad, 2.f * weight);
  TRY(pull_dots(V));
  if (loss) *loss = (double)weight * V->hfsc[6];
  return FD3_OK;
}

// project_mobile3 with the learned FCG in front: FCG from the current p with the network as the
// preconditioner, then the reference's acceptance loop, whose multigrid-PCG takes over when FCG
// stalled (and does nothing more than the checks when FCG reached the tolerance).
int fd3_project_learned(fd3_volume* V, fd3_unet* N, float scale, float k1, uint32_t max_iters, uint32_t max_fcg,
                        fd3_report* rep, uint32_t* fcg_iterations, int* fell_back) {
  if (!V || !N || !rep) return FD3_ERR_INVALID_ARGUMENT;
  if (V->nz % 4 || V->ny % 4 || V->nx % 4) return FD3_ERR_SHAPE;
  if ((long long)V->n > N->cap) return FD3_ERR_SCRATCH_LIMIT;
  TRY(attach_learned(V));
  CK(cudaMemcpyAsync(V->sv_p, V->p, (size_t)V->n * 4, cudaMemcpyDeviceToDevice, V->stream));
  TRY(assemble_device(V, scale));
  if (N->mode == 1) {
    if (!V->has_mg || V->levels.empty()) return FD3_ERR_DOMAIN;
    prepare_multigrid(V);
  }
  Geo G = V->geo();
  LAUNCH(V, k_zero_dry, V->n, G, V->p);
  residual(V, (int)FIN_RR0);
  uint32_t it = 0;
  int stalled = 0;
  int e = fcg(V, N, max_fcg, 0.5, &it, &stalled);
  // A stalled FCG iterate is discarded: plain MGPCG, the fallback, starts from the pressure the call
  // started with.  (Measured: continuing from the stalled iterate saved a few multigrid iterations
  // on 64^3 lakes like the training set, but cost 16 more at 256^3.)
  if (!e && stalled)
    if (cudaMemcpyAsync(V->p, V->sv_p, (size_t)V->n * 4, cudaMemcpyDeviceToDevice, V->stream) != cudaSuccess)
      e = cuda_fail(cudaGetLastError(), "restore p", __LINE__);
  if (!e) e = project_mobile3(V, scale, k1, max_iters, rep);
  if (e) {
    cudaMemcpyAsync(V->u, V->us, (size_t)V->nu * 4, cudaMemcpyDeviceToDevice, V->stream);
    cudaMemcpyAsync(V->v, V->vs, (size_t)V->nv * 4, cudaMemcpyDeviceToDevice, V->stream);
    cudaMemcpyAsync(V->w, V->ws, (size_t)V->nw * 4, cudaMemcpyDeviceToDevice, V->stream);
    cudaMemcpyAsync(V->p, V->sv_p, (size_t)V->n * 4, cudaMemcpyDeviceToDevice, V->stream);
    cudaStreamSynchronize(V->stream);
    return e;
  }
  if (fcg_iterations) *fcg_iterations = it;
  if (fell_back) *fell_back = rep->iterations > 0 ? 1 : 0;
  return FD3_OK;
}

}  // extern "C"
