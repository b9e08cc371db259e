// Host driver and C ABI of the delta (δ) pressure projection on B200.
//
// The driver mirrors water-core's `Volume3` (code/water-core/src/delta3d.rs, delta3d_mobile.rs,
// delta3d_multigrid.rs): the same entry points, error codes and atomic refusals.  All arithmetic
// on fields runs in the kernels of fd3_kernels.cuh / fd3_cut.cuh; the host only sequences launches
// and reads back a few scalars (the reference's outer acceptance loop, delta3d_mobile.rs:513-588).
// Scalars of the inner PCG loop (alpha, beta, the loop condition) live on the device, so an
// iteration is a fixed launch sequence that can be replayed from a CUDA graph.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstddef>
#include <cstdio>
#include <cstring>
#include <limits>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <type_traits>
#include <utility>
#include <vector>

#include "../../include/fluidisim_delta3d.h"
#include "fd3_cut.cuh"
#include "fd3_zmarch4.cuh"
#include "fd3_tmarch.cuh"
#include "fd3_batch.cuh"
#include "fd3_linear.cuh"
#include "fd3_levels.cuh"

using namespace fd3;

namespace {

thread_local std::string g_last_cuda_error;

int cuda_fail(cudaError_t e, const char* what, int line) {
  char buf[512];
  snprintf(buf, sizeof buf, "%s (line %d): %s", what, line, cudaGetErrorString(e));
  g_last_cuda_error = buf;
  return e == cudaErrorMemoryAllocation ? FD3_ERR_OUT_OF_MEMORY : FD3_ERR_CUDA;
}

#define CK(call)                                                   \
  do {                                                             \
    cudaError_t e_ = (call);                                       \
    if (e_ != cudaSuccess) return cuda_fail(e_, #call, __LINE__); \
  } while (0)

#define TRY(expr)        \
  do {                   \
    int s_ = (expr);     \
    if (s_) return s_;   \
  } while (0)

inline int blocks_for(long long n) { return (int)((n + TPB - 1) / TPB); }

// Makes `dev` the calling thread's current device for one scope and restores the previous one.
struct ScopedDevice {
  int prev = -1;
  cudaError_t err = cudaSuccess;
  explicit ScopedDevice(int dev) {
    err = cudaGetDevice(&prev);
    if (err == cudaSuccess && prev != dev) err = cudaSetDevice(dev);
    else if (err == cudaSuccess) prev = -1;  // already current: nothing to restore
  }
  ~ScopedDevice() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};


// Coarse levels of at most this many cells issue their passes' loads before the row code and the
// gate, and restrict their residual in the same pass that computes it (k_level_restrict8).  These
// are the latency-bound levels: measured 2% and 1.4% faster at 128^3; the loads ahead of the code
// were 1% slower on the throughput-bound 128^3 level of a 256^3 volume.
#ifndef FD3_SPEC_MAX
#define FD3_SPEC_MAX 262144
#endif
constexpr int SPEC_MAX_CELLS = FD3_SPEC_MAX;

// Volumes from this many cells run the four-cells-per-thread fine kernels by default (kernels = 0).
constexpr long long kQuadMinCells = 1LL << 23;

// Coarse levels of at most this many cells are solved together by one CTA (k_coarse_tail).
constexpr int TAIL_MAX_CELLS = 512;

// PROJECTION_DIVERGENCE_TOLERANCE (delta_projection.rs:192)
constexpr double kDivTol = 1e-5;
// gamma_8 and gamma_10 of u = 2^-24 (delta_projection.rs:200-203, delta3d.rs:69-72)
constexpr float kRoundoff2D = 8.0f * (1.0f / 16777216.0f) / (1.0f - 8.0f * (1.0f / 16777216.0f));
constexpr float kRoundoff3D = 10.0f * (1.0f / 16777216.0f) / (1.0f - 10.0f * (1.0f / 16777216.0f));
static_assert(kRoundoff2D == BATCH_ROUNDOFF_2D && kRoundoff3D == BATCH_ROUNDOFF_3D && kDivTol == BATCH_DIV_TOL,
              "the persistent batch shares the outer loop's constants");

}  // namespace

struct fd3_volume {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaStream_t own_stream = nullptr;  // created at configure; capturable (not the legacy stream)
  int nx = 0, ny = 0, nz = 0, n = 0, nu = 0, nv = 0, nw = 0, ncol = 0;
  float dx = 0, rho = 0, g = 0, rest = 0, z0 = 0;
  bool cut = false;
  // geometry (cut only)
  float *frac = nullptr, *ou = nullptr, *ov = nullptr, *ow = nullptr, *floor_ = nullptr;
  // state and work fields (delta3d.rs:102-184)
  float *eta = nullptr, *rof = nullptr, *u = nullptr, *v = nullptr, *w = nullptr;
  float *us = nullptr, *vs = nullptr, *ws = nullptr, *p = nullptr, *rhs = nullptr, *res = nullptr;
  float *dir = nullptr, *dir2 = nullptr, *tmp = nullptr, *prec = nullptr;
  unsigned short* codes = nullptr;  // row codes of the current projection
  float *sv_u = nullptr, *sv_v = nullptr, *sv_w = nullptr, *sv_p = nullptr, *sv_eta = nullptr, *sv_rof = nullptr;
  float *flux_x = nullptr, *flux_y = nullptr;
  // a volume configured with a solid: its node SDF buffer and the bottom-only base geometry the
  // cut is redone from when the solid moves (Base3, delta3d_cut.rs:53-80): fractions, apertures,
  // floors, the solid volume per column and the water it deposited
  float *sdf = nullptr, *bfrac = nullptr, *bou = nullptr, *bov = nullptr, *bow = nullptr, *bfloor = nullptr;
  // the solid's rigid motion from the last set_solid_rigid (delta3d.rs:408-410): wall = 2 when it
  // rotates, 1 when it only translates, 0 at rest (Geo::wall)
  Rigid motion{};
  int wall = 0;
  float *bcol = nullptr, *bdep = nullptr;
  // the sparse column set (Sparse3, delta3d_sparse.rs:31-44): device mask, a scratch mask of the
  // columns leaving it, and the host copy the refusals and the published counts read
  bool sparse = false;
  unsigned char *act = nullptr, *act_next = nullptr;
  std::vector<unsigned char> hact;
  unsigned char* tiles = nullptr;  // per 32 x 8 tile of columns: any column in the set (Geo::tiles)
  // multigrid
  bool has_mg = false;
  bool linear = false;            // the current projection is the linear path's
  // homogeneous ghosts (refine_mobile3).  Only the assembly and the correction read ghost values;
  // the inner loop's kernels read ghost coefficients only, so the loop graph does not depend on it.
  bool homog = false;
  bool precondition_cut = true;   // Jacobi on the linear cut path (set_precondition_cut, delta3d.rs:526)
  bool advection_correction = false;  // the second-order advection term (delta3d_advection.rs:17-26)
  float *z = nullptr, *z2 = nullptr;
  std::vector<Lev> levels;
  Lev* dlev = nullptr;   // the level table in device memory (for the single-CTA coarse tail)
  int tail_first = 0;    // first level small enough for the single-CTA tail
  size_t tail_smem_bytes = 0;  // dynamic shared memory of the shared-memory tail (0: global tail)
  bool tail_reg = false;       // every tail level fits one cell per thread of k_coarse_tail_reg
  // reductions and scalars
  double* p64 = nullptr;
  int p64_cap = 0;  // f64 partial slots
  float* p32 = nullptr;
  unsigned* count = nullptr;
  Scalars* dS = nullptr;
  Scalars* hS = nullptr;  // pinned
  int* dflag = nullptr;
  int* hflag = nullptr;   // pinned
  double* fsc = nullptr;  // dot products of the learned FCG and the training hooks
  double* hfsc = nullptr; // pinned
  float *fz = nullptr, *fin = nullptr;  // FCG preconditioned residual and network input (on first use)
  fd3_options opt{};
  bool has_refused = false;
  fd3_report refused{};
  unsigned long long launches = 0;
  std::vector<void*> allocations;
  // opt-in per-kernel timing: events around every launch, collected at each synchronisation
  bool prof = false;
  std::vector<cudaEvent_t> ev_pool;
  size_t ev_next = 0;
  struct Pending { const char* name; cudaEvent_t a, b; };
  std::vector<Pending> pending;
  std::vector<std::string> prof_names;
  std::vector<unsigned long long> prof_count;
  std::vector<double> prof_ms;
  // the inner loop as a CUDA graph with a WHILE node
  cudaGraphExec_t loop_exec = nullptr;
  int loop_mode = -1;
  cudaStream_t loop_stream = nullptr;
  unsigned long long body_nodes = 0;
  // tensor maps of the TMA-staged fine kernels (kernels = 5), made on first use; the buffers they
  // describe are allocated once, so the maps stay valid for the volume's life
  struct TmaSet {
    CUtensorMap hz, hz2, hdir, hdir2, hprec, hres, hp;  // halo boxes
    CUtensorMap oprec, ores, orhs;                      // tile boxes
    CUtensorMap codes, par;                         // row codes; level 0's x (parent box)
  };
  TmaSet* tma = nullptr;
  int tma_state = 0;  // 0 not tried, 1 ready, -1 the driver refused a map

  Geo geo() const {
    Geo G;
    G.nx = nx; G.ny = ny; G.nz = nz; G.n = n;
    G.cut = cut ? 1 : 0;
    G.linear = linear ? 1 : 0;
    G.homog = homog ? 1 : 0;
    G.dx = dx;
    G.inv = 1.f / (dx * dx);
    G.rho_g = rho * g;
    G.rest = rest;
    G.eta = eta; G.rof = rof;
    G.frac = frac; G.ou = ou; G.ov = ov; G.ow = ow;
    G.act = sparse ? act : nullptr;
    G.tiles = sparse && !opt.no_tile_skip ? tiles : nullptr;
    G.wall = wall;
    G.rig = motion;
    G.bou = bou; G.bov = bov; G.bow = bow;
    return G;
  }
  bool ord() const { return opt.reduction == FD3_REDUCE_ORDERED_F32; }
  bool blocked() const { return !ord() && opt.kernels != 1; }
  bool paired() const {
    return blocked() && (opt.kernels == 0 || opt.kernels == 3 || opt.kernels == 4 || opt.kernels == 5) && nx % 2 == 0;
  }
  // TMA-staged fine kernels (fd3_tmarch.cuh) for the V-cycle's and the direction's passes: f32 storage,
  // nx % 8 == 0 and the multigrid, chosen explicitly (kernels = 5) or by default on volumes of at least
  // kQuadMinCells, where the passes stream from HBM (measured on the 256^3 wave: 19.3 against 20.0 ms
  // per projection with four cells per thread; on the 128^3 basin, which sits in L2, 3.07 against
  // 3.03 ms with two cells per thread, which stays the default there)
  bool tmaf() const {
    if (!blocked() || nx % 8 != 0 || opt.storage == FD3_STORAGE_F16 || !mg_on() || tma_state < 0) return false;
    return opt.kernels == 5 || (opt.kernels == 0 && (long long)n >= kQuadMinCells);
  }
  // four cells per thread: with f32 storage and nx % 4 == 0, chosen explicitly (kernels = 4) or by
  // default on volumes of at least kQuadMinCells, where the passes stream from HBM (measured: 256^3
  // 20.9 against 21.5 ms per projection; at 128^3, where the working set sits in L2 and the passes
  // are latency-bound, two cells per thread is faster, 3.20 against 3.47 ms)
  bool quad() const {
    if (!blocked() || nx % 4 != 0 || opt.storage == FD3_STORAGE_F16) return false;
    return opt.kernels == 4 || (opt.kernels == 0 && (long long)n >= kQuadMinCells);
  }
  bool mg_on() const { return has_mg && !linear; }  // the linear path has no multigrid
  // FP16 storage of the V-cycle vectors (fd3_set_options accepts it only with the paired kernels)
  bool half() const { return opt.storage == FD3_STORAGE_F16 && paired() && mg_on(); }
  int loop_key() const {
    return (ord() ? 1 : 0) | (mg_on() ? 2 : 0) | (blocked() ? 4 : 0) | (opt.no_overlap ? 8 : 0) | (linear ? 16 : 0) |
           (paired() ? 32 : 0) | (half() ? 64 : 0) | (sparse ? 128 : 0) |  // the captured Geo holds the set's mask
           (opt.no_tile_skip ? 256 : 0) | (quad() ? 512 : 0) | (tmaf() ? 1024 : 0);
  }
  Red red() const { return Red{p64, p32, count}; }
};

namespace {

int dalloc(fd3_volume* V, float** ptr, size_t count) {
  void* q = nullptr;
  CK(cudaMalloc(&q, count * sizeof(float) + 16));
  CK(cudaMemsetAsync(q, 0, count * sizeof(float) + 16, V->stream));
  V->allocations.push_back(q);
  *ptr = (float*)q;
  return FD3_OK;
}

void release(fd3_volume* V) {
  if (V->stream) cudaStreamSynchronize(V->stream);
  if (V->loop_exec) cudaGraphExecDestroy(V->loop_exec);
  for (cudaEvent_t e : V->ev_pool) cudaEventDestroy(e);
  for (void* q : V->allocations) cudaFree(q);
  if (V->hS) cudaFreeHost(V->hS);
  if (V->hflag) cudaFreeHost(V->hflag);
  if (V->hfsc) cudaFreeHost(V->hfsc);
  if (V->own_stream) cudaStreamDestroy(V->own_stream);
  delete V->tma;
  V->tma = nullptr;
}

cudaEvent_t next_event(fd3_volume* V) {
  if (V->ev_next == V->ev_pool.size()) {
    cudaEvent_t e;
    cudaEventCreate(&e);
    V->ev_pool.push_back(e);
  }
  return V->ev_pool[V->ev_next++];
}

// Every kernel launch of the library goes through here: grid x block on the handle's stream,
// counted, and bracketed by events when profiling is on.
// Launch with the programmatic-stream-serialization attribute (see KSTART in fd3_kernels.cuh).
template <class... P, class... A>
void launch_pdl(fd3_volume* V, int grid, int block, size_t smem, void (*kernel)(P...), A... args) {
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(block);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = V->stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = V->opt.no_overlap ? 0 : 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cudaLaunchKernelEx(&cfg, kernel, ((P)args)...);
}

template <class K, class... A>
void launch_grid(fd3_volume* V, const char* name, int grid, int block, K kernel, A... args) {
  cudaEvent_t a = nullptr, b = nullptr;
  if (V->prof) { a = next_event(V); cudaEventRecord(a, V->stream); }
  launch_pdl(V, grid, block, 0, kernel, args...);
  if (V->prof) { b = next_event(V); cudaEventRecord(b, V->stream); V->pending.push_back({name, a, b}); }
  V->launches++;
}
#define LAUNCH(V, KERNEL, N, ...) launch_grid((V), #KERNEL, blocks_for(N), TPB, KERNEL, __VA_ARGS__)

// The same with dynamic shared memory.
template <class K, class... A>
void launch_grid_smem(fd3_volume* V, const char* name, int grid, int block, size_t smem, K kernel, A... args) {
  cudaEvent_t a = nullptr, b = nullptr;
  if (V->prof) { a = next_event(V); cudaEventRecord(a, V->stream); }
  launch_pdl(V, grid, block, smem, kernel, args...);
  if (V->prof) { b = next_event(V); cudaEventRecord(b, V->stream); V->pending.push_back({name, a, b}); }
  V->launches++;
}
#define LAUNCH_G(V, KERNEL, GRID, BLOCK, ...) launch_grid((V), #KERNEL, (GRID), (BLOCK), KERNEL, __VA_ARGS__)

void prof_collect(fd3_volume* V) {
  for (auto& r : V->pending) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, r.a, r.b);
    size_t q = 0;
    while (q < V->prof_names.size() && V->prof_names[q] != r.name) ++q;
    if (q == V->prof_names.size()) { V->prof_names.emplace_back(r.name); V->prof_count.push_back(0); V->prof_ms.push_back(0.0); }
    V->prof_count[q] += 1;
    V->prof_ms[q] += ms;
  }
  V->pending.clear();
  V->ev_next = 0;
}

int sync(fd3_volume* V) {
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(V->stream));
  if (V->prof) prof_collect(V);
  return FD3_OK;
}

int pull(fd3_volume* V) {
  CK(cudaMemcpyAsync(V->hS, V->dS, sizeof(Scalars), cudaMemcpyDeviceToHost, V->stream));
  return sync(V);
}

// Grid of the grid-stride update: no more blocks than groups of four cells need.
inline int update_blocks(int n) { return std::min(UPDATE_BLOCKS, std::max(1, blocks_for((n + 3) / 4))); }
// The sparse set for kv_update_rn's skip (four cells of a row share a 4-byte mask word when nx % 4 == 0).
inline const unsigned char* update_mask(const fd3_volume* V) {
  return V->sparse && !V->opt.no_tile_skip && V->nx % 4 == 0 ? V->act : nullptr;
}

#define DISPATCH(V, KERNEL, N, ...)                                                               \
  do {                                                                                           \
    if ((V)->ord()) launch_grid((V), #KERNEL, blocks_for(N), TPB, KERNEL<RED_ORD>, __VA_ARGS__);   \
    else launch_grid((V), #KERNEL, blocks_for(N), TPB, KERNEL<RED_F64>, __VA_ARGS__);              \
  } while (0)

// ------------------------------------------------------------------------------------ multigrid
// prepare_multigrid3 (delta3d_multigrid.rs:370-387): coarse geometry follows the surface.
// Two launches per level (kinds and apertures, then diagonal and codes); the levels of at most
// PREP_SMALL_CELLS cells below the first run in one CTA (the 24 launches of a 128^3 hierarchy become
// 7; with the 16^3 level in the one-CTA kernel too, that kernel alone took 27.7 us).
constexpr int PREP_SMALL_CELLS = 512;
void prepare_multigrid(fd3_volume* V) {
  if (!V->has_mg || V->levels.empty()) return;
  Geo G = V->geo();
  const int nl = (int)V->levels.size();
  for (int l = 0; l < nl; ++l) {
    const Lev& C = V->levels[l];
    if (l > 0 && C.n <= PREP_SMALL_CELLS) {
      LAUNCH_G(V, k_levels_prepare_small, 1, PREP_SMALL_THREADS, (const Lev*)V->dlev, l, nl - 1);
      return;
    }
    const long long nfaces = (long long)(C.nx + 1) * C.ny * C.nz + (long long)C.nx * (C.ny + 1) * C.nz +
                             (long long)C.nx * C.ny * (C.nz + 1);
    LAUNCH(V, k_level_prepare_a, C.n + nfaces, G, l > 0 ? V->levels[l - 1] : Lev{}, C, l == 0 ? 1 : 0);
    LAUNCH(V, k_level_prepare_b, C.n, C);
  }
}

// coarse_cycle3 (delta3d_multigrid.rs:303-332); levels[0].r already restricted.  Levels from
// V->tail_first on are solved by one CTA; the larger ones by grid-wide fused kernels.  T is the
// storage of the level vectors; with FP16 storage the tail is the one-cell-per-thread CTA, or, if
// the tail does not fit it, every level is launched.
template <class T>
void coarse_cycle_t(fd3_volume* V, int gate) {
  std::vector<Lev>& Ls = V->levels;
  const int last = (int)Ls.size() - 1;
  const bool half = Store<T>::half;
  const int first_tail = (half && !V->tail_reg) ? (int)Ls.size() : V->tail_first;
  const Scalars* S = V->dS;
  for (int l = 0; l < first_tail && l <= last; ++l) {
    Lev& L = Ls[l];
    if (l == last) {  // a large coarsest level: its 8 sweeps one by one
      for (int s = 0; s < 8; ++s)
        LAUNCH(V, k_level_sweep_c<T>, L.n, L, (const float*)((s % 2 == 0) ? L.x : L.x2), (s % 2 == 0) ? L.x2 : L.x,
               s == 0 ? 1 : 0, S, gate);
    } else {
      const long long n8 = 8LL * Ls[l + 1].n;  // one thread per child of each next-level cell
      if (L.n <= SPEC_MAX_CELLS) {
        launch_grid(V, "k_level_pre", blocks_for(L.n), TPB, k_level_pre<T, true>, L, S, gate);
        launch_grid(V, "k_level_restrict8", blocks_for(n8), TPB, k_level_restrict8<T, true>, L, Ls[l + 1], S, gate);
      } else {
        launch_grid(V, "k_level_pre", blocks_for(L.n), TPB, k_level_pre<T, false>, L, S, gate);
        launch_grid(V, "k_level_resid", blocks_for(L.n), TPB, k_level_resid<T, false>, L, S, gate);
        LAUNCH(V, k_level_sum8<T>, Ls[l + 1].n, L, Ls[l + 1], S, gate);
      }
    }
  }
  if (first_tail <= last) {
    if (V->tail_reg) {
      TailLevs tl{};
      for (int l = first_tail; l <= last; ++l) tl.L[l - first_tail] = Ls[l];
      LAUNCH_G(V, k_coarse_tail_reg<T>, 1, TAIL_REG_THREADS, tl, last - first_tail + 1, S, gate);
    }
    else if (V->tail_smem_bytes > 0)
      launch_grid_smem(V, "k_coarse_tail_smem", 1, TAIL_THREADS, V->tail_smem_bytes, k_coarse_tail_smem,
                       (const Lev*)V->dlev, first_tail, last, S, gate);
    else
      LAUNCH_G(V, k_coarse_tail, 1, TAIL_THREADS, (const Lev*)V->dlev, first_tail, last, S, gate);
  }
  // Level l's second post-sweep is folded into level l - 1's first (k_level_post21) when both are
  // small, level l is no tail level, and level l - 1 exists.
  const int top = std::min(first_tail, last) - 1;
  auto fused = [&](int l) { return l >= 0 && l + 1 <= top && Ls[l].n <= SPEC_MAX_CELLS; };
  for (int l = top; l >= 0; --l) {
    if (Ls[l].n <= SPEC_MAX_CELLS) {
      if (fused(l))
        launch_grid(V, "k_level_post21", blocks_for(8LL * Ls[l + 1].n), TPB, k_level_post21<T>, Ls[l], Ls[l + 1], S,
                    gate);
      else
        launch_grid(V, "k_level_post1", blocks_for(Ls[l].n), TPB, k_level_post1<T, true>, Ls[l], Ls[l + 1], S, gate);
      if (!fused(l - 1))
        launch_grid(V, "k_level_post2", blocks_for(Ls[l].n), TPB, k_level_post2<T, true>, Ls[l], S, gate);
    } else {
      launch_grid(V, "k_level_post1", blocks_for(Ls[l].n), TPB, k_level_post1<T, false>, Ls[l], Ls[l + 1], S, gate);
      launch_grid(V, "k_level_post2", blocks_for(Ls[l].n), TPB, k_level_post2<T, false>, Ls[l], S, gate);
    }
  }
}
void coarse_cycle(fd3_volume* V, int gate) {
  if (V->half()) coarse_cycle_t<__half>(V, gate);
  else coarse_cycle_t<float>(V, gate);
}

// The fine passes of the V-cycle with the paired kernels of K2 layers per CTA.
// T: the storage of z, z2 and the coarse vectors (f32, or FP16 in the mixed-precision mode).
template <int K2, class T>
void paired_vcycle(fd3_volume* V, int gate, int op) {
  Geo G = V->geo();
  const Scalars* S = V->dS;
  const bool levels = !V->levels.empty();
  Lev L0 = levels ? V->levels[0] : Lev{};
  const unsigned short* codes = V->codes;
  const int zb = zblocks2(V->nx, V->ny, V->nz, K2);
  T* z = reinterpret_cast<T*>(V->z);
  T* z2 = reinterpret_cast<T*>(V->z2);
  launch_grid(V, "kx_fine_pre<K2>", zb, Z2T, kx_fine_pre<K2, T>, G, codes, (const float*)V->prec,
              (const float*)V->res, z, S, gate);
  if (levels) {
    launch_grid(V, "kx_fine_restrict<K2>", zb, Z2T, kx_fine_restrict<K2, T>, G, codes, (const float*)V->res,
                (const T*)z, L0, S, gate);
    coarse_cycle(V, gate);
  }
  launch_grid(V, "kx_fine_post1<K2>", zb, Z2T, kx_fine_post1<K2, T>, G, codes, (const float*)V->prec,
              (const float*)V->res, (const T*)z, L0, levels ? 1 : 0, z2, S, gate);
  launch_grid(V, "kx_fine_post2_rz<K2>", zb, Z2T, kx_fine_post2_rz<K2, T>, G, codes, (const float*)V->prec,
              (const float*)V->res, (const T*)z2, z, V->red(), V->dS, gate, op);
}
template <int K2>
void paired_vcycle(fd3_volume* V, int gate, int op) {
  if (V->half()) paired_vcycle<K2, __half>(V, gate, op);
  else paired_vcycle<K2, float>(V, gate, op);
}

// The tiling of the four-cells-per-thread kernels: QX lanes per row (a tile 4 QX cells wide, 256 /
// QX rows), K4 layers per CTA (8 when that still gives two waves of CTAs at two per SM, else 4).
template <int N>
using IC = std::integral_constant<int, N>;
inline int quad_qx(int nx) { return nx >= 128 ? 32 : 16; }
template <class F>
void quad_dispatch(const fd3_volume* V, F f) {
  const bool wide = quad_qx(V->nx) == 32;
  const int k8 = wide ? zblocks4<32>(V->nx, V->ny, V->nz, 8) : zblocks4<16>(V->nx, V->ny, V->nz, 8);
  const bool deep = k8 >= 2 * 2 * 148;
  if (wide) { if (deep) f(IC<32>{}, IC<8>{}); else f(IC<32>{}, IC<4>{}); }
  else { if (deep) f(IC<16>{}, IC<8>{}); else f(IC<16>{}, IC<4>{}); }
}

// The fine passes of the V-cycle with the four-cells-per-thread kernels (f32 storage).
void quad_vcycle(fd3_volume* V, int gate, int op) {
  quad_dispatch(V, [&](auto qx, auto k4) {
    constexpr int QX = decltype(qx)::value, K4 = decltype(k4)::value;
    Geo G = V->geo();
    const Scalars* S = V->dS;
    const bool levels = !V->levels.empty();
    Lev L0 = levels ? V->levels[0] : Lev{};
    const unsigned short* codes = V->codes;
    const int zb = zblocks4<QX>(V->nx, V->ny, V->nz, K4);
    launch_grid(V, "kq_fine_pre", zb, Z4T, kq_fine_pre<QX, K4>, G, codes, (const float*)V->prec,
                (const float*)V->res, V->z, S, gate);
    if (levels) {
      launch_grid(V, "kq_fine_restrict", zb, Z4T, kq_fine_restrict<QX, K4>, G, codes, (const float*)V->res,
                  (const float*)V->z, L0, S, gate);
      coarse_cycle(V, gate);
    }
    launch_grid(V, "kq_fine_post1", zb, Z4T, kq_fine_post1<QX, K4>, G, codes, (const float*)V->prec,
                (const float*)V->res, (const float*)V->z, L0, levels ? 1 : 0, V->z2, S, gate);
    launch_grid(V, "kq_fine_post2_rz", zb, Z4T, kq_fine_post2_rz<QX, K4>, G, codes, (const float*)V->prec,
                (const float*)V->res, (const float*)V->z2, V->z, V->red(), V->dS, gate, op);
  });
}

// ------------------------------------------------------------------ TMA-staged fine kernels
// cuTensorMapEncodeTiled from the driver the runtime is bound to (no link against libcuda).
typedef CUresult (*TmapEncodeFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                 const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
TmapEncodeFn tmap_encoder() {
  static TmapEncodeFn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &f, 12000, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<TmapEncodeFn>(f);
  });
  return fn;
}

// A 3-D map of an nx x ny x nz array (f32, or u16 row codes) copied in boxes of bw x bh x 1; cells
// outside the array read as zero.
bool make_tmap(CUtensorMap* m, const void* base, bool u16, int nx, int ny, int nz, int bw, int bh) {
  TmapEncodeFn enc = tmap_encoder();
  if (!enc) return false;
  const cuuint64_t es = u16 ? 2 : 4;
  const cuuint64_t dims[3] = {(cuuint64_t)nx, (cuuint64_t)ny, (cuuint64_t)nz};
  const cuuint64_t strides[2] = {(cuuint64_t)nx * es, (cuuint64_t)nx * ny * es};
  const cuuint32_t box[3] = {(cuuint32_t)bw, (cuuint32_t)bh, 1u};
  const cuuint32_t estr[3] = {1u, 1u, 1u};
  return enc(m, u16 ? CU_TENSOR_MAP_DATA_TYPE_UINT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<void*>(base), dims,
             strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
             CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// The volume's tensor maps, made once; false (and the family is off for good) if the driver refuses one.
bool tma_ready(fd3_volume* V) {
  if (V->tma_state != 0) return V->tma_state > 0;
  V->tma_state = -1;
  fd3_volume::TmaSet* T = new (std::nothrow) fd3_volume::TmaSet();
  if (!T) return false;
  const int nx = V->nx, ny = V->ny, nz = V->nz;
  bool ok = make_tmap(&T->hz, V->z, false, nx, ny, nz, TMW, TMH) && make_tmap(&T->hz2, V->z2, false, nx, ny, nz, TMW, TMH) &&
            make_tmap(&T->hdir, V->dir, false, nx, ny, nz, TMW, TMH) &&
            make_tmap(&T->hdir2, V->dir2, false, nx, ny, nz, TMW, TMH) &&
            make_tmap(&T->hprec, V->prec, false, nx, ny, nz, TMW, TMH) &&
            make_tmap(&T->hres, V->res, false, nx, ny, nz, TMW, TMH) &&
            make_tmap(&T->hp, V->p, false, nx, ny, nz, TMW, TMH) &&
            make_tmap(&T->oprec, V->prec, false, nx, ny, nz, TMX, TMY) &&
            make_tmap(&T->ores, V->res, false, nx, ny, nz, TMX, TMY) &&
            make_tmap(&T->orhs, V->rhs, false, nx, ny, nz, TMX, TMY) &&
            make_tmap(&T->codes, V->codes, true, nx, ny, nz, TMX, TMY);
  if (ok && !V->levels.empty()) {
    const Lev& L = V->levels[0];
    ok = L.nx * 2 == nx && L.ny * 2 == ny && L.nz * 2 == nz && make_tmap(&T->par, L.x, false, L.nx, L.ny, L.nz, TMPW, TMPH);
  }
  if (!ok) { delete T; return false; }
  V->tma = T;
  V->tma_state = 1;
  return true;
}

template <int PASS, int K, int D, int Q>
void launch_tpass(fd3_volume* V, const char* name, const TMaps& M, const TArgs& a) {
  constexpr int MINB = Q == 4 ? 5 : FD3_TMINB;
  static std::once_flag attr_once;  // one per instantiation: the opt-in above 48 KiB of shared memory
  std::call_once(attr_once, [] {
    cudaFuncSetAttribute(kt_pass<PASS, K, D, Q, MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)TPass<PASS, D>::SMEM_LAUNCH);
  });
  launch_grid_smem(V, name, zblocks_t(V->nx, V->ny, V->nz, K), TQ<Q>::NT, TPass<PASS, D>::SMEM_LAUNCH,
                   kt_pass<PASS, K, D, Q, MINB>, M, V->geo(), a, V->red(), V->dS);
}

// Layers per CTA of the TMA-staged kernels: 8 when the grid still gives two waves at four CTAs per SM,
// else 4 (measured: at 128^3, 8 and 16 layers took 3.95 and 4.70 ms per projection against 3.07 with
// 4; at 256^3, 16 layers were no faster than 8).  Two cells per thread and two layers in flight:
// four cells per thread (CTAs of 128 threads) and deeper rings (fewer CTAs per SM) were slower at both
// sizes, one layer in flight slower at 128^3.
inline int pick_kt(int nx, int ny, int nz) { return zblocks_t(nx, ny, nz, 8) >= 2 * 4 * 148 ? 8 : 4; }
template <class F>
void kt_dispatch(const fd3_volume* V, F f) {
  if (pick_kt(V->nx, V->ny, V->nz) == 8) f(IC<8>{}, IC<2>{}, IC<2>{});
  else f(IC<4>{}, IC<2>{}, IC<2>{});
}

template <int K, int Q, int D>
void tma_vcycle_k(fd3_volume* V, int gate, int op) {
  const fd3_volume::TmaSet& T = *V->tma;
  const bool levels = !V->levels.empty();
  TArgs a{};
  a.gate = gate;
  a.L = levels ? V->levels[0] : Lev{};
  TMaps M{};
  // z = the two pre-sweeps from zero: halo prec, r
  M.m[0] = T.hprec; M.m[1] = T.hres; M.m[2] = T.codes;
  a.out0 = V->z;
  launch_tpass<TP_PRE, K, D, Q>(V, "kt_fine_pre", M, a);
  if (levels) {  // residual and its eight-child mean into level 0's r: halo z, tile r
    M.m[0] = T.hz; M.m[1] = T.ores; M.m[2] = T.codes;
    launch_tpass<TP_RESTRICT, K, D, Q>(V, "kt_fine_restrict", M, a);
    coarse_cycle(V, gate);
  }
  // z2 = prolongation + the first post-sweep: halo z, prec; tile r; codes; parent
  M.m[0] = T.hz; M.m[1] = T.hprec; M.m[2] = T.ores; M.m[3] = T.codes; M.m[4] = levels ? T.par : T.codes;
  a.out0 = V->z2;
  a.prolong = levels ? 1 : 0;
  launch_tpass<TP_POST1, K, D, Q>(V, "kt_fine_post1", M, a);
  // z = the second post-sweep with r.z: halo z2; tile prec, r
  M.m[0] = T.hz2; M.m[1] = T.oprec; M.m[2] = T.ores; M.m[3] = T.codes;
  a.out0 = V->z;
  a.op = op;
  launch_tpass<TP_POST2, K, D, Q>(V, "kt_fine_post2_rz", M, a);
}
void tma_vcycle(fd3_volume* V, int gate, int op) {
  kt_dispatch(V, [&](auto k, auto q, auto d) {
    tma_vcycle_k<decltype(k)::value, decltype(q)::value, decltype(d)::value>(V, gate, op);
  });
}
// d = z (+ beta d) from din into dout, q = A d, d.q and alpha.
void tma_dir(fd3_volume* V, int parity) {
  const fd3_volume::TmaSet& T = *V->tma;
  TMaps M{};
  M.m[0] = T.hz; M.m[1] = parity ? T.hdir2 : T.hdir; M.m[2] = T.codes;
  TArgs a{};
  a.out0 = parity ? V->dir : V->dir2;
  a.out1 = V->tmp;
  kt_dispatch(V, [&](auto k, auto q, auto d) {
    launch_tpass<TP_DIR, decltype(k)::value, decltype(d)::value, decltype(q)::value>(V, "kt_dir_apply_dot", M, a);
  });
}

// res = rhs - A p with res.res (FIN_RR0 or FIN_ACTUAL): halo p, tile rhs.
void tma_residual(fd3_volume* V, int op) {
  const fd3_volume::TmaSet& T = *V->tma;
  TMaps M{};
  M.m[0] = T.hp; M.m[1] = T.orhs; M.m[2] = T.codes;
  TArgs a{};
  a.out0 = V->res;
  a.op = op;
  kt_dispatch(V, [&](auto k, auto q, auto d) {
    launch_tpass<TP_RESID, decltype(k)::value, decltype(d)::value, decltype(q)::value>(V, "kt_residual", M, a);
  });
}

// v_cycle3 (delta3d_multigrid.rs:393-429) with res.z at its end (op FIN_RZ_PRIME or FIN_RZ_ITER);
// z = M^-1 res is left in V->z.
void vcycle(fd3_volume* V, int gate, int op) {
  Geo G = V->geo();
  const Scalars* S = V->dS;
  const bool levels = !V->levels.empty();
  Lev L0 = levels ? V->levels[0] : Lev{};
  const unsigned short* codes = V->codes;
  if (V->tmaf() && tma_ready(V)) {  // TMA-staged 2.5-D blocked kernels (f64 reductions, f32 storage)
    tma_vcycle(V, gate, op);
    return;
  }
  if (V->quad()) {  // 2.5-D blocked kernels, four cells per thread (f64 reductions, f32 storage)
    quad_vcycle(V, gate, op);
    return;
  }
  if (V->paired()) {  // 2.5-D blocked kernels, two cells per thread (f64 reductions)
    if (pick_k2(V->nx, V->ny, V->nz) == 8) paired_vcycle<8>(V, gate, op);
    else paired_vcycle<4>(V, gate, op);
    return;
  }
  if (V->blocked()) {  // 2.5-D blocked kernels (f64 reductions)
    const int zb = zblocks(V->nx, V->ny, V->nz);
    const bool full = zfull(V->nx, V->ny, V->nz);
    if (full) LAUNCH_G(V, kz_fine_pre<true>, zb, ZT, G, codes, (const float*)V->prec, (const float*)V->res, V->z, S, gate);
    else LAUNCH_G(V, kz_fine_pre<false>, zb, ZT, G, codes, (const float*)V->prec, (const float*)V->res, V->z, S, gate);
    if (levels) {
      if (full) LAUNCH_G(V, kz_fine_restrict<true>, zb, ZT, G, codes, (const float*)V->res, (const float*)V->z, L0, S, gate);
      else LAUNCH_G(V, kz_fine_restrict<false>, zb, ZT, G, codes, (const float*)V->res, (const float*)V->z, L0, S, gate);
      coarse_cycle(V, gate);
    }
    if (full)
      LAUNCH_G(V, kz_fine_post1<true>, zb, ZT, G, codes, (const float*)V->prec, (const float*)V->res, (const float*)V->z,
               L0, levels ? 1 : 0, V->z2, S, gate);
    else
      LAUNCH_G(V, kz_fine_post1<false>, zb, ZT, G, codes, (const float*)V->prec, (const float*)V->res, (const float*)V->z,
               L0, levels ? 1 : 0, V->z2, S, gate);
    if (full)
      LAUNCH_G(V, kz_fine_post2_rz<true>, zb, ZT, G, codes, (const float*)V->prec, (const float*)V->res,
               (const float*)V->z2, V->z, V->red(), V->dS, gate, op);
    else
      LAUNCH_G(V, kz_fine_post2_rz<false>, zb, ZT, G, codes, (const float*)V->prec, (const float*)V->res,
               (const float*)V->z2, V->z, V->red(), V->dS, gate, op);
    return;
  }
  LAUNCH(V, k_fine_pre, V->n, G, codes, (const float*)V->prec, (const float*)V->res, V->z, S, gate);
  if (levels) {
    LAUNCH(V, k_fine_restrict_c, L0.n, G, codes, (const float*)V->res, (const float*)V->z, L0, S, gate);
    coarse_cycle(V, gate);
  }
  LAUNCH(V, k_fine_post1, V->n, G, codes, (const float*)V->prec, (const float*)V->res, (const float*)V->z, L0,
         levels ? 1 : 0, V->z2, S, gate);
  DISPATCH(V, k_fine_post2_rz, V->n, G, codes, (const float*)V->prec, (const float*)V->res, (const float*)V->z2, V->z,
           V->red(), V->dS, gate, op);
}

// prime_multigrid3 / prime_mobile3 with beta = 0 (delta3d_mobile.rs:517, 587): rz of a fresh
// direction; with the multigrid the direction itself is formed by the next k_dir_apply_dot.
void prime(fd3_volume* V) {
  if (V->mg_on()) {
    vcycle(V, 0, FIN_RZ_PRIME);
  } else {
    LAUNCH(V, k_jacobi_dir, V->n, V->n, (const float*)V->prec, (const float*)V->res, V->dir, (const Scalars*)V->dS, 0, 0);
    DISPATCH(V, k_dot_prec_fin, V->n, V->n, (const float*)V->res, (const float*)V->prec, V->red(), V->dS, 0,
             (int)FIN_RZ_PRIME);
  }
}

// One inner PCG iteration (delta3d_mobile.rs:515-545), every kernel gated on S->active.  With the
// multigrid, the direction alternates between dir and dir2 (parity) because it is recomputed at
// the stencil points of the operator.
void iteration(fd3_volume* V, int parity) {
  Geo G = V->geo();
  if (V->mg_on()) {
    float* din = parity ? V->dir2 : V->dir;
    float* dout = parity ? V->dir : V->dir2;
    if (V->tmaf() && tma_ready(V)) {
      tma_dir(V, parity);
      LAUNCH_G(V, kv_update_rn, update_blocks(V->n), TPB, V->n, V->p, V->res, (const float*)dout,
               (const float*)V->tmp, V->red(), V->dS, update_mask(V), V->ncol);
    } else if (V->quad()) {
      quad_dispatch(V, [&](auto qx, auto k4) {
        constexpr int QX = decltype(qx)::value, K4 = decltype(k4)::value;
        launch_grid(V, "kq_dir_apply_dot", zblocks4<QX>(V->nx, V->ny, V->nz, K4), Z4T, kq_dir_apply_dot<QX, K4>, G,
                    (const unsigned short*)V->codes, (const float*)V->z, (const float*)din, dout, V->tmp, V->red(),
                    V->dS);
      });
      LAUNCH_G(V, kv_update_rn, update_blocks(V->n), TPB, V->n, V->p, V->res, (const float*)dout,
               (const float*)V->tmp, V->red(), V->dS, update_mask(V), V->ncol);
    } else if (V->paired()) {
      const int k2 = pick_k2(V->nx, V->ny, V->nz);
      const int zb = zblocks2(V->nx, V->ny, V->nz, k2);
      const unsigned short* codes = V->codes;
      const float* z = V->z;
      if (V->half()) {
        const __half* zh = reinterpret_cast<const __half*>(z);
        if (k2 == 8)
          launch_grid(V, "kx_dir_apply_dot<8>", zb, Z2T, kx_dir_apply_dot<8, __half>, G, codes, zh, (const float*)din,
                      dout, V->tmp, V->red(), V->dS);
        else
          launch_grid(V, "kx_dir_apply_dot<4>", zb, Z2T, kx_dir_apply_dot<4, __half>, G, codes, zh, (const float*)din,
                      dout, V->tmp, V->red(), V->dS);
      } else {
        if (k2 == 8)
          launch_grid(V, "kx_dir_apply_dot<8>", zb, Z2T, kx_dir_apply_dot<8, float>, G, codes, z, (const float*)din,
                      dout, V->tmp, V->red(), V->dS);
        else
          launch_grid(V, "kx_dir_apply_dot<4>", zb, Z2T, kx_dir_apply_dot<4, float>, G, codes, z, (const float*)din,
                      dout, V->tmp, V->red(), V->dS);
      }
      LAUNCH_G(V, kv_update_rn, update_blocks(V->n), TPB, V->n, V->p, V->res, (const float*)dout,
               (const float*)V->tmp, V->red(), V->dS, update_mask(V), V->ncol);
    } else if (V->blocked()) {
      if (zfull(V->nx, V->ny, V->nz))
        LAUNCH_G(V, kz_dir_apply_dot<true>, zblocks(V->nx, V->ny, V->nz), ZT, G, (const unsigned short*)V->codes,
                 (const float*)V->z, (const float*)din, dout, V->tmp, V->red(), V->dS);
      else
        LAUNCH_G(V, kz_dir_apply_dot<false>, zblocks(V->nx, V->ny, V->nz), ZT, G, (const unsigned short*)V->codes,
                 (const float*)V->z, (const float*)din, dout, V->tmp, V->red(), V->dS);
      LAUNCH_G(V, kv_update_rn, update_blocks(V->n), TPB, V->n, V->p, V->res, (const float*)dout,
               (const float*)V->tmp, V->red(), V->dS, update_mask(V), V->ncol);
    } else {
      DISPATCH(V, k_dir_apply_dot, V->n, G, (const unsigned short*)V->codes, (const float*)V->z, (const float*)din, dout,
               V->tmp, V->red(), V->dS);
      DISPATCH(V, k_update_rn, V->n, V->n, V->p, V->res, (const float*)dout, (const float*)V->tmp, V->red(), V->dS);
    }
    vcycle(V, 1, FIN_RZ_ITER);
  } else {
    DISPATCH(V, k_apply_dot_c, V->n, G, (const unsigned short*)V->codes, (const float*)V->dir, V->tmp, V->red(), V->dS);
    DISPATCH(V, k_update_rn, V->n, V->n, V->p, V->res, (const float*)V->dir, (const float*)V->tmp, V->red(), V->dS);
    DISPATCH(V, k_dot_prec_fin, V->n, V->n, (const float*)V->res, (const float*)V->prec, V->red(), V->dS, 1,
             (int)FIN_RZ_ITER);
    LAUNCH(V, k_jacobi_dir, V->n, V->n, (const float*)V->prec, (const float*)V->res, V->dir, (const Scalars*)V->dS, 1, 1);
  }
}

// The inner loop as one CUDA graph: a WHILE node whose body is two iterations and the condition
// kernel, so the whole loop runs on the device without a host round trip per iteration.
int build_loop_graph(fd3_volume* V) {
  if (V->loop_exec) { cudaGraphExecDestroy(V->loop_exec); V->loop_exec = nullptr; }
  cudaGraph_t graph;
  CK(cudaGraphCreate(&graph, 0));
  cudaGraphConditionalHandle handle;
  cudaError_t e = cudaGraphConditionalHandleCreate(&handle, graph, 1, cudaGraphCondAssignDefault);
  if (e != cudaSuccess) { cudaGraphDestroy(graph); return cuda_fail(e, "cudaGraphConditionalHandleCreate", __LINE__); }
  cudaGraphNodeParams params{};
  params.type = cudaGraphNodeTypeConditional;
  params.conditional.handle = handle;
  params.conditional.type = cudaGraphCondTypeWhile;
  params.conditional.size = 1;
  cudaGraphNode_t node;
  e = cudaGraphAddNode(&node, graph, nullptr, 0, &params);
  if (e != cudaSuccess) { cudaGraphDestroy(graph); return cuda_fail(e, "cudaGraphAddNode(while)", __LINE__); }
  cudaGraph_t body = params.conditional.phGraph_out[0];
  e = cudaStreamBeginCaptureToGraph(V->stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) { cudaGraphDestroy(graph); return cuda_fail(e, "cudaStreamBeginCaptureToGraph", __LINE__); }
  unsigned long long before = V->launches;
  iteration(V, 0);
  iteration(V, 1);
  LAUNCH_G(V, k_loop_cond, 1, 1, handle, V->dS);
  cudaGraph_t captured = body;
  e = cudaStreamEndCapture(V->stream, &captured);
  V->body_nodes = V->launches - before;
  V->launches = before;
  if (e != cudaSuccess) { cudaGraphDestroy(graph); return cuda_fail(e, "cudaStreamEndCapture", __LINE__); }
  e = cudaGraphInstantiate(&V->loop_exec, graph, 0);
  cudaGraphDestroy(graph);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGraphInstantiate(loop)", __LINE__);
  V->loop_mode = V->loop_key();
  V->loop_stream = V->stream;
  return FD3_OK;
}

// Run the inner loop until S->active drops.
int run_inner(fd3_volume* V, uint32_t it_before) {
  const bool graphs = V->opt.use_graphs && !V->prof;
  if (graphs) {
    int mode = V->loop_key();
    if (!V->loop_exec || V->loop_mode != mode || V->loop_stream != V->stream) TRY(build_loop_graph(V));
    CK(cudaGraphLaunch(V->loop_exec, V->stream));
    TRY(pull(V));
    unsigned ran = V->hS->it > it_before ? V->hS->it - it_before : 1;
    V->launches += (unsigned long long)((ran + 1) / 2) * V->body_nodes;
    return FD3_OK;
  }
  // The device clears S->active within max_iters iterations (FIN_RN); the host bound is a guard.
  for (unsigned guard = 0;; ++guard) {
    if (guard > V->hS->max_iters + 2u) return FD3_ERR_CUDA;
    iteration(V, guard & 1);
    TRY(pull(V));
    if (!V->hS->active) break;
  }
  return FD3_OK;
}

// Max-reductions and the fingerprint (fmax slots and hash are reset before each use).
__global__ void k_reset_diag(Scalars* S, int mask) {
  if (mask & 1) { S->fmax[0] = 0.f; S->fmax[1] = 0.f; S->fmax[2] = 0.f; }
  if (mask & 2) S->fmax[3] = 0.f;
  if (mask & 4) S->hash = 0ull;
}


// The checks that end or restart the outer loop (delta3d_mobile.rs:547-585), launched together:
// the true residual, the corrected field and its divergence metric (delta3d_mobile.rs:398-433),
// the backward error (:243-271) and the fingerprint of p.  Correcting before knowing whether the
// solve is accepted is harmless: us is untouched and every exit corrects from it again or restores
// res = rhs - A p with res.res (FIN_RR0 or FIN_ACTUAL): on the paired march where the loop runs on
// it (f64 reductions), else one cell per thread (the ordered mode's chunk order).
void residual(fd3_volume* V, int op) {
  Geo G = V->geo();
  if (V->tmaf() && tma_ready(V)) {
    tma_residual(V, op);
    return;
  }
  if (V->quad()) {
    quad_dispatch(V, [&](auto qx, auto k4) {
      constexpr int QX = decltype(qx)::value, K4 = decltype(k4)::value;
      launch_grid(V, "kq_residual", zblocks4<QX>(V->nx, V->ny, V->nz, K4), Z4T, kq_residual<QX, K4>, G,
                  (const unsigned short*)V->codes, (const float*)V->p, (const float*)V->rhs, V->res, V->red(), V->dS,
                  op);
    });
    return;
  }
  if (V->paired()) {
    const int k2 = pick_k2(V->nx, V->ny, V->nz);
    const int zb = zblocks2(V->nx, V->ny, V->nz, k2);
    if (k2 == 8)
      launch_grid(V, "kx_residual<8>", zb, Z2T, kx_residual<8>, G, (const unsigned short*)V->codes, (const float*)V->p,
                  (const float*)V->rhs, V->res, V->red(), V->dS, op);
    else
      launch_grid(V, "kx_residual<4>", zb, Z2T, kx_residual<4>, G, (const unsigned short*)V->codes, (const float*)V->p,
                  (const float*)V->rhs, V->res, V->red(), V->dS, op);
    return;
  }
  DISPATCH(V, k_residual_c, V->n, G, (const unsigned short*)V->codes, (const float*)V->p, (const float*)V->rhs, V->res,
           V->red(), V->dS, op);
}

// u.  One synchronisation.
struct Checks { double actual, all, plain; float be; unsigned long long hash; int status; };

int outer_checks(fd3_volume* V, float k1, Checks* out) {
  Geo G = V->geo();
  residual(V, (int)FIN_ACTUAL);
  if (V->linear) {
    LAUNCH(V, k_correct_linear_uv, (long long)V->nu + V->nv, G, k1, (const float*)V->p, (const float*)V->us,
           (const float*)V->vs, V->u, V->v);
    LAUNCH(V, k_correct_linear_w, V->nw, G, k1, (const float*)V->p, (const float*)V->ws, V->w);
    LAUNCH_G(V, k_reset_diag, 1, 1, V->dS, 7);
    LAUNCH(V, k_div_metric_linear, V->n, G, (const float*)V->u, (const float*)V->v, (const float*)V->w, V->dS);
    LAUNCH_G(V, k_maxabs3, 8 * 148, TPB, (const float*)V->u, V->nu, (const float*)V->v, V->nv, (const float*)V->w,
             V->nw, V->dS, 2);
  } else {
    // the correction, the divergence metric and the largest |u| in one pass (they took four launches:
    // 369 us per outer iteration at 256^3, where a projection runs about four outer iterations)
    LAUNCH_G(V, k_reset_diag, 1, 1, V->dS, 7);
    LAUNCH_G(V, k_correct_metric, cm_blocks(V->nx, V->ny, V->nz), CM_X * CM_Y, G, (const unsigned short*)V->codes, k1,
             (const float*)V->p, (const float*)V->us, (const float*)V->vs, (const float*)V->ws, V->u, V->v, V->w,
             V->dS);
  }
  if (V->linear) {
    LAUNCH(V, k_backward_error_linear, V->n, G, (const float*)V->p, (const float*)V->rhs, (const float*)V->res, V->dS);
    LAUNCH_G(V, k_hash, 592, TPB, V->n, (const float*)V->p, V->dS);
  } else {  // the backward error and the fingerprint in one pass
    LAUNCH_G(V, k_backward_hash, cm_blocks(V->nx, V->ny, V->nz), CM_X * CM_Y, G, (const unsigned short*)V->codes,
             (const float*)V->p, (const float*)V->rhs, (const float*)V->res, V->dS);
  }
  TRY(pull(V));
  const Scalars* S = V->hS;
  // delta3d_mobile.rs:426-432; the linear metric (delta3d.rs:1043-1052) has no velocity floor
  float all = S->fmax[0], plain = S->fmax[1], mx = S->fmax[2];
  float echelle = V->linear ? mx : std::fmax(mx, PROJECTION_VELOCITY_FLOOR);
  float ratio = mx > 0.f ? V->dx / echelle : 0.f;
  out->actual = S->actual;
  out->all = (double)(all * ratio);
  out->plain = (double)(plain * ratio);
  out->be = S->fmax[3];
  out->hash = S->hash;
  out->status = S->status;
  return FD3_OK;
}

__global__ void k_widen(int n, const __half* __restrict__ a, float* __restrict__ b) {
  KSTART();
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c < n) b[c] = __half2float(a[c]);
}

// vk: 6 sqrt(n) / dx^2 in the FP16-storage mode (Scalars::vinv), else 0.
__global__ void k_reset_scalars(Scalars* S, float vk) {
  Scalars z;
  memset(&z, 0, sizeof z);
  z.vk = vk;
  z.vinv = 1.f;
  *S = z;
}
float vscale_k(const fd3_volume* V) {
  return V->half() ? (float)(6.0 * std::sqrt((double)V->n) / ((double)V->dx * (double)V->dx)) : 0.f;
}

// project_mobile3 (delta3d_mobile.rs:465-609), or, with V->linear, project (delta3d.rs:1060-1196):
// the same loop and outer logic on the linear rows, CG or Jacobi-PCG, from p = 0 everywhere.
int project_mobile3(fd3_volume* V, float scale, float k1, uint32_t max_iters, fd3_report* rep) {
  const bool ord = V->ord();
  Geo G = V->geo();
  LAUNCH_G(V, k_reset_scalars, 1, 1, V->dS, vscale_k(V));
  LAUNCH(V, k_divergence, V->n, G, (const float*)V->us, (const float*)V->vs, (const float*)V->ws, V->rhs);
  if (V->linear) {
    const int jacobi = V->cut && V->precondition_cut && V->ny > 1;  // delta3d.rs:1091
    DISPATCH(V, k_rhs_linear, V->n, G, scale, jacobi, V->rhs, V->prec, V->red(), V->dS);
    LAUNCH(V, k_row_codes_linear, V->n, G, V->codes);
    CK(cudaMemsetAsync(V->p, 0, (size_t)V->n * sizeof(float), V->stream));
  } else {
    // the assembly also zeroes p on the dry cells (delta3d_mobile.rs:486-495)
    DISPATCH(V, k_rhs_b2, V->n, G, scale, V->rhs, V->prec, V->red(), V->dS, 1, V->codes, V->p);
    if (V->has_mg) prepare_multigrid(V);
  }
  residual(V, (int)FIN_RR0);
  // With f64 reductions and the loop graph, every outer iteration goes out with one synchronisation;
  // the first is enqueued whole: the prime,
  // the loop (started on the device from the set-up's scalars: it does not run when the host's test
  // would not have started it) and the outer checks, with one synchronisation at their end.  A
  // prime that turns out unneeded changes nothing the checks or the report read; a non-finite
  // set-up stops the loop on the device and is reported after the checks, as before them.
  const bool speculate = !ord && V->mg_on() && V->opt.use_graphs && !V->prof;
  Checks ck{};
  bool have_checks = false;
  if (speculate) {
    prime(V);
    LAUNCH_G(V, k_loop_start_dev, 1, 1, V->dS, max_iters);
    const int mode = V->loop_key();
    if (!V->loop_exec || V->loop_mode != mode || V->loop_stream != V->stream) TRY(build_loop_graph(V));
    CK(cudaGraphLaunch(V->loop_exec, V->stream));
    TRY(outer_checks(V, k1, &ck));
    if (V->hS->status) return V->hS->status;
    V->launches += (unsigned long long)((std::max(V->hS->it, 1u) + 1) / 2) * V->body_nodes;
    have_checks = true;
  } else {
    TRY(pull(V));
    if (V->hS->status) return V->hS->status;
  }
  const double b2 = V->hS->b2;
  double rr = V->hS->rr;
  // tol = 1e-12_f32 (delta3d_mobile.rs:507); tol*b2 in f32 in the reference's arithmetic
  const double tolb2 = ord ? (double)(1e-12f * (float)b2) : 1e-12 * b2;
  bool primed = have_checks;
  uint32_t it = have_checks ? V->hS->it : 0;
  bool floor_stop = false;
  double phys = std::numeric_limits<double>::infinity();
  bool has_checkpoint = false;
  unsigned long long checkpoint = 0;
  uint32_t power = 1, since = 0;
  double actual_rr = 0;
  bool settled = false;
  double settled_d[2] = {0, 0};
  auto above = [&](double r) {
    if (ord) return (float)r > (float)tolb2 || (float)r > (float)phys;
    return r > tolb2 || r > phys;
  };
  for (;;) {
    uint32_t before = have_checks ? 0u : it;
    if (have_checks) {  // the first outer iteration ran whole on the device
      have_checks = false;
      rr = V->hS->rr;
    } else {
    if (b2 > 0 && above(rr) && it < max_iters) {
      if (!primed) {
        prime(V);
        primed = true;
      }
      LAUNCH_G(V, k_loop_start, 1, 1, V->dS, rr, tolb2, phys, it, max_iters);
      V->hS->max_iters = max_iters;
      if (speculate) {  // the loop and the checks behind it, one synchronisation (the checks keep it and rr)
        const int mode = V->loop_key();
        if (!V->loop_exec || V->loop_mode != mode || V->loop_stream != V->stream) TRY(build_loop_graph(V));
        CK(cudaGraphLaunch(V->loop_exec, V->stream));
        TRY(outer_checks(V, k1, &ck));
        if (V->hS->status) return V->hS->status;
        const unsigned ran = V->hS->it > it ? V->hS->it - it : 1;
        V->launches += (unsigned long long)((ran + 1) / 2) * V->body_nodes;
        it = V->hS->it;
        rr = V->hS->rr;
      } else {
        TRY(run_inner(V, it));
        if (V->hS->status) return V->hS->status;
        it = V->hS->it;
        rr = V->hS->rr;
        TRY(outer_checks(V, k1, &ck));
      }
    } else {
      TRY(outer_checks(V, k1, &ck));
    }
    }
    if (ck.status) return ck.status;
    const double actual = ck.actual;
    bool exhausted = it >= max_iters || it == before;
    bool has_measured = false;
    double measured[2] = {0, 0};
    bool converged = ord ? (float)actual <= (float)tolb2 : actual <= tolb2;
    if (converged) {
      if (exhausted) { actual_rr = actual; break; }
      if (ck.plain <= kDivTol) { actual_rr = actual; settled = true; settled_d[0] = ck.all; settled_d[1] = ck.plain; break; }
      has_measured = true; measured[0] = ck.all; measured[1] = ck.plain;
      if (ord) {
        float ratio = (float)(kDivTol / ck.plain);
        phys = (double)((float)actual * ratio * ratio);
      } else {
        double ratio = kDivTol / ck.plain;
        phys = actual * ratio * ratio;
      }
    } else if (exhausted) {
      actual_rr = actual;
      break;
    }
    if (ck.be <= (V->ny == 1 && !V->linear ? kRoundoff2D : kRoundoff3D)) {
      floor_stop = true; actual_rr = actual;
      if (has_measured) { settled = true; settled_d[0] = measured[0]; settled_d[1] = measured[1]; }
      break;
    }
    if (has_checkpoint && checkpoint == ck.hash) {
      floor_stop = true; actual_rr = actual;
      if (has_measured) { settled = true; settled_d[0] = measured[0]; settled_d[1] = measured[1]; }
      break;
    }
    since += 1;
    if (since == power) {
      has_checkpoint = true; checkpoint = ck.hash;
      power = power > 0x7fffffffu ? 0xffffffffu : power * 2;
      since = 0;
    }
    rr = actual;
    prime(V);
  }
  double residual;
  if (ord) residual = b2 > 0 ? (double)std::sqrt((float)actual_rr / (float)b2) : 0.0;
  else residual = b2 > 0 ? std::sqrt(actual_rr / b2) : 0.0;
  // The last checks ran on the final p: their correction and metrics are the reference's tail
  // (delta3d_mobile.rs:592-598).
  double div_all = settled ? settled_d[0] : ck.all, div_plain = settled ? settled_d[1] : ck.plain;
  bool conv = ord ? (float)actual_rr <= (float)tolb2 : actual_rr <= tolb2;
  bool accepted = (conv || floor_stop) && div_plain <= kDivTol;
  memset(rep, 0, sizeof *rep);
  rep->refinements = 0;
  rep->iterations = it;
  rep->degraded = (b2 > 0 && !accepted) ? 1 : 0;
  rep->residual = residual;
  rep->divergence = div_all;
  rep->floor = floor_stop ? 1 : 0;
  rep->backward_error = (double)ck.be;
  rep->divergence_plain = div_plain;
  return FD3_OK;
}

// ---------------------------------------------------------------------------- input validation
__global__ void k_check_finite(long long n, const float* __restrict__ x, int* flag) {
  bool bad = false;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
    bad |= !isfinite(x[q]);
  if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(flag, 1);
}

// A face of a column whose byte in `m` equals `mark` (clear_column_faces, delta3d_sparse.rs:213-233):
// the column's two u faces, two v faces and every w face.
__device__ __forceinline__ bool column_face(const unsigned char* __restrict__ m, unsigned char mark, int nx, int ny,
                                            int axis, int i, int j) {
  if (axis == 0) return (i < nx && m[j * nx + i] == mark) || (i > 0 && m[j * nx + i - 1] == mark);
  if (axis == 1) return (j < ny && m[j * nx + i] == mark) || (j > 0 && m[(j - 1) * nx + i] == mark);
  return m[j * nx + i] == mark;
}

// close_walls (delta3d.rs:666-690): walls, bottom, and faces the cut closes have no velocity;
// then close_sparse_walls (delta3d_sparse.rs:236-247): nor has any face of a column outside the
// sparse set (g.act, 0 for those columns).
__global__ void k_close_walls(Geo g, float* __restrict__ u, float* __restrict__ v, float* __restrict__ w) {
  KSTART();
  const unsigned char* out = g.act;
  int nu = (g.nx + 1) * g.ny * g.nz, nv = g.nx * (g.ny + 1) * g.nz, nw = g.nx * g.ny * (g.nz + 1);
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q < nu) {
    int i = q % (g.nx + 1), j = (q / (g.nx + 1)) % g.ny;
    if (i == 0 || i == g.nx || (g.cut && g.ou[q] == 0.f) || (out && column_face(out, 0, g.nx, g.ny, 0, i, j))) u[q] = 0.f;
    return;
  }
  q -= nu;
  if (q < nv) {
    int i = q % g.nx, j = (q / g.nx) % (g.ny + 1);
    if (j == 0 || j == g.ny || (g.cut && g.ov[q] == 0.f) || (out && column_face(out, 0, g.nx, g.ny, 1, i, j))) v[q] = 0.f;
    return;
  }
  q -= nv;
  if (q < nw) {
    int k = q / (g.nx * g.ny), col = q % (g.nx * g.ny);
    if (k == 0 || (g.cut && g.ow[q] == 0.f) || (out && out[col] == 0)) w[q] = 0.f;
  }
}

// Columns leaving the sparse set go to rest (apply_sparse, delta3d_sparse.rs:181-210): surface,
// roundoff, pressure and every face of the column.  `leave` marks them; vmax collects the largest
// |velocity| cleared, as the bits of a non-negative float (ordered like the integers).
__global__ void k_sparse_leave(Geo g, const unsigned char* __restrict__ leave, float rest, float* __restrict__ eta,
                               float* __restrict__ rof, float* __restrict__ p, float* __restrict__ u,
                               float* __restrict__ v, float* __restrict__ w, int* vmax) {
  KSTART();
  const int nx = g.nx, ny = g.ny, ncol = nx * ny;
  const int nu = (nx + 1) * ny * g.nz, nv = nx * (ny + 1) * g.nz, nw = ncol * (g.nz + 1);
  long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  int cleared = 0;
  if (q < ncol) {
    if (leave[q]) { eta[q] = rest; rof[q] = 0.f; }
  } else if ((q -= ncol) < g.n) {
    if (leave[q % ncol]) p[q] = 0.f;
  } else if ((q -= g.n) < nu) {
    int i = (int)(q % (nx + 1)), j = (int)((q / (nx + 1)) % ny);
    if (column_face(leave, 1, nx, ny, 0, i, j)) { cleared = __float_as_int(fabsf(u[q])); u[q] = 0.f; }
  } else if ((q -= nu) < nv) {
    int i = (int)(q % nx), j = (int)((q / nx) % (ny + 1));
    if (column_face(leave, 1, nx, ny, 1, i, j)) { cleared = __float_as_int(fabsf(v[q])); v[q] = 0.f; }
  } else if ((q -= nv) < nw) {
    if (leave[q % ncol]) { cleared = __float_as_int(fabsf(w[q])); w[q] = 0.f; }
  }
  if (cleared) atomicMax(vmax, cleared);
}

// Geometry copies: fractions, the three aperture families and the floors.
int copy_cut(fd3_volume* V, float* frac, float* ou, float* ov, float* ow, float* floor, const float* sfrac,
             const float* sou, const float* sov, const float* sow, const float* sfloor) {
  CK(cudaMemcpyAsync(frac, sfrac, (size_t)V->n * 4, cudaMemcpyDeviceToDevice, V->stream));
  CK(cudaMemcpyAsync(ou, sou, (size_t)V->nu * 4, cudaMemcpyDeviceToDevice, V->stream));
  CK(cudaMemcpyAsync(ov, sov, (size_t)V->nv * 4, cudaMemcpyDeviceToDevice, V->stream));
  CK(cudaMemcpyAsync(ow, sow, (size_t)V->nw * 4, cudaMemcpyDeviceToDevice, V->stream));
  CK(cudaMemcpyAsync(floor, sfloor, (size_t)V->ncol * 4, cudaMemcpyDeviceToDevice, V->stream));
  return FD3_OK;
}

// solid_columns (delta3d.rs:85-98): the solid volume of each column, (sum over k of base - frac in
// f64, in k order) * dx^3, rounded to f32.
__global__ void k_solid_columns(int nx, int ny, int nz, float dx, const float* __restrict__ base,
                                const float* __restrict__ frac, float* __restrict__ out) {
  KSTART();
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nx * ny) return;
  double s = 0.;
  for (int k = 0; k < nz; ++k) s += (double)(base[(long long)k * nx * ny + c] - frac[(long long)k * nx * ny + c]);
  const double d = (double)dx;
  out[c] = (float)(s * (d * d * d));
}

// delta3d.rs:412-441: a face the new cut closes loses its velocity; a face it opens starts at the
// wall's velocity at the face centre.
__global__ void k_wall_faces(int nx, int ny, int nz, float dx, const float* __restrict__ ou, const float* __restrict__ ov,
                             const float* __restrict__ ow, const float* __restrict__ old_u,
                             const float* __restrict__ old_v, const float* __restrict__ old_w, float* __restrict__ u,
                             float* __restrict__ v, float* __restrict__ w, Rigid R) {
  KSTART();
  const long long nu = (long long)(nx + 1) * ny * nz, nv = (long long)nx * (ny + 1) * nz,
                  nw = (long long)nx * ny * (nz + 1);
  long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (q < nu) {
    const int i = (int)(q % (nx + 1)), t = (int)(q / (nx + 1)), j = t % ny, k = t / ny;
    if (ou[q] == 0.f) u[q] = 0.f;
    else if (old_u[q] == 0.f) u[q] = wall_velocity(R, 0, (float)i * dx, ((float)j + 0.5f) * dx, ((float)k + 0.5f) * dx);
    return;
  }
  q -= nu;
  if (q < nv) {
    const int i = (int)(q % nx), t = (int)(q / nx), j = t % (ny + 1), k = t / (ny + 1);
    if (ov[q] == 0.f) v[q] = 0.f;
    else if (old_v[q] == 0.f) v[q] = wall_velocity(R, 1, ((float)i + 0.5f) * dx, (float)j * dx, ((float)k + 0.5f) * dx);
    return;
  }
  q -= nv;
  if (q < nw) {
    const int i = (int)(q % nx), t = (int)(q / nx), j = t % ny, k = t / ny;
    if (ow[q] == 0.f) w[q] = 0.f;
    else if (old_w[q] == 0.f) w[q] = wall_velocity(R, 2, ((float)i + 0.5f) * dx, ((float)j + 0.5f) * dx, (float)k * dx);
  }
}

// delta3d.rs:443-453: the solid volume a column gains raises its surface, a compensated f32 sum
// on (eta, roundoff); the deposit and the base column volume follow.
__global__ void k_displace_columns(int ncol, float area, const float* __restrict__ cols, float* __restrict__ bcol,
                                   float* __restrict__ bdep, float* __restrict__ eta, float* __restrict__ rof) {
  KSTART();
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncol) return;
  const float nc = cols[c], oc = bcol[c];
  bdep[c] += (nc - oc) / area;
  const float increment = (nc - oc) / area - rof[c];
  const float height = eta[c] + increment;
  rof[c] = (height - eta[c]) - increment;
  eta[c] = height;
  bcol[c] = nc;
}

int check_finite_device(fd3_volume* V, const float* x, long long n, bool* ok) {
  CK(cudaMemsetAsync(V->dflag, 0, sizeof(int), V->stream));
  LAUNCH_G(V, k_check_finite, 592, TPB, n, x, V->dflag);
  CK(cudaMemcpyAsync(V->hflag, V->dflag, sizeof(int), cudaMemcpyDeviceToHost, V->stream));
  TRY(sync(V));
  *ok = *V->hflag == 0;
  return FD3_OK;
}

// ------------------------------------------------------------------------------------ configure
int alloc_state(fd3_volume* V) {
  TRY(dalloc(V, &V->eta, V->ncol)); TRY(dalloc(V, &V->rof, V->ncol));
  TRY(dalloc(V, &V->u, V->nu)); TRY(dalloc(V, &V->v, V->nv)); TRY(dalloc(V, &V->w, V->nw));
  TRY(dalloc(V, &V->us, V->nu)); TRY(dalloc(V, &V->vs, V->nv)); TRY(dalloc(V, &V->ws, V->nw));
  TRY(dalloc(V, &V->p, V->n)); TRY(dalloc(V, &V->rhs, V->n)); TRY(dalloc(V, &V->res, V->n));
  TRY(dalloc(V, &V->dir, V->n)); TRY(dalloc(V, &V->dir2, V->n)); TRY(dalloc(V, &V->tmp, V->n));
  TRY(dalloc(V, &V->prec, V->n));
  float* cq;
  TRY(dalloc(V, &cq, (size_t)(V->n + 1) / 2)); V->codes = (unsigned short*)cq;
  TRY(dalloc(V, &cq, 4)); V->count = (unsigned*)cq;
  TRY(dalloc(V, &V->sv_u, V->nu)); TRY(dalloc(V, &V->sv_v, V->nv)); TRY(dalloc(V, &V->sv_w, V->nw));
  TRY(dalloc(V, &V->sv_p, V->n)); TRY(dalloc(V, &V->sv_eta, V->ncol)); TRY(dalloc(V, &V->sv_rof, V->ncol));
  TRY(dalloc(V, &V->flux_x, (size_t)(V->nx + 1) * V->ny)); TRY(dalloc(V, &V->flux_y, (size_t)V->nx * (V->ny + 1)));
  float* q;
  // one f64 partial per block of the largest reduction launch: linear (one cell per thread),
  // 2.5-D blocked, or the grid-stride update
  V->p64_cap = std::max(std::max(blocks_for(V->n), std::max(zblocks(V->nx, V->ny, V->nz), zblocks2(V->nx, V->ny, V->nz, 4))),
                        UPDATE_BLOCKS);
  TRY(dalloc(V, &q, (size_t)V->p64_cap * 2 + 64)); V->p64 = (double*)q;
  TRY(dalloc(V, &V->p32, (size_t)(V->n + CHUNK - 1) / CHUNK + 64));
  TRY(dalloc(V, &q, sizeof(Scalars) / sizeof(float) + 16)); V->dS = (Scalars*)q;
  TRY(dalloc(V, &q, 16)); V->dflag = (int*)q;
  CK(cudaMallocHost((void**)&V->hS, sizeof(Scalars)));
  CK(cudaMallocHost((void**)&V->hflag, sizeof(int)));
  TRY(dalloc(V, &q, 32)); V->fsc = (double*)q;
  CK(cudaMallocHost((void**)&V->hfsc, 8 * sizeof(double)));
  memset(V->hS, 0, sizeof(Scalars));
  // eta = z0 everywhere (delta3d.rs:255)
  std::vector<float> z0(V->ncol, V->z0);
  CK(cudaMemcpyAsync(V->eta, z0.data(), V->ncol * sizeof(float), cudaMemcpyHostToDevice, V->stream));
  CK(cudaMemcpyAsync(V->sv_eta, z0.data(), V->ncol * sizeof(float), cudaMemcpyHostToDevice, V->stream));
  return sync(V);
}

int configure(const fd3_domain* dom, float rho, float g_eff, fd3_volume** out) {
  if (!dom || !out) return FD3_ERR_INVALID_ARGUMENT;
  uint64_t nx = dom->nx, ny = dom->ny, nz = dom->nz;
  float dx = dom->dx;
  // delta3d.rs:212-243
  if (nx == 0 || ny == 0 || nz == 0 || !std::isfinite(dx) || dx <= 0.f) return FD3_ERR_DOMAIN;
  if (!std::isfinite(rho) || rho <= 0.f || !std::isfinite(g_eff)) return FD3_ERR_NOT_FINITE;
  // Index arithmetic on the device is 32-bit: every array must hold fewer than 2^31 entries.
  const uint64_t lim = (1ull << 31) - 1;
  if (nx > lim || ny > lim || nz > lim) return FD3_ERR_DOMAIN;
  unsigned __int128 cells = (unsigned __int128)nx * ny * nz;
  unsigned __int128 nw = (unsigned __int128)nx * ny * (nz + 1);
  unsigned __int128 nu = (unsigned __int128)(nx + 1) * ny * nz;
  unsigned __int128 nv = (unsigned __int128)nx * (ny + 1) * nz;
  if (cells > lim || nw > lim || nu > lim || nv > lim) return FD3_ERR_DOMAIN;
  float z0 = (float)nz * dx;
  if (!(std::isfinite(z0) && std::isfinite((float)nx * dx) && std::isfinite((float)ny * dx))) return FD3_ERR_DOMAIN;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return FD3_ERR_NO_DEVICE;
  fd3_volume* V = new (std::nothrow) fd3_volume();
  if (!V) return FD3_ERR_OUT_OF_MEMORY;
  cudaGetDevice(&V->device);
  if (cudaStreamCreateWithFlags(&V->own_stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete V;
    return cuda_fail(cudaGetLastError(), "cudaStreamCreateWithFlags", __LINE__);
  }
  V->stream = V->own_stream;
  V->nx = (int)nx; V->ny = (int)ny; V->nz = (int)nz;
  V->n = (int)cells; V->nu = (int)nu; V->nv = (int)nv; V->nw = (int)nw; V->ncol = (int)(nx * ny);
  V->dx = dx; V->rho = rho; V->g = g_eff; V->z0 = z0; V->rest = z0;
  V->opt.reduction = FD3_REDUCE_F64;
  V->opt.mg_max_levels = 0;
  V->opt.use_graphs = 1;
  int e = alloc_state(V);
  if (e) { release(V); delete V; return e; }
  *out = V;
  return FD3_OK;
}

int build_bottom_cut(fd3_volume* V, const float* bottom) {
  TRY(dalloc(V, &V->frac, V->n)); TRY(dalloc(V, &V->ou, V->nu)); TRY(dalloc(V, &V->ov, V->nv));
  TRY(dalloc(V, &V->ow, V->nw)); TRY(dalloc(V, &V->floor_, V->ncol));
  float *dbottom, *corner;
  TRY(dalloc(V, &dbottom, V->ncol));
  TRY(dalloc(V, &corner, (size_t)(V->nx + 1) * (V->ny + 1)));
  CK(cudaMemcpyAsync(dbottom, bottom, V->ncol * sizeof(float), cudaMemcpyHostToDevice, V->stream));
  LAUNCH(V, k_corners, (long long)(V->nx + 1) * (V->ny + 1), V->nx, V->ny, (const float*)dbottom, corner);
  CutGeo C{V->nx, V->ny, V->nz, V->dx, corner, V->frac, V->ou, V->ov, V->ow, V->floor_};
  LAUNCH(V, k_cut_frac, V->n, C);
  LAUNCH(V, k_cut_faces, (long long)V->nu + V->nv + V->nw, C);
  LAUNCH(V, k_seal_isolated, V->n, C);
  LAUNCH(V, k_floor, V->ncol, C);
  V->cut = true;
  return sync(V);
}

int validate_bottom(const fd3_domain* dom, const float* bottom, size_t len) {
  uint64_t cols;
  if (__builtin_mul_overflow(dom->nx, dom->ny, &cols)) return FD3_ERR_DOMAIN;
  if (len != cols) return FD3_ERR_SHAPE;
  if (!bottom && len) return FD3_ERR_INVALID_ARGUMENT;
  float z0 = (float)dom->nz * dom->dx;
  for (size_t q = 0; q < len; ++q)
    if (!std::isfinite(bottom[q]) || bottom[q] < 0.f || bottom[q] >= z0) return FD3_ERR_NOT_FINITE;
  return FD3_OK;
}


int in_bounds(fd3_volume* V, bool* ok) {
  CK(cudaMemsetAsync(V->dflag, 0, sizeof(int), V->stream));
  LAUNCH(V, k_in_bounds, V->ncol, V->geo(), (const float*)V->floor_, V->dflag);
  CK(cudaMemcpyAsync(V->hflag, V->dflag, sizeof(int), cudaMemcpyDeviceToHost, V->stream));
  TRY(sync(V));
  *ok = *V->hflag == 0;
  return FD3_OK;
}

int save_state(fd3_volume* V) {
  CK(cudaMemcpyAsync(V->sv_u, V->u, (size_t)V->nu * 4, cudaMemcpyDeviceToDevice, V->stream));
  CK(cudaMemcpyAsync(V->sv_v, V->v, (size_t)V->nv * 4, cudaMemcpyDeviceToDevice, V->stream));
  CK(cudaMemcpyAsync(V->sv_w, V->w, (size_t)V->nw * 4, cudaMemcpyDeviceToDevice, V->stream));
  CK(cudaMemcpyAsync(V->sv_p, V->p, (size_t)V->n * 4, cudaMemcpyDeviceToDevice, V->stream));
  CK(cudaMemcpyAsync(V->sv_eta, V->eta, (size_t)V->ncol * 4, cudaMemcpyDeviceToDevice, V->stream));
  CK(cudaMemcpyAsync(V->sv_rof, V->rof, (size_t)V->ncol * 4, cudaMemcpyDeviceToDevice, V->stream));
  return FD3_OK;
}

void restore_state(fd3_volume* V) {
  cudaMemcpyAsync(V->u, V->sv_u, (size_t)V->nu * 4, cudaMemcpyDeviceToDevice, V->stream);
  cudaMemcpyAsync(V->v, V->sv_v, (size_t)V->nv * 4, cudaMemcpyDeviceToDevice, V->stream);
  cudaMemcpyAsync(V->w, V->sv_w, (size_t)V->nw * 4, cudaMemcpyDeviceToDevice, V->stream);
  cudaMemcpyAsync(V->p, V->sv_p, (size_t)V->n * 4, cudaMemcpyDeviceToDevice, V->stream);
  cudaMemcpyAsync(V->eta, V->sv_eta, (size_t)V->ncol * 4, cudaMemcpyDeviceToDevice, V->stream);
  cudaMemcpyAsync(V->rof, V->sv_rof, (size_t)V->ncol * 4, cudaMemcpyDeviceToDevice, V->stream);
  cudaStreamSynchronize(V->stream);
}

// The body of step_surface_mobile after the saves (delta3d_mobile.rs:857-911).
int step_body(fd3_volume* V, float scale, float correction, float transport, float advection, uint32_t max_iters,
              fd3_report* rep) {
  Geo G = V->geo();
  LAUNCH(V, k_advect, (long long)V->nu + V->nv + V->nw, G, advection, (const float*)V->u, (const float*)V->v,
         (const float*)V->w, V->us, V->vs, V->ws);
  if (V->advection_correction)  // delta3d_mobile.rs:858-860
    LAUNCH(V, k_correct_advection, (long long)V->nu + V->nv + V->nw, G, advection, (const float*)V->u,
           (const float*)V->v, (const float*)V->w, V->us, V->vs, V->ws);
  TRY(project_mobile3(V, scale, correction, max_iters, rep));
  if (rep->degraded) {
    V->has_refused = true;
    V->refused = *rep;
    return FD3_ERR_CONVERGENCE;
  }
  LAUNCH(V, k_extrapolate, 3LL * V->ncol, G, V->u, V->v, V->w);
  LAUNCH(V, k_transport_flux, (long long)(V->nx + 1) * V->ny + (long long)V->nx * (V->ny + 1), G, (const float*)V->u,
         (const float*)V->v, V->flux_x, V->flux_y);
  LAUNCH(V, k_transport_eta, V->ncol, G, transport, (const float*)V->flux_x, (const float*)V->flux_y, V->eta, V->rof);
  // every field finite (delta3d_mobile.rs:885-906)
  struct { const float* x; long long n; } fields[] = {
      {V->u, V->nu}, {V->v, V->nv}, {V->w, V->nw}, {V->p, V->n}, {V->eta, V->ncol}, {V->rof, V->ncol},
      {V->us, V->nu}, {V->vs, V->nv}, {V->ws, V->nw}, {V->rhs, V->n}, {V->res, V->n}, {V->dir, V->n},
      {V->tmp, V->n}, {V->prec, V->n}};
  CK(cudaMemsetAsync(V->dflag, 0, sizeof(int), V->stream));
  for (auto& f : fields) {
    LAUNCH_G(V, k_check_finite, 592, TPB, f.n, f.x, V->dflag);
  }
  CK(cudaMemcpyAsync(V->hflag, V->dflag, sizeof(int), cudaMemcpyDeviceToHost, V->stream));
  TRY(sync(V));
  if (*V->hflag) return FD3_ERR_NOT_FINITE;
  if (!std::isfinite(rep->residual) || !std::isfinite(rep->divergence)) return FD3_ERR_NOT_FINITE;
  bool ok;
  TRY(in_bounds(V, &ok));
  if (!ok) return FD3_ERR_DOMAIN;
  return FD3_OK;
}

// step_surface_mobile (delta3d_mobile.rs:819-927).
int step_surface_mobile(fd3_volume* V, uint64_t duration_us, uint32_t max_iters, fd3_report* rep) {
  if (duration_us == 0 || duration_us > (1ull << 53)) return FD3_ERR_NOT_FINITE;
  double dt = (double)duration_us * 1e-6;
  bool ok;
  TRY(in_bounds(V, &ok));
  if (V->g <= 0.f || dt * dt * (double)V->g / (double)V->dx > 1. || !ok) return FD3_ERR_DOMAIN;
  float scale = (float)(-(double)V->rho / dt);
  float correction = (float)(dt / (double)V->rho);
  float transport = (float)(dt / (double)V->dx);
  float advection = (float)dt;
  if (!std::isfinite(scale) || !std::isfinite(correction) || correction == 0.f || !std::isfinite(transport) ||
      transport == 0.f || !(advection > 0.f))
    return FD3_ERR_NOT_FINITE;
  TRY(save_state(V));
  int e = step_body(V, scale, correction, transport, advection, max_iters, rep);
  if (e) restore_state(V);
  return e;
}

// The linear path's projection of the prediction in us/vs/ws (V->linear for its duration).
int project_linear(fd3_volume* V, float scale, float k1, uint32_t max_iters, fd3_report* rep) {
  V->linear = true;
  int e = project_mobile3(V, scale, k1, max_iters, rep);
  V->linear = false;
  return e;
}

// linear (delta3d.rs:1255-1357) after the saves, without a sponge or a graded column.
int linear_body(fd3_volume* V, float scale, float correction, float transport, uint32_t max_iters, fd3_report* rep) {
  if (V->cut) {  // the lid must stay fully open (delta3d.rs:1261-1268)
    CK(cudaMemsetAsync(V->dflag, 0, sizeof(int), V->stream));
    LAUNCH(V, k_lid_open, V->ncol, V->geo(), V->dflag);
    CK(cudaMemcpyAsync(V->hflag, V->dflag, sizeof(int), cudaMemcpyDeviceToHost, V->stream));
    TRY(sync(V));
    if (*V->hflag) return FD3_ERR_DOMAIN;
  }
  CK(cudaMemcpyAsync(V->us, V->u, (size_t)V->nu * 4, cudaMemcpyDeviceToDevice, V->stream));
  CK(cudaMemcpyAsync(V->vs, V->v, (size_t)V->nv * 4, cudaMemcpyDeviceToDevice, V->stream));
  CK(cudaMemcpyAsync(V->ws, V->w, (size_t)V->nw * 4, cudaMemcpyDeviceToDevice, V->stream));
  TRY(project_linear(V, scale, correction, max_iters, rep));
  if (rep->degraded) return FD3_ERR_CONVERGENCE;
  LAUNCH(V, k_linear_transport, V->ncol, V->geo(), transport, (const float*)V->u, (const float*)V->v, V->eta, V->rof);
  // every field finite (delta3d.rs:1347-1353)
  struct { const float* x; long long n; } fields[] = {
      {V->u, V->nu}, {V->v, V->nv}, {V->w, V->nw}, {V->p, V->n}, {V->eta, V->ncol}, {V->rof, V->ncol},
      {V->rhs, V->n}, {V->res, V->n}, {V->dir, V->n}, {V->tmp, V->n}};
  CK(cudaMemsetAsync(V->dflag, 0, sizeof(int), V->stream));
  for (auto& f : fields) {
    LAUNCH_G(V, k_check_finite, 592, TPB, f.n, f.x, V->dflag);
  }
  CK(cudaMemcpyAsync(V->hflag, V->dflag, sizeof(int), cudaMemcpyDeviceToHost, V->stream));
  TRY(sync(V));
  if (*V->hflag) return FD3_ERR_NOT_FINITE;
  if (!std::isfinite(rep->residual) || !std::isfinite(rep->divergence)) return FD3_ERR_NOT_FINITE;
  return FD3_OK;
}

// step_surface_linear (delta3d.rs:1209-1253).
int step_surface_linear(fd3_volume* V, uint64_t duration_us, uint32_t max_iters, fd3_report* rep) {
  if (duration_us == 0 || duration_us > (1ull << 53)) return FD3_ERR_NOT_FINITE;
  double dt = (double)duration_us * 1e-6;
  if (V->g <= 0.f || dt * dt * (double)V->g / (double)V->dx > 1.) return FD3_ERR_DOMAIN;
  float scale = (float)(-(double)V->rho / dt);
  float correction = (float)(dt / (double)V->rho);
  float transport = (float)(dt / (double)V->dx);
  if (!std::isfinite(scale) || !std::isfinite(correction) || correction == 0.f || !std::isfinite(transport) ||
      transport == 0.f)
    return FD3_ERR_NOT_FINITE;
  TRY(save_state(V));
  int e = linear_body(V, scale, correction, transport, max_iters, rep);
  if (e) restore_state(V);
  return e;
}

}  // namespace

// =============================================================================== C ABI
extern "C" {

const char* fd3_version(void) { return "fluidisim_b200 delta3d 0.1 (sm_100a)"; }
const char* fd3_last_cuda_error(void) { return g_last_cuda_error.c_str(); }

int fd3_status_name(int status, char* buf, size_t len) {
  const char* s;
  switch (status) {
    case FD3_OK: s = "Ok"; break;
    case FD3_ERR_DOMAIN: s = "Domain"; break;
    case FD3_ERR_NOT_FINITE: s = "NotFinite"; break;
    case FD3_ERR_SHAPE: s = "Shape"; break;
    case FD3_ERR_BUDGET: s = "Budget"; break;
    case FD3_ERR_CLOCK: s = "Clock"; break;
    case FD3_ERR_CONVERGENCE: s = "Convergence"; break;
    case FD3_ERR_BACKGROUND_CONTEXT: s = "BackgroundContext"; break;
    case FD3_ERR_NON_PLANAR: s = "NonPlanar"; break;
    case FD3_ERR_CUDA: s = "Cuda"; break;
    case FD3_ERR_NO_DEVICE: s = "NoDevice"; break;
    case FD3_ERR_INVALID_ARGUMENT: s = "InvalidArgument"; break;
    case FD3_ERR_OUT_OF_MEMORY: s = "OutOfMemory"; break;
    default: s = "Unknown"; break;
  }
  if (buf && len) { strncpy(buf, s, len - 1); buf[len - 1] = 0; }
  return FD3_OK;
}

int fd3_configure(const fd3_domain* domain, float rho, float g_eff, fd3_volume** out) {
  return configure(domain, rho, g_eff, out);
}

// delta3d.rs:300-321
int fd3_configure_with_bottom(const fd3_domain* domain, float rho, float g_eff, const float* bottom, size_t len,
                              fd3_volume** out) {
  if (!domain || !out) return FD3_ERR_INVALID_ARGUMENT;
  TRY(validate_bottom(domain, bottom, len));
  fd3_volume* V;
  TRY(configure(domain, rho, g_eff, &V));
  int e = build_bottom_cut(V, bottom);
  if (e) { release(V); delete V; return e; }
  *out = V;
  return FD3_OK;
}

// delta3d.rs:327-365
int fd3_configure_with_solid(const fd3_domain* domain, float rho, float g_eff, const float* bottom, size_t blen,
                             const float* solid, size_t slen, fd3_volume** out) {
  if (!domain || !out) return FD3_ERR_INVALID_ARGUMENT;
  unsigned __int128 nodes = (unsigned __int128)(domain->nx + 1) * (domain->ny + 1) * (domain->nz + 1);
  if (nodes > (unsigned __int128)SIZE_MAX) return FD3_ERR_DOMAIN;
  if (slen != (size_t)nodes) return FD3_ERR_SHAPE;
  if (!solid && slen) return FD3_ERR_INVALID_ARGUMENT;
  for (size_t q = 0; q < slen; ++q)
    if (!std::isfinite(solid[q])) return FD3_ERR_NOT_FINITE;
  fd3_volume* V;
  TRY(fd3_configure_with_bottom(domain, rho, g_eff, bottom, blen, &V));
  auto fail = [&](int e) { release(V); delete V; return e; };
  float* dsdf;
  int e = dalloc(V, &dsdf, slen);
  if (e) return fail(e);
  if (cudaMemcpyAsync(dsdf, solid, slen * sizeof(float), cudaMemcpyHostToDevice, V->stream) != cudaSuccess)
    return fail(cuda_fail(cudaGetLastError(), "solid upload", __LINE__));
  SolidGeo S{V->nx, V->ny, V->nz, V->dx, dsdf, 0};
  cudaMemsetAsync(V->dflag, 0, sizeof(int), V->stream);
  long long all = (long long)V->n + V->nu + V->nv + V->nw;
  LAUNCH(V, k_check_solid, all, S, (const float*)V->frac, (const float*)V->ou, (const float*)V->ov, (const float*)V->ow, V->dflag);
  cudaMemcpyAsync(V->hflag, V->dflag, sizeof(int), cudaMemcpyDeviceToHost, V->stream);
  if ((e = sync(V))) return fail(e);
  if (*V->hflag) return fail(FD3_ERR_DOMAIN);
  // the bottom-only cut, kept as the base (delta3d.rs:359-363)
  V->sdf = dsdf;
  if ((e = dalloc(V, &V->bfrac, V->n)) || (e = dalloc(V, &V->bou, V->nu)) || (e = dalloc(V, &V->bov, V->nv)) ||
      (e = dalloc(V, &V->bow, V->nw)) || (e = dalloc(V, &V->bfloor, V->ncol)) || (e = dalloc(V, &V->bcol, V->ncol)) ||
      (e = dalloc(V, &V->bdep, V->ncol)))
    return fail(e);
  if ((e = copy_cut(V, V->bfrac, V->bou, V->bov, V->bow, V->bfloor, V->frac, V->ou, V->ov, V->ow, V->floor_)))
    return fail(e);
  LAUNCH(V, k_add_solid, all, S, V->frac, V->ou, V->ov, V->ow, V->floor_);
  CutGeo C{V->nx, V->ny, V->nz, V->dx, nullptr, V->frac, V->ou, V->ov, V->ow, V->floor_};
  LAUNCH(V, k_seal_isolated, V->n, C);
  LAUNCH(V, k_solid_columns, V->ncol, V->nx, V->ny, V->nz, V->dx, (const float*)V->bfrac, (const float*)V->frac,
         V->bcol);
  if ((e = sync(V))) return fail(e);
  *out = V;
  return FD3_OK;
}

// set_solid_rigid (delta3d.rs:382-509).  Volumes of this API carry a solid that may not reach the
// lid layer (configure_with_solid: piercing = false, check_solid), so no lid face is ever cut and
// the partial-lid transfer of delta3d.rs:460-503 moves nothing; it is not carried out.  The cut
// is redone from the base on the device: k_check_solid against the base, the base copied back,
// k_add_solid and k_seal_isolated; then the faces' velocities, the solid volume per column and
// the compensated rise of the surface.  The previous apertures go to the saved-velocity buffers,
// free between steps as in the reference, and the new column volumes to rhs.
int fd3_set_solid_rigid(fd3_volume* V, const float* solid, size_t len, const float* velocity, const float* angular,
                        const float* center) {
  if (!V || !solid || !velocity || !angular || !center) return FD3_ERR_INVALID_ARGUMENT;
  if (len != (size_t)(V->nx + 1) * (V->ny + 1) * (V->nz + 1)) return FD3_ERR_SHAPE;
  for (int a = 0; a < 3; ++a)
    if (!std::isfinite(velocity[a]) || !std::isfinite(angular[a]) || !std::isfinite(center[a]))
      return FD3_ERR_NOT_FINITE;
  if (!V->sdf) return FD3_ERR_DOMAIN;
  CK(cudaMemcpyAsync(V->sdf, solid, len * sizeof(float), cudaMemcpyHostToDevice, V->stream));
  bool ok = false;
  TRY(check_finite_device(V, V->sdf, (long long)len, &ok));
  if (!ok) return FD3_ERR_NOT_FINITE;
  SolidGeo S{V->nx, V->ny, V->nz, V->dx, V->sdf, 0};
  const long long all = (long long)V->n + V->nu + V->nv + V->nw;
  CK(cudaMemsetAsync(V->dflag, 0, sizeof(int), V->stream));
  LAUNCH(V, k_check_solid, all, S, (const float*)V->bfrac, (const float*)V->bou, (const float*)V->bov,
         (const float*)V->bow, V->dflag);
  CK(cudaMemcpyAsync(V->hflag, V->dflag, sizeof(int), cudaMemcpyDeviceToHost, V->stream));
  TRY(sync(V));
  if (*V->hflag) return FD3_ERR_DOMAIN;
  CK(cudaMemcpyAsync(V->sv_u, V->ou, (size_t)V->nu * 4, cudaMemcpyDeviceToDevice, V->stream));
  CK(cudaMemcpyAsync(V->sv_v, V->ov, (size_t)V->nv * 4, cudaMemcpyDeviceToDevice, V->stream));
  CK(cudaMemcpyAsync(V->sv_w, V->ow, (size_t)V->nw * 4, cudaMemcpyDeviceToDevice, V->stream));
  TRY(copy_cut(V, V->frac, V->ou, V->ov, V->ow, V->floor_, V->bfrac, V->bou, V->bov, V->bow, V->bfloor));
  LAUNCH(V, k_add_solid, all, S, V->frac, V->ou, V->ov, V->ow, V->floor_);
  CutGeo C{V->nx, V->ny, V->nz, V->dx, nullptr, V->frac, V->ou, V->ov, V->ow, V->floor_};
  LAUNCH(V, k_seal_isolated, V->n, C);
  Rigid R;
  for (int a = 0; a < 3; ++a) { R.v[a] = velocity[a]; R.w[a] = angular[a]; R.c[a] = center[a]; }
  V->motion = R;
  const bool spins = angular[0] != 0.f || angular[1] != 0.f || angular[2] != 0.f;
  const bool moves = velocity[0] != 0.f || velocity[1] != 0.f || velocity[2] != 0.f;
  V->wall = spins ? 2 : (moves ? 1 : 0);
  LAUNCH(V, k_wall_faces, (long long)V->nu + V->nv + V->nw, V->nx, V->ny, V->nz, V->dx, (const float*)V->ou,
         (const float*)V->ov, (const float*)V->ow, (const float*)V->sv_u, (const float*)V->sv_v,
         (const float*)V->sv_w, V->u, V->v, V->w, R);
  LAUNCH(V, k_solid_columns, V->ncol, V->nx, V->ny, V->nz, V->dx, (const float*)V->bfrac, (const float*)V->frac,
         V->rhs);
  LAUNCH(V, k_displace_columns, V->ncol, V->ncol, V->dx * V->dx, (const float*)V->rhs, V->bcol, V->bdep, V->eta,
         V->rof);
  return sync(V);
}

// Volume3::set_solid (delta3d.rs:376-378): set_solid_rigid without rotation.
int fd3_set_solid(fd3_volume* V, const float* solid, size_t len, const float* velocity) {
  const float zero[3] = {0.f, 0.f, 0.f};
  return fd3_set_solid_rigid(V, solid, len, velocity, zero, zero);
}

void fd3_destroy(fd3_volume* v) {
  if (!v) return;
  if (v->stream) cudaStreamSynchronize(v->stream);
  release(v);
  delete v;
}

int fd3_set_options(fd3_volume* v, const fd3_options* o) {
  if (!v || !o) return FD3_ERR_INVALID_ARGUMENT;
  if (o->reduction > 1 || o->kernels > 5 || o->no_overlap > 1 || o->storage > 1 || o->no_tile_skip > 1)
    return FD3_ERR_DOMAIN;
  if (o->kernels == 4 && (v->nx % 4 != 0 || o->storage == FD3_STORAGE_F16)) return FD3_ERR_DOMAIN;
  if (o->kernels == 5 && (v->nx % 8 != 0 || o->storage == FD3_STORAGE_F16)) return FD3_ERR_DOMAIN;
  // FP16 storage runs on the paired fine kernels: f64 reductions, kernels = 0 or 3 and an even nx
  if (o->storage == FD3_STORAGE_F16 &&
      (o->reduction != FD3_REDUCE_F64 || (o->kernels != 0 && o->kernels != 3) || v->nx % 2 != 0))
    return FD3_ERR_DOMAIN;
  v->opt = *o;
  return FD3_OK;
}

int fd3_get_options(const fd3_volume* v, fd3_options* o) {
  if (!v || !o) return FD3_ERR_INVALID_ARGUMENT;
  *o = v->opt;
  return FD3_OK;
}

int fd3_set_stream(fd3_volume* v, void* stream) {
  if (!v) return FD3_ERR_INVALID_ARGUMENT;
  TRY(sync(v));
  v->stream = stream ? (cudaStream_t)stream : v->own_stream;
  if (v->loop_exec) { cudaGraphExecDestroy(v->loop_exec); v->loop_exec = nullptr; }
  return FD3_OK;
}

// delta3d_multigrid.rs:339-349: coarse levels while all dims are even and >= 4.
int fd3_enable_multigrid(fd3_volume* V) {
  if (!V) return FD3_ERR_INVALID_ARGUMENT;
  if (V->has_mg) return FD3_OK;
  TRY(dalloc(V, &V->z, V->n));
  TRY(dalloc(V, &V->z2, V->n));
  int x = V->nx, y = V->ny, zz = V->nz;
  float h = V->dx;
  while (x % 2 == 0 && y % 2 == 0 && zz % 2 == 0 && x >= 4 && y >= 4 && zz >= 4 &&
         (V->opt.mg_max_levels == 0 || V->levels.size() < V->opt.mg_max_levels)) {
    int cx = x / 2, cy = y / 2, cz = zz / 2;
    h *= 2.f;
    Lev L{};
    L.nx = cx; L.ny = cy; L.nz = cz; L.n = cx * cy * cz;
    L.inv = 1.f / (h * h);
    TRY(dalloc(V, &L.ou, (size_t)(cx + 1) * cy * cz));
    TRY(dalloc(V, &L.ov, (size_t)cx * (cy + 1) * cz));
    TRY(dalloc(V, &L.ow, (size_t)cx * cy * (cz + 1)));
    TRY(dalloc(V, &L.kind, L.n)); TRY(dalloc(V, &L.diag, L.n));
    TRY(dalloc(V, &L.x, L.n)); TRY(dalloc(V, &L.x2, L.n)); TRY(dalloc(V, &L.r, L.n)); TRY(dalloc(V, &L.t, L.n));
    float* cq;
    TRY(dalloc(V, &cq, (size_t)(L.n + 1) / 2)); L.code = (unsigned short*)cq;
    V->levels.push_back(L);
    x = cx; y = cy; zz = cz;
  }
  V->tail_first = (int)V->levels.size();
  while (V->tail_first > 0 && V->levels[V->tail_first - 1].n <= TAIL_MAX_CELLS) --V->tail_first;
  V->tail_reg = (int)V->levels.size() - V->tail_first <= TAIL_REG_LEVELS;
  for (size_t l = V->tail_first; l < V->levels.size(); ++l) V->tail_reg = V->tail_reg && V->levels[l].n <= TAIL_REG_THREADS;
  // shared-memory tail when every tail level fits (at most 200 KiB of the 227 KiB per block)
  V->tail_smem_bytes = 0;
  if (V->tail_first < (int)V->levels.size() && (int)V->levels.size() - V->tail_first <= MAX_TAIL_LEVELS) {
    size_t floats = 0;
    for (size_t l = V->tail_first; l < V->levels.size(); ++l)
      floats += tail_level_floats(V->levels[l].nx, V->levels[l].ny, V->levels[l].nz);
    if (floats * sizeof(float) <= 200 * 1024) {
      V->tail_smem_bytes = floats * sizeof(float);
      // the largest size any volume may ask for: the attribute is per function, shared by every volume
      CK(cudaFuncSetAttribute(k_coarse_tail_smem, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    }
  }
  if (!V->levels.empty()) {
    float* q;
    TRY(dalloc(V, &q, (V->levels.size() * sizeof(Lev) + 3) / 4));
    V->dlev = (Lev*)q;
    CK(cudaMemcpyAsync(V->dlev, V->levels.data(), V->levels.size() * sizeof(Lev), cudaMemcpyHostToDevice, V->stream));
  }
  V->has_mg = true;
  return sync(V);
}

int fd3_multigrid_levels(const fd3_volume* v) { return v && v->has_mg ? (int)v->levels.size() : -1; }

// sparse_surface_ok (delta3d_sparse.rs:327-332): outside the set the surface is `rest`, to the bit.
static bool sparse_surface_ok(const fd3_volume* V, const float* eta, float rest) {
  if (!V->sparse) return true;
  uint32_t rb;
  std::memcpy(&rb, &rest, 4);
  for (int c = 0; c < V->ncol; ++c) {
    uint32_t eb;
    std::memcpy(&eb, eta + c, 4);
    if (!V->hact[c] && eb != rb) return false;
  }
  return true;
}

// delta3d_mobile.rs:9-25
int fd3_set_free_surface(fd3_volume* V, const float* eta, size_t len, float rest) {
  if (!V || (!eta && len)) return FD3_ERR_INVALID_ARGUMENT;
  if (len != (size_t)V->ncol) return FD3_ERR_SHAPE;
  if (!std::isfinite(rest)) return FD3_ERR_NOT_FINITE;
  for (size_t q = 0; q < len; ++q)
    if (!std::isfinite(eta[q])) return FD3_ERR_NOT_FINITE;
  if (!sparse_surface_ok(V, eta, rest)) return FD3_ERR_DOMAIN;  // delta3d_mobile.rs:16-19
  CK(cudaMemcpyAsync(V->eta, eta, len * sizeof(float), cudaMemcpyHostToDevice, V->stream));
  CK(cudaMemsetAsync(V->rof, 0, len * sizeof(float), V->stream));
  CK(cudaMemsetAsync(V->p, 0, (size_t)V->n * sizeof(float), V->stream));
  V->rest = rest;
  return sync(V);
}

// delta3d.rs:614-628
int fd3_set_surface(fd3_volume* V, const float* eta, size_t len) {
  if (!V || (!eta && len)) return FD3_ERR_INVALID_ARGUMENT;
  if (len != (size_t)V->ncol) return FD3_ERR_SHAPE;
  for (size_t q = 0; q < len; ++q)
    if (!std::isfinite(eta[q])) return FD3_ERR_NOT_FINITE;
  if (!sparse_surface_ok(V, eta, V->rest)) return FD3_ERR_DOMAIN;  // delta3d.rs:621-624
  CK(cudaMemcpyAsync(V->eta, eta, len * sizeof(float), cudaMemcpyHostToDevice, V->stream));
  CK(cudaMemsetAsync(V->rof, 0, len * sizeof(float), V->stream));
  return sync(V);
}

// delta3d.rs:631-645: the faces are staged in us/vs/ws, checked on the device, then published.
// The staged faces are checked with one flag and one host round trip for the three arrays, then
// copied into u, v, w (the published fields, which fd3_device_fields exposes: the call returns once
// they are written).
static int set_velocity_staged(fd3_volume* V) {
  CK(cudaMemsetAsync(V->dflag, 0, sizeof(int), V->stream));
  LAUNCH_G(V, k_check_finite, 592, TPB, (long long)V->nu, (const float*)V->us, V->dflag);
  LAUNCH_G(V, k_check_finite, 592, TPB, (long long)V->nv, (const float*)V->vs, V->dflag);
  LAUNCH_G(V, k_check_finite, 592, TPB, (long long)V->nw, (const float*)V->ws, V->dflag);
  CK(cudaMemcpyAsync(V->hflag, V->dflag, sizeof(int), cudaMemcpyDeviceToHost, V->stream));
  TRY(sync(V));
  if (*V->hflag != 0) return FD3_ERR_NOT_FINITE;
  CK(cudaMemcpyAsync(V->u, V->us, (size_t)V->nu * 4, cudaMemcpyDeviceToDevice, V->stream));
  CK(cudaMemcpyAsync(V->v, V->vs, (size_t)V->nv * 4, cudaMemcpyDeviceToDevice, V->stream));
  CK(cudaMemcpyAsync(V->w, V->ws, (size_t)V->nw * 4, cudaMemcpyDeviceToDevice, V->stream));
  LAUNCH(V, k_close_walls, (long long)V->nu + V->nv + V->nw, V->geo(), V->u, V->v, V->w);
  return sync(V);
}

int fd3_set_velocity(fd3_volume* V, const float* u, size_t nu, const float* vv, size_t nv, const float* w, size_t nw) {
  if (!V || !u || !vv || !w) return FD3_ERR_INVALID_ARGUMENT;
  if (nu != (size_t)V->nu || nv != (size_t)V->nv || nw != (size_t)V->nw) return FD3_ERR_SHAPE;
  CK(cudaMemcpyAsync(V->us, u, nu * 4, cudaMemcpyHostToDevice, V->stream));
  CK(cudaMemcpyAsync(V->vs, vv, nv * 4, cudaMemcpyHostToDevice, V->stream));
  CK(cudaMemcpyAsync(V->ws, w, nw * 4, cudaMemcpyHostToDevice, V->stream));
  return set_velocity_staged(V);
}

int fd3_set_velocity_device(fd3_volume* V, const float* u, const float* vv, const float* w) {
  if (!V || !u || !vv || !w) return FD3_ERR_INVALID_ARGUMENT;
  CK(cudaMemcpyAsync(V->us, u, (size_t)V->nu * 4, cudaMemcpyDeviceToDevice, V->stream));
  CK(cudaMemcpyAsync(V->vs, vv, (size_t)V->nv * 4, cudaMemcpyDeviceToDevice, V->stream));
  CK(cudaMemcpyAsync(V->ws, w, (size_t)V->nw * 4, cudaMemcpyDeviceToDevice, V->stream));
  return set_velocity_staged(V);
}

// ------------------------------------------------------------------------------- sparse sets
// Geo::tiles from the host copy of the set: 1 for a 32 x 8 tile of columns with a column in it.
static int upload_tiles(fd3_volume* V) {
  const int ntx = (V->nx + TILE_X - 1) / TILE_X, nty = (V->ny + TILE_Y - 1) / TILE_Y;
  std::vector<unsigned char> t((size_t)ntx * nty, 0);
  for (int j = 0; j < V->ny; ++j)
    for (int i = 0; i < V->nx; ++i)
      if (V->hact[(size_t)j * V->nx + i]) t[(size_t)(j / TILE_Y) * ntx + i / TILE_X] = 1;
  CK(cudaMemcpyAsync(V->tiles, t.data(), t.size(), cudaMemcpyHostToDevice, V->stream));
  return sync(V);
}

// enable_sparse (delta3d_sparse.rs:105-117): the masks are reserved here, every column in the set.
int fd3_enable_sparse(fd3_volume* V) {
  if (!V) return FD3_ERR_INVALID_ARGUMENT;
  if (V->sparse) return FD3_ERR_DOMAIN;
  float *a, *b;
  TRY(dalloc(V, &a, ((size_t)V->ncol + 3) / 4));
  TRY(dalloc(V, &b, ((size_t)V->ncol + 3) / 4));
  const size_t ntiles = (size_t)((V->nx + TILE_X - 1) / TILE_X) * ((V->ny + TILE_Y - 1) / TILE_Y);
  float* t;
  TRY(dalloc(V, &t, (ntiles + 3) / 4));
  V->act = (unsigned char*)a;
  V->act_next = (unsigned char*)b;
  V->tiles = (unsigned char*)t;
  V->hact.assign(V->ncol, 1);
  CK(cudaMemcpyAsync(V->act, V->hact.data(), V->ncol, cudaMemcpyHostToDevice, V->stream));
  TRY(upload_tiles(V));
  V->sparse = true;
  return FD3_OK;
}

// apply_sparse (delta3d_sparse.rs:181-210): `next` replaces the set.  What the leaving columns
// carried is counted on the host in the reference's column order (its f64 sum is published), then
// one kernel puts them to rest.
static int apply_sparse(fd3_volume* V, const std::vector<unsigned char>& next, fd3_sparse_change* out) {
  const int nx = V->nx, ny = V->ny, ncol = V->ncol;
  std::vector<float> e(ncol), r(ncol);
  CK(cudaMemcpyAsync(e.data(), V->eta, (size_t)ncol * 4, cudaMemcpyDeviceToHost, V->stream));
  CK(cudaMemcpyAsync(r.data(), V->rof, (size_t)ncol * 4, cudaMemcpyDeviceToHost, V->stream));
  TRY(sync(V));
  fd3_sparse_change ch{};
  std::vector<unsigned char> leave(ncol, 0);
  const double area = (double)V->dx * (double)V->dx;
  for (int j = 0; j < ny; ++j)
    for (int i = 0; i < nx; ++i) {
      const int c = j * nx + i;
      const bool was = V->hact[c] != 0, will = next[c] != 0;
      if (was && !will) {
        ++ch.deactivated;
        leave[c] = 1;
        const double h = ((double)e[c] - (double)r[c]) - (double)V->rest;
        ch.volume_removed += h * area;
        ch.height_removed = std::max(ch.height_removed, std::fabs(e[c] - V->rest));
      } else if (!was && will) {
        ++ch.activated;
      }
    }
  if (ch.deactivated) {
    CK(cudaMemcpyAsync(V->act_next, leave.data(), ncol, cudaMemcpyHostToDevice, V->stream));
    CK(cudaMemsetAsync(V->dflag, 0, sizeof(int), V->stream));
    LAUNCH(V, k_sparse_leave, (long long)ncol + V->n + V->nu + V->nv + V->nw, V->geo(),
           (const unsigned char*)V->act_next, V->rest, V->eta, V->rof, V->p, V->u, V->v, V->w, V->dflag);
    CK(cudaMemcpyAsync(V->hflag, V->dflag, sizeof(int), cudaMemcpyDeviceToHost, V->stream));
    // The blocked kernels skip tiles outside the set (Geo::tiles) and rely on every vector they
    // write being 0 there.  The work vectors are scratch of each projection and the coarse
    // levels' of each V-cycle, so they are zeroed whole; p was zeroed in the leaving columns.
    for (float* f : {V->res, V->dir, V->dir2, V->tmp, V->z, V->z2})
      if (f) CK(cudaMemsetAsync(f, 0, (size_t)V->n * 4, V->stream));
    for (Lev& L : V->levels)
      for (float* f : {L.x, L.x2, L.r, L.t}) CK(cudaMemsetAsync(f, 0, (size_t)L.n * 4, V->stream));
  }
  V->hact = next;
  CK(cudaMemcpyAsync(V->act, V->hact.data(), ncol, cudaMemcpyHostToDevice, V->stream));
  TRY(upload_tiles(V));
  TRY(sync(V));
  if (ch.deactivated) std::memcpy(&ch.velocity_removed, V->hflag, 4);
  for (unsigned char a : V->hact) ch.active_columns += a != 0;
  if (out) *out = ch;
  return FD3_OK;
}

// set_active_columns (delta3d_sparse.rs:147-158)
int fd3_set_active_columns(fd3_volume* V, const uint8_t* mask, size_t len, fd3_sparse_change* change) {
  if (!V || (!mask && len)) return FD3_ERR_INVALID_ARGUMENT;
  if (!V->sparse) return FD3_ERR_DOMAIN;
  if (len != (size_t)V->ncol) return FD3_ERR_SHAPE;
  std::vector<unsigned char> next(V->ncol);
  for (int c = 0; c < V->ncol; ++c) next[c] = mask[c] != 0;
  return apply_sparse(V, next, change);
}

// set_active_blocks (delta3d_sparse.rs:163-178): block (bi, bj) covers the columns
// [(bi - origin_i) * 8, +8) x [(bj - origin_j) * 8, +8) of the window, clipped to it.
int fd3_set_active_blocks(fd3_volume* V, const int32_t* blocks, size_t count, int32_t origin_i, int32_t origin_j,
                          fd3_sparse_change* change) {
  if (!V || (!blocks && count)) return FD3_ERR_INVALID_ARGUMENT;
  if (!V->sparse) return FD3_ERR_DOMAIN;
  const long long side = FD3_BLOCK, nx = V->nx, ny = V->ny;
  std::vector<unsigned char> next(V->ncol, 0);
  for (size_t b = 0; b < count; ++b) {
    const long long i0 = ((long long)blocks[2 * b] - origin_i) * side, j0 = ((long long)blocks[2 * b + 1] - origin_j) * side;
    for (long long j = std::max(j0, 0LL); j < std::min(j0 + side, ny); ++j)
      for (long long i = std::max(i0, 0LL); i < std::min(i0 + side, nx); ++i) next[(size_t)(j * nx + i)] = 1;
  }
  return apply_sparse(V, next, change);
}

int fd3_active_columns(const fd3_volume* V, uint8_t* out, size_t len) {
  if (!V || (!out && len)) return FD3_ERR_INVALID_ARGUMENT;
  if (!V->sparse) return FD3_ERR_DOMAIN;
  if (len != (size_t)V->ncol) return FD3_ERR_SHAPE;
  std::memcpy(out, V->hact.data(), len);
  return FD3_OK;
}

uint64_t fd3_sparse_cells(const fd3_volume* V) {
  if (!V) return 0;
  if (!V->sparse) return (uint64_t)V->n;
  uint64_t cols = 0;
  for (unsigned char a : V->hact) cols += a != 0;
  return cols * (uint64_t)V->nz;
}

// perturbation_volume (delta3d_balance.rs:105-113): summed on the host in column order, in f64.
static int perturbation_volume(fd3_volume* V, double* out) {
  std::vector<float> e(V->ncol), r(V->ncol);
  CK(cudaMemcpyAsync(e.data(), V->eta, (size_t)V->ncol * 4, cudaMemcpyDeviceToHost, V->stream));
  CK(cudaMemcpyAsync(r.data(), V->rof, (size_t)V->ncol * 4, cudaMemcpyDeviceToHost, V->stream));
  TRY(sync(V));
  const double area = (double)V->dx * (double)V->dx, rest = (double)V->rest;
  double total = 0.0;
  for (int c = 0; c < V->ncol; ++c) total += ((double)e[c] - (double)r[c]) - rest;
  *out = total * area;
  return FD3_OK;
}

int fd3_perturbation_volume(fd3_volume* V, double* out) {
  if (!V || !out) return FD3_ERR_INVALID_ARGUMENT;
  return perturbation_volume(V, out);
}

// resample_from (delta3d_levels.rs:43-69).  Refusal (FD3_ERR_DOMAIN) writes nothing.
int fd3_resample_from(fd3_volume* V, fd3_volume* S, fd3_level_change* change) {
  if (!V || !S || V == S) return FD3_ERR_INVALID_ARGUMENT;
  if (V->device != S->device) return FD3_ERR_INVALID_ARGUMENT;
  auto extent = [](int n, float dx) { return (double)n * (double)dx; };
  auto same = [](double a, double b) { return std::fabs(a - b) <= 1e-6 * std::max(std::fabs(a), std::fabs(b)); };
  auto fbits = [](float x) { uint32_t b; std::memcpy(&b, &x, 4); return b; };
  if (!same(extent(V->nx, V->dx), extent(S->nx, S->dx)) || !same(extent(V->ny, V->dx), extent(S->ny, S->dx)) ||
      !same(extent(V->nz, V->dx), extent(S->nz, S->dx)) || fbits(V->rest) != fbits(S->rest) ||
      fbits(V->rho) != fbits(S->rho) || fbits(V->g) != fbits(S->g) || V->cut || S->cut)
    return FD3_ERR_DOMAIN;
  fd3_level_change ch{};
  TRY(perturbation_volume(S, &ch.volume_before));  // also orders S's stream before V's launches
  LevelSrc src{S->nx, S->ny, S->nz, S->dx, S->rest, S->eta, S->rof, S->u, S->v, S->w, S->sparse ? S->act : nullptr};
  const int n = std::max((int)std::ceil((double)V->dx / (double)S->dx), 1);
  LAUNCH(V, k_resample_surface, V->ncol, src, V->nx, V->ny, V->dx, V->rest,
         (const unsigned char*)(V->sparse ? V->act : nullptr), V->eta, V->rof);
  LAUNCH(V, k_resample_faces, (long long)V->nu + V->nv + V->nw, src, V->nx, V->ny, V->nz, n, V->u, V->v, V->w);
  CK(cudaMemsetAsync(V->p, 0, (size_t)V->n * 4, V->stream));
  LAUNCH(V, k_close_walls, (long long)V->nu + V->nv + V->nw, V->geo(), V->u, V->v, V->w);
  TRY(perturbation_volume(V, &ch.volume_after));
  if (change) *change = ch;
  return FD3_OK;
}

int fd3_reset_pressure(fd3_volume* V) {
  if (!V) return FD3_ERR_INVALID_ARGUMENT;
  CK(cudaMemsetAsync(V->p, 0, (size_t)V->n * sizeof(float), V->stream));
  return FD3_OK;
}

// tests_delta3d.rs:392-395: us = u, then project_mobile3.  A refusal leaves u, v, w, p untouched.
int fd3_project_mobile(fd3_volume* V, float scale, float k1, uint32_t max_iters, fd3_report* rep) {
  if (!V || !rep) return FD3_ERR_INVALID_ARGUMENT;
  CK(cudaMemcpyAsync(V->us, V->u, (size_t)V->nu * 4, cudaMemcpyDeviceToDevice, V->stream));
  CK(cudaMemcpyAsync(V->vs, V->v, (size_t)V->nv * 4, cudaMemcpyDeviceToDevice, V->stream));
  CK(cudaMemcpyAsync(V->ws, V->w, (size_t)V->nw * 4, cudaMemcpyDeviceToDevice, V->stream));
  CK(cudaMemcpyAsync(V->sv_p, V->p, (size_t)V->n * 4, cudaMemcpyDeviceToDevice, V->stream));
  int e = project_mobile3(V, scale, k1, max_iters, rep);
  if (e) {
    cudaMemcpyAsync(V->u, V->us, (size_t)V->nu * 4, cudaMemcpyDeviceToDevice, V->stream);
    cudaMemcpyAsync(V->v, V->vs, (size_t)V->nv * 4, cudaMemcpyDeviceToDevice, V->stream);
    cudaMemcpyAsync(V->w, V->ws, (size_t)V->nw * 4, cudaMemcpyDeviceToDevice, V->stream);
    cudaMemcpyAsync(V->p, V->sv_p, (size_t)V->n * 4, cudaMemcpyDeviceToDevice, V->stream);
    cudaStreamSynchronize(V->stream);
  }
  return e;
}

__global__ void k_add_into(int n, float* __restrict__ p, const float* __restrict__ base) {
  KSTART();
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c < n) p[c] += base[c];
}

// refine_mobile3 (delta3d_coupling.rs:226-248): the pressure before the call is the base; the
// current field is projected again from p = 0 with homogeneous ghosts and the increment is added
// to the base.  A refusal leaves u, v, w, p untouched.
int fd3_refine_mobile(fd3_volume* V, float scale, float k1, uint32_t max_iters, fd3_report* rep) {
  if (!V || !rep) return FD3_ERR_INVALID_ARGUMENT;
  CK(cudaMemcpyAsync(V->us, V->u, (size_t)V->nu * 4, cudaMemcpyDeviceToDevice, V->stream));
  CK(cudaMemcpyAsync(V->vs, V->v, (size_t)V->nv * 4, cudaMemcpyDeviceToDevice, V->stream));
  CK(cudaMemcpyAsync(V->ws, V->w, (size_t)V->nw * 4, cudaMemcpyDeviceToDevice, V->stream));
  CK(cudaMemcpyAsync(V->sv_p, V->p, (size_t)V->n * 4, cudaMemcpyDeviceToDevice, V->stream));
  CK(cudaMemsetAsync(V->p, 0, (size_t)V->n * 4, V->stream));
  V->homog = true;
  int e = project_mobile3(V, scale, k1, max_iters, rep);
  V->homog = false;
  if (e) {
    cudaMemcpyAsync(V->u, V->us, (size_t)V->nu * 4, cudaMemcpyDeviceToDevice, V->stream);
    cudaMemcpyAsync(V->v, V->vs, (size_t)V->nv * 4, cudaMemcpyDeviceToDevice, V->stream);
    cudaMemcpyAsync(V->w, V->ws, (size_t)V->nw * 4, cudaMemcpyDeviceToDevice, V->stream);
    cudaMemcpyAsync(V->p, V->sv_p, (size_t)V->n * 4, cudaMemcpyDeviceToDevice, V->stream);
    cudaStreamSynchronize(V->stream);
    return e;
  }
  LAUNCH(V, k_add_into, V->n, V->n, V->p, (const float*)V->sv_p);
  TRY(sync(V));
  rep->refinements = 1;
  return FD3_OK;
}

int fd3_step_surface_mobile(fd3_volume* V, uint64_t duration_us, uint32_t max_iters, fd3_report* rep) {
  if (!V || !rep) return FD3_ERR_INVALID_ARGUMENT;
  return step_surface_mobile(V, duration_us, max_iters, rep);
}

// tests_delta3d.rs:143-148: us = u, then project.  A refusal leaves u, v, w, p untouched.
int fd3_project_linear(fd3_volume* V, float scale, float k1, uint32_t max_iters, fd3_report* rep) {
  if (!V || !rep) return FD3_ERR_INVALID_ARGUMENT;
  if (V->sparse) return FD3_ERR_DOMAIN;  // the linear path does not carry a sparse set (delta3d.rs:1210-1211)
  CK(cudaMemcpyAsync(V->us, V->u, (size_t)V->nu * 4, cudaMemcpyDeviceToDevice, V->stream));
  CK(cudaMemcpyAsync(V->vs, V->v, (size_t)V->nv * 4, cudaMemcpyDeviceToDevice, V->stream));
  CK(cudaMemcpyAsync(V->ws, V->w, (size_t)V->nw * 4, cudaMemcpyDeviceToDevice, V->stream));
  CK(cudaMemcpyAsync(V->sv_p, V->p, (size_t)V->n * 4, cudaMemcpyDeviceToDevice, V->stream));
  int e = project_linear(V, scale, k1, max_iters, rep);
  if (e) {
    cudaMemcpyAsync(V->u, V->us, (size_t)V->nu * 4, cudaMemcpyDeviceToDevice, V->stream);
    cudaMemcpyAsync(V->v, V->vs, (size_t)V->nv * 4, cudaMemcpyDeviceToDevice, V->stream);
    cudaMemcpyAsync(V->w, V->ws, (size_t)V->nw * 4, cudaMemcpyDeviceToDevice, V->stream);
    cudaMemcpyAsync(V->p, V->sv_p, (size_t)V->n * 4, cudaMemcpyDeviceToDevice, V->stream);
    cudaStreamSynchronize(V->stream);
  }
  return e;
}

int fd3_step_surface_linear(fd3_volume* V, uint64_t duration_us, uint32_t max_iters, fd3_report* rep) {
  if (!V || !rep) return FD3_ERR_INVALID_ARGUMENT;
  if (V->sparse) return FD3_ERR_DOMAIN;  // delta3d.rs:1210-1211
  return step_surface_linear(V, duration_us, max_iters, rep);
}

// enable_advection_correction / advection_correction (delta3d_advection.rs:17-26)
int fd3_enable_advection_correction(fd3_volume* V) {
  if (!V) return FD3_ERR_INVALID_ARGUMENT;
  V->advection_correction = true;
  return FD3_OK;
}
int fd3_advection_correction(const fd3_volume* V) { return V && V->advection_correction ? 1 : 0; }

// The predictor alone, as tests_delta3d.rs:2136-2160 runs it: advect_mobile3, the second-order term
// when enabled, then u = us (no projection).
int fd3_advect_for_tests(fd3_volume* V, float dt) {
  if (!V) return FD3_ERR_INVALID_ARGUMENT;
  if (!(dt > 0.f) || !std::isfinite(dt)) return FD3_ERR_NOT_FINITE;
  Geo G = V->geo();
  LAUNCH(V, k_advect, (long long)V->nu + V->nv + V->nw, G, dt, (const float*)V->u, (const float*)V->v,
         (const float*)V->w, V->us, V->vs, V->ws);
  if (V->advection_correction)
    LAUNCH(V, k_correct_advection, (long long)V->nu + V->nv + V->nw, G, dt, (const float*)V->u, (const float*)V->v,
           (const float*)V->w, V->us, V->vs, V->ws);
  CK(cudaMemcpyAsync(V->u, V->us, (size_t)V->nu * 4, cudaMemcpyDeviceToDevice, V->stream));
  CK(cudaMemcpyAsync(V->v, V->vs, (size_t)V->nv * 4, cudaMemcpyDeviceToDevice, V->stream));
  CK(cudaMemcpyAsync(V->w, V->ws, (size_t)V->nw * 4, cudaMemcpyDeviceToDevice, V->stream));
  return sync(V);
}

int fd3_set_precondition_cut(fd3_volume* V, int on) {
  if (!V) return FD3_ERR_INVALID_ARGUMENT;
  V->precondition_cut = on != 0;
  return FD3_OK;
}

// Many independent volumes (patches) projected concurrently: each keeps its own stream and its
// device-side PCG loop; `threads` host workers (0 = up to 16) feed the GPU, largest patches first.
int fd3_project_batch(fd3_volume* const* vols, size_t count, const float* scales, const float* k1s,
                      uint32_t max_iters, int threads, fd3_report* reports, int* statuses) {
  if ((!vols || !scales || !k1s || !reports || !statuses) && count) return FD3_ERR_INVALID_ARGUMENT;
  std::vector<size_t> order(count);
  for (size_t i = 0; i < count; ++i) {
    if (!vols[i]) return FD3_ERR_INVALID_ARGUMENT;
    order[i] = i;
  }
  std::sort(order.begin(), order.end(), [&](size_t a, size_t b) { return vols[a]->n > vols[b]->n; });
  if (count > 1) {  // one volume twice would race on its buffers
    std::vector<const fd3_volume*> seen(vols, vols + count);
    std::sort(seen.begin(), seen.end());
    if (std::adjacent_find(seen.begin(), seen.end()) != seen.end()) return FD3_ERR_INVALID_ARGUMENT;
  }
  size_t T = threads > 0 ? (size_t)threads : 16;
  T = std::max<size_t>(1, std::min(T, count));
  std::atomic<size_t> next{0};
  auto worker = [&]() {
    for (;;) {
      const size_t q = next.fetch_add(1);
      if (q >= count) break;
      const size_t i = order[q];
      cudaSetDevice(vols[i]->device);
      statuses[i] = fd3_project_mobile(vols[i], scales[i], k1s[i], max_iters, &reports[i]);
    }
  };
  std::vector<std::thread> pool;
  for (size_t t = 1; t < T; ++t) pool.emplace_back(worker);
  worker();
  for (auto& th : pool) th.join();
  return FD3_OK;
}

}  // extern "C"

// ------------------------------------------------------------------------- the persistent batch
struct fd3_batch {
  int device = 0;
  cudaStream_t stream = nullptr;
  int cluster = 0, clusters = 0;
  std::vector<fd3_volume*> vols;
  std::vector<cudaEvent_t> ready;  // one per volume: its stream's work before the launch
  BatchPatch* hp = nullptr;        // pinned: the patch table, refreshed per call
  BatchResult* hres = nullptr;     // pinned
  BatchPatch* dp = nullptr;
  BatchResult* dres = nullptr;
  int *dorder = nullptr, *dstart = nullptr;
  std::vector<int> order, start;
  unsigned long long launches = 0;
};

namespace {

void batch_release(fd3_batch* B) {
  if (B->stream) cudaStreamSynchronize(B->stream);
  for (cudaEvent_t e : B->ready) cudaEventDestroy(e);
  if (B->hp) cudaFreeHost(B->hp);
  if (B->hres) cudaFreeHost(B->hres);
  if (B->dp) cudaFree(B->dp);
  if (B->dres) cudaFree(B->dres);
  if (B->dorder) cudaFree(B->dorder);
  if (B->dstart) cudaFree(B->dstart);
  if (B->stream) cudaStreamDestroy(B->stream);
}

cudaLaunchConfig_t batch_config(fd3_batch* B, cudaLaunchAttribute* attr, int clusters) {
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3((unsigned)(clusters * B->cluster));
  cfg.blockDim = dim3(BATCH_THREADS);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = B->stream;
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = (unsigned)B->cluster;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cfg;
}

}  // namespace

extern "C" {

int fd3_batch_create(fd3_volume* const* vols, size_t count, int cluster_size, fd3_batch** out) {
  if (!out || !vols || !count) return FD3_ERR_INVALID_ARGUMENT;
  if (cluster_size != 1 && cluster_size != 2 && cluster_size != 4 && cluster_size != 8) return FD3_ERR_INVALID_ARGUMENT;
  std::vector<const fd3_volume*> seen(vols, vols + count);
  for (const fd3_volume* V : seen) {
    if (!V) return FD3_ERR_INVALID_ARGUMENT;
    if (V->device != vols[0]->device) return FD3_ERR_INVALID_ARGUMENT;
    // the batched projection: f64 reductions, f32 storage, the mobile rows with multigrid
    if (!V->has_mg || V->ord() || V->opt.storage != FD3_STORAGE_F32) return FD3_ERR_DOMAIN;
  }
  std::sort(seen.begin(), seen.end());
  if (std::adjacent_find(seen.begin(), seen.end()) != seen.end()) return FD3_ERR_INVALID_ARGUMENT;
  fd3_batch* B = new (std::nothrow) fd3_batch();
  if (!B) return FD3_ERR_OUT_OF_MEMORY;
  B->device = vols[0]->device;
  B->cluster = cluster_size;
  B->vols.assign(vols, vols + count);
  ScopedDevice on(B->device);
  auto fail = [&](int e) { batch_release(B); delete B; return e; };
  if (on.err != cudaSuccess) return fail(cuda_fail(on.err, "cudaSetDevice", __LINE__));
  cudaError_t e = cudaStreamCreateWithFlags(&B->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) return fail(cuda_fail(e, "cudaStreamCreateWithFlags", __LINE__));
  // clusters resident at once: the patches are dealt to that many solvers
  cudaLaunchAttribute attr[1];
  cudaLaunchConfig_t cfg = batch_config(B, attr, 1);
  int active = 0;
  e = cudaOccupancyMaxActiveClusters(&active, k_batch_project, &cfg);
  if (e != cudaSuccess || active <= 0) return fail(cuda_fail(e != cudaSuccess ? e : cudaErrorInvalidConfiguration,
                                                             "cudaOccupancyMaxActiveClusters", __LINE__));
  B->clusters = (int)std::min<size_t>((size_t)active, count);
  // largest patch first to the least loaded cluster (cells as the cost)
  std::vector<int> idx(count);
  for (size_t i = 0; i < count; ++i) idx[i] = (int)i;
  std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) { return vols[a]->n > vols[b]->n; });
  std::vector<std::vector<int>> lists(B->clusters);
  std::vector<long long> load(B->clusters, 0);
  for (int i : idx) {
    int c = (int)(std::min_element(load.begin(), load.end()) - load.begin());
    lists[c].push_back(i);
    load[c] += vols[i]->n;
  }
  B->start.push_back(0);
  for (auto& l : lists) {
    B->order.insert(B->order.end(), l.begin(), l.end());
    B->start.push_back((int)B->order.size());
  }
  if ((e = cudaMallocHost(&B->hp, count * sizeof(BatchPatch))) != cudaSuccess ||
      (e = cudaMallocHost(&B->hres, count * sizeof(BatchResult))) != cudaSuccess ||
      (e = cudaMalloc(&B->dp, count * sizeof(BatchPatch))) != cudaSuccess ||
      (e = cudaMalloc(&B->dres, count * sizeof(BatchResult))) != cudaSuccess ||
      (e = cudaMalloc(&B->dorder, count * sizeof(int))) != cudaSuccess ||
      (e = cudaMalloc(&B->dstart, B->start.size() * sizeof(int))) != cudaSuccess)
    return fail(cuda_fail(e, "batch allocation", __LINE__));
  e = cudaMemcpyAsync(B->dorder, B->order.data(), count * sizeof(int), cudaMemcpyHostToDevice, B->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(B->dstart, B->start.data(), B->start.size() * sizeof(int), cudaMemcpyHostToDevice, B->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(B->stream);
  if (e != cudaSuccess) return fail(cuda_fail(e, "batch tables", __LINE__));
  B->ready.resize(count, nullptr);
  for (size_t i = 0; i < count; ++i)
    if ((e = cudaEventCreateWithFlags(&B->ready[i], cudaEventDisableTiming)) != cudaSuccess)
      return fail(cuda_fail(e, "cudaEventCreateWithFlags", __LINE__));
  *out = B;
  return FD3_OK;
}

void fd3_batch_destroy(fd3_batch* B) {
  if (!B) return;
  ScopedDevice on(B->device);
  batch_release(B);
  delete B;
}

int fd3_batch_clusters(const fd3_batch* B, int* clusters, int* cluster_size) {
  if (!B) return FD3_ERR_INVALID_ARGUMENT;
  if (clusters) *clusters = B->clusters;
  if (cluster_size) *cluster_size = B->cluster;
  return FD3_OK;
}

uint64_t fd3_batch_kernel_launches(const fd3_batch* B) { return B ? B->launches : 0; }

int fd3_batch_project(fd3_batch* B, const float* scales, const float* k1s, uint32_t max_iters, int reset_pressure,
                      const float* const* in_u, const float* const* in_v, const float* const* in_w,
                      fd3_report* reports, int* statuses) {
  if (!B || !scales || !k1s || !reports || !statuses) return FD3_ERR_INVALID_ARGUMENT;
  const size_t count = B->vols.size();
  if ((in_u || in_v || in_w) && !(in_u && in_v && in_w)) return FD3_ERR_INVALID_ARGUMENT;
  ScopedDevice on(B->device);
  if (on.err != cudaSuccess) return cuda_fail(on.err, "cudaSetDevice", __LINE__);
  for (size_t i = 0; i < count; ++i) {
    fd3_volume* V = B->vols[i];
    if (!std::isfinite(scales[i]) || !std::isfinite(k1s[i])) return FD3_ERR_NOT_FINITE;
    V->linear = false;
    BatchPatch& P = B->hp[i];
    P.g = V->geo();
    P.codes = V->codes;
    P.u = V->u; P.v = V->v; P.w = V->w; P.us = V->us; P.vs = V->vs; P.ws = V->ws;
    P.p = V->p; P.sv_p = V->sv_p; P.rhs = V->rhs; P.prec = V->prec; P.res = V->res;
    P.sv_u = V->sv_u; P.sv_v = V->sv_v; P.sv_w = V->sv_w;
    P.dir = V->dir; P.dir2 = V->dir2; P.q = V->tmp; P.z = V->z; P.z2 = V->z2;
    P.in_u = in_u ? in_u[i] : nullptr;
    P.in_v = in_v ? in_v[i] : nullptr;
    P.in_w = in_w ? in_w[i] : nullptr;
    P.lev = V->dlev;
    P.nlev = (int)V->levels.size();
    P.nu = V->nu; P.nv = V->nv; P.nw = V->nw;
    P.scale = scales[i]; P.k1 = k1s[i];
    P.max_iters = max_iters;
    P.flat2d = V->ny == 1 ? 1 : 0;
    P.reset_p = reset_pressure ? 1 : 0;
    P.S = V->dS;
    // the volume's earlier work (on its own stream) comes before the launch
    CK(cudaEventRecord(B->ready[i], V->stream));
    CK(cudaStreamWaitEvent(B->stream, B->ready[i], 0));
  }
  CK(cudaMemcpyAsync(B->dp, B->hp, count * sizeof(BatchPatch), cudaMemcpyHostToDevice, B->stream));
  cudaLaunchAttribute attr[1];
  cudaLaunchConfig_t cfg = batch_config(B, attr, B->clusters);
  CK(cudaLaunchKernelEx(&cfg, k_batch_project, (const BatchPatch*)B->dp, (const int*)B->dorder,
                        (const int*)B->dstart, B->dres));
  B->launches++;
  CK(cudaMemcpyAsync(B->hres, B->dres, count * sizeof(BatchResult), cudaMemcpyDeviceToHost, B->stream));
  CK(cudaStreamSynchronize(B->stream));
  for (size_t i = 0; i < count; ++i) {
    const BatchResult& R = B->hres[i];
    statuses[i] = R.status;
    fd3_report& rep = reports[i];
    memset(&rep, 0, sizeof rep);
    if (R.status) continue;
    rep.iterations = R.iterations;
    rep.degraded = (uint8_t)R.degraded;
    rep.residual = R.residual;
    rep.divergence = R.divergence;
    rep.floor = (uint8_t)R.floor_stop;
    rep.backward_error = R.backward_error;
    rep.divergence_plain = R.divergence_plain;
  }
  return FD3_OK;
}

int fd3_last_refused_report(const fd3_volume* V, fd3_report* rep) {
  if (!V || !rep) return FD3_ERR_INVALID_ARGUMENT;
  if (!V->has_refused) return FD3_ERR_DOMAIN;
  *rep = V->refused;
  return FD3_OK;
}

static int copy_d2h(fd3_volume* V, float* dst, const float* src, size_t len, size_t want) {
  if (!dst && len) return FD3_ERR_INVALID_ARGUMENT;
  if (len != want) return FD3_ERR_SHAPE;
  CK(cudaMemcpyAsync(dst, src, len * 4, cudaMemcpyDeviceToHost, V->stream));
  return FD3_OK;
}

int fd3_get_pressure(const fd3_volume* cv, float* out, size_t len) {
  if (!cv) return FD3_ERR_INVALID_ARGUMENT;
  fd3_volume* V = const_cast<fd3_volume*>(cv);
  TRY(copy_d2h(V, out, V->p, len, V->n));
  return sync(V);
}

int fd3_get_velocity(const fd3_volume* cv, float* u, size_t nu, float* vv, size_t nv, float* w, size_t nw) {
  if (!cv) return FD3_ERR_INVALID_ARGUMENT;
  fd3_volume* V = const_cast<fd3_volume*>(cv);
  TRY(copy_d2h(V, u, V->u, nu, V->nu));
  TRY(copy_d2h(V, vv, V->v, nv, V->nv));
  TRY(copy_d2h(V, w, V->w, nw, V->nw));
  return sync(V);
}

int fd3_get_surface(const fd3_volume* cv, float* eta, float* roundoff, size_t len) {
  if (!cv) return FD3_ERR_INVALID_ARGUMENT;
  fd3_volume* V = const_cast<fd3_volume*>(cv);
  TRY(copy_d2h(V, eta, V->eta, len, V->ncol));
  TRY(copy_d2h(V, roundoff, V->rof, len, V->ncol));
  return sync(V);
}

int fd3_device_fields(const fd3_volume* V, float** p, float** u, float** vv, float** w) {
  if (!V) return FD3_ERR_INVALID_ARGUMENT;
  if (p) *p = V->p;
  if (u) *u = V->u;
  if (vv) *vv = V->v;
  if (w) *w = V->w;
  return FD3_OK;
}

int fd3_get_geometry(const fd3_volume* cv, float* frac, float* ou, float* ov, float* ow, float* floor) {
  if (!cv) return FD3_ERR_INVALID_ARGUMENT;
  if (!cv->cut) return FD3_ERR_DOMAIN;
  fd3_volume* V = const_cast<fd3_volume*>(cv);
  TRY(copy_d2h(V, frac, V->frac, V->n, V->n));
  TRY(copy_d2h(V, ou, V->ou, V->nu, V->nu));
  TRY(copy_d2h(V, ov, V->ov, V->nv, V->nv));
  TRY(copy_d2h(V, ow, V->ow, V->nw, V->nw));
  TRY(copy_d2h(V, floor, V->floor_, V->ncol, V->ncol));
  return sync(V);
}

__global__ void k_count_wet(Geo g, unsigned long long* count) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  bool wet = false;
  if (c < g.n) { int i, j, k; cell_ijk(g, c, i, j, k); wet = wet3(g, i, j, k); }
  unsigned m = __ballot_sync(0xffffffffu, wet);
  if ((threadIdx.x & 31) == 0 && m) atomicAdd(count, (unsigned long long)__popc(m));
}

uint64_t fd3_wet_cells(const fd3_volume* cv) {
  if (!cv) return 0;
  fd3_volume* V = const_cast<fd3_volume*>(cv);
  LAUNCH_G(V, k_reset_diag, 1, 1, V->dS, 4);
  LAUNCH(V, k_count_wet, V->n, V->geo(), &V->dS->hash);
  if (pull(V)) return 0;
  return V->hS->hash;
}

// delta3d_mobile.rs:936-953
int fd3_apply_pressure_operator_for_trials(fd3_volume* V, const float* p, float* out, size_t len) {
  if (!V || !p || !out) return FD3_ERR_INVALID_ARGUMENT;
  if (len != (size_t)V->n) return FD3_ERR_DOMAIN;
  CK(cudaMemcpyAsync(V->tmp, p, len * 4, cudaMemcpyHostToDevice, V->stream));
  bool ok;
  TRY(check_finite_device(V, V->tmp, V->n, &ok));
  if (!ok) return FD3_ERR_NOT_FINITE;
  LAUNCH(V, k_apply, V->n, V->geo(), (const float*)V->tmp, V->dir);
  CK(cudaMemcpyAsync(out, V->dir, len * 4, cudaMemcpyDeviceToHost, V->stream));
  return sync(V);
}

// delta3d_mobile.rs:960-979
int fd3_assemble_pressure_problem_for_trials(fd3_volume* V, const float* divergence, float scale, float* rhs,
                                             float* prec, size_t len) {
  if (!V || !divergence || !rhs || !prec) return FD3_ERR_INVALID_ARGUMENT;
  if (len != (size_t)V->n) return FD3_ERR_DOMAIN;
  if (!std::isfinite(scale)) return FD3_ERR_NOT_FINITE;
  CK(cudaMemcpyAsync(V->tmp, divergence, len * 4, cudaMemcpyHostToDevice, V->stream));
  bool ok;
  TRY(check_finite_device(V, V->tmp, V->n, &ok));
  if (!ok) return FD3_ERR_NOT_FINITE;
  CK(cudaMemcpyAsync(V->rhs, V->tmp, len * 4, cudaMemcpyDeviceToDevice, V->stream));
  DISPATCH(V, k_rhs_b2, V->n, V->geo(), scale, V->rhs, V->prec, V->red(), V->dS, 0, (unsigned short*)nullptr,
           (float*)nullptr);
  CK(cudaMemcpyAsync(rhs, V->rhs, len * 4, cudaMemcpyDeviceToHost, V->stream));
  CK(cudaMemcpyAsync(prec, V->prec, len * 4, cudaMemcpyDeviceToHost, V->stream));
  return sync(V);
}

// tests_delta3d.rs:1840-1873 set-up, then v_cycle3.
int fd3_vcycle_for_tests(fd3_volume* V, const float* x, float* z, size_t len) {
  if (!V || !x || !z) return FD3_ERR_INVALID_ARGUMENT;
  if (!V->has_mg) return FD3_ERR_DOMAIN;
  if (len != (size_t)V->n) return FD3_ERR_SHAPE;
  CK(cudaMemsetAsync(V->rhs, 0, len * 4, V->stream));
  DISPATCH(V, k_rhs_b2, V->n, V->geo(), 1.f, V->rhs, V->prec, V->red(), V->dS, 0, V->codes, (float*)nullptr);
  prepare_multigrid(V);
  CK(cudaMemcpyAsync(V->res, x, len * 4, cudaMemcpyHostToDevice, V->stream));
  if (V->half()) LAUNCH_G(V, k_reset_scalars, 1, 1, V->dS, 0.f);  // FP16 storage, r unscaled (vinv = 1)
  vcycle(V, 0, FIN_RZ_PRIME);
  const float* zf = V->z;
  if (V->half()) {
    LAUNCH(V, k_widen, V->n, V->n, (const __half*)V->z, V->tmp);
    zf = V->tmp;
  }
  CK(cudaMemcpyAsync(z, zf, len * 4, cudaMemcpyDeviceToHost, V->stream));
  return sync(V);
}

int fd3_level_geometry(const fd3_volume* cv, uint32_t l, float* kind, float* diag, float* ou, float* ov, float* ow) {
  if (!cv) return FD3_ERR_INVALID_ARGUMENT;
  if (!cv->has_mg || l >= cv->levels.size()) return FD3_ERR_DOMAIN;
  fd3_volume* V = const_cast<fd3_volume*>(cv);
  const Lev& L = V->levels[l];
  size_t nu = (size_t)(L.nx + 1) * L.ny * L.nz, nv = (size_t)L.nx * (L.ny + 1) * L.nz, nw = (size_t)L.nx * L.ny * (L.nz + 1);
  TRY(copy_d2h(V, kind, L.kind, L.n, L.n));
  TRY(copy_d2h(V, diag, L.diag, L.n, L.n));
  TRY(copy_d2h(V, ou, L.ou, nu, nu));
  TRY(copy_d2h(V, ov, L.ov, nv, nv));
  TRY(copy_d2h(V, ow, L.ow, nw, nw));
  return sync(V);
}

uint64_t fd3_kernel_launches(const fd3_volume* V) { return V ? V->launches : 0; }

int fd3_profile(fd3_volume* V, int on) {
  if (!V) return FD3_ERR_INVALID_ARGUMENT;
  TRY(sync(V));
  V->prof = on != 0;
  V->pending.clear();
  V->ev_next = 0;
  if (on) { V->prof_names.clear(); V->prof_count.clear(); V->prof_ms.clear(); }
  return FD3_OK;
}

int fd3_profile_count(const fd3_volume* V) { return V ? (int)V->prof_names.size() : 0; }

int fd3_profile_entry(const fd3_volume* V, int idx, char* name, size_t len, uint64_t* launches, double* total_ms) {
  if (!V || idx < 0 || idx >= (int)V->prof_names.size()) return FD3_ERR_INVALID_ARGUMENT;
  if (name && len) { strncpy(name, V->prof_names[idx].c_str(), len - 1); name[len - 1] = 0; }
  if (launches) *launches = V->prof_count[idx];
  if (total_ms) *total_ms = V->prof_ms[idx];
  return FD3_OK;
}

}  // extern "C"

// =============================================================================== learned preconditioner
#include "fd3_learned.cuh"

// =============================================================================== no-alloc entry
// fd3_assemble_pressure_problem_noalloc: the assembly of the pressure problem (rhs_mobile3 with
// the norm of its right-hand side) for callers that may not allocate device memory at call time,
// e.g. a host whose memory arena is sealed after set-up (no allocation after `seal()`), or a
// real-time loop in which a cudaMalloc would stall the frame.  It allocates nothing: its scratch
// (per-block partial sums, the completion counter, the finiteness flag) is the file-scope array
// below, which every GPU that loads this library holds until the process exits.
namespace {

constexpr int kNoAllocMaxCells = 4194304;                      // largest volume accepted (cells)
constexpr int kNoAllocMaxBlocks = kNoAllocMaxCells / TPB;       // 16384 partial sums
constexpr size_t kNoAllocScratchBytes = (size_t)kNoAllocMaxBlocks * sizeof(double) + 256;

// Layout: [0, 8*kNoAllocMaxBlocks) partials (f64) | counter (u32) | flag (i32) | sum (f64).
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

struct NoAllocScratch {
  double* partials;
  unsigned* counter;
  int* flag;
  double* sum;
};

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mutex;
void* g_noalloc_addr[kMaxDevices] = {};


// The device address of g_noalloc_scratch on device `dev` (which must be current), looked up once
// per device: in host code the symbol is only a host-side stand-in, not a device address.
int noalloc_scratch(int dev, NoAllocScratch* out) {
  if (dev < 0 || dev >= kMaxDevices) return FD3_ERR_NO_DEVICE;
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (!g_noalloc_addr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) return cuda_fail(e != cudaSuccess ? e : cudaErrorInvalidSymbol, "cudaGetSymbolAddress", __LINE__);
    g_noalloc_addr[dev] = p;
  }
  unsigned char* base = (unsigned char*)g_noalloc_addr[dev];
  out->partials = (double*)base;
  out->counter = (unsigned*)(base + (size_t)kNoAllocMaxBlocks * sizeof(double));
  out->flag = (int*)(base + (size_t)kNoAllocMaxBlocks * sizeof(double) + 8);
  out->sum = (double*)(base + (size_t)kNoAllocMaxBlocks * sizeof(double) + 16);
  return FD3_OK;
}

// rhs_mobile3 (delta3d_mobile.rs:215-241) of a caller's divergence field into the caller's rhs and
// prec, with |rhs|^2 in f64: block partials in the scratch, the last block sums them in a fixed
// order.  The divergence is checked finite on the way (flag).
__global__ void __launch_bounds__(TPB) k_assemble_noalloc(Geo g, float scale, const float* __restrict__ div,
                                                          float* __restrict__ rhs, float* __restrict__ prec,
                                                          NoAllocScratch sc) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  float b = 0.f;
  bool bad = false;
  if (c < g.n) {
    float dv = div[c];
    bad = !isfinite(dv);
    int i, j, k; cell_ijk(g, c, i, j, k);
    if (!wet3(g, i, j, k)) { rhs[c] = 0.f; prec[c] = 0.f; }
    else {
      RowE row[6]; mobile_row(g, i, j, k, row);
      b = scale * dv;
      float diag = 0.f;
#pragma unroll
      for (int f = 0; f < 6; ++f) {
        if (row[f].n >= 0) diag += row[f].a;
        else if (row[f].a > 0.f) {
          diag += row[f].a * row[f].it;
          b += row[f].a * row[f].val * row[f].it * g.inv;
        }
      }
      rhs[c] = b;
      prec[c] = diag > 0.f ? 1.f / (diag * g.inv) : 0.f;
    }
  }
  if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(sc.flag, 1);
  __shared__ double sw[TPB / 32];
  double s = (double)b * (double)b;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) sw[threadIdx.x >> 5] = s;
  __syncthreads();
  __shared__ bool last;
  if (threadIdx.x == 0) {
    double t = 0.0;
#pragma unroll
    for (int w = 0; w < TPB / 32; ++w) t += sw[w];
    sc.partials[blockIdx.x] = t;
    __threadfence();
    last = atomicAdd(sc.counter, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  __shared__ double sm[TPB];
  double t = 0.0;
  for (int q = threadIdx.x; q < (int)gridDim.x; q += blockDim.x) t += __ldcg(sc.partials + q);
  sm[threadIdx.x] = t;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) sm[threadIdx.x] += sm[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) { *sc.sum = sm[0]; *sc.counter = 0u; }
}

}  // namespace

extern "C" int fd3_assemble_pressure_problem_noalloc(fd3_volume* V, const float* d_divergence, float scale,
                                                     float* d_rhs, float* d_prec, size_t len, double* rhs_norm2) {
  if (!V || !d_divergence || !d_rhs || !d_prec || !rhs_norm2) return FD3_ERR_INVALID_ARGUMENT;
  if (len != (size_t)V->n) return FD3_ERR_DOMAIN;
  if (len > (size_t)kNoAllocMaxCells) return FD3_ERR_SCRATCH_LIMIT;
  if (!std::isfinite(scale)) return FD3_ERR_NOT_FINITE;
  // the volume's device is made current for the call (and the caller's restored on return), so the
  // scratch looked up, the memset and the launch all belong to the device the volume lives on
  ScopedDevice on(V->device);
  if (on.err != cudaSuccess) return cuda_fail(on.err, "cudaSetDevice", __LINE__);
  NoAllocScratch sc;
  TRY(noalloc_scratch(V->device, &sc));
  // the counter, the flag and the sum start at zero on every call (the array keeps the last call's
  // contents); the partials are all overwritten
  CK(cudaMemsetAsync(sc.counter, 0, 24, V->stream));
  k_assemble_noalloc<<<blocks_for(V->n), TPB, 0, V->stream>>>(V->geo(), scale, d_divergence, d_rhs, d_prec, sc);
  CK(cudaGetLastError());
  int flag = 0;
  CK(cudaMemcpyAsync(&flag, sc.flag, sizeof(int), cudaMemcpyDeviceToHost, V->stream));
  CK(cudaMemcpyAsync(rhs_norm2, sc.sum, sizeof(double), cudaMemcpyDeviceToHost, V->stream));
  CK(cudaStreamSynchronize(V->stream));
  V->launches++;
  return flag ? FD3_ERR_NOT_FINITE : FD3_OK;
}
