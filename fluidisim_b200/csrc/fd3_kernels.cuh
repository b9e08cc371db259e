// Device code of the delta (δ) MAC-grid pressure projection for sm_100a.
//
// Every per-cell and per-face operation evaluates the same f32 expressions, in the same order, as
// the reference (paths relative to code/water-core/src/); the library is compiled with
// --fmad=false so no multiply-add is contracted, as in Rust.  Hence, with the ordered f32
// reduction mode, a projection reproduces the reference bit for bit.
//
// Layout in HBM: the reference's own (delta3d.rs:187-206).  Cells x-fastest, one f32 per cell
// per field; u/v/w faces in their own arrays; columns (eta, roundoff) x-fastest.  The operator is
// matrix-free, as `apply_mobile3` (delta3d_mobile.rs:190-213): each row is rebuilt from the
// column heights, the fluid fractions and the face apertures, so an SpMV reads x plus the
// geometry (nothing for a flat bottom) instead of stored coefficients.
#pragma once

#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace fd3 {

constexpr int TPB = 256;            // threads per block of the per-cell kernels
constexpr int CHUNK = 64;           // the reference's reduction grain (delta3d.rs:867)
constexpr int CHUNKS_PER_BLOCK = TPB / CHUNK;
constexpr float SURFACE_THETA_MIN = 1e-3f;        // delta_mobile.rs:14
constexpr float PROJECTION_VELOCITY_FLOOR = 1e-4f; // delta3d.rs:41
constexpr float OMEGA = 6.f / 7.f;                // delta3d_multigrid.rs:28

enum Mode { RED_F64 = 0, RED_ORD = 1 };

// Programmatic dependent launch (sm_90+): every kernel of the library is launched so that its CTAs
// may be scheduled while the previous kernel on the stream is still running.  KSTART, the first
// statement of every kernel, waits until that previous grid has completed and its memory is
// visible (griddepcontrol.wait; a no-op when launched without the attribute), then lets the next
// kernel start scheduling (griddepcontrol.launch_dependents).  Nothing is read before the wait.
#define KSTART()                                              \
  do {                                                        \
    asm volatile("griddepcontrol.wait;" ::: "memory");        \
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); \
  } while (0)

// Fine-level geometry, passed by value to every fine kernel.
// The rigid motion of a solid: translation v, rotation w (rad/s) about c.
struct Rigid {
  float v[3], w[3], c[3];
};
// wall_velocity (delta3d.rs:75-82): component `axis` of v + w x (x - c).
__device__ __forceinline__ float wall_velocity(const Rigid& R, int axis, float x0, float x1, float x2) {
  const float r0 = x0 - R.c[0], r1 = x1 - R.c[1], r2 = x2 - R.c[2];
  if (axis == 0) return R.v[0] + (R.w[1] * r2 - R.w[2] * r1);
  if (axis == 1) return R.v[1] + (R.w[2] * r0 - R.w[0] * r2);
  return R.v[2] + (R.w[0] * r1 - R.w[1] * r0);
}

struct Geo {
  int nx, ny, nz, n;
  int cut;                // 0: flat bottom (every aperture 1, nothing solid)
  int linear;             // 1: the linear path's rows (the only ghost is the lid, coefficient 2)
  int homog;              // 1: homogeneous ghosts, value 0 (refine_mobile3, delta3d_coupling.rs:238)
  float dx, inv, rho_g, rest;
  const float* eta;       // column heights
  const float* rof;       // column roundoff (compensated sum)
  const float* frac;      // fluid fraction per cell (cut only)
  const float* ou;        // apertures (cut only)
  const float* ov;
  const float* ow;
  const unsigned char* act;  // sparse column set, 1 per column in the domain (null: every column)
  // per 32 x 8 tile of columns, 1 if any column of the tile is in the sparse set (null: every tile).
  // The blocked fine kernels skip the other tiles: every cell there is solid, every vector the
  // projection writes is 0 there (the set change zeroes them), and a skipped tile adds exactly 0 to
  // each reduction, so skipping changes no bit.
  const unsigned char* tiles;
  // A solid set in motion by set_solid_rigid: wall = 1 in translation, 2 in rotation, 0 at rest or
  // without a solid.  The divergence then adds the flux of the parts of the faces the solid covers
  // (base apertures bou/bov/bow, the bottom-only cut, minus the apertures).
  int wall;
  Rigid rig;
  const float* bou;
  const float* bov;
  const float* bow;
};
constexpr int TILE_X = 32, TILE_Y = 8;

// A coarse level (Level3, delta3d_multigrid.rs:37-52).
struct Lev {
  int nx, ny, nz, n;
  float inv;
  float* ou; float* ov; float* ow;
  float* kind; float* diag;
  float* x; float* x2; float* r; float* t;
  unsigned short* code;   // row codes of the level (k_level_prepare_b)
};

// Device-resident scalars of one projection.  Reduced values are held in double; in ordered
// mode they are exact f32 values and the algebra is done in f32.
struct Scalars {
  double b2, rr, rz, dq, rn, zn, actual;
  double tolb2;            // tol*b2 (f32 product in ordered mode)
  double phys;             // physical_target (delta3d_mobile.rs:566-567)
  float alpha, beta;       // applied step lengths
  int active;              // the inner PCG loop is running
  int status;              // 0, or 2 (NotFinite)
  int brk;                 // dq <= 0 stopped the loop
  unsigned it, max_iters;
  int any_nonzero;         // ordered-mode norm2 guard (delta3d.rs:871-875)
  float fmax[4];           // max-reductions (divergence all/plain, |u| max, backward error)
  unsigned long long hash; // fingerprint of p
  int dir_mode;            // next direction: 0 d = z (after a prime), 1 d = z + beta d
  unsigned body_runs;      // executions of the device loop body since the loop started
  // FP16-storage V-cycle: it runs on r * vinv, vinv = vk / |r| = 6 sqrt(n) / (dx^2 |r|), i.e. on
  // r / sigma with sigma = rms(r) dx^2 / 6, so its vectors stay near 1 whatever the pressure scale.
  // vk = 0 (f32 storage) leaves vinv unused.
  float vk, vinv;
};

// Storage of the V-cycle vectors (the fine z, z2 and every coarse level's x, x2, r, t): f32, or
// FP16 with f32 arithmetic.  Stores round to nearest and clamp to the finite FP16 range (a NaN
// stays a NaN, so the non-finite checks still see it).
template <class T>
struct Store;
template <>
struct Store<float> {
  static constexpr bool half = false;
  __device__ __forceinline__ static float ld(const float* p, int c) { return p[c]; }
  __device__ __forceinline__ static float2 ld2(const float* p, int c) { return *reinterpret_cast<const float2*>(p + c); }
  __device__ __forceinline__ static void st(float* p, int c, float v) { p[c] = v; }
  __device__ __forceinline__ static void st2(float* p, int c, float a, float b) {
    *reinterpret_cast<float2*>(p + c) = make_float2(a, b);
  }
  __device__ __forceinline__ static float rt(float v) { return v; }  // the value a load returns after a store
};
__device__ __forceinline__ float clamp_h(float v) { return v > 65504.f ? 65504.f : (v < -65504.f ? -65504.f : v); }
template <>
struct Store<__half> {
  static constexpr bool half = true;
  __device__ __forceinline__ static float ld(const __half* p, int c) { return __half2float(p[c]); }
  __device__ __forceinline__ static float2 ld2(const __half* p, int c) {
    return __half22float2(*reinterpret_cast<const __half2*>(p + c));
  }
  __device__ __forceinline__ static void st(__half* p, int c, float v) { p[c] = __float2half_rn(clamp_h(v)); }
  __device__ __forceinline__ static void st2(__half* p, int c, float a, float b) {
    *reinterpret_cast<__half2*>(p + c) = __floats2half2_rn(clamp_h(a), clamp_h(b));
  }
  __device__ __forceinline__ static float rt(float v) { return __half2float(__float2half_rn(clamp_h(v))); }
};
// A level's vector buffers are allocated as f32 arrays; the FP16 mode uses their first half.
template <class T>
__device__ __forceinline__ T* as(float* p) { return reinterpret_cast<T*>(p); }
// The scale applied to r on its way into the V-cycle (1 in f32 storage).
template <class T>
__device__ __forceinline__ float vscale(const Scalars* S) { return Store<T>::half ? S->vinv : 1.f; }

// Reduction scratch: per-block f64 partials, or per-64-chunk f32 partials.
struct Red {
  double* p64;
  float* p32;
  unsigned* count;         // blocks done, for the last-block finish (reset by that block)
};

// ------------------------------------------------------------------------------------------------
// Geometry predicates (delta3d_mobile.rs:92-124)

// The sparse column set (delta3d_sparse.rs:256-319).  A column outside the set is solid for every
// operator; an interior u or v face touching such a column, and every w face of one, is closed.
// Faces on the box's boundary keep the box's treatment.
__device__ __forceinline__ bool col_active(const Geo& g, int i, int j) {
  return !g.act || __ldg(g.act + j * g.nx + i) != 0;
}
__device__ __forceinline__ bool sparse_closed_ij(const unsigned char* __restrict__ act, int nx, int ny, int axis,
                                                 int i, int j) {
  if (axis == 0) return i > 0 && i < nx && (__ldg(act + j * nx + i - 1) == 0 || __ldg(act + j * nx + i) == 0);
  if (axis == 1) return j > 0 && j < ny && (__ldg(act + (j - 1) * nx + i) == 0 || __ldg(act + j * nx + i) == 0);
  return __ldg(act + j * nx + i) == 0;
}
__device__ __forceinline__ bool sparse_closed3(const Geo& g, int axis, int f) {
  int i, j;
  if (axis == 0) { i = f % (g.nx + 1); j = (f / (g.nx + 1)) % g.ny; }
  else if (axis == 1) { i = f % g.nx; j = (f / g.nx) % (g.ny + 1); }
  else { const int col = f % (g.nx * g.ny); i = col % g.nx; j = col / g.nx; }
  return sparse_closed_ij(g.act, g.nx, g.ny, axis, i, j);
}
// sparse_outside3 (delta3d_sparse.rs:307-319): the face of axis `axis` at column position (i, j)
// touches no column of the set.
__device__ __forceinline__ bool sparse_outside3(const Geo& g, int axis, int i, int j) {
  if (!g.act) return false;
  if (axis == 0) return !((i > 0 && col_active(g, i - 1, j)) || (i < g.nx && col_active(g, i, j)));
  if (axis == 1) return !((j > 0 && col_active(g, i, j - 1)) || (j < g.ny && col_active(g, i, j)));
  return !col_active(g, i, j);
}

__device__ __forceinline__ bool solid3(const Geo& g, int c) {
  if (g.cut && __ldg(g.frac + c) == 0.f) return true;
  return g.act && __ldg(g.act + c % (g.nx * g.ny)) == 0;
}

__device__ __forceinline__ bool wet3(const Geo& g, int i, int j, int k) {
  int c = (k * g.ny + j) * g.nx + i;
  if (solid3(g, c)) return false;
  return ((float)k + 0.5f) * g.dx < __ldg(g.eta + j * g.nx + i);
}

// The cut's aperture of a face, 1 on a flat bottom.  The hot stencils read it only on a face a row
// code marks live, which the sparse set never closes.
__device__ __forceinline__ float aper3(const Geo& g, int axis, int f) {
  if (!g.cut) return 1.f;
  return __ldg((axis == 0 ? g.ou : (axis == 1 ? g.ov : g.ow)) + f);
}

// open3 (delta3d_mobile.rs:105-119): 0 on a face the sparse set closes, else the cut's aperture.
__device__ __forceinline__ float open3(const Geo& g, int axis, int f) {
  if (g.act && sparse_closed3(g, axis, f)) return 0.f;
  return aper3(g, axis, f);
}

__device__ __forceinline__ int fu(const Geo& g, int i, int j, int k) { return (k * g.ny + j) * (g.nx + 1) + i; }
__device__ __forceinline__ int fv(const Geo& g, int i, int j, int k) { return (k * (g.ny + 1) + j) * g.nx + i; }
__device__ __forceinline__ int fw(const Geo& g, int i, int j, int k) { return (k * g.ny + j) * g.nx + i; }

// divergence_cut's moving-wall term (delta3d.rs:824-852), for g.wall != 0: in rotation, each face
// part the solid covers moves at the wall's velocity at the face centre; in translation, at the
// solid's velocity.  The caller adds it to the cell's divergence.
__device__ __forceinline__ float wall_flux(const Geo& g, int i, int j, int k) {
  const int ul = fu(g, i, j, k), ur = fu(g, i + 1, j, k), vl = fv(g, i, j, k), vr = fv(g, i, j + 1, k);
  const int wl = fw(g, i, j, k), wr = fw(g, i, j, k + 1);
  const float cul = __ldg(g.bou + ul) - __ldg(g.ou + ul), cur = __ldg(g.bou + ur) - __ldg(g.ou + ur);
  const float cvl = __ldg(g.bov + vl) - __ldg(g.ov + vl), cvr = __ldg(g.bov + vr) - __ldg(g.ov + vr);
  const float cwl = __ldg(g.bow + wl) - __ldg(g.ow + wl), cwr = __ldg(g.bow + wr) - __ldg(g.ow + wr);
  const float dx = g.dx;
  if (g.wall == 2) {
    const float xc = ((float)i + 0.5f) * dx, yc = ((float)j + 0.5f) * dx, zc = ((float)k + 0.5f) * dx;
    const float x0 = (float)i * dx, x1 = (float)(i + 1) * dx;
    const float y0 = (float)j * dx, y1 = (float)(j + 1) * dx;
    const float z0 = (float)k * dx, z1 = (float)(k + 1) * dx;
    const float fx = cur * wall_velocity(g.rig, 0, x1, yc, zc) - cul * wall_velocity(g.rig, 0, x0, yc, zc);
    const float fy = cvr * wall_velocity(g.rig, 1, xc, y1, zc) - cvl * wall_velocity(g.rig, 1, xc, y0, zc);
    const float fz = cwr * wall_velocity(g.rig, 2, xc, yc, z1) - cwl * wall_velocity(g.rig, 2, xc, yc, z0);
    return (fx + fy + fz) / dx;
  }
  const float x = cur - cul, y = cvr - cvl, z = cwr - cwl;
  return (g.rig.v[0] * x + g.rig.v[1] * y + g.rig.v[2] * z) / dx;
}

// ghost_up3 (delta3d_mobile.rs:126-134)
__device__ __forceinline__ void ghost_up3(const Geo& g, int i, int j, int k, float& it, float& value) {
  int col = j * g.nx + i;
  float h = __ldg(g.eta + col);
  float theta = fmaxf((h - ((float)k + 0.5f) * g.dx) / g.dx, SURFACE_THETA_MIN);
  value = g.homog ? 0.f : g.rho_g * ((h - g.rest) - __ldg(g.rof + col));
  it = 1.f / theta;
}

// ghost_side3 (delta3d_mobile.rs:136-147)
__device__ __forceinline__ void ghost_side3(const Geo& g, int i, int j, int k, int x, int y, float& it, float& value) {
  float zc = ((float)k + 0.5f) * g.dx;
  float h = __ldg(g.eta + j * g.nx + i);
  float theta = fmaxf((h - zc) / (h - __ldg(g.eta + y * g.nx + x)), SURFACE_THETA_MIN);
  value = g.homog ? 0.f : g.rho_g * (zc - g.rest);
  it = 1.f / theta;
}

struct RowE { int n; float a, it, val; };  // n < 0: no fluid neighbour (a wall, a ghost or nothing)

// mobile_row (delta3d_mobile.rs:152-188): order x-, x+, y-, y+, z-, z+.  Every operand the decisions
// may need (apertures, the neighbours' solid tests and column heights) is loaded first, each behind
// its bounds test, so the loads go out together; the decisions then follow the reference's order.
__device__ __forceinline__ void mobile_row(const Geo& g, int i, int j, int k, RowE row[6]) {
#pragma unroll
  for (int f = 0; f < 6; ++f) row[f] = RowE{-1, 0.f, 0.f, 0.f};
  const int nxny = g.nx * g.ny;
  const int c = (k * g.ny + j) * g.nx + i;
  const bool ok[4] = {i > 0, i + 1 < g.nx, j > 0, j + 1 < g.ny};
  const int xs[4] = {i - 1, i + 1, i, i}, ys[4] = {j, j, j - 1, j + 1};
  const int fi[4] = {fu(g, i, j, k), fu(g, i + 1, j, k), fv(g, i, j, k), fv(g, i, j + 1, k)};
  float a[4], hn[4];
  bool sol[4];
#pragma unroll
  for (int f = 0; f < 4; ++f) {
    const int cn = (k * g.ny + ys[f]) * g.nx + xs[f];
    a[f] = ok[f] ? open3(g, f < 2 ? 0 : 1, fi[f]) : 0.f;
    sol[f] = ok[f] ? solid3(g, cn) : true;
    hn[f] = ok[f] ? __ldg(g.eta + ys[f] * g.nx + xs[f]) : 0.f;
  }
  const float down = open3(g, 2, fw(g, i, j, k));
  const bool sol_down = k > 0 ? solid3(g, c - nxny) : true;
  const float up = open3(g, 2, fw(g, i, j, k + 1));
  const bool above = k + 1 < g.nz;
  const bool sol_up = above ? solid3(g, c + nxny) : true;
  const float hc = __ldg(g.eta + j * g.nx + i);
#pragma unroll
  for (int f = 0; f < 4; ++f) {
    if (!ok[f]) continue;
    if (a[f] == 0.f || sol[f]) continue;
    const int x = xs[f], y = ys[f];
    const int cn = (k * g.ny + y) * g.nx + x;
    if (((float)k + 0.5f) * g.dx < hn[f]) row[f] = RowE{cn, a[f], 0.f, 0.f};  // wet3 of the neighbour
    else { float it, b; ghost_side3(g, i, j, k, x, y, it, b); row[f] = RowE{-1, a[f], it, b}; }
  }
  if (k > 0 && down > 0.f && !sol_down) row[4] = RowE{c - nxny, down, 0.f, 0.f};
  if (up > 0.f) {
    if (above && !sol_up && ((float)(k + 1) + 0.5f) * g.dx < hc) row[5] = RowE{c + nxny, up, 0.f, 0.f};
    else { float it, b; ghost_up3(g, i, j, k, it, b); row[5] = RowE{-1, up, it, b}; }
  }
}

// One row of apply_mobile3 (delta3d_mobile.rs:197-209) at a wet cell.
__device__ __forceinline__ float apply_row(const Geo& g, int i, int j, int k, int c, const float* __restrict__ p) {
  RowE row[6];
  mobile_row(g, i, j, k, row);
  float pc = p[c];
  float acc = 0.f;
#pragma unroll
  for (int f = 0; f < 6; ++f) {
    if (row[f].n >= 0) acc += row[f].a * (pc - p[row[f].n]);
    else if (row[f].a > 0.f) acc += row[f].a * pc * row[f].it;
  }
  return acc * g.inv;
}

__device__ __forceinline__ void cell_ijk(const Geo& g, int c, int& i, int& j, int& k) {
  i = c % g.nx;
  int t = c / g.nx;
  j = t % g.ny;
  k = t / g.ny;
}

// ------------------------------------------------------------------------------------------------
// Block reductions.  F64: f64 tree per block -> Red.p64[block].  ORD: the reference's order: each
// 64-cell chunk summed serially in f32 from +0 (delta3d.rs:864-866) -> Red.p32[chunk]; the chunks
// are merged serially by k_finish.

template <int MODE> struct Acc;
template <> struct Acc<RED_F64> {
  typedef double T;
  static __device__ __forceinline__ double prod(float a, float b) { return (double)a * (double)b; }
  static __device__ __forceinline__ double prod3(float a, float b, float c) { return (double)a * (double)b * (double)c; }
};
template <> struct Acc<RED_ORD> {
  typedef float T;
  static __device__ __forceinline__ float prod(float a, float b) { return a * b; }
  static __device__ __forceinline__ float prod3(float a, float b, float c) { return a * b * c; }
};

template <int MODE>
__device__ __forceinline__ void block_reduce(typename Acc<MODE>::T v, int c, int n, Red red) {
  if (MODE == RED_F64) {
    __shared__ double sw[TPB / 32];
    double s = (c < n) ? (double)v : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) sw[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
#pragma unroll
      for (int w = 0; w < TPB / 32; ++w) t += sw[w];
      red.p64[blockIdx.x] = t;
    }
  } else {
    __shared__ float sv[TPB];
    sv[threadIdx.x] = (float)v;
    __syncthreads();
    if (threadIdx.x < CHUNKS_PER_BLOCK) {
      int q = blockIdx.x * CHUNKS_PER_BLOCK + threadIdx.x;
      int start = q * CHUNK;
      if (start < n) {
        int cnt = min(CHUNK, n - start);
        float acc = 0.f;
        for (int e = 0; e < cnt; ++e) acc += sv[threadIdx.x * CHUNK + e];
        red.p32[q] = acc;
      }
    }
  }
}

__device__ __forceinline__ void flag_nonzero(bool nz, Scalars* S) {
  if (__syncthreads_or(nz) && threadIdx.x == 0) atomicOr(&S->any_nonzero, 1);
}

// ------------------------------------------------------------------------------------------------
// Assembly

// divergence / divergence_cut (delta3d.rs:747-763, 806-855) of cell c, a solid at rest.
__device__ __forceinline__ float divergence_at(const Geo& g, const float* __restrict__ u,
                                               const float* __restrict__ v, const float* __restrict__ w, int c) {
  int i, j, k; cell_ijk(g, c, i, j, k);
  if (g.cut) {
    if (__ldg(g.frac + c) == 0.f) return 0.f;
    float fl = __ldg(g.ou + fu(g, i, j, k)) * u[fu(g, i, j, k)];
    float fr = __ldg(g.ou + fu(g, i + 1, j, k)) * u[fu(g, i + 1, j, k)];
    float ff = __ldg(g.ov + fv(g, i, j, k)) * v[fv(g, i, j, k)];
    float fk = __ldg(g.ov + fv(g, i, j + 1, k)) * v[fv(g, i, j + 1, k)];
    float fb = __ldg(g.ow + fw(g, i, j, k)) * w[fw(g, i, j, k)];
    float ft = __ldg(g.ow + fw(g, i, j, k + 1)) * w[fw(g, i, j, k + 1)];
    float d = ((fr - fl + ft - fb) + (fk - ff)) / g.dx;
    if (g.wall) d = d + wall_flux(g, i, j, k);
    return d;
  }
  float fl = u[fu(g, i, j, k)], fr = u[fu(g, i + 1, j, k)];
  float ff = v[fv(g, i, j, k)], fk = v[fv(g, i, j + 1, k)];
  float fb = w[fw(g, i, j, k)], ft = w[fw(g, i, j, k + 1)];
  return ((fr - fl + ft - fb) + (fk - ff)) / g.dx;
}
__global__ void k_divergence(Geo g, const float* __restrict__ u, const float* __restrict__ v,
                             const float* __restrict__ w, float* __restrict__ out) {
  KSTART();
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= g.n) return;
  out[c] = divergence_at(g, u, v, w, c);
}

// p = 0 on dry cells (delta3d_mobile.rs:485-494).
__global__ void k_zero_dry(Geo g, float* __restrict__ p) {
  KSTART();
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= g.n) return;
  int i, j, k; cell_ijk(g, c, i, j, k);
  if (!wet3(g, i, j, k)) p[c] = 0.f;
}

// out = A x (apply_mobile3).
__global__ void k_apply(Geo g, const float* __restrict__ x, float* __restrict__ out) {
  KSTART();
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= g.n) return;
  int i, j, k; cell_ijk(g, c, i, j, k);
  out[c] = wet3(g, i, j, k) ? apply_row(g, i, j, k, c, x) : 0.f;
}

// dir = z + beta dir, z = prec res (prime_mobile3, delta3d_mobile.rs:435-445).  use_beta = 0 is
// the `beta == 0` branch (dir = z).
__global__ void k_jacobi_dir(int n, const float* __restrict__ prec, const float* __restrict__ r, float* __restrict__ d,
                             const Scalars* S, int gate, int use_beta) {
  KSTART();
  if (gate && !S->active) return;
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n) return;
  float beta = use_beta ? S->beta : 0.f;
  float z = prec[c] * r[c];
  d[c] = beta == 0.f ? z : z + beta * d[c];
}

// ------------------------------------------------------------------------------------------------
// Coarse levels (row_sums, smooth3, restrict3, prolong_add3, coarse_cycle3;
// delta3d_multigrid.rs:216-332).

// One row of row_sums with p given (kind > 0 at c).
__device__ __forceinline__ float level_row(const Lev& L, int i, int j, int k, int c, const float* __restrict__ p) {
  const float pc = p[c];
  float acc = 0.f;
  const int nxny = L.nx * L.ny;
  auto face = [&](float a, bool has, int m, bool top) {
    if (a == 0.f) return;
    if (has) {
      float km = L.kind[m];
      if (km > 0.f) acc += a * (pc - p[m]);
      else if (km < 0.f) acc += 2.f * a * pc;
    } else if (top) {
      acc += 2.f * a * pc;
    }
  };
  face(L.ou[(k * L.ny + j) * (L.nx + 1) + i], i > 0, c - 1, false);
  face(L.ou[(k * L.ny + j) * (L.nx + 1) + i + 1], i + 1 < L.nx, c + 1, false);
  face(L.ov[(k * (L.ny + 1) + j) * L.nx + i], j > 0, c - L.nx, false);
  face(L.ov[(k * (L.ny + 1) + j + 1) * L.nx + i], j + 1 < L.ny, c + L.nx, false);
  face(L.ow[(k * L.ny + j) * L.nx + i], k > 0, c - nxny, false);
  face(L.ow[((k + 1) * L.ny + j) * L.nx + i], k + 1 < L.nz, c + nxny, true);
  return acc * L.inv;
}

// The diagonal: row_sums with p absent (delta3d_multigrid.rs:205, 236-241).
__device__ __forceinline__ float level_diag_at(const Lev& L, int c) {
  int i = c % L.nx, t = c / L.nx, j = t % L.ny, k = t / L.ny;
  if (L.kind[c] <= 0.f) return 0.f;
  float acc = 0.f;
  const int nxny = L.nx * L.ny;
  auto face = [&](float a, bool has, int m, bool top) {
    if (a == 0.f) return;
    if (has) {
      float km = L.kind[m];
      if (km > 0.f) acc += a;
      else if (km < 0.f) acc += 2.f * a * 1.f;
    } else if (top) {
      acc += 2.f * a * 1.f;
    }
  };
  face(L.ou[(k * L.ny + j) * (L.nx + 1) + i], i > 0, c - 1, false);
  face(L.ou[(k * L.ny + j) * (L.nx + 1) + i + 1], i + 1 < L.nx, c + 1, false);
  face(L.ov[(k * (L.ny + 1) + j) * L.nx + i], j > 0, c - L.nx, false);
  face(L.ov[(k * (L.ny + 1) + j + 1) * L.nx + i], j + 1 < L.ny, c + L.nx, false);
  face(L.ow[(k * L.ny + j) * L.nx + i], k > 0, c - nxny, false);
  face(L.ow[((k + 1) * L.ny + j) * L.nx + i], k + 1 < L.nz, c + nxny, true);
  return acc * L.inv;
}

// Damped Jacobi sweep (smooth3): xout = xin + w (r - L xin) / diag where diag > 0.  zero_in = 1
// is the first sweep after `x.fill(0)`: L 0 = +0 exactly, so xout = 0 + w (r - 0) / diag.
__global__ void k_level_sweep(Lev L, const float* __restrict__ xin, float* __restrict__ xout, int zero_in,
                              const Scalars* S, int gate) {
  KSTART();
  if (gate && !S->active) return;
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= L.n) return;
  float dg = L.diag[c];
  if (zero_in) {
    xout[c] = dg > 0.f ? 0.f + OMEGA * (L.r[c] - 0.f) / dg : 0.f;
    return;
  }
  float xc = xin[c];
  if (dg > 0.f) {
    int i = c % L.nx, t = c / L.nx, j = t % L.ny, k = t / L.ny;
    float tv = level_row(L, i, j, k, c, xin);  // diag > 0 implies kind > 0
    xc += OMEGA * (L.r[c] - tv) / dg;
  }
  xout[c] = xc;
}

// Coarse r of level C = mean over 8 children of (r - L x) on level F.
__global__ void k_level_restrict(Lev F, Lev C, const Scalars* S, int gate) {
  KSTART();
  if (gate && !S->active) return;
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= C.n) return;
  int ci = q % C.nx, t = q / C.nx, cj = t % C.ny, ck = t / C.ny;
  float s = 0.f;
#pragma unroll
  for (int e = 0; e < 8; ++e) {
    int i = 2 * ci + (e & 1), j = 2 * cj + ((e >> 1) & 1), k = 2 * ck + (e >> 2);
    int c = (k * F.ny + j) * F.nx + i;
    float lx = F.kind[c] > 0.f ? level_row(F, i, j, k, c, F.x) : 0.f;
    s += F.r[c] - lx;
  }
  C.r[q] = 0.125f * s;
}

// ------------------------------------------------------------------------------------------------
// coarsen3 (delta3d_multigrid.rs:141-206) and fine_kind3 (:357-367)

__device__ __forceinline__ float coarsen_kind_fine_at(const Geo& g, const Lev& C, int q) {
  int ci = q % C.nx, t = q / C.nx, cj = t % C.ny, ck = t / C.ny;
  bool active = false, air = false;
#pragma unroll
  for (int e = 0; e < 8; ++e) {
    int i = 2 * ci + (e & 1), j = 2 * cj + ((e >> 1) & 1), k = 2 * ck + (e >> 2);
    int c = (k * g.ny + j) * g.nx + i;
    float v = wet3(g, i, j, k) ? 1.f : (solid3(g, c) ? 0.f : -1.f);
    if (v > 0.f) active = true;
    else if (v < 0.f) air = true;
  }
  return active ? 1.f : (air ? -1.f : 0.f);
}

__device__ __forceinline__ float coarsen_kind_level_at(const Lev& F, const Lev& C, int q) {
  int ci = q % C.nx, t = q / C.nx, cj = t % C.ny, ck = t / C.ny;
  bool active = false, air = false;
#pragma unroll
  for (int e = 0; e < 8; ++e) {
    int i = 2 * ci + (e & 1), j = 2 * cj + ((e >> 1) & 1), k = 2 * ck + (e >> 2);
    float v = F.kind[(k * F.ny + j) * F.nx + i];
    if (v > 0.f) active = true;
    else if (v < 0.f) air = true;
  }
  return active ? 1.f : (air ? -1.f : 0.f);
}

// Coarse apertures: mean of the 4 fine faces a coarse face covers.  `fo*` are the fine apertures
// (nullptr: a flat fine level, every aperture 1).  fnx/fny are the fine dimensions.
__device__ __forceinline__ void coarsen_open_at(int fnx, int fny, const float* __restrict__ fou,
                                                const float* __restrict__ fov, const float* __restrict__ fow,
                                                const unsigned char* __restrict__ act, const Lev& C, int q) {
  int cx = C.nx, cy = C.ny, cz = C.nz;
  int nu = (cx + 1) * cy * cz, nv = cx * (cy + 1) * cz, nw = cx * cy * (cz + 1);
  if (q < nu) {
    int i = q % (cx + 1), t = q / (cx + 1), j = t % cy, k = t / cy;
    float s = 0.f;
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      int dj = e & 1, dk = e >> 1;
      float a = fou ? fou[((2 * k + dk) * fny + 2 * j + dj) * (fnx + 1) + 2 * i] : 1.f;
      if (act && sparse_closed_ij(act, fnx, fny, 0, 2 * i, 2 * j + dj)) a = 0.f;
      s += a;
    }
    C.ou[q] = 0.25f * s;
    return;
  }
  q -= nu;
  if (q < nv) {
    int i = q % cx, t = q / cx, j = t % (cy + 1), k = t / (cy + 1);
    float s = 0.f;
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      int di = e & 1, dk = e >> 1;
      float a = fov ? fov[((2 * k + dk) * (fny + 1) + 2 * j) * fnx + 2 * i + di] : 1.f;
      if (act && sparse_closed_ij(act, fnx, fny, 1, 2 * i + di, 2 * j)) a = 0.f;
      s += a;
    }
    C.ov[q] = 0.25f * s;
    return;
  }
  q -= nv;
  if (q < nw) {
    int i = q % cx, t = q / cx, j = t % cy, k = t / cy;
    float s = 0.f;
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      int di = e & 1, dj = e >> 1;
      float a = fow ? fow[((2 * k) * fny + 2 * j + dj) * fnx + 2 * i + di] : 1.f;
      if (act && sparse_closed_ij(act, fnx, fny, 2, 2 * i + di, 2 * j + dj)) a = 0.f;
      s += a;
    }
    C.ow[q] = 0.25f * s;
  }
}

// ------------------------------------------------------------------------------------------------
// Correction and diagnostics

// Order-independent float max of non-negative values (NaN-free inputs compare as their bits).
__device__ __forceinline__ void atomic_fmax_nonneg(float* addr, float v) {
  if (!(v > 0.f)) return;  // +0 initial value; NaN is ignored, as Rust's f32::max does
  atomicMax(reinterpret_cast<int*>(addr), __float_as_int(v));
}

// The block's maxima of two nonnegative values (warp shuffles, then the warps' maxima through
// shared memory) merged into addr0 / addr1 by thread 0: one atomic per block and value.  Atomics on
// one address serialise in L2, so a metric over millions of cells keeps them to one per block.
// Every thread of the block calls it (it holds a barrier).  NaN is ignored, as fmaxf does.
__device__ __forceinline__ void block_fmax2_atomic(float a, float b, float* addr0, float* addr1) {
  __shared__ float pa[32], pb[32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    a = fmaxf(a, __shfl_down_sync(0xffffffffu, a, o));
    b = fmaxf(b, __shfl_down_sync(0xffffffffu, b, o));
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) { pa[wid] = a; pb[wid] = b; }
  __syncthreads();
  if (wid == 0) {
    const bool on = lane < (int)(blockDim.x >> 5);
    a = on ? pa[lane] : 0.f;
    b = on ? pb[lane] : 0.f;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      a = fmaxf(a, __shfl_down_sync(0xffffffffu, a, o));
      b = fmaxf(b, __shfl_down_sync(0xffffffffu, b, o));
    }
    if (lane == 0) {
      if (addr0) atomic_fmax_nonneg(addr0, a);
      if (addr1) atomic_fmax_nonneg(addr1, b);
    }
  }
}

// Cells per thread of the max-metric kernels (a block covers METRIC_CELLS * blockDim.x cells).
constexpr int METRIC_CELLS = 4;

// max |x| over the three face families into S->fmax[slot] (one launch, 16-byte loads; each array
// starts on a 16-byte boundary).
__global__ void k_maxabs3(const float* __restrict__ u, int nu, const float* __restrict__ v, int nv,
                          const float* __restrict__ w, int nw, Scalars* S, int slot) {
  KSTART();
  const int stride = gridDim.x * blockDim.x, tid = blockIdx.x * blockDim.x + threadIdx.x;
  float m = 0.f;
  auto scan = [&](const float* __restrict__ x, int n) {
    const int n4 = n / 4;
    const float4* x4 = reinterpret_cast<const float4*>(x);
    for (int q = tid; q < n4; q += stride) {
      const float4 a = x4[q];
      m = fmaxf(m, fabsf(a.x));
      m = fmaxf(m, fabsf(a.y));
      m = fmaxf(m, fabsf(a.z));
      m = fmaxf(m, fabsf(a.w));
    }
    for (int q = 4 * n4 + tid; q < n; q += stride) m = fmaxf(m, fabsf(x[q]));
  };
  scan(u, nu);
  scan(v, nv);
  scan(w, nw);
  block_fmax2_atomic(m, 0.f, &S->fmax[slot], nullptr);
}

// Fingerprint of the exact bits of p for cycle detection (the role of fingerprint,
// delta3d.rs:1360-1369).  The reference hashes the bytes serially (FNV-1a); a serial chain does
// not map to a GPU, so each element's bits are mixed with its index (SplitMix64 finaliser) and the
// mixes are summed mod 2^64: a function of the exact bits of p, independent of the launch shape.
__device__ __forceinline__ unsigned long long mix64(unsigned long long z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
__device__ __forceinline__ unsigned long long hash_val(float x, int q) {
  return mix64(((unsigned long long)(unsigned)__float_as_int(x) << 32 | (unsigned)q) + 0x9E3779B97F4A7C15ull);
}
__device__ __forceinline__ unsigned long long hash_at(const float* __restrict__ p, int q) { return hash_val(p[q], q); }
__global__ void k_hash(int n, const float* __restrict__ p, Scalars* S) {
  KSTART();
  unsigned long long h = 0;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) h += hash_at(p, q);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) h += __shfl_down_sync(0xffffffffu, h, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(&S->hash, h);
}

// ------------------------------------------------------------------------------------------------
// Finishing a reduction, then the scalar algebra of the PCG step that consumes it.

enum FinOp {
  FIN_B2 = 0,      // b2 = |rhs|^2 (norm2 checks)
  FIN_RR0 = 1,     // rr = |res|^2 initial (norm2 checks)
  FIN_DQ = 2,      // dq; alpha = rz/dq or stop (delta3d_mobile.rs:528-531)
  FIN_RN = 3,      // rn = |r|^2 (norm2 checks); decides whether the loop continues
  FIN_RZ_ITER = 4, // zn; beta = zn/rz; rz = zn; rr = rn; it++ (delta3d_mobile.rs:538-545)
  FIN_RZ_PRIME = 5,// rz of a fresh direction (prime_*: delta3d_mobile.rs:517, 587)
  FIN_ACTUAL = 6   // true residual |b - A p|^2 (norm2 checks)
};

__device__ __forceinline__ bool loop_continues(const Scalars* S, double rn, unsigned it_next, int ord) {
  bool above = ord ? ((float)rn > (float)S->tolb2 || (float)rn > (float)S->phys) : (rn > S->tolb2 || rn > S->phys);
  return above && it_next < S->max_iters;
}

// ------------------------------------------------------------------------------------------------
// The rest of the mobile step (delta3d_mobile.rs:615-813)

// advect_mobile3 (delta3d_mobile.rs:615-732): centred MAC advection of every open interior face
// into us/vs/ws; every other face copies the current velocity.
__global__ void k_advect(Geo g, float dt, const float* __restrict__ u, const float* __restrict__ v,
                         const float* __restrict__ w, float* __restrict__ us, float* __restrict__ vs,
                         float* __restrict__ ws) {
  KSTART();
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int nu = (nx + 1) * ny * nz, nv = nx * (ny + 1) * nz, nw = nx * ny * (nz + 1);
  const float h = 0.5f / g.dx;
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q < nu + nv) {
    const int axis = q < nu ? 0 : 1;
    const int f = axis == 0 ? q : q - nu;
    int i, j, k;
    if (axis == 0) { i = f % (nx + 1); int t = f / (nx + 1); j = t % ny; k = t / ny; }
    else { i = f % nx; int t = f / nx; j = t % (ny + 1); k = t / (ny + 1); }
    const int a = axis == 0 ? i : j, b = axis == 0 ? j : i;
    const int na = axis == 0 ? nx : ny, nb = axis == 0 ? ny : nx;
    float cur = axis == 0 ? u[f] : v[f];
    if (a >= 1 && a < na && open3(g, axis, f) != 0.f) {
      auto val = [&](int A, int B, int K) { return axis == 0 ? u[fu(g, A, B, K)] : v[fv(g, B, A, K)]; };
      auto vertical = [&](int A, int B, int K) { return axis == 0 ? w[fw(g, A, B, K)] : w[fw(g, B, A, K)]; };
      auto transverse = [&](int A, int B, int K) { return axis == 0 ? v[fv(g, A, B, K)] : u[fu(g, B, A, K)]; };
      float uc = val(a, b, k);
      float ux = (val(a + 1, b, k) - val(a - 1, b, k)) * h;
      float upv = k + 1 < nz ? val(a, b, k + 1) : uc;
      float dn = k > 0 ? val(a, b, k - 1) : uc;
      float uz = (upv - dn) * h;
      float wc = 0.25f * (vertical(a - 1, b, k) + vertical(a, b, k) + vertical(a - 1, b, k + 1) + vertical(a, b, k + 1));
      // the edge of the sparse set reads as the box's edge (delta3d_mobile.rs:664-667)
      auto outside = [&](int A, int B) { return axis == 0 ? sparse_outside3(g, 0, A, B) : sparse_outside3(g, 1, B, A); };
      float rt = b + 1 < nb && !outside(a, b + 1) ? val(a, b + 1, k) : uc;
      float lf = b > 0 && !outside(a, b - 1) ? val(a, b - 1, k) : uc;
      float uy = (rt - lf) * h;
      float vc = 0.25f * (transverse(a - 1, b, k) + transverse(a, b, k) + transverse(a - 1, b + 1, k) + transverse(a, b + 1, k));
      cur = uc - dt * (uc * ux + wc * uz + vc * uy);
    }
    if (axis == 0) us[f] = cur; else vs[f] = cur;
    return;
  }
  q -= nu + nv;
  if (q >= nw) return;
  const int f = q;
  const int i = f % nx, t = f / nx, j = t % ny, k = t / ny;
  float cur = w[f];
  if (k >= 1 && k < nz && open3(g, 2, f) != 0.f) {
    float wc = w[f];
    float rt = i + 1 < nx && !sparse_outside3(g, 2, i + 1, j) ? w[fw(g, i + 1, j, k)] : wc;
    float lf = i > 0 && !sparse_outside3(g, 2, i - 1, j) ? w[fw(g, i - 1, j, k)] : wc;
    float wx = (rt - lf) * h;
    float wz = (w[fw(g, i, j, k + 1)] - w[fw(g, i, j, k - 1)]) * h;
    float uc = 0.25f * (u[fu(g, i, j, k - 1)] + u[fu(g, i + 1, j, k - 1)] + u[fu(g, i, j, k)] + u[fu(g, i + 1, j, k)]);
    float bk = j + 1 < ny && !sparse_outside3(g, 2, i, j + 1) ? w[fw(g, i, j + 1, k)] : wc;
    float fr = j > 0 && !sparse_outside3(g, 2, i, j - 1) ? w[fw(g, i, j - 1, k)] : wc;
    float wy = (bk - fr) * h;
    float vc = 0.25f * (v[fv(g, i, j, k - 1)] + v[fv(g, i, j + 1, k - 1)] + v[fv(g, i, j, k)] + v[fv(g, i, j + 1, k)]);
    cur = wc - dt * (uc * wx + wc * wz + vc * wy);
  }
  ws[f] = cur;
}

// The velocity of family `axis` at position p (velocity3, delta3d_coupling.rs:298-305).
__device__ __forceinline__ float vel3(const Geo& g, const float* __restrict__ u, const float* __restrict__ v,
                                      const float* __restrict__ w, int axis, int i, int j, int k) {
  if (axis == 0) return u[fu(g, i, j, k)];
  if (axis == 1) return v[fv(g, i, j, k)];
  return w[fw(g, i, j, k)];
}

// correct_advection3 (delta3d_advection.rs:31-111) of the uncoupled step: + (dt^2/2) sum_ab V_a V_b
// d_a d_b u on the predicted us/vs/ws, V collocated at the face (collocated3, delta3d_coupling.rs:
// 308-328), derivatives of the velocities at the start of the step.  A direction with a neighbour
// outside its axis's grid (the box's or the sparse set's) is left out, and so is a cross term with
// a diagonal neighbour outside the set.  One thread per face; a face reads u, v, w and writes only
// itself.
__global__ void k_correct_advection(Geo g, float dt, const float* __restrict__ u, const float* __restrict__ v,
                                    const float* __restrict__ w, float* __restrict__ us, float* __restrict__ vs,
                                    float* __restrict__ ws) {
  KSTART();
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int nu = (nx + 1) * ny * nz, nv = nx * (ny + 1) * nz, nw = nx * ny * (nz + 1);
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  int axis;
  if (q < nu) axis = 0;
  else if ((q -= nu) < nv) axis = 1;
  else if ((q -= nv) < nw) axis = 2;
  else return;
  const int dims[3] = {nx, ny, nz};
  const int end[3] = {nx + (axis == 0), ny + (axis == 1), nz + (axis == 2)};
  const int p[3] = {q % end[0], (q / end[0]) % end[1], q / (end[0] * end[1])};
  if (p[axis] == 0 || (axis < 2 && p[axis] == dims[axis])) return;
  if (open3(g, axis, q) == 0.f) return;
  auto V = [&](int a, const int r[3]) { return vel3(g, u, v, w, a, r[0], r[1], r[2]); };
  float vel[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    float col;
    if (a == axis) {
      col = V(a, p);
    } else {
      int lo[3] = {p[0], p[1], p[2]};
      lo[axis] -= 1;
      int hi[3] = {lo[0], lo[1], lo[2]};
      hi[a] += 1;
      if (axis == 2 && p[2] == nz) {
        col = 0.5f * (V(a, lo) + V(a, hi));
      } else {
        int qq[3] = {lo[0], lo[1], lo[2]}, rr[3] = {hi[0], hi[1], hi[2]};
        qq[axis] += 1;
        rr[axis] += 1;
        col = a < axis ? 0.25f * (V(a, lo) + V(a, hi) + V(a, qq) + V(a, rr))
                       : 0.25f * (V(a, lo) + V(a, qq) + V(a, hi) + V(a, rr));
      }
    }
    vel[a] = 0.f + col;  // the carried background velocity is 0 on the uncoupled step
  }
  const float c = V(axis, p);
  auto shifted = [&](int da, int sa, int db, int sb, int r[3]) {
    r[0] = p[0]; r[1] = p[1]; r[2] = p[2];
    r[da] += sa;
    if (db >= 0) r[db] += sb;
  };
  auto at = [&](int da, int sa, int db, int sb) { int r[3]; shifted(da, sa, db, sb, r); return V(axis, r); };
  auto outside = [&](int da, int sa, int db, int sb) {
    if (!g.act) return false;
    int r[3]; shifted(da, sa, db, sb, r);
    return sparse_outside3(g, axis, r[0], r[1]);
  };
  auto inside = [&](int a) { return p[a] > 0 && p[a] + 1 < end[a] && !outside(a, 1, -1, 0) && !outside(a, -1, -1, 0); };
  float acc = 0.f;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    if (!inside(a)) continue;
    acc += vel[a] * vel[a] * (at(a, 1, -1, 0) - 2.f * c + at(a, -1, -1, 0));
#pragma unroll
    for (int b = a + 1; b < 3; ++b) {
      if (!inside(b)) continue;
      if (outside(a, 1, b, 1) || outside(a, 1, b, -1) || outside(a, -1, b, 1) || outside(a, -1, b, -1)) continue;
      const float cross = at(a, 1, b, 1) - at(a, 1, b, -1) - at(a, -1, b, 1) + at(a, -1, b, -1);
      acc += 2.f * vel[a] * vel[b] * 0.25f * cross;
    }
  }
  const float scale = 0.5f * dt * dt;
  const float term = scale * acc / (g.dx * g.dx);
  if (axis == 0) us[q] += term;
  else if (axis == 1) vs[q] += term;
  else ws[q] += term;
}

// extrapolate_mobile3 (delta3d_mobile.rs:345-394): one thread per column and axis walks up the
// column and copies the last solved face into the unsolved open faces above it.
__global__ void k_extrapolate(Geo g, float* __restrict__ u, float* __restrict__ v, float* __restrict__ w) {
  KSTART();
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= 3 * g.nx * g.ny) return;
  const int axis = q / (g.nx * g.ny);
  const int col = q % (g.nx * g.ny);
  const int i = col % g.nx, j = col / g.nx;
  if ((axis == 0 && i == 0) || (axis == 1 && j == 0)) return;
  float* field = axis == 0 ? u : (axis == 1 ? v : w);
  bool has_last = false;
  float last = 0.f;
  const int start = axis == 2 ? 1 : 0, end = axis == 2 ? g.nz + 1 : g.nz;
  for (int k = start; k < end; ++k) {
    int f;
    bool solved;
    if (axis == 0) {
      f = fu(g, i, j, k);
      solved = open3(g, 0, f) > 0.f && !solid3(g, (k * g.ny + j) * g.nx + i - 1) && !solid3(g, (k * g.ny + j) * g.nx + i) &&
               (wet3(g, i - 1, j, k) || wet3(g, i, j, k));
    } else if (axis == 1) {
      f = fv(g, i, j, k);
      solved = open3(g, 1, f) > 0.f && !solid3(g, (k * g.ny + j - 1) * g.nx + i) && !solid3(g, (k * g.ny + j) * g.nx + i) &&
               (wet3(g, i, j - 1, k) || wet3(g, i, j, k));
    } else {
      f = fw(g, i, j, k);
      solved = open3(g, 2, f) > 0.f && wet3(g, i, j, k - 1);
    }
    if (open3(g, axis, f) == 0.f) continue;
    if (solved) { last = field[f]; has_last = true; }
    else if (has_last) field[f] = last;
  }
}

// transport_mobile3 (delta3d_mobile.rs:734-782), fluxes: wet column flux through every interior
// lateral face, read from eta^n.  Boundary entries stay zero (the walls).
__global__ void k_transport_flux(Geo g, const float* __restrict__ u, const float* __restrict__ v,
                                 float* __restrict__ flux_x, float* __restrict__ flux_y) {
  KSTART();
  const int nfx = (g.nx + 1) * g.ny, nfy = g.nx * (g.ny + 1);
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nfx + nfy) return;
  const int axis = q < nfx ? 0 : 1;
  int i, j;
  if (axis == 0) { i = q % (g.nx + 1); j = q / (g.nx + 1); }
  else { int r = q - nfx; i = r % g.nx; j = r / g.nx; }
  float qf = 0.f;
  bool interior = axis == 0 ? (i >= 1 && i < g.nx) : (j >= 1 && j < g.ny);
  if (interior) {
    int x = axis == 0 ? i - 1 : i, y = axis == 0 ? j : j - 1;
    float surface = 0.5f * (g.eta[y * g.nx + x] + g.eta[j * g.nx + i]);
    for (int k = 0; k < g.nz; ++k) {
      float wet = (surface - (float)k * g.dx) / g.dx;
      wet = wet < 0.f ? 0.f : (wet > 1.f ? 1.f : wet);
      if (wet == 0.f) break;
      float uu, a;
      if (axis == 0) { int f = fu(g, i, j, k); uu = u[f]; a = open3(g, 0, f); }
      else { int f = fv(g, i, j, k); uu = v[f]; a = open3(g, 1, f); }
      qf += a * uu * g.dx * wet;
    }
  }
  if (axis == 0) flux_x[q] = qf; else flux_y[q - nfx] = qf;
}

// transport_mobile3, heights: compensated f32 sum per column (delta3d_mobile.rs:770-781).
__global__ void k_transport_eta(Geo g, float transport, const float* __restrict__ flux_x,
                                const float* __restrict__ flux_y, float* __restrict__ eta, float* __restrict__ rof) {
  KSTART();
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= g.nx * g.ny) return;
  int i = c % g.nx, j = c / g.nx;
  float x = flux_x[j * (g.nx + 1) + i + 1] - flux_x[j * (g.nx + 1) + i];
  float y = flux_y[(j + 1) * g.nx + i] - flux_y[j * g.nx + i];
  float increment = -transport * (x + y) - rof[c];
  float height = eta[c] + increment;
  rof[c] = (height - eta[c]) - increment;
  eta[c] = height;
}

// mobile_in_bounds (delta3d_mobile.rs:801-813): sets *flag when a column leaves its bounds.
__global__ void k_in_bounds(Geo g, const float* __restrict__ floor, int* flag) {
  KSTART();
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  bool bad = false;
  if (c < g.nx * g.ny) {
    float top = (float)(g.nz - 1) * g.dx;
    float e = g.eta[c];
    float fl = g.cut ? floor[c] + 2.f * g.dx : 2.f * g.dx;
    bad = !(e >= fl && e <= top);
  }
  if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(flag, 1);
}

}  // namespace fd3
