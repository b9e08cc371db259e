// The 2.5-D blocked fine-level kernels with two cells per thread along x.
//
// Each CTA owns a 64 x 8 tile of columns (32 threads per row, each thread a pair of adjacent
// cells i0 = 2 * lane, i0 + 1) and marches up K2 layers.  Against one cell per thread (the march of
// fd3_zmarch.cuh) this halves the per-cell cost of everything that is per thread rather than per
// cell: the tile's index arithmetic and bounds tests, the halo duties, the barrier, the register
// pipeline of the layer loop, and the loads, which become 8-byte vector loads (two row codes in one
// 32-bit load).  The operand of the 7-point row lives in shared memory for the current layer (row
// layout: [pad][x halo][64 cells][x halo][pad], the cells at an even offset so pairs are float2),
// and in registers for the layers below and above.
//
// The per-cell arithmetic is that of the other kernel families (apply_code_nb with the same
// neighbour values): the same expressions in the same order, bit-identical cell values; only the
// order in which the f64 reduction partials are summed differs.  Needs nx even (the multigrid's
// coarsening rule guarantees it for every volume that uses these kernels).
#pragma once

#include "fd3_zmarch.cuh"

namespace fd3 {

// Resident CTAs per SM the register budget is cut for: 3 (up to 85 registers, no spills) for the
// sweeps, 4 (64) for the lighter direction and restriction passes; measured at 128^3 on one box:
// 349.4 projections/s, against 345.7 with 3 for every pass; 3 for every pass against 4 for every
// pass (the sweeps spilling), 344.6 against 342.1 on another.
#ifndef FD3_ZMINB2
#define FD3_ZMINB2 3
#endif
#ifndef FD3_ZMINB2_LIGHT
#define FD3_ZMINB2_LIGHT 4
#endif
// Layers per CTA (K2) is a template parameter: 8 when the grid still yields two waves of CTAs at
// four per SM (measured best at 256^3), else 4 (best at 128^3, where 8 leaves SMs idle).
constexpr int Z2X = 64, Z2Y = 8, Z2T = 256, Z2ROW = Z2X + 4;

inline int zblocks2(int nx, int ny, int nz, int k2) {
  return ((nx + Z2X - 1) / Z2X) * ((ny + Z2Y - 1) / Z2Y) * ((nz + k2 - 1) / k2);
}
inline int pick_k2(int nx, int ny, int nz) { return zblocks2(nx, ny, nz, 8) >= 2 * 4 * 148 ? 8 : 4; }

struct ZTile2 {
  int i0, j, k0, k1, x0;
  bool inside;
};
template <int K2>
__device__ __forceinline__ ZTile2 ztile2(const Geo& g) {
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  const int ntx = (g.nx + Z2X - 1) / Z2X, nty = (g.ny + Z2Y - 1) / Z2Y;
  int b = blockIdx.x;
  const int bx = b % ntx; b /= ntx;
  const int by = b % nty; b /= nty;
  ZTile2 t;
  t.x0 = bx * Z2X;
  t.i0 = t.x0 + 2 * tx;
  t.j = by * Z2Y + ty;
  t.k0 = b * K2;
  t.k1 = min(t.k0 + K2, g.nz);
  t.inside = t.i0 < g.nx && t.j < g.ny;  // nx even: i0 + 1 < nx too
  return t;
}

__device__ __forceinline__ float2 ld2(const float* __restrict__ p, int c) {
  return *reinterpret_cast<const float2*>(p + c);
}
__device__ __forceinline__ void st2(float* __restrict__ p, int c, float a, float b) {
  *reinterpret_cast<float2*>(p + c) = make_float2(a, b);
}

// The march.  A loader L provides, for the pair at (i0, j, k), c = its first cell:
//   L.full2(i0, j, k, c) -> Raw2   every load the pair's rows and epilogue need
//   L.pv2(Raw2) -> float2         the pair's operand values
//   L.halo2(i0, j, k, c) -> Halo2 / L.hv2: the operand of a pair in a neighbouring row (y halo)
//   L.halo(i, j, k, c) -> Halo / L.hv: the operand of one cell (x halo)
// E(c, Raw2, pc, ax0, ax1) consumes A.P at the pair (ax = 0 at a dry cell); A(k) runs after each
// layer (all threads).
template <int K2, class L, class E, class A = NoAfter>
__device__ __forceinline__ void zmarch2(const Geo& g, const unsigned short* __restrict__ codes, const L& ld, E epi,
                                        A after = A()) {
  typedef typename L::Raw2 Raw2;
  typedef typename L::Halo Halo;
  typedef typename L::Halo2 Halo2;
  __shared__ __align__(16) float sbuf[2][Z2Y + 2][Z2ROW];
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  const ZTile2 t = ztile2<K2>(g);
  if (g.tiles) {  // a 64 x 8 tile is two 32 x 8 tiles of the set's tile flags
    const int ntx = (g.nx + TILE_X - 1) / TILE_X, row = (t.j / TILE_Y) * ntx, a = t.x0 / TILE_X;
    if (!g.tiles[row + a] && (a + 1 >= ntx || !g.tiles[row + a + 1])) return;  // no column of the set
  }
  const int nxny = g.nx * g.ny;
  const int base = t.j * g.nx + t.i0;
  // x halo: lane 0 the cell left of the tile, lane 31 the cell right of it
  const int hxi = tx == 0 ? t.x0 - 1 : (tx == 31 ? t.x0 + Z2X : -1);
  const bool hx_on = hxi >= 0 && hxi < g.nx && t.j < g.ny;
  const int hxs = tx == 0 ? 1 : Z2X + 2;
  // y halo: row 0 the pairs below the tile, row 7 the pairs above
  const int hyj = ty == 0 ? t.j - 1 : (ty == Z2Y - 1 ? t.j + 1 : -1);
  const bool hy_on = hyj >= 0 && hyj < g.ny && t.i0 < g.nx;
  const int hys = ty == 0 ? 0 : Z2Y + 1;
  auto fetch_full = [&](int k) { return (t.inside && k < g.nz && k >= 0) ? ld.full2(t.i0, t.j, k, base + k * nxny) : Raw2(); };
  auto fetch_hx = [&](int k) { return (hx_on && k < t.k1) ? ld.halo(hxi, t.j, k, t.j * g.nx + hxi + k * nxny) : Halo(); };
  auto fetch_hy = [&](int k) { return (hy_on && k < t.k1) ? ld.halo2(t.i0, hyj, k, hyj * g.nx + t.i0 + k * nxny) : Halo2(); };
  auto fetch_code = [&](int k) {
    return (t.inside && k < t.k1) ? *reinterpret_cast<const unsigned*>(codes + base + k * nxny) : 0u;
  };

  float2 pprev = make_float2(0.f, 0.f);
  if (t.k0 > 0 && t.inside) pprev = ld.pv2(fetch_full(t.k0 - 1));
  Raw2 rc = fetch_full(t.k0);
  Raw2 rn = fetch_full(t.k0 + 1);
  Halo hx = fetch_hx(t.k0);
  Halo2 hy = fetch_hy(t.k0);
  unsigned code = fetch_code(t.k0);
  for (int k = t.k0; k < t.k1; ++k) {
    const int c = base + k * nxny;
    Raw2 rnn = fetch_full(k + 2 <= t.k1 ? k + 2 : g.nz);
    Halo hx2 = fetch_hx(k + 1);
    Halo2 hy2 = fetch_hy(k + 1);
    const unsigned code2 = fetch_code(k + 1);
    const float2 pc = t.inside ? ld.pv2(rc) : make_float2(0.f, 0.f);
    const float2 pn = (t.inside && k + 1 < g.nz) ? ld.pv2(rn) : make_float2(0.f, 0.f);
    float (*s)[Z2ROW] = sbuf[(k - t.k0) & 1];
    *reinterpret_cast<float2*>(&s[ty + 1][2 + 2 * tx]) = pc;
    if (hxi >= 0 || tx == 0 || tx == 31) s[ty + 1][hxs] = hx_on ? ld.hv(hx) : 0.f;
    if (hyj >= 0 || ty == 0 || ty == Z2Y - 1)
      *reinterpret_cast<float2*>(&s[hys][2 + 2 * tx]) = hy_on ? ld.hv2(hy) : make_float2(0.f, 0.f);
    __syncthreads();
    if (t.inside) {
      const unsigned c0 = code & 0xffffu, c1 = code >> 16;
      const float xm0 = s[ty + 1][1 + 2 * tx], xp1 = s[ty + 1][4 + 2 * tx];
      const float2 ym = *reinterpret_cast<const float2*>(&s[ty][2 + 2 * tx]);
      const float2 yp = *reinterpret_cast<const float2*>(&s[ty + 2][2 + 2 * tx]);
      float ax0 = 0.f, ax1 = 0.f;
      if (c0 & RC_WET) ax0 = apply_code_nb(g, c0, t.i0, t.j, k, pc.x, xm0, pc.y, ym.x, yp.x, pprev.x, pn.x);
      if (c1 & RC_WET) ax1 = apply_code_nb(g, c1, t.i0 + 1, t.j, k, pc.y, pc.x, xp1, ym.y, yp.y, pprev.y, pn.y);
      epi(c, rc, pc, ax0, ax1);
    }
    after(k);
    pprev = pc;
    rc = rn;
    rn = rnn;
    hx = hx2;
    hy = hy2;
    code = code2;
  }
}

// Loaders.  T is the storage of the V-cycle vectors (z, z2, the coarse x): f32, or FP16 in the
// mixed-precision mode, where the V-cycle also sees r scaled by rs (Scalars::vinv).
template <class T>
struct L2Dir {  // d = z (+ beta d)
  const T* __restrict__ z;
  const float* __restrict__ din;
  int mode;
  float beta;
  struct Raw2 { float2 z = make_float2(0.f, 0.f), d = make_float2(0.f, 0.f); };
  typedef Raw2 Halo2;
  struct Halo { float z = 0.f, d = 0.f; };
  __device__ __forceinline__ Raw2 full2(int, int, int, int c) const {
    Raw2 o; o.z = Store<T>::ld2(z, c); if (mode) o.d = ld2(din, c); return o;
  }
  __device__ __forceinline__ Halo2 halo2(int i, int j, int k, int c) const { return full2(i, j, k, c); }
  __device__ __forceinline__ Halo halo(int, int, int, int c) const {
    Halo h; h.z = Store<T>::ld(z, c); if (mode) h.d = din[c]; return h;
  }
  __device__ __forceinline__ float v(float zz, float dd) const { return mode ? zz + beta * dd : zz; }
  __device__ __forceinline__ float2 pv2(const Raw2& o) const { return make_float2(v(o.z.x, o.d.x), v(o.z.y, o.d.y)); }
  __device__ __forceinline__ float2 hv2(const Halo2& o) const { return pv2(o); }
  __device__ __forceinline__ float hv(const Halo& h) const { return v(h.z, h.d); }
};
// r as the V-cycle sees it: r * rs in the FP16 mode, r itself (no multiply) in f32.
template <class T>
__device__ __forceinline__ float rsc(float r, float rs) { return Store<T>::half ? r * rs : r; }
template <class T>
struct L2Z1 {  // first pre-sweep from zero: w prec r where prec > 0
  const float* __restrict__ prec;
  const float* __restrict__ r;
  float rs;
  struct Raw2 { float2 m = make_float2(0.f, 0.f), r = make_float2(0.f, 0.f); };
  typedef Raw2 Halo2;
  struct Halo { float m = 0.f, r = 0.f; };
  __device__ __forceinline__ Raw2 full2(int, int, int, int c) const { Raw2 o; o.m = ld2(prec, c); o.r = ld2(r, c); return o; }
  __device__ __forceinline__ Halo2 halo2(int i, int j, int k, int c) const { return full2(i, j, k, c); }
  __device__ __forceinline__ Halo halo(int, int, int, int c) const { Halo h; h.m = prec[c]; h.r = r[c]; return h; }
  __device__ __forceinline__ float v(float m, float rr) const {
    return m > 0.f ? 0.f + OMEGA * m * (rsc<T>(rr, rs) - 0.f) : 0.f;
  }
  __device__ __forceinline__ float2 pv2(const Raw2& o) const { return make_float2(v(o.m.x, o.r.x), v(o.m.y, o.r.y)); }
  __device__ __forceinline__ float2 hv2(const Halo2& o) const { return pv2(o); }
  __device__ __forceinline__ float hv(const Halo& h) const { return v(h.m, h.r); }
};
template <class T>
struct L2Prolong {  // z + parent x, zeroed where prec == 0 (or z alone without prolongation)
  const T* __restrict__ zin;
  const float* __restrict__ prec;
  const float* __restrict__ r;
  const T* __restrict__ xc;
  int lnx, lny, prolong;
  struct Raw2 { float2 z = make_float2(0.f, 0.f), m = make_float2(0.f, 0.f), r = make_float2(0.f, 0.f); float x = 0.f; };
  struct Halo2 { float2 z = make_float2(0.f, 0.f), m = make_float2(0.f, 0.f); float x = 0.f; };
  struct Halo { float z = 0.f, m = 0.f, x = 0.f; };
  __device__ __forceinline__ float parent(int i, int j, int k) const {  // the pair (even i0, i0 + 1) shares it
    return prolong ? Store<T>::ld(xc, ((k >> 1) * lny + (j >> 1)) * lnx + (i >> 1)) : 0.f;
  }
  __device__ __forceinline__ Raw2 full2(int i, int j, int k, int c) const {
    Raw2 o; o.z = Store<T>::ld2(zin, c); o.m = ld2(prec, c); o.r = ld2(r, c); o.x = parent(i, j, k); return o;
  }
  __device__ __forceinline__ Halo2 halo2(int i, int j, int k, int c) const {
    Halo2 h; h.z = Store<T>::ld2(zin, c); if (prolong) h.m = ld2(prec, c); h.x = parent(i, j, k); return h;
  }
  __device__ __forceinline__ Halo halo(int i, int j, int k, int c) const {
    Halo h; h.z = Store<T>::ld(zin, c); h.m = prolong ? prec[c] : 0.f; h.x = parent(i, j, k); return h;
  }
  __device__ __forceinline__ float val(float z, float m, float x) const {
    if (!prolong) return z;
    float v = z + x;
    return m == 0.f ? 0.f : v;
  }
  __device__ __forceinline__ float2 pv2(const Raw2& o) const { return make_float2(val(o.z.x, o.m.x, o.x), val(o.z.y, o.m.y, o.x)); }
  __device__ __forceinline__ float2 hv2(const Halo2& h) const { return make_float2(val(h.z.x, h.m.x, h.x), val(h.z.y, h.m.y, h.x)); }
  __device__ __forceinline__ float hv(const Halo& h) const { return val(h.z, h.m, h.x); }
};
template <class T>
struct L2Sweep {  // z, with prec and r carried for the epilogue
  const T* __restrict__ zin;
  const float* __restrict__ prec;
  const float* __restrict__ r;
  struct Raw2 { float2 z = make_float2(0.f, 0.f), m = make_float2(0.f, 0.f), r = make_float2(0.f, 0.f); };
  struct Halo2 { float2 z = make_float2(0.f, 0.f); };
  struct Halo { float z = 0.f; };
  __device__ __forceinline__ Raw2 full2(int, int, int, int c) const {
    Raw2 o; o.z = Store<T>::ld2(zin, c); o.m = ld2(prec, c); o.r = ld2(r, c); return o;
  }
  __device__ __forceinline__ Halo2 halo2(int, int, int, int c) const { Halo2 h; h.z = Store<T>::ld2(zin, c); return h; }
  __device__ __forceinline__ Halo halo(int, int, int, int c) const { Halo h; h.z = Store<T>::ld(zin, c); return h; }
  __device__ __forceinline__ float2 pv2(const Raw2& o) const { return o.z; }
  __device__ __forceinline__ float2 hv2(const Halo2& h) const { return h.z; }
  __device__ __forceinline__ float hv(const Halo& h) const { return h.z; }
};
template <class T>
struct L2LoadR {  // operand x, with r carried for the epilogue
  const T* __restrict__ x;
  const float* __restrict__ r;
  struct Raw2 { float2 v = make_float2(0.f, 0.f), r = make_float2(0.f, 0.f); };
  struct Halo2 { float2 v = make_float2(0.f, 0.f); };
  struct Halo { float v = 0.f; };
  __device__ __forceinline__ Raw2 full2(int, int, int, int c) const { Raw2 o; o.v = Store<T>::ld2(x, c); o.r = ld2(r, c); return o; }
  __device__ __forceinline__ Halo2 halo2(int, int, int, int c) const { Halo2 h; h.v = Store<T>::ld2(x, c); return h; }
  __device__ __forceinline__ Halo halo(int, int, int, int c) const { Halo h; h.v = Store<T>::ld(x, c); return h; }
  __device__ __forceinline__ float2 pv2(const Raw2& o) const { return o.v; }
  __device__ __forceinline__ float2 hv2(const Halo2& h) const { return h.v; }
  __device__ __forceinline__ float hv(const Halo& h) const { return h.v; }
};

// res = rhs - A p with res.res (FIN_RR0 or FIN_ACTUAL): k_residual_c on the paired march.
template <int K2>
__global__ void __launch_bounds__(Z2T, FD3_ZMINB2) kx_residual(Geo g, const unsigned short* __restrict__ codes,
                                                             const float* __restrict__ p, const float* __restrict__ rhs,
                                                             float* __restrict__ res, Red red, Scalars* S, int op) {
  KSTART();
  L2LoadR<float> ld{p, rhs};
  double acc = 0.0;
  zmarch2<K2>(g, codes, ld, [&](int c, const L2LoadR<float>::Raw2& o, float2, float a0, float a1) {
    const float r0 = o.r.x - a0, r1 = o.r.y - a1;
    st2(res, c, r0, r1);
    acc += (double)r0 * (double)r0;
    acc += (double)r1 * (double)r1;
  });
  zreduce_finish(acc, red, S, op);
}

// d = z (+ beta d); q = A d; d.q; alpha (FIN_DQ).
template <int K2, class T>
__global__ void __launch_bounds__(Z2T, FD3_ZMINB2_LIGHT) kx_dir_apply_dot(Geo g, const unsigned short* __restrict__ codes,
                                                                  const T* __restrict__ z,
                                                                  const float* __restrict__ din, float* __restrict__ dout,
                                                                  float* __restrict__ q, Red red, Scalars* S) {
  KSTART();
  if (!S->active) return;
  L2Dir<T> ld{z, din, S->dir_mode, S->beta};
  double acc = 0.0;
  zmarch2<K2>(g, codes, ld, [&](int c, const typename L2Dir<T>::Raw2&, float2 pc, float a0, float a1) {
    st2(dout, c, pc.x, pc.y);
    st2(q, c, a0, a1);
    acc += (double)pc.x * (double)a0;
    acc += (double)pc.y * (double)a1;
  });
  zreduce_finish(acc, red, S, FIN_DQ);
}

// The two pre-sweeps from z = 0.
template <int K2, class T>
__global__ void __launch_bounds__(Z2T, FD3_ZMINB2) kx_fine_pre(Geo g, const unsigned short* __restrict__ codes,
                                                             const float* __restrict__ prec, const float* __restrict__ r,
                                                             T* __restrict__ z2, const Scalars* S, int gate) {
  KSTART();
  if (gate && !S->active) return;
  const float rs = vscale<T>(S);
  L2Z1<T> ld{prec, r, rs};
  zmarch2<K2>(g, codes, ld, [&](int c, const typename L2Z1<T>::Raw2& o, float2 pc, float a0, float a1) {
    float z0 = pc.x, z1 = pc.y;
    if (o.m.x > 0.f) z0 += OMEGA * o.m.x * (rsc<T>(o.r.x, rs) - a0);
    if (o.m.y > 0.f) z1 += OMEGA * o.m.y * (rsc<T>(o.r.y, rs) - a1);
    Store<T>::st2(z2, c, z0, z1);
  });
}

// Prolongation + zeroing + first post-sweep (or the plain third sweep without coarse levels).
template <int K2, class T>
__global__ void __launch_bounds__(Z2T, FD3_ZMINB2) kx_fine_post1(Geo g, const unsigned short* __restrict__ codes,
                                                               const float* __restrict__ prec, const float* __restrict__ r,
                                                               const T* __restrict__ zin, Lev L, int prolong,
                                                               T* __restrict__ zout, const Scalars* S, int gate) {
  KSTART();
  if (gate && !S->active) return;
  const float rs = vscale<T>(S);
  L2Prolong<T> ld{zin, prec, r, as<T>(L.x), L.nx, L.ny, prolong};
  zmarch2<K2>(g, codes, ld, [&](int c, const typename L2Prolong<T>::Raw2& o, float2 pc, float a0, float a1) {
    float z0 = pc.x, z1 = pc.y;
    if (o.m.x > 0.f) z0 += OMEGA * o.m.x * (rsc<T>(o.r.x, rs) - a0);
    if (o.m.y > 0.f) z1 += OMEGA * o.m.y * (rsc<T>(o.r.y, rs) - a1);
    Store<T>::st2(zout, c, z0, z1);
  });
}

// Second post-sweep with r.z (FIN_RZ_PRIME or FIN_RZ_ITER).  The dot takes the z that is stored
// (the value the direction update reads back) and the unscaled r.
template <int K2, class T>
__global__ void __launch_bounds__(Z2T, FD3_ZMINB2) kx_fine_post2_rz(Geo g, const unsigned short* __restrict__ codes,
                                                                  const float* __restrict__ prec,
                                                                  const float* __restrict__ r,
                                                                  const T* __restrict__ zin, T* __restrict__ zout,
                                                                  Red red, Scalars* S, int gate, int op) {
  KSTART();
  if (gate && !S->active) return;
  const float rs = vscale<T>(S);
  L2Sweep<T> ld{zin, prec, r};
  double acc = 0.0;
  zmarch2<K2>(g, codes, ld, [&](int c, const typename L2Sweep<T>::Raw2& o, float2 pc, float a0, float a1) {
    float z0 = pc.x, z1 = pc.y;
    if (o.m.x > 0.f) z0 += OMEGA * o.m.x * (rsc<T>(o.r.x, rs) - a0);
    if (o.m.y > 0.f) z1 += OMEGA * o.m.y * (rsc<T>(o.r.y, rs) - a1);
    Store<T>::st2(zout, c, z0, z1);
    acc += (double)o.r.x * (double)Store<T>::rt(z0);
    acc += (double)o.r.y * (double)Store<T>::rt(z1);
  });
  zreduce_finish(acc, red, S, op);
}

// Residual r - A z at every fine cell and its 8-child mean (restrict3, delta3d_multigrid.rs:258-272):
// each thread's pair is one coarse cell's x children; the even rows sum the eight children, in the
// reference's CHILDREN order, from the two layers kept in shared memory.
template <int K2, class T>
__global__ void __launch_bounds__(Z2T, FD3_ZMINB2_LIGHT) kx_fine_restrict(Geo g, const unsigned short* __restrict__ codes,
                                                                  const float* __restrict__ r,
                                                                  const T* __restrict__ z, Lev L, const Scalars* S,
                                                                  int gate) {
  KSTART();
  if (gate && !S->active) return;
  __shared__ __align__(8) float tr[2][Z2Y][Z2X];
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  const ZTile2 t = ztile2<K2>(g);
  const int nxny = g.nx * g.ny;
  const float rs = vscale<T>(S);
  L2LoadR<T> ld{z, r};
  zmarch2<K2>(
      g, codes, ld,
      [&](int c, const typename L2LoadR<T>::Raw2& o, float2, float a0, float a1) {
        *reinterpret_cast<float2*>(&tr[(c / nxny) & 1][ty][2 * tx]) =
            make_float2(rsc<T>(o.r.x, rs) - a0, rsc<T>(o.r.y, rs) - a1);
      },
      [&](int k) {
        if (k & 1) {
          __syncthreads();  // the epilogue's tr writes before the reads below
          if (t.inside && !(ty & 1)) {
            float sum = 0.f;
            sum += tr[0][ty][2 * tx];
            sum += tr[0][ty][2 * tx + 1];
            sum += tr[0][ty + 1][2 * tx];
            sum += tr[0][ty + 1][2 * tx + 1];
            sum += tr[1][ty][2 * tx];
            sum += tr[1][ty][2 * tx + 1];
            sum += tr[1][ty + 1][2 * tx];
            sum += tr[1][ty + 1][2 * tx + 1];
            Store<T>::st(as<T>(L.r), ((k >> 1) * L.ny + (t.j >> 1)) * L.nx + (t.i0 >> 1), 0.125f * sum);
          }
        }
      });
}

}  // namespace fd3
