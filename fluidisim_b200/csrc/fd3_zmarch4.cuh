// The 2.5-D blocked fine-level kernels with four cells per thread along x (f32 storage).
//
// Each CTA owns a (4 QX) x (256 / QX) tile of columns: a row of the tile is QX lanes, each lane a
// quad of adjacent cells i0 = x0 + 4 lane .. i0 + 3, loaded and stored as 16-byte vectors (the four
// row codes in one 8-byte load).  The CTA marches up K4 layers.  Against the paired march
// (fd3_zmarch2.cuh) the per-thread work of a layer is spread over four cells instead of two, and:
//   - the x neighbours come from the neighbouring lanes by warp shuffles (only the first and the
//     last lane of a row load a halo cell), so shared memory holds one float4 per lane and row;
//   - the operand of the next layer is computed once and carried into the current one;
//   - a quad whose four rows are all interior (every face open onto a fluid neighbour with
//     aperture 1, the bulk of a domain) sums its six differences without decoding the codes.
// The per-cell arithmetic is that of the other kernel families (apply_code_nb, the same
// expressions in the same order): bit-identical cell values; only the order in which the f64
// reduction partials are summed differs.  Needs nx % 4 == 0.
#pragma once

#include "fd3_zmarch2.cuh"

namespace fd3 {

// Resident CTAs per SM the register budget is cut for: 2 (up to 128 registers) for the passes that
// carry three raw operand arrays per layer, 3 (up to 85) for the lighter direction and restriction
// passes, which fit without spilling and gain from the occupancy (measured at 256^3).
#ifndef FD3_ZMINB4
#define FD3_ZMINB4 2
#endif
#ifndef FD3_ZMINB4_LIGHT
#define FD3_ZMINB4_LIGHT 3
#endif
constexpr int Z4T = 256;

template <int QX>
inline int zblocks4(int nx, int ny, int nz, int k4) {
  constexpr int TX = 4 * QX, TY = Z4T / QX;
  return ((nx + TX - 1) / TX) * ((ny + TY - 1) / TY) * ((nz + k4 - 1) / k4);
}

struct ZTile4 {
  int i0, j, k0, k1, x0, y0;
  bool inside;
};
template <int QX, int K4>
__device__ __forceinline__ ZTile4 ztile4(const Geo& g) {
  constexpr int TX = 4 * QX, TY = Z4T / QX;
  const int tx = threadIdx.x % QX, ty = threadIdx.x / QX;
  const int ntx = (g.nx + TX - 1) / TX, nty = (g.ny + TY - 1) / TY;
  int b = blockIdx.x;
  const int bx = b % ntx; b /= ntx;
  const int by = b % nty; b /= nty;
  ZTile4 t;
  t.x0 = bx * TX;
  t.y0 = by * TY;
  t.i0 = t.x0 + 4 * tx;
  t.j = t.y0 + ty;
  t.k0 = b * K4;
  t.k1 = min(t.k0 + K4, g.nz);
  t.inside = t.i0 < g.nx && t.j < g.ny;  // nx % 4 == 0: i0 + 3 < nx too
  return t;
}

__device__ __forceinline__ float4 zero4() { return make_float4(0.f, 0.f, 0.f, 0.f); }
__device__ __forceinline__ float4 ld4(const float* __restrict__ p, int c) {
  return *reinterpret_cast<const float4*>(p + c);
}
__device__ __forceinline__ void st4(float* __restrict__ p, int c, float4 v) { *reinterpret_cast<float4*>(p + c) = v; }

// The code of an interior row, twice (the two codes of one 32-bit word of the quad's codes).
constexpr unsigned RC_INTERIOR2 = RC_INTERIOR | (RC_INTERIOR << 16);

// The interior row: the six differences in the reference's face order, the sum starting at +0
// (so a sum of zeros has the sign apply_code_nb gives it).
__device__ __forceinline__ float interior_row(float pc, float xm, float xp, float ym, float yp, float zm, float zp,
                                              float inv) {
  float acc = 0.f;
  acc += pc - xm;
  acc += pc - xp;
  acc += pc - ym;
  acc += pc - yp;
  acc += pc - zm;
  acc += pc - zp;
  return acc * inv;
}

// A.P at the quad's four cells (0 at a dry cell).
__device__ __forceinline__ float4 quad_apply(const Geo& g, uint2 code, int i0, int j, int k, float4 pc, float xl,
                                             float xr, float4 ym, float4 yp, float4 zm, float4 zp) {
  float4 a;
  if (code.x == RC_INTERIOR2 && code.y == RC_INTERIOR2) {
    a.x = interior_row(pc.x, xl, pc.y, ym.x, yp.x, zm.x, zp.x, g.inv);
    a.y = interior_row(pc.y, pc.x, pc.z, ym.y, yp.y, zm.y, zp.y, g.inv);
    a.z = interior_row(pc.z, pc.y, pc.w, ym.z, yp.z, zm.z, zp.z, g.inv);
    a.w = interior_row(pc.w, pc.z, xr, ym.w, yp.w, zm.w, zp.w, g.inv);
    return a;
  }
  const unsigned c0 = code.x & 0xffffu, c1 = code.x >> 16, c2 = code.y & 0xffffu, c3 = code.y >> 16;
  a.x = (c0 & RC_WET) ? apply_code_nb(g, c0, i0, j, k, pc.x, xl, pc.y, ym.x, yp.x, zm.x, zp.x) : 0.f;
  a.y = (c1 & RC_WET) ? apply_code_nb(g, c1, i0 + 1, j, k, pc.y, pc.x, pc.z, ym.y, yp.y, zm.y, zp.y) : 0.f;
  a.z = (c2 & RC_WET) ? apply_code_nb(g, c2, i0 + 2, j, k, pc.z, pc.y, pc.w, ym.z, yp.z, zm.z, zp.z) : 0.f;
  a.w = (c3 & RC_WET) ? apply_code_nb(g, c3, i0 + 3, j, k, pc.w, pc.z, xr, ym.w, yp.w, zm.w, zp.w) : 0.f;
  return a;
}

// The march.  A loader L provides, for the quad at (i0, j, k), c = its first cell:
//   L.full4(i0, j, k, c) -> Raw4   every load the quad's rows and epilogue need
//   L.pv4(Raw4) -> float4          the quad's operand values
//   L.halo4 / L.hv4                the operand of a quad in a neighbouring row (y halo)
//   L.halo / L.hv                  the operand of one cell (x halo)
// E(c, Raw4, pc, a) consumes a = A.P at the quad (0 at a dry cell); A(k) runs after each layer
// (all threads).
template <int QX, int K4, class L, class E, class A = NoAfter>
__device__ __forceinline__ void zmarch4(const Geo& g, const unsigned short* __restrict__ codes, const L& ld, E epi,
                                        A after = A()) {
  typedef typename L::Raw4 Raw4;
  typedef typename L::Halo Halo;
  typedef typename L::Halo4 Halo4;
  constexpr int TX = 4 * QX, TY = Z4T / QX;
  __shared__ __align__(16) float4 sbuf[2][TY + 2][QX];
  const int tx = threadIdx.x % QX, ty = threadIdx.x / QX;
  const ZTile4 t = ztile4<QX, K4>(g);
  if (g.tiles) {  // the tile's 32 x 8 tile flags of the sparse set: skip a tile with no column of the set
    const int ntx = (g.nx + TILE_X - 1) / TILE_X, nty = (g.ny + TILE_Y - 1) / TILE_Y;
    const int ax = t.x0 / TILE_X, bx = min(ntx, (t.x0 + TX + TILE_X - 1) / TILE_X);
    const int ay = t.y0 / TILE_Y, by = min(nty, (t.y0 + TY + TILE_Y - 1) / TILE_Y);
    bool any = false;
    for (int y = ay; y < by; ++y)
      for (int x = ax; x < bx; ++x) any |= g.tiles[y * ntx + x] != 0;
    if (!any) return;
  }
  const int nxny = g.nx * g.ny;
  const int base = t.j * g.nx + t.i0;
  // x halo: lane 0 of a row the cell left of the tile, lane QX-1 the cell right of it
  const int hxi = tx == 0 ? t.x0 - 1 : (tx == QX - 1 ? t.x0 + TX : -1);
  const bool hx_on = hxi >= 0 && hxi < g.nx && t.j < g.ny;
  // y halo: row 0 the quads below the tile, row TY - 1 the quads above
  const int hyj = ty == 0 ? t.y0 - 1 : (ty == TY - 1 ? t.y0 + TY : -1);
  const bool hy_on = hyj >= 0 && hyj < g.ny && t.i0 < g.nx;
  const int hys = ty == 0 ? 0 : TY + 1;
  auto fetch_full = [&](int k) {
    return (t.inside && k < g.nz && k >= 0) ? ld.full4(t.i0, t.j, k, base + k * nxny) : Raw4();
  };
  auto fetch_hx = [&](int k) { return (hx_on && k < t.k1) ? ld.halo(hxi, t.j, k, t.j * g.nx + hxi + k * nxny) : Halo(); };
  auto fetch_hy = [&](int k) {
    return (hy_on && k < t.k1) ? ld.halo4(t.i0, hyj, k, hyj * g.nx + t.i0 + k * nxny) : Halo4();
  };
  auto fetch_code = [&](int k) {
    return (t.inside && k < t.k1) ? *reinterpret_cast<const uint2*>(codes + base + k * nxny) : make_uint2(0u, 0u);
  };

  float4 pprev = zero4();
  if (t.k0 > 0 && t.inside) pprev = ld.pv4(fetch_full(t.k0 - 1));
  Raw4 rc = fetch_full(t.k0);
  float4 pc = t.inside ? ld.pv4(rc) : zero4();
  Raw4 rn = fetch_full(t.k0 + 1);
  Halo hx = fetch_hx(t.k0);
  Halo4 hy = fetch_hy(t.k0);
  uint2 code = fetch_code(t.k0);
  for (int k = t.k0; k < t.k1; ++k) {
    const int c = base + k * nxny;
    Raw4 rnn = fetch_full(k + 2 <= t.k1 ? k + 2 : g.nz);
    Halo hx2 = fetch_hx(k + 1);
    Halo4 hy2 = fetch_hy(k + 1);
    const uint2 code2 = fetch_code(k + 1);
    const float4 pn = (t.inside && k + 1 < g.nz) ? ld.pv4(rn) : zero4();
    float4(*s)[QX] = sbuf[(k - t.k0) & 1];
    s[ty + 1][tx] = pc;
    if (ty == 0 || ty == TY - 1) s[hys][tx] = hy_on ? ld.hv4(hy) : zero4();
    float xl = __shfl_up_sync(0xffffffffu, pc.w, 1, QX);
    float xr = __shfl_down_sync(0xffffffffu, pc.x, 1, QX);
    if (tx == 0) xl = hx_on ? ld.hv(hx) : 0.f;
    if (tx == QX - 1) xr = hx_on ? ld.hv(hx) : 0.f;
    __syncthreads();
    if (t.inside) {
      const float4 ym = s[ty][tx], yp = s[ty + 2][tx];
      const float4 a = quad_apply(g, code, t.i0, t.j, k, pc, xl, xr, ym, yp, pprev, pn);
      epi(c, rc, pc, a);
    }
    after(k);
    pprev = pc;
    pc = pn;
    rc = rn;
    rn = rnn;
    hx = hx2;
    hy = hy2;
    code = code2;
  }
}

// Loaders (f32 storage).
struct Q4Dir {  // d = z (+ beta d)
  const float* __restrict__ z;
  const float* __restrict__ din;
  int mode;
  float beta;
  struct Raw4 { float4 z = zero4(), d = zero4(); };
  typedef Raw4 Halo4;
  struct Halo { float z = 0.f, d = 0.f; };
  __device__ __forceinline__ Raw4 full4(int, int, int, int c) const {
    Raw4 o; o.z = ld4(z, c); if (mode) o.d = ld4(din, c); return o;
  }
  __device__ __forceinline__ Halo4 halo4(int i, int j, int k, int c) const { return full4(i, j, k, c); }
  __device__ __forceinline__ Halo halo(int, int, int, int c) const { Halo h; h.z = z[c]; if (mode) h.d = din[c]; return h; }
  __device__ __forceinline__ float v(float zz, float dd) const { return mode ? zz + beta * dd : zz; }
  __device__ __forceinline__ float4 pv4(const Raw4& o) const {
    return make_float4(v(o.z.x, o.d.x), v(o.z.y, o.d.y), v(o.z.z, o.d.z), v(o.z.w, o.d.w));
  }
  __device__ __forceinline__ float4 hv4(const Halo4& o) const { return pv4(o); }
  __device__ __forceinline__ float hv(const Halo& h) const { return v(h.z, h.d); }
};
struct Q4Z1 {  // first pre-sweep from zero: w prec r where prec > 0
  const float* __restrict__ prec;
  const float* __restrict__ r;
  struct Raw4 { float4 m = zero4(), r = zero4(); };
  typedef Raw4 Halo4;
  struct Halo { float m = 0.f, r = 0.f; };
  __device__ __forceinline__ Raw4 full4(int, int, int, int c) const { Raw4 o; o.m = ld4(prec, c); o.r = ld4(r, c); return o; }
  __device__ __forceinline__ Halo4 halo4(int i, int j, int k, int c) const { return full4(i, j, k, c); }
  __device__ __forceinline__ Halo halo(int, int, int, int c) const { Halo h; h.m = prec[c]; h.r = r[c]; return h; }
  __device__ __forceinline__ float v(float m, float rr) const { return m > 0.f ? 0.f + OMEGA * m * (rr - 0.f) : 0.f; }
  __device__ __forceinline__ float4 pv4(const Raw4& o) const {
    return make_float4(v(o.m.x, o.r.x), v(o.m.y, o.r.y), v(o.m.z, o.r.z), v(o.m.w, o.r.w));
  }
  __device__ __forceinline__ float4 hv4(const Halo4& o) const { return pv4(o); }
  __device__ __forceinline__ float hv(const Halo& h) const { return v(h.m, h.r); }
};
struct Q4Prolong {  // z + parent x, zeroed where prec == 0 (or z alone without prolongation)
  const float* __restrict__ zin;
  const float* __restrict__ prec;
  const float* __restrict__ r;
  const float* __restrict__ xc;
  int lnx, lny, prolong;
  struct Raw4 { float4 z = zero4(), m = zero4(), r = zero4(); float2 x = make_float2(0.f, 0.f); };
  struct Halo4 { float4 z = zero4(), m = zero4(); float2 x = make_float2(0.f, 0.f); };
  struct Halo { float z = 0.f, m = 0.f, x = 0.f; };
  // the quad's two parents (i0 / 2 is even, so the pair is one aligned 8-byte load)
  __device__ __forceinline__ float2 parents(int i0, int j, int k) const {
    return prolong ? ld2(xc, ((k >> 1) * lny + (j >> 1)) * lnx + (i0 >> 1)) : make_float2(0.f, 0.f);
  }
  __device__ __forceinline__ Raw4 full4(int i, int j, int k, int c) const {
    Raw4 o; o.z = ld4(zin, c); o.m = ld4(prec, c); o.r = ld4(r, c); o.x = parents(i, j, k); return o;
  }
  __device__ __forceinline__ Halo4 halo4(int i, int j, int k, int c) const {
    Halo4 h; h.z = ld4(zin, c); if (prolong) h.m = ld4(prec, c); h.x = parents(i, j, k); return h;
  }
  __device__ __forceinline__ Halo halo(int i, int j, int k, int c) const {
    Halo h; h.z = zin[c];
    if (prolong) { h.m = prec[c]; h.x = xc[((k >> 1) * lny + (j >> 1)) * lnx + (i >> 1)]; }
    return h;
  }
  __device__ __forceinline__ float val(float z, float m, float x) const {
    if (!prolong) return z;
    float v = z + x;
    return m == 0.f ? 0.f : v;
  }
  __device__ __forceinline__ float4 pv4(const Raw4& o) const {
    return make_float4(val(o.z.x, o.m.x, o.x.x), val(o.z.y, o.m.y, o.x.x), val(o.z.z, o.m.z, o.x.y),
                       val(o.z.w, o.m.w, o.x.y));
  }
  __device__ __forceinline__ float4 hv4(const Halo4& h) const {
    return make_float4(val(h.z.x, h.m.x, h.x.x), val(h.z.y, h.m.y, h.x.x), val(h.z.z, h.m.z, h.x.y),
                       val(h.z.w, h.m.w, h.x.y));
  }
  __device__ __forceinline__ float hv(const Halo& h) const { return val(h.z, h.m, h.x); }
};
struct Q4Sweep {  // z, with prec and r carried for the epilogue
  const float* __restrict__ zin;
  const float* __restrict__ prec;
  const float* __restrict__ r;
  struct Raw4 { float4 z = zero4(), m = zero4(), r = zero4(); };
  struct Halo4 { float4 z = zero4(); };
  struct Halo { float z = 0.f; };
  __device__ __forceinline__ Raw4 full4(int, int, int, int c) const {
    Raw4 o; o.z = ld4(zin, c); o.m = ld4(prec, c); o.r = ld4(r, c); return o;
  }
  __device__ __forceinline__ Halo4 halo4(int, int, int, int c) const { Halo4 h; h.z = ld4(zin, c); return h; }
  __device__ __forceinline__ Halo halo(int, int, int, int c) const { Halo h; h.z = zin[c]; return h; }
  __device__ __forceinline__ float4 pv4(const Raw4& o) const { return o.z; }
  __device__ __forceinline__ float4 hv4(const Halo4& h) const { return h.z; }
  __device__ __forceinline__ float hv(const Halo& h) const { return h.z; }
};
struct Q4LoadR {  // operand x, with r carried for the epilogue
  const float* __restrict__ x;
  const float* __restrict__ r;
  struct Raw4 { float4 v = zero4(), r = zero4(); };
  struct Halo4 { float4 v = zero4(); };
  struct Halo { float v = 0.f; };
  __device__ __forceinline__ Raw4 full4(int, int, int, int c) const { Raw4 o; o.v = ld4(x, c); o.r = ld4(r, c); return o; }
  __device__ __forceinline__ Halo4 halo4(int, int, int, int c) const { Halo4 h; h.v = ld4(x, c); return h; }
  __device__ __forceinline__ Halo halo(int, int, int, int c) const { Halo h; h.v = x[c]; return h; }
  __device__ __forceinline__ float4 pv4(const Raw4& o) const { return o.v; }
  __device__ __forceinline__ float4 hv4(const Halo4& h) const { return h.v; }
  __device__ __forceinline__ float hv(const Halo& h) const { return h.v; }
};

// One damped-Jacobi update of a cell (smooth3 on the fine level): z + w prec (r - A z) where prec > 0.
__device__ __forceinline__ float jac(float z, float m, float r, float a) {
  if (m > 0.f) z += OMEGA * m * (r - a);
  return z;
}
__device__ __forceinline__ float4 jac4(float4 z, float4 m, float4 r, float4 a) {
  return make_float4(jac(z.x, m.x, r.x, a.x), jac(z.y, m.y, r.y, a.y), jac(z.z, m.z, r.z, a.z), jac(z.w, m.w, r.w, a.w));
}
__device__ __forceinline__ double dot4(float4 a, float4 b) {
  double s = (double)a.x * (double)b.x;
  s += (double)a.y * (double)b.y;
  s += (double)a.z * (double)b.z;
  s += (double)a.w * (double)b.w;
  return s;
}

// res = rhs - A p with res.res (FIN_RR0 or FIN_ACTUAL).
template <int QX, int K4>
__global__ void __launch_bounds__(Z4T, FD3_ZMINB4) kq_residual(Geo g, const unsigned short* __restrict__ codes,
                                                             const float* __restrict__ p, const float* __restrict__ rhs,
                                                             float* __restrict__ res, Red red, Scalars* S, int op) {
  KSTART();
  Q4LoadR ld{p, rhs};
  double acc = 0.0;
  zmarch4<QX, K4>(g, codes, ld, [&](int c, const Q4LoadR::Raw4& o, float4, float4 a) {
    const float4 rr = make_float4(o.r.x - a.x, o.r.y - a.y, o.r.z - a.z, o.r.w - a.w);
    st4(res, c, rr);
    acc += dot4(rr, rr);
  });
  zreduce_finish(acc, red, S, op);
}

// d = z (+ beta d); q = A d; d.q; alpha (FIN_DQ).
template <int QX, int K4>
__global__ void __launch_bounds__(Z4T, FD3_ZMINB4_LIGHT) kq_dir_apply_dot(Geo g, const unsigned short* __restrict__ codes,
                                                                  const float* __restrict__ z,
                                                                  const float* __restrict__ din, float* __restrict__ dout,
                                                                  float* __restrict__ q, Red red, Scalars* S) {
  KSTART();
  if (!S->active) return;
  Q4Dir ld{z, din, S->dir_mode, S->beta};
  double acc = 0.0;
  zmarch4<QX, K4>(g, codes, ld, [&](int c, const Q4Dir::Raw4&, float4 pc, float4 a) {
    st4(dout, c, pc);
    st4(q, c, a);
    acc += dot4(pc, a);
  });
  zreduce_finish(acc, red, S, FIN_DQ);
}

// The two pre-sweeps from z = 0.
template <int QX, int K4>
__global__ void __launch_bounds__(Z4T, FD3_ZMINB4) kq_fine_pre(Geo g, const unsigned short* __restrict__ codes,
                                                             const float* __restrict__ prec, const float* __restrict__ r,
                                                             float* __restrict__ z2, const Scalars* S, int gate) {
  KSTART();
  if (gate && !S->active) return;
  Q4Z1 ld{prec, r};
  zmarch4<QX, K4>(g, codes, ld, [&](int c, const Q4Z1::Raw4& o, float4 pc, float4 a) {
    st4(z2, c, jac4(pc, o.m, o.r, a));
  });
}

// Prolongation + zeroing + first post-sweep (or the plain third sweep without coarse levels).
template <int QX, int K4>
__global__ void __launch_bounds__(Z4T, FD3_ZMINB4) kq_fine_post1(Geo g, const unsigned short* __restrict__ codes,
                                                               const float* __restrict__ prec, const float* __restrict__ r,
                                                               const float* __restrict__ zin, Lev L, int prolong,
                                                               float* __restrict__ zout, const Scalars* S, int gate) {
  KSTART();
  if (gate && !S->active) return;
  Q4Prolong ld{zin, prec, r, L.x, L.nx, L.ny, prolong};
  zmarch4<QX, K4>(g, codes, ld, [&](int c, const Q4Prolong::Raw4& o, float4 pc, float4 a) {
    st4(zout, c, jac4(pc, o.m, o.r, a));
  });
}

// Second post-sweep with r.z (FIN_RZ_PRIME or FIN_RZ_ITER).
template <int QX, int K4>
__global__ void __launch_bounds__(Z4T, FD3_ZMINB4) kq_fine_post2_rz(Geo g, const unsigned short* __restrict__ codes,
                                                                  const float* __restrict__ prec,
                                                                  const float* __restrict__ r,
                                                                  const float* __restrict__ zin, float* __restrict__ zout,
                                                                  Red red, Scalars* S, int gate, int op) {
  KSTART();
  if (gate && !S->active) return;
  Q4Sweep ld{zin, prec, r};
  double acc = 0.0;
  zmarch4<QX, K4>(g, codes, ld, [&](int c, const Q4Sweep::Raw4& o, float4 pc, float4 a) {
    const float4 z = jac4(pc, o.m, o.r, a);
    st4(zout, c, z);
    acc += dot4(o.r, z);
  });
  zreduce_finish(acc, red, S, op);
}

// Residual r - A z at every fine cell and its 8-child mean (restrict3, delta3d_multigrid.rs:258-272):
// each lane's quad holds the x children of two coarse cells; after every odd layer the even rows
// sum each coarse cell's eight children, in the reference's CHILDREN order, from the two layers
// kept in shared memory.  Needs even ny, nz (the coarsening rule guarantees them) and even K4.
template <int QX, int K4>
__global__ void __launch_bounds__(Z4T, FD3_ZMINB4_LIGHT) kq_fine_restrict(Geo g, const unsigned short* __restrict__ codes,
                                                                  const float* __restrict__ r,
                                                                  const float* __restrict__ z, Lev L, const Scalars* S,
                                                                  int gate) {
  KSTART();
  if (gate && !S->active) return;
  constexpr int TY = Z4T / QX;
  __shared__ __align__(16) float4 tr[2][TY][QX];
  const int tx = threadIdx.x % QX, ty = threadIdx.x / QX;
  const ZTile4 t = ztile4<QX, K4>(g);
  const int nxny = g.nx * g.ny;
  Q4LoadR ld{z, r};
  zmarch4<QX, K4>(
      g, codes, ld,
      [&](int c, const Q4LoadR::Raw4& o, float4, float4 a) {
        tr[(c / nxny) & 1][ty][tx] = make_float4(o.r.x - a.x, o.r.y - a.y, o.r.z - a.z, o.r.w - a.w);
      },
      [&](int k) {
        if (k & 1) {
          __syncthreads();  // the epilogue's tr writes before the reads below
          if (t.inside && !(ty & 1)) {
            const float4 a0 = tr[0][ty][tx], b0 = tr[0][ty + 1][tx], a1 = tr[1][ty][tx], b1 = tr[1][ty + 1][tx];
            float s0 = 0.f, s1 = 0.f;
            s0 += a0.x; s0 += a0.y; s0 += b0.x; s0 += b0.y; s0 += a1.x; s0 += a1.y; s0 += b1.x; s0 += b1.y;
            s1 += a0.z; s1 += a0.w; s1 += b0.z; s1 += b0.w; s1 += a1.z; s1 += a1.w; s1 += b1.z; s1 += b1.w;
            st2(L.r, ((k >> 1) * L.ny + (t.j >> 1)) * L.nx + (t.i0 >> 1), 0.125f * s0, 0.125f * s1);
          }
        }
      });
}

}  // namespace fd3
