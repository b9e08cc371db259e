// 2.5-D blocked fine-level kernels for the f64-reduction mode.
//
// Each CTA owns a 32 x 8 tile of columns and marches up a range of KZ layers.  The operand of the
// 7-point row is held for the layers below, at and above the current one in registers, and the
// current layer (with a one-cell halo in x and y) in shared memory, so each value is fetched from
// memory about once per pass instead of once per neighbour.  The per-cell arithmetic is that of
// the linear kernels (fd3_fast.cuh): same expressions, same order, bit-identical cell values.
// Only the order in which the f64 reduction partials are summed differs, which is why the ordered
// (bit-exact, reference-order) mode keeps the linear kernels, whose blocks are 64-cell chunks.
#pragma once

#include "fd3_fast.cuh"

namespace fd3 {

#ifndef FD3_ZK
#define FD3_ZK 8
#endif
#ifndef FD3_ZMINB
#define FD3_ZMINB 4
#endif
// Shared-memory planes of the march: with two, consecutive layers alternate and one barrier per
// layer suffices (a plane is rewritten only after every thread has passed the next layer's barrier).
#ifndef FD3_PLANES
#define FD3_PLANES 2
#endif
constexpr int ZX = 32, ZY = 8, ZK = FD3_ZK, ZT = ZX * ZY;

// apply_code with the six neighbour values given (only fluid-neighbour faces read them).
__device__ __forceinline__ float apply_code_nb(const Geo& g, unsigned code, int i, int j, int k, float pc,
                                               float xm, float xp, float ym, float yp, float zm, float zp) {
  float acc = 0.f;
  if (rc_plain(code)) {  // a = 1 on every live face, no ghost: the masked sum (see rc_plain)
    acc += (code & (1u << 1)) ? pc - xm : 0.f;
    acc += (code & (1u << 3)) ? pc - xp : 0.f;
    acc += (code & (1u << 5)) ? pc - ym : 0.f;
    acc += (code & (1u << 7)) ? pc - yp : 0.f;
    acc += (code & (1u << 9)) ? pc - zm : 0.f;
    acc += (code & (1u << 11)) ? pc - zp : 0.f;
    return acc * g.inv;
  }
  const bool unit = code & RC_UNIT;
  unsigned st = face_state(code, 0);
  if (st) {
    float a = unit ? 1.f : aper3(g, 0, fu(g, i, j, k));
    if (st == 1) acc += a * (pc - xm); else acc += a * pc * ghost_it_side(g, i, j, k, i - 1, j);
  }
  st = face_state(code, 1);
  if (st) {
    float a = unit ? 1.f : aper3(g, 0, fu(g, i + 1, j, k));
    if (st == 1) acc += a * (pc - xp); else acc += a * pc * ghost_it_side(g, i, j, k, i + 1, j);
  }
  st = face_state(code, 2);
  if (st) {
    float a = unit ? 1.f : aper3(g, 1, fv(g, i, j, k));
    if (st == 1) acc += a * (pc - ym); else acc += a * pc * ghost_it_side(g, i, j, k, i, j - 1);
  }
  st = face_state(code, 3);
  if (st) {
    float a = unit ? 1.f : aper3(g, 1, fv(g, i, j + 1, k));
    if (st == 1) acc += a * (pc - yp); else acc += a * pc * ghost_it_side(g, i, j, k, i, j + 1);
  }
  st = face_state(code, 4);
  if (st) {
    float a = unit ? 1.f : aper3(g, 2, fw(g, i, j, k));
    acc += a * (pc - zm);
  }
  st = face_state(code, 5);
  if (st) {
    float a = unit ? 1.f : aper3(g, 2, fw(g, i, j, k + 1));
    if (st == 1) acc += a * (pc - zp);
    else if (g.linear) acc += 2.f * a * pc;
    else acc += a * pc * ghost_it_up(g, i, j, k);
  }
  return acc * g.inv;
}

// Tile coordinates of a 1-D launch: blockIdx.x enumerates (tile x, tile y, k range).
struct ZTile {
  int i, j, k0, k1;
  bool inside;
};
__device__ __forceinline__ ZTile ztile(const Geo& g) {
  const int tx = threadIdx.x % ZX, ty = threadIdx.x / ZX;
  const int ntx = (g.nx + ZX - 1) / ZX, nty = (g.ny + ZY - 1) / ZY;
  int b = blockIdx.x;
  const int bx = b % ntx; b /= ntx;
  const int by = b % nty; b /= nty;
  ZTile t;
  t.i = bx * ZX + tx;
  t.j = by * ZY + ty;
  t.k0 = b * ZK;
  t.k1 = min(t.k0 + ZK, g.nz);
  t.inside = t.i < g.nx && t.j < g.ny;
  return t;
}
inline int zblocks(int nx, int ny, int nz) {
  return ((nx + ZX - 1) / ZX) * ((ny + ZY - 1) / ZY) * ((nz + ZK - 1) / ZK);
}

// The march, register-pipelined.  A loader L provides, for a cell (i, j, k, c):
//   L.full(i, j, k, c) -> Raw    every load the cell's own row and epilogue need (issued early)
//   L.halo(i, j, k, c) -> Halo   the loads a neighbour's operand value needs
//   L.pv(Raw), L.hv(Halo)        the operand value from those loads
// Loads for layer k+2 (own column) and for the halo of layer k+1 are issued during layer k, so
// each layer's arithmetic waits on loads started a whole layer earlier.  E(c, Raw, p, ax) consumes
// A.P at a cell (ax = 0 at a dry cell); A(k) runs after each layer's second barrier (all threads).
struct NoAfter {
  __device__ __forceinline__ void operator()(int) const {}
};

template <class L, class E, class A = NoAfter>
__device__ __forceinline__ void zmarch(const Geo& g, const unsigned short* __restrict__ codes, const L& ld, E epi,
                                       A after = A()) {
  typedef typename L::Raw Raw;
  typedef typename L::Halo Halo;
  __shared__ float sbuf[FD3_PLANES][ZY + 2][ZX + 2];
  const int tx = threadIdx.x % ZX, ty = threadIdx.x / ZX;
  const ZTile t = ztile(g);
  if (g.tiles && !g.tiles[(t.j / TILE_Y) * ((g.nx + TILE_X - 1) / TILE_X) + t.i / TILE_X]) return;  // no column of the set
  const int nxny = g.nx * g.ny;
  const int base = t.j * g.nx + t.i;
  // this thread's halo duty in x and in y (at most one each)
  const int hxi = tx == 0 ? t.i - 1 : (tx == ZX - 1 ? t.i + 1 : -1);
  const int hyj = ty == 0 ? t.j - 1 : (ty == ZY - 1 ? t.j + 1 : -1);
  const bool hx_on = hxi >= 0 && hxi < g.nx && t.j < g.ny;
  const bool hy_on = hyj >= 0 && hyj < g.ny && t.i < g.nx;
  const int hxs = tx == 0 ? 0 : ZX + 1;
  const int hys = ty == 0 ? 0 : ZY + 1;
  auto fetch_full = [&](int k) { return (t.inside && k < g.nz && k >= 0) ? ld.full(t.i, t.j, k, base + k * nxny) : Raw(); };
  auto fetch_hx = [&](int k) { return (hx_on && k < t.k1) ? ld.halo(hxi, t.j, k, t.j * g.nx + hxi + k * nxny) : Halo(); };
  auto fetch_hy = [&](int k) { return (hy_on && k < t.k1) ? ld.halo(t.i, hyj, k, hyj * g.nx + t.i + k * nxny) : Halo(); };
  auto fetch_code = [&](int k) { return (t.inside && k < t.k1) ? (unsigned)codes[base + k * nxny] : 0u; };

  float pprev = 0.f;
  if (t.k0 > 0) { Raw rp = fetch_full(t.k0 - 1); pprev = t.inside ? ld.pv(rp) : 0.f; }
  Raw rc = fetch_full(t.k0);
  Raw rn = fetch_full(t.k0 + 1);
  Halo hx = fetch_hx(t.k0), hy = fetch_hy(t.k0);
  unsigned code = fetch_code(t.k0);
  for (int k = t.k0; k < t.k1; ++k) {
    const int c = base + k * nxny;
    // issue the next layers' loads now
    Raw rnn = fetch_full(k + 2 <= t.k1 ? k + 2 : g.nz);
    Halo hx2 = fetch_hx(k + 1), hy2 = fetch_hy(k + 1);
    unsigned code2 = fetch_code(k + 1);
    const float pc = t.inside ? ld.pv(rc) : 0.f;
    const float pn = (t.inside && k + 1 < g.nz) ? ld.pv(rn) : 0.f;
    float (*s)[ZX + 2] = sbuf[(k - t.k0) % FD3_PLANES];
    s[ty + 1][tx + 1] = pc;
    if (hxi >= 0) s[ty + 1][hxs] = hx_on ? ld.hv(hx) : 0.f;
    if (hyj >= 0) s[hys][tx + 1] = hy_on ? ld.hv(hy) : 0.f;
    __syncthreads();
    if (t.inside) {
      float ax = 0.f;
      if (code & RC_WET)
        ax = apply_code_nb(g, code, t.i, t.j, k, pc, s[ty + 1][tx], s[ty + 1][tx + 2], s[ty][tx + 1], s[ty + 2][tx + 1],
                           pprev, pn);
      epi(c, rc, pc, ax);
    }
    if (FD3_PLANES == 1) __syncthreads();  // with two planes, the next layer's barrier orders the reuse
    after(k);
    pprev = pc;
    rc = rn;
    rn = rnn;
    hx = hx2;
    hy = hy2;
    code = code2;
  }
}

// The same march for full tiles (nx % ZX == 0, ny % ZY == 0, nz % ZK == 0): every thread owns a
// cell in every layer, so the per-cell bounds tests go, and the ZK-layer loop is unrolled so the
// register window rotates for free.  Halo threads on the domain boundary still read nothing.
template <class L, class E, class A = NoAfter>
__device__ __forceinline__ void zmarch_full(const Geo& g, const unsigned short* __restrict__ codes, const L& ld, E epi,
                                            A after = A()) {
  typedef typename L::Raw Raw;
  typedef typename L::Halo Halo;
  __shared__ float sbuf[FD3_PLANES][ZY + 2][ZX + 2];
  const int tx = threadIdx.x % ZX, ty = threadIdx.x / ZX;
  const ZTile t = ztile(g);
  if (g.tiles && !g.tiles[(t.j / TILE_Y) * ((g.nx + TILE_X - 1) / TILE_X) + t.i / TILE_X]) return;  // no column of the set
  const int nxny = g.nx * g.ny;
  const int base = t.j * g.nx + t.i;
  const int hxi = tx == 0 ? t.i - 1 : (tx == ZX - 1 ? t.i + 1 : -1);
  const int hyj = ty == 0 ? t.j - 1 : (ty == ZY - 1 ? t.j + 1 : -1);
  const bool hx_on = hxi >= 0 && hxi < g.nx;
  const bool hy_on = hyj >= 0 && hyj < g.ny;
  const int hx_off = hxi - t.i;          // -1 or +1 (when hx_on)
  const int hy_off = (hyj - t.j) * g.nx;  // -nx or +nx (when hy_on)
  const int hxs = tx == 0 ? 0 : ZX + 1;
  const int hys = ty == 0 ? 0 : ZY + 1;
  const bool last_chunk = t.k0 + ZK >= g.nz;

  float pprev = 0.f;
  if (t.k0 > 0) pprev = ld.pv(ld.full(t.i, t.j, t.k0 - 1, base + (t.k0 - 1) * nxny));
  Raw rc = ld.full(t.i, t.j, t.k0, base + t.k0 * nxny);
  Raw rn = ld.full(t.i, t.j, t.k0 + 1, base + (t.k0 + 1) * nxny);  // ZK >= 2 and nz % ZK == 0
  Halo hx = hx_on ? ld.halo(hxi, t.j, t.k0, base + hx_off + t.k0 * nxny) : Halo();
  Halo hy = hy_on ? ld.halo(t.i, hyj, t.k0, base + hy_off + t.k0 * nxny) : Halo();
  unsigned code = codes[base + t.k0 * nxny];
#pragma unroll
  for (int kk = 0; kk < ZK; ++kk) {
    const int k = t.k0 + kk;
    const int c = base + k * nxny;
    Raw rnn;
    if (kk + 2 < ZK || (!last_chunk && kk + 2 == ZK)) rnn = ld.full(t.i, t.j, k + 2, c + 2 * nxny);
    Halo hx2, hy2;
    unsigned code2 = 0;
    if (kk + 1 < ZK) {
      if (hx_on) hx2 = ld.halo(hxi, t.j, k + 1, c + nxny + hx_off);
      if (hy_on) hy2 = ld.halo(t.i, hyj, k + 1, c + nxny + hy_off);
      code2 = codes[c + nxny];
    }
    const float pc = ld.pv(rc);
    const float pn = (kk + 1 < ZK || !last_chunk) ? ld.pv(rn) : 0.f;
    float (*s)[ZX + 2] = sbuf[kk % FD3_PLANES];
    s[ty + 1][tx + 1] = pc;
    if (hxi >= 0) s[ty + 1][hxs] = hx_on ? ld.hv(hx) : 0.f;
    if (hyj >= 0) s[hys][tx + 1] = hy_on ? ld.hv(hy) : 0.f;
    __syncthreads();
    float ax = 0.f;
    if (code & RC_WET)
      ax = apply_code_nb(g, code, t.i, t.j, k, pc, s[ty + 1][tx], s[ty + 1][tx + 2], s[ty][tx + 1], s[ty + 2][tx + 1],
                         pprev, pn);
    epi(c, rc, pc, ax);
    if (FD3_PLANES == 1) __syncthreads();
    after(k);
    pprev = pc;
    rc = rn;
    rn = rnn;
    hx = hx2;
    hy = hy2;
    code = code2;
  }
}

inline bool zfull(int nx, int ny, int nz) { return nx % ZX == 0 && ny % ZY == 0 && nz % ZK == 0; }

// Full tiles or not, chosen by the kernel's FULL template parameter.
#define ZMARCH(...)                      \
  do {                                   \
    if (FULL) zmarch_full(__VA_ARGS__);  \
    else zmarch(__VA_ARGS__);            \
  } while (0)

// Loaders.
struct LdLoad {  // operand = x
  const float* __restrict__ x;
  struct Raw { float v = 0.f; };
  typedef Raw Halo;
  __device__ __forceinline__ Raw full(int, int, int, int c) const { Raw r; r.v = x[c]; return r; }
  __device__ __forceinline__ Halo halo(int, int, int, int c) const { Halo h; h.v = x[c]; return h; }
  __device__ __forceinline__ float pv(const Raw& r) const { return r.v; }
  __device__ __forceinline__ float hv(const Halo& h) const { return h.v; }
};
struct LdLoadR {  // operand = x, with r carried for the epilogue
  const float* __restrict__ x;
  const float* __restrict__ r;
  struct Raw { float v = 0.f, r = 0.f; };
  struct Halo { float v = 0.f; };
  __device__ __forceinline__ Raw full(int, int, int, int c) const { Raw o; o.v = x[c]; o.r = r[c]; return o; }
  __device__ __forceinline__ Halo halo(int, int, int, int c) const { Halo h; h.v = x[c]; return h; }
  __device__ __forceinline__ float pv(const Raw& o) const { return o.v; }
  __device__ __forceinline__ float hv(const Halo& h) const { return h.v; }
};
struct LdDir {  // d = z (+ beta d)
  const float* __restrict__ z;
  const float* __restrict__ din;
  int mode;
  float beta;
  struct Raw { float z = 0.f, d = 0.f; };
  typedef Raw Halo;
  __device__ __forceinline__ Raw full(int, int, int, int c) const { Raw o; o.z = z[c]; o.d = mode ? din[c] : 0.f; return o; }
  __device__ __forceinline__ Halo halo(int i, int j, int k, int c) const { return full(i, j, k, c); }
  __device__ __forceinline__ float pv(const Raw& o) const { return mode ? o.z + beta * o.d : o.z; }
  __device__ __forceinline__ float hv(const Halo& o) const { return pv(o); }
};
struct LdZ1 {  // first pre-sweep from zero: w prec r where prec > 0
  const float* __restrict__ prec;
  const float* __restrict__ r;
  struct Raw { float m = 0.f, r = 0.f; };
  typedef Raw Halo;
  __device__ __forceinline__ Raw full(int, int, int, int c) const { Raw o; o.m = prec[c]; o.r = r[c]; return o; }
  __device__ __forceinline__ Halo halo(int i, int j, int k, int c) const { return full(i, j, k, c); }
  __device__ __forceinline__ float pv(const Raw& o) const { return o.m > 0.f ? 0.f + OMEGA * o.m * (o.r - 0.f) : 0.f; }
  __device__ __forceinline__ float hv(const Halo& o) const { return pv(o); }
};
struct LdProlong {  // z + parent x, zeroed where prec == 0 (or z alone without prolongation)
  const float* __restrict__ zin;
  const float* __restrict__ prec;
  const float* __restrict__ r;
  const float* __restrict__ xc;
  int lnx, lny, prolong;
  struct Raw { float z = 0.f, m = 0.f, x = 0.f, r = 0.f; };
  struct Halo { float z = 0.f, m = 0.f, x = 0.f; };
  __device__ __forceinline__ float parent(int i, int j, int k) const {
    return prolong ? xc[((k >> 1) * lny + (j >> 1)) * lnx + (i >> 1)] : 0.f;
  }
  __device__ __forceinline__ Raw full(int i, int j, int k, int c) const {
    Raw o; o.z = zin[c]; o.m = prec[c]; o.r = r[c]; o.x = parent(i, j, k); return o;
  }
  __device__ __forceinline__ Halo halo(int i, int j, int k, int c) const {
    Halo h; h.z = zin[c]; h.m = prolong ? prec[c] : 0.f; h.x = parent(i, j, k); return h;
  }
  __device__ __forceinline__ float val(float z, float m, float x) const {
    if (!prolong) return z;
    float v = z + x;
    return m == 0.f ? 0.f : v;
  }
  __device__ __forceinline__ float pv(const Raw& o) const { return val(o.z, o.m, o.x); }
  __device__ __forceinline__ float hv(const Halo& h) const { return val(h.z, h.m, h.x); }
};
struct LdSweep {  // z, with prec and r carried for the epilogue
  const float* __restrict__ zin;
  const float* __restrict__ prec;
  const float* __restrict__ r;
  struct Raw { float z = 0.f, m = 0.f, r = 0.f; };
  struct Halo { float z = 0.f; };
  __device__ __forceinline__ Raw full(int, int, int, int c) const { Raw o; o.z = zin[c]; o.m = prec[c]; o.r = r[c]; return o; }
  __device__ __forceinline__ Halo halo(int, int, int, int c) const { Halo h; h.z = zin[c]; return h; }
  __device__ __forceinline__ float pv(const Raw& o) const { return o.z; }
  __device__ __forceinline__ float hv(const Halo& h) const { return h.z; }
};

// Reduction of one f64 value per thread, finished by the last block (the same as reduce_finish in
// f64 mode, with every thread's value valid).
__device__ __forceinline__ void zreduce_finish(double v, Red red, Scalars* S, int op) {
  reduce_finish<RED_F64>(v, 0, 1, red, S, op);
}

// d = z (+ beta d); q = A d; d.q; alpha (FIN_DQ).
template <bool FULL>
__global__ void __launch_bounds__(ZT, FD3_ZMINB) kz_dir_apply_dot(Geo g, const unsigned short* __restrict__ codes,
                                                       const float* __restrict__ z, const float* __restrict__ din,
                                                       float* __restrict__ dout, float* __restrict__ q, Red red,
                                                       Scalars* S) {
  KSTART();
  if (!S->active) return;
  LdDir ld{z, din, S->dir_mode, S->beta};
  double acc = 0.0;
  ZMARCH(g, codes, ld, [&](int c, const LdDir::Raw&, float pc, float ax) {
    dout[c] = pc;
    q[c] = ax;
    acc += (double)pc * (double)ax;
  });
  zreduce_finish(acc, red, S, FIN_DQ);
}

// The two pre-sweeps from z = 0.
template <bool FULL>
__global__ void __launch_bounds__(ZT, FD3_ZMINB) kz_fine_pre(Geo g, const unsigned short* __restrict__ codes,
                                                  const float* __restrict__ prec, const float* __restrict__ r,
                                                  float* __restrict__ z2, const Scalars* S, int gate) {
  KSTART();
  if (gate && !S->active) return;
  LdZ1 ld{prec, r};
  ZMARCH(g, codes, ld, [&](int c, const LdZ1::Raw& o, float pc, float ax) {
    float zc = pc;
    if (o.m > 0.f) zc += OMEGA * o.m * (o.r - ax);
    z2[c] = zc;
  });
}

// Prolongation + zeroing + first post-sweep (or the plain third sweep without coarse levels).
template <bool FULL>
__global__ void __launch_bounds__(ZT, FD3_ZMINB) kz_fine_post1(Geo g, const unsigned short* __restrict__ codes,
                                                    const float* __restrict__ prec, const float* __restrict__ r,
                                                    const float* __restrict__ zin, Lev L, int prolong,
                                                    float* __restrict__ zout, const Scalars* S, int gate) {
  KSTART();
  if (gate && !S->active) return;
  LdProlong ld{zin, prec, r, L.x, L.nx, L.ny, prolong};
  ZMARCH(g, codes, ld, [&](int c, const LdProlong::Raw& o, float pc, float ax) {
    float zc = pc;
    if (o.m > 0.f) zc += OMEGA * o.m * (o.r - ax);
    zout[c] = zc;
  });
}

// Second post-sweep with r.z (FIN_RZ_PRIME or FIN_RZ_ITER).
template <bool FULL>
__global__ void __launch_bounds__(ZT, FD3_ZMINB) kz_fine_post2_rz(Geo g, const unsigned short* __restrict__ codes,
                                                       const float* __restrict__ prec, const float* __restrict__ r,
                                                       const float* __restrict__ zin, float* __restrict__ zout, Red red,
                                                       Scalars* S, int gate, int op) {
  KSTART();
  if (gate && !S->active) return;
  LdSweep ld{zin, prec, r};
  double acc = 0.0;
  ZMARCH(g, codes, ld, [&](int c, const LdSweep::Raw& o, float pc, float ax) {
    float zc = pc;
    if (o.m > 0.f) zc += OMEGA * o.m * (o.r - ax);
    zout[c] = zc;
    acc += (double)o.r * (double)zc;
  });
  zreduce_finish(acc, red, S, op);
}

// Residual r - A z at every fine cell and its 8-child mean (restrict3, delta3d_multigrid.rs:258-272),
// two layers at a time: the even thread of each 2 x 2 column group sums its coarse cell's eight
// children in the reference's CHILDREN order from the two layers kept in shared memory.  Needs even
// nx, ny, nz (the coarsening rule guarantees them) and even ZX, ZY, ZK.
template <bool FULL>
__global__ void __launch_bounds__(ZT, FD3_ZMINB) kz_fine_restrict(Geo g, const unsigned short* __restrict__ codes,
                                                       const float* __restrict__ r, const float* __restrict__ z, Lev L,
                                                       const Scalars* S, int gate) {
  KSTART();
  if (gate && !S->active) return;
  __shared__ float tr[2][ZY][ZX];
  const int tx = threadIdx.x % ZX, ty = threadIdx.x / ZX;
  const ZTile t = ztile(g);
  const int nxny = g.nx * g.ny;
  LdLoadR ld{z, r};
  ZMARCH(
      g, codes, ld,
      [&](int c, const LdLoadR::Raw& o, float, float ax) { tr[(c / nxny) & 1][ty][tx] = o.r - ax; },
      [&](int k) {
        if (FD3_PLANES > 1 && (k & 1)) __syncthreads();  // the epilogue's tr writes before the reads below
        if ((k & 1) && t.inside && !(tx & 1) && !(ty & 1)) {
          float sum = 0.f;
          sum += tr[0][ty][tx];
          sum += tr[0][ty][tx + 1];
          sum += tr[0][ty + 1][tx];
          sum += tr[0][ty + 1][tx + 1];
          sum += tr[1][ty][tx];
          sum += tr[1][ty][tx + 1];
          sum += tr[1][ty + 1][tx];
          sum += tr[1][ty + 1][tx + 1];
          L.r[((k >> 1) * L.ny + (t.j >> 1)) * L.nx + (t.i >> 1)] = 0.125f * sum;
        }
      });
}

// p += alpha d, r -= alpha q, r.r (FIN_RN): four cells per thread with 16-byte loads, grid-stride.
constexpr int UPDATE_BLOCKS = 592;
// `act` (the sparse set, with nx % 4 == 0; else null): four cells of one row whose columns are all
// outside the set are skipped (p, r, d, q are 0 there and stay 0).
__global__ void __launch_bounds__(TPB) kv_update_rn(int n, float* __restrict__ p, float* __restrict__ r,
                                                    const float* __restrict__ d, const float* __restrict__ q, Red red,
                                                    Scalars* S, const unsigned char* __restrict__ act, int ncol) {
  KSTART();
  if (!S->active) return;
  const float alpha = S->alpha;
  const int stride = gridDim.x * blockDim.x;
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  double acc = 0.0;
  bool nz = false;
  const int n4 = n / 4;
  float4* p4 = reinterpret_cast<float4*>(p);
  float4* r4 = reinterpret_cast<float4*>(r);
  const float4* d4 = reinterpret_cast<const float4*>(d);
  const float4* q4 = reinterpret_cast<const float4*>(q);
  for (int v = tid; v < n4; v += stride) {
    if (act && *reinterpret_cast<const unsigned*>(act + (4 * v) % ncol) == 0u) continue;
    float4 P = p4[v], R = r4[v];
    const float4 D = d4[v], Q = q4[v];
    P.x += alpha * D.x; P.y += alpha * D.y; P.z += alpha * D.z; P.w += alpha * D.w;
    R.x = R.x - alpha * Q.x; R.y = R.y - alpha * Q.y; R.z = R.z - alpha * Q.z; R.w = R.w - alpha * Q.w;
    p4[v] = P;
    r4[v] = R;
    acc += (double)R.x * (double)R.x;
    acc += (double)R.y * (double)R.y;
    acc += (double)R.z * (double)R.z;
    acc += (double)R.w * (double)R.w;
    nz = nz || R.x != 0.f || R.y != 0.f || R.z != 0.f || R.w != 0.f;
  }
  for (int c = n4 * 4 + tid; c < n; c += stride) {
    p[c] += alpha * d[c];
    float rn = r[c] - alpha * q[c];
    r[c] = rn;
    acc += (double)rn * (double)rn;
    nz = nz || rn != 0.f;
  }
  if (__syncthreads_or(nz) && threadIdx.x == 0) atomicOr(&S->any_nonzero, 1);
  zreduce_finish(acc, red, S, FIN_RN);
}

}  // namespace fd3
