// The hot path of the MG-PCG iteration on sm_100a: fused passes over the fine level, fused coarse
// sweeps, a single-CTA solve of the small coarse levels, and reductions finished by the last block.
//
// Every fusion recomputes, at each stencil point, the value the unfused sequence would have
// stored (the same f32 expression in the same order), so a fused iteration is bit-identical to
// the reference's sequence of passes (delta3d_mobile.rs:515-545, delta3d_multigrid.rs:393-465).
#pragma once

#include "fd3_kernels.cuh"

namespace fd3 {

// ------------------------------------------------------------------------------------------------
// Row codes.  The mobile row (delta3d_mobile.rs:152-188) depends on the surface, which is frozen
// during a projection, so its structure is encoded once per projection in 16 bits:
//   bit 0        wet
//   bits 1+2f    face f (x-, x+, y-, y+, z-, z+): 0 nothing, 1 fluid neighbour, 2 surface ghost
//   bit 13       every live face has aperture 1 (no aperture load needed)
// A hot stencil then reads 2 bytes instead of rebuilding the row from the fractions, the
// apertures and six wet tests.  Apertures of cut faces and ghost coefficients are recomputed with
// the reference's own expressions, so an encoded row evaluates to the same bits.
constexpr unsigned RC_WET = 1u;
constexpr unsigned RC_UNIT = 1u << 13;

__device__ __forceinline__ unsigned face_state(unsigned code, int f) { return (code >> (1 + 2 * f)) & 3u; }

// The code of a wet cell's row.
__device__ __forceinline__ unsigned row_code_of(const RowE (&row)[6]) {
  unsigned code = RC_WET;
  bool unit = true;
#pragma unroll
  for (int f = 0; f < 6; ++f) {
    unsigned st = row[f].n >= 0 ? 1u : (row[f].a > 0.f ? 2u : 0u);
    code |= st << (1 + 2 * f);
    if (st && row[f].a != 1.f) unit = false;
  }
  if (unit) code |= RC_UNIT;
  return code;
}


// 1/max(theta, 1e-3) of ghost_side3 and ghost_up3 (delta3d_mobile.rs:126-147).
__device__ __forceinline__ float ghost_it_side(const Geo& g, int i, int j, int k, int x, int y) {
  float zc = ((float)k + 0.5f) * g.dx;
  float h = __ldg(g.eta + j * g.nx + i);
  float theta = fmaxf((h - zc) / (h - __ldg(g.eta + y * g.nx + x)), SURFACE_THETA_MIN);
  return 1.f / theta;
}
__device__ __forceinline__ float ghost_it_up(const Geo& g, int i, int j, int k) {
  float h = __ldg(g.eta + j * g.nx + i);
  float theta = fmaxf((h - ((float)k + 0.5f) * g.dx) / g.dx, SURFACE_THETA_MIN);
  return 1.f / theta;
}

// One row of apply_mobile3 from its code; P(n) yields the operand at cell n (a load, or a value
// recomputed on the fly by a fused kernel).
// The code of a wet cell whose six faces are open (aperture 1) onto fluid neighbours: the bulk.
constexpr unsigned RC_INTERIOR = RC_WET | RC_UNIT | (1u << 1) | (1u << 3) | (1u << 5) | (1u << 7) | (1u << 9) | (1u << 11);
// The high bit of every face state: set on a ghost (or, on a coarse level, Dirichlet) face.
constexpr unsigned RC_GHOSTS = (2u << 1) | (2u << 3) | (2u << 5) | (2u << 7) | (2u << 9) | (2u << 11);
// A row whose live faces all have aperture 1 and all lead to a fluid neighbour: the bulk, and also
// the cells along walls, closed faces and solids.  Its sum is the six differences masked by the
// face states: a = 1 makes a (pc - x) exactly pc - x, and a missing face adds +0, which changes no
// partial sum (the sum starts at +0 and a sum of such terms is never -0).  So the masked sum has
// the bits of the reference's sum over the live faces in the same order.
__device__ __forceinline__ bool rc_plain(unsigned code) { return (code & (RC_UNIT | RC_GHOSTS)) == RC_UNIT; }

template <class P>
__device__ __forceinline__ float apply_code(const Geo& g, unsigned code, int i, int j, int k, int c, P p) {
  const float pc = p(c);
  const bool unit = code & RC_UNIT;
  const int nxny = g.nx * g.ny;
  float acc = 0.f;
  if (rc_plain(code)) {  // a = 1 on every live face, no ghost: the masked sum, without the decoding
    acc += (code & (1u << 1)) ? pc - p(c - 1) : 0.f;
    acc += (code & (1u << 3)) ? pc - p(c + 1) : 0.f;
    acc += (code & (1u << 5)) ? pc - p(c - g.nx) : 0.f;
    acc += (code & (1u << 7)) ? pc - p(c + g.nx) : 0.f;
    acc += (code & (1u << 9)) ? pc - p(c - nxny) : 0.f;
    acc += (code & (1u << 11)) ? pc - p(c + nxny) : 0.f;
    return acc * g.inv;
  }
  unsigned st = face_state(code, 0);
  if (st) {
    float a = unit ? 1.f : aper3(g, 0, fu(g, i, j, k));
    if (st == 1) acc += a * (pc - p(c - 1)); else acc += a * pc * ghost_it_side(g, i, j, k, i - 1, j);
  }
  st = face_state(code, 1);
  if (st) {
    float a = unit ? 1.f : aper3(g, 0, fu(g, i + 1, j, k));
    if (st == 1) acc += a * (pc - p(c + 1)); else acc += a * pc * ghost_it_side(g, i, j, k, i + 1, j);
  }
  st = face_state(code, 2);
  if (st) {
    float a = unit ? 1.f : aper3(g, 1, fv(g, i, j, k));
    if (st == 1) acc += a * (pc - p(c - g.nx)); else acc += a * pc * ghost_it_side(g, i, j, k, i, j - 1);
  }
  st = face_state(code, 3);
  if (st) {
    float a = unit ? 1.f : aper3(g, 1, fv(g, i, j + 1, k));
    if (st == 1) acc += a * (pc - p(c + g.nx)); else acc += a * pc * ghost_it_side(g, i, j, k, i, j + 1);
  }
  st = face_state(code, 4);  // the face below is never a ghost
  if (st) {
    float a = unit ? 1.f : aper3(g, 2, fw(g, i, j, k));
    acc += a * (pc - p(c - nxny));
  }
  st = face_state(code, 5);
  if (st) {
    float a = unit ? 1.f : aper3(g, 2, fw(g, i, j, k + 1));
    if (st == 1) acc += a * (pc - p(c + nxny));
    else if (g.linear) acc += 2.f * a * pc;  // the lid of apply / apply_cut (delta3d.rs:741, 797)
    else acc += a * pc * ghost_it_up(g, i, j, k);
  }
  return acc * g.inv;
}

struct Load {
  const float* __restrict__ x;
  __device__ __forceinline__ float operator()(int n) const { return x[n]; }
};
template <class T>
struct LoadT {
  const T* __restrict__ x;
  __device__ __forceinline__ float operator()(int n) const { return Store<T>::ld(x, n); }
};

// ------------------------------------------------------------------------------------------------
// The outer loop's metrics from the projection's row codes (the surface is the one the codes were
// built for), instead of rebuilding each row from the geometry.

// One cell of divergence_mobile3 (delta3d_mobile.rs:398-433): |div u| of a wet row into the
// maximum over all wet rows and, without a surface ghost (no face state 2), over the plain ones;
// the cell's six face velocities (x-, x+, y-, y+, z-, z+) are given.
__device__ __forceinline__ void div_metric_vals(const Geo& g, unsigned code, int i, int j, int k, float ul, float ur,
                                                float vf, float vk, float wb, float wt, float& all, float& plain) {
  float dv;
  if (g.cut) {
    float fl = __ldg(g.ou + fu(g, i, j, k)) * ul;
    float fr = __ldg(g.ou + fu(g, i + 1, j, k)) * ur;
    float ff = __ldg(g.ov + fv(g, i, j, k)) * vf;
    float fk = __ldg(g.ov + fv(g, i, j + 1, k)) * vk;
    float fb = __ldg(g.ow + fw(g, i, j, k)) * wb;
    float ft = __ldg(g.ow + fw(g, i, j, k + 1)) * wt;
    dv = ((fr - fl + ft - fb) + (fk - ff)) / g.dx;
    if (g.wall) dv = dv + wall_flux(g, i, j, k);
  } else {
    dv = ((ur - ul + wt - wb) + (vk - vf)) / g.dx;
  }
  const float d = fabsf(dv);
  all = fmaxf(all, d);
  if (!(code & RC_GHOSTS)) plain = fmaxf(plain, d);
}
__device__ __forceinline__ void div_metric_cell(const Geo& g, unsigned code, const float* __restrict__ u,
                                                const float* __restrict__ v, const float* __restrict__ w, int c,
                                                float& all, float& plain) {
  if (!(code & RC_WET)) return;
  int i, j, k; cell_ijk(g, c, i, j, k);
  div_metric_vals(g, code, i, j, k, u[fu(g, i, j, k)], u[fu(g, i + 1, j, k)], v[fv(g, i, j, k)], v[fv(g, i, j + 1, k)],
                  w[fw(g, i, j, k)], w[fw(g, i, j, k + 1)], all, plain);
}

// correct_mobile3 (delta3d_mobile.rs:284-343) from the row codes.  A u or v face between cells l
// and r is corrected when r's row has it live (state 1: both wet, the gradient; state 2: l is air,
// r's ghost) or, r being dry, when l's row has it as a ghost (r is air, l's ghost).  Those are
// exactly the faces the reference corrects: open, neither cell solid, at least one wet.  A w face
// is corrected when the row of the cell below has it live.  Ghost coefficients and values are the
// reference's (ghost_side3, ghost_up3).
// The corrected value of the u (axis 0) or v (axis 1) face (i, j, k) whose staged value is `val`,
// given the codes and pressures of the cells on its + side (cr, pr) and - side (cl, pl), which only
// an interior face reads.
__device__ __forceinline__ float corrected_uv_vals(const Geo& g, float k1, float val, int axis, int i, int j, int k,
                                                  unsigned cr, unsigned cl, float pr, float pl) {
  const bool interior = axis == 0 ? (i > 0 && i < g.nx) : (j > 0 && j < g.ny);
  if (interior) {
    const int x = axis == 0 ? i - 1 : i, y = axis == 0 ? j : j - 1;
    const unsigned sr = face_state(cr, axis == 0 ? 0 : 2);  // r's face toward l
    if (sr == 1) {
      val -= k1 * (pr - pl) / g.dx;
    } else if (sr == 2) {
      float a, b; ghost_side3(g, i, j, k, x, y, a, b);
      val -= k1 * (pr - b) * a / g.dx;
    } else if (!(cr & RC_WET) && face_state(cl, axis == 0 ? 1 : 3) == 2) {  // l's face toward r
      float a, b; ghost_side3(g, x, y, k, i, j, a, b);
      val -= k1 * (b - pl) * a / g.dx;
    }
  }
  return val;
}
__device__ __forceinline__ float corrected_uv(const Geo& g, const unsigned short* __restrict__ codes, float k1,
                                             const float* __restrict__ p, float val, int axis, int i, int j, int k) {
  const bool interior = axis == 0 ? (i > 0 && i < g.nx) : (j > 0 && j < g.ny);
  if (!interior) return val;
  const int x = axis == 0 ? i - 1 : i, y = axis == 0 ? j : j - 1;
  const int l = (k * g.ny + y) * g.nx + x, r = (k * g.ny + j) * g.nx + i;
  return corrected_uv_vals(g, k1, val, axis, i, j, k, codes[r], codes[l], p[r], p[l]);
}
__device__ __forceinline__ void correct_uv_at(const Geo& g, const unsigned short* __restrict__ codes, float k1,
                                              const float* __restrict__ p, const float* __restrict__ us,
                                              const float* __restrict__ vs, float* __restrict__ u,
                                              float* __restrict__ v, int q) {
  const int nu = (g.nx + 1) * g.ny * g.nz, nv = g.nx * (g.ny + 1) * g.nz;
  int axis, f, i, j, k;
  if (q < nu) { axis = 0; f = q; i = f % (g.nx + 1); int t = f / (g.nx + 1); j = t % g.ny; k = t / g.ny; }
  else if (q < nu + nv) { axis = 1; f = q - nu; i = f % g.nx; int t = f / g.nx; j = t % (g.ny + 1); k = t / (g.ny + 1); }
  else return;
  const float val = corrected_uv(g, codes, k1, p, axis == 0 ? us[f] : vs[f], axis, i, j, k);
  if (axis == 0) u[f] = val; else v[f] = val;
}

// The corrected value of the w face (i, j, k) (k its layer) whose staged value is `val`, given the
// code and pressure of the cell below (cb, pb) and the pressure of the cell above (pa), which only
// a face with a cell below reads.
__device__ __forceinline__ float corrected_w_vals(const Geo& g, float k1, float val, int i, int j, int k, unsigned cb,
                                                 float pb, float pa) {
  if (k >= 1) {
    const unsigned st = face_state(cb, 5);  // the face above the cell below
    if (st == 1) {
      val -= k1 * (pa - pb) / g.dx;
    } else if (st == 2) {
      float a, b; ghost_up3(g, i, j, k - 1, a, b);
      val -= k1 * (b - pb) * a / g.dx;
    }
  }
  return val;
}
__device__ __forceinline__ float corrected_w(const Geo& g, const unsigned short* __restrict__ codes, float k1,
                                            const float* __restrict__ p, float val, int f, int i, int j, int k) {
  if (k < 1) return val;
  const int nxny = g.nx * g.ny;
  const int below = f - nxny;
  const unsigned cb = codes[below];
  // the cell above exists wherever the face below it is live (state 1)
  const float pa = face_state(cb, 5) == 1u ? p[below + nxny] : 0.f;
  return corrected_w_vals(g, k1, val, i, j, k, cb, p[below], pa);
}
__device__ __forceinline__ void correct_w_at(const Geo& g, const unsigned short* __restrict__ codes, float k1,
                                             const float* __restrict__ p, const float* __restrict__ ws,
                                             float* __restrict__ w, int f) {
  const int nw = g.nx * g.ny * (g.nz + 1);
  if (f >= nw) return;
  const int nxny = g.nx * g.ny;
  const int k = f / nxny, col = f % nxny, i = col % g.nx, j = col / g.nx;
  w[f] = corrected_w(g, codes, k1, p, ws[f], f, i, j, k);
}

// correct_mobile3, divergence_mobile3 and the largest |u| (delta3d_mobile.rs:284-343, 398-433) in
// one pass.  Cell c forms the corrected values of its six faces with the expressions of
// correct_uv_at and correct_w_at (a face shared by two cells gets the same value from both), stores
// the faces it owns (x-, y-, z-, and the + faces on the volume's upper edges, so every face is stored
// once), takes |div u| of its row from the six values, and the largest |value| of its own faces.
// Maxima into S->fmax[0] (all rows), [1] (plain rows), [2] (|u|), reset before, by one atomic each
// per block.
__device__ __forceinline__ void block_fmax3_atomic(float a, float b, float c, float* addr0, float* addr1,
                                                   float* addr2) {
  __shared__ float pa[32], pb[32], pc[32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    a = fmaxf(a, __shfl_down_sync(0xffffffffu, a, o));
    b = fmaxf(b, __shfl_down_sync(0xffffffffu, b, o));
    c = fmaxf(c, __shfl_down_sync(0xffffffffu, c, o));
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) { pa[wid] = a; pb[wid] = b; pc[wid] = c; }
  __syncthreads();
  if (wid == 0) {
    const bool on = lane < (int)(blockDim.x >> 5);
    a = on ? pa[lane] : 0.f;
    b = on ? pb[lane] : 0.f;
    c = on ? pc[lane] : 0.f;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      a = fmaxf(a, __shfl_down_sync(0xffffffffu, a, o));
      b = fmaxf(b, __shfl_down_sync(0xffffffffu, b, o));
      c = fmaxf(c, __shfl_down_sync(0xffffffffu, c, o));
    }
    if (lane == 0) {
      atomic_fmax_nonneg(addr0, a);
      atomic_fmax_nonneg(addr1, b);
      atomic_fmax_nonneg(addr2, c);
    }
  }
}
// Columns of 32 x 8 cells (a warp per row) marching CM_K layers: the indices advance by constant
// strides, the codes and pressures of the cells below and above ride in registers from layer to
// layer, and a cell's top w face is the next layer's bottom one, formed once and carried.
// Resident CTAs per SM for the assembly (k_rhs_b2) and the backward error pass: eight (32 registers,
// a few spilled) measured 17.48 -> 16.79 ms per 256^3 projection against the unbounded 48-50
// registers (six: 16.86), the same box.
#ifndef FD3_SETUP_MINB
#define FD3_SETUP_MINB 8
#endif
constexpr int CM_X = 32, CM_Y = 8, CM_K = 8;
inline int cm_blocks(int nx, int ny, int nz) {
  return ((nx + CM_X - 1) / CM_X) * ((ny + CM_Y - 1) / CM_Y) * ((nz + CM_K - 1) / CM_K);
}
// Five resident CTAs per SM (48 registers): 256^3 projection 17.00 ms against 17.92 with the 76
// registers the kernel takes unbounded (three CTAs per SM), the same box.
#ifndef FD3_CM_MINB
#define FD3_CM_MINB 5
#endif
__global__ void __launch_bounds__(CM_X * CM_Y, FD3_CM_MINB) k_correct_metric(Geo g, const unsigned short* __restrict__ codes,
                                                                float k1, const float* __restrict__ p,
                                                                const float* __restrict__ us,
                                                                const float* __restrict__ vs,
                                                                const float* __restrict__ ws, float* __restrict__ u,
                                                                float* __restrict__ v, float* __restrict__ w,
                                                                Scalars* S) {
  KSTART();
  float all = 0.f, plain = 0.f, mx = 0.f;
  const int ntx = (g.nx + CM_X - 1) / CM_X, nty = (g.ny + CM_Y - 1) / CM_Y;
  int b = blockIdx.x;
  const int bx = b % ntx; b /= ntx;
  const int by = b % nty; b /= nty;
  const int i = bx * CM_X + (int)(threadIdx.x & 31), j = by * CM_Y + (int)(threadIdx.x >> 5);
  const int k0 = b * CM_K, ke = min(k0 + CM_K, g.nz);
  if (i < g.nx && j < g.ny) {
    const int nxny = g.nx * g.ny, su = g.ny * (g.nx + 1), sv = (g.ny + 1) * g.nx;
    const bool xm = i > 0, xp = i + 1 < g.nx, ym = j > 0, yp = j + 1 < g.ny;
    int c = (k0 * g.ny + j) * g.nx + i;                 // the cell, and its w face below (fw)
    int ful = (k0 * g.ny + j) * (g.nx + 1) + i;         // its u face x-
    int fvf = (k0 * (g.ny + 1) + j) * g.nx + i;         // its v face y-
    unsigned cc = codes[c];
    float pc = p[c];
    float wb;
    {
      const unsigned cb = k0 > 0 ? codes[c - nxny] : 0u;
      const float pb = k0 > 0 ? p[c - nxny] : 0.f;
      wb = corrected_w_vals(g, k1, ws[c], i, j, k0, cb, pb, pc);
    }
    for (int k = k0; k < ke; ++k) {
      const bool zp = k + 1 < g.nz;
      const unsigned ca = zp ? codes[c + nxny] : 0u;
      const float pa = zp ? p[c + nxny] : 0.f;
      const unsigned cxm = xm ? codes[c - 1] : 0u, cxp = xp ? codes[c + 1] : 0u;
      const unsigned cym = ym ? codes[c - g.nx] : 0u, cyp = yp ? codes[c + g.nx] : 0u;
      const float pxm = xm ? p[c - 1] : 0.f, pxp = xp ? p[c + 1] : 0.f;
      const float pym = ym ? p[c - g.nx] : 0.f, pyp = yp ? p[c + g.nx] : 0.f;
      const float ul = corrected_uv_vals(g, k1, us[ful], 0, i, j, k, cc, cxm, pc, pxm);
      const float ur = corrected_uv_vals(g, k1, us[ful + 1], 0, i + 1, j, k, cxp, cc, pxp, pc);
      const float vf = corrected_uv_vals(g, k1, vs[fvf], 1, i, j, k, cc, cym, pc, pym);
      const float vk = corrected_uv_vals(g, k1, vs[fvf + g.nx], 1, i, j + 1, k, cyp, cc, pyp, pc);
      const float wt = corrected_w_vals(g, k1, ws[c + nxny], i, j, k + 1, cc, pc, pa);
      u[ful] = ul;
      v[fvf] = vf;
      w[c] = wb;
      mx = fmaxf(mx, fabsf(ul));
      mx = fmaxf(mx, fabsf(vf));
      mx = fmaxf(mx, fabsf(wb));
      if (!xp) { u[ful + 1] = ur; mx = fmaxf(mx, fabsf(ur)); }
      if (!yp) { v[fvf + g.nx] = vk; mx = fmaxf(mx, fabsf(vk)); }
      if (!zp) { w[c + nxny] = wt; mx = fmaxf(mx, fabsf(wt)); }
      if (cc & RC_WET) div_metric_vals(g, cc, i, j, k, ul, ur, vf, vk, wb, wt, all, plain);
      cc = ca;
      pc = pa;
      wb = wt;
      c += nxny;
      ful += su;
      fvf += sv;
    }
  }
  block_fmax3_atomic(all, plain, mx, &S->fmax[0], &S->fmax[1], &S->fmax[2]);
}

// One row of backward_error_mobile3 (delta3d_mobile.rs:243-271): |r_i| / (|b| + |A||p|)_i of a wet
// row (0 for a dry row or a zero scale), from the pressures of the cell and its six neighbours (x-,
// x+, y-, y+, z-, z+; a neighbour's is read only across a live face), b_i and r_i.  The apertures and
// ghost coefficients are apply_code's.
__device__ __forceinline__ float backward_error_vals(const Geo& g, unsigned code, int i, int j, int k, float pcv,
                                                    float pxm, float pxp, float pym, float pyp, float pzm, float pzp,
                                                    float bc, float rc) {
  if (!(code & RC_WET)) return 0.f;
  const bool unit = code & RC_UNIT;
  const float pc = fabsf(pcv);
  float acc = 0.f;
  auto face = [&](int f, int axis, int fi, float pm, int x, int y) {
    const unsigned st = face_state(code, f);
    if (!st) return;
    const float a = unit ? 1.f : aper3(g, axis, fi);
    if (st == 1) acc += a * (pc + fabsf(pm));
    else acc += a * pc * (f == 5 ? ghost_it_up(g, i, j, k) : ghost_it_side(g, i, j, k, x, y));
  };
  face(0, 0, fu(g, i, j, k), pxm, i - 1, j);
  face(1, 0, fu(g, i + 1, j, k), pxp, i + 1, j);
  face(2, 1, fv(g, i, j, k), pym, i, j - 1);
  face(3, 1, fv(g, i, j + 1, k), pyp, i, j + 1);
  face(4, 2, fw(g, i, j, k), pzm, i, j);
  face(5, 2, fw(g, i, j, k + 1), pzp, i, j);
  const float scale = fabsf(bc) + acc * g.inv;
  return scale > 0.f ? fabsf(rc) / scale : 0.f;
}
__device__ __forceinline__ float backward_error_cell(const Geo& g, unsigned code, const float* __restrict__ p,
                                                     const float* __restrict__ rhs, const float* __restrict__ res,
                                                     int c) {
  if (!(code & RC_WET)) return 0.f;
  int i, j, k; cell_ijk(g, c, i, j, k);
  const int nxny = g.nx * g.ny;
  return backward_error_vals(g, code, i, j, k, p[c], i > 0 ? p[c - 1] : 0.f, i + 1 < g.nx ? p[c + 1] : 0.f,
                             j > 0 ? p[c - g.nx] : 0.f, j + 1 < g.ny ? p[c + g.nx] : 0.f, k > 0 ? p[c - nxny] : 0.f,
                             k + 1 < g.nz ? p[c + nxny] : 0.f, rhs[c], res[c]);
}

// backward_error_mobile3 (delta3d_mobile.rs:243-271) and the fingerprint of p in one pass, marching
// the columns as k_correct_metric does (the pressures below and above ride in registers): the
// largest |r_i| / (|b| + |A||p|)_i over the wet rows into S->fmax[3] (one atomic per block), and the
// wrapping sum of hash_at over every cell into S->hash (one atomic per warp; the sum does not depend
// on the order).  Both reset before.
__global__ void __launch_bounds__(CM_X * CM_Y, FD3_SETUP_MINB) k_backward_hash(Geo g, const unsigned short* __restrict__ codes,
                                                               const float* __restrict__ p,
                                                               const float* __restrict__ rhs,
                                                               const float* __restrict__ res, Scalars* S) {
  KSTART();
  float worst = 0.f;
  unsigned long long h = 0ull;
  const int ntx = (g.nx + CM_X - 1) / CM_X, nty = (g.ny + CM_Y - 1) / CM_Y;
  int b = blockIdx.x;
  const int bx = b % ntx; b /= ntx;
  const int by = b % nty; b /= nty;
  const int i = bx * CM_X + (int)(threadIdx.x & 31), j = by * CM_Y + (int)(threadIdx.x >> 5);
  const int k0 = b * CM_K, ke = min(k0 + CM_K, g.nz);
  if (i < g.nx && j < g.ny) {
    const int nxny = g.nx * g.ny;
    const bool xm = i > 0, xp = i + 1 < g.nx, ym = j > 0, yp = j + 1 < g.ny;
    int c = (k0 * g.ny + j) * g.nx + i;
    float pb = k0 > 0 ? p[c - nxny] : 0.f;
    float pc = p[c];
    for (int k = k0; k < ke; ++k, c += nxny) {
      const float pa = k + 1 < g.nz ? p[c + nxny] : 0.f;
      const unsigned code = codes[c];
      const float pxm = xm ? p[c - 1] : 0.f, pxp = xp ? p[c + 1] : 0.f;
      const float pym = ym ? p[c - g.nx] : 0.f, pyp = yp ? p[c + g.nx] : 0.f;
      const float bc = rhs[c], rc = res[c];
      worst = fmaxf(worst, backward_error_vals(g, code, i, j, k, pc, pxm, pxp, pym, pyp, pb, pa, bc, rc));
      h += hash_val(pc, c);
      pb = pc;
      pc = pa;
    }
  }
  block_fmax2_atomic(worst, 0.f, &S->fmax[3], nullptr);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) h += __shfl_down_sync(0xffffffffu, h, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(&S->hash, h);
}

// ------------------------------------------------------------------------------------------------
// Reductions finished in the kernel that produces them: each block leaves its partial(s), the last
// block to arrive (a counter) merges them in a fixed order and applies the PCG scalar step.

template <int MODE>
__device__ void finish_block(Red red, int nparts, Scalars* S, int op);

__device__ __forceinline__ void apply_op(Scalars* S, double val, int op, int ord) {
  const bool finite = isfinite(val);
  const bool zero_but_nonzero = ord && val == 0.0 && S->any_nonzero;
  switch (op) {
    case FIN_B2:
      S->b2 = val;
      if (!finite || zero_but_nonzero) S->status = 2;
      break;
    case FIN_RR0:
    case FIN_ACTUAL:
      if (op == FIN_RR0) S->rr = val; else S->actual = val;
      if (!finite || zero_but_nonzero) S->status = 2;
      if (S->vk > 0.f && val > 0.0) S->vinv = (float)((double)S->vk / sqrt(val));
      break;
    case FIN_DQ:
      S->dq = val;
      if (!(val > 0.0)) { S->active = 0; S->brk = 1; }
      else S->alpha = ord ? (float)S->rz / (float)val : (float)(S->rz / val);
      break;
    case FIN_RN:
      S->rn = val;
      if (!finite || zero_but_nonzero) { S->status = 2; S->active = 0; break; }
      if (S->vk > 0.f && val > 0.0) S->vinv = (float)((double)S->vk / sqrt(val));
      if (!loop_continues(S, val, S->it + 1, ord)) { S->rr = val; S->it += 1; S->active = 0; }
      break;
    case FIN_RZ_ITER:
      if (!finite) { S->status = 2; S->active = 0; break; }
      S->zn = val;
      S->beta = ord ? (float)val / (float)S->rz : (float)(val / S->rz);
      S->rz = val;
      S->rr = S->rn;
      S->it += 1;
      S->dir_mode = 1;
      break;
    case FIN_RZ_PRIME:
      if (!finite) S->status = 2;
      S->rz = val;
      S->dir_mode = 0;
      break;
  }
  S->any_nonzero = 0;
}

template <>
__device__ void finish_block<RED_F64>(Red red, int nparts, Scalars* S, int op) {
  __shared__ double sm[TPB];
  double s = 0.0;
  // each thread's partials in index order, their loads issued eight at a time (the sums are the same)
  const int step = blockDim.x;
  int q = threadIdx.x;
  for (; q + 7 * step < nparts; q += 8 * step) {
    double v[8];
#pragma unroll
    for (int e = 0; e < 8; ++e) v[e] = __ldcg(red.p64 + q + e * step);
#pragma unroll
    for (int e = 0; e < 8; ++e) s += v[e];
  }
  for (; q < nparts; q += step) s += __ldcg(red.p64 + q);
  sm[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) sm[threadIdx.x] += sm[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) apply_op(S, sm[0], op, 0);
}

template <>
__device__ void finish_block<RED_ORD>(Red red, int nparts, Scalars* S, int op) {
  if (threadIdx.x != 0) return;
  // serial in-order merge in f32 (host_impl.rs:75-92, merge of delta3d.rs:867)
  float acc = 0.f;
  int q = 0;
  for (; q + 8 <= nparts; q += 8) {
    float v[8];
#pragma unroll
    for (int e = 0; e < 8; ++e) v[e] = __ldcg(red.p32 + q + e);
#pragma unroll
    for (int e = 0; e < 8; ++e) acc = acc + v[e];
  }
  for (; q < nparts; ++q) acc = acc + __ldcg(red.p32 + q);
  apply_op(S, (double)acc, op, 1);
}

template <int MODE>
__device__ __forceinline__ void reduce_finish(typename Acc<MODE>::T v, int c, int n, Red red, Scalars* S, int op) {
  block_reduce<MODE>(v, c, n, red);
  __shared__ bool last;
  // the partials must be visible before the block counts in: in f64 mode thread 0 wrote the block's
  // one partial and alone fences (the other threads' stores need no ordering here: the next kernel
  // sees them after the grid completes); in ordered mode several threads wrote chunk partials
  if (MODE == RED_ORD) __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    if (MODE != RED_ORD) __threadfence();
    last = atomicAdd(red.count, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  const int nparts = MODE == RED_ORD ? (n + CHUNK - 1) / CHUNK : (int)gridDim.x;
  finish_block<MODE>(red, nparts, S, op);
  if (threadIdx.x == 0) *red.count = 0u;
}

// ------------------------------------------------------------------------------------------------
// The PCG step (delta3d_mobile.rs:523-545) with the multigrid preconditioner.

// d = z (S->dir_mode 0, after a prime) or d = z + beta d (1, direction_multigrid3), written to
// dout; q = A d; d.q; alpha = rz/dq or a stop (FIN_DQ).  d is recomputed at each stencil point.
template <int MODE>
__global__ void __launch_bounds__(TPB) k_dir_apply_dot(Geo g, const unsigned short* __restrict__ codes,
                                                       const float* __restrict__ z, const float* __restrict__ din,
                                                       float* __restrict__ dout, float* __restrict__ q, Red red,
                                                       Scalars* S) {
  KSTART();
  if (!S->active) return;
  const int mode = S->dir_mode;
  const float beta = S->beta;
  auto D = [&](int n) { return mode ? z[n] + beta * din[n] : z[n]; };
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  float dc = 0.f, qc = 0.f;
  if (c < g.n) {
    dc = D(c);
    unsigned code = codes[c];
    if (code & RC_WET) { int i, j, k; cell_ijk(g, c, i, j, k); qc = apply_code(g, code, i, j, k, c, D); }
    dout[c] = dc;
    q[c] = qc;
  }
  reduce_finish<MODE>(Acc<MODE>::prod(dc, qc), c, g.n, red, S, FIN_DQ);
}

// p += alpha d, r -= alpha q, with r.r (FIN_RN decides whether the loop continues).
template <int MODE>
__global__ void __launch_bounds__(TPB) k_update_rn(int n, float* __restrict__ p, float* __restrict__ r,
                                                   const float* __restrict__ d, const float* __restrict__ q, Red red,
                                                   Scalars* S) {
  KSTART();
  if (!S->active) return;
  const float alpha = S->alpha;
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  float rn = 0.f;
  if (c < n) {
    p[c] += alpha * d[c];
    rn = r[c] - alpha * q[c];
    r[c] = rn;
  }
  if (__syncthreads_or(c < n && rn != 0.f) && threadIdx.x == 0) atomicOr(&S->any_nonzero, 1);
  reduce_finish<MODE>(Acc<MODE>::prod(rn, rn), c, n, red, S, FIN_RN);
}

// The two pre-sweeps from z = 0 (v_cycle3, delta3d_multigrid.rs:398-405): z1 = w prec r is
// recomputed at each stencil point, z2 = z1 + w prec (r - A z1) is written.
__global__ void __launch_bounds__(TPB) k_fine_pre(Geo g, const unsigned short* __restrict__ codes,
                                                  const float* __restrict__ prec, const float* __restrict__ r,
                                                  float* __restrict__ z2, const Scalars* S, int gate) {
  KSTART();
  if (gate && !S->active) return;
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= g.n) return;
  auto Z1 = [&](int n) {
    float m = prec[n];
    return m > 0.f ? 0.f + OMEGA * m * (r[n] - 0.f) : 0.f;
  };
  float m = prec[c];
  float zc = Z1(c);
  if (m > 0.f) {
    int i, j, k; cell_ijk(g, c, i, j, k);
    zc += OMEGA * m * (r[c] - apply_code(g, (unsigned)codes[c], i, j, k, c, Z1));
  }
  z2[c] = zc;
}

// Coarse r = mean over the 8 children of (r - A z) (restrict3).
__global__ void __launch_bounds__(TPB) k_fine_restrict_c(Geo g, const unsigned short* __restrict__ codes,
                                                         const float* __restrict__ r, const float* __restrict__ z,
                                                         Lev L, const Scalars* S, int gate) {
  KSTART();
  if (gate && !S->active) return;
  int qi = blockIdx.x * blockDim.x + threadIdx.x;
  if (qi >= L.n) return;
  int ci = qi % L.nx, t = qi / L.nx, cj = t % L.ny, ck = t / L.ny;
  Load Z{z};
  float s = 0.f;
#pragma unroll
  for (int e = 0; e < 8; ++e) {
    int i = 2 * ci + (e & 1), j = 2 * cj + ((e >> 1) & 1), k = 2 * ck + (e >> 2);
    int c = (k * g.ny + j) * g.nx + i;
    unsigned code = codes[c];
    float az = (code & RC_WET) ? apply_code(g, code, i, j, k, c, Z) : 0.f;
    s += r[c] - az;
  }
  L.r[qi] = 0.125f * s;
}

// Prolongation (z += parent x; z = 0 where prec == 0) fused with the first post-sweep; without
// coarse levels (prolong = 0) the plain third sweep.
__global__ void __launch_bounds__(TPB) k_fine_post1(Geo g, const unsigned short* __restrict__ codes,
                                                    const float* __restrict__ prec, const float* __restrict__ r,
                                                    const float* __restrict__ zin, Lev L, int prolong,
                                                    float* __restrict__ zout, const Scalars* S, int gate) {
  KSTART();
  if (gate && !S->active) return;
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= g.n) return;
  const int nx = g.nx;
  auto ZP = [&](int n) {
    if (!prolong) return zin[n];
    int i = n % nx, t = n / nx, j = t % g.ny, k = t / g.ny;
    float v = zin[n] + L.x[((k >> 1) * L.ny + (j >> 1)) * L.nx + (i >> 1)];
    return prec[n] == 0.f ? 0.f : v;
  };
  float m = prec[c];
  float zc = ZP(c);
  if (m > 0.f) {
    int i, j, k; cell_ijk(g, c, i, j, k);
    zc += OMEGA * m * (r[c] - apply_code(g, (unsigned)codes[c], i, j, k, c, ZP));
  }
  zout[c] = zc;
}

// The last post-sweep fused with res.z (prime: FIN_RZ_PRIME; iteration: FIN_RZ_ITER).
template <int MODE>
__global__ void __launch_bounds__(TPB) k_fine_post2_rz(Geo g, const unsigned short* __restrict__ codes,
                                                       const float* __restrict__ prec, const float* __restrict__ r,
                                                       const float* __restrict__ zin, float* __restrict__ zout,
                                                       Red red, Scalars* S, int gate, int op) {
  KSTART();
  if (gate && !S->active) return;
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  float rc = 0.f, zc = 0.f;
  if (c < g.n) {
    Load Z{zin};
    float m = prec[c];
    rc = r[c];
    zc = zin[c];
    if (m > 0.f) {
      int i, j, k; cell_ijk(g, c, i, j, k);
      zc += OMEGA * m * (rc - apply_code(g, (unsigned)codes[c], i, j, k, c, Z));
    }
    zout[c] = zc;
  }
  reduce_finish<MODE>(Acc<MODE>::prod(rc, zc), c, g.n, red, S, op);
}

// ------------------------------------------------------------------------------------------------
// Jacobi-preconditioned step (the reference's default without enable_multigrid).

template <int MODE>
__global__ void __launch_bounds__(TPB) k_apply_dot_c(Geo g, const unsigned short* __restrict__ codes,
                                                     const float* __restrict__ d, float* __restrict__ q, Red red,
                                                     Scalars* S) {
  KSTART();
  if (!S->active) return;
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  float dc = 0.f, qc = 0.f;
  if (c < g.n) {
    dc = d[c];
    unsigned code = codes[c];
    if (code & RC_WET) { int i, j, k; cell_ijk(g, c, i, j, k); qc = apply_code(g, code, i, j, k, c, Load{d}); }
    q[c] = qc;
  }
  reduce_finish<MODE>(Acc<MODE>::prod(dc, qc), c, g.n, red, S, FIN_DQ);
}

template <int MODE>
__global__ void __launch_bounds__(TPB) k_dot_prec_fin(int n, const float* __restrict__ r, const float* __restrict__ prec,
                                                      Red red, Scalars* S, int gate, int op) {
  KSTART();
  if (gate && !S->active) return;
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  float x = 0.f, m = 0.f;
  if (c < n) { x = r[c]; m = prec[c]; }
  reduce_finish<MODE>(Acc<MODE>::prod3(x, m, x), c, n, red, S, op);
}

// ------------------------------------------------------------------------------------------------
// Coarse levels.  level_row with an operand functor.
template <class P>
__device__ __forceinline__ float level_row_f(const Lev& L, int i, int j, int k, int c, P p) {
  const float pc = p(c);
  float acc = 0.f;
  const int nxny = L.nx * L.ny;
  auto face = [&](float a, bool has, int m, bool top) {
    if (a == 0.f) return;
    if (has) {
      float km = L.kind[m];
      if (km > 0.f) acc += a * (pc - p(m));
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

// Row codes of a coarse level (row_sums, delta3d_multigrid.rs:216-255), once per projection after
// coarsen3: bit 0 active (kind > 0); per face 0 nothing, 1 active neighbour (a (pc - p_m)),
// 2 Dirichlet (an air neighbour or the top of the domain: 2 a pc); bit 13 every live aperture is 1.
__device__ __forceinline__ unsigned level_codes_at(const Lev& L, int c) {
  unsigned code = 0;
  if (L.kind[c] > 0.f) {
    int i = c % L.nx, t = c / L.nx, j = t % L.ny, k = t / L.ny;
    const int nxny = L.nx * L.ny;
    code = RC_WET;
    bool unit = true;
    auto face = [&](int f, float a, bool has, int m, bool top) {
      unsigned st = 0;
      if (a != 0.f) {
        if (has) {
          float km = L.kind[m];
          st = km > 0.f ? 1u : (km < 0.f ? 2u : 0u);
        } else if (top) {
          st = 2u;
        }
      }
      code |= st << (1 + 2 * f);
      if (st && a != 1.f) unit = false;
    };
    face(0, L.ou[(k * L.ny + j) * (L.nx + 1) + i], i > 0, c - 1, false);
    face(1, L.ou[(k * L.ny + j) * (L.nx + 1) + i + 1], i + 1 < L.nx, c + 1, false);
    face(2, L.ov[(k * (L.ny + 1) + j) * L.nx + i], j > 0, c - L.nx, false);
    face(3, L.ov[(k * (L.ny + 1) + j + 1) * L.nx + i], j + 1 < L.ny, c + L.nx, false);
    face(4, L.ow[(k * L.ny + j) * L.nx + i], k > 0, c - nxny, false);
    face(5, L.ow[((k + 1) * L.ny + j) * L.nx + i], k + 1 < L.nz, c + nxny, true);
    if (unit) code |= RC_UNIT;
  }
  return code;
}
// prepare_multigrid3 (delta3d_multigrid.rs:370-387) of one level in two passes: the kinds and the
// apertures (coarsen3 from the fine volume, `fine`, or from level F; cells, then faces, in one index
// space), then the diagonal and the row codes, which read only those.
__global__ void k_level_prepare_a(Geo g, Lev F, Lev C, int fine) {
  KSTART();
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q < C.n) {
    C.kind[q] = fine ? coarsen_kind_fine_at(g, C, q) : coarsen_kind_level_at(F, C, q);
    return;
  }
  q -= C.n;
  if (fine) coarsen_open_at(g.nx, g.ny, g.ou, g.ov, g.ow, g.act, C, q);
  else coarsen_open_at(F.nx, F.ny, F.ou, F.ov, F.ow, nullptr, C, q);
}
__global__ void k_level_prepare_b(Lev C) {
  KSTART();
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= C.n) return;
  C.diag[c] = level_diag_at(C, c);
  C.code[c] = (unsigned short)level_codes_at(C, c);
}
// The same for levels first .. last (first >= 1, every one small) in one CTA: the kinds and
// apertures level by level, a barrier after each, then every level's diagonal and codes.
constexpr int PREP_SMALL_THREADS = 1024;
__global__ void __launch_bounds__(PREP_SMALL_THREADS) k_levels_prepare_small(const Lev* __restrict__ levs, int first,
                                                                          int last) {
  KSTART();
  for (int l = first; l <= last; ++l) {
    const Lev F = levs[l - 1], C = levs[l];
    const int nfaces = (C.nx + 1) * C.ny * C.nz + C.nx * (C.ny + 1) * C.nz + C.nx * C.ny * (C.nz + 1);
    for (int q = threadIdx.x; q < C.n + nfaces; q += blockDim.x) {
      if (q < C.n) C.kind[q] = coarsen_kind_level_at(F, C, q);
      else coarsen_open_at(F.nx, F.ny, F.ou, F.ov, F.ow, nullptr, C, q - C.n);
    }
    __syncthreads();
  }
  for (int l = first; l <= last; ++l) {
    const Lev C = levs[l];
    for (int c = threadIdx.x; c < C.n; c += blockDim.x) {
      C.diag[c] = level_diag_at(C, c);
      C.code[c] = (unsigned short)level_codes_at(C, c);
    }
  }
}

// One row of row_sums (with p) from its code: the same terms, in the same order, as level_row_f.
template <class P>
__device__ __forceinline__ float level_row_code(const Lev& L, unsigned code, int i, int j, int k, int c, P p) {
  const float pc = p(c);
  const int nxny = L.nx * L.ny;
  float acc = 0.f;
  if (rc_plain(code)) {  // unit apertures, no Dirichlet face: the masked sum (see rc_plain)
    acc += (code & (1u << 1)) ? pc - p(c - 1) : 0.f;
    acc += (code & (1u << 3)) ? pc - p(c + 1) : 0.f;
    acc += (code & (1u << 5)) ? pc - p(c - L.nx) : 0.f;
    acc += (code & (1u << 7)) ? pc - p(c + L.nx) : 0.f;
    acc += (code & (1u << 9)) ? pc - p(c - nxny) : 0.f;
    acc += (code & (1u << 11)) ? pc - p(c + nxny) : 0.f;
    return acc * L.inv;
  }
  const bool unit = code & RC_UNIT;
  auto face = [&](int f, const float* ap, int fi, int m) {
    unsigned st = face_state(code, f);
    if (!st) return;
    float a = unit ? 1.f : ap[fi];
    if (st == 1) acc += a * (pc - p(m));
    else acc += 2.f * a * pc;
  };
  face(0, L.ou, (k * L.ny + j) * (L.nx + 1) + i, c - 1);
  face(1, L.ou, (k * L.ny + j) * (L.nx + 1) + i + 1, c + 1);
  face(2, L.ov, (k * (L.ny + 1) + j) * L.nx + i, c - L.nx);
  face(3, L.ov, (k * (L.ny + 1) + j + 1) * L.nx + i, c + L.nx);
  face(4, L.ow, (k * L.ny + j) * L.nx + i, c - nxny);
  face(5, L.ow, ((k + 1) * L.ny + j) * L.nx + i, c + nxny);
  return acc * L.inv;
}

// x0 = 0 + w (r - 0)/diag (first sweep), recomputed per stencil point.  T: the storage of the
// level's vectors (f32, or FP16 in the mixed-precision mode).
template <class T = float>
__device__ __forceinline__ float level_x1(const Lev& L, int n) {
  float dg = L.diag[n];
  return dg > 0.f ? 0.f + OMEGA * (Store<T>::ld(as<T>(L.r), n) - 0.f) / dg : 0.f;
}

// The small coarse levels' passes are latency-bound: a pass is one dependent chain of loads per
// thread.  There (SPEC) every load a cell may need is issued before its row code (and the loop's
// gate) arrive: the six neighbours' operands at indices clamped to the grid (a neighbour outside
// the grid has face state 0 and its value is never used) and the six apertures; then the gate is
// checked before anything is stored.  The row is then summed without branches (level_row_sel):
// in a latency-bound pass a warp whose rows take different branches pays for each divergent path
// and its reconvergence in series, which cost more than the selects.
struct Nb6 {
  float xm, xp, ym, yp, zm, zp;
};
// P(n, i, j, k): the operand at cell n = (i, j, k).
template <class P>
__device__ __forceinline__ Nb6 level_nb(const Lev& L, int i, int j, int k, int c, const P& p) {
  const int nxny = L.nx * L.ny;
  const bool xl = i > 0, xr = i + 1 < L.nx, yl = j > 0, yr = j + 1 < L.ny, zl = k > 0, zr = k + 1 < L.nz;
  Nb6 b;
  b.xm = p(xl ? c - 1 : c, xl ? i - 1 : i, j, k);
  b.xp = p(xr ? c + 1 : c, xr ? i + 1 : i, j, k);
  b.ym = p(yl ? c - L.nx : c, i, yl ? j - 1 : j, k);
  b.yp = p(yr ? c + L.nx : c, i, yr ? j + 1 : j, k);
  b.zm = p(zl ? c - nxny : c, i, j, zl ? k - 1 : k);
  b.zp = p(zr ? c + nxny : c, i, j, zr ? k + 1 : k);
  return b;
}
// The six apertures of a coarse cell's faces, loaded whatever its row code (every face index of a
// cell is valid), so that they are in flight with the code.
struct Ap6 {
  float a[6];
};
__device__ __forceinline__ Ap6 level_ap6(const Lev& L, int i, int j, int k) {
  Ap6 o;
  o.a[0] = L.ou[(k * L.ny + j) * (L.nx + 1) + i];
  o.a[1] = L.ou[(k * L.ny + j) * (L.nx + 1) + i + 1];
  o.a[2] = L.ov[(k * (L.ny + 1) + j) * L.nx + i];
  o.a[3] = L.ov[(k * (L.ny + 1) + j + 1) * L.nx + i];
  o.a[4] = L.ow[(k * L.ny + j) * L.nx + i];
  o.a[5] = L.ow[((k + 1) * L.ny + j) * L.nx + i];
  return o;
}
// level_row_code of any row from preloaded neighbours and apertures, without branches: each face
// adds a (pc - x) (fluid neighbour), 2 a pc (Dirichlet face) or +0 (no face), selected by its state.
// Adding +0 changes no partial sum (the sum starts at +0 and is never -0), so the bits are those of
// level_row_code, which skips the missing faces; a plain row's a is exactly 1.
__device__ __forceinline__ float level_row_sel(const Lev& L, unsigned code, float pc, const Nb6& b, const Ap6& ap) {
  const bool unit = code & RC_UNIT;
  const float v[6] = {b.xm, b.xp, b.ym, b.yp, b.zm, b.zp};
  float acc = 0.f;
#pragma unroll
  for (int f = 0; f < 6; ++f) {
    const unsigned st = face_state(code, f);
    const float a = unit ? 1.f : ap.a[f];
    const float t1 = a * (pc - v[f]);
    const float t2 = 2.f * a * pc;
    acc += st == 1u ? t1 : (st == 2u ? t2 : 0.f);
  }
  return acc * L.inv;
}
// One damped Jacobi update x + w (r - row) / diag where diag > 0, x itself elsewhere, with the
// division done by every lane and the result selected: the bits of the guarded update.  Used by the
// one-CTA tail, whose phases are one warp's dependent chain; in the level kernels, whose dry cells
// come in whole warps, the guarded division measured faster.
__device__ __forceinline__ float jacobi_sel(float x, float r, float row, float dg) {
  const float y = x + OMEGA * (r - row) / (dg > 0.f ? dg : 1.f);
  return dg > 0.f ? y : x;
}
__device__ __forceinline__ void level_ijk(const Lev& L, int c, int& i, int& j, int& k) {
  i = c % L.nx;
  const int t = c / L.nx;
  j = t % L.ny;
  k = t / L.ny;
}

// The two pre-sweeps of a coarse level from x = 0, written to L.x (smooth3 twice after fill(0)).
template <class T, bool SPEC>
__global__ void __launch_bounds__(TPB) k_level_pre(Lev L, const Scalars* S, int gate) {
  KSTART();
  if (!SPEC && gate && !S->active) return;
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= L.n) return;
  auto X1 = [&](int n) { return level_x1<T>(L, n); };
  auto X1c = [&](int n, int, int, int) { return level_x1<T>(L, n); };
  int i, j, k;
  level_ijk(L, c, i, j, k);
  const unsigned code = L.code[c];
  const float dg = L.diag[c];
  const float rc = Store<T>::ld(as<T>(L.r), c);
  float xc = X1(c);
  if (SPEC) {
    const Ap6 ap = level_ap6(L, i, j, k);
    const Nb6 b = level_nb(L, i, j, k, c, X1c);
    if (gate && !S->active) return;
    if (dg > 0.f) xc += OMEGA * (rc - level_row_sel(L, code, xc, b, ap)) / dg;
  } else if (dg > 0.f) {
    xc += OMEGA * (rc - level_row_code(L, code, i, j, k, c, X1)) / dg;
  }
  Store<T>::st(as<T>(L.x), c, xc);
}

// t = r - L x on every cell of a coarse level (0 on inactive rows), the restriction's operand.
template <class T, bool SPEC>
__global__ void __launch_bounds__(TPB) k_level_resid(Lev L, const Scalars* S, int gate) {
  KSTART();
  if (!SPEC && gate && !S->active) return;
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= L.n) return;
  const LoadT<T> X{as<T>(L.x)};
  auto Xc = [&](int n, int, int, int) { return X(n); };
  int i, j, k;
  level_ijk(L, c, i, j, k);
  const unsigned code = L.code[c];
  const float rc = Store<T>::ld(as<T>(L.r), c);
  const float pc = X(c);
  float lx = 0.f;
  if (SPEC) {
    const Ap6 ap = level_ap6(L, i, j, k);
    const Nb6 b = level_nb(L, i, j, k, c, Xc);
    if (gate && !S->active) return;
    if (code & RC_WET) lx = level_row_sel(L, code, pc, b, ap);
  } else if (code & RC_WET) {
    lx = level_row_code(L, code, i, j, k, c, X);
  }
  Store<T>::st(as<T>(L.t), c, rc - lx);
}

// C.r = mean of the 8 children of F.t, in the reference's CHILDREN order (restrict3).
template <class T>
__global__ void __launch_bounds__(TPB) k_level_sum8(Lev F, Lev C, const Scalars* S, int gate) {
  KSTART();
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= C.n) return;
  int ci = q % C.nx, t = q / C.nx, cj = t % C.ny, ck = t / C.ny;
  float v[8];
#pragma unroll
  for (int e = 0; e < 8; ++e) {
    int i = 2 * ci + (e & 1), j = 2 * cj + ((e >> 1) & 1), k = 2 * ck + (e >> 2);
    v[e] = Store<T>::ld(as<T>(F.t), (k * F.ny + j) * F.nx + i);
  }
  if (gate && !S->active) return;
  float s = 0.f;
#pragma unroll
  for (int e = 0; e < 8; ++e) s += v[e];
  Store<T>::st(as<T>(C.r), q, 0.125f * s);
}

// k_level_resid and k_level_sum8 in one pass, with one thread per fine cell as k_level_resid has:
// the eight threads of a coarse cell (consecutive lanes, child e = lane % 8 in the reference's
// CHILDREN order) each evaluate one child's t = r - L x, rounded through the storage type as the
// stored t would be, and the first of them sums the eight in order (restrict3).
template <class T, bool SPEC>
__global__ void __launch_bounds__(TPB) k_level_restrict8(Lev F, Lev C, const Scalars* S, int gate) {
  KSTART();
  if (!SPEC && gate && !S->active) return;
  const int q8 = blockIdx.x * blockDim.x + threadIdx.x;
  const int q = q8 >> 3, e = q8 & 7;
  const bool own = q < C.n;
  float tv = 0.f;
  unsigned code = 0u;
  int i = 0, j = 0, k = 0, c = 0;
  float rc = 0.f, pc = 0.f;
  const LoadT<T> X{as<T>(F.x)};
  if (own) {
    const int ci = q % C.nx, t = q / C.nx, cj = t % C.ny, ck = t / C.ny;
    i = 2 * ci + (e & 1);
    j = 2 * cj + ((e >> 1) & 1);
    k = 2 * ck + (e >> 2);
    c = (k * F.ny + j) * F.nx + i;
    code = F.code[c];
    rc = Store<T>::ld(as<T>(F.r), c);
    pc = X(c);
  }
  if (SPEC) {
    Nb6 b{};
    Ap6 ap{};
    if (own) {
      ap = level_ap6(F, i, j, k);
      b = level_nb(F, i, j, k, c, [&](int n, int, int, int) { return X(n); });
    }
    if (gate && !S->active) return;
    if (own) tv = Store<T>::rt(rc - ((code & RC_WET) ? level_row_sel(F, code, pc, b, ap) : 0.f));
  } else if (own) {
    tv = Store<T>::rt(rc - ((code & RC_WET) ? level_row_code(F, code, i, j, k, c, X) : 0.f));
  }
  const int lane0 = threadIdx.x & 24;  // first lane of the eight
  float sum = 0.f;
#pragma unroll
  for (int a = 0; a < 8; ++a) sum += __shfl_sync(0xffffffffu, tv, lane0 + a);
  if (own && e == 0) Store<T>::st(as<T>(C.r), q, 0.125f * sum);
}

// Prolongation from C (x += parent) fused with the first post-sweep, L.x -> L.x2.
template <class T, bool SPEC>
__global__ void __launch_bounds__(TPB) k_level_post1(Lev L, Lev C, const Scalars* S, int gate) {
  KSTART();
  if (!SPEC && gate && !S->active) return;
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= L.n) return;
  auto XPc = [&](int n, int i, int j, int k) {
    return Store<T>::ld(as<T>(L.x), n) + Store<T>::ld(as<T>(C.x), ((k >> 1) * C.ny + (j >> 1)) * C.nx + (i >> 1));
  };
  auto XP = [&](int n) {
    int i, j, k;
    level_ijk(L, n, i, j, k);
    return XPc(n, i, j, k);
  };
  int i, j, k;
  level_ijk(L, c, i, j, k);
  const unsigned code = L.code[c];
  const float dg = L.diag[c];
  const float rc = Store<T>::ld(as<T>(L.r), c);
  float xc = XPc(c, i, j, k);
  if (SPEC) {
    const Ap6 ap = level_ap6(L, i, j, k);
    const Nb6 b = level_nb(L, i, j, k, c, XPc);
    if (gate && !S->active) return;
    if (dg > 0.f) xc += OMEGA * (rc - level_row_sel(L, code, xc, b, ap)) / dg;
  } else if (dg > 0.f) {
    xc += OMEGA * (rc - level_row_code(L, code, i, j, k, c, XP)) / dg;
  }
  Store<T>::st(as<T>(L.x2), c, xc);
}

// The second post-sweep, L.x2 -> L.x.
template <class T, bool SPEC>
__global__ void __launch_bounds__(TPB) k_level_post2(Lev L, const Scalars* S, int gate) {
  KSTART();
  if (!SPEC && gate && !S->active) return;
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= L.n) return;
  const LoadT<T> X{as<T>(L.x2)};
  auto Xc = [&](int n, int, int, int) { return X(n); };
  int i, j, k;
  level_ijk(L, c, i, j, k);
  const unsigned code = L.code[c];
  const float dg = L.diag[c];
  const float rc = Store<T>::ld(as<T>(L.r), c);
  float xc = X(c);
  if (SPEC) {
    const Ap6 ap = level_ap6(L, i, j, k);
    const Nb6 b = level_nb(L, i, j, k, c, Xc);
    if (gate && !S->active) return;
    if (dg > 0.f) xc += OMEGA * (rc - level_row_sel(L, code, xc, b, ap)) / dg;
  } else if (dg > 0.f) {
    xc += OMEGA * (rc - level_row_code(L, code, i, j, k, c, X)) / dg;
  }
  Store<T>::st(as<T>(L.x), c, xc);
}

// k_level_post2 of the coarser level C fused into k_level_post1 of L: the eight threads of a C
// cell (consecutive lanes, child e = lane % 8) are its eight children in L.  Lanes 0..6 evaluate
// C's second post-sweep at the cell and at its six neighbours (the parents of the children's
// stencil points), with k_level_post2's expression, rounded through the storage type as the stored
// C.x would be; the warp shares the seven values; each child then sweeps its own row with
// k_level_post1's expression.  C.x is never stored: only this pass would read it.
template <class T>
__global__ void __launch_bounds__(TPB) k_level_post21(Lev L, Lev C, const Scalars* S, int gate) {
  KSTART();
  const int q8 = blockIdx.x * blockDim.x + threadIdx.x;
  const int q = q8 >> 3, e = q8 & 7;
  const bool own = q < C.n;
  const int ci = own ? q % C.nx : 0, cj = own ? (q / C.nx) % C.ny : 0, ck = own ? q / (C.nx * C.ny) : 0;
  // the C cell this lane sweeps: 0 the parent, 1..6 its x-, x+, y-, y+, z-, z+ neighbours
  int pi = ci, pj = cj, pk = ck;
  if (e == 1) pi -= 1; else if (e == 2) pi += 1; else if (e == 3) pj -= 1;
  else if (e == 4) pj += 1; else if (e == 5) pk -= 1; else if (e == 6) pk += 1;
  const bool psweep = own && e < 7 && pi >= 0 && pi < C.nx && pj >= 0 && pj < C.ny && pk >= 0 && pk < C.nz;
  const LoadT<T> X2{as<T>(C.x2)};
  unsigned pcode = 0u;
  float pdg = 0.f, pr = 0.f, px2 = 0.f;
  Nb6 pb{};
  Ap6 pap{};
  int pc = 0;
  if (psweep) {
    pc = (pk * C.ny + pj) * C.nx + pi;
    pcode = C.code[pc];
    pdg = C.diag[pc];
    pr = Store<T>::ld(as<T>(C.r), pc);
    px2 = X2(pc);
    pb = level_nb(C, pi, pj, pk, pc, [&](int n, int, int, int) { return X2(n); });
    pap = level_ap6(C, pi, pj, pk);
  }
  // the child's own row
  const int i = 2 * ci + (e & 1), j = 2 * cj + ((e >> 1) & 1), k = 2 * ck + (e >> 2);
  const int c = (k * L.ny + j) * L.nx + i;
  const LoadT<T> X{as<T>(L.x)};
  unsigned code = 0u;
  float dg = 0.f, rc = 0.f, xc0 = 0.f;
  Nb6 b{};
  Ap6 ap{};
  if (own) {
    code = L.code[c];
    dg = L.diag[c];
    rc = Store<T>::ld(as<T>(L.r), c);
    xc0 = X(c);
    b = level_nb(L, i, j, k, c, [&](int n, int, int, int) { return X(n); });
    ap = level_ap6(L, i, j, k);
  }
  if (gate && !S->active) return;
  float xp = px2;  // C's final x at the lane's cell (k_level_post2)
  if (psweep && pdg > 0.f) xp += OMEGA * (pr - level_row_sel(C, pcode, px2, pb, pap)) / pdg;
  xp = Store<T>::rt(xp);
  const int lane0 = threadIdx.x & 24;
  float par[7];
#pragma unroll
  for (int a = 0; a < 7; ++a) par[a] = __shfl_sync(0xffffffffu, xp, lane0 + a);
  if (!own) return;
  // x + the parent's x at the child and its six neighbours (a neighbour across the parent's face
  // has the parent's neighbour as its parent)
  const float own_p = par[0];
  const float pxm = (e & 1) ? own_p : par[1], pxp = (e & 1) ? par[2] : own_p;
  const float pym = ((e >> 1) & 1) ? own_p : par[3], pyp = ((e >> 1) & 1) ? par[4] : own_p;
  const float pzm = (e >> 2) ? own_p : par[5], pzp = (e >> 2) ? par[6] : own_p;
  const float xc = xc0 + own_p;
  Nb6 v;
  v.xm = b.xm + pxm; v.xp = b.xp + pxp; v.ym = b.ym + pym; v.yp = b.yp + pyp; v.zm = b.zm + pzm; v.zp = b.zp + pzp;
  const int nxny = L.nx * L.ny;
  auto XP = [&](int n) {
    return n == c ? xc : n == c - 1 ? v.xm : n == c + 1 ? v.xp : n == c - L.nx ? v.ym : n == c + L.nx ? v.yp
         : n == c - nxny ? v.zm : v.zp;
  };
  float out = xc;
  if (dg > 0.f) out += OMEGA * (rc - level_row_sel(L, code, xc, v, ap)) / dg;
  Store<T>::st(as<T>(L.x2), c, out);
}

// One damped Jacobi sweep from codes (a large coarsest level's 8 sweeps); zero_in: from x = 0.
template <class T>
__global__ void __launch_bounds__(TPB) k_level_sweep_c(Lev L, const float* __restrict__ xin_, float* __restrict__ xout_,
                                                       int zero_in, const Scalars* S, int gate) {
  KSTART();
  if (gate && !S->active) return;
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= L.n) return;
  const T* xin = reinterpret_cast<const T*>(xin_);
  T* xout = reinterpret_cast<T*>(xout_);
  float dg = L.diag[c];
  const float rc = Store<T>::ld(as<T>(L.r), c);
  if (zero_in) { Store<T>::st(xout, c, dg > 0.f ? 0.f + OMEGA * (rc - 0.f) / dg : 0.f); return; }
  float xc = Store<T>::ld(xin, c);
  if (dg > 0.f) {
    int i = c % L.nx, t = c / L.nx, j = t % L.ny, k = t / L.ny;
    xc += OMEGA * (rc - level_row_code(L, L.code[c], i, j, k, c, LoadT<T>{xin})) / dg;
  }
  Store<T>::st(xout, c, xc);
}

// All levels from `first` to `last` in one CTA (coarse_cycle3 restricted to them): each phase is a
// block-strided loop, phases are separated by __syncthreads (global writes of a block are visible
// to the block after the barrier).  levels[first].r is already restricted; leaves levels[first].x.
constexpr int TAIL_THREADS = 1024;

// The threads of one CTA as a team: rank, size and barrier of the tail's strided phases.
struct BlockTeam {
  __device__ __forceinline__ int rank() const { return threadIdx.x; }
  __device__ __forceinline__ int size() const { return blockDim.x; }
  __device__ __forceinline__ void sync() const { __syncthreads(); }
};

template <class Team>
__device__ __forceinline__ void tail_sweep_t(const Team& tm, const Lev& L, const float* xin, float* xout, bool zero_in) {
  for (int c = tm.rank(); c < L.n; c += tm.size()) {
    float dg = L.diag[c];
    if (zero_in) { xout[c] = dg > 0.f ? 0.f + OMEGA * (L.r[c] - 0.f) / dg : 0.f; continue; }
    float xc = xin[c];
    if (dg > 0.f) {
      int i = c % L.nx, t = c / L.nx, j = t % L.ny, k = t / L.ny;
      xc += OMEGA * (L.r[c] - level_row_f(L, i, j, k, c, Load{xin})) / dg;
    }
    xout[c] = xc;
  }
  tm.sync();
}
__device__ __forceinline__ void tail_sweep(const Lev& L, const float* xin, float* xout, bool zero_in) {
  tail_sweep_t(BlockTeam{}, L, xin, xout, zero_in);
}

// coarse_cycle3 (delta3d_multigrid.rs:303-332) over levels first..last of Ls, in two halves: the way
// down (tail_down_t: the pre-sweeps of levels first..stop-1, eight sweeps on the coarsest, and each
// level's residual restricted to the next one while l < last) and the way up (tail_up_t:
// prolongation from level l + 1 and two post-sweeps, for l = from .. first).  A team can run a
// part of the hierarchy and another team the rest, in that order.
template <class Team>
__device__ __forceinline__ void tail_down_t(const Team& tm, const Lev* Ls, int first, int stop, int last) {
  for (int l = first; l < stop; ++l) {
    const Lev L = Ls[l];
    const int sweeps = l == last ? 8 : 2;  // COARSE_SWEEPS_3D, PRE_SWEEPS_3D
    for (int s = 0; s < sweeps; ++s)
      tail_sweep_t(tm, L, (s % 2 == 0) ? L.x : L.x2, (s % 2 == 0) ? L.x2 : L.x, s == 0);
    if (l < last) {
      const Lev C = Ls[l + 1];
      for (int q = tm.rank(); q < C.n; q += tm.size()) {
        int ci = q % C.nx, t = q / C.nx, cj = t % C.ny, ck = t / C.ny;
        float s = 0.f;
#pragma unroll
        for (int e = 0; e < 8; ++e) {
          int i = 2 * ci + (e & 1), j = 2 * cj + ((e >> 1) & 1), k = 2 * ck + (e >> 2);
          int c = (k * L.ny + j) * L.nx + i;
          float lx = L.kind[c] > 0.f ? level_row_f(L, i, j, k, c, Load{L.x}) : 0.f;
          s += L.r[c] - lx;
        }
        C.r[q] = 0.125f * s;
      }
      tm.sync();
    }
  }
}
template <class Team>
__device__ __forceinline__ void tail_up_t(const Team& tm, const Lev* Ls, int first, int from) {
  for (int l = from; l >= first; --l) {
    const Lev L = Ls[l];
    const Lev C = Ls[l + 1];
    for (int c = tm.rank(); c < L.n; c += tm.size()) {
      int i = c % L.nx, t = c / L.nx, j = t % L.ny, k = t / L.ny;
      L.x[c] += C.x[((k >> 1) * C.ny + (j >> 1)) * C.nx + (i >> 1)];
    }
    tm.sync();
    tail_sweep_t(tm, L, L.x, L.x2, false);
    tail_sweep_t(tm, L, L.x2, L.x, false);
  }
}
template <class Team>
__device__ __forceinline__ void tail_run_t(const Team& tm, const Lev* Ls, int first, int last) {
  tail_down_t(tm, Ls, first, last + 1, last);
  tail_up_t(tm, Ls, first, last - 1);
}
__device__ __forceinline__ void tail_run(const Lev* Ls, int first, int last) {
  tail_run_t(BlockTeam{}, Ls, first, last);
}

// The levels in global memory (fallback when they do not fit in shared memory).
__global__ void __launch_bounds__(TAIL_THREADS) k_coarse_tail(const Lev* __restrict__ T, int first, int last,
                                                              const Scalars* S, int gate) {
  KSTART();
  if (gate && !S->active) return;
  tail_run(T, first, last);
}

// Floats of shared memory a level takes in the shared-memory tail: five cell arrays and three face
// arrays, each rounded up to a multiple of four floats (16 bytes), as k_coarse_tail_smem carves them.
__host__ __device__ inline int round4(int c) { return (c + 3) & ~3; }
__host__ __device__ inline int tail_level_floats(int nx, int ny, int nz) {
  const int n = nx * ny * nz;
  return 5 * round4(n) + round4((nx + 1) * ny * nz) + round4(nx * (ny + 1) * nz) + round4(nx * ny * (nz + 1));
}

// The same with every level copied into dynamic shared memory first: geometry (kind, diag,
// apertures) of all tail levels and the restricted r of the first; only the first level's x goes
// back to global memory (the level above prolongates from it).
constexpr int MAX_TAIL_LEVELS = 12;
__global__ void __launch_bounds__(TAIL_THREADS) k_coarse_tail_smem(const Lev* __restrict__ T, int first, int last,
                                                                   const Scalars* S, int gate) {
  KSTART();
  if (gate && !S->active) return;
  extern __shared__ float4 tail_smem4[];
  float* sm = reinterpret_cast<float*>(tail_smem4);
  __shared__ Lev Ls[MAX_TAIL_LEVELS];
  if (threadIdx.x == 0) {
    int off = 0;
    for (int l = first; l <= last; ++l) {
      Lev L = T[l];
      const int n = L.n;
      const int nu = (L.nx + 1) * L.ny * L.nz, nv = L.nx * (L.ny + 1) * L.nz, nw = L.nx * L.ny * (L.nz + 1);
      auto take = [&](int cnt) { float* p = sm + off; off += round4(cnt); return p; };
      Lev M = L;
      M.kind = take(n); M.diag = take(n); M.r = take(n); M.x = take(n); M.x2 = take(n);
      M.ou = take(nu); M.ov = take(nv); M.ow = take(nw);
      Ls[l - first] = M;
    }
  }
  __syncthreads();
  for (int l = first; l <= last; ++l) {
    const Lev G = T[l];
    const Lev M = Ls[l - first];
    const int nu = (G.nx + 1) * G.ny * G.nz, nv = G.nx * (G.ny + 1) * G.nz, nw = G.nx * G.ny * (G.nz + 1);
    for (int q = threadIdx.x; q < G.n; q += blockDim.x) {
      M.kind[q] = G.kind[q];
      M.diag[q] = G.diag[q];
      if (l == first) M.r[q] = G.r[q];
    }
    for (int q = threadIdx.x; q < nu; q += blockDim.x) M.ou[q] = G.ou[q];
    for (int q = threadIdx.x; q < nv; q += blockDim.x) M.ov[q] = G.ov[q];
    for (int q = threadIdx.x; q < nw; q += blockDim.x) M.ow[q] = G.ow[q];
  }
  __syncthreads();
  tail_run(Ls, 0, last - first);
  const Lev G = T[first];
  const Lev M = Ls[0];
  for (int q = threadIdx.x; q < G.n; q += blockDim.x) G.x[q] = M.x[q];
}

// The coarse tail with one cell per thread.  Every tail level has at most TAIL_REG_THREADS cells;
// thread c owns cell c of each level and keeps its rows (code, apertures, diagonal) for all levels
// in registers, fetched once at the start with independent loads, so the phases below touch only
// shared memory: a sweep is six shared-memory reads, the row, one write and one barrier.  The
// phases and their arithmetic are those of coarse_cycle3 (delta3d_multigrid.rs:303-332): 2
// pre-sweeps, residual, 8-child mean, ..., 8 sweeps on the coarsest level, then prolongation and 2
// post-sweeps per level on the way up.
constexpr int TAIL_REG_THREADS = 512;
constexpr int TAIL_REG_LEVELS = 5;  // 40 KiB of static shared memory

struct TailRow {
  unsigned code;
  float a[6];
  float diag;
};

__device__ __forceinline__ TailRow tail_row(const Lev& L, int c) {
  TailRow w;
  w.code = 0;
  w.diag = 0.f;
#pragma unroll
  for (int f = 0; f < 6; ++f) w.a[f] = 0.f;
  if (c >= L.n) return w;
  // the six apertures are loaded with the code, not after it: every face index of a cell is valid
  const int i = c % L.nx, t = c / L.nx, j = t % L.ny, k = t / L.ny;
  const int fi[6] = {(k * L.ny + j) * (L.nx + 1) + i, (k * L.ny + j) * (L.nx + 1) + i + 1,
                     (k * (L.ny + 1) + j) * L.nx + i, (k * (L.ny + 1) + j + 1) * L.nx + i,
                     (k * L.ny + j) * L.nx + i, ((k + 1) * L.ny + j) * L.nx + i};
  float ap[6];
#pragma unroll
  for (int f = 0; f < 6; ++f) ap[f] = (f < 2 ? L.ou : (f < 4 ? L.ov : L.ow))[fi[f]];
  w.code = L.code[c];
  w.diag = L.diag[c];
  const bool unit = w.code & RC_UNIT;
#pragma unroll
  for (int f = 0; f < 6; ++f)
    if (face_state(w.code, f)) w.a[f] = unit ? 1.f : ap[f];
  return w;
}

// row_sums at cell c of a level with dims (nx, ny), the neighbours' values read from X (shared
// memory); the terms are added in face order x-, x+, y-, y+, z-, z+.  As level_row_sel: the six
// reads are issued together (indices clamped into the array; a face leading out of the level has
// state 0 and its value is unused) and the terms selected, not branched on.
__device__ __forceinline__ float tail_rowsum(const TailRow& w, int c, int nx, int nxny, float pc, const float* X,
                                             float inv) {
  const int mm[6] = {c - 1, c + 1, c - nx, c + nx, c - nxny, c + nxny};
  float v[6];
#pragma unroll
  for (int f = 0; f < 6; ++f) v[f] = X[min(max(mm[f], 0), TAIL_REG_THREADS - 1)];
  float acc = 0.f;
#pragma unroll
  for (int f = 0; f < 6; ++f) {
    const unsigned st = face_state(w.code, f);
    const float t1 = w.a[f] * (pc - v[f]);
    const float t2 = 2.f * w.a[f] * pc;
    acc += st == 1u ? t1 : (st == 2u ? t2 : 0.f);
  }
  return acc * inv;
}

// The tail's levels, passed by value: the kernel reads them from its parameters, not memory.
struct TailLevs {
  Lev L[TAIL_REG_LEVELS];
};

template <class ST>
__global__ void __launch_bounds__(TAIL_REG_THREADS) k_coarse_tail_reg(const TailLevs Ls_, int nl, const Scalars* S,
                                                                     int gate) {
  KSTART();
  // per level: XA, XB (sweep ping-pong), XF (final x of the level), R (right-hand side)
  __shared__ float XA[TAIL_REG_LEVELS][TAIL_REG_THREADS];
  __shared__ float XB[TAIL_REG_LEVELS][TAIL_REG_THREADS];
  __shared__ float XF[TAIL_REG_LEVELS][TAIL_REG_THREADS];
  __shared__ float R[TAIL_REG_LEVELS][TAIL_REG_THREADS];
  const Lev (&Ls)[TAIL_REG_LEVELS] = Ls_.L;
  const int c = threadIdx.x;
  // every row of every level, and the right-hand side of the first, in one round of loads issued
  // before the loop's gate is read (the gate is checked before anything is written to memory)
  TailRow w[TAIL_REG_LEVELS];
#pragma unroll
  for (int l = 0; l < TAIL_REG_LEVELS; ++l) {
    if (l < nl) w[l] = tail_row(Ls[l], c);
  }
  const float r0 = c < Ls[0].n ? Store<ST>::ld(as<ST>(Ls[0].r), c) : 0.f;
  if (gate && !S->active) return;
  if (c < Ls[0].n) R[0][c] = r0;
  __syncthreads();
  // descent
#pragma unroll
  for (int l = 0; l < TAIL_REG_LEVELS; ++l) {
    if (l < nl) {
      const Lev& L = Ls[l];
      const bool own = c < L.n;
      const int nx = L.nx, nxny = L.nx * L.ny;
      const float inv = L.inv;
      const float r = own ? R[l][c] : 0.f;
      const int sweeps = l == nl - 1 ? 8 : 2;  // COARSE_SWEEPS_3D, PRE_SWEEPS_3D
      float x = 0.f;
      for (int s = 0; s < sweeps; ++s) {
        float* out = (s & 1) ? XB[l] : XA[l];
        const float* in = (s & 1) ? XA[l] : XB[l];
        float xn = x;
        if (own) {
          if (s == 0) xn = w[l].diag > 0.f ? 0.f + OMEGA * (r - 0.f) / w[l].diag : 0.f;
          else xn = jacobi_sel(x, r, tail_rowsum(w[l], c, nx, nxny, x, in, inv), w[l].diag);
          out[c] = xn;
        }
        __syncthreads();
        x = xn;
      }
      if (own) XF[l][c] = x;
      if (l < nl - 1) {
        // residual t = r - L x (0 on inactive rows), then the 8-child mean into the next level
        const float* xs = ((sweeps - 1) & 1) ? XB[l] : XA[l];
        float tv = 0.f;
        if (own) tv = r - ((w[l].code & RC_WET) ? tail_rowsum(w[l], c, nx, nxny, x, xs, inv) : 0.f);
        __syncthreads();
        if (own) XA[l][c] = tv;
        __syncthreads();
        const Lev& C = Ls[l + 1];
        if (c < C.n) {
          int ci = c % C.nx, t = c / C.nx, cj = t % C.ny, ck = t / C.ny;
          float sum = 0.f;
#pragma unroll
          for (int e = 0; e < 8; ++e) {
            int i = 2 * ci + (e & 1), j = 2 * cj + ((e >> 1) & 1), k = 2 * ck + (e >> 2);
            sum += XA[l][(k * L.ny + j) * L.nx + i];
          }
          R[l + 1][c] = 0.125f * sum;
        }
        __syncthreads();
      }
    }
  }
  // ascent
#pragma unroll
  for (int l = TAIL_REG_LEVELS - 2; l >= 0; --l) {
    if (l <= nl - 2) {
      const Lev& L = Ls[l];
      const Lev& C = Ls[l + 1];
      const bool own = c < L.n;
      const int nx = L.nx, nxny = L.nx * L.ny;
      const float inv = L.inv;
      const float r = own ? R[l][c] : 0.f;
      float x = 0.f;
      if (own) {
        int i = c % L.nx, t = c / L.nx, j = t % L.ny, k = t / L.ny;
        x = XF[l][c] + XF[l + 1][((k >> 1) * C.ny + (j >> 1)) * C.nx + (i >> 1)];
        XB[l][c] = x;
      }
      __syncthreads();
      for (int s = 0; s < 2; ++s) {  // POST_SWEEPS_3D
        float* out = (s & 1) ? XB[l] : XA[l];
        const float* in = (s & 1) ? XA[l] : XB[l];
        float xn = x;
        if (own) xn = jacobi_sel(x, r, tail_rowsum(w[l], c, nx, nxny, x, in, inv), w[l].diag);
        if (own) out[c] = xn;
        __syncthreads();
        x = xn;
      }
      if (own) XF[l][c] = x;
      __syncthreads();
    }
  }
  if (c < Ls[0].n) Store<ST>::st(as<ST>(Ls[0].x), c, XF[0][c]);
}

// ------------------------------------------------------------------------------------------------
// The WHILE node of the inner loop repeats its body (two iterations) while this sets 1.  Each
// iteration that runs advances S->it, so the loop ends within max_iters iterations; as a guard
// independent of that logic, the body never runs more than max_iters + 2 times (status 100).
__global__ void k_loop_cond(cudaGraphConditionalHandle handle, Scalars* S) {
  KSTART();
  unsigned runs = ++S->body_runs;
  bool go = S->active != 0;
  if (go && runs > S->max_iters + 2u) { S->active = 0; S->status = 100; go = false; }
  cudaGraphSetConditional(handle, go ? 1u : 0u);
}

// ------------------------------------------------------------------------------------------------
// Set-up reductions with the in-kernel finish.

// One row of rhs_mobile3 (delta3d_mobile.rs:215-241): rhs and prec of cell c (the divergence in
// rhs is replaced by the right-hand side), its row code into codes and p = 0 on a dry cell when
// those are not null; returns b.
__device__ __forceinline__ float rhs_b2_at(const Geo& g, float scale, float* __restrict__ rhs, float* __restrict__ prec,
                                           unsigned short* __restrict__ codes, float* __restrict__ pdry, int c) {
  int i, j, k; cell_ijk(g, c, i, j, k);
  if (!wet3(g, i, j, k)) {
    rhs[c] = 0.f; prec[c] = 0.f;
    if (codes) codes[c] = 0;
    if (pdry) pdry[c] = 0.f;
    return 0.f;
  }
  RowE row[6]; mobile_row(g, i, j, k, row);
  float b = scale * rhs[c];
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
  if (codes) codes[c] = (unsigned short)row_code_of(row);
  return b;
}

// rhs_mobile3 (delta3d_mobile.rs:215-241) with b.b (FIN_B2) when `reduce`.
// With `codes` not null, the same pass also writes each cell's row code (row_code_of the same
// row; 0 for a dry cell); with `pdry` not null it zeroes that pressure on the dry cells.
template <int MODE>
__global__ void __launch_bounds__(TPB, FD3_SETUP_MINB) k_rhs_b2(Geo g, float scale, float* __restrict__ rhs, float* __restrict__ prec,
                                                Red red, Scalars* S, int reduce, unsigned short* __restrict__ codes,
                                                float* __restrict__ pdry) {
  KSTART();
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  const float b = c < g.n ? rhs_b2_at(g, scale, rhs, prec, codes, pdry, c) : 0.f;
  if (!reduce) return;
  if (__syncthreads_or(c < g.n && b != 0.f) && threadIdx.x == 0) atomicOr(&S->any_nonzero, 1);
  reduce_finish<MODE>(Acc<MODE>::prod(b, b), c, g.n, red, S, FIN_B2);
}

// res = rhs - A p with res.res (FIN_RR0 or FIN_ACTUAL), from the row codes.
template <int MODE>
__global__ void __launch_bounds__(TPB) k_residual_c(Geo g, const unsigned short* __restrict__ codes,
                                                    const float* __restrict__ p, const float* __restrict__ rhs,
                                                    float* __restrict__ res, Red red, Scalars* S, int op) {
  KSTART();
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  float r = 0.f;
  if (c < g.n) {
    unsigned code = codes[c];
    float ap = 0.f;
    if (code & RC_WET) { int i, j, k; cell_ijk(g, c, i, j, k); ap = apply_code(g, code, i, j, k, c, Load{p}); }
    r = rhs[c] - ap;
    res[c] = r;
  }
  if (__syncthreads_or(c < g.n && r != 0.f) && threadIdx.x == 0) atomicOr(&S->any_nonzero, 1);
  reduce_finish<MODE>(Acc<MODE>::prod(r, r), c, g.n, red, S, op);
}

// Loop start: the host's view of the loop state; a pending NotFinite keeps the loop closed.
// The first inner loop of a projection started from the device's own scalars (f64 reductions): the
// host's test before it (b2 > 0, rr above tol b2, iterations left; delta3d_mobile.rs:513-516) is made
// here, so the set-up, the loop and the outer checks go out without a host round trip between them.
__global__ void k_loop_start_dev(Scalars* S, unsigned max_iters) {
  KSTART();
  const double tolb2 = 1e-12 * S->b2;
  S->tolb2 = tolb2;
  S->phys = (double)INFINITY;
  S->it = 0;
  S->max_iters = max_iters;
  S->brk = 0;
  S->body_runs = 0;
  S->active = (S->status == 0 && S->b2 > 0.0 && S->rr > tolb2 && max_iters > 0u) ? 1 : 0;
}

__global__ void k_loop_start(Scalars* S, double rr, double tolb2, double phys, unsigned it, unsigned max_iters) {
  KSTART();
  S->rr = rr;
  S->tolb2 = tolb2;
  S->phys = phys;
  S->it = it;
  S->max_iters = max_iters;
  S->brk = 0;
  S->body_runs = 0;
  S->active = S->status ? 0 : 1;
}

}  // namespace fd3
