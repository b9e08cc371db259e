// The linear (fixed-lid) path of Volume3 (delta3d.rs:697-1357): the same PCG machinery as the
// mobile projection, on the operator with Neumann walls and bottom and a homogeneous Dirichlet lid
// half a cell above the top layer, every non-solid cell a row.
//
// The rows are encoded in the mobile projection's 16-bit codes, so the PCG kernels of fd3_fast.cuh
// run unchanged: face state 1 is an open face onto a non-solid neighbour, state 2 the lid (the
// only ghost this operator has), whose term `2 a p_c` is selected by Geo::linear inside apply_code.
// Plain CG (the flat bottom, or a cut one with ny == 1 or the preconditioner off) runs as the
// Jacobi-PCG with prec = 1: z = 1 * r is r, r.z is r.r to the bit, and z + beta d is r + beta d,
// so its iterates are those of project's CG branch (delta3d.rs:1123-1128).
#pragma once

#include "fd3_fast.cuh"

namespace fd3 {

// Row codes of apply / apply_cut (delta3d.rs:721-744, 771-802).
__global__ void k_row_codes_linear(Geo g, unsigned short* __restrict__ codes) {
  KSTART();
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= g.n) return;
  int i, j, k; cell_ijk(g, c, i, j, k);
  unsigned code = 0;
  if (!solid3(g, c)) {
    const int nxny = g.nx * g.ny;
    code = RC_WET;
    bool unit = true;
    float a[6] = {open3(g, 0, fu(g, i, j, k)), open3(g, 0, fu(g, i + 1, j, k)), open3(g, 1, fv(g, i, j, k)),
                  open3(g, 1, fv(g, i, j + 1, k)), open3(g, 2, fw(g, i, j, k)), open3(g, 2, fw(g, i, j, k + 1))};
    bool has[6] = {i > 0, i + 1 < g.nx, j > 0, j + 1 < g.ny, k > 0, k + 1 < g.nz};
    int m[6] = {c - 1, c + 1, c - g.nx, c + g.nx, c - nxny, c + nxny};
#pragma unroll
    for (int f = 0; f < 6; ++f) {
      unsigned st = 0;
      if (a[f] != 0.f) {
        if (has[f]) st = solid3(g, m[f]) ? 0u : 1u;
        else if (f == 5) st = 2u;  // the lid
      }
      code |= st << (1 + 2 * f);
      if (st && a[f] != 1.f) unit = false;
    }
    if (unit) code |= RC_UNIT;
  }
  codes[c] = (unsigned short)code;
}

// lid (delta3d.rs:697-715), fully open.
__device__ __forceinline__ float lid_value(const Geo& g, int i, int j) {
  const int cc = j * g.nx + i;
  return g.rho_g * ((__ldg(g.eta + cc) - (float)g.nz * g.dx) - __ldg(g.rof + cc));
}

// The right-hand side of project (delta3d.rs:1066-1086), the Jacobi diagonal of prec_cut
// (delta3d.rs:557-591) or 1 for plain CG, and b.b.
template <int MODE>
__global__ void __launch_bounds__(TPB) k_rhs_linear(Geo g, float scale, int jacobi, float* __restrict__ rhs,
                                                    float* __restrict__ prec, Red red, Scalars* S) {
  KSTART();
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  float b = 0.f;
  if (c < g.n) {
    int i, j, k; cell_ijk(g, c, i, j, k);
    b = scale * rhs[c];
    float m = 1.f;
    if (g.cut) {
      const float fr = __ldg(g.frac + c);
      if (fr == 0.f) b = 0.f;
      else if (k + 1 == g.nz) {
        const float a = __ldg(g.ow + fw(g, i, j, k + 1));
        if (a > 0.f) b += 2.f * a * lid_value(g, i, j) * g.inv;
      }
      if (jacobi) {
        if (fr == 0.f) m = 0.f;
        else {
          const int nxny = g.nx * g.ny;
          float a[6] = {__ldg(g.ou + fu(g, i, j, k)), __ldg(g.ou + fu(g, i + 1, j, k)), __ldg(g.ov + fv(g, i, j, k)),
                        __ldg(g.ov + fv(g, i, j + 1, k)), __ldg(g.ow + fw(g, i, j, k)), __ldg(g.ow + fw(g, i, j, k + 1))};
          bool has[6] = {i > 0, i + 1 < g.nx, j > 0, j + 1 < g.ny, k > 0, k + 1 < g.nz};
          int nb[6] = {c - 1, c + 1, c - g.nx, c + g.nx, c - nxny, c + nxny};
          float diag = 0.f;
#pragma unroll
          for (int f = 0; f < 6; ++f) {
            if (a[f] == 0.f) continue;
            if (has[f]) { if (__ldg(g.frac + nb[f]) > 0.f) diag += a[f]; }
            else if (f == 5) diag += 2.f * a[f];
          }
          m = diag > 0.f ? 1.f / (diag * g.inv) : 0.f;
        }
      }
    } else if (k + 1 == g.nz) {
      b += 2.f * lid_value(g, i, j) * g.inv;
    }
    rhs[c] = b;
    prec[c] = m;
  }
  if (__syncthreads_or(c < g.n && b != 0.f) && threadIdx.x == 0) atomicOr(&S->any_nonzero, 1);
  reduce_finish<MODE>(Acc<MODE>::prod(b, b), c, g.n, red, S, FIN_B2);
}

// correct (delta3d.rs:949-987) and correct_cut (:989-1038): u and v faces.
__global__ void k_correct_linear_uv(Geo g, float k1, const float* __restrict__ p, const float* __restrict__ us,
                                    const float* __restrict__ vs, float* __restrict__ u, float* __restrict__ v) {
  KSTART();
  int nu = (g.nx + 1) * g.ny * g.nz, nv = g.nx * (g.ny + 1) * g.nz;
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q < nu) {
    int f = q, i = f % (g.nx + 1), t = f / (g.nx + 1), j = t % g.ny, k = t / g.ny;
    float val = us[f];
    if (i > 0 && i < g.nx) {
      int l = (k * g.ny + j) * g.nx + i - 1, r = l + 1;
      if (!g.cut || (__ldg(g.ou + f) != 0.f && __ldg(g.frac + l) > 0.f && __ldg(g.frac + r) > 0.f))
        val -= k1 * (p[r] - p[l]) / g.dx;
    }
    u[f] = val;
    return;
  }
  q -= nu;
  if (q < nv) {
    int f = q, i = f % g.nx, t = f / g.nx, j = t % (g.ny + 1), k = t / (g.ny + 1);
    float val = vs[f];
    if (j > 0 && j < g.ny) {
      int a = (k * g.ny + j - 1) * g.nx + i, b = a + g.nx;
      if (!g.cut || (__ldg(g.ov + f) != 0.f && __ldg(g.frac + a) > 0.f && __ldg(g.frac + b) > 0.f))
        val -= k1 * (p[b] - p[a]) / g.dx;
    }
    v[f] = val;
  }
}

// w faces, the lid at half a cell (delta3d.rs:971-985, 1019-1036).
__global__ void k_correct_linear_w(Geo g, float k1, const float* __restrict__ p, const float* __restrict__ ws,
                                   float* __restrict__ w) {
  KSTART();
  int nw = g.nx * g.ny * (g.nz + 1);
  int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= nw) return;
  int i = f % g.nx, t = f / g.nx, j = t % g.ny, k = t / g.ny;
  float val = ws[f];
  if (k >= 1) {
    int below = ((k - 1) * g.ny + j) * g.nx + i;
    bool open = !g.cut || (__ldg(g.ow + f) != 0.f && __ldg(g.frac + below) > 0.f);
    if (open) {
      if (k < g.nz) {
        int above = below + g.nx * g.ny;
        if (!g.cut || __ldg(g.frac + above) > 0.f) val -= k1 * (p[above] - p[below]) / g.dx;
      } else {
        val -= k1 * (lid_value(g, i, j) - p[below]) / (0.5f * g.dx);
      }
    }
  }
  w[f] = val;
}

// max |div u| over every cell (divergence_metric, delta3d.rs:1043-1052) into S->fmax[0] and [1].
__global__ void k_div_metric_linear(Geo g, const float* __restrict__ u, const float* __restrict__ v,
                                    const float* __restrict__ w, Scalars* S) {
  KSTART();
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  float d = 0.f;
  if (c < g.n) {
    int i, j, k; cell_ijk(g, c, i, j, k);
    float dv = 0.f;
    if (g.cut) {
      if (__ldg(g.frac + c) != 0.f) {
        float fl = __ldg(g.ou + fu(g, i, j, k)) * u[fu(g, i, j, k)];
        float fr = __ldg(g.ou + fu(g, i + 1, j, k)) * u[fu(g, i + 1, j, k)];
        float ff = __ldg(g.ov + fv(g, i, j, k)) * v[fv(g, i, j, k)];
        float fk = __ldg(g.ov + fv(g, i, j + 1, k)) * v[fv(g, i, j + 1, k)];
        float fb = __ldg(g.ow + fw(g, i, j, k)) * w[fw(g, i, j, k)];
        float ft = __ldg(g.ow + fw(g, i, j, k + 1)) * w[fw(g, i, j, k + 1)];
        dv = ((fr - fl + ft - fb) + (fk - ff)) / g.dx;
        if (g.wall) dv = dv + wall_flux(g, i, j, k);
      }
    } else {
      float fl = u[fu(g, i, j, k)], fr = u[fu(g, i + 1, j, k)];
      float ff = v[fv(g, i, j, k)], fk = v[fv(g, i, j + 1, k)];
      float fb = w[fw(g, i, j, k)], ft = w[fw(g, i, j, k + 1)];
      dv = ((fr - fl + ft - fb) + (fk - ff)) / g.dx;
    }
    d = fabsf(dv);
  }
  block_fmax2_atomic(d, d, &S->fmax[0], &S->fmax[1]);
}

// backward_error (delta3d.rs:881-907) and backward_error_cut (:909-945) into S->fmax[3].
__global__ void k_backward_error_linear(Geo g, const float* __restrict__ p, const float* __restrict__ rhs,
                                        const float* __restrict__ res, Scalars* S) {
  KSTART();
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  float worst = 0.f;
  if (c < g.n && !solid3(g, c)) {
    int i, j, k; cell_ijk(g, c, i, j, k);
    const int nxny = g.nx * g.ny;
    const float pc = fabsf(p[c]);
    float acc = 0.f;
    bool has[6] = {i > 0, i + 1 < g.nx, j > 0, j + 1 < g.ny, k > 0, k + 1 < g.nz};
    int nb[6] = {c - 1, c + 1, c - g.nx, c + g.nx, c - nxny, c + nxny};
    if (!g.cut) {
#pragma unroll
      for (int f = 0; f < 6; ++f) {
        if (has[f]) acc += pc + fabsf(p[nb[f]]);
        else if (f == 5) acc += pc * 2.f;
      }
    } else {
      float a[6] = {__ldg(g.ou + fu(g, i, j, k)), __ldg(g.ou + fu(g, i + 1, j, k)), __ldg(g.ov + fv(g, i, j, k)),
                    __ldg(g.ov + fv(g, i, j + 1, k)), __ldg(g.ow + fw(g, i, j, k)), __ldg(g.ow + fw(g, i, j, k + 1))};
#pragma unroll
      for (int f = 0; f < 6; ++f) {
        if (a[f] == 0.f) continue;
        if (has[f]) { if (__ldg(g.frac + nb[f]) > 0.f) acc += a[f] * (pc + fabsf(p[nb[f]])); }
        else if (f == 5) acc += a[f] * pc * 2.f;
      }
    }
    float scale = fabsf(rhs[c]) + acc * g.inv;
    if (scale > 0.f) worst = fabsf(res[c]) / scale;
  }
  block_fmax2_atomic(worst, 0.f, &S->fmax[3], nullptr);
}

// The heights carried by the column fluxes (delta3d.rs:1305-1336): each column sums its four side
// faces from the bottom layer up, in the reference's order (the same sums its neighbours form for
// the shared faces), then the compensated update, the x part before the y part.
__device__ __forceinline__ float column_flux(const Geo& g, const float* __restrict__ vel, const float* __restrict__ ap,
                                             int f0, int stride) {
  float q = 0.f;
  for (int k = 0; k < g.nz; ++k) {
    const int f = f0 + k * stride;
    if (g.cut) q += __ldg(ap + f) * vel[f] * g.dx;
    else q += vel[f] * g.dx;
  }
  return q;
}
__global__ void k_linear_transport(Geo g, float transport, const float* __restrict__ u, const float* __restrict__ v,
                                   float* __restrict__ eta, float* __restrict__ rof) {
  KSTART();
  int cc = blockIdx.x * blockDim.x + threadIdx.x;
  if (cc >= g.nx * g.ny) return;
  const int i = cc % g.nx, j = cc / g.nx;
  const int su = (g.nx + 1) * g.ny, sv = g.nx * (g.ny + 1);
  const float left = column_flux(g, u, g.ou, j * (g.nx + 1) + i, su);
  const float right = column_flux(g, u, g.ou, j * (g.nx + 1) + i + 1, su);
  const float front = column_flux(g, v, g.ov, j * g.nx + i, sv);
  const float back = column_flux(g, v, g.ov, (j + 1) * g.nx + i, sv);
  const float e = eta[cc];
  const float increment = -transport * ((right - left) + (back - front)) - rof[cc];
  const float height = e + increment;
  rof[cc] = (height - e) - increment;
  eta[cc] = height;
}

// 1 where a lid face is not fully open (the linear step's refusal, delta3d.rs:1261-1268).
__global__ void k_lid_open(Geo g, int* flag) {
  int cc = blockIdx.x * blockDim.x + threadIdx.x;
  if (cc < g.nx * g.ny && g.cut && __ldg(g.ow + g.nz * g.nx * g.ny + cc) != 1.f) atomicOr(flag, 1);
}

}  // namespace fd3
