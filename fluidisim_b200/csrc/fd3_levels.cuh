// The level change (delta3d_levels.rs): a volume receives the state of another volume that covers
// the same window at another dx.  One thread per destination column (the surface, by overlap of a
// conservative linear reconstruction of each source column) and one per destination face (the
// velocity, trilinear on the source's staggered grid, averaged over n x n sub-faces when the
// destination is coarser).  Everything is f64 in the reference's order; the library is built with
// --fmad=false, so no product is fused into a sum.
#pragma once

#include "fd3_kernels.cuh"

namespace fd3 {

// The source volume, read only.
struct LevelSrc {
  int nx, ny, nz;
  float dx, rest;
  const float* eta;
  const float* rof;
  const float* u;
  const float* v;
  const float* w;
  const unsigned char* act;  // sparse column set, null without one
};

__device__ __forceinline__ bool lv_active(const LevelSrc& s, int i, int j) { return !s.act || s.act[j * s.nx + i] != 0; }

// The compensated height of column (i, j) in f64 (delta3d_levels.rs:71-74).
__device__ __forceinline__ double lv_comp(const LevelSrc& s, int i, int j) {
  const int c = j * s.nx + i;
  return (double)s.eta[c] - (double)s.rof[c];
}

// surface_slope (delta3d_levels.rs:76-90): centred inside, one-sided at the box's or the set's edge.
__device__ double lv_slope(const LevelSrc& s, int i, int j, int axis) {
  const int n = axis == 0 ? s.nx : s.ny, k = axis == 0 ? i : j;
  if (n < 2) return 0.0;
  auto inside = [&](int m) { return axis == 0 ? lv_active(s, m, j) : lv_active(s, i, m); };
  auto at = [&](int m) { return axis == 0 ? lv_comp(s, m, j) : lv_comp(s, i, m); };
  const int lo = k > 0 && inside(k - 1) ? k - 1 : k;
  const int hi = k + 1 < n && inside(k + 1) ? k + 1 : k;
  if (hi == lo) return 0.0;
  return (at(hi) - at(lo)) / ((double)(hi - lo) * (double)s.dx);
}

// surface_twist (delta3d_levels.rs:95-107): the four-point cross difference, 0 at an edge.
__device__ double lv_twist(const LevelSrc& s, int i, int j) {
  if (i == 0 || j == 0 || i + 1 >= s.nx || j + 1 >= s.ny) return 0.0;
  if (!lv_active(s, i - 1, j - 1) || !lv_active(s, i + 1, j - 1) || !lv_active(s, i - 1, j + 1) ||
      !lv_active(s, i + 1, j + 1))
    return 0.0;
  const double d = (double)s.dx;
  return (lv_comp(s, i + 1, j + 1) - lv_comp(s, i + 1, j - 1) - lv_comp(s, i - 1, j + 1) + lv_comp(s, i - 1, j - 1)) /
         (4.0 * d * d);
}

// resample_surface (delta3d_levels.rs:109-155), one thread per destination column.
__global__ void k_resample_surface(LevelSrc s, int nx, int ny, float dxf, float rest,
                                   const unsigned char* __restrict__ act, float* __restrict__ eta,
                                   float* __restrict__ rof) {
  KSTART();
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nx * ny) return;
  const int i = c % nx, j = c / nx;
  if (act && act[c] == 0) {  // a column outside the destination's set stays at rest
    eta[c] = rest;
    rof[c] = 0.f;
    return;
  }
  const double dd = (double)dxf;
  const double sx = (double)nx * dd / (double)s.nx, sy = (double)ny * dd / (double)s.ny;
  const double y0 = (double)j * dd, y1 = (double)(j + 1) * dd;
  const double x0 = (double)i * dd, x1 = (double)(i + 1) * dd;
  const int i0 = (int)floor(x0 / sx), i1 = min((int)ceil(x1 / sx), s.nx);
  const int j0 = (int)floor(y0 / sy), j1 = min((int)ceil(y1 / sy), s.ny);
  double total = 0.0;
  for (int sj = j0; sj < j1; ++sj) {
    const double ya = fmax(y0, (double)sj * sy), yb = fmin(y1, (double)(sj + 1) * sy);
    if (yb <= ya) continue;
    for (int si = i0; si < i1; ++si) {
      const double xa = fmax(x0, (double)si * sx), xb = fmin(x1, (double)(si + 1) * sx);
      if (xb <= xa) continue;
      const double area = (xb - xa) * (yb - ya);
      const double cx = 0.5 * (xa + xb) - ((double)si + 0.5) * sx;
      const double cy = 0.5 * (ya + yb) - ((double)sj + 0.5) * sy;
      double h;
      if (lv_active(s, si, sj))
        h = lv_comp(s, si, sj) + lv_slope(s, si, sj, 0) * cx + lv_slope(s, si, sj, 1) * cy + lv_twist(s, si, sj) * cx * cy;
      else
        h = (double)s.rest;
      total += area * h;
    }
  }
  const double h = total / (dd * dd);
  const float e = (float)h;
  eta[c] = e;
  rof[c] = (float)((double)e - h);
}

__device__ __forceinline__ float lv_velocity(const LevelSrc& s, int axis, const int p[3]) {
  if (axis == 0) return s.u[(p[2] * s.ny + p[1]) * (s.nx + 1) + p[0]];
  if (axis == 1) return s.v[(p[2] * (s.ny + 1) + p[1]) * s.nx + p[0]];
  return s.w[(p[2] * s.ny + p[1]) * s.nx + p[0]];
}

// sparse_outside3 (delta3d_sparse.rs:307-319) of the source's set.
__device__ __forceinline__ bool lv_outside(const LevelSrc& s, int axis, int i, int j) {
  if (axis == 0) return !((i > 0 && lv_active(s, i - 1, j)) || (i < s.nx && lv_active(s, i, j)));
  if (axis == 1) return !((j > 0 && lv_active(s, i, j - 1)) || (j < s.ny && lv_active(s, i, j)));
  return !lv_active(s, i, j);
}

// staggered_at (delta3d_levels.rs:159-200) and, with a sparse source, staggered_in_set (:204-245):
// trilinear on the staggered grid, indices clamped; in a set, a corner outside the set's grid takes,
// axis by axis, its neighbour's value inside it.
__device__ float lv_staggered(const LevelSrc& s, int axis, const double rel[3]) {
  const int dims[3] = {s.nx + (axis == 0), s.ny + (axis == 1), s.nz + (axis == 2)};
  const int cells[3] = {s.nx, s.ny, s.nz};
  int base[3];
  double frac[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    double f = rel[a] * (double)cells[a] - (a == axis ? 0.0 : 0.5);
    const double top = (double)(dims[a] - 1);
    f = fmin(fmax(f, 0.0), top);
    const int b = min((int)floor(f), dims[a] >= 2 ? dims[a] - 2 : 0);
    base[a] = b;
    frac[a] = dims[a] < 2 ? 0.0 : f - (double)b;
  }
  double values[8];
  bool outside[8];
#pragma unroll
  for (int corner = 0; corner < 8; ++corner) {
    int p[3] = {base[0], base[1], base[2]};
#pragma unroll
    for (int a = 0; a < 3; ++a)
      if (((corner >> a) & 1) && dims[a] >= 2) p[a] += 1;
    values[corner] = (double)lv_velocity(s, axis, p);
    outside[corner] = s.act ? lv_outside(s, axis, p[0], p[1]) : false;
  }
  if (s.act) {
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      if (dims[a] < 2) continue;
#pragma unroll
      for (int corner = 0; corner < 8; ++corner) {
        if ((corner >> a) & 1) continue;
        const int up = corner | (1 << a);
        if (outside[corner] && !outside[up]) { values[corner] = values[up]; outside[corner] = false; }
        else if (outside[up] && !outside[corner]) { values[up] = values[corner]; outside[up] = false; }
      }
    }
  }
  double acc = 0.0;
#pragma unroll
  for (int corner = 0; corner < 8; ++corner) {
    double weight = 1.0;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const bool up = (corner >> a) & 1;
      if (dims[a] < 2) { if (up) weight = 0.0; continue; }
      weight *= up ? frac[a] : 1.0 - frac[a];
    }
    if (weight != 0.0) acc += weight * values[corner];
  }
  return (float)acc;
}

// resample_faces (delta3d_levels.rs:249-288), one thread per destination face; `n` sub-faces per
// direction of the face's plane.
__global__ void k_resample_faces(LevelSrc s, int nx, int ny, int nz, int n, float* __restrict__ u,
                                 float* __restrict__ v, float* __restrict__ w) {
  KSTART();
  const long long nu = (long long)(nx + 1) * ny * nz, nv = (long long)nx * (ny + 1) * nz,
                  nw = (long long)nx * ny * (nz + 1);
  long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  int axis;
  if (q < nu) axis = 0;
  else if ((q -= nu) < nv) axis = 1;
  else if ((q -= nv) < nw) axis = 2;
  else return;
  const int dims[3] = {nx + (axis == 0), ny + (axis == 1), nz + (axis == 2)};
  const int p[3] = {(int)(q % dims[0]), (int)((q / dims[0]) % dims[1]), (int)(q / ((long long)dims[0] * dims[1]))};
  const double cells[3] = {(double)nx, (double)ny, (double)nz};
  double centre[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) centre[a] = ((double)p[a] + (a == axis ? 0.0 : 0.5)) / cells[a];
  const int t1 = (axis + 1) % 3, t2 = (axis + 2) % 3;
  double acc = 0.0;
  for (int a = 0; a < n; ++a)
    for (int b = 0; b < n; ++b) {
      double r[3] = {centre[0], centre[1], centre[2]};
      r[t1] += (((double)a + 0.5) / (double)n - 0.5) / cells[t1];
      r[t2] += (((double)b + 0.5) / (double)n - 0.5) / cells[t2];
      acc += (double)lv_staggered(s, axis, r);
    }
  const float val = (float)(acc / (double)(n * n));
  if (axis == 0) u[q] = val;
  else if (axis == 1) v[q] = val;
  else w[q] = val;
}

}  // namespace fd3
