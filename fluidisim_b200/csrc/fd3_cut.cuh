// Cut-cell geometry on the GPU: the bottom cut and the solid cut of the reference
// (code/water-core/src/delta3d_cut.rs; the 2D helpers cut_fraction/open_below of
// delta_projection.rs:795-827).  Same f32 arithmetic for the bottom, same f64 arithmetic for the
// solid, same sort order (Rust's total_cmp), so the fractions and apertures are bit-identical.
// One thread per cell, face or column; run once per geometry at configure time.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

namespace fd3 {

__host__ __device__ __forceinline__ int fbits(float a) {
#ifdef __CUDA_ARCH__
  return __float_as_int(a);
#else
  int x;
  memcpy(&x, &a, 4);
  return x;
#endif
}
__host__ __device__ __forceinline__ long long dbits(double a) {
#ifdef __CUDA_ARCH__
  return __double_as_longlong(a);
#else
  long long x;
  memcpy(&x, &a, 8);
  return x;
#endif
}

__host__ __device__ __forceinline__ bool total_less(float a, float b) {
  int x = fbits(a), y = fbits(b);
  x ^= (int)(((unsigned)(x >> 31)) >> 1);
  y ^= (int)(((unsigned)(y >> 31)) >> 1);
  return x < y;
}
__host__ __device__ __forceinline__ bool total_less(double a, double b) {
  long long x = dbits(a), y = dbits(b);
  x ^= (long long)(((unsigned long long)(x >> 63)) >> 1);
  y ^= (long long)(((unsigned long long)(y >> 63)) >> 1);
  return x < y;
}
// Ascending sort in Rust's total_cmp order (what `sort_by(total_cmp)` returns) by fixed
// compare-exchange networks: equal keys under the total order are equal bits, so stability is moot.
template <class T>
__host__ __device__ __forceinline__ void cswap(T& a, T& b) {
  if (total_less(b, a)) { T t = a; a = b; b = t; }
}
template <class T>
__host__ __device__ __forceinline__ void sort3(T& a, T& b, T& c) {
  cswap(a, b); cswap(b, c); cswap(a, b);
}
template <class T>
__host__ __device__ __forceinline__ void sort4(T& a, T& b, T& c, T& d) {
  cswap(a, b); cswap(c, d); cswap(a, c); cswap(b, d); cswap(b, c);
}

__device__ __forceinline__ float clamp01f(float x) { return x < 0.f ? 0.f : (x > 1.f ? 1.f : x); }

// delta_projection.rs:795-805
__device__ float open_below(float a, float b, float z) {
  float open;
  if (a < z && b < z) open = 1.f;
  else if (a >= z && b >= z) open = 0.f;
  else {
    float t = (z - a) / (b - a);
    open = a < z ? t : 1.f - t;
  }
  return clamp01f(open);
}

// delta_projection.rs:816-827
__device__ float cut_fraction(float a, float b, float top, float dx) {
  float low = fminf(a, b), high = fmaxf(a, b);
  if (low >= top) return 0.f;
  if (high <= top - dx) return 1.f;
  if (low == high) return clamp01f((top - low) / dx);
  float span = high - low;
  float full = clamp01f((top - dx - low) / span);
  float wet = clamp01f((top - low) / span);
  float h0 = clamp01f((top - low) / dx);
  float h1 = clamp01f((top - high) / dx);
  return clamp01f(full + (wet - full) * (0.5f * (h0 + h1)));
}

// delta3d_cut.rs:114-129
__device__ float triangle_below(float w0, float w1, float w2, float s) {
  float v0 = w0, v1 = w1, v2 = w2;
  sort3(v0, v1, v2);
  if (s <= v0) return 0.f;
  if (s >= v2) return 1.f;
  if (s <= v1) return (s - v0) * (s - v0) / ((v1 - v0) * (v2 - v0));
  return 1.f - (v2 - s) * (v2 - s) / ((v2 - v0) * (v2 - v1));
}

// delta3d_cut.rs:134-164
__device__ float triangle_fraction(float w0, float w1, float w2, float d) {
  float v0 = w0, v1 = w1, v2 = w2;
  sort3(v0, v1, v2);
  if (v2 <= 0.f) return 1.f;
  if (v0 >= d) return 0.f;
  float g1 = v2 > v0 ? (v1 - v0) * (v1 - v0) / (3.f * (v2 - v0)) : 0.f;
  auto primitive = [&](float s) -> float {
    if (s <= v0) return 0.f;
    if (v2 == v0) return s - v0;
    if (s <= v1) return (s - v0) * (s - v0) * (s - v0) / (3.f * (v1 - v0) * (v2 - v0));
    if (s < v2) {
      float a = v2 - v1, b = v2 - s;
      return g1 + (s - v1) - (a * a * a - b * b * b) / (3.f * (v2 - v0) * a);
    }
    float a = v2 - v1;
    float g2 = g1 + a - a * a / (3.f * (v2 - v0));
    return g2 + (s - v2);
  };
  return clamp01f((primitive(d) - primitive(0.f)) / d);
}

// delta3d_cut.rs:85-110: bottom at footprint corners, (nx+1)(ny+1).
__global__ void k_corners(int nx, int ny, const float* __restrict__ bottom, float* __restrict__ out) {
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= (nx + 1) * (ny + 1)) return;
  int i = q % (nx + 1), j = q / (nx + 1);
  auto b = [&](int a, int c) { return bottom[c * nx + a]; };
  auto edge = [&](int a, int c) -> float {
    if (a == 0) return b(0, c);
    if (a == nx) return b(nx - 1, c);
    return 0.5f * (b(a - 1, c) + b(a, c));
  };
  out[q] = j == 0 ? edge(i, 0) : (j == ny ? edge(i, ny - 1) : 0.5f * (edge(i, j - 1) + edge(i, j)));
}

struct CutGeo {
  int nx, ny, nz;
  float dx;
  const float* corner;  // (nx+1)(ny+1)
  float* frac; float* ou; float* ov; float* ow; float* floor;
};

__device__ __forceinline__ void footprint(const CutGeo& G, int i, int j, float c[4]) {
  const float* K = G.corner;
  c[0] = K[j * (G.nx + 1) + i];
  c[1] = K[j * (G.nx + 1) + i + 1];
  c[2] = K[(j + 1) * (G.nx + 1) + i + 1];
  c[3] = K[(j + 1) * (G.nx + 1) + i];
}

// delta3d_cut.rs:184-198: fluid fraction of every cell above the bottom.
__global__ void k_cut_frac(CutGeo G) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= G.nx * G.ny * G.nz) return;
  int i = c % G.nx, t = c / G.nx, j = t % G.ny, k = t / G.ny;
  float bas = (float)k * G.dx, top = (float)(k + 1) * G.dx;
  float q[4]; footprint(G, i, j, q);
  float f;
  if (q[0] == q[3] && q[1] == q[2]) f = cut_fraction(q[0], q[1], top, G.dx);
  else {
    float m = 0.25f * (q[0] + q[1] + q[2] + q[3]);
    float tr[4][3] = {{q[0], q[1], m}, {q[1], q[2], m}, {q[2], q[3], m}, {q[3], q[0], m}};
    float part[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) part[e] = triangle_fraction(tr[e][0] - bas, tr[e][1] - bas, tr[e][2] - bas, G.dx);
    f = 0.25f * (part[0] + part[1] + part[2] + part[3]);
  }
  G.frac[c] = f;
}

// delta3d_cut.rs:201-212 (u and v faces) and 216-231 (w faces).
__global__ void k_cut_faces(CutGeo G) {
  int nx = G.nx, ny = G.ny, nz = G.nz;
  int nu = (nx + 1) * ny * nz, nv = nx * (ny + 1) * nz, nw = nx * ny * (nz + 1);
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  const float* K = G.corner;
  auto corner = [&](int a, int b) { return K[b * (nx + 1) + a]; };
  if (q < nu) {
    int i = q % (nx + 1), t = q / (nx + 1), j = t % ny, k = t / ny;
    float top = (float)(k + 1) * G.dx;
    float o = 0.f;
    if (!(i == 0 || i == nx)) {
      float a = corner(i, j), b = corner(i, j + 1);
      o = a == b ? clamp01f((top - a) / G.dx) : cut_fraction(a, b, top, G.dx);
    }
    G.ou[q] = o;
    return;
  }
  q -= nu;
  if (q < nv) {
    int i = q % nx, t = q / nx, j = t % (ny + 1), k = t / (ny + 1);
    float top = (float)(k + 1) * G.dx;
    float o = 0.f;
    if (!(j == 0 || j == ny)) {
      float a = corner(i, j), b = corner(i + 1, j);
      o = a == b ? clamp01f((top - a) / G.dx) : cut_fraction(a, b, top, G.dx);
    }
    G.ov[q] = o;
    return;
  }
  q -= nv;
  if (q < nw) {
    int i = q % nx, t = q / nx, j = t % ny, k = t / ny;
    float o = 0.f;  // the bottom of the domain is closed
    if (k >= 1) {
      float z = (float)k * G.dx;
      float c[4]; footprint(G, i, j, c);
      if (c[0] == c[3] && c[1] == c[2]) o = open_below(c[0], c[1], z);
      else {
        float m = 0.25f * (c[0] + c[1] + c[2] + c[3]);
        o = 0.25f * (triangle_below(c[0], c[1], m, z) + triangle_below(c[1], c[2], m, z) +
                     triangle_below(c[2], c[3], m, z) + triangle_below(c[3], c[0], m, z));
      }
    }
    G.ow[q] = o;
  }
}

// delta3d_cut.rs:234-251 / 401-424: a fluid cell with no open face is declared solid.
__global__ void k_seal_isolated(CutGeo G) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  int nx = G.nx, ny = G.ny;
  if (c >= nx * ny * G.nz) return;
  if (G.frac[c] == 0.f) return;
  int i = c % nx, t = c / nx, j = t % ny, k = t / ny;
  float a = G.ou[(k * ny + j) * (nx + 1) + i] + G.ou[(k * ny + j) * (nx + 1) + i + 1] +
            G.ov[(k * (ny + 1) + j) * nx + i] + G.ov[(k * (ny + 1) + j + 1) * nx + i] +
            G.ow[(k * ny + j) * nx + i] + G.ow[((k + 1) * ny + j) * nx + i];
  if (a == 0.f) G.frac[c] = 0.f;
}

// delta3d_cut.rs:252-255: the highest footprint corner of each column.
__global__ void k_floor(CutGeo G) {
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= G.nx * G.ny) return;
  int i = q % G.nx, j = q / G.nx;
  float c[4]; footprint(G, i, j, c);
  float m = -INFINITY;
#pragma unroll
  for (int e = 0; e < 4; ++e) m = fmaxf(m, c[e]);
  G.floor[q] = m;
}

// ---------------------------------------------------------------------------------------- solid
// delta3d_cut.rs:277-292
__host__ __device__ double tri_negative(double a0, double a1, double a2) {
  double v0 = a0, v1 = a1, v2 = a2;
  sort3(v0, v1, v2);
  if (v0 >= 0.) return 0.;
  if (v2 < 0.) return 1.;
  if (v1 >= 0.) { double a = -v0; return a * a / ((a + v1) * (a + v2)); }
  return 1. - v2 * v2 / ((v2 - v0) * (v2 - v1));
}

// delta3d_cut.rs:297-316
__host__ __device__ double tet_negative(double a0, double a1, double a2, double a3) {
  double v0 = a0, v1 = a1, v2 = a2, v3 = a3;
  sort4(v0, v1, v2, v3);
  if (v0 >= 0.) return 0.;
  if (v3 < 0.) return 1.;
  if (v1 >= 0.) { double a = -v0; return a * a * a / ((a + v1) * (a + v2) * (a + v3)); }
  if (v2 >= 0.) {
    double a = -v0, b = -v1, c = v2, d = v3;
    return (c * d * (a * a + a * b + b * b) + (c + d) * a * b * (a + b) + a * a * b * b) /
           ((c + a) * (d + a) * (c + b) * (d + b));
  }
  return 1. - v3 * v3 * v3 / ((v3 - v0) * (v3 - v1) * (v3 - v2));
}

// delta3d_cut.rs:319-326
__host__ __device__ double face_negative(double c0, double c1, double c2, double c3) {
  double m = 0.25 * (c0 + c1 + c2 + c3);
  return 0.25 * (tri_negative(c0, c1, m) + tri_negative(c1, c2, m) + tri_negative(c2, c3, m) + tri_negative(c3, c0, m));
}

// The four tetrahedra of one cell face (corners c0..c3 in cyclic order, m the cell centre),
// accumulated into s one by one in the reference's order (delta3d_cut.rs:375-378).
__host__ __device__ __forceinline__ void face_tets(double& s, double c0, double c1, double c2, double c3, double m) {
  double fc = 0.25 * (c0 + c1 + c2 + c3);
  s += tet_negative(c0, c1, fc, m);
  s += tet_negative(c1, c2, fc, m);
  s += tet_negative(c2, c3, fc, m);
  s += tet_negative(c3, c0, fc, m);
}

// delta3d_cut.rs:370-381: 24 tetrahedra of equal volume, one per face triangle, closed at the
// centre.  Faces in the order of CELL_FACES (delta3d_cut.rs:367), nodes indexed x + 2y + 4z.  Every
// index is a compile-time constant (no table lookup into the local node array).
__host__ __device__ __forceinline__ double cell_negative(const double (&n)[8]) {
  double m = 0.;
  m += n[0]; m += n[1]; m += n[2]; m += n[3]; m += n[4]; m += n[5]; m += n[6]; m += n[7];
  m = m / 8.;
  double s = 0.;
  face_tets(s, n[0], n[2], n[6], n[4], m);
  face_tets(s, n[1], n[3], n[7], n[5], m);
  face_tets(s, n[0], n[1], n[5], n[4], m);
  face_tets(s, n[2], n[3], n[7], n[6], m);
  face_tets(s, n[0], n[1], n[3], n[2], m);
  face_tets(s, n[4], n[5], n[7], n[6], m);
  return s / 24.;
}

struct SolidGeo {
  int nx, ny, nz;
  float dx;
  const float* sdf;  // (nx+1)(ny+1)(nz+1)
  int piercing;
};

__device__ __forceinline__ double node(const SolidGeo& S, int a, int b, int c) {
  return (double)S.sdf[(c * (S.ny + 1) + b) * (S.nx + 1) + a];
}

__device__ __forceinline__ void cell_nodes(const SolidGeo& S, int i, int j, int k, double (&n)[8]) {
  n[0] = node(S, i, j, k); n[1] = node(S, i + 1, j, k); n[2] = node(S, i, j + 1, k); n[3] = node(S, i + 1, j + 1, k);
  n[4] = node(S, i, j, k + 1); n[5] = node(S, i + 1, j, k + 1); n[6] = node(S, i, j + 1, k + 1); n[7] = node(S, i + 1, j + 1, k + 1);
}

// check_solid (delta3d_cut.rs:485-531): sets *refused when the solid shares a cell or a face with
// the bottom cut, or reaches the lid layer.
__global__ void k_check_solid(SolidGeo S, const float* __restrict__ frac, const float* __restrict__ ou,
                              const float* __restrict__ ov, const float* __restrict__ ow, int* refused) {
  int nx = S.nx, ny = S.ny, nz = S.nz;
  int ncell = nx * ny * nz, nu = (nx + 1) * ny * nz, nv = nx * (ny + 1) * nz, nw = nx * ny * (nz + 1);
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  bool bad = false;
  if (q < ncell) {
    int i = q % nx, t = q / nx, j = t % ny, k = t / ny;
    double n[8]; cell_nodes(S, i, j, k, n);
    bad = cell_negative(n) > 0. && (frac[q] < 1.f || (k + 1 == nz && !S.piercing));
  } else if ((q -= ncell) < nu) {
    int i = q % (nx + 1), t = q / (nx + 1), j = t % ny, k = t / ny;
    if (i >= 1 && i < nx)
      bad = ou[q] < 1.f && face_negative(node(S, i, j, k), node(S, i, j + 1, k), node(S, i, j + 1, k + 1), node(S, i, j, k + 1)) > 0.;
  } else if ((q -= nu) < nv) {
    int i = q % nx, t = q / nx, j = t % (ny + 1), k = t / (ny + 1);
    if (j >= 1 && j < ny)
      bad = ov[q] < 1.f && face_negative(node(S, i, j, k), node(S, i + 1, j, k), node(S, i + 1, j, k + 1), node(S, i, j, k + 1)) > 0.;
  } else if ((q -= nv) < nw) {
    int i = q % nx, t = q / nx, j = t % ny, k = t / ny;
    if (k >= 1)
      bad = ow[q] < 1.f && face_negative(node(S, i, j, k), node(S, i + 1, j, k), node(S, i + 1, j + 1, k), node(S, i, j + 1, k)) > 0.;
  }
  if (bad) atomicOr(refused, 1);
}

__device__ __forceinline__ void atomic_max_nonneg(float* addr, float v) {
  atomicMax(reinterpret_cast<int*>(addr), __float_as_int(v));
}

// add_solid (delta3d_cut.rs:429-482) after check_solid accepted: cell fractions, floors, faces.
__global__ void k_add_solid(SolidGeo S, float* __restrict__ frac, float* __restrict__ ou, float* __restrict__ ov,
                            float* __restrict__ ow, float* __restrict__ floor) {
  int nx = S.nx, ny = S.ny, nz = S.nz;
  int ncell = nx * ny * nz, nu = (nx + 1) * ny * nz, nv = nx * (ny + 1) * nz, nw = nx * ny * (nz + 1);
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q < ncell) {
    int i = q % nx, t = q / nx, j = t % ny, k = t / ny;
    double n[8]; cell_nodes(S, i, j, k, n);
    double s = cell_negative(n);
    if (s > 0.) {
      frac[q] = (float)(1. - s);
      float top = (float)(k + 1) * S.dx;
      // floor >= 0 (the bottom lies in [0, z0)), so the integer order of the bits is the float order
      atomic_max_nonneg(floor + j * nx + i, top);
    }
    return;
  }
  q -= ncell;
  double s = 0.;
  float* dst = nullptr;
  if (q < nu) {
    int i = q % (nx + 1), t = q / (nx + 1), j = t % ny, k = t / ny;
    if (i >= 1 && i < nx) { s = face_negative(node(S, i, j, k), node(S, i, j + 1, k), node(S, i, j + 1, k + 1), node(S, i, j, k + 1)); dst = ou + q; }
  } else if ((q -= nu) < nv) {
    int i = q % nx, t = q / nx, j = t % (ny + 1), k = t / (ny + 1);
    if (j >= 1 && j < ny) { s = face_negative(node(S, i, j, k), node(S, i + 1, j, k), node(S, i + 1, j, k + 1), node(S, i, j, k + 1)); dst = ov + q; }
  } else if ((q -= nv) < nw) {
    int i = q % nx, t = q / nx, j = t % ny, k = t / ny;
    if (k >= 1) { s = face_negative(node(S, i, j, k), node(S, i + 1, j, k), node(S, i + 1, j + 1, k), node(S, i, j + 1, k)); dst = ow + q; }
  }
  if (dst && s > 0.) *dst = (float)(1. - s);
}

}  // namespace fd3
