// Oracle: CPU restatement of water-core's local volumetric (delta) MAC-grid pressure projection.
//
// TEST INFRASTRUCTURE ONLY.  This file is the parity checker and the timed CPU baseline; the
// product (fluidisim_b200/csrc) never links, loads or calls it.  Only tests/, the smoke check and
// bench.py's CPU-baseline leg use it.
//
// It restates, function by function and in the same floating-point evaluation order, the Rust
// reference (paths relative to the reference project):
//   code/water-core/src/delta3d.rs           Domain3, Volume3 buffers, configure*, set_*, divergence*,
//                                             dot/norm2, fingerprint, the linear path (lid, apply*,
//                                             backward_error*, correct*, project, step_surface_linear)
//   code/water-core/src/delta3d_mobile.rs    wet3/open3/solid3, ghosts, mobile_row, apply/rhs/backward
//                                             error/correct/extrapolate/divergence, project_mobile3,
//                                             advect/transport, step_surface_mobile, trial hooks
//   code/water-core/src/delta3d_multigrid.rs the V-cycle preconditioner (damped Jacobi 6/7, 2/2/8 sweeps)
//   code/water-core/src/delta3d_cut.rs       bottom cut and solid SDF cut (24 tetrahedra per cell)
//   code/water-core/src/delta_projection.rs  Error/Report, tolerances, cut_fraction, open_below
//   code/water-core/src/host.rs, code/water-harness/src/host_impl.rs  ordered grain-64 reduction
//
// Build with -ffp-contract=off (Rust never contracts to FMA).  Compiling with -DOD3_REAL=double
// gives the same algorithm in FP64, used as the error reference (solved to a tighter tolerance).
// OpenMP only splits loops whose writes are disjoint; every floating-point reduction keeps the
// reference's order (chunk partials of 64 are independent, the merge is sequential), so the result
// does not depend on the thread count.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <new>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#ifndef OD3_REAL
#define OD3_REAL float
#endif
typedef OD3_REAL R;

namespace {

// Error codes: the order of `Error` in delta_projection.rs:133-150, shifted by one (0 = Ok).
enum Err : int {
  OK = 0, DOMAIN = 1, NOT_FINITE = 2, SHAPE = 3, BUDGET = 4, CLOCK = 5, CONVERGENCE = 6,
  INVALID = 102
};

// delta_projection.rs:192
const double PROJECTION_DIVERGENCE_TOLERANCE = 1e-5;
// delta_mobile.rs:14
const R SURFACE_THETA_MIN = (R)1e-3;
// delta3d.rs:41
const R PROJECTION_VELOCITY_FLOOR = (R)1e-4;
// delta_projection.rs:200-203: gamma_8 with u = 2^-24
const float ROUNDOFF_BACKWARD_ERROR = (float)(8.0f * (1.0f / 16777216.0f) / (1.0f - 8.0f * (1.0f / 16777216.0f)));
// delta3d.rs:69-72: gamma_10
const float ROUNDOFF_BACKWARD_ERROR_3D = (float)(10.0f * (1.0f / 16777216.0f) / (1.0f - 10.0f * (1.0f / 16777216.0f)));
// delta3d_multigrid.rs:28-34
const R SMOOTH_DAMPING_3D = (R)6. / (R)7.;
const int PRE_SWEEPS_3D = 2, POST_SWEEPS_3D = 2, COARSE_SWEEPS_3D = 8;

inline R rmax(R a, R b) { return std::fmax(a, b); }  // Rust f32::max ignores a NaN operand, as fmax does
inline R clamp01(R x) { return x < (R)0 ? (R)0 : (x > (R)1 ? (R)1 : x); }

int g_threads = 1;

// Smoother of the V-cycle: 0 = the reference's damped Jacobi (delta3d_multigrid.rs:28, 290-299);
// 1 = red-black Gauss-Seidel (omega = 1), pre-sweeps red then black, post-sweeps black then red,
// the coarsest level's sweeps forward then backward, so the preconditioner stays symmetric.
// 0: damped Jacobi everywhere (the reference); 1: red-black Gauss-Seidel on every level;
// 2: red-black on the fine level only, Jacobi on the coarse levels; 3: the converse
int g_smoother = 0;
bool rb_fine() { return g_smoother == 1 || g_smoother == 2; }
bool rb_coarse() { return g_smoother == 1 || g_smoother == 3; }
int g_transfer = 0;  // 0: the reference's 8-child mean and injection; 1: trilinear (restrict3_tri)

// Storage of the V-cycle vectors.  0 = the reference's f32.  1 = the B200 library's mixed-precision
// mode (no reference counterpart): the V-cycle runs on r / sigma, sigma = rms(r over all cells) *
// dx^2 / 6 (a positive scalar per V-cycle, which leaves PCG's iterates unchanged in exact
// arithmetic), with f32 arithmetic and FP16 storage.  The rounding is emulated here by a round trip
// through _Float16 (round to nearest even, clamped to +-65504) at the points where the device
// stores a V-cycle vector: the fine z after the two pre-sweeps and after each post-sweep, every
// restricted residual, and on levels of more than TAIL_CELLS cells the x after the pre-sweeps and
// after each post-sweep, and the residual before restriction.  Smaller levels run in f32 in one
// CTA on the device; only the x of the first of them is stored.
int g_storage = 0;
const size_t TAIL_CELLS = 512;
double g_zmax = 0;  // largest |z| a V-cycle returned since the last reset (FP16-mode statistics)

inline R h16(R v) {
  float f = (float)v;
  f = f > 65504.f ? 65504.f : (f < -65504.f ? -65504.f : f);
  return (R)(float)(_Float16)f;
}
inline void round16(std::vector<R>& a) {
  if (g_storage) for (auto& x : a) x = h16(x);
}

// ---------------------------------------------------------------------------------------------
// Ordered reduction: host.rs:60-72 contract, host_impl.rs:75-92 sequential reference.  Chunks of
// `grain` are reduced in index order inside the chunk; the chunk results are merged in increasing
// chunk order.  The merge of delta3d.rs:867 is `(x as f32 + y as f32) as f64`, i.e. an f32 add.
template <class F>
R reduce_ordered(size_t n, size_t grain, F chunk) {
  size_t g = grain ? grain : 1;
  size_t m = (n + g - 1) / g;
  std::vector<R> part(m);
#pragma omp parallel for schedule(static) num_threads(g_threads) if (m > 256)
  for (long long q = 0; q < (long long)m; ++q) {
    size_t s = (size_t)q * g, e = std::min(n, s + g);
    part[(size_t)q] = chunk(s, e);
  }
  R acc = 0;
  for (size_t q = 0; q < m; ++q) acc = acc + part[q];
  return acc;
}

struct Domain3 {
  size_t nx, ny, nz;
  R dx;
  R z0() const { return (R)nz * dx; }
  size_t cells() const { return nx * ny * nz; }
  size_t columns() const { return nx * ny; }
};

// Rust `total_cmp` order on finite and non-finite values (used by the sorts of delta3d_cut.rs).
inline bool total_less(float a, float b) {
  int32_t x, y; std::memcpy(&x, &a, 4); std::memcpy(&y, &b, 4);
  x ^= (int32_t)(((uint32_t)(x >> 31)) >> 1); y ^= (int32_t)(((uint32_t)(y >> 31)) >> 1);
  return x < y;
}
inline bool total_less(double a, double b) {
  int64_t x, y; std::memcpy(&x, &a, 8); std::memcpy(&y, &b, 8);
  x ^= (int64_t)(((uint64_t)(x >> 63)) >> 1); y ^= (int64_t)(((uint64_t)(y >> 63)) >> 1);
  return x < y;
}
template <class T, size_t N>
void sort_total(T (&v)[N]) {  // stable insertion sort, as `sort_by(total_cmp)` on tiny arrays
  for (size_t i = 1; i < N; ++i) {
    T x = v[i]; size_t j = i;
    while (j > 0 && total_less(x, v[j - 1])) { v[j] = v[j - 1]; --j; }
    v[j] = x;
  }
}

// ------------------------------------------------------------------- delta_projection.rs:795-827
R open_below(R a, R b, R z) {
  R open;
  if (a < z && b < z) open = 1;
  else if (a >= z && b >= z) open = 0;
  else {
    R t = (z - a) / (b - a);
    open = a < z ? t : (R)1 - t;
  }
  return clamp01(open);
}

R cut_fraction(R a, R b, R top, R dx) {
  R low = std::fmin(a, b), high = std::fmax(a, b);
  if (low >= top) return 0;
  if (high <= top - dx) return 1;
  if (low == high) return clamp01((top - low) / dx);
  R span = high - low;
  R full = clamp01((top - dx - low) / span);
  R wet = clamp01((top - low) / span);
  R h0 = clamp01((top - low) / dx);
  R h1 = clamp01((top - high) / dx);
  return clamp01(full + (wet - full) * ((R)0.5 * (h0 + h1)));
}

// ------------------------------------------------------------------- delta3d_cut.rs
struct Base3 {
  std::vector<R> frac, open_u, open_v, open_w, floor, solid_col, deposit;
};

struct Cut3 {
  std::vector<R> frac, open_u, open_v, open_w, floor;
  bool has_base = false;
  Base3 base;
  bool piercing = false;
  // the solid's rigid motion, set by set_solid_rigid (delta3d_cut.rs:42-46; delta3d.rs:408-410)
  float solid_velocity[3] = {0.f, 0.f, 0.f}, solid_angular[3] = {0.f, 0.f, 0.f}, solid_center[3] = {0.f, 0.f, 0.f};
};

// delta3d.rs:75-82: the axis component of the rigid wall velocity V + W x (x - c) at x.
static R wall_velocity(const float vel[3], const float ang[3], const float cen[3], int axis, R x0, R x1, R x2) {
  R r0 = x0 - (R)cen[0], r1 = x1 - (R)cen[1], r2 = x2 - (R)cen[2];
  if (axis == 0) return (R)vel[0] + ((R)ang[1] * r2 - (R)ang[2] * r1);
  if (axis == 1) return (R)vel[1] + ((R)ang[2] * r0 - (R)ang[0] * r2);
  return (R)vel[2] + ((R)ang[0] * r1 - (R)ang[1] * r0);
}

// delta3d_cut.rs:85-110
std::vector<R> corners(const Domain3& d, const R* bottom) {
  size_t nx = d.nx, ny = d.ny;
  auto b = [&](size_t i, size_t j) { return bottom[j * nx + i]; };
  auto edge = [&](size_t i, size_t j) -> R {
    if (i == 0) return b(0, j);
    if (i == nx) return b(nx - 1, j);
    return (R)0.5 * (b(i - 1, j) + b(i, j));
  };
  std::vector<R> out((nx + 1) * (ny + 1), (R)0);
  for (size_t j = 0; j <= ny; ++j)
    for (size_t i = 0; i <= nx; ++i)
      out[j * (nx + 1) + i] = j == 0 ? edge(i, 0) : (j == ny ? edge(i, ny - 1) : (R)0.5 * (edge(i, j - 1) + edge(i, j)));
  return out;
}

// delta3d_cut.rs:114-129
R triangle_below(const R w[3], R s) {
  R v[3] = {w[0], w[1], w[2]};
  sort_total(v);
  R v0 = v[0], v1 = v[1], v2 = v[2];
  if (s <= v0) return 0;
  if (s >= v2) return 1;
  if (s <= v1) return (s - v0) * (s - v0) / ((v1 - v0) * (v2 - v0));
  return (R)1 - (v2 - s) * (v2 - s) / ((v2 - v0) * (v2 - v1));
}

// delta3d_cut.rs:134-164
R triangle_fraction(const R w[3], R d) {
  R v[3] = {w[0], w[1], w[2]};
  sort_total(v);
  R v0 = v[0], v1 = v[1], v2 = v[2];
  if (v2 <= 0) return 1;
  if (v0 >= d) return 0;
  R g1 = v2 > v0 ? (v1 - v0) * (v1 - v0) / ((R)3 * (v2 - v0)) : (R)0;
  auto primitive = [&](R s) -> R {
    if (s <= v0) return 0;
    if (v2 == v0) return s - v0;
    if (s <= v1) return (s - v0) * (s - v0) * (s - v0) / ((R)3 * (v1 - v0) * (v2 - v0));
    if (s < v2) {
      R a = v2 - v1, b = v2 - s;
      return g1 + (s - v1) - (a * a * a - b * b * b) / ((R)3 * (v2 - v0) * a);
    }
    R a = v2 - v1;
    R g2 = g1 + a - a * a / ((R)3 * (v2 - v0));
    return g2 + (s - v2);
  };
  R r = (primitive(d) - primitive((R)0)) / d;
  return clamp01(r);
}

// delta3d_cut.rs:168-171
void triangles(const R c[4], R t[4][3]) {
  R m = (R)0.25 * (c[0] + c[1] + c[2] + c[3]);
  R tt[4][3] = {{c[0], c[1], m}, {c[1], c[2], m}, {c[2], c[3], m}, {c[3], c[0], m}};
  std::memcpy(t, tt, sizeof(tt));
}

// delta3d_cut.rs:172-260
Cut3 cut(const Domain3& d, const R* bottom) {
  size_t nx = d.nx, ny = d.ny, nz = d.nz;
  R dx = d.dx;
  std::vector<R> k0 = corners(d, bottom);
  auto corner = [&](size_t i, size_t j) { return k0[j * (nx + 1) + i]; };
  auto footprint = [&](size_t i, size_t j, R c[4]) {
    c[0] = corner(i, j); c[1] = corner(i + 1, j); c[2] = corner(i + 1, j + 1); c[3] = corner(i, j + 1);
  };
  auto plane_in_y = [](const R c[4]) { return c[0] == c[3] && c[1] == c[2]; };
  Cut3 g;
  g.frac.assign(nx * ny * nz, (R)0);
  g.open_u.assign((nx + 1) * ny * nz, (R)0);
  g.open_v.assign(nx * (ny + 1) * nz, (R)0);
  g.open_w.assign(nx * ny * (nz + 1), (R)0);
  for (size_t k = 0; k < nz; ++k) {
    R bas = (R)k * dx, top = (R)(k + 1) * dx;
    for (size_t j = 0; j < ny; ++j)
      for (size_t i = 0; i < nx; ++i) {
        R c[4]; footprint(i, j, c);
        R f;
        if (plane_in_y(c)) f = cut_fraction(c[0], c[1], top, dx);
        else {
          R t[4][3]; triangles(c, t);
          R s = 0;
          R part[4];
          for (int e = 0; e < 4; ++e) {
            R w[3] = {t[e][0] - bas, t[e][1] - bas, t[e][2] - bas};
            part[e] = triangle_fraction(w, dx);
          }
          s = part[0] + part[1] + part[2] + part[3];
          f = (R)0.25 * s;
        }
        g.frac[(k * ny + j) * nx + i] = f;
      }
    auto side = [&](R a, R b) -> R { return a == b ? clamp01((top - a) / dx) : cut_fraction(a, b, top, dx); };
    for (size_t j = 0; j < ny; ++j)
      for (size_t i = 0; i <= nx; ++i)
        g.open_u[(k * ny + j) * (nx + 1) + i] = (i == 0 || i == nx) ? (R)0 : side(corner(i, j), corner(i, j + 1));
    for (size_t j = 0; j <= ny; ++j)
      for (size_t i = 0; i < nx; ++i)
        g.open_v[(k * (ny + 1) + j) * nx + i] = (j == 0 || j == ny) ? (R)0 : side(corner(i, j), corner(i + 1, j));
  }
  for (size_t k = 1; k <= nz; ++k) {
    R z = (R)k * dx;
    for (size_t j = 0; j < ny; ++j)
      for (size_t i = 0; i < nx; ++i) {
        R c[4]; footprint(i, j, c);
        R o;
        if (plane_in_y(c)) o = open_below(c[0], c[1], z);
        else {
          R t[4][3]; triangles(c, t);
          o = (R)0.25 * (triangle_below(t[0], z) + triangle_below(t[1], z) + triangle_below(t[2], z) + triangle_below(t[3], z));
        }
        g.open_w[(k * ny + j) * nx + i] = o;
      }
  }
  for (size_t k = 0; k < nz; ++k)
    for (size_t j = 0; j < ny; ++j)
      for (size_t i = 0; i < nx; ++i) {
        size_t c = (k * ny + j) * nx + i;
        if (g.frac[c] == 0) continue;
        R a = g.open_u[(k * ny + j) * (nx + 1) + i] + g.open_u[(k * ny + j) * (nx + 1) + i + 1] +
              g.open_v[(k * (ny + 1) + j) * nx + i] + g.open_v[(k * (ny + 1) + j + 1) * nx + i] +
              g.open_w[(k * ny + j) * nx + i] + g.open_w[((k + 1) * ny + j) * nx + i];
        if (a == 0) g.frac[c] = 0;
      }
  g.floor.resize(nx * ny);
  for (size_t j = 0; j < ny; ++j)
    for (size_t i = 0; i < nx; ++i) {
      R c[4]; footprint(i, j, c);
      R m = -std::numeric_limits<R>::infinity();
      for (int e = 0; e < 4; ++e) m = std::fmax(m, c[e]);
      g.floor[j * nx + i] = m;
    }
  return g;
}

// delta3d_cut.rs:277-292
double tri_negative(const double w[3]) {
  double v[3] = {w[0], w[1], w[2]};
  sort_total(v);
  double v0 = v[0], v1 = v[1], v2 = v[2];
  if (v0 >= 0.) return 0.;
  if (v2 < 0.) return 1.;
  if (v1 >= 0.) { double a = -v0; return a * a / ((a + v1) * (a + v2)); }
  return 1. - v2 * v2 / ((v2 - v0) * (v2 - v1));
}

// delta3d_cut.rs:297-316
double tet_negative(const double w[4]) {
  double v[4] = {w[0], w[1], w[2], w[3]};
  sort_total(v);
  double v0 = v[0], v1 = v[1], v2 = v[2], v3 = v[3];
  if (v0 >= 0.) return 0.;
  if (v3 < 0.) return 1.;
  if (v1 >= 0.) { double a = -v0; return a * a * a / ((a + v1) * (a + v2) * (a + v3)); }
  if (v2 >= 0.) {
    double a = -v0, b = -v1, c = v2, dd = v3;
    return (c * dd * (a * a + a * b + b * b) + (c + dd) * a * b * (a + b) + a * a * b * b) /
           ((c + a) * (dd + a) * (c + b) * (dd + b));
  }
  return 1. - v3 * v3 * v3 / ((v3 - v0) * (v3 - v1) * (v3 - v2));
}

// delta3d_cut.rs:319-326
double face_negative(const double c[4]) {
  double m = 0.25 * (c[0] + c[1] + c[2] + c[3]);
  double t0[3] = {c[0], c[1], m}, t1[3] = {c[1], c[2], m}, t2[3] = {c[2], c[3], m}, t3[3] = {c[3], c[0], m};
  return 0.25 * (tri_negative(t0) + tri_negative(t1) + tri_negative(t2) + tri_negative(t3));
}

// delta3d_cut.rs:367
const int CELL_FACES[6][4] = {{0, 2, 6, 4}, {1, 3, 7, 5}, {0, 1, 5, 4}, {2, 3, 7, 6}, {0, 1, 3, 2}, {4, 5, 7, 6}};

// delta3d_cut.rs:370-381
double cell_negative(const double n[8]) {
  double m = 0.;
  for (int q = 0; q < 8; ++q) m += n[q];
  m = m / 8.;
  double s = 0.;
  for (int f = 0; f < 6; ++f) {
    double c[4] = {n[CELL_FACES[f][0]], n[CELL_FACES[f][1]], n[CELL_FACES[f][2]], n[CELL_FACES[f][3]]};
    double fc = 0.25 * (c[0] + c[1] + c[2] + c[3]);
    for (int e = 0; e < 4; ++e) {
      double t[4] = {c[e], c[(e + 1) % 4], fc, m};
      s += tet_negative(t);
    }
  }
  return s / 24.;
}

// delta3d_cut.rs:384-398
void cell_nodes(const Domain3& d, const float* solid, size_t i, size_t j, size_t k, double n[8]) {
  size_t nx = d.nx, ny = d.ny;
  auto node = [&](size_t a, size_t b, size_t c) { return (double)solid[(c * (ny + 1) + b) * (nx + 1) + a]; };
  n[0] = node(i, j, k); n[1] = node(i + 1, j, k); n[2] = node(i, j + 1, k); n[3] = node(i + 1, j + 1, k);
  n[4] = node(i, j, k + 1); n[5] = node(i + 1, j, k + 1); n[6] = node(i, j + 1, k + 1); n[7] = node(i + 1, j + 1, k + 1);
}

// delta3d_cut.rs:401-424
void seal_isolated(Cut3& g, const Domain3& d) {
  size_t nx = d.nx, ny = d.ny, nz = d.nz;
  for (size_t k = 0; k < nz; ++k)
    for (size_t j = 0; j < ny; ++j)
      for (size_t i = 0; i < nx; ++i) {
        size_t c = (k * ny + j) * nx + i;
        if (g.frac[c] == 0) continue;
        R a = g.open_u[(k * ny + j) * (nx + 1) + i] + g.open_u[(k * ny + j) * (nx + 1) + i + 1] +
              g.open_v[(k * (ny + 1) + j) * nx + i] + g.open_v[(k * (ny + 1) + j + 1) * nx + i] +
              g.open_w[(k * ny + j) * nx + i] + g.open_w[((k + 1) * ny + j) * nx + i];
        if (a == 0) g.frac[c] = 0;
      }
}

// delta3d_cut.rs:485-531
int check_solid(const std::vector<R>& frac, const std::vector<R>& open_u, const std::vector<R>& open_v,
                const std::vector<R>& open_w, const Domain3& d, const float* solid, bool piercing) {
  size_t nx = d.nx, ny = d.ny, nz = d.nz;
  auto node = [&](size_t a, size_t b, size_t c) { return (double)solid[(c * (ny + 1) + b) * (nx + 1) + a]; };
  for (size_t k = 0; k < nz; ++k)
    for (size_t j = 0; j < ny; ++j)
      for (size_t i = 0; i < nx; ++i) {
        double n[8]; cell_nodes(d, solid, i, j, k, n);
        if (cell_negative(n) > 0. && (frac[(k * ny + j) * nx + i] < 1 || (k + 1 == nz && !piercing))) return DOMAIN;
      }
  auto partage = [&](R open, const double c[4]) { return open < 1 && face_negative(c) > 0.; };
  for (size_t k = 0; k < nz; ++k) {
    for (size_t j = 0; j < ny; ++j)
      for (size_t i = 1; i < nx; ++i) {
        double c[4] = {node(i, j, k), node(i, j + 1, k), node(i, j + 1, k + 1), node(i, j, k + 1)};
        if (partage(open_u[(k * ny + j) * (nx + 1) + i], c)) return DOMAIN;
      }
    for (size_t j = 1; j < ny; ++j)
      for (size_t i = 0; i < nx; ++i) {
        double c[4] = {node(i, j, k), node(i + 1, j, k), node(i + 1, j, k + 1), node(i, j, k + 1)};
        if (partage(open_v[(k * (ny + 1) + j) * nx + i], c)) return DOMAIN;
      }
  }
  for (size_t k = 1; k <= nz; ++k)
    for (size_t j = 0; j < ny; ++j)
      for (size_t i = 0; i < nx; ++i) {
        double c[4] = {node(i, j, k), node(i + 1, j, k), node(i + 1, j + 1, k), node(i, j + 1, k)};
        if (partage(open_w[(k * ny + j) * nx + i], c)) return DOMAIN;
      }
  return OK;
}

// delta3d_cut.rs:429-482
int add_solid(Cut3& g, const Domain3& d, const float* solid) {
  int e = check_solid(g.frac, g.open_u, g.open_v, g.open_w, d, solid, g.piercing);
  if (e) return e;
  size_t nx = d.nx, ny = d.ny, nz = d.nz;
  R dx = d.dx;
  auto node = [&](size_t a, size_t b, size_t c) { return (double)solid[(c * (ny + 1) + b) * (nx + 1) + a]; };
  for (size_t k = 0; k < nz; ++k)
    for (size_t j = 0; j < ny; ++j)
      for (size_t i = 0; i < nx; ++i) {
        double n[8]; cell_nodes(d, solid, i, j, k, n);
        double s = cell_negative(n);
        if (s > 0.) {
          size_t c = (k * ny + j) * nx + i;
          g.frac[c] = (R)(1. - s);
          R top = (R)(k + 1) * dx;
          if (top > g.floor[j * nx + i]) g.floor[j * nx + i] = top;
        }
      }
  auto face = [&](R& open, const double c[4]) {
    double s = face_negative(c);
    if (s > 0.) open = (R)(1. - s);
  };
  for (size_t k = 0; k < nz; ++k) {
    for (size_t j = 0; j < ny; ++j)
      for (size_t i = 1; i < nx; ++i) {
        double c[4] = {node(i, j, k), node(i, j + 1, k), node(i, j + 1, k + 1), node(i, j, k + 1)};
        face(g.open_u[(k * ny + j) * (nx + 1) + i], c);
      }
    for (size_t j = 1; j < ny; ++j)
      for (size_t i = 0; i < nx; ++i) {
        double c[4] = {node(i, j, k), node(i + 1, j, k), node(i + 1, j, k + 1), node(i, j, k + 1)};
        face(g.open_v[(k * (ny + 1) + j) * nx + i], c);
      }
  }
  for (size_t k = 1; k <= nz; ++k)
    for (size_t j = 0; j < ny; ++j)
      for (size_t i = 0; i < nx; ++i) {
        double c[4] = {node(i, j, k), node(i + 1, j, k), node(i + 1, j + 1, k), node(i, j + 1, k)};
        face(g.open_w[(k * ny + j) * nx + i], c);
      }
  seal_isolated(g, d);
  return OK;
}

// delta3d.rs:86-99
void solid_columns(const Domain3& d, const std::vector<R>& base, const std::vector<R>& frac, std::vector<R>& out) {
  size_t nx = d.nx, ny = d.ny, nz = d.nz;
  double dd = (double)d.dx;
  double cube = dd * dd * dd;  // powi(3)
  for (size_t j = 0; j < ny; ++j)
    for (size_t i = 0; i < nx; ++i) {
      double s = 0.;
      for (size_t k = 0; k < nz; ++k) {
        size_t c = (k * ny + j) * nx + i;
        s += (double)(base[c] - frac[c]);
      }
      out[j * nx + i] = (R)(s * cube);
    }
}

// ------------------------------------------------------------------- delta3d_multigrid.rs
// delta3d_multigrid.rs:73-75
bool coarsens3(size_t nx, size_t ny, size_t nz) {
  return nx % 2 == 0 && ny % 2 == 0 && nz % 2 == 0 && nx >= 4 && ny >= 4 && nz >= 4;
}
// delta3d_multigrid.rs:78-88
size_t level_count3(size_t nx, size_t ny, size_t nz) {
  size_t n = 0;
  while (coarsens3(nx, ny, nz)) { nx /= 2; ny /= 2; nz /= 2; ++n; }
  return n;
}
// delta3d_multigrid.rs:92-105
bool hierarchy_floats3(size_t nx, size_t ny, size_t nz, size_t* out) {
  size_t fine, total;
  if (__builtin_mul_overflow(nx, ny, &fine) || __builtin_mul_overflow(fine, nz, &fine)) return false;
  if (__builtin_mul_overflow(fine, (size_t)2, &total)) return false;
  size_t x = nx, y = ny, z = nz;
  while (coarsens3(x, y, z)) {
    size_t cx = x / 2, cy = y / 2, cz = z / 2;
    size_t cells = cx * cy * cz;
    size_t faces = (cx + 1) * cy * cz + cx * (cy + 1) * cz + cx * cy * (cz + 1);
    size_t c5;
    if (__builtin_mul_overflow(cells, (size_t)5, &c5) || __builtin_add_overflow(total, c5, &total) ||
        __builtin_add_overflow(total, faces, &total))
      return false;
    x = cx; y = cy; z = cz;
  }
  *out = total;
  return true;
}

struct Level3 {
  size_t nx, ny, nz;
  R inv;
  std::vector<R> open_u, open_v, open_w, kind, diag, x, r, t;
  size_t cells() const { return nx * ny * nz; }
  size_t c(size_t i, size_t j, size_t k) const { return (k * ny + j) * nx + i; }
};

struct Multigrid3 {
  std::vector<Level3> levels;
  std::vector<R> z, t;
};

// delta3d_multigrid.rs:109-137 (max_levels caps the hierarchy depth; 0 keeps the reference's rule)
Multigrid3 make_multigrid(size_t nx, size_t ny, size_t nz, R dx, size_t max_levels) {
  Multigrid3 mg;
  size_t x = nx, y = ny, z = nz;
  R h = dx;
  while (coarsens3(x, y, z) && (max_levels == 0 || mg.levels.size() < max_levels)) {
    size_t cx = x / 2, cy = y / 2, cz = z / 2;
    h *= (R)2;
    Level3 l;
    l.nx = cx; l.ny = cy; l.nz = cz;
    l.inv = (R)1 / (h * h);
    size_t cells = cx * cy * cz;
    l.open_u.assign((cx + 1) * cy * cz, 0); l.open_v.assign(cx * (cy + 1) * cz, 0); l.open_w.assign(cx * cy * (cz + 1), 0);
    l.kind.assign(cells, 0); l.diag.assign(cells, 0); l.x.assign(cells, 0); l.r.assign(cells, 0); l.t.assign(cells, 0);
    mg.levels.push_back(std::move(l));
    x = cx; y = cy; z = cz;
  }
  mg.z.assign(nx * ny * nz, 0);
  mg.t.assign(nx * ny * nz, 0);
  return mg;
}

const int CHILDREN[8][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {1, 1, 0}, {0, 0, 1}, {1, 0, 1}, {0, 1, 1}, {1, 1, 1}};
const int QUARTER[4][2] = {{0, 0}, {1, 0}, {0, 1}, {1, 1}};

// delta3d_multigrid.rs:216-255.  `p == nullptr` gives the diagonal.
void row_sums(const Level3& L, const R* p, R* out) {
  size_t nx = L.nx, ny = L.ny, nz = L.nz;
#pragma omp parallel for schedule(static) num_threads(g_threads) if (nz * ny * nx > 32768)
  for (long long kk = 0; kk < (long long)nz; ++kk) {
    size_t k = (size_t)kk;
    for (size_t j = 0; j < ny; ++j)
      for (size_t i = 0; i < nx; ++i) {
        size_t c = L.c(i, j, k);
        if (L.kind[c] <= 0) { out[c] = 0; continue; }
        R pc = p ? p[c] : (R)0;
        R acc = 0;
        auto face = [&](R a, bool has, size_t m, bool top) {
          if (a == 0) return;
          if (has) {
            if (L.kind[m] > 0) acc += p ? a * (pc - p[m]) : a;
            else if (L.kind[m] < 0) acc += (R)2 * a * (p ? pc : (R)1);
          } else if (top) {
            acc += (R)2 * a * (p ? pc : (R)1);
          }
        };
        face(L.open_u[(k * ny + j) * (nx + 1) + i], i > 0, c - 1, false);
        face(L.open_u[(k * ny + j) * (nx + 1) + i + 1], i + 1 < nx, c + 1, false);
        face(L.open_v[(k * (ny + 1) + j) * nx + i], j > 0, c - nx, false);
        face(L.open_v[(k * (ny + 1) + j + 1) * nx + i], j + 1 < ny, c + nx, false);
        face(L.open_w[(k * ny + j) * nx + i], k > 0, c - nx * ny, false);
        face(L.open_w[((k + 1) * ny + j) * nx + i], k + 1 < nz, c + nx * ny, true);
        out[c] = acc * L.inv;
      }
  }
}

// delta3d_multigrid.rs:141-206
template <class OpenF, class KindF>
void coarsen3(size_t nx, size_t ny, OpenF open, KindF kind, Level3& L) {
  size_t cx = L.nx, cy = L.ny, cz = L.nz;
  auto fc = [&](size_t i, size_t j, size_t k) { return (k * ny + j) * nx + i; };
  auto fu = [&](size_t i, size_t j, size_t k) { return (k * ny + j) * (nx + 1) + i; };
  auto fv = [&](size_t i, size_t j, size_t k) { return (k * (ny + 1) + j) * nx + i; };
  auto fw = [&](size_t i, size_t j, size_t k) { return (k * ny + j) * nx + i; };
  for (size_t k = 0; k < cz; ++k)
    for (size_t j = 0; j < cy; ++j)
      for (size_t i = 0; i < cx; ++i) {
        bool active = false, air = false;
        for (int q = 0; q < 8; ++q) {
          R v = kind(fc(2 * i + CHILDREN[q][0], 2 * j + CHILDREN[q][1], 2 * k + CHILDREN[q][2]));
          if (v > 0) active = true;
          else if (v < 0) air = true;
        }
        L.kind[L.c(i, j, k)] = active ? (R)1 : (air ? (R)-1 : (R)0);
      }
  for (size_t k = 0; k < cz; ++k)
    for (size_t j = 0; j < cy; ++j)
      for (size_t i = 0; i <= cx; ++i) {
        R s = 0;
        for (int q = 0; q < 4; ++q) s += open(0, fu(2 * i, 2 * j + QUARTER[q][0], 2 * k + QUARTER[q][1]));
        L.open_u[(k * cy + j) * (cx + 1) + i] = (R)0.25 * s;
      }
  for (size_t k = 0; k < cz; ++k)
    for (size_t j = 0; j <= cy; ++j)
      for (size_t i = 0; i < cx; ++i) {
        R s = 0;
        for (int q = 0; q < 4; ++q) s += open(1, fv(2 * i + QUARTER[q][0], 2 * j, 2 * k + QUARTER[q][1]));
        L.open_v[(k * (cy + 1) + j) * cx + i] = (R)0.25 * s;
      }
  for (size_t k = 0; k <= cz; ++k)
    for (size_t j = 0; j < cy; ++j)
      for (size_t i = 0; i < cx; ++i) {
        R s = 0;
        for (int q = 0; q < 4; ++q) s += open(2, fw(2 * i + QUARTER[q][0], 2 * j + QUARTER[q][1], 2 * k));
        L.open_w[(k * cy + j) * cx + i] = (R)0.25 * s;
      }
  row_sums(L, nullptr, L.diag.data());
}

void restrict3_tri(size_t nx, size_t ny, const R* fine, Level3& L);

// delta3d_multigrid.rs:258-272
void restrict3(size_t nx, size_t ny, const R* fine, Level3& L) {
  if (g_transfer == 1) { restrict3_tri(nx, ny, fine, L); return; }
  size_t cx = L.nx, cy = L.ny, cz = L.nz;
#pragma omp parallel for schedule(static) num_threads(g_threads) if (cx * cy * cz > 32768)
  for (long long kk = 0; kk < (long long)cz; ++kk) {
    size_t k = (size_t)kk;
    for (size_t j = 0; j < cy; ++j)
      for (size_t i = 0; i < cx; ++i) {
        R s = 0;
        for (int q = 0; q < 8; ++q)
          s += fine[((2 * k + CHILDREN[q][2]) * ny + 2 * j + CHILDREN[q][1]) * nx + 2 * i + CHILDREN[q][0]];
        L.r[L.c(i, j, k)] = (R)0.125 * s;
      }
  }
}

// An alternative grid transfer for experiments, not the reference's (od3_set_transfer(1)):
// cell-centred trilinear prolongation (weights 3/4, 1/4 per axis) that interpolates from active
// coarse cells, takes air cells (kind < 0) as the value 0 and renormalises its weights over the
// cells that are not solid or outside the level; and its adjoint restriction scaled by 1/8 (full
// weighting in the bulk, where every coarse cell's weights sum to 8 over the fine cells).  The coarse operators
// stay the reference's rediscretised ones.
// The trilinear weights of fine cell (i, j, k) over its 8 candidate coarse cells, 0 where the coarse
// cell is outside the level or not active; returns their count and fills idx / w (renormalised).
int tri_weights(const Level3& L, size_t i, size_t j, size_t k, size_t idx[8], R w[8]) {
  long I = (long)(i / 2), J = (long)(j / 2), K = (long)(k / 2);
  long Io = (i & 1) ? I + 1 : I - 1, Jo = (j & 1) ? J + 1 : J - 1, Ko = (k & 1) ? K + 1 : K - 1;
  const long xs[2] = {I, Io}, ys[2] = {J, Jo}, zs[2] = {K, Ko};
  const R wt[2] = {(R)0.75, (R)0.25};
  int n = 0;
  R sum = 0;
  for (int c = 0; c < 2; ++c)
    for (int b = 0; b < 2; ++b)
      for (int a = 0; a < 2; ++a) {
        long x = xs[a], y = ys[b], z = zs[c];
        if (x < 0 || y < 0 || z < 0 || x >= (long)L.nx || y >= (long)L.ny || z >= (long)L.nz) continue;
        size_t cc = L.c((size_t)x, (size_t)y, (size_t)z);
        if (L.kind[cc] == 0) continue;       // solid: no value, renormalise over the rest
        R wq = wt[a] * wt[b] * wt[c];
        sum += wq;
        if (L.kind[cc] < 0) continue;        // air: the value 0 (Dirichlet), weight kept in the sum
        idx[n] = cc;
        w[n] = wq;
        ++n;
      }
  for (int q = 0; q < n; ++q) w[q] = w[q] / sum;
  return n;
}

void restrict3_tri(size_t nx, size_t ny, const R* fine, Level3& L) {
  std::fill(L.r.begin(), L.r.end(), (R)0);
  size_t nz = 2 * L.nz;
  size_t idx[8];
  R w[8];
  for (size_t k = 0; k < nz; ++k)
    for (size_t j = 0; j < ny; ++j)
      for (size_t i = 0; i < nx; ++i) {
        R t = fine[(k * ny + j) * nx + i];
        int n = tri_weights(L, i, j, k, idx, w);
        for (int q = 0; q < n; ++q) L.r[idx[q]] += w[q] * t;
      }
  for (auto& x : L.r) x = (R)0.125 * x;
}

void prolong_add3_tri(size_t nx, size_t ny, R* fine, const Level3& L) {
  size_t nz = 2 * L.nz;
  size_t idx[8];
  R w[8];
  for (size_t k = 0; k < nz; ++k)
    for (size_t j = 0; j < ny; ++j)
      for (size_t i = 0; i < nx; ++i) {
        int n = tri_weights(L, i, j, k, idx, w);
        R v = 0;
        for (int q = 0; q < n; ++q) v += w[q] * L.x[idx[q]];
        fine[(k * ny + j) * nx + i] += v;
      }
}

// delta3d_multigrid.rs:275-287
void prolong_add3(size_t nx, size_t ny, R* fine, const Level3& L) {
  if (g_transfer == 1) { prolong_add3_tri(nx, ny, fine, L); return; }
  size_t cx = L.nx, cy = L.ny, cz = L.nz;
#pragma omp parallel for schedule(static) num_threads(g_threads) if (cx * cy * cz > 32768)
  for (long long kk = 0; kk < (long long)cz; ++kk) {
    size_t k = (size_t)kk;
    for (size_t j = 0; j < cy; ++j)
      for (size_t i = 0; i < cx; ++i) {
        R v = L.x[L.c(i, j, k)];
        for (int q = 0; q < 8; ++q)
          fine[((2 * k + CHILDREN[q][2]) * ny + 2 * j + CHILDREN[q][1]) * nx + 2 * i + CHILDREN[q][0]] += v;
      }
  }
}

// delta3d_multigrid.rs:290-299
void smooth3(Level3& L) {
  row_sums(L, L.x.data(), L.t.data());
  size_t n = L.cells();
  for (size_t c = 0; c < n; ++c)
    if (L.diag[c] > 0) L.x[c] += SMOOTH_DAMPING_3D * (L.r[c] - L.t[c]) / L.diag[c];
}

// One red-black Gauss-Seidel half sweep of a coarse level on cells of `color` ((i+j+k) & 1).
void smooth3_rb(Level3& L, int color) {
  size_t nx = L.nx, ny = L.ny, nz = L.nz;
  row_sums(L, L.x.data(), L.t.data());
  for (size_t k = 0; k < nz; ++k)
    for (size_t j = 0; j < ny; ++j)
      for (size_t i = 0; i < nx; ++i) {
        if ((int)((i + j + k) & 1) != color) continue;
        size_t c = L.c(i, j, k);
        if (L.diag[c] > 0) L.x[c] += (L.r[c] - L.t[c]) / L.diag[c];
      }
}
// `count` smoothing sweeps of a coarse level; `forward` orders each sweep red then black.
void smooth_level(Level3& L, int count, bool forward) {
  for (int s = 0; s < count; ++s) {
    if (!rb_coarse()) { smooth3(L); continue; }
    smooth3_rb(L, forward ? 0 : 1);
    smooth3_rb(L, forward ? 1 : 0);
  }
}

// delta3d_multigrid.rs:303-332
void coarse_cycle3(std::vector<Level3>& levels) {
  size_t last = levels.size() - 1;
  auto big = [&](size_t l) { return levels[l].cells() > TAIL_CELLS; };
  for (size_t l = 0; l <= last; ++l) {
    int sweeps = l == last ? COARSE_SWEEPS_3D : PRE_SWEEPS_3D;
    Level3& L = levels[l];
    std::fill(L.x.begin(), L.x.end(), (R)0);
    if (g_storage && big(l) && l == last) {
      for (int s = 0; s < sweeps; ++s) { smooth_level(L, 1, true); round16(L.x); }
    } else if (!rb_coarse() || l < last) {
      smooth_level(L, sweeps, true);
      if (big(l)) round16(L.x);
    } else { smooth_level(L, sweeps / 2, true); smooth_level(L, sweeps / 2, false); }
    if (l < last) {
      row_sums(L, L.x.data(), L.t.data());
      for (size_t c = 0; c < L.cells(); ++c) L.t[c] = L.r[c] - L.t[c];
      if (big(l)) round16(L.t);
      restrict3(L.nx, L.ny, L.t.data(), levels[l + 1]);
      if (big(l)) round16(levels[l + 1].r);
    }
  }
  for (size_t l = last; l-- > 0;) {
    Level3& L = levels[l];
    prolong_add3(L.nx, L.ny, L.x.data(), levels[l + 1]);
    if (g_storage && big(l)) {
      for (int s = 0; s < POST_SWEEPS_3D; ++s) { smooth_level(L, 1, false); round16(L.x); }
    } else {
      smooth_level(L, POST_SWEEPS_3D, false);
    }
    if (!big(l) && (l == 0 || big(l - 1))) round16(L.x);  // the tail's top level, read by the level above
  }
  if (!big(0) && last == 0) round16(levels[0].x);
}

// ------------------------------------------------------------------- delta3d.rs Volume3
struct Row { bool has; size_t n; R a, it, value; };

struct Volume3 {
  Domain3 d;
  R rho, g_eff, rest;
  bool homogeneous_ghost = false;  // delta3d.rs:110: ghost values 0 (the refinement's increment problem)
  std::vector<R> prec, eta, eta_roundoff, u, v, w, us, vs, ws, p, rhs, res, dir, tmp;
  std::vector<R> saved_u, saved_v, saved_w, saved_p, saved_eta, saved_eta_roundoff, flux_x, flux_y;
  bool has_cut = false;
  Cut3 g;
  bool precondition_cut = true, partial_lid = true;
  R lid_floor = 1;
  bool has_mg = false;
  Multigrid3 mg;
  size_t mg_max_levels = 0;
  bool has_refused = false;
  double refused[8] = {0};
  float tol = 1e-12f;  // squared relative residual target (delta3d_mobile.rs:507)

  size_t c(size_t i, size_t j, size_t k) const { return (k * d.ny + j) * d.nx + i; }
  size_t fu(size_t i, size_t j, size_t k) const { return (k * d.ny + j) * (d.nx + 1) + i; }
  size_t fv(size_t i, size_t j, size_t k) const { return (k * (d.ny + 1) + j) * d.nx + i; }
  size_t fw(size_t i, size_t j, size_t k) const { return (k * d.ny + j) * d.nx + i; }
  size_t col(size_t i, size_t j) const { return j * d.nx + i; }

  // The sparse column set (delta3d_sparse.rs:31-44): one byte per column, 1 in the domain.
  // `next_active` holds a requested set before it replaces `active`.
  bool has_sparse = false;
  std::vector<uint8_t> active, next_active;
  bool column_active(size_t i, size_t j) const { return !has_sparse || active[col(i, j)] != 0; }
  // delta3d_sparse.rs:272-277: every cell of a column outside the set is solid
  bool sparse_solid3(size_t cc) const { return has_sparse && active[cc % (d.nx * d.ny)] == 0; }
  // delta3d_sparse.rs:283-300: an interior u/v face touching a column outside the set, or a w face
  // of such a column, is closed; the faces on the box's boundary keep the box's treatment
  bool sparse_closed3(int axis, size_t f) const {
    if (!has_sparse) return false;
    size_t nx = d.nx, ny = d.ny;
    if (axis == 0) {
      size_t i = f % (nx + 1), j = (f / (nx + 1)) % ny;
      return i > 0 && i < nx && (active[j * nx + i - 1] == 0 || active[j * nx + i] == 0);
    }
    if (axis == 1) {
      size_t i = f % nx, j = (f / nx) % (ny + 1);
      return j > 0 && j < ny && (active[(j - 1) * nx + i] == 0 || active[j * nx + i] == 0);
    }
    return active[f % (nx * ny)] == 0;
  }
  // delta3d_sparse.rs:307-319: the face of axis `axis` at (i, j) touches no column of the set
  bool sparse_outside3(int axis, size_t i, size_t j) const {
    if (!has_sparse) return false;
    if (axis == 0) return !((i > 0 && column_active(i - 1, j)) || (i < d.nx && column_active(i, j)));
    if (axis == 1) return !((j > 0 && column_active(i, j - 1)) || (j < d.ny && column_active(i, j)));
    return !column_active(i, j);
  }

  // delta3d_mobile.rs:92-124
  R height3(size_t i, size_t j) const { return eta[col(i, j)]; }
  bool solid3(size_t cc) const { return (has_cut && g.frac[cc] == 0) || sparse_solid3(cc); }
  bool wet3(size_t i, size_t j, size_t k) const {
    if (solid3(c(i, j, k))) return false;
    return ((R)k + (R)0.5) * d.dx < height3(i, j);
  }
  R open3(int axis, size_t f) const {
    if (sparse_closed3(axis, f)) return 0;
    if (!has_cut) return 1;
    return axis == 0 ? g.open_u[f] : (axis == 1 ? g.open_v[f] : g.open_w[f]);
  }
  // delta3d_mobile.rs:126-134
  void ghost_up3(size_t i, size_t j, size_t k, R& it, R& value) const {
    size_t cc = col(i, j);
    R theta = rmax((height3(i, j) - ((R)k + (R)0.5) * d.dx) / d.dx, SURFACE_THETA_MIN);
    value = homogeneous_ghost ? (R)0 : rho * g_eff * ((eta[cc] - rest) - eta_roundoff[cc]);
    it = (R)1 / theta;
  }
  // delta3d_mobile.rs:136-147
  void ghost_side3(size_t i, size_t j, size_t k, size_t x, size_t y, R& it, R& value) const {
    R zc = ((R)k + (R)0.5) * d.dx;
    R h = height3(i, j);
    R theta = rmax((h - zc) / (h - height3(x, y)), SURFACE_THETA_MIN);
    value = homogeneous_ghost ? (R)0 : rho * g_eff * (zc - rest);
    it = (R)1 / theta;
  }
  // delta3d_mobile.rs:152-188
  void mobile_row(size_t i, size_t j, size_t k, Row row[6]) const {
    size_t nx = d.nx, ny = d.ny, nz = d.nz;
    for (int f = 0; f < 6; ++f) row[f] = Row{false, 0, 0, 0, 0};
    struct Nb { bool ok; size_t x, y; R a; } nb[4] = {
        {i > 0, i > 0 ? i - 1 : 0, j, open3(0, fu(i, j, k))},
        {i + 1 < nx, i + 1, j, open3(0, fu(i + 1, j, k))},
        {j > 0, i, j > 0 ? j - 1 : 0, open3(1, fv(i, j, k))},
        {j + 1 < ny, i, j + 1, open3(1, fv(i, j + 1, k))},
    };
    for (int f = 0; f < 4; ++f) {
      if (!nb[f].ok) continue;
      size_t x = nb[f].x, y = nb[f].y;
      R a = nb[f].a;
      if (a == 0 || solid3(c(x, y, k))) continue;
      if (wet3(x, y, k)) row[f] = Row{true, c(x, y, k), a, 0, 0};
      else {
        R it, b; ghost_side3(i, j, k, x, y, it, b);
        row[f] = Row{false, 0, a, it, b};
      }
    }
    R down = open3(2, fw(i, j, k));
    if (k > 0 && down > 0 && !solid3(c(i, j, k - 1))) row[4] = Row{true, c(i, j, k - 1), down, 0, 0};
    R up = open3(2, fw(i, j, k + 1));
    if (up > 0) {
      if (k + 1 < nz && wet3(i, j, k + 1)) row[5] = Row{true, c(i, j, k + 1), up, 0, 0};
      else {
        R it, b; ghost_up3(i, j, k, it, b);
        row[5] = Row{false, 0, up, it, b};
      }
    }
  }

  template <class F>
  void for_cells(F f) const {
    size_t nx = d.nx, ny = d.ny, nz = d.nz;
#pragma omp parallel for schedule(static) num_threads(g_threads) if (nx * ny * nz > 32768)
    for (long long kk = 0; kk < (long long)nz; ++kk)
      for (size_t j = 0; j < ny; ++j)
        for (size_t i = 0; i < nx; ++i) f(i, j, (size_t)kk);
  }

  // delta3d_mobile.rs:190-213
  void apply_mobile3(const R* pp, R* out) const {
    R inv = (R)1 / (d.dx * d.dx);
    for_cells([&](size_t i, size_t j, size_t k) {
      size_t cc = c(i, j, k);
      if (!wet3(i, j, k)) { out[cc] = 0; return; }
      Row row[6]; mobile_row(i, j, k, row);
      R acc = 0;
      for (int f = 0; f < 6; ++f) {
        if (row[f].has) acc += row[f].a * (pp[cc] - pp[row[f].n]);
        else if (row[f].a > 0) acc += row[f].a * pp[cc] * row[f].it;
      }
      out[cc] = acc * inv;
    });
  }

  // delta3d_mobile.rs:215-241
  void rhs_mobile3(R scale) {
    R inv = (R)1 / (d.dx * d.dx);
    for_cells([&](size_t i, size_t j, size_t k) {
      size_t cc = c(i, j, k);
      if (!wet3(i, j, k)) { rhs[cc] = 0; prec[cc] = 0; return; }
      R b = scale * rhs[cc], diag = 0;
      Row row[6]; mobile_row(i, j, k, row);
      for (int f = 0; f < 6; ++f) {
        if (row[f].has) diag += row[f].a;
        else if (row[f].a > 0) {
          diag += row[f].a * row[f].it;
          b += row[f].a * row[f].value * row[f].it * inv;
        }
      }
      rhs[cc] = b;
      prec[cc] = diag > 0 ? (R)1 / (diag * inv) : (R)0;
    });
  }

  // delta3d_mobile.rs:243-271
  R backward_error_mobile3() const {
    R inv = (R)1 / (d.dx * d.dx);
    size_t nx = d.nx, ny = d.ny, nz = d.nz;
    std::vector<R> plane(nz, (R)0);
#pragma omp parallel for schedule(static) num_threads(g_threads) if (nx * ny * nz > 32768)
    for (long long kk = 0; kk < (long long)nz; ++kk) {
      size_t k = (size_t)kk;
      R worst = 0;
      for (size_t j = 0; j < ny; ++j)
        for (size_t i = 0; i < nx; ++i) {
          if (!wet3(i, j, k)) continue;
          size_t cc = c(i, j, k);
          R pc = std::fabs(p[cc]);
          R acc = 0;
          Row row[6]; mobile_row(i, j, k, row);
          for (int f = 0; f < 6; ++f) {
            if (row[f].has) acc += row[f].a * (pc + std::fabs(p[row[f].n]));
            else if (row[f].a > 0) acc += row[f].a * pc * row[f].it;
          }
          R scale = std::fabs(rhs[cc]) + acc * inv;
          if (scale > 0) worst = rmax(worst, std::fabs(res[cc]) / scale);
        }
      plane[k] = worst;
    }
    R worst = 0;
    for (R x : plane) worst = rmax(worst, x);
    return worst;
  }

  float mobile_roundoff() const { return d.ny == 1 ? ROUNDOFF_BACKWARD_ERROR : ROUNDOFF_BACKWARD_ERROR_3D; }

  // delta3d_mobile.rs:284-343
  void correct_mobile3(R k1) {
    size_t nx = d.nx, ny = d.ny, nz = d.nz;
    R dx = d.dx;
    u = us; v = vs; w = ws;
    for_cells([&](size_t i, size_t j, size_t k) {
      for (int axis = 0; axis < 2; ++axis) {
        if ((axis == 0 && i == 0) || (axis == 1 && j == 0)) continue;
        size_t x = axis == 0 ? i - 1 : i, y = axis == 0 ? j : j - 1;
        size_t l = c(x, y, k), r = c(i, j, k);
        size_t face = axis == 0 ? fu(i, j, k) : fv(i, j, k);
        if (open3(axis, face) == 0 || solid3(l) || solid3(r)) continue;
        bool wl = wet3(x, y, k), wr = wet3(i, j, k);
        R change;
        if (wl && wr) change = k1 * (p[r] - p[l]) / dx;
        else if (wl && !wr) { R a, b; ghost_side3(x, y, k, i, j, a, b); change = k1 * (b - p[l]) * a / dx; }
        else if (!wl && wr) { R a, b; ghost_side3(i, j, k, x, y, a, b); change = k1 * (p[r] - b) * a / dx; }
        else continue;
        if (axis == 0) u[face] -= change; else v[face] -= change;
      }
    });
#pragma omp parallel for schedule(static) num_threads(g_threads) if (nx * ny * nz > 32768)
    for (long long kk = 1; kk <= (long long)nz; ++kk) {
      size_t k = (size_t)kk;
      for (size_t j = 0; j < ny; ++j)
        for (size_t i = 0; i < nx; ++i) {
          size_t f = fw(i, j, k);
          if (open3(2, f) == 0 || !wet3(i, j, k - 1)) continue;
          size_t below = c(i, j, k - 1);
          if (k < nz && wet3(i, j, k)) w[f] -= k1 * (p[c(i, j, k)] - p[below]) / dx;
          else { R a, b; ghost_up3(i, j, k - 1, a, b); w[f] -= k1 * (b - p[below]) * a / dx; }
        }
    }
  }

  // delta3d_mobile.rs:345-394
  void extrapolate_mobile3() {
    size_t nx = d.nx, ny = d.ny, nz = d.nz;
#pragma omp parallel for schedule(static) num_threads(g_threads) if (nx * ny * nz > 32768)
    for (long long jj = 0; jj < (long long)ny; ++jj) {
      size_t j = (size_t)jj;
      for (size_t i = 0; i < nx; ++i)
        for (int axis = 0; axis < 3; ++axis) {
          if ((axis == 0 && i == 0) || (axis == 1 && j == 0)) continue;
          bool has_last = false;
          R last = 0;
          size_t start = axis == 2 ? 1 : 0, end = axis == 2 ? nz + 1 : nz;
          for (size_t k = start; k < end; ++k) {
            size_t f;
            bool solved;
            if (axis == 0) {
              f = fu(i, j, k);
              solved = open3(0, f) > 0 && !solid3(c(i - 1, j, k)) && !solid3(c(i, j, k)) && (wet3(i - 1, j, k) || wet3(i, j, k));
            } else if (axis == 1) {
              f = fv(i, j, k);
              solved = open3(1, f) > 0 && !solid3(c(i, j - 1, k)) && !solid3(c(i, j, k)) && (wet3(i, j - 1, k) || wet3(i, j, k));
            } else {
              f = fw(i, j, k);
              solved = open3(2, f) > 0 && wet3(i, j, k - 1);
            }
            if (open3(axis, f) == 0) continue;
            std::vector<R>& field = axis == 0 ? u : (axis == 1 ? v : w);
            if (solved) { last = field[f]; has_last = true; }
            else if (has_last) field[f] = last;
          }
        }
    }
  }

  // The flux of a moving solid through the parts of a cell's faces that it covers (base aperture
  // minus aperture): in rotation, at the wall's velocity at each face centre; in translation, at
  // the solid's velocity (delta3d.rs:824-852).  Zero terms are not added: a solid at rest, or a
  // volume without the bottom-only base, leaves the divergence as it is.
  bool wall_moves() const {
    if (!has_cut || !g.has_base) return false;
    for (int a = 0; a < 3; ++a)
      if (g.solid_angular[a] != 0.f || g.solid_velocity[a] != 0.f) return true;
    return false;
  }
  R wall_flux(size_t i, size_t j, size_t k) const {
    const Base3& b = g.base;
    const R dx = d.dx;
    auto cu = [&](size_t f) { return b.open_u[f] - g.open_u[f]; };
    auto cv = [&](size_t f) { return b.open_v[f] - g.open_v[f]; };
    auto cw = [&](size_t f) { return b.open_w[f] - g.open_w[f]; };
    if (g.solid_angular[0] != 0.f || g.solid_angular[1] != 0.f || g.solid_angular[2] != 0.f) {
      auto pw = [&](int axis, R x0, R x1, R x2) {
        return wall_velocity(g.solid_velocity, g.solid_angular, g.solid_center, axis, x0, x1, x2);
      };
      const R xc = ((R)i + (R)0.5) * dx, yc = ((R)j + (R)0.5) * dx, zc = ((R)k + (R)0.5) * dx;
      const R x0 = (R)i * dx, x1 = (R)(i + 1) * dx;
      const R y0 = (R)j * dx, y1 = (R)(j + 1) * dx;
      const R z0 = (R)k * dx, z1 = (R)(k + 1) * dx;
      const R fx = cu(fu(i + 1, j, k)) * pw(0, x1, yc, zc) - cu(fu(i, j, k)) * pw(0, x0, yc, zc);
      const R fy = cv(fv(i, j + 1, k)) * pw(1, xc, y1, zc) - cv(fv(i, j, k)) * pw(1, xc, y0, zc);
      const R fz = cw(fw(i, j, k + 1)) * pw(2, xc, yc, z1) - cw(fw(i, j, k)) * pw(2, xc, yc, z0);
      return (fx + fy + fz) / dx;
    }
    const R x = cu(fu(i + 1, j, k)) - cu(fu(i, j, k));
    const R y = cv(fv(i, j + 1, k)) - cv(fv(i, j, k));
    const R z = cw(fw(i, j, k + 1)) - cw(fw(i, j, k));
    return ((R)g.solid_velocity[0] * x + (R)g.solid_velocity[1] * y + (R)g.solid_velocity[2] * z) / dx;
  }

  // delta3d.rs:747-763 and 806-855
  void divergence(const R* uu, const R* vv, const R* ww, R* out) const {
    R dx = d.dx;
    const bool moving = wall_moves();
    for_cells([&](size_t i, size_t j, size_t k) {
      size_t cc = c(i, j, k);
      if (has_cut) {
        if (g.frac[cc] == 0) { out[cc] = 0; return; }
        R fl = g.open_u[fu(i, j, k)] * uu[fu(i, j, k)];
        R fr = g.open_u[fu(i + 1, j, k)] * uu[fu(i + 1, j, k)];
        R ff = g.open_v[fv(i, j, k)] * vv[fv(i, j, k)];
        R fk = g.open_v[fv(i, j + 1, k)] * vv[fv(i, j + 1, k)];
        R fb = g.open_w[fw(i, j, k)] * ww[fw(i, j, k)];
        R ft = g.open_w[fw(i, j, k + 1)] * ww[fw(i, j, k + 1)];
        out[cc] = ((fr - fl + ft - fb) + (fk - ff)) / dx;
        if (moving) out[cc] += wall_flux(i, j, k);
      } else {
        R fl = uu[fu(i, j, k)], fr = uu[fu(i + 1, j, k)];
        R ff = vv[fv(i, j, k)], fk = vv[fv(i, j + 1, k)];
        R fb = ww[fw(i, j, k)], ft = ww[fw(i, j, k + 1)];
        out[cc] = ((fr - fl + ft - fb) + (fk - ff)) / dx;
      }
    });
  }

  // delta3d_mobile.rs:398-433
  void divergence_mobile3(double& all_out, double& plain_out) {
    divergence(u.data(), v.data(), w.data(), tmp.data());
    size_t nx = d.nx, ny = d.ny, nz = d.nz;
    std::vector<R> pall(nz, (R)0), pplain(nz, (R)0);
#pragma omp parallel for schedule(static) num_threads(g_threads) if (nx * ny * nz > 32768)
    for (long long kk = 0; kk < (long long)nz; ++kk) {
      size_t k = (size_t)kk;
      R all = 0, plain = 0;
      for (size_t j = 0; j < ny; ++j)
        for (size_t i = 0; i < nx; ++i) {
          if (!wet3(i, j, k)) continue;
          R dd = std::fabs(tmp[c(i, j, k)]);
          all = rmax(all, dd);
          Row row[6]; mobile_row(i, j, k, row);
          bool ghost = false;
          for (int f = 0; f < 6; ++f) ghost = ghost || (!row[f].has && row[f].a > 0);
          if (!ghost) plain = rmax(plain, dd);
        }
      pall[k] = all; pplain[k] = plain;
    }
    R all = 0, plain = 0;
    for (size_t k = 0; k < nz; ++k) { all = rmax(all, pall[k]); plain = rmax(plain, pplain[k]); }
    R mx = 0;
    for (R x : u) mx = rmax(mx, std::fabs(x));
    for (R x : v) mx = rmax(mx, std::fabs(x));
    for (R x : w) mx = rmax(mx, std::fabs(x));
    R echelle = rmax(mx, PROJECTION_VELOCITY_FLOOR);
    R ratio = mx > 0 ? d.dx / echelle : (R)0;
    all_out = (double)(all * ratio);
    plain_out = (double)(plain * ratio);
  }

  // delta3d.rs:860-876
  R dot(const R* a, const R* b) const {
    return reduce_ordered(p.size(), 64, [&](size_t s, size_t e) {
      R acc = 0;
      for (size_t q = s; q < e; ++q) acc += a[q] * b[q];
      return acc;
    });
  }
  int norm2(const R* a, R& out) const {
    R n = dot(a, a);
    if (!std::isfinite(n)) return NOT_FINITE;
    if (n == 0) {
      for (size_t q = 0; q < p.size(); ++q)
        if (a[q] != 0) return NOT_FINITE;
    }
    out = n;
    return OK;
  }

  // delta3d_mobile.rs:447-461
  int dot_prec3(R& out) const {
    R value = reduce_ordered(p.size(), 64, [&](size_t s, size_t e) {
      R acc = 0;
      for (size_t q = s; q < e; ++q) acc += res[q] * prec[q] * res[q];
      return acc;
    });
    if (!std::isfinite(value)) return NOT_FINITE;
    out = value;
    return OK;
  }
  // delta3d_mobile.rs:435-445
  int prime_mobile3(R beta, R& out) {
    size_t n = dir.size();
#pragma omp parallel for schedule(static) num_threads(g_threads) if (n > 32768)
    for (long long q = 0; q < (long long)n; ++q) {
      R z = prec[q] * res[q];
      dir[q] = beta == 0 ? z : z + beta * dir[q];
    }
    return dot_prec3(out);
  }

  // delta3d_multigrid.rs:357-367
  R fine_kind3(size_t cc) const {
    size_t nx = d.nx, ny = d.ny;
    size_t i = cc % nx, j = (cc / nx) % ny, k = cc / (nx * ny);
    if (wet3(i, j, k)) return 1;
    if (solid3(cc)) return 0;
    return -1;
  }
  // delta3d_multigrid.rs:370-387
  void prepare_multigrid3() {
    if (!has_mg || mg.levels.empty()) return;
    coarsen3(d.nx, d.ny, [&](int axis, size_t f) { return open3(axis, f); }, [&](size_t cc) { return fine_kind3(cc); },
             mg.levels[0]);
    for (size_t l = 1; l < mg.levels.size(); ++l) {
      const Level3& fine = mg.levels[l - 1];
      coarsen3(fine.nx, fine.ny,
               [&](int axis, size_t f) { return axis == 0 ? fine.open_u[f] : (axis == 1 ? fine.open_v[f] : fine.open_w[f]); },
               [&](size_t cc) { return fine.kind[cc]; }, mg.levels[l]);
    }
  }
  // delta3d_multigrid.rs:393-429
  std::vector<R> res_scaled;  // r / sigma in the FP16-storage mode
  void v_cycle3() {
    size_t nx = d.nx, ny = d.ny, cells = p.size();
    std::fill(mg.z.begin(), mg.z.end(), (R)0);
    const R* rv = res.data();
    if (g_storage) {
      double ss = 0;  // r is 0 on dry rows: the rms over all cells, as the device computes it
      for (size_t q = 0; q < cells; ++q) ss += (double)res[q] * (double)res[q];
      double sigma = std::sqrt(ss / (double)cells) * (double)d.dx * (double)d.dx / 6.0;
      R inv = (sigma > 0 && std::isfinite(sigma)) ? (R)(float)(1.0 / sigma) : (R)1;
      res_scaled.resize(cells);
      for (size_t q = 0; q < cells; ++q) res_scaled[q] = res[q] * inv;
      rv = res_scaled.data();
    }
    // one fine sweep: Jacobi (the reference) or a red-black half sweep pair in the given order
    auto fine_sweep = [&](bool forward) {
      if (!rb_fine()) {
        apply_mobile3(mg.z.data(), mg.t.data());
        for (size_t q = 0; q < cells; ++q)
          if (prec[q] > 0) mg.z[q] += SMOOTH_DAMPING_3D * prec[q] * (rv[q] - mg.t[q]);
        return;
      }
      for (int h = 0; h < 2; ++h) {
        int color = forward ? h : 1 - h;
        apply_mobile3(mg.z.data(), mg.t.data());
        for (size_t q = 0; q < cells; ++q) {
          size_t i = q % nx, j = (q / nx) % ny, k = q / (nx * ny);
          if ((int)((i + j + k) & 1) != color) continue;
          if (prec[q] > 0) mg.z[q] += prec[q] * (rv[q] - mg.t[q]);
        }
      }
    };
    for (int s = 0; s < PRE_SWEEPS_3D; ++s) fine_sweep(true);
    round16(mg.z);
    if (!mg.levels.empty()) {
      apply_mobile3(mg.z.data(), mg.t.data());
      for (size_t q = 0; q < cells; ++q) mg.t[q] = rv[q] - mg.t[q];
      restrict3(nx, ny, mg.t.data(), mg.levels[0]);
      round16(mg.levels[0].r);
      coarse_cycle3(mg.levels);
      prolong_add3(nx, ny, mg.z.data(), mg.levels[0]);
      for (size_t q = 0; q < cells; ++q)
        if (prec[q] == 0) mg.z[q] = 0;
    }
    for (int s = 0; s < POST_SWEEPS_3D; ++s) { fine_sweep(false); round16(mg.z); }
    if (g_storage)
      for (size_t q = 0; q < cells; ++q) g_zmax = std::max(g_zmax, (double)std::fabs(mg.z[q]));
  }
  // delta3d_multigrid.rs:433-465
  int prime_multigrid3(R beta, R& out) {
    v_cycle3();
    R rz = dot(res.data(), mg.z.data());
    for (size_t q = 0; q < dir.size(); ++q) dir[q] = beta == 0 ? mg.z[q] : mg.z[q] + beta * dir[q];
    if (!std::isfinite(rz)) return NOT_FINITE;
    out = rz;
    return OK;
  }
  int precondition_multigrid3(R& out) {
    v_cycle3();
    R rz = dot(res.data(), mg.z.data());
    if (!std::isfinite(rz)) return NOT_FINITE;
    out = rz;
    return OK;
  }
  void direction_multigrid3(R beta) {
    for (size_t q = 0; q < dir.size(); ++q) dir[q] = mg.z[q] + beta * dir[q];
  }

  // delta3d.rs:1360-1369
  static uint64_t fingerprint(const std::vector<R>& values) {
    uint64_t h = 0xcbf29ce484222325ull;
    for (R x : values) {
      float f = (float)x;  // the reference hashes f32 bits
      uint32_t bits; std::memcpy(&bits, &f, 4);
      for (int b = 0; b < 4; ++b) { h ^= (uint64_t)((bits >> (8 * b)) & 0xff); h *= 0x100000001b3ull; }
    }
    return h;
  }

  // delta3d_mobile.rs:465-609
  int project_mobile3(R scale, R k1, uint32_t max_iters, double rep[8]) {
    divergence(us.data(), vs.data(), ws.data(), rhs.data());
    rhs_mobile3(scale);
    bool multigrid = has_mg;
    if (multigrid) prepare_multigrid3();
    R b2;
    int e = norm2(rhs.data(), b2);
    if (e) return e;
    for_cells([&](size_t i, size_t j, size_t k) {
      if (!wet3(i, j, k)) p[c(i, j, k)] = 0;
    });
    apply_mobile3(p.data(), tmp.data());
    for (size_t q = 0; q < res.size(); ++q) res[q] = rhs[q] - tmp[q];
    R rr;
    if ((e = norm2(res.data(), rr))) return e;
    R rz = 0;
    bool primed = false;
    uint32_t it = 0;
    R tolr = (R)tol;
    bool floor_stop = false;
    R physical_target = std::numeric_limits<R>::infinity();
    bool has_checkpoint = false;
    uint64_t checkpoint = 0;
    uint32_t power = 1, since = 0;
    R actual_rr;
    bool settled = false;
    double settled_d[2] = {0, 0};
    for (;;) {
      uint32_t before = it;
      while (b2 > 0 && (rr > tolr * b2 || rr > physical_target) && it < max_iters) {
        if (!primed) {
          if ((e = multigrid ? prime_multigrid3(0, rz) : prime_mobile3(0, rz))) return e;
          primed = true;
        }
        apply_mobile3(dir.data(), tmp.data());
        R dq = dot(dir.data(), tmp.data());
        if (!(dq > 0)) break;
        R alpha = rz / dq;
        for (size_t q = 0; q < p.size(); ++q) {
          p[q] += alpha * dir[q];
          res[q] -= alpha * tmp[q];
        }
        R rn;
        if ((e = norm2(res.data(), rn))) return e;
        if (multigrid) {
          R zn;
          if ((e = precondition_multigrid3(zn))) return e;
          direction_multigrid3(zn / rz);
          rz = zn;
        } else {
          R zn;
          if ((e = dot_prec3(zn))) return e;
          R beta = zn / rz;
          R dummy;
          if ((e = prime_mobile3(beta, dummy))) return e;
          rz = zn;
        }
        rr = rn;
        ++it;
      }
      apply_mobile3(p.data(), tmp.data());
      for (size_t q = 0; q < res.size(); ++q) res[q] = rhs[q] - tmp[q];
      R actual;
      if ((e = norm2(res.data(), actual))) return e;
      bool exhausted = it >= max_iters || it == before;
      bool has_measured = false;
      double measured[2] = {0, 0};
      if (actual <= tolr * b2) {
        if (exhausted) { actual_rr = actual; break; }
        correct_mobile3(k1);
        double all, plain;
        divergence_mobile3(all, plain);
        if (plain <= PROJECTION_DIVERGENCE_TOLERANCE) {
          actual_rr = actual; settled = true; settled_d[0] = all; settled_d[1] = plain; break;
        }
        has_measured = true; measured[0] = all; measured[1] = plain;
        R ratio = (R)(PROJECTION_DIVERGENCE_TOLERANCE / plain);
        physical_target = actual * ratio * ratio;
      } else if (exhausted) {
        actual_rr = actual; break;
      }
      if ((float)backward_error_mobile3() <= mobile_roundoff()) {
        floor_stop = true; actual_rr = actual;
        if (has_measured) { settled = true; settled_d[0] = measured[0]; settled_d[1] = measured[1]; }
        break;
      }
      uint64_t state = fingerprint(p);
      if (has_checkpoint && checkpoint == state) {
        floor_stop = true; actual_rr = actual;
        if (has_measured) { settled = true; settled_d[0] = measured[0]; settled_d[1] = measured[1]; }
        break;
      }
      since += 1;
      if (since == power) {
        has_checkpoint = true; checkpoint = state;
        power = power > 0x7fffffffu ? 0xffffffffu : power * 2;
        since = 0;
      }
      rr = actual;
      if ((e = multigrid ? prime_multigrid3(0, rz) : prime_mobile3(0, rz))) return e;
    }
    R residual = b2 > 0 ? std::sqrt(actual_rr / b2) : (R)0;
    double div_all, div_plain;
    if (settled) { div_all = settled_d[0]; div_plain = settled_d[1]; }
    else { correct_mobile3(k1); divergence_mobile3(div_all, div_plain); }
    bool accepted = (actual_rr <= tolr * b2 || floor_stop) && div_plain <= PROJECTION_DIVERGENCE_TOLERANCE;
    rep[0] = 0;                                   // refinements
    rep[1] = (double)it;                          // iterations
    rep[2] = (b2 > 0 && !accepted) ? 1.0 : 0.0;   // degraded
    rep[3] = (double)residual;                    // residual
    rep[4] = div_all;                             // divergence
    rep[5] = floor_stop ? 1.0 : 0.0;              // floor
    rep[6] = (double)backward_error_mobile3();    // backward_error
    rep[7] = div_plain;                           // divergence_plain
    return OK;
  }

  // delta3d_mobile.rs:615-732
  void advect_mobile3(R dt) {
    size_t nx = d.nx, ny = d.ny, nz = d.nz;
    R h = (R)0.5 / d.dx;
    us = u; vs = v; ws = w;
    for (int axis = 0; axis < 2; ++axis) {
      size_t na = axis == 0 ? nx : ny, nb = axis == 0 ? ny : nx;
#pragma omp parallel for schedule(static) num_threads(g_threads) if (nx * ny * nz > 32768)
      for (long long bb = 0; bb < (long long)nb; ++bb) {
        size_t b = (size_t)bb;
        for (size_t a = 1; a < na; ++a)
          for (size_t k = 0; k < nz; ++k) {
            size_t i = axis == 0 ? a : b, j = axis == 0 ? b : a;
            size_t face = axis == 0 ? fu(i, j, k) : fv(i, j, k);
            if (open3(axis, face) == 0) continue;
            auto val = [&](size_t A, size_t B, size_t K) { return axis == 0 ? u[fu(A, B, K)] : v[fv(B, A, K)]; };
            auto vertical = [&](size_t A, size_t B, size_t K) { return axis == 0 ? w[fw(A, B, K)] : w[fw(B, A, K)]; };
            auto transverse = [&](size_t A, size_t B, size_t K) { return axis == 0 ? v[fv(A, B, K)] : u[fu(B, A, K)]; };
            R uc = val(a, b, k);
            R ux = (val(a + 1, b, k) - val(a - 1, b, k)) * h;
            R upv = k + 1 < nz ? val(a, b, k + 1) : uc;
            R dn = k > 0 ? val(a, b, k - 1) : uc;
            R uz = (upv - dn) * h;
            R wc = (R)0.25 * (vertical(a - 1, b, k) + vertical(a, b, k) + vertical(a - 1, b, k + 1) + vertical(a, b, k + 1));
            // the edge of the sparse set reads as the box's edge (delta3d_mobile.rs:664-667)
            auto outside = [&](size_t A, size_t B) { return axis == 0 ? sparse_outside3(0, A, B) : sparse_outside3(1, B, A); };
            R rt = b + 1 < nb && !outside(a, b + 1) ? val(a, b + 1, k) : uc;
            R lf = b > 0 && !outside(a, b - 1) ? val(a, b - 1, k) : uc;
            R uy = (rt - lf) * h;
            R vc = (R)0.25 * (transverse(a - 1, b, k) + transverse(a, b, k) + transverse(a - 1, b + 1, k) + transverse(a, b + 1, k));
            R next = uc - dt * (uc * ux + wc * uz + vc * uy);
            if (axis == 0) us[fu(i, j, k)] = next; else vs[fv(i, j, k)] = next;
          }
      }
    }
#pragma omp parallel for schedule(static) num_threads(g_threads) if (nx * ny * nz > 32768)
    for (long long jj = 0; jj < (long long)ny; ++jj) {
      size_t j = (size_t)jj;
      for (size_t i = 0; i < nx; ++i)
        for (size_t k = 1; k < nz; ++k) {
          size_t f = fw(i, j, k);
          if (open3(2, f) == 0) continue;
          R wc = w[f];
          R rt = i + 1 < nx && !sparse_outside3(2, i + 1, j) ? w[fw(i + 1, j, k)] : wc;
          R lf = i > 0 && !sparse_outside3(2, i - 1, j) ? w[fw(i - 1, j, k)] : wc;
          R wx = (rt - lf) * h;
          R wz = (w[fw(i, j, k + 1)] - w[fw(i, j, k - 1)]) * h;
          R uc = (R)0.25 * (u[fu(i, j, k - 1)] + u[fu(i + 1, j, k - 1)] + u[fu(i, j, k)] + u[fu(i + 1, j, k)]);
          R bk = j + 1 < ny && !sparse_outside3(2, i, j + 1) ? w[fw(i, j + 1, k)] : wc;
          R fr = j > 0 && !sparse_outside3(2, i, j - 1) ? w[fw(i, j - 1, k)] : wc;
          R wy = (bk - fr) * h;
          R vc = (R)0.25 * (v[fv(i, j, k - 1)] + v[fv(i, j + 1, k - 1)] + v[fv(i, j, k)] + v[fv(i, j + 1, k)]);
          ws[f] = wc - dt * (uc * wx + wc * wz + vc * wy);
        }
    }
  }

  // collocated3 (delta3d_coupling.rs:308-328): component a at the centre of a face of axis `axis`,
  // four neighbours (two at the top w face)
  R collocated3(int axis, int a, const size_t p[3]) const {
    if (a == axis) return velocity3(a, p);
    size_t lo[3] = {p[0], p[1], p[2]};
    lo[axis] -= 1;
    size_t hi[3] = {lo[0], lo[1], lo[2]};
    hi[a] += 1;
    if (axis == 2 && p[2] == d.nz) return (R)0.5 * (velocity3(a, lo) + velocity3(a, hi));
    size_t q[3] = {lo[0], lo[1], lo[2]}, r[3] = {hi[0], hi[1], hi[2]};
    q[axis] += 1;
    r[axis] += 1;
    const size_t *b = a < axis ? hi : q, *c2 = a < axis ? q : hi;
    return (R)0.25 * (velocity3(a, lo) + velocity3(a, b) + velocity3(a, c2) + velocity3(a, r));
  }

  // correct_advection3 (delta3d_advection.rs:31-111) of the uncoupled step: + (dt^2/2) sum
  // V_a V_b d_a d_b u on the predicted us/vs/ws, from the velocities at the start of the step.  A
  // direction with a neighbour outside its axis's grid (the box's or the sparse set's) is left out;
  // so is a cross term with a diagonal neighbour outside the set.
  bool advection_correction = false;
  void correct_advection3(R dt) {
    if (!advection_correction) return;
    const size_t dims[3] = {d.nx, d.ny, d.nz};
    const R scale = (R)0.5 * dt * dt;
    for (int axis = 0; axis < 3; ++axis) {
      const size_t end[3] = {d.nx + (axis == 0), d.ny + (axis == 1), d.nz + (axis == 2)};
      for (size_t k = 0; k < end[2]; ++k)
        for (size_t j = 0; j < end[1]; ++j)
          for (size_t i = 0; i < end[0]; ++i) {
            const size_t p[3] = {i, j, k};
            if (p[axis] == 0 || (axis < 2 && p[axis] == dims[axis])) continue;
            const size_t f = axis == 0 ? fu(i, j, k) : (axis == 1 ? fv(i, j, k) : fw(i, j, k));
            if (open3(axis, f) == 0) continue;
            R vel[3];
            for (int a = 0; a < 3; ++a) vel[a] = (R)0 + collocated3(axis, a, p);
            const R c0 = velocity3(axis, p);
            auto shifted = [&](int da, int sa, int db, int sb, size_t out[3]) {
              out[0] = p[0]; out[1] = p[1]; out[2] = p[2];
              if (da >= 0) out[da] = (size_t)((long long)out[da] + sa);
              if (db >= 0) out[db] = (size_t)((long long)out[db] + sb);
            };
            auto at = [&](int da, int sa, int db, int sb) { size_t q[3]; shifted(da, sa, db, sb, q); return velocity3(axis, q); };
            auto outside = [&](int da, int sa, int db, int sb) {
              size_t q[3]; shifted(da, sa, db, sb, q);
              return sparse_outside3(axis, q[0], q[1]);
            };
            auto inside = [&](int a) {
              return p[a] > 0 && p[a] + 1 < end[a] && !outside(a, 1, -1, 0) && !outside(a, -1, -1, 0);
            };
            R acc = 0;
            for (int a = 0; a < 3; ++a) {
              if (!inside(a)) continue;
              acc += vel[a] * vel[a] * (at(a, 1, -1, 0) - (R)2 * c0 + at(a, -1, -1, 0));
              for (int b = a + 1; b < 3; ++b) {
                if (!inside(b)) continue;
                if (outside(a, 1, b, 1) || outside(a, 1, b, -1) || outside(a, -1, b, 1) || outside(a, -1, b, -1)) continue;
                R cross = at(a, 1, b, 1) - at(a, 1, b, -1) - at(a, -1, b, 1) + at(a, -1, b, -1);
                acc += (R)2 * vel[a] * vel[b] * (R)0.25 * cross;
              }
            }
            const R term = scale * acc / (d.dx * d.dx);
            if (axis == 0) us[f] += term; else if (axis == 1) vs[f] += term; else ws[f] += term;
          }
    }
  }

  // delta3d_mobile.rs:734-782
  void transport_mobile3(R transport) {
    size_t nx = d.nx, ny = d.ny, nz = d.nz;
    R dx = d.dx;
    std::fill(flux_x.begin(), flux_x.end(), (R)0);
    std::fill(flux_y.begin(), flux_y.end(), (R)0);
    for (size_t j = 0; j < ny; ++j)
      for (size_t i = 0; i < nx; ++i)
        for (int axis = 0; axis < 2; ++axis) {
          if ((axis == 0 && i == 0) || (axis == 1 && j == 0)) continue;
          size_t x = axis == 0 ? i - 1 : i, y = axis == 0 ? j : j - 1;
          R surface = (R)0.5 * (eta[col(x, y)] + eta[col(i, j)]);
          R q = 0;
          for (size_t k = 0; k < nz; ++k) {
            R wet = clamp01((surface - (R)k * dx) / dx);
            if (wet == 0) break;
            R uu, a;
            if (axis == 0) { size_t f = fu(i, j, k); uu = u[f]; a = open3(0, f); }
            else { size_t f = fv(i, j, k); uu = v[f]; a = open3(1, f); }
            q += a * uu * dx * wet;
          }
          if (axis == 0) flux_x[j * (nx + 1) + i] = q; else flux_y[j * nx + i] = q;
        }
    for (size_t j = 0; j < ny; ++j)
      for (size_t i = 0; i < nx; ++i) {
        size_t cc = col(i, j);
        R x = flux_x[j * (nx + 1) + i + 1] - flux_x[j * (nx + 1) + i];
        R y = flux_y[(j + 1) * nx + i] - flux_y[j * nx + i];
        R increment = -transport * (x + y) - eta_roundoff[cc];
        R height = eta[cc] + increment;
        eta_roundoff[cc] = (height - eta[cc]) - increment;
        eta[cc] = height;
      }
  }

  // delta3d_mobile.rs:801-813
  bool mobile_in_bounds() const {
    R dx = d.dx;
    R top = (R)(d.nz - 1) * dx;
    for (size_t j = 0; j < d.ny; ++j)
      for (size_t i = 0; i < d.nx; ++i) {
        R e = height3(i, j);
        R floor = has_cut ? g.floor[col(i, j)] + (R)2 * dx : (R)2 * dx;
        if (!(e >= floor && e <= top)) return false;
      }
    return true;
  }

  // delta3d.rs:557-591
  void prec_cut() {
    size_t nx = d.nx, ny = d.ny, nz = d.nz;
    R inv = (R)1 / (d.dx * d.dx);
    for (size_t k = 0; k < nz; ++k)
      for (size_t j = 0; j < ny; ++j)
        for (size_t i = 0; i < nx; ++i) {
          size_t cc = c(i, j, k);
          if (g.frac[cc] == 0) { prec[cc] = 0; continue; }
          R diag = 0;
          auto face = [&](R a, bool has, size_t m, bool lid) {
            if (a == 0) return;
            if (has) { if (g.frac[m] > 0) diag += a; }
            else if (lid) diag += (R)2 * a;
          };
          face(g.open_u[fu(i, j, k)], i > 0, c(i, j, k) - 1, false);
          face(g.open_u[fu(i + 1, j, k)], i + 1 < nx, cc + 1, false);
          face(g.open_v[fv(i, j, k)], j > 0, cc - nx, false);
          face(g.open_v[fv(i, j + 1, k)], j + 1 < ny, cc + nx, false);
          face(g.open_w[fw(i, j, k)], k > 0, cc - nx * ny, false);
          face(g.open_w[fw(i, j, k + 1)], k + 1 < nz, cc + nx * ny, true);
          prec[cc] = diag > 0 ? (R)1 / (diag * inv) : (R)0;
        }
  }

  // perturbation_volume (delta3d_balance.rs:105-113): f64, in column order
  double perturbation_volume() const {
    const double area = (double)(float)d.dx * (double)(float)d.dx, r = (double)(float)rest;
    double total = 0;
    for (size_t q = 0; q < eta.size(); ++q) total += ((double)eta[q] - (double)eta_roundoff[q]) - r;
    return total * area;
  }

  // ---- the level change (delta3d_levels.rs:38-292)
  double compensated(size_t i, size_t j) const { return (double)eta[col(i, j)] - (double)eta_roundoff[col(i, j)]; }
  // delta3d_levels.rs:76-90: centred inside, one-sided at the box's or the set's edge
  double surface_slope(size_t i, size_t j, int axis) const {
    size_t n = axis == 0 ? d.nx : d.ny, k = axis == 0 ? i : j;
    if (n < 2) return 0;
    auto at = [&](size_t m) { return axis == 0 ? compensated(m, j) : compensated(i, m); };
    auto inside = [&](size_t m) { return axis == 0 ? column_active(m, j) : column_active(i, m); };
    size_t lo = k > 0 && inside(k - 1) ? k - 1 : k;
    size_t hi = k + 1 < n && inside(k + 1) ? k + 1 : k;
    if (hi == lo) return 0;
    return (at(hi) - at(lo)) / ((double)(hi - lo) * (double)(float)d.dx);
  }
  // delta3d_levels.rs:95-107
  double surface_twist(size_t i, size_t j) const {
    size_t nx = d.nx, ny = d.ny;
    if (i == 0 || j == 0 || i + 1 >= nx || j + 1 >= ny) return 0;
    if (!column_active(i - 1, j - 1) || !column_active(i + 1, j - 1) || !column_active(i - 1, j + 1) ||
        !column_active(i + 1, j + 1))
      return 0;
    double dx64 = (double)(float)d.dx;
    return (compensated(i + 1, j + 1) - compensated(i + 1, j - 1) - compensated(i - 1, j + 1) + compensated(i - 1, j - 1)) /
           (4. * dx64 * dx64);
  }
  R velocity3(int axis, const size_t p[3]) const {
    return axis == 0 ? u[fu(p[0], p[1], p[2])] : (axis == 1 ? v[fv(p[0], p[1], p[2])] : w[fw(p[0], p[1], p[2])]);
  }
  // staggered_at (delta3d_levels.rs:159-200): trilinear on the staggered grid, indices clamped
  float staggered_at(int axis, const double rel[3]) const {
    const size_t dims[3] = {d.nx + (axis == 0), d.ny + (axis == 1), d.nz + (axis == 2)};
    const size_t cells[3] = {d.nx, d.ny, d.nz};
    size_t base[3];
    double frac[3];
    for (int a = 0; a < 3; ++a) {
      double f = rel[a] * (double)cells[a] - (a == axis ? 0. : 0.5);
      double top = (double)(dims[a] - 1);
      f = std::min(std::max(f, 0.), top);
      size_t b = std::min((size_t)std::floor(f), dims[a] >= 2 ? dims[a] - 2 : 0);
      base[a] = b;
      frac[a] = dims[a] < 2 ? 0. : f - (double)b;
    }
    if (has_sparse) return (float)staggered_in_set(axis, base, frac, dims);
    double acc = 0;
    for (int corner = 0; corner < 8; ++corner) {
      size_t p[3] = {base[0], base[1], base[2]};
      double weight = 1;
      for (int a = 0; a < 3; ++a) {
        bool up = (corner >> a) & 1;
        if (dims[a] < 2) { if (up) weight = 0; continue; }
        if (up) { p[a] += 1; weight *= frac[a]; } else { weight *= 1. - frac[a]; }
      }
      if (weight != 0.) acc += weight * (double)(float)velocity3(axis, p);
    }
    return (float)acc;
  }
  // staggered_in_set (delta3d_levels.rs:204-245): a corner outside the set's grid takes, axis by
  // axis, its neighbour's value inside the set
  double staggered_in_set(int axis, const size_t base[3], const double frac[3], const size_t dims[3]) const {
    double values[8];
    bool outside[8];
    for (int corner = 0; corner < 8; ++corner) {
      size_t p[3] = {base[0], base[1], base[2]};
      for (int a = 0; a < 3; ++a) if (((corner >> a) & 1) && dims[a] >= 2) p[a] += 1;
      values[corner] = (double)(float)velocity3(axis, p);
      outside[corner] = sparse_outside3(axis, p[0], p[1]);
    }
    for (int a = 0; a < 3; ++a) {
      if (dims[a] < 2) continue;
      for (int corner = 0; corner < 8; ++corner) {
        if ((corner >> a) & 1) continue;
        int up = corner | (1 << a);
        if (outside[corner] && !outside[up]) { values[corner] = values[up]; outside[corner] = false; }
        else if (outside[up] && !outside[corner]) { values[up] = values[corner]; outside[up] = false; }
      }
    }
    double acc = 0;
    for (int corner = 0; corner < 8; ++corner) {
      double weight = 1;
      for (int a = 0; a < 3; ++a) {
        bool up = (corner >> a) & 1;
        if (dims[a] < 2) { if (up) weight = 0; continue; }
        weight *= up ? frac[a] : 1. - frac[a];
      }
      if (weight != 0.) acc += weight * values[corner];
    }
    return acc;
  }
  // resample_surface (delta3d_levels.rs:109-155)
  void resample_surface(const Volume3& src) {
    const Domain3 &dd_ = d, &ss = src.d;
    const double dd = (double)(float)dd_.dx;
    const double sx = (double)dd_.nx * dd / (double)ss.nx, sy = (double)dd_.ny * dd / (double)ss.ny;
    for (size_t j = 0; j < dd_.ny; ++j) {
      const double y0 = (double)j * dd, y1 = (double)(j + 1) * dd;
      for (size_t i = 0; i < dd_.nx; ++i) {
        const double x0 = (double)i * dd, x1 = (double)(i + 1) * dd;
        double total = 0;
        const size_t i0 = (size_t)std::floor(x0 / sx), i1 = std::min((size_t)std::ceil(x1 / sx), ss.nx);
        const size_t j0 = (size_t)std::floor(y0 / sy), j1 = std::min((size_t)std::ceil(y1 / sy), ss.ny);
        const size_t cc = col(i, j);
        if (!column_active(i, j)) { eta[cc] = rest; eta_roundoff[cc] = 0; continue; }
        for (size_t sj = j0; sj < j1; ++sj) {
          const double ya = std::max(y0, (double)sj * sy), yb = std::min(y1, (double)(sj + 1) * sy);
          if (yb <= ya) continue;
          for (size_t si = i0; si < i1; ++si) {
            const double xa = std::max(x0, (double)si * sx), xb = std::min(x1, (double)(si + 1) * sx);
            if (xb <= xa) continue;
            const double area = (xb - xa) * (yb - ya);
            const double cx = 0.5 * (xa + xb) - ((double)si + 0.5) * sx, cy = 0.5 * (ya + yb) - ((double)sj + 0.5) * sy;
            double h;
            if (src.column_active(si, sj))
              h = src.compensated(si, sj) + src.surface_slope(si, sj, 0) * cx + src.surface_slope(si, sj, 1) * cy +
                  src.surface_twist(si, sj) * cx * cy;
            else
              h = (double)(float)src.rest;
            total += area * h;
          }
        }
        const double h = total / (dd * dd);
        eta[cc] = (R)(float)h;
        eta_roundoff[cc] = (R)(float)((double)(float)eta[cc] - h);
      }
    }
  }
  // resample_faces (delta3d_levels.rs:249-288)
  void resample_faces(const Volume3& src) {
    const size_t n = std::max((size_t)std::ceil((double)(float)d.dx / (double)(float)src.d.dx), (size_t)1);
    const double cells[3] = {(double)d.nx, (double)d.ny, (double)d.nz};
    for (int axis = 0; axis < 3; ++axis) {
      const size_t dims[3] = {d.nx + (axis == 0), d.ny + (axis == 1), d.nz + (axis == 2)};
      const int t1 = (axis + 1) % 3, t2 = (axis + 2) % 3;
      for (size_t k = 0; k < dims[2]; ++k)
        for (size_t j = 0; j < dims[1]; ++j)
          for (size_t i = 0; i < dims[0]; ++i) {
            const size_t p[3] = {i, j, k};
            double centre[3];
            for (int a = 0; a < 3; ++a) centre[a] = ((double)p[a] + (a == axis ? 0. : 0.5)) / cells[a];
            double acc = 0;
            for (size_t a = 0; a < n; ++a)
              for (size_t b = 0; b < n; ++b) {
                double q[3] = {centre[0], centre[1], centre[2]};
                q[t1] += (((double)a + 0.5) / (double)n - 0.5) / cells[t1];
                q[t2] += (((double)b + 0.5) / (double)n - 0.5) / cells[t2];
                acc += (double)src.staggered_at(axis, q);
              }
            const float val = (float)(acc / (double)(n * n));
            if (axis == 0) u[fu(i, j, k)] = val; else if (axis == 1) v[fv(i, j, k)] = val; else w[fw(i, j, k)] = val;
          }
    }
  }

  // delta3d.rs:666-690
  void close_walls() {
    size_t nx = d.nx, ny = d.ny, nz = d.nz;
    for (size_t k = 0; k < nz; ++k) {
      for (size_t j = 0; j < ny; ++j) { u[fu(0, j, k)] = 0; u[fu(nx, j, k)] = 0; }
      for (size_t i = 0; i < nx; ++i) { v[fv(i, 0, k)] = 0; v[fv(i, ny, k)] = 0; }
    }
    for (size_t j = 0; j < ny; ++j)
      for (size_t i = 0; i < nx; ++i) w[fw(i, j, 0)] = 0;
    if (has_cut) {
      for (size_t q = 0; q < u.size(); ++q) if (g.open_u[q] == 0) u[q] = 0;
      for (size_t q = 0; q < v.size(); ++q) if (g.open_v[q] == 0) v[q] = 0;
      for (size_t q = 0; q < w.size(); ++q) if (g.open_w[q] == 0) w[q] = 0;
    }
  }

  // clear_column_faces (delta3d_sparse.rs:213-233): zeroes the column's two u faces, two v faces
  // and nz+1 w faces per layer, and returns the largest |velocity| it cleared.
  float clear_column_faces(size_t i, size_t j) {
    float worst = 0;
    for (size_t k = 0; k < d.nz; ++k) {
      for (size_t f : {fu(i, j, k), fu(i + 1, j, k)}) { worst = std::max(worst, std::fabs((float)u[f])); u[f] = 0; }
      for (size_t f : {fv(i, j, k), fv(i, j + 1, k)}) { worst = std::max(worst, std::fabs((float)v[f])); v[f] = 0; }
    }
    for (size_t k = 0; k <= d.nz; ++k) { size_t f = fw(i, j, k); worst = std::max(worst, std::fabs((float)w[f])); w[f] = 0; }
    return worst;
  }

  // close_sparse_walls (delta3d_sparse.rs:236-247)
  void close_sparse_walls() {
    if (!has_sparse) return;
    for (size_t j = 0; j < d.ny; ++j)
      for (size_t i = 0; i < d.nx; ++i)
        if (!column_active(i, j)) clear_column_faces(i, j);
  }

  // sparse_surface_ok (delta3d_sparse.rs:327-332): outside the set the surface is `rest`, to the bit
  bool sparse_surface_ok(const float* e, float r) const {
    if (!has_sparse) return true;
    uint32_t rb; std::memcpy(&rb, &r, 4);
    for (size_t q = 0; q < active.size(); ++q) {
      uint32_t eb; std::memcpy(&eb, &e[q], 4);
      if (!active[q] && eb != rb) return false;
    }
    return true;
  }

  // apply_sparse (delta3d_sparse.rs:181-210): `next_active` replaces `active`; a column that leaves
  // goes to rest (surface, roundoff, pressure, faces) and what it carried is counted.
  // out: activated, deactivated, active columns, volume removed, height removed, velocity removed
  void apply_sparse(double out[6]) {
    size_t deact = 0, act = 0;
    double volume = 0;
    float height = 0, speed = 0;
    const double area = (double)d.dx * (double)d.dx;
    for (size_t j = 0; j < d.ny; ++j)
      for (size_t i = 0; i < d.nx; ++i) {
        size_t cc = col(i, j);
        bool was = active[cc] != 0, will = next_active[cc] != 0;
        if (was && !will) {
          ++deact;
          double h = ((double)(float)eta[cc] - (double)(float)eta_roundoff[cc]) - (double)(float)rest;
          volume += h * area;
          height = std::max(height, std::fabs((float)eta[cc] - (float)rest));
          eta[cc] = rest;
          eta_roundoff[cc] = 0;
          for (size_t k = 0; k < d.nz; ++k) p[c(i, j, k)] = 0;
          speed = std::max(speed, clear_column_faces(i, j));
        } else if (!was && will) {
          ++act;
        }
      }
    std::swap(active, next_active);
    size_t count = 0;
    for (uint8_t a : active) count += a != 0;
    out[0] = (double)act; out[1] = (double)deact; out[2] = (double)count;
    out[3] = volume; out[4] = height; out[5] = speed;
  }

  // delta3d_mobile.rs:819-927
  int step_surface_mobile(uint64_t duration_us, uint32_t max_iters, double rep[8]) {
    if (duration_us == 0 || duration_us > (1ull << 53)) return NOT_FINITE;
    double dt = (double)duration_us * 1e-6;
    R dx = d.dx;
    if (g_eff <= 0 || dt * dt * (double)g_eff / (double)dx > 1. || !mobile_in_bounds()) return DOMAIN;
    R scale = (R)(-(double)rho / dt);
    R correction = (R)(dt / (double)rho);
    R transport = (R)(dt / (double)dx);
    R advection = (R)dt;
    if (!std::isfinite(scale) || !std::isfinite(correction) || correction == 0 || !std::isfinite(transport) ||
        transport == 0 || !(advection > 0))
      return NOT_FINITE;
    saved_u = u; saved_v = v; saved_w = w; saved_p = p; saved_eta = eta; saved_eta_roundoff = eta_roundoff;
    int e = [&]() -> int {
      advect_mobile3(advection);
      correct_advection3(advection);  // the second-order term, when enabled (delta3d_mobile.rs:858-860)
      int err = project_mobile3(scale, correction, max_iters, rep);
      if (err) return err;
      if (rep[2] != 0) {
        has_refused = true;
        std::memcpy(refused, rep, sizeof(refused));
        return CONVERGENCE;
      }
      extrapolate_mobile3();
      transport_mobile3(transport);
      const std::vector<R>* fields[] = {&u, &v, &w, &p, &eta, &eta_roundoff, &us, &vs, &ws, &rhs, &res, &dir, &tmp, &prec};
      for (auto f : fields)
        for (R x : *f)
          if (!std::isfinite(x)) return NOT_FINITE;
      if (!std::isfinite(rep[3]) || !std::isfinite(rep[4])) return NOT_FINITE;
      if (!mobile_in_bounds()) return DOMAIN;
      return OK;
    }();
    if (e) {
      u = saved_u; v = saved_v; w = saved_w; p = saved_p; eta = saved_eta; eta_roundoff = saved_eta_roundoff;
    }
    if (has_cut) prec_cut();
    return e;
  }

  // ------------------------------------------------------------------ the linear (fixed-lid) path
  // delta3d.rs:697-715.  The partial-lid branch needs a lid aperture strictly between 0 and 1,
  // which only a hull piercing the lid produces; the linear step refuses any lid that is not fully
  // open (delta3d.rs:1261-1268), so the fully open value is the one used here.
  R lid(size_t i, size_t j) const {
    size_t cc = col(i, j);
    return rho * g_eff * ((eta[cc] - d.z0()) - eta_roundoff[cc]);
  }

  // apply (delta3d.rs:721-744) and apply_cut (:771-802): Neumann walls and bottom, homogeneous
  // Dirichlet lid half a cell above the top layer; cut rows weighted by the apertures.
  void apply_linear(const R* pp, R* out) const {
    size_t nx = d.nx, ny = d.ny, nz = d.nz;
    R inv = (R)1 / (d.dx * d.dx);
    for_cells([&](size_t i, size_t j, size_t k) {
      size_t cc = c(i, j, k);
      if (!has_cut) {
        R pc = pp[cc];
        R acc = 0;
        if (i > 0) acc += pc - pp[cc - 1];
        if (i + 1 < nx) acc += pc - pp[cc + 1];
        if (j > 0) acc += pc - pp[cc - nx];
        if (j + 1 < ny) acc += pc - pp[cc + nx];
        if (k > 0) acc += pc - pp[cc - nx * ny];
        if (k + 1 < nz) acc += pc - pp[cc + nx * ny]; else acc += (R)2 * pc;
        out[cc] = acc * inv;
        return;
      }
      if (g.frac[cc] == 0) { out[cc] = 0; return; }
      R acc = 0;
      auto face = [&](R a, bool has, size_t m, bool top) {
        if (a == 0) return;
        if (has) { if (g.frac[m] > 0) acc += a * (pp[cc] - pp[m]); }
        else if (top) acc += (R)2 * a * pp[cc];
      };
      face(g.open_u[fu(i, j, k)], i > 0, cc - 1, false);
      face(g.open_u[fu(i + 1, j, k)], i + 1 < nx, cc + 1, false);
      face(g.open_v[fv(i, j, k)], j > 0, cc - nx, false);
      face(g.open_v[fv(i, j + 1, k)], j + 1 < ny, cc + nx, false);
      face(g.open_w[fw(i, j, k)], k > 0, cc - nx * ny, false);
      face(g.open_w[fw(i, j, k + 1)], k + 1 < nz, cc + nx * ny, true);
      out[cc] = acc * inv;
    });
  }

  // The right-hand side of project (delta3d.rs:1066-1086): scale * div, the lid value entering
  // through the top layer, zero on solid cells.
  void rhs_linear(R scale) {
    size_t nz = d.nz;
    R inv = (R)1 / (d.dx * d.dx);
    for_cells([&](size_t i, size_t j, size_t k) {
      size_t cc = c(i, j, k);
      R b = scale * rhs[cc];
      if (has_cut) {
        if (g.frac[cc] == 0) b = 0;
        else if (k + 1 == nz) {
          R a = g.open_w[fw(i, j, k + 1)];
          if (a > 0) b += (R)2 * a * lid(i, j) * inv;
        }
      } else if (k + 1 == nz) {
        b += (R)2 * lid(i, j) * inv;
      }
      rhs[cc] = b;
    });
  }

  // backward_error (delta3d.rs:881-907) and backward_error_cut (:909-945).
  R backward_error_linear() const {
    size_t nx = d.nx, ny = d.ny, nz = d.nz;
    R inv = (R)1 / (d.dx * d.dx);
    std::vector<R> part(nz, (R)0);
#pragma omp parallel for schedule(static) num_threads(g_threads) if (nx * ny * nz > 32768)
    for (long long kk = 0; kk < (long long)nz; ++kk) {
      size_t k = (size_t)kk;
      R worst = 0;
      for (size_t j = 0; j < ny; ++j)
        for (size_t i = 0; i < nx; ++i) {
          size_t cc = c(i, j, k);
          R pc = std::fabs(p[cc]);
          R acc = 0;
          if (!has_cut) {
            if (i > 0) acc += pc + std::fabs(p[cc - 1]);
            if (i + 1 < nx) acc += pc + std::fabs(p[cc + 1]);
            if (j > 0) acc += pc + std::fabs(p[cc - nx]);
            if (j + 1 < ny) acc += pc + std::fabs(p[cc + nx]);
            if (k > 0) acc += pc + std::fabs(p[cc - nx * ny]);
            if (k + 1 < nz) acc += pc + std::fabs(p[cc + nx * ny]); else acc += pc * (R)2;
          } else {
            if (g.frac[cc] == 0) continue;
            auto face = [&](R a, bool has, size_t m, bool top) {
              if (a == 0) return;
              if (has) { if (g.frac[m] > 0) acc += a * (pc + std::fabs(p[m])); }
              else if (top) acc += a * pc * (R)2;
            };
            face(g.open_u[fu(i, j, k)], i > 0, cc - 1, false);
            face(g.open_u[fu(i + 1, j, k)], i + 1 < nx, cc + 1, false);
            face(g.open_v[fv(i, j, k)], j > 0, cc - nx, false);
            face(g.open_v[fv(i, j + 1, k)], j + 1 < ny, cc + nx, false);
            face(g.open_w[fw(i, j, k)], k > 0, cc - nx * ny, false);
            face(g.open_w[fw(i, j, k + 1)], k + 1 < nz, cc + nx * ny, true);
          }
          R scale = std::fabs(rhs[cc]) + acc * inv;
          if (scale > 0) worst = rmax(worst, std::fabs(res[cc]) / scale);
        }
      part[k] = worst;
    }
    R worst = 0;
    for (R x : part) worst = rmax(worst, x);
    return worst;
  }

  // correct (delta3d.rs:949-987) and correct_cut (:989-1038).
  void correct_linear(R k1) {
    size_t nx = d.nx, ny = d.ny, nz = d.nz;
    R dx = d.dx;
    u = us; v = vs; w = ws;
    for (size_t k = 0; k < nz; ++k)
      for (size_t j = 0; j < ny; ++j)
        for (size_t i = 1; i < nx; ++i) {
          size_t f = fu(i, j, k), l = c(i - 1, j, k), r = c(i, j, k);
          if (!has_cut || (g.open_u[f] != 0 && g.frac[l] > 0 && g.frac[r] > 0)) u[f] -= k1 * (p[r] - p[l]) / dx;
        }
    for (size_t k = 0; k < nz; ++k)
      for (size_t j = 1; j < ny; ++j)
        for (size_t i = 0; i < nx; ++i) {
          size_t f = fv(i, j, k), a = c(i, j - 1, k), b = c(i, j, k);
          if (!has_cut || (g.open_v[f] != 0 && g.frac[a] > 0 && g.frac[b] > 0)) v[f] -= k1 * (p[b] - p[a]) / dx;
        }
    for (size_t k = 1; k <= nz; ++k)
      for (size_t j = 0; j < ny; ++j)
        for (size_t i = 0; i < nx; ++i) {
          size_t f = fw(i, j, k), below = c(i, j, k - 1);
          if (has_cut && (g.open_w[f] == 0 || g.frac[below] == 0)) continue;
          if (k < nz) {
            size_t above = c(i, j, k);
            if (!has_cut || g.frac[above] > 0) w[f] -= k1 * (p[above] - p[below]) / dx;
          } else {
            w[f] -= k1 * (lid(i, j) - p[below]) / ((R)0.5 * dx);
          }
        }
  }

  // divergence_metric (delta3d.rs:1043-1052): max|div u| dx / max|u|, every row plain.
  double divergence_metric_linear() {
    divergence(u.data(), v.data(), w.data(), tmp.data());
    R dmax = 0;
    for (R x : tmp) dmax = rmax(dmax, std::fabs(x));
    R umax = 0;
    for (R x : u) umax = rmax(umax, std::fabs(x));
    for (R x : v) umax = rmax(umax, std::fabs(x));
    for (R x : w) umax = rmax(umax, std::fabs(x));
    R ratio = umax > 0 ? d.dx / umax : (R)0;
    return (double)(dmax * ratio);
  }

  // project (delta3d.rs:1060-1196): CG from p = 0, or Jacobi-PCG on a cut bottom with ny > 1
  // (precondition_cut, S326); the acceptance, tightening and floor logic of project_mobile3.
  int project_linear(R scale, R k1, uint32_t max_iters, double rep[8]) {
    divergence(us.data(), vs.data(), ws.data(), rhs.data());
    rhs_linear(scale);
    R b2;
    int e = norm2(rhs.data(), b2);
    if (e) return e;
    std::fill(p.begin(), p.end(), (R)0);
    res = rhs;
    R rr = b2;
    bool primed = false;
    const bool jacobi = has_cut && precondition_cut && d.ny > 1;
    R rz = 0;
    uint32_t it = 0;
    R tolr = (R)tol;
    bool floor_stop = false;
    R physical_target = std::numeric_limits<R>::infinity();
    bool has_checkpoint = false;
    uint64_t checkpoint = 0;
    uint32_t power = 1, since = 0;
    R actual_rr;
    bool settled = false;
    double settled_d = 0;
    for (;;) {
      uint32_t before = it;
      while (b2 > 0 && (rr > tolr * b2 || rr > physical_target) && it < max_iters) {
        if (!primed) {
          if (jacobi) { if ((e = prime_mobile3(0, rz))) return e; }
          else dir = res;
          primed = true;
        }
        apply_linear(dir.data(), tmp.data());
        R dq = dot(dir.data(), tmp.data());
        if (!(dq > 0)) break;
        R alpha = jacobi ? rz / dq : rr / dq;
        for (size_t q = 0; q < p.size(); ++q) {
          p[q] += alpha * dir[q];
          res[q] -= alpha * tmp[q];
        }
        R rn;
        if ((e = norm2(res.data(), rn))) return e;
        if (jacobi) {
          R zn;
          if ((e = dot_prec3(zn))) return e;
          R beta = zn / rz;
          R dummy;
          if ((e = prime_mobile3(beta, dummy))) return e;
          rz = zn;
        } else {
          R beta = rn / rr;
          for (size_t q = 0; q < dir.size(); ++q) dir[q] = res[q] + beta * dir[q];
        }
        rr = rn;
        ++it;
      }
      apply_linear(p.data(), tmp.data());
      for (size_t q = 0; q < res.size(); ++q) res[q] = rhs[q] - tmp[q];
      R actual;
      if ((e = norm2(res.data(), actual))) return e;
      bool exhausted = it >= max_iters || it == before;
      bool has_measured = false;
      double measured = 0;
      if (actual <= tolr * b2) {
        if (exhausted) { actual_rr = actual; break; }
        correct_linear(k1);
        double reached = divergence_metric_linear();
        if (reached <= PROJECTION_DIVERGENCE_TOLERANCE) { actual_rr = actual; settled = true; settled_d = reached; break; }
        has_measured = true; measured = reached;
        R ratio = (R)(PROJECTION_DIVERGENCE_TOLERANCE / reached);
        physical_target = actual * ratio * ratio;
      } else if (exhausted) {
        actual_rr = actual; break;
      }
      if ((float)backward_error_linear() <= ROUNDOFF_BACKWARD_ERROR_3D) {
        floor_stop = true; actual_rr = actual;
        if (has_measured) { settled = true; settled_d = measured; }
        break;
      }
      uint64_t state = fingerprint(p);
      if (has_checkpoint && checkpoint == state) {
        floor_stop = true; actual_rr = actual;
        if (has_measured) { settled = true; settled_d = measured; }
        break;
      }
      since += 1;
      if (since == power) {
        has_checkpoint = true; checkpoint = state;
        power = power > 0x7fffffffu ? 0xffffffffu : power * 2;
        since = 0;
      }
      rr = actual;
      if (jacobi) { if ((e = prime_mobile3(0, rz))) return e; }
      else dir = res;
    }
    R residual = b2 > 0 ? std::sqrt(actual_rr / b2) : (R)0;
    double divergence_out;
    if (settled) divergence_out = settled_d;
    else { correct_linear(k1); divergence_out = divergence_metric_linear(); }
    bool accepted = (actual_rr <= tolr * b2 || floor_stop) && divergence_out <= PROJECTION_DIVERGENCE_TOLERANCE;
    rep[0] = 0;
    rep[1] = (double)it;
    rep[2] = (b2 > 0 && !accepted) ? 1.0 : 0.0;
    rep[3] = (double)residual;
    rep[4] = divergence_out;
    rep[5] = floor_stop ? 1.0 : 0.0;
    rep[6] = (double)backward_error_linear();
    rep[7] = divergence_out;
    return OK;
  }

  // step_surface_linear (delta3d.rs:1209-1253) and linear (:1255-1357), without a sponge or a
  // graded column: pressure first, then the heights carried by the column fluxes.
  int step_surface_linear(uint64_t duration_us, uint32_t max_iters, double rep[8]) {
    if (duration_us == 0 || duration_us > (1ull << 53)) return NOT_FINITE;
    double dt = (double)duration_us * 1e-6;
    R dx = d.dx;
    if (g_eff <= 0 || dt * dt * (double)g_eff / (double)dx > 1.) return DOMAIN;
    R scale = (R)(-(double)rho / dt);
    R correction = (R)(dt / (double)rho);
    R transport = (R)(dt / (double)dx);
    if (!std::isfinite(scale) || !std::isfinite(correction) || correction == 0 || !std::isfinite(transport) ||
        transport == 0)
      return NOT_FINITE;
    saved_u = u; saved_v = v; saved_w = w; saved_p = p; saved_eta = eta; saved_eta_roundoff = eta_roundoff;
    int e = [&]() -> int {
      size_t nx = d.nx, ny = d.ny, nz = d.nz;
      if (has_cut) {
        for (size_t q = 0; q < nx * ny; ++q)
          if (g.open_w[nz * nx * ny + q] != 1) return DOMAIN;
      }
      us = u; vs = v; ws = w;
      int err = project_linear(scale, correction, max_iters, rep);
      if (err) return err;
      if (rep[2] != 0) return CONVERGENCE;
      for (size_t j = 0; j < ny; ++j)
        for (size_t i = 0; i <= nx; ++i) {
          R q = 0;
          for (size_t k = 0; k < nz; ++k) {
            size_t f = fu(i, j, k);
            if (has_cut) q += g.open_u[f] * u[f] * dx; else q += u[f] * dx;
          }
          flux_x[j * (nx + 1) + i] = q;
        }
      for (size_t j = 0; j <= ny; ++j)
        for (size_t i = 0; i < nx; ++i) {
          R q = 0;
          for (size_t k = 0; k < nz; ++k) {
            size_t f = fv(i, j, k);
            if (has_cut) q += g.open_v[f] * v[f] * dx; else q += v[f] * dx;
          }
          flux_y[j * nx + i] = q;
        }
      for (size_t j = 0; j < ny; ++j)
        for (size_t i = 0; i < nx; ++i) {
          R left = flux_x[j * (nx + 1) + i], right = flux_x[j * (nx + 1) + i + 1];
          R front = flux_y[j * nx + i], back = flux_y[(j + 1) * nx + i];
          size_t cc = col(i, j);
          R increment = -transport * ((right - left) + (back - front)) - eta_roundoff[cc];
          R height = eta[cc] + increment;
          eta_roundoff[cc] = (height - eta[cc]) - increment;
          eta[cc] = height;
        }
      const std::vector<R>* fields[] = {&u, &v, &w, &p, &eta, &eta_roundoff, &rhs, &res, &dir, &tmp};
      for (auto f : fields)
        for (R x : *f)
          if (!std::isfinite(x)) return NOT_FINITE;
      if (!std::isfinite(rep[3]) || !std::isfinite(rep[4])) return NOT_FINITE;
      return OK;
    }();
    if (e) {
      u = saved_u; v = saved_v; w = saved_w; p = saved_p; eta = saved_eta; eta_roundoff = saved_eta_roundoff;
    }
    return e;
  }
};

// delta3d.rs:210-294
int configure(const Domain3& d, R rho, R g_eff, Volume3** out) {
  size_t nx = d.nx, ny = d.ny, nz = d.nz;
  if (nx == 0 || ny == 0 || nz == 0 || !std::isfinite(d.dx) || d.dx <= 0) return DOMAIN;
  if (!std::isfinite(rho) || rho <= 0 || !std::isfinite(g_eff)) return NOT_FINITE;
  size_t cells, cols, nu, nv, nw, t;
  if (__builtin_mul_overflow(nx, ny, &cols) || __builtin_mul_overflow(cols, nz, &cells)) return DOMAIN;
  if (__builtin_mul_overflow(nx + 1, ny, &t) || __builtin_mul_overflow(t, nz, &nu)) return DOMAIN;
  if (__builtin_mul_overflow(ny + 1, nx, &t) || __builtin_mul_overflow(t, nz, &nv)) return DOMAIN;
  if (__builtin_mul_overflow(nz + 1, cols, &nw)) return DOMAIN;
  if (!(std::isfinite(d.z0()) && std::isfinite((R)nx * d.dx) && std::isfinite((R)ny * d.dx))) return DOMAIN;
  if (cells > ((size_t)1 << 34)) return DOMAIN;  // the test harness's arena bound
  Volume3* v = new (std::nothrow) Volume3();
  if (!v) return DOMAIN;
  R z0 = d.z0();
  v->d = d; v->rho = rho; v->g_eff = g_eff; v->rest = z0;
  v->prec.assign(cells, 0); v->eta.assign(cols, z0); v->eta_roundoff.assign(cols, 0);
  v->u.assign(nu, 0); v->v.assign(nv, 0); v->w.assign(nw, 0);
  v->us.assign(nu, 0); v->vs.assign(nv, 0); v->ws.assign(nw, 0);
  v->p.assign(cells, 0); v->rhs.assign(cells, 0); v->res.assign(cells, 0); v->dir.assign(cells, 0); v->tmp.assign(cells, 0);
  v->saved_u.assign(nu, 0); v->saved_v.assign(nv, 0); v->saved_w.assign(nw, 0); v->saved_p.assign(cells, 0);
  v->saved_eta.assign(cols, z0); v->saved_eta_roundoff.assign(cols, 0);
  v->flux_x.assign((nx + 1) * ny, 0); v->flux_y.assign((ny + 1) * nx, 0);
  *out = v;
  return OK;
}

}  // namespace

// =============================================================================================
// C API (oracle): mirrors the product's fd3_* entry points with an od3_ prefix.  Inputs are f32
// (as the reference's API); outputs are in the oracle's real type R (f32 or f64 build).
extern "C" {

struct od3_domain { uint64_t nx, ny, nz; float dx; };

int od3_real_bytes(void) { return (int)sizeof(R); }
void od3_set_threads(int n) { g_threads = n > 0 ? n : 1; }
void od3_set_smoother(int s) { g_smoother = (s >= 0 && s <= 3) ? s : 0; }
void od3_set_transfer(int t) { g_transfer = t == 1 ? 1 : 0; }
void od3_set_storage(int s) { g_storage = s == 1 ? 1 : 0; }
double od3_take_zmax(void) { double z = g_zmax; g_zmax = 0; return z; }
int od3_max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

int od3_configure(const od3_domain* dom, float rho, float g, Volume3** out) {
  if (!dom || !out) return INVALID;
  Domain3 d{dom->nx, dom->ny, dom->nz, (R)dom->dx};
  return configure(d, (R)rho, (R)g, out);
}

// delta3d.rs:300-321
int od3_configure_with_bottom(const od3_domain* dom, float rho, float g, const float* bottom, uint64_t len, Volume3** out) {
  if (!dom || !out || (!bottom && len)) return INVALID;
  Domain3 d{dom->nx, dom->ny, dom->nz, (R)dom->dx};
  size_t cols;
  if (__builtin_mul_overflow(d.nx, d.ny, &cols)) return DOMAIN;
  if (len != cols) return SHAPE;
  for (size_t q = 0; q < len; ++q) {
    R b = (R)bottom[q];
    if (!std::isfinite(b) || b < 0 || b >= d.z0()) return NOT_FINITE;
  }
  Volume3* v;
  int e = configure(d, (R)rho, (R)g, &v);
  if (e) return e;
  std::vector<R> b(bottom, bottom + len);
  v->g = cut(d, b.data());
  v->has_cut = true;
  v->prec_cut();
  *out = v;
  return OK;
}

// delta3d.rs:327-365 (piercing = false: configure_with_solid)
int od3_configure_with_solid(const od3_domain* dom, float rho, float g, const float* bottom, uint64_t blen,
                             const float* solid, uint64_t slen, Volume3** out) {
  if (!dom || !out || (!solid && slen)) return INVALID;
  size_t nodes, t;
  if (__builtin_mul_overflow((size_t)dom->nx + 1, (size_t)dom->ny + 1, &t) || __builtin_mul_overflow(t, (size_t)dom->nz + 1, &nodes))
    return DOMAIN;
  if (slen != nodes) return SHAPE;
  for (size_t q = 0; q < slen; ++q)
    if (!std::isfinite(solid[q])) return NOT_FINITE;
  Volume3* v;
  int e = od3_configure_with_bottom(dom, rho, g, bottom, blen, &v);
  if (e) return e;
  Domain3 d = v->d;
  v->g.piercing = false;
  Base3 base{v->g.frac, v->g.open_u, v->g.open_v, v->g.open_w, v->g.floor,
             std::vector<R>(d.nx * d.ny, 0), std::vector<R>(d.nx * d.ny, 0)};
  if ((e = add_solid(v->g, d, solid))) { delete v; return e; }
  solid_columns(d, base.frac, v->g.frac, base.solid_col);
  v->g.base = std::move(base);
  v->g.has_base = true;
  v->prec_cut();
  *out = v;
  return OK;
}

// set_solid_rigid (delta3d.rs:382-509): the solid moved as a rigid body.  The cut is redone from
// the bottom-only base; a face that opens takes the wall's normal velocity at its centre, a face
// that closes loses its own; the solid volume a column gains raises its surface (compensated f32
// sum).  Volumes of this API carry a solid that may not reach the lid layer (configure_with_solid,
// piercing = false), so no lid face is ever cut and the partial-lid transfer of delta3d.rs:460-503
// moves nothing: it is not restated.  Refusal is atomic: Shape, NotFinite, Domain (no solid, or
// check_solid fails).
int od3_set_solid_rigid(Volume3* v, const float* solid, uint64_t len, const float* vel, const float* ang,
                        const float* cen) {
  if (!v || !vel || !ang || !cen || (!solid && len)) return INVALID;
  const Domain3 d = v->d;
  const size_t nx = d.nx, ny = d.ny, nz = d.nz;
  if (len != (nx + 1) * (ny + 1) * (nz + 1)) return SHAPE;
  for (size_t q = 0; q < len; ++q) if (!std::isfinite(solid[q])) return NOT_FINITE;
  for (int a = 0; a < 3; ++a) if (!std::isfinite(vel[a]) || !std::isfinite(ang[a]) || !std::isfinite(cen[a])) return NOT_FINITE;
  if (!v->has_cut || !v->g.has_base) return DOMAIN;
  Cut3& g = v->g;
  Base3& base = g.base;
  int e = check_solid(base.frac, base.open_u, base.open_v, base.open_w, d, solid, g.piercing);
  if (e) return e;
  v->saved_u = g.open_u; v->saved_v = g.open_v; v->saved_w = g.open_w;
  g.frac = base.frac; g.open_u = base.open_u; g.open_v = base.open_v; g.open_w = base.open_w; g.floor = base.floor;
  add_solid(g, d, solid);
  for (int a = 0; a < 3; ++a) {
    g.solid_velocity[a] = vel[a];
    g.solid_angular[a] = ang[a];
    g.solid_center[a] = cen[a];
  }
  const R dx = d.dx;
  for (size_t k = 0; k < nz; ++k) {
    for (size_t j = 0; j < ny; ++j)
      for (size_t i = 0; i <= nx; ++i) {
        size_t f = (k * ny + j) * (nx + 1) + i;
        if (g.open_u[f] == 0) v->u[f] = 0;
        else if (v->saved_u[f] == 0) v->u[f] = wall_velocity(vel, ang, cen, 0, (R)i * dx, ((R)j + (R)0.5) * dx, ((R)k + (R)0.5) * dx);
      }
    for (size_t j = 0; j <= ny; ++j)
      for (size_t i = 0; i < nx; ++i) {
        size_t f = (k * (ny + 1) + j) * nx + i;
        if (g.open_v[f] == 0) v->v[f] = 0;
        else if (v->saved_v[f] == 0) v->v[f] = wall_velocity(vel, ang, cen, 1, ((R)i + (R)0.5) * dx, (R)j * dx, ((R)k + (R)0.5) * dx);
      }
  }
  for (size_t k = 0; k <= nz; ++k)
    for (size_t j = 0; j < ny; ++j)
      for (size_t i = 0; i < nx; ++i) {
        size_t f = (k * ny + j) * nx + i;
        if (g.open_w[f] == 0) v->w[f] = 0;
        else if (v->saved_w[f] == 0) v->w[f] = wall_velocity(vel, ang, cen, 2, ((R)i + (R)0.5) * dx, ((R)j + (R)0.5) * dx, (R)k * dx);
      }
  std::vector<R> cols(nx * ny);
  solid_columns(d, base.frac, g.frac, cols);
  const R area = dx * dx;
  for (size_t c = 0; c < nx * ny; ++c) {
    base.deposit[c] += (cols[c] - base.solid_col[c]) / area;
    R increment = (cols[c] - base.solid_col[c]) / area - v->eta_roundoff[c];
    R height = v->eta[c] + increment;
    v->eta_roundoff[c] = (height - v->eta[c]) - increment;
    v->eta[c] = height;
    base.solid_col[c] = cols[c];
  }
  v->prec_cut();
  return OK;
}

void od3_destroy(Volume3* v) { delete v; }

// delta3d_multigrid.rs:339-349 (max_levels 0 = the reference hierarchy)
int od3_enable_multigrid(Volume3* v, uint32_t max_levels) {
  if (!v) return INVALID;
  if (v->has_mg) return OK;
  size_t floats;
  if (!hierarchy_floats3(v->d.nx, v->d.ny, v->d.nz, &floats)) return DOMAIN;
  v->mg = make_multigrid(v->d.nx, v->d.ny, v->d.nz, v->d.dx, max_levels);
  v->mg_max_levels = max_levels;
  v->has_mg = true;
  return OK;
}
int od3_multigrid_levels(const Volume3* v) { return v && v->has_mg ? (int)v->mg.levels.size() : -1; }
uint64_t od3_level_count3(uint64_t nx, uint64_t ny, uint64_t nz) { return level_count3(nx, ny, nz); }
uint64_t od3_hierarchy_floats3(uint64_t nx, uint64_t ny, uint64_t nz) {
  size_t f;
  return hierarchy_floats3(nx, ny, nz, &f) ? f : 0;
}

// delta3d_mobile.rs:9-25
int od3_set_free_surface(Volume3* v, const float* eta, uint64_t len, float rest) {
  if (!v || (!eta && len)) return INVALID;
  if (len != v->eta.size()) return SHAPE;
  if (!std::isfinite(rest)) return NOT_FINITE;
  for (size_t q = 0; q < len; ++q) if (!std::isfinite(eta[q])) return NOT_FINITE;
  if (!v->sparse_surface_ok(eta, rest)) return DOMAIN;  // delta3d_mobile.rs:16-19
  for (size_t q = 0; q < len; ++q) v->eta[q] = (R)eta[q];
  std::fill(v->eta_roundoff.begin(), v->eta_roundoff.end(), (R)0);
  std::fill(v->p.begin(), v->p.end(), (R)0);
  v->rest = (R)rest;
  return OK;
}

// delta3d.rs:614-628
int od3_set_surface(Volume3* v, const float* eta, uint64_t len) {
  if (!v || (!eta && len)) return INVALID;
  if (len != v->eta.size()) return SHAPE;
  for (size_t q = 0; q < len; ++q) if (!std::isfinite(eta[q])) return NOT_FINITE;
  if (!v->sparse_surface_ok(eta, (float)v->rest)) return DOMAIN;  // delta3d.rs:621-624
  for (size_t q = 0; q < len; ++q) v->eta[q] = (R)eta[q];
  std::fill(v->eta_roundoff.begin(), v->eta_roundoff.end(), (R)0);
  return OK;
}

// delta3d.rs:631-645
int od3_set_velocity(Volume3* v, const float* u, uint64_t nu, const float* vv, uint64_t nv, const float* w, uint64_t nw) {
  if (!v) return INVALID;
  if (nu != v->u.size() || nv != v->v.size() || nw != v->w.size()) return SHAPE;
  for (size_t q = 0; q < nu; ++q) if (!std::isfinite(u[q])) return NOT_FINITE;
  for (size_t q = 0; q < nv; ++q) if (!std::isfinite(vv[q])) return NOT_FINITE;
  for (size_t q = 0; q < nw; ++q) if (!std::isfinite(w[q])) return NOT_FINITE;
  for (size_t q = 0; q < nu; ++q) v->u[q] = (R)u[q];
  for (size_t q = 0; q < nv; ++q) v->v[q] = (R)vv[q];
  for (size_t q = 0; q < nw; ++q) v->w[q] = (R)w[q];
  v->close_walls();
  v->close_sparse_walls();
  return OK;
}

// Squared relative residual target (1e-12 in the reference); the FP64 error reference tightens it.
int od3_set_tolerance(Volume3* v, float tol) { if (!v) return INVALID; v->tol = tol; return OK; }

// Projects the current velocity field: us = u, then project_mobile3 (tests_delta3d.rs:389-400).
int od3_project_mobile(Volume3* v, float scale, float k1, uint32_t max_iters, double rep[8]) {
  if (!v || !rep) return INVALID;
  v->us = v->u; v->vs = v->v; v->ws = v->w;
  return v->project_mobile3((R)scale, (R)k1, max_iters, rep);
}

// refine_mobile3 (delta3d_coupling.rs:226-248): one defect-correction pass of the mobile projection.
// The corrected field is projected again from p = 0 with homogeneous ghosts, and the pressure
// increment is added to the pressure it starts from.
int od3_refine_mobile(Volume3* v, float scale, float k1, uint32_t max_iters, double rep[8]) {
  if (!v || !rep) return INVALID;
  std::vector<R> base = v->p;
  v->us = v->u; v->vs = v->v; v->ws = v->w;
  std::fill(v->p.begin(), v->p.end(), (R)0);
  v->homogeneous_ghost = true;
  int e = v->project_mobile3((R)scale, (R)k1, max_iters, rep);
  v->homogeneous_ghost = false;
  if (e) return e;
  for (size_t q = 0; q < v->p.size(); ++q) v->p[q] += base[q];
  rep[0] = 1;  // refinements
  return OK;
}

// Projects the current velocity field on the linear (fixed-lid) path: us = u, then project
// (tests_delta3d.rs:143-148).
int od3_project_linear(Volume3* v, float scale, float k1, uint32_t max_iters, double rep[8]) {
  if (!v || !rep) return INVALID;
  if (v->has_sparse) return DOMAIN;  // the linear path does not carry a sparse set (delta3d.rs:1210-1211)
  v->us = v->u; v->vs = v->v; v->ws = v->w;
  return v->project_linear((R)scale, (R)k1, max_iters, rep);
}

int od3_step_surface_linear(Volume3* v, uint64_t duration_us, uint32_t max_iters, double rep[8]) {
  if (!v || !rep) return INVALID;
  if (v->has_sparse) return DOMAIN;  // delta3d.rs:1210-1211
  return v->step_surface_linear(duration_us, max_iters, rep);
}

// set_precondition_cut (delta3d.rs:526-528).
int od3_set_precondition_cut(Volume3* v, int on) {
  if (!v) return INVALID;
  v->precondition_cut = on != 0;
  return OK;
}

int od3_step_surface_mobile(Volume3* v, uint64_t duration_us, uint32_t max_iters, double rep[8]) {
  if (!v || !rep) return INVALID;
  return v->step_surface_mobile(duration_us, max_iters, rep);
}

// enable_sparse (delta3d_sparse.rs:105-117): every column starts in the set.
int od3_enable_sparse(Volume3* v) {
  if (!v) return INVALID;
  if (v->has_sparse) return DOMAIN;
  v->has_sparse = true;
  v->active.assign(v->d.nx * v->d.ny, 1);
  v->next_active.assign(v->d.nx * v->d.ny, 1);
  return OK;
}

// set_active_columns (delta3d_sparse.rs:147-158); change[6] as apply_sparse writes it
int od3_set_active_columns(Volume3* v, const uint8_t* mask, uint64_t len, double change[6]) {
  if (!v || !change || (!mask && len)) return INVALID;
  if (!v->has_sparse) return DOMAIN;
  if (len != v->active.size()) return SHAPE;
  for (size_t q = 0; q < len; ++q) v->next_active[q] = mask[q] != 0;
  v->apply_sparse(change);
  return OK;
}

// set_active_blocks (delta3d_sparse.rs:163-178): block b covers the columns
// [(b.i - origin.i)*8, +8) x [(b.j - origin.j)*8, +8) of the window, clipped to it.
// blocks: count (i, j) pairs.
int od3_set_active_blocks(Volume3* v, const int32_t* blocks, uint64_t count, int32_t oi, int32_t oj, double change[6]) {
  if (!v || !change || (!blocks && count)) return INVALID;
  if (!v->has_sparse) return DOMAIN;
  const long long side = 8, nx = (long long)v->d.nx, ny = (long long)v->d.ny;
  std::fill(v->next_active.begin(), v->next_active.end(), (uint8_t)0);
  for (uint64_t b = 0; b < count; ++b) {
    long long i0 = ((long long)blocks[2 * b] - oi) * side, j0 = ((long long)blocks[2 * b + 1] - oj) * side;
    for (long long j = std::max(j0, 0LL); j < std::min(j0 + side, ny); ++j)
      for (long long i = std::max(i0, 0LL); i < std::min(i0 + side, nx); ++i) v->next_active[(size_t)(j * nx + i)] = 1;
  }
  v->apply_sparse(change);
  return OK;
}

// resample_from (delta3d_levels.rs:43-69): the state of `src`, which covers the same window at
// another dx.  out: volume before (src), volume after (dst).
int od3_resample_from(Volume3* v, const Volume3* src, double out[2]) {
  if (!v || !src || !out) return INVALID;
  const Domain3 &d = v->d, &s = src->d;
  auto extent = [](size_t n, float dx) { return (double)n * (double)dx; };
  auto same = [](double a, double b) { return std::fabs(a - b) <= 1e-6 * std::max(std::fabs(a), std::fabs(b)); };
  auto fbits = [](float x) { uint32_t b; std::memcpy(&b, &x, 4); return b; };
  if (!same(extent(d.nx, (float)d.dx), extent(s.nx, (float)s.dx)) || !same(extent(d.ny, (float)d.dx), extent(s.ny, (float)s.dx)) ||
      !same(extent(d.nz, (float)d.dx), extent(s.nz, (float)s.dx)) || fbits((float)v->rest) != fbits((float)src->rest) ||
      fbits((float)v->rho) != fbits((float)src->rho) || fbits((float)v->g_eff) != fbits((float)src->g_eff) ||
      v->has_cut || src->has_cut)
    return DOMAIN;
  out[0] = src->perturbation_volume();
  v->resample_surface(*src);
  v->resample_faces(*src);
  std::fill(v->p.begin(), v->p.end(), (R)0);
  v->close_walls();
  v->close_sparse_walls();
  out[1] = v->perturbation_volume();
  return OK;
}

double od3_perturbation_volume(const Volume3* v) { return v ? v->perturbation_volume() : 0.; }

// The predictor alone, as tests_delta3d.rs:2136-2160 runs it: advect, the second-order term when
// on, then u = us.
int od3_advect_for_tests(Volume3* v, float dt) {
  if (!v) return INVALID;
  v->advect_mobile3((R)dt);
  v->correct_advection3((R)dt);
  v->u = v->us; v->v = v->vs; v->w = v->ws;
  return OK;
}

// enable_advection_correction (delta3d_advection.rs:17-21)
int od3_enable_advection_correction(Volume3* v) {
  if (!v) return INVALID;
  v->advection_correction = true;
  return OK;
}

// active_columns / sparse_cells (delta3d_sparse.rs:129-141)
int od3_active_columns(const Volume3* v, uint8_t* out, uint64_t len) {
  if (!v || !out) return INVALID;
  if (!v->has_sparse) return DOMAIN;
  if (len != v->active.size()) return SHAPE;
  std::memcpy(out, v->active.data(), len);
  return OK;
}
uint64_t od3_sparse_cells(const Volume3* v) {
  if (!v) return 0;
  if (!v->has_sparse) return (uint64_t)v->d.nx * v->d.ny * v->d.nz;
  uint64_t cols = 0;
  for (uint8_t a : v->active) cols += a != 0;
  return cols * v->d.nz;
}

int od3_last_refused_report(const Volume3* v, double rep[8]) {
  if (!v || !rep || !v->has_refused) return DOMAIN;
  std::memcpy(rep, v->refused, sizeof(v->refused));
  return OK;
}

static int copy_out(const std::vector<R>& src, R* dst, uint64_t len) {
  if (!dst && len) return INVALID;
  if (len != src.size()) return SHAPE;
  std::memcpy(dst, src.data(), len * sizeof(R));
  return OK;
}
int od3_get_pressure(const Volume3* v, R* out, uint64_t len) { return v ? copy_out(v->p, out, len) : INVALID; }
int od3_get_velocity(const Volume3* v, R* u, uint64_t nu, R* vv, uint64_t nv, R* w, uint64_t nw) {
  if (!v) return INVALID;
  int e;
  if ((e = copy_out(v->u, u, nu)) || (e = copy_out(v->v, vv, nv)) || (e = copy_out(v->w, w, nw))) return e;
  return OK;
}
int od3_get_surface(const Volume3* v, R* eta, R* roundoff, uint64_t len) {
  if (!v) return INVALID;
  int e;
  if ((e = copy_out(v->eta, eta, len)) || (e = copy_out(v->eta_roundoff, roundoff, len))) return e;
  return OK;
}
int od3_get_rhs_prec(const Volume3* v, R* rhs, R* prec, uint64_t len) {
  if (!v) return INVALID;
  int e;
  if ((e = copy_out(v->rhs, rhs, len)) || (e = copy_out(v->prec, prec, len))) return e;
  return OK;
}
// Cut geometry (frac, open_u/v/w, floor); SHAPE on a flat bottom.
int od3_get_geometry(const Volume3* v, R* frac, R* ou, R* ov, R* ow, R* floor) {
  if (!v) return INVALID;
  if (!v->has_cut) return DOMAIN;
  std::memcpy(frac, v->g.frac.data(), v->g.frac.size() * sizeof(R));
  std::memcpy(ou, v->g.open_u.data(), v->g.open_u.size() * sizeof(R));
  std::memcpy(ov, v->g.open_v.data(), v->g.open_v.size() * sizeof(R));
  std::memcpy(ow, v->g.open_w.data(), v->g.open_w.size() * sizeof(R));
  std::memcpy(floor, v->g.floor.data(), v->g.floor.size() * sizeof(R));
  return OK;
}
uint64_t od3_wet_cells(const Volume3* v) {
  uint64_t n = 0;
  for (size_t k = 0; k < v->d.nz; ++k)
    for (size_t j = 0; j < v->d.ny; ++j)
      for (size_t i = 0; i < v->d.nx; ++i) n += v->wet3(i, j, k);
  return n;
}

// delta3d_mobile.rs:936-953
int od3_apply_pressure_operator_for_trials(const Volume3* v, const float* p, R* out, uint64_t len) {
  if (!v) return INVALID;
  if (len != v->p.size()) return DOMAIN;
  for (size_t q = 0; q < len; ++q) if (!std::isfinite(p[q])) return NOT_FINITE;
  std::vector<R> pp(p, p + len);
  v->apply_mobile3(pp.data(), out);
  return OK;
}

// delta3d_mobile.rs:960-979
int od3_assemble_pressure_problem_for_trials(Volume3* v, const float* divergence, float scale, R* rhs, R* prec, uint64_t len) {
  if (!v) return INVALID;
  if (len != v->p.size()) return DOMAIN;
  if (!std::isfinite(scale)) return NOT_FINITE;
  for (size_t q = 0; q < len; ++q) if (!std::isfinite(divergence[q])) return NOT_FINITE;
  for (size_t q = 0; q < len; ++q) v->rhs[q] = (R)divergence[q];
  v->rhs_mobile3((R)scale);
  std::memcpy(rhs, v->rhs.data(), len * sizeof(R));
  std::memcpy(prec, v->prec.data(), len * sizeof(R));
  return OK;
}

// The V-cycle on a given residual, set up as tests_delta3d.rs:1840-1873 does: rhs = 0,
// rhs_mobile3(1), prepare_multigrid3(), res = x, v_cycle3().  Writes z.
int od3_vcycle_for_tests(Volume3* v, const float* x, R* z, uint64_t len) {
  if (!v || !v->has_mg) return DOMAIN;
  if (len != v->p.size()) return SHAPE;
  std::fill(v->rhs.begin(), v->rhs.end(), (R)0);
  v->rhs_mobile3((R)1);
  v->prepare_multigrid3();
  for (size_t q = 0; q < len; ++q) v->res[q] = (R)x[q];
  v->v_cycle3();
  std::memcpy(z, v->mg.z.data(), len * sizeof(R));
  return OK;
}

// Coarse level `l` geometry after prepare (kind, diag, open_u/v/w), for hierarchy parity.
int od3_level_geometry(const Volume3* v, uint32_t l, R* kind, R* diag, R* ou, R* ov, R* ow) {
  if (!v || !v->has_mg || l >= v->mg.levels.size()) return DOMAIN;
  const Level3& L = v->mg.levels[l];
  std::memcpy(kind, L.kind.data(), L.kind.size() * sizeof(R));
  std::memcpy(diag, L.diag.data(), L.diag.size() * sizeof(R));
  std::memcpy(ou, L.open_u.data(), L.open_u.size() * sizeof(R));
  std::memcpy(ov, L.open_v.data(), L.open_v.size() * sizeof(R));
  std::memcpy(ow, L.open_w.data(), L.open_w.size() * sizeof(R));
  return OK;
}

uint64_t od3_fingerprint(const float* p, uint64_t len) {
  std::vector<R> x(p, p + len);
  return Volume3::fingerprint(x);
}

}  // extern "C"
