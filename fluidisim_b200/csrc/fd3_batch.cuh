// Many δ patches projected in one persistent launch (no reference counterpart; the reference
// projects one Volume3 at a time).
//
// k_batch_project runs thread-block clusters as independent solvers: cluster c takes the patches
// order[start[c]] .. order[start[c + 1] - 1] one after another (the host deals them largest first
// to the least loaded cluster) and runs each one's whole project_mobile3 (delta3d_mobile.rs:465-609)
// on the device: assembly, the multigrid hierarchy, the MG-preconditioned CG loop, the outer
// checks and their decisions, the report.  Every phase is a loop over the patch's cells (or faces)
// strided over all the cluster's threads, closed by the cluster's hardware barrier; no CTA ever
// waits on another cluster, so the launch needs no co-residency beyond the cluster's own.
//
// Reductions are deterministic: warp shuffles, then the CTA's warps in order, then every CTA
// reads the cluster's per-CTA partials through distributed shared memory in rank order, so all
// CTAs hold the same total and apply the same scalar step (apply_op) to their own shared-memory
// copy of the patch's Scalars; their control flow, which only those scalars decide, is therefore
// the same in every CTA, and each CTA meets every cluster barrier.
//
// Per-cell arithmetic is the library's (apply_code, rhs_b2_at, the coarse tail, the correction and
// metric functions): the values of each cell are those of the one-cell-per-thread kernels.  Only
// f64 reductions, f32 storage and the mobile (free-surface) rows with multigrid are handled.
#pragma once

#include <cooperative_groups.h>

#include "fd3_fast.cuh"

namespace fd3 {

// gamma_8 and gamma_10 of u = 2^-24 (delta_projection.rs:200-203, delta3d.rs:69-72)
constexpr float BATCH_ROUNDOFF_2D = 8.0f * (1.0f / 16777216.0f) / (1.0f - 8.0f * (1.0f / 16777216.0f));
constexpr float BATCH_ROUNDOFF_3D = 10.0f * (1.0f / 16777216.0f) / (1.0f - 10.0f * (1.0f / 16777216.0f));
constexpr double BATCH_DIV_TOL = 1e-5;  // PROJECTION_DIVERGENCE_TOLERANCE (delta_projection.rs:192)
#ifndef FD3_BATCH_THREADS
#define FD3_BATCH_THREADS 1024
#endif
constexpr int BATCH_THREADS = FD3_BATCH_THREADS;  // threads of a CTA (one CTA per SM)

// One patch of a batch: its geometry and every device buffer its projection touches.
struct BatchPatch {
  Geo g;
  unsigned short* codes;
  float *u, *v, *w, *us, *vs, *ws, *p, *sv_p, *rhs, *prec, *res, *dir, *dir2, *q, *z, *z2;
  float *sv_u, *sv_v, *sv_w;        // the velocity before the call, kept when inputs are given
  const float *in_u, *in_v, *in_w;  // optional inputs copied into u, v, w first (null: the current field)
  const Lev* lev;                   // the coarse levels (device table), nlev of them
  int nlev;
  int nu, nv, nw;
  float scale, k1;
  unsigned max_iters;
  int flat2d;                       // ny == 1: the 2-D roundoff floor
  int reset_p;                      // 1: project from p = 0
  Scalars* S;                       // the patch's scalars, written back at the end
};

// Result of one patch: the report fields and a status (0 or an fd3_status).
struct BatchResult {
  unsigned iterations;
  int status;
  int degraded, floor_stop;
  double residual, divergence, backward_error, divergence_plain;
};

// The threads of one thread-block cluster as a team for the strided phases of the coarse tail.
struct ClusterTeam {
  int r, n;
  __device__ __forceinline__ ClusterTeam() {
    cooperative_groups::cluster_group cl = cooperative_groups::this_cluster();
    r = (int)cl.block_rank() * (int)blockDim.x + (int)threadIdx.x;
    n = (int)cl.num_blocks() * (int)blockDim.x;
  }
  __device__ __forceinline__ int rank() const { return r; }
  __device__ __forceinline__ int size() const { return n; }
  __device__ __forceinline__ void sync() const { cooperative_groups::this_cluster().sync(); }
};

// Shared state of one CTA.
struct BatchShared {
  Scalars S;                     // this CTA's copy of the patch's scalars
  double slot[2][6];             // the CTA's partials of a reduction (two sets, used alternately)
  unsigned long long hslot[2];
  double warp[32][6];
  unsigned long long hwarp[32];
  BatchPatch P;
};

// The cluster-wide reduction of K per-thread values (sums, or maxima where `mx` has bit k set)
// and, when `h` is not null, of a 64-bit wrapping sum.  Every thread of every CTA of the cluster
// calls it and gets the same totals; it holds one cluster barrier.  `ph` alternates the slot
// set, so a slow reader of this reduction never sees the next one's partials.
template <int K>
__device__ __forceinline__ void crew_reduce(BatchShared& sh, int& ph, double (&v)[K], unsigned mx,
                                            unsigned long long* h) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int k = 0; k < K; ++k)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const double t = __shfl_down_sync(0xffffffffu, v[k], o);
      v[k] = (mx >> k) & 1 ? fmax(v[k], t) : v[k] + t;
    }
  unsigned long long hv = h ? *h : 0ull;
  if (h)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) hv += __shfl_down_sync(0xffffffffu, hv, o);
  if (lane == 0) {
#pragma unroll
    for (int k = 0; k < K; ++k) sh.warp[wid][k] = v[k];
    sh.hwarp[wid] = hv;
  }
  __syncthreads();
  const int s = ph & 1;
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < K; ++k) {
      double t = sh.warp[0][k];
      for (int q = 1; q < nw; ++q) t = (mx >> k) & 1 ? fmax(t, sh.warp[q][k]) : t + sh.warp[q][k];
      sh.slot[s][k] = t;
    }
    unsigned long long t = 0ull;
    for (int q = 0; q < nw; ++q) t += sh.hwarp[q];
    sh.hslot[s] = t;
  }
  cooperative_groups::cluster_group cl = cooperative_groups::this_cluster();
  cl.sync();
  const unsigned nb = cl.num_blocks();
#pragma unroll
  for (int k = 0; k < K; ++k) {
    double t = *cl.map_shared_rank(&sh.slot[s][k], 0u);
    for (unsigned r = 1; r < nb; ++r) {
      const double x = *cl.map_shared_rank(&sh.slot[s][k], r);
      t = (mx >> k) & 1 ? fmax(t, x) : t + x;
    }
    v[k] = t;
  }
  if (h) {
    unsigned long long t = 0ull;
    for (unsigned r = 0; r < nb; ++r) t += *cl.map_shared_rank(&sh.hslot[s], r);
    *h = t;
  }
  ++ph;
}

// A scalar step applied by thread 0 of each CTA to its copy of the scalars, then seen by all.
__device__ __forceinline__ void crew_apply(BatchShared& sh, double val, int op) {
  if (threadIdx.x == 0) apply_op(&sh.S, val, op, 0);
  __syncthreads();
}

// f(c) for this thread's cells c of [0, n) in the cluster-strided order, FD3_BATCH_UNROLL at a time
// (the per-thread order of the cells is unchanged).  Measured on the 256-patch set: 44.4 ms per set
// with 1, 45.8 with 2, 51.0 with 4; at 1024 threads a CTA has 64 registers a thread, and the
// unrolled bodies spill.
#ifndef FD3_BATCH_UNROLL
#define FD3_BATCH_UNROLL 1
#endif
template <class F>
__device__ __forceinline__ void strided_cells(const ClusterTeam& tm, int n, F f) {
  constexpr int U = FD3_BATCH_UNROLL;
  const int T = tm.size();
  int c = tm.rank();
  for (; c + (U - 1) * T < n; c += U * T) {
#pragma unroll
    for (int u = 0; u < U; ++u) f(c + u * T);
  }
  for (; c < n; c += T) f(c);
}

// Coarse levels of at most this many cells are solved by the cluster's first CTA alone, with CTA
// barriers instead of cluster barriers (the single-volume path's coarse tail does the same).
constexpr int BATCH_CTA_LEVEL_CELLS = 4096;

// v_cycle3 (delta3d_multigrid.rs:393-429) of P.res into P.z with res.z at its end (op), the
// one-cell-per-thread passes of the library and the coarse tail over every level.
__device__ __forceinline__ void batch_vcycle(const ClusterTeam& tm, BatchShared& sh, int& ph, int op) {
  const BatchPatch& P = sh.P;
  const Geo& g = P.g;
  const float* __restrict__ prec = P.prec;
  const float* __restrict__ r = P.res;
  const unsigned short* __restrict__ codes = P.codes;
  float* __restrict__ z = P.z;
  float* __restrict__ z2 = P.z2;
  // the two pre-sweeps from z = 0 (k_fine_pre): z1 = w prec r recomputed at the stencil points
  {
    auto Z1 = [&](int n) {
      float m = prec[n];
      return m > 0.f ? 0.f + OMEGA * m * (r[n] - 0.f) : 0.f;
    };
    strided_cells(tm, g.n, [&](int c) {
      float m = prec[c];
      float zc = Z1(c);
      if (m > 0.f) {
        int i, j, k; cell_ijk(g, c, i, j, k);
        zc += OMEGA * m * (r[c] - apply_code(g, (unsigned)codes[c], i, j, k, c, Z1));
      }
      z[c] = zc;
    });
    tm.sync();
  }
  const bool levels = P.nlev > 0;
  if (levels) {  // restrict3 of r - A z (k_fine_restrict_c), then the coarse levels
    const Lev L = P.lev[0];
    Load Z{z};
    float* __restrict__ lr = L.r;
    strided_cells(tm, L.n, [&](int qi) {
      int ci = qi % L.nx, t = qi / L.nx, cj = t % L.ny, ck = t / L.ny;
      float s = 0.f;
#pragma unroll
      for (int e = 0; e < 8; ++e) {
        int i = 2 * ci + (e & 1), j = 2 * cj + ((e >> 1) & 1), k = 2 * ck + (e >> 2);
        int c = (k * g.ny + j) * g.nx + i;
        unsigned code = codes[c];
        float az = (code & RC_WET) ? apply_code(g, code, i, j, k, c, Z) : 0.f;
        s += r[c] - az;
      }
      lr[qi] = 0.125f * s;
    });
    tm.sync();
    // the small levels from `t` down are solved by the first CTA alone
    const int last = P.nlev - 1;
    int t = P.nlev;
    while (t > 0 && P.lev[t - 1].n <= BATCH_CTA_LEVEL_CELLS) --t;
    if (t >= P.nlev) {
      tail_run_t(tm, P.lev, 0, last);
    } else {
      tail_down_t(tm, P.lev, 0, t, last);
      if (cooperative_groups::this_cluster().block_rank() == 0) tail_run_t(BlockTeam{}, P.lev, t, last);
      tm.sync();
      tail_up_t(tm, P.lev, 0, t - 1);
    }
  }
  // prolongation, dry cells zeroed, first post-sweep (k_fine_post1)
  {
    const Lev L = levels ? P.lev[0] : Lev{};
    const float* __restrict__ zin = z;
    const float* __restrict__ lx = L.x;
    auto ZP = [&](int n) {
      if (!levels) return zin[n];
      int i = n % g.nx, t = n / g.nx, j = t % g.ny, k = t / g.ny;
      float v = zin[n] + lx[((k >> 1) * L.ny + (j >> 1)) * L.nx + (i >> 1)];
      return prec[n] == 0.f ? 0.f : v;
    };
    strided_cells(tm, g.n, [&](int c) {
      float m = prec[c];
      float zc = ZP(c);
      if (m > 0.f) {
        int i, j, k; cell_ijk(g, c, i, j, k);
        zc += OMEGA * m * (r[c] - apply_code(g, (unsigned)codes[c], i, j, k, c, ZP));
      }
      z2[c] = zc;
    });
    tm.sync();
  }
  // the last post-sweep with r.z (k_fine_post2_rz)
  double acc[1] = {0.0};
  {
    Load Z{z2};
    strided_cells(tm, g.n, [&](int c) {
      float m = prec[c];
      float rc = r[c];
      float zc = z2[c];
      if (m > 0.f) {
        int i, j, k; cell_ijk(g, c, i, j, k);
        zc += OMEGA * m * (rc - apply_code(g, (unsigned)codes[c], i, j, k, c, Z));
      }
      z[c] = zc;
      acc[0] += (double)rc * (double)zc;
    });
  }
  crew_reduce<1>(sh, ph, acc, 0u, nullptr);
  crew_apply(sh, acc[0], op);
}

// res = rhs - A p with res.res (FIN_RR0 or FIN_ACTUAL).
__device__ __forceinline__ void batch_residual(const ClusterTeam& tm, BatchShared& sh, int& ph, int op) {
  const BatchPatch& P = sh.P;
  const Geo& g = P.g;
  const unsigned short* __restrict__ codes = P.codes;
  const float* __restrict__ rhs = P.rhs;
  float* __restrict__ res = P.res;
  Load Pl{P.p};
  double acc[1] = {0.0};
  strided_cells(tm, g.n, [&](int c) {
    unsigned code = codes[c];
    float ap = 0.f;
    if (code & RC_WET) { int i, j, k; cell_ijk(g, c, i, j, k); ap = apply_code(g, code, i, j, k, c, Pl); }
    const float rv = rhs[c] - ap;
    res[c] = rv;
    acc[0] += (double)rv * (double)rv;
  });
  crew_reduce<1>(sh, ph, acc, 0u, nullptr);
  crew_apply(sh, acc[0], op);
}

// One PCG iteration (delta3d_mobile.rs:523-545) with the direction buffers of `parity`; every
// phase after one that closed the loop is skipped, as the gated kernels of the loop graph are.
__device__ __forceinline__ void batch_iteration(const ClusterTeam& tm, BatchShared& sh, int& ph, int parity) {
  const BatchPatch& P = sh.P;
  const Geo& g = P.g;
  const float* __restrict__ din = parity ? P.dir2 : P.dir;
  float* __restrict__ dout = parity ? P.dir : P.dir2;
  const unsigned short* __restrict__ codes = P.codes;
  float* __restrict__ q = P.q;
  {  // d = z (+ beta d), q = A d, d.q, alpha (k_dir_apply_dot)
    const int mode = sh.S.dir_mode;
    const float beta = sh.S.beta;
    const float* __restrict__ z = P.z;
    auto D = [&](int n) { return mode ? z[n] + beta * din[n] : z[n]; };
    double acc[1] = {0.0};
    strided_cells(tm, g.n, [&](int c) {
      const float dc = D(c);
      const unsigned code = codes[c];
      float qc = 0.f;
      if (code & RC_WET) { int i, j, k; cell_ijk(g, c, i, j, k); qc = apply_code(g, code, i, j, k, c, D); }
      dout[c] = dc;
      q[c] = qc;
      acc[0] += (double)dc * (double)qc;
    });
    crew_reduce<1>(sh, ph, acc, 0u, nullptr);
    crew_apply(sh, acc[0], FIN_DQ);
  }
  if (!sh.S.active) return;
  {  // p += alpha d, r -= alpha q, r.r (k_update_rn)
    const float alpha = sh.S.alpha;
    float* __restrict__ p = P.p;
    float* __restrict__ res = P.res;
    double acc[1] = {0.0};
    strided_cells(tm, g.n, [&](int c) {
      p[c] += alpha * dout[c];
      const float rn = res[c] - alpha * q[c];
      res[c] = rn;
      acc[0] += (double)rn * (double)rn;
    });
    crew_reduce<1>(sh, ph, acc, 0u, nullptr);
    crew_apply(sh, acc[0], FIN_RN);
  }
  if (!sh.S.active) return;
  batch_vcycle(tm, sh, ph, FIN_RZ_ITER);
}

struct BatchChecks {
  double actual, all, plain;
  float be;
  unsigned long long hash;
  int status;
};

// The checks that end or restart the outer loop (delta3d_mobile.rs:547-585): the true residual,
// the corrected field and its divergence metric (:398-433), the backward error (:243-271) and the
// fingerprint of p.
__device__ __forceinline__ BatchChecks batch_outer_checks(const ClusterTeam& tm, BatchShared& sh, int& ph) {
  const BatchPatch& P = sh.P;
  const Geo& g = P.g;
  batch_residual(tm, sh, ph, FIN_ACTUAL);
  for (int q = tm.rank(); q < P.nu + P.nv; q += tm.size()) correct_uv_at(g, P.codes, P.k1, P.p, P.us, P.vs, P.u, P.v, q);
  for (int f = tm.rank(); f < P.nw; f += tm.size()) correct_w_at(g, P.codes, P.k1, P.p, P.ws, P.w, f);
  tm.sync();
  float all = 0.f, plain = 0.f, mx = 0.f, be = 0.f;
  unsigned long long h = 0ull;
  for (int c = tm.rank(); c < g.n; c += tm.size()) {
    const unsigned code = P.codes[c];
    div_metric_cell(g, code, P.u, P.v, P.w, c, all, plain);
    be = fmaxf(be, backward_error_cell(g, code, P.p, P.rhs, P.res, c));
    h += hash_at(P.p, c);
  }
  for (int f = tm.rank(); f < P.nu; f += tm.size()) mx = fmaxf(mx, fabsf(P.u[f]));
  for (int f = tm.rank(); f < P.nv; f += tm.size()) mx = fmaxf(mx, fabsf(P.v[f]));
  for (int f = tm.rank(); f < P.nw; f += tm.size()) mx = fmaxf(mx, fabsf(P.w[f]));
  double m[4] = {(double)all, (double)plain, (double)mx, (double)be};
  crew_reduce<4>(sh, ph, m, 0xfu, &h);
  // delta3d_mobile.rs:426-432
  const float fall = (float)m[0], fplain = (float)m[1], fmx = (float)m[2];
  const float echelle = fmaxf(fmx, PROJECTION_VELOCITY_FLOOR);
  const float ratio = fmx > 0.f ? g.dx / echelle : 0.f;
  BatchChecks ck;
  ck.actual = sh.S.actual;
  ck.all = (double)(fall * ratio);
  ck.plain = (double)(fplain * ratio);
  ck.be = (float)m[3];
  ck.hash = h;
  ck.status = sh.S.status;
  return ck;
}

// project_mobile3 (delta3d_mobile.rs:465-609) of the patch in sh.P, its result into *out.
__device__ __forceinline__ void batch_project_one(const ClusterTeam& tm, BatchShared& sh, int& ph, BatchResult* out) {
  const BatchPatch& P = sh.P;
  const Geo& g = P.g;
  if (threadIdx.x == 0) {
    memset(&sh.S, 0, sizeof sh.S);
    sh.S.vinv = 1.f;
  }
  // the inputs: us = the field to project (the given one when set, else u); u itself is written
  // only by the correction, so a refusal before it leaves u as it was, and with given fields u is
  // saved first for a later refusal; the pressure is kept for a refusal; a non-finite input
  // refuses the patch
  double bad[1] = {0.0};
  for (int f = tm.rank(); f < P.nu + P.nv + P.nw; f += tm.size()) {
    float* dst;
    float* keep;
    float* save;
    const float* src;
    int q;
    if (f < P.nu) { q = f; dst = P.u; keep = P.us; save = P.sv_u; src = P.in_u; }
    else if (f < P.nu + P.nv) { q = f - P.nu; dst = P.v; keep = P.vs; save = P.sv_v; src = P.in_v; }
    else { q = f - P.nu - P.nv; dst = P.w; keep = P.ws; save = P.sv_w; src = P.in_w; }
    const float x = src ? src[q] : dst[q];
    if (!isfinite(x)) bad[0] = 1.0;
    if (src) save[q] = dst[q];
    keep[q] = x;
  }
  for (int c = tm.rank(); c < g.n; c += tm.size()) {
    P.sv_p[c] = P.p[c];
    if (P.reset_p) P.p[c] = 0.f;
  }
  crew_reduce<1>(sh, ph, bad, 1u, nullptr);
  BatchResult res{};
  if (bad[0] > 0.0) {
    res.status = FD3_ERR_NOT_FINITE;
  } else {
    // divergence of us (k_divergence)
    for (int c = tm.rank(); c < g.n; c += tm.size()) P.rhs[c] = divergence_at(g, P.us, P.vs, P.ws, c);
    tm.sync();
    // rhs_mobile3 with b.b, the row codes, p = 0 on the dry cells (k_rhs_b2)
    double b2v[1] = {0.0};
    for (int c = tm.rank(); c < g.n; c += tm.size()) {
      const float b = rhs_b2_at(g, P.scale, P.rhs, P.prec, P.codes, P.p, c);
      b2v[0] += (double)b * (double)b;
    }
    crew_reduce<1>(sh, ph, b2v, 0u, nullptr);
    crew_apply(sh, b2v[0], FIN_B2);
    // prepare_multigrid3 (delta3d_multigrid.rs:370-387): kinds and apertures, then diagonal and codes
    for (int l = 0; l < P.nlev; ++l) {
      const Lev C = P.lev[l];
      const int nfaces = (C.nx + 1) * C.ny * C.nz + C.nx * (C.ny + 1) * C.nz + C.nx * C.ny * (C.nz + 1);
      if (l == 0) {
        for (int q = tm.rank(); q < C.n; q += tm.size()) C.kind[q] = coarsen_kind_fine_at(g, C, q);
        for (int q = tm.rank(); q < nfaces; q += tm.size()) coarsen_open_at(g.nx, g.ny, g.ou, g.ov, g.ow, g.act, C, q);
      } else {
        const Lev F = P.lev[l - 1];
        for (int q = tm.rank(); q < C.n; q += tm.size()) C.kind[q] = coarsen_kind_level_at(F, C, q);
        for (int q = tm.rank(); q < nfaces; q += tm.size()) coarsen_open_at(F.nx, F.ny, F.ou, F.ov, F.ow, nullptr, C, q);
      }
      tm.sync();
      for (int c = tm.rank(); c < C.n; c += tm.size()) {
        C.diag[c] = level_diag_at(C, c);
        C.code[c] = (unsigned short)level_codes_at(C, c);
      }
      tm.sync();
    }
    batch_residual(tm, sh, ph, FIN_RR0);
    res.status = sh.S.status;
  }
  if (!res.status) {
    // the outer loop of project_mobile3 (the f64-reduction branch of the library's host loop)
    const double b2 = sh.S.b2;
    double rr = sh.S.rr;
    const double tolb2 = 1e-12 * b2;
    bool primed = false;
    unsigned it = 0;
    bool floor_stop = false;
    double phys = (double)INFINITY;
    bool has_checkpoint = false;
    unsigned long long checkpoint = 0ull;
    unsigned power = 1, since = 0;
    double actual_rr = 0.0;
    bool settled = false;
    double settled_d[2] = {0.0, 0.0};
    BatchChecks ck{};
    for (;;) {
      const unsigned before = it;
      if (b2 > 0 && (rr > tolb2 || rr > phys) && it < P.max_iters) {
        if (!primed) {
          batch_vcycle(tm, sh, ph, FIN_RZ_PRIME);
          primed = true;
        }
        if (threadIdx.x == 0) {  // k_loop_start
          sh.S.rr = rr; sh.S.tolb2 = tolb2; sh.S.phys = phys; sh.S.it = it; sh.S.max_iters = P.max_iters;
          sh.S.brk = 0; sh.S.body_runs = 0; sh.S.active = sh.S.status ? 0 : 1;
        }
        __syncthreads();
        int parity = 0;
        unsigned runs = 0;
        while (sh.S.active) {  // the guard of k_loop_cond: no more than max_iters + 2 iterations
          if (++runs > P.max_iters + 2u) {
            if (threadIdx.x == 0) { sh.S.active = 0; sh.S.status = 100; }
            __syncthreads();
            break;
          }
          batch_iteration(tm, sh, ph, parity);
          parity ^= 1;
        }
        if (sh.S.status) { res.status = sh.S.status; break; }
        it = sh.S.it;
        rr = sh.S.rr;
      }
      ck = batch_outer_checks(tm, sh, ph);
      if (ck.status) { res.status = ck.status; break; }
      const double actual = ck.actual;
      const bool exhausted = it >= P.max_iters || it == before;
      bool has_measured = false;
      double measured[2] = {0.0, 0.0};
      const bool converged = actual <= tolb2;
      if (converged) {
        if (exhausted) { actual_rr = actual; break; }
        if (ck.plain <= BATCH_DIV_TOL) { actual_rr = actual; settled = true; settled_d[0] = ck.all; settled_d[1] = ck.plain; break; }
        has_measured = true; measured[0] = ck.all; measured[1] = ck.plain;
        const double ratio = BATCH_DIV_TOL / ck.plain;
        phys = actual * ratio * ratio;
      } else if (exhausted) {
        actual_rr = actual;
        break;
      }
      if (ck.be <= (P.flat2d ? BATCH_ROUNDOFF_2D : BATCH_ROUNDOFF_3D)) {
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
      batch_vcycle(tm, sh, ph, FIN_RZ_PRIME);
    }
    if (!res.status) {
      const double div_all = settled ? settled_d[0] : ck.all, div_plain = settled ? settled_d[1] : ck.plain;
      const bool conv = actual_rr <= tolb2;
      const bool accepted = (conv || floor_stop) && div_plain <= BATCH_DIV_TOL;
      res.iterations = it;
      res.degraded = (b2 > 0 && !accepted) ? 1 : 0;
      res.residual = b2 > 0 ? sqrt(actual_rr / b2) : 0.0;
      res.divergence = div_all;
      res.floor_stop = floor_stop ? 1 : 0;
      res.backward_error = (double)ck.be;
      res.divergence_plain = div_plain;
    }
  }
  if (res.status) {  // a refusal publishes nothing: the fields the call started with come back
    const bool given = P.in_u != nullptr;
    for (int f = tm.rank(); f < P.nu; f += tm.size()) P.u[f] = given ? P.sv_u[f] : P.us[f];
    for (int f = tm.rank(); f < P.nv; f += tm.size()) P.v[f] = given ? P.sv_v[f] : P.vs[f];
    for (int f = tm.rank(); f < P.nw; f += tm.size()) P.w[f] = given ? P.sv_w[f] : P.ws[f];
    for (int c = tm.rank(); c < g.n; c += tm.size()) P.p[c] = P.sv_p[c];
  }
  tm.sync();
  if (tm.rank() == 0) {
    *out = res;
    *P.S = sh.S;
  }
}

// The persistent launch: cluster c projects order[start[c]] .. order[start[c + 1] - 1].
__global__ void __launch_bounds__(BATCH_THREADS, 1) k_batch_project(const BatchPatch* __restrict__ patches,
                                                                    const int* __restrict__ order,
                                                                    const int* __restrict__ start,
                                                                    BatchResult* __restrict__ results) {
  __shared__ BatchShared sh;
  const ClusterTeam tm;
  cooperative_groups::cluster_group cl = cooperative_groups::this_cluster();
  const int cid = (int)(blockIdx.x / cl.num_blocks());
  int ph = 0;
  for (int q = start[cid]; q < start[cid + 1]; ++q) {
    const int idx = order[q];
    if (threadIdx.x == 0) sh.P = patches[idx];
    __syncthreads();
    batch_project_one(tm, sh, ph, results + idx);
    __syncthreads();  // sh.P is rewritten for the next patch only after every thread is done with it
  }
}

}  // namespace fd3
