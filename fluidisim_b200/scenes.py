"""Seeded synthetic scenes for the delta projection.

Every scene is plain numpy data in the reference's layouts (code/water-core/src/delta3d.rs:24-28):
cells and columns x-fastest, faces u/v/w per axis, SDF nodes (nx+1)(ny+1)(nz+1) x-fastest.
Scalar f32 arithmetic that the reference performs in f32 is done here in f32 too, and
transcendental functions go through the C library's `sinf`/`expf` (what Rust's f32 methods call
on Linux), so that the oracle and the GPU see bit-identical inputs.

Scenes:
  * `s385_case`       the multigrid bench of code/water-core/examples/delta3d_multigrille.rs:26-94
  * `noise`           the xorshift U[-1,1) generator of code/water-core/src/tests_delta3d.rs:66-75
  * `sphere_lake`     64^3 closed box, 8 random spheres, lower half liquid, U[-1,1] faces
  * `box_basin`       128^3, 16 random boxes, sinusoidal surface, curl background + N(0,0.5)
Random draws use the project's SplitMix64 (`SplitMix64`), never numpy's global generator.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

_libm = C.CDLL("libm.so.6")
_libm.sinf.argtypes = [C.c_float]
_libm.sinf.restype = C.c_float
_libm.expf.argtypes = [C.c_float]
_libm.expf.restype = C.c_float

f32 = np.float32
TAU32 = f32(2.0 * math.pi)  # core::f32::consts::TAU


def sinf(x) -> np.float32:
    return f32(_libm.sinf(float(f32(x))))


def expf(x) -> np.float32:
    return f32(_libm.expf(float(f32(x))))


class SplitMix64:
    """SplitMix64 (Steele, Lea, Flood 2014): the project's seeded generator."""

    M = (1 << 64) - 1

    def __init__(self, seed: int):
        self.s = seed & self.M

    def next_u64(self) -> int:
        self.s = (self.s + 0x9E3779B97F4A7C15) & self.M
        z = self.s
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & self.M
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & self.M
        return z ^ (z >> 31)

    def uniform(self, lo=0.0, hi=1.0) -> float:
        return lo + (hi - lo) * ((self.next_u64() >> 11) * (1.0 / (1 << 53)))

    def normal_array(self, n: int, sigma: float) -> np.ndarray:
        """n draws of N(0, sigma) (f32) by Box-Muller on two counter-based SplitMix64 streams."""
        m = (n + 1) // 2
        u1 = self._unit_stream(m, offset=0.5)
        u2 = self._unit_stream(m, offset=0.0)
        r = np.sqrt(-2.0 * np.log(u1))
        t = 2.0 * np.pi * u2
        z = np.concatenate([r * np.cos(t), r * np.sin(t)])[:n]
        return (sigma * z).astype(np.float32)

    def _unit_stream(self, n: int, offset: float = 0.0) -> np.ndarray:
        """n f64 values in [0,1) (offset 0.5 shifts them into (0,1)) from a SplitMix64 counter stream
        whose base is the next draw of this generator."""
        base = np.uint64(self.next_u64())
        idx = np.arange(n, dtype=np.uint64)
        with np.errstate(over="ignore"):
            z = base + (idx + np.uint64(1)) * np.uint64(0x9E3779B97F4A7C15)
            z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
            z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
            z = z ^ (z >> np.uint64(31))
        return ((z >> np.uint64(11)).astype(np.float64) + offset) * (1.0 / (1 << 53))

    def uniform_array(self, n: int, lo: float, hi: float) -> np.ndarray:
        """n draws of U[lo, hi) as f32 from a counter-based SplitMix64 stream."""
        return (lo + (hi - lo) * self._unit_stream(n)).astype(np.float32)


def noise(n: int, seed: int) -> np.ndarray:
    """Deterministic U[-1,1) f32 (tests_delta3d.rs:66-75): xorshift on a u64 state."""
    M = (1 << 64) - 1
    s = ((seed * 0x9E3779B97F4A7C15) & M) | 1
    out = np.empty(n, dtype=np.float32)
    for q in range(n):
        s ^= (s << 13) & M
        s ^= s >> 7
        s ^= (s << 17) & M
        out[q] = f32(f32(f32(s >> 40) / f32(1 << 24)) * f32(2.0)) - f32(1.0)
    return out


# ----------------------------------------------------------------------------------------------
# The reference's multigrid bench (examples/delta3d_multigrille.rs): 8 x 4 x 6 m, surface at rest
# 4 m, a 1 cm sine along x, dt = 2 ms; flat bottom or the off-centre bump of S324.
S385_LX, S385_LZ, S385_A = f32(8.0), f32(4.0), f32(0.01)
S385_RHO, S385_G, S385_DT_US = 1025.0, 9.81, 2000


def s385_bump(x: np.float32, y: np.float32) -> np.float32:
    a = f32(f32(x - f32(3.0)) / f32(1.2))
    b = f32(f32(y - f32(1.3)) / f32(0.9))
    return f32(0.4) + f32(0.6) * expf(-(f32(a * a) + f32(b * b)))


def s385_case(nx: int, bump: bool = False) -> dict:
    """Domain, bottom (None for flat) and free surface of the S385 bench at resolution nx."""
    ny, nz = nx // 2, 3 * nx // 4
    dx = f32(S385_LX / f32(nx))
    row = np.array([S385_LZ + S385_A * sinf(f32(f32(TAU32 * f32(f32(i) + f32(0.5))) * dx) / S385_LX)
                    for i in range(nx)], dtype=np.float32)
    eta = np.tile(row, ny)
    bottom = None
    if bump:
        bottom = np.array([s385_bump(f32(f32(f32(i) + f32(0.5)) * dx), f32(f32(f32(j) + f32(0.5)) * dx))
                           for j in range(ny) for i in range(nx)], dtype=np.float32)
    return dict(nx=nx, ny=ny, nz=nz, dx=float(dx), rho=S385_RHO, g=S385_G, bottom=bottom, eta=eta,
                rest=float(S385_LZ), dt_us=S385_DT_US)


# ----------------------------------------------------------------------------------------------
# The linear path's cut-bottom bench (examples/delta3d_fond_coupe.rs): 8 x 4 x 4 m, lid
# eta = z0 + 0.01 sin(2 pi x / 8), one 2 ms step from rest; the smooth bottom of S232 (independent
# of y) or the off-centre bump.

def s324_smooth(x: np.float32, y: np.float32) -> np.float32:
    d = f32(f32(x - f32(3.0)) / f32(1.2))
    return f32(0.4) + f32(0.6) * expf(-f32(d * d))


def s324_case(nx: int, bump: bool = True) -> dict:
    """Domain nx x nx/2 x nx/2, dx = 8/nx, its bottom and its lid heights."""
    ny = nz = nx // 2
    dx = f32(S385_LX / f32(nx))
    fond = s385_bump if bump else s324_smooth
    bottom = np.array([fond(f32(f32(f32(i) + f32(0.5)) * dx), f32(f32(f32(j) + f32(0.5)) * dx))
                       for j in range(ny) for i in range(nx)], dtype=np.float32)
    z0 = f32(f32(nz) * dx)
    row = np.array([z0 + S385_A * sinf(f32(f32(TAU32 * f32(f32(i) + f32(0.5))) * dx) / S385_LX)
                    for i in range(nx)], dtype=np.float32)
    return dict(nx=nx, ny=ny, nz=nz, dx=float(dx), rho=S385_RHO, g=S385_G, bottom=bottom, eta=np.tile(row, ny),
                dt_us=S385_DT_US)


def open_flux_x(ou: np.ndarray, u: np.ndarray, nx: int, ny: int, nz: int, dx: float) -> float:
    """Open flux through x = L/2, sum of aperture * u * dx^2 in f64 (delta3d_fond_coupe.rs:83-90)."""
    i = nx // 2
    f = (np.arange(nz)[:, None] * ny + np.arange(ny)[None, :]) * (nx + 1) + i
    q = 0.0
    for ff in f.ravel():
        q += float(ou[ff]) * float(u[ff]) * float(dx) * float(dx)
    return q


def oblique_wave(n: int, g: float = 9.81) -> dict:
    """Mode (1, 1) of an 8 x 4 m tank, h = 4 m, A = 1 cm, at rest (tests_delta3d.rs:312-343)."""
    lx, ly, h, a = 8.0, 4.0, 4.0, 0.01
    dx = lx / n
    nx, ny, nz = n, int(ly / dx), int(h / dx)
    kx, ky = np.pi / lx, np.pi / ly
    jj, ii = np.meshgrid(np.arange(ny), np.arange(nx), indexing="ij")
    mode = np.cos(kx * (ii + 0.5) * dx) * np.cos(ky * (jj + 0.5) * dx)
    return dict(nx=nx, ny=ny, nz=nz, dx=float(np.float32(dx)), rho=1025.0, g=float(np.float32(g)),
                eta=(h + a * mode).astype(np.float32).ravel(), mode=mode.ravel(), h=h, a=a, kx=kx, ky=ky)


def scheme_frequency(kx: float, ky: float, dx: float, nz: int, g: float, dt: float):
    """Frequency of the linear scheme for mode (kx, ky) and its symplectic half-step term
    (tests_delta3d.rs:281-310): discrete horizontal eigenvalue, vertical structure of the
    Neumann-bottom / half-cell-Dirichlet-lid problem (Thomas), symplectic Euler."""
    kappa2 = 4.0 / (dx * dx) * (np.sin(kx * dx / 2.0) ** 2 + np.sin(ky * dx / 2.0) ** 2)
    a = [0.0] * nz
    b = [0.0] * nz
    c = [0.0] * nz
    d = [0.0] * nz
    for k in range(nz):
        diag = kappa2 * dx * dx
        if k > 0:
            diag += 1.0
            a[k] = -1.0
        if k + 1 < nz:
            diag += 1.0
            c[k] = -1.0
        else:
            diag += 2.0
            d[k] = 2.0
        b[k] = diag
    for k in range(1, nz):
        m = a[k] / b[k - 1]
        b[k] -= m * c[k - 1]
        d[k] -= m * d[k - 1]
    phi = [0.0] * nz
    phi[nz - 1] = d[nz - 1] / b[nz - 1]
    for k in range(nz - 2, -1, -1):
        phi[k] = (d[k] - c[k] * phi[k + 1]) / b[k]
    ws2 = g * kappa2 * sum(x * dx for x in phi)
    big = np.arccos(1.0 - ws2 * dt * dt / 2.0) / dt
    return big, -ws2 * dt * dt / (2.0 * np.sin(big * dt))


# ----------------------------------------------------------------------------------------------
# Signed distances at the nodes, (nx+1)(ny+1)(nz+1) x-fastest, negative inside (delta3d.rs:322-327).

def _node_axes(nx, ny, nz, dx):
    """Node coordinates per axis, shaped to broadcast over the (z, y, x) node grid."""
    d = float(f32(dx))
    return (np.arange(nx + 1)[None, None, :] * d, np.arange(ny + 1)[None, :, None] * d,
            np.arange(nz + 1)[:, None, None] * d)


def spheres_sdf(nx, ny, nz, dx, centres, radii) -> np.ndarray:
    """Union of spheres (centres, radii in metres), as the sphere nodes of tests_delta3d.rs:1161-1179.
    Each sphere's distance is evaluated by broadcasting the three axes, one z layer block at a time
    (the same f64 operations, node by node, as on a full mesh grid)."""
    x, y, z = _node_axes(nx, ny, nz, dx)
    out = np.full((nz + 1, ny + 1, nx + 1), np.inf)
    for (cx, cy, cz), r in zip(centres, radii):
        xy = (x - cx) ** 2 + (y - cy) ** 2
        for k0 in range(0, nz + 1, 16):
            zz = z[k0:k0 + 16]
            np.minimum(out[k0:k0 + 16], np.sqrt(xy + (zz - cz) ** 2) - r, out=out[k0:k0 + 16])
    return out.astype(np.float32).ravel()


def boxes_sdf(nx, ny, nz, dx, centres, halves) -> np.ndarray:
    """Union of boxes (centre, half sizes in metres), the box distance of tests_delta3d.rs:1332-1350."""
    x, y, z = _node_axes(nx, ny, nz, dx)
    out = np.full((nz + 1, ny + 1, nx + 1), np.inf)
    for c, h in zip(centres, halves):
        qx, qy = np.abs(x - c[0]) - h[0], np.abs(y - c[1]) - h[1]
        sx, sy = np.maximum(qx, 0.0) ** 2, np.maximum(qy, 0.0) ** 2
        mxy = np.maximum(qx, qy)
        for k0 in range(0, nz + 1, 16):
            qz = np.abs(z[k0:k0 + 16] - c[2]) - h[2]
            outside = np.sqrt(0 + sx + sy + np.maximum(qz, 0.0) ** 2)
            inside = np.minimum(np.maximum(mxy, qz), 0.0)
            np.minimum(out[k0:k0 + 16], outside + inside, out=out[k0:k0 + 16])
    return out.astype(np.float32).ravel()


def face_counts(nx, ny, nz):
    return (nx + 1) * ny * nz, nx * (ny + 1) * nz, nx * ny * (nz + 1)


def sphere_lake(n: int = 64, seed: int = 1, dx: float = 0.1, spheres: int = 8) -> dict:
    """Closed n^3 box, `spheres` random solid spheres (radius U[3,8] cells, clear of the walls, of the
    lid layer and of the top two liquid layers), liquid filling the lower half, faces U[-1,1] m/s
    (set_velocity zeroes the closed faces).  dt = 1/60 s; project with scale = -rho/dt, k1 = dt/rho."""
    rng = SplitMix64(seed)
    d = float(f32(dx))
    eta_cells = n // 2
    centres, radii = [], []
    for _ in range(spheres):
        r = rng.uniform(3.0, 8.0)
        cx = rng.uniform(r + 1.0, n - r - 1.0)
        cy = rng.uniform(r + 1.0, n - r - 1.0)
        cz = rng.uniform(r + 1.0, eta_cells - 2.0 - r)
        centres.append((cx * d, cy * d, cz * d))
        radii.append(r * d)
    sdf = spheres_sdf(n, n, n, dx, centres, radii)
    nu, nv, nw = face_counts(n, n, n)
    return dict(nx=n, ny=n, nz=n, dx=float(f32(dx)), rho=1025.0, g=9.81, bottom=np.zeros(n * n, np.float32),
                solid=sdf, eta=np.full(n * n, f32(eta_cells * d), np.float32), rest=float(f32(eta_cells * d)),
                u=rng.uniform_array(nu, -1.0, 1.0), v=rng.uniform_array(nv, -1.0, 1.0),
                w=rng.uniform_array(nw, -1.0, 1.0), dt=1.0 / 60.0)


def box_basin(n: int = 128, seed: int = 2, dx: float = 0.1, boxes: int = 16, noise_sigma: float = 0.5) -> dict:
    """n^3 basin: free surface h = n/2 + sum_{k=1..6} a_k sin(kx x + ky y + phi_k) cells with a_k ~
    U[1,4] (one height per column: the reference's vertical axis is z), `boxes` random submerged
    solid boxes, a divergence-free background (discrete curl of a seeded smooth vector potential on
    the cell edges) plus i.i.d. N(0, noise_sigma) m/s face noise."""
    rng = SplitMix64(seed)
    d = float(f32(dx))
    i = (np.arange(n) + 0.5)
    X, Y = np.meshgrid(i, i, indexing="xy")
    h = np.full((n, n), 0.5 * n)
    for _ in range(6):
        a = rng.uniform(1.0, 4.0)
        kx = rng.uniform(-3.0, 3.0) * 2 * np.pi / n
        ky = rng.uniform(-3.0, 3.0) * 2 * np.pi / n
        ph = rng.uniform(0.0, 2 * np.pi)
        h += a * np.sin(kx * X + ky * Y + ph)
    hmin = float(h.min())
    eta = (h * d).astype(np.float32).ravel()
    centres, halves = [], []
    top_limit = hmin - 4.0
    for _ in range(boxes):
        hx, hy, hz = rng.uniform(2.0, 8.0), rng.uniform(2.0, 8.0), rng.uniform(2.0, 6.0)
        cx = rng.uniform(hx + 1.0, n - hx - 1.0)
        cy = rng.uniform(hy + 1.0, n - hy - 1.0)
        cz = rng.uniform(hz + 1.0, max(hz + 1.5, top_limit - hz))
        centres.append((cx * d, cy * d, cz * d))
        halves.append((hx * d, hy * d, hz * d))
    sdf = boxes_sdf(n, n, n, dx, centres, halves)
    # vector potential on the edges: Ax at (i+1/2, j, k), Ay at (i, j+1/2, k), Az at (i, j, k+1/2)
    def potential(sx, sy, sz):
        zz, yy, xx = np.meshgrid(np.arange(n + 1) + sz, np.arange(n + 1) + sy, np.arange(n + 1) + sx, indexing="ij")
        out = np.zeros(xx.shape)
        for _ in range(4):
            kx, ky, kz = (rng.uniform(0.5, 3.0) * 2 * np.pi / n for _ in range(3))
            amp = rng.uniform(0.5, 1.5) * n * d / (2 * np.pi * 3)
            ph = rng.uniform(0.0, 2 * np.pi)
            out += amp * np.sin(kx * xx + ky * yy + kz * zz + ph)
        return out
    Ax = potential(0.5, 0.0, 0.0)
    Ay = potential(0.0, 0.5, 0.0)
    Az = potential(0.0, 0.0, 0.5)
    # u(i,j,k) at x = i, y = j+1/2, z = k+1/2: dAz/dy - dAy/dz
    u = ((Az[:n, 1:n + 1, :n + 1] - Az[:n, :n, :n + 1]) - (Ay[1:n + 1, :n, :n + 1] - Ay[:n, :n, :n + 1])) / d
    v = ((Ax[1:n + 1, :n + 1, :n] - Ax[:n, :n + 1, :n]) - (Az[:n, :n + 1, 1:n + 1] - Az[:n, :n + 1, :n])) / d
    w = ((Ay[:n + 1, :n, 1:n + 1] - Ay[:n + 1, :n, :n]) - (Ax[:n + 1, 1:n + 1, :n] - Ax[:n + 1, :n, :n])) / d
    nu, nv, nw = face_counts(n, n, n)
    u = u.astype(np.float32).ravel() + rng.normal_array(nu, noise_sigma)
    v = v.astype(np.float32).ravel() + rng.normal_array(nv, noise_sigma)
    w = w.astype(np.float32).ravel() + rng.normal_array(nw, noise_sigma)
    return dict(nx=n, ny=n, nz=n, dx=float(f32(dx)), rho=1025.0, g=9.81, bottom=np.zeros(n * n, np.float32),
                solid=sdf, eta=eta, rest=float(f32(0.5 * n * d)), u=u.astype(np.float32), v=v.astype(np.float32),
                w=w.astype(np.float32), dt=1.0 / 60.0)


def breaking_wave(n: int = 256, seed: int = 5, dx: float = 0.1, obstacles: int = 32, crest_speed: float = 2.0,
                  noise_sigma: float = 0.3) -> dict:
    """n^3 breaking-wave state: h = 0.4 n + 0.15 n tanh((x - x0)/8) (1 + 0.1 sin(y/5)) cells (x, y in
    cells, x0 = n/2; one height per column, the reference's vertical axis being z), `obstacles`
    random submerged solids (spheres and boxes alternately, clear of the walls and 4 cells below
    the lowest surface), u = crest_speed m/s on the wet u faces of the crest (the columns with
    h > 0.45 n) plus i.i.d. N(0, noise_sigma) m/s on every face."""
    rng = SplitMix64(seed)
    d = float(f32(dx))
    i = np.arange(n) + 0.5
    X, Y = np.meshgrid(i, i, indexing="xy")
    x0 = 0.5 * n
    h = 0.4 * n + 0.15 * n * np.tanh((X - x0) / 8.0) * (1.0 + 0.1 * np.sin(Y / 5.0))
    hmin = float(h.min())
    eta = (h * d).astype(np.float32).ravel()
    top_limit = hmin - 4.0
    sph_c, sph_r, box_c, box_h = [], [], [], []
    for q in range(obstacles):
        if q % 2 == 0:
            r = rng.uniform(3.0, 8.0)
            cx = rng.uniform(r + 1.0, n - r - 1.0)
            cy = rng.uniform(r + 1.0, n - r - 1.0)
            cz = rng.uniform(r + 1.0, max(r + 1.5, top_limit - r))
            sph_c.append((cx * d, cy * d, cz * d))
            sph_r.append(r * d)
        else:
            hx, hy, hz = rng.uniform(2.0, 8.0), rng.uniform(2.0, 8.0), rng.uniform(2.0, 6.0)
            cx = rng.uniform(hx + 1.0, n - hx - 1.0)
            cy = rng.uniform(hy + 1.0, n - hy - 1.0)
            cz = rng.uniform(hz + 1.0, max(hz + 1.5, top_limit - hz))
            box_c.append((cx * d, cy * d, cz * d))
            box_h.append((hx * d, hy * d, hz * d))
    sdf = np.minimum(spheres_sdf(n, n, n, dx, sph_c, sph_r), boxes_sdf(n, n, n, dx, box_c, box_h))
    nu, nv, nw = face_counts(n, n, n)
    # u faces (i, j, k), x = i: crest columns on either side, wet below the surface
    crest = h > 0.45 * n
    col_crest = np.zeros((n, n + 1), bool)
    col_crest[:, :n] |= crest
    col_crest[:, 1:] |= crest
    zc = (np.arange(n) + 0.5)[:, None, None]
    hh = np.zeros((n, n + 1))
    hh[:, :n] = h
    hh[:, n] = h[:, n - 1]
    wet_u = zc < hh[None, :, :]
    u = np.where(col_crest[None, :, :] & wet_u, crest_speed, 0.0).astype(np.float32).ravel()
    u = u + rng.normal_array(nu, noise_sigma)
    v = rng.normal_array(nv, noise_sigma)
    w = rng.normal_array(nw, noise_sigma)
    return dict(nx=n, ny=n, nz=n, dx=float(f32(dx)), rho=1025.0, g=9.81, bottom=np.zeros(n * n, np.float32),
                solid=sdf.astype(np.float32), eta=eta, rest=float(f32(0.4 * n * d)), u=u.astype(np.float32),
                v=v.astype(np.float32), w=w.astype(np.float32), dt=1.0 / 60.0)


def projection_scalars(scene: dict):
    """(scale, k1) of a projection with the scene's dt: -rho/dt and dt/rho, rounded to f32 as
    step_surface_mobile does (delta3d_mobile.rs:838-840)."""
    dt, rho = scene["dt"], scene["rho"]
    return float(f32(-rho / dt)), float(f32(dt / rho))


# ------------------------------------------------------------------------------------------------
# Sparse column sets (delta3d_sparse.rs), the scenes of tests_delta3d_sparse.rs:8-36, 198-225.

SPARSE_DX, SPARSE_NZ, SPARSE_REST = 0.25, 12, 2.0


def rect_mask(nx: int, ny: int, rects) -> np.ndarray:
    """Column mask (j*nx + i) of the union of rectangles [i0, i1) x [j0, j1)."""
    m = np.zeros((ny, nx), np.uint8)
    for i0, i1, j0, j1 in rects:
        m[j0:j1, i0:i1] = 1
    return m.ravel()


def bumps_in(nx: int, ny: int, mask, centres, rest: float = SPARSE_REST) -> np.ndarray:
    """Surface of a window: rest + sum of 5 cm Gaussian bumps exp(-r^2/8) (r in cells) in the set's
    columns, exactly `rest` outside the set."""
    mask = np.asarray(mask).reshape(-1)
    out = np.empty(nx * ny, np.float32)
    r = f32(rest)
    for c in range(nx * ny):
        if mask[c] == 0:
            out[c] = r
            continue
        i, j = c % nx, c // nx
        s = f32(0.0)
        for cx, cy in centres:
            x = f32(f32(i) + f32(0.5)) - f32(cx)
            y = f32(f32(j) + f32(0.5)) - f32(cy)
            s = f32(s + f32(f32(0.05) * expf(f32(-(f32(x * x) + f32(y * y))) / f32(8.0))))
        out[c] = f32(r + s)
    return out


def sparse_window(n: int = 256, nz: int = 32, seed: int = 6, half_width_blocks: int = 3) -> dict:
    """A n x n x nz window at 25 cm, 4 m of water at rest, whose sparse set is the blocks of 8 x 8
    columns within `half_width_blocks` blocks of a curved path across it (the kind of set that
    follows a moving source).  In the set: a train of 5 cm bumps along the path and N(0, 0.3) m/s
    face noise; outside it the surface is at rest (the faces there are closed by set_velocity)."""
    rng = SplitMix64(seed)
    nb = n // 8
    blocks = np.zeros((nb, nb), np.uint8)
    path = []
    jj, ii = np.mgrid[0:nb, 0:nb]
    for t in np.linspace(0.0, 1.0, 4 * nb):
        bx = 0.15 * nb + 0.7 * nb * t
        by = 0.5 * nb + 0.3 * nb * math.sin(2 * math.pi * t)
        path.append((bx, by))
        blocks |= ((np.abs(ii + 0.5 - bx) <= half_width_blocks) & (np.abs(jj + 0.5 - by) <= half_width_blocks)).astype(np.uint8)
    mask = np.kron(blocks, np.ones((8, 8), np.uint8)).ravel()
    dx, rest = float(f32(0.25)), float(f32(4.0))
    centres = [(8 * bx, 8 * by) for bx, by in path[:: max(1, len(path) // 6)]]
    j, i = np.mgrid[0:n, 0:n]
    h = np.zeros((n, n))
    for cx, cy in centres:
        h += 0.05 * np.exp(-((i + 0.5 - cx) ** 2 + (j + 0.5 - cy) ** 2) / 32.0)
    eta = np.where(mask.reshape(n, n) != 0, rest + h, rest).astype(np.float32).ravel()
    nu, nv, nw = face_counts(n, n, nz)
    return dict(nx=n, ny=n, nz=nz, dx=dx, rho=1000.0, g=9.81, mask=mask, eta=eta, rest=rest,
                u=rng.normal_array(nu, 0.3), v=rng.normal_array(nv, 0.3), w=rng.normal_array(nw, 0.3), dt=0.02)
