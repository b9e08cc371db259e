"""The cut geometry (delta3d_cut.rs) in the oracle against independent exact formulas (CPU only).

tests_delta3d_cut.rs:98-345 (S324, S329): a plane bottom gives the exact fluid fraction of each
interior cell; the cut is mirror-symmetric; a flat solid is the flat bottom of the same height and
an absent solid changes no bit; an oblique solid plane leaves each cell the exact solid part of a
cube cut by a plane; an immersed sphere's displaced volume converges at order >= 1.8, mirror-
symmetric; a solid sharing a cell with the bottom or reaching the lid layer is refused.  The GPU's
cut geometry is bit-identical to the oracle's (tests/test_gpu_parity.py).
"""
import math

import numpy as np
import pytest

from fluidisim_b200 import scenes
from oracle import oracle as O

f32 = np.float32


@pytest.fixture(scope="module", autouse=True)
def _threads():
    O.build()
    O.set_threads(min(8, O.max_threads()))


def nodes(nx, ny, nz, dx, f):
    """A signed distance evaluated in f64 at the nodes (x fastest), rounded to f32."""
    d = np.float64(f32(dx))
    k, j, i = np.meshgrid(np.arange(nz + 1), np.arange(ny + 1), np.arange(nx + 1), indexing="ij")
    return f(i * d, j * d, k * d).astype(np.float32).ravel()


def plane_fraction(p0, alpha, beta, dx, low, samples=200_000):
    """The fluid fraction of the cell [low, low + dx] above the plane p0 + alpha X + beta Y over its
    footprint: the mean over the cell's heights of P(bottom < z), the bottom being min + U with U
    the sum of two uniform variables on [0, |alpha| dx] and [0, |beta| dx] (a trapezoidal law)."""
    a, b = abs(alpha * dx), abs(beta * dx)
    a, b = max(a, b), min(a, b)
    lowest = p0 + min(alpha * dx, 0.0) + min(beta * dx, 0.0)
    u = low + (np.arange(samples) + 0.5) * (dx / samples) - lowest
    cdf = np.where(u <= b, u * u / (2 * a * b),
                   np.where(u <= a, (2 * u - b) / (2 * a), 1 - (a + b - u) ** 2 / (2 * a * b)))
    cdf = np.where(u <= 0, 0.0, np.where(u >= a + b, 1.0, cdf))
    return float(cdf.mean())


def test_a_plane_bottom_is_cut_exactly():
    """tests_delta3d_cut.rs:127-148: 7 x 6 x 12 cells of 0.25 m over 0.37 + 0.21 x - 0.13 y; every
    interior footprint's fractions within 2e-6 of the exact ones."""
    nx, ny, nz, dx = 7, 6, 12, f32(0.25)
    g, alpha, beta = f32(0.37), f32(0.21), f32(-0.13)
    plane = lambda x, y: g + alpha * x + beta * y  # noqa: E731
    bottom = np.array([plane((f32(i) + f32(0.5)) * dx, (f32(j) + f32(0.5)) * dx) for j in range(ny) for i in range(nx)],
                      np.float32)
    frac = O.OracleVolume(nx, ny, nz, dx, 1025.0, 9.81, bottom=bottom).geometry()[0].reshape(nz, ny, nx)
    worst = 0.0
    for j in range(1, ny - 1):
        for i in range(1, nx - 1):
            p0 = float(plane(f32(i) * dx, f32(j) * dx))
            for k in range(nz):
                exact = plane_fraction(p0, float(alpha), float(beta), float(dx), k * float(dx))
                worst = max(worst, abs(float(frac[k, j, i]) - exact))
    assert worst < 2e-6, worst


def test_the_cut_is_mirror_symmetric():
    """tests_delta3d_cut.rs:200-216: the bottom mirrored in x gives the mirrored fractions to 1e-6."""
    nx, ny, nz, dx = 8, 5, 9, 0.25

    def h(i, j):
        return f32(0.9) + f32(0.3) * scenes.sinf(f32(i * i) * f32(0.37)) + f32(0.2) * f32(math.cos(float(f32(j) * f32(1.3))))

    bottom = np.array([h(i, j) for j in range(ny) for i in range(nx)], np.float32)
    mirror = np.array([h(nx - 1 - i, j) for j in range(ny) for i in range(nx)], np.float32)
    a = O.OracleVolume(nx, ny, nz, dx, 1025.0, 9.81, bottom=bottom).geometry()[0].reshape(nz, ny, nx)
    b = O.OracleVolume(nx, ny, nz, dx, 1025.0, 9.81, bottom=mirror).geometry()[0].reshape(nz, ny, nx)
    assert np.max(np.abs(a - b[:, :, ::-1])) < 1e-6


def test_a_flat_solid_is_a_flat_bottom_and_an_absent_one_changes_nothing():
    """tests_delta3d_cut.rs:236-260: a horizontal solid plane at 0.61 m cuts like a bottom at 0.61 m
    (1e-6); a solid that is nowhere (distance 1 at every node) leaves a bump's cut to the bit."""
    nx, ny, nz, dx = 6, 5, 8, 0.25
    zp = f32(0.61)
    flat = nodes(nx, ny, nz, dx, lambda x, y, z: z - np.float64(zp))
    g = O.OracleVolume(nx, ny, nz, dx, 1025.0, 9.81, bottom=np.zeros(nx * ny, np.float32), solid=flat).geometry()
    h = O.OracleVolume(nx, ny, nz, dx, 1025.0, 9.81, bottom=np.full(nx * ny, zp, np.float32)).geometry()
    for a, b in zip(g[:4], h[:4]):
        assert np.max(np.abs(a - b)) <= 1e-6
    bump = np.array([f32(0.2) + f32(0.3) * scenes.expf(-(((f32(i) + f32(0.5)) * f32(0.25) - f32(0.7)) ** 2
                                                         + ((f32(j) + f32(0.5)) * f32(0.25) - f32(0.6)) ** 2) / f32(0.1))
                     for j in range(ny) for i in range(nx)], np.float32)
    absent = np.ones((nx + 1) * (ny + 1) * (nz + 1), np.float32)
    g = O.OracleVolume(nx, ny, nz, dx, 1025.0, 9.81, bottom=bump, solid=absent).geometry()
    h = O.OracleVolume(nx, ny, nz, dx, 1025.0, 9.81, bottom=bump).geometry()
    for a, b in zip(g, h):
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


def test_an_oblique_solid_plane_is_cut_exactly():
    """tests_delta3d_cut.rs:262-289: the solid 0.3 x + 0.5 y + 0.8 z < 0.55 in 8^3 cells of
    0.125 m; each cell's solid part within 2e-6 of the cube-plane volume by inclusion-exclusion
    over its eight vertices, and more than 50 cells cut."""
    n, dx = 8, 0.125
    a, b, c, e = 0.3, 0.5, 0.8, 0.55
    solid = nodes(n, n, n, dx, lambda x, y, z: a * x + b * y + c * z - e)
    frac = O.OracleVolume(n, n, n, dx, 1025.0, 9.81, bottom=np.zeros(n * n, np.float32),
                          solid=solid).geometry()[0].reshape(n, n, n)
    al, be, ga = a * dx, b * dx, c * dx
    cut = 0
    for k in range(n):
        for j in range(n):
            for i in range(n):
                rest = e - (a * i + b * j + c * k) * dx
                v = 0.0
                for s in range(8):
                    p, q, r = s & 1, (s >> 1) & 1, s >> 2
                    sign = 1.0 if bin(s).count("1") % 2 == 0 else -1.0
                    v += sign * max(rest - al * p - be * q - ga * r, 0.0) ** 3
                exact = min(max(v / (6 * al * be * ga), 0.0), 1.0)
                assert abs((1.0 - float(frac[k, j, i])) - exact) <= 2e-6, (i, j, k)
                cut += 0.0 < exact < 1.0
    assert cut > 50


def test_an_immersed_sphere_displaces_its_volume_at_second_order():
    """tests_delta3d_cut.rs:300-333 (the volume part): a sphere of 0.3 m in a 1.2 m cube at 12, 24 and
    48 cells: mirror-symmetric fractions (1e-6) and the displaced volume converging to 4/3 pi R^3 at
    order >= 1.8."""
    exact = 4.0 / 3.0 * math.pi * 0.3 ** 3
    errors = []
    for n in (12, 24, 48):
        dx = f32(1.2) / f32(n)
        s = scenes.spheres_sdf(n, n, n, dx, [(0.6, 0.6, 0.55)], [0.3])
        frac = O.OracleVolume(n, n, n, dx, 1025.0, 9.81, bottom=np.zeros(n * n, np.float32),
                              solid=s).geometry()[0].reshape(n, n, n)
        assert np.max(np.abs(frac - frac[:, :, ::-1])) <= 1e-6
        volume = float(np.sum(1.0 - frac.astype(np.float64)) * np.float64(dx) ** 3)
        errors.append(volume - exact)
    o1 = math.log2(abs(errors[0] / errors[1]))
    o2 = math.log2(abs(errors[1] / errors[2]))
    assert o1 >= 1.8 and o2 >= 1.8, (o1, o2)


@pytest.mark.parametrize("bottom,cz", [(0.3, 0.4), (0.0, 0.85)])
def test_a_solid_sharing_a_cell_with_the_bottom_or_reaching_the_lid_is_refused(bottom, cz):
    """tests_delta3d_cut.rs:335-345: a sphere of 0.2 m at (0.5, 0.5, cz) in 8^3 cells of 0.125 m."""
    n, dx = 8, 0.125
    s = nodes(n, n, n, dx, lambda x, y, z: np.sqrt((x - 0.5) ** 2 + (y - 0.5) ** 2 + (z - cz) ** 2) - 0.2)
    with pytest.raises(O.OracleError) as e:
        O.OracleVolume(n, n, n, dx, 1025.0, 9.81, bottom=np.full(n * n, bottom, np.float32), solid=s)
    assert e.value.kind == "Domain"
