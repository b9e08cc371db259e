"""A truly three-dimensional cut bottom in the oracle (CPU only).

The reference's own criteria for the cut bottom (tests_delta3d.rs:845-1159, S324, S326, S328):
a lake at rest on the bump stays at rest to the bit in the linear and the mobile step; one linear
step from a bumpy surface leaves an open field within the divergence tolerance with nothing on the
closed faces and a transverse flow; the Jacobi preconditioner of the cut path keeps the solution
and halves the iterations at least; a bottom without y keeps its mobile slices identical; a free
surface within two cells of the bottom's highest corner is refused with the state kept.
"""
import numpy as np
import pytest

from fluidisim_b200 import scenes
from oracle import oracle as O

TOL = 1e-5  # PROJECTION_DIVERGENCE_TOLERANCE (delta_projection.rs:192)


@pytest.fixture(scope="module", autouse=True)
def _threads():
    O.build()
    O.set_threads(min(8, O.max_threads()))


f32 = np.float32


def bump(x, y):
    """0.4 + 0.6 exp(-(a^2 + b^2)), a = (x - 3) / 1.2, b = (y - 1.3) / 0.9, in f32
    (tests_delta3d.rs:863-867)."""
    a, b = (f32(x) - f32(3.0)) / f32(1.2), (f32(y) - f32(1.3)) / f32(0.9)
    return f32(0.4) + f32(0.6) * scenes.expf(-(a * a + b * b))


def s232_bottom(shape, x):
    """The three bottoms of S232 (tests_delta3d.rs:852-860)."""
    d = (f32(x) - f32(3.0)) / f32(1.2)
    if shape == 0:
        return f32(0.5)
    hump = f32(0.4) + f32(0.6) * scenes.expf(-(d * d))
    if shape == 1:
        return hump
    return hump + f32(0.125) * (f32(1.0) + f32(np.tanh(f32(2.0) * (f32(x) - f32(6.0)))))


def bump_bottom(nx, ny, dx):
    dx = f32(dx)
    return np.array([bump((f32(i) + f32(0.5)) * dx, (f32(j) + f32(0.5)) * dx) for j in range(ny) for i in range(nx)],
                    np.float32)


def volume(nx, ny, nz, dx, bottom):
    return O.OracleVolume(nx, ny, nz, dx, 1025.0, 9.81, bottom=bottom)


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def all_zero_bits(v):
    return all(np.all(bits(x) == 0) for x in v.velocity())


NX, NY, NZ, DX = 24, 12, 10, 0.25


def test_a_lake_at_rest_on_a_cut_bottom_stays_exactly_at_rest():
    """tests_delta3d.rs:928-943: 100 linear steps, velocities and surface to the bit."""
    v = volume(NX, NY, NZ, DX, bump_bottom(NX, NY, DX))
    rest = bits(v.surface()[0]).copy()
    for _ in range(100):
        assert not v.step_surface_linear(2000, 2000)["degraded"]
    assert all_zero_bits(v)
    assert np.array_equal(bits(v.surface()[0]), rest)


def test_a_step_on_a_cut_bottom_leaves_an_open_divergence_free_field():
    """tests_delta3d.rs:971-990: one linear step from z0 + 0.01 sin(0.8 x) cos(1.1 y)."""
    v = volume(NX, NY, NZ, DX, bump_bottom(NX, NY, DX))
    z0, dx = f32(NZ) * f32(DX), f32(DX)
    eta = np.array([z0 + f32(0.01) * scenes.sinf((f32(i) + f32(0.5)) * dx * f32(0.8))
                    * f32(np.cos(np.float64((f32(j) + f32(0.5)) * dx * f32(1.1))))
                    for j in range(NY) for i in range(NX)], np.float32)
    v.set_surface(eta)
    r = v.step_surface_linear(2000, 4000)
    assert not r["degraded"] and r["divergence"] <= TOL, r
    _, ou, ov, ow, _ = v.geometry()
    for a, x in zip((ou, ov, ow), v.velocity()):
        assert np.all(bits(x[a == 0]) == 0)
    assert np.any(v.velocity()[1] != 0)


def test_jacobi_on_the_cut_path_keeps_the_solution_and_cuts_the_iterations():
    """tests_delta3d.rs:1006-1040: 64 x 32 x 32 cells of 0.125 m on the bump, one linear step from
    z0 + 0.01 sin(2 pi x / 8): with Jacobi, fewer than half the iterations, the flux through the
    middle section within 1e-5 relative, the divergence within the tolerance."""
    nx, ny, nz, dx = 64, 32, 32, 0.125
    out = []
    for jacobi in (False, True):
        v = volume(nx, ny, nz, dx, bump_bottom(nx, ny, dx))
        v.set_precondition_cut(jacobi)
        z0 = f32(nz) * f32(dx)
        row = np.array([z0 + f32(0.01) * scenes.sinf(f32(2 * np.pi) * (f32(i) + f32(0.5)) * f32(dx) / f32(8.0))
                        for i in range(nx)], np.float32)
        v.set_surface(np.tile(row, ny))
        r = v.step_surface_linear(2000, 20_000)
        ou = v.geometry()[1].reshape(nz, ny, nx + 1)
        u = v.velocity()[0].reshape(nz, ny, nx + 1)
        q = float(np.sum(ou[:, :, nx // 2].astype(np.float64) * u[:, :, nx // 2].astype(np.float64))
                  * np.float64(f32(dx) * f32(dx)))
        out.append((r["iterations"], q, r["divergence"]))
    (it_plain, q_plain, _), (it_jacobi, q_jacobi, d_jacobi) = out
    assert 2 * it_jacobi < it_plain, (it_jacobi, it_plain)
    assert abs((q_jacobi - q_plain) / q_plain) < 1e-5, (q_jacobi, q_plain)
    assert d_jacobi <= TOL


def test_a_lake_at_rest_on_a_cut_bottom_stays_at_rest_in_mobile_mode():
    """tests_delta3d.rs:1086-1100: 100 mobile steps at 2 m, velocities and surface to the bit."""
    v = volume(NX, NY, NZ, DX, bump_bottom(NX, NY, DX))
    v.set_free_surface(np.full(NX * NY, 2.0, np.float32), 2.0)
    for step in range(100):
        v.step_surface_mobile(2000, 4000)
        assert all_zero_bits(v), step
        assert np.all(bits(v.surface()[0]) == bits(f32(2.0))), step


def mobile_surface(nx, ny, rest, a):
    """rest + a cos(pi (i + 1/2) / nx) on every row, in f64 rounded to f32 (tests_delta3d.rs:1045-1049)."""
    i = np.arange(nx, dtype=np.float64)
    row = (np.float64(f32(rest)) + np.float64(f32(a)) * np.cos(np.pi * (i + 0.5) / nx)).astype(np.float32)
    return np.tile(row, ny)


def test_a_bottom_without_y_keeps_the_mobile_slices_identical():
    """tests_delta3d.rs:1103-1134: the hump of S232 at ny = 4: the four slices agree to the bit after
    100 mobile steps, the transverse flow stays at roundoff (<= 1e-6 of u), and the surface is
    within 1e-5 of the amplitude of the ny = 1 one."""
    n, nz = 32, 16
    dx = f32(8.0) / f32(n)
    rest, a = 2.5, 0.1
    surfaces = []
    for ny in (1, 4):
        row = np.array([s232_bottom(1, (f32(i) + f32(0.5)) * dx) for i in range(n)], np.float32)
        v = volume(n, ny, nz, dx, np.tile(row, ny))
        v.set_free_surface(mobile_surface(n, ny, rest, a), rest)
        for _ in range(100):
            v.step_surface_mobile(1000, 4000)
        s = v.surface()[0].reshape(ny, n)
        for j in range(1, ny):
            assert np.array_equal(bits(s[j]), bits(s[0])), j
        u, vv, _ = v.velocity()
        assert np.max(np.abs(vv)) <= 1e-6 * np.max(np.abs(u))
        surfaces.append(s[0].copy())
    worst = float(np.max(np.abs((surfaces[1] - f32(rest)) - (surfaces[0] - f32(rest)))))
    assert worst / a <= 1e-5, worst


def test_a_surface_too_close_to_the_cut_bottom_is_refused():
    """tests_delta3d.rs:1137-1158: 1.4 m leaves less than two cells above the bump's top (about 1 m):
    refused (Domain), every published field keeps its bits; over a flat 0.3 m bottom it steps."""
    v = volume(NX, NY, NZ, DX, bump_bottom(NX, NY, DX))
    v.set_free_surface(np.full(NX * NY, 1.4, np.float32), 1.4)
    state = lambda: [bits(x).copy() for x in (v.surface()[0], *v.velocity(), v.pressure())]  # noqa: E731
    before = state()
    with pytest.raises(O.OracleError) as e:
        v.step_surface_mobile(2000, 4000)
    assert e.value.kind == "Domain"
    assert all(np.array_equal(a, b) for a, b in zip(before, state()))
    w = volume(NX, NY, NZ, DX, np.full(NX * NY, 0.3, np.float32))
    w.set_free_surface(np.full(NX * NY, 1.4, np.float32), 1.4)
    w.step_surface_mobile(2000, 4000)


@pytest.mark.parametrize("bottom,kind", [(np.full(23, 0.3, np.float32), "Shape"),
                                         (np.full(24, -0.1, np.float32), "NotFinite"),
                                         (np.full(24, 2.5, np.float32), "NotFinite")])
def test_a_bottom_it_cannot_hold_is_refused(bottom, kind):
    """tests_delta3d.rs:871-891: 6 x 4 x 5 cells of 0.5 m (z0 = 2.5 m): a bottom of the wrong size
    (Shape), below 0 or at the lid (NotFinite, the reference's code for a height outside [0, z0[)."""
    with pytest.raises(O.OracleError) as e:
        volume(6, 4, 5, 0.5, bottom)
    assert e.value.kind == kind
