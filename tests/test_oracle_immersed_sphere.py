"""An immersed sphere, at rest and moving, in the oracle (CPU only).

The reference's own criteria for a solid inside the volume (tests_delta3d.rs:1161-1328, S329 and
S330): a lake at rest around the sphere stays at rest to the bit in the linear and the mobile step,
a wave passes with its divergence under the tolerance and no velocity on a closed face, a surface
too close to the sphere is refused with the state kept, setting the same solid at rest changes no
bit, a sphere crossing cells keeps its faces sound, and the water displaced follows the solid's
discrete volume to 1e-9 m^3.
"""
import numpy as np
import pytest

from fluidisim_b200 import scenes
from oracle import oracle as O

N = 24
DX = np.float32(1.2) / np.float32(N)  # 1.2 / n in f32, as the reference's volume_sphere
Z0 = np.float32(N) * DX               # Domain3::z0
TOL = 1e-5                            # PROJECTION_DIVERGENCE_TOLERANCE (delta_projection.rs:192)


@pytest.fixture(scope="module", autouse=True)
def _threads():
    O.build()
    O.set_threads(min(8, O.max_threads()))


def sphere_nodes(cx=0.6):
    """The sphere of tests_delta3d.rs:1161-1170, 1233-1245 (centre (cx, 0.6, 0.55), radius 0.3)."""
    return scenes.spheres_sdf(N, N, N, DX, [(cx, 0.6, 0.55)], [0.3])


def volume():
    return O.OracleVolume(N, N, N, DX, 1025.0, 9.81, bottom=np.zeros(N * N, np.float32), solid=sphere_nodes())


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def wave(mean):
    """mean + 0.01 cos(2 pi (i + 1/2) / n) along x, in f32."""
    i = np.arange(N, dtype=np.float32)
    row = np.float32(mean) + np.float32(0.01) * np.cos(np.float32(2 * np.pi) * (i + np.float32(0.5)) / np.float32(N))
    return np.tile(row.astype(np.float32), N)


def closed_faces_carry_nothing(v):
    _, ou, ov, ow, _ = v.geometry()
    for a, x in zip((ou, ov, ow), v.velocity()):
        assert np.all(np.isfinite(x))
        assert np.all(x[a == 0] == 0)


def test_a_lake_at_rest_around_the_sphere_stays_at_rest_to_the_bit():
    """tests_delta3d.rs:1182-1200: 100 linear steps under the lid, 100 mobile steps at 1.05 m."""
    lin = volume()
    lin.set_surface(np.full(N * N, Z0, np.float32))
    for step in range(100):
        lin.step_surface_linear(2000, 4000)
        assert all(np.all(bits(x) == 0) for x in lin.velocity()), step
    mob = volume()
    mob.set_free_surface(np.full(N * N, 1.05, np.float32), 1.05)
    for step in range(100):
        mob.step_surface_mobile(2000, 4000)
        assert all(np.all(bits(x) == 0) for x in mob.velocity()), step
        assert np.all(bits(mob.surface()[0]) == bits(np.float32(1.05))), step


def test_a_wave_passes_over_the_sphere():
    """tests_delta3d.rs:1201-1213: 20 mobile steps, plain divergence under the tolerance, no velocity
    on a closed face, and the wave moves the water."""
    v = volume()
    v.set_free_surface(wave(1.05), 1.05)
    for _ in range(20):
        r = v.step_surface_mobile(2000, 4000)
        assert r["divergence_plain"] <= TOL, r
    closed_faces_carry_nothing(v)
    assert np.any(v.velocity()[0] != 0)


def test_a_surface_too_close_to_the_sphere_is_refused():
    """tests_delta3d.rs:1217-1227: the sphere's top is at 0.85 m; a surface at 0.95 m is refused
    (Domain) and the state keeps its bits."""
    v = volume()
    v.set_free_surface(np.full(N * N, 0.95, np.float32), 0.95)
    before = [bits(v.surface()[0]).copy(), bits(v.velocity()[0]).copy()]
    with pytest.raises(O.OracleError) as e:
        v.step_surface_mobile(2000, 4000)
    assert e.value.kind == "Domain"
    after = [bits(v.surface()[0]), bits(v.velocity()[0])]
    assert all(np.array_equal(a, b) for a, b in zip(before, after))


def test_setting_the_same_solid_at_rest_changes_nothing():
    """tests_delta3d.rs:1248-1270: 50 linear steps under a wave, one volume re-setting its sphere at
    rest before each step: the same iterations and the same bits."""
    a, b = volume(), volume()
    eta = wave(Z0)
    a.set_surface(eta)
    b.set_surface(eta)
    s = sphere_nodes(0.6)
    for step in range(50):
        b.set_solid_rigid(s, (0.0, 0.0, 0.0))
        ra, rb = a.step_surface_linear(2000, 4000), b.step_surface_linear(2000, 4000)
        assert ra["iterations"] == rb["iterations"], step
        assert np.array_equal(bits(a.surface()[0]), bits(b.surface()[0])), step
        for x, y in zip(a.velocity(), b.velocity()):
            assert np.array_equal(bits(x), bits(y)), step


def test_a_moving_sphere_keeps_the_faces_sound():
    """tests_delta3d.rs:1273-1305: the sphere crosses two cells at 1 m/s over 50 linear steps; faces
    open, the divergence stays under the tolerance, no closed face carries a velocity, nothing is
    non-finite; a solid reaching the lid layer is refused and writes nothing."""
    v = volume()
    v.set_surface(np.full(N * N, Z0, np.float32))
    born = 0
    for step in range(1, 51):
        before = v.geometry()[1].copy()
        v.set_solid_rigid(sphere_nodes(0.6 + 1.0 * 0.002 * step), (1.0, 0.0, 0.0))
        after = v.geometry()[1]
        born += int(np.count_nonzero((after > 0) & (before == 0)))
        r = v.step_surface_linear(2000, 4000)
        assert r["divergence"] <= TOL, (step, r)
        closed_faces_carry_nothing(v)
    assert born > 0
    top = sphere_nodes(0.6).reshape(N + 1, (N + 1) * (N + 1)).copy()
    top[N - 1:] = -1.0
    keep = bits(v.geometry()[1]).copy()
    with pytest.raises(O.OracleError) as e:
        v.set_solid_rigid(top.ravel(), (0.0, 0.0, 0.0))
    assert e.value.kind == "Domain"
    assert np.array_equal(keep, bits(v.geometry()[1]))


def solid_volume(v):
    """The solid's discrete volume summed over the columns, each column as delta3d.rs:86-99 forms
    it: f32 of the f64 sum over k of (base - frac), times dx^3 (base = 1 above a flat bottom)."""
    frac = v.geometry()[0].reshape(N, N * N)
    col = (np.float32(1.0) - frac).astype(np.float64).sum(axis=0) * (np.float64(DX) ** 3)
    return float(col.astype(np.float32).astype(np.float64).sum())


def test_a_moving_sphere_displaces_exactly_its_discrete_volume():
    """tests_delta3d.rs:1308-1328: step after step, the water volume sum((eta - roundoff - z0) dx^2)
    follows the change of the solid's discrete volume to 1e-9 m^3."""
    v = volume()
    v.set_surface(np.full(N * N, Z0, np.float32))
    v0 = solid_volume(v)
    d2 = np.float64(DX) ** 2
    worst = 0.0
    for step in range(1, 51):
        v.set_solid_rigid(sphere_nodes(0.6 + 0.002 * step), (1.0, 0.0, 0.0))
        v.step_surface_linear(2000, 4000)
        eta, roundoff = v.surface()
        water = float(np.sum((eta.astype(np.float64) - roundoff.astype(np.float64) - np.float64(Z0)) * d2))
        worst = max(worst, abs(water - (solid_volume(v) - v0)))
    assert worst <= 1e-9, worst


def spin_residual(n, nodes, z0):
    """One linear step under the lid after setting the solid spinning at 2 rad/s about z through
    (0.6, 0.6, 0.55); the largest velocity it leaves."""
    dx = np.float32(1.2) / np.float32(n)
    v = O.OracleVolume(n, n, n, dx, 1025.0, 9.81, bottom=np.zeros(n * n, np.float32), solid=nodes)
    v.set_surface(np.full(n * n, z0, np.float32))
    v.set_solid_rigid(nodes, (0.0, 0.0, 0.0), (0.0, 0.0, 2.0), (0.6, 0.6, 0.55))
    v.step_surface_linear(2000, 4000)
    return max(float(np.max(np.abs(x))) for x in v.velocity())


def test_a_spinning_sphere_pushes_no_water_a_spinning_box_does():
    """tests_delta3d.rs:1354-1384: a sphere spinning on itself leaves at most 1% of its rim speed
    (Omega R = 0.6 m/s) at 12 cells per radius, less than at 6 (published: 1.08% then 0.73%); a box
    of half side 0.2 m spinning the same way pushes at least 10% of 2 x 0.2 m/s."""
    def sphere(n):
        d = np.float32(1.2) / np.float32(n)
        return spin_residual(n, scenes.spheres_sdf(n, n, n, d, [(0.6, 0.6, 0.55)], [0.3]), np.float32(n) * d)
    coarse, fine = sphere(24), sphere(48)
    assert fine <= 0.01 * 0.6, fine
    assert fine < coarse
    assert round(100 * coarse / 0.6, 2) == 1.08 and round(100 * fine / 0.6, 2) == 0.73, (coarse, fine)
    box = scenes.boxes_sdf(N, N, N, DX, [(0.6, 0.6, 0.55)], [(0.2, 0.2, 0.2)])
    assert spin_residual(N, box, np.float32(1.2)) >= 0.1 * 2.0 * 0.2
