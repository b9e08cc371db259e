"""The oracle against the reference's own known answers (no GPU).

Pins (paths relative to the reference project):
  * docs/validation/MULTIGRILLE-3D-S385.md:57-60: iterations of the first mobile step from rest on
    the S385 bench (code/water-core/examples/delta3d_multigrille.rs): multigrid 9/10/11 on the flat
    and the bumped bottom, Jacobi 102/191/365 (flat) and 117/219/444 (bump);
  * code/water-core/src/tests_delta3d.rs: :352 symmetric ghost rows, :389 conservative mobile
    projection, :1814 hierarchy counts, :1840 symmetric positive V-cycle, :1875 same surface with
    fewer iterations, :180 rest projects to exact zero.
"""
import numpy as np
import pytest

import golden_cases as G
from fluidisim_b200 import scenes
from oracle import oracle as O

# The published counts, from the golden fixture that cites them.
_KA = G.known_answers()
PUBLISHED_MG = {(bump, int(n)): c for bump in (False, True)
                for n, c in _KA["s385_multigrid_iterations"]["bump" if bump else "flat"].items()}
PUBLISHED_JACOBI = {(bump, int(n)): c for bump in (False, True)
                    for n, c in _KA["s385_jacobi_iterations"]["bump" if bump else "flat"].items()}


def s385_volume(nx, bump, mg, real="f32"):
    s = scenes.s385_case(nx, bump)
    v = O.OracleVolume(s["nx"], s["ny"], s["nz"], s["dx"], s["rho"], s["g"], bottom=s["bottom"], real=real)
    if mg:
        v.enable_multigrid()
    v.set_free_surface(s["eta"], s["rest"])
    return v, s


@pytest.mark.parametrize("bump", [False, True])
@pytest.mark.parametrize("nx", [32, 64, 128])
def test_s385_multigrid_iterations_match_the_published_counts(nx, bump):
    O.set_threads(O.max_threads())
    v, s = s385_volume(nx, bump, True)
    r = v.step_surface_mobile(s["dt_us"], 20000)
    assert not r["degraded"]
    assert r["iterations"] == PUBLISHED_MG[(bump, nx)]


@pytest.mark.parametrize("bump", [False, True])
@pytest.mark.parametrize("nx", [32, 64, pytest.param(128, marks=pytest.mark.slow)])
def test_s385_jacobi_iterations_match_the_published_counts(nx, bump):
    O.set_threads(O.max_threads())
    v, s = s385_volume(nx, bump, False)
    r = v.step_surface_mobile(s["dt_us"], 20000)
    assert not r["degraded"]
    assert r["iterations"] == PUBLISHED_JACOBI[(bump, nx)]


def test_thread_count_changes_no_bit():
    outs = []
    for t in (1, 4):
        O.set_threads(t)
        v, s = s385_volume(32, True, True)
        r = v.step_surface_mobile(s["dt_us"], 20000)
        outs.append((r["iterations"], v.pressure().tobytes(), b"".join(x.tobytes() for x in v.velocity())))
    assert outs[0] == outs[1]


def test_hierarchy_counts():
    assert O.level_count3(32, 16, 24) == 3
    assert O.level_count3(7, 16, 24) == 0
    assert O.level_count3(120, 112, 28) == 2
    # floats held: 2 fine buffers + per level 5 cell fields + 3 face families
    for dims in [(32, 16, 24), (16, 8, 12), (7, 5, 3)]:
        nx, ny, nz = dims
        total = 2 * nx * ny * nz
        while nx % 2 == 0 and ny % 2 == 0 and nz % 2 == 0 and min(nx, ny, nz) >= 4:
            nx, ny, nz = nx // 2, ny // 2, nz // 2
            total += 5 * nx * ny * nz + (nx + 1) * ny * nz + nx * (ny + 1) * nz + nx * ny * (nz + 1)
        assert O.hierarchy_floats3(*dims) == total


def _dot(a, b):
    return float(np.dot(a.astype(np.float64), b.astype(np.float64)))


@pytest.mark.parametrize("ny", [1, 4])
def test_mobile_operator_is_symmetric_and_positive(ny):
    v = O.OracleVolume(7, ny, 8, 0.25)
    eta = np.array([1.0 + 0.21 * np.sin(np.float32(c) * np.float32(1.7)) for c in range(7 * ny)], np.float32)
    v.set_free_surface(eta, 1.0)
    x, y = scenes.noise(v.cells, 4), scenes.noise(v.cells, 8)
    _, prec = v.assemble_pressure_problem_for_trials(np.zeros(v.cells, np.float32), 1.0)
    wet = v.apply_pressure_operator_for_trials(np.ones(v.cells, np.float32)) != 0
    # dry cells are zero in both vectors (tests_delta3d.rs:356-358 masks with wet3)
    kk = np.arange(v.cells) // (7 * ny)
    col = np.arange(v.cells) % (7 * ny)
    wet = (kk + 0.5) * np.float32(0.25) < eta[col]
    x[~wet] = 0
    y[~wet] = 0
    ax, ay = v.apply_pressure_operator_for_trials(x), v.apply_pressure_operator_for_trials(y)
    assert abs(_dot(x, ay) - _dot(y, ax)) < 1e-5 * np.sqrt(_dot(x, x) * _dot(ay, ay))
    assert _dot(x, ax) > 0


@pytest.mark.parametrize("bump", [False, True])
def test_vcycle_is_symmetric_and_positive(bump):
    v, s = s385_volume(32, bump, True)
    _, prec = v.assemble_pressure_problem_for_trials(np.zeros(v.cells, np.float32), 1.0)
    vecs = [scenes.noise(v.cells, 11), scenes.noise(v.cells, 13)]
    for x in vecs:
        x[prec == 0] = 0
    imgs = [v.vcycle_for_tests(x) for x in vecs]
    ab, ba = _dot(imgs[0], vecs[1]), _dot(imgs[1], vecs[0])
    assert abs(ab - ba) <= 1e-5 * np.sqrt(_dot(imgs[0], imgs[0]) * _dot(vecs[1], vecs[1]))
    for z, x in zip(imgs, vecs):
        assert _dot(z, x) > 0
        assert np.all(z[prec == 0] == 0)


@pytest.mark.parametrize("ny", [1, 4])
def test_mobile_projection_is_conservative(ny):
    v = O.OracleVolume(9, ny, 9, 0.25)
    eta = np.array([1.25 + 0.2 * np.sin(np.float32(c) * np.float32(1.7)) for c in range(9 * ny)], np.float32)
    v.set_free_surface(eta, 1.25)
    v.set_velocity(scenes.noise(v.nu, 1), scenes.noise(v.nv, 2), scenes.noise(v.nw, 3))
    r = v.project_mobile(-1025.0 / 0.002, 0.002 / 1025.0, 4000)
    assert not r["degraded"]
    assert r["divergence_plain"] <= 1e-5


def test_rest_projects_to_exact_zero():
    v = O.OracleVolume(6, 4, 5, 0.5)
    v.set_free_surface(np.full(24, 2.0, np.float32), 2.0)
    r = v.project_mobile(-1025.0 / 0.002, 0.002 / 1025.0, 100)
    assert (r["iterations"], r["degraded"], r["residual"], r["divergence"]) == (0, False, 0.0, 0.0)
    assert not np.any(v.pressure().view(np.uint32))


@pytest.mark.parametrize("bump", [False, True])
def test_multigrid_reaches_the_same_surface_with_fewer_iterations(bump):
    O.set_threads(O.max_threads())
    a, s = s385_volume(32, bump, False)
    b, _ = s385_volume(32, bump, True)
    ia = ib = 0
    for _ in range(20):
        ra = a.step_surface_mobile(2000, 20000)
        rb = b.step_surface_mobile(2000, 20000)
        assert not ra["degraded"] and not rb["degraded"]
        ia += ra["iterations"]
        ib += rb["iterations"]
    worst = np.max(np.abs(a.surface()[0] - b.surface()[0]))
    assert worst <= 1e-6
    assert 2 * ib < ia


def test_refusals():
    with pytest.raises(O.OracleError) as e:
        O.OracleVolume(0, 2, 2, 1.0)
    assert e.value.kind == "Domain"
    with pytest.raises(O.OracleError) as e:
        O.OracleVolume(2, 2, 2, 1.0, rho=0.0)
    assert e.value.kind == "NotFinite"
    v = O.OracleVolume(4, 4, 4, 0.25)
    with pytest.raises(O.OracleError) as e:
        v.set_velocity(np.zeros(3), np.zeros(v.nv), np.zeros(v.nw))
    assert e.value.kind == "Shape"
    u = np.zeros(v.nu, np.float32)
    u[3] = np.nan
    with pytest.raises(O.OracleError) as e:
        v.set_velocity(u, np.zeros(v.nv), np.zeros(v.nw))
    assert e.value.kind == "NotFinite"
