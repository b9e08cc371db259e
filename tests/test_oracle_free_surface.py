"""The mobile free surface's own criteria in the oracle (CPU only).

tests_delta3d.rs:77-93 and 453-518 (S295, S296): configuration refuses the domains and constants
it cannot hold; the mobile step is symmetric under the exchange of x and y and keeps a lake at rest
exactly at rest; a refused step (iteration cap, surface out of range, zero duration, the guard after
transport) publishes nothing; the mobile operator's matrix is symmetric to the bit and the Jacobi
preconditioner is the inverse of its diagonal, to the bit.
"""
import numpy as np
import pytest

from fluidisim_b200 import scenes
from oracle import oracle as O

f32 = np.float32


@pytest.fixture(scope="module", autouse=True)
def _threads():
    O.build()
    O.set_threads(min(8, O.max_threads()))


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def state(v):
    e, r = v.surface()
    return [bits(x).copy() for x in (*v.velocity(), v.pressure(), e, r)]


def same(a, b):
    return all(np.array_equal(x, y) for x, y in zip(a, b))


@pytest.mark.parametrize("dims", [(0, 2, 2, 1.0), (2, 0, 2, 1.0), (2, 2, 0, 1.0), (2, 2, 2, 0.0),
                                  (2, 2, 2, float("nan")), (2 ** 64 - 1, 2, 2, 1.0)])
def test_configuration_refuses_a_domain_it_cannot_hold(dims):
    """tests_delta3d.rs:77-84."""
    with pytest.raises(O.OracleError) as e:
        O.OracleVolume(*dims, 1025.0, 9.81)
    assert e.value.kind == "Domain"


@pytest.mark.parametrize("rho,g", [(0.0, 9.81), (1025.0, float("inf"))])
def test_configuration_refuses_non_finite_constants(rho, g):
    """tests_delta3d.rs:86-87."""
    with pytest.raises(O.OracleError) as e:
        O.OracleVolume(2, 2, 2, 1.0, rho, g)
    assert e.value.kind == "NotFinite"


def test_the_mobile_step_is_symmetric_in_x_and_y_and_keeps_rest_exact():
    """tests_delta3d.rs:453-474: 12 x 7 against 7 x 12 with the transposed surface, 300 steps of
    1 ms, within 2e-6 m; then a lake at 2.013 m steps 50 times with no iteration, every field at
    its rest bits."""
    x = O.OracleVolume(12, 7, 12, 0.25, 1025.0, 9.81)
    y = O.OracleVolume(7, 12, 12, 0.25, 1025.0, 9.81)
    c = np.arange(84)
    eta = (f32(2.0) + f32(0.05) * np.cos(f32(np.pi) * (c % 12).astype(np.float32) / f32(12.0))).astype(np.float32)
    trans = eta.reshape(7, 12).T.ravel().copy()
    x.set_free_surface(eta, 2.0)
    y.set_free_surface(trans, 2.0)
    worst = 0.0
    for _ in range(300):
        x.step_surface_mobile(1000, 4000)
        y.step_surface_mobile(1000, 4000)
        ex, ey = x.surface()[0].reshape(7, 12), y.surface()[0].reshape(12, 7)
        worst = max(worst, float(np.max(np.abs(ex - ey.T))))
    assert worst < 2e-6, worst
    x.set_free_surface(np.full(84, 2.013, np.float32), 2.013)
    x.set_velocity(np.zeros(x.nu), np.zeros(x.nv), np.zeros(x.nw))
    for _ in range(50):
        assert x.step_surface_mobile(1000, 4000)["iterations"] == 0
        assert np.all(bits(x.surface()[0]) == bits(f32(2.013)))
        assert all(np.all(bits(a) == 0) for a in (*x.velocity(), x.pressure()))


def test_refused_mobile_steps_publish_nothing():
    """tests_delta3d.rs:477-504: the iteration cap (Convergence), a surface below or above what the
    column holds (Domain), a zero duration (NotFinite), and the guard after transport, reached by a
    crest within 1604 steps (Domain): each leaves every published field at its bits."""
    v = O.OracleVolume(16, 5, 12, 0.25, 1025.0, 9.81)
    eta = np.array([f32(2.0) + f32(0.1) * scenes.sinf(f32(c) * f32(0.7)) for c in range(80)], np.float32)
    v.set_free_surface(eta, 2.0)
    for _ in range(5):
        v.step_surface_mobile(1000, 4000)
    before = state(v)
    with pytest.raises(O.OracleError) as e:
        v.step_surface_mobile(1000, 0)
    assert e.value.kind == "Convergence"
    assert same(state(v), before)
    for height in (0.49, 2.76):
        v.set_free_surface(np.full(80, height, np.float32), 2.0)
        before = state(v)
        with pytest.raises(O.OracleError) as e:
            v.step_surface_mobile(1000, 4000)
        assert e.value.kind == "Domain", height
        assert same(state(v), before)
    with pytest.raises(O.OracleError) as e:
        v.step_surface_mobile(0, 4000)
    assert e.value.kind == "NotFinite"

    w = O.OracleVolume(16, 1, 18, 0.125, 1025.0, 9.81)
    crest = np.array([f32(2.0) + f32(0.125 * np.cos(np.pi * (i + 0.5) / 16.0)) for i in range(16)], np.float32)
    w.set_free_surface(crest, 2.0)
    refused = False
    for _ in range(1604):
        before = state(w)
        try:
            w.step_surface_mobile(1000, 4000)
        except O.OracleError as err:
            assert err.kind == "Domain"
            assert same(state(w), before)
            refused = True
            break
    assert refused


def test_the_mobile_matrix_is_symmetric_and_jacobi_is_its_inverse_diagonal():
    """tests_delta3d.rs:507-518: 4 x 3 x 7 cells under a bumpy surface; the operator's columns
    form a matrix symmetric to the bit, and prec = 1 / diagonal (0 where the diagonal is 0)."""
    v = O.OracleVolume(4, 3, 7, 0.25, 1025.0, 9.81)
    eta = np.array([f32(1.1) + f32(0.2) * scenes.sinf(f32(c) * f32(1.9)) for c in range(12)], np.float32)
    v.set_free_surface(eta, 1.1)
    n = v.cells
    _, prec = v.assemble_pressure_problem_for_trials(np.zeros(n, np.float32), 0.0)
    m = np.empty((n, n), np.float32)
    for c in range(n):
        e = np.zeros(n, np.float32)
        e[c] = 1.0
        m[c] = v.apply_pressure_operator_for_trials(e)
    assert np.array_equal(bits(m), bits(m.T))
    diag = np.diagonal(m)
    inverse = np.where(diag > 0, f32(1.0) / np.where(diag > 0, diag, f32(1.0)), f32(0.0)).astype(np.float32)
    assert np.array_equal(bits(prec), bits(inverse))
