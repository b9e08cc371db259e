"""The oracle's linear (fixed-lid) path against the reference's own known answers (CPU only).

Pins: the iteration counts and open fluxes of the cut-bottom bench (FACES-COUPEES-3D-S324.md,
tables of sections 3 and 6), the oblique standing wave's errors and mean iteration count
(DELTA3D-LINEAIRE-S295.md section 2), and the properties of tests_delta3d.rs:150-277.
"""
import math

import numpy as np
import pytest

import golden_cases as G
from fluidisim_b200 import scenes
from oracle import oracle as O


@pytest.fixture(scope="module", autouse=True)
def _threads():
    O.build()
    O.set_threads(min(8, O.max_threads()))


def s324_step(nx, bump, jacobi):
    s = scenes.s324_case(nx, bump)
    v = O.OracleVolume(s["nx"], s["ny"], s["nz"], s["dx"], s["rho"], s["g"], bottom=s["bottom"])
    v.set_precondition_cut(jacobi)
    v.set_surface(s["eta"])
    r = v.step_surface_linear(s["dt_us"], 20000)
    q = scenes.open_flux_x(v.geometry()[1], v.velocity()[0], s["nx"], s["ny"], s["nz"], s["dx"])
    return r, q


_KA = G.known_answers()


# FACES-COUPEES-3D-S324.md:136 (S326, Jacobi) and :85 (S324, no preconditioner)
@pytest.mark.parametrize("nx,jacobi,iters,flux,digits", [
    (r["nx"], r["jacobi"], r["iterations"], r["flux"], r["digits"]) for r in _KA["s324_cut_bump_linear"]["rows"]])
def test_cut_bump_step_matches_the_published_bench(nx, jacobi, iters, flux, digits):
    r, q = s324_step(nx, True, jacobi)
    assert r["iterations"] == iters
    assert round(q, digits + 3) == pytest.approx(flux, rel=0.5 * 10 ** (1 - digits))
    assert not r["degraded"] and r["divergence"] <= 1e-5


# FACES-COUPEES-3D-S324.md:85: the smooth bottom without y, no preconditioner, 95 / 179 iterations;
# its flux per unit width 2.2524960e-4 / 2.2584836e-4 m^2/s (width 4 m).
@pytest.mark.parametrize("nx,iters,flux_per_width", [
    (r["nx"], r["iterations"], r["flux_per_width"]) for r in _KA["s324_smooth_bottom_linear"]["rows"]])
def test_smooth_bottom_witness_matches_the_published_bench(nx, iters, flux_per_width):
    r, q = s324_step(nx, False, False)
    assert r["iterations"] == iters
    assert q / 4.0 == pytest.approx(flux_per_width, rel=5e-8)


def test_oblique_standing_wave_follows_its_scheme():
    """DELTA3D-LINEAIRE-S295.md:35-36: n = 16, 2 ms, g = 9.81: 2.3165 % against the continuous
    dispersion, 0.0046 % against the scheme's, 17.9 iterations per step (500 steps)."""
    w = scenes.oblique_wave(16)
    v = O.OracleVolume(w["nx"], w["ny"], w["nz"], w["dx"], w["rho"], w["g"])
    v.set_surface(w["eta"])
    us = 2000
    big, beta = scenes.scheme_frequency(w["kx"], w["ky"], 8.0 / 16, w["nz"], 9.81, us * 1e-6)
    k = math.hypot(w["kx"], w["ky"])
    omega = math.sqrt(9.81 * k * math.tanh(k * w["h"]))
    e_cont = e_scheme = 0.0
    its = 0
    steps = 1_000_000 // us
    for step in range(1, steps + 1):
        r = v.step_surface_linear(us, 4000)
        its += r["iterations"]
        t = step * us * 1e-6
        hn = v.surface()[0].astype(np.float64) - w["h"]
        e_cont = max(e_cont, float(np.max(np.abs(hn - w["a"] * w["mode"] * math.cos(omega * t)))) / w["a"])
        ph = big * t
        e_scheme = max(e_scheme, float(np.max(np.abs(hn - w["a"] * w["mode"] * (math.cos(ph) + beta * math.sin(ph)))))
                       / w["a"])
    want = _KA["s295_oblique_standing_wave"]
    assert round(100 * e_cont, 4) == want["error_vs_continuous_percent"]
    assert round(100 * e_scheme, 4) == want["error_vs_scheme_percent"]
    assert round(its / steps, 1) == want["mean_iterations"]


@pytest.mark.parametrize("shape", [(8, 6, 5), (12, 1, 7), (5, 9, 4)])
def test_projection_leaves_a_divergence_free_field(shape):
    """tests_delta3d.rs:150-178."""
    nx, ny, nz = shape
    v = O.OracleVolume(nx, ny, nz, 0.25, 1025.0, 9.81)
    nu, nv, nw = (nx + 1) * ny * nz, nx * (ny + 1) * nz, nx * ny * (nz + 1)
    v.set_velocity(scenes.noise(nu, 1), scenes.noise(nv, 2), scenes.noise(nw, 3))
    r = v.project_linear(-1025.0 / 0.002, 0.002 / 1025.0, 4000)
    assert not r["degraded"] and r["iterations"] > 0 and r["divergence"] <= 1e-5
    u, vv, w = v.velocity()
    ui = u.reshape(nz, ny, nx + 1)
    vi = vv.reshape(nz, ny + 1, nx)
    assert np.all(ui[:, :, 0] == 0) and np.all(ui[:, :, nx] == 0)
    assert np.all(vi[:, 0, :] == 0) and np.all(vi[:, ny, :] == 0)
    # the published divergence is that of the published field (tests_delta3d.rs:160-165)
    wi = w.reshape(nz + 1, ny, nx)
    fl, fr, ff, fk, fb, ft = ui[:, :, :-1], ui[:, :, 1:], vi[:, :-1, :], vi[:, 1:, :], wi[:-1], wi[1:]
    dv = ((((fr - fl) + ft) - fb) + (fk - ff)) / np.float32(0.25)  # divergence's f32 order, delta3d.rs:759
    umax = max(np.abs(u).max(), np.abs(vv).max(), np.abs(w).max())
    d = float(np.abs(dv).max()) * 0.25 / float(umax)
    assert abs(d - r["divergence"]) <= 1e-5 * d


def test_rest_projects_to_exact_zero():
    """tests_delta3d.rs:180-186."""
    v = O.OracleVolume(6, 4, 5, 0.5, 1025.0, 9.81)
    r = v.project_linear(-1025.0 / 0.002, 0.002 / 1025.0, 100)
    assert (r["iterations"], r["degraded"], r["residual"], r["divergence"]) == (0, False, 0.0, 0.0)
    assert not np.any(v.pressure()) and not any(np.any(x) for x in v.velocity())


def test_rest_is_exact_and_guards_refuse():
    """tests_delta3d.rs:248-260."""
    v = O.OracleVolume(8, 6, 4, 1.0, 1025.0, 9.81)
    for _ in range(100):
        r = v.step_surface_linear(2000, 100)
        assert r["iterations"] == 0
    assert np.all(v.surface()[0] == 4.0)
    with pytest.raises(O.OracleError) as e:
        v.step_surface_linear(0, 100)
    assert e.value.kind == "NotFinite"
    with pytest.raises(O.OracleError) as e:
        v.step_surface_linear(500_000, 100)
    assert e.value.kind == "Domain"
    neg = O.OracleVolume(8, 6, 4, 1.0, 1025.0, -1.0)
    with pytest.raises(O.OracleError) as e:
        neg.step_surface_linear(2000, 100)
    assert e.value.kind == "Domain"


def test_refusal_restores_every_published_field():
    """tests_delta3d.rs:262-277."""
    v = O.OracleVolume(12, 8, 6, 0.5, 1025.0, 9.81)
    c = np.arange(12 * 8)
    eta = (3.0 + 0.02 * np.sin((c % 12).astype(np.float32) * np.float32(0.7))
           * np.cos((c // 12).astype(np.float32) * np.float32(0.4))).astype(np.float32)
    v.set_surface(eta)
    for _ in range(5):
        v.step_surface_linear(2000, 2000)
    before = [x.copy() for x in (*v.velocity(), v.pressure(), *v.surface())]
    with pytest.raises(O.OracleError) as e:
        v.step_surface_linear(2000, 1)
    assert e.value.kind == "Convergence"
    after = [x.copy() for x in (*v.velocity(), v.pressure(), *v.surface())]
    for a, b in zip(before, after):
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    v.step_surface_linear(2000, 2000)


def test_a_surface_independent_of_y_stays_independent_of_y():
    """tests_delta3d.rs:223-244 (60 steps instead of 200 to keep the CPU suite short)."""
    nx, ny, nz = 16, 5, 8
    v = O.OracleVolume(nx, ny, nz, 0.5, 1025.0, 9.81)
    line = np.array([4.0 + 0.01 * math.cos(math.pi * (i + 0.5) / nx) for i in range(nx)], dtype=np.float32)
    v.set_surface(np.tile(line, ny))
    for _ in range(60):
        v.step_surface_linear(2000, 2000)
    eta = v.surface()[0].reshape(ny, nx)
    u, vv, w = v.velocity()
    assert np.all(eta == eta[0:1])
    assert np.all(u.reshape(nz, ny, nx + 1) == u.reshape(nz, ny, nx + 1)[:, 0:1])
    assert np.all(w.reshape(nz + 1, ny, nx) == w.reshape(nz + 1, ny, nx)[:, 0:1])
    assert not np.any(vv)
    assert eta[0, 0] < 4.01
