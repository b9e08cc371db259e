"""Parity of the sm_100a linear (fixed-lid) path with the oracle, through the C ABI (needs a GPU).

Ordered f32 reductions: every published field bit-identical to the oracle's, step after step.
Default f64 reductions: the reference's acceptance and the oracle's pressure to 1e-5 relative.
"""
import math

import numpy as np
import pytest

from fluidisim_b200 import scenes
from fluidisim_b200.delta3d import REDUCE_F64, REDUCE_ORDERED_F32, Delta3dError, Volume3
from oracle import oracle as O

pytestmark = pytest.mark.gpu

P_TOL = 1e-5  # pressure L-inf difference, relative to L-inf of the oracle's pressure


def assert_bits(a, b, what):
    a = np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)
    b = np.ascontiguousarray(b, dtype=np.float32).view(np.uint32)
    bad = np.nonzero(a != b)[0]
    assert bad.size == 0, f"{what}: {bad.size} differ, first at {bad[:5]}"


def same_state(o, d, what):
    assert_bits(d.pressure(), o.pressure(), f"{what} p")
    for name, a, b in zip("uvw", d.velocity(), o.velocity()):
        assert_bits(a, b, f"{what} {name}")
    de, dr = d.surface_and_roundoff()
    oe, orr = o.surface()
    assert_bits(de, oe, f"{what} eta")
    assert_bits(dr, orr, f"{what} roundoff")


def pair(nx, ny, nz, dx, g=9.81, bottom=None, reduction=REDUCE_ORDERED_F32):
    o = O.OracleVolume(nx, ny, nz, dx, 1025.0, g, bottom=bottom)
    if bottom is not None:
        d = Volume3.configure_with_bottom(nx, ny, nz, dx, 1025.0, g, bottom)
    else:
        d = Volume3.configure(nx, ny, nz, dx, 1025.0, g)
    d.set_options(reduction=reduction)
    return o, d


@pytest.mark.parametrize("shape", [(8, 6, 5), (12, 1, 7), (5, 9, 4)])
def test_linear_projection_of_noise_is_bit_exact(shape):
    nx, ny, nz = shape
    o, d = pair(nx, ny, nz, 0.25)
    nu, nv, nw = (nx + 1) * ny * nz, nx * (ny + 1) * nz, nx * ny * (nz + 1)
    u, v, w = scenes.noise(nu, 1), scenes.noise(nv, 2), scenes.noise(nw, 3)
    for x in (o, d):
        x.set_velocity(u, v, w)
    ro = o.project_linear(-1025.0 / 0.002, 0.002 / 1025.0, 4000)
    rd = d.project(-1025.0 / 0.002, 0.002 / 1025.0, 4000)
    assert rd.iterations == ro["iterations"] and rd.degraded == ro["degraded"]
    assert rd.divergence == pytest.approx(ro["divergence"], rel=1e-12)
    same_state(o, d, f"{shape}")


@pytest.mark.parametrize("bump,jacobi", [(True, True), (True, False), (False, False)])
def test_cut_bottom_step_is_bit_exact(bump, jacobi):
    s = scenes.s324_case(32, bump)
    o, d = pair(s["nx"], s["ny"], s["nz"], s["dx"], bottom=s["bottom"])
    for x in (o, d):
        x.set_precondition_cut(jacobi)
        x.set_surface(s["eta"])
    for step in range(3):
        ro = o.step_surface_linear(s["dt_us"], 20000)
        rd = d.step_surface_linear(s["dt_us"], 20000)
        assert rd.iterations == ro["iterations"], step
        same_state(o, d, f"step {step}")


def test_first_cut_bump_step_matches_the_published_count():
    """FACES-COUPEES-3D-S324.md:136: 220 iterations and 9.169151446e-4 m^3/s at 64."""
    s = scenes.s324_case(64, True)
    d = Volume3.configure_with_bottom(s["nx"], s["ny"], s["nz"], s["dx"], 1025.0, 9.81, s["bottom"])
    d.set_options(reduction=REDUCE_ORDERED_F32)
    d.set_surface(s["eta"])
    r = d.step_surface_linear(s["dt_us"], 20000)
    assert r.iterations == 220
    q = scenes.open_flux_x(d.geometry()[1], d.velocity()[0], s["nx"], s["ny"], s["nz"], s["dx"])
    assert q == pytest.approx(9.169151446e-4, rel=1e-9)


def test_oblique_wave_steps_are_bit_exact():
    w = scenes.oblique_wave(16)
    o, d = pair(w["nx"], w["ny"], w["nz"], w["dx"], g=w["g"])
    for x in (o, d):
        x.set_surface(w["eta"])
    for step in range(40):
        ro = o.step_surface_linear(2000, 4000)
        rd = d.step_surface_linear(2000, 4000)
        assert rd.iterations == ro["iterations"], step
    same_state(o, d, "after 40 steps")


def test_refusal_restores_every_published_field():
    o, d = pair(12, 8, 6, 0.5)
    c = np.arange(12 * 8)
    eta = (3.0 + 0.02 * np.sin((c % 12).astype(np.float32) * np.float32(0.7))
           * np.cos((c // 12).astype(np.float32) * np.float32(0.4))).astype(np.float32)
    for x in (o, d):
        x.set_surface(eta)
    for _ in range(5):
        d.step_surface_linear(2000, 2000)
        o.step_surface_linear(2000, 2000)
    before = [x.copy() for x in (*d.velocity(), d.pressure(), *d.surface_and_roundoff())]
    with pytest.raises(Delta3dError) as e:
        d.step_surface_linear(2000, 1)
    assert e.value.kind == "Convergence"
    after = [x.copy() for x in (*d.velocity(), d.pressure(), *d.surface_and_roundoff())]
    for a, b in zip(before, after):
        assert_bits(a, b, "restored")
    d.step_surface_linear(2000, 2000)
    o.step_surface_linear(2000, 2000)
    same_state(o, d, "after the retry")


def test_rest_and_guards():
    d = Volume3.configure(8, 6, 4, 1.0, 1025.0, 9.81)
    for _ in range(20):
        r = d.step_surface_linear(2000, 100)
        assert r.iterations == 0
    assert np.all(d.surface_and_roundoff()[0] == 4.0)
    assert not np.any(d.pressure()) and not any(np.any(x) for x in d.velocity())
    with pytest.raises(Delta3dError) as e:
        d.step_surface_linear(0, 100)
    assert e.value.kind == "NotFinite"
    with pytest.raises(Delta3dError) as e:
        d.step_surface_linear(500_000, 100)
    assert e.value.kind == "Domain"
    neg = Volume3.configure(8, 6, 4, 1.0, 1025.0, -1.0)
    with pytest.raises(Delta3dError) as e:
        neg.step_surface_linear(2000, 100)
    assert e.value.kind == "Domain"


def test_f64_reductions_reach_the_acceptance_and_the_oracle_pressure():
    s = scenes.s324_case(64, True)
    o, d = pair(s["nx"], s["ny"], s["nz"], s["dx"], bottom=s["bottom"], reduction=REDUCE_F64)
    for x in (o, d):
        x.set_surface(s["eta"])
    ro = o.step_surface_linear(s["dt_us"], 20000)
    rd = d.step_surface_linear(s["dt_us"], 20000)
    assert not rd.degraded and rd.residual <= 1e-6 and rd.divergence <= 1e-5
    assert abs(rd.iterations - ro["iterations"]) <= 3
    po, pd = o.pressure(), d.pressure()
    assert np.max(np.abs(pd - po)) <= P_TOL * np.max(np.abs(po))


def test_multigrid_volume_uses_the_linear_operator_on_the_linear_path():
    """enable_multigrid does not change the linear path: the same bits with and without it."""
    s = scenes.s324_case(32, True)
    a = Volume3.configure_with_bottom(s["nx"], s["ny"], s["nz"], s["dx"], 1025.0, 9.81, s["bottom"])
    b = Volume3.configure_with_bottom(s["nx"], s["ny"], s["nz"], s["dx"], 1025.0, 9.81, s["bottom"])
    for x in (a, b):
        x.set_options(reduction=REDUCE_ORDERED_F32)
        x.set_surface(s["eta"])
    b.enable_multigrid()
    ra = a.step_surface_linear(s["dt_us"], 20000)
    rb = b.step_surface_linear(s["dt_us"], 20000)
    assert ra.iterations == rb.iterations == 117
    assert_bits(a.pressure(), b.pressure(), "p")
