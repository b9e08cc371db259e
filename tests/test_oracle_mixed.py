"""The oracle's emulation of the library's FP16-storage V-cycle (CPU only).

The V-cycle runs on r / sigma (sigma = rms(r) dx^2 / 6) with every stored V-cycle vector rounded
through FP16.  The projection must still reach the reference's acceptance (relative residual
<= 1e-6, plain divergence <= 1e-5) with about as many iterations as f32 storage, its pressure must
stay within 1e-5 (relative L-infinity) of the f32 projection, its error against an FP64 solve to a
relative residual of 1e-12 must be no worse than f32 storage's, and the scaled vectors must stay
far inside the FP16 range although the pressure itself exceeds it.
"""
import numpy as np
import pytest

from fluidisim_b200 import scenes
from oracle import oracle as O

P_TOL = 1e-5


def solve(s, real="f32", storage=0):
    O.set_storage(storage, real)
    try:
        o = O.OracleVolume(s["nx"], s["ny"], s["nz"], s["dx"], s["rho"], s["g"], bottom=s["bottom"], solid=s["solid"],
                           real=real)
        o.enable_multigrid()
        o.set_free_surface(s["eta"], s["rest"])
        o.set_velocity(s["u"], s["v"], s["w"])
        if real == "f64":
            o.set_tolerance(1e-24)  # |r|^2 <= 1e-24 |b|^2: relative residual 1e-12
        scale, k1 = scenes.projection_scalars(s)
        rep = o.project_mobile(scale, k1, 4000)
        zmax = O.take_zmax(real)
        return rep, o.pressure().astype(np.float64), zmax
    finally:
        O.set_storage(0, real)


@pytest.mark.parametrize("scene", ["box", "lake"])
def test_fp16_storage_meets_the_acceptance_and_the_fp64_solution(scene):
    s = scenes.box_basin(32) if scene == "box" else scenes.sphere_lake(32, spheres=4)
    r64, p64, _ = solve(s, "f64")
    r32, p32, _ = solve(s, "f32", 0)
    r16, p16, zmax = solve(s, "f32", 1)
    assert not r16["degraded"] and r16["residual"] <= 1e-6 and r16["divergence_plain"] <= 1e-5
    assert r16["iterations"] <= r32["iterations"] + 2
    assert np.abs(p16 - p32).max() <= P_TOL * np.abs(p32).max()
    pmax = np.abs(p64).max()
    err16, err32 = np.abs(p16 - p64).max() / pmax, np.abs(p32 - p64).max() / pmax
    assert err16 <= 1.5 * err32 + 5e-6, (err16, err32)
    assert 1.0 <= zmax <= 4096.0, zmax  # well inside FP16 (max 65504), far from its subnormals


def test_fp16_storage_leaves_the_f32_mode_untouched():
    s = scenes.sphere_lake(16, spheres=2)
    ra, pa, _ = solve(s, "f32", 0)
    solve(s, "f32", 1)
    rb, pb, _ = solve(s, "f32", 0)
    assert ra == rb
    assert np.array_equal(pa.astype(np.float32).view(np.uint32), pb.astype(np.float32).view(np.uint32))
