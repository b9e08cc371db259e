"""refine_mobile3 (delta3d_coupling.rs:226-248) in the oracle (CPU only).

After a projection stopped early (capped iterations: degraded), one refinement projects the
corrected field from p = 0 with homogeneous ghosts and adds the increment: the result must meet
the reference's acceptance, report one refinement, and give the pressure of a full projection
(both are solutions of the same problem to a relative residual of 1e-6).
"""
import numpy as np

from fluidisim_b200 import scenes
from oracle import oracle as O


def lake():
    s = scenes.sphere_lake(32, spheres=4)
    o = O.OracleVolume(s["nx"], s["ny"], s["nz"], s["dx"], s["rho"], s["g"], bottom=s["bottom"], solid=s["solid"])
    o.enable_multigrid()
    o.set_free_surface(s["eta"], s["rest"])
    o.set_velocity(s["u"], s["v"], s["w"])
    return o, s


def test_refinement_completes_a_capped_projection():
    o, s = lake()
    scale, k1 = scenes.projection_scalars(s)
    capped = o.project_mobile(scale, k1, 3)
    assert capped["degraded"] and capped["refinements"] == 0
    r = o.refine_mobile(scale, k1, 4000)
    assert r["refinements"] == 1 and not r["degraded"]
    assert r["residual"] <= 1e-6 and r["divergence_plain"] <= 1e-5
    full, _ = lake()
    full.project_mobile(scale, k1, 4000)
    pf = full.pressure().astype(np.float64)
    assert np.abs(o.pressure() - pf).max() <= 1e-5 * np.abs(pf).max()


def test_refinement_leaves_the_ghosts_inhomogeneous_afterwards():
    o, s = lake()
    scale, k1 = scenes.projection_scalars(s)
    o.project_mobile(scale, k1, 4000)
    o.refine_mobile(scale, k1, 4000)
    # the next projection assembles the same right-hand side as a fresh volume's
    fresh, _ = lake()
    o.set_velocity(s["u"], s["v"], s["w"])
    o.set_free_surface(s["eta"], s["rest"])
    a = o.project_mobile(scale, k1, 4000)
    b = fresh.project_mobile(scale, k1, 4000)
    assert a == b
    assert np.array_equal(o.pressure().view(np.uint32), fresh.pressure().view(np.uint32))
