"""The oracle's alternative multigrid recipes, against the reference's, by iterations at relative
residual 1e-6 (CPU).

The reference's V-cycle (delta3d_multigrid.rs:258-299, 393-429) smooths with damped Jacobi
(omega = 6/7), restricts by the mean of the 8 children and prolongates by injection.  The oracle
also has (oracle.set_transfer, oracle.set_smoother):

- trilinear prolongation from the active coarse cells (air as 0, weights renormalised over the
  cells that are neither solid nor outside) with its adjoint, full-weighting restriction;
- red-black Gauss-Seidel in a symmetric order (red first going down, black first coming up), on
  every level, on the fine level only, or on the coarse levels only.

The counts below are what these recipes take on the same scenes.  They are why the library keeps
the reference's recipe on the GPU: trilinear transfer, next to solids and air on this
rediscretised hierarchy, needs up to four times the reference's iterations, and red-black
Gauss-Seidel, which halves them, turns each sweep into two dependent half-sweeps.
"""
import pytest

from fluidisim_b200 import scenes
from oracle import oracle as O

# scene -> {(transfer, smoother): iterations}; smoother 0 Jacobi, 1 RB everywhere, 2 RB fine, 3 RB coarse
EXPECTED = {
    "basin64": {(0, 0): 15, (1, 0): 15, (0, 1): 10, (1, 1): 10, (0, 2): 13, (0, 3): 12},
    "s385_flat64": {(0, 0): 10, (1, 0): 7, (0, 1): 5, (1, 1): 6},
    "s385_bump64": {(0, 0): 10, (1, 0): 19, (0, 1): 5, (1, 1): 16, (0, 2): 8, (0, 3): 7},
    "lake64": {(0, 0): 9, (1, 0): 35, (0, 1): 5, (1, 1): 22, (0, 2): 6, (0, 3): 7},
}


def scene(name):
    return {"basin64": lambda: scenes.box_basin(64), "s385_flat64": lambda: scenes.s385_case(64, False),
            "s385_bump64": lambda: scenes.s385_case(64, True), "lake64": lambda: scenes.sphere_lake(64)}[name]()


def iterations(s, transfer, smoother):
    O.set_transfer(transfer)
    O.set_smoother(smoother)
    try:
        o = O.OracleVolume(s["nx"], s["ny"], s["nz"], s["dx"], s["rho"], s["g"], bottom=s.get("bottom"),
                           solid=s.get("solid"))
        o.enable_multigrid()
        o.set_free_surface(s["eta"], s["rest"])
        if "u" in s:
            o.set_velocity(s["u"], s["v"], s["w"])
            scale, k1 = scenes.projection_scalars(s)
            r = o.project_mobile(scale, k1, 4000)
        else:  # the S385 bench case: its first mobile step from rest
            r = o.step_surface_mobile(s["dt_us"], 20000)
        assert not r["degraded"] and r["residual"] <= 1e-6
        return r["iterations"]
    finally:
        O.set_transfer(0)
        O.set_smoother(0)


@pytest.mark.parametrize("name", sorted(EXPECTED))
def test_transfer_and_smoother_iteration_counts(name):
    O.build()
    O.set_threads(O.max_threads())
    s = scene(name)
    got = {key: iterations(s, *key) for key in EXPECTED[name]}
    assert got == EXPECTED[name]
