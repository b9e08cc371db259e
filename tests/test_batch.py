"""Host logic of the batched patches: scene generation and the autotuner (CPU only)."""
import numpy as np

from fluidisim_b200 import batch


def test_patch_scenes_follow_the_recipe():
    ps = batch.patch_scenes(6, seed=3)
    for p in ps:
        for n in (p["nx"], p["ny"], p["nz"]):
            assert 16 <= n <= 96 and n % 8 == 0
        assert 0.3 <= p["fill"] <= 0.8
        assert 0.05 <= p["solid_target"] <= 0.15
        nodes = (p["nx"] + 1) * (p["ny"] + 1) * (p["nz"] + 1)
        assert p["solid"].size == nodes
        # the solid fraction of the nodes tracks the target (spheres may overlap)
        frac = float(np.mean(p["solid"] < 0))
        assert 0.5 * p["solid_target"] <= frac <= 2.0 * p["solid_target"] + 0.02, (frac, p["solid_target"])
    # deterministic in the seed
    again = batch.patch_scenes(2, seed=3)
    assert again[0]["nx"] == ps[0]["nx"] and np.array_equal(again[1]["u"], ps[1]["u"])


def test_size_classes_partition_the_cell_counts():
    assert batch.size_class(16 ** 3) == "small"
    assert batch.size_class(48 ** 3) == "medium"
    assert batch.size_class(80 ** 3) == "large"
    groups = batch.by_class([{"nx": 16, "ny": 16, "nz": 16}, {"nx": 96, "ny": 96, "nz": 96}])
    assert len(groups["small"]) == 1 and len(groups["large"]) == 1 and not groups["medium"]


def test_autotune_keeps_the_fastest_candidate_per_class():
    cost = {(0, 0): 5.0, (1, 0): 3.0, (2, 0): 9.0, (0, 3): 4.0, (1, 3): 2.5}
    seen = []

    def timer(scene, kernels, levels):
        seen.append((scene["nx"], kernels, levels))
        bias = 0.0 if scene["nx"] < 40 else (10.0 if kernels == 1 else 0.0)
        return cost[(kernels, levels)] + bias

    groups = {"small": [{"nx": 16, "ny": 16, "nz": 16}, {"nx": 24, "ny": 16, "nz": 16}],
              "medium": [], "large": [{"nx": 96, "ny": 96, "nz": 96}]}
    tuned = batch.autotune(groups, timer=timer)
    assert (tuned["small"].kernels, tuned["small"].levels) == (1, 3)
    assert (tuned["large"].kernels, tuned["large"].levels) == (0, 3)
    assert "medium" not in tuned
    assert {nx for nx, _, _ in seen} == {24, 96}  # the largest patch of each class
