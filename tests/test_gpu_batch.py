"""fd3_project_batch on the GPU: concurrent patches give each patch's own projection, bit for bit."""
import numpy as np
import pytest

from fluidisim_b200 import batch, scenes
from fluidisim_b200.delta3d import Delta3dError

pytestmark = pytest.mark.gpu


def test_batch_equals_one_projection_at_a_time():
    ps = batch.patch_scenes(12, seed=3, hi=48)
    vols = [batch.configure(p) for p in ps]
    sk = [scenes.projection_scalars(p) for p in ps]
    reps, st = batch.project_batch(vols, [a for a, _ in sk], [b for _, b in sk], threads=6)
    assert st == [0] * len(ps)
    for p, v, r, (scale, k1) in zip(ps, vols, reps, sk):
        assert not r.degraded and r.residual <= 1e-6 and r.divergence_plain <= 1e-5
        alone = batch.configure(p)
        ra = alone.project_mobile3(scale, k1, 4000)
        assert ra.iterations == r.iterations
        assert np.array_equal(alone.pressure().view(np.uint32), v.pressure().view(np.uint32))


def test_batch_refuses_a_volume_listed_twice():
    p = batch.patch_scenes(1, seed=4, hi=24)[0]
    v = batch.configure(p)
    scale, k1 = scenes.projection_scalars(p)
    with pytest.raises(Delta3dError) as e:
        batch.project_batch([v, v], [scale, scale], [k1, k1])
    assert e.value.kind == "InvalidArgument"
