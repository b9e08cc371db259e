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


# ------------------------------------------------------------------- the persistent batch (one launch)
def _persistent_case(count=12, seed=3, hi=48, cluster=4):
    ps = batch.patch_scenes(count, seed=seed, hi=hi)
    vols = [batch.configure(p) for p in ps]
    sk = [scenes.projection_scalars(p) for p in ps]
    pb = batch.PersistentBatch(vols, cluster_size=cluster)
    return ps, vols, sk, pb


def test_persistent_batch_matches_one_projection_at_a_time():
    ps, vols, sk, pb = _persistent_case()
    reps, st = pb.project([a for a, _ in sk], [b for _, b in sk])
    assert st == [0] * len(ps)
    assert pb.kernel_launches() == 1
    for p, v, r, (scale, k1) in zip(ps, vols, reps, sk):
        assert not r.degraded and r.residual <= 1e-6 and r.divergence_plain <= 1e-5, r
        alone = batch.configure(p)
        ra = alone.project_mobile3(scale, k1, 4000)
        assert abs(ra.iterations - r.iterations) <= 1, (ra.iterations, r.iterations)
        pa = alone.pressure().astype(np.float64)
        assert np.abs(v.pressure() - pa).max() <= 1e-5 * np.abs(pa).max()
        alone.close()
    pb.close()


@pytest.mark.parametrize("cluster", [1, 2, 8])
def test_persistent_batch_cluster_sizes_agree(cluster):
    ps, vols, sk, pb = _persistent_case(count=6, seed=5, cluster=cluster)
    reps, st = pb.project([a for a, _ in sk], [b for _, b in sk])
    assert st == [0] * len(ps)
    ps2, vols2, _, pb4 = _persistent_case(count=6, seed=5, cluster=4)
    reps4, st4 = pb4.project([a for a, _ in sk], [b for _, b in sk])
    assert st4 == [0] * len(ps)
    for r, r4, v, v4 in zip(reps, reps4, vols, vols2):
        assert abs(r.iterations - r4.iterations) <= 1
        p4 = v4.pressure().astype(np.float64)
        assert np.abs(v.pressure() - p4).max() <= 1e-5 * np.abs(p4).max()
    pb.close()
    pb4.close()


def test_persistent_batch_is_deterministic_and_restores_its_inputs():
    """Two calls from the same device-resident inputs give the same bits (the cluster reductions
    have a fixed order); the inputs are copied in by the launch itself."""
    import torch
    ps, vols, sk, pb = _persistent_case(count=8, seed=7)
    inputs = [tuple(torch.from_numpy(p[k]).cuda() for k in ("u", "v", "w")) for p in ps]
    ptrs = [tuple(t.data_ptr() for t in x) for x in inputs]
    torch.cuda.synchronize()
    out = []
    for _ in range(2):
        reps, st = pb.project([a for a, _ in sk], [b for _, b in sk], reset_pressure=True, inputs=ptrs)
        assert st == [0] * len(ps)
        out.append(([r.as_dict() for r in reps], [v.pressure().copy() for v in vols], [v.velocity()[0] for v in vols]))
    assert out[0][0] == out[1][0]
    for a, b in zip(out[0][1] + out[0][2], out[1][1] + out[1][2]):
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    pb.close()


def test_persistent_batch_refuses_a_nan_input_and_keeps_that_volume():
    import torch
    ps, vols, sk, pb = _persistent_case(count=5, seed=9)
    before = [(v.pressure(), v.velocity()) for v in vols]
    inputs = [tuple(torch.from_numpy(p[k]).cuda() for k in ("u", "v", "w")) for p in ps]
    inputs[2][1][17] = float("nan")
    torch.cuda.synchronize()
    reps, st = pb.project([a for a, _ in sk], [b for _, b in sk], inputs=[tuple(t.data_ptr() for t in x) for x in inputs])
    assert st[2] == 2 and [s for i, s in enumerate(st) if i != 2] == [0] * 4
    p2, (u2, v2, w2) = vols[2].pressure(), vols[2].velocity()
    for a, b in zip((p2, u2, v2, w2), (before[2][0], *before[2][1])):
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    for i in (0, 1, 3, 4):
        assert not reps[i].degraded and reps[i].residual <= 1e-6
    pb.close()


def test_persistent_batch_refuses_unsupported_volumes():
    from fluidisim_b200.delta3d import REDUCE_ORDERED_F32
    ps = batch.patch_scenes(2, seed=4, hi=24)
    vols = [batch.configure(p) for p in ps]
    with pytest.raises(Delta3dError) as e:
        batch.PersistentBatch([vols[0], vols[0]])
    assert e.value.kind == "InvalidArgument"
    vols[1].set_options(reduction=REDUCE_ORDERED_F32)
    with pytest.raises(Delta3dError) as e:
        batch.PersistentBatch(vols)
    assert e.value.kind == "Domain"
    with pytest.raises(Delta3dError):
        batch.PersistentBatch(vols[:1], cluster_size=3)
