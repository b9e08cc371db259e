"""An immersed sphere, at rest and moving, through the C ABI (needs a GPU).

The reference's criteria of tests_delta3d.rs:1182-1200 and 1273-1328 on the library: a lake at
rest around the sphere stays at rest to the bit in the mobile step, and a sphere crossing cells at
1 m/s under the lid (set_solid_rigid, then a linear step, 20 times) gives the oracle's bits in the
ordered-f32 mode, step after step.
"""
import numpy as np
import pytest

from fluidisim_b200 import scenes
from fluidisim_b200.delta3d import REDUCE_ORDERED_F32, Volume3
from oracle import oracle as O

pytestmark = pytest.mark.gpu

N = 24
DX = np.float32(1.2) / np.float32(N)
Z0 = np.float32(N) * DX


def sphere_nodes(cx=0.6):
    return scenes.spheres_sdf(N, N, N, DX, [(cx, 0.6, 0.55)], [0.3])


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def pair():
    bottom = np.zeros(N * N, np.float32)
    o = O.OracleVolume(N, N, N, DX, 1025.0, 9.81, bottom=bottom, solid=sphere_nodes())
    d = Volume3.configure_with_solid(N, N, N, DX, 1025.0, 9.81, bottom, sphere_nodes())
    d.set_options(reduction=REDUCE_ORDERED_F32)
    return o, d


def test_a_lake_at_rest_around_the_sphere_stays_at_rest_to_the_bit():
    _, d = pair()
    d.set_free_surface(np.full(N * N, 1.05, np.float32), 1.05)
    for step in range(100):
        d.step_surface_mobile(2000, 4000)
        assert all(np.all(bits(x) == 0) for x in d.velocity()), step
        assert np.all(bits(d.surface()) == bits(np.float32(1.05))), step
    d.close()


def test_a_moving_sphere_matches_the_oracle_step_after_step():
    o, d = pair()
    for v in (o, d):
        v.set_surface(np.full(N * N, Z0, np.float32))
    for step in range(1, 21):
        s = sphere_nodes(0.6 + 0.002 * step)
        o.set_solid_rigid(s, (1.0, 0.0, 0.0))
        d.set_solid_rigid(s, (1.0, 0.0, 0.0))
        ro, rd = o.step_surface_linear(2000, 4000), d.step_surface_linear(2000, 4000)
        assert rd.iterations == ro["iterations"], step
        oe, orr = o.surface()
        de, dr = d.surface_and_roundoff()
        assert np.array_equal(bits(oe), bits(de)) and np.array_equal(bits(orr), bits(dr)), step
        for a, b in zip(o.velocity(), d.velocity()):
            assert np.array_equal(bits(a), bits(b)), step
    for a, b in zip(o.geometry(), d.geometry()):
        assert np.array_equal(bits(a), bits(b))
    d.close()
