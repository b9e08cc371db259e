"""set_solid_rigid (delta3d.rs:382-509) in the oracle: the solid of a volume moves (CPU only).

The cut is redone from the bottom-only base, so the new geometry must equal the geometry of a
volume configured directly with the moved solid, bit for bit.  A face that opens takes the wall's
velocity at its centre, a face that closes loses its own, and the solid volume each column gains
raises its surface.  Refusals change nothing.
"""
import numpy as np
import pytest

from fluidisim_b200 import scenes
from oracle import oracle as O

N, DX = 16, 0.1
CENTRES = [(0.62, 0.71, 0.43), (1.05, 0.98, 0.55)]
RADII = [0.27, 0.22]


def sdf(shift=(0.0, 0.0, 0.0)):
    c = [(x + shift[0], y + shift[1], z + shift[2]) for x, y, z in CENTRES]
    return scenes.spheres_sdf(N, N, N, DX, c, RADII)


def volume(solid):
    o = O.OracleVolume(N, N, N, DX, 1025.0, 9.81, bottom=np.zeros(N * N, np.float32), solid=solid)
    o.set_free_surface(np.full(N * N, 1.2, np.float32), 1.2)
    return o


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def test_moving_the_solid_recuts_from_the_base():
    o = volume(sdf())
    moved = sdf((0.13, -0.04, 0.05))
    o.set_solid_rigid(moved, (0.5, -0.2, 0.1), (0.0, 0.3, -0.2), (0.8, 0.8, 0.5))
    direct = volume(moved)
    for a, b in zip(o.geometry(), direct.geometry()):
        assert np.array_equal(bits(a), bits(b))


def test_opened_faces_take_the_wall_velocity_and_closed_faces_lose_theirs():
    o = volume(sdf())
    rng = np.random.default_rng(4)
    u, v, w = (rng.uniform(-1, 1, n).astype(np.float32) for n in scenes.face_counts(N, N, N))
    o.set_velocity(u, v, w)
    before = o.geometry()
    vel, ang, cen = (0.5, -0.2, 0.1), (0.0, 0.3, -0.2), (0.8, 0.8, 0.5)
    o.set_solid_rigid(sdf((0.13, -0.04, 0.05)), vel, ang, cen)
    after = o.geometry()
    uu, vv, ww = o.velocity()
    ou0, ou1 = before[1], after[1]
    assert np.all(uu[ou1 == 0] == 0)
    opened = np.nonzero((ou0 == 0) & (ou1 != 0))[0]
    assert opened.size > 0
    for f in opened[:20]:
        i, t = f % (N + 1), f // (N + 1)
        j, k = t % N, t // N
        x = np.float32([i * np.float32(DX), (j + np.float32(0.5)) * np.float32(DX), (k + np.float32(0.5)) * np.float32(DX)])
        r = x - np.float32(cen)
        expect = np.float32(vel[0]) + (np.float32(ang[1]) * r[2] - np.float32(ang[2]) * r[1])
        assert uu[f] == expect
    kept = np.nonzero((ou0 != 0) & (ou1 != 0))[0]
    assert np.array_equal(bits(uu[kept]), bits(u[kept]))


def test_the_displaced_volume_raises_the_surface():
    o = volume(sdf())
    eta0 = o.surface()[0].astype(np.float64)
    frac0 = o.geometry()[0].astype(np.float64)
    o.set_solid_rigid(sdf((0.0, 0.0, 0.3)))  # lifted: the solid volume moves up within the columns
    o.set_solid_rigid(sdf((0.3, 0.0, 0.0)))  # then sideways: columns gain and lose solid
    eta1 = o.surface()[0].astype(np.float64)
    frac1 = o.geometry()[0].astype(np.float64)
    gained = (frac0 - frac1).reshape(N, N, N).sum(axis=0).ravel() * DX ** 3
    assert np.abs((eta1 - eta0) * DX * DX - gained).max() < 1e-6


@pytest.mark.parametrize("case", ["shape", "nan", "lid"])
def test_refusals_change_nothing(case):
    o = volume(sdf())
    before = [x.copy() for x in (*o.geometry(), *o.velocity(), *o.surface())]
    if case == "shape":
        bad, err = sdf()[:-1], "Shape"
    elif case == "nan":
        bad, err = sdf().copy(), "NotFinite"
        bad[7] = np.nan
    else:
        bad, err = scenes.spheres_sdf(N, N, N, DX, [(0.8, 0.8, 1.55)], [0.2]), "Domain"  # reaches the lid layer
    with pytest.raises(O.OracleError) as e:
        o.set_solid_rigid(bad)
    assert e.value.kind == err
    after = [*o.geometry(), *o.velocity(), *o.surface()]
    for a, b in zip(before, after):
        assert np.array_equal(bits(a), bits(b))
