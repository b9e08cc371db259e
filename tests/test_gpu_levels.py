"""The level change (delta3d_levels.rs) on the GPU, through the C ABI (needs a GPU).

Every field a level change writes, and its LevelChange, must be bit-identical to the oracle's: the
surface and its roundoff, the three velocity families, the zero pressure.  The cases are the
reference's own (tests_delta3d_levels.rs): dyadic ratios both ways, the ratio 2.5, sparse sets on
either side, and refusals that write nothing.
"""
import math

import numpy as np
import pytest

from fluidisim_b200.delta3d import Delta3dError, Volume3
from oracle import oracle as O

pytestmark = pytest.mark.gpu

REST = np.float32(2.0)


def bits(a):
    return np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)


def assert_bits(a, b, what):
    a, b = bits(a), bits(b)
    bad = np.nonzero(a != b)[0]
    assert bad.size == 0, f"{what}: {bad.size} differ, first at {bad[:5]}"


def dims(lx, ly, dx):
    f = np.float32
    return (int(round(float(f(lx) / f(dx)))), int(round(float(f(ly) / f(dx)))), int(round(float(f(3.0) / f(dx)))))


def pair(lx, ly, dx, rects=None):
    """The same lx x ly x 3 m volume, at rest at 2 m, in the oracle and on the GPU."""
    nx, ny, nz = dims(lx, ly, dx)
    o = O.OracleVolume(nx, ny, nz, dx, 1000.0, 9.81)
    d = Volume3.configure(nx, ny, nz, dx, 1000.0, 9.81)
    for v in (o, d):
        v.set_free_surface(np.full(nx * ny, REST, np.float32), REST)
    if rects is not None:
        m = np.zeros((ny, nx), np.uint8)
        for i0, i1, j0, j1 in rects:
            m[j0:j1, i0:i1] = 1
        for v in (o, d):
            v.enable_sparse()
            v.set_active_columns(m.ravel())
    return o, d


def smooth_state(vs, nx, ny, nz, dx, corner, mask=None):
    """tests_delta3d_levels.rs:158-201 on both volumes of a pair."""
    d = float(np.float32(dx))
    j, i = np.mgrid[0:ny, 0:nx]
    x, y = (i + 0.5) * d - corner[0], (j + 0.5) * d - corner[1]
    h = 0.05 * np.exp(-((x - 1.5) ** 2 + (y - 0.8) ** 2) / 0.5) + 0.01 * np.sin(2 * math.pi * (x + 0.5 * y) / 1.7)
    eta = (REST + h.astype(np.float32)).astype(np.float32).ravel()
    if mask is not None:
        eta = np.where(mask != 0, eta, REST).astype(np.float32)

    def field(axis, shape, off):
        k, jj, ii = np.mgrid[0:shape[0], 0:shape[1], 0:shape[2]]
        xx, yy, zz = (ii + off[0]) * d - corner[0], (jj + off[1]) * d - corner[1], (k + off[2]) * d
        if axis == 0:
            return (0.1 * np.sin(1.3 * xx + 0.7 * yy + 0.4 * zz)).astype(np.float32).ravel()
        if axis == 1:
            return (0.08 * np.cos(0.9 * xx - 1.1 * yy + 0.3 * zz)).astype(np.float32).ravel()
        return (0.05 * np.sin(0.5 * xx + 0.6 * yy - 0.8 * zz)).astype(np.float32).ravel()

    u = field(0, (nz, ny, nx + 1), (0.0, 0.5, 0.5))
    v = field(1, (nz, ny + 1, nx), (0.5, 0.0, 0.5))
    w = field(2, (nz + 1, ny, nx), (0.5, 0.5, 0.0))
    for vol in vs:
        vol.set_free_surface(eta, REST)
        vol.set_velocity(u, v, w)


def compare(o, d, what):
    e, r = o.surface()
    de, dr = d.surface_and_roundoff()
    assert_bits(e, de, what + " eta")
    assert_bits(r, dr, what + " roundoff")
    for a, b, name in zip(o.velocity(), d.velocity(), "uvw"):
        assert_bits(a, b, what + " " + name)
    assert_bits(o.pressure(), d.pressure(), what + " p")


def same_change(a, b):
    for k in ("volume_before", "volume_after"):
        assert np.float64(a[k]).view(np.uint64) == np.float64(b[k]).view(np.uint64), (k, a, b)


@pytest.mark.parametrize("rects", [None, "sparse"])
def test_a_level_change_down_and_back_is_bit_identical_to_the_oracle(rects):
    """25 -> 50 -> 25 cm, dense or with sparse sets (tests_delta3d_levels.rs:232-258)."""
    fr = None if rects is None else [(8, 24, 8, 16)]
    cr = None if rects is None else [(4, 12, 4, 8)]
    of, df = pair(8, 6, 0.25, fr)
    mask = None if fr is None else df.active_columns()
    smooth_state((of, df), 32, 24, 12, 0.25, (2.0, 2.0), mask)
    oc, dc = pair(8, 6, 0.5, cr)
    same_change(oc.resample_from(of), dc.resample_from(df))
    compare(oc, dc, "down")
    ob, db = pair(8, 6, 0.25, fr)
    same_change(ob.resample_from(oc), db.resample_from(dc))
    compare(ob, db, "back")


def test_a_non_dyadic_ratio_is_bit_identical_to_the_oracle():
    """10 -> 25 cm (ratio 2.5, n = 3 sub-faces per direction) and back (tests_delta3d_levels.rs:77-95)."""
    of, df = pair(8, 4, 0.1)
    smooth_state((of, df), 80, 40, 30, 0.1, (1.0, 1.0))
    om, dm = pair(8, 4, 0.25)
    same_change(om.resample_from(of), dm.resample_from(df))
    compare(om, dm, "10 -> 25 cm")
    ob, db = pair(8, 4, 0.1)
    same_change(ob.resample_from(om), db.resample_from(dm))
    compare(ob, db, "25 -> 10 cm")


def test_a_set_that_does_not_cover_loses_what_it_leaves_out():
    """tests_delta3d_levels.rs:260-283, against the oracle."""
    of, df = pair(8, 6, 0.25, [(8, 24, 8, 16)])
    smooth_state((of, df), 32, 24, 12, 0.25, (2.0, 2.0), df.active_columns())
    oh, dh = pair(8, 6, 0.5, [(4, 8, 4, 8)])
    a, b = oh.resample_from(of), dh.resample_from(df)
    same_change(a, b)
    assert b["volume_before"] - b["volume_after"] > 1e-4
    compare(oh, dh, "half")


def test_a_transferred_state_steps_on():
    """tests_delta3d_levels.rs:151-166: the coarse volume keeps its volume over ten mobile steps."""
    _, fine = pair(8, 4, 0.25)
    j, i = np.mgrid[0:16, 0:32]
    x, y = (i + 0.5) * 0.25, (j + 0.5) * 0.25
    fine.set_free_surface((REST + (0.05 * np.exp(-((x - 4) ** 2 + (y - 2) ** 2))).astype(np.float32)).ravel(), REST)
    for _ in range(10):
        fine.step_surface_mobile(20_000, 20_000)
    _, coarse = pair(8, 4, 0.5)
    c = coarse.resample_from(fine)
    assert abs(c["volume_after"] - c["volume_before"]) <= 1e-10
    for _ in range(10):
        coarse.step_surface_mobile(20_000, 20_000)
    assert abs(coarse.perturbation_volume() - c["volume_after"]) < 1e-9


def test_different_frames_are_refused_and_nothing_is_written():
    """T4 (tests_delta3d_levels.rs:133-149)."""
    _, fine = pair(8, 4, 0.25)
    others = [Volume3.configure(20, 8, 6, 0.5, 1000.0, 9.81), Volume3.configure(16, 8, 6, 0.5, 1000.0, 1.62),
              Volume3.configure_with_bottom(16, 8, 6, 0.5, 1000.0, 9.81, np.zeros(16 * 8, np.float32))]
    for d in others:
        d.set_free_surface(np.full(d.nx * d.ny, REST, np.float32), REST)
        with pytest.raises(Delta3dError) as e:
            d.resample_from(fine)
        assert e.value.code == 1
        assert np.all(bits(d.surface()) == bits(REST))
    rest = Volume3.configure(16, 8, 6, 0.5, 1000.0, 9.81)
    rest.set_free_surface(np.full(16 * 8, 1.5, np.float32), 1.5)
    with pytest.raises(Delta3dError):
        rest.resample_from(fine)
