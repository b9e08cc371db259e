"""The level change (delta3d_levels.rs): a volume receives the state of another that covers the same
window at another dx (CPU only).

The reference's own criteria (tests_delta3d_levels.rs): a uniform state crosses levels unchanged
to the bit, the perturbation volume is kept to f64 roundoff, a round trip of a smooth wave loses
little and at least at second order, different frames are refused, a transferred state steps on,
and a rectangle of a sparse set crosses levels as its dense rectangle.
"""
import math

import numpy as np
import pytest

from oracle import oracle as O

REST = np.float32(2.0)
DT_US = 20_000


def dims(lx, ly, dx):
    f = np.float32
    return (int(round(float(f(lx) / f(dx)))), int(round(float(f(ly) / f(dx)))), int(round(float(f(3.0) / f(dx)))))


def domain(lx, ly, dx, g=9.81, rest=REST):
    """A lx x ly x 3 m volume at dx, at rest at 2 m (tests_delta3d_levels.rs:9-18)."""
    nx, ny, nz = dims(lx, ly, dx)
    v = O.OracleVolume(nx, ny, nz, dx, 1000.0, g)
    v.set_free_surface(np.full(nx * ny, rest, np.float32), rest)
    return v


def sparse_domain(lx, ly, dx, rects):
    v = domain(lx, ly, dx)
    v.enable_sparse()
    m = np.zeros((v.ny, v.nx), np.uint8)
    for i0, i1, j0, j1 in rects:
        m[j0:j1, i0:i1] = 1
    v.set_active_columns(m.ravel())
    return v


def surface(v, f):
    """rest + f(x, y) at the column centres (tests_delta3d_levels.rs:21-27)."""
    dx = float(np.float32(v.dx))
    j, i = np.mgrid[0:v.ny, 0:v.nx]
    h = f((i + 0.5) * dx, (j + 0.5) * dx).astype(np.float32)
    return (REST + h).astype(np.float32).ravel()


def smooth_state(v, corner, active=None):
    """A smooth state relative to `corner` (m): a bump, an oblique wave and three velocity fields
    (tests_delta3d_levels.rs:158-201); outside the set the surface is at rest."""
    d = float(np.float32(v.dx))
    j, i = np.mgrid[0:v.ny, 0:v.nx]
    x, y = (i + 0.5) * d - corner[0], (j + 0.5) * d - corner[1]
    h = 0.05 * np.exp(-((x - 1.5) ** 2 + (y - 0.8) ** 2) / 0.5) + 0.01 * np.sin(2 * math.pi * (x + 0.5 * y) / 1.7)
    eta = (REST + h.astype(np.float32)).astype(np.float32).ravel()
    if active is not None:
        eta = np.where(active != 0, eta, REST).astype(np.float32)
    v.set_free_surface(eta, REST)

    def field(axis, shape, off):
        k, j, i = np.mgrid[0:shape[0], 0:shape[1], 0:shape[2]]
        x = (i + off[0]) * d - corner[0]
        y = (j + off[1]) * d - corner[1]
        z = (k + off[2]) * d
        if axis == 0:
            return (0.1 * np.sin(1.3 * x + 0.7 * y + 0.4 * z)).astype(np.float32).ravel()
        if axis == 1:
            return (0.08 * np.cos(0.9 * x - 1.1 * y + 0.3 * z)).astype(np.float32).ravel()
        return (0.05 * np.sin(0.5 * x + 0.6 * y - 0.8 * z)).astype(np.float32).ravel()

    nx, ny, nz = v.nx, v.ny, v.nz
    v.set_velocity(field(0, (nz, ny, nx + 1), (0.0, 0.5, 0.5)), field(1, (nz, ny + 1, nx), (0.5, 0.0, 0.5)),
                   field(2, (nz + 1, ny, nx), (0.5, 0.5, 0.0)))


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def test_a_uniform_state_crosses_levels_unchanged():
    """T1 (tests_delta3d_levels.rs:29-63)."""
    fine, coarse = domain(8, 4, 0.25), domain(8, 4, 0.5)
    nx, ny, nz = 32, 16, 12
    fine.set_free_surface(np.full(nx * ny, REST + np.float32(0.0125), np.float32), REST)
    u = np.zeros((nz, ny, nx + 1), np.float32)
    u[:, :, 1:nx] = np.float32(0.1)
    fine.set_velocity(u.ravel(), np.zeros(fine.nv, np.float32), np.zeros(fine.nw, np.float32))
    coarse.resample_from(fine)
    e, r = coarse.surface()
    assert np.all(bits(e) == bits(REST + np.float32(0.0125))) and np.all(r == 0)
    cu = coarse.velocity()[0].reshape(6, 8, 17)
    assert np.all(bits(cu[:, :, 1:16]) == bits(np.float32(0.1)))
    back = domain(8, 4, 0.25)
    back.resample_from(coarse)
    assert np.all(bits(back.surface()[0]) == bits(REST + np.float32(0.0125)))
    bu = back.velocity()[0].reshape(nz, ny, nx + 1)
    assert np.all(bits(bu[:, :, 2:nx - 1]) == bits(np.float32(0.1)))


def test_the_perturbation_volume_is_kept_across_levels():
    """T2 (tests_delta3d_levels.rs:65-96): 25 -> 50 -> 25 cm and 10 -> 25 cm (ratio 2.5)."""
    bump = lambda x, y: 0.05 * np.exp(-((x - 3.1) ** 2 + (y - 1.7) ** 2) / 0.8) + 0.002 * x
    fine = domain(8, 4, 0.25)
    fine.set_free_surface(surface(fine, bump), REST)
    coarse = domain(8, 4, 0.5)
    down = coarse.resample_from(fine)
    back = domain(8, 4, 0.25)
    up = back.resample_from(coarse)
    for c in (down, up):
        assert abs(c["volume_after"] - c["volume_before"]) <= 1e-10, c
    finer = domain(8, 4, 0.1)
    finer.set_free_surface(surface(finer, bump), REST)
    mid = domain(8, 4, 0.25)
    odd = mid.resample_from(finer)
    area = lambda v: (v.nx * float(np.float32(v.dx))) * (v.ny * float(np.float32(v.dx)))
    before, after = odd["volume_before"] / area(finer), odd["volume_after"] / area(mid)
    assert abs(after - before) <= 1e-12 * abs(before), (before, after)


def round_trip(lam):
    k = 2 * math.pi / lam
    wave = lambda x, y: 0.05 * np.cos(k * x) * np.cos(k * y)
    fine = domain(16, 16, 0.25)
    fine.set_free_surface(surface(fine, wave), REST)
    coarse = domain(16, 16, 0.5)
    coarse.resample_from(fine)
    back = domain(16, 16, 0.25)
    back.resample_from(coarse)
    a = back.surface()[0].reshape(64, 64).astype(np.float64)
    b = fine.surface()[0].reshape(64, 64).astype(np.float64)
    return float(np.max(np.abs(a[2:62, 2:62] - b[2:62, 2:62]))) / 0.05


def test_a_round_trip_of_a_smooth_wave_loses_little():
    """T3 (tests_delta3d_levels.rs:120-131): lambda = 8 m within 1 %, and at least second order."""
    e8, e16 = round_trip(8.0), round_trip(16.0)
    assert e8 <= 0.01, e8
    assert e8 / e16 >= 3.0, e8 / e16


def test_different_frames_are_refused():
    """T4 (tests_delta3d_levels.rs:133-149): extent, rest, gravity; nothing is written."""
    fine = domain(8, 4, 0.25)
    for other in (domain(10, 4, 0.5), domain(8, 4, 0.5, rest=np.float32(1.5)), domain(8, 4, 0.5, g=1.62)):
        before = other.surface()[0].copy()
        with pytest.raises(O.OracleError) as e:
            other.resample_from(fine)
        assert e.value.kind == "Domain"
        assert np.array_equal(bits(other.surface()[0]), bits(before))
    cut = O.OracleVolume(16, 8, 6, 0.5, 1000.0, 9.81, bottom=np.zeros(16 * 8, np.float32))
    with pytest.raises(O.OracleError):
        cut.resample_from(fine)


def test_a_transferred_state_steps_on():
    """tests_delta3d_levels.rs:151-166: the volume is kept by the steps that follow."""
    fine = domain(8, 4, 0.25)
    fine.set_free_surface(surface(fine, lambda x, y: 0.05 * np.exp(-((x - 4) ** 2 + (y - 2) ** 2) / 1.0)), REST)
    for _ in range(10):
        fine.step_surface_mobile(DT_US, 20_000)
    coarse = domain(8, 4, 0.5)
    c = coarse.resample_from(fine)
    for _ in range(10):
        coarse.step_surface_mobile(DT_US, 20_000)
    assert abs(coarse.perturbation_volume() - c["volume_after"]) < 1e-9


def window_gap(window, dense, i0, j0):
    e = window.surface()[0].reshape(window.ny, window.nx)[j0:j0 + dense.ny, i0:i0 + dense.nx]
    h = float(np.max(np.abs(e - dense.surface()[0].reshape(dense.ny, dense.nx))))
    wu, wv, ww = window.velocity()
    du, dv, dw = dense.velocity()
    nx, ny, nz = dense.nx, dense.ny, dense.nz
    gaps = [
        np.abs(wu.reshape(nz, window.ny, window.nx + 1)[:, j0:j0 + ny, i0:i0 + nx + 1] - du.reshape(nz, ny, nx + 1)),
        np.abs(wv.reshape(nz, window.ny + 1, window.nx)[:, j0:j0 + ny + 1, i0:i0 + nx] - dv.reshape(nz, ny + 1, nx)),
        np.abs(ww.reshape(nz + 1, window.ny, window.nx)[:, j0:j0 + ny, i0:i0 + nx] - dw.reshape(nz + 1, ny, nx)),
    ]
    return h, max(float(g.max()) for g in gaps)


def outside_at_rest(v):
    act = v.active_columns().reshape(v.ny, v.nx)
    e, r = v.surface()
    u, vv, w = v.velocity()
    U = u.reshape(v.nz, v.ny, v.nx + 1)
    Vv = vv.reshape(v.nz, v.ny + 1, v.nx)
    W = w.reshape(v.nz + 1, v.ny, v.nx)
    for j, i in zip(*np.nonzero(act == 0)):
        c = j * v.nx + i
        if bits(e[c]) != bits(REST) or r[c] != 0:
            return False
        if np.any(U[:, j, i] != 0) or np.any(U[:, j, i + 1] != 0) or np.any(Vv[:, j, i] != 0) or np.any(Vv[:, j + 1, i] != 0):
            return False
        if np.any(W[:, j, i] != 0):
            return False
    return True


def test_a_rectangle_of_the_set_crosses_levels_as_its_dense_rectangle():
    """S404 criterion 3 (tests_delta3d_levels.rs:232-258): within 1 um and 1 um/s, volumes exact."""
    fine = sparse_domain(8, 6, 0.25, [(8, 24, 8, 16)])
    dense_fine = domain(4, 2, 0.25)
    smooth_state(fine, (2.0, 2.0), fine.active_columns())
    smooth_state(dense_fine, (0.0, 0.0))
    assert window_gap(fine, dense_fine, 8, 8) == (0.0, 0.0)
    coarse = sparse_domain(8, 6, 0.5, [(4, 12, 4, 8)])
    dense_coarse = domain(4, 2, 0.5)
    a, b = coarse.resample_from(fine), dense_coarse.resample_from(dense_fine)
    down = window_gap(coarse, dense_coarse, 4, 4)
    back = sparse_domain(8, 6, 0.25, [(8, 24, 8, 16)])
    dense_back = domain(4, 2, 0.25)
    c, d = back.resample_from(coarse), dense_back.resample_from(dense_coarse)
    up = window_gap(back, dense_back, 8, 8)
    assert max(down + up) <= 1e-6, (down, up)
    for ch in (a, b, c, d):
        assert abs(ch["volume_after"] - ch["volume_before"]) <= 1e-10, ch
    assert outside_at_rest(coarse) and outside_at_rest(back)


def test_a_set_that_does_not_cover_loses_what_it_leaves_out_and_says_so():
    """tests_delta3d_levels.rs:260-283."""
    fine = sparse_domain(8, 6, 0.25, [(8, 24, 8, 16)])
    smooth_state(fine, (2.0, 2.0), fine.active_columns())
    half = sparse_domain(8, 6, 0.5, [(4, 8, 4, 8)])
    ch = half.resample_from(fine)
    e, r = fine.surface()
    right = 0.0
    for j in range(8, 16):
        for i in range(16, 24):
            c = j * fine.nx + i
            right += ((float(e[c]) - float(r[c])) - float(REST)) * 0.0625
    assert abs((ch["volume_before"] - ch["volume_after"]) - right) <= 1e-12, (ch, right)
    assert abs(right) > 1e-4
    assert outside_at_rest(half)
    dense = domain(8, 6, 0.5)
    full = dense.resample_from(fine)
    assert abs(full["volume_after"] - full["volume_before"]) <= 1e-10, full
