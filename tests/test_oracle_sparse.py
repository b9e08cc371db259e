"""The sparse column set (delta3d_sparse.rs) in the oracle (CPU only).

A set of columns inside the box's window is the domain: a column outside it is solid for every
operator, a face touching it is closed, and it stays at rest.  These are the reference's own
criteria (tests_delta3d_sparse.rs): a full set is the box to the bit, a column that leaves goes to
rest and what it carried is published, paths that do not carry a set refuse it, blocks cover their
columns clipped to the window, and a rectangle of the set behaves as the dense rectangle.
"""
import numpy as np
import pytest

from fluidisim_b200 import scenes
from oracle import oracle as O

DX, NZ, REST = scenes.SPARSE_DX, scenes.SPARSE_NZ, scenes.SPARSE_REST
DT_US = 20_000


def domain(nx, ny, sparse, mg=False):
    """configure + clear_to_rest (tests_delta3d_sparse.rs:15-24, 188-198)."""
    v = O.OracleVolume(nx, ny, NZ, DX, 1000.0, 9.81)
    v.set_free_surface(np.full(nx * ny, REST, np.float32), REST)
    if mg:
        v.enable_multigrid()
    if sparse:
        v.enable_sparse()
    return v


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def state(v):
    e, r = v.surface()
    return [bits(x) for x in (e, r, *v.velocity(), v.pressure())]


def perturbation_volume(v):
    """perturbation_volume (delta3d_balance.rs:105-113), summed in column order in f64."""
    e, r = v.surface()
    total = 0.0
    for h, lost in zip(e.astype(np.float64), r.astype(np.float64)):
        total += (h - lost) - np.float64(np.float32(REST))
    return total * (np.float64(np.float32(DX)) ** 2)


@pytest.mark.parametrize("correction", [False, True])
def test_a_full_set_is_the_box_at_bit(correction):
    """Criterion 1 (tests_delta3d_sparse.rs:52-72): with every column in the set, fifty mobile steps
    are bit-identical to the steps without a set, with and without the second-order advection term."""
    plain, sparse = domain(24, 16, False), domain(24, 16, True)
    eta = scenes.bumps_in(24, 16, np.ones(24 * 16), [(9.0, 7.0)])
    for v in (plain, sparse):
        v.set_free_surface(eta, REST)
        if correction:
            v.enable_advection_correction()
    assert sparse.sparse_cells() == plain.cells
    for s in range(50):
        a, b = plain.step_surface_mobile(DT_US, 20_000), sparse.step_surface_mobile(DT_US, 20_000)
        assert a["iterations"] == b["iterations"], s
        for x, y in zip(state(plain), state(sparse)):
            assert np.array_equal(x, y), s


def test_a_column_that_leaves_goes_to_rest_and_what_it_carried_is_published():
    """tests_delta3d_sparse.rs:74-131."""
    nx, ny = 24, 16
    v = domain(nx, ny, True)
    v.set_free_surface(scenes.bumps_in(nx, ny, np.ones(nx * ny), [(9.0, 7.0)]), REST)
    for _ in range(10):
        v.step_surface_mobile(DT_US, 20_000)
    before = perturbation_volume(v)
    e, r = v.surface()
    carried, high = 0.0, np.float32(0.0)
    for j in range(ny):
        for i in range(16, nx):
            c = j * nx + i
            carried += ((np.float64(e[c]) - np.float64(r[c])) - np.float64(np.float32(REST))) * np.float64(np.float32(DX)) ** 2
            high = max(high, np.float32(abs(np.float32(e[c] - np.float32(REST)))))
    mask = (np.arange(nx * ny) % nx < 16).astype(np.uint8)
    ch = v.set_active_columns(mask)
    assert (ch["activated"], ch["deactivated"], ch["active_columns"]) == (0, 8 * ny, 16 * ny)
    assert np.float64(ch["volume_removed"]).view(np.uint64) == np.float64(carried).view(np.uint64)
    assert np.float32(ch["height_removed"]) == high
    assert ch["velocity_removed"] > 0
    assert abs(perturbation_volume(v) - (before - carried)) < 1e-12
    assert v.sparse_cells() == 16 * ny * NZ
    for _ in range(10):
        v.step_surface_mobile(DT_US, 20_000)
    e, _ = v.surface()
    u, vv, w = v.velocity()
    p = v.pressure().reshape(NZ, ny, nx)
    U = u.reshape(NZ, ny, nx + 1)
    Vv = vv.reshape(NZ, ny + 1, nx)
    W = w.reshape(NZ + 1, ny, nx)
    assert np.all(bits(e.reshape(ny, nx)[:, 16:]) == bits(np.float32(REST)))
    assert np.all(U[:, :, 17:] == 0) and np.all(Vv[:, :, 16:] == 0) and np.all(W[:, :, 16:] == 0)
    assert np.all(p[:, :, 16:] == 0)
    assert np.all(U[:, :, 16] == 0)  # the edge of the set is a wall
    back = v.set_active_columns(np.ones(nx * ny, np.uint8))
    assert (back["activated"], back["deactivated"], back["volume_removed"], back["velocity_removed"]) == \
        (8 * ny, 0, 0.0, 0.0)


def test_paths_that_do_not_carry_the_set_refuse_it():
    """tests_delta3d_sparse.rs:133-172 (the paths this library has)."""
    nx, ny = 16, 8
    v = domain(nx, ny, True)
    out = np.ones(nx * ny, np.uint8)
    out[0] = 0
    v.set_active_columns(out)
    with pytest.raises(O.OracleError) as e:
        v.step_surface_linear(DT_US, 100)
    assert e.value.kind == "Domain"
    with pytest.raises(O.OracleError) as e:
        v.enable_sparse()
    assert e.value.kind == "Domain"
    eta = np.full(nx * ny, REST, np.float32)
    eta[0] = np.float32(REST + 0.01)
    with pytest.raises(O.OracleError) as e:
        v.set_free_surface(eta, REST)
    assert e.value.kind == "Domain"
    with pytest.raises(O.OracleError) as e:
        v.set_surface(eta)
    assert e.value.kind == "Domain"
    assert bits(v.surface()[0][0]) == bits(np.float32(REST))
    plain = domain(nx, ny, False)
    with pytest.raises(O.OracleError) as e:
        plain.set_active_columns(out)
    assert e.value.kind == "Domain"
    with pytest.raises(O.OracleError) as e:
        v.set_active_columns(out[1:])
    assert e.value.kind == "Shape"


def test_blocks_cover_their_columns_clipped_to_the_window():
    """tests_delta3d_sparse.rs:174-194: blocks of 8 x 8 columns relative to an origin block."""
    nx, ny = 20, 12
    v = domain(nx, ny, True)
    ch = v.set_active_blocks([(10, -1), (11, 0), (12, 0), (10, 1)], origin=(10, 0))
    active = v.active_columns().reshape(ny, nx)
    j, i = np.mgrid[0:ny, 0:nx]
    want = ((j < 8) & (i >= 8)) | ((j >= 8) & (i < 8))
    assert np.array_equal(active != 0, want)
    assert ch["active_columns"] == 8 * 8 + 4 * 8 + 8 * 4


def gap(window, dense, i0, j0):
    wn = window.nx
    e, _ = window.surface()
    d, _ = dense.surface()
    e = e.reshape(window.ny, wn)[j0:j0 + dense.ny, i0:i0 + dense.nx]
    return float(np.max(np.abs(e - d.reshape(dense.ny, dense.nx))))


@pytest.mark.parametrize("mg", [False, True])
def test_a_rectangle_of_the_set_is_the_dense_rectangle(mg):
    """tests_delta3d_sparse.rs:240-262 (a): a 16 x 8 rectangle in a 32 x 24 window against the dense
    16 x 8 domain; the surfaces agree to the solver's roundoff (criterion 1e-5 m).  60 steps here
    (the reference runs 250)."""
    nx, ny = 32, 24
    mask = scenes.rect_mask(nx, ny, [(8, 24, 8, 16)])
    window = domain(nx, ny, True, mg)
    window.set_active_columns(mask)
    window.set_free_surface(scenes.bumps_in(nx, ny, mask, [(14.0, 11.0)]), REST)
    dense = domain(16, 8, False, mg)
    dense.set_free_surface(scenes.bumps_in(16, 8, np.ones(128), [(6.0, 3.0)]), REST)
    worst = 0.0
    for _ in range(60):
        window.step_surface_mobile(DT_US, 20_000)
        dense.step_surface_mobile(DT_US, 20_000)
        worst = max(worst, gap(window, dense, 8, 8))
    assert worst <= 1e-5, worst


def test_two_disjoint_rectangles_are_two_dense_domains():
    """tests_delta3d_sparse.rs:264-290 (b): the columns between the rectangles stay at rest to the bit."""
    nx, ny = 40, 16
    mask = scenes.rect_mask(nx, ny, [(0, 16, 0, 16), (24, 40, 0, 16)])
    window = domain(nx, ny, True)
    window.set_active_columns(mask)
    window.set_free_surface(scenes.bumps_in(nx, ny, mask, [(12.0, 6.0), (29.0, 9.0)]), REST)
    a, b = domain(16, 16, False), domain(16, 16, False)
    a.set_free_surface(scenes.bumps_in(16, 16, np.ones(256), [(12.0, 6.0)]), REST)
    b.set_free_surface(scenes.bumps_in(16, 16, np.ones(256), [(5.0, 9.0)]), REST)
    worst = 0.0
    for _ in range(40):
        for v in (window, a, b):
            v.step_surface_mobile(DT_US, 20_000)
        worst = max(worst, gap(window, a, 0, 0), gap(window, b, 24, 0))
    e, _ = window.surface()
    assert np.all(bits(e.reshape(ny, nx)[:, 16:24]) == bits(np.float32(REST)))
    assert worst <= 1e-5, worst


def test_an_l_shaped_set_keeps_its_volume():
    """tests_delta3d_sparse.rs:292-313 (c): the perturbation volume of an L of blocks drifts no more
    than ten times the dense tank's floor."""
    nx, ny = 24, 24
    mask = scenes.rect_mask(nx, ny, [(0, 24, 0, 8), (0, 8, 8, 24)])
    l_set = domain(nx, ny, True)
    l_set.set_active_columns(mask)
    l_set.set_free_surface(scenes.bumps_in(nx, ny, mask, [(6.0, 6.0)]), REST)
    dense = domain(nx, ny, False)
    dense.set_free_surface(scenes.bumps_in(nx, ny, np.ones(nx * ny), [(6.0, 6.0)]), REST)
    v0, d0 = perturbation_volume(l_set), perturbation_volume(dense)
    drift = floor = 0.0
    for _ in range(40):
        l_set.step_surface_mobile(DT_US, 20_000)
        dense.step_surface_mobile(DT_US, 20_000)
        drift = max(drift, abs(perturbation_volume(l_set) - v0))
        floor = max(floor, abs(perturbation_volume(dense) - d0))
    assert drift <= 10 * max(floor, 1e-15), (drift, floor)
