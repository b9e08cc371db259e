"""The sparse column set (delta3d_sparse.rs) on the GPU, through the C ABI (needs a GPU).

With the ordered f32 reductions every published field and every SparseChange must be
bit-identical to the oracle's; with the default f64 reductions and the blocked kernels a full set
must be bit-identical to the box, and a rectangle of the set must behave as the dense rectangle
to the reference's criterion (1e-5 m, tests_delta3d_sparse.rs:240-262).
"""
import numpy as np
import pytest

from fluidisim_b200 import scenes
from fluidisim_b200.delta3d import REDUCE_F64, REDUCE_ORDERED_F32, Delta3dError, Volume3
from oracle import oracle as O

pytestmark = pytest.mark.gpu

DX, NZ, REST = scenes.SPARSE_DX, scenes.SPARSE_NZ, scenes.SPARSE_REST
DT_US = 20_000


def bits(a):
    return np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)


def assert_bits(a, b, what):
    a, b = bits(a), bits(b)
    bad = np.nonzero(a != b)[0]
    assert bad.size == 0, f"{what}: {bad.size} differ, first at {bad[:5]}"


def gpu(nx, ny, sparse, mg=False, reduction=REDUCE_ORDERED_F32, nz=NZ):
    d = Volume3.configure(nx, ny, nz, DX, 1000.0, 9.81)
    d.set_options(reduction=reduction)
    d.set_free_surface(np.full(nx * ny, REST, np.float32), REST)
    if mg:
        d.enable_multigrid()
    if sparse:
        d.enable_sparse()
    return d


def oracle(nx, ny, sparse, mg=False, nz=NZ):
    o = O.OracleVolume(nx, ny, nz, DX, 1000.0, 9.81)
    o.set_free_surface(np.full(nx * ny, REST, np.float32), REST)
    if mg:
        o.enable_multigrid()
    if sparse:
        o.enable_sparse()
    return o


def fields(v):
    if isinstance(v, Volume3):
        e, r = v.surface_and_roundoff()
    else:
        e, r = v.surface()
    return [e, r, *v.velocity(), v.pressure()]


NAMES = ["eta", "roundoff", "u", "v", "w", "p"]


@pytest.mark.parametrize("reduction", [REDUCE_ORDERED_F32, REDUCE_F64])
@pytest.mark.parametrize("mg", [False, True])
@pytest.mark.parametrize("correction", [False, True])
def test_a_full_set_is_the_box_at_bit(reduction, mg, correction):
    """Criterion 1 (tests_delta3d_sparse.rs:52-72), in both reduction modes and kernel families, with
    and without the second-order advection term."""
    nx, ny = 24, 16
    plain, sparse = gpu(nx, ny, False, mg, reduction), gpu(nx, ny, True, mg, reduction)
    eta = scenes.bumps_in(nx, ny, np.ones(nx * ny), [(9.0, 7.0)])
    for v in (plain, sparse):
        v.set_free_surface(eta, REST)
        if correction:
            v.enable_advection_correction()
    assert sparse.sparse_cells() == nx * ny * NZ
    for s in range(20):
        a, b = plain.step_surface_mobile(DT_US, 20_000), sparse.step_surface_mobile(DT_US, 20_000)
        assert a.iterations == b.iterations, s
    for x, y, name in zip(fields(plain), fields(sparse), NAMES):
        assert_bits(x, y, name)


@pytest.mark.parametrize("mg", [False, True])
def test_steps_on_an_l_shaped_set_are_bit_identical_to_the_oracle(mg):
    """Ordered mode: twenty mobile steps on an L of blocks, every field bit for bit."""
    nx, ny = 24, 24
    mask = scenes.rect_mask(nx, ny, [(0, 24, 0, 8), (0, 8, 8, 24)])
    eta = scenes.bumps_in(nx, ny, mask, [(6.0, 6.0)])
    o, d = oracle(nx, ny, True, mg), gpu(nx, ny, True, mg)
    for v in (o, d):
        v.set_active_columns(mask)
        v.set_free_surface(eta, REST)
    for s in range(20):
        a, b = o.step_surface_mobile(DT_US, 20_000), d.step_surface_mobile(DT_US, 20_000)
        assert a["iterations"] == b.iterations, s
    for x, y, name in zip(fields(o), fields(d), NAMES):
        assert_bits(x, y, name)


def test_a_column_that_leaves_matches_the_oracle():
    """tests_delta3d_sparse.rs:74-131 against the oracle: the published change to the bit, the columns
    at rest, the edge of the set a wall, and ten more steps bit for bit."""
    nx, ny = 24, 16
    eta = scenes.bumps_in(nx, ny, np.ones(nx * ny), [(9.0, 7.0)])
    o, d = oracle(nx, ny, True), gpu(nx, ny, True)
    for v in (o, d):
        v.set_free_surface(eta, REST)
    for _ in range(10):
        o.step_surface_mobile(DT_US, 20_000)
        d.step_surface_mobile(DT_US, 20_000)
    mask = (np.arange(nx * ny) % nx < 16).astype(np.uint8)
    co, cd = o.set_active_columns(mask), d.set_active_columns(mask)
    assert (cd.activated, cd.deactivated, cd.active_columns) == (0, 8 * ny, 16 * ny)
    assert (co["activated"], co["deactivated"], co["active_columns"]) == (cd.activated, cd.deactivated,
                                                                          cd.active_columns)
    assert np.float64(cd.volume_removed).view(np.uint64) == np.float64(co["volume_removed"]).view(np.uint64)
    assert np.float32(cd.height_removed) == np.float32(co["height_removed"])
    assert np.float32(cd.velocity_removed) == np.float32(co["velocity_removed"]) and cd.velocity_removed > 0
    assert d.sparse_cells() == 16 * ny * NZ
    assert np.array_equal(d.active_columns(), mask)
    for x, y, name in zip(fields(o), fields(d), NAMES):
        assert_bits(x, y, "after the change: " + name)
    for _ in range(10):
        o.step_surface_mobile(DT_US, 20_000)
        d.step_surface_mobile(DT_US, 20_000)
    for x, y, name in zip(fields(o), fields(d), NAMES):
        assert_bits(x, y, name)
    e = d.surface()
    u, v, w = d.velocity()
    assert np.all(bits(e.reshape(ny, nx)[:, 16:]) == bits(np.float32(REST)))
    assert np.all(u.reshape(NZ, ny, nx + 1)[:, :, 16:] == 0)
    assert np.all(v.reshape(NZ, ny + 1, nx)[:, :, 16:] == 0)
    assert np.all(w.reshape(NZ + 1, ny, nx)[:, :, 16:] == 0)
    assert np.all(d.pressure().reshape(NZ, ny, nx)[:, :, 16:] == 0)
    back = d.set_active_columns(np.ones(nx * ny, np.uint8))
    assert (back.activated, back.deactivated, back.volume_removed, back.velocity_removed) == (8 * ny, 0, 0.0, 0.0)


def test_set_velocity_closes_the_faces_outside_the_set():
    """set_velocity (delta3d.rs:631-645): close_walls, then close_sparse_walls, as the oracle."""
    nx, ny = 20, 12
    mask = scenes.rect_mask(nx, ny, [(3, 14, 2, 9), (14, 20, 5, 12)])
    o, d = oracle(nx, ny, True), gpu(nx, ny, True)
    rng = np.random.default_rng(7)
    u, v, w = (rng.uniform(-1, 1, n).astype(np.float32) for n in scenes.face_counts(nx, ny, NZ))
    for x in (o, d):
        x.set_active_columns(mask)
        x.set_velocity(u, v, w)
    for a, b, name in zip(o.velocity(), d.velocity(), "uvw"):
        assert_bits(a, b, name)


def test_paths_that_do_not_carry_the_set_refuse_it():
    """tests_delta3d_sparse.rs:133-172 (the paths this library has); nothing is written."""
    nx, ny = 16, 8
    d = gpu(nx, ny, True)
    out = np.ones(nx * ny, np.uint8)
    out[0] = 0
    d.set_active_columns(out)
    for call in (lambda: d.step_surface_linear(DT_US, 100), lambda: d.project(-1e5, 1e-5, 100), d.enable_sparse):
        with pytest.raises(Delta3dError) as e:
            call()
        assert e.value.code == 1
    eta = np.full(nx * ny, REST, np.float32)
    eta[0] = np.float32(REST + 0.01)
    for call in (lambda: d.set_free_surface(eta, REST), lambda: d.set_surface(eta)):
        with pytest.raises(Delta3dError) as e:
            call()
        assert e.value.code == 1
    assert bits(d.surface()[0]) == bits(np.float32(REST))
    plain = gpu(nx, ny, False)
    assert plain.active_columns() is None
    with pytest.raises(Delta3dError) as e:
        plain.set_active_columns(out)
    assert e.value.code == 1
    with pytest.raises(Delta3dError) as e:
        d.set_active_columns(out[1:])
    assert e.value.code == 3


def test_blocks_cover_their_columns_clipped_to_the_window():
    """tests_delta3d_sparse.rs:174-194."""
    nx, ny = 20, 12
    d = gpu(nx, ny, True)
    ch = d.set_active_blocks([(10, -1), (11, 0), (12, 0), (10, 1)], origin=(10, 0))
    j, i = np.mgrid[0:ny, 0:nx]
    want = ((j < 8) & (i >= 8)) | ((j >= 8) & (i < 8))
    assert np.array_equal(d.active_columns().reshape(ny, nx) != 0, want)
    assert ch.active_columns == 8 * 8 + 4 * 8 + 8 * 4


@pytest.mark.parametrize("mg", [False, True])
def test_a_rectangle_of_the_set_is_the_dense_rectangle(mg):
    """tests_delta3d_sparse.rs:240-262 (a) with the default f64 reductions and blocked kernels: a
    16 x 8 rectangle in a 32 x 24 window against the dense 16 x 8 domain, 250 steps of 20 ms,
    surfaces within 1e-5 m."""
    nx, ny = 32, 24
    mask = scenes.rect_mask(nx, ny, [(8, 24, 8, 16)])
    window = gpu(nx, ny, True, mg, REDUCE_F64)
    window.set_active_columns(mask)
    window.set_free_surface(scenes.bumps_in(nx, ny, mask, [(14.0, 11.0)]), REST)
    dense = gpu(16, 8, False, mg, REDUCE_F64)
    dense.set_free_surface(scenes.bumps_in(16, 8, np.ones(128), [(6.0, 3.0)]), REST)
    worst = 0.0
    for _ in range(250):
        window.step_surface_mobile(DT_US, 20_000)
        dense.step_surface_mobile(DT_US, 20_000)
        e = window.surface().reshape(ny, nx)[8:16, 8:24]
        worst = max(worst, float(np.max(np.abs(e - dense.surface().reshape(8, 16)))))
    assert worst <= 1e-5, worst


def test_a_sparse_set_over_a_cut_lake_matches_the_oracle():
    """Ordered mode: a 32^3 lake with solid spheres, multigrid, and a set of blocks with a re-entrant
    corner; the projection's fields bit for bit."""
    s = scenes.sphere_lake(32, seed=1, spheres=4)
    o = O.OracleVolume(32, 32, 32, s["dx"], s["rho"], s["g"], bottom=s["bottom"], solid=s["solid"])
    d = Volume3.configure_with_solid(32, 32, 32, s["dx"], s["rho"], s["g"], s["bottom"], s["solid"])
    d.set_options(reduction=REDUCE_ORDERED_F32)
    mask = scenes.rect_mask(32, 32, [(0, 24, 0, 16), (8, 32, 16, 32)])
    eta = np.where(mask != 0, s["eta"], np.float32(s["rest"])).astype(np.float32)
    for v in (o, d):
        v.enable_multigrid()
        v.enable_sparse()
        v.set_active_columns(mask)
        v.set_free_surface(eta, s["rest"])
        v.set_velocity(s["u"], s["v"], s["w"])
    scale, k1 = scenes.projection_scalars(s)
    a, b = o.project_mobile(scale, k1), d.project_mobile3(scale, k1)
    assert a["iterations"] == b.iterations
    for x, y, name in zip([*o.velocity(), o.pressure()], [*d.velocity(), d.pressure()], ["u", "v", "w", "p"]):
        assert_bits(x, y, name)


@pytest.mark.parametrize("kernels", [0, 2, 3, 4, 5])
def test_skipping_the_tiles_outside_the_set_changes_no_bit(kernels):
    """The blocked fine kernels skip the column tiles with no column of the set (32 x 8 with one cell
    per thread, 64 x 8 with two, 128 x 8 with four, 64 x 8 TMA-staged: kernels 2, 3 (and 0 here), 4
    and 5, nx = 128).
    Against the same volume processing every tile: every field bit for bit, through steps, a set
    change that empties tiles and one that refills them."""
    nx, ny = 128, 64
    vols = []
    for skip in (0, 1):
        d = Volume3.configure(nx, ny, NZ, DX, 1000.0, 9.81)
        d.set_options(reduction=REDUCE_F64, kernels=kernels, no_tile_skip=skip)
        d.set_free_surface(np.full(nx * ny, REST, np.float32), REST)
        d.enable_multigrid()
        d.enable_sparse()
        vols.append(d)
    masks = [scenes.rect_mask(nx, ny, [(0, 40, 0, 24), (70, 128, 30, 64)]),
             scenes.rect_mask(nx, ny, [(0, 40, 0, 24), (70, 100, 30, 64)]),
             scenes.rect_mask(nx, ny, [(0, 128, 0, 24), (70, 128, 30, 64)])]
    first = True
    for mask in masks:
        for d in vols:
            d.set_active_columns(mask)
            if first:
                d.set_free_surface(scenes.bumps_in(nx, ny, mask, [(20.0, 12.0), (90.0, 45.0)]), REST)
        first = False
        for s in range(8):
            a, b = (d.step_surface_mobile(DT_US, 20_000) for d in vols)
            assert a.iterations == b.iterations, s
        for x, y, name in zip(fields(vols[0]), fields(vols[1]), NAMES):
            assert_bits(x, y, name)


def _solid_pair(mask):
    """A 32^3 cut volume with two solid spheres, multigrid, ordered reductions, and the sparse set
    `mask`, in the oracle and on the GPU."""
    n, dx = 32, 0.1
    centres = [(1.24, 1.42, 0.86), (2.10, 1.96, 1.10)]
    radii = [0.54, 0.44]
    sdf = scenes.spheres_sdf(n, n, n, dx, centres, radii)
    bottom = np.zeros(n * n, np.float32)
    o = O.OracleVolume(n, n, n, dx, 1025.0, 9.81, bottom=bottom, solid=sdf)
    d = Volume3.configure_with_solid(n, n, n, dx, 1025.0, 9.81, bottom, sdf)
    d.set_options(reduction=REDUCE_ORDERED_F32)
    rng = np.random.default_rng(9)
    u, v, w = (rng.uniform(-1, 1, k).astype(np.float32) for k in scenes.face_counts(n, n, n))
    for x in (o, d):
        x.enable_multigrid()
        x.enable_sparse()
        x.set_active_columns(mask)
        x.set_free_surface(np.full(n * n, 2.1, np.float32), 2.1)
        x.set_velocity(u, v, w)
    moved = scenes.spheres_sdf(n, n, n, dx, [(x + 0.13, y - 0.06, z + 0.08) for x, y, z in centres], radii)
    return o, d, moved


def test_a_moving_solid_in_a_sparse_set_matches_the_oracle():
    """set_solid_rigid on a volume with a sparse set whose edge crosses the spheres: the moved
    geometry, the face velocities, the raised surface and the next projection, bit for bit."""
    mask = scenes.rect_mask(32, 32, [(0, 20, 0, 32), (20, 32, 8, 24)])
    o, d, moved = _solid_pair(mask)
    motion = ((0.5, -0.2, 0.1), (0.0, 0.3, -0.2), (1.6, 1.6, 1.0))
    o.set_solid_rigid(moved, *motion)
    d.set_solid_rigid(moved, *motion)
    for a, b, name in zip(o.velocity(), d.velocity(), "uvw"):
        assert_bits(a, b, name)
    for a, b in zip(o.surface(), d.surface_and_roundoff()):
        assert_bits(a, b, "eta/roundoff")
    ro = o.project_mobile(-1025.0 * 60.0, 1.0 / (60.0 * 1025.0), 4000)
    rd = d.project_mobile3(-1025.0 * 60.0, 1.0 / (60.0 * 1025.0), 4000)
    assert ro["iterations"] == rd.iterations
    for a, b, name in zip([*o.velocity(), o.pressure()], [*d.velocity(), d.pressure()], ["u", "v", "w", "p"]):
        assert_bits(a, b, name)


def test_a_refinement_in_a_sparse_set_matches_the_oracle():
    """refine_mobile3 after a capped projection on a volume with a sparse set, bit for bit."""
    mask = scenes.rect_mask(32, 32, [(4, 28, 0, 16), (4, 12, 16, 32)])
    o, d, _ = _solid_pair(mask)
    scale, k1 = -1025.0 * 60.0, 1.0 / (60.0 * 1025.0)
    o.project_mobile(scale, k1, 3)
    d.project_mobile3(scale, k1, 3)
    ro, rd = o.refine_mobile(scale, k1, 4000), d.refine_mobile3(scale, k1, 4000)
    assert ro["iterations"] == rd.iterations
    for a, b, name in zip([*o.velocity(), o.pressure()], [*d.velocity(), d.pressure()], ["u", "v", "w", "p"]):
        assert_bits(a, b, name)


def test_fp16_storage_skips_the_tiles_outside_the_set_without_changing_a_bit():
    """The FP16-storage V-cycle (its vectors are half-width) with tiles skipped, against every tile
    processed, through steps and a set change."""
    from fluidisim_b200.delta3d import STORAGE_F16
    nx, ny = 128, 64
    vols = []
    for skip in (0, 1):
        d = Volume3.configure(nx, ny, NZ, DX, 1000.0, 9.81)
        d.set_options(reduction=REDUCE_F64, kernels=0, storage=STORAGE_F16, no_tile_skip=skip)
        d.set_free_surface(np.full(nx * ny, REST, np.float32), REST)
        d.enable_multigrid()
        d.enable_sparse()
        vols.append(d)
    masks = [scenes.rect_mask(nx, ny, [(0, 40, 0, 24), (70, 128, 30, 64)]),
             scenes.rect_mask(nx, ny, [(0, 128, 0, 24), (70, 128, 30, 64)])]
    for q, mask in enumerate(masks):
        for d in vols:
            d.set_active_columns(mask)
            if q == 0:
                d.set_free_surface(scenes.bumps_in(nx, ny, mask, [(20.0, 12.0), (90.0, 45.0)]), REST)
        for s in range(6):
            a, b = (d.step_surface_mobile(DT_US, 20_000) for d in vols)
            assert a.iterations == b.iterations and not a.degraded, s
        for x, y, name in zip(fields(vols[0]), fields(vols[1]), NAMES):
            assert_bits(x, y, name)
