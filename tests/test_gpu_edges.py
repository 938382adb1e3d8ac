"""Edge cases and full-size properties of the CUDA path (GPU only).

Edge cases the reference's own tests and the format allow: an empty model, a model whose
every gaussian is culled, sixteen views of ragged sizes in one step (the most a step takes),
and one gaussian covering every tile. Then the full benchmark size (1M gaussians SH3, 8 views
of 1080x1920), where the oracle would take minutes, checked through size-independent
properties: the pair list is sorted by tile and stable (depth order within a tile), the tile
ranges and per-view pair counts add up, every pixel's contributor count lies within its
tile's list, a batched step's per-view losses equal the single views', and two runs agree
bit for bit.
"""
import numpy as np
import pytest

import oracle as O
from gs_b200 import frame as F
from gs_b200 import scenes as S
from helpers import GROUPS, frame_for, rel_l2

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    from gs_b200.cuda import Context

    c = Context(0)
    yield c
    c.close()


def background_losses(bg, target):
    """The loss sums of a render that is the background everywhere (no coverage)."""
    t = target.reshape(-1, 4)[:, :3].astype(np.float64) / 255.0
    e = np.asarray(bg, np.float64)[None, :] - t
    return np.abs(e).sum(), (e * e).sum()


def test_empty_model(ctx):
    scene = S.make_test_scene(10, 1, 3)
    empty = S.Scene(scene.params[:0].copy(), scene.sh[:0].copy(), 1)
    ds = S.make_test_dataset(40, 24, 1, False, 2)
    bg = (0.25, 0.5, 0.75)
    fr = frame_for(empty, ds.camera(0), F.frozen_options(1, False), bg)
    ctx.model_init(empty.params, empty.sh, capacity=16)
    ctx.set_views([fr], [ds.rgba[0]])
    res = ctx.step(True)
    assert res.pairs[0] == 0 and res.overflow == 0
    img = ctx.snapshot("image").view(np.uint8).reshape(-1, 4)
    assert (img[:, :3] == np.round(np.array(bg) * 255).astype(np.uint8)).all() and (img[:, 3] == 0).all()
    l1, l2 = background_losses(bg, ds.rgba[0])
    assert abs(res.losses[0][0] - l1) <= 1e-5 * l1 and abs(res.losses[0][1] - l2) <= 1e-5 * l2
    np.testing.assert_array_equal(ctx.render(fr).reshape(-1, 4)[:, :3], img[:, :3])


def test_every_gaussian_culled(ctx):
    """Behind the camera, below the opacity cut or with zero alive flag: no pairs, the
    background everywhere and no gradient."""
    ds = S.make_test_dataset(48, 32, 1, False, 4)
    scene = S.make_test_scene(300, 1, 5)
    cam = ds.camera(0)
    p = scene.params
    third = len(p) // 3
    # Behind: mirror the first third through the camera centre.
    p[:third, 0:3] = 2.0 * np.asarray(cam.position, np.float32) - p[:third, 0:3]
    p[third:2 * third, 3] = -20.0  # opacity below 1/255
    p[2 * third:, 7] = 0.0  # free slots
    bg = (0.1, 0.2, 0.3)
    fr = frame_for(scene, cam, F.frozen_options(1, False), bg)
    ctx.model_init(scene.params, scene.sh)
    ctx.set_views([fr], [ds.rgba[0]])
    res = ctx.step(True)
    assert res.pairs[0] == 0
    assert not ctx.snapshot("tiles").any()
    l1, _ = background_losses(bg, ds.rgba[0])
    assert abs(res.losses[0][0] - l1) <= 1e-5 * l1
    m = ctx.moments()
    assert not m["m"].any() and not m["m_sh"].any()


@pytest.mark.parametrize("tuning", [dict(), dict(deterministic=0), dict(deterministic=0, forward_pixels=1, backward_pixels=2),
                                    dict(deterministic=0, forward_pixels=4, backward_pixels=8),
                                    dict(deterministic=1, backward_pixels=8)])
def test_sixteen_ragged_views_match_oracle(ctx, tuning):
    """GS_MAX_VIEWS views of different sizes (none a multiple of 16) in one step: per-view
    pair counts and losses, and the summed gradient, against the oracle; under the default
    tuning, the fast mode's independent-warp kernels at each warp layout, and one warp per
    tile in both modes (work items of ragged edge tiles, views of uneven size in one queue)."""
    scene = S.make_scene(2000, 6, 1, radius=1.0, log_scale_mu=-3.5, log_scale_sigma=0.4)
    rng = np.random.default_rng(13)
    frames, targets = [], []
    opt = F.frozen_options(1, False)
    for v in range(16):
        w, h = int(rng.integers(17, 90)), int(rng.integers(9, 70))
        cam = S.orbit_cameras(16, 3.0, 0.5, w, h, 0.9 * w)[v]
        frames.append(frame_for(scene, cam, opt, (0.2, 0.1, 0.0)))
        t = rng.integers(0, 256, size=(h, w, 4), dtype=np.uint8)
        t[..., 3] = 255
        targets.append(t)
    default = ctx.tuning()
    ctx.set_tuning(**tuning)
    try:
        ctx.model_init(scene.params, scene.sh)
        ctx.set_views(frames, targets)
        res = ctx.step(True)
        g16, gsh = ctx.first_step_gradients()
    finally:
        ctx.set_tuning(**{k: getattr(default, k) for k in ("deterministic", "forward_pixels", "backward_pixels")})
    assert res.n_views == 16
    model = O.Model.create(scene.params, scene.sh)
    results, ref16, refsh, _ = O.train_step(model, frames, targets)
    for v, r in enumerate(results):
        assert res.pairs[v] == r.pairs, v
        for k in (0, 1, 2):
            assert abs(res.losses[v][k] - r.sums[k]) <= 1e-4 * abs(r.sums[k]) + 1e-6, (v, k)
    for name, cols in GROUPS.items():
        assert rel_l2(g16[:, cols], ref16[:, cols]) < 1e-3, name
    assert rel_l2(gsh, refsh) < 1e-3


@pytest.mark.parametrize("width,height,focal", [(100, 70, 80.0), (1200, 64, 400.0)])
def test_one_gaussian_covers_every_tile(ctx, width, height, focal):
    """A footprint larger than the view: more than 6 tile rows (100x70), or rows of 75
    tiles (1200x64), both beyond what the projection packs for the pair emission, which
    then walks the rows again."""
    scene = S.make_test_scene(1, 0, 3)
    scene.params[0, 0:3] = 0.0
    scene.params[0, 4:7] = np.log(2.0)  # far wider than the view
    scene.params[0, 3] = 2.0
    cam = S.front_camera(width, height, focal)
    opt = F.frozen_options(0, False)
    fr = frame_for(scene, cam, opt, (0.0, 0.0, 0.0))
    target = np.full((height, width, 4), 200, np.uint8)
    ctx.model_init(scene.params, scene.sh)
    ctx.set_views([fr], [target])
    res = ctx.step(True)
    tiles = ((width + 15) // 16) * ((height + 15) // 16)
    assert res.pairs[0] == tiles and ctx.snapshot("tiles")[0] == tiles
    r = O.forward_view(fr, scene.params, scene.sh, target, ssim=True, backward=False,
                       projected=ctx.snapshot("projected"), depth_keys=ctx.snapshot("depth_key"))
    diff = np.abs(ctx.snapshot("image").view(np.uint8).reshape(-1, 4).astype(int)
                  - r.image.view(np.uint8).reshape(-1, 4).astype(int))
    assert diff.max() <= 1


@pytest.fixture(scope="module")
def full_size():
    """The benchmark's workload: 1M gaussians SH3 (radius-2 ball, log-scales N(-5, 0.5)),
    8 orbit views of 1080x1920 at f = 1400, noise targets."""
    scene = S.make_scene(1_000_000, 0, 3, radius=2.0, log_scale_mu=-5.0, log_scale_sigma=0.5)
    cams = S.orbit_cameras(8, 3.0, 0.5, 1080, 1920, 1400.0)
    opt = F.TrainOptions(iterations=30000, sh_degree=3, sh_degree_interval=0, masked=False,
                         random_background=False, lambda_dssim=0.2, lambda_dssim_end=-1.0)
    frames = [frame_for(scene, c, opt, (0.0, 0.0, 0.0)) for c in cams]
    rng = np.random.default_rng(21)
    targets = [rng.integers(0, 256, size=(1920, 1080, 4), dtype=np.uint8) for _ in cams]
    for t in targets:
        t[..., 3] = 255
    return scene, frames, targets


def test_full_size_pair_list_properties(ctx, full_size):
    scene, frames, targets = full_size
    ctx.model_init(scene.params, scene.sh)
    ctx.set_views(frames, targets)
    res = ctx.step(True)
    pairs = [int(res.pairs[v]) for v in range(8)]
    total = sum(pairs)
    assert res.overflow == 0 and res.tile_mismatch == 0 and total > 10_000_000
    # Each view's pairs: its gaussians' tile counts, and its tiles' ranges.
    for v in range(8):
        assert int(ctx.snapshot("tiles", v).astype(np.int64).sum()) == pairs[v]
        rg = ctx.snapshot("ranges", v).reshape(-1, 2).astype(np.int64)
        assert int((rg[:, 1] - rg[:, 0]).sum()) == pairs[v]
    # The render order: a permutation of the pairs, sorted by (view, tile), stable (the
    # pre-sort index, which is depth order, increases within a tile).
    order = ctx.snapshot("render_order", 0).astype(np.int64)
    tile = ctx.snapshot("pair_tile", 0).astype(np.int64)  # global tile: view 0's base is 0
    assert order.size == total and np.array_equal(np.sort(order), np.arange(total))
    t = tile[order]
    assert (np.diff(t) >= 0).all()
    same = np.diff(t) == 0
    assert (np.diff(order)[same] > 0).all()
    # Every pixel's last contributor lies within its tile's list (view 0).
    rg = ctx.snapshot("ranges", 0).reshape(-1, 2).astype(np.int64)
    count = ctx.snapshot("pixel_count", 0).reshape(1920, 1080).astype(np.int64)
    tiles_x = (1080 + 15) // 16
    tid = (np.arange(1920)[:, None] // 16) * tiles_x + (np.arange(1080)[None, :] // 16)
    assert (count <= (rg[tid, 1] - rg[tid, 0])).all()


def test_full_size_batched_equals_single_views_and_is_bit_stable(ctx, full_size):
    scene, frames, targets = full_size
    ctx.model_init(scene.params, scene.sh)
    ctx.set_views(frames, targets)
    a = ctx.step(True)
    ma = ctx.moments()["m"].copy()
    ctx.model_init(scene.params, scene.sh)
    ctx.set_views(frames, targets)
    b = ctx.step(True)
    np.testing.assert_array_equal(ma, ctx.moments()["m"])
    for v in range(8):
        assert list(a.losses[v]) == list(b.losses[v])
    # The forward of a view does not depend on the others in the step: the same losses alone.
    for v in (0, 5):
        ctx.model_init(scene.params, scene.sh)
        ctx.set_views([frames[v]], [targets[v]])
        s = ctx.step(False)
        assert list(s.losses[0]) == list(a.losses[v]) and s.pairs[0] == a.pairs[v]


def test_sixteen_full_views_multi_chunk_scans(ctx, full_size):
    """GS_MAX_VIEWS views of 1080x1920 over the 1M-gaussian model: 16M (view, slot) items
    and about 65M pairs, so the offset scan's tile-sum scan and the pair sort's per-digit
    tile scans each run over more than one chunk. The pair list must still be a stable
    sort by tile with consistent ranges and per-view counts, and a view's losses must not
    depend on the other views of the step."""
    scene, frames8, targets8 = full_size
    cams = S.orbit_cameras(16, 3.0, 0.5, 1080, 1920, 1400.0)
    opt = F.TrainOptions(iterations=30000, sh_degree=3, sh_degree_interval=0, masked=False,
                         random_background=False, lambda_dssim=0.2, lambda_dssim_end=-1.0)
    frames = [frame_for(scene, c, opt, (0.0, 0.0, 0.0)) for c in cams]
    targets = [targets8[v % 8] for v in range(16)]
    ctx.model_init(scene.params, scene.sh)
    ctx.set_views(frames, targets)
    res = ctx.step(False)
    pairs = [int(res.pairs[v]) for v in range(16)]
    total = sum(pairs)
    assert res.overflow == 0 and res.tile_mismatch == 0
    assert total > 9216 * 3840  # more pair-sort tiles than one k_tile_scan chunk
    for v in (0, 7, 15):
        assert int(ctx.snapshot("tiles", v).astype(np.int64).sum()) == pairs[v]
        rg = ctx.snapshot("ranges", v).reshape(-1, 2).astype(np.int64)
        assert int((rg[:, 1] - rg[:, 0]).sum()) == pairs[v]
    order = ctx.snapshot("render_order", 0).astype(np.int64)
    tile = ctx.snapshot("pair_tile", 0).astype(np.int64)
    assert order.size == total and np.array_equal(np.sort(order), np.arange(total))
    t = tile[order]
    assert (np.diff(t) >= 0).all()
    same = np.diff(t) == 0
    assert (np.diff(order)[same] > 0).all()
    for v in (3, 12):
        ctx.model_init(scene.params, scene.sh)
        ctx.set_views([frames[v]], [targets[v]])
        s = ctx.step(False)
        assert list(s.losses[0]) == list(res.losses[v]) and s.pairs[0] == res.pairs[v]
