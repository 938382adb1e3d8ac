"""CUDA path vs the CPU oracle, through the C ABI (GPU only).

Integer stages (tile counts, pair order, tile ranges, densify masks) must match
bit-exactly when the oracle is fed the GPU's own float inputs (the reference keeps
train_project and train_emit consistent the same way: train_common.glsl:163-168).
Float stages: projection within 1e-5 relative; rendered colour within 1e-4 max abs on
pixels whose contributor count agrees (a count can differ only where a float lands within
an ulp of the 1/255 alpha or 1e-4 transmittance cut, and such pixels must stay rare);
gradients within 1e-3 relative L2 per parameter group; FP64 finite differences with the
reference's own rule (|err| <= 5% |fd| + 2e-6, at most 1/20 off per group).
"""
import numpy as np
import pytest

import oracle as O
from gs_b200 import frame as F
from gs_b200 import scenes as S
from helpers import GROUPS, fd_check, frame_for, rel_l2

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    from gs_b200.cuda import Context

    c = Context(0)
    yield c
    c.close()


def small_view():
    """20k gaussians, SH 0, one 360x640 view at (0, 0, 3), f = 500; target rendered from an
    independent seed-1 set (the plain single-view configuration)."""
    scene = S.make_scene(20000, 0, 0, radius=1.0, log_scale_mu=-4.0, log_scale_sigma=0.5)
    truth = S.make_scene(20000, 1, 0, radius=1.0, log_scale_mu=-4.0, log_scale_sigma=0.5)
    cam = S.front_camera(360, 640, 500.0)
    opt = F.frozen_options(0, False)
    opt.lambda_dssim, opt.lambda_dssim_end = 0.2, -1.0
    fr_t = frame_for(truth, cam, opt, (0, 0, 0), ssim=False)
    rt = O.forward_view(fr_t, truth.params, truth.sh, np.zeros((640, 360, 4), np.uint8), ssim=False, backward=False)
    target = rt.image.view(np.uint8).reshape(640, 360, 4).copy()
    target[..., 3] = 255
    return scene, cam, opt, target


def gpu_step(ctx, scene, frames, targets, train=True, capacity=None):
    ctx.model_init(scene.params, scene.sh, capacity)
    ctx.set_views(frames, targets)
    return ctx.step(train)


def test_projection_and_pairs_match_oracle(ctx):
    scene, cam, opt, target = small_view()
    fr = frame_for(scene, cam, opt, (0, 0, 0))
    res = gpu_step(ctx, scene, [fr], [target], train=False)
    assert res.overflow == 0 and res.tile_mismatch == 0
    proj = ctx.snapshot("projected")
    tiles = ctx.snapshot("tiles")
    keys = ctx.snapshot("depth_key")
    ref = O.forward_view(fr, scene.params, scene.sh, target, ssim=False, backward=False)
    # Projection floats (oracle's own projection) within 1e-5 relative.
    both = (tiles > 0) & (ref.tiles > 0)
    assert both.sum() > 0.99 * (ref.tiles > 0).sum()
    for cols in ([0, 1], [2, 3], [4, 5, 6], [8, 9, 10]):
        a, b = proj[both][:, cols].astype(np.float64), ref.projected[both][:, cols].astype(np.float64)
        assert np.abs(a - b).max() <= 1e-5 * np.abs(b).max() + 1e-6, cols
    # Tile counts: the oracle's walk over the GPU's stored records gives the same counts.
    counts = np.zeros_like(tiles)
    O.lib().gso_footprint_counts(fr.ctypes.data, np.ascontiguousarray(proj), scene.count, counts)
    np.testing.assert_array_equal(counts, tiles)
    # Depth keys from the GPU's depth: within one quantisation step of the oracle's formula.
    z = proj[:, 2].astype(np.float32)
    want = np.where(tiles > 0, (np.clip(np.log2(z / np.float32(0.02)) / np.float32(15.6096404744), 0, 1)
                                * np.float32(65535.0)).astype(np.uint32), 0xFFFF)
    assert np.abs(keys.astype(np.int64) - want.astype(np.int64)).max() <= 1
    # Pairs, order and ranges bit-exact given the GPU's projection and keys.
    r = O.forward_view(fr, scene.params, scene.sh, target, ssim=False, backward=False, projected=proj,
                       depth_keys=keys)
    assert res.pairs[0] == r.pairs
    np.testing.assert_array_equal(ctx.snapshot("pair_tile"), r.pair_tile[: r.pairs])
    np.testing.assert_array_equal(ctx.snapshot("pair_gaussian"), r.pair_gaussian[: r.pairs])
    np.testing.assert_array_equal(ctx.snapshot("render_order"), r.render_order[: r.pairs])
    np.testing.assert_array_equal(ctx.snapshot("offsets")[tiles > 0], r.offsets[tiles > 0])
    ntiles = 23 * 40
    np.testing.assert_array_equal(ctx.snapshot("ranges").reshape(-1), r.ranges[: 2 * ntiles])


def _stage_oracle(ctx, fr, scene, target, ssim=True):
    """The oracle's forward/loss/backward fed the GPU's projection and depth keys."""
    proj = ctx.snapshot("projected")
    keys = ctx.snapshot("depth_key")
    return O.forward_view(fr, scene.params, scene.sh, target, ssim=ssim, backward=True, projected=proj,
                          depth_keys=keys)


@pytest.mark.parametrize("backward_pixels", [4, 8])
def test_forward_loss_backward_match_oracle(ctx, backward_pixels):
    """Backward at 4 pixels per thread (two warps per tile) and at 8 (one warp per tile)."""
    scene, cam, opt, target = small_view()
    fr = frame_for(scene, cam, opt, (0.1, 0.2, 0.3))
    ctx.set_tuning(backward_pixels=backward_pixels)
    try:
        res = gpu_step(ctx, scene, [fr], [target], train=True)
    finally:
        ctx.set_tuning(backward_pixels=4)
    r = _stage_oracle(ctx, fr, scene, target)
    count = ctx.snapshot("pixel_count")
    same = count == r.pixel_count
    assert same.mean() > 0.9995, same.mean()
    out = ctx.snapshot("pixel_out")
    ref_out = r.ssim_input[:, :3]
    assert np.abs(out[same, :3] - ref_out[same]).max() <= 1e-4
    pg = ctx.snapshot("pixel_grad")
    assert np.abs(pg[same, 3] - r.pixel_grad[same, 3]).max() <= 1e-5
    # dL/dC (L1 + SSIM parts) per pixel.
    assert rel_l2(pg[same, :3], r.pixel_grad[same, :3]) < 1e-3
    # Loss sums per view.
    sums = np.array(res.losses[0][:8])
    for k in (0, 1, 2, 3, 4, 5):
        assert abs(sums[k] - r.sums[k]) <= 1e-4 * abs(r.sums[k]) + 1e-6, k
    # Per-pair gradients (pre-sort order) vs the oracle's back-to-front formulation.
    pgr = ctx.snapshot("pair_grads")
    ref_pg = r.pair_grads[: r.pairs]
    for name, cols in {"mean2d": [0, 1], "conic": [2, 3, 4], "opacity": [5], "colour": [6, 7, 8],
                       "abs_mean": [9, 10]}.items():
        assert rel_l2(pgr[:, cols], ref_pg[:, cols]) < 1e-3, name


def test_gradients_end_to_end_match_oracle(ctx):
    """First-step gradients (m / (1 - beta1)) of a plain step vs the oracle's own full step."""
    scene, cam, opt, target = small_view()
    fr = frame_for(scene, cam, opt, (0.1, 0.2, 0.3))
    gpu_step(ctx, scene, [fr], [target], train=True)
    g16, gsh = ctx.first_step_gradients()
    model = O.Model.create(scene.params, scene.sh)
    _, ref16, _, _ = O.train_step(model, [fr], [target])
    for name, cols in GROUPS.items():
        assert rel_l2(g16[:, cols], ref16[:, cols]) < 1e-3, name
    params, _ = ctx.export()
    np.testing.assert_array_equal(params, scene.params)  # learning rates are zero


@pytest.mark.parametrize("masked,lam", [(False, 0.2), (True, 0.2), (True, 0.0), (False, 1.0)])
def test_gradients_against_fd(ctx, masked, lam):
    """test_gradients (test_trainer.cpp:28-54) on the GPU path."""
    ds = S.make_test_dataset(64, 48, 1, masked, 3)
    scene = S.make_test_scene(10, 2, 11)
    cam = ds.camera(0)
    opt = F.frozen_options(2, masked)
    opt.lambda_dssim, opt.lambda_dssim_end = lam, -1.0
    bg = (0.2, 0.5, 0.7)
    fr = frame_for(scene, cam, opt, bg, masked=masked, ssim=lam > 0)
    res = gpu_step(ctx, scene, [fr], [ds.rgba[0]], train=True)
    ref_loss, ref_img = O.reference_loss(cam.as_dict(), 64, 48, scene.params.astype(np.float64),
                                         scene.sh.astype(np.float64), 2, ds.rgba[0], bg, masked, lam,
                                         want_image=True)
    img = ctx.snapshot("image").view(np.uint8).reshape(-1, 4)[:, :3] / 255.0
    assert np.abs(img - np.clip(ref_img, 0, 1)).max() < 2.5 / 255.0
    s = res.losses[0]
    loss = ((1 - lam) * s[3] + lam * (s[5] - s[4])) / (3.0 * 64 * 48)
    assert abs(loss - ref_loss) < 1e-4
    g16, gsh = ctx.first_step_gradients()
    report = fd_check(scene, cam, ds.rgba[0], g16, gsh, bg, masked, lam)
    for name, g in report.items():
        assert g["bad"] <= g["checked"] // 20, (name, g)


def test_adjoint_sh3_against_oracle_and_fd(ctx):
    """512 gaussians with overlapping footprints (log-scales N(-2.5, 0.3)), SH degree 3,
    one 128x128 view, f = 200: per-group relative L2 vs the oracle's analytic gradients,
    and FP64 central differences (h = 1e-4) on a sample of parameters."""
    scene = S.make_scene(512, 7, 3, radius=1.0, log_scale_mu=-2.5, log_scale_sigma=0.3)
    cam = S.front_camera(128, 128, 200.0)
    rng = np.random.default_rng(3)
    target = rng.integers(0, 256, size=(128, 128, 4), dtype=np.uint8)
    target[..., 3] = 255
    opt = F.frozen_options(3, False)
    opt.lambda_dssim, opt.lambda_dssim_end = 0.2, -1.0
    bg = (0.0, 0.0, 0.0)
    fr = frame_for(scene, cam, opt, bg)
    gpu_step(ctx, scene, [fr], [target], train=True)
    g16, gsh = ctx.first_step_gradients()
    model = O.Model.create(scene.params, scene.sh)
    _, ref16, refsh, _ = O.train_step(model, [fr], [target])
    for name, cols in GROUPS.items():
        assert rel_l2(g16[:, cols], ref16[:, cols]) < 1e-3, name
    assert rel_l2(gsh, refsh) < 1e-3
    sample = [(int(i), int(off)) for i, off in zip(rng.integers(0, 512, 120),
                                                    rng.choice([0, 1, 2, 3, 4, 5, 6, 8, 9, 10, 11, 12, 13, 14, -1,
                                                                -7, -20, -44], 120))]
    report = fd_check(scene, cam, target, g16, gsh, bg, False, 0.2, eps=1e-4, params=sample, skip_crossings=True)
    checked = sum(g["checked"] for g in report.values())
    assert checked >= 40, report
    for name, g in report.items():
        assert g["bad"] <= max(1, g["checked"] // 20), (name, g)


@pytest.mark.parametrize("backward_pixels", [4, 8])
def test_deterministic_mode_is_bit_stable(ctx, backward_pixels):
    scene, cam, opt, target = small_view()
    fr = frame_for(scene, cam, opt, (0.1, 0.2, 0.3))
    ctx.set_tuning(backward_pixels=backward_pixels)
    try:
        gpu_step(ctx, scene, [fr], [target])
        a = ctx.moments()
        pa = ctx.snapshot("pair_grads")
        gpu_step(ctx, scene, [fr], [target])
        b = ctx.moments()
        pb = ctx.snapshot("pair_grads")
    finally:
        ctx.set_tuning(backward_pixels=4)
    np.testing.assert_array_equal(a["m"], b["m"])
    np.testing.assert_array_equal(pa, pb)


def test_pair_overflow_retry(ctx):
    """test_pair_overflow_retry (test_trainer.cpp:832-853): a step whose pairs overflow the
    first guess leaves the model alone, grows the buffers and reruns bit-identically."""
    ds = S.make_test_dataset(64, 48, 1, False, 41)
    scene = S.make_test_scene(300, 1, 43)
    scene.params[:, 4:7] += 1.5
    opt = F.frozen_options(1, False)
    bg = (0.1, 0.1, 0.1)
    fr = frame_for(scene, ds.camera(0), opt, bg)
    from gs_b200.cuda import Context

    with Context(0) as small:
        small.set_tuning(min_pair_capacity=16, initial_pairs=16)
        res_small = gpu_step(small, scene, [fr], [ds.rgba[0]])
        g_small = small.first_step_gradients()[0]
    res = gpu_step(ctx, scene, [fr], [ds.rgba[0]])
    g = ctx.first_step_gradients()[0]
    assert res_small.retries >= 1 and res_small.overflow == 0
    assert res_small.pairs[0] == res.pairs[0] > 300 * 4 * 2
    np.testing.assert_array_equal(g_small, g)


def test_overflow_without_retry_leaves_model(ctx):
    ds = S.make_test_dataset(64, 48, 1, False, 41)
    scene = S.make_test_scene(300, 1, 43)
    scene.params[:, 4:7] += 1.5
    opt = F.scaled_options(100)
    opt.sh_degree = 1
    fr = frame_for(scene, ds.camera(0), opt, (0.1, 0.1, 0.1))
    from gs_b200.cuda import Context

    with Context(0) as small:
        small.set_tuning(min_pair_capacity=16, initial_pairs=16, retry=0)
        res = gpu_step(small, scene, [fr], [ds.rgba[0]])
        params, _ = small.export()
        m = small.moments()["m"]
    assert res.overflow == 1
    np.testing.assert_array_equal(params, scene.params)
    assert not m.any()


def test_batched_views_match_summed_oracle(ctx):
    """Views of uneven resolution in one step: per-view losses equal the single-view ones and
    the gradient is the sum of the per-view gradients (one Adam step)."""
    scene = S.make_scene(3000, 4, 1, radius=1.0, log_scale_mu=-3.5, log_scale_sigma=0.4)
    cams = [S.orbit_cameras(5, 3.0, 0.5, 96, 64, 90.0)[1], S.orbit_cameras(5, 3.0, 0.5, 160, 120, 150.0)[3],
            S.front_camera(80, 48, 70.0)]
    rng = np.random.default_rng(9)
    targets = []
    for c in cams:
        t = rng.integers(0, 256, size=(c.height, c.width, 4), dtype=np.uint8)
        t[..., 3] = 255
        targets.append(t)
    opt = F.frozen_options(1, False)
    frames = [frame_for(scene, c, opt, (0.2, 0.1, 0.0)) for c in cams]
    res = gpu_step(ctx, scene, frames, targets)
    g16, gsh = ctx.first_step_gradients()
    model = O.Model.create(scene.params, scene.sh)
    results, ref16, refsh, _ = O.train_step(model, frames, targets)
    for name, cols in GROUPS.items():
        assert rel_l2(g16[:, cols], ref16[:, cols]) < 1e-3, name
    assert rel_l2(gsh, refsh) < 1e-3
    for v, r in enumerate(results):
        assert res.pairs[v] == r.pairs
        for k in (0, 1, 2):
            assert abs(res.losses[v][k] - r.sums[k]) <= 1e-4 * abs(r.sums[k]) + 1e-6


def test_densify_masks_match_oracle(ctx):
    """Densify after a training step: spawn masks bit-exact, placement and counters equal
    to the oracle's (deterministic compaction) applied to the same state."""
    ds = S.make_test_dataset(64, 48, 1, False, 5)
    scene = S.make_test_scene(200, 1, 3)
    scene.params[::7, 3] = -6.0  # some below the prune opacity
    scene.params[1::3, 4:7] = np.log(0.02)  # some small enough to clone (percent_dense x extent = 0.033)
    opt = F.scaled_options(100)
    opt.sh_degree = 1
    opt.densify_grad_threshold = 2e-5
    fr = frame_for(scene, ds.camera(0), opt, (0, 0, 0))
    gpu_step(ctx, scene, [fr], [ds.rgba[0]], capacity=320)
    params, sh = ctx.export()
    mo = ctx.moments()
    stats = ctx.snapshot("stats")
    model = O.Model.create(params, sh, capacity=320)
    model.m[:200], model.v[:200], model.m_sh[:200], model.v_sh[:200] = mo["m"], mo["v"], mo["m_sh"], mo["v_sh"]
    model.stats[:200] = stats
    counters, spawn = O.densify(model, fr, 320)
    got = ctx.densify(fr)
    np.testing.assert_array_equal(ctx.snapshot("spawn"), spawn)
    assert list(got[:3]) == list(counters[:3])
    p2, s2 = ctx.export()
    n = p2.shape[0]
    assert (spawn == 1).any() and (spawn == 2).any() and counters[2] > 0
    np.testing.assert_allclose(p2, model.params[:n], rtol=1e-5, atol=1e-6)
    np.testing.assert_allclose(s2, model.sh[:n], rtol=0, atol=0)


def test_render_matches_forward(ctx):
    """gs_render's RGBA8 image against the oracle's forward on the GPU's projection: within
    one RGBA8 step (the colour is within 1e-4, the alpha within 1e-5, before rounding) on
    every pixel whose contributor count agrees, and those are at least 99.95% of the image."""
    scene, cam, opt, target = small_view()
    fr = frame_for(scene, cam, opt, (0, 0, 0), ssim=False)
    ctx.model_init(scene.params, scene.sh)
    img = ctx.render(fr)
    count = ctx.snapshot("pixel_count")
    ref = O.forward_view(fr, scene.params, scene.sh, target, ssim=False, backward=False,
                         projected=ctx.snapshot("projected"), depth_keys=ctx.snapshot("depth_key"))
    diff = np.abs(img.reshape(-1, 4).astype(int) - ref.image.view(np.uint8).reshape(-1, 4).astype(int))
    same = count == ref.pixel_count
    assert same.mean() > 0.9995
    assert diff[same].max() <= 1
    assert (ref.image.view(np.uint8).reshape(-1, 4)[:, 3] > 0).mean() > 0.5  # the view is mostly covered


def _mixed_views(scene, opt, seed, step=0):
    """Four views of different resolution on an orbit, noise targets."""
    rng = np.random.default_rng(seed)
    sizes = [(96, 64, 90.0), (160, 120, 150.0), (80, 48, 70.0), (64, 64, 60.0)]
    frames, targets = [], []
    for k, (w, h, f) in enumerate(sizes):
        cam = S.orbit_cameras(7, 3.0, 0.5, w, h, f)[(seed + 2 * k) % 7]
        frames.append(frame_for(scene, cam, opt, (0.2, 0.1, 0.0), step=step))
        t = rng.integers(0, 256, size=(h, w, 4), dtype=np.uint8)
        t[..., 3] = 255
        targets.append(t)
    return frames, targets


def test_graph_replay_matches_direct_steps(ctx):
    """Training through the captured CUDA graph equals stepping directly, bit for bit, while
    the three views of each step change cameras and resolutions (the graph is replayed with
    a new step table, not recaptured, once the buffers have grown)."""
    from gs_b200.cuda import Context

    scene = S.make_scene(3000, 4, 1, radius=1.0, log_scale_mu=-3.5, log_scale_sigma=0.4)
    opt = F.scaled_options(100)
    opt.sh_degree = 1
    runs = []
    for graph in (0, 1):
        with Context(0) as c:
            c.set_tuning(graph=graph)
            c.model_init(scene.params, scene.sh)
            for step in range(6):
                frames, targets = _mixed_views(scene, opt, step, step)
                pick = [(step + k) % 4 for k in range(3)]
                c.set_views([frames[k] for k in pick], [targets[k] for k in pick])
                r = c.step(True)
                assert r.overflow == 0
            runs.append((c.export(), c.moments()["m"]))
    (pa, sa), ma = runs[0]
    (pb, sb), mb = runs[1]
    np.testing.assert_array_equal(pa, pb)
    np.testing.assert_array_equal(sa, sb)
    np.testing.assert_array_equal(ma, mb)


def test_dataset_targets_match_host_targets(ctx):
    scene = S.make_scene(3000, 5, 1, radius=1.0, log_scale_mu=-3.5, log_scale_sigma=0.4)
    opt = F.frozen_options(1, False)
    frames, targets = _mixed_views(scene, opt, 3)
    ctx.model_init(scene.params, scene.sh)
    ctx.set_views(frames, targets)
    ra = ctx.step(True)
    ga = ctx.first_step_gradients()[0]
    ctx.model_init(scene.params, scene.sh)
    ctx.set_dataset(targets[::-1])
    ctx.set_views_dataset(frames, [3, 2, 1, 0])
    rb = ctx.step(True)
    gb = ctx.first_step_gradients()[0]
    np.testing.assert_array_equal(ga, gb)
    for v in range(4):
        assert ra.pairs[v] == rb.pairs[v]
        assert list(ra.losses[v]) == list(rb.losses[v])
