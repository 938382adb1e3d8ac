"""Camera pose gradient and exposure-fit sums on the CUDA path (GPU only).

The pose gradient is pinned the way the reference pins it (test_pose_gradient,
test_trainer.cpp:404-460): moving the camera is moving every gaussian the other way, so
the summed pose gradient must equal what the per-gaussian gradients (themselves checked
against the oracle) imply. A shift d of the camera-space positions gives
dL/dd = W sum dL/dp; a turn w about the camera centre c gives
dL/dw = W sum((p - c) x dL/dp + tau), tau the orientation's share. SH degree 0, since the
pose gradient leaves the view-direction term out.
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


def expected_pose_gradient(scene, cam, g16):
    """The pose gradient the per-gaussian first-step gradients imply (test_trainer.cpp:427-452)."""
    p = scene.params.astype(np.float64)
    g = g16.astype(np.float64)
    sum_d = g[:, 0:3].sum(axis=0)
    rel = p[:, 0:3] - np.asarray(cam.position, np.float64)
    sum_w = np.cross(rel, g[:, 0:3]).sum(axis=0)
    q = p[:, 8:12]
    qlen = np.linalg.norm(q, axis=1, keepdims=True)
    qn = q / qlen
    w, u = qn[:, :1], qn[:, 1:]
    gw, gu = g[:, 8:9] * qlen, g[:, 9:12] * qlen
    sum_w += (0.5 * (-gw * u + w * gu + np.cross(u, gu))).sum(axis=0)
    R = np.asarray(cam.rotation, np.float64).reshape(3, 3)
    return np.concatenate([R @ sum_d, R @ sum_w])


def pose_frame(scene, cam, lam, bg=(0.2, 0.3, 0.4), flags=F.FLAG_POSE_GRAD):
    opt = F.frozen_options(0, True)
    opt.lambda_dssim, opt.lambda_dssim_end = lam, -1.0
    fr = frame_for(scene, cam, opt, bg, masked=True, ssim=lam > 0)
    fr["model"][0, 3] |= flags
    return fr


@pytest.mark.parametrize("lam", [0.0, 0.2])
def test_pose_gradient_matches_gaussian_gradients(ctx, lam):
    ds = S.make_test_dataset(64, 48, 2, True, 3)
    scene = S.make_test_scene(120, 0, 9)
    cam = ds.camera(0)
    fr = pose_frame(scene, cam, lam)
    ctx.model_init(scene.params, scene.sh)
    ctx.set_views([fr], [ds.rgba[0]])
    res = ctx.step(True)
    assert res.overflow == 0
    got = np.array(res.pose_grad[0][:])
    g16, _ = ctx.first_step_gradients()
    want = expected_pose_gradient(scene, cam, g16)
    largest = np.abs(want).max()
    assert largest > 0.0
    assert np.abs(got - want).max() <= 1e-3 * largest, (got, want)


def test_pose_gradient_zero_without_the_flag(ctx):
    ds = S.make_test_dataset(64, 48, 2, True, 3)
    scene = S.make_test_scene(120, 0, 9)
    fr = pose_frame(scene, ds.camera(0), 0.2, flags=0)
    ctx.model_init(scene.params, scene.sh)
    ctx.set_views([fr], [ds.rgba[0]])
    res = ctx.step(True)
    assert not np.any(np.array(res.pose_grad[0][:]))


def test_pose_only_step_changes_nothing(ctx):
    """GS_FLAG_POSE_ONLY (train_step.glsl:92-100, 222): the same pose gradient as a training
    step, but parameters, moments and densification statistics stay as they were."""
    ds = S.make_test_dataset(64, 48, 2, True, 3)
    scene = S.make_test_scene(120, 2, 9)
    opt = F.TrainOptions()  # non-zero learning rates
    opt.lambda_dssim, opt.lambda_dssim_end = 0.2, -1.0
    cam = ds.camera(1)
    base = frame_for(scene, cam, opt, (0.2, 0.3, 0.4), masked=True)
    train = base.copy()
    train["model"][0, 3] |= F.FLAG_POSE_GRAD
    only = base.copy()
    only["model"][0, 3] |= F.FLAG_POSE_GRAD | F.FLAG_POSE_ONLY
    ctx.model_init(scene.params, scene.sh)
    ctx.set_views([only], [ds.rgba[1]])
    r_only = ctx.step(True)
    params, sh = ctx.export()
    np.testing.assert_array_equal(params, scene.params)
    np.testing.assert_array_equal(sh, scene.sh)
    assert not np.any(ctx.snapshot("stats"))
    m = ctx.moments()
    assert not any(np.any(v) for v in m.values())
    ctx.model_init(scene.params, scene.sh)
    ctx.set_views([train], [ds.rgba[1]])
    r_train = ctx.step(True)
    np.testing.assert_array_equal(np.array(r_only.pose_grad[0][:]), np.array(r_train.pose_grad[0][:]))
    assert np.any(np.array(r_train.pose_grad[0][:]))
    params, _ = ctx.export()
    assert np.any(params != scene.params)


def test_batched_pose_gradients_equal_single_views(ctx):
    """Each view of a batched step gets its own pose gradient, bitwise the single view's."""
    ds = S.make_test_dataset(64, 48, 3, True, 3)
    scene = S.make_test_scene(120, 0, 9)
    frames = [pose_frame(scene, ds.camera(v), 0.2) for v in range(3)]
    frames[1]["model"][0, 3] &= ~np.uint32(F.FLAG_POSE_GRAD)  # the middle view does not ask
    ctx.model_init(scene.params, scene.sh)
    ctx.set_views(frames, [ds.rgba[v] for v in range(3)])
    batched = ctx.step(True)
    for v in range(3):
        ctx.model_init(scene.params, scene.sh)
        ctx.set_views([frames[v]], [ds.rgba[v]])
        single = ctx.step(True)
        np.testing.assert_array_equal(np.array(batched.pose_grad[v][:]), np.array(single.pose_grad[0][:]))
    assert not np.any(np.array(batched.pose_grad[1][:]))


def head_and_gain_frame(scene, cam, masked):
    """A frame with a head region (centre, radius 20 px, weight 3) and colour gains."""
    opt = F.frozen_options(0, masked)
    opt.lambda_dssim, opt.lambda_dssim_end = 0.2, -1.0
    fr = frame_for(scene, cam, opt, (0.0, 0.0, 0.0), masked=masked)
    fr["head"][0] = (0.45 * cam.width, 0.55 * cam.height, 20.0, 3.0)
    fr["exposure"][0, :3] = (1.0 / 0.8, 1.0 / 0.85, 1.0 / 0.9)
    return fr


@pytest.mark.parametrize("masked", [False, True])
def test_head_weight_and_exposure_match_oracle(ctx, masked):
    """Head weighting (train_forward.comp: pixel weight, head sums) and colour gains: the
    step's 16 loss and fit sums and its first-step gradients against the oracle's."""
    ds = S.make_test_dataset(128, 96, 2, masked, 3)
    scene = S.make_test_scene(300, 0, 9)
    cam = ds.camera(1)
    target = ds.rgba[1]
    fr = head_and_gain_frame(scene, cam, masked)
    ctx.model_init(scene.params, scene.sh)
    ctx.set_views([fr], [target])
    res = ctx.step(True)
    r = O.forward_view(fr, scene.params, scene.sh, target, ssim=True, backward=False,
                       projected=ctx.snapshot("projected"), depth_keys=ctx.snapshot("depth_key"))
    want = r.tile_loss.reshape(-1, 16).astype(np.float64).sum(axis=0)
    got = np.concatenate([np.array(res.losses[0][:]), np.array(res.fit[0][:])])
    assert want[7] > 0 and want[11] > 0  # head pixels and opaque fit pixels present
    for k in (0, 1, 3, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15):
        assert abs(got[k] - want[k]) <= 1e-4 * abs(want[k]) + 1e-5, (k, got[k], want[k])
    g16, _ = ctx.first_step_gradients()
    model = O.Model.create(scene.params, scene.sh)
    _, ref16, _, _ = O.train_step(model, [fr], [target])
    for name, cols in GROUPS.items():
        assert rel_l2(g16[:, cols], ref16[:, cols]) < 1e-3, name


def test_exposure_fit_sums(ctx):
    """fit (train_forward.comp:142-151): over pixels where the target is opaque (alpha >
    0.95) and the render too (T < 0.05), sums of R^2 and R P per channel and their count;
    then the pixels with any target alpha. Checked against the step's own render."""
    ds = S.make_test_dataset(128, 96, 1, False, 3)
    scene = S.make_test_scene(300, 0, 9)
    opt = F.frozen_options(0, False)
    fr = frame_for(scene, ds.camera(0), opt, (0.0, 0.0, 0.0), masked=False, ssim=False)
    ctx.model_init(scene.params, scene.sh)
    ctx.set_views([fr], [ds.rgba[0]])
    res = ctx.step(False)
    out = ctx.snapshot("pixel_out").reshape(-1, 4).astype(np.float64)  # colour over black: R
    T = ctx.snapshot("pixel_grad").reshape(-1, 4)[:, 3]
    tgt = ds.rgba[0].reshape(-1, 4)
    ta = tgt[:, 3] / 255.0
    photo = tgt[:, :3] / 255.0
    sel = (ta > 0.95) & (T < 0.05)
    assert sel.sum() > 20
    want = np.concatenate([(out[sel, :3] ** 2).sum(axis=0), [sel.sum()],
                           (out[sel, :3] * photo[sel]).sum(axis=0), [(ta > 0).sum()]])
    got = np.array(res.fit[0][:])
    np.testing.assert_allclose(got, want, rtol=1e-5)
