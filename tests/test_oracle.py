"""Pins the CPU oracle to the reference's own known-answer tests (CPU only).

The reference ships no golden vectors; these are its checks restated:
- SSIM window: the shaders' hard-coded weights (train_common.glsl:61-62) against the
  normalised Gaussian the CPU self-test builds (train_selftest.cpp:176-181).
- test_gradients (test_trainer.cpp:28-54, train_selftest.cpp:356-486): forward image within
  2.5/255 and loss within 1e-4 of the FP64 reference; every parameter group's analytic
  gradient against FP64 central differences (|err| <= 5% |fd| + 2e-6, at most 1/20 off).
- test_pair_order (test_trainer.cpp:197-233), test_footprint (test_trainer.cpp:235-289),
  test_scan_and_densify (test_trainer.cpp:866-888), test_radix_sort (test_engine.cpp:27-68).
"""
import numpy as np
import pytest

import oracle as O
from gs_b200 import frame as F
from gs_b200 import scenes as S
from helpers import fd_check, frame_for, image_f


def test_ssim_window_matches_gaussian():
    k = np.arange(-5, 6, dtype=np.float64)
    w = np.exp(-(k * k) / (2.0 * 1.5 * 1.5))
    w /= w.sum()
    # 9 significant digits stored as float32: equal to float32 precision.
    np.testing.assert_allclose(O.ssim_window().astype(np.float64), w, rtol=1e-7, atol=0)


def test_depth_order_is_stable_sort():
    rng = np.random.default_rng(5)
    for n, mask in [(1, 0xFFFF), (1000, 0xF), (4096, 0xFFFF), (100000, 0xFF)]:
        keys = (rng.integers(0, 1 << 16, n) & mask).astype(np.uint32)
        order = np.zeros(n, np.uint32)
        O.lib().gso_depth_order(keys, n, order)
        np.testing.assert_array_equal(order, np.argsort(keys, kind="stable"))


def _loss_from_sums(sums, lam, W, H):
    """Trainer::set_view_stats (trainer.cpp:797-805)."""
    n = 3.0 * W * H
    return ((1.0 - lam) * sums[3] + lam * (sums[5] - sums[4])) / n


@pytest.mark.parametrize("masked,lam", [(False, 0.2), (True, 0.2), (True, 0.0), (False, 1.0)])
def test_gradients_against_fd(masked, lam):
    ds = S.make_test_dataset(64, 48, 1, masked, 3)
    scene = S.make_test_scene(10, 2, 11)
    cam = ds.camera(0)
    opt = F.frozen_options(2, masked)
    opt.lambda_dssim = lam
    opt.lambda_dssim_end = -1.0
    bg = (0.2, 0.5, 0.7)
    fr = frame_for(scene, cam, opt, bg, masked=masked, ssim=lam > 0)
    model = O.Model.create(scene.params, scene.sh)
    results, g16, gsh, _ = O.train_step(model, [fr], [ds.rgba[0]], ssim=lam > 0)
    r = results[0]
    ref_loss, ref_img = O.reference_loss(cam.as_dict(), 64, 48, scene.params.astype(np.float64),
                                         scene.sh.astype(np.float64), 2, ds.rgba[0], bg, masked, lam,
                                         want_image=True)
    img = image_f(r.image)[:, :3]
    assert np.abs(img - np.clip(ref_img, 0, 1)).max() < 2.5 / 255.0
    assert abs(_loss_from_sums(r.sums, lam, 64, 48) - ref_loss) < 1e-4
    report = fd_check(scene, cam, ds.rgba[0], g16, gsh, bg, masked, lam)
    assert set(report) == {"position", "opacity", "log_scale", "rotation", "sh_dc", "sh_rest"}
    for name, g in report.items():
        assert g["bad"] <= g["checked"] // 20, (name, g)
    # Forward bookkeeping: covered pixels have a count (test_trainer.cpp:45-46).
    covered = r.pixel_grad[:, 3] < 0.999
    assert covered.any() and (r.pixel_count[covered] > 0).all()


def test_pair_order():
    ds = S.make_test_dataset(64, 48, 1, False, 31)
    scene = S.make_test_scene(400, 1, 37)
    fr = frame_for(scene, ds.camera(0), F.frozen_options(1, False), (0, 0, 0), ssim=False)
    r = O.forward_view(fr, scene.params, scene.sh, ds.rgba[0], ssim=False, backward=False)
    gauss = r.pair_gaussian[: r.pairs]
    want = np.lexsort((gauss, r.depth_keys[gauss], r.pair_tile[: r.pairs]))
    got = r.render_order[: r.pairs]
    assert r.pairs > 500 and len(np.unique(r.depth_keys[r.tiles > 0])) > 100
    np.testing.assert_array_equal(r.pair_tile[got], r.pair_tile[want])
    np.testing.assert_array_equal(gauss[got], gauss[want])


def test_footprint():
    ds = S.make_test_dataset(64, 48, 1, False, 11)
    scene = S.make_test_scene(200, 1, 13)
    scene.params[::2, 4] += 1.5
    fr = frame_for(scene, ds.camera(0), F.frozen_options(1, False), (0, 0, 0), ssim=False)
    r = O.forward_view(fr, scene.params, scene.sh, ds.rgba[0], ssim=False, backward=False)
    tx, ty = 4, 3
    needed = emitted = missing = duplicate = 0
    ys, xs = np.mgrid[0:48, 0:64]
    for i in np.nonzero(r.tiles)[0]:
        q = r.projected[i]
        t = 2.0 * np.log(255.0 * float(q[3]))
        dx, dy = float(q[0]) - (xs + 0.5), float(q[1]) - (ys + 0.5)
        inside = q[4] * dx * dx + 2.0 * q[5] * dx * dy + q[6] * dy * dy <= t
        want = np.zeros(tx * ty, int)
        want[np.unique((ys[inside] // 16) * tx + xs[inside] // 16)] = 1
        tiles = r.pair_tile[r.offsets[i]: r.offsets[i] + r.tiles[i]]
        got = np.bincount(tiles, minlength=tx * ty)
        duplicate += int((got > 1).sum())
        missing += int(((want > 0) & (got == 0)).sum())
        needed += int(want.sum())
        emitted += int(r.tiles[i])
    assert missing == 0 and duplicate == 0
    assert emitted <= needed + needed // 20
    assert r.mismatch == 0


def test_scan_and_densify():
    ds = S.make_test_dataset(64, 48, 1, False, 5)
    scene = S.make_test_scene(40, 0, 3)
    opt = F.frozen_options(0, False)
    opt.densify_grad_threshold = 0.0
    fr = frame_for(scene, ds.camera(0), opt, (0, 0, 0), ssim=True)
    model = O.Model.create(scene.params, scene.sh, capacity=60)
    O.train_step(model, [fr], [ds.rgba[0]])
    counters, spawn = O.densify(model, fr, 60)
    free, spawned, pruned = int(counters[0]), int(counters[1]), int(counters[2])
    placed = min(spawned, free + (60 - 40))
    slots = 40 + max(0, placed - free)
    alive = 40 - pruned + placed
    assert slots == 60 and alive == 60
    assert np.isfinite(model.params[:60, :3]).all()
    assert set(np.unique(spawn)) <= {0, 1, 2}


def test_frozen_step_keeps_parameters():
    ds = S.make_test_dataset(64, 48, 1, False, 7)
    scene = S.make_test_scene(30, 1, 9)
    opt = F.frozen_options(1, False)
    fr = frame_for(scene, ds.camera(0), opt, (0.1, 0.2, 0.3))
    model = O.Model.create(scene.params, scene.sh)
    _, g16, gsh, _ = O.train_step(model, [fr], [ds.rgba[0]])
    np.testing.assert_array_equal(model.params, scene.params)
    np.testing.assert_allclose(model.m / np.float32(0.1), g16, rtol=1e-6, atol=1e-12)
    np.testing.assert_allclose(model.m_sh / np.float32(0.1), gsh, rtol=1e-6, atol=1e-12)
