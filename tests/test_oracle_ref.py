"""Pins the CPU oracle to the reference's own code (CPU only).

oracle/_ref/libgs_ref.so is the reference's FP64 CPU forward + loss
(engine/src/train_selftest.cpp:27-283: `project`, `reference_ssim`, `reference_loss`),
compiled from a reference checkout by `make -C oracle ref`. These tests check:
- the oracle's restatement (gso_reference_loss, gso_reference_ssim) reproduces it bit for
  bit: loss, FP64 image and SSIM, on the reference's own test scene (masks, head weight,
  every lambda) and on the small workloads' scenes (20k gaussians SH0 at 360x640, 512
  gaussians SH3 at 128x128, at reduced and full size);
- the oracle's FP32 training passes (the checker of the CUDA path) render within the
  reference's own bars of its FP64 forward: image within 2.5/255 and loss within 1e-4
  (test_trainer.cpp:34-35);
- the oracle's analytic gradients pass the reference's finite-difference rule
  (train_selftest.cpp:418-446) against central differences of the reference's own loss.
Skipped when neither the library nor a reference checkout is present.
"""
import numpy as np
import pytest

import oracle as O
from gs_b200 import frame as F
from gs_b200 import scenes as S
from helpers import fd_check, frame_for, image_f

pytestmark = pytest.mark.skipif(O.ref_lib() is None, reason="no oracle/_ref build and no reference checkout")


def _both(cam, W, H, scene, target, bg, masked, lam, head=None):
    p64, s64 = scene.params.astype(np.float64), scene.sh.astype(np.float64)
    ref, ref_img = O.ref_reference_loss(cam.as_dict(), W, H, p64, s64, scene.degree, target, bg, masked, lam,
                                        want_image=True, head=head)
    ours, our_img = O.reference_loss(cam.as_dict(), W, H, p64, s64, scene.degree, target, bg, masked, lam,
                                     want_image=True, head=head)
    return ref, ref_img, ours, our_img


@pytest.mark.parametrize("masked,lam,head", [(False, 0.2, None), (True, 0.2, None), (True, 0.0, None),
                                             (False, 1.0, None), (True, 0.2, (30.0, 20.0, 14.0, 3.0))])
def test_restatement_equals_reference_on_its_test_scene(masked, lam, head):
    """make_test_dataset / make_test_scene (train_selftest.cpp:285-332), 64x48, 10 gaussians
    SH2, as check_gradients builds them (train_selftest.cpp:358-360)."""
    ds = S.make_test_dataset(64, 48, 1, masked, 3)
    scene = S.make_test_scene(10, 2, 11)
    ref, ref_img, ours, our_img = _both(ds.camera(0), 64, 48, scene, ds.rgba[0], (0.2, 0.5, 0.7), masked, lam, head)
    assert ours == ref
    np.testing.assert_array_equal(our_img, ref_img)


@pytest.mark.parametrize("name,n,degree,W,H,focal,mu,sigma", [
    ("512 gaussians SH3, 128x128", 512, 3, 128, 128, 200.0, -2.5, 0.3),
    ("the 20k-gaussian 360x640 workload at 1/16 the pixels and 1/10 the gaussians", 2000, 0, 90, 160, 125.0, -4.0, 0.5),
    ("the 20k-gaussian workload's shapes with SH3, 1/16 the pixels", 2000, 3, 90, 160, 125.0, -3.5, 0.5),
])
def test_restatement_equals_reference_on_workload_scenes(name, n, degree, W, H, focal, mu, sigma):
    scene = S.make_scene(n, 0, degree, radius=1.0, log_scale_mu=mu, log_scale_sigma=sigma)
    cam = S.front_camera(W, H, focal)
    rng = np.random.default_rng(1)
    target = rng.integers(0, 256, (H, W, 4), dtype=np.uint8)
    target[..., 3] = 255
    ref, ref_img, ours, our_img = _both(cam, W, H, scene, target, (0.0, 0.0, 0.0), False, 0.2)
    assert ours == ref, name
    np.testing.assert_array_equal(our_img, ref_img, err_msg=name)


def test_restatement_ssim_equals_reference():
    rng = np.random.default_rng(4)
    for W, H in [(64, 48), (37, 23), (11, 11), (1, 1)]:
        x = rng.uniform(0, 1, (W * H, 3))
        y = rng.uniform(0, 1, (W * H, 3))
        w = rng.uniform(0.5, 3.0, W * H)
        assert O.lib().gso_reference_ssim(x, y, W, H, None) == O.ref_reference_ssim(x, y, W, H)
        assert O.lib().gso_reference_ssim(x, y, W, H, O._ptr(w)) == O.ref_reference_ssim(x, y, W, H, w)


def _loss_from_sums(sums, lam, W, H):
    """Trainer::set_view_stats (trainer.cpp:797-805)."""
    n = 3.0 * W * H
    return ((1.0 - lam) * sums[3] + lam * (sums[5] - sums[4])) / n


@pytest.mark.parametrize("n,degree,W,H,focal,mu,sigma", [(512, 3, 128, 128, 200.0, -2.5, 0.3),
                                                         (2000, 0, 90, 160, 125.0, -4.0, 0.5)])
def test_fp32_passes_within_reference_bars(n, degree, W, H, focal, mu, sigma):
    """The FP32 passes the CUDA path is checked against render within 2.5/255 of the
    reference's FP64 image and give its loss within 1e-4 (test_trainer.cpp:34-35)."""
    scene = S.make_scene(n, 0, degree, radius=1.0, log_scale_mu=mu, log_scale_sigma=sigma)
    cam = S.front_camera(W, H, focal)
    rng = np.random.default_rng(2)
    target = rng.integers(0, 256, (H, W, 4), dtype=np.uint8)
    target[..., 3] = 255
    opt = F.TrainOptions(sh_degree=degree, sh_degree_interval=0, lambda_dssim=0.2, lambda_dssim_end=-1.0)
    fr = frame_for(scene, cam, opt, (0.0, 0.0, 0.0))
    r = O.forward_view(fr, scene.params, scene.sh, target)
    ref, ref_img = O.ref_reference_loss(cam.as_dict(), W, H, scene.params.astype(np.float64),
                                        scene.sh.astype(np.float64), degree, target, (0.0, 0.0, 0.0), False, 0.2,
                                        want_image=True)
    img = image_f(r.image)[:, :3]
    assert np.abs(img - np.clip(ref_img, 0, 1)).max() < 2.5 / 255.0
    assert abs(_loss_from_sums(r.sums, 0.2, W, H) - ref) < 1e-4


@pytest.mark.parametrize("masked,lam", [(False, 0.2), (True, 0.2), (False, 1.0)])
def test_oracle_gradients_against_reference_finite_differences(masked, lam):
    """check_gradients (train_selftest.cpp:356-486) with the reference's own reference_loss
    as the function differentiated: |err| <= 5% |fd| + 2e-6, at most 1/20 off per group."""
    ds = S.make_test_dataset(64, 48, 1, masked, 3)
    scene = S.make_test_scene(10, 2, 11)
    cam = ds.camera(0)
    opt = F.frozen_options(2, masked)
    opt.lambda_dssim = lam
    opt.lambda_dssim_end = -1.0
    bg = (0.2, 0.5, 0.7)
    fr = frame_for(scene, cam, opt, bg, masked=masked, ssim=lam > 0)
    model = O.Model.create(scene.params, scene.sh)
    _, g16, gsh, _ = O.train_step(model, [fr], [ds.rgba[0]], ssim=lam > 0)
    report = fd_check(scene, cam, ds.rgba[0], g16, gsh, bg, masked, lam, loss_impl=O.ref_reference_loss)
    assert set(report) == {"position", "opacity", "log_scale", "rotation", "sh_dc", "sh_rest"}
    for name, g in report.items():
        assert g["checked"] > 0 and g["bad"] <= g["checked"] // 20, (name, g)
