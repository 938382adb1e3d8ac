"""Tuning knobs and the autotuner (GPU): every setting computes the same step.

- The sort's digit width changes the passes, not the order: render order, ranges and pair
  lists are bit-identical at every width (the reference's radix sort is stable at any
  digit width, test_engine.cpp:27-68).
- gs_autotune times training steps under candidate settings and restores the model: the
  parameters, both moment sets and the densification statistics are bit-identical before
  and after, and the chosen tuning is one of the candidates (Trainer's retune,
  trainer.cpp:876-897, keeps training where it was the same way).
"""
import numpy as np
import pytest

import oracle as O
from gs_b200 import frame as F
from gs_b200 import scenes as S
from helpers import frame_for, rel_l2

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    from gs_b200.cuda import Context

    c = Context(0)
    yield c
    c.close()


def view_and_target(n=20000, degree=1):
    scene = S.make_scene(n, 0, degree, radius=1.0, log_scale_mu=-4.0, log_scale_sigma=0.5)
    truth = S.make_scene(n, 1, degree, radius=1.0, log_scale_mu=-4.0, log_scale_sigma=0.5)
    cam = S.front_camera(360, 640, 500.0)
    opt = F.TrainOptions(sh_degree=degree, sh_degree_interval=0, lambda_dssim=0.2, lambda_dssim_end=-1.0)
    fr_t = frame_for(truth, cam, opt, (0, 0, 0), ssim=False)
    rt = O.forward_view(fr_t, truth.params, truth.sh, np.zeros((640, 360, 4), np.uint8), ssim=False, backward=False)
    target = rt.image.view(np.uint8).reshape(640, 360, 4).copy()
    target[..., 3] = 255
    return scene, cam, opt, target


def test_sort_digit_widths_give_the_same_order(ctx):
    scene, cam, opt, target = view_and_target()
    fr = frame_for(scene, cam, opt, (0, 0, 0))
    ctx.model_init(scene.params, scene.sh)
    ctx.set_views([fr], [target])
    ref = None
    for digits in (8, 7, 6, 5, 4):
        ctx.set_tuning(sort_digit_bits=digits)
        ctx.step(train=False)
        got = {k: ctx.snapshot(k) for k in ("render_order", "ranges", "pair_tile", "offsets", "pixel_count")}
        if ref is None:
            ref = got
        else:
            for k in got:
                np.testing.assert_array_equal(got[k], ref[k], err_msg=f"{k} at {digits}-bit digits")
    ctx.set_tuning(sort_digit_bits=8)


def test_autotune_restores_the_model_and_picks_a_candidate(ctx):
    scene, cam, opt, target = view_and_target()
    fr = frame_for(scene, cam, opt, (0, 0, 0), step=5)
    ctx.model_init(scene.params, scene.sh)
    ctx.set_views([fr], [target])
    ctx.step(train=True)  # moments and statistics that are not all zero
    before = (ctx.export(), ctx.moments(), ctx.snapshot("stats"))
    t = ctx.autotune(1)
    after = (ctx.export(), ctx.moments(), ctx.snapshot("stats"))
    np.testing.assert_array_equal(before[0][0], after[0][0])
    np.testing.assert_array_equal(before[0][1], after[0][1])
    for k in before[1]:
        np.testing.assert_array_equal(before[1][k], after[1][k], err_msg=k)
    np.testing.assert_array_equal(before[2], after[2])
    assert t.forward_pixels in (1, 2, 4)
    assert (t.backward_pixels, t.backward_batch) in ((2, 32), (2, 64), (4, 32), (4, 64)) or t.backward_pixels == 8
    assert t.sort_digit_bits in (6, 7, 8)
    cur = ctx.tuning()
    assert (cur.forward_pixels, cur.backward_pixels, cur.backward_batch, cur.sort_digit_bits) == (
        t.forward_pixels, t.backward_pixels, t.backward_batch, t.sort_digit_bits)


def test_tunings_compute_the_same_gradients(ctx):
    """First-step gradients under the default tuning and under every other pixel and batch
    setting agree to summation order (1e-5 relative L2)."""
    scene, cam, opt, target = view_and_target()
    frozen = F.frozen_options(1, False)
    frozen.lambda_dssim, frozen.lambda_dssim_end = 0.2, -1.0
    fr = frame_for(scene, cam, frozen, (0, 0, 0))

    def grads(**kw):
        ctx.set_tuning(**kw)
        ctx.model_init(scene.params, scene.sh)
        ctx.set_views([fr], [target])
        ctx.step(train=True)
        return ctx.first_step_gradients()

    ref16, refsh = grads(forward_pixels=2, backward_pixels=4, backward_batch=64, sort_digit_bits=8)
    for kw in (dict(forward_pixels=1), dict(forward_pixels=4), dict(backward_pixels=2, backward_batch=32),
               dict(backward_pixels=1, backward_batch=64), dict(sort_digit_bits=5), dict(forward_batch=64),
               dict(forward_batch=128, forward_pixels=4), dict(stage_async=1), dict(stage_async=1, forward_batch=128),
               dict(stage_async=1, backward_pixels=2, backward_batch=32), dict(deterministic=0),
               dict(deterministic=0, stage_async=1, backward_pixels=1, backward_batch=32), dict(backward_pixels=8),
               dict(backward_pixels=8, deterministic=0)):
        base = dict(forward_pixels=2, backward_pixels=4, backward_batch=64, sort_digit_bits=8, forward_batch=256,
                    stage_async=0, deterministic=1)
        base.update(kw)
        g16, gsh = grads(**base)
        assert rel_l2(g16, ref16) < 1e-5, kw
        assert rel_l2(gsh, refsh) < 1e-5, kw
    ctx.set_tuning(forward_pixels=2, backward_pixels=4, backward_batch=64, sort_digit_bits=8, forward_batch=256,
                   stage_async=0, deterministic=1)


def test_async_staging_is_bit_identical(ctx):
    """Copying the next round of splats with cp.async while the current one is used changes
    when the records arrive, not what is computed: the forward's outputs, the per-pair
    gradients and the moments equal the plain-load staging bit for bit, at every forward
    batch and both backward batches (the batch changes how a tile's list is cut into rounds,
    not the order or the sums), on a view whose tiles hold several rounds of splats. Without
    cp.async the forward runs its independent-warp kernel (each warp staging its own rounds
    of 32, its last warp per tile adding the warps' tile sums), so this also checks that
    kernel, tile sums included, against the block kernel bit for bit."""
    scene, cam, opt, target = view_and_target(n=60000)
    frozen = F.frozen_options(1, False)
    frozen.lambda_dssim, frozen.lambda_dssim_end = 0.2, -1.0
    fr = frame_for(scene, cam, frozen, (0.1, 0.2, 0.3))
    outs = {}
    for fb, bb, stage in ((256, 64, 0), (256, 64, 1), (128, 32, 1), (64, 64, 1)):
        ctx.set_tuning(forward_batch=fb, backward_batch=bb, stage_async=stage, deterministic=1)
        ctx.model_init(scene.params, scene.sh)
        ctx.set_views([fr], [target])
        ctx.step(train=True)
        outs[(fb, bb, stage)] = {k: ctx.snapshot(k)
                                 for k in ("pixel_count", "pixel_out", "pixel_grad", "pair_grads", "tile_loss")}
        outs[(fb, bb, stage)]["m"] = ctx.moments()["m"]
    ref = outs[(256, 64, 0)]
    assert (ref["pixel_count"] > 256).any()  # tiles with more than one forward round
    for key, got in outs.items():
        for k in ref:
            np.testing.assert_array_equal(got[k], ref[k], err_msg=f"{k} {key}")
    ctx.set_tuning(forward_batch=256, backward_batch=64, stage_async=0, deterministic=1)


def test_atomic_steps_sort_gaussians(ctx):
    """An atomic training step sorts each pair's gaussian (no pre-sort index): the pair-order,
    per-pair gaussian and first-pair offset snapshots are refused with a message, also after
    a graph replay that follows a step run without the graph; the tile ranges and gradients
    are those of the deterministic step, and a forward-only step afterwards has the pair
    order again."""
    from gs_b200.cuda import GsError

    scene, cam, opt, target = view_and_target()
    frozen = F.frozen_options(1, False)
    fr = frame_for(scene, cam, frozen, (0, 0, 0))
    ctx.set_tuning(deterministic=1)
    ctx.model_init(scene.params, scene.sh)
    ctx.set_views([fr], [target])
    ctx.step(train=True)
    ref_ranges, ref_g = ctx.snapshot("ranges"), ctx.first_step_gradients()[0]
    ref_order = ctx.snapshot("render_order")
    ctx.set_tuning(deterministic=0)
    ctx.model_init(scene.params, scene.sh)
    ctx.set_views([fr], [target])
    ctx.step(train=True)
    np.testing.assert_array_equal(ctx.snapshot("ranges"), ref_ranges)
    assert rel_l2(ctx.first_step_gradients()[0], ref_g) < 1e-5
    for kind in ("render_order", "pair_gaussian", "offsets"):  # an atomic step keeps none of them
        with pytest.raises(GsError, match="atomic training step"):
            ctx.snapshot(kind)
    # A counting forward between two replays of the training graph runs without the graph;
    # the replay after it is an atomic step again.
    ctx.step(train=False, count=True)
    ctx.snapshot("offsets")
    ctx.step(train=True)
    with pytest.raises(GsError, match="atomic training step"):
        ctx.snapshot("offsets")
    ctx.step(train=False)
    np.testing.assert_array_equal(ctx.snapshot("render_order"), ref_order)
    ctx.snapshot("pair_gaussian")
    ctx.set_tuning(deterministic=1)


def test_counting_forward(ctx):
    """GS_STEP_COUNT: the counting forward renders exactly what the plain one does, and its
    count of blending evaluations is the same at every pixels-per-thread setting, positive
    and below E (the sum of every pixel's last-contributor position, which also counts the
    pairs a pixel skips)."""
    scene, cam, opt, target = view_and_target()
    frozen = F.frozen_options(1, False)
    fr = frame_for(scene, cam, frozen, (0, 0, 0))
    ctx.model_init(scene.params, scene.sh)
    ctx.set_views([fr], [target])
    ctx.step(train=False)
    plain = {k: ctx.snapshot(k) for k in ("pixel_count", "pixel_out", "image")}
    counts = []
    for px in (1, 2, 4):
        ctx.set_tuning(forward_pixels=px)
        ctx.step(train=False, count=True)
        for k in plain:
            np.testing.assert_array_equal(ctx.snapshot(k), plain[k], err_msg=f"{k} at {px} pixels per thread")
        counts.append(int(ctx.snapshot("contributions")[0]))
    ctx.set_tuning(forward_pixels=2)
    E = int(plain["pixel_count"].astype(np.int64).sum())
    assert counts[0] == counts[1] == counts[2] and 0 < counts[0] < E, (counts, E)
    # Every pixel with a last contributor blended at least once.
    assert counts[0] >= int((plain["pixel_count"] > 0).sum())
