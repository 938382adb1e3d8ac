"""The optimizer step at nonzero learning rates and the densify statistics, CUDA path vs
the oracle, through the C ABI (GPU only).

The reference's step: Adam on the 16 parameters of a slot (train_step.glsl:62-68, 242-251)
and on the active SH coefficients (train_step_sh.comp:21-44), with
  m = mix(g, m, beta1), v = mix(g^2, v, beta2), p -= lr (m c1) / (sqrt(v c2) + eps),
beta1 = 0.9, beta2 = 0.999, eps = 1e-15 (trainer.cpp:68-70); and the densify statistics of
each view a slot is drawn in (train_step.glsl:90-100): the NDC-scaled norms of dL/dmean2d
and of its absolute sums, the view count and the largest radius.

Tolerances:
- The Adam arithmetic on the GPU's own moments: the kernels take the square root and the
  division in the hardware's approximate forms (sqrt.approx.f32, relative error within
  2^-23; div.full.f32, within 2 ulp), and the update and the moments may be contracted into
  fused multiply-adds (one rounding fewer). So |p_gpu - p_expected| <= lr |u| 2^-20 +
  2 ulp(p), with u = m c1 / (sqrt(v c2) + eps) evaluated in double from the GPU's m and v:
  2^-20 covers sqrt (2^-23, halved through the quotient's denominator), the division
  (2 x 2^-24), the product with lr and one contraction, with margin.
- Against the oracle's own gradients (which differ by summation order, within 1e-3 relative
  L2 per group): moments and statistics within 1e-3 relative L2 per group (v within 2e-3:
  it is quadratic in g); parameter updates within 2e-3, because Adam gives every element a
  step of about lr whatever its gradient's size, so the elements with small gradients (and
  the largest relative summation error) weigh as much in the update's L2 norm as the large
  ones; view counts exact on all but 1e-4 of the slots (a
  slot at the edge of a view can gain or lose its last tile through a float of the
  projection); radii within 1e-5 relative.
"""
import numpy as np
import pytest

import oracle as O
from gs_b200 import frame as F
from gs_b200 import scenes as S
from helpers import GROUPS, frame_for, rel_l2

pytestmark = pytest.mark.gpu

N, W, H, FOCAL = 20000, 360, 640, 500.0


@pytest.fixture(scope="module")
def ctx():
    from gs_b200.cuda import Context

    c = Context(0)
    yield c
    c.close()


def options() -> F.TrainOptions:
    """The plain-training learning rates (means 1.6e-4 x extent with decay, scales 5e-3,
    rotations 1e-3, opacity 5e-2, SH DC 2.5e-3, SH rest 2.5e-3 / 20), fixed lambda 0.2."""
    o = F.TrainOptions(iterations=3000, sh_degree=3, sh_degree_interval=0, masked=False, random_background=False,
                       lr_opacity=5e-2, lambda_dssim=0.2, lambda_dssim_end=-1.0)
    return o


def scene_and_views():
    scene = S.make_scene(N, 0, 3, radius=1.0, log_scale_mu=-4.0, log_scale_sigma=0.5)
    truth = S.make_scene(N, 1, 3, radius=1.0, log_scale_mu=-4.0, log_scale_sigma=0.5)
    cams = S.orbit_cameras(6, 3.0, 0.5, W, H, FOCAL)[:2]
    opt = options()
    targets = []
    for cam in cams:
        fr_t = frame_for(truth, cam, opt, (0, 0, 0), ssim=False)
        r = O.forward_view(fr_t, truth.params, truth.sh, np.zeros((H, W, 4), np.uint8), ssim=False, backward=False)
        t = r.image.view(np.uint8).reshape(H, W, 4).copy()
        t[..., 3] = 255
        targets.append(t)
    return scene, cams, opt, targets


def gpu_state(ctx) -> dict:
    p, s = ctx.export()
    mo = ctx.moments()
    return {"params": p, "sh": s, **mo, "stats": ctx.snapshot("stats")}


def element_lr(fr) -> np.ndarray:
    """The learning rate of each of the 16 parameters (gso_adam's table)."""
    l0, l1 = fr["lr0"][0], fr["lr1"][0]
    return np.array([l0[0], l0[0], l0[0], l0[3], l0[1], l0[1], l0[1], 0.0, l0[2], l0[2], l0[2], l0[2],
                     l1[0], l1[0], l1[0], 0.0], np.float64)


def check_adam_arithmetic(before: np.ndarray, after: np.ndarray, m: np.ndarray, v: np.ndarray, lr, fr) -> None:
    c1, c2 = float(fr["bias"][0][0]), float(fr["bias"][0][1])
    eps = float(fr["adam"][0][2])
    u = (m.astype(np.float64) * c1) / (np.sqrt(v.astype(np.float64) * c2) + eps)
    want = before.astype(np.float64) - lr * u
    bound = lr * np.abs(u) * 2.0 ** -20 + 2.0 * np.spacing(np.abs(after).astype(np.float32)).astype(np.float64)
    err = np.abs(after.astype(np.float64) - want)
    assert (err <= bound).all(), float((err - bound).max())


def oracle_model(state: dict) -> O.Model:
    model = O.Model.create(state["params"], state["sh"])
    model.m[:], model.v[:] = state["m"], state["v"]
    model.m_sh[:], model.v_sh[:] = state["m_sh"], state["v_sh"]
    model.stats[:] = state["stats"]
    return model


def two_steps(ctx):
    """Two GPU training steps on the same view (steps 0 and 1), the states before and
    after each, and the oracle's second step from the GPU's state after the first."""
    scene, cams, opt, targets = scene_and_views()
    fr0 = frame_for(scene, cams[0], opt, (0, 0, 0), step=0)
    fr1 = frame_for(scene, cams[0], opt, (0, 0, 0), step=1)
    ctx.model_init(scene.params, scene.sh)
    s0 = gpu_state(ctx)
    ctx.set_views([fr0], [targets[0]])
    assert ctx.step(True).overflow == 0
    s1 = gpu_state(ctx)
    ctx.set_views([fr1], [targets[0]])
    assert ctx.step(True).overflow == 0
    s2 = gpu_state(ctx)
    model = oracle_model(s1)
    O.train_step(model, [fr1], [targets[0]])
    first = O.Model.create(scene.params, scene.sh)
    O.train_step(first, [fr0], [targets[0]])
    return scene, (fr0, fr1), (s0, s1, s2), model, first


@pytest.fixture(scope="module")
def stepped(ctx):
    return two_steps(ctx)


def test_adam_update_is_the_reference_formula(stepped):
    """p_new = p - lr (m c1) / (sqrt(v c2) + eps) on the GPU's own moments, both steps, all
    16 parameters and every SH coefficient, within the approximate-arithmetic bound."""
    scene, (fr0, fr1), (s0, s1, s2), _, _ = stepped
    for fr, a, b in ((fr0, s0, s1), (fr1, s1, s2)):
        check_adam_arithmetic(a["params"], b["params"], b["m"], b["v"], element_lr(fr)[None, :], fr)
        check_adam_arithmetic(a["sh"], b["sh"], b["m_sh"], b["v_sh"], float(fr["lr1"][0][1]), fr)
    # The moments are the reference's mix() of the previous ones: m2 - beta1 m1 and
    # v2 - beta2 v1 are (1 - beta1) g and (1 - beta2) g^2 of one g.
    b1, b2 = np.float32(fr1["adam"][0][0]), np.float32(fr1["adam"][0][1])
    g = (s2["m"].astype(np.float64) - float(b1) * s1["m"]) / float(np.float32(1) - b1)
    want_v = float(np.float32(1) - b2) * g * g + float(b2) * s1["v"].astype(np.float64)
    big = np.abs(g) > 1e-3 * np.abs(g).max()
    assert rel_l2(s2["v"][big], want_v[big]) < 1e-5


def test_first_step_moments_and_update_match_oracle(stepped):
    """Step 0 from zero moments at nonzero learning rates: m, v (16 parameters and SH) of the
    GPU and of the oracle's own step. The update itself is sign(g) lr c1 / sqrt(c2) there
    (Adam's first step), so it is compared where |g| is clear of summation noise."""
    _, (fr0, _), (s0, s1, _), _, first = stepped
    n = s0["params"].shape[0]
    for name, cols in GROUPS.items():
        assert rel_l2(s1["m"][:, cols], first.m[:n, cols]) < 1e-3, name
        assert rel_l2(s1["v"][:, cols], first.v[:n, cols]) < 2e-3, name
        g = first.m[:n, cols].astype(np.float64)
        clear = np.abs(g) > 1e-2 * np.sqrt(np.mean(g * g))
        d_gpu = (s1["params"] - s0["params"])[:, cols][clear]
        d_ref = (first.params[:n] - s0["params"])[:, cols][clear]
        assert clear.sum() > 1000 and rel_l2(d_gpu, d_ref) < 1e-3, name
    assert rel_l2(s1["m_sh"], first.m_sh[:n]) < 1e-3
    assert rel_l2(s1["v_sh"], first.v_sh[:n]) < 2e-3


def test_second_step_matches_oracle(stepped):
    """Step 1 from the GPU's state after step 0, on both sides: moments per group within
    1e-3 relative L2 (v 2e-3), parameter and SH updates within 2e-3."""
    _, _, (_, s1, s2), model, _ = stepped
    n = s1["params"].shape[0]
    for name, cols in GROUPS.items():
        d_gpu = (s2["params"] - s1["params"])[:, cols]
        d_ref = (model.params[:n] - s1["params"])[:, cols]
        assert rel_l2(d_gpu, d_ref) < 2e-3, name
        assert rel_l2(s2["m"][:, cols], model.m[:n, cols]) < 1e-3, name
        assert rel_l2(s2["v"][:, cols], model.v[:n, cols]) < 2e-3, name
    assert rel_l2(s2["sh"] - s1["sh"], model.sh[:n] - s1["sh"]) < 2e-3
    assert rel_l2(s2["m_sh"], model.m_sh[:n]) < 1e-3
    assert rel_l2(s2["v_sh"], model.v_sh[:n]) < 2e-3


def test_densify_statistics_match_oracle(stepped):
    """train_step.glsl:90-100 after two steps, GPU vs the oracle's own statistics (the oracle
    computing both steps' statistics from its own gradients and projection)."""
    _, _, (_, s1, s2), model, first = stepped
    n = s2["stats"].shape[0]
    # Step 0 alone: the oracle from the initial state.
    st1, ref1 = s1["stats"], first.stats[:n]
    # Step 1 on top of the GPU's step-0 statistics.
    st2, ref2 = s2["stats"], model.stats[:n]
    for got, ref in ((st1, ref1), (st2, ref2)):
        assert (ref[:, 1] > 0).sum() > 0.5 * n
        assert rel_l2(got[:, 0], ref[:, 0]) < 1e-3  # sum of |dL/dmean2d| (NDC)
        assert rel_l2(got[:, 3], ref[:, 3]) < 1e-3  # sum of the absolute-gradient norms
        assert (got[:, 1] != ref[:, 1]).mean() <= 1e-4  # views drawn in
        same = got[:, 1] == ref[:, 1]
        np.testing.assert_allclose(got[same, 2], ref[same, 2], rtol=1e-5, atol=1e-5)  # largest radius


def test_densify_from_gpu_statistics_matches_oracle(ctx, stepped):
    """Densify after the two steps, each side on its own statistics (the oracle's summed
    over its own two steps, not the GPU's copied in), on the GPU's parameters: spawn masks
    equal wherever the mean gradient is clear of the threshold by the gradients' summation
    tolerance, and the prune set equal everywhere."""
    scene, _, (_, s1, s2), model, first = stepped
    n = s2["params"].shape[0]
    own = first.stats[:n].copy()
    own[:, [0, 1, 3]] += model.stats[:n][:, [0, 1, 3]] - s1["stats"][:, [0, 1, 3]]
    own[:, 2] = np.maximum(own[:, 2], model.stats[:n, 2])
    mean = np.where(own[:, 1] > 0, own[:, 0] / np.maximum(own[:, 1], 1), 0.0)
    threshold = float(np.median(mean[own[:, 1] > 0]))
    opt = options()
    opt.densify_grad_threshold = threshold
    fr = F.make_frame(S.orbit_cameras(6, 3.0, 0.5, W, H, FOCAL)[0], n, scene.sh.shape[1], 2, opt, (0, 0, 0), 3.3)
    ref = oracle_model(s2)
    ref.stats[:n] = own
    _, spawn_ref = O.densify(ref, fr, n)
    ctx.densify(fr)
    spawn = ctx.snapshot("spawn")[:n]
    near = np.abs(mean - threshold) <= 2e-3 * threshold
    assert (spawn_ref == 1).sum() > 100 and (spawn_ref == 2).sum() > 100
    assert near.mean() < 0.01
    np.testing.assert_array_equal(spawn[~near], spawn_ref[~near])
    pruned = s2["params"][:, 3] < np.log(0.005 / 0.995)
    assert (spawn[pruned] == 0).all()
