"""Subject motion (SC-GS) on the CUDA path (GPU only).

- The binding: every slot's 4 nearest nodes and normalised weights exp(-d^2 / (2 r^2))
  (train_motion_bind.comp) against a numpy restatement.
- The motion gradient at rest, pinned the way the reference pins it (test_motion_gradient,
  test_trainer.cpp:549-606): with every node at rest, a shift s of node k moves its
  gaussians by w s and a turn u about the node moves them by w u x (p - n_k) and turns their
  orientation by w u, so the per-node gradient must equal what the per-gaussian gradients
  (checked against the oracle elsewhere) imply.
- A step with the nodes moved equals the oracle's step on the scene moved on the host
  (positions x = sum w (R p + b), orientations turned by exp(sum w turn)): the same loss
  sums and image, and gradients that map back to the rest parameters by the chain rule
  (positions through A^T = (sum w R)^T, quaternions through the turn's left product).
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


def place_nodes(positions, k, seed):
    """k of the gaussians as nodes; radius: mean distance to the 3 nearest other nodes."""
    rng = np.random.default_rng(seed)
    idx = rng.choice(len(positions), k, replace=False)
    n = positions[idx].astype(np.float64)
    d = np.linalg.norm(n[:, None] - n[None], axis=2)
    np.fill_diagonal(d, np.inf)
    r = np.sort(d, axis=1)[:, :3].mean(axis=1)
    return np.concatenate([n, (1.0 / (2.0 * r * r))[:, None]], axis=1).astype(np.float32)


def turn_matrix(w):
    t = np.linalg.norm(w)
    K = np.array([[0, -w[2], w[1]], [w[2], 0, -w[0]], [-w[1], w[0], 0]])
    if t < 1e-12:
        return np.eye(3)
    return np.eye(3) + np.sin(t) / t * K + (1 - np.cos(t)) / t ** 2 * (K @ K)


def node_table(nodes4, turns, shifts):
    """(K, 20) float32: rows of [R | b] with b = c - R n, the turn, the moved centre c."""
    out = np.zeros((len(nodes4), 20), np.float64)
    for k, (n, w, s) in enumerate(zip(nodes4[:, :3].astype(np.float64), turns, shifts)):
        R = turn_matrix(w)
        c = n + s
        out[k, 0:12] = np.concatenate([R, (c - R @ n)[:, None]], axis=1).reshape(-1)
        out[k, 12:15] = w
        out[k, 16:19] = c
    return out.astype(np.float32)


def bind_numpy(positions, nodes4):
    d2 = ((positions[:, None, :].astype(np.float32) - nodes4[None, :, :3]) ** 2).sum(axis=2)
    order = np.argsort(d2, axis=1, kind="stable")[:, :4]
    dist = np.take_along_axis(d2, order, axis=1)
    w = np.exp(-dist * nodes4[order, 3])
    return order, w / w.sum(axis=1, keepdims=True), dist


def binding(ctx):
    b = ctx.snapshot("motion_bind")
    return b[:, :4].astype(np.int64), b[:, 4:].copy().view(np.float32)


def rest_grads(scene, g16):
    """Per gaussian: position gradient and the orientation's turn share tau
    (test_trainer.cpp:437-443)."""
    p = scene.params.astype(np.float64)
    g = g16.astype(np.float64)
    q = p[:, 8:12]
    qlen = np.linalg.norm(q, axis=1, keepdims=True)
    qn = q / qlen
    w, u = qn[:, :1], qn[:, 1:]
    gw, gu = g[:, 8:9] * qlen, g[:, 9:12] * qlen
    tau = 0.5 * (-gw * u + w * gu + np.cross(u, gu))
    return g[:, 0:3], tau


def motion_frame(scene, cam, flags, lam=0.2, masked=True, bg=(0.2, 0.3, 0.4)):
    opt = F.frozen_options(0, masked)
    opt.lambda_dssim, opt.lambda_dssim_end = lam, -1.0
    fr = frame_for(scene, cam, opt, bg, masked=masked, ssim=lam > 0)
    fr["model"][0, 3] |= flags
    return fr


@pytest.mark.parametrize("k", [8, 64, 100])
def test_motion_gradient_at_rest(ctx, k):
    ds = S.make_test_dataset(64, 48, 2, True, 3)
    scene = S.make_test_scene(400 if k > 64 else 120, 0, 9)
    nodes = place_nodes(scene.params[:, 0:3], k, 5)
    fr = motion_frame(scene, ds.camera(1), F.FLAG_MOTION | F.FLAG_MOTION_GRAD)
    ctx.model_init(scene.params, scene.sh)
    ctx.motion_nodes(nodes)
    ctx.set_views([fr], [ds.rgba[1]])
    ctx.set_view_motion(0, node_table(nodes, np.zeros((k, 3)), np.zeros((k, 3))))
    res = ctx.step(True)
    assert res.overflow == 0
    got = ctx.motion_gradient(0, k)
    g16, _ = ctx.first_step_gradients()
    bn, bw = binding(ctx)
    # The binding against the restatement (slots whose 4th and 5th nearest are not tied).
    ref_nodes, ref_w, dist = bind_numpy(scene.params[:, 0:3], nodes)
    d2 = np.sort(((scene.params[:, None, 0:3] - nodes[None, :, :3]) ** 2).sum(axis=2), axis=1)
    clear = np.all(np.diff(d2[:, :5], axis=1) > 1e-6 * d2[:, 1:5], axis=1)
    assert clear.mean() > 0.95
    np.testing.assert_array_equal(bn[clear], ref_nodes[clear])
    np.testing.assert_allclose(bw[clear], ref_w[clear], rtol=1e-5, atol=1e-7)
    assert np.abs(bw.sum(axis=1) - 1.0).max() < 1e-5
    # The gradient the per-gaussian gradients imply.
    gp, tau = rest_grads(scene, g16)
    want = np.zeros((k, 6))
    for j in range(4):
        w = bw[:, j].astype(np.float64)
        kk = bn[:, j]
        r = scene.params[:, 0:3].astype(np.float64) - nodes[kk, :3].astype(np.float64)
        np.add.at(want, (kk, slice(0, 3)), w[:, None] * gp)
        np.add.at(want, (kk, slice(3, 6)), w[:, None] * (np.cross(r, gp) + tau))
    largest = np.abs(want).max()
    assert largest > 0
    assert np.abs(got - want).max() <= 1e-3 * largest, (np.abs(got - want).max(), largest)


def quat_left(q):
    """The matrix of q (w, x, y, z) times a quaternion (Hamilton product)."""
    w, x, y, z = q
    return np.array([[w, -x, -y, -z], [x, w, -z, y], [y, z, w, -x], [z, -y, x, w]])


def deformed_scene(scene, nodes, table, turns, bn, bw):
    """The scene moved on the host (float64): positions, quaternions turned, and per slot
    A = sum w R and the quaternion's left-product matrix."""
    p = scene.params.astype(np.float64)
    out = scene.params.copy()
    A = np.zeros((len(p), 3, 3))
    Lq = np.zeros((len(p), 4, 4))
    rows = table[:, :12].astype(np.float64).reshape(-1, 3, 4)
    for i in range(len(p)):
        x = np.zeros(3)
        turn = np.zeros(3)
        for j in range(4):
            w, k = float(bw[i, j]), int(bn[i, j])
            if w == 0.0:
                continue
            x += w * (rows[k, :, :3] @ p[i, 0:3] + rows[k, :, 3])
            A[i] += w * rows[k, :, :3]
            turn += w * turns[k]
        t = np.linalg.norm(turn)
        qu = np.concatenate([[np.cos(t / 2)], np.sin(t / 2) * turn / t]) if t > 0 else np.array([1.0, 0, 0, 0])
        Lq[i] = quat_left(qu)
        out[i, 0:3] = x
        out[i, 8:12] = Lq[i] @ p[i, 8:12]
    return out.astype(np.float32), A, Lq


def test_moved_step_matches_oracle_on_moved_scene(ctx):
    ds = S.make_test_dataset(128, 96, 2, False, 3)
    scene = S.make_test_scene(300, 0, 9)
    k = 8
    nodes = place_nodes(scene.params[:, 0:3], k, 6)
    rng = np.random.default_rng(11)
    turns, shifts = rng.normal(0, 0.1, (k, 3)), rng.normal(0, 0.03, (k, 3))
    table = node_table(nodes, turns, shifts)
    cam = ds.camera(1)
    target = ds.rgba[1]
    fr = motion_frame(scene, cam, F.FLAG_MOTION, masked=False, bg=(0.0, 0.0, 0.0))
    ctx.model_init(scene.params, scene.sh)
    ctx.motion_nodes(nodes)
    ctx.set_views([fr], [target])
    ctx.set_view_motion(0, table)
    res = ctx.step(True)
    image = ctx.snapshot("image").copy()
    g16, _ = ctx.first_step_gradients()
    bn, bw = binding(ctx)
    moved, A, Lq = deformed_scene(scene, nodes, table, turns.astype(np.float32).astype(np.float64), bn, bw)
    plain = fr.copy()
    plain["model"][0, 3] &= ~np.uint32(F.FLAG_MOTION)
    model = O.Model.create(moved, scene.sh)
    results, ref16, _, _ = O.train_step(model, [plain], [target])
    r = results[0]
    # The image and the loss sums.
    same = ctx.snapshot("pixel_count") == r.pixel_count
    assert same.mean() > 0.999
    diff = np.abs(image.view(np.uint8).reshape(-1, 4).astype(int) - r.image.view(np.uint8).reshape(-1, 4).astype(int))
    assert diff[same].max() <= 1
    sums = np.array(res.losses[0][:8])
    for kk in (0, 1, 3, 5):
        assert abs(sums[kk] - r.sums[kk]) <= 1e-4 * abs(r.sums[kk]) + 1e-6, kk
    # Gradients back to the rest parameters.
    want = ref16.astype(np.float64).copy()
    want[:, 0:3] = np.einsum("nrc,nr->nc", A, ref16[:, 0:3].astype(np.float64))
    want[:, 8:12] = np.einsum("nrc,nr->nc", Lq, ref16[:, 8:12].astype(np.float64))
    for name, cols in {"position": [0, 1, 2], "opacity": [3], "log_scale": [4, 5, 6], "rotation": [8, 9, 10, 11],
                       "sh_dc": [12, 13, 14]}.items():
        assert rel_l2(g16[:, cols], want[:, cols]) < 1e-3, name
    # gs_render with the motion flag uses view 0's node motions: the step's image.
    np.testing.assert_array_equal(ctx.render(fr).reshape(-1), image.view(np.uint8).reshape(-1))


def test_batched_motion_gradients_equal_single_views(ctx):
    ds = S.make_test_dataset(64, 48, 3, True, 3)
    scene = S.make_test_scene(200, 1, 9)
    k = 16
    nodes = place_nodes(scene.params[:, 0:3], k, 7)
    rng = np.random.default_rng(12)
    tables = [node_table(nodes, rng.normal(0, 0.05, (k, 3)), rng.normal(0, 0.02, (k, 3))) for _ in range(2)]
    frames = [motion_frame(scene, ds.camera(v + 1), F.FLAG_MOTION | F.FLAG_MOTION_GRAD) for v in range(2)]
    ctx.model_init(scene.params, scene.sh)
    ctx.motion_nodes(nodes)
    ctx.set_views(frames, [ds.rgba[1], ds.rgba[2]])
    for v in range(2):
        ctx.set_view_motion(v, tables[v])
    ctx.step(True)
    batched = [ctx.motion_gradient(v, k) for v in range(2)]
    for v in range(2):
        ctx.model_init(scene.params, scene.sh)
        ctx.motion_nodes(nodes)
        ctx.set_views([frames[v]], [ds.rgba[v + 1]])
        ctx.set_view_motion(0, tables[v])
        ctx.step(True)
        np.testing.assert_array_equal(batched[v], ctx.motion_gradient(0, k))
    assert np.abs(batched[0]).max() > 0


def test_motion_gradient_needs_the_flag(ctx):
    ds = S.make_test_dataset(64, 48, 2, True, 3)
    scene = S.make_test_scene(120, 0, 9)
    nodes = place_nodes(scene.params[:, 0:3], 8, 5)
    ctx.model_init(scene.params, scene.sh)
    ctx.motion_nodes(nodes)
    ctx.set_views([motion_frame(scene, ds.camera(1), 0)], [ds.rgba[1]])
    ctx.step(True)
    from gs_b200.cuda import GsError

    with pytest.raises(GsError):
        ctx.motion_gradient(0, 8)
