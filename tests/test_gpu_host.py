"""gs_train, gs_render and gs::Trainer (the C++ host layer over libgs_cuda) on a GPU.

- The reference's convergence check through gs::Trainer: its known-scene fit
  (fit_known_scene, train_selftest.cpp:692-739) must end with held-out PSNR above 35 dB and
  8 dB above the start (test_training_converges, test_trainer.cpp:890-897), plain and batched.
- Short synthetic orbit runs of gs_train, plain and batched (held-out PSNR rises and
  densification runs), and a headless render of the PLY the trainer wrote through the
  --views camera-file mode.
"""
import json
import os
import subprocess

import numpy as np
import pytest

from gs_b200 import scenes as S

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "on-divice-gsplate_b200", "bin")
SMALL = ["--gt-gaussians", "20000", "--init-gaussians", "4000", "--cameras", "24", "--sh", "1"]


def train(tmp_path, name, *extra):
    out_ply = tmp_path / f"{name}.ply"
    metrics = tmp_path / f"{name}.json"
    cmd = [os.path.join(BIN, "gs_train"), "synthetic:orbit", str(out_ply), "--json", str(metrics), *SMALL, *extra]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    return out_ply, json.loads(metrics.read_text()), r.stdout


def ply_vertices(path):
    data = open(path, "rb").read()
    head, _, _ = data.partition(b"end_header\n")
    for line in head.decode().splitlines():
        if line.startswith("element vertex"):
            return int(line.split()[-1])
    raise AssertionError("no vertex element")


@pytest.fixture(scope="module")
def plain_run(tmp_path_factory):
    tmp = tmp_path_factory.mktemp("plain")
    return train(tmp, "plain", "--iters", "400", "--eval-every", "100")


def test_gs_train_plain_learns(plain_run):
    ply, m, log = plain_run
    evals = [e["psnr"] for e in m["eval"]]
    assert len(evals) == 4 and all(np.isfinite(evals)), log
    assert evals[-1] > evals[0] + 1.0, log
    assert m["spawned"] > 0, log  # densification ran (schedule 40..333 every 13 steps)
    assert m["overflow_steps"] == 0
    assert ply_vertices(ply) == m["gaussians"]


def test_gs_train_batched_learns(tmp_path):
    _, m, log = train(tmp_path, "batched", "--iters", "200", "--eval-every", "100", "--views-per-step", "4")
    evals = [e["psnr"] for e in m["eval"]]
    assert m["views"] == 800 and m["views_per_step"] == 4
    assert evals[-1] > evals[0], log


def test_gs_render_views(plain_run, tmp_path):
    ply, _, _ = plain_run
    cams = [S.front_camera(320, 240, 300.0, 3.0), S.front_camera(200, 100, 150.0, 4.0)]
    with open(tmp_path / "cameras.txt", "w") as f:
        for c in cams:
            m = np.concatenate([c.rotation.reshape(3, 3), c.translation.reshape(3, 1)], axis=1).reshape(-1)
            f.write(" ".join(str(v) for v in [c.width, c.height, c.fx, c.fy, c.cx, c.cy, *m]) + "\n")
    r = subprocess.run([os.path.join(BIN, "gs_render"), str(ply), "--views", str(tmp_path / "cameras.txt"),
                        str(tmp_path)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    for i, c in enumerate(cams):
        data = open(tmp_path / f"view_{i:05d}.ppm", "rb").read()
        head = f"P6\n{c.width} {c.height}\n255\n".encode()
        assert data.startswith(head)
        px = np.frombuffer(data[len(head):], np.uint8)
        assert px.size == c.width * c.height * 3
        assert px.max() > 0  # the trained scene is in view


def test_gs_train_capture_folder(tmp_path):
    """gs_train on a transforms.json capture: PNG views of a known scene (rendered through
    libgs_cuda) with its coverage as masks (the default random backgrounds composite over
    them), a point cloud from noisy scene means; held-out PSNR rises."""
    from gs_b200 import frame as F
    from gs_b200.cuda import Context
    from test_dataset_loader import write_png

    truth = S.make_scene(8000, 1, 1, radius=1.0, log_scale_mu=-3.5, log_scale_sigma=0.4)
    opt = F.TrainOptions(sh_degree=1, sh_degree_interval=0)
    frames = []
    with Context(0) as ctx:
        ctx.model_init(truth.params, truth.sh)
        for i in range(16):
            a = 2 * np.pi * i / 16
            c2w = F.look_at_c2w_gl((3 * np.sin(a), 0.5, 3 * np.cos(a)), (0.0, 0.0, 0.0))
            cam = F.dataset_camera(c2w, 120.0, 120.0, 64.0, 48.0, 128, 96)
            img = ctx.render(F.make_frame(cam, truth.count, truth.sh.shape[1], 0, opt, (0, 0, 0), 3.3))
            write_png(tmp_path / f"view_{i:02d}.png", img[..., :3], 2)
            write_png(tmp_path / f"mask_{i:02d}.png", img[..., 3:4], 0)
            frames.append({"file_path": f"view_{i:02d}.png", "mask_path": f"mask_{i:02d}.png",
                           "transform_matrix": c2w.astype(float).tolist()})
    rng = np.random.default_rng(2)
    pts = truth.params[:3000, :3] + rng.normal(0, 0.02, (3000, 3)).astype(np.float32)
    rec = np.zeros(3000, dtype=[("p", "<f4", 3), ("c", "u1", 3)])
    rec["p"], rec["c"] = pts, 128
    head = ("ply\nformat binary_little_endian 1.0\nelement vertex 3000\nproperty float x\nproperty float y\n"
            "property float z\nproperty uchar red\nproperty uchar green\nproperty uchar blue\nend_header\n")
    open(tmp_path / "points.ply", "wb").write(head.encode() + rec.tobytes())
    (tmp_path / "transforms.json").write_text(json.dumps(
        {"w": 128, "h": 96, "fl_x": 120.0, "cx": 64.0, "cy": 48.0, "frames": frames, "ply_file_path": "points.ply"}))
    out_ply, metrics = tmp_path / "out.ply", tmp_path / "m.json"
    r = subprocess.run([os.path.join(BIN, "gs_train"), str(tmp_path), str(out_ply), "--iters", "300", "--width", "96",
                        "--sh", "1", "--eval-every", "100", "--json", str(metrics)],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "initial gaussians from points: 3000" in r.stdout
    m = json.loads(metrics.read_text())
    evals = [e["psnr"] for e in m["eval"]]
    assert evals[-1] > evals[0] + 1.0, r.stdout
    assert ply_vertices(out_ply) == m["gaussians"]


def refine_selftest(*args):
    r = subprocess.run([os.path.join(BIN, "gs_refine_selftest"), *args], capture_output=True, text=True, timeout=600)
    return r.returncode, r.stdout + r.stderr


@pytest.mark.parametrize("lam", ["0.0", "0.2"])
def test_trainer_pose_gradient(lam):
    """test_pose_gradient (test_trainer.cpp:404-460) through gs::Trainer: the pose gradient
    of a step equals what its per-gaussian gradients imply, within 1e-3 of the largest."""
    rc, out = refine_selftest("pose-gradient", lam)
    assert rc == 0, out


def test_trainer_pose_recovery():
    """test_pose_recovery (test_trainer.cpp:505-547): a camera moved 10 cm and 1.5 degrees
    comes back to within a quarter of that by refining its pose with frozen gaussians."""
    rc, out = refine_selftest("pose-recovery")
    assert rc == 0, out


def test_trainer_exposure_recovery():
    """test_exposure_recovery (test_trainer.cpp:700-742): gains of a darkened, tinted view
    come out in the ratio it was dimmed by (2%), centred on the trained views."""
    rc, out = refine_selftest("exposure-recovery")
    assert rc == 0, out


def test_trainer_aligns_held_out_views():
    """evaluate with refine_poses: a held-out view given 2 px off is aligned before it is
    measured (align_camera, trainer.cpp:1164-1212)."""
    rc, out = refine_selftest("align")
    assert rc == 0, out


def test_gs_train_with_refinement(tmp_path):
    """gs_train with pose and exposure refinement and a pose export runs and still learns."""
    poses = tmp_path / "poses.json"
    _, m, out = train(tmp_path, "refine", "--iters", "300", "--eval-every", "150", "--views-per-step", "4",
                      "--refine-poses", "--pose-from", "50", "--refine-exposure", "--eval-pose-steps", "4",
                      "--pose-out", str(poses))
    assert "poses: shift" in out and "exposure: luminance gain" in out and "at the poses as given" in out
    assert m["eval"][-1]["psnr"] > m["eval"][0]["psnr"]
    frames = json.loads(poses.read_text())["frames"]
    assert len(frames) == 24 and sum(f["holdout"] for f in frames) == 3
    for f in frames:
        M = np.array(f["transform_matrix"])
        assert M.shape == (4, 4) and np.allclose(M[:3, :3] @ M[:3, :3].T, np.eye(3), atol=1e-4)


@pytest.mark.parametrize("nodes", ["8", "100"])
def test_trainer_motion_gradient(nodes):
    """test_motion_gradient (test_trainer.cpp:549-606) through gs::Trainer: with the nodes
    at rest the motion gradient equals what the per-gaussian gradients imply."""
    rc, out = refine_selftest("motion-gradient", nodes)
    assert rc == 0, out


def test_trainer_motion_recovery():
    """test_motion_recovery (test_trainer.cpp:660-690): one node moved 9 cm and 11 degrees in
    a view's target; refining that view's motion with frozen gaussians brings them back
    to within a quarter of the on-screen distance."""
    rc, out = refine_selftest("motion-recovery")
    assert rc == 0, out


def test_trainer_motion_batched():
    """test_motion_batched (test_trainer.cpp:744-782) with 3 views per step: every view of
    every step from motion_from updates its motion, through densification."""
    rc, out = refine_selftest("motion-batched")
    assert rc == 0, out


def test_gs_train_with_motion(tmp_path):
    """gs_train --refine-motion writes the nodes and every view's motion and still learns."""
    motion = tmp_path / "nodes.json"
    _, m, out = train(tmp_path, "motion", "--iters", "300", "--eval-every", "150", "--views-per-step", "2",
                      "--refine-motion", "--motion-nodes", "16", "--motion-from", "50", "--motion-out", str(motion))
    assert "motion: 16 nodes" in out and "view updates" in out
    assert m["eval"][-1]["psnr"] > m["eval"][0]["psnr"]
    data = json.loads(motion.read_text())
    assert len(data["nodes"]) == 16 and len(data["frames"]) == 24
    assert all(len(f["turn"]) == 16 and len(f["shift"]) == 16 for f in data["frames"])
    assert np.isfinite(np.array([f["shift"] for f in data["frames"]])).all()


def test_trainer_select_backward_variants():
    """select_backward (trainer.h:324; variant equality, test_trainer.cpp:56-125): every
    tuning, deterministic or atomic, gives the default's first-step gradients (within float
    summation order), and unknown names are refused."""
    rc, out = refine_selftest("variants")
    assert rc == 0, out


@pytest.mark.parametrize("views", ["1", "4"])
def test_training_converges(views):
    """test_training_converges (test_trainer.cpp:890-897) through gs::Trainer: the known-scene
    fit of train_selftest.cpp:692-739 (96x72, 24 masked views, 60 gaussians, 600 steps) ends
    with held-out PSNR above 35 dB and 8 dB above its start; also with 4 views per step."""
    rc, out = refine_selftest("converge", views)
    assert rc == 0, out
    m = json.loads(next(line for line in out.splitlines() if line.startswith('{"views_per_step"')))
    assert m["psnr_after"] > 35.0 and m["psnr_after"] > m["psnr_before"] + 8.0, out
