"""The C++ host layer (libgs_host: gs::Trainer, scenes, datasets) on CPU.

Runs the in-tree bin/gs_host_selftest: PLY round trips (bit-exact), SPZ v3/v2 round trips
(within the format's quantization; the layout is the published one, no SPZ files from
other writers are available here), axis conversion, and the
FrameData the C++ trainer writes compared word for word with the Python mirror
(gs_b200.frame.make_frame, itself pinned to the oracle by the GPU parity tests).
"""
import json
import os
import struct
import subprocess

import numpy as np
import pytest

from gs_b200 import frame as F
from gs_b200 import scenes as S

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "on-divice-gsplate_b200", "bin")
SELFTEST = os.path.join(BIN, "gs_host_selftest")


def run(*args):
    if not os.path.exists(SELFTEST):
        pytest.fail("bin/gs_host_selftest is not built (make -C on-divice-gsplate_b200)")
    out = subprocess.run([SELFTEST, *args], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stderr
    return out.stdout


def test_ply_round_trip_and_axis_conversion(tmp_path):
    assert run("scene", str(tmp_path)).strip() == "ok"
    # The written file is a standard 3DGS PLY: header properties in the standard order.
    head = open(tmp_path / "scene_3.ply", "rb").read(4096).split(b"end_header\n")[0].decode()
    props = [line.split()[-1] for line in head.splitlines() if line.startswith("property")]
    assert props[:9] == ["x", "y", "z", "nx", "ny", "nz", "f_dc_0", "f_dc_1", "f_dc_2"]
    assert props[9:54] == [f"f_rest_{i}" for i in range(45)]
    assert props[54:] == ["opacity", "scale_0", "scale_1", "scale_2", "rot_0", "rot_1", "rot_2", "rot_3"]


def test_camera_matches_python_mirror():
    vals = np.array([float(v) for v in run("camera").split()], np.float32)
    cam = S.front_camera(360, 640, 500.0)
    np.testing.assert_allclose(vals[:9], cam.rotation.reshape(-1), atol=1e-7)
    np.testing.assert_allclose(vals[9:], cam.translation, atol=1e-6)


@pytest.mark.parametrize("step", [0, 7, 4000])
def test_batch_frames_equal_single_frames(step):
    """make_frames gives the same bytes as make_frame per camera, for views of mixed sizes."""
    cams = S.orbit_cameras(5, 3.0, 0.5, 1920, 1080, 1400.0) + [S.front_camera(37, 23, 50.0),
                                                               S.front_camera(360, 640, 500.0)]
    opt = F.TrainOptions(iterations=30000, sh_degree=3, sh_degree_interval=1000, lambda_dssim=0.2,
                         lambda_dssim_end=0.1, opacity_reset_interval=3000)
    for masked, ssim, cap in [(False, True, 0), (True, False, 12345)]:
        want = np.concatenate([F.make_frame(c, 70000, 45, step, opt, (0.1, 0.2, 0.3), 3.3, masked, ssim, cap)
                               for c in cams])
        got = F.make_frames(cams, 70000, 45, step, opt, (0.1, 0.2, 0.3), 3.3, masked, ssim, cap)
        assert got.dtype == F.FRAME_DTYPE and got.shape == (len(cams),)
        np.testing.assert_array_equal(got.view(np.uint32), want.view(np.uint32))
    assert F.make_frames([], 1, 0, 0, opt, (0.0, 0.0, 0.0), 1.0).shape == (0,)


def test_frame_matches_python_mirror():
    words = np.array([int(w, 16) for w in run("frame").split()], np.uint32)
    assert words.size == 72
    cam = S.front_camera(360, 640, 500.0)
    ref = F.make_frame(cam, 20000, 45, 10, F.TrainOptions(), (0.1, 0.2, 0.3), 3.3).view(np.uint32).reshape(-1)
    got = words.view(np.float32)
    want = ref.view(np.float32)
    # Integer words (image, model, limits, the seed) exactly; float words to float rounding
    # (the position learning rate's decay and the loss weight are computed in float here, as
    # the reference does, and in double by the mirror).
    integer = np.zeros(72, bool)
    for name in ("image", "model", "limits"):
        off = F.FRAME_DTYPE.fields[name][1] // 4
        integer[off:off + 4] = True
    integer[F._SEED_WORD] = True
    np.testing.assert_array_equal(words[integer], ref[integer])
    np.testing.assert_allclose(got[~integer], want[~integer], rtol=2e-6, atol=0)


def head_region_numpy(p, up):
    """estimate_head (dataset.cpp:252-289) restated in float32 numpy: the top 13% of the
    extent along up (lowest 1% and highest 0.5% ignored), centre at the slab's per-axis
    median off the up axis, 8.5% of the extent below the top; radius a tenth of the extent."""
    n = len(p)
    up = np.asarray(up, np.float32)
    h = (p[:, 0] * up[0] + p[:, 1] * up[1]) + p[:, 2] * up[2]
    s = np.sort(h)
    lo, hi = s[n // 100], s[n - 1 - n // 200]
    extent = np.float32(hi - lo)
    if not extent >= 1.0:
        return None
    slab = np.float32(hi - np.float32(0.13) * extent)
    sel = (h >= slab) & (h <= hi)
    across = p[sel] - h[sel, None] * up[None, :]
    level = np.float32(hi - np.float32(0.085) * extent)
    center = np.array([np.sort(across[:, k])[sel.sum() // 2] + level * up[k] for k in range(3)], np.float32)
    return center, np.float32(0.1) * extent, extent


def standing_person(rng, n=6000):
    """Points on a 1.75-tall figure: a body cylinder, a head sphere and a few strays."""
    body = n * 4 // 5
    a = rng.uniform(0, 2 * np.pi, body)
    y = rng.uniform(0.0, 1.5, body)
    pts = [np.stack([0.2 * np.cos(a) + 0.1, y, 0.2 * np.sin(a) - 0.05], 1)]
    d = rng.normal(size=(n - body - 20, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    pts.append(np.array([0.1, 1.62, -0.05]) + 0.12 * d)
    pts.append(rng.uniform(-3, 3, (20, 3)))
    return np.concatenate(pts).astype(np.float32)


@pytest.mark.parametrize("axis", [1, 2])
def test_head_region_matches_numpy_restatement(tmp_path, axis):
    rng = np.random.default_rng(7)
    p = standing_person(rng)
    up = np.zeros(3, np.float32)
    up[axis] = 1.0
    if axis == 2:  # the same figure standing along z
        p = p[:, [0, 2, 1]].copy()
        p[:, 1] *= -1.0
    f = tmp_path / "xyz.f32"
    f.write_bytes(p.tobytes())
    out = run("head", str(f), *[str(float(u)) for u in up], "3.0")
    import json
    got = json.loads(out)
    want = head_region_numpy(p, up)
    assert got["found"] and want is not None
    np.testing.assert_allclose(got["center"], want[0], rtol=1e-6, atol=1e-6)
    np.testing.assert_allclose([got["radius"], got["height"]], [want[1], want[2]], rtol=1e-6)
    # The head lands on the figure's head sphere.
    assert abs(got["center"][axis] - (1.62 - np.float32(0.0))) < 0.1
    # FrameData words for the test camera (write_frame, trainer.cpp:531-544): the projected
    # centre and radius, the weight (the head is small in a 640-tall view), 1 / gain.
    cam = S.front_camera(360, 640, 500.0)
    t = cam.rotation.reshape(3, 3).astype(np.float64) @ np.asarray(got["center"]) + cam.translation
    want_head = [cam.fx * t[0] / t[2] + cam.cx, cam.fy * t[1] / t[2] + cam.cy, cam.fx * got["radius"] / t[2], 3.0]
    np.testing.assert_allclose(got["frame_head"], want_head, rtol=1e-5)
    np.testing.assert_allclose(got["frame_exposure"], [1 / 0.8, 1.0, 1 / 1.25], rtol=1e-7)


def test_no_head_region_for_small_or_sparse_subjects(tmp_path):
    rng = np.random.default_rng(8)
    small = standing_person(rng) * np.float32(0.5)  # under 1 unit tall: a close-up
    f = tmp_path / "xyz.f32"
    f.write_bytes(small.tobytes())
    import json
    got = json.loads(run("head", str(f), "0", "1", "0", "3.0"))
    assert not got["found"] and got["frame_head"] == [0, 0, 0, 1]
    f.write_bytes(standing_person(rng)[:150].tobytes())  # under 200 points
    assert not json.loads(run("head", str(f), "0", "1", "0", "3.0"))["found"]


def test_refinement_arithmetic():
    """The trainer's pose, exposure and motion-rig arithmetic on the CPU: rotation
    exp/log/composition/slerp, a correction followed by steps against the composed camera,
    Adam's first step, capture-order spans, centred and blended gains, node placement, and
    the rig energies' gradients against central differences (to 1e-5 of the largest)."""
    m = json.loads(run("refine").strip().splitlines()[-1])
    assert m["rotation_err"] < 1e-9 and m["rig_gradient_err"] < 1e-5
