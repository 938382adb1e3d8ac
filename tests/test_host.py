"""The C++ host layer (libgs_host: gs::Trainer, scenes, datasets) on CPU.

Runs the in-tree bin/gs_host_selftest: PLY round trips (bit-exact), SPZ v3/v2 round trips
(within the format's quantization; the layout is the published one, no SPZ files from
other writers are available here), axis conversion, and the
FrameData the C++ trainer writes compared word for word with the Python mirror
(gs_b200.frame.make_frame, itself pinned to the oracle by the GPU parity tests).
"""
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
