"""JPEG frames in capture folders, decoded on the GPU by nvJPEG (GPU only).

The reference decodes its photos with stb_image (engine/src/image_io.cpp:27-30); here
libgs_host hands JPEG files to nvJPEG. A capture of JPEG frames (baseline 4:4:4, baseline
4:2:0 and progressive) is loaded through gs::load_dataset and each frame compared with an
independent decoder's output (Pillow's libjpeg). JPEG leaves decoders free in their inverse
DCT's rounding and in how they upsample subsampled chroma (libjpeg interpolates, others
replicate), so the check is on luma, which is never subsampled: mean difference under one
level and 99% of the pixels within 3 levels (luma computed from RGB also moves where a
decoder's chroma pushes a saturated colour past 0 or 255 and it is clipped: a few pixels
on the edge of the test image's disc); and, for 4:4:4, RGB within a mean of one level and 6
levels everywhere.
"""
import io
import json
import os
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SELFTEST = os.path.join(ROOT, "on-divice-gsplate_b200", "bin", "gs_host_selftest")
W, H = 96, 64


def smooth_image(rng):
    y, x = np.mgrid[0:H, 0:W].astype(np.float64)
    img = np.stack([128 + 100 * np.sin(x / 13 + rng.uniform(0, 6)), 128 + 90 * np.cos(y / 9 + rng.uniform(0, 6)),
                    128 + 80 * np.sin((x + y) / 17 + rng.uniform(0, 6))], -1)
    cx, cy = rng.uniform(20, 76), rng.uniform(15, 50)
    img[(x - cx) ** 2 + (y - cy) ** 2 < 150] = rng.uniform(0, 255, 3)
    return np.clip(img, 0, 255).astype(np.uint8)


@pytest.mark.parametrize("kind", ["444", "420", "progressive"])
def test_jpeg_frames_decode_on_the_gpu(tmp_path, kind):
    from PIL import Image

    rng = np.random.default_rng(11)
    frames, decoded = [], []
    for i in range(4):
        img = smooth_image(rng)
        buf = io.BytesIO()
        opts = {"quality": 92, "subsampling": 0 if kind == "444" else 2, "progressive": kind == "progressive"}
        Image.fromarray(img).save(buf, "JPEG", **opts)
        (tmp_path / f"f{i}.jpg").write_bytes(buf.getvalue())
        decoded.append(np.asarray(Image.open(io.BytesIO(buf.getvalue())).convert("RGB")))
        c2w = np.eye(4)
        c2w[:3, 3] = [3 * np.sin(i), 0.5, 3 * np.cos(i)]
        frames.append({"file_path": f"f{i}.jpg", "transform_matrix": c2w.tolist()})
    meta = {"w": W, "h": H, "fl_x": 80.0, "frames": frames}
    (tmp_path / "transforms.json").write_text(json.dumps(meta))
    out = subprocess.run([SELFTEST, "dataset", str(tmp_path), "1000", "64"], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stderr
    s = json.loads(out.stdout)
    assert s["frames"] == 4 and s["skipped"] == 0, s
    got = np.frombuffer((tmp_path / "frame0.rgba").read_bytes(), np.uint8).reshape(H, W, 4)
    assert (got[..., 3] == 255).all()
    luma = np.array([0.299, 0.587, 0.114])
    dy = np.abs(got[..., :3].astype(np.float64) @ luma - decoded[0].astype(np.float64) @ luma)
    assert dy.mean() < 1.0 and np.quantile(dy, 0.99) <= 3.0, (dy.mean(), np.quantile(dy, 0.99))
    if kind == "444":
        diff = np.abs(got[..., :3].astype(int) - decoded[0].astype(int))
        assert diff.mean() < 1.0 and diff.max() <= 6, (diff.mean(), diff.max())


def test_broken_jpeg_frames_are_skipped(tmp_path):
    """A damaged JPEG is skipped and listed like any unreadable frame (the loader's rule for
    damaged downloads), and the capture still loads."""
    from PIL import Image

    rng = np.random.default_rng(12)
    frames = []
    for i in range(4):
        buf = io.BytesIO()
        Image.fromarray(smooth_image(rng)).save(buf, "JPEG", quality=90)
        data = buf.getvalue()
        if i == 2:
            data = data[:40]
        (tmp_path / f"f{i}.jpg").write_bytes(data)
        c2w = np.eye(4)
        c2w[:3, 3] = [3 * np.sin(i), 0.5, 3 * np.cos(i)]
        frames.append({"file_path": f"f{i}.jpg", "transform_matrix": c2w.tolist()})
    (tmp_path / "transforms.json").write_text(json.dumps({"w": W, "h": H, "fl_x": 80.0, "frames": frames}))
    out = subprocess.run([SELFTEST, "dataset", str(tmp_path), "1000", "64"], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stderr
    s = json.loads(out.stdout)
    assert s["frames"] == 3 and s["skipped"] == 1 and "f2.jpg" in s["skipped_why"][0]
