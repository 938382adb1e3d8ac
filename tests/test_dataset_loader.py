"""Capture-folder loading (gs::load_dataset) and initial gaussians (gs::initialize_gaussians) on CPU.

Writes a small transforms.json capture with PNG images of every colour type the loader
reads (RGB, RGBA 16-bit, palette, grey + alpha) using every PNG row filter, grey masks, a
point-cloud PLY and one damaged JPEG frame, then checks what bin/gs_host_selftest reports
against the reference's rules (dataset.cpp:85-223, 291-523): short side resized to the
target width by area, intrinsics scaled with it, masks in alpha, every 8th frame held out,
unreadable frames skipped and listed, points merged per voxel to the budget; and the depth
source of the initial gaussians (16-bit PNG and PGM depth maps with confidence maps,
back-projected through each frame's camera). Decoding real JPEG frames needs the GPU
(nvJPEG): tests/test_gpu_jpeg.py.
"""
import json
import os
import struct
import subprocess
import zlib

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SELFTEST = os.path.join(ROOT, "on-divice-gsplate_b200", "bin", "gs_host_selftest")
W, H = 45, 30


def _chunk(kind, data):
    return struct.pack(">I", len(data)) + kind + data + struct.pack(">I", zlib.crc32(kind + data) & 0xFFFFFFFF)


def _paeth(a, b, c):
    p = a + b - c
    pa, pb, pc = np.abs(p - a), np.abs(p - b), np.abs(p - c)
    return np.where((pa <= pb) & (pa <= pc), a, np.where(pb <= pc, b, c))


def write_png(path, samples, colour_type, depth=8, palette=None, alpha=None):
    """samples: H x W x channels array of the file's samples (uint8 or uint16)."""
    h, w = samples.shape[:2]
    raw = samples.astype(">u2" if depth == 16 else np.uint8).reshape(h, -1).view(np.uint8).astype(np.int32)
    bpp = raw.shape[1] // w
    rows = []
    for y in range(h):
        x = raw[y]
        up = raw[y - 1] if y > 0 else np.zeros_like(x)
        left = np.concatenate([np.zeros(bpp, np.int32), x[:-bpp]])
        upleft = np.concatenate([np.zeros(bpp, np.int32), up[:-bpp]])
        f = y % 5  # every filter type in turn
        pred = [0, left, up, (left + up) // 2, _paeth(left, up, upleft)][f]
        rows.append(bytes([f]) + ((x - pred) % 256).astype(np.uint8).tobytes())
    ihdr = struct.pack(">IIBBBBB", w, h, depth, colour_type, 0, 0, 0)
    out = b"\x89PNG\r\n\x1a\n" + _chunk(b"IHDR", ihdr)
    if palette is not None:
        out += _chunk(b"PLTE", palette.astype(np.uint8).tobytes())
    if alpha is not None:
        out += _chunk(b"tRNS", alpha.astype(np.uint8).tobytes())
    out += _chunk(b"IDAT", zlib.compress(b"".join(rows))) + _chunk(b"IEND", b"")
    open(path, "wb").write(out)


def area_resize(img, ow, oh):
    """Coverage-weighted mean resampling, in float64."""
    def weights(n, o):
        m = np.zeros((o, n))
        s = n / o
        for i in range(o):
            lo, hi = i * s, (i + 1) * s
            for j in range(int(np.floor(lo)), min(n, int(np.ceil(hi)))):
                m[i, j] = (min(hi, j + 1) - max(lo, j)) / s
        return m
    wy, wx = weights(img.shape[0], oh), weights(img.shape[1], ow)
    return np.einsum("yi,ijc,xj->yxc", wy, img.astype(np.float64), wx)


def make_capture(d, rng, with_points=True, n_frames=10):
    frames, rgba = [], []
    for i in range(n_frames):
        name = f"img_{i:02d}.png"
        full = rng.integers(0, 256, (H, W, 4), dtype=np.uint16).astype(np.uint8)
        full[..., 3] = 255
        if i == 3:  # RGBA, 16 bits per sample (the loader keeps the high byte)
            s16 = full.astype(np.uint16) * 257 + rng.integers(0, 256, full.shape).astype(np.uint16) % 1
            write_png(d / name, s16, 6, depth=16)
        elif i == 5:  # palette
            pal = rng.integers(0, 256, (16, 3))
            idx = rng.integers(0, 16, (H, W, 1))
            full[..., :3] = pal[idx[..., 0]]
            write_png(d / name, idx, 3, palette=pal)
        elif i == 7:  # grey + alpha
            g = rng.integers(0, 256, (H, W, 2))
            full[..., 0] = full[..., 1] = full[..., 2] = g[..., 0]
            write_png(d / name, g, 4)
        elif i == 8:  # a damaged JPEG: skipped
            name = f"img_{i:02d}.jpg"
            open(d / name, "wb").write(b"\xff\xd8\xff\xe0" + bytes(64))
        else:
            write_png(d / name, full[..., :3], 2)
        mask = rng.integers(0, 256, (H, W, 1))
        write_png(d / f"mask_{i:02d}.png", mask, 0)
        full[..., 3] = mask[..., 0]
        a = 2 * np.pi * i / n_frames
        eye = np.array([3 * np.sin(a), 0.5, 3 * np.cos(a)])
        c2w = np.eye(4)
        c2w[:3, 3] = eye
        frames.append({"file_path": name, "mask_path": f"mask_{i:02d}.png", "transform_matrix": c2w.tolist()})
        rgba.append(full)
    meta = {"w": W, "h": H, "fl_x": 40.0, "fl_y": 41.0, "cx": 22.0, "cy": 15.5, "frames": frames}
    if with_points:
        pts = rng.normal(size=(500, 3)).astype(np.float32)
        col = rng.integers(0, 256, (500, 3)).astype(np.uint8)
        head = ("ply\nformat binary_little_endian 1.0\nelement vertex 500\nproperty float x\nproperty float y\n"
                "property float z\nproperty uchar red\nproperty uchar green\nproperty uchar blue\nend_header\n")
        rec = np.zeros(500, dtype=[("p", "<f4", 3), ("c", "u1", 3)])
        rec["p"], rec["c"] = pts, col
        open(d / "points.ply", "wb").write(head.encode() + rec.tobytes())
        meta["ply_file_path"] = "points.ply"
    (d / "transforms.json").write_text(json.dumps(meta))
    return rgba


def load(d, width, max_init):
    if not os.path.exists(SELFTEST):
        pytest.fail("bin/gs_host_selftest is not built (make -C on-divice-gsplate_b200)")
    out = subprocess.run([SELFTEST, "dataset", str(d), str(width), str(max_init)], capture_output=True, text=True,
                         timeout=120)
    assert out.returncode == 0, out.stderr
    return json.loads(out.stdout)


def test_capture_folder(tmp_path):
    rng = np.random.default_rng(3)
    rgba = make_capture(tmp_path, rng)
    s = load(tmp_path, 20, 100)
    # Short side 30 -> 20: scale 2/3.
    assert (s["width"], s["height"]) == (30, 20)
    np.testing.assert_allclose([s["fx"], s["fy"], s["cx"], s["cy"]], [40 * 2 / 3, 41 * 2 / 3, 22 * 2 / 3, 15.5 * 2 / 3],
                               rtol=1e-5)
    assert s["frames"] == 9 and s["skipped"] == 1 and "img_08.jpg" not in s["names"]
    assert s["holdout"] == 1  # frame 0 (frame 8, also every 8th, was skipped)
    assert s["has_masks"] and s["points"] == 500 and s["name"] == tmp_path.name
    got = np.frombuffer(open(tmp_path / "frame0.rgba", "rb").read(), np.uint8).reshape(20, 30, 4)
    want = np.rint(area_resize(rgba[0], 30, 20))
    assert np.abs(got.astype(int) - want).max() <= 1
    # 500 points over a budget of 100: merged per voxel to at most 100.
    assert s["init_source"] == "points" and s["init_raw"] == 500
    assert 0 < s["init_count"] <= 100 and s["init_voxel"] > 0
    assert np.isfinite([s["log_scale_min"], s["log_scale_max"]]).all() and s["log_scale_min"] <= s["log_scale_max"]
    np.testing.assert_allclose(s["init_opacity_logit"], np.log(0.2 / 0.8), rtol=1e-5)


def test_capture_without_points_or_upscaling(tmp_path):
    rng = np.random.default_rng(4)
    rgba = make_capture(tmp_path, rng, with_points=False)
    s = load(tmp_path, 100, 64)  # never enlarged: stays 45 x 30
    assert (s["width"], s["height"]) == (W, H)
    got = np.frombuffer(open(tmp_path / "frame0.rgba", "rb").read(), np.uint8).reshape(H, W, 4)
    np.testing.assert_array_equal(got, rgba[0])
    assert s["init_source"] == "random" and s["init_count"] == 64


def test_png_colour_types_decode_exactly(tmp_path):
    """Frames 3 (RGBA 16-bit), 5 (palette) and 7 (grey + alpha) at full size equal their sources."""
    rng = np.random.default_rng(5)
    rgba = make_capture(tmp_path, rng)
    original = json.loads((tmp_path / "transforms.json").read_text())
    for i in (3, 5, 7):
        meta = dict(original)
        meta["frames"] = [original["frames"][i]] * 2
        (tmp_path / "transforms.json").write_text(json.dumps(meta))
        s = load(tmp_path, 100, 10)
        assert s["frames"] == 2
        got = np.frombuffer(open(tmp_path / "frame0.rgba", "rb").read(), np.uint8).reshape(H, W, 4)
        np.testing.assert_array_equal(got, rgba[i], err_msg=f"frame {i}")


def _depth_frames(d, rng, meta, dw=15, dh=10):
    """Adds a depth map (16-bit PNG, or 16-bit PGM for frame 4) and a confidence map to every
    frame of the capture in `d`; returns them as {frame: (depth16, confidence)}."""
    maps = {}
    for i, fr in enumerate(meta["frames"]):
        depth = (1500 + rng.integers(0, 1000, (dh, dw))).astype(np.uint16)
        depth[rng.random((dh, dw)) < 0.1] = 0  # missing samples
        conf = rng.integers(0, 256, (dh, dw, 1)).astype(np.uint8)
        if i == 4:
            name = f"depth_{i:02d}.pgm"
            open(d / name, "wb").write(b"P5\n%d %d\n65535\n" % (dw, dh) + depth.astype(">u2").tobytes())
        else:
            name = f"depth_{i:02d}.png"
            write_png(d / name, depth[..., None], 0, depth=16)
        write_png(d / f"conf_{i:02d}.png", conf, 0)
        fr["depth_file_path"] = name
        fr["depth_confidence_path"] = f"conf_{i:02d}.png"
        maps[i] = (depth, conf[..., 0])
    meta["depth_unit_scale_factor"] = 0.001
    (d / "transforms.json").write_text(json.dumps(meta))
    return maps


def test_depth_initialisation(tmp_path):
    """initialize_gaussians from depth maps (dataset.cpp:297-320's source): every confident
    sample of a training frame inside the subject mask, back-projected through the frame's
    camera, and nothing else; log-scales from the 3 nearest neighbours."""
    rng = np.random.default_rng(6)
    rgba = make_capture(tmp_path, rng, with_points=True)
    meta = json.loads((tmp_path / "transforms.json").read_text())
    maps = _depth_frames(tmp_path, rng, meta)
    s = load(tmp_path, 100, 100000)
    assert s["has_depth"] and s["init_source"] == "depth"
    want = []
    fx, fy, cx, cy = 40.0, 41.0, 22.0, 15.5
    for i, (depth, conf) in maps.items():
        if i % 8 == 0 or i == 8:  # held out, or skipped (the JPEG frame)
            continue
        c2w = np.array(meta["frames"][i]["transform_matrix"])
        dh, dw = depth.shape
        for v in range(dh):
            for u in range(dw):
                z = np.float32(float(depth[v, u]) * 0.001)
                if not z > 0 or conf[v, u] < np.float32(0.3) * np.float32(255.0):
                    continue
                px, py = (u + 0.5) * W / dw, (v + 0.5) * H / dh
                if rgba[i][min(H - 1, int(py)), min(W - 1, int(px)), 3] < 128:
                    continue
                x, y = (px - cx) / fx * z, (py - cy) / fy * z
                want.append(c2w[:3, 0] * x - c2w[:3, 1] * y - c2w[:3, 2] * z + c2w[:3, 3])
    want = np.array(want)
    got = np.frombuffer(open(tmp_path / "init.xyz", "rb").read(), np.float32).reshape(-1, 3)
    assert s["init_raw"] == len(want) == len(got) > 100
    order_w = np.lexsort(want.T[::-1])
    order_g = np.lexsort(got.T[::-1])
    np.testing.assert_allclose(got[order_g], want[order_w], atol=2e-5)
    # Scales: the mean distance to the 3 nearest other points, clamped to [1e-4, 0.02] x
    # the robust extent (0.5%..99.5% box diagonal).
    d = np.sqrt(((got[:, None, :].astype(np.float64) - got[None, :, :]) ** 2).sum(-1))
    np.fill_diagonal(d, np.inf)
    mean3 = np.sort(d, axis=1)[:, :3].mean(1)
    lo = np.sort(got, axis=0)[len(got) // 200]
    hi = np.sort(got, axis=0)[len(got) - 1 - len(got) // 200]
    extent = np.sqrt(((hi.astype(np.float64) - lo) ** 2).sum())
    want_scale = np.log(np.clip(mean3, 1e-4 * extent, 0.02 * extent))
    logscale = np.frombuffer(open(tmp_path / "init.logscale", "rb").read(), np.float32).reshape(-1, 3)
    np.testing.assert_allclose(logscale[:, 0], want_scale, atol=1e-4)


def test_depth_merge_to_budget(tmp_path):
    """Over budget, depth points are merged per occupied cell to at most max_gaussians and
    close under it (the cell size is fitted to the budget)."""
    rng = np.random.default_rng(7)
    make_capture(tmp_path, rng, with_points=False)
    meta = json.loads((tmp_path / "transforms.json").read_text())
    _depth_frames(tmp_path, rng, meta, dw=45, dh=30)
    for budget in (50, 400, 1500):
        s = load(tmp_path, 100, budget)
        assert s["init_source"] == "depth" and s["init_raw"] > budget
        assert 0.5 * budget <= s["init_count"] <= budget and s["init_voxel"] > 0, (budget, s["init_count"])
