"""Seeded synthetic scenes and camera sets.

No public dataset is available: every benchmark and test scene is drawn from a seeded
numpy generator (PCG64) with the shapes, sizes and value distributions the workloads
name, and targets are rendered from a ground-truth scene or drawn as noise.

- `make_scene`: N gaussians with means uniform in a ball, log-scales N(mu, sigma) per
  axis, rotations uniform on S^3, opacity logits N(0, 1), and either DC ~ U(0, 1) (SH
  degree 0) or all SH coefficients ~ N(0, 0.2).
- `make_test_scene` / `make_test_dataset`: the distributions of the reference's test
  fixtures (train_selftest.cpp:285-332), drawn with numpy instead of std::mt19937.
- `orbit_cameras`: cameras on a circle looking at the origin through `look_at_c2w_gl`
  and `dataset_camera`.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from .frame import Camera, dataset_camera, look_at_c2w_gl, sh_rest_coeffs


@dataclass
class Scene:
    """Gaussians in the reference's slot layout: params (n, 16), sh (n, stride)."""

    params: np.ndarray
    sh: np.ndarray
    degree: int

    @property
    def count(self) -> int:
        return self.params.shape[0]


def pack_params(positions, log_scales, rotations, opacity_logits, sh_dc) -> np.ndarray:
    n = positions.shape[0]
    p = np.zeros((n, 16), np.float32)
    p[:, 0:3] = positions
    p[:, 3] = opacity_logits
    p[:, 4:7] = log_scales
    p[:, 7] = 1.0
    p[:, 8:12] = rotations
    p[:, 12:15] = sh_dc
    return p


def make_scene(n: int, seed: int, degree: int, radius: float = 1.0, log_scale_mu: float = -4.0,
               log_scale_sigma: float = 0.5, sh_sigma: float | None = None) -> Scene:
    """Gaussians as the benchmark workloads describe them (see the module docstring)."""
    rng = np.random.default_rng(seed)
    u = rng.normal(size=(n, 3))
    u /= np.linalg.norm(u, axis=1, keepdims=True)
    r = radius * rng.random(n) ** (1.0 / 3.0)
    positions = (u * r[:, None]).astype(np.float32)
    log_scales = rng.normal(log_scale_mu, log_scale_sigma, size=(n, 3)).astype(np.float32)
    q = rng.normal(size=(n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    opacity = rng.normal(0.0, 1.0, size=n).astype(np.float32)
    coeffs = sh_rest_coeffs(degree)
    if degree == 0 and sh_sigma is None:
        dc = rng.random((n, 3)).astype(np.float32)
        rest = np.zeros((n, 0), np.float32)
    else:
        s = 0.2 if sh_sigma is None else sh_sigma
        dc = rng.normal(0.0, s, size=(n, 3)).astype(np.float32)
        rest = rng.normal(0.0, s, size=(n, coeffs * 3)).astype(np.float32)
    return Scene(pack_params(positions, log_scales, q.astype(np.float32), opacity, dc), rest, degree)


def make_test_scene(n: int, degree: int, seed: int) -> Scene:
    """The distributions of make_test_scene (train_selftest.cpp:314-332)."""
    rng = np.random.default_rng(seed)
    U = lambda *shape: rng.uniform(-1.0, 1.0, size=shape).astype(np.float32)  # noqa: E731
    positions = 0.7 * U(n, 3)
    log_scales = np.log(0.08 + 0.06 * U(n, 3)).astype(np.float32)
    dc = 0.8 * U(n, 3)
    rot = U(n, 4)
    rot[:, 0] += 1.5
    opacity = 0.6 * U(n) - 0.2
    rest = 0.25 * U(n, sh_rest_coeffs(degree) * 3)
    return Scene(pack_params(positions, log_scales, rot, opacity, dc), rest.astype(np.float32), degree)


@dataclass
class Dataset:
    """Frames of one resolution: camera-to-world (OpenGL), RGBA8 targets, hold-out flags."""

    width: int
    height: int
    fx: float
    fy: float
    cx: float
    cy: float
    c2w: list
    rgba: list
    holdout: list
    camera_extent: float

    def camera(self, i: int) -> Camera:
        return dataset_camera(self.c2w[i], self.fx, self.fy, self.cx, self.cy, self.width, self.height)


def make_test_dataset(width: int, height: int, frames: int, masks: bool, seed: int) -> Dataset:
    """make_test_dataset (train_selftest.cpp:285-312): an orbit at 3 m, noise targets,
    every 8th frame held out, camera extent 3.3."""
    rng = np.random.default_rng(seed)
    c2w, rgba, hold = [], [], []
    for i in range(frames):
        angle = 6.2831853 * i / max(frames, 1)
        eye = (3.0 * math.sin(angle), 0.6 + 0.3 * math.sin(3.0 * angle), 3.0 * math.cos(angle))
        c2w.append(look_at_c2w_gl(eye, (0.0, 0.0, 0.0)))
        img = rng.integers(0, 256, size=(height, width, 4), dtype=np.uint8)
        if not masks:
            img[..., 3] = 255
        rgba.append(img)
        hold.append(frames > 1 and i % 8 == 0)
    return Dataset(width, height, 0.9 * width, 0.9 * width, width * 0.5, height * 0.5, c2w, rgba, hold, 3.3)


def orbit_cameras(count: int, radius: float, height: float, width_px: int, height_px: int, focal: float) -> list:
    """`count` cameras evenly spaced on a circle of `radius` at `height`, looking at the origin."""
    cams = []
    for i in range(count):
        a = 2.0 * math.pi * i / count
        eye = (radius * math.sin(a), height, radius * math.cos(a))
        cams.append(dataset_camera(look_at_c2w_gl(eye, (0.0, 0.0, 0.0)), focal, focal, width_px * 0.5,
                                   height_px * 0.5, width_px, height_px))
    return cams


def front_camera(width: int, height: int, focal: float, distance: float = 3.0) -> Camera:
    """A pinhole at (0, 0, distance) looking at the origin."""
    return dataset_camera(look_at_c2w_gl((0.0, 0.0, distance), (0.0, 0.0, 0.0)), focal, focal, width * 0.5,
                          height * 0.5, width, height)
