"""FrameData, cameras and training-option schedules of the reference's host code.

FrameData (train_common.glsl:15-37) is filled as `Trainer::write_frame` fills it
(engine/src/trainer.cpp:440-547); cameras follow `gs::Camera` (engine/include/gs/camera.h)
and `dataset_camera` (engine/src/dataset.cpp:226-250); the option defaults and schedules
follow `TrainOptions` (engine/include/gs/trainer.h:20-167), `scaled_options`
(trainer.cpp:133-145), `sh_degree_at` / `lambda_at` (trainer.cpp:427-438).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

FRAME_DTYPE = np.dtype([
    ("rot", "<f4", (3, 4)),
    ("cam_pos", "<f4", (4,)),
    ("intrinsics", "<f4", (4,)),
    ("image", "<u4", (4,)),
    ("model", "<u4", (4,)),
    ("background", "<f4", (4,)),
    ("lr0", "<f4", (4,)),
    ("lr1", "<f4", (4,)),
    ("adam", "<f4", (4,)),
    ("bias", "<f4", (4,)),
    ("densify0", "<f4", (4,)),
    ("densify1", "<f4", (4,)),
    ("limits", "<u4", (4,)),
    ("loss", "<f4", (4,)),
    ("head", "<f4", (4,)),
    ("exposure", "<f4", (4,)),
])
assert FRAME_DTYPE.itemsize == 288
_SEED_WORD = FRAME_DTYPE.fields["densify1"][1] // 4 + 1

TILE = 16
FLAG_MASKED_TARGET = 1
FLAG_SSIM = 4
FLAG_POSE_GRAD = 8  # sum the view's camera pose gradient (StepResult.pose_grad)
FLAG_POSE_ONLY = 16  # on the first view: gradients only, the model and its statistics stay
FLAG_MOTION = 32  # the gaussians follow the view's node motions (Context.set_view_motion)
FLAG_MOTION_GRAD = 64  # sum the gradient per motion node (Context.motion_gradient)
FLAG_SPARSE_ADAM = 128
BETA1, BETA2, EPSILON = 0.9, 0.999, 1e-15  # trainer.cpp:68-70


def sh_rest_coeffs(degree: int) -> int:
    return 0 if degree == 0 else (degree + 1) * (degree + 1) - 1


@dataclass
class Camera:
    """gs::Camera: scene -> camera rotation (row-major, OpenCV axes), translation, centre."""

    rotation: np.ndarray
    translation: np.ndarray
    position: np.ndarray
    fx: float
    fy: float
    cx: float
    cy: float
    width: int
    height: int

    def as_dict(self) -> dict:
        return {"rotation": self.rotation, "translation": self.translation, "position": self.position,
                "fx": self.fx, "fy": self.fy, "cx": self.cx, "cy": self.cy}


def look_at_c2w_gl(eye, target) -> np.ndarray:
    """OpenGL camera-to-world looking from `eye` at `target`, world up +y
    (train_selftest.cpp:152-174)."""
    eye = np.asarray(eye, np.float32)
    f = np.asarray(target, np.float32) - eye
    f = f / np.float32(np.sqrt(np.sum(f * f)))
    up = np.array([0, 1, 0], np.float32)
    r = np.cross(f, up).astype(np.float32)
    r = r / np.float32(np.sqrt(np.sum(r * r)))
    u = np.cross(r, f).astype(np.float32)
    c2w = np.eye(4, dtype=np.float32)
    c2w[:3, 0] = r
    c2w[:3, 1] = u
    c2w[:3, 2] = -f
    c2w[:3, 3] = eye
    return c2w


def dataset_camera(c2w_gl: np.ndarray, fx: float, fy: float, cx: float, cy: float, width: int, height: int) -> Camera:
    """OpenGL camera-to-world -> OpenCV world-to-camera (dataset.cpp:226-250)."""
    rot_cv = np.empty((3, 3), np.float32)
    rot_cv[:, 0] = c2w_gl[:3, 0]
    rot_cv[:, 1] = -c2w_gl[:3, 1]
    rot_cv[:, 2] = -c2w_gl[:3, 2]
    rotation = rot_cv.T.copy()
    position = c2w_gl[:3, 3].astype(np.float32).copy()
    translation = -(rotation @ position).astype(np.float32)
    return Camera(rotation, translation, position, float(fx), float(fy), float(cx), float(cy), int(width), int(height))


@dataclass
class TrainOptions:
    """The subset of gs::TrainOptions (trainer.h:20-167) the training step reads."""

    iterations: int = 3000
    max_gaussians: int = 300000
    sh_degree: int = 3
    sh_degree_interval: int = 500
    masked: bool = True
    random_background: bool = True
    background: tuple = (0.0, 0.0, 0.0)
    lr_position: float = 1.6e-4
    lr_position_final: float = 1.6e-6
    lr_scale: float = 5e-3
    lr_rotation: float = 1e-3
    lr_opacity: float = 2.5e-2
    lr_sh_dc: float = 2.5e-3
    lr_sh_rest: float = float(np.float32(2.5e-3) / np.float32(20.0))  # 2.5e-3f / 20.0f
    lambda_dssim: float = 0.2
    lambda_dssim_end: float = 1.0
    head_weight: float = 1.0
    sparse_adam: bool = False
    densify_from: int = 300
    densify_until: int = 2000
    densify_interval: int = 100
    opacity_reset_interval: int = 0
    densify_grad_threshold: float = 2e-4
    percent_dense: float = 0.01
    prune_opacity: float = 0.005
    min_pair_capacity: int = 1 << 16
    seed: int = 1

    def sh_degree_at(self, step: int) -> int:
        """trainer.cpp:434-437"""
        return min(self.sh_degree, step // self.sh_degree_interval if self.sh_degree_interval > 0 else self.sh_degree)

    def lambda_at(self, step: int) -> float:
        """trainer.cpp:427-431"""
        if self.lambda_dssim_end < 0.0 or self.iterations <= 1:
            return self.lambda_dssim
        t = min(1.0, step / float(self.iterations - 1))
        return self.lambda_dssim + (self.lambda_dssim_end - self.lambda_dssim) * t

    def uses_ssim(self) -> bool:
        return self.lambda_dssim > 0.0 or self.lambda_dssim_end > 0.0


def scaled_options(iterations: int) -> TrainOptions:
    """trainer.cpp:133-145: the default schedule rescaled to `iterations`."""
    o = TrainOptions()
    scale = iterations / float(o.iterations)
    o.iterations = iterations
    o.densify_from = int(o.densify_from * scale)
    o.densify_until = int(o.densify_until * scale)
    o.opacity_reset_interval = int(o.opacity_reset_interval * scale)
    o.sh_degree_interval = max(1, int(o.sh_degree_interval * scale))
    return o


def frozen_options(degree: int, masked: bool) -> TrainOptions:
    """frozen_train_options (train_selftest.cpp:334-346): all learning rates zero."""
    o = TrainOptions()
    o.iterations = 1
    o.max_gaussians = 0
    o.sh_degree = degree
    o.sh_degree_interval = 0
    o.masked = masked
    o.random_background = False
    o.lr_position = o.lr_position_final = o.lr_scale = o.lr_rotation = 0.0
    o.lr_opacity = o.lr_sh_dc = o.lr_sh_rest = 0.0
    o.densify_from = o.densify_until = 1000000
    o.opacity_reset_interval = 0
    return o


def make_frame(camera: Camera, slots: int, sh_stride: int, step: int, options: TrainOptions, background,
               camera_extent: float, masked_target: bool = False, ssim: bool = True,
               pair_capacity: int = 0) -> np.ndarray:
    """Trainer::write_frame (trainer.cpp:440-547) without pose, motion, exposure or head."""
    f = np.zeros(1, FRAME_DTYPE)
    W, H = camera.width, camera.height
    f["rot"][0, :, :3] = camera.rotation.reshape(3, 3)
    f["rot"][0, :, 3] = camera.translation
    f["cam_pos"][0, :3] = camera.position
    f["intrinsics"][0] = (camera.fx, camera.fy, camera.cx, camera.cy)
    f["image"][0] = (W, H, (W + TILE - 1) // TILE, (H + TILE - 1) // TILE)
    flags = (FLAG_MASKED_TARGET if masked_target else 0) | (FLAG_SSIM if ssim else 0) | \
        (FLAG_SPARSE_ADAM if options.sparse_adam else 0)
    f["model"][0] = (slots, options.sh_degree_at(step), sh_stride, flags)
    f["background"][0, :3] = background
    f["background"][0, 3] = np.float32(1.0) / (np.float32(3.0) * np.float32(W) * np.float32(H))
    t = min(1.0, step / float(options.iterations)) if options.iterations > 0 else 1.0
    lr_pos = np.float32(options.lr_position)
    if options.lr_position > 0.0 and options.lr_position_final > 0.0:
        lr_pos = np.float32(math.exp(math.log(np.float32(options.lr_position)) * (1.0 - t) +
                                     math.log(np.float32(options.lr_position_final)) * t))
    f["lr0"][0] = (lr_pos * np.float32(camera_extent), options.lr_scale, options.lr_rotation, options.lr_opacity)
    f["lr1"][0, :2] = (options.lr_sh_dc, options.lr_sh_rest)
    f["adam"][0, :3] = (BETA1, BETA2, EPSILON)
    # In double from the float constants, as trainer.cpp:510-511 computes them.
    n = float(step) + 1.0
    b1, b2 = float(np.float32(BETA1)), float(np.float32(BETA2))
    f["bias"][0, :2] = (1.0 / (1.0 - b1 ** n), 1.0 / (1.0 - b2 ** n))
    prune_big = options.opacity_reset_interval > 0 and step > options.opacity_reset_interval
    f["densify0"][0] = (options.densify_grad_threshold, options.percent_dense * camera_extent, options.prune_opacity,
                        0.1 * camera_extent if prune_big else 0.0)
    seed = (options.seed * 9781 + step * 6271) & 0xFFFFFFFF
    f["densify1"][0, 0] = 20.0 if prune_big else 0.0
    f["densify1"][0, 2] = 1.6
    # The seed travels as raw uint bits in a float slot (trainer.cpp:519-520).
    f.view(np.uint32)[_SEED_WORD] = seed
    f["limits"][0] = (pair_capacity, 0, 0, pair_capacity)
    f["loss"][0, :3] = (options.lambda_at(step), 0.01 * 0.01, 0.03 * 0.03)
    f["head"][0, 3] = 1.0
    f["exposure"][0, :3] = 1.0
    return f


def make_frames(cameras: list[Camera], slots: int, sh_stride: int, step: int, options: TrainOptions, background,
                camera_extent: float, masked_target: bool = False, ssim: bool = True,
                pair_capacity: int = 0) -> np.ndarray:
    """The frames of one step's views, as make_frame gives them one by one (the same bytes),
    in one FRAME_DTYPE array: the step's schedule is worked out once and the camera fields
    are filled for all views together."""
    if not cameras:
        return np.zeros(0, FRAME_DTYPE)
    f = np.repeat(make_frame(cameras[0], slots, sh_stride, step, options, background, camera_extent, masked_target,
                             ssim, pair_capacity), len(cameras))
    n = len(cameras)
    rot = np.empty((n, 3, 4), np.float32)
    pos = np.empty((n, 3), np.float32)
    intr = np.empty((n, 4), np.float32)
    image = np.empty((n, 4), np.uint32)
    for k, c in enumerate(cameras):
        rot[k, :, :3] = np.asarray(c.rotation).reshape(3, 3)
        rot[k, :, 3] = c.translation
        pos[k] = c.position
        intr[k] = (c.fx, c.fy, c.cx, c.cy)
        image[k] = (c.width, c.height, (c.width + TILE - 1) // TILE, (c.height + TILE - 1) // TILE)
    f["rot"] = rot
    f["cam_pos"][:, :3] = pos
    f["intrinsics"] = intr
    f["image"] = image
    W, H = image[:, 0].astype(np.float32), image[:, 1].astype(np.float32)
    f["background"][:, 3] = np.float32(1.0) / (np.float32(3.0) * W * H)
    return f
