"""ctypes binding of libgs_cuda's C ABI (include/gs_cuda.h).

This is the binding a Python caller of the reference's training step would add; the
product path is the CUDA library itself, so a missing library is an error, never a
fallback.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from .frame import FRAME_DTYPE

PKG = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(PKG, "lib", "libgs_cuda.so")

GS_OK, GS_ERR_INVALID, GS_ERR_NO_MEMORY, GS_ERR_CAPACITY, GS_ERR_TIMEOUT, GS_ERR_CUDA = range(6)
GS_MAX_VIEWS = 16
GS_STEP_TRAIN = 1
GS_STEP_PROFILE = 2
GS_STEP_COUNT = 4
PASSES = ("project", "sort", "rasterize", "loss", "backward", "optimize")

SNAP = {
    "pixel_count": (0, np.uint32, 1), "pixel_grad": (1, np.float32, 4), "projected": (2, np.float32, 16),
    "tiles": (3, np.uint32, 1), "offsets": (4, np.uint32, 1), "pair_grads": (5, np.float32, 12),
    "pair_tile": (6, np.uint32, 1), "render_order": (7, np.uint32, 1), "depth_key": (8, np.uint32, 1),
    "image": (9, np.uint32, 1), "ranges": (10, np.uint32, 2), "tile_loss": (11, np.float32, 16),
    "pixel_dot": (12, np.float32, 1), "stats": (13, np.float32, 4), "pair_gaussian": (14, np.uint32, 1),
    "pixel_out": (15, np.float32, 4), "spawn": (16, np.uint32, 1), "motion_bind": (17, np.uint32, 8),
    "contributions": (18, np.uint64, 1),
}

EXPORTED = ["gs_last_error", "gs_create", "gs_destroy", "gs_model_init", "gs_model_info_get", "gs_model_export",
            "gs_model_moments", "gs_set_views", "gs_step", "gs_render", "gs_densify", "gs_reset_opacity",
            "gs_snapshot", "gs_set_tuning", "gs_get_tuning", "gs_dataset_set", "gs_set_views_dataset",
            "gs_sort_pairs_noalloc", "gs_autotune", "gs_motion_nodes", "gs_motion_bind", "gs_set_view_motion",
            "gs_motion_gradient"]


class StepResult(ctypes.Structure):
    _fields_ = [("n_views", ctypes.c_uint32), ("overflow", ctypes.c_uint32), ("retries", ctypes.c_uint32),
                ("tile_mismatch", ctypes.c_uint32), ("pairs", ctypes.c_uint64 * GS_MAX_VIEWS),
                ("losses", (ctypes.c_double * 8) * GS_MAX_VIEWS), ("gpu_ms", ctypes.c_float),
                ("kernels", ctypes.c_uint32), ("pass_ms", ctypes.c_float * 6),
                ("fit", (ctypes.c_double * 8) * GS_MAX_VIEWS), ("pose_grad", (ctypes.c_double * 6) * GS_MAX_VIEWS)]


class Tuning(ctypes.Structure):
    _fields_ = [("min_pair_capacity", ctypes.c_uint32), ("initial_pairs", ctypes.c_uint64),
                ("deterministic", ctypes.c_uint32), ("forward_pixels", ctypes.c_uint32),
                ("backward_pixels", ctypes.c_uint32), ("retry", ctypes.c_uint32), ("graph", ctypes.c_uint32),
                ("backward_batch", ctypes.c_uint32), ("sort_digit_bits", ctypes.c_uint32),
                ("forward_batch", ctypes.c_uint32), ("tune_reduction", ctypes.c_uint32),
                ("stage_async", ctypes.c_uint32)]


class ModelInfo(ctypes.Structure):
    _fields_ = [("capacity", ctypes.c_uint32), ("slots", ctypes.c_uint32), ("sh_stride", ctypes.c_uint32),
                ("pair_capacity", ctypes.c_uint64), ("device_bytes", ctypes.c_uint64)]


class GsError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"libgs_cuda error {code}: {message}")
        self.code = code


_lib = None


def load(path: str = LIB_PATH):
    """Loads libgs_cuda; raises if it has not been built (no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} is missing: build it first (make -C on-divice-gsplate_b200)")
    L = ctypes.CDLL(path)
    vp, u32, u64 = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint64
    L.gs_last_error.restype = ctypes.c_char_p
    L.gs_create.argtypes = [ctypes.c_int, ctypes.POINTER(vp)]
    L.gs_destroy.argtypes = [vp]
    L.gs_model_init.argtypes = [vp, u32, u32, vp, vp, u32]
    L.gs_model_info_get.argtypes = [vp, ctypes.POINTER(ModelInfo)]
    L.gs_model_export.argtypes = [vp, vp, vp, u32, ctypes.POINTER(u32)]
    L.gs_model_moments.argtypes = [vp, vp, vp, vp, vp]
    L.gs_set_views.argtypes = [vp, u32, vp, ctypes.POINTER(ctypes.c_void_p)]
    L.gs_step.argtypes = [vp, u32, ctypes.POINTER(StepResult)]
    L.gs_render.argtypes = [vp, vp, vp]
    L.gs_densify.argtypes = [vp, vp, ctypes.POINTER(u32 * 4)]
    L.gs_reset_opacity.argtypes = [vp, ctypes.c_float]
    L.gs_snapshot.argtypes = [vp, u32, ctypes.c_int, vp, ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t)]
    L.gs_set_tuning.argtypes = [vp, ctypes.POINTER(Tuning)]
    L.gs_get_tuning.argtypes = [vp, ctypes.POINTER(Tuning)]
    L.gs_dataset_set.argtypes = [vp, u32, vp, vp, ctypes.POINTER(ctypes.c_void_p)]
    L.gs_set_views_dataset.argtypes = [vp, u32, vp, vp]
    L.gs_sort_pairs_noalloc.argtypes = [vp, vp, u32, u32, vp]
    L.gs_autotune.argtypes = [vp, u32, vp]
    L.gs_motion_nodes.argtypes = [vp, u32, vp]
    L.gs_motion_bind.argtypes = [vp]
    L.gs_set_view_motion.argtypes = [vp, u32, vp]
    L.gs_motion_gradient.argtypes = [vp, u32, vp, u32]
    for name in EXPORTED[1:]:
        getattr(L, name).restype = ctypes.c_int
    _lib = L
    return L


def _check(code: int) -> None:
    if code != GS_OK:
        raise GsError(code, load().gs_last_error().decode())


def _frames(frames) -> np.ndarray:
    """The views' FrameData as one contiguous array (no copies beyond the concatenation when
    they already are FRAME_DTYPE records; none for an array of them, as make_frames gives)."""
    if isinstance(frames, np.ndarray) and frames.dtype == FRAME_DTYPE:
        return np.ascontiguousarray(frames.reshape(-1))
    if all(isinstance(f, np.ndarray) and f.dtype == FRAME_DTYPE for f in frames):
        return np.concatenate([f.reshape(1) for f in frames])
    return np.ascontiguousarray(np.concatenate([np.asarray(f, FRAME_DTYPE).reshape(1) for f in frames]))


def _ptr(a):
    return None if a is None else ctypes.c_void_p(a.ctypes.data)


class Context:
    """One libgs_cuda context (a device and its stream)."""

    def __init__(self, device: int = 0):
        self.lib = load()
        h = ctypes.c_void_p()
        _check(self.lib.gs_create(device, ctypes.byref(h)))
        self.h = h
        self._keep = []

    def close(self) -> None:
        if self.h:
            _check(self.lib.gs_destroy(self.h))
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- model ----
    def model_init(self, params: np.ndarray, sh: np.ndarray, capacity: int | None = None) -> None:
        params = np.ascontiguousarray(params, np.float32)
        n = params.shape[0]
        stride = sh.shape[1] if sh is not None and sh.ndim == 2 else 0
        sh_c = np.ascontiguousarray(sh, np.float32) if stride else None
        _check(self.lib.gs_model_init(self.h, max(capacity or n, n, 1), stride, _ptr(params), _ptr(sh_c), n))

    def info(self) -> ModelInfo:
        out = ModelInfo()
        _check(self.lib.gs_model_info_get(self.h, ctypes.byref(out)))
        return out

    def export(self) -> tuple[np.ndarray, np.ndarray]:
        info = self.info()
        p = np.zeros((info.slots, 16), np.float32)
        s = np.zeros((info.slots, info.sh_stride), np.float32)
        slots = ctypes.c_uint32()
        _check(self.lib.gs_model_export(self.h, _ptr(p), _ptr(s) if info.sh_stride else None, info.slots,
                                        ctypes.byref(slots)))
        return p, s

    def moments(self) -> dict:
        info = self.info()
        m = np.zeros((info.slots, 16), np.float32)
        v = np.zeros((info.slots, 16), np.float32)
        ms = np.zeros((info.slots, info.sh_stride), np.float32)
        vs = np.zeros((info.slots, info.sh_stride), np.float32)
        st = info.sh_stride > 0
        _check(self.lib.gs_model_moments(self.h, _ptr(m), _ptr(v), _ptr(ms) if st else None, _ptr(vs) if st else None))
        return {"m": m, "v": v, "m_sh": ms, "v_sh": vs}

    def first_step_gradients(self) -> tuple[np.ndarray, np.ndarray]:
        """Trainer::first_step_gradients (trainer.cpp:1802-1811): m / (1 - beta1)."""
        mo = self.moments()
        return mo["m"] / np.float32(0.1), mo["m_sh"] / np.float32(0.1)

    # ---- step ----
    def set_views(self, frames: list[np.ndarray], targets: list[np.ndarray] | None) -> None:
        fr = _frames(frames)
        tptr = None
        keep = [fr]
        if targets is not None:
            arrs = [np.ascontiguousarray(t, np.uint8) for t in targets]
            keep += arrs
            tptr = (ctypes.c_void_p * len(arrs))(*[a.ctypes.data for a in arrs])
        self._keep = keep  # the library may read the targets until the next step returns
        _check(self.lib.gs_set_views(self.h, len(fr), _ptr(fr), tptr))

    def set_dataset(self, images: list[np.ndarray]) -> None:
        """Keeps RGBA8 target images (H x W x 4 uint8) in HBM across steps."""
        arrs = [np.ascontiguousarray(t, np.uint8) for t in images]
        w = np.array([a.shape[1] for a in arrs], np.uint32)
        h = np.array([a.shape[0] for a in arrs], np.uint32)
        ptrs = (ctypes.c_void_p * max(len(arrs), 1))(*[a.ctypes.data for a in arrs])
        _check(self.lib.gs_dataset_set(self.h, len(arrs), _ptr(w), _ptr(h), ptrs))

    def set_views_dataset(self, frames: list[np.ndarray], images: list[int]) -> None:
        fr = _frames(frames)
        idx = np.ascontiguousarray(images, np.uint32)
        self._keep = [fr]
        _check(self.lib.gs_set_views_dataset(self.h, len(fr), _ptr(fr), _ptr(idx)))

    def step(self, train: bool = True, profile: bool = False, count: bool = False) -> StepResult:
        """One step; `profile`: per-pass device times; `count`: the forward also counts its
        blending evaluations (snapshot "contributions"), without the step's graph."""
        out = StepResult()
        flags = (GS_STEP_TRAIN if train else 0) | (GS_STEP_PROFILE if profile else 0) | (GS_STEP_COUNT if count else 0)
        _check(self.lib.gs_step(self.h, flags, ctypes.byref(out)))
        return out

    def render(self, frame: np.ndarray) -> np.ndarray:
        f = np.ascontiguousarray(np.asarray(frame, FRAME_DTYPE).reshape(1))
        W, H = int(f["image"][0][0]), int(f["image"][0][1])
        out = np.zeros((H, W, 4), np.uint8)
        _check(self.lib.gs_render(self.h, _ptr(f), _ptr(out)))
        return out

    def densify(self, frame: np.ndarray) -> np.ndarray:
        f = np.ascontiguousarray(np.asarray(frame, FRAME_DTYPE).reshape(1))
        c = (ctypes.c_uint32 * 4)()
        _check(self.lib.gs_densify(self.h, _ptr(f), ctypes.byref(c)))
        return np.array(list(c), np.uint32)

    def reset_opacity(self, max_logit: float) -> None:
        _check(self.lib.gs_reset_opacity(self.h, ctypes.c_float(max_logit)))

    def snapshot(self, which: str, view: int = 0) -> np.ndarray:
        kind, dtype, width = SNAP[which]
        need = ctypes.c_size_t()
        _check(self.lib.gs_snapshot(self.h, view, kind, None, 0, ctypes.byref(need)))
        n = need.value // (np.dtype(dtype).itemsize * width)
        out = np.zeros((n, width) if width > 1 else n, dtype)
        _check(self.lib.gs_snapshot(self.h, view, kind, _ptr(out), out.nbytes, ctypes.byref(need)))
        return out

    def tuning(self) -> Tuning:
        t = Tuning()
        _check(self.lib.gs_get_tuning(self.h, ctypes.byref(t)))
        return t

    def set_tuning(self, **kw) -> None:
        t = self.tuning()
        for k, v in kw.items():
            setattr(t, k, v)
        _check(self.lib.gs_set_tuning(self.h, ctypes.byref(t)))

    def motion_nodes(self, nodes4: np.ndarray) -> None:
        """Control nodes at rest, (K, 4) float32: position, 1 / (2 r^2); binds the slots."""
        n = np.ascontiguousarray(nodes4, np.float32).reshape(-1, 4)
        _check(self.lib.gs_motion_nodes(self.h, n.shape[0], _ptr(n) if n.size else None))

    def motion_bind(self) -> None:
        _check(self.lib.gs_motion_bind(self.h))

    def set_view_motion(self, view: int, nodes20: np.ndarray) -> None:
        """View `view`'s node motions, (K, 20) float32: rows of [R | b], turn, moved centre."""
        n = np.ascontiguousarray(nodes20, np.float32).reshape(-1, 20)
        _check(self.lib.gs_set_view_motion(self.h, view, _ptr(n)))

    def motion_gradient(self, view: int, count: int) -> np.ndarray:
        """(count, 6): dL/dshift, dL/dturn per node (world axes) of the latest step."""
        out = np.zeros((count, 6), np.float64)
        _check(self.lib.gs_motion_gradient(self.h, view, _ptr(out), count))
        return out

    def autotune(self, steps_per_candidate: int = 2) -> Tuning:
        """gs_autotune on the views set last: the fastest tuning becomes the context's; the
        model is left as it was."""
        t = Tuning()
        _check(self.lib.gs_autotune(self.h, steps_per_candidate, ctypes.byref(t)))
        return t
