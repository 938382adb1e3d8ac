"""CPU oracle driver — TEST INFRASTRUCTURE ONLY.

Loads oracle/libgs_oracle.so (a plain-C restatement of the reference engine's training
passes, see gs_oracle.h) and chains its stages into one training step the way
`Trainer::run_view` records them (engine/src/trainer.cpp:807-844): project, depth sort,
gather/scan/emit, pair sort, ranges, forward, SSIM, SSIM gradient, backward, pair sum,
projection backward, Adam. Only tests/, `__graft_entry__.smoke()` and bench.py's CPU
baseline / reference leg use it, as the checker.

Arrays use the reference's layouts: params (n, 16) float32, sh (n, stride) float32,
frames as the 256-byte FrameData (train_common.glsl:15-37).
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libgs_oracle.so")

_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_vp = ctypes.c_void_p

_lib = None


def build() -> None:
    """Compiles the oracle library (gcc, OpenMP, no contraction)."""
    import subprocess

    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        u32, u64 = ctypes.c_uint32, ctypes.c_uint64
        L.gso_project.argtypes = [_vp, _f32p, _vp, u32, _f32p, _u32p, _u32p]
        L.gso_footprint_counts.argtypes = [_vp, _f32p, u32, _u32p]
        L.gso_footprint_tiles.argtypes = [_vp, _f32p, _u32p, u32]
        L.gso_footprint_tiles.restype = u32
        L.gso_depth_order.argtypes = [_u32p, u32, _u32p]
        L.gso_emit.argtypes = [_vp, _f32p, _u32p, _u32p, u32, u64, _u32p, _u32p, _u32p, _vp, _u32p]
        L.gso_emit.restype = u64
        L.gso_sort_pairs.argtypes = [_u32p, u64, u32, _u32p, _u32p, _u32p]
        L.gso_forward.argtypes = [_vp, _f32p, _u32p, _u32p, _u32p, _u32p, _f32p, _u32p, _u32p, _f32p, _u32p, _f32p, _f32p]
        L.gso_ssim.argtypes = [_vp, _f32p, _u32p, _f32p, _f32p]
        L.gso_ssim_grad.argtypes = [_vp, _f32p, _f32p, _u32p, _f32p, _f32p]
        L.gso_backward.argtypes = [_vp, _f32p, _u32p, _u32p, _u32p, _f32p, _u32p, _u32p, _f32p]
        L.gso_pair_sum.argtypes = [u32, _u32p, _u32p, _f32p, _f32p]
        L.gso_project_backward.argtypes = [_vp, _f32p, _vp, _u32p, _f32p, _f32p, _f32p, _f32p, _f32p, _u8p]
        L.gso_sh_gradient.argtypes = [_vp, _f32p, _f32p, _vp]
        L.gso_adam.argtypes = [_vp, _f32p, _vp, _f32p, _f32p, _vp, _vp, _f32p, _vp, _u8p]
        L.gso_densify_mark.argtypes = [_vp, _f32p, _vp, _f32p, _f32p, _vp, _vp, _f32p, _u32p, _u32p, _u32p]
        L.gso_densify_spawn.argtypes = [_vp, _f32p, _vp, _f32p, _f32p, _vp, _vp, _u32p, _u32p, _u32p, u32]
        L.gso_reset_opacity.argtypes = [_vp, _f32p, _f32p, _f32p, ctypes.c_float]
        L.gso_reference_loss.argtypes = [_f64p, u32, u32, _f64p, _vp, u32, ctypes.c_int, ctypes.c_int, _u8p,
                                         _f32p, ctypes.c_int, ctypes.c_double, _vp, _vp, _vp]
        L.gso_reference_loss.restype = ctypes.c_double
        L.gso_reference_ssim.argtypes = [_f64p, _f64p, u32, u32, _vp]
        L.gso_reference_ssim.restype = ctypes.c_double
        L.gso_ssim_window.argtypes = [_f32p]
        L.gso_pcg_hash.argtypes = [u32]
        L.gso_pcg_hash.restype = u32
        L.gso_set_threads.argtypes = [ctypes.c_int]
        L.gso_get_threads.restype = ctypes.c_int
        _lib = L
    return _lib


def _ptr(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def _sh_ptr(sh):
    # A zero-stride SH array still needs a valid pointer.
    return _ptr(sh) if sh is not None and sh.size > 0 else _ptr(np.zeros(1, np.float32))


def set_threads(n: int) -> None:
    lib().gso_set_threads(int(n))


def threads() -> int:
    return int(lib().gso_get_threads())


@dataclass
class ViewResult:
    """Intermediate and final buffers of one view (the reference's DebugSnapshot plus more)."""

    projected: np.ndarray = None
    tiles: np.ndarray = None
    depth_keys: np.ndarray = None
    depth_order: np.ndarray = None
    offsets: np.ndarray = None
    pairs: int = 0
    pair_tile: np.ndarray = None
    pair_gaussian: np.ndarray = None
    render_order: np.ndarray = None
    ranges: np.ndarray = None
    mismatch: int = 0
    pixel_grad: np.ndarray = None
    pixel_count: np.ndarray = None
    image: np.ndarray = None
    tile_loss: np.ndarray = None
    tile_count: np.ndarray = None
    ssim_input: np.ndarray = None
    ssim_maps: np.ndarray = None
    pixel_dot: np.ndarray = None
    pair_grads: np.ndarray = None
    grad_sum: np.ndarray = None
    sums: np.ndarray = field(default_factory=lambda: np.zeros(8))


def forward_view(frame: np.ndarray, params: np.ndarray, sh: np.ndarray, target: np.ndarray,
                 capacity: int | None = None, ssim: bool = True, backward: bool = True,
                 projected: np.ndarray | None = None, depth_keys: np.ndarray | None = None) -> ViewResult:
    """Project -> sort -> forward -> loss (-> per-pair backward -> pair sum) for one view.

    `projected`/`depth_keys`: optional externally computed (e.g. GPU) projection inputs; the
    integer stages are then recomputed from them, as the reference's emit recomputes the
    footprint from stored records (train_common.glsl:163-168).
    """
    L = lib()
    f = frame.ctypes.data_as(ctypes.c_void_p)
    n = int(frame["model"][0][0])
    width, height, tx, ty = (int(v) for v in frame["image"][0])
    ntiles = tx * ty
    r = ViewResult()
    if projected is None:
        r.projected = np.zeros((n, 16), np.float32)
        r.tiles = np.zeros(n, np.uint32)
        r.depth_keys = np.zeros(n, np.uint32)
        if n:
            L.gso_project(f, np.ascontiguousarray(params[:n]), _sh_ptr(sh), n, r.projected, r.tiles, r.depth_keys)
    else:
        r.projected = np.ascontiguousarray(projected[:n], np.float32)
        r.tiles = np.zeros(n, np.uint32)
        if n:
            L.gso_footprint_counts(f, r.projected, n, r.tiles)
        r.depth_keys = np.ascontiguousarray(depth_keys[:n], np.uint32)
    r.depth_order = np.zeros(max(n, 1), np.uint32)
    if n:
        L.gso_depth_order(r.depth_keys, n, r.depth_order)
    total = int(r.tiles.astype(np.uint64).sum())
    cap = total if capacity is None else min(int(capacity), total)
    r.offsets = np.zeros(max(n, 1), np.uint32)
    r.pair_tile = np.zeros(max(cap, 1), np.uint32)
    r.pair_gaussian = np.zeros(max(cap, 1), np.uint32)
    r.pair_grads = np.zeros((max(cap, 1), 12), np.float32)
    mismatch = np.zeros(1, np.uint32)
    if n:
        r.pairs = int(L.gso_emit(f, r.projected, r.tiles, r.depth_order, n, cap, r.offsets, r.pair_tile,
                                 r.pair_gaussian, _ptr(r.pair_grads), mismatch))
    r.mismatch = int(mismatch[0])
    stored = min(r.pairs, cap)
    r.render_order = np.zeros(max(stored, 1), np.uint32)
    sorted_tile = np.zeros(max(stored, 1), np.uint32)
    r.ranges = np.zeros((ntiles + 1) * 2, np.uint32)
    L.gso_sort_pairs(r.pair_tile, stored, ntiles, r.render_order, sorted_tile, r.ranges)
    pixels = width * height
    r.pixel_grad = np.zeros((pixels, 4), np.float32)
    r.pixel_count = np.zeros(pixels, np.uint32)
    r.image = np.zeros(pixels, np.uint32)
    r.tile_loss = np.zeros((ntiles, 16), np.float32)
    r.tile_count = np.zeros(ntiles, np.uint32)
    r.ssim_input = np.zeros((pixels, 8), np.float32)
    r.pixel_dot = np.zeros(pixels, np.float32)
    tgt = np.ascontiguousarray(target.reshape(-1).view(np.uint32)) if target.dtype == np.uint8 else target
    L.gso_forward(f, r.projected, r.ranges, r.render_order, r.pair_gaussian, tgt, r.pixel_grad, r.pixel_count,
                  r.image, r.tile_loss, r.tile_count, r.ssim_input, r.pixel_dot)
    if ssim:
        r.ssim_maps = np.zeros((pixels, 9), np.float32)
        L.gso_ssim(f, r.ssim_input, r.ranges, r.ssim_maps, r.tile_loss)
        if backward:
            L.gso_ssim_grad(f, r.ssim_input, r.ssim_maps, r.ranges, r.pixel_grad, r.pixel_dot)
    r.sums = r.tile_loss[:, :8].astype(np.float64).sum(axis=0)
    if backward:
        L.gso_backward(f, r.projected, r.ranges, r.render_order, r.pair_gaussian, r.pixel_grad, r.pixel_count,
                       r.tile_count, r.pair_grads)
        r.grad_sum = np.zeros((max(n, 1), 12), np.float32)
        if n:
            L.gso_pair_sum(n, r.tiles, r.offsets, r.pair_grads, r.grad_sum)
    return r


@dataclass
class Model:
    """Parameters and Adam moments in the reference's layout."""

    params: np.ndarray
    sh: np.ndarray
    m: np.ndarray
    v: np.ndarray
    m_sh: np.ndarray
    v_sh: np.ndarray
    stats: np.ndarray

    @staticmethod
    def create(params: np.ndarray, sh: np.ndarray, capacity: int | None = None) -> "Model":
        n = params.shape[0]
        cap = max(capacity or n, n)
        stride = sh.shape[1] if sh.ndim == 2 else 0
        P = np.zeros((cap, 16), np.float32)
        P[:n] = params
        S = np.zeros((cap, stride), np.float32)
        if stride:
            S[:n] = sh
        return Model(P, S, np.zeros_like(P), np.zeros_like(P), np.zeros_like(S), np.zeros_like(S),
                     np.zeros((cap, 4), np.float32))


def train_step(model: Model, frames: list[np.ndarray], targets: list[np.ndarray], ssim: bool = True,
               capacity: int | None = None) -> tuple[list[ViewResult], np.ndarray, np.ndarray, np.ndarray]:
    """One training step over `frames` (one or more views): per view forward + backward,
    gradients summed over the views, one Adam step with the first frame's constants.
    With one view this is the reference step (trainer.cpp:825-831). Returns the view
    results, grad16 (n, 16), grad_sh (n, stride) and the drew bits."""
    L = lib()
    f0 = frames[0]
    n = int(f0["model"][0][0])
    stride = model.sh.shape[1]
    grad16 = np.zeros((max(n, 1), 16), np.float32)
    grad_sh = np.zeros((max(n, 1), max(stride, 1)), np.float32)
    drew = np.zeros(max(n, 1), np.uint8)
    results = []
    for frame, target in zip(frames, targets):
        r = forward_view(frame, model.params, model.sh, target, capacity=capacity, ssim=ssim, backward=True)
        results.append(r)
        limit = int(frame["limits"][0][3])
        if limit and r.pairs > limit:
            continue
        sh_input = np.zeros((max(n, 1), 8), np.float32)
        f = frame.ctypes.data_as(ctypes.c_void_p)
        if n:
            L.gso_project_backward(f, model.params, _sh_ptr(model.sh), r.tiles, r.grad_sum, r.projected,
                                   model.stats, grad16, sh_input, drew)
            if stride:
                g = np.zeros((n, stride), np.float32)
                L.gso_sh_gradient(f, model.params, sh_input, _ptr(g))
                grad_sh[:n, :stride] += g
    if any(int(fr["limits"][0][3]) and r.pairs > int(fr["limits"][0][3]) for fr, r in zip(frames, results)):
        return results, grad16, grad_sh, drew
    if n:
        gs = np.ascontiguousarray(grad_sh[:n, :stride]) if stride else None
        L.gso_adam(f0.ctypes.data_as(ctypes.c_void_p), model.params, _sh_ptr(model.sh), model.m, model.v,
                   _sh_ptr(model.m_sh), _sh_ptr(model.v_sh), np.ascontiguousarray(grad16[:n]),
                   _ptr(gs) if gs is not None else _ptr(np.zeros(1, np.float32)), drew)
    return results, grad16[:n], grad_sh[:n, :stride], drew[:n]


def densify(model: Model, frame: np.ndarray, capacity: int) -> np.ndarray:
    """train_densify_mark + train_densify_spawn with deterministic slot order. Returns
    counters [free, spawned, pruned, 0] and the spawn mask."""
    L = lib()
    n = int(frame["model"][0][0])
    f = frame.ctypes.data_as(ctypes.c_void_p)
    spawn = np.zeros(max(n, 1), np.uint32)
    free_list = np.zeros(max(n, 1), np.uint32)
    counters = np.zeros(4, np.uint32)
    L.gso_densify_mark(f, model.params, _sh_ptr(model.sh), model.m, model.v, _sh_ptr(model.m_sh),
                       _sh_ptr(model.v_sh), model.stats, spawn, free_list, counters)
    L.gso_densify_spawn(f, model.params, _sh_ptr(model.sh), model.m, model.v, _sh_ptr(model.m_sh),
                        _sh_ptr(model.v_sh), spawn, free_list, counters, capacity)
    model.stats[:] = 0
    return counters, spawn[:n]


def footprint_tiles(frame: np.ndarray, proj16: np.ndarray) -> np.ndarray:
    L = lib()
    out = np.zeros(1 << 16, np.uint32)
    k = L.gso_footprint_tiles(frame.ctypes.data_as(ctypes.c_void_p), np.ascontiguousarray(proj16, np.float32),
                              out, out.size)
    return out[:k].copy()


def _camera_vector(camera: dict) -> np.ndarray:
    """The camera as 19 doubles, each rounded to float first: gs::Camera stores floats
    (engine/include/gs/camera.h:10-16), so the reference's FP64 code sees float values."""
    v = np.concatenate([np.asarray(camera["rotation"], np.float64).reshape(9),
                        np.asarray(camera["translation"], np.float64).reshape(3),
                        np.asarray(camera["position"], np.float64).reshape(3),
                        np.array([camera["fx"], camera["fy"], camera["cx"], camera["cy"]], np.float64)])
    return v.astype(np.float32).astype(np.float64)


def reference_loss(camera: dict, width: int, height: int, params64: np.ndarray, sh64: np.ndarray, degree: int,
                   target: np.ndarray, bg, masked: bool, lam: float, want_image: bool = False, head=None,
                   want_signature: bool = False):
    """FP64 forward + loss of train_selftest.cpp:211-283. With want_signature, also the hash
    of its blend decisions (equal hashes: no alpha / transmittance / clamp cut-off crossed)."""
    L = lib()
    cam = _camera_vector(camera)
    n = params64.shape[0]
    stride = sh64.shape[1] if sh64.ndim == 2 else 0
    img = np.zeros((width * height, 3), np.float64) if want_image else None
    h = None if head is None else np.asarray(head, np.float64)
    sig = np.zeros(1, np.uint64) if want_signature else None
    loss = L.gso_reference_loss(cam, width, height, np.ascontiguousarray(params64, np.float64),
                                _ptr(np.ascontiguousarray(sh64, np.float64)) if stride else None, n, stride,
                                degree, np.ascontiguousarray(target.reshape(-1), np.uint8),
                                np.asarray(bg, np.float32), int(masked), float(lam), _ptr(img), _ptr(h), _ptr(sig))
    if want_signature:
        return (loss, img, int(sig[0])) if want_image else (loss, int(sig[0]))
    return (loss, img) if want_image else loss


def ssim_window() -> np.ndarray:
    out = np.zeros(11, np.float32)
    lib().gso_ssim_window(out)
    return out


def pcg_hash(v: int) -> int:
    return int(lib().gso_pcg_hash(v))


# The reference's own FP64 CPU forward + loss (engine/src/train_selftest.cpp:27-283),
# compiled from a reference checkout by `make -C oracle ref` into oracle/_ref/ (see
# ref_shim.cpp). It pins the restatement above: gso_reference_loss / gso_reference_ssim must
# reproduce it, and finite differences of it check the analytic gradients.
REF_LIB_PATH = os.path.join(HERE, "_ref", "libgs_ref.so")
REFERENCE_SOURCE = os.path.join(os.environ.get("GS_REFERENCE", "/root/reference"), "engine", "src",
                                "train_selftest.cpp")
_ref = None


def ref_lib():
    """The reference's CPU library, built first if a reference checkout is present; None if
    neither the library nor a checkout is present."""
    global _ref
    if _ref is None:
        if not os.path.exists(REF_LIB_PATH):
            if not os.path.exists(REFERENCE_SOURCE):
                return None
            import subprocess

            subprocess.run(["make", "-s", "-C", HERE, "ref",
                            f"REFERENCE={os.path.dirname(os.path.dirname(os.path.dirname(REFERENCE_SOURCE)))}"],
                           check=True)
        L = ctypes.CDLL(REF_LIB_PATH)
        u32 = ctypes.c_uint32
        L.gsr_reference_loss.argtypes = [_f64p, u32, u32, _f64p, _vp, u32, ctypes.c_int, ctypes.c_int, _u8p,
                                         _f32p, ctypes.c_int, ctypes.c_double, _vp, _vp]
        L.gsr_reference_loss.restype = ctypes.c_double
        L.gsr_reference_ssim.argtypes = [_f64p, _f64p, u32, u32, _vp]
        L.gsr_reference_ssim.restype = ctypes.c_double
        _ref = L
    return _ref




def ref_reference_loss(camera: dict, width: int, height: int, params64: np.ndarray, sh64: np.ndarray, degree: int,
                       target: np.ndarray, bg, masked: bool, lam: float, want_image: bool = False, head=None):
    """gs::reference_loss itself (the reference's code), same arguments as reference_loss."""
    L = ref_lib()
    n = params64.shape[0]
    stride = sh64.shape[1] if sh64.ndim == 2 else 0
    img = np.zeros((width * height, 3), np.float64) if want_image else None
    h = None if head is None else np.asarray(head, np.float64)
    loss = L.gsr_reference_loss(_camera_vector(camera), width, height, np.ascontiguousarray(params64, np.float64),
                                _ptr(np.ascontiguousarray(sh64, np.float64)) if stride else None, n, stride, degree,
                                np.ascontiguousarray(target.reshape(-1), np.uint8), np.asarray(bg, np.float32),
                                int(masked), float(lam), _ptr(img), _ptr(h))
    return (loss, img) if want_image else loss


def ref_reference_ssim(x: np.ndarray, y: np.ndarray, width: int, height: int, weights=None) -> float:
    """gs::reference_ssim itself (x, y: (pixels, 3) float64)."""
    w = None if weights is None else np.ascontiguousarray(weights, np.float64)
    return float(ref_lib().gsr_reference_ssim(np.ascontiguousarray(x, np.float64), np.ascontiguousarray(y, np.float64),
                                              width, height, _ptr(w)))
