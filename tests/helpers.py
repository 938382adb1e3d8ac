"""Shared fixtures of the parity tests: the reference's test scenes and checks."""
from __future__ import annotations

import numpy as np

import oracle as O
from gs_b200 import frame as F
from gs_b200 import scenes as S


def frame_for(scene: S.Scene, cam: F.Camera, opt: F.TrainOptions, bg, masked: bool = False, ssim: bool = True,
              step: int = 0, extent: float = 3.3) -> np.ndarray:
    return F.make_frame(cam, scene.count, scene.sh.shape[1], step, opt, bg, extent, masked_target=masked,
                        ssim=ssim)


def params64(scene: S.Scene) -> tuple[np.ndarray, np.ndarray]:
    return scene.params.astype(np.float64), scene.sh.astype(np.float64)


GROUPS = {"position": [0, 1, 2], "opacity": [3], "log_scale": [4, 5, 6], "rotation": [8, 9, 10, 11],
          "sh_dc": [12, 13, 14]}


def fd_check(scene: S.Scene, cam: F.Camera, target: np.ndarray, grad16: np.ndarray, grad_sh: np.ndarray,
             bg, masked: bool, lam: float, eps: float = 1e-5, params: list | None = None,
             skip_crossings: bool = False, loss_impl=None) -> dict:
    """check_gradients (train_selftest.cpp:418-446): central finite differences of the FP64
    reference loss, |err| <= 5% |fd| + 2e-6, per parameter group. `params`: optional list of
    (slot, offset) to check (offset < 0: SH coefficient -1 - offset); default all.
    skip_crossings: leave out parameters whose stencil changes any blend decision of the FP64
    forward (an alpha or transmittance cut-off, a clamp or the depth order), where central
    differences measure a jump, not the derivative; they are counted as `skipped`.
    loss_impl: the FP64 loss to differentiate (default the oracle's restatement; the
    reference's own, O.ref_reference_loss, where it is built). Decision signatures always
    come from the restatement, which reproduces the reference bit for bit."""
    p64, s64 = params64(scene)
    W, H = cam.width, cam.height
    camd = cam.as_dict()
    stride = scene.sh.shape[1]

    def loss():
        if loss_impl is None:
            return O.reference_loss(camd, W, H, p64, s64, scene.degree, target, bg, masked, lam, want_signature=True)
        value = loss_impl(camd, W, H, p64, s64, scene.degree, target, bg, masked, lam)
        sig = 0
        if skip_crossings:
            _, sig = O.reference_loss(camd, W, H, p64, s64, scene.degree, target, bg, masked, lam,
                                      want_signature=True)
        return value, sig

    _, sig0 = loss()

    todo = params
    if todo is None:
        todo = [(i, off) for i in range(scene.count) for g in GROUPS.values() for off in g]
        todo += [(i, -1 - k) for i in range(scene.count) for k in range(stride)]
    report = {}
    for i, off in todo:
        arr, idx = (p64, (i, off)) if off >= 0 else (s64, (i, -1 - off))
        saved = arr[idx]
        arr[idx] = saved + eps
        up, sig_up = loss()
        arr[idx] = saved - eps
        down, sig_down = loss()
        arr[idx] = saved
        fd = (up - down) / (2 * eps)
        got = float(grad16[i, off]) if off >= 0 else float(grad_sh[i, -1 - off])
        group = next((k for k, v in GROUPS.items() if off in v), "sh_rest") if off >= 0 else "sh_rest"
        g = report.setdefault(group, {"checked": 0, "bad": 0, "max_err": 0.0, "max_ref": 0.0, "skipped": 0})
        if skip_crossings and (sig_up != sig0 or sig_down != sig0):
            g["skipped"] += 1
            continue
        err = abs(got - fd)
        g["checked"] += 1
        g["max_err"] = max(g["max_err"], err)
        g["max_ref"] = max(g["max_ref"], abs(fd))
        if not err <= 0.05 * abs(fd) + 2e-6:
            g["bad"] += 1
    return report


def rel_l2(a, b) -> float:
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    den = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / den) if den > 0 else float(np.linalg.norm(a - b))


def image_f(img_u32: np.ndarray) -> np.ndarray:
    return img_u32.view(np.uint8).reshape(-1, 4).astype(np.float64) / 255.0
