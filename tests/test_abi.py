"""The C-ABI library loads and exports every function include/gs_cuda.h declares (CPU)."""
import ctypes
import os
import re
import subprocess

import numpy as np

from gs_b200 import cuda
from gs_b200.frame import FRAME_DTYPE

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "gs_cuda.h")


def declared_functions():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^(?:int|const char\*)\s+(gs_\w+)\s*\(", text, re.M)))


def test_header_declares_the_binding():
    assert declared_functions() == sorted(cuda.EXPORTED)


def test_library_exports_every_symbol():
    lib = cuda.load()
    for name in declared_functions():
        assert hasattr(lib, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", cuda.LIB_PATH], capture_output=True, text=True, check=True)
    exported = set(re.findall(r"\sT\s(gs_\w+)", out.stdout))
    assert set(declared_functions()) <= exported


def test_struct_layouts_match_header():
    # gs_frame_data is FrameData (train_common.glsl:15-37): 18 vec4 = 288 bytes.
    assert FRAME_DTYPE.itemsize == 288
    assert ctypes.sizeof(cuda.Tuning) == 56
    assert ctypes.sizeof(cuda.StepResult) == 16 + 8 * 16 + 8 * 8 * 16 + 4 + 4 + 24 + 8 * 8 * 16 + 6 * 8 * 16


def test_ctypes_offsets_match_the_c_compiler(tmp_path):
    """Every field of the ctypes mirrors sits where gcc puts it in the header's structs."""
    structs = {"gs_step_result": cuda.StepResult, "gs_tuning": cuda.Tuning, "gs_model_info": cuda.ModelInfo}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "gs_cuda.h"', "int main(void) {"]
    for cname, cls in structs.items():
        lines.append(f'  printf("{cname} %zu\\n", sizeof({cname}));')
        for field, _ in cls._fields_:
            lines.append(f'  printf("{cname}.{field} %zu\\n", offsetof({cname}, {field}));')
    lines.append("  return 0;\n}")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = dict(line.split() for line in subprocess.run([str(exe)], capture_output=True, text=True,
                                                       check=True).stdout.splitlines())
    for cname, cls in structs.items():
        assert int(got[cname]) == ctypes.sizeof(cls), cname
        for field, _ in cls._fields_:
            assert int(got[f"{cname}.{field}"]) == getattr(cls, field).offset, (cname, field)


def test_no_device_call_errors_cleanly():
    """Without a GPU the library reports an error code and message, not a crash."""
    lib = cuda.load()
    h = ctypes.c_void_p()
    code = lib.gs_create(0, ctypes.byref(h))
    if code == cuda.GS_OK:  # a GPU is present: nothing to check here
        lib.gs_destroy(h)
        return
    assert code in (cuda.GS_ERR_INVALID, cuda.GS_ERR_CUDA)
    assert lib.gs_last_error().decode()
    assert lib.gs_step(None, 1, None) == cuda.GS_ERR_INVALID
    assert b"null" in lib.gs_last_error()


def test_frame_builder_fields():
    from gs_b200 import frame as F
    from gs_b200 import scenes as S

    cam = S.front_camera(360, 640, 500.0)
    opt = F.TrainOptions()
    f = F.make_frame(cam, 20000, 45, 10, opt, (0.1, 0.2, 0.3), 3.3)
    assert list(f["image"][0]) == [360, 640, 23, 40]
    assert f["model"][0][0] == 20000 and f["model"][0][2] == 45
    assert f.view(np.uint32)[53] == (opt.seed * 9781 + 10 * 6271) & 0xFFFFFFFF
    np.testing.assert_allclose(f["bias"][0][0], 1.0 / (1.0 - 0.9 ** 11), rtol=1e-6)
    # Camera at (0, 0, 3) looking at the origin: the origin is 3 in front.
    t = cam.rotation @ np.zeros(3, np.float32) + cam.translation
    np.testing.assert_allclose(t, [0, 0, 3], atol=1e-6)
