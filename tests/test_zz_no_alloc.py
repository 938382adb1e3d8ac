"""gs_sort_pairs_noalloc, the allocation-free sort entry point, against the step's own sort (GPU).

Callers that cannot allocate device memory (a runtime whose pool owns all of it, a plugin
handed only its buffers) sort through gs_sort_pairs_noalloc, whose scratch is a static
device array. These tests call it through the C ABI on two calls in a row and compare its
order with the depth order the training step's radix sort produced for the same keys
(gs_step -> DEPTH_KEY / OFFSETS snapshots) and with numpy's stable argsort: bit-exact, as
for every sort here. The file is named to be collected last, so the shared array has
already seen other sorts' leftovers when the suite runs in one process.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N_GAUSSIANS = 20000


def _step_depth_order():
    """Depth keys of one 360x640 view and the order the step's own sort gave them."""
    from gs_b200 import cuda
    from gs_b200 import frame as F
    from gs_b200 import scenes as S

    scene = S.make_test_scene(N_GAUSSIANS, 0, 5)
    cam = S.front_camera(360, 640, 500.0)
    fr = F.make_frame(cam, scene.count, scene.sh.shape[1], 0, F.frozen_options(0, False), (0.0, 0.0, 0.0), 3.3,
                      ssim=False)
    target = np.zeros((640, 360, 4), np.uint8)
    target[..., 3] = 255
    with cuda.Context(0) as ctx:
        ctx.model_init(scene.params, scene.sh)
        ctx.set_views([fr], [target])
        ctx.step(train=False)
        depth_key = ctx.snapshot("depth_key", 0)
        tiles = ctx.snapshot("tiles", 0)
        offsets = ctx.snapshot("offsets", 0)
    return depth_key, tiles, offsets


def _sort(lib, keys_np, values_np, key_bits):
    import torch

    keys = torch.from_numpy(keys_np.view(np.int32)).cuda()
    values = torch.from_numpy(values_np.view(np.int32)).cuda()
    stream = torch.cuda.current_stream().cuda_stream
    code = lib.gs_sort_pairs_noalloc(ctypes.c_void_p(keys.data_ptr()), ctypes.c_void_p(values.data_ptr()),
                                     len(keys_np), key_bits, ctypes.c_void_p(stream))
    assert code == 0, lib.gs_last_error().decode()
    return keys.cpu().numpy().view(np.uint32), values.cpu().numpy().view(np.uint32)


def test_noalloc_sort_matches_the_step_sort():
    from gs_b200 import cuda

    lib = cuda.load()
    depth_key, tiles, offsets = _step_depth_order()
    keys16 = (depth_key & 0xFFFF).astype(np.uint32)
    visible = np.nonzero(tiles > 0)[0]
    # The step emits pairs in its depth order, so the visible slots' pair offsets rise
    # along that order.
    step_order = visible[np.argsort(offsets[visible], kind="stable")]
    rng = np.random.default_rng(11)
    for call in range(2):
        perm = np.arange(N_GAUSSIANS, dtype=np.uint32) if call == 0 else rng.permutation(N_GAUSSIANS).astype(np.uint32)
        k_in = keys16[perm]
        k_out, v_out = _sort(lib, k_in, perm.copy(), 16)
        expect = perm[np.argsort(k_in, kind="stable")]
        np.testing.assert_array_equal(v_out, expect)
        np.testing.assert_array_equal(k_out, keys16[expect])
        if call == 0:
            got_visible = v_out[np.isin(v_out, visible)]
            np.testing.assert_array_equal(got_visible, step_order)


def test_noalloc_sort_odd_widths_and_sizes():
    """Key widths that end in the alternate buffers (odd pass counts) and ragged sizes."""
    from gs_b200 import cuda

    lib = cuda.load()
    rng = np.random.default_rng(3)
    for n, bits in ((2, 8), (3841, 24), (100003, 32), (1 << 20, 20)):
        keys = rng.integers(0, 1 << bits, n, dtype=np.uint64).astype(np.uint32)
        values = np.arange(n, dtype=np.uint32)
        k_out, v_out = _sort(lib, keys, values, bits)
        expect = np.argsort(keys, kind="stable").astype(np.uint32)
        np.testing.assert_array_equal(v_out, expect)
        np.testing.assert_array_equal(k_out, keys[expect])


def test_noalloc_sort_rejects_oversized_input():
    from gs_b200 import cuda

    lib = cuda.load()
    code = lib.gs_sort_pairs_noalloc(None, None, (1 << 20) + 1, 16, None)
    assert code == cuda.GS_ERR_INVALID
    assert b"maximum" in lib.gs_last_error()


def test_noalloc_sort_trivial_sizes_and_bad_widths():
    """n = 0 and n = 1 succeed and leave the buffers as they were (the first call on the
    device still does its set-up); key widths outside 1..32 are refused."""
    import torch

    from gs_b200 import cuda

    lib = cuda.load()
    for n in (0, 1):
        keys = torch.tensor([7, 3], dtype=torch.int32, device="cuda")
        values = torch.tensor([11, 12], dtype=torch.int32, device="cuda")
        code = lib.gs_sort_pairs_noalloc(ctypes.c_void_p(keys.data_ptr()), ctypes.c_void_p(values.data_ptr()), n, 8,
                                         None)
        assert code == cuda.GS_OK, lib.gs_last_error().decode()
        assert keys.tolist() == [7, 3] and values.tolist() == [11, 12]
    keys = torch.zeros(4, dtype=torch.int32, device="cuda")
    for bits in (0, 33):
        code = lib.gs_sort_pairs_noalloc(ctypes.c_void_p(keys.data_ptr()), ctypes.c_void_p(keys.data_ptr()), 4, bits,
                                         None)
        assert code == cuda.GS_ERR_INVALID
        assert b"key_bits" in lib.gs_last_error()


def test_noalloc_sort_on_a_side_stream():
    """A sort issued on a stream other than the default one, after work queued on it."""
    import torch

    from gs_b200 import cuda

    lib = cuda.load()
    rng = np.random.default_rng(8)
    n = 70001
    keys_np = rng.integers(0, 1 << 13, n, dtype=np.uint64).astype(np.uint32)
    side = torch.cuda.Stream()
    with torch.cuda.stream(side):
        keys = torch.from_numpy(keys_np.view(np.int32)).cuda(non_blocking=False)
        values = torch.arange(n, dtype=torch.int32, device="cuda")
        keys.add_(0)  # queued on the side stream ahead of the sort
        code = lib.gs_sort_pairs_noalloc(ctypes.c_void_p(keys.data_ptr()), ctypes.c_void_p(values.data_ptr()), n, 13,
                                         ctypes.c_void_p(side.cuda_stream))
    assert code == cuda.GS_OK, lib.gs_last_error().decode()
    side.synchronize()
    expect = np.argsort(keys_np, kind="stable").astype(np.uint32)
    np.testing.assert_array_equal(values.cpu().numpy().view(np.uint32), expect)
    np.testing.assert_array_equal(keys.cpu().numpy().view(np.uint32), keys_np[expect])
