"""B200 (sm_100a) 3D Gaussian Splatting training step: Python host side.

The compute path is libgs_cuda (CUDA kernels behind the C ABI of include/gs_cuda.h);
this package holds the reference's host-side pieces needed to drive it from Python:
FrameData and the option schedules (`frame`), seeded synthetic scenes (`scenes`) and the
ctypes binding (`cuda`).
"""
from . import frame, scenes  # noqa: F401
