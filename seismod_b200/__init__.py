"""seismod_b200 -- the seismod FDTD hot path (e_iso split-PML 2D elastic and
a_iso_3d CPML 3D acoustic time steps) on NVIDIA B200 (sm_100a).

The compute path is libseismod_gpu.so (C ABI: include/seismod_gpu.h):
hand-written CUDA kernels behind a C host that keeps the reference's file
formats and set-up arithmetic.  This package adds a ctypes front end
(api), the reference file formats (formats) and seeded workloads
(workloads).
"""
__all__ = ["api", "formats", "workloads"]
