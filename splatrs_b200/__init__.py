"""splatrs_b200: the differentiable render-and-train path of splatrs (3D Gaussian
splatting) as hand-written sm_100a CUDA kernels behind a C ABI (include/splat_gpu.h).

Submodules:
  build   nvcc recipe for the in-tree libsplatrs_b200.so
  _lib    ctypes binding of the C ABI (raises if the library is missing)
  gpu     Python mirror of the reference API on device tensors
  scenes  seeded synthetic scenes with the benchmark configurations' shapes
"""
__all__ = ["build", "gpu", "scenes"]
