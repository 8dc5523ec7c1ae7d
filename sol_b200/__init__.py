"""B200 path tracer behind SoL's Scene / Renderer / Image interface.

Submodules:
  build     compiles the CUDA library (sol_b200/lib/libsol_gpu.so)
  capi      ctypes binding of include/sol_gpu.h (fails to import without the library)
  scene     flat scene description -> SolGpuSceneDesc
  scenes    seeded procedural scenes of the benchmark configurations
  renderer  Image / GpuScene / GpuPathTracer, the Python mirror of SoL's renderer API
"""
__all__ = ["build", "capi", "scene", "scenes", "renderer"]
