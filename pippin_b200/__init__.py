"""pippin_b200: batched FP64 rigid-body physics for Pippin on one NVIDIA B200.

The CUDA backend (sm_100a kernels + C-ABI, lib/libpippin_b200.so) plugs in
behind the reference's `Physics` trait; `CudaPhysics` is its Python face.
"""
from .physics import (CameraDesc, CudaPhysics, Dims, Field, GeomVisual, Mesh, Param, PhysicsError, Scene, Shape,
                      Solver, WarmStart)

__all__ = ["CudaPhysics", "Dims", "Field", "Param", "PhysicsError", "Scene", "GeomVisual", "Mesh", "CameraDesc",
           "Shape", "Solver", "WarmStart"]
