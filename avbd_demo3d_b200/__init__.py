"""B200-native (sm_100a) Augmented Vertex Block Descent step.

A drop-in for the reference's ``Solver::step`` (ts-jls/avbd-demo3d): the whole step
(broadphase, box narrowphase, warm start, coloured primal solve, dual update, velocity
update) runs as CUDA kernels behind the C ABI in include/avbd_cuda.h.
"""
from . import scenes  # noqa: F401
from .solver import (CudaAvbdBackend, IgnoreCollision, Joint, Rigid, Solver, Spring,  # noqa: F401
                     World, box_properties, rotate32)

__all__ = ["scenes", "World", "Solver", "Rigid", "Joint", "Spring", "IgnoreCollision", "CudaAvbdBackend",
           "box_properties", "rotate32"]
