"""B200 (sm_100a) implementation of Plato Analyze's linear-tet hot path.

The compute lives in libpa_b200.so (CUDA kernels behind the C ABI of
include/pa_b200.h); this package is the host-side mirror of the reference's
Problem / VectorFunction / PhysicsScalarFunction interfaces over that ABI.
Importing it loads the library and fails if it has not been built.
"""
from . import _abi
from .api import LearnedPreconditioner, Mesh, PhysicsScalarFunction, Problem, SolveOptions, VectorFunction, read_exodus

_abi.load()

__all__ = ["Mesh", "Problem", "VectorFunction", "PhysicsScalarFunction", "SolveOptions",
           "LearnedPreconditioner", "read_exodus"]
