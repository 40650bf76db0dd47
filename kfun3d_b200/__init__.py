"""kfun3d_b200: KFUN3D's pseudo-transient Newton-Krylov hot path on B200.

The compute path is the C ABI of ``kfun3d_b200/_lib/libkfun3d_b200.so``
(declared in ``include/kfun3d_b200.h``): the reference's own entry points
(ComputeFlux, ComputeTimeStep, ComputeA, ComputeNumericalILU,
ComputeSparseTriangularSolve, ComputeForces, the BLAS-1 helpers and Kernel)
implemented with hand-written sm_100a kernels.  This package is a thin Python
mirror of that interface for tests, benchmarks and scripting.  Importing it
fails loudly when the library has not been built; there is no CPU fallback.
"""
from .api import (  # noqa: F401
    KFUN3D_MODE_EXACT, KFUN3D_MODE_FAST, Mesh, SolverParams, Step, generate_mesh, lib,
    set_aoa, get_aoa, freestream, set_mode, get_mode, set_precision, set_ilu_order, get_ilu_order, set_schwarz, get_schwarz,
    set_first_order,
    set_verbose, last_status, last_error, clear_status, set_abort_on_error,
    launch_count, reset_launch_count, LIB_PATH,
)
