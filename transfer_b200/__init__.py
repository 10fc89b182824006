"""B200-native radiative-transfer hot path of uranix/Transfer.

The even-parity spherical-harmonics Galerkin operator on P1 tetrahedral
meshes, its CG / defect-correction solves and the moment reduction, as CUDA
kernels for sm_100a behind a C ABI (include/transfer_b200.h); and the
discrete-ordinates upwind sweep with scattering source iteration over the
same problem data (Sweep).  This package
is the Python binding of that library; it has no CPU fallback.
"""
from ._lib import (TR_BC_INCIDENT, TR_BC_REFLECTIVE, TR_BC_VACUUM, TR_ENGINE_GRAPH, TR_ENGINE_LAUNCH,  # noqa: F401
                   TR_ENGINE_PERSISTENT, TR_ENGINE_PERSISTENT_SR, TR_MODE_FP64, TR_MODE_MIXED, TR_PREC_JACOBI, TR_PREC_NONE,
                   TR_PREC_REFERENCE, TR_OPERATOR_SIMT, TR_OPERATOR_TENSOR, LIB_PATH, TransferError, check, lib)
from .core import (FACE_DTYPE, TET_DTYPE, AngularData, Config, CudaContext, MeshData, Physics,  # noqa: F401
                   solve_options, trieig)
from .sweep import (Sweep, adjoint_gradient, adjoint_problem, lebedev, ordinates_product,  # noqa: F401
                    sweep_apply_batch, sweep_autotune_batch, sweep_solve_batch)

__all__ = ["AngularData", "Config", "CudaContext", "MeshData", "Physics", "Sweep", "TransferError",
           "ordinates_product", "lebedev", "sweep_apply_batch", "sweep_autotune_batch", "sweep_solve_batch", "solve_options", "trieig", "lib", "LIB_PATH"]
