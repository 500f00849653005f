"""bevy_xpbd_b200 — B200-native (sm_100a) XPBD cloth substep with the interface of the `bevy_softbody` crate.

The solver runs in libxpbd_cuda.so (hand-written CUDA kernels behind the C ABI of include/xpbd_cuda.h); this package
is the host-side binding (plugin.py), the seeded workload generators (workloads.py) and the build recipe (build.py).
"""
from ._native import XpbdError, load  # noqa: F401
from .plugin import (  # noqa: F401
    ALL, COLLISION_NONE, COLLISION_REST_FILTER, COLLISION_RING_FILTER, INNER_ITERS, JACOBI_DEFAULT_OMEGA,
    LAMBDA_PER_SUBSTEP, LAMBDA_RESET_PER_ITERATION, ORDER_COLOR_INDEX, ORDER_COLOR_REFERENCE, ORDER_PRESORTED,
    RELAX_AVERAGE, RELAX_OMEGA, SOLVER_GAUSS_SEIDEL, SOLVER_JACOBI, SUBSTEPS, ClothComputePlugin,
    ClothMaterialPlugin, ClothSimConfig, ClothSimUniforms, XpbdCpuTimeStepParams,
)
