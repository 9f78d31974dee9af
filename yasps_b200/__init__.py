"""yasps_b200: the YASPS Newton inner loop on NVIDIA B200 (sm_100a).

Element gradients and SPD-projected Hessians, deterministic block assembly,
symmetric block SpMV and PCG (block-Jacobi or multilevel additive Schwarz)
as hand-written CUDA behind a C ABI (``include/ys_newton.h``), driven from
the reference's scene / energy / solver API.
"""

from .graph import attribute, connectivity, mesh, primitive, primitiveUnion  # noqa: F401
from .energies import inertia, stable_neo_hookean  # noqa: F401
from .hessian import hessian, vector  # noqa: F401
from .scene import minimizer, scene  # noqa: F401
from .solver import jacobianPCGSolver, masSolver, solver  # noqa: F401

__all__ = ["attribute", "connectivity", "mesh", "primitive", "primitiveUnion", "inertia", "stable_neo_hookean",
           "hessian", "vector", "minimizer", "scene", "solver", "jacobianPCGSolver", "masSolver"]
