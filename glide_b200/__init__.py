"""glide_b200: B200-native coupled SSA momentum + mass-conservation solver.

Drop-in for the hot path of JacobDowns/glide: the same Python surface
(`Multigrid`, field managers, `FASCDSolver` / `FASAdjointSolver` and their
option objects, `IceDynamics`, `GlideStep`, plus the `IcePhysics` facade) over
a C-ABI library of hand-written sm_100a CUDA kernels (include/glide_b200.h).
Arrays are torch tensors; the default precision is binary64.
"""
__version__ = "0.1.0"

from ._lib import GlideError  # noqa: F401


def __getattr__(name):
    # lazy imports keep `import glide_b200` cheap and CPU-safe
    if name in ("Multigrid", "FASCDSolver", "FASAdjointSolver"):
        from . import multigrid
        return getattr(multigrid, name)
    if name == "IceDynamics":
        from .model import IceDynamics
        return IceDynamics
    if name == "IcePhysics":
        from .physics import IcePhysics
        return IcePhysics
    if name == "Grid":
        from .grid import Grid
        return Grid
    if name == "GlideStep":
        from .torch import GlideStep
        return GlideStep
    raise AttributeError(name)
