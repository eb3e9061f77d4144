"""B200-native DiffPhD projective-dynamics step and adjoint.

``SolverDiffPhD`` keeps the interface of the reference Newton solver plugin
(``src/newton_solver_diff_phd/_src/solvers/diff_phd/solver.py``); its step and
backward pass run as persistent sm_100a kernels behind the C ABI in
``include/pd_b200.h``.
"""

from .meshes import Mesh
from .model import Control, Model, ModelBuilder, State
from .solver import ConvergenceError, HexElements, SolverDiffPhD, Tape

__all__ = [
    "SolverDiffPhD",
    "ConvergenceError",
    "Tape",
    "Mesh",
    "HexElements",
    "Model",
    "ModelBuilder",
    "State",
    "Control",
]
