"""B200-native DiffPhD projective-dynamics step and adjoint.

``SolverDiffPhD`` keeps the interface of the reference Newton solver plugin
(``src/newton_solver_diff_phd/_src/solvers/diff_phd/solver.py``); its step and
backward pass run as persistent sm_100a kernels behind the C ABI in
``include/pd_b200.h``. ``SolverDiffPD`` is the reference's DiffPD ``pd_eigen``
forward step (L-BFGS on the same projective-dynamics matrix) on the same library.
"""

from .meshes import Mesh
from .model import Control, Model, ModelBuilder, State
from .diff_pd import SolverDiffPD
from .solver import ConvergenceError, HexElements, SolverDiffPhD, Tape

__all__ = [
    "SolverDiffPhD",
    "SolverDiffPD",
    "ConvergenceError",
    "Tape",
    "Mesh",
    "HexElements",
    "Model",
    "ModelBuilder",
    "State",
    "Control",
]
