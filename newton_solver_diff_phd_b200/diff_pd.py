"""``SolverDiffPD``: the reference's DiffPD ``pd_eigen`` forward step on sm_100a.

This mirrors ``SolverDiffPD`` of the reference
(``src/newton_solver_diff_phd/_src/solvers/diff_pd/solver.py:65-591``): the
same keywords, validation messages, state-force packing, status bits and
``check_status`` / ``read_status``, ``iterations``, ``positions``,
``velocities``, ``notify_model_changed`` and ``step``. Each step minimises
``Phi(x) = 1/2 m/h^2 |x - rhs|^2 + E_pd(x)`` by L-BFGS with the constant
projective-dynamics matrix as initial Hessian and a backtracking Armijo line
search, in one persistent cooperative launch of the library
(``pd_diffpd_step``); the matrix and its exact inverse factor are those of a
DiffPhD solver built with ``mu = w_c / 2`` and ``lambda = w_v`` on every
element. There is no CPU fallback.
"""

from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from .solver import ConvergenceError, Tape, _stream

# Parameter counts of the reference state forces (solver.py:20-21).
STATE_FORCES = {"planar_contact": 8, "arc_contact": 15}
STATE_FORCE_WIDTH = 18
STATUS_NOT_CONVERGED = 1
STATUS_SINGULAR = 2
STATUS_LINE_SEARCH = 4


def pack_state_force(kind: str, parameters) -> tuple[int, np.ndarray]:
    """``(kind code, packed row)`` of one contact state force, as the reference packs it."""
    if kind not in STATE_FORCES:
        raise ValueError("state force kinds are 'planar_contact' and 'arc_contact'")
    values = np.asarray(parameters, dtype=np.float64)
    if values.shape != (STATE_FORCES[kind],) or not np.isfinite(values).all():
        raise ValueError(f"{kind} takes {STATE_FORCES[kind]} finite parameters")
    row = np.zeros(STATE_FORCE_WIDTH, dtype=np.float64)
    if kind == "planar_contact":
        normal, offset = values[:3], values[3]
        norm = np.linalg.norm(normal)
        if not norm > 1.0e-5:
            raise ValueError("planar_contact: Singular normal.")
        row[:3] = normal / norm
        row[3] = offset / norm
        row[4] = int(values[4])
        row[5:8] = values[5:8]
        return 0, row
    axis, start = values[3:6], values[6:9]
    if np.linalg.norm(axis) == 0.0 or np.linalg.norm(start) == 0.0:
        raise ValueError("arc_contact direction and start vectors must be nonzero")
    axis = axis / np.linalg.norm(axis)
    start = start / np.linalg.norm(start)
    row[:3] = values[:3]
    row[3:6] = axis
    row[6:9] = start
    row[9:12] = np.cross(axis, start)
    row[12:14] = values[9:11]
    row[14] = int(values[11])
    row[15:18] = values[12:15]
    return 1, row


def _positive_integer(name: str, value, minimum: int) -> int:
    if isinstance(value, bool) or not isinstance(value, (int, np.integer)) or value < minimum:
        raise ValueError(f"{name} must be an integer >= {minimum}")
    return int(value)


class SolverDiffPD:
    """The DiffPD ``pd_eigen`` forward step (``use_bfgs = 1``) on the B200 library.

    Keywords and conventions are the reference's (see the module docstring):
    every particle has the mass ``density * Vbar``, every element the mean
    rest volume ``Vbar``, the energy weights are global scalars, gravity and
    the contacts are explicit state forces of the start-of-step state, and
    particles with zero inverse mass are held at their start positions.

    Added keywords: ``blocks`` (persistent grid size, 0 = automatic) and
    ``recursion``: ``"two_loop"`` runs the reference's two loops (one team
    sum per stored pair and loop); ``"gram"`` runs the same recursion from
    the Gram matrix ``s_i . y_j`` of the stored pairs and the products
    ``s_i . g`` (two batched team sums per iteration), with its dot products
    rounded in another order.
    """

    ConvergenceError = ConvergenceError

    def __init__(self, model, *, density: float, corotated_stiffness: float | None = None,
                 volume_stiffness: float | None = None, state_forces=(), gravity=None, rest_positions=None,
                 max_pd_iter: int = 4000, max_ls_iter: int = 10, abs_tol: float = 1.0e-9, rel_tol: float = 1.0e-4,
                 bfgs_history_size: int = 10, blocks: int = 0, recursion: str = "two_loop"):
        if model.tet_count == 0 or model.particle_count == 0:
            raise ValueError("SolverDiffPD requires tetrahedral soft bodies")
        if getattr(model, "body_count", 0) or getattr(model, "hex_count", 0):
            raise ValueError("SolverDiffPD accepts tetrahedral particles without rigid bodies or hexahedra")
        if not np.isfinite(density) or density <= 0:
            raise ValueError("density must be finite and positive")
        for name, value in (("corotated_stiffness", corotated_stiffness), ("volume_stiffness", volume_stiffness)):
            if value is not None and (not np.isfinite(value) or value < 0):
                raise ValueError(f"{name} must be None or finite and nonnegative")
        for name, value in (("abs_tol", abs_tol), ("rel_tol", rel_tol)):
            if not np.isfinite(value) or value < 0:
                raise ValueError(f"{name} must be finite and nonnegative")
        self.max_pd_iter = _positive_integer("max_pd_iter", max_pd_iter, 1)
        self.max_ls_iter = _positive_integer("max_ls_iter", max_ls_iter, 1)
        self.bfgs_history_size = _positive_integer("bfgs_history_size", bfgs_history_size, 2)
        if self.bfgs_history_size > 32:
            raise ValueError("bfgs_history_size must be at most 32")
        if recursion not in ("two_loop", "gram"):
            raise ValueError("recursion must be 'two_loop' or 'gram'")
        self.recursion = recursion
        self.abs_tol = float(abs_tol)
        self.rel_tol = float(rel_tol)
        self.corotated_stiffness = None if corotated_stiffness is None else float(corotated_stiffness)
        self.volume_stiffness = None if volume_stiffness is None else float(volume_stiffness)
        packed = []
        for entry in state_forces:
            if len(entry) != 2:
                raise ValueError("state_forces entries are (kind, parameters)")
            packed.append(pack_state_force(*entry))
        self.gravity = None
        if gravity is not None:
            self.gravity = np.asarray(gravity, dtype=np.float64)
            if self.gravity.shape != (3,) or not np.isfinite(self.gravity).all():
                raise ValueError("gravity must be three finite values")
        self.model = model
        self.device = model.particle_q.device
        self._n = model.particle_count
        tets = model.tet_indices.cpu().numpy().reshape(-1, 4).astype(np.int32)
        if not np.array_equal(np.unique(tets), np.arange(self._n)):
            raise ValueError("Every particle must belong to a tetrahedron")
        if rest_positions is None:
            rest = model.particle_q.detach().cpu().numpy().astype(np.float64)
        else:
            rest = np.array(rest_positions, dtype=np.float64, copy=True)
            if rest.shape != (self._n, 3) or not np.isfinite(rest).all():
                raise ValueError("rest_positions must be finite with shape (particle_count, 3)")
        # Rest gradients G = [-(B0 + B1 + B2); B0; B1; B2] with B the inverse
        # rest edge matrix, and the sequentially summed mean volume
        # (TetDeformable::InitializeFiniteElementSamples, Mesh::ComputeElementVolume).
        corners = rest[tets]
        edges = np.transpose(corners[:, 1:] - corners[:, :1], (0, 2, 1))
        a, b, c = edges[:, :, 0], edges[:, :, 1], edges[:, :, 2]
        cross = np.stack((b[:, 1] * c[:, 2] - b[:, 2] * c[:, 1], b[:, 2] * c[:, 0] - b[:, 0] * c[:, 2],
                          b[:, 0] * c[:, 1] - b[:, 1] * c[:, 0]), axis=1)
        volumes = np.abs((a[:, 0] * cross[:, 0] + a[:, 1] * cross[:, 1] + a[:, 2] * cross[:, 2]) / 6.0)
        if not np.all(np.isfinite(volumes)) or np.any(volumes <= 0):
            raise ValueError("tetrahedra must have nondegenerate rest shapes")
        inverse = np.linalg.inv(edges)
        self._tets = tets
        self._gradients = np.ascontiguousarray(np.concatenate((-inverse.sum(axis=1)[:, None], inverse), axis=1))
        total = 0.0
        for volume in volumes.tolist():
            total += volume
        self.mean_volume = total / len(volumes)
        self.density = float(density)
        self.particle_mass = self.density * self.mean_volume
        self._blocks = int(blocks)
        self._packed = packed
        self._lib = _lib.library()
        self._handle = None
        self._free = None
        self._factor_key = None
        self._model_changed = True

    # ------------------------------------------------------------------ status
    def read_status(self) -> int:
        """Read and clear the status bits without raising; one host synchronization.

        Bits: 1 a step reached ``max_pd_iter``, 2 a singular deformation
        gradient met the volume projection, 4 a line search used all
        ``max_ls_iter`` halvings (informational, as in the reference).
        """
        if self._handle is None:
            return 0
        bits = ctypes.c_int32()
        _lib.check(self._lib.pd_read_status(self._handle, ctypes.byref(bits), _stream()))
        return int(bits.value)

    def check_status(self) -> None:
        """Read and clear the status bits, raising the reference's failures since the last check."""
        bits = self.read_status()
        if bits & STATUS_SINGULAR:
            raise ValueError("DiffPD volume projection met a singular deformation gradient (reference 'Singular F.')")
        if bits & STATUS_NOT_CONVERGED:
            raise ConvergenceError(f"PD method fails to converge within {self.max_pd_iter} iterations")

    def _results(self, iterations=False):
        positions, velocities, count = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_int32()
        _lib.check(self._lib.pd_diffpd_results(self._handle, ctypes.byref(positions), ctypes.byref(velocities),
                                               ctypes.byref(count) if iterations else None, _stream()))
        return positions.value, velocities.value, int(count.value)

    @property
    def iterations(self) -> np.ndarray:
        """L-BFGS iteration count of the last step, as a one-entry array (``solver.iterations``)."""
        return np.array([self._results(iterations=True)[2]], dtype=np.int32)

    def _view(self, pointer) -> torch.Tensor:
        return torch.as_tensor(_lib.DeviceView(pointer, (self._n, 3), "<f8", self), device=self.device)

    @property
    def positions(self) -> torch.Tensor:
        """Float64 positions after the last step, before rounding into the state."""
        return self._view(self._results()[0])

    @property
    def velocities(self) -> torch.Tensor:
        """Float64 velocities after the last step, before rounding into the state."""
        return self._view(self._results()[1])

    def notify_model_changed(self, flags: int = 0) -> None:
        """Rebuild the Dirichlet mask and the factor before the next step."""
        if torch.cuda.is_current_stream_capturing():
            raise RuntimeError("notify_model_changed cannot run during graph capture")
        self._model_changed = True

    # ------------------------------------------------------------------ build and step
    def _validate_model(self):
        model = self.model
        for name, description in (("tri_materials", "triangle elasticity"), ("spring_stiffness", "springs"),
                                  ("edge_bending_properties", "edge bending")):
            array = getattr(model, name, None)
            if array is not None and array.numel() and bool(torch.any(array != 0)):
                raise ValueError(f"SolverDiffPD does not support {description}")
        flags = getattr(model, "particle_flags", None)
        if flags is not None and bool(torch.any((flags & 1) == 0)):
            raise ValueError("SolverDiffPD requires ACTIVE particles; pin particles with zero inverse mass")
        inverse_mass = model.particle_inv_mass.detach().cpu().numpy()
        if not np.all(np.isfinite(inverse_mass)) or np.any(inverse_mass < 0):
            raise ValueError("Particle inverse masses must be finite and nonnegative")
        return inverse_mass > 0

    def _build(self, dt: float):
        if torch.cuda.is_current_stream_capturing():
            raise RuntimeError("SolverDiffPD must factor A; step once outside graph capture first")
        free = self._validate_model()
        if self._handle is None or not np.array_equal(free, self._free):
            self._close()
            free_u8 = np.ascontiguousarray(free.astype(np.uint8))
            desc = _lib.PdMeshDesc(self._n, len(self._tets), 4,
                                   self._tets.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                                   self._gradients.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), self.mean_volume,
                                   free_u8.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)))
            options = _lib.PdOptions(0, 1, 0.0, 0.0, 0, self.density, 0, _lib.PRECISION_FP64, 0, self._blocks, 1, 0, 0,
                                     0)
            handle = ctypes.c_void_p()
            index = self.device.index if self.device.index is not None else torch.cuda.current_device()
            _lib.check(self._lib.pd_create(ctypes.byref(desc), ctypes.byref(options), index, ctypes.byref(handle)))
            self._handle = handle
            self._free = free
            kinds = np.ascontiguousarray([k for k, _ in self._packed], dtype=np.int32)
            rows = np.ascontiguousarray([r for _, r in self._packed], dtype=np.float64).reshape(-1, STATE_FORCE_WIDTH)
            _lib.check(self._lib.pd_diffpd_set_state_forces(self._handle, len(self._packed), _lib.ptr(kinds),
                                                            _lib.ptr(rows)))
        # A = m/h^2 I + (w_c + w_v) Vbar sum G G^T: the PD matrix of mu = w_c/2, lambda = w_v.
        # (The solver requires mu > 0: without a corotated energy a negligible
        # mu stands in for zero.)
        mu = max(0.5 * (self.corotated_stiffness or 0.0), 1.0e-300)
        lam = self.volume_stiffness or 0.0
        materials = np.ascontiguousarray(np.tile([mu, lam], (len(self._tets), 1)), dtype=np.float64)
        _lib.check(self._lib.pd_set_materials(self._handle, _lib.ptr(materials)))
        _lib.check(self._lib.pd_build(self._handle, float(dt)))
        self._factor_key = dt
        self._model_changed = False

    def _options(self):
        return _lib.PdDiffPdOptions(self.max_pd_iter, self.max_ls_iter, self.bfgs_history_size,
                                    int(self.corotated_stiffness is not None), int(self.volume_stiffness is not None),
                                    self.corotated_stiffness or 0.0, self.volume_stiffness or 0.0, self.abs_tol,
                                    self.rel_tol,
                                    _lib.DIFFPD_GRAM if self.recursion == "gram" else _lib.DIFFPD_TWO_LOOP)

    def step(self, state_in, state_out, control, contacts, dt: float) -> None:
        """Advance one step of length ``dt`` [s] on the current CUDA stream."""
        if contacts is not None:
            raise NotImplementedError("SolverDiffPD does not consume Newton contacts; pass contacts=None")
        if Tape.current() is not None:
            raise NotImplementedError("SolverDiffPD has no backward pass yet; step outside a Tape")
        if not np.isfinite(dt) or dt <= 0:
            raise ValueError("dt must be finite and positive")
        if state_in is state_out or state_in.particle_q.data_ptr() == state_out.particle_q.data_ptr():
            raise ValueError("DiffPD requires distinct input and output states")
        dt = float(dt)
        if self._model_changed or self._factor_key != dt:
            self._build(dt)
        if self.gravity is not None:
            gravity = self.gravity
        else:
            gravity = self.model.gravity[0].detach().cpu().numpy().astype(np.float64)
        gravity = np.ascontiguousarray(gravity, dtype=np.float64)
        options = self._options()
        tensors = [t.contiguous() for t in (state_in.particle_q, state_in.particle_qd, state_in.particle_f)]
        _lib.check(self._lib.pd_diffpd_step(self._handle, ctypes.byref(options), *(_lib.ptr(t) for t in tensors),
                                            _lib.ptr(gravity), dt, _lib.ptr(state_out.particle_q),
                                            _lib.ptr(state_out.particle_qd), _stream()))

    def _close(self):
        if self._handle is not None:
            self._lib.pd_destroy(self._handle)
            self._handle = None

    def __del__(self):
        try:
            self._close()
        except Exception:
            pass
