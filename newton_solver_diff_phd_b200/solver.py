"""``SolverDiffPhD``: the reference solver plugin's interface over the sm_100a library.

This mirrors ``SolverDiffPhD`` of the reference
(``src/newton_solver_diff_phd/_src/solvers/diff_phd/solver.py:47-827``): the same
constructor keywords, validation messages, status bits, ``check_status`` /
``read_status``, ``notify_model_changed``, ``deformation_determinants`` and
``step(state_in, state_out, control, contacts, dt, dirichlet_positions=...)``.
All arithmetic of the step and its adjoint runs in the CUDA library through
the C ABI (``include/pd_b200.h``); this module validates inputs with NumPy
exactly like the reference, computes the rest-shape data, and hands device
pointers to the library. There is no CPU fallback.

Added keywords: ``precision`` (``"fp64"`` as the reference; ``"fp32+refine"``:
float32 factor products corrected by a float64 residual every iteration, so
the converged positions are the float64 solver's; ``"fp32"``: float32 local
projections as well, whose fixed point moves by about cond(A) times the
float32 rounding), ``adjoint`` (``"reference"``: the reference's mean-weight
local Jacobian; ``"exact"``: per-element weights, the derivative of the
forward map), ``adjoint_solver`` (``"auto"``: the reference's Anderson fixed
point for ``"reference"``, conjugate gradients preconditioned by the factor for
``"exact"``; or ``"fixed_point"`` / ``"cg"``), ``blocks`` (persistent grid
size, 0 = automatic), ``resident`` and ``svd_warm_start`` (kernel tuning).

``state_dtype=torch.float64`` (added) keeps particle states and their
gradients in float64 between steps; the default float32 matches Newton.

Differences from the reference: frictional boundaries are not available in
this build (``NotImplementedError``; ``mesh_contact`` is); gravity is taken from
one world; Hex8 steps can be recorded for the backward pass (the reference
rejects them, ``solver.py:726-729``).
"""

from __future__ import annotations

import ctypes
import threading

import numpy as np
import torch

from . import _lib
from .meshes import Mesh

MATERIALS = {"pd": 0, "neo_hookean": 1}
BOUNDARY_KINDS = {"planar": 0, "spherical": 1, "mesh": 2}
PRECISIONS = {"fp64": _lib.PRECISION_FP64, "fp32+refine": _lib.PRECISION_FP32_REFINE, "fp32": _lib.PRECISION_FP32}
ADJOINTS = {"reference": _lib.ADJOINT_REFERENCE, "exact": _lib.ADJOINT_EXACT}
ADJOINT_SOLVERS = {"auto": 0, "fixed_point": 1, "cg": 2}
MAX_WINDOW = 8


class ConvergenceError(RuntimeError):
    """A forward step or a recorded backward fixed point did not converge (``exceptions.py:7``)."""


class Tape:
    """Records differentiable solver steps, like ``wp.Tape`` in the reference.

    ``with Tape() as tape: solver.step(...)`` records; ``tape.backward(grads={tensor: seed})``
    seeds output gradients and replays the recorded backward passes in reverse,
    accumulating into the ``.grad`` of the step inputs (and of
    ``model.tet_materials`` / activations when those have ``.grad``).
    """

    _local = threading.local()

    def __init__(self):
        self.records = []

    @classmethod
    def current(cls):
        stack = getattr(cls._local, "stack", None)
        return stack[-1] if stack else None

    def __enter__(self):
        if not hasattr(Tape._local, "stack"):
            Tape._local.stack = []
        Tape._local.stack.append(self)
        return self

    def __exit__(self, *exc):
        Tape._local.stack.pop()
        return False

    def record_func(self, backward, arrays):
        self.records.append((backward, arrays))

    def backward(self, loss=None, grads=None):
        if loss is not None:
            raise NotImplementedError("seed output gradients with grads={tensor: value}")
        for tensor, value in (grads or {}).items():
            if tensor.grad is None:
                tensor.grad = torch.zeros_like(tensor)
            tensor.grad.add_(value.to(tensor.grad.dtype))
        for backward, _arrays in reversed(self.records):
            backward()

    def reset(self):
        self.records.clear()


def _grad(tensor):
    return None if tensor is None else tensor.grad


def _stream() -> int:
    return torch.cuda.current_stream().cuda_stream


class HexElements:
    """Validated binary-order cubes and their shared Gauss gradients (``hex.py:27-92``)."""

    def __init__(self, mesh, particle_count):
        vertices = np.asarray(mesh.vertices, dtype=np.float64)
        indices = np.asarray(mesh.indices)
        if vertices.shape != (particle_count, 3) or not np.isfinite(vertices).all():
            raise ValueError("hex_mesh vertices must contain a finite rest position for every model particle")
        if (
            indices.ndim != 2
            or indices.shape[1] != 8
            or len(indices) == 0
            or not np.issubdtype(indices.dtype, np.integer)
            or np.any(indices < 0)
            or np.any(indices >= particle_count)
            or np.any(np.diff(np.sort(indices, axis=1), axis=1) == 0)
        ):
            raise ValueError("hex_mesh indices must have shape (element_count,8) with eight distinct valid vertices")
        if not np.array_equal(np.unique(indices), np.arange(particle_count)):
            raise ValueError("Every particle must belong to a hexahedron")
        self.elements = indices.astype(np.int32, copy=True)
        corners = np.array([[a, b, c] for a in range(2) for b in range(2) for c in range(2)], dtype=np.float64)
        rest = vertices[self.elements]
        edges = rest[:, [1, 2, 4]] - rest[:, :1]
        self.volumes = np.abs(np.einsum("ij,ij->i", edges[:, 0], np.cross(edges[:, 1], edges[:, 2])))
        # Python's sequential sum over the cells, divided by the count.
        self.mean_volume = sum(float(value) for value in self.volumes) / len(self.elements)
        if not np.isfinite(self.mean_volume) or self.mean_volume <= 0 or np.any(self.volumes <= 0):
            raise ValueError("Hex8 cells must have positive, finite rest volume")
        dx = self.mean_volume ** (1.0 / 3.0)
        expected = rest[:, :1] + dx * corners[None]
        if not np.allclose(rest, expected, rtol=0.0, atol=1.0e-9 * dx):
            raise ValueError("Reference Hex8 requires equally sized axis-aligned cubes in binary corner order")
        self.width = dx
        inv_dx = 1.0 / dx
        samples = ((corners - 0.5) * (1.0 / np.sqrt(3.0)) + 0.5) * dx
        gradients = np.empty((8, 8, 3), dtype=np.float64)
        for s, point in enumerate(samples):
            nx, ny, nz = point * inv_dx
            cnx, cny, cnz = 1.0 - nx, 1.0 - ny, 1.0 - nz
            # Trilinear shape gradients; products in the reference's order.
            gradients[s] = [
                [-inv_dx * cny * cnz, cnx * -inv_dx * cnz, cnx * cny * -inv_dx],
                [-inv_dx * cny * nz, cnx * -inv_dx * nz, cnx * cny * inv_dx],
                [-inv_dx * ny * cnz, cnx * inv_dx * cnz, cnx * ny * -inv_dx],
                [-inv_dx * ny * nz, cnx * inv_dx * nz, cnx * ny * inv_dx],
                [inv_dx * cny * cnz, nx * -inv_dx * cnz, nx * cny * -inv_dx],
                [inv_dx * cny * nz, nx * -inv_dx * nz, nx * cny * inv_dx],
                [inv_dx * ny * cnz, nx * inv_dx * cnz, nx * ny * -inv_dx],
                [inv_dx * ny * nz, nx * inv_dx * nz, nx * ny * inv_dx],
            ]
        self.sample_gradients = gradients


class SolverDiffPhD:
    """Projective dynamics with the executed conventions of the DiffPhD reference, on sm_100a.

    See the module docstring for the keyword surface; the arithmetic follows
    the reference step and adjoint (``solver.py``, ``kernels.py``, ``hex.py``,
    ``anderson.py``, ``adjoint.py``) with float64 as the reference precision.
    """

    ConvergenceError = ConvergenceError

    def __init__(
        self,
        model,
        *,
        density: float,
        material: str = "pd",
        max_iterations: int = 10000,
        abs_tol: float = 1.0e-9,
        rel_tol: float = 1.0e-6,
        anderson_window: int = 5,
        muscle_directions=None,
        muscle_stiffness=None,
        integrate_pinned_velocities: bool = False,
        frictional_boundary=None,
        frictional_vertices=None,
        friction: float = 0.0,
        restitution: float = 0.0,
        mesh_contact=None,
        hex_mesh=None,
        hex_materials=None,
        muscle_targets=None,
        planar_energies=None,
        precision: str = "fp64",
        adjoint: str = "reference",
        blocks: int = 0,
        resident: bool = True,
        svd_warm_start: bool = True,
        adjoint_solver: str = "auto",
        state_dtype: torch.dtype = torch.float32,
    ):
        if material not in MATERIALS:
            raise ValueError("material must be 'pd' or 'neo_hookean'")
        if model.particle_count == 0 or (model.tet_count == 0 and hex_mesh is None):
            raise ValueError("SolverDiffPhD requires tetrahedral soft bodies or an explicit hex_mesh")
        if getattr(model, "body_count", 0):
            raise ValueError("SolverDiffPhD requires particles without rigid bodies; supply Hex8 using hex_mesh")
        if (hex_mesh is None) != (hex_materials is None):
            raise ValueError("hex_mesh and hex_materials must be supplied together")
        if hex_mesh is not None and model.tet_count:
            raise ValueError("hex_mesh cannot be combined with model tetrahedra")
        if hex_mesh is None and (muscle_targets is not None or planar_energies is not None):
            raise ValueError("Explicit muscle_targets and planar_energies currently require hex_mesh")
        if hex_mesh is not None and any(x is not None for x in (frictional_boundary, mesh_contact)):
            raise NotImplementedError("Hex8 currently supports planar_energies, not frictional or mesh contact")
        self._frictional_args = None
        if frictional_boundary is not None:
            self._frictional_args = self._validate_frictional(model, frictional_boundary, frictional_vertices, friction,
                                                              restitution, hex_mesh)
        elif frictional_vertices is not None or friction or restitution:
            raise ValueError("frictional_vertices, friction and restitution need a frictional_boundary")
        if mesh_contact is not None:
            if len(mesh_contact) != 7:
                raise ValueError("mesh_contact is (contact_radius, kn_left, kn_right, kf, mu, faces_a, faces_b)")
            mesh_faces = []
            for faces in mesh_contact[5:]:
                faces = np.ascontiguousarray(np.asarray(faces).reshape(-1, 3), dtype=np.int32)
                mesh_faces.append(faces)
            self._mesh_contact_args = (tuple(float(value) for value in mesh_contact[:5]), mesh_faces)
        else:
            self._mesh_contact_args = None
        if not np.isfinite(density) or density <= 0:
            raise ValueError("density must be finite and positive")
        for name, value in (("abs_tol", abs_tol), ("rel_tol", rel_tol)):
            if not np.isfinite(value) or value < 0:
                raise ValueError(f"{name} must be finite and nonnegative")
        if not np.isfinite(max_iterations) or max_iterations < 1 or int(max_iterations) != max_iterations:
            raise ValueError("max_iterations must be a positive integer")
        if int(anderson_window) != anderson_window or not 0 <= anderson_window <= MAX_WINDOW:
            raise ValueError(f"anderson_window must be an integer in [0, {MAX_WINDOW}]")
        if precision not in PRECISIONS:
            raise ValueError("precision must be 'fp64', 'fp32+refine' or 'fp32'")
        if adjoint not in ADJOINTS:
            raise ValueError("adjoint must be 'reference' or 'exact'")
        if adjoint_solver not in ADJOINT_SOLVERS:
            raise ValueError("adjoint_solver must be 'auto', 'fixed_point' or 'cg'")
        if state_dtype not in (torch.float32, torch.float64):
            raise ValueError("state_dtype must be torch.float32 (Newton states) or torch.float64")
        self.state_dtype = state_dtype
        self.model = model
        self.device = model.device
        if self.device.type != "cuda":
            raise ValueError("SolverDiffPhD runs on CUDA devices only")
        self.material = material
        self.max_iterations = int(max_iterations)
        self.abs_tol = float(abs_tol)
        self.rel_tol = float(rel_tol)
        self.precision = precision
        self.adjoint_mode = adjoint
        self.integrate_pinned_velocities = bool(integrate_pinned_velocities)
        self._n = model.particle_count
        self._hex = None if hex_mesh is None else HexElements(hex_mesh, self._n)
        if self._hex is None:
            self._tets = model.tet_indices.cpu().numpy().reshape(-1, 4).astype(np.int32)
            if not np.array_equal(np.unique(self._tets), np.arange(self._n)):
                raise ValueError("Every particle must belong to a tetrahedron")
            self._elements = self._tets
            rest_poses = model.tet_poses.cpu().numpy().astype(np.float64)
            self._gradients = np.concatenate((-rest_poses.sum(axis=1)[:, None], rest_poses), axis=1)
            self._volumes = np.abs(1.0 / np.linalg.det(rest_poses)) / 6.0
            if not np.all(np.isfinite(self._volumes)) or np.any(self._volumes <= 0):
                raise ValueError("tetrahedra must have nondegenerate rest shapes")
            self.mean_volume = float(self._volumes.mean())
            self.hex_materials = None
        else:
            self._elements = self._hex.elements
            self._volumes = self._hex.volumes
            self.mean_volume = self._hex.mean_volume
            if isinstance(hex_materials, torch.Tensor):
                if hex_materials.dtype != torch.float64:
                    raise ValueError("hex_materials tensor must be float64")
                self.hex_materials = hex_materials
            else:
                self.hex_materials = torch.tensor(np.asarray(hex_materials, dtype=np.float64), device=self.device)
            count = len(self._elements)
            if tuple(self.hex_materials.shape) not in ((count, 2), (count, 3)):
                raise ValueError("hex_materials must have shape (element_count,2 or 3): mu,lambda[,damping]")
        self._element_count = len(self._elements)
        self._sample_count = 1 if self._hex is None else 8
        self._sample_volume = self.mean_volume / self._sample_count
        worlds = model.particle_world.cpu().numpy()
        if np.any(worlds < -1) or np.any(worlds >= len(model.gravity)):
            raise ValueError("particle_world must reference an existing world or global world -1")
        if len(np.unique(np.maximum(worlds, 0))) > 1:
            raise NotImplementedError("SolverDiffPhD in this build takes gravity from a single world")
        self._gravity_world = int(max(int(worlds.max()), 0)) if len(worlds) else 0
        self.density = float(density)
        self.particle_mass = self.density * self.mean_volume
        self._initialize_muscles(muscle_directions, muscle_stiffness)
        if self._hex is not None:
            if muscle_targets is not None and not self._has_muscles:
                raise ValueError("muscle_targets requires enabled muscle_directions and muscle_stiffness")
            targets = np.ones(self._element_count) if muscle_targets is None else muscle_targets
            targets = targets.cpu().numpy() if isinstance(targets, torch.Tensor) else np.asarray(targets, np.float64)
            if targets.shape != (self._element_count,):
                raise ValueError("muscle_targets must have shape (element_count,)")
            if not np.isfinite(targets).all() or np.any(targets < 0):
                raise ValueError("muscle_targets must be finite nonnegative native target lengths")
            self.muscle_targets = torch.tensor(targets, dtype=torch.float64, device=self.device)
        self._planar = None
        if planar_energies is not None:
            self._planar = self._validate_planar(planar_energies)

        free = model.particle_inv_mass.cpu().numpy() > 0
        self._free_host = free
        lib = _lib.library()
        self._lib = lib
        indices = np.ascontiguousarray(self._elements, dtype=np.int32)
        gradients = np.ascontiguousarray(
            self._gradients if self._hex is None else self._hex.sample_gradients, dtype=np.float64
        )
        free_u8 = np.ascontiguousarray(free.astype(np.uint8))
        desc = _lib.PdMeshDesc(
            self._n,
            self._element_count,
            4 if self._hex is None else 8,
            indices.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
            gradients.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
            self.mean_volume,
            free_u8.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)),
        )
        options = _lib.PdOptions(
            MATERIALS[material],
            self.max_iterations,
            self.abs_tol,
            self.rel_tol,
            int(anderson_window),
            self.density,
            int(self.integrate_pinned_velocities),
            PRECISIONS[precision],
            ADJOINTS[adjoint],
            int(blocks),
            int(bool(resident)),
            int(bool(svd_warm_start)),
            ADJOINT_SOLVERS[adjoint_solver],
            1 if state_dtype == torch.float64 else 0,
        )
        handle = ctypes.c_void_p()
        device_index = self.device.index if self.device.index is not None else torch.cuda.current_device()
        _lib.check(lib.pd_create(ctypes.byref(desc), ctypes.byref(options), device_index, ctypes.byref(handle)))
        self._handle = handle
        self.anderson_window = int(anderson_window)
        if self._has_muscles:
            _lib.check(
                lib.pd_set_muscles(handle, _lib.ptr(self._muscle_directions_host), _lib.ptr(self._muscle_stiffness_host))
            )
        if self._hex is not None:
            self._targets_host = self.muscle_targets.cpu().numpy()
            _lib.check(lib.pd_set_muscle_targets(handle, _lib.ptr(np.ascontiguousarray(self._targets_host))))
        if self._planar is not None:
            vertices, stiffness, plane = self._planar
            _lib.check(
                lib.pd_set_planar_energies(handle, len(vertices), _lib.ptr(vertices), _lib.ptr(stiffness), _lib.ptr(plane))
            )
        if self._mesh_contact_args is not None:
            (radius, kn_left, kn_right, kf, mu), (faces_a, faces_b) = self._mesh_contact_args
            _lib.check(lib.pd_set_mesh_contact(handle, radius, kn_left, kn_right, kf, mu, len(faces_a), _lib.ptr(faces_a),
                                               len(faces_b), _lib.ptr(faces_b)))
        self.boundary_parameters = None
        self.contact_multipliers = None
        if self._frictional_args is not None:
            kind, parameters, nodes, friction_value, restitution_value, split, left, right = self._frictional_args
            _lib.check(lib.pd_set_frictional_boundary(
                handle, kind, _lib.ptr(parameters), len(nodes), _lib.ptr(nodes), friction_value, restitution_value,
                split, len(left), _lib.ptr(left), len(right), _lib.ptr(right)))
            params_ptr, multipliers_ptr, count = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_int32()
            _lib.check(lib.pd_frictional_buffers(handle, ctypes.byref(params_ptr), ctypes.byref(multipliers_ptr),
                                                 ctypes.byref(count)))
            # Views of the solver's own device arrays: edits take effect at the next step.
            self.boundary_parameters = torch.as_tensor(
                _lib.DeviceView(params_ptr.value, (1, 4), "<f8", self), device=self.device)
            self.contact_multipliers = torch.as_tensor(
                _lib.DeviceView(multipliers_ptr.value, (count.value,), "<f8", self), device=self.device)
            self.frictional_vertices = nodes
        self._x = torch.zeros((self._n, 3), dtype=torch.float64, device=self.device)
        self._factor_key = None
        self._model_changed = True
        self._recorded = None
        self._activation_source = None

    # ------------------------------------------------------------------ setup
    def _validate_frictional(self, model, boundary, vertices, friction, restitution, hex_mesh):
        """Host checks of ``frictional_boundary`` (contact.py:715-760) and the default
        registered vertices (solver.py:303-309): the mesh's face vertices, else the
        surface vertices of the tetrahedra."""
        if len(boundary) != 2:
            raise ValueError("frictional_boundary is (kind, parameters)")
        kind, parameters = boundary
        if kind not in BOUNDARY_KINDS:
            raise ValueError("frictional boundary must be 'planar', 'spherical' or 'mesh'")
        split, left, right = 0, np.zeros((0, 3), np.int32), np.zeros((0, 3), np.int32)
        if kind == "mesh":
            if len(parameters) != 4:
                raise ValueError("mesh boundary parameters are (contact_radius, split_index, faces_left, faces_right)")
            split = int(parameters[1])
            left, right = (np.ascontiguousarray(np.asarray(f, dtype=np.int32).reshape(-1, 3)) for f in parameters[2:4])
            values = np.array([float(parameters[0]), 0.0, 0.0, 0.0])
        else:
            values = np.asarray(parameters, dtype=np.float64)
            if values.shape != (4,):
                raise ValueError("frictional boundary parameters must be four finite values")
        if vertices is None:
            if kind == "mesh":
                vertices = np.unique(np.concatenate([left.reshape(-1), right.reshape(-1)]))
            else:
                tets = model.tet_indices.cpu().numpy().reshape(-1, 4)
                faces = np.sort(np.concatenate([tets[:, [0, 1, 2]], tets[:, [0, 1, 3]], tets[:, [0, 2, 3]],
                                                tets[:, [1, 2, 3]]]), axis=1)
                unique, counts = np.unique(faces, axis=0, return_counts=True)
                vertices = np.unique(unique[counts == 1])
        vertices = np.asarray(vertices.cpu().numpy() if isinstance(vertices, torch.Tensor) else vertices)
        if vertices.ndim != 1:
            raise ValueError("frictional vertices must be unique particle indices")
        nodes = np.ascontiguousarray(vertices, dtype=np.int32)
        return (BOUNDARY_KINDS[kind], np.ascontiguousarray(values, dtype=np.float64), nodes, float(friction),
                float(restitution), split, left, right)

    def frictional_state(self):
        """``(multipliers, omega, normals, candidates)`` of the last step as device tensors, or None."""
        if self._frictional_args is None:
            return None
        count = len(self._frictional_args[2])
        multiplier = torch.empty(count, dtype=torch.float64, device=self.device)
        omega = torch.empty_like(multiplier)
        normal = torch.empty((count, 3), dtype=torch.float64, device=self.device)
        candidate = torch.empty(count, dtype=torch.int32, device=self.device)
        _lib.check(self._lib.pd_frictional_state(self._handle, _lib.ptr(multiplier), _lib.ptr(omega), _lib.ptr(normal),
                                                 _lib.ptr(candidate), _stream()))
        return multiplier, omega, normal, candidate

    def _initialize_muscles(self, directions, stiffness):
        count = self._element_count
        self._has_muscles = False
        self._muscle_directions_host = None
        self._muscle_stiffness_host = None
        if directions is None and stiffness is None:
            return
        if directions is None or stiffness is None:
            raise ValueError("muscle_directions and muscle_stiffness must be supplied together")
        directions = np.array(directions, dtype=np.float64, copy=True)
        stiffness = np.array(stiffness, dtype=np.float64, copy=True)
        if stiffness.ndim == 0:
            stiffness = np.full(count, float(stiffness))
        if directions.shape != (count, 3) or stiffness.shape != (count,):
            raise ValueError(
                "Muscle directions must have shape (element_count,3), stiffness scalar or (element_count,)"
            )
        if not np.isfinite(directions).all() or not np.isfinite(stiffness).all() or np.any(stiffness < 0):
            raise ValueError("Muscle directions and stiffness must be finite, with nonnegative stiffness")
        lengths = np.linalg.norm(directions, axis=1)
        active = stiffness > 0
        if np.any(active & (lengths <= np.finfo(np.float64).eps)):
            raise ValueError("Active muscle directions must have nonzero length")
        directions[active] /= lengths[active, None]
        directions[~active] = 0.0
        self._has_muscles = bool(np.any(active))
        self._muscle_directions_host = np.ascontiguousarray(directions)
        self._muscle_stiffness_host = np.ascontiguousarray(stiffness)

    def _validate_planar(self, specification):
        indices, stiffness, plane = specification
        indices = np.asarray(indices)
        if (
            indices.ndim != 1
            or not np.issubdtype(indices.dtype, np.integer)
            or np.any(indices < 0)
            or np.any(indices >= self._n)
            or len(np.unique(indices)) != len(indices)
        ):
            raise ValueError("planar_energies needs distinct valid particle indices")
        stiffness = np.broadcast_to(np.asarray(stiffness, dtype=np.float64), indices.shape)
        plane = np.asarray(plane, dtype=np.float64)
        with np.errstate(over="ignore"):
            normal_length = np.linalg.norm(plane[:3]) if plane.shape == (4,) else 0.0
        if plane.shape != (4,) or not np.isfinite(plane).all() or not np.isfinite(normal_length) or normal_length <= 1.0e-5:
            raise ValueError("planar_energies needs a finite (nx,ny,nz,offset) with nonzero normal")
        if not np.isfinite(stiffness).all() or np.any(stiffness < 0):
            raise ValueError("planar_energies stiffness must be finite and nonnegative")
        return (
            np.ascontiguousarray(indices, dtype=np.int32),
            np.ascontiguousarray(stiffness, dtype=np.float64),
            np.ascontiguousarray(plane / normal_length, dtype=np.float64),
        )

    def _validate_model(self):
        model = self.model
        source = model.tet_materials if self._hex is None else self.hex_materials
        materials = source.detach().cpu().numpy().astype(np.float64)
        if not np.all(np.isfinite(materials)) or np.any(materials[:, 0] <= 0) or np.any(materials[:, 1] < 0):
            raise ValueError("DiffPhD requires positive shear modulus and nonnegative Lame lambda")
        if materials.shape[1] == 3 and np.any(materials[:, 2] != 0):
            raise ValueError("The reference DiffPhD solver has no damping; element damping must be zero")
        activations = getattr(model, "tet_activations", None)
        if not self._has_muscles and activations is not None and bool(torch.any(activations != 0)):
            raise ValueError("Tetrahedral activations require muscle_directions and muscle_stiffness")
        flags = model.particle_flags.cpu().numpy()
        if np.any((flags & 1) == 0):
            raise ValueError("SolverDiffPhD requires ACTIVE particles; pin particles with zero inverse mass")
        inverse_mass = model.particle_inv_mass.cpu().numpy()
        if not np.all(np.isfinite(inverse_mass)) or np.any(inverse_mass < 0):
            raise ValueError("Particle inverse masses must be finite and nonnegative")
        free = inverse_mass > 0
        if not np.any(free):
            raise ValueError("SolverDiffPhD needs at least one dynamic particle")
        if not np.array_equal(free, self._free_host):
            raise ValueError("the set of Dirichlet particles changed; create a new solver")
        return materials

    def _build(self, dt: float):
        materials = self._validate_model()
        self._materials_host = np.ascontiguousarray(materials[:, :2])
        _lib.check(self._lib.pd_set_materials(self._handle, _lib.ptr(self._materials_host)))
        _lib.check(self._lib.pd_set_tolerances(self._handle, self.max_iterations, self.abs_tol, self.rel_tol))
        _lib.check(self._lib.pd_build(self._handle, float(dt)))
        self._nh_mu = float(materials[:, 0].mean())
        self._nh_lame = float(materials[:, 1].mean())
        self._inertia = self.particle_mass / dt**2
        self._gravity = np.ascontiguousarray(
            self.model.gravity[self._gravity_world].detach().cpu().numpy().astype(np.float64)
        )
        self._factor_key = dt
        self._model_changed = False

    @property
    def mesh_contact_pairs(self) -> int | None:
        """Vertex-face pairs within the contact radius in the last step, or None (one host synchronization)."""
        if self._mesh_contact_args is None:
            return None
        pairs = ctypes.c_int32()
        _lib.check(self._lib.pd_mesh_contact_pairs(self._handle, ctypes.byref(pairs), _stream()))
        return pairs.value

    def mesh_contact_force(self, positions: torch.Tensor, velocities: torch.Tensor) -> torch.Tensor:
        """The mesh_contact force [N] of a float64 ``(N, 3)`` state (``MeshContact.evaluate``)."""
        if self._mesh_contact_args is None:
            raise RuntimeError("the solver has no mesh_contact")
        q = positions.detach().to(self.device, torch.float64).contiguous()
        v = velocities.detach().to(self.device, torch.float64).contiguous()
        force = torch.empty_like(q)
        _lib.check(self._lib.pd_mesh_contact_force(self._handle, _lib.ptr(q), _lib.ptr(v), _lib.ptr(force), None,
                                                   _stream()))
        return force

    def set_anderson_window(self, window: int) -> None:
        """Change the Anderson window (0..8) of the following steps and backward passes (added)."""
        if int(window) != window or not 0 <= window <= MAX_WINDOW:
            raise ValueError(f"anderson_window must be an integer in [0, {MAX_WINDOW}]")
        _lib.check(self._lib.pd_set_anderson_window(self._handle, int(window)))
        self.anderson_window = int(window)

    def set_tolerances(self, *, rel_tol: float | None = None, abs_tol: float | None = None,
                       max_iterations: int | None = None) -> None:
        """Change the stopping rule of later steps (and of batches created afterwards) without
        rebuilding the factor; arguments left as ``None`` keep their values."""
        rel = self.rel_tol if rel_tol is None else rel_tol
        absolute = self.abs_tol if abs_tol is None else abs_tol
        limit = self.max_iterations if max_iterations is None else max_iterations
        for name, value in (("abs_tol", absolute), ("rel_tol", rel)):
            if not np.isfinite(value) or value < 0:
                raise ValueError(f"{name} must be finite and nonnegative")
        if not np.isfinite(limit) or limit < 1 or int(limit) != limit:
            raise ValueError("max_iterations must be a positive integer")
        _lib.check(self._lib.pd_set_tolerances(self._handle, int(limit), float(absolute), float(rel)))
        self.rel_tol, self.abs_tol, self.max_iterations = float(rel), float(absolute), int(limit)

    def set_factor_device(self, enabled: bool = True) -> None:
        """Compute the rows of L^{-1} of later factor builds on the solver's device instead of the
        host threads (added); the factor is bit-identical either way."""
        _lib.check(self._lib.pd_set_factor_device(self._handle, 1 if enabled else 0))

    def notify_model_changed(self, flags: int = 0) -> None:
        """Rebuild the material weights and inverse factor before the next step."""
        if torch.cuda.is_current_stream_capturing():
            raise RuntimeError("notify_model_changed cannot run during graph capture")
        self._model_changed = True

    def factor_stats(self):
        """``(rows, nnz(S), nnz(L))`` of the current inverse factor."""
        rows, nnz_s, nnz_l = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
        _lib.check(self._lib.pd_factor_stats(self._handle, ctypes.byref(rows), ctypes.byref(nnz_s), ctypes.byref(nnz_l)))
        return rows.value, nnz_s.value, nnz_l.value

    # ------------------------------------------------------------------ status
    @property
    def iterations(self) -> np.ndarray:
        """Local/global iteration count of the last step (one host synchronization)."""
        forward, backward = ctypes.c_int32(), ctypes.c_int32()
        _lib.check(self._lib.pd_iterations(self._handle, ctypes.byref(forward), ctypes.byref(backward), _stream()))
        return np.array([forward.value], dtype=np.int32)

    @property
    def backward_iterations(self) -> int:
        forward, backward = ctypes.c_int32(), ctypes.c_int32()
        _lib.check(self._lib.pd_iterations(self._handle, ctypes.byref(forward), ctypes.byref(backward), _stream()))
        return int(backward.value)

    def read_status(self) -> int:
        """Read and clear the device status bits without raising; one host synchronization."""
        bits = ctypes.c_int32()
        _lib.check(self._lib.pd_read_status(self._handle, ctypes.byref(bits), _stream()))
        return int(bits.value)

    def check_status(self) -> None:
        """Read and clear the status bits, raising like the reference (``solver.py:392-417``)."""
        bits = self.read_status()
        if bits & _lib.STATUS_BARRIER_TIMEOUT:
            raise RuntimeError("a device barrier of the persistent step kernel gave up; the step result is invalid")
        if bits & _lib.STATUS_SINGULAR:
            raise ValueError("DiffPhD volume projection met a singular deformation gradient (reference 'Singular F.')")
        if bits & _lib.STATUS_ACTIVATION:
            if self._hex is not None:
                raise ValueError("Hex8 muscle target lengths must be finite and nonnegative")
            raise ValueError("Muscle activations must be finite and <= 1, and zero for disabled fibres")
        if bits & _lib.STATUS_NOT_CONVERGED:
            raise ConvergenceError(f"DiffPhD did not converge within {self.max_iterations} iterations")
        if bits & _lib.STATUS_ADJOINT_NOT_CONVERGED:
            raise ConvergenceError("A DiffPhD backward fixed point did not converge")
        if bits & _lib.STATUS_ADJOINT_SAFEGUARD:
            raise ConvergenceError("A reference DiffPhD backward safeguard modified the gradient")

    def deformation_determinants(self, state) -> torch.Tensor:
        """``det(F)`` at all eight Hex8 Gauss samples as ``(cells, 8)`` float64."""
        if self._hex is None:
            raise NotImplementedError("deformation_determinants currently requires hex_mesh")
        q = state.particle_q.detach()
        if q.device != self.device or tuple(q.shape) != (self._n, 3):
            raise ValueError("state must have this solver's particle count and device")
        result = torch.empty((self._element_count, 8), dtype=torch.float64, device=self.device)
        _lib.check(self._lib.pd_deformation_determinants(self._handle, _lib.ptr(q.contiguous()), _lib.ptr(result), _stream()))
        return result

    def apply_inverse(self, rhs: torch.Tensor) -> torch.Tensor:
        """``A^{-1} rhs`` through the uploaded factor, ``rhs`` float64 ``(N, 3)`` on the device."""
        if self._factor_key is None:
            raise RuntimeError("the factor is built by the first step")
        rhs = rhs.to(device=self.device, dtype=torch.float64).contiguous()
        out = torch.empty_like(rhs)
        _lib.check(self._lib.pd_apply_inverse(self._handle, _lib.ptr(rhs), _lib.ptr(out), _stream()))
        return out

    # ------------------------------------------------------------------ step
    def _activations(self, control):
        if not self._has_muscles:
            return None
        if self._hex is not None:
            if control is not None and control.tet_activations is not None and control.tet_activations.numel():
                raise ValueError("Hex8 uses solver.muscle_targets; tet_activations cannot control Hex8 fibres")
            return None
        source = self.model.tet_activations
        if control is not None and control.tet_activations is not None:
            source = control.tet_activations
        if source is None or tuple(source.shape) != (len(self._tets),) or source.dtype != torch.float32:
            raise ValueError("Muscle activations must be a float32 (tet_count,) array")
        self._activation_source = source
        return source.detach().contiguous()

    def _sync_hex_targets(self):
        if self._hex is None:
            return
        targets = self.muscle_targets.detach().cpu().numpy()
        if not np.array_equal(targets, self._targets_host):
            self._targets_host = targets.copy()
            _lib.check(self._lib.pd_set_muscle_targets(self._handle, _lib.ptr(np.ascontiguousarray(targets))))

    def step(self, state_in, state_out, control, contacts, dt: float, *, dirichlet_positions=None,
             record: torch.Tensor | None = None) -> None:
        """Advance one step of length ``dt`` [s] on the current CUDA stream.

        ``record`` (added): an optional float64 ``(N, 3)`` device tensor that
        receives the converged positions for :meth:`backward_step`.
        """
        if contacts is not None:
            raise NotImplementedError("SolverDiffPhD does not consume Newton contacts; pass contacts=None")
        if not np.isfinite(dt) or dt <= 0:
            raise ValueError("dt must be finite and positive")
        if state_in is state_out or state_in.particle_q.data_ptr() == state_out.particle_q.data_ptr():
            raise ValueError("DiffPhD requires distinct input and output states")
        if dirichlet_positions is not None:
            if not isinstance(dirichlet_positions, torch.Tensor):
                raise TypeError("dirichlet_positions must be a tensor")
            if dirichlet_positions.dtype != self.state_dtype or tuple(dirichlet_positions.shape) != (self._n, 3):
                raise ValueError("dirichlet_positions must have the state dtype and shape (particle_count, 3)")
            if dirichlet_positions.device != self.device:
                raise ValueError("dirichlet_positions must be on the solver device")
            if dirichlet_positions.data_ptr() in (state_out.particle_q.data_ptr(), state_out.particle_qd.data_ptr()):
                raise ValueError("dirichlet_positions must not alias an output state")
        tape = Tape.current()
        if tape is not None:
            if torch.cuda.is_current_stream_capturing():
                raise RuntimeError("Recording SolverDiffPhD steps on a Tape during graph capture is unsupported")
            self._check_aliasing(tape, state_in, state_out)
        dt = float(dt)
        if self._model_changed or self._factor_key != dt:
            if torch.cuda.is_current_stream_capturing():
                raise RuntimeError("SolverDiffPhD must rebuild its factor; step once outside graph capture first")
            self._build(dt)
        self._sync_hex_targets()
        activations = self._activations(control)
        _lib.check(self._lib.pd_set_activations(self._handle, _lib.ptr(activations)))
        gravity = self._gravity
        q = state_in.particle_q.detach()
        qd = state_in.particle_qd.detach()
        f = state_in.particle_f.detach()
        for name, tensor in (("particle_q", q), ("particle_qd", qd), ("particle_f", f),
                             ("particle_q out", state_out.particle_q), ("particle_qd out", state_out.particle_qd)):
            if tensor.dtype != self.state_dtype or tuple(tensor.shape) != (self._n, 3) or not tensor.is_contiguous():
                raise ValueError(f"state {name} must be a contiguous {self.state_dtype} (particle_count, 3) tensor")
        dirichlet = None if dirichlet_positions is None else dirichlet_positions.detach().contiguous()
        _lib.check(
            self._lib.pd_step(
                self._handle,
                _lib.ptr(q),
                _lib.ptr(qd),
                _lib.ptr(f),
                _lib.ptr(dirichlet),
                _lib.ptr(gravity),
                dt,
                _lib.ptr(state_out.particle_q.detach()),
                _lib.ptr(state_out.particle_qd.detach()),
                _lib.ptr(self._x if record is None else record),
                _stream(),
            )
        )
        self._last_record = self._x if record is None else record
        if tape is not None:
            self._record(tape, state_in, state_out, activations, dirichlet_positions, dt)

    def _check_aliasing(self, tape, state_in, state_out):
        seen = getattr(tape, "_diff_phd_state_buffers", None)
        if seen is None or self._recorded is not tape or not tape.records:
            seen = set()
        outputs = {state_out.particle_q.data_ptr(), state_out.particle_qd.data_ptr()}
        inputs = {state_in.particle_q.data_ptr(), state_in.particle_qd.data_ptr()}
        if outputs & (seen | inputs):
            raise ValueError("Recorded DiffPhD steps require distinct output states; ping-pong reuse aliases gradients")
        tape._diff_phd_state_buffers = seen | inputs | outputs
        self._recorded = tape

    def _record(self, tape, state_in, state_out, activations, dirichlet_positions, dt):
        x_record = self._last_record.clone()
        factor_key = self._factor_key
        materials = self.model.tet_materials if self._hex is None else self.hex_materials
        # The control's (or model's) tensor is the one whose gradient the user reads.
        activation_source = self._activation_source if activations is not None else None
        # StepRecord.contact (adjoint.py:834-841): the multipliers, omega and normals the step ended with.
        contact = None
        if self._frictional_args is not None and len(self._frictional_args[2]):
            multiplier, omega, normal, _candidate = self.frictional_state()
            contact = (multiplier, omega, normal)

        def backward():
            if self._factor_key != factor_key or self._model_changed:
                raise RuntimeError("the factor of a recorded step was rebuilt; record and replay with one build")
            self.backward_step(
                x_record,
                dt,
                state_in,
                state_out,
                activations=activations,
                activation_grad=_grad(activation_source) if activation_source is not None else None,
                materials=materials,
                dirichlet_positions=dirichlet_positions,
                contact=contact,
            )

        tape.record_func(backward, [state_in.particle_q, state_out.particle_q])

    def backward_step(self, x_record, dt, state_in, state_out, *, activations=None, activation_grad=None,
                      materials=None, dirichlet_positions=None, contact=None):
        """Backward pass of one recorded step (``adjoint.py:1088-1259``).

        Reads ``state_out`` gradients and accumulates into ``state_in`` gradients,
        ``materials.grad[:, :2]`` (float32, as the reference) and the activation
        and Dirichlet-target gradients when present. ``contact`` is the step's
        ``(multipliers, omega, normals)`` of the frictional boundary (float64
        device tensors); parameter gradients then use the contact projection.
        """
        gq_out = _grad(state_out.particle_q)
        gqd_out = _grad(state_out.particle_qd)
        gq = _grad(state_in.particle_q)
        gqd = _grad(state_in.particle_qd)
        gf = _grad(state_in.particle_f)
        gdirichlet = _grad(dirichlet_positions) if dirichlet_positions is not None else None
        material_grad = None
        direct = False
        if materials is not None and materials.grad is not None:
            grad = materials.grad
            direct = (grad.dtype == torch.float64 and tuple(grad.shape) == (self._element_count, 2)
                      and grad.is_contiguous())
            material_grad = grad if direct else torch.zeros((self._element_count, 2), dtype=torch.float64,
                                                            device=self.device)
        snapshot = (None, None, None) if contact is None else tuple(t.contiguous() for t in contact)
        _lib.check(
            self._lib.pd_backward_contact(
                self._handle,
                _lib.ptr(x_record),
                _lib.ptr(activations),
                float(dt),
                _lib.ptr(gq_out),
                _lib.ptr(gqd_out),
                _lib.ptr(gq),
                _lib.ptr(gqd),
                _lib.ptr(gf),
                _lib.ptr(gdirichlet),
                _lib.ptr(material_grad),
                _lib.ptr(activation_grad),
                *(_lib.ptr(t) for t in snapshot),
                _stream(),
            )
        )
        if material_grad is not None and not direct:
            materials.grad[:, :2] += material_grad.to(materials.grad.dtype)

    def __del__(self):
        handle = getattr(self, "_handle", None)
        if handle is not None and handle.value:
            try:
                self._lib.pd_destroy(handle)
            except Exception:
                pass
            self._handle = None


__all__ = ["SolverDiffPhD", "ConvergenceError", "Tape", "Mesh", "HexElements"]
