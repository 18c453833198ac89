"""ctypes binding of the C ABI declared in ``include/ando_gpu.h``.

This is the binding any non-pybind11 host would write against
``libando_gpu.so`` (it mirrors the header's structs field for field). The GPU
parity tests call the library through it, and it is the ctypes stub shown in
the integration notes.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path
from typing import Iterable, List, Optional, Sequence, Tuple

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "lib" / "libando_gpu.so"

ANDO_OK = 0
ANDO_ERR_CAPACITY = 6
SEMANTICS = {"reference": 0, "corrected": 1}
PRECOND = {"block_jacobi": 0, "learned": 1}

# Every symbol the header declares (checked by the CPU test suite).
EXPORTED = [
    "ando_abi_version", "ando_status_string", "ando_last_error", "ando_ctx_create", "ando_ctx_destroy",
    "ando_mesh_upload", "ando_mesh_set_vertices", "ando_state_upload", "ando_state_download",
    "ando_apply_gravity", "ando_step", "ando_compute_contacts", "ando_compute_contacts_corrected", "ando_last_system",
    "ando_eval_system",
    "ando_last_gradient", "ando_last_contact_blocks", "ando_profile_enable", "ando_profile_read", "ando_ctx_stream",
    "ando_broad_phase", "ando_pcg_solve_noalloc", "ando_ctx_keep_system",
    "ando_collision_metrics", "ando_state_moments", "ando_edge_triangle_crossings",
]

PHASES = ["setup", "strain", "gradient", "assemble", "pcg", "line_search", "finish", "precond"]


class Material(C.Structure):
    _fields_ = [(n, C.c_double) for n in ("youngs_modulus", "poisson_ratio", "density", "thickness", "bending_stiffness")]


class Params(C.Structure):
    _fields_ = [
        ("dt", C.c_double), ("beta_max", C.c_double),
        ("min_newton_steps", C.c_int32), ("max_newton_steps", C.c_int32), ("friction_min_newton_steps", C.c_int32),
        ("pcg_tol", C.c_double), ("pcg_max_iters", C.c_int32),
        ("contact_gap_max", C.c_double), ("wall_gap", C.c_double), ("enable_ccd", C.c_int32),
        ("contact_normal_epsilon", C.c_double), ("barrier_tolerance", C.c_double),
        ("enable_friction", C.c_int32), ("friction_mu", C.c_double), ("friction_epsilon", C.c_double),
        ("friction_tangent_threshold", C.c_double), ("velocity_damping", C.c_double), ("contact_restitution", C.c_double),
        ("enable_strain_limiting", C.c_int32), ("strain_limit", C.c_double), ("strain_tau", C.c_double),
        ("strain_epsilon", C.c_double), ("strain_svd_epsilon", C.c_double), ("hessian_epsilon", C.c_double),
        ("min_gap", C.c_double), ("semantics", C.c_int32), ("precond", C.c_int32), ("precond_refresh", C.c_int32),
        ("membrane_hessian", C.c_int32),
    ]


class Pin(C.Structure):
    _fields_ = [("vertex", C.c_int32), ("active", C.c_int32), ("target", C.c_double * 3)]


# numpy twin of Pin (same 32-byte layout), so pin sets are built without a Python loop
PIN_DTYPE = np.dtype([("vertex", "<i4"), ("active", "<i4"), ("target", "<f8", (3,))])
assert PIN_DTYPE.itemsize == C.sizeof(Pin)


def pin_array(pins) -> np.ndarray:
    """Pins as a PIN_DTYPE array; accepts (vertex, target) pairs or an existing array."""
    if isinstance(pins, np.ndarray) and pins.dtype == PIN_DTYPE:
        return np.ascontiguousarray(pins)
    pins = list(pins)
    a = np.zeros(len(pins), PIN_DTYPE)
    if pins:
        a["vertex"] = [int(i) for i, _ in pins]
        a["active"] = 1
        a["target"] = np.asarray([t for _, t in pins], dtype=np.float64).reshape(len(pins), 3)
    return a


class Wall(C.Structure):
    _fields_ = [("normal", C.c_double * 3), ("offset", C.c_double), ("gap", C.c_double), ("active", C.c_int32), ("pad_", C.c_int32)]


class Rigid(C.Structure):
    _fields_ = [
        ("num_vertices", C.c_int32), ("num_triangles", C.c_int32),
        ("local_vertices", C.POINTER(C.c_double)), ("triangles", C.POINTER(C.c_int32)),
        ("mass", C.c_double), ("inertia_body_inv", C.c_double * 9), ("position", C.c_double * 3),
        ("rotation", C.c_double * 9), ("linear_velocity", C.c_double * 3), ("angular_velocity", C.c_double * 3),
    ]


class Contact(C.Structure):
    _fields_ = [
        ("type", C.c_int32), ("idx0", C.c_int32), ("idx1", C.c_int32), ("idx2", C.c_int32), ("idx3", C.c_int32),
        ("rigid_body_index", C.c_int32), ("vertex_count", C.c_int32), ("pad_", C.c_int32),
        ("gap", C.c_double), ("normal", C.c_double * 3), ("witness_p", C.c_double * 3), ("witness_q", C.c_double * 3),
        ("barycentric", C.c_double * 3), ("weights", C.c_double * 4),
    ]


class Metrics(C.Structure):
    _fields_ = [(n, C.c_int32) for n in ("num_total_contacts", "num_point_triangle", "num_edge_edge", "num_wall",
                                          "num_penetrations", "num_major_penetrations", "num_tunneling",
                                          "num_ccd_contacts", "num_relative_velocities")] + \
               [(n, C.c_double) for n in ("min_gap", "max_gap", "sum_gap", "max_penetration", "sum_penetration",
                                          "max_relative_velocity", "sum_relative_velocity")]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class Moments(C.Structure):
    _fields_ = [("kinetic_energy", C.c_double), ("linear_momentum", C.c_double * 3),
                ("angular_momentum", C.c_double * 3), ("max_speed", C.c_double)]


class Profile(C.Structure):
    _fields_ = [("launches", C.c_int64), ("phase_launches", C.c_int64 * 8), ("phase_ms", C.c_double * 8),
                ("pcg_iterations", C.c_int64), ("newton_iterations", C.c_int64), ("pcg_learned_iterations", C.c_int64),
                ("pcg_extra_block_iterations", C.c_int64)]

    def as_dict(self) -> dict:
        return {"launches": self.launches, "pcg_iterations": self.pcg_iterations, "newton_iterations": self.newton_iterations,
                "pcg_learned_iterations": self.pcg_learned_iterations,
                "pcg_extra_block_iterations": self.pcg_extra_block_iterations,
                "phase_ms": {p: self.phase_ms[i] for i, p in enumerate(PHASES)},
                "phase_launches": {p: self.phase_launches[i] for i, p in enumerate(PHASES)}}


class StepStats(C.Structure):
    _fields_ = [
        ("newton_iters", C.c_int32), ("pcg_iters", C.c_int32), ("pcg_max_per_newton", C.c_int32),
        ("pcg_not_converged", C.c_int32), ("line_search_fail", C.c_int32), ("contacts", C.c_int32),
        ("strain_active", C.c_int32), ("status", C.c_int32), ("precond_fallbacks", C.c_int32), ("graph_launched", C.c_int32),
        ("beta", C.c_double), ("last_alpha", C.c_double), ("device_ms", C.c_double), ("substeps", C.c_int32), ("pad_", C.c_int32),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_ if name != "pad_"}


_lib: Optional[C.CDLL] = None


def lib() -> C.CDLL:
    """Load libando_gpu.so and declare the prototypes."""
    global _lib
    if _lib is not None:
        return _lib
    L = C.CDLL(str(LIB_PATH))
    P, I32, D = C.c_void_p, C.c_int32, C.c_double
    pd, pi, pf = C.POINTER(C.c_double), C.POINTER(C.c_int32), C.POINTER(C.c_float)
    L.ando_abi_version.restype = I32
    L.ando_status_string.restype = C.c_char_p; L.ando_status_string.argtypes = [I32]
    L.ando_last_error.restype = C.c_char_p
    L.ando_ctx_create.restype = I32; L.ando_ctx_create.argtypes = [I32, C.POINTER(P)]
    L.ando_ctx_destroy.restype = None; L.ando_ctx_destroy.argtypes = [P]
    L.ando_mesh_upload.restype = I32; L.ando_mesh_upload.argtypes = [P, pd, I32, pi, I32, pd, pd, C.POINTER(Material)]
    L.ando_mesh_set_vertices.restype = I32; L.ando_mesh_set_vertices.argtypes = [P, pd, I32]
    L.ando_state_upload.restype = I32; L.ando_state_upload.argtypes = [P, pd, pd, pd, pd, I32]
    L.ando_state_download.restype = I32; L.ando_state_download.argtypes = [P, pd, pd, I32]
    L.ando_apply_gravity.restype = I32; L.ando_apply_gravity.argtypes = [P, pd, D]
    L.ando_step.restype = I32
    L.ando_step.argtypes = [P, C.POINTER(Params), C.POINTER(Pin), I32, C.POINTER(Wall), I32, C.POINTER(Rigid), I32, C.POINTER(StepStats)]
    L.ando_step_batch.restype = I32; L.ando_step_batch.argtypes = [C.POINTER(BatchItem), I32, I32]
    L.ando_eval_system.restype = I32
    L.ando_eval_system.argtypes = [P, C.POINTER(Params), C.POINTER(Pin), I32, C.POINTER(Wall), I32, C.POINTER(Rigid), I32]
    L.ando_compute_contacts.restype = I32
    L.ando_compute_contacts.argtypes = [P, C.POINTER(Rigid), I32, C.POINTER(Contact), I32, pi]
    L.ando_compute_contacts_corrected.restype = I32
    L.ando_compute_contacts_corrected.argtypes = [P, C.c_double, C.POINTER(Rigid), I32, C.POINTER(Contact), I32, pi]
    L.ando_last_system.restype = I32; L.ando_last_system.argtypes = [P, pi, pi, pi, pi, pf, pf, pf]
    L.ando_last_gradient.restype = I32; L.ando_last_gradient.argtypes = [P, pd, I32]
    L.ando_last_contact_blocks.restype = I32; L.ando_last_contact_blocks.argtypes = [P, pi, pi, pi, pf]
    L.ando_profile_enable.restype = I32; L.ando_profile_enable.argtypes = [P, I32]
    L.ando_profile_read.restype = I32; L.ando_profile_read.argtypes = [P, C.POINTER(Profile)]
    L.ando_ctx_stream.restype = I32; L.ando_ctx_stream.argtypes = [P, C.POINTER(C.c_void_p)]
    L.ando_ctx_select_pcg_shape.restype = I32; L.ando_ctx_select_pcg_shape.argtypes = [P, I32, I32]
    L.ando_ctx_select_assembly_tpb.restype = I32; L.ando_ctx_select_assembly_tpb.argtypes = [P, I32]
    L.ando_ctx_assembly_tpb.restype = I32; L.ando_ctx_assembly_tpb.argtypes = [P, pi, pi]
    L.ando_ctx_set_pair_capacity.restype = I32; L.ando_ctx_set_pair_capacity.argtypes = [P, I32]
    L.ando_ctx_keep_system.restype = I32; L.ando_ctx_keep_system.argtypes = [P, I32]
    L.ando_ctx_set_refit_top_capacity.restype = I32; L.ando_ctx_set_refit_top_capacity.argtypes = [P, I32]
    L.ando_ctx_pcg_shape.restype = I32; L.ando_ctx_pcg_shape.argtypes = [P, I32, pi, pi, pd]
    L.ando_broad_phase.restype = I32; L.ando_broad_phase.argtypes = [P, I32, D, pi, I32, pi]
    pu8 = C.POINTER(C.c_ubyte)
    L.ando_precond_num_params.restype = I32
    L.ando_precond_init_weights.restype = I32; L.ando_precond_init_weights.argtypes = [C.c_uint64, pf, I32]
    L.ando_ctx_set_precond_weights.restype = I32; L.ando_ctx_set_precond_weights.argtypes = [P, pf, I32]
    L.ando_precond_eval.restype = I32; L.ando_precond_eval.argtypes = [P]
    L.ando_last_precond.restype = I32; L.ando_last_precond.argtypes = [P, pf]
    L.ando_last_scaled_system.restype = I32; L.ando_last_scaled_system.argtypes = [P, pf, pf, pf, pf, pd]
    L.ando_trainer_create.restype = I32; L.ando_trainer_create.argtypes = [I32, pf, I32, C.POINTER(P)]
    L.ando_trainer_destroy.restype = None; L.ando_trainer_destroy.argtypes = [P]
    L.ando_trainer_add_system.restype = I32; L.ando_trainer_add_system.argtypes = [P, P, I32, D, I32]
    L.ando_trainer_num_systems.restype = I32; L.ando_trainer_num_systems.argtypes = [P]
    L.ando_trainer_probes.restype = I32; L.ando_trainer_probes.argtypes = [P, I32, pf, pd, pi]
    L.ando_trainer_loss.restype = I32; L.ando_trainer_loss.argtypes = [P, I32, pd, pf]
    L.ando_trainer_step.restype = I32; L.ando_trainer_step.argtypes = [P, C.c_float, pd]
    L.ando_trainer_get_weights.restype = I32; L.ando_trainer_get_weights.argtypes = [P, pf, I32]
    L.ando_trainer_set_weights.restype = I32; L.ando_trainer_set_weights.argtypes = [P, pf, I32]
    L.ando_collision_metrics.restype = I32; L.ando_collision_metrics.argtypes = [P, D, I32, C.POINTER(Metrics)]
    L.ando_state_moments.restype = I32; L.ando_state_moments.argtypes = [P, C.POINTER(Moments)]
    L.ando_edge_triangle_crossings.restype = I32; L.ando_edge_triangle_crossings.argtypes = [P, C.POINTER(C.c_int64)]
    L.ando_pcg_solve_noalloc.restype = I32
    L.ando_pcg_solve_noalloc.argtypes = [I32, P, I32, P, P, P, P, P, P, C.c_int64, D, I32, pi, pi, pd]
    _lib = L
    return L


class AbiError(RuntimeError):
    pass


def _check(rc: int, what: str) -> None:
    if rc != ANDO_OK:
        L = lib()
        raise AbiError(f"{what}: {L.ando_status_string(rc).decode()} ({L.ando_last_error().decode()})")


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _iptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_int32))


def _fptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def rest_state(vertices: np.ndarray, triangles: np.ndarray) -> Tuple[np.ndarray, np.ndarray]:
    """Per-face rest area and Dm_inv (row-major 2x2) in the local 2D frame (mesh.cpp:18-75)."""
    v = np.asarray(vertices, dtype=np.float64)
    t = np.asarray(triangles, dtype=np.int64)
    e1 = v[t[:, 1]] - v[t[:, 0]]
    e2 = v[t[:, 2]] - v[t[:, 0]]
    l1 = (e1 * e1).sum(1)
    l2 = (e2 * e2).sum(1)
    n = np.cross(e1, e2)
    nl = np.linalg.norm(n, axis=1)
    ok = (l1 >= 1e-12) & (l2 >= 1e-12) & (nl >= 1e-12)
    area = np.where(ok, nl * 0.5, 0.0)
    with np.errstate(divide="ignore", invalid="ignore"):
        nu = n / nl[:, None]
        t1 = e1 / np.sqrt(l1)[:, None]
        t2 = np.cross(nu, t1)
        a = (e1 * t1).sum(1); b = (e2 * t1).sum(1); c = (e1 * t2).sum(1); d = (e2 * t2).sum(1)
        det = a * d - b * c
        inv = 1.0 / det
        dm = np.stack([d * inv, -b * inv, -c * inv, a * inv], axis=1)
    dm[~ok] = 0.0
    return np.ascontiguousarray(area), np.ascontiguousarray(dm)


def lumped_masses(num_vertices: int, triangles: np.ndarray, area: np.ndarray, thickness: float, density: float) -> np.ndarray:
    """m_i = sum over incident faces of area * thickness * density / 3 (state.cpp:18-32)."""
    m = np.zeros(num_vertices)
    fm = area * thickness * density / 3.0
    for k in range(3):
        np.add.at(m, triangles[:, k], fm)
    return m


def make_params(params: dict, semantics: str = "reference", precond: str = "block_jacobi", precond_refresh: int = 1) -> Params:
    """Params with the reference's SimParams defaults (types.h:60-100), overridden by `params`."""
    d = dict(dt=0.002, beta_max=0.25, min_newton_steps=2, max_newton_steps=8, friction_min_newton_steps=32,
             pcg_tol=1e-3, pcg_max_iters=1000, contact_gap_max=0.001, wall_gap=0.001, enable_ccd=1,
             contact_normal_epsilon=1e-8, barrier_tolerance=1e-12, enable_friction=0, friction_mu=0.1,
             friction_epsilon=1e-5, friction_tangent_threshold=1e-6, velocity_damping=0.0, contact_restitution=0.0,
             enable_strain_limiting=0, strain_limit=0.05, strain_tau=0.05, strain_epsilon=0.0, strain_svd_epsilon=1e-6,
             hessian_epsilon=1e-8, min_gap=1e-8, membrane_hessian=0)
    d.update({k: v for k, v in params.items()})
    p = Params()
    for name, typ in Params._fields_:
        if name in ("semantics", "precond", "precond_refresh"):
            continue
        val = d[name]
        setattr(p, name, int(val) if typ is C.c_int32 else float(val))
    p.semantics = SEMANTICS[semantics]
    p.precond = PRECOND[precond]
    p.precond_refresh = int(precond_refresh)
    return p


class Scene:
    """One device context holding a mesh and its state."""

    def __init__(self, vertices, triangles, material: dict, device: int = 0):
        L = lib()
        self.V = int(len(vertices))
        self.T = int(len(triangles))
        self.vertices = np.ascontiguousarray(vertices, dtype=np.float64)
        self.triangles = np.ascontiguousarray(triangles, dtype=np.int32)
        mat = dict(youngs_modulus=1e6, poisson_ratio=0.3, density=1000.0, thickness=0.001, bending_stiffness=0.0)
        mat.update(material)
        self.material = Material(**mat)
        self.area, self.dm_inv = rest_state(self.vertices, self.triangles)
        self.masses = lumped_masses(self.V, self.triangles, self.area, mat["thickness"], mat["density"])
        self.ctx = C.c_void_p()
        _check(L.ando_ctx_create(device, C.byref(self.ctx)), "ando_ctx_create")
        _check(L.ando_mesh_upload(self.ctx, _dptr(self.vertices), self.V, _iptr(self.triangles), self.T,
                                  _dptr(self.area), _dptr(self.dm_inv), C.byref(self.material)), "ando_mesh_upload")
        zeros = np.zeros((self.V, 3))
        self.upload(self.vertices, zeros, self.vertices, self.masses)

    def close(self):
        if self.ctx:
            lib().ando_ctx_destroy(self.ctx)
            self.ctx = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def upload(self, x=None, v=None, x_prev=None, masses=None):
        arrs = [None if a is None else np.ascontiguousarray(a, dtype=np.float64) for a in (x, v, x_prev, masses)]
        ptrs = [None if a is None else _dptr(a) for a in arrs]
        _check(lib().ando_state_upload(self.ctx, *ptrs, self.V), "ando_state_upload")

    def download(self) -> Tuple[np.ndarray, np.ndarray]:
        x = np.empty((self.V, 3)); v = np.empty((self.V, 3))
        _check(lib().ando_state_download(self.ctx, _dptr(x), _dptr(v), self.V), "ando_state_download")
        return x, v

    def apply_gravity(self, g, dt: float):
        ga = np.ascontiguousarray(g, dtype=np.float64)
        _check(lib().ando_apply_gravity(self.ctx, _dptr(ga), float(dt)), "ando_apply_gravity")

    @staticmethod
    def _constraints(pins, walls):
        pa = pin_array(pins)
        wa = (Wall * max(1, len(walls)))()
        for k, (n, off, gap) in enumerate(walls):
            n = np.asarray(n, dtype=np.float64)
            nn = np.linalg.norm(n)
            n = n / nn if nn > 0 else n
            for q in range(3):
                wa[k].normal[q] = float(n[q])
            wa[k].offset = float(off); wa[k].gap = float(gap); wa[k].active = 1
        return pa, wa

    def step(self, params: Params, pins: Sequence = (), walls: Sequence = (), rigids: Optional[List[Rigid]] = None) -> dict:
        pa, wa = self._constraints(pins, list(walls))
        st = StepStats()
        nr = len(rigids) if rigids else 0
        ra = (Rigid * max(1, nr))(*(rigids or []))
        _check(lib().ando_step(self.ctx, C.byref(params), pa.ctypes.data_as(C.POINTER(Pin)), len(pa), wa, len(walls), ra, nr,
                               C.byref(st)), "ando_step")
        if rigids:
            for k in range(nr):
                C.pointer(rigids[k])[0] = ra[k]
        return st.as_dict()

    def eval_system(self, params: Params, pins: Sequence = (), walls: Sequence = (), rigids: Optional[List[Rigid]] = None):
        pa, wa = self._constraints(pins, list(walls))
        nr = len(rigids) if rigids else 0
        ra = (Rigid * max(1, nr))(*(rigids or []))
        _check(lib().ando_eval_system(self.ctx, C.byref(params), pa.ctypes.data_as(C.POINTER(Pin)), len(pa), wa, len(walls), ra, nr),
               "ando_eval_system")

    def last_gradient(self) -> np.ndarray:
        g = np.empty(3 * self.V)
        _check(lib().ando_last_gradient(self.ctx, _dptr(g), self.V), "ando_last_gradient")
        return g

    def keep_system(self, keep: bool = True):
        """CORRECTED steps also keep the unscaled system for last_system (off by default)."""
        _check(lib().ando_ctx_keep_system(self.ctx, int(bool(keep))), "ando_ctx_keep_system")

    def system_size(self) -> Tuple[int, int]:
        """(block rows, static block slots) of the mesh's system."""
        V = C.c_int32(); nnzb = C.c_int32()
        _check(lib().ando_last_system(self.ctx, C.byref(V), C.byref(nnzb), None, None, None, None, None), "ando_last_system")
        return V.value, nnzb.value

    def last_system(self):
        V = C.c_int32(); nnzb = C.c_int32()
        _check(lib().ando_last_system(self.ctx, C.byref(V), C.byref(nnzb), None, None, None, None, None), "ando_last_system")
        rowptr = np.empty(V.value + 1, dtype=np.int32)
        cols = np.empty(nnzb.value, dtype=np.int32)
        vals = np.empty(9 * nnzb.value, dtype=np.float32)
        rhs = np.empty(3 * V.value, dtype=np.float32)
        sol = np.empty(3 * V.value, dtype=np.float32)
        _check(lib().ando_last_system(self.ctx, C.byref(V), C.byref(nnzb), _iptr(rowptr), _iptr(cols), _fptr(vals),
                                      _fptr(rhs), _fptr(sol)), "ando_last_system")
        return rowptr, cols, vals.reshape(-1, 3, 3), rhs, sol

    def last_contact_blocks(self):
        n = C.c_int32()
        _check(lib().ando_last_contact_blocks(self.ctx, C.byref(n), None, None, None), "ando_last_contact_blocks")
        rows = np.empty(n.value, dtype=np.int32); cols = np.empty(n.value, dtype=np.int32)
        vals = np.empty(9 * n.value, dtype=np.float32)
        if n.value:
            _check(lib().ando_last_contact_blocks(self.ctx, C.byref(n), _iptr(rows), _iptr(cols), _fptr(vals)),
                   "ando_last_contact_blocks")
        return rows, cols, vals.reshape(-1, 3, 3)

    def broad_phase(self, kind: int, pad: float = 0.0) -> np.ndarray:
        """Sorted candidate pairs, shape (n, 2): kind 0 (vertex, triangle), kind 1 (edge, edge)."""
        n = C.c_int32()
        rc = lib().ando_broad_phase(self.ctx, kind, float(pad), None, 0, C.byref(n))
        if rc not in (ANDO_OK, ANDO_ERR_CAPACITY):
            _check(rc, "ando_broad_phase")
        out = np.empty((max(n.value, 1), 2), dtype=np.int32)
        if n.value:
            _check(lib().ando_broad_phase(self.ctx, kind, float(pad), _iptr(out), n.value, C.byref(n)), "ando_broad_phase")
        return out[:n.value]

    def profile_enable(self, enable: bool = True):
        _check(lib().ando_profile_enable(self.ctx, 1 if enable else 0), "ando_profile_enable")

    def profile(self) -> dict:
        pr = Profile()
        _check(lib().ando_profile_read(self.ctx, C.byref(pr)), "ando_profile_read")
        return pr.as_dict()

    def stream(self) -> int:
        sp = C.c_void_p()
        _check(lib().ando_ctx_stream(self.ctx, C.byref(sp)), "ando_ctx_stream")
        return sp.value or 0

    def set_pair_capacity(self, pairs: int):
        """Start the broad-phase candidate buffers at `pairs` (they grow on demand)."""
        _check(lib().ando_ctx_set_pair_capacity(self.ctx, pairs), "ando_ctx_set_pair_capacity")

    def set_refit_top_capacity(self, nodes: int):
        """Top nodes the one-CTA refit finishes in shared memory (-1: 4096); more go through global counters."""
        _check(lib().ando_ctx_set_refit_top_capacity(self.ctx, nodes), "ando_ctx_set_refit_top_capacity")

    def select_assembly_tpb(self, index: int = -1):
        """Fix scaled-assembly block-size candidate `index` (-1: autotune on the next first assembly)."""
        _check(lib().ando_ctx_select_assembly_tpb(self.ctx, index), "ando_ctx_select_assembly_tpb")

    def assembly_tpb(self) -> dict:
        n = C.c_int32(); t = C.c_int32()
        _check(lib().ando_ctx_assembly_tpb(self.ctx, C.byref(n), C.byref(t)), "ando_ctx_assembly_tpb")
        return dict(candidates=n.value, tpb=t.value)

    def select_pcg_shape(self, learned: bool, index: int = -1):
        """Fix scaled-PCG launch candidate `index` (-1: autotune on the next first solve)."""
        _check(lib().ando_ctx_select_pcg_shape(self.ctx, 1 if learned else 0, index), "ando_ctx_select_pcg_shape")

    def pcg_shape(self, learned: bool) -> dict:
        n = C.c_int32(); sh = (C.c_int32 * 3)(); t = C.c_double()
        _check(lib().ando_ctx_pcg_shape(self.ctx, 1 if learned else 0, C.byref(n), sh, C.byref(t)), "ando_ctx_pcg_shape")
        return dict(candidates=n.value, tpb=sh[0], grid=sh[1], unroll=sh[2], tune_ms=t.value)

    def set_precond_weights(self, w: np.ndarray):
        w = np.ascontiguousarray(w, dtype=np.float32)
        _check(lib().ando_ctx_set_precond_weights(self.ctx, _fptr(w), len(w)), "ando_ctx_set_precond_weights")

    def precond_eval(self) -> np.ndarray:
        """S of the current scaled system under the loaded weights, (nnzb, 3, 3)."""
        _check(lib().ando_precond_eval(self.ctx), "ando_precond_eval")
        return self.last_precond()

    def last_precond(self) -> np.ndarray:
        V = C.c_int32(); nnzb = C.c_int32()
        _check(lib().ando_last_system(self.ctx, C.byref(V), C.byref(nnzb), None, None, None, None, None), "ando_last_system")
        S = np.empty(9 * nnzb.value, dtype=np.float32)
        _check(lib().ando_last_precond(self.ctx, _fptr(S)), "ando_last_precond")
        return S.reshape(-1, 3, 3)

    def last_scaled_system(self) -> dict:
        """Scaled system of the last CORRECTED Newton iteration (see ando_last_scaled_system)."""
        rowptr, cols, _, _, _ = self.last_system()
        xr, xc, _ = self.last_contact_blocks()
        valh = np.empty(9 * len(cols), dtype=np.float32)
        xvalh = np.empty(max(9 * len(xr), 9), dtype=np.float32)
        bhat = np.empty(3 * self.V, dtype=np.float32)
        Lf = np.empty(6 * self.V, dtype=np.float32)
        Linv = np.empty(6 * self.V)
        _check(lib().ando_last_scaled_system(self.ctx, _fptr(valh), _fptr(xvalh), _fptr(bhat), _fptr(Lf), _dptr(Linv)),
               "ando_last_scaled_system")
        return dict(rowptr=rowptr, cols=cols, valh=valh.reshape(-1, 3, 3), xrow=xr, xcol=xc,
                    xvalh=xvalh[:9 * len(xr)].reshape(-1, 3, 3), bhat=bhat, Lf=Lf.reshape(-1, 6), Linv=Linv.reshape(-1, 6))

    def collision_metrics(self, gap_max: float, ccd: bool = True) -> dict:
        """CollisionValidator sums over the context's current contact list, reduced on the device."""
        m = Metrics()
        _check(lib().ando_collision_metrics(self.ctx, float(gap_max), int(bool(ccd)), C.byref(m)), "ando_collision_metrics")
        return m.as_dict()

    def moments(self) -> dict:
        """Kinetic energy, linear / angular momentum and largest speed of the device state."""
        m = Moments()
        _check(lib().ando_state_moments(self.ctx, C.byref(m)), "ando_state_moments")
        return {"kinetic_energy": m.kinetic_energy, "linear_momentum": np.array(m.linear_momentum[:]),
                "angular_momentum": np.array(m.angular_momentum[:]), "max_speed": m.max_speed}

    def edge_triangle_crossings(self) -> int:
        """Mesh edges passing through a triangle they share no vertex with, at the current positions."""
        n = C.c_int64()
        _check(lib().ando_edge_triangle_crossings(self.ctx, C.byref(n)), "ando_edge_triangle_crossings")
        return int(n.value)

    def contacts(self, rigids: Optional[List[Rigid]] = None, semantics: str = "reference", gap_max: float = 1e-3) -> List[Contact]:
        """Contacts at the current state: the reference's query, or (semantics="corrected") the
        self and rigid contacts within gap_max that the CORRECTED step uses."""
        nr = len(rigids) if rigids else 0
        ra = (Rigid * max(1, nr))(*(rigids or []))
        if semantics == "corrected":
            name = "ando_compute_contacts_corrected"
            query = lambda b, cap, n: lib().ando_compute_contacts_corrected(self.ctx, float(gap_max), ra, nr, b, cap, n)
        else:
            name = "ando_compute_contacts"
            query = lambda b, cap, n: lib().ando_compute_contacts(self.ctx, ra, nr, b, cap, n)
        n = C.c_int32()
        buf = (Contact * 1)()
        rc = query(buf, 0, C.byref(n))
        if rc not in (ANDO_OK, ANDO_ERR_CAPACITY):
            _check(rc, name)
        if n.value == 0:
            return []
        buf = (Contact * n.value)()
        _check(query(buf, n.value, C.byref(n)), name)
        return list(buf)


def make_rigid(vertices, triangles, density: float, keep: list) -> Rigid:
    """Rigid body as RigidBody::initialize builds it (rigid_body.cpp:11-91); `keep` holds the arrays alive."""
    v = np.asarray(vertices, dtype=np.float64)
    c = v.mean(axis=0)
    local = np.ascontiguousarray(v - c)
    tris = np.ascontiguousarray(triangles, dtype=np.int32)
    ext = v.max(0) - v.min(0)
    vol = max(ext[0], 1e-6) * max(ext[1], 1e-6) * max(ext[2], 1e-6)
    mass = max(density * vol, 1e-3)
    I = np.array([(mass / 12.0) * (ext[1] ** 2 + ext[2] ** 2), (mass / 12.0) * (ext[0] ** 2 + ext[2] ** 2),
                  (mass / 12.0) * (ext[0] ** 2 + ext[1] ** 2)])
    I = np.maximum(I, 1e-6)
    keep.extend([local, tris])
    r = Rigid()
    r.num_vertices = len(local); r.num_triangles = len(tris)
    r.local_vertices = _dptr(local); r.triangles = _iptr(tris)
    r.mass = mass
    for k in range(9):
        r.inertia_body_inv[k] = 0.0
        r.rotation[k] = 1.0 if k in (0, 4, 8) else 0.0
    r.inertia_body_inv[0], r.inertia_body_inv[4], r.inertia_body_inv[8] = 1 / I[0], 1 / I[1], 1 / I[2]
    for q in range(3):
        r.position[q] = c[q]; r.linear_velocity[q] = 0.0; r.angular_velocity[q] = 0.0
    return r


def precond_num_params() -> int:
    return int(lib().ando_precond_num_params())


def precond_init_weights(seed: int = 0) -> np.ndarray:
    """Initial preconditioner weights (ando_precond_init_weights)."""
    w = np.empty(precond_num_params(), dtype=np.float32)
    _check(lib().ando_precond_init_weights(C.c_uint64(seed), _fptr(w), len(w)), "ando_precond_init_weights")
    return w


class BatchItem(C.Structure):
    _fields_ = [("ctx", C.c_void_p), ("params", C.POINTER(Params)), ("pins", C.POINTER(Pin)), ("num_pins", C.c_int32),
                ("walls", C.POINTER(Wall)), ("num_walls", C.c_int32), ("rigids", C.POINTER(Rigid)), ("num_rigids", C.c_int32),
                ("stats", C.POINTER(StepStats)), ("status", C.c_int32)]


def step_batch(scenes: Sequence["Scene"], params: Sequence[Params], pins: Sequence, walls: Sequence, threads: int = 0) -> List[dict]:
    """One ando_step_batch call: scene i steps with params[i], pins[i] ([(vertex, target)]) and walls[i]
    ([(normal, offset, gap)]); the scenes run concurrently. Returns each scene's step statistics."""
    n = len(scenes)
    items = (BatchItem * n)()
    keep = []
    stats = [StepStats() for _ in range(n)]
    for k, S in enumerate(scenes):
        pa, wa = Scene._constraints(pins[k], list(walls[k]))
        keep += [pa, wa]
        items[k].ctx = S.ctx
        items[k].params = C.pointer(params[k])
        items[k].pins = pa.ctypes.data_as(C.POINTER(Pin))
        items[k].num_pins = len(pa)
        items[k].walls = C.cast(wa, C.POINTER(Wall))
        items[k].num_walls = len(walls[k])
        items[k].num_rigids = 0
        items[k].stats = C.pointer(stats[k])
    _check(lib().ando_step_batch(items, n, threads), "ando_step_batch")
    return [st.as_dict() for st in stats]


class Trainer:
    """Device-side trainer of the learned preconditioner (ando_trainer_*)."""

    def __init__(self, weights: np.ndarray, device: int = 0):
        w = np.ascontiguousarray(weights, dtype=np.float32)
        self.t = C.c_void_p()
        _check(lib().ando_trainer_create(device, _fptr(w), len(w), C.byref(self.t)), "ando_trainer_create")

    def close(self):
        if self.t:
            lib().ando_trainer_destroy(self.t)
            self.t = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add_system(self, scene: "Scene", max_probes: int = 6, tol: float = 1e-6, max_iters: int = 2000):
        _check(lib().ando_trainer_add_system(self.t, scene.ctx, max_probes, tol, max_iters), "ando_trainer_add_system")

    def __len__(self) -> int:
        return int(lib().ando_trainer_num_systems(self.t))

    def probes(self, idx: int, V: int):
        n = C.c_int32()
        _check(lib().ando_trainer_probes(self.t, idx, None, None, C.byref(n)), "ando_trainer_probes")
        pr = np.empty(3 * V * n.value, dtype=np.float32)
        nr = np.empty(n.value)
        _check(lib().ando_trainer_probes(self.t, idx, _fptr(pr), _dptr(nr), C.byref(n)), "ando_trainer_probes")
        return pr.reshape(n.value, 3 * V), nr

    def loss(self, idx: int, grad: bool = False):
        L = C.c_double()
        g = np.empty(precond_num_params(), dtype=np.float32) if grad else None
        _check(lib().ando_trainer_loss(self.t, idx, C.byref(L), _fptr(g) if grad else None), "ando_trainer_loss")
        return (L.value, g) if grad else L.value

    def step(self, lr: float) -> float:
        L = C.c_double()
        _check(lib().ando_trainer_step(self.t, C.c_float(lr), C.byref(L)), "ando_trainer_step")
        return L.value

    def weights(self) -> np.ndarray:
        w = np.empty(precond_num_params(), dtype=np.float32)
        _check(lib().ando_trainer_get_weights(self.t, _fptr(w), len(w)), "ando_trainer_get_weights")
        return w

    def set_weights(self, w: np.ndarray):
        w = np.ascontiguousarray(w, dtype=np.float32)
        _check(lib().ando_trainer_set_weights(self.t, _fptr(w), len(w)), "ando_trainer_set_weights")
