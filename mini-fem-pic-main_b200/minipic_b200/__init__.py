"""ctypes binding of libminipic_cuda.so (include/minipic_cuda.h).

The library is the product; this module only marshals arrays.  It mirrors the
reference's host objects closely enough that a loop written like the
reference's ``main`` (src/mini-pic.cpp:124-167) reads the same:

    deck  = Deck.load(dir)                      # Parameters + LoadVolumeMesh/LoadSurfaceMesh
    ctx   = Context(deck.mesh)                  # DeviceData (mesh upload once)
    ctx.fe_setup(deck.fe(...))                  # FESolver ctor + preAssembly
    inj   = Injector(deck.mesh)                 # InjectIons' RNG and face data
    for ts in range(max_iter):
        ctx.append(*inj.sample(...), rewind=...)    # InjectIons
        ctx.push(q_over_m, dt, spwt)                # MoveParticles
        ctx.compute_phi(method)                     # FESolver::computePhi
        ctx.update_ef()                             # FESolver::updateEf

There is no CPU fallback: without the built library or without an sm_100
device the calls raise.
"""
from __future__ import annotations

import ctypes as C
import os
import re
from dataclasses import dataclass, field

import numpy as np

_PKG = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(_PKG, "lib", "libminipic_cuda.so")

# status codes and enums, include/minipic_cuda.h
MP_OK = 0
STATUS = {0: "MP_OK", 1: "MP_ERR_ARG", 2: "MP_ERR_OOM", 3: "MP_ERR_CUDA", 4: "MP_ERR_WALK_LIMIT",
          5: "MP_ERR_NOT_CONVERGED", 6: "MP_ERR_SINGULAR", 7: "MP_ERR_STATE", 8: "MP_ERR_NO_DEVICE",
          9: "MP_ERR_TIMEOUT", 10: "MP_ERR_LIMIT"}
NONLINEAR, GAUSS_SEIDEL, LAPACK, SPARSE_CG, SPARSE_NEWTON = 0, 1, 2, 3, 4
FE_DENSE, FE_SPARSE = 0, 1
FP64, MIXED = 0, 1
MIXED_AUTO, MIXED_TF32, MIXED_FP16, MIXED_TF32X3 = 0, 1, 2, 3
MIXED_FP16_FROM = 16384  # MIXED_AUTO: FP16 operands from this many unknowns (the header's MP_MIXED_FP16_FROM)
WALK_LIMIT_ERROR, WALK_LIMIT_ABSORB = 0, 1
SCATTER_ATOMIC, SCATTER_FIXED = 0, 1
ORDER_STORAGE, ORDER_ID = 0, 1
VEC = {"F0": 0, "F1": 1, "d": 2, "g": 3, "uh": 4, "den": 5, "ef": 6, "G": 7, "y": 8, "K": 16, "J": 17}
NODE_NORMAL, NODE_OPEN, NODE_INLET, NODE_FIXED = 0, 1, 2, 3

# reference constants, src/FESolver.h:18-21
EPS0 = 8.8541878e-12
QE = 1.602e-19
AMU = 1.660538921e-27
KB = 8.617333262e-5

EXPORTED = [
    "mp_error_string", "mp_last_error", "mp_version", "mp_create", "mp_destroy", "mp_synchronize",
    "mp_get_stream", "mp_set_walk_limit", "mp_set_scatter_mode", "mp_set_sort_period",
    "mp_set_particle_form", "mp_particles_reserve", "mp_particles_append", "mp_particles_append_device",
    "mp_particles_count", "mp_particles_download", "mp_particles_clear", "mp_push_scatter",
    "mp_density_download", "mp_sort_by_tet", "mp_fe_setup", "mp_fe_upload", "mp_fe_download",
    "mp_compute_phi", "mp_fe_build_f1", "mp_fe_residual", "mp_fe_build_j", "mp_fe_solve_linear",
    "mp_update_ef", "mp_field_download", "mp_mesh_geometry", "mp_fe_geometry", "mp_inlet_faces",
    "mp_injector_create", "mp_injector_destroy", "mp_injector_sample", "mp_injector_count",
    "mp_injector_get_rem", "mp_injector_set_rem", "mp_set_track_ids", "mp_kernel_launches",
    "mp_device_buffer", "mp_push_particles_noalloc", "mp_set_mixed_factor",
    "mp_adjoint_setup", "mp_adjoint_add_particles", "mp_adjoint_forward", "mp_adjoint_flux",
    "mp_adjoint_backward", "mp_adjoint_tangent", "mp_set_walk_policy", "mp_inject_device",
    "mp_set_fe_storage", "mp_set_sparse_solver", "mp_fe_sparse_matrix",
    "mp_mesh_geometry_device", "mp_inlet_faces_device", "mp_fe_geometry_device",
    "mp_output_mesh", "mp_output_particles", "mp_output_wait", "mp_set_gs_max_sweeps",
    "mp_set_kernel_timing", "mp_kernel_timing",
]
KT_PUSH, KT_UPDATE, KT_DIAG, KT_PANEL, KT_TRSV = 0, 1, 2, 3, 4
# the classes a timed run brackets with events: few launches a step each
KT_TIMED = (1 << KT_PUSH) | (1 << KT_UPDATE) | (1 << KT_TRSV)


class MpError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS.get(status, status)}: {msg}")
        self.status = status


class MeshDesc(C.Structure):
    _fields_ = [
        ("n_nodes", C.c_int32), ("n_tets", C.c_int32),
        ("con", C.c_void_p), ("con_stride", C.c_int64),
        ("volume", C.c_void_p), ("volume_stride", C.c_int64),
        ("alpha", C.c_void_p), ("alpha_stride", C.c_int64),
        ("beta", C.c_void_p), ("beta_stride", C.c_int64),
        ("gamma", C.c_void_p), ("gamma_stride", C.c_int64),
        ("delta", C.c_void_p), ("delta_stride", C.c_int64),
        ("cell_con", C.c_void_p), ("cell_con_stride", C.c_int64),
        ("node_pos", C.c_void_p), ("node_pos_stride", C.c_int64),
        ("node_volume", C.c_void_p), ("node_volume_stride", C.c_int64),
    ]


class FeDesc(C.Structure):
    _fields_ = [
        ("neq", C.c_int32), ("ID", C.c_void_p), ("nx", C.c_void_p), ("detJ", C.c_void_p),
        ("g", C.c_void_p), ("K_rows", C.c_void_p), ("K_dense", C.c_void_p), ("F0", C.c_void_p),
        ("n0", C.c_double), ("phi0", C.c_double), ("kTe", C.c_double),
    ]


class StepStats(C.Structure):
    _fields_ = [("n_before", C.c_int64), ("n_after", C.c_int64), ("total_hops", C.c_int64),
                ("max_hops", C.c_int32), ("near_face_fp64", C.c_int32), ("ms_kernel", C.c_double),
                ("ms_step", C.c_double), ("lost", C.c_int64)]


class NewtonStats(C.Structure):
    _fields_ = [("newton_iterations", C.c_int32), ("linear_iterations", C.c_int32), ("l2", C.c_double),
                ("linear_residual", C.c_double), ("ms_total", C.c_double), ("ms_factor", C.c_double),
                ("linear_failures", C.c_int32), ("reserved", C.c_int32)]


class AdjointStats(C.Structure):
    _fields_ = [("slots", C.c_int64), ("alive", C.c_int64), ("wall_exits", C.c_int64),
                ("other_exits", C.c_int64), ("flux", C.c_double), ("ms", C.c_float)]


_lib = None


def lib():
    """Loads the built library; raises if it is missing (no fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is not built; run minipic_b200.build.build()")
        L = C.CDLL(LIB_PATH)
        vp, i32, i64, d = C.c_void_p, C.c_int32, C.c_int64, C.c_double
        L.mp_error_string.restype = C.c_char_p
        L.mp_error_string.argtypes = [C.c_int]
        L.mp_last_error.restype = C.c_char_p
        L.mp_last_error.argtypes = [vp]
        for name in EXPORTED:
            f = getattr(L, name)
            if name not in ("mp_error_string", "mp_last_error"):
                f.restype = C.c_int
        L.mp_create.argtypes = [C.c_int, C.POINTER(MeshDesc), C.POINTER(vp)]
        L.mp_particles_append.argtypes = [vp, i64, vp, i64, vp, i64, vp, i64, C.c_int, d, d]
        L.mp_particles_append_device.argtypes = [vp, i64, vp, vp, vp, C.c_int, d, d]
        L.mp_particles_download.argtypes = [vp, i64, vp, i64, vp, i64, vp, i64, vp, i64, vp, C.c_int]
        L.mp_push_scatter.argtypes = [vp, d, d, d, vp, C.POINTER(StepStats)]
        L.mp_compute_phi.argtypes = [vp, vp, C.c_int, C.c_int, C.POINTER(NewtonStats)]
        L.mp_fe_solve_linear.argtypes = [vp, C.c_int, C.c_int, vp, C.POINTER(NewtonStats)]
        L.mp_fe_setup.argtypes = [vp, C.POINTER(FeDesc)]
        L.mp_mesh_geometry.argtypes = [i32, vp, i32, vp] + [vp] * 8
        L.mp_mesh_geometry_device.argtypes = [C.c_int, i32, vp, i32, vp] + [vp] * 8
        L.mp_inlet_faces_device.argtypes = [C.c_int, i32, vp, i32, vp, i32, vp, C.c_int, vp, vp, vp, vp, vp]
        L.mp_fe_geometry_device.argtypes = [C.c_int, i32, vp, vp, i32, vp, vp, vp, vp, vp]
        L.mp_fe_geometry.argtypes = [i32, vp, vp, i32, vp, vp, vp, vp, vp]
        L.mp_inlet_faces.argtypes = [i32, vp, i32, vp, i32, vp, C.c_int, vp, vp, vp, vp, vp]
        L.mp_injector_create.argtypes = [i32, vp, vp, vp, vp, vp, vp, vp, C.c_uint32, C.POINTER(vp)]
        L.mp_injector_sample.argtypes = [vp, d, d, d, d, i64, vp, i64, vp, i64, vp, i64, C.POINTER(i64)]
        L.mp_injector_count.argtypes = [vp, d, d, d, d, C.POINTER(i64)]
        L.mp_injector_get_rem.argtypes = [vp, C.POINTER(d)]
        L.mp_injector_set_rem.argtypes = [vp, d]
        for name in ("mp_destroy", "mp_synchronize", "mp_particles_clear", "mp_sort_by_tet", "mp_fe_residual",
                     "mp_injector_destroy"):
            getattr(L, name).argtypes = [vp]
        L.mp_get_stream.argtypes = [vp, C.POINTER(vp)]
        L.mp_set_walk_limit.argtypes = [vp, i32]
        L.mp_set_scatter_mode.argtypes = [vp, C.c_int]
        L.mp_set_sort_period.argtypes = [vp, i32]
        L.mp_set_mixed_factor.argtypes = [vp, C.c_int]
        L.mp_set_walk_policy.argtypes = [vp, C.c_int]
        L.mp_set_fe_storage.argtypes = [vp, C.c_int]
        L.mp_output_mesh.argtypes = [vp, i32, C.c_char_p, vp, i64]
        L.mp_output_particles.argtypes = [vp, C.c_char_p]
        L.mp_output_wait.argtypes = [vp]
        L.mp_set_sparse_solver.argtypes = [vp, d, i32]
        L.mp_fe_sparse_matrix.argtypes = [vp, C.POINTER(i64), vp, vp, vp]
        L.mp_inject_device.argtypes = [vp, vp, d, d, d, d, d, d, C.c_uint64, C.c_uint64, C.POINTER(i64)]
        L.mp_adjoint_setup.argtypes = [vp, i32, i32, d, d, d, d, vp, vp, vp, C.c_int]
        L.mp_adjoint_add_particles.argtypes = [vp, i32, C.c_int, i64, vp, vp, vp]
        L.mp_adjoint_forward.argtypes = [vp, vp, d, C.c_int, vp, C.POINTER(AdjointStats)]
        L.mp_adjoint_flux.argtypes = [vp, C.POINTER(d)]
        L.mp_adjoint_backward.argtypes = [vp, vp, d, vp, C.POINTER(d)]
        L.mp_adjoint_tangent.argtypes = [vp, vp, d, vp, C.POINTER(d)]
        L.mp_set_particle_form.argtypes = [vp, C.c_int]
        L.mp_set_track_ids.argtypes = [vp, C.c_int]
        L.mp_kernel_launches.argtypes = [vp, C.POINTER(i64)]
        L.mp_set_kernel_timing.argtypes = [vp, C.c_int]
        L.mp_kernel_timing.argtypes = [vp, C.c_int, C.POINTER(i64), C.POINTER(d), C.POINTER(d)]
        L.mp_set_gs_max_sweeps.argtypes = [vp, C.c_int32]
        L.mp_device_buffer.argtypes = [vp, C.c_int, C.POINTER(vp), C.POINTER(i64)]
        L.mp_push_particles_noalloc.argtypes = [vp, vp, i64, vp, i32, vp, vp, i32, d, d, vp, C.POINTER(i64)]
        L.mp_particles_reserve.argtypes = [vp, i64]
        L.mp_particles_count.argtypes = [vp, C.POINTER(i64)]
        L.mp_density_download.argtypes = [vp, vp]
        L.mp_fe_upload.argtypes = [vp, C.c_int, vp]
        L.mp_fe_download.argtypes = [vp, C.c_int, vp]
        L.mp_fe_build_f1.argtypes = [vp, vp]
        L.mp_fe_build_j.argtypes = [vp, C.c_int]
        L.mp_update_ef.argtypes = [vp, vp]
        L.mp_field_download.argtypes = [vp, vp, vp, vp]
        _lib = L
    return _lib


def _p(a):
    if a is None:
        return None
    assert isinstance(a, np.ndarray) and a.flags.c_contiguous, "arrays must be C-contiguous"
    return a.ctypes.data_as(C.c_void_p)


def _check(rc: int, ctx_handle=None) -> None:
    if rc != MP_OK:
        L = lib()
        msg = L.mp_last_error(ctx_handle).decode() if ctx_handle else ""
        raise MpError(rc, msg or L.mp_error_string(rc).decode())


# ---------------------------------------------------------------------------
# deck: Parameters + meshes (host setup, no device)
# ---------------------------------------------------------------------------

@dataclass
class Parameters:
    """The reference's Parameters (src/parameters.h:20-39, parameters.cpp:18-86)."""
    plasma_den: float = 1e20
    ion_velocity: float = 7000.0
    electron_temperature: float = 24000.0
    max_iter: int = 250
    wall_potential: float = 100.0
    dt: float = 1e-7
    mesh_files: dict = field(default_factory=dict)
    invert_normals: bool = False
    plasma_species: str = "Deuterium"
    fesolver_method: int = NONLINEAR

    @classmethod
    def read(cls, path: str) -> "Parameters":
        p = cls()
        with open(path) as f:
            for line in f:
                line = line.rstrip("\n").rstrip("\r")
                line = re.sub(r"\s*(#.*)?$", "", line)
                if not line:
                    continue
                m = re.fullmatch(r"(\w+)\s*=\s*(.*)", line)
                if not m:
                    continue
                key, value = m.group(1), m.group(2)
                if key in ("plasma_den", "ion_velocity", "electron_temperature", "wall_potential", "dt"):
                    setattr(p, key, float(value))
                elif key == "max_iter":
                    p.max_iter = int(value)
                elif key in ("global_mesh", "inlet_mesh", "wall_mesh"):
                    p.mesh_files.setdefault(key, value)
                elif key == "invert_normals":
                    if re.fullmatch(r"t(rue)?", value, re.I) or value == "1":
                        p.invert_normals = True
                    elif re.fullmatch(r"f(alse)?", value, re.I) or value == "0":
                        p.invert_normals = False
                elif key == "plasma_species":
                    if re.fullmatch(r"D(uterium)?", value):
                        p.plasma_species = "Deuterium"
                    elif re.fullmatch(r"O(xygen)?", value):
                        p.plasma_species = "Oxygen"
                    else:
                        raise ValueError(f"Invalid plasma species: '{value}'")
                elif key == "fesolver_method":
                    methods = {"nonlinear": NONLINEAR, "gaussseidel": GAUSS_SEIDEL, "lapack": LAPACK}
                    if value.lower() not in methods:
                        raise ValueError(f"Invalid fesolver_method: '{value}'")
                    p.fesolver_method = methods[value.lower()]
                else:
                    raise ValueError(f"Unrecognised parameter: '{key}'")
        return p


def read_volume_dat(path: str):
    """Salome volume file, the way LoadVolumeMesh reads it (meshes.cpp:28-73):
    node coordinates divided by 1000, type-304 tets, other elements skipped."""
    with open(path) as f:
        n_nodes, n_elements = (int(t) for t in f.readline().split()[:2])
        pos = np.zeros((n_nodes, 3))
        for n in range(n_nodes):
            t = f.readline().split()
            pos[n] = (float(t[1]) / 1000.0, float(t[2]) / 1000.0, float(t[3]) / 1000.0)
        tets = []
        for _ in range(n_elements):
            t = f.readline().split()
            if len(t) >= 6 and t[1] == "304":
                tets.append((int(t[2]) - 1, int(t[3]) - 1, int(t[4]) - 1, int(t[5]) - 1))
    return pos, np.array(tets, dtype=np.int32).reshape(-1, 4)


def read_surface_dat(path: str):
    """Surface file (meshes.cpp:268-303): listed node ids (0-based) and type-203 triangles."""
    with open(path) as f:
        n_nodes, n_elements = (int(t) for t in f.readline().split()[:2])
        nodes = np.zeros(n_nodes, dtype=np.int64)
        for n in range(n_nodes):
            nodes[n] = int(f.readline().split()[0]) - 1
        tris = []
        for _ in range(n_elements):
            t = f.readline().split()
            if len(t) >= 5 and t[1] == "203":
                tris.append((int(t[2]) - 1, int(t[3]) - 1, int(t[4]) - 1))
    return nodes, np.array(tris, dtype=np.int32).reshape(-1, 3)


@dataclass
class Mesh:
    """Volume + inlet faces with the geometry the kernels consume (the
    reference's Volume, src/meshes.h:57-64)."""
    node_pos: np.ndarray
    node_type: np.ndarray
    node_volume: np.ndarray
    con: np.ndarray
    volume: np.ndarray
    alpha: np.ndarray
    beta: np.ndarray
    gamma: np.ndarray
    delta: np.ndarray
    cell_con: np.ndarray
    inlet_con: np.ndarray
    inlet_cell: np.ndarray
    inlet_u: np.ndarray
    inlet_v: np.ndarray
    inlet_normal: np.ndarray
    inlet_area: np.ndarray

    @property
    def n_nodes(self):
        return int(self.node_pos.shape[0])

    @property
    def n_tets(self):
        return int(self.con.shape[0])

    @classmethod
    def build(cls, node_pos: np.ndarray, tets: np.ndarray, inlet_nodes, inlet_tris, fixed_nodes,
              invert_normals: bool = False, device: int | None = None) -> "Mesh":
        """LoadVolumeMesh + LoadSurfaceMesh's geometry, on the host helpers or,
        with `device`, on that GPU (the same arrays bit for bit)."""
        L = lib()
        node_pos = np.ascontiguousarray(node_pos, dtype=np.float64)
        con = np.ascontiguousarray(tets, dtype=np.int32).copy()
        nn, nt = node_pos.shape[0], con.shape[0]
        vol = np.zeros(nt)
        al, be, ga, de = (np.zeros((nt, 4)) for _ in range(4))
        cc = np.zeros((nt, 4), dtype=np.int32)
        nvol = np.zeros(nn)
        nopen = np.zeros(nn, dtype=np.int32)
        if device is None:
            _check(L.mp_mesh_geometry(nn, _p(node_pos), nt, _p(con), _p(vol), _p(al), _p(be), _p(ga), _p(de),
                                      _p(cc), _p(nvol), _p(nopen)))
        else:
            _check(L.mp_mesh_geometry_device(device, nn, _p(node_pos), nt, _p(con), _p(vol), _p(al), _p(be),
                                             _p(ga), _p(de), _p(cc), _p(nvol), _p(nopen)))
        ntype = np.where(nopen == 1, NODE_OPEN, NODE_NORMAL).astype(np.int32)
        ntype[np.asarray(inlet_nodes, dtype=np.int64)] = NODE_INLET
        ntype[np.asarray(fixed_nodes, dtype=np.int64)] = NODE_FIXED
        tris = np.ascontiguousarray(inlet_tris, dtype=np.int32)
        nf = tris.shape[0]
        fcell = np.zeros(nf, dtype=np.int32)
        u, v, nrm = np.zeros((nf, 3)), np.zeros((nf, 3)), np.zeros((nf, 3))
        area = np.zeros(nf)
        if device is None:
            _check(L.mp_inlet_faces(nn, _p(node_pos), nt, _p(con), nf, _p(tris), int(invert_normals), _p(fcell),
                                    _p(u), _p(v), _p(nrm), _p(area)))
        else:
            _check(L.mp_inlet_faces_device(device, nn, _p(node_pos), nt, _p(con), nf, _p(tris), int(invert_normals),
                                           _p(fcell), _p(u), _p(v), _p(nrm), _p(area)))
        return cls(node_pos, ntype, nvol, con, vol, al, be, ga, de, cc, tris, fcell, u, v, nrm, area)

    def desc(self) -> MeshDesc:
        d = MeshDesc()
        d.n_nodes, d.n_tets = self.n_nodes, self.n_tets
        d.con, d.con_stride = _p(self.con).value, 16
        d.volume, d.volume_stride = _p(self.volume).value, 8
        d.alpha, d.alpha_stride = _p(self.alpha).value, 32
        d.beta, d.beta_stride = _p(self.beta).value, 32
        d.gamma, d.gamma_stride = _p(self.gamma).value, 32
        d.delta, d.delta_stride = _p(self.delta).value, 32
        d.cell_con, d.cell_con_stride = _p(self.cell_con).value, 16
        d.node_pos, d.node_pos_stride = _p(self.node_pos).value, 24
        d.node_volume, d.node_volume_stride = _p(self.node_volume).value, 8
        return d

    def fe_geometry(self, device: int | None = None):
        """ID, NX, detJ, neq as FESolver's constructor computes them (on the
        host, or on GPU `device`)."""
        L = lib()
        ID = np.zeros(self.n_nodes, dtype=np.int32)
        nx = np.zeros((self.n_tets, 4, 3))
        detJ = np.zeros(self.n_tets)
        neq = C.c_int32(0)
        args = (self.n_nodes, _p(self.node_pos), _p(self.node_type), self.n_tets, _p(self.con), _p(ID), _p(nx),
                _p(detJ), C.byref(neq))
        _check(L.mp_fe_geometry(*args) if device is None else L.mp_fe_geometry_device(device, *args))
        return ID, nx, detJ, int(neq.value)


@dataclass
class Deck:
    params: Parameters
    mesh: Mesh
    sphere_nodes: np.ndarray

    @classmethod
    def load(cls, directory: str, device: int | None = None) -> "Deck":
        params = Parameters.read(os.path.join(directory, "system.param"))
        mf = {k: os.path.join(directory, v) for k, v in params.mesh_files.items()}
        pos, tets = read_volume_dat(mf["global_mesh"])
        inlet_nodes, inlet_tris = read_surface_dat(mf["inlet_mesh"])
        wall_nodes, _ = read_surface_dat(mf["wall_mesh"])
        sphere_nodes = np.zeros(0, dtype=np.int64)
        sp = os.path.join(directory, "sphere.dat")
        if os.path.exists(sp):
            sphere_nodes, _ = read_surface_dat(sp)
        fixed = np.concatenate([wall_nodes, sphere_nodes])
        mesh = Mesh.build(pos, tets, inlet_nodes, inlet_tris, fixed, params.invert_normals, device=device)
        return cls(params, mesh, sphere_nodes)

    def dirichlet(self, sphere_potential: float | None = None) -> np.ndarray:
        """g per src/mini-pic.cpp:98-102 (INLET 0, FIXED -wall_potential), with the
        sphere's nodes at their own potential when given."""
        g = np.zeros(self.mesh.n_nodes)
        g[self.mesh.node_type == NODE_FIXED] = -self.params.wall_potential
        if sphere_potential is not None and self.sphere_nodes.size:
            g[self.sphere_nodes] = sphere_potential
        return g

    def fe_desc_arrays(self, sphere_potential: float | None = None, phi0: float = 0.0):
        ID, nx, detJ, neq = self.mesh.fe_geometry()
        g = self.dirichlet(sphere_potential)
        return dict(ID=ID, nx=np.ascontiguousarray(nx), detJ=detJ, g=g, neq=neq,
                    n0=self.params.plasma_den, phi0=phi0, kTe=KB * self.params.electron_temperature)


# ---------------------------------------------------------------------------
# device context
# ---------------------------------------------------------------------------

class Context:
    """One device context (the reference's DeviceData plus FESolver's state)."""

    def __init__(self, mesh: Mesh, device: int = 0):
        L = lib()
        self._keep = mesh
        h = C.c_void_p()
        desc = mesh.desc()
        _check(L.mp_create(device, C.byref(desc), C.byref(h)))
        self.h = h
        self.mesh = mesh
        self.neq = 0

    def close(self):
        if getattr(self, "h", None):
            lib().mp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _c(self, rc):
        _check(rc, self.h)

    # options
    def set_walk_limit(self, n):
        self._c(lib().mp_set_walk_limit(self.h, n))

    def inject_device(self, injector, plasma_den, ion_velocity, dt, spwt, thermal_sigma, q_over_m, seed, step):
        """InjectIons on the device (Philox sampling, the reference's counts); returns the count."""
        n = C.c_int64(0)
        self._c(lib().mp_inject_device(self.h, injector.h, plasma_den, ion_velocity, dt, spwt, thermal_sigma,
                                       q_over_m, seed, step, C.byref(n)))
        return n.value

    def set_walk_policy(self, policy):
        """WALK_LIMIT_ERROR (default) or WALK_LIMIT_ABSORB: what a walk that reaches the hop limit does."""
        self._c(lib().mp_set_walk_policy(self.h, policy))

    def set_scatter_mode(self, mode):
        self._c(lib().mp_set_scatter_mode(self.h, mode))

    def set_mixed_factor(self, mode):
        """MIXED_AUTO (default), MIXED_TF32, MIXED_FP16 or MIXED_TF32X3: tensor-core arithmetic
        of the mixed-form factorization (AUTO: TF32X3 below 16,384 unknowns, FP16 from there;
        FP16: the trailing updates on scaled FP16 copies of their operands)."""
        self._c(lib().mp_set_mixed_factor(self.h, mode))

    def set_sort_period(self, steps):
        self._c(lib().mp_set_sort_period(self.h, steps))

    def set_track_ids(self, on: bool):
        self._c(lib().mp_set_track_ids(self.h, int(bool(on))))

    def device_buffer(self, name: str):
        """(device pointer, length) of an FP64 context vector, e.g. "den"."""
        ptr, n = C.c_void_p(), C.c_int64()
        self._c(lib().mp_device_buffer(self.h, VEC[name], C.byref(ptr), C.byref(n)))
        return ptr.value, int(n.value)

    def launches(self) -> int:
        n = C.c_int64()
        self._c(lib().mp_kernel_launches(self.h, C.byref(n)))
        return int(n.value)

    def set_form(self, form):
        self._c(lib().mp_set_particle_form(self.h, form))

    def stream(self) -> int:
        s = C.c_void_p()
        self._c(lib().mp_get_stream(self.h, C.byref(s)))
        return s.value or 0

    def synchronize(self):
        self._c(lib().mp_synchronize(self.h))

    # particles
    def reserve(self, n):
        self._c(lib().mp_particles_reserve(self.h, int(n)))

    def append(self, pos, vel, cell, rewind=False, q_over_m=0.0, half_dt=0.0):
        pos = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1, 3)
        vel = np.ascontiguousarray(vel, dtype=np.float64).reshape(-1, 3)
        cell = np.ascontiguousarray(cell, dtype=np.int32).ravel()
        n = cell.size
        self._c(lib().mp_particles_append(self.h, n, _p(pos), 24, _p(vel), 24, _p(cell), 4, int(bool(rewind)),
                                          float(q_over_m), float(half_dt)))

    def append_device(self, pos_soa_ptr, vel_soa_ptr, cell_ptr, n, rewind=False, q_over_m=0.0, half_dt=0.0):
        self._c(lib().mp_particles_append_device(self.h, int(n), pos_soa_ptr, vel_soa_ptr, cell_ptr,
                                                 int(bool(rewind)), float(q_over_m), float(half_dt)))

    def count(self) -> int:
        n = C.c_int64()
        self._c(lib().mp_particles_count(self.h, C.byref(n)))
        return int(n.value)

    def download(self, order=ORDER_ID):
        n = self.count()
        pos, vel, lc = np.zeros((n, 3)), np.zeros((n, 3)), np.zeros((n, 4))
        cell = np.zeros(n, dtype=np.int32)
        ids = np.zeros(n, dtype=np.int64)
        self._c(lib().mp_particles_download(self.h, n, _p(pos), 24, _p(vel), 24, _p(cell), 4, _p(lc), 32, _p(ids),
                                            order))
        return dict(pos=pos, vel=vel, cell=cell, lc=lc, id=ids)

    def clear(self):
        self._c(lib().mp_particles_clear(self.h))

    def push(self, q_over_m, dt, spwt, den_out: np.ndarray | None = None) -> StepStats:
        st = StepStats()
        self._c(lib().mp_push_scatter(self.h, float(q_over_m), float(dt), float(spwt), _p(den_out), C.byref(st)))
        return st

    def density(self) -> np.ndarray:
        out = np.zeros(self.mesh.n_nodes)
        self._c(lib().mp_density_download(self.h, _p(out)))
        return out

    def sort_by_tet(self):
        self._c(lib().mp_sort_by_tet(self.h))

    # field
    def set_fe_storage(self, storage):
        """FE_DENSE (default: dense K and J plus a sparse K) or FE_SPARSE (the
        sparse K only; SPARSE_CG and SPARSE_NEWTON).  Before fe_setup."""
        self._c(lib().mp_set_fe_storage(self.h, storage))

    def set_kernel_timing(self, on=True):
        """CUDA events around every launch of the kernel classes (KT_*); resets
        the clocks.  on: True (every class), False, or a bit mask of classes."""
        mask = (1 if on else 0) if isinstance(on, bool) else int(on)
        self._c(lib().mp_set_kernel_timing(self.h, mask))

    def kernel_timing(self, kclass: int) -> dict:
        """launches, device ms and algorithmic work (bytes or flops) of a kernel class."""
        n, ms, w = C.c_int64(0), C.c_double(0), C.c_double(0)
        self._c(lib().mp_kernel_timing(self.h, int(kclass), C.byref(n), C.byref(ms), C.byref(w)))
        return {"launches": int(n.value), "ms": float(ms.value), "work": float(w.value)}

    def set_gs_max_sweeps(self, sweeps=10000):
        """Gauss-Seidel sweep limit (the reference's is 10000)."""
        self._c(lib().mp_set_gs_max_sweeps(self.h, int(sweeps)))

    def set_sparse_solver(self, rtol=1e-12, max_iterations=20000):
        """Conjugate-gradient stop: ||G - J y|| <= rtol ||G||."""
        self._c(lib().mp_set_sparse_solver(self.h, float(rtol), int(max_iterations)))

    def fe_sparse_matrix(self):
        """The sparse K as CSR arrays (row_ptr, col, val), columns ascending."""
        nnz = C.c_int64()
        self._c(lib().mp_fe_sparse_matrix(self.h, C.byref(nnz), None, None, None))
        row_ptr = np.zeros(self.neq + 1, dtype=np.int64)
        col = np.zeros(nnz.value, dtype=np.int32)
        val = np.zeros(nnz.value)
        self._c(lib().mp_fe_sparse_matrix(self.h, C.byref(nnz), _p(row_ptr), _p(col), _p(val)))
        return row_ptr, col, val

    def fe_setup(self, ID, nx, detJ, g, neq, n0, phi0, kTe, K=None, F0=None):
        d = FeDesc()
        self._fe_keep = [np.ascontiguousarray(ID, dtype=np.int32), np.ascontiguousarray(nx, dtype=np.float64),
                         np.ascontiguousarray(detJ, dtype=np.float64), np.ascontiguousarray(g, dtype=np.float64)]
        d.neq = int(neq)
        d.ID, d.nx, d.detJ, d.g = (_p(a).value for a in self._fe_keep)
        if K is not None:
            Kc = np.ascontiguousarray(K, dtype=np.float64)
            F0c = np.ascontiguousarray(F0, dtype=np.float64)
            self._fe_keep += [Kc, F0c]
            d.K_dense = _p(Kc).value
            d.F0 = _p(F0c).value
        d.n0, d.phi0, d.kTe = float(n0), float(phi0), float(kTe)
        self._c(lib().mp_fe_setup(self.h, C.byref(d)))
        self.neq = int(neq)

    def fe_get(self, name: str) -> np.ndarray:
        w = VEC[name]
        if name in ("K", "J"):
            out = np.zeros((self.neq, self.neq))
        elif name in ("F0", "F1", "d", "G", "y"):
            out = np.zeros(self.neq)
        elif name == "ef":
            out = np.zeros((self.mesh.n_tets, 3))
        else:
            out = np.zeros(self.mesh.n_nodes)
        self._c(lib().mp_fe_download(self.h, w, _p(out)))
        return out

    def fe_set(self, name: str, values) -> None:
        a = np.ascontiguousarray(values, dtype=np.float64)
        self._c(lib().mp_fe_upload(self.h, VEC[name], _p(a)))

    def compute_phi(self, method=LAPACK, form=FP64, ion_den: np.ndarray | None = None) -> NewtonStats:
        st = NewtonStats()
        den = None if ion_den is None else np.ascontiguousarray(ion_den, dtype=np.float64)
        self._c(lib().mp_compute_phi(self.h, _p(den), method, form, C.byref(st)))
        return st

    def build_f1(self, ion_den=None):
        den = None if ion_den is None else np.ascontiguousarray(ion_den, dtype=np.float64)
        self._c(lib().mp_fe_build_f1(self.h, _p(den)))

    def residual(self):
        self._c(lib().mp_fe_residual(self.h))

    def build_j(self, method=LAPACK):
        self._c(lib().mp_fe_build_j(self.h, method))

    def solve_linear(self, method=LAPACK, form=FP64, b=None) -> NewtonStats:
        st = NewtonStats()
        bb = None if b is None else np.ascontiguousarray(b, dtype=np.float64)
        self._c(lib().mp_fe_solve_linear(self.h, method, form, _p(bb), C.byref(st)))
        return st

    def update_ef(self, uh=None):
        u = None if uh is None else np.ascontiguousarray(uh, dtype=np.float64)
        self._c(lib().mp_update_ef(self.h, _p(u)))

    def output_mesh(self, ts: int, directory: str, node_type: np.ndarray) -> None:
        """OutputMesh: mesh_<ts+1>.vtu in `directory`, written by a background
        thread (output_wait joins it)."""
        self._out_types = np.ascontiguousarray(node_type, dtype=np.int32)
        self._c(lib().mp_output_mesh(self.h, int(ts), directory.encode(), _p(self._out_types), 4))

    def output_particles(self, path: str) -> None:
        """OutputParticles into `path`, written by a background thread."""
        self._c(lib().mp_output_particles(self.h, path.encode()))

    def output_wait(self) -> None:
        self._c(lib().mp_output_wait(self.h))

    def field(self):
        d = np.zeros(self.neq) if self.neq else None
        uh = np.zeros(self.mesh.n_nodes) if self.neq else None
        ef = np.zeros((self.mesh.n_tets, 3))
        self._c(lib().mp_field_download(self.h, _p(d), _p(uh), _p(ef)))
        return d, uh, ef


class Injector:
    """InjectIons' sampling (src/mini-pic.cpp:208-265) with the reference's RNG stream."""

    def __init__(self, mesh: Mesh, seed: int = 0):
        L = lib()
        h = C.c_void_p()
        self._keep = [np.ascontiguousarray(a) for a in (mesh.inlet_con, mesh.inlet_u, mesh.inlet_v,
                                                        mesh.inlet_normal, mesh.inlet_area, mesh.inlet_cell,
                                                        mesh.node_pos)]
        _check(L.mp_injector_create(mesh.inlet_con.shape[0], *(_p(a) for a in self._keep), seed, C.byref(h)))
        self.h = h

    def __del__(self):
        try:
            if self.h:
                lib().mp_injector_destroy(self.h)
                self.h = None
        except Exception:
            pass

    @property
    def rem(self) -> float:
        r = C.c_double()
        _check(lib().mp_injector_get_rem(self.h, C.byref(r)))
        return r.value

    @rem.setter
    def rem(self, value: float):
        _check(lib().mp_injector_set_rem(self.h, float(value)))

    def sample(self, plasma_den, ion_velocity, dt, spwt):
        n = C.c_int64()
        _check(lib().mp_injector_count(self.h, plasma_den, ion_velocity, dt, spwt, C.byref(n)))
        cap = max(int(n.value), 1)
        pos, vel = np.zeros((cap, 3)), np.zeros((cap, 3))
        cell = np.zeros(cap, dtype=np.int32)
        got = C.c_int64()
        _check(lib().mp_injector_sample(self.h, plasma_den, ion_velocity, dt, spwt, cap, _p(pos), 24, _p(vel), 24,
                                        _p(cell), 4, C.byref(got)))
        k = int(got.value)
        return pos[:k], vel[:k], cell[:k]
