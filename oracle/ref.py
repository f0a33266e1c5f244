"""Test infrastructure: ctypes access to oracle/_ref/libref_oracle.so, the
reference's own compiled translation units plus the harness in ref_harness.cpp.

Only tests, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg use
this module, as the checker.  Record layouts mirror the reference's POD
structs (src/meshes.h:33-43 Tetra, src/particles.h:21-26 Particle), which the
reference copies bytewise to its device (src/mini-pic.cpp:275, 337).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libref_oracle.so")
# the same harness linked with the C++ drop-in shim (mini-fem-pic-main_b200/shim)
# and libminipic_cuda.so: the reference's own types driven through the device path
SHIM_PATH = os.path.join(HERE, "_ref", "libref_shim.so")

TETRA_DTYPE = np.dtype({
    "names": ["con", "volume", "alpha", "beta", "gamma", "delta", "cell_con"],
    "formats": [("<i4", 4), "<f8", ("<f8", 4), ("<f8", 4), ("<f8", 4), ("<f8", 4), ("<i4", 4)],
    "offsets": [0, 16, 24, 56, 88, 120, 152],
    "itemsize": 168,
})
PARTICLE_DTYPE = np.dtype({
    "names": ["pos", "vel", "lc", "cell_index"],
    "formats": [("<f8", 3), ("<f8", 3), ("<f8", 4), "<i4"],
    "offsets": [0, 24, 48, 80],
    "itemsize": 88,
})

# FESolver::Method (src/FESolver.h:26)
NONLINEAR, GAUSS_SEIDEL, LAPACK = 0, 1, 2

_libs = {}


def available() -> bool:
    return os.path.exists(LIB_PATH)


def shim_available() -> bool:
    return os.path.exists(SHIM_PATH)


def lib(shim: bool = False):
    if shim not in _libs:
        L = C.CDLL(SHIM_PATH if shim else LIB_PATH)
        vp, i, d, l = C.c_void_p, C.c_int, C.c_double, C.c_long
        sig = {
            "ref_sizeof_tetra": (i, []), "ref_sizeof_particle": (i, []),
            "ref_open": (vp, [C.c_char_p]), "ref_add_fixed_surface": (i, [vp, C.c_char_p]),
            "ref_init_solver": (None, [vp]), "ref_set_g": (None, [vp, i, d]),
            "ref_assemble": (None, [vp]), "ref_init_species": (None, [vp, d, d]),
            "ref_close": (None, [vp]), "ref_n_nodes": (i, [vp]), "ref_n_tets": (i, [vp]),
            "ref_n_inlet": (i, [vp]), "ref_neq": (i, [vp]), "ref_n_particles": (l, [vp]),
            "ref_rem": (d, [vp]), "ref_param": (d, [vp, i]),
            "ref_get_tetra_raw": (None, [vp, vp]), "ref_get_nodes": (None, [vp, vp, vp, vp]),
            "ref_get_inlet": (None, [vp] * 7), "ref_get_fe": (None, [vp] * 5),
            "ref_get_matrix": (None, [vp, i, vp]), "ref_get_vec": (None, [vp, i, vp]),
            "ref_set_vec": (None, [vp, i, vp]), "ref_get_particles": (None, [vp, vp]),
            "ref_set_particles": (None, [vp, vp, l]), "ref_set_rem": (None, [vp, d]),
            "ref_inject": (i, [vp]), "ref_push_only": (None, [vp, i]),
            "ref_compact_normalise": (l, [vp]), "ref_move": (l, [vp, i]),
            "ref_compute_phi": (None, [vp, i]), "ref_update_ef": (None, [vp]),
            "ref_build_f1": (None, [vp, vp]), "ref_build_j": (None, [vp, i]),
            "ref_residual": (None, [vp, vp]), "ref_solve_gs": (None, [vp, vp, vp]),
            "ref_solve_lapack": (None, [vp, vp, vp]),
            "ref_time_move": (d, [vp, i, i, vp]), "ref_max_threads": (i, []),
            "ref_reseed": (None, [C.c_uint]),
            "ref_output_mesh": (d, [vp, i, C.c_char_p]), "ref_output_particles": (d, [vp, C.c_char_p]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        if shim:
            for name, (res, args) in {"ref_shim_device": (vp, [vp]), "ref_shim_free": (None, [vp]),
                                      "ref_shim_move": (None, [vp, vp]), "ref_shim_compute_phi": (None, [vp, vp, i]),
                                      "ref_shim_update_ef": (None, [vp, vp]),
                                      "ref_shim_mesh_check": (l, [vp, vp]),
                                      "ref_shim_output": (i, [vp, vp, i, C.c_char_p]),
                                      "ref_shim_set_storage": (None, [vp, i])}.items():
                f = getattr(L, name)
                f.restype = res
                f.argtypes = args
        assert L.ref_sizeof_tetra() == TETRA_DTYPE.itemsize
        assert L.ref_sizeof_particle() == PARTICLE_DTYPE.itemsize
        _libs[shim] = L
    return _libs[shim]


def _p(a: np.ndarray):
    assert a.flags.c_contiguous
    return a.ctypes.data_as(C.c_void_p)


class RefSim:
    """One reference simulation: Parameters, Volume, FESolver and Species, set up
    the way ``main`` does (src/mini-pic.cpp:75-116)."""

    def __init__(self, deck_dir: str, *, spwt: float = 200.0, mass_amu: float = 16.0,
                 extra_fixed: dict | None = None, shim: bool = False):
        self.L = L = lib(shim)
        self.device = None
        L.ref_reseed(0)  # each simulation starts the reference's RNG stream afresh
        self.h = L.ref_open(deck_dir.encode())
        if not self.h:
            raise RuntimeError(f"reference failed to load deck {deck_dir}")
        extra_fixed = extra_fixed or {}
        for path in extra_fixed:
            if L.ref_add_fixed_surface(self.h, path.encode()) != 0:
                raise RuntimeError(f"failed to load {path}")
        L.ref_init_solver(self.h)
        for path, (nodes, value) in extra_fixed.items():
            for n in nodes:
                L.ref_set_g(self.h, int(n), float(value))
        L.ref_assemble(self.h)
        L.ref_init_species(self.h, spwt, mass_amu)
        self.n_nodes = L.ref_n_nodes(self.h)
        self.n_tets = L.ref_n_tets(self.h)
        self.n_inlet = L.ref_n_inlet(self.h)
        self.neq = L.ref_neq(self.h)

    def close(self):
        if getattr(self, "device", None):
            self.L.ref_shim_free(self.device)
            self.device = None
        if self.h:
            self.L.ref_close(self.h)
            self.h = None

    # ---- the device path through the C++ drop-in (shim libraries only) ----
    def shim_device(self) -> None:
        """DeviceData device(volume), as main() creates it."""
        self.device = self.L.ref_shim_device(self.h)

    def shim_move(self) -> None:
        """MoveParticles(ions, volume, solver, params, device) of the drop-in."""
        self.L.ref_shim_move(self.h, self.device)

    def shim_compute_phi(self, method: int) -> None:
        self.L.ref_shim_compute_phi(self.h, self.device, method)

    def shim_update_ef(self) -> None:
        self.L.ref_shim_update_ef(self.h, self.device)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def param(self, which: int) -> float:
        return self.L.ref_param(self.h, which)

    @property
    def dt(self):
        return self.param(4)

    @property
    def q_over_m(self):
        return self.param(8) / self.param(9)

    @property
    def spwt(self):
        return self.param(10)

    def tetra(self) -> np.ndarray:
        out = np.zeros(self.n_tets, dtype=TETRA_DTYPE)
        self.L.ref_get_tetra_raw(self.h, _p(out))
        return out

    def nodes(self):
        pos = np.zeros((self.n_nodes, 3))
        typ = np.zeros(self.n_nodes, dtype=np.int32)
        vol = np.zeros(self.n_nodes)
        self.L.ref_get_nodes(self.h, _p(pos), _p(typ), _p(vol))
        return pos, typ, vol

    def inlet(self) -> dict:
        n = self.n_inlet
        con = np.zeros((n, 3), dtype=np.int32)
        area = np.zeros(n)
        u = np.zeros((n, 3))
        v = np.zeros((n, 3))
        cell = np.zeros(n, dtype=np.int32)
        normal = np.zeros((n, 3))
        self.L.ref_get_inlet(self.h, _p(con), _p(area), _p(u), _p(v), _p(cell), _p(normal))
        return dict(con=con, area=area, u=u, v=v, cell_con=cell, normal=normal)

    def fe(self) -> dict:
        ID = np.zeros(self.n_nodes, dtype=np.int32)
        LM = np.zeros((self.n_tets, 4), dtype=np.int32)
        NX = np.zeros((self.n_tets, 4, 3))
        detJ = np.zeros(self.n_tets)
        self.L.ref_get_fe(self.h, _p(ID), _p(LM), _p(NX), _p(detJ))
        return dict(ID=ID, LM=LM, NX=NX, detJ=detJ)

    def matrix(self, which: int = 0) -> np.ndarray:
        out = np.zeros((self.neq, self.neq))
        self.L.ref_get_matrix(self.h, which, _p(out))
        return out

    _VEC = {"F0": 0, "F1": 1, "d": 2, "g": 3, "uh": 4, "den": 5, "ef": 6}

    def _veclen(self, name):
        if name in ("F0", "F1", "d"):
            return self.neq
        if name == "ef":
            return 3 * self.n_tets
        return self.n_nodes

    def get(self, name: str) -> np.ndarray:
        out = np.zeros(self._veclen(name))
        self.L.ref_get_vec(self.h, self._VEC[name], _p(out))
        return out.reshape(-1, 3) if name == "ef" else out

    def set(self, name: str, values) -> None:
        a = np.ascontiguousarray(values, dtype=np.float64).ravel()
        assert a.size == self._veclen(name)
        self.L.ref_set_vec(self.h, self._VEC[name], _p(a))

    def particles(self) -> np.ndarray:
        out = np.zeros(self.L.ref_n_particles(self.h), dtype=PARTICLE_DTYPE)
        if out.size:
            self.L.ref_get_particles(self.h, _p(out))
        return out

    def set_particles(self, parts: np.ndarray) -> None:
        parts = np.ascontiguousarray(parts, dtype=PARTICLE_DTYPE)
        self.L.ref_set_particles(self.h, _p(parts) if parts.size else None, parts.size)

    @property
    def rem(self):
        return self.L.ref_rem(self.h)

    def inject(self) -> int:
        return self.L.ref_inject(self.h)

    def push_only(self, nthreads: int = 1) -> None:
        self.L.ref_push_only(self.h, nthreads)

    def compact_normalise(self) -> int:
        return self.L.ref_compact_normalise(self.h)

    def move(self, nthreads: int = 1) -> int:
        return self.L.ref_move(self.h, nthreads)

    def compute_phi(self, method: int) -> None:
        self.L.ref_compute_phi(self.h, method)

    def update_ef(self) -> None:
        self.L.ref_update_ef(self.h)

    def build_f1(self, den: np.ndarray) -> None:
        den = np.ascontiguousarray(den, dtype=np.float64)
        self.L.ref_build_f1(self.h, _p(den))

    def build_j(self, method: int) -> None:
        self.L.ref_build_j(self.h, method)

    def residual(self) -> np.ndarray:
        G = np.zeros(self.neq)
        self.L.ref_residual(self.h, _p(G))
        return G

    def solve_gs(self, b: np.ndarray, x0: np.ndarray | None = None) -> np.ndarray:
        b = np.ascontiguousarray(b, dtype=np.float64)
        x = np.zeros(self.neq) if x0 is None else np.array(x0, dtype=np.float64)
        self.L.ref_solve_gs(self.h, _p(b), _p(x))
        return x

    def solve_lapack(self, b: np.ndarray) -> np.ndarray:
        b = np.ascontiguousarray(b, dtype=np.float64)
        x = np.zeros(self.neq)
        self.L.ref_solve_lapack(self.h, _p(b), _p(x))
        return x

    def time_move(self, steps: int, nthreads: int):
        sec = C.c_double(0)
        rate = self.L.ref_time_move(self.h, steps, nthreads, C.byref(sec))
        return rate, sec.value


def max_threads() -> int:
    return lib().ref_max_threads()


def compute_phi_isolated(deck_dir: str, method: int, d, F1, den, *, spwt: float = 200.0,
                         extra_fixed: dict | None = None, timeout: float = 600.0) -> dict:
    """The reference's computePhi from the state (d, F1, ion density) in a
    child process (oracle/ref_isolated.py), since its NonLinear method may end
    the process.  Returns exitcode, the reference's printed messages (log) and,
    when it returned, d and uh."""
    with tempfile.TemporaryDirectory() as wd:
        inp, out = os.path.join(wd, "in.npz"), os.path.join(wd, "out.npz")
        extra = {}
        for path, (nodes, value) in (extra_fixed or {}).items():
            extra = dict(fixed_file=path, fixed_nodes=np.asarray(nodes, dtype=np.int64), fixed_value=value)
        np.savez(inp, method=method, spwt=spwt, d=np.asarray(d, dtype=np.float64),
                 F1=np.asarray(F1, dtype=np.float64), den=np.asarray(den, dtype=np.float64), **extra)
        root = os.path.dirname(HERE)
        p = subprocess.run([sys.executable, "-m", "oracle.ref_isolated", deck_dir, inp, out], cwd=root,
                           capture_output=True, text=True, timeout=timeout,
                           env=dict(os.environ, CUDA_VISIBLE_DEVICES=""))
        res = {"exitcode": p.returncode, "log": p.stdout + p.stderr}
        if p.returncode == 0:
            r = dict(np.load(out))
            res.update(d=r["d"], uh=r["uh"], F1=r["F1"])
    return res
