"""Test infrastructure: ctypes access to oracle/liboracle.so (oracle.c, the C
restatement of the reference's hot path).  Used only by tests, smoke() and
bench.py's CPU-baseline leg, as the checker."""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")

_lib = None


class MT(C.Structure):
    _fields_ = [("mt", C.c_uint32 * 624), ("idx", C.c_int)]


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        L = C.CDLL(LIB_PATH)
        vp, i, d, l = C.c_void_p, C.c_int, C.c_double, C.c_long
        sig = {
            "or_mt_seed": (None, [vp, C.c_uint32]), "or_mt_next": (C.c_uint32, [vp]), "or_rnd": (d, [vp]),
            "or_inject": (l, [vp, vp, i, vp, vp, vp, vp, vp, vp, vp, d, d, d, d, l, vp, vp, vp]),
            "or_rewind": (None, [l, vp, vp, vp, d, d]),
            "or_push": (l, [l, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, d, d, vp, i, vp]),
            "or_compact": (l, [l, vp, vp, vp, vp]),
            "or_normalise": (None, [i, vp, vp, d]),
            "or_update_ef": (None, [i, vp, vp, vp, vp]),
            "or_build_f1": (None, [i, i, i, vp, vp, vp, vp, vp, d, d, d, vp]),
            "or_build_fp": (None, [i, i, vp, vp, vp, vp, d, d, d, vp]),
            "or_residual": (None, [i, vp, vp, vp, vp, vp]),
            "or_build_j": (None, [i, vp, vp, vp]),
            "or_gauss_seidel": (i, [i, vp, vp, vp, vp]),
            "or_solve_dense": (i, [i, vp, vp]),
            "or_assemble": (None, [i, i, vp, vp, vp, vp, vp, vp, vp]),
            "or_uh": (None, [i, vp, vp, vp, vp]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _p(a):
    if a is None:
        return None
    assert a.flags.c_contiguous
    return a.ctypes.data_as(C.c_void_p)


class Rng:
    """std::mt19937(seed) + uniform_real_distribution<double>(0,1)."""

    def __init__(self, seed: int = 0):
        self.g = MT()
        lib().or_mt_seed(C.byref(self.g), seed)

    def rnd(self) -> float:
        return lib().or_rnd(C.byref(self.g))


class Injector:
    def __init__(self, mesh, seed: int = 0):
        self.rng = Rng(seed)
        self.rem = C.c_double(0.0)
        self.m = mesh

    def sample(self, plasma_den, ion_velocity, dt, spwt, max_n=1_000_000):
        m = self.m
        pos, vel = np.zeros((max_n, 3)), np.zeros((max_n, 3))
        cell = np.zeros(max_n, dtype=np.int32)
        k = lib().or_inject(C.byref(self.rng.g), C.byref(self.rem), m.inlet_con.shape[0], _p(m.inlet_con),
                            _p(m.inlet_u), _p(m.inlet_v), _p(m.inlet_normal), _p(m.inlet_area), _p(m.inlet_cell),
                            _p(m.node_pos), plasma_den, ion_velocity, dt, spwt, max_n, _p(pos), _p(vel), _p(cell))
        assert k <= max_n
        return pos[:k].copy(), vel[:k].copy(), cell[:k].copy()


def rewind(vel, cell, ef, q_over_m, half_dt):
    lib().or_rewind(cell.size, _p(vel), _p(cell), _p(np.ascontiguousarray(ef)), q_over_m, half_dt)


class Particles:
    """The oracle's particle state: packed arrays in the reference's order."""

    def __init__(self):
        self.pos = np.zeros((0, 3))
        self.vel = np.zeros((0, 3))
        self.cell = np.zeros(0, dtype=np.int32)
        self.id = np.zeros(0, dtype=np.int64)
        self.next_id = 0

    def append(self, pos, vel, cell):
        k = len(cell)
        self.pos = np.ascontiguousarray(np.concatenate([self.pos, pos]))
        self.vel = np.ascontiguousarray(np.concatenate([self.vel, vel]))
        self.cell = np.ascontiguousarray(np.concatenate([self.cell, cell]).astype(np.int32))
        self.id = np.ascontiguousarray(np.concatenate([self.id, np.arange(self.next_id, self.next_id + k)]))
        self.next_id += k


def move(parts: Particles, mesh, ef, q_over_m, dt, spwt, want_lc=False):
    """MoveParticles (src/mini-pic.cpp:268-320): push in order, erase exits,
    normalise.  Returns (den, removed, hops, lc-before-compaction)."""
    n = parts.cell.size
    den = np.zeros(mesh.n_nodes)
    lc = np.zeros((n, 4)) if want_lc else None
    hops = C.c_long(0)
    ef = np.ascontiguousarray(ef, dtype=np.float64)
    removed = lib().or_push(n, _p(parts.pos), _p(parts.vel), _p(parts.cell), _p(lc), _p(mesh.con), _p(mesh.volume),
                            _p(mesh.alpha), _p(mesh.beta), _p(mesh.gamma), _p(mesh.delta), _p(mesh.cell_con), _p(ef),
                            q_over_m, dt, _p(den), mesh.n_nodes, C.byref(hops))
    keep = parts.cell >= 0
    if lc is not None:
        lc = lc[keep]
    w = lib().or_compact(n, _p(parts.pos), _p(parts.vel), _p(parts.cell), _p(parts.id))
    parts.pos = np.ascontiguousarray(parts.pos[:w])
    parts.vel = np.ascontiguousarray(parts.vel[:w])
    parts.cell = np.ascontiguousarray(parts.cell[:w])
    parts.id = np.ascontiguousarray(parts.id[:w])
    lib().or_normalise(mesh.n_nodes, _p(den), _p(mesh.node_volume), spwt)
    return den, removed, hops.value, lc


def update_ef(mesh, nx, uh):
    ef = np.zeros((mesh.n_tets, 3))
    lib().or_update_ef(mesh.n_tets, _p(mesh.con), _p(np.ascontiguousarray(nx)), _p(np.ascontiguousarray(uh)), _p(ef))
    return ef


class FE:
    """FESolver's state and methods, restated (src/FESolver.cpp)."""

    def __init__(self, mesh, ID, nx, detJ, g, neq, n0, phi0, kTe):
        self.mesh = mesh
        self.ID = np.ascontiguousarray(ID, dtype=np.int32)
        self.nx = np.ascontiguousarray(nx, dtype=np.float64)
        self.detJ = np.ascontiguousarray(detJ)
        self.g = np.ascontiguousarray(g)
        self.neq, self.n0, self.phi0, self.kTe = int(neq), n0, phi0, kTe
        self.K = np.zeros((neq, neq))
        self.F0 = np.zeros(neq)
        self.F1 = np.zeros(neq)
        self.d = np.zeros(neq)
        self.uh = np.zeros(mesh.n_nodes)
        self.FP = np.zeros(neq)
        self.J = np.zeros((neq, neq))
        lib().or_assemble(mesh.n_tets, neq, _p(self.ID), _p(mesh.con), _p(self.nx), _p(self.detJ), _p(self.g),
                          _p(self.K), _p(self.F0))

    def build_f1(self, den):
        m = self.mesh
        lib().or_build_f1(m.n_nodes, m.n_tets, self.neq, _p(self.ID), _p(m.con), _p(self.detJ),
                          _p(np.ascontiguousarray(den)), _p(self.d), self.n0, self.phi0, self.kTe, _p(self.F1))

    def residual(self):
        G = np.zeros(self.neq)
        lib().or_residual(self.neq, _p(self.K), _p(self.d), _p(self.F0), _p(self.F1), _p(G))
        return G

    def build_j(self):
        m = self.mesh
        lib().or_build_fp(m.n_tets, self.neq, _p(self.ID), _p(m.con), _p(self.detJ), _p(self.d), self.n0, self.phi0,
                          self.kTe, _p(self.FP))
        lib().or_build_j(self.neq, _p(self.K), _p(self.FP), _p(self.J))

    def gauss_seidel(self, b, x):
        L2 = C.c_double()
        it = lib().or_gauss_seidel(self.neq, _p(self.J), _p(np.ascontiguousarray(b)), _p(x), C.byref(L2))
        return it, L2.value

    def solve_dense(self, b):
        A = self.J.copy()
        x = np.array(b, dtype=np.float64)
        rc = lib().or_solve_dense(self.neq, _p(A), _p(x))
        if rc:
            raise ArithmeticError(f"zero pivot at {rc - 1}")
        return x

    def compute_phi(self, den, method):
        """computePhi for the GaussSeidel and Lapack methods (one Newton step),
        src/FESolver.cpp:290-321, 604-619."""
        y = np.zeros(self.neq)
        self.build_f1(den)
        G = self.residual()
        self.build_j()
        if method == 1:
            self.gauss_seidel(G, y)
        else:
            y = self.solve_dense(G)
        self.d -= y
        lib().or_uh(self.mesh.n_nodes, _p(self.ID), _p(self.g), _p(self.d), _p(self.uh))
        return y

    def update_ef(self):
        return update_ef(self.mesh, self.nx, self.uh)


# ---------------------------------------------------------------------------
# dual-number (forward-mode) build of the push: oracle/dual.cpp -> libdual.so

DUAL_PATH = os.path.join(HERE, "libdual.so")
_dual = None


def dual_available() -> bool:
    return os.path.exists(DUAL_PATH)


def _dual_lib():
    global _dual
    if _dual is None:
        L = C.CDLL(DUAL_PATH)
        vp, i, d, l = C.c_void_p, C.c_int, C.c_double, C.c_long
        L.or_dual_ksteps.restype = i
        L.or_dual_ksteps.argtypes = ([i] + [vp] * 8 + [i, vp, vp, l] + [vp] * 5 + [i, d, d, d, d, vp, vp, vp, d, d]
                                     + [vp] * 10)
        _dual = L
    return _dual


def dual_ksteps(mesh, nx, wall_nodes, slots, K, qm, mass, dt, spwt, inlet_dir, phi, vd, dphi=None, dvd=0.0):
    """K push + scatter steps with phi held (the adjoint's model) in dual
    numbers.  slots: dict of first [n] int32, inj [n] uint8, pos/vel [n][3],
    cell [n] int32.  Returns dict den, dden, flux, dflux, kind, exit, pos,
    vel, cell."""
    n = int(slots["cell"].size)
    f = lambda a, t: np.ascontiguousarray(a, dtype=t)  # noqa: E731
    first, inj = f(slots["first"], np.int32), f(slots["inj"], np.uint8)
    pos, vel, cell = f(slots["pos"], np.float64), f(slots["vel"], np.float64), f(slots["cell"], np.int32)
    out = {"den": np.zeros(mesh.n_nodes), "dden": np.zeros(mesh.n_nodes), "kind": np.zeros(n, np.int32),
           "exit": np.zeros(n, np.int32), "pos": np.zeros((n, 3)), "vel": np.zeros((n, 3)),
           "cell": np.zeros(n, np.int32), "path": np.zeros(n, np.uint64)}
    flux, dflux = C.c_double(0), C.c_double(0)
    dphi = None if dphi is None else f(dphi, np.float64)
    rc = _dual_lib().or_dual_ksteps(
        mesh.n_tets, _p(mesh.con), _p(mesh.volume), _p(mesh.alpha), _p(mesh.beta), _p(mesh.gamma), _p(mesh.delta),
        _p(mesh.cell_con), _p(f(nx, np.float64)), mesh.n_nodes, _p(mesh.node_volume), _p(f(wall_nodes, np.uint8)),
        n, _p(first), _p(inj), _p(pos), _p(vel), _p(cell), K, qm, mass, dt, spwt, _p(f(inlet_dir, np.float64)),
        _p(f(phi, np.float64)), _p(dphi), vd, dvd, _p(out["den"]), _p(out["dden"]), C.byref(flux), C.byref(dflux),
        _p(out["kind"]), _p(out["exit"]), _p(out["pos"]), _p(out["vel"]), _p(out["cell"]), _p(out["path"]))
    if rc != 0:
        raise RuntimeError("dual push: a tet walk did not end")
    out["flux"], out["dflux"] = flux.value, dflux.value
    return out
