"""Synthetic Kuhn-box decks written in the reference's Salome ``.dat`` format.

A deck is the directory the reference's ``mini-pic <system.param>`` runs from:
``mesh.dat`` (volume, element type 304), ``inlet.dat`` (type 203 triangles on
x=0), ``wall.dat`` (nodes on x=L, held at ``-wall_potential``) and
``system.param``.  Optionally a spherical inclusion is cut out of the box and
its surface nodes are listed in ``sphere.dat``; the caller holds those at their
own potential (the reference's deck format has only one wall potential, so the
harness sets ``g`` for them directly, as ``main`` does in
src/mini-pic.cpp:98-102).

File formats follow the readers in src/meshes.cpp:28-73 (volume) and
src/meshes.cpp:268-303 (surfaces): a ``n_nodes n_elements`` header, node lines
``index x y z`` in millimetres (the loader divides by 1000, meshes.cpp:45), and
element lines ``index type n1 n2 n3 [n4]`` with 1-based node indices.

The box is split into n^3 hexes and each hex into the 6 Kuhn (Freudenthal)
tetrahedra along its (0,0,0)->(1,1,1) diagonal, which conform across hexes.
Tet ``6*hex + perm`` is the tet of permutation ``PERMS[perm]``; the analytic
point location in :func:`locate` relies on that numbering.
"""
from __future__ import annotations

import os
from dataclasses import dataclass, field

import numpy as np

# Axis orders of the 6 Kuhn tets of one hex: vertices are
# v0 = corner, v1 = v0 + e[p0], v2 = v1 + e[p1], v3 = corner + (1,1,1).
PERMS = ((0, 1, 2), (0, 2, 1), (1, 0, 2), (1, 2, 0), (2, 0, 1), (2, 1, 0))

KB_EV = 8.617333262e-5  # Boltzmann constant in eV/K, src/FESolver.h:21


@dataclass
class KuhnDeck:
    n: int
    length_mm: float
    nodes_mm: np.ndarray          # [n_nodes, 3] float64, millimetres as written
    tets: np.ndarray              # [n_tets, 4] int32, 0-based node ids as written
    inlet_tris: np.ndarray        # [n_in, 3] int32, 0-based, +x normal
    wall_tris: np.ndarray         # [n_wall, 3] int32
    inlet_nodes: np.ndarray       # 0-based node ids on x=0
    wall_nodes: np.ndarray        # 0-based node ids on x=L
    sphere_nodes: np.ndarray      # 0-based node ids on the sphere surface (may be empty)
    tet_hex_perm: np.ndarray      # [n_tets, 2] (hex id, perm id) of each kept tet
    hexperm_to_tet: np.ndarray    # [n^3*6] tet id or -1 if removed
    params: dict = field(default_factory=dict)

    @property
    def n_nodes(self) -> int:
        return int(self.nodes_mm.shape[0])

    @property
    def n_tets(self) -> int:
        return int(self.tets.shape[0])


def build(n: int, length_mm: float = 100.0, sphere: tuple | None = None) -> KuhnDeck:
    """Kuhn mesh of the box [0, length_mm]^3 with n^3 hexes.

    ``sphere`` = (cx, cy, cz, r) in millimetres removes the tets whose centroid
    lies inside it and drops nodes no remaining tet uses.
    """
    n1 = n + 1
    h = length_mm / n
    ii, jj, kk = np.meshgrid(np.arange(n1), np.arange(n1), np.arange(n1), indexing="ij")
    # node id = i + n1*j + n1^2*k
    coords = np.zeros((n1 ** 3, 3))
    gid = (ii + n1 * jj + n1 * n1 * kk).ravel()
    coords[gid, 0] = (ii.ravel() * h)
    coords[gid, 1] = (jj.ravel() * h)
    coords[gid, 2] = (kk.ravel() * h)

    hi, hj, hk = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    hex_id = (hi + n * hj + n * n * hk).ravel()
    order = np.argsort(hex_id)
    hi = hi.ravel()[order]
    hj = hj.ravel()[order]
    hk = hk.ravel()[order]
    unit = np.eye(3, dtype=np.int64)
    tets = np.zeros((n ** 3, 6, 4), dtype=np.int64)
    for p, perm in enumerate(PERMS):
        c = np.stack([hi, hj, hk], axis=1)
        v0 = c
        v1 = v0 + unit[perm[0]]
        v2 = v1 + unit[perm[1]]
        v3 = c + 1
        for s, v in enumerate((v0, v1, v2, v3)):
            tets[:, p, s] = v[:, 0] + n1 * v[:, 1] + n1 * n1 * v[:, 2]
    tets = tets.reshape(-1, 4)
    hexperm = np.stack([np.repeat(np.arange(n ** 3), 6), np.tile(np.arange(6), n ** 3)], axis=1)

    keep = np.ones(tets.shape[0], dtype=bool)
    if sphere is not None:
        cx, cy, cz, r = sphere
        cen = coords[tets].mean(axis=1)
        d2 = (cen[:, 0] - cx) ** 2 + (cen[:, 1] - cy) ** 2 + (cen[:, 2] - cz) ** 2
        keep = d2 >= r * r
    kept = tets[keep]
    removed = tets[~keep]
    used = np.zeros(coords.shape[0], dtype=bool)
    used[kept.ravel()] = True
    new_id = -np.ones(coords.shape[0], dtype=np.int64)
    new_id[used] = np.arange(int(used.sum()))
    nodes = coords[used]
    kept_new = new_id[kept].astype(np.int32)
    hexperm_to_tet = -np.ones(tets.shape[0], dtype=np.int64)
    hexperm_to_tet[np.nonzero(keep)[0]] = np.arange(int(keep.sum()))

    # Inlet/wall triangles follow the Kuhn face diagonal (0,j,k)-(0,j+1,k+1).
    # Vertex order (p0, p_diag, p_side) gives the +x normal with the
    # reference's normal = v x u convention (meshes.cpp:335-340).
    in_tris, wall_tris = [], []
    for k in range(n):
        for j in range(n):
            a = 0 + n1 * j + n1 * n1 * k
            b = 0 + n1 * (j + 1) + n1 * n1 * k
            c = 0 + n1 * j + n1 * n1 * (k + 1)
            d = 0 + n1 * (j + 1) + n1 * n1 * (k + 1)
            in_tris.append((a, d, b))
            in_tris.append((a, c, d))
            wall_tris.append((a + n, b + n, d + n))
            wall_tris.append((a + n, d + n, c + n))
    in_tris = new_id[np.array(in_tris)].astype(np.int32)
    wall_tris = new_id[np.array(wall_tris)].astype(np.int32)
    inlet_nodes = np.nonzero(used & (coords[:, 0] == 0.0))[0]
    wall_nodes = np.nonzero(used & (coords[:, 0] == length_mm))[0]
    sphere_nodes = np.array([], dtype=np.int64)
    if removed.size:
        on_sphere = np.zeros(coords.shape[0], dtype=bool)
        on_sphere[np.intersect1d(removed.ravel(), kept.ravel())] = True
        sphere_nodes = new_id[np.nonzero(on_sphere)[0]]
    return KuhnDeck(
        n=n, length_mm=length_mm, nodes_mm=nodes, tets=kept_new,
        inlet_tris=in_tris, wall_tris=wall_tris,
        inlet_nodes=new_id[inlet_nodes].astype(np.int32),
        wall_nodes=new_id[wall_nodes].astype(np.int32),
        sphere_nodes=np.sort(sphere_nodes).astype(np.int32),
        tet_hex_perm=hexperm[keep].astype(np.int64),
        hexperm_to_tet=hexperm_to_tet,
    )


def _fmt(x: float) -> str:
    # Shortest round-trip decimal: the C++ stream reader and Python's float()
    # both parse it back to the same double.
    return repr(float(x))


def _write_surface(path: str, deck: KuhnDeck, node_ids: np.ndarray, tris: np.ndarray) -> None:
    with open(path, "w") as f:
        f.write(f"{len(node_ids)} {len(tris)}\n")
        for nid in node_ids:
            x, y, z = deck.nodes_mm[nid]
            f.write(f"{nid + 1} {_fmt(x)} {_fmt(y)} {_fmt(z)}\n")
        for e, t in enumerate(tris):
            f.write(f"{e + 1} 203 {t[0] + 1} {t[1] + 1} {t[2] + 1}\n")


def write(deck: KuhnDeck, directory: str, *, plasma_den: float = 1e10, ion_velocity: float = 7000.0,
          kTe_eV: float = 2.0, wall_potential: float = 5.0, dt: float = 1e-7, max_iter: int = 200,
          method: str = "lapack", species: str = "O") -> str:
    """Write the deck files; returns the path of ``system.param``."""
    os.makedirs(directory, exist_ok=True)
    with open(os.path.join(directory, "mesh.dat"), "w") as f:
        f.write(f"{deck.n_nodes} {deck.n_tets}\n")
        lines = [f"{i + 1} {_fmt(x)} {_fmt(y)} {_fmt(z)}" for i, (x, y, z) in enumerate(deck.nodes_mm)]
        f.write("\n".join(lines) + "\n")
        lines = [f"{e + 1} 304 {t[0] + 1} {t[1] + 1} {t[2] + 1} {t[3] + 1}" for e, t in enumerate(deck.tets)]
        f.write("\n".join(lines) + "\n")
    _write_surface(os.path.join(directory, "inlet.dat"), deck, deck.inlet_nodes, deck.inlet_tris)
    _write_surface(os.path.join(directory, "wall.dat"), deck, deck.wall_nodes, deck.wall_tris)
    if deck.sphere_nodes.size:
        _write_surface(os.path.join(directory, "sphere.dat"), deck, deck.sphere_nodes,
                       np.zeros((0, 3), dtype=np.int32))
    params = dict(plasma_den=plasma_den, ion_velocity=ion_velocity,
                  electron_temperature=kTe_eV / KB_EV, wall_potential=wall_potential,
                  max_iter=max_iter, dt=dt)
    with open(os.path.join(directory, "system.param"), "w") as f:
        f.write("# Kuhn box deck\n")
        for k, v in params.items():
            f.write(f"{k} = {_fmt(v) if isinstance(v, float) else v}\n")
        f.write(f"plasma_species = {species}\n")
        f.write(f"fesolver_method = {method}\n")
        f.write("global_mesh = mesh.dat\ninlet_mesh = inlet.dat\nwall_mesh = wall.dat\n")
        f.write("invert_normals = false\n")
    deck.params = dict(params, species=species, method=method)
    return os.path.join(directory, "system.param")


def locate(deck: KuhnDeck, pos_m: np.ndarray) -> np.ndarray:
    """Tet id containing each point (metres), by the Kuhn construction.

    The hex is floor(x/h); inside it, the Kuhn tet is the one whose axis order
    sorts the fractional coordinates in descending order.  Returns -1 for points
    in removed tets.  Used to seed synthetic particle populations; the kernels
    re-check containment with the barycentric test.
    """
    n = deck.n
    h = deck.length_mm / 1000.0 / n
    f = pos_m / h
    c = np.clip(np.floor(f).astype(np.int64), 0, n - 1)
    fr = f - c
    order = np.argsort(-fr, axis=1, kind="stable")
    perm_lut = {p: i for i, p in enumerate(PERMS)}
    code = order[:, 0] * 9 + order[:, 1] * 3 + order[:, 2]
    lut = -np.ones(27, dtype=np.int64)
    for p, i in perm_lut.items():
        lut[p[0] * 9 + p[1] * 3 + p[2]] = i
    perm = lut[code]
    hexid = c[:, 0] + n * c[:, 1] + n * n * c[:, 2]
    return deck.hexperm_to_tet[hexid * 6 + perm]
