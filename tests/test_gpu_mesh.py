"""GPU: mesh setup on the device (mp_mesh_geometry_device, mp_inlet_faces_device,
mp_fe_geometry_device) against the reference's own LoadVolumeMesh /
LoadSurfaceMesh / FESolver output (golden vectors from its compiled code) and
against the host helpers, bit for bit:
  - the golden decks (Kuhn 4^3 box, with and without the sphere cavity);
  - an irregular mesh: node positions jittered, tets shuffled, each tet's
    vertices in a random order (about half of them negatively oriented, so
    the orientation fix runs);
  - a 48^3 box minus the sphere (641,304 tets);
and the error cases the reference exits on (a face held by three tets, an
inlet face held by no tet) plus an out-of-range node index."""
from __future__ import annotations

import os
import tempfile

import numpy as np
import pytest

from conftest import GOLDEN
import minipic_b200 as mp
from minipic_b200 import kuhn

pytestmark = pytest.mark.gpu

GEOM = ("con", "volume", "alpha", "beta", "gamma", "delta", "cell_con", "node_volume", "node_type",
        "inlet_cell", "inlet_u", "inlet_v", "inlet_normal", "inlet_area")


def same_mesh(a: mp.Mesh, b: mp.Mesh):
    for f in GEOM:
        assert np.array_equal(getattr(a, f), getattr(b, f)), f
    for x, y in zip(a.fe_geometry(), b.fe_geometry(device=0)):
        assert np.array_equal(np.asarray(x), np.asarray(y))


@pytest.mark.parametrize("name", ["kuhn4", "kuhn4s"])
def test_device_geometry_matches_reference_bitwise(name):
    g = dict(np.load(os.path.join(GOLDEN, f"golden_{name}.npz"), allow_pickle=False))
    m = mp.Deck.load(os.path.join(GOLDEN, name), device=0).mesh
    for f in ("con", "volume", "alpha", "beta", "gamma", "delta", "cell_con"):
        assert np.array_equal(getattr(m, f), g["tet_" + f]), f
    assert np.array_equal(m.node_volume, g["node_volume"])
    assert np.array_equal(m.node_type, g["node_type"])
    for f, k in (("inlet_cell", "inlet_cell_con"), ("inlet_u", "inlet_u"), ("inlet_v", "inlet_v"),
                 ("inlet_normal", "inlet_normal"), ("inlet_area", "inlet_area")):
        assert np.array_equal(getattr(m, f), g[k]), f
    ID, nx, detJ, neq = m.fe_geometry(device=0)
    assert np.array_equal(ID, g["ID"]) and np.array_equal(nx, g["NX"]) and np.array_equal(detJ, g["detJ"])
    assert neq == g["K"].shape[0]


def _irregular(n=10, seed=3):
    kd = kuhn.build(n, sphere=(50.0, 50.0, 50.0, 20.0))
    rng = np.random.default_rng(seed)
    h = kd.length_mm / n / 1000.0
    pos = kd.nodes_mm / 1000.0
    interior = np.all((pos > 1e-9) & (pos < kd.length_mm / 1000.0 - 1e-9), axis=1)
    pos[interior] += rng.uniform(-0.2 * h, 0.2 * h, size=(int(interior.sum()), 3))
    tets = kd.tets[rng.permutation(kd.tets.shape[0])]
    tets = np.take_along_axis(tets, np.argsort(rng.random(tets.shape), axis=1), axis=1)
    return kd, pos, tets


def test_device_geometry_irregular_mesh():
    kd, pos, tets = _irregular()
    args = (pos, tets, kd.inlet_nodes, kd.inlet_tris, np.concatenate([kd.wall_nodes, kd.sphere_nodes]))
    host = mp.Mesh.build(*args)
    dev = mp.Mesh.build(*args, device=0)
    flipped = np.any(host.con != tets.astype(np.int32), axis=1).mean()
    assert 0.3 < flipped < 0.7
    same_mesh(host, dev)


def test_device_geometry_large():
    kd = kuhn.build(48, sphere=(50.0, 50.0, 50.0, 20.0))
    with tempfile.TemporaryDirectory() as d:
        kuhn.write(kd, d)
        host = mp.Deck.load(d).mesh
        dev = mp.Deck.load(d, device=0).mesh
    assert host.n_tets == 641_304
    same_mesh(host, dev)


def test_device_geometry_errors():
    kd = kuhn.build(4)
    L = mp.lib()
    pos = np.ascontiguousarray(kd.nodes_mm / 1000.0)
    nn = pos.shape[0]

    def geom(tets):
        con = np.ascontiguousarray(tets, dtype=np.int32).copy()
        nt = con.shape[0]
        out = [np.zeros(nt), *(np.zeros((nt, 4)) for _ in range(4)), np.zeros((nt, 4), dtype=np.int32),
               np.zeros(nn), np.zeros(nn, dtype=np.int32)]
        return L.mp_mesh_geometry_device(0, nn, mp._p(pos), nt, mp._p(con), *(mp._p(a) for a in out))

    assert geom(kd.tets) == mp.MP_OK
    assert geom(np.concatenate([kd.tets, kd.tets[:1]])) == 1      # faces held by three tets
    bad = kd.tets.copy()
    bad[5, 2] = nn
    assert geom(bad) == 1                                          # node index out of range
    tris = np.array([[0, 1, nn - 1]], dtype=np.int32)               # no tet holds this face
    con = np.ascontiguousarray(kd.tets, dtype=np.int32)
    outs = [np.zeros(1, dtype=np.int32), np.zeros(3), np.zeros(3), np.zeros(3), np.zeros(1)]
    rc = L.mp_inlet_faces_device(0, nn, mp._p(pos), con.shape[0], mp._p(con), 1, mp._p(tris), 0,
                                 *(mp._p(a) for a in outs))
    assert rc == 1
