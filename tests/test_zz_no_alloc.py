"""GPU: the allocation-free push entry point (mp_push_particles_noalloc).

It serves callers that cannot allocate device memory -- code whose GPU memory
is all owned by another allocator or runtime, and latency-critical code where
cudaMalloc is off limits because it can synchronise the whole device.  The
test owns every buffer (allocated here with torch), calls the entry point
through the C ABI twice in a row on the same state, and checks each call
against the context entry point mp_push_scatter on the same particles:
positions, velocities and cells bit-identical, weights bit-identical to the
walk's, density within 1e-12 relative once normalised like MoveParticles.
The same holds when the output buffer is the input buffer.  Records with a
cell index outside the mesh (the reference's removed state, -1, included) are
rejected with MP_ERR_ARG without any out-of-bounds read.
Collected last so a failure here leaves every other test already run."""
from __future__ import annotations

import ctypes as C
import os

import numpy as np
import pytest

from conftest import make_deck
import minipic_b200 as mp
from minipic_b200 import kuhn

pytestmark = pytest.mark.gpu

PARTICLE = np.dtype({"names": ["pos", "vel", "lc", "cell"], "formats": [("<f8", 3), ("<f8", 3), ("<f8", 4), "<i4"],
                     "offsets": [0, 24, 48, 80], "itemsize": 88})
TETRA = np.dtype({"names": ["con", "volume", "alpha", "beta", "gamma", "delta", "cell_con"],
                  "formats": [("<i4", 4), "<f8", ("<f8", 4), ("<f8", 4), ("<f8", 4), ("<f8", 4), ("<i4", 4)],
                  "offsets": [0, 16, 24, 56, 88, 120, 152], "itemsize": 168})


def _dev(torch, arr: np.ndarray):
    return torch.from_numpy(np.frombuffer(np.ascontiguousarray(arr).tobytes(), dtype=np.uint8).copy()).cuda()


@pytest.mark.parametrize("in_place", [False, True], ids=["two_buffers", "in_place"])
def test_noalloc_push_matches_context_push(tmp_path, in_place):
    torch = pytest.importorskip("torch")
    kd, path = make_deck(tmp_path, 8)
    dk = mp.Deck.load(path)
    m = dk.mesh
    rng = np.random.default_rng(11)
    n = 60_000
    pos = rng.uniform(0.0005, 0.0995, size=(n, 3))
    cell = kuhn.locate(kd, pos).astype(np.int32)
    vel = rng.normal(0.0, 3e4, size=(n, 3))
    vel[:, 0] += 7e4
    ef = rng.normal(0.0, 2e3, size=(m.n_tets, 3))
    qm, dt, spwt = mp.QE / (16 * mp.AMU), 2e-7, 100.0

    # the existing entry point
    ctx = mp.Context(m)
    ctx.fe_set("ef", ef)
    ctx.append(pos, vel, cell)

    # caller-owned buffers for the allocation-free one
    parts = np.zeros(n, dtype=PARTICLE)
    parts["pos"], parts["vel"], parts["cell"] = pos, vel, cell
    tet = np.zeros(m.n_tets, dtype=TETRA)
    tet["con"], tet["volume"], tet["cell_con"] = m.con, m.volume, m.cell_con
    tet["alpha"], tet["beta"], tet["gamma"], tet["delta"] = m.alpha, m.beta, m.gamma, m.delta
    d_in = _dev(torch, parts)
    d_out = d_in if in_place else torch.zeros_like(d_in)
    d_tet = _dev(torch, tet)
    d_ef = torch.from_numpy(np.ascontiguousarray(ef)).cuda()
    d_den = torch.zeros(m.n_nodes, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    L = mp.lib()
    stream = torch.cuda.current_stream().cuda_stream
    n_cur = n
    for call in range(2):
        n_out = C.c_int64(-1)
        rc = L.mp_push_particles_noalloc(d_in.data_ptr(), d_out.data_ptr(), n_cur, d_tet.data_ptr(), m.n_tets,
                                         d_ef.data_ptr(), d_den.data_ptr(), m.n_nodes, qm, dt, stream,
                                         C.byref(n_out))
        assert rc == 0, mp.STATUS.get(rc, rc)
        den_ref = np.zeros(m.n_nodes)
        st = ctx.push(qm, dt, spwt, den_out=den_ref)
        assert n_out.value == st.n_after
        got = np.frombuffer(d_out.cpu().numpy().tobytes(), dtype=PARTICLE)[: n_out.value]
        ref = ctx.download(mp.ORDER_ID)
        assert np.array_equal(got["cell"], ref["cell"])
        assert np.array_equal(got["pos"], ref["pos"])
        assert np.array_equal(got["vel"], ref["vel"])
        assert np.array_equal(got["lc"], ref["lc"])
        den = d_den.cpu().numpy() * (spwt / m.node_volume)
        assert np.abs(den - den_ref).max() <= 1e-12 * np.abs(den_ref).max()
        d_in, d_out = d_out, d_in
        n_cur = n_out.value
    assert n_cur < n  # some particles left the box over the two calls


def test_noalloc_rejects_oversize(tmp_path):
    torch = pytest.importorskip("torch")
    kd, path = make_deck(tmp_path, 4)
    m = mp.Deck.load(path).mesh
    buf = torch.zeros(1024, dtype=torch.uint8, device="cuda")
    den = torch.zeros(m.n_nodes, dtype=torch.float64, device="cuda")
    n_out = C.c_int64(-1)
    rc = mp.lib().mp_push_particles_noalloc(buf.data_ptr(), buf.data_ptr(), 8388609, buf.data_ptr(), m.n_tets,
                                            buf.data_ptr(), den.data_ptr(), m.n_nodes, 1.0, 1e-7, None,
                                            C.byref(n_out))
    assert rc == 10  # MP_ERR_LIMIT
    assert n_out.value == -1


def test_noalloc_rejects_cells_outside_the_mesh(tmp_path):
    """One valid record between a record flagged for removal (cell -1, the
    reference's state before std::erase_if) and one past the last tet: the call
    returns MP_ERR_ARG, the two bad records come out as they went in, and the
    density holds the valid particle's weights only."""
    torch = pytest.importorskip("torch")
    kd, path = make_deck(tmp_path, 4)
    m = mp.Deck.load(path).mesh
    pos = np.array([[0.03, 0.04, 0.05], [0.05, 0.05, 0.05], [0.06, 0.02, 0.07]])
    cell = kuhn.locate(kd, pos).astype(np.int32)
    cell[0], cell[2] = -1, m.n_tets
    vel = np.array([[7e3, 0.0, 0.0], [7e3, 1e2, -1e2], [7e3, 0.0, 0.0]])
    parts = np.zeros(3, dtype=PARTICLE)
    parts["pos"], parts["vel"], parts["cell"] = pos, vel, cell
    parts["lc"] = 0.25
    tet = np.zeros(m.n_tets, dtype=TETRA)
    tet["con"], tet["volume"], tet["cell_con"] = m.con, m.volume, m.cell_con
    tet["alpha"], tet["beta"], tet["gamma"], tet["delta"] = m.alpha, m.beta, m.gamma, m.delta
    d_in = _dev(torch, parts)
    d_out = torch.zeros_like(d_in)
    d_tet = _dev(torch, tet)
    d_ef = torch.zeros(3 * m.n_tets, dtype=torch.float64, device="cuda")
    d_den = torch.zeros(m.n_nodes, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    n_out = C.c_int64(-1)
    rc = mp.lib().mp_push_particles_noalloc(d_in.data_ptr(), d_out.data_ptr(), 3, d_tet.data_ptr(), m.n_tets,
                                            d_ef.data_ptr(), d_den.data_ptr(), m.n_nodes, 1.0, 1e-7,
                                            torch.cuda.current_stream().cuda_stream, C.byref(n_out))
    assert rc == 1  # MP_ERR_ARG
    assert n_out.value == 3
    got = np.frombuffer(d_out.cpu().numpy().tobytes(), dtype=PARTICLE)
    for k in (0, 2):
        assert got[k]["cell"] == cell[k]
        assert np.array_equal(got[k]["pos"], pos[k]) and np.array_equal(got[k]["vel"], vel[k])
    assert got[1]["cell"] >= 0
    den = d_den.cpu().numpy()
    assert abs(den.sum() - 1.0) < 1e-12  # the valid particle's four weights
    assert np.count_nonzero(den) <= 4
