"""CPU, 2 gloo ranks: the sharded step's host logic.  Each rank pushes its
share of one seeded population (the C restatement stands in for the device
push), the node density is summed over ranks, and the result must equal the
single-process push of the whole population: same density within 1e-12
relative, same number of kept particles, and the shards' survivors
concatenated in rank order equal the single-process survivors."""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest

from conftest import GOLDEN, ROOT

WORLD = 2


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _population(m, kd_n=4, n=4000, seed=3):
    import minipic_b200 as mp
    rng = np.random.default_rng(seed)
    # points inside tets, taken as random barycentric combinations of the vertices
    t = rng.integers(0, m.n_tets, size=n)
    w = rng.dirichlet(np.ones(4), size=n)
    pos = np.einsum("nk,nkd->nd", w, m.node_pos[m.con[t]])
    vel = rng.normal(0, 2e4, size=(n, 3))
    vel[:, 0] += 5e4
    return np.ascontiguousarray(pos), np.ascontiguousarray(vel), t.astype(np.int32)


def _rank_main(rank, port, out_path):
    import sys
    sys.path.insert(0, os.path.join(ROOT, "mini-fem-pic-main_b200"))
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    import minipic_b200 as mp
    from minipic_b200 import sharding
    from oracle import port as oport

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=WORLD)
    dk = mp.Deck.load(os.path.join(GOLDEN, "kuhn4"))
    m = dk.mesh
    pos, vel, cell = _population(m)
    sl = sharding.shard_range(len(cell), rank, WORLD)
    parts = oport.Particles()
    parts.append(pos[sl], vel[sl], cell[sl])
    ef = np.zeros((m.n_tets, 3))
    qm, dt, spwt = 6.0e6, 2e-7, 100.0
    den, _, _, _ = oport.move(parts, m, ef, qm, dt, spwt)
    den = sharding.allreduce_density_host(den)
    import torch
    kept = torch.tensor([parts.cell.size], dtype=torch.int64)
    dist.all_reduce(kept)
    np.savez(out_path + f".{rank}.npz", den=den, kept=kept.numpy(), pos=parts.pos, cell=parts.cell)
    dist.barrier()
    dist.destroy_process_group()


def test_sharded_density_equals_single_process(tmp_path):
    torch = pytest.importorskip("torch")
    import torch.multiprocessing as tmp
    import minipic_b200 as mp
    from oracle import port as oport

    port = _free_port()
    out = str(tmp_path / "res")
    tmp.spawn(_rank_main, args=(port, out), nprocs=WORLD, join=True)
    dk = mp.Deck.load(os.path.join(GOLDEN, "kuhn4"))
    m = dk.mesh
    pos, vel, cell = _population(m)
    parts = oport.Particles()
    parts.append(pos, vel, cell)
    den1, _, _, _ = oport.move(parts, m, np.zeros((m.n_tets, 3)), 6.0e6, 2e-7, 100.0)
    r = [np.load(out + f".{k}.npz") for k in range(WORLD)]
    for k in range(WORLD):
        assert np.abs(r[k]["den"] - den1).max() <= 1e-12 * np.abs(den1).max()
        assert int(r[k]["kept"][0]) == parts.cell.size
    assert np.array_equal(np.concatenate([r[k]["cell"] for k in range(WORLD)]), parts.cell)
    assert np.array_equal(np.concatenate([r[k]["pos"] for k in range(WORLD)]), parts.pos)


def test_shard_range_partitions():
    from minipic_b200 import sharding
    for n in (0, 1, 7, 100, 1001):
        for w in (1, 2, 3, 8):
            sl = [sharding.shard_range(n, r, w) for r in range(w)]
            assert sl[0].start == 0 and sl[-1].stop == n
            assert all(sl[i].stop == sl[i + 1].start for i in range(w - 1))
            sizes = [s.stop - s.start for s in sl]
            assert max(sizes) - min(sizes) <= 1
