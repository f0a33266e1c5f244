"""GPU: contexts are independent.  Every device buffer of a solve or a
transfer belongs to its context (the reference's DeviceData owns its own
buffers, src/mini-pic.cpp:322-355), so two contexts driven at the same time
from two host threads -- on meshes with the same and with different numbers
of unknowns -- give exactly what each gives alone.  A step: host-injected ions
appended, MoveParticles with the deterministic fixed-point density, one
Lapack Newton step in FP64 (bit for bit) and in the mixed form (within 1e-12
relative: its refinement stops on reduced norms), updateEf."""
from __future__ import annotations

import threading

import numpy as np
import pytest

from conftest import make_deck
import minipic_b200 as mp
from minipic_b200 import kuhn

pytestmark = pytest.mark.gpu

STEPS = 4


def _case(tmp_path, n, seed):
    kd, path = make_deck(tmp_path / f"k{n}_{seed}", n, dt=1e-7)
    dk = mp.Deck.load(path)
    rng = np.random.default_rng(seed)
    m = 20_000
    pos = rng.uniform(0.001, 0.099, size=(m, 3))
    vel = rng.normal(0.0, 800.0, size=(m, 3))
    vel[:, 0] += 7000.0
    cell = kuhn.locate(kd, pos).astype(np.int32)
    return dk, (pos, vel, cell)


def _run(dk, pop, out):
    ctx = mp.Context(dk.mesh)
    ctx.fe_setup(**dk.fe_desc_arrays())
    ctx.set_scatter_mode(mp.SCATTER_FIXED)
    ctx.append(*pop)
    inj = mp.Injector(dk.mesh)
    P = dk.params
    qm, dt, spwt = mp.QE / (16 * mp.AMU), P.dt, 50.0
    res = []
    for k in range(STEPS):
        p, v, c = inj.sample(P.plasma_den, P.ion_velocity, dt, spwt)
        ctx.append(p, v, c, rewind=True, q_over_m=qm, half_dt=0.5 * dt)
        den = np.zeros(dk.mesh.n_nodes)
        ctx.push(qm, dt, spwt, den_out=den)
        form = mp.FP64 if k % 2 == 0 else mp.MIXED
        ctx.compute_phi(mp.LAPACK, form)
        ctx.update_ef()
        d, uh, ef = ctx.field()
        res.append((form, den, d, uh, ef))
    g = ctx.download(mp.ORDER_ID)
    res.append(g)
    ctx.close()
    out.append(res)


def _same(a, b):
    for (fa, *xa), (fb, *xb) in zip(a[:-1], b[:-1]):
        assert fa == fb
        for u, v in zip(xa, xb):
            if fa == mp.FP64:
                assert np.array_equal(u, v)
            else:
                assert np.abs(u - v).max() <= 1e-12 * max(np.abs(v).max(), 1e-300)
    for key in ("pos", "vel", "cell", "id"):
        assert np.array_equal(a[-1][key], b[-1][key])


@pytest.mark.parametrize("sizes", [(12, 12), (12, 8)], ids=["same_unknowns", "different_unknowns"])
def test_two_contexts_on_two_threads(tmp_path, sizes):
    cases = [_case(tmp_path, n, seed) for seed, n in enumerate(sizes)]
    alone = []
    for dk, pop in cases:
        r = []
        _run(dk, pop, r)
        alone.append(r[0])
    for _ in range(2):
        outs = [[], []]
        th = [threading.Thread(target=_run, args=(dk, pop, outs[i])) for i, (dk, pop) in enumerate(cases)]
        for t in th:
            t.start()
        for t in th:
            t.join()
        for i in range(2):
            assert len(outs[i]) == 1, "a thread failed"
            _same(outs[i][0], alone[i])
