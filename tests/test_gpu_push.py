"""GPU parity of MoveParticles (push + walk + scatter + removal + normalisation)
through the C ABI, against the reference's own compiled code (oracle/_ref) or,
where that is absent, the C restatement (oracle/oracle.c) pinned to it.

Bar (FP64 form): positions, velocities, cell indices and barycentric weights
bit-identical to the reference's FP64 CPU path on identical seeded injections
in the reference's particle order; node densities within 1e-12 relative
(atomic accumulation order differs).  Open loop: the reference's E field is
fed to both sides each step."""
from __future__ import annotations

import os

import numpy as np
import pytest

from conftest import DEN_RTOL, GOLDEN, den_close as _den_close, gpu_context, ref_available, run_open_loop
import minipic_b200 as mp
from oracle import port

pytestmark = pytest.mark.gpu


@pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built")
def test_push_bitexact_vs_reference_kuhn6(deck6):
    kd, path = deck6
    run_open_loop(path, kd, steps=40, spwt=2000.0)


@pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built")
def test_push_bitexact_vs_reference_sphere(deck6s):
    kd, path = deck6s
    run_open_loop(path, kd, steps=40, spwt=2000.0)


@pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built")
def test_push_bitexact_with_tet_sort(deck6):
    """Re-sorting by tet permutes storage; the ID-ordered download must still be
    the reference's order and values."""
    kd, path = deck6
    run_open_loop(path, kd, steps=30, spwt=2000.0, sort_period=3)


@pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built")
def test_push_fixed_point_scatter(deck6):
    kd, path = deck6
    run_open_loop(path, kd, steps=25, spwt=2000.0, scatter=mp.SCATTER_FIXED, check_every=5)


def test_push_against_golden():
    """The committed golden vectors of the reference (no reference needed)."""
    for name in ("kuhn4", "kuhn4s"):
        g = dict(np.load(os.path.join(GOLDEN, f"golden_{name}.npz")))
        dk = mp.Deck.load(os.path.join(GOLDEN, name))
        ctx = gpu_context(dk, fe=False)
        qm, dt, spwt = float(g["q_over_m"]), float(g["dt"]), float(g["spwt"])
        for ts in range(len(g["counts"])):
            inj = g[f"s{ts}_injected"]
            ctx.fe_set("ef", g[f"s{ts}_ef_in"])
            # injected records already carry the rewind: append as they are
            if inj.size:
                ctx.append(np.ascontiguousarray(inj["pos"]), np.ascontiguousarray(inj["vel"]),
                           np.ascontiguousarray(inj["cell_index"]))
            den = np.zeros(dk.mesh.n_nodes)
            ctx.push(qm, dt, spwt, den_out=den)
            d = ctx.download(mp.ORDER_ID)
            assert np.array_equal(d["pos"], g[f"s{ts}_pos"])
            assert np.array_equal(d["vel"], g[f"s{ts}_vel"])
            assert np.array_equal(d["cell"], g[f"s{ts}_cell"])
            assert _den_close(den, g[f"s{ts}_den"]) < DEN_RTOL
            if f"s{ts}_lc" in g:
                assert np.array_equal(d["lc"], g[f"s{ts}_lc"])


def test_push_against_oracle_port_large(deck8):
    """A larger population (about 150k particles, several hops per step) against
    the C restatement, which the CPU suite pins to the reference."""
    kd, path = deck8
    dk = mp.Deck.load(path)
    ctx = gpu_context(dk, fe=False)
    m = dk.mesh
    rng = np.random.default_rng(7)
    n = 150_000
    pos = rng.uniform(0.0005, 0.0995, size=(n, 3))
    cell = kuhn_locate(kd, pos)
    vel = rng.normal(0, 3e4, size=(n, 3))
    vel[:, 0] += 7e4
    ef = rng.normal(0, 2e3, size=(m.n_tets, 3))
    ctx.fe_set("ef", ef)
    ctx.append(pos, vel, cell)
    parts = port.Particles()
    parts.append(pos, vel, cell)
    qm, dt, spwt = mp.QE / (16 * mp.AMU), 2e-7, 100.0
    for ts in range(6):
        den = np.zeros(m.n_nodes)
        st = ctx.push(qm, dt, spwt, den_out=den)
        den_o, removed, hops, _ = port.move(parts, m, ef, qm, dt, spwt)
        assert st.total_hops == hops
        g = ctx.download(mp.ORDER_ID)
        assert np.array_equal(g["cell"], parts.cell)
        assert np.array_equal(g["pos"], parts.pos)
        assert np.array_equal(g["vel"], parts.vel)
        assert np.array_equal(g["id"], parts.id)
        assert _den_close(den, den_o) < DEN_RTOL


def kuhn_locate(kd, pos):
    from minipic_b200 import kuhn
    return kuhn.locate(kd, pos).astype(np.int32)


def test_push_empty_population(deck4):
    kd, path = deck4
    dk = mp.Deck.load(path)
    ctx = gpu_context(dk, fe=False)
    den = np.full(dk.mesh.n_nodes, 7.0)
    st = ctx.push(1.0, 1e-7, 200.0, den_out=den)
    assert st.n_before == 0 and st.n_after == 0
    assert np.all(den == 0)
    assert ctx.count() == 0


def test_all_particles_leave(deck4):
    """Every particle crosses the wall in one step: all removed, zero density."""
    kd, path = deck4
    dk = mp.Deck.load(path)
    ctx = gpu_context(dk, fe=False)
    n = 5000
    pos = np.column_stack([np.full(n, 0.09), np.linspace(0.01, 0.09, n), np.full(n, 0.05)])
    cell = kuhn_locate(kd, pos)
    vel = np.column_stack([np.full(n, 1e6), np.zeros(n), np.zeros(n)])
    ctx.append(pos, vel, cell)
    den = np.zeros(dk.mesh.n_nodes)
    st = ctx.push(0.0, 1e-7, 1.0, den_out=den)
    assert st.n_after == 0
    assert np.all(den == 0)


def test_walk_limit_reports_error(deck6):
    """A hop limit of 1 with particles that must cross several tets: the call
    returns MP_ERR_WALK_LIMIT (the reference's walk has no bound)."""
    kd, path = deck6
    dk = mp.Deck.load(path)
    ctx = gpu_context(dk, fe=False)
    ctx.set_walk_limit(1)
    pos = np.array([[0.001, 0.05, 0.05]])
    cell = kuhn_locate(kd, pos)
    ctx.append(pos, np.array([[3e5, 0.0, 0.0]]), cell)
    with pytest.raises(mp.MpError) as e:
        ctx.push(0.0, 1e-7, 1.0)
    assert e.value.status == 4
    ctx.set_walk_limit(4096)
    ctx.push(0.0, 1e-7, 1.0)  # the context stays usable


@pytest.mark.parametrize("form", [mp.FP64, mp.MIXED])
def test_walk_limit_absorb_policy(deck6, form):
    """WALK_LIMIT_ABSORB: a walk that reaches the hop limit removes the particle
    (counted in StepStats.lost, not an error); the others are pushed as usual."""
    kd, path = deck6
    dk = mp.Deck.load(path)
    ctx = gpu_context(dk, fe=False)
    if form == mp.MIXED:
        ctx.set_form(mp.MIXED)
    ctx.set_walk_limit(1)
    ctx.set_walk_policy(mp.WALK_LIMIT_ABSORB)
    pos = np.array([[0.001, 0.05, 0.05], [0.05, 0.05, 0.05]])
    cell = kuhn_locate(kd, pos)
    vel = np.array([[3e5, 0.0, 0.0], [0.0, 0.0, 0.0]])  # the first must cross many tets, the second stays
    ctx.append(pos, vel, cell)
    st = ctx.push(0.0, 1e-7, 1.0)
    assert st.lost == 1 and st.n_after == 1
    out = ctx.download(mp.ORDER_ID)
    assert out["cell"].size == 1 and out["cell"][0] == cell[1]


def test_mixed_walk_point_on_shared_face(tmp_path):
    """Mixed form: an ion exactly on the face shared by two Kuhn tets (the
    x - x0 = z - z0 diagonal plane, FP32 offsets with rx == rz).  The
    reference's weight formula puts it slightly outside both tets, so a walk
    on those weights hops between them without end; the mixed form keeps a
    point within 1e-10 of its tet's faces in the tet."""
    from conftest import make_deck
    _, path = make_deck(tmp_path, 20)
    dk = mp.Deck.load(path)
    m = dk.mesh
    a, b = 47012, 47013
    fa, fb = list(m.cell_con[a]).index(b), list(m.cell_con[b]).index(a)
    assert m.con[a, 0] == m.con[b, 0]
    x0 = m.node_pos[m.con[a, 0]]
    r = np.array([0.0029650903306901455, 0.0030226900707930326, 0.0029650903306901455], dtype=np.float32)
    X = x0 + r.astype(np.float64)

    def lam(t):  # src/meshes.h:84-85, every operation rounded on its own
        q = (1.0 / 6.0) * (((m.alpha[t] - X[0] * m.beta[t]) + X[1] * m.gamma[t]) - X[2] * m.delta[t])
        return q / m.volume[t]

    la, lb = lam(a), lam(b)
    assert la[fa] < 0 and lb[fb] < 0 and la.argmin() == fa and lb.argmin() == fb
    ctx = gpu_context(dk, fe=False)
    ctx.set_form(mp.MIXED)
    ctx.append(X[None, :], np.zeros((1, 3)), np.array([a], dtype=np.int32))
    st = ctx.push(0.0, 5e-8, 1.0)
    assert st.n_after == 1 and st.total_hops == 0
    assert ctx.download(mp.ORDER_ID)["cell"][0] == a


def test_append_rejects_bad_cell(deck4):
    kd, path = deck4
    dk = mp.Deck.load(path)
    ctx = gpu_context(dk, fe=False)
    with pytest.raises(mp.MpError):
        ctx.append(np.zeros((1, 3)), np.zeros((1, 3)), np.array([dk.mesh.n_tets + 5], dtype=np.int32))


def test_mixed_form_errors_against_fp64(deck8):
    """Mixed form (FP32 tet-relative particles, FP64 near-face re-test, FP64
    density): density L2 error and the fraction of differing cell assignments
    against the FP64 form on the same seeded run."""
    kd, path = deck8
    dk = mp.Deck.load(path)
    m = dk.mesh
    rng = np.random.default_rng(3)
    n = 200_000
    pos = rng.uniform(0.0005, 0.0995, size=(n, 3))
    cell = kuhn_locate(kd, pos)
    vel = rng.normal(0, 800.0, size=(n, 3))
    vel[:, 0] += 7000.0
    ef = rng.normal(0, 50.0, size=(m.n_tets, 3))
    qm, dt, spwt = mp.QE / (16 * mp.AMU), 1e-7, 100.0
    a = gpu_context(dk, fe=False)
    b = gpu_context(dk, fe=False)
    for c in (a, b):
        c.fe_set("ef", ef)
        c.append(pos, vel, cell)
    b.set_form(mp.MIXED)
    for ts in range(20):
        da, db = np.zeros(m.n_nodes), np.zeros(m.n_nodes)
        a.push(qm, dt, spwt, den_out=da)
        sb = b.push(qm, dt, spwt, den_out=db)
    l2 = np.linalg.norm(db - da) / np.linalg.norm(da)
    ga, gb = a.download(mp.ORDER_ID), b.download(mp.ORDER_ID)
    ids = np.union1d(ga["id"], gb["id"])
    ca = dict(zip(ga["id"], ga["cell"]))
    cb = dict(zip(gb["id"], gb["cell"]))
    differ = sum(1 for i in ids if ca.get(i, -1) != cb.get(i, -1)) / len(ids)
    assert l2 < 1e-5, l2
    assert differ < 1e-4, differ
    common = np.intersect1d(ga["id"], gb["id"])
    ia = np.searchsorted(ga["id"], common)
    ib = np.searchsorted(gb["id"], common)
    # a particle whose cell assignment flipped near a face once got another
    # tet's kick (the field is piecewise constant): allow those few, bound the rest
    dx = np.abs(ga["pos"][ia] - gb["pos"][ib]).max(axis=1)
    assert np.mean(dx > 1e-6) < 1e-3
    assert np.median(dx) < 1e-8
