"""Shared fixtures.  CPU tests (-m "not gpu") check the oracle against the
committed golden vectors and the reference's own compiled code, the host-side
setup, and that the C ABI library loads and exports every declared symbol.
GPU tests (-m gpu) are the parity tests of the CUDA path through the C ABI."""
from __future__ import annotations

import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "mini-fem-pic-main_b200"))
sys.path.insert(0, ROOT)

import minipic_b200 as mp  # noqa: E402
from minipic_b200 import kuhn  # noqa: E402

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 GPU (B200); calls the CUDA path through the C ABI")


def make_deck(tmp_root, n, sphere=None, **kw):
    d = kuhn.build(n, sphere=sphere)
    path = os.path.join(str(tmp_root), f"kuhn{n}{'s' if sphere else ''}")
    kuhn.write(d, path, **kw)
    return d, path


@pytest.fixture(scope="session")
def deck4(tmp_path_factory):
    return make_deck(tmp_path_factory.mktemp("d4"), 4)


@pytest.fixture(scope="session")
def deck6(tmp_path_factory):
    return make_deck(tmp_path_factory.mktemp("d6"), 6)


@pytest.fixture(scope="session")
def deck8(tmp_path_factory):
    return make_deck(tmp_path_factory.mktemp("d8"), 8)


@pytest.fixture(scope="session")
def deck6s(tmp_path_factory):
    return make_deck(tmp_path_factory.mktemp("d6s"), 6, sphere=(50.0, 50.0, 50.0, 20.0))


def ref_available():
    from oracle import ref
    return ref.available()


def ref_sim(path, kdeck, **kw):
    """The reference's own simulation on a deck (sphere nodes at -10 V)."""
    from oracle import ref
    extra = {}
    if kdeck.sphere_nodes.size:
        extra = {os.path.join(path, "sphere.dat"): (kdeck.sphere_nodes, -10.0)}
    return ref.RefSim(path, extra_fixed=extra, **kw)


def gpu_context(deck: "mp.Deck", sphere_potential=None, fe=True):
    ctx = mp.Context(deck.mesh)
    if fe:
        ctx.fe_setup(**deck.fe_desc_arrays(sphere_potential))
    return ctx


def rel_err(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = max(np.abs(b).max(), 1e-300)
    return float(np.abs(a - b).max() / den)


DEN_RTOL = 1e-12


def den_close(a, b):
    scale = max(np.abs(b).max(), 1e-300)
    return float(np.abs(a - b).max() / scale)


def run_open_loop(path, kdeck, steps, spwt, *, sort_period=0, scatter=0, method=2, check_every=1,
                  initial=None, threads=1, sort_first=False):
    """MoveParticles of the CUDA path against the reference's own (oracle/_ref),
    open loop: both sides push the same particles in the reference's E field,
    which the reference solves after each step (FESolver method `method`) and
    which is fed to the device each step.  Each step the reference's injector
    and the library's host injector give the same ions.  initial = (pos, vel,
    cell) seeds both sides with a population first.  Checked every
    `check_every` steps and at the last: cells, positions, velocities and
    weights bit-identical in the reference's order, node density within
    DEN_RTOL every step."""
    dk = mp.Deck.load(path)
    s = ref_sim(path, kdeck, spwt=spwt)
    ctx = gpu_context(dk, sphere_potential=-10.0, fe=False)
    ctx.set_sort_period(sort_period)
    ctx.set_scatter_mode(scatter)
    if initial is not None:
        from oracle import ref
        pos, vel, cell = initial
        parts = np.zeros(len(cell), dtype=ref.PARTICLE_DTYPE)
        parts["pos"], parts["vel"], parts["cell_index"] = pos, vel, cell
        s.set_particles(parts)
        ctx.reserve(int(len(cell) * 1.2) + 100_000)
        ctx.append(pos, vel, cell)
        if sort_first:
            ctx.sort_by_tet()
    inj = mp.Injector(dk.mesh)
    P = dk.params
    qm, dt = s.q_over_m, P.dt
    worst = 0.0
    for ts in range(steps):
        k = s.inject()
        pos, vel, cell = inj.sample(P.plasma_den, P.ion_velocity, dt, spwt)
        assert len(cell) == k
        ctx.append(pos, vel, cell, rewind=True, q_over_m=qm, half_dt=0.5 * dt)
        s.move(threads)
        den = np.zeros(dk.mesh.n_nodes)
        st = ctx.push(qm, dt, spwt, den_out=den)
        rp = s.particles()
        assert st.n_after == len(rp)
        if ts % check_every == 0 or ts == steps - 1:
            g = ctx.download(mp.ORDER_ID)
            assert np.array_equal(g["cell"], rp["cell_index"]), f"cell mismatch at step {ts}"
            assert np.array_equal(g["pos"], rp["pos"]), f"pos mismatch at step {ts}"
            assert np.array_equal(g["vel"], rp["vel"]), f"vel mismatch at step {ts}"
            assert np.array_equal(g["lc"], rp["lc"]), f"lc mismatch at step {ts}"
            assert np.all(np.diff(g["id"]) > 0)
        e = den_close(den, s.get("den"))
        worst = max(worst, e)
        assert e < DEN_RTOL, f"density rel error {e} at step {ts}"
        s.compute_phi(method)
        s.update_ef()
        ctx.fe_set("ef", s.get("ef"))
    return worst, s, ctx
