"""CPU: the oracle (oracle/oracle.c) and the library's host-side setup against
the golden vectors that the reference's own compiled code produced
(tests/golden/make_golden.py).  Pins the oracle without needing the reference."""
from __future__ import annotations

import os

import numpy as np
import pytest

from conftest import GOLDEN, rel_err
import minipic_b200 as mp
from oracle import port

CASES = ["kuhn4", "kuhn4s"]


def load(name):
    return dict(np.load(os.path.join(GOLDEN, f"golden_{name}.npz"), allow_pickle=False))


def deck(name):
    return mp.Deck.load(os.path.join(GOLDEN, name))


@pytest.mark.parametrize("name", CASES)
def test_host_geometry_matches_reference_bitwise(name):
    g = load(name)
    m = deck(name).mesh
    for f in ("con", "volume", "alpha", "beta", "gamma", "delta", "cell_con"):
        assert np.array_equal(getattr(m, f), g["tet_" + f]), f
    assert np.array_equal(m.node_pos, g["node_pos"])
    assert np.array_equal(m.node_volume, g["node_volume"])
    assert np.array_equal(m.node_type, g["node_type"])
    for f, k in (("inlet_con", "inlet_con"), ("inlet_cell", "inlet_cell_con"), ("inlet_u", "inlet_u"),
                 ("inlet_v", "inlet_v"), ("inlet_normal", "inlet_normal"), ("inlet_area", "inlet_area")):
        assert np.array_equal(getattr(m, f), g[k]), f


@pytest.mark.parametrize("name", CASES)
def test_host_fe_geometry_matches_reference_bitwise(name):
    g = load(name)
    ID, nx, detJ, neq = deck(name).mesh.fe_geometry()
    assert np.array_equal(ID, g["ID"])
    assert np.array_equal(nx, g["NX"])
    assert np.array_equal(detJ, g["detJ"])
    assert neq == g["K"].shape[0]


@pytest.mark.parametrize("name", CASES)
def test_oracle_assembly_bitwise(name):
    g = load(name)
    dk = deck(name)
    fa = dk.fe_desc_arrays(sphere_potential=-10.0)
    assert np.array_equal(fa["g"], g["g"])
    fe = port.FE(dk.mesh, **fa)
    assert np.array_equal(fe.K, g["K"])
    assert np.array_equal(fe.F0, g["F0"])


@pytest.mark.parametrize("name", CASES)
def test_oracle_injection_and_push_bitwise(name):
    """InjectIons + MoveParticles open loop: positions, velocities, cells
    bit-identical, density bit-identical (the oracle pushes in the reference's order)."""
    g = load(name)
    dk = deck(name)
    m = dk.mesh
    P = dk.params
    inj = port.Injector(m)
    parts = port.Particles()
    qm, dt, spwt = float(g["q_over_m"]), float(g["dt"]), float(g["spwt"])
    for ts in range(len(g["counts"])):
        ef_in = g[f"s{ts}_ef_in"]
        pos, vel, cell = inj.sample(P.plasma_den, P.ion_velocity, dt, spwt)
        port.rewind(vel, cell, ef_in, qm, 0.5 * dt)
        injected = g[f"s{ts}_injected"]
        assert np.array_equal(pos, injected["pos"]) and np.array_equal(vel, injected["vel"])
        parts.append(pos, vel, cell)
        den, _, _, lc = port.move(parts, m, ef_in, qm, dt, spwt, want_lc=True)
        assert np.array_equal(parts.pos, g[f"s{ts}_pos"])
        assert np.array_equal(parts.vel, g[f"s{ts}_vel"])
        assert np.array_equal(parts.cell, g[f"s{ts}_cell"])
        assert np.array_equal(den, g[f"s{ts}_den"])
        if f"s{ts}_lc" in g:
            assert np.array_equal(lc, g[f"s{ts}_lc"])


@pytest.mark.parametrize("name", CASES)
def test_oracle_newton_step(name):
    """One Newton step per step (Lapack / GaussSeidel alternately) from the
    captured d, F1 and density: F1 accumulation bit-exact, d and E field within
    1e-10 relative (the oracle's dense solve stands in for dsysv_)."""
    g = load(name)
    dk = deck(name)
    fa = dk.fe_desc_arrays(sphere_potential=-10.0)
    fe = port.FE(dk.mesh, **fa)
    for ts in range(len(g["counts"])):
        fe.d = g[f"s{ts}_d_in"].copy()
        fe.F1 = g[f"s{ts}_F1_in"].copy()
        fe.compute_phi(g[f"s{ts}_den"], int(g[f"s{ts}_method"]))
        assert np.array_equal(fe.F1, g[f"s{ts}_F1"])
        tol = 1e-10 if int(g[f"s{ts}_method"]) == 2 else 1e-7
        assert rel_err(fe.d, g[f"s{ts}_d"]) < tol
        assert rel_err(fe.uh, g[f"s{ts}_uh"]) < tol
        assert rel_err(fe.update_ef(), g[f"s{ts}_ef"]) < tol * 10


def test_injector_rng_stream():
    """std::mt19937(0) + uniform_real_distribution<double>: the oracle's
    restatement against the library's host injector (the standard library)."""
    m = deck("kuhn4").mesh
    a = port.Injector(m)
    b = mp.Injector(m)
    for _ in range(5):
        pa = a.sample(1e10, 7000.0, 2e-6, 20000.0)
        pb = b.sample(1e10, 7000.0, 2e-6, 20000.0)
        for x, y in zip(pa, pb):
            assert np.array_equal(x, y)
    assert a.rem.value == b.rem
