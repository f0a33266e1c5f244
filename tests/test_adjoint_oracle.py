"""CPU: the dual-number build of the push (oracle/dual.cpp), which checks the
adjoint, pinned to the reference itself.

1. Its value part equals the reference's own compiled MoveParticles
   (oracle/_ref) bit for bit over K steps with phi held: node density after
   the last step, survivors' positions, velocities and cells.
2. Its tangent part equals central finite differences of its value part,
   with no cell or exit changing between the +h and -h runs.
"""
from __future__ import annotations

import numpy as np
import pytest

import minipic_b200 as mp
from minipic_b200 import adjoint, workloads
from oracle import port, ref

SMALL = dict(n=4, n_ions=3000, dt=1e-7, spwt=100.0, sphere=None, label="kuhn4_adjoint")
MASS = 16 * mp.AMU


def _case(tmp_path, steps=6, seed=7):
    deck, slots, K = workloads.make_adjoint_case(SMALL, str(tmp_path), seed=seed, steps=steps)
    nx = deck.fe_desc_arrays()["nx"]
    return deck, slots, K, nx


@pytest.mark.skipif(not (ref.available() and port.dual_available()), reason="oracle libraries not built")
def test_dual_value_equals_reference_push(tmp_path):
    deck, slots, K, nx = _case(tmp_path)
    m = deck.mesh
    sim = ref.RefSim(str(tmp_path), spwt=SMALL["spwt"])
    phi = workloads.adjoint_phi(m)
    sim.set("uh", phi)
    sim.update_ef()
    ef = sim.get("ef")
    qm, dt, vd = sim.q_over_m, SMALL["dt"], deck.params.ion_velocity
    dirn = m.inlet_normal[0]
    assert np.allclose(m.inlet_normal, dirn)
    parts = np.zeros(0, dtype=ref.PARTICLE_DTYPE)
    for k in range(K):
        for inj in (0, 1):
            sel = (slots["first"] == k) & (slots["inj"] == inj)
            if not sel.any():
                continue
            new = np.zeros(int(sel.sum()), dtype=ref.PARTICLE_DTYPE)
            new["pos"] = slots["pos"][sel]
            c = slots["cell"][sel]
            v = slots["vel"][sel].copy()
            if inj:
                # InjectIons: vel = normal*ion_velocity (+ thermal part); vel -= charge/mass*ef*(0.5*dt)
                v = dirn[None, :] * vd + v
                v = v - (qm * ef[c]) * (0.5 * dt)
            new["vel"], new["cell_index"] = v, c
            parts = np.concatenate([sim.particles(), new])
            sim.set_particles(parts)
        sim.move(1)
    den_ref = sim.get("den")
    surv = sim.particles()
    out = port.dual_ksteps(m, nx, adjoint.wall_nodes_of(m), slots, K, qm, MASS, dt, SMALL["spwt"], dirn, phi, vd)
    alive = out["kind"] == 0
    assert surv.size == int(alive.sum()) and surv.size > 100
    assert np.array_equal(out["den"], den_ref)
    assert np.array_equal(out["pos"][alive], surv["pos"])
    assert np.array_equal(out["vel"][alive], surv["vel"])
    assert np.array_equal(out["cell"][alive], surv["cell_index"])
    assert (out["kind"] == 1).sum() + (out["kind"] == 2).sum() > 0  # some exits happened


@pytest.mark.skipif(not port.dual_available(), reason="oracle/libdual.so not built")
def test_dual_tangent_equals_central_differences(tmp_path):
    deck, slots, K, nx = _case(tmp_path, steps=8, seed=11)
    m = deck.mesh
    wall = adjoint.wall_nodes_of(m)
    qm, dt, vd = mp.QE / MASS, SMALL["dt"], deck.params.ion_velocity
    dirn = m.inlet_normal[0]
    phi = workloads.adjoint_phi(m)
    rng = np.random.default_rng(3)
    args = (m, nx, wall, slots, K, qm, MASS, dt, SMALL["spwt"], dirn)
    base = port.dual_ksteps(*args, phi, vd)
    checked = 0
    for trial in range(6):
        u = rng.normal(size=m.n_nodes)
        dvd = float(rng.normal()) * 10.0
        t = port.dual_ksteps(*args, phi, vd, dphi=u, dvd=dvd)
        h = 1e-4 * np.abs(phi).max() / np.abs(u).max()  # central differences at h = 1e-4 relative
        p = port.dual_ksteps(*args, phi + h * u, vd + h * dvd)
        q = port.dual_ksteps(*args, phi - h * u, vd - h * dvd)
        flips = sum(int((r["kind"] != base["kind"]).sum() + (r["path"] != base["path"]).sum()) for r in (p, q))
        if flips:
            continue  # a perturbation moved a cell or an exit: not the piecewise-fixed model
        fd = (p["den"] - q["den"]) / (2 * h)
        assert np.abs(fd - t["dden"]).max() <= 1e-6 * np.abs(t["dden"]).max()
        fdf = (p["flux"] - q["flux"]) / (2 * h)
        assert abs(fdf - t["dflux"]) <= 1e-6 * max(abs(t["dflux"]), 1e-300)
        checked += 1
    assert checked >= 2
