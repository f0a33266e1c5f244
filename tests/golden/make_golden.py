"""Generates the golden fixtures of tests/golden/ by running the reference's own
compiled code (oracle/_ref/libref_oracle.so, built from the reference's
sources by oracle/Makefile) on small Kuhn decks.

    python tests/golden/make_golden.py

Writes golden_kuhn4.npz (+ its deck under kuhn4/) and golden_kuhn4s.npz (a
4^3 box with a sphere cut, + kuhn4s/): mesh geometry, FE setup, 10 steps of
InjectIons + MoveParticles with the particle state and density after each, and
per step one Newton step (Lapack method on even steps, GaussSeidel on odd) with
d, uh and ef.  The reference's E field is fed back each step (open loop).
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "mini-fem-pic-main_b200"))
sys.path.insert(0, ROOT)

from minipic_b200 import kuhn  # noqa: E402
from oracle import ref  # noqa: E402

STEPS = 10


def make(name, n, sphere=None, dt=2e-6, spwt=20000.0):
    kd = kuhn.build(n, sphere=sphere)
    deck_dir = os.path.join(HERE, name)
    kuhn.write(kd, deck_dir, dt=dt, max_iter=STEPS, method="lapack")
    extra = {}
    if kd.sphere_nodes.size:
        extra = {os.path.join(deck_dir, "sphere.dat"): (kd.sphere_nodes, -10.0)}
    s = ref.RefSim(deck_dir, spwt=spwt, extra_fixed=extra)
    out = {}
    t = s.tetra()
    for f in ("con", "volume", "alpha", "beta", "gamma", "delta", "cell_con"):
        out["tet_" + f] = t[f]
    pos, typ, vol = s.nodes()
    out.update(node_pos=pos, node_type=typ, node_volume=vol)
    for k, v in s.inlet().items():
        out["inlet_" + k] = v
    fe = s.fe()
    out.update(ID=fe["ID"], LM=fe["LM"], NX=fe["NX"], detJ=fe["detJ"], K=s.matrix(0), F0=s.get("F0"), g=s.get("g"))
    out.update(q_over_m=s.q_over_m, dt=s.dt, spwt=s.spwt, n0=s.param(6), phi0=s.param(7), kTe=s.param(5))
    counts = []
    for ts in range(STEPS):
        k = s.inject()
        out[f"s{ts}_ef_in"] = s.get("ef")
        out[f"s{ts}_injected"] = s.particles()[-k:] if k else s.particles()[:0]
        s.move(1)
        p = s.particles()
        out[f"s{ts}_pos"] = p["pos"]
        out[f"s{ts}_vel"] = p["vel"]
        if ts == STEPS - 1:
            out[f"s{ts}_lc"] = p["lc"]
        out[f"s{ts}_cell"] = p["cell_index"]
        out[f"s{ts}_den"] = s.get("den")
        out[f"s{ts}_F1_in"] = s.get("F1")
        out[f"s{ts}_d_in"] = s.get("d")
        method = ref.LAPACK if ts % 2 == 0 else ref.GAUSS_SEIDEL
        s.compute_phi(method)
        s.update_ef()
        out[f"s{ts}_method"] = method
        out[f"s{ts}_d"] = s.get("d")
        out[f"s{ts}_F1"] = s.get("F1")
        out[f"s{ts}_uh"] = s.get("uh")
        out[f"s{ts}_ef"] = s.get("ef")
        counts.append(len(p))
    out["counts"] = np.array(counts)
    np.savez_compressed(os.path.join(HERE, f"golden_{name}.npz"), **out)
    s.close()
    print(name, "particles per step:", counts)


if __name__ == "__main__":
    make("kuhn4", 4)
    make("kuhn4s", 4, sphere=(50.0, 50.0, 50.0, 22.0))
