"""Synthetic workloads of the benchmark configurations, and single-kernel
drivers for profiling them.

Configurations (Kuhn box 0.1 m, O+ ions, n0 = 1e10 m^-3, 7 km/s drift,
kTe = 2 eV, inlet x=0 at 0 V, wall x=0.1 at -5 V):
  0  8^3 hexes (3,072 tets), ~50k ions, dt 1e-7, spwt 200
  1  20^3 hexes (48,000 tets), ~2M ions, dt 5e-8, spwt 5
  2  32^3 hexes minus a centred r=0.02 m sphere at -10 V, ~50M ions, dt 5e-8
  3  16^3 hexes (24,576 tets), ~1M ions, adjoint over K=20 steps, checkpoints every 5
  4  40^3 hexes minus the sphere (371,004 tets, 62,788 unknowns), ~193M ions, spwt 0.05,
     re-sort every 10 steps, adjoint over K=10 steps (the combined-stress workload, stress.py)
The ion population is seeded at steady state: uniform in the box, drift plus
a 0.1 eV Maxwellian (sigma = sqrt(kTi*QE/m) ~ 776 m/s), each ion in the Kuhn
tet that contains it.

    python workloads.py push   --config 1 --steps 4 [--form mixed] [--sort 10]
    python workloads.py newton --config 0 --steps 2 [--form mixed] [--mixed-factor tf32]

The drivers print one JSON line per run with the device times measured by
CUDA events inside the library (push kernel; Newton step).
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import tempfile

import numpy as np

if __package__ in (None, ""):
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import minipic_b200 as mp  # noqa: E402
    from minipic_b200 import kuhn  # noqa: E402
else:
    from . import kuhn
    import minipic_b200 as mp

CONFIGS = {
    0: dict(n=8, n_ions=50_000, dt=1e-7, spwt=200.0, sphere=None, label="kuhn8_50k_fp64"),
    1: dict(n=20, n_ions=2_000_000, dt=5e-8, spwt=5.0, sphere=None, label="kuhn20_2M_fp64"),
    2: dict(n=32, n_ions=50_000_000, dt=5e-8, spwt=0.2, sphere=(50.0, 50.0, 50.0, 20.0), label="kuhn32s_50M_mixed"),
    3: dict(n=16, n_ions=1_000_000, dt=1e-7, spwt=5.0, sphere=None, label="kuhn16_1M_adjoint_K20",
            adjoint_steps=20, checkpoint_every=5),
    4: dict(n=40, n_ions=200_000_000, dt=5e-8, spwt=0.05, sphere=(50.0, 50.0, 50.0, 20.0),
            label="kuhn40s_200M_stress", adjoint_steps=10, checkpoint_every=5, sort_period=10),
}
KTI_EV = 0.1
SPHERE_POTENTIAL = -10.0


def write_deck(cfg: dict, workdir: str):
    """The configuration's Kuhn deck in the reference's own file format (numpy
    only; no library call).  Returns the Kuhn deck."""
    kd = kuhn.build(cfg["n"], sphere=cfg["sphere"])
    kuhn.write(kd, workdir, dt=cfg["dt"], method="lapack")
    return kd


def seed_population(kd, cfg: dict, seed: int, n_ions: int | None = None):
    """The steady-state ion population (numpy only): uniform in the box, the
    7 km/s drift along +x plus a 0.1 eV Maxwellian, each ion in the Kuhn tet
    that contains it; ions that fall in the removed sphere are dropped.
    Returns (pos, vel, cell)."""
    rng = np.random.default_rng(seed)
    n = cfg["n_ions"] if n_ions is None else n_ions
    L = kd.length_mm / 1000.0
    pos = rng.uniform(1e-6 * L, (1 - 1e-6) * L, size=(n, 3))
    sigma = np.sqrt(KTI_EV * mp.QE / (16 * mp.AMU))
    vel = rng.normal(0.0, sigma, size=(n, 3))
    vel[:, 0] += float(kd.params["ion_velocity"])
    cell = kuhn.locate(kd, pos).astype(np.int32)
    keep = cell >= 0
    if keep.all():
        return pos, vel, cell
    return np.ascontiguousarray(pos[keep]), np.ascontiguousarray(vel[keep]), cell[keep]


def make_workload(cfg: dict, workdir: str, seed: int, n_ions: int | None = None):
    """Writes the deck into workdir, loads it as the reference would, and seeds
    the ion population.  Returns (kuhn deck, Deck, pos, vel, cell)."""
    kd = write_deck(cfg, workdir)
    deck = mp.Deck.load(workdir)
    pos, vel, cell = seed_population(kd, cfg, seed, n_ions)
    return kd, deck, pos, vel, cell


def absorb_cavity_walks(ctx):
    """Sphere workloads: an ion that steps into the cavity lies in no tet and the
    reference's greedy walk can cycle around it; such walks end at 256 hops and
    the ion is absorbed (counted in StepStats.lost)."""
    ctx.set_walk_limit(256)
    ctx.set_walk_policy(mp.WALK_LIMIT_ABSORB)


def fe_arrays(cfg: dict, deck):
    return deck.fe_desc_arrays(SPHERE_POTENTIAL if cfg["sphere"] else None)


def adjoint_phi(mesh, wall_potential: float = -5.0) -> np.ndarray:
    """A smooth node potential for the adjoint workloads: the inlet-to-wall ramp
    (0 V at x=0, wall_potential at x=L) plus a transverse bump of 0.5 V."""
    L = float(mesh.node_pos[:, 0].max())
    x, y, z = (mesh.node_pos[:, d] / L for d in range(3))
    return wall_potential * x + 0.5 * np.sin(np.pi * x) * np.sin(np.pi * y) * np.sin(np.pi * z)


def make_adjoint_case(cfg: dict, workdir: str, seed: int, n_ions: int | None = None, steps: int | None = None):
    """The adjoint workload: the deck, the initial population (first step 0)
    and K steps of the reference injector's inlet samples with a 0.1 eV
    Maxwellian thermal part (injected = 1, first step k).  Returns (deck,
    slots dict of first/inj/pos/vel/cell, K)."""
    kd, deck, pos, vel, cell = make_workload(cfg, workdir, seed, n_ions=n_ions)
    K = steps or cfg.get("adjoint_steps", 20)
    m = deck.mesh
    rng = np.random.default_rng(seed + 1)
    sigma = np.sqrt(KTI_EV * mp.QE / (16 * mp.AMU))
    inj = mp.Injector(m, seed=0)
    P = deck.params
    firsts, injs, ps, vs, cs = [np.zeros(len(cell), np.int32)], [np.zeros(len(cell), np.uint8)], [pos], [vel], [cell]
    for k in range(K):
        p, _, c = inj.sample(P.plasma_den, P.ion_velocity, cfg["dt"], cfg["spwt"])
        firsts.append(np.full(len(c), k, np.int32))
        injs.append(np.ones(len(c), np.uint8))
        ps.append(p)
        vs.append(rng.normal(0.0, sigma, size=(len(c), 3)))
        cs.append(c.astype(np.int32))
    slots = {"first": np.concatenate(firsts), "inj": np.concatenate(injs), "pos": np.concatenate(ps),
             "vel": np.concatenate(vs), "cell": np.concatenate(cs)}
    return deck, slots, K


def load_adjoint(adj, slots):
    """Adds the slots to an Adjoint, grouped by (first step, injected)."""
    keys = slots["first"].astype(np.int64) * 2 + slots["inj"]
    for key in np.unique(keys):
        sel = keys == key
        adj.add_particles(int(key // 2), bool(key % 2), slots["pos"][sel], slots["vel"][sel], slots["cell"][sel])


def push_driver(args):
    cfg = CONFIGS[args.config]
    with tempfile.TemporaryDirectory() as wd:
        kd, deck, pos, vel, cell = make_workload(cfg, wd, seed=1234)
        ctx = mp.Context(deck.mesh)
        if cfg["sphere"]:
            absorb_cavity_walks(ctx)
        ctx.set_track_ids(False)
        ctx.set_sort_period(args.sort)
        ctx.reserve(len(cell) + 1024)
        ctx.append(pos, vel, cell)
        if args.sort:
            ctx.sort_by_tet()
        if args.form == "mixed":
            ctx.set_form(mp.MIXED)
        rng = np.random.default_rng(5)
        ctx.fe_set("ef", rng.normal(0.0, 20.0, size=(deck.mesh.n_tets, 3)))
        qm = mp.QE / (16 * mp.AMU)
        bpp = 52.0 if args.form == "fp64" else 28.0
        out = []
        for k in range(args.steps):
            st = ctx.push(qm, cfg["dt"], cfg["spwt"])
            gbs = (st.n_before + st.n_after) * bpp / (st.ms_kernel * 1e-3) / 1e9
            out.append({"step": k, "n": st.n_before, "push_kernel_ms": st.ms_kernel, "push_call_ms": st.ms_step,
                        "alg_GBps": gbs, "hops": st.total_hops})
        print(json.dumps({"driver": "push", "config": cfg["label"], "form": args.form, "sort": args.sort,
                          "steps": out}))
        ctx.close()


METHODS = {"lapack": mp.LAPACK, "sparse_cg": mp.SPARSE_CG, "sparse_newton": mp.SPARSE_NEWTON,
           "gs": mp.GAUSS_SEIDEL, "nonlinear": mp.NONLINEAR}


def newton_driver(args):
    cfg = dict(CONFIGS[args.config])
    if args.n:
        cfg["n"] = args.n
    form = mp.MIXED if args.form == "mixed" else mp.FP64
    with tempfile.TemporaryDirectory() as wd:
        kd, deck, pos, vel, cell = make_workload(cfg, wd, seed=1234, n_ions=min(cfg["n_ions"], 200_000))
        ctx = mp.Context(deck.mesh)
        if cfg["sphere"]:
            absorb_cavity_walks(ctx)
        ctx.set_mixed_factor({"auto": mp.MIXED_AUTO, "tf32": mp.MIXED_TF32, "fp16": mp.MIXED_FP16,
                              "tf32x3": mp.MIXED_TF32X3}[getattr(args, "mixed_factor", "auto")])
        if getattr(args, "storage", "dense") == "sparse":
            ctx.set_fe_storage(mp.FE_SPARSE)
        ctx.fe_setup(**fe_arrays(cfg, deck))
        ctx.append(pos, vel, cell)
        ctx.push(mp.QE / (16 * mp.AMU), cfg["dt"], cfg["spwt"] * cfg["n_ions"] / len(cell))
        out = []
        if getattr(args, "ktime", False):
            ctx.set_kernel_timing(True)
        for k in range(args.steps):
            st = ctx.compute_phi(METHODS[getattr(args, "method", "lapack")], form)
            out.append({"step": k, "newton_ms": st.ms_total, "factor_ms": st.ms_factor,
                        "newton_iterations": st.newton_iterations, "linear_iterations": st.linear_iterations,
                        "linear_failures": st.linear_failures, "residual": st.linear_residual})
        classes = {name: ctx.kernel_timing(kc) for name, kc in
                   (("update", mp.KT_UPDATE), ("diag", mp.KT_DIAG), ("panel", mp.KT_PANEL), ("trsv", mp.KT_TRSV))
                   } if getattr(args, "ktime", False) else None
        print(json.dumps({"driver": "newton", "config": cfg["label"], "form": args.form,
                          "method": getattr(args, "method", "lapack"), "storage": getattr(args, "storage", "dense"),
                          "mixed_factor": getattr(args, "mixed_factor", "auto"),
                          "unknowns": int(fe_arrays(cfg, deck)["neq"]), "steps": out, "kernel_classes": classes}))
        ctx.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("driver", choices=["push", "newton"])
    ap.add_argument("--config", type=int, default=1, choices=sorted(CONFIGS))
    ap.add_argument("--steps", type=int, default=4)
    ap.add_argument("--form", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--sort", type=int, default=0)
    ap.add_argument("--n", type=int, default=0, help="override the mesh's hexes per side (newton driver)")
    ap.add_argument("--mixed-factor", default="auto", choices=["auto", "tf32", "fp16", "tf32x3"],
                    help="tensor-core arithmetic of the mixed-form factorization (newton driver)")
    ap.add_argument("--method", default="lapack", choices=sorted(METHODS), help="newton driver")
    ap.add_argument("--storage", default="dense", choices=["dense", "sparse"], help="newton driver: storage of K")
    ap.add_argument("--ktime", action="store_true", help="newton driver: CUDA-event times of the kernel classes")
    args = ap.parse_args()
    (push_driver if args.driver == "push" else newton_driver)(args)


if __name__ == "__main__":
    main()
