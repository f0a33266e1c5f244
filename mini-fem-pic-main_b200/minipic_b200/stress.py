"""The combined-stress workload on one GPU: the 40^3-hex Kuhn box minus the
centred r = 0.02 m sphere held at -10 V (371,004 tets, 67,298 nodes, 62,788
unknowns; the dense FP64 K is 31.6 GB), about 193M O+ ions (spwt 0.05) with a
tet re-sort every 10 steps, the mixed-precision step (FP32 tet-relative
particles, tcgen05 LDL^T on FP16 operands with FP64 refinement), the adjoint of K = 10
push + scatter steps with checkpoints every 5 on the whole population, and the
FP64 form of the same steps beside it.

Memory plan (one B200, 180 GB): the mixed run holds K (31.6 GB), its FP32
factor (15.8 GB), the particles (two buffers, 60 B a slot, 24 GB) and then the
adjoint's slots (inputs, two checkpoints and outcomes, about 160 B a slot,
31 GB); the FP64 run afterwards holds K, the FP64 J (31.6 GB) and the particles.
The two never share the device.  The population is generated and appended in
chunks of 16M ions, so the host never holds it whole.

    python bench.py --stress [--steps S --warmup W]
"""
from __future__ import annotations

import tempfile
import time

import numpy as np

import minipic_b200 as mp
from minipic_b200 import kuhn, workloads

CHUNK = 16_000_000


def _chunks(kd, cfg, seed):
    """The seeded population, chunk by chunk (each chunk its own stream)."""
    total = cfg["n_ions"]
    for i, lo in enumerate(range(0, total, CHUNK)):
        n = min(CHUNK, total - lo)
        yield workloads.seed_population(kd, cfg, seed * 1000 + i, n_ions=n)


def _context(deck, fe, form, cfg, kd, device, seed):
    c = mp.Context(deck.mesh, device=device)
    c.fe_setup(**fe)
    c.set_track_ids(False)
    workloads.absorb_cavity_walks(c)
    c.reserve(int(cfg["n_ions"] * 1.02) + 2_000_000)
    n0 = 0
    for pos, vel, cell in _chunks(kd, cfg, seed):
        c.append(pos, vel, cell)
        n0 += len(cell)
    c.sort_by_tet()
    c.set_sort_period(cfg["sort_period"])
    if form == mp.MIXED:
        c.set_form(mp.MIXED)
    return c, n0


def _steps(c, form, cfg, deck, steps, warmup, torch, device, keep):
    P = deck.params
    qm = mp.QE / (16 * mp.AMU)
    sigma = float(np.sqrt(workloads.KTI_EV * mp.QE / (16 * mp.AMU)))
    inj = mp.Injector(deck.mesh, seed=0)
    stream = torch.cuda.ExternalStream(c.stream(), device=device)
    out = {"step_ms": [], "newton_ms": [], "push_ms": [], "n": [], "lost": []}
    for k in range(warmup + steps):
        if k == warmup:
            c.set_kernel_timing(mp.KT_TIMED)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        c.inject_device(inj, P.plasma_den, P.ion_velocity, cfg["dt"], cfg["spwt"], sigma, qm, 1000, k)
        st = c.push(qm, cfg["dt"], cfg["spwt"])
        nt = c.compute_phi(mp.LAPACK, form)
        c.update_ef()
        e1.record(stream)
        e1.synchronize()
        keep.append((c.density(), c.field()[1]))
        if k >= warmup:
            out["step_ms"].append(e0.elapsed_time(e1))
            out["newton_ms"].append(nt.ms_total)
            out["push_ms"].append(st.ms_kernel)
            out["n"].append(st.n_before)
            out["lost"].append(st.lost)
    return out


def _summary(r, c, pk):
    push = c.kernel_timing(mp.KT_PUSH)
    upd = c.kernel_timing(mp.KT_UPDATE)
    gbs = push["work"] / (push["ms"] * 1e-3) / 1e9
    tfs = upd["work"] / (upd["ms"] * 1e-3) / 1e12
    return {"particle_steps_per_s": float(np.sum(r["n"]) / (np.sum(r["step_ms"]) / 1e3)),
            "ms_per_step": float(np.mean(r["step_ms"])), "newton_step_ms": float(np.mean(r["newton_ms"])),
            "push_kernel_ms": float(np.mean(r["push_ms"])), "ions": int(np.mean(r["n"])),
            "absorbed_at_walk_limit_per_step": float(np.mean(r["lost"])),
            "push_hbm": {"achieved_GBps": gbs, "frac": gbs / pk["hbm_gbs"], "peak_kind": pk["kind"]},
            "trailing_update": {"achieved_TFLOPs": tfs, "frac_of_bf16_sustained": tfs / pk["bf16_tflops_sustained"],
                                "launches": upd["launches"], "ms": upd["ms"]}}


def run(args, device, torch, pk):
    cfg = workloads.CONFIGS[4]
    steps, warmup = max(2, args.steps), max(1, min(args.warmup, 3))
    t_all = time.time()
    with tempfile.TemporaryDirectory() as wd:
        kd = workloads.write_deck(cfg, wd)
        deck = mp.Deck.load(wd)
    fe = workloads.fe_arrays(cfg, deck)
    out = {"workload": cfg["label"], "tets": deck.mesh.n_tets, "nodes": deck.mesh.n_nodes,
           "unknowns": int(fe["neq"]), "dense_K_GB": 8 * fe["neq"] * ((fe["neq"] + 31) // 32 * 32) / 1e9}
    # mixed form
    t0 = time.time()
    c, n0 = _context(deck, fe, mp.MIXED, cfg, kd, device, seed=7)
    out["setup_s_mixed"] = time.time() - t0
    out["ions_initial"] = n0
    keep_m = []
    rm = _steps(c, mp.MIXED, cfg, deck, steps, warmup, torch, device, keep_m)
    out["mixed"] = _summary(rm, c, pk)
    out["mixed"]["refined_newton"] = ("tcgen05 LDL^T (FP16-operand trailing updates from %d unknowns, 3xTF32 below), "
                                      "FP64 refinement to ||r|| <= 1e-14 ||G||" % mp.MIXED_FP16_FROM)
    free, total = torch.cuda.mem_get_info(device)
    out["mixed"]["device_memory_used_GB"] = (total - free) / 1e9
    # adjoint of K push + scatter steps over the whole population, phi held at the last step's
    from minipic_b200 import adjoint as adj_mod
    c.set_kernel_timing(False)
    phi = c.field()[1]
    m = deck.mesh
    K, C = cfg["adjoint_steps"], cfg["checkpoint_every"]
    qm = mp.QE / (16 * mp.AMU)
    wall = (m.node_type == mp.NODE_FIXED).astype(np.uint8)
    a = adj_mod.Adjoint(c, K, C, qm, 16 * mp.AMU, cfg["dt"], cfg["spwt"], np.array([1.0, 0.0, 0.0]), wall)
    t0 = time.time()
    n_slots = 0
    for pos, vel, cell in _chunks(kd, cfg, seed=11):
        a.add_particles(0, False, pos, vel, cell)
        n_slots += len(cell)
    inj = mp.Injector(m, seed=0)
    rng = np.random.default_rng(5)
    sigma = float(np.sqrt(workloads.KTI_EV * mp.QE / (16 * mp.AMU)))
    P = deck.params
    for k in range(K):
        p, _, cc = inj.sample(P.plasma_den, P.ion_velocity, cfg["dt"], cfg["spwt"])
        a.add_particles(k, True, p, rng.normal(0.0, sigma, size=(len(cc), 3)), cc)
        n_slots += len(cc)
    add_s = time.time() - t0
    free, total = torch.cuda.mem_get_info(device)
    stream = torch.cuda.ExternalStream(c.stream(), device=device)
    gbar = rng.standard_normal(m.n_nodes)

    def timed(fn):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        r = fn()
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1), r

    _, (den, st) = timed(lambda: a.forward(phi, 7000.0))
    tf, (den, st) = timed(lambda: a.forward(phi, 7000.0))
    tb, _ = timed(lambda: a.backward(gbar, 1.0))
    out["adjoint"] = {"K": K, "checkpoint_every": C, "slots": n_slots, "forward_ms": float(st.ms),
                      "forward_call_ms": tf, "reverse_ms": tb, "alive": int(st.alive),
                      "wall_exits": int(st.wall_exits), "add_particles_s": add_s,
                      "device_memory_used_GB": (total - free) / 1e9}
    c.close()
    del a
    torch.cuda.synchronize(device)
    # FP64 form on the same population and injections
    t0 = time.time()
    c, _ = _context(deck, fe, mp.FP64, cfg, kd, device, seed=7)
    out["setup_s_fp64"] = time.time() - t0
    keep_f = []
    f_steps = max(2, min(steps, 3))
    rf = _steps(c, mp.FP64, cfg, deck, f_steps, warmup, torch, device, keep_f)
    out["fp64"] = _summary(rf, c, pk)
    free, total = torch.cuda.mem_get_info(device)
    out["fp64"]["device_memory_used_GB"] = (total - free) / 1e9
    c.close()
    out["mixed_over_fp64"] = out["mixed"]["particle_steps_per_s"] / out["fp64"]["particle_steps_per_s"]
    n_cmp = min(len(keep_m), len(keep_f))
    out["errors_vs_fp64"] = {
        "steps_compared": n_cmp,
        "density_l2_rel": max(float(np.linalg.norm(keep_m[i][0] - keep_f[i][0]) / np.linalg.norm(keep_f[i][0]))
                              for i in range(n_cmp)),
        "phi_closed_loop_max_abs_V": max(float(np.abs(keep_m[i][1] - keep_f[i][1]).max()) for i in range(n_cmp))}
    out["wall_s"] = time.time() - t_all
    return out
