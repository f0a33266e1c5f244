"""Benchmark of the mini-pic hot path on B200: MoveParticles (push + tet walk +
density scatter + removal + normalisation) and FESolver's Newton step.

    python bench.py [--gpus N --steps K --warmup W] [--config 1] [--impl reference]

Workload (default): the 20x20x20-hex Kuhn box (48,000 tets, 9,261 nodes,
8,379 unknowns), O+ ions, n0 = 1e10 m^-3, 7 km/s drift + 0.1 eV Maxwellian,
dt = 5e-8 s, spwt = 5 -> about 2M live ions, seeded synthetic population at
steady state plus the reference injector's ~7,000 new ions per step.  A step
is InjectIons -> MoveParticles -> computePhi (Lapack method: one Newton step,
direct solve) -> updateEf.  FP64 form; the mixed form is measured beside it
on the same seeded population with its errors against FP64.

value      particle-steps/s of MoveParticles, device-resident inputs (each
           step's ions injected on the device), L2 flushed between steps
e2e        the same through the C ABI with host buffers: the step's injected
           particles H2D from host memory, node density D2H each step
e2e_full_step    the whole step through the C ABI (adds computePhi, updateEf
           and the potential D2H)
newton_step_ms   computePhi device time per step
N > 1: weak scaling, every rank pushes its own 2M-ion shard; the node density
is summed over ranks (NCCL all-reduce) before the replicated field solve.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "mini-fem-pic-main_b200"))
sys.path.insert(0, ROOT)

import minipic_b200 as mp  # noqa: E402
from minipic_b200 import kuhn, sharding, workloads  # noqa: E402

METRIC = "particle-steps/sec and Newton-step ms on 1 B200: mixed vs FP64 at stated error"
KTI_EV = workloads.KTI_EV
CONFIGS = workloads.CONFIGS
make_workload = workloads.make_workload
FLUSH_BYTES = 512 << 20
# DRAM bytes of one k_push_fp64 launch on the 2M-ion workload, from ncu
# (dram__bytes_read.sum 113.3 MB + dram__bytes_write.sum 45.6 MB)
PUSH_TRAFFIC_BYTES = 158_962_176
SORT_PERIOD = 10


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), "--query-gpu=clocks.sm,clocks.max.sm,power.draw,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except FileNotFoundError:
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        self.proc.wait()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 7:
                continue
            try:
                sm.append(float(f[0]))
                mx.append(float(f[1]))
            except ValueError:
                continue
            for nm, v in zip(names, f[3:7]):
                if v.lower() == "active":
                    reasons.add(nm)
        os.unlink(self.path)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def run_form(form, args, cfg, deck, pop, inj_batches, device, rank, world, torch, flush, measure_e2e):
    """Runs warm-up + timed steps for one arithmetic form; returns a dict."""
    pos, vel, cell = pop
    m = deck.mesh
    ctx = mp.Context(m, device=device)
    fe = deck.fe_desc_arrays()
    ctx.fe_setup(**fe)
    ctx.set_track_ids(False)
    ctx.reserve(int(len(cell) * 1.3) + 100_000)
    ctx.append(pos, vel, cell)
    ctx.sort_by_tet()  # a steady-state population has been sorted before
    ctx.set_sort_period(SORT_PERIOD)
    if form == mp.MIXED:
        ctx.set_form(mp.MIXED)
    qm = mp.QE / (16 * mp.AMU)
    dt, spwt = cfg["dt"], cfg["spwt"] / world
    stream = torch.cuda.ExternalStream(ctx.stream(), device=device)
    # device-resident steps inject on the device (the reference's counts, Philox
    # Maxwellian sampling); the end-to-end steps upload the host injector's ions
    inj_dev = mp.Injector(m, seed=rank)
    P = deck.params
    sigma = np.sqrt(KTI_EV * mp.QE / (16 * mp.AMU))
    torch.cuda.synchronize(device)

    def step(k, host):
        if host:
            hp, hv, hc = inj_batches[k % len(inj_batches)]
            ctx.append(hp, hv, hc, rewind=True, q_over_m=qm, half_dt=0.5 * dt)
            st = ctx.push(qm, dt, spwt, den_out=den_host)
        else:
            ctx.inject_device(inj_dev, P.plasma_den, P.ion_velocity, dt, cfg["spwt"], sigma, qm, 1000 + rank, k)
            st = ctx.push(qm, dt, spwt)
        if world > 1:
            sharding.allreduce_density(ctx, device)
        nt = ctx.compute_phi(mp.LAPACK, form)
        ctx.update_ef()
        if host:
            ctx._c(mp.lib().mp_field_download(ctx.h, None, mp._p(uh_host), None))
        return st, nt

    den_host = np.zeros(m.n_nodes)
    uh_host = np.zeros(m.n_nodes)
    for k in range(args.warmup):
        step(k, False)
    torch.cuda.synchronize(device)
    res = {"push_ms": [], "push_call_ms": [], "newton_ms": [], "factor_ms": [], "step_ms": [], "n_before": [],
           "n_after": [], "hops": [], "near": []}
    launches0 = ctx.launches()
    for k in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize(device)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        st, nt = step(args.warmup + k, False)
        e1.record(stream)
        e1.synchronize()
        res["push_ms"].append(st.ms_kernel)
        res["push_call_ms"].append(st.ms_step)
        res["newton_ms"].append(nt.ms_total)
        res["factor_ms"].append(nt.ms_factor)
        res["step_ms"].append(e0.elapsed_time(e1))
        res["n_before"].append(st.n_before)
        res["n_after"].append(st.n_after)
        res["hops"].append(st.total_hops)
        res["near"].append(st.near_face_fp64)
    res["launches"] = ctx.launches() - launches0
    if measure_e2e:
        # through the C ABI with host buffers: the step's injected ions H2D from
        # host memory (with the device-side velocity rewind), MoveParticles, the
        # node density D2H into host memory; then the rest of the step (field
        # solve, updateEf, potential D2H) for the full-step figure
        e2e_ms, full_ms, h2d, d2h = [], [], [], []
        for k in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize(device)
            e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
            hp, hv, hc = inj_batches[(args.warmup + args.steps + k) % len(inj_batches)]
            e0.record(stream)
            ctx.append(hp, hv, hc, rewind=True, q_over_m=qm, half_dt=0.5 * dt)
            st = ctx.push(qm, dt, spwt, den_out=den_host)
            e1.record(stream)
            if world > 1:
                sharding.allreduce_density(ctx, device)
            ctx.compute_phi(mp.LAPACK, form)
            ctx.update_ef()
            ctx._c(mp.lib().mp_field_download(ctx.h, None, mp._p(uh_host), None))
            e2.record(stream)
            e2.synchronize()
            e2e_ms.append(e0.elapsed_time(e1))
            full_ms.append(e0.elapsed_time(e2))
            h2d.append(hp.nbytes + hv.nbytes + hc.nbytes)
            d2h.append(den_host.nbytes)
            res.setdefault("e2e_push_n", []).append(st.n_before)
        res["e2e_ms"] = e2e_ms
        res["e2e_full_ms"] = full_ms
        res["h2d"] = float(np.mean(h2d))
        res["d2h"] = float(np.mean(d2h))
        res["d2h_full"] = float(np.mean(d2h)) + uh_host.nbytes
    res["ctx"] = ctx
    return res


def error_metrics(deck, pop, inj_batches, cfg, device, steps=5):
    """Mixed vs FP64 on the same seeded run: density L2, differing cells, phi."""
    pos, vel, cell = pop
    out = []
    qm = mp.QE / (16 * mp.AMU)
    dt, spwt = cfg["dt"], cfg["spwt"]
    ctxs = []
    for form in (mp.FP64, mp.MIXED):
        c = mp.Context(deck.mesh, device=device)
        c.fe_setup(**deck.fe_desc_arrays())
        c.append(pos, vel, cell)
        if form == mp.MIXED:
            c.set_form(mp.MIXED)
        ctxs.append(c)
    for k in range(steps):
        p, v, cc = inj_batches[k % len(inj_batches)]
        dens, uhs = [], []
        for form, c in zip((mp.FP64, mp.MIXED), ctxs):
            c.append(p, v, cc, rewind=True, q_over_m=qm, half_dt=0.5 * dt)
            den = np.zeros(deck.mesh.n_nodes)
            c.push(qm, dt, spwt, den_out=den)
            c.compute_phi(mp.LAPACK, form)
            c.update_ef()
            _, uh, _ = c.field()
            dens.append(den)
            uhs.append(uh)
        out.append((np.linalg.norm(dens[1] - dens[0]) / np.linalg.norm(dens[0]), np.abs(uhs[1] - uhs[0]).max()))
    ga, gb = ctxs[0].download(mp.ORDER_ID), ctxs[1].download(mp.ORDER_ID)
    ids = np.union1d(ga["id"], gb["id"])
    ia = np.full(ids.size, -1)
    ib = np.full(ids.size, -1)
    ia[np.searchsorted(ids, ga["id"])] = ga["cell"]
    ib[np.searchsorted(ids, gb["id"])] = gb["cell"]
    for c in ctxs:
        c.close()
    return {"density_l2_rel": float(max(e[0] for e in out)), "phi_max_abs_V": float(max(e[1] for e in out)),
            "cells_differing_frac": float(np.mean(ia != ib)), "steps": steps}


def mixed_vs_fp64_at_scale(args, device, torch, flush, steps=3, warmup=2):
    """The mixed-form workload (32^3 Kuhn box minus the r = 0.02 m sphere at
    -10 V, ~50M ions): the FP64 and mixed forms run in lockstep on the same
    seeded population and injections.  Per form: full-step particle-steps/s
    (inject + push + scatter + computePhi + updateEf, device time), Newton-step
    ms, push-kernel ms; the mixed form's errors against the FP64 form: node
    density L2, max |phi| difference per step, and the fraction of particles
    whose cell differs at the end."""
    cfg = CONFIGS[2]
    qm = mp.QE / (16 * mp.AMU)
    with tempfile.TemporaryDirectory() as wd:
        kd, deck, pos, vel, cell = make_workload(cfg, wd, seed=4321)
        fe = workloads.fe_arrays(cfg, deck)
        inj = mp.Injector(deck.mesh, seed=0)
        P = deck.params
        batches = [inj.sample(P.plasma_den, P.ion_velocity, cfg["dt"], cfg["spwt"]) for _ in range(warmup + steps)]
        ctxs = {}
        for name, form, method in (("fp64", mp.FP64, mp.LAPACK), ("mixed", mp.MIXED, mp.LAPACK),
                                   ("fp64_sparse_cg", mp.FP64, mp.SPARSE_CG)):
            c = mp.Context(deck.mesh, device=device)
            c.fe_setup(**fe)
            c.set_track_ids(True)  # for the cell comparison at the end
            # an ion stepping into the sphere lies in no tet; the reference's greedy walk can
            # cycle around the cavity without end: absorb such walks (counted) instead
            c.set_walk_limit(256)
            c.set_walk_policy(mp.WALK_LIMIT_ABSORB)
            c.reserve(int(len(cell) * 1.05) + 100_000)
            c.append(pos, vel, cell)
            c.sort_by_tet()
            c.set_sort_period(SORT_PERIOD)
            if form == mp.MIXED:
                c.set_form(mp.MIXED)
            ctxs[name] = (c, form, method, torch.cuda.ExternalStream(c.stream(), device=device))
        del pos, vel, cell
        res = {k: {"step_ms": [], "newton_ms": [], "push_ms": [], "n": [], "refinements": [], "lost": []} for k in ctxs}
        den_err, phi_err, sparse_phi_err = [], [], []
        for k in range(warmup + steps):
            hp, hv, hc = batches[k]
            dens, uhs = {}, {}
            for name, (c, form, method, stream) in ctxs.items():
                flush.zero_()
                torch.cuda.synchronize(device)
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                c.append(hp, hv, hc, rewind=True, q_over_m=qm, half_dt=0.5 * cfg["dt"])
                st = c.push(qm, cfg["dt"], cfg["spwt"])
                nt = c.compute_phi(method, form)
                c.update_ef()
                e1.record(stream)
                e1.synchronize()
                if k >= warmup:
                    r = res[name]
                    r["step_ms"].append(e0.elapsed_time(e1))
                    r["newton_ms"].append(nt.ms_total)
                    r["push_ms"].append(st.ms_kernel)
                    r["n"].append(st.n_before)
                    r["refinements"].append(nt.linear_iterations)
                    r["lost"].append(st.lost)
                den = np.zeros(deck.mesh.n_nodes)
                c._c(mp.lib().mp_density_download(c.h, mp._p(den)))
                _, uh, _ = c.field()
                dens[name], uhs[name] = den, uh
            den_err.append(float(np.linalg.norm(dens["mixed"] - dens["fp64"]) / np.linalg.norm(dens["fp64"])))
            phi_err.append(float(np.abs(uhs["mixed"] - uhs["fp64"]).max()))
            sparse_phi_err.append(float(np.abs(uhs["fp64_sparse_cg"] - uhs["fp64"]).max()))
        # the solver's own precision: one Newton step of each form from the same state
        # (d, the accumulated F1) and the same density, the FP64 context's
        c64, cm, csp = ctxs["fp64"][0], ctxs["mixed"][0], ctxs["fp64_sparse_cg"][0]
        for name in ("d", "F1"):
            v = c64.fe_get(name)
            cm.fe_set(name, v)
            csp.fe_set(name, v)
        c64.compute_phi(mp.LAPACK, mp.FP64, ion_den=dens["fp64"])
        cm.compute_phi(mp.LAPACK, mp.MIXED, ion_den=dens["fp64"])
        nt_sp = csp.compute_phi(mp.SPARSE_CG, mp.FP64, ion_den=dens["fp64"])
        phi_solve_err = float(np.abs(cm.field()[1] - c64.field()[1]).max())
        sparse_solve_err = float(np.abs(csp.field()[1] - c64.field()[1]).max())
        ga, gb = ctxs["fp64"][0].download(mp.ORDER_ID), ctxs["mixed"][0].download(mp.ORDER_ID)
        ids = np.union1d(ga["id"], gb["id"])
        ia = np.full(ids.size, -1)
        ib = np.full(ids.size, -1)
        ia[np.searchsorted(ids, ga["id"])] = ga["cell"]
        ib[np.searchsorted(ids, gb["id"])] = gb["cell"]
        for c, _, _, _ in ctxs.values():
            c.close()
    out = {"workload": cfg["label"], "mesh_hexes": cfg["n"] ** 3, "tets": deck.mesh.n_tets,
           "unknowns": int(fe["neq"]), "ions": int(np.mean(res["fp64"]["n"])), "steps": steps, "warmup": warmup,
           "l2": f"flushed ({FLUSH_BYTES >> 20} MiB write) before each timed step"}
    for name, r in res.items():
        out[name] = {"full_step_particle_steps_per_s": float(np.sum(r["n"]) / (np.sum(r["step_ms"]) / 1e3)),
                     "newton_step_ms": float(np.mean(r["newton_ms"])), "push_kernel_ms": float(np.mean(r["push_ms"])),
                     "refinement_solves": int(max(r["refinements"])),
                     "absorbed_at_walk_limit_per_step": float(np.mean(r["lost"]))}
    out["mixed_over_fp64_full_step"] = (out["mixed"]["full_step_particle_steps_per_s"] /
                                        out["fp64"]["full_step_particle_steps_per_s"])
    out["fp64_sparse_cg"].pop("refinement_solves")
    out["fp64_sparse_cg"]["cg_iterations"] = int(nt_sp.linear_iterations)
    out["fp64_sparse_cg"]["errors_vs_fp64_lapack"] = {
        "phi_solve_max_abs_V": sparse_solve_err, "phi_closed_loop_max_abs_V": max(sparse_phi_err),
        "what": "the FP64 particles with the Newton step's J y = G solved by conjugate gradients on the sparse K "
                "(||r|| <= 1e-12 ||G||) against the dense LDL^T FP64 step"}
    out["errors_vs_fp64"] = {"density_l2_rel": max(den_err),
                             "phi_solve_max_abs_V": phi_solve_err,
                             "phi_closed_loop_max_abs_V": max(phi_err),
                             "cells_differing_frac": float(np.mean(ia != ib)), "steps": warmup + steps,
                             "what": "density and cells: the mixed form's particles against the FP64 form's on "
                                     "the same seeded run; phi_solve: the mixed Newton step against the FP64 one "
                                     "from the same state and density; phi_closed_loop: the two runs' potentials, "
                                     "which also carry their density difference"}
    return out


def sparse_field_at_scale(device, n=64, reps=3):
    """The sparse field solve where the dense one cannot run: a 64^3 Kuhn box
    minus the r = 0.02 m sphere at -10 V (255,822 unknowns; the dense K and J
    would take 523 GB each) in sparse storage.  Node ion density: the plasma
    density with 10 % seeded noise.  Times (CUDA events inside the library)
    one SPARSE_CG Newton step from zero potential and the SPARSE_NEWTON loop,
    each from the same state, and reports the conjugate-gradient iterations."""
    with tempfile.TemporaryDirectory() as wd:
        kd = kuhn.build(n, sphere=(50.0, 50.0, 50.0, 20.0))
        kuhn.write(kd, wd, dt=5e-8, method="lapack")
        deck = mp.Deck.load(wd)
    fe = deck.fe_desc_arrays(workloads.SPHERE_POTENTIAL)
    c = mp.Context(deck.mesh, device=device)
    c.set_fe_storage(mp.FE_SPARSE)
    c.fe_setup(**fe)
    neq = c.neq
    nnz = int(c.fe_sparse_matrix()[0][-1])
    rng = np.random.default_rng(17)
    ion = deck.params.plasma_den * (1 + 0.1 * rng.standard_normal(deck.mesh.n_nodes))
    out = {"workload": f"kuhn{n}s sparse field solve", "unknowns": int(neq), "nonzeros": nnz,
           "dense_K_bytes": 8 * neq * neq, "sparse_K_bytes": 12 * nnz}
    for key, method in (("sparse_cg_newton_step", mp.SPARSE_CG), ("sparse_newton_loop", mp.SPARSE_NEWTON)):
        ms, its, nits = [], [], []
        for r in range(reps + 1):
            c.fe_set("d", np.zeros(neq))
            c.fe_set("F1", np.zeros(neq))
            st = c.compute_phi(method, mp.FP64, ion_den=ion)
            if r:
                ms.append(st.ms_total)
                its.append(st.linear_iterations)
                nits.append(st.newton_iterations)
        out[key] = {"ms": float(np.mean(ms)), "newton_iterations": int(max(nits)),
                    "cg_iterations_last_solve": int(max(its))}
    c.close()
    # the mesh setup of the same mesh: the host helpers against the device ones
    pos, fixed = kd.nodes_mm / 1000.0, np.concatenate([kd.wall_nodes, kd.sphere_nodes])
    setup = {}
    for key, dev in (("host_s", None), ("device_s", device), ("device_s", device)):
        t0 = time.perf_counter()
        m = mp.Mesh.build(pos, kd.tets, kd.inlet_nodes, kd.inlet_tris, fixed, device=dev)
        m.fe_geometry(device=dev)
        setup[key] = time.perf_counter() - t0  # the device entry is timed a second time, warm
    out["mesh_setup"] = dict(setup, tets=int(m.n_tets),
                             what="LoadVolumeMesh + LoadSurfaceMesh geometry + FESolver ID/NX/detJ, wall clock "
                                  "including the host-device copies")
    return out


def vtk_output_leg(device, cfg=CONFIGS[2]):
    """OutputMesh of the 32^3 box minus sphere from the device buffers: the time
    until the call returns (snapshot + writer start) and until the file is
    complete; the reference's own OutputMesh on the same arrays when the
    oracle library is present (reported beside, as its CPU baseline)."""
    with tempfile.TemporaryDirectory() as wd:
        kd = kuhn.build(cfg["n"], sphere=cfg["sphere"])
        kuhn.write(kd, wd)
        deck = mp.Deck.load(wd)
        c = mp.Context(deck.mesh, device=device)
        c.fe_setup(**deck.fe_desc_arrays(workloads.SPHERE_POTENTIAL))
        rng = np.random.default_rng(3)
        uh, den = rng.normal(size=deck.mesh.n_nodes), rng.normal(size=deck.mesh.n_nodes)
        ef = rng.normal(size=(deck.mesh.n_tets, 3))
        for name, v in (("uh", uh), ("den", den), ("ef", ef)):
            c.fe_set(name, v)
        c.output_mesh(0, wd, deck.mesh.node_type)
        c.output_wait()
        t0 = time.perf_counter()
        c.output_mesh(1, wd, deck.mesh.node_type)
        t1 = time.perf_counter()
        c.output_wait()
        t2 = time.perf_counter()
        out = {"workload": cfg["label"] + " OutputMesh", "nodes": deck.mesh.n_nodes, "tets": deck.mesh.n_tets,
               "bytes": os.path.getsize(os.path.join(wd, "mesh_0002.vtu")), "call_ms": (t1 - t0) * 1e3,
               "file_complete_ms": (t2 - t0) * 1e3}
        c.close()
        out["reference_ms"] = reference_output_mesh_ms(wd, kd, uh, den, ef)
    return out


def reference_output_mesh_ms(wd, kd, uh, den, ef):
    """CPU baseline of the VTK leg: the reference's OutputMesh (oracle/_ref)."""
    from oracle import ref
    if not ref.available():
        return None
    s = ref.RefSim(wd, spwt=1.0, extra_fixed={os.path.join(wd, "sphere.dat"): (kd.sphere_nodes, -10.0)})
    for name, v in (("uh", uh), ("den", den), ("ef", ef)):
        s.set(name, v)
    out_dir = os.path.join(wd, "reference")
    os.makedirs(out_dir)
    sec = s.L.ref_output_mesh(s.h, 1, out_dir.encode())
    s.close()
    return sec * 1e3 if sec >= 0 else None


def cpu_baseline(cfg, workdir, pop, budget_s=20.0):
    """The reference's own MoveParticles (oracle/_ref, OpenMP over all host
    threads) on the same population; one Lapack Newton step if it fits."""
    from oracle import ref
    if not ref.available():
        return None
    threads = os.cpu_count() or 1
    s = ref.RefSim(workdir, spwt=cfg["spwt"])
    pos, vel, cell = pop
    parts = np.zeros(len(cell), dtype=ref.PARTICLE_DTYPE)
    parts["pos"], parts["vel"], parts["cell_index"] = pos, vel, cell
    s.set_particles(parts)
    rate1, sec1 = s.time_move(1, threads)
    steps = int(max(1, min(50, budget_s / max(sec1, 1e-3))))
    s.set_particles(parts)
    rate, sec = s.time_move(steps, threads)
    t0 = time.perf_counter()
    s.compute_phi(ref.LAPACK)
    s.update_ef()
    newton_ms = (time.perf_counter() - t0) * 1e3
    s.close()
    return {"value": rate, "unit": "particle-steps/s", "cores": threads, "kind": "reference",
            "sample": f"{steps} MoveParticles steps on the full {len(cell)}-ion population "
                      f"({sec:.1f} s) + 1 Lapack Newton step",
            "newton_step_ms": newton_ms}


def reference_arm(args):
    """--impl reference: the reference's own CPU path (oracle/_ref) timed on the
    host cores, same config/metric; rank 0 only."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    cfg = CONFIGS[args.config]
    from oracle import ref
    if not ref.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libref_oracle.so was not built"}))
        return
    with tempfile.TemporaryDirectory() as wd:
        kd, deck, pos, vel, cell = make_workload(cfg, wd, seed=1234)
        threads = os.cpu_count() or 1
        s = ref.RefSim(wd, spwt=cfg["spwt"])
        parts = np.zeros(len(cell), dtype=ref.PARTICLE_DTYPE)
        parts["pos"], parts["vel"], parts["cell_index"] = pos, vel, cell
        s.set_particles(parts)
        for _ in range(max(1, args.warmup)):
            s.move(threads)
        rate, sec = s.time_move(args.steps, threads)
        n_live = len(s.particles())
        t0 = time.perf_counter()
        s.compute_phi(ref.LAPACK)
        s.update_ef()
        newton_ms = (time.perf_counter() - t0) * 1e3
        full_rate = n_live / (sec / args.steps + newton_ms / 1e3)
        line = {"metric": METRIC, "value": rate, "unit": "particle-steps/s", "impl": "reference",
                "n_gpus": 0, "steps": args.steps, "warmup": args.warmup, "ms_per_step": sec / args.steps * 1e3,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic", "config": {"workload": cfg["label"], "mesh_hexes": cfg["n"] ** 3,
                                                "tets": deck.mesh.n_tets, "nodes": deck.mesh.n_nodes,
                                                "unknowns": int(deck.fe_desc_arrays()["neq"]),
                                                "ions_per_gpu": int(len(cell)), "dt": cfg["dt"],
                                                "method": "lapack (1 Newton step)", "form": "fp64",
                                                "device": f"host CPU, {threads} OpenMP threads"},
                "newton_step_ms": newton_ms,
                "full_step_particle_steps_per_s": full_rate,
                "cpu_baseline": {"value": rate, "unit": "particle-steps/s", "cores": threads, "kind": "reference",
                                 "sample": f"{args.steps} MoveParticles steps, OpenMP over {threads} threads"},
                "e2e": {"value": rate, "unit": "particle-steps/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        s.close()
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--config", type=int, default=1, choices=sorted(CONFIGS))
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-mixed", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-scale", action="store_true", help="skip the mixed-vs-FP64 run on the 32^3 sphere workload")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        reference_arm(args)
        return
    import torch
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))
    cfg = CONFIGS[args.config]
    hbm_peak, peak_kind = peaks()
    with tempfile.TemporaryDirectory() as wd:
        kd, deck, pos, vel, cell = make_workload(cfg, wd, seed=1234 + rank)
        pop = (pos, vel, cell)
        inj = mp.Injector(deck.mesh, seed=rank)
        P = deck.params
        n_batches = args.warmup + 2 * args.steps
        batches = []
        for _ in range(n_batches):
            p, v, c = inj.sample(P.plasma_den, P.ion_velocity, cfg["dt"], cfg["spwt"])
            batches.append((np.ascontiguousarray(p), np.ascontiguousarray(v), np.ascontiguousarray(c)))
        flush = torch.empty(FLUSH_BYTES // 4, dtype=torch.float32, device=local)
        clocks = Clocks(local)
        if world > 1:
            torch.distributed.barrier()
        clocks.start()
        r64 = run_form(mp.FP64, args, cfg, deck, pop, batches, local, rank, world, torch, flush, True)
        clk = clocks.stop()
        r32 = None
        if not args.no_mixed:
            r32 = run_form(mp.MIXED, args, cfg, deck, pop, batches, local, rank, world, torch, flush, False)
        errors = None
        if not args.no_mixed and rank == 0 and world == 1:
            errors = error_metrics(deck, pop, batches, cfg, local)
        cpu = None
        if rank == 0 and world == 1 and not args.no_cpu:
            cpu = cpu_baseline(cfg, wd, pop)
    scale = sparse_big = vtk = None
    if rank == 0 and world == 1 and not args.no_scale and args.config == 1:
        scale = mixed_vs_fp64_at_scale(args, local, torch, flush)
        sparse_big = sparse_field_at_scale(local)
        vtk = vtk_output_leg(local)

    def agg(r):
        push_ms = np.array(r["push_ms"])
        nb, na = np.array(r["n_before"], float), np.array(r["n_after"], float)
        step_ms = np.array(r["step_ms"])
        return push_ms, nb, na, step_ms

    push_ms, nb, na, step_ms = agg(r64)
    psteps = nb.sum()
    push_call_s = np.sum(r64["push_call_ms"]) / 1e3
    e2e_n = float(np.sum(r64["e2e_push_n"]))
    stats = np.array([psteps, push_call_s, step_ms.sum() / 1e3, np.sum(r64["e2e_ms"]) / 1e3,
                      np.mean(r64["newton_ms"]), e2e_n, np.sum(r64["e2e_full_ms"]) / 1e3], dtype=np.float64)
    if world > 1:
        t = torch.tensor(stats, device=local)
        tmax = t.clone()
        torch.distributed.all_reduce(tmax, op=torch.distributed.ReduceOp.MAX)
        tsum = t.clone()
        torch.distributed.all_reduce(tsum, op=torch.distributed.ReduceOp.SUM)
        psteps_all, e2e_n_all = float(tsum[0]), float(tsum[5])
        push_s, step_s, e2e_s, newton_ms = float(tmax[1]), float(tmax[2]), float(tmax[3]), float(tmax[4])
        e2e_full_s = float(tmax[6])
    else:
        psteps_all, e2e_n_all = psteps, e2e_n
        push_s, step_s, e2e_s, newton_ms, e2e_full_s = stats[1], stats[2], stats[3], stats[4], stats[6]
    if rank == 0:
        bytes_per = 52.0  # pos 24 + vel 24 + tet 4, read and written once (FP64 SoA)
        alg_bytes = (nb + na) * bytes_per
        achieved = float(np.mean(alg_bytes / (push_ms * 1e-3)) / 1e9)
        line = {
            "metric": METRIC, "value": psteps_all / push_s, "unit": "particle-steps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": float(step_s / args.steps * 1e3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded Kuhn-box ions at steady state + reference injector)",
            "config": {"workload": cfg["label"], "mesh_hexes": cfg["n"] ** 3, "tets": deck.mesh.n_tets,
                       "nodes": deck.mesh.n_nodes, "unknowns": int(deck.fe_desc_arrays()["neq"]),
                       "ions_per_gpu": int(np.mean(nb)), "dt": cfg["dt"], "method": "lapack (1 Newton step)",
                       "form": "fp64", "l2": f"flushed ({FLUSH_BYTES >> 20} MiB write) between timed steps",
                       "tet_sort_every": SORT_PERIOD,
                       "injection": "device (the reference's per-face counts; Philox4x32-10 positions and "
                                    "0.1 eV Maxwellian velocities) in the device-resident steps; the host "
                                    "injector's ions uploaded in the end-to-end steps",
                       "parallelism": f"particles sharded x{world}, density all-reduce" if world > 1 else "1 GPU"},
            "newton_step_ms": float(newton_ms),
            "full_step_particle_steps_per_s": psteps_all / step_s,
            "push_kernel_ms": float(np.mean(push_ms)),
            "hops_per_particle_step": float(np.sum(r64["hops"]) / psteps),
            "e2e": {"value": e2e_n_all / e2e_s, "unit": "particle-steps/s",
                    "what": "MoveParticles through the C ABI: injected ions H2D from host memory, push + walk + "
                            "scatter + normalisation, node density D2H to host memory",
                    "h2d_bytes_per_step": int(r64["h2d"]), "d2h_bytes_per_step": int(r64["d2h"]),
                    "ms_per_step": float(e2e_s / args.steps * 1e3)},
            "e2e_full_step": {"value": e2e_n_all / e2e_full_s, "unit": "particle-steps/s",
                              "what": "the whole step through the C ABI: InjectIons H2D, MoveParticles, computePhi "
                                      "(Lapack, one Newton step), updateEf, density and potential D2H",
                              "h2d_bytes_per_step": int(r64["h2d"]), "d2h_bytes_per_step": int(r64["d2h_full"]),
                              "ms_per_step": float(e2e_full_s / args.steps * 1e3)},
            "gpu_launches": int(r64["launches"]),
            "roofline": {"kernel": "k_push_fp64", "bound": "hbm", "achieved": achieved, "peak": hbm_peak,
                         "unit": "GB/s", "frac": achieved / hbm_peak, "traffic": PUSH_TRAFFIC_BYTES,
                         "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one k_push_fp64 "
                                           "launch on this workload",
                         "peak_kind": peak_kind,
                         "bytes_per_particle_step": 104},
            "clocks": clk,
        }
        if r32 is not None:
            pm, nb32, na32, sm32 = agg(r32)
            ach32 = float(np.mean((nb32 + na32) * 28.0 / (pm * 1e-3)) / 1e9)
            line["mixed"] = {
                "value": float(nb32.sum() / (np.sum(r32["push_call_ms"]) / 1e3)),
                "full_step_particle_steps_per_s": float(nb32.sum() / (sm32.sum() / 1e3)),
                "newton_step_ms": float(np.mean(r32["newton_ms"])),
                "push_kernel_ms": float(np.mean(pm)),
                "roofline": {"kernel": "k_push_mixed", "bound": "hbm", "achieved": ach32, "peak": hbm_peak,
                             "unit": "GB/s", "frac": ach32 / hbm_peak, "bytes_per_particle_step": 56},
                "near_face_fp64_per_step": float(np.mean(r32["near"])),
                "errors_vs_fp64": errors,
            }
        if cpu is not None:
            line["cpu_baseline"] = cpu
        if scale is not None:
            line["mixed_vs_fp64_kuhn32s_50M"] = scale
        if sparse_big is not None:
            line["sparse_field_kuhn64s"] = sparse_big
        if vtk is not None:
            line["vtk_output"] = vtk
        print(json.dumps(line))
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
