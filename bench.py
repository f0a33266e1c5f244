"""Benchmark of the mini-pic hot path on B200: InjectIons -> MoveParticles
(push + tet walk + density scatter + removal + normalisation) -> computePhi
(Poisson-Boltzmann Newton step) -> updateEf, in the mixed-precision form and
the FP64 form side by side.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]
                    [--legs all|none|kuhn20,nonlinear,adjoint,sparse64,vtk]
    python bench.py --horizon 500     # mixed vs FP64 error growth over a long run
    python bench.py --stress          # the combined-stress workload (40^3 box, 200M ions)

Headline workload (the metric's mixed-precision configuration): the 32^3-hex
Kuhn box minus the centred r = 0.02 m sphere held at -10 V (189,972 tets,
35,156 nodes, 32,244 unknowns; dense FP64 Jacobian 8.3 GB), O+ ions seeded at
steady state (48.3M inside the domain: drift 7 km/s + 0.1 eV Maxwellian),
spwt 0.2, dt 5e-8 s, the reference's per-face injection counts every step
(about 175k ions), a tet re-sort every 10 steps.  A step is InjectIons ->
MoveParticles -> computePhi (Lapack method: one Newton step, dense LDL^T) ->
updateEf.  The synthetic seeded population stands in for a physical run.

value        particle-steps/s of the mixed form's whole step (device-resident:
             ions injected on the device), sum of particles pushed / sum of the
             steps' device time (CUDA events on the context's stream)
fp64         the same for the FP64 form in lockstep on the same population
errors_vs_fp64   the mixed form against the FP64 form on the same seeded run
e2e          the mixed whole step through the C ABI with host buffers: the
             step's injected ions H2D from host memory, node density and
             potential D2H into host memory
roofline     the kernel class with the largest device time in the mixed step
roofline_push    the push kernels on the 20^3 box (2M ions, no particle IDs)
N > 1: weak scaling.  Every rank pushes its own seeded population with its own
device injections (weights spwt/N, so the summed density is the single-GPU
one); the node density is summed over ranks (NCCL all-reduce in place) before
the replicated field solve.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
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
HEADLINE = 2
FLUSH_BYTES = 512 << 20
SORT_PERIOD = 10
POP_SEED = 4321
QM = mp.QE / (16 * mp.AMU)
SIGMA = float(np.sqrt(KTI_EV * mp.QE / (16 * mp.AMU)))
LEGS = ("kuhn20", "nonlinear", "adjoint", "sparse64", "vtk")
# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of one ncu capture
# per kernel, per unit of its algorithmic work; a launch's traffic is scaled by
# its units (a K = 1,024 trailing update of 55.4 GFLOP moves 444.3 MB in 3xTF32,
# profiles/k_update_tc_kuhn20_newton.md, and 232.4 MB in TF32,
# profiles/k_update_tc_tf32_kuhn20_newton.md; one of 41.0 GFLOP with FP16
# operands moves 140.3 MB, profiles/k_update_tc_tma_f16_kuhn20_newton.md;
# profiles/k_push_*_kuhn20_2M.md:
# 160.5 MB and 65.1 MB for 1.99M particles, in and out)
TRAFFIC_PER_UNIT = {("tc3", "update"): 444.3e6 / 55.4e9, ("tc1", "update"): 232.4e6 / 55.4e9,
                    ("tc2", "update"): 140.3e6 / 41.0e9,
                    ("fp64", "push"): 160.5e6 / (2 * 1.99e6), ("mixed", "push"): 65.1e6 / (2 * 1.99e6)}
# FP64 tensor-pipe rate implied by one ncu capture of k_update_f64_mma (26.4
# TFLOP/s at 76.6 % DMMA-pipe activity); this pool's peaks file has no FP64 figure
FP64_TENSOR_TFLOPS = 26.4 / 0.766
KT_NAMES = {mp.KT_PUSH: "push", mp.KT_UPDATE: "trailing_update", mp.KT_DIAG: "diagonal_factor",
            mp.KT_PANEL: "panel", mp.KT_TRSV: "triangular_solve"}
KT_KERNEL = {mp.KT_PUSH: {mp.FP64: "k_push_fp64", mp.MIXED: "k_push_mixed"},
             mp.KT_UPDATE: {mp.FP64: "k_update_f64_mma (FP64 mma.sync m8n8k4)", mp.MIXED: "tc::k_update_tc (tcgen05)"},
             mp.KT_DIAG: {mp.FP64: "k_ldlt_diag<double>", mp.MIXED: "k_ldlt_diag<float>"},
             mp.KT_PANEL: {mp.FP64: "k_ldlt_step_dmma", mp.MIXED: "k_ldlt_step_tc"},
             mp.KT_TRSV: {mp.FP64: "k_trsv_ll<double>", mp.MIXED: "k_trsv_ll<float>"}}


def peaks():
    """HBM copy GB/s and dense bf16 TFLOP/s (burst, sustained) measured on this
    pool's B200s, else the pool's earlier measurement."""
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return {"hbm_gbs": float(d["hbm_gbs"]), "bf16_tflops": float(d["bf16_tflops"]),
                "bf16_tflops_sustained": float(d.get("bf16_tflops_sustained", d["bf16_tflops"])),
                "kind": "measured"}
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0, "kind": "fallback"}


class Clocks:
    """nvidia-smi sampling of the SM clock and throttle reasons during a timed region."""

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


def workload_config(cfg, n_tets, n_nodes, neq, n_ions):
    """The workload description both arms print (same keys and values)."""
    return {"workload": cfg["label"], "mesh_hexes": cfg["n"] ** 3, "tets": int(n_tets), "nodes": int(n_nodes),
            "unknowns": int(neq), "ions": int(n_ions), "dt": cfg["dt"], "spwt": cfg["spwt"],
            "sphere_potential_V": workloads.SPHERE_POTENTIAL if cfg["sphere"] else None,
            "method": "lapack (one Newton step per step)",
            "injection": "the reference's per-face counts every step",
            "population": f"seeded steady state (seed {POP_SEED}): uniform, 7 km/s drift + {KTI_EV} eV Maxwellian"}


def make_context(deck, fe, form, n_pop, device, track_ids, sphere):
    c = mp.Context(deck.mesh, device=device)
    c.fe_setup(**fe)
    c.set_track_ids(track_ids)
    if sphere:
        # an ion stepping into the sphere lies in no tet; the reference's greedy walk
        # can cycle around the cavity: walks end at 256 hops and the ion is absorbed
        workloads.absorb_cavity_walks(c)
    c.reserve(int(n_pop * 1.05) + 400_000)
    return c


def load_population(c, pos, vel, cell, form, chunk=8_000_000):
    for lo in range(0, len(cell), chunk):
        hi = min(len(cell), lo + chunk)
        c.append(pos[lo:hi], vel[lo:hi], cell[lo:hi])
    c.sort_by_tet()  # a steady-state population has been sorted before
    c.set_sort_period(SORT_PERIOD)
    if form == mp.MIXED:
        c.set_form(mp.MIXED)


def mixed_terms(neq):
    """Arithmetic of the mixed factorization's trailing update under the
    library's default (MIXED_AUTO): 3 (3xTF32) or 2 (FP16 operands)."""
    return mp.MIXED_FP16 if neq >= mp.MIXED_FP16_FROM else mp.MIXED_TF32X3


def kernel_roofline(ctx, form, pk, step_ms_total, sustained=True, neq=0):
    """The kernel classes' device time in the timed region and the roofline of
    the one with the largest share."""
    classes = {k: ctx.kernel_timing(k) for k in KT_NAMES if mp.KT_TIMED >> k & 1}
    share = {KT_NAMES[k]: {"launches": v["launches"], "ms": v["ms"], "share_of_step": v["ms"] / step_ms_total}
             for k, v in classes.items()}
    share["diagonal_factor + panel + the rest"] = {
        "ms": step_ms_total - sum(v["ms"] for v in classes.values()),
        "what": "not bracketed by events in the timed run (hundreds of small launches a step)"}
    top = max(classes, key=lambda k: classes[k]["ms"])
    v = classes[top]
    terms = mixed_terms(neq)
    kname = KT_KERNEL[top][form]
    if top == mp.KT_UPDATE and form == mp.MIXED:
        kname = ("tc::k_update_tc<1> (3xTF32, tcgen05 kind::tf32)" if terms == mp.MIXED_TF32X3 else
                 "tc::k_update_tc_tma<2> (FP16 operands, tcgen05 kind::f16, old values of A moved by TMA)")
    out = {"kernel": kname, "class": KT_NAMES[top], "launches": v["launches"],
           "avg_launch_ms": v["ms"] / max(v["launches"], 1)}
    if top == mp.KT_PUSH:
        ach = v["work"] / (v["ms"] * 1e-3) / 1e9
        out.update(bound="hbm", achieved=ach, peak=pk["hbm_gbs"], unit="GB/s", frac=ach / pk["hbm_gbs"],
                   peak_kind=pk["kind"] + " HBM copy",
                   algorithmic="(particles before + after the push) x %d B" % (52 if form == mp.FP64 else 28))
        key = ("fp64" if form == mp.FP64 else "mixed", "push")
        bpp = 52.0 if form == mp.FP64 else 28.0
        out["traffic"] = TRAFFIC_PER_UNIT[key] * v["work"] / bpp / max(v["launches"], 1)
        out["traffic_source"] = "ncu DRAM bytes per particle (20^3 box, 2M ions) x this launch's particles"
    elif top == mp.KT_UPDATE and form == mp.FP64:
        ach = v["work"] / (v["ms"] * 1e-3) / 1e12
        out.update(bound="tensor (FP64)", achieved=ach, peak=FP64_TENSOR_TFLOPS, unit="TFLOP/s",
                   frac=ach / FP64_TENSOR_TFLOPS,
                   peak_kind="FP64 tensor pipe: 26.4 TFLOP/s at 76.6 % pipe activity in one ncu capture "
                             "(profiles/k_update_f64_kuhn20_newton.md); no measured FP64 peak on this pool",
                   algorithmic="2 flops per multiply-add of the trailing update's lower triangle",
                   frac_of_bf16_sustained=ach / pk["bf16_tflops_sustained"])
    elif top == mp.KT_UPDATE:
        ach = v["work"] / (v["ms"] * 1e-3) / 1e12
        peak = pk["bf16_tflops_sustained"] if sustained else pk["bf16_tflops"]
        out.update(bound="tensor", achieved=ach, peak=peak, unit="TFLOP/s", frac=ach / peak,
                   peak_kind=pk["kind"] + (" bf16 dense, sustained" if sustained else " bf16 dense, burst"),
                   algorithmic="2 flops per multiply-add of the trailing update's lower triangle")
        if form == mp.MIXED and terms == mp.MIXED_TF32X3:
            out["note"] = ("kind::tf32 MMAs run at half the bf16 rate, and the 3xTF32 split issues three "
                           "per term: issued TF32 rate = 3 x achieved")
            out["tf32_issued_frac_of_half_bf16_peak"] = 3 * ach / (peak / 2)
        elif form == mp.MIXED:
            out["note"] = ("kind::f16 MMAs (the bf16 rate) on FP16 copies of the trailing updates' operands; "
                           "the strips inside a super-panel (3.5 % of the flops at 32,244 unknowns) stay on TF32")
        if form == mp.MIXED and ("tc%d" % terms, "update") in TRAFFIC_PER_UNIT:
            out["traffic"] = TRAFFIC_PER_UNIT[("tc%d" % terms, "update")] * v["work"] / max(v["launches"], 1)
            out["traffic_source"] = ("ncu DRAM bytes per flop of a K = 1,024 trailing update (8,379 unknowns) x "
                                     "this workload's average flops per launch (the strips, K = 256, move more "
                                     "bytes per flop: an estimate)")
    else:
        out.update(bound="latency", achieved=None, peak=None, unit=None, frac=None,
                   note="a serial chain of small launches; no throughput bound applies")
    out.setdefault("traffic", None)
    out["classes"] = share
    p = classes.get(mp.KT_PUSH)
    if p and p["ms"] > 0:
        gbs = p["work"] / (p["ms"] * 1e-3) / 1e9
        out["push_kernel"] = {"kernel": KT_KERNEL[mp.KT_PUSH][form], "achieved": gbs, "unit": "GB/s",
                              "frac": gbs / pk["hbm_gbs"], "avg_launch_ms": p["ms"] / max(p["launches"], 1),
                              "bytes_per_particle_step": 104 if form == mp.FP64 else 56}
    return out


def run_headline(args, device, rank, world, torch, flush, pk):
    """Mixed and FP64 forms in lockstep on the headline workload; then the
    mixed form's end-to-end steps through the C ABI."""
    cfg = CONFIGS[args.config]
    sphere = cfg["sphere"] is not None
    wd = tempfile.mkdtemp()
    kd = workloads.write_deck(cfg, wd)
    deck = mp.Deck.load(wd)
    pos, vel, cell = workloads.seed_population(kd, cfg, POP_SEED + rank)
    fe = workloads.fe_arrays(cfg, deck)
    neq = int(fe["neq"])
    n0 = len(cell)
    P = deck.params
    dt, spwt = cfg["dt"], cfg["spwt"]
    spwt_push = spwt / world
    forms = {"mixed": mp.MIXED, "fp64": mp.FP64}
    ctxs = {}
    for name, form in forms.items():
        c = make_context(deck, fe, form, n0, device, True, sphere)
        load_population(c, pos, vel, cell, form)
        ctxs[name] = (c, form, torch.cuda.ExternalStream(c.stream(), device=device))
    del pos, vel, cell
    inj = {name: mp.Injector(deck.mesh, seed=rank) for name in forms}
    res = {k: {"step_ms": [], "newton_ms": [], "push_ms": [], "n": [], "refinements": [], "lost": [], "hops": []}
           for k in forms}
    den_err, phi_err = [], []
    launches0 = {k: v[0].launches() for k, v in ctxs.items()}

    def step(name, k):
        c, form, _ = ctxs[name]
        c.inject_device(inj[name], P.plasma_den, P.ion_velocity, dt, spwt, SIGMA, QM, 1000 + rank, k)
        st = c.push(QM, dt, spwt_push)
        if world > 1:
            sharding.allreduce_density(c, device)
        nt = c.compute_phi(mp.LAPACK, form)
        c.update_ef()
        return st, nt

    clocks = Clocks(device)
    for k in range(args.warmup + args.steps):
        timed = k >= args.warmup
        if k == args.warmup:
            for c, _, _ in ctxs.values():
                c.set_kernel_timing(mp.KT_TIMED)
            launches0 = {n: v[0].launches() for n, v in ctxs.items()}
            if world > 1:
                torch.distributed.barrier()
            clocks.start()
        dens, uhs = {}, {}
        for name, (c, form, stream) in ctxs.items():
            flush.zero_()
            torch.cuda.synchronize(device)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            st, nt = step(name, k)
            e1.record(stream)
            e1.synchronize()
            if timed:
                r = res[name]
                r["step_ms"].append(e0.elapsed_time(e1))
                r["newton_ms"].append(nt.ms_total)
                r["push_ms"].append(st.ms_kernel)
                r["n"].append(st.n_before)
                r["refinements"].append(nt.linear_iterations)
                r["lost"].append(st.lost)
                r["hops"].append(st.total_hops)
            dens[name] = c.density()
            uhs[name] = c.field()[1]
        if timed:
            den_err.append(float(np.linalg.norm(dens["mixed"] - dens["fp64"]) / np.linalg.norm(dens["fp64"])))
            phi_err.append(float(np.abs(uhs["mixed"] - uhs["fp64"]).max()))
    clk = clocks.stop()
    if world > 1:
        torch.distributed.barrier()
    out = {"cfg": cfg, "deck": deck, "neq": neq, "n0": n0, "res": res, "clocks": clk,
           "launches": {n: ctxs[n][0].launches() - launches0[n] for n in ctxs}}
    out["roofline"] = {n: kernel_roofline(ctxs[n][0], ctxs[n][1], pk, float(np.sum(res[n]["step_ms"])), neq=neq)
                       for n in ctxs}
    for c, _, _ in ctxs.values():
        c.set_kernel_timing(False)
    # the solver's own precision: one Newton step of each form from the same state
    # (d, the accumulated F1) and the same density
    c64, cm = ctxs["fp64"][0], ctxs["mixed"][0]
    for nm in ("d", "F1"):
        cm.fe_set(nm, c64.fe_get(nm))
    den64 = c64.density()
    c64.compute_phi(mp.LAPACK, mp.FP64, ion_den=den64)
    cm.compute_phi(mp.LAPACK, mp.MIXED, ion_den=den64)
    phi_solve = float(np.abs(cm.field()[1] - c64.field()[1]).max())
    # cells of the same particles in the two forms
    ga, gb = c64.download(mp.ORDER_ID), cm.download(mp.ORDER_ID)
    ids = np.union1d(ga["id"], gb["id"])
    ia = np.full(ids.size, -1)
    ib = np.full(ids.size, -1)
    ia[np.searchsorted(ids, ga["id"])] = ga["cell"]
    ib[np.searchsorted(ids, gb["id"])] = gb["cell"]
    del ga, gb
    out["errors"] = {"density_l2_rel": max(den_err), "density_l2_rel_per_step": den_err,
                     "phi_closed_loop_max_abs_V": max(phi_err), "phi_closed_loop_per_step_V": phi_err,
                     "phi_solve_max_abs_V": phi_solve, "cells_differing_frac": float(np.mean(ia != ib)),
                     "steps_compared": args.steps + args.warmup,
                     "what": "the mixed form's density, potential and cells against the FP64 form's on the same "
                             "seeded run (same population, same device injections); phi_solve: the mixed Newton "
                             "step against the FP64 one from the same state and density"}
    # e2e: the mixed form through the C ABI with host buffers
    cm.set_kernel_timing(False)
    host_inj = mp.Injector(deck.mesh, seed=100 + rank)
    batches = [host_inj.sample(P.plasma_den, P.ion_velocity, dt, spwt) for _ in range(args.steps)]
    stream = ctxs["mixed"][2]
    den_host = np.zeros(deck.mesh.n_nodes)
    uh_host = np.zeros(deck.mesh.n_nodes)
    e2e_ms, e2e_n, h2d = [], [], []
    for k in range(args.steps):
        hp, hv, hc = batches[k]
        flush.zero_()
        torch.cuda.synchronize(device)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        cm.append(hp, hv, hc, rewind=True, q_over_m=QM, half_dt=0.5 * dt)
        if world > 1:
            # the density read back is the one summed over ranks
            st = cm.push(QM, dt, spwt_push)
            sharding.allreduce_density(cm, device)
            cm._c(mp.lib().mp_density_download(cm.h, mp._p(den_host)))
        else:
            st = cm.push(QM, dt, spwt_push, den_out=den_host)
        cm.compute_phi(mp.LAPACK, mp.MIXED)
        cm.update_ef()
        cm._c(mp.lib().mp_field_download(cm.h, None, mp._p(uh_host), None))
        e1.record(stream)
        e1.synchronize()
        e2e_ms.append(e0.elapsed_time(e1))
        e2e_n.append(st.n_before)
        h2d.append(hp.nbytes + hv.nbytes + hc.nbytes)
    out["e2e"] = {"ms": e2e_ms, "n": e2e_n, "h2d": float(np.mean(h2d)), "d2h": float(den_host.nbytes + uh_host.nbytes)}
    for c, _, _ in ctxs.values():
        c.close()
    return out


def run_kuhn20(args, device, torch, flush, pk):
    """The FP64 throughput configuration (20^3 box, 2M ions): push-kernel
    lines of both forms (particle IDs off, re-sort every 10 steps) with their
    rooflines, and the Newton step of both forms."""
    cfg = CONFIGS[1]
    with tempfile.TemporaryDirectory() as wd:
        kd = workloads.write_deck(cfg, wd)
        deck = mp.Deck.load(wd)
        pos, vel, cell = workloads.seed_population(kd, cfg, 1234)
        fe = workloads.fe_arrays(cfg, deck)
        P = deck.params
        out = {"workload": cfg["label"], "tets": deck.mesh.n_tets, "unknowns": int(fe["neq"]), "ions": len(cell)}
        keep = None
        for name, form in (("fp64", mp.FP64), ("mixed", mp.MIXED)):
            c = make_context(deck, fe, form, len(cell), device, False, False)
            load_population(c, pos, vel, cell, form)
            inj = mp.Injector(deck.mesh, seed=0)
            newton, push, psteps = [], [], 0
            for k in range(args.warmup + args.steps):
                if k == args.warmup:
                    c.set_kernel_timing(mp.KT_TIMED)
                flush.zero_()
                torch.cuda.synchronize(device)
                c.inject_device(inj, P.plasma_den, P.ion_velocity, cfg["dt"], cfg["spwt"], SIGMA, QM, 1000, k)
                st = c.push(QM, cfg["dt"], cfg["spwt"])
                nt = c.compute_phi(mp.LAPACK, form)
                c.update_ef()
                if k >= args.warmup:
                    newton.append(nt.ms_total)
                    push.append(st.ms_kernel)
                    psteps += st.n_before
            t = c.kernel_timing(mp.KT_PUSH)
            ach = t["work"] / (t["ms"] * 1e-3) / 1e9
            out[name] = {"push_particle_steps_per_s": psteps / (np.sum(push) / 1e3),
                         "push_kernel_ms": float(np.mean(push)), "newton_step_ms": float(np.mean(newton)),
                         "roofline": {"kernel": KT_KERNEL[mp.KT_PUSH][form], "bound": "hbm", "achieved": ach,
                                      "peak": pk["hbm_gbs"], "unit": "GB/s", "frac": ach / pk["hbm_gbs"],
                                      "launches": t["launches"], "avg_launch_ms": t["ms"] / max(t["launches"], 1),
                                      "peak_kind": pk["kind"] + " HBM copy",
                                      "bytes_per_particle_step": 104 if form == mp.FP64 else 56,
                                      "traffic": TRAFFIC_PER_UNIT[(name, "push")] * t["work"] /
                                      (52.0 if form == mp.FP64 else 28.0) / max(t["launches"], 1),
                                      "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum per "
                                                        "particle of one launch on this workload x the launch's "
                                                        "particles"}}
            if name == "fp64":
                keep = c
            else:
                c.close()
        return out, keep, deck


def run_gs_sweeps(ctx, pk, sweeps=100):
    """Gauss-Seidel sweeps as a bandwidth kernel: the solveLinear iteration on
    the 20^3 FP64 Jacobian (8,379 unknowns), right-hand side scaled so that
    the tolerance is not met, `sweeps` sweeps; one sweep reads J once
    (8 neq^2 bytes)."""
    neq = ctx.neq
    den = ctx.density()
    ctx.build_f1(den)
    ctx.residual()
    ctx.build_j(mp.GAUSS_SEIDEL)
    G = ctx.fe_get("G") * 1e8
    ctx.set_gs_max_sweeps(sweeps)
    ctx.set_kernel_timing(True)
    try:
        ctx.solve_linear(mp.GAUSS_SEIDEL, mp.FP64, b=G)
        status = 0
    except mp.MpError as e:
        status = e.status  # MP_ERR_NOT_CONVERGED: the sweeps ran out, as intended
    t = ctx.kernel_timing(mp.KT_TRSV)  # every sweep launch with its x_old pass (up to 25 sweeps a launch)
    ctx.set_kernel_timing(False)
    ctx.set_gs_max_sweeps(10000)
    ms = t["ms"] / sweeps
    ach = 8.0 * neq * neq / (ms * 1e-3) / 1e9
    return {"workload": "kuhn20 Gauss-Seidel sweeps (FP64 J, 8,379 unknowns)", "sweeps": sweeps,
            "launches": t["launches"], "ms_per_sweep": ms, "status": status,
            "roofline": {"kernel": "k_gs_sweeps (fused sweeps) + k_gs_upper", "bound": "hbm", "achieved": ach,
                         "peak": pk["hbm_gbs"],
                         "unit": "GB/s", "frac": ach / pk["hbm_gbs"], "bytes_per_sweep": 8 * neq * neq,
                         "peak_kind": pk["kind"] + " HBM copy"}}


def run_nonlinear(ctx, deck):
    """The NonLinear method (Newton with Gauss-Seidel inner solves) from the
    state the 20^3 FP64 run left: one computePhi, its Newton iterations and
    sweeps, and the sweep bandwidth (8 neq^2 bytes of J per sweep)."""
    neq = ctx.neq
    ctx.set_kernel_timing(False)
    den = ctx.density()
    st = mp.NewtonStats()
    d0, f0 = ctx.fe_get("d"), ctx.fe_get("F1")
    rc = mp.lib().mp_compute_phi(ctx.h, mp._p(np.ascontiguousarray(den)), mp.NONLINEAR, mp.FP64,
                                 mp.C.byref(st))
    ctx.fe_set("d", d0)
    ctx.fe_set("F1", f0)
    return {"workload": "kuhn20 NonLinear computePhi (FP64 Gauss-Seidel inner solves)", "status": int(rc),
            "ms": st.ms_total, "newton_iterations": st.newton_iterations,
            "gs_sweeps_last_solve": st.linear_iterations, "gs_solves_out_of_sweeps": st.linear_failures,
            "l2": st.l2}


def run_adjoint(args, device, torch, pk):
    """The adjoint configuration: 16^3 box, 1M ions, K = 20 push + scatter
    steps, checkpoints every 5; forward, reverse (vector-Jacobian product) and
    tangent (Jacobian-vector product) device times."""
    from minipic_b200 import adjoint as adj_mod
    cfg = CONFIGS[3]
    with tempfile.TemporaryDirectory() as wd:
        deck, slots, K = workloads.make_adjoint_case(cfg, wd, seed=77)
    m = deck.mesh
    c = mp.Context(m, device=device)
    c.fe_setup(**deck.fe_desc_arrays())
    stream = torch.cuda.ExternalStream(c.stream(), device=device)
    wall = (m.node_type == mp.NODE_FIXED).astype(np.uint8)
    a = adj_mod.Adjoint(c, K, cfg["checkpoint_every"], QM, 16 * mp.AMU, cfg["dt"], cfg["spwt"],
                        np.array([1.0, 0.0, 0.0]), wall)
    workloads.load_adjoint(a, slots)
    phi = workloads.adjoint_phi(m)
    rng = np.random.default_rng(3)
    gbar = rng.standard_normal(m.n_nodes)
    dphi = rng.standard_normal(m.n_nodes)

    def timed(fn):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        r = fn()
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1), r

    fw, bw, tg = [], [], []
    for k in range(args.warmup + args.steps):
        tf, (den, st) = timed(lambda: a.forward(phi, 7000.0))
        tb, _ = timed(lambda: a.backward(gbar, 1.0))
        tt, _ = timed(lambda: a.tangent(dphi, 1.0))
        if k >= args.warmup:
            fw.append(st.ms)
            bw.append(tb)
            tg.append(tt)
    n_slots = int(st.slots)
    slot_steps = float(np.sum((K - slots["first"])))
    C = cfg["checkpoint_every"]
    # forward: slot inputs read once (6 FP64 + cell + first step + flag = 57 B),
    # a 52 B checkpoint every C steps, the outcome byte
    fwd_bytes = n_slots * (57 + 52 * (K // C) + 1)
    c.close()
    return {"workload": cfg["label"], "slots": n_slots, "K": K, "checkpoint_every": C,
            "slot_steps": slot_steps, "forward_ms": float(np.mean(fw)), "reverse_ms": float(np.mean(bw)),
            "tangent_ms": float(np.mean(tg)),
            "forward_slot_steps_per_s": slot_steps / (np.mean(fw) / 1e3),
            "reverse_slot_steps_per_s": slot_steps / (np.mean(bw) / 1e3),
            "forward_bytes_per_slot_step": fwd_bytes / slot_steps,
            "forward_hbm_frac": fwd_bytes / (np.mean(fw) * 1e-3) / 1e9 / pk["hbm_gbs"],
            "what": "one thread carries a slot through its steps in registers; the tet records and field are "
                    "gathered from L2, so the kernels are gather-latency bound, not HBM bound",
            "alive": int(st.alive), "wall_exits": int(st.wall_exits)}


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
    return out


def vtk_output_leg(device, cfg=CONFIGS[2]):
    """OutputMesh of the 32^3 box minus sphere from the device buffers: the time
    until the call returns (snapshot + writer start) and until the file is
    complete."""
    with tempfile.TemporaryDirectory() as wd:
        kd = kuhn.build(cfg["n"], sphere=cfg["sphere"])
        kuhn.write(kd, wd)
        deck = mp.Deck.load(wd)
        c = mp.Context(deck.mesh, device=device)
        c.fe_setup(**deck.fe_desc_arrays(workloads.SPHERE_POTENTIAL))
        rng = np.random.default_rng(3)
        for name, v in (("uh", rng.normal(size=deck.mesh.n_nodes)), ("den", rng.normal(size=deck.mesh.n_nodes)),
                        ("ef", rng.normal(size=(deck.mesh.n_tets, 3)))):
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
    return out


# ---- the reference's CPU path (oracle/_ref): the CPU baseline and the reference arm ----

def reference_sim(cfg, wd, kd, seed, spwt=None):
    """The reference's own loaders, FESolver and Species on the configuration's
    deck, with the same seeded population (no call into this library)."""
    from oracle import ref
    extra = {}
    if cfg["sphere"]:
        extra = {os.path.join(wd, "sphere.dat"): (kd.sphere_nodes, workloads.SPHERE_POTENTIAL)}
    s = ref.RefSim(wd, spwt=cfg["spwt"] if spwt is None else spwt, extra_fixed=extra)
    pos, vel, cell = workloads.seed_population(kd, cfg, seed)
    parts = np.zeros(len(cell), dtype=ref.PARTICLE_DTYPE)
    parts["pos"], parts["vel"], parts["cell_index"] = pos, vel, cell
    del pos, vel
    s.set_particles(parts)
    return s, len(cell)


def cpu_baseline(config, budget_s=25.0):
    """The reference's MoveParticles with its InjectIons (oracle/_ref, OpenMP
    over all host threads) on the headline population, a bounded number of
    steps; the reference's Newton step at this size (dense dsysv_ on 32,244
    unknowns, minutes) is timed by the reference arm instead."""
    from oracle import ref
    if not ref.available():
        return None
    cfg = CONFIGS[config]
    threads = ref.max_threads()
    with tempfile.TemporaryDirectory() as wd:
        kd = workloads.write_deck(cfg, wd)
        s, n0 = reference_sim(cfg, wd, kd, POP_SEED)
        s.inject()
        s.move(threads)  # first touch of the population
        psteps, sec, steps = 0.0, 0.0, 0
        while sec < budget_s and steps < 20:
            t0 = time.perf_counter()
            s.inject()
            n_before = s.L.ref_n_particles(s.h)
            s.move(threads)
            sec += time.perf_counter() - t0
            psteps += n_before
            steps += 1
        s.close()
    return {"value": psteps / sec, "unit": "particle-steps/s", "cores": threads, "kind": "reference",
            "sample": f"{steps} InjectIons + MoveParticles steps of the reference on the headline workload's "
                      f"{n0}-ion population ({sec:.1f} s); the Newton step is excluded (the reference arm times it)"}


def reference_arm(args):
    """--impl reference: the reference's own CPU path (oracle/_ref: its
    translation units, OpenMP over the host threads, OpenBLAS dsysv_) on the
    headline workload: W + K steps of InjectIons + MoveParticles on the full
    population, and one Newton step (Lapack) + updateEf as the bounded sample
    of the field solve.  Rank 0 only."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import ref
    if not ref.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libref_oracle.so was not built"}))
        return
    cfg = CONFIGS[args.config]
    threads = ref.max_threads()
    with tempfile.TemporaryDirectory() as wd:
        kd = workloads.write_deck(cfg, wd)
        s, n0 = reference_sim(cfg, wd, kd, POP_SEED)
        push_s, psteps = [], []
        for k in range(args.warmup + args.steps):
            t0 = time.perf_counter()
            s.inject()
            nb = s.L.ref_n_particles(s.h)
            s.move(threads)
            if k >= args.warmup:
                push_s.append(time.perf_counter() - t0)
                psteps.append(nb)
        t0 = time.perf_counter()
        s.compute_phi(ref.LAPACK)
        newton_s = time.perf_counter() - t0
        t0 = time.perf_counter()
        s.update_ef()
        ef_s = time.perf_counter() - t0
        conf = workload_config(cfg, s.n_tets, s.n_nodes, s.neq, n0)
        s.close()
    step_s = float(np.mean(push_s)) + newton_s + ef_s
    value = float(np.mean(psteps)) / step_s
    line = {"metric": METRIC, "value": value, "unit": "particle-steps/s", "impl": "reference",
            "n_gpus": 0, "steps": args.steps, "warmup": args.warmup, "ms_per_step": step_s * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded Kuhn-box ions at steady state; the reference's own injector)",
            "config": conf, "device": f"host CPU, {threads} OpenMP threads (the reference's CPU path)",
            "newton_step_ms": newton_s * 1e3, "push_step_ms": float(np.mean(push_s)) * 1e3,
            "push_particle_steps_per_s": float(np.sum(psteps) / np.sum(push_s)),
            "cpu_baseline": {"value": value, "unit": "particle-steps/s", "cores": threads, "kind": "reference",
                             "sample": f"{args.steps} timed InjectIons + MoveParticles steps on the full population "
                                       f"after {args.warmup} untimed, plus one Lapack Newton step (dsysv_ on "
                                       f"{conf['unknowns']} unknowns) and updateEf; value = mean particles per "
                                       f"step / (mean push step + Newton step + updateEf)"},
            "e2e": {"value": value, "unit": "particle-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


# ---- long runs ----

def run_horizon(args, device, torch):
    """Mixed vs FP64 over a long run of the headline workload: per step the
    density L2 error and the closed-loop potential difference, every 50 steps
    the fraction of particles in different cells."""
    cfg = CONFIGS[args.config]
    wd = tempfile.mkdtemp()
    kd = workloads.write_deck(cfg, wd)
    deck = mp.Deck.load(wd)
    pos, vel, cell = workloads.seed_population(kd, cfg, POP_SEED)
    fe = workloads.fe_arrays(cfg, deck)
    P = deck.params
    ctxs = {}
    for name, form in (("fp64", mp.FP64), ("mixed", mp.MIXED)):
        c = make_context(deck, fe, form, len(cell), device, True, cfg["sphere"] is not None)
        load_population(c, pos, vel, cell, form)
        ctxs[name] = c
    del pos, vel, cell
    inj = {n: mp.Injector(deck.mesh, seed=0) for n in ctxs}
    rows = []
    t_start = time.time()
    for k in range(args.horizon):
        den, uh, n = {}, {}, {}
        for name, c in ctxs.items():
            form = mp.FP64 if name == "fp64" else mp.MIXED
            c.inject_device(inj[name], P.plasma_den, P.ion_velocity, cfg["dt"], cfg["spwt"], SIGMA, QM, 1000, k)
            st = c.push(QM, cfg["dt"], cfg["spwt"])
            c.compute_phi(mp.LAPACK, form)
            c.update_ef()
            den[name], uh[name], n[name] = c.density(), c.field()[1], st.n_after
        row = {"step": k, "density_l2_rel": float(np.linalg.norm(den["mixed"] - den["fp64"]) /
                                                  np.linalg.norm(den["fp64"])),
               "phi_max_abs_V": float(np.abs(uh["mixed"] - uh["fp64"]).max()),
               "n_fp64": n["fp64"], "n_mixed": n["mixed"]}
        if k % 50 == 49 or k == args.horizon - 1:
            ga, gb = ctxs["fp64"].download(mp.ORDER_ID), ctxs["mixed"].download(mp.ORDER_ID)
            ids = np.union1d(ga["id"], gb["id"])
            ia = np.full(ids.size, -1)
            ib = np.full(ids.size, -1)
            ia[np.searchsorted(ids, ga["id"])] = ga["cell"]
            ib[np.searchsorted(ids, gb["id"])] = gb["cell"]
            row["cells_differing_frac"] = float(np.mean(ia != ib))
            del ga, gb
        rows.append(row)
    for c in ctxs.values():
        c.close()
    d = np.array([r["density_l2_rel"] for r in rows])
    ph = np.array([r["phi_max_abs_V"] for r in rows])
    cells = [(r["step"], r["cells_differing_frac"]) for r in rows if "cells_differing_frac" in r]
    print(json.dumps({"horizon": args.horizon, "workload": cfg["label"], "wall_s": time.time() - t_start,
                      "density_l2_rel": {"max": float(d.max()), "median": float(np.median(d)), "last": float(d[-1]),
                                         "per_50": [float(d[i:i + 50].max()) for i in range(0, len(d), 50)]},
                      "phi_closed_loop_max_abs_V": {"max": float(ph.max()), "median": float(np.median(ph)),
                                                    "last": float(ph[-1]),
                                                    "per_50": [float(ph[i:i + 50].max()) for i in range(0, len(ph), 50)]},
                      "cells_differing_frac": cells,
                      "ions_last": {"fp64": rows[-1]["n_fp64"], "mixed": rows[-1]["n_mixed"]}}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", type=int, default=HEADLINE, choices=sorted(CONFIGS),
                    help="workload of the headline step (default: the mixed-precision configuration)")
    ap.add_argument("--legs", default="all", help="secondary legs: all, none, or a comma list of " + ",".join(LEGS))
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline")
    ap.add_argument("--horizon", type=int, default=0, help="run the long mixed-vs-FP64 comparison instead")
    ap.add_argument("--stress", action="store_true", help="run the combined-stress workload instead")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    legs = set(LEGS) if args.legs == "all" else set() if args.legs == "none" else set(args.legs.split(","))
    if args.impl == "reference":
        reference_arm(args)
        return
    import torch
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if args.horizon:
        run_horizon(args, local, torch)
        return
    if args.stress:
        from minipic_b200 import stress
        print(json.dumps(stress.run(args, local, torch, peaks())))
        return
    if world > 1:
        import datetime
        import torch.distributed as dist
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=torch.device("cuda", local))
    pk = peaks()
    flush = torch.empty(FLUSH_BYTES // 4, dtype=torch.float32, device=local)
    h = run_headline(args, local, rank, world, torch, flush, pk)
    extra = {}
    if rank == 0 and world == 1:
        if "kuhn20" in legs or "nonlinear" in legs:
            k20, ctx20, deck20 = run_kuhn20(args, local, torch, flush, pk)
            extra["kuhn20_2M"] = k20
            if "nonlinear" in legs:
                extra["nonlinear_kuhn20"] = run_nonlinear(ctx20, deck20)
                extra["gauss_seidel_kuhn20"] = run_gs_sweeps(ctx20, pk)
            ctx20.close()
        if "adjoint" in legs:
            extra["adjoint_kuhn16_1M_K20"] = run_adjoint(args, local, torch, pk)
        if "sparse64" in legs:
            extra["sparse_field_kuhn64s"] = sparse_field_at_scale(local)
        if "vtk" in legs:
            extra["vtk_output"] = vtk_output_leg(local)
    cpu = cpu_baseline(args.config) if (rank == 0 and world == 1 and not args.no_cpu) else None

    res = h["res"]
    stats = []
    for name in ("mixed", "fp64"):
        r = res[name]
        stats += [float(np.sum(r["n"])), float(np.sum(r["step_ms"]) / 1e3), float(np.mean(r["newton_ms"])),
                  float(np.sum(r["push_ms"]) / 1e3)]
    stats += [float(np.sum(h["e2e"]["n"])), float(np.sum(h["e2e"]["ms"]) / 1e3)]
    if world > 1:
        t = torch.tensor(stats, dtype=torch.float64, device=local)
        tmax, tsum = t.clone(), t.clone()
        torch.distributed.all_reduce(tmax, op=torch.distributed.ReduceOp.MAX)
        torch.distributed.all_reduce(tsum, op=torch.distributed.ReduceOp.SUM)
        tot = [float(tsum[i]) if i in (0, 4, 8) else float(tmax[i]) for i in range(len(stats))]
    else:
        tot = stats
    if rank == 0:
        m_ps, m_s, m_newton, m_push, f_ps, f_s, f_newton, f_push, e_ps, e_s = tot
        cfg, deck = h["cfg"], h["deck"]
        conf = workload_config(cfg, deck.mesh.n_tets, deck.mesh.n_nodes, h["neq"], h["n0"])
        rm, rf = res["mixed"], res["fp64"]
        line = {
            "metric": METRIC, "value": m_ps / m_s, "unit": "particle-steps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": m_s / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64",
            "data": "synthetic (seeded Kuhn-box ions at steady state; device injection with the reference's counts)",
            "config": conf,
            "form": "mixed: FP32 tet-relative particles, FP64 near-face test and density, %s tcgen05 LDL^T "
                    "with FP64 refinement" % ("FP16-operand" if mixed_terms(h["neq"]) == mp.MIXED_FP16 else "3xTF32"),
            "parallelism": f"particles sharded x{world}, density all-reduce, field solve replicated"
            if world > 1 else "1 GPU",
            "l2": f"inputs larger than L2 (the particle arrays); {FLUSH_BYTES >> 20} MiB written between steps",
            "newton_step_ms": m_newton,
            "push_kernel_ms": m_push / args.steps * 1e3,
            "fp64": {"value": f_ps / f_s, "unit": "particle-steps/s", "ms_per_step": f_s / args.steps * 1e3,
                     "newton_step_ms": f_newton, "push_kernel_ms": f_push / args.steps * 1e3,
                     "roofline": h["roofline"]["fp64"]},
            "mixed_over_fp64": (m_ps / m_s) / (f_ps / f_s),
            "errors_vs_fp64": h["errors"],
            "refinement_solves": int(max(rm["refinements"])),
            "absorbed_at_walk_limit_per_step": float(np.mean(rm["lost"])),
            "hops_per_particle_step": float(np.sum(rm["hops"]) / max(np.sum(rm["n"]), 1)),
            "e2e": {"value": e_ps / e_s, "unit": "particle-steps/s",
                    "what": "the mixed whole step through the C ABI: the host injector's ions H2D from host "
                            "memory (velocity rewind on the device), MoveParticles, computePhi, updateEf, node "
                            "density and potential D2H to host memory",
                    "h2d_bytes_per_step": int(h["e2e"]["h2d"]), "d2h_bytes_per_step": int(h["e2e"]["d2h"]),
                    "ms_per_step": e_s / args.steps * 1e3},
            "gpu_launches": int(h["launches"]["mixed"]),
            "gpu_launches_fp64": int(h["launches"]["fp64"]),
            "roofline": h["roofline"]["mixed"],
            "clocks": h["clocks"],
        }
        if "kuhn20_2M" in extra:
            line["roofline_push"] = {"fp64": extra["kuhn20_2M"]["fp64"]["roofline"],
                                     "mixed": extra["kuhn20_2M"]["mixed"]["roofline"],
                                     "workload": "kuhn20_2M (20^3 box, 2M ions, particle IDs off)"}
        line.update(extra)
        if cpu is not None:
            line["cpu_baseline"] = cpu
        print(json.dumps(line))
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
