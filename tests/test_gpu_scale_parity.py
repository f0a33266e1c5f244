"""GPU parity at the sizes the benchmarks run, against the reference's own
compiled code (oracle/_ref):

* the dense LDL^T solve (FP64, and the mixed form's FP32 factor with FP64
  refinement) past one 1,024-column super-panel, where the factorization
  switches to its two-level structure (trailing update per super-panel, strip
  updates, ready words over many blocks): the 12^3 Kuhn box (1,859 unknowns)
  and the 20^3 box of the FP64 throughput workload (8,379 unknowns), against
  dsysv_ (solveLinearLapack, src/FESolver.cpp:528-558), the mixed form in each
  of its factor arithmetics (TF32, FP16 operands, 3xTF32).  Bar: y within 1e-9
  relative, a whole computePhi step's potential within 1e-9 relative (FP64)
  and within 1e-8 V (mixed);
* MoveParticles on the 20^3 box with 2M seeded ions (0.2 hops per
  particle-step, tet re-sort every 2 steps), open loop in the reference's field
  (src/mini-pic.cpp:287-319): cells, positions, velocities and weights
  bit-identical, density within 1e-12;
* the 8^3 box at its configuration (spwt 200, dt 1e-7) for 200 steps from an
  empty domain, open loop, checked every 10 steps;
* the Gauss-Seidel solve (solveLinear, src/FESolver.cpp:561-601) on the 12^3
  box (30 row blocks: the fused multi-sweep kernel's wavefront and the
  transposed row-band reads), against the reference's: y within 1e-7;
* the NonLinear method (solveNonLinear, src/FESolver.cpp:324-364) per step on
  states captured from the reference's own run: where the reference converges,
  the same Newton iteration count and d within the Gauss-Seidel tolerance;
  where it exits with "NR failed to converge", MP_ERR_NOT_CONVERGED with the
  same number of Gauss-Seidel solves that ran out of sweeps."""
from __future__ import annotations

import ctypes as C
import re

import numpy as np
import pytest

from conftest import gpu_context, make_deck, ref_available, ref_sim, rel_err, run_open_loop
import minipic_b200 as mp
from minipic_b200 import kuhn, workloads

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built")]


@pytest.mark.parametrize("n", [12, 20], ids=["kuhn12_1859", "kuhn20_8379"])
def test_ldlt_past_one_superpanel_vs_dsysv(tmp_path, n):
    kd, path = make_deck(tmp_path, n, dt=5e-8)
    dk = mp.Deck.load(path)
    s = ref_sim(path, kd, spwt=5.0)
    neq = s.neq
    assert neq > 1024
    rng = np.random.default_rng(n)
    den = dk.params.plasma_den * (1.0 + 0.1 * rng.standard_normal(dk.mesh.n_nodes))
    d0 = rng.normal(0.0, 0.05, neq)  # a Newton state away from zero
    zero = np.zeros(neq)
    # one linear solve J y = G
    s.set("d", d0)
    s.set("F1", zero)
    s.build_f1(den)
    G = s.residual()
    s.build_j(mp.LAPACK)
    y_ref = s.solve_lapack(G)
    # one whole computePhi step (Lapack method) from the same state
    s.set("d", d0)
    s.set("F1", zero)
    s.set("den", den)
    s.compute_phi(mp.LAPACK)
    uh_ref = s.get("uh")
    ctx = gpu_context(dk)
    assert ctx.neq == neq
    # the mixed form in each tensor-core arithmetic of its factorization
    for form, mf in ((mp.FP64, mp.MIXED_AUTO), (mp.MIXED, mp.MIXED_AUTO), (mp.MIXED, mp.MIXED_TF32),
                     (mp.MIXED, mp.MIXED_FP16), (mp.MIXED, mp.MIXED_TF32X3)):
        ctx.set_mixed_factor(mf)
        ctx.fe_set("d", d0)
        ctx.fe_set("F1", zero)
        ctx.build_f1(den)
        ctx.build_j(mp.LAPACK)
        st = ctx.solve_linear(mp.LAPACK, form, b=G)
        y = ctx.fe_get("y")
        assert rel_err(y, y_ref) < 1e-9, (form, mf, rel_err(y, y_ref))
        assert st.linear_residual < 1e-12 * max(1.0, np.abs(G).max())
        ctx.fe_set("d", d0)
        ctx.fe_set("F1", zero)
        ctx.compute_phi(mp.LAPACK, form, ion_den=den)
        _, uh, _ = ctx.field()
        if form == mp.FP64:
            assert rel_err(uh, uh_ref) < 1e-9
        else:
            assert np.abs(uh - uh_ref).max() < 1e-8


def test_gauss_seidel_many_blocks_vs_reference(tmp_path):
    kd, path = make_deck(tmp_path, 12, dt=5e-8)
    dk = mp.Deck.load(path)
    s = ref_sim(path, kd, spwt=5.0)
    rng = np.random.default_rng(7)
    den = dk.params.plasma_den * (1.0 + 0.1 * rng.standard_normal(dk.mesh.n_nodes))
    d0 = rng.normal(0.0, 0.05, s.neq)
    zero = np.zeros(s.neq)
    s.set("d", d0)
    s.set("F1", zero)
    s.build_f1(den)
    G = s.residual()
    s.build_j(1)
    y_ref = s.solve_gs(G)
    ctx = gpu_context(dk)
    ctx.fe_set("d", d0)
    ctx.fe_set("F1", zero)
    ctx.build_f1(den)
    ctx.build_j(1)
    st = ctx.solve_linear(mp.GAUSS_SEIDEL, mp.FP64, b=G)
    assert st.linear_failures == 0
    assert rel_err(ctx.fe_get("y"), y_ref) < 1e-7


def test_push_kuhn20_2M_open_loop_vs_reference(tmp_path):
    """The FP64 throughput workload's mesh and population: 20^3 Kuhn box, 2M
    ions at steady state (drift + 0.1 eV Maxwellian), spwt 5, dt 5e-8, tet
    re-sort before the first step and every 2 steps, 3 steps."""
    from oracle import ref
    cfg = workloads.CONFIGS[1]
    kd, deck, pos, vel, cell = workloads.make_workload(cfg, str(tmp_path), seed=1234)
    assert len(cell) > 1_900_000
    worst, s, ctx = run_open_loop(str(tmp_path), kd, steps=3, spwt=cfg["spwt"], sort_period=2,
                                  initial=(pos, vel, cell), threads=ref.max_threads(), sort_first=True)
    assert worst < 1e-12


def test_push_kuhn8_200_steps_open_loop_vs_reference(tmp_path):
    """The small FP64 configuration as the reference runs it: 8^3 Kuhn box,
    spwt 200, dt 1e-7, 200 steps from an empty domain (about 40k ions at the
    peak), the reference's Lapack step between pushes."""
    kd, path = make_deck(tmp_path, 8, dt=1e-7)
    worst, s, ctx = run_open_loop(path, kd, steps=200, spwt=200.0, check_every=10)
    assert worst < 1e-12
    assert len(s.particles()) > 5000


def _ref_messages(log: str):
    conv = re.findall(r"NR converged in (\d+) iterations with L2=(\S+)", log)
    fail = re.findall(r"NR failed to converge, L2 = (\S+)", log)
    gs_fail = len(re.findall(r"GS failed to converge", log))
    return conv, fail, gs_fail


def test_nonlinear_per_step_on_captured_states(tmp_path):
    """States (d, F1, ion density) captured before computePhi at steps of the
    reference's own Lapack run on the 8^3 box (spwt 200, dt 1e-7); the NonLinear
    method from each, in the reference (in a child process: it exits on
    failure) and on the device."""
    from oracle import ref
    kd, path = make_deck(tmp_path, 8, dt=1e-7)
    dk = mp.Deck.load(path)
    s = ref_sim(path, kd, spwt=200.0)
    capture = (3, 60, 130, 145, 160, 180)
    states = {}
    for ts in range(max(capture) + 1):
        s.inject()
        s.move(0)
        if ts in capture:
            states[ts] = (s.get("d"), s.get("F1"), s.get("den"))
        s.compute_phi(mp.LAPACK)
        s.update_ef()
    ctx = gpu_context(dk)
    L = mp.lib()
    outcomes = []
    for ts, (d, F1, den) in states.items():
        r = ref.compute_phi_isolated(path, ref.NONLINEAR, d, F1, den, spwt=200.0)
        conv, fail, gs_fail = _ref_messages(r["log"])
        ctx.fe_set("d", d)
        ctx.fe_set("F1", F1)
        st = mp.NewtonStats()
        den_c = np.ascontiguousarray(den)
        rc = L.mp_compute_phi(ctx.h, mp._p(den_c), mp.NONLINEAR, mp.FP64, C.byref(st))
        assert st.linear_failures == gs_fail, (ts, st.linear_failures, gs_fail)
        if r["exitcode"] == 0:
            assert conv and rc == 0, (ts, rc)
            assert st.newton_iterations == int(conv[0][0])
            dd, uh, _ = ctx.field()
            assert rel_err(dd, r["d"]) < 1e-7, (ts, rel_err(dd, r["d"]))
            assert rel_err(uh, r["uh"]) < 1e-7
            outcomes.append("converged")
        else:
            assert fail and rc == 5, (ts, rc)  # MP_ERR_NOT_CONVERGED
            assert st.newton_iterations == 10
            assert abs(st.l2 - float(fail[0])) <= 1e-2 * float(fail[0])
            outcomes.append("failed")
    # the captured steps cover both outcomes of the reference
    assert "converged" in outcomes and "failed" in outcomes
