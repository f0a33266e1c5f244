"""GPU: the adjoint of K push + scatter steps (mp_adjoint_*) through the C ABI.

Checks, against the dual-number build of the reference push (oracle/dual.cpp,
itself pinned bit for bit to the reference's MoveParticles by the CPU tests):
  - the forward's density, flux and exit counts;
  - the tangent (JVP) in phi and in the inlet drift velocity;
  - the reverse (VJP): <gbar, J u> + Fbar dF == <phibar, u> + vdbar dvd;
  - checkpoint intervals 1, 3 and K give the same reverse;
and, at the adjoint workload's size (16^3 Kuhn mesh, ~1M ions, K = 20,
checkpoints every 5), the reverse against central finite differences
(h = 1e-4 relative) on 64 random phi directions and on v_drift, with the walk
pinned to the forward's recorded cells (the piecewise-fixed model itself) and
with the free walk in the directions where no particle's path changed; plus
torch.autograd.gradcheck through the autograd wrapper.
"""
from __future__ import annotations

import tempfile

import numpy as np
import pytest

import minipic_b200 as mp
from minipic_b200 import adjoint, workloads
from oracle import port

pytestmark = pytest.mark.gpu

MASS = 16 * mp.AMU
SMALL = dict(n=4, n_ions=4000, dt=1e-7, spwt=100.0, sphere=None, label="kuhn4_adjoint")


class Case:
    def __init__(self, cfg, steps, ckpt, n_ions=None, seed=5, record=False):
        self.wd = tempfile.TemporaryDirectory()
        self.cfg = cfg
        self.deck, self.slots, self.K = workloads.make_adjoint_case(cfg, self.wd.name, seed, n_ions=n_ions,
                                                                     steps=steps)
        m = self.deck.mesh
        self.m = m
        self.nx = self.deck.fe_desc_arrays()["nx"]
        self.wall = adjoint.wall_nodes_of(m)
        self.dir = m.inlet_normal[0]
        self.qm = mp.QE / MASS
        self.phi = workloads.adjoint_phi(m)
        self.vd = self.deck.params.ion_velocity
        self.ctx = mp.Context(m)
        self.adj = self.make(ckpt, record)

    def make(self, ckpt, record=False):
        a = adjoint.Adjoint(self.ctx, self.K, ckpt, self.qm, MASS, self.cfg["dt"], self.cfg["spwt"], self.dir,
                            self.wall, nx=self.nx, record_path=record)
        workloads.load_adjoint(a, self.slots)
        return a

    def dual(self, phi=None, vd=None, dphi=None, dvd=0.0):
        return port.dual_ksteps(self.m, self.nx, self.wall, self.slots, self.K, self.qm, MASS, self.cfg["dt"],
                                self.cfg["spwt"], self.dir, self.phi if phi is None else phi,
                                self.vd if vd is None else vd, dphi=dphi, dvd=dvd)

    def close(self):
        self.ctx.close()
        self.wd.cleanup()


@pytest.fixture(scope="module")
def small():
    c = Case(SMALL, steps=8, ckpt=3)
    yield c
    c.close()


def test_forward_matches_dual_oracle(small):
    den, st = small.adj.forward(small.phi, small.vd)
    ref = small.dual()
    assert st.slots == small.slots["cell"].size
    assert st.alive == int((ref["kind"] == 0).sum())
    assert st.wall_exits == int((ref["kind"] == 1).sum()) and st.wall_exits > 0
    assert st.other_exits == int((ref["kind"] == 2).sum())
    assert np.abs(den - ref["den"]).max() <= 1e-12 * np.abs(ref["den"]).max()
    assert abs(st.flux - ref["flux"]) <= 1e-12 * abs(ref["flux"])


def test_tangent_matches_dual_oracle(small):
    small.adj.forward(small.phi, small.vd)
    rng = np.random.default_rng(1)
    for _ in range(3):
        u = rng.normal(size=small.m.n_nodes)
        dvd = float(rng.normal()) * 100.0
        dden, dflux = small.adj.tangent(u, dvd)
        ref = small.dual(dphi=u, dvd=dvd)
        assert np.abs(dden - ref["dden"]).max() <= 1e-10 * np.abs(ref["dden"]).max()
        assert abs(dflux - ref["dflux"]) <= 1e-10 * abs(ref["dflux"])


def test_reverse_is_the_transpose_of_the_tangent(small):
    small.adj.forward(small.phi, small.vd)
    rng = np.random.default_rng(2)
    gbar = rng.normal(size=small.m.n_nodes)
    fbar = float(rng.normal()) * 1e24  # the flux is O(1e-14) J: scale its weight to the density's
    phibar, vdbar = small.adj.backward(gbar, fbar)
    for _ in range(4):
        u = rng.normal(size=small.m.n_nodes)
        dvd = float(rng.normal()) * 100.0
        ref = small.dual(dphi=u, dvd=dvd)
        lhs = float(gbar @ ref["dden"] + fbar * ref["dflux"])
        rhs = float(phibar @ u + vdbar * dvd)
        scale = float(np.abs(gbar) @ np.abs(ref["dden"]) + abs(fbar * ref["dflux"]))
        assert abs(lhs - rhs) <= 1e-10 * scale


def test_checkpoint_intervals_agree(small):
    rng = np.random.default_rng(4)
    gbar = rng.normal(size=small.m.n_nodes)
    fbar = 1e24
    out = []
    for ck in (1, 3, small.K):
        a = small.make(ck)
        a.forward(small.phi, small.vd)
        out.append(a.backward(gbar, fbar))
    for pb, vb in out[1:]:
        assert np.abs(pb - out[0][0]).max() <= 1e-12 * np.abs(out[0][0]).max()
        assert abs(vb - out[0][1]) <= 1e-12 * abs(out[0][1])


def test_autograd_gradcheck():
    torch = pytest.importorskip("torch")
    c = Case(dict(n=3, n_ions=400, dt=1e-7, spwt=100.0, sphere=None, label="kuhn3"), steps=5, ckpt=2, record=True)
    try:
        c.adj.forward(c.phi, c.vd)  # walk once: records the path the pinned calls replay
        fn = adjoint.push_scatter_function()
        dev = torch.device("cuda", 0)

        def f(phi, vd):
            den, flux = fn.apply(phi, vd, c.adj, adjoint.PINNED)
            return den * 1e-8, flux * 1e14  # O(1) outputs

        phi = torch.tensor(c.phi, dtype=torch.float64, device=dev, requires_grad=True)
        vd = torch.tensor(c.vd, dtype=torch.float64, device=dev, requires_grad=True)
        # FP64 atomics make repeated backward passes differ in the last bits
        assert torch.autograd.gradcheck(f, (phi, vd), eps=1e-4, atol=1e-7, rtol=1e-6, nondet_tol=1e-10)
    finally:
        c.close()


@pytest.fixture(scope="module")
def adjoint_workload():
    cfg = workloads.CONFIGS[3]
    c = Case(cfg, steps=cfg["adjoint_steps"], ckpt=cfg["checkpoint_every"], seed=9, record=True)
    yield c
    c.close()


def test_reverse_against_central_differences_at_adjoint_size(adjoint_workload):
    c = adjoint_workload
    den0, st = c.adj.forward(c.phi, c.vd)  # walked: records the path
    assert st.slots > 1_000_000 and st.wall_exits > 0
    rng = np.random.default_rng(7)
    gbar = rng.normal(size=c.m.n_nodes)
    fbar = 1e24
    phibar, vdbar = c.adj.backward(gbar, fbar)

    def S(phi, vd, mode):
        den, s = c.adj.forward(phi, vd, mode)
        return float(gbar @ den + fbar * s.flux), s

    hp = 1e-4 * np.abs(c.phi).max()
    free_ok = 0
    for _ in range(64):
        u = rng.normal(size=c.m.n_nodes)
        u /= np.abs(u).max()
        sp, _ = S(c.phi + hp * u, c.vd, adjoint.PINNED)
        sm, _ = S(c.phi - hp * u, c.vd, adjoint.PINNED)
        fd = (sp - sm) / (2 * hp)
        ad = float(phibar @ u)
        assert abs(fd - ad) <= 1e-6 * abs(ad)
    # v_drift, h = 1e-4 relative
    hv = 1e-4 * c.vd
    sp, _ = S(c.phi, c.vd + hv, adjoint.PINNED)
    sm, _ = S(c.phi, c.vd - hv, adjoint.PINNED)
    assert abs((sp - sm) / (2 * hv) - vdbar) <= 1e-6 * abs(vdbar)
    # free walk: where no path changed the derivative is the same
    for _ in range(8):
        u = rng.normal(size=c.m.n_nodes)
        u /= np.abs(u).max()
        sp, a = S(c.phi + hp * u, c.vd, adjoint.WALK)
        sm, b = S(c.phi - hp * u, c.vd, adjoint.WALK)
        if (a.alive, a.wall_exits, b.alive, b.wall_exits) != (st.alive, st.wall_exits, st.alive, st.wall_exits):
            continue
        fd = (sp - sm) / (2 * hp)
        if abs(fd - float(phibar @ u)) <= 1e-6 * abs(float(phibar @ u)):
            free_ok += 1
    c.adj.forward(c.phi, c.vd)  # restore the walked tape
    print(f"free-walk central differences within 1e-6: {free_ok}/8 directions")
