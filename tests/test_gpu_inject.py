"""GPU: InjectIons on the device (mp_inject_device), against the host injector
(the reference's InjectIons restated with its mt19937 stream).

  - per-step counts equal the host injector's, and so does the shared
    remainder it carries across faces and steps;
  - every particle lies on an inlet triangle (the x = 0 plane of the Kuhn box)
    inside the face's tet (barycentric weights in [0, 1]);
  - velocities: normal*ion_velocity plus the Maxwellian thermal part, mean and
    standard deviation per component within 5 standard errors;
  - the same seed and step give the same particles; another step gives others.
"""
from __future__ import annotations

import os

import numpy as np
import pytest

import minipic_b200 as mp
from conftest import GOLDEN, gpu_context

pytestmark = pytest.mark.gpu

DEN, VD, DT, SPWT = 1e10, 7000.0, 1e-7, 0.01
SIGMA = 776.0
QM = mp.QE / (16 * mp.AMU)


def _deck():
    return mp.Deck.load(os.path.join(GOLDEN, "kuhn4"))


def test_counts_and_remainder_match_host_injector():
    dk = _deck()
    ctx = gpu_context(dk, fe=False)
    host, dev = mp.Injector(dk.mesh, seed=0), mp.Injector(dk.mesh, seed=0)
    total = 0
    for step in range(6):
        p, _, _ = host.sample(DEN, VD, DT, SPWT)
        n = ctx.inject_device(dev, DEN, VD, DT, SPWT, SIGMA, QM, 1234, step)
        assert n == len(p) and n > 1000
        assert dev.rem == host.rem
        total += n
    assert ctx.count() == total


def test_positions_on_inlet_faces_and_velocity_statistics():
    dk = _deck()
    ctx = gpu_context(dk, fe=False)
    inj = mp.Injector(dk.mesh, seed=0)
    for step in range(10):
        ctx.inject_device(inj, DEN, VD, DT, SPWT, SIGMA, QM, 99, step)
    out = ctx.download(mp.ORDER_ID)
    pos, vel, lc, cell = out["pos"], out["vel"], out["lc"], out["cell"]
    n = len(cell)
    assert n > 50_000
    assert np.all(pos[:, 0] == 0.0)  # the inlet plane
    assert np.all((pos[:, 1:] >= 0) & (pos[:, 1:] <= 0.1))
    assert np.all(np.isin(cell, dk.mesh.inlet_cell))
    assert lc.min() >= -1e-12 and lc.max() <= 1 + 1e-12  # inside the face's tet
    se = SIGMA / np.sqrt(n)
    mean = vel.mean(axis=0)
    assert abs(mean[0] - VD) < 5 * se and abs(mean[1]) < 5 * se and abs(mean[2]) < 5 * se
    std = vel.std(axis=0)
    assert np.all(np.abs(std - SIGMA) < 5 * SIGMA / np.sqrt(2 * n))
    # uniform on the triangles: the inlet's y and z are uniform on [0, 0.1]
    for d in (1, 2):
        h, _ = np.histogram(pos[:, d], bins=10, range=(0, 0.1))
        assert np.all(np.abs(h - n / 10) < 6 * np.sqrt(n / 10))


def test_reproducible_for_seed_and_step():
    dk = _deck()
    a, b = gpu_context(dk, fe=False), gpu_context(dk, fe=False)
    ia, ib = mp.Injector(dk.mesh, seed=0), mp.Injector(dk.mesh, seed=0)
    a.inject_device(ia, DEN, VD, DT, SPWT, SIGMA, QM, 7, 3)
    b.inject_device(ib, DEN, VD, DT, SPWT, SIGMA, QM, 7, 3)
    pa, pb = a.download(mp.ORDER_ID), b.download(mp.ORDER_ID)
    assert np.array_equal(pa["pos"], pb["pos"]) and np.array_equal(pa["vel"], pb["vel"])
    c = gpu_context(dk, fe=False)
    c.inject_device(mp.Injector(dk.mesh, seed=0), DEN, VD, DT, SPWT, SIGMA, QM, 7, 4)
    assert not np.array_equal(c.download(mp.ORDER_ID)["pos"], pa["pos"])
