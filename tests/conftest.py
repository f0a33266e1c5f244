"""Shared fixtures.  CPU tests (-m "not gpu") check the oracle against the
committed golden vectors and the reference's own compiled code, the host-side
setup, and that the C ABI library loads and exports every declared symbol.
GPU tests (-m gpu) are the parity tests of the CUDA path through the C ABI."""
from __future__ import annotations

import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "mini-fem-pic-main_b200"))
sys.path.insert(0, ROOT)

import minipic_b200 as mp  # noqa: E402
from minipic_b200 import kuhn  # noqa: E402

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 GPU (B200); calls the CUDA path through the C ABI")


def make_deck(tmp_root, n, sphere=None, **kw):
    d = kuhn.build(n, sphere=sphere)
    path = os.path.join(str(tmp_root), f"kuhn{n}{'s' if sphere else ''}")
    kuhn.write(d, path, **kw)
    return d, path


@pytest.fixture(scope="session")
def deck4(tmp_path_factory):
    return make_deck(tmp_path_factory.mktemp("d4"), 4)


@pytest.fixture(scope="session")
def deck6(tmp_path_factory):
    return make_deck(tmp_path_factory.mktemp("d6"), 6)


@pytest.fixture(scope="session")
def deck8(tmp_path_factory):
    return make_deck(tmp_path_factory.mktemp("d8"), 8)


@pytest.fixture(scope="session")
def deck6s(tmp_path_factory):
    return make_deck(tmp_path_factory.mktemp("d6s"), 6, sphere=(50.0, 50.0, 50.0, 20.0))


def ref_available():
    from oracle import ref
    return ref.available()


def ref_sim(path, kdeck, **kw):
    """The reference's own simulation on a deck (sphere nodes at -10 V)."""
    from oracle import ref
    extra = {}
    if kdeck.sphere_nodes.size:
        extra = {os.path.join(path, "sphere.dat"): (kdeck.sphere_nodes, -10.0)}
    return ref.RefSim(path, extra_fixed=extra, **kw)


def gpu_context(deck: "mp.Deck", sphere_potential=None, fe=True):
    ctx = mp.Context(deck.mesh)
    if fe:
        ctx.fe_setup(**deck.fe_desc_arrays(sphere_potential))
    return ctx


def rel_err(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = max(np.abs(b).max(), 1e-300)
    return float(np.abs(a - b).max() / den)
