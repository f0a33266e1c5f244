"""GPU: the asynchronous VTK writers (mp_output_mesh, mp_output_particles)
against the reference's own OutputMesh and OutputParticles (oracle/_ref), byte
for byte: a reference simulation is advanced a few steps, its potential,
field, density and particles are handed to a device context, and both sides
write their files."""
from __future__ import annotations

import os

import numpy as np
import pytest

from conftest import gpu_context, ref_available, ref_sim
import minipic_b200 as mp

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built")]


def _advanced(path, kd, steps=5, spwt=2000.0):
    s = ref_sim(path, kd, spwt=spwt)
    for _ in range(steps):
        s.inject()
        s.move(1)
        s.compute_phi(2)
        s.update_ef()
    return s


def _read(p):
    with open(p, "rb") as f:
        return f.read()


@pytest.mark.parametrize("which", ["deck6", "deck6s"])
def test_output_mesh_matches_reference_bytes(which, request, tmp_path):
    kd, path = request.getfixturevalue(which)
    dk = mp.Deck.load(path)
    s = _advanced(path, kd)
    ctx = gpu_context(dk, sphere_potential=-10.0)
    ctx.fe_set("uh", s.get("uh"))
    ctx.fe_set("ef", s.get("ef"))
    ctx.fe_set("den", s.get("den"))
    _, types, _ = s.nodes()
    a, b = tmp_path / "ours", tmp_path / "ref"
    a.mkdir()
    b.mkdir()
    for ts in (9, 123):
        ctx.output_mesh(ts, str(a), types)
        assert s.L.ref_output_mesh(s.h, ts, str(b).encode()) >= 0
    ctx.output_wait()
    for name in ("mesh_0010.vtu", "mesh_0124.vtu"):
        ours, ref = _read(a / name), _read(b / name)
        assert len(ours) > 10_000
        assert ours == ref, name


def test_output_particles_match_reference_bytes(deck6s, tmp_path):
    kd, path = deck6s
    dk = mp.Deck.load(path)
    s = _advanced(path, kd, spwt=20.0)
    parts = s.particles()
    assert parts.size > 1000
    ctx = gpu_context(dk, sphere_potential=-10.0)
    ctx.append(parts["pos"], parts["vel"], parts["cell_index"])
    ctx.output_particles(str(tmp_path / "particles.vtp"))
    ctx.output_wait()
    (tmp_path / "ref").mkdir()
    assert s.L.ref_output_particles(s.h, str(tmp_path / "ref").encode()) >= 0
    assert _read(tmp_path / "particles.vtp") == _read(tmp_path / "ref" / "particles.vtp")


def test_output_errors_and_overlap(deck4, tmp_path):
    kd, path = deck4
    dk = mp.Deck.load(path)
    ctx = gpu_context(dk)
    types = dk.mesh.node_type
    with pytest.raises(mp.MpError) as e:
        ctx.output_mesh(0, str(tmp_path / "no" / "such" / "dir"), types)
    assert e.value.status == 1
    # back-to-back calls: each joins the previous writer; the files are complete
    for ts in range(4):
        ctx.output_mesh(ts, str(tmp_path), types)
    ctx.output_wait()
    for ts in range(4):
        text = _read(tmp_path / f"mesh_{ts + 1:04d}.vtu")
        assert text.endswith(b"</VTKFile>\n")
    ctx.output_mesh(7, str(tmp_path), types)
    ctx.close()  # joins the running writer
    assert _read(tmp_path / "mesh_0008.vtu").endswith(b"</VTKFile>\n")
