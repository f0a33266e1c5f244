"""GPU: the C++ drop-in (mini-fem-pic-main_b200/shim/mini_pic_cuda.cpp) driven
with the reference's own objects, compiled against the reference's headers
(oracle/_ref/libref_shim.so: the reference's translation units, the harness
and the drop-in, linked with libminipic_cuda.so).

Two reference simulations start from the same deck: A runs the reference's
CPU path (InjectIons, the MoveParticles kernel body and its erase_if +
normalisation, FESolver::computePhi with the Lapack method, updateEf); B hands
the same kinds of objects to the drop-in's DeviceData, MoveParticles,
computePhiDevice and updateEfDevice.  Each step B gets A's E field and the
same injections (the reference's RNG reseeded per step), so the particle
comparison is open loop (the reference's own closed loop is not stable):
  - particles after MoveParticles: positions, velocities, cells and weights
    bit for bit, in the reference's order;
  - node density within 1e-12 relative;
  - the potential and the E field from the device solve within 1e-9 relative
    of dsysv_'s;
  - after the last step, the drop-in's OutputMeshDevice / OutputParticlesDevice
    files byte for byte those of the reference's OutputMesh / OutputParticles
    on the same simulation's host arrays.
A third simulation runs the drop-in with sparse storage (the Lapack method
becomes the conjugate-gradient Newton step): potential within 1e-9 relative.
The drop-in's MeshGeometryDevice + InletFacesDevice, run on a copy of the
loaded Volume with its geometry cleared, reproduce the reference loaders'
values bit for bit.
"""
from __future__ import annotations

import ctypes
import os
import tempfile

import numpy as np
import pytest

import minipic_b200 as mp
from conftest import GOLDEN
from oracle import ref

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not ref.shim_available(), reason="oracle/_ref/libref_shim.so not built")]

STEPS = 6


def _sims(name):
    deck = os.path.join(GOLDEN, name)
    extra = {}
    sphere = os.path.join(deck, "sphere.dat")
    if os.path.exists(sphere):
        extra = {sphere: (mp.read_surface_dat(sphere)[0], -10.0)}
    a = ref.RefSim(deck, spwt=20000.0, extra_fixed=extra, shim=True)
    b = ref.RefSim(deck, spwt=20000.0, extra_fixed=extra, shim=True)
    b.shim_device()
    return a, b


@pytest.mark.parametrize("name", ["kuhn4", "kuhn4s"])
def test_drop_in_matches_reference_cpu_path(name):
    a, b = _sims(name)
    L = a.L
    try:
        for k in range(STEPS):
            b.set("ef", a.get("ef"))  # open loop: B pushes in A's field
            L.ref_reseed(1000 + k)
            na = a.inject()
            L.ref_reseed(1000 + k)
            nb = b.inject()
            assert na == nb
            a.move(1)
            b.shim_move()
            pa, pb = a.particles(), b.particles()
            assert pa.size == pb.size and pa.size > 0
            for f in ("pos", "vel", "lc", "cell_index"):
                assert np.array_equal(pa[f], pb[f]), (k, f)
            da, db = a.get("den"), b.get("den")
            assert np.abs(da - db).max() <= 1e-12 * np.abs(da).max()
            a.compute_phi(ref.LAPACK)
            b.shim_compute_phi(ref.LAPACK)
            ua, ub = a.get("uh"), b.get("uh")
            assert np.abs(ua - ub).max() <= 1e-9 * np.abs(ua).max(), k
            a.update_ef()
            b.shim_update_ef()
            ea, eb = a.get("ef"), b.get("ef")
            assert np.abs(ea - eb).max() <= 1e-8 * np.abs(ea).max(), k
        with tempfile.TemporaryDirectory() as d1, tempfile.TemporaryDirectory() as d2:
            assert L.ref_shim_output(b.h, b.device, STEPS - 1, d1.encode()) == 0
            assert L.ref_output_mesh(b.h, STEPS - 1, d2.encode()) >= 0
            assert L.ref_output_particles(b.h, d2.encode()) >= 0
            for f in (f"mesh_{STEPS:04d}.vtu", "particles.vtp"):
                with open(os.path.join(d1, f), "rb") as x, open(os.path.join(d2, f), "rb") as y:
                    assert x.read() == y.read(), f
    finally:
        b.close()
        a.close()


@pytest.mark.parametrize("name", ["kuhn4", "kuhn4s"])
def test_drop_in_sparse_storage(name):
    a, b = _sims(name)
    L = a.L
    try:
        L.ref_shim_set_storage(b.device, mp.FE_SPARSE)
        for k in range(3):
            b.set("ef", a.get("ef"))
            L.ref_reseed(1000 + k)
            a.inject()
            L.ref_reseed(1000 + k)
            b.inject()
            a.move(1)
            b.shim_move()
            a.compute_phi(ref.LAPACK)
            b.shim_compute_phi(ref.LAPACK)
            ua, ub = a.get("uh"), b.get("uh")
            assert np.abs(ua - ub).max() <= 1e-9 * np.abs(ua).max(), k
            a.update_ef()
    finally:
        b.close()
        a.close()


@pytest.mark.parametrize("name", ["kuhn4", "kuhn4s"])
def test_drop_in_mesh_setup_on_device(name):
    a, b = _sims(name)
    try:
        _, tets = mp.read_volume_dat(os.path.join(GOLDEN, name, "mesh.dat"))
        con = np.ascontiguousarray(tets, dtype=np.int32)
        assert a.L.ref_shim_mesh_check(a.h, con.ctypes.data_as(ctypes.c_void_p)) == 0
    finally:
        b.close()
        a.close()
