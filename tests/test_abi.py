"""CPU: the C ABI library loads and exports every entry point that
include/minipic_cuda.h declares; host-only entry points validate arguments;
without a GPU, context creation fails loudly (no CPU fallback)."""
from __future__ import annotations

import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT
import minipic_b200 as mp


def declared_symbols():
    names = set()
    inc = os.path.join(ROOT, "include")
    for f in os.listdir(inc):
        if f.endswith(".h"):
            text = open(os.path.join(inc, f)).read()
            names |= set(re.findall(r"^\s*(?:int|const char \*|void)\s*\*?\s*(mp_\w+)\s*\(", text, re.M))
    return names


def test_header_and_binding_agree():
    assert declared_symbols() == set(mp.EXPORTED)


def header_constants():
    """Every MP_* constant the header defines, by enum entry or #define."""
    text = open(os.path.join(ROOT, "include", "minipic_cuda.h")).read()
    vals = {k: int(v) for k, v in re.findall(r"\b(MP_\w+)\s*=\s*(-?\d+)", text)}
    vals.update({k: int(v) for k, v in re.findall(r"^#define\s+(MP_\w+)\s+(-?\d+)\s*$", text, re.M)})
    return vals


def test_python_constants_mirror_the_header():
    h = header_constants()
    # names the Python package spells the same way without the MP_ prefix
    same = {k[3:]: v for k, v in h.items() if hasattr(mp, k[3:])}
    for name in ("MIXED_AUTO", "MIXED_TF32", "MIXED_FP16", "MIXED_TF32X3", "MIXED_FP16_FROM",
                 "ORDER_STORAGE", "ORDER_ID", "WALK_LIMIT_ERROR", "WALK_LIMIT_ABSORB", "KT_PUSH", "KT_UPDATE"):
        assert name in same, name
    for name, v in same.items():
        assert getattr(mp, name) == v, (name, getattr(mp, name), v)
    # the forms and storage the package names differently
    assert (mp.FP64, mp.MIXED) == (h["MP_FORM_FP64"], h["MP_FORM_MIXED"])
    assert (mp.FE_DENSE, mp.FE_SPARSE) == (h["MP_FE_STORAGE_DENSE"], h["MP_FE_STORAGE_SPARSE"])


def test_mixed_factor_arguments_checked():
    L = mp.lib()
    for mode in (mp.MIXED_AUTO, mp.MIXED_TF32, mp.MIXED_FP16, mp.MIXED_TF32X3, 4, -1):
        assert L.mp_set_mixed_factor(None, mode) == 1  # MP_ERR_ARG: no context


def test_library_exports_every_declared_symbol():
    L = mp.lib()
    for name in declared_symbols():
        assert hasattr(L, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", mp.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (mp_\w+)", out))
    assert declared_symbols() <= exported


def test_error_strings():
    L = mp.lib()
    for code in range(11):
        assert L.mp_error_string(code)
    assert L.mp_version() >= 10000


def test_null_arguments_rejected():
    L = mp.lib()
    assert L.mp_create(0, None, None) == 1  # MP_ERR_ARG
    assert L.mp_push_scatter(None, 1.0, 1.0, 1.0, None, None) == 1
    assert L.mp_compute_phi(None, None, 0, 0, None) == 1


def test_no_cpu_fallback_without_device():
    """On a machine without an sm_100 device, mp_create must fail loudly."""
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    dk = mp.Deck.load(os.path.join(ROOT, "tests", "golden", "kuhn4"))
    with pytest.raises(mp.MpError) as e:
        mp.Context(dk.mesh)
    assert e.value.status == 8  # MP_ERR_NO_DEVICE


def test_mesh_geometry_rejects_bad_connectivity():
    L = mp.lib()
    pos = np.zeros((4, 3))
    con = np.array([[0, 1, 2, 7]], dtype=np.int32)  # node 7 does not exist
    out = [np.zeros(1), np.zeros(4), np.zeros(4), np.zeros(4), np.zeros(4), np.zeros(4, dtype=np.int32),
           np.zeros(4), np.zeros(4, dtype=np.int32)]
    rc = L.mp_mesh_geometry(4, pos.ctypes.data_as(C.c_void_p), 1, con.ctypes.data_as(C.c_void_p),
                            *[o.ctypes.data_as(C.c_void_p) for o in out])
    assert rc == 1


def test_inlet_face_without_tet_rejected():
    """The reference exits when an inlet face has no owning tet (meshes.cpp:323-326)."""
    dk = mp.Deck.load(os.path.join(ROOT, "tests", "golden", "kuhn4"))
    m = dk.mesh
    bad = np.array([[0, 1, 50]], dtype=np.int32)
    with pytest.raises(mp.MpError):
        mp.Mesh.build(m.node_pos, m.con, [], bad, [])


def test_injector_capacity_checked():
    dk = mp.Deck.load(os.path.join(ROOT, "tests", "golden", "kuhn4"))
    inj = mp.Injector(dk.mesh)
    L = mp.lib()
    n = C.c_int64()
    pos, vel = np.zeros((1, 3)), np.zeros((1, 3))
    cell = np.zeros(1, dtype=np.int32)
    rc = L.mp_injector_sample(inj.h, 1e10, 7000.0, 2e-6, 20000.0, 1, pos.ctypes.data_as(C.c_void_p), 24,
                              vel.ctypes.data_as(C.c_void_p), 24, cell.ctypes.data_as(C.c_void_p), 4, C.byref(n))
    assert rc == 1


def test_drop_in_harness_links():
    """The C++ drop-in compiled against the reference's headers links with the
    library and exports its entry points (no device needed to load it)."""
    from oracle import ref
    if not ref.shim_available():
        pytest.skip("oracle/_ref/libref_shim.so not built (needs the reference sources)")
    L = ref.lib(shim=True)
    for name in ("ref_shim_device", "ref_shim_move", "ref_shim_compute_phi", "ref_shim_update_ef"):
        assert getattr(L, name)
