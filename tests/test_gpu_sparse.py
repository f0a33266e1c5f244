"""GPU: the sparse field solve through the C ABI, against the reference's own
compiled FESolver (oracle/_ref) and the dense device solvers.

- The sparse K equals the reference's K (src/FESolver.cpp:434-485) entry for
  entry, bit for bit, in both storages (gathered from the dense K, or
  assembled straight into the sliced layout), and so does F0.
- G = K d - F0 - F1 from the sparse product equals the reference's
  matVecMultiply + vecVecSubtract bit for bit (the dense sum in column order
  with its zero products left out).
- SPARSE_CG (the Lapack method's Newton step, J y = G by Jacobi-preconditioned
  conjugate gradients in FP64 to ||r|| <= 1e-12 ||G||): y within 1e-9
  relative of dsysv_'s, whole computePhi steps within 1e-9 relative in d and
  uh (about 1e-10 V).
- SPARSE_NEWTON (the NonLinear loop with conjugate-gradient inner solves):
  the same Newton iterations and potential within 1e-8 V as the dense loop
  with refined LDL^T inner solves (the reference's loop, with Gauss-Seidel
  inner solves stopped at ||r||/neq < 1e-4, is 2e-3 relative away).
- At 108,226 unknowns (a 48^3 Kuhn mesh around a sphere; the dense K and J
  would take 94 GB each) in sparse storage: linearity and symmetry of the
  solve, and J y - G consistent with J = K - diag(FP) for one diagonal.
"""
from __future__ import annotations

import tempfile

import numpy as np
import pytest

from conftest import gpu_context, ref_available, ref_sim, rel_err
import minipic_b200 as mp
from minipic_b200 import kuhn

pytestmark = pytest.mark.gpu
needs_ref = pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built")


def sparse_context(dk, sphere_potential=-10.0):
    ctx = mp.Context(dk.mesh)
    ctx.set_fe_storage(mp.FE_SPARSE)
    ctx.fe_setup(**dk.fe_desc_arrays(sphere_potential))
    return ctx


def csr_to_dense(row_ptr, col, val, n):
    A = np.zeros((n, n))
    rows = np.repeat(np.arange(n), np.diff(row_ptr))
    A[rows, col] = val
    return A


def advanced(path, kd, steps=8, spwt=2000.0):
    s = ref_sim(path, kd, spwt=spwt)
    for _ in range(steps):
        s.inject()
        s.move(1)
        s.compute_phi(2)
        s.update_ef()
    return s


@needs_ref
@pytest.mark.parametrize("which", ["deck6", "deck6s"])
def test_sparse_k_bitexact(which, request):
    kd, path = request.getfixturevalue(which)
    dk = mp.Deck.load(path)
    s = ref_sim(path, kd)
    Kref = s.matrix(0)
    n = Kref.shape[0]
    dense = gpu_context(dk, sphere_potential=-10.0)
    sparse = sparse_context(dk)
    rp, col, val = dense.fe_sparse_matrix()
    assert np.all(np.diff(rp) > 0) and all(np.all(np.diff(col[rp[i]:rp[i + 1]]) > 0) for i in range(n))
    assert np.array_equal(csr_to_dense(rp, col, val, n), Kref)
    rp2, col2, val2 = sparse.fe_sparse_matrix()
    assert np.array_equal(rp2, rp) and np.array_equal(col2, col) and np.array_equal(val2, val)
    assert np.array_equal(sparse.fe_get("F0"), s.get("F0"))
    assert rp[-1] < 20 * n  # about 15 nonzeros a row


@needs_ref
@pytest.mark.parametrize("which", ["deck6", "deck6s"])
def test_sparse_residual_bitexact(which, request):
    kd, path = request.getfixturevalue(which)
    dk = mp.Deck.load(path)
    s = advanced(path, kd)
    s.build_f1(s.get("den"))
    G = s.residual()
    for ctx in (gpu_context(dk, sphere_potential=-10.0), sparse_context(dk)):
        ctx.fe_set("d", s.get("d"))
        ctx.fe_set("F1", s.get("F1"))
        ctx.residual()
        assert np.array_equal(ctx.fe_get("G"), G)


@needs_ref
@pytest.mark.parametrize("which", ["deck6", "deck6s"])
def test_sparse_cg_vs_dsysv(which, request):
    kd, path = request.getfixturevalue(which)
    dk = mp.Deck.load(path)
    s = advanced(path, kd)
    s.build_f1(s.get("den"))
    G = s.residual()
    s.build_j(2)
    y_ref = s.solve_lapack(G)
    for ctx in (gpu_context(dk, sphere_potential=-10.0), sparse_context(dk)):
        ctx.fe_set("d", s.get("d"))
        ctx.build_j(mp.SPARSE_CG)
        st = ctx.solve_linear(mp.SPARSE_CG, mp.FP64, b=G)
        y = ctx.fe_get("y")
        assert rel_err(y, y_ref) < 1e-9
        assert st.linear_iterations > 0
        assert st.linear_residual * ctx.neq <= 1.01e-12 * np.linalg.norm(G)


@needs_ref
@pytest.mark.parametrize("which", ["deck6", "deck6s"])
def test_sparse_cg_compute_phi_steps(which, request):
    """Whole computePhi + updateEf steps from identical state (den, d, F1):
    the reference's Lapack method against SPARSE_CG in both storages."""
    kd, path = request.getfixturevalue(which)
    dk = mp.Deck.load(path)
    s = advanced(path, kd)
    ctxs = (gpu_context(dk, sphere_potential=-10.0), sparse_context(dk))
    for _ in range(3):
        s.inject()
        s.move(1)
        den = s.get("den")
        d0, F10 = s.get("d"), s.get("F1")
        s.compute_phi(mp.LAPACK)
        s.update_ef()
        for ctx in ctxs:
            ctx.fe_set("d", d0)
            ctx.fe_set("F1", F10)
            st = ctx.compute_phi(mp.SPARSE_CG, mp.FP64, ion_den=den)
            ctx.update_ef()
            d, uh, ef = ctx.field()
            assert st.newton_iterations == 1
            assert rel_err(d, s.get("d")) < 1e-9
            assert rel_err(uh, s.get("uh")) < 1e-9
            assert rel_err(ef, s.get("ef")) < 1e-7
            assert rel_err(ctx.fe_get("F1"), s.get("F1")) < 1e-13  # exp(): CUDA's vs libm's last bit


@needs_ref
def test_sparse_newton_vs_dense_newton(deck8):
    kd, path = deck8
    dk = mp.Deck.load(path)
    s = advanced(path, kd, steps=10)
    den, d0, F10 = s.get("den"), s.get("d"), s.get("F1")
    dense = gpu_context(dk, sphere_potential=None)
    dense.fe_set("d", d0)
    dense.fe_set("F1", F10)
    st_d = dense.compute_phi(mp.NONLINEAR, mp.MIXED, ion_den=den)
    _, uh_d, _ = dense.field()
    sp = mp.Context(dk.mesh)
    sp.set_fe_storage(mp.FE_SPARSE)
    sp.fe_setup(**dk.fe_desc_arrays(None))
    sp.fe_set("d", d0)
    sp.fe_set("F1", F10)
    st_s = sp.compute_phi(mp.SPARSE_NEWTON, mp.FP64, ion_den=den)
    _, uh_s, _ = sp.field()
    assert st_s.newton_iterations == st_d.newton_iterations
    assert np.abs(uh_s - uh_d).max() < 1e-8
    assert np.array_equal(sp.fe_get("F1"), dense.fe_get("F1"))
    # the reference's own NonLinear loop stops its Gauss-Seidel inner solves at
    # ||r||/neq < 1e-4, which leaves its potential 2e-3 relative (about 10 mV)
    # from the exact-inner-solve loops on this deck: a sanity bound only
    s.compute_phi(mp.NONLINEAR)
    assert rel_err(uh_s, s.get("uh")) < 1e-2


def test_sparse_storage_rules(deck4):
    kd, path = deck4
    dk = mp.Deck.load(path)
    ctx = sparse_context(dk, sphere_potential=None)
    for method in (mp.NONLINEAR, mp.GAUSS_SEIDEL, mp.LAPACK):
        with pytest.raises(mp.MpError) as e:
            ctx.compute_phi(method, mp.FP64, ion_den=np.zeros(dk.mesh.n_nodes))
        assert e.value.status == 7
    with pytest.raises(mp.MpError) as e:
        ctx.fe_get("K")
    assert e.value.status == 7
    with pytest.raises(mp.MpError) as e:
        ctx.set_fe_storage(mp.FE_DENSE)
    assert e.value.status == 7
    with pytest.raises(mp.MpError) as e:
        ctx.set_sparse_solver(0.0, 10)
    assert e.value.status == 1
    st = ctx.compute_phi(mp.SPARSE_CG, mp.FP64, ion_den=np.zeros(dk.mesh.n_nodes))
    assert st.newton_iterations == 1
    # an iteration limit below what the solve needs is reported, and the
    # context stays usable
    ctx.set_sparse_solver(1e-12, 2)
    ctx.fe_set("d", np.zeros(ctx.neq))
    with pytest.raises(mp.MpError) as e:
        ctx.compute_phi(mp.SPARSE_CG, mp.FP64, ion_den=np.full(dk.mesh.n_nodes, 1e12))
    assert e.value.status == 5
    ctx.set_sparse_solver()
    ctx.fe_set("d", np.zeros(ctx.neq))
    ctx.compute_phi(mp.SPARSE_CG, mp.FP64, ion_den=np.full(dk.mesh.n_nodes, 1e12))


@pytest.fixture(scope="module")
def big_sparse():
    kd = kuhn.build(48, sphere=(50.0, 50.0, 50.0, 20.0))
    d = tempfile.mkdtemp()
    kuhn.write(kd, d, dt=5e-8, method="lapack")
    dk = mp.Deck.load(d)
    ctx = sparse_context(dk)
    return dk, ctx


def test_sparse_at_scale(big_sparse):
    dk, ctx = big_sparse
    n = ctx.neq
    assert n > 100_000
    rng = np.random.default_rng(5)
    ion = np.abs(rng.normal(1e12, 2e11, size=dk.mesh.n_nodes))
    st = ctx.compute_phi(mp.SPARSE_NEWTON, mp.FP64, ion_den=ion)
    assert 1 <= st.newton_iterations <= 10 and st.l2 < 1e-2
    _, uh, _ = ctx.field()
    assert np.all(np.isfinite(uh))
    # linear solves with the J of the current d
    ctx.build_j(mp.SPARSE_CG)
    b1, b2 = rng.normal(size=n), rng.normal(size=n)
    ys = []
    for b in (b1, b2, b1 + b2):
        st = ctx.solve_linear(mp.SPARSE_CG, mp.FP64, b=b)
        assert st.linear_residual * n <= 1.01e-12 * np.linalg.norm(b)
        ys.append(ctx.fe_get("y"))
    y1, y2, y3 = ys
    assert np.abs(y3 - (y1 + y2)).max() <= 1e-9 * np.abs(y3).max()
    assert abs(b2 @ y1 - b1 @ y2) <= 1e-9 * abs(b1 @ y2)
    # J = K - diag(FP): K y - b is FP * y for one diagonal FP
    rp, col, val = ctx.fe_sparse_matrix()
    rows = np.repeat(np.arange(n), np.diff(rp))

    def Ky(y):
        return np.bincount(rows, weights=val * y[col], minlength=n)

    # the diagonal read off the first solve, FP = (K y1 - b1) / y1, must close
    # the second: K y2 - FP y2 - b2 ~ 0 (rows where y1 is not small)
    fp = (Ky(y1) - b1) / y1
    ok = np.abs(y1) > 1e-3 * np.abs(y1).max()
    assert ok.sum() > n // 2
    assert np.all(np.sign(fp[ok]) == np.sign(fp[ok][0]))
    r2 = (Ky(y2) - fp * y2 - b2)[ok]
    assert np.linalg.norm(r2) <= 1e-8 * np.linalg.norm(b2)
