"""Derivatives of K push + scatter steps (the C ABI's mp_adjoint_*): node ion
density and wall energy flux as functions of the node potential phi and the
inlet drift velocity, with their vector-Jacobian (reverse) and
Jacobian-vector (tangent) products, plus a torch.autograd.Function over them.

The model (phi held for the K steps; the walk piecewise fixed) is the one
documented in include/minipic_cuda.h beside mp_adjoint_setup.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

import minipic_b200 as mp

WALK, PINNED = 0, 1


def _ptr(a):
    """Host numpy array or CUDA torch tensor -> void*; the library copies with
    cudaMemcpyDefault, so either memory works."""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        assert a.flags.c_contiguous
        return a.ctypes.data_as(C.c_void_p)
    assert a.is_contiguous()
    return C.c_void_p(a.data_ptr())


class Adjoint:
    """Adjoint state on a Context: slots, checkpoints and the last forward's tape."""

    def __init__(self, ctx: "mp.Context", steps: int, checkpoint_every: int, q_over_m: float, mass: float,
                 dt: float, spwt: float, inlet_dir, wall_nodes, nx=None, record_path: bool = False):
        self.ctx = ctx
        self.steps, self.checkpoint_every = steps, checkpoint_every
        d = np.ascontiguousarray(inlet_dir, dtype=np.float64)
        w = np.ascontiguousarray(wall_nodes, dtype=np.uint8)
        nxa = None if nx is None else np.ascontiguousarray(nx, dtype=np.float64)
        ctx._c(mp.lib().mp_adjoint_setup(ctx.h, steps, checkpoint_every, q_over_m, mass, dt, spwt, _ptr(d), _ptr(w),
                                         _ptr(nxa), 1 if record_path else 0))
        self.n_nodes = int(w.size)
        self.tape_id = 0  # forwards run so far; the tape is the last one's

    def add_particles(self, first_step: int, injected: bool, pos, vel, cell):
        pos = np.ascontiguousarray(pos, dtype=np.float64)
        vel = np.ascontiguousarray(vel, dtype=np.float64)
        cell = np.ascontiguousarray(cell, dtype=np.int32)
        self.ctx._c(mp.lib().mp_adjoint_add_particles(self.ctx.h, first_step, 1 if injected else 0, cell.size,
                                                      _ptr(pos), _ptr(vel), _ptr(cell)))

    def forward(self, phi, v_drift: float, mode: int = WALK, den_out=None):
        """Returns (den, stats); den is den_out if given (numpy or CUDA tensor)."""
        if den_out is None:
            den_out = np.zeros(self.n_nodes)
        st = mp.AdjointStats()
        self.ctx._c(mp.lib().mp_adjoint_forward(self.ctx.h, _ptr(phi), float(v_drift), mode, _ptr(den_out),
                                                C.byref(st)))
        self.tape_id += 1
        return den_out, st

    def backward(self, den_bar, flux_bar: float, phi_bar_out=None):
        """Returns (phi_bar, v_drift_bar) at the last forward."""
        if phi_bar_out is None:
            phi_bar_out = np.zeros(self.n_nodes)
        vdb = C.c_double(0)
        self.ctx._c(mp.lib().mp_adjoint_backward(self.ctx.h, _ptr(den_bar), float(flux_bar), _ptr(phi_bar_out),
                                                 C.byref(vdb)))
        return phi_bar_out, vdb.value

    def tangent(self, dphi, dv_drift: float, dden_out=None):
        """Returns (dden, dflux) at the last forward."""
        if dden_out is None:
            dden_out = np.zeros(self.n_nodes)
        df = C.c_double(0)
        self.ctx._c(mp.lib().mp_adjoint_tangent(self.ctx.h, _ptr(dphi), float(dv_drift), _ptr(dden_out),
                                                C.byref(df)))
        return dden_out, df.value


def push_scatter_function():
    """torch.autograd.Function: (phi [n_nodes] f64, v_drift [] f64) -> (den, flux)."""
    import torch

    class PushScatterK(torch.autograd.Function):
        @staticmethod
        def forward(ctx, phi, v_drift, adj: Adjoint, mode: int = WALK):
            dev = phi.device
            if phi.is_cuda:
                torch.cuda.current_stream(dev).synchronize()
            phi_c = phi.detach().contiguous()
            den = torch.zeros(adj.n_nodes, dtype=torch.float64, device=dev)
            _, st = adj.forward(phi_c if phi.is_cuda else phi_c.numpy(), float(v_drift),
                                mode, den if phi.is_cuda else den.numpy())
            ctx.adj, ctx.dev, ctx.mode = adj, dev, mode
            ctx.tape = adj.tape_id
            ctx.phi, ctx.vd = phi_c.clone(), float(v_drift)
            return den, torch.tensor(st.flux, dtype=torch.float64, device=dev)

        @staticmethod
        def backward(ctx, gden, gflux):
            adj = ctx.adj
            if adj.tape_id != ctx.tape:  # another forward ran since: rebuild this call's tape
                phi = ctx.phi
                adj.forward(phi if phi.is_cuda else phi.numpy(), ctx.vd, ctx.mode)
            gden = torch.zeros(adj.n_nodes, dtype=torch.float64, device=ctx.dev) if gden is None else gden
            gflux = 0.0 if gflux is None else float(gflux)
            if gden.is_cuda:
                torch.cuda.current_stream(gden.device).synchronize()
            g = gden.detach().contiguous()
            pb = torch.zeros(adj.n_nodes, dtype=torch.float64, device=ctx.dev)
            _, vdb = adj.backward(g if g.is_cuda else g.numpy(), gflux, pb if pb.is_cuda else pb.numpy())
            return pb, torch.tensor(vdb, dtype=torch.float64, device=ctx.dev), None, None

    return PushScatterK


def wall_nodes_of(mesh) -> np.ndarray:
    """Wall nodes of a deck: the FIXED (Dirichlet wall) nodes."""
    return (mesh.node_type == mp.NODE_FIXED).astype(np.uint8)
