"""Gradients of the Hamiltonian-constraint loss of a BSSN evolution
(amss_adjoint_* and amss_lousto_vjp of include/amss_b200.h).

The forward is the level-0 RK4 step of the engine (bssn_class::Step,
bssn_class.C:2981-3700: enforce_ga, the split-form right-hand side, Sommerfeld
outer faces, lowerboundset) on one block in FP64; the loss is
L = sum over cells at least 3 cells from every face of H^2 dx dy dz, H the
Hamiltonian constraint of the final state.  The reverse sweep runs on the GPU
with hand-written VJP kernels and a checkpoint every `ck` steps.

Two torch.autograd.Functions compose into the gradient with respect to the
puncture masses / positions and the initial fields:

    state = BrillLindquist.apply(masses, positions, X, Y, Z) + perturbation
    loss = EvolveHamiltonianLoss.apply(state, adjoint, dt, nsteps, ck)
    loss.backward()
"""
import ctypes

import numpy as np
import torch

from ._lib import _DP, AmssError, check, last_error, lib
from . import dropin

NFIELDS = 24


def _p(a):
    return a.ctypes.data_as(_DP)


class Adjoint:
    """One cell-centred block of ex points on bbox (a level-0 patch of its own,
    no symmetry, GAUGE 0) with device storage for the forward, its checkpoints
    and the reverse sweep."""

    def __init__(self, ex, bbox, eps=0.1, chitiny=1e-5):
        self.ex = tuple(int(e) for e in ex)
        self._h = lib().amss_adjoint_create((ctypes.c_int * 3)(*self.ex), (ctypes.c_double * 6)(*bbox), eps,
                                            chitiny)
        if not self._h:
            raise AmssError("amss_adjoint_create failed: " + last_error())
        self.bbox = tuple(bbox)
        self.shape = (NFIELDS, self.ex[2], self.ex[1], self.ex[0])
        self._forward_args = None

    def close(self):
        if self._h:
            lib().amss_adjoint_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _arr(self, a):
        a = np.ascontiguousarray(a, dtype=np.float64)
        if a.shape != self.shape:
            raise AmssError(f"state must have shape {self.shape}, got {a.shape}")
        return a

    def set_state(self, state):
        check(lib().amss_adjoint_set_state(self._h, _p(self._arr(state))), "amss_adjoint_set_state")

    def get_state(self):
        out = np.empty(self.shape)
        check(lib().amss_adjoint_get_state(self._h, _p(out)), "amss_adjoint_get_state")
        return out

    def forward(self, dt, nsteps, ck):
        """nsteps RK4 steps of dt from the state set; returns the loss of the
        final state (the device keeps a checkpoint every ck steps)."""
        loss = ctypes.c_double(0.0)
        check(lib().amss_adjoint_forward(self._h, dt, nsteps, ck, ctypes.byref(loss)), "amss_adjoint_forward")
        return loss.value

    def backward(self):
        """dL/d(the state the last forward started from), shape (24, ez, ey, ex)."""
        g = np.empty(self.shape)
        check(lib().amss_adjoint_backward(self._h, _p(g)), "amss_adjoint_backward")
        return g

    @property
    def stream(self):
        return lib().amss_adjoint_stream(self._h)

    @property
    def launches(self):
        return lib().amss_adjoint_launch_count(self._h)


class EvolveHamiltonianLoss(torch.autograd.Function):
    """loss = L(evolve(state)) with L the interior sum of H^2 dV; backward
    through the GPU reverse sweep.  state: float64 tensor (24, ez, ey, ex)."""

    @staticmethod
    def forward(ctx, state, adjoint, dt, nsteps, ck):
        adjoint.set_state(state.detach().to("cpu", torch.float64).numpy())
        loss = adjoint.forward(dt, nsteps, ck)
        ctx.adjoint = adjoint
        ctx.device = state.device
        return torch.tensor(loss, dtype=torch.float64, device=state.device)

    @staticmethod
    def backward(ctx, gl):
        g = torch.from_numpy(ctx.adjoint.backward()).to(ctx.device)
        return gl * g, None, None, None, None


class BrillLindquist(torch.autograd.Function):
    """The 24-field Brill-Lindquist state (get_lousto_nbhs with zero momenta
    and spins) of punctures masses[N], positions[N, 3] on the cell centres
    X, Y, Z; differentiable in the masses and positions."""

    @staticmethod
    def forward(ctx, masses, positions, X, Y, Z):
        m = masses.detach().cpu().numpy().astype(np.float64)
        pos = positions.detach().cpu().numpy().astype(np.float64)
        st = dropin.get_lousto_nbhs(X, Y, Z, m, pos)
        ctx.save = (np.asarray(X, dtype=np.float64), np.asarray(Y, dtype=np.float64),
                    np.asarray(Z, dtype=np.float64), m, pos)
        ctx.device = masses.device
        return torch.from_numpy(st).to(masses.device)

    @staticmethod
    def backward(ctx, gs):
        X, Y, Z, m, pos = ctx.save
        dm, dp = dropin.lousto_vjp(X, Y, Z, m, pos, gs.detach().cpu().numpy())
        return (torch.from_numpy(dm).to(ctx.device), torch.from_numpy(dp).to(ctx.device), None, None, None)


def hamiltonian_loss(state, adjoint, dt, nsteps, ck):
    """L(evolve(state)) as a differentiable torch scalar."""
    return EvolveHamiltonianLoss.apply(state, adjoint, dt, nsteps, ck)
