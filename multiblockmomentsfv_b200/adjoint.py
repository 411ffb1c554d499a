"""Sensitivities of the Heun path: the discrete adjoint (mbm_adjoint_run) and a
thin torch.autograd.Function over it.

The functional is, by default, J = sum over interior cells of qx^2 + qy^2 of the
state after N Heun steps (the squared, unweighted l2 norm of the final heat flux);
`functional` selects the sum of theta or of the deviatoric temperature tensor's
squares (T11 - theta)^2 + 2 T12^2 + (T22 - theta)^2 instead.  The
parameters are the initial temperature field theta0 (one value per interior cell;
density and velocity fixed, T_ij = theta0 delta_ij, q = 0 as in SetInitial,
src/Scenario.c:140-152) and the Knudsen number.  dt is frozen from the forward run:
the gradient is that of the map the adjoint sees, which mbm_replay evaluates for
finite-difference checks.
"""
from __future__ import annotations

import ctypes as C
from typing import List, Optional, Sequence

import numpy as np

from . import _abi
from . import blockfile as bf
from . import scenario as sc
from . import solver as sv

NG, NV = bf.NG, bf.NV


def _dptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _bind(L):
    dp = C.POINTER(C.c_double)
    L.mbm_adjoint_run.argtypes = [C.c_void_p, dp, C.c_int, C.c_int, C.c_double, dp, dp, dp, dp, dp]
    L.mbm_replay.argtypes = [C.c_void_p, dp, C.c_int, dp]
    L.mbm_set_physics.argtypes = [C.c_void_p, C.c_double, C.c_double]
    L.mbm_set_functional.argtypes = [C.c_void_p, C.c_int]
    return L


FUNCTIONALS = {"heat_flux": 0, "temperature": 1, "deviatoric": 2}


def state_from_theta(deck: bf.Deck, base: Sequence[np.ndarray], theta0: Sequence[np.ndarray]) -> List[np.ndarray]:
    """Padded layers whose interior has the density and velocity of `base` (padded
    moment layers, e.g. scenario.initial_block) and temperature theta0[b] (ny, nx),
    T_ij = theta delta_ij, q = 0; ghosts zero (set by the ghost fill)."""
    out = []
    for b, B0, th in zip(deck.blocks, base, theta0):
        U = np.zeros((b.nyp, b.nxp, NV))
        inner = (slice(NG, b.nyp - NG), slice(NG, b.nxp - NG))
        r = B0[inner][..., 0]
        U[inner] = sc.moments(r, B0[inner][..., 1] / r, B0[inner][..., 2] / r, np.asarray(th, dtype=np.float64))
        out.append(U)
    return out


def smooth_base(deck: bf.Deck, seed: int, amp: float = 0.1) -> List[np.ndarray]:
    """A smooth, nowhere-flat base state (density and velocity from a few random
    Fourier modes): finite differences of J are only meaningful where the limiters
    are differentiable, and a flat region sits on every limiter's kink."""
    rng = np.random.default_rng(seed)
    k = rng.uniform(1, 4, size=(3, 4, 2))
    ph = rng.uniform(0, 2 * np.pi, size=(3, 4))
    out = []
    for b in deck.blocks:
        x, y = b.centres()
        f = [sum(np.sin(k[q, m, 0] * x + k[q, m, 1] * y + ph[q, m]) for m in range(4)) / 4 for q in range(3)]
        rho = 1.0 + amp * f[0]
        out.append(sc.moments(rho, 0.2 * f[1], 0.2 * f[2], np.ones_like(rho)))
    return out


def dU_dtheta(U_inner: np.ndarray) -> np.ndarray:
    """d(moments)/d(theta) at fixed rho, v, with T_ij = theta delta_ij, q = 0."""
    r = U_inner[..., 0]
    u = U_inner[..., 1] / r
    v = U_inner[..., 2] / r
    d = np.zeros(U_inner.shape)
    d[..., 3] = 1.5 * r
    d[..., 4] = r
    d[..., 6] = r
    d[..., 7] = 2.5 * r * u
    d[..., 8] = 2.5 * r * v
    return d


class Sensitivity:
    """A single-case device context set up for adjoint runs; `base` gives the
    density and velocity of the initial states (padded moment layers)."""

    def __init__(self, deck: bf.Deck, base: Sequence[np.ndarray], device: int = 0, stream=None,
                 scenario: Optional[sc.Scenario] = None, mode: str = "exact", functional: str = "heat_flux"):
        self.deck = deck
        self.base = list(base)
        self.s = sv.Solver(deck, scenario, device=device, show_every=0, stream=stream, adjoint=True, mode=mode)
        self.L = _bind(self.s.L)
        _abi.check(self.L.mbm_set_functional(self.s.ctx, FUNCTIONALS[functional]), self.s.ctx)

    def close(self):
        self.s.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def load(self, layers: Sequence[np.ndarray], Kn: Optional[float] = None) -> None:
        if Kn is not None:
            _abi.check(self.L.mbm_set_physics(self.s.ctx, Kn, self.deck.F), self.s.ctx)
        for b, U in enumerate(layers):
            self.s.upload(sv.L_DATA, b, U)
        self.s.set_boundary(sv.L_DATA, 0.0)

    def run(self, nsteps: int, every: int = 20):
        """Forward Steps run and reverse sweep.  Returns (J, dJ/du0 per block (padded
        layers, ghosts zero), dJ/dKn, dts, (forward ms, adjoint ms))."""
        t = C.c_double(0.0)
        J = C.c_double(0.0)
        gK = C.c_double(0.0)
        grad = np.zeros(sum(b.cells for b in self.deck.blocks) * NV)
        dts = np.zeros(nsteps)
        ms = np.zeros(2)
        _abi.check(self.L.mbm_adjoint_run(self.s.ctx, C.byref(t), nsteps, every, self.deck.CFL, C.byref(J),
                                          _dptr(grad), C.byref(gK), _dptr(dts), _dptr(ms)), self.s.ctx)
        out, o = [], 0
        for b in self.deck.blocks:
            out.append(grad[o:o + b.cells * NV].reshape(b.nyp, b.nxp, NV))
            o += b.cells * NV
        return J.value, out, gK.value, dts, (float(ms[0]), float(ms[1]))

    def replay(self, dts: np.ndarray) -> float:
        """J after the frozen-dt steps from the loaded state."""
        J = C.c_double(0.0)
        d = np.ascontiguousarray(dts, dtype=np.float64)
        _abi.check(self.L.mbm_replay(self.s.ctx, _dptr(d), len(d), C.byref(J)), self.s.ctx)
        return J.value


def theta_gradient(deck: bf.Deck, layers0: Sequence[np.ndarray], grad_u0: Sequence[np.ndarray]):
    """dJ/dtheta0 per block (ny, nx) from dJ/du0 by the chain rule through SetInitial."""
    out = []
    for b, U, g in zip(deck.blocks, layers0, grad_u0):
        inner = (slice(NG, b.nyp - NG), slice(NG, b.nxp - NG))
        out.append(np.sum(g[inner] * dU_dtheta(U[inner]), axis=-1))
    return out


def make_autograd(sens: Sensitivity, nsteps: int, every: int = 20):
    """torch.autograd.Function: (theta0 (nblocks, ny, nx) tensor, Kn scalar tensor) -> J.
    Backward returns dJ/dtheta0 and dJ/dKn from one adjoint run (dt frozen)."""
    import torch

    class HeatFluxNorm(torch.autograd.Function):
        @staticmethod
        def forward(ctx, theta0, Kn):
            th = theta0.detach().cpu().numpy()
            layers = state_from_theta(sens.deck, sens.base, list(th))
            sens.load(layers, float(Kn))
            J, g, gK, dts, _ = sens.run(nsteps, every)
            gth = np.stack(theta_gradient(sens.deck, layers, g))
            ctx.save_for_backward(torch.from_numpy(gth).to(theta0.dtype), torch.tensor(gK, dtype=theta0.dtype))
            ctx.dts = dts
            return torch.tensor(J, dtype=theta0.dtype)

        @staticmethod
        def backward(ctx, gout):
            gth, gK = ctx.saved_tensors
            return gout * gth, gout * gK

    return HeatFluxNorm.apply
