"""Initial and Dirichlet states.

``initial_state`` restates the reference's ``SetInitial`` (src/Scenario.c:72-153):
a moment vector built from {rho, v, theta} with T_ij = theta delta_ij and q = 0,
evaluated with the reference's operand order so the arrays match the C solver
bit for bit.  Scenarios:

* ``riemann2d``  -- rho = 5 inside r < 0.4, else 1, at rest, theta = 1 (the
  state the reference goldens were made with, src/Scenario.c:79-98);
* ``ffs``        -- uniform Mach-2 stream (src/Scenario.c:125-138);
* ``quadrant``   -- four constant states, one per quadrant about the origin,
  drawn from a seed (the seeded workloads of the benchmark);
* ``uniform``    -- one constant state.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import List, Optional, Tuple

import numpy as np

from .blockfile import NG, NV, Block

KIND_RIEMANN2D, KIND_FFS, KIND_QUADRANT, KIND_UNIFORM = 0, 1, 2, 3
_KINDS = {"riemann2d": KIND_RIEMANN2D, "ffs": KIND_FFS, "quadrant": KIND_QUADRANT,
          "uniform": KIND_UNIFORM}
_TYPE_NAMES = {KIND_RIEMANN2D: "Riemann2D", KIND_FFS: "ForwardFacingStep",
               KIND_QUADRANT: "Quadrant", KIND_UNIFORM: "Uniform"}


@dataclass
class Scenario:
    kind: int = KIND_RIEMANN2D
    # {rho, vx, vy, theta} per quadrant k = (x >= 0) + 2*(y >= 0)
    states: List[Tuple[float, float, float, float]] = field(default_factory=lambda: [(1.0, 0.0, 0.0, 1.0)] * 4)

    @property
    def type_name(self) -> str:
        return _TYPE_NAMES[self.kind]

    @classmethod
    def named(cls, name: str) -> "Scenario":
        return cls(_KINDS[name])

    @classmethod
    def seeded_quadrant(cls, seed: int) -> "Scenario":
        """Quadrant states: rho, theta ~ U[0.5, 2], vx, vy ~ U[-0.3, 0.3] from
        ``numpy.random.default_rng(seed)``, drawn quadrant by quadrant."""
        rng = np.random.default_rng(seed)
        states = []
        for _ in range(4):
            rho, th = rng.uniform(0.5, 2.0, size=2)
            vx, vy = rng.uniform(-0.3, 0.3, size=2)
            states.append((float(rho), float(vx), float(vy), float(th)))
        return cls(KIND_QUADRANT, states)

    def env_string(self) -> str:
        """The scenario spec understood by the reference build's scenario file."""
        if self.kind == KIND_RIEMANN2D:
            return "riemann2d"
        if self.kind == KIND_FFS:
            return "ffs"
        n = 4 if self.kind == KIND_QUADRANT else 1
        body = ";".join(",".join(repr(float(v)) for v in s) for s in self.states[:n])
        return ("quadrant:" if self.kind == KIND_QUADRANT else "uniform:") + body


def moments(rho, v1, v2, th):
    """Moment vector of {rho, v, theta} with T_ij = theta delta_ij, q = 0
    (src/Scenario.c:140-152).  Returns an array with a trailing axis of 9."""
    rho, v1, v2, th = np.broadcast_arrays(*(np.asarray(a, dtype=np.float64) for a in (rho, v1, v2, th)))
    T11 = th
    T12 = np.zeros_like(th)
    T22 = th
    q1 = np.zeros_like(th)
    q2 = np.zeros_like(th)
    vs = v1 * v1 + v2 * v2
    E = 0.5 * rho * vs + 1.5 * rho * th
    U = np.empty(rho.shape + (NV,))
    U[..., 0] = rho
    U[..., 1] = rho * v1
    U[..., 2] = rho * v2
    U[..., 3] = E
    U[..., 4] = rho * (T11 + v1 * v1)
    U[..., 5] = rho * (T12 + v1 * v2)
    U[..., 6] = rho * (T22 + v2 * v2)
    U[..., 7] = q1 + E * v1 + rho * (T11 * v1 + T12 * v2)
    U[..., 8] = q2 + E * v2 + rho * (T12 * v1 + T22 * v2)
    return U


def initial_state(s: Scenario, x, y, t: float = 0.0) -> np.ndarray:
    """SetInitial(U, (x,y), t) over arrays of points (src/Scenario.c:72-153)."""
    x = np.asarray(x, dtype=np.float64)
    y = np.asarray(y, dtype=np.float64)
    one = np.ones(np.broadcast(x, y).shape)
    if s.kind == KIND_RIEMANN2D:
        rho = np.where(np.sqrt(x * x + y * y) < 0.4, 5.0, 1.0) * one
        return moments(rho, 0.0 * one, 0.0 * one, one)
    if s.kind == KIND_FFS:
        return moments(one, 2.0 * np.sqrt(5.0 / 3.0) * one, 0.0 * one, one)
    st = np.asarray(s.states, dtype=np.float64)
    if s.kind == KIND_UNIFORM:
        k = np.zeros(one.shape, dtype=np.int64)
    else:
        k = (x >= 0.0).astype(np.int64) + 2 * (y >= 0.0).astype(np.int64)
    return moments(st[k, 0], st[k, 1], st[k, 2], st[k, 3])


def initial_block(s: Scenario, b: Block) -> np.ndarray:
    """Interior of L_DATA set from the scenario, ghosts zero (src/Main.c:113-136).
    Returns (nyp, nxp, 9), x fastest.  Piecewise-constant states are evaluated once
    per state and scattered (the same bits as evaluating every cell)."""
    U = np.zeros((b.nyp, b.nxp, NV))
    x, y = b.centres()
    inner = (slice(NG, b.nyp - NG), slice(NG, b.nxp - NG))
    if s.kind in (KIND_QUADRANT, KIND_UNIFORM):
        st = np.asarray(s.states, dtype=np.float64)
        table = moments(st[:, 0], st[:, 1], st[:, 2], st[:, 3])          # (4, 9)
        if s.kind == KIND_UNIFORM:
            U[inner] = table[0]
        else:
            k = (x[inner] >= 0.0).astype(np.int64) + 2 * (y[inner] >= 0.0).astype(np.int64)
            U[inner] = table[k]
        return U
    U[inner] = initial_state(s, x[inner], y[inner], 0.0)
    return U


def dirichlet_edge(s: Scenario, b: Block, side: int, t: float = 0.0) -> np.ndarray:
    """Dirichlet ghost values of one edge in FillEdge order: tangential index
    outer (full range, corners included), ghost layer n = 1..3 inner
    (src/Boundary.c:105-129).  Returns (nt, 3, 9)."""
    x, y = b.centres()
    nt = b.nyp if side < 2 else b.nxp
    ti = np.arange(nt)
    out = np.empty((nt, NG, NV))
    for n in range(1, NG + 1):
        if side == 0:
            I, J = np.full(nt, NG - n), ti
        elif side == 1:
            I, J = np.full(nt, b.nxp - 1 - NG + n), ti
        elif side == 2:
            I, J = ti, np.full(nt, NG - n)
        else:
            I, J = ti, np.full(nt, b.nyp - 1 - NG + n)
        out[:, n - 1, :] = initial_state(s, x[J, I], y[J, I], t)
    return out
