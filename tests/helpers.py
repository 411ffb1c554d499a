"""Shared helpers for the tests: decks, seeded states, bitwise comparison."""
from __future__ import annotations

import os
from typing import List, Sequence

import numpy as np

from multiblockmomentsfv_b200 import blockfile as bf
from multiblockmomentsfv_b200 import scenario as sc

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")
DECKS = os.path.join(GOLDEN, "decks")
NV, NG = bf.NV, bf.NG


def deck(name: str, **kw) -> bf.Deck:
    d = bf.parse_file(os.path.join(DECKS, name + ".txt"))
    for k, v in kw.items():
        setattr(d, k, v)
    return d


def moments_from_prims(P: np.ndarray) -> np.ndarray:
    """Conservative (src/Flux.c:61-74) over a trailing axis of 9 primitives."""
    rho, v1, v2, th, T11, T12, T22, q1, q2 = (P[..., k] for k in range(NV))
    vs = v1 * v1 + v2 * v2
    E = 0.5 * rho * vs + 1.5 * rho * th
    U = np.empty_like(P)
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


def random_layer(rng: np.random.Generator, blk: bf.Block, noise: float = 0.15) -> np.ndarray:
    """A physically admissible but rough state over the padded block: smooth
    background plus cell noise, non-equilibrium stress and heat flux."""
    ny, nx = blk.nyp, blk.nxp
    yy, xx = np.meshgrid(np.linspace(0, 1, ny), np.linspace(0, 1, nx), indexing="ij")
    base = 1.0 + 0.3 * np.sin(3 * xx + 1.7 * yy)
    P = np.empty((ny, nx, NV))
    P[..., 0] = base * (1 + noise * rng.uniform(-1, 1, (ny, nx)))
    P[..., 1] = 0.3 * np.cos(2 * yy) + noise * rng.uniform(-1, 1, (ny, nx))
    P[..., 2] = 0.2 * np.sin(2 * xx) + noise * rng.uniform(-1, 1, (ny, nx))
    th = 1.0 + 0.2 * np.cos(xx - yy) + 0.5 * noise * rng.uniform(-1, 1, (ny, nx))
    P[..., 3] = th
    P[..., 4] = th * (1 + 0.1 * rng.uniform(-1, 1, (ny, nx)))
    P[..., 5] = 0.05 * th * rng.uniform(-1, 1, (ny, nx))
    P[..., 6] = th * (1 + 0.1 * rng.uniform(-1, 1, (ny, nx)))
    P[..., 7] = 0.05 * rng.uniform(-1, 1, (ny, nx))
    P[..., 8] = 0.05 * rng.uniform(-1, 1, (ny, nx))
    return moments_from_prims(P)


def interior(U: np.ndarray) -> np.ndarray:
    return U[NG:-NG, NG:-NG, :]


def bits(a: np.ndarray) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64).view(np.uint64)


def assert_bitwise(a: np.ndarray, b: np.ndarray, what: str = "") -> None:
    a = np.ascontiguousarray(a, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    assert a.shape == b.shape, (what, a.shape, b.shape)
    if not np.array_equal(bits(a), bits(b)):
        d = np.abs(a - b)
        i = np.unravel_index(np.nanargmax(np.where(np.isnan(d), -1, d)), d.shape)
        n = int(np.count_nonzero(bits(a) != bits(b)))
        raise AssertionError(f"{what}: {n} values differ; worst at {i}: {a[i]!r} vs {b[i]!r}")


def apply_ghost_map(entries: np.ndarray, layers: List[np.ndarray], dirichlet=None) -> None:
    """Fill the ghost cells of layers (each (nyp, nxp, 9)) from a resolved map."""
    sx = np.ones(NV)
    sx[[1, 5, 7]] = -1
    sy = np.ones(NV)
    sy[[2, 5, 8]] = -1
    flat = [L.reshape(-1, NV) for L in layers]
    for db, dc, src, sf in entries:
        sb, fl = sf & 0xFFFF, sf >> 16
        v = flat[sb][src].copy() if src >= 0 else dirichlet[-(src + 1)].copy()
        if fl & 1:
            v = v * sx
        if fl & 2:
            v = v * sy
        flat[db][dc] = v


def random_deck(rng: np.random.Generator, max_n: int = 12) -> bf.Deck:
    """A random conforming multi-block layout: 1..4 blocks as strips or a 2x2
    tiling, random edge kinds (open, wall, Dirichlet) on the outer edges."""
    layout = rng.integers(0, 4)
    kinds = [0, -1, -2]
    def outer():
        return int(rng.choice(kinds))
    nx = [int(rng.integers(3, max_n + 1)) for _ in range(2)]
    ny = [int(rng.integers(3, max_n + 1)) for _ in range(2)]
    B = bf.Block
    if layout == 0:
        blocks = [B(1, -1.0, 1.0, -1.0, 1.0, nx[0], ny[0], (outer(), outer(), outer(), outer()))]
    elif layout == 1:       # two blocks side by side
        blocks = [B(1, -1.0, 0.2, -1.0, 1.0, nx[0], ny[0], (outer(), 2, outer(), outer())),
                  B(2, 0.2, 1.0, -1.0, 1.0, nx[1], ny[0], (1, outer(), outer(), outer()))]
    elif layout == 2:       # three stacked strips
        blocks = [B(1, -1.0, 1.0, -1.0, -0.3, nx[0], ny[0], (outer(), outer(), outer(), 2)),
                  B(2, -1.0, 1.0, -0.3, 0.4, nx[0], ny[1], (outer(), outer(), 1, 3)),
                  B(3, -1.0, 1.0, 0.4, 1.0, nx[0], ny[0], (outer(), outer(), 2, outer()))]
    else:                   # 2x2 tiling like square4
        blocks = [B(1, -1.0, 0.3, -1.0, 0.2, nx[0], ny[0], (outer(), 2, outer(), 4)),
                  B(2, 0.3, 1.0, -1.0, 0.2, nx[1], ny[0], (1, outer(), outer(), 3)),
                  B(3, 0.3, 1.0, 0.2, 1.0, nx[1], ny[1], (4, outer(), 2, outer())),
                  B(4, -1.0, 0.3, 0.2, 1.0, nx[0], ny[1], (outer(), 3, 1, outer()))]
    d = bf.Deck(Kn=float(10 ** rng.uniform(-3, -1)), limiter=int(rng.integers(0, 5)), CFL=0.95)
    d.blocks = blocks
    return d


quadrant_deck = bf.quadrant_deck

# The reference's own regression tool (tools/compare_solution.py) and golden result
# files, staged into oracle/_ref by `make -C oracle check` (part of the reference build).
REF_BUILD = os.path.normpath(os.path.join(HERE, "..", "oracle", "_ref"))
REF_COMPARE = os.path.join(REF_BUILD, "compare_solution.py")


def reference_compare(new: str, ref: str, abstol=None, reltol=None):
    """Run the reference's compare_solution.py on two .hdr/.dat results, as its
    `make check` does; returns (passed, its stdout).  Skips the calling test when the
    tool is not staged."""
    import subprocess
    import sys
    import pytest
    if not os.path.exists(REF_COMPARE):
        pytest.skip("reference regression tool not staged (make -C oracle check)")
    args = [sys.executable, REF_COMPARE, new, ref]
    if abstol is not None:
        args += [repr(float(abstol)), repr(float(reltol))]
    r = subprocess.run(args, capture_output=True, text=True, timeout=1800)
    assert r.returncode in (0, 1), r.stdout + r.stderr
    return r.returncode == 0, r.stdout
