"""Block-file reader: the ``key = value`` header and the positional block table.

Mirrors the reference's ``ParseHeader`` / ``SetBlocks`` (src/Mesh.c:60-196) and the
CLI overrides of ``main`` (src/Main.c:70-106), so a deck that drives the reference
solver drives this one with the same parameters, grids and output times.
"""
from __future__ import annotations

import re
from dataclasses import dataclass, field, replace
from typing import List, Optional, Sequence

import numpy as np

NG = 3            # ghost layers per edge (src/defs.h:14)
NV = 9            # moments per cell (src/defs.h:11)
NB_MAX = 32       # maximum block number (src/defs.h:13)
NOUT = 50         # maximum number of output times (src/defs.h:15)

LIMITERS = ("none", "average", "minmod", "superbee", "harmonic")   # src/Limiter.h:9-15
LIM_NONE, LIM_AVERAGE, LIM_MINMOD, LIM_SUPERBEE, LIM_HARMONIC = range(5)

BC_OPEN, BC_WALL, BC_DIRICHLET = 0, -1, -2      # codes > 0 synchronise with that block


def limiter_code(name: str) -> int:
    """Limiter name -> code; unknown names fall back to harmonic (src/Limiter.c:66-75)."""
    return LIMITERS.index(name) if name in LIMITERS else LIM_HARMONIC


def limiter_name(code: int) -> str:
    """Limiter code -> name (src/Limiter.c:77-86)."""
    return LIMITERS[code] if 0 <= code < 4 else "harmonic"


@dataclass
class Block:
    """One Cartesian block; the fields of the reference's DB_Block it needs
    (src/defs.h:59-68), derived from the block-table extents as SetBlocks does
    (src/Mesh.c:341-373)."""
    block_id: int
    xmin: float
    xmax: float
    ymin: float
    ymax: float
    nx: int            # interior cells after refinement
    ny: int
    bc: Sequence[int]  # left, right, bottom, top codes
    refine: int = 1

    @property
    def dx(self) -> float:
        return (self.xmax - self.xmin) / self.nx

    @property
    def dy(self) -> float:
        return (self.ymax - self.ymin) / self.ny

    @property
    def x0(self) -> float:     # centre of padded cell (0,0): B.x = xmin - (nst/2-0.5)*dx
        return self.xmin - (NG - 0.5) * self.dx

    @property
    def y0(self) -> float:
        return self.ymin - (NG - 0.5) * self.dy

    @property
    def nxp(self) -> int:      # cells per row, ghosts included
        return self.nx + 2 * NG

    @property
    def nyp(self) -> int:
        return self.ny + 2 * NG

    @property
    def cells(self) -> int:
        return self.nxp * self.nyp

    def centres(self):
        """Cell centres (x[J, I], y[J, I]) of the padded grid, GetPoint (src/tools.c:97-104)."""
        I = np.arange(self.nxp, dtype=np.float64)
        J = np.arange(self.nyp, dtype=np.float64)
        x = self.x0 + I * self.dx
        y = self.y0 + J * self.dy
        return np.broadcast_to(x[None, :], (self.nyp, self.nxp)), np.broadcast_to(y[:, None], (self.nyp, self.nxp))


@dataclass
class Deck:
    """Parameters, blocks and output times of a block file."""
    Kn: float = 0.001
    R13: float = 0.0
    F: float = 0.0
    CFL: float = 0.95
    limiter: int = LIM_HARMONIC
    refine: int = 1
    dt_out: float = 0.0
    t_list: List[float] = field(default_factory=list)
    t_out: List[float] = field(default_factory=list)
    blocks: List[Block] = field(default_factory=list)

    @property
    def full_grid_size(self) -> int:
        """Interior cells over all blocks, FullGridSize (src/tools.c:87-95)."""
        return sum(b.nx * b.ny for b in self.blocks)

    def with_cli(self, Kn=None, R13=None, CFL=None, limiter=None) -> "Deck":
        """Command-line overrides.  Numeric flags pass through ``float`` as in the
        reference's get_float_argument (src/tools.c:38-46, src/Main.c:97-106)."""
        d = replace(self)
        if CFL is not None:
            d.CFL = float(np.float32(CFL))
        if Kn is not None:
            d.Kn = float(np.float32(Kn))
        if R13 is not None:
            d.R13 = float(np.float32(R13))
        if limiter is not None:
            d.limiter = limiter_code(limiter)
        return d


def output_times(dt_out: float, t_list: Sequence[float]) -> List[float]:
    """Post-initial output times from dt_out and t_list (src/Mesh.c:89-108)."""
    if dt_out > 0.0:
        tfin = t_list[0] if t_list else 0.0
        n = int((tfin + 1e-10) / dt_out)
        n = min(n, NOUT - 1)
        out = [(i + 1) * dt_out for i in range(n)]
        if n * dt_out < tfin - 1e-10:
            out.append(tfin)
        return out
    return list(t_list)


_NUM = re.compile(r"\s*[-+]?(\d+\.?\d*|\.\d+)([eE][-+]?\d+)?")


def _atof(s: str) -> float:
    m = _NUM.match(s)
    return float(m.group(0)) if m else 0.0


def _atoi(s: str) -> int:
    m = re.match(r"\s*[-+]?\d+", s)
    return int(m.group(0)) if m else 0


_BLOCK = re.compile(
    r"\s*(-?\d+)/([^,/]+),([^,/]+)/([^,/]+),([^,/]+)/(-?\d+),(-?\d+)/(-?\d+),(-?\d+),(-?\d+),(-?\d+)/")


def parse_text(text: str, refine: Optional[int] = None) -> Deck:
    """Parse block-file text.  ``refine`` mirrors the -refine flag, which takes
    precedence over the file's ``refine`` key (src/Main.c:87-91)."""
    d = Deck()
    lines = text.splitlines()
    k = 0
    t_list: List[float] = []
    dt_out = 0.0
    file_refine = 1
    while k < len(lines):
        p = lines[k].lstrip(" \t")
        k += 1
        if not p or p.startswith("#") or p.startswith("//"):
            continue
        if p[:10].lower() == "block data":
            break
        m = re.match(r"([^= \t]+)\s*=\s*(.*)$", p)
        if not m or m.group(2) == "":
            continue
        key, val = m.group(1), m.group(2)
        if "#" in val:
            val = val[:val.index("#")]
        kl = key.lower()
        if kl == "kn":
            d.Kn = _atof(val)
        elif kl == "r13":
            d.R13 = _atof(val)
        elif kl == "f":
            d.F = _atof(val)
        elif kl == "cfl":
            d.CFL = _atof(val)
        elif kl == "dt_out":
            dt_out = _atof(val)
        elif kl == "t_list":
            t_list = []
            rest = val
            while len(t_list) < NOUT:
                m2 = _NUM.match(rest)
                if not m2:
                    break
                v = float(m2.group(0))
                if v == 0.0:
                    break
                t_list.append(v)
                rest = rest[m2.end():]
        elif kl == "refine":
            file_refine = _atoi(val)
        elif kl == "limiter":
            toks = val.split()
            d.limiter = limiter_code(toks[0] if toks else "")
    d.refine = refine if refine is not None else file_refine
    if d.refine < 1:
        d.refine = 1
    d.dt_out = dt_out
    d.t_list = t_list
    d.t_out = output_times(dt_out, t_list)
    # the line after the marker is the table's column legend (src/Mesh.c:151)
    k += 1
    blocks = {}
    for line in lines[k:]:
        m = _BLOCK.match(line)
        if not m:
            continue
        bid = int(m.group(1))
        if bid < 1 or bid > NB_MAX:
            raise ValueError(f"block number {bid} out of range [1,{NB_MAX}]")
        xmin, xmax, ymin, ymax = (float(m.group(i)) for i in range(2, 6))
        nx, ny = int(m.group(6)) * d.refine, int(m.group(7)) * d.refine
        bc = tuple(int(m.group(i)) for i in range(8, 12))
        blocks[bid] = Block(bid, xmin, xmax, ymin, ymax, nx, ny, bc, d.refine)
    d.blocks = [blocks[i] for i in sorted(blocks)]
    if [b.block_id for b in d.blocks] != list(range(1, len(d.blocks) + 1)):
        raise ValueError("block numbers must run 1..nblocks")
    return d


def parse_file(path: str, refine: Optional[int] = None) -> Deck:
    with open(path) as f:
        return parse_text(f.read(), refine)


def format_deck(d: Deck, title: str = "generated deck") -> str:
    """Write a deck in the block-file format (inverse of parse_text for the
    parameters this package uses)."""
    out = [f"# {title}",
           f"Kn      = {d.Kn!r}",
           f"R13     = {d.R13!r}",
           f"F       = {d.F!r}",
           f"CFL     = {d.CFL!r}",
           f"limiter = {limiter_name(d.limiter)}",
           f"dt_out  = {d.dt_out!r}",
           "t_list  = " + " ".join(repr(t) for t in d.t_list),
           f"refine  = {d.refine}",
           "",
           "Block data (Maximal NB blocks!):",
           "number/xmin,xmax/ymin,ymax/nstx,nsty/leftbound,rightbound,bottombound,topbound/"]
    for b in d.blocks:
        nx, ny = b.nx // b.refine, b.ny // b.refine
        out.append(f"{b.block_id}/{b.xmin!r},{b.xmax!r}/{b.ymin!r},{b.ymax!r}/{nx},{ny}/"
                   f"{b.bc[0]},{b.bc[1]},{b.bc[2]},{b.bc[3]}/")
    return "\n".join(out) + "\n"


def quadrant_deck(n: int, Kn: float = 0.01, limiter: int = LIM_HARMONIC, R13: float = 1.0,
                  nblocks_side: int = 2) -> "Deck":
    """The scaled square4 layout: blocks of n x n cells tiling [-1,1]^2, all outer
    edges open (extrapolation), inner edges synchronised."""
    k = nblocks_side
    h = 2.0 / k
    blocks = []
    for j in range(k):
        for i in range(k):
            bid = j * k + i + 1
            left = bid - 1 if i > 0 else 0
            right = bid + 1 if i < k - 1 else 0
            bottom = bid - k if j > 0 else 0
            top = bid + k if j < k - 1 else 0
            blocks.append(Block(bid, -1.0 + i * h, -1.0 + (i + 1) * h, -1.0 + j * h,
                                -1.0 + (j + 1) * h, n, n, (left, right, bottom, top)))
    d = Deck(Kn=Kn, R13=R13, limiter=limiter, CFL=0.95)
    d.blocks = blocks
    return d
