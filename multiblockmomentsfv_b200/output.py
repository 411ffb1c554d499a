"""Solution output: the reference's two-file ``.hdr`` (ASCII manifest) + ``.dat``
(raw little-endian payload) format, written and read.

``write`` restates ``Output``/``WriteManifest``/``Convert`` (src/Output.c:60-267):
the same file names, the same ZONE records and the same 10 physical fields
``rho vx vy T p Pxx Pxy Pyy qx qy`` over the interior plus one ghost ring, x
outer / y inner, variable fastest, Float32 by default or Float64.  The field
arithmetic keeps the reference's operand order, so payloads compare bit for bit.
"""
from __future__ import annotations

import os
import re
import struct
import time
from typing import List, Optional, Sequence, Tuple

import numpy as np

from .blockfile import NG, NV, Deck

NVARS_OUT = 10
FORMAT_VERSION = 1


def convert(a: float) -> str:
    """Compact number token for file names, e.g. 0.05 -> "0p05" (src/Output.c:60-71)."""
    i = int(abs(a + 1e-7))
    j = int(abs(10 * (a - i + 1e-7)))
    k = int(abs(100 * (a - i - 0.1 * j + 1e-7)))
    l = int(abs(1000 * (a - i - 0.1 * j - 0.01 * k + 1e-7)))
    if l != 0:
        return f"{i}p{j}{k}{l}"
    if k != 0:
        return f"{i}p{j}{k}"
    return f"{i}p{j}"


def primitive(U: np.ndarray) -> np.ndarray:
    """Primitive variables of moment vectors (src/Flux.c:30-56), trailing axis 9."""
    rho = U[..., 0]
    v1 = U[..., 1] / rho
    v2 = U[..., 2] / rho
    vs = v1 * v1 + v2 * v2
    th = (2 * U[..., 3] / rho - vs) / 3
    E = U[..., 3]
    T11 = U[..., 4] / rho - v1 * v1
    T12 = U[..., 5] / rho - v1 * v2
    T22 = U[..., 6] / rho - v2 * v2
    q1 = U[..., 7] - E * v1 - rho * (T11 * v1 + T12 * v2)
    q2 = U[..., 8] - E * v2 - rho * (T12 * v1 + T22 * v2)
    return np.stack([rho, v1, v2, th, T11, T12, T22, q1, q2], axis=-1)


def physical_fields(U: np.ndarray) -> np.ndarray:
    """The 10 output fields of moment vectors (src/Output.c:220-234)."""
    P = primitive(U)
    out = np.empty(U.shape[:-1] + (NVARS_OUT,))
    out[..., 0] = P[..., 0]
    out[..., 1] = P[..., 1]
    out[..., 2] = P[..., 2]
    out[..., 3] = P[..., 3]
    out[..., 4] = P[..., 0] * P[..., 3]
    out[..., 5] = P[..., 0] * P[..., 4]
    out[..., 6] = P[..., 0] * P[..., 5]
    out[..., 7] = P[..., 0] * P[..., 6]
    out[..., 8] = P[..., 7]
    out[..., 9] = P[..., 8]
    return out


def zone_payload(U: np.ndarray, nx: int, ny: int, single: bool) -> bytes:
    """Payload of one block: interior plus one ghost ring, x outer, y inner,
    variables fastest (src/Output.c:195-247).  U is (ny+6, nx+6, 9)."""
    g = NG - 1
    win = U[g:ny + 2 * NG - g, g:nx + 2 * NG - g, :]          # (ny+2, nx+2, 9)
    vals = physical_fields(win).transpose(1, 0, 2)            # (nx+2, ny+2, 10)
    return np.ascontiguousarray(vals, dtype="<f4" if single else "<f8").tobytes()


class Writer:
    """Appends time levels to a ``..._tAll.{hdr,dat}`` pair like Output(B, bMax, n, t, Add)."""

    def __init__(self, out_dir: str, deck: Deck, type_name: str, single: bool = True,
                 git_commit: str = "unknown"):
        self.out_dir = out_dir
        self.deck = deck
        self.type_name = type_name
        self.single = single
        self.git_commit = git_commit
        solv = ("Grad13" if deck.R13 < 1.0 else "Reg13") + type_name
        self.solver_name = solv
        prefix = (out_dir + "/") if out_dir else ""
        self.base = f"{prefix}{solv}_nst{deck.full_grid_size}_Kn{convert(deck.Kn)}_tAll"
        self.hdr = self.base + ".hdr"
        self.dat = self.base + ".dat"

    def _manifest(self) -> str:
        d = self.deck
        now = time.strftime("%Y-%m-%dT%H:%M:%SZ", time.gmtime())
        t_out = "t_output = 0.0" + "".join(" %.10g" % t for t in d.t_out)
        return (
            "# MultiBlockMomentsFV binary output header\n"
            f"# FORMAT_VERSION = {FORMAT_VERSION}\n"
            f"# CREATED_UTC = {now}\n"
            f"# GIT_COMMIT = {self.git_commit}\n\n"
            "[RUN]\n"
            f"solver = {self.solver_name}\n"
            "Kn = %.10g\n" % d.Kn +
            "R13 = %.10g\n" % d.R13 +
            f"Type = {self.type_name}\n"
            f"FullGridSize = {d.full_grid_size}\n"
            f"refine = {d.refine}\n"
            f"{t_out}\n\n"
            "[BINARY]\n"
            f"BINARY_FILE = {os.path.basename(self.dat)}\n"
            f"NVARS = {NVARS_OUT}\n"
            "ORDER = variable-fastest\n"
            f"PRECISION = {'Float32' if self.single else 'Float64'}\n"
            "ENDIAN = little\n\n"
            "[VARIABLES]\n"
            "rho vx vy T p Pxx Pxy Pyy qx qy\n\n"
            "[ZONES]\n"
            "# block I J NVARS BX BY DX DY LFB_I LFB_J ISTART JSTART NGHOST SOLUTIONTIME STRANDID OFFSET NBYTES\n")

    def write(self, layers: Sequence[np.ndarray], t: float, add: int) -> None:
        """layers[b] = L_DATA of block b, (ny+6, nx+6, 9).  add <= 0 starts fresh
        files (STRANDID 1); add > 0 appends with STRANDID add+1."""
        self._write([zone_payload(U, b.nx, b.ny, self.single) for b, U in zip(self.deck.blocks, layers)], t, add)

    def write_solver(self, solver, t: float, add: int) -> None:
        """The same from a device solver: the payload is formed on the GPU
        (mbm_output_fields) and only the output fields cross to the host."""
        self._write([solver.output_fields(b, self.single).tobytes() for b in range(len(self.deck.blocks))], t, add)

    def _write(self, payloads, t: float, add: int) -> None:
        if self.out_dir:
            os.makedirs(self.out_dir, exist_ok=True)
        fresh = add <= 0
        if fresh:
            add = 0
        mode = "w" if fresh else "a"
        with open(self.hdr, mode) as fh, open(self.dat, mode + "b") as fd:
            if fresh:
                fh.write(self._manifest())
            esize = 4 if self.single else 8
            for nb, (b, payload) in enumerate(zip(self.deck.blocks, payloads)):
                ni = b.ny + 2
                nj = b.nx + 2
                offset = fd.tell()
                fd.write(payload)
                nbytes = ni * nj * NVARS_OUT * esize
                fh.write("ZONE block=%d I=%d J=%d NVARS=%d "
                         "BX=%.16g BY=%.16g DX=%.16g DY=%.16g LFB_I=%d LFB_J=%d "
                         "ISTART=%d JSTART=%d NGHOST=%d "
                         "SOLUTIONTIME=%.16g STRANDID=%d OFFSET=%d NBYTES=%d\n"
                         % (nb + 1, ni, nj, NVARS_OUT, b.x0, b.y0, b.dx, b.dy, 1, 1,
                            NG, NG, 1, t, add + 1, offset, nbytes))


def companion(path: str) -> Tuple[str, str]:
    base = path[:-4] if path.endswith((".hdr", ".dat")) else path
    return base + ".hdr", base + ".dat"


def read(path: str, keep_dtype: bool = False):
    """Read a result pair: returns (zones, precision) where zones is a list of
    dicts with block, I, J, time and values (I*J, 10) as float64 (keep_dtype: in the
    file's precision, float32 for Float32 files)."""
    hdr, dat = companion(path)
    prec = "Float64"
    zones = []
    with open(hdr) as f:
        for line in f:
            m = re.match(r"\s*PRECISION\s*=\s*(\S+)", line)
            if m:
                prec = m.group(1)
            s = line.strip()
            if not s.startswith("ZONE"):
                continue
            g = lambda k: re.search(rf"\b{k}\s*=\s*(\S+)", s).group(1)
            zones.append(dict(block=int(g("block")), I=int(g("I")), J=int(g("J")),
                              nvars=int(g("NVARS")), offset=int(g("OFFSET")),
                              time=float(g("SOLUTIONTIME")), strand=int(g("STRANDID"))))
    dt = np.dtype("<f4") if prec == "Float32" else np.dtype("<f8")
    raw = np.fromfile(dat, dtype=np.uint8)
    for z in zones:
        n = z["nvars"] * z["I"] * z["J"]
        v = raw[z["offset"]:z["offset"] + n * dt.itemsize].view(dt)
        z["values"] = (v.copy() if keep_dtype else v.astype(np.float64)).reshape(-1, z["nvars"])
    return zones, prec


def compare(new: str, ref: str, abstol: Optional[float] = None, reltol: Optional[float] = None):
    """The reference's regression gate (tools/compare_solution.py): zone structure
    must match and every value must satisfy |a-b| <= abstol + reltol*|ref|.
    Returns (ok, max_abs_diff, message)."""
    zn, pn = read(new)
    zr, pr = read(ref)
    single = "Float32" in (pn, pr)
    abstol = abstol if abstol is not None else (1e-6 if single else 1e-10)
    reltol = reltol if reltol is not None else (1e-5 if single else 1e-8)
    kn = [(z["block"], z["I"], z["J"], z["nvars"]) for z in zn]
    kr = [(z["block"], z["I"], z["J"], z["nvars"]) for z in zr]
    if kn != kr:
        return False, float("inf"), f"zone structure differs ({len(kn)} vs {len(kr)} zones)"
    a = np.concatenate([z["values"].ravel() for z in zn]) if zn else np.zeros(0)
    b = np.concatenate([z["values"].ravel() for z in zr]) if zr else np.zeros(0)
    d = np.abs(a - b)
    mx = float(d.max()) if d.size else 0.0
    bad = d > abstol + reltol * np.abs(b)
    if bad.any():
        i = int(np.argmax(bad))
        return False, mx, f"value mismatch at index {i}: {a[i]:.12g} vs {b[i]:.12g}"
    return True, mx, f"{a.size} values match (abstol={abstol:g}, reltol={reltol:g})"
