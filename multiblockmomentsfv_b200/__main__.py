"""Command line of the reference solver (src/Main.c:61-164) on the GPU path.

    python -m multiblockmomentsfv_b200 -bfile cases/squareSmall.txt -out runs/ss [-double]
        [-refine n] [-CFL x] [-Kn x] [-R13 x] [-limiter name] [-sfile file]
        [-scenario riemann2d|ffs|quadrant:SEED|uniform:r,u,v,th] [-device k] [-fast]
        [-restart-faithful]

Flags keep the reference's meaning and its quirks: numeric overrides pass through
``float`` (src/tools.c:38-46), -refine precedes the block file, and -sfile reloads the
first zones of a result pair into L_DATA with the reference's mapping of the stored
fields (src/Mesh.c:198-283: the stored pressure p goes where the temperature belongs and
P_ij where T_ij belongs; -restart-faithful reads the last level with the correct
mapping instead).  -scenario picks the initial/Dirichlet state that the
reference hard-codes in src/Scenario.c (default riemann2d).  -fast runs the stage
kernel in fast arithmetic (MBM_MODE_FAST: within 1e-10 of the reference per field after
one step, 1e-8 at the end time, not bitwise).
"""
from __future__ import annotations

import os
import sys
import time

import numpy as np

from . import blockfile as bf
from . import output as out
from . import scenario as sc
from . import solver as sv


def _arg(argv, key, default=None):
    for i, a in enumerate(argv[1:], 1):
        if a == key:
            return argv[i + 1] if i + 1 < len(argv) else None
    return default


def _scenario(spec: str) -> sc.Scenario:
    if spec.startswith("quadrant:"):
        return sc.Scenario.seeded_quadrant(int(spec.split(":", 1)[1]))
    if spec.startswith("uniform:"):
        v = [float(x) for x in spec.split(":", 1)[1].split(",")]
        return sc.Scenario(sc.KIND_UNIFORM, [tuple(v)] * 4)
    return sc.Scenario.named(spec)


def load_restart(deck: bf.Deck, path: str, faithful: bool = False):
    """LoadData (src/Mesh.c:198-283): the first len(blocks) zones fill the interior
    plus one ghost ring of L_DATA; the remaining cells stay zero.  Like the reference,
    the stored pressure goes where the temperature belongs and P_ij where T_ij belongs,
    and the first zones of a multi-level file are its t = 0 level.

    faithful=True (CLI -restart-faithful) reads the last time level instead and maps
    the fields to the state they came from: theta = T, T_ij = P_ij / rho."""
    zones, _ = out.read(path)
    nb = len(deck.blocks)
    sel = zones[len(zones) - nb:] if faithful else zones[:nb]
    layers = []
    for b, z in zip(deck.blocks, sel):
        U = np.zeros((b.nyp, b.nxp, bf.NV))
        vals = z["values"].reshape(b.nx + 2, b.ny + 2, 10)      # x outer, y inner
        P = np.empty((b.nx + 2, b.ny + 2, bf.NV))
        P[..., 0:3] = vals[..., 0:3]
        if faithful:
            P[..., 3] = vals[..., 3]
            P[..., 4:7] = vals[..., 5:8] / vals[..., 0:1]
        else:
            P[..., 3:7] = vals[..., 4:8]
        P[..., 7:9] = vals[..., 8:10]
        rho, v1, v2, th = P[..., 0], P[..., 1], P[..., 2], P[..., 3]
        vs = v1 * v1 + v2 * v2
        E = 0.5 * rho * vs + 1.5 * rho * th
        C = np.empty_like(P)
        C[..., 0] = rho
        C[..., 1] = rho * v1
        C[..., 2] = rho * v2
        C[..., 3] = E
        C[..., 4] = rho * (P[..., 4] + v1 * v1)
        C[..., 5] = rho * (P[..., 5] + v1 * v2)
        C[..., 6] = rho * (P[..., 6] + v2 * v2)
        C[..., 7] = P[..., 7] + E * v1 + rho * (P[..., 4] * v1 + P[..., 5] * v2)
        C[..., 8] = P[..., 8] + E * v2 + rho * (P[..., 5] * v1 + P[..., 6] * v2)
        U[2:b.ny + 4, 2:b.nx + 4, :] = C.transpose(1, 0, 2)
        layers.append(U)
    return layers


def restart_payloads(deck: bf.Deck, path: str, faithful: bool = False):
    """The zones LoadData reads (src/Mesh.c:198-283) as stored, in the file's precision:
    the first len(blocks) zones (the t = 0 level of a multi-level file), or with faithful
    the last level; for mbm_load_fields, which forms the moments on the device."""
    zones, _ = out.read(path, keep_dtype=True)
    nb = len(deck.blocks)
    sel = zones[len(zones) - nb:] if faithful else zones[:nb]
    for b, z in zip(deck.blocks, sel):
        if z["values"].shape != ((b.nx + 2) * (b.ny + 2), 10):
            raise ValueError("restart file zone %d does not match block %d" % (z["block"], b.block_id))
    return [z["values"] for z in sel]


def main(argv=None) -> int:
    argv = sys.argv if argv is None else argv
    if "-h" in argv[1:] or "--help" in argv[1:]:
        print(__doc__)
        return 0
    out_dir = _arg(argv, "-out", "")
    refine = _arg(argv, "-refine")
    bfile = _arg(argv, "-bfile", "blockfile.txt")
    if not bfile or not os.path.isfile(bfile):
        print("block file not found: %s (-h for the flags)" % bfile, file=sys.stderr)
        return 1
    deck = bf.parse_file(bfile, refine=max(1, int(float(refine))) if refine is not None else None)
    deck = deck.with_cli(Kn=_arg(argv, "-Kn"), R13=_arg(argv, "-R13"), CFL=_arg(argv, "-CFL"),
                         limiter=_arg(argv, "-limiter"))
    scn = _scenario(_arg(argv, "-scenario", "riemann2d"))
    single = "-double" not in argv
    device = int(_arg(argv, "-device", "0"))
    print("\n Running: Kn = %.4g, R13 = %g, CFL = %.2f, limiter = %s, BlockFile = \"%s\"" %
          (deck.Kn, deck.R13, deck.CFL, bf.limiter_name(deck.limiter), _arg(argv, "-bfile", "blockfile.txt")))
    sfile = _arg(argv, "-sfile")
    faithful = "-restart-faithful" in argv
    restart = (restart_payloads(deck, sfile, faithful), faithful) if sfile else None
    mode = "fast" if "-fast" in argv else "exact"
    sv.run(deck, scn, out_dir, single=single, device=device, verbose=True, mode=mode, restart=restart)
    return 0


if __name__ == "__main__":
    sys.exit(main())
