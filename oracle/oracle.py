"""ctypes front end of the oracle (liboracle.so, the C restatement in mbm_oracle.c)
and of the reference build under oracle/_ref.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
cpu_baseline / reference legs of bench.py, never by the product package.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import sys
from typing import List, Optional, Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
if REPO not in sys.path:
    sys.path.insert(0, REPO)

from multiblockmomentsfv_b200 import blockfile as bf          # noqa: E402
from multiblockmomentsfv_b200 import scenario as sc           # noqa: E402
from multiblockmomentsfv_b200 import output as out            # noqa: E402

LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")
# the reference checkout (only read when the reference build is made here)
REF_ROOT = os.environ.get("MBM_REFERENCE_ROOT", "/root/reference")
REF_SRC = os.path.join(REF_ROOT, "src")

NV, NG = 9, 3
DATA, TMP, NEW = 0, 1, 2


class OrcBlock(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("x0", C.c_double), ("y0", C.c_double),
                ("dx", C.c_double), ("dy", C.c_double), ("bc", C.c_int * 4)]


class OrcParams(C.Structure):
    _fields_ = [("Kn", C.c_double), ("F", C.c_double), ("limiter", C.c_int)]


class OrcScenario(C.Structure):
    _fields_ = [("kind", C.c_int), ("q", (C.c_double * 4) * 4)]


def build(force: bool = False) -> None:
    """Compile liboracle.so (and oracle/_ref when the reference sources exist)."""
    if force or not os.path.exists(LIB_PATH):
        subprocess.run(["make", "-C", HERE, "liboracle.so"], check=True,
                       stdout=subprocess.DEVNULL)
    if os.path.isdir(REF_SRC):
        subprocess.run(["make", "-C", HERE, "ref"], check=True, stdout=subprocess.DEVNULL)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        P = C.POINTER
        dp = P(C.c_double)
        L.orc_create.restype = C.c_void_p
        L.orc_create.argtypes = [P(OrcBlock), C.c_int, P(OrcParams), P(OrcScenario)]
        L.orc_destroy.argtypes = [C.c_void_p]
        L.orc_set_params.argtypes = [C.c_void_p, P(OrcParams)]
        L.orc_set_layer.argtypes = [C.c_void_p, C.c_int, C.c_int, dp]
        L.orc_get_layer.argtypes = [C.c_void_p, C.c_int, C.c_int, dp]
        L.orc_initialise.argtypes = [C.c_void_p]
        L.orc_initial_state.argtypes = [P(OrcScenario), C.c_double, C.c_double, C.c_double, dp]
        L.orc_set_boundary.argtypes = [C.c_void_p, C.c_int, C.c_double]
        L.orc_update.restype = C.c_double
        L.orc_update.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int,
                                 C.c_double, C.c_double, C.c_int]
        L.orc_time_update.restype = C.c_double
        L.orc_time_update.argtypes = [C.c_void_p, C.c_double, C.c_double]
        L.orc_steps.restype = C.c_int
        L.orc_steps.argtypes = [C.c_void_p, P(C.c_double), C.c_double, C.c_double, C.c_double,
                                C.c_int, P(C.c_int), C.c_int, dp, C.c_int, P(C.c_int)]
        L.orc_primitive.argtypes = [dp, dp]
        L.orc_conservative.argtypes = [dp, dp]
        L.orc_flux2d.argtypes = [dp, dp, C.c_double, C.c_double]
        L.orc_relax.restype = C.c_double
        L.orc_relax.argtypes = [P(OrcParams), dp, dp, C.c_double, C.c_int]
        L.orc_limit.restype = C.c_double
        L.orc_limit.argtypes = [C.c_int, C.c_double, C.c_double]
        L.orc_hll.restype = C.c_double
        L.orc_hll.argtypes = [dp, dp, dp, C.c_int, C.c_double]
        _lib = L
    return _lib


def _dptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_double))


def c_blocks(blocks: Sequence[bf.Block]):
    arr = (OrcBlock * len(blocks))()
    for i, b in enumerate(blocks):
        arr[i].nx, arr[i].ny = b.nx, b.ny
        arr[i].x0, arr[i].y0, arr[i].dx, arr[i].dy = b.x0, b.y0, b.dx, b.dy
        for s in range(4):
            arr[i].bc[s] = b.bc[s]
    return arr


def c_scenario(s: sc.Scenario) -> OrcScenario:
    o = OrcScenario()
    o.kind = s.kind
    for k, st in enumerate(s.states[:4]):
        for m in range(4):
            o.q[k][m] = st[m]
    return o


class Oracle:
    """The oracle's solver state for one deck (three layers per block)."""

    def __init__(self, deck: bf.Deck, scenario: sc.Scenario):
        self.deck = deck
        self.scenario = scenario
        self.L = lib()
        self._blocks = c_blocks(deck.blocks)
        self._params = OrcParams(deck.Kn, deck.F, deck.limiter)
        self._scn = c_scenario(scenario)
        self.ctx = self.L.orc_create(self._blocks, len(deck.blocks), C.byref(self._params),
                                     C.byref(self._scn))
        if not self.ctx:
            raise ValueError("orc_create failed")

    def close(self):
        if self.ctx:
            self.L.orc_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        self.close()

    def initialise(self):
        self.L.orc_initialise(self.ctx)

    def set_layer(self, layer: int, b: int, U: np.ndarray):
        U = np.ascontiguousarray(U, dtype=np.float64)
        blk = self.deck.blocks[b]
        assert U.size == blk.cells * NV
        self.L.orc_set_layer(self.ctx, layer, b, _dptr(U))

    def get_layer(self, layer: int, b: int) -> np.ndarray:
        blk = self.deck.blocks[b]
        U = np.empty((blk.nyp, blk.nxp, NV))
        self.L.orc_get_layer(self.ctx, layer, b, _dptr(U))
        return U

    def layers(self, layer: int = DATA) -> List[np.ndarray]:
        return [self.get_layer(layer, b) for b in range(len(self.deck.blocks))]

    def set_boundary(self, layer: int, t: float):
        self.L.orc_set_boundary(self.ctx, layer, t)

    def update(self, b, out_layer, in_layer, data0_layer, dt, t, heun) -> float:
        return self.L.orc_update(self.ctx, b, out_layer, in_layer, data0_layer, dt, t, heun)

    def time_update(self, dt: float, t: float) -> float:
        return self.L.orc_time_update(self.ctx, dt, t)

    def steps(self, t: float, tend: float, CFLmax: float = 1.0, CFLreg: Optional[float] = None,
              max_steps: int = 0, show_every: int = 20):
        """Steps(); returns (t, nsteps, nrej, trace[k] = (step, CFL, t, dt))."""
        CFLreg = self.deck.CFL if CFLreg is None else CFLreg
        tt = C.c_double(t)
        nrej = C.c_int(0)
        cap = 4096
        trace = np.zeros((cap, 4))
        ntr = C.c_int(0)
        n = self.L.orc_steps(self.ctx, C.byref(tt), tend, CFLmax, CFLreg, max_steps,
                             C.byref(nrej), show_every, _dptr(trace), cap, C.byref(ntr))
        return tt.value, n, nrej.value, trace[:ntr.value].copy()


def run_deck(deck: bf.Deck, scenario: sc.Scenario, out_dir: str, single: bool = True,
             max_steps: int = 0):
    """The reference's main(): initial state, output at t=0, then Steps/Output for
    every output time (src/Main.c:113-156), with the oracle as the solver.
    Returns (writer, total steps)."""
    o = Oracle(deck, scenario)
    o.initialise()
    w = out.Writer(out_dir, deck, scenario.type_name, single)
    w.write(o.layers(), 0.0, -1)
    t, nmax = 0.0, 0
    for tn in deck.t_out:
        t, n, _, _ = o.steps(t, tn, 1.0, deck.CFL, max_steps=max_steps)
        nmax += n
        w.write(o.layers(), t, nmax)
    o.close()
    return w, nmax


def ref_binary(name: str = "moments") -> Optional[str]:
    p = os.path.join(REF_DIR, name)
    return p if os.path.exists(p) else None


def run_reference(deck_path: str, out_dir: str, scenario: sc.Scenario, extra=(),
                  binary: str = "moments", threads: Optional[int] = None):
    """Run the reference solver built under oracle/_ref on a block file."""
    exe = ref_binary(binary)
    if exe is None:
        raise FileNotFoundError("reference build missing: make -C oracle ref")
    env = dict(os.environ, MBM_SCENARIO=scenario.env_string())
    if threads:
        env.update(OMP_NUM_THREADS=str(threads), OMP_PROC_BIND="close", OMP_PLACES="cores")
    os.makedirs(out_dir, exist_ok=True)
    return subprocess.run([exe, "-bfile", deck_path, "-out", out_dir, *extra], env=env,
                          capture_output=True, text=True, check=True)


# ------------------------------------------------------------------------------
# the reference itself (oracle/_ref/libmbmref.so: the reference's sources, main renamed)
class _DBPoint(C.Structure):
    _fields_ = [("i", C.c_int), ("j", C.c_int)]


class _DBRange(C.Structure):
    _fields_ = [("level", C.c_uint), ("lfb", _DBPoint), ("rbt", _DBPoint)]


class DBBlock(C.Structure):
    """DB_Block of src/defs.h:59-68."""
    _fields_ = [("layer", C.c_void_p * 3), ("Aux", C.c_void_p), ("block_id", C.c_int),
                ("range", _DBRange), ("x", C.c_double), ("y", C.c_double), ("z", C.c_double),
                ("dx", C.c_double), ("dy", C.c_double), ("dz", C.c_double),
                ("boundary", C.c_int * 4)]


_ref = None


def ref_lib():
    """Load oracle/_ref/libmbmref.so (None when the reference was not built here)."""
    global _ref
    if _ref is None:
        p = os.path.join(REF_DIR, "libmbmref.so")
        if not os.path.exists(p):
            return None
        L = C.CDLL(p)
        P = C.POINTER
        L.Update.restype = C.c_double
        L.Update.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, DBBlock, C.c_void_p,
                             C.c_double, C.c_double, C.c_int]
        L.TimeUpdate.restype = C.c_double
        L.TimeUpdate.argtypes = [P(DBBlock), C.c_int, C.c_double, C.c_double]
        L.SetBoundary.argtypes = [P(DBBlock), C.c_int, C.c_int, C.c_double]
        L.Steps.restype = C.c_int
        L.Steps.argtypes = [P(DBBlock), C.c_int, P(C.c_double), C.c_double, C.c_double, C.c_double]
        _ref = L
    return _ref


class Reference:
    """The reference's own Update / TimeUpdate / SetBoundary / Steps on numpy layers."""

    def __init__(self, deck: bf.Deck):
        self.L = ref_lib()
        if self.L is None:
            raise FileNotFoundError("oracle/_ref/libmbmref.so not built")
        self.deck = deck
        nb = len(deck.blocks)
        self.B = (DBBlock * nb)()
        self.layer = [[None] * nb for _ in range(3)]
        self.aux = []
        for k, b in enumerate(deck.blocks):
            for l in range(3):
                self.layer[l][k] = np.zeros((b.nyp, b.nxp, NV))
                self.B[k].layer[l] = self.layer[l][k].ctypes.data
            self.aux.append(np.zeros((b.nyp, b.nxp, 3 * NV)))
            self.B[k].Aux = self.aux[k].ctypes.data
            self.B[k].block_id = b.block_id
            self.B[k].range.level = 0
            self.B[k].range.lfb.i = self.B[k].range.lfb.j = 1
            self.B[k].range.rbt.i = b.nxp
            self.B[k].range.rbt.j = b.nyp
            self.B[k].x, self.B[k].y, self.B[k].z = b.x0, b.y0, 0.0
            self.B[k].dx, self.B[k].dy, self.B[k].dz = b.dx, b.dy, 1.0
            for s in range(4):
                self.B[k].boundary[s] = b.bc[s]
        self.set_params(deck)

    def set_params(self, deck: bf.Deck):
        C.c_double.in_dll(self.L, "Kn").value = deck.Kn
        C.c_double.in_dll(self.L, "F").value = deck.F
        C.c_double.in_dll(self.L, "R13").value = deck.R13
        C.c_int.in_dll(self.L, "Limiter").value = deck.limiter

    def set_layer(self, l: int, b: int, U: np.ndarray):
        self.layer[l][b][...] = U.reshape(self.layer[l][b].shape)

    def get_layer(self, l: int, b: int) -> np.ndarray:
        return self.layer[l][b].copy()

    def update(self, b, out_l, in_l, d0_l, dt, t, heun) -> float:
        return self.L.Update(self.layer[out_l][b].ctypes.data, self.layer[in_l][b].ctypes.data,
                             self.aux[b].ctypes.data, self.B[b], self.layer[d0_l][b].ctypes.data,
                             dt, t, heun)

    def set_boundary(self, l: int, t: float):
        self.L.SetBoundary(self.B, len(self.deck.blocks), l, t)

    def time_update(self, dt: float, t: float) -> float:
        return self.L.TimeUpdate(self.B, len(self.deck.blocks), dt, t)
