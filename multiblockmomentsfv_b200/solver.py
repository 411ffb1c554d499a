"""Python front end of the device solver: the reference's host loop (main(),
src/Main.c:61-164) over the C ABI.

    deck = blockfile.parse_file("cases/squareSmall.txt")
    with Solver(deck, Scenario.named("riemann2d")) as s:
        s.initialise()
        t, n, rej = s.steps(0.0, 0.05)
"""
from __future__ import annotations

import ctypes as C
import time
from typing import List, Optional, Sequence

import numpy as np

from . import _abi
from . import blockfile as bf
from . import output as out
from . import scenario as sc

L_DATA, L_TMP, L_NEW = _abi.L_DATA, _abi.L_TMP, _abi.L_NEW


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class Solver:
    """Device state of one deck: three layers per block on one GPU."""

    def __init__(self, deck: bf.Deck, scenario: Optional[sc.Scenario] = None, device: int = 0,
                 show_every: int = 20, stream: Optional[int] = None, segment_rows: int = 0,
                 max_attempts: int = 0, adjoint: bool = False, mode: str = "exact"):
        """mode: "exact" (bit for bit the reference) or "fast" (MBM_MODE_FAST)."""
        self.deck = deck
        self.scenario = scenario
        self.L = _abi.lib()
        self._descs = _abi.block_descs(deck.blocks)
        p = _abi.Params()
        p.Kn, p.F, p.limiter, p.mode = deck.Kn, deck.F, deck.limiter, _abi.MODES[mode]
        p.device, p.show_every, p.max_attempts, p.segment_rows = device, show_every, max_attempts, segment_rows
        p.stream = stream
        p.adjoint = 1 if adjoint else 0
        self._params = p
        ctx = C.c_void_p()
        st = self.L.mbm_create(self._descs, len(deck.blocks), C.byref(p), C.byref(ctx))
        if st != _abi.MBM_OK:
            raise _abi.MBMError(st, self.L.mbm_last_error(None).decode())
        self.ctx = ctx
        if scenario is not None:
            self.set_dirichlet_from(scenario, 0.0)

    # -- lifetime -------------------------------------------------------------
    def close(self) -> None:
        if getattr(self, "ctx", None):
            self.L.mbm_destroy(self.ctx)
            self.ctx = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st: int) -> None:
        _abi.check(st, self.ctx)

    # -- data -----------------------------------------------------------------
    def upload(self, layer: int, b: int, U: np.ndarray) -> None:
        blk = self.deck.blocks[b]
        U = np.ascontiguousarray(U, dtype=np.float64)
        if U.size != blk.cells * bf.NV:
            raise ValueError("layer array has the wrong size")
        self._check(self.L.mbm_upload(self.ctx, layer, b, _dptr(U)))

    def download(self, layer: int, b: int, out_arr: Optional[np.ndarray] = None) -> np.ndarray:
        blk = self.deck.blocks[b]
        U = out_arr if out_arr is not None else np.empty((blk.nyp, blk.nxp, bf.NV))
        self._check(self.L.mbm_download(self.ctx, layer, b, _dptr(U)))
        return U

    def layers(self, layer: int = L_DATA) -> List[np.ndarray]:
        return [self.download(layer, b) for b in range(len(self.deck.blocks))]

    def load_fields(self, b: int, payload: np.ndarray, faithful: bool = False) -> None:
        """LoadData of block b on the device (mbm_load_fields): payload is the block's zone
        of a result file as stored, ((nx+2)*(ny+2), 10), float32 or float64."""
        blk = self.deck.blocks[b]
        p = np.ascontiguousarray(payload)
        if p.dtype not in (np.float32, np.float64) or p.size != (blk.nx + 2) * (blk.ny + 2) * 10:
            raise ValueError("payload has the wrong type or size")
        self._check(self.L.mbm_load_fields(self.ctx, b, int(p.dtype == np.float32), p.ctypes.data_as(C.c_void_p),
                                           int(bool(faithful))))

    def output_fields(self, b: int, single: bool = True) -> np.ndarray:
        """Output's payload of block b computed on the device: ((nx+2)*(ny+2), 10)."""
        blk = self.deck.blocks[b]
        a = np.empty(((blk.nx + 2) * (blk.ny + 2), 10), dtype=np.float32 if single else np.float64)
        self._check(self.L.mbm_output_fields(self.ctx, b, 1 if single else 0, a.ctypes.data))
        return a

    def output_fields_async(self, b: int, out, single: bool = True) -> None:
        """Start forming block b's payload and copying it to `out`, page-locked host
        memory of ((nx+2)*(ny+2), 10) float32/float64 (see PinnedArray); the copy runs
        beside the next step loop until output_wait()."""
        self._check(self.L.mbm_output_fields_async(self.ctx, b, 1 if single else 0, out.ctypes.data))

    def output_wait(self) -> None:
        self._check(self.L.mbm_output_wait(self.ctx))

    def set_dirichlet(self, b: int, side: int, values: np.ndarray) -> None:
        v = np.ascontiguousarray(values, dtype=np.float64)
        self._check(self.L.mbm_set_dirichlet(self.ctx, b, side, _dptr(v)))

    def set_dirichlet_from(self, s: sc.Scenario, t: float = 0.0) -> None:
        for b, blk in enumerate(self.deck.blocks):
            for side in range(4):
                if blk.bc[side] <= -2:
                    self.set_dirichlet(b, side, sc.dirichlet_edge(s, blk, side, t))

    def initialise(self) -> None:
        """Interior from the scenario, ghosts by SetBoundary (src/Main.c:113-138)."""
        if self.scenario is None:
            raise ValueError("no scenario given")
        for b, blk in enumerate(self.deck.blocks):
            self.upload(L_DATA, b, sc.initial_block(self.scenario, blk))
        self.set_boundary(L_DATA, 0.0)

    # -- the path ---------------------------------------------------------------
    def set_boundary(self, layer: int, t: float) -> None:
        self._check(self.L.mbm_set_boundary(self.ctx, layer, t))

    def update(self, out_layer: int, in_layer: int, data0_layer: int, dt: float, t: float,
               heun: int) -> np.ndarray:
        cfl = np.zeros(len(self.deck.blocks))
        self._check(self.L.mbm_update(self.ctx, out_layer, in_layer, data0_layer, dt, t, heun, _dptr(cfl)))
        return cfl

    def time_update(self, dt: float, t: float) -> float:
        v = C.c_double(0.0)
        self._check(self.L.mbm_time_update(self.ctx, dt, t, C.byref(v)))
        return v.value

    def steps(self, t: float, tend: float, CFLmax: float = 1.0, CFLreg: Optional[float] = None,
              max_steps: int = 0):
        """Steps(): returns (t, accepted steps, rejected attempts).  max_steps > 0
        also ends the loop after that many accepted steps."""
        CFLreg = self.deck.CFL if CFLreg is None else CFLreg
        tt = C.c_double(t)
        n = C.c_int(0)
        r = C.c_int(0)
        self._check(self.L.mbm_steps_capped(self.ctx, C.byref(tt), tend, CFLmax, CFLreg, max_steps,
                                            C.byref(n), C.byref(r)))
        return tt.value, n.value, r.value

    def steps_async(self, t: float, tend: float, CFLmax: float = 1.0, CFLreg: Optional[float] = None,
                    max_steps: int = 0) -> None:
        """Launch Steps() and return at once; steps_wait() collects (t, steps, rejections)."""
        CFLreg = self.deck.CFL if CFLreg is None else CFLreg
        tt = np.array([t], dtype=np.float64)
        te = np.array([tend], dtype=np.float64)
        self._check(self.L.mbm_steps_batch_async(self.ctx, _dptr(tt), _dptr(te), CFLmax, CFLreg, max_steps))

    def steps_wait(self):
        tt = np.zeros(1)
        n, r = C.c_int(0), C.c_int(0)
        self._check(self.L.mbm_steps_batch_wait(self.ctx, _dptr(tt), C.byref(n), C.byref(r)))
        return float(tt[0]), n.value, r.value

    def attempts(self) -> int:
        a = C.c_int(0)
        self._check(self.L.mbm_attempts(self.ctx, C.byref(a)))
        return a.value

    def config(self) -> dict:
        """Launch configuration: rows per work item, work items, persistent CTAs (stage 1),
        and both stages' under "stages"."""
        a, b, c = C.c_int(0), C.c_int(0), C.c_int(0)
        self._check(self.L.mbm_config(self.ctx, C.byref(a), C.byref(b), C.byref(c)))
        stages = []
        for heun in (0, 1):
            r, n, g = C.c_double(0.0), C.c_int(0), C.c_int(0)
            self._check(self.L.mbm_config_stage(self.ctx, heun, C.byref(r), C.byref(n), C.byref(g)))
            stages.append({"segment_rows": round(r.value, 3), "work_items": n.value, "ctas": g.value})
        return {"segment_rows": a.value, "work_items": b.value, "ctas": c.value, "stages": stages}

    def bulk_copies(self) -> bool:
        """Whether the fast stage 2 fills its rows by bulk tensor copies (TMA)."""
        on = C.c_int(0)
        self._check(self.L.mbm_bulk_copies(self.ctx, C.byref(on)))
        return bool(on.value)

    def dependent_launch(self) -> bool:
        """Whether the step loop's kernels use programmatic dependent launch."""
        on = C.c_int(0)
        self._check(self.L.mbm_dependent_launch(self.ctx, C.byref(on)))
        return bool(on.value)

    def ghost_scatter(self) -> bool:
        """Whether the step loop's ghost fills are done inside the stage kernels."""
        on = C.c_int(0)
        self._check(self.L.mbm_ghost_scatter(self.ctx, C.byref(on)))
        return bool(on.value)

    def time_stage(self, heun: int, dt: float, reps: int = 10) -> float:
        """Mean device milliseconds of one stage-kernel launch (CUDA events)."""
        ms = C.c_double(0.0)
        self._check(self.L.mbm_time_stage(self.ctx, heun, dt, reps, C.byref(ms)))
        return ms.value

    def trace(self) -> np.ndarray:
        cap = 4096
        buf = np.zeros((cap, 4))
        n = C.c_int(0)
        self._check(self.L.mbm_trace(self.ctx, _dptr(buf), cap, C.byref(n)))
        return buf[:n.value].copy()


class BatchSolver:
    """Many independent cases (each a deck with its own blocks, Kn, F and limiter) in
    one device context, advanced together by one CUDA-graph loop with per-case dt."""

    def __init__(self, cases, device: int = 0, show_every: int = 0, stream: Optional[int] = None,
                 segment_rows: int = 0, max_attempts: int = 0, mode: str = "exact"):
        """cases: list of (Deck, Scenario or None); mode "exact" or "fast"."""
        self.cases = list(cases)
        self.L = _abi.lib()
        blocks, descs = [], (_abi.CaseDesc * len(self.cases))()
        self.first = []
        for k, (d, _) in enumerate(self.cases):
            descs[k].first_block = len(blocks)
            descs[k].nblocks = len(d.blocks)
            descs[k].Kn, descs[k].F, descs[k].limiter = d.Kn, d.F, d.limiter
            self.first.append(len(blocks))
            blocks.extend(d.blocks)
        self.blocks = blocks
        self._bd = _abi.block_descs(blocks)
        self._cd = descs
        p = _abi.Params()
        p.mode, p.device, p.show_every, p.max_attempts, p.segment_rows = (_abi.MODES[mode], device,
                                                                          show_every, max_attempts, segment_rows)
        p.stream = stream
        p.Kn, p.limiter = self.cases[0][0].Kn, self.cases[0][0].limiter
        self._params = p
        ctx = C.c_void_p()
        st = self.L.mbm_create_batch(self._bd, len(blocks), descs, len(self.cases), C.byref(p), C.byref(ctx))
        if st != _abi.MBM_OK:
            raise _abi.MBMError(st, self.L.mbm_last_error(None).decode())
        self.ctx = ctx
        for k, (d, scn) in enumerate(self.cases):
            if scn is None:
                continue
            for b, blk in enumerate(d.blocks):
                for side in range(4):
                    if blk.bc[side] <= -2:
                        v = np.ascontiguousarray(sc.dirichlet_edge(scn, blk, side, 0.0))
                        _abi.check(self.L.mbm_set_dirichlet(self.ctx, self.first[k] + b, side, _dptr(v)), self.ctx)

    def close(self) -> None:
        if getattr(self, "ctx", None):
            self.L.mbm_destroy(self.ctx)
            self.ctx = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def upload(self, layer: int, k: int, b: int, U: np.ndarray) -> None:
        U = np.ascontiguousarray(U, dtype=np.float64)
        _abi.check(self.L.mbm_upload(self.ctx, layer, self.first[k] + b, _dptr(U)), self.ctx)

    def download(self, layer: int, k: int, b: int) -> np.ndarray:
        blk = self.cases[k][0].blocks[b]
        U = np.empty((blk.nyp, blk.nxp, bf.NV))
        _abi.check(self.L.mbm_download(self.ctx, layer, self.first[k] + b, _dptr(U)), self.ctx)
        return U

    def initialise(self) -> None:
        for k, (d, scn) in enumerate(self.cases):
            for b, blk in enumerate(d.blocks):
                self.upload(L_DATA, k, b, sc.initial_block(scn, blk))
        _abi.check(self.L.mbm_set_boundary(self.ctx, L_DATA, 0.0), self.ctx)

    def steps(self, t, tend, max_steps: int = 0, CFLmax: float = 1.0, CFLreg: float = 0.95,
              check: bool = True):
        """Advance every case; returns (t[], nsteps[], nrej[]).  check=False leaves
        cases that stopped on a non-finite value or the attempt limit to
        case_status() instead of raising."""
        n = len(self.cases)
        tt = np.ascontiguousarray(np.broadcast_to(np.asarray(t, dtype=np.float64), (n,)).copy())
        te = np.ascontiguousarray(np.broadcast_to(np.asarray(tend, dtype=np.float64), (n,)).copy())
        ns = (C.c_int * n)()
        nr = (C.c_int * n)()
        st = self.L.mbm_steps_batch(self.ctx, _dptr(tt), _dptr(te), CFLmax, CFLreg, max_steps, ns, nr)
        if check or st not in (_abi.MBM_ENONFINITE, _abi.MBM_ESTEPLIMIT):
            _abi.check(st, self.ctx)
        return tt, np.array(ns[:]), np.array(nr[:])

    def case_status(self) -> np.ndarray:
        """Per-case status of the last steps() call (MBM_OK, MBM_ENONFINITE, MBM_ESTEPLIMIT)."""
        n = len(self.cases)
        s = (C.c_int * n)()
        _abi.check(self.L.mbm_case_status(self.ctx, s, n), self.ctx)
        return np.array(s[:])

    def attempts(self) -> int:
        a = C.c_int(0)
        _abi.check(self.L.mbm_attempts(self.ctx, C.byref(a)), self.ctx)
        return a.value


def batch_workload(seed: int, ncases: int = 64, nmin: int = 64, nmax: int = 1024):
    """The many-case workload: seeded cases of 1-4 blocks tiling [-1,1]^2 (one block,
    two or three strips, or a 2 x 2 tiling; conforming interfaces), n in [nmin, nmax]
    cells per block side, Kn log-uniform in [1e-3, 1e-1], R13 in {0, 1}, limiter
    uniform over the five, seeded quadrant initial state, open outer edges.
    Returns a list of (Deck, Scenario)."""
    rng = np.random.default_rng(seed)
    out_cases = []
    for k in range(ncases):
        nb = int(rng.integers(1, 5))
        n = int(rng.integers(nmin, nmax + 1))
        B = bf.Block
        if nb == 1:
            blocks = [B(1, -1.0, 1.0, -1.0, 1.0, n, n, (0, 0, 0, 0))]
        elif nb == 2:
            blocks = [B(1, -1.0, 0.0, -1.0, 1.0, n, n, (0, 2, 0, 0)),
                      B(2, 0.0, 1.0, -1.0, 1.0, n, n, (1, 0, 0, 0))]
        elif nb == 3:
            h = 2.0 / 3.0
            blocks = [B(1, -1.0, 1.0, -1.0, -1.0 + h, n, n, (0, 0, 0, 2)),
                      B(2, -1.0, 1.0, -1.0 + h, -1.0 + 2 * h, n, n, (0, 0, 1, 3)),
                      B(3, -1.0, 1.0, -1.0 + 2 * h, 1.0, n, n, (0, 0, 2, 0))]
        else:
            blocks = [B(1, -1.0, 0.0, -1.0, 0.0, n, n, (0, 2, 0, 3)),
                      B(2, 0.0, 1.0, -1.0, 0.0, n, n, (1, 0, 0, 4)),
                      B(3, -1.0, 0.0, 0.0, 1.0, n, n, (0, 4, 1, 0)),
                      B(4, 0.0, 1.0, 0.0, 1.0, n, n, (3, 0, 2, 0))]
        d = bf.Deck(Kn=float(10 ** rng.uniform(-3, -1)), R13=float(rng.integers(0, 2)),
                    limiter=int(rng.integers(0, 5)), CFL=0.95)
        d.blocks = blocks
        out_cases.append((d, sc.Scenario.seeded_quadrant(seed * 1000 + k)))
    return out_cases


def ghost_map(blocks: Sequence[bf.Block]) -> np.ndarray:
    """Resolved ghost sources (host only, no GPU): rows {dst_block, dst_cell, src,
    src_block | flags << 16}."""
    L = _abi.lib()
    descs = _abi.block_descs(blocks)
    n = C.c_int(0)
    _abi.check(L.mbm_ghost_map(descs, len(blocks), None, 0, C.byref(n)))
    arr = np.zeros((max(1, n.value), 4), dtype=np.int32)
    _abi.check(L.mbm_ghost_map(descs, len(blocks), arr.ctypes.data_as(C.POINTER(C.c_int)), n.value,
                               C.byref(n)))
    return arr[:n.value]


class PinnedArray:
    """A numpy array over page-locked host memory (mbm_host_alloc), for the
    asynchronous output copies."""

    def __init__(self, shape, dtype):
        self.L = _abi.lib()
        dt = np.dtype(dtype)
        nbytes = int(np.prod(shape)) * dt.itemsize
        p = C.c_void_p()
        _abi.check(self.L.mbm_host_alloc(nbytes, C.byref(p)))
        self._p = p
        buf = (C.c_char * max(1, nbytes)).from_address(p.value)
        self.array = np.frombuffer(buf, dtype=dt, count=int(np.prod(shape))).reshape(shape)

    def __del__(self):
        try:
            if self._p:
                self.L.mbm_host_free(self._p)
                self._p = None
        except Exception:
            pass


def run(deck: bf.Deck, scenario: sc.Scenario, out_dir: str, single: bool = True, device: int = 0,
        verbose: bool = True, show_every: int = 20, mode: str = "exact", overlap: bool = True,
        initial: Optional[Sequence[np.ndarray]] = None, restart=None):
    """The reference's main() loop on the device: initial state and output at t=0,
    then Steps + Output per output time (src/Main.c:138-156).  Returns (writer, steps).
    overlap: each interval's output is formed on the device right after the interval,
    copied to the host beside the next interval and written to the files while the
    GPU steps on (same files as without).  initial: L_DATA layers to start from instead
    of the scenario's initial state; restart: (per-block payloads as stored in a result
    file, faithful) to start from a restart, loaded on the device (mbm_load_fields)."""
    w = out.Writer(out_dir, deck, scenario.type_name, single)
    ft = np.float32 if single else np.float64
    with Solver(deck, scenario, device=device, show_every=show_every, mode=mode) as s:
        if restart is not None:
            payloads, faithful = restart
            for b, p in enumerate(payloads):
                s.load_fields(b, p, faithful)
            s.set_boundary(L_DATA, 0.0)
        elif initial is not None:
            for b, U in enumerate(initial):
                s.upload(L_DATA, b, U)
            s.set_boundary(L_DATA, 0.0)
        else:
            s.initialise()
        w.write_solver(s, 0.0, -1)
        t, nmax = 0.0, 0
        cells = deck.full_grid_size
        pins = [PinnedArray(((b.nx + 2) * (b.ny + 2), 10), ft) for b in deck.blocks] if overlap else None
        pending = None                      # (t, step count) of an output staged but not written
        for tn in deck.t_out:
            t0 = time.perf_counter()
            if overlap:
                s.steps_async(t, tn, 1.0, deck.CFL)
                if pending is not None:     # the previous output goes to disk while this interval runs
                    s.output_wait()
                    w._write([p.array.tobytes() for p in pins], *pending)
                    pending = None
                t, n, rej = s.steps_wait()
            else:
                t, n, rej = s.steps(t, tn, 1.0, deck.CFL)
            el = time.perf_counter() - t0
            if verbose:
                for step, cfl, tt, dt in s.trace():
                    print(" step: %3d... done.  CFL: %lf, time: %lf, next dt: %lf" % (step, cfl, tt, dt))
                perf = el * 1e6 / max(1, cells * (n + rej))
                print("   %d steps (%d rejected) to t = %g, %.4f us per cell-update" % (n, rej, t, perf))
            nmax += n
            if overlap:
                for b in range(len(deck.blocks)):
                    s.output_fields_async(b, pins[b].array, single)
                pending = (t, nmax)
            else:
                w.write_solver(s, t, nmax)
        if pending is not None:
            s.output_wait()
            w._write([p.array.tobytes() for p in pins], *pending)
    if verbose:
        print("\n Done after %d steps.\n" % nmax)
    return w, nmax
