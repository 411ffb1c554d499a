"""Times the reference's own CPU implementation of the Heun path on this host.

TEST/BENCH INFRASTRUCTURE: run by bench.py in a separate process (so its OpenMP
runtime is not shared with torch's) for the cpu_baseline and reference legs.

It loads oracle/_ref/libmbmref_omp.so (the reference's sources built with
-fopenmp; its parallelism is OpenMP over blocks, src/Main.c:236,268,275) and calls
the reference's own Steps (src/Main.c:189-244: TimeUpdate, accept/reject, next dt,
the OpenMP New->Data copy) on the scaled square4 workload: 4 blocks of n x n cells,
seeded quadrant state, open outer edges.  Steps runs to an end time, not a step
count, and restarts dt at 1e-4 on every call; the end time of each call is set from
the step size the CFL control settles at (one TimeUpdate at dt = 1e-4 gives the CFL
number, which scales with dt), so that a call makes about the requested number of
accepted steps; the figure is the accepted steps Steps returns x cells / wall time.
Its progress lines are sent to /dev/null.  Prints one JSON line.
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=0, help="cells per block side; 0 = sized to --budget")
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=0)
    ap.add_argument("--threads", type=int, default=os.cpu_count() or 1)
    ap.add_argument("--budget", type=float, default=60.0, help="seconds of timed CPU work when --n is 0")
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--Kn", type=float, default=0.01)
    ap.add_argument("--limiter", type=int, default=4)
    ap.add_argument("--serial", action="store_true", help="use the serial build")
    a = ap.parse_args()

    os.environ["OMP_NUM_THREADS"] = str(a.threads)
    os.environ.setdefault("OMP_PROC_BIND", "close")
    os.environ.setdefault("OMP_PLACES", "cores")
    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, here)
    import oracle as O
    from multiblockmomentsfv_b200 import scenario as sc
    sys.path.insert(0, os.path.join(os.path.dirname(here), "tests"))
    import helpers as H

    libname = "libmbmref.so" if a.serial else "libmbmref_omp.so"
    O._ref = None
    path = os.path.join(O.REF_DIR, libname)
    if not os.path.exists(path):
        print(json.dumps({"unavailable": f"{libname} not built (make -C oracle ref)"}))
        return
    import ctypes as C
    lib = C.CDLL(path)
    lib.TimeUpdate.restype = C.c_double
    lib.TimeUpdate.argtypes = [C.POINTER(O.DBBlock), C.c_int, C.c_double, C.c_double]
    lib.SetBoundary.argtypes = [C.POINTER(O.DBBlock), C.c_int, C.c_int, C.c_double]
    lib.Steps.restype = C.c_int
    lib.Steps.argtypes = [C.POINTER(O.DBBlock), C.c_int, C.POINTER(C.c_double), C.c_double, C.c_double,
                          C.c_double]
    O._ref = lib
    libc = C.CDLL(None)

    scn = sc.Scenario.seeded_quadrant(a.seed)

    def make(n):
        d = H.quadrant_deck(n, Kn=a.Kn, limiter=a.limiter)
        R = O.Reference(d)
        for b, blk in enumerate(d.blocks):
            R.set_layer(0, b, sc.initial_block(scn, blk))
        R.set_boundary(0, 0.0)
        return d, R

    def settled_dt(R, d, t):
        """the step size the CFL control settles at: dt CFLreg / CFL(dt) at dt = 1e-4
        (TimeUpdate leaves DATA as it is)"""
        cfl = R.time_update(1e-4, t)
        return 1e-4 * d.CFL / cfl

    def run(R, d, t, tend):
        """the reference's Steps (src/Main.c:189-244) from t to tend; returns the new
        time and the accepted steps"""
        tt = C.c_double(t)
        libc.fflush(None)
        saved = os.dup(1)
        null = os.open(os.devnull, os.O_WRONLY)
        os.dup2(null, 1)
        try:
            acc = lib.Steps(R.B, len(d.blocks), C.byref(tt), tend, 1.0, d.CFL)
        finally:
            libc.fflush(None)
            os.dup2(saved, 1)
            os.close(saved)
            os.close(null)
        return tt.value, acc

    n = a.n
    if n <= 0:                                # calibrate on a small grid, then size the sample
        d, R = make(128)
        t0 = time.perf_counter()
        R.time_update(1e-4, 0.0)
        rate = d.full_grid_size / (time.perf_counter() - t0)
        cells = rate * a.budget / max(1, a.steps)
        n = int(max(32, min(1024, (cells / 4) ** 0.5)) // 8 * 8)
    d, R = make(n)
    t = 0.0
    if a.warmup:
        t, _ = run(R, d, t, t + a.warmup * settled_dt(R, d, t))
    tend = t + a.steps * settled_dt(R, d, t)      # about a.steps settled steps (+ the first)
    t0 = time.perf_counter()
    t, acc = run(R, d, t, tend)
    el = time.perf_counter() - t0
    cells = d.full_grid_size
    print(json.dumps({
        "value": cells * acc / el, "unit": "cell-updates/s", "seconds": el,
        "steps": acc, "cells": cells, "n": n,
        "threads": a.threads, "cores": min(a.threads, len(d.blocks)) if not a.serial else 1,
        "build": libname, "driver": "Steps",
    }))


if __name__ == "__main__":
    main()
