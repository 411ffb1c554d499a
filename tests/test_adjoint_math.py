"""The hand-written reverse-mode derivatives of the adjoint (mbm_adjoint_math.cuh),
compiled for the host, against central finite differences of the same maps."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

import helpers as H

SRC = r'''
#include "mbm_adjoint_math.cuh"
using namespace mbm_adj;
extern "C" {
void t_cons(const double* P, double* U) { cons(P, U); }
void t_cons_adj(const double* P, const double* Ub, double* Pb) { cons_adj(P, Ub, Pb); }
void t_prim(const double* U, double* P) { prim(U, P); }
void t_prim_adj(const double* U, const double* Pb, double* Ub) { prim_adj(U, Pb, Ub); }
void t_relax(const double* P, double* Q, double dt, double Kn, double F, int flag) { relax_p(P, Q, dt, Kn, F, flag); }
void t_relax_adj(const double* P, const double* Qb, double* Pb, double* Knb, double dt, double Kn, int flag) {
  relax_p_adj(P, Qb, Pb, Knb, dt, Kn, flag); }
void t_hll(const double* PL, const double* PR, double* f, int dir) { hll_p(PL, PR, f, dir); }
void t_hll_adj(const double* PL, const double* PR, const double* fb, double* PLb, double* PRb, int dir) {
  hll_p_adj(PL, PR, fb, PLb, PRb, dir); }
double t_limit(int lim, double a, double b) { return limit_val(lim, a, b); }
void t_limit_grad(int lim, double a, double b, double* g) { limit_grad(lim, a, b, g, g + 1); }
}
'''


@pytest.fixture(scope="module")
def lib(tmp_path_factory):
    d = tmp_path_factory.mktemp("adj")
    src = d / "t.cpp"
    src.write_text(SRC)
    inc = os.path.join(H.HERE, "..", "multiblockmomentsfv_b200", "csrc")
    so = d / "t.so"
    subprocess.run(["g++", "-O2", "-fPIC", "-shared", "-I", inc, str(src), "-o", str(so)], check=True)
    return C.CDLL(str(so))


def dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def rand_prims(rng):
    return np.array([rng.uniform(0.5, 2), rng.uniform(-0.5, 0.5), rng.uniform(-0.5, 0.5), rng.uniform(0.5, 2),
                     rng.uniform(0.6, 1.8), rng.uniform(-0.2, 0.2), rng.uniform(0.6, 1.8),
                     rng.uniform(-0.1, 0.1), rng.uniform(-0.1, 0.1)])


def check_vjp(f, fadj, x, nout, rng, eps=1e-6, tol=1e-7):
    """<ybar, J v> by central differences against <xbar, v> from the adjoint."""
    for _ in range(4):
        v = rng.standard_normal(x.size)
        yb = rng.standard_normal(nout)
        yp, ym = f(x + eps * v), f(x - eps * v)
        fd = yb @ (yp - ym) / (2 * eps)
        ad = fadj(x, yb) @ v
        assert abs(fd - ad) <= tol * max(1.0, abs(fd)), (fd, ad)


@pytest.mark.parametrize("seed", range(5))
def test_cons_prim_adjoints(lib, seed):
    rng = np.random.default_rng(seed)
    P = rand_prims(rng)
    U = np.zeros(9)
    lib.t_cons(dp(P), dp(U))

    def f_c(x):
        y = np.zeros(9); lib.t_cons(dp(np.ascontiguousarray(x)), dp(y)); return y

    def a_c(x, yb):
        g = np.zeros(9); lib.t_cons_adj(dp(np.ascontiguousarray(x)), dp(np.ascontiguousarray(yb)), dp(g)); return g

    def f_p(x):
        y = np.zeros(9); lib.t_prim(dp(np.ascontiguousarray(x)), dp(y)); return y

    def a_p(x, yb):
        g = np.zeros(9); lib.t_prim_adj(dp(np.ascontiguousarray(x)), dp(np.ascontiguousarray(yb)), dp(g)); return g

    check_vjp(f_c, a_c, P, 9, rng)
    check_vjp(f_p, a_p, U, 9, rng)


@pytest.mark.parametrize("flag", [-1, 0, 1, 2, 3])
def test_relax_adjoint(lib, flag):
    rng = np.random.default_rng(10 + flag)
    P = rand_prims(rng)
    dt, Kn, F = 0.003, 0.01, 0.3
    x = np.append(P, Kn)

    def f(x):
        y = np.zeros(9); lib.t_relax(dp(np.ascontiguousarray(x[:9])), dp(y), dt, x[9], F, flag); return y

    def a(x, yb):
        g = np.zeros(9); kb = C.c_double(0.0)
        lib.t_relax_adj(dp(np.ascontiguousarray(x[:9])), dp(np.ascontiguousarray(yb)), dp(g), C.byref(kb), dt, x[9], flag)
        return np.append(g, kb.value)

    check_vjp(f, a, x, 9, rng, eps=1e-7)


@pytest.fixture(autouse=True)
def _types(lib):
    dpp = C.POINTER(C.c_double)
    lib.t_relax.argtypes = [dpp, dpp, C.c_double, C.c_double, C.c_double, C.c_int]
    lib.t_relax_adj.argtypes = [dpp, dpp, dpp, dpp, C.c_double, C.c_double, C.c_int]


@pytest.mark.parametrize("dirn", [1, 2])
@pytest.mark.parametrize("seed", range(6))
def test_hll_adjoint(lib, seed, dirn):
    rng = np.random.default_rng(seed)
    PL, PR = rand_prims(rng), rand_prims(rng)
    if seed % 3 == 2:                      # supersonic: one of the speeds clipped at 0
        PL[dirn] += 3.0
        PR[dirn] += 3.0
    x = np.concatenate([PL, PR])

    def f(x):
        y = np.zeros(9); lib.t_hll(dp(np.ascontiguousarray(x[:9])), dp(np.ascontiguousarray(x[9:])), dp(y), dirn); return y

    def a(x, yb):
        gl, gr = np.zeros(9), np.zeros(9)
        lib.t_hll_adj(dp(np.ascontiguousarray(x[:9])), dp(np.ascontiguousarray(x[9:])), dp(np.ascontiguousarray(yb)),
                      dp(gl), dp(gr), dirn)
        return np.concatenate([gl, gr])

    check_vjp(f, a, x, 9, rng)


@pytest.mark.parametrize("lim", range(5))
def test_limiter_gradient(lib, lim):
    lib.t_limit.restype = C.c_double
    lib.t_limit.argtypes = [C.c_int, C.c_double, C.c_double]
    rng = np.random.default_rng(lim)
    for _ in range(50):
        a, b = rng.uniform(-1, 1, 2)
        g = np.zeros(2)
        lib.t_limit_grad(lim, C.c_double(a), C.c_double(b), dp(g))
        e = 1e-7
        fa = (lib.t_limit(lim, a + e, b) - lib.t_limit(lim, a - e, b)) / (2 * e)
        fb = (lib.t_limit(lim, a, b + e) - lib.t_limit(lim, a, b - e)) / (2 * e)
        assert abs(fa - g[0]) < 1e-5 and abs(fb - g[1]) < 1e-5, (lim, a, b, g, fa, fb)
