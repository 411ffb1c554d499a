"""The stage kernel's shared-reciprocal division (Markstein's correction step:
q = RN(x*r), RN(q + RN(x - q*y)*r) with r = RN(1/y), the inner remainder one FMA)
restated for the host and compared with IEEE x/y bit for bit, inside the range the
kernel admits (mk_in: biased exponent of x in [543, 1503] or x = +-0, y likewise),
and the range test itself against its definition."""
import ctypes as C
import subprocess

import numpy as np
import pytest

SRC = r'''
#include <math.h>
#include <stdint.h>
#include <string.h>
static int64_t bits(double x) { int64_t b; memcpy(&b, &x, 8); return b; }
/* the kernel's mk_in / mk_div, on the host (fma is the correctly rounded libm fma) */
int in_range(double x) {
  const int64_t b = bits(x);
  return (((unsigned)(b >> 52) & 0x7ffu) - 543u <= 960u) || ((b << 1) == 0);
}
double mk_div(double x, double y, double r) {
  const double q = x * r;
  const double m = fma(fma(-q, y, x), r, q);
  return ((bits(x) << 1) == 0) ? q : m;
}
/* count of pairs whose quotient differs from x / y in any bit */
long check(const double* x, const double* y, long n) {
  long bad = 0;
  for (long i = 0; i < n; i++) {
    const double r = 1.0 / y[i];
    const double a = mk_div(x[i], y[i], r), b = x[i] / y[i];
    if (bits(a) != bits(b)) bad++;
  }
  return bad;
}
'''


@pytest.fixture(scope="module")
def lib(tmp_path_factory):
    d = tmp_path_factory.mktemp("div")
    src = d / "d.c"
    src.write_text(SRC)
    so = d / "d.so"
    subprocess.run(["gcc", "-O2", "-ffp-contract=off", "-fPIC", "-shared", str(src), "-o", str(so), "-lm"],
                   check=True)
    L = C.CDLL(str(so))
    L.check.restype = C.c_long
    L.check.argtypes = [C.c_void_p, C.c_void_p, C.c_long]
    L.in_range.argtypes = [C.c_double]
    return L


def _rand(rng, n, emin, emax):
    """Doubles with uniform random mantissas, exponents in [emin, emax], random signs."""
    m = rng.uniform(1.0, 2.0, n)
    e = rng.integers(emin, emax + 1, n)
    s = rng.choice([-1.0, 1.0], n)
    return s * np.ldexp(m, e)


@pytest.mark.parametrize("emin,emax", [(-4, 4), (-60, 60), (-480, 480)])
def test_shared_reciprocal_division_is_ieee(lib, emin, emax):
    rng = np.random.default_rng(emax)
    n = 2_000_000
    x = _rand(rng, n, emin, emax)
    y = _rand(rng, n, emin, emax)
    # the kernel only takes the fast path when both operands are in range
    assert lib.check(x.ctypes.data, y.ctypes.data, n) == 0


def test_quotients_of_near_ties_and_exact_values(lib):
    rng = np.random.default_rng(1)
    y = _rand(rng, 200_000, -30, 30)
    q = _rand(rng, 200_000, -30, 30)
    x = q * y                                    # exact or nearly exact quotients
    x2 = np.nextafter(x, np.inf)
    for a in (x, x2, -x, np.zeros_like(x), -np.zeros_like(x)):
        a = np.ascontiguousarray(a)
        assert lib.check(a.ctypes.data, y.ctypes.data, len(a)) == 0


def test_range_flag(lib):
    assert lib.in_range(0.0) and lib.in_range(-0.0)
    assert lib.in_range(1.0) and lib.in_range(-3.5)
    assert lib.in_range(np.ldexp(1.0, 480)) and lib.in_range(np.ldexp(1.0, -480))
    assert not lib.in_range(np.ldexp(1.0, 481)) and not lib.in_range(np.ldexp(1.0, -481))
    assert not lib.in_range(float("inf")) and not lib.in_range(float("nan"))
    assert not lib.in_range(5e-324)
