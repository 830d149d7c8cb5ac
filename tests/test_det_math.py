"""The library's own exp / log / tanh (dev_common.cuh: det_exp_neg, det_log,
det_tanh_pos) against the C library, over their whole domains (CPU).

They are written from +, *, / and ldexp/frexp so that the device and the
oracle compute k-omega SST's blending functions and the wall functions'
log-law alike, bit for bit.  Their error against libm (numpy's exp/log/tanh,
correctly rounded to within an ulp) is bounded here:

  exp(y), y in [-745, 0]:   <= 2 ulp (results above the subnormal range),
                             within one subnormal step below it;
  log(x), x in [1e-300, 1e300] and near 1: <= 2 ulp;
  tanh(x), x >= 0.1:        <= 8 ulp;  x < 0.1: absolute error <= 2.2e-16
                             (1 - e^-2x cancels there; the SST blending uses
                             tanh as a switch between 0 and 1);
  x^-1.30 (det_pow):         relative 4e-16 (1 + |1.3 log x|).
"""
import ctypes as C

import numpy as np
import pytest


@pytest.fixture(scope="module")
def ev(x):
    from importlib import import_module
    L = import_module(x.__name__ + "._lib").lib()

    def f(which, a):
        a = np.ascontiguousarray(a, dtype=np.float64)
        o = np.empty_like(a)
        assert L.xcal_det_math(which, a.ctypes.data_as(C.POINTER(C.c_double)),
                               o.ctypes.data_as(C.POINTER(C.c_double)), a.size) == 0
        return o
    return f


def ulps(a, ref):
    return np.abs(a - ref) / np.spacing(np.abs(ref))


def test_exp(ev):
    rng = np.random.default_rng(0)
    y = -np.concatenate([np.exp(rng.uniform(np.log(1e-300), np.log(745.0), 200_000)),
                         [0.0, 1e-320, 1e-10, 0.5, 1.0, 700.0, 744.0, 745.0]])
    got, ref = ev(0, y), np.exp(y)
    normal = ref >= np.finfo(np.float64).tiny
    assert ulps(got, ref)[normal].max() <= 2.0
    assert np.abs(got - ref)[~normal].max() <= 5e-324
    assert got[y == 0.0][0] == 1.0
    assert ev(0, np.array([-746.0, -1e4]))[0] == 0.0


def test_log(ev):
    rng = np.random.default_rng(1)
    xs = np.concatenate([np.exp(rng.uniform(np.log(1e-300), np.log(1e300), 200_000)),
                         1.0 + rng.uniform(-1e-3, 1e-3, 50_000), [1.0, 2.0, 0.5, np.sqrt(0.5), 10.0]])
    got, ref = ev(1, xs), np.log(xs)
    nz = ref != 0.0
    assert ulps(got, ref)[nz].max() <= 2.0
    assert np.all(got[~nz] == 0.0)


def test_tanh(ev):
    rng = np.random.default_rng(2)
    xs = np.concatenate([rng.uniform(0.0, 30.0, 200_000), np.exp(rng.uniform(np.log(1e-12), np.log(0.1), 50_000)),
                         [0.0, 0.1, 1.0, 19.99, 20.0, 20.01, 1e3]])
    got, ref = ev(2, xs), np.tanh(xs)
    big = xs >= 0.1
    assert ulps(got, ref)[big].max() <= 8.0
    assert np.abs(got - ref)[~big].max() <= 2.2e-16
    assert np.all((got >= 0.0) & (got <= 1.0))
    assert ev(2, np.array([0.0]))[0] == 0.0


def test_pow_m130(ev):
    """x^-1.30 = exp(-1.3 log x) (k-omega LKE's Re_upsilon^-1.30): the log's
    rounding is carried through the product, so the relative error grows
    with |1.3 log x|: within 4e-16 (1 + |1.3 log x|) over [1e-100, 1e100]
    (about 12 ulp over [1e-3, 1e3]); 0 -> Inf, Inf -> 0, 1 -> 1."""
    rng = np.random.default_rng(3)
    xs = np.exp(rng.uniform(np.log(1e-100), np.log(1e100), 200_000))
    got, ref = ev(3, xs), xs ** -1.30
    assert np.all(np.abs(got / ref - 1.0) <= 4e-16 * (1.0 + np.abs(1.3 * np.log(xs))))
    near = np.exp(rng.uniform(np.log(1e-3), np.log(1e3), 100_000))
    assert ulps(ev(3, near), near ** -1.30).max() <= 16.0
    assert ev(3, np.array([1.0]))[0] == 1.0
    z = ev(3, np.array([0.0, np.inf]))
    assert z[0] == np.inf and z[1] == 0.0
