"""CPU tests of include/st_math.h (exp, sin, cos shared by the kernels and the oracle) against the C library."""
import ctypes as C
import os
import subprocess
import tempfile

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def mathlib():
    src = r'''
#include "st_math.h"
void v_exp(const float* x, float* y, int n) { for (int i = 0; i < n; i++) y[i] = st_expf(x[i]); }
void v_sincos(const float* x, float* s, float* c, int n) { for (int i = 0; i < n; i++) st_sincosf(x[i], &s[i], &c[i]); }
'''
    d = tempfile.mkdtemp()
    c = os.path.join(d, "m.c")
    so = os.path.join(d, "libm_st.so")
    open(c, "w").write(src)
    subprocess.run(["gcc", "-O2", "-ffp-contract=off", "-fPIC", "-shared", "-I", os.path.join(ROOT, "include"), c, "-o", so, "-lm"], check=True)
    lib = C.CDLL(so)
    fp = C.POINTER(C.c_float)
    lib.v_exp.argtypes = [fp, fp, C.c_int]
    lib.v_sincos.argtypes = [fp, fp, fp, C.c_int]
    return lib


def _ulp_err(got, want64):
    want32 = want64.astype(np.float32)
    ulp = np.abs(np.spacing(want32)).astype(np.float64)
    return np.abs(got.astype(np.float64) - want64) / ulp


def call(lib, name, x, nout):
    x = np.ascontiguousarray(x, np.float32)
    outs = [np.zeros_like(x) for _ in range(nout)]
    fp = lambda a: a.ctypes.data_as(C.POINTER(C.c_float))
    getattr(lib, name)(fp(x), *[fp(o) for o in outs], len(x))
    return outs


def test_exp_within_two_ulp(mathlib):
    x = np.concatenate([np.linspace(-87, 88, 200001), np.random.default_rng(0).uniform(-20, 5, 200000)]).astype(np.float32)
    (y,) = call(mathlib, "v_exp", x, 1)
    err = _ulp_err(y, np.exp(x.astype(np.float64)))
    assert err.max() <= 2.0, err.max()


def test_exp_edges(mathlib):
    x = np.array([0.0, -0.0, 1.0, -1.0, 88.7, 89.0, -103.0, -104.0, -87.5, np.nan], np.float32)
    (y,) = call(mathlib, "v_exp", x, 1)
    assert y[0] == 1.0 and y[1] == 1.0
    assert np.isinf(y[5]) and y[7] == 0.0 and np.isnan(y[9])
    assert abs(y[2] / np.e - 1) < 3e-7
    assert 0.0 < y[6] < 1.2e-44 and y[8] > 0.0


def test_sincos_within_two_ulp_on_angles(mathlib):
    x = np.random.default_rng(1).uniform(0.0, 6.2831853, 400000).astype(np.float32)
    s, c = call(mathlib, "v_sincos", x, 2)
    x64 = x.astype(np.float64)
    # absolute error against the magnitude 1 of the unit vector the step builds from them
    assert np.max(np.abs(s - np.sin(x64))) < 2.5e-7
    assert np.max(np.abs(c - np.cos(x64))) < 2.5e-7
    assert np.max(np.abs(s.astype(np.float64) ** 2 + c.astype(np.float64) ** 2 - 1)) < 1e-6
