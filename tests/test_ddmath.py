"""The correctly rounded exp/log of the step-size controller (fosite_b200/csrc/fgpu_ddmath.h):
compiled for the host and checked against binary128 (libquadmath) rounded once to double,
and against Python's decimal module on arguments where libm is known to round differently."""
import ctypes as C
import os
import shutil
import subprocess
import tempfile
from decimal import Decimal, getcontext

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)

SRC = r'''
#include <quadmath.h>
#include "fgpu_ddmath.h"
extern "C" {
double dd_exp(double x) { return fgpu::ddm::exp_cr(x); }
double dd_log(double x) { return fgpu::ddm::log_cr(x); }
double q_exp(double x) { return (double)expq((__float128)x); }
double q_log(double x) { return (double)logq((__float128)x); }
}
'''


@pytest.fixture(scope="module")
def lib():
    cxx = shutil.which("g++") or "g++"
    d = tempfile.mkdtemp()
    src = os.path.join(d, "dd.cpp")
    out = os.path.join(d, "libdd.so")
    with open(src, "w") as f:
        f.write(SRC)
    subprocess.check_call([cxx, "-O2", "-std=c++17", "-ffp-contract=off", "-fPIC", "-shared",
                           "-I", os.path.join(ROOT, "fosite_b200", "csrc"), "-o", out, src, "-l:libquadmath.so.0"])
    L = C.CDLL(out)
    for nm in ("dd_exp", "dd_log", "q_exp", "q_log"):
        getattr(L, nm).argtypes = [C.c_double]
        getattr(L, nm).restype = C.c_double
    return L


def test_matches_binary128(lib):
    rng = np.random.default_rng(5)
    xs = np.exp(rng.uniform(-46.0, 46.0, 20000))
    ys = rng.uniform(-60.0, 60.0, 20000)
    assert all(lib.dd_log(float(x)) == lib.q_log(float(x)) for x in xs)
    assert all(lib.dd_exp(float(y)) == lib.q_exp(float(y)) for y in ys)


def test_hard_cases_against_decimal(lib):
    """Arguments for which glibc 2.39's exp/log are not correctly rounded."""
    getcontext().prec = 80
    for x in ("0x1.4937e52d5064p+0", "-0x1.488fe8772112p+2", "0x1.6a3f34e97562p+3"):
        v = float.fromhex(x)
        assert lib.dd_exp(v) == float(Decimal(v).exp())
    for x in ("0x1.7a0251046d972p-2", "0x1.2556ba996d88bp+0"):
        v = float.fromhex(x)
        assert lib.dd_log(v) == float(Decimal(v).ln())
