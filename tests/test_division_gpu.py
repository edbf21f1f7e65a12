"""clv::div_by (division through a correctly rounded reciprocal with two
Markstein corrections) must give CUDA's IEEE quotient bit for bit: every float
dividend for each divisor the kernels use, and 2^30 double dividends per
divisor. The check kernels are built from tests/cuda/div_check.cu."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope='module')
def divlib(tmp_path_factory, cuda_lib):
    out = str(tmp_path_factory.mktemp('div') / 'libdivcheck.so')
    subprocess.check_call(['nvcc', '-gencode', 'arch=compute_100a,code=sm_100a', '-O3', '--fmad=false', '-prec-div=true',
                           '-prec-sqrt=true', '-Xcompiler', '-fPIC', '-shared', '-o', out,
                           os.path.join(HERE, 'cuda', 'div_check.cu')])
    lib = ctypes.CDLL(out)
    lib.run_f32.argtypes = [ctypes.c_float, ctypes.POINTER(ctypes.c_ulonglong), ctypes.POINTER(ctypes.c_uint)]
    lib.run_f64.argtypes = [ctypes.c_double, ctypes.c_ulonglong, ctypes.c_ulonglong,
                            ctypes.POINTER(ctypes.c_ulonglong), ctypes.POINTER(ctypes.c_ulonglong)]
    return lib


def divisors():
    f = np.float32
    fixed = [0.08, 0.16, 0.3, 0.8, 0.15, 0.6, 0.01, 0.02, 0.04, 0.005, 3.0, 0.002, 0.01 * 1000]
    out = [f(x) for x in fixed] + [f(0.002) * f(1555)]
    for n in (0, 1, 7, 40, 333, 939, 2000):  # tau of successive steps (dt 0.01 / 0.02) and tau*DZ
        tau = f(0.6 + n * 0.01)
        out += [tau, f(0.15) * tau, f(0.6 + n * 0.02)]
    rng = np.random.default_rng(5)  # per-cell denominators: 1 + DT/tau_pi, e + p
    out += [f(x) for x in np.exp(rng.uniform(np.log(1e-7), np.log(1e4), 12))]
    return out


def test_div_by_f32_exhaustive(divlib):
    bad = ctypes.c_ulonglong()
    first = (ctypes.c_uint * 4)()
    for b in divisors():
        assert divlib.run_f32(float(b), ctypes.byref(bad), first) == 0
        assert bad.value == 0, (float(b), bad.value, [hex(x) for x in first])


def test_div_by_f64_random(divlib):
    bad = ctypes.c_ulonglong()
    first = (ctypes.c_ulonglong * 4)()
    for i, b in enumerate(divisors()):
        bd = float(b)
        for d in (bd, 1.0 / 3.0 * bd):
            assert divlib.run_f64(d, 1 << 30, 1234 + i, ctypes.byref(bad), first) == 0
            assert bad.value == 0, (d, bad.value, [hex(x) for x in first])
