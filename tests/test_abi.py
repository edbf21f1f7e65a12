"""The C-ABI library loads without a GPU and exports every entry point the
public header declares; the Python binding covers the same set."""
import ctypes
import os
import re

import numpy as np

from clvisc_b200 import _lib, build
from clvisc_b200.config import float_literal, read_config

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, 'include')):
        if fn.endswith('.h'):
            text = open(os.path.join(ROOT, 'include', fn)).read()
            text = re.sub(r'/\*.*?\*/', '', text, flags=re.S)
            names |= set(re.findall(r'\b(clv_\w+)\s*\(', text))
    return sorted(names)


def test_library_exports_header_symbols():
    build.build()
    lib = ctypes.CDLL(_lib.LIB_PATH)
    names = header_functions()
    assert len(names) >= 14
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_header():
    assert sorted(_lib.exported_symbols()) == header_functions()


def test_version_and_errors_without_gpu():
    lib = _lib.load()
    assert lib.clv_version() & 0xff00 == 0x0100
    assert lib.clv_alignment() == 16
    p = _lib.ClvParams()
    p.precision = 3
    rc = lib.clv_visc_stage(ctypes.byref(p), 1, 0.6, 3, None, None)
    assert rc == -1
    assert b'precision' in lib.clv_last_error()


def test_float_literals():
    """'%sf' % value as a C compiler reads it (ideal.py:149)."""
    for v in (0.02, 0.16, 0.08, 0.6, 0.15, 0.137, 0.28059564120062497, 1e-05, 30.0, -10.0):
        assert float_literal(v) == float(np.float32(v))
    assert float_literal(0.1) == float(np.float32(0.1))


def test_read_config_overrides():
    cfg = read_config(['--NX', '33', '--DT', '0.005', '--use_float32', 'false', '--riemann_test'])
    assert cfg.NX == 33 and cfg.DT == 0.005
    assert cfg.real == np.float64 and cfg.sz_real == 8
    assert cfg.riemann_test
    assert read_config([]).real == np.float32


def test_params_struct_size_matches_library():
    """The ctypes mirror of clv_params has the library's layout size (a
    binding that drops fields would make the library read past its struct)."""
    lib = _lib.load()
    assert lib.clv_params_size() == ctypes.sizeof(_lib.ClvParams)


def test_arithmetic_flag():
    from clvisc_b200.ideal import fast_arithmetic
    cfg = read_config([])
    assert cfg.arithmetic == 'fast' and fast_arithmetic(cfg)
    cfg.use_float32 = False
    assert fast_arithmetic(cfg)
    cfg.arithmetic = 'auto'
    assert fast_arithmetic(cfg)
    cfg.arithmetic = 'exact'
    assert not fast_arithmetic(cfg)
