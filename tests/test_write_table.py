"""The library's text-table writer (clv_write_table, used for hypersf.dat,
sf_txyz.dat and pimnsf.dat) against numpy.savetxt(fmt='%.6e', header=...),
which the reference calls (ideal.py:304-312, visc.py:413-419): the files must
be equal byte for byte, including special values and empty tables. Host code:
runs without a GPU."""
import numpy as np
import pytest


def _special(dtype):
    vals = [0.0, -0.0, np.inf, -np.inf, np.nan, -np.nan, 1.0, -1.0, 1e-45, -1e-45, 3.4e38, -3.4e38, 1e-38,
            0.1, 2.5e-7, 9.9999995e-7, 123456.789, -0.000123]
    if dtype == np.float64:
        vals += [1e-300, 5e-324, 1.7e308, 0.30000000000000004, 9.9999995e-7]
    a = np.array(vals, dtype=dtype)
    # NaN with the sign bit set
    neg_nan = np.array([np.nan], dtype=dtype).view(np.uint32 if dtype == np.float32 else np.uint64)
    neg_nan |= (1 << (31 if dtype == np.float32 else 63))
    return np.concatenate([a, neg_nan.view(dtype)])


@pytest.mark.parametrize('dtype', [np.float32, np.float64])
@pytest.mark.parametrize('rows,cols', [(0, 10), (1, 8), (1000, 4), (70001, 8)])
def test_write_table_matches_savetxt(tmp_path, dtype, rows, cols):
    from clvisc_b200 import _lib
    rng = np.random.default_rng(rows + cols)
    a = (rng.standard_normal((rows, cols)) * 10.0 ** rng.integers(-12, 12, (rows, cols))).astype(dtype)
    if rows:
        sp = _special(dtype)
        flat = a.reshape(-1)
        flat[:min(flat.size, sp.size)] = sp[:flat.size]
    header = 'Tfrz=%.6e ; other rows: dS0, dS1, dS2, dS3, vx, vy, veta, etas' % 0.137
    want, got = tmp_path / 'want.dat', tmp_path / 'got.dat'
    np.savetxt(want, a, fmt='%.6e', header=header)
    _lib.write_table(str(got), header, a)
    assert got.read_bytes() == want.read_bytes()
