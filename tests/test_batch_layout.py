"""Host-side layout of the batched runner (no GPU): every event's blocks are
aligned, disjoint and cover the arenas; the ctypes mirrors of the C structs
have the C sizes."""
import ctypes

import pytest

from clvisc_b200.batch import _Batch, _Ctl, _Event, arena_layout
from clvisc_b200.ideal import plane_stride


@pytest.mark.parametrize('npi', [10, 11])
def test_arena_layout(npi):
    grids = [(121, 121, 1), (301, 301, 1), (17, 15, 5), (1, 1, 1), (255, 3, 2)]
    rows, sizes = arena_layout(grids, npi)
    ends = {'ev': 0, 'pi': 0, 'src': 0, 'cell': 0}
    for (nx, ny, nz), (ld, oe, op, os_, oc) in zip(grids, rows):
        assert ld == plane_stride(nx * ny * nz) and ld % 64 == 0 and ld >= nx * ny * nz
        # consecutive, non-overlapping blocks starting on 64-element (256-byte FP32) boundaries
        assert (oe, op, os_, oc) == (ends['ev'], ends['pi'], ends['src'], ends['cell'])
        for o in (oe, op, os_, oc):
            assert o % 64 == 0
        ends['ev'] += 4 * ld
        ends['pi'] += npi * ld
        ends['src'] += (4 + npi) * ld
        ends['cell'] += ld
    assert sizes == ends


def test_struct_sizes():
    # clv_batch_event: 4 ints + 5 long longs; clv_batch_ctl: int, int, long long, int, int
    assert ctypes.sizeof(_Event) == 56
    assert ctypes.sizeof(_Ctl) == 24
    # clv_batch: 20 pointers/ints laid out with natural alignment (x86-64)
    offs = {f[0]: getattr(_Batch, f[0]).offset for f in _Batch._fields_}
    assert offs['ev'] == 16 and offs['pi'] == 40 and offs['hist_cap'] == 136 and offs['tau0'] == 144
    assert ctypes.sizeof(_Batch) == 176
