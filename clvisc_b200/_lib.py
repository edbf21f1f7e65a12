"""ctypes binding of libclvisc_b200.so (include/clvisc_b200.h).

The library is the only compute path: if it cannot be loaded, every entry
point raises, there is no CPU fallback.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, 'libclvisc_b200.so')

CLV_PART_IS = 1
CLV_PART_KT = 2
CLV_FLAG_RIEMANN_TEST = 1
CLV_FLAG_GUBSER_VISC_TEST = 2
CLV_FLAG_PIMN_OMEGA_COUPLING = 4
CLV_FLAG_OMEGA_OMEGA_COUPLING = 8
CLV_FLAG_BULK = 16
CLV_FLAG_FAST = 32

CLV_OPT_STAGE_KERNEL = 1
CLV_OPT_TILE = 4
CLV_OPT_CHUNK = 2
CLV_OPT_TILED_BLOCKS = 3
CLV_OPT_TILE2D_ROWS = 5
CLV_OPT_CHUNK2D = 6


def set_option(option, value):
    """Process-wide tuning option of the CUDA library (clv_set_option)."""
    check(load().clv_set_option(int(option), int(value)), 'clv_set_option')

CLV_ERR = {-1: 'invalid argument', -2: 'CUDA error', -3: 'capacity exceeded'}


class ClvParams(ctypes.Structure):
    _fields_ = [
        ('nx', ctypes.c_int), ('ny', ctypes.c_int), ('nz', ctypes.c_int),
        ('ld', ctypes.c_longlong),
        ('precision', ctypes.c_int),
        ('dt', ctypes.c_float), ('dx', ctypes.c_float), ('dy', ctypes.c_float), ('dz', ctypes.c_float),
        ('tau0', ctypes.c_float),
        ('etaos_xmin', ctypes.c_float), ('etaos_ymin', ctypes.c_float),
        ('etaos_left_slop', ctypes.c_float), ('etaos_right_slop', ctypes.c_float), ('lam1', ctypes.c_float),
        ('efrz', ctypes.c_float),
        ('nxskip', ctypes.c_int), ('nyskip', ctypes.c_int), ('nzskip', ctypes.c_int),
        ('eos_ed_start', ctypes.c_float), ('eos_ed_step', ctypes.c_float),
        ('eos_num_ed', ctypes.c_int), ('eos_nrow', ctypes.c_int), ('eos_ncol', ctypes.c_int),
        ('eos_table', ctypes.c_void_p),
        ('flags', ctypes.c_int),
        ('zetaos_max', ctypes.c_float), ('zetaos_t0', ctypes.c_float), ('zetaos_width', ctypes.c_float),
        ('zetaos_skew', ctypes.c_float), ('zetaos_tmin', ctypes.c_float),
        ('opt_stage_kernel', ctypes.c_int), ('opt_chunk', ctypes.c_int), ('opt_tiled_blocks', ctypes.c_int),
        ('opt_tile', ctypes.c_int),
        ('eos_p2', ctypes.c_void_p),
    ]


class ClvGlauber(ctypes.Structure):
    _fields_ = [(n, ctypes.c_float) for n in ('num_of_nucleons', 'sqrts', 'ro0', 'r', 'eta', 'si0',
                                                'impact_parameter', 'edmax', 'hwn', 'eta_flat', 'eta_gw')]


class ClvViscBuffers(ctypes.Structure):
    _fields_ = [
        ('ev_st', ctypes.c_void_p), ('pi_st', ctypes.c_void_p),
        ('ev1', ctypes.c_void_p), ('ev2_ed', ctypes.c_void_p),
        ('pi1', ctypes.c_void_p), ('pi_n', ctypes.c_void_p), ('pi_new_in', ctypes.c_void_p),
        ('ev_new', ctypes.c_void_p), ('pi_new', ctypes.c_void_p),
        ('src', ctypes.c_void_p), ('udiff', ctypes.c_void_p), ('goodcell', ctypes.c_void_p),
        ('edmax_key', ctypes.c_void_p),
        ('write_src', ctypes.c_int), ('write_udiff', ctypes.c_int),
    ]


_lib = None
_load_error = None

_P = ctypes.POINTER(ClvParams)
_VP = ctypes.c_void_p
_SIGS = {
    'clv_version': ([], ctypes.c_int),
    'clv_last_error': ([], ctypes.c_char_p),
    'clv_alignment': ([], ctypes.c_int),
    'clv_set_option': ([ctypes.c_int, ctypes.c_int], ctypes.c_int),
    'clv_ideal_stage': ([_P, ctypes.c_int, ctypes.c_double, _VP, _VP, _VP, _VP, ctypes.c_int, _VP, _VP], ctypes.c_int),
    'clv_visc_stage': ([_P, ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.POINTER(ClvViscBuffers), _VP],
                       ctypes.c_int),
    'clv_visc_initialize': ([_P, _VP, _VP, _VP, _VP, ctypes.c_double, _VP], ctypes.c_int),
    'clv_get_udiff': ([_P, _VP, _VP, _VP, _VP], ctypes.c_int),
    'clv_max_ed_reset': ([_P, _VP, _VP], ctypes.c_int),
    'clv_max_ed': ([_P, _VP, _VP, _VP], ctypes.c_int),
    'clv_max_ed_read': ([_P, _VP, ctypes.POINTER(ctypes.c_double), _VP], ctypes.c_int),
    'clv_hypersf_scratch_bytes': ([_P], ctypes.c_size_t),
    'clv_status': ([_P, _VP, _VP, ctypes.c_int, _VP, _VP, ctypes.c_longlong, _VP, _VP, _VP], ctypes.c_int),
    'clv_params_size': ([], ctypes.c_size_t),
    'clv_hypersf_append': ([_P, ctypes.c_int, ctypes.c_double, ctypes.c_double, _VP, _VP, _VP, _VP, _VP, _VP, _VP,
                            ctypes.c_longlong, _VP, _VP, ctypes.c_size_t, _VP], ctypes.c_int),
    'clv_hypersf_append_noalloc': ([_P, ctypes.c_int, ctypes.c_double, ctypes.c_double, _VP, _VP, _VP, _VP, _VP,
                                    _VP, _VP, ctypes.c_longlong, _VP, _VP], ctypes.c_int),
    'clv_aos_to_soa': ([_P, _VP, _VP, ctypes.c_longlong, ctypes.c_int, _VP], ctypes.c_int),
    'clv_soa_to_aos': ([_P, _VP, _VP, ctypes.c_longlong, ctypes.c_int, _VP], ctypes.c_int),
    # batched events (clv_batch is passed as a pointer to its ctypes mirror in batch.py)
    'clv_batch_stage': ([_P, ctypes.c_int, _VP, ctypes.c_int, ctypes.c_int, ctypes.c_int, _VP], ctypes.c_int),
    'clv_batch_advance': ([_P, _VP, ctypes.c_int, _VP], ctypes.c_int),
    'clv_batch_occupancy': ([_P, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int)], ctypes.c_int),
    'clv_batch_stage_tiled': ([_P, ctypes.c_int, _VP, ctypes.c_int, ctypes.c_int, ctypes.c_int, _VP], ctypes.c_int),
    'clv_batch_occupancy_tiled': ([_P, ctypes.c_int, ctypes.POINTER(ctypes.c_int)], ctypes.c_int),
    # initial conditions (clv_glauber is passed as a pointer to ClvGlauber)
    'clv_glauber_ini': ([_P, _VP, _VP, _VP], ctypes.c_int),
    'clv_glauber_nbinary': ([_P, _VP, _VP, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                             ctypes.c_int, ctypes.c_int, _VP], ctypes.c_int),
    'clv_hotspot_scratch_bytes': ([_P, ctypes.c_int], ctypes.c_size_t),
    # Cooper-Frye spectra (clv_spectra_args is passed as a pointer to spectra.SpectraArgs)
    'clv_spectra_scratch_bytes': ([ctypes.c_longlong, ctypes.c_int, ctypes.c_int, ctypes.c_int], ctypes.c_size_t),
    'clv_spectra': ([_VP, _VP, _VP, ctypes.c_size_t, _VP], ctypes.c_int),
    # learned surrogate (clv_unet_conv is passed as a pointer to surrogate.UnetConv)
    'clv_unet_conv3x3': ([_VP, _VP], ctypes.c_int),
    'clv_unet_set_conv_path': ([ctypes.c_int], ctypes.c_int),
    'clv_write_table': ([ctypes.c_char_p, ctypes.c_char_p, _VP, ctypes.c_int, ctypes.c_longlong, ctypes.c_int],
                        ctypes.c_int),
    'clv_unet_timeouts': ([ctypes.POINTER(ctypes.c_int), ctypes.c_int], ctypes.c_int),
    'clv_unet_wgrad_scratch_bytes': ([ctypes.c_int] * 5, ctypes.c_size_t),
    'clv_unet_wgrad3x3': ([_VP, ctypes.c_int, ctypes.c_int, _VP] + [ctypes.c_int] * 5 + [_VP, ctypes.c_int, _VP,
                          ctypes.c_size_t, _VP], ctypes.c_int),
    'clv_unet_rows_scratch_bytes': ([ctypes.c_int], ctypes.c_size_t),
    'clv_unet_bias_grad': ([_VP, ctypes.c_int, ctypes.c_longlong, ctypes.c_int, _VP, _VP, ctypes.c_size_t, _VP],
                           ctypes.c_int),
    'clv_unet_first_fwd': ([_VP, _VP, _VP] + [ctypes.c_int] * 4 + [_VP, _VP, ctypes.c_int, ctypes.c_int, _VP],
                           ctypes.c_int),
    'clv_unet_first_wgrad': ([_VP, _VP] + [ctypes.c_int] * 4 + [_VP, _VP, ctypes.c_size_t, _VP], ctypes.c_int),
    'clv_unet_head_fwd': ([_VP, ctypes.c_int, ctypes.c_int, _VP, _VP, ctypes.c_longlong, ctypes.c_int, ctypes.c_int,
                           _VP, _VP], ctypes.c_int),
    'clv_unet_head_bwd': ([_VP, ctypes.c_int, ctypes.c_int, _VP, _VP, _VP, ctypes.c_longlong, ctypes.c_int,
                           ctypes.c_int, _VP, _VP, _VP, ctypes.c_size_t, _VP], ctypes.c_int),
    'clv_unet_pool': ([_VP, ctypes.c_int, ctypes.c_int] + [ctypes.c_int] * 4 + [_VP, _VP], ctypes.c_int),
    'clv_unet_up': ([_VP] + [ctypes.c_int] * 4 + [_VP, ctypes.c_int, ctypes.c_int, _VP], ctypes.c_int),
    'clv_unet_skip_grad': ([_VP, ctypes.c_int, ctypes.c_int, _VP, _VP] + [ctypes.c_int] * 4 + [_VP, _VP],
                           ctypes.c_int),
    'clv_unet_up_grad': ([_VP, ctypes.c_int, ctypes.c_int, _VP] + [ctypes.c_int] * 4 + [_VP, _VP], ctypes.c_int),
    'clv_unet_mse': ([_VP, _VP, _VP, ctypes.c_longlong, ctypes.c_int, ctypes.c_float, _VP, _VP, ctypes.c_int, _VP],
                     ctypes.c_int),
    'clv_unet_adam': ([_VP, _VP, _VP, _VP, ctypes.c_longlong, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                       ctypes.c_float, _VP], ctypes.c_int),
    'clv_unet_pack': ([_VP, ctypes.c_int, ctypes.c_int, _VP, _VP, _VP], ctypes.c_int),
    # bulk-evolution diagnostics
    'clv_bulk_slices_size': ([_P], ctypes.c_longlong),
    'clv_bulk_slices': ([_P, _VP, _VP, _VP, _VP], ctypes.c_int),
    'clv_bulk_sums': ([_P, _VP, _VP, _VP, _VP], ctypes.c_int),
    'clv_bulk_lab_scratch_bytes': ([], ctypes.c_size_t),
    'clv_bulk_lab_totals': ([_P, _VP, ctypes.c_double, ctypes.c_double, _VP, _VP, ctypes.c_size_t, _VP],
                            ctypes.c_int),
    'clv_hotspot_ini': ([_P, _VP, _VP, ctypes.c_int] + [ctypes.c_double] * 7 + [_VP, ctypes.c_size_t, _VP],
                        ctypes.c_int),
}


def exported_symbols():
    """Names of the entry points this binding expects the library to export."""
    return sorted(_SIGS)


def load(path=LIB_PATH):
    """Load the CUDA library (raises if it is missing or incomplete)."""
    global _lib, _load_error
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError('libclvisc_b200.so not built (%s); run python -m clvisc_b200.build' % path)
    lib = ctypes.CDLL(path)
    for name, (args, res) in _SIGS.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = res
    _lib = lib
    return lib


def check(rc, what):
    if rc != 0:
        msg = _lib.clv_last_error().decode() if _lib is not None else ''
        raise RuntimeError('%s failed: %s (%d) %s' % (what, CLV_ERR.get(rc, 'error'), rc, msg))


def write_table(path, header, rows):
    """numpy.savetxt(path, rows, fmt='%.6e', header=header), byte for byte,
    by the library's parallel writer; rows is a (n, cols) float32 or float64
    array."""
    import numpy as np
    a = np.ascontiguousarray(rows)
    if a.dtype not in (np.float32, np.float64) or a.ndim != 2:
        raise ValueError('write_table takes a 2-D float32 or float64 array')
    lib = load()
    check(lib.clv_write_table(path.encode(), None if header is None else header.encode(),
                              a.ctypes.data_as(ctypes.c_void_p), a.dtype.itemsize, a.shape[0], a.shape[1]),
          'clv_write_table')


def ptr(t):
    """Device pointer of a torch tensor (or None)."""
    return None if t is None else ctypes.c_void_p(t.data_ptr())
