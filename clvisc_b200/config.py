"""Run configuration, mirroring pyvisc/config.py.

read_config() parses hydro.info (sections path, glauber, geometry, intrinsic,
opencl) and lets every key be overridden on the command line as --KEY value,
plus the boolean switches --riemann_test, --gubser_visc_test,
--pimn_omega_coupling, --omega_omega_coupling, --use_float32 and
--save_to_hdf5 (config.py:69-228). The returned argparse Namespace carries
`real` (numpy float32 or float64) and the byte sizes sz_int, sz_real,
sz_real4, sz_real8. write_config() writes hydro.info into fPathOut
(config.py:13-66).
"""
import argparse
import configparser
import ctypes
import ctypes.util
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))

_libc = ctypes.CDLL(ctypes.util.find_library('c'))
_libc.strtof.restype = ctypes.c_float
_libc.strtof.argtypes = [ctypes.c_char_p, ctypes.c_void_p]


def float_literal(value):
    """The float value of the C literal '%sf' % value, i.e. what the reference
    host passes to its kernels as -D KEY=valuef (ideal.py:149, eos.py:194-197,
    ideal.py:194). Parsed with strtof, so it is the correctly rounded float of
    the decimal text, not of the double."""
    return float(_libc.strtof(str(value).encode(), None))


def set_real(cfg):
    """Element type and sizes for the precision flag (ideal.py:121-136)."""
    cfg.sz_int = 4
    if cfg.use_float32:
        cfg.real = np.float32
        cfg.sz_real, cfg.sz_real4, cfg.sz_real8 = 4, 16, 32
    else:
        cfg.real = np.float64
        cfg.sz_real, cfg.sz_real4, cfg.sz_real8 = 8, 32, 64
    return cfg


def read_config(argv=None, info_path=None):
    """Defaults from hydro.info, updated with command-line options."""
    parser_ini = configparser.ConfigParser()
    parser_ini.read(info_path or os.path.join(_HERE, 'hydro.info'))
    g = parser_ini.get
    gf = parser_ini.getfloat
    gi = parser_ini.getint
    config = {
        'fPathIni': (g('path', 'fPathIni'), 'initial condition path'),
        'fPathOut': (g('path', 'fPathOut'), 'output directory'),
        'Edmax': (gf('glauber', 'Edmax'), 'peak initial energy density'),
        'NumOfNucleons': (gf('glauber', 'NumOfNucleons'), 'nucleons per nucleus'),
        'SQRTS': (gf('glauber', 'SQRTS'), 'beam energy per nucleon pair'),
        'NucleonDensity': (gf('glauber', 'NucleonDensity'), 'Woods-Saxon central density'),
        'Ra': (gf('glauber', 'Ra'), 'nuclear radius'),
        'Eta': (gf('glauber', 'Eta'), 'Woods-Saxon diffuseness'),
        'Si0': (gf('glauber', 'Si0'), 'inelastic cross section'),
        'ImpactParameter': (gf('glauber', 'ImpactParameter'), 'impact parameter'),
        'Hwn': (gf('glauber', 'Hwn'), 'wounded-nucleon fraction'),
        'Eta_flat': (gf('glauber', 'Eta_flat'), 'plateau width in eta_s'),
        'Eta_gw': (gf('glauber', 'Eta_gw'), 'Gaussian fall-off in eta_s'),
        'NX': (gi('geometry', 'NX'), 'cells along x'),
        'NY': (gi('geometry', 'NY'), 'cells along y'),
        'NZ': (gi('geometry', 'NZ'), 'cells along eta_s'),
        'ntskip': (gi('geometry', 'ntskip'), 'output every ntskip steps'),
        'nxskip': (gi('geometry', 'nxskip'), 'output coarsening along x'),
        'nyskip': (gi('geometry', 'nyskip'), 'output coarsening along y'),
        'nzskip': (gi('geometry', 'nzskip'), 'output coarsening along eta_s'),
        'DT': (gf('geometry', 'DT'), 'time step'),
        'DX': (gf('geometry', 'DX'), 'x spacing'),
        'DY': (gf('geometry', 'DY'), 'y spacing'),
        'DZ': (gf('geometry', 'DZ'), 'eta_s spacing'),
        'TAU0': (gf('intrinsic', 'TAU0'), 'starting proper time'),
        'eos_type': (g('intrinsic', 'eos_type'), 'equation of state'),
        'TFRZ': (gf('intrinsic', 'TFRZ'), 'freeze-out temperature'),
        'ETAOS_XMIN': (gf('intrinsic', 'ETAOS_XMIN'), 'T of the eta/s kink'),
        'ETAOS_YMIN': (gf('intrinsic', 'ETAOS_YMIN'), 'eta/s at the kink'),
        'ETAOS_LEFT_SLOP': (gf('intrinsic', 'ETAOS_LEFT_SLOP'), 'eta/s slope below the kink'),
        'ETAOS_RIGHT_SLOP': (gf('intrinsic', 'ETAOS_RIGHT_SLOP'), 'eta/s slope above the kink'),
        'LAM1': (gf('intrinsic', 'LAM1'), 'lambda_1 of the pi^2 term'),
        'ZETAOS_MAX': (gf('intrinsic', 'ZETAOS_MAX'), 'peak zeta/s of the bulk sector (0: off)'),
        'ZETAOS_T0': (gf('intrinsic', 'ZETAOS_T0'), 'T of the zeta/s peak'),
        'ZETAOS_WIDTH': (gf('intrinsic', 'ZETAOS_WIDTH'), 'width of the zeta/s peak'),
        'ZETAOS_SKEW': (gf('intrinsic', 'ZETAOS_SKEW'), 'skewness of the zeta/s peak'),
        'ZETAOS_TMIN': (gf('intrinsic', 'ZETAOS_TMIN'), 'no bulk pressure below this temperature'),
        'BSZ': (gi('opencl', 'local_workgroup_size'), 'work-group size (accepted, unused)'),
        # arithmetic of the fused viscous stage (no counterpart in the
        # reference): 'exact' reproduces the reference's arithmetic bit for
        # bit; 'fast' (the default; 'auto' is the same) contracts
        # multiply-adds and divides through reciprocals, within 1e-5 (FP32) /
        # 1e-11 (FP64) of each field's scale
        'arithmetic': ('fast', 'fused-stage arithmetic: fast or exact'),
    }
    parser = argparse.ArgumentParser(description='CLVisc B200 hydro configuration')
    for key, (val, hlp) in config.items():
        parser.add_argument('--' + key, nargs='?', const=1, type=type(val), default=val, help=hlp)
    for key, default, hlp in [('riemann_test', False, 'drop the Milne source terms'),
                              ('gubser_visc_test', False, 'second-order Gubser test terms'),
                              ('pimn_omega_coupling', False, 'pi-vorticity coupling'),
                              ('omega_omega_coupling', False, 'vorticity-vorticity coupling'),
                              ('use_float32', True, 'float32 (else float64)'),
                              ('save_to_hdf5', False, 'accepted; bulk output is written as text'),
                              ('opencl_interactive', False, 'accepted, unused')]:
        parser.add_argument('--' + key, nargs='?', const=1, type=_str2bool, default=default, help=hlp)
    args, _ = parser.parse_known_args(argv if argv is not None else [])
    return set_real(args)


def _str2bool(v):
    if isinstance(v, bool):
        return v
    return str(v).lower() in ('1', 'true', 'yes', 'on')


def write_config(configs, comments=''):
    """Write the run configuration to fPathOut/hydro.info (config.py:13-66)."""
    os.makedirs(configs.fPathOut, exist_ok=True)
    c = configparser.ConfigParser()
    c.optionxform = str
    c['path'] = {'fPathIni': configs.fPathIni, 'fPathOut': configs.fPathOut}
    c['glauber'] = {k: str(getattr(configs, k)) for k in (
        'Edmax', 'NumOfNucleons', 'SQRTS', 'NucleonDensity', 'Ra', 'Eta', 'Si0', 'ImpactParameter', 'Hwn',
        'Eta_flat', 'Eta_gw')}
    c['geometry'] = {k: str(getattr(configs, k)) for k in (
        'NX', 'NY', 'NZ', 'ntskip', 'nxskip', 'nyskip', 'nzskip', 'DT', 'DX', 'DY', 'DZ')}
    c['intrinsic'] = {k: str(getattr(configs, k)) for k in (
        'TAU0', 'eos_type', 'TFRZ', 'ETAOS_XMIN', 'ETAOS_YMIN', 'ETAOS_LEFT_SLOP', 'ETAOS_RIGHT_SLOP', 'LAM1',
        'ZETAOS_MAX', 'ZETAOS_T0', 'ZETAOS_WIDTH', 'ZETAOS_SKEW', 'ZETAOS_TMIN', 'BSZ')}
    with open(os.path.join(configs.fPathOut, 'hydro.info'), 'w') as f:
        c.write(f)
        f.write('#comments: ' + comments)


cfg = read_config()
