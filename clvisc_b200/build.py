"""Build libclvisc_b200.so in-tree with nvcc for sm_100a.

The library is compiled without fused multiply-add contraction and with IEEE
division and square root, so each kernel's arithmetic matches a plain
evaluation of the reference OpenCL source in the same precision; the one
exception is clv_fast.cu, the tolerance-arithmetic stage (CLV_FLAG_FAST),
compiled with contraction and approximate division and square root. The
translation units compile in parallel into objects under _build/ and are then
linked into one shared library.

    python -m clvisc_b200.build          # build if sources changed
    python -m clvisc_b200.build --force  # rebuild
"""
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, 'libclvisc_b200.so')
OBJDIR = os.path.join(HERE, '_build')
SOURCES = ['csrc/clv_capi.cu', 'csrc/clv_noalloc.cu', 'csrc/clv_batch.cu', 'csrc/clv_initial.cu',
           'csrc/clv_bulkinfo.cu', 'csrc/clv_spectra.cu', 'csrc/clv_unet.cu', 'csrc/clv_io.cu',
           'csrc/clv_fast.cu']
DEPS = ['csrc/clv_device.cuh', 'csrc/clv_stage.cuh', 'csrc/clv_stage_tiled.cuh', 'csrc/clv_stage_tiled2d.cuh',
        'csrc/clv_misc.cuh',
        'csrc/clv_hypersf.cuh', 'csrc/clv_batch.cuh', 'csrc/clv_initial.cuh',
        'csrc/clv_bulkinfo.cuh', 'csrc/clv_spectra.cuh', 'csrc/clv_unet.cuh', 'csrc/clv_fast.h', 'csrc/clv_batch_launch.cuh', 'csrc/clv_smem16.cuh',
        '../include/clvisc_b200.h']

NVCC_FLAGS = [
    '-gencode', 'arch=compute_100a,code=sm_100a',
    '-O3', '-lineinfo', '-std=c++17',
    '--fmad=false', '-prec-div=true', '-prec-sqrt=true', '-ftz=false',
    '-Xcompiler', '-fPIC',
]
# the tolerance-arithmetic stage (CLV_FLAG_FAST): contraction and approximate
# division / square root in its own translation unit
FAST_FLAGS = [
    '-gencode', 'arch=compute_100a,code=sm_100a',
    '-O3', '-lineinfo', '-std=c++17',
    '--fmad=true', '-prec-div=false', '-prec-sqrt=false', '-ftz=false',
    '-Xcompiler', '-fPIC',
]


def nvcc():
    for cand in (os.environ.get('NVCC'), '/usr/local/cuda/bin/nvcc', 'nvcc'):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return 'nvcc'


def stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(os.path.join(HERE, s)) > t for s in SOURCES + DEPS)


def build(force=False, verbose=False, extra=()):
    if not force and not stale():
        return LIB
    os.makedirs(OBJDIR, exist_ok=True)
    objs = [os.path.join(OBJDIR, os.path.basename(s).replace('.cu', '.o')) for s in SOURCES]

    def compile_one(src_obj):
        src, obj = src_obj
        flags = FAST_FLAGS if src.endswith('clv_fast.cu') else NVCC_FLAGS
        cmd = [nvcc()] + flags + list(extra) + ['-c', '-o', obj, os.path.join(HERE, src)]
        if verbose:
            print(' '.join(cmd), flush=True)
        r = subprocess.run(cmd, cwd=HERE, capture_output=True, text=True)
        return cmd, r

    with ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        results = list(ex.map(compile_one, zip(SOURCES, objs)))
    for cmd, r in results:
        if verbose or r.returncode:
            sys.stdout.write(r.stdout)
            sys.stderr.write(r.stderr)
        if r.returncode:
            raise subprocess.CalledProcessError(r.returncode, cmd)
    link = [nvcc(), '-gencode', 'arch=compute_100a,code=sm_100a', '-shared', '-o', LIB] + objs
    if verbose:
        print(' '.join(link), flush=True)
    subprocess.check_call(link, cwd=HERE)
    return LIB


if __name__ == '__main__':
    extra = ['-Xptxas', '-v'] if '-v' in sys.argv else []
    print(build(force='--force' in sys.argv, verbose=True, extra=extra))
