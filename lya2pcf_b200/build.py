"""Build recipe of the native library ``liblya2pcf.so`` (sm_100a only).

    python -m lya2pcf_b200.build          # compile into lya2pcf_b200/
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, 'csrc')
LIB = os.path.join(HERE, 'liblya2pcf.so')
SOURCES = ['context.cu', 'pairs.cu', 'corr.cu', 'adjoint.cu', 'distortion.cu', 'covariance.cu', 'noalloc.cu', 'probe.cu']

NVCC_FLAGS = ['-gencode', 'arch=compute_100a,code=sm_100a', '-O3', '-lineinfo', '-std=c++17',
              '-Xcompiler', '-fPIC', '-cudart', 'static', '--expt-relaxed-constexpr']


def nvcc():
    cand = os.path.join(os.environ.get('CUDA_HOME', '/usr/local/cuda'), 'bin', 'nvcc')
    return cand if os.path.exists(cand) else 'nvcc'


def _stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(ROOT, 'include', 'lya2pcf.h')]
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False, extra=()):
    if not force and not _stale():
        return LIB
    objs = []
    os.makedirs(os.path.join(HERE, '_build'), exist_ok=True)
    for src in SOURCES:
        obj = os.path.join(HERE, '_build', src.replace('.cu', '.o'))
        cmd = [nvcc(), *NVCC_FLAGS, *extra, '-I', os.path.join(ROOT, 'include'), '-I', CSRC, '-c',
               os.path.join(CSRC, src), '-o', obj]
        if verbose:
            print(' '.join(cmd))
        subprocess.run(cmd, check=True)
        objs.append(obj)
    tmp = LIB + '.tmp'
    cmd = [nvcc(), '-gencode', 'arch=compute_100a,code=sm_100a', '-shared', '-cudart', 'static', '-o', tmp, *objs]
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == '__main__':
    build(force='--force' in sys.argv, verbose=True,
          extra=['-Xptxas', '-v'] if '--ptxas' in sys.argv else [])
    print(LIB)
