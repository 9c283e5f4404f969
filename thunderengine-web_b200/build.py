"""Build the in-tree CUDA library ``libthunderstep.so`` for sm_100a with nvcc.

Arithmetic flags are part of the numerics contract: ``-ftz=true`` (the reference's
results assume flushed subnormals), ``-prec-div=true -prec-sqrt=true`` (correctly
rounded division/sqrt, the reference's div_cr/sqrt_cr) and ``-fmad=false`` (no
multiply-add contraction; fma only where the kernels call fmaf).
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, 'csrc')
LIB = os.path.join(HERE, 'libthunderstep.so')
SOURCES = ['te_player.cu', 'te_kernels.cu', 'te_kernels_fast.cu', 'te_fused.cu', 'te_static_solve.cu',
           'te_adjoint.cu', 'te_ensemble.cu', 'te_selfcheck.cu']
NVCC = os.environ.get('NVCC', '/usr/local/cuda/bin/nvcc')
FLAGS = ['-gencode', 'arch=compute_100a,code=sm_100a', '-O3', '-lineinfo', '-std=c++17',
         '-ftz=true', '-prec-div=true', '-prec-sqrt=true', '-fmad=false',
         '-Xcompiler', '-fPIC', '-Xcompiler', '-fvisibility=default', '--expt-relaxed-constexpr']


def needs_build():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(HERE, '..', 'include', 'thunderstep.h'),
                                                                 __file__]
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force=False, verbose=False):
    if not force and not needs_build():
        return LIB
    objs = []
    procs = []
    for src in SOURCES:
        obj = os.path.join(CSRC, '_' + src.replace('.cu', '.o'))
        cmd = [NVCC] + FLAGS + ['-c', os.path.join(CSRC, src), '-o', obj]
        if verbose:
            print(' '.join(cmd))
        procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
        objs.append(obj)
    for src, p in procs:
        out = p.communicate()[0].decode()
        if p.returncode != 0:
            raise RuntimeError('nvcc failed on %s:\n%s' % (src, out))
        if verbose and out.strip():
            print(out)
    cmd = [NVCC, '-shared', '-gencode', 'arch=compute_100a,code=sm_100a', '-o', LIB] + objs + ['-lcudart']
    out = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)
    if out.returncode != 0:
        raise RuntimeError('link failed:\n' + out.stdout.decode())
    for o in objs:
        os.remove(o)
    return LIB


if __name__ == '__main__':
    build(force='--force' in sys.argv, verbose=True)
    print(LIB)
