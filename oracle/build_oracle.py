"""Build recipe of the CPU oracle (test infrastructure, see oracle_smc.cpp).

    python oracle/build_oracle.py <model>    -> oracle/lib/liboracle_<model>.so

The model header must have been emitted first (plomgpu.build.write_header).
Compiled with -ffp-contract=off so that every floating-point operation is
rounded as written, like the reference's plain C build (model_builder/C/Makefile:2).
"""

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
PKG = os.path.join(REPO, 'iterated-inference-pipeline_b200')
OUT = os.path.join(HERE, 'lib')


def lib_path(name):
    return os.path.join(OUT, 'liboracle_%s.so' % name)


def build(name, force=False):
    header = os.path.join(PKG, 'generated', 'model_%s.cuh' % name)
    if not os.path.exists(header):
        raise FileNotFoundError(header)
    out = lib_path(name)
    csrc = os.path.join(PKG, 'csrc')
    srcs = [os.path.join(HERE, 'oracle_smc.cpp'), header, os.path.join(REPO, 'include', 'plomgpu.h')] + \
        [os.path.join(csrc, f) for f in sorted(os.listdir(csrc)) if f.endswith('.h')]
    if not force and os.path.exists(out) and all(os.path.getmtime(out) >= os.path.getmtime(s) for s in srcs):
        return out
    os.makedirs(OUT, exist_ok=True)
    cmd = ['g++', '-O2', '-std=c++17', '-fopenmp', '-ffp-contract=off', '-fPIC', '-shared',
           '-Wno-unknown-pragmas', '-DPLOM_MODEL_HEADER="model_%s.cuh"' % name,
           '-I', os.path.join(PKG, 'csrc'), '-I', os.path.join(PKG, 'generated'), '-I', os.path.join(REPO, 'include'),
           os.path.join(HERE, 'oracle_smc.cpp'), '-o', out]
    subprocess.run(cmd, check=True)
    return out


if __name__ == '__main__':
    for n in sys.argv[1:]:
        print(build(n, force=True))
