"""Per-model build: emit the model header and compile the sm_100a engine.

Mirrors the reference's per-model build (``pmbuilder`` renders the model's C
then ``make`` builds ``libplomtpl.a`` and the binaries,
model_builder/Builder.py:286-344, model_builder/C/templates/Makefile:9-14):
here the emitter writes ``generated/model_<name>.cuh`` and nvcc builds
``lib/libplomgpu_<name>.so`` for sm_100a.
"""

import hashlib
import json
import os
import subprocess
import sys

from .emit import Emitter
from .model import PlomModel

PKG_ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REPO_ROOT = os.path.dirname(PKG_ROOT)
CSRC = os.path.join(PKG_ROOT, 'csrc')
GEN = os.path.join(PKG_ROOT, 'generated')
LIB = os.path.join(PKG_ROOT, 'lib')
INCLUDE = os.path.join(REPO_ROOT, 'include')

NVCC = os.environ.get('NVCC', '/usr/local/cuda/bin/nvcc')
ARCH = ['-gencode', 'arch=compute_100a,code=sm_100a']
SMEM_STATE_WORDS = 48


def header_path(name):
    return os.path.join(GEN, 'model_%s.cuh' % name)


def lib_path(name):
    return os.path.join(LIB, 'libplomgpu_%s.so' % name)


def write_header(model, name):
    """Writes the model header if its text changed; returns (path, n_state_words)."""
    os.makedirs(GEN, exist_ok=True)
    em = Emitter(model)
    text = em.header(name)
    path = header_path(name)
    old = open(path).read() if os.path.exists(path) else None
    if old != text:
        with open(path, 'w') as f:
            f.write(text)
    nd = len(model.drift_par_proc)
    S = len(model.par_sv) * model.N_CAC + nd * model.N_CAC + model.N_TS_INC_UNIQUE
    return path, S


def _sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(('.h', '.cuh', '.cu'))) + \
        [os.path.join(INCLUDE, 'plomgpu.h')]


def _stamp(name, extra):
    h = hashlib.sha256()
    for p in _sources() + [header_path(name)]:
        with open(p, 'rb') as f:
            h.update(f.read())
    h.update(json.dumps(extra, sort_keys=True).encode())
    return h.hexdigest()


def nvcc_command(name, S, out=None, verbose_ptxas=False):
    smem = 1 if S > SMEM_STATE_WORDS else 0
    # single precision: flush denormals, hardware-rate sqrt and division, and the
    # special-function-unit forms of exp / log / sin / cos / pow (the FP32 path
    # is assessed statistically; its quantities that cancel are computed in
    # double, and FP64 arithmetic is unaffected).  The approximate forms took
    # the SEIR 20x2 sde step from 0.529 to 0.514 ms and its psr step from 12.4
    # to 11.1 ms per interval.
    cmd = [NVCC] + ARCH + ['-lineinfo', '-O3', '-std=c++17', '--expt-relaxed-constexpr',
                           '--use_fast_math', '-ftz=true', '-prec-div=false', '-prec-sqrt=false',
                           '-Xcompiler', '-fPIC', '-shared',
                           '-DPLOM_MODEL_HEADER="model_%s.cuh"' % name, '-DPLOM_SMEM_STATE=%d' % smem,
                           '-I', CSRC, '-I', GEN, '-I', INCLUDE,
                           os.path.join(CSRC, 'plomgpu_api.cu'), '-o', out or lib_path(name)]
    if verbose_ptxas:
        cmd.insert(1, '-Xptxas=-v')
    return cmd


def build_model(model, name, force=False, verbose=False, out=None):
    """Emit + compile; skips the compile when sources and header are unchanged."""
    _, S = write_header(model, name)
    out = out or lib_path(name)
    os.makedirs(os.path.dirname(out), exist_ok=True)
    stamp_file = out + '.stamp'
    cmd = nvcc_command(name, S, out=out)
    # the compile line (flags included, output path excluded, directories relative to
    # the repository so that a moved checkout keeps its builds) is part of the stamp
    stamp = _stamp(name, {'S': S, 'arch': ARCH,
                          'cmd': [c.replace(REPO_ROOT, '<repo>') for c in cmd if c != out]})
    if not force and os.path.exists(out) and os.path.exists(stamp_file) and open(stamp_file).read() == stamp:
        return out
    if verbose:
        print(' '.join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    with open(stamp_file, 'w') as f:
        f.write(stamp)
    return out


def build_from_files(context, process, link, name, **kw):
    return build_model(PlomModel(context, process, link), name, **kw)


LAUNCHER = """#!/bin/sh
# %(cmd)s for this model directory, on the B200 engine
PYTHONPATH="%(pkg)s${PYTHONPATH:+:$PYTHONPATH}" exec "%(python)s" -m plomgpu %(cmd)s "$@"
"""


def model_dir_name(context, process, link):
    h = hashlib.sha256(json.dumps([context, process, link], sort_keys=True).encode()).hexdigest()
    return 'm%s' % h[:12]


def build_model_dir(context, process, link, out_dir, force=False, name=None, shared_lib=False):
    """A model directory: .settings.json (Builder.write_settings, model_builder/Builder.py:349-351),
    the manifest read by the drivers, the engine library, and smc / pmcmc / mif launchers.
    ``shared_lib`` keeps the library in the package's library folder under ``name``
    (models built once and used from several directories)."""
    model = PlomModel(context, process, link)
    os.makedirs(out_dir, exist_ok=True)
    name = name or model_dir_name(context, process, link)
    lib = lib_path(name) if shared_lib else os.path.join(out_dir, 'lib', 'libplomgpu_%s.so' % name)
    build_model(model, name, force=force, out=lib)
    with open(os.path.join(out_dir, '.settings.json'), 'w') as f:
        json.dump(model.settings(), f)
    with open(os.path.join(out_dir, '.plomgpu.json'), 'w') as f:
        json.dump({'context': context, 'process': process, 'link': link, 'name': name,
                   'library': lib if shared_lib else os.path.join('lib', os.path.basename(lib))}, f)
    for cmd in ('smc', 'pmcmc', 'mif'):
        p = os.path.join(out_dir, cmd)
        with open(p, 'w') as f:
            f.write(LAUNCHER % {'cmd': cmd, 'pkg': PKG_ROOT, 'python': sys.executable})
        os.chmod(p, 0o755)
    return out_dir
