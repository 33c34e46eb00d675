"""Test models: the workloads, the reference's example models (from the golden
fixture) and a small coupled SEIR; builders for the GPU and oracle libraries."""

import copy
import functools
import json
import os

from plomgpu import build, model, problem, workloads

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, 'golden', 'reference_codegen.json')


@functools.lru_cache(maxsize=1)
def golden():
    with open(GOLDEN) as f:
        return json.load(f)


@functools.lru_cache(maxsize=None)
def _files(name):
    if name in ('noise', 'drift', 'seir_local'):
        g = golden()['models'][name]
        return g['context'], g['process'], g['link'], g['theta']
    if name == 'sir':
        return workloads.load('sir')
    if name == 'sir_short':
        return workloads.with_data(workloads.sir(n_obs=12), seed=3)
    if name == 'seir3':
        return workloads.with_data(workloads.seir20x2(n_obs=30, n_pop=3), seed=5)
    if name == 'seir20x2':
        return workloads.load('seir20x2')
    raise KeyError(name)


def files(name):
    return copy.deepcopy(_files(name))


LIB_NAME = {'sir_short': 'sir'}  # same model text, other data


def lib_name(name):
    return LIB_NAME.get(name, name)


def plom_model(name):
    c, p, l, _ = files(name)
    return model.PlomModel(c, p, l)


def make_problem(name, **kw):
    c, p, l, th = files(name)
    m = model.PlomModel(c, p, l)
    return problem.Problem(m, m.settings(), th, **kw)


def build_gpu(name):
    return build.build_model(plom_model(name), lib_name(name))


def build_oracle(name):
    build.write_header(plom_model(name), lib_name(name))
    from oracle import Oracle
    return Oracle(lib_name(name))


def engine(name):
    build_gpu(name)
    from plomgpu.native import Engine
    return Engine(lib_name(name))
