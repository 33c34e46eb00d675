"""Log-likelihood error of the FP32 production arithmetic against FP64.

The production filter keeps particle states, rates, noises, observation
densities and log-weights in FP32 and the log-likelihood accumulation, the
log-sum-exp normalisation and the cumulative weights in FP64.  Its error is
measured conditionally, one interval at a time: the same FP64 particle cloud
is advanced over one observation interval by the FP32 and by the FP64 filter
with paired draws (the FP32 filter consumes the FP64 filter's normals and
resampling uniforms, rounded), and the two llike_n (log mean weight,
model_builder/C/core/smc.c:76) are compared.  The clouds come from one FP64
filter run in segments (its resampled particles after interval n - 1 start
interval n), so the sampled intervals follow a realistic filter path.

Whole filters are not compared this way: on a filter whose weights
degenerate (SEIR 20x2 with 20 series), one ancestor that flips in the last
bits of a weight sends the two filters down different paths, and their
difference is the estimator's own spread (hundreds of nats), not the
precision error.
"""

import copy

import numpy as np


def conditional_interval_errors(engine, problem, stride=1, seed=1, intervals=None):
    """FP32 - FP64 llike of single intervals from the same FP64 cloud, at every ``stride``-th interval
    (or the sorted ``intervals``) of ``problem``: returns (intervals, differences)."""
    off_inc = engine.info.off_inc
    todo = sorted(intervals) if intervals is not None else list(range(0, problem.n_obs, stride))
    cloud = None  # the replicated initial particle
    at = 0        # interval the cloud starts
    out = []
    for n in todo:
        if n > at:
            seg = problem.segment_problem(at, n, cloud)
            seg.seed = seed + 104729 * (at + 1)
            seg.paired_draws = False
            cloud = engine.smc(seg, precision=64, x_final=True).x_final[:off_inc].copy()
            at = n
        q = problem.interval_problem(n, cloud)
        q.seed = seed + 7919 * (n + 1)
        q.paired_draws = True
        l32 = engine.smc(q, precision=32).llike_n[0]
        l64 = engine.smc(q, precision=64).llike_n[0]
        out.append(l32 - l64)
    return np.array(todo), np.array(out)


def summary(problem, intervals, d):
    """Per-interval bias and its standard error, and the whole filter's error they imply
    (n_obs x the per-interval mean)."""
    n = len(d)
    mean = float(np.mean(d))
    se = float(np.std(d, ddof=1) / np.sqrt(n)) if n > 1 else None
    T = problem.n_obs
    return {'per_interval_mean': mean, 'per_interval_se': se, 'per_interval_mean_abs': float(np.mean(np.abs(d))),
            'intervals_sampled': n, 'implied_filter_bias': T * mean,
            'implied_filter_se': None if se is None else T * se, 'unit': 'nats', 'gate_per_filter': 0.5}


def paired_filter_errors(engine, problem, seeds):
    """FP32 - FP64 log-likelihood of whole filters with paired draws, one per seed (meaningful where the
    filter does not degenerate, e.g. the SIR model)."""
    out = []
    for s in seeds:
        q = copy.copy(problem)
        q.seed = s
        q.paired_draws = True
        out.append(engine.smc(q, precision=32).loglik - engine.smc(q, precision=64).loglik)
    return np.array(out)
