"""Batches of filters of one model: many parameter sets, particle counts,
series lengths and data sets evaluated in one persistent launch.

A :class:`BatchProblem` shares the time grid and covariates of one
:class:`~plomgpu.problem.Problem` (the longest series) and carries, per
filter, the natural parameters and initial state of its theta, its particle
count, its number of intervals, its data rows and its seed.
"""

import copy

import numpy as np

from .problem import Problem
from .theta import Parameters


class BatchProblem(object):
    def __init__(self, base, thetas, J, n_obs, data, seeds=None):
        """base: Problem with the longest time grid; thetas: list of theta documents;
        J, n_obs: per filter; data: list of [n_obs_i][N_TS] arrays."""
        if not isinstance(base, Problem):
            raise TypeError('base must be a Problem')
        n = len(thetas)
        if not (len(J) == len(n_obs) == len(data) == n):
            raise ValueError('thetas, J, n_obs and data must have the same length')
        m = base.model
        self.base = base
        self.J = np.asarray(J, dtype=np.int32)
        self.n_obs = np.asarray(n_obs, dtype=np.int32)
        if np.any(self.n_obs > base.n_obs):
            raise ValueError('a filter is longer than the base time grid')
        self.seed = np.asarray(seeds if seeds is not None else np.arange(n) + 1, dtype=np.uint64)
        rows = []
        self.data_row = np.zeros(n, dtype=np.int64)
        r = 0
        for i, d in enumerate(data):
            d = np.asarray(d, dtype=float).reshape(-1, m.N_TS)
            if d.shape[0] != self.n_obs[i]:
                raise ValueError('filter %d: %d data rows for %d intervals' % (i, d.shape[0], self.n_obs[i]))
            self.data_row[i] = r
            rows.append(d)
            r += d.shape[0]
        self.data = np.concatenate(rows, axis=0) if rows else np.zeros((1, m.N_TS))
        pc, pt, x0 = [], [], []
        for th in thetas:
            prm = Parameters(m, th)
            pc.append(prm.par_cac())
            pt.append(prm.par_ts())
            x0.append(prm.x0(base.pop_size_t0))
        self.par_cac = np.array(pc)
        self.par_ts = np.array(pt)
        self.x0 = np.array(x0)

    @property
    def particle_steps(self):
        return int(np.sum(self.J.astype(np.int64) * self.n_obs))

    def single(self, i, precision=None):
        """Problem of filter i alone (same model, data, parameters and seed)."""
        p = copy.copy(self.base)
        p.J = int(self.J[i])
        p.n_obs = int(self.n_obs[i])
        n_sub = self.base.n_sub[:p.n_obs]
        p.n_sub = n_sub
        p.t_sub = self.base.t_sub[:int(np.sum(n_sub))]
        p.t_obs = self.base.t_obs[:p.n_obs]
        p.cov_cac = self.base.cov_cac[:int(np.sum(n_sub))]
        p.cov_ts = self.base.cov_ts[:p.n_obs]
        r = int(self.data_row[i])
        p.data = self.data[r:r + p.n_obs]
        p.par_cac = self.par_cac[i]
        p.par_ts = self.par_ts[i]
        p.x0 = self.x0[i]
        p.seed = int(self.seed[i])
        if precision is not None:
            p.precision = precision
        return p
