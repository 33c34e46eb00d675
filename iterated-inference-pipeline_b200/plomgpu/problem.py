"""Filter problems: settings + theta + options -> the engine's descriptor arrays.

Host-side data preparation of the reference's smc binary
(model_builder/C/smc/main.c:243-278):

* data rows with ``None`` -> NaN (build_data, model_builder/C/core/build.c:757-827);
* integration step ``dt = 1/round(1/dt)`` (build_X, build.c:1299-1303) and
  the substep times of each interval, replaying ``t = t0; while (t < t1)
  {...; t += dt}`` in double (f_prediction_sde_*,
  model_builder/C/core/prediction_util.c:197-287) so that device and oracle
  see the same substep count and times;
* covariates ("par_fixed") interpolated with a natural cubic spline when
  more than 3 points are given, linearly otherwise, a constant for one point
  (build_p_calc, build.c:1067-1210); outside the data range the end value
  is kept (GSL would report a domain error);
* population size at t = 0 for the initial conditions (build.c:1183-1188).
"""

import math

import numpy as np

from .model import PlomModel
from .theta import Parameters


def round_dt(dt):
    if dt <= 0.0:
        dt = 0.25 / 365.0 * 365.0  # default 0.25 day with ONE_YEAR = 365 days (build.c:1297-1300)
    return 1.0 / float(round(1.0 / dt))


def substep_times(t0, t1, dt):
    ts = []
    t = float(t0)
    while t < t1:
        ts.append(t)
        t += dt
    return ts


class Spline(object):
    """Interpolant of one covariate series (natural cubic, linear or constant)."""

    def __init__(self, x, y):
        self.x = np.asarray(x, dtype=float)
        self.y = np.asarray(y, dtype=float)
        n = len(self.x)
        self.kind = 'const' if n == 1 else ('cspline' if n > 3 else 'linear')
        if self.kind == 'cspline':
            self._init_natural()

    def _init_natural(self):
        x, y = self.x, self.y
        n = len(x)
        h = np.diff(x)
        # second derivatives m with m[0] = m[n-1] = 0 (natural boundary)
        A = np.zeros((n - 2, n - 2))
        rhs = np.zeros(n - 2)
        for i in range(1, n - 1):
            k = i - 1
            A[k, k] = 2.0 * (h[i - 1] + h[i])
            if k > 0:
                A[k, k - 1] = h[i - 1]
            if k < n - 3:
                A[k, k + 1] = h[i]
            rhs[k] = 6.0 * ((y[i + 1] - y[i]) / h[i] - (y[i] - y[i - 1]) / h[i - 1])
        m = np.zeros(n)
        if n > 2:
            m[1:-1] = np.linalg.solve(A, rhs)
        self.m = m

    def __call__(self, t):
        x, y = self.x, self.y
        if self.kind == 'const':
            return float(y[0])
        if t <= x[0]:
            return float(y[0])
        if t >= x[-1]:
            return float(y[-1])
        i = int(np.searchsorted(x, t, side='right') - 1)
        i = min(max(i, 0), len(x) - 2)
        h = x[i + 1] - x[i]
        a = (x[i + 1] - t) / h
        b = (t - x[i]) / h
        if self.kind == 'linear':
            return float(a * y[i] + b * y[i + 1])
        mi, mj = self.m[i], self.m[i + 1]
        return float(a * y[i] + b * y[i + 1] + ((a ** 3 - a) * mi + (b ** 3 - b) * mj) * h * h / 6.0)


class Problem(object):
    """Everything one filter needs, as numpy arrays in the descriptor layout."""

    def __init__(self, model, settings, theta, J=1000, dt=1.0, nb_obs=-1, like_min=1e-17,
                 noises_off=0, filter=True, seed=2, precision=32, u_data='D', freeze_forcing=-1.0,
                 ode=False, eps_abs=1e-6, eps_rel=1e-3, psr=False, paired_draws=False):
        if not isinstance(model, PlomModel):
            raise TypeError('model must be a PlomModel')
        m = self.model = model
        self.settings = settings
        self.J = int(J)
        self.like_min = float(like_min)
        self.noises_off = int(noises_off)
        self.filter = bool(filter)
        self.seed = int(seed)
        self.precision = int(precision)
        self.dt = round_dt(dt)
        # deterministic skeleton integrated with step control (the "ode" implementation)
        self.ode = bool(ode)
        self.eps_abs = float(eps_abs)
        self.eps_rel = float(eps_rel)
        if self.ode:
            self.noises_off = 7
        # Poisson system with stochastic rates (the "psr" implementation)
        self.psr = bool(psr)
        # draws of the FP64 filter of the same seed in any precision (precision-error measurement)
        self.paired_draws = bool(paired_draws)
        # optional initial particles one by one, [off_inc][J]
        self.x0_particles = None
        if self.psr and self.ode:
            raise ValueError('psr and ode exclude each other')
        data = settings['data']
        times = data['times']
        rows = data['data']
        n_data = len(rows)
        n_obs = n_data if (nb_obs is None or nb_obs < 0 or nb_obs > n_data) else int(nb_obs)
        self.n_obs = n_obs
        self.data = np.array([[np.nan if v is None else float(v) for v in r] for r in rows[:n_obs]],
                             dtype=float).reshape(n_obs, m.N_TS)
        n_sub, t_sub, t_obs = [], [], []
        for n in range(n_obs):
            ts = substep_times(times[n], times[n + 1], self.dt)
            n_sub.append(len(ts))
            t_sub.extend(ts)
            t_obs.append(float(times[n + 1]))
        self.n_sub = np.array(n_sub, dtype=np.int32)
        self.t_sub = np.array(t_sub, dtype=float)
        self.t_obs = np.array(t_obs, dtype=float)
        # covariates
        em_cov_cac = [p for p in m.par_fixed if p not in m.par_fixed_obs]
        em_cov_ts = [p for p in m.par_fixed if p in m.par_fixed_obs]
        pfv = data.get('par_fixed_values', {})
        self.splines_cac = [[self._spline(pfv[p][c], freeze_forcing) for c in range(m.N_CAC)] for p in em_cov_cac]
        self.splines_ts = [[self._spline(pfv[p][t], freeze_forcing) for t in range(m.N_TS)] for p in em_cov_ts]
        self.cov_cac = np.zeros((len(t_sub), len(em_cov_cac), m.N_CAC))
        for k in range(len(em_cov_cac)):
            for c in range(m.N_CAC):
                sp = self.splines_cac[k][c]
                self.cov_cac[:, k, c] = [sp(t) for t in t_sub]
        self.cov_ts = np.zeros((n_obs, len(em_cov_ts), m.N_TS))
        for k in range(len(em_cov_ts)):
            for t in range(m.N_TS):
                sp = self.splines_ts[k][t]
                self.cov_ts[:, k, t] = [sp(x) for x in t_obs]
        # observation covariates at t = 0, for the summaries of the initial particles
        self.cov_ts0 = np.array([[self.splines_ts[k][t](0.0) for t in range(m.N_TS)]
                                 for k in range(len(em_cov_ts))]).reshape(len(em_cov_ts), m.N_TS)
        if 'N' in em_cov_cac:
            kN = em_cov_cac.index('N')
            self.pop_size_t0 = np.array([self.splines_cac[kN][c](0.0) for c in range(m.N_CAC)])
            # N at 0 and at every observation time (remainder rows of the summaries)
            self.pop_size = np.array([[self.splines_cac[kN][c](t) for c in range(m.N_CAC)]
                                      for t in [0.0] + list(t_obs)])
        else:
            self.pop_size_t0 = np.ones(m.N_CAC)
            self.pop_size = None
        self.coupling = (np.array(data['coupling'], dtype=float) if 'coupling' in data else
                         (np.array(m.coupling, dtype=float) if m.coupling is not None else None))
        self.set_theta(theta, u_data)

    @staticmethod
    def _spline(v, freeze_forcing):
        x, y = list(v['x']), list(v['y'])
        mult = 1.0
        if 'unit' in v:
            from .theta import get_multiplier
            mult = get_multiplier('D', v, 0)
        y = [yy * mult for yy in y]
        if freeze_forcing >= 0.0:
            sp = Spline(x, y)
            c = sp(min(freeze_forcing, x[-1]))
            return Spline([x[0]], [c])
        return Spline(x, y)

    def spline_tables(self):
        """(meta [n_cov_cac * N_CAC][3], x, y, m2): the interpolants of the process covariates for
        the ODE integrator (kind 0 constant, 1 linear, 2 natural cubic; knots, offset)."""
        meta, xs, ys, ms = [], [], [], []
        kinds = {'const': 0, 'linear': 1, 'cspline': 2}
        for per_cac in self.splines_cac:
            for sp in per_cac:
                meta.append((kinds[sp.kind], len(sp.x), len(xs)))
                xs.extend(sp.x.tolist())
                ys.extend(sp.y.tolist())
                ms.extend(sp.m.tolist() if sp.kind == 'cspline' else [0.0] * len(sp.x))
        return (np.array(meta, dtype=np.int32).reshape(-1, 3), np.array(xs, dtype=float),
                np.array(ys, dtype=float), np.array(ms, dtype=float))

    def set_theta(self, theta, u_data='D'):
        self.theta = theta
        self.params = Parameters(self.model, theta, u_data)
        self.par_cac = self.params.par_cac()
        self.par_ts = self.params.par_ts()
        self.x0 = self.params.x0(self.pop_size_t0)
        (self.drift_group, self.drift_ngroups, self.drift_bt, self.drift_vol, _) = self.params.drift_tables()

    def segment_problem(self, n0, n1, x0_particles=None):
        """The filter of observation intervals n0 .. n1 - 1: their substeps, covariates and data
        rows, started from the particles x0_particles ([off_inc][J], FP64) when given."""
        import copy
        if not 0 <= n0 < n1 <= self.n_obs:
            raise ValueError('intervals [%d, %d) outside [0, %d)' % (n0, n1, self.n_obs))
        q = copy.copy(self)
        s0 = int(np.sum(self.n_sub[:n0]))
        s1 = int(np.sum(self.n_sub[:n1]))
        q.n_obs = n1 - n0
        q.n_sub = self.n_sub[n0:n1].copy()
        q.t_sub = self.t_sub[s0:s1].copy()
        q.t_obs = self.t_obs[n0:n1].copy()
        q.data = self.data[n0:n1].copy()
        q.cov_cac = self.cov_cac[s0:s1].copy()
        q.cov_ts = self.cov_ts[n0:n1].copy()
        if n0 > 0:
            q.cov_ts0 = self.cov_ts[n0 - 1].copy()
        if self.pop_size is not None:
            q.pop_size = self.pop_size[n0:n1 + 1].copy()
        q.x0_particles = None if x0_particles is None else np.ascontiguousarray(x0_particles, dtype=float)
        return q

    def interval_problem(self, n, x0_particles=None):
        """The one-interval filter of observation interval n (segment n .. n)."""
        if not 0 <= n < self.n_obs:
            raise ValueError('interval %d outside [0, %d)' % (n, self.n_obs))
        return self.segment_problem(n, n + 1, x0_particles)

    @property
    def particle_steps(self):
        return self.J * self.n_obs

    @classmethod
    def from_files(cls, context, process, link, theta, **kw):
        m = PlomModel(context, process, link)
        return cls(m, m.settings(), theta, **kw)
