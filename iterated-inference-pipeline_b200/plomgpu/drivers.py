"""pmcmc and mif drivers with the reference's flags and output files.

Each likelihood evaluation is one filter on the GPU (a captured plan,
re-launched with new parameters); the drivers restate the host logic of
the reference's binaries around it:

* pmcmc (model_builder/C/pmcmc/main.c, pmcmc.c:39-300): particle marginal
  Metropolis-Hastings with sequential (one component per iteration, shuffled
  every cycle) or full multivariate proposals, the adaptive scaling of the
  full update and the switch to the empirical covariance
  (model_builder/C/core/mcmc_util.c:88-260, mvn.c:97-240), proposals
  constrained so that the initial proportions sum to at most one
  (model_builder/C/core/proposal.c:40-118), the acceptance ratio with priors
  and the change-of-variable terms of the proposal density
  (metropolis_hastings_prior.c:24-56, proposal.c:121-190), a trajectory
  sampled from the genealogy after every full iteration (print.c:715-784);
* mif (model_builder/C/mif/main.c, mif.c:18-247): iterated filtering through
  :class:`plomgpu.mif.Mif`.

Random numbers of the host logic (proposals, acceptance uniforms, shuffles,
trajectory draws, observation draws) come from a numpy Philox stream seeded
with ``--seed`` (default 2 + id); the filters use the engine's Philox streams
with a seed derived per iteration.
"""

import argparse
import math
import sys
import time

import numpy as np

from .best import Best, fmt_g
from .cli import (CliError, NO_DRIFT, common_parser, drift_groups, duration_line, header_x, load_model_dir, log,
                  make_problem, model_name, path_of, read_theta, unlink_done, write_done)


# ---------------------------------------------------------------- change of variable
def f_inv_derivative(kind, x, a, b):
    """router->f_inv_derivative (model_builder/C/core/transform.c:111-180, 330-400).

    The identity and scale_pow10 transformations use f_id as their
    "derivative", which returns x itself; that is restated as is."""
    if kind in ('identity', 'scale_pow10'):
        return x
    if kind in ('log', 'scale_pow10_neg'):
        return math.exp(x)
    if kind == 'logit':
        if x > 0:
            return math.exp(-x) / (1.0 + math.exp(-x)) ** 2
        return math.exp(x) / (1.0 + math.exp(x)) ** 2
    # logit_ab and the bounded scale transformations
    if a == b:
        return x
    if x > 0:
        return (b - a) * math.exp(-x) / (math.exp(-x) + 1.0) ** 2
    return (b - a) * math.exp(x) / (math.exp(x) + 1.0) ** 2


def gaussian_pdf(x, sd):
    return math.exp(-0.5 * (x / sd) ** 2) / (math.sqrt(2.0 * math.pi) * sd)


# ---------------------------------------------------------------- pMCMC state
class McmcState(object):
    """struct s_mcmc_calc_data (build_mcmc_calc_data, model_builder/C/core/mcmc_util.c:18-58)."""

    def __init__(self, best, a, m_switch, m_epsilon, epsilon_max, smooth, alpha):
        n = best.n
        self.acceptance_rates = np.ones(n)
        self.smoothed_acceptance_rates = np.ones(n)
        self.global_acceptance_rate = 0.0
        self.smoothed_global_acceptance_rate = 0.0
        self.has_cycled = True
        self.m_full_iteration = 0
        self.cycle_id = len(best.to_be_estimated) - 1
        self.epsilon = 1.0
        self.epsilon_max = epsilon_max
        self.a = a
        self.alpha = alpha
        self.smooth = smooth
        ne = len(best.to_be_estimated)
        min_switch = 5 * ne * ne
        self.m_switch = min_switch if m_switch < 0 else m_switch
        if 0 <= m_switch < min_switch:
            sys.stderr.write('WARNING: attention: covariance switching iteration (%d) is smaller than proposed one (%d)\n'
                             % (m_switch, min_switch))
        self.m_epsilon = m_epsilon


class Pmcmc(object):
    """One pMCMC chain on the GPU engine."""

    def __init__(self, engine, model, settings, theta, args, plan_factory=None):
        from .native import Plan
        self.args = args
        self.model = model
        self.best = Best(model, theta, is_bayesian=True)
        self.problem = make_problem(model, settings, theta, args)
        self.engine = engine
        self.n_traj = min(args.iter, args.n_traj)
        self.want_traj = self.n_traj > 0 and self.problem.n_obs > 0
        self.plan = (plan_factory or Plan)(engine, self.problem, traj=self.want_traj)
        self.rng = np.random.Generator(np.random.Philox(self.problem.seed))
        self.state = McmcState(self.best, args.cooling, args.switch, args.epsilon, args.epsilon_max, args.smooth,
                               args.alpha)
        self.full = args.full
        n = self.best.n
        self.mean_sampling = np.zeros(n)
        self.var_sampling = np.zeros((n, n))
        self.filter_seed = self.problem.seed

    # -- one likelihood evaluation
    def loglik(self, x):
        self.problem.set_theta(self.best.theta_for(x))
        p = self.problem
        self.filter_seed += 1
        self.plan.update(p.par_cac, p.par_ts, p.x0, self.filter_seed)
        if self.model.drift_par_proc:
            self.plan.update_drift(p.drift_vol)
        self.plan.launch()
        out = self.plan.results()
        return out.loglik

    # -- proposals
    def get_var_and_sd_fac(self, m):
        st, best = self.state, self.best
        ne = len(best.to_be_estimated)
        if self.full:
            if m > st.m_epsilon and m * st.global_acceptance_rate < st.m_switch:
                ar = st.smoothed_global_acceptance_rate if st.smooth else st.global_acceptance_rate
                st.epsilon *= math.exp(math.pow(st.a, m - 1.0) * (ar - 0.234))
            else:
                st.epsilon = 1.0
            st.epsilon = min(st.epsilon, st.epsilon_max)
            sd_fac = st.epsilon * 2.38 / math.sqrt(ne) if ne else 0.0
            var = self.var_sampling if m * st.global_acceptance_rate >= st.m_switch else best.var
            return var, sd_fac
        if ne > 0 and st.has_cycled:
            self.rng.shuffle(best.to_be_estimated)
        return best.var, 1.0

    def ran_proposal(self, proposed, var, sd_fac):
        best, st = self.best, self.state
        if self.full:
            idx = best.to_be_estimated
            n = len(idx)
            proposed[:] = best.mean
            if n:
                work = var[np.ix_(idx, idx)] * sd_fac * sd_fac
                try:
                    L = np.linalg.cholesky(work)
                except np.linalg.LinAlgError:
                    sys.stderr.write('Covariance matrix is not positive definite\n')
                    L = np.linalg.cholesky(work + 1e-12 * np.eye(n))
                proposed[idx] = best.mean[idx] + L @ self.rng.standard_normal(n)
        elif len(best.to_be_estimated):
            k = best.to_be_estimated[st.cycle_id]
            proposed[k] = best.mean[k] + self.rng.normal(0.0, sd_fac * math.sqrt(var[k, k]))

    def check_ic(self, proposed):
        """plom_check_IC_assign_theta_remainder (proposal.c:78-118): number of populations whose
        initial proportions sum above one; assigns the theta remainder."""
        best, model = self.best, self.model
        errors = 0
        sv = [k for k, e in enumerate(best.entries) if e['kind'] == 'sv']
        by_name = {}
        for k in sv:
            by_name.setdefault(best.entries[k]['name'], []).append(k)
        for c in range(model.N_CAC):
            prop = 0.0
            rem_k = None
            for name in model.par_sv:
                ks = by_name[name]
                r = best.entries[ks[0]]['router']
                k = ks[r.map[c]]
                if best.entries[k]['remainder']:
                    rem_k = k
                    continue
                prop += r.natural(r.map[c], proposed[k])
            if prop > 1.0:
                errors += 1
            elif rem_k is not None:
                e = best.entries[rem_k]
                proposed[rem_k] = best._f(e, 1.0 - prop)
        return errors

    def apply_following(self, proposed):
        best = self.best
        index = dict(((e['name'], e['g']), k) for k, e in enumerate(best.entries))
        for k, e in enumerate(best.entries):
            if e['follower']:
                proposed[k] = proposed[index[(e['follow'], e['g'])]]

    def log_prob_proposal(self, proposed, mean, var, sd_fac):
        """log_prob_proposal (proposal.c:121-190); the multivariate density cancels in the ratio."""
        best = self.best
        lp = 0.0
        p_mvn = 1.0
        for k, e in enumerate(best.entries):
            if not best.is_estimated[k]:
                continue
            r, g = e['router'], e['g']
            if self.full:
                p = p_mvn
            else:
                p = gaussian_pdf(proposed[k] - mean[k], sd_fac * math.sqrt(var[k, k]))
            p /= f_inv_derivative(r.f_inv[g], proposed[k], r.min[g], r.max[g])
            if math.isnan(p) or math.isinf(p) or p < 0.0:
                return None
            if self.full:
                p_mvn = p
            else:
                lp += math.log(p)
        if self.full:
            lp = math.log(p_mvn) if p_mvn > 0.0 else float('-inf')
        if math.isinf(lp) or math.isnan(lp):
            return None
        return lp

    def metropolis_hastings(self, ll_new, ll_prev, proposed, var, sd_fac):
        best = self.best
        lq_new = self.log_prob_proposal(proposed, best.mean, var, sd_fac)
        lq_prev = self.log_prob_proposal(best.mean, proposed, var, sd_fac)
        lp_new, err_new = best.log_prob_prior(proposed, self.args.LIKE_MIN)
        lp_prev, err_prev = best.log_prob_prior(best.mean, self.args.LIKE_MIN)
        if lq_new is None or lq_prev is None or err_new or err_prev:
            return False, 0.0
        with np.errstate(over='ignore'):
            alpha = math.exp(min(700.0, ll_new - ll_prev + lq_prev - lq_new + lp_new - lp_prev))
        return self.rng.uniform() < alpha, alpha

    def increment_counters(self):
        st, ne = self.state, len(self.best.to_be_estimated)
        if self.full:
            st.has_cycled = True
            st.m_full_iteration += 1
            st.cycle_id = ne
        elif st.cycle_id >= ne - 1:
            st.has_cycled = True
            st.m_full_iteration += 1
            st.cycle_id = 0
        else:
            st.has_cycled = False
            st.cycle_id += 1

    def compute_acceptance_rates(self, accepted, m):
        st, best = self.state, self.best
        a = 1.0 if accepted else 0.0
        if not self.full and len(best.to_be_estimated):
            mm = best.to_be_estimated[st.cycle_id]
            st.smoothed_acceptance_rates[mm] = (1.0 - st.alpha) * st.smoothed_acceptance_rates[mm] + st.alpha * a
            st.acceptance_rates[mm] += (a - st.acceptance_rates[mm]) / float(st.m_full_iteration)
        st.smoothed_global_acceptance_rate = (1.0 - st.alpha) * st.smoothed_global_acceptance_rate + st.alpha * a
        st.global_acceptance_rate += (a - st.global_acceptance_rate) / float(m)

    def eval_var_emp(self, m):
        """eval_var_emp (mvn.c:196-240): running covariance of the chain's accepted values."""
        x, xb, cov = self.best.mean, self.mean_sampling, self.var_sampling
        d = x - xb
        cov[:] = ((m - 1.0) * cov + ((m - 1.0) / m) * np.outer(d, d)) / m
        xb += d / m

    # -- outputs
    def traj_rows(self, m):
        """sample_traj_and_print: one trajectory of the last filter, printed with index m."""
        rows_t, states = self.plan.sample_traj(self.rng.uniform())
        info = self.engine.info
        p = self.problem
        v = self.engine.particle_values(p, states.T, rows_t)
        nc = info.n_cac
        nsv = info.n_par_sv * nc
        nrem = 0 if info.pop_size_eq_sum_sv else nc
        nts = info.n_ts
        drift = [] if (p.noises_off & NO_DRIFT) else drift_groups(self.model, p)
        mean = v[nsv + nrem:nsv + nrem + nts]
        var = v[info.n_hat:info.n_hat + nts]
        with np.errstate(invalid='ignore'):
            y = mean + np.sqrt(var) * self.rng.standard_normal(mean.shape)
        y = np.where(y > 0.0, y, 0.0)
        times = [0.0] + list(p.t_obs)
        out = []
        base = nsv + nrem + nts
        for r in range(len(rows_t)):
            s = '%d,%s,' % (m, fmt_g(times[rows_t[r]]))
            s += ''.join('%s,' % fmt_g(v[q, r]) for q in range(nsv + nrem + nts))
            for i, (_, groups) in enumerate(drift):
                s += ''.join('%s,' % fmt_g(v[base + i * nc + g, r]) for g in range(len(groups)))
            s += ','.join(fmt_g(y[ts, r]) for ts in range(nts))
            out.append(s + '\n')
        return out

    def acc_header(self):
        s = 'index,epsilon,global_ar'
        if not self.full:
            s += ''.join(',%s:%s' % (e['name'], e['group']) for e in self.best.entries)
        return s + '\n'

    def acc_row(self):
        st = self.state
        s = '%d,%s,%s' % (st.m_full_iteration, fmt_g(st.epsilon), fmt_g(st.global_acceptance_rate))
        if not self.full:
            s += ''.join(',%s' % fmt_g(x) for x in st.acceptance_rates)
        return s + '\n'

    def covariance_text(self):
        """header_covariance + print_covariance (mcmc_util.c:272-340)."""
        vis = self.best.visible()
        lines = [','.join('%s:%s' % (self.best.entries[k]['name'], self.best.entries[k]['group']) for k in vis) + '\n']
        for i in vis:
            lines.append(','.join(fmt_g(self.var_sampling[i, k]) for k in vis) + '\n')
        return lines

    def run(self):
        args, best, st = self.args, self.best, self.state
        f_trace = open(path_of(args, 'trace'), 'w')
        f_trace.write(best.trace_header())
        f_x = None
        if self.want_traj:
            f_x = open(path_of(args, 'X'), 'w')
            f_x.write(header_x(self.model, self.problem))
        f_acc = None
        if args.acc:
            f_acc = open(path_of(args, 'acc'), 'w')
            f_acc.write(self.acc_header())
        thin = max(1, int(float(args.iter) / float(self.n_traj))) if self.n_traj > 0 else 1
        proposed = best.mean.copy()
        t0 = time.time()
        ll = self.loglik(proposed)
        if f_x is not None and self.plan.problem.n_obs:
            f_x.writelines(self.traj_rows(0))
        ll_prev = ll
        best.mean[:] = proposed
        f_trace.write(best.trace_row(0, ll))
        accept = 0
        log(args, 'iteration number:%d\t logV: %s\t accepted:%d computed in:= %s'
            % (0, fmt_g(ll), accept, duration_line(time.time() - t0)[len('Done in:= '):]))
        ne = len(best.to_be_estimated)
        for m in range(1, args.iter):
            t0 = time.time()
            self.increment_counters()
            var, sd_fac = self.get_var_and_sd_fac(m)
            while True:
                self.ran_proposal(proposed, var, sd_fac)
                if self.check_ic(proposed) == 0:
                    break
            self.apply_following(proposed)
            ll_new = self.loglik(proposed)
            accepted, alpha = self.metropolis_hastings(ll_new, ll_prev, proposed, var, sd_fac)
            if accepted:
                ll_prev = ll_new
                best.mean[:] = proposed
                accept += 1
            elif not self.full and ne:
                k = best.to_be_estimated[st.cycle_id]
                proposed[k] = best.mean[k]
            self.compute_acceptance_rates(accepted, m)
            log(args, 'iteration number: %d (%d / %d)\t logV: %s (previous was %s) accepted: %d computed in:= %s'
                % (st.m_full_iteration, st.cycle_id, ne, fmt_g(ll_new), fmt_g(ll_prev), accept,
                   duration_line(time.time() - t0)[len('Done in:= '):]))
            if st.cycle_id >= ne - 1:
                self.eval_var_emp(float(st.m_full_iteration))
                if f_x is not None and st.m_full_iteration % thin == 0:
                    f_x.writelines(self.traj_rows(st.m_full_iteration))
                f_trace.write(best.trace_row(st.m_full_iteration, ll_prev))
                if f_acc is not None:
                    f_acc.write(self.acc_row())
                log(args, 'acceptance rate(s) at iteration %d: %s (smoothed: %s)'
                    % (st.m_full_iteration, fmt_g(st.global_acceptance_rate),
                       fmt_g(st.smoothed_global_acceptance_rate)))
        f_trace.close()
        if f_x is not None:
            f_x.close()
        if f_acc is not None:
            f_acc.close()
        with open(path_of(args, 'covariance'), 'w') as f:
            f.writelines(self.covariance_text())

    def close(self):
        self.plan.close()


def pmcmc_parser():
    ap = common_parser('pmcmc', 'PLOM pMCMC')
    ap.set_defaults(J=1)
    ap.add_argument('--full', action='store_true')
    ap.add_argument('-r', '--acc', action='store_true')
    ap.add_argument('-n', '--n_traj', type=int, default=1000)
    ap.add_argument('-M', '--iter', type=int, default=10)
    ap.add_argument('-a', '--cooling', type=float, default=0.999)
    ap.add_argument('-S', '--switch', type=int, default=-1)
    ap.add_argument('-E', '--epsilon', type=int, default=50)
    ap.add_argument('-f', '--epsilon_max', type=float, default=50.0)
    ap.add_argument('--smooth', action='store_true')
    ap.add_argument('-G', '--alpha', type=float, default=0.02)
    ap.add_argument('-Z', '--zmq', action='store_true')
    ap.add_argument('-c', '--chunk', type=int, default=1)
    return ap


def pmcmc_main(argv, stdin=None, model_dir='.'):
    from .native import Engine
    args = pmcmc_parser().parse_args(argv)
    if args.help:
        print(pmcmc_parser().format_help())
        return 1
    if args.pipe:
        args.quiet = True
    if args.zmq:
        raise CliError('-Z/--zmq: particles are not dispatched across machines; every filter runs on this GPU')
    unlink_done(args)
    model, settings, lib = load_model_dir(model_dir)
    theta = read_theta(stdin)
    engine = Engine(model_name(lib), lib)
    chain = Pmcmc(engine, model, settings, theta, args)
    log(args, 'Starting plom-pmcmc with the following options: i = %d, J = %d, LIKE_MIN = %s, M = %d, n_threads = %d'
        % (args.id, args.J, fmt_g(args.LIKE_MIN), args.iter, args.n_thread))
    t0 = time.time()
    try:
        chain.run()
    finally:
        chain.close()
    write_done(args, chain.best)
    log(args, duration_line(time.time() - t0))
    log(args, 'clean up...')
    return 0


# ---------------------------------------------------------------- MIF
def mif_parser():
    ap = common_parser('mif', 'PLOM MIF')
    ap.set_defaults(J=100)
    ap.add_argument('-r', '--traj', action='store_true')
    ap.add_argument('-M', '--iter', type=int, default=1)
    ap.add_argument('-a', '--cooling', type=float, default=0.975)
    ap.add_argument('-b', '--heat', type=float, default=2.0)
    ap.add_argument('-L', '--lag', type=float, default=0.75)
    ap.add_argument('-S', '--switch', type=int, default=5)
    ap.add_argument('-f', '--ic_only', action='store_true')
    return ap


def mif_main(argv, stdin=None, model_dir='.'):
    from .mif import Mif, MifError
    from .native import Engine
    args = mif_parser().parse_args(argv)
    if args.help:
        print(mif_parser().format_help())
        return 1
    if args.pipe:
        args.quiet = True
    unlink_done(args)
    model, settings, lib = load_model_dir(model_dir)
    theta = read_theta(stdin)
    # L = floor(lag * N_DATA); with -f the filter stops after interval L
    # (build_mif, model_builder/C/mif/build.c:27-45)
    n_data = len(settings['data']['data'])
    L = int(math.floor(args.lag * n_data))
    if L > n_data:
        raise CliError('L > N_DATA (%d > %d). Please choose a L <= %d' % (L, n_data, n_data))
    if args.ic_only:
        args.nb_obs = min(L + 1, n_data)
    problem = make_problem(model, settings, theta, args)
    best = Best(model, theta, is_bayesian=args.prior)
    engine = Engine(model_name(lib), lib)
    try:
        run = Mif(engine, problem, n_runs=1, a=args.cooling, b=args.heat, switch=args.switch, lag=L,
                  prior=best if args.prior else None)
    except MifError as e:
        raise CliError(str(e))
    log(args, 'Starting plom-mif with the following options: i = %d, J = %d, LIKE_MIN = %s, M = %d, a = %s, b = %s, '
        'L = %s, SWITCH = %d, N_THREADS = %d' % (args.id, args.J, fmt_g(args.LIKE_MIN), args.iter, fmt_g(args.cooling),
                                                fmt_g(args.heat), fmt_g(args.lag), args.switch, args.n_thread))
    t_all = time.time()
    index = dict(((e['name'], e['g']), k) for k, e in enumerate(best.entries))
    slots = [index[(c['name'], c['g'])] for c in run.comp]
    f_trace = open(path_of(args, 'trace'), 'w')
    f_trace.write(best.trace_header())
    f_trace.write(best.trace_row(0, float('nan')))
    f_trace.flush()
    f_mif = None
    if args.traj:
        f_mif = open(path_of(args, 'mif'), 'w')
        vis = best.visible()
        f_mif.write('index,time,' + ''.join('mean:%s:%s,var:%s:%s,' % (best.entries[k]['name'], best.entries[k]['group'],
                                                                      best.entries[k]['name'], best.entries[k]['group'])
                                             for k in vis) + 'ess\n')
    seed = problem.seed
    try:
        for m in range(1, args.iter + 1):
            t0 = time.time()
            freeze, sd_init, sd_mut, vt_add = run.schedules(m)
            ll, nf, bart, vt = run.plan.iteration(run.theta_hat, sd_init, sd_mut, vt_add, seed + 1000003 * m)
            run.update(m, bart, vt, run.fixed_lag_means())
            best.mean[slots] = run.theta_hat[0]
            if f_mif is not None:
                f_mif.writelines(_mif_rows(best, run, problem, m, bart[0], vt[0], slots))
            log(args, 'iteration number:%d\t logV: %s\t n_all_fail: %d\t computed in:= %s'
                % (m, fmt_g(ll[0]), nf[0], duration_line(time.time() - t0)[len('Done in:= '):]))
            f_trace.write(best.trace_row(m, ll[0]))
            f_trace.flush()
    finally:
        run.close()
        f_trace.close()
        if f_mif is not None:
            f_mif.close()
    write_done(args, best)
    log(args, duration_line(time.time() - t_all))
    log(args, 'clean up...')
    return 0


def _mif_rows(best, run, problem, m, bart, vt, slots):
    """print_mean_var_theoretical_mif: filtered mean and variance per interval with data
    (values of parameters not fitted are their current best value, variance 0)."""
    rows = []
    vis = best.visible()
    for n in range(problem.n_obs):
        if not run.has_data[n]:
            continue
        s = '%d,%s,' % (m, fmt_g(problem.t_obs[n]))
        for k in vis:
            if k in slots:
                q = slots.index(k)
                s += '%s,%s,' % (fmt_g(bart[n, q]), fmt_g(vt[n, q]))
            else:
                s += '%s,%s,' % (fmt_g(best.mean[k]), fmt_g(0.0))
        rows.append(s + 'nan\n')
    return rows


def main(cmd, argv):
    if cmd == 'pmcmc':
        return pmcmc_main(argv)
    if cmd == 'mif':
        return mif_main(argv)
    raise CliError('unknown command %r' % cmd)
