"""Command-line drivers with the reference's flags and output files.

``python -m plomgpu <command> ...`` where command is

* ``pmbuilder context.json process.json link.json [-o model]``: build a model
  directory (scripts/pmbuilder + Builder.prepare/render/write_settings,
  model_builder/Builder.py:283-351): ``.settings.json``, the model manifest,
  the sm_100a engine library, and ``smc`` / ``pmcmc`` / ``mif`` launchers;
* ``smc [ode|sde|psr] [options] < theta.json``, run in a model directory
  (model_builder/C/smc/main.c): one particle filter, writing
  ``trace_<id>.csv``, ``hat_<id>.csv``, ``pred_res_<id>.csv`` (and
  ``X_<id>.csv`` with ``-r``), then ``.done_<id>.json`` or, with ``-P``, the
  theta document on stdout;
* ``pmcmc`` and ``mif``: see :mod:`plomgpu.drivers`.

Every filter runs on the GPU through the C ABI; there is no CPU path.
"""

import argparse
import json
import os
import sys
import time

import numpy as np

from .best import Best, fmt_g

IMPLEMENTATIONS = ('ode', 'sde', 'psr')
NO_DEM, NO_ENV, NO_DRIFT = 1, 2, 4
MANIFEST = '.plomgpu.json'
SETTINGS = '.settings.json'


class CliError(Exception):
    pass


# ---------------------------------------------------------------- arguments
def common_parser(prog, description):
    """Options shared by smc / pmcmc / mif (model_builder/C/smc/main.c:90-206)."""
    ap = argparse.ArgumentParser(prog=prog, description=description, add_help=False)
    ap.add_argument('implementation', nargs='?', default='psr', choices=IMPLEMENTATIONS)
    ap.add_argument('-x', '--no_dem_sto', action='store_true')
    ap.add_argument('-y', '--no_white_noise', action='store_true')
    ap.add_argument('-z', '--no_diff', action='store_true')
    ap.add_argument('-s', '--DT', type=float, default=0.0)
    ap.add_argument('-v', '--eps_abs', type=float, default=1e-6)
    ap.add_argument('-w', '--eps_rel', type=float, default=1e-3)
    ap.add_argument('-o', '--nb_obs', type=int, default=-1)
    ap.add_argument('-g', '--freeze_forcing', type=float, default=-1.0)
    ap.add_argument('-h', '--help', action='store_true')
    ap.add_argument('-p', '--path', default='./')
    ap.add_argument('--prior', action='store_true')
    ap.add_argument('-i', '--id', type=int, default=0)
    ap.add_argument('-N', '--n_thread', type=int, default=1)
    ap.add_argument('-J', type=int, default=1)
    ap.add_argument('-l', '--LIKE_MIN', type=float, default=1e-17)
    ap.add_argument('-q', '--quiet', action='store_true')
    ap.add_argument('-P', '--pipe', action='store_true')
    # B200 engine options (no counterpart in the reference)
    ap.add_argument('--precision', type=int, choices=(32, 64), default=32,
                    help='particle state precision on the GPU (reductions are FP64 either way)')
    ap.add_argument('--seed', type=int, default=None, help='Philox seed (default 2 + id, as the reference seeds its RNG)')
    return ap


def noises_off_of(args):
    n = 0
    if args.no_dem_sto:
        n |= NO_DEM
    if args.no_white_noise:
        n |= NO_ENV
    if args.no_diff:
        n |= NO_DRIFT
    if args.implementation == 'ode':
        n |= NO_DEM | NO_ENV | NO_DRIFT
    return n


def path_of(args, name, ext='csv'):
    return '%s%s_%d.%s' % (args.path, name, args.id, ext)


def log(args, msg):
    if not args.quiet:
        print(msg)
        sys.stdout.flush()


# ---------------------------------------------------------------- model directory
def load_model_dir(path='.'):
    """(PlomModel, settings dict, engine library name) of a model directory."""
    from .model import PlomModel
    man = os.path.join(path, MANIFEST)
    if not os.path.exists(man):
        raise CliError('%s not found: run the command in a model directory made by pmbuilder' % man)
    with open(man) as f:
        m = json.load(f)
    with open(os.path.join(path, SETTINGS)) as f:
        settings = json.load(f)
    model = PlomModel(m['context'], m['process'], m['link'])
    lib = m['library']
    if not os.path.isabs(lib):
        lib = os.path.join(os.path.abspath(path), lib)
    return model, settings, lib


def read_theta(stream=None):
    """One line of JSON on stdin (load_json, model_builder/C/core/json.c:359-383)."""
    line = (stream or sys.stdin).readline()
    try:
        return json.loads(line)
    except ValueError as e:
        raise CliError('could not parse theta.json\nerror: %s' % e)


def make_problem(model, settings, theta, args, J=None, filter=True):
    from .problem import Problem
    seed = args.seed if args.seed is not None else 2 + args.id
    noises_off = noises_off_of(args)
    # sde with every noise and the drift off is integrated as the ode (get_f_pred,
    # model_builder/C/core/prediction_util.c:138-150)
    ode = args.implementation == 'ode' or (args.implementation == 'sde' and noises_off == 7)
    return Problem(model, settings, theta, J=J or args.J, dt=args.DT, nb_obs=args.nb_obs, like_min=args.LIKE_MIN,
                   noises_off=noises_off, filter=filter, seed=seed, precision=args.precision,
                   freeze_forcing=args.freeze_forcing, ode=ode, eps_abs=args.eps_abs, eps_rel=args.eps_rel,
                   psr=(args.implementation == 'psr'))


# ---------------------------------------------------------------- output formats
def header_hat(model, problem, drift=True):
    """header_hat (model_builder/C/core/print.c:146-186)."""
    s = 'time,'
    for name in model.par_sv:
        for cac in model.cac_id:
            s += 'low95:%s:%s,%s:%s,high95:%s:%s,' % (name, cac, name, cac, name, cac)
    if model.remainder is not None:
        for cac in model.cac_id:
            r = model.remainder
            s += 'low95:%s:%s,%s:%s,high95:%s:%s,' % (r, cac, r, cac, r, cac)
    ts = model.ts_id
    for i, t in enumerate(ts):
        s += 'low95:%s,%s,high95:%s%s' % (t, t, t, ',' if i < len(ts) - 1 else '')
    for name, groups in (drift_groups(model, problem) if drift else []):
        for g in groups:
            s += ',low95:diff:%s:%s,diff:%s:%s,high95:diff:%s:%s' % (name, g, name, g, name, g)
    return s + '\n'


def drift_groups(model, problem=None, params=None):
    """[(parameter, [group names])] of the drifted parameters (p_it_only_drift)."""
    out = []
    params = params if params is not None else (problem.params if problem is not None else None)
    for p in model.drift_par_proc:
        out.append((p, list(params.routers[p].group_name) if params is not None else []))
    return out


def hat_rows(model, problem, hat, drift=True):
    """print_p_hat (print.c:445-573): one row per time (0, then every t_obs)."""
    nc = model.N_CAC
    nsv = len(model.par_sv) * nc
    nrem = 0 if model.remainder is None else nc
    nts = model.N_TS
    times = [0.0] + list(problem.t_obs)
    dg = drift_groups(model, problem)
    rows = []
    for n, t in enumerate(times):
        h = hat[n]
        s = '%s,' % fmt_g(t)
        for q in range(nsv + nrem):
            s += '%s,%s,%s,' % (fmt_g(h[q, 0]), fmt_g(h[q, 1]), fmt_g(h[q, 2]))
        for i in range(nts):
            q = nsv + nrem + i
            s += '%s,%s,%s%s' % (fmt_g(h[q, 0]), fmt_g(h[q, 1]), fmt_g(h[q, 2]), ',' if i < nts - 1 else '')
        if drift:
            base = nsv + nrem + nts
            for i, (_, groups) in enumerate(dg):
                for g in range(len(groups)):
                    q = base + i * nc + g
                    s += ',%s,%s,%s' % (fmt_g(h[q, 0]), fmt_g(h[q, 1]), fmt_g(h[q, 2]))
        rows.append(s + '\n')
    return rows


def header_pred_res(model):
    """header_prediction_residuals (print.c:132-143)."""
    return 'time,' + ''.join('mean:%s,res:%s,' % (t, t) for t in model.ts_id) + 'ess\n'


def pred_res_rows(problem, pred_res, ess):
    """print_prediction_residuals (print.c:632-711): intervals that were filtered."""
    rows = []
    if not problem.filter:
        return rows
    for n in range(problem.n_obs):
        if np.all(np.isnan(problem.data[n])):
            continue
        s = '%s,' % fmt_g(problem.t_obs[n])
        for ts in range(pred_res.shape[1]):
            s += '%s,%s,' % (fmt_g(pred_res[n, ts, 0]), fmt_g(pred_res[n, ts, 1]))
        rows.append(s + '%s\n' % fmt_g(ess[n]))
    return rows


def write_done(args, best, x=None):
    """plom_print_done (print.c:33-67): theta with the guesses of the vector."""
    theta = best.theta_with(x)
    if args.pipe:
        sys.stdout.write(json.dumps(theta))
        sys.stdout.flush()
    else:
        with open('%s.done_%d.json' % (args.path, args.id), 'w') as f:
            json.dump(theta, f)


def unlink_done(args):
    try:
        os.unlink('%s.done_%d.json' % (args.path, args.id))
    except OSError:
        pass


def duration_line(seconds):
    """time_exec (model_builder/C/core/utils.c) as printed by the drivers."""
    d = int(seconds // 86400)
    seconds -= d * 86400
    h = int(seconds // 3600)
    seconds -= h * 3600
    m = int(seconds // 60)
    seconds -= m * 60
    return 'Done in:= %dd %dh %dm %gs' % (d, h, m, seconds)


# ---------------------------------------------------------------- smc
SMC_HELP = """PLOM Sequential Monte Carlo (B200 engine)
usage:
smc [implementation] [--no_dem_sto] [--no_white_noise] [--no_diff]
                     [-r, --traj] [-p, --path <path>] [-i, --id <integer>] [-N, --n_thread <integer>]
                     [-g, --freeze_forcing <float>]
                     [-t, --no_filter] [-b, --no_trace] [-e, --no_hat]
                     [-s, --DT <float>] [--eps_abs <float>] [--eps_rel <float>]
                     [-l, --LIKE_MIN <float>] [-J <integer>] [--prior]
                     [-q, --quiet] [-P, --pipe]                     [-h, --help]
                     [--precision 32|64] [--seed <integer>]
where implementation is 'ode', 'sde' or 'psr' (default)
"""


def smc_parser():
    ap = common_parser('smc', 'PLOM Sequential Monte Carlo')
    ap.add_argument('-r', '--traj', action='store_true')
    ap.add_argument('-t', '--no_filter', action='store_true')
    ap.add_argument('-b', '--no_trace', action='store_true')
    ap.add_argument('-e', '--no_hat', action='store_true')
    ap.add_argument('-d', '--no_pred_res', action='store_true')
    return ap


def smc_main(argv, stdin=None, model_dir='.'):
    from .native import Engine
    args = smc_parser().parse_args(argv)
    if args.help:
        print(SMC_HELP)
        return 1
    if args.pipe:
        args.quiet = True
    unlink_done(args)
    model, settings, lib = load_model_dir(model_dir)
    theta = read_theta(stdin)
    filt = not args.no_filter
    problem = make_problem(model, settings, theta, args, filter=filt)
    best = Best(model, theta)
    want_hat = not args.no_hat
    want_pred = not args.no_pred_res
    drift_on = not (problem.noises_off & NO_DRIFT)
    f_hat = f_pred = f_x = None
    if want_hat:
        f_hat = open(path_of(args, 'hat'), 'w')
        f_hat.write(header_hat(model, problem, drift_on))
    if want_pred:
        f_pred = open(path_of(args, 'pred_res'), 'w')
        f_pred.write(header_pred_res(model))
    if args.traj:
        f_x = open(path_of(args, 'X'), 'w')
        f_x.write(header_x(model, problem))
    log(args, 'Starting plom-smc with the following options: i = %d, J = %d, LIKE_MIN = %s, n_threads = %d'
        % (args.id, args.J, fmt_g(args.LIKE_MIN), args.n_thread))
    t0 = time.time()
    eng = Engine(model_name(lib), lib)
    out = eng.smc(problem, hat=want_hat or want_pred, ancestors=args.traj, x_pred=args.traj)
    loglik = out.loglik
    if args.prior:
        lp, _ = best.log_prob_prior(like_min=args.LIKE_MIN)
        loglik += lp
    if f_hat:
        f_hat.writelines(hat_rows(model, problem, out.hat, drift_on))
        f_hat.close()
    if f_pred:
        f_pred.writelines(pred_res_rows(problem, out.pred_res, out.ess_n))
        f_pred.close()
    if f_x:
        f_x.writelines(x_rows(eng, model, problem, out))
        f_x.close()
    if filt:
        log(args, 'logV: %s, J: %d,  n_all_fail: %d' % (fmt_g(loglik), args.J, out.n_all_fail))
    log(args, duration_line(time.time() - t0))
    if not args.no_trace:
        with open(path_of(args, 'trace'), 'w') as f:
            f.write(best.trace_header())
            f.write(best.trace_row(0, loglik))
    write_done(args, best)
    log(args, 'clean up...')
    return 0


def model_name(lib):
    b = os.path.basename(lib)
    if b.startswith('libplomgpu_') and b.endswith('.so'):
        return b[len('libplomgpu_'):-3]
    return b


# ---------------------------------------------------------------- X (trajectories of every particle)
def header_x(model, problem):
    """header_X (print.c:88-129)."""
    s = 'index,time,'
    for name in model.par_sv:
        for cac in model.cac_id:
            s += '%s:%s,' % (name, cac)
    if model.remainder is not None:
        for cac in model.cac_id:
            s += '%s:%s,' % (model.remainder, cac)
    for t in model.ts_id:
        s += 'obs_mean:%s,' % t
    if not (problem.noises_off & NO_DRIFT):
        for name, groups in drift_groups(model, problem):
            for g in groups:
                s += 'drift:%s:%s,' % (name, g)
    s += ','.join('obs_real:%s' % t for t in model.ts_id)
    return s + '\n'


def x_rows(eng, model, problem, out):
    """print_X at time 0 and after each interval (print.c:301-393): every
    resampled particle.  The per-particle columns are evaluated on the GPU
    (plomgpu_particle_values) from the particle history (propagated states and
    ancestors); the observation draws max(0, mean + sd * N(0, 1)) of
    ``observation`` (core_template.c:392-407) use a Philox stream seeded from
    the run's seed."""
    rng = np.random.Generator(np.random.Philox(problem.seed))
    info = eng.info
    nc = info.n_cac
    nsv = info.n_par_sv * nc
    nrem = 0 if info.pop_size_eq_sum_sv else nc
    nts = info.n_ts
    drift = [] if (problem.noises_off & NO_DRIFT) else drift_groups(model, problem)
    rows = []
    J = problem.J
    x0 = np.repeat(problem.x0[:, None], J, axis=1)
    x0[info.off_inc:] = 0.0
    snaps = [(0, 0.0, x0)]
    for n in range(problem.n_obs):
        x = out.x_pred[n]
        if out.ancestors is not None:
            x = x[:, out.ancestors[n]]
        snaps.append((n + 1, problem.t_obs[n], x))
    for row, t, x in snaps:
        v = eng.particle_values(problem, x, row)
        mean = v[nsv + nrem:nsv + nrem + nts]
        var = v[info.n_hat:info.n_hat + nts]
        with np.errstate(invalid='ignore'):
            y = mean + np.sqrt(var) * rng.standard_normal(mean.shape)
        y = np.where(y > 0.0, y, 0.0)
        base = nsv + nrem + nts
        for j in range(J):
            s = '%d,%s,' % (j, fmt_g(t))
            s += ''.join('%s,' % fmt_g(v[q, j]) for q in range(nsv + nrem + nts))
            for i, (_, groups) in enumerate(drift):
                s += ''.join('%s,' % fmt_g(v[base + i * nc + g, j]) for g in range(len(groups)))
            s += ','.join(fmt_g(y[ts, j]) for ts in range(nts))
            rows.append(s + '\n')
    return rows


# ---------------------------------------------------------------- pmbuilder
def pmbuilder_main(argv):
    from .build import build_model_dir
    ap = argparse.ArgumentParser(prog='pmbuilder', description='pmbuilder: build a model for json files')
    ap.add_argument('context_file')
    ap.add_argument('process_file')
    ap.add_argument('link_file')
    ap.add_argument('-o', '--output', default='model')
    a = ap.parse_args(argv)
    files = []
    for p in (a.context_file, a.process_file, a.link_file):
        try:
            with open(p) as f:
                files.append(json.load(f))
        except IOError:
            sys.stderr.write('FAILURE! %s could not be found\n' % os.path.abspath(p))
            return 1
        except ValueError:
            sys.stderr.write('FAILURE! %s could not be parsed. Go check your JSON!\n' % os.path.abspath(p))
            return 1
    out = os.path.abspath(a.output)
    print('preparing model...')
    print('coding model...')
    build_model_dir(files[0], files[1], files[2], out)
    print('writting settings...')
    print('SUCCESS: model created in %s' % out)
    return 0


def main(argv=None):
    argv = list(sys.argv[1:] if argv is None else argv)
    if not argv:
        sys.stderr.write('usage: python -m plomgpu {pmbuilder,smc,pmcmc,mif} ...\n')
        return 2
    cmd, rest = argv[0], argv[1:]
    try:
        if cmd == 'smc':
            return smc_main(rest)
        if cmd == 'pmbuilder':
            return pmbuilder_main(rest)
        if cmd in ('pmcmc', 'mif'):
            from . import drivers
            return drivers.main(cmd, rest)
    except CliError as e:
        sys.stderr.write('%s\n' % e)
        return 1
    except Exception as e:  # engine errors end the run as print_err + exit(EXIT_FAILURE) do
        from .native import PlomGpuError
        if not isinstance(e, PlomGpuError):
            raise
        sys.stderr.write('%s\n' % e)
        return 1
    sys.stderr.write('unknown command %r\n' % cmd)
    return 2
