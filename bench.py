"""Benchmark: particle-steps/s of the SMC filter on the SEIR 20x2 workload.

One step = one complete particle filter over the workload (J particles, T
observation intervals of K Euler substeps, weighting, log-sum-exp
normalisation, systematic resampling and log-likelihood accumulation at every
interval).  ``value`` is measured with the inputs resident in HBM (a captured
plan replayed), ``e2e`` through the one-shot C-ABI call plomgpu_smc_run with
host buffers (upload of every input, run, download of the results).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference] [--workload seir20x2|sir]

With torchrun (N > 1) every rank runs an independent filter (replicas, no
collective in the data path); time is the max over ranks.
"""

import argparse
import copy
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, 'iterated-inference-pipeline_b200'))

WORKLOADS = {
    # name: (model library, J, observation intervals, dt in days)
    'seir20x2': ('seir20x2', 100000, 520, 1.0),
    # the same filter with the reference's default implementation (Poisson system with stochastic rates)
    'seir20x2_psr': ('seir20x2', 100000, 520, 1.0),
    # the same filter without demographic noise (--no_dem_sto: environmental noise only)
    'seir20x2_nodem': ('seir20x2', 100000, 520, 1.0),
    # the deterministic Euler skeleton of the same filter (--no_dem_sto --no_white_noise)
    'seir20x2_skel': ('seir20x2', 100000, 520, 1.0),
    'sir': ('sir', 1000, 52, 1.0),
    # the SIR filter's Euler skeleton with 2^24 particles (4 state words: the HBM-bound case)
    'sir_skel_large': ('sir', 1 << 24, 52, 1.0),
    # 4096 SIR parameter sets, J in 256..16384, T in 52..520 weeks, one persistent launch
    'sir_batch': ('sir', None, None, 1.0),
    # 64 iterated-filtering runs of the SEIR 20x2 model, J = 20000 each (per-iteration timing)
    'mif_seir': ('seir20x2', 20000, 520, 1.0),
    # 32 pMCMC chains (16 SIR J=2000, 16 SEIR 20x2 J=20000), Poisson arrivals at 2000 req/s
    'serve': (None, None, None, 1.0),
}
METRIC = 'particle-steps/s at matched loglik error'
# noises_off of the workloads that turn noise terms off (bit 0: demographic, bit 1: environmental)
NOISES_OFF = {'seir20x2_nodem': 1, 'seir20x2_skel': 3, 'sir_skel_large': 3}
NOISE_TEXT = {0: 'sde full (demographic + environmental)', 1: 'sde without demographic noise (--no_dem_sto)',
              3: 'Euler skeleton (--no_dem_sto --no_white_noise)'}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=5)
    ap.add_argument('--warmup', type=int, default=3)
    ap.add_argument('--impl', default='ours', choices=['ours', 'reference'])
    ap.add_argument('--workload', default='seir20x2', choices=sorted(WORKLOADS))
    ap.add_argument('--no-cpu-baseline', action='store_true')
    ap.add_argument('--e2e-runs', type=int, default=3, help='one-shot C-ABI calls timed for e2e (0: skip)')
    ap.add_argument('--error-samples', type=int, default=26,
                    help='intervals sampled for loglik_error (0: skip)')
    ap.add_argument('--serve-load', type=float, default=0.6,
                    help='serve: offered load, as a fraction of the measured saturation rate, of the latency runs')
    ap.add_argument('--plan-pool', type=int, default=0, help='serve: run the shared-memory model on a pool of this '
                    'many concurrent plans instead of the tiled device loop (0: device loop)')
    ap.add_argument('--particles', type=int, default=0,
                    help='a smaller case of the workload for profiling captures: J (0: the workload\'s)')
    ap.add_argument('--intervals', type=int, default=0,
                    help='a smaller case of the workload for profiling captures: T (0: the workload\'s)')
    return ap.parse_args()


def workload_problem(name, precision=32, seed=0, J=None, nb_obs=-1):
    from plomgpu import workloads, model, problem
    lib, J0, T, dt = WORKLOADS[name]
    c, p, l, th = workloads.load(lib)
    m = model.PlomModel(c, p, l)
    return problem.Problem(m, m.settings(), th, J=J or J0, dt=dt, precision=precision, seed=seed, nb_obs=nb_obs,
                           psr=name.endswith('_psr'), noises_off=NOISES_OFF.get(name, 0))


def state_words(prob):
    m = prob.model
    return len(m.par_sv) * m.N_CAC + len(m.drift_par_proc) * m.N_CAC + m.N_TS_INC_UNIQUE


def bytes_per_particle_step(prob, b_state):
    # algorithmic bytes: state read + write, log-weight write + read, ancestor write + read
    return 2 * state_words(prob) * b_state + 2 * 4 + 2 * 4


class Clocks(object):
    """Samples SM clocks and throttle reasons with nvidia-smi during the timed region."""

    FIELDS = ('index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,'
              'clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,'
              'clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap')

    def __init__(self, device_index):
        self.dev = device_index
        self.proc = None
        self.out = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ['nvidia-smi', '-i', str(self.dev), '--query-gpu=' + self.FIELDS, '--format=csv,noheader,nounits',
                 '-lms', '100'], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, ValueError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.out.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.t.join(timeout=2)

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ['hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap']
        for line in self.out:
            f = [x.strip() for x in line.split(',')]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for k, nm in enumerate(names):
                if f[5 + k].lower().startswith('active'):
                    reasons.add(nm)
        if not sm:
            return {'sm_mhz': None, 'sm_max_mhz': None, 'reasons': ['unsampled'], 'samples': 0}
        return {'sm_mhz': statistics.median(sm), 'sm_max_mhz': max(mx), 'reasons': sorted(reasons),
                'samples': len(sm)}


def measured_peak_hbm():
    path = os.path.join(ROOT, 'MEASURED_PEAKS.json')
    try:
        with open(path) as f:
            return float(json.load(f)['hbm_gbs']), 'measured'
    except (OSError, KeyError, ValueError):
        return 6650.0, 'fallback'


def ncu_traffic(workload):
    """Per-launch DRAM bytes of the propagate kernel from the committed ncu summary, scaled to J, and
    where they come from (the summary file and the date of its capture)."""
    path = os.path.join(ROOT, 'profiles', 'k_propagate_%s.json' % workload)
    try:
        with open(path) as f:
            d = json.load(f)
        src = 'profiles/k_propagate_%s.json (ncu capture of %s, not this run)' % (workload, d.get('captured', '?'))
        return float(d['dram_bytes_per_particle']) * WORKLOADS[workload][1], src
    except (OSError, KeyError, ValueError):
        return None, None


def loglik_error(eng, prob, samples):
    """Precision error of the production arithmetic at the workload's size, one interval at a time:
    the same FP64 particle cloud advanced over one interval by the FP32 and the FP64 filter with paired
    draws (the FP32 filter consumes the FP64 filter's normals and resampling uniforms), at ``samples``
    intervals spread over an FP64 filter path (plomgpu.precision)."""
    from plomgpu import precision
    if prob.psr or samples <= 0:
        return None
    p = copy.copy(prob)
    stride = max(1, p.n_obs // samples)
    n, d = precision.conditional_interval_errors(eng, p, stride=stride, seed=7000)
    out = precision.summary(p, n, d)
    out['method'] = ('conditional per interval: the same FP64 cloud advanced one interval in FP32 state / FP64 '
                     'reductions and in FP64 everywhere with the same normals and uniforms, every %d-th interval '
                     'of an FP64 filter path at the benchmark size; implied_filter_bias = T x the per-interval '
                     'mean' % stride)
    return out


def max_over_ranks(x, dist, device):
    """The slowest rank's time (every rank runs an independent replica)."""
    import torch
    t = torch.tensor([float(x)], device=device, dtype=torch.float64)
    if dist is not None:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(psteps_per_rank, world, ms_step):
    """Whole-job particle-steps/s: every rank advances its own filter of psteps_per_rank
    particle-steps in a step that lasts the slowest rank's ms_step (weak scaling)."""
    return psteps_per_rank * world / (ms_step / 1000.0)


def ncu_issue(workload, J=None, avg_launch_ms=None, sm_mhz=None):
    """Issue-side utilisation of the propagate kernel from the committed ncu summary (the bound that
    binds: the full-noise step is instruction-issue bound, not HBM bound), and its issue roofline for
    this run: the captured warp instructions per particle x J over 148 SMs x 4 schedulers x the SM
    clock (one warp instruction per scheduler per cycle), against the measured launch time."""
    path = os.path.join(ROOT, 'profiles', 'k_propagate_%s.json' % workload)
    try:
        with open(path) as f:
            d = json.load(f)
        out = {'issue_slots_active_pct': d['issue_active_pct'], 'ipc': d['ipc'],
               'warps_active_per_sm': d['warps_active_per_sm'],
               'source': '%s (ncu capture of %s, not this run)' % (
                   d.get('summary', 'profiles/k_propagate_%s.md' % workload), d.get('captured', '?'))}
        if J and avg_launch_ms and 'warp_instructions_per_particle' in d:
            clock = (sm_mhz or 1965.0) * 1e6
            floor_ms = d['warp_instructions_per_particle'] * J / (148 * 4 * clock) * 1e3
            out.update({'floor_ms': floor_ms, 'frac': floor_ms / avg_launch_ms,
                        'floor': 'warp instructions / (148 SMs x 4 schedulers x SM clock)'})
        return out
    except (OSError, KeyError, ValueError):
        return None


def cpu_baseline(workload, budget_s=12.0, threads=0):
    """Times the FP64 oracle (OpenMP, all host threads) on a bounded sample of the workload."""
    sys.path.insert(0, os.path.join(ROOT, 'oracle'))
    from oracle import Oracle
    lib = WORKLOADS[workload][0]
    orc = Oracle(lib)
    J0 = WORKLOADS[workload][1]
    J = min(J0, 20000)
    n = 1
    while True:
        p = workload_problem(workload, precision=64, seed=3, J=J, nb_obs=n)
        t = time.perf_counter()
        orc.smc(p, n_threads=threads)
        el = time.perf_counter() - t
        if el > budget_s / 4 or n >= WORKLOADS[workload][2]:
            break
        n = min(WORKLOADS[workload][2], max(n + 1, int(n * (budget_s / 3) / max(el, 1e-3))))
    cores = threads if threads > 0 else (os.cpu_count() or 1)
    return {'value': p.J * p.n_obs / el, 'unit': 'particle-steps/s', 'cores': cores, 'kind': 'port',
            'sample': '%s: J=%d particles x %d observation intervals (%d Euler substeps each), FP64 oracle, %.2f s'
                      % (workload, p.J, p.n_obs, int(p.n_sub[0]), el)}


def run_reference(args):
    rank = int(os.environ.get('RANK', '0'))
    if rank != 0:
        return 0
    base = cpu_baseline(args.workload, budget_s=8.0)
    vals = []
    for _ in range(args.warmup):
        pass
    lib, J0, T, dt = WORKLOADS[args.workload]
    sys.path.insert(0, os.path.join(ROOT, 'oracle'))
    from oracle import Oracle
    orc = Oracle(lib)
    J = min(J0, 20000)
    n = max(1, min(T, int(round(base['value'] * 4.0 / J))))
    p = workload_problem(args.workload, precision=64, seed=4, J=J, nb_obs=n)
    for _ in range(max(args.warmup, 1)):
        orc.smc(p)
    for _ in range(args.steps):
        t = time.perf_counter()
        orc.smc(p)
        vals.append(time.perf_counter() - t)
    ms = 1000.0 * statistics.mean(vals)
    v = p.J * p.n_obs / (ms / 1000.0)
    base['value'] = v
    base['sample'] = '%s: J=%d x %d intervals per step, FP64 oracle (reference CPU path restated), all host threads' % (
        args.workload, p.J, p.n_obs)
    line = {'impl': 'reference', 'metric': METRIC, 'value': v, 'unit': 'particle-steps/s', 'n_gpus': args.gpus,
            'steps': args.steps, 'warmup': args.warmup, 'ms_per_step': ms, 'higher_is_better': True,
            'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f64', 'data': 'synthetic',
            'config': {'workload': args.workload, 'J': WORKLOADS[args.workload][1],
                       'T': WORKLOADS[args.workload][2], 'sample_J': p.J, 'sample_T': p.n_obs},
            'cpu_baseline': base,
            'e2e': {'value': v, 'unit': 'particle-steps/s', 'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 0}}
    print(json.dumps(line))
    return 0


def run_batch(args):
    """Batched filters (4096 SIR parameter sets) beside the plain single-filter path."""
    import numpy as np
    import torch
    from plomgpu import workloads
    from plomgpu.native import Engine, Batch, Plan
    torch.cuda.set_device(int(os.environ.get('LOCAL_RANK', '0')))
    eng = Engine('sir')
    bp = workloads.sir_batch(n_sets=4096, seed=2)
    b = Batch(eng, bp, precision=32)
    stream = torch.cuda.ExternalStream(b.stream)
    for _ in range(args.warmup):
        b.launch()
    torch.cuda.synchronize()
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    with Clocks(int(os.environ.get('LOCAL_RANK', '0'))) as clk:
        start.record(stream)
        for _ in range(args.steps):
            b.launch()
        end.record(stream)
        torch.cuda.synchronize()
    ms = start.elapsed_time(end) / args.steps
    ll, nf, ess = b.results()
    bt, ppt, grid = b.config
    b.close()
    value = bp.particle_steps / (ms / 1000.0)
    # plain single-filter path on the config-0 filter (J = 1000, T = 52), graph replay
    single = workload_problem('sir', precision=32, seed=5)
    plan = Plan(eng, single)
    s2 = torch.cuda.ExternalStream(plan.stream)
    for _ in range(5):
        plan.launch()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    reps = 50
    e0.record(s2)
    for _ in range(reps):
        plan.launch()
    e1.record(s2)
    torch.cuda.synchronize()
    ms_single = e0.elapsed_time(e1) / reps
    plan.close()
    single_value = single.J * single.n_obs / (ms_single / 1000.0)
    # log-likelihood error of the FP32 arithmetic against the FP64 path on every 16th
    # set (256 sets), with paired draws (the FP32 filter consumes the FP64 filter's
    # normals and resampling uniforms): the difference is due to precision alone
    sample = list(range(0, 4096, 16))
    errs = []
    for i in sample:
        p = bp.single(i)
        p.paired_draws = True
        errs.append(eng.smc(p, precision=32).loglik - eng.smc(p, precision=64).loglik)
    line = {'metric': METRIC, 'value': value, 'unit': 'particle-steps/s', 'n_gpus': 1, 'steps': args.steps,
            'warmup': args.warmup, 'ms_per_step': ms, 'higher_is_better': True, 'scaling': 'weak',
            'vs_baseline': None, 'dtype': 'f32 state / f64 reductions', 'data': 'synthetic',
            'config': {'workload': 'sir_batch', 'filters': 4096, 'particle_steps': bp.particle_steps,
                       'J_range': [256, 16384], 'T_range': [52, 520], 'block_threads': bt,
                       'particles_per_thread': ppt, 'grid': grid, 'tuned_by': 'plomgpu batch autotuner'},
            'plain_single_filter': {'value': single_value, 'ms_per_filter': ms_single, 'J': single.J,
                                    'T': single.n_obs},
            'batched_over_plain': value / single_value,
            'loglik_error': {
                'fp32_minus_fp64_mean': float(np.mean(errs)), 'se': float(np.std(errs, ddof=1) / math.sqrt(len(errs))),
                'mean_abs': float(np.mean(np.abs(errs))), 'max_abs': float(np.max(np.abs(errs))),
                'filters': len(sample), 'unit': 'nats per filter', 'gate': 0.5,
                'method': 'paired draws, plain one-shot filters of every 16th set (the batched kernel equals '
                          'them per filter: tests/test_gpu_batch.py)'},
            'clocks': clk.summary(), 'gpu_launches': args.steps}
    print(json.dumps(line))
    return 0


def run_mif(args):
    """64 MIF runs on SEIR 20x2 (J = 20000 each), iterations batched in-device.

    The per-particle random walk has sd 0.02 on the log scale at the first
    iteration and cools by 0.95 per iteration: with the reference's
    FREEZE * sqrt(delta_t) * sd_transf / sqrt(nb_obs) (delta_t = 7 days,
    nb_obs = 520) that is sd_transf = 0.02 * sqrt(520 / 7), a = 0.95.
    """
    import numpy as np
    import torch
    from plomgpu import mif
    from plomgpu.native import Engine
    torch.cuda.set_device(int(os.environ.get('LOCAL_RANK', '0')))
    eng = Engine('seir20x2')
    prob = workload_problem('mif_seir', precision=32, seed=11)
    sd = 0.02 * math.sqrt(520.0 / 7.0)
    names = ['r0', 'v', 'eps', 'sto', 'rep', 'phi']
    run = mif.Mif(eng, prob, n_runs=64, names=names, sd_transf=dict((n, sd) for n in names), a=0.95, b=2.0)
    rng = np.random.Generator(np.random.Philox(3))
    run.theta_hat = run.theta_hat + 0.1 * rng.standard_normal(run.theta_hat.shape)
    for m in range(1, args.warmup + 1):
        run.run(1, seed=m)
    times = []
    with Clocks(int(os.environ.get('LOCAL_RANK', '0'))) as clk:
        for k in range(args.steps):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            tr = run.run(1, seed=100 + k)
            times.append(time.perf_counter() - t0)
    run.close()
    it_s = statistics.median(times)
    psteps = 64 * prob.J * prob.n_obs
    line = {'metric': METRIC, 'value': psteps / it_s, 'unit': 'particle-steps/s', 'n_gpus': 1,
            'steps': args.steps, 'warmup': args.warmup, 'ms_per_step': 1000.0 * it_s, 'higher_is_better': True,
            'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f32 state / f64 reductions', 'data': 'synthetic',
            'config': {'workload': 'mif_seir', 'runs': 64, 'J': prob.J, 'T': prob.n_obs, 'step': 'one MIF iteration of all runs',
                       'theta_components': names, 'rw_sd_first_iteration': 0.02, 'cooling': 0.95,
                       'time_for_100_iterations_s': 100 * it_s},
            'loglik_mean_over_runs': float(np.mean(tr[-1]['loglik'])), 'clocks': clk.summary()}
    print(json.dumps(line))
    return 0


def serve_class_profile(c, rng, load):
    """One request class on its server alone: the saturation rate (a backlog of requests submitted at
    once, completed per second) and the p50 / p99 latency of Poisson arrivals at ``load`` x that rate."""
    import numpy as np
    sv, J, p = c['server'], c['J'], c['prob']
    n_sat = 64 if J > 5000 else 512
    t0 = time.perf_counter()
    ts = [sv.submit(J, par_cac=p.par_cac * np.exp(0.02 * rng.standard_normal(p.par_cac.shape)), seed=50000 + i)
          for i in range(n_sat)]
    for t in ts:
        sv.wait(t, 600.0)
    sat = n_sat / (time.perf_counter() - t0)
    rate = load * sat
    n_req = 48 if J > 5000 else 400
    arrivals = np.cumsum(rng.exponential(1.0 / rate, size=n_req))
    pending, lat = [], []
    start = time.perf_counter()
    k = 0
    while k < n_req or pending:
        now = time.perf_counter() - start
        if k < n_req and now >= arrivals[k]:
            pending.append(sv.submit(J, seed=60000 + k))
            k += 1
            continue
        for t in list(pending):
            r = sv.poll(t)
            if r is not None:
                lat.append(r[2])
                pending.remove(t)
        time.sleep(1e-4)
    pct = lambda q: float(np.percentile(lat, q))
    return {'saturation_requests_per_s': sat, 'saturation_particle_steps_per_s': sat * J * p.n_obs,
            'load': load, 'offered_requests_per_s': rate, 'requests': n_req,
            'latency_s': {'p50': pct(50), 'p99': pct(99)}}


def run_serve(args, window_s=0.25, rate=2000.0):
    """Served pMCMC likelihoods: asynchronous random-walk chains submit requests as
    Poisson arrivals; results feed Metropolis-Hastings accept / reject."""
    import numpy as np
    import torch
    from plomgpu.native import Engine, Server
    torch.cuda.set_device(int(os.environ.get('LOCAL_RANK', '0')))
    classes = {
        'sir': {'lib': 'sir', 'J': 2000, 'prob': workload_problem('sir', precision=32, seed=1, J=2000)},
        'seir': {'lib': 'seir20x2', 'J': 20000, 'prob': workload_problem('seir20x2', precision=32, seed=1, J=20000)},
    }
    for c in classes.values():
        c['eng'] = Engine(c['lib'])
        c['server'] = Server(c['eng'], c['prob'], max_J=c['J'], memory_budget=150e9 / 2, plan_pool=args.plan_pool,
                             precision=32, use_plan_pool=args.plan_pool > 0)
    rng = np.random.Generator(np.random.Philox(12))
    chains = []
    for i in range(32):
        cl = 'sir' if i < 16 else 'seir'
        p = classes[cl]['prob']
        chains.append({'cls': cl, 'theta': p.par_cac.copy(), 'll': -np.inf, 'accepted': 0, 'done': 0})
    # warm up both servers (kernels, plans)
    for c in classes.values():
        c['server'].wait(c['server'].submit(c['J'], seed=1))
    gaps = rng.exponential(1.0 / rate, size=int(rate * window_s * 3))
    arrivals = np.cumsum(gaps)
    arrivals = arrivals[arrivals < window_s]
    owners = rng.integers(0, 32, size=len(arrivals))
    outstanding = {}
    lat = {'sir': [], 'seir': []}
    t_start = time.perf_counter()
    k = 0

    def harvest(block=False):
        for key in list(outstanding):
            cl, tk = key
            ch, _, th = outstanding[key]
            r = classes[cl]['server'].poll(tk) if not block else classes[cl]['server'].wait(tk, 600.0)
            if r is None:
                continue
            ll, nf, latency = r
            lat[cl].append(latency)
            c = chains[ch]
            c['done'] += 1
            if np.log(rng.uniform()) < ll - c['ll']:
                c['theta'], c['ll'] = th, ll
                c['accepted'] += 1
            del outstanding[key]

    with Clocks(int(os.environ.get('LOCAL_RANK', '0'))) as clk:
        while k < len(arrivals):
            now = time.perf_counter() - t_start
            if now >= arrivals[k]:
                ch = int(owners[k])
                c = chains[ch]
                th = c['theta'] * np.exp(0.02 * rng.standard_normal(c['theta'].shape))
                sv = classes[c['cls']]['server']
                tk = sv.submit(classes[c['cls']]['J'], par_cac=th, seed=int(1 + k))
                # tickets are numbered per server: key them by class too
                outstanding[(c['cls'], tk)] = (ch, c['cls'], th)
                k += 1
            else:
                harvest()
                time.sleep(min(2e-4, max(0.0, arrivals[k] - now)))
        harvest(block=True)
    t_total = time.perf_counter() - t_start
    stats = dict((cl, c['server'].stats()) for cl, c in classes.items())
    n_req = sum(len(v) for v in lat.values())
    per_class = dict((cl, serve_class_profile(c, rng, args.serve_load)) for cl, c in classes.items())
    psteps = sum(len(lat[cl]) * classes[cl]['J'] * classes[cl]['prob'].n_obs for cl in lat)
    # plain filter per request: one-shot plomgpu_smc_run, sequential, on a sample
    plain = {}
    for cl, c in classes.items():
        ts = []
        for i in range(3 if cl == 'sir' else 2):
            p = c['prob']
            t0 = time.perf_counter()
            c['eng'].smc(p)
            ts.append(time.perf_counter() - t0)
        plain[cl] = statistics.median(ts)
    plain_time = sum(len(lat[cl]) * plain[cl] for cl in lat)
    for c in classes.values():
        c['server'].close()
    pct = lambda v, q: float(np.percentile(v, q)) if v else None
    line = {'metric': METRIC, 'value': psteps / t_total, 'unit': 'particle-steps/s', 'n_gpus': 1, 'steps': 1,
            'warmup': 1, 'ms_per_step': 1000.0 * t_total, 'higher_is_better': True, 'scaling': 'weak',
            'vs_baseline': None, 'dtype': 'f32 state / f64 reductions', 'data': 'synthetic',
            'config': {'workload': 'serve', 'chains': {'sir_J2000_T52': 16, 'seir20x2_J20000_T520': 16},
                       'arrival_rate_per_s': rate, 'arrival_window_s': window_s, 'requests': n_req,
                       'memory_budget_GB': 150},
            'requests_per_s': n_req / t_total,
            'latency_s': dict((cl, {'p50': pct(lat[cl], 50), 'p99': pct(lat[cl], 99), 'n': len(lat[cl])}) for cl in lat),
            'plain_filter_per_request': {'latency_s': plain, 'total_s_for_same_requests': plain_time,
                                         'speedup_of_serving': plain_time / t_total},
            'per_class_alone': per_class,
            'server_stats': stats, 'acceptance': [c['accepted'] / max(c['done'], 1) for c in chains],
            'clocks': clk.summary()}
    print(json.dumps(line))
    return 0


def main():
    args = parse()
    if args.workload == 'serve':
        return run_serve(args)
    if args.impl == 'reference':
        return run_reference(args)
    if args.workload == 'sir_batch':
        return run_batch(args)
    if args.workload == 'mif_seir':
        return run_mif(args)
    import numpy as np
    import torch
    world = int(os.environ.get('WORLD_SIZE', '1'))
    rank = int(os.environ.get('RANK', '0'))
    local = int(os.environ.get('LOCAL_RANK', '0'))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group('nccl', timeout=datetime.timedelta(seconds=120))
    from plomgpu.native import Engine, Plan
    from plomgpu import build
    lib = WORKLOADS[args.workload][0]
    eng = Engine(lib)
    prob = workload_problem(args.workload, precision=32, seed=1000 + rank, J=args.particles or None,
                            nb_obs=args.intervals or -1)
    # the timed plan carries no events between its kernels (they would break the chained launches of
    # an interval); a second plan with an event around every propagate launch measures that kernel
    plan = Plan(eng, prob)
    stream = torch.cuda.ExternalStream(plan.stream)

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()

    for _ in range(args.warmup):
        plan.launch()
    barrier()
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    prop_ms = []
    with Clocks(local) as clk:
        start.record(stream)
        for _ in range(args.steps):
            plan.launch()
        end.record(stream)
        torch.cuda.synchronize()
    ms_total = start.elapsed_time(end)
    tplan = Plan(eng, prob, timing=True)
    for _ in range(2):
        tplan.launch()
    torch.cuda.synchronize()
    tot_prop, n_prop = tplan.propagate_time()
    tplan.close()
    res = plan.results()
    ms_step = ms_total / args.steps
    ms_step = max_over_ranks(ms_step, dist, 'cuda')
    psteps = prob.J * prob.n_obs
    value = replica_throughput(psteps, world, ms_step)
    kernels_per_step = plan.kernel_count
    plan.close()

    # end to end through the one-shot C ABI call with host buffers
    from plomgpu.native import DescHolder
    e2e_times = []
    for i in range(args.e2e_runs):
        barrier()
        t0 = time.perf_counter()
        out = eng.smc(prob)
        e2e_times.append(time.perf_counter() - t0)
    h = DescHolder(prob)
    h2d = sum(a.nbytes for a in h.arrays.values())
    d2h = 8 * 2 * prob.n_obs + 16
    e2e_s = statistics.median(e2e_times) if e2e_times else float('nan')
    e2e_max = max_over_ranks(e2e_s, dist, 'cuda')
    e2e_value = psteps * world / e2e_max if e2e_times else None

    if rank == 0:
        peak, peak_kind = measured_peak_hbm()
        B = bytes_per_particle_step(prob, 4)
        avg_prop_ms = tot_prop / max(n_prop, 1)
        achieved = B * prob.J / (avg_prop_ms / 1000.0) / 1e9
        traffic, traffic_src = ncu_traffic(args.workload)
        err = loglik_error(eng, prob, args.error_samples)
        line = {
            'metric': METRIC, 'value': value, 'unit': 'particle-steps/s', 'n_gpus': world, 'steps': args.steps,
            'warmup': args.warmup, 'ms_per_step': ms_step, 'higher_is_better': True, 'scaling': 'weak',
            'vs_baseline': None, 'dtype': 'f32 state / f64 reductions', 'data': 'synthetic',
            'config': {'workload': args.workload, 'J': prob.J, 'T': prob.n_obs, 'K': int(prob.n_sub[0]),
                       'state_words': state_words(prob),
                       'noise': ('psr (multinomial + Poisson + Gamma white noise)' if prob.psr else
                                 NOISE_TEXT[prob.noises_off]),
                       'parallelism': 'replicas' if world > 1 else 'single GPU',
                       'l2': 'inputs larger than L2 (two state generations of %.0f MB)' %
                             (2 * state_words(prob) * 4 * prob.J / 1e6)},
            'loglik': res.loglik,
            'loglik_error': err,
            'euler_substeps_per_s': value * float(np.mean(prob.n_sub)),
            'gpu_launches': kernels_per_step * args.steps,
            'roofline': {'bound': 'hbm', 'achieved': achieved, 'peak': peak, 'unit': 'GB/s',
                         'frac': achieved / peak, 'traffic': traffic, 'traffic_source': traffic_src,
                         'step_achieved': B * prob.J * prob.n_obs / (ms_step / 1000.0) / 1e9,
                         'step_frac': B * prob.J * prob.n_obs / (ms_step / 1000.0) / 1e9 / peak,
                         'kernel': 'k_propagate', 'bytes_per_particle_step': B,
                         'avg_launch_ms': avg_prop_ms, 'peak_kind': peak_kind,
                         'propagate_share': tot_prop / (ms_total / args.steps),
                         'issue': ncu_issue(args.workload, prob.J, avg_prop_ms, clk.summary()['sm_mhz'])},
            'clocks': clk.summary(),
            'e2e': {'value': e2e_value, 'unit': 'particle-steps/s', 'h2d_bytes_per_step': h2d,
                    'd2h_bytes_per_step': d2h, 'call': 'plomgpu_smc_run (host buffers, one-shot)'},
        }
        if world == 1 and not args.no_cpu_baseline:
            line['cpu_baseline'] = cpu_baseline(args.workload)
        print(json.dumps(line))
    if dist is not None:
        dist.destroy_process_group()
    return 0


if __name__ == '__main__':
    sys.exit(main())
