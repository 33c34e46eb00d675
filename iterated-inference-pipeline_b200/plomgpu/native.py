"""ctypes binding of the C ABI in include/plomgpu.h.

The CUDA library is mandatory: loading fails loudly when it is missing or
when no GPU is present at call time; nothing falls back to a CPU path.
"""

import ctypes as C
import os

import numpy as np

from . import build as _build


class PlomGpuError(RuntimeError):
    def __init__(self, code, msg):
        RuntimeError.__init__(self, 'plomgpu error %d: %s' % (code, msg))
        self.code = code


class ModelInfo(C.Structure):
    _fields_ = [(n, C.c_int) for n in (
        'n_par_sv', 'n_c', 'n_ac', 'n_cac', 'n_ts', 'n_ts_inc_unique', 'n_obs_inc', 'n_obs_prev',
        'n_drift', 'off_drift', 'off_inc', 'n_state', 'n_par_proc', 'n_par_obs', 'n_cov_cac', 'n_cov_ts',
        'n_reac', 'n_white_noise', 'coupled', 'pop_size_eq_sum_sv')] + [('name', C.c_char_p), ('n_hat', C.c_int)]


class BackTransform(C.Structure):
    _fields_ = [('f_inv', C.c_int), ('scale', C.c_int), ('is_duration', C.c_int), ('pad', C.c_int),
                ('a', C.c_double), ('b', C.c_double), ('multiplier', C.c_double)]


_P = C.POINTER
_dp = _P(C.c_double)
_ip = _P(C.c_int)
_up = _P(C.c_uint32)


class SmcDesc(C.Structure):
    _fields_ = [('J', C.c_int), ('n_obs', C.c_int), ('n_sub', _ip), ('t_sub', _dp), ('t_obs', _dp),
                ('dt', C.c_double), ('data', _dp), ('par_cac', _dp), ('par_ts', _dp), ('cov_cac', _dp),
                ('cov_ts', _dp), ('coupling', _dp), ('drift_group', _ip), ('drift_ngroups', _ip),
                ('drift_bt', _P(BackTransform)), ('drift_vol', _dp), ('x0', _dp), ('noises_off', C.c_int),
                ('filter', C.c_int), ('like_min', C.c_double), ('seed', C.c_uint64), ('precision', C.c_int),
                ('crn_normals', _dp), ('crn_uniforms', _dp), ('pop_size', _dp), ('cov_ts0', _dp),
                ('ode', C.c_int), ('eps_abs', C.c_double), ('eps_rel', C.c_double), ('cov_spline_meta', _ip),
                ('cov_spline_x', _dp), ('cov_spline_y', _dp), ('cov_spline_m2', _dp), ('cov_spline_knots', C.c_int),
                ('psr', C.c_int), ('paired_draws', C.c_int), ('x0_particles', _dp)]


class BatchDesc(C.Structure):
    _fields_ = [('n_filters', C.c_int), ('J', _ip), ('n_obs', _ip), ('data_row', _P(C.c_longlong)),
                ('data', _dp), ('n_rows', C.c_longlong), ('par_cac', _dp), ('par_ts', _dp), ('x0', _dp),
                ('seed', _P(C.c_uint64)), ('max_obs', C.c_int), ('n_sub', _ip), ('t_sub', _dp), ('t_obs', _dp),
                ('dt', C.c_double), ('cov_cac', _dp), ('cov_ts', _dp), ('coupling', _dp), ('drift_group', _ip),
                ('drift_ngroups', _ip), ('drift_bt', _P(BackTransform)), ('drift_vol', _dp), ('noises_off', C.c_int),
                ('filter', C.c_int), ('like_min', C.c_double), ('precision', C.c_int), ('block_threads', C.c_int),
                ('particles_per_thread', C.c_int)]


class MifDesc(C.Structure):
    _fields_ = [('n_runs', C.c_int), ('n_theta', C.c_int), ('proc_slot', _ip), ('obs_slot', _ip),
                ('theta_bt', _P(BackTransform)), ('estimated', _ip), ('proc_cac_slot', _ip), ('obs_ts_slot', _ip),
                ('fls', _ip), ('x0_slot', _ip), ('pop0', _dp), ('vol_slot', _ip), ('lag', C.c_int),
                ('prior', C.c_int), ('prior_kind', _ip), ('prior_lo', _dp), ('prior_hi', _dp),
                ('prior_finv', _P(BackTransform))]


class ServerOpts(C.Structure):
    _fields_ = [('max_J', C.c_int), ('memory_budget', C.c_double), ('ring_slots', C.c_int), ('plan_pool', C.c_int),
                ('precision', C.c_int), ('use_plan_pool', C.c_int), ('task_budget', C.c_int)]


class ServerStats(C.Structure):
    _fields_ = [('pending', C.c_longlong), ('in_flight', C.c_longlong), ('completed', C.c_longlong),
                ('launches', C.c_longlong), ('peak_in_flight', C.c_longlong), ('bytes_in_use', C.c_double),
                ('peak_bytes', C.c_double), ('persistent_loop', C.c_int)]


class SmcResult(C.Structure):
    _fields_ = [('loglik', C.c_double), ('n_all_fail', C.c_int), ('status', C.c_int),
                ('llike_n', _dp), ('ess_n', _dp), ('ancestors', _up), ('x_pred', _dp), ('x_final', _dp),
                ('hat', _dp), ('pred_res', _dp)]


API_SYMBOLS = ['plomgpu_get_model_info', 'plomgpu_draws_per_substep', 'plomgpu_smc_run', 'plomgpu_plan_create',
               'plomgpu_plan_create_ex', 'plomgpu_plan_propagate_time',
               'plomgpu_plan_update', 'plomgpu_plan_launch', 'plomgpu_plan_results', 'plomgpu_plan_stream',
               'plomgpu_plan_kernel_count', 'plomgpu_plan_destroy', 'plomgpu_debug_systematic_points',
               'plomgpu_debug_fail_boundary', 'plomgpu_release_memory',
               'plomgpu_resample_noalloc', 'plomgpu_last_error', 'plomgpu_batch_create', 'plomgpu_batch_launch',
               'plomgpu_batch_results', 'plomgpu_batch_stream', 'plomgpu_batch_config', 'plomgpu_batch_destroy',
               'plomgpu_batch_run', 'plomgpu_mif_create', 'plomgpu_mif_iteration', 'plomgpu_mif_destroy',
               'plomgpu_server_create', 'plomgpu_server_submit', 'plomgpu_server_poll', 'plomgpu_server_wait',
               'plomgpu_server_get_stats', 'plomgpu_server_destroy', 'plomgpu_particle_values',
               'plomgpu_plan_sample_traj', 'plomgpu_plan_update_drift', 'plomgpu_debug_draws',
               'plomgpu_mif_fls_means']


def _ptr(a, t):
    return a.ctypes.data_as(t) if a is not None else None


class DescHolder(object):
    """Keeps the numpy arrays of a descriptor alive."""

    def __init__(self, problem, crn_normals=None, crn_uniforms=None, precision=None):
        p = problem
        self.arrays = {}

        def keep(name, arr, dtype):
            if arr is None:
                return None
            a = np.ascontiguousarray(arr, dtype=dtype)
            self.arrays[name] = a
            return a

        n_sub = keep('n_sub', p.n_sub, np.int32)
        t_sub = keep('t_sub', p.t_sub if len(p.t_sub) else np.zeros(1), np.float64)
        t_obs = keep('t_obs', p.t_obs if len(p.t_obs) else np.zeros(1), np.float64)
        data = keep('data', p.data if p.data.size else np.full((1,), np.nan), np.float64)
        par_cac = keep('par_cac', p.par_cac if p.par_cac.size else np.zeros(1), np.float64)
        par_ts = keep('par_ts', p.par_ts if p.par_ts.size else np.zeros(1), np.float64)
        cov_cac = keep('cov_cac', p.cov_cac if p.cov_cac.size else np.zeros(1), np.float64)
        cov_ts = keep('cov_ts', p.cov_ts if p.cov_ts.size else np.zeros(1), np.float64)
        coupling = keep('coupling', p.coupling, np.float64) if p.coupling is not None else None
        dg = keep('drift_group', p.drift_group, np.int32)
        dng = keep('drift_ngroups', p.drift_ngroups, np.int32)
        dvol = keep('drift_vol', p.drift_vol, np.float64)
        nd, ncac = len(p.drift_bt), len(p.drift_bt[0])
        bts = (BackTransform * (nd * ncac))()
        for i in range(nd):
            for c in range(ncac):
                f, s, dur, a, b, mult = p.drift_bt[i][c]
                bts[i * ncac + c] = BackTransform(int(f), int(s), int(dur), 0, float(a), float(b), float(mult))
        self.bts = bts
        x0 = keep('x0', p.x0, np.float64)
        crn = keep('crn', crn_normals, np.float64) if crn_normals is not None else None
        crnu = keep('crnu', crn_uniforms, np.float64) if crn_uniforms is not None else None
        pop = keep('pop_size', getattr(p, 'pop_size', None), np.float64) if getattr(p, 'pop_size', None) is not None \
            else None
        cts0 = getattr(p, 'cov_ts0', None)
        cts0 = keep('cov_ts0', cts0 if cts0 is not None and cts0.size else np.zeros(1), np.float64)
        self.desc = SmcDesc(
            J=p.J, n_obs=p.n_obs, n_sub=_ptr(n_sub, _ip), t_sub=_ptr(t_sub, _dp), t_obs=_ptr(t_obs, _dp),
            dt=p.dt, data=_ptr(data, _dp), par_cac=_ptr(par_cac, _dp), par_ts=_ptr(par_ts, _dp),
            cov_cac=_ptr(cov_cac, _dp), cov_ts=_ptr(cov_ts, _dp), coupling=_ptr(coupling, _dp),
            drift_group=_ptr(dg, _ip), drift_ngroups=_ptr(dng, _ip), drift_bt=C.cast(bts, _P(BackTransform)),
            drift_vol=_ptr(dvol, _dp), x0=_ptr(x0, _dp), noises_off=p.noises_off, filter=1 if p.filter else 0,
            like_min=p.like_min, seed=p.seed, precision=precision or p.precision,
            crn_normals=_ptr(crn, _dp), crn_uniforms=_ptr(crnu, _dp), pop_size=_ptr(pop, _dp),
            cov_ts0=_ptr(cts0, _dp))
        self.desc.psr = 1 if getattr(p, 'psr', False) else 0
        self.desc.paired_draws = 1 if getattr(p, 'paired_draws', False) else 0
        if getattr(p, 'x0_particles', None) is not None:
            xp = keep('x0_particles', p.x0_particles, np.float64)
            if xp.shape != (self.model_off_inc(p), p.J):
                raise ValueError('x0_particles must be [off_inc][J]')
            self.desc.x0_particles = _ptr(xp, _dp)
        if getattr(p, 'ode', False):
            meta, xs, ys, m2 = p.spline_tables()
            meta = keep('sp_meta', meta if meta.size else np.zeros(3, np.int32), np.int32)
            xs = keep('sp_x', xs if xs.size else np.zeros(1), np.float64)
            ys = keep('sp_y', ys if ys.size else np.zeros(1), np.float64)
            m2 = keep('sp_m2', m2 if m2.size else np.zeros(1), np.float64)
            d = self.desc
            d.ode = 1
            d.eps_abs = p.eps_abs
            d.eps_rel = p.eps_rel
            d.cov_spline_meta = _ptr(meta, _ip)
            d.cov_spline_x = _ptr(xs, _dp)
            d.cov_spline_y = _ptr(ys, _dp)
            d.cov_spline_m2 = _ptr(m2, _dp)
            d.cov_spline_knots = int(xs.size)


    @staticmethod
    def model_off_inc(p):
        m = p.model
        return len(m.par_sv) * m.N_CAC + len(m.drift_par_proc) * m.N_CAC


class Outputs(object):
    def __init__(self, J, n_obs, S, ancestors=False, x_pred=False, x_final=False, n_hat=0, n_ts=0):
        self.llike_n = np.zeros(max(n_obs, 1))
        self.ess_n = np.zeros(max(n_obs, 1))
        self.ancestors = np.zeros((n_obs, J), dtype=np.uint32) if ancestors else None
        self.x_pred = np.zeros((n_obs, S, J)) if x_pred else None
        self.x_final = np.zeros((S, J)) if x_final else None
        self.hat = np.zeros((n_obs + 1, n_hat, 3)) if n_hat else None
        self.pred_res = np.zeros((max(n_obs, 1), n_ts, 2)) if n_hat else None
        self.res = SmcResult(0.0, 0, 0, _ptr(self.llike_n, _dp), _ptr(self.ess_n, _dp),
                             _ptr(self.ancestors, _up), _ptr(self.x_pred, _dp), _ptr(self.x_final, _dp),
                             _ptr(self.hat, _dp), _ptr(self.pred_res, _dp))

    @property
    def loglik(self):
        return self.res.loglik

    @property
    def n_all_fail(self):
        return self.res.n_all_fail


def _declare(lib):
    lib.plomgpu_get_model_info.argtypes = [_P(ModelInfo)]
    lib.plomgpu_draws_per_substep.argtypes = [C.c_int]
    lib.plomgpu_smc_run.argtypes = [_P(SmcDesc), _P(SmcResult)]
    lib.plomgpu_plan_create.argtypes = [_P(SmcDesc), _P(C.c_void_p)]
    lib.plomgpu_plan_create_ex.argtypes = [_P(SmcDesc), C.c_int, _P(C.c_void_p)]
    lib.plomgpu_plan_propagate_time.argtypes = [C.c_void_p, _dp, _ip]
    lib.plomgpu_plan_update.argtypes = [C.c_void_p, _dp, _dp, _dp, C.c_uint64]
    lib.plomgpu_plan_launch.argtypes = [C.c_void_p]
    lib.plomgpu_plan_sample_traj.argtypes = [C.c_void_p, C.c_double, _ip, _ip, _dp]
    lib.plomgpu_plan_update_drift.argtypes = [C.c_void_p, _dp]
    lib.plomgpu_plan_results.argtypes = [C.c_void_p, _P(SmcResult)]
    lib.plomgpu_plan_stream.argtypes = [C.c_void_p]
    lib.plomgpu_plan_stream.restype = C.c_void_p
    lib.plomgpu_plan_kernel_count.argtypes = [C.c_void_p]
    lib.plomgpu_plan_destroy.argtypes = [C.c_void_p]
    lib.plomgpu_plan_destroy.restype = None
    lib.plomgpu_debug_systematic_points.argtypes = [C.c_double, C.c_int, _dp]
    lib.plomgpu_debug_fail_boundary.argtypes = [C.c_double]
    lib.plomgpu_debug_fail_boundary.restype = C.c_double
    lib.plomgpu_debug_draws.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, C.c_uint64, C.c_int, C.c_int, _dp]
    lib.plomgpu_resample_noalloc.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_double, C.c_double,
                                             C.c_void_p, C.c_void_p, C.c_void_p]
    lib.plomgpu_last_error.restype = C.c_char_p
    lib.plomgpu_particle_values.argtypes = [_P(SmcDesc), _dp, C.c_int, _ip, _dp]
    lib.plomgpu_batch_create.argtypes = [_P(BatchDesc), _P(C.c_void_p)]
    lib.plomgpu_batch_launch.argtypes = [C.c_void_p]
    lib.plomgpu_batch_results.argtypes = [C.c_void_p, _dp, _ip, _dp]
    lib.plomgpu_batch_stream.argtypes = [C.c_void_p]
    lib.plomgpu_batch_stream.restype = C.c_void_p
    lib.plomgpu_batch_config.argtypes = [C.c_void_p, _ip, _ip, _ip]
    lib.plomgpu_batch_destroy.argtypes = [C.c_void_p]
    lib.plomgpu_batch_destroy.restype = None
    lib.plomgpu_batch_run.argtypes = [_P(BatchDesc), _dp, _ip]
    lib.plomgpu_mif_create.argtypes = [_P(SmcDesc), _P(MifDesc), _P(C.c_void_p)]
    lib.plomgpu_mif_iteration.argtypes = [C.c_void_p, _dp, _dp, _dp, _dp, C.c_uint64, _dp, _ip, _dp, _dp]
    lib.plomgpu_mif_fls_means.argtypes = [C.c_void_p, _dp, _ip]
    lib.plomgpu_mif_destroy.argtypes = [C.c_void_p]
    lib.plomgpu_mif_destroy.restype = None
    lib.plomgpu_server_create.argtypes = [_P(SmcDesc), _P(ServerOpts), _P(C.c_void_p)]
    lib.plomgpu_server_submit.argtypes = [C.c_void_p, C.c_int, _dp, _dp, _dp, C.c_uint64, _P(C.c_longlong)]
    lib.plomgpu_server_poll.argtypes = [C.c_void_p, C.c_longlong, _ip, _dp, _ip, _dp]
    lib.plomgpu_server_wait.argtypes = [C.c_void_p, C.c_longlong, C.c_double, _dp, _ip, _dp]
    lib.plomgpu_server_get_stats.argtypes = [C.c_void_p, _P(ServerStats)]
    lib.plomgpu_server_destroy.argtypes = [C.c_void_p]
    lib.plomgpu_server_destroy.restype = None
    return lib


_LIBS = {}


def load(name, path=None):
    """Loads libplomgpu_<name>.so (raises if it is not built)."""
    path = path or _build.lib_path(name)
    if path in _LIBS:
        return _LIBS[path]
    if not os.path.exists(path):
        raise PlomGpuError(-1, 'CUDA library %s is not built (run __graft_entry__.build())' % path)
    lib = _declare(C.CDLL(path))
    _LIBS[path] = lib
    return lib


def check(lib, rc):
    if rc != 0:
        raise PlomGpuError(rc, lib.plomgpu_last_error().decode())


def model_info(lib):
    mi = ModelInfo()
    check(lib, lib.plomgpu_get_model_info(C.byref(mi)))
    return mi


class Engine(object):
    """The GPU engine of one model library."""

    def __init__(self, name, path=None):
        self.lib = load(name, path)
        self.info = model_info(self.lib)

    def smc(self, problem, crn_normals=None, crn_uniforms=None, ancestors=False, x_pred=False, x_final=False,
            precision=None, hat=False):
        """One filter.  ``hat`` adds the filtered summaries (out.hat, [n_obs+1][n_hat][low, mean, high])
        and the prediction residuals (out.pred_res, [n_obs][n_ts][pred, res])."""
        h = DescHolder(problem, crn_normals, crn_uniforms, precision)
        out = Outputs(problem.J, problem.n_obs, self.info.n_state, ancestors, x_pred, x_final,
                      self.info.n_hat if hat else 0, self.info.n_ts)
        check(self.lib, self.lib.plomgpu_smc_run(C.byref(h.desc), C.byref(out.res)))
        return out

    def draws_per_substep(self, noises_off):
        return self.lib.plomgpu_draws_per_substep(noises_off)

    def release_memory(self):
        """Returns the unused memory of the library's plan memory pool (current device) to the driver."""
        check(self.lib, self.lib.plomgpu_release_memory())

    def particle_values(self, problem, X, rows):
        """[n_hat + n_ts][P]: summarised quantities then observation variances of particles X ([S][P]),
        particle i at time row rows[i] (0 = time 0, n + 1 = t_obs[n]; an int applies to all)."""
        h = DescHolder(problem, precision=64)
        X = np.ascontiguousarray(X, dtype=np.float64)
        P = X.shape[1]
        r = np.ascontiguousarray(np.broadcast_to(np.asarray(rows, dtype=np.int32), (P,)))
        out = np.zeros((self.info.n_hat + self.info.n_ts, P))
        check(self.lib, self.lib.plomgpu_particle_values(C.byref(h.desc), _ptr(X, _dp), P, _ptr(r, _ip),
                                                         _ptr(out, _dp)))
        return out

    def systematic_points(self, U, J):
        out = np.zeros(J)
        check(self.lib, self.lib.plomgpu_debug_systematic_points(U, J, _ptr(out, _dp)))
        return out

    DRAW_KINDS = {'normal': 0, 'binomial': 1, 'poisson': 2, 'gamma': 3, 'psr_normal': 4}

    def draws(self, kind, a=0.0, b=0.0, seed=1, streams=1024, per_stream=64, precision=32):
        """Draws of the device generators (test hook plomgpu_debug_draws): [streams * per_stream],
        stream-major."""
        out = np.zeros(int(streams) * int(per_stream))
        check(self.lib, self.lib.plomgpu_debug_draws(self.DRAW_KINDS[kind], int(precision), float(a), float(b),
                                                     int(seed), int(streams), int(per_stream), _ptr(out, _dp)))
        return out


PLAN_TIMING, PLAN_TRAJ, PLAN_SUMMARIES = 1, 2, 4


class Plan(object):
    """A captured filter (plomgpu_plan_*), for repeated likelihood evaluations."""

    def __init__(self, engine, problem, precision=None, timing=False, traj=False, summaries=False):
        self.engine = engine
        self.lib = engine.lib
        self.h = DescHolder(problem, precision=precision)
        self.p = C.c_void_p()
        flags = (PLAN_TIMING if timing else 0) | (PLAN_TRAJ if traj else 0) | (PLAN_SUMMARIES if summaries else 0)
        self.flags = flags
        check(self.lib, self.lib.plomgpu_plan_create_ex(C.byref(self.h.desc), flags, C.byref(self.p)))
        self.problem = problem

    def sample_traj(self, u):
        """(time rows [R], states [R][S]) of one trajectory of the last launch, in print order."""
        T, S = self.problem.n_obs, self.engine.info.n_state
        rows = np.zeros(T + 2, dtype=np.int32)
        states = np.zeros((T + 2, S))
        n = C.c_int()
        check(self.lib, self.lib.plomgpu_plan_sample_traj(self.p, float(u), C.byref(n), _ptr(rows, _ip),
                                                          _ptr(states, _dp)))
        return rows[:n.value].copy(), states[:n.value].copy()

    def propagate_time(self):
        """(total ms, launches) of the propagate kernels of the last launch."""
        ms, n = C.c_double(), C.c_int()
        check(self.lib, self.lib.plomgpu_plan_propagate_time(self.p, C.byref(ms), C.byref(n)))
        return ms.value, n.value

    def update(self, par_cac=None, par_ts=None, x0=None, seed=0):
        def ptr(a):
            return None if a is None else np.ascontiguousarray(a, dtype=np.float64).ctypes.data_as(_dp)
        keep = [np.ascontiguousarray(a, dtype=np.float64) if a is not None else None for a in (par_cac, par_ts, x0)]
        check(self.lib, self.lib.plomgpu_plan_update(
            self.p, *(k.ctypes.data_as(_dp) if k is not None else None for k in keep), C.c_uint64(seed)))

    def update_drift(self, drift_vol):
        v = np.ascontiguousarray(drift_vol, dtype=np.float64)
        check(self.lib, self.lib.plomgpu_plan_update_drift(self.p, _ptr(v, _dp)))

    def launch(self):
        check(self.lib, self.lib.plomgpu_plan_launch(self.p))

    def results(self, ancestors=False, x_pred=False):
        info = self.engine.info
        summ = bool(self.flags & PLAN_SUMMARIES)
        out = Outputs(self.problem.J, self.problem.n_obs, info.n_state, ancestors, x_pred, False,
                      info.n_hat if summ else 0, info.n_ts)
        check(self.lib, self.lib.plomgpu_plan_results(self.p, C.byref(out.res)))
        return out

    @property
    def stream(self):
        return self.lib.plomgpu_plan_stream(self.p)

    @property
    def kernel_count(self):
        return self.lib.plomgpu_plan_kernel_count(self.p)

    def close(self):
        if self.p:
            self.lib.plomgpu_plan_destroy(self.p)
            self.p = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch(object):
    """Many filters of one model in one persistent launch (plomgpu_batch_*)."""

    def __init__(self, engine, bp, precision=32, block_threads=0, particles_per_thread=0):
        self.engine = engine
        self.lib = engine.lib
        self.bp = bp
        self.keep = {}

        def k(name, a, dt):
            arr = np.ascontiguousarray(a, dtype=dt)
            self.keep[name] = arr
            return arr

        base = bp.base
        J = k('J', bp.J, np.int32)
        n_obs = k('n_obs', bp.n_obs, np.int32)
        rows = k('rows', bp.data_row, np.int64)
        data = k('data', bp.data, np.float64)
        par_cac = k('par_cac', bp.par_cac, np.float64)
        par_ts = k('par_ts', bp.par_ts, np.float64)
        x0 = k('x0', bp.x0, np.float64)
        seed = k('seed', bp.seed, np.uint64)
        n_sub = k('n_sub', base.n_sub, np.int32)
        t_sub = k('t_sub', base.t_sub, np.float64)
        t_obs = k('t_obs', base.t_obs, np.float64)
        cov_cac = k('cov_cac', base.cov_cac if base.cov_cac.size else np.zeros(1), np.float64)
        cov_ts = k('cov_ts', base.cov_ts if base.cov_ts.size else np.zeros(1), np.float64)
        coup = k('coup', base.coupling, np.float64) if base.coupling is not None else None
        dg = k('dg', base.drift_group, np.int32)
        dng = k('dng', base.drift_ngroups, np.int32)
        dvol = k('dvol', base.drift_vol, np.float64)
        nd, ncac = len(base.drift_bt), len(base.drift_bt[0])
        bts = (BackTransform * (nd * ncac))()
        for i in range(nd):
            for c in range(ncac):
                f, s_, dur, a_, b_, mult = base.drift_bt[i][c]
                bts[i * ncac + c] = BackTransform(int(f), int(s_), int(dur), 0, float(a_), float(b_), float(mult))
        self.keep['bts'] = bts
        self.desc = BatchDesc(
            n_filters=len(bp.J), J=_ptr(J, _ip), n_obs=_ptr(n_obs, _ip), data_row=rows.ctypes.data_as(_P(C.c_longlong)),
            data=_ptr(data, _dp), n_rows=data.shape[0], par_cac=_ptr(par_cac, _dp), par_ts=_ptr(par_ts, _dp),
            x0=_ptr(x0, _dp), seed=seed.ctypes.data_as(_P(C.c_uint64)), max_obs=base.n_obs, n_sub=_ptr(n_sub, _ip),
            t_sub=_ptr(t_sub, _dp), t_obs=_ptr(t_obs, _dp), dt=base.dt, cov_cac=_ptr(cov_cac, _dp),
            cov_ts=_ptr(cov_ts, _dp), coupling=_ptr(coup, _dp), drift_group=_ptr(dg, _ip),
            drift_ngroups=_ptr(dng, _ip), drift_bt=C.cast(bts, _P(BackTransform)), drift_vol=_ptr(dvol, _dp),
            noises_off=base.noises_off, filter=1 if base.filter else 0, like_min=base.like_min,
            precision=precision, block_threads=block_threads, particles_per_thread=particles_per_thread)
        self.p = C.c_void_p()
        check(self.lib, self.lib.plomgpu_batch_create(C.byref(self.desc), C.byref(self.p)))

    def launch(self):
        check(self.lib, self.lib.plomgpu_batch_launch(self.p))

    def results(self):
        n = len(self.bp.J)
        ll = np.zeros(n)
        nf = np.zeros(n, dtype=np.int32)
        ess = np.zeros(n)
        check(self.lib, self.lib.plomgpu_batch_results(self.p, _ptr(ll, _dp), _ptr(nf, _ip), _ptr(ess, _dp)))
        return ll, nf, ess

    @property
    def stream(self):
        return self.lib.plomgpu_batch_stream(self.p)

    @property
    def config(self):
        """(threads per block, particles per thread, CTAs) chosen by the autotuner."""
        bt, ppt, grid = C.c_int(), C.c_int(), C.c_int()
        check(self.lib, self.lib.plomgpu_batch_config(self.p, C.byref(bt), C.byref(ppt), C.byref(grid)))
        return bt.value, ppt.value, grid.value

    def close(self):
        if self.p:
            self.lib.plomgpu_batch_destroy(self.p)
            self.p = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class MifDescHolder(object):
    """plomgpu_mif_desc of n_runs runs over the components ``components``: list of
    (kind, index, back_transform tuple, estimated[, members]) with kind 'proc' or 'obs'
    (parameters of the step or the observation model) or 'fls' (initial conditions and
    drift start values, placed by set_fixed_lag); ``members`` lists the populations
    (process) or series (observation) a component applies to when the parameter is fitted
    per group (None: all)."""

    def __init__(self, n_runs, components, n_par_proc, n_par_obs, n_cac=1, n_ts=1):
        self.R = int(n_runs)
        self.Q = len(components)
        self.proc_slot = np.full(max(n_par_proc, 1), -1, dtype=np.int32)
        self.obs_slot = np.full(max(n_par_obs, 1), -1, dtype=np.int32)
        self.proc_cac = np.full((max(n_par_proc, 1), max(n_cac, 1)), -1, dtype=np.int32)
        self.obs_ts = np.full((max(n_par_obs, 1), max(n_ts, 1)), -1, dtype=np.int32)
        self.bts = (BackTransform * max(self.Q, 1))()
        self.estimated = np.zeros(max(self.Q, 1), dtype=np.int32)
        for q, comp in enumerate(components):
            kind, idx, bt, est = comp[:4]
            members = comp[4] if len(comp) > 4 else None
            if kind in ('proc', 'obs'):
                slots, table = (self.proc_slot, self.proc_cac) if kind == 'proc' else (self.obs_slot, self.obs_ts)
                if members is None:
                    slots[idx] = q
                else:
                    slots[idx] = -2
                    table[idx, list(members)] = q
            f, s_, dur, a_, b_, mult = bt
            self.bts[q] = BackTransform(int(f), int(s_), int(dur), 0, float(a_), float(b_), float(mult))
            self.estimated[q] = 1 if est else 0
        multi_p = bool(np.any(self.proc_slot == -2))
        multi_o = bool(np.any(self.obs_slot == -2))
        self.desc = MifDesc(self.R, self.Q, _ptr(self.proc_slot, _ip), _ptr(self.obs_slot, _ip),
                            C.cast(self.bts, _P(BackTransform)), _ptr(self.estimated, _ip),
                            _ptr(self.proc_cac, _ip) if multi_p else None,
                            _ptr(self.obs_ts, _ip) if multi_o else None)

    def set_fixed_lag(self, fls, x0_slot, pop0, lag):
        """Components fitted by fixed-lag smoothing (fls[q]), the component of every initial state word
        (x0_slot[off_inc], -1: x0), N at t = 0 and the lag L."""
        self.fls = np.ascontiguousarray(fls, dtype=np.int32)
        self.x0_slot = np.ascontiguousarray(x0_slot, dtype=np.int32)
        self.pop0 = np.ascontiguousarray(pop0, dtype=np.float64)
        self.desc.fls = _ptr(self.fls, _ip)
        self.desc.x0_slot = _ptr(self.x0_slot, _ip) if np.any(self.x0_slot >= 0) else None
        self.desc.pop0 = _ptr(self.pop0, _dp)
        self.desc.lag = int(lag)

    def set_vol_slot(self, vol_slot):
        """[n_drift][n_cac] component of every drift volatility (-1: the problem's table)."""
        self.vol_slot = np.ascontiguousarray(vol_slot, dtype=np.int32)
        self.desc.vol_slot = _ptr(self.vol_slot, _ip) if np.any(self.vol_slot >= 0) else None

    def set_prior(self, kinds, lo, hi, finv, lag):
        """The --prior patch: per component prior kind (0 flat, 1 normal, 2 pseudo-uniform), bounds and the
        back-transform to the prior's scale (tuples as theta_bt)."""
        self.prior_kind = np.ascontiguousarray(kinds, dtype=np.int32)
        self.prior_lo = np.ascontiguousarray(lo, dtype=np.float64)
        self.prior_hi = np.ascontiguousarray(hi, dtype=np.float64)
        self.prior_finv = (BackTransform * max(self.Q, 1))()
        for q, bt in enumerate(finv):
            f, s_, dur, a_, b_, mult = bt
            self.prior_finv[q] = BackTransform(int(f), int(s_), int(dur), 0, float(a_), float(b_), float(mult))
        self.desc.prior = 1
        self.desc.prior_kind = _ptr(self.prior_kind, _ip)
        self.desc.prior_lo = _ptr(self.prior_lo, _dp)
        self.desc.prior_hi = _ptr(self.prior_hi, _dp)
        self.desc.prior_finv = C.cast(self.prior_finv, _P(BackTransform))
        self.desc.lag = int(lag)


class MifPlan(object):
    """plomgpu_mif_*: lock-stepped iterated-filtering runs on the GPU."""

    def __init__(self, engine, problem, mif_holder, precision=None):
        self.engine = engine
        self.lib = engine.lib
        self.h = DescHolder(problem, precision=precision)
        self.m = mif_holder
        self.problem = problem
        self.p = C.c_void_p()
        check(self.lib, self.lib.plomgpu_mif_create(C.byref(self.h.desc), C.byref(self.m.desc), C.byref(self.p)))

    def iteration(self, theta_hat, sd_init, sd_mut, vt_add, seed):
        R, Q, T = self.m.R, self.m.Q, self.problem.n_obs
        ll = np.zeros(R)
        nf = np.zeros(R, dtype=np.int32)
        bart = np.zeros((R, T, Q))
        vt = np.zeros((R, T, Q))
        a = [np.ascontiguousarray(x, dtype=np.float64) for x in (theta_hat, sd_init, sd_mut, vt_add)]
        check(self.lib, self.lib.plomgpu_mif_iteration(self.p, *(x.ctypes.data_as(_dp) for x in a), C.c_uint64(seed),
                                                       _ptr(ll, _dp), _ptr(nf, _ip), _ptr(bart, _dp), _ptr(vt, _dp)))
        return ll, nf, bart, vt

    def fls_means(self):
        """([n_runs][n_theta] fixed-lag means of the last iteration (NaN outside the fixed-lag
        components), whether interval L was reached)."""
        out = np.zeros((self.m.R, self.m.Q))
        upd = C.c_int()
        check(self.lib, self.lib.plomgpu_mif_fls_means(self.p, _ptr(out, _dp), C.byref(upd)))
        return out, bool(upd.value)

    def close(self):
        if self.p:
            self.lib.plomgpu_mif_destroy(self.p)
            self.p = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server(object):
    """plomgpu_server_*: concurrent likelihood requests on one data set."""

    def __init__(self, engine, problem, max_J, memory_budget=0.0, ring_slots=0, plan_pool=0, precision=32,
                 use_plan_pool=False, task_budget=0):
        self.engine = engine
        self.lib = engine.lib
        self.h = DescHolder(problem, precision=precision)
        self.opts = ServerOpts(int(max_J), float(memory_budget), int(ring_slots), int(plan_pool), int(precision),
                               1 if use_plan_pool else 0, int(task_budget))
        self.p = C.c_void_p()
        check(self.lib, self.lib.plomgpu_server_create(C.byref(self.h.desc), C.byref(self.opts), C.byref(self.p)))

    def submit(self, J, par_cac=None, par_ts=None, x0=None, seed=0):
        keep = [None if a is None else np.ascontiguousarray(a, dtype=np.float64) for a in (par_cac, par_ts, x0)]
        t = C.c_longlong()
        check(self.lib, self.lib.plomgpu_server_submit(self.p, int(J), *(None if a is None else a.ctypes.data_as(_dp)
                                                                          for a in keep), C.c_uint64(seed),
                                                       C.byref(t)))
        return t.value

    def poll(self, ticket):
        done, ll, nf, lat = C.c_int(), C.c_double(), C.c_int(), C.c_double()
        check(self.lib, self.lib.plomgpu_server_poll(self.p, ticket, C.byref(done), C.byref(ll), C.byref(nf),
                                                     C.byref(lat)))
        return (ll.value, nf.value, lat.value) if done.value else None

    def wait(self, ticket, timeout=60.0):
        ll, nf, lat = C.c_double(), C.c_int(), C.c_double()
        check(self.lib, self.lib.plomgpu_server_wait(self.p, ticket, timeout, C.byref(ll), C.byref(nf), C.byref(lat)))
        return ll.value, nf.value, lat.value

    def stats(self):
        st = ServerStats()
        check(self.lib, self.lib.plomgpu_server_get_stats(self.p, C.byref(st)))
        return dict((f, getattr(st, f)) for f, _ in ServerStats._fields_)

    def close(self):
        if self.p:
            self.lib.plomgpu_server_destroy(self.p)
            self.p = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
