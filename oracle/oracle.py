"""ctypes wrapper of the CPU oracle (test infrastructure only).

Used by tests/, __graft_entry__.smoke() and the CPU-baseline leg of bench.py
as the checker; the product never imports it.
"""

import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), 'iterated-inference-pipeline_b200'))

from plomgpu import native  # noqa: E402  (descriptor structs shared with the C ABI)

from build_oracle import build as _build, lib_path  # noqa: E402

_dp = C.POINTER(C.c_double)


class Oracle(object):
    def __init__(self, name, build=True):
        path = _build(name) if build else lib_path(name)
        self.lib = C.CDLL(path)
        L = self.lib
        L.oracle_model_info.argtypes = [C.POINTER(native.ModelInfo)]
        L.oracle_draws_per_substep.argtypes = [C.c_int]
        L.oracle_smc_run.argtypes = [C.POINTER(native.SmcDesc), C.POINTER(native.SmcResult), C.c_int]
        L.oracle_systematic_points_sequential.argtypes = [C.c_double, C.c_int, _dp]
        L.oracle_systematic_points_sequential.restype = None
        L.oracle_systematic_points_table.argtypes = [C.c_double, C.c_int, _dp]
        L.oracle_step.argtypes = [_dp, C.c_double, C.c_double, C.c_int, C.POINTER(native.SmcDesc), C.c_int, _dp]
        L.oracle_obs_loglik.argtypes = [_dp, C.POINTER(native.SmcDesc), C.c_int]
        L.oracle_obs_loglik.restype = C.c_double
        L.oracle_obs_moments.argtypes = [C.c_double, C.c_int, C.c_double, C.POINTER(native.SmcDesc), _dp, _dp]
        L.oracle_obs_moments.restype = None
        L.oracle_like.argtypes = [C.c_double, C.c_double, C.c_double, C.c_double]
        L.oracle_like.restype = C.c_double
        L.oracle_log_like_terms.argtypes = [C.c_int, _dp, _dp, _dp, C.c_double, _dp, _dp, C.POINTER(C.c_int),
                                            C.POINTER(C.c_int)]
        L.oracle_log_like_terms.restype = None
        L.oracle_weight_and_resample.argtypes = [_dp, C.c_int, C.c_double, C.c_double, _dp, _dp,
                                                 C.POINTER(C.c_uint32)]
        L.oracle_mif_iteration.argtypes = [C.POINTER(native.SmcDesc), C.POINTER(native.MifDesc), _dp, _dp, _dp, _dp,
                                           _dp, C.POINTER(C.c_int), _dp, _dp, _dp]
        L.oracle_psr_samples.argtypes = [C.c_int, C.c_double, C.c_double, C.c_uint64, C.c_int, _dp]
        L.oracle_psr_samples.restype = None
        L.oracle_psr_samples_f.argtypes = [C.c_int, C.c_double, C.c_double, C.c_uint64, C.c_int, _dp]
        L.oracle_psr_samples_f.restype = None
        L.oracle_ci95.argtypes = [_dp, _dp, C.c_int, _dp, _dp]
        L.oracle_ci95.restype = None
        L.oracle_proj2obs.argtypes = [_dp, _dp]
        L.oracle_proj2obs.restype = None
        self.info = native.ModelInfo()
        L.oracle_model_info(C.byref(self.info))
        self.n_hat = self.info.n_hat

    def draws_per_substep(self, noises_off):
        return self.lib.oracle_draws_per_substep(noises_off)

    def smc(self, problem, crn_normals=None, crn_uniforms=None, ancestors=False, x_pred=False, x_final=False,
            n_threads=0, hat=False):
        h = native.DescHolder(problem, crn_normals, crn_uniforms, precision=64)
        out = native.Outputs(problem.J, problem.n_obs, self.info.n_state, ancestors, x_pred, x_final,
                             self.n_hat if hat else 0, self.info.n_ts)
        rc = self.lib.oracle_smc_run(C.byref(h.desc), C.byref(out.res), n_threads)
        if rc:
            raise RuntimeError('oracle failed: %d' % rc)
        return out

    def weight_and_resample(self, likes, U, like_min=1e-17):
        """weight() then systematic_sampling() on linear likelihoods: (normalised, select, llike_n, ess, all_fail)."""
        w = np.ascontiguousarray(likes, dtype=np.float64).copy()
        sel = np.zeros(len(w), dtype=np.uint32)
        ll, ess = C.c_double(), C.c_double()
        fail = self.lib.oracle_weight_and_resample(w.ctypes.data_as(_dp), len(w), like_min, U, C.byref(ll),
                                                   C.byref(ess), sel.ctypes.data_as(C.POINTER(C.c_uint32)))
        return w, sel, ll.value, ess.value, fail

    def mif_iteration(self, problem, mif_desc_holder, theta_hat, sd_init, sd_mut, vt_add, seed):
        """One iterated-filtering iteration of every run (FP64, Philox draws of the GPU's FP64 mode)."""
        import copy as _copy
        p = _copy.copy(problem)
        p.seed = seed
        h = native.DescHolder(p, precision=64)
        R, Q, T = mif_desc_holder.R, mif_desc_holder.Q, problem.n_obs
        ll = np.zeros(R)
        nf = np.zeros(R, dtype=np.int32)
        bart = np.zeros((R, T, Q))
        vt = np.zeros((R, T, Q))
        fls = np.full((R, Q), np.nan)
        a = [np.ascontiguousarray(x, dtype=np.float64) for x in (theta_hat, sd_init, sd_mut, vt_add)]
        rc = self.lib.oracle_mif_iteration(C.byref(h.desc), C.byref(mif_desc_holder.desc),
                                           *(x.ctypes.data_as(_dp) for x in a),
                                           ll.ctypes.data_as(_dp), nf.ctypes.data_as(C.POINTER(C.c_int)),
                                           bart.ctypes.data_as(_dp), vt.ctypes.data_as(_dp), fls.ctypes.data_as(_dp))
        if rc:
            raise RuntimeError('oracle mif iteration failed: %d' % rc)
        self.last_fls_means = fls
        return ll, nf, bart, vt

    def systematic_points(self, U, J, table=False):
        out = np.zeros(J)
        if table:
            ns = self.lib.oracle_systematic_points_table(U, J, out.ctypes.data_as(_dp))
            if ns < 0:
                raise RuntimeError('systematic table overflow')
        else:
            self.lib.oracle_systematic_points_sequential(U, J, out.ctypes.data_as(_dp))
        return out

    def step(self, problem, x, t, sub, normals, noises_off=0):
        h = native.DescHolder(problem, precision=64)
        x = np.ascontiguousarray(x, dtype=np.float64).copy()
        nz = np.ascontiguousarray(normals, dtype=np.float64)
        self.lib.oracle_step(x.ctypes.data_as(_dp), t, problem.dt, noises_off, C.byref(h.desc), sub,
                             nz.ctypes.data_as(_dp))
        return x

    def obs_loglik(self, problem, x, n):
        h = native.DescHolder(problem, precision=64)
        x = np.ascontiguousarray(x, dtype=np.float64)
        return self.lib.oracle_obs_loglik(x.ctypes.data_as(_dp), C.byref(h.desc), n)

    def obs_moments(self, problem, x, ts, t):
        h = native.DescHolder(problem, precision=64)
        mu, var = C.c_double(), C.c_double()
        self.lib.oracle_obs_moments(x, ts, t, C.byref(h.desc), C.byref(mu), C.byref(var))
        return mu.value, var.value

    def like(self, y, mu, var, like_min):
        return self.lib.oracle_like(y, mu, var, like_min)

    def log_like_terms(self, y, mu, var, like_min):
        """(log term in double, in single precision, floor flags of each) for arrays y, mu, var."""
        y, mu, var = (np.ascontiguousarray(a, dtype=np.float64) for a in (y, mu, var))
        n = len(y)
        o64, o32 = np.zeros(n), np.zeros(n)
        f64, f32 = np.zeros(n, dtype=np.int32), np.zeros(n, dtype=np.int32)
        ip = C.POINTER(C.c_int)
        self.lib.oracle_log_like_terms(n, y.ctypes.data_as(_dp), mu.ctypes.data_as(_dp), var.ctypes.data_as(_dp),
                                       like_min, o64.ctypes.data_as(_dp), o32.ctypes.data_as(_dp),
                                       f64.ctypes.data_as(ip), f32.ctypes.data_as(ip))
        return o64, o32, f64, f32

    def proj2obs(self, x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        obs = np.zeros(self.info.n_ts)
        self.lib.oracle_proj2obs(x.ctypes.data_as(_dp), obs.ctypes.data_as(_dp))
        return obs

    def ci95(self, values, weights=None):
        """get_CI95: (low, high) of values under weights (None: 1/J)."""
        v = np.ascontiguousarray(values, dtype=np.float64)
        w = None if weights is None else np.ascontiguousarray(weights, dtype=np.float64)
        lo, hi = C.c_double(), C.c_double()
        self.lib.oracle_ci95(v.ctypes.data_as(_dp), None if w is None else w.ctypes.data_as(_dp), len(v),
                             C.byref(lo), C.byref(hi))
        return lo.value, hi.value

    def psr_samples(self, kind, a, b=0.0, seed=1, count=10000, precision=64):
        """Draws of the psr samplers: 'binomial' (n=a, p=b), 'poisson' (mu=a), 'gamma' (shape a, scale b);
        precision 32: the single-precision samplers of FP32 particle states."""
        out = np.zeros(count)
        k = {'binomial': 0, 'poisson': 1, 'gamma': 2}[kind]
        fn = self.lib.oracle_psr_samples if precision == 64 else self.lib.oracle_psr_samples_f
        fn(k, float(a), float(b), int(seed), int(count), out.ctypes.data_as(_dp))
        return out
