// Many independent particle filters in one persistent launch.
//
// Every CTA takes whole filters from a work queue (an atomic ticket over a
// host-given order, longest first) and runs all of a filter's observation
// intervals itself: the propagate loop over its particles, then a block-level
// log-sum-exp reduction, cumulative-weight scan and ancestor search
// (weight() / systematic_sampling() / resample_X(), model_builder/C/core/
// smc.c:27-161), separated by __syncthreads.  The per-filter state lives in a
// per-CTA workspace in HBM; the whole batch needs one launch, no host
// round trip between intervals.
//
// The draws of filter f are keyed by its own seed (PhiloxKey(seed_f, 0)), so
// a filter of the batch consumes exactly the draws of the single-filter path
// (plomgpu_smc_run) with that seed.
#pragma once

#include "smc_engine.cuh"

namespace plomgpu {

struct BatchFilter {
  int J;
  int n_obs;
  long long data_row;  // first data row of the filter
  uint64_t seed;
};

template <class T>
struct BatchArgs {
  const BatchFilter* filters;
  const int* order;         // processing order of the filters
  int n_filters;
  unsigned* queue;          // work ticket (reset by the host before each launch)
  const double* par_cac;    // [n][N_PAR_PROC][N_CAC]
  const double* par_ts;     // [n][N_PAR_OBS][N_TS]
  const double* x0;         // [n][S]
  const double* data;       // concatenated rows [*][N_TS]
  // time grid shared by all filters (of the longest one)
  const int* n_sub;         // [max_obs]
  const int* sub0;          // [max_obs]
  const double* t_sub;
  const double* t_obs;
  const T* cov_cac;         // [sub][N_COV_CAC][N_CAC]
  const double* cov_ts;     // [max_obs][N_COV_TS][N_TS]
  const T* coupling;
  const int* drift_group;
  const int* drift_ngroups;
  const plomrt::BackTransform* drift_bt;
  const T* drift_vol;
  double dt, like_min, log_like_min;
  double fail_b;  // largest log-weight that fails: exp(l) <= LIKE_MIN^N_TS (fail_boundary)
  int filter_on;
  // per-CTA workspace
  unsigned char* ws;
  size_t ws_stride;
  int max_J;
  // outputs
  double* loglik;
  int* n_all_fail;
  double* ess_min;
  int* error;
};

template <class T>
struct BatchWs {
  T* X[2];
  T* lw;
  double* C;
  uint32_t* anc;
};

template <class T>
__host__ __device__ inline size_t batch_ws_bytes(int max_J) {
  const size_t mj = (size_t)((max_J + 31) & ~31);
  return 2 * (size_t)M::S * mj * sizeof(T) + mj * sizeof(T) + mj * sizeof(double) + mj * sizeof(uint32_t) + 256;
}

template <class T>
__device__ inline BatchWs<T> batch_ws(unsigned char* base, int max_J) {
  const size_t mj = (size_t)((max_J + 31) & ~31);
  BatchWs<T> w;
  unsigned char* p = base;
  w.C = reinterpret_cast<double*>(p);
  p += mj * sizeof(double);
  w.X[0] = reinterpret_cast<T*>(p);
  p += (size_t)M::S * mj * sizeof(T);
  w.X[1] = reinterpret_cast<T*>(p);
  p += (size_t)M::S * mj * sizeof(T);
  w.lw = reinterpret_cast<T*>(p);
  p += mj * sizeof(T);
  w.anc = reinterpret_cast<uint32_t*>(p);
  return w;
}

// block-wide helpers (fixed order: deterministic for a fixed block size)
template <int BT>
__device__ inline LseAcc block_lse(LseAcc a, LseAcc* sh) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) a = lse_shfl(a, off);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) sh[warp] = a;
  __syncthreads();
  if (warp == 0) {
    a = (lane < BT / 32) ? sh[lane] : LseAcc{-INFINITY, 0.0, 0.0, 0};
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) a = lse_shfl(a, off);
    if (lane == 0) sh[0] = a;
  }
  __syncthreads();
  a = sh[0];
  __syncthreads();
  return a;
}

// exclusive scan of one double per thread; returns the exclusive prefix, total in *tot
template <int BT>
__device__ inline double block_exscan(double v, double* sh, double* tot) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  double x = v;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const double o = __shfl_up_sync(0xffffffffu, x, off);
    if (lane >= off) x += o;
  }
  if (lane == 31) sh[warp] = x;
  __syncthreads();
  if (warp == 0) {
    double w = (lane < BT / 32) ? sh[lane] : 0.0;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const double o = __shfl_up_sync(0xffffffffu, w, off);
      if (lane >= off) w += o;
    }
    if (lane < BT / 32) sh[lane] = w;
  }
  __syncthreads();
  const double excl = (warp > 0 ? sh[warp - 1] : 0.0) + (x - v);
  *tot = sh[BT / 32 - 1];
  __syncthreads();
  return excl;
}

// Shared memory of one CTA running whole filters.
template <class T, int BT>
struct CtaShared {
  LseAcc lse[BT / 32];
  double scan[BT / 32];
  plomrt::SysSeg seg[plomrt::SYS_MAX_SEG];
  int f, ns, fail;
  double m, s1;
  __align__(16) T coup[kSmemCoup > 0 ? kSmemCoup : 4];
  __align__(16) T par[kSmemPar > 0 ? kSmemPar : 4];
  double par_ts[M::N_PAR_OBS * M::N_TS > 0 ? M::N_PAR_OBS * M::N_TS : 1];
};

// One filter on the calling CTA: every interval of `job` (propagate, block
// log-sum-exp, chunked FP64 scan, ancestor search).  All threads of the CTA
// call it; outputs are written by thread 0.
struct FilterJob {
  int J;
  int n_obs;
  uint64_t seed;
  const double* data;     // first row of the filter's data
  const double* par_cac;  // [N_PAR_PROC][N_CAC]
  const double* par_ts;   // [N_PAR_OBS][N_TS]
  const double* x0;       // [S]
};

// PPT particles per thread are advanced together (particles j, j + BT, ...):
// their independent Philox / Box-Muller chains fill each other's latency.
template <class T, int V, bool DRIFT, int BT, int PPT = 1>
__device__ void cta_filter(CtaShared<T, BT>& sh, const BatchArgs<T>& a, const FilterJob& job, const BatchWs<T>& ws,
                           const size_t ld, double* out_ll, int* out_nf, double* out_ess) {
  const int J = job.J;
  for (int i = threadIdx.x; i < M::N_PAR_PROC * M::N_CAC; i += BT) sh.par[i] = (T)job.par_cac[i];
  for (int i = threadIdx.x; i < M::N_PAR_OBS * M::N_TS; i += BT) sh.par_ts[i] = job.par_ts[i];
  for (int j = threadIdx.x; j < J; j += BT) {
#pragma unroll
    for (int w = 0; w < M::OFF_INC; ++w) ws.X[0][(size_t)w * ld + j] = (T)job.x0[w];
  }
  __syncthreads();
  ProcEnv<T> e;
  e.par_ = sh.par;
  e.coup_ = sh.coup;
  e.dgroup_ = a.drift_group;
  e.dng_ = a.drift_ngroups;
  e.dbt_ = a.drift_bt;
  e.dvol_ = a.drift_vol;
  ObsEnv oe;
  oe.par_ts_ = sh.par_ts;
  const plomrt::PhiloxKey key = plomrt::make_key(job.seed, 0u);
  const T dt = (T)a.dt;
  double loglik = 0.0, ess_min = INFINITY;
  int n_all_fail = 0;
  int cur = 0;
  bool resampled = false;
  for (int n = 0; n < job.n_obs; ++n) {
    const double* y = job.data + (size_t)n * M::N_TS;
    bool any = false;
#pragma unroll
    for (int ts = 0; ts < M::N_TS; ++ts) any |= !isnan(y[ts]);
    const bool weigh = a.filter_on && any;
    oe.cov_ts_ = a.cov_ts + (size_t)n * M::N_COV_TS * M::N_TS;
    const int K = __ldg(a.n_sub + n), sub0 = __ldg(a.sub0 + n);
    const double t_obs = __ldg(a.t_obs + n);
    const T* Xp = ws.X[cur];
    T* Xn = ws.X[cur ^ 1];
    LseAcc acc = {-INFINITY, 0.0, 0.0, 0};
    for (int j0 = threadIdx.x; j0 < J; j0 += BT * PPT) {
      // a lane past the end recomputes the last particle and stores nothing
      int jj[PPT];
      RegState<T, M::S> x[PPT];
#pragma unroll
      for (int q = 0; q < PPT; ++q) {
        jj[q] = min(j0 + q * BT, J - 1);
        const uint32_t src = resampled ? ws.anc[jj[q]] : (uint32_t)jj[q];
#pragma unroll
        for (int w = 0; w < M::OFF_INC; ++w) x[q][w] = Xp[(size_t)w * ld + src];
#pragma unroll
        for (int w = M::OFF_INC; w < M::S; ++w) x[q][w] = T(0);
      }
      for (int k = 0; k < K; ++k) {
        const int sub = sub0 + k;
        e.cov_ = a.cov_cac + (size_t)sub * M::N_COV_CAC * M::N_CAC;
        const T t = (T)__ldg(a.t_sub + sub);
#pragma unroll
        for (int q = 0; q < PPT; ++q) {
          PhiloxDraws<T, V> d;
          d.key = key;
          d.j = (uint32_t)jj[q];
          d.n = (uint32_t)n;
          d.sub = (uint32_t)k;
          M::template step<V, DRIFT, T>(x[q], t, dt, e, d);
        }
      }
#pragma unroll
      for (int q = 0; q < PPT; ++q) {
        const int j = j0 + q * BT;
        if (j >= J) continue;
#pragma unroll
        for (int w = 0; w < M::OFF_INC; ++w) Xn[(size_t)w * ld + j] = x[q][w];
        if (weigh) {
          double obs[M::N_TS];
          M::template proj2obs<T>(x[q], obs);
          double ll = 0.0;
          int fl = 0;
#pragma unroll
          for (int ts = 0; ts < M::N_TS; ++ts) {
            const double yy = y[ts];
            if (isnan(yy)) continue;
            const double mu = M::obs_mean(obs[ts], ts, t_obs, oe);
            const double var = M::obs_var(obs[ts], ts, t_obs, oe);
            ll += plomrt::log_like_term_p<T>(yy, mu, var, a.like_min, &fl);
          }
          const T l = (T)plomrt::finish_loglik(ll, fl, M::N_TS);
          ws.lw[j] = l;
          if (weight_fails_at(l, a.fail_b)) {
            acc.nfail += 1;
          } else {
            LseAcc b = {(double)l, 1.0, 1.0, 0};
            acc = lse_merge(acc, b);
          }
        }
      }
    }
    cur ^= 1;
    if (!weigh) {
      resampled = false;
      __syncthreads();
      continue;
    }
    acc = block_lse<BT>(acc, sh.lse);  // (syncs: Xn / lw visible to the block)
    if (threadIdx.x == 0) {
      const int all_fail = (acc.nfail == J);
      double llike, ess;
      if (all_fail) {
        llike = a.log_like_min * (double)M::N_TS;
        ess = 0.0;
        n_all_fail += 1;
      } else {
        llike = acc.m + log(acc.s1 / (double)J);
        ess = (acc.s1 * acc.s1) / acc.s2;
      }
      loglik += llike;
      ess_min = fmin(ess_min, ess);
      sh.fail = all_fail;
      sh.m = acc.m;
      sh.s1 = acc.s1;
      const double inc = 1.0 / (double)J;
      const double U = inc * plomrt::resample_uniform(key, (uint32_t)n);
      int ns = plomrt::systematic_table(U, inc, J, sh.seg, plomrt::SYS_MAX_SEG);
      if (ns < 0) {
        atomicOr(a.error, (int)ERR_SYS_TABLE);
        ns = 0;
      }
      sh.ns = ns;
    }
    __syncthreads();
    if (sh.fail || sh.ns == 0) {
      for (int j = threadIdx.x; j < J; j += BT) ws.anc[j] = (uint32_t)j;
    } else {
      // cumulative normalised weights: each thread a contiguous chunk
      const int P = (J + BT - 1) / BT;
      const int i0 = threadIdx.x * P;
      const int i1 = min(J, i0 + P);
      const double m = sh.m, s1 = sh.s1;
      double run = 0.0;
      for (int i = i0; i < i1; ++i) {
        const T l = ws.lw[i];
        run += weight_fails_at(l, a.fail_b) ? 0.0 : exp((double)l - m) / s1;
      }
      double tot;
      const double pre = block_exscan<BT>(run, sh.scan, &tot);
      run = pre;
      for (int i = i0; i < i1; ++i) {
        const T l = ws.lw[i];
        run += weight_fails_at(l, a.fail_b) ? 0.0 : exp((double)l - m) / s1;
        ws.C[i] = run;
      }
      __syncthreads();
      const int ns = sh.ns;
      for (int j = threadIdx.x; j < J; j += BT) {
        const double ran = plomrt::systematic_point(sh.seg, ns, j);
        int lo = 0, hi = J - 1;
        while (lo < hi) {
          const int mid = (lo + hi) >> 1;
          if (ran > ws.C[mid]) lo = mid + 1; else hi = mid;
        }
        ws.anc[j] = (uint32_t)lo;
      }
    }
    resampled = true;
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    *out_ll = loglik;
    *out_nf = n_all_fail;
    if (out_ess) *out_ess = ess_min;
  }
}

template <class T, int V, bool DRIFT, int BT, int PPT = 1>
__global__ void __launch_bounds__(BT) k_batch(const BatchArgs<T> a) {
  __shared__ CtaShared<T, BT> sh;
  if constexpr (M::COUPLED) {
    for (int i = threadIdx.x; i < M::N_CAC * M::N_CAC; i += BT) sh.coup[i] = a.coupling[i];
  }
  const BatchWs<T> ws = batch_ws<T>(a.ws + blockIdx.x * a.ws_stride, a.max_J);
  const size_t ld = (size_t)((a.max_J + 31) & ~31);
  for (;;) {
    __syncthreads();
    if (threadIdx.x == 0) {
      const unsigned t = atomicAdd(a.queue, 1u);
      sh.f = (t < (unsigned)a.n_filters) ? a.order[t] : -1;
    }
    __syncthreads();
    const int f = sh.f;
    if (f < 0) break;
    const BatchFilter fl = a.filters[f];
    FilterJob job;
    job.J = fl.J;
    job.n_obs = fl.n_obs;
    job.seed = fl.seed;
    job.data = a.data + (size_t)fl.data_row * M::N_TS;
    job.par_cac = a.par_cac + (size_t)f * M::N_PAR_PROC * M::N_CAC;
    job.par_ts = a.par_ts + (size_t)f * M::N_PAR_OBS * M::N_TS;
    job.x0 = a.x0 + (size_t)f * M::S;
    cta_filter<T, V, DRIFT, BT, PPT>(sh, a, job, ws, ld, a.loglik + f, a.n_all_fail + f,
                                     a.ess_min ? a.ess_min + f : nullptr);
  }
}

}  // namespace plomgpu
