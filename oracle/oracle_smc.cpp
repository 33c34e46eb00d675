// ORACLE — test infrastructure only.  CPU FP64 restatement of the
// reference's SMC path, used by tests/ (parity), __graft_entry__.smoke() and
// the CPU-baseline leg of bench.py.  Nothing in the product links it.
//
// Restates, in order of the loop body of run_SMC
// (model_builder/C/core/smc.c:204-307):
//   * replicate_J_p_X_0                         smc.c:167-176
//   * copy X[n] -> X[n+1], reset_inc            smc.c:250-253, prediction_util.c:25-33
//   * f_prediction_sde_* (while t < t1 step)    prediction_util.c:197-287
//     with the generated step of the model (the emitted header, whose text
//     follows core_template.c:215-339 and Ccoder.py:366-508)
//   * proj2obs, get_log_likelihood, exp()       core_template.c:52-102, likelihood.c:56-70, smc.c:271-273
//   * weight()                                  smc.c:27-83   (linear space, as the reference)
//   * systematic_sampling()                     smc.c:90-112  (sequential cumulative sum and ran += inc)
//   * resample_X()                              smc.c:142-161 (AoS gather)
// Particles are AoS like struct s_X (plom.h:476-483); the particle loop runs
// under OpenMP like run_SMC with FLAG_OMP (smc.c:255-274); weighting and
// resampling are serial like the reference.
//
// Draws: either the common-random-number table of the descriptor (every
// normal and every resampling uniform injected), or Philox4x32-10 with the
// same counter layout as the GPU's FP64 mode.  The GSL mt19937 / ranlxs0
// streams of the reference (build.c:1019-1030) cannot be matched by a
// parallel device and are not reproduced.
//
// Deviation kept on purpose: systematic_sampling stops at the last particle
// when rounding leaves ran above the final cumulative weight (the reference
// would read past the end of prob[]).
#include PLOM_MODEL_HEADER
#include "plomgpu.h"
#include "ode_rkf45.h"

#include <algorithm>
#include <math.h>
#include <stdint.h>
#include <string.h>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef plomgen::Model M;

namespace {

struct HostState {
  static constexpr bool DYNAMIC = true;
  double* b;
  double& operator[](int i) const { return b[i]; }
};

struct HostEnv {
  const double* par_;
  const double* cov_;
  const double* coup_;
  const int* dgroup_;
  const int* dng_;
  const plomgpu_back_transform* dbt_;
  const double* dvol_;
  double par(int p, int cac) const { return par_[p * M::N_CAC + cac]; }
  double cov(int k, int cac) const { return cov_[k * M::N_CAC + cac]; }
  double coupling(int a, int b) const { return coup_[a * M::N_CAC + b]; }
  plomrt::V4<double> coupling4(int a, int b) const {
    const double* w = coup_ + a * M::N_CAC + b;
    return plomrt::V4<double>{w[0], w[1], w[2], w[3]};
  }
  int drift_group(int i, int cac) const { return dgroup_[i * M::N_CAC + cac]; }
  int drift_ngroups(int i) const { return dng_[i]; }
  double drift_vol(int i, int g) const { return dvol_[i * M::N_CAC + g]; }
  double drift_value(int i, int g, double xw) const {
    plomrt::BackTransform bt;
    memcpy(&bt, &dbt_[i * M::N_CAC + g], sizeof(bt));
    return plomrt::back_transform<double>(xw, bt);
  }
};

// the ODE right-hand side reads its covariates from a buffer refreshed at
// every stage time (plomrt::rkf45_interval)
struct HostOdeEnv : HostEnv {
  double* covl_;
  double cov(int k, int cac) const { return covl_[k * M::N_CAC + cac]; }
};

// Deterministic skeleton over interval n (f_prediction_ode restated by
// plomrt::rkf45_interval, the integrator the GPU engine uses).
int ode_propagate(double* x, const plomgpu_smc_desc* d, int n, int sub0) {
  HostOdeEnv e;
  e.par_ = d->par_cac;
  e.cov_ = nullptr;
  e.coup_ = d->coupling;
  e.dgroup_ = d->drift_group;
  e.dng_ = d->drift_ngroups;
  e.dbt_ = d->drift_bt;
  e.dvol_ = d->drift_vol;
  std::vector<double> covl(M::N_COV_CAC * M::N_CAC > 0 ? M::N_COV_CAC * M::N_CAC : 1);
  e.covl_ = covl.data();
  plomrt::CovSplines cs{d->cov_spline_meta, d->cov_spline_x, d->cov_spline_y, d->cov_spline_m2};
  std::vector<double> work(8 * M::S);
  const double t0 = d->n_sub[n] > 0 ? d->t_sub[sub0] : d->t_obs[n];
  int steps = 0;
  return plomrt::rkf45_interval<M, double>(x, t0, d->t_obs[n], d->dt, d->eps_abs, d->eps_rel, e, cs, work.data(),
                                           1000000, &steps);
}

struct HostObsEnv {
  const double* par_ts_;
  const double* cov_ts_;
  double par_ts(int p, int ts) const { return par_ts_[p * M::N_TS + ts]; }
  double cov_ts(int k, int ts) const { return cov_ts_[k * M::N_TS + ts]; }
};

template <int V>
struct TableSource {
  static constexpr int PER_BLOCK = 1;
  const double* p;
  template <int N>
  void normals(int cac, double* out) const {
    for (int i = 0; i < N; ++i) out[i] = p[cac * N + i];
  }
  double drift_normal(int i, int g) const { return p[M::N_CAC * M::draws_per_cac(V) + i * M::N_CAC + g]; }
};

template <int V>
struct PhiloxSource {
  static constexpr int PER_BLOCK = plomrt::NormalGen<double>::per_block();
  plomrt::PhiloxKey key;
  uint32_t j, n, sub;
  template <int N>
  void normals(int cac, double* out) const {
    plomrt::NormalGen<double>::fill<N>(key, j, n, (sub * (uint32_t)(M::N_CAC + 1) + (uint32_t)cac) << 12, out);
  }
  double drift_normal(int i, int g) const {
    double z[1];
    plomrt::NormalGen<double>::fill<1>(
        key, j, n, ((sub * (uint32_t)(M::N_CAC + 1) + (uint32_t)M::N_CAC) << 12) + (uint32_t)(i * M::N_CAC + g), z);
    return z[0];
  }
};

// Poisson-system step over interval n (step_psr + f_prediction_psr,
// model_builder/C/core/prediction_util.c:290-317) with the GPU's Philox
// streams.
template <bool DRIFT, bool NOENV>
void propagate_psr(double* x, const plomgpu_smc_desc* d, int n, int j, int sub0) {
  HostEnv e;
  e.par_ = d->par_cac;
  e.coup_ = d->coupling;
  e.dgroup_ = d->drift_group;
  e.dng_ = d->drift_ngroups;
  e.dbt_ = d->drift_bt;
  e.dvol_ = d->drift_vol;
  HostState xs;
  xs.b = x;
  const plomrt::PhiloxKey key = plomrt::make_key(d->seed, 0u);
  for (int k = 0; k < d->n_sub[n]; ++k) {
    const int sub = sub0 + k;
    e.cov_ = d->cov_cac ? d->cov_cac + (size_t)sub * M::N_COV_CAC * M::N_CAC : nullptr;
    PhiloxSource<0> src;
    src.key = key;
    src.j = (uint32_t)j;
    src.n = (uint32_t)n;
    src.sub = (uint32_t)k;
    M::step_psr<DRIFT, NOENV, double>(xs, d->t_sub[sub], d->dt, e, key, (uint32_t)j, (uint32_t)n, (uint32_t)k, src);
  }
}

typedef void (*PsrFn)(double*, const plomgpu_smc_desc*, int, int, int);

PsrFn pick_psr(int noises_off) {
  const bool drift = M::N_DRIFT > 0 && !(noises_off & PLOMGPU_NO_DRIFT);
  const bool noenv = (noises_off & PLOMGPU_NO_ENV_STO) != 0;
  if (drift) return noenv ? &propagate_psr<true, true> : &propagate_psr<true, false>;
  return noenv ? &propagate_psr<false, true> : &propagate_psr<false, false>;
}

int draws_per_substep(int noises_off) {
  const bool drift = M::N_DRIFT > 0 && !(noises_off & PLOMGPU_NO_DRIFT);
  return M::N_CAC * M::draws_per_cac(noises_off & 3) + (drift ? M::N_DRIFT * M::N_CAC : 0);
}

template <int V, bool DRIFT>
void propagate(double* x, const plomgpu_smc_desc* d, int n, int j, int sub0, const double* crn_interval, int D) {
  HostEnv e;
  e.par_ = d->par_cac;
  e.coup_ = d->coupling;
  e.dgroup_ = d->drift_group;
  e.dng_ = d->drift_ngroups;
  e.dbt_ = d->drift_bt;
  e.dvol_ = d->drift_vol;
  HostState xs;
  xs.b = x;
  const int K = d->n_sub[n];
  for (int k = 0; k < K; ++k) {
    const int sub = sub0 + k;
    e.cov_ = d->cov_cac ? d->cov_cac + (size_t)sub * M::N_COV_CAC * M::N_CAC : nullptr;
    const double t = d->t_sub[sub];
    if (crn_interval) {
      TableSource<V> src;
      src.p = crn_interval + ((size_t)j * K + k) * D;
      M::step<V, DRIFT, double>(xs, t, d->dt, e, src);
    } else {
      PhiloxSource<V> src;
      src.key = plomrt::make_key(d->seed, 0u);
      src.j = (uint32_t)j;
      src.n = (uint32_t)n;
      src.sub = (uint32_t)k;
      M::step<V, DRIFT, double>(xs, t, d->dt, e, src);
    }
  }
}

typedef void (*PropFn)(double*, const plomgpu_smc_desc*, int, int, int, const double*, int);

PropFn pick(int noises_off) {
  const int v = noises_off & 3;
  const bool drift = M::N_DRIFT > 0 && !(noises_off & PLOMGPU_NO_DRIFT);
  if (drift) {
    switch (v) {
      case 0: return &propagate<0, true>;
      case 1: return &propagate<1, true>;
      case 2: return &propagate<2, true>;
      default: return &propagate<3, true>;
    }
  }
  switch (v) {
    case 0: return &propagate<0, false>;
    case 1: return &propagate<1, false>;
    case 2: return &propagate<2, false>;
    default: return &propagate<3, false>;
  }
}

double log_likelihood(const double* x, const plomgpu_smc_desc* d, int n) {
  double obs[M::N_TS];
  HostState xs;
  xs.b = const_cast<double*>(x);
  M::proj2obs<double>(xs, obs);
  HostObsEnv oe;
  oe.par_ts_ = d->par_ts;
  oe.cov_ts_ = d->cov_ts ? d->cov_ts + (size_t)n * M::N_COV_TS * M::N_TS : nullptr;
  const double* y = d->data + (size_t)n * M::N_TS;
  double ll = 0.0;
  int fl = 0;
  for (int ts = 0; ts < M::N_TS; ++ts) {
    if (isnan(y[ts])) continue;
    const double mu = M::obs_mean(obs[ts], ts, d->t_obs[n], oe);
    const double var = M::obs_var(obs[ts], ts, d->t_obs[n], oe);
    ll += plomrt::log_like_term(y[ts], mu, var, d->like_min, &fl);
  }
  return plomrt::finish_loglik(ll, fl, M::N_TS);
}

// weight(), smc.c:27-83
int weight(std::vector<double>& w, int J, double like_min, double* llike_n, double* ess, double* Llike,
           int* n_all_fail, uint32_t* select) {
  double like_tot = 0.0;
  int nfail = 0;
  double e = 0.0;
  const double thresh = pow(like_min, (double)M::N_TS);
  for (int j = 0; j < J; ++j) {
    if (w[j] <= thresh) {
      w[j] = 0.0;
      nfail += 1;
    } else {
      like_tot += w[j];
      e += w[j] * w[j];
    }
  }
  int success = 1;
  if (nfail == J) {
    success = 0;
    *n_all_fail += 1;
    *llike_n = log(like_min) * M::N_TS;
    const double invJ = 1.0 / (double)J;
    for (int j = 0; j < J; ++j) {
      w[j] = invJ;
      select[j] = (uint32_t)j;
    }
    e = 0.0;
  } else {
    for (int j = 0; j < J; ++j) w[j] /= like_tot;
    *llike_n = log(like_tot / (double)J);
    e = (like_tot * like_tot) / e;
  }
  *ess = e;
  *Llike += *llike_n;
  return success;
}

// systematic_sampling(), smc.c:90-112, with the end-of-array guard
void systematic_sampling(const std::vector<double>& prob, int J, double U, uint32_t* select) {
  const double inc = 1.0 / (double)J;
  double ran = U;
  int i = 0;
  double weight_cum = prob[0];
  for (int j = 0; j < J; ++j) {
    while (ran > weight_cum && i < J - 1) {
      i++;
      weight_cum += prob[i];
    }
    select[j] = (uint32_t)i;
    ran += inc;
  }
}

}  // namespace

// ---------------------------------------------------------------------------
// Filtered summaries.  get_CI95 (model_builder/C/core/hat.c:28-57): sort the
// values, accumulate the weights in sorted order until they reach 2.5 % /
// 97.5 %, take the value where the sum crossed.  compute_hat / compute_hat_nn
// (hat.c:68-260): weighted (or 1/J) mean and interval of every state word,
// remainder N(t) - sum of states, observation mean per series, and drifted
// parameter mapped by f_inv.
namespace {

constexpr int kNHat = M::N_PAR_SV * M::N_CAC + (M::POP_SIZE_EQ_SUM_SV ? 0 : M::N_CAC) + M::N_TS +
                      M::N_DRIFT * M::N_CAC;

void ci95(const std::vector<double>& v, const double* w, int J, double* lo, double* hi) {
  std::vector<int> idx(J);
  for (int j = 0; j < J; ++j) idx[j] = j;
  std::sort(idx.begin(), idx.end(), [&](int a, int b) { return v[a] < v[b]; });
  const double invJ = 1.0 / (double)J;
  const double level[2] = {0.025, 0.975};
  double* out[2] = {lo, hi};
  for (int q = 0; q < 2; ++q) {
    int k = 0;
    double cum = 0.0;
    while (cum < level[q] && k < J) {
      cum += w ? w[idx[k]] : invJ;
      ++k;
    }
    *out[q] = v[idx[(k - 1) < 0 ? 0 : k - 1]];
  }
}

// X: AoS particles [J][S]; w: normalised weights or null (1/J); hat: [kNHat][3]
void compute_hat(const std::vector<double>& X, int J, const double* w, const plomgpu_smc_desc* d,
                 const double* cov_ts, const double* pop, double t, double* hat) {
  const int S = M::S;
  std::vector<double> v(J);
  int q = 0;
  auto summarise = [&]() {
    double mean = 0.0;
    for (int j = 0; j < J; ++j) mean += v[j] * (w ? w[j] : 1.0);
    if (!w) mean /= (double)J;
    ci95(v, w, J, &hat[q * 3 + 0], &hat[q * 3 + 2]);
    hat[q * 3 + 1] = mean;
    ++q;
  };
  for (int i = 0; i < M::N_PAR_SV * M::N_CAC; ++i) {
    for (int j = 0; j < J; ++j) v[j] = X[(size_t)j * S + i];
    summarise();
  }
  if (!M::POP_SIZE_EQ_SUM_SV) {
    for (int c = 0; c < M::N_CAC; ++c) {
      for (int j = 0; j < J; ++j) {
        double sv = 0.0;
        for (int i = 0; i < M::N_PAR_SV; ++i) sv += X[(size_t)j * S + i * M::N_CAC + c];
        v[j] = pop[c] - sv;
      }
      summarise();
    }
  }
  HostObsEnv oe;
  oe.par_ts_ = d->par_ts;
  oe.cov_ts_ = cov_ts;
  for (int ts = 0; ts < M::N_TS; ++ts) {
    for (int j = 0; j < J; ++j) {
      HostState xs;
      xs.b = const_cast<double*>(&X[(size_t)j * S]);
      double obs[M::N_TS];
      M::proj2obs<double>(xs, obs);
      v[j] = M::obs_mean(obs[ts], ts, t, oe);
    }
    summarise();
  }
  for (int i = 0; i < M::N_DRIFT * M::N_CAC; ++i) {
    plomrt::BackTransform b;
    memcpy(&b, &d->drift_bt[i], sizeof(b));
    b.scale = 0;
    b.multiplier = 1.0;
    b.is_duration = 0;
    for (int j = 0; j < J; ++j) v[j] = plomrt::back_transform<double>(X[(size_t)j * S + M::OFF_DRIFT + i], b);
    summarise();
  }
}

// print_prediction_residuals (model_builder/C/core/print.c:632-711) on the
// resampled particles: running mean / M2 of the observation means, mean of
// the observation variances.  out: [N_TS][2] = pred, res.
void pred_res(const std::vector<double>& X, int J, const plomgpu_smc_desc* d, const double* cov_ts, double t,
              const double* y, double* out) {
  HostObsEnv oe;
  oe.par_ts_ = d->par_ts;
  oe.cov_ts_ = cov_ts;
  for (int ts = 0; ts < M::N_TS; ++ts) {
    double kn = 0.0, pred = 0.0, var_obs = 0.0, M2 = 0.0;
    for (int j = 0; j < J; ++j) {
      HostState xs;
      xs.b = const_cast<double*>(&X[(size_t)j * M::S]);
      double obs[M::N_TS];
      M::proj2obs<double>(xs, obs);
      kn += 1.0;
      const double x = M::obs_mean(obs[ts], ts, t, oe);
      const double delta = x - pred;
      pred += delta / kn;
      M2 += delta * (x - pred);
      var_obs += M::obs_var(obs[ts], ts, t, oe);
    }
    const double var_state = M2 / (kn - 1.0);
    var_obs /= (double)J;
    out[ts * 2 + 0] = pred;
    out[ts * 2 + 1] = (y[ts] - pred) / sqrt(var_state + var_obs);
  }
}

}  // namespace

extern "C" {

int oracle_model_info(plomgpu_model_info* o) {
  o->n_par_sv = M::N_PAR_SV;
  o->n_c = M::N_C;
  o->n_ac = M::N_AC;
  o->n_cac = M::N_CAC;
  o->n_ts = M::N_TS;
  o->n_ts_inc_unique = M::N_TS_INC_UNIQUE;
  o->n_obs_inc = M::N_OBS_INC;
  o->n_obs_prev = M::N_OBS_PREV;
  o->n_drift = M::N_DRIFT;
  o->off_drift = M::OFF_DRIFT;
  o->off_inc = M::OFF_INC;
  o->n_state = M::S;
  o->n_par_proc = M::N_PAR_PROC;
  o->n_par_obs = M::N_PAR_OBS;
  o->n_cov_cac = M::N_COV_CAC;
  o->n_cov_ts = M::N_COV_TS;
  o->n_reac = M::N_REAC;
  o->n_white_noise = M::N_WN;
  o->coupled = M::COUPLED ? 1 : 0;
  o->pop_size_eq_sum_sv = M::POP_SIZE_EQ_SUM_SV ? 1 : 0;
  o->name = M::NAME;
  o->n_hat = kNHat;
  return 0;
}

int oracle_draws_per_substep(int noises_off) { return draws_per_substep(noises_off); }

// Draws of the psr samplers from one uniform stream (distribution tests).
// kind 0 binomial(a, b), 1 Poisson(a), 2 Gamma(shape a, scale b).
void oracle_psr_samples(int kind, double a, double b, uint64_t seed, int count, double* out) {
  plomrt::UniformStream rs;
  rs.init(plomrt::make_key(seed, 0u), 0u, 0u, 0u);
  for (int i = 0; i < count; ++i) {
    if (kind == 0) out[i] = plomrt::binomial(rs, a, b);
    else if (kind == 1) out[i] = plomrt::poisson(rs, a);
    else out[i] = plomrt::gamma(rs, a, b);
  }
}

// The same draws with the single-precision samplers of FP32 particle states
// (host build of the device code's algorithm).
void oracle_psr_samples_f(int kind, double a, double b, uint64_t seed, int count, double* out) {
  plomrt::UniformStreamF rs;
  rs.init(plomrt::make_key(seed, 0u), 0u, 0u, 0u);
  for (int i = 0; i < count; ++i) {
    if (kind == 0) out[i] = plomrt::binomial(rs, (float)a, (float)b);
    else if (kind == 1) out[i] = plomrt::poisson(rs, (float)a);
    else out[i] = plomrt::gamma(rs, (float)a, (float)b);
  }
}

// get_CI95 on given values and weights (null: 1/J), known-answer tests.
void oracle_ci95(const double* v, const double* w, int J, double* lo, double* hi) {
  std::vector<double> vv(v, v + J);
  ci95(vv, w, J, lo, hi);
}

// run_SMC restated.  n_threads <= 0: OpenMP default.
int oracle_smc_run(const plomgpu_smc_desc* d, plomgpu_smc_result* r, int n_threads) {
  const int J = d->J, S = M::S;
  if (J < 1 || d->precision != 64 && d->precision != 32) return PLOMGPU_EINVAL;
#ifdef _OPENMP
  if (n_threads > 0) omp_set_num_threads(n_threads);
#endif
  const PropFn prop = pick(d->noises_off);
  const PsrFn psr_prop = pick_psr(d->noises_off);
  int ode_fail = 0;
  if (d->psr && (d->ode || d->crn_normals)) return PLOMGPU_EINVAL;
  const int D = d->crn_normals ? draws_per_substep(d->noises_off) : 0;
  // AoS particles: proj[S] per particle, two generations
  std::vector<double> X((size_t)J * S), Xn((size_t)J * S);
  for (int j = 0; j < J; ++j)
    for (int w = 0; w < S; ++w)
      X[(size_t)j * S + w] = (w < M::OFF_INC) ? (d->x0_particles ? d->x0_particles[(size_t)w * J + j] : d->x0[w]) : 0.0;
  std::vector<double> wts(J);
  std::vector<uint32_t> select(J);
  if (r->hat) compute_hat(X, J, nullptr, d, d->cov_ts0, d->pop_size, 0.0, r->hat);
  double Llike = 0.0;
  int n_all_fail = 0;
  size_t crn_off = 0;
  int sub0 = 0;
  for (int n = 0; n < d->n_obs; ++n) {
    const double* y = d->data + (size_t)n * M::N_TS;
    const double* cov_n = d->cov_ts ? d->cov_ts + (size_t)n * M::N_COV_TS * M::N_TS : nullptr;
    int n_nonan = 0;
    for (int ts = 0; ts < M::N_TS; ++ts)
      if (!isnan(y[ts])) ++n_nonan;
    const bool weigh = d->filter && n_nonan > 0;
    const double* crn_n = d->crn_normals ? d->crn_normals + crn_off : nullptr;
#pragma omp parallel for schedule(static)
    for (int j = 0; j < J; ++j) {
      double* x = &Xn[(size_t)j * S];
      memcpy(x, &X[(size_t)j * S], sizeof(double) * S);
      for (int w = M::OFF_INC; w < S; ++w) x[w] = 0.0;  // reset_inc
      if (d->ode) {
        if (ode_propagate(x, d, n, sub0) != plomrt::ODE_OK) ode_fail = 1;
      } else if (d->psr) {
        psr_prop(x, d, n, j, sub0);
      } else {
        prop(x, d, n, j, sub0, crn_n, D);
      }
      if (n_nonan) wts[j] = exp(log_likelihood(x, d, n));
    }
    if (r->x_pred) {
      for (int j = 0; j < J; ++j)
        for (int w = 0; w < S; ++w) r->x_pred[((size_t)n * S + w) * J + j] = Xn[(size_t)j * S + w];
    }
    crn_off += (size_t)J * d->n_sub[n] * D;
    sub0 += d->n_sub[n];
    double llike_n = 0.0, ess = 0.0;
    if (weigh) {
      if (weight(wts, J, d->like_min, &llike_n, &ess, &Llike, &n_all_fail, select.data())) {
        double u;
        if (d->crn_normals) {
          u = d->crn_uniforms[n];
        } else {
          u = plomrt::resample_uniform(plomrt::make_key(d->seed, 0u), (uint32_t)n);
        }
        const double U = (1.0 / (double)J) * u;
        systematic_sampling(wts, J, U, select.data());
      }
      if (r->hat)
        compute_hat(Xn, J, wts.data(), d, cov_n, d->pop_size ? d->pop_size + (size_t)(n + 1) * M::N_CAC : nullptr,
                    d->t_obs[n], r->hat + (size_t)(n + 1) * kNHat * 3);
      // resample_X: gather the state words (incidences are reset next interval)
      for (int j = 0; j < J; ++j) {
        const size_t s = (size_t)select[j] * S;
        for (int w = 0; w < S; ++w) X[(size_t)j * S + w] = Xn[s + w];
      }
      if (r->pred_res) pred_res(X, J, d, cov_n, d->t_obs[n], y, r->pred_res + (size_t)n * M::N_TS * 2);
    } else {
      for (int j = 0; j < J; ++j) select[j] = (uint32_t)j;
      if (r->hat)
        compute_hat(Xn, J, nullptr, d, cov_n, d->pop_size ? d->pop_size + (size_t)(n + 1) * M::N_CAC : nullptr,
                    d->t_obs[n], r->hat + (size_t)(n + 1) * kNHat * 3);
      X.swap(Xn);
    }
    if (r->llike_n) r->llike_n[n] = llike_n;
    if (r->ess_n) r->ess_n[n] = ess;
    if (r->ancestors) memcpy(r->ancestors + (size_t)n * J, select.data(), sizeof(uint32_t) * J);
  }
  if (r->x_final) {
    for (int j = 0; j < J; ++j)
      for (int w = 0; w < S; ++w) r->x_final[(size_t)w * J + j] = X[(size_t)j * S + w];
  }
  r->loglik = Llike;
  r->n_all_fail = n_all_fail;
  r->status = ode_fail ? PLOMGPU_EINVAL : 0;
  return ode_fail ? PLOMGPU_EINVAL : 0;
}

// weight() + systematic_sampling() on given likelihoods (known-answer tests).
int oracle_weight_and_resample(double* w, int J, double like_min, double U, double* llike_n, double* ess,
                               uint32_t* select) {
  std::vector<double> v(w, w + J);
  double Llike = 0.0;
  int n_all_fail = 0;
  if (weight(v, J, like_min, llike_n, ess, &Llike, &n_all_fail, select)) systematic_sampling(v, J, U, select);
  memcpy(w, v.data(), sizeof(double) * J);
  return n_all_fail;
}

// ---------------------------------------------------------------------------
// One iteration of iterated filtering for R runs (the body of the m loop of
// mif(), model_builder/C/mif/mif.c:115-200, with diagonal proposals):
// per-particle parameters proposed around theta_hat (ran_proposal), per
// interval back-transformed (back_transform_theta2par), particles propagated
// and weighted, weighted mean / prediction variance of every component
// (mean_var_theta_theoretical_mif, C/mif/methods.c:133-192), systematic
// resampling, parameters resampled and perturbed (resample_and_mut_theta_mif,
// methods.c:261-367), particles resampled.  Draws: Philox with the counter
// layout of the GPU's FP64 mode.
}  // extern "C"

namespace {

// uni: parameters from the particle; a per-group one (cslot / tslot) picks
// the component of the population / series
struct HostMifEnv : HostEnv {
  double parp[M::N_PAR_PROC > 0 ? M::N_PAR_PROC : 1];
  unsigned uni;
  const int* slot;
  const int* cslot;
  const int* vslot;  // [N_DRIFT][N_CAC] volatility components, NULL: table
  const double* nat;
  double par(int p, int cac) const {
    if (!((uni >> p) & 1u)) return par_[p * M::N_CAC + cac];
    return slot[p] == -2 ? nat[cslot[p * M::N_CAC + cac]] : parp[p];
  }
  double drift_vol(int i, int g) const {
    if (vslot && vslot[i * M::N_CAC + g] >= 0) return nat[vslot[i * M::N_CAC + g]];
    return dvol_[i * M::N_CAC + g];
  }
};

struct HostMifObsEnv : HostObsEnv {
  double obsp[M::N_PAR_OBS > 0 ? M::N_PAR_OBS : 1];
  unsigned uni;
  const int* slot;
  const int* tslot;
  const double* nat;
  double par_ts(int p, int ts) const {
    if (!((uni >> p) & 1u)) return par_ts_[p * M::N_TS + ts];
    return slot[p] == -2 ? nat[tslot[p * M::N_TS + ts]] : obsp[p];
  }
};

template <int V, bool DRIFT>
void mif_propagate(double* x, const plomgpu_smc_desc* d, const HostMifEnv& e0, int n, int j, int sub0, uint32_t run) {
  HostMifEnv e = e0;
  HostState xs;
  xs.b = x;
  for (int k = 0; k < d->n_sub[n]; ++k) {
    const int sub = sub0 + k;
    e.cov_ = d->cov_cac ? d->cov_cac + (size_t)sub * M::N_COV_CAC * M::N_CAC : nullptr;
    PhiloxSource<V> src;
    src.key = plomrt::make_key(d->seed, run);
    src.j = (uint32_t)j;
    src.n = (uint32_t)n;
    src.sub = (uint32_t)k;
    M::step<V, DRIFT, double>(xs, d->t_sub[sub], d->dt, e, src);
  }
}

}  // namespace

extern "C" {

int oracle_mif_iteration(const plomgpu_smc_desc* d, const plomgpu_mif_desc* mf, const double* theta_hat,
                         const double* sd_init, const double* sd_mut, const double* vt_add, double* loglik,
                         int* n_all_fail_out, double* bart, double* vt, double* fls_out) {
  const int J = d->J, S = M::S, Q = mf->n_theta, R = mf->n_runs;
  const int v = d->noises_off & 3;
  const bool drift = M::N_DRIFT > 0 && !(d->noises_off & PLOMGPU_NO_DRIFT);
  typedef void (*MP)(double*, const plomgpu_smc_desc*, const HostMifEnv&, int, int, int, uint32_t);
  MP prop;
  if (drift) prop = v == 0 ? &mif_propagate<0, true> : v == 1 ? &mif_propagate<1, true> : v == 2 ? &mif_propagate<2, true> : &mif_propagate<3, true>;
  else prop = v == 0 ? &mif_propagate<0, false> : v == 1 ? &mif_propagate<1, false> : v == 2 ? &mif_propagate<2, false> : &mif_propagate<3, false>;
  for (int r = 0; r < R; ++r) {
    const plomrt::PhiloxKey key = plomrt::make_key(d->seed, (uint32_t)r);
    std::vector<double> X((size_t)J * S), Xn((size_t)J * S), th((size_t)J * Q), thn((size_t)J * Q), w(J);
    std::vector<uint32_t> select(J);
    // weights before the first weighted interval (read by the fixed-lag means only)
    for (int j = 0; j < J; ++j) w[j] = 1.0 / (double)J;
    for (int j = 0; j < J; ++j) {
      for (int s = 0; s < S; ++s) X[(size_t)j * S + s] = (s < M::OFF_INC) ? d->x0[s] : 0.0;
      // propose_safe_theta_and_load_X0 (C/core/proposal.c:40-62): propose until the
      // initial proportions of every cac sum to at most 1 (models with a remainder)
      for (int attempt = 0;; ++attempt) {
        for (int q = 0; q < Q; ++q) {
          double t = theta_hat[(size_t)r * Q + q];
          if (mf->estimated[q]) {
            double z[1];
            plomrt::NormalGen<double>::fill<1>(key, (uint32_t)j, (uint32_t)attempt, (uint32_t)q, z,
                                               (uint32_t)plomrt::STREAM_INIT);
            t += sd_init[q] * z[0];
          }
          th[(size_t)j * Q + q] = t;
        }
        if (!mf->x0_slot || M::POP_SIZE_EQ_SUM_SV) break;
        bool ok = true;
        for (int c = 0; c < M::N_CAC && ok; ++c) {
          double sum = 0.0;
          for (int i = 0; i < M::N_PAR_SV; ++i) {
            const int wd = i * M::N_CAC + c, q = mf->x0_slot[wd];
            plomrt::BackTransform bt;
            if (q >= 0) memcpy(&bt, &mf->theta_bt[q], sizeof(bt));
            sum += q >= 0 ? plomrt::back_transform<double>(th[(size_t)j * Q + q], bt) : d->x0[wd] / mf->pop0[c];
          }
          if (sum > 1.0) ok = false;
        }
        if (ok) break;
        if (attempt + 1 >= 1000) return 8;
      }
      if (mf->x0_slot) {
        for (int wd = 0; wd < M::OFF_INC; ++wd) {
          const int q = mf->x0_slot[wd];
          if (q < 0) continue;
          const double t = th[(size_t)j * Q + q];
          if (wd < M::N_PAR_SV * M::N_CAC) {
            plomrt::BackTransform bt;
            memcpy(&bt, &mf->theta_bt[q], sizeof(bt));
            X[(size_t)j * S + wd] = plomrt::back_transform<double>(t, bt) * mf->pop0[wd % M::N_CAC];
          } else {
            X[(size_t)j * S + wd] = t;
          }
        }
      }
    }
    const bool is_fls_q = mf->fls != nullptr;
    auto fls_of = [&](int q) { return is_fls_q && mf->fls[q] != 0; };
    double Llike = 0.0;
    int n_all_fail = 0;
    int sub0 = 0;
    for (int n = 0; n < d->n_obs; ++n) {
      const double* y = d->data + (size_t)n * M::N_TS;
      int n_nonan = 0;
      for (int ts = 0; ts < M::N_TS; ++ts)
        if (!isnan(y[ts])) ++n_nonan;
#pragma omp parallel for schedule(static)
      for (int j = 0; j < J; ++j) {
        HostMifEnv e;
        e.par_ = d->par_cac;
        e.coup_ = d->coupling;
        e.dgroup_ = d->drift_group;
        e.dng_ = d->drift_ngroups;
        e.dbt_ = d->drift_bt;
        e.dvol_ = d->drift_vol;
        e.uni = 0u;
        HostMifObsEnv oe;
        oe.par_ts_ = d->par_ts;
        oe.cov_ts_ = d->cov_ts ? d->cov_ts + (size_t)n * M::N_COV_TS * M::N_TS : nullptr;
        oe.uni = 0u;
        double nat[32];
        for (int q = 0; q < Q; ++q) {
          plomrt::BackTransform bt;
          memcpy(&bt, &mf->theta_bt[q], sizeof(bt));
          nat[q] = plomrt::back_transform<double>(th[(size_t)j * Q + q], bt);
        }
        e.slot = mf->proc_slot;
        e.cslot = mf->proc_cac_slot;
        e.vslot = mf->vol_slot;
        e.nat = nat;
        oe.slot = mf->obs_slot;
        oe.tslot = mf->obs_ts_slot;
        oe.nat = nat;
        for (int k = 0; k < M::N_PAR_PROC; ++k) {
          e.parp[k] = mf->proc_slot[k] >= 0 ? nat[mf->proc_slot[k]] : 0.0;
          if (mf->proc_slot[k] >= 0 || mf->proc_slot[k] == -2) e.uni |= 1u << k;
        }
        for (int k = 0; k < M::N_PAR_OBS; ++k) {
          oe.obsp[k] = mf->obs_slot[k] >= 0 ? nat[mf->obs_slot[k]] : 0.0;
          if (mf->obs_slot[k] >= 0 || mf->obs_slot[k] == -2) oe.uni |= 1u << k;
        }
        double* x = &Xn[(size_t)j * S];
        memcpy(x, &X[(size_t)j * S], sizeof(double) * S);
        for (int s = M::OFF_INC; s < S; ++s) x[s] = 0.0;
        prop(x, d, e, n, j, sub0, (uint32_t)r);
        if (n_nonan) {
          double obs[M::N_TS];
          HostState xs;
          xs.b = x;
          M::proj2obs<double>(xs, obs);
          double ll = 0.0;
          int fl = 0;
          for (int ts = 0; ts < M::N_TS; ++ts) {
            if (isnan(y[ts])) continue;
            const double mu = M::obs_mean(obs[ts], ts, d->t_obs[n], oe);
            const double var = M::obs_var(obs[ts], ts, d->t_obs[n], oe);
            ll += plomrt::log_like_term(y[ts], mu, var, d->like_min, &fl);
          }
          // patch_likelihood_prior (C/mif/methods.c:469-520), in log space
          double lpr = 0.0;
          if (mf->prior) {
            for (int q = 0; q < Q; ++q) {
              if (!mf->estimated[q]) continue;
              const bool f = fls_of(q);
              if (f && !(n < mf->lag)) continue;
              plomrt::BackTransform fb;
              memcpy(&fb, &mf->prior_finv[q], sizeof(fb));
              const double xn = plomrt::back_transform<double>(th[(size_t)j * Q + q], fb);
              const double pr = plomrt::prior_density(mf->prior_kind[q], xn, mf->prior_lo[q], mf->prior_hi[q]);
              lpr += plomrt::log_sanitized(pr, d->like_min) *
                     (f ? 1.0 / (double)mf->lag : 1.0 / (double)d->n_obs);
            }
          }
          w[j] = exp(plomrt::finish_loglik(ll, fl, M::N_TS) + lpr);
        }
      }
      sub0 += d->n_sub[n];
      const bool weigh = d->filter && n_nonan > 0;
      if (weigh) {
        double llike_n = 0.0, ess = 0.0;
        const int ok = weight(w, J, d->like_min, &llike_n, &ess, &Llike, &n_all_fail, select.data());
        // moments of the parameters used in this interval (weights normalised)
        for (int q = 0; q < Q; ++q) {
          double bt = 0.0, kn = 0.0, avg = 0.0, M2 = 0.0;
          for (int j = 0; j < J; ++j) {
            const double t = th[(size_t)j * Q + q];
            kn += 1.0;
            const double delta = t - avg;
            avg += delta / kn;
            M2 += delta * (t - avg);
            bt += w[j] * t;
          }
          double var = M2 / (kn - 1.0);
          if (!(var >= 0.0) || isinf(var)) var = 0.0;
          const size_t o = ((size_t)r * d->n_obs + n) * Q + q;
          bart[o] = bt;
          vt[o] = var + vt_add[(size_t)n * Q + q];
        }
        if (ok) {
          const double u = plomrt::resample_uniform(key, (uint32_t)n);
          systematic_sampling(w, J, (1.0 / (double)J) * u, select.data());
        }
        for (int j = 0; j < J; ++j) {
          const size_t s = (size_t)select[j];
          for (int k = 0; k < S; ++k) X[(size_t)j * S + k] = Xn[s * S + k];
          for (int q = 0; q < Q; ++q) {
            double t = th[s * Q + q];
            if (mf->estimated[q] && !fls_of(q)) {
              double z[1];
              plomrt::NormalGen<double>::fill<1>(key, (uint32_t)j, (uint32_t)(n + 1), (uint32_t)q, z,
                                                 (uint32_t)plomrt::STREAM_MUTATE);
              t += sd_mut[(size_t)n * Q + q] * z[0];
            }
            thn[(size_t)j * Q + q] = t;
          }
        }
        th.swap(thn);
      } else {
        X.swap(Xn);
      }
      // update_fixed_lag_smoothing at n == L (C/mif/mif.c:196-198, methods.c:370-392):
      // resampled components times the weights of the last weighting
      if (n == mf->lag && fls_out) {
        for (int q = 0; q < Q; ++q) {
          if (!fls_of(q)) continue;
          double acc = 0.0;
          for (int j = 0; j < J; ++j) acc += th[(size_t)j * Q + q] * w[j];
          fls_out[(size_t)r * Q + q] = acc;
        }
      }
    }
    loglik[r] = Llike;
    n_all_fail_out[r] = n_all_fail;
  }
  return 0;
}

// Systematic points exactly as the reference walks them (ran += inc).
void oracle_systematic_points_sequential(double U, int J, double* out) {
  const double inc = 1.0 / (double)J;
  double ran = U;
  for (int j = 0; j < J; ++j) {
    out[j] = ran;
    ran += inc;
  }
}

// The closed form shared with the device code, evaluated on the host.
int oracle_systematic_points_table(double U, int J, double* out) {
  static plomrt::SysSeg seg[plomrt::SYS_MAX_SEG];
  const int ns = plomrt::systematic_table(U, 1.0 / (double)J, J, seg, plomrt::SYS_MAX_SEG);
  if (ns < 0) return -1;
  for (int j = 0; j < J; ++j) out[j] = plomrt::systematic_point(seg, ns, j);
  return ns;
}

// One generated Euler step of one particle with injected normals (golden-vector checks).
int oracle_step(double* x, double t, double dt, int noises_off, const plomgpu_smc_desc* d, int sub,
                const double* normals) {
  HostEnv e;
  e.par_ = d->par_cac;
  e.cov_ = d->cov_cac ? d->cov_cac + (size_t)sub * M::N_COV_CAC * M::N_CAC : nullptr;
  e.coup_ = d->coupling;
  e.dgroup_ = d->drift_group;
  e.dng_ = d->drift_ngroups;
  e.dbt_ = d->drift_bt;
  e.dvol_ = d->drift_vol;
  HostState xs;
  xs.b = x;
  const int v = noises_off & 3;
  const bool drift = M::N_DRIFT > 0 && !(noises_off & PLOMGPU_NO_DRIFT);
#define ORACLE_STEP(VV, DD)              \
  {                                      \
    TableSource<VV> src;                 \
    src.p = normals;                     \
    M::step<VV, DD, double>(xs, t, dt, e, src); \
  }
  if (drift) {
    if (v == 0) ORACLE_STEP(0, true) else if (v == 1) ORACLE_STEP(1, true) else if (v == 2) ORACLE_STEP(2, true) else ORACLE_STEP(3, true)
  } else {
    if (v == 0) ORACLE_STEP(0, false) else if (v == 1) ORACLE_STEP(1, false) else if (v == 2) ORACLE_STEP(2, false) else ORACLE_STEP(3, false)
  }
#undef ORACLE_STEP
  return 0;
}

// Observation density of one series (golden-vector checks).
double oracle_obs_loglik(const double* x, const plomgpu_smc_desc* d, int n) { return log_likelihood(x, d, n); }

// Mean and variance of the observation model of series ts at time t (golden-vector checks).
void oracle_obs_moments(double x, int ts, double t, const plomgpu_smc_desc* d, double* mu, double* var) {
  HostObsEnv oe;
  oe.par_ts_ = d->par_ts;
  oe.cov_ts_ = d->cov_ts;
  *mu = M::obs_mean(x, ts, t, oe);
  *var = M::obs_var(x, ts, t, oe);
}

// One series' log-density term in both precisions (the single-precision
// version is that of FP32 particle states), with their floor counts.
void oracle_log_like_terms(int n, const double* y, const double* mu, const double* var, double like_min,
                           double* out64, double* out32, int* floor64, int* floor32) {
  for (int i = 0; i < n; ++i) {
    floor64[i] = 0;
    floor32[i] = 0;
    out64[i] = plomrt::log_like_term(y[i], mu[i], var[i], like_min, floor64 + i);
    out32[i] = plomrt::log_like_term_f(y[i], mu[i], var[i], like_min, floor32 + i);
  }
}

double oracle_like(double y, double mu, double var, double like_min) {
  return plomrt::disc_normal_like(y, mu, var, like_min);
}

void oracle_proj2obs(const double* x, double* obs) {
  HostState xs;
  xs.b = const_cast<double*>(x);
  M::proj2obs<double>(xs, obs);
}

}  // extern "C"
