// sm_100a kernels of one SMC filter for a generated model ``plomgen::Model``.
//
// Per observation interval n (model_builder/C/core/smc.c:235-305):
//   k_propagate  gather the ancestors' state (resample_X, smc.c:142-161),
//                reset incidences (prediction_util.c:25-33), run the Euler
//                substeps (f_prediction_sde_*, prediction_util.c:197-287),
//                map to observations (proj2obs) and write the log-weight
//                (get_log_likelihood, likelihood.c:56-70);
//   k_weight     failure test, log-sum-exp normalisation in FP64, ESS,
//                log-likelihood accumulation and the all-fail rule
//                (weight(), smc.c:27-83); the last block also lays out the
//                systematic points of the interval (smc.c:97-111);
//   k_scan       cumulative normalised weights in FP64 (smc.c:102-108);
//   k_search     ancestor of each particle slot (systematic_sampling,
//                smc.c:104-111) = first i with cum[i] >= point[j].
//
// State is struct-of-arrays X[w][j] in HBM (two generations), log-weights
// lw[j] in the state precision, cumulative weights and every reduction in
// FP64.  The particle loop of the reference (OpenMP / ZeroMQ workers,
// worker_inproc.c:71-80) is the kernel grid.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <type_traits>
#include "plom_rt.h"

namespace plomgpu {

using plomgen::Model;
typedef Model M;

// ------------------------------------------------------------------ state stores
template <class T, int S>
struct RegState {
  static constexpr bool DYNAMIC = false;
  T v[S];
  PLOM_HD T& operator[](int i) { return v[i]; }
  PLOM_HD const T& operator[](int i) const { return v[i]; }
};

template <class T, int STRIDE>
struct SmemState {
  static constexpr bool DYNAMIC = true;
  T* b;
  PLOM_HD T& operator[](int i) const { return b[i * STRIDE]; }
};

// ------------------------------------------------------------------ environments
template <class T>
struct ProcEnv {
  const T* par_;
  const T* cov_;
  const T* coup_;
  const int* dgroup_;
  const int* dng_;
  const plomrt::BackTransform* dbt_;
  const T* dvol_;
  __device__ __forceinline__ T par(int p, int cac) const { return par_[p * M::N_CAC + cac]; }
  __device__ __forceinline__ T cov(int k, int cac) const { return __ldg(cov_ + k * M::N_CAC + cac); }
  __device__ __forceinline__ T coupling(int a, int b) const { return coup_[a * M::N_CAC + b]; }
  __device__ __forceinline__ plomrt::V4<T> coupling4(int a, int b) const {
    return *reinterpret_cast<const plomrt::V4<T>*>(coup_ + a * M::N_CAC + b);
  }
  __device__ __forceinline__ int drift_group(int i, int cac) const { return __ldg(dgroup_ + i * M::N_CAC + cac); }
  __device__ __forceinline__ int drift_ngroups(int i) const { return __ldg(dng_ + i); }
  __device__ __forceinline__ T drift_vol(int i, int g) const { return __ldg(dvol_ + i * M::N_CAC + g); }
  __device__ __forceinline__ T drift_value(int i, int g, T xw) const {
    return plomrt::back_transform<T>(xw, dbt_[i * M::N_CAC + g]);
  }
};

struct ObsEnv {
  const double* par_ts_;
  const double* cov_ts_;
  __device__ __forceinline__ double par_ts(int p, int ts) const { return __ldg(par_ts_ + p * M::N_TS + ts); }
  __device__ __forceinline__ double cov_ts(int k, int ts) const { return __ldg(cov_ts_ + k * M::N_TS + ts); }
};

// ------------------------------------------------------------------ draw sources
template <class T, int V>
struct PhiloxDraws {
  static constexpr int PER_BLOCK = plomrt::NormalGen<T>::per_block();
  plomrt::PhiloxKey key;
  uint32_t j, n, sub;
  template <int N>
  __device__ __forceinline__ void normals(int cac, T* out) const {
    plomrt::NormalGen<T>::template fill<N>(key, j, n, (sub * (uint32_t)(M::N_CAC + 1) + (uint32_t)cac) << 12, out);
  }
  __device__ __forceinline__ T drift_normal(int i, int g) const {
    T z[1];
    plomrt::NormalGen<T>::template fill<1>(
        key, j, n, ((sub * (uint32_t)(M::N_CAC + 1) + (uint32_t)M::N_CAC) << 12) + (uint32_t)(i * M::N_CAC + g), z);
    return z[0];
  }
};

template <class T, int V>
struct TableDraws {
  static constexpr int PER_BLOCK = 1;
  const double* p;  // draws of this particle and substep
  template <int N>
  __device__ __forceinline__ void normals(int cac, T* out) const {
#pragma unroll
    for (int i = 0; i < N; ++i) out[i] = (T)__ldg(p + cac * N + i);
  }
  __device__ __forceinline__ T drift_normal(int i, int g) const {
    return (T)__ldg(p + M::N_CAC * M::draws_per_cac(V) + i * M::N_CAC + g);
  }
};

// ------------------------------------------------------------------ arguments
template <class T>
struct Tables {
  const T* par_cac;          // [N_PAR_PROC][N_CAC]
  const T* cov_cac;          // [sub_total][N_COV_CAC][N_CAC]
  const T* coupling;         // [N_CAC][N_CAC]
  const int* drift_group;    // [N_DRIFT][N_CAC]
  const int* drift_ngroups;  // [N_DRIFT]
  const plomrt::BackTransform* drift_bt;  // [N_DRIFT][N_CAC]
  const T* drift_vol;        // [N_DRIFT][N_CAC]
  const double* par_ts;      // [N_PAR_OBS][N_TS]
  const double* t_sub;       // [sub_total]
  double dt;
  double like_min;
  const uint64_t* seed;      // device copy of the Philox seed (updatable without re-capture)
  uint32_t filter_id;
  int J;
};

struct StepArgs {
  int n;                  // interval index
  int n_sub;              // substeps of the interval
  int sub0;               // index of its first substep in t_sub / cov_cac
  int weigh;              // 1: compute log-weights (row has data and filtering is on)
  double t_obs;           // t1
  const double* y;        // data row [N_TS]
  const double* cov_ts;   // [N_COV_TS][N_TS] at t1
  const void* X_prev;     // [OFF_INC][J] (T)
  void* X_next;           // [S][J] (T)
  const uint32_t* anc;    // ancestors of the previous interval, NULL = identity
  void* lw;               // [J] (T)
  const double* crn;      // CRN draws of this interval [J][n_sub][D] or NULL
  int crn_d;              // D
  double* x_hist;         // optional [S][J] double copy of the propagated particles
  int write_inc;          // 1: also store the incidence words in X_next
};

// ------------------------------------------------------------------ propagate
// shared-memory layout of k_propagate: coupling matrix, per-cac parameters
// (both read by every thread with the same address), then the state
// columns of the block's particles when the state does not fit registers
constexpr int pad4(int n) { return (n + 3) & ~3; }
constexpr int kSmemCoup = M::COUPLED ? pad4(M::N_CAC * M::N_CAC) : 0;
constexpr int kSmemPar = pad4(M::N_PAR_PROC * M::N_CAC);

template <class T, bool SMEM, int BT>
constexpr size_t propagate_smem_bytes() {
  return (size_t)(kSmemCoup + kSmemPar) * sizeof(T) + (SMEM ? (size_t)M::S * BT * sizeof(T) : 0);
}

template <class T, int V, bool DRIFT, bool CRN, bool SMEM, int BT>
__global__ void __launch_bounds__(BT) k_propagate(const Tables<T> tb, const StepArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* s_coup = reinterpret_cast<T*>(smem_raw);
  T* s_par = s_coup + kSmemCoup;
  T* s_state = s_par + kSmemPar;
  if constexpr (M::COUPLED) {
    for (int i = threadIdx.x; i < M::N_CAC * M::N_CAC; i += BT) s_coup[i] = tb.coupling[i];
  }
  for (int i = threadIdx.x; i < M::N_PAR_PROC * M::N_CAC; i += BT) s_par[i] = tb.par_cac[i];
  __syncthreads();
  const int J = tb.J;
  const int j = blockIdx.x * BT + threadIdx.x;
  if (j >= J) return;
  const uint32_t src = a.anc ? __ldg(a.anc + j) : (uint32_t)j;
  const T* __restrict__ Xp = (const T*)a.X_prev;
  T* __restrict__ Xn = (T*)a.X_next;

  typedef typename std::conditional<SMEM, SmemState<T, BT>, RegState<T, M::S>>::type Store;
  Store x;
  if constexpr (SMEM) {
    x.b = s_state + threadIdx.x;
  }
#pragma unroll
  for (int w = 0; w < M::OFF_INC; ++w) x[w] = Xp[(size_t)w * J + src];
#pragma unroll
  for (int w = M::OFF_INC; w < M::S; ++w) x[w] = T(0);  // reset_inc

  ProcEnv<T> e;
  e.par_ = s_par;
  e.coup_ = s_coup;
  e.dgroup_ = tb.drift_group;
  e.dng_ = tb.drift_ngroups;
  e.dbt_ = tb.drift_bt;
  e.dvol_ = tb.drift_vol;
  const T dt = (T)tb.dt;
  const plomrt::PhiloxKey key = plomrt::make_key(CRN ? 0ull : *tb.seed, tb.filter_id);

  for (int k = 0; k < a.n_sub; ++k) {
    const int sub = a.sub0 + k;
    e.cov_ = tb.cov_cac + (size_t)sub * M::N_COV_CAC * M::N_CAC;
    const T t = (T)__ldg(tb.t_sub + sub);
    if constexpr (CRN) {
      TableDraws<T, V> d;
      d.p = a.crn + ((size_t)j * a.n_sub + k) * a.crn_d;
      M::template step<V, DRIFT, T>(x, t, dt, e, d);
    } else {
      PhiloxDraws<T, V> d;
      d.key = key;
      d.j = (uint32_t)j;
      d.n = (uint32_t)a.n;
      d.sub = (uint32_t)k;
      M::template step<V, DRIFT, T>(x, t, dt, e, d);
    }
  }

#pragma unroll
  for (int w = 0; w < M::S; ++w) {
    if (w < M::OFF_INC || a.write_inc) Xn[(size_t)w * J + j] = x[w];
  }
  if (a.x_hist) {
#pragma unroll
    for (int w = 0; w < M::S; ++w) a.x_hist[(size_t)w * J + j] = (double)x[w];
  }

  if (a.weigh) {
    double obs[M::N_TS];
    M::template proj2obs<T>(x, obs);
    ObsEnv oe;
    oe.par_ts_ = tb.par_ts;
    oe.cov_ts_ = a.cov_ts;
    double ll = 0.0;
#pragma unroll
    for (int ts = 0; ts < M::N_TS; ++ts) {
      const double y = __ldg(a.y + ts);
      if (isnan(y)) continue;
      const double mu = M::obs_mean(obs[ts], ts, a.t_obs, oe);
      const double var = M::obs_var(obs[ts], ts, a.t_obs, oe);
      ll += log(plomrt::disc_normal_like(y, mu, var, tb.like_min));
    }
    ((T*)a.lw)[j] = (T)ll;
  }
}

// ------------------------------------------------------------------ weights
struct LseAcc {
  double m;   // running max of the surviving log-weights
  double s1;  // sum exp(l - m)
  double s2;  // sum exp(2 (l - m))
  int nfail;
};

__device__ __forceinline__ LseAcc lse_merge(LseAcc a, LseAcc b) {
  LseAcc r;
  r.nfail = a.nfail + b.nfail;
  if (b.m > a.m) { LseAcc t = a; a = b; b = t; }
  r.m = a.m;
  if (b.s1 > 0.0) {
    const double f = exp(b.m - a.m);
    r.s1 = a.s1 + b.s1 * f;
    r.s2 = a.s2 + b.s2 * f * f;
  } else {
    r.s1 = a.s1;
    r.s2 = a.s2;
  }
  return r;
}

__device__ __forceinline__ LseAcc lse_shfl(LseAcc a, int off) {
  LseAcc b;
  b.m = __shfl_xor_sync(0xffffffffu, a.m, off);
  b.s1 = __shfl_xor_sync(0xffffffffu, a.s1, off);
  b.s2 = __shfl_xor_sync(0xffffffffu, a.s2, off);
  b.nfail = __shfl_xor_sync(0xffffffffu, a.nfail, off);
  return lse_merge(a, b);
}

struct TileStatus {
  double agg;
  int flag;
  int pad;
};

// Per-filter device state of the current interval.
struct StepState {
  double m, s1, s2;
  int all_fail;
  int nseg;
  double U;
  plomrt::SysSeg seg[plomrt::SYS_MAX_SEG];
};

struct FilterAcc {
  double loglik;
  int n_all_fail;
  int error;        // bit 0: scan wait ran out; bit 1: systematic table overflow
  unsigned ticket;  // block ticket of k_weight
  unsigned tile_ticket;
};

enum { ERR_SCAN_WAIT = 1, ERR_SYS_TABLE = 2 };

template <class T>
__device__ __forceinline__ bool weight_fails(T l, double thresh) {
  // weight() (smc.c:44): the particle fails if exp(loglik) <= LIKE_MIN^N_TS
  return !(exp((double)l) > thresh);
}

template <class T, int BT>
__global__ void __launch_bounds__(BT) k_weight(const T* __restrict__ lw, int J, double thresh, double log_like_min,
                                               LseAcc* part, StepState* st, FilterAcc* acc, TileStatus* tstat,
                                               int ntiles, int n, double U_crn, const uint64_t* seed, uint32_t filter_id,
                                               double* llike_out, double* ess_out) {
  __shared__ LseAcc sh[BT / 32];
  __shared__ bool last;
  LseAcc a = {-INFINITY, 0.0, 0.0, 0};
  for (int i = blockIdx.x * BT + threadIdx.x; i < J; i += gridDim.x * BT) {
    const T l = lw[i];
    if (weight_fails(l, thresh)) {
      a.nfail += 1;
    } else {
      LseAcc b = {(double)l, 1.0, 1.0, 0};
      a = lse_merge(a, b);
    }
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) a = lse_shfl(a, off);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = a;
  __syncthreads();
  if (threadIdx.x < 32) {
    a = (threadIdx.x < BT / 32) ? sh[threadIdx.x] : LseAcc{-INFINITY, 0.0, 0.0, 0};
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) a = lse_shfl(a, off);
    if (threadIdx.x == 0) {
      part[blockIdx.x] = a;
      __threadfence();
      const unsigned t = atomicAdd(&acc->ticket, 1u);
      last = (t == gridDim.x - 1);
    }
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  // the last block folds the partials in a fixed order
  a = LseAcc{-INFINITY, 0.0, 0.0, 0};
  for (int b = threadIdx.x; b < (int)gridDim.x; b += BT) {
    volatile LseAcc* p = part + b;
    LseAcc v = {p->m, p->s1, p->s2, p->nfail};
    a = lse_merge(a, v);
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) a = lse_shfl(a, off);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = a;
  __syncthreads();
  for (int i = threadIdx.x; i < ntiles; i += BT) tstat[i].flag = 0;
  if (threadIdx.x < 32) {
    a = (threadIdx.x < BT / 32) ? sh[threadIdx.x] : LseAcc{-INFINITY, 0.0, 0.0, 0};
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) a = lse_shfl(a, off);
    if (threadIdx.x == 0) {
      acc->ticket = 0u;
      acc->tile_ticket = 0u;
      double llike, ess;
      int all_fail = (a.nfail == J);
      if (all_fail) {
        // every particle failed: equal weights, identity ancestors (smc.c:55-69)
        llike = log_like_min * (double)M::N_TS;
        ess = 0.0;
        acc->n_all_fail += 1;
      } else {
        llike = a.m + log(a.s1 / (double)J);
        ess = (a.s1 * a.s1) / a.s2;
      }
      acc->loglik += llike;
      st->m = a.m;
      st->s1 = a.s1;
      st->s2 = a.s2;
      st->all_fail = all_fail;
      if (llike_out) llike_out[n] = llike;
      if (ess_out) ess_out[n] = ess;
      const double inc = 1.0 / (double)J;
      const double u = (U_crn >= 0.0) ? U_crn : plomrt::resample_uniform(plomrt::make_key(*seed, filter_id), (uint32_t)n);
      const double U = inc * u;  // gsl_ran_flat(0, inc) = 0*(1-u) + inc*u
      st->U = U;
      int ns = plomrt::systematic_table(U, inc, J, st->seg, plomrt::SYS_MAX_SEG);
      if (ns < 0) {
        acc->error |= ERR_SYS_TABLE;
        ns = 0;
      }
      st->nseg = ns;
    }
  }
}

// ------------------------------------------------------------------ cumulative weights
// Tiles are claimed in launch order through a ticket, publish their
// aggregate, and take their exclusive prefix as the sum of all earlier
// aggregates in a fixed order (lane l adds tiles l, l+32, ... then a fixed
// butterfly), so the result does not depend on timing.  A tile only waits for
// tiles claimed before it; every wait is bounded.
template <class T, int BT, int IPT>
__global__ void __launch_bounds__(BT) k_scan(const T* __restrict__ lw, int J, double thresh, const StepState* st,
                                             TileStatus* tstat, FilterAcc* acc, double* __restrict__ C) {
  constexpr int TILE = BT * IPT;
  __shared__ double sv[TILE];
  __shared__ double swarp[BT / 32];
  __shared__ int s_tile;
  __shared__ double s_prefix;
  if (st->all_fail) return;
  if (threadIdx.x == 0) s_tile = (int)atomicAdd(&acc->tile_ticket, 1u);
  __syncthreads();
  const int tile = s_tile;
  const int base = tile * TILE;
  const double m = st->m, s1 = st->s1;
  for (int k = threadIdx.x; k < TILE; k += BT) {
    const int i = base + k;
    double p = 0.0;
    if (i < J) {
      const T l = lw[i];
      p = weight_fails(l, thresh) ? 0.0 : exp((double)l - m) / s1;
    }
    sv[k] = p;
  }
  __syncthreads();
  // thread-sequential inclusive sums of IPT consecutive items
  double run = 0.0;
  double loc[IPT];
#pragma unroll
  for (int k = 0; k < IPT; ++k) {
    run += sv[threadIdx.x * IPT + k];
    loc[k] = run;
  }
  // block exclusive scan of the thread totals
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  double v = run;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const double o = __shfl_up_sync(0xffffffffu, v, off);
    if (lane >= off) v += o;
  }
  if (lane == 31) swarp[warp] = v;
  __syncthreads();
  if (warp == 0) {
    double w = (lane < BT / 32) ? swarp[lane] : 0.0;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const double o = __shfl_up_sync(0xffffffffu, w, off);
      if (lane >= off) w += o;
    }
    if (lane < BT / 32) swarp[lane] = w;  // inclusive warp totals
  }
  __syncthreads();
  const double warp_excl = (warp > 0) ? swarp[warp - 1] : 0.0;
  const double thread_excl = warp_excl + (v - run);
  const double tile_total = swarp[BT / 32 - 1];
  if (threadIdx.x == 0) {
    volatile TileStatus* ts = tstat + tile;
    ts->agg = tile_total;
    __threadfence();
    ts->flag = 1;
  }
  // exclusive prefix from earlier aggregates, fixed order
  if (warp == 0) {
    double s = 0.0;
    bool timeout = false;
    for (int k = lane; k < tile; k += 32) {
      volatile TileStatus* ts = tstat + k;
      int spins = 0;
      while (ts->flag == 0) {
        if (++spins > (1 << 22)) { timeout = true; break; }
        __nanosleep(64);
      }
      __threadfence();
      s += ts->agg;
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
    if (__any_sync(0xffffffffu, timeout) && lane == 0) atomicOr(&acc->error, (int)ERR_SCAN_WAIT);
    if (lane == 0) s_prefix = s;
  }
  __syncthreads();
  const double prefix = s_prefix + thread_excl;
#pragma unroll
  for (int k = 0; k < IPT; ++k) {
    const int i = base + threadIdx.x * IPT + k;
    if (i < J) C[i] = prefix + loc[k];
  }
}

// ------------------------------------------------------------------ ancestors
template <int BT>
__global__ void __launch_bounds__(BT) k_search(const double* __restrict__ C, int J, const StepState* st,
                                               uint32_t* __restrict__ anc, uint32_t* __restrict__ anc_hist) {
  __shared__ plomrt::SysSeg seg[plomrt::SYS_MAX_SEG];
  __shared__ int s_ns, s_fail;
  if (threadIdx.x == 0) {
    s_ns = st->nseg;
    s_fail = st->all_fail;
  }
  __syncthreads();
  const int ns = s_ns;
  for (int i = threadIdx.x; i < ns; i += BT) seg[i] = st->seg[i];
  __syncthreads();
  const int j = blockIdx.x * BT + threadIdx.x;
  if (j >= J) return;
  uint32_t r;
  if (s_fail || ns == 0) {
    r = (uint32_t)j;
  } else {
    const double ran = plomrt::systematic_point(seg, ns, j);
    int lo = 0, hi = J - 1;
    while (lo < hi) {  // first i with !(ran > C[i])  (smc.c:105-108)
      const int mid = (lo + hi) >> 1;
      if (ran > __ldg(C + mid)) lo = mid + 1; else hi = mid;
    }
    r = (uint32_t)lo;
  }
  anc[j] = r;
  if (anc_hist) anc_hist[j] = r;
}

// ------------------------------------------------------------------ helpers
template <class T>
__global__ void k_init_state(const double* __restrict__ x0, int J, T* __restrict__ X) {
  const size_t total = (size_t)M::OFF_INC * J;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
    const int w = (int)(i / J);
    X[i] = (T)x0[w];
  }
}

template <class T>
__global__ void k_gather_final(const T* __restrict__ X, const uint32_t* __restrict__ anc, int J, int nw,
                               double* __restrict__ out) {
  const size_t total = (size_t)nw * J;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
    const int w = (int)(i / J);
    const int j = (int)(i - (size_t)w * J);
    const uint32_t s = anc ? anc[j] : (uint32_t)j;
    out[i] = (double)X[(size_t)w * J + s];
  }
}

__global__ void k_identity(uint32_t* __restrict__ out, int J) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < J; j += gridDim.x * blockDim.x) out[j] = (uint32_t)j;
}

__global__ void k_reset_acc(FilterAcc* acc) {
  acc->loglik = 0.0;
  acc->n_all_fail = 0;
  acc->error = 0;
  acc->ticket = 0u;
  acc->tile_ticket = 0u;
}

__global__ void k_sys_points(double U, int J, double* out, int* err) {
  __shared__ plomrt::SysSeg seg[plomrt::SYS_MAX_SEG];
  __shared__ int s_ns;
  if (threadIdx.x == 0) s_ns = plomrt::systematic_table(U, 1.0 / (double)J, J, seg, plomrt::SYS_MAX_SEG);
  __syncthreads();
  if (s_ns < 0) {
    if (threadIdx.x == 0) *err = 1;
    return;
  }
  for (int j = threadIdx.x; j < J; j += blockDim.x) out[j] = plomrt::systematic_point(seg, s_ns, j);
}

}  // namespace plomgpu
