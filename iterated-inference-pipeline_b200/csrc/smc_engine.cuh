// sm_100a kernels of one SMC filter for a generated model ``plomgen::Model``.
//
// Per observation interval n (model_builder/C/core/smc.c:235-305):
//   k_propagate  gather the ancestors' state (resample_X, smc.c:142-161),
//                reset incidences (prediction_util.c:25-33), run the Euler
//                substeps (f_prediction_sde_*, prediction_util.c:197-287),
//                map to observations (proj2obs) and write the log-weight
//                (get_log_likelihood, likelihood.c:56-70);
//   k_weight_tiles    failure test, log-sum-exp normalisation in FP64, ESS,
//                     log-likelihood accumulation and the all-fail rule
//                     (weight(), smc.c:27-83); the last block also lays out
//                     the systematic points of the interval (smc.c:97-111);
//   k_resample_tiles  cumulative normalised weights in FP64 (smc.c:102-108)
//                     and the ancestor of each particle slot
//                     (systematic_sampling, smc.c:104-111) = first i with
//                     cum[i] >= point[j];
//   k_resample_heavy  the same for tiles that took many points.
//
// State is struct-of-arrays X[w][j] in HBM (two generations), log-weights
// lw[j] in the state precision, their exponentials, cumulative weights and
// every sum in FP64.  The particle loop of the reference (OpenMP / ZeroMQ workers,
// worker_inproc.c:71-80) is the kernel grid.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <type_traits>
#include "plom_rt.h"
#include "ode_rkf45.h"

namespace plomgpu {

using plomgen::Model;
typedef Model M;

// Launched with programmatic stream serialisation (launch_chained on the
// host), a kernel may start while the previous kernel of the stream still
// runs; it waits here, before it reads anything that kernel writes.  A
// kernel launched without it passes straight through.
__device__ __forceinline__ void wait_for_previous_kernel() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

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

// Incidence sums of a shared-memory particle in the words after its state
// (S .. S + N_TS_INC_UNIQUE - 1 of its column): a term goes to its series by
// an indexed shared-memory add instead of a compare chain over registers.
template <class T, int STRIDE>
struct SmemIncAcc {
  T* b;
  PLOM_HD explicit SmemIncAcc(SmemState<T, STRIDE>& x) : b(x.b + (size_t)M::S * STRIDE) {}
  PLOM_HD void zero() {
#pragma unroll
    for (int w = 0; w < M::N_TS_INC_UNIQUE; ++w) b[w * STRIDE] = T(0);
  }
  PLOM_HD void add(int w, T d) { b[w * STRIDE] += d; }
  PLOM_HD T get(int w) const { return b[w * STRIDE]; }
};

// the propagate kernel's shared memory: coupling matrix, per-cac parameters
// (both read by every thread with the same address), then the state columns
// of the block's particles when the state does not fit registers, followed by
// their incidence sums when those words keep the blocks per SM (FP32 only:
// FP64 states run the parity modes, with the register sums)
constexpr int pad4(int n) { return (n + 3) & ~3; }
constexpr int kSmemCoup = M::COUPLED ? pad4(M::N_CAC * M::N_CAC) : 0;
constexpr int kSmemPar = pad4(M::N_PAR_PROC * M::N_CAC);

template <class T, int BT>
constexpr bool inc_in_smem() {
#if defined(PLOM_INC_REGS)
  return false;
#else
  constexpr size_t sm = 228 * 1024, per_block_resv = 1024, block_max = 227 * 1024;
  constexpr size_t base = ((size_t)kSmemCoup + kSmemPar + (size_t)M::S * BT) * sizeof(T);
  constexpr size_t ext = base + (size_t)M::N_TS_INC_UNIQUE * BT * sizeof(T);
  return sizeof(T) == 4 && M::N_TS_INC_UNIQUE > 0 && ext <= block_max &&
         sm / (ext + per_block_resv) >= sm / (base + per_block_resv);
#endif
}

}  // namespace plomgpu

namespace plomrt {
template <class T, int STRIDE, int N>
struct IncAccFor<plomgpu::SmemState<T, STRIDE>, T, N> {
  typedef typename std::conditional<plomgpu::inc_in_smem<T, STRIDE>(), plomgpu::SmemIncAcc<T, STRIDE>,
                                    RegIncAcc<T, N>>::type type;
};
}  // namespace plomrt

namespace plomgpu {

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
  __device__ __forceinline__ double par_ts(int p, int ts) const { return par_ts_[p * M::N_TS + ts]; }
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

// Common random numbers, one cac at a time: from an injected table, or,
// without a table (paired draws), the normals that the FP64 filter of the
// same seed draws for this (particle, interval, substep, cac), rounded to T.
// Paired draws let an FP32 filter consume exactly the FP64 filter's normals,
// so that the difference of their log-likelihoods is the precision error.
template <class T, int V>
struct TableDraws {
  static constexpr int PER_BLOCK = 1;
  const double* p;  // draws of this particle and substep, NULL: paired Philox draws
  plomrt::PhiloxKey key;
  uint32_t j, n, sub;
  template <int N>
  __device__ __forceinline__ void normals(int cac, T* out) const {
    if (p) {
#pragma unroll
      for (int i = 0; i < N; ++i) out[i] = (T)__ldg(p + cac * N + i);
      return;
    }
    // the FP64 step draws groups of G64 cacs from consecutive Philox blocks
    // (whole blocks of 2 normals), the cacs after the last whole group one by one
    constexpr int G64 = M::draw_group(N, plomrt::NormalGen<double>::per_block());
    constexpr int NMAIN64 = M::N_CAC - (M::N_CAC % G64);
    const int c0 = (cac < NMAIN64) ? cac - cac % G64 : cac;
    const uint32_t blk0 = (sub * (uint32_t)(M::N_CAC + 1) + (uint32_t)c0) << 12;
    const int i0 = (cac - c0) * N;
    double z[2] = {0.0, 0.0};
    int have = -1;
    for (int q = 0; q < N; ++q) {
      const int i = i0 + q;
      if ((i >> 1) != have) {
        have = i >> 1;
        plomrt::NormalGen<double>::block(key, j, n, blk0 + (uint32_t)have, (uint32_t)plomrt::STREAM_PROCESS, &z[0],
                                         &z[1]);
      }
      out[q] = (T)z[i & 1];
    }
  }
  __device__ __forceinline__ T drift_normal(int i, int g) const {
    if (p) return (T)__ldg(p + M::N_CAC * M::draws_per_cac(V) + i * M::N_CAC + g);
    double z0, z1;
    plomrt::NormalGen<double>::block(
        key, j, n, ((sub * (uint32_t)(M::N_CAC + 1) + (uint32_t)M::N_CAC) << 12) + (uint32_t)(i * M::N_CAC + g),
        (uint32_t)plomrt::STREAM_PROCESS, &z0, &z1);
    return (T)z0;
  }
};

// ------------------------------------------------------------------ arguments
constexpr int kMaxTheta = 16;

// Iterated filtering: fixed-lag smoothing and the --prior patch
// (update_fixed_lag_smoothing / patch_likelihood_prior,
// model_builder/C/mif/methods.c:370-392,469-520).
struct MifTables {
  unsigned fls_mask;   // components fitted by fixed-lag smoothing
  int lag;             // L
  int prior;           // 1: --prior patch
  double inv_nobs;     // exponent of the random-walk components' prior
  double inv_lag;      // exponent of the fixed-lag components' prior while n < L
  int prior_kind[kMaxTheta];
  double prior_lo[kMaxTheta];
  double prior_hi[kMaxTheta];
  plomrt::BackTransform prior_finv[kMaxTheta];
};

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
  uint32_t filter_id;        // Philox key of run r uses filter_id + r
  int J;                     // particles per run
  int R;                     // runs advanced in lock step (1 for a plain filter)
  // per-particle parameters (iterated filtering); unused when the kernel has MIF = false
  int Q;                                 // theta components (<= kMaxTheta)
  unsigned est_mask;                     // components perturbed by the random walk
  const plomrt::BackTransform* theta_bt; // [Q] transformed -> natural
  const int* proc_slot;                  // [N_PAR_PROC] component of each process parameter, -1: table, -2: per cac
  const int* obs_slot;                   // [N_PAR_OBS] component of each observation parameter, -1: table, -2: per series
  const int* proc_cslot;                 // [N_PAR_PROC][N_CAC] components of the per-cac parameters
  const int* obs_tslot;                  // [N_PAR_OBS][N_TS] components of the per-series parameters
  unsigned mut_mask;                     // components perturbed by the random walk (estimated, not fixed-lag)
  const int* vol_slot;                   // [N_DRIFT][N_CAC] component of each drift volatility, NULL: table
  const MifTables* mx;                   // fixed-lag smoothing / prior patch, NULL: off
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
  const void* theta_prev; // [Q][R*J] (T) per-particle transformed parameters, MIF only
  void* theta_next;       // [Q][R*J] (T)
  const double* sd_mut;   // [Q] random-walk sd applied when gathering from ancestors, NULL: none
  const double* x0_rep;   // [S] initial particle read by every particle instead of X_prev, NULL: X_prev
};

// environments with per-particle parameters (iterated filtering)
// uni: parameters taken from the particle; with MULTI, multi marks those of
// them whose component depends on the population / series (one per group),
// looked up in cslot and selected from the particle's natural values natq
// (the instantiation without MULTI keeps the registers of the plain case).
template <class T, bool MULTI>
struct MifProcEnv : ProcEnv<T> {
  T parp[M::N_PAR_PROC > 0 ? M::N_PAR_PROC : 1];
  unsigned uni, multi;
  const int* cslot;  // [N_PAR_PROC][N_CAC]
  const int* vslot;  // [N_DRIFT][N_CAC] volatility components (MULTI only), NULL: table
  T natq[MULTI ? kMaxTheta : 1];
  // the volatility of drift i, group g, from the particle's parameters when
  // it is a component (back_transform_theta2par per particle feeds
  // compute_drift, model_builder/C/core/drift.c:27-41)
  __device__ __forceinline__ T drift_vol(int i, int g) const {
    if constexpr (MULTI) {
      if (vslot) {
        const int q = __ldg(vslot + i * M::N_CAC + g);
        if (q >= 0) {
          T v = T(0);
#pragma unroll
          for (int qq = 0; qq < kMaxTheta; ++qq)
            if (qq == q) v = natq[qq];
          return v;
        }
      }
    }
    return ProcEnv<T>::drift_vol(i, g);
  }
  __device__ __forceinline__ T par(int p, int cac) const {
    if (!((uni >> p) & 1u)) return this->par_[p * M::N_CAC + cac];
    if constexpr (!MULTI) return parp[p];
    if (!((multi >> p) & 1u)) return parp[p];
    const int q = __ldg(cslot + p * M::N_CAC + cac);
    T v = T(0);
#pragma unroll
    for (int qq = 0; qq < kMaxTheta; ++qq)
      if (qq == q) v = natq[qq];
    return v;
  }
};

template <bool MULTI>
struct MifObsEnv : ObsEnv {
  double obsp[M::N_PAR_OBS > 0 ? M::N_PAR_OBS : 1];
  unsigned uni, multi;
  const int* tslot;  // [N_PAR_OBS][N_TS]
  double natq[MULTI ? kMaxTheta : 1];
  __device__ __forceinline__ double par_ts(int p, int ts) const {
    if (!((uni >> p) & 1u)) return par_ts_[p * M::N_TS + ts];
    if constexpr (!MULTI) return obsp[p];
    if (!((multi >> p) & 1u)) return obsp[p];
    const int q = __ldg(tslot + p * M::N_TS + ts);
    double v = 0.0;
#pragma unroll
    for (int qq = 0; qq < kMaxTheta; ++qq)
      if (qq == q) v = natq[qq];
    return v;
  }
};

// ------------------------------------------------------------------ propagate
template <class T, bool SMEM, int BT>
constexpr size_t propagate_smem_bytes() {
  return (size_t)(kSmemCoup + kSmemPar) * sizeof(T) +
         (SMEM ? ((size_t)M::S + (inc_in_smem<T, BT>() ? M::N_TS_INC_UNIQUE : 0)) * BT * sizeof(T) : 0);
}

// PSR: the Poisson-system step (M::step_psr, the reference's default "psr"
// implementation) instead of Euler-Maruyama; bit 1 of V turns its white
// noise off.
// The propagate block's shared tables: the coupling matrix (when
// `coupling`) and the per-cac parameters, read by every thread at the same
// address.  Ends with a block barrier.
template <class T, int BT>
__device__ __forceinline__ void propagate_tables(const Tables<T>& tb, unsigned char* smem_raw, bool coupling) {
  T* s_coup = reinterpret_cast<T*>(smem_raw);
  T* s_par = s_coup + kSmemCoup;
  if constexpr (M::COUPLED) {
    if (coupling)
      for (int i = threadIdx.x; i < M::N_CAC * M::N_CAC; i += BT) s_coup[i] = tb.coupling[i];
  }
  for (int i = threadIdx.x; i < M::N_PAR_PROC * M::N_CAC; i += BT) s_par[i] = tb.par_cac[i];
  __syncthreads();
}

// Particle g (of all runs) over one interval: gather, substeps, store,
// log-weight.  Returns the log-weight written (NaN when the interval is not
// weighted).  The shared tables must be loaded; the particle's shared-memory
// state column is the calling thread's.
template <class T, int V, bool DRIFT, bool CRN, bool SMEM, bool MIF, int BT, bool PSR, bool MULTI>
__device__ __forceinline__ double propagate_particle(const Tables<T>& tb, const StepArgs& a, size_t g,
                                                     unsigned char* smem_raw) {
  T* s_coup = reinterpret_cast<T*>(smem_raw);
  T* s_par = s_coup + kSmemCoup;
  T* s_state = s_par + kSmemPar;
  const int J = tb.J;
  const size_t RJ = (size_t)tb.R * J;
  const int r = (int)(g / J);
  const int j = (int)(g - (size_t)r * J);                  // slot within its run
  const size_t src = (size_t)r * J + (a.anc ? __ldg(a.anc + g) : (uint32_t)j);
  const T* __restrict__ Xp = (const T*)a.X_prev;
  T* __restrict__ Xn = (T*)a.X_next;

  typedef typename std::conditional<SMEM, SmemState<T, BT>, RegState<T, M::S>>::type Store;
  Store x;
  if constexpr (SMEM) {
    x.b = s_state + threadIdx.x;
  }
  if (a.x0_rep) {
    // the initial particle, replicated (build_D_J_p_X / replicate_J_p_X_0, smc.c:167-176)
#pragma unroll
    for (int w = 0; w < M::OFF_INC; ++w) x[w] = (T)__ldg(a.x0_rep + w);
  } else {
#pragma unroll
    for (int w = 0; w < M::OFF_INC; ++w) x[w] = Xp[(size_t)w * RJ + src];
  }
#pragma unroll
  for (int w = M::OFF_INC; w < M::S; ++w) x[w] = T(0);  // reset_inc

  typedef typename std::conditional<MIF, MifProcEnv<T, MULTI>, ProcEnv<T>>::type PEnv;
  PEnv e;
  e.par_ = s_par;
  e.coup_ = s_coup;
  e.dgroup_ = tb.drift_group;
  e.dng_ = tb.drift_ngroups;
  e.dbt_ = tb.drift_bt;
  e.dvol_ = tb.drift_vol;
  const T dt = (T)tb.dt;
  const plomrt::PhiloxKey key = plomrt::make_key(*tb.seed, tb.filter_id + (uint32_t)r);

  typedef typename std::conditional<MIF, MifObsEnv<MULTI>, ObsEnv>::type OEnv;
  OEnv oe;
  oe.par_ts_ = tb.par_ts;
  oe.cov_ts_ = a.cov_ts;
  if constexpr (MIF) {
    // gather this particle's parameters from its ancestor, perturb them
    // (resample_and_mut_theta_mif, model_builder/C/mif/methods.c:261-367), keep
    // them for the next interval and back-transform them
    // (back_transform_theta2par per particle, C/mif/mif.c:142-144)
    const T* __restrict__ thp = (const T*)a.theta_prev;
    T* __restrict__ thn = (T*)a.theta_next;
    double nat[kMaxTheta];
#pragma unroll
    for (int q = 0; q < kMaxTheta; ++q) {
      nat[q] = 0.0;
      if (q < tb.Q) {
        T v = thp[(size_t)q * RJ + src];
        if (a.sd_mut && ((tb.mut_mask >> q) & 1u)) {
          T z[1];
          plomrt::NormalGen<T>::template fill<1>(key, (uint32_t)j, (uint32_t)a.n, (uint32_t)q, z,
                                                 (uint32_t)plomrt::STREAM_MUTATE);
          v += (T)__ldg(a.sd_mut + q) * z[0];
        }
        thn[(size_t)q * RJ + g] = v;
        nat[q] = (double)plomrt::back_transform<T>(v, tb.theta_bt[q]);
      }
    }
    e.uni = 0u;
    e.multi = 0u;
    e.cslot = tb.proc_cslot;
    e.vslot = tb.vol_slot;
    if constexpr (MULTI) {
#pragma unroll
      for (int q = 0; q < kMaxTheta; ++q) e.natq[q] = (T)nat[q];
    }
#pragma unroll
    for (int k = 0; k < M::N_PAR_PROC; ++k) {
      const int slot = __ldg(tb.proc_slot + k);
      T v = T(0);
#pragma unroll
      for (int q = 0; q < kMaxTheta; ++q)
        if (q == slot) v = (T)nat[q];
      e.parp[k] = v;
      if (slot >= 0 || slot == -2) e.uni |= 1u << k;
      if (slot == -2) e.multi |= 1u << k;
    }
    oe.uni = 0u;
    oe.multi = 0u;
    oe.tslot = tb.obs_tslot;
    if constexpr (MULTI) {
#pragma unroll
      for (int q = 0; q < kMaxTheta; ++q) oe.natq[q] = nat[q];
    }
#pragma unroll
    for (int k = 0; k < M::N_PAR_OBS; ++k) {
      const int slot = __ldg(tb.obs_slot + k);
      double v = 0.0;
#pragma unroll
      for (int q = 0; q < kMaxTheta; ++q)
        if (q == slot) v = nat[q];
      oe.obsp[k] = v;
      if (slot >= 0 || slot == -2) oe.uni |= 1u << k;
      if (slot == -2) oe.multi |= 1u << k;
    }
  }

  for (int k = 0; k < a.n_sub; ++k) {
    const int sub = a.sub0 + k;
    e.cov_ = tb.cov_cac + (size_t)sub * M::N_COV_CAC * M::N_CAC;
    const T t = (T)__ldg(tb.t_sub + sub);
    if constexpr (PSR) {
      PhiloxDraws<T, V> d;
      d.key = key;
      d.j = (uint32_t)j;
      d.n = (uint32_t)a.n;
      d.sub = (uint32_t)k;
      M::template step_psr<DRIFT, (V & 2) != 0, T>(x, t, dt, e, key, (uint32_t)j, (uint32_t)a.n, (uint32_t)k, d);
    } else if constexpr (CRN) {
      TableDraws<T, V> d;
      d.p = a.crn ? a.crn + ((size_t)g * a.n_sub + k) * a.crn_d : nullptr;
      d.key = key;
      d.j = (uint32_t)j;
      d.n = (uint32_t)a.n;
      d.sub = (uint32_t)k;
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
    if (w < M::OFF_INC || a.write_inc) Xn[(size_t)w * RJ + g] = x[w];
  }
  if (a.x_hist) {
#pragma unroll
    for (int w = 0; w < M::S; ++w) a.x_hist[(size_t)w * RJ + g] = (double)x[w];
  }

  if (a.weigh) {
    double obs[M::N_TS];
    M::template proj2obs<T>(x, obs);
    double ll = 0.0;
    int fl = 0;
#pragma unroll
    for (int ts = 0; ts < M::N_TS; ++ts) {
      const double y = __ldg(a.y + ts);
      if (isnan(y)) continue;
      const double mu = M::obs_mean(obs[ts], ts, a.t_obs, oe);
      const double var = M::obs_var(obs[ts], ts, a.t_obs, oe);
      ll += plomrt::log_like_term_p<T>(y, mu, var, tb.like_min, &fl);
    }
    double lpr = 0.0;
    if constexpr (MIF) {
      // --prior: weight x prior^(1/n_obs) for the random-walk components,
      // prior^(1/L) for the fixed-lag ones while n < L (patch_likelihood_prior,
      // model_builder/C/mif/methods.c:469-520), on the parameters of this interval
      const MifTables* mx = tb.mx;
      if (mx && mx->prior) {
        const T* __restrict__ thn = (const T*)a.theta_next;
        for (int q = 0; q < tb.Q; ++q) {
          if (!((tb.est_mask >> q) & 1u)) continue;
          const bool fls = (mx->fls_mask >> q) & 1u;
          if (fls && !(a.n < mx->lag)) continue;
          const double x = plomrt::back_transform<double>((double)thn[(size_t)q * RJ + g], mx->prior_finv[q]);
          const double pr = plomrt::prior_density(mx->prior_kind[q], x, mx->prior_lo[q], mx->prior_hi[q]);
          lpr += plomrt::log_sanitized(pr, tb.like_min) * (fls ? mx->inv_lag : mx->inv_nobs);
        }
      }
    }
    const T lwv = (T)(plomrt::finish_loglik(ll, fl, M::N_TS) + lpr);
    ((T*)a.lw)[g] = lwv;
    return (double)lwv;
  }
  return NAN;
}


// ------------------------------------------------------------------ propagate, one team per particle
// For models whose state lives in shared memory, a team of TP lanes of one
// warp advances one particle: the compartment-age classes are split between
// the team's lanes (M::step_team), so a block holds BT / TP particles and an
// SM several times more warps than with one thread per particle.  Draws,
// equations and the order of the incidence and likelihood sums are those of
// the single-thread kernel up to the association of the team sums.
template <int TP_>
struct Team {
  static constexpr int TP = TP_;
  int rank;
  unsigned mask;
  __device__ __forceinline__ void sync() const { __syncwarp(mask); }
  // sum over the team, the same butterfly on every lane (identical results)
  template <class U>
  __device__ __forceinline__ U sum(U v) const {
#pragma unroll
    for (int o = 1; o < TP; o <<= 1) v += __shfl_xor_sync(mask, v, o);
    return v;
  }
};

// Column stride (in words) of the state in shared memory: the smallest
// stride >= PB that minimises bank conflicts when the TP ranks of the teams
// of a warp touch compartments G apart (the access pattern of cac_body).
template <int TP, int G>
constexpr int team_stride(int PB) {
  int best = PB, best_deg = 1 << 30;
  for (int st = PB; st < PB + 32; ++st) {
    int deg = 0;
    for (int bank = 0; bank < 32; ++bank) {
      int cnt = 0;
      for (int lane = 0; lane < 32; ++lane) {
        const int t = lane / TP, r = lane % TP;
        const long addr = (long)r * G * st + t;
        if ((int)(addr % 32) == bank) ++cnt;
      }
      if (cnt > deg) deg = cnt;
    }
    if (deg < best_deg) {
      best_deg = deg;
      best = st;
    }
  }
  return best;
}

template <class T, int V, int BT, int TP>
struct TeamLayout {
  static constexpr int NW = M::draws_per_cac(V);
  static constexpr int G = M::draw_group(NW, plomrt::NormalGen<T>::per_block());
  static constexpr int PB = BT / TP;
  static constexpr int STRIDE = team_stride<TP, G>(PB);
  static constexpr size_t pre_bytes = sizeof(typename M::template Pre<T>);
  static constexpr size_t bytes() {
    return (size_t)(kSmemCoup + kSmemPar) * sizeof(T) + (size_t)M::S * STRIDE * sizeof(T) + (size_t)PB * pre_bytes +
           16;
  }
};

#ifndef PLOM_TEAM_MIN_BLOCKS
#define PLOM_TEAM_MIN_BLOCKS 4
#endif

template <class T, int V, bool DRIFT, bool CRN, int BT, int TP>
__global__ void __launch_bounds__(BT, PLOM_TEAM_MIN_BLOCKS) k_propagate_team(const Tables<T> tb, const StepArgs a) {
  typedef TeamLayout<T, V, BT, TP> L;
  typedef typename M::template Pre<T> PreT;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* s_coup = reinterpret_cast<T*>(smem_raw);
  T* s_par = s_coup + kSmemCoup;
  T* s_state = s_par + kSmemPar;
  unsigned char* pre_raw = reinterpret_cast<unsigned char*>(s_state + (size_t)M::S * L::STRIDE);
  pre_raw += (16 - ((uintptr_t)pre_raw & 15)) & 15;
  PreT* s_pre = reinterpret_cast<PreT*>(pre_raw);
  if constexpr (M::COUPLED) {
    for (int i = threadIdx.x; i < M::N_CAC * M::N_CAC; i += BT) s_coup[i] = tb.coupling[i];
  }
  for (int i = threadIdx.x; i < M::N_PAR_PROC * M::N_CAC; i += BT) s_par[i] = tb.par_cac[i];
  __syncthreads();
  wait_for_previous_kernel();
  const int J = tb.J;
  const size_t RJ = (size_t)tb.R * J;
  const int lp = threadIdx.x / TP;
  const size_t g = (size_t)blockIdx.x * L::PB + lp;  // particle of all runs
  if (g >= RJ) return;                               // the whole team leaves together
  Team<TP> tm;
  tm.rank = threadIdx.x % TP;
  tm.mask = (TP == 32) ? 0xffffffffu : (((1u << TP) - 1u) << ((threadIdx.x & 31) & ~(TP - 1)));
  const int r = (int)(g / J);
  const int j = (int)(g - (size_t)r * J);
  const size_t src = (size_t)r * J + (a.anc ? __ldg(a.anc + g) : (uint32_t)j);
  const T* __restrict__ Xp = (const T*)a.X_prev;
  T* __restrict__ Xn = (T*)a.X_next;
  SmemState<T, L::STRIDE> x;
  x.b = s_state + lp;
  for (int w = tm.rank; w < M::OFF_INC; w += TP) x[w] = Xp[(size_t)w * RJ + src];
  for (int w = M::OFF_INC + tm.rank; w < M::S; w += TP) x[w] = T(0);  // reset_inc
  tm.sync();

  ProcEnv<T> e;
  e.par_ = s_par;
  e.coup_ = s_coup;
  e.dgroup_ = tb.drift_group;
  e.dng_ = tb.drift_ngroups;
  e.dbt_ = tb.drift_bt;
  e.dvol_ = tb.drift_vol;
  const T dt = (T)tb.dt;
  const plomrt::PhiloxKey key = plomrt::make_key(*tb.seed, tb.filter_id + (uint32_t)r);
  for (int k = 0; k < a.n_sub; ++k) {
    const int sub = a.sub0 + k;
    e.cov_ = tb.cov_cac + (size_t)sub * M::N_COV_CAC * M::N_CAC;
    const T t = (T)__ldg(tb.t_sub + sub);
    if constexpr (CRN) {
      TableDraws<T, V> d;
      d.p = a.crn ? a.crn + ((size_t)g * a.n_sub + k) * a.crn_d : nullptr;
      d.key = key;
      d.j = (uint32_t)j;
      d.n = (uint32_t)a.n;
      d.sub = (uint32_t)k;
      M::template step_team<V, DRIFT, T>(x, t, dt, e, d, tm, s_pre[lp]);
    } else {
      PhiloxDraws<T, V> d;
      d.key = key;
      d.j = (uint32_t)j;
      d.n = (uint32_t)a.n;
      d.sub = (uint32_t)k;
      M::template step_team<V, DRIFT, T>(x, t, dt, e, d, tm, s_pre[lp]);
    }
  }
  for (int w = tm.rank; w < M::S; w += TP)
    if (w < M::OFF_INC || a.write_inc) Xn[(size_t)w * RJ + g] = x[w];
  if (a.x_hist) {
    for (int w = tm.rank; w < M::S; w += TP) a.x_hist[(size_t)w * RJ + g] = (double)x[w];
  }
  if (a.weigh) {
    double obs[M::N_TS];
    M::template proj2obs<T>(x, obs);
    ObsEnv oe;
    oe.par_ts_ = tb.par_ts;
    oe.cov_ts_ = a.cov_ts;
    double ll = 0.0;
    int fl = 0;
#pragma unroll
    for (int ts = 0; ts < M::N_TS; ++ts) {
      if (ts % TP != tm.rank) continue;
      const double y = __ldg(a.y + ts);
      if (isnan(y)) continue;
      const double mu = M::obs_mean(obs[ts], ts, a.t_obs, oe);
      const double var = M::obs_var(obs[ts], ts, a.t_obs, oe);
      ll += plomrt::log_like_term_p<T>(y, mu, var, tb.like_min, &fl);
    }
    ll = tm.sum(ll);
    fl = tm.sum(fl);
    if (tm.rank == 0) ((T*)a.lw)[g] = (T)plomrt::finish_loglik(ll, fl, M::N_TS);
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

// The systematic points of one interval: U and the run table of ran += 1/J.
struct SysTable {
  double U;
  int ns;  // runs (0 if the table overflowed)
  int pad;
  plomrt::SysSeg seg[plomrt::SYS_MAX_SEG];
};

// Per-filter device state of the current interval.
struct StepState {
  double m, s1, s2;
  int all_fail;
  unsigned long long heavy;  // tiles left to k_resample_heavy << 32 | their points
  SysTable tab;  // the interval's systematic points where no table array holds them (serving loop, no-allocation call)
};

struct FilterAcc {
  double loglik;
  int n_all_fail;
  int error;        // bit 1: systematic table overflow; bit 2: ODE step control failed; bit 3: no valid initial condition
  unsigned ticket;  // block ticket of k_weight_tiles
};

enum { ERR_SYS_TABLE = 2, ERR_ODE = 4, ERR_IC = 8 };

// weight() (smc.c:44): the particle fails if exp(loglik) <= LIKE_MIN^N_TS.
// fail_b is the largest double whose exponential is <= LIKE_MIN^N_TS
// (fail_boundary on the host, with the host's exp as in the reference), so
// the test needs no exponential: the particle fails exactly when l <= fail_b.
template <class T>
__device__ __forceinline__ bool weight_fails_at(T l, double fail_b) {
  return !((double)l > fail_b);
}

// ------------------------------------------------------------------ tiled resampling
// weight() + systematic_sampling() (model_builder/C/core/smc.c:27-112) over
// tiles of TILE consecutive particles, in two launches (a third only when
// the weights concentrate):
//   k_weight_tiles    per tile: (max, sum exp(l - max), sum exp(2 (l - max)),
//                     failures); the last block folds them in tile order
//                     (llike, ESS, all-fail rule, systematic points) and lays
//                     out the exclusive prefix P[b] of the tiles' normalised
//                     weights;
//   k_resample_tiles  per tile: the cumulative weights of its particles,
//                     C_i = P[b] + (prefix of exp(l - max_b)) * exp(max_b - max) / sum,
//                     in shared memory, and the ancestors of the systematic
//                     points that fall in the tile (P[b] < point <= P[b + 1]):
//                     the first i of the tile with C_i >= point (smc.c:105-108);
//   k_resample_heavy  the points of tiles that hold more than kHeavyPoints of
//                     them, shared by all blocks (the weights have concentrated
//                     on a few tiles; the tile's cumulative weights go through
//                     global memory).
// The cumulative weights never make a round trip through global memory in
// the common case, the tile prefixes come from the fold (no look-back across
// tiles), and every reduction runs in a fixed order (results do not depend on
// timing).  Tile ends are the fold's prefixes P[b], so every point belongs to
// exactly one tile; a point that rounding leaves above the tile's last C_i
// goes to the tile's last particle (the reference reads on past the array).
// b: the failure boundary (fail_boundary)
template <class T>
__device__ __forceinline__ double surviving_exp(T l, double b, double m) {
  return weight_fails_at(l, b) ? 0.0 : exp((double)l - m);
}

// points of a tile resampled by its own block; above, the tile goes to k_resample_heavy
constexpr int kHeavyTiles = 8;  // in tiles' worth of points

// (tile, first point, end of points, particles, points of the tiles listed
// before it) of a tile left to k_resample_heavy
struct HeavyTile {
  int b, jlo, jhi, n_in, off;
};

// #{j in [0, J) : point_j <= x}: points are U + j / J to within rounding far
// below their spacing, so an estimate is corrected by a step or two.
__device__ inline int points_at_or_below(const plomrt::SysSeg* seg, int ns, int J, double U, double x) {
  if (!(x >= U)) return 0;
  const double e = floor((x - U) * (double)J) + 1.0;
  int c = (e >= (double)J) ? J : (int)e;
  while (c > 0 && !(plomrt::systematic_point(seg, ns, c - 1) <= x)) --c;
  while (c < J && plomrt::systematic_point(seg, ns, c) <= x) ++c;
  return c;
}

// first i in [0, n) with !(x > c[i]), or n - 1 if every c[i] < x
__device__ __forceinline__ int tile_lower_bound(const double* c, int n, double x) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (x > c[mid]) lo = mid + 1; else hi = mid;
  }
  return lo;
}

// Shared scratch of the weighting / resampling of one tile (BT threads,
// IPT particles each); placed by the caller (static in the stand-alone
// kernels, inside the dynamic region of the serving loop).
template <int BT, int IPT>
struct TileScratch {
  double sC[BT * IPT];
  double swarp[BT / 32];
  LseAcc lse[BT / 32];
  plomrt::SysSeg seg[plomrt::SYS_MAX_SEG];
  int ns, fail, jlo, jhi;
};

// (max, sum exp(l - max), sum exp(2 (l - max)), failures) of the threads'
// partials merged over the block (fixed order); every thread gets it.  The
// block maximum first, then every partial rescaled to it once and the sums
// added: one exponential per thread instead of one per merge of a tree.
template <int BT>
__device__ __forceinline__ LseAcc block_lse_all(LseAcc a, LseAcc* sh) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  double m = a.m;
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, off));
  if (lane == 0) sh[warp].m = m;
  __syncthreads();
  m = sh[0].m;
#pragma unroll
  for (int w = 1; w < BT / 32; ++w) m = fmax(m, sh[w].m);
  const double f = (a.s1 > 0.0) ? exp(a.m - m) : 0.0;
  double s1 = a.s1 * f, s2 = a.s2 * f * f;
  int nf = a.nfail;
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    s1 += __shfl_xor_sync(0xffffffffu, s1, off);
    s2 += __shfl_xor_sync(0xffffffffu, s2, off);
    nf += __shfl_xor_sync(0xffffffffu, nf, off);
  }
  __syncthreads();
  if (lane == 0) sh[warp] = LseAcc{m, s1, s2, nf};
  __syncthreads();
  LseAcc r = {m, 0.0, 0.0, 0};
#pragma unroll
  for (int w = 0; w < BT / 32; ++w) {
    r.s1 += sh[w].s1;
    r.s2 += sh[w].s2;
    r.nfail += sh[w].nfail;
  }
  __syncthreads();
  return r;
}

// The systematic points of interval n (smc.c:97-101): U = inc * u and the
// run table of the J points ran += inc.  They depend on the interval's
// uniform alone, not on the weights.
__device__ inline void sys_table(SysTable* t, FilterAcc* acc, int J, int n, double U_crn, plomrt::PhiloxKey key) {
  const double inc = 1.0 / (double)J;
  const double u = (U_crn >= 0.0) ? U_crn : plomrt::resample_uniform(key, (uint32_t)n);
  const double U = inc * u;  // gsl_ran_flat(0, inc) = 0*(1-u) + inc*u
  t->U = U;
  int ns = plomrt::systematic_table(U, inc, J, t->seg, plomrt::SYS_MAX_SEG);
  if (ns < 0) {
    atomicOr(&acc->error, (int)ERR_SYS_TABLE);
    ns = 0;
  }
  t->ns = ns;
}

// Every interval's systematic points of R filters, one thread per (filter,
// interval), before the first interval: out[r * n_obs + n].  u_one >= 0
// gives the uniform of a single interval; else crn_u[n] (common random
// numbers) or the filter's Philox uniform (filter_id + r).
__global__ void k_sys_tables(int J, int n_obs, int R, const uint64_t* seed, uint32_t filter_id,
                             const double* __restrict__ crn_u, double u_one, SysTable* out, FilterAcc* acc) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n_obs * R) return;
  const int r = t / n_obs, n = t - r * n_obs;
  const double Uc = (u_one >= 0.0) ? u_one : (crn_u ? crn_u[n] : -1.0);
  sys_table(out + t, acc + r, J, n, Uc, plomrt::make_key(seed ? *seed : 0ull, filter_id + (uint32_t)r));
}

// The fold of the tile partials by one block (all threads call it): the
// filter's (max, sums, failures) in tile order, the exclusive prefix P[b] of
// the tiles' normalised weights (P[ntiles] = their total), llike, ESS, the
// all-fail rule (smc.c:55-69) and the systematic points of the interval.
template <int BT>
__device__ void fold_tiles(const LseAcc* part, int ntiles, int J, double log_like_min, double* P, StepState* st,
                           FilterAcc* acc, int n, double* llike_out, double* ess_out, LseAcc* sh, double* shd) {
  const int chunk = (ntiles + BT - 1) / BT;
  const int b0 = threadIdx.x * chunk, b1 = min(ntiles, b0 + chunk);
  // the partials of the other blocks are read from L2 (written before their
  // ticket, after a fence), FC at a time with their loads issued together:
  // each pass costs one round trip to L2 per FC tiles of the chunk
  constexpr int FC = 8;
  // the chunk's maximum, then its sums rescaled to it (one exponential per tile)
  LseAcc a = {-INFINITY, 0.0, 0.0, 0};
  for (int bb = b0; bb < b1; bb += FC) {
    double s1v[FC], mv[FC];
#pragma unroll
    for (int k = 0; k < FC; ++k) {
      const bool in = bb + k < b1;
      s1v[k] = in ? __ldcg(&part[bb + k].s1) : 0.0;
      mv[k] = in ? __ldcg(&part[bb + k].m) : -INFINITY;
    }
#pragma unroll
    for (int k = 0; k < FC; ++k)
      if (s1v[k] > 0.0) a.m = fmax(a.m, mv[k]);
  }
  for (int bb = b0; bb < b1; bb += FC) {
    double s1v[FC], mv[FC], s2v[FC];
    int nfv[FC];
#pragma unroll
    for (int k = 0; k < FC; ++k) {
      const bool in = bb + k < b1;
      s1v[k] = in ? __ldcg(&part[bb + k].s1) : 0.0;
      mv[k] = in ? __ldcg(&part[bb + k].m) : -INFINITY;
      s2v[k] = in ? __ldcg(&part[bb + k].s2) : 0.0;
      nfv[k] = in ? __ldcg(&part[bb + k].nfail) : 0;
    }
#pragma unroll
    for (int k = 0; k < FC; ++k) {
      a.nfail += nfv[k];
      if (s1v[k] > 0.0) {
        const double f = (mv[k] == a.m) ? 1.0 : exp(mv[k] - a.m);
        a.s1 += s1v[k] * f;
        a.s2 += s2v[k] * f * f;
      }
    }
  }
  a = block_lse_all<BT>(a, sh);
  const int all_fail = (a.nfail == J);
  // exclusive prefix of the tiles' normalised weights: chunk totals, a block
  // scan of them, then each chunk written in order
  double tot = 0.0;
  if (!all_fail) {
    for (int bb = b0; bb < b1; bb += FC) {
      double s1v[FC], mv[FC];
#pragma unroll
      for (int k = 0; k < FC; ++k) {
        const bool in = bb + k < b1;
        s1v[k] = in ? __ldcg(&part[bb + k].s1) : 0.0;
        mv[k] = in ? __ldcg(&part[bb + k].m) : 0.0;
      }
#pragma unroll
      for (int k = 0; k < FC; ++k)
        if (s1v[k] > 0.0) tot += s1v[k] * (exp(mv[k] - a.m) / a.s1);
    }
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  double v = tot;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const double o = __shfl_up_sync(0xffffffffu, v, off);
    if (lane >= off) v += o;
  }
  if (lane == 31) shd[warp] = v;
  __syncthreads();
  if (warp == 0) {
    double w = (lane < BT / 32) ? shd[lane] : 0.0;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const double o = __shfl_up_sync(0xffffffffu, w, off);
      if (lane >= off) w += o;
    }
    if (lane < BT / 32) shd[lane] = w;
  }
  __syncthreads();
  double run = ((warp > 0) ? shd[warp - 1] : 0.0) + (v - tot);
  for (int bb = b0; bb < b1; bb += FC) {
    double s1v[FC], mv[FC];
    if (!all_fail) {
#pragma unroll
      for (int k = 0; k < FC; ++k) {
        const bool in = bb + k < b1;
        s1v[k] = in ? __ldcg(&part[bb + k].s1) : 0.0;
        mv[k] = in ? __ldcg(&part[bb + k].m) : 0.0;
      }
    }
#pragma unroll
    for (int k = 0; k < FC; ++k) {
      if (bb + k >= b1) break;
      P[bb + k] = run;
      if (!all_fail && s1v[k] > 0.0) run += s1v[k] * (exp(mv[k] - a.m) / a.s1);
    }
  }
  if (b1 == ntiles && b0 < b1) P[ntiles] = run;
  if (threadIdx.x == 0) {
    double llike, ess;
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
    st->heavy = 0ull;
  }
}

// ntiles tiles of BT * IPT particles per filter over gridDim.x blocks (a
// block takes tiles b, b + gridDim.x, ...): the tile partials, then one
// ticket per block; the last block folds them.
template <class T, int BT, int IPT>
__global__ void __launch_bounds__(BT) k_weight_tiles(const T* __restrict__ lw, int J, int ntiles, double fail_b,
                                                     double log_like_min, LseAcc* part, double* P, StepState* st,
                                                     FilterAcc* acc, int n, double* llike_out, double* ess_out,
                                                     int out_stride) {
  __shared__ LseAcc sh[BT / 32];
  __shared__ double shd[BT / 32];
  __shared__ bool last;
  wait_for_previous_kernel();
  {
    const int r = blockIdx.y;
    lw += (size_t)r * J;
    part += (size_t)r * ntiles;
    P += (size_t)r * (ntiles + 1);
    st += r;
    acc += r;
    if (llike_out) llike_out += (size_t)r * out_stride;
    if (ess_out) ess_out += (size_t)r * out_stride;
  }
  for (int b = blockIdx.x; b < ntiles; b += gridDim.x) {
    const int base = b * BT * IPT;
    // the thread's maximum, then its sums relative to it
    T lv[IPT];
    bool ok[IPT];
    LseAcc a = {-INFINITY, 0.0, 0.0, 0};
#pragma unroll
    for (int k = 0; k < IPT; ++k) {
      const int i = base + k * BT + threadIdx.x;
      lv[k] = (i < J) ? lw[i] : T(0);
      ok[k] = (i < J) && !weight_fails_at(lv[k], fail_b);
      if (i < J && !ok[k]) a.nfail += 1;
      if (ok[k]) a.m = fmax(a.m, (double)lv[k]);
    }
#pragma unroll
    for (int k = 0; k < IPT; ++k) {
      if (!ok[k]) continue;
      const double e = ((double)lv[k] == a.m) ? 1.0 : exp((double)lv[k] - a.m);
      a.s1 += e;
      a.s2 += e * e;
    }
    a = block_lse_all<BT>(a, sh);
    if (threadIdx.x == 0) part[b] = a;
  }
  if (threadIdx.x == 0) {
    __threadfence();
    const unsigned t = atomicAdd(&acc->ticket, 1u);
    last = (t == gridDim.x - 1u);
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  if (threadIdx.x == 0) acc->ticket = 0u;
  fold_tiles<BT>(part, ntiles, J, log_like_min, P, st, acc, n, llike_out, ess_out, sh, shd);
}

// The propagate launch: PPT particles per thread, BT apart (one for
// shared-memory states).  (Merging the block's log-weights here, so that no
// separate launch re-reads them, measured slower: the epilogue's registers
// cost the propagate loop more, 0.563 against 0.505 ms per SEIR 20x2
// interval, than the launch it saves.)
template <class T, int V, bool DRIFT, bool CRN, bool SMEM, bool MIF, int BT, bool PSR = false, bool MULTI = false,
          int PPT = 1>
__global__ void __launch_bounds__(BT) k_propagate(const Tables<T> tb, const StepArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  static_assert(PPT == 1 || !SMEM, "one particle per shared-memory state column");
  propagate_tables<T, BT>(tb, smem_raw, true);  // tables no kernel of the filter writes
  wait_for_previous_kernel();
  const size_t RJ = (size_t)tb.R * tb.J;
  const size_t g0 = (size_t)blockIdx.x * BT * PPT + threadIdx.x;  // particle of all runs
#pragma unroll
  for (int p = 0; p < PPT; ++p) {
    const size_t g = g0 + (size_t)p * BT;
    if (g < RJ) propagate_particle<T, V, DRIFT, CRN, SMEM, MIF, BT, PSR, MULTI>(tb, a, g, smem_raw);
  }
}

// Cumulative normalised weights of tile b: sC[i] = P[b] + (prefix of
// exp(l - max_b) in particle order) * exp(max_b - max) / sum, i < n_in
// (all threads of the block call it).
template <class T, int BT, int IPT>
__device__ void cum_tile(const T* __restrict__ lw, int J, double fail_b, const LseAcc* __restrict__ part,
                         const double* __restrict__ P, const StepState* st, int b, TileScratch<BT, IPT>& sc) {
  constexpr int TILE = BT * IPT;
  const int base = b * TILE;
  const int n_in = min(TILE, J - base);
  const double mb = __ldcg(&part[b].m);
  const double s1b = __ldcg(&part[b].s1);
  const double f = (s1b > 0.0) ? exp(mb - st->m) / st->s1 : 0.0;
  const double Pb = __ldcg(P + b);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  double carry = 0.0;
#pragma unroll
  for (int k = 0; k < IPT; ++k) {
    const int ii = k * BT + threadIdx.x;
    const double p = (ii < n_in) ? surviving_exp(lw[base + ii], fail_b, mb) : 0.0;
    double v = p;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const double o = __shfl_up_sync(0xffffffffu, v, off);
      if (lane >= off) v += o;
    }
    if (lane == 31) sc.swarp[warp] = v;
    __syncthreads();
    if (warp == 0) {
      double w = (lane < BT / 32) ? sc.swarp[lane] : 0.0;
#pragma unroll
      for (int off = 1; off < 32; off <<= 1) {
        const double o = __shfl_up_sync(0xffffffffu, w, off);
        if (lane >= off) w += o;
      }
      if (lane < BT / 32) sc.swarp[lane] = w;
    }
    __syncthreads();
    const double incl = carry + ((warp > 0) ? sc.swarp[warp - 1] : 0.0) + v;
    sc.sC[ii] = Pb + incl * f;
    carry += sc.swarp[BT / 32 - 1];
    __syncthreads();
  }
}

// run of the table that holds point j: the last with j0 <= j
__device__ __forceinline__ int sys_run(const plomrt::SysSeg* seg, int ns, int j) {
  int lo = 0, hi = ns - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (seg[mid].j0 <= j) lo = mid; else hi = mid - 1;
  }
  return lo;
}

// Ancestors of the consecutive points [ja, jb) over the cumulative weights
// c[0, n) of the tile starting at particle `first`: the first i with
// c[i] >= point (n - 1 if none), by one search for ja and a walk for the rest
// (points and weights both ascend).  Point values are systematic_point's.
__device__ __forceinline__ void place_points(const plomrt::SysSeg* seg, int ns, int ja, int jb, const double* c,
                                             int n, int first, uint32_t* __restrict__ anc,
                                             uint32_t* __restrict__ anc_hist) {
  if (ja >= jb) return;
  int sg = sys_run(seg, ns, ja);
  double ran = seg[sg].x0 + (double)(ja - seg[sg].j0) * seg[sg].step;
  int i = tile_lower_bound(c, n, ran);
  for (int j = ja;;) {
    const uint32_t r = (uint32_t)(first + i);
    anc[j] = r;
    if (anc_hist) anc_hist[j] = r;
    if (++j >= jb) break;
    while (sg + 1 < ns && seg[sg + 1].j0 <= j) ++sg;
    ran = seg[sg].x0 + (double)(j - seg[sg].j0) * seg[sg].step;
    while (i < n - 1 && ran > c[i]) ++i;
  }
}

// Tile b of one filter: its cumulative weights and the ancestors of the
// systematic points that fall in it (all threads of the block call it),
// each thread a run of consecutive points.  heavy == nullptr: the block
// places all of its points however many; else a tile with more than
// kHeavyTiles * TILE points writes its cumulative weights to C and is listed
// for k_resample_heavy.  Identity ancestors when every particle failed
// (smc.c:55-69).
template <class T, int BT, int IPT>
__device__ void resample_tile(const T* __restrict__ lw, int J, double fail_b, const LseAcc* __restrict__ part,
                              const double* __restrict__ P, StepState* st, const SysTable* tab, int b, int ntiles,
                              uint32_t* __restrict__ anc, uint32_t* __restrict__ anc_hist, double* __restrict__ C,
                              HeavyTile* heavy, TileScratch<BT, IPT>& sc) {
  constexpr int TILE = BT * IPT;
  static_assert(BT >= 64, "two warps find the tile's points");
  const int base = b * TILE;
  const int n_in = min(TILE, J - base);
  if (threadIdx.x == 0) {
    sc.ns = tab->ns;
    sc.fail = st->all_fail;
  }
  __syncthreads();
  if (sc.fail || sc.ns == 0) {
    for (int i = threadIdx.x; i < n_in; i += BT) {
      anc[base + i] = (uint32_t)(base + i);
      if (anc_hist) anc_hist[base + i] = (uint32_t)(base + i);
    }
    __syncthreads();
    return;
  }
  const int ns = sc.ns;
  for (int i = threadIdx.x; i < ns; i += BT) sc.seg[i] = tab->seg[i];
  __syncthreads();
  // the tile's points, P[b] < point <= P[b + 1] (the first tile from point 0,
  // the last to point J - 1), while the other warps start the weights
  const double U = tab->U;
  if (threadIdx.x == 0) sc.jlo = (b == 0) ? 0 : points_at_or_below(sc.seg, ns, J, U, __ldcg(P + b));
  if (threadIdx.x == 32) sc.jhi = (b == ntiles - 1) ? J : points_at_or_below(sc.seg, ns, J, U, __ldcg(P + b + 1));
  cum_tile<T, BT, IPT>(lw, J, fail_b, part, P, st, b, sc);
  const int jlo = sc.jlo, jhi = max(sc.jlo, sc.jhi);
  const int np = jhi - jlo;
  if (heavy && np > kHeavyTiles * TILE) {
    for (int i = threadIdx.x; i < n_in; i += BT) C[base + i] = sc.sC[i];
    if (threadIdx.x == 0) {
      const unsigned long long k = atomicAdd(&st->heavy, (1ull << 32) | (unsigned long long)np);
      heavy[k >> 32] = HeavyTile{b, jlo, jhi, n_in, (int)(k & 0xffffffffull)};
    }
  } else {
    const int per = (np + BT - 1) / BT;
    const int ja = jlo + threadIdx.x * per;
    place_points(sc.seg, ns, ja, min(jhi, ja + per), sc.sC, n_in, base, anc, anc_hist);
  }
  __syncthreads();  // the scratch of one tile before the next
}

template <class T, int BT, int IPT>
__global__ void __launch_bounds__(BT) k_resample_tiles(const T* __restrict__ lw, int J, double fail_b,
                                                       const LseAcc* __restrict__ part, const double* __restrict__ P,
                                                       StepState* st, const SysTable* tab, int tab_stride,
                                                       uint32_t* __restrict__ anc, uint32_t* __restrict__ anc_hist,
                                                       double* __restrict__ C, HeavyTile* heavy) {
  __shared__ TileScratch<BT, IPT> sc;
  wait_for_previous_kernel();
  const int ntiles = gridDim.x;
  const int r = blockIdx.y;
  resample_tile<T, BT, IPT>(lw + (size_t)r * J, J, fail_b, part + (size_t)r * ntiles, P + (size_t)r * (ntiles + 1),
                            st + r, tab + (size_t)r * tab_stride, blockIdx.x, ntiles, anc + (size_t)r * J,
                            anc_hist ? anc_hist + (size_t)r * J : nullptr, C + (size_t)r * J,
                            heavy + (size_t)r * ntiles, sc);
}

// largest tile of the weighting / resampling launches (a listed tile's
// cumulative weights are staged in shared memory)
constexpr int kMaxTile = 1024;

// The points of the tiles listed by resample_tile, spread evenly over all
// blocks: a block takes a contiguous share of the listed points, stages the
// cumulative weights of each listed tile its share touches in shared memory
// (one coalesced read) and gives each thread a run of consecutive points:
// the first i of the tile with C_i >= point.
template <int BT>
__global__ void __launch_bounds__(BT) k_resample_heavy(const double* __restrict__ C, int J, int ntiles, int tile,
                                                       const StepState* st, const SysTable* tab, int tab_stride,
                                                       const HeavyTile* __restrict__ heavy, uint32_t* __restrict__ anc,
                                                       uint32_t* __restrict__ anc_hist) {
  __shared__ plomrt::SysSeg seg[plomrt::SYS_MAX_SEG];
  __shared__ double sc[kMaxTile];
  __shared__ unsigned long long s_h;
  __shared__ int s_ns, s_e;
  wait_for_previous_kernel();
  const int r = blockIdx.y;
  st += r;
  tab += (size_t)r * tab_stride;
  if (threadIdx.x == 0) {
    s_h = st->all_fail ? 0ull : st->heavy;
    s_ns = tab->ns;
  }
  __syncthreads();
  const int nh = (int)(s_h >> 32);
  const long long total = (long long)(s_h & 0xffffffffull);
  const int ns = s_ns;
  if (nh == 0) return;
  const long long per_blk = (total + gridDim.x - 1) / gridDim.x;
  long long q0 = (long long)blockIdx.x * per_blk;
  const long long q1 = min(total, q0 + per_blk);
  if (q0 >= q1) return;
  C += (size_t)r * J;
  heavy += (size_t)r * ntiles;
  anc += (size_t)r * J;
  if (anc_hist) anc_hist += (size_t)r * J;
  for (int i = threadIdx.x; i < ns; i += BT) seg[i] = tab->seg[i];
  if (threadIdx.x == 0) {  // the listed tile holding point q0: the last with off <= q0
    int lo = 0, hi = nh - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if ((long long)__ldg(&heavy[mid].off) <= q0) lo = mid; else hi = mid - 1;
    }
    s_e = lo;
  }
  __syncthreads();
  for (int e = s_e; q0 < q1 && e < nh; ++e) {
    const HeavyTile h = heavy[e];
    const long long e1 = min(q1, (long long)h.off + (h.jhi - h.jlo));  // this block's points of tile e: [q0, e1)
    for (int i = threadIdx.x; i < h.n_in; i += BT) sc[i] = __ldg(C + (size_t)h.b * tile + i);
    __syncthreads();
    const long long np = e1 - q0;
    const long long per = (np + BT - 1) / BT;
    const long long qa = q0 + threadIdx.x * per;
    const long long qb = min(e1, qa + per);
    if (qa < qb)
      place_points(seg, ns, h.jlo + (int)(qa - h.off), h.jlo + (int)(qb - h.off), sc, h.n_in, h.b * tile, anc,
                   anc_hist);
    __syncthreads();  // sc of the next listed tile
    q0 = e1;
  }
}

// ------------------------------------------------------------------ helpers
// the initial particles: x0 in every particle, incidences zero (the time-0
// summaries read them; the buffers come from a pool and hold old values)
template <class T>
__global__ void k_init_state(const double* __restrict__ x0, int J, T* __restrict__ X) {
  const size_t total = (size_t)M::S * J;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
    const int w = (int)(i / J);
    X[i] = (w < M::OFF_INC) ? (T)x0[w] : T(0);
  }
}

// initial particles given one by one: cloud [OFF_INC][J] (FP64), incidences zero
template <class T>
__global__ void k_init_cloud(const double* __restrict__ cloud, int J, T* __restrict__ X) {
  const size_t total = (size_t)M::S * J, n_cloud = (size_t)M::OFF_INC * J;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x)
    X[i] = (i < n_cloud) ? (T)cloud[i] : T(0);
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

__global__ void k_reset_acc(FilterAcc* acc, int R = 1) {
  for (int r = threadIdx.x; r < R; r += blockDim.x) {
    acc[r].loglik = 0.0;
    acc[r].n_all_fail = 0;
    acc[r].error = 0;
    acc[r].ticket = 0u;
  }
}

// ------------------------------------------------------------------ iterated filtering
// Initial parameters of every particle of every run: theta_hat of the run plus a
// Gaussian proposal on the estimated components (propose_safe_theta_and_load_X0
// with ran_proposal, model_builder/C/mif/mif.c:119-121, C/core/proposal.c:40-79),
// and, for components that are initial conditions (x0_slot), the particle's
// initial state: proportion x N(0) for compartments (prop2Xpop_size), the
// transformed value for drift words (theta_driftIC2Xdrift).  A proposal whose
// proportions of one cac sum above 1 in a model with a remainder compartment
// is drawn again (plom_check_IC_assign_theta_remainder, proposal.c:87-114), at
// most kMaxIcAttempts times (then ERR_IC).
constexpr int kMaxIcAttempts = 1000;

template <class T>
__global__ void k_mif_init(const double* __restrict__ theta_hat, const double* __restrict__ sd_init, int Q,
                           unsigned est_mask, int R, int J, const uint64_t* seed, uint32_t filter_id,
                           T* __restrict__ theta, const int* __restrict__ x0_slot, const double* __restrict__ pop0,
                           const double* __restrict__ x0, const plomrt::BackTransform* __restrict__ theta_bt,
                           T* __restrict__ X, FilterAcc* acc) {
  const size_t RJ = (size_t)R * J;
  for (size_t g = blockIdx.x * (size_t)blockDim.x + threadIdx.x; g < RJ; g += (size_t)gridDim.x * blockDim.x) {
    const int r = (int)(g / J);
    const int j = (int)(g - (size_t)r * J);
    const plomrt::PhiloxKey key = plomrt::make_key(*seed, filter_id + (uint32_t)r);
    double th[kMaxTheta];
    for (int attempt = 0;; ++attempt) {
      for (int q = 0; q < Q; ++q) {
        double v = theta_hat[(size_t)r * Q + q];
        if ((est_mask >> q) & 1u) {
          T z[1];
          plomrt::NormalGen<T>::template fill<1>(key, (uint32_t)j, (uint32_t)attempt, (uint32_t)q, z,
                                                 (uint32_t)plomrt::STREAM_INIT);
          v += sd_init[q] * (double)z[0];
        }
        th[q] = (double)(T)v;
      }
      if (!x0_slot || M::POP_SIZE_EQ_SUM_SV) break;
      bool ok = true;
      for (int c = 0; c < M::N_CAC && ok; ++c) {
        double sum = 0.0;
        for (int i = 0; i < M::N_PAR_SV; ++i) {
          const int w = i * M::N_CAC + c;
          const int q = x0_slot[w];
          sum += q >= 0 ? plomrt::back_transform<double>(th[q], theta_bt[q]) : x0[w] / pop0[c];
        }
        if (sum > 1.0) ok = false;
      }
      if (ok) break;
      if (attempt + 1 >= kMaxIcAttempts) {
        atomicOr(&acc[r].error, (int)ERR_IC);
        break;
      }
    }
    for (int q = 0; q < Q; ++q) theta[(size_t)q * RJ + g] = (T)th[q];
    if (x0_slot) {
      for (int w = 0; w < M::OFF_INC; ++w) {
        const int q = x0_slot[w];
        if (q < 0) continue;
        const double v = (w < M::N_PAR_SV * M::N_CAC)
                             ? plomrt::back_transform<double>(th[q], theta_bt[q]) * pop0[w % M::N_CAC]
                             : th[q];
        X[(size_t)w * RJ + g] = (T)v;
      }
    }
  }
}

// Fixed-lag means of every run (update_fixed_lag_smoothing,
// model_builder/C/mif/methods.c:370-392): at interval L the reference sums the
// resampled components (index j of the new population) times the weights of
// the interval (index j of the population before resampling), i.e.
// sum_j theta[q][anc[j]] w[j].  Without a weighted interval up to L the
// weights are 1/J and the components those of the initial proposal (anc
// NULL).  Grid (Q, R); components outside fls_mask are skipped.
template <class T, int BT>
__global__ void __launch_bounds__(BT) k_mif_fls(const T* __restrict__ lw, const T* __restrict__ theta,
                                                const uint32_t* __restrict__ anc, int J, int R, double fail_b,
                                                const StepState* st, unsigned fls_mask, int Q, double* out) {
  const int q = blockIdx.x, r = blockIdx.y;
  if (!((fls_mask >> q) & 1u)) return;
  const size_t RJ = (size_t)R * J;
  const StepState* s = st + r;
  const bool uni = anc == nullptr || s->all_fail;
  const double m = uni ? 0.0 : s->m, s1 = uni ? 1.0 : s->s1;
  double acc = 0.0;
  for (int j = threadIdx.x; j < J; j += BT) {
    const size_t gj = (size_t)r * J + j;
    double w;
    if (uni) {
      w = 1.0 / (double)J;
    } else {
      const T l = lw[gj];
      w = weight_fails_at(l, fail_b) ? 0.0 : exp((double)l - m) / s1;
    }
    const size_t src = (size_t)r * J + (anc ? anc[gj] : (uint32_t)j);
    acc += (double)theta[(size_t)q * RJ + src] * w;
  }
  __shared__ double sh[BT / 32];
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < BT / 32; ++w) t += sh[w];
    out[(size_t)r * Q + q] = t;
  }
}

// Filtered mean (weighted) and prediction variance (unweighted, plus the
// theoretical variance of the perturbation) of every component, per run
// (mean_var_theta_theoretical_mif, model_builder/C/mif/methods.c:133-192).
// Grid (Q, R); the sums are shifted by theta_hat for a stable variance.
template <class T, int BT>
__global__ void __launch_bounds__(BT) k_mif_moments(const T* __restrict__ lw, const T* __restrict__ theta, int J, int R,
                                                    double fail_b, const StepState* st,
                                                    const double* __restrict__ theta_hat, const double* __restrict__ vt_add,
                                                    int Q, int n, int n_obs, double* bart, double* vt) {
  const int q = blockIdx.x, r = blockIdx.y;
  const size_t RJ = (size_t)R * J;
  const StepState* s = st + r;
  const double m = s->m, s1 = s->s1;
  const int all_fail = s->all_fail;
  const double c = theta_hat[(size_t)r * Q + q];
  double sw = 0.0, sd = 0.0, sd2 = 0.0;
  for (int j = threadIdx.x; j < J; j += BT) {
    const size_t g = (size_t)r * J + j;
    const double th = (double)theta[(size_t)q * RJ + g];
    double w;
    if (all_fail) {
      w = 1.0 / (double)J;
    } else {
      const T l = lw[g];
      w = weight_fails_at(l, fail_b) ? 0.0 : exp((double)l - m) / s1;
    }
    sw += w * th;
    const double d = th - c;
    sd += d;
    sd2 += d * d;
  }
  __shared__ double sh[3][BT / 32];
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    sw += __shfl_xor_sync(0xffffffffu, sw, off);
    sd += __shfl_xor_sync(0xffffffffu, sd, off);
    sd2 += __shfl_xor_sync(0xffffffffu, sd2, off);
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
    sh[0][warp] = sw;
    sh[1][warp] = sd;
    sh[2][warp] = sd2;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0.0, b = 0.0, c2 = 0.0;
    for (int w = 0; w < BT / 32; ++w) {
      a += sh[0][w];
      b += sh[1][w];
      c2 += sh[2][w];
    }
    double var = (J > 1) ? (c2 - b * b / (double)J) / ((double)J - 1.0) : 0.0;
    if (!(var >= 0.0) || isinf(var)) var = 0.0;
    const size_t o = ((size_t)r * n_obs + n) * Q + q;
    bart[o] = a;
    vt[o] = var + vt_add[(size_t)n * Q + q];
  }
}

// ------------------------------------------------------------------ deterministic skeleton (ode)
// Process environment of the ODE right-hand side: covariates come from a
// per-thread buffer refreshed at every stage time.
template <class T>
struct OdeProcEnv : ProcEnv<T> {
  T* covl_;
  __device__ __forceinline__ T cov(int k, int cac) const { return covl_[k * M::N_CAC + cac]; }
};

struct OdeArgs {
  double t0;          // start of the interval
  double eps_abs, eps_rel;
  int max_steps;      // attempted steps per interval before giving up
  plomrt::CovSplines cs;
  FilterAcc* acc;     // error flags
};

// One particle per thread: gather from the ancestor, reset the incidences,
// integrate the skeleton over [t0, t_obs] with RKF45 (f_prediction_ode,
// model_builder/C/core/prediction_util.c:176-193), store, weigh.
template <class T, int BT>
__global__ void __launch_bounds__(BT) k_propagate_ode(const Tables<T> tb, const StepArgs a, const OdeArgs o) {
  __shared__ __align__(16) T s_coup[kSmemCoup > 0 ? kSmemCoup : 1];
  __shared__ __align__(16) T s_par[kSmemPar > 0 ? kSmemPar : 1];
  if constexpr (M::COUPLED) {
    for (int i = threadIdx.x; i < M::N_CAC * M::N_CAC; i += BT) s_coup[i] = tb.coupling[i];
  }
  for (int i = threadIdx.x; i < M::N_PAR_PROC * M::N_CAC; i += BT) s_par[i] = tb.par_cac[i];
  __syncthreads();
  const int J = tb.J;
  const size_t RJ = (size_t)tb.R * J;
  const size_t g = (size_t)blockIdx.x * BT + threadIdx.x;
  if (g >= RJ) return;
  const int r = (int)(g / J);
  const int j = (int)(g - (size_t)r * J);
  const size_t src = (size_t)r * J + (a.anc ? __ldg(a.anc + g) : (uint32_t)j);
  const T* __restrict__ Xp = (const T*)a.X_prev;
  T* __restrict__ Xn = (T*)a.X_next;
  T y[M::S];
  T work[8 * M::S];
  T covl[M::N_COV_CAC * M::N_CAC > 0 ? M::N_COV_CAC * M::N_CAC : 1];
  for (int w = 0; w < M::OFF_INC; ++w) y[w] = Xp[(size_t)w * RJ + src];
  for (int w = M::OFF_INC; w < M::S; ++w) y[w] = T(0);  // reset_inc
  OdeProcEnv<T> e;
  e.par_ = s_par;
  e.coup_ = s_coup;
  e.cov_ = nullptr;
  e.dgroup_ = tb.drift_group;
  e.dng_ = tb.drift_ngroups;
  e.dbt_ = tb.drift_bt;
  e.dvol_ = tb.drift_vol;
  e.covl_ = covl;
  int steps = 0;
  const int rc = plomrt::rkf45_interval<M, T>(y, o.t0, a.t_obs, tb.dt, o.eps_abs, o.eps_rel, e, o.cs, work,
                                              o.max_steps, &steps);
  if (rc != plomrt::ODE_OK) atomicOr(&o.acc[r].error, (int)ERR_ODE);
  for (int w = 0; w < M::S; ++w)
    if (w < M::OFF_INC || a.write_inc) Xn[(size_t)w * RJ + g] = y[w];
  if (a.x_hist) {
    for (int w = 0; w < M::S; ++w) a.x_hist[(size_t)w * RJ + g] = (double)y[w];
  }
  if (a.weigh) {
    const plomrt::ArrayView<T> xv{y};
    double obs[M::N_TS];
    M::template proj2obs<T>(xv, obs);
    ObsEnv oe;
    oe.par_ts_ = tb.par_ts;
    oe.cov_ts_ = a.cov_ts;
    double ll = 0.0;
    int fl = 0;
#pragma unroll
    for (int ts = 0; ts < M::N_TS; ++ts) {
      const double yy = __ldg(a.y + ts);
      if (isnan(yy)) continue;
      const double mu = M::obs_mean(obs[ts], ts, a.t_obs, oe);
      const double var = M::obs_var(obs[ts], ts, a.t_obs, oe);
      ll += plomrt::log_like_term_p<T>(yy, mu, var, tb.like_min, &fl);
    }
    ((T*)a.lw)[g] = (T)plomrt::finish_loglik(ll, fl, M::N_TS);
  }
}

// ------------------------------------------------------------------ filtered summaries
// Quantities summarised per interval (compute_hat, model_builder/C/core/hat.c:68-176):
// state words of the compartments, remainders N(t) - sum of states (when the
// model has a remainder), observation means per series, drifted parameters
// mapped to the natural scale by f_inv; the observation variances per series
// follow them for the prediction residuals (print_prediction_residuals,
// print.c:632-711).
constexpr int kHatSv = M::N_PAR_SV * M::N_CAC;
constexpr int kHatRem = M::POP_SIZE_EQ_SUM_SV ? 0 : M::N_CAC;
constexpr int kHatObs = M::N_TS;
constexpr int kHatDrift = M::N_DRIFT * M::N_CAC;
constexpr int kHatQ = kHatSv + kHatRem + kHatObs + kHatDrift;  // summarised quantities
constexpr int kHatW = kHatQ + M::N_TS;                         // column of the particle weights
constexpr int kHatVals = kHatW + 1;                            // + observation variances, + weights

// Read-only view of particle j's state words straight from the SoA array.
template <class T>
struct ColumnView {
  const T* p;
  size_t ld;
  __device__ __forceinline__ double operator[](int w) const { return (double)p[(size_t)w * ld]; }
};

// The printed quantities of one particle: state words, remainders, observation
// means, drifted parameters (f_inv of their state word), then observation
// variances; out[q * stride] for q < kHatQ + N_TS.
template <class X>
__device__ __forceinline__ void particle_values(const X& x, const double* pop_size, const double* par_ts,
                                                const double* cov_ts, double t,
                                                const plomrt::BackTransform* drift_bt, double* out, size_t stride) {
  int q = 0;
  for (int i = 0; i < kHatSv; ++i) out[(size_t)(q++) * stride] = x[i];
  for (int c = 0; c < kHatRem; ++c) {
    double sv = 0.0;
    for (int i = 0; i < M::N_PAR_SV; ++i) sv += x[i * M::N_CAC + c];
    out[(size_t)(q++) * stride] = pop_size[c] - sv;
  }
  double obs[M::N_TS];
  M::template proj2obs<double>(x, obs);
  ObsEnv oe;
  oe.par_ts_ = par_ts;
  oe.cov_ts_ = cov_ts;
  for (int ts = 0; ts < M::N_TS; ++ts) out[(size_t)(q++) * stride] = M::obs_mean(obs[ts], ts, t, oe);
  for (int i = 0; i < kHatDrift; ++i) {
    double v = x[M::OFF_DRIFT + i];
    if (drift_bt) {
      plomrt::BackTransform b = drift_bt[i];
      b.scale = 0;
      b.multiplier = 1.0;
      b.is_duration = 0;
      v = plomrt::back_transform<double>(v, b);
    }
    out[(size_t)(q++) * stride] = v;
  }
  for (int ts = 0; ts < M::N_TS; ++ts) out[(size_t)(q++) * stride] = M::obs_var(obs[ts], ts, t, oe);
}

// Values of every summarised quantity per particle (column-major [kHatVals][J])
// and the particle's weight: its normalised weight when the interval was
// weighted and not all particles failed, else 1 (a count; the quantile ranks
// of equal weights are then integers).
template <class T>
__global__ void k_hat_values(const T* __restrict__ X, int J, const double* __restrict__ pop_size,
                             const double* __restrict__ par_ts, const double* __restrict__ cov_ts, double t_obs,
                             const plomrt::BackTransform* __restrict__ drift_bt, const T* __restrict__ lw,
                             const StepState* st, int weighted, double fail_b, double* __restrict__ vals) {
  const bool uni = !weighted || st->all_fail;
  const double m = uni ? 0.0 : st->m, s1 = uni ? 1.0 : st->s1;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < J; j += gridDim.x * blockDim.x) {
    const ColumnView<T> x{X + j, (size_t)J};
    particle_values(x, pop_size, par_ts, cov_ts, t_obs, drift_bt, vals + j, (size_t)J);
    double w = 1.0;
    if (!uni) {
      const T l = lw[j];
      w = weight_fails_at(l, fail_b) ? 0.0 : exp((double)l - m) / s1;
    }
    vals[(size_t)kHatW * J + j] = w;
  }
}

// Printed quantities of particles taken at different times: particle i is
// X[:, i] at time row rows[i] (0 = time 0, n + 1 = t_obs[n]); out is
// [kHatQ + N_TS][P].  Tables: pop_size [n_obs + 1][N_CAC], cov_ts
// [n_obs][N_COV_TS][N_TS], cov_ts0 [N_COV_TS][N_TS].
__global__ void k_particle_values(const double* __restrict__ X, int P, const int* __restrict__ rows,
                                  const double* __restrict__ t_obs, const double* __restrict__ pop_size,
                                  const double* __restrict__ par_ts, const double* __restrict__ cov_ts,
                                  const double* __restrict__ cov_ts0, const plomrt::BackTransform* __restrict__ drift_bt,
                                  double* __restrict__ out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < P; i += gridDim.x * blockDim.x) {
    const int r = rows[i];
    const ColumnView<double> x{X + i, (size_t)P};
    const double* cov = r == 0 ? cov_ts0 : (cov_ts ? cov_ts + (size_t)(r - 1) * M::N_COV_TS * M::N_TS : nullptr);
    const double t = r == 0 ? 0.0 : t_obs[r - 1];
    particle_values(x, pop_size ? pop_size + (size_t)r * M::N_CAC : nullptr, par_ts, cov, t, drift_bt, out + i,
                    (size_t)P);
  }
}

__device__ __forceinline__ uint64_t order_key(double v) {
  const uint64_t b = (uint64_t)__double_as_longlong(v);
  return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}
__device__ __forceinline__ double key_value(uint64_t k) {
  const uint64_t b = (k >> 63) ? (k & 0x7fffffffffffffffull) : ~k;
  return __longlong_as_double((long long)b);
}

template <int BT>
__device__ __forceinline__ double block_sum(double v, double* sh) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  double t = 0.0;
  for (int w = 0; w < BT / 32; ++w) t += sh[w];
  __syncthreads();
  return t;
}

// Weighted mean and 2.5 % / 97.5 % quantiles of every quantity (block per
// quantity).  The quantile is the smallest value whose cumulative weight in
// value order reaches the target (get_CI95, hat.c:28-57): found by a radix
// select over the order-preserving 64-bit keys of the values, 8 bits per pass,
// both quantiles in the same passes.  Targets: the levels for normalised
// weights; for equal weights the ranks rank_lo / rank_hi at which the
// reference's running sum of 1/J first reaches the levels (computed once on
// the host), compared against exact integer counts.
template <class T, int BT>
__global__ void __launch_bounds__(BT) k_hat_stats(const double* __restrict__ vals, int J, const StepState* st,
                                                  int weighted, double rank_lo, double rank_hi,
                                                  double* __restrict__ hat) {
  __shared__ double sh[BT / 32];
  __shared__ double hist[2][256];
  __shared__ uint64_t s_prefix[2];
  __shared__ double s_below[2];
  const int q = blockIdx.x;
  const double* v = vals + (size_t)q * J;
  const double* w = vals + (size_t)kHatW * J;
  const bool uni = !weighted || st->all_fail;
  double acc = 0.0;
  for (int j = threadIdx.x; j < J; j += BT) acc += w[j] * v[j];
  double mean = block_sum<BT>(acc, sh);
  if (uni) mean /= (double)J;
  const double target[2] = {uni ? rank_lo : 0.025, uni ? rank_hi : 0.975};
  if (threadIdx.x < 2) {
    s_prefix[threadIdx.x] = 0ull;
    s_below[threadIdx.x] = 0.0;
  }
  for (int shift = 56; shift >= 0; shift -= 8) {
    for (int i = threadIdx.x; i < 512; i += BT) (&hist[0][0])[i] = 0.0;
    __syncthreads();
    const uint64_t hi_mask = (shift == 56) ? 0ull : (~0ull << (shift + 8));
    const uint64_t p0 = s_prefix[0] & hi_mask, p1 = s_prefix[1] & hi_mask;
    for (int j0 = 0; j0 < J; j0 += BT) {
      const int j = j0 + threadIdx.x;
      const bool in = j < J;
      const uint64_t key = in ? order_key(v[j]) : 0ull;
      const double wj = in ? w[j] : 0.0;
      const int bin = (int)((key >> shift) & 255u);
#pragma unroll
      for (int k = 0; k < 2; ++k) {
        const bool match = in && ((key & hi_mask) == (k ? p1 : p0));
        // warp-aggregate when every lane hits the same bin (the common case
        // in the high passes, where the values share sign and exponent)
        const unsigned ballot = __ballot_sync(0xffffffffu, match);
        const int b0 = __shfl_sync(0xffffffffu, bin, 0);
        const bool same = (ballot == 0xffffffffu) && __all_sync(0xffffffffu, bin == b0);
        if (same) {
          double t = wj;
#pragma unroll
          for (int off = 16; off > 0; off >>= 1) t += __shfl_xor_sync(0xffffffffu, t, off);
          if ((threadIdx.x & 31) == 0) atomicAdd(&hist[k][b0], t);
        } else if (match) {
          atomicAdd(&hist[k][bin], wj);
        }
      }
    }
    __syncthreads();
    if (threadIdx.x < 2) {
      const int k = threadIdx.x;
      double cum = s_below[k];
      int d = -1, last = -1;
      double cum_last = cum;
      for (int b = 0; b < 256; ++b) {
        const double h = hist[k][b];
        if (h == 0.0) continue;
        if (cum + h >= target[k]) {
          d = b;
          break;
        }
        last = b;
        cum_last = cum;
        cum += h;
      }
      if (d < 0) {  // rounding left the total below the target: the largest value
        d = last >= 0 ? last : 0;
        cum = cum_last;
      }
      s_prefix[k] |= (uint64_t)d << shift;
      s_below[k] = cum;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    hat[(size_t)q * 3 + 0] = key_value(s_prefix[0]);
    hat[(size_t)q * 3 + 1] = mean;
    hat[(size_t)q * 3 + 2] = key_value(s_prefix[1]);
  }
}

// Prediction residuals of every series over the resampled particles: mean and
// variance of the observation means, mean of the observation variances
// (print_prediction_residuals, print.c:632-711).  Block per series.
template <int BT>
__global__ void __launch_bounds__(BT) k_pred_res(const double* __restrict__ vals, const uint32_t* __restrict__ anc,
                                                 int J, const double* __restrict__ y, double* __restrict__ out) {
  __shared__ double sh[BT / 32];
  const int ts = blockIdx.x;
  const double* om = vals + (size_t)(kHatSv + kHatRem + ts) * J;
  const double* ov = vals + (size_t)(kHatQ + ts) * J;
  double a = 0.0, b = 0.0;
  for (int j = threadIdx.x; j < J; j += BT) {
    const uint32_t s = anc ? anc[j] : (uint32_t)j;
    a += om[s];
    b += ov[s];
  }
  const double pred = block_sum<BT>(a, sh) / (double)J;
  const double var_obs = block_sum<BT>(b, sh) / (double)J;
  double m2 = 0.0;
  for (int j = threadIdx.x; j < J; j += BT) {
    const uint32_t s = anc ? anc[j] : (uint32_t)j;
    const double d = om[s] - pred;
    m2 += d * d;
  }
  const double M2 = block_sum<BT>(m2, sh);
  if (threadIdx.x == 0) {
    const double var_state = M2 / ((double)J - 1.0);
    out[ts * 2 + 0] = pred;
    out[ts * 2 + 1] = (y[ts] - pred) / sqrt(var_state + var_obs);
  }
}

// ------------------------------------------------------------------ sampled trajectory
// One trajectory drawn from the filter's genealogy as sample_traj_and_print
// does (model_builder/C/core/print.c:715-784), including its indexing:
// * the final particle j is the first whose running weight (last weighted
//   interval, in particle order) reaches u, and it indexes the resampled
//   population;
// * walking back, the ancestor index at a data interval is taken from that
//   interval's own selection (select[indn]) for every data interval but the
//   last, and intervals without data keep j.
// post(n, j) = x_hist[n][:, anc_hist[n][j]] is particle j after interval n
// (anc_hist is the identity where nothing was resampled); time -1 is x0.
// Rows are written in print order: rows_t[r] = time row (n + 1), states
// [r][S].  One block; the walk is serial (T steps), the gathers parallel.
template <class T, int BT>
__global__ void __launch_bounds__(BT) k_sample_traj(const T* __restrict__ lw, int J, const StepState* st,
                                                    double fail_b, double u, int n_obs,
                                                    const int* __restrict__ data_idx, int n_data,
                                                    const uint32_t* __restrict__ anc_hist,
                                                    const double* __restrict__ x_hist, const double* __restrict__ x0,
                                                    int* __restrict__ rows_t, int* __restrict__ rows_j,
                                                    double* __restrict__ states, int* __restrict__ n_rows) {
  __shared__ double s_part[BT];
  __shared__ int s_sel;
  const bool uni = st->all_fail;
  const double m = uni ? 0.0 : st->m, s1 = uni ? 1.0 : st->s1;
  auto wgt = [&](int j) -> double {
    if (uni) return 1.0 / (double)J;
    const T l = lw[j];
    return weight_fails_at(l, fail_b) ? 0.0 : exp((double)l - m) / s1;
  };
  // first j with inclusive running weight >= u: chunk sums, a serial scan of
  // BT partial sums, then a serial search inside the chunk that crosses
  const int chunk = (J + BT - 1) / BT;
  const int lo = threadIdx.x * chunk, hi = min(J, lo + chunk);
  double acc = 0.0;
  for (int j = lo; j < hi; ++j) acc += wgt(j);
  s_part[threadIdx.x] = acc;
  if (threadIdx.x == 0) s_sel = J - 1;
  __syncthreads();
  if (threadIdx.x == 0) {
    double run = 0.0;
    for (int t = 0; t < BT; ++t) {
      const double next = run + s_part[t];
      if (next >= u && t * chunk < J) {
        int j = t * chunk;
        const int e = min(J, j + chunk);
        double c = run;
        for (; j < e; ++j) {
          c += wgt(j);
          if (c >= u) break;
        }
        s_sel = j < e ? j : e - 1;
        break;
      }
      run = next;
    }
    // the walk
    int j = s_sel, r = 0;
    auto put = [&](int n, int jj) {
      rows_t[r] = n + 1;
      rows_j[r] = (n < 0) ? 0 : (int)anc_hist[(size_t)n * J + jj];
      ++r;
    };
    put(n_obs - 1, j);
    for (int nn = data_idx[n_data - 1] - 1; nn > data_idx[n_data - 2]; --nn) put(nn, j);
    for (int k = n_data - 2; k >= 1; --k) {
      const int indn = data_idx[k];
      j = (int)anc_hist[(size_t)indn * J + j];
      put(indn, j);
      for (int nn = indn - 1; nn > data_idx[k - 1]; --nn) put(nn, j);
    }
    const int indn = data_idx[0];
    j = (int)anc_hist[(size_t)indn * J + j];
    for (int nn = indn; nn >= -1; --nn) put(nn, j);
    *n_rows = r;
    s_sel = r;
  }
  __syncthreads();
  const int R = s_sel;
  for (int i = threadIdx.x; i < R * M::S; i += BT) {
    const int r = i / M::S, w = i % M::S;
    const int n = rows_t[r] - 1;
    states[i] = (n < 0) ? (w < M::OFF_INC ? x0[w] : 0.0) : x_hist[((size_t)n * M::S + w) * J + rows_j[r]];
  }
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
