// C ABI of the SMC engine for one generated model (declared in include/plomgpu.h).
//
// Host orchestration of the time loop of run_SMC (model_builder/C/core/smc.c:
// 204-307): per observation interval one propagate launch, and, when the
// data row has a value and filtering is on, the weight / scan / search
// launches.  The whole loop is captured once into a CUDA graph per plan and
// replayed per likelihood evaluation.
#include PLOM_MODEL_HEADER
#include "smc_engine.cuh"
#include "plomgpu.h"

#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>
#include <string.h>
#include <algorithm>
#include <utility>
#include <mutex>
#include <string>
#include <vector>

using namespace plomgpu;

static_assert(sizeof(plomgpu_back_transform) == sizeof(plomrt::BackTransform), "back-transform layout");

namespace {

thread_local std::string g_err;

int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}

// The largest double x with exp(x) <= thresh, by bisection over the doubles
// in order (exp is non-decreasing): weight() (model_builder/C/core/smc.c:44)
// fails a particle when exp(loglik) <= LIKE_MIN^N_TS, which is loglik <= x,
// with the host's exp as the reference computes it.
double fail_boundary(double thresh) {
  auto key = [](double v) -> int64_t {
    int64_t b;
    memcpy(&b, &v, sizeof b);
    return b >= 0 ? b : -(b & INT64_MAX);
  };
  auto val = [](int64_t k) -> double {
    const int64_t b = k >= 0 ? k : ((-k) | INT64_MIN);
    double v;
    memcpy(&v, &b, sizeof v);
    return v;
  };
  int64_t lo = key(-HUGE_VAL), hi = key(HUGE_VAL);  // exp(lo) <= thresh < exp(hi)
  if (!(exp(val(hi)) > thresh)) return val(hi);      // nothing survives
  // the keys span more than int64_t: distances in uint64_t
  while ((uint64_t)hi - (uint64_t)lo > 1u) {
    const int64_t mid = (int64_t)((uint64_t)lo + ((uint64_t)hi - (uint64_t)lo) / 2u);
    if (exp(val(mid)) <= thresh) lo = mid; else hi = mid;
  }
  return val(lo);
}

#define CK(call)                                                                              \
  do {                                                                                        \
    cudaError_t e_ = (call);                                                                  \
    if (e_ != cudaSuccess) {                                                                  \
      return fail(e_ == cudaErrorMemoryAllocation ? PLOMGPU_ENOMEM : PLOMGPU_ECUDA,           \
                  std::string(#call) + ": " + cudaGetErrorString(e_));                        \
    }                                                                                         \
  } while (0)

constexpr bool kSmem = (M::S > 48);
constexpr int kBtProp = 128;
// lanes per particle of the team kernel (state in shared memory); 1 = one
// thread per particle.  One thread per particle is the default: on SEIR 20x2
// (J = 1e5) it measured 1.02 ms per interval against 1.26 / 1.80 / 2.96 ms
// for teams of 2 / 4 / 8 lanes (the team's shared coupling terms and
// barriers cost more than the extra warps recover).
#ifndef PLOM_TEAM
#define PLOM_TEAM 1
#endif
constexpr int kTeam = kSmem ? PLOM_TEAM : 1;
// particles per thread of the register-state propagate launch (shared-memory
// states: one)
#ifndef PLOM_PROP_PPT
#define PLOM_PROP_PPT 1
#endif
constexpr int kPropPpt = kSmem ? 1 : PLOM_PROP_PPT;
constexpr int kBtOde = 64;
constexpr int kOdeMaxSteps = 1000000;  // attempted RKF45 steps per interval
static_assert(kTeam == 1 || kTeam == 2 || kTeam == 4 || kTeam == 8 || kTeam == 16 || kTeam == 32,
              "team size must be a power of two up to 32");
// tiles of the filters' weighting / resampling (k_weight_tiles, k_resample_tiles):
// the propagate block's particles for shared-memory models (the tiles of the
// serving loop, so that a served request and the plain filter reduce in the
// same order), 1024 particles otherwise
constexpr int kBtRes = kSmem ? kBtProp : 256;
constexpr int kIptRes = kSmem ? 1 : 4;
constexpr int kTileRes = kBtRes * kIptRes;
static_assert(kTileRes <= kMaxTile, "k_resample_heavy stages a tile in shared memory");

int variant_of(int noises_off) { return noises_off & 3; }
bool drift_on(int noises_off) { return M::N_DRIFT > 0 && !(noises_off & PLOMGPU_NO_DRIFT); }

int draws_per_substep(int noises_off) {
  return M::N_CAC * M::draws_per_cac(variant_of(noises_off)) + (drift_on(noises_off) ? M::N_DRIFT * M::N_CAC : 0);
}

}  // namespace

struct plomgpu_plan {
  int J = 0, n_obs = 0, sub_total = 0, precision = 32, noises_off = 0, filter = 1;
  bool crn = false, want_anc = false, want_xpred = false, want_llike = true;
  bool paired = false;           // CRN kernels on the FP64 Philox draws (no table)
  double* x0_cloud = nullptr;    // optional [OFF_INC][J] initial particles
  double dt = 1.0, like_min = 1e-17, fail_b = 0.0, log_like_min = 0.0;
  std::vector<int> n_sub, sub0;
  std::vector<double> t_obs, crn_u;
  std::vector<char> weigh;
  int ntiles = 1;
  int kernels = 0;
  size_t tsize = 4;
  cudaStream_t stream = nullptr;
  // device buffers
  void* X[2] = {nullptr, nullptr};
  void* lw = nullptr;
  double* P = nullptr;            // [R][ntiles + 1] tile prefixes of the normalised weights
  double* C = nullptr;            // [R][J] cumulative normalised weights of tiles left to k_resample_heavy
  HeavyTile* heavy = nullptr;     // [R][ntiles] those tiles
  int heavy_blocks = 1;
  int weight_blocks = 1;          // blocks of k_weight_tiles (each folds a share of the tiles)
  SysTable* sys = nullptr;        // [R][n_obs] systematic points of every interval
  double* crn_u_d = nullptr;      // [n_obs] injected resampling uniforms
  uint32_t* anc[2] = {nullptr, nullptr};
  LseAcc* part = nullptr;         // [R][ntiles] tile partials
  StepState* st = nullptr;
  FilterAcc* acc = nullptr;
  void* par_cac = nullptr;        // T
  double* par_cac_d = nullptr;    // double staging
  void* cov_cac = nullptr;        // T
  void* coupling = nullptr;       // T
  void* drift_vol = nullptr;      // T
  int* drift_group = nullptr;
  int* drift_ngroups = nullptr;
  plomrt::BackTransform* drift_bt = nullptr;
  double* par_ts = nullptr;
  double* t_sub = nullptr;
  double* cov_ts = nullptr;
  double* data = nullptr;
  double* x0 = nullptr;
  double* crn_tab = nullptr;
  uint64_t* seed = nullptr;
  double* llike = nullptr;
  double* ess = nullptr;
  uint32_t* anc_hist = nullptr;
  double* x_hist = nullptr;
  double* x_final = nullptr;
  // pinned host mirror of the accumulator
  FilterAcc* acc_h = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  // one-shot filters (plomgpu_smc_run) enqueue the time loop on the stream
  // instead of capturing it, and read the accumulator through pageable
  // memory: a graph that runs once, and a pinned page read once, cost more
  // than they save (SIR J = 1000, T = 52: 2.6 against 3.3 ms per call; SEIR
  // 20x2 J = 1e5, T = 520: 319 against 322 ms)
  bool direct = false;
  // optional timing events around every propagate launch (event record nodes of the graph)
  bool timing = false;
  std::vector<cudaEvent_t> ev;  // [2 * n_obs]: before / after propagate n
  // lock-stepped runs and iterated filtering (per-particle parameters)
  int R = 1;
  bool mif = false;
  int Q = 0;
  unsigned est_mask = 0;
  void* theta[2] = {nullptr, nullptr};  // T [Q][R*J]
  double* theta_hat = nullptr;          // [R][Q]
  double* sd_init = nullptr;            // [Q]
  double* sd_mut = nullptr;             // [n_obs][Q]
  double* vt_add = nullptr;             // [n_obs][Q]
  double* bart = nullptr;               // [R][n_obs][Q]
  double* vt = nullptr;                 // [R][n_obs][Q]
  plomrt::BackTransform* theta_bt = nullptr;
  int* proc_slot = nullptr;
  int* obs_slot = nullptr;
  std::vector<FilterAcc> acc_runs_h;
  // filtered summaries
  bool want_hat = false;
  double* vals = nullptr;      // [kHatVals][J]
  double* hat = nullptr;       // [n_obs][kHatQ][3]
  double* pred = nullptr;      // [n_obs][N_TS][2]
  double* pop = nullptr;       // [n_obs + 1][N_CAC]
  double* cov_ts0 = nullptr;   // [N_COV_TS][N_TS] at time 0
  double hat_rank[2] = {1.0, 1.0};  // quantile ranks under equal weights
  bool psr = false;  // Poisson system with stochastic rates
  int* proc_cslot = nullptr;  // iterated filtering, per-group components
  int* obs_tslot = nullptr;
  // iterated filtering: fixed-lag smoothing and the --prior patch
  unsigned mut_mask = 0u;     // components perturbed by the random walk
  unsigned fls_mask = 0u;     // components fitted by fixed-lag smoothing
  int fls_n = -2;             // interval whose weights give the fixed-lag means (-1: initial proposal, -2: none)
  MifTables* mx = nullptr;    // device
  int* vol_slot = nullptr;    // device [N_DRIFT][N_CAC]
  int* x0_slot = nullptr;     // device [OFF_INC]
  double* pop0 = nullptr;     // device [N_CAC]
  double* fls_out = nullptr;  // device [R][Q]
  // deterministic skeleton
  bool ode = false;
  double eps_abs = 1e-6, eps_rel = 1e-3;
  std::vector<double> t_start;  // start of every interval
  int* sp_meta = nullptr;
  double *sp_x = nullptr, *sp_y = nullptr, *sp_m2 = nullptr;
  // sampled trajectories
  int n_data = 0;
  int* data_idx = nullptr;     // device: intervals with data, ascending
  int* traj_t = nullptr;       // device [n_obs + 2]
  int* traj_j = nullptr;       // device [n_obs + 2]
  int* traj_n = nullptr;       // device scalar
  double* traj_x = nullptr;    // device [n_obs + 2][S]
};

// Rank (1-based) at which a running sum of 1/J, accumulated as the reference
// does (get_CI95, model_builder/C/core/hat.c:40-55), first reaches `level`.
int equal_weight_rank(int J, double level) {
  const double invJ = 1.0 / (double)J;
  double cum = 0.0;
  int k = 0;
  while (cum < level && k < J) {
    cum += invJ;
    ++k;
  }
  return k < 1 ? 1 : k;
}

namespace {

template <class T>
__global__ void k_convert(const double* __restrict__ in, T* __restrict__ out, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) out[i] = (T)in[i];
}

template <class T>
int upload_as(const double* h, size_t n, void** d, cudaStream_t s) {
  if (n == 0) return PLOMGPU_OK;
  std::vector<T> tmp(n);
  for (size_t i = 0; i < n; ++i) tmp[i] = (T)h[i];
  CK(cudaMalloc(d, n * sizeof(T)));
  CK(cudaMemcpyAsync(*d, tmp.data(), n * sizeof(T), cudaMemcpyHostToDevice, s));
  CK(cudaStreamSynchronize(s));
  return PLOMGPU_OK;
}

template <class U>
int upload(const U* h, size_t n, U** d, cudaStream_t s) {
  if (n == 0 || h == nullptr) return PLOMGPU_OK;
  CK(cudaMalloc((void**)d, n * sizeof(U)));
  CK(cudaMemcpyAsync(*d, h, n * sizeof(U), cudaMemcpyHostToDevice, s));
  return PLOMGPU_OK;
}

// Plan buffers come from a stream-ordered memory pool of the library, one
// per device, that keeps freed memory (release threshold: all of it): after
// the first filter of a size a one-shot filter costs no cudaMalloc and no
// cudaFree (they took 12-19 ms of a 0.28 s SEIR 20x2 filter).
// plomgpu_release_memory trims it.  The pool belongs to the context that
// created it; a handle that no longer answers (its context was reset) is
// replaced.
constexpr int kMaxDevices = 64;
std::mutex g_pool_mu;
cudaMemPool_t g_plan_pool[kMaxDevices] = {};

cudaError_t plan_mem_pool(cudaMemPool_t* out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_pool_mu);
  if (g_plan_pool[dev]) {
    uint64_t v = 0;
    if (cudaMemPoolGetAttribute(g_plan_pool[dev], cudaMemPoolAttrReleaseThreshold, &v) == cudaSuccess) {
      *out = g_plan_pool[dev];
      return cudaSuccess;
    }
    (void)cudaGetLastError();
    g_plan_pool[dev] = nullptr;
  }
  cudaMemPoolProps props = {};
  props.allocType = cudaMemAllocationTypePinned;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = dev;
  cudaMemPool_t mp = nullptr;
  if ((e = cudaMemPoolCreate(&mp, &props)) != cudaSuccess) return e;
  uint64_t keep = ~(uint64_t)0;
  if ((e = cudaMemPoolSetAttribute(mp, cudaMemPoolAttrReleaseThreshold, &keep)) != cudaSuccess) return e;
  g_plan_pool[dev] = mp;
  *out = mp;
  return cudaSuccess;
}

// the stream a plan being built allocates on (stream-ordered: its buffers
// are valid on that stream at once, elsewhere after a synchronisation)
thread_local cudaStream_t g_alloc_stream = nullptr;

template <class P>
cudaError_t palloc(P** ptr, size_t bytes) {
  cudaMemPool_t mp = nullptr;
  cudaError_t e = plan_mem_pool(&mp);
  if (e != cudaSuccess) return e;
  return cudaMallocFromPoolAsync((void**)ptr, bytes > 0 ? bytes : 1, mp, g_alloc_stream);
}

template <class T>
int pupload_as(const double* h, size_t n, void** d, cudaStream_t s) {
  if (n == 0) return PLOMGPU_OK;
  std::vector<T> tmp(n);
  for (size_t i = 0; i < n; ++i) tmp[i] = (T)h[i];
  CK(palloc(d, n * sizeof(T)));
  CK(cudaMemcpyAsync(*d, tmp.data(), n * sizeof(T), cudaMemcpyHostToDevice, s));
  CK(cudaStreamSynchronize(s));
  return PLOMGPU_OK;
}

template <class U>
int pupload(const U* h, size_t n, U** d, cudaStream_t s) {
  if (n == 0 || h == nullptr) return PLOMGPU_OK;
  CK(palloc(d, n * sizeof(U)));
  CK(cudaMemcpyAsync(*d, h, n * sizeof(U), cudaMemcpyHostToDevice, s));
  return PLOMGPU_OK;
}

// A kernel of the per-interval chain (propagate, weighting, resampling),
// launched with programmatic stream serialisation: it may be scheduled while
// the previous kernel of the stream drains, and waits (griddepcontrol.wait,
// wait_for_previous_kernel) before it reads that kernel's results.  Saves
// the launch gap at each of the four kernel boundaries of an interval.
template <class... KArgs, class... Args>
cudaError_t launch_chained(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                           Args&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

template <class T>
using PropKernel = void (*)(const Tables<T>, const StepArgs);

// a propagate kernel with its launch shape
template <class T>
struct PropLaunch {
  PropKernel<T> k = nullptr;
  int bt = 0;         // threads per block
  int per_block = 0;  // particles per block
  size_t smem = 0;    // dynamic shared memory
  explicit operator bool() const { return k != nullptr; }
};

template <class T, int V, bool DRIFT, bool CRN, bool MIF, bool PSR = false, bool MULTI = false>
PropLaunch<T> pick4() {
  PropLaunch<T> l;
  if constexpr (PSR) {
    l.k = &k_propagate<T, V, DRIFT, false, kSmem, false, kBtProp, true>;
    l.bt = kBtProp;
    l.per_block = kBtProp;
    l.smem = propagate_smem_bytes<T, kSmem, kBtProp>();
  } else if constexpr (kTeam > 1 && !MIF) {
    typedef TeamLayout<T, V, kBtProp, kTeam> L;
    l.k = &k_propagate_team<T, V, DRIFT, CRN, kBtProp, kTeam>;
    l.bt = kBtProp;
    l.per_block = L::PB;
    l.smem = L::bytes();
  } else {
    l.k = &k_propagate<T, V, DRIFT, CRN, kSmem, MIF, kBtProp, false, MULTI, kPropPpt>;
    l.bt = kBtProp;
    l.per_block = kBtProp * kPropPpt;
    l.smem = propagate_smem_bytes<T, kSmem, kBtProp>();
  }
  return l;
}

template <class T, bool CRN, bool MIF, bool MULTI = false>
PropLaunch<T> pick_v(int v, bool drift) {
  if (drift) {
    if constexpr (M::N_DRIFT > 0) {
      switch (v) {
        case 0: return pick4<T, 0, true, CRN, MIF, false, MULTI>();
        case 1: return pick4<T, 1, true, CRN, MIF, false, MULTI>();
        case 2: return pick4<T, 2, true, CRN, MIF, false, MULTI>();
        default: return pick4<T, 3, true, CRN, MIF, false, MULTI>();
      }
    }
  }
  switch (v) {
    case 0: return pick4<T, 0, false, CRN, MIF, false, MULTI>();
    case 1: return pick4<T, 1, false, CRN, MIF, false, MULTI>();
    case 2: return pick4<T, 2, false, CRN, MIF, false, MULTI>();
    default: return pick4<T, 3, false, CRN, MIF, false, MULTI>();
  }
}

// the Poisson-system step: white noise on / off, drift on / off
template <class T>
PropLaunch<T> pick_psr(int noises_off) {
  const bool noenv = (noises_off & PLOMGPU_NO_ENV_STO) != 0;
  if (drift_on(noises_off)) {
    if constexpr (M::N_DRIFT > 0) {
      return noenv ? pick4<T, 2, true, false, false, true>() : pick4<T, 0, true, false, false, true>();
    }
  }
  return noenv ? pick4<T, 2, false, false, false, true>() : pick4<T, 0, false, false, false, true>();
}

template <class T>
PropLaunch<T> pick_prop(int noises_off, bool crn, bool mif, bool psr = false, bool multi = false) {
  if (psr) {
    if (crn || mif) return PropLaunch<T>();
    return pick_psr<T>(noises_off);
  }
  const int v = variant_of(noises_off);
  const bool d = drift_on(noises_off);
  if (mif) {
    if (crn) return PropLaunch<T>();
    return multi ? pick_v<T, false, true, true>(v, d) : pick_v<T, false, true>(v, d);
  }
  if (crn) return pick_v<T, true, false>(v, d);
  return pick_v<T, false, false>(v, d);
}

// Filtered summaries of the particles in X (row `row` of the summary table:
// 0 = time 0, n + 1 = after interval n), weighted by the normalised weights of
// the interval when `weighted`, by 1/J otherwise.
template <class T>
int enqueue_hat(plomgpu_plan* p, const T* X, int row, const double* cov_ts, double t, bool weighted, cudaStream_t s) {
  const int J = p->J;
  const double* pop = p->pop ? p->pop + (size_t)row * M::N_CAC : nullptr;
  const int g = (J + 255) / 256 < 4096 ? (J + 255) / 256 : 4096;
  k_hat_values<T><<<g, 256, 0, s>>>(X, J, pop, p->par_ts, cov_ts, t, p->drift_bt, (const T*)p->lw, p->st,
                                    weighted ? 1 : 0, p->fail_b, p->vals);
  k_hat_stats<T, 256><<<kHatQ, 256, 0, s>>>(p->vals, J, p->st, weighted ? 1 : 0, p->hat_rank[0], p->hat_rank[1],
                                            p->hat + (size_t)row * kHatQ * 3);
  return 2;
}

template <class T>
int enqueue_filter(plomgpu_plan* p) {
  cudaStream_t s = p->stream;
  const int J = p->J;
  int kernels = 0;
  Tables<T> tb;
  tb.par_cac = (const T*)p->par_cac;
  tb.cov_cac = (const T*)p->cov_cac;
  tb.coupling = (const T*)p->coupling;
  tb.drift_group = p->drift_group;
  tb.drift_ngroups = p->drift_ngroups;
  tb.drift_bt = p->drift_bt;
  tb.drift_vol = (const T*)p->drift_vol;
  tb.par_ts = p->par_ts;
  tb.t_sub = p->t_sub;
  tb.dt = p->dt;
  tb.like_min = p->like_min;
  tb.seed = p->seed;
  tb.filter_id = 0;
  tb.J = J;
  tb.R = p->R;
  tb.Q = p->Q;
  tb.est_mask = p->est_mask;
  tb.theta_bt = p->theta_bt;
  tb.proc_slot = p->proc_slot;
  tb.obs_slot = p->obs_slot;
  tb.proc_cslot = p->proc_cslot;
  tb.obs_tslot = p->obs_tslot;
  tb.mut_mask = p->mut_mask;
  tb.vol_slot = p->vol_slot;
  tb.mx = p->mx;
  const int R = p->R;
  const size_t RJ = (size_t)R * J;

  const PropLaunch<T> kp = pick_prop<T>(p->noises_off, p->crn, p->mif, p->psr,
                                        p->proc_cslot != nullptr || p->obs_tslot != nullptr || p->vol_slot != nullptr);
  if (!kp) return fail(PLOMGPU_EINVAL, "no propagate kernel for these options");
  const size_t smem = kp.smem;
  if (smem > 48 * 1024) CK(cudaFuncSetAttribute(kp.k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));

  const int n_par = M::N_PAR_PROC * M::N_CAC;
  if (n_par > 0) {
    k_convert<T><<<(n_par + 255) / 256, 256, 0, s>>>(p->par_cac_d, (T*)p->par_cac, n_par);
    ++kernels;
  }
  k_reset_acc<<<1, 128, 0, s>>>(p->acc, R);
  ++kernels;
  // every interval's systematic points (they depend on the seed alone)
  k_sys_tables<<<(p->n_obs * R + 63) / 64, 64, 0, s>>>(J, p->n_obs, R, p->seed, 0u, p->crn_u_d, -1.0, p->sys, p->acc);
  ++kernels;
  {
    const size_t total = (size_t)M::S * RJ;
    const int g = (int)((total + 255) / 256 < 4096 ? (total + 255) / 256 : 4096);
    if (p->x0_cloud) k_init_cloud<T><<<g > 0 ? g : 1, 256, 0, s>>>(p->x0_cloud, (int)RJ, (T*)p->X[0]);
    else k_init_state<T><<<g > 0 ? g : 1, 256, 0, s>>>(p->x0, (int)RJ, (T*)p->X[0]);
    ++kernels;
  }
  // summaries of the initial particles (time 0, incidences reset, equal weights)
  if (p->want_hat) kernels += enqueue_hat<T>(p, (const T*)p->X[0], 0, p->cov_ts0, 0.0, false, s);
  int th_cur = 0;
  if (p->mif) {
    const int g = (int)((RJ + 255) / 256 < 4096 ? (RJ + 255) / 256 : 4096);
    k_mif_init<T><<<g, 256, 0, s>>>(p->theta_hat, p->sd_init, p->Q, p->est_mask, R, J, p->seed, 0u,
                                    (T*)p->theta[0], p->x0_slot, p->pop0, p->x0, p->theta_bt, (T*)p->X[0], p->acc);
    ++kernels;
    if (p->fls_n == -1) {
      k_mif_fls<T, 256><<<dim3(p->Q, R), 256, 0, s>>>(nullptr, (const T*)p->theta[0], nullptr, J, R, p->fail_b, p->st,
                                                      p->fls_mask, p->Q, p->fls_out);
      ++kernels;
    }
  }
  const int D = p->crn ? draws_per_substep(p->noises_off) : 0;
  size_t crn_off = 0;
  int cur = 0;           // generation holding the particles before interval n
  int anc_cur = -1;      // ancestors to apply when loading (index into p->anc), -1 = identity
  const int gprop = (int)((RJ + kp.per_block - 1) / kp.per_block);
  for (int n = 0; n < p->n_obs; ++n) {
    StepArgs a;
    a.n = n;
    a.n_sub = p->n_sub[n];
    a.sub0 = p->sub0[n];
    a.weigh = p->weigh[n];
    a.t_obs = p->t_obs[n];
    a.y = p->data + (size_t)n * M::N_TS;
    a.cov_ts = p->cov_ts ? p->cov_ts + (size_t)n * M::N_COV_TS * M::N_TS : nullptr;
    a.X_prev = p->X[cur];
    a.X_next = p->X[cur ^ 1];
    a.anc = anc_cur >= 0 ? p->anc[anc_cur] : nullptr;
    a.lw = p->lw;
    a.crn = p->crn_tab ? p->crn_tab + crn_off : nullptr;
    a.crn_d = D;
    a.x_hist = p->x_hist ? p->x_hist + (size_t)n * M::S * RJ : nullptr;
    a.write_inc = ((p->x_final != nullptr && n == p->n_obs - 1) || p->want_hat) ? 1 : 0;
    a.theta_prev = p->mif ? p->theta[th_cur] : nullptr;
    a.theta_next = p->mif ? p->theta[th_cur ^ 1] : nullptr;
    // the random walk applies where the previous interval resampled (C/mif/mif.c:190-191)
    a.sd_mut = (p->mif && n > 0 && p->weigh[n - 1]) ? p->sd_mut + (size_t)(n - 1) * p->Q : nullptr;
    a.x0_rep = nullptr;
    crn_off += RJ * p->n_sub[n] * D;
    if (p->timing) CK(cudaEventRecordWithFlags(p->ev[2 * n], s, cudaEventRecordExternal));
    if (p->ode) {
      OdeArgs o;
      o.t0 = p->t_start[n];
      o.eps_abs = p->eps_abs;
      o.eps_rel = p->eps_rel;
      o.max_steps = kOdeMaxSteps;
      o.cs.meta = p->sp_meta;
      o.cs.x = p->sp_x;
      o.cs.y = p->sp_y;
      o.cs.m2 = p->sp_m2;
      o.acc = p->acc;
      k_propagate_ode<T, kBtOde><<<(unsigned)((RJ + kBtOde - 1) / kBtOde), kBtOde, 0, s>>>(tb, a, o);
    } else {
      CK(launch_chained(kp.k, dim3(gprop), dim3(kp.bt), smem, s, tb, a));
    }
    if (p->timing) CK(cudaEventRecordWithFlags(p->ev[2 * n + 1], s, cudaEventRecordExternal));
    ++kernels;
    cur ^= 1;
    if (p->mif) th_cur ^= 1;
    if (a.weigh) {
      const int nxt = (anc_cur == 0) ? 1 : 0;
      CK(launch_chained(&k_weight_tiles<T, kBtRes, kIptRes>, dim3(p->weight_blocks, R), dim3(kBtRes), 0, s,
                        (const T*)p->lw, J, p->ntiles, p->fail_b, p->log_like_min, p->part, p->P, p->st, p->acc, n,
                        p->llike, p->ess, p->n_obs));
      ++kernels;
      if (p->mif) {
        k_mif_moments<T, 256><<<dim3(p->Q, R), 256, 0, s>>>((const T*)p->lw, (const T*)p->theta[th_cur], J, R,
                                                            p->fail_b, p->st, p->theta_hat, p->vt_add, p->Q, n,
                                                            p->n_obs, p->bart, p->vt);
        ++kernels;
      }
      if (p->want_hat) kernels += enqueue_hat<T>(p, (const T*)a.X_next, n + 1, a.cov_ts, a.t_obs, true, s);
      CK(launch_chained(&k_resample_tiles<T, kBtRes, kIptRes>, dim3(p->ntiles, R), dim3(kBtRes), 0, s,
                        (const T*)p->lw, J, p->fail_b, (const LseAcc*)p->part, (const double*)p->P, p->st,
                        (const SysTable*)(p->sys + n), p->n_obs, p->anc[nxt],
                        p->anc_hist ? p->anc_hist + (size_t)n * J : (uint32_t*)nullptr, p->C, p->heavy));
      CK(launch_chained(&k_resample_heavy<256>, dim3(p->heavy_blocks, R), dim3(256), 0, s, (const double*)p->C, J,
                        p->ntiles, kTileRes, (const StepState*)p->st, (const SysTable*)(p->sys + n), p->n_obs,
                        (const HeavyTile*)p->heavy, p->anc[nxt],
                        p->anc_hist ? p->anc_hist + (size_t)n * J : (uint32_t*)nullptr));
      kernels += 2;
      if (p->want_hat) {
        k_pred_res<256><<<M::N_TS, 256, 0, s>>>(p->vals, p->anc[nxt], J, a.y, p->pred + (size_t)n * M::N_TS * 2);
        ++kernels;
      }
      if (p->mif && n == p->fls_n) {
        k_mif_fls<T, 256><<<dim3(p->Q, R), 256, 0, s>>>((const T*)p->lw, (const T*)p->theta[th_cur], p->anc[nxt], J, R,
                                                        p->fail_b, p->st, p->fls_mask, p->Q, p->fls_out);
        ++kernels;
      }
      anc_cur = nxt;
    } else {
      if (p->anc_hist) {
        k_identity<<<(J + 255) / 256, 256, 0, s>>>(p->anc_hist + (size_t)n * J, J);
        ++kernels;
      }
      if (p->want_hat) kernels += enqueue_hat<T>(p, (const T*)a.X_next, n + 1, a.cov_ts, a.t_obs, false, s);
      anc_cur = -1;
    }
  }
  if (p->x_final) {
    const size_t total = (size_t)M::S * J;
    const int g = (int)((total + 255) / 256 < 4096 ? (total + 255) / 256 : 4096);
    k_gather_final<T><<<g, 256, 0, s>>>((const T*)p->X[cur], anc_cur >= 0 ? p->anc[anc_cur] : nullptr, J, M::S,
                                        p->x_final);
    ++kernels;
  }
  CK(cudaGetLastError());
  p->kernels = kernels;
  return PLOMGPU_OK;
}

// Draws of the production generators as this library compiles them (the
// fast-math build of the FP32 path), for distribution tests: stream s is the
// particle slot of the Philox counter, per_stream draws each.  kind 0: the
// normals of the sde step (NormalGen<T>, Box-Muller); 1 / 2 / 3: the psr
// samplers binomial(a, b), Poisson(a), Gamma(shape a, scale b) of precision T;
// 4: the normals of the psr uniform stream (Gamma white noise).
template <class T>
__global__ void k_debug_draws(int kind, double a, double b, uint64_t seed, int streams, int per_stream,
                              double* __restrict__ out) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= streams) return;
  const plomrt::PhiloxKey key = plomrt::make_key(seed, 0u);
  double* o = out + (size_t)s * per_stream;
  if (kind == 0) {
    constexpr int P = plomrt::NormalGen<T>::per_block();
    for (int i = 0; i < per_stream; i += P) {
      T z[P];
      plomrt::NormalGen<T>::template fill<P>(key, (uint32_t)s, 0u, (uint32_t)(i / P), z);
      for (int q = 0; q < P && i + q < per_stream; ++q) o[i + q] = (double)z[q];
    }
    return;
  }
  typename plomrt::PsrStream<T>::type rs;
  rs.init(key, (uint32_t)s, 0u, 0u);
  for (int i = 0; i < per_stream; ++i) {
    double v;
    if (kind == 1) v = (double)plomrt::binomial(rs, (T)a, (T)b);
    else if (kind == 2) v = (double)plomrt::poisson(rs, (T)a);
    else if (kind == 3) v = (double)plomrt::gamma(rs, (T)a, (T)b);
    else v = (double)rs.normal();
    o[i] = v;
  }
}

int check_desc(const plomgpu_smc_desc* d) {
  if (!d) return fail(PLOMGPU_EINVAL, "null descriptor");
  if (d->J < 1) return fail(PLOMGPU_EINVAL, "J must be >= 1");
  if (d->n_obs < 0) return fail(PLOMGPU_EINVAL, "n_obs must be >= 0");
  if (d->precision != 32 && d->precision != 64) return fail(PLOMGPU_EINVAL, "precision must be 32 or 64");
  if (d->n_obs > 0 && (!d->n_sub || !d->t_obs || !d->data)) return fail(PLOMGPU_EINVAL, "missing n_sub / t_obs / data");
  if (!d->x0) return fail(PLOMGPU_EINVAL, "missing x0");
  if (M::N_PAR_PROC > 0 && !d->par_cac) return fail(PLOMGPU_EINVAL, "missing par_cac");
  if (M::N_PAR_OBS > 0 && !d->par_ts) return fail(PLOMGPU_EINVAL, "missing par_ts");
  if (M::COUPLED && !d->coupling) return fail(PLOMGPU_EINVAL, "coupled model needs a coupling matrix");
  if (drift_on(d->noises_off) && (!d->drift_group || !d->drift_ngroups || !d->drift_bt || !d->drift_vol))
    return fail(PLOMGPU_EINVAL, "drift tables missing");
  if (d->crn_normals && !d->crn_uniforms) return fail(PLOMGPU_EINVAL, "crn_uniforms missing");
  if (d->paired_draws && (d->crn_normals || d->psr || d->ode))
    return fail(PLOMGPU_EINVAL, "paired draws replace the Philox draws of the sde implementation only");
  if (!(d->dt > 0.0)) return fail(PLOMGPU_EINVAL, "dt must be > 0");
  if (!(d->like_min > 0.0)) return fail(PLOMGPU_EINVAL, "like_min must be > 0");
  long long sub_total = 0;
  for (int n = 0; n < d->n_obs; ++n) {
    if (d->n_sub[n] < 0) return fail(PLOMGPU_EINVAL, "negative substep count");
    if ((long long)d->n_sub[n] * (M::N_CAC + 1) >= (1LL << 20))
      return fail(PLOMGPU_EINVAL, "too many substeps per interval for the draw counter layout");
    sub_total += d->n_sub[n];
  }
  if (sub_total > 0 && !d->t_sub) return fail(PLOMGPU_EINVAL, "missing t_sub");
  if (sub_total > 0 && M::N_COV_CAC > 0 && !d->cov_cac) return fail(PLOMGPU_EINVAL, "missing cov_cac");
  if (d->n_obs > 0 && M::N_COV_TS > 0 && !d->cov_ts) return fail(PLOMGPU_EINVAL, "missing cov_ts");
  if (drift_on(d->noises_off)) {
    for (int i = 0; i < M::N_DRIFT; ++i) {
      if (d->drift_ngroups[i] < 1 || d->drift_ngroups[i] > M::N_CAC) return fail(PLOMGPU_EINVAL, "bad drift group count");
      for (int c = 0; c < M::N_CAC; ++c) {
        const int g = d->drift_group[i * M::N_CAC + c];
        if (g < 0 || g >= d->drift_ngroups[i]) return fail(PLOMGPU_EINVAL, "bad drift group index");
      }
    }
  }
  return PLOMGPU_OK;
}

template <class T>
int plan_build(const plomgpu_smc_desc* d, plomgpu_plan* p) {
  cudaStream_t s = p->stream;
  const int J = d->J;
  p->tsize = sizeof(T);
  int rc;
  const size_t RJ = (size_t)p->R * J;
  CK(palloc(&p->X[0], (size_t)M::S * RJ * sizeof(T)));
  CK(palloc(&p->X[1], (size_t)M::S * RJ * sizeof(T)));
  CK(palloc(&p->lw, RJ * sizeof(T)));
  CK(palloc((void**)&p->C, RJ * sizeof(double)));
  CK(palloc((void**)&p->anc[0], RJ * sizeof(uint32_t)));
  CK(palloc((void**)&p->anc[1], RJ * sizeof(uint32_t)));
  if (p->mif) {
    CK(palloc(&p->theta[0], (size_t)p->Q * RJ * sizeof(T)));
    CK(palloc(&p->theta[1], (size_t)p->Q * RJ * sizeof(T)));
  }
  p->ntiles = (J + kTileRes - 1) / kTileRes;
  CK(palloc((void**)&p->part, (size_t)p->R * p->ntiles * sizeof(LseAcc)));
  CK(palloc((void**)&p->P, (size_t)p->R * (p->ntiles + 1) * sizeof(double)));
  CK(palloc((void**)&p->heavy, (size_t)p->R * p->ntiles * sizeof(HeavyTile)));
  p->heavy_blocks = std::min(p->ntiles, 2 * 148);
  // the weighting launch in one wave: its blocks loop over the tiles, and a
  // second wave would repeat a block's whole share (256-thread blocks of 80
  // registers: 3 per SM, so 4 x 148 blocks took 1.33 waves)
  {
    int dev = 0, sms = 148, per_sm = 1;
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_weight_tiles<T, kBtRes, kIptRes>, kBtRes, 0));
    p->weight_blocks = std::max(1, std::min(p->ntiles, std::max(1, per_sm) * sms));
  }
  CK(palloc((void**)&p->sys, (size_t)p->R * p->n_obs * sizeof(SysTable)));
  CK(palloc((void**)&p->st, (size_t)p->R * sizeof(StepState)));
  CK(palloc((void**)&p->acc, (size_t)p->R * sizeof(FilterAcc)));
  CK(cudaMemsetAsync(p->acc, 0, (size_t)p->R * sizeof(FilterAcc), s));
  // a reused plan reads its accumulator through pinned memory; a one-shot
  // filter reads it once, and pinning a page costs more than the copy
  if (p->direct) p->acc_h = new FilterAcc();
  else CK(cudaMallocHost((void**)&p->acc_h, sizeof(FilterAcc)));

  const size_t n_par = (size_t)M::N_PAR_PROC * M::N_CAC;
  if (n_par > 0) {
    CK(palloc(&p->par_cac, n_par * sizeof(T)));
    if ((rc = pupload<double>(d->par_cac, n_par, &p->par_cac_d, s))) return rc;
  }
  if ((rc = pupload_as<T>(d->cov_cac, (size_t)p->sub_total * M::N_COV_CAC * M::N_CAC, &p->cov_cac, s))) return rc;
  if (M::COUPLED) {
    if ((rc = pupload_as<T>(d->coupling, (size_t)M::N_CAC * M::N_CAC, &p->coupling, s))) return rc;
  }
  if (drift_on(d->noises_off)) {
    if ((rc = pupload_as<T>(d->drift_vol, (size_t)M::N_DRIFT * M::N_CAC, &p->drift_vol, s))) return rc;
    if ((rc = pupload<int>(d->drift_group, (size_t)M::N_DRIFT * M::N_CAC, &p->drift_group, s))) return rc;
    if ((rc = pupload<int>(d->drift_ngroups, (size_t)M::N_DRIFT, &p->drift_ngroups, s))) return rc;
    if ((rc = pupload<plomrt::BackTransform>((const plomrt::BackTransform*)d->drift_bt, (size_t)M::N_DRIFT * M::N_CAC,
                                            &p->drift_bt, s)))
      return rc;
  }
  if ((rc = pupload<double>(d->par_ts, (size_t)M::N_PAR_OBS * M::N_TS, &p->par_ts, s))) return rc;
  if ((rc = pupload<double>(d->t_sub, (size_t)p->sub_total, &p->t_sub, s))) return rc;
  if ((rc = pupload<double>(d->cov_ts, (size_t)d->n_obs * M::N_COV_TS * M::N_TS, &p->cov_ts, s))) return rc;
  {
    // data rows: at least one row so that every interval has a valid pointer
    std::vector<double> rows((size_t)(d->n_obs > 0 ? d->n_obs : 1) * M::N_TS, NAN);
    if (d->n_obs > 0) memcpy(rows.data(), d->data, (size_t)d->n_obs * M::N_TS * sizeof(double));
    if ((rc = pupload<double>(rows.data(), rows.size(), &p->data, s))) return rc;
    CK(cudaStreamSynchronize(s));
  }
  if ((rc = pupload<double>(d->x0, (size_t)M::S, &p->x0, s))) return rc;
  if (d->x0_particles && (rc = pupload<double>(d->x0_particles, (size_t)M::OFF_INC * J, &p->x0_cloud, s))) return rc;
  if (p->ode && M::N_COV_CAC > 0) {
    if ((rc = pupload<int>(d->cov_spline_meta, (size_t)3 * M::N_COV_CAC * M::N_CAC, &p->sp_meta, s))) return rc;
    if ((rc = pupload<double>(d->cov_spline_x, (size_t)d->cov_spline_knots, &p->sp_x, s))) return rc;
    if ((rc = pupload<double>(d->cov_spline_y, (size_t)d->cov_spline_knots, &p->sp_y, s))) return rc;
    if ((rc = pupload<double>(d->cov_spline_m2, (size_t)d->cov_spline_knots, &p->sp_m2, s))) return rc;
  }
  CK(palloc((void**)&p->seed, sizeof(uint64_t)));
  CK(cudaMemcpyAsync(p->seed, &d->seed, sizeof(uint64_t), cudaMemcpyHostToDevice, s));
  if (d->crn_normals) {
    const size_t nd = (size_t)J * p->sub_total * draws_per_substep(d->noises_off);
    if ((rc = pupload<double>(d->crn_normals, nd, &p->crn_tab, s))) return rc;
    if ((rc = pupload<double>(p->crn_u.data(), p->crn_u.size(), &p->crn_u_d, s))) return rc;
  }
  if (p->want_llike) {
    const size_t no = (size_t)p->R * (d->n_obs > 0 ? d->n_obs : 1);
    CK(palloc((void**)&p->llike, no * sizeof(double)));
    CK(palloc((void**)&p->ess, no * sizeof(double)));
    CK(cudaMemsetAsync(p->llike, 0, no * sizeof(double), s));
    CK(cudaMemsetAsync(p->ess, 0, no * sizeof(double), s));
  }
  if (p->mif) {
    const size_t nq = (size_t)(d->n_obs > 0 ? d->n_obs : 1) * p->Q;
    CK(palloc((void**)&p->theta_hat, (size_t)p->R * p->Q * sizeof(double)));
    CK(palloc((void**)&p->sd_init, (size_t)p->Q * sizeof(double)));
    CK(palloc((void**)&p->sd_mut, nq * sizeof(double)));
    CK(palloc((void**)&p->vt_add, nq * sizeof(double)));
    CK(palloc((void**)&p->bart, (size_t)p->R * nq * sizeof(double)));
    CK(palloc((void**)&p->vt, (size_t)p->R * nq * sizeof(double)));
    CK(cudaMemsetAsync(p->theta_hat, 0, (size_t)p->R * p->Q * sizeof(double), s));
    CK(cudaMemsetAsync(p->sd_init, 0, (size_t)p->Q * sizeof(double), s));
    CK(cudaMemsetAsync(p->sd_mut, 0, nq * sizeof(double), s));
    CK(cudaMemsetAsync(p->vt_add, 0, nq * sizeof(double), s));
    CK(cudaMemsetAsync(p->bart, 0, (size_t)p->R * nq * sizeof(double), s));
    CK(cudaMemsetAsync(p->vt, 0, (size_t)p->R * nq * sizeof(double), s));
  }
  if (p->want_anc) CK(palloc((void**)&p->anc_hist, (size_t)d->n_obs * J * sizeof(uint32_t)));
  if (p->want_xpred) CK(palloc((void**)&p->x_hist, (size_t)d->n_obs * M::S * J * sizeof(double)));
  if (p->want_anc && p->want_xpred && p->R == 1) {
    std::vector<int> idx;
    for (int n = 0; n < d->n_obs; ++n)
      if (p->weigh[n]) idx.push_back(n);
    p->n_data = (int)idx.size();
    if (!idx.empty()) {
      int rc2 = pupload<int>(idx.data(), idx.size(), &p->data_idx, s);
      if (rc2) return rc2;
    }
    CK(palloc((void**)&p->traj_t, (size_t)(d->n_obs + 2) * sizeof(int)));
    CK(palloc((void**)&p->traj_j, (size_t)(d->n_obs + 2) * sizeof(int)));
    CK(palloc((void**)&p->traj_n, sizeof(int)));
    CK(palloc((void**)&p->traj_x, (size_t)(d->n_obs + 2) * M::S * sizeof(double)));
  }
  if (p->want_hat) {
    if (p->R != 1) return fail(PLOMGPU_EINVAL, "filtered summaries need a single run");
    if (!M::POP_SIZE_EQ_SUM_SV && !d->pop_size) return fail(PLOMGPU_EINVAL, "summaries of a remainder need pop_size");
    CK(palloc((void**)&p->vals, (size_t)kHatVals * J * sizeof(double)));
    p->hat_rank[0] = (double)equal_weight_rank(J, 0.025);
    p->hat_rank[1] = (double)equal_weight_rank(J, 0.975);
    CK(palloc((void**)&p->hat, (size_t)(d->n_obs + 1) * kHatQ * 3 * sizeof(double)));
    CK(palloc((void**)&p->pred, (size_t)(d->n_obs > 0 ? d->n_obs : 1) * M::N_TS * 2 * sizeof(double)));
    CK(cudaMemsetAsync(p->pred, 0, (size_t)(d->n_obs > 0 ? d->n_obs : 1) * M::N_TS * 2 * sizeof(double), s));
    if (d->pop_size) {
      int rc2 = pupload<double>(d->pop_size, (size_t)(d->n_obs + 1) * M::N_CAC, &p->pop, s);
      if (rc2) return rc2;
    }
    if (M::N_COV_TS > 0) {
      if (!d->cov_ts0) return fail(PLOMGPU_EINVAL, "summaries of observations with covariates need cov_ts0");
      int rc3 = pupload<double>(d->cov_ts0, (size_t)M::N_COV_TS * M::N_TS, &p->cov_ts0, s);
      if (rc3) return rc3;
    }
  }
  if (p->timing) {
    p->ev.assign(2 * (size_t)d->n_obs, nullptr);
    for (auto& e : p->ev) CK(cudaEventCreate(&e));
  }
  CK(cudaStreamSynchronize(s));
  if (p->direct) return PLOMGPU_OK;

  // capture the time loop
  CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
  rc = enqueue_filter<T>(p);
  cudaGraph_t g = nullptr;
  cudaError_t ce = cudaStreamEndCapture(s, &g);
  if (rc) {
    if (g) cudaGraphDestroy(g);
    return rc;
  }
  CK(ce);
  p->graph = g;
  CK(cudaGraphInstantiate(&p->exec, g, 0));
  return PLOMGPU_OK;
}

void plan_free(plomgpu_plan* p) {
  if (!p) return;
  if (p->stream) cudaStreamSynchronize(p->stream);
  if (p->exec) cudaGraphExecDestroy(p->exec);
  if (p->graph) cudaGraphDestroy(p->graph);
  void* bufs[] = {p->X[0], p->X[1], p->lw, p->P, p->C, p->heavy, p->sys, p->crn_u_d, p->anc[0], p->anc[1], p->part, p->st, p->acc,
                  p->par_cac, p->par_cac_d, p->cov_cac, p->coupling, p->drift_vol, p->drift_group,
                  p->drift_ngroups, p->drift_bt, p->par_ts, p->t_sub, p->cov_ts, p->data, p->x0, p->crn_tab,
                  p->seed, p->llike, p->ess, p->anc_hist, p->x_hist, p->x_final, p->theta[0], p->theta[1],
                  p->theta_hat, p->sd_init, p->sd_mut, p->vt_add, p->bart, p->vt, p->theta_bt, p->proc_slot,
                  p->obs_slot, p->proc_cslot, p->obs_tslot, p->vals, p->hat, p->pred, p->pop, p->cov_ts0, p->sp_meta, p->sp_x, p->sp_y, p->sp_m2, p->data_idx, p->traj_t,
                  p->traj_j, p->traj_n, p->traj_x, p->x0_cloud, p->mx, p->vol_slot, p->x0_slot, p->pop0,
                  p->fls_out};
  for (void* b : bufs)
    if (b) cudaFreeAsync(b, p->stream);
  if (p->acc_h) {
    if (p->direct) delete p->acc_h;
    else cudaFreeHost(p->acc_h);
  }
  for (cudaEvent_t e : p->ev)
    if (e) cudaEventDestroy(e);
  if (p->stream) cudaStreamDestroy(p->stream);
  delete p;
}

// per-group component tables of iterated filtering (slots of -2)
int mif_group_tables(const plomgpu_mif_desc* mif, plomgpu_plan* p) {
  bool proc_multi = false, obs_multi = false;
  for (int k = 0; k < M::N_PAR_PROC; ++k) proc_multi |= mif->proc_slot[k] == -2;
  for (int k = 0; k < M::N_PAR_OBS; ++k) obs_multi |= mif->obs_slot[k] == -2;
  if ((proc_multi && !mif->proc_cac_slot) || (obs_multi && !mif->obs_ts_slot))
    return fail(PLOMGPU_EINVAL, "a slot of -2 needs its per-group table");
  int rc = PLOMGPU_OK;
  if (proc_multi && (rc = pupload<int>(mif->proc_cac_slot, (size_t)M::N_PAR_PROC * M::N_CAC, &p->proc_cslot, p->stream)))
    return rc;
  if (obs_multi && (rc = pupload<int>(mif->obs_ts_slot, (size_t)M::N_PAR_OBS * M::N_TS, &p->obs_tslot, p->stream)))
    return rc;
  return PLOMGPU_OK;
}

// fixed-lag smoothing and prior tables of iterated filtering
int mif_fls_tables(const plomgpu_smc_desc* d, const plomgpu_mif_desc* mif, plomgpu_plan* p) {
  const int Q = mif->n_theta;
  cudaStream_t s = p->stream;
  int rc = PLOMGPU_OK;
  if (mif->vol_slot && M::N_DRIFT > 0) {
    for (int i = 0; i < M::N_DRIFT * M::N_CAC; ++i)
      if (mif->vol_slot[i] < -1 || mif->vol_slot[i] >= Q) return fail(PLOMGPU_EINVAL, "bad vol_slot");
    if ((rc = pupload<int>(mif->vol_slot, (size_t)M::N_DRIFT * M::N_CAC, &p->vol_slot, s))) return rc;
  }
  if (mif->x0_slot) {
    if (!mif->pop0) return fail(PLOMGPU_EINVAL, "x0_slot needs pop0");
    for (int w = 0; w < M::OFF_INC; ++w)
      if (mif->x0_slot[w] < -1 || mif->x0_slot[w] >= Q) return fail(PLOMGPU_EINVAL, "bad x0_slot");
    for (int c = 0; c < M::N_CAC; ++c)
      if (!(mif->pop0[c] > 0.0)) return fail(PLOMGPU_EINVAL, "pop0 must be > 0");
    if ((rc = pupload<int>(mif->x0_slot, (size_t)M::OFF_INC, &p->x0_slot, s))) return rc;
    if ((rc = pupload<double>(mif->pop0, (size_t)M::N_CAC, &p->pop0, s))) return rc;
  }
  if (mif->prior && (!mif->prior_kind || !mif->prior_lo || !mif->prior_hi || !mif->prior_finv))
    return fail(PLOMGPU_EINVAL, "the prior patch needs prior_kind / prior_lo / prior_hi / prior_finv");
  if (p->fls_mask || mif->prior) {
    if (mif->lag < 0) return fail(PLOMGPU_EINVAL, "lag must be >= 0");
    MifTables h;
    memset(&h, 0, sizeof h);
    h.fls_mask = p->fls_mask;
    h.lag = mif->lag;
    h.prior = mif->prior ? 1 : 0;
    h.inv_nobs = d->n_obs > 0 ? 1.0 / (double)d->n_obs : 0.0;
    h.inv_lag = mif->lag > 0 ? 1.0 / (double)mif->lag : 0.0;
    for (int q = 0; q < Q && mif->prior; ++q) {
      h.prior_kind[q] = mif->prior_kind[q];
      h.prior_lo[q] = mif->prior_lo[q];
      h.prior_hi[q] = mif->prior_hi[q];
      memcpy(&h.prior_finv[q], &mif->prior_finv[q], sizeof(plomrt::BackTransform));
    }
    if ((rc = pupload<MifTables>(&h, 1, &p->mx, s))) return rc;
    CK(cudaStreamSynchronize(s));
  }
  if (p->fls_mask) {
    // the means are taken at interval L from the weights of the last weighted
    // interval up to L (the reference's weights persist over intervals without data)
    p->fls_n = -2;
    if (mif->lag < d->n_obs) {
      p->fls_n = -1;
      for (int n = 0; n <= mif->lag; ++n) {
        bool any = false;
        for (int ts = 0; ts < M::N_TS; ++ts)
          if (!isnan(d->data[(size_t)n * M::N_TS + ts])) any = true;
        if (d->filter && any) p->fls_n = n;
      }
    }
    CK(palloc((void**)&p->fls_out, (size_t)p->R * Q * sizeof(double)));
    std::vector<double> nanv((size_t)p->R * Q, NAN);
    CK(cudaMemcpy(p->fls_out, nanv.data(), nanv.size() * sizeof(double), cudaMemcpyHostToDevice));
  }
  return PLOMGPU_OK;
}

int plan_create(const plomgpu_smc_desc* d, plomgpu_plan** out, bool want_anc, bool want_xpred, bool want_final,
                bool timing = false, const plomgpu_mif_desc* mif = nullptr, bool want_hat = false,
                bool direct = false) {
  *out = nullptr;
  int rc = check_desc(d);
  if (rc) return rc;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(PLOMGPU_ENODEV, "no CUDA device");
  plomgpu_plan* p = new plomgpu_plan();
  p->J = d->J;
  p->n_obs = d->n_obs;
  p->precision = d->precision;
  p->noises_off = d->noises_off;
  p->filter = d->filter;
  p->paired = d->paired_draws != 0;
  p->crn = d->crn_normals != nullptr || p->paired;
  p->want_anc = want_anc;
  p->want_xpred = want_xpred;
  p->timing = timing;
  p->want_hat = want_hat;
  p->direct = direct;
  p->ode = d->ode != 0;
  p->psr = d->psr != 0;
  if (p->psr && (p->ode || p->crn || mif)) {
    delete p;
    return fail(PLOMGPU_EINVAL, "psr runs with Philox draws, without ode, common random numbers or iterated filtering");
  }
  if (p->ode) {
    if (mif) {
      delete p;
      return fail(PLOMGPU_EINVAL, "iterated filtering runs the stochastic implementations only");
    }
    if (!(d->eps_abs > 0.0) || !(d->eps_rel >= 0.0)) {
      delete p;
      return fail(PLOMGPU_EINVAL, "ode needs eps_abs > 0 and eps_rel >= 0");
    }
    if (M::N_COV_CAC > 0 && (!d->cov_spline_meta || !d->cov_spline_x || !d->cov_spline_y || !d->cov_spline_m2)) {
      delete p;
      return fail(PLOMGPU_EINVAL, "ode needs the covariate interpolants");
    }
    p->eps_abs = d->eps_abs;
    p->eps_rel = d->eps_rel;
  }
  if (mif) {
    p->R = mif->n_runs;
    p->mif = true;
    p->Q = mif->n_theta;
    p->est_mask = 0u;
    p->fls_mask = 0u;
    for (int q = 0; q < mif->n_theta; ++q) {
      if (mif->estimated[q]) p->est_mask |= 1u << q;
      if (mif->fls && mif->fls[q]) p->fls_mask |= 1u << q;
    }
    p->mut_mask = p->est_mask & ~p->fls_mask;
  }
  p->dt = d->dt;
  p->like_min = d->like_min;
  p->fail_b = fail_boundary(pow(d->like_min, (double)M::N_TS));
  p->log_like_min = log(d->like_min);
  p->n_sub.assign(d->n_sub, d->n_sub + d->n_obs);
  p->t_obs.assign(d->t_obs, d->t_obs + d->n_obs);
  p->sub0.resize(d->n_obs);
  p->weigh.resize(d->n_obs);
  int tot = 0;
  for (int n = 0; n < d->n_obs; ++n) {
    p->sub0[n] = tot;
    tot += d->n_sub[n];
    bool any = false;
    for (int ts = 0; ts < M::N_TS; ++ts)
      if (!isnan(d->data[(size_t)n * M::N_TS + ts])) any = true;
    p->weigh[n] = (d->filter && any) ? 1 : 0;
  }
  p->t_start.resize(d->n_obs);
  for (int n = 0; n < d->n_obs; ++n) p->t_start[n] = d->n_sub[n] > 0 ? d->t_sub[p->sub0[n]] : d->t_obs[n];
  p->sub_total = tot;
  if (d->crn_normals) p->crn_u.assign(d->crn_uniforms, d->crn_uniforms + d->n_obs);
  if (d->x0_particles && mif) {
    delete p;
    return fail(PLOMGPU_EINVAL, "initial particles one by one are for plain filters");
  }
  cudaError_t e = cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    delete p;
    return fail(PLOMGPU_ECUDA, std::string("cudaStreamCreate: ") + cudaGetErrorString(e));
  }
  g_alloc_stream = p->stream;
  if (want_final) {
    e = palloc((void**)&p->x_final, (size_t)M::S * d->J * sizeof(double));
    if (e != cudaSuccess) {
      plan_free(p);
      return fail(PLOMGPU_ENOMEM, "x_final allocation failed");
    }
  }
  if (mif) {
    int rc2;
    if ((rc2 = pupload<plomrt::BackTransform>((const plomrt::BackTransform*)mif->theta_bt, (size_t)mif->n_theta,
                                             &p->theta_bt, p->stream)) ||
        (rc2 = pupload<int>(mif->proc_slot, (size_t)(M::N_PAR_PROC > 0 ? M::N_PAR_PROC : 0), &p->proc_slot, p->stream)) ||
        (rc2 = pupload<int>(mif->obs_slot, (size_t)(M::N_PAR_OBS > 0 ? M::N_PAR_OBS : 0), &p->obs_slot, p->stream)) ||
        (rc2 = mif_group_tables(mif, p)) || (rc2 = mif_fls_tables(d, mif, p))) {
      std::string keep = g_err;
      plan_free(p);
      g_err = keep;
      return rc2;
    }
  }
  rc = (d->precision == 64) ? plan_build<double>(d, p) : plan_build<float>(d, p);
  if (rc) {
    std::string keep = g_err;
    plan_free(p);
    g_err = keep;
    return rc;
  }
  *out = p;
  return PLOMGPU_OK;
}

int plan_results(plomgpu_plan* p, plomgpu_smc_result* r) {
  CK(cudaMemcpyAsync(p->acc_h, p->acc, sizeof(FilterAcc), cudaMemcpyDeviceToHost, p->stream));
  if (r->llike_n && p->llike && p->n_obs > 0)
    CK(cudaMemcpyAsync(r->llike_n, p->llike, (size_t)p->n_obs * sizeof(double), cudaMemcpyDeviceToHost, p->stream));
  if (r->ess_n && p->ess && p->n_obs > 0)
    CK(cudaMemcpyAsync(r->ess_n, p->ess, (size_t)p->n_obs * sizeof(double), cudaMemcpyDeviceToHost, p->stream));
  if (r->ancestors && p->anc_hist)
    CK(cudaMemcpyAsync(r->ancestors, p->anc_hist, (size_t)p->n_obs * p->J * sizeof(uint32_t), cudaMemcpyDeviceToHost,
                       p->stream));
  if (r->x_pred && p->x_hist)
    CK(cudaMemcpyAsync(r->x_pred, p->x_hist, (size_t)p->n_obs * M::S * p->J * sizeof(double), cudaMemcpyDeviceToHost,
                       p->stream));
  if (r->x_final && p->x_final)
    CK(cudaMemcpyAsync(r->x_final, p->x_final, (size_t)M::S * p->J * sizeof(double), cudaMemcpyDeviceToHost,
                       p->stream));
  if (r->hat && p->hat)
    CK(cudaMemcpyAsync(r->hat, p->hat, (size_t)(p->n_obs + 1) * kHatQ * 3 * sizeof(double), cudaMemcpyDeviceToHost,
                       p->stream));
  if (r->pred_res && p->pred && p->n_obs > 0)
    CK(cudaMemcpyAsync(r->pred_res, p->pred, (size_t)p->n_obs * M::N_TS * 2 * sizeof(double), cudaMemcpyDeviceToHost,
                       p->stream));
  CK(cudaStreamSynchronize(p->stream));
  r->loglik = p->acc_h->loglik;
  r->n_all_fail = p->acc_h->n_all_fail;
  if (p->acc_h->error) {
    r->status = PLOMGPU_ETIMEOUT;
    if (p->acc_h->error & ERR_ODE) {
      r->status = PLOMGPU_EINVAL;
      return fail(PLOMGPU_EINVAL, "ode: integration time step is too small to match the desired precision");
    }
    return fail(PLOMGPU_ETIMEOUT, "systematic point table overflow");
  }
  r->status = PLOMGPU_OK;
  return PLOMGPU_OK;
}

}  // namespace

extern "C" {

int plomgpu_get_model_info(plomgpu_model_info* o) {
  if (!o) return fail(PLOMGPU_EINVAL, "null");
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
  o->n_hat = kHatQ;
  return PLOMGPU_OK;
}

int plomgpu_draws_per_substep(int noises_off) { return draws_per_substep(noises_off); }

int plomgpu_plan_create(const plomgpu_smc_desc* d, plomgpu_plan** out) {
  if (!out) return fail(PLOMGPU_EINVAL, "null output");
  return plan_create(d, out, false, false, false);
}

int plomgpu_plan_create_ex(const plomgpu_smc_desc* d, int flags, plomgpu_plan** out) {
  if (!out) return fail(PLOMGPU_EINVAL, "null output");
  const bool traj = (flags & PLOMGPU_PLAN_TRAJ) != 0;
  return plan_create(d, out, traj, traj, false, (flags & PLOMGPU_PLAN_TIMING) != 0, nullptr,
                     (flags & PLOMGPU_PLAN_SUMMARIES) != 0);
}

int plomgpu_plan_sample_traj(plomgpu_plan* p, double u, int* n_rows, int* rows_t, double* states) {
  if (!p || !n_rows || !rows_t || !states) return fail(PLOMGPU_EINVAL, "null argument");
  if (!p->traj_x) return fail(PLOMGPU_EINVAL, "plan was created without PLOMGPU_PLAN_TRAJ");
  if (p->n_data < 2) return fail(PLOMGPU_EINVAL, "trajectory sampling needs at least two intervals with data");
  cudaStream_t s = p->stream;
  if (p->precision == 64)
    k_sample_traj<double, 256><<<1, 256, 0, s>>>((const double*)p->lw, p->J, p->st, p->fail_b, u, p->n_obs,
                                                 p->data_idx, p->n_data, p->anc_hist, p->x_hist, p->x0, p->traj_t,
                                                 p->traj_j, p->traj_x, p->traj_n);
  else
    k_sample_traj<float, 256><<<1, 256, 0, s>>>((const float*)p->lw, p->J, p->st, p->fail_b, u, p->n_obs,
                                                p->data_idx, p->n_data, p->anc_hist, p->x_hist, p->x0, p->traj_t,
                                                p->traj_j, p->traj_x, p->traj_n);
  CK(cudaGetLastError());
  int n = 0;
  CK(cudaMemcpyAsync(&n, p->traj_n, sizeof(int), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  if (n < 1 || n > p->n_obs + 2) return fail(PLOMGPU_ECUDA, "trajectory walk produced a bad row count");
  CK(cudaMemcpyAsync(rows_t, p->traj_t, (size_t)n * sizeof(int), cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(states, p->traj_x, (size_t)n * M::S * sizeof(double), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  *n_rows = n;
  return PLOMGPU_OK;
}

int plomgpu_plan_propagate_time(plomgpu_plan* p, double* total_ms, int* launches) {
  if (!p || !total_ms || !launches) return fail(PLOMGPU_EINVAL, "null argument");
  if (!p->timing) return fail(PLOMGPU_EINVAL, "plan was created without PLOMGPU_PLAN_TIMING");
  CK(cudaStreamSynchronize(p->stream));
  double tot = 0.0;
  for (int n = 0; n < p->n_obs; ++n) {
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, p->ev[2 * n], p->ev[2 * n + 1]));
    tot += ms;
  }
  *total_ms = tot;
  *launches = p->n_obs;
  return PLOMGPU_OK;
}

int plomgpu_plan_update(plomgpu_plan* p, const double* par_cac, const double* par_ts, const double* x0,
                        uint64_t seed) {
  if (!p) return fail(PLOMGPU_EINVAL, "null plan");
  if (par_cac && M::N_PAR_PROC > 0)
    CK(cudaMemcpyAsync(p->par_cac_d, par_cac, (size_t)M::N_PAR_PROC * M::N_CAC * sizeof(double),
                       cudaMemcpyHostToDevice, p->stream));
  if (par_ts && M::N_PAR_OBS > 0)
    CK(cudaMemcpyAsync(p->par_ts, par_ts, (size_t)M::N_PAR_OBS * M::N_TS * sizeof(double), cudaMemcpyHostToDevice,
                       p->stream));
  if (x0) CK(cudaMemcpyAsync(p->x0, x0, (size_t)M::S * sizeof(double), cudaMemcpyHostToDevice, p->stream));
  // the seed is copied from a host temporary: make that copy synchronous w.r.t. the host
  static thread_local uint64_t seed_h;
  seed_h = seed;
  CK(cudaMemcpyAsync(p->seed, &seed_h, sizeof(uint64_t), cudaMemcpyHostToDevice, p->stream));
  CK(cudaStreamSynchronize(p->stream));
  return PLOMGPU_OK;
}

int plomgpu_plan_update_drift(plomgpu_plan* p, const double* drift_vol) {
  if (!p || !drift_vol) return fail(PLOMGPU_EINVAL, "null argument");
  if (!p->drift_vol) return PLOMGPU_OK;  // drift off for this plan: nothing reads the table
  const size_t n = (size_t)M::N_DRIFT * M::N_CAC;
  if (p->precision == 64) {
    CK(cudaMemcpyAsync(p->drift_vol, drift_vol, n * sizeof(double), cudaMemcpyHostToDevice, p->stream));
  } else {
    std::vector<float> f(drift_vol, drift_vol + n);
    CK(cudaMemcpyAsync(p->drift_vol, f.data(), n * sizeof(float), cudaMemcpyHostToDevice, p->stream));
  }
  CK(cudaStreamSynchronize(p->stream));
  return PLOMGPU_OK;
}

int plomgpu_plan_launch(plomgpu_plan* p) {
  if (!p) return fail(PLOMGPU_EINVAL, "null plan");
  if (p->direct) return (p->tsize == sizeof(double)) ? enqueue_filter<double>(p) : enqueue_filter<float>(p);
  CK(cudaGraphLaunch(p->exec, p->stream));
  return PLOMGPU_OK;
}

int plomgpu_plan_results(plomgpu_plan* p, plomgpu_smc_result* r) {
  if (!p || !r) return fail(PLOMGPU_EINVAL, "null argument");
  return plan_results(p, r);
}

void* plomgpu_plan_stream(plomgpu_plan* p) { return p ? (void*)p->stream : nullptr; }

int plomgpu_plan_kernel_count(plomgpu_plan* p) { return p ? p->kernels : 0; }

void plomgpu_plan_destroy(plomgpu_plan* p) { plan_free(p); }

int plomgpu_smc_run(const plomgpu_smc_desc* d, plomgpu_smc_result* r) {
  if (!r) return fail(PLOMGPU_EINVAL, "null result");
  plomgpu_plan* p = nullptr;
  int rc = plan_create(d, &p, r->ancestors != nullptr, r->x_pred != nullptr, r->x_final != nullptr, false, nullptr,
                       r->hat != nullptr || r->pred_res != nullptr, /*direct=*/true);
  if (rc) {
    r->status = rc;
    return rc;
  }
  rc = plomgpu_plan_launch(p);
  if (!rc) rc = plan_results(p, r);
  std::string keep = g_err;
  plan_free(p);
  g_err = keep;
  r->status = rc;
  return rc;
}

int plomgpu_release_memory(void) {
  cudaMemPool_t mp = nullptr;
  CK(plan_mem_pool(&mp));
  CK(cudaMemPoolTrimTo(mp, 0));
  return PLOMGPU_OK;
}

double plomgpu_debug_fail_boundary(double thresh) { return fail_boundary(thresh); }

int plomgpu_debug_systematic_points(double U, int J, double* out) {
  if (J < 1 || !out) return fail(PLOMGPU_EINVAL, "bad arguments");
  double* d = nullptr;
  int* err = nullptr;
  CK(cudaMalloc((void**)&d, (size_t)J * sizeof(double)));
  CK(cudaMalloc((void**)&err, sizeof(int)));
  CK(cudaMemset(err, 0, sizeof(int)));
  k_sys_points<<<1, 256>>>(U, J, d, err);
  CK(cudaGetLastError());
  int herr = 0;
  CK(cudaMemcpy(out, d, (size_t)J * sizeof(double), cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(&herr, err, sizeof(int), cudaMemcpyDeviceToHost));
  cudaFree(d);
  cudaFree(err);
  if (herr) return fail(PLOMGPU_EINVAL, "systematic point table overflow");
  return PLOMGPU_OK;
}

int plomgpu_debug_draws(int kind, int precision, double a, double b, uint64_t seed, int streams, int per_stream,
                        double* out) {
  if (kind < 0 || kind > 4 || streams < 1 || per_stream < 1 || !out) return fail(PLOMGPU_EINVAL, "bad arguments");
  if (precision != 32 && precision != 64) return fail(PLOMGPU_EINVAL, "precision must be 32 or 64");
  if ((long long)streams * per_stream > (1LL << 28)) return fail(PLOMGPU_EINVAL, "too many draws");
  const size_t n = (size_t)streams * per_stream;
  double* d = nullptr;
  CK(cudaMalloc((void**)&d, n * sizeof(double)));
  const int g = (streams + 127) / 128;
  if (precision == 32) k_debug_draws<float><<<g, 128>>>(kind, a, b, seed, streams, per_stream, d);
  else k_debug_draws<double><<<g, 128>>>(kind, a, b, seed, streams, per_stream, d);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpy(out, d, n * sizeof(double), cudaMemcpyDeviceToHost);
  cudaFree(d);
  if (e != cudaSuccess) return fail(PLOMGPU_ECUDA, std::string("debug draws: ") + cudaGetErrorString(e));
  return PLOMGPU_OK;
}

int plomgpu_particle_values(const plomgpu_smc_desc* d, const double* X, int P, const int* rows, double* out) {
  if (!d || !X || !rows || !out || P < 1) return fail(PLOMGPU_EINVAL, "bad arguments");
  for (int i = 0; i < P; ++i)
    if (rows[i] < 0 || rows[i] > d->n_obs) return fail(PLOMGPU_EINVAL, "time rows must be in [0, n_obs]");
  if (!M::POP_SIZE_EQ_SUM_SV && !d->pop_size) return fail(PLOMGPU_EINVAL, "a model with a remainder needs pop_size");
  if (M::N_COV_TS > 0 && (!d->cov_ts0 || (d->n_obs > 0 && !d->cov_ts)))
    return fail(PLOMGPU_EINVAL, "missing observation covariates");
  double *dX = nullptr, *dv = nullptr, *dpar = nullptr, *dcov = nullptr, *dcov0 = nullptr, *dpop = nullptr,
         *dt = nullptr;
  int* drows = nullptr;
  plomrt::BackTransform* dbt = nullptr;
  cudaStream_t s = 0;
  int rc = PLOMGPU_OK;
  do {
    if ((rc = upload<double>(X, (size_t)M::S * P, &dX, s))) break;
    if ((rc = upload<int>(rows, (size_t)P, &drows, s))) break;
    if (d->n_obs > 0 && (rc = upload<double>(d->t_obs, (size_t)d->n_obs, &dt, s))) break;
    if (M::N_PAR_OBS > 0 && (rc = upload<double>(d->par_ts, (size_t)M::N_PAR_OBS * M::N_TS, &dpar, s))) break;
    if (M::N_COV_TS > 0) {
      if ((rc = upload<double>(d->cov_ts0, (size_t)M::N_COV_TS * M::N_TS, &dcov0, s))) break;
      if (d->n_obs > 0 && (rc = upload<double>(d->cov_ts, (size_t)d->n_obs * M::N_COV_TS * M::N_TS, &dcov, s))) break;
    }
    if (d->pop_size && (rc = upload<double>(d->pop_size, (size_t)(d->n_obs + 1) * M::N_CAC, &dpop, s))) break;
    if (M::N_DRIFT > 0 && d->drift_bt) {
      if (cudaMalloc((void**)&dbt, (size_t)M::N_DRIFT * M::N_CAC * sizeof(plomrt::BackTransform)) != cudaSuccess ||
          cudaMemcpy(dbt, d->drift_bt, (size_t)M::N_DRIFT * M::N_CAC * sizeof(plomrt::BackTransform),
                     cudaMemcpyHostToDevice) != cudaSuccess) {
        rc = fail(PLOMGPU_ECUDA, "drift table upload failed");
        break;
      }
    }
    const size_t n_out = (size_t)(kHatQ + M::N_TS) * P;
    if (cudaMalloc((void**)&dv, n_out * sizeof(double)) != cudaSuccess) {
      rc = fail(PLOMGPU_ECUDA, "allocation failed");
      break;
    }
    const int g = (P + 255) / 256 < 4096 ? (P + 255) / 256 : 4096;
    k_particle_values<<<g, 256, 0, s>>>(dX, P, drows, dt, dpop, dpar, dcov, dcov0, dbt, dv);
    if (cudaGetLastError() != cudaSuccess ||
        cudaMemcpy(out, dv, n_out * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess)
      rc = fail(PLOMGPU_ECUDA, "particle values kernel failed");
  } while (0);
  for (void* b : {(void*)dX, (void*)dv, (void*)dpar, (void*)dcov, (void*)dcov0, (void*)dpop, (void*)dt, (void*)drows,
                  (void*)dbt})
    if (b) cudaFree(b);
  return rc;
}

const char* plomgpu_last_error(void) { return g_err.c_str(); }

}  // extern "C"

// ---------------------------------------------------------------------------
// Iterated filtering: R runs of J particles with per-particle parameters,
// advanced in lock step by one captured graph per iteration.
extern "C" int plomgpu_mif_create(const plomgpu_smc_desc* base, const plomgpu_mif_desc* m, plomgpu_mif** out) {
  if (!out || !base || !m) return fail(PLOMGPU_EINVAL, "null argument");
  *out = nullptr;
  if (m->n_runs < 1) return fail(PLOMGPU_EINVAL, "n_runs must be >= 1");
  if (m->n_theta < 1 || m->n_theta > kMaxTheta)
    return fail(PLOMGPU_EINVAL, "n_theta must be in [1, " + std::to_string(kMaxTheta) + "]");
  if (!m->theta_bt || !m->estimated || (M::N_PAR_PROC > 0 && !m->proc_slot) || (M::N_PAR_OBS > 0 && !m->obs_slot))
    return fail(PLOMGPU_EINVAL, "missing arrays");
  for (int k = 0; k < M::N_PAR_PROC; ++k) {
    const int sl = m->proc_slot[k];
    if (sl < -2 || sl >= m->n_theta) return fail(PLOMGPU_EINVAL, "bad proc_slot");
    if (sl == -2) {
      if (!m->proc_cac_slot) return fail(PLOMGPU_EINVAL, "proc_slot -2 needs proc_cac_slot");
      for (int c = 0; c < M::N_CAC; ++c) {
        const int q = m->proc_cac_slot[k * M::N_CAC + c];
        if (q < 0 || q >= m->n_theta) return fail(PLOMGPU_EINVAL, "bad proc_cac_slot");
      }
    }
  }
  for (int k = 0; k < M::N_PAR_OBS; ++k) {
    const int sl = m->obs_slot[k];
    if (sl < -2 || sl >= m->n_theta) return fail(PLOMGPU_EINVAL, "bad obs_slot");
    if (sl == -2) {
      if (!m->obs_ts_slot) return fail(PLOMGPU_EINVAL, "obs_slot -2 needs obs_ts_slot");
      for (int ts = 0; ts < M::N_TS; ++ts) {
        const int q = m->obs_ts_slot[k * M::N_TS + ts];
        if (q < 0 || q >= m->n_theta) return fail(PLOMGPU_EINVAL, "bad obs_ts_slot");
      }
    }
  }
  if (base->crn_normals) return fail(PLOMGPU_EINVAL, "iterated filtering draws its own numbers");
  if ((long long)m->n_runs * base->J > (1LL << 31) - 1) return fail(PLOMGPU_EINVAL, "n_runs * J too large");
  return plan_create(base, out, false, false, false, false, m);
}

extern "C" int plomgpu_mif_iteration(plomgpu_mif* p, const double* theta_hat, const double* sd_init,
                                     const double* sd_mut, const double* vt_add, uint64_t seed, double* loglik,
                                     int* n_all_fail, double* bart, double* vt) {
  if (!p || !p->mif) return fail(PLOMGPU_EINVAL, "not an iterated-filtering plan");
  if (!theta_hat || !sd_init || !sd_mut || !vt_add) return fail(PLOMGPU_EINVAL, "null input");
  const size_t nq = (size_t)p->n_obs * p->Q;
  cudaStream_t s = p->stream;
  CK(cudaMemcpyAsync(p->theta_hat, theta_hat, (size_t)p->R * p->Q * sizeof(double), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(p->sd_init, sd_init, (size_t)p->Q * sizeof(double), cudaMemcpyHostToDevice, s));
  if (nq) {
    CK(cudaMemcpyAsync(p->sd_mut, sd_mut, nq * sizeof(double), cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(p->vt_add, vt_add, nq * sizeof(double), cudaMemcpyHostToDevice, s));
  }
  CK(cudaMemcpyAsync(p->seed, &seed, sizeof(uint64_t), cudaMemcpyHostToDevice, s));
  CK(cudaStreamSynchronize(s));
  CK(cudaGraphLaunch(p->exec, s));
  p->acc_runs_h.resize(p->R);
  CK(cudaMemcpyAsync(p->acc_runs_h.data(), p->acc, (size_t)p->R * sizeof(FilterAcc), cudaMemcpyDeviceToHost, s));
  if (bart && nq) CK(cudaMemcpyAsync(bart, p->bart, (size_t)p->R * nq * sizeof(double), cudaMemcpyDeviceToHost, s));
  if (vt && nq) CK(cudaMemcpyAsync(vt, p->vt, (size_t)p->R * nq * sizeof(double), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  int err = 0;
  for (int r = 0; r < p->R; ++r) {
    if (loglik) loglik[r] = p->acc_runs_h[r].loglik;
    if (n_all_fail) n_all_fail[r] = p->acc_runs_h[r].n_all_fail;
    err |= p->acc_runs_h[r].error;
  }
  if (err & ERR_IC)
    return fail(PLOMGPU_EINVAL, "initial conditions: no proposal with proportions summing to at most 1 in " +
                                    std::to_string(kMaxIcAttempts) + " draws");
  if (err) return fail(PLOMGPU_ETIMEOUT, "systematic point table overflow");
  return PLOMGPU_OK;
}

extern "C" int plomgpu_mif_fls_means(plomgpu_mif* p, double* out, int* updated) {
  if (!p || !p->mif || !out) return fail(PLOMGPU_EINVAL, "bad arguments");
  if (updated) *updated = (p->fls_mask && p->fls_n != -2) ? 1 : 0;
  const size_t n = (size_t)p->R * p->Q;
  if (!p->fls_out) {
    for (size_t i = 0; i < n; ++i) out[i] = NAN;
    return PLOMGPU_OK;
  }
  CK(cudaMemcpyAsync(out, p->fls_out, n * sizeof(double), cudaMemcpyDeviceToHost, p->stream));
  CK(cudaStreamSynchronize(p->stream));
  return PLOMGPU_OK;
}

extern "C" void plomgpu_mif_destroy(plomgpu_mif* p) { plan_free(p); }

// ---------------------------------------------------------------------------
// Resampling without allocation.
//
// Some callers cannot allocate device memory: a plug-in hosted inside another
// runtime whose caching allocator owns the GPU memory (a raw cudaMalloc there
// bypasses the pool and can fail or stall once the pool holds the memory),
// and latency-bounded loops such as a serving loop, where cudaMalloc and
// cudaFree synchronise the device.  For them plomgpu_resample_noalloc runs the
// weighting / cumulative-weight / ancestor kernels of one observation interval
// on caller-owned inputs and outputs, with its scratch in the fixed array
// below instead of allocated buffers.
namespace {

constexpr int kNoAllocMaxJ = 1 << 18;  // largest particle count the fixed scratch serves
constexpr int kNoAllocBt = 256, kNoAllocIpt = 4, kNoAllocTile = kNoAllocBt * kNoAllocIpt;
constexpr int kNoAllocTiles = (kNoAllocMaxJ + kNoAllocTile - 1) / kNoAllocTile;
static_assert(kNoAllocTile <= kMaxTile, "k_resample_heavy stages a tile in shared memory");

struct NoAllocScratch {
  LseAcc part[kNoAllocTiles];
  double P[kNoAllocTiles + 1];
  StepState st;
  FilterAcc acc;
  HeavyTile heavy[kNoAllocTiles];
  double C[kNoAllocMaxJ];
};

// Shared by every call on a device and held by every GPU that loads this
// library until the process exits (about 2.1 MB).  Host code only knows its
// name; the device address belongs to the CUDA context that loaded the
// module, so it is looked up in the context current at every call.
static __device__ __align__(256) unsigned char g_noalloc_scratch[sizeof(NoAllocScratch)];

__global__ void k_noalloc_out(const StepState* st, const FilterAcc* acc, double* out) {
  out[2] = (double)st->all_fail;
  out[3] = (double)acc->error;
}

// the filters' own weighting / resampling launches (k_sys_tables,
// k_weight_tiles, k_resample_tiles, k_resample_heavy) over tiles of 1024
// particles
template <class T>
int noalloc_run(const T* lw, int J, double like_min, double u, uint32_t* anc, double* out, cudaStream_t s,
                NoAllocScratch* sc) {
  const double fail_b = fail_boundary(pow(like_min, (double)M::N_TS));
  const int ntiles = (J + kNoAllocTile - 1) / kNoAllocTile;
  // the accumulator and its ticket must start at zero; the previous call's
  // contents are still there
  k_reset_acc<<<1, 1, 0, s>>>(&sc->acc);
  k_sys_tables<<<1, 32, 0, s>>>(J, 1, 1, nullptr, 0u, nullptr, u, &sc->st.tab, &sc->acc);
  k_weight_tiles<T, kNoAllocBt, kNoAllocIpt><<<ntiles, kNoAllocBt, 0, s>>>(lw, J, ntiles, fail_b, log(like_min),
                                                                           sc->part, sc->P, &sc->st, &sc->acc, 0,
                                                                           out, out + 1, 0);
  k_resample_tiles<T, kNoAllocBt, kNoAllocIpt><<<ntiles, kNoAllocBt, 0, s>>>(
      lw, J, fail_b, sc->part, sc->P, &sc->st, &sc->st.tab, 0, anc, nullptr, sc->C, sc->heavy);
  k_resample_heavy<256><<<ntiles, 256, 0, s>>>(sc->C, J, ntiles, kNoAllocTile, &sc->st, &sc->st.tab, 0, sc->heavy,
                                               anc, nullptr);
  k_noalloc_out<<<1, 1, 0, s>>>(&sc->st, &sc->acc, out);
  CK(cudaGetLastError());
  return PLOMGPU_OK;
}

}  // namespace

extern "C" int plomgpu_resample_noalloc(const void* log_weights, int precision, int J, double like_min, double u,
                                        uint32_t* ancestors, double* out, void* stream) {
  if (!log_weights || !ancestors || !out) return fail(PLOMGPU_EINVAL, "null pointer");
  if (precision != 32 && precision != 64) return fail(PLOMGPU_EINVAL, "precision must be 32 or 64");
  if (J < 1) return fail(PLOMGPU_EINVAL, "J must be >= 1");
  if (J > kNoAllocMaxJ)
    return fail(PLOMGPU_EINVAL, "J = " + std::to_string(J) + " exceeds the no-allocation limit of " +
                                    std::to_string(kNoAllocMaxJ) + " particles");
  if (!(like_min > 0.0)) return fail(PLOMGPU_EINVAL, "like_min must be > 0");
  if (!(u >= 0.0 && u < 1.0)) return fail(PLOMGPU_EINVAL, "u must be in [0, 1)");
  // the scratch array's address in the context current now (the host-side
  // name is not a device address).  Looked up at every call rather than
  // cached per device index: a host runtime may make another context current
  // or reset the device between calls, and an address kept from an earlier
  // context would point at memory that is not this array.  The first call in
  // a context loads this library's device code there.
  void* base = nullptr;
  CK(cudaGetSymbolAddress(&base, g_noalloc_scratch));
  if (!base) return fail(PLOMGPU_ECUDA, "no device address for the no-allocation scratch");
  NoAllocScratch* sc = reinterpret_cast<NoAllocScratch*>(base);
  cudaStream_t s = (cudaStream_t)stream;
  if (precision == 64) return noalloc_run<double>((const double*)log_weights, J, like_min, u, ancestors, out, s, sc);
  return noalloc_run<float>((const float*)log_weights, J, like_min, u, ancestors, out, s, sc);
}

// ---------------------------------------------------------------------------
// Batched filters: many independent filters of one model in one persistent
// launch (see smc_batch.cuh).
#include "smc_batch.cuh"
#include <algorithm>
#include <numeric>

struct plomgpu_batch {
  int n = 0, max_obs = 0, max_J = 0, precision = 32, noises_off = 0, filter = 1;
  int bt = 0, ppt = 0, grid = 0, kernels = 1;
  double dt = 1.0, like_min = 1e-17;
  cudaStream_t stream = nullptr;
  std::vector<BatchFilter> filters_h;
  std::vector<int> order_h;
  BatchFilter* filters = nullptr;
  int* order = nullptr;
  unsigned* queue = nullptr;
  double *par_cac = nullptr, *par_ts = nullptr, *x0 = nullptr, *data = nullptr;
  int *n_sub = nullptr, *sub0 = nullptr;
  double *t_sub = nullptr, *t_obs = nullptr, *cov_ts = nullptr;
  void *cov_cac = nullptr, *coupling = nullptr, *drift_vol = nullptr;
  int *drift_group = nullptr, *drift_ngroups = nullptr;
  plomrt::BackTransform* drift_bt = nullptr;
  unsigned char* ws = nullptr;
  size_t ws_stride = 0;
  double* loglik = nullptr;
  int* n_all_fail = nullptr;
  double* ess_min = nullptr;
  int* error = nullptr;
};

namespace {

template <class T>
using BatchKernel = void (*)(const BatchArgs<T>);

template <class T, int BT, int PPT>
BatchKernel<T> pick_batch_bt(int v, bool drift) {
  if constexpr (!kSmem) {
    if (drift) {
      if constexpr (M::N_DRIFT > 0) {
        switch (v) {
          case 0: return &k_batch<T, 0, true, BT, PPT>;
          case 1: return &k_batch<T, 1, true, BT, PPT>;
          case 2: return &k_batch<T, 2, true, BT, PPT>;
          default: return &k_batch<T, 3, true, BT, PPT>;
        }
      }
      return nullptr;
    }
    switch (v) {
      case 0: return &k_batch<T, 0, false, BT, PPT>;
      case 1: return &k_batch<T, 1, false, BT, PPT>;
      case 2: return &k_batch<T, 2, false, BT, PPT>;
      default: return &k_batch<T, 3, false, BT, PPT>;
    }
  }
  return nullptr;
}

// the batched kernel of a block size and a count of particles per thread
// (FP64, the parity mode: 256 threads, one particle per thread)
template <class T>
BatchKernel<T> pick_batch(int bt, int ppt, int noises_off) {
  const int v = variant_of(noises_off);
  const bool d = drift_on(noises_off);
  if constexpr (std::is_same<T, double>::value) {
    if (bt == 256 && ppt == 1) return pick_batch_bt<T, 256, 1>(v, d);
    return nullptr;
  } else {
    if (ppt == 1) {
      switch (bt) {
        case 128: return pick_batch_bt<T, 128, 1>(v, d);
        case 256: return pick_batch_bt<T, 256, 1>(v, d);
        case 512: return pick_batch_bt<T, 512, 1>(v, d);
        default: return nullptr;
      }
    }
    if (ppt == 2) {
      switch (bt) {
        case 128: return pick_batch_bt<T, 128, 2>(v, d);
        case 256: return pick_batch_bt<T, 256, 2>(v, d);
        case 512: return pick_batch_bt<T, 512, 2>(v, d);
        default: return nullptr;
      }
    }
    return nullptr;
  }
}

template <class T>
BatchArgs<T> batch_args(plomgpu_batch* b, const BatchFilter* filters, int n, const int* order) {
  BatchArgs<T> a;
  a.filters = filters;
  a.order = order;
  a.n_filters = n;
  a.queue = b->queue;
  a.par_cac = b->par_cac;
  a.par_ts = b->par_ts;
  a.x0 = b->x0;
  a.data = b->data;
  a.n_sub = b->n_sub;
  a.sub0 = b->sub0;
  a.t_sub = b->t_sub;
  a.t_obs = b->t_obs;
  a.cov_cac = (const T*)b->cov_cac;
  a.cov_ts = b->cov_ts;
  a.coupling = (const T*)b->coupling;
  a.drift_group = b->drift_group;
  a.drift_ngroups = b->drift_ngroups;
  a.drift_bt = b->drift_bt;
  a.drift_vol = (const T*)b->drift_vol;
  a.dt = b->dt;
  a.like_min = b->like_min;
  a.fail_b = fail_boundary(pow(b->like_min, (double)M::N_TS));
  a.log_like_min = log(b->like_min);
  a.filter_on = b->filter;
  a.ws = b->ws;
  a.ws_stride = b->ws_stride;
  a.max_J = b->max_J;
  a.loglik = b->loglik;
  a.n_all_fail = b->n_all_fail;
  a.ess_min = b->ess_min;
  a.error = b->error;
  return a;
}

template <class T>
int batch_enqueue(plomgpu_batch* b, int bt, int ppt, int grid, const BatchFilter* filters, int n, const int* order) {
  BatchKernel<T> k = pick_batch<T>(bt, ppt, b->noises_off);
  if (!k) return fail(PLOMGPU_EINVAL, "no batched kernel for this block size / precision / model");
  CK(cudaMemsetAsync(b->queue, 0, sizeof(unsigned), b->stream));
  CK(cudaMemsetAsync(b->error, 0, sizeof(int), b->stream));
  k<<<grid, bt, 0, b->stream>>>(batch_args<T>(b, filters, n, order));
  CK(cudaGetLastError());
  return PLOMGPU_OK;
}

template <class T>
int batch_occupancy(int bt, int ppt, int noises_off, int* per_sm) {
  BatchKernel<T> k = pick_batch<T>(bt, ppt, noises_off);
  if (!k) return fail(PLOMGPU_EINVAL, "no batched kernel");
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, k, bt, 0));
  return PLOMGPU_OK;
}

// Picks the block size and the particles per thread (and the grid from the
// occupancy of that kernel) by timing the candidates on a sample of the
// batch: the longest filters, cut to a few intervals.
template <class T>
int batch_autotune(plomgpu_batch* b, int sms) {
  std::vector<std::pair<int, int>> cands;
  if (std::is_same<T, double>::value) {
    cands = {{256, 1}};
  } else {
    for (int bt : {128, 256, 512})
      for (int ppt : {1, 2}) cands.push_back({bt, ppt});
  }
  {
    std::vector<std::pair<int, int>> keep;
    for (auto c : cands)
      if ((b->bt <= 0 || c.first == b->bt) && (b->ppt <= 0 || c.second == b->ppt)) keep.push_back(c);
    cands = keep;
  }
  int best_bt = 0, best_ppt = 0, best_grid = 0;
  float best = 1e30f;
  // sample: enough filters to fill the largest grid twice, 12 intervals each
  std::vector<BatchFilter> sample;
  for (int i = 0; i < b->n && (int)sample.size() < 2 * sms * 8; ++i) {
    BatchFilter f = b->filters_h[b->order_h[i]];
    f.n_obs = std::min(f.n_obs, 12);
    sample.push_back(f);
  }
  std::vector<int> sorder(sample.size());
  std::iota(sorder.begin(), sorder.end(), 0);
  BatchFilter* d_sample = nullptr;
  int* d_sorder = nullptr;
  CK(cudaMalloc((void**)&d_sample, sample.size() * sizeof(BatchFilter)));
  CK(cudaMalloc((void**)&d_sorder, sorder.size() * sizeof(int)));
  CK(cudaMemcpy(d_sample, sample.data(), sample.size() * sizeof(BatchFilter), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(d_sorder, sorder.data(), sorder.size() * sizeof(int), cudaMemcpyHostToDevice));
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  int rc = PLOMGPU_OK;
  for (auto c : cands) {
    const int bt = c.first, ppt = c.second;
    int per_sm = 0;
    if ((rc = batch_occupancy<T>(bt, ppt, b->noises_off, &per_sm))) break;
    if (per_sm < 1) continue;
    const int grid = sms * per_sm;
    if (grid > b->grid) continue;  // workspace sized for b->grid
    if ((rc = batch_enqueue<T>(b, bt, ppt, grid, d_sample, (int)sample.size(), d_sorder))) break;  // warm
    CK(cudaEventRecord(e0, b->stream));
    if ((rc = batch_enqueue<T>(b, bt, ppt, grid, d_sample, (int)sample.size(), d_sorder))) break;
    CK(cudaEventRecord(e1, b->stream));
    CK(cudaEventSynchronize(e1));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, e0, e1));
    if (ms < best) {
      best = ms;
      best_bt = bt;
      best_ppt = ppt;
      best_grid = grid;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(d_sample);
  cudaFree(d_sorder);
  if (rc) return rc;
  if (!best_bt) return fail(PLOMGPU_EINVAL, "no batched configuration fits");
  b->bt = best_bt;
  b->ppt = best_ppt;
  b->grid = best_grid;
  return PLOMGPU_OK;
}

void batch_free(plomgpu_batch* b) {
  if (!b) return;
  if (b->stream) cudaStreamSynchronize(b->stream);
  void* bufs[] = {b->filters, b->order, b->queue, b->par_cac, b->par_ts, b->x0, b->data, b->n_sub, b->sub0,
                  b->t_sub, b->t_obs, b->cov_ts, b->cov_cac, b->coupling, b->drift_vol, b->drift_group,
                  b->drift_ngroups, b->drift_bt, b->ws, b->loglik, b->n_all_fail, b->ess_min, b->error};
  for (void* p : bufs)
    if (p) cudaFree(p);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
}

template <class T>
int batch_build(const plomgpu_batch_desc* d, plomgpu_batch* b) {
  cudaStream_t s = b->stream;
  int rc;
  const int n = d->n_filters;
  long long total_sub = 0;
  std::vector<int> sub0(d->max_obs);
  for (int i = 0; i < d->max_obs; ++i) {
    sub0[i] = (int)total_sub;
    total_sub += d->n_sub[i];
  }
  if ((rc = upload<BatchFilter>(b->filters_h.data(), (size_t)n, &b->filters, s))) return rc;
  if ((rc = upload<int>(b->order_h.data(), (size_t)n, &b->order, s))) return rc;
  CK(cudaMalloc((void**)&b->queue, sizeof(unsigned)));
  CK(cudaMalloc((void**)&b->error, sizeof(int)));
  if ((rc = upload<double>(d->par_cac, (size_t)n * M::N_PAR_PROC * M::N_CAC, &b->par_cac, s))) return rc;
  if ((rc = upload<double>(d->par_ts, (size_t)n * M::N_PAR_OBS * M::N_TS, &b->par_ts, s))) return rc;
  if ((rc = upload<double>(d->x0, (size_t)n * M::S, &b->x0, s))) return rc;
  if ((rc = upload<double>(d->data, (size_t)d->n_rows * M::N_TS, &b->data, s))) return rc;
  if ((rc = upload<int>(d->n_sub, (size_t)d->max_obs, &b->n_sub, s))) return rc;
  if ((rc = upload<int>(sub0.data(), (size_t)d->max_obs, &b->sub0, s))) return rc;
  if ((rc = upload<double>(d->t_sub, (size_t)total_sub, &b->t_sub, s))) return rc;
  if ((rc = upload<double>(d->t_obs, (size_t)d->max_obs, &b->t_obs, s))) return rc;
  if ((rc = upload_as<T>(d->cov_cac, (size_t)total_sub * M::N_COV_CAC * M::N_CAC, &b->cov_cac, s))) return rc;
  if ((rc = upload<double>(d->cov_ts, (size_t)d->max_obs * M::N_COV_TS * M::N_TS, &b->cov_ts, s))) return rc;
  if (M::COUPLED && (rc = upload_as<T>(d->coupling, (size_t)M::N_CAC * M::N_CAC, &b->coupling, s))) return rc;
  if (drift_on(d->noises_off)) {
    if ((rc = upload_as<T>(d->drift_vol, (size_t)M::N_DRIFT * M::N_CAC, &b->drift_vol, s))) return rc;
    if ((rc = upload<int>(d->drift_group, (size_t)M::N_DRIFT * M::N_CAC, &b->drift_group, s))) return rc;
    if ((rc = upload<int>(d->drift_ngroups, (size_t)M::N_DRIFT, &b->drift_ngroups, s))) return rc;
    if ((rc = upload<plomrt::BackTransform>((const plomrt::BackTransform*)d->drift_bt, (size_t)M::N_DRIFT * M::N_CAC,
                                            &b->drift_bt, s)))
      return rc;
  }
  CK(cudaMalloc((void**)&b->loglik, (size_t)n * sizeof(double)));
  CK(cudaMalloc((void**)&b->n_all_fail, (size_t)n * sizeof(int)));
  CK(cudaMalloc((void**)&b->ess_min, (size_t)n * sizeof(double)));
  // workspace for the largest grid any candidate block size can use
  int dev = 0, sms = 0;
  CK(cudaGetDevice(&dev));
  CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  int max_grid = 0;
  for (int bt : {128, 256, 512}) {
    for (int ppt : {1, 2}) {
      if (std::is_same<T, double>::value && (bt != 256 || ppt != 1)) continue;
      if (d->block_threads > 0 && bt != d->block_threads) continue;
      if (d->particles_per_thread > 0 && ppt != d->particles_per_thread) continue;
      int per_sm = 0;
      if ((rc = batch_occupancy<T>(bt, ppt, d->noises_off, &per_sm))) return rc;
      max_grid = std::max(max_grid, sms * per_sm);
    }
  }
  if (max_grid < 1) return fail(PLOMGPU_EINVAL, "batched kernel does not fit on the device");
  b->ws_stride = (batch_ws_bytes<T>(b->max_J) + 255) & ~(size_t)255;
  b->grid = max_grid;
  CK(cudaMalloc((void**)&b->ws, b->ws_stride * (size_t)max_grid));
  CK(cudaStreamSynchronize(s));
  b->bt = d->block_threads;
  b->ppt = d->particles_per_thread;
  if ((rc = batch_autotune<T>(b, sms))) return rc;
  return PLOMGPU_OK;
}

}  // namespace

extern "C" {

int plomgpu_batch_create(const plomgpu_batch_desc* d, plomgpu_batch** out) {
  if (!out || !d) return fail(PLOMGPU_EINVAL, "null argument");
  *out = nullptr;
  if (kSmem) return fail(PLOMGPU_EINVAL, "batched filters need a model whose particle fits registers");
  if (d->n_filters < 1) return fail(PLOMGPU_EINVAL, "n_filters must be >= 1");
  if (d->precision != 32 && d->precision != 64) return fail(PLOMGPU_EINVAL, "precision must be 32 or 64");
  if (!d->J || !d->n_obs || !d->data_row || !d->seed || !d->x0 || !d->n_sub || !d->t_obs)
    return fail(PLOMGPU_EINVAL, "missing arrays");
  if (M::COUPLED && !d->coupling) return fail(PLOMGPU_EINVAL, "coupled model needs a coupling matrix");
  if (d->block_threads != 0 && d->block_threads != 128 && d->block_threads != 256 && d->block_threads != 512)
    return fail(PLOMGPU_EINVAL, "block_threads must be 0 (autotune), 128, 256 or 512");
  if (d->particles_per_thread != 0 && d->particles_per_thread != 1 && d->particles_per_thread != 2)
    return fail(PLOMGPU_EINVAL, "particles_per_thread must be 0 (autotune), 1 or 2");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(PLOMGPU_ENODEV, "no CUDA device");
  plomgpu_batch* b = new plomgpu_batch();
  b->n = d->n_filters;
  b->max_obs = d->max_obs;
  b->precision = d->precision;
  b->noises_off = d->noises_off;
  b->filter = d->filter;
  b->dt = d->dt;
  b->like_min = d->like_min;
  b->filters_h.resize(b->n);
  for (int i = 0; i < b->n; ++i) {
    if (d->J[i] < 1 || d->n_obs[i] < 0 || d->n_obs[i] > d->max_obs) {
      delete b;
      return fail(PLOMGPU_EINVAL, "filter " + std::to_string(i) + ": bad J or n_obs");
    }
    if (d->data_row[i] < 0 || d->data_row[i] + d->n_obs[i] > d->n_rows) {
      delete b;
      return fail(PLOMGPU_EINVAL, "filter " + std::to_string(i) + ": data rows out of range");
    }
    b->filters_h[i] = BatchFilter{d->J[i], d->n_obs[i], d->data_row[i], d->seed[i]};
    b->max_J = std::max(b->max_J, d->J[i]);
  }
  // longest filters first (list scheduling over the persistent CTAs)
  b->order_h.resize(b->n);
  std::iota(b->order_h.begin(), b->order_h.end(), 0);
  std::stable_sort(b->order_h.begin(), b->order_h.end(), [&](int x, int y) {
    return (long long)b->filters_h[x].J * b->filters_h[x].n_obs > (long long)b->filters_h[y].J * b->filters_h[y].n_obs;
  });
  cudaError_t e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    delete b;
    return fail(PLOMGPU_ECUDA, std::string("cudaStreamCreate: ") + cudaGetErrorString(e));
  }
  int rc = (d->precision == 64) ? batch_build<double>(d, b) : batch_build<float>(d, b);
  if (rc) {
    std::string keep = g_err;
    batch_free(b);
    g_err = keep;
    return rc;
  }
  *out = b;
  return PLOMGPU_OK;
}

int plomgpu_batch_launch(plomgpu_batch* b) {
  if (!b) return fail(PLOMGPU_EINVAL, "null batch");
  return (b->precision == 64) ? batch_enqueue<double>(b, b->bt, b->ppt, b->grid, b->filters, b->n, b->order)
                              : batch_enqueue<float>(b, b->bt, b->ppt, b->grid, b->filters, b->n, b->order);
}

int plomgpu_batch_results(plomgpu_batch* b, double* loglik, int* n_all_fail, double* ess_min) {
  if (!b) return fail(PLOMGPU_EINVAL, "null batch");
  int err = 0;
  if (loglik) CK(cudaMemcpyAsync(loglik, b->loglik, (size_t)b->n * sizeof(double), cudaMemcpyDeviceToHost, b->stream));
  if (n_all_fail)
    CK(cudaMemcpyAsync(n_all_fail, b->n_all_fail, (size_t)b->n * sizeof(int), cudaMemcpyDeviceToHost, b->stream));
  if (ess_min) CK(cudaMemcpyAsync(ess_min, b->ess_min, (size_t)b->n * sizeof(double), cudaMemcpyDeviceToHost, b->stream));
  CK(cudaMemcpyAsync(&err, b->error, sizeof(int), cudaMemcpyDeviceToHost, b->stream));
  CK(cudaStreamSynchronize(b->stream));
  if (err) return fail(PLOMGPU_ETIMEOUT, "systematic point table overflow");
  return PLOMGPU_OK;
}

void* plomgpu_batch_stream(plomgpu_batch* b) { return b ? (void*)b->stream : nullptr; }

int plomgpu_batch_config(plomgpu_batch* b, int* block_threads, int* particles_per_thread, int* grid) {
  if (!b) return fail(PLOMGPU_EINVAL, "null batch");
  if (block_threads) *block_threads = b->bt;
  if (particles_per_thread) *particles_per_thread = b->ppt;
  if (grid) *grid = b->grid;
  return PLOMGPU_OK;
}

void plomgpu_batch_destroy(plomgpu_batch* b) { batch_free(b); }

int plomgpu_batch_run(const plomgpu_batch_desc* d, double* loglik, int* n_all_fail) {
  plomgpu_batch* b = nullptr;
  int rc = plomgpu_batch_create(d, &b);
  if (rc) return rc;
  rc = plomgpu_batch_launch(b);
  if (!rc) rc = plomgpu_batch_results(b, loglik, n_all_fail, nullptr);
  std::string keep = g_err;
  batch_free(b);
  g_err = keep;
  return rc;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Likelihood server (see serve_host.cuh / smc_serve.cuh).
#include "serve_host.cuh"

namespace {

template <class T>
int server_build(plomgpu_server* sv, int dev) {
  cudaStream_t s = sv->stream;
  int rc;
  const plomgpu_smc_desc& d = sv->base;
  std::vector<int> sub0(d.n_obs);
  long long tot = 0;
  for (int n = 0; n < d.n_obs; ++n) {
    sub0[n] = (int)tot;
    tot += d.n_sub[n];
  }
  if ((rc = upload<int>(d.n_sub, (size_t)d.n_obs, &sv->d_n_sub, s))) return rc;
  if ((rc = upload<int>(sub0.data(), sub0.size(), &sv->d_sub0, s))) return rc;
  if ((rc = upload<double>(d.t_sub, (size_t)tot, &sv->d_t_sub, s))) return rc;
  if ((rc = upload<double>(d.t_obs, (size_t)d.n_obs, &sv->d_t_obs, s))) return rc;
  if ((rc = upload<double>(d.data, (size_t)d.n_obs * M::N_TS, &sv->d_data, s))) return rc;
  if ((rc = upload_as<T>(d.cov_cac, (size_t)tot * M::N_COV_CAC * M::N_CAC, &sv->d_cov_cac, s))) return rc;
  if ((rc = upload<double>(d.cov_ts, (size_t)d.n_obs * M::N_COV_TS * M::N_TS, &sv->d_cov_ts, s))) return rc;
  if (M::COUPLED && (rc = upload_as<T>(d.coupling, (size_t)M::N_CAC * M::N_CAC, &sv->d_coupling, s))) return rc;
  if (drift_on(d.noises_off)) {
    if ((rc = upload_as<T>(d.drift_vol, (size_t)M::N_DRIFT * M::N_CAC, &sv->d_drift_vol, s))) return rc;
    if ((rc = upload<int>(d.drift_group, (size_t)M::N_DRIFT * M::N_CAC, &sv->d_drift_group, s))) return rc;
    if ((rc = upload<int>(d.drift_ngroups, (size_t)M::N_DRIFT, &sv->d_drift_ngroups, s))) return rc;
    if ((rc = upload<plomrt::BackTransform>((const plomrt::BackTransform*)d.drift_bt, (size_t)M::N_DRIFT * M::N_CAC,
                                            &sv->d_drift_bt, s)))
      return rc;
  }
  CK(cudaMalloc((void**)&sv->d_error, sizeof(int)));
  CK(cudaMemsetAsync(sv->d_error, 0, sizeof(int), s));
  CK(cudaHostAlloc((void**)&sv->slots_h, (size_t)sv->ring * sizeof(ServeSlot), cudaHostAllocMapped | cudaHostAllocPortable));
  CK(cudaHostAlloc((void**)&sv->ctl_h, sizeof(ServeCtl), cudaHostAllocMapped | cudaHostAllocPortable));
  CK(cudaHostAlloc((void**)&sv->map_h, (size_t)sv->ring * sizeof(int), cudaHostAllocMapped | cudaHostAllocPortable));
  memset(sv->slots_h, 0, (size_t)sv->ring * sizeof(ServeSlot));
  memset(sv->ctl_h, 0, sizeof(ServeCtl));
  memset(sv->map_h, 0, (size_t)sv->ring * sizeof(int));
  CK(cudaHostGetDevicePointer((void**)&sv->slots_d, sv->slots_h, 0));
  CK(cudaHostGetDevicePointer((void**)&sv->ctl_d, sv->ctl_h, 0));
  if (sv->tiled) {
    CK(cudaMalloc((void**)&sv->ctl_dev, sizeof(ServeCtl)));
    CK(cudaMemsetAsync(sv->ctl_dev, 0, sizeof(ServeCtl), s));
    int lo = 0, hi = 0;
    CK(cudaDeviceGetStreamPriorityRange(&lo, &hi));
    CK(cudaStreamCreateWithPriority(&sv->ctl_stream, cudaStreamNonBlocking, hi));
  }
  CK(cudaHostGetDevicePointer((void**)&sv->map_d, sv->map_h, 0));
  CK(cudaMalloc((void**)&sv->d_head, sizeof(unsigned long long)));
  CK(cudaMemsetAsync(sv->d_head, 0, sizeof(unsigned long long), s));
  size_t free_b = 0, total_b = 0;
  CK(cudaMemGetInfo(&free_b, &total_b));
  size_t pool = std::min(sv->budget, (size_t)sv->ring * serve_ws_bytes(sv, sv->max_J));
  pool = std::min(pool, (size_t)(0.8 * (double)free_b));
  if (pool < serve_ws_bytes(sv, sv->max_J)) return fail(PLOMGPU_ENOMEM, "memory budget below one request");
  CK(cudaMalloc((void**)&sv->d_pool, pool));
  sv->pool.init(pool);
  int sms = 0, per_sm = 0;
  CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  if (sv->tiled) {
    ServeTilesKernel<T> k = pick_serve_tiles<T>(d.noises_off);
    if (!k) return fail(PLOMGPU_EINVAL, "no serving kernel for this model");
    sv->bt = kBtProp;
    sv->tiles_smem = serve_tiles_smem<T, kBtProp>();
    if (sv->tiles_smem > 48 * 1024)
      CK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sv->tiles_smem));
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, sv->bt, sv->tiles_smem));
    CK(cudaMalloc((void**)&sv->d_live, (size_t)kServeLive * sizeof(long long)));
    CK(cudaMemsetAsync(sv->d_live, 0xff, (size_t)kServeLive * sizeof(long long), s));  // -1: free
  } else {
    ServeKernel<T> k = pick_serve<T>(d.noises_off);
    if (!k) return fail(PLOMGPU_EINVAL, "no serving kernel for this model");
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, sv->bt, 0));
  }
  sv->grid = sms * std::max(per_sm, 1);
  CK(cudaStreamSynchronize(s));
  return PLOMGPU_OK;
}

void server_free(plomgpu_server* sv) {
  if (!sv) return;
  {
    std::lock_guard<std::mutex> lock(sv->mu);
    sv->stop = true;
  }
  sv->cv.notify_all();
  if (sv->worker.joinable()) sv->worker.join();
  if (sv->ctl_h) __atomic_store_n(&sv->ctl_h->stop, 1, __ATOMIC_RELEASE);
  if (sv->ctl_dev && sv->ctl_stream) {
    cudaMemcpyAsync(&sv->ctl_dev->stop, &sv->ctl_h->stop, sizeof(int), cudaMemcpyHostToDevice, sv->ctl_stream);
    cudaStreamSynchronize(sv->ctl_stream);
  }
  for (int i = 1; i < plomgpu_server::kLoops; ++i)
    if (sv->loop_stream[i]) cudaStreamSynchronize(sv->loop_stream[i]);
  if (sv->stream) cudaStreamSynchronize(sv->stream);
  for (auto& pp : sv->plans) {
    if (pp.plan) plan_free(pp.plan);
    if (pp.done_ev) cudaEventDestroy(pp.done_ev);
  }
  void* bufs[] = {sv->d_n_sub, sv->d_sub0, sv->d_t_sub, sv->d_t_obs, sv->d_cov_ts, sv->d_data, sv->d_cov_cac,
                  sv->d_coupling, sv->d_drift_vol, sv->d_drift_group, sv->d_drift_ngroups, sv->d_drift_bt,
                  sv->d_error, sv->d_head, sv->d_pool, sv->d_live, sv->ctl_dev};
  for (void* b : bufs)
    if (b) cudaFree(b);
  if (sv->slots_h) cudaFreeHost(sv->slots_h);
  if (sv->ctl_h) cudaFreeHost(sv->ctl_h);
  if (sv->map_h) cudaFreeHost(sv->map_h);
  for (int i = 1; i < plomgpu_server::kLoops; ++i) {
    if (sv->loop_ev[i]) cudaEventDestroy(sv->loop_ev[i]);
    if (sv->loop_stream[i]) cudaStreamDestroy(sv->loop_stream[i]);
  }
  if (sv->ctl_stream) cudaStreamDestroy(sv->ctl_stream);
  if (sv->kernel_ev) cudaEventDestroy(sv->kernel_ev);
  if (sv->stream) cudaStreamDestroy(sv->stream);
  delete sv;
}

}  // namespace

extern "C" {

int plomgpu_server_create(const plomgpu_smc_desc* d, const plomgpu_server_opts* o, plomgpu_server** out) {
  if (!d || !o || !out) return fail(PLOMGPU_EINVAL, "null argument");
  *out = nullptr;
  if (o->max_J < 1) return fail(PLOMGPU_EINVAL, "max_J must be >= 1");
  if (d->ode || d->psr) return fail(PLOMGPU_EINVAL, "the server runs the sde implementation only");
  plomgpu_smc_desc chk = *d;
  chk.J = o->max_J;
  chk.crn_normals = nullptr;
  chk.crn_uniforms = nullptr;
  chk.paired_draws = 0;
  chk.x0_particles = nullptr;
  chk.precision = o->precision;
  int rc = check_desc(&chk);
  if (rc) return rc;
  int dev = 0, ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(PLOMGPU_ENODEV, "no CUDA device");
  CK(cudaGetDevice(&dev));
  plomgpu_server* sv = new plomgpu_server();
  sv->precision = o->precision;
  sv->max_J = o->max_J;
  sv->ring = o->ring_slots > 0 ? o->ring_slots : 1024;
  sv->plan_pool = o->plan_pool > 0 ? o->plan_pool : 4;
  sv->task_budget = o->task_budget == 0 ? 64 : (o->task_budget < 0 ? 0 : o->task_budget);
  if (kSmem && o->use_plan_pool) {
    sv->persistent = false;
    sv->tiled = false;
  }
  sv->budget = o->memory_budget > 0 ? (size_t)o->memory_budget : (size_t)150e9;
  // keep host copies of the shared problem
  const int n = d->n_obs;
  long long tot = 0;
  for (int i = 0; i < n; ++i) tot += d->n_sub[i];
  sv->n_sub_h.assign(d->n_sub, d->n_sub + n);
  sv->t_sub_h.assign(d->t_sub, d->t_sub + tot);
  sv->t_obs_h.assign(d->t_obs, d->t_obs + n);
  sv->data_h.assign(d->data, d->data + (size_t)n * M::N_TS);
  if (d->cov_cac) sv->cov_cac_h.assign(d->cov_cac, d->cov_cac + (size_t)tot * M::N_COV_CAC * M::N_CAC);
  if (d->cov_ts) sv->cov_ts_h.assign(d->cov_ts, d->cov_ts + (size_t)n * M::N_COV_TS * M::N_TS);
  if (d->coupling) sv->coupling_h.assign(d->coupling, d->coupling + (size_t)M::N_CAC * M::N_CAC);
  if (drift_on(d->noises_off)) {
    sv->drift_vol_h.assign(d->drift_vol, d->drift_vol + (size_t)M::N_DRIFT * M::N_CAC);
    sv->drift_group_h.assign(d->drift_group, d->drift_group + (size_t)M::N_DRIFT * M::N_CAC);
    sv->drift_ngroups_h.assign(d->drift_ngroups, d->drift_ngroups + M::N_DRIFT);
    sv->drift_bt_h.assign(d->drift_bt, d->drift_bt + (size_t)M::N_DRIFT * M::N_CAC);
  }
  sv->par_cac_h.assign(d->par_cac, d->par_cac + (size_t)M::N_PAR_PROC * M::N_CAC);
  sv->par_ts_h.assign(d->par_ts, d->par_ts + (size_t)M::N_PAR_OBS * M::N_TS);
  sv->x0_h.assign(d->x0, d->x0 + M::S);
  sv->base = *d;
  sv->base.precision = o->precision;
  sv->base.crn_normals = nullptr;
  sv->base.crn_uniforms = nullptr;
  sv->base.paired_draws = 0;
  sv->base.x0_particles = nullptr;
  sv->base.n_sub = sv->n_sub_h.data();
  sv->base.t_sub = sv->t_sub_h.data();
  sv->base.t_obs = sv->t_obs_h.data();
  sv->base.data = sv->data_h.data();
  sv->base.cov_cac = sv->cov_cac_h.empty() ? nullptr : sv->cov_cac_h.data();
  sv->base.cov_ts = sv->cov_ts_h.empty() ? nullptr : sv->cov_ts_h.data();
  sv->base.coupling = sv->coupling_h.empty() ? nullptr : sv->coupling_h.data();
  sv->base.drift_vol = sv->drift_vol_h.empty() ? nullptr : sv->drift_vol_h.data();
  sv->base.drift_group = sv->drift_group_h.empty() ? nullptr : sv->drift_group_h.data();
  sv->base.drift_ngroups = sv->drift_ngroups_h.empty() ? nullptr : sv->drift_ngroups_h.data();
  sv->base.drift_bt = sv->drift_bt_h.empty() ? nullptr : sv->drift_bt_h.data();
  sv->base.par_cac = sv->par_cac_h.data();
  sv->base.par_ts = sv->par_ts_h.data();
  sv->base.x0 = sv->x0_h.data();
  // the tiled loop fills whatever the GPU leaves free (lowest priority); a
  // one-CTA-per-request loop serves small, latency-bound requests (highest)
  int prio_low = 0, prio_high = 0;
  cudaDeviceGetStreamPriorityRange(&prio_low, &prio_high);
  const int prio = sv->tiled ? prio_low : prio_high;
  cudaError_t e = cudaStreamCreateWithPriority(&sv->stream, cudaStreamNonBlocking, prio);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&sv->kernel_ev, cudaEventDisableTiming);
  if (e == cudaSuccess) {
    sv->loop_stream[0] = sv->stream;
    sv->loop_ev[0] = sv->kernel_ev;
    for (int i = 1; i < plomgpu_server::kLoops && e == cudaSuccess; ++i) {
      e = cudaStreamCreateWithPriority(&sv->loop_stream[i], cudaStreamNonBlocking, prio);
      if (e == cudaSuccess) e = cudaEventCreateWithFlags(&sv->loop_ev[i], cudaEventDisableTiming);
    }
  }
  if (e != cudaSuccess) {
    server_free(sv);
    return fail(PLOMGPU_ECUDA, std::string("stream/event: ") + cudaGetErrorString(e));
  }
  if (sv->persistent) {
    rc = (o->precision == 64) ? server_build<double>(sv, dev) : server_build<float>(sv, dev);
    if (rc) {
      std::string keep = g_err;
      server_free(sv);
      g_err = keep;
      return rc;
    }
    sv->slot_ticket.assign(sv->ring, -1);
    sv->slot_off.assign(sv->ring, 0);
    sv->slot_bytes.assign(sv->ring, 0);
    sv->slot_t.assign(sv->ring, Clock::now());
    for (int i = 0; i < sv->ring; ++i) sv->free_slots.push_back(i);
  }
  sv->worker = std::thread([sv, dev]() {
    cudaSetDevice(dev);
    serve_loop(sv);
  });
  *out = sv;
  return PLOMGPU_OK;
}

int plomgpu_server_submit(plomgpu_server* sv, int J, const double* par_cac, const double* par_ts, const double* x0,
                          uint64_t seed, long long* ticket) {
  if (!sv || !ticket) return fail(PLOMGPU_EINVAL, "null argument");
  if (J < 1 || J > sv->max_J) return fail(PLOMGPU_EINVAL, "J out of range [1, max_J]");
  ServeRequest rq;
  rq.J = J;
  rq.seed = seed;
  rq.par_cac.assign(par_cac ? par_cac : sv->par_cac_h.data(),
                    (par_cac ? par_cac : sv->par_cac_h.data()) + (size_t)M::N_PAR_PROC * M::N_CAC);
  rq.par_ts.assign(par_ts ? par_ts : sv->par_ts_h.data(),
                   (par_ts ? par_ts : sv->par_ts_h.data()) + (size_t)M::N_PAR_OBS * M::N_TS);
  rq.x0.assign(x0 ? x0 : sv->x0_h.data(), (x0 ? x0 : sv->x0_h.data()) + M::S);
  rq.t_submit = Clock::now();
  {
    std::lock_guard<std::mutex> lock(sv->mu);
    rq.ticket = sv->next_ticket++;
    *ticket = rq.ticket;
    sv->results[rq.ticket] = ServeResult();
    sv->pending.push_back(std::move(rq));
  }
  sv->cv.notify_all();
  return PLOMGPU_OK;
}

int plomgpu_server_poll(plomgpu_server* sv, long long ticket, int* done, double* loglik, int* n_all_fail,
                        double* latency_s) {
  if (!sv || !done) return fail(PLOMGPU_EINVAL, "null argument");
  std::lock_guard<std::mutex> lock(sv->mu);
  auto it = sv->results.find(ticket);
  if (it == sv->results.end()) return fail(PLOMGPU_EINVAL, "unknown ticket");
  *done = it->second.done ? 1 : 0;
  if (it->second.done) {
    if (loglik) *loglik = it->second.loglik;
    if (n_all_fail) *n_all_fail = it->second.n_all_fail;
    if (latency_s) *latency_s = it->second.latency_s;
    if (it->second.status) return fail(it->second.status, "request failed");
  }
  return PLOMGPU_OK;
}

int plomgpu_server_wait(plomgpu_server* sv, long long ticket, double timeout_s, double* loglik, int* n_all_fail,
                        double* latency_s) {
  if (!sv) return fail(PLOMGPU_EINVAL, "null argument");
  std::unique_lock<std::mutex> lock(sv->mu);
  auto it = sv->results.find(ticket);
  if (it == sv->results.end()) return fail(PLOMGPU_EINVAL, "unknown ticket");
  const auto until = Clock::now() + std::chrono::duration<double>(timeout_s);
  while (!sv->results[ticket].done) {
    if (sv->cv_done.wait_until(lock, until) == std::cv_status::timeout && !sv->results[ticket].done)
      return fail(PLOMGPU_ETIMEOUT, "request not finished before the timeout");
  }
  const ServeResult& r = sv->results[ticket];
  if (loglik) *loglik = r.loglik;
  if (n_all_fail) *n_all_fail = r.n_all_fail;
  if (latency_s) *latency_s = r.latency_s;
  if (r.status) return fail(r.status, "request failed");
  return PLOMGPU_OK;
}

int plomgpu_server_get_stats(plomgpu_server* sv, plomgpu_server_stats* st) {
  if (!sv || !st) return fail(PLOMGPU_EINVAL, "null argument");
  std::lock_guard<std::mutex> lock(sv->mu);
  st->pending = (long long)sv->pending.size();
  st->in_flight = sv->in_flight;
  st->completed = sv->completed;
  st->launches = sv->launches;
  st->peak_in_flight = sv->peak_in_flight;
  st->bytes_in_use = (double)(sv->pool.used + sv->plan_bytes_total);
  st->peak_bytes = (double)(sv->pool.peak + sv->plan_bytes_total);
  st->persistent_loop = sv->persistent ? 1 : 0;
  return PLOMGPU_OK;
}

void plomgpu_server_destroy(plomgpu_server* sv) { server_free(sv); }

}  // extern "C"
