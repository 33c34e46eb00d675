// Host side of the likelihood server (plomgpu_server_*): request queue,
// admission by HBM footprint, the persistent device loops (smc_serve.cuh):
// one CTA per request for models whose particle fits registers, tiles of
// particles for the others; a pool of captured plans (one stream each)
// remains as an option.  Included by plomgpu_api.cu.
#pragma once

#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <thread>

#include "smc_serve.cuh"

namespace {

using Clock = std::chrono::steady_clock;

struct ServeRequest {
  long long ticket;
  int J;
  uint64_t seed;
  std::vector<double> par_cac, par_ts, x0;
  Clock::time_point t_submit;
};

struct ServeResult {
  bool done = false;
  int status = PLOMGPU_OK;
  double loglik = 0.0;
  int n_all_fail = 0;
  double latency_s = 0.0;
};

// first-fit allocator over [0, size)
struct PoolAlloc {
  std::map<size_t, size_t> free_;  // offset -> bytes
  size_t used = 0, peak = 0;
  void init(size_t size) {
    free_.clear();
    free_[0] = size;
    used = peak = 0;
  }
  bool alloc(size_t bytes, size_t* off) {
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second >= bytes) {
        *off = it->first;
        const size_t rest = it->second - bytes;
        const size_t o = it->first;
        free_.erase(it);
        if (rest) free_[o + bytes] = rest;
        used += bytes;
        peak = std::max(peak, used);
        return true;
      }
    }
    return false;
  }
  void release(size_t off, size_t bytes) {
    used -= bytes;
    auto it = free_.emplace(off, bytes).first;
    auto nx = std::next(it);
    if (nx != free_.end() && it->first + it->second == nx->first) {
      it->second += nx->second;
      free_.erase(nx);
    }
    if (it != free_.begin()) {
      auto pv = std::prev(it);
      if (pv->first + pv->second == it->first) {
        pv->second += it->second;
        free_.erase(it);
      }
    }
  }
};

struct PooledPlan {
  plomgpu_plan* plan = nullptr;
  int J = 0;
  size_t bytes = 0;
  bool busy = false;
  long long ticket = -1;
  Clock::time_point t_submit;
  cudaEvent_t done_ev = nullptr;
};

}  // namespace

struct plomgpu_server {
  // configuration
  int precision = 32, max_J = 0, ring = 1024, plan_pool = 4;
  size_t budget = 0;
  bool persistent = true;
  bool tiled = kSmem;           // the tiled loop (shared-memory particles)
  size_t tiles_smem = 0;        // its dynamic shared memory
  long long* d_live = nullptr;  // its live-request table [kServeLive]
  int task_budget = 64;         // tasks a CTA of the tiled loop runs before it returns
  int bt = 256, grid = 0;
  long long idle_limit = 20000;  // microseconds a loop CTA waits for work before it returns
  // base problem (host copies; every request shares it)
  plomgpu_smc_desc base{};
  std::vector<int> n_sub_h;
  std::vector<double> t_sub_h, t_obs_h, data_h, cov_cac_h, cov_ts_h, coupling_h, drift_vol_h, par_cac_h, par_ts_h, x0_h;
  std::vector<int> drift_group_h, drift_ngroups_h;
  std::vector<plomgpu_back_transform> drift_bt_h;
  // device copies for the persistent loop
  void* d_args_storage = nullptr;
  int* d_n_sub = nullptr;
  int* d_sub0 = nullptr;
  double *d_t_sub = nullptr, *d_t_obs = nullptr, *d_cov_ts = nullptr, *d_data = nullptr;
  void *d_cov_cac = nullptr, *d_coupling = nullptr, *d_drift_vol = nullptr;
  int *d_drift_group = nullptr, *d_drift_ngroups = nullptr, *d_error = nullptr;
  plomrt::BackTransform* d_drift_bt = nullptr;
  ServeSlot* slots_h = nullptr;  // mapped
  ServeSlot* slots_d = nullptr;
  ServeCtl* ctl_h = nullptr;     // mapped
  ServeCtl* ctl_d = nullptr;
  // a device-memory copy of the control block for the tiled loop, refreshed
  // by a small copy after every publication: its CTAs poll device memory,
  // not the host's
  ServeCtl* ctl_dev = nullptr;
  cudaStream_t ctl_stream = nullptr;
  int* map_h = nullptr;          // mapped: ring position -> slot
  int* map_d = nullptr;
  unsigned long long* d_head = nullptr;
  unsigned char* d_pool = nullptr;
  PoolAlloc pool;
  cudaStream_t stream = nullptr;
  cudaEvent_t kernel_ev = nullptr;
  bool kernel_live = false;
  // Instances of the device loop.  Each is launched with about as many CTAs
  // as requests wait for one (at least 8, and at least half the live CTAs so
  // that a burst is met in a few launches; never more than `grid`, the CTAs
  // the GPU holds at once), so that a loop serving a few requests leaves the
  // other SMs to other work; a backlog beyond the live CTAs starts another
  // instance on the next stream, and CTAs that find no work for a while
  // return.  Instance 0 uses `stream` / `kernel_ev`.
  static constexpr int kLoops = 8;
  cudaStream_t loop_stream[kLoops] = {};
  cudaEvent_t loop_ev[kLoops] = {};
  int loop_grid[kLoops] = {};
  bool loop_live[kLoops] = {};
  unsigned long long published = 0;
  unsigned long long pushed_tail = 0;  // tail last copied to ctl_dev
  std::vector<long long> slot_ticket;  // ring slot -> ticket (-1 free)
  std::vector<size_t> slot_off, slot_bytes;
  std::vector<Clock::time_point> slot_t;
  std::deque<int> free_slots;
  // plan pool (models served per plan)
  std::vector<PooledPlan> plans;
  size_t plan_bytes_total = 0;
  // queues
  std::mutex mu;
  std::condition_variable cv, cv_done;
  std::deque<ServeRequest> pending;
  std::map<long long, ServeResult> results;
  long long next_ticket = 0;
  bool stop = false;
  std::thread worker;
  // statistics
  long long launches = 0, completed = 0, in_flight = 0, peak_in_flight = 0;
  std::string last_error;
};

namespace {

template <class T>
BatchArgs<T> serve_args(plomgpu_server* sv) {
  BatchArgs<T> a{};
  a.data = sv->d_data;
  a.n_sub = sv->d_n_sub;
  a.sub0 = sv->d_sub0;
  a.t_sub = sv->d_t_sub;
  a.t_obs = sv->d_t_obs;
  a.cov_cac = (const T*)sv->d_cov_cac;
  a.cov_ts = sv->d_cov_ts;
  a.coupling = (const T*)sv->d_coupling;
  a.drift_group = sv->d_drift_group;
  a.drift_ngroups = sv->d_drift_ngroups;
  a.drift_bt = sv->d_drift_bt;
  a.drift_vol = (const T*)sv->d_drift_vol;
  a.dt = sv->base.dt;
  a.like_min = sv->base.like_min;
  a.fail_b = fail_boundary(pow(sv->base.like_min, (double)M::N_TS));
  a.log_like_min = log(sv->base.like_min);
  a.filter_on = sv->base.filter;
  a.error = sv->d_error;
  return a;
}

template <class T>
using ServeKernel = void (*)(const BatchArgs<T>, ServeSlot*, const int*, int, ServeCtl*, unsigned long long*,
                             unsigned char*, long long);

template <class T>
ServeKernel<T> pick_serve(int noises_off) {
  if constexpr (!kSmem) {
    const int v = variant_of(noises_off);
    if (drift_on(noises_off)) {
      if constexpr (M::N_DRIFT > 0) {
        switch (v) {
          case 0: return &k_serve<T, 0, true, 256>;
          case 1: return &k_serve<T, 1, true, 256>;
          case 2: return &k_serve<T, 2, true, 256>;
          default: return &k_serve<T, 3, true, 256>;
        }
      }
      return nullptr;
    }
    switch (v) {
      case 0: return &k_serve<T, 0, false, 256>;
      case 1: return &k_serve<T, 1, false, 256>;
      case 2: return &k_serve<T, 2, false, 256>;
      default: return &k_serve<T, 3, false, 256>;
    }
  }
  return nullptr;
}

template <class T>
using ServeTilesKernel = void (*)(const BatchArgs<T>, ServeSlot*, const int*, int, ServeCtl*, unsigned long long*,
                                  unsigned char*, long long*, long long, int);

template <class T>
ServeTilesKernel<T> pick_serve_tiles(int noises_off) {
  if constexpr (kSmem) {
    const int v = variant_of(noises_off);
    if (drift_on(noises_off)) {
      if constexpr (M::N_DRIFT > 0) {
        switch (v) {
          case 0: return &k_serve_tiles<T, 0, true, kBtProp>;
          case 1: return &k_serve_tiles<T, 1, true, kBtProp>;
          case 2: return &k_serve_tiles<T, 2, true, kBtProp>;
          default: return &k_serve_tiles<T, 3, true, kBtProp>;
        }
      }
      return nullptr;
    }
    switch (v) {
      case 0: return &k_serve_tiles<T, 0, false, kBtProp>;
      case 1: return &k_serve_tiles<T, 1, false, kBtProp>;
      case 2: return &k_serve_tiles<T, 2, false, kBtProp>;
      default: return &k_serve_tiles<T, 3, false, kBtProp>;
    }
  }
  return nullptr;
}

template <class T>
int serve_launch(plomgpu_server* sv, int inst, int grid) {
  cudaStream_t st = sv->loop_stream[inst];
  if (sv->tiled) {
    ServeTilesKernel<T> k = pick_serve_tiles<T>(sv->base.noises_off);
    if (!k) return fail(PLOMGPU_EINVAL, "no serving kernel for this model");
    k<<<grid, sv->bt, sv->tiles_smem, st>>>(serve_args<T>(sv), sv->slots_d, sv->map_d, sv->ring, sv->ctl_dev,
                                            sv->d_head, sv->d_pool, sv->d_live, sv->idle_limit, sv->task_budget);
  } else {
    ServeKernel<T> k = pick_serve<T>(sv->base.noises_off);
    if (!k) return fail(PLOMGPU_EINVAL, "no serving kernel for this model");
    k<<<grid, sv->bt, 0, st>>>(serve_args<T>(sv), sv->slots_d, sv->map_d, sv->ring, sv->ctl_d, sv->d_head,
                               sv->d_pool, sv->idle_limit);
  }
  CK(cudaGetLastError());
  CK(cudaEventRecord(sv->loop_ev[inst], st));
  sv->loop_live[inst] = true;
  sv->loop_grid[inst] = grid;
  sv->kernel_live = true;
  sv->launches++;
  return PLOMGPU_OK;
}

size_t serve_ws_bytes(plomgpu_server* sv, int J) {
  size_t b;
  if (sv->tiled) b = (sv->precision == 64) ? tile_req_bytes<double, kBtProp>(J) : tile_req_bytes<float, kBtProp>(J);
  else b = (sv->precision == 64) ? batch_ws_bytes<double>(J) : batch_ws_bytes<float>(J);
  return (b + 255) & ~(size_t)255;
}

size_t plan_footprint(plomgpu_server* sv, int J) {
  const size_t tb = sv->precision == 64 ? 8 : 4;
  return (size_t)J * (2 * M::S * tb + tb + 8 + 8) + (size_t)(1 << 20);
}

void record_result(plomgpu_server* sv, long long ticket, int status, double ll, int nf, Clock::time_point t0) {
  ServeResult& r = sv->results[ticket];
  r.done = true;
  r.status = status;
  r.loglik = ll;
  r.n_all_fail = nf;
  r.latency_s = std::chrono::duration<double>(Clock::now() - t0).count();
  sv->completed++;
  sv->in_flight--;
}

// one pass of the dispatcher; called with sv->mu held
void serve_pass(plomgpu_server* sv) {
  // completions of the persistent loop
  if (sv->persistent) {
    for (int i = 0; i < sv->ring; ++i) {
      if (sv->slot_ticket[i] < 0) continue;
      if (__atomic_load_n(&sv->slots_h[i].done, __ATOMIC_ACQUIRE)) {
        const int status = sv->slots_h[i].status ? PLOMGPU_ETIMEOUT : PLOMGPU_OK;
        record_result(sv, sv->slot_ticket[i], status, sv->slots_h[i].loglik, sv->slots_h[i].n_all_fail,
                      sv->slot_t[i]);
        sv->pool.release(sv->slot_off[i], sv->slot_bytes[i]);
        sv->slot_ticket[i] = -1;
        sv->free_slots.push_back(i);
        sv->cv_done.notify_all();
      }
    }
  }
  // completions of the plan pool
  for (auto& pp : sv->plans) {
    if (!pp.busy) continue;
    if (cudaEventQuery(pp.done_ev) == cudaSuccess) {
      plomgpu_smc_result r{};
      const int rc = plan_results(pp.plan, &r);
      record_result(sv, pp.ticket, rc, r.loglik, r.n_all_fail, pp.t_submit);
      pp.busy = false;
      sv->cv_done.notify_all();
    }
  }
  // admission, first come first served
  while (!sv->pending.empty()) {
    ServeRequest& rq = sv->pending.front();
    if (sv->persistent) {
      if (sv->free_slots.empty()) break;
      const size_t bytes = serve_ws_bytes(sv, rq.J);
      size_t off = 0;
      if (!sv->pool.alloc(bytes, &off)) break;
      const int i = sv->free_slots.front();
      sv->free_slots.pop_front();
      ServeSlot& sl = sv->slots_h[i];
      sl.J = rq.J;
      sl.n_obs = sv->base.n_obs;
      sl.seed = rq.seed;
      sl.ws_offset = off;
      sl.status = 0;
      memcpy(sl.par_cac, rq.par_cac.data(), sizeof(double) * rq.par_cac.size());
      memcpy(sl.par_ts, rq.par_ts.data(), sizeof(double) * rq.par_ts.size());
      memcpy(sl.x0, rq.x0.data(), sizeof(double) * rq.x0.size());
      __atomic_store_n(&sl.done, 0, __ATOMIC_RELAXED);
      sv->slot_ticket[i] = rq.ticket;
      sv->slot_off[i] = off;
      sv->slot_bytes[i] = bytes;
      sv->slot_t[i] = rq.t_submit;
      sv->map_h[sv->published % (unsigned long long)sv->ring] = i;
      std::atomic_thread_fence(std::memory_order_release);
      sv->published++;
      __atomic_store_n(&sv->ctl_h->tail, sv->published, __ATOMIC_RELEASE);
      sv->in_flight++;
      sv->peak_in_flight = std::max(sv->peak_in_flight, sv->in_flight);
      sv->pending.pop_front();
    } else {
      PooledPlan* use = nullptr;
      for (auto& pp : sv->plans)
        if (!pp.busy && pp.J == rq.J) {
          use = &pp;
          break;
        }
      if (!use) {
        const size_t fp = plan_footprint(sv, rq.J);
        if ((int)sv->plans.size() < sv->plan_pool && sv->plan_bytes_total + fp <= sv->budget) {
          plomgpu_smc_desc d = sv->base;
          d.J = rq.J;
          PooledPlan pp;
          pp.J = rq.J;
          pp.bytes = fp;
          if (plan_create(&d, &pp.plan, false, false, false) != PLOMGPU_OK) {
            record_result(sv, rq.ticket, PLOMGPU_ENOMEM, 0.0, 0, rq.t_submit);
            sv->in_flight++;  // record_result decremented it
            sv->pending.pop_front();
            continue;
          }
          cudaEventCreateWithFlags(&pp.done_ev, cudaEventDisableTiming);
          sv->plan_bytes_total += fp;
          sv->plans.push_back(pp);
          use = &sv->plans.back();
        } else {
          // evict an idle plan of another size if that makes room
          bool evicted = false;
          for (size_t k = 0; k < sv->plans.size(); ++k) {
            if (!sv->plans[k].busy && sv->plans[k].J != rq.J) {
              plan_free(sv->plans[k].plan);
              cudaEventDestroy(sv->plans[k].done_ev);
              sv->plan_bytes_total -= sv->plans[k].bytes;
              sv->plans.erase(sv->plans.begin() + (long)k);
              evicted = true;
              break;
            }
          }
          if (evicted) continue;
          break;
        }
      }
      if (plomgpu_plan_update(use->plan, rq.par_cac.data(), rq.par_ts.data(), rq.x0.data(), rq.seed) != PLOMGPU_OK ||
          plomgpu_plan_launch(use->plan) != PLOMGPU_OK) {
        sv->in_flight++;
        record_result(sv, rq.ticket, PLOMGPU_ECUDA, 0.0, 0, rq.t_submit);
        sv->pending.pop_front();
        continue;
      }
      cudaEventRecord(use->done_ev, use->plan->stream);
      use->busy = true;
      use->ticket = rq.ticket;
      use->t_submit = rq.t_submit;
      sv->in_flight++;
      sv->peak_in_flight = std::max(sv->peak_in_flight, sv->in_flight);
      sv->pending.pop_front();
      sv->launches++;
    }
  }
  if (sv->tiled && sv->ctl_dev && sv->published != sv->pushed_tail) {
    cudaMemcpyAsync(&sv->ctl_dev->tail, &sv->ctl_h->tail, sizeof(unsigned long long), cudaMemcpyHostToDevice,
                    sv->ctl_stream);
    sv->pushed_tail = sv->published;
  }
  // (re)start device loops while published requests outnumber the live CTAs
  if (sv->persistent) {
    long long live_ctas = 0;
    for (int i = 0; i < plomgpu_server::kLoops; ++i) {
      if (sv->loop_live[i] && cudaEventQuery(sv->loop_ev[i]) == cudaSuccess) sv->loop_live[i] = false;
      if (sv->loop_live[i]) live_ctas += sv->loop_grid[i];
    }
    sv->kernel_live = live_ctas > 0;
    long long waiting = 0;
    for (int i = 0; i < sv->ring; ++i) waiting += sv->slot_ticket[i] >= 0;
    if (sv->tiled) {
      // instances of every resident CTA slot: the tiles of all live requests
      // share them.  Their CTAs return after a budget of tasks, so a next
      // instance is kept queued behind the running one while requests wait;
      // the loop's streams have the lowest priority, so that the blocks of
      // other kernels (a one-CTA-per-request loop, plain filters) take the
      // slots they free first.
      int live_inst = 0;
      for (int i = 0; i < plomgpu_server::kLoops; ++i) live_inst += sv->loop_live[i] ? 1 : 0;
      if (waiting > 0 && live_inst < 2) {
        for (int i = 0; i < plomgpu_server::kLoops; ++i) {
          if (sv->loop_live[i]) continue;
          const int rc =
              (sv->precision == 64) ? serve_launch<double>(sv, i, sv->grid) : serve_launch<float>(sv, i, sv->grid);
          if (rc) sv->last_error = g_err;
          break;
        }
      }
    } else if (waiting > live_ctas && live_ctas < sv->grid) {
      for (int i = 0; i < plomgpu_server::kLoops; ++i) {
        if (sv->loop_live[i]) continue;
        const long long want = std::max<long long>(std::max<long long>(waiting - live_ctas, (live_ctas + 1) / 2), 8);
        const int grid = (int)std::min<long long>(want, (long long)sv->grid - live_ctas);
        const int rc = (sv->precision == 64) ? serve_launch<double>(sv, i, grid) : serve_launch<float>(sv, i, grid);
        if (rc) sv->last_error = g_err;
        break;
      }
    }
  }
}

void serve_loop(plomgpu_server* sv) {
  int dev = 0;
  cudaGetDevice(&dev);
  std::unique_lock<std::mutex> lock(sv->mu);
  while (!sv->stop) {
    serve_pass(sv);
    sv->cv.wait_for(lock, std::chrono::microseconds(50));
  }
}

}  // namespace
