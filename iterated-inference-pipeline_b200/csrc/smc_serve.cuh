// Device-resident request loop: a persistent kernel whose CTAs take
// likelihood requests from a ring in mapped (host-pinned, device-visible)
// memory and run each one as a whole filter (cta_filter).  Requests are
// published by the host (fields, then a release store of the ring tail) and
// completed by the device (result, then a release store of the slot's done
// flag), both at system scope.  Each CTA takes the next request as soon as
// it finishes one, so requests that arrive while others run start on the
// CTAs that free up (continuous batching).  Every wait is bounded: a CTA that
// finds no request for `idle_limit` polls returns, and the host relaunches
// the loop when new requests arrive.
//
// Callers: concurrent pmcmc chains evaluating one likelihood per iteration
// (model_builder/C/pmcmc/pmcmc.c:186-266, run_propag at pmcmc.c:24-37).
#pragma once

#include <cuda/atomic>

#include "smc_batch.cuh"

namespace plomgpu {

constexpr int kServeParCac = (M::N_PAR_PROC * M::N_CAC) > 0 ? (M::N_PAR_PROC * M::N_CAC) : 1;
constexpr int kServeParTs = (M::N_PAR_OBS * M::N_TS) > 0 ? (M::N_PAR_OBS * M::N_TS) : 1;

struct ServeSlot {
  // written by the host before the tail is published
  int J;
  int n_obs;
  uint64_t seed;
  unsigned long long ws_offset;  // bytes into the device workspace pool
  double par_cac[kServeParCac];
  double par_ts[kServeParTs];
  double x0[M::S];
  // written by the device
  double loglik;
  int n_all_fail;
  int done;
};

struct ServeCtl {
  unsigned long long tail;  // requests published so far
  int stop;                 // 1: the loop returns at its next poll
  int pad;
};

// Request p (in publication order) lives in slot ring_map[p % ring].
template <class T, int V, bool DRIFT, int BT>
__global__ void __launch_bounds__(BT) k_serve(const BatchArgs<T> a, ServeSlot* slots, const int* ring_map, int ring,
                                              ServeCtl* ctl, unsigned long long* head, unsigned char* pool,
                                              long long idle_limit) {
  __shared__ CtaShared<T, BT> sh;
  __shared__ long long s_req;
  __shared__ int s_slot;
  __shared__ int s_J, s_n_obs;
  __shared__ uint64_t s_seed;
  __shared__ unsigned long long s_ws;
  __shared__ double s_ll;
  __shared__ int s_nf;
  if constexpr (M::COUPLED) {
    for (int i = threadIdx.x; i < M::N_CAC * M::N_CAC; i += BT) sh.coup[i] = a.coupling[i];
  }
  cuda::atomic_ref<unsigned long long, cuda::thread_scope_system> tail_ref(ctl->tail);
  cuda::atomic_ref<int, cuda::thread_scope_system> stop_ref(ctl->stop);
  for (;;) {
    __syncthreads();
    if (threadIdx.x == 0) {
      long long got = -1;
      long long spins = 0;
      for (;;) {
        if (stop_ref.load(cuda::memory_order_acquire)) break;
        const unsigned long long t = tail_ref.load(cuda::memory_order_acquire);
        const unsigned long long h = atomicAdd(head, 0ull);
        if (h < t) {
          if (atomicCAS(head, h, h + 1ull) == h) {
            got = (long long)h;
            break;
          }
          continue;
        }
        if (++spins > idle_limit) break;
        __nanosleep(1000);
      }
      s_req = got;
      if (got >= 0) {
        s_slot = ring_map[got % ring];
        const ServeSlot* sl = slots + s_slot;
        s_J = sl->J;
        s_n_obs = sl->n_obs;
        s_seed = sl->seed;
        s_ws = sl->ws_offset;
      }
    }
    __syncthreads();
    const long long req = s_req;
    if (req < 0) return;
    cuda::atomic_thread_fence(cuda::memory_order_acquire, cuda::thread_scope_system);
    ServeSlot* sl = slots + s_slot;
    FilterJob job;
    job.J = s_J;
    job.n_obs = s_n_obs;
    job.seed = s_seed;
    job.data = a.data;
    job.par_cac = sl->par_cac;
    job.par_ts = sl->par_ts;
    job.x0 = sl->x0;
    const BatchWs<T> ws = batch_ws<T>(pool + s_ws, s_J);
    const size_t ld = (size_t)((s_J + 31) & ~31);
    cta_filter<T, V, DRIFT, BT>(sh, a, job, ws, ld, &s_ll, &s_nf, nullptr);
    __syncthreads();
    if (threadIdx.x == 0) {
      sl->loglik = s_ll;
      sl->n_all_fail = s_nf;
      cuda::atomic_ref<int, cuda::thread_scope_system> done_ref(sl->done);
      done_ref.store(1, cuda::memory_order_release);
    }
  }
}

}  // namespace plomgpu
