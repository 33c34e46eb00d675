// Device-resident request loop: a persistent kernel whose CTAs take
// likelihood requests from a ring in mapped (host-pinned, device-visible)
// memory and run each one as a whole filter (cta_filter).  Requests are
// published by the host (fields, then a release store of the ring tail) and
// completed by the device (result, then a release store of the slot's done
// flag), both at system scope.  Each CTA takes the next request as soon as
// it finishes one, so requests that arrive while others run start on the
// CTAs that free up (continuous batching).  Every wait is bounded: a CTA that
// finds no request for `idle_limit` microseconds (the GPU's global timer)
// returns, and the host relaunches the loop when new requests arrive.  The
// bound is in time, not in polls: polls of host memory by many idle CTAs
// slow each other down, and a count of them kept a grown loop resident (and
// its SMs from other kernels) for seconds after its last request.
//
// Callers: concurrent pmcmc chains evaluating one likelihood per iteration
// (model_builder/C/pmcmc/pmcmc.c:186-266, run_propag at pmcmc.c:24-37).
#pragma once

#include <cuda/atomic>
#include <climits>

#include "smc_batch.cuh"

namespace plomgpu {

// nanoseconds of the GPU's global timer
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

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
  int status;  // 0, or the error flags of the filter (ERR_*)
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
      const unsigned long long t_idle = global_ns();
      for (;;) {
        if ((spins & 255) == 0 && stop_ref.load(cuda::memory_order_acquire)) break;
        const unsigned long long t = tail_ref.load(cuda::memory_order_acquire);
        const unsigned long long h = atomicAdd(head, 0ull);
        if (h < t) {
          if (atomicCAS(head, h, h + 1ull) == h) {
            got = (long long)h;
            break;
          }
          continue;
        }
        ++spins;
        if (global_ns() - t_idle > (unsigned long long)idle_limit * 1000ull) break;
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

// ---------------------------------------------------------------------------
// Device-resident request loop for models whose particles live in shared
// memory (SEIR 20x2: 180 words per particle), too large for one CTA per
// request.  A request is split into tiles of BT particles, and one tile of
// one phase of one request is the unit of work:
//   propagate(n)  the tile's particles over interval n (gather from the
//                 ancestors, substeps, log-weights) and the tile's
//                 log-sum-exp partial;
//   resample(n)   the cumulative normalised weights of the tile and the
//                 ancestors of the systematic points that fall in it
//                 (resample_tile).
// The CTA that finishes the last tile of a phase does the phase's serial
// part itself (the fold of the partials: llike, ESS, all-fail rule,
// systematic points, tile prefixes) and publishes the next phase; nothing
// waits on another CTA, so every CTA only polls for work, with a bound.
// Up to kServeLive requests are live at once; a CTA claims a tile of the
// oldest live request that has one, else admits the next published
// request, so requests that arrive while others run share the SMs with
// them tile by tile (continuous batching).  Each request keeps the draws,
// arithmetic and reduction order of the plain filter with its seed.
constexpr int kServeLive = 64;

// device state of one admitted request, at the start of its workspace
// The claim counter, the completion counter and the rest sit in cache lines
// of their own: every polling CTA reads the first, every finishing one adds
// to the second.
struct TileReq {
  alignas(128) unsigned long long phase;  // (phase number << 32) | next unclaimed tile; phase numbers
                                          // start at order << 12, so a stale read of a reused workspace
                                          // never matches
  alignas(128) unsigned done;             // tiles of the current phase finished
  alignas(128) int n;                     // interval of the current phase
  int kind;                  // 0 propagate, 1 resample
  int cur;                   // generation holding the particles before interval n
  int resampled;             // the ancestors of interval n - 1 apply (else identity)
  int slot;                  // ring slot of the request (its result)
  int J, ntiles;
  int n_obs;                 // intervals of the request
  long long order;           // publication order (older requests first)
  uint64_t seed;
  StepState st;
  FilterAcc acc;
};

// tiles a CTA claims at once: one propagate tile, a few of the short phases
constexpr int kServeShortClaim = 4;

template <class T>
struct TileReqWs {
  TileReq* q;
  LseAcc* part;
  double* P;
  T* lw;
  uint32_t* anc;
  T* X[2];
  T* par_cac;
  double* par_ts;
  double* x0;
};

constexpr size_t ws_align(size_t b) { return (b + 255) & ~(size_t)255; }

template <class T, int BT>
__host__ __device__ inline size_t tile_req_bytes(int J) {
  const size_t nt = (size_t)((J + BT - 1) / BT);
  const size_t mj = (size_t)((J + 31) & ~31);
  return ws_align(sizeof(TileReq)) + ws_align(nt * sizeof(LseAcc)) + ws_align((nt + 1) * sizeof(double)) +
         ws_align(mj * sizeof(T)) + ws_align(mj * sizeof(uint32_t)) + 2 * ws_align((size_t)M::S * mj * sizeof(T)) +
         ws_align((size_t)kServeParCac * sizeof(T)) + ws_align((size_t)kServeParTs * sizeof(double)) +
         ws_align((size_t)M::S * sizeof(double));
}

template <class T, int BT>
__device__ inline TileReqWs<T> tile_req_ws(unsigned char* base, int J) {
  const size_t nt = (size_t)((J + BT - 1) / BT);
  const size_t mj = (size_t)((J + 31) & ~31);
  TileReqWs<T> w;
  unsigned char* p = base;
  w.q = reinterpret_cast<TileReq*>(p);
  p += ws_align(sizeof(TileReq));
  w.part = reinterpret_cast<LseAcc*>(p);
  p += ws_align(nt * sizeof(LseAcc));
  w.P = reinterpret_cast<double*>(p);
  p += ws_align((nt + 1) * sizeof(double));
  w.lw = reinterpret_cast<T*>(p);
  p += ws_align(mj * sizeof(T));
  w.anc = reinterpret_cast<uint32_t*>(p);
  p += ws_align(mj * sizeof(uint32_t));
  w.X[0] = reinterpret_cast<T*>(p);
  p += ws_align((size_t)M::S * mj * sizeof(T));
  w.X[1] = reinterpret_cast<T*>(p);
  p += ws_align((size_t)M::S * mj * sizeof(T));
  w.par_cac = reinterpret_cast<T*>(p);
  p += ws_align((size_t)kServeParCac * sizeof(T));
  w.par_ts = reinterpret_cast<double*>(p);
  p += ws_align((size_t)kServeParTs * sizeof(double));
  w.x0 = reinterpret_cast<double*>(p);
  return w;
}

// dynamic shared memory of the tiled loop: the propagate block's (tables +
// state columns), which also holds the tile scratch between propagate phases
template <class T, int BT>
constexpr size_t serve_tiles_smem() {
  constexpr size_t prop = propagate_smem_bytes<T, kSmem, BT>();
  constexpr size_t scratch = ((size_t)(kSmemCoup + kSmemPar) * sizeof(T) + 15) / 16 * 16 + sizeof(TileScratch<BT, 1>);
  return prop > scratch ? prop : scratch;
}

template <class T, int V, bool DRIFT, int BT>
__global__ void __launch_bounds__(BT) k_serve_tiles(const BatchArgs<T> a, ServeSlot* slots, const int* ring_map,
                                                    int ring, ServeCtl* ctl, unsigned long long* head,
                                                    unsigned char* pool, long long* live, long long idle_limit,
                                                    int task_budget) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  // the tile scratch sits after the coupling / parameter tables
  TileScratch<BT, 1>& sc = *reinterpret_cast<TileScratch<BT, 1>*>(
      smem_raw + ((size_t)(kSmemCoup + kSmemPar) * sizeof(T) + 15) / 16 * 16);
  __shared__ long long s_off;   // workspace of the claimed request, -1: none
  __shared__ int s_tile;        // first claimed tile, -1: admission of a new request
  __shared__ int s_ntask;       // tiles claimed
  __shared__ int s_entry;       // live-table entry of an admission
  __shared__ long long s_req;   // publication order of an admission
  __shared__ int s_last;
  // ctl is a device-memory copy of the host's control block (the host copies
  // it after every publication)
  cuda::atomic_ref<unsigned long long, cuda::thread_scope_device> tail_ref(ctl->tail);
  cuda::atomic_ref<int, cuda::thread_scope_device> stop_ref(ctl->stop);
  if constexpr (M::COUPLED) {
    T* s_coup = reinterpret_cast<T*>(smem_raw);
    for (int i = threadIdx.x; i < M::N_CAC * M::N_CAC; i += BT) s_coup[i] = a.coupling[i];
  }
  // after task_budget tasks a CTA returns (the host keeps a next instance
  // queued), so that its SM slot can go to other kernels between tasks
  int tasks = 0;
  for (;;) {
    __syncthreads();
    if (task_budget > 0 && tasks >= task_budget) return;
    ++tasks;
    if (threadIdx.x < 32) {
      // warp 0 polls: lane l looks at live entries l and l + 32 in parallel
      const int lane = threadIdx.x;
      if (lane == 0) s_off = -1;
      __syncwarp();
      const unsigned long long t_idle = global_ns();
      unsigned backoff = 128u;  // ns between polls that find nothing, doubling up to 8 us
      for (;;) {
        int stop = 0;
        if (lane == 0) stop = stop_ref.load(cuda::memory_order_relaxed);
        if (__shfl_sync(0xffffffffu, stop, 0)) break;
        // a tile of the oldest live request that has one
        long long my_off = -1, my_order = LLONG_MAX;
        unsigned long long my_v = 0;
        int free_entry = -1, live_here = 0;
        for (int e = lane; e < kServeLive; e += 32) {
          const long long off = *(volatile long long*)(live + e);
          if (off == -1) {
            if (free_entry < 0) free_entry = e;
            continue;
          }
          live_here = 1;
          if (off < 0) continue;  // being admitted
          TileReq* q = reinterpret_cast<TileReq*>(pool + off);
          const unsigned long long v = *(volatile unsigned long long*)&q->phase;
          const long long ord = *(volatile long long*)&q->order;
          if ((int)(v & 0xffffffffull) < *(volatile int*)&q->ntiles && ord < my_order) {
            my_off = off;
            my_order = ord;
            my_v = v;
          }
        }
        // the lane holding the oldest claimable request
        long long best = my_order;
        int my_kind = 0;
        if (my_off >= 0) my_kind = *(volatile int*)&reinterpret_cast<TileReq*>(pool + my_off)->kind;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) best = min(best, __shfl_xor_sync(0xffffffffu, best, o));
        const unsigned who = __ballot_sync(0xffffffffu, my_off >= 0 && my_order == best);
        const int any_live = __any_sync(0xffffffffu, live_here);
        if (who) {
          int got = 0;
          if (lane == __ffs(who) - 1) {
            // fetch-and-add hands out the tiles of the phase one by one; a
            // count past the tiles (the phase is taken, or the workspace was
            // reused by a newer request after the read above) claims nothing
            TileReq* q = reinterpret_cast<TileReq*>(pool + my_off);
            const int k = (my_kind == 0) ? 1 : kServeShortClaim;
            const unsigned long long v = atomicAdd(&q->phase, (unsigned long long)k);
            __threadfence();
            const int t0 = (int)(v & 0xffffffffull), nt = *(volatile int*)&q->ntiles;
            if (t0 < nt) {
              s_off = my_off;
              s_tile = t0;
              s_ntask = min(k, nt - t0);
              got = 1;
            }
          }
          if (__shfl_sync(0xffffffffu, got, __ffs(who) - 1)) break;
          continue;  // look again
        }
        // else the next published request, if a live entry is free
        const unsigned freem = __ballot_sync(0xffffffffu, free_entry >= 0);
        if (freem) {
          int done_here = 0, again = 0;
          if (lane == __ffs(freem) - 1) {
            const unsigned long long t = tail_ref.load(cuda::memory_order_acquire);
            const unsigned long long h = atomicAdd(head, 0ull);
            if (h < t) {
              again = 1;
              if (atomicCAS((unsigned long long*)(live + free_entry), (unsigned long long)-1ll,
                            (unsigned long long)-2ll) == (unsigned long long)-1ll) {
                if (atomicCAS(head, h, h + 1ull) == h) {
                  const ServeSlot* sl = slots + ring_map[h % ring];
                  s_off = (long long)sl->ws_offset;
                  s_tile = -1;
                  s_entry = free_entry;
                  s_req = (long long)h;
                  done_here = 1;
                } else {
                  atomicExch((unsigned long long*)(live + free_entry), (unsigned long long)-1ll);
                }
              }
            }
          }
          const int src = __ffs(freem) - 1;
          if (__shfl_sync(0xffffffffu, done_here, src)) break;
          if (__shfl_sync(0xffffffffu, again, src)) continue;
        }
        // nothing to do now: while requests are live the wait is long (their
        // serial parts run on one CTA), else short; bounded either way
        if (global_ns() - t_idle > (unsigned long long)idle_limit * (any_live ? 2500000ull : 1000ull)) break;
        __nanosleep(backoff);
        backoff = backoff < 8192u ? 2u * backoff : 8192u;
      }
    }
    __syncthreads();
    if (s_off < 0) return;
    // the tiles' data come from other CTAs of this GPU (device-scope
    // acquire); only an admission reads a slot the host wrote (system scope,
    // which costs about as much as a whole tile of propagation)
    __threadfence();
    unsigned char* base = pool + s_off;
    if (s_tile < 0) {
      cuda::atomic_thread_fence(cuda::memory_order_acquire, cuda::thread_scope_system);
      // admission: the request's device state and its parameters in the state precision
      const int slot = ring_map[s_req % ring];
      const ServeSlot* sl = slots + slot;
      const int J = sl->J;
      const TileReqWs<T> w = tile_req_ws<T, BT>(base, J);
      for (int i = threadIdx.x; i < M::N_PAR_PROC * M::N_CAC; i += BT) w.par_cac[i] = (T)sl->par_cac[i];
      for (int i = threadIdx.x; i < M::N_PAR_OBS * M::N_TS; i += BT) w.par_ts[i] = sl->par_ts[i];
      for (int i = threadIdx.x; i < M::S; i += BT) w.x0[i] = sl->x0[i];
      __threadfence();
      __syncthreads();
      if (threadIdx.x == 0) {
        TileReq* q = w.q;
        q->done = 0u;
        q->n = 0;
        q->kind = 0;
        q->cur = 0;
        q->resampled = 0;
        q->slot = slot;
        q->J = J;
        q->ntiles = (J + BT - 1) / BT;
        q->n_obs = sl->n_obs;
        q->order = s_req;
        q->seed = sl->seed;
        q->acc.loglik = 0.0;
        q->acc.n_all_fail = 0;
        q->acc.error = 0;
        q->acc.ticket = 0u;
        __threadfence();
        atomicExch(&q->phase, ((unsigned long long)(s_req & 0xfffff) << 12) << 32);
        __threadfence();
        atomicExch((unsigned long long*)(live + s_entry), (unsigned long long)s_off);
      }
      continue;
    }
    TileReq* q = reinterpret_cast<TileReq*>(base);
    const int J = q->J, ntiles = q->ntiles, n = q->n, kind = q->kind, ntask = s_ntask;
    const TileReqWs<T> w = tile_req_ws<T, BT>(base, J);
    const double* y = a.data + (size_t)n * M::N_TS;
    bool any = false;
    for (int ts = 0; ts < M::N_TS; ++ts) any |= !isnan(__ldg(y + ts));
    const bool weigh = a.filter_on && any;
    for (int tile = s_tile; tile < s_tile + ntask; ++tile) {
    if (kind == 0) {
      Tables<T> tb{};
      tb.par_cac = w.par_cac;
      tb.cov_cac = a.cov_cac;
      tb.coupling = a.coupling;
      tb.drift_group = a.drift_group;
      tb.drift_ngroups = a.drift_ngroups;
      tb.drift_bt = a.drift_bt;
      tb.drift_vol = a.drift_vol;
      tb.par_ts = w.par_ts;
      tb.t_sub = a.t_sub;
      tb.dt = a.dt;
      tb.like_min = a.like_min;
      tb.seed = &q->seed;
      tb.filter_id = 0u;
      tb.J = J;
      tb.R = 1;
      StepArgs sa{};
      sa.n = n;
      sa.n_sub = __ldg(a.n_sub + n);
      sa.sub0 = __ldg(a.sub0 + n);
      sa.weigh = weigh ? 1 : 0;
      sa.t_obs = __ldg(a.t_obs + n);
      sa.y = y;
      sa.cov_ts = a.cov_ts + (size_t)n * M::N_COV_TS * M::N_TS;
      sa.X_prev = w.X[q->cur];
      sa.X_next = w.X[q->cur ^ 1];
      sa.anc = q->resampled ? w.anc : nullptr;
      sa.lw = w.lw;
      sa.x0_rep = (n == 0) ? w.x0 : nullptr;
      propagate_tables<T, BT>(tb, smem_raw, false);
      const size_t g = (size_t)tile * BT + threadIdx.x;
      double l = NAN;
      if (g < (size_t)J) l = propagate_particle<T, V, DRIFT, false, kSmem, false, BT, false, false>(tb, sa, g, smem_raw);
      __syncthreads();  // the state columns are free again
      // the interval's systematic points: one thread of the first tile, before its completion count
      if (weigh && tile == 0 && threadIdx.x == 32)
        sys_table(&q->st.tab, &q->acc, J, n, -1.0, plomrt::make_key(q->seed, 0u));
      if (weigh) {
        LseAcc acc = {-INFINITY, 0.0, 0.0, 0};
        if (g < (size_t)J) {
          if (weight_fails_at(l, a.fail_b)) acc.nfail = 1;
          else acc = LseAcc{l, 1.0, 1.0, 0};
        }
        acc = block_lse_all<BT>(acc, sc.lse);
        if (threadIdx.x == 0) w.part[tile] = acc;
      }
    } else {
      resample_tile<T, BT, 1>(w.lw, J, a.fail_b, w.part, w.P, &q->st, &q->st.tab, tile, ntiles, w.anc, nullptr,
                              nullptr, nullptr, sc);
    }
    __syncthreads();  // the shared scratch of one tile before the next
    }
    // the last tile of the phase does its serial part and publishes the next phase
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0)
      s_last = (atomicAdd(&q->done, (unsigned)ntask) + (unsigned)ntask == (unsigned)ntiles) ? 1 : 0;
    __syncthreads();
    if (!s_last) continue;
    __threadfence();
    const int T_obs = q->n_obs;
    bool finished = false;
    int next_kind = 0, next_n = n, next_cur = q->cur, next_res = q->resampled;
    if (kind == 0) {
      next_cur = q->cur ^ 1;
      if (weigh) {
        fold_tiles<BT>(w.part, ntiles, J, a.log_like_min, w.P, &q->st, &q->acc, n, nullptr, nullptr, sc.lse,
                       sc.swarp);
        if (n == T_obs - 1) finished = true;
        else next_kind = 1;
      } else {
        next_res = 0;
        next_n = n + 1;
        if (next_n == T_obs) finished = true;
      }
    } else {
      next_kind = 0;
      next_res = 1;
      next_n = n + 1;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      if (finished) {
        ServeSlot* out = slots + q->slot;
        out->loglik = q->acc.loglik;
        out->n_all_fail = q->acc.n_all_fail;
        out->status = q->acc.error;
        for (int e = 0; e < kServeLive; ++e)
          if (atomicAdd((unsigned long long*)(live + e), 0ull) == (unsigned long long)s_off)
            atomicExch((unsigned long long*)(live + e), (unsigned long long)-1ll);
        cuda::atomic_ref<int, cuda::thread_scope_system> done_ref(out->done);
        done_ref.store(1, cuda::memory_order_release);
      } else {
        q->n = next_n;
        q->kind = next_kind;
        q->cur = next_cur;
        q->resampled = next_res;
        q->done = 0u;
        __threadfence();
        const unsigned long long v = atomicAdd(&q->phase, 0ull);
        atomicExch(&q->phase, ((v >> 32) + 1ull) << 32);
      }
    }
  }
}

}  // namespace plomgpu
