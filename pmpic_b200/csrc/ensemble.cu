// ensemble.cu -- a batch of independent plumes on one GPU.
//
// The reference runs one model per MPI job; an ensemble of independent plumes
// of uneven sizes is an addition of this library (it has no counterpart in the
// reference).  Each member is a full context with its own CUDA stream.  A pool
// of host threads steps members concurrently, largest first, so the small
// members' launch-bound kernels overlap each other and the large members'
// bandwidth-bound ones instead of running back to back.  Two knobs are tuned:
//  - per distinct grid size, the column-segment length of the par2grid row
//    pass (short segments give small grids more warps), timed on the member's
//    own parcels without changing its state;
//  - the number of host threads, online: the first steps of a run try one
//    candidate each and the remaining steps use the fastest.
// Device time of a run spans all member streams: a start event on a control
// stream that every member stream waits on, and an end event recorded after
// the control stream has waited on every member's end event.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <map>
#include <thread>
#include <tuple>
#include <vector>

#include "common.cuh"

struct pmpic_ensemble {
  std::vector<pmpic_ctx*> m;
  std::vector<int> order;      // members by decreasing parcel count
  int device = 0;
  int threads = 0;             // 0: tune online on the next run
  bool tuned_threads = false;
  cudaStream_t ctl = nullptr;
  cudaEvent_t t0 = nullptr, t1 = nullptr;
  std::vector<cudaEvent_t> ends;
};

namespace {

int run_members(pmpic_ensemble* e, int nsteps, int threads, float* ms) {
  const int n = (int)e->m.size();
  if (cudaEventRecord(e->t0, e->ctl) != cudaSuccess) return PMPIC_ERR_CUDA;
  for (pmpic_ctx* c : e->m)
    if (cudaStreamWaitEvent(c->stream, e->t0, 0) != cudaSuccess) return PMPIC_ERR_CUDA;
  std::atomic<int> next(0);
  std::atomic<int> first_err(0);
  auto worker = [&]() {
    cudaSetDevice(e->device);
    for (;;) {
      const int k = next.fetch_add(1);
      if (k >= n) break;
      const int i = e->order[k];
      int rc = pmpic_step(e->m[i], nsteps);
      if (rc) {
        int z = 0;
        first_err.compare_exchange_strong(z, rc);
      }
      cudaEventRecord(e->ends[i], e->m[i]->stream);
    }
  };
  const int t = std::max(1, std::min(threads, n));
  std::vector<std::thread> pool;
  for (int w = 1; w < t; ++w) pool.emplace_back(worker);
  worker();
  for (auto& th : pool) th.join();
  cudaSetDevice(e->device);
  for (int i = 0; i < n; ++i)
    if (cudaStreamWaitEvent(e->ctl, e->ends[i], 0) != cudaSuccess) return PMPIC_ERR_CUDA;
  if (cudaEventRecord(e->t1, e->ctl) != cudaSuccess) return PMPIC_ERR_CUDA;
  if (cudaEventSynchronize(e->t1) != cudaSuccess) return PMPIC_ERR_CUDA;
  float v = 0.f;
  if (cudaEventElapsedTime(&v, e->t0, e->t1) != cudaSuccess) return PMPIC_ERR_CUDA;
  if (ms) *ms = v;
  return first_err.load();
}

}  // namespace

extern "C" {

int pmpic_ensemble_create(int n, const pmpic_config* cfgs, pmpic_ensemble** out) {
  if (n < 1 || !cfgs || !out) return PMPIC_ERR_ARG;
  *out = nullptr;
  for (int i = 1; i < n; ++i)
    if (cfgs[i].device != cfgs[0].device) return PMPIC_ERR_CONFIG;  // one GPU per ensemble
  pmpic_ensemble* e = new pmpic_ensemble();
  e->device = cfgs[0].device;
  int rc = 0;
  for (int i = 0; i < n && !rc; ++i) {
    pmpic_ctx* c = nullptr;
    rc = pmpic_create(&cfgs[i], &c);
    if (!rc) e->m.push_back(c);
  }
  cudaSetDevice(e->device);
  // Stream priorities by size: the smaller a member, the higher its stream's
  // priority.  Small members are bound by the latency of their short kernels;
  // with priority their blocks are dispatched as soon as an SM frees up
  // instead of queueing behind the large members' blocks, which fill the
  // bandwidth either way.  (Each member's stream is replaced before any work
  // is queued on it: pmpic_create's own set-up is synchronous.)
  if (!rc) {
    int least = 0, greatest = 0;
    if (cudaDeviceGetStreamPriorityRange(&least, &greatest) != cudaSuccess) rc = PMPIC_ERR_CUDA;
    const int levels = least - greatest + 1;  // greatest is the numerically lowest (highest priority)
    std::vector<int> by(n);
    for (int i = 0; i < n; ++i) by[i] = i;
    std::stable_sort(by.begin(), by.end(), [&](int a, int b) { return e->m[a]->cap < e->m[b]->cap; });
    for (int r = 0; r < n && !rc && levels > 1; ++r) {
      pmpic_ctx* c = e->m[by[r]];
      const int prio = greatest + (int)((int64_t)r * levels / n);  // smallest members: greatest priority
      cudaStream_t s = nullptr;
      if (cudaStreamCreateWithPriority(&s, cudaStreamNonBlocking, prio) != cudaSuccess) {
        rc = PMPIC_ERR_CUDA;
        break;
      }
      cudaStreamSynchronize(c->stream);
      cudaStreamDestroy(c->stream);
      c->stream = s;
    }
  }
  if (!rc && cudaStreamCreateWithFlags(&e->ctl, cudaStreamNonBlocking) != cudaSuccess) rc = PMPIC_ERR_CUDA;
  if (!rc && (cudaEventCreate(&e->t0) != cudaSuccess || cudaEventCreate(&e->t1) != cudaSuccess)) rc = PMPIC_ERR_CUDA;
  e->ends.assign(n, nullptr);
  for (int i = 0; i < n && !rc; ++i)
    if (cudaEventCreateWithFlags(&e->ends[i], cudaEventDisableTiming) != cudaSuccess) rc = PMPIC_ERR_CUDA;
  if (rc) {
    pmpic_ensemble_destroy(e);
    return rc;
  }
  *out = e;
  return PMPIC_OK;
}

void pmpic_ensemble_destroy(pmpic_ensemble* e) {
  if (!e) return;
  cudaSetDevice(e->device);
  for (pmpic_ctx* c : e->m) pmpic_destroy(c);
  for (cudaEvent_t ev : e->ends)
    if (ev) cudaEventDestroy(ev);
  if (e->t0) cudaEventDestroy(e->t0);
  if (e->t1) cudaEventDestroy(e->t1);
  if (e->ctl) cudaStreamDestroy(e->ctl);
  delete e;
}

pmpic_ctx* pmpic_ensemble_member(pmpic_ensemble* e, int i) {
  if (!e || i < 0 || i >= (int)e->m.size()) return nullptr;
  return e->m[i];
}

int pmpic_ensemble_set_concurrency(pmpic_ensemble* e, int threads) {
  if (!e || threads < 0) return PMPIC_ERR_ARG;
  e->threads = threads;
  e->tuned_threads = threads > 0;
  return PMPIC_OK;
}

int pmpic_set_p2g_segment(pmpic_ctx* ctx, int xseg) {
  if (!ctx || xseg < 1 || xseg > 4096) return PMPIC_ERR_ARG;
  ctx->p2g_xseg = xseg;
  return PMPIC_OK;
}

int pmpic_ensemble_autotune(pmpic_ensemble* e) {
  if (!e) return PMPIC_ERR_ARG;
  static const int cand[] = {8, 16, 32, 64};
  std::map<std::tuple<int, int, int, bool>, int> best;  // (nx, ny, nz, mixed) -> segment
  for (pmpic_ctx* c : e->m) {
    const auto key = std::make_tuple(c->g.Nx, c->g.Ny, c->g.Nz, c->mixed);
    auto it = best.find(key);
    if (it != best.end()) {
      c->p2g_xseg = it->second;
      continue;
    }
    if (c->n == 0) continue;  // nothing to time on
    const int props[4] = {PMPIC_PROP_P, PMPIC_PROP_Q, PMPIC_PROP_R, PMPIC_PROP_B};
    const int grids[4] = {PMPIC_GRID_P, PMPIC_GRID_Q, PMPIC_GRID_R, PMPIC_GRID_B};
    float tbest = 1e30f;
    int sbest = c->p2g_xseg;
    for (int s : cand) {
      if (s > 2 * c->g.Nx && s != 64) continue;
      c->p2g_xseg = s;
      int rc = pmpic_op_par2grid_multi(c, 4, props, grids);  // warm
      if (rc) return rc;
      if ((rc = pmpic_event_record(c, 6))) return rc;
      for (int r = 0; r < 3 && !rc; ++r) rc = pmpic_op_par2grid_multi(c, 4, props, grids);
      if (rc) return rc;
      if ((rc = pmpic_event_record(c, 7))) return rc;
      float ms = 0.f;
      if ((rc = pmpic_event_elapsed(c, 6, 7, &ms))) return rc;
      if (ms < tbest) {
        tbest = ms;
        sbest = s;
      }
    }
    c->p2g_xseg = sbest;
    best[key] = sbest;
  }
  return PMPIC_OK;
}

int pmpic_ensemble_step(pmpic_ensemble* e, int nsteps, float* device_ms) {
  if (!e || nsteps < 0) return PMPIC_ERR_ARG;
  cudaSetDevice(e->device);
  const int n = (int)e->m.size();
  // largest members first, so the last ones to finish are small
  e->order.resize(n);
  for (int i = 0; i < n; ++i) e->order[i] = i;
  std::stable_sort(e->order.begin(), e->order.end(),
                   [&](int a, int b) { return e->m[a]->n > e->m[b]->n; });
  float total = 0.f;
  int done = 0;
  if (!e->tuned_threads) {
    static const int cand[] = {2, 4, 8, 16, 32, 64};
    std::vector<int> tries;  // candidates up to the member count (at least one)
    for (int t : cand)
      if (t <= n || tries.empty()) tries.push_back(t);
    float tbest = 1e30f;
    int best = 1;
    for (int t : tries) {
      if (done >= nsteps) break;
      float ms = 0.f;
      int rc = run_members(e, 1, t, &ms);
      if (rc) return rc;
      ++done;
      total += ms;
      if (ms < tbest) {
        tbest = ms;
        best = t;
      }
    }
    if (done < (int)tries.size()) {
      if (device_ms) *device_ms = total;
      return PMPIC_OK;  // not every candidate tried yet: tune again on the next run
    }
    e->threads = best;
    e->tuned_threads = true;
  }
  if (done < nsteps) {
    float ms = 0.f;
    int rc = run_members(e, nsteps - done, e->threads, &ms);
    if (rc) return rc;
    total += ms;
  }
  if (device_ms) *device_ms = total;
  return PMPIC_OK;
}

int pmpic_ensemble_tuning(pmpic_ensemble* e, int* threads, int32_t* xseg) {
  if (!e) return PMPIC_ERR_ARG;
  if (threads) *threads = e->threads;
  if (xseg)
    for (size_t i = 0; i < e->m.size(); ++i) xseg[i] = e->m[i]->p2g_xseg;
  return PMPIC_OK;
}

}  // extern "C"
