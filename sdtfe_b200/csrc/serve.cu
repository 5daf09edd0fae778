// serve.cu - the serving loop (dtfe_server_*): continuous batching of map
// requests over many device-resident meshes.
//
// One host thread runs the loop.  Each pass it
//   1. retires finished iterations and starts the device->host copy of every
//      request whose tiles have all been walked,
//   2. completes requests whose copies have landed (maps for pageable host
//      memory are copied by a second thread, so the loop never waits on them),
//   3. admits queued requests while a slot is free and the request's map plus
//      any walk records it still needs fit the device budget (records of idle
//      (mesh, axis) pairs are evicted least recently used first; a request
//      that could never fit is refused with DTFE_ERR_ADMISSION),
//   4. launches the next iteration: one persistent batch kernel per precision
//      over a slice of every active request's remaining tiles, quantum_rays
//      rays in all, more (up to 8x) while a backlog waits (DTFE_SERVE_FAIR:
//      split evenly, smallest remainder first; DTFE_SERVE_FIFO: oldest first).
// Iterations alternate between two streams and two may be in flight, so the
// next one fills the SMs while the previous one drains.  New requests join at
// the next iteration: continuous batching, not a queue in front of whole
// maps.  A request's pixels are each formed by one block from the pixel's
// own samples, so its map does not depend on what else shares a launch.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <new>
#include <thread>
#include <unordered_map>
#include <utility>
#include <vector>

#include "mesh.h"

using namespace sdtfe;
using Clock = std::chrono::steady_clock;

namespace {

constexpr int kSlots = 3;     // iteration job-table buffers
constexpr int kInFlight = 2;  // iterations on the GPU at once

struct Request {
  uint64_t id = 0;
  int mesh_id = 0;
  dtfe_map_params_t p{};
  double* host_map = nullptr;
  Clock::time_point t_submit, t_admit;
  MapGeom g{};
  size_t map_bytes = 0;
  double* d_map = nullptr;
  bool pageable = false;       // host_map is not pinned: the copier thread copies it
  int stat_slot = -1;
  long long tiles = 0, next_tile = 0;
  double rays_per_tile = 1;
  int inflight = 0;            // unfinished iterations holding some of its tiles
  int iterations = 0;
  bool holds_records = false;  // counted in its (mesh, axis) records' references
  bool copying = false, done = false;
  cudaEvent_t ev_copy = nullptr;
  cudaEvent_t ev_ready = nullptr;  // its records, map and counters are set up
  bool ready = false;              // ev_ready has been seen complete
  dtfe_request_info_t info{};
};

struct Resident {
  size_t bytes = 0;
  int refs = 0;
  unsigned long long last_use = 0;
};

struct Slot {
  bool busy = false;
  cudaEvent_t ev = nullptr;
  std::vector<Request*> reqs;
  unsigned char* h_jobs = nullptr;  // pinned
  void* d_jobs = nullptr;
  size_t cap = 0;
  void* d_loc = nullptr;  // mixed tiles' shared point locations
  size_t loc_cap = 0;
  unsigned long long* d_queue = nullptr;  // two counters: mixed, FP64
};

}  // namespace

struct dtfe_server_s {
  dtfe_server_config_t cfg{};
  int device = 0;
  std::vector<dtfe_mesh_t> meshes;
  bool auto_budget = false;  // device_budget follows the device's memory (config 0)
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<Request*> pending;
  std::vector<Request*> active;  // admission order
  std::unordered_map<uint64_t, Request*> requests;
  std::map<std::pair<int, int>, Resident> resident;
  std::vector<int> free_stat_slots;
  size_t in_use = 0, peak = 0;
  uint64_t next_id = 1;
  unsigned long long use_clock = 0;
  bool stop = false;
  dtfe_status_t fatal = DTFE_OK;
  std::thread thread;
  // requests whose map goes to the caller's pageable memory: copied by this
  // thread on its own stream (a pageable copy blocks the thread that issues
  // it), so that the loop keeps launching while large maps are copied out
  std::thread copier;
  cudaStream_t copy_out = nullptr;
  std::deque<Request*> copy_q;
  std::condition_variable cv_copy;
  bool copier_stop = false;
  cudaStream_t setup = nullptr, copy = nullptr, streams[2] = {nullptr, nullptr};
  cudaEvent_t ev_setup = nullptr;
  cudaMemPool_t pool = nullptr;
  Slot slot[kSlots];
  int next_stream = 0;
  unsigned long long* d_stats = nullptr;  // kStatCount per stat slot
  unsigned long long* h_stats = nullptr;  // pinned mirror
  dtfe_server_stats_t st{};
};

namespace {

using Server = dtfe_server_s;

double ms_between(Clock::time_point a, Clock::time_point b) {
  return std::chrono::duration<double, std::milli>(b - a).count();
}

// record bytes a request of (axis, precision) still needs on its mesh
size_t missing_record_bytes(const Mesh& m, int axis, int precision) {
  return mesh_missing_record_bytes(m, axis, precision);
}

size_t record_bytes(const Mesh& m, int axis) { return mesh_record_bytes(m, axis); }

void note_use(Server* S) {
  if (S->in_use > S->peak) S->peak = S->in_use;
}

// drops idle records, least recently used first, until `need` more bytes fit
bool make_room(Server* S, size_t need, std::pair<int, int> keep) {
  while (S->in_use + need > S->cfg.device_budget) {
    auto victim = S->resident.end();
    for (auto it = S->resident.begin(); it != S->resident.end(); ++it) {
      if (it->second.refs > 0 || it->first == keep || it->second.bytes == 0) continue;
      if (victim == S->resident.end() || it->second.last_use < victim->second.last_use) victim = it;
    }
    if (victim == S->resident.end()) return false;
    dtfe_mesh_t h = S->meshes[victim->first.first];
    {
      std::lock_guard<std::mutex> lk(h->mu);
      mesh_drop_records(&h->m, victim->first.second);
    }
    S->in_use -= victim->second.bytes;
    victim->second.bytes = 0;
    ++S->st.evictions;
  }
  return true;
}

void fail_request(Server* S, Request* r, dtfe_status_t s) {
  r->info.status = s;
  r->done = true;
  ++S->st.failed;
  S->cv_done.notify_all();
}

// releases what an admitted request holds (its tiles are no longer in flight)
void release(Server* S, Request* r) {
  if (r->d_map) {
    cudaFreeAsync(r->d_map, S->copy);
    S->in_use -= r->map_bytes;
    r->d_map = nullptr;
  }
  if (r->stat_slot >= 0) {
    S->free_stat_slots.push_back(r->stat_slot);
    r->stat_slot = -1;
  }
  if (r->holds_records) {
    auto it = S->resident.find({r->mesh_id, r->p.axis});
    if (it != S->resident.end()) --it->second.refs;
    r->holds_records = false;
  }
  if (r->ev_copy) {
    cudaEventDestroy(r->ev_copy);
    r->ev_copy = nullptr;
  }
  if (r->ev_ready) {
    cudaEventDestroy(r->ev_ready);
    r->ev_ready = nullptr;
  }
  S->active.erase(std::remove(S->active.begin(), S->active.end(), r), S->active.end());
}

dtfe_status_t admit_one(Server* S, Request* r) {
  dtfe_mesh_t h = S->meshes[r->mesh_id];
  Mesh& m = h->m;
  const std::pair<int, int> key{r->mesh_id, r->p.axis};
  Resident& res = S->resident[key];
  {
    std::lock_guard<std::mutex> lk(h->mu);
    const size_t before = record_bytes(m, r->p.axis);
    SDTFE_TRY(prepare_axis(m, r->p.axis, r->p.precision));
    const size_t after = record_bytes(m, r->p.axis);
    res.bytes += after - before;
    S->in_use += after - before;
    SDTFE_CUDA(cudaEventRecord(S->ev_setup, m.stream));
    SDTFE_CUDA(cudaStreamWaitEvent(S->setup, S->ev_setup, 0));
  }
  ++res.refs;
  r->holds_records = true;
  res.last_use = ++S->use_clock;
  r->g = map_geometry(m, r->p);
  SDTFE_CUDA(cudaMallocFromPoolAsync(reinterpret_cast<void**>(&r->d_map), r->map_bytes, S->pool, S->setup));
  S->in_use += r->map_bytes;
  note_use(S);
  SDTFE_CUDA(cudaMemsetAsync(r->d_map, 0, r->map_bytes, S->setup));
  r->stat_slot = S->free_stat_slots.back();
  S->free_stat_slots.pop_back();
  SDTFE_CUDA(cudaMemsetAsync(S->d_stats + (size_t)r->stat_slot * kStatCount, 0,
                             sizeof(unsigned long long) * kStatCount, S->setup));
  // only the iterations that walk this request's tiles wait for its set-up
  // (launch_iteration); the others keep the GPU busy meanwhile
  SDTFE_CUDA(cudaEventCreateWithFlags(&r->ev_ready, cudaEventDisableTiming));
  SDTFE_CUDA(cudaEventRecord(r->ev_ready, S->setup));
  r->ready = false;
  // pinned caller buffers take the copy directly
  cudaPointerAttributes pa{};
  const bool pinned = cudaPointerGetAttributes(&pa, r->host_map) == cudaSuccess &&
                      pa.type == cudaMemoryTypeHost;
  cudaGetLastError();  // a pageable pointer may leave an error behind on old drivers
  r->pageable = !pinned;
  SDTFE_CUDA(cudaEventCreateWithFlags(&r->ev_copy, cudaEventDisableTiming));
  r->tiles = r->p.precision == DTFE_MIXED ? map_tiles32(r->g, S->cfg.variant) : map_tiles64(r->g);
  r->rays_per_tile = (double)r->p.grid_dim * r->p.grid_dim * r->p.n_samples / (double)r->tiles;
  r->next_tile = 0;
  r->t_admit = Clock::now();
  r->info.queue_ms = ms_between(r->t_submit, r->t_admit);
  return DTFE_OK;
}

bool admit(Server* S) {
  bool progress = false;
  while (!S->pending.empty() && (int)S->active.size() < S->cfg.max_active) {
    Request* r = S->pending.front();
    const Mesh& m = S->meshes[r->mesh_id]->m;
    const std::pair<int, int> key{r->mesh_id, r->p.axis};
    const size_t need = r->map_bytes + missing_record_bytes(m, r->p.axis, r->p.precision);
    if (!make_room(S, need, key)) {
      bool idle = S->active.empty();
      for (const Slot& sl : S->slot) idle = idle && !sl.busy;
      if (!idle) break;  // wait for running requests to free memory
      // alone on the device and still too large: it can never run
      S->pending.pop_front();
      set_error(DTFE_ERR_ADMISSION, "request %llu needs %zu bytes; the budget is %zu",
                (unsigned long long)r->id, need, S->cfg.device_budget);
      fail_request(S, r, DTFE_ERR_ADMISSION);
      progress = true;
      continue;
    }
    S->pending.pop_front();
    S->active.push_back(r);
    dtfe_status_t s = admit_one(S, r);
    if (s == DTFE_ERR_NOMEM) {
      // the device had less room than the budget assumed: return the pool's
      // cached map memory, drop every idle (mesh, axis) record set and try
      // once more
      release(S, r);
      cudaStreamSynchronize(S->copy);
      cudaMemPoolTrimTo(S->pool, 0);
      make_room(S, S->cfg.device_budget + 1, key);
      S->active.push_back(r);
      s = admit_one(S, r);
    }
    if (s != DTFE_OK) {
      release(S, r);
      fail_request(S, r, s);
    }
    progress = true;
  }
  return progress;
}

// tiles of each request for the next iteration
void share_tiles(Server* S, std::vector<std::pair<Request*, long long>>* out) {
  // requests whose set-up (record build, map clearing) has finished first; the
  // others only when no ready request has tiles left, so that a record build
  // does not hold up the requests already running
  std::vector<Request*> rs, waiting;
  for (Request* r : S->active) {
    if (r->next_tile >= r->tiles) continue;
    if (!r->ready && r->ev_ready && cudaEventQuery(r->ev_ready) == cudaSuccess) r->ready = true;
    (r->ready ? rs : waiting).push_back(r);
  }
  if (rs.empty()) rs.swap(waiting);
  if (rs.empty()) return;
  auto rest = [](const Request* r) { return (double)(r->tiles - r->next_tile) * r->rays_per_tile; };
  // The iteration's rays: quantum_rays under light load (short iterations, so
  // new requests join soon); with a backlog, a quarter of the remaining work,
  // up to 8x the quantum (fewer, longer iterations: less per-launch cost).
  double backlog = 0.0;
  for (const Request* r : rs) backlog += rest(r);
  const double q = (double)S->cfg.quantum_rays;
  double budget = std::min(8.0 * q, std::max(q, 0.25 * backlog));
  if (S->cfg.policy == DTFE_SERVE_FAIR)
    std::stable_sort(rs.begin(), rs.end(), [&](Request* a, Request* b) { return rest(a) < rest(b); });
  size_t left = rs.size();
  for (Request* r : rs) {
    const double share = S->cfg.policy == DTFE_SERVE_FAIR ? budget / (double)left : budget;
    double rays = std::min(rest(r), share);
    long long t = (long long)(rays / r->rays_per_tile + 0.999999);
    if (t < 1) t = 1;
    if (t > r->tiles - r->next_tile) t = r->tiles - r->next_tile;
    out->push_back({r, t});
    budget -= (double)t * r->rays_per_tile;
    --left;
    if (budget <= 0) break;
  }
}

dtfe_status_t launch_iteration(Server* S, Slot& sl, const std::vector<std::pair<Request*, long long>>& take,
                               cudaStream_t s) {
  std::vector<BatchMap> maps[2];  // mixed, FP64
  for (const auto& rt : take) {
    Request* r = rt.first;
    if (!r->ready) SDTFE_CUDA(cudaStreamWaitEvent(s, r->ev_ready, 0));
    BatchMap b;
    b.mesh = &S->meshes[r->mesh_id]->m;
    b.g = r->g;
    b.d_map = r->d_map;
    b.stats = S->d_stats + (size_t)r->stat_slot * kStatCount;
    b.tile0 = (int)r->next_tile;
    b.count = (int)rt.second;
    maps[r->p.precision == DTFE_MIXED ? 0 : 1].push_back(b);
  }
  BatchPlan plans[2];
  SDTFE_TRY(plan_batch32(maps[0].data(), (int)maps[0].size(), S->cfg.variant, &plans[0]));
  SDTFE_TRY(plan_batch64(maps[1].data(), (int)maps[1].size(), &plans[1]));
  const size_t b0 = (plans[0].jobs.size() + 255) & ~size_t(255);
  const size_t bytes = b0 + plans[1].jobs.size();
  if (bytes > sl.cap) {
    if (sl.h_jobs) cudaFreeHost(sl.h_jobs);
    if (sl.d_jobs) cudaFree(sl.d_jobs);
    sl.h_jobs = nullptr;
    sl.d_jobs = nullptr;
    sl.cap = 0;
    const size_t cap = bytes * 2;
    SDTFE_CUDA(cudaMallocHost(reinterpret_cast<void**>(&sl.h_jobs), cap));
    SDTFE_CUDA(cudaMalloc(&sl.d_jobs, cap));
    sl.cap = cap;
  }
  // the slot's previous iteration has finished: its buffers can be replaced
  const size_t loc_bytes = kLocBytes * (size_t)plans[0].total_tiles;
  if (loc_bytes > sl.loc_cap) {
    if (sl.d_loc) cudaFree(sl.d_loc);
    sl.d_loc = nullptr;
    sl.loc_cap = 0;
    SDTFE_CUDA(cudaMalloc(&sl.d_loc, loc_bytes * 2));
    sl.loc_cap = loc_bytes * 2;
  }
  if (!plans[0].jobs.empty()) memcpy(sl.h_jobs, plans[0].jobs.data(), plans[0].jobs.size());
  if (!plans[1].jobs.empty()) memcpy(sl.h_jobs + b0, plans[1].jobs.data(), plans[1].jobs.size());
  SDTFE_CUDA(cudaMemcpyAsync(sl.d_jobs, sl.h_jobs, bytes, cudaMemcpyHostToDevice, s));
  SDTFE_CUDA(cudaMemsetAsync(sl.d_queue, 0, 2 * sizeof(unsigned long long), s));
  unsigned char* dj = static_cast<unsigned char*>(sl.d_jobs);
  if (plans[0].n_jobs) {
    int grid = 0, block = 0;
    SDTFE_TRY(batch_grid32(plans[0].variant, plans[0].smem, &grid, &block));
    SDTFE_TRY(launch_batch32(plans[0], dj, sl.d_queue, sl.d_loc, grid, s));
    ++S->st.iterations;
  }
  if (plans[1].n_jobs) {
    int grid = 0, block = 0;
    SDTFE_TRY(batch_grid64(plans[1].smem, &grid, &block));
    SDTFE_TRY(launch_batch64(plans[1], dj + b0, sl.d_queue + 1, grid, s));
    ++S->st.iterations;
  }
  SDTFE_CUDA(cudaEventRecord(sl.ev, s));
  return DTFE_OK;
}

bool launch_next(Server* S) {
  int busy = 0, free_slot = -1;
  for (int k = 0; k < kSlots; ++k) {
    if (S->slot[k].busy) ++busy;
    else if (free_slot < 0) free_slot = k;
  }
  if (busy >= kInFlight || free_slot < 0) return false;
  std::vector<std::pair<Request*, long long>> take;
  share_tiles(S, &take);
  if (take.empty()) return false;
  Slot& sl = S->slot[free_slot];
  cudaStream_t s = S->streams[S->next_stream];
  S->next_stream ^= 1;
  const dtfe_status_t st = launch_iteration(S, sl, take, s);
  if (st != DTFE_OK) {
    // a launch error is sticky for these requests: fail them
    S->fatal = st;
    for (const auto& rt : take) {
      Request* r = rt.first;
      if (r->inflight == 0) {
        release(S, r);
        fail_request(S, r, st);
      } else {
        r->next_tile = r->tiles;  // finishes (as failed) when its iterations retire
        r->info.status = st;
      }
    }
    return true;
  }
  sl.busy = true;
  sl.reqs.clear();
  for (const auto& rt : take) {
    Request* r = rt.first;
    r->next_tile += rt.second;
    ++r->inflight;
    ++r->iterations;
    sl.reqs.push_back(r);
  }
  return true;
}

void start_copy(Server* S, Request* r) {
  if (r->pageable) {  // every iteration holding its tiles has finished: the map is ready
    S->copy_q.push_back(r);
    S->cv_copy.notify_one();
    return;
  }
  cudaError_t e = cudaMemcpyAsync(r->host_map, r->d_map, r->map_bytes, cudaMemcpyDeviceToHost,
                                  S->copy);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(S->h_stats + (size_t)r->stat_slot * kStatCount,
                        S->d_stats + (size_t)r->stat_slot * kStatCount,
                        sizeof(unsigned long long) * kStatCount, cudaMemcpyDeviceToHost, S->copy);
  if (e == cudaSuccess) e = cudaEventRecord(r->ev_copy, S->copy);
  if (e != cudaSuccess) {
    set_error(DTFE_ERR_CUDA, "result copy: %s", cudaGetErrorString(e));
    release(S, r);
    fail_request(S, r, DTFE_ERR_CUDA);
    return;
  }
  r->copying = true;
}

bool retire(Server* S) {
  bool progress = false;
  for (Slot& sl : S->slot) {
    if (!sl.busy) continue;
    const cudaError_t e = cudaEventQuery(sl.ev);
    if (e == cudaErrorNotReady) continue;
    sl.busy = false;
    progress = true;
    for (Request* r : sl.reqs) {
      --r->inflight;
      if (e != cudaSuccess && r->info.status == DTFE_OK) {
        set_error(DTFE_ERR_CUDA, "iteration: %s", cudaGetErrorString(e));
        r->info.status = DTFE_ERR_CUDA;
      }
      if (r->inflight == 0 && r->next_tile >= r->tiles) {
        if (r->info.status != DTFE_OK) {
          release(S, r);
          fail_request(S, r, (dtfe_status_t)r->info.status);
        } else {
          start_copy(S, r);
        }
      }
    }
    sl.reqs.clear();
  }
  return progress;
}

// with S->mu held: the request's counters and latency, then its resources
void complete(Server* S, Request* r) {
  const unsigned long long* c = S->h_stats + (size_t)r->stat_slot * kStatCount;
  dtfe_map_stats_t& s = r->info.stats;
  memset(&s, 0, sizeof(s));
  s.rays = c[kStatRays];
  s.visits = c[kStatVisits];
  for (int k = 0; k < DTFE_N_RAY_STATUS; ++k) s.status[k] = c[kStatStatus0 + k];
  s.fp64_fallbacks = c[kStatFallback];
  r->info.iterations = r->iterations;
  r->info.latency_ms = ms_between(r->t_submit, Clock::now());
  r->info.status = DTFE_OK;
  release(S, r);
  r->done = true;
  ++S->st.completed;
  S->st.rays += s.rays;
  S->st.visits += s.visits;
}

bool finish_copies(Server* S) {
  std::vector<Request*> landed;
  for (Request* r : S->active)
    if (r->copying && cudaEventQuery(r->ev_copy) == cudaSuccess) landed.push_back(r);
  if (landed.empty()) return false;
  for (Request* r : landed) {
    r->copying = false;
    complete(S, r);
  }
  S->cv_done.notify_all();
  return true;
}

void copy_out_loop(Server* S) {
  cudaSetDevice(S->device);
  std::unique_lock<std::mutex> lk(S->mu);
  for (;;) {
    S->cv_copy.wait(lk, [&] { return S->copier_stop || !S->copy_q.empty(); });
    if (S->copy_q.empty()) return;  // stopping, nothing left
    Request* r = S->copy_q.front();
    S->copy_q.pop_front();
    unsigned long long* h = S->h_stats + (size_t)r->stat_slot * kStatCount;
    const unsigned long long* d = S->d_stats + (size_t)r->stat_slot * kStatCount;
    lk.unlock();
    cudaError_t e = cudaMemcpyAsync(r->host_map, r->d_map, r->map_bytes, cudaMemcpyDeviceToHost,
                                    S->copy_out);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(h, d, sizeof(unsigned long long) * kStatCount, cudaMemcpyDeviceToHost,
                          S->copy_out);
    if (e == cudaSuccess) e = cudaStreamSynchronize(S->copy_out);
    lk.lock();
    if (e == cudaSuccess) {
      complete(S, r);
    } else {
      set_error(DTFE_ERR_CUDA, "result copy: %s", cudaGetErrorString(e));
      release(S, r);
      fail_request(S, r, DTFE_ERR_CUDA);
    }
    S->cv_done.notify_all();
    S->cv_work.notify_one();  // the loop may be waiting for the memory this freed
  }
}

void loop(Server* S) {
  cudaSetDevice(S->device);
  std::unique_lock<std::mutex> lk(S->mu);
  for (;;) {
    bool progress = retire(S);
    progress |= finish_copies(S);
    progress |= admit(S);
    progress |= launch_next(S);
    bool busy = !S->active.empty();
    for (const Slot& sl : S->slot) busy = busy || sl.busy;
    if (S->stop && !busy && S->pending.empty()) break;
    if (!progress) {
      if (busy) S->cv_work.wait_for(lk, std::chrono::microseconds(50));
      else S->cv_work.wait(lk);
    }
  }
}

void free_server(Server* S) {
  for (cudaStream_t s : {S->setup, S->copy, S->copy_out, S->streams[0], S->streams[1]})
    if (s) cudaStreamSynchronize(s);
  for (auto& kv : S->requests) {
    Request* r = kv.second;
    if (r->d_map) cudaFreeAsync(r->d_map, S->copy);
    if (r->ev_copy) cudaEventDestroy(r->ev_copy);
    if (r->ev_ready) cudaEventDestroy(r->ev_ready);
    delete r;
  }
  if (S->copy) cudaStreamSynchronize(S->copy);
  for (Slot& sl : S->slot) {
    if (sl.ev) cudaEventDestroy(sl.ev);
    if (sl.h_jobs) cudaFreeHost(sl.h_jobs);
    if (sl.d_jobs) cudaFree(sl.d_jobs);
    if (sl.d_loc) cudaFree(sl.d_loc);
    if (sl.d_queue) cudaFree(sl.d_queue);
  }
  if (S->d_stats) cudaFree(S->d_stats);
  if (S->h_stats) cudaFreeHost(S->h_stats);
  if (S->ev_setup) cudaEventDestroy(S->ev_setup);
  for (cudaStream_t s : {S->setup, S->copy, S->copy_out, S->streams[0], S->streams[1]})
    if (s) cudaStreamDestroy(s);
  if (S->pool) cudaMemPoolDestroy(S->pool);
  delete S;
}

// The default budget: the device memory that is free now, less a reserve for
// everything else on the device (other allocations, the CUDA context's
// growth), plus what the server already accounts for (walk records of the
// registered meshes, live maps), which is in use and so not in the free
// figure.  Memory the record pool keeps for reuse counts as free: the
// server's record builds draw on the same pool.
dtfe_status_t set_auto_budget(Server* S) {
  SDTFE_CUDA(cudaDeviceSynchronize());
  mesh_trim_record_pool();
  size_t fr = 0, total = 0;
  SDTFE_CUDA(cudaMemGetInfo(&fr, &total));
  const size_t reserve = std::max<size_t>(size_t(2) << 30, total / 20);
  S->cfg.device_budget = (fr > reserve ? fr - reserve : 0) + S->in_use;
  S->st.budget = S->cfg.device_budget;
  return DTFE_OK;
}

}  // namespace

extern "C" {

dtfe_status_t dtfe_server_create(const dtfe_server_config_t* cfg, dtfe_server_t* out) {
  if (!out) return set_error(DTFE_ERR_INVALID, "out is NULL");
  *out = nullptr;
  auto* S = new (std::nothrow) Server();
  if (!S) return set_error(DTFE_ERR_NOMEM, "host allocation failed");
  if (cfg) S->cfg = *cfg;
  else S->cfg.variant = -1;
  if (S->cfg.max_active <= 0) S->cfg.max_active = 64;
  if (S->cfg.quantum_rays <= 0) S->cfg.quantum_rays = 1LL << 20;
  if (S->cfg.policy != DTFE_SERVE_FIFO) S->cfg.policy = DTFE_SERVE_FAIR;
  if (S->cfg.variant < -1 || S->cfg.variant >= num_map32_variants()) S->cfg.variant = -1;
  dtfe_status_t st = DTFE_OK;
  auto cuda = [&](cudaError_t e, const char* what) {
    if (e != cudaSuccess && st == DTFE_OK)
      st = set_error(e == cudaErrorMemoryAllocation ? DTFE_ERR_NOMEM : DTFE_ERR_CUDA, "%s: %s", what,
                     cudaGetErrorString(e));
  };
  cuda(cudaGetDevice(&S->device), "device");
  if (st == DTFE_OK && S->cfg.device_budget == 0) {
    S->auto_budget = true;
    st = set_auto_budget(S);
  }
  for (cudaStream_t* s : {&S->setup, &S->copy, &S->copy_out, &S->streams[0], &S->streams[1]})
    if (st == DTFE_OK) cuda(cudaStreamCreateWithFlags(s, cudaStreamNonBlocking), "stream");
  if (st == DTFE_OK) cuda(cudaEventCreateWithFlags(&S->ev_setup, cudaEventDisableTiming), "event");
  for (Slot& sl : S->slot) {
    if (st == DTFE_OK) cuda(cudaEventCreateWithFlags(&sl.ev, cudaEventDisableTiming), "event");
    if (st == DTFE_OK) cuda(cudaMalloc(&sl.d_queue, 2 * sizeof(unsigned long long)), "queue");
  }
  const size_t stat_bytes = sizeof(unsigned long long) * kStatCount * S->cfg.max_active;
  if (st == DTFE_OK) cuda(cudaMalloc(&S->d_stats, stat_bytes), "stats");
  if (st == DTFE_OK) cuda(cudaMallocHost(&S->h_stats, stat_bytes), "stats");
  if (st == DTFE_OK) {
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = S->device;
    cuda(cudaMemPoolCreate(&S->pool, &props), "memory pool");
    if (st == DTFE_OK) {
      uint64_t keep = S->cfg.device_budget;  // keep freed maps for reuse up to the budget
      cuda(cudaMemPoolSetAttribute(S->pool, cudaMemPoolAttrReleaseThreshold, &keep), "pool");
    }
  }
  if (st != DTFE_OK) {
    free_server(S);
    return st;
  }
  for (int k = S->cfg.max_active - 1; k >= 0; --k) S->free_stat_slots.push_back(k);
  S->st.budget = S->cfg.device_budget;
  try {
    S->copier = std::thread(copy_out_loop, S);
    S->thread = std::thread(loop, S);
  } catch (...) {
    if (S->copier.joinable()) {
      {
        std::lock_guard<std::mutex> lk(S->mu);
        S->copier_stop = true;
      }
      S->cv_copy.notify_all();
      S->copier.join();
    }
    free_server(S);
    return set_error(DTFE_ERR_NOMEM, "could not start the serving threads");
  }
  *out = S;
  return DTFE_OK;
}

dtfe_status_t dtfe_server_add_mesh(dtfe_server_t S, dtfe_mesh_t mesh, int* mesh_id) {
  if (!S || !mesh || !mesh_id) return set_error(DTFE_ERR_INVALID, "NULL argument");
  std::lock_guard<std::mutex> lk(S->mu);
  for (dtfe_mesh_t h : S->meshes)
    if (h == mesh) return set_error(DTFE_ERR_INVALID, "mesh already registered");
  // the projected hulls of all three axes now, so that no request waits for
  // one (they are small, and their build synchronises the mesh stream)
  {
    std::lock_guard<std::mutex> mk(mesh->mu);
    for (int a = 0; a < 3; ++a) SDTFE_TRY(mesh_hull(&mesh->m, a, nullptr, nullptr));
  }
  const int id = (int)S->meshes.size();
  S->meshes.push_back(mesh);
  for (int a = 0; a < 3; ++a) {
    size_t b = 0;
    {
      std::lock_guard<std::mutex> mk(mesh->mu);
      b = record_bytes(mesh->m, a);
    }
    if (!b) continue;
    Resident& r = S->resident[{id, a}];
    r.bytes = b;
    r.last_use = ++S->use_clock;
    S->in_use += b;
  }
  if (S->auto_budget) SDTFE_TRY(set_auto_budget(S));  // this mesh's records are in use, not free
  make_room(S, 0, {-1, -1});  // evict down to the budget (records of idle pairs only)
  note_use(S);
  *mesh_id = id;
  return DTFE_OK;
}

dtfe_status_t dtfe_server_submit(dtfe_server_t S, int mesh_id, const dtfe_map_params_t* p,
                                 double* map, uint64_t* request_id) {
  if (!S || !p || !map) return set_error(DTFE_ERR_INVALID, "NULL argument");
  auto* r = new (std::nothrow) Request();
  if (!r) return set_error(DTFE_ERR_NOMEM, "host allocation failed");
  std::unique_lock<std::mutex> lk(S->mu);
  if (mesh_id < 0 || mesh_id >= (int)S->meshes.size()) {
    delete r;
    return set_error(DTFE_ERR_INVALID, "mesh id %d not registered", mesh_id);
  }
  if (S->stop) {
    delete r;
    return set_error(DTFE_ERR_INVALID, "server is shutting down");
  }
  if (S->fatal != DTFE_OK) {  // a launch failed: the device context may be unusable
    delete r;
    return set_error(S->fatal, "server stopped after a failed launch");
  }
  const dtfe_status_t c = check_params(S->meshes[mesh_id]->m, p);
  if (c != DTFE_OK) {
    delete r;
    return c;
  }
  r->id = S->next_id++;
  r->mesh_id = mesh_id;
  r->p = *p;
  r->host_map = map;
  r->map_bytes = sizeof(double) * (size_t)p->grid_dim * p->grid_dim;
  r->t_submit = Clock::now();
  S->requests[r->id] = r;
  S->pending.push_back(r);
  ++S->st.submitted;
  if (request_id) *request_id = r->id;
  lk.unlock();
  S->cv_work.notify_one();
  return DTFE_OK;
}

dtfe_status_t dtfe_server_wait(dtfe_server_t S, uint64_t request_id, int timeout_ms,
                               dtfe_request_info_t* info) {
  if (!S) return set_error(DTFE_ERR_INVALID, "NULL server");
  std::unique_lock<std::mutex> lk(S->mu);
  auto it = S->requests.find(request_id);
  if (it == S->requests.end())
    return set_error(DTFE_ERR_INVALID, "request %llu unknown or already collected",
                     (unsigned long long)request_id);
  Request* r = it->second;
  auto ready = [&] { return r->done; };
  if (timeout_ms < 0) S->cv_done.wait(lk, ready);
  else if (!S->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready))
    return set_error(DTFE_ERR_TIMEOUT, "request %llu still running", (unsigned long long)request_id);
  if (info) *info = r->info;
  const dtfe_status_t s = (dtfe_status_t)r->info.status;
  S->requests.erase(it);
  delete r;
  if (s != DTFE_OK) return set_error(s, "request %llu failed (status %d)", (unsigned long long)request_id, (int)s);
  return DTFE_OK;
}

dtfe_status_t dtfe_server_stats(dtfe_server_t S, dtfe_server_stats_t* out) {
  if (!S || !out) return set_error(DTFE_ERR_INVALID, "NULL argument");
  std::lock_guard<std::mutex> lk(S->mu);
  *out = S->st;
  out->budget = S->cfg.device_budget;
  out->in_use = S->in_use;
  out->peak = S->peak;
  out->active = (int)S->active.size();
  out->queued = (int)S->pending.size();
  return DTFE_OK;
}

dtfe_status_t dtfe_server_destroy(dtfe_server_t S) {
  if (!S) return DTFE_OK;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    S->stop = true;
  }
  S->cv_work.notify_all();
  if (S->thread.joinable()) S->thread.join();  // returns once nothing is active
  {
    std::lock_guard<std::mutex> lk(S->mu);
    S->copier_stop = true;
  }
  S->cv_copy.notify_all();
  if (S->copier.joinable()) S->copier.join();
  free_server(S);
  return DTFE_OK;
}

}  // extern "C"
