// Continuous-batching request server over the segpu C-ABI (include/segpu.h).
//
// Requests (a Helmholtz/Poisson solve, or an n-step first-order SL advection
// job) are queued by se_server_submit from any thread. One worker thread
// owns the GPU work: it admits queued requests in arrival order into free
// execution slots (one CUDA stream each) whenever the device-memory budget
// allows the resources the request needs, queues the request's whole device
// work on the slot's stream without waiting, and completes requests by
// polling each slot's completion event. Requests that arrive while others run
// are admitted as slots and memory free up, so their device work overlaps.
//
// Resources are cached per configuration (mesh, boundary conditions,
// coefficients, solver options): a finished request returns its instance to
// a free list, and the least recently used free instances are released when
// a new configuration does not fit the budget. Every result is computed by
// the same deterministic kernels whether a request runs alone or in a mix.
#include <cuda_runtime.h>

#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <list>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/segpu.h"

namespace {

double now_ms() {
  using namespace std::chrono;
  return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}

struct Instance {
  std::string key;
  size_t bytes = 0;
  int kind = 0;
  se_mesh* mesh = nullptr;
  se_bcs* bcs = nullptr;
  se_field* a = nullptr;  // Helmholtz: right-hand side;  advection: tracer
  se_field* b = nullptr;  // Helmholtz: solution;         advection: velocity
  se_linsys* ls = nullptr;
  se_advector* adv = nullptr;
  se_field* sl = nullptr;  // advection: fieldSL (owned by adv)
  int nv = 0;
  bool busy = false;
  unsigned long long last_used = 0;
};

void release(Instance* in) {
  if (in->adv) se_advector_destroy(in->adv);
  if (in->ls) se_linsys_destroy(in->ls);
  if (in->a) se_field_destroy(in->a);
  if (in->b) se_field_destroy(in->b);
  if (in->bcs) se_bcs_destroy(in->bcs);
  if (in->mesh) se_mesh_destroy(in->mesh);
  delete in;
}

struct Job {
  long long ticket = 0;
  se_request req;
  std::string key;  // configuration key, formed by the submitting thread
  double t_submit = 0, t_admit = 0, t_done = 0;
  Instance* inst = nullptr;
  int slot = -1;
  bool done = false;
  bool out_direct = false;  // the result is copied straight into req.out
  se_result res;
};

// Page-locked host memory can be the source or destination of an
// asynchronous copy directly; other memory goes through the slot's staging.
// The answer is cached per address (clients reuse their buffers); a stale
// entry only changes the copy path, not the result: pageable memory given to
// an asynchronous copy is copied synchronously by the runtime.
bool pinned(const void* p) {
  static thread_local std::unordered_map<const void*, bool> cache;
  auto it = cache.find(p);
  if (it != cache.end()) return it->second;
  cudaPointerAttributes at;
  bool pin = false;
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess)
    cudaGetLastError();
  else
    pin = at.type == cudaMemoryTypeHost;
  if (cache.size() > 4096) cache.clear();
  cache[p] = pin;
  return pin;
}

struct Slot {
  cudaStream_t s = nullptr;
  cudaEvent_t ev = nullptr;
  double* h = nullptr;  // pinned staging: [cap] in, [2*cap] aux, [cap] out
  size_t cap = 0;
  Job* job = nullptr;
};

}  // namespace

struct se_server {
  std::thread worker;
  std::mutex mu;
  std::condition_variable cv_submit, cv_done;
  std::deque<Job*> queue;
  std::map<long long, Job*> jobs;
  long long next_ticket = 1;
  std::vector<Slot> slots;
  std::map<std::string, std::list<Instance*>> pool;  // all instances by key
  size_t budget = 0, used = 0;
  unsigned long long clock = 0;
  bool stop = false;
  int device = 0;
  int active = 0;
};

namespace {

std::string key_of(const se_request& r) {
  char buf[512];
  if (r.kind == SE_REQ_HELMHOLTZ)
    snprintf(buf, sizeof(buf), "H|%d|%d|%d|%.17g|%.17g|%.17g|%.17g|%d%d|%d%d%d%d|%.17g|%.17g|%.17g|%d|%d|%d|%d|%d",
             r.nEls[0], r.nEls[1], r.N, r.min[0], r.min[1], r.max[0], r.max[1], r.periodic[0],
             r.periodic[1], r.bcs[0], r.bcs[1], r.bcs[2], r.bcs[3], r.c, r.nu, r.dt, r.poisson,
             r.opts.method, r.opts.precision, r.opts.mode, r.opts.norm_type);
  else
    snprintf(buf, sizeof(buf), "A|%d|%d|%d|%.17g|%.17g|%.17g|%.17g|%d%d", r.nEls[0], r.nEls[1],
             r.N, r.min[0], r.min[1], r.max[0], r.max[1], r.periodic[0], r.periodic[1]);
  return buf;
}

int nverts(const se_request& r) {
  return (r.nEls[0] * r.N + 1) * (r.nEls[1] * r.N + 1);
}

// Device bytes an instance of this request holds (fields, solver vectors,
// fast-diagonalization buffers and eigenvectors, CUDA-graph workspace).
size_t estimate(const se_request& r) {
  const size_t nv = (size_t)nverts(r);
  if (r.kind == SE_REQ_ADVECT) return nv * 8 * 4;  // tracer, velocity (2), fieldSL
  const size_t gx = (size_t)r.nEls[0] * r.N + 1, gy = (size_t)r.nEls[1] * r.N + 1;
  return nv * 8 * 2 + nv * 8 * 13 + (gx * gx + gy * gy) * 8 * 2 + (4u << 20);
}

int create(se_server* S, const se_request& r, Instance** out) {
  Instance* in = new Instance();
  in->kind = r.kind;
  in->key = key_of(r);
  in->bytes = estimate(r);
  int rc = se_mesh_create(r.nEls, r.N, r.min, r.max, r.periodic, &in->mesh);
  if (!rc) rc = se_mesh_sizes(in->mesh, nullptr, &in->nv);
  if (!rc && r.kind == SE_REQ_HELMHOLTZ) {
    rc = se_bcs_create(in->mesh, r.bcs[0], r.bcs[1], r.bcs[2], r.bcs[3], &in->bcs);
    if (!rc) rc = se_field_create(in->mesh, 1, in->bcs, &in->a);
    if (!rc) rc = se_field_create(in->mesh, 1, in->bcs, &in->b);
    if (!rc)
      rc = r.poisson ? se_poisson_create(in->b, in->a, r.c, &r.opts, &in->ls)
                     : se_helmholtz_create(in->b, in->a, r.c, r.nu, r.dt, 0, &r.opts, &in->ls);
  } else if (!rc) {
    rc = se_field_create(in->mesh, 1, nullptr, &in->a);
    if (!rc) rc = se_field_create(in->mesh, 2, nullptr, &in->b);
    if (!rc) rc = se_advector_create(in->a, in->b, nullptr, nullptr, &in->adv);
    if (!rc) rc = se_advector_field_sl(in->adv, &in->sl);
  }
  if (rc) {
    release(in);
    return rc;
  }
  S->pool[in->key].push_back(in);
  S->used += in->bytes;
  *out = in;
  return SE_OK;
}

// A free instance for the request, creating one (after releasing least
// recently used free instances) if the budget allows. Returns SE_OK with
// *out == nullptr when the request must wait for memory.
int acquire(se_server* S, const se_request& r, const std::string& key, Instance** out) {
  *out = nullptr;
  auto& lst = S->pool[key];
  for (Instance* in : lst)
    if (!in->busy) {
      *out = in;
      return SE_OK;
    }
  const size_t need = estimate(r);
  while (S->used + need > S->budget) {
    Instance* victim = nullptr;
    for (auto& kv : S->pool)
      for (Instance* in : kv.second)
        if (!in->busy && (!victim || in->last_used < victim->last_used)) victim = in;
    if (!victim) break;
    S->pool[victim->key].remove(victim);
    S->used -= victim->bytes;
    release(victim);
  }
  if (S->used + need > S->budget && S->active > 0) return SE_OK;  // wait for running work
  return create(S, r, out);
}

// The worker thread's last library message, or the CUDA error pending on it.
void note_error(Job* j, int rc) {
  if (rc == SE_OK || j->res.error[0]) return;
  const char* m = se_last_error();
  const cudaError_t e = cudaGetLastError();
  if (m && m[0])
    snprintf(j->res.error, sizeof(j->res.error), "%s", m);
  else
    snprintf(j->res.error, sizeof(j->res.error), "%s", cudaGetErrorString(e));
}

void fail_job(se_server* S, Job* j, int rc) {
  note_error(j, rc);
  j->res.status = rc;
  j->t_done = now_ms();
  j->res.queued_ms = (j->t_admit > 0 ? j->t_admit : j->t_done) - j->t_submit;
  j->res.latency_ms = j->t_done - j->t_submit;
  j->done = true;
  S->cv_done.notify_all();
}

// Record a failed CUDA runtime call in the job's result.
int cuda_failed(Job* j, cudaError_t e, const char* what) {
  snprintf(j->res.error, sizeof(j->res.error), "%s: %s", what, cudaGetErrorString(e));
  cudaGetLastError();
  return e == cudaErrorMemoryAllocation ? SE_ERR_OOM : SE_ERR_CUDA;
}

// Queue the request's device work on the slot's stream.
int start(se_server* S, Job* j, Slot& sl) {
  const se_request& r = j->req;
  Instance* in = j->inst;
  const size_t nv = (size_t)in->nv;
  cudaError_t e;
  if (sl.cap < nv) {
    if (sl.h) cudaFreeHost(sl.h);
    sl.h = nullptr;
    sl.cap = 0;
    if ((e = cudaMallocHost((void**)&sl.h, sizeof(double) * 4 * nv)) != cudaSuccess)
      return cuda_failed(j, e, "staging cudaMallocHost");
    sl.cap = nv;
  }
  double *h_in = sl.h, *h_aux = sl.h + sl.cap, *h_out = sl.h + 3 * sl.cap;
  se_set_stream(sl.s);
  double *da = nullptr, *db = nullptr;
  se_field_device_ptr(in->a, &da);
  se_field_device_ptr(in->b, &db);
  // host -> device through staging unless the caller's array is page-locked
  auto upload = [&](double* dst, const double* src, double* stage, size_t count) {
    const double* from = src;
    if (!pinned(src)) {
      std::memcpy(stage, src, sizeof(double) * count);
      from = stage;
    }
    const cudaError_t ue =
        cudaMemcpyAsync(dst, from, sizeof(double) * count, cudaMemcpyHostToDevice, sl.s);
    return ue == cudaSuccess ? SE_OK : cuda_failed(j, ue, "input upload");
  };
  j->out_direct = pinned(r.out);
  double* dst_out = j->out_direct ? r.out : h_out;
  if (int rc = upload(da, r.in, h_in, nv)) return rc;
  int rc = SE_OK;
  if (r.kind == SE_REQ_HELMHOLTZ) {
    if (r.aux) {
      if (int rc2 = upload(db, r.aux, h_aux, nv)) return rc2;
    } else if ((e = cudaMemsetAsync(db, 0, sizeof(double) * nv, sl.s)) != cudaSuccess) {
      return cuda_failed(j, e, "solution clear");
    }
    rc = se_linsys_assemble(in->ls);  // the Dirichlet lifting of this request's values
    if (!rc) rc = se_linsys_solve_async(in->ls, 0);
    if (rc) return rc;
    if ((e = cudaMemcpyAsync(dst_out, db, sizeof(double) * nv, cudaMemcpyDeviceToHost, sl.s)) != cudaSuccess)
      return cuda_failed(j, e, "result download");
  } else {
    if (int rc2 = upload(db, r.aux, h_aux, 2 * nv)) return rc2;
    for (int k = 0; k < r.steps && !rc; k++) {
      rc = se_advect(in->adv, r.sl_dt);
      if (!rc) rc = se_field_copy(in->a, in->sl);
    }
    if (rc) return rc;
    if ((e = cudaMemcpyAsync(dst_out, da, sizeof(double) * nv, cudaMemcpyDeviceToHost, sl.s)) != cudaSuccess)
      return cuda_failed(j, e, "result download");
  }
  if ((e = cudaEventRecord(sl.ev, sl.s)) != cudaSuccess) return cuda_failed(j, e, "completion event");
  return SE_OK;
}

void finish(se_server* S, Slot& sl) {
  Job* j = sl.job;
  Instance* in = j->inst;
  se_set_stream(sl.s);
  int rc = SE_OK;
  if (in->kind == SE_REQ_HELMHOLTZ) {
    se_solve_stats st;
    rc = se_linsys_solve_finish(in->ls, &st);
    j->res.reason = st.reason;
    j->res.its = st.its;
    if (rc == SE_ERR_NOT_CONVERGED) rc = SE_OK;  // reported through reason
  }
  note_error(j, rc);
  if (!j->out_direct) std::memcpy(j->req.out, sl.h + 3 * sl.cap, sizeof(double) * in->nv);
  std::lock_guard<std::mutex> lk(S->mu);
  in->busy = false;
  in->last_used = ++S->clock;
  sl.job = nullptr;
  S->active--;
  j->res.status = rc;
  j->t_done = now_ms();
  j->res.queued_ms = j->t_admit - j->t_submit;
  j->res.latency_ms = j->t_done - j->t_submit;
  j->done = true;
  S->cv_done.notify_all();
}

void worker_loop(se_server* S) {
  cudaSetDevice(S->device);
  for (;;) {
    bool progress = false;
    // admit in arrival order while slots and memory allow
    for (;;) {
      std::unique_lock<std::mutex> lk(S->mu);
      if (S->queue.empty()) break;
      int free_slot = -1;
      for (size_t k = 0; k < S->slots.size(); k++)
        if (!S->slots[k].job) {
          free_slot = (int)k;
          break;
        }
      if (free_slot < 0) break;
      Job* j = S->queue.front();
      Instance* in = nullptr;
      lk.unlock();
      int rc = acquire(S, j->req, j->key, &in);
      lk.lock();
      if (rc) {
        S->queue.pop_front();
        fail_job(S, j, rc);
        progress = true;
        continue;
      }
      if (!in) break;  // waits for memory held by running requests
      S->queue.pop_front();
      in->busy = true;
      j->inst = in;
      j->slot = free_slot;
      j->t_admit = now_ms();
      Slot& sl = S->slots[free_slot];
      sl.job = j;
      S->active++;
      lk.unlock();
      rc = start(S, j, sl);
      if (rc) {
        lk.lock();
        in->busy = false;
        sl.job = nullptr;
        S->active--;
        fail_job(S, j, rc);
      }
      progress = true;
    }
    // complete finished requests
    for (Slot& sl : S->slots)
      if (sl.job && cudaEventQuery(sl.ev) == cudaSuccess) {
        finish(S, sl);
        progress = true;
      }
    std::unique_lock<std::mutex> lk(S->mu);
    if (S->stop && S->queue.empty() && S->active == 0) break;
    if (!progress) {
      if (S->active > 0) {
        lk.unlock();
        std::this_thread::yield();
      } else {
        S->cv_submit.wait_for(lk, std::chrono::milliseconds(5));
      }
    }
  }
}

}  // namespace

extern "C" {

int se_server_create(int slots, double device_gib, se_server** out) {
  if (!out || slots < 1 || slots > 64 || !(device_gib > 0)) return SE_ERR_ARG;
  *out = nullptr;
  se_server* S = new se_server();
  cudaGetDevice(&S->device);
  S->budget = (size_t)(device_gib * (1ull << 30));
  S->slots.resize(slots);
  for (Slot& sl : S->slots) {
    if (cudaStreamCreateWithFlags(&sl.s, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&sl.ev, cudaEventDisableTiming) != cudaSuccess) {
      delete S;
      return SE_ERR_CUDA;
    }
  }
  S->worker = std::thread(worker_loop, S);
  *out = S;
  return SE_OK;
}

int se_server_submit(se_server* S, const se_request* req, long long* ticket) {
  if (!S || !req || !ticket || !req->in || !req->out) return SE_ERR_ARG;
  if (req->kind != SE_REQ_HELMHOLTZ && req->kind != SE_REQ_ADVECT) return SE_ERR_ARG;
  if (req->kind == SE_REQ_ADVECT && (!req->aux || req->steps < 0)) return SE_ERR_ARG;
  Job* j = new Job();
  j->req = *req;
  j->key = key_of(*req);
  std::memset(&j->res, 0, sizeof(j->res));
  j->t_submit = now_ms();
  {
    std::lock_guard<std::mutex> lk(S->mu);
    if (S->stop) {
      delete j;
      return SE_ERR_ARG;
    }
    j->ticket = S->next_ticket++;
    S->jobs[j->ticket] = j;
    S->queue.push_back(j);
    *ticket = j->ticket;
  }
  S->cv_submit.notify_one();
  return SE_OK;
}

int se_server_wait(se_server* S, long long ticket, se_result* res) {
  if (!S) return SE_ERR_ARG;
  std::unique_lock<std::mutex> lk(S->mu);
  auto it = S->jobs.find(ticket);
  if (it == S->jobs.end()) return SE_ERR_ARG;
  Job* j = it->second;
  S->cv_done.wait(lk, [&] { return j->done; });
  if (res) *res = j->res;
  S->jobs.erase(it);
  delete j;
  return SE_OK;
}

int se_server_destroy(se_server* S) {
  if (!S) return SE_OK;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    S->stop = true;
  }
  S->cv_submit.notify_one();
  if (S->worker.joinable()) S->worker.join();
  for (auto& kv : S->pool)
    for (Instance* in : kv.second) release(in);
  for (Slot& sl : S->slots) {
    if (sl.h) cudaFreeHost(sl.h);
    if (sl.ev) cudaEventDestroy(sl.ev);
    if (sl.s) cudaStreamDestroy(sl.s);
  }
  for (auto& kv : S->jobs) delete kv.second;
  delete S;
  return SE_OK;
}

}  // extern "C"
