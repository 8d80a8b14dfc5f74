// serve.cu -- the serving loop (sparc_serve_* of include/sparc_gpu.h): solve
// requests (grid, background, source, duration) arrive at any time, are
// admitted first-in first-out by a device-memory budget and a slot count,
// and run as members of one batch (batch.cu) whose steps overlap on the
// device with the set-up of newly admitted requests.  A worker thread owns
// the batch: each round it adds the requests whose handles were attached,
// enqueues `quantum` batched steps, waits for them, retires the members
// that finished and admits queued requests as budget frees up.
//
// Request life cycle (ticket states):
//   QUEUED   submitted (parameters only; nothing allocated)
//   ADMITTED budget reserved at the peak set-up size; the client now builds
//            the handle (sparc_create / set_background / set_source)
//   RUNNING  attached; a member of the batch (reservation drops to the
//            resident size)
//   DONE     its iterations are done; removed from the batch
//   COLLECTED the client took the handle back (sparc_serve_result)
// sparc_serve_release ends the ticket and returns its budget.
//
// The reference has no counterpart (one simulation per MPI job).

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "internal.h"

namespace sparc {

// Device bytes of a SPARC_FP32 handle: resident (state, carry, FP32
// coefficients, CPML fields and profiles, forcing tables) and at the peak
// of its set-up (plus the FP64 setup arrays released after conversion).
void estimate_bytes32(const sparc_params &P, int64_t *resident, int64_t *peak) {
  const long long N = (long long)P.nx * P.ny * P.nz;
  const bool mhd = P.magnetic == 2;
  const int V = mhd ? 8 : 5, Pp = mhd ? 6 : 2;
  const bool hp = P.use_hpml != 0, pml = P.use_pml != 0 || hp;
  long long face_cnt = 0;
  if (pml) face_cnt += (long long)P.nx * P.ny * (P.npml_zb + P.npml_zt);
  if (hp)
    face_cnt += (long long)P.ny * P.nz * (P.npml_xb + P.npml_xt) +
                (long long)P.nx * P.nz * (P.npml_yb + P.npml_yt);
  const bool bg1d = P.magnetic == 0 && P.periodic;
  const long long bg3d = mhd ? 18 : (bg1d ? 0 : 7);
  long long res = 4 * (3LL * V * N + V * N);       // state buffers + carry
  res += 4 * (bg3d * N + 2 * N);                   // background, source damping
  res += 4 * face_cnt * (2 * Pp + 3);              // psi, stage psi, profiles
  res += 8 * (long long)P.nz * 8 + (1 << 20);      // profiles, tables, bookkeeping
  res += 12 * (long long)P.nx * P.ny * std::max(1, P.nz / 4);  // PSR forcing planes
  long long fp64 = 8 * (23LL * N + 3 * face_cnt);  // setup arrays (released)
  *resident = res;
  *peak = res + fp64;
}

struct Ticket {
  int64_t id = 0;
  sparc_params p{};
  int64_t first = 0, steps = 0;
  int state = SPARC_REQ_QUEUED;
  int64_t resident = 0, peak = 0, reserved = 0;
  Handle *h = nullptr;
  int slot = -1;
  int64_t left = 0;    // iterations left when last seen
  bool taken_build = false;    // ADMITTED ticket handed to a client to build
  bool taken_collect = false;  // DONE/FAILED ticket handed to a client
  double t_submit = 0, t_admit = 0, t_start = 0, t_done = 0;
};

struct Server {
  int device = 0;
  sparc_batch *batch = nullptr;
  int capacity = 0, quantum = 10;
  int64_t budget = 0, used = 0;
  std::thread worker;
  std::mutex mu;
  std::condition_variable cv;
  bool stop = false;
  int64_t next_id = 1;
  std::deque<int64_t> queue;
  std::map<int64_t, Ticket> tickets;
  std::vector<int64_t> to_attach;
  int active = 0;  // ADMITTED + RUNNING
  int max_active = 0;
  int running = 0, max_running = 0;  // members of the batch
  int64_t joined = 0;                // attached while others were running
  // steps per round: as many as fit in about round_s seconds (at most
  // quantum), so a built request waits about that long to be attached
  double round_s = 0.25, step_s = 0.0;
  int64_t steps_run = 0, rounds = 0;
  double point_updates = 0, gpu_busy_s = 0;
  std::string err;
  std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
  double now() const {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  }
};

static void admit_locked(Server *s) {
  while (!s->queue.empty() && s->active < s->capacity) {
    Ticket &t = s->tickets[s->queue.front()];
    if (s->used + t.peak > s->budget) break;  // first-in first-out
    s->queue.pop_front();
    t.state = SPARC_REQ_ADMITTED;
    t.reserved = t.peak;
    s->used += t.peak;
    t.t_admit = s->now();
    ++s->active;
    s->max_active = std::max(s->max_active, s->active);
  }
}

static void serve_loop(Server *s) {
  cudaSetDevice(s->device);
  std::vector<int64_t> rem(s->capacity);
  std::vector<double> pts(s->capacity, 0.0);
  while (true) {
    std::vector<int64_t> attach;
    bool work = false;
    {
      std::unique_lock<std::mutex> lock(s->mu);
      admit_locked(s);
      s->cv.notify_all();
      attach.swap(s->to_attach);
      for (auto &kv : s->tickets)
        if (kv.second.state == SPARC_REQ_RUNNING) work = true;
      if (!work && attach.empty()) {
        if (s->stop) return;
        s->cv.wait_for(lock, std::chrono::milliseconds(2));
        continue;
      }
    }
    for (int64_t id : attach) {  // batch calls happen on this thread only
      Ticket *t;
      {
        std::lock_guard<std::mutex> lock(s->mu);
        t = &s->tickets[id];
      }
      int slot = -1;
      int r = sparc_batch_add(s->batch, reinterpret_cast<sparc_handle *>(t->h), t->first,
                              t->steps, &slot);
      std::lock_guard<std::mutex> lock(s->mu);
      if (r) {
        t->state = SPARC_REQ_FAILED;
        t->t_done = s->now();
        s->err = sparc_batch_last_error(s->batch);
        continue;
      }
      t->slot = slot;
      t->left = t->steps;
      t->state = SPARC_REQ_RUNNING;
      t->t_start = s->now();
      if (s->running > 0) ++s->joined;
      ++s->running;
      s->max_running = std::max(s->max_running, s->running);
      s->used -= t->reserved - t->resident;  // set-up memory is released
      t->reserved = t->resident;
      pts[slot] = (double)t->p.nx * t->p.ny * t->p.nz;
      work = true;
    }
    if (!work) continue;
    int steps = s->quantum;
    if (s->step_s > 0.0)
      steps = std::max(1, std::min(s->quantum, (int)(s->round_s / s->step_s)));
    const double g0 = s->now();
    int r = sparc_batch_run(s->batch, steps);
    if (!r) r = sparc_batch_remaining(s->batch, rem.data());  // waits for the steps
    const double g1 = s->now();
    std::lock_guard<std::mutex> lock(s->mu);
    s->gpu_busy_s += g1 - g0;
    s->step_s = (g1 - g0) / steps;
    ++s->rounds;
    s->steps_run += steps;
    if (r) {
      s->err = sparc_batch_last_error(s->batch);
      for (auto &kv : s->tickets)
        if (kv.second.state == SPARC_REQ_RUNNING) {
          kv.second.state = SPARC_REQ_FAILED;
          kv.second.t_done = g1;
        }
      s->running = 0;
      s->stop = true;
      s->cv.notify_all();
      return;
    }
    for (auto &kv : s->tickets) {
      Ticket &t = kv.second;
      if (t.state != SPARC_REQ_RUNNING) continue;
      s->point_updates += pts[t.slot] * (double)(t.left - rem[t.slot]);
      t.left = rem[t.slot];
      if (rem[t.slot] == 0) {
        sparc_batch_remove(s->batch, t.slot);
        t.slot = -1;
        t.state = SPARC_REQ_DONE;
        t.t_done = g1;
        --s->running;
      }
    }
    s->cv.notify_all();
  }
}

}  // namespace sparc

using namespace sparc;

struct sparc_server : Server {};

extern "C" {

int sparc_estimate_bytes(const sparc_params *p, int64_t *resident, int64_t *peak) {
  if (!p || !resident || !peak) return SPARC_ERR_INVALID;
  estimate_bytes32(*p, resident, peak);
  return SPARC_OK;
}

int sparc_server_create(int device, int capacity, int64_t budget_bytes, int quantum,
                        sparc_server **out) {
  if (!out || capacity < 1 || budget_bytes <= 0 || quantum < 1) return SPARC_ERR_INVALID;
  *out = nullptr;
  sparc_server *s = new (std::nothrow) sparc_server();
  if (!s) return SPARC_ERR_NOMEM;
  int r = sparc_batch_create(device, capacity, &s->batch);
  if (r) {
    delete s;
    return r;
  }
  s->device = device;
  s->capacity = capacity;
  s->budget = budget_bytes;
  s->quantum = quantum;
  s->worker = std::thread(serve_loop, s);
  *out = s;
  return SPARC_OK;
}

int sparc_server_destroy(sparc_server *s) {
  if (!s) return SPARC_ERR_INVALID;
  {
    std::lock_guard<std::mutex> lock(s->mu);
    s->stop = true;
    for (auto &kv : s->tickets)  // members stop stepping
      if (kv.second.state == SPARC_REQ_RUNNING) kv.second.state = SPARC_REQ_FAILED;
    s->to_attach.clear();
  }
  s->cv.notify_all();
  if (s->worker.joinable()) s->worker.join();
  sparc_batch_destroy(s->batch);  // removes remaining members
  delete s;
  return SPARC_OK;
}

int sparc_serve_submit(sparc_server *s, const sparc_params *p, int64_t first, int64_t steps,
                       int64_t *ticket) {
  if (!s || !p || !ticket || steps < 0) return SPARC_ERR_INVALID;
  if (p->precision != SPARC_FP32) {
    s->err = "served requests use SPARC_FP32";
    return SPARC_ERR_INVALID;
  }
  Ticket t;
  t.p = *p;
  t.first = first;
  t.steps = steps;
  estimate_bytes32(*p, &t.resident, &t.peak);
  std::lock_guard<std::mutex> lock(s->mu);
  if (t.peak > s->budget) {
    s->err = "request needs " + std::to_string(t.peak) + " bytes, above the budget of " +
             std::to_string(s->budget);
    return SPARC_ERR_NOMEM;
  }
  if (s->stop) return SPARC_ERR_ORDER;
  t.id = s->next_id++;
  t.t_submit = s->now();
  s->tickets[t.id] = t;
  s->queue.push_back(t.id);
  *ticket = t.id;
  s->cv.notify_all();
  return SPARC_OK;
}

// Waits up to timeout_ms for a ticket in `state` (ADMITTED or DONE) that no
// client has taken yet; returns SPARC_ERR_TIMEOUT when none came.
int sparc_serve_next(sparc_server *s, int state, int64_t timeout_ms, int64_t *ticket) {
  if (!s || !ticket || (state != SPARC_REQ_ADMITTED && state != SPARC_REQ_DONE))
    return SPARC_ERR_INVALID;
  std::unique_lock<std::mutex> lock(s->mu);
  bool found = false;
  auto pick = [&]() -> bool {
    for (auto &kv : s->tickets) {
      Ticket &t = kv.second;
      const bool match = t.state == state ||
                         (state == SPARC_REQ_DONE && t.state == SPARC_REQ_FAILED);
      bool &taken = state == SPARC_REQ_ADMITTED ? t.taken_build : t.taken_collect;
      if (match && !taken) {
        taken = true;
        *ticket = t.id;
        found = true;
        return true;
      }
    }
    return false;
  };
  s->cv.wait_for(lock, std::chrono::milliseconds(std::max<int64_t>(0, timeout_ms)),
                 [&] { return pick() || s->stop; });
  return found ? SPARC_OK : SPARC_ERR_TIMEOUT;
}

int sparc_serve_params(sparc_server *s, int64_t ticket, sparc_params *p, int64_t *first,
                       int64_t *steps) {
  if (!s || !p) return SPARC_ERR_INVALID;
  std::lock_guard<std::mutex> lock(s->mu);
  auto it = s->tickets.find(ticket);
  if (it == s->tickets.end()) return SPARC_ERR_INVALID;
  *p = it->second.p;
  if (first) *first = it->second.first;
  if (steps) *steps = it->second.steps;
  return SPARC_OK;
}

int sparc_serve_attach(sparc_server *s, int64_t ticket, sparc_handle *hh) {
  if (!s || !hh) return SPARC_ERR_INVALID;
  Handle *h = reinterpret_cast<Handle *>(hh);
  std::lock_guard<std::mutex> lock(s->mu);
  auto it = s->tickets.find(ticket);
  if (it == s->tickets.end() || it->second.state != SPARC_REQ_ADMITTED)
    return SPARC_ERR_ORDER;
  const sparc_params &p = it->second.p;
  if (h->nx != p.nx || h->ny != p.ny || h->nz != p.nz || !h->fp32 || !h->bg_ready) {
    s->err = "handle does not match the admitted request";
    return SPARC_ERR_INVALID;
  }
  it->second.h = h;
  s->to_attach.push_back(ticket);
  s->cv.notify_all();
  return SPARC_OK;
}

// Gives back the handle of a DONE (or FAILED) ticket and its timestamps
// (seconds since the server started): submit, admit, start, done.
int sparc_serve_result(sparc_server *s, int64_t ticket, sparc_handle **h, double *times4,
                       int *state) {
  if (!s || !h) return SPARC_ERR_INVALID;
  std::lock_guard<std::mutex> lock(s->mu);
  auto it = s->tickets.find(ticket);
  if (it == s->tickets.end()) return SPARC_ERR_INVALID;
  Ticket &t = it->second;
  if (t.state != SPARC_REQ_DONE && t.state != SPARC_REQ_FAILED) return SPARC_ERR_ORDER;
  *h = reinterpret_cast<sparc_handle *>(t.h);
  if (times4) {
    times4[0] = t.t_submit;
    times4[1] = t.t_admit;
    times4[2] = t.t_start;
    times4[3] = t.t_done;
  }
  if (state) *state = t.state;
  if (t.state == SPARC_REQ_DONE) t.state = SPARC_REQ_COLLECTED;
  return SPARC_OK;
}

// Ends a ticket (the client destroyed or kept its handle) and returns its
// budget; an ADMITTED ticket whose set-up failed is released the same way.
int sparc_serve_release(sparc_server *s, int64_t ticket) {
  if (!s) return SPARC_ERR_INVALID;
  std::lock_guard<std::mutex> lock(s->mu);
  auto it = s->tickets.find(ticket);
  if (it == s->tickets.end()) return SPARC_ERR_INVALID;
  Ticket &t = it->second;
  if (t.state == SPARC_REQ_RUNNING || t.state == SPARC_REQ_QUEUED ||
      (t.state == SPARC_REQ_ADMITTED &&
       std::find(s->to_attach.begin(), s->to_attach.end(), ticket) != s->to_attach.end()))
    return SPARC_ERR_ORDER;
  if (t.state == SPARC_REQ_ADMITTED || t.state == SPARC_REQ_COLLECTED ||
      t.state == SPARC_REQ_DONE || t.state == SPARC_REQ_FAILED) {
    s->used -= t.reserved;
    --s->active;
  }
  s->tickets.erase(it);
  s->cv.notify_all();
  return SPARC_OK;
}

int sparc_serve_state(sparc_server *s, int64_t ticket, int *state) {
  if (!s || !state) return SPARC_ERR_INVALID;
  std::lock_guard<std::mutex> lock(s->mu);
  auto it = s->tickets.find(ticket);
  if (it == s->tickets.end()) return SPARC_ERR_INVALID;
  *state = it->second.state;
  return SPARC_OK;
}

// stats[0..11]: queued, admitted, running, done (not yet released), budget
// used (bytes), max concurrent active, batched steps run, service rounds,
// point updates, seconds the worker waited on batched steps, max members
// running at once, requests attached while others were running
int sparc_serve_stats(sparc_server *s, double *stats12) {
  if (!s || !stats12) return SPARC_ERR_INVALID;
  std::lock_guard<std::mutex> lock(s->mu);
  double q = 0, a = 0, r = 0, d = 0;
  for (auto &kv : s->tickets) {
    const int st = kv.second.state;
    q += st == SPARC_REQ_QUEUED;
    a += st == SPARC_REQ_ADMITTED;
    r += st == SPARC_REQ_RUNNING;
    d += st == SPARC_REQ_DONE || st == SPARC_REQ_COLLECTED;
  }
  const double v[12] = {q, a, r, d, (double)s->used, (double)s->max_active,
                        (double)s->steps_run, (double)s->rounds, s->point_updates,
                        s->gpu_busy_s, (double)s->max_running, (double)s->joined};
  for (int i = 0; i < 12; ++i) stats12[i] = v[i];
  return SPARC_OK;
}

const char *sparc_server_last_error(const sparc_server *s) { return s ? s->err.c_str() : ""; }

}  // extern "C"
