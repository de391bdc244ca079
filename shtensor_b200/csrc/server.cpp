// server.cpp -- serving loop: continuous batching of block-sparse contractions on one GPU,
// in the batched FP64 or the split-precision form.
//
// shtensor itself has no request loop; this is the library's own.  A server runs one loop
// thread and `planners` planner threads.  A request moves through
//   queued    submitted, waiting for a slot, for pool memory, or for an earlier request that
//             touches the same tensor (the loop decides admission);
//   planning  with a planner thread: matching, C pattern, work list and operands in matrix form
//             on that planner's own stream, ending with an event;
//   ready     planned, waiting for the next launch;
//   running   in one of at most two persistent launches queued on the exec stream.
// Every launch takes all ready requests (up to max_batch), so requests that arrived while the
// previous launch ran join the next one: batching is continuous, not by fixed windows.  The
// planner streams have the higher priority and a serving launch leaves CTA slots free on
// every SM, so planning overlaps the running launch; several planners overlap each other's
// host round trips.  Completion is signalled by a waiter thread that blocks on an event recorded
// after each launch (no host function in the exec stream, which would hold back the next launch
// until the CPU ran it).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <thread>
#include <unordered_map>

#include "contract.h"

namespace {

using Clock = std::chrono::steady_clock;

double ms_between(Clock::time_point a, Clock::time_point b) {
  return std::chrono::duration<double, std::milli>(b - a).count();
}

// SHT_SERVER_TRACE=1: one stderr line per state change (no stream syncs)
void strace(const char* fmt, long long a = 0, long long b = 0) {
  static const bool on = [] {
    const char* e = std::getenv("SHT_SERVER_TRACE");
    return e && e[0] == '1';
  }();
  if (!on) return;
  static const Clock::time_point t0 = Clock::now();
  char line[160];
  std::snprintf(line, sizeof(line), fmt, a, b);
  std::fprintf(stderr, "[sht-server %10.3f ms] %s\n", ms_between(t0, Clock::now()), line);
}

struct Request {
  int64_t id = 0;
  std::string expr;
  double alpha = 1.0, beta = 0.0, eps = 0.0;
  sht_norm norm = SHT_NORM_FROBENIUS;
  sht_tensor *A = nullptr, *B = nullptr, *C = nullptr;
  Clock::time_point t_submit, t_plan0, t_plan1, t_launch, t_done;
  double gpu_ms = 0.0;  // device time of its launch (exec stream reaching it -> done)
  std::unique_ptr<sht_plan> plan;
  cudaStream_t pstream = nullptr;  // the planner stream that planned it
  cudaEvent_t planned = nullptr;   // recorded on pstream after its planning work
  sht_status plan_status = SHT_OK;
  std::string plan_msg;
  bool finished = false;
  sht_status status = SHT_OK;
  std::string msg;
  int64_t batch = -1;
  int batch_size = 0;
  int deferrals = 0;
  bool waiting_memory = false;  // deferred; retried after the next retired launch
  int64_t deferred_at = -1;     // retired-launch count when it was deferred
  int64_t npairs = 0;
  double flops = 0.0;
  int form = SHT_MODE_BATCHED_FP64;  // the form it was planned in
  int kind = -1;                     // split form: the launch kind (slice count, reassembly)
};
using ReqPtr = std::shared_ptr<Request>;

struct Launch {
  int64_t id = 0;
  int slot = 0;
  std::vector<ReqPtr> reqs;
  sht::PoolBuf descs, counter;
  cudaEvent_t start = nullptr, done = nullptr;  // timed: the launch's device duration
};

bool touches(const Request& r, const sht_tensor* t) { return r.A == t || r.B == t || r.C == t; }

// r must wait for o: one of them writes a tensor the other reads or writes
bool conflicts(const Request& r, const Request& o) { return touches(o, r.C) || touches(r, o.C); }

void insert_by_id(std::deque<ReqPtr>& q, ReqPtr r) {
  auto it = std::upper_bound(q.begin(), q.end(), r->id, [](int64_t id, const ReqPtr& x) { return id < x->id; });
  q.insert(it, std::move(r));
}

}  // namespace

struct sht_server {
  sht_ctx* ctx = nullptr;
  std::shared_ptr<sht::DevicePool> keep;
  int max_active = 64, max_batch = 32, nplanners = 8, ctas_per_sm = 0;
  int mode = SHT_MODE_BATCHED_FP64;  // the served form
  size_t reserve_bytes = 0;
  cudaStream_t exec_stream = nullptr;
  std::vector<cudaStream_t> plan_streams;
  void* pinned[2] = {nullptr, nullptr};  // launch descriptors, one buffer per launch slot
  bool slot_busy[2] = {false, false};

  // shared with callers and planners: guarded by mu
  std::mutex mu;
  std::condition_variable wake;      // the loop: new work, a planned request, a completion, stop
  std::condition_variable finished;  // waiters: a request finished
  std::condition_variable plan_cv;   // planners: a request to plan, or stop
  std::deque<ReqPtr> incoming;
  std::deque<ReqPtr> to_plan, planned;
  std::unordered_map<int64_t, ReqPtr> table;
  int64_t next_id = 1;
  bool stop = false, stop_planners = false;
  int completions = 0;  // launch completions seen by the waiter, not yet handled
  // statistics since the last reset
  int64_t submitted = 0, completed = 0, failed = 0, batches = 0, batched_reqs = 0, deferrals = 0;
  int max_active_seen = 0;
  std::vector<double> latencies;
  double done_flops = 0.0;
  bool have_first = false;
  Clock::time_point first_submit, last_done;

  // loop-owned
  std::deque<ReqPtr> queued;
  std::vector<ReqPtr> planning;  // handed to the planners, not yet collected
  std::vector<ReqPtr> ready;
  std::deque<std::unique_ptr<Launch>> running;
  std::vector<cudaEvent_t> spare_events;
  int64_t next_launch = 0;
  int64_t retired_launches = 0;
  std::thread thread;
  std::vector<std::thread> planner_threads;
  // completion waiter: blocks on one event per launch and wakes the loop.  A host function
  // queued on the exec stream would hold back the next launch until the CPU ran it.
  std::thread waiter_thread;
  std::deque<cudaEvent_t> wait_q;   // guarded by mu; the waiter destroys each event it took
  std::condition_variable wait_cv;
  bool stop_waiter = false;
  void waiter();

  void loop();
  void planner(int index);
  bool retire();
  bool collect();
  bool admit();
  bool launch();
  void defer(Request& r);
  void finish(const ReqPtr& r, sht_status st, const std::string& msg, Clock::time_point t);
  int active() const {
    int n = (int)ready.size() + (int)planning.size();
    for (const auto& l : running) n += (int)l->reqs.size();
    return n;
  }
};

namespace {


// device bytes a request needs beyond its tensors, estimated before planning: the operands in
// matrix form (batched: about 10 bytes per element with padding) or as slices (split: S bytes
// per element of rows padded to the tile height and k to 32, about 24 at S = 7), plus pair,
// work and C-pattern arrays (C's own growth is not known until matching)
size_t estimate_bytes(const Request& r, int mode) {
  const double elems = (double)r.A->nnz + (double)r.B->nnz;
  const double blocks = (double)r.A->nblocks + (double)r.B->nblocks + (double)r.C->nblocks;
  const double per = mode == SHT_MODE_SPLIT ? 24.0 : 10.0;
  return (size_t)(elems * per + blocks * 64.0) + (size_t(1) << 20);
}

}  // namespace

void sht_server::finish(const ReqPtr& r, sht_status st, const std::string& msg, Clock::time_point t) {
  // A failed request may have left planning work queued: let it drain before its memory can
  // be reused.  Completed requests have nothing left on any stream.
  if (st != SHT_OK && r->pstream) cudaStreamSynchronize(r->pstream);
  // The plan's buffers are freed now, against the planner stream.  The tensors belong to the
  // caller and may be freed after the server is gone, so they must not keep a server stream:
  // the legacy stream orders their reuse (their work on the server's streams is complete).
  if (r->plan) sht::plan_touch(r->plan.get(), r->pstream);
  r->plan.reset();
  for (sht_tensor* x : {r->A, r->B, r->C}) sht::tensor_touch(x, nullptr);
  if (r->planned) {
    spare_events.push_back(r->planned);
    r->planned = nullptr;
  }
  strace("finish request %lld status %lld", (long long)r->id, (long long)st);
  std::lock_guard<std::mutex> lk(mu);
  r->status = st;
  r->msg = msg;
  r->t_done = t;
  r->finished = true;
  if (st == SHT_OK) {
    ++completed;
    latencies.push_back(ms_between(r->t_submit, t));
    done_flops += r->flops;
    if (t > last_done) last_done = t;
  } else {
    ++failed;
  }
  finished.notify_all();
}

// Finish the launches whose work has completed, oldest first.
bool sht_server::retire() {
  bool any = false;
  while (!running.empty()) {
    Launch& l = *running.front();
    const cudaError_t q = cudaEventQuery(l.done);
    if (q == cudaErrorNotReady) break;
    const Clock::time_point t = Clock::now();
    sht_status st = q == cudaSuccess ? SHT_OK : SHT_ERR_CUDA;
    std::string msg = q == cudaSuccess ? "" : std::string("serving launch failed: ") + cudaGetErrorString(q);
    // a split launch whose bounded wait ran out recorded it on the context's error word
    if (st == SHT_OK) {
      if (const int e = sht::ctx_take_error(ctx)) {
        st = (sht_status)e;
        msg = "serving launch failed: a bounded wait on the tensor cores expired";
      }
    }
    if (q != cudaSuccess) (void)cudaGetLastError();
    float gms = 0.0f;
    if (q == cudaSuccess && cudaEventElapsedTime(&gms, l.start, l.done) != cudaSuccess) (void)cudaGetLastError();
    strace("retire launch %lld (%lld requests)", (long long)l.id, (long long)l.reqs.size());
    strace("  device time of launch %lld: %lld us", (long long)l.id, (long long)(gms * 1000.0f));
    for (const ReqPtr& r : l.reqs) {
      r->gpu_ms = gms;
      finish(r, st, msg, t);
    }
    // the launch's work is complete: its buffers may be reused as soon as a planner gets to them
    l.descs.use_on(plan_streams[0]);
    l.counter.use_on(plan_streams[0]);
    slot_busy[l.slot] = false;
    cudaEventDestroy(l.start);
    cudaEventDestroy(l.done);
    running.pop_front();
    ++retired_launches;
    any = true;
  }
  return any;
}

void sht_server::defer(Request& r) {
  r.deferred_at = retired_launches;
  if (r.waiting_memory) return;
  r.waiting_memory = true;
  ++r.deferrals;
  std::lock_guard<std::mutex> lk(mu);
  ++deferrals;
}

// Take the planners' results: planned requests become ready; a plan that ran out of pool
// memory while other requests hold memory goes back to the queue; other failures finish.
bool sht_server::collect() {
  std::deque<ReqPtr> got;
  {
    std::lock_guard<std::mutex> lk(mu);
    got.swap(planned);
  }
  for (ReqPtr& r : got) {
    planning.erase(std::find(planning.begin(), planning.end(), r));
    if (r->plan_status == SHT_OK) {
      r->waiting_memory = false;
      ready.push_back(std::move(r));
    } else if (r->plan_status == SHT_ERR_OOM && active() > 0) {
      strace("defer request %lld (out of pool memory)", (long long)r->id);
      defer(*r);
      insert_by_id(queued, std::move(r));
    } else {
      finish(r, r->plan_status, r->plan_msg, Clock::now());
    }
  }
  return !got.empty();
}

// Hand queued requests to the planners while slots and pool memory allow, in submission
// order except that a request blocked by a conflict does not hold back unrelated ones.
bool sht_server::admit() {
  {
    std::lock_guard<std::mutex> lk(mu);
    while (!incoming.empty()) {
      queued.push_back(std::move(incoming.front()));
      incoming.pop_front();
    }
  }
  bool any = false;
  std::vector<const Request*> busy;  // admitted and not finished, then passed-over queued ones
  for (const ReqPtr& o : planning) busy.push_back(o.get());
  for (const ReqPtr& o : ready) busy.push_back(o.get());
  for (const auto& l : running)
    for (const ReqPtr& o : l->reqs) busy.push_back(o.get());
  for (auto it = queued.begin(); it != queued.end();) {
    if (active() >= max_active) break;
    Request& r = **it;
    bool blocked = false;
    for (const Request* o : busy) blocked = blocked || conflicts(r, *o);
    if (blocked) {
      busy.push_back(&r);
      ++it;
      continue;
    }
    const bool others = active() > 0;
    // a deferred request waits for a retired launch to return memory; later requests keep
    // their order behind it
    if (others && r.waiting_memory && r.deferred_at == retired_launches) break;
    // requests with the planners may not have taken their memory yet: count their estimates
    size_t planning_bytes = 0;
    for (const ReqPtr& o : planning) planning_bytes += estimate_bytes(*o, mode);
    const size_t free_now = ctx->pool->free_bytes();
    const size_t avail = free_now > planning_bytes ? free_now - planning_bytes : 0;
    if (others && avail < reserve_bytes + estimate_bytes(r, mode)) {
      strace("defer request %lld (estimate)", (long long)r.id);
      defer(r);
      break;
    }
    try {
      // host index of the tensors current before several planners read them
      for (sht_tensor* t : {r.A, r.B, r.C}) sht::tensor_sync_host(t, plan_streams[0]);
      if (!r.planned) {
        if (!spare_events.empty()) {
          r.planned = spare_events.back();
          spare_events.pop_back();
        } else {
          SHT_CUDA(cudaEventCreateWithFlags(&r.planned, cudaEventDisableTiming));
        }
      }
    } catch (const sht::Error& e) {
      ReqPtr keep = *it;
      it = queued.erase(it);
      finish(keep, e.code, e.msg, Clock::now());
      any = true;
      continue;
    }
    r.plan_status = SHT_OK;
    r.plan_msg.clear();
    ReqPtr rp = *it;
    it = queued.erase(it);
    busy.push_back(rp.get());
    planning.push_back(rp);
    {
      std::lock_guard<std::mutex> lk(mu);
      to_plan.push_back(rp);
      max_active_seen = std::max(max_active_seen, active());
    }
    plan_cv.notify_one();
    strace("admit request %lld", (long long)rp->id);
    any = true;
  }
  return any;
}

void sht_server::planner(int index) {
  cudaSetDevice(ctx->device);
  cudaStream_t s = plan_streams[index];
  for (;;) {
    ReqPtr r;
    {
      std::unique_lock<std::mutex> lk(mu);
      plan_cv.wait(lk, [&] { return stop_planners || !to_plan.empty(); });
      if (to_plan.empty()) return;  // stop_planners
      r = std::move(to_plan.front());
      to_plan.pop_front();
    }
    r->pstream = s;
    r->t_plan0 = Clock::now();
    try {
      bool split = false;
      if (mode == SHT_MODE_SPLIT) {
        // split form: pairs, C pattern, slices and records; the slicer's flags are read here (the
        // planner synchronizes anyway), and a request they rule out is planned again in the
        // batched FP64 form
        r->plan.reset(sht::plan_create(ctx, r->expr, r->A, r->B, r->C, r->eps, r->norm, SHT_MODE_SPLIT, s));
        sht::split_prepare(r->plan.get(), ctx->split_slices ? ctx->split_slices : sht::split_slices_default(), s);
        sht::split_slice(r->plan.get(), r->alpha, s);
        split = sht::split_flags_clear(r->plan.get(), s);
        if (!split) r->plan.reset();
      }
      if (split) {
        r->form = SHT_MODE_SPLIT;
        r->kind = sht::split_kind(r->plan.get());
      } else {
        r->form = SHT_MODE_BATCHED_FP64;
        r->kind = -1;
        r->plan.reset(sht::plan_create(ctx, r->expr, r->A, r->B, r->C, r->eps, r->norm, SHT_MODE_BATCHED_FP64, s));
        sht::batched_prepare(r->plan.get(), s);
        const sht::SparseArgs g = sht::sparse_args(r->plan.get(), r->alpha, r->beta);
        if (!g.sc.alpha_zero) sht::matform_execute(r->plan.get(), r->alpha, s);
      }
      SHT_CUDA(cudaEventRecord(r->planned, s));
      r->npairs = r->plan->npairs;
      r->flops = sht::plan_flops(r->plan.get(), s);
    } catch (const sht::Error& e) {
      r->plan.reset();
      cudaStreamSynchronize(s);
      r->plan_status = e.code;
      r->plan_msg = e.msg;
    } catch (const std::exception& e) {
      r->plan.reset();
      cudaStreamSynchronize(s);
      r->plan_status = SHT_ERR_INVALID;
      r->plan_msg = e.what();
    }
    r->t_plan1 = Clock::now();
    strace("planned request %lld status %lld", (long long)r->id, (long long)r->plan_status);
    {
      std::lock_guard<std::mutex> lk(mu);
      planned.push_back(std::move(r));
    }
    wake.notify_one();
  }
}

// Put the ready requests of the oldest ready request's kind (batched FP64, or one split kind),
// up to max_batch, into one persistent launch on the exec stream.
bool sht_server::launch() {
  if (ready.empty() || running.size() >= 2) return false;
  const int slot = slot_busy[0] ? 1 : 0;
  auto l = std::make_unique<Launch>();
  l->id = next_launch++;
  l->slot = slot;
  const int kind = (*std::min_element(ready.begin(), ready.end(),
                                      [](const ReqPtr& a, const ReqPtr& b) { return a->id < b->id; }))->kind;
  for (auto it = ready.begin(); it != ready.end() && l->reqs.size() < (size_t)max_batch;) {
    if ((*it)->kind == kind) {
      l->reqs.push_back(*it);
      it = ready.erase(it);
    } else {
      ++it;
    }
  }
  const size_t n = l->reqs.size();
  const Clock::time_point t = Clock::now();
  try {
    SHT_CUDA(cudaEventCreate(&l->start));
    SHT_CUDA(cudaEventRecord(l->start, exec_stream));
    std::vector<sht_plan*> plans;
    std::vector<sht::SparseArgs> args;
    for (const ReqPtr& r : l->reqs) {
      SHT_CUDA(cudaStreamWaitEvent(exec_stream, r->planned, 0));
      sht::plan_touch(r->plan.get(), exec_stream);
      plans.push_back(r->plan.get());
      args.push_back(sht::sparse_args(r->plan.get(), r->alpha, r->beta));
      r->t_launch = t;
      r->batch = l->id;
      r->batch_size = (int)n;
    }
    if (kind >= 0) {
      sht::split_multi_launch(ctx, plans, args, pinned[slot], l->descs, exec_stream);
    } else {
      const int per_sm = ctas_per_sm > 0 ? ctas_per_sm : std::max(1, sht::batched_ctas_per_sm(ctx) - 1);
      sht::batched_multi_launch(ctx, plans, args, pinned[slot], l->descs, l->counter, per_sm, exec_stream);
    }
    l->descs.use_on(exec_stream);
    l->counter.use_on(exec_stream);
    SHT_CUDA(cudaEventCreate(&l->done));
    SHT_CUDA(cudaEventRecord(l->done, exec_stream));
    // the waiter's own event (blocking sync: the waiter sleeps in the driver, it does not spin)
    cudaEvent_t w = nullptr;
    SHT_CUDA(cudaEventCreateWithFlags(&w, cudaEventBlockingSync | cudaEventDisableTiming));
    SHT_CUDA(cudaEventRecord(w, exec_stream));
    {
      std::lock_guard<std::mutex> lk(mu);
      wait_q.push_back(w);
    }
    wait_cv.notify_one();
    strace("launch %lld with %lld requests", (long long)l->id, (long long)n);
  } catch (const sht::Error& e) {
    // nothing of this launch is known to run: wait for the stream, then fail its requests
    cudaStreamSynchronize(exec_stream);
    (void)cudaGetLastError();
    if (l->start) cudaEventDestroy(l->start);
    if (l->done) cudaEventDestroy(l->done);
    for (const ReqPtr& r : l->reqs) finish(r, e.code, e.msg, Clock::now());
    return true;
  }
  slot_busy[slot] = true;
  {
    std::lock_guard<std::mutex> lk(mu);
    ++batches;
    batched_reqs += (int64_t)n;
  }
  running.push_back(std::move(l));
  return true;
}

void sht_server::waiter() {
  cudaSetDevice(ctx->device);
  for (;;) {
    cudaEvent_t ev = nullptr;
    {
      std::unique_lock<std::mutex> lk(mu);
      wait_cv.wait(lk, [&] { return stop_waiter || !wait_q.empty(); });
      if (wait_q.empty()) return;  // stop_waiter, nothing left to wait for
      ev = wait_q.front();
      wait_q.pop_front();
    }
    cudaEventSynchronize(ev);  // an error surfaces on the launch's own event in retire()
    cudaEventDestroy(ev);
    {
      std::lock_guard<std::mutex> lk(mu);
      ++completions;
    }
    wake.notify_one();
  }
}

void sht_server::loop() {
  cudaSetDevice(ctx->device);
  for (;;) {
    bool progressed = retire();
    progressed = collect() || progressed;
    progressed = admit() || progressed;
    progressed = launch() || progressed;
    std::unique_lock<std::mutex> lk(mu);
    if (stop && incoming.empty() && queued.empty() && planning.empty() && ready.empty() && running.empty()) break;
    if (progressed) continue;
    if (completions > 0) {
      completions = 0;
      continue;
    }
    // idle: sleep until a submit, a planned request, a completion or stop; the
    // timeout bounds the wait for a launch whose callback cannot arrive (a failed stream)
    if (incoming.empty() && planned.empty())
      wake.wait_for(lk, std::chrono::milliseconds(running.empty() ? 50 : 2),
                    [&] { return stop || !incoming.empty() || !planned.empty() || completions > 0; });
    completions = 0;
  }
}

using namespace sht;

extern "C" {

sht_status sht_server_create(sht_ctx* ctx, const sht_server_config* cfg, sht_server** out) {
  return guard([&] {
    if (!ctx || !out) fail(SHT_ERR_INVALID, "null argument");
    auto s = std::make_unique<sht_server>();
    s->ctx = ctx;
    s->keep = ctx->pool;
    if (cfg) {
      if (cfg->max_active < 0 || cfg->max_batch < 0 || cfg->planners < 0 || cfg->ctas_per_sm < 0)
        fail(SHT_ERR_INVALID, "negative server setting");
      if (cfg->max_active) s->max_active = cfg->max_active;
      if (cfg->max_batch) s->max_batch = cfg->max_batch;
      if (cfg->planners) s->nplanners = std::min(cfg->planners, 64);
      s->ctas_per_sm = cfg->ctas_per_sm;
      s->reserve_bytes = cfg->reserve_bytes;
      if (cfg->mode != 0 && cfg->mode != SHT_MODE_BATCHED_FP64 && cfg->mode != SHT_MODE_SPLIT)
        fail(SHT_ERR_INVALID, "a server serves the batched FP64 or the split-precision form");
      s->mode = cfg->mode == SHT_MODE_SPLIT ? SHT_MODE_SPLIT : SHT_MODE_BATCHED_FP64;
    }
    SHT_CUDA(cudaSetDevice(ctx->device));
    int lo = 0, hi = 0;
    SHT_CUDA(cudaDeviceGetStreamPriorityRange(&lo, &hi));  // hi is the numerically smaller
    // the streams exist before any thread starts, so a failure here leaves nothing running
    auto cleanup = [&] {
      for (cudaStream_t st : s->plan_streams) cudaStreamDestroy(st);
      if (s->exec_stream) cudaStreamDestroy(s->exec_stream);
      for (void* p : s->pinned)
        if (p) cudaFreeHost(p);
    };
    try {
      for (int i = 0; i < s->nplanners; ++i) {
        cudaStream_t st = nullptr;
        SHT_CUDA(cudaStreamCreateWithPriority(&st, cudaStreamNonBlocking, hi));
        s->plan_streams.push_back(st);
      }
      SHT_CUDA(cudaStreamCreateWithPriority(&s->exec_stream, cudaStreamNonBlocking, lo));
      for (void*& p : s->pinned)
        SHT_CUDA(cudaMallocHost(&p, (size_t)s->max_batch * std::max(batched_desc_bytes(), split_desc_bytes())));
    } catch (...) {
      cleanup();
      throw;
    }
    sht_server* raw = s.get();
    for (int i = 0; i < s->nplanners; ++i) s->planner_threads.emplace_back([raw, i] { raw->planner(i); });
    s->waiter_thread = std::thread([raw] { raw->waiter(); });
    s->thread = std::thread([raw] { raw->loop(); });
    *out = s.release();
  });
}

sht_status sht_server_submit(sht_server* srv, const char* expr, double alpha, sht_tensor* A, sht_tensor* B,
                             double beta, sht_tensor* C, double eps, sht_norm norm, int64_t* request_id) {
  return guard([&] {
    if (!srv || !expr || !A || !B || !C || !request_id) fail(SHT_ERR_INVALID, "null argument");
    if (norm < SHT_NORM_FROBENIUS || norm > SHT_NORM_FROBENIUS_REFCOMPAT) fail(SHT_ERR_INVALID, "unknown norm");
    for (sht_tensor* t : {A, B, C})
      if (t->ctx != srv->ctx) fail(SHT_ERR_INVALID, "tensor from another context");
    auto r = std::make_shared<Request>();
    r->expr = expr;
    r->alpha = alpha;
    r->beta = beta;
    r->eps = eps;
    r->norm = norm;
    r->A = A;
    r->B = B;
    r->C = C;
    r->t_submit = Clock::now();
    {
      std::lock_guard<std::mutex> lk(srv->mu);
      if (srv->stop) fail(SHT_ERR_STATE, "server is stopping");
      r->id = srv->next_id++;
      srv->table[r->id] = r;
      srv->incoming.push_back(r);
      ++srv->submitted;
      if (!srv->have_first) {
        srv->have_first = true;
        srv->first_submit = r->t_submit;
      }
    }
    srv->wake.notify_one();
    *request_id = r->id;
  });
}

sht_status sht_server_poll(sht_server* srv, int64_t request_id, int* state) {
  return guard([&] {
    if (!srv || !state) fail(SHT_ERR_INVALID, "null argument");
    std::lock_guard<std::mutex> lk(srv->mu);
    auto it = srv->table.find(request_id);
    if (it == srv->table.end()) fail(SHT_ERR_INVALID, "unknown request id");
    *state = it->second->finished ? 1 : 0;
  });
}

sht_status sht_server_wait(sht_server* srv, int64_t request_id, double timeout_s, sht_request_report* rep) {
  ReqPtr r;
  const sht_status st = guard([&] {
    if (!srv) fail(SHT_ERR_INVALID, "null server");
    std::unique_lock<std::mutex> lk(srv->mu);
    auto it = srv->table.find(request_id);
    if (it == srv->table.end()) fail(SHT_ERR_INVALID, "unknown request id");
    r = it->second;
    auto done = [&] { return r->finished; };
    if (timeout_s < 0) {
      srv->finished.wait(lk, done);
    } else if (!srv->finished.wait_for(lk, std::chrono::duration<double>(timeout_s), done)) {
      fail(SHT_ERR_TIMEOUT, "request " + std::to_string(request_id) + " still pending");
    }
    srv->table.erase(it);
  });
  if (st != SHT_OK) return st;
  if (rep) {
    std::memset(rep, 0, sizeof(*rep));
    rep->status = r->status;
    rep->npairs = r->npairs;
    rep->flops = r->flops;
    const bool planned = r->t_plan0 != Clock::time_point{};
    rep->queue_ms = ms_between(r->t_submit, planned ? r->t_plan0 : r->t_done);
    rep->plan_ms = r->t_plan1 != Clock::time_point{} ? ms_between(r->t_plan0, r->t_plan1) : 0.0;
    rep->run_ms = r->batch >= 0 ? ms_between(r->t_launch, r->t_done) : 0.0;
    rep->gpu_ms = r->gpu_ms;
    rep->latency_ms = ms_between(r->t_submit, r->t_done);
    rep->batch = r->batch;
    rep->form = r->form;
    rep->batch_size = r->batch_size;
    rep->deferrals = r->deferrals;
  }
  if (r->status != SHT_OK) set_last_error(r->msg);
  return r->status;
}

static double percentile(std::vector<double> v, double q) {
  if (v.empty()) return 0.0;
  std::sort(v.begin(), v.end());
  // nearest rank
  size_t k = (size_t)std::ceil(q * (double)v.size());
  k = std::min(std::max<size_t>(k, 1), v.size());
  return v[k - 1];
}

sht_status sht_server_get_stats(sht_server* srv, sht_server_stats* out) {
  return guard([&] {
    if (!srv || !out) fail(SHT_ERR_INVALID, "null argument");
    std::lock_guard<std::mutex> lk(srv->mu);
    std::memset(out, 0, sizeof(*out));
    out->submitted = srv->submitted;
    out->completed = srv->completed;
    out->failed = srv->failed;
    out->batches = srv->batches;
    out->deferrals = srv->deferrals;
    out->max_active_seen = srv->max_active_seen;
    out->mean_batch = srv->batches ? (double)srv->batched_reqs / (double)srv->batches : 0.0;
    out->p50_ms = percentile(srv->latencies, 0.50);
    out->p99_ms = percentile(srv->latencies, 0.99);
    out->max_ms = srv->latencies.empty() ? 0.0 : *std::max_element(srv->latencies.begin(), srv->latencies.end());
    out->flops = srv->done_flops;
    out->span_s = (srv->have_first && srv->completed) ? ms_between(srv->first_submit, srv->last_done) / 1e3 : 0.0;
    out->gflops = out->span_s > 0 ? out->flops / out->span_s / 1e9 : 0.0;
  });
}

sht_status sht_server_reset_stats(sht_server* srv) {
  return guard([&] {
    if (!srv) fail(SHT_ERR_INVALID, "null server");
    std::lock_guard<std::mutex> lk(srv->mu);
    srv->submitted = srv->completed = srv->failed = srv->batches = srv->batched_reqs = srv->deferrals = 0;
    srv->max_active_seen = 0;
    srv->latencies.clear();
    srv->done_flops = 0.0;
    srv->have_first = false;
    srv->last_done = Clock::time_point{};
  });
}

sht_status sht_server_destroy(sht_server* srv) {
  return guard([&] {
    if (!srv) return;
    {
      std::lock_guard<std::mutex> lk(srv->mu);
      srv->stop = true;
    }
    srv->wake.notify_one();
    if (srv->thread.joinable()) srv->thread.join();  // returns once every request finished
    {
      std::lock_guard<std::mutex> lk(srv->mu);
      srv->stop_planners = true;
    }
    srv->plan_cv.notify_all();
    for (std::thread& t : srv->planner_threads) t.join();
    {
      std::lock_guard<std::mutex> lk(srv->mu);
      srv->stop_waiter = true;
    }
    srv->wait_cv.notify_all();
    if (srv->waiter_thread.joinable()) srv->waiter_thread.join();  // after its queue is empty
    cudaSetDevice(srv->ctx->device);
    cudaStreamSynchronize(srv->exec_stream);
    for (cudaStream_t st : srv->plan_streams) {
      cudaStreamSynchronize(st);
      cudaStreamDestroy(st);
    }
    for (void* p : srv->pinned)
      if (p) cudaFreeHost(p);
    for (cudaEvent_t e : srv->spare_events) cudaEventDestroy(e);
    if (srv->exec_stream) cudaStreamDestroy(srv->exec_stream);
    delete srv;
  });
}

}  // extern "C"
