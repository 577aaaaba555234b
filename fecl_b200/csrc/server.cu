// A decode server with continuous batching.
//
// Requests (n frames of one codec, host L-values in, host decisions out) enter a
// queue from any thread.  A scheduler thread keeps up to `slots` batches in flight,
// each on its own CUDA stream with its own device arena (device_budget / slots
// bytes) and pinned staging buffers.  Whenever a slot is free it admits the oldest
// waiting requests that fit its arena and its frame limit -- requests that arrived
// while the other slots' batches were on the GPU join the next batch as soon as a
// slot and its memory free up -- and launches them: every LTE turbo frame of the
// batch in one persistent mixed-K launch on the slot's stream, the other frames one
// launch sequence per codec spread over the slot's side streams, so codecs of one batch
// and batches of different slots overlap on the device.  The same thread
// harvests finished slots, copies each request's decisions out and stamps its
// completion time.  Results do not depend on what a request was
// batched with: every kernel decodes each frame independently of the others.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <set>
#include <thread>
#include <unordered_map>
#include <vector>

#include "codec.hpp"

namespace {

template <class F>
int guarded(F&& f) {
  try {
    f();
    return FECL_OK;
  } catch (const Error& e) {
    fecl::set_last_error(e.msg);
    return e.code;
  } catch (const std::invalid_argument& e) {
    fecl::set_last_error(e.what());
    return FECL_EINVAL;
  } catch (const std::bad_alloc&) {
    fecl::set_last_error("host allocation failed");
    return FECL_ENOMEM;
  } catch (const std::exception& e) {
    fecl::set_last_error(e.what());
    return FECL_EINVAL;
  }
}

using Clock = std::chrono::steady_clock;

// Pinned staging memory of a slot.  It grows at least twofold when a batch needs more,
// and the buffers it outgrows are released only with the server: cudaFreeHost waits
// for the whole device, so freeing one while other slots' batches run would stall
// them (on a ramping load, batch after batch).  The retired buffers add up to less
// than the current one.
struct PinnedBuffer {
  void* ptr = nullptr;
  size_t bytes = 0;
  std::vector<void*> retired;
  ~PinnedBuffer() {
    if (ptr) cudaFreeHost(ptr);
    for (void* q : retired) cudaFreeHost(q);
  }
  void reserve(size_t n) {
    if (n <= bytes) return;
    n = std::max(n, 2 * bytes);
    void* q = nullptr;
    cuda_check(cudaHostAlloc(&q, n, cudaHostAllocDefault), "cudaHostAlloc");
    if (ptr) retired.push_back(ptr);
    ptr = q;
    bytes = n;
  }
  char* as() const { return static_cast<char*>(ptr); }
};

struct Request {
  uint64_t ticket = 0;
  fecl_codec_s* c = nullptr;
  const void* llr = nullptr;
  int32_t dtype = FECL_F32;
  uint64_t n = 0;
  uint8_t* msg = nullptr;
  int32_t* iters = nullptr;
  bool lte = false;
  size_t in_bytes = 0;
  Clock::time_point t_submit, t_done;
  int status = FECL_OK;
  bool done = false;
  // placement in the slot
  size_t llr_off = 0, msg_off = 0, it_off = 0;
};

constexpr int kSideStreams = 8;  // per slot: codec groups of a batch run on these at once
// Pinned staging reserved per slot at creation: the L-values (and turbo descriptors)
// of a few hundred frames, and their decisions.
constexpr size_t kInitialStagingIn = size_t(64) << 20;
constexpr size_t kInitialStagingOut = size_t(16) << 20;

struct Slot {
  cudaStream_t stream = nullptr;
  cudaStream_t side[kSideStreams] = {};
  cudaEvent_t fork = nullptr, joined[kSideStreams] = {};
  cudaEvent_t done = nullptr;
  cudaEvent_t start = nullptr;  // timing: the batch's first operation
  DeviceBuffer arena;
  PinnedBuffer in, out;
  size_t out_begin = 0;  // arena offset of out's first byte
  std::vector<std::shared_ptr<Request>> reqs;
  bool busy = false;
};

}  // namespace

struct fecl_server_s {
  fecl_server_options opt{};
  int device = 0;
  std::vector<std::unique_ptr<Slot>> slots;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<std::shared_ptr<Request>> queue;
  std::unordered_map<uint64_t, std::shared_ptr<Request>> live;
  uint64_t next_ticket = 1;
  bool stopping = false;
  std::thread worker;
  // statistics since creation or the last reset
  std::vector<double> latencies;
  uint64_t frames_done = 0, bits_done = 0, batches = 0;
  double gpu_s_sum = 0.0, host_s_sum = 0.0;
  Clock::time_point first_submit{}, last_done{};
  bool any_submit = false;
  std::string error;

  size_t arena_bytes() const { return size_t(opt.device_budget_bytes / opt.slots); }

  void run();
  bool launch(Slot& s, std::vector<std::shared_ptr<Request>>& batch);
  void harvest(Slot& s);
};

namespace {

size_t al256(size_t x) { return (x + 255) & ~size_t(255); }

// Requests of one codec and L-value type: their frames are laid out back to back, so
// the group is decoded by one launch sequence.
struct Group {
  fecl_codec_s* c = nullptr;
  int32_t dtype = FECL_F32;
  bool lte = false;
  uint64_t n = 0;
  std::vector<Request*> reqs;
  size_t llr_off = 0, msg_off = 0, it_off = 0, scratch_off = 0;
  ScratchPlan sp;
};

// The FP16 LDPC groups of a batch keep a launch sequence per codec: shared check and
// bit launches over every code (ldpc_shared.hpp, an option of mixed batches) measured
// on Poisson loads of 5k frames/s tripled the device time of a batch (27 ms against
// 8.7 ms per ~70 frames), each shared launch being sized for the largest group it
// serves.

// Admission accounting of a forming batch: an upper bound of the arena bytes, kept
// up to date request by request.
struct Admission {
  std::map<std::pair<fecl_codec_s*, int32_t>, uint64_t> frames;
  std::map<std::pair<fecl_codec_s*, int32_t>, size_t> scratch;
  size_t io = 0, scratch_sum = 0, lte_scratch = 0;
  uint64_t lte_frames = 0;
  size_t bytes_with(const Request& r) {
    const auto key = std::make_pair(r.c, r.dtype);
    size_t sc = scratch_sum;
    if (!r.lte) {
      const size_t old = scratch.count(key) ? scratch[key] : 0;
      sc = sc - old + al256(plan_scratch(r.c, frames[key] + r.n, false).bytes);
    }
    const size_t lte = lte_scratch + (r.lte ? r.n * al256(fecl::turbo_lte_frame_floats(int(r.c->msg())) * sizeof(float)) : 0);
    const uint64_t lf = lte_frames + (r.lte ? r.n : 0);
    // per group three I/O regions (rounded), descriptors and counters for up to three algorithms
    return io + 3 * 256 * (frames.size() + 1) + al256(r.in_bytes) + al256(r.n * r.c->msg()) + al256(r.n * 4) + sc + lte +
           al256(lf * sizeof(fecl::TurboLteBatchFrame)) * 2 + 3 * 256;
  }
  void add(const Request& r) {
    const auto key = std::make_pair(r.c, r.dtype);
    io += al256(r.in_bytes) + al256(r.n * r.c->msg()) + al256(r.n * 4);
    frames[key] += r.n;
    if (r.lte) {
      lte_scratch += r.n * al256(fecl::turbo_lte_frame_floats(int(r.c->msg())) * sizeof(float));
      lte_frames += r.n;
    } else {
      const size_t old = scratch.count(key) ? scratch[key] : 0;
      scratch[key] = al256(plan_scratch(r.c, frames[key], false).bytes);
      scratch_sum = scratch_sum - old + scratch[key];
    }
  }
};

}  // namespace

bool fecl_server_s::launch(Slot& s, std::vector<std::shared_ptr<Request>>& batch) {
  // ---- layout: per group the L-values, then every group's decisions and iteration
  // counts (one copy back), then scratch, turbo frame scratch and descriptors
  std::map<std::pair<fecl_codec_s*, int32_t>, Group> groups;
  for (auto& r : batch) {
    Group& g = groups[std::make_pair(r->c, r->dtype)];
    g.c = r->c;
    g.dtype = r->dtype;
    g.lte = r->lte;
    g.n += r->n;
    g.reqs.push_back(r.get());
  }
  Carver cv;
  for (auto& kv : groups) {
    Group& g = kv.second;
    g.llr_off = cv.take(g.n * g.c->parity() * dsize(g.dtype));
    size_t o = g.llr_off;
    for (Request* r : g.reqs) {
      r->llr_off = o;
      o += r->in_bytes;
    }
  }
  const size_t in_end = cv.off;
  const size_t out_begin = cv.off;
  for (auto& kv : groups) {
    Group& g = kv.second;
    g.msg_off = cv.take(g.n * g.c->msg());
    size_t o = g.msg_off;
    for (Request* r : g.reqs) {
      r->msg_off = o;
      o += r->n * g.c->msg();
    }
  }
  for (auto& kv : groups) {
    Group& g = kv.second;
    g.it_off = cv.take(g.n * 4);
    size_t o = g.it_off;
    for (Request* r : g.reqs) {
      r->it_off = o;
      o += r->n * 4;
    }
  }
  const size_t out_end = cv.off;
  // every non-LTE group gets its codec's decoder and scratch
  for (auto& kv : groups) {
    Group& g = kv.second;
    if (g.lte) continue;
    g.sp = plan_scratch(g.c, g.n, false);
    g.scratch_off = cv.take(g.sp.bytes);
  }
  char* base = s.arena.as<char>();
  std::map<int, std::vector<fecl::TurboLteBatchFrame>> tdesc;
  for (auto& kv : groups) {
    Group& g = kv.second;
    if (!g.lte) continue;
    const int K = int(g.c->msg());
    for (uint64_t f = 0; f < g.n; ++f) {
      fecl::TurboLteBatchFrame d;
      d.llr = base + g.llr_off + f * g.c->parity() * dsize(g.dtype);
      d.hard = reinterpret_cast<uint8_t*>(base + g.msg_off) + f * K;
      d.iters = reinterpret_cast<int32_t*>(base + g.it_off) + f;
      d.scratch = reinterpret_cast<float*>(base + cv.take(fecl::turbo_lte_frame_floats(K) * sizeof(float)));
      d.perm = g.c->tdev.c[1].perm;
      d.sf = g.c->tdev.sf;
      d.crc = g.c->crc_table();
      d.K = K;
      d.iterations = g.c->tdev.iterations;
      d.llr_dtype = g.dtype;
      tdesc[g.c->tdev.algorithm].push_back(d);
    }
  }
  std::map<int, std::pair<size_t, size_t>> tdev_off;  // algorithm -> descriptors, counter
  for (auto& kv : tdesc) {
    const size_t d = cv.take(kv.second.size() * sizeof(fecl::TurboLteBatchFrame));
    tdev_off[kv.first] = {d, cv.take(sizeof(int32_t))};
  }
  if (cv.off > s.arena.bytes) fail(FECL_ENOMEM, "batch exceeds the slot's arena");

  // ---- host staging and copies in
  size_t host_desc = al256(in_end);
  size_t host_end = host_desc;
  for (auto& kv : tdesc) host_end += al256(kv.second.size() * sizeof(fecl::TurboLteBatchFrame));
  s.in.reserve(std::max<size_t>(host_end, 256));
  s.out.reserve(std::max<size_t>(out_end - out_begin, 256));  // holds [out_begin, out_end)
  s.out_begin = out_begin;
  for (auto& r : batch) std::memcpy(s.in.as() + r->llr_off, r->llr, r->in_bytes);
  cuda_check(cudaEventRecord(s.start, s.stream), "cudaEventRecord");
  cuda_check(cudaMemcpyAsync(base, s.in.as(), in_end, cudaMemcpyHostToDevice, s.stream), "copy in");
  for (auto& kv : tdesc) {
    auto& v = kv.second;
    std::stable_sort(v.begin(), v.end(), [](const fecl::TurboLteBatchFrame& a, const fecl::TurboLteBatchFrame& b) {
      return a.K > b.K;
    });
    std::memcpy(s.in.as() + host_desc, v.data(), v.size() * sizeof(v[0]));
    cuda_check(cudaMemcpyAsync(base + tdev_off[kv.first].first, s.in.as() + host_desc, v.size() * sizeof(v[0]),
                               cudaMemcpyHostToDevice, s.stream),
               "copy descriptors");
    host_desc += al256(v.size() * sizeof(v[0]));
  }

  // ---- launches: every turbo frame in one mixed-K launch per algorithm on the slot's
  // stream, one launch sequence per other group on the side streams, forked after the
  // copies in (before the turbo launch, which the LDPC decoders need not wait for) and
  // joined before the copy out, so that the turbo frames and groups of different codes
  // run at once
  cuda_check(cudaEventRecord(s.fork, s.stream), "cudaEventRecord");
  for (auto& kv : tdesc) {
    fecl::TurboLteBatchParams p;
    p.frames = reinterpret_cast<const fecl::TurboLteBatchFrame*>(base + tdev_off[kv.first].first);
    p.nframes = int64_t(kv.second.size());
    p.counter = reinterpret_cast<int32_t*>(base + tdev_off[kv.first].second);
    p.max_K = kv.second.front().K;
    p.algorithm = kv.first;
    cuda_check(fecl::launch_turbo_lte_batch(p, s.stream), "turbo batch launch");
  }
  bool used[kSideStreams] = {};
  // longest first, each to the side stream with the least work so far; a group's work
  // is estimated by its parity bits times its iteration limit times its frames
  std::vector<Group*> order;
  for (auto& kv : groups)
    if (!kv.second.lte) order.push_back(&kv.second);
  auto cost = [](const Group* g) {
    const double it = g->c->kind == 0 ? double(std::max(1, g->c->ldev.iterations)) : 1.0;
    return double(g->c->parity()) * it * double(g->n);
  };
  std::stable_sort(order.begin(), order.end(), [&](const Group* a, const Group* b) { return cost(a) > cost(b); });
  double load[kSideStreams] = {};
  for (Group* gp : order) {
    Group& g = *gp;
    int q = 0;
    for (int i = 1; i < kSideStreams; ++i)
      if (load[i] < load[q]) q = i;
    load[q] += cost(gp);
    if (!used[q]) cuda_check(cudaStreamWaitEvent(s.side[q], s.fork, 0), "cudaStreamWaitEvent");
    used[q] = true;
    Launch d;
    d.llr = base + g.llr_off;
    d.hard = reinterpret_cast<uint8_t*>(base + g.msg_off);
    d.iters = reinterpret_cast<int32_t*>(base + g.it_off);
    d.scratch = base + g.scratch_off;
    launch_decode(g.c, d, g.sp, g.n, g.dtype, FECL_F32, false, false, s.side[q]);
  }
  for (int q = 0; q < kSideStreams; ++q) {
    if (!used[q]) continue;
    cuda_check(cudaEventRecord(s.joined[q], s.side[q]), "cudaEventRecord");
    cuda_check(cudaStreamWaitEvent(s.stream, s.joined[q], 0), "cudaStreamWaitEvent");
  }
  cuda_check(cudaMemcpyAsync(s.out.as(), base + out_begin, out_end - out_begin, cudaMemcpyDeviceToHost,
                             s.stream),
             "copy out");
  cuda_check(cudaEventRecord(s.done, s.stream), "cudaEventRecord");
  s.reqs = batch;
  s.busy = true;
  return true;
}

void fecl_server_s::harvest(Slot& s) {
  for (auto& r : s.reqs) {
    std::memcpy(r->msg, s.out.as() + (r->msg_off - s.out_begin), r->n * r->c->msg());
    if (r->iters) std::memcpy(r->iters, s.out.as() + (r->it_off - s.out_begin), r->n * 4);
  }
  const auto now = Clock::now();
  float gpu_ms = 0.0f;
  if (cudaEventElapsedTime(&gpu_ms, s.start, s.done) != cudaSuccess) cudaGetLastError();
  std::lock_guard<std::mutex> lk(mu);
  gpu_s_sum += 1e-3 * double(gpu_ms);
  for (auto& r : s.reqs) {
    r->t_done = now;
    r->done = true;
    latencies.push_back(std::chrono::duration<double>(now - r->t_submit).count());
    frames_done += r->n;
    bits_done += r->n * r->c->msg();
  }
  last_done = now;
  ++batches;
  s.reqs.clear();
  s.busy = false;
  cv_done.notify_all();
}

void fecl_server_s::run() {
  cudaSetDevice(device);
  std::vector<std::shared_ptr<Request>> batch;
  for (;;) {
    bool progressed = false;
    for (auto& sp : slots) {
      Slot& s = *sp;
      if (!s.busy) continue;
      const cudaError_t q = cudaEventQuery(s.done);
      if (q == cudaErrorNotReady) continue;
      if (q != cudaSuccess) {
        cudaGetLastError();
        std::lock_guard<std::mutex> lk(mu);
        for (auto& r : s.reqs) {
          r->status = FECL_ECUDA;
          r->done = true;
        }
        error = cudaGetErrorString(q);
        s.reqs.clear();
        s.busy = false;
        cv_done.notify_all();
        continue;
      }
      harvest(s);
      progressed = true;
    }
    Slot* free_slot = nullptr;
    for (auto& sp : slots)
      if (!sp->busy) {
        free_slot = sp.get();
        break;
      }
    batch.clear();
    {
      std::unique_lock<std::mutex> lk(mu);
      if (stopping && queue.empty()) {
        bool idle = true;
        for (auto& sp : slots) idle = idle && !sp->busy;
        if (idle) return;
      }
      if (free_slot && !queue.empty()) {
        // admit the oldest requests that fit the slot's arena and frame limit
        Admission adm;
        uint64_t frames = 0;
        while (!queue.empty()) {
          auto r = queue.front();
          if (!batch.empty() && frames + r->n > opt.max_batch_frames) break;
          if (adm.bytes_with(*r) > arena_bytes()) {
            if (batch.empty()) {  // does not fit even alone
              r->status = FECL_ENOMEM;
              r->done = true;
              queue.pop_front();
              cv_done.notify_all();
              continue;
            }
            break;
          }
          adm.add(*r);
          batch.push_back(r);
          frames += r->n;
          queue.pop_front();
        }
      } else if (!progressed) {
        // nothing to launch or harvest: sleep until a submit, or briefly while batches run
        bool any_busy = false;
        for (auto& sp : slots) any_busy = any_busy || sp->busy;
        if (any_busy) cv_work.wait_for(lk, std::chrono::microseconds(20));
        else cv_work.wait_for(lk, std::chrono::milliseconds(5));
        continue;
      }
    }
    if (!batch.empty()) {
      try {
        // the batch's codecs stay locked while their kernels are planned and launched
        std::set<fecl_codec_s*> cs;
        for (auto& r : batch) cs.insert(r->c);
        std::vector<std::unique_lock<std::mutex>> locks;
        for (auto* c : cs) locks.emplace_back(c->mu);
        const auto t0 = Clock::now();
        launch(*free_slot, batch);
        const double host_s = std::chrono::duration<double>(Clock::now() - t0).count();
        std::lock_guard<std::mutex> lk(mu);
        host_s_sum += host_s;
      } catch (const Error& e) {
        std::lock_guard<std::mutex> lk(mu);
        for (auto& r : batch) {
          r->status = e.code;
          r->done = true;
        }
        error = e.msg;
        free_slot->busy = false;
        cv_done.notify_all();
      }
    }
  }
}

extern "C" {

int fecl_server_create(const fecl_server_options* options, fecl_server_t* out) {
  return guarded([&] {
    if (!out) fail(FECL_EINVAL, "null output");
    *out = nullptr;
    std::unique_ptr<fecl_server_s> s(new fecl_server_s);
    fecl_server_options o{};
    o.device_budget_bytes = 40ull << 30;
    o.max_batch_frames = 2048;
    o.slots = 3;
    if (options) {
      if (options->device_budget_bytes) o.device_budget_bytes = options->device_budget_bytes;
      if (options->max_batch_frames) o.max_batch_frames = options->max_batch_frames;
      if (options->slots) o.slots = options->slots;
    }
    if (o.slots > 16) fail(FECL_EINVAL, "at most 16 slots");
    s->opt = o;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
      cudaGetLastError();
      fail(FECL_ENODEV, "no CUDA device is visible");
    }
    cuda_check(cudaGetDevice(&s->device), "cudaGetDevice");
    cuda_check(fecl::init_device_constants(), "constant tables");
    for (uint32_t i = 0; i < o.slots; ++i) {
      std::unique_ptr<Slot> sl(new Slot);
      cuda_check(cudaStreamCreateWithFlags(&sl->stream, cudaStreamNonBlocking), "cudaStreamCreate");
      cuda_check(cudaEventCreate(&sl->done), "cudaEventCreate");
      cuda_check(cudaEventCreate(&sl->start), "cudaEventCreate");
      cuda_check(cudaEventCreateWithFlags(&sl->fork, cudaEventDisableTiming), "cudaEventCreate");
      for (int q = 0; q < kSideStreams; ++q) {
        cuda_check(cudaStreamCreateWithFlags(&sl->side[q], cudaStreamNonBlocking), "cudaStreamCreate");
        cuda_check(cudaEventCreateWithFlags(&sl->joined[q], cudaEventDisableTiming), "cudaEventCreate");
      }
      sl->arena.reserve(s->arena_bytes());
      sl->in.reserve(kInitialStagingIn);
      sl->out.reserve(kInitialStagingOut);
      s->slots.push_back(std::move(sl));
    }
    s->worker = std::thread([p = s.get()] { p->run(); });
    *out = s.release();
  });
}

int fecl_server_submit(fecl_server_t server, fecl_codec_t codec, const void* llr, int32_t llr_dtype, uint64_t nframes,
                       uint8_t* msg, int32_t* iterations, uint64_t* ticket) {
  return guarded([&] {
    if (!server || !codec || !llr || !msg || !ticket) fail(FECL_EINVAL, "null argument");
    if (nframes == 0) fail(FECL_EINVAL, "empty request");
    auto r = std::make_shared<Request>();
    {
      std::lock_guard<std::mutex> lk(codec->mu);
      codec->ensure_device();
      if (codec->device != server->device) fail(FECL_EINVAL, "the codec lives on another device than the server");
      r->lte = codec->kind == 1 && codec->lte_batch_ok();
    }
    r->c = codec;
    r->llr = llr;
    r->dtype = llr_dtype;
    r->n = nframes;
    r->msg = msg;
    r->iters = iterations;
    r->in_bytes = nframes * codec->parity() * dsize(llr_dtype);
    r->t_submit = Clock::now();
    std::lock_guard<std::mutex> lk(server->mu);
    if (server->stopping) fail(FECL_EINVAL, "server is stopping");
    r->ticket = server->next_ticket++;
    if (!server->any_submit) {
      server->first_submit = r->t_submit;
      server->any_submit = true;
    }
    server->live[r->ticket] = r;
    server->queue.push_back(r);
    *ticket = r->ticket;
    server->cv_work.notify_one();
  });
}

int fecl_server_wait(fecl_server_t server, uint64_t ticket, double timeout_s, double* latency_s) {
  return guarded([&] {
    if (!server) fail(FECL_EINVAL, "null server");
    std::unique_lock<std::mutex> lk(server->mu);
    auto it = server->live.find(ticket);
    if (it == server->live.end()) fail(FECL_EINVAL, "unknown ticket");
    auto r = it->second;
    const auto until = Clock::now() + std::chrono::duration_cast<Clock::duration>(std::chrono::duration<double>(timeout_s));
    while (!r->done) {
      if (server->cv_done.wait_until(lk, until) == std::cv_status::timeout && !r->done)
        fail(FECL_ETIMEDOUT, "request not finished");
    }
    server->live.erase(it);
    if (latency_s) *latency_s = std::chrono::duration<double>(r->t_done - r->t_submit).count();
    if (r->status != FECL_OK) fail(r->status, server->error.empty() ? "request failed" : server->error);
  });
}

int fecl_server_report(fecl_server_t server, fecl_server_stats* st) {
  return guarded([&] {
    if (!server || !st) fail(FECL_EINVAL, "null argument");
    std::lock_guard<std::mutex> lk(server->mu);
    std::vector<double> l(server->latencies);
    std::sort(l.begin(), l.end());
    auto pct = [&](double q) { return l.empty() ? 0.0 : l[std::min(l.size() - 1, size_t(q * double(l.size())))]; };
    st->requests = l.size();
    st->frames = server->frames_done;
    st->info_bits = server->bits_done;
    st->batches = server->batches;
    st->p50_s = pct(0.50);
    st->p99_s = pct(0.99);
    st->max_s = l.empty() ? 0.0 : l.back();
    st->wall_s = server->any_submit ? std::chrono::duration<double>(server->last_done - server->first_submit).count() : 0.0;
    const double nb = server->batches ? double(server->batches) : 1.0;
    st->batch_gpu_s = server->gpu_s_sum / nb;
    st->batch_host_s = server->host_s_sum / nb;
    st->batch_frames = double(server->frames_done) / nb;
  });
}

int fecl_server_reset_stats(fecl_server_t server) {
  return guarded([&] {
    if (!server) fail(FECL_EINVAL, "null server");
    std::lock_guard<std::mutex> lk(server->mu);
    server->latencies.clear();
    server->frames_done = server->bits_done = server->batches = 0;
    server->gpu_s_sum = server->host_s_sum = 0.0;
    server->any_submit = false;
  });
}

int fecl_server_replay(fecl_server_t server, uint64_t nreq, const double* arrival_s, const fecl_codec_t* codecs,
                       const void* const* llr, const int32_t* llr_dtype, const uint64_t* nframes, uint8_t* const* msg,
                       int32_t* const* iterations, double* latency_s) {
  return guarded([&] {
    if (!server || (nreq && (!arrival_s || !codecs || !llr || !llr_dtype || !nframes || !msg)))
      fail(FECL_EINVAL, "null argument");
    std::vector<uint64_t> tickets(nreq, 0);
    const auto t0 = Clock::now();
    for (uint64_t i = 0; i < nreq; ++i) {
      const auto due = t0 + std::chrono::duration_cast<Clock::duration>(std::chrono::duration<double>(arrival_s[i]));
      while (Clock::now() < due) {
        if (due - Clock::now() > std::chrono::microseconds(200)) std::this_thread::sleep_for(std::chrono::microseconds(50));
      }
      const int st = fecl_server_submit(server, codecs[i], llr[i], llr_dtype[i], nframes[i], msg[i],
                                        iterations ? iterations[i] : nullptr, &tickets[i]);
      if (st != FECL_OK) fail(st, "submit failed");
    }
    for (uint64_t i = 0; i < nreq; ++i) {
      double lat = 0.0;
      const int st = fecl_server_wait(server, tickets[i], 600.0, &lat);
      if (st != FECL_OK) fail(st, "request failed");
      if (latency_s) latency_s[i] = lat;
    }
  });
}

void fecl_server_destroy(fecl_server_t server) {
  if (!server) return;
  {
    std::lock_guard<std::mutex> lk(server->mu);
    server->stopping = true;
    server->cv_work.notify_all();
  }
  if (server->worker.joinable()) server->worker.join();
  int prev = -1;
  cudaGetDevice(&prev);
  cudaSetDevice(server->device);
  for (auto& s : server->slots) {
    cudaStreamSynchronize(s->stream);
    for (int q = 0; q < kSideStreams; ++q) {
      cudaStreamSynchronize(s->side[q]);
      cudaEventDestroy(s->joined[q]);
      cudaStreamDestroy(s->side[q]);
    }
    cudaEventDestroy(s->fork);
    cudaEventDestroy(s->done);
    cudaEventDestroy(s->start);
    cudaStreamDestroy(s->stream);
  }
  delete server;
  if (prev >= 0) cudaSetDevice(prev);
}

}  // extern "C"
