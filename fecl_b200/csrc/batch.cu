// Mixed batches: frames of several codecs -- LDPC codes of any size and rate, LTE
// turbo codes of any K -- decoded by one CUDA graph launch.
//
// At creation the batch
//   1. puts every LTE turbo job the windowed kernel covers into one persistent
//      mixed-K launch per algorithm (frames ordered longest first, so the long
//      frames start early and the short ones fill the tail);
//   2. gives every other job (LDPC, other turbo codes) the decoder fecl_decode would
//      use -- or, with FECL_BATCH_AUTOTUNE, the fastest of the candidate kernel
//      shapes, all of which compute the same bits (lane-batched LDPC with several
//      wave sizes, cluster-resident LDPC with several cluster shapes), timed on
//      the job's own inputs and remembered per (code, batch size) for the process;
//   3. carves every job's scratch out of one workspace and captures the launches
//      into a graph: the turbo launch on one branch, the other jobs spread over eight
//      more branches forked from it (longest first, each to the branch with the least
//      work so far), so they all run at once on different SMs.
// fecl_batch_run replays the graph.  The codecs' options and tables are read when
// the graph is built: changing a codec's options or destroying it invalidates the
// batch.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <map>
#include <mutex>
#include <set>
#include <sstream>
#include <string>
#include <vector>

#include "codec.hpp"
#include "ldpc_shared.hpp"

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

// A kernel choice for one non-turbo-batch job: the codec selection fields that
// plan_scratch / launch_decode read.
struct Choice {
  int kernel = FECL_KERNEL_AUTO;
  int cluster = 0, threads = 0, wave = 0;
  std::string text() const {
    std::ostringstream o;
    switch (kernel) {
      case FECL_KERNEL_LANES: o << "lanes wave=" << (wave ? std::to_string(wave) : std::string("auto")); break;
      case FECL_KERNEL_CLUSTER: o << "cluster C=" << cluster << " threads=" << threads; break;
      case FECL_KERNEL_GENERIC: o << "generic"; break;
      default: o << "auto" << (wave ? " wave=" + std::to_string(wave) : std::string());
    }
    return o.str();
  }
};

// Process-wide autotuning results, keyed by code signature and batch size.
std::mutex g_tune_mu;
std::map<std::string, std::pair<Choice, double>> g_tuned;

std::string signature(fecl_codec_s* c, uint64_t n, int32_t dtype) {
  std::ostringstream o;
  if (c->kind == 0) {
    const auto& d = c->ldpc->decoder();
    o << "ldpc " << c->ldpc->checks().rows << "x" << c->ldpc->checks().cols << " e" << c->ldpc->checks().nnz() << " a"
      << d.algorithm << " p" << d.precision << " i" << d.iterations << " f" << d.fixed_iterations;
    for (const auto& row : d.scaling)
      for (double v : row) o << " " << v;
  } else {
    o << "turbo k" << c->msg() << " p" << c->parity();
  }
  o << " n" << n << " t" << dtype;
  return o.str();
}

// Candidate choices for an LDPC job; every one computes the same bits.
std::vector<Choice> ldpc_candidates(fecl_codec_s* c, uint64_t n) {
  std::vector<Choice> v;
  v.push_back(Choice{});
  if (c->ldpc_h2_ok()) {  // the packed FP16 kernel: only its wave size is free
    const int groups = int((n + 63) / 64);
    for (int w : {1, 2, 4, 8, groups})
      if (w <= groups) v.push_back(Choice{FECL_KERNEL_AUTO, 0, 0, w});
    return v;
  }
  if (c->ldpc_lanes_ok()) {
    const int groups = int((n + 31) / 32);
    for (int w : {1, 2, 4, 8, groups})
      if (w <= groups) v.push_back(Choice{FECL_KERNEL_LANES, 0, 0, w});
  }
  if (c->ldpc->max_check_degree() <= 32)
    for (int C : {1, 2, 4, 8, 16})
      for (int t : {256, 512, 1024}) {
        if (t == 1024 && c->ldpc->max_check_degree() > 16) continue;
        if (t == 256 && c->ldpc->max_check_degree() <= 16) continue;
        v.push_back(Choice{FECL_KERNEL_CLUSTER, C, t, 0});
      }
  return v;
}

// Applies a choice to the codec for the duration of a scope.
struct ChoiceScope {
  fecl_codec_s* c;
  int k, cl, th, w;
  ChoiceScope(fecl_codec_s* codec, const Choice& ch)
      : c(codec), k(codec->kernel_sel), cl(codec->cluster_size_sel), th(codec->cluster_threads_sel),
        w(codec->lanes_wave) {
    c->kernel_sel = ch.kernel;
    c->cluster_size_sel = ch.cluster;
    c->cluster_threads_sel = ch.threads;
    c->lanes_wave = ch.wave;
  }
  ~ChoiceScope() {
    c->kernel_sel = k;
    c->cluster_size_sel = cl;
    c->cluster_threads_sel = th;
    c->lanes_wave = w;
  }
};

}  // namespace

constexpr int kBranches = 8;  // graph branches the non-turbo-batch jobs are spread over

struct fecl_batch_s {
  int device = 0;
  cudaStream_t cap = nullptr, cap2[kBranches] = {};
  cudaEvent_t fork = nullptr, join[kBranches] = {};
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  DeviceBuffer ws;
  std::string plan;
  std::vector<std::pair<fecl_codec_s*, uint64_t>> codecs;  // with their option generation at build time
  ~fecl_batch_s() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    if (cap) cudaStreamSynchronize(cap);
    for (int q = 0; q < kBranches; ++q) {
      if (cap2[q]) cudaStreamSynchronize(cap2[q]);
      if (join[q]) cudaEventDestroy(join[q]);
      if (cap2[q]) cudaStreamDestroy(cap2[q]);
    }
    if (fork) cudaEventDestroy(fork);
    if (cap) cudaStreamDestroy(cap);
  }
};

namespace {

struct JobState {
  const fecl_batch_job* job;
  fecl_codec_s* c;
  bool lte = false;
  bool multi = false;  // in the shared persistent LDPC launch
  Choice choice;
  ScratchPlan sp;
  size_t off = 0;  // scratch offset in the workspace
};

// Times one decode of the job under `ch` (device time of the second of two runs).
double time_choice(JobState& js, const Choice& ch, cudaStream_t s, DeviceBuffer& tmp) {
  ChoiceScope scope(js.c, ch);
  ScratchPlan sp;
  try {
    sp = plan_scratch(js.c, js.job->nframes, false);
  } catch (const Error&) {
    return -1.0;
  }
  if (tmp.bytes < sp.bytes) {
    cuda_check(cudaStreamSynchronize(s), "cudaStreamSynchronize");
    tmp.reserve(sp.bytes);
  }
  Launch d;
  d.llr = js.job->llr;
  d.hard = js.job->msg;
  d.iters = js.job->iterations;
  d.scratch = tmp.as<char>();
  cudaEvent_t e0, e1;
  cuda_check(cudaEventCreate(&e0), "cudaEventCreate");
  cuda_check(cudaEventCreate(&e1), "cudaEventCreate");
  float ms = -1.0f;
  try {
    launch_decode(js.c, d, sp, js.job->nframes, js.job->llr_dtype, FECL_F32, false, false, s);
    cuda_check(cudaEventRecord(e0, s), "cudaEventRecord");
    launch_decode(js.c, d, sp, js.job->nframes, js.job->llr_dtype, FECL_F32, false, false, s);
    cuda_check(cudaEventRecord(e1, s), "cudaEventRecord");
    cuda_check(cudaEventSynchronize(e1), "cudaEventSynchronize");
    cuda_check(cudaEventElapsedTime(&ms, e0, e1), "cudaEventElapsedTime");
  } catch (const Error& e) {
    if (e.code != FECL_EUNSUPPORTED) {
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      throw;
    }
    ms = -1.0f;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return ms;
}

}  // namespace

extern "C" {

int fecl_batch_create(const fecl_batch_job* jobs, uint32_t njobs, int32_t flags, fecl_batch_t* out) {
  return guarded([&] {
    if (!out) fail(FECL_EINVAL, "null output");
    *out = nullptr;
    if (!jobs || njobs == 0) fail(FECL_EINVAL, "empty batch");
    if (flags & ~(FECL_BATCH_AUTOTUNE | FECL_BATCH_SHARED_LDPC | FECL_BATCH_SHARED_PERSISTENT))
      fail(FECL_EINVAL, "Invalid batch flags");
    const bool persistent = (flags & FECL_BATCH_SHARED_PERSISTENT) != 0;
    std::vector<JobState> js(njobs);
    std::set<fecl_codec_s*> codecs;
    for (uint32_t i = 0; i < njobs; ++i) {
      const auto& j = jobs[i];
      if (!j.codec) fail(FECL_EINVAL, "null codec");
      if (j.nframes == 0 || !j.llr || !j.msg) fail(FECL_EINVAL, "empty job or null buffer");
      dsize(j.llr_dtype);
      js[i].job = &j;
      js[i].c = j.codec;
      codecs.insert(j.codec);
    }
    // Lock every codec once, in address order (a codec may appear in several jobs).
    std::vector<std::unique_lock<std::mutex>> locks;
    for (auto* c : codecs) locks.emplace_back(c->mu);
    for (auto* c : codecs) c->ensure_device();
    const int dev = (*codecs.begin())->device;
    for (auto* c : codecs)
      if (c->device != dev) fail(FECL_EINVAL, "every codec of a batch must live on one device");
    DeviceGuard dg(dev);
    for (auto* c : codecs)
      if (c->pending) cuda_check(cudaEventSynchronize(c->done), "cudaEventSynchronize");
    cuda_check(fecl::init_device_constants(), "constant tables");

    std::unique_ptr<fecl_batch_s> b(new fecl_batch_s);
    b->device = dev;
    cuda_check(cudaStreamCreateWithFlags(&b->cap, cudaStreamNonBlocking), "cudaStreamCreate");
    for (int q = 0; q < kBranches; ++q) {
      cuda_check(cudaStreamCreateWithFlags(&b->cap2[q], cudaStreamNonBlocking), "cudaStreamCreate");
      cuda_check(cudaEventCreateWithFlags(&b->join[q], cudaEventDisableTiming), "cudaEventCreate");
    }
    cuda_check(cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming), "cudaEventCreate");

    // ---- 1. turbo frames for the mixed-K launch, per algorithm
    std::map<int, std::vector<fecl::TurboLteBatchFrame>> tframes;
    std::map<int, int> tmax_k;
    for (auto& s : js) {
      s.lte = s.c->kind == 1 && s.c->lte_batch_ok();
      if (!s.lte) continue;
      const int K = int(s.c->msg());
      const int alg = s.c->tdev.algorithm;
      for (uint64_t f = 0; f < s.job->nframes; ++f) {
        fecl::TurboLteBatchFrame d;
        d.llr = static_cast<const char*>(s.job->llr) + f * s.c->parity() * dsize(s.job->llr_dtype);
        d.hard = s.job->msg + f * K;
        d.iters = s.job->iterations ? s.job->iterations + f : nullptr;
        d.perm = s.c->tdev.c[1].perm;
        d.sf = s.c->tdev.sf;
        d.crc = s.c->crc_table();
        d.K = K;
        d.iterations = s.c->tdev.iterations;
        d.llr_dtype = s.job->llr_dtype;
        tframes[alg].push_back(d);
      }
      tmax_k[alg] = std::max(tmax_k[alg], K);
    }

    // ---- 2. other jobs: choice of kernel (autotuned when asked) and scratch
    DeviceBuffer tmp;
    std::ostringstream plan;
    for (auto& s : js) {
      if (s.lte) continue;
      if ((flags & (FECL_BATCH_SHARED_LDPC | FECL_BATCH_SHARED_PERSISTENT)) && SharedLdpc::eligible(s.c)) {
        s.multi = true;
        continue;
      }
      if ((flags & FECL_BATCH_AUTOTUNE) && s.c->kind == 0 && s.c->kernel_sel == FECL_KERNEL_AUTO) {
        const std::string key = signature(s.c, s.job->nframes, s.job->llr_dtype);
        bool found = false;
        {
          std::lock_guard<std::mutex> lk(g_tune_mu);
          auto it = g_tuned.find(key);
          if (it != g_tuned.end()) {
            s.choice = it->second.first;
            found = true;
          }
        }
        if (!found) {
          double best = -1.0;
          for (const Choice& ch : ldpc_candidates(s.c, s.job->nframes)) {
            const double ms = time_choice(s, ch, b->cap, tmp);
            if (ms >= 0.0 && (best < 0.0 || ms < best)) {
              best = ms;
              s.choice = ch;
            }
          }
          std::lock_guard<std::mutex> lk(g_tune_mu);
          g_tuned[key] = {s.choice, best};
        }
      } else {
        s.choice = Choice{s.c->kernel_sel, s.c->cluster_size_sel, s.c->cluster_threads_sel, s.c->lanes_wave};
      }
      ChoiceScope scope(s.c, s.choice);
      s.sp = plan_scratch(s.c, s.job->nframes, false);
      if (s.sp.cluster) s.c->upload_cluster(s.c->cluster_plan(s.sp.cluster));  // no copies during capture
    }
    cuda_check(cudaStreamSynchronize(b->cap), "cudaStreamSynchronize");

    // ---- 3. workspace: job scratch | turbo frame scratch | descriptors | counters
    Carver cv;
    SharedLdpc shared;
    for (auto& s : js) {
      if (s.lte) continue;
      if (s.multi) {
        SharedLdpcJob j;
        j.c = s.c;
        j.n = s.job->nframes;
        j.llr = s.job->llr;
        j.dtype = s.job->llr_dtype;
        j.msg = s.job->msg;
        j.iters = s.job->iterations;
        j.scratch_off = cv.take(SharedLdpc::scratch_bytes(j));
        shared.jobs.push_back(j);
      } else {
        s.off = cv.take(s.sp.bytes);
      }
    }
    shared.plan(cv);
    std::map<int, size_t> desc_off, cnt_off;
    std::vector<std::pair<size_t, size_t>> frame_scratch;  // per turbo frame: offset
    for (auto& kv : tframes) {
      auto& v = kv.second;
      std::stable_sort(v.begin(), v.end(), [](const fecl::TurboLteBatchFrame& a, const fecl::TurboLteBatchFrame& b2) {
        return a.K > b2.K;
      });
      for (auto& d : v) {
        const size_t o = cv.take(fecl::turbo_lte_frame_floats(d.K) * sizeof(float));
        d.scratch = reinterpret_cast<float*>(o);  // relocated below
      }
      desc_off[kv.first] = cv.take(v.size() * sizeof(fecl::TurboLteBatchFrame));
      cnt_off[kv.first] = cv.take(sizeof(int32_t));
    }
    b->ws.reserve(std::max<size_t>(cv.off, 256));
    char* base = b->ws.as<char>();
    for (auto& kv : tframes) {
      for (auto& d : kv.second) d.scratch = reinterpret_cast<float*>(base + reinterpret_cast<size_t>(d.scratch));
      cuda_check(cudaMemcpy(base + desc_off[kv.first], kv.second.data(), kv.second.size() * sizeof(fecl::TurboLteBatchFrame),
                            cudaMemcpyHostToDevice),
                 "upload descriptors");
    }
    if (!shared.empty()) {
      const size_t t0 = shared.tables_begin(), t1 = shared.tables_end();
      std::vector<char> image(t1);
      shared.fill(base, image.data());
      cuda_check(cudaMemcpy(base + t0, image.data() + t0, t1 - t0, cudaMemcpyHostToDevice), "upload LDPC tables");
    }

    // ---- 4. capture
    cuda_check(cudaStreamBeginCapture(b->cap, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture");
    try {
      cuda_check(cudaEventRecord(b->fork, b->cap), "cudaEventRecord");
      for (int q = 0; q < kBranches; ++q) cuda_check(cudaStreamWaitEvent(b->cap2[q], b->fork, 0), "cudaStreamWaitEvent");
      for (auto& kv : tframes) {
        fecl::TurboLteBatchParams p;
        p.frames = reinterpret_cast<const fecl::TurboLteBatchFrame*>(base + desc_off[kv.first]);
        p.nframes = int64_t(kv.second.size());
        p.counter = reinterpret_cast<int32_t*>(base + cnt_off[kv.first]);
        p.max_K = tmax_k[kv.first];
        p.algorithm = kv.first;
        cuda_check(fecl::launch_turbo_lte_batch(p, b->cap), "turbo batch launch");
        plan << "turbo LTE mixed-K x" << kv.second.size() << " (alg " << kv.first << ", max K " << p.max_K << ")\n";
      }
      // the shared LDPC launches on branch 0: stage every job, run every class, finish
      // every job
      if (!shared.empty()) {
        shared.launch(base, b->cap2[0], persistent);
        plan << shared.describe(persistent);
      }
      const int first = shared.empty() ? 0 : 1;  // branch 0 holds the shared launches
      // longest first, each to the least loaded branch; a job's work is estimated by
      // its parity bits times its iteration limit times its frames
      std::vector<JobState*> order;
      for (auto& s : js)
        if (!s.lte && !s.multi) order.push_back(&s);
      auto cost = [](const JobState* s) {
        const double it = s->c->kind == 0 ? double(std::max(1, s->c->ldev.iterations)) : 1.0;
        return double(s->c->parity()) * it * double(s->job->nframes);
      };
      std::stable_sort(order.begin(), order.end(), [&](const JobState* a, const JobState* c) { return cost(a) > cost(c); });
      double load[kBranches] = {};
      for (JobState* sp : order) {
        auto& s = *sp;
        int q = first;
        for (int i = first + 1; i < kBranches; ++i)
          if (load[i] < load[q]) q = i;
        load[q] += cost(sp);
        cudaStream_t st = b->cap2[q];
        ChoiceScope scope(s.c, s.choice);
        Launch d;
        d.llr = s.job->llr;
        d.hard = s.job->msg;
        d.iters = s.job->iterations;
        d.scratch = base + s.off;
        launch_decode(s.c, d, s.sp, s.job->nframes, s.job->llr_dtype, FECL_F32, false, false, st);
        plan << (s.c->kind == 0 ? "ldpc " : "turbo ") << s.c->msg() << "/" << s.c->parity() << " x" << s.job->nframes
             << ": " << (s.sp.cluster ? "cluster C=" + std::to_string(s.sp.cluster) + " threads=" + std::to_string(s.sp.threads)
                                      : s.choice.text())
             << "\n";
      }
      for (int q = 0; q < kBranches; ++q) {
        cuda_check(cudaEventRecord(b->join[q], b->cap2[q]), "cudaEventRecord");
        cuda_check(cudaStreamWaitEvent(b->cap, b->join[q], 0), "cudaStreamWaitEvent");
      }
    } catch (...) {
      cudaGraph_t g = nullptr;
      cudaStreamEndCapture(b->cap, &g);
      if (g) cudaGraphDestroy(g);
      cudaGetLastError();
      throw;
    }
    cuda_check(cudaStreamEndCapture(b->cap, &b->graph), "cudaStreamEndCapture");
    cuda_check(cudaGraphInstantiate(&b->exec, b->graph, 0), "cudaGraphInstantiate");
    b->plan = plan.str();
    for (auto* c : codecs) b->codecs.emplace_back(c, c->generation.load());
    *out = b.release();
  });
}

int fecl_batch_run(fecl_batch_t batch, void* stream) {
  return guarded([&] {
    if (!batch) fail(FECL_EINVAL, "null batch");
    for (const auto& cg : batch->codecs)
      if (cg.first->generation.load() != cg.second)
        fail(FECL_EINVAL, "a codec's decoder options changed after the batch was built; build it again");
    DeviceGuard dg(batch->device);
    cuda_check(cudaGraphLaunch(batch->exec, static_cast<cudaStream_t>(stream)), "cudaGraphLaunch");
  });
}

int fecl_batch_describe(fecl_batch_t batch, char* text, uint64_t size) {
  return guarded([&] {
    if (!batch) fail(FECL_EINVAL, "null batch");
    if (text && size) {
      const size_t n = std::min<size_t>(size - 1, batch->plan.size());
      std::memcpy(text, batch->plan.data(), n);
      text[n] = 0;
    }
  });
}

void fecl_batch_destroy(fecl_batch_t batch) {
  if (!batch) return;
  int prev = -1;
  cudaGetDevice(&prev);
  cudaSetDevice(batch->device);
  delete batch;
  if (prev >= 0) cudaSetDevice(prev);
}

}  // extern "C"
