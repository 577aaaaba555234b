// The C-ABI entry points declared in include/fecl_b200.h.
//
// Each codec owns its host description (LdpcCode / TurboCode), the device copy of
// that description, a device workspace that grows to the largest batch seen, and a
// stream for host-memory calls.  Calls on one codec are serialised by a mutex; a
// device-memory call leaves an event behind that the next call on the codec waits
// for before it reuses the workspace.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <tuple>
#include <string>
#include <vector>

#include "codec.hpp"

namespace {

thread_local std::string g_error;

template <class F>
int guarded(F&& f) {
  try {
    f();
    return FECL_OK;
  } catch (const Error& e) {
    g_error = e.msg;
    return e.code;
  } catch (const std::invalid_argument& e) {
    g_error = e.what();
    return FECL_EINVAL;
  } catch (const std::bad_alloc&) {
    g_error = "host allocation failed";
    return FECL_ENOMEM;
  } catch (const std::exception& e) {
    g_error = e.what();
    return FECL_EINVAL;
  }
}

}  // namespace

namespace fecl {
// Lets entry points in other translation units report errors through fecl_last_error().
void set_last_error(const std::string& msg) { g_error = msg; }
}  // namespace fecl


namespace {

fecl::LdpcDecoderConfig ldpc_config(const fecl_ldpc_options* o, uint32_t max_degree) {
  fecl::LdpcDecoderConfig cfg;
  if (!o) return cfg;
  cfg.algorithm = o->algorithm;
  cfg.iterations = o->iterations;
  if (o->iterations == 0) fail(FECL_EINVAL, "Invalid number of iterations");
  cfg.precision = o->precision;
  cfg.fixed_iterations = o->fixed_iterations;
  if (o->scaling) {
    if (o->scaling_iterations == 0 || o->scaling_degrees == 0) fail(FECL_EINVAL, "Wrong size for scaling factor");
    cfg.scaling.assign(o->scaling_iterations, {});
    for (uint32_t i = 0; i < o->scaling_iterations; ++i)
      cfg.scaling[i].assign(o->scaling + size_t(i) * o->scaling_degrees,
                            o->scaling + size_t(i + 1) * o->scaling_degrees);
  }
  (void)max_degree;
  return cfg;
}

fecl::TurboDecoderConfig turbo_config(const fecl_turbo_options* o) {
  fecl::TurboDecoderConfig cfg;
  if (!o) return cfg;
  cfg.algorithm = o->algorithm;
  cfg.iterations = o->iterations;
  cfg.scheduling = o->scheduling;
  cfg.crc = o->crc;
  if (o->scheduling == FECL_CUSTOM) {
    if (o->n_stages && (!o->stage_counts || !o->activation || !o->transfer_counts)) fail(FECL_EINVAL, "null schedule");
    size_t a = 0, t = 0;
    for (uint32_t st = 0; st < o->n_stages; ++st) {
      fecl::TurboStage stage;
      for (uint32_t k = 0; k < o->stage_counts[st]; ++k, ++a) {
        stage.activation.push_back(o->activation[a]);
        const uint32_t n = o->transfer_counts[a];
        if (n && !o->transfer) fail(FECL_EINVAL, "null schedule");
        stage.transfer.emplace_back(o->transfer + t, o->transfer + t + n);
        t += n;
      }
      cfg.schedule.push_back(std::move(stage));
    }
  }
  cfg.precision = o->precision;
  if (o->scaling) {
    if (o->scaling_rows == 0 || o->scaling_cols == 0) fail(FECL_EINVAL, "Wrong size for scaling factor");
    cfg.scaling.assign(o->scaling_rows, {});
    for (uint32_t r = 0; r < o->scaling_rows; ++r)
      cfg.scaling[r].assign(o->scaling + size_t(r) * o->scaling_cols, o->scaling + size_t(r + 1) * o->scaling_cols);
  }
  return cfg;
}

fecl::Csr csr_in(uint32_t rows, uint32_t cols, const uint32_t* row_ptr, const uint32_t* col_idx) {
  if (!row_ptr || !col_idx) fail(FECL_EINVAL, "null check matrix");
  fecl::Csr H;
  H.rows = rows;
  H.cols = cols;
  H.row_ptr.assign(row_ptr, row_ptr + rows + 1);
  if (H.row_ptr[0] != 0) fail(FECL_EINVAL, "row_ptr must start at 0");
  for (uint32_t r = 0; r < rows; ++r)
    if (H.row_ptr[r + 1] < H.row_ptr[r]) fail(FECL_EINVAL, "row_ptr must be non-decreasing");
  H.col_idx.assign(col_idx, col_idx + H.row_ptr[rows]);
  return H;
}

void csr_out(const fecl::Csr& H, uint32_t* rows, uint32_t* cols, uint64_t* nnz, uint32_t* row_ptr, uint32_t* col_idx) {
  if (rows) *rows = H.rows;
  if (cols) *cols = H.cols;
  if (nnz) *nnz = H.nnz();
  if (row_ptr) {
    std::memcpy(row_ptr, H.row_ptr.data(), H.row_ptr.size() * sizeof(uint32_t));
    if (col_idx) std::memcpy(col_idx, H.col_idx.data(), H.col_idx.size() * sizeof(uint32_t));
  }
}

fecl_codec_s* checked(fecl_codec_t c) {
  if (!c) fail(FECL_EINVAL, "null codec");
  return c;
}



}  // namespace

namespace fecl {
namespace capi {

ScratchPlan plan_scratch(fecl_codec_s* c, uint64_t n, bool lte_fast, bool soft) {
  Carver cv;
  ScratchPlan sp;
  const uint64_t P = c->parity(), X = c->state();
  if (c->kind == 2) {
    sp.o1 = cv.take(std::max(fecl::viterbi_scratch_bytes(c->cdev, int64_t(n)), fecl::conv_map_scratch_bytes(c->cdev, int64_t(n))));
    sp.bytes = cv.off;
    return sp;
  }
  uint32_t C = 0;
  int threads = 0;
  // LDPC kernel choice under FECL_KERNEL_AUTO: the lane-batched decoder where it
  // applies, else the cluster-resident one where the code fits, else the generic one.
  const bool want_cluster = c->kind == 0 && (c->kernel_sel == FECL_KERNEL_CLUSTER ||
                                             (c->kernel_sel == FECL_KERNEL_AUTO && !c->ldpc_lanes_ok()));
  if (want_cluster && c->ldpc_cluster_shape(n, &C, &threads)) {
    auto& d = c->cluster_plan(C);
    auto it = d.max_active.find(threads);
    if (it == d.max_active.end()) {
      fecl::LdpcClusterParams q;
      q.cluster = int32_t(C);
      q.threads = threads;
      q.max_edges = int64_t(d.plan.max_edges);
      q.max_bits = int64_t(d.plan.max_bits);
      q.msg_type = c->ldpc->decoder().precision;
      it = d.max_active.emplace(threads, fecl::ldpc_cluster_max_active(q)).first;
    }
    if (it->second > 0) {
      sp.cluster = C;
      sp.threads = threads;
      sp.clusters = it->second;
      sp.o1 = cv.take(256);  // frame counter
      sp.bytes = cv.off;
      return sp;
    }
  }
  if (c->kind == 0 && c->kernel_sel == FECL_KERNEL_CLUSTER)
    fail(FECL_EUNSUPPORTED, "the code's messages do not fit a thread-block cluster");
  if (c->kind == 0 && c->ldpc_lanes_ok()) {
    size_t b = fecl::ldpc_lanes_scratch_bytes(int64_t(P), int64_t(X), int64_t(n), c->ldpc->decoder().precision);
    if (c->ldpc_h2_ok()) b = std::max(b, fecl::ldpc_lanes_h2_scratch_bytes(int64_t(P), int64_t(X), int64_t(n)));
    sp.o1 = cv.take(b);
  } else if (lte_fast) {
    sp.o1 = cv.take(fecl::turbo_lte_scratch_bytes(int(c->msg()), int64_t(n), soft || c->tdev.scheduling == 1));
  } else if (c->kind == 0) {
    sp.o1 = cv.take(n * c->ldev.E * 4);
    sp.o2 = cv.take(n * P * 4);
    sp.o3 = cv.take(n * P * 4);
  } else {
    sp.o1 = cv.take(n * P * 4);
    sp.o2 = cv.take(n * P * 4);
    sp.o3 = cv.take(n * X * 4);
    sp.o4 = cv.take(n * X * 4);
    sp.o5 = cv.take(n * uint64_t(c->tdev.max_steps) * c->tdev.max_states * 4);
  }
  sp.bytes = cv.off;
  return sp;
}

fecl::LdpcLanesParams lanes_params(fecl_codec_s* c, const Launch& d, uint64_t n, int32_t in_dtype, int32_t out_dtype) {
  fecl::LdpcLanesParams r;
  const auto& L = c->ldev;
  r.M = L.M;
  r.N = L.N;
  r.msg = L.msg;
  r.d_max = L.d_max;
  r.E = L.E;
  r.row_ptr = L.row_ptr;
  r.col_idx = L.col_idx;
  r.col_ptr = L.col_ptr;
  r.col_edges = L.col_edges;
  r.sf = L.sf;
  r.n_sf = L.n_sf;
  r.sf_stride = L.sf_stride;
  r.algorithm = L.algorithm;
  r.iterations = L.iterations;
  r.fixed_iterations = L.fixed_iterations;
  r.msg_type = c->ldpc->decoder().precision;
  r.wave_groups = c->lanes_wave;
  r.persist = c->lanes_persist;
  r.nframes = int64_t(n);
  r.llr = d.llr;
  r.llr_dtype = in_dtype;
  r.syst_in = d.syst;
  r.state_in = d.state;
  r.hard = d.hard;
  r.iters = d.iters;
  r.msg_out = d.msg;
  r.syst_out = d.syst_out;
  r.parity_out = d.parity_out;
  r.state_out = d.state_out;
  r.out_dtype = out_dtype;
  return r;
}

void launch_decode(fecl_codec_s* c, const Launch& d, const ScratchPlan& sp, uint64_t n, int32_t in_dtype,
                   int32_t out_dtype, bool soft, bool lte_fast, cudaStream_t s) {
  cudaError_t e;
  auto at = [&](size_t off) { return d.scratch + off; };
  if (c->kind == 2) {
    if (soft) {
      fecl::ConvMapRun r;
      r.nframes = int64_t(n);
      r.algorithm = c->conv->decoder().algorithm;
      r.sf = float(c->conv->decoder().scaling);
      r.llr = d.llr;
      r.syst_in = d.syst;
      r.llr_dtype = in_dtype;
      r.msg_out = d.msg;
      r.syst_out = d.syst_out;
      r.parity_out = d.parity_out;
      r.out_dtype = out_dtype;
      e = fecl::launch_conv_map(c->cdev, r, at(sp.o1), s);
    } else {
      fecl::ViterbiRun r;
      r.nframes = int64_t(n);
      r.llr = d.llr;
      r.llr_dtype = in_dtype;
      r.hard = d.hard;
      r.trace = reinterpret_cast<uint8_t*>(at(sp.o1));
      e = fecl::launch_viterbi(c->cdev, r, s);
      if (e == cudaSuccess && d.iters) e = cudaMemsetAsync(d.iters, 0, n * sizeof(int32_t), s);
    }
  } else if (c->kind == 0 && sp.cluster) {
    auto& cd = c->cluster_plan(sp.cluster);
    c->upload_cluster(cd);
    fecl::LdpcClusterParams r;
    const auto& L = c->ldev;
    r.M = L.M;
    r.N = L.N;
    r.msg = L.msg;
    r.d_max = L.d_max;
    r.E = L.E;
    r.row_ptr = L.row_ptr;
    r.chk_addr = cd.chk_addr.as<uint32_t>();
    r.bit_ptr = cd.bit_ptr.as<uint32_t>();
    r.bit_addr = cd.bit_addr.as<uint32_t>();
    r.row_split = cd.row_split.as<uint32_t>();
    r.bit_split = cd.bit_split.as<uint32_t>();
    r.sf = L.sf;
    r.n_sf = L.n_sf;
    r.sf_stride = L.sf_stride;
    r.algorithm = L.algorithm;
    r.iterations = L.iterations;
    r.fixed_iterations = L.fixed_iterations;
    r.separate_syndrome = 0;
    for (const auto& row : c->ldpc->decoder().scaling)
      if (row != c->ldpc->decoder().scaling[0]) r.separate_syndrome = 1;
    r.msg_type = c->ldpc->decoder().precision;
    r.cluster = int32_t(sp.cluster);
    r.threads = sp.threads;
    r.clusters = sp.clusters;
    r.max_edges = int64_t(cd.plan.max_edges);
    r.max_bits = int64_t(cd.plan.max_bits);
    r.counter = reinterpret_cast<int32_t*>(at(sp.o1));
    r.nframes = int64_t(n);
    r.llr = d.llr;
    r.llr_dtype = in_dtype;
    r.syst_in = d.syst;
    r.state_in = d.state;
    r.hard = d.hard;
    r.iters = d.iters;
    r.msg_out = d.msg;
    r.syst_out = d.syst_out;
    r.parity_out = d.parity_out;
    r.state_out = d.state_out;
    r.out_dtype = out_dtype;
    e = fecl::launch_ldpc_cluster(r, s);
  } else if (c->kind == 0 && c->ldpc_lanes_ok()) {
    const fecl::LdpcLanesParams r = lanes_params(c, d, n, in_dtype, out_dtype);
    if (c->ldpc_h2_ok() && !d.state) e = fecl::launch_ldpc_lanes_h2(r, at(sp.o1), s);
    else e = fecl::launch_ldpc_lanes(r, at(sp.o1), s);
  } else if (c->kind == 0) {
    if (c->ldpc->decoder().precision != 0)
      fail(FECL_EUNSUPPORTED, "FP16 / int8 messages need check degrees <= 32 and a scaling constant across iterations");
    fecl::LdpcRun r;
    r.nframes = int64_t(n);
    r.llr = d.llr;
    r.llr_dtype = in_dtype;
    r.syst_in = d.syst;
    r.state_in = d.state;
    r.hard = d.hard;
    r.iters = d.iters;
    r.msg_out = d.msg;
    r.syst_out = d.syst_out;
    r.parity_out = d.parity_out;
    r.state_out = d.state_out;
    r.out_dtype = out_dtype;
    r.c2v = reinterpret_cast<float*>(at(sp.o1));
    r.app = reinterpret_cast<float*>(at(sp.o2));
    r.chan = reinterpret_cast<float*>(at(sp.o3));
    e = fecl::launch_ldpc_flood(c->ldev, r, s);
  } else if (lte_fast) {
    fecl::TurboLteParams r;
    r.nframes = int64_t(n);
    r.K = int32_t(c->msg());
    r.iterations = c->tdev.iterations;
    r.algorithm = c->tdev.algorithm;
    r.train = c->lte_train;
    r.segs = c->lte_segs;
    r.perm[0] = c->tdev.c[0].perm;
    r.perm[1] = c->tdev.c[1].perm;
    r.sf = c->tdev.sf;
    r.llr = d.llr;
    r.llr_dtype = in_dtype;
    r.hard = d.hard;
    r.iters = d.iters;
    r.scratch = reinterpret_cast<float*>(at(sp.o1));
    if (!c->stats.ptr) {
      c->stats.reserve(3 * sizeof(unsigned long long));
      cuda_check(cudaMemset(c->stats.ptr, 0, 3 * sizeof(unsigned long long)), "cudaMemset");
    }
    r.stats = c->stats.as<unsigned long long>();
    r.crc = soft ? nullptr : c->crc_table();
    r.parallel = c->tdev.scheduling == 1 ? 1 : 0;
    if (soft) {
      r.soft = 1;
      r.hard = nullptr;
      r.iters = nullptr;
      r.syst_in = d.syst;
      r.state_in = d.state;
      r.msg_out = d.msg;
      r.syst_out = d.syst_out;
      r.parity_out = d.parity_out;
      r.state_out = d.state_out;
      r.out_dtype = out_dtype;
    }
    e = fecl::launch_turbo_lte(r, s);
  } else {
    fecl::TurboRun r;
    if (!soft) r.crc = c->crc_table();
    r.nframes = int64_t(n);
    r.soft = soft ? 1 : 0;
    r.llr = d.llr;
    r.llr_dtype = in_dtype;
    r.syst_in = d.syst;
    r.state_in = d.state;
    r.hard = d.hard;
    r.iters = d.iters;
    r.msg_out = d.msg;
    r.syst_out = d.syst_out;
    r.parity_out = d.parity_out;
    r.state_out = d.state_out;
    r.out_dtype = out_dtype;
    r.parity_in = reinterpret_cast<float*>(at(sp.o1));
    r.parity_buf = reinterpret_cast<float*>(at(sp.o2));
    r.ext = reinterpret_cast<float*>(at(sp.o3));
    r.ext_buf = reinterpret_cast<float*>(at(sp.o4));
    r.alpha = reinterpret_cast<float*>(at(sp.o5));
    e = fecl::launch_turbo_generic(c->tdev, r, s);
  }
  if (e == cudaErrorInvalidValue) fail(FECL_EUNSUPPORTED, "code shape not supported by the device decoder");
  cuda_check(e, "kernel launch");
}

}  // namespace capi
}  // namespace fecl

namespace {

// Grows the workspace to `bytes`; the old one may still be read by queued work.
void reserve_workspace(fecl_codec_s* c, size_t bytes) {
  if (c->ws.bytes >= bytes) return;
  if (c->pending) cuda_check(cudaEventSynchronize(c->done), "cudaEventSynchronize");
  c->sync_pipes();
  c->ws.reserve(bytes);
}

// Runs a decode.  Device-memory calls launch on the caller's stream.  Host-memory
// calls pipeline the batch in chunks and return when every result is on the host:
// every chunk has its own device buffers; the chunks are copied in one after the
// other on one stream, so each arrives at the full host link bandwidth and the first
// one early; a chunk's decode (and its copy out) starts on one of the codec's decode
// streams as soon as its inputs are in, while later chunks are still being copied,
// and the decodes of neighbouring chunks share the GPU.  So the copy of the batch is
// hidden behind decoding except for the first chunk.
void run_decode(fecl_codec_s* c, const fecl_so_io* io, uint64_t n, uint8_t* hard, int32_t* iters, bool soft,
                int32_t flags, cudaStream_t user_stream) {
  if (flags != FECL_HOST_MEMORY && flags != FECL_DEVICE_MEMORY) fail(FECL_EINVAL, "Invalid memory flag");
  c->ensure_device();
  DeviceGuard dg(c->device);
  const bool host = (flags == FECL_HOST_MEMORY);
  const size_t isz = dsize(io->in_dtype);
  const size_t osz = soft ? dsize(io->out_dtype) : 4;
  const uint64_t P = c->parity(), S = c->syst(), M = c->msg(), X = c->state();
  const bool lte_fast = c->kind == 1 && c->lte_fast_ok();

  if (!host) {
    const ScratchPlan sp = plan_scratch(c, n, lte_fast, soft);
    c->wait_previous(user_stream);
    reserve_workspace(c, sp.bytes);
    Launch d;
    d.llr = io->parity;
    d.syst = io->syst;
    d.state = io->state;
    d.hard = hard;
    d.iters = iters;
    d.msg = io->msg;
    d.syst_out = io->syst_out;
    d.parity_out = io->parity_out;
    d.state_out = io->state_out;
    d.scratch = c->ws.as<char>();
    launch_decode(c, d, sp, n, io->in_dtype, io->out_dtype, soft, lte_fast, user_stream);
    c->mark(user_stream);
    return;
  }

  // Chunks of at least one frame group of the kernel that runs (32 frames, 64 for the
  // packed FP16 LDPC kernel), at most kMaxChunks per call, each with its own buffers;
  // decodes go round robin over the decode streams.
  constexpr uint64_t kMaxChunks = fecl_codec_s::kMaxChunks;
  const uint64_t min_chunk = (c->ldpc_h2_ok() && !io->state) ? 64 : 32;
  const uint64_t nchunks = std::max<uint64_t>(1, std::min<uint64_t>(kMaxChunks, n / min_chunk));
  const uint64_t chunk = (n + nchunks - 1) / nchunks;
  const int nslots = int(nchunks);
  Carver cv;
  const size_t o_llr = cv.take(chunk * P * isz);
  const size_t o_syst = io->syst ? cv.take(chunk * S * isz) : 0;
  const size_t o_state = io->state ? cv.take(chunk * X * isz) : 0;
  const size_t o_hard = hard ? cv.take(chunk * M) : 0;
  const size_t o_iters = iters ? cv.take(chunk * 4) : 0;
  const size_t o_msg = io->msg ? cv.take(chunk * M * osz) : 0;
  const size_t o_so = io->syst_out ? cv.take(chunk * S * osz) : 0;
  const size_t o_po = io->parity_out ? cv.take(chunk * P * osz) : 0;
  const size_t o_sto = io->state_out ? cv.take(chunk * X * osz) : 0;
  const ScratchPlan sp = plan_scratch(c, chunk, lte_fast, soft);
  const size_t o_scr = cv.take(sp.bytes);
  const size_t slot_bytes = cv.off;
  if (c->pending) {
    for (cudaStream_t st : c->pipe) cuda_check(cudaStreamWaitEvent(st, c->done, 0), "cudaStreamWaitEvent");
    cuda_check(cudaStreamWaitEvent(c->copy_in, c->done, 0), "cudaStreamWaitEvent");
  }
  reserve_workspace(c, slot_bytes * nslots);
  const char* hp = static_cast<const char*>(io->parity);
  // If a step fails part way, the copies already queued still read and write the
  // caller's host buffers: let them finish before the error returns.
  struct Drain {
    fecl_codec_s* c;
    bool armed = true;
    ~Drain() {
      if (!armed) return;
      for (cudaStream_t st : c->pipe) cudaStreamSynchronize(st);
      cudaStreamSynchronize(c->copy_in);
      cudaGetLastError();
    }
  } drain{c};
  for (uint64_t k = 0; k < nchunks; ++k) {
    const uint64_t f0 = k * chunk;
    if (f0 >= n) break;
    const uint64_t nk = std::min(chunk, n - f0);
    const int slot = int(k);
    cudaStream_t st = c->pipe[k % fecl_codec_s::kPipe];
    cudaStream_t in = c->copy_in;
    char* base = c->ws.as<char>() + slot * slot_bytes;
    Launch d;
    cuda_check(cudaMemcpyAsync(base + o_llr, hp + f0 * P * isz, nk * P * isz, cudaMemcpyHostToDevice, in), "copy in");
    d.llr = base + o_llr;
    if (io->syst) {
      cuda_check(cudaMemcpyAsync(base + o_syst, static_cast<const char*>(io->syst) + f0 * S * isz, nk * S * isz,
                                 cudaMemcpyHostToDevice, in), "copy in");
      d.syst = base + o_syst;
    }
    if (io->state) {
      cuda_check(cudaMemcpyAsync(base + o_state, static_cast<const char*>(io->state) + f0 * X * isz, nk * X * isz,
                                 cudaMemcpyHostToDevice, in), "copy in");
      d.state = base + o_state;
    }
    cuda_check(cudaEventRecord(c->arrived[k], in), "cudaEventRecord");
    cuda_check(cudaStreamWaitEvent(st, c->arrived[k], 0), "cudaStreamWaitEvent");
    if (hard) d.hard = reinterpret_cast<uint8_t*>(base + o_hard);
    if (iters) d.iters = reinterpret_cast<int32_t*>(base + o_iters);
    if (io->msg) d.msg = base + o_msg;
    if (io->syst_out) d.syst_out = base + o_so;
    if (io->parity_out) d.parity_out = base + o_po;
    if (io->state_out) d.state_out = base + o_sto;
    d.scratch = base + o_scr;
    launch_decode(c, d, sp, nk, io->in_dtype, io->out_dtype, soft, lte_fast, st);
    if (hard) cuda_check(cudaMemcpyAsync(hard + f0 * M, d.hard, nk * M, cudaMemcpyDeviceToHost, st), "copy out");
    if (iters) cuda_check(cudaMemcpyAsync(iters + f0, d.iters, nk * 4, cudaMemcpyDeviceToHost, st), "copy out");
    if (io->msg)
      cuda_check(cudaMemcpyAsync(static_cast<char*>(io->msg) + f0 * M * osz, d.msg, nk * M * osz,
                                 cudaMemcpyDeviceToHost, st), "copy out");
    if (io->syst_out)
      cuda_check(cudaMemcpyAsync(static_cast<char*>(io->syst_out) + f0 * S * osz, d.syst_out, nk * S * osz,
                                 cudaMemcpyDeviceToHost, st), "copy out");
    if (io->parity_out)
      cuda_check(cudaMemcpyAsync(static_cast<char*>(io->parity_out) + f0 * P * osz, d.parity_out, nk * P * osz,
                                 cudaMemcpyDeviceToHost, st), "copy out");
    if (io->state_out)
      cuda_check(cudaMemcpyAsync(static_cast<char*>(io->state_out) + f0 * X * osz, d.state_out, nk * X * osz,
                                 cudaMemcpyDeviceToHost, st), "copy out");
  }
  c->sync_pipes();
  drain.armed = false;
  c->pending = false;
}

}  // namespace

extern "C" {

const char* fecl_version(void) { return "fecl_b200 0.1 (sm_100a)"; }

const char* fecl_last_error(void) { return g_error.c_str(); }

const char* fecl_strerror(int status) {
  switch (status) {
    case FECL_OK: return "success";
    case FECL_EINVAL: return "invalid argument";
    case FECL_ECUDA: return "CUDA error";
    case FECL_ENOMEM: return "out of memory";
    case FECL_ETIMEDOUT: return "device wait timed out";
    case FECL_EUNSUPPORTED: return "unsupported on the device";
    case FECL_ENODEV: return "no CUDA device";
  }
  return "unknown status";
}

int fecl_dvbs2_matrix(uint32_t n, uint32_t rate_num, uint32_t rate_den, uint32_t* rows, uint32_t* cols, uint64_t* nnz,
                      uint32_t* row_ptr, uint32_t* col_idx) {
  return guarded([&] {
    if (rate_den == 0) fail(FECL_EINVAL, "Invalid rate");
    csr_out(fecl::dvbs2_matrix(n, rate_num, rate_den), rows, cols, nnz, row_ptr, col_idx);
  });
}

int fecl_gallager_matrix(uint32_t n, uint32_t wc, uint32_t wr, uint64_t seed, uint32_t* rows, uint64_t* nnz,
                         uint32_t* row_ptr, uint32_t* col_idx) {
  return guarded([&] { csr_out(fecl::gallager_matrix(n, wc, wr, seed), rows, nullptr, nnz, row_ptr, col_idx); });
}

int fecl_ldpc_create(uint32_t rows, uint32_t cols, const uint32_t* row_ptr, const uint32_t* col_idx,
                     const fecl_ldpc_options* options, fecl_codec_t* out) {
  return guarded([&] {
    if (!out) fail(FECL_EINVAL, "null output");
    std::unique_ptr<fecl_codec_s> c(new fecl_codec_s);
    c->kind = 0;
    c->ldpc.reset(new fecl::LdpcCode(csr_in(rows, cols, row_ptr, col_idx)));
    if (options) c->ldpc->set_decoder(ldpc_config(options, c->ldpc->max_check_degree()));
    *out = c.release();
  });
}

int fecl_ldpc_set_options(fecl_codec_t codec, const fecl_ldpc_options* options) {
  return guarded([&] {
    auto c = checked(codec);
    if (c->kind != 0) fail(FECL_EINVAL, "not an LDPC codec");
    std::lock_guard<std::mutex> lk(c->mu);
    c->ldpc->set_decoder(ldpc_config(options, c->ldpc->max_check_degree()));
    c->generation.fetch_add(1);
    if (c->on_device) {
      DeviceGuard dg(c->device);
      if (c->pending) cuda_check(cudaEventSynchronize(c->done), "cudaEventSynchronize");
      c->upload_ldpc_options();
    }
  });
}

int fecl_ldpc_checks(fecl_codec_t codec, uint32_t* rows, uint32_t* cols, uint64_t* nnz, uint32_t* row_ptr,
                     uint32_t* col_idx) {
  return guarded([&] {
    auto c = checked(codec);
    if (c->kind != 0) fail(FECL_EINVAL, "not an LDPC codec");
    csr_out(c->ldpc->checks(), rows, cols, nnz, row_ptr, col_idx);
  });
}

int fecl_trellis_build(uint32_t ninputs, const uint32_t* constraint_lengths, uint32_t noutputs,
                       const uint64_t* generators, const uint64_t* feedback, uint32_t* state_count,
                       uint32_t* input_count, uint32_t* output_size, uint32_t* next_state, uint32_t* output) {
  return guarded([&] {
    if (ninputs == 0 || noutputs == 0 || !constraint_lengths || !generators) fail(FECL_EINVAL, "Invalid number of generators");
    std::vector<uint32_t> cl(constraint_lengths, constraint_lengths + ninputs);
    for (auto v : cl)
      if (v < 2) fail(FECL_EINVAL, "Invalid constraint length");
    std::vector<std::vector<uint64_t>> gen(ninputs);
    for (uint32_t i = 0; i < ninputs; ++i) gen[i].assign(generators + size_t(i) * noutputs, generators + size_t(i + 1) * noutputs);
    std::vector<uint64_t> fb;
    if (feedback) fb.assign(feedback, feedback + ninputs);
    auto t = fecl::Trellis::from_generators(cl, gen, fb);
    if (state_count) *state_count = t.state_count;
    if (input_count) *input_count = t.input_count;
    if (output_size) *output_size = t.output_size;
    if (next_state) std::memcpy(next_state, t.next_state.data(), t.next_state.size() * 4);
    if (output) std::memcpy(output, t.output.data(), t.output.size() * 4);
  });
}

int fecl_turbo_create(uint32_t n_constituents, const fecl_trellis* trellis, uint32_t n_trellis, const uint32_t* perm_data,
                      const uint32_t* perm_len, const int32_t* termination, uint32_t n_termination,
                      const fecl_turbo_options* options, fecl_codec_t* out) {
  return guarded([&] {
    if (!out) fail(FECL_EINVAL, "null output");
    if (!trellis || n_trellis == 0) fail(FECL_EINVAL, "Trellis and Permutation count don't match");
    std::vector<fecl::Trellis> tr;
    for (uint32_t i = 0; i < n_trellis; ++i)
      tr.push_back(fecl::Trellis::from_tables(trellis[i].state_count, trellis[i].input_count, trellis[i].output_size,
                                              trellis[i].next_state, trellis[i].output));
    std::vector<std::vector<uint32_t>> perms(n_constituents);
    size_t off = 0;
    for (uint32_t i = 0; i < n_constituents; ++i) {
      const uint32_t len = perm_len ? perm_len[i] : 0;
      if (len && !perm_data) fail(FECL_EINVAL, "null interleaver data");
      perms[i].assign(perm_data + off, perm_data + off + len);
      off += len;
    }
    std::vector<int> term;
    if (termination && n_termination)
      term.assign(termination, termination + n_termination);
    else
      term.push_back(FECL_TAIL);
    std::unique_ptr<fecl_codec_s> c(new fecl_codec_s);
    c->kind = 1;
    c->turbo.reset(new fecl::TurboCode(tr, perms, term));
    if (options) c->turbo->set_decoder(turbo_config(options));
    *out = c.release();
  });
}

int fecl_conv_create(const fecl_trellis* trellis, uint32_t length, int32_t termination, const fecl_conv_options* options,
                     fecl_codec_t* out) {
  return guarded([&] {
    if (!out || !trellis) fail(FECL_EINVAL, "null argument");
    std::unique_ptr<fecl_codec_s> c(new fecl_codec_s);
    c->kind = 2;
    c->conv.reset(new fecl::ConvCode(fecl::Trellis::from_tables(trellis->state_count, trellis->input_count,
                                                                trellis->output_size, trellis->next_state, trellis->output),
                                     length, termination));
    if (options) c->conv->set_decoder(fecl::ConvDecoderConfig{options->algorithm, options->scaling});
    *out = c.release();
  });
}

int fecl_conv_set_options(fecl_codec_t codec, const fecl_conv_options* options) {
  return guarded([&] {
    auto c = checked(codec);
    if (c->kind != 2) fail(FECL_EINVAL, "not a convolutional codec");
    if (!options) fail(FECL_EINVAL, "null options");
    std::lock_guard<std::mutex> lk(c->mu);
    c->conv->set_decoder(fecl::ConvDecoderConfig{options->algorithm, options->scaling});
    c->generation.fetch_add(1);
  });
}

int fecl_conv_puncturing(fecl_codec_t codec, const uint8_t* mask, uint32_t mask_len, const uint8_t* tail_mask,
                         uint32_t tail_mask_len, uint32_t* seq, uint64_t* seq_len) {
  return guarded([&] {
    auto c = checked(codec);
    if (c->kind != 2) fail(FECL_EINVAL, "not a convolutional codec");
    if (!seq_len) fail(FECL_EINVAL, "null output");
    std::vector<uint8_t> m(mask, mask + (mask ? mask_len : 0)), t(tail_mask, tail_mask + (tail_mask ? tail_mask_len : 0));
    const auto v = fecl::conv_puncturing(*c->conv, m, t);
    *seq_len = v.size();
    if (seq) std::memcpy(seq, v.data(), v.size() * sizeof(uint32_t));
  });
}

int fecl_lte_interleaver(uint32_t K, uint32_t* perm) {
  return guarded([&] {
    auto p = fecl::lte_interleaver(K);
    if (perm) std::memcpy(perm, p.data(), p.size() * 4);
  });
}

int fecl_turbo_create_lte(uint32_t K, const fecl_turbo_options* options, fecl_codec_t* out) {
  return guarded([&] {
    if (!out) fail(FECL_EINVAL, "null output");
    auto t = fecl::lte_trellis();
    std::vector<std::vector<uint32_t>> perms{{}, fecl::lte_interleaver(K)};
    std::unique_ptr<fecl_codec_s> c(new fecl_codec_s);
    c->kind = 1;
    c->turbo.reset(new fecl::TurboCode({t}, perms, {FECL_TAIL}));
    if (options) c->turbo->set_decoder(turbo_config(options));
    *out = c.release();
  });
}

int fecl_turbo_set_options(fecl_codec_t codec, const fecl_turbo_options* options) {
  return guarded([&] {
    auto c = checked(codec);
    if (c->kind != 1) fail(FECL_EINVAL, "not a turbo codec");
    std::lock_guard<std::mutex> lk(c->mu);
    c->turbo->set_decoder(turbo_config(options));
    c->generation.fetch_add(1);
    if (c->on_device) {
      DeviceGuard dg(c->device);
      if (c->pending) cuda_check(cudaEventSynchronize(c->done), "cudaEventSynchronize");
      c->upload_turbo_options();
    }
  });
}

int fecl_codec_sizes(fecl_codec_t codec, fecl_sizes* sizes) {
  return guarded([&] {
    auto c = checked(codec);
    if (!sizes) fail(FECL_EINVAL, "null output");
    sizes->msg = c->msg();
    sizes->syst = c->syst();
    sizes->parity = c->parity();
    sizes->state = c->state();
  });
}

int fecl_encode(fecl_codec_t codec, const uint8_t* msg, uint64_t nframes, uint8_t* parity, int32_t flags, void* stream) {
  return guarded([&] {
    auto c = checked(codec);
    if (!msg || !parity) fail(FECL_EINVAL, "null buffer");
    const uint64_t M = c->msg(), P = c->parity();
    if (flags == FECL_DEVICE_MEMORY) {
      // the device encoders (device/encode.cu), asynchronous on the caller's stream
      std::lock_guard<std::mutex> lk(c->mu);
      c->ensure_device();
      DeviceGuard dg(c->device);
      cudaStream_t s = static_cast<cudaStream_t>(stream);
      if (c->kind == 0) cuda_check(fecl::launch_ldpc_encode(c->ltab, msg, parity, int64_t(nframes), s), "encode");
      else if (c->kind == 1) cuda_check(fecl::launch_turbo_encode(c->tdev, msg, parity, int64_t(nframes), s), "encode");
      else cuda_check(fecl::launch_conv_encode(c->cdev, msg, parity, int64_t(nframes), s), "encode");
      return;
    }
    if (flags != FECL_HOST_MEMORY) fail(FECL_EINVAL, "Invalid memory flag");
    for (uint64_t f = 0; f < nframes; ++f) {
      if (c->kind == 0) c->ldpc->encode(msg + f * M, parity + f * P);
      else if (c->kind == 1) c->turbo->encode(msg + f * M, parity + f * P);
      else c->conv->encode(msg + f * M, parity + f * P);
    }
  });
}

int fecl_awgn_llr(const uint8_t* bits, uint64_t n, double ebn0_db, double rate, uint64_t seed, int32_t out_dtype, void* out,
                  void* stream) {
  return guarded([&] {
    if (!bits || !out) fail(FECL_EINVAL, "null buffer");
    if (!(rate > 0.0)) fail(FECL_EINVAL, "rate must be positive");
    dsize(out_dtype);
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
      cudaGetLastError();
      fail(FECL_ENODEV, "no CUDA device is visible");
    }
    const double esn0 = std::pow(10.0, ebn0_db / 10.0) * rate;
    cuda_check(fecl::launch_awgn(bits, int64_t(n), esn0, seed, out_dtype, out, static_cast<cudaStream_t>(stream)), "awgn");
  });
}

int fecl_check(fecl_codec_t codec, const uint8_t* parity, uint64_t nframes, int32_t* ok) {
  return guarded([&] {
    auto c = checked(codec);
    if (!parity || !ok) fail(FECL_EINVAL, "null buffer");
    const uint64_t P = c->parity();
    int32_t r = 1;
    for (uint64_t f = 0; f < nframes && r; ++f) {
      const uint8_t* q = parity + f * P;
      r = (c->kind == 0 ? c->ldpc->check(q) : c->kind == 1 ? c->turbo->check(q) : c->conv->check(q)) ? 1 : 0;
    }
    *ok = r;
  });
}

int fecl_decode(fecl_codec_t codec, const void* llr, int32_t llr_dtype, uint64_t nframes, uint8_t* msg, int32_t* iterations,
                int32_t flags, void* stream) {
  return guarded([&] {
    auto c = checked(codec);
    if (nframes == 0) return;  // nothing to decode: empty buffers may be null
    if (!llr || !msg) fail(FECL_EINVAL, "null buffer");
    std::lock_guard<std::mutex> lk(c->mu);
    fecl_so_io io{};
    io.parity = llr;
    io.in_dtype = llr_dtype;
    io.out_dtype = FECL_F32;
    run_decode(c, &io, nframes, msg, iterations, false, flags, static_cast<cudaStream_t>(stream));
  });
}

int fecl_so_decode(fecl_codec_t codec, const fecl_so_io* io, uint64_t nframes, int32_t flags, void* stream) {
  return guarded([&] {
    auto c = checked(codec);
    if (!io) fail(FECL_EINVAL, "null io");
    if (io->out_dtype != FECL_F64 && io->out_dtype != FECL_F32) fail(FECL_EINVAL, "Invalid output element type");
    if (nframes == 0) return;  // nothing to decode: empty buffers may be null
    if (!io->parity) fail(FECL_EINVAL, "Input must contains parity");
    std::lock_guard<std::mutex> lk(c->mu);
    run_decode(c, io, nframes, nullptr, nullptr, true, flags, static_cast<cudaStream_t>(stream));
  });
}

// Process-wide results of the windowed turbo decoder's autotuner: (K, frames,
// algorithm, iterations, scheduling) -> (segments, training steps).
static std::mutex g_window_mu;
static std::map<std::tuple<uint64_t, uint64_t, int, int, int>, std::pair<int, int>> g_window_tuned;

int fecl_turbo_tune_window(fecl_codec_t codec, const void* llr, int32_t llr_dtype, uint64_t nframes, uint8_t* msg,
                           void* stream, int32_t* segments, int32_t* training) {
  return guarded([&] {
    auto c = checked(codec);
    if (c->kind != 1) fail(FECL_EINVAL, "not a turbo codec");
    if (!llr || !msg || nframes == 0) fail(FECL_EINVAL, "null buffer or no frames");
    std::lock_guard<std::mutex> lk(c->mu);
    if (!c->lte_fast_ok()) fail(FECL_EUNSUPPORTED, "the codec does not take the windowed decoder");
    const auto& d = c->turbo->decoder();
    const auto key = std::make_tuple(c->msg(), nframes, int(d.algorithm), int(d.iterations), int(d.scheduling));
    std::pair<int, int> best{0, -1};
    bool cached = false;
    {
      std::lock_guard<std::mutex> g(g_window_mu);
      auto it = g_window_tuned.find(key);
      if (it != g_window_tuned.end()) {
        best = it->second;
        cached = true;
      }
    }
    if (!cached) {
      // Every candidate computes the full-frame recursion up to FP32 rounding; each is
      // timed on the caller's own L-values (second of two decodes) and the fastest kept.
      cudaStream_t s = static_cast<cudaStream_t>(stream);
      cudaEvent_t e0, e1;
      cuda_check(cudaEventCreate(&e0), "cudaEventCreate");
      cuda_check(cudaEventCreate(&e1), "cudaEventCreate");
      float best_ms = -1.0f;
      fecl_so_io io{};
      io.parity = llr;
      io.in_dtype = llr_dtype;
      io.out_dtype = FECL_F32;
      try {
        // 0: the launcher's own choice (balanced rounds of the 32- and 64-segment
        // shapes, or 128 segments for at most one frame per SM)
        for (int segs : {0, 128, 64, 32})
          for (int train : {48, 64, 80, 96, 128}) {
            c->lte_segs = segs;
            c->lte_train = train;
            run_decode(c, &io, nframes, msg, nullptr, false, FECL_DEVICE_MEMORY, s);
            cuda_check(cudaEventRecord(e0, s), "cudaEventRecord");
            run_decode(c, &io, nframes, msg, nullptr, false, FECL_DEVICE_MEMORY, s);
            cuda_check(cudaEventRecord(e1, s), "cudaEventRecord");
            cuda_check(cudaEventSynchronize(e1), "cudaEventSynchronize");
            float ms = 0.0f;
            cuda_check(cudaEventElapsedTime(&ms, e0, e1), "cudaEventElapsedTime");
            if (best_ms < 0.0f || ms < best_ms) {
              best_ms = ms;
              best = {segs, train};
            }
          }
      } catch (...) {
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        throw;
      }
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      std::lock_guard<std::mutex> g(g_window_mu);
      g_window_tuned[key] = best;
    }
    c->lte_segs = best.first;
    c->lte_train = best.second;
    if (segments) *segments = best.first;
    if (training) *training = best.second;
  });
}

int fecl_crc24_attach(const uint8_t* bits, uint64_t len, uint64_t nframes, int32_t kind, uint8_t* out, void* stream) {
  return guarded([&] {
    if (!bits || !out) fail(FECL_EINVAL, "null buffer");
    if (kind != FECL_CRC24A && kind != FECL_CRC24B) fail(FECL_EINVAL, "Invalid CRC");
    cuda_check(fecl::launch_crc24_attach(bits, int64_t(len), int64_t(nframes), kind == FECL_CRC24A ? fecl::kCrc24A : fecl::kCrc24B,
                                         out, static_cast<cudaStream_t>(stream)),
               "crc");
  });
}

int fecl_crc24_check(const uint8_t* bits, uint64_t len, uint64_t nframes, int32_t kind, int32_t* ok, void* stream) {
  return guarded([&] {
    if (!bits || !ok) fail(FECL_EINVAL, "null buffer");
    if (kind != FECL_CRC24A && kind != FECL_CRC24B) fail(FECL_EINVAL, "Invalid CRC");
    cuda_check(fecl::launch_crc24_check(bits, int64_t(len), int64_t(nframes), kind == FECL_CRC24A ? fecl::kCrc24A : fecl::kCrc24B,
                                        ok, static_cast<cudaStream_t>(stream)),
               "crc");
  });
}

int fecl_ldpc_puncturing(fecl_codec_t codec, const uint8_t* mask, uint32_t mask_len, const uint8_t* syst_mask,
                         uint32_t syst_mask_len, uint32_t* seq, uint64_t* seq_len) {
  return guarded([&] {
    auto c = checked(codec);
    if (c->kind != 0) fail(FECL_EINVAL, "not an LDPC codec");
    if (!seq_len) fail(FECL_EINVAL, "null output");
    std::vector<uint8_t> m(mask, mask + (mask ? mask_len : 0)), sm(syst_mask, syst_mask + (syst_mask ? syst_mask_len : 0));
    const auto v = fecl::ldpc_puncturing(*c->ldpc, m, sm);
    *seq_len = v.size();
    if (seq) std::memcpy(seq, v.data(), v.size() * sizeof(uint32_t));
  });
}

int fecl_turbo_puncturing(fecl_codec_t codec, const uint8_t* mask_data, const uint32_t* mask_len, uint32_t n_masks,
                          const uint8_t* tail_data, const uint32_t* tail_len, uint32_t n_tail, int32_t bit_ordering,
                          uint32_t* seq, uint64_t* seq_len) {
  return guarded([&] {
    auto c = checked(codec);
    if (c->kind != 1) fail(FECL_EINVAL, "not a turbo codec");
    if (!seq_len) fail(FECL_EINVAL, "null output");
    auto split = [](const uint8_t* data, const uint32_t* len, uint32_t n) {
      std::vector<std::vector<uint8_t>> v(n);
      size_t off = 0;
      for (uint32_t i = 0; i < n; ++i) {
        if (len[i] && !data) fail(FECL_EINVAL, "null mask data");
        v[i].assign(data + off, data + off + len[i]);
        off += len[i];
      }
      return v;
    };
    if ((n_masks && !mask_len) || (n_tail && !tail_len)) fail(FECL_EINVAL, "null mask lengths");
    const auto v = fecl::turbo_puncturing(*c->turbo, split(mask_data, mask_len, n_masks), split(tail_data, tail_len, n_tail),
                                          bit_ordering);
    *seq_len = v.size();
    if (seq) std::memcpy(seq, v.data(), v.size() * sizeof(uint32_t));
  });
}

int fecl_permutation_create(const uint32_t* seq, uint64_t output_size, uint64_t input_size, fecl_permutation_t* out) {
  return guarded([&] {
    if (!out || (output_size && !seq)) fail(FECL_EINVAL, "null argument");
    if (input_size >= 0xffffffffull) fail(FECL_EINVAL, "permutation input too large");
    std::vector<uint32_t> fwd(seq, seq + output_size), inv(input_size, 0xffffffffu);
    for (uint64_t i = 0; i < output_size; ++i) {
      if (fwd[i] >= input_size) fail(FECL_EINVAL, "permutation index out of range");
      inv[fwd[i]] = uint32_t(i);
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
      cudaGetLastError();
      fail(FECL_ENODEV, "no CUDA device is visible");
    }
    std::unique_ptr<fecl_permutation_s> p(new fecl_permutation_s);
    cuda_check(cudaGetDevice(&p->device), "cudaGetDevice");
    p->out_size = output_size;
    p->in_size = input_size;
    p->fwd.upload(fwd);
    p->inv.upload(inv);
    *out = p.release();
  });
}

int fecl_permute(fecl_permutation_t perm, const void* in, int32_t elem_type, uint64_t nblocks, void* out, int32_t inverse,
                 void* stream) {
  return guarded([&] {
    if (!perm || !in || !out) fail(FECL_EINVAL, "null argument");
    const int bytes = elem_type == FECL_U8 ? 1 : int(dsize(elem_type));
    DeviceGuard dg(perm->device);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (!inverse)
      cuda_check(fecl::launch_gather(in, out, perm->fwd.as<uint32_t>(), int64_t(perm->in_size), int64_t(perm->out_size),
                                     int64_t(nblocks), bytes, 0, s),
                 "permute");
    else
      cuda_check(fecl::launch_gather(in, out, perm->inv.as<uint32_t>(), int64_t(perm->out_size), int64_t(perm->in_size),
                                     int64_t(nblocks), bytes, 1, s),
                 "dePermute");
  });
}

void fecl_permutation_destroy(fecl_permutation_t perm) {
  if (!perm) return;
  int prev = -1;
  cudaGetDevice(&prev);
  cudaSetDevice(perm->device);
  delete perm;
  if (prev >= 0) cudaSetDevice(prev);
}

int fecl_set_kernel(fecl_codec_t codec, int32_t kernel) {
  return guarded([&] {
    auto c = checked(codec);
    if (kernel != FECL_KERNEL_AUTO && kernel != FECL_KERNEL_GENERIC && kernel != FECL_KERNEL_LANES &&
        kernel != FECL_KERNEL_CLUSTER)
      fail(FECL_EINVAL, "Invalid kernel selection");
    if ((kernel == FECL_KERNEL_LANES || kernel == FECL_KERNEL_CLUSTER) && c->kind != 0)
      fail(FECL_EINVAL, "kernel selection applies to LDPC codecs");
    std::lock_guard<std::mutex> lk(c->mu);
    c->kernel_sel = kernel;
  });
}

int fecl_ldpc_set_cluster_shape(fecl_codec_t codec, int32_t cluster, int32_t threads) {
  return guarded([&] {
    auto c = checked(codec);
    if (c->kind != 0) fail(FECL_EINVAL, "not an LDPC codec");
    if (cluster != 0 && cluster != 1 && cluster != 2 && cluster != 4 && cluster != 8 && cluster != 16)
      fail(FECL_EINVAL, "cluster size must be 1, 2, 4, 8 or 16");
    if (threads != 0 && threads != 256 && threads != 512 && threads != 1024)
      fail(FECL_EINVAL, "threads per CTA must be 256, 512 or 1024");
    std::lock_guard<std::mutex> lk(c->mu);
    c->cluster_size_sel = cluster;
    c->cluster_threads_sel = threads;
  });
}

int fecl_ldpc_set_wave(fecl_codec_t codec, int32_t groups) {
  return guarded([&] {
    auto c = checked(codec);
    if (c->kind != 0) fail(FECL_EINVAL, "not an LDPC codec");
    if (groups < 0 || groups > 65535) fail(FECL_EINVAL, "wave must be 0..65535 groups");
    std::lock_guard<std::mutex> lk(c->mu);
    c->lanes_wave = groups;
  });
}

int fecl_ldpc_set_persistent(fecl_codec_t codec, int32_t mode) {
  return guarded([&] {
    auto c = checked(codec);
    if (c->kind != 0) fail(FECL_EINVAL, "not an LDPC codec");
    if (mode < -1 || mode > 1) fail(FECL_EINVAL, "persistent mode must be -1, 0 or 1");
    std::lock_guard<std::mutex> lk(c->mu);
    c->lanes_persist = mode;
  });
}

int fecl_turbo_set_window_training(fecl_codec_t codec, int32_t steps) {
  return guarded([&] {
    auto c = checked(codec);
    if (c->kind != 1) fail(FECL_EINVAL, "not a turbo codec");
    if (steps != -1 && (steps < 0 || steps % 8 != 0 || steps > 4096)) fail(FECL_EINVAL, "training steps must be a multiple of 8");
    std::lock_guard<std::mutex> lk(c->mu);
    c->lte_train = steps;
  });
}

int fecl_turbo_set_window_segments(fecl_codec_t codec, int32_t segments) {
  return guarded([&] {
    auto c = checked(codec);
    if (c->kind != 1) fail(FECL_EINVAL, "not a turbo codec");
    if (segments != 0 && segments != 32 && segments != 64 && segments != 128)
      fail(FECL_EINVAL, "window segments must be 0, 32, 64 or 128");
    std::lock_guard<std::mutex> lk(c->mu);
    c->lte_segs = segments;
  });
}

int fecl_turbo_window_stats(fecl_codec_t codec, uint64_t* passes, uint64_t* fixup_rounds, uint64_t* recomputed) {
  return guarded([&] {
    auto c = checked(codec);
    if (c->kind != 1) fail(FECL_EINVAL, "not a turbo codec");
    std::lock_guard<std::mutex> lk(c->mu);
    unsigned long long v[3] = {0, 0, 0};
    if (c->stats.ptr) {
      DeviceGuard dg(c->device);
      if (c->pending) cuda_check(cudaEventSynchronize(c->done), "cudaEventSynchronize");
      c->sync_pipes();
      cuda_check(cudaMemcpy(v, c->stats.ptr, sizeof(v), cudaMemcpyDeviceToHost), "stats");
      cuda_check(cudaMemset(c->stats.ptr, 0, sizeof(v)), "stats");
    }
    if (passes) *passes = v[0];
    if (fixup_rounds) *fixup_rounds = v[1];
    if (recomputed) *recomputed = v[2];
  });
}

void fecl_destroy(fecl_codec_t codec) {
  if (!codec) return;
  if (!codec->on_device) {
    delete codec;
    return;
  }
  int prev = -1;
  cudaGetDevice(&prev);
  cudaSetDevice(codec->device);
  delete codec;
  if (prev >= 0) cudaSetDevice(prev);
}

}  // extern "C"
