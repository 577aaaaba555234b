// Internal state of a codec handle and the helpers the C-ABI translation units
// share (capi.cu: the codec entry points; batch.cu: mixed batches).  Not part of
// the public interface.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>
#include "../../include/fecl_b200.h"
#include "device/kernels.hpp"
#include "host/codes.hpp"
#include "host/ldpc_plan.hpp"
#include "host/puncture.hpp"

namespace fecl {
// Sets the message fecl_last_error() returns on this thread.
void set_last_error(const std::string& msg);

namespace capi {
struct Error {
  int code;
  std::string msg;
};

[[noreturn]] inline void fail(int code, const std::string& msg) { throw Error{code, msg}; }

inline void cuda_check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) {
    cudaGetLastError();
    fail(e == cudaErrorMemoryAllocation ? FECL_ENOMEM : FECL_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
  }
}


// A device allocation owned by a codec.
struct DeviceBuffer {
  void* ptr = nullptr;
  size_t bytes = 0;
  DeviceBuffer() = default;
  DeviceBuffer(const DeviceBuffer&) = delete;
  DeviceBuffer& operator=(const DeviceBuffer&) = delete;
  ~DeviceBuffer() {
    if (ptr) cudaFree(ptr);
  }
  void reserve(size_t n) {
    if (n <= bytes) return;
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    bytes = 0;
    cuda_check(cudaMalloc(&ptr, n), "cudaMalloc");
    bytes = n;
  }
  template <class T>
  void upload(const std::vector<T>& v) {
    reserve(std::max<size_t>(v.size() * sizeof(T), 16));
    if (!v.empty()) cuda_check(cudaMemcpy(ptr, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice), "upload");
  }
  template <class T>
  T* as() const {
    return static_cast<T*>(ptr);
  }
};

// Carves aligned slices out of one workspace allocation.
struct Carver {
  size_t off = 0;
  size_t take(size_t bytes) {
    size_t o = off;
    off += (bytes + 255) & ~size_t(255);
    return o;
  }
};

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    cudaGetDevice(&prev);
    if (prev != dev) cuda_check(cudaSetDevice(dev), "cudaSetDevice");
  }
  ~DeviceGuard() {
    int cur = -1;
    cudaGetDevice(&cur);
    if (prev >= 0 && cur != prev) cudaSetDevice(prev);
  }
};

inline size_t dsize(int dtype) {
  switch (dtype) {
    case FECL_F64: return 8;
    case FECL_F32: return 4;
    case FECL_F16: return 2;
  }
  fail(FECL_EINVAL, "Invalid element type");
}

}  // namespace capi
}  // namespace fecl

using namespace fecl::capi;

struct fecl_codec_s {
  int kind = 0;  // 0 LDPC, 1 turbo
  int device = 0;
  std::unique_ptr<fecl::LdpcCode> ldpc;
  std::unique_ptr<fecl::TurboCode> turbo;
  std::unique_ptr<fecl::ConvCode> conv;  // kind 2
  fecl::TurboDeviceConstituent cdev{};   // the convolutional trellis on the device
  std::mutex mu;
  static constexpr int kPipe = 4, kMaxChunks = 8;
  cudaStream_t pipe[kPipe] = {};          // host-memory calls: decode and copy-out streams
  cudaStream_t copy_in = nullptr;         // host-memory calls: every chunk's copy in, in order
  cudaEvent_t arrived[kMaxChunks] = {};   // chunk k's inputs are on the device
  cudaEvent_t done = nullptr;
  bool pending = false;
  // device description
  DeviceBuffer row_ptr, col_idx, col_ptr, col_edges, sf;
  std::vector<std::unique_ptr<DeviceBuffer>> tables;
  fecl::LdpcDeviceCode ldev;
  DeviceBuffer sched[4];  // custom turbo schedule (stage_ptr, act_con, act_tptr, transfer)
  DeviceBuffer crc_tab;   // CRC syndrome table of the turbo decoder's CRC stop
  // The CRC stop's syndrome table on the device, or null when the decoder has none.
  const uint32_t* crc_table() const { return (kind == 1 && turbo->decoder().crc) ? crc_tab.as<uint32_t>() : nullptr; }
  DeviceBuffer enc[8];  // LDPC generator pieces (DC, A, B, T as CSR) for the device encoder
  fecl::LdpcEncodeTables ltab;
  fecl::TurboDeviceCode tdev;
  // workspace
  DeviceBuffer ws;

  ~fecl_codec_s() {
    for (cudaStream_t st : pipe)
      if (st) {
        cudaStreamSynchronize(st);
        cudaStreamDestroy(st);
      }
    if (copy_in) {
      cudaStreamSynchronize(copy_in);
      cudaStreamDestroy(copy_in);
    }
    for (cudaEvent_t e : arrived)
      if (e) cudaEventDestroy(e);
    if (done) cudaEventDestroy(done);
  }

  // Waits for every host-memory pipeline stream.
  void sync_pipes() const {
    for (cudaStream_t st : pipe) cuda_check(cudaStreamSynchronize(st), "cudaStreamSynchronize");
    cuda_check(cudaStreamSynchronize(copy_in), "cudaStreamSynchronize");
  }

  uint64_t msg() const { return kind == 0 ? ldpc->msg_size() : kind == 1 ? turbo->msg_size() : conv->msg_size(); }
  uint64_t syst() const { return kind == 0 ? ldpc->syst_size() : kind == 1 ? turbo->syst_size() : conv->syst_size(); }
  uint64_t parity() const { return kind == 0 ? ldpc->parity_size() : kind == 1 ? turbo->parity_size() : conv->parity_size(); }
  uint64_t state() const { return kind == 0 ? ldpc->state_size() : kind == 1 ? turbo->state_size() : 0; }

  void init_runtime() {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
      cudaGetLastError();
      fail(FECL_ENODEV, "no CUDA device is visible");
    }
    cuda_check(cudaGetDevice(&device), "cudaGetDevice");
    for (cudaStream_t& st : pipe) cuda_check(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "cudaStreamCreate");
    cuda_check(cudaStreamCreateWithFlags(&copy_in, cudaStreamNonBlocking), "cudaStreamCreate");
    for (cudaEvent_t& e : arrived) cuda_check(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "cudaEventCreate");
    cuda_check(cudaEventCreateWithFlags(&done, cudaEventDisableTiming), "cudaEventCreate");
    cuda_check(cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device), "attribute");
    cuda_check(cudaDeviceGetAttribute(&sm_count, cudaDevAttrMultiProcessorCount, device), "attribute");
  }

  void upload_ldpc() {
    const fecl::Csr& H = ldpc->checks();
    row_ptr.upload(H.row_ptr);
    col_idx.upload(H.col_idx);
    // per-bit edge lists in increasing edge order
    std::vector<uint32_t> cp(H.cols + 1, 0), ce(H.nnz());
    for (auto c : H.col_idx) cp[c + 1]++;
    for (uint32_t b = 0; b < H.cols; ++b) cp[b + 1] += cp[b];
    std::vector<uint32_t> fill(cp.begin(), cp.end() - 1);
    for (uint64_t e = 0; e < H.nnz(); ++e) ce[fill[H.col_idx[e]]++] = uint32_t(e);
    col_ptr.upload(cp);
    col_edges.upload(ce);
    ldev.M = int32_t(H.rows);
    ldev.N = int32_t(H.cols);
    ldev.E = int64_t(H.nnz());
    ldev.msg = int32_t(ldpc->msg_size());
    ldev.d_max = int32_t(ldpc->max_check_degree());
    ldev.row_ptr = row_ptr.as<uint32_t>();
    ldev.col_idx = col_idx.as<uint32_t>();
    ldev.col_ptr = col_ptr.as<uint32_t>();
    ldev.col_edges = col_edges.as<uint32_t>();
    const fecl::Csr* parts[4] = {&ldpc->gen_dc(), &ldpc->gen_a(), &ldpc->gen_b(), &ldpc->gen_t()};
    for (int i = 0; i < 4; ++i) {
      enc[2 * i].upload(parts[i]->row_ptr);
      enc[2 * i + 1].upload(parts[i]->col_idx);
    }
    ltab.K = int32_t(ldpc->msg_size());
    ltab.N = int32_t(H.cols);
    ltab.gap = int32_t(ldpc->gen_dc().rows);
    ltab.dc_rows = int32_t(ldpc->gen_dc().rows);
    ltab.a_rows = int32_t(ldpc->gen_a().rows);
    ltab.b_rows = int32_t(ldpc->gen_b().rows);
    ltab.t_rows = int32_t(ldpc->gen_t().rows);
    ltab.dc_ptr = enc[0].as<uint32_t>();
    ltab.dc_idx = enc[1].as<uint32_t>();
    ltab.a_ptr = enc[2].as<uint32_t>();
    ltab.a_idx = enc[3].as<uint32_t>();
    ltab.b_ptr = enc[4].as<uint32_t>();
    ltab.b_idx = enc[5].as<uint32_t>();
    ltab.t_ptr = enc[6].as<uint32_t>();
    ltab.t_idx = enc[7].as<uint32_t>();
    upload_ldpc_options();
  }

  void upload_ldpc_options() {
    const auto& d = ldpc->decoder();
    const int stride = int(ldpc->max_check_degree()) - 1;
    std::vector<float> t;
    for (auto& row : d.scaling)
      for (int k = 0; k < stride; ++k) t.push_back(float(row[k]));
    sf.upload(t);
    ldev.sf = sf.as<float>();
    ldev.n_sf = int32_t(d.scaling.size());
    ldev.sf_stride = stride;
    ldev.algorithm = d.algorithm;
    ldev.iterations = int32_t(d.iterations);
    ldev.fixed_iterations = d.fixed_iterations;
  }

  void upload_turbo() {
    const auto& cs = turbo->constituents();
    if (cs.size() > size_t(fecl::kMaxConstituents)) fail(FECL_EUNSUPPORTED, "too many constituents for the device decoder");
    tables.clear();
    tdev.n = int32_t(cs.size());
    tdev.msg = int32_t(turbo->msg_size());
    tdev.syst = int32_t(turbo->syst_size());
    tdev.parity = int32_t(turbo->parity_size());
    tdev.state = int32_t(turbo->state_size());
    tdev.tail = int32_t(turbo->syst_tail_size());
    tdev.max_steps = 0;
    tdev.max_states = 0;
    for (size_t j = 0; j < cs.size(); ++j) {
      const auto& c = cs[j];
      auto& k = tdev.c[j];
      k.state_count = int32_t(c.trellis.state_count);
      k.input_count = int32_t(c.trellis.input_count);
      k.input_size = int32_t(c.trellis.input_size);
      k.output_size = int32_t(c.trellis.output_size);
      k.length = int32_t(c.length);
      k.tail = int32_t(c.tail);
      k.termination = c.termination;
      k.msg_size = int32_t(c.msg_size());
      k.syst_size = int32_t(c.syst_size());
      k.syst_tail_size = int32_t(c.syst_tail_size());
      k.parity_size = int32_t(c.parity_size());
      // interleavers are padded with zeros so that 8-entry vector loads never leave them
      std::vector<uint32_t> padded_perm(c.perm);
      padded_perm.resize(c.perm.size() + 16, 0);
      for (const std::vector<uint32_t>* v : {&c.trellis.next_state, &c.trellis.output,
                                             static_cast<const std::vector<uint32_t>*>(&padded_perm)}) {
        tables.emplace_back(new DeviceBuffer);
        tables.back()->upload(*v);
      }
      k.next_state = tables[tables.size() - 3]->as<uint32_t>();
      k.output = tables[tables.size() - 2]->as<uint32_t>();
      k.perm = tables[tables.size() - 1]->as<uint32_t>();
      tdev.max_steps = std::max(tdev.max_steps, int32_t(c.length + c.tail));
      tdev.max_states = std::max(tdev.max_states, int32_t(c.trellis.state_count));
    }
    upload_turbo_options();
  }

  void upload_conv() {
    const fecl::Constituent& c = conv->constituent();
    if (c.trellis.state_count > 64 || c.trellis.input_count > 4 || c.trellis.output_size > 6)
      fail(FECL_EUNSUPPORTED, "trellis too large for the device decoder");
    tables.clear();
    std::vector<uint32_t> padded_perm(c.perm);
    padded_perm.resize(c.perm.size() + 16, 0);
    for (const std::vector<uint32_t>* v : {&c.trellis.next_state, &c.trellis.output,
                                           static_cast<const std::vector<uint32_t>*>(&padded_perm)}) {
      tables.emplace_back(new DeviceBuffer);
      tables.back()->upload(*v);
    }
    cdev.state_count = int32_t(c.trellis.state_count);
    cdev.input_count = int32_t(c.trellis.input_count);
    cdev.input_size = int32_t(c.trellis.input_size);
    cdev.output_size = int32_t(c.trellis.output_size);
    cdev.length = int32_t(c.length);
    cdev.tail = int32_t(c.tail);
    cdev.termination = c.termination;
    cdev.msg_size = int32_t(c.msg_size());
    cdev.syst_size = int32_t(c.syst_size());
    cdev.syst_tail_size = int32_t(c.syst_tail_size());
    cdev.parity_size = int32_t(c.parity_size());
    cdev.next_state = tables[0]->as<uint32_t>();
    cdev.output = tables[1]->as<uint32_t>();
    cdev.perm = tables[2]->as<uint32_t>();
  }

  void upload_turbo_options() {
    const auto& d = turbo->decoder();
    std::vector<float> t;
    for (size_t j = 0; j < turbo->constituents().size(); ++j)
      for (uint32_t i = 0; i < std::max<uint32_t>(d.iterations, 1); ++i) t.push_back(float(turbo->scaling_factor(i, j)));
    sf.upload(t);
    tdev.sf = sf.as<float>();
    tdev.algorithm = d.algorithm;
    tdev.iterations = int32_t(d.iterations);
    tdev.scheduling = d.scheduling;
    std::vector<int32_t> sp{0}, ac, ap{0}, tr;
    for (const auto& st : d.schedule) {
      for (size_t k = 0; k < st.activation.size(); ++k) {
        ac.push_back(int32_t(st.activation[k]));
        for (auto v : st.transfer[k]) tr.push_back(int32_t(v));
        ap.push_back(int32_t(tr.size()));
      }
      sp.push_back(int32_t(ac.size()));
    }
    sched[0].upload(sp);
    sched[1].upload(ac);
    sched[2].upload(ap);
    sched[3].upload(tr);
    if (d.crc) crc_tab.upload(fecl::crc24_syndrome_table(turbo->msg_size(), d.crc == 1 ? fecl::kCrc24A : fecl::kCrc24B));
    tdev.n_stages = int32_t(d.schedule.size());
    tdev.stage_ptr = sched[0].as<int32_t>();
    tdev.act_con = sched[1].as<int32_t>();
    tdev.act_tptr = sched[2].as<int32_t>();
    tdev.transfer = sched[3].as<int32_t>();
  }

  bool on_device = false;
  std::atomic<uint64_t> generation{0};  // bumped whenever the decoder options (and their device tables) change
  int lte_train = -1;
  int lte_segs = 0;  // windowed LTE decoder: segments per direction (0: built-in choice)
  int kernel_sel = FECL_KERNEL_AUTO;
  bool force_generic_() const { return kernel_sel == FECL_KERNEL_GENERIC; }

  // Cluster-resident LDPC decoder: partition tables per cluster size, uploaded on use.
  struct ClusterDev {
    fecl::LdpcClusterPlan plan;
    bool uploaded = false;
    DeviceBuffer row_split, bit_split, chk_addr, bit_ptr, bit_addr;
    std::map<int, int> max_active;  // threads -> resident clusters
  };
  std::map<uint32_t, std::unique_ptr<ClusterDev>> cplans;
  int cluster_size_sel = 0, cluster_threads_sel = 0;  // 0: chosen by the heuristic
  int lanes_wave = 0;                                 // 0: chosen by the launcher
  int lanes_persist = 0;                              // persistent launch: 1 where it applies, 0 / -1 never
  int smem_optin = 0, sm_count = 0;

  ClusterDev& cluster_plan(uint32_t C) {
    auto& slot = cplans[C];
    if (!slot) {
      slot.reset(new ClusterDev);
      slot->plan = fecl::build_ldpc_cluster_plan(ldpc->checks(), C);
    }
    return *slot;
  }
  size_t cluster_smem(uint32_t C) {
    auto& d = cluster_plan(C);
    return fecl::ldpc_cluster_smem_bytes(int64_t(d.plan.max_edges), int64_t(d.plan.max_bits), ldpc->decoder().precision);
  }
  // Shape of the cluster decoder for a batch of n frames: the cluster size and the
  // threads per CTA, or false when the code's messages do not fit a cluster.  The
  // smallest cluster whose shares fit in shared memory is doubled while the batch
  // would leave more than half of the SMs idle (up to 8 CTAs).
  bool ldpc_cluster_shape(uint64_t n, uint32_t* C_out, int* threads_out) {
    if (kind != 0 || kernel_sel == FECL_KERNEL_GENERIC || kernel_sel == FECL_KERNEL_LANES) return false;
    if (ldpc->max_check_degree() > 32) return false;
    const size_t limit = size_t(smem_optin) - 1024;  // static shared memory of the kernel
    uint32_t C = 0;
    for (uint32_t c = 1; c <= 16; c *= 2) {
      if (cluster_size_sel && c != uint32_t(cluster_size_sel)) continue;
      try {
        if (cluster_smem(c) <= limit) {
          C = c;
          break;
        }
      } catch (const std::invalid_argument&) {
        return false;
      }
    }
    if (C == 0) return false;
    if (!cluster_size_sel)
      while (C < 8 && n * C * 2 <= uint64_t(sm_count) && cluster_smem(C * 2) <= limit) C *= 2;
    int threads = cluster_threads_sel;
    if (!threads) threads = ldpc->max_check_degree() <= 16 ? 1024 : 512;
    if ((threads == 1024 && ldpc->max_check_degree() > 16) || (threads == 256 && ldpc->max_check_degree() <= 16))
      threads = 512;
    *C_out = C;
    *threads_out = threads;
    return true;
  }
  void upload_cluster(ClusterDev& d) {
    if (d.uploaded) return;
    d.row_split.upload(d.plan.row_split);
    d.bit_split.upload(d.plan.bit_split);
    d.chk_addr.upload(d.plan.chk_addr);
    d.bit_ptr.upload(d.plan.bit_ptr);
    d.bit_addr.upload(d.plan.bit_addr);
    d.uploaded = true;
  }
  DeviceBuffer stats;  // windowed turbo counters
  // The lane-batched LDPC kernel needs check degrees <= 32 and, unless the iteration
  // count is fixed, a scaling that does not change across iterations (its stop test
  // runs inside the check update of the next iteration).
  bool ldpc_lanes_ok() const {
    if (kind != 0 || force_generic_()) return false;
    if (ldpc->max_check_degree() > 32) return false;
    const auto& d = ldpc->decoder();
    if (d.fixed_iterations) return true;
    for (const auto& row : d.scaling)
      if (row != d.scaling[0]) return false;
    return true;
  }
  // FP16 normalised min-sum goes to the packed two-frames-per-lane kernel unless a
  // kernel is forced (FECL_KERNEL_LANES keeps FP32 check-node arithmetic).
  bool ldpc_h2_ok() const {
    if (kind != 0 || kernel_sel != FECL_KERNEL_AUTO || !ldpc_lanes_ok()) return false;
    const auto& d = ldpc->decoder();
    return d.precision == 1 && d.algorithm == 2;
  }
  // The windowed kernel covers the LTE RSC pair with serial scheduling and FP32 messages
  // for any K whose two exchange arrays fit in shared memory.
  bool lte_fast_ok() const {
    if (force_generic_() || kind != 1 || !turbo->is_lte_shape()) return false;
    const auto& d = turbo->decoder();
    if (d.scheduling > 1 || d.precision != 0 || d.iterations == 0) return false;
    static const fecl::Trellis lte = fecl::lte_trellis();
    for (const auto& c : turbo->constituents())
      if (c.trellis.next_state != lte.next_state || c.trellis.output != lte.output) return false;
    return turbo->msg_size() <= 12288;
  }
  // The mixed-K batch kernel (batches and the server): serial scheduling only.
  bool lte_batch_ok() const { return lte_fast_ok() && turbo->decoder().scheduling == 0; }
  // Device resources are created at the first decode, so that host-side operations
  // (encode, check, the transformed matrix) work without a GPU.
  void ensure_device() {
    if (on_device) return;
    init_runtime();
    if (kind == 0) upload_ldpc();
    else if (kind == 1) upload_turbo();
    else upload_conv();
    on_device = true;
  }

  // Orders this call after the previous device-memory call on the codec.
  void wait_previous(cudaStream_t s) {
    if (pending) cuda_check(cudaStreamWaitEvent(s, done, 0), "cudaStreamWaitEvent");
  }
  void mark(cudaStream_t s) {
    cuda_check(cudaEventRecord(done, s), "cudaEventRecord");
    pending = true;
  }
};

// A permutation on the device: the gather map and its last-writer inverse.
struct fecl_permutation_s {
  int device = 0;
  uint64_t out_size = 0, in_size = 0;
  DeviceBuffer fwd, inv;
};

namespace fecl {
namespace capi {

// Device pointers of one decode launch (inputs, outputs, scratch).
struct Launch {
  const void *llr = nullptr, *syst = nullptr, *state = nullptr;
  uint8_t* hard = nullptr;
  int32_t* iters = nullptr;
  void *msg = nullptr, *syst_out = nullptr, *parity_out = nullptr, *state_out = nullptr;
  char* scratch = nullptr;
};

// Scratch of the decoder kernels for n frames, with the offsets of its parts.
struct ScratchPlan {
  size_t bytes = 0, o1 = 0, o2 = 0, o3 = 0, o4 = 0, o5 = 0;
  uint32_t cluster = 0;  // > 0: the cluster-resident LDPC decoder with this many CTAs per frame
  int threads = 0, clusters = 0;
};

// The kernel and scratch for a batch of n frames of codec c (lte_fast: the windowed
// LTE turbo kernel applies).
ScratchPlan plan_scratch(fecl_codec_s* c, uint64_t n, bool lte_fast, bool soft = false);
// The lane-batched LDPC decoder's parameters for n frames of codec c (pointers in d
// are device memory); the launcher fills the scratch layout.
fecl::LdpcLanesParams lanes_params(fecl_codec_s* c, const Launch& d, uint64_t n, int32_t in_dtype, int32_t out_dtype);
// Launches the decode of n frames on stream s; pointers in d are device memory.
void launch_decode(fecl_codec_s* c, const Launch& d, const ScratchPlan& sp, uint64_t n, int32_t in_dtype,
                   int32_t out_dtype, bool soft, bool lte_fast, cudaStream_t s);

}  // namespace capi
}  // namespace fecl
