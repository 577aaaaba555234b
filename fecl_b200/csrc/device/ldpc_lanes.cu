// LDPC flooding belief propagation for batches: 32 frames per warp, one frame per
// lane.
//
// Same decoder as ldpc_flood.cu (BpDecoderImpl, src/detail/BpDecoder/BpDecoderImpl.cpp:37-179),
// laid out for streaming instead of one CTA per frame.  Frames are grouped by 32;
// within a group every per-bit and per-edge array is stored lane-minor,
//     chan[g][n][32], app[g][n][32] (FP32), c2v[g][e][32] (FP32, FP16 or int8),
// so when a warp works on one check row (or one bit) for its 32 frames, every load
// and store is one contiguous 128-byte (or 64- / 32-byte) line, and the column
// indices are the same for all lanes.  Each iteration is two launches:
//   check: warp per (group, row): v = app - c2v, the reference's forward/backward
//          boxplus order (min-sum, whose chain is exact, as two minima and a sign
//          parity), scaled c2v out; for iteration >= 1 it also folds the row's
//          syndrome bit of the previous APP into a per-group failure mask (ballot +
//          one atomicOr), which is the reference's stop test (:53-59);
//   bit:   warp per (group, bit): app = chan + sum c2v in edge order; one block per
//          group retires the frames whose syndrome held (their lanes are masked from
//          then on) and records their iteration counts.
// Groups are decoded in waves whose working set (chan, app, c2v) fits in L2: every
// iteration of a wave runs before the next wave starts, so the messages of a wave
// stay on chip and HBM sees each group's data about once per decode.
// A frame that stops at iteration i has had exactly the reference's sequence: its
// last check update ran with the scaling of iteration i, which equals that of
// iteration I-1 because this kernel is used only when the scaling does not change
// across iterations (or with fixed iterations).
//
// Messages may be stored in FP16 or in saturated int8 (Q5.2, step 1/4, +-31.75);
// every sum and every boxplus runs in FP32.
#include <cuda_fp16.h>
#include <math.h>

#include <mutex>

#include "common.cuh"
#include "grid_sync.cuh"
#include "kernels.hpp"
#include "ldpc_math.cuh"

namespace fecl {
namespace {

using ldpc::kApproximate;
using ldpc::kExact;
using ldpc::kLinear;
using ldpc::Msg;
constexpr int kLanes = 32;
constexpr int kWarpsPerBlock = 8;

__constant__ LinearLut c_lut;
// The Linear table copied to shared memory by the check kernels: the lanes of a warp
// (different frames) look up different entries, which constant memory serves one
// address at a time and shared memory (eight words in eight banks) at once.
__shared__ LinearLut s_lut;

__device__ __forceinline__ void share_lut() {
  if (threadIdx.x < 8) s_lut.y[threadIdx.x] = c_lut.y[threadIdx.x];
  __syncthreads();
}

__device__ __forceinline__ int lane_id() { return threadIdx.x & 31; }

// Lane masks of a group at iteration `it`: active[it & 1][g] holds the frames still
// decoding, fail[it & 1][g] collects the rows whose syndrome bit is set.  The bit pass
// of iteration it retires frames and writes the masks of iteration it + 1, so a
// kernel never reads a mask that the same launch writes.
__device__ __forceinline__ uint32_t* active_of(const LdpcLanesParams& p, int it) { return p.active + (it & 1) * p.groups; }
__device__ __forceinline__ uint32_t* fail_of(const LdpcLanesParams& p, int it) { return p.fail + (it & 1) * p.groups; }

// One check row r of group g for this lane's frame: loads of v, the row update, the
// stores of c2v for active lanes; returns the row's parity of the hard decision.
template <int ALG, int MSG, int DMAX>
__device__ __forceinline__ void load_row(const LdpcLanesParams& p, int g, int r, int lane, uint32_t& e0, int& d,
                                         float v[DMAX], unsigned& parity) {
  using M = Msg<MSG>;
  const auto* c2v = static_cast<const typename M::T*>(p.c2v);
  e0 = __ldg(p.row_ptr + r);
  d = int(__ldg(p.row_ptr + r + 1) - e0);
  const typename M::T* cg = c2v + (int64_t(g) * p.E + e0) * kLanes + lane;
  const float* ag = p.app + int64_t(g) * p.N * kLanes + lane;
  parity = 0;
#pragma unroll
  for (int j = 0; j < DMAX; ++j) {
    if (j < d) {
      const uint32_t col = __ldg(p.col_idx + e0 + j);
      const float a = ag[int64_t(col) * kLanes];
      parity ^= unsigned(a >= 0.0f);
      v[j] = a - M::load(cg + j * kLanes);
    }
  }
}

template <int ALG, int MSG, int DMAX>
__device__ __forceinline__ void store_row(const LdpcLanesParams& p, int g, uint32_t e0, int d, int lane, const float* sf_row,
                                          const float v[DMAX], bool mine) {
  using M = Msg<MSG>;
  auto* c2v = static_cast<typename M::T*>(p.c2v);
  if (ALG == kApproximate) {
    // Min-sum: each output is sf * (+-m1) or sf * (+-m2).  The product and the storage
    // encoding are odd in the sign, so the two magnitudes are scaled and encoded once
    // per row and every edge selects one and negates it: the same stored values as
    // encoding sf * (+-m) edge by edge.
    float m1, m2;
    int i1;
    unsigned par;
    ldpc::min_sum_scan<DMAX>(v, d, m1, m2, i1, par);
    const float sf = sf_row[d >= 2 ? d - 2 : 0];
    const typename M::T q1 = M::encode(sf * m1), q2 = M::encode(sf * m2);
    // d - 1 inputs: the result's sign bit is (d - 2) xor the parity of the others' sign bits.
    const unsigned base = unsigned((d - 2) & 1) ^ par;
    if (mine) {
      typename M::T* cg = c2v + (int64_t(g) * p.E + e0) * kLanes + lane;
#pragma unroll
      for (int j = 0; j < DMAX; ++j) {
        if (j < d) {
          const typename M::T q = (j == i1) ? q2 : q1;
          cg[j * kLanes] = (base ^ unsigned(ldpc::neg(v[j]))) ? M::negate(q) : q;
        }
      }
    }
    return;
  }
  float out[DMAX];
  ldpc::row_update<ALG, DMAX>(s_lut, v, out, d, sf_row[d >= 2 ? d - 2 : 0]);
  if (mine) {
    typename M::T* cg = c2v + (int64_t(g) * p.E + e0) * kLanes + lane;
#pragma unroll
    for (int j = 0; j < DMAX; ++j)
      if (j < d) M::store(cg + j * kLanes, out[j]);
  }
}

// Rows r .. r + kRows - 1 (kRows = 2 for short rows, so that twice the loads are in
// flight) of group g at iteration `it`: the row updates, stored for the lanes in
// `mine`; returns the ballot of lanes whose syndrome bit of one of these rows is set.
template <int ALG, int MSG, int DMAX>
__device__ __forceinline__ uint32_t check_rows(const LdpcLanesParams& p, int g, int r, int lane, bool mine,
                                               bool check_syndrome, const float* sf_row) {
  constexpr int kRows = DMAX <= 8 ? 2 : 1;
  float v[kRows][DMAX];
  uint32_t e0[kRows];
  int d[kRows];
  unsigned parity[kRows];
  uint32_t bad = 0;
#pragma unroll
  for (int q = 0; q < kRows; ++q) {
    d[q] = 0;
    parity[q] = 0;
    if (r + q < p.M) load_row<ALG, MSG, DMAX>(p, g, r + q, lane, e0[q], d[q], v[q], parity[q]);
  }
#pragma unroll
  for (int q = 0; q < kRows; ++q) {
    if (d[q] > 0) {
      if (check_syndrome) bad |= __ballot_sync(0xffffffffu, parity[q] != 0);
      store_row<ALG, MSG, DMAX>(p, g, e0[q], d[q], lane, sf_row, v[q], mine);
    }
  }
  return bad;
}

// Check pass of iteration `it` over groups [g0, g0 + gridDim.y): a warp per row (or
// row pair).
template <int ALG, int MSG, int DMAX>
__global__ void __launch_bounds__(kWarpsPerBlock * 32) lanes_check(LdpcLanesParams p, int it, int g0) {
  pdl_enter();
  constexpr int kRows = DMAX <= 8 ? 2 : 1;
  const int lane = lane_id();
  const int warps = int(gridDim.x) * kWarpsPerBlock;
  const bool check_syndrome = it > 0 && !p.fixed_iterations;
  const float* sf_row = p.sf + size_t(it % p.n_sf) * p.sf_stride;
  const int g = g0 + int(blockIdx.y);
  const uint32_t active = active_of(p, it)[g];
  if (active == 0) return;  // the same for the whole block (one group per grid row)
  if constexpr (ALG == kLinear) share_lut();
  const bool mine = (active >> lane) & 1;
  uint32_t bad = 0;
  const int w0 = int(blockIdx.x) * kWarpsPerBlock + (threadIdx.x >> 5);
  for (int r = w0 * kRows; r < p.M; r += warps * kRows)
    bad |= check_rows<ALG, MSG, DMAX>(p, g, r, lane, mine, check_syndrome, sf_row);
  bad &= active;
  if (bad && lane == 0) atomicOr(fail_of(p, it) + g, bad);
}

// Retirement of group g after the check pass of iteration `it`: the frames whose
// syndrome held, or all of them at the last iteration, record their iteration count
// and leave the active mask of iteration it + 1.
__device__ __forceinline__ void retire_group(const LdpcLanesParams& p, int it, int g, uint32_t active) {
  uint32_t done = 0;
  if (it == p.iterations - 1) done = active;
  else if (it > 0 && !p.fixed_iterations) done = active & ~fail_of(p, it)[g];
  for (uint32_t m = done; m; m &= m - 1) p.iters_ws[int64_t(g) * kLanes + (__ffs(m) - 1)] = it + 1;
  active_of(p, it + 1)[g] = active & ~done;
  fail_of(p, it + 1)[g] = 0;
}

// app = chan + sum of c2v over bit b's edges, in increasing edge order, for this lane.
// The edges go in runs of 8 (one run for most bits): every edge id of a run is loaded,
// then every message, then they are added in order, so a bit costs three dependent
// loads rather than two per edge.
template <int MSG>
__device__ __forceinline__ void bit_one(const LdpcLanesParams& p, int g, int b, int lane) {
  using M = Msg<MSG>;
  constexpr uint32_t kRun = 8;
  const typename M::T* cg = static_cast<const typename M::T*>(p.c2v) + int64_t(g) * p.E * kLanes + lane;
  const int64_t base = (int64_t(g) * p.N + b) * kLanes + lane;
  const uint32_t k0 = __ldg(p.col_ptr + b), k1 = __ldg(p.col_ptr + b + 1);
  float acc = p.chan[base];
  for (uint32_t k = k0; k < k1; k += kRun) {
    uint32_t e[kRun];
    float x[kRun];
#pragma unroll
    for (uint32_t j = 0; j < kRun; ++j) e[j] = k + j < k1 ? __ldg(p.col_edges + k + j) : 0u;
#pragma unroll
    for (uint32_t j = 0; j < kRun; ++j) x[j] = k + j < k1 ? M::load(cg + int64_t(e[j]) * kLanes) : 0.0f;
#pragma unroll
    for (uint32_t j = 0; j < kRun; ++j)
      if (k + j < k1) acc += x[j];
  }
  p.app[base] = acc;
}

// Bit pass of iteration `it` (or, with it < 0, the initial APP from chan and the
// staged c2v for every lane).  Block (0, y) of each group retires its frames and
// writes the group's masks for iteration it + 1.
template <int MSG>
__global__ void __launch_bounds__(kWarpsPerBlock * 32) lanes_bit(LdpcLanesParams p, int it, int g0) {
  pdl_enter();
  const int lane = lane_id();
  const int warps = int(gridDim.x) * kWarpsPerBlock;
  const int g = g0 + int(blockIdx.y);
  const uint32_t active = it < 0 ? 0xffffffffu : active_of(p, it)[g];
  if (it >= 0 && blockIdx.x == 0 && threadIdx.x == 0) retire_group(p, it, g, active);
  if (!((active >> lane) & 1)) return;
  for (int b = int(blockIdx.x) * kWarpsPerBlock + (threadIdx.x >> 5); b < p.N; b += warps) bit_one<MSG>(p, g, b, lane);
}

// Persistent decoder for a small batch (at most kPersistGroups groups, all in one wave):
// one launch runs the initial APP and every iteration, the check and bit passes of
// all groups spread over the whole grid and separated by grid barriers, so a decode of
// a few frame groups costs one launch instead of two per iteration.  It computes
// exactly the rows, bits and retirements of lanes_check / lanes_bit.  A barrier that
// gives up marks every frame's iteration count -1 (not decoded).
constexpr int kPersistGroups = 16;

template <int ALG, int MSG, int DMAX>
__global__ void __launch_bounds__(kWarpsPerBlock * 32) lanes_persist(LdpcLanesParams p) {
  constexpr int kRows = DMAX <= 8 ? 2 : 1;
  __shared__ uint32_t s_bad[kPersistGroups];
  const int lane = lane_id();
  const int warp = int(blockIdx.x) * kWarpsPerBlock + (threadIdx.x >> 5);
  const int warps = int(gridDim.x) * kWarpsPerBlock;
  const int ng = p.groups;
  unsigned epoch = 0;
  if constexpr (ALG == kLinear) share_lut();
  for (int64_t u = warp; u < int64_t(ng) * p.N; u += warps) bit_one<MSG>(p, int(u / p.N), int(u % p.N), lane);
  bool ok = grid_barrier(p.barrier, p.barrier + 1, epoch);
  const int rows = (p.M + kRows - 1) / kRows;
  for (int it = 0; ok && it < p.iterations; ++it) {
    const bool check_syndrome = it > 0 && !p.fixed_iterations;
    const float* sf_row = p.sf + size_t(it % p.n_sf) * p.sf_stride;
    if (threadIdx.x < kPersistGroups) s_bad[threadIdx.x] = 0;
    __syncthreads();
    // check pass: units (group, row pair) group-major; a warp's bad lanes ORed per group
    int g_cur = -1;
    uint32_t bad = 0, active = 0;
    for (int64_t u = warp; u < int64_t(ng) * rows; u += warps) {
      const int g = int(u / rows);
      if (g != g_cur) {
        if (bad && lane == 0) atomicOr(&s_bad[g_cur], bad & active);
        g_cur = g;
        bad = 0;
        active = active_of(p, it)[g];
      }
      if (active == 0) continue;
      bad |= check_rows<ALG, MSG, DMAX>(p, g, int(u % rows) * kRows, lane, (active >> lane) & 1, check_syndrome, sf_row);
    }
    if (bad && lane == 0) atomicOr(&s_bad[g_cur], bad & active);
    __syncthreads();
    if (threadIdx.x < ng && s_bad[threadIdx.x]) atomicOr(fail_of(p, it) + threadIdx.x, s_bad[threadIdx.x]);
    if (!(ok = grid_barrier(p.barrier, p.barrier + 1, epoch))) break;
    // bit pass, and block 0 retires the frames
    if (blockIdx.x == 0 && threadIdx.x < ng) retire_group(p, it, threadIdx.x, active_of(p, it)[threadIdx.x]);
    g_cur = -1;
    for (int64_t u = warp; u < int64_t(ng) * p.N; u += warps) {
      const int g = int(u / p.N);
      if (g != g_cur) {
        g_cur = g;
        active = active_of(p, it)[g];
      }
      if ((active >> lane) & 1) bit_one<MSG>(p, g, int(u % p.N), lane);
    }
    if (!(ok = grid_barrier(p.barrier, p.barrier + 1, epoch))) break;
    uint32_t left = 0;
    for (int g = 0; g < ng; ++g) left |= active_of(p, it + 1)[g];
    if (left == 0) break;
  }
  if (!ok && blockIdx.x == 0)
    for (int i = threadIdx.x; i < ng * kLanes; i += blockDim.x) p.iters_ws[i] = -1;
}

// Frame-major inputs -> lane-minor scratch for group blockIdx.y: chan (+ a-priori on
// systematic bits), c2v (state or zero), lane masks.
template <int MSG>
__global__ void lanes_stage(LdpcLanesParams p) {
  using M = Msg<MSG>;
  auto* c2v = static_cast<typename M::T*>(p.c2v);
  const int g = int(blockIdx.y);
  const int stride = int(gridDim.x) * blockDim.x;
  const int t0 = int(blockIdx.x) * blockDim.x + threadIdx.x;
  for (int i = t0; i < p.N * kLanes; i += stride) {
    const int lane = i % kLanes, b = i / kLanes;
    const int64_t f = int64_t(g) * kLanes + lane;
    float x = 0.0f;
    if (f < p.nframes) {
      x = load_llr(p.llr, p.llr_dtype, f * p.N + b);
      if (p.syst_in && b < p.msg) x += load_llr(p.syst_in, p.llr_dtype, f * p.msg + b);
    }
    p.chan[int64_t(g) * p.N * kLanes + i] = x;
  }
  for (int64_t i = t0; i < p.E * kLanes; i += stride) {
    const int lane = int(i % kLanes);
    const int64_t e = i / kLanes;
    const int64_t f = int64_t(g) * kLanes + lane;
    float v = 0.0f;
    if (p.state_in && f < p.nframes) v = load_llr(p.state_in, p.llr_dtype, f * p.E + e);
    M::store(c2v + int64_t(g) * p.E * kLanes + i, v);
  }
  if (t0 == 0) {
    const int64_t left = p.nframes - int64_t(g) * kLanes;
    p.active[g] = left >= kLanes ? 0xffffffffu : ((1u << left) - 1u);
    p.active[p.groups + g] = 0;
    p.fail[g] = 0;
    p.fail[p.groups + g] = 0;
  }
}

// Outputs of group blockIdx.y: hard bits from app >= 0 (:67-69), or the soft outputs
// of :111-129.
template <int MSG>
__global__ void lanes_finish(LdpcLanesParams p) {
  using M = Msg<MSG>;
  const auto* c2v = static_cast<const typename M::T*>(p.c2v);
  const int g = int(blockIdx.y);
  const int stride = int(gridDim.x) * blockDim.x;
  const int t0 = int(blockIdx.x) * blockDim.x + threadIdx.x;
  const bool soft = p.msg_out || p.syst_out || p.parity_out;
  const typename M::T* cg = c2v + int64_t(g) * p.E * kLanes;
  for (int i = t0; i < p.N * kLanes; i += stride) {
    const int lane = i % kLanes, b = i / kLanes;
    const int64_t f = int64_t(g) * kLanes + lane;
    if (f >= p.nframes) continue;
    const int64_t at = int64_t(g) * p.N * kLanes + i;
    if (p.hard && b < p.msg) p.hard[f * p.msg + b] = uint8_t(p.app[at] >= 0.0f);
    if (soft) {
      float ext = 0.0f;
      for (uint32_t k = __ldg(p.col_ptr + b); k < __ldg(p.col_ptr + b + 1); ++k)
        ext += M::load(cg + int64_t(__ldg(p.col_edges + k)) * kLanes + lane);
      if (p.parity_out) store_llr(p.parity_out, p.out_dtype, f * p.N + b, ext);
      if (b < p.msg) {
        if (p.syst_out) store_llr(p.syst_out, p.out_dtype, f * p.msg + b, ext);
        if (p.msg_out) store_llr(p.msg_out, p.out_dtype, f * p.msg + b, p.chan[at] + ext);
      }
    }
  }
  if (p.state_out) {
    for (int64_t i = t0; i < p.E * kLanes; i += stride) {
      const int lane = int(i % kLanes);
      const int64_t e = i / kLanes;
      const int64_t f = int64_t(g) * kLanes + lane;
      if (f < p.nframes) store_llr(p.state_out, p.out_dtype, f * p.E + e, M::load(cg + i));
    }
  }
  if (p.iters && t0 < kLanes) {
    const int64_t f = int64_t(g) * kLanes + t0;
    if (f < p.nframes) p.iters[f] = p.iters_ws[f];
  }
}

// Grid of a per-row or per-bit pass over `groups` groups: y = group, x strides over
// `per_group` rows or bits with one warp each, about 16 blocks per SM over the grid.
dim3 grid_for(int64_t per_group, int groups) {
  const int64_t need = (per_group + kWarpsPerBlock - 1) / kWarpsPerBlock;
  const int64_t share = (148 * 16 + groups - 1) / groups;
  const int64_t x = need < share ? need : share;
  return dim3(unsigned(x > 0 ? x : 1), unsigned(groups));
}

// Working set of one group in bytes: chan, app and c2v, the arrays every iteration
// touches.
int64_t group_bytes(const LdpcLanesParams& p) {
  const int64_t mb = p.msg_type == 1 ? 2 : (p.msg_type == 2 ? 1 : 4);
  return int64_t(kLanes) * (2 * 4 * int64_t(p.N) + mb * p.E);
}

// Groups decoded together: all iterations of a wave run before the next wave starts,
// so that a wave whose working set fits in L2 never goes back to HBM for its messages.
// A wave is the most groups whose working set fits in kWaveCap (at least one group):
// on B200 (126 MB of L2) DVB-S2 normal frames ran fastest at 91 to 95 MB per wave
// (FP32 2 groups, int8 4 groups: 933 and 1029 Mbit/s against 877 and 987 with 46 and
// 71 MB) and lost 15 % at 124 MB, where the passes re-read HBM.
constexpr int64_t kWaveCap = 96ll << 20;

int wave_for(const LdpcLanesParams& p, int64_t gb) {
  if (p.wave_groups > 0) return p.wave_groups < p.groups ? p.wave_groups : p.groups;
  int64_t wave = kWaveCap / gb;
  if (wave < 1) wave = 1;
  return int(wave < p.groups ? wave : p.groups);
}

// Whether a batch runs as one persistent launch: asked for (persist == 1), small
// enough (at most kPersistGroups groups, one wave) and on a stream that is not being
// captured into a graph.  The built-in choice is the two launches per iteration: with
// programmatic dependent launch they measured faster on every batch tried (DVB-S2
// short frames x 64: 0.82 ms against 1.05 ms), because the persistent kernel's
// occupancy is set by its check pass's registers and its bit pass is latency-bound.

bool use_persistent(const LdpcLanesParams& p, int wave, cudaStream_t s) {
  if (p.persist <= 0 || p.groups > kPersistGroups || wave < p.groups) return false;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(s, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) {
    cudaGetLastError();
    return false;
  }
  return true;
}

}  // namespace

// Persistent launches of one device run one after the other, whatever their streams,
// so that two of them never hold parts of the GPU while each waits for the rest: every
// such launch waits for an event the previous one recorded.
namespace {
std::mutex g_persist_mu;
cudaEvent_t g_persist_ev[64] = {};
}  // namespace

cudaError_t ldpc_persist_launch(cudaStream_t s, const void* kern, unsigned blocks, unsigned threads, void** args) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lk(g_persist_mu);
  if (!g_persist_ev[dev] && (e = cudaEventCreateWithFlags(&g_persist_ev[dev], cudaEventDisableTiming)) != cudaSuccess)
    return e;
  if ((e = cudaStreamWaitEvent(s, g_persist_ev[dev], 0)) != cudaSuccess) return e;
  if ((e = cudaLaunchCooperativeKernel(kern, dim3(blocks), dim3(threads), args, 0, s)) != cudaSuccess) return e;
  return cudaEventRecord(g_persist_ev[dev], s);
}

namespace {

template <int ALG, int MSG, int DMAX>
cudaError_t launch_persistent(LdpcLanesParams p, cudaStream_t s) {
  auto kern = lanes_persist<ALG, MSG, DMAX>;
  int per_sm = 0, dev = 0, sms = 0;
  cudaError_t e;
  if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kWarpsPerBlock * 32, 0)) != cudaSuccess) return e;
  if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
  if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
  constexpr int kRows = DMAX <= 8 ? 2 : 1;
  const int64_t rows = (p.M + kRows - 1) / kRows;
  const int64_t units = int64_t(p.groups) * (int64_t(p.N) > rows ? int64_t(p.N) : rows);
  int64_t blocks = (units + kWarpsPerBlock - 1) / kWarpsPerBlock;
  if (blocks > int64_t(per_sm) * sms) blocks = int64_t(per_sm) * sms;
  if (blocks < 1) return cudaErrorInvalidConfiguration;
  if ((e = cudaMemsetAsync(p.barrier, 0, 2 * sizeof(unsigned), s)) != cudaSuccess) return e;
  void* args[] = {&p};
  return ldpc_persist_launch(s, reinterpret_cast<const void*>(kern), unsigned(blocks), kWarpsPerBlock * 32, args);
}

template <int ALG, int MSG, int DMAX>
cudaError_t run(const LdpcLanesParams& p, cudaStream_t s) {
  if (p.groups > 65535) return cudaErrorInvalidValue;
  const int wave = wave_for(p, group_bytes(p));
  const dim3 gs((148 * 8 + p.groups - 1) / p.groups, p.groups);
  lanes_stage<MSG><<<gs, 256, 0, s>>>(p);
  bool done = false;
  if (use_persistent(p, wave, s)) {
    const cudaError_t e = launch_persistent<ALG, MSG, DMAX>(p, s);
    if (e == cudaSuccess) done = true;
    else if (e != cudaErrorCooperativeLaunchTooLarge && e != cudaErrorNotSupported && e != cudaErrorInvalidConfiguration)
      return e;
    else cudaGetLastError();
  }
  for (int w0 = 0; !done && w0 < p.groups; w0 += wave) {
    const int nw = p.groups - w0 < wave ? p.groups - w0 : wave;
    const dim3 gbit = grid_for(p.N, nw);
    const dim3 gchk = grid_for((p.M + (DMAX <= 8 ? 1 : 0)) / (DMAX <= 8 ? 2 : 1), nw);
    cudaError_t e = launch_pdl(lanes_bit<MSG>, gbit, dim3(kWarpsPerBlock * 32), s, p, -1, w0);
    for (int it = 0; e == cudaSuccess && it < p.iterations; ++it) {
      e = launch_pdl(lanes_check<ALG, MSG, DMAX>, gchk, dim3(kWarpsPerBlock * 32), s, p, it, w0);
      if (e == cudaSuccess) e = launch_pdl(lanes_bit<MSG>, gbit, dim3(kWarpsPerBlock * 32), s, p, it, w0);
    }
    if (e != cudaSuccess) return e;
  }
  lanes_finish<MSG><<<gs, 256, 0, s>>>(p);
  return cudaGetLastError();
}

template <int ALG, int MSG>
cudaError_t run_d(const LdpcLanesParams& p, cudaStream_t s) {
  if (p.d_max <= 8) return run<ALG, MSG, 8>(p, s);
  if (p.d_max <= 16) return run<ALG, MSG, 16>(p, s);
  if (p.d_max <= 32) return run<ALG, MSG, 32>(p, s);
  return cudaErrorInvalidValue;
}

template <int ALG>
cudaError_t run_m(const LdpcLanesParams& p, cudaStream_t s) {
  switch (p.msg_type) {
    case 1: return run_d<ALG, 1>(p, s);
    case 2: return run_d<ALG, 2>(p, s);
    default: return run_d<ALG, 0>(p, s);
  }
}

}  // namespace

cudaError_t ldpc_lanes_init() {
  static std::atomic<unsigned long long> done{0};
  return once_per_device(done, [] {
    const LinearLut l = make_linear_lut();
    return cudaMemcpyToSymbol(c_lut, &l, sizeof(l));
  });
}

size_t ldpc_lanes_scratch_bytes(int64_t N, int64_t E, int64_t nframes, int msg_type) {
  const int64_t groups = (nframes + kLanes - 1) / kLanes;
  const size_t msg_bytes = msg_type == 1 ? 2 : (msg_type == 2 ? 1 : 4);
  auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
  return al(size_t(groups) * N * kLanes * 4) * 2 + al(size_t(groups) * E * kLanes * msg_bytes) +
         al(size_t(groups) * 16) + al(size_t(groups) * kLanes * 4) + al(2 * sizeof(unsigned));
}

cudaError_t launch_ldpc_lanes(LdpcLanesParams p, void* scratch, cudaStream_t s) {
  cudaError_t e0 = ldpc_lanes_init();
  if (e0 != cudaSuccess) return e0;
  if (p.nframes <= 0) return cudaSuccess;
  p.groups = int32_t((p.nframes + kLanes - 1) / kLanes);
  const size_t msg_bytes = p.msg_type == 1 ? 2 : (p.msg_type == 2 ? 1 : 4);
  auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
  char* q = static_cast<char*>(scratch);
  p.chan = reinterpret_cast<float*>(q);
  q += al(size_t(p.groups) * p.N * kLanes * 4);
  p.app = reinterpret_cast<float*>(q);
  q += al(size_t(p.groups) * p.N * kLanes * 4);
  p.c2v = q;
  q += al(size_t(p.groups) * p.E * kLanes * msg_bytes);
  p.active = reinterpret_cast<uint32_t*>(q);  // [2][groups]
  p.fail = p.active + 2 * p.groups;          // [2][groups]
  q += al(size_t(p.groups) * 16);
  p.iters_ws = reinterpret_cast<int32_t*>(q);
  q += al(size_t(p.groups) * kLanes * 4);
  p.barrier = reinterpret_cast<unsigned*>(q);
  switch (p.algorithm) {
    case kExact: return run_m<kExact>(p, s);
    case kLinear: return run_m<kLinear>(p, s);
    default: return run_m<kApproximate>(p, s);
  }
}

}  // namespace fecl
