// LDPC normalised min-sum with FP16 messages, packed: two frames per lane, 64 frames
// per warp.
//
// The decoder of ldpc_lanes.cu (BpDecoderImpl, src/detail/BpDecoder/BpDecoderImpl.cpp:37-179,
// min-sum boxplus src/detail/LlrMetrics.h:184-191) in FP16 message passing with FP32
// bit-node sums.  Lane l of group g holds frames 64 g + l (the .x halves) and
// 64 g + 32 + l (the .y halves):
//     chan[g][n][32], app[g][n][32]  float2 (FP32 bit-node values of the two frames)
//     c2v[g][e][32]                  half2  (the two frames' check-to-bit messages)
// so every warp access is 256 (float2) or 128 (half2) contiguous bytes, and one
// packed instruction serves two frames:
//   check  v = app - c2v in FP32 (packed f32x2), rounded to FP16; |v|, the two
//          smallest magnitudes (m2 = min(m2, max(m1, |v|)), m1 = min(m1, |v|)) and
//          the sign parity in half2; edge j gets m2 where |v_j| == m1, else m1, its
//          sign, times the scaling, as one half2 store;
//   bit    app = chan + sum of c2v in edge order, FP32 (packed f32x2 adds).
// Ties are exact: two equal minima give m2 == m1.  The syndrome stop, the retirement
// of frames and the waves are those of ldpc_lanes.cu, with a pair of lane masks per
// group (.x frames, .y frames).
//
// Narrow groups.  The per-pass kernels also take groups of W = 2, 4, 8 or 16 lanes
// (2 W frames):
// chan / app [g][n][W] and c2v [g][e][W], a warp serving 32 / W rows (or bits) of its
// group at once, lane l on row (or bit) l / W and frame pair l % W.  A batch of a few
// frames then runs as many warps per pass as its frames need (one frame of a 64800-bit
// code: 64800 / 16 warps per bit pass with W = 2, against 64800 with W = 32), with the
// same arithmetic per frame, so the results do not depend on W.
#include <cuda_fp16.h>
#include <math.h>

#include "common.cuh"
#include "grid_sync.cuh"
#include "kernels.hpp"

namespace fecl {
namespace {

constexpr int kLanes = 32;
constexpr int kWarps = 8;
constexpr uint32_t kSigns = 0x80008000u;

__device__ __forceinline__ uint32_t bits(__half2 h) { return *reinterpret_cast<uint32_t*>(&h); }
__device__ __forceinline__ __half2 from_bits(uint32_t u) { return *reinterpret_cast<__half2*>(&u); }

// (v.x, v.y) rounded to nearest FP16, overflow saturated to +-65504, as one
// conversion: the same bits as rounding and then clamping to [-65504, 65504] for
// every finite or infinite input.  The PTX operand order puts the first source in
// the upper half.
__device__ __forceinline__ __half2 half2_satfinite(float2 v) {
  uint32_t r;
  asm("cvt.rn.satfinite.f16x2.f32 %0, %1, %2;" : "=r"(r) : "f"(v.y), "f"(v.x));
  return from_bits(r);
}

// active[it & 1][g][2] and fail[it & 1][g][2]: .x and .y frame masks.
__device__ __forceinline__ uint32_t* active_of(const LdpcLanesParams& p, int it) { return p.active + (it & 1) * 2 * p.groups; }
__device__ __forceinline__ uint32_t* fail_of(const LdpcLanesParams& p, int it) { return p.fail + (it & 1) * 2 * p.groups; }

template <int DMAX>
struct Row {
  uint32_t e0;
  int d;
  __half2 v[DMAX];
  unsigned px, py;  // parity of the hard decisions of the previous APP
};

template <int DMAX, int W = kLanes>
__device__ __forceinline__ void load_row(const LdpcLanesParams& p, int g, int r, int sub, Row<DMAX>& w) {
  const __half2* c2v = static_cast<const __half2*>(p.c2v);
  const float2* app = reinterpret_cast<const float2*>(p.app);
  w.e0 = __ldg(p.row_ptr + r);
  w.d = int(__ldg(p.row_ptr + r + 1) - w.e0);
  const __half2* cg = c2v + (int64_t(g) * p.E + w.e0) * W + sub;
  const float2* ag = app + int64_t(g) * p.N * W + sub;
  w.px = w.py = 0;
#pragma unroll
  for (int j = 0; j < DMAX; ++j) {
    if (j < w.d) {
      const uint32_t col = __ldg(p.col_idx + w.e0 + j);
      const float2 a = ag[int64_t(col) * W];
      const float2 c = __half22float2(cg[j * W]);
      w.px ^= unsigned(a.x >= 0.0f);
      w.py ^= unsigned(a.y >= 0.0f);
      // a - c in FP32, rounded to FP16 and kept finite (saturated at +-65504)
      w.v[j] = half2_satfinite(__ffma2_rn(c, make_float2(-1.0f, -1.0f), a));
    }
  }
}

template <int DMAX, int W = kLanes>
__device__ __forceinline__ void store_row(const LdpcLanesParams& p, int g, int sub, const Row<DMAX>& w, __half2 sf2,
                                          bool mine_x, bool mine_y, bool keep_all) {
  __half2* c2v = static_cast<__half2*>(p.c2v);
  const __half2 inf2 = __floats2half2_rn(INFINITY, INFINITY);
  __half2 m1 = inf2, m2 = inf2;
  uint32_t sg = 0;
#pragma unroll
  for (int j = 0; j < DMAX; ++j) {
    if (j < w.d) {
      const __half2 a = __habs2(w.v[j]);
      m2 = __hmin2(m2, __hmax2(m1, a));
      m1 = __hmin2(m1, a);
      sg ^= bits(w.v[j]);
    }
  }
  // d - 1 inputs per output: the sign is (d - 2) xor the parity of the others' signs.
  sg = (sg & kSigns) ^ (((w.d - 2) & 1) ? kSigns : 0u);
  // Lanes whose frames are not decoding keep their messages where the soft outputs,
  // which are sums of these messages, are wanted; a hard-decision decode reads only
  // the a-posteriori values, which the bit pass freezes for retired frames.
  const uint32_t keep = keep_all ? (mine_x ? 0u : 0x0000ffffu) | (mine_y ? 0u : 0xffff0000u) : 0u;
  __half2* cg = c2v + (int64_t(g) * p.E + w.e0) * W + sub;
  // The scaling is applied to the two magnitudes once per row: rounding to nearest is
  // symmetric, so (-m) * s is -(m * s) bit for bit and the edge's sign can be xored
  // into the scaled magnitude.
  if constexpr (DMAX > 16) {
    // Rows of degree > 16 also take the row's sign parity into the two magnitudes,
    // leaving each edge its own sign bit (one operation fewer per edge; measured
    // faster for these rows, slower for the rows of degree <= 16 below).
    const uint32_t b1 = bits(__hmul2(m1, sf2)) ^ sg, b2 = bits(__hmul2(m2, sf2)) ^ sg;
#pragma unroll
    for (int j = 0; j < DMAX; ++j) {
      if (j < w.d) {
        const uint32_t eq = __heq2_mask(__habs2(w.v[j]), m1);
        const __half2 out = from_bits(((b2 & eq) | (b1 & ~eq)) ^ (bits(w.v[j]) & kSigns));
        if (keep == 0u) {
          cg[j * W] = out;
        } else if (keep != 0xffffffffu) {
          const uint32_t old = bits(cg[j * W]);
          cg[j * W] = from_bits((bits(out) & ~keep) | (old & keep));
        }
      }
    }
    return;
  }
  const uint32_t b1 = bits(__hmul2(m1, sf2)), b2 = bits(__hmul2(m2, sf2));
#pragma unroll
  for (int j = 0; j < DMAX; ++j) {
    if (j < w.d) {
      const uint32_t eq = __heq2_mask(__habs2(w.v[j]), m1);
      const uint32_t mag = (b2 & eq) | (b1 & ~eq);
      const uint32_t sign = (sg ^ bits(w.v[j])) & kSigns;
      const __half2 out = from_bits(mag ^ sign);
      if (keep == 0u) {
        cg[j * W] = out;
      } else if (keep != 0xffffffffu) {
        const uint32_t old = bits(cg[j * W]);
        cg[j * W] = from_bits((bits(out) & ~keep) | (old & keep));
      }
    }
  }
}

// The lanes of a W-lane group whose bit is set in a warp ballot (lane l standing for
// frame pair l % W).
template <int W>
__device__ __forceinline__ uint32_t fold_lanes(uint32_t b) {
  if constexpr (W == 32) {
    return b;
  } else {
#pragma unroll
    for (int s = W; s < 32; s *= 2) b |= b >> s;
    return b & ((1u << W) - 1u);
  }
}

// Rows per lane: two for rows of degree <= 8 (more loads in flight per warp), except
// in groups of 2 or 4 lanes, whose batches of a few frames want warps, not loads per
// warp (one DVB-S2 normal r=1/2 frame, 50 iterations: 0.50 ms against 0.57 with two;
// with 8 or 16 lanes two rows measured faster, 1.00 against 1.13 ms for 12 frames).
template <int DMAX, int W>
constexpr int rows_per_lane() { return DMAX <= 8 && W >= 8 ? 2 : 1; }

// Rows r .. r + kRows - 1 of group g at iteration `it` (kRows = rows_per_lane; r is
// this lane's, rows past the last are skipped): the row updates; bx / by collect the
// lanes whose syndrome bit is set.  Every lane of the warp calls it.
template <int DMAX, int W = kLanes>
__device__ __forceinline__ void check_rows(const LdpcLanesParams& p, int it, int g, int r, int sub, bool mx, bool my,
                                           bool keep_all, bool check_syndrome, uint32_t& bx, uint32_t& by) {
  constexpr int kRows = rows_per_lane<DMAX, W>();
  Row<DMAX> w[kRows];
#pragma unroll
  for (int q = 0; q < kRows; ++q) {
    w[q].d = 0;
    if (r + q < p.M) load_row<DMAX, W>(p, g, r + q, sub, w[q]);
  }
#pragma unroll
  for (int q = 0; q < kRows; ++q) {
    if (check_syndrome) {
      bx |= fold_lanes<W>(__ballot_sync(0xffffffffu, w[q].d > 0 && w[q].px != 0));
      by |= fold_lanes<W>(__ballot_sync(0xffffffffu, w[q].d > 0 && w[q].py != 0));
    }
    if (w[q].d > 0) {
      // the scaling of rows of this degree (constant across iterations on this path)
      const float s = p.sf[size_t(it % p.n_sf) * p.sf_stride + (w[q].d >= 2 ? w[q].d - 2 : 0)];
      store_row<DMAX, W>(p, g, sub, w[q], __float2half2_rn(s), mx, my, keep_all);
    }
  }
}

template <int DMAX, int W>
__global__ void __launch_bounds__(kWarps * 32) h2_check(LdpcLanesParams p, int it, int g0) {
  pdl_enter();
  constexpr int kRows = rows_per_lane<DMAX, W>();
  constexpr int kSlots = 32 / W;  // rows (or row pairs) per warp step
  const int lane = threadIdx.x & 31;
  const int sub = lane % W, slot = lane / W;
  const int warps = int(gridDim.x) * kWarps;
  const bool check_syndrome = it > 0 && !p.fixed_iterations;
  const int g = g0 + int(blockIdx.y);
  const uint32_t ax = active_of(p, it)[2 * g], ay = active_of(p, it)[2 * g + 1];
  if ((ax | ay) == 0) return;
  const bool mx = (ax >> sub) & 1, my = (ay >> sub) & 1;
  const bool keep_all = p.msg_out || p.syst_out || p.parity_out || p.state_out;
  uint32_t bx = 0, by = 0;
  const int w0 = int(blockIdx.x) * kWarps + (threadIdx.x >> 5);
  for (int r = w0 * kSlots * kRows; r < p.M; r += warps * kSlots * kRows)
    check_rows<DMAX, W>(p, it, g, r + slot * kRows, sub, mx, my, keep_all, check_syndrome, bx, by);
  bx &= ax;
  by &= ay;
  if (lane == 0) {
    if (bx) atomicOr(fail_of(p, it) + 2 * g, bx);
    if (by) atomicOr(fail_of(p, it) + 2 * g + 1, by);
  }
}

// Retirement of the .x (h = 0) or .y (h = 1) frames of group g after the check pass of
// iteration `it`, and their masks for iteration it + 1.
template <int W = kLanes>
__device__ __forceinline__ void retire_half(const LdpcLanesParams& p, int it, int g, int h) {
  const uint32_t a = active_of(p, it)[2 * g + h];
  uint32_t done = 0;
  if (it == p.iterations - 1) done = a;
  else if (it > 0 && !p.fixed_iterations) done = a & ~fail_of(p, it)[2 * g + h];
  for (uint32_t m = done; m; m &= m - 1) p.iters_ws[int64_t(g) * 2 * W + h * W + (__ffs(m) - 1)] = it + 1;
  active_of(p, it + 1)[2 * g + h] = a & ~done;
  fail_of(p, it + 1)[2 * g + h] = 0;
}

// app = chan + sum of c2v over bit b's edges (edge order, FP32) for this lane's two
// frames; a retired frame's value stays.  The edges go in runs of 8 (one run for most
// bits): every edge id of a run is loaded, then every message, then they are added in
// order, so a bit costs three dependent loads rather than two per edge.
template <int W = kLanes>
__device__ __forceinline__ void bit_one(const LdpcLanesParams& p, int g, int b, int sub, bool mx, bool my) {
  constexpr uint32_t kRun = 8;
  const __half2* cg = static_cast<const __half2*>(p.c2v) + int64_t(g) * p.E * W + sub;
  const float2* chan = reinterpret_cast<const float2*>(p.chan);
  float2* app = reinterpret_cast<float2*>(p.app);
  const int64_t base = (int64_t(g) * p.N + b) * W + sub;
  const uint32_t k0 = __ldg(p.col_ptr + b), k1 = __ldg(p.col_ptr + b + 1);
  float2 acc = chan[base];
  for (uint32_t k = k0; k < k1; k += kRun) {
    uint32_t e[kRun];
    __half2 x[kRun];
#pragma unroll
    for (uint32_t j = 0; j < kRun; ++j) e[j] = k + j < k1 ? __ldg(p.col_edges + k + j) : 0u;
#pragma unroll
    for (uint32_t j = 0; j < kRun; ++j) x[j] = k + j < k1 ? cg[int64_t(e[j]) * W] : __half2{};
#pragma unroll
    for (uint32_t j = 0; j < kRun; ++j)
      if (k + j < k1) acc = __fadd2_rn(acc, __half22float2(x[j]));
  }
  if (mx && my) {
    app[base] = acc;
  } else {  // one of the lane's frames has retired: its APP stays
    float2 out = app[base];
    if (mx) out.x = acc.x;
    if (my) out.y = acc.y;
    app[base] = out;
  }
}

// Bit pass; with it < 0 the initial APP for every lane.  Block (0, y) retires frames
// and writes the group's masks for iteration it + 1.
template <int W>
__global__ void __launch_bounds__(kWarps * 32) h2_bit(LdpcLanesParams p, int it, int g0) {
  pdl_enter();
  constexpr int kSlots = 32 / W;
  const int lane = threadIdx.x & 31;
  const int sub = lane % W, slot = lane / W;
  const int warps = int(gridDim.x) * kWarps;
  const int g = g0 + int(blockIdx.y);
  const uint32_t ax = it < 0 ? 0xffffffffu : active_of(p, it)[2 * g];
  const uint32_t ay = it < 0 ? 0xffffffffu : active_of(p, it)[2 * g + 1];
  if (it >= 0 && blockIdx.x == 0 && threadIdx.x < 2) retire_half<W>(p, it, g, threadIdx.x);
  const bool mx = (ax >> sub) & 1, my = (ay >> sub) & 1;
  if (!mx && !my) return;
  for (int b = (int(blockIdx.x) * kWarps + (threadIdx.x >> 5)) * kSlots + slot; b < p.N; b += warps * kSlots)
    bit_one<W>(p, g, b, sub, mx, my);
}

// Persistent decoder for a small batch (at most kPersistGroups groups of 64 frames,
// one wave): one launch runs the initial APP and every iteration, the passes of all
// groups spread over the whole grid and separated by grid barriers.  It computes
// exactly the rows, bits and retirements of h2_check / h2_bit.  A barrier that gives
// up marks every frame's iteration count -1 (not decoded).
constexpr int kPersistGroups = 16;

template <int DMAX>
__global__ void __launch_bounds__(kWarps * 32) h2_persist(LdpcLanesParams p) {
  constexpr int kRows = DMAX <= 8 ? 2 : 1;
  __shared__ uint32_t s_bad[2 * kPersistGroups];
  const int lane = threadIdx.x & 31;
  const int warp = int(blockIdx.x) * kWarps + (threadIdx.x >> 5);
  const int warps = int(gridDim.x) * kWarps;
  const int ng = p.groups;
  const bool keep_all = p.msg_out || p.syst_out || p.parity_out || p.state_out;
  unsigned epoch = 0;
  for (int64_t u = warp; u < int64_t(ng) * p.N; u += warps) bit_one(p, int(u / p.N), int(u % p.N), lane, true, true);
  bool ok = grid_barrier(p.barrier, p.barrier + 1, epoch);
  const int rows = (p.M + kRows - 1) / kRows;
  for (int it = 0; ok && it < p.iterations; ++it) {
    const bool check_syndrome = it > 0 && !p.fixed_iterations;
    if (threadIdx.x < 2 * kPersistGroups) s_bad[threadIdx.x] = 0;
    __syncthreads();
    int g_cur = -1;
    uint32_t bx = 0, by = 0, ax = 0, ay = 0;
    for (int64_t u = warp; u < int64_t(ng) * rows; u += warps) {
      const int g = int(u / rows);
      if (g != g_cur) {
        if (lane == 0 && (bx & ax)) atomicOr(&s_bad[2 * g_cur], bx & ax);
        if (lane == 0 && (by & ay)) atomicOr(&s_bad[2 * g_cur + 1], by & ay);
        g_cur = g;
        bx = by = 0;
        ax = active_of(p, it)[2 * g];
        ay = active_of(p, it)[2 * g + 1];
      }
      if ((ax | ay) == 0) continue;
      check_rows<DMAX>(p, it, g, int(u % rows) * kRows, lane, (ax >> lane) & 1, (ay >> lane) & 1, keep_all,
                       check_syndrome, bx, by);
    }
    if (lane == 0 && g_cur >= 0 && (bx & ax)) atomicOr(&s_bad[2 * g_cur], bx & ax);
    if (lane == 0 && g_cur >= 0 && (by & ay)) atomicOr(&s_bad[2 * g_cur + 1], by & ay);
    __syncthreads();
    if (threadIdx.x < 2 * ng && s_bad[threadIdx.x]) atomicOr(fail_of(p, it) + threadIdx.x, s_bad[threadIdx.x]);
    if (!(ok = grid_barrier(p.barrier, p.barrier + 1, epoch))) break;
    if (blockIdx.x == 0 && threadIdx.x < 2 * ng) retire_half(p, it, threadIdx.x >> 1, threadIdx.x & 1);
    g_cur = -1;
    for (int64_t u = warp; u < int64_t(ng) * p.N; u += warps) {
      const int g = int(u / p.N);
      if (g != g_cur) {
        g_cur = g;
        ax = active_of(p, it)[2 * g];
        ay = active_of(p, it)[2 * g + 1];
      }
      const bool mx = (ax >> lane) & 1, my = (ay >> lane) & 1;
      if (mx || my) bit_one(p, g, int(u % p.N), lane, mx, my);
    }
    if (!(ok = grid_barrier(p.barrier, p.barrier + 1, epoch))) break;
    uint32_t left = 0;
    for (int i = 0; i < 2 * ng; ++i) left |= active_of(p, it + 1)[i];
    if (left == 0) break;
  }
  if (!ok && blockIdx.x == 0)
    for (int i = threadIdx.x; i < ng * 64; i += blockDim.x) p.iters_ws[i] = -1;
}

// ---- several codes in one launch ------------------------------------------------

// The groups of every job of a mixed batch (each job one code, its own scratch) whose
// check degrees are at most DMAX (8, 16 or 32) in one persistent launch: waves of
// groups, from any codes, whose working sets fit in L2 together; per wave the initial
// APP and every iteration, each pass spreading every group's rows (or bits) over the
// whole grid, passes separated by grid barriers.  A group runs exactly the rows, bits
// and retirements of h2_check / h2_bit with its own code's tables, scaling and
// iteration limit, so every frame's result is that of its job decoded alone.  A
// barrier that gives up marks the iteration counts of every frame -1 (not decoded).
__device__ __forceinline__ bool wave_left(const LdpcMultiParams& m, const LdpcLanesParams* codes, int q0, int q1,
                                          int it) {
  uint32_t left = 0;
  for (int q = q0; q < q1; ++q) {
    const LdpcMultiGroup gr = m.groups[q];
    const LdpcLanesParams& p = codes[gr.code];
    left |= active_of(p, it)[2 * gr.group] | active_of(p, it)[2 * gr.group + 1];
  }
  return left != 0;
}

template <int DMAX>
__global__ void __launch_bounds__(kWarps * 32, DMAX <= 16 ? 3 : 2) h2_multi(LdpcMultiParams m) {
  constexpr int kRows = DMAX <= 8 ? 2 : 1;
  __shared__ LdpcLanesParams s_codes[kMultiMaxCodes];
  __shared__ uint32_t s_bad[2 * kMultiMaxWaveGroups];
  {
    const uint32_t* src = reinterpret_cast<const uint32_t*>(m.codes);
    uint32_t* dst = reinterpret_cast<uint32_t*>(s_codes);
    const int words = int(m.ncodes * sizeof(LdpcLanesParams) / 4);
    for (int i = threadIdx.x; i < words; i += blockDim.x) dst[i] = src[i];
  }
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int warp = int(blockIdx.x) * kWarps + (threadIdx.x >> 5);
  const int warps = int(gridDim.x) * kWarps;
  unsigned epoch = 0;
  bool ok = true;
  for (int w = 0; ok && w < m.nwaves; ++w) {
    const int q0 = m.wave_ptr[w], q1 = m.wave_ptr[w + 1];
    int max_it = 0;
    for (int q = q0; q < q1; ++q) max_it = max(max_it, s_codes[m.groups[q].code].iterations);
    for (int q = q0; q < q1; ++q) {
      const LdpcMultiGroup gr = m.groups[q];
      const LdpcLanesParams& p = s_codes[gr.code];
      for (int b = warp; b < p.N; b += warps) bit_one(p, gr.group, b, lane, true, true);
    }
    ok = grid_barrier(m.barrier, m.barrier + 1, epoch);
    for (int it = 0; ok && it < max_it; ++it) {
      if (threadIdx.x < 2 * kMultiMaxWaveGroups) s_bad[threadIdx.x] = 0;
      __syncthreads();
      for (int q = q0; q < q1; ++q) {
        const LdpcMultiGroup gr = m.groups[q];
        const LdpcLanesParams& p = s_codes[gr.code];
        const uint32_t ax = active_of(p, it)[2 * gr.group], ay = active_of(p, it)[2 * gr.group + 1];
        if ((ax | ay) == 0) continue;
        const bool keep_all = p.msg_out || p.syst_out || p.parity_out || p.state_out;
        const bool check_syndrome = it > 0 && !p.fixed_iterations;
        uint32_t bx = 0, by = 0;
        for (int r = warp * kRows; r < p.M; r += warps * kRows)
          check_rows<DMAX>(p, it, gr.group, r, lane, (ax >> lane) & 1, (ay >> lane) & 1, keep_all, check_syndrome, bx,
                           by);
        if (lane == 0 && (bx & ax)) atomicOr(&s_bad[2 * (q - q0)], bx & ax);
        if (lane == 0 && (by & ay)) atomicOr(&s_bad[2 * (q - q0) + 1], by & ay);
      }
      __syncthreads();
      if (threadIdx.x < 2 * (q1 - q0) && s_bad[threadIdx.x]) {
        const LdpcMultiGroup gr = m.groups[q0 + (threadIdx.x >> 1)];
        atomicOr(fail_of(s_codes[gr.code], it) + 2 * gr.group + (threadIdx.x & 1), s_bad[threadIdx.x]);
      }
      if (!(ok = grid_barrier(m.barrier, m.barrier + 1, epoch))) break;
      if (blockIdx.x == 0 && threadIdx.x < 2 * (q1 - q0)) {
        const LdpcMultiGroup gr = m.groups[q0 + (threadIdx.x >> 1)];
        retire_half(s_codes[gr.code], it, gr.group, threadIdx.x & 1);
      }
      for (int q = q0; q < q1; ++q) {
        const LdpcMultiGroup gr = m.groups[q];
        const LdpcLanesParams& p = s_codes[gr.code];
        const uint32_t ax = active_of(p, it)[2 * gr.group], ay = active_of(p, it)[2 * gr.group + 1];
        const bool mx = (ax >> lane) & 1, my = (ay >> lane) & 1;
        if (!mx && !my) continue;
        for (int b = warp; b < p.N; b += warps) bit_one(p, gr.group, b, lane, mx, my);
      }
      if (!(ok = grid_barrier(m.barrier, m.barrier + 1, epoch))) break;
      if (!wave_left(m, s_codes, q0, q1, it + 1)) break;
    }
  }
  if (!ok && blockIdx.x == 0)
    for (int c = 0; c < m.ncodes; ++c)
      for (int i = threadIdx.x; i < s_codes[c].groups * 64; i += blockDim.x) s_codes[c].iters_ws[i] = -1;
}

// Frame f of a W-lane group g sits in lane f % W, half (f / W) % 2.
template <int W>
__device__ __forceinline__ int64_t frame_of(int g, int sub, int h) { return int64_t(g) * 2 * W + h * W + sub; }

template <int W>
__global__ void h2_stage(LdpcLanesParams p) {
  float2* chan = reinterpret_cast<float2*>(p.chan);
  __half2* c2v = static_cast<__half2*>(p.c2v);
  const int g = int(blockIdx.y);
  const int stride = int(gridDim.x) * blockDim.x;
  const int t0 = int(blockIdx.x) * blockDim.x + threadIdx.x;
  for (int i = t0; i < p.N * W; i += stride) {
    const int sub = i % W, b = i / W;
    float v[2];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int64_t f = frame_of<W>(g, sub, h);
      v[h] = 0.0f;
      if (f < p.nframes) {
        v[h] = load_llr(p.llr, p.llr_dtype, f * p.N + b);
        if (p.syst_in && b < p.msg) v[h] += load_llr(p.syst_in, p.llr_dtype, f * p.msg + b);
      }
    }
    chan[int64_t(g) * p.N * W + i] = make_float2(v[0], v[1]);
  }
  for (int64_t i = t0; i < p.E * W; i += stride) c2v[int64_t(g) * p.E * W + i] = __floats2half2_rn(0.0f, 0.0f);
  if (t0 == 0) {
    constexpr uint32_t kAll = W == 32 ? 0xffffffffu : (1u << W) - 1u;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int64_t left = p.nframes - int64_t(g) * 2 * W - h * W;
      p.active[2 * g + h] = left >= W ? kAll : (left > 0 ? ((1u << left) - 1u) : 0u);
      p.active[2 * p.groups + 2 * g + h] = 0;
      p.fail[2 * g + h] = 0;
      p.fail[2 * p.groups + 2 * g + h] = 0;
    }
  }
}

template <int W>
__global__ void h2_finish(LdpcLanesParams p) {
  const float2* chan = reinterpret_cast<const float2*>(p.chan);
  const float2* app = reinterpret_cast<const float2*>(p.app);
  const __half2* c2v = static_cast<const __half2*>(p.c2v);
  const int g = int(blockIdx.y);
  const int stride = int(gridDim.x) * blockDim.x;
  const int t0 = int(blockIdx.x) * blockDim.x + threadIdx.x;
  const bool soft = p.msg_out || p.syst_out || p.parity_out;
  const __half2* cg = c2v + int64_t(g) * p.E * W;
  for (int i = t0; i < p.N * W; i += stride) {
    const int sub = i % W, b = i / W;
    const int64_t at = int64_t(g) * p.N * W + i;
    const float2 a = app[at];
    float2 ext = make_float2(0.0f, 0.0f);
    if (soft)
      for (uint32_t k = __ldg(p.col_ptr + b); k < __ldg(p.col_ptr + b + 1); ++k)
        ext = __fadd2_rn(ext, __half22float2(cg[int64_t(__ldg(p.col_edges + k)) * W + sub]));
    const float2 ch = chan[at];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int64_t f = frame_of<W>(g, sub, h);
      if (f >= p.nframes) continue;
      const float av = h ? a.y : a.x, ev = h ? ext.y : ext.x, cv = h ? ch.y : ch.x;
      if (p.hard && b < p.msg) p.hard[f * p.msg + b] = uint8_t(av >= 0.0f);
      if (soft) {
        if (p.parity_out) store_llr(p.parity_out, p.out_dtype, f * p.N + b, ev);
        if (b < p.msg) {
          if (p.syst_out) store_llr(p.syst_out, p.out_dtype, f * p.msg + b, ev);
          if (p.msg_out) store_llr(p.msg_out, p.out_dtype, f * p.msg + b, cv + ev);
        }
      }
    }
  }
  if (p.state_out) {
    for (int64_t i = t0; i < p.E * W; i += stride) {
      const int sub = int(i % W);
      const int64_t e = i / W;
      const float2 c = __half22float2(cg[i]);
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int64_t f = frame_of<W>(g, sub, h);
        if (f < p.nframes) store_llr(p.state_out, p.out_dtype, f * p.E + e, h ? c.y : c.x);
      }
    }
  }
  if (p.iters && t0 < 2 * W) {
    const int64_t f = int64_t(g) * 2 * W + t0;
    if (f < p.nframes) p.iters[f] = p.iters_ws[f];
  }
}

dim3 grid_for(int64_t per_group, int groups) {
  const int64_t need = (per_group + kWarps - 1) / kWarps;
  const int64_t share = (148 * 16 + groups - 1) / groups;
  const int64_t x = need < share ? need : share;
  return dim3(unsigned(x > 0 ? x : 1), unsigned(groups));
}

// Waves as in ldpc_lanes.cu: the most groups whose working set fits in kWaveCap (one
// packed group of DVB-S2 normal frames is 62 MB: one group per wave ran 15 % faster
// than two).
constexpr int64_t kWaveCap = 96ll << 20;

// ---- several codes, one launch per pass ---------------------------------------

// The passes of h2_check / h2_bit over the groups [q0, q0 + gridDim.y) of a group
// table spanning several codes (each group's code parameters copied to shared memory
// by its blocks), so that one check launch per check-degree class and one bit launch
// serve every code of a batch in an iteration.  A block's rows (or bits) are those of
// h2_check / h2_bit for its group, so every frame gets exactly its own code's passes;
// blocks past their group's rows return at once.
__device__ __forceinline__ void load_group_params(const LdpcMultiParams& m, int q, LdpcLanesParams& sp, int& g) {
  const LdpcMultiGroup gr = m.groups[q];
  const uint32_t* src = reinterpret_cast<const uint32_t*>(m.codes + gr.code);
  uint32_t* dst = reinterpret_cast<uint32_t*>(&sp);
  for (int i = threadIdx.x; i < int(sizeof(LdpcLanesParams) / 4); i += blockDim.x) dst[i] = src[i];
  g = gr.group;
  __syncthreads();
}

// The rows of group g spread over the x blocks of its grid row (a warp per row or row
// pair), the lanes whose syndrome failed accumulated in bx / by.
template <int DMAX>
__device__ __forceinline__ void check_group(const LdpcLanesParams& p, int it, int g, int lane, bool mx, bool my,
                                            bool keep_all, bool check_syndrome, uint32_t& bx, uint32_t& by) {
  constexpr int kRows = DMAX <= 8 ? 2 : 1;
  const int warps = int(gridDim.x) * kWarps;
  const int w0 = int(blockIdx.x) * kWarps + (threadIdx.x >> 5);
  for (int r = w0 * kRows; r < p.M; r += warps * kRows)
    check_rows<DMAX>(p, it, g, r, lane, mx, my, keep_all, check_syndrome, bx, by);
}

// DMAX = 0: groups of every check-degree class in one launch, each block taking its
// group's class (blocks of a grid row share a group, so the choice is uniform).
template <int DMAX>
__global__ void __launch_bounds__(kWarps * 32) h2_check_many(LdpcMultiParams m, int it, int q0) {
  pdl_enter();
  __shared__ LdpcLanesParams sp;
  int g;
  load_group_params(m, q0 + int(blockIdx.y), sp, g);
  const LdpcLanesParams& p = sp;
  if (it >= p.iterations) return;
  const int lane = threadIdx.x & 31;
  const bool check_syndrome = it > 0 && !p.fixed_iterations;
  const uint32_t ax = active_of(p, it)[2 * g], ay = active_of(p, it)[2 * g + 1];
  if ((ax | ay) == 0) return;
  const bool mx = (ax >> lane) & 1, my = (ay >> lane) & 1;
  const bool keep_all = p.msg_out || p.syst_out || p.parity_out || p.state_out;
  uint32_t bx = 0, by = 0;
  const int cls = DMAX ? DMAX : (p.d_max <= 8 ? 8 : (p.d_max <= 16 ? 16 : 32));
  if (cls == 8) check_group<8>(p, it, g, lane, mx, my, keep_all, check_syndrome, bx, by);
  else if (cls == 16) check_group<16>(p, it, g, lane, mx, my, keep_all, check_syndrome, bx, by);
  else check_group<32>(p, it, g, lane, mx, my, keep_all, check_syndrome, bx, by);
  bx &= ax;
  by &= ay;
  if (lane == 0) {
    if (bx) atomicOr(fail_of(p, it) + 2 * g, bx);
    if (by) atomicOr(fail_of(p, it) + 2 * g + 1, by);
  }
}

__global__ void __launch_bounds__(kWarps * 32) h2_bit_many(LdpcMultiParams m, int it, int q0) {
  pdl_enter();
  __shared__ LdpcLanesParams sp;
  int g;
  load_group_params(m, q0 + int(blockIdx.y), sp, g);
  const LdpcLanesParams& p = sp;
  if (it >= p.iterations) return;
  const int lane = threadIdx.x & 31;
  const int warps = int(gridDim.x) * kWarps;
  const uint32_t ax = it < 0 ? 0xffffffffu : active_of(p, it)[2 * g];
  const uint32_t ay = it < 0 ? 0xffffffffu : active_of(p, it)[2 * g + 1];
  if (it >= 0 && blockIdx.x == 0 && threadIdx.x < 2) retire_half(p, it, g, threadIdx.x);
  const bool mx = (ax >> lane) & 1, my = (ay >> lane) & 1;
  if (!mx && !my) return;
  for (int b = int(blockIdx.x) * kWarps + (threadIdx.x >> 5); b < p.N; b += warps) bit_one(p, g, b, lane, mx, my);
}

// One persistent launch when asked for (persist == 1) for batches of at most
// kPersistGroups groups, all in one wave, on a stream that is not capturing (the
// per-pass launches are the built-in choice: see ldpc_lanes.cu).

bool use_persistent(const LdpcLanesParams& p, int64_t wave, cudaStream_t s) {
  if (p.persist <= 0 || p.groups > kPersistGroups || wave < p.groups) return false;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(s, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) {
    cudaGetLastError();
    return false;
  }
  return true;
}

template <int DMAX>
cudaError_t launch_persistent(LdpcLanesParams p, cudaStream_t s) {
  auto kern = h2_persist<DMAX>;
  int per_sm = 0, dev = 0, sms = 0;
  cudaError_t e;
  if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kWarps * 32, 0)) != cudaSuccess) return e;
  if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
  if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
  constexpr int kRows = DMAX <= 8 ? 2 : 1;
  const int64_t rows = (p.M + kRows - 1) / kRows;
  const int64_t units = int64_t(p.groups) * (int64_t(p.N) > rows ? int64_t(p.N) : rows);
  int64_t blocks = (units + kWarps - 1) / kWarps;
  if (blocks > int64_t(per_sm) * sms) blocks = int64_t(per_sm) * sms;
  if (blocks < 1) return cudaErrorInvalidConfiguration;
  if ((e = cudaMemsetAsync(p.barrier, 0, 2 * sizeof(unsigned), s)) != cudaSuccess) return e;
  void* args[] = {&p};
  return ldpc_persist_launch(s, reinterpret_cast<const void*>(kern), unsigned(blocks), kWarps * 32, args);
}

// The grid of the staging and finishing kernels: 256 threads per block over the
// larger of a group's bit and edge slots, at most about eight blocks per SM in all.
dim3 stage_grid(const LdpcLanesParams& p, int W) {
  const int64_t need = ((p.N > p.E ? int64_t(p.N) : p.E) * W + 255) / 256;
  const int64_t share = (148 * 8 + p.groups - 1) / p.groups;
  const int64_t x = need < share ? need : share;
  return dim3(unsigned(x > 0 ? x : 1), unsigned(p.groups));
}

template <int DMAX, int W>
cudaError_t run(const LdpcLanesParams& p, cudaStream_t s) {
  if (p.groups > 65535) return cudaErrorInvalidValue;
  constexpr int kSlots = 32 / W;
  const int64_t gb = int64_t(W) * (2 * 8 * int64_t(p.N) + 4 * p.E);
  int64_t wave = p.wave_groups > 0 ? p.wave_groups : kWaveCap / gb;
  if (wave < 1) wave = 1;
  if (wave > p.groups) wave = p.groups;
  const dim3 gs = stage_grid(p, W);
  h2_stage<W><<<gs, 256, 0, s>>>(p);
  bool done = false;
  if (W == kLanes && use_persistent(p, wave, s)) {
    const cudaError_t e = launch_persistent<DMAX>(p, s);
    if (e == cudaSuccess) done = true;
    else if (e != cudaErrorCooperativeLaunchTooLarge && e != cudaErrorNotSupported && e != cudaErrorInvalidConfiguration)
      return e;
    else cudaGetLastError();
  }
  for (int w0 = 0; !done && w0 < p.groups; w0 += int(wave)) {
    const int nw = p.groups - w0 < wave ? p.groups - w0 : int(wave);
    constexpr int kRows = rows_per_lane<DMAX, W>();
    const dim3 gbit = grid_for((p.N + kSlots - 1) / kSlots, nw);
    const dim3 gchk = grid_for((p.M + kRows * kSlots - 1) / (kRows * kSlots), nw);
    cudaError_t e = launch_pdl(h2_bit<W>, gbit, dim3(kWarps * 32), s, p, -1, w0);
    for (int it = 0; e == cudaSuccess && it < p.iterations; ++it) {
      e = launch_pdl(h2_check<DMAX, W>, gchk, dim3(kWarps * 32), s, p, it, w0);
      if (e == cudaSuccess) e = launch_pdl(h2_bit<W>, gbit, dim3(kWarps * 32), s, p, it, w0);
    }
    if (e != cudaSuccess) return e;
  }
  h2_finish<W><<<gs, 256, 0, s>>>(p);
  return cudaGetLastError();
}

template <int DMAX>
cudaError_t run_width(const LdpcLanesParams& p, int W, cudaStream_t s) {
  switch (W) {
    case 2: return run<DMAX, 2>(p, s);
    case 4: return run<DMAX, 4>(p, s);
    case 8: return run<DMAX, 8>(p, s);
    case 16: return run<DMAX, 16>(p, s);
    default: return run<DMAX, kLanes>(p, s);
  }
}

template <int DMAX>
int multi_blocks() {
  int per_sm = 0, dev = 0, sms = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, h2_multi<DMAX>, kWarps * 32, 0) != cudaSuccess ||
      cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return per_sm * sms;
}

template <int DMAX>
cudaError_t launch_multi(LdpcMultiParams m, cudaStream_t s) {
  const int blocks = multi_blocks<DMAX>();
  if (blocks <= 0) return cudaErrorInvalidConfiguration;
  cudaError_t e = cudaMemsetAsync(m.barrier, 0, 2 * sizeof(unsigned), s);
  if (e != cudaSuccess) return e;
  // A cooperative launch (all blocks resident, so the grid barriers are safe).  Outside
  // a stream capture it is ordered after the device's previous persistent launch;
  // under capture it goes through cudaLaunchKernelEx, which records a cooperative
  // graph node.
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if ((e = cudaStreamIsCapturing(s, &cs)) != cudaSuccess) return e;
  if (cs == cudaStreamCaptureStatusNone) {
    void* args[] = {&m};
    return ldpc_persist_launch(s, reinterpret_cast<const void*>(h2_multi<DMAX>), unsigned(blocks), kWarps * 32, args);
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(unsigned(blocks));
  cfg.blockDim = dim3(kWarps * 32);
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, h2_multi<DMAX>, m);
}

}  // namespace

size_t ldpc_lanes_h2_scratch_bytes(int64_t N, int64_t E, int64_t nframes) {
  const int64_t groups = (nframes + 63) / 64;
  auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
  return al(size_t(groups) * N * kLanes * 8) * 2 + al(size_t(groups) * E * kLanes * 4) + al(size_t(groups) * 32) +
         al(size_t(groups) * 64 * 4) + al(2 * sizeof(unsigned));
}

void ldpc_lanes_h2_layout(LdpcLanesParams& p, void* scratch, int W) {
  p.groups = int32_t((p.nframes + 2 * W - 1) / (2 * W));
  auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
  char* q = static_cast<char*>(scratch);
  p.chan = reinterpret_cast<float*>(q);
  q += al(size_t(p.groups) * p.N * W * 8);
  p.app = reinterpret_cast<float*>(q);
  q += al(size_t(p.groups) * p.N * W * 8);
  p.c2v = q;
  q += al(size_t(p.groups) * p.E * W * 4);
  p.active = reinterpret_cast<uint32_t*>(q);  // [2][groups][2]
  p.fail = p.active + 4 * p.groups;          // [2][groups][2]
  q += al(size_t(p.groups) * 32);
  p.iters_ws = reinterpret_cast<int32_t*>(q);
  q += al(size_t(p.groups) * 2 * W * 4);
  p.barrier = reinterpret_cast<unsigned*>(q);
}

// Lanes per group for a batch of n frames.  Up to 16 frames: the narrowest power of
// two from 2 to 8 whose group (2 W frames) holds the batch.  Beyond: 32, 16 or 8
// lanes, whichever leaves the fewest idle frame slots in the last group, the wider
// unless a narrower one saves more than n / 16 of them -- groups of 8 lanes and up
// still use every 32-byte sector they touch, narrower ones would not.
int ldpc_lanes_h2_width(int64_t nframes) {
  if (nframes <= 16) {
    int W = 2;
    while (2 * W < nframes) W *= 2;
    return W;
  }
  auto idle = [&](int64_t w) { return (nframes + 2 * w - 1) / (2 * w) * (2 * w) - nframes; };
  int best = kLanes;
  for (int W : {16, 8})
    if (idle(best) - idle(W) > nframes / 16) best = W;
  return best;
}

int64_t ldpc_lanes_h2_group_bytes(int64_t N, int64_t E) { return int64_t(kLanes) * (2 * 8 * N + 4 * E); }

cudaError_t launch_ldpc_h2_stage(const LdpcLanesParams& p, cudaStream_t s) {
  if (p.groups <= 0) return cudaSuccess;
  h2_stage<kLanes><<<dim3((148 * 8 + p.groups - 1) / p.groups, p.groups), 256, 0, s>>>(p);
  return cudaGetLastError();
}

cudaError_t launch_ldpc_h2_finish(const LdpcLanesParams& p, cudaStream_t s) {
  if (p.groups <= 0) return cudaSuccess;
  h2_finish<kLanes><<<dim3((148 * 8 + p.groups - 1) / p.groups, p.groups), 256, 0, s>>>(p);
  return cudaGetLastError();
}

cudaError_t launch_ldpc_h2_many(const LdpcMultiParams& m, const LdpcManyWave& w, int d_max, cudaStream_t s) {
  if (w.groups <= 0 || w.groups > 65535) return w.groups == 0 ? cudaSuccess : cudaErrorInvalidValue;
  const dim3 gbit = grid_for(w.max_bits, w.groups);
  const int kRows = d_max > 0 && d_max <= 8 ? 2 : 1;
  const dim3 gchk = grid_for((w.max_rows + kRows - 1) / kRows, w.groups);
  cudaError_t e = launch_pdl(h2_bit_many, gbit, dim3(kWarps * 32), s, m, -1, w.q0);
  for (int it = 0; e == cudaSuccess && it < w.iterations; ++it) {
    if (d_max <= 0) e = launch_pdl(h2_check_many<0>, gchk, dim3(kWarps * 32), s, m, it, w.q0);
    else if (d_max <= 8) e = launch_pdl(h2_check_many<8>, gchk, dim3(kWarps * 32), s, m, it, w.q0);
    else if (d_max <= 16) e = launch_pdl(h2_check_many<16>, gchk, dim3(kWarps * 32), s, m, it, w.q0);
    else e = launch_pdl(h2_check_many<32>, gchk, dim3(kWarps * 32), s, m, it, w.q0);
    if (e == cudaSuccess) e = launch_pdl(h2_bit_many, gbit, dim3(kWarps * 32), s, m, it, w.q0);
  }
  return e;
}

cudaError_t launch_ldpc_h2_multi(LdpcMultiParams m, int d_max, cudaStream_t s) {
  if (m.nwaves <= 0) return cudaSuccess;
  if (m.ncodes <= 0 || m.ncodes > kMultiMaxCodes) return cudaErrorInvalidValue;
  if (d_max <= 8) return launch_multi<8>(m, s);
  if (d_max <= 16) return launch_multi<16>(m, s);
  if (d_max <= 32) return launch_multi<32>(m, s);
  return cudaErrorInvalidValue;
}

cudaError_t launch_ldpc_lanes_h2(LdpcLanesParams p, void* scratch, cudaStream_t s) {
  if (p.nframes <= 0) return cudaSuccess;
  if (p.state_in || p.algorithm != 2) return cudaErrorInvalidValue;
  const int W = ldpc_lanes_h2_width(p.nframes);
  ldpc_lanes_h2_layout(p, scratch, W);
  if (p.d_max <= 8) return run_width<8>(p, W, s);
  if (p.d_max <= 16) return run_width<16>(p, W, s);
  if (p.d_max <= 32) return run_width<32>(p, W, s);
  return cudaErrorInvalidValue;
}

}  // namespace fecl
