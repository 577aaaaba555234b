// LDPC flooding belief propagation for batches: 32 frames per warp, one frame per
// lane.
//
// Same decoder as ldpc_flood.cu (BpDecoderImpl, src/detail/BpDecoder/BpDecoderImpl.cpp:37-179),
// laid out for HBM streaming instead of one CTA per frame.  Frames are grouped by 32;
// within a group every per-bit and per-edge array is stored lane-minor,
//     chan[g][n][32], app[g][n][32] (FP32), c2v[g][e][32] (FP32, FP16 or int8),
// so when a warp works on one check row (or one bit) for its 32 frames, every load
// and store is one contiguous 128-byte (or 64- / 32-byte) line, and the column
// indices are the same for all lanes.  Each iteration is three launches:
//   check: warp per (group, row): v = app - c2v, the reference's forward/backward
//          boxplus order (min-sum, whose chain is exact, as two minima and a sign
//          parity), scaled c2v out; for iteration >= 1 it also folds the row's
//          syndrome bit of the previous APP into a per-group failure mask (ballot +
//          one atomicOr), which is the reference's stop test (:53-59);
//   bit:   warp per (group, bit): app = chan + sum c2v in edge order;
//   update: per group, frames whose syndrome held stop (their lanes are masked from
//          then on) with the iteration count recorded.
// A frame that stops at iteration i has had exactly the reference's sequence: its
// last check update ran with the scaling of iteration i, which equals that of
// iteration I-1 because this kernel is used only when the scaling does not change
// across iterations (or with fixed iterations).
//
// Messages may be stored in FP16 or in saturated int8 (Q5.2, step 1/4, +-31.75);
// every sum and every boxplus runs in FP32.
#include <cuda_fp16.h>
#include <math.h>

#include "common.cuh"
#include "kernels.hpp"

namespace fecl {
namespace {

constexpr int kExact = 0, kLinear = 1, kApproximate = 2;
constexpr int kLanes = 32;
constexpr int kWarpsPerBlock = 8;

__constant__ LinearLut c_lut;

__device__ __forceinline__ bool neg(float x) { return (__float_as_uint(x) >> 31) != 0; }

__device__ __forceinline__ float box_linear(float a, float b) {
  const float m = fminf(fabsf(a), fabsf(b));
  const float s = (neg(a) != neg(b)) ? m : -m;
  return s - lut_log1pexpm(c_lut, fabsf(a + b)) + lut_log1pexpm(c_lut, fabsf(a - b));
}

__device__ __forceinline__ float phi(float x) { return log1pf(2.0f / expm1f(x)); }

// Message storage.
template <int MSG>
struct Msg;
template <>
struct Msg<0> {
  using T = float;
  __device__ static float load(const T* p) { return *p; }
  __device__ static void store(T* p, float v) { *p = v; }
};
template <>
struct Msg<1> {
  using T = __half;
  __device__ static float load(const T* p) { return __half2float(*p); }
  __device__ static void store(T* p, float v) { *p = __float2half_rn(v); }
};
template <>
struct Msg<2> {
  using T = int8_t;
  __device__ static float load(const T* p) { return float(*p) * 0.25f; }
  __device__ static void store(T* p, float v) {
    const float q = fminf(fmaxf(rintf(v * 4.0f), -127.0f), 127.0f);
    *p = int8_t(q);
  }
};

// One check row for this lane's frame: v[] in, c2v out (scaled), in the forward /
// backward order of BpDecoderImpl::checkUpdate (:132-159).
template <int ALG, int DMAX>
__device__ __forceinline__ void row_update(const float v[DMAX], float out[DMAX], int d, float sf) {
  if (ALG == kExact) {
    float m[DMAX], fs[DMAX];
    unsigned fn[DMAX];
#pragma unroll
    for (int j = 0; j < DMAX; ++j)
      if (j < d) m[j] = phi(fminf(fabsf(v[j]), 80.0f));
    fs[0] = m[0];
    fn[0] = neg(v[0]);
#pragma unroll
    for (int j = 1; j < DMAX; ++j)
      if (j < d - 1) {
        fs[j] = fs[j - 1] + m[j];
        fn[j] = fn[j - 1] ^ unsigned(neg(v[j]));
      }
    float bs = 0.0f;
    unsigned bn = 0;
    const unsigned odd = unsigned(d & 1);
#pragma unroll
    for (int j = DMAX - 1; j >= 0; --j) {
      if (j < d) {
        const int jp = j > 0 ? j - 1 : 0;
        float s;
        unsigned n;
        if (j == d - 1) {
          s = fs[jp];
          n = fn[jp];
        } else if (j == 0) {
          s = bs;
          n = bn;
        } else {
          s = fs[jp] + bs;
          n = fn[jp] ^ bn;
        }
        const float mag = phi(s);
        out[j] = sf * ((n ^ odd) ? -mag : mag);
        if (j == d - 1) {
          bs = m[j];
          bn = unsigned(neg(v[j]));
        } else {
          bs = bs + m[j];
          bn = bn ^ unsigned(neg(v[j]));
        }
      }
    }
  } else if (ALG == kApproximate) {
    // Min-sum: the chain of MinBoxSum::sum over the other inputs is exact (a minimum
    // and a sign parity: each pairwise sum is negative iff its operands' sign bits
    // agree), so the two smallest magnitudes and the sign-bit parity give the same
    // values bit for bit with a handful of registers.
    float m1 = INFINITY, m2 = INFINITY;
    int i1 = 0;
    unsigned par = 0;
#pragma unroll
    for (int j = 0; j < DMAX; ++j) {
      if (j < d) {
        const float a = fabsf(v[j]);
        par ^= unsigned(neg(v[j]));
        if (a < m1) {
          m2 = m1;
          m1 = a;
          i1 = j;
        } else if (a < m2) {
          m2 = a;
        }
      }
    }
    // d - 1 inputs: the result's sign bit is (d - 2) xor the parity of the others' sign bits.
    const unsigned base = unsigned((d - 2) & 1);
#pragma unroll
    for (int j = 0; j < DMAX; ++j) {
      if (j < d) {
        const float m = (j == i1) ? m2 : m1;
        const unsigned nb = base ^ par ^ unsigned(neg(v[j]));
        out[j] = sf * (nb ? -m : m);
      }
    }
  } else {
    float fwd[DMAX];
    fwd[0] = v[0];
#pragma unroll
    for (int j = 1; j < DMAX; ++j)
      if (j < d - 1) fwd[j] = box_linear(fwd[j - 1], v[j]);
    float bwd = 0.0f;
#pragma unroll
    for (int j = DMAX - 1; j >= 0; --j) {
      if (j < d) {
        const int jp = j > 0 ? j - 1 : 0;
        float o;
        if (j == d - 1) o = fwd[jp];
        else if (j == 0) o = bwd;
        else o = box_linear(fwd[jp], bwd);
        out[j] = sf * o;
        if (j == d - 1) bwd = v[j];
        else bwd = box_linear(bwd, v[j]);
      }
    }
  }
}

__device__ __forceinline__ int lane_id() { return threadIdx.x & 31; }

template <int ALG, int MSG, int DMAX>
__global__ void __launch_bounds__(kWarpsPerBlock * 32) lanes_check(LdpcLanesParams p, int it) {
  using M = Msg<MSG>;
  auto* c2v = static_cast<typename M::T*>(p.c2v);
  const int lane = lane_id();
  const int64_t warps = int64_t(gridDim.x) * kWarpsPerBlock;
  const int64_t tasks = int64_t(p.groups) * p.M;
  const bool check_syndrome = it > 0 && !p.fixed_iterations;
  const float* sf_row = p.sf + size_t(it % p.n_sf) * p.sf_stride;
  for (int64_t t = int64_t(blockIdx.x) * kWarpsPerBlock + (threadIdx.x >> 5); t < tasks; t += warps) {
    const int g = int(t / p.M);
    const int r = int(t - int64_t(g) * p.M);
    const uint32_t active = p.active[g];
    if (active == 0) continue;
    const bool mine = (active >> lane) & 1;
    const uint32_t e0 = __ldg(p.row_ptr + r);
    const int d = int(__ldg(p.row_ptr + r + 1) - e0);
    typename M::T* cg = c2v + (int64_t(g) * p.E + e0) * kLanes + lane;
    const float* ag = p.app + int64_t(g) * p.N * kLanes + lane;
    float v[DMAX];
    unsigned parity = 0;
#pragma unroll
    for (int j = 0; j < DMAX; ++j) {
      if (j < d) {
        const uint32_t col = __ldg(p.col_idx + e0 + j);
        const float a = ag[int64_t(col) * kLanes];
        parity ^= unsigned(a >= 0.0f);
        v[j] = a - M::load(cg + j * kLanes);
      }
    }
    if (check_syndrome) {
      const uint32_t bad = __ballot_sync(0xffffffffu, parity != 0) & active;
      if (bad && lane == 0) atomicOr(p.fail + g, bad);
    }
    float out[DMAX];
    row_update<ALG, DMAX>(v, out, d, sf_row[d - 2]);
    if (mine) {
#pragma unroll
      for (int j = 0; j < DMAX; ++j)
        if (j < d) M::store(cg + j * kLanes, out[j]);
    }
  }
}

// app = chan + sum of c2v over the bit's edges, in increasing edge order.
template <int MSG>
__global__ void __launch_bounds__(kWarpsPerBlock * 32) lanes_bit(LdpcLanesParams p, int all_lanes) {
  using M = Msg<MSG>;
  const auto* c2v = static_cast<const typename M::T*>(p.c2v);
  const int lane = lane_id();
  const int64_t warps = int64_t(gridDim.x) * kWarpsPerBlock;
  const int64_t tasks = int64_t(p.groups) * p.N;
  for (int64_t t = int64_t(blockIdx.x) * kWarpsPerBlock + (threadIdx.x >> 5); t < tasks; t += warps) {
    const int g = int(t / p.N);
    const int b = int(t - int64_t(g) * p.N);
    const uint32_t active = all_lanes ? 0xffffffffu : p.active[g];
    if (!((active >> lane) & 1)) continue;
    const int64_t base = (int64_t(g) * p.N + b) * kLanes + lane;
    float acc = p.chan[base];
    const uint32_t k1 = __ldg(p.col_ptr + b + 1);
    const typename M::T* cg = c2v + int64_t(g) * p.E * kLanes + lane;
    for (uint32_t k = __ldg(p.col_ptr + b); k < k1; ++k) acc += M::load(cg + int64_t(__ldg(p.col_edges + k)) * kLanes);
    p.app[base] = acc;
  }
}

// Frames whose syndrome held at this iteration (or every frame at the last one) stop.
__global__ void lanes_update(LdpcLanesParams p, int it) {
  for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < p.groups; g += gridDim.x * blockDim.x) {
    const uint32_t active = p.active[g];
    uint32_t done = 0;
    if (it == p.iterations - 1) done = active;
    else if (it > 0 && !p.fixed_iterations) done = active & ~p.fail[g];
    for (uint32_t m = done; m; m &= m - 1) {
      const int l = __ffs(m) - 1;
      p.iters_ws[int64_t(g) * kLanes + l] = it + 1;
    }
    p.active[g] = active & ~done;
    p.fail[g] = 0;
  }
}

// Frame-major inputs -> lane-minor scratch: chan (+ a-priori on systematic bits),
// c2v (state or zero), lane masks.  One thread per (group, position, lane).
template <int MSG>
__global__ void lanes_stage(LdpcLanesParams p) {
  using M = Msg<MSG>;
  auto* c2v = static_cast<typename M::T*>(p.c2v);
  const int64_t tot_bits = int64_t(p.groups) * p.N * kLanes;
  const int64_t tot_edges = int64_t(p.groups) * p.E * kLanes;
  const int64_t stride = int64_t(gridDim.x) * blockDim.x;
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < tot_bits; i += stride) {
    const int lane = int(i % kLanes);
    const int64_t gb = i / kLanes;
    const int g = int(gb / p.N);
    const int b = int(gb - int64_t(g) * p.N);
    const int64_t f = int64_t(g) * kLanes + lane;
    float x = 0.0f;
    if (f < p.nframes) {
      x = load_llr(p.llr, p.llr_dtype, f * p.N + b);
      if (p.syst_in && b < p.msg) x += load_llr(p.syst_in, p.llr_dtype, f * p.msg + b);
    }
    p.chan[i] = x;
  }
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < tot_edges; i += stride) {
    const int lane = int(i % kLanes);
    const int64_t ge = i / kLanes;
    const int g = int(ge / p.E);
    const int64_t e = ge - int64_t(g) * p.E;
    const int64_t f = int64_t(g) * kLanes + lane;
    float v = 0.0f;
    if (p.state_in && f < p.nframes) v = load_llr(p.state_in, p.llr_dtype, f * p.E + e);
    M::store(c2v + i, v);
  }
  for (int64_t g = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; g < p.groups; g += stride) {
    const int64_t left = p.nframes - g * kLanes;
    p.active[g] = left >= kLanes ? 0xffffffffu : ((1u << left) - 1u);
    p.fail[g] = 0;
  }
}

// Outputs: hard bits from app >= 0 (:67-69), or the soft outputs of :111-129.
template <int MSG>
__global__ void lanes_finish(LdpcLanesParams p) {
  using M = Msg<MSG>;
  const auto* c2v = static_cast<const typename M::T*>(p.c2v);
  const int64_t stride = int64_t(gridDim.x) * blockDim.x;
  const int64_t tot_bits = int64_t(p.groups) * p.N * kLanes;
  const bool soft = p.msg_out || p.syst_out || p.parity_out;
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < tot_bits; i += stride) {
    const int lane = int(i % kLanes);
    const int64_t gb = i / kLanes;
    const int g = int(gb / p.N);
    const int b = int(gb - int64_t(g) * p.N);
    const int64_t f = int64_t(g) * kLanes + lane;
    if (f >= p.nframes) continue;
    if (p.hard && b < p.msg) p.hard[f * p.msg + b] = uint8_t(p.app[i] >= 0.0f);
    if (soft) {
      float ext = 0.0f;
      const typename M::T* cg = c2v + int64_t(g) * p.E * kLanes + lane;
      for (uint32_t k = __ldg(p.col_ptr + b); k < __ldg(p.col_ptr + b + 1); ++k)
        ext += M::load(cg + int64_t(__ldg(p.col_edges + k)) * kLanes);
      if (p.parity_out) store_llr(p.parity_out, p.out_dtype, f * p.N + b, ext);
      if (b < p.msg) {
        if (p.syst_out) store_llr(p.syst_out, p.out_dtype, f * p.msg + b, ext);
        if (p.msg_out) store_llr(p.msg_out, p.out_dtype, f * p.msg + b, p.chan[i] + ext);
      }
    }
  }
  if (p.state_out) {
    const int64_t tot_edges = int64_t(p.groups) * p.E * kLanes;
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < tot_edges; i += stride) {
      const int lane = int(i % kLanes);
      const int64_t ge = i / kLanes;
      const int g = int(ge / p.E);
      const int64_t e = ge - int64_t(g) * p.E;
      const int64_t f = int64_t(g) * kLanes + lane;
      if (f < p.nframes) store_llr(p.state_out, p.out_dtype, f * p.E + e, M::load(c2v + i));
    }
  }
  for (int64_t f = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; f < p.nframes; f += stride)
    if (p.iters) p.iters[f] = p.iters_ws[f];
}

int grid_for(int64_t tasks_warps) {
  const int64_t blocks = (tasks_warps + kWarpsPerBlock - 1) / kWarpsPerBlock;
  return int(blocks < 148 * 16 ? (blocks > 0 ? blocks : 1) : 148 * 16);
}

template <int ALG, int MSG, int DMAX>
cudaError_t run(const LdpcLanesParams& p, cudaStream_t s) {
  const int gb = grid_for(int64_t(p.groups) * p.N);
  const int gc = grid_for(int64_t(p.groups) * p.M);
  lanes_stage<MSG><<<1184, 256, 0, s>>>(p);
  lanes_bit<MSG><<<gb, kWarpsPerBlock * 32, 0, s>>>(p, 1);
  for (int it = 0; it < p.iterations; ++it) {
    lanes_check<ALG, MSG, DMAX><<<gc, kWarpsPerBlock * 32, 0, s>>>(p, it);
    lanes_bit<MSG><<<gb, kWarpsPerBlock * 32, 0, s>>>(p, 0);
    lanes_update<<<(p.groups + 127) / 128, 128, 0, s>>>(p, it);
  }
  lanes_finish<MSG><<<1184, 256, 0, s>>>(p);
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

size_t ldpc_lanes_scratch_bytes(int64_t N, int64_t E, int64_t nframes, int msg_type) {
  const int64_t groups = (nframes + kLanes - 1) / kLanes;
  const size_t msg_bytes = msg_type == 1 ? 2 : (msg_type == 2 ? 1 : 4);
  auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
  return al(size_t(groups) * N * kLanes * 4) * 2 + al(size_t(groups) * E * kLanes * msg_bytes) +
         al(size_t(groups) * 8) + al(size_t(groups) * kLanes * 4);
}

cudaError_t launch_ldpc_lanes(LdpcLanesParams p, void* scratch, cudaStream_t s) {
  static bool lut_ready = false;
  if (!lut_ready) {
    LinearLut l;
    for (int i = 0; i < 8; ++i) l.y[i] = float(log(1.0 + exp(-(double(i) / 2.0))));
    cudaError_t e = cudaMemcpyToSymbol(c_lut, &l, sizeof(l));
    if (e != cudaSuccess) return e;
    lut_ready = true;
  }
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
  p.active = reinterpret_cast<uint32_t*>(q);
  p.fail = p.active + p.groups;
  q += al(size_t(p.groups) * 8);
  p.iters_ws = reinterpret_cast<int32_t*>(q);
  switch (p.algorithm) {
    case kExact: return run_m<kExact>(p, s);
    case kLinear: return run_m<kLinear>(p, s);
    default: return run_m<kApproximate>(p, s);
  }
}

}  // namespace fecl
