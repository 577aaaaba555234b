// Viterbi decoding of the convolutional codec (Convolutional::decodeBlocks ->
// ViterbiDecoderImpl::decodeBlock, src/detail/ViterbiDecoder/ViterbiDecoderImpl.cpp).
//
// One thread per frame walks the reference's steps: path metrics start at
// [0, -inf, ...]; per trellis step the branch metrics are the correlations of each
// output word with the step's L-values; every (state, input) pair is compared in
// state-then-input order and the later one wins ties (>=), recording its state and
// input for the traceback; no normalisation.  Tail termination traces back from
// state 0, Truncate from the first state of largest metric.  The metrics are FP64,
// as the reference's (FloatLlrMetrics::Type is double), so the survivors -- and the
// decisions -- are the reference's bit for bit.  The traceback rows (one byte of
// state and one of input per state and step) live in the caller's scratch.
#include <math.h>

#include "common.cuh"
#include "kernels.hpp"

namespace fecl {
namespace {

constexpr int kMaxStates = 64;
constexpr int kMaxOutputs = 64;

__global__ void __launch_bounds__(64) viterbi_kernel(TurboDeviceConstituent k, ViterbiRun r) {
  const int64_t f = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (f >= r.nframes) return;
  const int S = k.state_count, U = k.input_count, O = 1 << k.output_size;
  const int T = k.length + k.tail;
  const int64_t P = k.parity_size;
  uint8_t* st = r.trace + f * int64_t(T) * S * 2;  // [T][S] states, then [T][S] inputs
  uint8_t* in = st + int64_t(T) * S;
  double pm[kMaxStates], nm[kMaxStates], bm[kMaxOutputs];
  pm[0] = 0.0;
  for (int s = 1; s < S; ++s) pm[s] = -INFINITY;
  for (int t = 0; t < T; ++t) {
    for (int o = 0; o < O; ++o) {
      double x = 0.0;
      for (int b = 0; b < k.output_size; ++b)
        if ((o >> b) & 1) x += double(load_llr(r.llr, r.llr_dtype, f * P + int64_t(t) * k.output_size + b));
      bm[o] = x;
    }
    for (int s = 0; s < S; ++s) nm[s] = -INFINITY;
    uint8_t* srow = st + int64_t(t) * S;
    uint8_t* irow = in + int64_t(t) * S;
    for (int j = 0; j < S; ++j)
      for (int u = 0; u < U; ++u) {
        const int n = int(k.next_state[j * U + u]);
        const double c = pm[j] + bm[k.output[j * U + u]];
        if (c >= nm[n]) {
          srow[n] = uint8_t(j);
          irow[n] = uint8_t(u);
          nm[n] = c;
        }
      }
    for (int s = 0; s < S; ++s) pm[s] = nm[s];
  }
  int best = 0;
  if (k.termination != 0)
    for (int s = 0; s < S; ++s)
      if (pm[s] > pm[best]) best = s;
  for (int t = T - 1; t >= 0; --t) {
    if (t < k.length) {
      const int u = in[int64_t(t) * S + best];
      for (int j = 0; j < k.input_size; ++j) r.hard[f * k.msg_size + int64_t(t) * k.input_size + j] = uint8_t((u >> j) & 1);
    }
    best = st[int64_t(t) * S + best];
  }
}

__global__ void conv_encode_kernel(TurboDeviceConstituent c, const uint8_t* msg, uint8_t* parity, int64_t nframes) {
  const int64_t f = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (f >= nframes) return;
  const uint8_t* m = msg + f * c.msg_size;
  uint8_t* out = parity + f * c.parity_size;
  uint32_t state = 0;
  for (int s = 0; s < c.length; ++s) {
    uint32_t u = 0;
    for (int k = 0; k < c.input_size; ++k) u |= uint32_t(m[s * c.input_size + k] & 1) << k;
    const uint32_t o = c.output[state * c.input_count + u];
    state = c.next_state[state * c.input_count + u];
    for (int k = 0; k < c.output_size; ++k) out[s * c.output_size + k] = uint8_t((o >> k) & 1);
  }
  // greedy termination (src/detail/Convolutional.cpp:189-211)
  for (int s = 0; s < c.tail; ++s) {
    int best_count = -1;
    uint32_t best = 0;
    for (int u = 0; u < c.input_count; ++u) {
      const int count = __popc(state) - __popc(c.next_state[state * c.input_count + u]);
      if (count > best_count) {
        best_count = count;
        best = uint32_t(u);
      }
    }
    const uint32_t o = c.output[state * c.input_count + best];
    for (int k = 0; k < c.output_size; ++k) out[(c.length + s) * c.output_size + k] = uint8_t((o >> k) & 1);
    state = c.next_state[state * c.input_count + best];
  }
}

}  // namespace

size_t viterbi_scratch_bytes(const TurboDeviceConstituent& k, int64_t nframes) {
  return size_t(nframes) * size_t(k.length + k.tail) * size_t(k.state_count) * 2 + 256;
}

cudaError_t launch_viterbi(const TurboDeviceConstituent& k, const ViterbiRun& r, cudaStream_t s) {
  if (r.nframes <= 0) return cudaSuccess;
  if (k.state_count > kMaxStates || k.output_size > 6 || k.input_count > 256) return cudaErrorInvalidValue;
  viterbi_kernel<<<unsigned((r.nframes + 63) / 64), 64, 0, s>>>(k, r);
  return cudaGetLastError();
}

cudaError_t launch_conv_encode(const TurboDeviceConstituent& c, const uint8_t* msg, uint8_t* parity, int64_t nframes,
                               cudaStream_t s) {
  if (nframes <= 0) return cudaSuccess;
  conv_encode_kernel<<<unsigned((nframes + 63) / 64), 64, 0, s>>>(c, msg, parity, nframes);
  return cudaGetLastError();
}

}  // namespace fecl
