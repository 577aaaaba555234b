// Flooding belief-propagation LDPC decoder, FP32 messages: the reference-parity path.
//
// Follows BpDecoderImpl (src/detail/BpDecoder/BpDecoderImpl.cpp):
//   - v->c messages start at the channel L-values (:42-46), or, when a soft state
//     is given, are rebuilt from it by a bit-node update (:81-94);
//   - each iteration is a check-node update (:132-159) then a bit-node update
//     (:161-179); after iteration i < I-1 the hard decision APP >= 0 (:53-55) is
//     checked against every parity equation and a satisfied syndrome stops the
//     loop (:56-59);
//   - one last check-node update with the scaling of iteration I-1 (:61), then the
//     a-posteriori values (:63-69) or the soft outputs (:111-129).
//
// Device layout: one CTA decodes one frame and runs every iteration; check rows
// and bits are strided over the CTA's threads.  v->c messages are not stored: a
// check row recomputes them as APP(bit) - c2v(edge), so per iteration the kernel
// reads c2v[E] + APP gathers and writes c2v[E] (check pass), then reads c2v through
// the per-bit edge lists and writes APP[N] (bit pass).
#include <math.h>

#include "common.cuh"
#include "kernels.hpp"

namespace fecl {
namespace {

constexpr int kExact = 0, kLinear = 1, kApproximate = 2;

__constant__ LinearLut c_lut;

__device__ __forceinline__ bool neg(float x) { return (__float_as_uint(x) >> 31) != 0; }

// MinBoxSum::sum, src/detail/LlrMetrics.h:184-191.
__device__ __forceinline__ float box_min(float a, float b) {
  const float m = fminf(fabsf(a), fabsf(b));
  return (neg(a) != neg(b)) ? m : -m;
}

// LinearBoxSum::sum, src/detail/LlrMetrics.h:152-159.
__device__ __forceinline__ float box_linear(float a, float b) {
  const float m = fminf(fabsf(a), fabsf(b));
  const float s = (neg(a) != neg(b)) ? m : -m;
  return s - lut_log1pexpm(c_lut, fabsf(a + b)) + lut_log1pexpm(c_lut, fabsf(a - b));
}

// phi(x) = -log(tanh(x/2)), its own inverse.  BoxSum (src/detail/LlrMetrics.h:126-140)
// multiplies tanh(-x/2) over a row and maps back with -2 atanh; in the phi domain the
// same boxplus is a sum of phi(|x|) and a sign parity, which keeps FP32 accurate where
// tanh rounds to +-1 (|x| > 17 in FP32).  Inputs are clamped to 80 so phi stays normal.
__device__ __forceinline__ float phi(float x) { return ldpc_phi(x); }

template <int ALG, int DMAX>
__device__ __forceinline__ void check_row(const LdpcDeviceCode& c, float* __restrict__ c2v,
                                          const float* __restrict__ app, int r, const float* sf_row) {
  const uint32_t e0 = c.row_ptr[r];
  const int d = int(c.row_ptr[r + 1] - e0);
  const float sf = sf_row[d >= 2 ? d - 2 : 0];
  float v[DMAX];
#pragma unroll
  for (int j = 0; j < DMAX; ++j)
    if (j < d) v[j] = app[c.col_idx[e0 + j]] - c2v[e0 + j];

  if (ALG == kExact) {
    float m[DMAX];
    float fs[DMAX];      // prefix sums of phi over 0..j
    unsigned fn[DMAX];   // prefix sign parity over 0..j
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
        float s;
        unsigned n;
        const int jp = j > 0 ? j - 1 : 0;
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
        c2v[e0 + j] = sf * ((n ^ odd) ? -mag : mag);
        if (j == d - 1) {
          bs = m[j];
          bn = unsigned(neg(v[j]));
        } else {
          bs = bs + m[j];
          bn = bn ^ unsigned(neg(v[j]));
        }
      }
    }
  } else {
    float fwd[DMAX];  // fwd[j] = v0 (+) ... (+) vj
    fwd[0] = v[0];
#pragma unroll
    for (int j = 1; j < DMAX; ++j)
      if (j < d - 1) fwd[j] = (ALG == kLinear) ? box_linear(fwd[j - 1], v[j]) : box_min(fwd[j - 1], v[j]);
    float bwd = 0.0f;
#pragma unroll
    for (int j = DMAX - 1; j >= 0; --j) {
      if (j < d) {
        const int jp = j > 0 ? j - 1 : 0;
        float out;
        if (j == d - 1) out = fwd[jp];
        else if (j == 0) out = bwd;
        else out = (ALG == kLinear) ? box_linear(fwd[jp], bwd) : box_min(fwd[jp], bwd);
        c2v[e0 + j] = sf * out;
        if (j == d - 1) bwd = v[j];
        else bwd = (ALG == kLinear) ? box_linear(bwd, v[j]) : box_min(bwd, v[j]);
      }
    }
  }
}

template <int ALG, int DMAX>
__global__ void __launch_bounds__(256) ldpc_flood_f32(LdpcDeviceCode c, LdpcRun p) {
  const int64_t f = blockIdx.x;
  const int N = c.N, M = c.M;
  const int64_t E = c.E;
  float* __restrict__ c2v = p.c2v + f * E;
  float* __restrict__ app = p.app + f * int64_t(N);
  float* __restrict__ chan = p.chan + f * int64_t(N);

  for (int b = threadIdx.x; b < N; b += blockDim.x) {
    float x = load_llr(p.llr, p.llr_dtype, f * N + b);
    if (p.syst_in && b < c.msg) x += load_llr(p.syst_in, p.llr_dtype, f * c.msg + b);
    chan[b] = x;
  }
  for (int64_t e = threadIdx.x; e < E; e += blockDim.x)
    c2v[e] = p.state_in ? load_llr(p.state_in, p.llr_dtype, f * E + e) : 0.0f;
  __syncthreads();
  for (int b = threadIdx.x; b < N; b += blockDim.x) {
    float acc = chan[b];
    if (p.state_in)
      for (uint32_t k = c.col_ptr[b]; k < c.col_ptr[b + 1]; ++k) acc += c2v[c.col_edges[k]];
    app[b] = acc;
  }
  __syncthreads();

  const int I = c.iterations;
  int ran = 0;
  for (int it = 0; it < I; ++it) {
    bool last = (it == I - 1);
    if (it > 0 && !c.fixed_iterations) {
      int fail = 0;
      for (int r = threadIdx.x; r < M && !fail; r += blockDim.x) {
        unsigned s = 0;
        for (uint32_t e = c.row_ptr[r]; e < c.row_ptr[r + 1]; ++e) s ^= unsigned(app[c.col_idx[e]] >= 0.0f);
        fail = int(s);
      }
      if (!__syncthreads_or(fail)) last = true;
    }
    const float* sf_row = c.sf + size_t((last ? I - 1 : it) % c.n_sf) * c.sf_stride;
    for (int r = threadIdx.x; r < M; r += blockDim.x) check_row<ALG, DMAX>(c, c2v, app, r, sf_row);
    __syncthreads();
    for (int b = threadIdx.x; b < N; b += blockDim.x) {
      float acc = chan[b];
      for (uint32_t k = c.col_ptr[b]; k < c.col_ptr[b + 1]; ++k) acc += c2v[c.col_edges[k]];
      app[b] = acc;
    }
    __syncthreads();
    ++ran;
    if (last) break;
  }

  if (p.iters && threadIdx.x == 0) p.iters[f] = ran;
  if (p.hard)
    for (int b = threadIdx.x; b < c.msg; b += blockDim.x) p.hard[f * c.msg + b] = uint8_t(app[b] >= 0.0f);
  if (p.msg_out || p.syst_out || p.parity_out) {
    for (int b = threadIdx.x; b < N; b += blockDim.x) {
      float ext = 0.0f;
      for (uint32_t k = c.col_ptr[b]; k < c.col_ptr[b + 1]; ++k) ext += c2v[c.col_edges[k]];
      if (p.parity_out) store_llr(p.parity_out, p.out_dtype, f * N + b, ext);
      if (b < c.msg) {
        if (p.syst_out) store_llr(p.syst_out, p.out_dtype, f * c.msg + b, ext);
        if (p.msg_out) store_llr(p.msg_out, p.out_dtype, f * c.msg + b, chan[b] + ext);
      }
    }
  }
  if (p.state_out)
    for (int64_t e = threadIdx.x; e < E; e += blockDim.x) store_llr(p.state_out, p.out_dtype, f * E + e, c2v[e]);
}

template <int ALG>
cudaError_t launch_alg(const LdpcDeviceCode& c, const LdpcRun& p, cudaStream_t s) {
  const dim3 grid(unsigned(p.nframes)), block(256);
  if (c.d_max <= 8) ldpc_flood_f32<ALG, 8><<<grid, block, 0, s>>>(c, p);
  else if (c.d_max <= 16) ldpc_flood_f32<ALG, 16><<<grid, block, 0, s>>>(c, p);
  else if (c.d_max <= 32) ldpc_flood_f32<ALG, 32><<<grid, block, 0, s>>>(c, p);
  else if (c.d_max <= 64) ldpc_flood_f32<ALG, 64><<<grid, block, 0, s>>>(c, p);
  else return cudaErrorInvalidValue;
  return cudaGetLastError();
}

}  // namespace

cudaError_t ldpc_flood_init() {
  static std::atomic<unsigned long long> done{0};
  return once_per_device(done, [] {
    const LinearLut l = make_linear_lut();
    return cudaMemcpyToSymbol(c_lut, &l, sizeof(l));
  });
}

cudaError_t launch_ldpc_flood(const LdpcDeviceCode& c, const LdpcRun& p, cudaStream_t s) {
  cudaError_t e0 = ldpc_flood_init();
  if (e0 != cudaSuccess) return e0;
  if (p.nframes <= 0) return cudaSuccess;
  switch (c.algorithm) {
    case kExact: return launch_alg<kExact>(c, p, s);
    case kLinear: return launch_alg<kLinear>(c, p, s);
    default: return launch_alg<kApproximate>(c, p, s);
  }
}

}  // namespace fecl
