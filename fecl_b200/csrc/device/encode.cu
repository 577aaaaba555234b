// Device encoders and the BPSK/AWGN channel.
//
// The encoders run the reference's encoding steps with one thread per frame (per
// frame and constituent for turbo codes), so their output is bit-exact with
// LdpcCode::encode / TurboCode::encode and the reference they restate:
//   LDPC  systematic copy, then the sparse XOR steps of Ldpc::Structure::encode
//         (src/detail/Ldpc.cpp:180-209): gap parity from the message (DC), the
//         B correction, the message part of the T rows (A), and the back
//         substitution through T;
//   turbo systematic copy, then per constituent the interleaved message through the
//         trellis and the greedy tail of Convolutional::Structure::encode
//         (src/detail/Convolutional.cpp:167-221), in Turbo::Structure::encode's
//         layout (src/detail/Turbo.cpp:155-170).
// The channel maps bit b to x = 2b - 1, adds N(0, sigma^2) noise with
// sigma^2 = 1 / (2 Es/N0) and returns L = 2 y / sigma^2 (the model of the bench and
// of the reference's test channel).  Its normal variates come from Philox-4x32-10
// (Salmon, Moraes, Dror, Shaw: "Parallel random numbers: as easy as 1, 2, 3",
// SC 2011), counter = (element / 4, seed), and the Box-Muller transform.
#include <math.h>

#include "common.cuh"
#include "kernels.hpp"

namespace fecl {
namespace {

__global__ void ldpc_encode_kernel(LdpcEncodeTables t, const uint8_t* msg, uint8_t* parity, int64_t nframes) {
  const int64_t f = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (f >= nframes) return;
  const uint8_t* m = msg + f * t.K;
  uint8_t* c = parity + f * t.N;
  for (int i = 0; i < t.K; ++i) c[i] = m[i] & 1;
  for (int i = t.K; i < t.N; ++i) c[i] = 0;
  uint8_t* p = c + t.K;
  for (int r = 0; r < t.dc_rows; ++r) {
    uint8_t v = p[r];
    for (uint32_t e = t.dc_ptr[r]; e < t.dc_ptr[r + 1]; ++e) v ^= m[t.dc_idx[e]] & 1;
    p[r] = v;
  }
  for (int r = 0; r < t.b_rows; ++r) {
    uint8_t v = p[t.gap + r];
    for (uint32_t e = t.b_ptr[r]; e < t.b_ptr[r + 1]; ++e) v ^= p[t.b_idx[e]];
    p[t.gap + r] = v;
  }
  uint8_t* p2 = p + t.gap;
  for (int r = 0; r < t.a_rows; ++r) {
    uint8_t v = p2[r];
    for (uint32_t e = t.a_ptr[r]; e < t.a_ptr[r + 1]; ++e) v ^= m[t.a_idx[e]] & 1;
    p2[r] = v;
  }
  for (int r = 0; r < t.t_rows; ++r) {
    const uint8_t v = p2[r];
    if (v)
      for (uint32_t e = t.t_ptr[r] + 1; e < t.t_ptr[r + 1]; ++e) p2[t.t_idx[e]] ^= 1;
  }
}

__device__ __forceinline__ int popc(uint32_t x) { return __popc(x); }

// Thread (frame, constituent j); constituent 0's thread also copies the message.
__global__ void turbo_encode_kernel(TurboDeviceCode code, const uint8_t* msg, uint8_t* parity, int64_t nframes) {
  const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  const int64_t f = t / code.n;
  const int j = int(t - f * code.n);
  if (f >= nframes) return;
  const uint8_t* m = msg + f * code.msg;
  uint8_t* out = parity + f * code.parity;
  if (j == 0)
    for (int i = 0; i < code.msg; ++i) out[i] = m[i] & 1;
  int syst_tail = code.msg, par = code.syst;
  for (int q = 0; q < j; ++q) {
    syst_tail += code.c[q].syst_tail_size;
    par += code.c[q].parity_size;
  }
  const TurboDeviceConstituent& c = code.c[j];
  uint32_t state = 0;
  for (int s = 0; s < c.length; ++s) {
    uint32_t in = 0;
    for (int k = 0; k < c.input_size; ++k) {
      const int i = s * c.input_size + k;
      in |= uint32_t(m[c.perm[i]] & 1) << k;
    }
    const uint32_t o = c.output[state * c.input_count + in];
    state = c.next_state[state * c.input_count + in];
    for (int k = 0; k < c.output_size; ++k) out[par + s * c.output_size + k] = uint8_t((o >> k) & 1);
  }
  int po = par + c.length * c.output_size, to = syst_tail;
  for (int s = 0; s < c.tail; ++s) {
    int best_count = -1;
    uint32_t best = 0;
    for (int u = 0; u < c.input_count; ++u) {
      const int count = popc(state) - popc(c.next_state[state * c.input_count + u]);
      if (count > best_count) {
        best_count = count;
        best = uint32_t(u);
      }
    }
    const uint32_t o = c.output[state * c.input_count + best];
    for (int k = 0; k < c.output_size; ++k) out[po + k] = uint8_t((o >> k) & 1);
    for (int k = 0; k < c.input_size; ++k) out[to + k] = uint8_t((best >> k) & 1);
    po += c.output_size;
    to += c.input_size;
    state = c.next_state[state * c.input_count + best];
  }
}

// Philox-4x32 with 10 rounds (Salmon et al. 2011, Section 4.2): a round multiplies
// the two even words by the round constants, swaps and xors the high halves with the
// odd words and the key; the key is bumped by the Weyl constants between rounds.
struct U4 {
  uint32_t x, y, z, w;
};
__device__ __forceinline__ U4 philox10(U4 ctr, uint32_t k0, uint32_t k1) {
  constexpr uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u, W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    const uint32_t hi0 = __umulhi(M0, ctr.x), lo0 = M0 * ctr.x;
    const uint32_t hi1 = __umulhi(M1, ctr.z), lo1 = M1 * ctr.z;
    ctr = U4{hi1 ^ ctr.y ^ k0, lo1, hi0 ^ ctr.w ^ k1, lo0};
    k0 += W0;
    k1 += W1;
  }
  return ctr;
}

// A uniform in (0, 1] from 32 random bits.
__device__ __forceinline__ float unit(uint32_t v) { return (float(v) + 1.0f) * 2.3283064365386963e-10f; }

__global__ void awgn_kernel(const uint8_t* bits, int64_t n, float sigma, float scale, uint64_t seed, int dtype, void* out) {
  const int64_t q = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;  // one Philox block = 4 elements
  if (q * 4 >= n) return;
  const U4 r = philox10(U4{uint32_t(q), uint32_t(uint64_t(q) >> 32), 0x46654331u, 0u}, uint32_t(seed),
                        uint32_t(seed >> 32));
  float z[4];
  {
    const float rad = sqrtf(-2.0f * logf(unit(r.x)));
    float s, c;
    sincospif(2.0f * unit(r.y), &s, &c);
    z[0] = rad * c;
    z[1] = rad * s;
  }
  {
    const float rad = sqrtf(-2.0f * logf(unit(r.z)));
    float s, c;
    sincospif(2.0f * unit(r.w), &s, &c);
    z[2] = rad * c;
    z[3] = rad * s;
  }
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int64_t i = q * 4 + k;
    if (i < n) {
      const float x = (bits[i] & 1) ? 1.0f : -1.0f;
      store_llr(out, dtype, size_t(i), scale * (x + sigma * z[k]));
    }
  }
}

unsigned blocks_for(int64_t threads, int per_block) {
  const int64_t b = (threads + per_block - 1) / per_block;
  return unsigned(b > 0 ? b : 1);
}

}  // namespace

cudaError_t launch_ldpc_encode(const LdpcEncodeTables& t, const uint8_t* msg, uint8_t* parity, int64_t nframes,
                               cudaStream_t s) {
  if (nframes <= 0) return cudaSuccess;
  ldpc_encode_kernel<<<blocks_for(nframes, 64), 64, 0, s>>>(t, msg, parity, nframes);
  return cudaGetLastError();
}

cudaError_t launch_turbo_encode(const TurboDeviceCode& code, const uint8_t* msg, uint8_t* parity, int64_t nframes,
                                cudaStream_t s) {
  if (nframes <= 0) return cudaSuccess;
  turbo_encode_kernel<<<blocks_for(nframes * code.n, 64), 64, 0, s>>>(code, msg, parity, nframes);
  return cudaGetLastError();
}

cudaError_t launch_awgn(const uint8_t* bits, int64_t n, double esn0, uint64_t seed, int dtype, void* out, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  const double sigma2 = 1.0 / (2.0 * esn0);
  awgn_kernel<<<blocks_for((n + 3) / 4, 256), 256, 0, s>>>(bits, n, float(sqrt(sigma2)), float(2.0 / sigma2), seed,
                                                            dtype, out);
  return cudaGetLastError();
}

}  // namespace fecl
