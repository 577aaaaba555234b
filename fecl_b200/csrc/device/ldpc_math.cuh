// Check-node arithmetic shared by the batched LDPC kernels (ldpc_lanes.cu,
// ldpc_cluster.cu), so that every batched path computes the same FP32 values bit
// for bit.
//
// One check row of degree d: the inputs v[j] = APP(bit j) - c2v(edge j) come in,
// the scaled extrinsic outputs c2v'(edge j) = sf * (boxplus over the other d-1
// inputs) go out, in the forward / backward order of BpDecoderImpl::checkUpdate
// (src/detail/BpDecoder/BpDecoderImpl.cpp:132-159) with the boxplus policies of
// src/detail/LlrMetrics.h:126-196.
#pragma once

#include <cuda_fp16.h>
#include <math.h>
#include <stdint.h>

#include "common.cuh"

namespace fecl {
namespace ldpc {

constexpr int kExact = 0, kLinear = 1, kApproximate = 2;

__device__ __forceinline__ bool neg(float x) { return (__float_as_uint(x) >> 31) != 0; }

// LinearBoxSum::sum, src/detail/LlrMetrics.h:152-159.
__device__ __forceinline__ float box_linear(const LinearLut& lut, float a, float b) {
  const float m = fminf(fabsf(a), fabsf(b));
  const float s = (neg(a) != neg(b)) ? m : -m;
  return s - lut_log1pexpm(lut, fabsf(a + b)) + lut_log1pexpm(lut, fabsf(a - b));
}

// phi(x) = -log(tanh(x/2)), its own inverse.  BoxSum (src/detail/LlrMetrics.h:126-140)
// multiplies tanh(-x/2) over a row and maps back with -2 atanh; in the phi domain the
// same boxplus is a sum of phi(|x|) and a sign parity, which keeps FP32 accurate where
// tanh rounds to +-1.  Inputs are clamped to 80 so phi stays normal.
__device__ __forceinline__ float phi(float x) { return ldpc_phi(x); }

// Storage of check-to-bit messages: FP32 (reference parity), saturated FP16 (+-65504),
// or saturated int8 in Q5.2 (step 1/4, range +-31.75).  Arithmetic is FP32 in every case.
// encode() is odd -- encode(-x) == negate(encode(x)) bit for bit -- because rounding
// to nearest (even) and the saturation bounds are symmetric in sign.
template <int MSG>
struct Msg;
template <>
struct Msg<0> {
  using T = float;
  __device__ static float load(const T* p) { return *p; }
  __device__ static T encode(float v) { return v; }
  __device__ static T negate(T q) { return -q; }
  __device__ static void store(T* p, float v) { *p = encode(v); }
  __device__ static float from_bits(uint32_t b) { return __uint_as_float(b); }
};
template <>
struct Msg<1> {
  using T = __half;
  __device__ static float load(const T* p) { return __half2float(*p); }
  // saturated at the largest finite FP16 value, so that no message becomes infinite
  __device__ static T encode(float v) { return __float2half_rn(fminf(fmaxf(v, -65504.0f), 65504.0f)); }
  __device__ static T negate(T q) { return __ushort_as_half((unsigned short)(__half_as_ushort(q) ^ 0x8000u)); }
  __device__ static void store(T* p, float v) { *p = encode(v); }
  __device__ static float from_bits(uint32_t b) { return __half2float(__ushort_as_half((unsigned short)b)); }
};
template <>
struct Msg<2> {
  using T = int8_t;
  __device__ static float load(const T* p) { return float(*p) * 0.25f; }
  __device__ static T encode(float v) { return int8_t(fminf(fmaxf(rintf(v * 4.0f), -127.0f), 127.0f)); }
  __device__ static T negate(T q) { return int8_t(-q); }
  __device__ static void store(T* p, float v) { *p = encode(v); }
  __device__ static float from_bits(uint32_t b) { return float(int8_t(uint8_t(b))) * 0.25f; }
};

// Min-sum scan of one row: the two smallest magnitudes m1 <= m2, the index of the
// first smallest, and the parity of the inputs' sign bits.
template <int DMAX>
__device__ __forceinline__ void min_sum_scan(const float v[DMAX], int d, float& m1, float& m2, int& i1,
                                             unsigned& par) {
  m1 = INFINITY;
  m2 = INFINITY;
  i1 = 0;
  par = 0;
#pragma unroll
  for (int j = 0; j < DMAX; ++j) {
    if (j < d) {
      const float a = fabsf(v[j]);
      par ^= unsigned(neg(v[j]));
      const bool lt1 = a < m1;
      m2 = lt1 ? m1 : fminf(m2, a);
      i1 = lt1 ? j : i1;
      m1 = lt1 ? a : m1;
    }
  }
}

// One check row: v[0..d) in, out[0..d) = sf * extrinsic boxplus out.
template <int ALG, int DMAX>
__device__ __forceinline__ void row_update(const LinearLut& lut, const float v[DMAX], float out[DMAX], int d,
                                           float sf) {
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
    // Written with selects, not branches: lanes hold different frames, and a branch
    // on the data would split the warp at every edge.
    float m1, m2;
    int i1;
    unsigned par;
    min_sum_scan<DMAX>(v, d, m1, m2, i1, par);
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
      if (j < d - 1) fwd[j] = box_linear(lut, fwd[j - 1], v[j]);
    float bwd = 0.0f;
#pragma unroll
    for (int j = DMAX - 1; j >= 0; --j) {
      if (j < d) {
        const int jp = j > 0 ? j - 1 : 0;
        float o;
        if (j == d - 1) o = fwd[jp];
        else if (j == 0) o = bwd;
        else o = box_linear(lut, fwd[jp], bwd);
        out[j] = sf * o;
        if (j == d - 1) bwd = v[j];
        else bwd = box_linear(lut, bwd, v[j]);
      }
    }
  }
}

}  // namespace ldpc
}  // namespace fecl
