// Generic turbo decoder, FP32 metrics: any number of constituents, any small
// trellis, Tail or Truncate, Serial or Parallel exchange, all three algorithms.
//
// One thread decodes one frame and walks the same sequence of operations as the
// reference, in FP32:
//   TurboDecoderImpl::decodeBlock / soDecodeBlock (src/detail/TurboDecoder/TurboDecoderImpl.cpp:31-150)
//   serialTransferUpdate / parallelTransferUpdate / aPosterioriUpdate (:152-250)
//   MapDecoderImpl branch/forward/backward/aPosteriori updates
//     (src/detail/MapDecoder/MapDecoderImpl.cpp:80-410), with the log-sum policies of
//     src/detail/LlrMetrics.h:48-121.
// Branch metrics are recomputed from the inputs where the reference stores them;
// forward metrics are stored per step, backward metrics are produced step by step
// together with the a-posteriori outputs.  This is the reference-shaped kernel used
// for arbitrary codes; the LTE code has its own windowed kernel.
#include <math.h>

#include "common.cuh"
#include "kernels.hpp"

namespace fecl {
namespace {

constexpr int kExact = 0, kLinear = 1, kApproximate = 2;
constexpr int kMaxS = 64;  // states
constexpr int kMaxU = 4;   // branches per state
constexpr float kNegInf = -INFINITY;

__constant__ LinearLut c_lut;

// Recursive log-sum (MaxLogSum / LinearLogSum) of two metrics.
template <int ALG>
__device__ __forceinline__ float lsum(float a, float b) {
  if (ALG == kApproximate) return fmaxf(a, b);
  if (a == b) return a;  // LinearLogSum::sum, src/detail/LlrMetrics.h:107-112
  return fmaxf(a, b) + lut_log1pexpm(c_lut, fabsf(a - b));
}

// Exact (LogSum) prior(x, max): 1 when x == max, exp(x - max) otherwise.
__device__ __forceinline__ float eprior(float x, float mx) { return (x == mx) ? 1.0f : expf(x - mx); }

struct Frame {
  float* pin;   // parityIn_  [parity]
  float* pout;  // parityOut_ [parity]
  float* ext;   // extrinsic_ [state]
  float* extb;  // extrinsicBuffer_ [state]
  float* alpha;
};

__device__ __forceinline__ float gamma_of(const TurboDeviceConstituent& k, const float* par, const float* sys, int t,
                                          int s, int u) {
  // correlation of the branch output with the parity L-values, then of the input
  // with the a-priori L-values (MapDecoderImpl.cpp:86-108)
  const uint32_t out = k.output[s * k.input_count + u];
  float g = 0.0f;
  for (int b = 0; b < k.output_size; ++b)
    if ((out >> b) & 1) g += par[t * k.output_size + b];
  float h = 0.0f;
  for (int b = 0; b < k.input_size; ++b)
    if ((u >> b) & 1) h += sys[t * k.input_size + b];
  return g + h;
}

// One MAP pass of constituent k.  sys: a-priori in, extrinsic out (in place).
// par: the constituent's parity L-values.  parity_out: optional parity extrinsic.
// app_out (optional): sf * L of the message steps' input bits (the convolutional
// codec's msg output, MapDecoderImpl.cpp:197-212).
template <int ALG>
__device__ void map_pass(const TurboDeviceConstituent& k, const float* par, float* sys, float* parity_out, float sf,
                         float* alpha, float* app_out = nullptr) {
  const int S = k.state_count, U = k.input_count;
  const int T = k.length + k.tail;
  // forward, MapDecoderImpl.cpp:117-139 (recursive) and :237-274 (LogSum)
  alpha[0] = 0.0f;
  for (int s = 1; s < S; ++s) alpha[s] = kNegInf;
  for (int t = 0; t + 1 < T; ++t) {
    const float* a = alpha + t * S;
    float* an = alpha + (t + 1) * S;
    if (ALG == kExact) {
      float mx[kMaxS], acc[kMaxS];
      for (int s = 0; s < S; ++s) mx[s] = kNegInf;
      for (int s = 0; s < S; ++s)
        for (int u = 0; u < U; ++u) {
          const int n = k.next_state[s * U + u];
          mx[n] = fmaxf(a[s] + gamma_of(k, par, sys, t, s, u), mx[n]);
        }
      for (int s = 0; s < S; ++s) acc[s] = 0.0f;
      for (int s = 0; s < S; ++s)
        for (int u = 0; u < U; ++u) {
          const int n = k.next_state[s * U + u];
          acc[n] = eprior(a[s] + gamma_of(k, par, sys, t, s, u), mx[n]) + acc[n];
        }
      for (int s = 0; s < S; ++s) an[s] = logf(acc[s]) + mx[s];
    } else {
      for (int s = 0; s < S; ++s) an[s] = kNegInf;
      for (int s = 0; s < S; ++s)
        for (int u = 0; u < U; ++u) {
          const int n = k.next_state[s * U + u];
          an[n] = lsum<ALG>(an[n], a[s] + gamma_of(k, par, sys, t, s, u));
        }
    }
    float m = kNegInf;
    for (int s = 0; s < S; ++s) m = fmaxf(an[s], m);
    for (int s = 0; s < S; ++s) an[s] -= m;
  }
  // backward + a-posteriori, MapDecoderImpl.cpp:141-235
  float beta[kMaxS], bprev[kMaxS];
  if (k.termination == 0) {
    beta[0] = 0.0f;
    for (int s = 1; s < S; ++s) beta[s] = kNegInf;
  } else {
    for (int s = 0; s < S; ++s) beta[s] = 0.0f;
  }
  for (int t = T - 1; t >= 0; --t) {
    const float* a = alpha + t * S;
    // delta[s][u] = gamma + alpha + beta(next)
    float delta[kMaxS * kMaxU];
    for (int s = 0; s < S; ++s)
      for (int u = 0; u < U; ++u)
        delta[s * U + u] = gamma_of(k, par, sys, t, s, u) + a[s] + beta[k.next_state[s * U + u]];
    // input bits
    float lin[4];
    for (int j = 0; j < k.input_size; ++j) {
      float r;
      if (ALG == kExact) {
        float mx0 = kNegInf, mx1 = kNegInf, m0 = 0.0f, m1 = 0.0f;
        for (int s = 0; s < S; ++s)
          for (int u = 0; u < U; ++u) {
            if ((u >> j) & 1) mx1 = fmaxf(delta[s * U + u], mx1);
            else mx0 = fmaxf(delta[s * U + u], mx0);
          }
        for (int s = 0; s < S; ++s)
          for (int u = 0; u < U; ++u) {
            if ((u >> j) & 1) m1 = eprior(delta[s * U + u], mx1) + m1;
            else m0 = eprior(delta[s * U + u], mx0) + m0;
          }
        r = (logf(m1) + mx1) - (logf(m0) + mx0);
      } else {
        float m0 = kNegInf, m1 = kNegInf;
        for (int s = 0; s < S; ++s)
          for (int u = 0; u < U; ++u) {
            if ((u >> j) & 1) m1 = lsum<ALG>(m1, delta[s * U + u]);
            else m0 = lsum<ALG>(m0, delta[s * U + u]);
          }
        r = m1 - m0;
      }
      lin[j] = r;
    }
    // parity bits (only when requested)
    if (parity_out) {
      for (int j = 0; j < k.output_size; ++j) {
        float r;
        if (ALG == kExact) {
          float mx0 = kNegInf, mx1 = kNegInf, m0 = 0.0f, m1 = 0.0f;
          for (int s = 0; s < S; ++s)
            for (int u = 0; u < U; ++u) {
              const bool b = (k.output[s * U + u] >> j) & 1;
              if (b) mx1 = fmaxf(delta[s * U + u], mx1);
              else mx0 = fmaxf(delta[s * U + u], mx0);
            }
          for (int s = 0; s < S; ++s)
            for (int u = 0; u < U; ++u) {
              const bool b = (k.output[s * U + u] >> j) & 1;
              if (b) m1 = eprior(delta[s * U + u], mx1) + m1;
              else m0 = eprior(delta[s * U + u], mx0) + m0;
            }
          r = (logf(m1) + mx1) - (logf(m0) + mx0);
        } else {
          float m0 = kNegInf, m1 = kNegInf;
          for (int s = 0; s < S; ++s)
            for (int u = 0; u < U; ++u) {
              const bool b = (k.output[s * U + u] >> j) & 1;
              if (b) m1 = lsum<ALG>(m1, delta[s * U + u]);
              else m0 = lsum<ALG>(m0, delta[s * U + u]);
            }
          r = m1 - m0;
        }
        parity_out[t * k.output_size + j] = sf * (r - par[t * k.output_size + j]);
      }
    }
    // next beta (state after step t-1) from beta and gamma_t
    if (t > 0) {
      if (ALG == kExact) {
        for (int s = 0; s < S; ++s) {
          float mx = kNegInf;
          float buf[kMaxU];
          for (int u = 0; u < U; ++u) {
            buf[u] = beta[k.next_state[s * U + u]] + gamma_of(k, par, sys, t, s, u);
            mx = fmaxf(buf[u], mx);
          }
          float acc = 0.0f;
          for (int u = 0; u < U; ++u) acc = eprior(buf[u], mx) + acc;
          bprev[s] = logf(acc) + mx;
        }
      } else {
        for (int s = 0; s < S; ++s) {
          float acc = kNegInf;
          for (int u = 0; u < U; ++u)
            acc = lsum<ALG>(acc, beta[k.next_state[s * U + u]] + gamma_of(k, par, sys, t, s, u));
          bprev[s] = acc;
        }
      }
      float m = kNegInf;
      for (int s = 0; s < S; ++s) m = fmaxf(bprev[s], m);
      for (int s = 0; s < S; ++s) beta[s] = bprev[s] - m;
    }
    // extrinsic on the input bits, written over the a-priori of this step
    for (int j = 0; j < k.input_size; ++j) {
      const int idx = t * k.input_size + j;
      if (app_out && t < k.length) app_out[idx] = sf * lin[j];
      sys[idx] = sf * (lin[j] - sys[idx]);
    }
  }
}

__device__ void serial_transfer(const TurboDeviceCode& c, Frame& fr, int i) {
  // TurboDecoderImpl::serialTransferUpdate, TurboDecoderImpl.cpp:225-250
  float* syst = fr.pout;
  for (int k = 0; k < c.msg; ++k) syst[k] = fr.pin[k];
  const float* systTail = fr.pin + c.msg;
  float* ext = fr.ext;
  for (int j = 0; j < i; ++j) {
    for (int k = 0; k < c.c[j].msg_size; ++k) syst[c.c[j].perm[k]] += ext[k];
    ext += c.c[j].syst_size;
    systTail += c.c[j].syst_tail_size;
  }
  float* slot = ext;
  ext += c.c[i].msg_size;
  for (int k = 0; k < c.c[i].syst_tail_size; ++k) ext[k] = systTail[k];
  ext += c.c[i].syst_tail_size;
  for (int j = i + 1; j < c.n; ++j) {
    for (int k = 0; k < c.c[j].msg_size; ++k) syst[c.c[j].perm[k]] += ext[k];
    ext += c.c[j].syst_size;
  }
  for (int k = 0; k < c.c[i].msg_size; ++k) slot[k] = syst[c.c[i].perm[k]];
}

__device__ void parallel_transfer(const TurboDeviceCode& c, Frame& fr) {
  // TurboDecoderImpl::parallelTransferUpdate, TurboDecoderImpl.cpp:191-223
  float* ext = fr.ext;
  float* tmp = fr.extb;
  const float* systTail = fr.pin + c.msg;
  float* syst = fr.pout;
  for (int k = 0; k < c.msg; ++k) syst[k] = 0.0f;
  for (int j = 0; j < c.n; ++j) {
    const TurboDeviceConstituent& q = c.c[j];
    for (int k = 0; k < q.msg_size; ++k) {
      tmp[k] = ext[k];
      ext[k] = syst[q.perm[k]];
      syst[q.perm[k]] += tmp[k];
    }
    ext += q.msg_size;
    tmp += q.msg_size;
    for (int k = 0; k < q.syst_tail_size; ++k) ext[k] = systTail[k];
    ext += q.syst_tail_size;
    systTail += q.syst_tail_size;
  }
  for (int k = 0; k < c.msg; ++k) syst[k] = fr.pin[k];
  for (int j = c.n - 1; j >= 0; --j) {
    const TurboDeviceConstituent& q = c.c[j];
    ext -= q.syst_size;
    tmp -= q.msg_size;
    for (int k = 0; k < q.msg_size; ++k) {
      ext[k] += syst[q.perm[k]];
      syst[q.perm[k]] += tmp[k];
    }
  }
}

// Membership in a sorted constituent list [lo, hi), advanced monotonically like the
// reference's iterator walks.
__device__ __forceinline__ bool take(const int32_t* list, int& at, int hi, int j) {
  while (at < hi && list[at] < j) ++at;
  return at < hi && list[at] == j;
}

// TurboDecoderImpl::customTransferUpdate, TurboDecoderImpl.cpp:252-289: the a-priori
// input of activation a (constituent i) is the channel systematic plus the
// de-interleaved extrinsic values of the listed constituents, interleaved into the
// buffer's slot of constituent i; the systematic tail is copied into the live
// extrinsic array (as the reference does), not into the buffer.
__device__ void custom_transfer(const TurboDeviceCode& c, Frame& fr, int a) {
  const int i = c.act_con[a];
  const int t_hi = c.act_tptr[a + 1];
  int at = c.act_tptr[a];
  float* syst = fr.pout;
  for (int k = 0; k < c.msg; ++k) syst[k] = fr.pin[k];
  const float* ext = fr.ext;
  float* tmp = fr.extb;
  const float* systTail = fr.pin + c.msg;
  for (int j = 0; j < i; ++j) {
    if (take(c.transfer, at, t_hi, j))
      for (int k = 0; k < c.c[j].msg_size; ++k) syst[c.c[j].perm[k]] += ext[k];
    ext += c.c[j].syst_size;
    tmp += c.c[j].syst_size;
    systTail += c.c[j].syst_tail_size;
  }
  float* slot = tmp;
  float* tail_dst = fr.ext + (ext - fr.ext) + c.c[i].msg_size;
  for (int k = 0; k < c.c[i].syst_tail_size; ++k) tail_dst[k] = systTail[k];
  ext += c.c[i].syst_size;
  for (int j = i + 1; j < c.n; ++j) {
    if (take(c.transfer, at, t_hi, j)) {
      for (int k = 0; k < c.c[j].msg_size; ++k) syst[c.c[j].perm[k]] += ext[k];
    } else if (at >= t_hi) {
      break;
    }
    ext += c.c[j].syst_size;
  }
  for (int k = 0; k < c.c[i].msg_size; ++k) slot[k] = syst[c.c[i].perm[k]];
}

// TurboDecoderImpl::customActivationUpdate, TurboDecoderImpl.cpp:170-189: the stage's
// constituents, in increasing order, each with the scaling of (iteration, constituent)
// -- in decode and soDecode alike.
template <int ALG>
__device__ void custom_activation(const TurboDeviceCode& c, Frame& fr, int it, int stage) {
  const int hi = c.stage_ptr[stage + 1];
  int at = c.stage_ptr[stage];
  const float* par = fr.pin + c.syst;
  float* ext = fr.ext;
  for (int j = 0; j < c.n; ++j) {
    if (take(c.act_con, at, hi, j)) map_pass<ALG>(c.c[j], par, ext, nullptr, c.sf[j * c.iterations + it], fr.alpha);
    else if (at >= hi) break;
    ext += c.c[j].syst_size;
    par += c.c[j].parity_size;
  }
}

__device__ void aposteriori(const TurboDeviceCode& c, Frame& fr) {
  // TurboDecoderImpl::aPosterioriUpdate, TurboDecoderImpl.cpp:152-168
  const float* ext = fr.ext;
  float* systTail = fr.pout + c.msg;
  float* syst = fr.pout;
  for (int j = 0; j < c.n; ++j) {
    const TurboDeviceConstituent& q = c.c[j];
    for (int k = 0; k < q.msg_size; ++k) syst[q.perm[k]] += ext[k];
    ext += q.msg_size;
    for (int k = 0; k < q.syst_tail_size; ++k) systTail[k] += ext[k];
    ext += q.syst_tail_size;
    systTail += q.syst_tail_size;
  }
}

// CRC stop (an extension): the decisions the frame would end with after this
// iteration -- channel systematic plus every constituent's extrinsic values, as at
// the end of decodeBlock -- and whether their CRC syndrome, the xor of the table
// entries of the bits that are 1, is zero.  Uses the systematic part of parity_buf,
// which every transfer rewrites before it reads it.
__device__ bool crc_passes(const TurboDeviceCode& c, Frame& fr, const uint32_t* crc) {
  for (int k = 0; k < c.msg; ++k) fr.pout[k] = fr.pin[k];
  aposteriori(c, fr);
  uint32_t syn = 0;
  for (int k = 0; k < c.msg; ++k)
    if (fr.pout[k] > 0.0f) syn ^= __ldg(crc + k);
  return syn == 0;
}

template <int ALG>
__global__ void __launch_bounds__(64) turbo_generic_f32(TurboDeviceCode c, TurboRun p) {
  const int64_t f = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (f >= p.nframes) return;
  Frame fr;
  fr.pin = p.parity_in + f * c.parity;
  fr.pout = p.parity_buf + f * c.parity;
  fr.ext = p.ext + f * c.state;
  fr.extb = p.ext_buf + f * c.state;
  fr.alpha = p.alpha + f * int64_t(c.max_steps) * c.max_states;

  for (int k = 0; k < c.parity; ++k) fr.pin[k] = load_llr(p.llr, p.llr_dtype, f * c.parity + k);
  if (p.syst_in)
    for (int k = 0; k < c.syst; ++k) fr.pin[k] += load_llr(p.syst_in, p.llr_dtype, f * c.syst + k);
  for (int k = 0; k < c.state; ++k) fr.ext[k] = p.state_in ? load_llr(p.state_in, p.llr_dtype, f * c.state + k) : 0.0f;
  for (int k = 0; k < c.parity; ++k) fr.pout[k] = 0.0f;

  const bool want_parity = p.soft && p.parity_out;
  if (p.soft && c.iterations == 0 && want_parity)
    for (int k = c.syst; k < c.parity; ++k) fr.pout[k] = 0.0f;

  int ran = c.iterations;
  for (int i = 0; i < c.iterations; ++i) {
    if (c.scheduling == 2) {
      for (int st = 0; st < c.n_stages; ++st) {
        for (int k = 0; k < c.state; ++k) fr.extb[k] = fr.ext[k];
        for (int a = c.stage_ptr[st]; a < c.stage_ptr[st + 1]; ++a) custom_transfer(c, fr, a);
        float* t = fr.ext;
        fr.ext = fr.extb;
        fr.extb = t;
        custom_activation<ALG>(c, fr, i, st);
      }
    } else {
      if (c.scheduling == 1) parallel_transfer(c, fr);
      const float* par = fr.pin + c.syst;
      float* pout = fr.pout + c.syst;
      float* ext = fr.ext;
      for (int j = 0; j < c.n; ++j) {
        if (c.scheduling == 0) serial_transfer(c, fr, j);
        const float sf = p.soft ? 1.0f : c.sf[j * c.iterations + i];
        const bool last = (i == c.iterations - 1);
        map_pass<ALG>(c.c[j], par, ext, (want_parity && last) ? pout : nullptr, sf, fr.alpha);
        ext += c.c[j].syst_size;
        par += c.c[j].parity_size;
        pout += c.c[j].parity_size;
      }
    }
    if (!p.soft && p.crc && i + 1 < c.iterations && crc_passes(c, fr, p.crc)) {
      ran = i + 1;
      break;
    }
  }

  if (!p.soft) {
    for (int k = 0; k < c.msg; ++k) fr.pout[k] = fr.pin[k];
    aposteriori(c, fr);
    for (int k = 0; k < c.msg; ++k) p.hard[f * c.msg + k] = uint8_t(fr.pout[k] > 0.0f);
  } else {
    for (int k = 0; k < c.syst; ++k) fr.pout[k] = 0.0f;
    aposteriori(c, fr);
    if (p.syst_out)
      for (int k = 0; k < c.syst; ++k) store_llr(p.syst_out, p.out_dtype, f * c.syst + k, fr.pout[k]);
    if (p.parity_out)
      for (int k = 0; k < c.parity; ++k) store_llr(p.parity_out, p.out_dtype, f * c.parity + k, fr.pout[k]);
    if (p.state_out)
      for (int k = 0; k < c.state; ++k) store_llr(p.state_out, p.out_dtype, f * c.state + k, fr.ext[k]);
    if (p.msg_out)
      for (int k = 0; k < c.msg; ++k) store_llr(p.msg_out, p.out_dtype, f * c.msg + k, fr.pin[k] + fr.pout[k]);
  }
  if (p.iters) p.iters[f] = ran;
}

// The convolutional codec's soDecode (Convolutional::soDecodeBlocks ->
// MapDecoderImpl::soDecodeBlock, src/detail/MapDecoder/MapDecoderImpl.cpp:56-78,
// :174-235): one MAP pass over the trellis per frame, one thread per frame.
template <int ALG>
__global__ void __launch_bounds__(64) conv_map_f32(TurboDeviceConstituent k, ConvMapRun r) {
  const int64_t f = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (f >= r.nframes) return;
  const int P = k.parity_size, Sy = k.syst_size, M = k.msg_size;
  const int T = k.length + k.tail;
  float* par = r.par + f * P;
  float* sys = r.sys + f * Sy;
  float* pout = r.parity_out ? r.pout + f * P : nullptr;
  float* app = r.app + f * M;
  float* alpha = r.alpha + f * int64_t(T) * k.state_count;
  for (int i = 0; i < P; ++i) par[i] = load_llr(r.llr, r.llr_dtype, f * P + i);
  for (int i = 0; i < Sy; ++i) sys[i] = r.syst_in ? load_llr(r.syst_in, r.llr_dtype, f * Sy + i) : 0.0f;
  map_pass<ALG>(k, par, sys, pout, r.sf, alpha, app);
  if (r.msg_out)
    for (int i = 0; i < M; ++i) store_llr(r.msg_out, r.out_dtype, f * M + i, app[i]);
  if (r.syst_out)
    for (int i = 0; i < Sy; ++i) store_llr(r.syst_out, r.out_dtype, f * Sy + i, sys[i]);
  if (r.parity_out)
    for (int i = 0; i < P; ++i) store_llr(r.parity_out, r.out_dtype, f * P + i, pout[i]);
}

}  // namespace

cudaError_t turbo_generic_init() {
  static std::atomic<unsigned long long> done{0};
  return once_per_device(done, [] {
    const LinearLut l = make_linear_lut();
    return cudaMemcpyToSymbol(c_lut, &l, sizeof(l));
  });
}

cudaError_t launch_turbo_generic(const TurboDeviceCode& c, const TurboRun& p, cudaStream_t s) {
  cudaError_t e0 = turbo_generic_init();
  if (e0 != cudaSuccess) return e0;
  if (p.nframes <= 0) return cudaSuccess;
  if (c.max_states > kMaxS) return cudaErrorInvalidValue;
  for (int j = 0; j < c.n; ++j)
    if (c.c[j].input_count > kMaxU || c.c[j].input_size > 4) return cudaErrorInvalidValue;
  const dim3 block(64), grid(unsigned((p.nframes + 63) / 64));
  switch (c.algorithm) {
    case kExact: turbo_generic_f32<kExact><<<grid, block, 0, s>>>(c, p); break;
    case kLinear: turbo_generic_f32<kLinear><<<grid, block, 0, s>>>(c, p); break;
    default: turbo_generic_f32<kApproximate><<<grid, block, 0, s>>>(c, p); break;
  }
  return cudaGetLastError();
}

size_t conv_map_scratch_bytes(const TurboDeviceConstituent& k, int64_t nframes) {
  const int64_t T = k.length + k.tail;
  return size_t(nframes) * size_t(2 * k.parity_size + k.syst_size + k.msg_size + T * k.state_count) * sizeof(float) + 1024;
}

cudaError_t launch_conv_map(const TurboDeviceConstituent& k, ConvMapRun r, void* scratch, cudaStream_t s) {
  cudaError_t e = turbo_generic_init();
  if (e != cudaSuccess) return e;
  if (r.nframes <= 0) return cudaSuccess;
  if (k.state_count > kMaxS || k.input_count > kMaxU) return cudaErrorInvalidValue;
  float* q = static_cast<float*>(scratch);
  r.par = q;
  q += r.nframes * k.parity_size;
  r.pout = q;
  q += r.nframes * k.parity_size;
  r.sys = q;
  q += r.nframes * k.syst_size;
  r.app = q;
  q += r.nframes * k.msg_size;
  r.alpha = q;
  const unsigned blocks = unsigned((r.nframes + 63) / 64);
  switch (r.algorithm) {
    case kExact: conv_map_f32<kExact><<<blocks, 64, 0, s>>>(k, r); break;
    case kLinear: conv_map_f32<kLinear><<<blocks, 64, 0, s>>>(k, r); break;
    default: conv_map_f32<kApproximate><<<blocks, 64, 0, s>>>(k, r); break;
  }
  return cudaGetLastError();
}

}  // namespace fecl
