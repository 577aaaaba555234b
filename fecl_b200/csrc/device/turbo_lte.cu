// Windowed turbo decoder for two 8-state rate-1/2 constituents with Tail
// termination (the LTE code of 3GPP TS 36.212 and every code of that shape),
// serial scheduling, hard-decision decode, FP32 metrics.
//
// What it computes is the reference's full-frame BCJR (MapDecoderImpl,
// src/detail/MapDecoder/MapDecoderImpl.cpp:80-235) inside the serial turbo loop
// (TurboDecoderImpl::decodeBlock, src/detail/TurboDecoder/TurboDecoderImpl.cpp:31-72);
// how it computes it is B200-shaped:
//
//   One CTA of 2 * SEGS threads decodes one frame for all iterations.  The frame's
//   two exchange arrays live in shared memory in natural bit order:
//     X[k] = Ls[k] + e0[k]          (a-priori of constituent 1 before interleaving;
//                                    also the partial a-posteriori sum)
//     Y[k] = e1 at natural index k  (constituent 1 writes e1(t) to Y[pi(t)])
//   so constituent 0 reads Ls + Y contiguously and constituent 1 gathers X[pi(t)].
//
//   Per half-iteration:
//   A. SEGS forward and SEGS backward segments run concurrently (one thread each).
//      A segment starts from metrics obtained by a training run of G steps from a
//      flat start, walks its steps and leaves metric checkpoints every 8 steps in
//      global memory (L2) plus its end metrics in shared memory.
//   A2. Verification.  Segment 0 (forward) and the last segment (backward) start
//      from the exact trellis termination.  The training start of segment w is
//      accepted when it matches, within FP32 rounding (close8), the end metrics
//      that segment w-1 computed from its own accepted start; otherwise segment w
//      is walked again from that end, until its metrics reproduce a checkpoint of
//      the earlier walk.  Rounds repeat until every boundary is accepted, so every
//      checkpoint equals the full-frame recursion up to rounding.  (Max-log and
//      log-MAP forget their start exponentially fast; training merely makes
//      fix-ups rare.)
//   B. Every 8-step block is then independent: a thread reloads the forward
//      checkpoint at the block start and the backward checkpoint at its end,
//      recomputes the 8 forward vectors in registers and walks backward emitting
//      the extrinsic values, scaled, minus the a-priori (MapDecoderImpl.cpp:203-212).
//
// The recursions subtract the largest state metric once per 8-step chunk (at every
// checkpoint) rather than after every step as the reference does: the subtraction
// cancels in every difference the decoder takes, so this changes FP32 rounding only,
// and it removes the eight-way maximum and the subtractions from seven steps of
// eight.  Global loads of the next chunk are issued one chunk ahead.
//
// Inputs are first converted into a padded FP32 scratch layout so that every
// block load is 16-byte aligned.
#include <math.h>

#include <map>
#include <mutex>
#include <utility>

#include "common.cuh"
#include "kernels.hpp"

namespace fecl {
namespace {

constexpr int kExact = 0, kLinear = 1, kApproximate = 2;
constexpr int kBlk = 8;  // checkpoint spacing / APP block length
constexpr float kNegInf = -INFINITY;
// Boundary acceptance: |x - y| <= abs + rel * max(|x|, |y|).  Two walks that have
// forgotten their starts differ by the rounding of the steps since, which grows with
// the metrics' magnitude (strong a-priori values late in a decode).  An accepted
// difference reaches the extrinsic values at most doubled, so soDecode, whose soft
// outputs must stay within 1e-4 relative of the reference, accepts only differences
// two orders of magnitude below that; decode, which outputs hard decisions, accepts
// 1e-3 (+ 1e-5 relative), which saves fix-up walks.
struct Tol {
  float abs, rel;
};
constexpr Tol kDecodeTol = {1e-3f, 1e-5f};
constexpr Tol kSoftTol = {1e-6f, 1e-6f};
constexpr int kDefaultSegs = 64;

__constant__ LinearLut c_lut;

// The LTE RSC, Trellis({4}, {{015}}, {013}) (src/Trellis.cpp:76-143): with state bits
// s0 s1 s2, the feedback bit is u ^ s0 ^ s1, the next state shifts it in at the top
// and the parity output is u ^ s1 ^ s2.  Compile-time tables keep every metric in
// registers.
__host__ __device__ constexpr int lte_next(int s, int u) { return (s >> 1) | (((u ^ s ^ (s >> 1)) & 1) << 2); }
__host__ __device__ constexpr int lte_out(int s, int u) { return (u ^ (s >> 1) ^ (s >> 2)) & 1; }

template <int ALG>
__device__ __forceinline__ float lsum(float a, float b) {
  if (ALG == kApproximate) return fmaxf(a, b);
  if (a == b) return a;
  return fmaxf(a, b) + lut_log1pexpm(c_lut, fabsf(a - b));
}

// max(a, b, c) in one instruction (the three-input form of max.f32, sm_100): the same
// value as fmaxf(fmaxf(a, b), c), a maximum being exact.
__device__ __forceinline__ float fmax3(float a, float b, float c) {
  float r;
  asm("max.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
  return r;
}

// v[s] -= max(v), with the subtraction as four packed f32x2 adds of -m (x - m is
// x + (-m) exactly).
__device__ __forceinline__ void normalize8(float v[8]) {
  const float m = fmax3(fmax3(v[0], v[1], v[2]), fmax3(v[3], v[4], v[5]), fmaxf(v[6], v[7]));
  const float2 nm = make_float2(-m, -m);
#pragma unroll
  for (int s = 0; s < 8; s += 2) {
    const float2 r = __fadd2_rn(make_float2(v[s], v[s + 1]), nm);
    v[s] = r.x;
    v[s + 1] = r.y;
  }
}

// Two-term log-sum in the Exact (LogSum) form: max, then exp-sum, then log.  The
// exponentials take arguments <= 0 and the logarithm arguments in [1, 16], where the
// hardware approximations (__expf, __logf) are within about 2^-22 relative and 2^-21
// absolute: every metric and extrinsic value moves by less than 1e-6 absolute per
// step, far inside the soft-output rule (1e-4 relative, 1e-4 absolute below 1), at a
// few instructions each instead of the accurate functions' range reductions.
__device__ __forceinline__ float esum2(float x0, float x1) {
  const float m = fmaxf(x0, x1);
  const float a = (x0 == m) ? 1.0f : __expf(x0 - m);
  const float b = (x1 == m) ? 1.0f : __expf(x1 - m);
  return __logf(a + b) + m;
}

struct Gam {
  float g[4];  // index (u << 1) | p : 0, Lp, La, La + Lp
  __device__ __forceinline__ void set(float la, float lp) {
    g[0] = 0.0f;
    g[1] = lp;
    g[2] = la;
    g[3] = lp + la;
  }
  // x + gamma(s, u).  In max-log the branch with no 1 bits adds nothing: x + 0 is x for
  // every metric but -0, and a -0 metric (x == 0) only ever meets +0 in a maximum or a
  // difference, which treat both alike; the other algorithms keep the reference's adds.
  template <int ALG>
  __device__ __forceinline__ float plus(float x, int s, int u) const {
    const int i = (u << 1) | lte_out(s, u);
    if (ALG == kApproximate && i == 0) return x;
    return x + g[i];
  }
};

// The log-MAP recursions keep the reference's normalisation after every step (max-log
// normalises once per chunk, see above): their table and exp/log corrections are not
// translation-invariant in FP32, so this keeps their rounding that of the reference.
template <int ALG>
__device__ __forceinline__ void normalize_step(float v[8]) {
  if constexpr (ALG != kApproximate) {
    float m = kNegInf;
#pragma unroll
    for (int s = 0; s < 8; ++s) m = fmaxf(v[s], m);
#pragma unroll
    for (int s = 0; s < 8; ++s) v[s] = v[s] - m;
  }
}

// alpha_{t+1} from alpha_t (MapDecoderImpl.cpp:117-139, :237-274); normalised here only
// by the log-MAP algorithms.
template <int ALG>
__device__ __forceinline__ void fwd_step(float a[8], const Gam& g) {
  float c0[8], c1[8];
  bool first[8];
#pragma unroll
  for (int s = 0; s < 8; ++s) first[s] = true;
#pragma unroll
  for (int s = 0; s < 8; ++s)
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      const int d = lte_next(s, u);
      const float v = g.plus<ALG>(a[s], s, u);
      if (first[d]) {
        c0[d] = v;
        first[d] = false;
      } else {
        c1[d] = v;
      }
    }
#pragma unroll
  for (int s = 0; s < 8; ++s) {
    if (ALG == kExact) a[s] = esum2(c0[s], c1[s]);
    else if (ALG == kApproximate) a[s] = fmaxf(c0[s], c1[s]);
    // Linear: the reference's accumulation starts from -inf, and lsum(-inf, c) is c
    // (the table gives 0 beyond 3.5), so it is left out; only a -0 metric would come
    // out as +0, which every later maximum and difference treats alike
    else a[s] = lsum<ALG>(c0[s], c1[s]);
  }
  normalize_step<ALG>(a);
}

// beta_t from beta_{t+1} (MapDecoderImpl.cpp:141-172, :276-329); normalised here only by
// the log-MAP algorithms.
template <int ALG>
__device__ __forceinline__ void bwd_step(float b[8], const Gam& g) {
  float n[8];
#pragma unroll
  for (int s = 0; s < 8; ++s) {
    const float x0 = g.plus<ALG>(b[lte_next(s, 0)], s, 0);
    const float x1 = g.plus<ALG>(b[lte_next(s, 1)], s, 1);
    if (ALG == kExact) n[s] = esum2(x0, x1);
    else if (ALG == kApproximate) n[s] = fmaxf(x0, x1);
    else n[s] = lsum<ALG>(x0, x1);  // as in fwd_step
  }
#pragma unroll
  for (int s = 0; s < 8; ++s) b[s] = n[s];
  normalize_step<ALG>(b);
}

// Extrinsic value of one step, L(u) - La (msgUpdateImpl, MapDecoderImpl.cpp:331-376).
// Max-log: L(u=1) = La + max_s(a[s] + b[next(s,1)] + p(s,1) Lp) and L(u=0) =
// max_s(a[s] + b[next(s,0)] + p(s,0) Lp), so the a-priori value cancels and each
// maximum splits by parity bit: the states with p(s,0) = 1 are 2..5 (and with
// p(s,1) = 1 the others), so Lp is added once per maximum instead of once per state.
template <int ALG>
__device__ __forceinline__ float ext_step(const float a[8], const float b[8], const Gam& g) {
  if constexpr (ALG == kApproximate) {
    float w0[8], w1[8];
#pragma unroll
    for (int s = 0; s < 8; ++s) {
      w0[s] = a[s] + b[lte_next(s, 0)];
      w1[s] = a[s] + b[lte_next(s, 1)];
    }
    const float lp = g.g[1];
    // u = 0: parity 0 at s in {0,1,6,7}, parity 1 at {2,3,4,5}; u = 1 the reverse.
    const float m0p0 = fmax3(fmaxf(w0[0], w0[1]), w0[6], w0[7]);
    const float m0p1 = fmax3(fmaxf(w0[2], w0[3]), w0[4], w0[5]);
    const float m1p0 = fmax3(fmaxf(w1[2], w1[3]), w1[4], w1[5]);
    const float m1p1 = fmax3(fmaxf(w1[0], w1[1]), w1[6], w1[7]);
    const float m0 = fmaxf(m0p0, m0p1 + lp);
    const float m1 = fmaxf(m1p0, m1p1 + lp);
    return m1 - m0;
  } else {
    float d[16];
#pragma unroll
    for (int s = 0; s < 8; ++s)
#pragma unroll
      for (int u = 0; u < 2; ++u) d[s * 2 + u] = g.plus<ALG>(a[s], s, u) + b[lte_next(s, u)];
    float l;
    if (ALG == kExact) {
      float mx0 = kNegInf, mx1 = kNegInf;
#pragma unroll
      for (int s = 0; s < 8; ++s) {
        mx0 = fmaxf(d[s * 2], mx0);
        mx1 = fmaxf(d[s * 2 + 1], mx1);
      }
      float m0 = 0.0f, m1 = 0.0f;
#pragma unroll
      for (int s = 0; s < 8; ++s) {
        m0 = ((d[s * 2] == mx0) ? 1.0f : __expf(d[s * 2] - mx0)) + m0;
        m1 = ((d[s * 2 + 1] == mx1) ? 1.0f : __expf(d[s * 2 + 1] - mx1)) + m1;
      }
      l = (__logf(m1) + mx1) - (__logf(m0) + mx0);  // esum2's approximations
    } else {
      float m0 = kNegInf, m1 = kNegInf;
#pragma unroll
      for (int s = 0; s < 8; ++s) {
        m0 = lsum<ALG>(m0, d[s * 2]);
        m1 = lsum<ALG>(m1, d[s * 2 + 1]);
      }
      l = m1 - m0;
    }
    return l - g.g[2];
  }
}

// Parity extrinsic value of one step, L(p) - Lp (parityUpdate, MapDecoderImpl.cpp:
// 376-410), for soDecode's parity output.  Max-log: the branches with p = 1 are
// (s in 2..5, u = 0) and (s in {0,1,6,7}, u = 1); Lp cancels and La is added once per
// maximum.
template <int ALG>
__device__ __forceinline__ float par_step(const float a[8], const float b[8], const Gam& g) {
  if constexpr (ALG == kApproximate) {
    float w0[8], w1[8];
#pragma unroll
    for (int s = 0; s < 8; ++s) {
      w0[s] = a[s] + b[lte_next(s, 0)];
      w1[s] = a[s] + b[lte_next(s, 1)];
    }
    const float la = g.g[2];
    const float m0p0 = fmax3(fmaxf(w0[0], w0[1]), w0[6], w0[7]);
    const float m0p1 = fmax3(fmaxf(w0[2], w0[3]), w0[4], w0[5]);
    const float m1p0 = fmax3(fmaxf(w1[2], w1[3]), w1[4], w1[5]);
    const float m1p1 = fmax3(fmaxf(w1[0], w1[1]), w1[6], w1[7]);
    return fmaxf(m0p1, m1p1 + la) - fmaxf(m0p0, m1p0 + la);
  } else {
    float d[16];
#pragma unroll
    for (int s = 0; s < 8; ++s)
#pragma unroll
      for (int u = 0; u < 2; ++u) d[s * 2 + u] = g.plus<ALG>(a[s], s, u) + b[lte_next(s, u)];
    float l;
    if (ALG == kExact) {
      float mx0 = kNegInf, mx1 = kNegInf;
#pragma unroll
      for (int s = 0; s < 8; ++s)
#pragma unroll
        for (int u = 0; u < 2; ++u) {
          if (lte_out(s, u)) mx1 = fmaxf(d[s * 2 + u], mx1);
          else mx0 = fmaxf(d[s * 2 + u], mx0);
        }
      float m0 = 0.0f, m1 = 0.0f;
#pragma unroll
      for (int s = 0; s < 8; ++s)
#pragma unroll
        for (int u = 0; u < 2; ++u) {
          const float x = d[s * 2 + u];
          if (lte_out(s, u)) m1 = ((x == mx1) ? 1.0f : __expf(x - mx1)) + m1;
          else m0 = ((x == mx0) ? 1.0f : __expf(x - mx0)) + m0;
        }
      l = (__logf(m1) + mx1) - (__logf(m0) + mx0);  // esum2's approximations
    } else {
      float m0 = kNegInf, m1 = kNegInf;
#pragma unroll
      for (int s = 0; s < 8; ++s)
#pragma unroll
        for (int u = 0; u < 2; ++u) {
          if (lte_out(s, u)) m1 = lsum<ALG>(m1, d[s * 2 + u]);
          else m0 = lsum<ALG>(m0, d[s * 2 + u]);
        }
      l = m1 - m0;
    }
    return l - g.g[1];
  }
}

struct Frame {
  const float* Ls;   // [Tp] systematic L-values, zero past K
  const float* Lp0;  // [Tp]  parity (with tail parity) of constituent 0
  const float* Lp1;  // [Tp]
  const float* ts;   // [8]   tail systematic of constituent 0 (3) then 1 (3)
  float* cka;        // [nblk + 1][8]
  float* ckb;        // [nblk + 1][8]
};

// A segment's boundary vectors: a forward segment's start (after training) is its
// first checkpoint and a backward segment's end its last, so those two stay in the
// checkpoint arrays (global memory); the other two are kept here.
template <int SEGS>
struct Shared {
  float bwd_start[SEGS][8];  // backward segment w's metrics at its end a1 after training
  float fwd_end[SEGS][8];    // forward segment w's metrics at a1
  float flat[8];             // training start: all states equal
  float term[8];             // trellis termination: state 0
  uint32_t crc_part[2 * SEGS / 32];  // per-warp CRC syndromes
};

// The global loads of one 8-step chunk [8c, 8c + 8): the parity L-values and either
// the systematic L-values (constituent 0) or the interleaver entries (constituent 1).
// Every array read here is padded to Tp = 8 * nblk entries, so the vector loads stay
// inside the frame's scratch even for the chunk holding the tail steps.
struct RawChunk {
  float4 p0, p1;  // parity
  uint4 q0, q1;   // systematic (as bits) or interleaver entries
};

__device__ __forceinline__ void load_raw(int j, int c, const Frame& fr, const uint32_t* __restrict__ perm,
                                         RawChunk& r) {
  const int t0 = c * kBlk;
  const float* Lp = j == 0 ? fr.Lp0 : fr.Lp1;
  r.p0 = __ldg(reinterpret_cast<const float4*>(Lp + t0));
  r.p1 = __ldg(reinterpret_cast<const float4*>(Lp + t0) + 1);
  const uint4* q = j == 0 ? reinterpret_cast<const uint4*>(fr.Ls + t0) : reinterpret_cast<const uint4*>(perm + t0);
  r.q0 = __ldg(q);
  r.q1 = __ldg(q + 1);
}

// A chunk's a-priori and parity L-values.
struct Chunk {
  float la[kBlk];
  float lp[kBlk];
};

__device__ __forceinline__ void resolve(int j, int c, int K, const Frame& fr, const float* X, const float* Y,
                                        const RawChunk& r, Chunk& ch) {
  const int t0 = c * kBlk;
  ch.lp[0] = r.p0.x; ch.lp[1] = r.p0.y; ch.lp[2] = r.p0.z; ch.lp[3] = r.p0.w;
  ch.lp[4] = r.p1.x; ch.lp[5] = r.p1.y; ch.lp[6] = r.p1.z; ch.lp[7] = r.p1.w;
  if (j == 0) {
    const float4 y0 = reinterpret_cast<const float4*>(Y + t0)[0];
    const float4 y1 = reinterpret_cast<const float4*>(Y + t0)[1];
    ch.la[0] = __uint_as_float(r.q0.x) + y0.x; ch.la[1] = __uint_as_float(r.q0.y) + y0.y;
    ch.la[2] = __uint_as_float(r.q0.z) + y0.z; ch.la[3] = __uint_as_float(r.q0.w) + y0.w;
    ch.la[4] = __uint_as_float(r.q1.x) + y1.x; ch.la[5] = __uint_as_float(r.q1.y) + y1.y;
    ch.la[6] = __uint_as_float(r.q1.z) + y1.z; ch.la[7] = __uint_as_float(r.q1.w) + y1.w;
  } else {
    ch.la[0] = X[r.q0.x]; ch.la[1] = X[r.q0.y]; ch.la[2] = X[r.q0.z]; ch.la[3] = X[r.q0.w];
    ch.la[4] = X[r.q1.x]; ch.la[5] = X[r.q1.y]; ch.la[6] = X[r.q1.z]; ch.la[7] = X[r.q1.w];
  }
  if (t0 + kBlk > K) {
#pragma unroll
    for (int i = 0; i < kBlk; ++i) {
      const int t = t0 + i;
      if (t >= K) ch.la[i] = (t < K + 3) ? fr.ts[j * 3 + (t - K)] : 0.0f;
    }
  }
}

__device__ __forceinline__ void store_ck(float* ck, const float v[8]) {
  float4* q = reinterpret_cast<float4*>(ck);
  q[0] = make_float4(v[0], v[1], v[2], v[3]);
  q[1] = make_float4(v[4], v[5], v[6], v[7]);
}

__device__ __forceinline__ void load_ck(const float* ck, float v[8]) {
  const float4* q = reinterpret_cast<const float4*>(ck);
  const float4 c0 = q[0], c1 = q[1];
  v[0] = c0.x; v[1] = c0.y; v[2] = c0.z; v[3] = c0.w;
  v[4] = c1.x; v[5] = c1.y; v[6] = c1.z; v[7] = c1.w;
}

__device__ __forceinline__ bool close8(const float* x, const float* y, Tol t) {
  bool ok = true;
#pragma unroll
  for (int s = 0; s < 8; ++s) {
    const float tol = t.abs + t.rel * fmaxf(fabsf(x[s]), fabsf(y[s]));
    ok = ok && ((x[s] == y[s]) || fabsf(x[s] - y[s]) <= tol);
  }
  return ok;
}

// One segment walk of constituent j, forward (fwd != 0) or backward.  The start
// metrics are read from vin (shared memory).  Training steps outside the segment
// run first without checkpoints -- forward over [t_train, a0), backward over
// [a1, t_train) -- then the metrics at the segment boundary are written to vstart,
// the segment's own steps run, leaving checkpoints at every multiple of 8 inside
// [a0, a1) (and at T for the last backward segment), and the final metrics go to
// vend.  Metrics are normalised at the end of every chunk, so every checkpoint and
// both boundary vectors have their largest state at 0.  The global loads of chunk
// c + 1 are issued before chunk c runs.  A fix-up walk (`refine`) starts from a
// corrected boundary over checkpoints an earlier walk of the same segment left; it
// stops at the first checkpoint its metrics reproduce (close8): from there on the
// earlier walk is the same recursion, so its checkpoints and end stand.  Kept out of
// line so that Phase A and the fix-up rounds share one copy of the code.
template <int ALG>
__device__ __noinline__ void segment_walk(int fwd, int j, int t_train, int a0, int a1, const float* vin, float* vstart,
                                          float* vend, int K, int T, Frame fr, const float* X, const float* Y,
                                          const uint32_t* perm, bool refine, Tol tol) {
  float v[8];
#pragma unroll
  for (int s = 0; s < 8; ++s) v[s] = vin[s];
  if (fwd) {
    const int c_end = (a1 + kBlk - 1) / kBlk;
    int c = t_train / kBlk;
    RawChunk nxt;
    load_raw(j, c, fr, perm, nxt);
    for (; c < c_end; ++c) {
      const RawChunk cur = nxt;
      if (c + 1 < c_end) load_raw(j, c + 1, fr, perm, nxt);
      const int t0 = c * kBlk;
      if (t0 == a0 && vstart) {
#pragma unroll
        for (int s = 0; s < 8; ++s) vstart[s] = v[s];
      }
      if (t0 >= a0) {
        if (refine && t0 > a0) {
          float old[8];
          load_ck(fr.cka + c * 8, old);
          if (close8(v, old, tol)) return;
        }
        store_ck(fr.cka + c * 8, v);
      }
      Chunk ch;
      resolve(j, c, K, fr, X, Y, cur, ch);
      const int n = min(kBlk, a1 - t0);
      if (n == kBlk) {  // every chunk but the frame's last: no per-step tests
#pragma unroll
        for (int i = 0; i < kBlk; ++i) {
          Gam g;
          g.set(ch.la[i], ch.lp[i]);
          fwd_step<ALG>(v, g);
        }
      } else {
#pragma unroll
        for (int i = 0; i < kBlk; ++i) {
          if (i < n) {
            Gam g;
            g.set(ch.la[i], ch.lp[i]);
            fwd_step<ALG>(v, g);
          }
        }
      }
      normalize8(v);
    }
  } else {
    const int nblk = (T + kBlk - 1) / kBlk;
    if (t_train == a1) {
      if (vstart) {
#pragma unroll
        for (int s = 0; s < 8; ++s) vstart[s] = v[s];
      }
      if (a1 == T) store_ck(fr.ckb + nblk * 8, v);
    }
    const int c_lo = a0 / kBlk;
    int c = (t_train - 1) / kBlk;
    RawChunk nxt;
    load_raw(j, c, fr, perm, nxt);
    for (; c >= c_lo; --c) {
      const RawChunk cur = nxt;
      if (c - 1 >= c_lo) load_raw(j, c - 1, fr, perm, nxt);
      Chunk ch;
      resolve(j, c, K, fr, X, Y, cur, ch);
      const int hi = min(kBlk, t_train - c * kBlk);
      if (hi == kBlk) {  // every chunk but the frame's last: no per-step tests
#pragma unroll
        for (int i = kBlk - 1; i >= 0; --i) {
          Gam g;
          g.set(ch.la[i], ch.lp[i]);
          bwd_step<ALG>(v, g);
        }
      } else {
#pragma unroll
        for (int i = kBlk - 1; i >= 0; --i) {
          if (i < hi) {
            Gam g;
            g.set(ch.la[i], ch.lp[i]);
            bwd_step<ALG>(v, g);
          }
        }
      }
      normalize8(v);
      const int tm = c * kBlk;  // v now holds the metrics at time tm
      if (tm == a1 && vstart) {
#pragma unroll
        for (int s = 0; s < 8; ++s) vstart[s] = v[s];
      }
      if (tm >= a0 && tm < a1) {
        if (refine) {
          float old[8];
          load_ck(fr.ckb + c * 8, old);
          if (close8(v, old, tol)) return;
        }
        store_ck(fr.ckb + c * 8, v);
      }
    }
  }
  if (vend) {
#pragma unroll
    for (int s = 0; s < 8; ++s) vend[s] = v[s];
  }
}

// Where soDecode's last iteration leaves its values: the constituent's extrinsic values
// of every trellis step (tail included) in its own order, and its parity extrinsic
// values (nullable) at element offset par0 of par, of type dtype.
struct SoftSink {
  float* ext = nullptr;  // [T]
  void* par = nullptr;
  int64_t par0 = 0;
  int32_t dtype = 1;
};

// Phase B for one 8-step block b of constituent j: reload the forward checkpoint at
// the block start and the backward one at its end, recompute the block's forward
// vectors in registers, walk backward emitting sf * extrinsic into out (X: Ls + e at
// t, Y: e at pi(t)).  FULL: all 8 steps are message steps (no per-step tests).  SOFT:
// soDecode's last iteration, which also records every step's extrinsic value (tail
// steps too) and parity extrinsic value in `sink`.
template <int ALG, bool FULL, bool SOFT>
__device__ __forceinline__ void ext_block(int j, int b, int K, int T, const Frame& fr, const float* X, const float* Y,
                                          const uint32_t* perm, float sf, float* out, const SoftSink& sink) {
  const int t0 = b * kBlk;
  const int n = FULL ? kBlk : min(kBlk, T - t0);
  RawChunk raw;
  load_raw(j, b, fr, perm, raw);
  float al[kBlk][8];
  load_ck(fr.cka + b * 8, al[0]);
  float be[8];
  load_ck(fr.ckb + (b + 1) * 8, be);
  Chunk in;
  resolve(j, b, K, fr, X, Y, raw, in);
#pragma unroll
  for (int i = 1; i < kBlk; ++i) {
    if (FULL || i < n) {
#pragma unroll
      for (int s = 0; s < 8; ++s) al[i][s] = al[i - 1][s];
      Gam g;
      g.set(in.la[i - 1], in.lp[i - 1]);
      fwd_step<ALG>(al[i], g);
    }
  }
  const float ls[kBlk] = {__uint_as_float(raw.q0.x), __uint_as_float(raw.q0.y), __uint_as_float(raw.q0.z),
                          __uint_as_float(raw.q0.w), __uint_as_float(raw.q1.x), __uint_as_float(raw.q1.y),
                          __uint_as_float(raw.q1.z), __uint_as_float(raw.q1.w)};
  const uint32_t pq[kBlk] = {raw.q0.x, raw.q0.y, raw.q0.z, raw.q0.w, raw.q1.x, raw.q1.y, raw.q1.z, raw.q1.w};
#pragma unroll
  for (int i = kBlk - 1; i >= 0; --i) {
    if (FULL || i < n) {
      Gam g;
      g.set(in.la[i], in.lp[i]);
      const float e = sf * ext_step<ALG>(al[i], be, g);
      if (FULL || t0 + i < K) {
        if (j == 0) out[t0 + i] = ls[i] + e;
        else out[pq[i]] = e;
      }
      if (SOFT) {
        sink.ext[t0 + i] = e;
        if (sink.par) store_llr(sink.par, sink.dtype, sink.par0 + t0 + i, par_step<ALG>(al[i], be, g));
      }
      if (i > 0) bwd_step<ALG>(be, g);
    }
  }
}

// One frame's geometry and buffers, as the decode loop below sees them.
struct LteJob {
  int32_t K = 0, Kp = 0, Tp = 0, seg_len = 0, train = 0, iterations = 0;
  const float* sf = nullptr;            // [2][iterations]
  const uint32_t* perm = nullptr;       // interleaver of constituent 1, padded by 16 entries
  const float* scratch = nullptr;       // staged L-values: Ls [Kp] | Lp0 [Tp] | Lp1 [Tp] | tail [8]
  float* ck = nullptr;                  // checkpoints [2][nblk + 1][8]
  uint8_t* hard = nullptr;              // [K]
  int32_t* iters = nullptr;             // nullable
  unsigned long long* stats = nullptr;  // nullable
  const uint32_t* crc = nullptr;        // [K] x^(K-1-i) mod g: stop when the decisions' CRC checks (nullable)
  // Parallel scheduling: constituent 1 runs first and leaves its extrinsic values in
  // ynew, copied into Y once constituent 0, which reads the old ones, is done.
  int32_t parallel = 0;
  float* ynew = nullptr;  // [Kp]
  // soDecode (decode_lte_frame<.., SOFT = true>): this frame's inputs and outputs in
  // FeCl's turbo layouts, as element offsets into the caller's buffers.
  float* soft_ext = nullptr;  // [2][Tp] scratch: each constituent's last extrinsic values by step
  const void* state_in = nullptr;
  int32_t in_dtype = 1, out_dtype = 1;
  void *msg_out = nullptr, *syst_out = nullptr, *parity_out = nullptr, *state_out = nullptr;
  int64_t frame = 0;  // frame index within the caller's buffers
};

// Segment length for a frame of T steps split into `segs` segments: a multiple of
// the checkpoint spacing, so every segment boundary is a checkpoint.
__host__ __device__ inline int lte_seg_len(int T, int segs) {
  const int L = (T + segs - 1) / segs;
  return (L + kBlk - 1) / kBlk * kBlk;
}

// Decodes one frame with the whole CTA; smem holds 2 * Kp floats + Shared<SEGS>.
// SOFT: soDecode (TurboDecoderImpl::soDecodeBlock, TurboDecoderImpl.cpp:75-150).
template <int ALG, int SEGS, bool SOFT = false>
__device__ __forceinline__ void decode_lte_frame(const LteJob& q, float* smem) {
  constexpr int kThreads = 2 * SEGS;
  const int K = q.K, T = q.K + 3;
  const int nblk = (T + kBlk - 1) / kBlk;
  const int nblk_msg = (K + kBlk - 1) / kBlk;
  float* X = smem;
  float* Y = smem + q.Kp;
  Shared<SEGS>& sh = *reinterpret_cast<Shared<SEGS>*>(smem + 2 * q.Kp);
  Frame fr;
  const float* base = q.scratch;
  fr.Ls = base;
  fr.Lp0 = base + q.Kp;
  fr.Lp1 = base + q.Kp + q.Tp;
  fr.ts = base + q.Kp + 2 * q.Tp;
  fr.cka = q.ck;
  fr.ckb = fr.cka + (nblk + 1) * 8;
  const int tid = threadIdx.x;
  const int L = q.seg_len;
  const int S = (T + L - 1) / L;
  const Tol tol = SOFT ? kSoftTol : kDecodeTol;

  // X = Ls + e0 with e0 = 0 (constituent 1 reads it first under Parallel scheduling)
  for (int k = tid; k < q.Kp; k += kThreads) {
    X[k] = fr.Ls[k];
    Y[k] = 0.0f;
  }
  if (tid < 8) {
    sh.flat[tid] = 0.0f;
    sh.term[tid] = tid == 0 ? 0.0f : kNegInf;  // Tail: the trellis starts and ends in state 0
  }
  __syncthreads();
  if (SOFT && q.state_in) {
    // the initial extrinsic values: X = Ls + e0, Y[pi(t)] = e1(t) (tail values are
    // replaced by the channel's tail bits before every pass, as in the reference)
    const int64_t s0 = q.frame * int64_t(2 * (K + 3));
    for (int k = tid; k < K; k += kThreads) {
      X[k] = fr.Ls[k] + load_llr(q.state_in, q.in_dtype, s0 + k);
      Y[__ldg(q.perm + k)] = load_llr(q.state_in, q.in_dtype, s0 + K + 3 + k);
    }
    __syncthreads();
  }

  int ran = q.iterations;
  for (int it = 0; it < q.iterations; ++it) {
    const bool last_soft = SOFT && it == q.iterations - 1;
    for (int jj = 0; jj < 2; ++jj) {
      const int j = q.parallel ? 1 - jj : jj;  // parallel: constituent 1 first, on the old X
      const uint32_t* perm = q.perm;
      // ---- A: segments with training starts
      {
        const bool fwd = tid < SEGS;
        const int w = fwd ? tid : tid - SEGS;
        if (w < S) {
          const int a0 = w * L, a1 = min(T, a0 + L);
          int t_train;
          const float* vin;
          if (fwd) {
            const bool exact = (w == 0 || a0 - q.train <= 0);
            t_train = exact ? 0 : a0 - q.train;
            vin = exact ? sh.term : sh.flat;
          } else {
            const bool exact = (w == S - 1 || a1 + q.train >= T);
            t_train = exact ? T : a1 + q.train;
            vin = exact ? sh.term : sh.flat;
          }
          // a forward start is the checkpoint at a0, a backward end the one at a0
          segment_walk<ALG>(fwd, j, t_train, a0, a1, vin, fwd ? nullptr : sh.bwd_start[w], fwd ? sh.fwd_end[w] : nullptr,
                            K, T, fr, X,
                            Y, perm, false, tol);
        }
      }
      __syncthreads();
      // ---- A2: verify boundaries; walk again the segments whose start disagrees.
      // One barrier both publishes and combines the checks; a round with a rejected
      // boundary adds two more.
      int rounds = 0;
      for (int round = 0; round < S; ++round) {
        const bool fwd = tid < SEGS;
        const int w = fwd ? tid : tid - SEGS;
        bool bad = false;
        if (w < S) {
          // forward: this segment's start (its checkpoint at a0) against the previous
          // segment's end; backward: this segment's start at a1 against the next
          // segment's end (its checkpoint at a1)
          if (fwd && w > 0) bad = !close8(fr.cka + (w * L / kBlk) * 8, sh.fwd_end[w - 1], tol);
          if (!fwd && w < S - 1) bad = !close8(sh.bwd_start[w], fr.ckb + ((w + 1) * L / kBlk) * 8, tol);
        }
        if (!__syncthreads_or(bad)) break;
        ++rounds;
        // Walk every rejected segment again from its neighbour's end.  The end is
        // copied to registers before the barrier and becomes the segment's start
        // after it, so a neighbour that is itself being walked again is read in its
        // old state; the next round checks the boundary again.
        float start[8];
        if (bad) {
#pragma unroll
          for (int s = 0; s < 8; ++s) start[s] = fwd ? sh.fwd_end[w - 1][s] : fr.ckb[((w + 1) * L / kBlk) * 8 + s];
        }
        __syncthreads();
        if (bad) {
          if (q.stats) atomicAdd(q.stats + 2, 1ull);
          // the walk reads its start from sv: a forward segment's checkpoint at a0
          // (which the walk writes again with the same values), a backward segment's
          // start vector
          float* sv = fwd ? fr.cka + (w * L / kBlk) * 8 : sh.bwd_start[w];
#pragma unroll
          for (int s = 0; s < 8; ++s) sv[s] = start[s];
          const int a0 = w * L, a1 = min(T, a0 + L);
          segment_walk<ALG>(fwd, j, fwd ? a0 : a1, a0, a1, sv, fwd ? nullptr : sv, fwd ? sh.fwd_end[w] : nullptr, K, T, fr,
                            X, Y, perm, true,
                            tol);
        }
        __syncthreads();
      }
      if (q.stats && tid == 0) {
        atomicAdd(q.stats + 0, 1ull);
        atomicAdd(q.stats + 1, (unsigned long long)rounds);
      }
      // ---- B: 8-step blocks, extrinsic output.  Only blocks holding message steps
      // run: the tail steps' a-priori values are the channel's tail bits, so their
      // extrinsic values are never read (with K a multiple of 8, as every LTE size
      // is, the last block is all tail).
      // soDecode does not scale the extrinsic values (TurboDecoderImpl.cpp:75-150)
      const float sf = SOFT ? 1.0f : q.sf[j * q.iterations + it];
      float* out = j == 0 ? X : (q.parallel ? q.ynew : Y);
      if (last_soft) {
        // soDecode's last iteration: every block, tail blocks too, recording the
        // extrinsic and parity extrinsic values
        SoftSink sink;
        sink.ext = q.soft_ext + j * q.Tp;
        sink.par = q.parity_out;
        sink.par0 = q.frame * int64_t(3 * K + 12) + K + 6 + j * (K + 3);
        sink.dtype = q.out_dtype;
        for (int b = tid; b < nblk; b += kThreads) ext_block<ALG, false, true>(j, b, K, T, fr, X, Y, perm, sf, out, sink);
      } else {
        const SoftSink none;
        for (int b = tid; b < nblk_msg; b += kThreads) {
          // in max-log a block of 8 message steps (every block but, when K is not a
          // multiple of 8, the last) runs without per-step tests (the log-MAP kernels
          // keep one form, which their registers hold without spilling)
          if (ALG == kApproximate && b * kBlk + kBlk <= K)
            ext_block<ALG, true, false>(j, b, K, T, fr, X, Y, perm, sf, out, none);
          else
            ext_block<ALG, false, false>(j, b, K, T, fr, X, Y, perm, sf, out, none);
        }
      }
      __syncthreads();
    }
    if (q.parallel) {
      for (int k = tid; k < K; k += kThreads) Y[k] = q.ynew[k];
      __syncthreads();
    }
    // CRC stop (an extension; LTE transport blocks end with a CRC-24): the decisions
    // after this iteration are those the frame would end with; the CRC syndrome of the
    // K decided bits is the xor of the table entries of the bits that are 1.
    if (q.crc) {
      uint32_t syn = 0;
      for (int k = tid; k < K; k += kThreads)
        if ((X[k] + Y[k]) > 0.0f) syn ^= __ldg(q.crc + k);
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) syn ^= __shfl_xor_sync(0xffffffffu, syn, o);
      if ((tid & 31) == 0) sh.crc_part[tid >> 5] = syn;
      __syncthreads();
      uint32_t all = 0;
#pragma unroll
      for (int w = 0; w < kThreads / 32; ++w) all ^= sh.crc_part[w];
      __syncthreads();
      if (all == 0) {
        ran = it + 1;
        break;
      }
    }
  }
  if constexpr (SOFT) {
    // aPosterioriUpdate (TurboDecoderImpl.cpp:152-168) and the soDecode outputs: syst =
    // (0 + e0) + e1 at natural positions, the tails' extrinsic values after them;
    // parity = syst | both constituents' parity extrinsic values (written above);
    // msg = channel (+ a-priori) + syst; state = e0 | e1 in each constituent's order.
    const float* e0 = q.soft_ext;
    const float* e1 = q.soft_ext + q.Tp;
    const int64_t f = q.frame;
    for (int k = tid; k < K + 6; k += kThreads) {
      float v;
      if (k < K) v = e0[k] + Y[k];
      else v = k < K + 3 ? e0[k] : e1[k - 3];
      if (q.syst_out) store_llr(q.syst_out, q.out_dtype, f * int64_t(K + 6) + k, v);
      if (q.parity_out) store_llr(q.parity_out, q.out_dtype, f * int64_t(3 * K + 12) + k, v);
      if (q.msg_out && k < K) store_llr(q.msg_out, q.out_dtype, f * int64_t(K) + k, fr.Ls[k] + v);
    }
    if (q.state_out)
      for (int t = tid; t < 2 * (K + 3); t += kThreads) {
        const float v = t < K + 3 ? e0[t] : e1[t - (K + 3)];
        store_llr(q.state_out, q.out_dtype, f * int64_t(2 * (K + 3)) + t, v);
      }
  } else {
    // a-posteriori and hard decision, TurboDecoderImpl.cpp:64-71
    for (int k = tid; k < K; k += kThreads) q.hard[k] = uint8_t((X[k] + Y[k]) > 0.0f);
    if (q.iters && tid == 0) *q.iters = ran;
  }
}

template <int ALG, int SEGS, bool SOFT = false>
__global__ void __launch_bounds__(2 * SEGS, SEGS == 32 ? 4 : (SEGS == 128 ? 1 : 3)) turbo_lte_kernel(TurboLteParams p) {
  extern __shared__ float smem[];
  const int64_t f = p.frame0 + blockIdx.x;
  const int nblk = (p.K + 3 + kBlk - 1) / kBlk;
  LteJob q;
  q.K = p.K;
  q.Kp = p.Kp;
  q.Tp = p.Tp;
  q.seg_len = p.seg_len;
  q.train = p.train;
  q.iterations = p.iterations;
  q.sf = p.sf;
  q.perm = p.perm[1];
  q.scratch = p.scratch + f * p.frame_stride;
  q.ck = p.ck + f * int64_t(2 * (nblk + 1) * 8);
  q.hard = p.hard + f * p.K;
  q.iters = p.iters ? p.iters + f : nullptr;
  q.stats = p.stats;
  q.crc = p.crc;
  q.parallel = p.parallel;
  if (p.ynew) {  // per frame: ynew [Tp] | soft_ext [2][Tp]
    q.ynew = p.ynew + f * int64_t(3 * p.Tp);
    q.soft_ext = q.ynew + p.Tp;
  }
  q.state_in = p.state_in;
  q.in_dtype = p.llr_dtype;
  q.out_dtype = p.out_dtype;
  q.msg_out = p.msg_out;
  q.syst_out = p.syst_out;
  q.parity_out = p.parity_out;
  q.state_out = p.state_out;
  q.frame = f;
  decode_lte_frame<ALG, SEGS, SOFT>(q, smem);
}


template <typename T>
__device__ __forceinline__ float to_f32(T v) { return float(v); }
template <>
__device__ __forceinline__ float to_f32<__half>(__half v) { return __half2float(v); }

// Input [f][3K+12] in FeCl's turbo layout -> padded FP32 scratch, one block per frame
// (grid-strided over frames): the systematic, parity and tail regions are copied by
// loops of their own, so no element needs a division to find its place, and the
// element type is fixed per launch.
template <typename T>
__global__ void turbo_lte_stage(TurboLteParams p) {
  const T* llr = static_cast<const T*>(p.llr);
  const int K = p.K, Kp = p.Kp, Tp = p.Tp;
  for (int64_t f = blockIdx.x; f < p.nframes; f += gridDim.x) {
    const T* in = llr + f * int64_t(3 * K + 12);
    float* out = p.scratch + f * p.frame_stride;
    // soDecode's a-priori input is added to the channel's systematic values and tails
    // (TurboDecoderImpl.cpp:77-82)
    const T* sys = p.syst_in ? static_cast<const T*>(p.syst_in) + f * int64_t(K + 6) : nullptr;
    // four elements per thread and step, all loaded before any is stored, so that each
    // thread keeps four loads in flight (load latency, not bandwidth, bounds the copy)
    constexpr int kU = 4;
    const int step = int(blockDim.x);
    for (int i0 = threadIdx.x; i0 < Kp; i0 += kU * step) {
      float v[kU];
#pragma unroll
      for (int u = 0; u < kU; ++u) {
        const int i = i0 + u * step;
        v[u] = i < K ? (sys ? to_f32(in[i]) + to_f32(sys[i]) : to_f32(in[i])) : 0.0f;
      }
#pragma unroll
      for (int u = 0; u < kU; ++u)
        if (i0 + u * step < Kp) out[i0 + u * step] = v[u];
    }
    for (int c = 0; c < 2; ++c) {
      const T* src = in + K + 6 + c * (K + 3);  // parity (with its tail) of constituent c
      float* dst = out + Kp + c * Tp;
      for (int t0 = threadIdx.x; t0 < Tp; t0 += kU * step) {
        float v[kU];
#pragma unroll
        for (int u = 0; u < kU; ++u) {
          const int t = t0 + u * step;
          v[u] = t < K + 3 ? to_f32(src[t]) : 0.0f;
        }
#pragma unroll
        for (int u = 0; u < kU; ++u)
          if (t0 + u * step < Tp) dst[t0 + u * step] = v[u];
      }
    }
    if (threadIdx.x < 8) {
      float v = 0.0f;
      if (threadIdx.x < 6) v = sys ? to_f32(in[K + threadIdx.x]) + to_f32(sys[K + threadIdx.x]) : to_f32(in[K + threadIdx.x]);
      out[Kp + 2 * Tp + threadIdx.x] = v;
    }
  }
}

// Geometry of a frame of K message bits: T trellis steps, nblk 8-step blocks, the
// padded systematic / parity lengths Kp = Tp, the staged-input stride and the
// segment length of the `segs` forward and `segs` backward segments.
struct LteGeometry {
  int T, nblk, Tp, Kp, stride, seg_len;
  __host__ __device__ LteGeometry(int K, int segs) {
    T = K + 3;
    nblk = (T + kBlk - 1) / kBlk;
    Tp = nblk * kBlk;
    Kp = Tp;
    stride = Kp + 2 * Tp + 8;
    seg_len = lte_seg_len(T, segs);
  }
  // Staged inputs then checkpoints, rounded to 128 bytes so frames share no cache line.
  __host__ __device__ int frame_floats() const { return (stride + 2 * (nblk + 1) * 8 + 31) & ~31; }
};

// Stages element i of a frame's staged inputs from FeCl's turbo layout
// | msg [K] | systTail1 [3] | systTail2 [3] | parity1 [K+3] | parity2 [K+3] |.
__device__ __forceinline__ float staged_value(const void* llr, int dtype, int64_t in0, int K, int Kp, int Tp, int i) {
  if (i < Kp) return i < K ? load_llr(llr, dtype, in0 + i) : 0.0f;
  if (i < Kp + 2 * Tp) {
    const int c = (i - Kp) / Tp, t = (i - Kp) % Tp;
    return t < K + 3 ? load_llr(llr, dtype, in0 + K + 6 + c * (K + 3) + t) : 0.0f;
  }
  const int t = i - Kp - 2 * Tp;
  return t < 6 ? load_llr(llr, dtype, in0 + K + t) : 0.0f;
}

// Mixed-K batch, staging: one block per frame (grid-strided).
__global__ void turbo_lte_batch_stage(TurboLteBatchParams p) {
  for (int64_t f = blockIdx.x; f < p.nframes; f += gridDim.x) {
    const TurboLteBatchFrame d = p.frames[f];
    const LteGeometry g(d.K, kDefaultSegs);
    for (int i = threadIdx.x; i < g.stride; i += blockDim.x)
      d.scratch[i] = staged_value(d.llr, d.llr_dtype, 0, d.K, g.Kp, g.Tp, i);
  }
}

// Mixed-K batch, decoding: persistent CTAs take frames from a counter in the order
// of the descriptor table (longest first), so frames of every size share one launch
// and the long ones do not trail behind.  Shared memory is sized for the largest K.
template <int ALG, int SEGS>
__global__ void __launch_bounds__(2 * SEGS, SEGS == 32 ? 4 : 3) turbo_lte_batch_kernel(TurboLteBatchParams p) {
  extern __shared__ float smem[];
  __shared__ int next;
  for (;;) {
    __syncthreads();  // every thread has read `next` (and finished the last frame)
    if (threadIdx.x == 0) next = atomicAdd(p.counter, 1);
    __syncthreads();
    const int64_t f = next;
    if (f >= p.nframes) break;
    const TurboLteBatchFrame d = p.frames[f];
    const LteGeometry g(d.K, SEGS);
    LteJob q;
    q.K = d.K;
    q.Kp = g.Kp;
    q.Tp = g.Tp;
    q.seg_len = g.seg_len;
    q.train = p.train;
    q.iterations = d.iterations;
    q.sf = d.sf;
    q.perm = d.perm;
    q.scratch = d.scratch;
    q.ck = d.scratch + g.stride;
    q.hard = d.hard;
    q.iters = d.iters;
    q.stats = p.stats;
    q.crc = d.crc;
    decode_lte_frame<ALG, SEGS>(q, smem);
  }
}

template <int SEGS>
size_t lte_smem_bytes(int max_K) {
  return size_t(2 * LteGeometry(max_K, SEGS).Kp) * sizeof(float) + sizeof(Shared<SEGS>);
}

int resolve_segs(int segs) { return segs == 32 || segs == 64 || segs == 128 ? segs : kDefaultSegs; }

// Streaming multiprocessors of the current device (0 if the query fails).
int device_sms() {
  int dev = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return sms;
}

// Training steps before each segment when the caller leaves them to the launcher.
// Max-log: 80 (K=6144 x 1024 at 0.7 dB: 1.10 ms against 1.13 ms with 96, the same
// decisions; 4x more segments are walked again, but a walk again stops at the first
// checkpoint it reproduces).  The log-MAP algorithms: 96, since their fix-up walks
// cost more than the training they save (Exact 54.8 ms with 80 against 40.7 ms).
int default_train(int algorithm) { return algorithm == kApproximate ? 80 : 96; }

// Resident CTAs of kern on the whole GPU (0 if the query fails).
template <class Kern>
int64_t resident_ctas(Kern kern, int threads, size_t smem) {
  int per_sm = 0, dev = 0, sms = 0;
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem) != cudaSuccess ||
      cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return int64_t(per_sm) * sms;
}

// Frames (from the first) that the 32-segment shape decodes when the segment count
// is left to the launcher; the rest take the 64-segment shape.  A CTA decodes one
// frame start to end, so n frames take ceil(n / resident) rounds of about equal time
// and a last round holding a few frames leaves most of the GPU idle for a whole
// frame's decode.  When the 64-segment shape (fewer resident CTAs: 3 per SM against
// 4, register-bound) would end on a round less than half full, whole rounds of the
// 32-segment shape go first so that the 64-segment rounds are full or nearly so:
// K=6144 x 1024 frames on 148 SMs is 592 + 432 frames in two rounds (1.12 ms measured)
// instead of 444 + 444 + 136 in three (1.23 ms).  Which frames take which shape does not
// change their results beyond FP32 rounding of the window boundaries.
template <int ALG>
int64_t split_frames(int K, int64_t nframes) {
  // resident CTAs of both shapes, remembered per (device, K)
  static std::mutex mu;
  static std::map<std::pair<int, int>, std::pair<int64_t, int64_t>> known;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  int64_t r64, r32;
  {
    std::lock_guard<std::mutex> lk(mu);
    auto it = known.find({dev, K});
    if (it == known.end()) {
      const std::pair<int64_t, int64_t> r{resident_ctas(turbo_lte_kernel<ALG, 64>, 128, lte_smem_bytes<64>(K)),
                                          resident_ctas(turbo_lte_kernel<ALG, 32>, 64, lte_smem_bytes<32>(K))};
      it = known.emplace(std::make_pair(dev, K), r).first;
    }
    r64 = it->second.first;
    r32 = it->second.second;
  }
  if (r64 <= 0 || r32 <= 0 || nframes <= r64) return 0;
  auto rounds = [](int64_t n, int64_t r) { return (n + r - 1) / r; };
  auto tail_ok = [&](int64_t n) { return n % r64 == 0 || 2 * (n % r64) >= r64; };
  if (tail_ok(nframes)) return 0;
  for (int64_t n32 = r32; n32 < nframes; n32 += r32) {
    const int64_t rest = nframes - n32;
    if (tail_ok(rest) && rounds(n32, r32) + rounds(rest, r64) <= rounds(nframes, r64)) return n32;
  }
  return 0;
}

}  // namespace

cudaError_t turbo_lte_init() {
  static std::atomic<unsigned long long> done{0};
  return once_per_device(done, [] {
    const LinearLut l = make_linear_lut();
    return cudaMemcpyToSymbol(c_lut, &l, sizeof(l));
  });
}

size_t turbo_lte_scratch_bytes(int K, int64_t nframes, bool extra) {
  const int T = K + 3;
  const int nblk = (T + kBlk - 1) / kBlk;
  const int Tp = nblk * kBlk;
  const int Kp = Tp;
  const int64_t stride = Kp + 2 * Tp + 8;
  return size_t(nframes) * (size_t(stride) + size_t(2 * (nblk + 1) * 8) + (extra ? size_t(3 * Tp) : 0)) * sizeof(float);
}

cudaError_t launch_turbo_lte(TurboLteParams p, cudaStream_t s) {
  cudaError_t e0 = turbo_lte_init();
  if (e0 != cudaSuccess) return e0;
  if (p.nframes <= 0) return cudaSuccess;
  const int segs = resolve_segs(p.segs);
  const LteGeometry g(p.K, segs);
  p.Tp = g.Tp;
  p.Kp = g.Kp;  // the systematic region and the exchange arrays are padded like the parity
  p.frame_stride = g.stride;
  p.ck = p.scratch + p.nframes * p.frame_stride;
  // parallel scheduling and soDecode: per frame ynew [Tp] | soft_ext [2][Tp] after the
  // checkpoints (turbo_lte_scratch_bytes(K, n, true))
  p.ynew = (p.parallel || p.soft) ? p.ck + p.nframes * int64_t(2 * (g.nblk + 1) * 8) : nullptr;
  if (p.soft) p.crc = nullptr;
  p.seg_len = g.seg_len;
  if (p.train < 0) p.train = default_train(p.algorithm);
  const unsigned stage_blocks = unsigned(p.nframes < 148 * 8 ? p.nframes : 148 * 8);
  switch (p.llr_dtype) {
    case kF64: turbo_lte_stage<double><<<stage_blocks, 256, 0, s>>>(p); break;
    case kF16: turbo_lte_stage<__half><<<stage_blocks, 256, 0, s>>>(p); break;
    default: turbo_lte_stage<float><<<stage_blocks, 256, 0, s>>>(p); break;
  }
  auto launch = [&](auto kern, int threads, size_t smem) -> cudaError_t {
    cudaError_t err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    if (err != cudaSuccess) return err;
    kern<<<unsigned(p.nframes), threads, smem, s>>>(p);
    return cudaGetLastError();
  };
  if (p.soft) {
    const size_t smem = lte_smem_bytes<64>(p.K);
    switch (p.algorithm) {
      case kExact: return launch(turbo_lte_kernel<kExact, 64, true>, 128, smem);
      case kLinear: return launch(turbo_lte_kernel<kLinear, 64, true>, 128, smem);
      default: return launch(turbo_lte_kernel<kApproximate, 64, true>, 128, smem);
    }
  }
  if (segs == 32) {
    const size_t smem = lte_smem_bytes<32>(p.K);
    switch (p.algorithm) {
      case kExact: return launch(turbo_lte_kernel<kExact, 32>, 64, smem);
      case kLinear: return launch(turbo_lte_kernel<kLinear, 32>, 64, smem);
      default: return launch(turbo_lte_kernel<kApproximate, 32>, 64, smem);
    }
  }
  // A batch of at most one frame per SM decodes in one round whose time is one
  // frame's latency: with the segment count left to the launcher it takes the
  // 128-segment shape (one CTA of 256 threads per frame: half as many phase B blocks
  // per thread and shorter segment walks than with 64), as does an explicit 128.
  if (segs == 128 || (p.segs == 0 && p.nframes <= device_sms())) {
    p.seg_len = LteGeometry(p.K, 128).seg_len;
    const size_t smem = lte_smem_bytes<128>(p.K);
    switch (p.algorithm) {
      case kExact: return launch(turbo_lte_kernel<kExact, 128>, 256, smem);
      case kLinear: return launch(turbo_lte_kernel<kLinear, 128>, 256, smem);
      default: return launch(turbo_lte_kernel<kApproximate, 128>, 256, smem);
    }
  }
  const size_t smem = lte_smem_bytes<64>(p.K);
  if (p.segs == 0) {
    // the launcher's choice: whole rounds of the 32-segment shape first where that
    // fills the rounds better (split_frames)
    const int64_t n32 = p.algorithm == kExact    ? split_frames<kExact>(p.K, p.nframes)
                        : p.algorithm == kLinear ? split_frames<kLinear>(p.K, p.nframes)
                                                 : split_frames<kApproximate>(p.K, p.nframes);
    if (n32 > 0) {
      TurboLteParams a = p;
      a.nframes = n32;
      a.seg_len = LteGeometry(p.K, 32).seg_len;
      const size_t smem32 = lte_smem_bytes<32>(p.K);
      auto run = [&](auto k32, auto k64) -> cudaError_t {
        cudaError_t err = cudaFuncSetAttribute(k32, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem32));
        if (err != cudaSuccess) return err;
        k32<<<unsigned(n32), 64, smem32, s>>>(a);
        if ((err = cudaGetLastError()) != cudaSuccess) return err;
        TurboLteParams b = p;
        b.frame0 = n32;
        if ((err = cudaFuncSetAttribute(k64, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem))) != cudaSuccess)
          return err;
        k64<<<unsigned(p.nframes - n32), 128, smem, s>>>(b);
        return cudaGetLastError();
      };
      switch (p.algorithm) {
        case kExact: return run(turbo_lte_kernel<kExact, 32>, turbo_lte_kernel<kExact, 64>);
        case kLinear: return run(turbo_lte_kernel<kLinear, 32>, turbo_lte_kernel<kLinear, 64>);
        default: return run(turbo_lte_kernel<kApproximate, 32>, turbo_lte_kernel<kApproximate, 64>);
      }
    }
  }
  switch (p.algorithm) {
    case kExact: return launch(turbo_lte_kernel<kExact, 64>, 128, smem);
    case kLinear: return launch(turbo_lte_kernel<kLinear, 64>, 128, smem);
    default: return launch(turbo_lte_kernel<kApproximate, 64>, 128, smem);
  }
}

size_t turbo_lte_frame_floats(int K) { return size_t(LteGeometry(K, kDefaultSegs).frame_floats()); }

int turbo_lte_batch_max_ctas(int max_K, int algorithm) {
  const size_t smem = lte_smem_bytes<kDefaultSegs>(max_K);
  int per_sm = 0, sms = 0, dev = 0;
  auto q = [&](auto kern) {
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 2 * kDefaultSegs, smem) != cudaSuccess) {
      cudaGetLastError();
      per_sm = 0;
    }
  };
  switch (algorithm) {
    case kExact: q(turbo_lte_batch_kernel<kExact, kDefaultSegs>); break;
    case kLinear: q(turbo_lte_batch_kernel<kLinear, kDefaultSegs>); break;
    default: q(turbo_lte_batch_kernel<kApproximate, kDefaultSegs>); break;
  }
  if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return per_sm * sms;
}

cudaError_t launch_turbo_lte_batch(const TurboLteBatchParams& p, cudaStream_t s) {
  cudaError_t e = turbo_lte_init();
  if (e != cudaSuccess) return e;
  if (p.nframes <= 0) return cudaSuccess;
  if (p.max_K <= 0 || p.max_K > 12288) return cudaErrorInvalidValue;
  TurboLteBatchParams q = p;
  if (q.train < 0) q.train = default_train(q.algorithm);
  e = cudaMemsetAsync(q.counter, 0, sizeof(int32_t), s);
  if (e != cudaSuccess) return e;
  const unsigned stage_blocks = unsigned(q.nframes < 148 * 8 ? q.nframes : 148 * 8);
  turbo_lte_batch_stage<<<stage_blocks, 256, 0, s>>>(q);
  const size_t smem = lte_smem_bytes<kDefaultSegs>(q.max_K);
  int ctas = q.ctas > 0 ? q.ctas : turbo_lte_batch_max_ctas(q.max_K, q.algorithm);
  if (ctas <= 0) return cudaErrorInvalidConfiguration;
  if (int64_t(ctas) > q.nframes) ctas = int(q.nframes);
  auto launch = [&](auto kern) -> cudaError_t {
    cudaError_t err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    if (err != cudaSuccess) return err;
    kern<<<unsigned(ctas), 2 * kDefaultSegs, smem, s>>>(q);
    return cudaGetLastError();
  };
  switch (q.algorithm) {
    case kExact: return launch(turbo_lte_batch_kernel<kExact, kDefaultSegs>);
    case kLinear: return launch(turbo_lte_batch_kernel<kLinear, kDefaultSegs>);
    default: return launch(turbo_lte_batch_kernel<kApproximate, kDefaultSegs>);
  }
}

}  // namespace fecl
