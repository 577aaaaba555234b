// Device-side helpers shared by the decoder kernels.
#pragma once

#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <atomic>
#include <utility>

namespace fecl {

// Element types of caller buffers (FECL_F64 / FECL_F32 / FECL_F16).
enum DType : int { kF64 = 0, kF32 = 1, kF16 = 2 };

__device__ __forceinline__ float load_llr(const void* p, int dtype, size_t i) {
  switch (dtype) {
    case kF64: return float(static_cast<const double*>(p)[i]);
    case kF16: return __half2float(static_cast<const __half*>(p)[i]);
    default: return static_cast<const float*>(p)[i];
  }
}

__device__ __forceinline__ void store_llr(void* p, int dtype, size_t i, float v) {
  switch (dtype) {
    case kF64: static_cast<double*>(p)[i] = double(v); break;
    case kF16: static_cast<__half*>(p)[i] = __float2half_rn(v); break;
    default: static_cast<float*>(p)[i] = v; break;
  }
}

inline size_t dtype_size(int dtype) { return dtype == kF64 ? 8 : (dtype == kF16 ? 2 : 4); }

// The reference's piecewise-linear log(1 + exp(-x)) (src/detail/LinearTable.h:56-81):
// eight samples at x = i/2, linear in between, zero from x >= 3.5.
struct LinearLut {
  float y[8];
};

// The table's values, computed on the host.
inline LinearLut make_linear_lut() {
  LinearLut l;
  for (int i = 0; i < 8; ++i) l.y[i] = float(log(1.0 + exp(-(double(i) / 2.0))));
  return l;
}

// Runs `upload` (which fills a translation unit's __constant__ tables) once per
// device, with that device current.  __constant__ memory is per device, so a
// process that decodes on several GPUs needs one upload on each.
template <class F>
inline cudaError_t once_per_device(std::atomic<unsigned long long>& done, F&& upload) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  const unsigned long long bit = 1ull << (dev & 63);
  if (done.load() & bit) return cudaSuccess;
  e = upload();
  if (e == cudaSuccess) done.fetch_or(bit);
  return e;
}

// Programmatic dependent launch.  A kernel launched with launch_pdl may be scheduled
// while the previous kernel of its stream is still running; pdl_enter, its first
// statement, waits until that kernel has completed and its writes are visible (a
// no-op for a kernel launched without the attribute), then lets the next kernel of the
// stream start launching.  Consecutive passes of a decoder thus overlap their launch
// latency with the previous pass's tail, and compute exactly what sequential
// launches compute.
__device__ __forceinline__ void pdl_enter() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

template <typename... KArgs, typename... Args>
inline cudaError_t launch_pdl(void (*kern)(KArgs...), dim3 grid, dim3 block, cudaStream_t s, Args&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kern, std::forward<Args>(args)...);
}

// phi(x) = log1p(2 / expm1(x)) = -log(tanh(x / 2)) for x >= 0 (+inf at 0, 0 at +inf),
// the Exact check node's transform (every LDPC kernel calls this one, so they agree
// bit for bit).  Built from the hardware exponential and logarithm (__expf, __logf:
// relative error about 2^-22) where their arguments are well conditioned, and from
// truncated Taylor series where they are not:
//   expm1(x) = x (1 + x/2 + x^2/6)  for x < 2^-7  (truncation below x^3/24 < 2^-22),
//   log1p(z) = z (1 - z/2 + z^2/3)  for z < 2^-7  (truncation below z^3/4 < 2^-22).
// Outside those ranges e^x - 1 keeps 2^-22 relative to e^x and 1 + z is exact to
// 2^-24, so the result stays within about 3e-5 relative where phi < 1 and 6e-6 above.
__device__ __forceinline__ float ldpc_phi(float x) {
  constexpr float kSmall = 0.0078125f;  // 2^-7
  const float em1 = x < kSmall ? x * fmaf(x, fmaf(x, 1.0f / 6.0f, 0.5f), 1.0f) : __expf(x) - 1.0f;
  const float z = __fdividef(2.0f, em1);
  return z < kSmall ? z * fmaf(z, fmaf(z, 1.0f / 3.0f, -0.5f), 1.0f) : __logf(1.0f + z);
}

__device__ __forceinline__ float lut_log1pexpm(const LinearLut& t, float x) {
  x *= 2.0f;
  if (x >= 7.0f) return 0.0f;
  const int i = int(x);
  return (t.y[i + 1] - t.y[i]) * (x - float(i)) + t.y[i];
}

}  // namespace fecl
