// Allocation-free entry point for the windowed LTE turbo decoder.
//
// Some callers cannot allocate device memory once they are running: a baseband
// pipeline that reserves its whole memory budget at start-up and forbids allocation
// on the data path, a real-time thread that must not block in cudaMalloc (which can
// synchronise the device and take milliseconds), or a plug-in host that owns the
// device memory pool.  fecl_lte_turbo_decode_noalloc serves them: it decodes with
// the same kernel as fecl_decode on an LTE turbo codec, but its scratch, its
// interleaver table and its scaling table live in file-scope __device__ arrays of
// fixed size, which every GPU that loads the library holds until the process exits.
//
// In host code the arrays' names are only host-side stand-ins, not device
// addresses; their device addresses come from cudaGetSymbolAddress, taken once per
// device, with that device current, by the first call on it.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../../include/fecl_b200.h"
#include "../host/codes.hpp"
#include "kernels.hpp"

namespace fecl {
void set_last_error(const std::string& msg);  // capi.cu
}

namespace {

constexpr uint32_t kMaxK = 6144;                       // largest LTE block size
constexpr size_t kScratchBytes = size_t(8) << 20;      // 8 MiB of scratch per device
constexpr uint32_t kMaxIterations = 64;
constexpr uint32_t kPermStride = kMaxK + 16;           // padded for 8-entry vector loads
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];
static __device__ __align__(256) uint32_t g_perm[2 * kPermStride];
static __device__ __align__(256) float g_scaling[2 * kMaxIterations];

struct DeviceAddresses {
  bool ready = false;
  float* scratch = nullptr;
  uint32_t* perm = nullptr;
  float* scaling = nullptr;
};
DeviceAddresses g_addr[kMaxDevices];
std::mutex g_addr_mu;

// Interleavers of the two constituents (identity, QPP) and unit scaling for this call.
__global__ void fill_tables(uint32_t* perm, float* scaling, uint32_t K, uint64_t f1, uint64_t f2, uint32_t iterations) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < kPermStride; i += gridDim.x * blockDim.x) {
    perm[i] = i < K ? i : 0u;
    perm[kPermStride + i] = i < K ? uint32_t((f1 * i + f2 * (uint64_t(i) * i)) % K) : 0u;
    if (i < 2 * iterations) scaling[i] = 1.0f;
  }
}

int fail(int status, const std::string& msg) {
  fecl::set_last_error(msg);
  return status;
}

}  // namespace

extern "C" int fecl_lte_turbo_decode_noalloc(uint32_t K, int32_t algorithm, uint32_t iterations, const void* llr,
                                             int32_t llr_dtype, uint64_t nframes, uint8_t* msg, void* stream) {
  uint32_t f1 = 0, f2 = 0;
  if (!fecl::lte_qpp_params(K, &f1, &f2)) return fail(FECL_EINVAL, "Invalid length: K is not an LTE block size");
  if (algorithm < FECL_EXACT || algorithm > FECL_APPROXIMATE) return fail(FECL_EINVAL, "Invalid decoder algorithm");
  if (iterations == 0 || iterations > kMaxIterations)
    return fail(FECL_EINVAL, "iterations must be between 1 and " + std::to_string(kMaxIterations));
  if (llr_dtype != FECL_F64 && llr_dtype != FECL_F32 && llr_dtype != FECL_F16)
    return fail(FECL_EINVAL, "Invalid element type");
  if (nframes == 0) return FECL_OK;
  if (!llr || !msg) return fail(FECL_EINVAL, "null buffer");
  // The frame count is compared with the capacity before any multiplication, so no
  // count, however large, can wrap the byte size into range.
  const size_t per_frame = fecl::turbo_lte_scratch_bytes(int(K), 1);
  const uint64_t max_frames = kScratchBytes / per_frame;
  if (nframes > max_frames)
    return fail(FECL_EINVAL, std::to_string(nframes) + " frames of K=" + std::to_string(K) + " need more than the " +
                                 std::to_string(kScratchBytes) + " bytes of scratch reserved; at most " +
                                 std::to_string(max_frames) + " frames of K=" + std::to_string(K) + " per call");
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail(FECL_ENODEV, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) return fail(FECL_EUNSUPPORTED, "device index out of range");
  DeviceAddresses a;
  {
    std::lock_guard<std::mutex> lk(g_addr_mu);
    if (!g_addr[dev].ready) {
      DeviceAddresses n;
      if ((e = cudaGetSymbolAddress(reinterpret_cast<void**>(&n.scratch), g_scratch)) != cudaSuccess ||
          (e = cudaGetSymbolAddress(reinterpret_cast<void**>(&n.perm), g_perm)) != cudaSuccess ||
          (e = cudaGetSymbolAddress(reinterpret_cast<void**>(&n.scaling), g_scaling)) != cudaSuccess)
        return fail(FECL_ECUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
      n.ready = true;
      g_addr[dev] = n;
    }
    a = g_addr[dev];
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  fill_tables<<<24, 256, 0, s>>>(a.perm, a.scaling, K, f1, f2, iterations);
  if ((e = cudaGetLastError()) != cudaSuccess) return fail(FECL_ECUDA, std::string("launch: ") + cudaGetErrorString(e));
  fecl::TurboLteParams p;
  p.nframes = int64_t(nframes);
  p.K = int32_t(K);
  p.iterations = int32_t(iterations);
  p.algorithm = algorithm;
  p.perm[0] = a.perm;
  p.perm[1] = a.perm + kPermStride;
  p.sf = a.scaling;
  p.llr = llr;
  p.llr_dtype = llr_dtype;
  p.hard = msg;
  p.scratch = a.scratch;
  if ((e = fecl::launch_turbo_lte(p, s)) != cudaSuccess)
    return fail(FECL_ECUDA, std::string("launch: ") + cudaGetErrorString(e));
  return FECL_OK;
}
