// CRC-24A / CRC-24B (3GPP TS 36.212 section 5.1.1) over frames of bits, one thread per
// frame: the bits, most significant first, shifted through a 24-bit register with the
// generator's feedback; the parity bits are the register, highest bit first, so that a
// frame with its parity appended leaves a zero register.
#include <stdint.h>

#include "kernels.hpp"

namespace fecl {
namespace {

__device__ __forceinline__ uint32_t crc_step(uint32_t r, uint32_t bit, uint32_t poly) {
  const uint32_t fb = ((r >> 23) & 1u) ^ bit;
  r = (r << 1) & 0xFFFFFFu;
  return fb ? (r ^ poly) : r;
}

__global__ void crc_attach_kernel(const uint8_t* bits, int64_t len, int64_t nframes, uint32_t poly, uint8_t* out) {
  const int64_t f = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (f >= nframes) return;
  const uint8_t* b = bits + f * len;
  uint8_t* o = out + f * (len + 24);
  uint32_t r = 0;
  for (int64_t i = 0; i < len; ++i) {
    const uint32_t v = b[i] & 1u;
    o[i] = uint8_t(v);
    r = crc_step(r, v, poly);
  }
  for (int k = 0; k < 24; ++k) o[len + k] = uint8_t((r >> (23 - k)) & 1u);
}

__global__ void crc_check_kernel(const uint8_t* bits, int64_t len, int64_t nframes, uint32_t poly, int32_t* ok) {
  const int64_t f = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (f >= nframes) return;
  const uint8_t* b = bits + f * len;
  uint32_t r = 0;
  for (int64_t i = 0; i < len; ++i) r = crc_step(r, b[i] & 1u, poly);
  ok[f] = r == 0 ? 1 : 0;
}

}  // namespace

cudaError_t launch_crc24_attach(const uint8_t* bits, int64_t len, int64_t nframes, uint32_t poly, uint8_t* out,
                                cudaStream_t s) {
  if (nframes <= 0) return cudaSuccess;
  crc_attach_kernel<<<unsigned((nframes + 127) / 128), 128, 0, s>>>(bits, len, nframes, poly, out);
  return cudaGetLastError();
}

cudaError_t launch_crc24_check(const uint8_t* bits, int64_t len, int64_t nframes, uint32_t poly, int32_t* ok,
                               cudaStream_t s) {
  if (nframes <= 0) return cudaSuccess;
  crc_check_kernel<<<unsigned((nframes + 127) / 128), 128, 0, s>>>(bits, len, nframes, poly, ok);
  return cudaGetLastError();
}

}  // namespace fecl
