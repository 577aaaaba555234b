// Permutation::permute / dePermute (src/Permutation.h:175-189) over batches of blocks:
// gather out[b][i] = in[b][seq[i]], and the inverse gather out[b][j] = in[b][inv[j]]
// (or zero where no output index maps to j: a punctured position is an erasure).
// inv[j] is the last i with seq[i] == j, as the reference's sequential scatter leaves it.
#include <stdint.h>

#include "common.cuh"
#include "kernels.hpp"

namespace fecl {
namespace {

template <class T>
__global__ void gather_kernel(const T* in, T* out, const uint32_t* map, int64_t in_size, int64_t out_size,
                              int64_t nblocks, int zero_fill) {
  const int64_t total = nblocks * out_size;
  for (int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < total; t += int64_t(gridDim.x) * blockDim.x) {
    const int64_t b = t / out_size;
    const int64_t i = t - b * out_size;
    const uint32_t src = map[i];
    out[t] = (zero_fill && src == 0xffffffffu) ? T(0) : in[b * in_size + src];
  }
}

template <class T>
cudaError_t run(const void* in, void* out, const uint32_t* map, int64_t in_size, int64_t out_size, int64_t nblocks,
                int zero_fill, cudaStream_t s) {
  const int64_t total = nblocks * out_size;
  const int64_t blocks = (total + 255) / 256;
  gather_kernel<T><<<unsigned(blocks < 148 * 32 ? (blocks > 0 ? blocks : 1) : 148 * 32), 256, 0, s>>>(
      static_cast<const T*>(in), static_cast<T*>(out), map, in_size, out_size, nblocks, zero_fill);
  return cudaGetLastError();
}

}  // namespace

cudaError_t launch_gather(const void* in, void* out, const uint32_t* map, int64_t in_size, int64_t out_size,
                          int64_t nblocks, int elem_bytes, int zero_fill, cudaStream_t s) {
  if (nblocks <= 0 || out_size <= 0) return cudaSuccess;
  switch (elem_bytes) {
    case 1: return run<uint8_t>(in, out, map, in_size, out_size, nblocks, zero_fill, s);
    case 2: return run<uint16_t>(in, out, map, in_size, out_size, nblocks, zero_fill, s);
    case 4: return run<uint32_t>(in, out, map, in_size, out_size, nblocks, zero_fill, s);
    case 8: return run<uint64_t>(in, out, map, in_size, out_size, nblocks, zero_fill, s);
  }
  return cudaErrorInvalidValue;
}

}  // namespace fecl
