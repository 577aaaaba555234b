// LDPC flooding belief propagation with each frame's messages resident in the
// shared memory of one thread-block cluster.
//
// The decoder is BpDecoderImpl (src/detail/BpDecoder/BpDecoderImpl.cpp:37-179) as in
// ldpc_lanes.cu, with the same FP32 arithmetic (ldpc_math.cuh), so the two kernels
// agree bit for bit.  The layout is what differs:
//
//   A cluster of C CTAs (C in {1, 2, 4, 8, 16}) decodes one frame at a time, for all
//   of its iterations.  CTA `rank` owns a contiguous block of check rows -- the
//   check-to-bit messages c2v of their edges, in CSR edge order -- and a contiguous
//   block of bits -- their channel values and a-posteriori sums APP, FP32.  All of
//   it lives in shared memory; HBM is read once per frame (the L-values) and written
//   once (the decisions).  A row whose bit lives in another CTA reads that bit's APP
//   through distributed shared memory (ld.shared::cluster), and so does a bit whose
//   edge lives in another CTA.  Per iteration:
//     check phase   every owned row: v = APP - c2v, row update, c2v' stored; from
//                   iteration 1 on, the row's parity of the previous hard decision
//                   (APP >= 0) is folded into a per-CTA failure flag -- the reference's
//                   syndrome stop (:53-59);
//     cluster barrier, then every CTA reads all C flags;
//     bit phase     every owned bit: APP = chan + sum of c2v over its edges in edge order;
//     cluster barrier.
//   A frame whose syndrome held at iteration i stops after that iteration's bit
//   phase.  Its last check update ran with the scaling of iteration i; when the
//   scaling changes across iterations (`separate_syndrome`), the syndrome is
//   instead tested in a pass of its own before the check update, which then uses
//   the scaling of iteration I-1, as :61 does.
//
//   Edge addresses are precomputed on the host per (code, C): for each edge in CSR
//   order the owner rank and offset of its bit, and for each edge in bit-major order
//   the owner rank and offset of the edge, packed as (rank << 28) | offset.
//
//   Clusters are persistent: the grid holds as many clusters as fit on the GPU and
//   each takes its next frame from a global counter, so frames that stop early free
//   their cluster for the next frame.
#include <cooperative_groups.h>
#include <cuda_fp16.h>
#include <math.h>

#include "common.cuh"
#include "kernels.hpp"
#include "ldpc_math.cuh"

namespace fecl {
namespace {

using ldpc::Msg;
namespace cg = cooperative_groups;

__constant__ LinearLut c_lut;
// The Linear table copied to shared memory by every CTA that uses it: lanes look up
// different entries, which constant memory serves one address at a time and shared
// memory (eight words in eight banks) at once.
__shared__ LinearLut s_lut;

constexpr uint32_t kOffMask = 0x0fffffffu;

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return uint32_t(__cvta_generic_to_shared(p)); }

__device__ __forceinline__ uint32_t map_rank(uint32_t a, uint32_t rank) {
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(rank));
  return r;
}

__device__ __forceinline__ float ld_cluster_f32(uint32_t a) {
  float v;
  asm volatile("ld.shared::cluster.f32 %0, [%1];" : "=f"(v) : "r"(a) : "memory");
  return v;
}
__device__ __forceinline__ uint32_t ld_cluster_u32(uint32_t a) {
  uint32_t v;
  asm volatile("ld.shared::cluster.u32 %0, [%1];" : "=r"(v) : "r"(a) : "memory");
  return v;
}
__device__ __forceinline__ uint32_t ld_cluster_u16(uint32_t a) {
  uint32_t v;
  asm volatile("ld.shared::cluster.u16 %0, [%1];" : "=r"(v) : "r"(a) : "memory");
  return v;
}
__device__ __forceinline__ uint32_t ld_cluster_u8(uint32_t a) {
  uint32_t v;
  asm volatile("ld.shared::cluster.u8 %0, [%1];" : "=r"(v) : "r"(a) : "memory");
  return v;
}
__device__ __forceinline__ void st_cluster_u32(uint32_t a, uint32_t v) {
  asm volatile("st.shared::cluster.u32 [%0], %1;" ::"r"(a), "r"(v) : "memory");
}

template <int MSG>
__device__ __forceinline__ float ld_cluster_msg(uint32_t a) {
  if (MSG == 0) return ld_cluster_f32(a);
  if (MSG == 1) return Msg<1>::from_bits(ld_cluster_u16(a));
  return Msg<2>::from_bits(ld_cluster_u8(a));
}

// Barrier over the cluster with release/acquire ordering of shared-memory writes
// (a CTA barrier when the cluster has one CTA).
template <bool CL>
__device__ __forceinline__ void cluster_barrier() {
  if (CL) {
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
  } else {
    __syncthreads();
  }
}

struct Ctl {
  uint32_t fail[2];  // per-iteration failure flags, double-buffered by iteration parity
  int32_t frame;     // frame this cluster decodes, written by rank 0
  int32_t pad;
};

template <int ALG, int MSG, int DMAX, int THREADS, bool CL>
__global__ void __launch_bounds__(THREADS, 1) ldpc_cluster_kernel(LdpcClusterParams p) {
  using M = Msg<MSG>;
  using T = typename M::T;
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ uint32_t app_base[16], c2v_base[16], ctl_base[16];
  __shared__ Ctl ctl;

  const int tid = threadIdx.x;
  const uint32_t rank = CL ? cg::this_cluster().block_rank() : 0;
  const uint32_t nrank = CL ? uint32_t(p.cluster) : 1;
  const int r0 = int(__ldg(p.row_split + rank)), r1 = int(__ldg(p.row_split + rank + 1));
  const int b0 = int(__ldg(p.bit_split + rank)), b1 = int(__ldg(p.bit_split + rank + 1));
  const uint32_t e_lo = __ldg(p.row_ptr + r0), e_hi = __ldg(p.row_ptr + r1);
  T* c2v = reinterpret_cast<T*>(smem);
  float* app = reinterpret_cast<float*>(smem + p.app_offset);
  float* chan = app + p.max_bits;
  const uint32_t app_sa = smem_addr(app), c2v_sa = smem_addr(c2v), ctl_sa = smem_addr(&ctl);
  if (tid < int(nrank)) {
    app_base[tid] = CL ? map_rank(app_sa, tid) : app_sa;
    c2v_base[tid] = CL ? map_rank(c2v_sa, tid) : c2v_sa;
    ctl_base[tid] = CL ? map_rank(ctl_sa, tid) : ctl_sa;
  }
  if (tid == 0) ctl.fail[0] = ctl.fail[1] = 0;
  if (ALG == ldpc::kLinear && tid < 8) s_lut.y[tid] = c_lut.y[tid];
  __syncthreads();

  const int I = p.iterations;
  const int64_t N = p.N, E = p.E, K = p.msg;
  const bool soft = p.msg_out || p.syst_out || p.parity_out;

  // APP of a bit (global index b's packed address) and a c2v message, wherever they live.
  auto app_at = [&](uint32_t a) -> float {
    if (CL) return ld_cluster_f32(app_base[a >> 28] + (a & kOffMask) * 4u);
    return app[a & kOffMask];
  };
  auto c2v_at = [&](uint32_t a) -> float {
    if (CL) return ld_cluster_msg<MSG>(c2v_base[a >> 28] + (a & kOffMask) * uint32_t(sizeof(T)));
    return M::load(c2v + (a & kOffMask));
  };
  // chan + sum of c2v over the bit's edges, in increasing edge order.  Each bit's
  // edge list starts at a multiple of 4 entries (bit_ptr = start | degree << 26), so
  // its addresses come in 16-byte loads and four messages are in flight at once.
  auto bit_sum = [&](int b, float acc) -> float {
    const uint32_t bp = __ldg(p.bit_ptr + b);
    const uint32_t k0 = bp & 0x03ffffffu, k1 = k0 + (bp >> 26);
    uint32_t k = k0;
    for (; k + 4 <= k1; k += 4) {
      const uint4 a = __ldg(reinterpret_cast<const uint4*>(p.bit_addr + k));
      const float x0 = c2v_at(a.x), x1 = c2v_at(a.y), x2 = c2v_at(a.z), x3 = c2v_at(a.w);
      acc += x0;
      acc += x1;
      acc += x2;
      acc += x3;
    }
    for (; k < k1; ++k) acc += c2v_at(__ldg(p.bit_addr + k));
    return acc;
  };

  for (;;) {
    // ---- next frame (rank 0 takes it from the counter and tells every CTA)
    if (rank == 0 && tid == 0) {
      const int f = atomicAdd(p.counter, 1);
      for (uint32_t r = 0; r < nrank; ++r) {
        if (CL) st_cluster_u32(ctl_base[r] + offsetof(Ctl, frame), uint32_t(f));
        else ctl.frame = f;
      }
    }
    cluster_barrier<CL>();
    const int64_t f = ctl.frame;
    if (f >= p.nframes) break;

    // ---- stage: channel values (+ a-priori on the systematic bits), c2v from the
    // soft state or zero; then APP = chan + sum c2v, as the reference rebuilds its
    // bit-to-check messages (:42-46, :81-94).
    for (int b = b0 + tid; b < b1; b += THREADS) {
      float x = load_llr(p.llr, p.llr_dtype, f * N + b);
      if (p.syst_in && b < K) x += load_llr(p.syst_in, p.llr_dtype, f * K + b);
      chan[b - b0] = x;
    }
    for (uint32_t e = e_lo + tid; e < e_hi; e += THREADS)
      M::store(c2v + (e - e_lo), p.state_in ? load_llr(p.state_in, p.llr_dtype, f * E + e) : 0.0f);
    cluster_barrier<CL>();
    for (int b = b0 + tid; b < b1; b += THREADS) app[b - b0] = bit_sum(b, chan[b - b0]);
    cluster_barrier<CL>();

    int it = 0;
    for (;; ++it) {
      const int slot = it & 1;
      bool stop_now = false;  // the syndrome held before this iteration's check update
      if (p.separate_syndrome && it > 0 && it < I - 1 && !p.fixed_iterations) {
        uint32_t bad = 0;
        for (int r = r0 + tid; r < r1 && !bad; r += THREADS) {
          const uint32_t e0 = __ldg(p.row_ptr + r), e1 = __ldg(p.row_ptr + r + 1);
          uint32_t par = 0;
          for (uint32_t e = e0; e < e1; ++e) par ^= uint32_t(app_at(__ldg(p.chk_addr + e)) >= 0.0f);
          bad = par;
        }
        if (bad) ctl.fail[slot] = 1;
        cluster_barrier<CL>();
        uint32_t any = 0;
        for (uint32_t r = 0; r < nrank; ++r) any |= CL ? ld_cluster_u32(ctl_base[r] + slot * 4u) : ctl.fail[slot];
        stop_now = !any;
      }
      // ---- check phase
      const bool fold = !p.separate_syndrome && it > 0 && !p.fixed_iterations;
      const int sf_it = (p.separate_syndrome && (stop_now || it == I - 1)) ? I - 1 : it;
      const float* sf_row = p.sf + size_t(sf_it % p.n_sf) * p.sf_stride;
      uint32_t bad = 0;
      for (int r = r0 + tid; r < r1; r += THREADS) {
        const uint32_t e0 = __ldg(p.row_ptr + r);
        const int d = int(__ldg(p.row_ptr + r + 1) - e0);
        T* cr = c2v + (e0 - e_lo);
        float v[DMAX];
        uint32_t par = 0;
#pragma unroll
        for (int j = 0; j < DMAX; ++j) {
          if (j < d) {
            const float a = app_at(__ldg(p.chk_addr + e0 + j));
            par ^= uint32_t(a >= 0.0f);
            v[j] = a - M::load(cr + j);
          }
        }
        bad |= par;
        float out[DMAX];
        ldpc::row_update<ALG, DMAX>(s_lut, v, out, d, sf_row[d >= 2 ? d - 2 : 0]);
#pragma unroll
        for (int j = 0; j < DMAX; ++j)
          if (j < d) M::store(cr + j, out[j]);
      }
      if (fold && bad) ctl.fail[slot] = 1;
      cluster_barrier<CL>();
      bool done = (it == I - 1) || stop_now;
      if (fold) {
        uint32_t any = 0;
        for (uint32_t r = 0; r < nrank; ++r) any |= CL ? ld_cluster_u32(ctl_base[r] + slot * 4u) : ctl.fail[slot];
        done = done || !any;
      }
      // ---- bit phase
      for (int b = b0 + tid; b < b1; b += THREADS) app[b - b0] = bit_sum(b, chan[b - b0]);
      if (tid == 0) ctl.fail[slot ^ 1] = 0;  // the next iteration's flag; last read before the previous barrier
      cluster_barrier<CL>();
      if (done) break;
    }

    // ---- outputs (the soft ones are those of :111-129)
    if (p.iters && rank == 0 && tid == 0) p.iters[f] = it + 1;
    if (p.hard)
      for (int b = b0 + tid; b < b1 && b < K; b += THREADS) p.hard[f * K + b] = uint8_t(app[b - b0] >= 0.0f);
    if (soft) {
      for (int b = b0 + tid; b < b1; b += THREADS) {
        const float ext = bit_sum(b, 0.0f);
        if (p.parity_out) store_llr(p.parity_out, p.out_dtype, f * N + b, ext);
        if (b < K) {
          if (p.syst_out) store_llr(p.syst_out, p.out_dtype, f * K + b, ext);
          if (p.msg_out) store_llr(p.msg_out, p.out_dtype, f * K + b, chan[b - b0] + ext);
        }
      }
    }
    if (p.state_out)
      for (uint32_t e = e_lo + tid; e < e_hi; e += THREADS)
        store_llr(p.state_out, p.out_dtype, f * E + e, M::load(c2v + (e - e_lo)));
    if (tid == 0) ctl.fail[0] = ctl.fail[1] = 0;
    // The frame barrier at the top of the loop orders these reads of other CTAs'
    // messages before the next frame's stage overwrites them.
  }
}

template <int ALG, int MSG, int DMAX, int THREADS, bool CL>
cudaError_t launch_one(const LdpcClusterParams& p, int clusters, size_t smem, cudaStream_t s) {
  auto kern = ldpc_cluster_kernel<ALG, MSG, DMAX, THREADS, CL>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
  if (e != cudaSuccess) return e;
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute attr[1];
  cfg.gridDim = dim3(unsigned(clusters * p.cluster));
  cfg.blockDim = dim3(THREADS);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  if (CL) {
    if (p.cluster > 8) {
      e = cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
      if (e != cudaSuccess) return e;
    }
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = unsigned(p.cluster);
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
  }
  return cudaLaunchKernelEx(&cfg, kern, p);
}

template <int ALG, int MSG, int DMAX, int THREADS>
cudaError_t launch_cl(const LdpcClusterParams& p, int clusters, size_t smem, cudaStream_t s) {
  return p.cluster > 1 ? launch_one<ALG, MSG, DMAX, THREADS, true>(p, clusters, smem, s)
                       : launch_one<ALG, MSG, DMAX, THREADS, false>(p, clusters, smem, s);
}

// Block sizes: 512 or 1024 threads for rows of degree <= 16 (64 registers per thread
// at 1024), 256 or 512 for degree <= 32.
template <int ALG, int MSG, int DMAX>
cudaError_t launch_t(const LdpcClusterParams& p, int clusters, size_t smem, cudaStream_t s) {
  if (p.threads == 512) return launch_cl<ALG, MSG, DMAX, 512>(p, clusters, smem, s);
  if constexpr (DMAX <= 16) {
    if (p.threads == 1024) return launch_cl<ALG, MSG, DMAX, 1024>(p, clusters, smem, s);
  } else {
    if (p.threads == 256) return launch_cl<ALG, MSG, DMAX, 256>(p, clusters, smem, s);
  }
  return cudaErrorInvalidValue;
}

template <int ALG, int MSG>
cudaError_t launch_d(const LdpcClusterParams& p, int clusters, size_t smem, cudaStream_t s) {
  if (p.d_max <= 8) return launch_t<ALG, MSG, 8>(p, clusters, smem, s);
  if (p.d_max <= 16) return launch_t<ALG, MSG, 16>(p, clusters, smem, s);
  if (p.d_max <= 32) return launch_t<ALG, MSG, 32>(p, clusters, smem, s);
  return cudaErrorInvalidValue;
}

template <int ALG>
cudaError_t launch_m(const LdpcClusterParams& p, int clusters, size_t smem, cudaStream_t s) {
  switch (p.msg_type) {
    case 1: return launch_d<ALG, 1>(p, clusters, smem, s);
    case 2: return launch_d<ALG, 2>(p, clusters, smem, s);
    default: return launch_d<ALG, 0>(p, clusters, smem, s);
  }
}

cudaError_t dispatch(const LdpcClusterParams& p, int clusters, size_t smem, cudaStream_t s) {
  switch (p.algorithm) {
    case ldpc::kExact: return launch_m<ldpc::kExact>(p, clusters, smem, s);
    case ldpc::kLinear: return launch_m<ldpc::kLinear>(p, clusters, smem, s);
    default: return launch_m<ldpc::kApproximate>(p, clusters, smem, s);
  }
}

size_t msg_bytes(int msg_type) { return msg_type == 1 ? 2 : (msg_type == 2 ? 1 : 4); }

}  // namespace

cudaError_t ldpc_cluster_init() {
  static std::atomic<unsigned long long> done{0};
  return once_per_device(done, [] {
    const LinearLut l = make_linear_lut();
    return cudaMemcpyToSymbol(c_lut, &l, sizeof(l));
  });
}

size_t ldpc_cluster_smem_bytes(int64_t max_edges, int64_t max_bits, int msg_type) {
  const size_t c2v = (size_t(max_edges) * msg_bytes(msg_type) + 15) & ~size_t(15);
  return c2v + size_t(max_bits) * 8;
}

cudaError_t launch_ldpc_cluster(LdpcClusterParams p, cudaStream_t s) {
  cudaError_t e0 = ldpc_cluster_init();
  if (e0 != cudaSuccess) return e0;
  if (p.nframes <= 0) return cudaSuccess;
  if (p.cluster < 1 || p.cluster > 16 || (p.cluster & (p.cluster - 1))) return cudaErrorInvalidValue;
  const size_t smem = ldpc_cluster_smem_bytes(p.max_edges, p.max_bits, p.msg_type);
  p.app_offset = int64_t((size_t(p.max_edges) * msg_bytes(p.msg_type) + 15) & ~size_t(15));
  cudaError_t e = cudaMemsetAsync(p.counter, 0, sizeof(int32_t), s);
  if (e != cudaSuccess) return e;
  int clusters = p.clusters;
  if (clusters <= 0) clusters = 1;
  if (int64_t(clusters) > p.nframes) clusters = int(p.nframes);
  return dispatch(p, clusters, smem, s);
}

// How many clusters of this shape can be resident at once (0 if none fits).
int ldpc_cluster_max_active(const LdpcClusterParams& p) {
  const size_t smem = ldpc_cluster_smem_bytes(p.max_edges, p.max_bits, p.msg_type);
  int result = 0;
  auto query = [&](auto kern) {
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)) != cudaSuccess) {
      cudaGetLastError();
      return;
    }
    if (p.cluster > 8) cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    cfg.gridDim = dim3(unsigned(p.cluster));
    cfg.blockDim = dim3(unsigned(p.threads));
    cfg.dynamicSmemBytes = smem;
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = unsigned(p.cluster);
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    if (cudaOccupancyMaxActiveClusters(&result, kern, &cfg) != cudaSuccess) {
      cudaGetLastError();
      result = 0;
    }
  };
  // Occupancy depends on the shared memory and the block size, not on the template
  // arguments that only change the arithmetic; one instance per block size is asked.
  switch (p.threads) {
    case 256: query(ldpc_cluster_kernel<ldpc::kApproximate, 0, 32, 256, true>); break;
    case 512: query(ldpc_cluster_kernel<ldpc::kApproximate, 0, 16, 512, true>); break;
    case 1024: query(ldpc_cluster_kernel<ldpc::kApproximate, 0, 16, 1024, true>); break;
    default: return 0;
  }
  return result;
}

}  // namespace fecl
