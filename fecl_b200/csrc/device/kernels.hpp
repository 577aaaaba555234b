// Host-callable launchers of the decoder kernels.  Plain structs of device
// pointers and sizes; no CUDA types beyond cudaStream_t/cudaError_t.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace fecl {

// ---- LDPC ----------------------------------------------------------------

// A check matrix laid out for the device: CSR by check (the edge order of the
// soft state), plus for every bit the ids of its edges in increasing order.
struct LdpcDeviceCode {
  int32_t M = 0, N = 0, msg = 0, d_max = 0;
  int64_t E = 0;
  const uint32_t* row_ptr = nullptr;    // [M+1]
  const uint32_t* col_idx = nullptr;    // [E]
  const uint32_t* col_ptr = nullptr;    // [N+1]
  const uint32_t* col_edges = nullptr;  // [E]
  const float* sf = nullptr;            // [n_sf][sf_stride], entry [i][d-2]
  int32_t n_sf = 1, sf_stride = 1;
  int32_t algorithm = 2;
  int32_t iterations = 1;
  int32_t fixed_iterations = 0;
};

struct LdpcRun {
  int64_t nframes = 0;
  const void* llr = nullptr;  // [nframes][N]
  int32_t llr_dtype = 1;
  const void* syst_in = nullptr;   // [nframes][msg] (soft decode only)
  const void* state_in = nullptr;  // [nframes][E]
  uint8_t* hard = nullptr;         // [nframes][msg]
  int32_t* iters = nullptr;        // [nframes]
  void* msg_out = nullptr;         // [nframes][msg]
  void* syst_out = nullptr;        // [nframes][msg]
  void* parity_out = nullptr;      // [nframes][N]
  void* state_out = nullptr;       // [nframes][E]
  int32_t out_dtype = 1;
  // scratch, FP32
  float* c2v = nullptr;   // [nframes][E]
  float* app = nullptr;   // [nframes][N]
  float* chan = nullptr;  // [nframes][N]
};

cudaError_t launch_ldpc_flood(const LdpcDeviceCode& code, const LdpcRun& run, cudaStream_t stream);

// Batched decoder with 32 frames per warp (one per lane), lane-minor scratch.
struct LdpcLanesParams {
  // code
  int32_t M = 0, N = 0, msg = 0, d_max = 0;
  int64_t E = 0;
  const uint32_t* row_ptr = nullptr;
  const uint32_t* col_idx = nullptr;
  const uint32_t* col_ptr = nullptr;
  const uint32_t* col_edges = nullptr;
  const float* sf = nullptr;
  int32_t n_sf = 1, sf_stride = 1;
  int32_t algorithm = 2, iterations = 1, fixed_iterations = 0;
  int32_t msg_type = 0;  // 0 FP32, 1 FP16, 2 saturated int8 (Q5.2)
  int32_t wave_groups = 0;  // groups decoded together (0: as many as fit in 64 MiB of L2)
  int32_t persist = 0;      // one persistent launch for small batches: 1 wherever it applies, 0 / -1 never
  // batch, frame-major caller buffers
  int64_t nframes = 0;
  const void* llr = nullptr;
  int32_t llr_dtype = 1;
  const void* syst_in = nullptr;
  const void* state_in = nullptr;
  uint8_t* hard = nullptr;
  int32_t* iters = nullptr;
  void* msg_out = nullptr;
  void* syst_out = nullptr;
  void* parity_out = nullptr;
  void* state_out = nullptr;
  int32_t out_dtype = 1;
  // filled by the launcher from the scratch buffer
  int32_t groups = 0;
  float* chan = nullptr;
  float* app = nullptr;
  void* c2v = nullptr;
  uint32_t* active = nullptr;
  uint32_t* fail = nullptr;
  int32_t* iters_ws = nullptr;
  unsigned* barrier = nullptr;  // [2] grid barrier counter and failure flag of the persistent launch
};

size_t ldpc_lanes_scratch_bytes(int64_t N, int64_t E, int64_t nframes, int msg_type);
// Cooperative launch of a persistent LDPC kernel, ordered after the previous one on
// this device (ldpc_lanes.cu).
cudaError_t ldpc_persist_launch(cudaStream_t s, const void* kern, unsigned blocks, unsigned threads, void** args);
cudaError_t launch_ldpc_lanes(LdpcLanesParams p, void* scratch, cudaStream_t stream);

// Normalised min-sum with FP16 messages and packed half2 check-node arithmetic, two
// frames per lane (ldpc_lanes_h2.cu).  Takes no soft state input.
size_t ldpc_lanes_h2_scratch_bytes(int64_t N, int64_t E, int64_t nframes);
cudaError_t launch_ldpc_lanes_h2(LdpcLanesParams p, void* scratch, cudaStream_t stream);

// The packed FP16 decoder over several codes in one persistent launch (a mixed
// batch's LDPC jobs of one check-degree class: d_max <= 8, <= 16 or <= 32): every
// job keeps its own layout (ldpc_lanes_h2_layout over its scratch), staged and
// finished by its own launches; the iterations of all of them run in one
// cooperative launch, wave by wave.
struct LdpcMultiGroup {
  int32_t code = 0;   // index into LdpcMultiParams::codes
  int32_t group = 0;  // group of 64 frames within that code's job
};
constexpr int kMultiMaxCodes = 16;       // codes per launch
constexpr int kMultiMaxWaveGroups = 32;  // groups per wave
struct LdpcMultiParams {
  const LdpcLanesParams* codes = nullptr;  // [ncodes] in device memory, layouts filled
  int32_t ncodes = 0;
  const LdpcMultiGroup* groups = nullptr;  // [wave_ptr[nwaves]], wave by wave
  const int32_t* wave_ptr = nullptr;       // [nwaves + 1]
  int32_t nwaves = 0;
  unsigned* barrier = nullptr;             // [2] zeroed by the launcher
};
void ldpc_lanes_h2_layout(LdpcLanesParams& p, void* scratch, int lanes = 32);
int64_t ldpc_lanes_h2_group_bytes(int64_t N, int64_t E);
cudaError_t launch_ldpc_h2_stage(const LdpcLanesParams& p, cudaStream_t s);
cudaError_t launch_ldpc_h2_finish(const LdpcLanesParams& p, cudaStream_t s);
cudaError_t launch_ldpc_h2_multi(LdpcMultiParams m, int d_max, cudaStream_t s);
// The same groups with one launch per pass instead of one persistent launch: per
// wave, the initial bit pass, then per iteration one check launch (all the wave's
// groups: of one check-degree class d_max, or of every class with d_max = 0) and one
// bit launch.
struct LdpcManyWave {
  int32_t q0 = 0, groups = 0;      // the wave's groups [q0, q0 + groups) of the table
  int32_t max_rows = 0, max_bits = 0, iterations = 0;  // largest M, N and iteration limit among them
};
cudaError_t launch_ldpc_h2_many(const LdpcMultiParams& m, const LdpcManyWave& w, int d_max, cudaStream_t s);

// Flooding BP with each frame's messages resident in the shared memory of a
// thread-block cluster of `cluster` CTAs (ldpc_cluster.cu).  The address tables are
// built per (code, cluster) by build_ldpc_cluster_plan (host/ldpc_plan.hpp).
struct LdpcClusterParams {
  // code
  int32_t M = 0, N = 0, msg = 0, d_max = 0;
  int64_t E = 0;
  const uint32_t* row_ptr = nullptr;    // [M+1] CSR by check
  const uint32_t* chk_addr = nullptr;   // [E]   CSR order: (rank << 28) | offset of the edge's bit
  const uint32_t* bit_ptr = nullptr;    // [N]   start (multiple of 4) | degree << 26 into bit_addr
  const uint32_t* bit_addr = nullptr;   // [..]  bit-major: (rank << 28) | offset of the edge
  const uint32_t* row_split = nullptr;  // [cluster+1] rows owned by each rank
  const uint32_t* bit_split = nullptr;  // [cluster+1] bits owned by each rank
  const float* sf = nullptr;
  int32_t n_sf = 1, sf_stride = 1;
  int32_t algorithm = 2, iterations = 1, fixed_iterations = 0;
  int32_t separate_syndrome = 0;  // scaling changes across iterations
  int32_t msg_type = 0;           // 0 FP32, 1 FP16, 2 saturated int8 (Q5.2)
  // shape
  int32_t cluster = 1, threads = 512, clusters = 1;  // CTAs per cluster, threads per CTA, clusters in the grid
  int64_t max_edges = 0, max_bits = 0;                // largest share of one rank
  int64_t app_offset = 0;                             // filled by the launcher
  int32_t* counter = nullptr;                         // device int, frames handed out
  // batch, frame-major caller buffers
  int64_t nframes = 0;
  const void* llr = nullptr;
  int32_t llr_dtype = 1;
  const void* syst_in = nullptr;
  const void* state_in = nullptr;
  uint8_t* hard = nullptr;
  int32_t* iters = nullptr;
  void* msg_out = nullptr;
  void* syst_out = nullptr;
  void* parity_out = nullptr;
  void* state_out = nullptr;
  int32_t out_dtype = 1;
};

// Dynamic shared memory of one CTA for the given largest shares.
size_t ldpc_cluster_smem_bytes(int64_t max_edges, int64_t max_bits, int msg_type);
cudaError_t launch_ldpc_cluster(LdpcClusterParams p, cudaStream_t stream);
int ldpc_cluster_max_active(const LdpcClusterParams& p);

// ---- Turbo ---------------------------------------------------------------

constexpr int kMaxConstituents = 8;

struct TurboDeviceConstituent {
  int32_t state_count, input_count, input_size, output_size;
  int32_t length, tail, termination;
  int32_t msg_size, syst_size, syst_tail_size, parity_size;
  const uint32_t* next_state;  // [state_count * input_count]
  const uint32_t* output;
  const uint32_t* perm;        // [msg_size]
};

struct TurboDeviceCode {
  int32_t n = 0;
  int32_t msg = 0, syst = 0, parity = 0, state = 0, tail = 0;
  int32_t max_steps = 0, max_states = 0;
  TurboDeviceConstituent c[kMaxConstituents];
  const float* sf = nullptr;  // [n][iterations] resolved scaling
  int32_t algorithm = 1, iterations = 6, scheduling = 0;
  // Custom scheduling: stage s holds activations [stage_ptr[s], stage_ptr[s+1]);
  // activation a decodes constituent act_con[a] with a-priori input from the
  // constituents transfer[act_tptr[a] .. act_tptr[a+1]) (each list sorted).
  int32_t n_stages = 0;
  const int32_t* stage_ptr = nullptr;
  const int32_t* act_con = nullptr;
  const int32_t* act_tptr = nullptr;
  const int32_t* transfer = nullptr;
};

struct TurboRun {
  int64_t nframes = 0;
  int32_t soft = 0;  // 1 for soDecode (scaling 1.0, outputs below)
  const void* llr = nullptr;  // [nframes][parity]
  int32_t llr_dtype = 1;
  const void* syst_in = nullptr;
  const void* state_in = nullptr;
  uint8_t* hard = nullptr;
  int32_t* iters = nullptr;
  void* msg_out = nullptr;
  void* syst_out = nullptr;
  void* parity_out = nullptr;
  void* state_out = nullptr;
  int32_t out_dtype = 1;
  const uint32_t* crc = nullptr;  // [msg] x^(msg-1-i) x^24 mod g: hard decode stops on a passing CRC (nullable)
  // scratch, FP32, per frame
  float* parity_in = nullptr;   // [nframes][parity]
  float* parity_buf = nullptr;  // [nframes][parity]
  float* ext = nullptr;         // [nframes][state]
  float* ext_buf = nullptr;     // [nframes][state]
  float* alpha = nullptr;       // [nframes][max_steps * max_states]
};

cudaError_t launch_turbo_generic(const TurboDeviceCode& code, const TurboRun& run, cudaStream_t stream);

// Windowed decoder for two constituents of the LTE RSC with Tail termination.
struct TurboLteParams {
  int64_t nframes = 0;
  int32_t K = 0;
  int32_t iterations = 6;
  int32_t algorithm = 2;
  int32_t train = -1;  // training steps before each segment (-1: default)
  int32_t segs = 0;    // segments per direction, 32 or 64 (0: default)
  const uint32_t* perm[2] = {nullptr, nullptr};  // interleavers of the constituents
  const float* sf = nullptr;                     // [2][iterations]
  const void* llr = nullptr;
  int32_t llr_dtype = 1;
  uint8_t* hard = nullptr;
  int32_t* iters = nullptr;
  float* scratch = nullptr;  // turbo_lte_scratch_bytes(K, nframes)
  unsigned long long* stats = nullptr;  // [3] passes, fix-up rounds, recomputed segments (nullable)
  const uint32_t* crc = nullptr;        // [K] CRC syndrome table: stop a frame when its CRC checks (nullable)
  // Parallel scheduling: both constituents take the other's extrinsic values of the
  // previous iteration (scratch: turbo_lte_scratch_bytes(K, nframes, true)).
  int32_t parallel = 0;
  // soDecode (soft != 0): a-priori inputs added to the channel values and initial
  // extrinsic state (both nullable), soft outputs in FeCl's turbo layouts (nullable),
  // no scaling of the extrinsic values, no CRC stop and no hard decisions.
  int32_t soft = 0;
  const void* syst_in = nullptr;   // [nframes][K + 6]
  const void* state_in = nullptr;  // [nframes][2 (K + 3)]
  void* msg_out = nullptr;         // [nframes][K]
  void* syst_out = nullptr;        // [nframes][K + 6]
  void* parity_out = nullptr;      // [nframes][3 K + 12]
  void* state_out = nullptr;       // [nframes][2 (K + 3)]
  int32_t out_dtype = 1;
  // filled by the launcher
  int32_t Kp = 0, Tp = 0, seg_len = 0;
  int64_t frame0 = 0;  // frame of the launch's first CTA
  int64_t frame_stride = 0;
  float* ck = nullptr;
  float* ynew = nullptr;  // parallel: [nframes][Kp] the constituent-1 extrinsic values of this iteration
};

// Scratch of the windowed decoder; `parallel` adds a buffer per frame.
size_t turbo_lte_scratch_bytes(int K, int64_t nframes, bool parallel = false);
cudaError_t launch_turbo_lte(TurboLteParams p, cudaStream_t s);

// The same windowed decoder over a batch of frames of different K (any K <= 12288),
// one descriptor per frame, in one persistent launch (plus one staging launch).
struct TurboLteBatchFrame {
  const void* llr = nullptr;       // [3K+12] L-values of llr_dtype, FeCl's turbo layout
  uint8_t* hard = nullptr;         // [K]
  int32_t* iters = nullptr;        // nullable
  float* scratch = nullptr;        // turbo_lte_frame_floats(K) floats, 16-byte aligned
  const uint32_t* perm = nullptr;  // interleaver of constituent 1, padded by 16 entries
  const float* sf = nullptr;       // [2][iterations] scaling of the extrinsic values
  const uint32_t* crc = nullptr;   // [K] CRC syndrome table, or null for no CRC stop
  int32_t K = 0, iterations = 0, llr_dtype = 1, pad = 0;
};
struct TurboLteBatchParams {
  const TurboLteBatchFrame* frames = nullptr;  // device array; frames are taken in this order
  int64_t nframes = 0;
  int32_t* counter = nullptr;  // device int, zeroed by the launcher
  int32_t max_K = 0;           // largest K in the batch (sizes shared memory)
  int32_t algorithm = 2;       // one algorithm per launch
  int32_t train = -1;          // training steps (-1: default)
  int32_t ctas = 0;            // persistent CTAs (0: as many as are resident at once)
  unsigned long long* stats = nullptr;
};
size_t turbo_lte_frame_floats(int K);
int turbo_lte_batch_max_ctas(int max_K, int algorithm);
cudaError_t launch_turbo_lte_batch(const TurboLteBatchParams& p, cudaStream_t s);

// ---- convolutional codec (conv.cu, turbo_generic.cu) -----------------------

struct ViterbiRun {
  int64_t nframes = 0;
  const void* llr = nullptr;  // [nframes][parity]
  int32_t llr_dtype = 1;
  uint8_t* hard = nullptr;    // [nframes][msg]
  uint8_t* trace = nullptr;   // viterbi_scratch_bytes
};
size_t viterbi_scratch_bytes(const TurboDeviceConstituent& k, int64_t nframes);
cudaError_t launch_viterbi(const TurboDeviceConstituent& k, const ViterbiRun& r, cudaStream_t s);
cudaError_t launch_conv_encode(const TurboDeviceConstituent& c, const uint8_t* msg, uint8_t* parity, int64_t nframes,
                               cudaStream_t s);

struct ConvMapRun {
  int64_t nframes = 0;
  int32_t algorithm = 2;
  float sf = 1.0f;
  const void* llr = nullptr;      // [nframes][parity]
  const void* syst_in = nullptr;  // [nframes][syst] or null
  int32_t llr_dtype = 1;
  void* msg_out = nullptr;        // [nframes][msg]
  void* syst_out = nullptr;       // [nframes][syst]
  void* parity_out = nullptr;     // [nframes][parity]
  int32_t out_dtype = 1;
  // scratch (filled by the launcher)
  float *par = nullptr, *pout = nullptr, *sys = nullptr, *app = nullptr, *alpha = nullptr;
};
size_t conv_map_scratch_bytes(const TurboDeviceConstituent& k, int64_t nframes);
cudaError_t launch_conv_map(const TurboDeviceConstituent& k, ConvMapRun r, void* scratch, cudaStream_t s);

// ---- CRC-24 (crc.cu) ----------------------------------------------------------

// The generator polynomials of 3GPP TS 36.212 section 5.1.1, without the x^24 term.
constexpr uint32_t kCrc24A = 0x864CFBu, kCrc24B = 0x800063u;
// Appends to each frame of `len` bits its 24 CRC bits (out: [nframes][len + 24]).
cudaError_t launch_crc24_attach(const uint8_t* bits, int64_t len, int64_t nframes, uint32_t poly, uint8_t* out,
                                cudaStream_t s);
// ok[f] = 1 when frame f (len bits, CRC included) has a zero syndrome.
cudaError_t launch_crc24_check(const uint8_t* bits, int64_t len, int64_t nframes, uint32_t poly, int32_t* ok,
                               cudaStream_t s);

// ---- encoders and channel (encode.cu) ---------------------------------------

// The generator pieces of LdpcCode::encode on the device (CSR each).
struct LdpcEncodeTables {
  int32_t K = 0, N = 0, gap = 0;
  int32_t dc_rows = 0, a_rows = 0, b_rows = 0, t_rows = 0;
  const uint32_t *dc_ptr = nullptr, *dc_idx = nullptr;
  const uint32_t *a_ptr = nullptr, *a_idx = nullptr;
  const uint32_t *b_ptr = nullptr, *b_idx = nullptr;
  const uint32_t *t_ptr = nullptr, *t_idx = nullptr;
};
cudaError_t launch_ldpc_encode(const LdpcEncodeTables& t, const uint8_t* msg, uint8_t* parity, int64_t nframes,
                               cudaStream_t s);
cudaError_t launch_turbo_encode(const TurboDeviceCode& code, const uint8_t* msg, uint8_t* parity, int64_t nframes,
                                cudaStream_t s);
// L = 2 y / sigma^2 with y = (2 b - 1) + N(0, sigma^2), sigma^2 = 1 / (2 esn0), for n bits.
cudaError_t launch_awgn(const uint8_t* bits, int64_t n, double esn0, uint64_t seed, int dtype, void* out, cudaStream_t s);

// out[b][i] = in[b][map[i]] for b < nblocks, i < out_size (permute.cu); with zero_fill,
// map[i] == 0xffffffff gives zero (dePermute of a punctured position).
cudaError_t launch_gather(const void* in, void* out, const uint32_t* map, int64_t in_size, int64_t out_size,
                          int64_t nblocks, int elem_bytes, int zero_fill, cudaStream_t s);

// Uploads of every translation unit's __constant__ tables to the current device
// (each launcher calls its own; a stream capture must run them before it starts).
cudaError_t ldpc_flood_init();
cudaError_t ldpc_lanes_init();
cudaError_t ldpc_cluster_init();
cudaError_t turbo_generic_init();
cudaError_t turbo_lte_init();
inline cudaError_t init_device_constants() {
  cudaError_t e;
  if ((e = ldpc_flood_init()) != cudaSuccess) return e;
  if ((e = ldpc_lanes_init()) != cudaSuccess) return e;
  if ((e = ldpc_cluster_init()) != cudaSuccess) return e;
  if ((e = turbo_generic_init()) != cudaSuccess) return e;
  return turbo_lte_init();
}

}  // namespace fecl
