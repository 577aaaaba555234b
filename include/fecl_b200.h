/*
 * fecl_b200 -- B200-native batched soft-decision decoding for FeCl codes.
 *
 * This is the C-ABI seam under FeCl's decode path.  In the reference the seam is
 * the pair of protected virtuals every code family overrides,
 *     Codec::decodeBlocks   (src/Codec.h:105; overridden in src/Ldpc.h:102, src/Turbo.h:110)
 *     Codec::soDecodeBlocks (src/Codec.h:115; overridden in src/Ldpc.h:103, src/Turbo.h:111)
 * reached from the public templates Codec::decode / soDecode / encode / check
 * (src/Codec.h:68-82, 137-307) and from the Matlab function table
 * (wrap/wrap.h:51-253).  Every function below takes plain pointers and sizes;
 * no CUDA or C++ type crosses it except an opaque `void* stream` (a cudaStream_t).
 *
 * Conventions kept from the reference:
 *   - L-values are L = ln p(x=1)/p(x=0): a positive value favours bit 1
 *     (src/Codec.h:203-205).
 *   - Buffers are frame-major: [nframes][paritySize] in, [nframes][msgSize] out,
 *     the soft-output layouts of src/Ldpc.h:45-57 and src/Turbo.h:36-53.
 *   - LDPC hard decisions use APP >= 0 -> 1 (src/detail/BpDecoder/BpDecoderImpl.cpp:68),
 *     turbo hard decisions use APP > 0 -> 1 (src/detail/TurboDecoder/TurboDecoderImpl.cpp:70).
 *   - Size mismatches and invalid options, which the reference reports by throwing
 *     std::invalid_argument, return FECL_EINVAL with the reference's message in
 *     fecl_last_error().
 *
 * Memory: with FECL_HOST_MEMORY every pointer is host memory and the call returns
 * when the results are written.  With FECL_DEVICE_MEMORY every pointer is device
 * memory of the current device and the call is asynchronous on `stream`.
 */
#ifndef FECL_B200_H
#define FECL_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---------------------------------------------------------- */
#define FECL_OK 0
#define FECL_EINVAL (-1)       /* bad size or option (std::invalid_argument in the reference) */
#define FECL_ECUDA (-2)        /* a CUDA runtime call failed */
#define FECL_ENOMEM (-3)       /* device or host allocation failed */
#define FECL_ETIMEDOUT (-4)    /* a bounded device-side wait gave up */
#define FECL_EUNSUPPORTED (-5) /* option combination not implemented on the device */
#define FECL_ENODEV (-6)       /* no CUDA device visible */

/* ---- enums (values follow the reference's enums) --------------------------- */
/* DecoderAlgorithm, src/DecoderAlgorithm.h:30-34 */
#define FECL_EXACT 0
#define FECL_LINEAR 1
#define FECL_APPROXIMATE 2
/* SchedulingType, src/SchedulingType.h:32-39 */
#define FECL_SERIAL 0
#define FECL_PARALLEL 1
#define FECL_CUSTOM 2
/* Trellis::Termination, src/Trellis.h */
#define FECL_TAIL 0
#define FECL_TRUNCATE 1
/* element types of L-value buffers (FECL_U8: bits, for fecl_permute) */
#define FECL_F64 0
#define FECL_F32 1
#define FECL_F16 2
#define FECL_U8 3
/* precision of the decoder's internal messages (an extension; FP32 is the reference-parity mode) */
#define FECL_MSG_F32 0
#define FECL_MSG_F16 1
#define FECL_MSG_I8 2
/* CRC polynomials (3GPP TS 36.212 section 5.1.1) */
#define FECL_CRC24A 1
#define FECL_CRC24B 2
/* memory flags */
#define FECL_HOST_MEMORY 0
#define FECL_DEVICE_MEMORY 1

typedef struct fecl_codec_s* fecl_codec_t;

typedef struct {
  uint64_t msg;    /* Codec::msgSize    (src/Codec.h:60) */
  uint64_t syst;   /* Codec::systSize   (src/Codec.h:61) */
  uint64_t parity; /* Codec::paritySize (src/Codec.h:62) */
  uint64_t state;  /* Codec::stateSize  (src/Codec.h:63) */
} fecl_sizes;

/* ---- LDPC ------------------------------------------------------------------ */

/* Ldpc::DecoderOptions, src/detail/Ldpc.h:56-74. */
typedef struct {
  int32_t algorithm;   /* FECL_EXACT / FECL_LINEAR / FECL_APPROXIMATE */
  uint32_t iterations; /* maximum iterations; the syndrome stop of
                          src/detail/BpDecoder/BpDecoderImpl.cpp:49-61 applies */
  /* Scaling of check-node outputs, row-major [scaling_iterations][scaling_degrees]:
   * entry [i][d-2] scales rows of degree d at iteration i (i taken modulo
   * scaling_iterations), as Ldpc::Structure::scalingFactor (src/detail/Ldpc.cpp:134-138).
   * NULL means 1.0 everywhere. */
  const double* scaling;
  uint32_t scaling_iterations;
  uint32_t scaling_degrees;
  int32_t precision;  /* FECL_MSG_F32 (reference parity) / FECL_MSG_F16 / FECL_MSG_I8 */
  int32_t fixed_iterations; /* 0: reference syndrome stop; 1: always run `iterations` (extension) */
} fecl_ldpc_options;

/* fec::Ldpc(EncoderOptions(H), DecoderOptions) -- src/Ldpc.h:83, src/detail/Ldpc.cpp:34-55.
 * H is given in CSR form (rows = checks); the constructor transforms it for
 * encoding exactly as src/detail/Ldpc.cpp:216-331 does, which may reorder rows
 * and permute columns; fecl_ldpc_checks returns the transformed matrix. */
int fecl_ldpc_create(uint32_t rows, uint32_t cols, const uint32_t* row_ptr, const uint32_t* col_idx,
                     const fecl_ldpc_options* options, fecl_codec_t* out);

/* Ldpc::setDecoderOptions -- src/Ldpc.h:91. */
int fecl_ldpc_set_options(fecl_codec_t codec, const fecl_ldpc_options* options);

/* The transformed check matrix the decoder iterates over (detail::Ldpc::Structure::checks,
 * src/detail/Ldpc.h:110).  Its edge order is the layout of the LDPC soft state.
 * Call with row_ptr == NULL to obtain the sizes. */
int fecl_ldpc_checks(fecl_codec_t codec, uint32_t* rows, uint32_t* cols, uint64_t* nnz, uint32_t* row_ptr,
                     uint32_t* col_idx);

/* Standard DVB-S2 parity-check matrix for n in {16200, 64800} and rate num/den
 * (Ldpc::DvbS2::matrix, src/DvbS2.cpp:1595-1645).  Built to ETSI EN 302 307 from the
 * same address tables; the reference builder is only correct for (64800, 1/2), where
 * the two agree edge for edge.  Call with row_ptr == NULL to obtain the sizes. */
int fecl_dvbs2_matrix(uint32_t n, uint32_t rate_num, uint32_t rate_den, uint32_t* rows, uint32_t* cols,
                      uint64_t* nnz, uint32_t* row_ptr, uint32_t* col_idx);

/* Ldpc::Gallager::matrix -- src/Ldpc.cpp:77-102 (same generator and draws). */
int fecl_gallager_matrix(uint32_t n, uint32_t wc, uint32_t wr, uint64_t seed, uint32_t* rows, uint64_t* nnz,
                         uint32_t* row_ptr, uint32_t* col_idx);

/* ---- Turbo ----------------------------------------------------------------- */

/* A trellis as next-state / output tables indexed [state * input_count + input]
 * (src/Trellis.h:131-172). */
typedef struct {
  uint32_t state_count;
  uint32_t input_count;  /* 2^inputSize */
  uint32_t output_size;  /* output bits per branch */
  const uint32_t* next_state;
  const uint32_t* output;
} fecl_trellis;

/* Trellis(constraintLengths, generator, feedback) -- src/Trellis.cpp:76-143.
 * generators[i * noutputs + k] is the generator of input i, output k; feedback may be NULL.
 * Writes state_count * input_count entries to next_state/output when they are non-NULL. */
int fecl_trellis_build(uint32_t ninputs, const uint32_t* constraint_lengths, uint32_t noutputs,
                       const uint64_t* generators, const uint64_t* feedback, uint32_t* state_count,
                       uint32_t* input_count, uint32_t* output_size, uint32_t* next_state, uint32_t* output);

/* Turbo::DecoderOptions -- src/detail/Turbo.h:77-101. */
typedef struct {
  int32_t algorithm;   /* default FECL_LINEAR in the reference */
  uint32_t iterations; /* default 6 */
  int32_t scheduling;  /* FECL_SERIAL / FECL_PARALLEL / FECL_CUSTOM (with the schedule below) */
  /* scaling[row][col], rows = 1 or constituent count, cols = 1 or iterations
   * (Turbo::Structure::scalingFactor, src/detail/Turbo.cpp:148-153). NULL = 1.0. */
  const double* scaling;
  uint32_t scaling_rows;
  uint32_t scaling_cols;
  int32_t precision; /* FECL_MSG_F32 (reference parity) / FECL_MSG_F16 */
  /* FECL_CUSTOM: a Turbo::Scheduling (src/detail/Turbo.h:38-48, DecoderOptions::scheduling):
   * n_stages stages; stage s activates stage_counts[s] constituents (ids concatenated in
   * `activation`); activation a takes its a-priori input from transfer_counts[a]
   * constituents (ids concatenated in `transfer`). */
  uint32_t n_stages;
  const uint32_t* stage_counts;
  const uint32_t* activation;
  const uint32_t* transfer_counts;
  const uint32_t* transfer;
  /* An extension: FECL_CRC24A / FECL_CRC24B when the last 24 message bits are that CRC
   * of the others (3GPP TS 36.212 section 5.1.1): decode stops a frame after the first
   * iteration whose decisions pass the CRC (its bits are then those of a decode with
   * that many iterations); 0 runs every iteration.  Any turbo code and scheduling;
   * soft-output decoding (fecl_so_decode) runs every iteration. */
  int32_t crc;
} fecl_turbo_options;

/* fec::Turbo(EncoderOptions(trellis, interleavers).termination(t), DecoderOptions)
 * -- src/Turbo.h:100, src/detail/Turbo.cpp:45-103.  n_trellis and n_termination are 1
 * or n_constituents.  perm_len[i] == 0 means the identity on the message. */
int fecl_turbo_create(uint32_t n_constituents, const fecl_trellis* trellis, uint32_t n_trellis,
                      const uint32_t* perm_data, const uint32_t* perm_len, const int32_t* termination,
                      uint32_t n_termination, const fecl_turbo_options* options, fecl_codec_t* out);

/* The LTE turbo code of 3GPP TS 36.212: RSC Trellis({4},{{015}},{013}), Tail, and
 * {identity, Turbo::Lte3Gpp::interleaver(K)} (src/Lte3Gpp.cpp:219-237). */
int fecl_turbo_create_lte(uint32_t K, const fecl_turbo_options* options, fecl_codec_t* out);

/* Turbo::Lte3Gpp::interleaver -- perm[i] = (f1*i + f2*i^2) mod K. */
int fecl_lte_interleaver(uint32_t K, uint32_t* perm);

/* Turbo::setDecoderOptions -- src/Turbo.h:105. */
int fecl_turbo_set_options(fecl_codec_t codec, const fecl_turbo_options* options);

/* ---- Convolutional ----------------------------------------------------------- */

/* Convolutional::DecoderOptions -- src/detail/Convolutional.h:48-62. */
typedef struct {
  int32_t algorithm; /* soDecode's MAP algorithm (default FECL_APPROXIMATE); decode is Viterbi */
  double scaling;    /* scaling factor of the soft outputs (default 1.0) */
} fecl_conv_options;

/* fec::Convolutional(EncoderOptions(trellis, length).termination(t), DecoderOptions)
 * -- src/Convolutional.h:51, src/detail/Convolutional.cpp:45-66.  The reference's
 * default termination is FECL_TRUNCATE.  decode runs Viterbi
 * (src/detail/ViterbiDecoder/ViterbiDecoderImpl.cpp), soDecode the MAP decoder. */
int fecl_conv_create(const fecl_trellis* trellis, uint32_t length, int32_t termination, const fecl_conv_options* options,
                     fecl_codec_t* out);
int fecl_conv_set_options(fecl_codec_t codec, const fecl_conv_options* options);
/* Convolutional::puncturing (src/Convolutional.h:73, src/detail/Convolutional.cpp:223-242). */
int fecl_conv_puncturing(fecl_codec_t codec, const uint8_t* mask, uint32_t mask_len, const uint8_t* tail_mask,
                         uint32_t tail_mask_len, uint32_t* seq, uint64_t* seq_len);

/* ---- every codec ----------------------------------------------------------- */

int fecl_codec_sizes(fecl_codec_t codec, fecl_sizes* sizes);

/* Codec::encode -- src/Codec.h:171-198.  Bits are one byte each (0/1).  With
 * FECL_DEVICE_MEMORY the frames are encoded on the GPU (one thread per frame, the
 * reference's encoding steps, bit-exact), asynchronously on `stream`. */
int fecl_encode(fecl_codec_t codec, const uint8_t* msg, uint64_t nframes, uint8_t* parity, int32_t flags,
                void* stream);

/* BPSK over AWGN on the GPU (an extension): bit b -> x = 2b - 1, y = x + N(0, s2) with
 * s2 = 1 / (2 Es/N0), Es/N0 = 10^(ebn0_db / 10) * rate, out = 2 y / s2 in out_dtype.
 * bits and out are device memory; counter-based Philox-4x32-10 noise keyed by `seed`
 * (the same seed gives the same L-values).  Asynchronous on `stream`. */
int fecl_awgn_llr(const uint8_t* bits, uint64_t n, double ebn0_db, double rate, uint64_t seed, int32_t out_dtype,
                  void* out, void* stream);

/* Codec::check -- src/Codec.h:137-145; *ok = 1 when every frame is a codeword. */
int fecl_check(fecl_codec_t codec, const uint8_t* parity, uint64_t nframes, int32_t* ok);

/* Codec::decode -- src/Codec.h:210-238.  llr: [nframes][paritySize] of llr_dtype;
 * msg: [nframes][msgSize] bytes 0/1.  iterations (nullable): per frame, the number
 * of iterations the decoder ran (LDPC: check-node updates; turbo: iterations).
 * nframes == 0 returns FECL_OK at once and the buffers may then be null (this and
 * fecl_so_decode), as the reference decodes an empty vector to an empty one. */
int fecl_decode(fecl_codec_t codec, const void* llr, int32_t llr_dtype, uint64_t nframes, uint8_t* msg,
                int32_t* iterations, int32_t flags, void* stream);

/* Codec::soDecode -- src/Codec.h:249-307.  Every pointer but `parity` may be NULL. */
typedef struct {
  const void* parity; /* [nframes][paritySize], required */
  const void* syst;   /* [nframes][systSize] a-priori on the systematic bits */
  const void* state;  /* [nframes][stateSize] decoder state to resume from */
  int32_t in_dtype;   /* element type of the three inputs */
  void* msg;          /* [nframes][msgSize]   a-posteriori L-values */
  void* syst_out;     /* [nframes][systSize]  extrinsic on systematic bits */
  void* parity_out;   /* [nframes][paritySize] extrinsic on every code bit */
  void* state_out;    /* [nframes][stateSize] decoder state */
  int32_t out_dtype;  /* element type of the four outputs (FECL_F64 or FECL_F32) */
} fecl_so_io;

int fecl_so_decode(fecl_codec_t codec, const fecl_so_io* io, uint64_t nframes, int32_t flags, void* stream);

void fecl_destroy(fecl_codec_t codec);

/* ---- CRC-24 (an extension) -------------------------------------------------- */

/* Appends to each of nframes frames of len bits its 24 CRC bits (kind FECL_CRC24A /
 * FECL_CRC24B): out is [nframes][len + 24].  Device memory, asynchronous on stream. */
int fecl_crc24_attach(const uint8_t* bits, uint64_t len, uint64_t nframes, int32_t kind, uint8_t* out, void* stream);
/* ok[f] = 1 when frame f (len bits, its CRC included) passes.  Device memory. */
int fecl_crc24_check(const uint8_t* bits, uint64_t len, uint64_t nframes, int32_t kind, int32_t* ok, void* stream);

/* ---- puncturing ------------------------------------------------------------ */

/* Ldpc::puncturing (src/Ldpc.h:94, src/detail/Ldpc.cpp:333-353): the kept code-bit
 * indices of Ldpc::PunctureOptions().mask(mask).systMask(syst_mask), the sequence of
 * the fec::Permutation the reference returns (input size paritySize).  Call with
 * seq == NULL for the length. */
int fecl_ldpc_puncturing(fecl_codec_t codec, const uint8_t* mask, uint32_t mask_len, const uint8_t* syst_mask,
                         uint32_t syst_mask_len, uint32_t* seq, uint64_t* seq_len);

/* Turbo::puncturing (src/Turbo.h:102, src/detail/Turbo.cpp:200-320): masks as
 * concatenated bytes with one length each -- n_masks 0 or constituents + 1 (systematic,
 * then each constituent's parity), n_tail 0 or 2 per constituent; bit_ordering 0 =
 * Alternate, 1 = Group (Turbo::BitOrdering). */
int fecl_turbo_puncturing(fecl_codec_t codec, const uint8_t* mask_data, const uint32_t* mask_len, uint32_t n_masks,
                          const uint8_t* tail_data, const uint32_t* tail_len, uint32_t n_tail, int32_t bit_ordering,
                          uint32_t* seq, uint64_t* seq_len);

/* fec::Permutation (src/Permutation.h) on the device: permute gathers
 * out[b][i] = in[b][seq[i]] (blocks of input_size -> output_size); the inverse,
 * dePermute, scatters back and leaves zeros (erasures) where nothing maps.  Buffers
 * are device memory of elem_type (FECL_F64 / F32 / F16 / U8); asynchronous on stream. */
typedef struct fecl_permutation_s* fecl_permutation_t;
int fecl_permutation_create(const uint32_t* seq, uint64_t output_size, uint64_t input_size, fecl_permutation_t* out);
int fecl_permute(fecl_permutation_t perm, const void* in, int32_t elem_type, uint64_t nblocks, void* out, int32_t inverse,
                 void* stream);
void fecl_permutation_destroy(fecl_permutation_t perm);

/* ---- extensions (no counterpart in the reference) ------------------------ */

/* Kernel selection: FECL_KERNEL_AUTO picks the fastest kernel that supports the
 * code and options; FECL_KERNEL_GENERIC forces the generic kernels, which walk the
 * reference's operation order in FP32 (one thread per turbo frame, one CTA per
 * LDPC frame). */
#define FECL_KERNEL_AUTO 0
#define FECL_KERNEL_GENERIC 1
/* LDPC only: the lane-batched decoder (32 frames per warp, messages in device
 * memory) or the cluster-resident decoder (each frame's messages in the shared
 * memory of a thread-block cluster).  Both compute the same values bit for bit. */
#define FECL_KERNEL_LANES 2
#define FECL_KERNEL_CLUSTER 3
int fecl_set_kernel(fecl_codec_t codec, int32_t kernel);

/* Shape of the cluster-resident LDPC decoder: CTAs per frame (1, 2, 4, 8 or 16) and
 * threads per CTA (256, 512 or 1024).  0 for either restores the built-in choice.
 * Shapes whose shares of the code do not fit in shared memory fall back to the
 * lane-batched decoder (or fail with FECL_EUNSUPPORTED under FECL_KERNEL_CLUSTER). */
int fecl_ldpc_set_cluster_shape(fecl_codec_t codec, int32_t cluster, int32_t threads);

/* Lane-batched LDPC decoder: frame groups (32 frames each) decoded together, every
 * iteration of one wave of groups before the next; 0 restores the built-in choice
 * (the groups whose messages fit in 64 MiB of L2). */
int fecl_ldpc_set_wave(fecl_codec_t codec, int32_t groups);

/* Lane-batched LDPC decoder: run a small batch (at most 16 frame groups, one wave)
 * as one persistent launch whose check and bit passes are separated by grid-wide
 * barriers, instead of two launches per iteration.  mode 1: wherever it applies;
 * 0 (the built-in choice) and -1: never -- the per-pass launches, which overlap their
 * launch latency through programmatic dependent launch, measured faster.  The
 * results are those of the two-launch form bit for bit.  A barrier wait is bounded
 * (2 s); a decode whose barrier gave up reports -1 iterations for its frames.
 * Extension: no counterpart in the reference. */
int fecl_ldpc_set_persistent(fecl_codec_t codec, int32_t mode);

/* Windowed turbo decoder: training steps run before each segment's forward and
 * backward walk (a multiple of 8; -1 restores the default: 80 for max-log, 96 for
 * the log-MAP algorithms).  Training only
 * sets how often a segment boundary fails verification and is recomputed; results
 * do not depend on it beyond FP32 rounding. */
int fecl_turbo_set_window_training(fecl_codec_t codec, int32_t steps);

/* Windowed turbo decoder: forward (and backward) segments per frame, 32, 64 or 128,
 * one thread each (0 restores the built-in choice: 128 for a batch of at most one
 * frame per SM, whose time is one frame's latency; otherwise 64, with whole GPU rounds
 * of 32-segment frames first where a batch would otherwise end on a round less than
 * half full).  soDecode always uses 64.
 * Fewer, longer segments spend a smaller share of each walk on training and fit more
 * frames on an SM; results do not depend on it beyond FP32 rounding.  Extension: no
 * counterpart in the reference. */
int fecl_turbo_set_window_segments(fecl_codec_t codec, int32_t segments);

/* Windowed turbo decoder autotuner: decodes the caller's `nframes` frames of device
 * memory L-values (into msg) with every equivalent window shape -- 32, 64 or 128
 * segments per direction or the launcher's choice (0), 48 to 128 training steps --
 * keeps the fastest in the
 * codec and returns it.  Results are remembered per (K, nframes, algorithm,
 * iterations, scheduling) for the process, so later calls only apply them.  Every
 * shape computes the full-frame recursion up to FP32 rounding.  Extension: no
 * counterpart in the reference. */
int fecl_turbo_tune_window(fecl_codec_t codec, const void* llr, int32_t llr_dtype, uint64_t nframes, uint8_t* msg,
                           void* stream, int32_t* segments, int32_t* training);

/* Windowed turbo decoder counters since the previous call (which resets them):
 * constituent passes run, verification rounds that found a boundary to
 * recompute, and segments recomputed. */
int fecl_turbo_window_stats(fecl_codec_t codec, uint64_t* passes, uint64_t* fixup_rounds, uint64_t* recomputed);

/* Allocation-free LTE turbo decode.  No counterpart in the reference.  For callers
 * that cannot allocate device memory once running -- a pipeline that reserves its
 * whole memory budget at start-up, a real-time thread that must not block in
 * cudaMalloc, a plug-in host that owns the memory pool -- this decodes `nframes`
 * LTE turbo frames (the code of fecl_turbo_create_lte, Serial scheduling, scaling
 * 1.0) with the windowed kernel of fecl_decode, bit-identical to it, but calls no
 * cudaMalloc, cudaFree or allocating library routine.  Its scratch, interleaver and
 * scaling tables are fixed-size static device arrays (8 MiB of scratch, K <= 6144,
 * iterations <= 64) that every GPU loading the library holds until process exit;
 * a batch needing more scratch than 8 MiB (more than 68 frames at K = 6144) is
 * rejected with FECL_EINVAL.  llr ([nframes][3K+12]) and msg ([nframes][K] bytes)
 * are device memory of the current device; the call is asynchronous on `stream`.
 * The first call on a device looks up the arrays' device addresses there, so make
 * it once with each device current before relying on the call being cheap.  All
 * calls on a device share the arrays and overwrite them: calls that overlap on the
 * GPU (different streams, or different host threads) race and must be serialised
 * by the caller.  Every scratch element a call reads it first writes itself, so no
 * state carries over from one call to the next. */
int fecl_lte_turbo_decode_noalloc(uint32_t K, int32_t algorithm, uint32_t iterations, const void* llr,
                                  int32_t llr_dtype, uint64_t nframes, uint8_t* msg, void* stream);

/* ---- mixed batches (an extension) ------------------------------------------
 *
 * A batch decodes the frames of several codecs -- LDPC codes of any size and rate,
 * LTE turbo codes of any K, any other turbo code -- with one CUDA graph launch.
 * Every LTE turbo frame goes into one persistent launch over all K (longest
 * frames first); every other job gets the decoder fecl_decode would pick for it
 * (with FECL_BATCH_SHARED_LDPC the packed FP16 LDPC jobs instead share their
 * launches),
 * or, with FECL_BATCH_AUTOTUNE, the fastest of the LDPC kernel shapes that compute
 * the same bits, timed on the job's own data at creation and remembered for the
 * process.  Results equal those of fecl_decode on each job alone, bit for bit.
 *
 * Buffers are device memory of the codecs' device and stay bound to the batch:
 * write new L-values into the same buffers and run the batch again.  Runs of one
 * batch share its workspace and must not overlap (run it on one stream).  A codec
 * must outlive every batch that uses it; changing a codec's decoder options makes
 * fecl_batch_run fail with FECL_EINVAL until the batch is built again. */
typedef struct fecl_batch_s* fecl_batch_t;
typedef struct {
  fecl_codec_t codec;
  uint64_t nframes;
  const void* llr;     /* [nframes][paritySize] of llr_dtype, device memory */
  int32_t llr_dtype;
  uint8_t* msg;        /* [nframes][msgSize] hard decisions, device memory */
  int32_t* iterations; /* [nframes] or NULL */
} fecl_batch_job;
#define FECL_BATCH_AUTOTUNE 1
/* The LDPC jobs that take the packed FP16 decoder share their launches: per wave of
 * frame groups (from every such code, fitting in L2 together) one launch per check
 * pass and check-degree class and one per bit pass -- or, with
 * FECL_BATCH_SHARED_PERSISTENT, one persistent launch per class with grid barriers
 * between the passes.  The same bits as each job's own launches. */
#define FECL_BATCH_SHARED_LDPC 2
#define FECL_BATCH_SHARED_PERSISTENT 4
int fecl_batch_create(const fecl_batch_job* jobs, uint32_t njobs, int32_t flags, fecl_batch_t* out);
/* Launches the batch's graph on `stream` (asynchronous). */
int fecl_batch_run(fecl_batch_t batch, void* stream);
/* The kernel each job got, one line per job, NUL-terminated into text[size]. */
int fecl_batch_describe(fecl_batch_t batch, char* text, uint64_t size);
void fecl_batch_destroy(fecl_batch_t batch);

/* ---- decode server (an extension) ---------------------------------------------
 *
 * Continuous batching of decode requests.  A request is n frames of one codec with
 * host L-values in and host decisions out; any thread may submit.  The server keeps
 * up to `slots` batches in flight, each on its own stream with device_budget / slots
 * bytes of device memory; whenever a slot is free it admits the oldest waiting
 * requests that fit that memory and max_batch_frames, so requests that arrive while
 * other batches are on the GPU are decoded in the next one, overlapping the batches
 * still running.  Every LTE turbo frame of a batch goes into one mixed-K launch,
 * the frames of each other codec into one launch sequence.  A request's decisions do
 * not depend on the requests it was batched with: they equal fecl_decode's.
 * The request's buffers must stay valid until fecl_server_wait returns for it; the
 * codecs must outlive the server and keep their options while it runs. */
typedef struct fecl_server_s* fecl_server_t;
typedef struct {
  uint64_t device_budget_bytes; /* device memory for batches in flight (0: 40 GiB) */
  uint32_t max_batch_frames;    /* frames admitted into one batch (0: 2048) */
  uint32_t slots;               /* batches in flight at once (0: 3; at most 16) */
} fecl_server_options;
typedef struct {
  uint64_t requests, frames, info_bits, batches; /* finished since creation or the last reset */
  double p50_s, p99_s, max_s; /* request latency, submission to decisions in host memory */
  double wall_s;              /* first submission to last completion */
  double batch_gpu_s;         /* mean device time of a batch, first copy in to last copy out */
  double batch_host_s;        /* mean host time to lay out and launch a batch */
  double batch_frames;        /* mean frames per batch */
} fecl_server_stats;
int fecl_server_create(const fecl_server_options* options, fecl_server_t* out);
/* Queues nframes frames of `codec`: llr [nframes][paritySize] of llr_dtype, msg
 * [nframes][msgSize] bytes, iterations [nframes] or NULL, all host memory. */
int fecl_server_submit(fecl_server_t server, fecl_codec_t codec, const void* llr, int32_t llr_dtype, uint64_t nframes,
                       uint8_t* msg, int32_t* iterations, uint64_t* ticket);
/* Blocks until the request is done (FECL_ETIMEDOUT after timeout_s); its latency in seconds. */
int fecl_server_wait(fecl_server_t server, uint64_t ticket, double timeout_s, double* latency_s);
int fecl_server_report(fecl_server_t server, fecl_server_stats* stats);
int fecl_server_reset_stats(fecl_server_t server);
/* Load generator: submits request i at arrival_s[i] seconds after the call starts, from
 * the calling thread, then waits for all of them; latency_s[i] (nullable) receives
 * each latency.  Arrays are indexed by request. */
int fecl_server_replay(fecl_server_t server, uint64_t nreq, const double* arrival_s, const fecl_codec_t* codecs,
                       const void* const* llr, const int32_t* llr_dtype, const uint64_t* nframes, uint8_t* const* msg,
                       int32_t* const* iterations, double* latency_s);
void fecl_server_destroy(fecl_server_t server);

const char* fecl_strerror(int status);
/* Message of the last failing call on this thread. */
const char* fecl_last_error(void);

/* Library version and the device architecture the kernels were built for. */
const char* fecl_version(void);

#ifdef __cplusplus
}
#endif

#endif /* FECL_B200_H */
