// Host-side code descriptions: the structures the CUDA decoders consume.
//
// These restate, in this project's own data layout, the parts of FeCl's code
// structures that define what the decoders compute:
//   LdpcCode   -- detail::Ldpc::Structure (src/detail/Ldpc.h:96-137)
//   Trellis    -- fec::Trellis            (src/Trellis.h:131-172)
//   TurboCode  -- detail::Turbo::Structure (src/detail/Turbo.h:106-180) with its
//                 detail::Convolutional::Structure constituents (src/detail/Convolutional.h:81-125)
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

namespace fecl {

// Compressed sparse rows of a binary matrix; column indices sorted within a row.
struct Csr {
  uint32_t rows = 0;
  uint32_t cols = 0;
  std::vector<uint32_t> row_ptr{0};
  std::vector<uint32_t> col_idx;
  uint64_t nnz() const { return col_idx.size(); }
  uint32_t degree(uint32_t r) const { return row_ptr[r + 1] - row_ptr[r]; }
  static Csr from_rows(uint32_t cols, const std::vector<std::vector<uint32_t>>& rows);
  Csr transpose() const;
};

// ---------------------------------------------------------------- LDPC

struct LdpcDecoderConfig {
  int algorithm = 2;  // Approximate (src/detail/Ldpc.h:71)
  uint32_t iterations = 50;
  std::vector<std::vector<double>> scaling{{1.0}};  // [iteration][degree-2], see LdpcCode::scaling_factor
  int precision = 0;
  int fixed_iterations = 0;
};

class LdpcCode {
 public:
  // Ldpc::Structure(EncoderOptions(H), ...) -- src/detail/Ldpc.cpp:34-55, 216-331.
  explicit LdpcCode(const Csr& H);

  uint32_t msg_size() const { return msg_size_; }
  uint32_t syst_size() const { return msg_size_; }
  uint32_t parity_size() const { return H_.cols; }
  uint64_t state_size() const { return H_.nnz(); }
  const Csr& checks() const { return H_; }
  uint32_t max_check_degree() const { return max_degree_; }

  // Ldpc::Structure::setDecoderOptions / scalingMapToVector (src/detail/Ldpc.cpp:57-112);
  // `scaling` is already the [iteration][degree-2] table, validated here.
  void set_decoder(const LdpcDecoderConfig& cfg);
  const LdpcDecoderConfig& decoder() const { return dec_; }
  // Ldpc::Structure::scalingFactor(i, d) -- src/detail/Ldpc.cpp:134-138.
  double scaling_factor(size_t iteration, size_t degree) const;

  // Ldpc::Structure::encode / check -- src/detail/Ldpc.cpp:160-209.
  void encode(const uint8_t* msg, uint8_t* parity) const;
  bool check(const uint8_t* parity) const;

  // The generator pieces encode() walks, for the device encoder.
  const Csr& gen_dc() const { return DC_; }
  const Csr& gen_a() const { return A_; }
  const Csr& gen_b() const { return B_; }
  const Csr& gen_t() const { return T_; }

 private:
  void compute_generator(Csr H);

  uint32_t msg_size_ = 0;
  uint32_t max_degree_ = 0;
  Csr H_;   // transformed check matrix
  Csr DC_;  // gap parity as a function of the message
  Csr A_;   // T-part rows restricted to message columns
  Csr B_;   // T-part rows restricted to gap parity columns
  Csr T_;   // T-part (transposed): for column c, the T rows holding it
  LdpcDecoderConfig dec_;
};

// Standard DVB-S2 parity-check matrix (ETSI EN 302 307, 5.3.2): the check rows of
// info bit m in group g = m/360 are (x + (m mod 360) q) mod (N-K) for each table
// address x of group g; parity bits form the accumulator staircase.
Csr dvbs2_matrix(uint32_t n, uint32_t rate_num, uint32_t rate_den);

// Ldpc::Gallager::matrix -- src/Ldpc.cpp:77-102.
Csr gallager_matrix(uint32_t n, uint32_t wc, uint32_t wr, uint64_t seed);

// ---------------------------------------------------------------- trellis / turbo

struct Trellis {
  uint32_t state_size = 0;   // register count
  uint32_t input_size = 0;   // bits per branch input
  uint32_t output_size = 0;  // bits per branch output
  uint32_t state_count = 0;
  uint32_t input_count = 0;
  std::vector<uint32_t> next_state;  // [s * input_count + u]
  std::vector<uint32_t> output;      // [s * input_count + u]

  // Trellis(constraintLengths, generator, feedback) -- src/Trellis.cpp:76-143.
  static Trellis from_generators(const std::vector<uint32_t>& constraint_lengths,
                                 const std::vector<std::vector<uint64_t>>& generators,
                                 std::vector<uint64_t> feedback);
  // Trellis given by tables (state/output counts must be powers of two).
  static Trellis from_tables(uint32_t state_count, uint32_t input_count, uint32_t output_size,
                             const uint32_t* next_state, const uint32_t* output);
};

struct Constituent {
  Trellis trellis;
  uint32_t length = 0;       // trellis steps carrying message bits
  int termination = 0;       // 0 Tail, 1 Truncate
  uint32_t tail = 0;         // tail steps (state_size under Tail)
  std::vector<uint32_t> perm;  // out[i] = msg[perm[i]]
  uint32_t msg_size() const { return length * trellis.input_size; }
  uint32_t syst_size() const { return (length + tail) * trellis.input_size; }
  uint32_t syst_tail_size() const { return tail * trellis.input_size; }
  uint32_t parity_size() const { return (length + tail) * trellis.output_size; }
  // Convolutional::Structure::encode(msg, parity, tail) -- src/detail/Convolutional.cpp:167-221.
  void encode(const uint8_t* msg, uint8_t* parity, uint8_t* tail_bits) const;
};

// A stage of a custom schedule (detail::Turbo::Stage, src/detail/Turbo.h:38-48): the
// constituents decoded in the stage, and for the k-th of them (after sorting) the
// constituents whose extrinsic values form its a-priori input.
struct TurboStage {
  std::vector<uint32_t> activation;
  std::vector<std::vector<uint32_t>> transfer;
};

struct TurboDecoderConfig {
  int algorithm = 1;  // Linear (src/detail/Turbo.h:99)
  uint32_t iterations = 6;
  int scheduling = 0;  // Serial
  std::vector<std::vector<double>> scaling{{1.0}};  // [constituent][iteration]
  int precision = 0;
  std::vector<TurboStage> schedule;  // scheduling == Custom
  int crc = 0;  // an extension: 0 none, 1 CRC-24A, 2 CRC-24B -- decode stops a frame whose CRC checks
};

// x^(K-1-i) x^24 mod g(x) for i < K: the CRC register a K-bit block with only bit i set
// leaves, so that a block's syndrome is the xor of the entries of its one bits.
std::vector<uint32_t> crc24_syndrome_table(uint32_t K, uint32_t poly);

class TurboCode {
 public:
  // Turbo::Structure::setEncoderOptions -- src/detail/Turbo.cpp:45-103.
  TurboCode(const std::vector<Trellis>& trellis, const std::vector<std::vector<uint32_t>>& perms,
            const std::vector<int>& termination);

  uint32_t msg_size() const { return msg_size_; }
  uint32_t syst_size() const { return syst_size_; }
  uint32_t parity_size() const { return parity_size_; }
  uint32_t state_size() const { return state_size_; }
  uint32_t syst_tail_size() const { return tail_size_; }
  const std::vector<Constituent>& constituents() const { return c_; }

  // Turbo::Structure::setDecoderOptions -- src/detail/Turbo.cpp:105-140.
  void set_decoder(const TurboDecoderConfig& cfg);
  const TurboDecoderConfig& decoder() const { return dec_; }
  // Turbo::Structure::scalingFactor(i, j) -- src/detail/Turbo.cpp:148-153.
  double scaling_factor(size_t iteration, size_t constituent) const;

  // Turbo::Structure::encode / check -- src/detail/Turbo.cpp:155-198.
  void encode(const uint8_t* msg, uint8_t* parity) const;
  bool check(const uint8_t* parity) const;

  // True for the LTE code shape the specialised kernel handles: two 8-state
  // rate-1/2 constituents with Tail termination, the first un-interleaved.
  bool is_lte_shape() const;

 private:
  uint32_t msg_size_ = 0, syst_size_ = 0, parity_size_ = 0, state_size_ = 0, tail_size_ = 0;
  std::vector<Constituent> c_;
  TurboDecoderConfig dec_;
};

// ---------------------------------------------------------------- convolutional

struct ConvDecoderConfig {
  int algorithm = 2;   // Approximate (src/detail/Convolutional.h:60)
  double scaling = 1.0;
};

// detail::Convolutional::Structure (src/detail/Convolutional.h:81-125,
// src/detail/Convolutional.cpp:45-221): one trellis over `length` steps, Truncate
// (the default) or Tail termination.  The codeword is the trellis output bits only;
// the tail inputs belong to the systematic part (systSize) but are not transmitted.
class ConvCode {
 public:
  ConvCode(const Trellis& trellis, uint32_t length, int termination);

  uint32_t msg_size() const { return c_.msg_size(); }
  uint32_t syst_size() const { return c_.syst_size(); }
  uint32_t parity_size() const { return c_.parity_size(); }
  uint32_t state_size() const { return 0; }
  const Constituent& constituent() const { return c_; }

  void set_decoder(const ConvDecoderConfig& cfg);
  const ConvDecoderConfig& decoder() const { return dec_; }

  // Convolutional::Structure::encode / check (src/detail/Convolutional.cpp:167-221,
  // and the greedy path search of check).
  void encode(const uint8_t* msg, uint8_t* parity) const;
  bool check(const uint8_t* parity) const;

 private:
  Constituent c_;
  ConvDecoderConfig dec_;
};

// Turbo::Lte3Gpp::interleaver -- src/Lte3Gpp.cpp:219-237.
std::vector<uint32_t> lte_interleaver(uint32_t K);
bool lte_qpp_params(uint32_t K, uint32_t* f1, uint32_t* f2);
// The LTE RSC, Trellis({4}, {{015}}, {013}).
Trellis lte_trellis();

}  // namespace fecl
