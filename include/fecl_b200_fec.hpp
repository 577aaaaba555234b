// fecl_b200_fec.hpp -- FeCl's C++ API (namespace fec) on top of the fecl_b200 C-ABI.
//
// Header-only.  A program written against the reference's headers (src/Codec.h,
// src/Ldpc.h, src/Turbo.h, src/Trellis.h, src/BitField.h, src/Permutation.h) keeps
// its calls: construct fec::Ldpc / fec::Turbo from the same option builders, then
// Codec::encode / check / decode / soDecode with std::vector buffers, with the
// same exceptions for invalid sizes and options (std::invalid_argument).  Decoding
// runs on the GPU through fecl_decode / fecl_so_decode; everything else is host
// code in libfecl_b200.so.  Link with -lfecl_b200.
//
// Also here: fec::Convolutional (Viterbi decode, MAP soDecode), Custom turbo
// scheduling (Turbo::DecoderOptions::scheduling(Scheduling)), Codec::puncturing with
// each family's PunctureOptions, and fec::Permutation's permute / dePermute.
//
// Not carried over: Boost serialization (save/load).
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>

#include "fecl_b200.h"

namespace fec {

namespace detail {
inline void check_status(int status) {
  if (status == FECL_OK) return;
  if (status == FECL_EINVAL) throw std::invalid_argument(fecl_last_error());
  throw std::runtime_error(std::string(fecl_last_error()) + " (" + fecl_strerror(status) + ")");
}
}  // namespace detail

// src/DecoderAlgorithm.h:30-34, src/SchedulingType.h:32-39
enum DecoderAlgorithm { Exact = FECL_EXACT, Linear = FECL_LINEAR, Approximate = FECL_APPROXIMATE };
enum SchedulingType { Serial = FECL_SERIAL, Parallel = FECL_PARALLEL, Custom = FECL_CUSTOM };

// One bit (or a small bit vector) per word, as src/BitField.h's BitField<size_t>.
template <typename T>
class BitField {
 public:
  BitField() = default;
  BitField(T v) : value_(v) {}
  operator T() const { return value_; }
  bool test(size_t i) const { return (value_ >> i) & 1; }
  void set(size_t i) { value_ |= T(1) << i; }
 private:
  T value_ = 0;
};

// A sparse binary matrix with sorted rows (the subset of src/BitMatrix.h the codes use).
class SparseBitMatrix {
 public:
  SparseBitMatrix() = default;
  SparseBitMatrix(size_t rows, size_t cols) : cols_(cols), rows_(rows) {}
  SparseBitMatrix(const std::vector<std::vector<size_t>>& rows, size_t cols) : cols_(cols), rows_(rows) {}
  size_t rows() const { return rows_.size(); }
  size_t cols() const { return cols_; }
  size_t size() const {
    size_t n = 0;
    for (auto& r : rows_) n += r.size();
    return n;
  }
  const std::vector<size_t>& row(size_t r) const { return rows_[r]; }
  // appends column j to row r; columns must be added in increasing order (as RowRef::set)
  void set(size_t r, size_t j) { rows_[r].push_back(j); }
  std::vector<size_t> rowSizes() const {
    std::vector<size_t> s;
    for (auto& r : rows_) s.push_back(r.size());
    return s;
  }
  void csr(std::vector<uint32_t>& row_ptr, std::vector<uint32_t>& col_idx) const {
    row_ptr.assign(1, 0);
    col_idx.clear();
    for (auto& r : rows_) {
      for (auto c : r) col_idx.push_back(uint32_t(c));
      row_ptr.push_back(uint32_t(col_idx.size()));
    }
  }
  static SparseBitMatrix from_csr(uint32_t rows, uint32_t cols, const std::vector<uint32_t>& row_ptr,
                                  const std::vector<uint32_t>& col_idx) {
    SparseBitMatrix m(rows, cols);
    for (uint32_t r = 0; r < rows; ++r)
      for (uint32_t e = row_ptr[r]; e < row_ptr[r + 1]; ++e) m.rows_[r].push_back(col_idx[e]);
    return m;
  }
 private:
  size_t cols_ = 0;
  std::vector<std::vector<size_t>> rows_;
};

// fec::Permutation, src/Permutation.h:32-70: out[i] = in[sequence[i]] per block of
// inputSize() values; dePermute scatters back (out[sequence[i]] = in[i]), so with a
// repeated index the last one wins and unmapped positions keep what the output held.
class Permutation {
 public:
  Permutation() = default;
  Permutation(const std::vector<size_t>& sequence) : seq_(sequence) {
    for (auto v : seq_) input_ = std::max(input_, v + 1);
  }
  Permutation(std::vector<size_t> sequence, size_t inputSize) : seq_(std::move(sequence)), input_(inputSize) {}
  size_t inputSize() const { return input_; }
  size_t outputSize() const { return seq_.size(); }
  size_t operator[](size_t i) const { return seq_[i]; }
  const std::vector<size_t>& sequence() const { return seq_; }

  template <typename T1, typename T2 = T1>
  void permute(const std::vector<T1>& in, std::vector<T2>& out) const {
    const size_t n = input_ ? in.size() / input_ : 0;
    out.resize(n * seq_.size());
    for (size_t b = 0; b < n; ++b)
      for (size_t i = 0; i < seq_.size(); ++i) out[b * seq_.size() + i] = in[b * input_ + seq_[i]];
  }
  template <typename T1, typename T2 = T1>
  void dePermute(const std::vector<T1>& in, std::vector<T2>& out) const {
    const size_t n = seq_.empty() ? 0 : in.size() / seq_.size();
    out.resize(n * input_);
    for (size_t b = 0; b < n; ++b)
      for (size_t i = 0; i < seq_.size(); ++i) out[b * input_ + seq_[i]] = in[b * seq_.size() + i];
  }
  template <typename T>
  std::vector<T> permute(const std::vector<T>& in) const {
    std::vector<T> out;
    permute(in, out);
    return out;
  }
  template <typename T>
  std::vector<T> dePermute(const std::vector<T>& in) const {
    std::vector<T> out;
    dePermute(in, out);
    return out;
  }

 private:
  std::vector<size_t> seq_;
  size_t input_ = 0;
};

namespace detail {
// The kept indices of a puncturing call, as a Permutation of paritySize() inputs.
template <class F>
Permutation puncture_list(size_t parity, F call) {
  uint64_t n = 0;
  check_status(call(nullptr, &n));
  std::vector<uint32_t> seq(n);
  check_status(call(seq.data(), &n));
  return Permutation(std::vector<size_t>(seq.begin(), seq.end()), parity);
}
inline std::vector<uint8_t> bytes(const std::vector<bool>& m) { return std::vector<uint8_t>(m.begin(), m.end()); }
}  // namespace detail

// src/Trellis.h:131-172; built by Trellis(constraintLengths, generator, feedback), src/Trellis.cpp:76-143.
class Trellis {
 public:
  enum Termination { Tail = FECL_TAIL, Truncate = FECL_TRUNCATE };
  Trellis(const std::vector<size_t>& constraintLengths, const std::vector<std::vector<BitField<size_t>>>& generator,
          const std::vector<BitField<size_t>>& feedback = {}) {
    std::vector<uint32_t> cl(constraintLengths.begin(), constraintLengths.end());
    if (generator.empty()) throw std::invalid_argument("Invalid number of generators");
    const size_t nout = generator[0].size();
    std::vector<uint64_t> gen;
    for (auto& g : generator) {
      if (g.size() != nout) throw std::invalid_argument("Invalid number of generators");
      for (auto v : g) gen.push_back(uint64_t(size_t(v)));
    }
    std::vector<uint64_t> fb;
    for (auto v : feedback) fb.push_back(uint64_t(size_t(v)));
    uint32_t sc = 0, ic = 0, os = 0;
    detail::check_status(fecl_trellis_build(uint32_t(cl.size()), cl.data(), uint32_t(nout), gen.data(),
                                            fb.empty() ? nullptr : fb.data(), &sc, &ic, &os, nullptr, nullptr));
    next_.resize(size_t(sc) * ic);
    out_.resize(size_t(sc) * ic);
    detail::check_status(fecl_trellis_build(uint32_t(cl.size()), cl.data(), uint32_t(nout), gen.data(),
                                            fb.empty() ? nullptr : fb.data(), &sc, &ic, &os, next_.data(), out_.data()));
    states_ = sc;
    inputs_ = ic;
    outputs_ = os;
  }
  size_t stateCount() const { return states_; }
  size_t inputCount() const { return inputs_; }
  size_t outputSize() const { return outputs_; }
  BitField<size_t> getNextState(size_t s, size_t u) const { return next_[s * inputs_ + u]; }
  BitField<size_t> getOutput(size_t s, size_t u) const { return out_[s * inputs_ + u]; }
  fecl_trellis table() const { return fecl_trellis{states_, inputs_, outputs_, next_.data(), out_.data()}; }
 private:
  uint32_t states_ = 0, inputs_ = 0, outputs_ = 0;
  std::vector<uint32_t> next_, out_;
};

// The syst / parity / state / msg bundle of Codec::soDecode (src/detail/Codec.h:142-171).
template <class Vector>
class Info {
 public:
  Info& syst(Vector& v) { syst_ = &v; return *this; }
  Info& parity(Vector& v) { parity_ = &v; return *this; }
  Info& state(Vector& v) { state_ = &v; return *this; }
  Info& msg(Vector& v) { msg_ = &v; return *this; }
  Vector& syst() const { return *syst_; }
  Vector& parity() const { return *parity_; }
  Vector& state() const { return *state_; }
  Vector& msg() const { return *msg_; }
  bool hasSyst() const { return syst_ != nullptr; }
  bool hasParity() const { return parity_ != nullptr; }
  bool hasState() const { return state_ != nullptr; }
  bool hasMsg() const { return msg_ != nullptr; }
 private:
  Vector* syst_ = nullptr;
  Vector* parity_ = nullptr;
  Vector* state_ = nullptr;
  Vector* msg_ = nullptr;
};

// fec::Codec, src/Codec.h:46-127.
class Codec {
 public:
  template <template <typename> class A = std::allocator>
  using Input = Info<const std::vector<double, A<double>>>;
  template <template <typename> class A = std::allocator>
  using Output = Info<std::vector<double, A<double>>>;

  virtual ~Codec() = default;
  size_t msgSize() const { return sizes_.msg; }
  size_t systSize() const { return sizes_.syst; }
  size_t paritySize() const { return sizes_.parity; }
  size_t stateSize() const { return sizes_.state; }
  int getWorkGroupSize() const { return work_group_; }
  void setWorkGroupSize(int n) { work_group_ = n; }  // a CPU thread count in the reference; ignored

  template <template <typename> class A = std::allocator>
  bool check(const std::vector<BitField<size_t>, A<BitField<size_t>>>& parity) const {
    const size_t n = blocks(parity.size(), paritySize(), "Invalid size for parity");
    std::vector<uint8_t> p(parity.begin(), parity.end());
    int32_t ok = 0;
    detail::check_status(fecl_check(handle(), p.data(), n, &ok));
    return ok != 0;
  }

  template <template <typename> class A = std::allocator>
  void encode(const std::vector<BitField<size_t>, A<BitField<size_t>>>& msg,
              std::vector<BitField<size_t>, A<BitField<size_t>>>& parity) const {
    const size_t n = blocks(msg.size(), msgSize(), "Invalid size for message");
    std::vector<uint8_t> m(msg.size()), p(n * paritySize());
    for (size_t i = 0; i < msg.size(); ++i) m[i] = uint8_t(size_t(msg[i]) & 1);
    detail::check_status(fecl_encode(handle(), m.data(), n, p.data(), FECL_HOST_MEMORY, nullptr));
    parity.assign(p.begin(), p.end());
  }
  template <template <typename> class A = std::allocator>
  std::vector<BitField<size_t>, A<BitField<size_t>>> encode(const std::vector<BitField<size_t>, A<BitField<size_t>>>& msg) const {
    std::vector<BitField<size_t>, A<BitField<size_t>>> p;
    encode(msg, p);
    return p;
  }

  template <template <typename> class A = std::allocator>
  void decode(const std::vector<double, A<double>>& parity, std::vector<BitField<size_t>, A<BitField<size_t>>>& msg) const {
    const size_t n = blocks(parity.size(), paritySize(), "Invalid size for parity");
    std::vector<uint8_t> m(n * msgSize());
    if (n) detail::check_status(fecl_decode(handle(), parity.data(), FECL_F64, n, m.data(), nullptr, FECL_HOST_MEMORY, nullptr));
    msg.assign(m.begin(), m.end());
  }
  template <template <typename> class A = std::allocator>
  std::vector<BitField<size_t>, A<BitField<size_t>>> decode(const std::vector<double, A<double>>& parity) const {
    std::vector<BitField<size_t>, A<BitField<size_t>>> m;
    decode(parity, m);
    return m;
  }

  // Codec::soDecode, src/Codec.h:249-307, with the same checks and messages.
  template <template <typename> class A = std::allocator>
  void soDecode(Input<A> input, Output<A> output) const {
    if (!input.hasParity()) throw std::invalid_argument("Input must contains parity");
    if (input.hasMsg()) throw std::invalid_argument("Input should not contain msg");
    const size_t n = blocks(input.parity().size(), paritySize(), "Invalid size for parity");
    if (input.hasSyst() && input.syst().size() != n * systSize()) throw std::invalid_argument("Invalid size for msg");
    if (input.hasState() && input.state().size() != n * stateSize()) throw std::invalid_argument("Invalid size for state");
    if (output.hasParity()) output.parity().resize(n * paritySize());
    if (output.hasSyst()) output.syst().resize(n * systSize());
    if (output.hasState()) output.state().resize(n * stateSize());
    if (output.hasMsg()) output.msg().resize(n * msgSize());
    if (n == 0) return;
    fecl_so_io io{};
    io.parity = input.parity().data();
    io.syst = input.hasSyst() ? input.syst().data() : nullptr;
    io.state = input.hasState() ? input.state().data() : nullptr;
    io.in_dtype = FECL_F64;
    io.msg = output.hasMsg() ? output.msg().data() : nullptr;
    io.syst_out = output.hasSyst() ? output.syst().data() : nullptr;
    io.parity_out = output.hasParity() ? output.parity().data() : nullptr;
    io.state_out = output.hasState() ? output.state().data() : nullptr;
    io.out_dtype = FECL_F64;
    detail::check_status(fecl_so_decode(handle(), &io, n, FECL_HOST_MEMORY, nullptr));
  }

 protected:
  Codec() = default;
  void attach(fecl_codec_t h) {
    handle_.reset(h, [](fecl_codec_t c) { fecl_destroy(c); });
    detail::check_status(fecl_codec_sizes(h, &sizes_));
  }
  fecl_codec_t handle() const { return handle_.get(); }
  static size_t blocks(size_t size, size_t unit, const char* what) {
    const size_t n = unit ? size / unit : 0;
    if (n * unit != size) throw std::invalid_argument(what);
    return n;
  }
 private:
  std::shared_ptr<fecl_codec_s> handle_;
  fecl_sizes sizes_{};
  int work_group_ = 8;
};

namespace detail {
struct LdpcDecoderOptions {  // src/detail/Ldpc.h:56-74 (iterations default to 50 here)
  LdpcDecoderOptions& algorithm(DecoderAlgorithm a) { algorithm_ = a; return *this; }
  LdpcDecoderOptions& iterations(size_t n) { iterations_ = n; return *this; }
  LdpcDecoderOptions& scalingFactor(double f) { scaling_ = {{0, {f}}}; return *this; }
  LdpcDecoderOptions& scalingFactor(const std::unordered_map<size_t, std::vector<double>>& f) { scaling_ = f; return *this; }
  DecoderAlgorithm algorithm() const { return algorithm_; }
  size_t iterations() const { return iterations_; }
  std::unordered_map<size_t, std::vector<double>> scalingFactor() const { return scaling_; }
  DecoderAlgorithm algorithm_ = Approximate;
  size_t iterations_ = 50;
  std::unordered_map<size_t, std::vector<double>> scaling_{{0, {1.0}}};
};

// Turbo::Stage, src/detail/Turbo.h:38-48: the constituents a stage activates and, per
// activation, the constituents whose extrinsic values form its a-priori input.
struct TurboStage {
  std::vector<size_t> activation;
  std::vector<std::vector<size_t>> transfer;
};

struct TurboDecoderOptions {  // src/detail/Turbo.h:77-101
  TurboDecoderOptions& iterations(size_t n) { iterations_ = n; return *this; }
  TurboDecoderOptions& scheduling(SchedulingType s) { scheduling_ = s; return *this; }
  TurboDecoderOptions& scheduling(const std::vector<TurboStage>& stages) {
    scheduling_ = Custom;
    stages_ = stages;
    return *this;
  }
  std::vector<TurboStage> scheduling() const { return stages_; }
  TurboDecoderOptions& algorithm(DecoderAlgorithm a) { algorithm_ = a; return *this; }
  TurboDecoderOptions& scalingFactor(double f) { scaling_ = {{f}}; return *this; }
  TurboDecoderOptions& scalingFactor(const std::vector<std::vector<double>>& f) { scaling_ = f; return *this; }
  size_t iterations() const { return iterations_; }
  SchedulingType schedulingType() const { return scheduling_; }
  DecoderAlgorithm algorithm() const { return algorithm_; }
  std::vector<std::vector<double>> scalingFactor() const { return scaling_; }
  size_t iterations_ = 6;
  SchedulingType scheduling_ = Serial;
  DecoderAlgorithm algorithm_ = Linear;
  std::vector<std::vector<double>> scaling_{{1.0}};
  std::vector<TurboStage> stages_;
};
}  // namespace detail

// fec::Ldpc, src/Ldpc.h:59-108.
class Ldpc : public Codec {
 public:
  struct EncoderOptions {
    EncoderOptions(const SparseBitMatrix& H) : checkMatrix_(H) {}
    SparseBitMatrix checkMatrix() const { return checkMatrix_; }
    SparseBitMatrix checkMatrix_;
  };
  using DecoderOptions = detail::LdpcDecoderOptions;
  struct PunctureOptions {  // src/detail/Ldpc.h:76-88
    PunctureOptions& mask(std::vector<bool> m) { mask_ = std::move(m); return *this; }
    PunctureOptions& systMask(std::vector<bool> m) { systMask_ = std::move(m); return *this; }
    std::vector<bool> mask_, systMask_;
  };
  struct DvbS2 {
    // the standard matrix for n in {16200, 64800}; rate as in src/DvbS2.cpp:27-29
    static SparseBitMatrix matrix(size_t n, double rate) {
      static const int fr[][2] = {{1, 4}, {1, 3}, {2, 5}, {1, 2}, {3, 5}, {2, 3}, {3, 4}, {4, 5}, {5, 6}, {8, 9}, {9, 10}};
      for (auto& f : fr) {
        if (std::fabs(rate - double(f[0]) / f[1]) < 1e-9) {
          uint32_t rows = 0, cols = 0;
          uint64_t nnz = 0;
          detail::check_status(fecl_dvbs2_matrix(uint32_t(n), f[0], f[1], &rows, &cols, &nnz, nullptr, nullptr));
          std::vector<uint32_t> rp(rows + 1), ci(nnz);
          detail::check_status(fecl_dvbs2_matrix(uint32_t(n), f[0], f[1], &rows, &cols, &nnz, rp.data(), ci.data()));
          return SparseBitMatrix::from_csr(rows, cols, rp, ci);
        }
      }
      throw std::invalid_argument("Invalid rate");
    }
  };
  struct Gallager {
    static SparseBitMatrix matrix(size_t n, size_t wc, size_t wr, uint64_t seed = 0) {
      uint32_t rows = 0;
      uint64_t nnz = 0;
      detail::check_status(fecl_gallager_matrix(uint32_t(n), uint32_t(wc), uint32_t(wr), seed, &rows, &nnz, nullptr, nullptr));
      std::vector<uint32_t> rp(rows + 1), ci(nnz);
      detail::check_status(fecl_gallager_matrix(uint32_t(n), uint32_t(wc), uint32_t(wr), seed, &rows, &nnz, rp.data(), ci.data()));
      return SparseBitMatrix::from_csr(rows, uint32_t(n), rp, ci);
    }
  };

  Ldpc(const EncoderOptions& encoder, const DecoderOptions& decoder = DecoderOptions(), int workGroupSize = 8)
      : H_(encoder.checkMatrix_) {
    std::vector<uint32_t> rp, ci;
    H_.csr(rp, ci);
    std::vector<double> table;
    fecl_ldpc_options o = options(decoder, table);
    fecl_codec_t h = nullptr;
    detail::check_status(fecl_ldpc_create(uint32_t(H_.rows()), uint32_t(H_.cols()), rp.data(), ci.data(), &o, &h));
    attach(h);
    decoder_ = decoder;
    setWorkGroupSize(workGroupSize);
  }
  void setDecoderOptions(const DecoderOptions& decoder) {
    std::vector<double> table;
    fecl_ldpc_options o = options(decoder, table);
    detail::check_status(fecl_ldpc_set_options(handle(), &o));
    decoder_ = decoder;
  }
  DecoderOptions getDecoderOptions() const { return decoder_; }
  // Ldpc::puncturing, src/Ldpc.h:94 (src/detail/Ldpc.cpp:333-353).
  Permutation puncturing(const PunctureOptions& o) const {
    const auto m = detail::bytes(o.mask_), sm = detail::bytes(o.systMask_);
    return detail::puncture_list(paritySize(), [&](uint32_t* seq, uint64_t* n) {
      return fecl_ldpc_puncturing(handle(), m.data(), uint32_t(m.size()), sm.data(), uint32_t(sm.size()), seq, n);
    });
  }

 private:
  // scalingMapToVector, src/detail/Ldpc.cpp:64-112: {degree: per-iteration} with key 0
  // as default -> [iterations or 1][maxDegree - 1].
  fecl_ldpc_options options(const DecoderOptions& d, std::vector<double>& table) const {
    const auto deg = H_.rowSizes();
    size_t maxd = 0;
    for (auto v : deg) maxd = std::max(maxd, v);
    const auto& m = d.scaling_;
    std::vector<std::vector<double>> vec;
    auto def = m.find(0);
    if (def != m.end()) {
      if (def->second.size() != 1 && def->second.size() != d.iterations_) throw std::invalid_argument("Wrong size for scaling factor");
      vec.resize(def->second.size());
      for (size_t i = 0; i < vec.size(); ++i) vec[i].assign(maxd - 1, def->second[i]);
      for (auto& kv : m)
        if (kv.first >= 2 && kv.first - 2 < maxd - 1) {
          if (kv.second.size() != vec.size()) throw std::invalid_argument("Wrong size for scaling factor");
          for (size_t j = 0; j < vec.size(); ++j) vec[j][kv.first - 2] = kv.second[j];
        }
    } else {
      size_t length = 0;
      for (auto& kv : m) length = std::max(length, kv.second.size());
      if (length != 1 && length != d.iterations_) throw std::invalid_argument("Wrong size for scaling factor");
      vec.assign(length, std::vector<double>(maxd - 1, 0.0));
      for (auto dg : deg) {
        auto it = m.find(dg);
        if (it == m.end()) throw std::invalid_argument("Scaling factor not defined and no default");
        if (it->second.size() != length) throw std::invalid_argument("Wrong size for scaling factor");
        for (size_t j = 0; j < length; ++j) vec[j][dg - 2] = it->second[j];
      }
    }
    table.clear();
    for (auto& r : vec) table.insert(table.end(), r.begin(), r.end());
    fecl_ldpc_options o{};
    o.algorithm = d.algorithm_;
    o.iterations = uint32_t(d.iterations_);
    o.scaling = table.data();
    o.scaling_iterations = uint32_t(vec.size());
    o.scaling_degrees = uint32_t(maxd - 1);
    return o;
  }
  SparseBitMatrix H_;
  DecoderOptions decoder_;
};

// fec::Turbo, src/Turbo.h:55-116.
class Turbo : public Codec {
 public:
  struct EncoderOptions {  // src/detail/Turbo.h:59-72
    EncoderOptions(const Trellis& t, const std::vector<Permutation>& p) : trellis_{t}, perms_(p) {}
    EncoderOptions(const std::vector<Trellis>& t, const std::vector<Permutation>& p) : trellis_(t), perms_(p) {}
    EncoderOptions& interleaver(const std::vector<Permutation>& p) { perms_ = p; return *this; }
    EncoderOptions& termination(Trellis::Termination t) { term_ = {t}; return *this; }
    EncoderOptions& termination(const std::vector<Trellis::Termination>& t) { term_ = t; return *this; }
    std::vector<Trellis> trellis_;
    std::vector<Permutation> perms_;
    std::vector<Trellis::Termination> term_{Trellis::Tail};
  };
  using DecoderOptions = detail::TurboDecoderOptions;
  using Stage = detail::TurboStage;
  using Scheduling = std::vector<Stage>;
  enum BitOrdering { Alternate = 0, Group = 1 };  // src/detail/Turbo.h:54-57
  struct PunctureOptions {                         // src/detail/Turbo.h:103-116
    PunctureOptions& mask(std::vector<std::vector<bool>> m) { mask_ = std::move(m); return *this; }
    PunctureOptions& tailMask(std::vector<std::vector<bool>> m) { tailMask_ = std::move(m); return *this; }
    PunctureOptions& bitOrdering(BitOrdering b) { bitOrdering_ = b; return *this; }
    std::vector<std::vector<bool>> mask_, tailMask_;
    BitOrdering bitOrdering_ = Alternate;
  };
  struct Lte3Gpp {
    static Permutation interleaver(size_t K) {
      std::vector<uint32_t> p(K);
      detail::check_status(fecl_lte_interleaver(uint32_t(K), p.data()));
      return Permutation(std::vector<size_t>(p.begin(), p.end()));
    }
  };

  Turbo(const EncoderOptions& e, const DecoderOptions& d = DecoderOptions(), int workGroupSize = 8) {
    std::vector<fecl_trellis> tr;
    for (auto& t : e.trellis_) tr.push_back(t.table());
    std::vector<uint32_t> data, len;
    for (auto& p : e.perms_) {
      for (auto v : p.sequence()) data.push_back(uint32_t(v));
      len.push_back(uint32_t(p.outputSize()));
    }
    std::vector<int32_t> term(e.term_.begin(), e.term_.end());
    std::vector<double> table;
    Schedule sched;
    fecl_turbo_options o = options(d, table, sched);
    fecl_codec_t h = nullptr;
    detail::check_status(fecl_turbo_create(uint32_t(e.perms_.size()), tr.data(), uint32_t(tr.size()),
                                           data.empty() ? nullptr : data.data(), len.data(), term.data(),
                                           uint32_t(term.size()), &o, &h));
    attach(h);
    decoder_ = d;
    setWorkGroupSize(workGroupSize);
  }
  void setDecoderOptions(const DecoderOptions& d) {
    std::vector<double> table;
    Schedule sched;
    fecl_turbo_options o = options(d, table, sched);
    detail::check_status(fecl_turbo_set_options(handle(), &o));
    decoder_ = d;
  }
  DecoderOptions getDecoderOptions() const { return decoder_; }
  // Turbo::puncturing, src/Turbo.h:102 (src/detail/Turbo.cpp:200-320).
  Permutation puncturing(const PunctureOptions& o) const {
    std::vector<uint8_t> md, td;
    std::vector<uint32_t> ml, tl;
    for (auto& m : o.mask_) {
      md.insert(md.end(), m.begin(), m.end());
      ml.push_back(uint32_t(m.size()));
    }
    for (auto& m : o.tailMask_) {
      td.insert(td.end(), m.begin(), m.end());
      tl.push_back(uint32_t(m.size()));
    }
    return detail::puncture_list(paritySize(), [&](uint32_t* seq, uint64_t* n) {
      return fecl_turbo_puncturing(handle(), md.data(), ml.data(), uint32_t(ml.size()), td.data(), tl.data(),
                                   uint32_t(tl.size()), int32_t(o.bitOrdering_), seq, n);
    });
  }

 private:
  // A Custom schedule flattened into the arrays of fecl_turbo_options.
  struct Schedule {
    std::vector<uint32_t> stage_counts, activation, transfer_counts, transfer;
  };
  static fecl_turbo_options options(const DecoderOptions& d, std::vector<double>& table, Schedule& sc) {
    // rows of 1 entry repeat over the iterations (Turbo::Structure::scalingFactor cycles them)
    size_t cols = 1;
    for (auto& r : d.scaling_) cols = std::max(cols, r.size());
    table.clear();
    for (auto& r : d.scaling_) {
      if (r.empty() || (r.size() != cols && r.size() != 1)) throw std::invalid_argument("Wrong size for scaling factor");
      for (size_t i = 0; i < cols; ++i) table.push_back(r[i % r.size()]);
    }
    fecl_turbo_options o{};
    o.algorithm = d.algorithm_;
    o.iterations = uint32_t(d.iterations_);
    o.scheduling = d.scheduling_;
    o.scaling = table.data();
    o.scaling_rows = uint32_t(d.scaling_.size());
    o.scaling_cols = uint32_t(cols);
    if (d.scheduling_ == Custom) {
      for (auto& st : d.stages_) {
        if (st.activation.size() != st.transfer.size())
          throw std::invalid_argument("Invalid scheduling : activation and transfer not the same size");
        sc.stage_counts.push_back(uint32_t(st.activation.size()));
        for (size_t a = 0; a < st.activation.size(); ++a) {
          sc.activation.push_back(uint32_t(st.activation[a]));
          sc.transfer_counts.push_back(uint32_t(st.transfer[a].size()));
          for (auto j : st.transfer[a]) sc.transfer.push_back(uint32_t(j));
        }
      }
      o.n_stages = uint32_t(sc.stage_counts.size());
      o.stage_counts = sc.stage_counts.data();
      o.activation = sc.activation.data();
      o.transfer_counts = sc.transfer_counts.data();
      o.transfer = sc.transfer.data();
    }
    return o;
  }
  DecoderOptions decoder_;
};

// fec::Convolutional, src/Convolutional.h:40-80: decode is the Viterbi decoder, soDecode
// one MAP pass.
namespace detail {
struct ConvEncoderOptions {  // src/detail/Convolutional.h:36-46
  ConvEncoderOptions(const Trellis& trellis, size_t length) : trellis_(trellis), length_(length) {}
  ConvEncoderOptions& termination(Trellis::Termination t) { termination_ = t; return *this; }
  Trellis trellis_;
  size_t length_;
  Trellis::Termination termination_ = Trellis::Truncate;
};
struct ConvDecoderOptions {  // src/detail/Convolutional.h:48-62
  ConvDecoderOptions& algorithm(DecoderAlgorithm a) { algorithm_ = a; return *this; }
  ConvDecoderOptions& scalingFactor(double f) { scaling_ = f; return *this; }
  DecoderAlgorithm algorithm() const { return algorithm_; }
  double scalingFactor() const { return scaling_; }
  DecoderAlgorithm algorithm_ = Approximate;
  double scaling_ = 1.0;
};
struct ConvPunctureOptions {  // src/detail/Convolutional.h:64-75
  ConvPunctureOptions& mask(std::vector<bool> m) { mask_ = std::move(m); return *this; }
  ConvPunctureOptions& tailMask(std::vector<bool> m) { tailMask_ = std::move(m); return *this; }
  std::vector<bool> mask_, tailMask_;
};
}  // namespace detail

class Convolutional : public Codec {
 public:
  using EncoderOptions = detail::ConvEncoderOptions;
  using DecoderOptions = detail::ConvDecoderOptions;
  using PunctureOptions = detail::ConvPunctureOptions;

  Convolutional(const EncoderOptions& e, const DecoderOptions& d = DecoderOptions(), int workGroupSize = 8) {
    const fecl_trellis t = e.trellis_.table();
    const fecl_conv_options o = options(d);
    fecl_codec_t h = nullptr;
    detail::check_status(fecl_conv_create(&t, uint32_t(e.length_), int32_t(e.termination_), &o, &h));
    attach(h);
    decoder_ = d;
    setWorkGroupSize(workGroupSize);
  }
  Convolutional(const EncoderOptions& e, int workGroupSize) : Convolutional(e, DecoderOptions(), workGroupSize) {}
  void setDecoderOptions(const DecoderOptions& d) {
    const fecl_conv_options o = options(d);
    detail::check_status(fecl_conv_set_options(handle(), &o));
    decoder_ = d;
  }
  DecoderOptions getDecoderOptions() const { return decoder_; }
  // Convolutional::puncturing, src/Convolutional.h:73 (src/detail/Convolutional.cpp:223-242).
  Permutation puncturing(const PunctureOptions& o) const {
    const auto m = detail::bytes(o.mask_), t = detail::bytes(o.tailMask_);
    return detail::puncture_list(paritySize(), [&](uint32_t* seq, uint64_t* n) {
      return fecl_conv_puncturing(handle(), m.data(), uint32_t(m.size()), t.data(), uint32_t(t.size()), seq, n);
    });
  }

 private:
  static fecl_conv_options options(const DecoderOptions& d) {
    fecl_conv_options o{};
    o.algorithm = d.algorithm_;
    o.scaling = d.scaling_;
    return o;
  }
  DecoderOptions decoder_;
};

}  // namespace fec
