// Exercises the C++ API of include/fecl_b200_fec.hpp the way a FeCl program uses
// fec::Ldpc / fec::Turbo / fec::Convolutional (the operations of test/Cpp/operations.h
// in the reference: encode then check, bad sizes throw, decode a noisy codeword,
// soDecode sizes), plus puncturing, fec::Permutation and Custom turbo scheduling.
//
//   fec_api_test cpu   construction, encode, check, option and size errors (no GPU)
//   fec_api_test gpu   the above plus decode and soDecode on the current CUDA device
//
// Prints one line per case and exits non-zero on the first failure.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <functional>
#include <random>
#include <stdexcept>
#include <string>
#include <vector>

#include "fecl_b200_fec.hpp"

namespace {

int g_failures = 0;

void expect(bool ok, const std::string& what) {
  std::printf("%s %s\n", ok ? "ok  " : "FAIL", what.c_str());
  if (!ok) ++g_failures;
}

template <class E>
void expect_throw(const std::function<void()>& f, const std::string& what) {
  bool thrown = false;
  try {
    f();
  } catch (const E&) {
    thrown = true;
  } catch (...) {
  }
  expect(thrown, what);
}

using Bits = std::vector<fec::BitField<size_t>>;

// BPSK over AWGN: L = 4*Es/N0 * y with y = +-1 + noise (bit 1 -> +1, L = ln p1/p0).
std::vector<double> noisy_llr(const Bits& code, double snr_db, uint32_t seed) {
  const double snr = std::pow(10.0, snr_db / 10.0);
  std::mt19937 gen(seed);
  std::normal_distribution<double> noise(0.0, std::sqrt(1.0 / (2.0 * snr)));
  std::vector<double> llr(code.size());
  for (size_t i = 0; i < code.size(); ++i) llr[i] = 4.0 * snr * ((size_t(code[i]) ? 1.0 : -1.0) + noise(gen));
  return llr;
}

Bits random_bits(size_t n, uint32_t seed) {
  std::mt19937 gen(seed);
  Bits b(n);
  for (auto& x : b) x = gen() & 1;
  return b;
}

void encode_check(const fec::Codec& code, const std::string& name, size_t frames) {
  Bits msg = random_bits(code.msgSize() * frames, 7);
  Bits parity;
  code.encode(msg, parity);
  expect(parity.size() == code.paritySize() * frames, name + ": encode size");
  expect(code.check(parity), name + ": encode then check");
  parity[parity.size() / 2] = size_t(parity[parity.size() / 2]) ^ 1;
  expect(!code.check(parity), name + ": check rejects a flipped bit");
  Bits ones(code.msgSize(), 1);
  expect(code.check(code.encode(ones)), name + ": all-ones message encodes to a codeword");
  expect_throw<std::invalid_argument>([&] { Bits m(code.msgSize() + 1), p; code.encode(m, p); },
                                      name + ": encode with a bad message size throws");
  expect_throw<std::invalid_argument>([&] { Bits p(code.paritySize() + 1); code.check(p); },
                                      name + ": check with a bad parity size throws");
}

void decode_ops(const fec::Codec& code, const std::string& name, double snr_db, size_t frames) {
  Bits msg = random_bits(code.msgSize() * frames, 11);
  Bits parity = code.encode(msg);
  std::vector<double> llr = noisy_llr(parity, snr_db, 3);
  Bits out;
  code.decode(llr, out);
  size_t errors = 0;
  for (size_t i = 0; i < msg.size(); ++i) errors += size_t(msg[i]) != size_t(out[i]);
  expect(out.size() == msg.size() && errors == 0, name + ": decode at " + std::to_string(snr_db) + " dB (" +
                                                      std::to_string(errors) + " bit errors)");
  expect_throw<std::invalid_argument>([&] { std::vector<double> l(code.paritySize() + 1); code.decode(l); },
                                      name + ": decode with a bad parity size throws");

  // soDecode: the sign of the a-posteriori message L-values gives the same bits.
  std::vector<double> app, ext, state;
  code.soDecode(fec::Codec::Input<>().parity(llr), fec::Codec::Output<>().msg(app).parity(ext).state(state));
  size_t differ = 0;
  for (size_t i = 0; i < out.size(); ++i) differ += size_t(out[i]) != size_t(app[i] >= 0.0 ? 1 : 0) ? 1 : 0;
  expect(app.size() == code.msgSize() * frames && ext.size() == code.paritySize() * frames &&
             state.size() == code.stateSize() * frames,
         name + ": soDecode output sizes");
  expect(differ <= frames, name + ": soDecode msg signs agree with decode (" + std::to_string(differ) + " ties)");
  expect_throw<std::invalid_argument>(
      [&] { std::vector<double> m; code.soDecode(fec::Codec::Input<>(), fec::Codec::Output<>().msg(m)); },
      name + ": soDecode without parity throws");
  expect_throw<std::invalid_argument>(
      [&] {
        std::vector<double> s(code.stateSize() * frames + 1), m;
        code.soDecode(fec::Codec::Input<>().parity(llr).state(s), fec::Codec::Output<>().msg(m));
      },
      name + ": soDecode with a bad state size throws");
}

// Every index of [0, size) at most once; all of them when `all`.
bool distinct_indices(const fec::Permutation& p, size_t size, bool all) {
  std::vector<int> seen(size, 0);
  for (size_t i = 0; i < p.outputSize(); ++i) {
    if (p[i] >= size || seen[p[i]]++) return false;
  }
  return !all || p.outputSize() == size;
}

void permutation_ops() {
  fec::Permutation p(std::vector<size_t>{2, 0, 3}, 4);
  const std::vector<int> in{10, 11, 12, 13, 20, 21, 22, 23};
  const auto out = p.permute(in);
  expect(out == std::vector<int>({12, 10, 13, 22, 20, 23}), "Permutation::permute over two blocks");
  expect(p.dePermute(out) == std::vector<int>({10, 0, 12, 13, 20, 0, 22, 23}),
         "Permutation::dePermute scatters back, zeros where nothing maps");
  fec::Permutation rep(std::vector<size_t>{1, 1, 0}, 2);
  expect(rep.dePermute(std::vector<int>{5, 6, 7}) == std::vector<int>({7, 6}),
         "Permutation::dePermute: a repeated index keeps the last value");
  expect(fec::Permutation(std::vector<size_t>{4, 1}).inputSize() == 5, "Permutation input size from its largest index");
}

}  // namespace

int main(int argc, char** argv) {
  const bool gpu = argc > 1 && std::strcmp(argv[1], "gpu") == 0;
  try {
    // LDPC: DVB-S2 short 1/2 and a Gallager (wc=3, wr=6) code.
    auto H = fec::Ldpc::DvbS2::matrix(16200, 1.0 / 2.0);
    // the short frame's nominal rate 1/2 carries 7200 information bits (ETSI EN 302 307, Table 5b)
    expect(H.rows() == 9000 && H.cols() == 16200, "DvbS2::matrix(16200, 1/2) shape");
    fec::Ldpc s2(fec::Ldpc::EncoderOptions(H),
                 fec::Ldpc::DecoderOptions().algorithm(fec::Approximate).iterations(30).scalingFactor(0.75));
    expect(s2.msgSize() == 7200 && s2.paritySize() == 16200, "DVB-S2 short sizes");
    encode_check(s2, "dvbs2 16200 1/2", 3);
    auto G = fec::Ldpc::Gallager::matrix(1024, 3, 6, 5);
    fec::Ldpc gal(fec::Ldpc::EncoderOptions(G), fec::Ldpc::DecoderOptions().algorithm(fec::Exact).iterations(20));
    encode_check(gal, "gallager 1024 (3,6)", 4);
    expect_throw<std::invalid_argument>([&] { fec::Ldpc::DvbS2::matrix(16200, 0.123); },
                                        "DvbS2::matrix with an unknown rate throws");
    expect_throw<std::invalid_argument>(
        [&] { s2.setDecoderOptions(fec::Ldpc::DecoderOptions().iterations(10).scalingFactor({{0, {1.0, 0.5}}})); },
        "LDPC scaling table of the wrong length throws");

    // Turbo: the LTE code built from its parts (RSC 13/15 octal, identity + QPP interleaver).
    fec::Trellis rsc({4}, {{015}}, {013});
    expect(rsc.stateCount() == 8 && rsc.inputCount() == 2 && rsc.outputSize() == 1, "LTE RSC trellis shape");
    for (size_t K : {40, 1024, 6144}) {
      auto pi = fec::Turbo::Lte3Gpp::interleaver(K);
      std::vector<size_t> id(K);
      for (size_t i = 0; i < K; ++i) id[i] = i;
      fec::Turbo lte(fec::Turbo::EncoderOptions(rsc, {fec::Permutation(id), pi}).termination(fec::Trellis::Tail),
                     fec::Turbo::DecoderOptions().algorithm(fec::Approximate).iterations(6));
      expect(lte.msgSize() == K && lte.paritySize() == 3 * K + 12, "LTE K=" + std::to_string(K) + " sizes");
      encode_check(lte, "lte K=" + std::to_string(K), 2);
      if (gpu) decode_ops(lte, "lte K=" + std::to_string(K), K < 100 ? 4.5 : 2.5, 8);
    }
    expect_throw<std::invalid_argument>([&] { fec::Turbo::Lte3Gpp::interleaver(41); },
                                        "Lte3Gpp::interleaver with a non-LTE size throws");

    permutation_ops();

    // Puncturing (Codec::puncturing): index lists of paritySize() inputs.
    {
      auto all = s2.puncturing(fec::Ldpc::PunctureOptions());
      expect(all.inputSize() == s2.paritySize() && distinct_indices(all, s2.paritySize(), true),
             "Ldpc::puncturing with no mask keeps every bit");
      auto half = s2.puncturing(fec::Ldpc::PunctureOptions().mask({true, false}));
      expect(half.outputSize() == s2.paritySize() / 2 && distinct_indices(half, s2.paritySize(), false),
             "Ldpc::puncturing with mask {1,0} keeps every other bit");
      const size_t K = 1024;
      std::vector<size_t> id(K);
      for (size_t i = 0; i < K; ++i) id[i] = i;
      fec::Turbo lte(fec::Turbo::EncoderOptions(rsc, {fec::Permutation(id), fec::Turbo::Lte3Gpp::interleaver(K)}),
                     fec::Turbo::DecoderOptions().algorithm(fec::Approximate).iterations(6));
      auto group = lte.puncturing(fec::Turbo::PunctureOptions().bitOrdering(fec::Turbo::Group));
      bool identity = group.outputSize() == lte.paritySize();
      for (size_t i = 0; identity && i < group.outputSize(); ++i) identity = group[i] == i;
      expect(identity, "Turbo::puncturing, Group order with no mask is the identity");
      auto alt = lte.puncturing(fec::Turbo::PunctureOptions());
      expect(distinct_indices(alt, lte.paritySize(), true), "Turbo::puncturing, Alternate order is a permutation");
      auto r12 = lte.puncturing(fec::Turbo::PunctureOptions().mask({{true}, {true, false}, {false, true}}));
      expect(r12.outputSize() > 2 * K && r12.outputSize() < 2 * K + 12 && distinct_indices(r12, lte.paritySize(), false),
             "Turbo::puncturing to rate 1/2 keeps 2K bits plus part of the tails");
      expect_throw<std::invalid_argument>([&] { lte.puncturing(fec::Turbo::PunctureOptions().mask({{true}, {true}})); },
                                          "Turbo::puncturing with a wrong mask count throws");
      // the punctured stream goes back to full length with zeros (erasures) at punctured bits
      std::vector<double> tx(r12.outputSize(), 1.0);
      auto rx = r12.dePermute(tx);
      size_t zeros = 0;
      for (double v : rx) zeros += v == 0.0;
      expect(rx.size() == lte.paritySize() && zeros == lte.paritySize() - r12.outputSize(),
             "dePermute of a punctured frame leaves erasures");
    }

    // Convolutional: the (171, 133) code and the LTE RSC, Tail and Truncate.
    fec::Convolutional cc(fec::Convolutional::EncoderOptions(fec::Trellis({7}, {{0171, 0133}}), 1000)
                              .termination(fec::Trellis::Tail));
    expect(cc.msgSize() == 1000 && cc.paritySize() == 2 * (1000 + 6), "Convolutional (171,133) Tail sizes");
    encode_check(cc, "conv (171,133) tail", 3);
    fec::Convolutional c75(fec::Convolutional::EncoderOptions(fec::Trellis({3}, {{07, 05}}), 512),
                           fec::Convolutional::DecoderOptions().algorithm(fec::Linear).scalingFactor(0.9));
    expect(c75.paritySize() == 1024 && c75.getDecoderOptions().scalingFactor() == 0.9,
           "Convolutional (7,5) Truncate sizes and options");
    encode_check(c75, "conv (7,5) truncate", 3);
    auto cp = cc.puncturing(fec::Convolutional::PunctureOptions().mask({true, true, true, false}));
    expect(cp.outputSize() == (cc.paritySize() * 3) / 4 && distinct_indices(cp, cc.paritySize(), false),
           "Convolutional::puncturing to rate 2/3");

    // Custom turbo scheduling: the serial order written as two stages.
    fec::Turbo::Scheduling serial(2);
    serial[0].activation = {0};
    serial[0].transfer = {{1}};
    serial[1].activation = {1};
    serial[1].transfer = {{0}};
    fec::Turbo custom(fec::Turbo::EncoderOptions(rsc, {fec::Permutation(std::vector<size_t>{}),
                                                      fec::Turbo::Lte3Gpp::interleaver(1024)}),
                      fec::Turbo::DecoderOptions().algorithm(fec::Approximate).iterations(6).scheduling(serial));
    expect(custom.getDecoderOptions().schedulingType() == fec::Custom &&
               custom.getDecoderOptions().scheduling().size() == 2,
           "Turbo DecoderOptions::scheduling(stages) selects Custom");
    fec::Turbo::Scheduling bad(1);
    bad[0].activation = {0, 1};
    bad[0].transfer = {{1}};
    expect_throw<std::invalid_argument>(
        [&] { custom.setDecoderOptions(fec::Turbo::DecoderOptions().scheduling(bad)); },
        "Custom schedule with activation and transfer of different sizes throws");
    if (gpu) {
      decode_ops(custom, "lte K=1024 custom schedule", 2.5, 8);
      decode_ops(cc, "conv (171,133) tail", 4.0, 6);
      c75.setDecoderOptions(fec::Convolutional::DecoderOptions().algorithm(fec::Approximate));
      decode_ops(c75, "conv (7,5) truncate", 6.0, 6);
    }

    if (gpu) {
      decode_ops(s2, "dvbs2 16200 1/2", 2.5, 4);
      gal.setDecoderOptions(fec::Ldpc::DecoderOptions().algorithm(fec::Linear).iterations(30));
      decode_ops(gal, "gallager 1024 (3,6)", 3.5, 8);
    }
  } catch (const std::exception& e) {
    std::printf("FAIL uncaught exception: %s\n", e.what());
    return 2;
  }
  std::printf("%d failure(s)\n", g_failures);
  return g_failures ? 1 : 0;
}
