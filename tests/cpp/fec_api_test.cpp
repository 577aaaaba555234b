// Exercises the C++ API of include/fecl_b200_fec.hpp the way a FeCl program uses
// fec::Ldpc / fec::Turbo (the operations of test/Cpp/operations.h in the reference:
// encode then check, bad sizes throw, decode a noisy codeword, soDecode sizes).
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
