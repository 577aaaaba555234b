#include "puncture.hpp"

#include <stdexcept>

namespace fecl {

namespace {

// Entry i of a repeating mask (an empty mask keeps everything).
bool keep(const std::vector<uint8_t>& m, size_t i) { return m.empty() || m[i % m.size()] != 0; }

}  // namespace

std::vector<uint32_t> ldpc_puncturing(const LdpcCode& code, const std::vector<uint8_t>& mask,
                                      const std::vector<uint8_t>& syst_mask) {
  std::vector<uint32_t> seq;
  const size_t syst = code.syst_size(), parity = code.parity_size();
  const bool by_syst = !syst_mask.empty();
  uint32_t at = 0;  // next output index; moves only when a systematic bit is kept
  for (size_t i = 0; i < syst; ++i) {
    const bool k = by_syst ? keep(syst_mask, at) : keep(mask, i);
    if (k) seq.push_back(at++);
  }
  for (size_t i = 0; i < parity - syst; ++i, ++at) {
    const bool k = by_syst ? keep(mask, at) : keep(mask, i);
    if (k) seq.push_back(at);
  }
  return seq;
}

std::vector<uint32_t> turbo_puncturing(const TurboCode& code, std::vector<std::vector<uint8_t>> mask,
                                       std::vector<std::vector<uint8_t>> tail_mask, int ordering) {
  const auto& cs = code.constituents();
  const size_t C = cs.size();
  if (mask.empty()) {
    mask.assign(C + 1, {1});
  } else if (mask.size() == C + 1) {
    for (auto& m : mask)
      if (m.empty()) m = {1};
  } else {
    throw std::invalid_argument("Invalid size for parity mask");
  }
  if (tail_mask.empty()) tail_mask.assign(2 * C, {});
  else if (tail_mask.size() != 2 * C) throw std::invalid_argument("Invalid size for tail mask");
  // a tail bit follows its own tail mask when one is given, else the stream's mask
  auto tail_keep = [&](size_t tm, size_t tail_i, size_t m, size_t stream_i) {
    return tail_mask[tm].empty() ? keep(mask[m], stream_i) : keep(tail_mask[tm], tail_i);
  };
  std::vector<uint32_t> seq;
  if (ordering == 0) {  // Alternate: per message step, its systematic bit then each constituent's parity bits
    size_t s = 0;
    for (size_t i = 0; i < code.msg_size(); ++i, ++s) {
      if (keep(mask[0], s)) seq.push_back(uint32_t(s));
      size_t base = code.syst_size();
      for (size_t j = 0; j < C; ++j) {
        const size_t out = cs[j].trellis.output_size;
        if (i < cs[j].length)
          for (size_t k = 0; k < out; ++k)
            if (keep(mask[j + 1], i * out + k)) seq.push_back(uint32_t(base + i * out + k));
        base += cs[j].parity_size();
      }
    }
    size_t p = code.syst_size();
    for (size_t i = 0; i < C; ++i) {
      const size_t in = cs[i].trellis.input_size, out = cs[i].trellis.output_size;
      p += cs[i].parity_size() - cs[i].tail * out;
      size_t ts = 0, tp = 0;
      for (size_t j = 0; j < cs[i].tail; ++j) {
        for (size_t k = 0; k < in; ++k, ++s, ++ts)
          if (tail_keep(2 * i, ts, 0, s)) seq.push_back(uint32_t(s));
        for (size_t k = 0; k < out; ++k, ++p, ++tp)
          if (tail_keep(2 * i + 1, tp, i + 1, p)) seq.push_back(uint32_t(p));
      }
    }
  } else if (ordering == 1) {  // Group: message, systematic tails, then each constituent's parity and tail
    size_t at = 0;
    for (size_t i = 0; i < code.msg_size(); ++i, ++at)
      if (keep(mask[0], at)) seq.push_back(uint32_t(at));
    for (size_t i = 0; i < C; ++i) {
      const size_t n = cs[i].tail * cs[i].trellis.input_size;
      for (size_t t = 0; t < n; ++t, ++at)
        if (tail_keep(2 * i, t, 0, at)) seq.push_back(uint32_t(at));
    }
    for (size_t i = 0; i < C; ++i) {
      const size_t out = cs[i].trellis.output_size;
      size_t pi = 0;
      for (size_t t = 0; t < cs[i].length * out; ++t, ++pi, ++at)
        if (keep(mask[i + 1], pi)) seq.push_back(uint32_t(at));
      for (size_t t = 0; t < cs[i].tail * out; ++t, ++pi, ++at)
        if (tail_keep(2 * i + 1, t, i + 1, pi)) seq.push_back(uint32_t(at));
    }
  }
  return seq;
}

std::vector<uint32_t> conv_puncturing(const ConvCode& code, const std::vector<uint8_t>& mask,
                                      const std::vector<uint8_t>& tail_mask) {
  const Constituent& c = code.constituent();
  const size_t out = c.trellis.output_size;
  std::vector<uint32_t> seq;
  size_t at = 0;
  for (size_t i = 0; i < size_t(c.length) * out; ++i, ++at)
    if (keep(mask, i)) seq.push_back(uint32_t(at));
  for (size_t i = 0; i < size_t(c.tail) * out; ++i, ++at)
    if (tail_mask.empty() ? keep(mask, i) : keep(tail_mask, at)) seq.push_back(uint32_t(at));
  return seq;
}

}  // namespace fecl
