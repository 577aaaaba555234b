// Puncturing patterns: the code-bit indices a punctured transmission keeps, as the
// reference's Codec::puncturing returns them in a fec::Permutation
// (src/Permutation.h; input size = paritySize).  A transmitter gathers the kept bits
// (Permutation::permute); a receiver scatters the received L-values back and leaves
// zeros (erasures) elsewhere (Permutation::dePermute).
#pragma once

#include <cstdint>
#include <vector>

#include "codes.hpp"

namespace fecl {

// Ldpc::Structure::puncturing, src/detail/Ldpc.cpp:333-353.  The reference advances
// its output index only for kept systematic bits; the indices returned here follow it.
std::vector<uint32_t> ldpc_puncturing(const LdpcCode& code, const std::vector<uint8_t>& mask,
                                      const std::vector<uint8_t>& syst_mask);

// Turbo::Structure::puncturing, src/detail/Turbo.cpp:200-320.  mask: empty or one mask
// per stream (systematic, then each constituent's parity); tail_mask: empty or two per
// constituent (systematic tail, parity tail); ordering 0 = Alternate, 1 = Group.
std::vector<uint32_t> turbo_puncturing(const TurboCode& code, std::vector<std::vector<uint8_t>> mask,
                                       std::vector<std::vector<uint8_t>> tail_mask, int ordering);

// Convolutional::Structure::puncturing, src/detail/Convolutional.cpp:223-242 (the tail
// bits follow the mask from its start, or the tail mask at their absolute index).
std::vector<uint32_t> conv_puncturing(const ConvCode& code, const std::vector<uint8_t>& mask,
                                      const std::vector<uint8_t>& tail_mask);

}  // namespace fecl
