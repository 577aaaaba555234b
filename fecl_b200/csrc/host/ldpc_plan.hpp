// Partition of an LDPC check matrix over the CTAs of a thread-block cluster, and
// the packed edge-address tables the cluster-resident decoder (ldpc_cluster.cu)
// walks.
#pragma once

#include <cstdint>
#include <vector>

#include "codes.hpp"

namespace fecl {

struct LdpcClusterPlan {
  uint32_t cluster = 1;
  std::vector<uint32_t> row_split;  // [cluster+1], rows of rank r: [row_split[r], row_split[r+1])
  std::vector<uint32_t> bit_split;  // [cluster+1]
  std::vector<uint32_t> chk_addr;   // [E] in CSR order: (owner rank of the bit << 28) | bit offset there
  std::vector<uint32_t> bit_ptr;    // [N] start (multiple of 4) | degree << 26
  std::vector<uint32_t> bit_addr;   // bit-major, padded: (owner rank of the edge << 28) | edge offset there
  uint64_t max_edges = 0;           // largest number of edges owned by one rank
  uint64_t max_bits = 0;            // largest number of bits owned by one rank
};

// Splits rows so that every rank owns about E / cluster edges, and bits so that every
// rank owns about E / cluster bit-node edges.  Throws std::invalid_argument when the
// matrix does not fit the packing (degree >= 64 on a bit, more than 2^26 padded
// bit-major entries, offsets of 2^28 or more).
LdpcClusterPlan build_ldpc_cluster_plan(const Csr& H, uint32_t cluster);

}  // namespace fecl
