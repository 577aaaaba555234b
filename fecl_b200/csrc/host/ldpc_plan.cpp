#include "ldpc_plan.hpp"

#include <algorithm>
#include <stdexcept>

namespace fecl {

namespace {

// Split points of a non-decreasing prefix sum `acc` ([n+1] entries) into `parts`
// blocks of about equal weight.
std::vector<uint32_t> balanced_split(const std::vector<uint64_t>& acc, uint32_t parts) {
  const uint32_t n = uint32_t(acc.size() - 1);
  std::vector<uint32_t> split(parts + 1, 0);
  split[parts] = n;
  for (uint32_t r = 1; r < parts; ++r) {
    const uint64_t target = acc[n] * r / parts;
    split[r] = uint32_t(std::lower_bound(acc.begin(), acc.end(), target) - acc.begin());
    split[r] = std::max(split[r], split[r - 1]);
  }
  return split;
}

uint32_t owner_of(const std::vector<uint32_t>& split, uint32_t i) {
  return uint32_t(std::upper_bound(split.begin(), split.end(), i) - split.begin()) - 1;
}

}  // namespace

LdpcClusterPlan build_ldpc_cluster_plan(const Csr& H, uint32_t cluster) {
  if (cluster == 0 || cluster > 16) throw std::invalid_argument("cluster size must be 1..16");
  LdpcClusterPlan p;
  p.cluster = cluster;
  const uint32_t M = H.rows, N = H.cols;
  const uint64_t E = H.nnz();

  std::vector<uint64_t> row_acc(M + 1);
  for (uint32_t r = 0; r <= M; ++r) row_acc[r] = H.row_ptr[r];
  p.row_split = balanced_split(row_acc, cluster);

  std::vector<uint32_t> deg(N, 0);
  for (uint32_t c : H.col_idx) deg[c]++;
  std::vector<uint64_t> bit_acc(N + 1, 0);
  for (uint32_t b = 0; b < N; ++b) bit_acc[b + 1] = bit_acc[b] + deg[b] + 1;  // +1: per-bit work
  p.bit_split = balanced_split(bit_acc, cluster);

  for (uint32_t r = 0; r < cluster; ++r) {
    p.max_edges = std::max<uint64_t>(p.max_edges, H.row_ptr[p.row_split[r + 1]] - H.row_ptr[p.row_split[r]]);
    p.max_bits = std::max<uint64_t>(p.max_bits, p.bit_split[r + 1] - p.bit_split[r]);
  }
  if (p.max_edges >= (1u << 28) || p.max_bits >= (1u << 28)) throw std::invalid_argument("LDPC code too large for the cluster decoder");

  // CSR order: where each edge's bit lives.
  p.chk_addr.resize(E);
  std::vector<uint32_t> bit_owner(N);
  for (uint32_t b = 0; b < N; ++b) bit_owner[b] = owner_of(p.bit_split, b);
  for (uint64_t e = 0; e < E; ++e) {
    const uint32_t b = H.col_idx[e], o = bit_owner[b];
    p.chk_addr[e] = (o << 28) | (b - p.bit_split[o]);
  }

  // Bit-major order (increasing edge id within a bit): where each edge's message lives.
  std::vector<uint32_t> start(N);
  uint64_t cur = 0;
  for (uint32_t b = 0; b < N; ++b) {
    if (deg[b] >= 64) throw std::invalid_argument("bit degree too large for the cluster decoder");
    cur = (cur + 3) & ~uint64_t(3);
    start[b] = uint32_t(cur);
    cur += deg[b];
  }
  if (cur >= (1u << 26)) throw std::invalid_argument("LDPC code too large for the cluster decoder");
  p.bit_addr.assign(size_t((cur + 3) & ~uint64_t(3)), 0);
  p.bit_ptr.resize(N);
  for (uint32_t b = 0; b < N; ++b) p.bit_ptr[b] = start[b] | (deg[b] << 26);
  std::vector<uint32_t> fill(start);
  uint32_t o = 0;
  for (uint32_t r = 0; r < M; ++r) {
    while (o + 1 < cluster && r >= p.row_split[o + 1]) ++o;
    const uint32_t e_lo = H.row_ptr[p.row_split[o]];
    for (uint32_t e = H.row_ptr[r]; e < H.row_ptr[r + 1]; ++e) p.bit_addr[fill[H.col_idx[e]]++] = (o << 28) | (e - e_lo);
  }
  return p;
}

}  // namespace fecl
