// Host-side code construction.  See codes.hpp for the reference structures each
// piece restates; the step-by-step notes below cite the reference lines whose
// behaviour must be reproduced exactly (matrix transform order, draw order of the
// Gallager generator, greedy tail choice), because they fix the codeword layout,
// the soft-state layout and the encoded bits.
#include "codes.hpp"

#include <algorithm>
#include <random>

#include "../tables/dvbs2_tables.h"
#include "../tables/lte_qpp_table.h"

namespace fecl {

namespace {

inline int popcount64(uint64_t x) { return __builtin_popcountll(x); }
inline bool parity64(uint64_t x) { return __builtin_parityll(x); }

bool row_has(const std::vector<uint32_t>& row, uint32_t c) { return std::binary_search(row.begin(), row.end(), c); }

// Swap membership of columns a and b in one sorted row.
void row_swap_cols(std::vector<uint32_t>& row, uint32_t a, uint32_t b) {
  bool ha = row_has(row, a), hb = row_has(row, b);
  if (ha == hb) return;
  uint32_t from = ha ? a : b, to = ha ? b : a;
  row.erase(std::lower_bound(row.begin(), row.end(), from));
  row.insert(std::lower_bound(row.begin(), row.end(), to), to);
}

// Move column a to position b, shifting the columns in between by one (the
// semantics of SparseBitMatrix/BitMatrix::moveCol, src/BitMatrix.h RowRef::move).
uint32_t moved_index(uint32_t c, uint32_t a, uint32_t b) {
  if (c == a) return b;
  if (a > b && c >= b && c < a) return c + 1;
  if (a < b && c > a && c <= b) return c - 1;
  return c;
}
void row_move_col(std::vector<uint32_t>& row, uint32_t a, uint32_t b) {
  for (auto& c : row) c = moved_index(c, a, b);
  std::sort(row.begin(), row.end());
}

// A dense bit row for the small elimination block.
struct DenseRow {
  std::vector<uint64_t> w;
  explicit DenseRow(uint32_t cols = 0) : w((cols + 63) / 64, 0) {}
  bool test(uint64_t c) const { return c / 64 < w.size() && ((w[c / 64] >> (c % 64)) & 1); }
  void set(uint32_t c, bool v) {
    if (v) w[c / 64] |= (uint64_t(1) << (c % 64));
    else w[c / 64] &= ~(uint64_t(1) << (c % 64));
  }
  void flip(uint32_t c) { w[c / 64] ^= (uint64_t(1) << (c % 64)); }
  void xor_with(const DenseRow& o) {
    for (size_t i = 0; i < w.size(); ++i) w[i] ^= o.w[i];
  }
  int64_t first() const {
    for (size_t i = 0; i < w.size(); ++i)
      if (w[i]) return int64_t(i * 64 + __builtin_ctzll(w[i]));
    return -1;
  }
  void swap_cols(uint32_t a, uint32_t b) {
    bool va = test(a), vb = test(b);
    set(a, vb);
    set(b, va);
  }
  void move_col(uint32_t a, uint32_t b, uint32_t cols) {
    DenseRow out(cols);
    for (uint32_t c = 0; c < cols; ++c)
      if (test(c)) out.set(moved_index(c, a, b), true);
    w.swap(out.w);
  }
};

Csr sub_matrix(const std::vector<std::vector<uint32_t>>& rows, uint32_t r0, uint32_t r1, uint32_t c0, uint32_t c1) {
  std::vector<std::vector<uint32_t>> out;
  for (uint32_t r = r0; r < r1; ++r) {
    std::vector<uint32_t> row;
    for (auto c : rows[r])
      if (c >= c0 && c < c1) row.push_back(c - c0);
    out.push_back(row);
  }
  return Csr::from_rows(c1 - c0, out);
}

}  // namespace

Csr Csr::from_rows(uint32_t cols, const std::vector<std::vector<uint32_t>>& rows) {
  Csr m;
  m.rows = uint32_t(rows.size());
  m.cols = cols;
  m.row_ptr.assign(1, 0);
  for (auto& r : rows) {
    m.col_idx.insert(m.col_idx.end(), r.begin(), r.end());
    m.row_ptr.push_back(uint32_t(m.col_idx.size()));
  }
  return m;
}

Csr Csr::transpose() const {
  std::vector<std::vector<uint32_t>> t(cols);
  for (uint32_t r = 0; r < rows; ++r)
    for (uint32_t e = row_ptr[r]; e < row_ptr[r + 1]; ++e) t[col_idx[e]].push_back(r);
  return from_rows(rows, t);
}

// ---------------------------------------------------------------- LDPC

LdpcCode::LdpcCode(const Csr& H) {
  if (H.rows == 0 || H.cols <= H.rows) throw std::invalid_argument("Invalid size for check matrix");
  for (uint32_t r = 0; r < H.rows; ++r) {
    for (uint32_t e = H.row_ptr[r]; e < H.row_ptr[r + 1]; ++e) {
      if (H.col_idx[e] >= H.cols) throw std::invalid_argument("Invalid column index in check matrix");
      if (e > H.row_ptr[r] && H.col_idx[e] <= H.col_idx[e - 1])
        throw std::invalid_argument("Check matrix rows must hold strictly increasing column indices");
    }
    if (H.degree(r) < 2) throw std::invalid_argument("Check matrix rows need at least two ones");
  }
  msg_size_ = H.cols - H.rows;  // src/detail/Ldpc.cpp:48
  compute_generator(H);
  for (uint32_t r = 0; r < H_.rows; ++r) max_degree_ = std::max(max_degree_, H_.degree(r));
  LdpcDecoderConfig cfg;
  set_decoder(cfg);
}

// The encoder transform of src/detail/Ldpc.cpp:216-331.  It brings H to an
// approximate lower-triangular form [A B T; C D E] by repeatedly retiring the
// lowest-weight column from the right together with the rows that hold it, then
// eliminates the gap block densely.  Rows are reordered and columns may be
// permuted; the decoder and the soft state use the resulting matrix.
void LdpcCode::compute_generator(Csr Hin) {
  const uint32_t N = Hin.cols;
  const uint32_t R = Hin.rows;
  std::vector<std::vector<uint32_t>> rows(R);
  for (uint32_t r = 0; r < R; ++r) rows[r].assign(Hin.col_idx.begin() + Hin.row_ptr[r], Hin.col_idx.begin() + Hin.row_ptr[r + 1]);

  // Column weights over the still-active rows [0, active).
  std::vector<uint64_t> weight(N, 0);
  for (auto& row : rows)
    for (auto c : row) weight[c]++;
  // The rows holding each column, by row identity, and each row's position, so that
  // retiring a column visits only the rows that hold it.
  std::vector<std::vector<uint32_t>> col_rows(N);
  for (uint32_t r = 0; r < R; ++r)
    for (auto c : rows[r]) col_rows[c].push_back(r);
  std::vector<uint32_t> row_id(R), row_pos(R);
  for (uint32_t r = 0; r < R; ++r) row_id[r] = row_pos[r] = r;
  std::vector<uint32_t> holding;
  uint64_t active = R;
  int64_t retired_cursor = int64_t(R) - 1;
  uint64_t t = 0;
  for (uint64_t i = N; i > 0; --i) {
    for (; retired_cursor >= int64_t(active); --retired_cursor)
      for (auto c : rows[retired_cursor]) weight[c]--;
    // Lowest non-zero weight among columns [0, i), scanning right to left; weight 1 wins at once.
    uint64_t best = uint64_t(-1);
    uint64_t best_idx = 0;
    for (int64_t j = int64_t(i) - 1; j >= 0; --j) {
      if (weight[j] == 1) {
        best_idx = uint64_t(j);
        best = 1;
        break;
      } else if (weight[j] < best && weight[j] >= 1) {
        best_idx = uint64_t(j);
        best = weight[j];
      }
    }
    if (best_idx != i - 1) {
      for (auto& row : rows) row_swap_cols(row, uint32_t(best_idx), uint32_t(i - 1));
      std::swap(col_rows[best_idx], col_rows[i - 1]);
    }
    std::swap(weight[best_idx], weight[i - 1]);
    // Active rows holding column i-1 go to the end of the active block, as the
    // reference's scan moves them: positions are visited in increasing order, and a
    // row holding the column is swapped with the last active row, whose replacement
    // at that position is examined next.  `holding` lists, in increasing order, the
    // active positions whose row holds the column; its front is the scan's next stop,
    // and the swapped-in row holds the column exactly when its position is the back.
    holding.clear();
    for (uint32_t rid : col_rows[i - 1])
      if (row_pos[rid] < active) holding.push_back(row_pos[rid]);
    std::sort(holding.begin(), holding.end());
    uint64_t end = active;
    size_t lo = 0, hi = holding.size();
    while (lo < hi) {
      const uint32_t r = holding[lo];
      --end;
      const bool end_holds = holding[hi - 1] == end;
      if (end != r) {
        std::swap(rows[end], rows[r]);
        std::swap(row_id[end], row_id[r]);
        row_pos[row_id[end]] = uint32_t(end);
        row_pos[row_id[r]] = r;
      }
      if (end_holds && end != r) --hi;  // position r now holds the row from the end
      else ++lo;
    }
    active -= std::max<uint64_t>(best, 1);
    if (active == 0) {
      t = N - i + 1;
      break;
    }
  }

  // Put a one on the diagonal of the T block, row by row.
  for (uint64_t i = 0; i < t; ++i) {
    uint32_t c = uint32_t(i + N - t);
    if (!row_has(rows[i], c)) {
      for (uint64_t r = i + 1; r < R; ++r) {
        if (row_has(rows[r], c)) {
          std::swap(rows[i], rows[r]);
          break;
        }
      }
    }
  }

  // Dense copy of the remaining rows, with the T columns eliminated.
  std::vector<DenseRow> cde;
  for (uint64_t r = t; r < R; ++r) {
    DenseRow d(N);
    for (auto c : rows[r]) d.set(c, true);
    cde.push_back(d);
  }
  for (int64_t i = int64_t(t) - 1; i >= 0; --i) {
    uint32_t c = uint32_t(i + N - t);
    for (auto& d : cde)
      if (d.test(c))
        for (auto x : rows[i]) d.flip(x);
  }

  // Forward elimination of the gap block; dependent rows grow the message.
  uint64_t msg = msg_size_;
  for (int64_t i = 0; i < int64_t(N - t - msg); ++i) {
    bool found = false;
    for (size_t r = size_t(i); r < cde.size(); ++r) {
      if (cde[r].test(uint64_t(i) + msg)) {
        std::swap(cde[r], cde[i]);
        found = true;
        break;
      }
    }
    if (!found) {
      for (size_t r = size_t(i); r < cde.size(); ++r) {
        int64_t k = cde[r].first();
        if (k != -1) {
          uint32_t a = uint32_t(k), b = uint32_t(uint64_t(i) + msg);
          if (a != b) {
            for (auto& row : rows) row_swap_cols(row, a, b);
            for (auto& d : cde) d.swap_cols(a, b);
          }
          std::swap(cde[r], cde[i]);
          found = true;
          break;
        }
      }
    }
    if (!found) {
      uint32_t a = uint32_t(uint64_t(i) + msg), b = uint32_t(msg);
      for (auto& row : rows) row_move_col(row, a, b);
      for (auto& d : cde) d.move_col(a, b, N);
      ++msg;
      --i;
      continue;
    }
    for (size_t r = size_t(i) + 1; r < cde.size(); ++r)
      if (cde[r].test(uint64_t(i) + msg)) cde[r].xor_with(cde[i]);
  }
  // Back substitution.
  for (int64_t i = int64_t(cde.size()) - 1; i >= 0; --i)
    for (int64_t r = i - 1; r >= 0; --r)
      if (cde[r].test(uint64_t(i) + msg)) cde[r].xor_with(cde[i]);

  msg_size_ = uint32_t(msg);
  H_ = Csr::from_rows(N, rows);
  const uint32_t gap = uint32_t(N - msg - t);
  std::vector<std::vector<uint32_t>> dc(gap);
  for (uint32_t r = 0; r < gap && r < cde.size(); ++r)
    for (uint32_t c = 0; c < msg; ++c)
      if (cde[r].test(c)) dc[r].push_back(c);
  DC_ = Csr::from_rows(uint32_t(msg), dc);
  A_ = sub_matrix(rows, 0, uint32_t(t), 0, uint32_t(msg));
  B_ = sub_matrix(rows, 0, uint32_t(t), uint32_t(msg), uint32_t(msg) + gap);
  T_ = sub_matrix(rows, 0, uint32_t(t), uint32_t(N - t), N).transpose();
}

void LdpcCode::set_decoder(const LdpcDecoderConfig& cfg) {
  if (cfg.algorithm < 0 || cfg.algorithm > 2) throw std::invalid_argument("Invalid decoder algorithm");
  if (cfg.precision < 0 || cfg.precision > 2) throw std::invalid_argument("Invalid message precision");
  if (cfg.scaling.empty()) throw std::invalid_argument("Wrong size for scaling factor");
  // src/detail/Ldpc.cpp:71-73,94-96: one row, or one row per iteration.
  if (cfg.scaling.size() != 1 && cfg.scaling.size() != cfg.iterations)
    throw std::invalid_argument("Wrong size for scaling factor");
  LdpcDecoderConfig c = cfg;
  for (auto& row : c.scaling) {
    if (row.size() == 1) row.assign(max_degree_ > 1 ? max_degree_ - 1 : 1, row[0]);
    if (row.size() + 1 < max_degree_) throw std::invalid_argument("Scaling factor not defined and no default");
  }
  dec_ = c;
}

double LdpcCode::scaling_factor(size_t i, size_t d) const {
  i %= dec_.scaling.size();
  return dec_.scaling[i][d - 2];
}

void LdpcCode::encode(const uint8_t* msg, uint8_t* parity) const {
  const uint32_t N = H_.cols;
  const uint32_t m = msg_size_;
  for (uint32_t i = 0; i < m; ++i) parity[i] = msg[i] & 1;
  for (uint32_t i = m; i < N; ++i) parity[i] = 0;
  uint8_t* p = parity + m;
  const uint32_t gap = DC_.rows;
  for (uint32_t r = 0; r < gap; ++r)
    for (uint32_t e = DC_.row_ptr[r]; e < DC_.row_ptr[r + 1]; ++e) p[r] ^= msg[DC_.col_idx[e]] & 1;
  for (uint32_t r = 0; r < B_.rows; ++r)
    for (uint32_t e = B_.row_ptr[r]; e < B_.row_ptr[r + 1]; ++e) p[gap + r] ^= p[B_.col_idx[e]];
  uint8_t* p2 = p + gap;
  for (uint32_t r = 0; r < A_.rows; ++r)
    for (uint32_t e = A_.row_ptr[r]; e < A_.row_ptr[r + 1]; ++e) p2[r] ^= msg[A_.col_idx[e]] & 1;
  for (uint32_t r = 0; r < T_.rows; ++r)
    for (uint32_t e = T_.row_ptr[r] + 1; e < T_.row_ptr[r + 1]; ++e) p2[T_.col_idx[e]] ^= p2[r];
}

bool LdpcCode::check(const uint8_t* parity) const {
  for (uint32_t r = 0; r < H_.rows; ++r) {
    uint8_t s = 0;
    for (uint32_t e = H_.row_ptr[r]; e < H_.row_ptr[r + 1]; ++e) s ^= parity[H_.col_idx[e]] & 1;
    if (s) return false;
  }
  return true;
}

Csr dvbs2_matrix(uint32_t n, uint32_t rate_num, uint32_t rate_den) {
  int code = -1;
  for (int i = 0; i < FECL_DVBS2_CODE_COUNT; ++i) {
    if (fecl_dvbs2_codes[i][0] == n && uint64_t(fecl_dvbs2_codes[i][1]) * rate_den == uint64_t(rate_num) * fecl_dvbs2_codes[i][2]) {
      code = i;
      break;
    }
  }
  if (code < 0) {
    bool length_ok = (n == 16200 || n == 64800);
    throw std::invalid_argument(length_ok ? "Invalid rate" : "Invalid length");
  }
  const uint32_t q = fecl_dvbs2_codes[code][3];
  const uint32_t first_row = fecl_dvbs2_codes[code][4];
  const uint32_t groups = fecl_dvbs2_codes[code][5];
  const uint32_t M = 360 * q;
  const uint32_t K = n - M;
  if (groups * 360 != K) throw std::invalid_argument("Inconsistent DVB-S2 table");
  std::vector<std::vector<uint32_t>> rows(M);
  for (uint32_t g = 0; g < groups; ++g) {
    const uint32_t off = fecl_dvbs2_rows[first_row + g][0];
    const uint32_t len = fecl_dvbs2_rows[first_row + g][1];
    for (uint32_t m = 0; m < 360; ++m) {
      const uint32_t bit = g * 360 + m;
      for (uint32_t a = 0; a < len; ++a) rows[(fecl_dvbs2_addr[off + a] + m * q) % M].push_back(bit);
    }
  }
  for (uint32_t i = 0; i < M; ++i) {
    rows[i].push_back(K + i);                  // parity bit i closes check i ...
    if (i + 1 < M) rows[i + 1].push_back(K + i);  // ... and feeds check i+1
  }
  for (auto& r : rows) std::sort(r.begin(), r.end());
  return Csr::from_rows(n, rows);
}

// src/Ldpc.cpp:77-102: wc bands of n/wr rows; band 0 holds wr consecutive columns
// per row, later bands are copies whose columns are permuted by successive swaps
// drawn from std::minstd_rand0 and std::uniform_int_distribution<int>.
Csr gallager_matrix(uint32_t n, uint32_t wc, uint32_t wr, uint64_t seed) {
  if (wr == 0 || wc == 0 || n < wr) throw std::invalid_argument("Invalid Gallager parameters");
  const uint32_t band = n / wr;
  const uint32_t R = band * wc;
  std::vector<std::vector<uint32_t>> rows(R);
  uint32_t elem = 0;
  for (uint32_t i = 0; i < band; ++i)
    for (uint32_t j = 0; j < wr; ++j) {
      for (uint32_t k = 0; k < R; k += band) rows[i + k].push_back(elem);
      ++elem;
    }
  std::minstd_rand0 gen((int)seed);
  for (uint32_t j = 0; j < n; ++j) {
    std::uniform_int_distribution<int> dist(int(j), int(n - 1));
    for (uint32_t i = band; i < R; i += band) {
      uint32_t other = uint32_t(dist(gen));
      if (other == j) continue;
      for (uint32_t r = i; r < i + band; ++r) row_swap_cols(rows[r], j, other);
    }
  }
  return Csr::from_rows(n, rows);
}

// ---------------------------------------------------------------- trellis

Trellis Trellis::from_generators(const std::vector<uint32_t>& cl, const std::vector<std::vector<uint64_t>>& gen,
                                 std::vector<uint64_t> feedback) {
  Trellis t;
  if (gen.empty()) throw std::invalid_argument("Invalid number of generators");
  t.input_size = uint32_t(gen.size());
  t.output_size = uint32_t(gen[0].size());
  if (cl.size() != gen.size()) throw std::invalid_argument("Invalid number of generators");
  if (cl.size() != feedback.size() && !feedback.empty()) throw std::invalid_argument("Invalid number of feedback");
  for (auto& g : gen)
    if (g.size() != t.output_size) throw std::invalid_argument("Invalid number of generators");
  if (feedback.empty())
    for (auto c : cl) feedback.push_back(uint64_t(1) << (c - 1));
  t.state_size = 0;
  for (auto c : cl) t.state_size += c - 1;
  if (t.state_size > 12 || t.input_size > 4 || t.output_size > 8)
    throw std::invalid_argument("Trellis too large for the device decoder");
  t.state_count = 1u << t.state_size;
  t.input_count = 1u << t.input_size;
  t.next_state.assign(t.state_count * t.input_count, 0);
  t.output.assign(t.state_count * t.input_count, 0);
  for (uint32_t s = 0; s < t.state_count; ++s) {
    for (uint32_t u = 0; u < t.input_count; ++u) {
      uint32_t next = 0, out = 0, j = 0;
      for (size_t i = 0; i < cl.size(); ++i) {
        const uint32_t regs = cl[i] - 1;
        const uint64_t st = (uint64_t(s) >> j) & ((uint64_t(1) << regs) - 1);
        const uint32_t in = (u >> i) & 1;
        const bool fb_loop = parity64(st & feedback[i]);
        for (uint32_t k = 0; k < t.output_size; ++k) {
          if ((gen[i][k] >> cl[i]) != 0) throw std::invalid_argument("Invalid connection in generator");
          const uint32_t top = uint32_t((gen[i][k] >> (cl[i] - 1)) & 1);
          const uint32_t bit = ((in ^ uint32_t(fb_loop)) & top) ^ uint32_t(parity64(st & gen[i][k]));
          out ^= bit << k;
        }
        if (((feedback[i] >> (cl[i] - 1)) & 1) != 1) throw std::invalid_argument("Feedback must connect systematic");
        const uint32_t newbit = (in & uint32_t((feedback[i] >> (cl[i] - 1)) & 1)) ^ uint32_t(fb_loop);
        next |= newbit << (j + cl[i] - 2);
        next |= uint32_t(st >> 1) << j;
        j += regs;
      }
      t.next_state[s * t.input_count + u] = next;
      t.output[s * t.input_count + u] = out;
    }
  }
  return t;
}

Trellis Trellis::from_tables(uint32_t state_count, uint32_t input_count, uint32_t output_size,
                             const uint32_t* next_state, const uint32_t* output) {
  Trellis t;
  auto log2u = [](uint32_t v) {
    uint32_t l = 0;
    while ((1u << l) < v) ++l;
    return ((1u << l) == v) ? l : 0xffffffffu;
  };
  t.state_size = log2u(state_count);
  t.input_size = log2u(input_count);
  t.output_size = output_size;
  if (t.state_size == 0xffffffffu || t.input_size == 0xffffffffu || t.state_size > 12 || t.input_size > 4 ||
      output_size > 8 || output_size == 0)
    throw std::invalid_argument("Invalid trellis tables");
  t.state_count = state_count;
  t.input_count = input_count;
  t.next_state.assign(next_state, next_state + state_count * input_count);
  t.output.assign(output, output + state_count * input_count);
  for (uint32_t i = 0; i < state_count * input_count; ++i)
    if (t.next_state[i] >= state_count || t.output[i] >= (1u << output_size))
      throw std::invalid_argument("Invalid trellis tables");
  return t;
}

Trellis lte_trellis() { return Trellis::from_generators({4}, {{015}}, {013}); }

// ---------------------------------------------------------------- turbo

void Constituent::encode(const uint8_t* msg, uint8_t* parity, uint8_t* tail_bits) const {
  const Trellis& t = trellis;
  uint32_t state = 0;
  for (uint32_t j = 0; j < length; ++j) {
    uint32_t in = 0;
    for (uint32_t k = 0; k < t.input_size; ++k) in |= uint32_t(msg[j * t.input_size + k] & 1) << k;
    const uint32_t out = t.output[state * t.input_count + in];
    state = t.next_state[state * t.input_count + in];
    for (uint32_t k = 0; k < t.output_size; ++k) parity[j * t.output_size + k] = (out >> k) & 1;
  }
  parity += length * t.output_size;
  // Greedy termination (src/detail/Convolutional.cpp:189-211): the input that
  // lowers the state's weight most, first such input on ties.
  for (uint32_t j = 0; j < tail; ++j) {
    int best_count = -1;
    uint32_t best = 0;
    for (uint32_t u = 0; u < t.input_count; ++u) {
      int count = popcount64(state) - popcount64(t.next_state[state * t.input_count + u]);
      if (count > best_count) {
        best_count = count;
        best = u;
      }
    }
    const uint32_t out = t.output[state * t.input_count + best];
    for (uint32_t k = 0; k < t.output_size; ++k) parity[k] = (out >> k) & 1;
    for (uint32_t k = 0; k < t.input_size; ++k) tail_bits[k] = (best >> k) & 1;
    parity += t.output_size;
    tail_bits += t.input_size;
    state = t.next_state[state * t.input_count + best];
  }
}

TurboCode::TurboCode(const std::vector<Trellis>& trellis, const std::vector<std::vector<uint32_t>>& perms,
                     const std::vector<int>& termination) {
  const size_t n = perms.size();
  if (n == 0) throw std::invalid_argument("Trellis and Permutation count don't match");
  if (trellis.size() != 1 && trellis.size() != n) throw std::invalid_argument("Trellis and Permutation count don't match");
  if (termination.size() != 1 && termination.size() != n)
    throw std::invalid_argument("Termination and Permutation count don't match");
  msg_size_ = 0;
  for (auto& p : perms)
    for (auto v : p) msg_size_ = std::max(msg_size_, v + 1);
  for (size_t i = 0; i < n; ++i) {
    Constituent c;
    c.perm = perms[i];
    if (c.perm.empty()) {
      c.perm.resize(msg_size_);
      for (uint32_t j = 0; j < msg_size_; ++j) c.perm[j] = j;
    }
    c.trellis = trellis[trellis.size() == 1 ? 0 : i];
    c.length = uint32_t(c.perm.size()) / c.trellis.input_size;
    if (c.length * c.trellis.input_size != c.perm.size()) throw std::invalid_argument("Invalid size for interleaver");
    c.termination = termination[termination.size() == 1 ? 0 : i];
    if (c.termination != 0 && c.termination != 1) throw std::invalid_argument("Invalid termination");
    c.tail = (c.termination == 0) ? c.trellis.state_size : 0;
    c_.push_back(c);
  }
  tail_size_ = parity_size_ = state_size_ = 0;
  for (auto& c : c_) {
    tail_size_ += c.syst_tail_size();
    parity_size_ += c.parity_size();
    state_size_ += c.syst_size();
  }
  syst_size_ = msg_size_ + tail_size_;
  parity_size_ += syst_size_;
  set_decoder(TurboDecoderConfig());
}

void TurboCode::set_decoder(const TurboDecoderConfig& cfg) {
  if (cfg.algorithm < 0 || cfg.algorithm > 2) throw std::invalid_argument("Invalid decoder algorithm");
  if (cfg.scheduling < 0 || cfg.scheduling > 2) throw std::invalid_argument("Invalid scheduling");
  TurboDecoderConfig c = cfg;
  if (c.scheduling == 2) {
    // src/detail/Turbo.cpp:106-124: activation and transfer lists of equal size, each
    // list sorted; a transfer list stays paired with the activation at its index after
    // the activation list is sorted.  Constituent ids must name a constituent (the
    // reference accepts an id equal to the count, which it then reads out of range).
    for (auto& st : c.schedule) {
      if (st.activation.size() != st.transfer.size())
        throw std::invalid_argument("Invalid scheduling : activation and transfer not the same size");
      std::sort(st.activation.begin(), st.activation.end());
      for (size_t j = 0; j < st.activation.size(); ++j) {
        if (st.activation[j] >= c_.size()) throw std::invalid_argument("Invalid scheduling : activation of an invalid constituent");
        for (auto t : st.transfer[j])
          if (t >= c_.size()) throw std::invalid_argument("Invalid scheduling : transfer from an invalid constituent");
        std::sort(st.transfer[j].begin(), st.transfer[j].end());
      }
    }
  } else {
    c.schedule.clear();
  }
  if (cfg.precision < 0 || cfg.precision > 1) throw std::invalid_argument("Invalid message precision");
  if (cfg.crc < 0 || cfg.crc > 2) throw std::invalid_argument("Invalid CRC");
  // src/detail/Turbo.cpp:127-135
  if (cfg.scaling.size() == c_.size()) {
    for (auto& r : cfg.scaling)
      if (r.size() != cfg.iterations && r.size() != 1) throw std::invalid_argument("Wrong size for scaling factor");
  } else if (cfg.scaling.size() != 1) {
    throw std::invalid_argument("Wrong size for scaling factor");
  }
  for (auto& r : cfg.scaling)
    if (r.empty()) throw std::invalid_argument("Wrong size for scaling factor");
  dec_ = c;
}

double TurboCode::scaling_factor(size_t i, size_t j) const {
  j %= dec_.scaling.size();
  i %= dec_.scaling[j].size();
  return dec_.scaling[j][i];
}

void TurboCode::encode(const uint8_t* msg, uint8_t* parity) const {
  for (uint32_t i = 0; i < msg_size_; ++i) parity[i] = msg[i] & 1;
  uint8_t* syst_tail = parity + msg_size_;
  uint8_t* out = parity + syst_size_;
  std::vector<uint8_t> inter;
  for (auto& c : c_) {
    inter.resize(c.perm.size());
    for (size_t k = 0; k < c.perm.size(); ++k) inter[k] = msg[c.perm[k]] & 1;
    c.encode(inter.data(), out, syst_tail);
    syst_tail += c.syst_tail_size();
    out += c.parity_size();
  }
}

bool TurboCode::check(const uint8_t* parity) const {
  std::vector<uint8_t> inter, par, tail;
  const uint8_t* par_in = parity + syst_size_;
  const uint8_t* tail_in = parity + msg_size_;
  for (auto& c : c_) {
    inter.resize(c.perm.size());
    par.resize(c.parity_size());
    tail.resize(c.syst_tail_size());
    for (size_t k = 0; k < c.perm.size(); ++k) inter[k] = parity[c.perm[k]] & 1;
    c.encode(inter.data(), par.data(), tail.data());
    for (size_t k = 0; k < par.size(); ++k)
      if (par[k] != (par_in[k] & 1)) return false;
    for (size_t k = 0; k < tail.size(); ++k)
      if (tail[k] != (tail_in[k] & 1)) return false;
    par_in += c.parity_size();
    tail_in += c.syst_tail_size();
  }
  return true;
}

bool TurboCode::is_lte_shape() const {
  if (c_.size() != 2) return false;
  for (auto& c : c_) {
    const Trellis& t = c.trellis;
    if (t.state_count != 8 || t.input_count != 2 || t.output_size != 1 || c.termination != 0) return false;
    if (c.length != msg_size_) return false;
  }
  for (uint32_t i = 0; i < msg_size_; ++i)
    if (c_[0].perm[i] != i) return false;
  return true;
}

bool lte_qpp_params(uint32_t K, uint32_t* f1, uint32_t* f2) {
  for (int i = 0; i < FECL_LTE_QPP_COUNT; ++i) {
    if (fecl_lte_qpp[i][0] == K) {
      *f1 = fecl_lte_qpp[i][1];
      *f2 = fecl_lte_qpp[i][2];
      return true;
    }
  }
  return false;
}

std::vector<uint32_t> lte_interleaver(uint32_t K) {
  uint32_t f1, f2;
  if (!lte_qpp_params(K, &f1, &f2)) throw std::invalid_argument("Invalid length");
  std::vector<uint32_t> p(K);
  for (uint64_t i = 0; i < K; ++i) p[i] = uint32_t((f1 * i + f2 * (i * i)) % K);
  return p;
}

ConvCode::ConvCode(const Trellis& trellis, uint32_t length, int termination) {
  if (length == 0) throw std::invalid_argument("Invalid length");
  if (termination != 0 && termination != 1) throw std::invalid_argument("Invalid termination");
  c_.trellis = trellis;
  c_.length = length;
  c_.termination = termination;
  c_.tail = termination == 0 ? trellis.state_size : 0;
  c_.perm.resize(size_t(length) * trellis.input_size);
  for (size_t i = 0; i < c_.perm.size(); ++i) c_.perm[i] = uint32_t(i);
}

void ConvCode::set_decoder(const ConvDecoderConfig& cfg) {
  if (cfg.algorithm < 0 || cfg.algorithm > 2) throw std::invalid_argument("Invalid decoder algorithm");
  dec_ = cfg;
}

void ConvCode::encode(const uint8_t* msg, uint8_t* parity) const {
  std::vector<uint8_t> tail_bits(size_t(c_.tail) * c_.trellis.input_size + 1);
  c_.encode(msg, parity, tail_bits.data());
}

bool ConvCode::check(const uint8_t* parity) const {
  const Trellis& t = c_.trellis;
  uint32_t state = 0;
  for (uint32_t j = 0; j < c_.length + c_.tail; ++j, parity += t.output_size) {
    bool found = false;
    for (uint32_t u = 0; u < t.input_count && !found; ++u) {
      const uint32_t out = t.output[state * t.input_count + u];
      bool equal = true;
      for (uint32_t k = 0; k < t.output_size && equal; ++k) equal = ((out >> k) & 1) == (parity[k] & 1);
      if (equal) {
        found = true;
        state = t.next_state[state * t.input_count + u];
      }
    }
    if (!found) return false;
  }
  return c_.termination == 0 ? state == 0 : true;
}

std::vector<uint32_t> crc24_syndrome_table(uint32_t K, uint32_t poly) {
  std::vector<uint32_t> t(K);
  uint32_t r = poly & 0xFFFFFFu;  // a single 1 as the last bit
  for (uint32_t i = K; i-- > 0;) {
    t[i] = r;
    const uint32_t fb = (r >> 23) & 1u;  // one more zero bit after it
    r = (r << 1) & 0xFFFFFFu;
    if (fb) r ^= poly;
  }
  return t;
}

}  // namespace fecl
