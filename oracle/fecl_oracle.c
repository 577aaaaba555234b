/*
 * Test infrastructure, not product code: CPU restatement of FeCl's decode path.
 * See fecl_oracle.h.  FP64 throughout, with the reference's loop and operation
 * order, so that the results equal the reference's bit for bit; compiled with
 * -ffp-contract=off, as the reference's C++11 build contracts nothing.
 */
#define _GNU_SOURCE
#include "fecl_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

#include "dvbs2_tables.h"
#include "lte_qpp_table.h"

/* ======================================================================== */
/* Small helpers                                                            */
/* ======================================================================== */

/* std::max(a, b) and std::min(a, b) of the reference: (a < b) ? b : a, (b < a) ? b : a */
static inline double smax(double a, double b) { return (a < b) ? b : a; }
static inline double smin(double a, double b) { return (b < a) ? b : a; }

static int popcount64(uint64_t x) { return __builtin_popcountll(x); }
static int parity64(uint64_t x) { return __builtin_parityll(x); }

/* Linearlog1pexpm (src/detail/LinearTable.h:56-81): 8 samples of log(1 + exp(-x)) at
 * x = i / 2, linear in between, 0 from x >= 3.5. */
static double g_lut[8];
static pthread_once_t g_lut_once = PTHREAD_ONCE_INIT;
static void lut_init(void) {
  for (int i = 0; i < 8; ++i) g_lut[i] = log(1.0 + exp(-((double)i / 2.0)));
}
static inline double log1pexpm(double x) {
  x *= 2.0;
  if (x >= 7.0) return 0.0;
  size_t i = (size_t)x;
  return (g_lut[i + 1] - g_lut[i]) * (x - (double)i) + g_lut[i];
}

typedef struct {
  uint32_t rows, cols;
  uint32_t* row_ptr; /* rows + 1 */
  uint32_t* col_idx;
} csr_t;

static void csr_free(csr_t* m) {
  free(m->row_ptr);
  free(m->col_idx);
  m->row_ptr = NULL;
  m->col_idx = NULL;
}

/* ======================================================================== */
/* LDPC structure: src/detail/Ldpc.cpp:46-55 and the transform of :216-331   */
/* ======================================================================== */

typedef struct {
  uint32_t* v;
  uint32_t n, cap;
} row_t;

static int row_has(const row_t* r, uint32_t c) {
  uint32_t lo = 0, hi = r->n;
  while (lo < hi) {
    uint32_t mid = (lo + hi) / 2;
    if (r->v[mid] < c) lo = mid + 1;
    else hi = mid;
  }
  return lo < r->n && r->v[lo] == c;
}

static void row_insert(row_t* r, uint32_t c) {
  if (r->n == r->cap) {
    r->cap = r->cap ? r->cap * 2 : 8;
    r->v = (uint32_t*)realloc(r->v, r->cap * sizeof(uint32_t));
  }
  uint32_t i = r->n;
  while (i > 0 && r->v[i - 1] > c) {
    r->v[i] = r->v[i - 1];
    --i;
  }
  r->v[i] = c;
  r->n++;
}

static void row_erase(row_t* r, uint32_t c) {
  uint32_t i = 0;
  while (i < r->n && r->v[i] != c) ++i;
  if (i == r->n) return;
  memmove(r->v + i, r->v + i + 1, (r->n - i - 1) * sizeof(uint32_t));
  r->n--;
}

/* SparseBitMatrix::RowRef::swap(a, b), src/BitMatrix.h: exchange membership of a and b. */
static void row_swap_cols(row_t* r, uint32_t a, uint32_t b) {
  int ha = row_has(r, a), hb = row_has(r, b);
  if (ha == hb) return;
  if (ha) {
    row_erase(r, a);
    row_insert(r, b);
  } else {
    row_erase(r, b);
    row_insert(r, a);
  }
}

/* moveCol(a, b): column a goes to b, the columns between shift by one. */
static uint32_t moved(uint32_t c, uint32_t a, uint32_t b) {
  if (c == a) return b;
  if (a > b && c >= b && c < a) return c + 1;
  if (a < b && c > a && c <= b) return c - 1;
  return c;
}

static int cmp_u32(const void* x, const void* y) {
  uint32_t a = *(const uint32_t*)x, b = *(const uint32_t*)y;
  return (a > b) - (a < b);
}

static void row_move_col(row_t* r, uint32_t a, uint32_t b) {
  for (uint32_t i = 0; i < r->n; ++i) r->v[i] = moved(r->v[i], a, b);
  qsort(r->v, r->n, sizeof(uint32_t), cmp_u32);
}

typedef struct {
  uint64_t* w;
} dense_t;

static int d_test(const dense_t* d, uint64_t words, uint64_t c) { return c / 64 < words && ((d->w[c / 64] >> (c % 64)) & 1); }
static void d_set(dense_t* d, uint64_t c, int v) {
  if (v) d->w[c / 64] |= (uint64_t)1 << (c % 64);
  else d->w[c / 64] &= ~((uint64_t)1 << (c % 64));
}

struct fo_ldpc {
  uint32_t msg, N, M, max_degree;
  csr_t H, DC, A, B, T; /* T stored transposed, as src/detail/Ldpc.cpp:330 */
};

static csr_t rows_to_csr(uint32_t cols, row_t* rows, uint32_t r0, uint32_t r1, uint32_t c0, uint32_t c1) {
  csr_t m;
  m.rows = r1 - r0;
  m.cols = c1 - c0;
  m.row_ptr = (uint32_t*)calloc(m.rows + 1, sizeof(uint32_t));
  uint64_t nnz = 0;
  for (uint32_t r = r0; r < r1; ++r)
    for (uint32_t i = 0; i < rows[r].n; ++i)
      if (rows[r].v[i] >= c0 && rows[r].v[i] < c1) ++nnz;
  m.col_idx = (uint32_t*)malloc((nnz ? nnz : 1) * sizeof(uint32_t));
  uint64_t e = 0;
  for (uint32_t r = r0; r < r1; ++r) {
    for (uint32_t i = 0; i < rows[r].n; ++i)
      if (rows[r].v[i] >= c0 && rows[r].v[i] < c1) m.col_idx[e++] = rows[r].v[i] - c0;
    m.row_ptr[r - r0 + 1] = (uint32_t)e;
  }
  (void)cols;
  return m;
}

static csr_t csr_transpose(const csr_t* m) {
  csr_t t;
  t.rows = m->cols;
  t.cols = m->rows;
  t.row_ptr = (uint32_t*)calloc(t.rows + 1, sizeof(uint32_t));
  uint64_t nnz = m->row_ptr[m->rows];
  t.col_idx = (uint32_t*)malloc((nnz ? nnz : 1) * sizeof(uint32_t));
  for (uint64_t e = 0; e < nnz; ++e) t.row_ptr[m->col_idx[e] + 1]++;
  for (uint32_t r = 0; r < t.rows; ++r) t.row_ptr[r + 1] += t.row_ptr[r];
  uint32_t* fill = (uint32_t*)malloc((t.rows + 1) * sizeof(uint32_t));
  memcpy(fill, t.row_ptr, (t.rows + 1) * sizeof(uint32_t));
  for (uint32_t r = 0; r < m->rows; ++r)
    for (uint32_t e = m->row_ptr[r]; e < m->row_ptr[r + 1]; ++e) t.col_idx[fill[m->col_idx[e]]++] = r;
  free(fill);
  return t;
}

fo_ldpc* fo_ldpc_create(uint32_t R, uint32_t N, const uint32_t* row_ptr, const uint32_t* col_idx) {
  if (R == 0 || N <= R) return NULL;
  fo_ldpc* c = (fo_ldpc*)calloc(1, sizeof(fo_ldpc));
  row_t* rows = (row_t*)calloc(R, sizeof(row_t));
  for (uint32_t r = 0; r < R; ++r) {
    uint32_t d = row_ptr[r + 1] - row_ptr[r];
    rows[r].cap = d + 8;
    rows[r].n = d;
    rows[r].v = (uint32_t*)malloc(rows[r].cap * sizeof(uint32_t));
    memcpy(rows[r].v, col_idx + row_ptr[r], d * sizeof(uint32_t));
  }
  uint64_t msg = N - R; /* src/detail/Ldpc.cpp:48 */

  /* Column weights over the active rows; retire the lowest-weight column from the
   * right with its rows (src/detail/Ldpc.cpp:218-258). */
  uint64_t* weight = (uint64_t*)calloc(N, sizeof(uint64_t));
  for (uint32_t r = 0; r < R; ++r)
    for (uint32_t i = 0; i < rows[r].n; ++i) weight[rows[r].v[i]]++;
  uint64_t active = R, t = 0;
  int64_t cursor = (int64_t)R - 1;
  for (uint64_t i = N; i > 0; --i) {
    for (; cursor >= (int64_t)active; --cursor)
      for (uint32_t k = 0; k < rows[cursor].n; ++k) weight[rows[cursor].v[k]]--;
    uint64_t best = (uint64_t)-1, best_idx = 0;
    for (int64_t j = (int64_t)i - 1; j >= 0; --j) {
      if (weight[j] == 1) {
        best_idx = (uint64_t)j;
        best = 1;
        break;
      } else if (weight[j] < best && weight[j] >= 1) {
        best_idx = (uint64_t)j;
        best = weight[j];
      }
    }
    if (best_idx != i - 1)
      for (uint32_t r = 0; r < R; ++r) row_swap_cols(&rows[r], (uint32_t)best_idx, (uint32_t)(i - 1));
    uint64_t tmpw = weight[best_idx];
    weight[best_idx] = weight[i - 1];
    weight[i - 1] = tmpw;
    int64_t end = (int64_t)active;
    for (int64_t r = 0; r < end; ++r) {
      if (row_has(&rows[r], (uint32_t)(i - 1))) {
        --end;
        row_t tr = rows[end];
        rows[end] = rows[r];
        rows[r] = tr;
        --r;
      }
    }
    active -= best > 1 ? best : 1;
    if (active == 0) {
      t = N - i + 1;
      break;
    }
  }
  free(weight);

  /* a one on the diagonal of the T block (:260-271) */
  for (uint64_t i = 0; i < t; ++i) {
    uint32_t col = (uint32_t)(i + N - t);
    if (!row_has(&rows[i], col)) {
      for (uint64_t r = i + 1; r < R; ++r) {
        if (row_has(&rows[r], col)) {
          row_t tr = rows[i];
          rows[i] = rows[r];
          rows[r] = tr;
          break;
        }
      }
    }
  }

  /* dense block of the remaining rows with the T columns eliminated (:273-281) */
  const uint64_t words = (N + 63) / 64;
  const uint64_t nc = R - t;
  dense_t* cde = (dense_t*)calloc(nc ? nc : 1, sizeof(dense_t));
  for (uint64_t r = 0; r < nc; ++r) {
    cde[r].w = (uint64_t*)calloc(words, sizeof(uint64_t));
    for (uint32_t k = 0; k < rows[t + r].n; ++k) d_set(&cde[r], rows[t + r].v[k], 1);
  }
  for (int64_t i = (int64_t)t - 1; i >= 0; --i) {
    uint64_t col = (uint64_t)i + N - t;
    for (uint64_t r = 0; r < nc; ++r)
      if (d_test(&cde[r], words, col))
        for (uint32_t k = 0; k < rows[i].n; ++k) cde[r].w[rows[i].v[k] / 64] ^= (uint64_t)1 << (rows[i].v[k] % 64);
  }

  /* forward elimination of the gap; dependent rows grow the message (:283-316) */
  for (int64_t i = 0; i < (int64_t)(N - t - msg); ++i) {
    int found = 0;
    for (uint64_t r = (uint64_t)i; r < nc; ++r) {
      if (d_test(&cde[r], words, (uint64_t)i + msg)) {
        dense_t tmp = cde[r];
        cde[r] = cde[i];
        cde[i] = tmp;
        found = 1;
        break;
      }
    }
    if (!found) {
      for (uint64_t r = (uint64_t)i; r < nc; ++r) {
        int64_t k = -1;
        for (uint64_t q = 0; q < words; ++q)
          if (cde[r].w[q]) {
            k = (int64_t)(q * 64 + __builtin_ctzll(cde[r].w[q]));
            break;
          }
        if (k != -1) {
          uint32_t a = (uint32_t)k, b = (uint32_t)((uint64_t)i + msg);
          if (a != b) {
            for (uint32_t rr = 0; rr < R; ++rr) row_swap_cols(&rows[rr], a, b);
            for (uint64_t rr = 0; rr < nc; ++rr) {
              int va = d_test(&cde[rr], words, a), vb = d_test(&cde[rr], words, b);
              d_set(&cde[rr], a, vb);
              d_set(&cde[rr], b, va);
            }
          }
          dense_t tmp = cde[r];
          cde[r] = cde[i];
          cde[i] = tmp;
          found = 1;
          break;
        }
      }
    }
    if (!found) {
      uint32_t a = (uint32_t)((uint64_t)i + msg), b = (uint32_t)msg;
      for (uint32_t rr = 0; rr < R; ++rr) row_move_col(&rows[rr], a, b);
      for (uint64_t rr = 0; rr < nc; ++rr) {
        uint64_t* nw = (uint64_t*)calloc(words, sizeof(uint64_t));
        for (uint32_t col = 0; col < N; ++col)
          if (d_test(&cde[rr], words, col)) {
            uint32_t m2 = moved(col, a, b);
            nw[m2 / 64] |= (uint64_t)1 << (m2 % 64);
          }
        free(cde[rr].w);
        cde[rr].w = nw;
      }
      ++msg;
      --i;
      continue;
    }
    for (uint64_t r = (uint64_t)i + 1; r < nc; ++r)
      if (d_test(&cde[r], words, (uint64_t)i + msg))
        for (uint64_t q = 0; q < words; ++q) cde[r].w[q] ^= cde[i].w[q];
  }
  /* back substitution (:318-324) */
  for (int64_t i = (int64_t)nc - 1; i >= 0; --i)
    for (int64_t r = i - 1; r >= 0; --r)
      if (d_test(&cde[r], words, (uint64_t)i + msg))
        for (uint64_t q = 0; q < words; ++q) cde[r].w[q] ^= cde[i].w[q];

  c->msg = (uint32_t)msg;
  c->N = N;
  c->M = R;
  c->H = rows_to_csr(N, rows, 0, R, 0, N);
  const uint32_t gap = (uint32_t)(N - msg - t);
  {
    row_t* dcr = (row_t*)calloc(gap ? gap : 1, sizeof(row_t));
    for (uint32_t r = 0; r < gap && r < nc; ++r)
      for (uint32_t col = 0; col < msg; ++col)
        if (d_test(&cde[r], words, col)) row_insert(&dcr[r], col);
    c->DC = rows_to_csr((uint32_t)msg, dcr, 0, gap, 0, (uint32_t)msg);
    for (uint32_t r = 0; r < gap; ++r) free(dcr[r].v);
    free(dcr);
  }
  c->A = rows_to_csr(N, rows, 0, (uint32_t)t, 0, (uint32_t)msg);
  c->B = rows_to_csr(N, rows, 0, (uint32_t)t, (uint32_t)msg, (uint32_t)msg + gap);
  {
    csr_t Tn = rows_to_csr(N, rows, 0, (uint32_t)t, (uint32_t)(N - t), N);
    c->T = csr_transpose(&Tn);
    csr_free(&Tn);
  }
  c->max_degree = 0;
  for (uint32_t r = 0; r < R; ++r)
    if (c->H.row_ptr[r + 1] - c->H.row_ptr[r] > c->max_degree) c->max_degree = c->H.row_ptr[r + 1] - c->H.row_ptr[r];
  for (uint64_t r = 0; r < nc; ++r) free(cde[r].w);
  free(cde);
  for (uint32_t r = 0; r < R; ++r) free(rows[r].v);
  free(rows);
  return c;
}

void fo_ldpc_destroy(fo_ldpc* c) {
  if (!c) return;
  csr_free(&c->H);
  csr_free(&c->DC);
  csr_free(&c->A);
  csr_free(&c->B);
  csr_free(&c->T);
  free(c);
}

void fo_ldpc_sizes(const fo_ldpc* c, uint64_t* msg, uint64_t* parity, uint64_t* state, uint32_t* max_degree) {
  if (msg) *msg = c->msg;
  if (parity) *parity = c->N;
  if (state) *state = c->H.row_ptr[c->M];
  if (max_degree) *max_degree = c->max_degree;
}

void fo_ldpc_checks(const fo_ldpc* c, uint32_t* row_ptr, uint32_t* col_idx) {
  memcpy(row_ptr, c->H.row_ptr, (c->M + 1) * sizeof(uint32_t));
  memcpy(col_idx, c->H.col_idx, c->H.row_ptr[c->M] * sizeof(uint32_t));
}

/* Ldpc::Structure::encode, src/detail/Ldpc.cpp:180-209 */
void fo_ldpc_encode(const fo_ldpc* c, const uint8_t* msg, uint8_t* parity) {
  for (uint32_t i = 0; i < c->msg; ++i) parity[i] = msg[i] & 1;
  for (uint32_t i = c->msg; i < c->N; ++i) parity[i] = 0;
  uint8_t* p = parity + c->msg;
  const uint32_t gap = c->DC.rows;
  for (uint32_t r = 0; r < gap; ++r)
    for (uint32_t e = c->DC.row_ptr[r]; e < c->DC.row_ptr[r + 1]; ++e) p[r] ^= msg[c->DC.col_idx[e]] & 1;
  for (uint32_t r = 0; r < c->B.rows; ++r)
    for (uint32_t e = c->B.row_ptr[r]; e < c->B.row_ptr[r + 1]; ++e) p[gap + r] ^= p[c->B.col_idx[e]];
  uint8_t* p2 = p + gap;
  for (uint32_t r = 0; r < c->A.rows; ++r)
    for (uint32_t e = c->A.row_ptr[r]; e < c->A.row_ptr[r + 1]; ++e) p2[r] ^= msg[c->A.col_idx[e]] & 1;
  for (uint32_t r = 0; r < c->T.rows; ++r)
    for (uint32_t e = c->T.row_ptr[r] + 1; e < c->T.row_ptr[r + 1]; ++e) p2[c->T.col_idx[e]] ^= p2[r];
}

/* Ldpc::Structure::check, src/detail/Ldpc.cpp:160-172 */
static int ldpc_check_bits(const fo_ldpc* c, const uint8_t* hard) {
  for (uint32_t r = 0; r < c->M; ++r) {
    uint8_t s = 0;
    for (uint32_t e = c->H.row_ptr[r]; e < c->H.row_ptr[r + 1]; ++e) s ^= hard[c->H.col_idx[e]];
    if (s) return 0;
  }
  return 1;
}
int fo_ldpc_check(const fo_ldpc* c, const uint8_t* parity) { return ldpc_check_bits(c, parity); }

/* ======================================================================== */
/* BP decoder: src/detail/BpDecoder/BpDecoderImpl.cpp                       */
/* ======================================================================== */

typedef struct {
  double* parity;     /* parity_ */
  double* bit;        /* bitMetrics_ */
  double* cm;         /* checkMetrics_ */
  double* cmb;        /* checkMetricsBuffer_ */
  uint8_t* hard;      /* hardParity_ */
} bp_work;

/* Box-sum policies, src/detail/LlrMetrics.h:126-196. */
static inline double bp_prior(int alg, double x) { return alg == 0 ? tanh(-x / 2.0) : x; }
static inline double bp_post(int alg, double x) { return alg == 0 ? -log((1.0 + x) / (1.0 - x)) : x; }
static inline double bp_sum(int alg, double a, double b) {
  if (alg == 0) return a * b;
  const int differ = (signbit(a) != 0) ^ (signbit(b) != 0);
  const double m = smin(fabs(a), fabs(b));
  if (alg == 1) return (differ ? m : -m) - log1pexpm(fabs(a + b)) + log1pexpm(fabs(a - b));
  return differ ? m : -m;
}

/* checkUpdate(i), BpDecoderImpl.cpp:132-159 */
static void bp_check_update(const fo_ldpc* c, int alg, const double* scaling, uint32_t n_scaling, size_t i,
                            bp_work* w) {
  double* tmp = w->cmb; /* checkMetricTmp, reused for every row */
  const size_t stride = c->max_degree - 1;
  for (uint32_t r = 0; r < c->M; ++r) {
    double* first = w->cm + c->H.row_ptr[r];
    const size_t size = c->H.row_ptr[r + 1] - c->H.row_ptr[r];
    const double sf = scaling[(i % n_scaling) * stride + (size - 2)];
    double prod = bp_prior(alg, first[0]);
    for (size_t j = 1; j < size - 1; ++j) {
      tmp[j] = bp_prior(alg, first[j]);
      first[j] = prod;
      prod = bp_sum(alg, prod, tmp[j]);
    }
    tmp[size - 1] = bp_prior(alg, first[size - 1]);
    first[size - 1] = sf * (bp_post(alg, prod));
    prod = tmp[size - 1];
    for (size_t j = size - 2; j > 0; --j) {
      first[j] = sf * (bp_post(alg, bp_sum(alg, first[j], prod)));
      prod = bp_sum(alg, prod, tmp[j]);
    }
    *first = sf * (bp_post(alg, prod));
  }
}

/* bitUpdate(), BpDecoderImpl.cpp:161-179 */
static void bp_bit_update(const fo_ldpc* c, bp_work* w) {
  const uint64_t E = c->H.row_ptr[c->M];
  memset(w->bit, 0, c->N * sizeof(double));
  for (uint64_t i = 0; i < E; ++i) {
    w->cmb[i] = w->cm[i];
    double* ref = &w->bit[c->H.col_idx[i]];
    w->cm[i] = *ref;
    *ref += w->cmb[i];
  }
  memcpy(w->bit, w->parity, c->N * sizeof(double));
  for (int64_t i = (int64_t)E - 1; i >= 0; --i) {
    double* ref = &w->bit[c->H.col_idx[i]];
    w->cm[i] += *ref;
    *ref += w->cmb[i];
  }
}

/* the iteration loop shared by decodeBlock and soDecodeBlock (:48-61) */
static int bp_iterate(const fo_ldpc* c, int alg, uint32_t iterations, const double* scaling, uint32_t n_scaling,
                      bp_work* w) {
  int ran = 0;
  for (int64_t i = 0; i < (int64_t)iterations - 1; ++i) {
    bp_check_update(c, alg, scaling, n_scaling, (size_t)i, w);
    bp_bit_update(c, w);
    ++ran;
    for (uint32_t j = 0; j < c->N; ++j) w->hard[j] = (w->bit[j] >= 0.0);
    if (ldpc_check_bits(c, w->hard)) break;
  }
  bp_check_update(c, alg, scaling, n_scaling, iterations - 1, w);
  return ran + 1;
}

static void bp_work_alloc(const fo_ldpc* c, bp_work* w) {
  const uint64_t E = c->H.row_ptr[c->M];
  w->parity = (double*)malloc(c->N * sizeof(double));
  w->bit = (double*)malloc(c->N * sizeof(double));
  w->cm = (double*)malloc(E * sizeof(double));
  w->cmb = (double*)malloc(E * sizeof(double));
  w->hard = (uint8_t*)malloc(c->N);
}
static void bp_work_free(bp_work* w) {
  free(w->parity);
  free(w->bit);
  free(w->cm);
  free(w->cmb);
  free(w->hard);
}

/* decodeBlock, BpDecoderImpl.cpp:37-70 */
static void bp_decode_block(const fo_ldpc* c, int alg, uint32_t iterations, const double* scaling, uint32_t n_scaling,
                            const double* llr, uint8_t* msg, int32_t* its, bp_work* w) {
  const uint64_t E = c->H.row_ptr[c->M];
  memcpy(w->parity, llr, c->N * sizeof(double));
  if (iterations > 0)
    for (uint64_t i = 0; i < E; ++i) w->cm[i] = w->parity[c->H.col_idx[i]];
  int ran = bp_iterate(c, alg, iterations, scaling, n_scaling, w);
  memcpy(w->bit, w->parity, c->N * sizeof(double));
  for (uint64_t i = 0; i < E; ++i) w->bit[c->H.col_idx[i]] += w->cm[i];
  for (uint32_t i = 0; i < c->msg; ++i) msg[i] = w->bit[i] >= 0;
  if (its) *its = ran;
}

/* soDecodeBlock, BpDecoderImpl.cpp:72-130 */
static void bp_so_decode_block(const fo_ldpc* c, int alg, uint32_t iterations, const double* scaling,
                               uint32_t n_scaling, const double* parity, const double* syst, const double* state,
                               double* msg, double* syst_out, double* parity_out, double* state_out, bp_work* w) {
  const uint64_t E = c->H.row_ptr[c->M];
  memcpy(w->parity, parity, c->N * sizeof(double));
  if (syst)
    for (uint32_t i = 0; i < c->msg; ++i) w->parity[i] += syst[i];
  if (state) memcpy(w->cm, state, E * sizeof(double));
  if (iterations > 0) {
    if (state) bp_bit_update(c, w);
    else
      for (uint64_t i = 0; i < E; ++i) w->cm[i] = w->parity[c->H.col_idx[i]];
  }
  bp_iterate(c, alg, iterations, scaling, n_scaling, w);
  memset(w->bit, 0, c->N * sizeof(double));
  for (uint64_t i = 0; i < E; ++i) w->bit[c->H.col_idx[i]] += w->cm[i];
  if (syst_out) memcpy(syst_out, w->bit, c->msg * sizeof(double));
  if (parity_out) memcpy(parity_out, w->bit, c->N * sizeof(double));
  if (state_out) memcpy(state_out, w->cm, E * sizeof(double));
  if (msg)
    for (uint32_t i = 0; i < c->msg; ++i) msg[i] = w->parity[i] + w->bit[i];
}

/* ---- frame-parallel driver (the reference splits blocks over std::threads,
 *      src/Codec.h:210-238; each frame is independent) ---- */

typedef struct {
  void (*fn)(void* ctx, uint64_t f, void* work);
  void* (*alloc)(void* ctx);
  void (*release)(void* work);
  void* ctx;
  uint64_t begin, end;
} job_t;

static void* job_run(void* arg) {
  job_t* j = (job_t*)arg;
  void* work = j->alloc(j->ctx);
  for (uint64_t f = j->begin; f < j->end; ++f) j->fn(j->ctx, f, work);
  j->release(work);
  return NULL;
}

static void run_frames(uint64_t nframes, int threads, void (*fn)(void*, uint64_t, void*), void* (*alloc)(void*),
                       void (*release)(void*), void* ctx) {
  if (threads < 1) threads = 1;
  if ((uint64_t)threads > nframes) threads = (int)(nframes ? nframes : 1);
  job_t* jobs = (job_t*)calloc(threads, sizeof(job_t));
  pthread_t* tids = (pthread_t*)calloc(threads, sizeof(pthread_t));
  const uint64_t step = (nframes + threads - 1) / threads;
  for (int t = 0; t < threads; ++t) {
    jobs[t].fn = fn;
    jobs[t].alloc = alloc;
    jobs[t].release = release;
    jobs[t].ctx = ctx;
    jobs[t].begin = t * step < nframes ? t * step : nframes;
    jobs[t].end = (t + 1) * step < nframes ? (t + 1) * step : nframes;
  }
  for (int t = 1; t < threads; ++t) pthread_create(&tids[t], NULL, job_run, &jobs[t]);
  job_run(&jobs[0]);
  for (int t = 1; t < threads; ++t) pthread_join(tids[t], NULL);
  free(jobs);
  free(tids);
}

typedef struct {
  const fo_ldpc* c;
  int alg;
  uint32_t iterations;
  const double* scaling;
  uint32_t n_scaling;
  const double *llr, *syst, *state;
  uint8_t* msg;
  int32_t* its;
  double *msg_out, *syst_out, *parity_out, *state_out;
} ldpc_ctx;

static void* ldpc_alloc(void* ctx) {
  bp_work* w = (bp_work*)malloc(sizeof(bp_work));
  bp_work_alloc(((ldpc_ctx*)ctx)->c, w);
  return w;
}
static void ldpc_release(void* w) {
  bp_work_free((bp_work*)w);
  free(w);
}
static void ldpc_decode_frame(void* vctx, uint64_t f, void* work) {
  ldpc_ctx* x = (ldpc_ctx*)vctx;
  const fo_ldpc* c = x->c;
  bp_decode_block(c, x->alg, x->iterations, x->scaling, x->n_scaling, x->llr + f * c->N, x->msg + f * c->msg,
                  x->its ? x->its + f : NULL, (bp_work*)work);
}
static void ldpc_so_decode_frame(void* vctx, uint64_t f, void* work) {
  ldpc_ctx* x = (ldpc_ctx*)vctx;
  const fo_ldpc* c = x->c;
  const uint64_t E = c->H.row_ptr[c->M];
  bp_so_decode_block(c, x->alg, x->iterations, x->scaling, x->n_scaling, x->llr + f * c->N,
                     x->syst ? x->syst + f * c->msg : NULL, x->state ? x->state + f * E : NULL,
                     x->msg_out ? x->msg_out + f * c->msg : NULL, x->syst_out ? x->syst_out + f * c->msg : NULL,
                     x->parity_out ? x->parity_out + f * c->N : NULL, x->state_out ? x->state_out + f * E : NULL,
                     (bp_work*)work);
}

int fo_ldpc_decode(const fo_ldpc* c, int algorithm, uint32_t iterations, const double* scaling, uint32_t n_scaling,
                   const double* llr, uint64_t nframes, uint8_t* msg, int32_t* iterations_run, int threads) {
  if (!c || iterations == 0 || !scaling || n_scaling == 0) return -1;
  pthread_once(&g_lut_once, lut_init);
  ldpc_ctx x = {c, algorithm, iterations, scaling, n_scaling, llr, NULL, NULL, msg, iterations_run,
                NULL, NULL, NULL, NULL};
  run_frames(nframes, threads, ldpc_decode_frame, ldpc_alloc, ldpc_release, &x);
  return 0;
}

int fo_ldpc_so_decode(const fo_ldpc* c, int algorithm, uint32_t iterations, const double* scaling,
                      uint32_t n_scaling, const double* parity, const double* syst, const double* state,
                      uint64_t nframes, double* msg, double* syst_out, double* parity_out, double* state_out,
                      int threads) {
  if (!c || iterations == 0 || !scaling || n_scaling == 0) return -1;
  pthread_once(&g_lut_once, lut_init);
  ldpc_ctx x = {c, algorithm, iterations, scaling, n_scaling, parity, syst, state, NULL, NULL,
                msg, syst_out, parity_out, state_out};
  run_frames(nframes, threads, ldpc_so_decode_frame, ldpc_alloc, ldpc_release, &x);
  return 0;
}

/* ======================================================================== */
/* DVB-S2 matrix                                                            */
/* ======================================================================== */

int fo_dvbs2_matrix(uint32_t n, uint32_t rate_num, uint32_t rate_den, uint32_t* out_rows, uint32_t* out_cols,
                    uint64_t* out_nnz, uint32_t* row_ptr, uint32_t* col_idx) {
  int code = -1;
  for (int i = 0; i < FECL_DVBS2_CODE_COUNT; ++i)
    if (fecl_dvbs2_codes[i][0] == n &&
        (uint64_t)fecl_dvbs2_codes[i][1] * rate_den == (uint64_t)rate_num * fecl_dvbs2_codes[i][2])
      code = i;
  if (code < 0) return -1;
  const uint32_t q = fecl_dvbs2_codes[code][3], first = fecl_dvbs2_codes[code][4], groups = fecl_dvbs2_codes[code][5];
  const uint32_t M = 360 * q, K = n - M;
  row_t* rows = (row_t*)calloc(M, sizeof(row_t));
  for (uint32_t g = 0; g < groups; ++g) {
    const uint32_t off = fecl_dvbs2_rows[first + g][0], len = fecl_dvbs2_rows[first + g][1];
    for (uint32_t m = 0; m < 360; ++m)
      for (uint32_t a = 0; a < len; ++a) row_insert(&rows[(fecl_dvbs2_addr[off + a] + m * q) % M], g * 360 + m);
  }
  for (uint32_t i = 0; i < M; ++i) {
    row_insert(&rows[i], K + i);
    if (i + 1 < M) row_insert(&rows[i + 1], K + i);
  }
  uint64_t nnz = 0;
  for (uint32_t r = 0; r < M; ++r) nnz += rows[r].n;
  if (out_rows) *out_rows = M;
  if (out_cols) *out_cols = n;
  if (out_nnz) *out_nnz = nnz;
  if (row_ptr) {
    uint64_t e = 0;
    row_ptr[0] = 0;
    for (uint32_t r = 0; r < M; ++r) {
      memcpy(col_idx + e, rows[r].v, rows[r].n * sizeof(uint32_t));
      e += rows[r].n;
      row_ptr[r + 1] = (uint32_t)e;
    }
  }
  for (uint32_t r = 0; r < M; ++r) free(rows[r].v);
  free(rows);
  return 0;
}

/* ======================================================================== */
/* Trellis, interleaver                                                     */
/* ======================================================================== */

int fo_trellis(uint32_t ninputs, const uint32_t* cl, uint32_t noutputs, const uint64_t* gen, const uint64_t* fb_in,
               uint32_t* state_count, uint32_t* input_count, uint32_t* next_state, uint32_t* output) {
  uint64_t fb[16];
  if (ninputs == 0 || ninputs > 16) return -1;
  uint32_t state_size = 0;
  for (uint32_t i = 0; i < ninputs; ++i) {
    fb[i] = fb_in ? fb_in[i] : ((uint64_t)1 << (cl[i] - 1));
    state_size += cl[i] - 1;
  }
  const uint32_t S = 1u << state_size, U = 1u << ninputs;
  if (state_count) *state_count = S;
  if (input_count) *input_count = U;
  if (!next_state) return 0;
  for (uint32_t s = 0; s < S; ++s)
    for (uint32_t u = 0; u < U; ++u) {
      uint32_t next = 0, out = 0, j = 0;
      for (uint32_t i = 0; i < ninputs; ++i) {
        const uint32_t regs = cl[i] - 1;
        const uint64_t st = ((uint64_t)s >> j) & (((uint64_t)1 << regs) - 1);
        const uint32_t in = (u >> i) & 1;
        const uint32_t loop = (uint32_t)parity64(st & fb[i]);
        for (uint32_t k = 0; k < noutputs; ++k) {
          const uint64_t g = gen[i * noutputs + k];
          if ((g >> cl[i]) != 0) return -1;
          out ^= ((((in ^ loop) & (uint32_t)((g >> (cl[i] - 1)) & 1))) ^ (uint32_t)parity64(st & g)) << k;
        }
        if (((fb[i] >> (cl[i] - 1)) & 1) != 1) return -1;
        next |= ((in & (uint32_t)((fb[i] >> (cl[i] - 1)) & 1)) ^ loop) << (j + cl[i] - 2);
        next |= (uint32_t)(st >> 1) << j;
        j += regs;
      }
      next_state[s * U + u] = next;
      output[s * U + u] = out;
    }
  return 0;
}

int fo_lte_interleaver(uint32_t K, uint32_t* perm) {
  for (int i = 0; i < FECL_LTE_QPP_COUNT; ++i) {
    if (fecl_lte_qpp[i][0] == K) {
      const uint64_t f1 = fecl_lte_qpp[i][1], f2 = fecl_lte_qpp[i][2];
      for (uint64_t k = 0; k < K; ++k) perm[k] = (uint32_t)((f1 * k + f2 * (k * k)) % K);
      return 0;
    }
  }
  return -1;
}

/* ======================================================================== */
/* Turbo structure: src/detail/Turbo.cpp:45-103, src/detail/Convolutional.cpp:45-67 */
/* ======================================================================== */

typedef struct {
  uint32_t S, U, in_size, out_size, state_size;
  uint32_t* next;
  uint32_t* out;
  uint32_t length, tail, termination;
  uint32_t* perm;
  uint32_t perm_len;
} constituent_t;

struct fo_turbo {
  uint32_t n;
  uint64_t msg, syst, parity, state, tail;
  constituent_t* c;
};

static uint32_t ilog2(uint32_t v) {
  uint32_t l = 0;
  while ((1u << l) < v) ++l;
  return l;
}

static uint32_t c_msg(const constituent_t* k) { return k->length * k->in_size; }
static uint32_t c_syst(const constituent_t* k) { return (k->length + k->tail) * k->in_size; }
static uint32_t c_syst_tail(const constituent_t* k) { return k->tail * k->in_size; }
static uint32_t c_parity(const constituent_t* k) { return (k->length + k->tail) * k->out_size; }

fo_turbo* fo_turbo_create(uint32_t n, const uint32_t* state_count, const uint32_t* input_count,
                          const uint32_t* output_size, const uint32_t* const* next_state,
                          const uint32_t* const* output, uint32_t n_trellis, const uint32_t* perm_data,
                          const uint32_t* perm_len, const int32_t* termination, uint32_t n_termination) {
  if (n == 0 || (n_trellis != 1 && n_trellis != n) || (n_termination != 1 && n_termination != n)) return NULL;
  fo_turbo* t = (fo_turbo*)calloc(1, sizeof(fo_turbo));
  t->n = n;
  t->c = (constituent_t*)calloc(n, sizeof(constituent_t));
  uint64_t off = 0, msg = 0;
  for (uint32_t i = 0; i < n; ++i) {
    for (uint32_t k = 0; k < perm_len[i]; ++k)
      if (perm_data[off + k] + 1 > msg) msg = perm_data[off + k] + 1;
    off += perm_len[i];
  }
  t->msg = msg;
  off = 0;
  for (uint32_t i = 0; i < n; ++i) {
    constituent_t* k = &t->c[i];
    const uint32_t ti = n_trellis == 1 ? 0 : i;
    k->S = state_count[ti];
    k->U = input_count[ti];
    k->in_size = ilog2(k->U);
    k->out_size = output_size[ti];
    k->state_size = ilog2(k->S);
    k->next = (uint32_t*)malloc(k->S * k->U * sizeof(uint32_t));
    k->out = (uint32_t*)malloc(k->S * k->U * sizeof(uint32_t));
    memcpy(k->next, next_state[ti], k->S * k->U * sizeof(uint32_t));
    memcpy(k->out, output[ti], k->S * k->U * sizeof(uint32_t));
    if (perm_len[i] == 0) {
      k->perm_len = (uint32_t)msg;
      k->perm = (uint32_t*)malloc((msg ? msg : 1) * sizeof(uint32_t));
      for (uint32_t q = 0; q < msg; ++q) k->perm[q] = q;
    } else {
      k->perm_len = perm_len[i];
      k->perm = (uint32_t*)malloc(perm_len[i] * sizeof(uint32_t));
      memcpy(k->perm, perm_data + off, perm_len[i] * sizeof(uint32_t));
    }
    off += perm_len[i];
    k->length = k->perm_len / k->in_size;
    k->termination = (uint32_t)termination[n_termination == 1 ? 0 : i];
    k->tail = k->termination == 0 ? k->state_size : 0;
  }
  t->tail = t->parity = t->state = 0;
  for (uint32_t i = 0; i < n; ++i) {
    t->tail += c_syst_tail(&t->c[i]);
    t->parity += c_parity(&t->c[i]);
    t->state += c_syst(&t->c[i]);
  }
  t->syst = t->msg + t->tail;
  t->parity += t->syst;
  return t;
}

void fo_turbo_destroy(fo_turbo* t) {
  if (!t) return;
  for (uint32_t i = 0; i < t->n; ++i) {
    free(t->c[i].next);
    free(t->c[i].out);
    free(t->c[i].perm);
  }
  free(t->c);
  free(t);
}

void fo_turbo_sizes(const fo_turbo* t, uint64_t* msg, uint64_t* syst, uint64_t* parity, uint64_t* state) {
  if (msg) *msg = t->msg;
  if (syst) *syst = t->syst;
  if (parity) *parity = t->parity;
  if (state) *state = t->state;
}

/* Convolutional::Structure::encode(msg, parity, tail), src/detail/Convolutional.cpp:167-221 */
static void conv_encode(const constituent_t* k, const uint8_t* msg, uint8_t* parity, uint8_t* tail) {
  uint32_t state = 0;
  for (uint32_t j = 0; j < k->length; ++j) {
    uint32_t in = 0;
    for (uint32_t b = 0; b < k->in_size; ++b) in |= (uint32_t)(msg[j * k->in_size + b] & 1) << b;
    const uint32_t out = k->out[state * k->U + in];
    state = k->next[state * k->U + in];
    for (uint32_t b = 0; b < k->out_size; ++b) parity[b] = (out >> b) & 1;
    parity += k->out_size;
  }
  for (uint32_t j = 0; j < k->tail; ++j) {
    int best_count = -1;
    uint32_t best = 0;
    for (uint32_t u = 0; u < k->U; ++u) {
      int cnt = popcount64(state) - popcount64(k->next[state * k->U + u]);
      if (cnt > best_count) {
        best_count = cnt;
        best = u;
      }
    }
    const uint32_t out = k->out[state * k->U + best];
    for (uint32_t b = 0; b < k->out_size; ++b) parity[b] = (out >> b) & 1;
    for (uint32_t b = 0; b < k->in_size; ++b) tail[b] = (best >> b) & 1;
    parity += k->out_size;
    tail += k->in_size;
    state = k->next[state * k->U + best];
  }
}

/* Turbo::Structure::encode, src/detail/Turbo.cpp:155-170 */
void fo_turbo_encode(const fo_turbo* t, const uint8_t* msg, uint8_t* parity) {
  for (uint64_t i = 0; i < t->msg; ++i) parity[i] = msg[i] & 1;
  uint8_t* systTail = parity + t->msg;
  uint8_t* out = parity + t->syst;
  for (uint32_t i = 0; i < t->n; ++i) {
    const constituent_t* k = &t->c[i];
    uint8_t* inter = (uint8_t*)malloc(k->perm_len ? k->perm_len : 1);
    for (uint32_t q = 0; q < k->perm_len; ++q) inter[q] = msg[k->perm[q]] & 1;
    conv_encode(k, inter, out, systTail);
    free(inter);
    systTail += c_syst_tail(k);
    out += c_parity(k);
  }
}

/* ======================================================================== */
/* MAP decoder: src/detail/MapDecoder/MapDecoderImpl.cpp                    */
/* ======================================================================== */

/* Log-sum policies, src/detail/LlrMetrics.h:48-121.  alg 0 LogSum (non-recursive),
 * 1 LinearLogSum, 2 MaxLogSum. */
static inline double ls_sum(int alg, double a, double b) {
  if (alg == 2) return smax(a, b);
  if (alg == 1) {
    if (a == b) return a;
    return smax(a, b) + log1pexpm(fabs(a - b));
  }
  return a + b;
}
static inline double ls_prior2(double x, double mx) { return (x == mx) ? 1.0 : exp(x - mx); }
static inline double ls_post2(double x, double mx) { return log(x) + mx; }

typedef struct {
  double* bm;   /* branchMetrics_ [T][S][U] */
  double* fm;   /* forwardMetrics_ [T][S] */
  double* bwm;  /* backwardMetrics_ [T][S] */
  double* buf;  /* bufferMetrics_ */
} map_work;

/* MapDecoderImpl::soDecodeBlockImpl (:67-78) for one constituent. */
static void map_decode(const constituent_t* k, int alg, double sf, const double* parity_in, double* syst,
                       int has_syst_in, double* parity_out, map_work* w) {
  const uint32_t S = k->S, U = k->U, T = k->length + k->tail, tsz = S * U;
  const double NINF = -INFINITY;
  /* branchUpdate, :80-115 */
  {
    const double* par = parity_in;
    const double* sy = syst;
    double* bm = w->bm;
    const uint32_t oc = 1u << k->out_size;
    for (uint32_t i = 0; i < T; ++i) {
      for (uint32_t j = 0; j < oc; ++j) {
        double x = 0;
        for (uint32_t b = 0; b < k->out_size; ++b)
          if ((j >> b) & 1) x += par[b];
        w->buf[j] = x;
      }
      double* bmt = bm;
      for (uint32_t s = 0; s < S; ++s)
        for (uint32_t u = 0; u < U; ++u) bm[s * U + u] = w->buf[k->out[s * U + u]];
      if (has_syst_in) {
        for (uint32_t j = 0; j < U; ++j) {
          double x = 0;
          for (uint32_t b = 0; b < k->in_size; ++b)
            if ((j >> b) & 1) x += sy[b];
          w->buf[j] = x;
        }
        for (uint32_t s = 0; s < S; ++s)
          for (uint32_t u = 0; u < U; ++u) bmt[s * U + u] += w->buf[u];
      }
      bm += tsz;
      par += k->out_size;
      sy += k->in_size;
    }
  }
  /* forwardUpdate, :117-139 with :237-274 */
  {
    double* fm = w->fm;
    fm[0] = 0;
    for (uint32_t s = 1; s < S; ++s) fm[s] = NINF;
    for (uint32_t t = 0; t + 1 < T; ++t) {
      const double* a = fm + t * S;
      double* an = fm + (t + 1) * S;
      const double* bm = w->bm + t * tsz;
      if (alg == 0) {
        double* bufm = w->buf;
        double* mx = w->buf + S * U;
        for (uint32_t s = 0; s < S; ++s) mx[s] = NINF;
        for (uint32_t s = 0; s < S; ++s)
          for (uint32_t u = 0; u < U; ++u) {
            bufm[s * U + u] = a[s] + bm[s * U + u];
            mx[k->next[s * U + u]] = smax(bufm[s * U + u], mx[k->next[s * U + u]]);
          }
        for (uint32_t s = 0; s < S; ++s) an[s] = 0;
        for (uint32_t s = 0; s < S; ++s)
          for (uint32_t u = 0; u < U; ++u) {
            const uint32_t nx = k->next[s * U + u];
            bufm[s * U + u] = ls_prior2(bufm[s * U + u], mx[nx]);
            an[nx] = bufm[s * U + u] + an[nx];
          }
        for (uint32_t s = 0; s < S; ++s) an[s] = ls_post2(an[s], mx[s]);
      } else {
        for (uint32_t s = 0; s < S; ++s) an[s] = NINF;
        for (uint32_t s = 0; s < S; ++s)
          for (uint32_t u = 0; u < U; ++u) {
            double* ref = &an[k->next[s * U + u]];
            *ref = ls_sum(alg, *ref, a[s] + bm[s * U + u]);
          }
      }
      double m = NINF;
      for (uint32_t s = 0; s < S; ++s) m = smax(an[s], m);
      for (uint32_t s = 0; s < S; ++s) an[s] -= m;
    }
  }
  /* backwardUpdate, :141-172 with :276-329 */
  {
    double* b = w->bwm + (T - 1) * S;
    if (k->termination == 0) {
      b[0] = 0;
      for (uint32_t s = 1; s < S; ++s) b[s] = NINF;
    } else {
      for (uint32_t s = 0; s < S; ++s) b[s] = 0.0;
    }
    for (int64_t t = (int64_t)T - 2; t >= 0; --t) {
      double* bb = w->bwm + t * S;
      const double* bn = bb + S;
      const double* bm = w->bm + (t + 1) * tsz;
      if (alg == 0) {
        double* bufm = w->buf;
        for (uint32_t s = 0; s < S; ++s) bb[s] = 0;
        for (uint32_t s = 0; s < S; ++s) {
          double mx = NINF;
          for (uint32_t u = 0; u < U; ++u) {
            bufm[s * U + u] = bn[k->next[s * U + u]] + bm[s * U + u];
            mx = smax(bufm[s * U + u], mx);
          }
          for (uint32_t u = 0; u < U; ++u) {
            bufm[s * U + u] = ls_prior2(bufm[s * U + u], mx);
            bb[s] = bufm[s * U + u] + bb[s];
          }
          bb[s] = ls_post2(bb[s], mx);
        }
      } else {
        for (uint32_t s = 0; s < S; ++s) {
          bb[s] = NINF;
          for (uint32_t u = 0; u < U; ++u) bb[s] = ls_sum(alg, bb[s], bn[k->next[s * U + u]] + bm[s * U + u]);
        }
      }
      double m = NINF;
      for (uint32_t s = 0; s < S; ++s) m = smax(bb[s], m);
      for (uint32_t s = 0; s < S; ++s) bb[s] -= m;
    }
  }
  /* aPosterioriUpdate, :174-235 with msgUpdateImpl / parityUpdateImpl :331-410 */
  {
    double* so = syst;
    const double* si = syst;
    double* po = parity_out;
    const double* pi = parity_in;
    for (uint32_t i = 0; i < T; ++i) {
      double* bm = w->bm + i * tsz;
      const double* fm = w->fm + i * S;
      const double* bw = w->bwm + i * S;
      for (uint32_t s = 0; s < S; ++s)
        for (uint32_t u = 0; u < U; ++u) bm[s * U + u] = bm[s * U + u] + fm[s] + bw[k->next[s * U + u]];
      for (uint32_t j = 0; j < k->in_size; ++j) {
        double tmp;
        if (alg == 0) {
          double mx[2] = {NINF, NINF}, mt[2] = {0, 0};
          for (uint32_t s = 0; s < S; ++s)
            for (uint32_t u = 0; u < U; ++u) mx[(u >> j) & 1] = smax(bm[s * U + u], mx[(u >> j) & 1]);
          for (uint32_t s = 0; s < S; ++s)
            for (uint32_t u = 0; u < U; ++u) mt[(u >> j) & 1] = ls_prior2(bm[s * U + u], mx[(u >> j) & 1]) + mt[(u >> j) & 1];
          tmp = ls_post2(mt[1], mx[1]) - ls_post2(mt[0], mx[0]);
        } else {
          double mt[2] = {NINF, NINF};
          for (uint32_t s = 0; s < S; ++s)
            for (uint32_t u = 0; u < U; ++u) mt[(u >> j) & 1] = ls_sum(alg, mt[(u >> j) & 1], bm[s * U + u]);
          tmp = mt[1] - mt[0];
        }
        so[j] = has_syst_in ? sf * (tmp - si[j]) : sf * (tmp);
      }
      si += k->in_size;
      so += k->in_size;
      if (po) {
        for (uint32_t j = 0; j < k->out_size; ++j) {
          double tmp;
          if (alg == 0) {
            double mx[2] = {NINF, NINF}, mt[2] = {0, 0};
            for (uint32_t s = 0; s < S; ++s)
              for (uint32_t u = 0; u < U; ++u) {
                const int c = (k->out[s * U + u] >> j) & 1;
                mx[c] = smax(bm[s * U + u], mx[c]);
              }
            for (uint32_t s = 0; s < S; ++s)
              for (uint32_t u = 0; u < U; ++u) {
                const int c = (k->out[s * U + u] >> j) & 1;
                mt[c] = ls_prior2(bm[s * U + u], mx[c]) + mt[c];
              }
            tmp = ls_post2(mt[1], mx[1]) - ls_post2(mt[0], mx[0]);
          } else {
            double mt[2] = {NINF, NINF};
            for (uint32_t s = 0; s < S; ++s)
              for (uint32_t u = 0; u < U; ++u) {
                const int c = (k->out[s * U + u] >> j) & 1;
                mt[c] = ls_sum(alg, mt[c], bm[s * U + u]);
              }
            tmp = mt[1] - mt[0];
          }
          po[j] = sf * (tmp - pi[j]);
        }
        pi += k->out_size;
        po += k->out_size;
      }
    }
  }
}

/* ======================================================================== */
/* Turbo decoder: src/detail/TurboDecoder/TurboDecoderImpl.cpp              */
/* ======================================================================== */

typedef struct {
  double* pin;   /* parityIn_ */
  double* pout;  /* parityOut_ */
  double* ext;   /* extrinsic_ */
  double* extb;  /* extrinsicBuffer_ */
  map_work m;
} turbo_work;

static void turbo_work_alloc(const fo_turbo* t, turbo_work* w) {
  uint32_t maxT = 0, maxS = 0, maxU = 0, maxO = 0;
  for (uint32_t i = 0; i < t->n; ++i) {
    const constituent_t* k = &t->c[i];
    if (k->length + k->tail > maxT) maxT = k->length + k->tail;
    if (k->S > maxS) maxS = k->S;
    if (k->U > maxU) maxU = k->U;
    if ((1u << k->out_size) > maxO) maxO = 1u << k->out_size;
  }
  w->pin = (double*)calloc(t->parity, sizeof(double));
  w->pout = (double*)calloc(t->parity, sizeof(double));
  w->ext = (double*)calloc(t->state ? t->state : 1, sizeof(double));
  w->extb = (double*)calloc(t->state ? t->state : 1, sizeof(double));
  w->m.bm = (double*)malloc((size_t)maxT * maxS * maxU * sizeof(double));
  w->m.fm = (double*)malloc((size_t)maxT * maxS * sizeof(double));
  w->m.bwm = (double*)malloc((size_t)maxT * maxS * sizeof(double));
  size_t nb = maxS * (maxU + 1);
  if (maxO > nb) nb = maxO;
  if (maxU > nb) nb = maxU;
  w->m.buf = (double*)malloc(nb * sizeof(double));
}

static void turbo_work_free(turbo_work* w) {
  free(w->pin);
  free(w->pout);
  free(w->ext);
  free(w->extb);
  free(w->m.bm);
  free(w->m.fm);
  free(w->m.bwm);
  free(w->m.buf);
}

/* aPosterioriUpdate, :152-168 */
static void turbo_aposteriori(const fo_turbo* t, turbo_work* w) {
  const double* ext = w->ext;
  double* systTail = w->pout + t->msg;
  double* syst = w->pout;
  for (uint32_t j = 0; j < t->n; ++j) {
    const constituent_t* k = &t->c[j];
    for (uint32_t q = 0; q < c_msg(k); ++q) syst[k->perm[q]] += ext[q];
    ext += c_msg(k);
    for (uint32_t q = 0; q < c_syst_tail(k); ++q) systTail[q] += ext[q];
    ext += c_syst_tail(k);
    systTail += c_syst_tail(k);
  }
}

/* parallelTransferUpdate, :191-223 */
static void turbo_parallel_transfer(const fo_turbo* t, turbo_work* w) {
  double* ext = w->ext;
  double* tmp = w->extb;
  const double* systTail = w->pin + t->msg;
  double* syst = w->pout;
  memset(w->pout, 0, t->msg * sizeof(double));
  for (uint32_t j = 0; j < t->n; ++j) {
    const constituent_t* k = &t->c[j];
    for (uint32_t q = 0; q < c_msg(k); ++q) {
      tmp[q] = ext[q];
      ext[q] = syst[k->perm[q]];
      syst[k->perm[q]] += tmp[q];
    }
    ext += c_msg(k);
    tmp += c_msg(k);
    memcpy(ext, systTail, c_syst_tail(k) * sizeof(double));
    ext += c_syst_tail(k);
    systTail += c_syst_tail(k);
  }
  memcpy(w->pout, w->pin, t->msg * sizeof(double));
  for (int64_t j = (int64_t)t->n - 1; j >= 0; --j) {
    const constituent_t* k = &t->c[j];
    ext -= c_syst(k);
    tmp -= c_msg(k);
    for (uint32_t q = 0; q < c_msg(k); ++q) {
      ext[q] += syst[k->perm[q]];
      syst[k->perm[q]] += tmp[q];
    }
  }
}

/* serialTransferUpdate, :225-250 */
static void turbo_serial_transfer(const fo_turbo* t, turbo_work* w, uint32_t i) {
  double* ext = w->ext;
  const double* systTail = w->pin + t->msg;
  double* syst = w->pout;
  memcpy(w->pout, w->pin, t->msg * sizeof(double));
  for (uint32_t j = 0; j < i; ++j) {
    const constituent_t* k = &t->c[j];
    for (uint32_t q = 0; q < c_msg(k); ++q) syst[k->perm[q]] += ext[q];
    ext += c_syst(k);
    systTail += c_syst_tail(k);
  }
  double* slot = ext;
  ext += c_msg(&t->c[i]);
  memcpy(ext, systTail, c_syst_tail(&t->c[i]) * sizeof(double));
  ext += c_syst_tail(&t->c[i]);
  for (uint32_t j = i + 1; j < t->n; ++j) {
    const constituent_t* k = &t->c[j];
    for (uint32_t q = 0; q < c_msg(k); ++q) syst[k->perm[q]] += ext[q];
    ext += c_syst(k);
  }
  for (uint32_t q = 0; q < t->c[i].perm_len; ++q) slot[q] = syst[t->c[i].perm[q]];
}

typedef struct {
  const fo_turbo* t;
  int alg, scheduling;
  uint32_t iterations;
  const double* scaling;
  uint32_t srows, scols;
  const double *llr, *syst, *state;
  uint8_t* msg;
  double *msg_out, *syst_out, *parity_out, *state_out;
  int soft;
} turbo_ctx;

static double turbo_sf(const turbo_ctx* x, uint32_t i, uint32_t j) {
  if (!x->scaling) return 1.0;
  const uint32_t r = j % x->srows;
  return x->scaling[r * x->scols + (i % x->scols)];
}

/* decodeBlock, :31-72 */
static void turbo_decode_block(const turbo_ctx* x, uint64_t f, turbo_work* w) {
  const fo_turbo* t = x->t;
  memcpy(w->pin, x->llr + f * t->parity, t->parity * sizeof(double));
  memset(w->ext, 0, t->state * sizeof(double));
  for (uint32_t i = 0; i < x->iterations; ++i) {
    if (x->scheduling == 1) turbo_parallel_transfer(t, w);
    const double* par = w->pin + t->syst;
    double* ext = w->ext;
    for (uint32_t j = 0; j < t->n; ++j) {
      if (x->scheduling == 0) turbo_serial_transfer(t, w, j);
      map_decode(&t->c[j], x->alg, turbo_sf(x, i, j), par, ext, 1, NULL, &w->m);
      ext += c_syst(&t->c[j]);
      par += c_parity(&t->c[j]);
    }
  }
  memcpy(w->pout, w->pin, t->msg * sizeof(double));
  turbo_aposteriori(t, w);
  for (uint64_t q = 0; q < t->msg; ++q) x->msg[f * t->msg + q] = w->pout[q] > 0;
}

/* soDecodeBlock, :75-150 (the constituents keep their scaling of 1.0) */
static void turbo_so_decode_block(const turbo_ctx* x, uint64_t f, turbo_work* w) {
  const fo_turbo* t = x->t;
  memcpy(w->pin, x->llr + f * t->parity, t->parity * sizeof(double));
  if (x->syst)
    for (uint64_t q = 0; q < t->syst; ++q) w->pin[q] += x->syst[f * t->syst + q];
  if (x->state) memcpy(w->ext, x->state + f * t->state, t->state * sizeof(double));
  else memset(w->ext, 0, t->state * sizeof(double));
  if (x->iterations == 0 && x->parity_out)
    for (uint64_t q = t->syst; q < t->parity; ++q) w->pout[q] = 0;
  for (uint32_t i = 0; i < x->iterations; ++i) {
    if (x->scheduling == 1) turbo_parallel_transfer(t, w);
    const double* par = w->pin + t->syst;
    double* pout = w->pout + t->syst;
    double* ext = w->ext;
    for (uint32_t j = 0; j < t->n; ++j) {
      if (x->scheduling == 0) turbo_serial_transfer(t, w, j);
      const int want_parity = (i == x->iterations - 1) && x->parity_out;
      map_decode(&t->c[j], x->alg, 1.0, par, ext, 1, want_parity ? pout : NULL, &w->m);
      ext += c_syst(&t->c[j]);
      par += c_parity(&t->c[j]);
      pout += c_parity(&t->c[j]);
    }
  }
  memset(w->pout, 0, t->syst * sizeof(double));
  turbo_aposteriori(t, w);
  if (x->syst_out) memcpy(x->syst_out + f * t->syst, w->pout, t->syst * sizeof(double));
  if (x->parity_out) memcpy(x->parity_out + f * t->parity, w->pout, t->parity * sizeof(double));
  if (x->state_out) memcpy(x->state_out + f * t->state, w->ext, t->state * sizeof(double));
  if (x->msg_out)
    for (uint64_t q = 0; q < t->msg; ++q) x->msg_out[f * t->msg + q] = w->pin[q] + w->pout[q];
}

static void* turbo_alloc(void* ctx) {
  turbo_work* w = (turbo_work*)malloc(sizeof(turbo_work));
  turbo_work_alloc(((turbo_ctx*)ctx)->t, w);
  return w;
}
static void turbo_release(void* w) {
  turbo_work_free((turbo_work*)w);
  free(w);
}
static void turbo_frame(void* ctx, uint64_t f, void* work) {
  turbo_ctx* x = (turbo_ctx*)ctx;
  if (x->soft) turbo_so_decode_block(x, f, (turbo_work*)work);
  else turbo_decode_block(x, f, (turbo_work*)work);
}

int fo_turbo_decode(const fo_turbo* t, int algorithm, uint32_t iterations, int scheduling, const double* scaling,
                    uint32_t scaling_rows, uint32_t scaling_cols, const double* llr, uint64_t nframes, uint8_t* msg,
                    int threads) {
  if (!t) return -1;
  pthread_once(&g_lut_once, lut_init);
  turbo_ctx x;
  memset(&x, 0, sizeof(x));
  x.t = t;
  x.alg = algorithm;
  x.scheduling = scheduling;
  x.iterations = iterations;
  x.scaling = scaling;
  x.srows = scaling_rows;
  x.scols = scaling_cols;
  x.llr = llr;
  x.msg = msg;
  run_frames(nframes, threads, turbo_frame, turbo_alloc, turbo_release, &x);
  return 0;
}

int fo_turbo_so_decode(const fo_turbo* t, int algorithm, uint32_t iterations, int scheduling, const double* parity,
                       const double* syst, const double* state, uint64_t nframes, double* msg, double* syst_out,
                       double* parity_out, double* state_out, int threads) {
  if (!t) return -1;
  pthread_once(&g_lut_once, lut_init);
  turbo_ctx x;
  memset(&x, 0, sizeof(x));
  x.t = t;
  x.alg = algorithm;
  x.scheduling = scheduling;
  x.iterations = iterations;
  x.llr = parity;
  x.syst = syst;
  x.state = state;
  x.msg_out = msg;
  x.syst_out = syst_out;
  x.parity_out = parity_out;
  x.state_out = state_out;
  x.soft = 1;
  run_frames(nframes, threads, turbo_frame, turbo_alloc, turbo_release, &x);
  return 0;
}
