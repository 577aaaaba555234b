/*
 * Test infrastructure, not product code.
 *
 * A C-ABI shim over the reference FeCl library compiled from its own sources
 * (see oracle/Makefile).  It exposes the reference's public C++ API -- the
 * fec::Codec decode/soDecode/encode/check templates (src/Codec.h:68-82), the
 * fec::Ldpc and fec::Turbo constructors (src/Ldpc.h:82-84, src/Turbo.h:99-101),
 * Ldpc::Gallager::matrix (src/Ldpc.cpp:77-102), Turbo::Lte3Gpp::interleaver
 * (src/Lte3Gpp.cpp:219-237) and the transformed check matrix that the BP decoder
 * iterates over (detail::Ldpc::Structure::checks, src/detail/Ldpc.h:110) -- as
 * plain functions with pointers and sizes, so that the Python test-suite can run
 * the reference decoder on exactly the LLRs that the CUDA path sees.
 *
 * Only tests/, the smoke check and bench.py's CPU baseline load this library.
 */
#include <cstdint>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "Convolutional.h"
#include "Ldpc.h"
#include "Turbo.h"
#include "Trellis.h"

namespace {

thread_local std::string g_last_error;

struct RefCodec {
  std::unique_ptr<fec::Codec> codec;
  std::unique_ptr<fec::detail::Ldpc::Structure> ldpc;    // set for LDPC codecs
  std::unique_ptr<fec::detail::Turbo::Structure> turbo;  // set for turbo codecs
  std::unique_ptr<fec::detail::Convolutional::Structure> conv;  // set for convolutional codecs
};

template <class F>
int guarded(F f) {
  try {
    f();
    return 0;
  } catch (std::exception& e) {
    g_last_error = e.what();
  } catch (...) {
    g_last_error = "unknown exception";
  }
  return -1;
}

fec::SparseBitMatrix csr_to_matrix(size_t rows, size_t cols, const uint32_t* rowptr, const uint32_t* colidx) {
  std::vector<size_t> sizes(rows);
  for (size_t r = 0; r < rows; ++r) sizes[r] = rowptr[r + 1] - rowptr[r];
  fec::SparseBitMatrix H(sizes, cols);
  for (size_t r = 0; r < rows; ++r) {
    auto row = H[r];
    for (uint32_t e = rowptr[r]; e < rowptr[r + 1]; ++e) row.set(colidx[e]);
  }
  return H;
}

void matrix_to_csr(const fec::SparseBitMatrix& H, uint32_t* rowptr, uint32_t* colidx) {
  size_t e = 0;
  size_t r = 0;
  rowptr[0] = 0;
  for (auto row = H.begin(); row < H.end(); ++row, ++r) {
    for (auto it = row->begin(); it < row->end(); ++it) colidx[e++] = uint32_t(*it);
    rowptr[r + 1] = uint32_t(e);
  }
}

fec::DecoderAlgorithm to_alg(int a) {
  switch (a) {
    case 0: return fec::Exact;
    case 1: return fec::Linear;
    default: return fec::Approximate;
  }
}

std::vector<fec::BitField<size_t>> to_bits(const uint8_t* p, size_t n) {
  std::vector<fec::BitField<size_t>> v(n);
  for (size_t i = 0; i < n; ++i) v[i] = p[i] ? 1 : 0;
  return v;
}

}  // namespace

extern "C" {

const char* fref_last_error() { return g_last_error.c_str(); }

/* Gallager matrix: call once with rowptr == nullptr to obtain rows/nnz. */
int fref_gallager(size_t n, size_t wc, size_t wr, uint64_t seed, size_t* rows, size_t* nnz,
                  uint32_t* rowptr, uint32_t* colidx) {
  return guarded([&] {
    auto H = fec::Ldpc::Gallager::matrix(n, wc, wr, seed);
    *rows = H.rows();
    *nnz = H.size();
    if (rowptr) matrix_to_csr(H, rowptr, colidx);
  });
}

/* The reference's own DVB-S2 builder.  Only (64800, 1/2) is safe to call: other
 * (n, rate) pairs build a wrong matrix or corrupt the heap (src/DvbS2.cpp:1619-1644). */
int fref_dvbs2_builtin(size_t n, double rate, size_t* rows, size_t* cols, size_t* nnz,
                       uint32_t* rowptr, uint32_t* colidx) {
  return guarded([&] {
    if (!(n == 64800 && rate == 0.5)) throw std::invalid_argument("only (64800, 1/2) is safe");
    auto H = fec::Ldpc::DvbS2::matrix(n, rate);
    *rows = H.rows();
    *cols = H.cols();
    *nnz = H.size();
    if (rowptr) matrix_to_csr(H, rowptr, colidx);
  });
}

int fref_ldpc_create(size_t rows, size_t cols, const uint32_t* rowptr, const uint32_t* colidx,
                     int algorithm, size_t iterations, const double* scaling, size_t nscaling,
                     int workgroup, void** out) {
  return guarded([&] {
    auto H = csr_to_matrix(rows, cols, rowptr, colidx);
    auto dec = fec::Ldpc::DecoderOptions().algorithm(to_alg(algorithm)).iterations(iterations);
    if (nscaling == 1) {
      dec.scalingFactor(scaling[0]);
    } else if (nscaling > 1) {
      std::unordered_map<size_t, std::vector<double>> m;
      m[0] = std::vector<double>(scaling, scaling + nscaling);
      dec.scalingFactor(m);
    }
    auto rc = new RefCodec;
    rc->ldpc.reset(new fec::detail::Ldpc::Structure(fec::Ldpc::EncoderOptions(H), dec));
    rc->codec.reset(new fec::Ldpc(*rc->ldpc, workgroup));
    *out = rc;
  });
}

/* The transformed check matrix H_ the decoder iterates over (row order = state layout). */
int fref_ldpc_checks(void* h, size_t* rows, size_t* cols, size_t* nnz, uint32_t* rowptr, uint32_t* colidx) {
  return guarded([&] {
    auto rc = static_cast<RefCodec*>(h);
    if (!rc->ldpc) throw std::invalid_argument("not an LDPC codec");
    const auto& H = rc->ldpc->checks();
    *rows = H.rows();
    *cols = H.cols();
    *nnz = H.size();
    if (rowptr) matrix_to_csr(H, rowptr, colidx);
  });
}

struct fref_trellis {
  size_t ninputs;
  const size_t* constraint_lengths; /* [ninputs] */
  size_t noutputs;
  const uint64_t* generators;       /* [ninputs * noutputs], octal values already decoded */
  const uint64_t* feedback;         /* [ninputs] or NULL */
};

static fec::Trellis make_trellis(const fref_trellis& t) {
  std::vector<size_t> cl(t.constraint_lengths, t.constraint_lengths + t.ninputs);
  std::vector<std::vector<fec::BitField<size_t>>> gen(t.ninputs);
  for (size_t i = 0; i < t.ninputs; ++i)
    for (size_t k = 0; k < t.noutputs; ++k) gen[i].push_back(t.generators[i * t.noutputs + k]);
  std::vector<fec::BitField<size_t>> fb;
  if (t.feedback)
    for (size_t i = 0; i < t.ninputs; ++i) fb.push_back(t.feedback[i]);
  return fec::Trellis(cl, gen, fb);
}

/* Trellis tables next_state[s * inputCount + u], output[s * inputCount + u]. */
int fref_trellis_tables(const fref_trellis* t, size_t* state_count, size_t* input_count, size_t* output_size,
                        uint32_t* next_state, uint32_t* output) {
  return guarded([&] {
    auto tr = make_trellis(*t);
    *state_count = tr.stateCount();
    *input_count = tr.inputCount();
    *output_size = tr.outputSize();
    if (next_state) {
      for (size_t s = 0; s < tr.stateCount(); ++s)
        for (size_t u = 0; u < tr.inputCount(); ++u) {
          next_state[s * tr.inputCount() + u] = uint32_t(size_t(tr.getNextState(s, u)));
          output[s * tr.inputCount() + u] = uint32_t(size_t(tr.getOutput(s, u)));
        }
    }
  });
}

int fref_lte_interleaver(size_t K, uint32_t* perm) {
  return guarded([&] {
    auto p = fec::Turbo::Lte3Gpp::interleaver(K);
    for (size_t i = 0; i < p.outputSize(); ++i) perm[i] = uint32_t(p[i]);
  });
}

/* termination: 0 = Tail, 1 = Truncate.  scheduling: 0 Serial, 1 Parallel.
 * scaling: [nscaling_rows][nscaling_cols] row-major (rows = constituents or 1). */
int fref_turbo_create(size_t nconst, const fref_trellis* trellis, size_t ntrellis, const uint32_t* perm_data,
                      const size_t* perm_len, int termination, int algorithm, int scheduling, size_t iterations,
                      const double* scaling, size_t nscaling_rows, size_t nscaling_cols, int workgroup, void** out) {
  return guarded([&] {
    std::vector<fec::Trellis> trs;
    for (size_t i = 0; i < ntrellis; ++i) trs.push_back(make_trellis(trellis[i]));
    std::vector<fec::Permutation> perms;
    size_t off = 0;
    for (size_t i = 0; i < nconst; ++i) {
      std::vector<size_t> seq(perm_data + off, perm_data + off + perm_len[i]);
      perms.push_back(fec::Permutation(seq));
      off += perm_len[i];
    }
    auto enc = fec::Turbo::EncoderOptions(trs, perms)
                   .termination(termination == 0 ? fec::Trellis::Tail : fec::Trellis::Truncate);
    auto dec = fec::Turbo::DecoderOptions()
                   .algorithm(to_alg(algorithm))
                   .iterations(iterations)
                   .scheduling(scheduling == 0 ? fec::Serial : fec::Parallel);
    if (nscaling_rows > 0) {
      std::vector<std::vector<double>> sf(nscaling_rows);
      for (size_t i = 0; i < nscaling_rows; ++i)
        sf[i].assign(scaling + i * nscaling_cols, scaling + (i + 1) * nscaling_cols);
      dec.scalingFactor(sf);
    }
    auto rc = new RefCodec;
    rc->turbo.reset(new fec::detail::Turbo::Structure(enc, dec));
    rc->codec.reset(new fec::Turbo(*rc->turbo, workgroup));
    *out = rc;
  });
}

// Ldpc::Structure::puncturing (src/detail/Ldpc.cpp:333-353): the kept code-bit
// indices and the permutation's input size.  Call with seq == NULL for the length.
int fref_ldpc_puncturing(void* h, const uint8_t* mask, size_t mask_len, const uint8_t* syst_mask, size_t syst_len,
                         uint32_t* seq, size_t* seq_len, size_t* input_size) {
  return guarded([&] {
    auto rc = static_cast<RefCodec*>(h);
    fec::Ldpc::PunctureOptions o;
    o.mask(std::vector<bool>(mask, mask + mask_len));
    o.systMask(std::vector<bool>(syst_mask, syst_mask + syst_len));
    const fec::Permutation p = rc->ldpc->puncturing(o);
    *seq_len = p.outputSize();
    *input_size = p.inputSize();
    if (seq)
      for (size_t i = 0; i < p.outputSize(); ++i) seq[i] = uint32_t(p[i]);
  });
}

// Turbo::Structure::puncturing (src/detail/Turbo.cpp:200-320); masks are given as
// concatenated bytes with one length per mask, ordering 0 = Alternate, 1 = Group.
int fref_turbo_puncturing(void* h, const uint8_t* mask_data, const size_t* mask_len, size_t n_masks,
                          const uint8_t* tail_data, const size_t* tail_len, size_t n_tail, int ordering, uint32_t* seq,
                          size_t* seq_len, size_t* input_size) {
  return guarded([&] {
    auto rc = static_cast<RefCodec*>(h);
    std::vector<std::vector<bool>> m(n_masks), t(n_tail);
    size_t off = 0;
    for (size_t i = 0; i < n_masks; ++i) {
      m[i].assign(mask_data + off, mask_data + off + mask_len[i]);
      off += mask_len[i];
    }
    off = 0;
    for (size_t i = 0; i < n_tail; ++i) {
      t[i].assign(tail_data + off, tail_data + off + tail_len[i]);
      off += tail_len[i];
    }
    fec::Turbo::PunctureOptions o;
    o.mask(m).tailMask(t).bitOrdering(ordering == 0 ? fec::Turbo::BitOrdering::Alternate : fec::Turbo::BitOrdering::Group);
    const fec::Permutation p = rc->turbo->puncturing(o);
    *seq_len = p.outputSize();
    *input_size = p.inputSize();
    if (seq)
      for (size_t i = 0; i < p.outputSize(); ++i) seq[i] = uint32_t(p[i]);
  });
}

// fec::Convolutional(EncoderOptions(trellis, length).termination(t),
// DecoderOptions().algorithm(a).scalingFactor(sf)) -- src/Convolutional.h:51.
int fref_conv_create(const fref_trellis* trellis, size_t length, int termination, int algorithm, double scaling,
                     int workgroup, void** out) {
  return guarded([&] {
    auto enc = fec::Convolutional::EncoderOptions(make_trellis(*trellis), length)
                   .termination(termination == 0 ? fec::Trellis::Tail : fec::Trellis::Truncate);
    auto dec = fec::Convolutional::DecoderOptions().algorithm(to_alg(algorithm)).scalingFactor(scaling);
    auto rc = new RefCodec;
    rc->conv.reset(new fec::detail::Convolutional::Structure(enc, dec));
    rc->codec.reset(new fec::Convolutional(*rc->conv, workgroup));
    *out = rc;
  });
}

// Convolutional::Structure::puncturing (src/detail/Convolutional.cpp:223-242).
int fref_conv_puncturing(void* h, const uint8_t* mask, size_t mask_len, const uint8_t* tail_mask, size_t tail_len,
                         uint32_t* seq, size_t* seq_len, size_t* input_size) {
  return guarded([&] {
    auto rc = static_cast<RefCodec*>(h);
    fec::Convolutional::PunctureOptions o;
    o.mask(std::vector<bool>(mask, mask + mask_len)).tailMask(std::vector<bool>(tail_mask, tail_mask + tail_len));
    const fec::Permutation p = rc->conv->puncturing(o);
    *seq_len = p.outputSize();
    *input_size = p.inputSize();
    if (seq)
      for (size_t i = 0; i < p.outputSize(); ++i) seq[i] = uint32_t(p[i]);
  });
}

// Sets a custom schedule (Turbo::DecoderOptions::scheduling(Scheduling), which also
// selects Custom scheduling) on a turbo codec made by fref_turbo_create; the layout
// of the arrays is fecl_turbo_options'.
int fref_turbo_set_schedule(void* h, int algorithm, size_t iterations, const double* scaling, size_t nscaling_rows,
                            size_t nscaling_cols, size_t n_stages, const uint32_t* stage_counts, const uint32_t* activation,
                            const uint32_t* transfer_counts, const uint32_t* transfer) {
  return guarded([&] {
    auto rc = static_cast<RefCodec*>(h);
    fec::Turbo::Scheduling sched(n_stages);
    size_t a = 0, t = 0;
    for (size_t s = 0; s < n_stages; ++s)
      for (uint32_t k = 0; k < stage_counts[s]; ++k, ++a) {
        sched[s].activation.push_back(activation[a]);
        sched[s].transfer.emplace_back(transfer + t, transfer + t + transfer_counts[a]);
        t += transfer_counts[a];
      }
    auto dec = fec::Turbo::DecoderOptions().algorithm(to_alg(algorithm)).iterations(iterations).scheduling(sched);
    if (nscaling_rows > 0) {
      std::vector<std::vector<double>> sf(nscaling_rows);
      for (size_t i = 0; i < nscaling_rows; ++i)
        sf[i].assign(scaling + i * nscaling_cols, scaling + (i + 1) * nscaling_cols);
      dec.scalingFactor(sf);
    }
    static_cast<fec::Turbo*>(rc->codec.get())->setDecoderOptions(dec);
  });
}

void fref_codec_destroy(void* h) { delete static_cast<RefCodec*>(h); }

int fref_codec_sizes(void* h, size_t* out4) {
  return guarded([&] {
    auto c = static_cast<RefCodec*>(h)->codec.get();
    out4[0] = c->msgSize();
    out4[1] = c->systSize();
    out4[2] = c->paritySize();
    out4[3] = c->stateSize();
  });
}

int fref_codec_set_workgroup(void* h, int n) {
  return guarded([&] { static_cast<RefCodec*>(h)->codec->setWorkGroupSize(n); });
}

int fref_codec_encode(void* h, const uint8_t* msg, size_t nframes, uint8_t* parity) {
  return guarded([&] {
    auto c = static_cast<RefCodec*>(h)->codec.get();
    auto m = to_bits(msg, nframes * c->msgSize());
    std::vector<fec::BitField<size_t>> p;
    c->encode(m, p);
    for (size_t i = 0; i < p.size(); ++i) parity[i] = uint8_t(size_t(p[i]) & 1);
  });
}

/* Returns 1 when every frame is a codeword, 0 otherwise, -1 on error. */
int fref_codec_check(void* h, const uint8_t* parity, size_t nframes) {
  int result = -1;
  int rc = guarded([&] {
    auto c = static_cast<RefCodec*>(h)->codec.get();
    auto p = to_bits(parity, nframes * c->paritySize());
    result = c->check(p) ? 1 : 0;
  });
  return rc == 0 ? result : -1;
}

int fref_codec_decode(void* h, const double* llr, size_t nframes, uint8_t* msg) {
  return guarded([&] {
    auto c = static_cast<RefCodec*>(h)->codec.get();
    std::vector<double> in(llr, llr + nframes * c->paritySize());
    std::vector<fec::BitField<size_t>> m;
    c->decode(in, m);
    for (size_t i = 0; i < m.size(); ++i) msg[i] = uint8_t(size_t(m[i]) & 1);
  });
}

/* Any of syst/state inputs and msg/syst/parity/state outputs may be NULL. */
int fref_codec_so_decode(void* h, size_t nframes, const double* parity, const double* syst, const double* state,
                         double* msg_out, double* syst_out, double* parity_out, double* state_out) {
  return guarded([&] {
    auto c = static_cast<RefCodec*>(h)->codec.get();
    std::vector<double> p(parity, parity + nframes * c->paritySize());
    std::vector<double> s, st, mo, so, po, sto;
    auto in = fec::Codec::Input<>().parity(p);
    if (syst) {
      s.assign(syst, syst + nframes * c->systSize());
      in.syst(s);
    }
    if (state) {
      st.assign(state, state + nframes * c->stateSize());
      in.state(st);
    }
    auto out = fec::Codec::Output<>();
    if (msg_out) out.msg(mo);
    if (syst_out) out.syst(so);
    if (parity_out) out.parity(po);
    if (state_out) out.state(sto);
    c->soDecode(in, out);
    if (msg_out) std::memcpy(msg_out, mo.data(), mo.size() * sizeof(double));
    if (syst_out) std::memcpy(syst_out, so.data(), so.size() * sizeof(double));
    if (parity_out) std::memcpy(parity_out, po.data(), po.size() * sizeof(double));
    if (state_out) std::memcpy(state_out, sto.data(), sto.size() * sizeof(double));
  });
}

}  // extern "C"
