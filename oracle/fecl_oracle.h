/*
 * Test infrastructure, not product code: a CPU restatement of FeCl's decode path in
 * plain C, FP64, in the reference's operation order, so that its outputs equal the
 * reference's bit for bit.  Only tests/, the smoke check and bench.py's CPU baseline
 * use it, and only as the checker.
 *
 * Every function cites the reference lines it restates (paths relative to the
 * reference repository).
 */
#ifndef FECL_ORACLE_H
#define FECL_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- LDPC ---------------------------------------------------------------- */

typedef struct fo_ldpc fo_ldpc;

/* detail::Ldpc::Structure(EncoderOptions(H)) -- src/detail/Ldpc.cpp:34-55, with the
 * generator transform of :216-331.  H: CSR, rows = checks, columns sorted. */
fo_ldpc* fo_ldpc_create(uint32_t rows, uint32_t cols, const uint32_t* row_ptr, const uint32_t* col_idx);
void fo_ldpc_destroy(fo_ldpc* c);
/* msg, parity (= N), state (= edges), max check degree */
void fo_ldpc_sizes(const fo_ldpc* c, uint64_t* msg, uint64_t* parity, uint64_t* state, uint32_t* max_degree);
/* the transformed matrix: row_ptr[rows+1], col_idx[state] */
void fo_ldpc_checks(const fo_ldpc* c, uint32_t* row_ptr, uint32_t* col_idx);
/* Ldpc::Structure::encode / check -- src/detail/Ldpc.cpp:160-209 */
void fo_ldpc_encode(const fo_ldpc* c, const uint8_t* msg, uint8_t* parity);
int fo_ldpc_check(const fo_ldpc* c, const uint8_t* parity);

/* BpDecoderImpl::decodeBlock / soDecodeBlock -- src/detail/BpDecoder/BpDecoderImpl.cpp:37-130.
 * algorithm: 0 Exact, 1 Linear, 2 Approximate.  scaling: [n_scaling][max_degree-1].
 * Frames are decoded independently, split over `threads` POSIX threads. */
int fo_ldpc_decode(const fo_ldpc* c, int algorithm, uint32_t iterations, const double* scaling, uint32_t n_scaling,
                   const double* llr, uint64_t nframes, uint8_t* msg, int32_t* iterations_run, int threads);
int fo_ldpc_so_decode(const fo_ldpc* c, int algorithm, uint32_t iterations, const double* scaling,
                      uint32_t n_scaling, const double* parity, const double* syst, const double* state,
                      uint64_t nframes, double* msg, double* syst_out, double* parity_out, double* state_out,
                      int threads);

/* Standard DVB-S2 matrix from the address tables (ETSI EN 302 307 5.3.2); call with
 * row_ptr == NULL for the sizes.  Returns 0, or -1 for an unknown (n, rate). */
int fo_dvbs2_matrix(uint32_t n, uint32_t rate_num, uint32_t rate_den, uint32_t* rows, uint32_t* cols,
                    uint64_t* nnz, uint32_t* row_ptr, uint32_t* col_idx);

/* ---- trellis / turbo ----------------------------------------------------- */

/* Trellis(constraintLengths, generator, feedback) -- src/Trellis.cpp:76-143.
 * generators[i * noutputs + k]; feedback may be NULL.  Returns -1 on invalid input. */
int fo_trellis(uint32_t ninputs, const uint32_t* constraint_lengths, uint32_t noutputs, const uint64_t* generators,
               const uint64_t* feedback, uint32_t* state_count, uint32_t* input_count, uint32_t* next_state,
               uint32_t* output);

/* Turbo::Lte3Gpp::interleaver -- src/Lte3Gpp.cpp:219-237. Returns -1 for an unknown K. */
int fo_lte_interleaver(uint32_t K, uint32_t* perm);

typedef struct fo_turbo fo_turbo;

/* detail::Turbo::Structure -- src/detail/Turbo.cpp:45-103.  Trellises given as
 * tables (state_count, input_count, output_size, next_state, output); n_trellis
 * and n_termination are 1 or n; perm_len[i] == 0 means the identity. */
fo_turbo* fo_turbo_create(uint32_t n, const uint32_t* state_count, const uint32_t* input_count,
                          const uint32_t* output_size, const uint32_t* const* next_state,
                          const uint32_t* const* output, uint32_t n_trellis, const uint32_t* perm_data,
                          const uint32_t* perm_len, const int32_t* termination, uint32_t n_termination);
void fo_turbo_destroy(fo_turbo* c);
void fo_turbo_sizes(const fo_turbo* c, uint64_t* msg, uint64_t* syst, uint64_t* parity, uint64_t* state);
/* Turbo::Structure::encode -- src/detail/Turbo.cpp:155-170 */
void fo_turbo_encode(const fo_turbo* c, const uint8_t* msg, uint8_t* parity);

/* TurboDecoderImpl::decodeBlock / soDecodeBlock -- src/detail/TurboDecoder/TurboDecoderImpl.cpp:31-150.
 * scheduling: 0 Serial, 1 Parallel.  scaling: [scaling_rows][scaling_cols] as
 * Turbo::Structure::scalingFactor (src/detail/Turbo.cpp:148-153), NULL = 1.0. */
int fo_turbo_decode(const fo_turbo* c, int algorithm, uint32_t iterations, int scheduling, const double* scaling,
                    uint32_t scaling_rows, uint32_t scaling_cols, const double* llr, uint64_t nframes, uint8_t* msg,
                    int threads);
int fo_turbo_so_decode(const fo_turbo* c, int algorithm, uint32_t iterations, int scheduling, const double* parity,
                       const double* syst, const double* state, uint64_t nframes, double* msg, double* syst_out,
                       double* parity_out, double* state_out, int threads);

#ifdef __cplusplus
}
#endif

#endif
