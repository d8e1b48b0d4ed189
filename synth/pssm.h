/*
 * synth — PSSM construction for the synthetic workloads (host only, no GPU).
 *
 * Builds int8 PSSM rows from family MSAs, following the reference's host code
 * so that synthetic workloads and golden fixtures use the same inputs as the
 * reference would.  Built into synth/libsynth.so, an input generator for the
 * tests and the benchmark; the product library does not contain it.
 */
#ifndef SYNTH_PSSM_H
#define SYNTH_PSSM_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Profile::from_numeric_msa (src/profile.rs:90-185) with compute_sequence_weights
 * (:219-255), compute_neff (:258-301), the substitution-matrix pseudocounts
 * (:146-166) and compute_log_pssm (:322-341), in the reference's f32 operation
 * order.  msa: n_rows x query_len residue codes (0..19 amino acids, 20 = X,
 * 0xFF = gap), row 0 = the query.  r: 20x20 pseudocount matrix R[a][b] = P(a|b)
 * as f32 (SubstitutionMatrix::r, src/matrix.rs:144-150); p_back: 21 background
 * frequencies (f64, SubstitutionMatrix::p_back).  Outputs pssm (query_len x 20
 * int8) and neff (query_len f32, may be NULL).  Returns 0, or -1 on empty input. */
int st_pssm_from_msa(const uint8_t* msa, uint32_t n_rows, uint32_t query_len, const float* r, const double* p_back,
                     float pca, float pcb, float score_bias, int8_t* pssm, float* neff);

/* Batch form over many MSAs (OpenMP over MSAs): MSA k has n_rows[k] rows of
 * query_len[k] codes starting at msa + msa_off[k]; its PSSM is written at
 * pssm + pssm_off[k] (query_len[k] x 20). */
int st_pssm_batch(const uint8_t* msa, const uint64_t* msa_off, const uint32_t* n_rows, const uint32_t* query_len,
                  uint32_t n_msas, const float* r, const double* p_back, float pca, float pcb, float score_bias,
                  int8_t* pssm, const uint64_t* pssm_off, int nthreads);

#ifdef __cplusplus
}
#endif
#endif
