/* Test infrastructure only: plain-C CPU restatement of the reference's PUSCH receive-path
 * stages, used by tests/ as the checker for the CUDA path. It is never linked into the
 * product. Parity of this restatement is pinned against the reference's own compiled code
 * (oracle/_ref/libocudu_ref.so) and the golden fixtures under tests/golden/.
 */
#ifndef PUSCH_ORACLE_H
#define PUSCH_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* CRC polynomials, same numbering as the product C ABI. */
enum { PGO_CRC16 = 0, PGO_CRC24A = 1, PGO_CRC24B = 2, PGO_CRC24C = 3, PGO_CRC11 = 4, PGO_CRC6 = 5 };

/* CRC of nbits bits packed MSB first, init 0, no final XOR. */
uint32_t pgo_crc(int poly, const uint8_t* packed, int nbits);

/* Lifted shift of edge e (row-major edge order) of base graph bg for lifting size Z. */
int pgo_ldpc_edge_shift(int bg, int Z, int edge);

/* Layered normalised min-sum decode of one codeblock with the reference's int8 arithmetic.
 * Returns the number of iterations on CRC success, 0 otherwise. out_packed holds K*Z hard bits
 * (packed MSB first) on return; it is set to all ones when the input carries fewer than K*Z
 * soft bits. crc_poly < 0 selects the no-early-stop mode (syndrome check after the last
 * iteration). */
int pgo_ldpc_decode(int bg, int Z, int nof_filler_bits, int crc_poly, int max_iterations, const int8_t* llrs,
                    int nof_llrs, uint8_t* out_packed);

/* LDPC rate dematching of E LLRs into the N-LLR buffer `out` (read first when new_data == 0). */
void pgo_rate_dematch(int bg, int Z, int rv, int qm, int Nref, int nof_filler_bits, int new_data, const int8_t* in,
                      int E, int8_t* out);

/* Soft demapping (modulation order 2, 4, 6, 8) with the arithmetic of the reference's AVX2
 * kernels: max-log LLR times 1/noise, scaled to +-120, round half to even. symbols are
 * interleaved (re, im) floats. */
void pgo_demodulate_soft(int qm, const float* symbols, const float* noise_vars, int nof_symbols, int8_t* llrs);

/* Saturating LLR sum with the reference's special cases. */
int8_t pgo_llr_sum(int8_t a, int8_t b);

#ifdef __cplusplus
}
#endif

#endif
