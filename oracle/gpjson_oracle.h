/*
 * CPU oracle for the GpJSON structural index and JSONPath query path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product library links, loads or
 * calls this code; it exists so that tests/, the smoke check and the CPU
 * baseline leg of bench.py can check the CUDA path against a plain restatement
 * of the reference algorithm.
 *
 * Every function restates one piece of Xinyu-Li-123/15418-project and cites
 * the reference file:line it follows.  All arithmetic is integer/bit; results
 * must match bit for bit.
 *
 * Bitmap layout (shared with the reference): bit b of word w <-> byte 64*w+b,
 * LSB first, words are 64-bit.  Leveled bitmaps are level-major:
 * LB[level * W + w] with W = ceil(n / 64).
 */
#ifndef GPJSON_ORACLE_H
#define GPJSON_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Number of 64-bit words covering n bytes: ceil(n / 64). */
uint64_t orc_num_words(uint64_t n);

/* Newline index: out[0] = 0, out[k] = offset of the k-th '\n'.  Writes at most
 * cap entries and returns the number of lines (= newline count + 1). */
uint64_t orc_newline_index(const uint8_t *in, uint64_t n, int64_t *out,
                           uint64_t cap);

/* Escape bitmap E with the word-local carry rule of the SHAREMEM builder. */
void orc_escape_index(const uint8_t *in, uint64_t n, uint64_t *E);

/* Quote bitmap Q = '"' & ~E (bits >= n are 0). */
void orc_quote_index(const uint8_t *in, uint64_t n, const uint64_t *E,
                     uint64_t *Q);

/* String mask S = inclusive prefix-XOR of Q over all W words. */
void orc_string_index(const uint64_t *Q, uint64_t W, uint64_t *S);

/* Leveled bitmaps LB[L*W] from the bytes and the string mask. */
void orc_leveled_bitmap_index(const uint8_t *in, uint64_t n, const uint64_t *S,
                              int num_levels, uint64_t *LB);

/* All of the above in one call.  E and Q may be NULL.  nl_cap bounds NL.
 * Returns the number of lines. */
uint64_t orc_build_index(const uint8_t *in, uint64_t n, int num_levels,
                         uint64_t *E, uint64_t *Q, uint64_t *S, uint64_t *LB,
                         int64_t *NL, uint64_t nl_cap);

/* Query interpreter: one compiled query over every record of one partition.
 * out has num_lines * num_results * 2 entries, -1 = no match.  Offsets are
 * partition-local.  LB holds num_levels levels; query level l reads bitmap
 * level l + base_level (base_level 1: the records are the elements of a
 * top-level array), and a level the index does not hold reads as empty. */
int orc_query(const uint8_t *in, uint64_t n, const int64_t *NL,
              uint64_t num_lines, const uint64_t *S, const uint64_t *LB,
              uint64_t W, int num_levels, int base_level, const uint8_t *ir,
              uint64_t ir_len, int num_results, int64_t *out);

/* orc_query that also returns status bits: ORC_STATUS_OVERFLOW when a record
 * had more results than num_results (only the extension opcodes can: a
 * recursive descent with more matches, or a "[*]" array or open slice longer
 * than its limit).  Extensions of this build, rejected by the reference's
 * compiler: 0x0A NUMBER_COMPARE (numeric filter), 0x0B DESCEND_KEY ("..name"
 * as the last step), 0x0C EXPECT_AT_MOST (element-count check of "[*]" and
 * the open slices), 0x0D EXPECT_FOLLOWING (an element of "[a:-b]" must be
 * followed by b more). */
#define ORC_STATUS_OVERFLOW 1u
/* A device assert of the reference's query kernel would fire on this input
 * (src/gpjson/query/kernels/orig/query.cu:230, 265, 276, 290, 321, 334, 370,
 * 384, 430); results are unaffected. */
#define ORC_STATUS_REF_ASSERT 2u
int orc_query_status(const uint8_t *in, uint64_t n, const int64_t *NL,
                     uint64_t num_lines, const uint64_t *S, const uint64_t *LB,
                     uint64_t W, int num_levels, int base_level, const uint8_t *ir,
                     uint64_t ir_len, int num_results, int64_t *out, uint32_t *status);

/* Reference-faithful serial escape state machine over one whole buffer with an
 * UNBOUNDED backslash-run carry (the test oracle is_escaped_quote rule of
 * tests/index/string_index_test.cpp:28-34).  Used only to show where the
 * word-local rule and the unbounded rule differ. */
void orc_escape_index_unbounded(const uint8_t *in, uint64_t n, uint64_t *E);

#ifdef __cplusplus
}
#endif

#endif /* GPJSON_ORACLE_H */
