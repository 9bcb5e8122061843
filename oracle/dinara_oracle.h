/*
 * CPU oracle for the batched alignment path: a plain-C restatement of dinara-align's own CPU
 * algorithms for the Gotoh scoring path and the unit-cost edit distance.
 *
 * TEST INFRASTRUCTURE ONLY. Nothing in the product library links, loads or calls this code; it is
 * the checker that parity tests, the package's smoke check and the benchmark's CPU-baseline leg run
 * beside the GPU path. Every function cites the reference file:line whose behaviour it restates.
 *
 * Conventions shared with the reference (dinara_align/scoring.mojo:127-215, gotoh.mojo:40-60):
 *   - `first` is the reference, read down the rows; `second` is the query, read across the columns.
 *   - letters are codes 0..size-1 into a row-major `size`x`size` int8 table.
 *   - gaps are in the kernels' terms: `open` scores a gap's first letter, `extend` each further one
 *     (a Scoring's opening o and extension e give open = o + e, extend = e).
 */
#ifndef DINARA_ORACLE_H
#define DINARA_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORACLE_GLOBAL 0
#define ORACLE_LOCAL 1

/* Best score of one pair over the whole matrix (gotoh.mojo:285-362 fill_rows; scoring.mojo:450-465
 * swept_score for empty sides). For LOCAL, the end cell (first maximum in row-major order, the
 * `beats` rule of gotoh.mojo:122-127) is written to *end_row / *end_column (0, 0 when the best is 0). */
/* The best score with up to the given letters at each end of each sequence unaligned for nothing
 * (scored.mojo:69-240 with gap_affine.mojo:421-447 EndsFree). */
int32_t oracle_gotoh_score_free(const uint8_t *first, int64_t rows, const uint8_t *second, int64_t columns,
                                const int8_t *table, int32_t size, int32_t open, int32_t extend,
                                int64_t reference_start, int64_t reference_end, int64_t query_start,
                                int64_t query_end);
/* The same score and where it ends (*end_row reference letters, *end_column query letters): of equal best
 * ends the one furthest along the reference less the query with `highest`, the least so without
 * (scored.mojo:69-100, 155-176). */
int32_t oracle_gotoh_end_free(const uint8_t *first, int64_t rows, const uint8_t *second, int64_t columns,
                              const int8_t *table, int32_t size, int32_t open, int32_t extend,
                              int64_t reference_start, int64_t reference_end, int64_t query_start,
                              int64_t query_end, int32_t highest, int64_t *end_row, int64_t *end_column);
/* An extension's best score from the origin and where it stops (scored.mojo:69-100, 272-300 FROM_ORIGIN):
 * the best cell above zero, of equal ones the furthest along both together, then along the reference;
 * (0, 0) scoring 0 when none is above zero. */
int32_t oracle_gotoh_extension(const uint8_t *first, int64_t rows, const uint8_t *second, int64_t columns,
                               const int8_t *table, int32_t size, int32_t open, int32_t extend, int64_t *end_row,
                               int64_t *end_column);
/* The same with a Z-drop of `zdrop` (and `slack`, the cheapest a gap grows a letter, a diagonal between two
 * bests), its anti-diagonals read in order (scored.mojo:272-300); *dropped set when the sweep ended early. */
int32_t oracle_gotoh_extension_zdrop(const uint8_t *first, int64_t rows, const uint8_t *second, int64_t columns,
                                     const int8_t *table, int32_t size, int32_t open, int32_t extend, int64_t zdrop,
                                     int64_t slack, int64_t *end_row, int64_t *end_column, int32_t *dropped);
int32_t oracle_gotoh_score(const uint8_t *first, int64_t rows, const uint8_t *second, int64_t columns,
                           const int8_t *table, int32_t size, int32_t open, int32_t extend, int32_t mode,
                           int64_t *end_row, int64_t *end_column);

/* An optimal alignment by the full-matrix walk (gotoh.mojo:365-510 walk/reconstruct/serial_align with
 * decide/advance :130-193). Writes the two gapped rows, as codes with 255 for a gap, reversed into
 * forward order, into `top`/`bottom` (each with room for rows + columns), their length to *length,
 * and returns the score. For LOCAL the walk starts at the best cell and stops where decide() says the
 * path starts; *first_used / *second_used give the letters each row spans. */
int32_t oracle_gotoh_align(const uint8_t *first, int64_t rows, const uint8_t *second, int64_t columns,
                           const int8_t *table, int32_t size, int32_t open, int32_t extend, int32_t mode,
                           uint8_t *top, uint8_t *bottom, int64_t *length);

/* The CIGAR of two gapped rows (gotoh.mojo:203-220 GappedAlignment.cigar): '=' / 'X' or 'M', 'D' a
 * letter of the first alone, 'I' one of the second. Returns the CIGAR's length (no NUL counted);
 * `cigar` needs room for 2 * length + 1 bytes. */
int64_t oracle_cigar(const uint8_t *top, const uint8_t *bottom, int64_t length, int32_t eqx, char *cigar);

/* Unit-cost edit distance by the plain full dynamic program (tests/test_python.py:16-23). */
int64_t oracle_edit_distance_dp(const uint8_t *a, int64_t n, const uint8_t *b, int64_t m);

/* Unit-cost global edit distance by Myers/Hyyro bit-vectors over the whole matrix, the shorter side
 * the pattern, exactly as device_edit.mojo:29-77 (myers_kernel) steps it, for any pattern length. */
int64_t oracle_myers_distance(const uint8_t *a, int64_t n, const uint8_t *b, int64_t m);

/* Plain band doubling (band.mojo:526-657 in its untrusted form, without seeds or checkpoints): a
 * Ukkonen band for threshold t (every path costing at most t lies inside it) is swept with block
 * bit-vectors; a result within t is the distance, else t doubles. Starts at `start` (raised to the
 * length difference). Writes rounds taken and 64-row words swept to *rounds / *words (may be NULL). */
int64_t oracle_band_doubling(const uint8_t *a, int64_t n, const uint8_t *b, int64_t m, int64_t start,
                             int64_t *rounds, int64_t *words);

/* One band round (threshold t) of the above: the banded distance, which is exact when <= t. */
int64_t oracle_banded_round(const uint8_t *a, int64_t n, const uint8_t *b, int64_t m, int64_t t, int64_t *words);

/* Whether a pair's scores could pass 2^28, which the reference refuses (scoring.mojo:218-249
 * ScoreReach): 1 refused, 0 accepted. `mode` ORACLE_LOCAL floors the cells at zero. */
int32_t oracle_score_reach_refuses(const int8_t *table, int32_t size, int32_t open, int32_t extend, int64_t rows,
                                   int64_t columns, int32_t mode);

/*
 * Batches on the host over `threads` threads, longest pair first (api.mojo:1009-1083), each pair on
 * one thread start to finish. Pair p's first sequence is tape[offsets[2p] .. offsets[2p+1]) and its
 * second tape[offsets[2p+1] .. offsets[2p+2]) (scoring.mojo:267-340 PairTape).
 */
void oracle_batch_scores(int64_t pairs, const uint8_t *tape, const int64_t *offsets, const int8_t *table,
                         int32_t size, int32_t open, int32_t extend, int32_t mode, int32_t threads, int32_t *results);

/* Batch alignments: score into results[p], CIGAR into cigars + p * cigar_stride (NUL-terminated; a
 * CIGAR longer than the stride is cut short and its length reported as -1). */
void oracle_batch_alignments(int64_t pairs, const uint8_t *tape, const int64_t *offsets, const int8_t *table,
                             int32_t size, int32_t open, int32_t extend, int32_t mode, int32_t eqx, int32_t threads,
                             int32_t *results, char *cigars, int64_t cigar_stride, int64_t *cigar_lengths);

/* Batch unit-cost distances by plain band doubling from `start` (or the whole matrix by Myers for a
 * negative start). */
void oracle_batch_distances(int64_t pairs, const uint8_t *tape, const int64_t *offsets, int64_t start,
                            int32_t threads, int64_t *results);


/*
 * CIGARs under Costs, by the Ties rule (modes.mojo:402-426). `first` is the reference, its letters the
 * columns; a 'D' is one of its letters alone, an 'I' one of the second's. `right` nonzero is Ties.RIGHT
 * (one search from the start traced back from the corner, WFA2-lib's); zero is Ties.LEFT (the same over
 * both sequences reversed, read forward). `cigar` needs 2 * (n + m) + 2 bytes; NUL-terminated.
 */

/* Unit costs with no cap (edit_distance.mojo:265-330 edit_cigar): the distance, or -2 for no room. */
int64_t oracle_edit_cigar(const uint8_t *first, int64_t n, const uint8_t *second, int64_t m, int32_t right,
                          int32_t eqx, char *cigar, int64_t capacity);

/* One-piece gap-affine costs, or unit costs under a cap (api.mojo:622-716 least_costly -> cigar_within,
 * the wavefront of gap_affine.mojo): a gap of k first-sequence letters costs deletion_opening +
 * k * deletion_extension, of the second's insertion_opening + k * insertion_extension. The cost, or -4
 * when it passes `max_cost` (negative for none), or -2 for no room. */
int64_t oracle_affine_cigar(const uint8_t *first, int64_t n, const uint8_t *second, int64_t m, int64_t mismatch,
                            int64_t deletion_opening, int64_t deletion_extension, int64_t insertion_opening,
                            int64_t insertion_extension, int64_t max_cost, int32_t right, int32_t eqx, char *cigar,
                            int64_t capacity);

/* Batch costs under one-piece gap-affine Costs by the wavefront, the reference's host path for a global
 * alignment under a uniform Scoring (scoring.mojo:414-440 global_on_host -> gap_affine.mojo's wavefront),
 * threaded as the batches above. Each pair's cost into costs[p] and, with `cigars` non-null, its Ties.RIGHT
 * CIGAR into cigars + p * cigar_stride (its length into cigar_lengths[p], -1 when it did not fit). */
void oracle_batch_wavefront(int64_t pairs, const uint8_t *tape, const int64_t *offsets, int64_t mismatch,
                            int64_t deletion_opening, int64_t deletion_extension, int64_t insertion_opening,
                            int64_t insertion_extension, int32_t eqx, int32_t threads, int64_t *costs, char *cigars,
                            int64_t cigar_stride, int64_t *cigar_lengths);

#ifdef __cplusplus
}
#endif

#endif
