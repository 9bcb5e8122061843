/*
 * CPU oracle for the batched alignment path (see dinara_oracle.h). TEST INFRASTRUCTURE ONLY: the
 * product library never links or calls it; tests, the smoke check and the benchmark's CPU-baseline
 * leg use it as the checker and as the timed restatement of the reference's CPU path.
 *
 * Citations are file:line inside the dinara-align reference (kokyriakidis/dinara-align).
 */
#include "dinara_oracle.h"

#include <pthread.h>
#include <stdatomic.h>
#include <stdlib.h>
#include <string.h>

#define GAP_CODE 255u

static inline int32_t max32(int32_t a, int32_t b) { return a > b ? a : b; }

/* AffineGapCosts.run, gotoh.mojo:56-59: a gap of `length` letters, nothing for none. */
static inline int32_t gap_run(int32_t open, int32_t extend, int64_t length) {
    return length == 0 ? 0 : open + (int32_t)(length - 1) * extend;
}

/* ---------------------------------------------------------------------------------------------- */
/* Gotoh over the whole matrix                                                                     */
/* ---------------------------------------------------------------------------------------------- */

typedef struct {
    int32_t *score, *deletion, *insertion;
    int64_t stride;
} layers;

/* fill_rows, gotoh.mojo:285-362 (FORWARD half, top run OPENS, RowMajor layout). The first row's
 * deletion layer is its border plus one opening, the first column's insertion layer likewise; the
 * first column's deletion layer is its border. Local borders are zero and every cell floors at zero
 * (anti_diagonals.mojo:23-73 gotoh_lanes with the local clamp). */
static int32_t fill_rows(const uint8_t *first, int64_t rows, const uint8_t *second, int64_t columns,
                         const int8_t *table, int32_t size, int32_t open, int32_t extend, int32_t mode, layers L,
                         int64_t *best_row, int64_t *best_column) {
    const int local = mode == ORACLE_LOCAL;
    const int32_t opening = open + extend;
    const int64_t stride = L.stride;
    for (int64_t c = 0; c <= columns; ++c) {
        int32_t border = local ? 0 : gap_run(open, extend, c);
        L.score[c] = border;
        L.deletion[c] = border + opening;
        L.insertion[c] = 0;
    }
    int32_t best = 0;
    int64_t brow = 0, bcol = 0;
    for (int64_t r = 1; r <= rows; ++r) {
        int32_t border = local ? 0 : gap_run(open, extend, r);
        int64_t row0 = r * stride;
        L.score[row0] = border;
        L.deletion[row0] = border;
        L.insertion[row0] = border + opening;
        const int8_t *table_row = table + (int64_t)first[r - 1] * size;
        for (int64_t c = 1; c <= columns; ++c) {
            int64_t cell = row0 + c, above = cell - stride;
            int32_t del = max32(L.score[above] + open, L.deletion[above] + extend);
            int32_t ins = max32(L.score[cell - 1] + open, L.insertion[cell - 1] + extend);
            int32_t h = max32(L.score[above - 1] + table_row[second[c - 1]], max32(del, ins));
            if (local) h = max32(h, 0);
            L.score[cell] = h;
            L.deletion[cell] = del;
            L.insertion[cell] = ins;
            /* beats(), gotoh.mojo:122-127: the first maximum in row-major order. */
            if (local && h > best) {
                best = h;
                brow = r;
                bcol = c;
            }
        }
    }
    if (best_row) *best_row = brow;
    if (best_column) *best_column = bcol;
    return best;
}

static int alloc_layers(layers *L, int64_t rows, int64_t columns) {
    int64_t cells = (rows + 1) * (columns + 1);
    L->stride = columns + 1;
    L->score = (int32_t *)malloc((size_t)cells * sizeof(int32_t));
    L->deletion = (int32_t *)malloc((size_t)cells * sizeof(int32_t));
    L->insertion = (int32_t *)malloc((size_t)cells * sizeof(int32_t));
    return L->score && L->deletion && L->insertion;
}

static void free_layers(layers *L) {
    free(L->score);
    free(L->deletion);
    free(L->insertion);
}

int32_t oracle_gotoh_score(const uint8_t *first, int64_t rows, const uint8_t *second, int64_t columns,
                           const int8_t *table, int32_t size, int32_t open, int32_t extend, int32_t mode,
                           int64_t *end_row, int64_t *end_column) {
    if (end_row) *end_row = 0;
    if (end_column) *end_column = 0;
    /* swept_score, scoring.mojo:450-465: against an empty side a global score is one gap, local 0. */
    if (rows == 0 || columns == 0) {
        if (mode == ORACLE_LOCAL) return 0;
        return gap_run(open, extend, rows + columns);
    }
    /* Two rolling rows suffice for a score. */
    int64_t stride = columns + 1;
    int32_t *s = (int32_t *)malloc((size_t)(2 * stride) * sizeof(int32_t));
    int32_t *d = (int32_t *)malloc((size_t)(2 * stride) * sizeof(int32_t));
    int32_t *i = (int32_t *)malloc((size_t)(2 * stride) * sizeof(int32_t));
    const int local = mode == ORACLE_LOCAL;
    const int32_t opening = open + extend;
    for (int64_t c = 0; c <= columns; ++c) {
        int32_t border = local ? 0 : gap_run(open, extend, c);
        s[c] = border;
        d[c] = border + opening;
        i[c] = 0;
    }
    int32_t best = 0;
    int64_t brow = 0, bcol = 0;
    for (int64_t r = 1; r <= rows; ++r) {
        int32_t *ps = s + ((r - 1) & 1) * stride, *pd = d + ((r - 1) & 1) * stride;
        int32_t *cs = s + (r & 1) * stride, *cd = d + (r & 1) * stride, *ci = i + (r & 1) * stride;
        int32_t border = local ? 0 : gap_run(open, extend, r);
        cs[0] = border;
        cd[0] = border;
        ci[0] = border + opening;
        const int8_t *table_row = table + (int64_t)first[r - 1] * size;
        for (int64_t c = 1; c <= columns; ++c) {
            int32_t del = max32(ps[c] + open, pd[c] + extend);
            int32_t ins = max32(cs[c - 1] + open, ci[c - 1] + extend);
            int32_t h = max32(ps[c - 1] + table_row[second[c - 1]], max32(del, ins));
            if (local) h = max32(h, 0);
            cs[c] = h;
            cd[c] = del;
            ci[c] = ins;
            if (local && h > best) {
                best = h;
                brow = r;
                bcol = c;
            }
        }
    }
    int32_t result = local ? best : s[(rows & 1) * stride + columns];
    free(s);
    free(d);
    free(i);
    if (local) {
        if (end_row) *end_row = brow;
        if (end_column) *end_column = bcol;
    }
    return result;
}

/* Decision, gotoh.mojo:130-170: low two bits the source (0 aligning, 1 deleting, 2 inserting, 3 a
 * local path's start), bit 2 the deletion extends a run, bit 3 the insertion does. */
enum { ALIGNING = 0, DELETING = 1, INSERTING = 2, ENDS = 3 };

/* decide, gotoh.mojo:173-186. A run extends only where extending scores strictly more than opening. */
static inline unsigned decide(int local, int32_t cell_score, int32_t cell_deletion, int32_t aligned,
                              int32_t above_score, int32_t above_deletion, int32_t left_score,
                              int32_t left_insertion, int32_t open, int32_t extend) {
    unsigned deletion_extends = above_deletion + extend > above_score + open;
    unsigned insertion_extends = left_insertion + extend > left_score + open;
    unsigned source;
    if (local && cell_score <= 0)
        source = ENDS;
    else if (cell_score == aligned)
        source = ALIGNING;
    else if (cell_score == cell_deletion)
        source = DELETING;
    else
        source = INSERTING;
    return source | (deletion_extends << 2) | (insertion_extends << 3);
}

int32_t oracle_gotoh_align(const uint8_t *first, int64_t rows, const uint8_t *second, int64_t columns,
                           const int8_t *table, int32_t size, int32_t open, int32_t extend, int32_t mode,
                           uint8_t *top, uint8_t *bottom, int64_t *length) {
    const int local = mode == ORACLE_LOCAL;
    layers L;
    if (!alloc_layers(&L, rows, columns)) {
        free_layers(&L);
        *length = -1;
        return 0;
    }
    int64_t brow = 0, bcol = 0;
    int32_t best = fill_rows(first, rows, second, columns, table, size, open, extend, mode, L, &brow, &bcol);
    int64_t row = local ? brow : rows, column = local ? bcol : columns;
    int32_t score = local ? best : L.score[row * L.stride + column];
    /* walk, gotoh.mojo:365-420, collecting columns last first. */
    int64_t n = 0;
    unsigned layer = ALIGNING;
    const int64_t stride = L.stride;
    while (row > 0 && column > 0) {
        int64_t here = row * stride + column;
        int32_t pair = table[(int64_t)first[row - 1] * size + second[column - 1]];
        unsigned decision = decide(local, L.score[here], L.deletion[here], L.score[here - stride - 1] + pair,
                                   L.score[here - stride], L.deletion[here - stride], L.score[here - 1],
                                   L.insertion[here - 1], open, extend);
        if (local && layer == ALIGNING && (decision & 3) == ENDS) break;
        /* advance, gotoh.mojo:189-200: from the aligning layer follow the source, taking the gap's
         * first step at once. */
        unsigned moving = layer == ALIGNING ? (decision & 3) : layer;
        if (moving == DELETING) {
            top[n] = first[row - 1];
            bottom[n] = GAP_CODE;
            row -= 1;
            layer = (decision >> 2) & 1 ? DELETING : ALIGNING;
        } else if (moving == INSERTING) {
            top[n] = GAP_CODE;
            bottom[n] = second[column - 1];
            column -= 1;
            layer = (decision >> 3) & 1 ? INSERTING : ALIGNING;
        } else {
            top[n] = first[row - 1];
            bottom[n] = second[column - 1];
            row -= 1;
            column -= 1;
            layer = ALIGNING;
        }
        ++n;
    }
    /* reconstruct, gotoh.mojo:440-447: a global walk's rest is gaps against the letters left. */
    if (!local) {
        for (; row > 0; --row, ++n) {
            top[n] = first[row - 1];
            bottom[n] = GAP_CODE;
        }
        for (; column > 0; --column, ++n) {
            top[n] = GAP_CODE;
            bottom[n] = second[column - 1];
        }
    }
    for (int64_t a = 0, b = n - 1; a < b; ++a, --b) {
        uint8_t t = top[a];
        top[a] = top[b];
        top[b] = t;
        t = bottom[a];
        bottom[a] = bottom[b];
        bottom[b] = t;
    }
    *length = n;
    free_layers(&L);
    return score;
}

int64_t oracle_cigar(const uint8_t *top, const uint8_t *bottom, int64_t length, int32_t eqx, char *cigar) {
    int64_t out = 0;
    char run = 0;
    int64_t count = 0;
    for (int64_t k = 0; k <= length; ++k) {
        char op = 0;
        if (k < length) {
            if (top[k] == GAP_CODE)
                op = 'I';
            else if (bottom[k] == GAP_CODE)
                op = 'D';
            else if (eqx)
                op = top[k] == bottom[k] ? '=' : 'X';
            else
                op = 'M';
        }
        if (op == run) {
            ++count;
            continue;
        }
        if (count > 0) {
            char digits[24];
            int nd = 0;
            for (int64_t v = count; v > 0; v /= 10) digits[nd++] = (char)('0' + v % 10);
            while (nd > 0) cigar[out++] = digits[--nd];
            cigar[out++] = run;
        }
        run = op;
        count = 1;
    }
    cigar[out] = 0;
    return out;
}

/* ---------------------------------------------------------------------------------------------- */
/* Unit-cost edit distance                                                                         */
/* ---------------------------------------------------------------------------------------------- */

int64_t oracle_edit_distance_dp(const uint8_t *a, int64_t n, const uint8_t *b, int64_t m) {
    int64_t *row = (int64_t *)malloc((size_t)(m + 1) * sizeof(int64_t));
    for (int64_t j = 0; j <= m; ++j) row[j] = j;
    for (int64_t i = 1; i <= n; ++i) {
        int64_t previous = row[0];
        row[0] = i;
        for (int64_t j = 1; j <= m; ++j) {
            int64_t v = row[j] + 1;
            if (row[j - 1] + 1 < v) v = row[j - 1] + 1;
            int64_t diag = previous + (a[i - 1] != b[j - 1]);
            if (diag < v) v = diag;
            previous = row[j];
            row[j] = v;
        }
    }
    int64_t result = row[m];
    free(row);
    return result;
}

/* Match vectors of a pattern: for each byte value a row of `words` words, one bit a pattern letter
 * (device_edit.mojo:176-207 fill_pair, with the byte itself as the symbol). */
static uint64_t *pattern_planes(const uint8_t *pattern, int64_t n, int64_t words, int16_t codes[256], int *count) {
    int k = 0;
    for (int v = 0; v < 256; ++v) codes[v] = -1;
    for (int64_t i = 0; i < n; ++i)
        if (codes[pattern[i]] < 0) codes[pattern[i]] = (int16_t)k++;
    uint64_t *planes = (uint64_t *)calloc((size_t)(k + 1) * (size_t)words, sizeof(uint64_t));
    for (int64_t i = 0; i < n; ++i) planes[(int64_t)codes[pattern[i]] * words + i / 64] |= 1ull << (i % 64);
    *count = k;
    return planes;
}

/* The Myers/Hyyro step of one word, device_edit.mojo:56-75, returning the step out of its bottom
 * (bit `bit`) and updating the word's vertical vectors. `carry` is the step into its top. */
static inline int myers_word(uint64_t equal, uint64_t *positive, uint64_t *negative, int carry, int bit) {
    uint64_t vertical_plus = *positive, vertical_minus = *negative;
    uint64_t carry_negative = carry < 0 ? 1u : 0u, carry_positive = carry > 0 ? 1u : 0u;
    uint64_t crossing = equal | vertical_minus;
    equal |= carry_negative;
    uint64_t horizontal = (((equal & vertical_plus) + vertical_plus) ^ vertical_plus) | equal;
    uint64_t plus = vertical_minus | ~(horizontal | vertical_plus);
    uint64_t minus = vertical_plus & horizontal;
    int out = (int)((plus >> bit) & 1) - (int)((minus >> bit) & 1);
    plus = (plus << 1) | carry_positive;
    minus = (minus << 1) | carry_negative;
    *positive = minus | ~(crossing | plus);
    *negative = plus & crossing;
    return out;
}

int64_t oracle_myers_distance(const uint8_t *a, int64_t n, const uint8_t *b, int64_t m) {
    /* api.mojo:1286-1294: an empty side costs the other's letters; the shorter side is the pattern. */
    if (n == 0 || m == 0) return n > m ? n : m;
    const uint8_t *pattern = a, *text = b;
    int64_t plen = n, tlen = m;
    if (m <= n) {
        pattern = b;
        text = a;
        plen = m;
        tlen = n;
    }
    int64_t words = (plen + 63) / 64;
    int16_t codes[256];
    int count;
    uint64_t *planes = pattern_planes(pattern, plen, words, codes, &count);
    uint64_t *positive = (uint64_t *)malloc((size_t)words * sizeof(uint64_t));
    uint64_t *negative = (uint64_t *)calloc((size_t)words, sizeof(uint64_t));
    for (int64_t w = 0; w < words; ++w) positive[w] = ~0ull;
    int last_bit = (int)((plen - 1) % 64);
    int64_t score = plen;
    for (int64_t j = 0; j < tlen; ++j) {
        int code = codes[text[j]] < 0 ? count : codes[text[j]];
        const uint64_t *row = planes + (int64_t)code * words;
        int carry = 1;
        for (int64_t w = 0; w < words; ++w)
            carry = myers_word(row[w], &positive[w], &negative[w], carry, w == words - 1 ? last_bit : 63);
        score += carry;
    }
    free(planes);
    free(positive);
    free(negative);
    return score;
}

/* One round of the banded sweep: every cell of diagonal d (column less row) with
 * |d| + |d - delta| <= t lies inside the words swept, cells outside them stand for real paths (a
 * straight run down from the band's last word, or along the row above its first), so every value is
 * the cost of some alignment and a result within t is exact. */
static int64_t banded_round_impl(const uint8_t *pattern, int64_t n, const uint8_t *text, int64_t m, int64_t t,
                                 const uint64_t *planes, const int16_t codes[256], int count, uint64_t *positive,
                                 uint64_t *negative, int64_t *swept) {
    (void)pattern; /* its letters reach the sweep through `planes` */
    const int64_t delta = m - n;
    if (t < delta) t = delta;
    const int64_t e = (t - delta) / 2;
    const int64_t words = (n + 63) / 64;
    const int last_bit = (int)((n - 1) % 64);
    int64_t top = 0;      /* first word of the band */
    int64_t computed = -1; /* last word holding a state */
    int64_t above = 0;    /* value of row 64 * top at the current column */
    int64_t total = 0;
    for (int64_t c = 1; c <= m; ++c) {
        int64_t rlo = c - delta - e, rhi = c + e;
        if (rlo < 1) rlo = 1;
        if (rhi > n) rhi = n;
        int64_t wlo = (rlo - 1) / 64, whi = (rhi - 1) / 64;
        while (top < wlo) {
            if (top <= computed)
                above += __builtin_popcountll(positive[top]) - __builtin_popcountll(negative[top]);
            else
                above += 64;
            ++top;
        }
        for (int64_t w = computed + 1; w <= whi; ++w) {
            positive[w] = ~0ull;
            negative[w] = 0;
        }
        if (whi > computed) computed = whi;
        int code = codes[text[c - 1]] < 0 ? count : codes[text[c - 1]];
        const uint64_t *row = planes + (int64_t)code * words;
        int carry = 1;
        for (int64_t w = top; w <= whi; ++w)
            carry = myers_word(row[w], &positive[w], &negative[w], carry, w == words - 1 ? last_bit : 63);
        total += whi - top + 1;
        above += 1;
    }
    int64_t result = above;
    for (int64_t w = top; w < words; ++w) {
        uint64_t mask = w == words - 1 && last_bit < 63 ? ((1ull << (last_bit + 1)) - 1) : ~0ull;
        result += __builtin_popcountll(positive[w] & mask) - __builtin_popcountll(negative[w] & mask);
    }
    if (swept) *swept += total;
    return result;
}

static int64_t band_doubling_impl(const uint8_t *a, int64_t n, const uint8_t *b, int64_t m, int64_t start,
                                  int64_t only_round, int64_t *rounds, int64_t *words_swept) {
    if (rounds) *rounds = 0;
    if (words_swept) *words_swept = 0;
    if (n == 0 || m == 0) return n > m ? n : m;
    const uint8_t *pattern = a, *text = b;
    int64_t plen = n, tlen = m;
    if (m < n) {
        pattern = b;
        text = a;
        plen = m;
        tlen = n;
    }
    int64_t words = (plen + 63) / 64;
    int16_t codes[256];
    int count;
    uint64_t *planes = pattern_planes(pattern, plen, words, codes, &count);
    uint64_t *positive = (uint64_t *)malloc((size_t)words * sizeof(uint64_t));
    uint64_t *negative = (uint64_t *)malloc((size_t)words * sizeof(uint64_t));
    int64_t delta = tlen - plen;
    int64_t t = start < delta ? delta : start;
    int64_t result, best = INT64_MAX;
    for (;;) {
        if (rounds) *rounds += 1;
        result = banded_round_impl(pattern, plen, text, tlen, t, planes, codes, count, positive, negative,
                                   words_swept);
        if (only_round || result <= t) break;
        /* band.mojo:619-657: the next bound doubles the last, capped by the cheapest alignment a round has
         * found so far (a round's result is a real alignment's cost); past the whole matrix any band is
         * exact. */
        if (t >= plen + tlen) break;
        if (result < best) best = result;
        t = t > 0 ? 2 * t : 1;
        if (best < t) t = best;
    }
    free(planes);
    free(positive);
    free(negative);
    return result;
}

int64_t oracle_band_doubling(const uint8_t *a, int64_t n, const uint8_t *b, int64_t m, int64_t start,
                             int64_t *rounds, int64_t *words) {
    return band_doubling_impl(a, n, b, m, start, 0, rounds, words);
}

int64_t oracle_banded_round(const uint8_t *a, int64_t n, const uint8_t *b, int64_t m, int64_t t, int64_t *words) {
    return band_doubling_impl(a, n, b, m, t, 1, NULL, words);
}

int32_t oracle_score_reach_refuses(const int8_t *table, int32_t size, int32_t open, int32_t extend, int64_t rows,
                                   int64_t columns, int32_t mode) {
    /* ScoreReach.of / check, scoring.mojo:228-249. */
    int32_t hi = -128, lo = 127;
    for (int32_t k = 0; k < size * size; ++k) {
        if (table[k] > hi) hi = table[k];
        if (table[k] < lo) lo = table[k];
    }
    int64_t opening = 2 * -(int64_t)open;
    int64_t step = hi > -lo ? hi : -lo;
    if (-(int64_t)extend > step) step = -(int64_t)extend;
    int64_t letters = mode == ORACLE_LOCAL ? (rows < columns ? rows : columns) : rows + columns;
    return opening + 2 * (letters + 2) * step >= (1ll << 28);
}

/* ---------------------------------------------------------------------------------------------- */
/* Batches on host threads, longest pair first                                                     */
/* ---------------------------------------------------------------------------------------------- */

typedef struct {
    int64_t pairs;
    const uint8_t *tape;
    const int64_t *offsets;
    const int8_t *table;
    int32_t size, open, extend, mode, eqx;
    int64_t start;
    int kind; /* 0 scores, 1 alignments, 2 distances */
    int32_t *scores;
    char *cigars;
    int64_t cigar_stride;
    int64_t *cigar_lengths;
    int64_t *distances;
    const int64_t *order;
    atomic_llong next;
} batch_job;

static void run_pair(batch_job *job, int64_t p) {
    const uint8_t *first = job->tape + job->offsets[2 * p];
    const uint8_t *second = job->tape + job->offsets[2 * p + 1];
    int64_t rows = job->offsets[2 * p + 1] - job->offsets[2 * p];
    int64_t columns = job->offsets[2 * p + 2] - job->offsets[2 * p + 1];
    if (job->kind == 0) {
        job->scores[p] = oracle_gotoh_score(first, rows, second, columns, job->table, job->size, job->open,
                                            job->extend, job->mode, NULL, NULL);
    } else if (job->kind == 1) {
        uint8_t *top = (uint8_t *)malloc((size_t)(rows + columns + 1));
        uint8_t *bottom = (uint8_t *)malloc((size_t)(rows + columns + 1));
        int64_t length = 0;
        job->scores[p] = oracle_gotoh_align(first, rows, second, columns, job->table, job->size, job->open,
                                            job->extend, job->mode, top, bottom, &length);
        char *cigar = (char *)malloc((size_t)(2 * length + 2));
        int64_t written = oracle_cigar(top, bottom, length, job->eqx, cigar);
        char *slot = job->cigars + p * job->cigar_stride;
        if (written < job->cigar_stride) {
            memcpy(slot, cigar, (size_t)written + 1);
            job->cigar_lengths[p] = written;
        } else {
            memcpy(slot, cigar, (size_t)job->cigar_stride - 1);
            slot[job->cigar_stride - 1] = 0;
            job->cigar_lengths[p] = -1;
        }
        free(cigar);
        free(top);
        free(bottom);
    } else {
        job->distances[p] = job->start < 0 ? oracle_myers_distance(first, rows, second, columns)
                                           : oracle_band_doubling(first, rows, second, columns, job->start, NULL,
                                                                  NULL);
    }
}

static void *batch_worker(void *argument) {
    batch_job *job = (batch_job *)argument;
    for (;;) {
        long long k = atomic_fetch_add(&job->next, 1);
        if (k >= job->pairs) break;
        run_pair(job, job->order[k]);
    }
    return NULL;
}

static const int64_t *batch_offsets_for_sort;
static int by_cells_descending(const void *x, const void *y) {
    int64_t a = *(const int64_t *)x, b = *(const int64_t *)y;
    const int64_t *o = batch_offsets_for_sort;
    int64_t ca = (o[2 * a + 1] - o[2 * a] + 1) * (o[2 * a + 2] - o[2 * a + 1] + 1);
    int64_t cb = (o[2 * b + 1] - o[2 * b] + 1) * (o[2 * b + 2] - o[2 * b + 1] + 1);
    if (ca != cb) return ca > cb ? -1 : 1;
    return a < b ? -1 : (a > b);
}

static pthread_mutex_t sort_lock = PTHREAD_MUTEX_INITIALIZER;

static void run_batch(batch_job *job, int32_t threads) {
    int64_t *order = (int64_t *)malloc((size_t)(job->pairs > 0 ? job->pairs : 1) * sizeof(int64_t));
    for (int64_t p = 0; p < job->pairs; ++p) order[p] = p;
    pthread_mutex_lock(&sort_lock);
    batch_offsets_for_sort = job->offsets;
    qsort(order, (size_t)job->pairs, sizeof(int64_t), by_cells_descending);
    pthread_mutex_unlock(&sort_lock);
    job->order = order;
    atomic_init(&job->next, 0);
    if (threads <= 1) {
        batch_worker(job);
    } else {
        pthread_t *pool = (pthread_t *)malloc((size_t)threads * sizeof(pthread_t));
        for (int32_t k = 0; k < threads; ++k) pthread_create(&pool[k], NULL, batch_worker, job);
        for (int32_t k = 0; k < threads; ++k) pthread_join(pool[k], NULL);
        free(pool);
    }
    free(order);
}

void oracle_batch_scores(int64_t pairs, const uint8_t *tape, const int64_t *offsets, const int8_t *table,
                         int32_t size, int32_t open, int32_t extend, int32_t mode, int32_t threads, int32_t *results) {
    batch_job job;
    memset(&job, 0, sizeof job);
    job.pairs = pairs;
    job.tape = tape;
    job.offsets = offsets;
    job.table = table;
    job.size = size;
    job.open = open;
    job.extend = extend;
    job.mode = mode;
    job.kind = 0;
    job.scores = results;
    run_batch(&job, threads);
}

void oracle_batch_alignments(int64_t pairs, const uint8_t *tape, const int64_t *offsets, const int8_t *table,
                             int32_t size, int32_t open, int32_t extend, int32_t mode, int32_t eqx, int32_t threads,
                             int32_t *results, char *cigars, int64_t cigar_stride, int64_t *cigar_lengths) {
    batch_job job;
    memset(&job, 0, sizeof job);
    job.pairs = pairs;
    job.tape = tape;
    job.offsets = offsets;
    job.table = table;
    job.size = size;
    job.open = open;
    job.extend = extend;
    job.mode = mode;
    job.eqx = eqx;
    job.kind = 1;
    job.scores = results;
    job.cigars = cigars;
    job.cigar_stride = cigar_stride;
    job.cigar_lengths = cigar_lengths;
    run_batch(&job, threads);
}

void oracle_batch_distances(int64_t pairs, const uint8_t *tape, const int64_t *offsets, int64_t start,
                            int32_t threads, int64_t *results) {
    batch_job job;
    memset(&job, 0, sizeof job);
    job.pairs = pairs;
    job.tape = tape;
    job.offsets = offsets;
    job.start = start;
    job.kind = 2;
    job.distances = results;
    run_batch(&job, threads);
}
