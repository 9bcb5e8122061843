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

/* Free ends, scored.mojo:69-240 (swept_cells, FROM_EDGE) with the letters gap_affine.mojo:421-447 EndsFree
 * allows: the first row's cell `c` query letters in scores edge(c, query_start) and the first column's
 * `r` reference letters in edge(r, reference_start), where edge is nothing within the free letters and a
 * gap from where they end past them; the score is the best end on the last row within `query_end` letters
 * of the last column, or on the last column within `reference_end` letters of the last row. Against an
 * empty side the alignment runs along the other's edge and ends within its free letters. Counts past a
 * sequence's length read as its length. */
static inline int32_t free_edge(int64_t letters, int64_t free_letters, int32_t open, int32_t extend) {
    return letters <= free_letters ? 0 : gap_run(open, extend, letters - free_letters);
}

/* An end of `value` at (r, c) against the best so far (scored.mojo:69-100 swept_cells' rule for ends from
 * the edges): higher, or as high and further along the reference less the query with `highest` (the
 * least so without). Each diagonal meets the last row and the last column at most once between them, so
 * no two ends tie on both. */
static inline void offer_end(int32_t value, int64_t r, int64_t c, int highest, int32_t *best, int64_t *best_row,
                             int64_t *best_column) {
    const int64_t key = r - c, best_key = *best_row - *best_column;
    if (value > *best || (value == *best && (highest ? key > best_key : key < best_key))) {
        *best = value;
        *best_row = r;
        *best_column = c;
    }
}

int32_t oracle_gotoh_end_free(const uint8_t *first, int64_t rows, const uint8_t *second, int64_t columns,
                              const int8_t *table, int32_t size, int32_t open, int32_t extend,
                              int64_t reference_start, int64_t reference_end, int64_t query_start,
                              int64_t query_end, int32_t highest, int64_t *end_row, int64_t *end_column) {
    const int64_t rs = reference_start < rows ? reference_start : rows;
    const int64_t re = reference_end < rows ? reference_end : rows;
    const int64_t qs = query_start < columns ? query_start : columns;
    const int64_t qe = query_end < columns ? query_end : columns;
    if (rows == 0 || columns == 0) {
        /* scored.mojo:155-176: along the other's edge, every end within its free letters at the end in
         * turn; of equal ones the later when the run goes along the reference and `highest` is asked (or
         * along the query and it is not), else the earlier. */
        const int64_t length = rows + columns;
        const int along_reference = rows > 0;
        const int64_t start = along_reference ? rs : qs, finish = along_reference ? re : qe;
        int32_t top = INT32_MIN;
        int64_t reach = 0;
        for (int64_t letters = 0; letters <= length; ++letters) {
            if (length - letters > finish) continue;
            const int32_t value = free_edge(letters, start, open, extend);
            if (value > top || (value == top && along_reference == (highest != 0))) {
                top = value;
                reach = letters;
            }
        }
        *end_row = rows > 0 ? reach : 0;
        *end_column = columns > 0 ? reach : 0;
        return length == 0 ? 0 : top;
    }
    const int32_t opening = open + extend;
    const int64_t stride = columns + 1;
    int32_t *s = (int32_t *)malloc((size_t)(2 * stride) * sizeof(int32_t));
    int32_t *d = (int32_t *)malloc((size_t)(2 * stride) * sizeof(int32_t));
    int32_t *i = (int32_t *)malloc((size_t)(2 * stride) * sizeof(int32_t));
    for (int64_t c = 0; c <= columns; ++c) {
        const int32_t border = free_edge(c, qs, open, extend);
        s[c] = border;
        d[c] = border + opening;
        i[c] = 0;
    }
    int32_t best = INT32_MIN;
    *end_row = 0;
    *end_column = 0;
    /* The last column's ends: row 0 among them when every reference letter may be left at the end. */
    if (rows <= re) offer_end(s[columns], 0, columns, highest, &best, end_row, end_column);
    for (int64_t r = 1; r <= rows; ++r) {
        int32_t *ps = s + ((r - 1) & 1) * stride, *pd = d + ((r - 1) & 1) * stride;
        int32_t *cs = s + (r & 1) * stride, *cd = d + (r & 1) * stride, *ci = i + (r & 1) * stride;
        const int32_t border = free_edge(r, rs, open, extend);
        cs[0] = border;
        cd[0] = border;
        ci[0] = border + opening;
        const int8_t *table_row = table + (int64_t)first[r - 1] * size;
        for (int64_t c = 1; c <= columns; ++c) {
            int32_t del = max32(ps[c] + open, pd[c] + extend);
            int32_t ins = max32(cs[c - 1] + open, ci[c - 1] + extend);
            cs[c] = max32(ps[c - 1] + table_row[second[c - 1]], max32(del, ins));
            cd[c] = del;
            ci[c] = ins;
        }
        if (rows - r <= re) offer_end(cs[columns], r, columns, highest, &best, end_row, end_column);
    }
    /* The last row's ends, column 0 among them when every query letter may be left at the end. */
    const int32_t *last = s + (rows & 1) * stride;
    for (int64_t c = columns - qe; c <= columns; ++c) offer_end(last[c], rows, c, highest, &best, end_row, end_column);
    free(s);
    free(d);
    free(i);
    return best;
}

/* An extension's stop, scored.mojo:69-100 and 272-300 (FROM_ORIGIN): Gotoh's global recurrence from the
 * origin, its stop the best cell anywhere above zero, of equal ones the furthest along both sequences
 * together, then along the reference; none above zero stops at the origin, scoring 0. */
int32_t oracle_gotoh_extension(const uint8_t *first, int64_t rows, const uint8_t *second, int64_t columns,
                               const int8_t *table, int32_t size, int32_t open, int32_t extend, int64_t *end_row,
                               int64_t *end_column) {
    int32_t best = 0;
    *end_row = 0;
    *end_column = 0;
    if (rows == 0 || columns == 0) return 0;
    const int32_t opening = open + extend;
    const int64_t stride = columns + 1;
    int32_t *s = (int32_t *)malloc((size_t)(2 * stride) * sizeof(int32_t));
    int32_t *d = (int32_t *)malloc((size_t)(2 * stride) * sizeof(int32_t));
    int32_t *i = (int32_t *)malloc((size_t)(2 * stride) * sizeof(int32_t));
    for (int64_t c = 0; c <= columns; ++c) {
        const int32_t border = c == 0 ? 0 : gap_run(open, extend, c);
        s[c] = border;
        d[c] = border + opening;
        i[c] = 0;
    }
    for (int64_t r = 1; r <= rows; ++r) {
        int32_t *ps = s + ((r - 1) & 1) * stride, *pd = d + ((r - 1) & 1) * stride;
        int32_t *cs = s + (r & 1) * stride, *cd = d + (r & 1) * stride, *ci = i + (r & 1) * stride;
        const int32_t border = gap_run(open, extend, r);
        cs[0] = border;
        cd[0] = border;
        ci[0] = border + opening;
        const int8_t *table_row = table + (int64_t)first[r - 1] * size;
        for (int64_t c = 1; c <= columns; ++c) {
            int32_t del = max32(ps[c] + open, pd[c] + extend);
            int32_t ins = max32(cs[c - 1] + open, ci[c - 1] + extend);
            cs[c] = max32(ps[c - 1] + table_row[second[c - 1]], max32(del, ins));
            cd[c] = del;
            ci[c] = ins;
            const int64_t along = r + c, best_along = *end_row + *end_column;
            if (cs[c] > 0 && (cs[c] > best || (cs[c] == best && (along > best_along ||
                                                                  (along == best_along && r > *end_row))))) {
                best = cs[c];
                *end_row = r;
                *end_column = c;
            }
        }
    }
    free(s);
    free(d);
    free(i);
    return best;
}

/* An extension with a Z-drop, scored.mojo:272-300 (FROM_ORIGIN in one strip): the anti-diagonals
 * (row + column) in order, each's best cell (its score; of equal ones the furthest along the reference);
 * a best above zero at or above the best so far is the new stop, and a best below it ends the sweep when
 * it lies more than `zdrop` plus `slack` a diagonal between them (each's reference less query letters)
 * below it. A Z-drop leaves every cell's score as it is, so the scores come from the row sweep and the
 * anti-diagonals' bests are read after it. *dropped says whether the sweep ended early. */
int32_t oracle_gotoh_extension_zdrop(const uint8_t *first, int64_t rows, const uint8_t *second, int64_t columns,
                                     const int8_t *table, int32_t size, int32_t open, int32_t extend, int64_t zdrop,
                                     int64_t slack, int64_t *end_row, int64_t *end_column, int32_t *dropped) {
    *end_row = 0;
    *end_column = 0;
    *dropped = 0;
    if (rows == 0 || columns == 0) return 0;
    const int64_t diagonals = rows + columns + 1;
    int32_t *most = (int32_t *)malloc((size_t)diagonals * sizeof(int32_t));
    int64_t *furthest = (int64_t *)malloc((size_t)diagonals * sizeof(int64_t));
    for (int64_t d = 0; d < diagonals; ++d) {
        most[d] = INT32_MIN;
        furthest[d] = 0;
    }
    const int32_t opening = open + extend;
    const int64_t stride = columns + 1;
    int32_t *s = (int32_t *)malloc((size_t)(2 * stride) * sizeof(int32_t));
    int32_t *dl = (int32_t *)malloc((size_t)(2 * stride) * sizeof(int32_t));
    int32_t *il = (int32_t *)malloc((size_t)(2 * stride) * sizeof(int32_t));
    for (int64_t c = 0; c <= columns; ++c) {
        const int32_t border = c == 0 ? 0 : gap_run(open, extend, c);
        s[c] = border;
        dl[c] = border + opening;
        il[c] = 0;
    }
    for (int64_t r = 1; r <= rows; ++r) {
        int32_t *ps = s + ((r - 1) & 1) * stride, *pd = dl + ((r - 1) & 1) * stride;
        int32_t *cs = s + (r & 1) * stride, *cd = dl + (r & 1) * stride, *ci = il + (r & 1) * stride;
        const int32_t border = gap_run(open, extend, r);
        cs[0] = border;
        cd[0] = border;
        ci[0] = border + opening;
        const int8_t *table_row = table + (int64_t)first[r - 1] * size;
        for (int64_t c = 1; c <= columns; ++c) {
            int32_t del = max32(ps[c] + open, pd[c] + extend);
            int32_t ins = max32(cs[c - 1] + open, ci[c - 1] + extend);
            cs[c] = max32(ps[c - 1] + table_row[second[c - 1]], max32(del, ins));
            cd[c] = del;
            ci[c] = ins;
            const int64_t d = r + c;
            if (cs[c] > most[d] || (cs[c] == most[d] && r > furthest[d])) {
                most[d] = cs[c];
                furthest[d] = r;
            }
        }
    }
    int64_t best = 0, best_row = 0, best_diagonal = 0;
    for (int64_t d = 2; d <= rows + columns; ++d) {
        if (most[d] > 0 && most[d] >= best) {
            best = most[d];
            best_row = furthest[d];
            best_diagonal = d;
        } else if (most[d] < best) {
            const int64_t lean = 2 * furthest[d] - d, best_lean = 2 * best_row - best_diagonal;
            const int64_t apart = lean > best_lean ? lean - best_lean : best_lean - lean;
            if (best - most[d] > zdrop + slack * apart) {
                *dropped = 1;
                break;
            }
        }
    }
    *end_row = best_row;
    *end_column = best_diagonal - best_row;
    free(most);
    free(furthest);
    free(s);
    free(dl);
    free(il);
    return (int32_t)best;
}

int32_t oracle_gotoh_score_free(const uint8_t *first, int64_t rows, const uint8_t *second, int64_t columns,
                                const int8_t *table, int32_t size, int32_t open, int32_t extend,
                                int64_t reference_start, int64_t reference_end, int64_t query_start,
                                int64_t query_end) {
    int64_t row = 0, column = 0;
    return oracle_gotoh_end_free(first, rows, second, columns, table, size, open, extend, reference_start,
                                 reference_end, query_start, query_end, 1, &row, &column);
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
/* CIGARs under Costs, by the Ties rule                                                             */
/* ---------------------------------------------------------------------------------------------- */

/* Runs of one CIGAR letter, joined when the same letter comes again (cigar.mojo:183-200 CigarWriter). */
typedef struct {
    char *letters;
    int64_t *lengths;
    int64_t count, capacity;
} cigar_runs;

static int runs_init(cigar_runs *r, int64_t capacity) {
    r->count = 0;
    r->capacity = capacity > 4 ? capacity : 4;
    r->letters = (char *)malloc((size_t)r->capacity);
    r->lengths = (int64_t *)malloc((size_t)r->capacity * sizeof(int64_t));
    return r->letters && r->lengths;
}

static void runs_free(cigar_runs *r) {
    free(r->letters);
    free(r->lengths);
}

static void runs_add(cigar_runs *r, char letter, int64_t length) {
    if (length <= 0) return;
    if (r->count > 0 && r->letters[r->count - 1] == letter) {
        r->lengths[r->count - 1] += length;
        return;
    }
    if (r->count == r->capacity) {
        r->capacity *= 2;
        r->letters = (char *)realloc(r->letters, (size_t)r->capacity);
        r->lengths = (int64_t *)realloc(r->lengths, (size_t)r->capacity * sizeof(int64_t));
    }
    r->letters[r->count] = letter;
    r->lengths[r->count] = length;
    r->count += 1;
}

/* The runs as CIGAR text, first to last or (`backwards`) last to first; returns the text's length. */
static int64_t runs_text(const cigar_runs *r, int backwards, char *out, int64_t capacity) {
    int64_t at = 0;
    for (int64_t i = 0; i < r->count; ++i) {
        const int64_t k = backwards ? r->count - 1 - i : i;
        char digits[24];
        int d = 0;
        int64_t v = r->lengths[k];
        do {
            digits[d++] = (char)('0' + v % 10);
            v /= 10;
        } while (v > 0);
        if (at + d + 2 > capacity) return -1;
        while (d > 0) out[at++] = digits[--d];
        out[at++] = r->letters[k];
    }
    if (at + 1 > capacity) return -1;
    out[at] = 0;
    return at;
}

static uint8_t *reversed_copy(const uint8_t *s, int64_t n) {
    uint8_t *out = (uint8_t *)malloc((size_t)(n > 0 ? n : 1));
    for (int64_t i = 0; i < n; ++i) out[i] = s[n - 1 - i];
    return out;
}

/* Every cost's front on diagonals lo ..= hi (a diagonal is the first sequence's letters less the
 * second's), its columns (the first sequence's letters) from cols[0]. */
typedef struct {
    int64_t lo, hi;
    int64_t *cols;
} dt_front;

#define DT_UNREACHED (-1)

static inline int64_t dt_at(const dt_front *f, int64_t k) {
    return k < f->lo || k > f->hi ? DT_UNREACHED : f->cols[k - f->lo];
}

/* furthest_source, diagonal.mojo:286-303: the furthest column a path of one more edit reaches on
 * `diagonal` before its matches, and its last move (0 a substitution, 1 a letter of the first sequence
 * alone, 2 one of the second); ties go to a substitution, then the first sequence's letter. */
static inline int64_t dt_source(int64_t same, int64_t left, int64_t up, int64_t diagonal, int64_t columns,
                                int64_t rows, int *move) {
    int64_t best = -1;
    *move = 0;
    if (same >= 0 && same < columns && same - diagonal < rows) best = same + 1;
    if (left >= 0 && left < columns && left + 1 > best) {
        best = left + 1;
        *move = 1;
    }
    if (up >= 0 && up - diagonal - 1 < rows && up > best) {
        best = up;
        *move = 2;
    }
    return best;
}

static inline int64_t slide(const uint8_t *first, int64_t columns, const uint8_t *second, int64_t rows, int64_t column,
                            int64_t diagonal) {
    int64_t row = column - diagonal;
    while (column < columns && row < rows && first[column] == second[row]) {
        ++column;
        ++row;
    }
    return column;
}

/* The unit-cost distance and the CIGAR `edit_cigar` gives (edit_distance.mojo:265-330): the fronts of
 * diagonal transition, each cost's furthest column on each diagonal after sliding over matches, traced
 * back from the corner by `best_source` (diagonal.mojo:306-316) as diagonal_cigar writes it
 * (traceback.mojo:803-900). Ties.RIGHT traces the pair itself; Ties.LEFT (`right` zero) traces both
 * sequences reversed, whose moves back from their corner run forward over the pair. */
static int64_t dt_cigar(const uint8_t *first, int64_t columns, const uint8_t *second, int64_t rows, int backwards,
                        int eqx, cigar_runs *runs) {
    int64_t capacity = 64, count = 0;
    dt_front *fronts = (dt_front *)malloc((size_t)capacity * sizeof(dt_front));
    const int64_t target = columns - rows;
    fronts[0].lo = fronts[0].hi = 0;
    fronts[0].cols = (int64_t *)malloc(sizeof(int64_t));
    fronts[0].cols[0] = slide(first, columns, second, rows, 0, 0);
    count = 1;
    int64_t distance = 0;
    while (!(target >= fronts[distance].lo && target <= fronts[distance].hi &&
             fronts[distance].cols[target - fronts[distance].lo] >= columns)) {
        const dt_front *last = &fronts[distance];
        if (count == capacity) {
            capacity *= 2;
            fronts = (dt_front *)realloc(fronts, (size_t)capacity * sizeof(dt_front));
            last = &fronts[distance];
        }
        dt_front *next = &fronts[count];
        next->lo = last->lo - 1 > -rows ? last->lo - 1 : -rows;
        next->hi = last->hi + 1 < columns ? last->hi + 1 : columns;
        next->cols = (int64_t *)malloc((size_t)(next->hi - next->lo + 1) * sizeof(int64_t));
        for (int64_t k = next->lo; k <= next->hi; ++k) {
            int move;
            int64_t best = dt_source(dt_at(last, k), dt_at(last, k - 1), dt_at(last, k + 1), k, columns, rows, &move);
            next->cols[k - next->lo] = best < 0 ? DT_UNREACHED : slide(first, columns, second, rows, best, k);
        }
        ++count;
        ++distance;
    }
    const char matched = eqx ? '=' : 'M', substituted = eqx ? 'X' : 'M';
    int64_t diagonal = target, column = columns;
    for (int64_t score = distance; score > 0; --score) {
        const dt_front *back = &fronts[score - 1];
        int move;
        const int64_t best = dt_source(dt_at(back, diagonal), dt_at(back, diagonal - 1), dt_at(back, diagonal + 1),
                                       diagonal, columns, rows, &move);
        if (column > best) runs_add(runs, matched, column - best);
        if (move == 0) {
            runs_add(runs, substituted, 1);
            column = best - 1;
        } else if (move == 1) {
            runs_add(runs, 'D', 1);
            column = best - 1;
            diagonal -= 1;
        } else {
            runs_add(runs, 'I', 1);
            column = best;
            diagonal += 1;
        }
    }
    if (column > 0) runs_add(runs, matched, column);
    (void)backwards;
    for (int64_t s = 0; s < count; ++s) free(fronts[s].cols);
    free(fronts);
    return distance;
}

int64_t oracle_edit_cigar(const uint8_t *first, int64_t n, const uint8_t *second, int64_t m, int32_t right,
                          int32_t eqx, char *cigar, int64_t capacity) {
    cigar_runs runs;
    if (!runs_init(&runs, 2 * (n + m) + 4)) return -2;
    int64_t distance;
    int64_t written;
    if (right) {
        distance = dt_cigar(first, n, second, m, 0, eqx, &runs);
        written = runs_text(&runs, 1, cigar, capacity);
    } else {
        uint8_t *a = reversed_copy(first, n), *b = reversed_copy(second, m);
        distance = dt_cigar(a, n, b, m, 1, eqx, &runs);
        written = runs_text(&runs, 0, cigar, capacity);
        free(a);
        free(b);
    }
    runs_free(&runs);
    return written < 0 ? -2 : distance;
}

/* The gap-affine wavefront of gap_affine.mojo (one gap piece): each cost's alignment front (its
 * furthest column a diagonal, after sliding over matches), its two gap layers' fronts and the flag of
 * which source won each (gap_affine.mojo:858-1010 with `record`), over the costs divided by their common
 * factor (Penalties.scale). A letter of the first sequence against a gap (the FIRST_GAP layer, a
 * deletion, its own opening and extension) comes from the diagonal below and moves a column; one of the
 * second (SECOND_GAP, an insertion) from the diagonal above, moving a row. */
#define WF_UNREACHED ((int64_t)-(1ll << 40))
#define WF_ALIGNED 0
#define WF_FIRST 1
#define WF_SECOND 2
#define WF_OPENED_FIRST 8
#define WF_OPENED_SECOND 16

typedef struct {
    int64_t lo, hi;
    int64_t at; /* the front's first entry in the pools: aligned, first_gap, second_gap at 3 * at; flags at at */
} wf_front;

/* Every cost's fronts of one search, in pools that grow and are kept from pair to pair on a thread. */
typedef struct {
    wf_front *fronts;
    int64_t fronts_capacity;
    int64_t *values; /* three layers a diagonal */
    uint8_t *flags;
    int64_t used, capacity;
} wf_pool;

static _Thread_local wf_pool thread_pool;

static int64_t wf_reserve(wf_pool *pool, int64_t width) {
    if (pool->used + width > pool->capacity) {
        int64_t grown = pool->capacity ? 2 * pool->capacity : 1 << 16;
        while (grown < pool->used + width) grown *= 2;
        pool->values = (int64_t *)realloc(pool->values, (size_t)grown * 3 * sizeof(int64_t));
        pool->flags = (uint8_t *)realloc(pool->flags, (size_t)grown);
        pool->capacity = grown;
    }
    const int64_t at = pool->used;
    pool->used += width;
    return at;
}

static inline int64_t wf_get(const wf_pool *pool, int64_t count, int64_t s, int layer, int64_t k) {
    if (s < 0 || s >= count) return WF_UNREACHED;
    const wf_front *f = &pool->fronts[s];
    if (f->lo > f->hi || k < f->lo || k > f->hi) return WF_UNREACHED;
    return pool->values[3 * (f->at + (k - f->lo)) + layer];
}

static inline int64_t gcd64(int64_t a, int64_t b) {
    while (b) {
        const int64_t t = a % b;
        a = b;
        b = t;
    }
    return a;
}

/* The single search of gap_affine.mojo over one direction and its trace (trace, :2028-2124), the moves
 * right to left into `runs`. Returns the cost (scaled back), or -4 when it passes `max_cost`. */
static int64_t wf_cigar(const uint8_t *first, int64_t columns, const uint8_t *second, int64_t rows, int64_t x,
                        int64_t od, int64_t ed, int64_t oi, int64_t ei, int64_t max_cost, int eqx, int trace,
                        cigar_runs *runs) {
    int64_t scale = gcd64(gcd64(gcd64(x, od), gcd64(ed, oi)), ei);
    if (scale <= 0) scale = 1;
    x /= scale;
    od /= scale;
    ed /= scale;
    oi /= scale;
    ei /= scale;
    const int64_t ceiling = max_cost < 0 ? INT64_MAX : max_cost / scale;
    wf_pool *pool = &thread_pool;
    pool->used = 0;
    int64_t count = 0;
    const int64_t target = columns - rows;
    int64_t cost = -1;
    for (int64_t s = 0;; ++s) {
        if (s > ceiling) break;
        if (count == pool->fronts_capacity) {
            pool->fronts_capacity = pool->fronts_capacity ? 2 * pool->fronts_capacity : 256;
            pool->fronts = (wf_front *)realloc(pool->fronts, (size_t)pool->fronts_capacity * sizeof(wf_front));
        }
        wf_front *f = &pool->fronts[count];
        if (s == 0) {
            f->lo = f->hi = 0;
        } else {
            /* The diagonals any source reaches. */
            int64_t lo = INT64_MAX, hi = INT64_MIN;
            const int64_t from[5] = {s - x, s - od - ed, s - ed, s - oi - ei, s - ei};
            const int64_t shift[5] = {0, 1, 1, -1, -1};
            for (int q = 0; q < 5; ++q) {
                if (from[q] < 0 || from[q] >= count) continue;
                const wf_front *g = &pool->fronts[from[q]];
                if (g->lo > g->hi) continue;
                if (g->lo + shift[q] < lo) lo = g->lo + shift[q];
                if (g->hi + shift[q] > hi) hi = g->hi + shift[q];
            }
            if (lo < -rows) lo = -rows;
            if (hi > columns) hi = columns;
            f->lo = lo;
            f->hi = hi;
        }
        const int64_t width = f->hi >= f->lo ? f->hi - f->lo + 1 : 0;
        f->at = wf_reserve(pool, width);
        ++count;
        for (int64_t k = f->lo; k <= f->hi; ++k) {
            int64_t *v = &pool->values[3 * (f->at + (k - f->lo))];
            uint8_t *flag_out = &pool->flags[f->at + (k - f->lo)];
            if (s == 0) {
                v[WF_ALIGNED] = slide(first, columns, second, rows, 0, 0);
                v[WF_FIRST] = v[WF_SECOND] = WF_UNREACHED;
                *flag_out = 0;
                continue;
            }
            const int64_t same = wf_get(pool, count, s - x, WF_ALIGNED, k);
            const int64_t opened_below = wf_get(pool, count, s - od - ed, WF_ALIGNED, k - 1);
            const int64_t extended_below = wf_get(pool, count, s - ed, WF_FIRST, k - 1);
            const int64_t opened_above = wf_get(pool, count, s - oi - ei, WF_ALIGNED, k + 1);
            const int64_t extended_above = wf_get(pool, count, s - ei, WF_SECOND, k + 1);
            const int64_t below = opened_below > extended_below ? opened_below : extended_below;
            const int64_t above = opened_above > extended_above ? opened_above : extended_above;
            const int64_t first_gap = below >= 0 && below < columns ? below + 1 : WF_UNREACHED;
            const int64_t second_gap = above >= 0 && above - k <= rows ? above : WF_UNREACHED;
            const int64_t substituted = same >= 0 && same < columns && same - k < rows ? same + 1 : WF_UNREACHED;
            const int64_t gapped = first_gap > second_gap ? first_gap : second_gap;
            uint8_t flag = 0;
            /* Ties as WFA2-lib's backtrace breaks them: a substitution, then a letter of the first
             * sequence alone before one of the second, and an extension before an opening. */
            if (opened_below > extended_below) flag |= WF_OPENED_FIRST;
            if (opened_above > extended_above) flag |= WF_OPENED_SECOND;
            if (!(substituted >= gapped)) flag |= first_gap >= second_gap ? WF_FIRST : WF_SECOND;
            *flag_out = flag;
            v[WF_FIRST] = first_gap;
            v[WF_SECOND] = second_gap;
            const int64_t start = substituted > gapped ? substituted : gapped;
            v[WF_ALIGNED] = start >= 0 ? slide(first, columns, second, rows, start, k) : WF_UNREACHED;
        }
        if (target >= f->lo && target <= f->hi && pool->values[3 * (f->at + (target - f->lo)) + WF_ALIGNED] >= columns) {
            cost = s;
            break;
        }
    }
    if (cost >= 0 && trace) {
        /* The trace, gap_affine.mojo:2028-2124, moves right to left. */
        const char matched = eqx ? '=' : 'M', substituted = eqx ? 'X' : 'M';
        int64_t spent = cost, k = target, c = columns;
        int current = WF_ALIGNED;
        for (;;) {
            if (current == WF_ALIGNED) {
                const int64_t row = c - k;
                if (c == 0) {
                    runs_add(runs, 'I', row);
                    break;
                }
                if (row == 0) {
                    runs_add(runs, 'D', c);
                    break;
                }
                if (spent == 0) {
                    const int64_t start = k > 0 ? k : 0;
                    runs_add(runs, matched, c - start);
                    c = start;
                    continue;
                }
                const wf_front *f = &pool->fronts[spent];
                const int source = pool->flags[f->at + (k - f->lo)] & 7;
                const int64_t entry = source == WF_ALIGNED ? wf_get(pool, count, spent - x, WF_ALIGNED, k) + 1
                                                           : wf_get(pool, count, spent, source, k);
                if (entry <= c) {
                    runs_add(runs, matched, c - entry);
                    c = entry;
                }
                if (source == WF_ALIGNED) {
                    runs_add(runs, substituted, 1);
                    c -= 1;
                    spent -= x;
                } else {
                    current = source;
                }
            } else {
                const wf_front *f = &pool->fronts[spent];
                const int opened =
                    (pool->flags[f->at + (k - f->lo)] & (current == WF_FIRST ? WF_OPENED_FIRST : WF_OPENED_SECOND)) != 0;
                if (current == WF_FIRST) {
                    runs_add(runs, 'D', 1);
                    c -= 1;
                    k -= 1;
                    if (c == 0) {
                        runs_add(runs, 'I', -k);
                        break;
                    }
                    if (opened) {
                        spent -= od + ed;
                        current = WF_ALIGNED;
                    } else {
                        spent -= ed;
                    }
                } else {
                    runs_add(runs, 'I', 1);
                    k += 1;
                    if (c - k == 0) {
                        runs_add(runs, 'D', c);
                        break;
                    }
                    if (opened) {
                        spent -= oi + ei;
                        current = WF_ALIGNED;
                    } else {
                        spent -= ei;
                    }
                }
            }
        }
    }
    return cost < 0 ? -4 : cost * scale;
}

int64_t oracle_affine_cigar(const uint8_t *first, int64_t n, const uint8_t *second, int64_t m, int64_t mismatch,
                            int64_t deletion_opening, int64_t deletion_extension, int64_t insertion_opening,
                            int64_t insertion_extension, int64_t max_cost, int32_t right, int32_t eqx, char *cigar,
                            int64_t capacity) {
    cigar_runs runs;
    if (!runs_init(&runs, 2 * (n + m) + 4)) return -2;
    int64_t cost;
    int64_t written = 0;
    if (right) {
        cost = wf_cigar(first, n, second, m, mismatch, deletion_opening, deletion_extension, insertion_opening,
                        insertion_extension, max_cost, eqx, 1, &runs);
        if (cost >= 0) written = runs_text(&runs, 1, cigar, capacity);
    } else {
        uint8_t *a = reversed_copy(first, n), *b = reversed_copy(second, m);
        cost = wf_cigar(a, n, b, m, mismatch, deletion_opening, deletion_extension, insertion_opening,
                        insertion_extension, max_cost, eqx, 1, &runs);
        if (cost >= 0) written = runs_text(&runs, 0, cigar, capacity);
        free(a);
        free(b);
    }
    runs_free(&runs);
    if (cost >= 0 && written < 0) return -2;
    if (cost < 0 && capacity > 0) cigar[0] = 0;
    return cost;
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
    int kind; /* 0 scores, 1 alignments, 2 distances, 3 wavefront costs (and CIGARs) */
    int64_t costs[5]; /* kind 3: mismatch, deletion opening and extension, insertion opening and extension */
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
    } else if (job->kind == 3) {
        /* The wavefront runs over the pair with the reference as its first sequence, its columns. */
        cigar_runs runs;
        runs_init(&runs, 64);
        const int trace = job->cigars != NULL;
        job->distances[p] = wf_cigar(first, rows, second, columns, job->costs[0], job->costs[1], job->costs[2],
                                     job->costs[3], job->costs[4], -1, job->eqx, trace, &runs);
        if (trace) {
            char *slot = job->cigars + p * job->cigar_stride;
            const int64_t written = runs_text(&runs, 1, slot, job->cigar_stride);
            job->cigar_lengths[p] = written;
        }
        runs_free(&runs);
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


void oracle_batch_wavefront(int64_t pairs, const uint8_t *tape, const int64_t *offsets, int64_t mismatch,
                            int64_t deletion_opening, int64_t deletion_extension, int64_t insertion_opening,
                            int64_t insertion_extension, int32_t eqx, int32_t threads, int64_t *costs, char *cigars,
                            int64_t cigar_stride, int64_t *cigar_lengths) {
    batch_job job;
    memset(&job, 0, sizeof job);
    job.pairs = pairs;
    job.tape = tape;
    job.offsets = offsets;
    job.kind = 3;
    job.eqx = eqx;
    job.costs[0] = mismatch;
    job.costs[1] = deletion_opening;
    job.costs[2] = deletion_extension;
    job.costs[3] = insertion_opening;
    job.costs[4] = insertion_extension;
    job.distances = costs;
    job.cigars = cigars;
    job.cigar_stride = cigar_stride;
    job.cigar_lengths = cigar_lengths;
    run_batch(&job, threads);
}
