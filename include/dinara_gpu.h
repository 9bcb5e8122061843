/*
 * dinara-align's batched alignment path on an NVIDIA B200 (sm_100a), as a C ABI.
 *
 * The library scores, aligns and measures batches of pairs on one GPU: global and local Gotoh
 * scores and CIGARs under a substitution table (a `Scoring`), and global unit-cost edit distances
 * by banded bit-vectors with band doubling, plain or started from a learned prediction. Every
 * result is exact: the same integers, and under a `Scoring` the same CIGAR, as dinara-align's own
 * implementation gives.
 *
 * The pair order, the reading of sequences (the first of each pair the reference, read down the
 * rows; the second the query, across the columns; `D` a reference letter alone, `I` a query letter
 * alone) and the error codes are dinara-align's (c/dinara.h in the reference). Functions take plain
 * host pointers; a context (`dinara_gpu`) holds one device's streams and the device buffers it
 * keeps between calls, and is used by one thread at a time.
 */
#ifndef DINARA_GPU_H
#define DINARA_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Codes shared with the reference's C ABI (c/dinara.h:35-49). */
#define DINARA_UNSUPPORTED_SYMBOLS (-1) /* a letter outside the alphabet (or 0xFE/0xFF at unit cost) */
#define DINARA_OUT_OF_MEMORY (-2)       /* device or host memory could not be had */
#define DINARA_INVALID_COSTS (-3)       /* a Scoring or costs that cannot be searched, or scores past 2^28 */
#define DINARA_ABOVE_MAX (-4)
#define DINARA_OUTSIDE_BAND (-5)
#define DINARA_INVALID_MODE (-6)        /* a mode or argument this entry point does not serve */
#define DINARA_INVALID_LENGTH (-7)      /* a negative length, or lists of different lengths */
/* GPU additions, distinct from the reference's codes. */
#define DINARA_DEVICE_FAILURE (-8)      /* a CUDA call failed; dinara_gpu_error() says which */
#define DINARA_DEVICE_TIMEOUT (-9)      /* a bounded wait (device flag or host wait) ran out */

/* dinara_mode kinds (c/dinara.h:69-76); under a Scoring the GPU serves ENDS_FREE (global, or with free
 * letters at the ends), EXTENSION (no match score of the mode's own; either anchor, Z-drop and end bonus)
 * and LOCAL. */
#define DINARA_ENDS_FREE 0
#define DINARA_EXTENSION 1
#define DINARA_LOCAL 2

/* The reference's structs, field for field (c/dinara.h:59-138). */
typedef struct {
    int64_t mismatch, opening, extension, opening2, extension2;
    int64_t deletion_opening, deletion_extension, deletion_opening2, deletion_extension2;
} dinara_costs;

typedef struct {
    int64_t kind, reference_start, reference_end, query_start, query_end;
    int64_t match_score, anchor, zdrop, end_bonus;
} dinara_mode;

typedef struct {
    int64_t band_low, band_high, max_cost, eqx, right_ties, max_memory;
} dinara_options;

typedef struct {
    int64_t cost, score, reference_start, reference_end, query_start, query_end;
    char *cigar;
    int64_t cigar_length;
} dinara_alignment;

/*
 * A Scoring (reference dinara_align/scoring.mojo:127-215; python Scoring, __init__.py:264-299): an
 * alphabet of 1 to 32 ASCII letters, its `alphabet_size` x `alphabet_size` table row by row, and a gap
 * of k letters scoring `opening + k * extension`, both zero or less.
 */
typedef struct {
    const char *alphabet;
    int64_t alphabet_size;
    const int8_t *table;
    int64_t opening;
    int64_t extension;
} dinara_scoring;

/* One device's context: streams, kernels' device buffers kept between calls, and the learned band
 * predictor. Null when the device cannot be opened; `dinara_gpu_last_error` says why. */
typedef struct dinara_gpu dinara_gpu;

dinara_gpu *dinara_gpu_new(int64_t device);
void dinara_gpu_free(dinara_gpu *gpu);
/* The last failure's message on this context (or, for a null context, the last dinara_gpu_new's). */
const char *dinara_gpu_last_error(const dinara_gpu *gpu);
/* The device's name and SM count, for reports. */
int64_t dinara_gpu_device_info(dinara_gpu *gpu, char *name, int64_t name_capacity, int64_t *multiprocessors);

/*
 * Scores under a Scoring, global or local (replaces the reference's device batch
 * dinara_align/api.mojo:843-892 `scores` -> scoring.mojo:1294-1409 `device_batch_scores`), or global
 * with free ends: a DINARA_ENDS_FREE mode with letter counts at the reference's and the query's starts
 * and ends (INFIX, PREFIX, SUFFIX, ends_free; no match score of the mode's own), scored as the
 * reference's host path scores them (scored.mojo:69-240), which its GPU refuses; or as an extension
 * (DINARA_EXTENSION, match score 0, from either anchor, with an end bonus; scoring.mojo:673-722).
 * Pair i is references[i] (reference_lengths[i] bytes) against queries[i]. Writes scores[i] and
 * statuses[i] (0, or the pair's own code: -1 a letter outside the alphabet, -3 scores that could pass
 * 2^28 as ScoreReach refuses, scoring.mojo:218-249). Returns 0, or a code failing the whole batch
 * (a bad Scoring or mode), and then writes nothing.
 */
int64_t dinara_gpu_scores(dinara_gpu *gpu, int64_t pairs, const char *const *references,
                          const int64_t *reference_lengths, const char *const *queries, const int64_t *query_lengths,
                          const dinara_scoring *scoring, const dinara_mode *mode, int32_t *scores, int64_t *statuses);

/* The same over one tape: pair i's reference is letters[offsets[2i] .. offsets[2i+1]) and its query
 * letters[offsets[2i+1] .. offsets[2i+2]), the reference's PairTape (scoring.mojo:267-340). */
int64_t dinara_gpu_scores_tape(dinara_gpu *gpu, int64_t pairs, const char *letters, const int64_t *offsets,
                               const dinara_scoring *scoring, const dinara_mode *mode, int32_t *scores,
                               int64_t *statuses);

/*
 * Alignments under a Scoring, global, local, with free ends (a DINARA_ENDS_FREE mode with letter
 * counts, as dinara_gpu_scores takes it) or as extensions, the CIGAR Gotoh's walk picks among equals.
 * An extension's span runs from its anchor to its stop (or the end bonus's choice, scoring.mojo:673-722)
 * and is aligned globally. Free ends are placed
 * as the reference's host path places them (scoring.mojo:690-813): the best end, of equal ones the
 * furthest along the reference less the query, the start found by a sweep back from it, and the
 * letters between aligned globally; a pair whose span's global score differs from its free-end score
 * reports DINARA_DEVICE_FAILURE in its status. (Replaces
 * api.mojo:895-1006 `alignments` on the GPU -> scoring.mojo:1436-1478 `device_batch_alignments` ->
 * device_align.mojo:278-441 `batch_kernel[record]`, and the reference's c/dinara.h:225-228 batch
 * shape). Each alignment's CIGAR is allocated here and freed with dinara_free; its spans are placed
 * as scoring.mojo:724-744 `as_alignment` places them. `eqx` nonzero writes '='/'X', else 'M'.
 */
int64_t dinara_gpu_alignments(dinara_gpu *gpu, int64_t pairs, const char *const *references,
                              const int64_t *reference_lengths, const char *const *queries,
                              const int64_t *query_lengths, const dinara_scoring *scoring, const dinara_mode *mode,
                              int64_t eqx, dinara_alignment *alignments, int64_t *statuses);

/*
 * Alignments over one tape with every CIGAR in one buffer: pair i's CIGAR is
 * cigar_bytes[cigar_offsets[i] .. cigar_offsets[i+1]) (no NULs), its score scores[i], its spans
 * spans[4i .. 4i+4) = reference_start, reference_end, query_start, query_end. `*cigar_bytes` is
 * allocated here (dinara_free). Same walk and placement as dinara_gpu_alignments.
 */
int64_t dinara_gpu_alignments_tape(dinara_gpu *gpu, int64_t pairs, const char *letters, const int64_t *offsets,
                                   const dinara_scoring *scoring, const dinara_mode *mode, int64_t eqx,
                                   int32_t *scores, int64_t *spans, int64_t *cigar_offsets, char **cigar_bytes,
                                   int64_t *statuses);

/* Frees a CIGAR or a CIGAR buffer this library allocated (c/dinara.h:207 dinara_free); null is nothing. */
void dinara_free(char *cigar);

/*
 * Global alignments under Costs, with the CIGAR the reference's Ties rule picks among equally good
 * ones (replaces the reference's CPU-only `alignments(references, queries, costs)`, api.mojo:1415-1526
 * -> least_costly api.mojo:622-716: edit_cigar, edit_distance.mojo:265-330, at unit costs with no cap;
 * the gap-affine wavefront and its trace, gap_affine.mojo:858-1010 and 2028-2124, otherwise).
 * `costs` is one gap piece (null for unit costs), deletions (reference letters alone) with costs of
 * their own when deletion_extension is above zero; `mode` null or global; `options` null, or no band,
 * `max_cost` (zero or more) a cap, `eqx`, and `right_ties` for Ties.RIGHT (WFA2-lib's backtrace from the
 * far corner) instead of Ties.LEFT (the same over both sequences reversed). `max_memory` is read as
 * unlimited: no pair is split, so a pair whose kept fronts would pass the reference's limit (80 MB by
 * default) takes the unsplit trace. results[i] is pair i's least cost or its code: -1 a 0xFE or 0xFF
 * byte, -4 past the cap, -2 fronts past the device budget. With `cigar_bytes` non-null, pair i's CIGAR
 * is (*cigar_bytes)[cigar_offsets[i] .. cigar_offsets[i+1]) (dinara_free the buffer); null measures
 * costs alone. A two-piece cost, a band or another mode fails the batch with DINARA_INVALID_MODE.
 */
int64_t dinara_gpu_cost_alignments_tape(dinara_gpu *gpu, int64_t pairs, const char *letters, const int64_t *offsets,
                                        const dinara_costs *costs, const dinara_mode *mode,
                                        const dinara_options *options, int64_t *results, int64_t *cigar_offsets,
                                        char **cigar_bytes);

/*
 * The reference's own C entry points under its names and argument lists (c/dinara.h:141-228), so a C
 * caller of the reference relinks against this library. They run on device 0 through a context the
 * library opens at the first call and keeps; calls from several threads take turns on it, and `threads`
 * is read as the device's own parallelism. Unit costs with no band or cap take band doubling (distances)
 * and the unit-cost trace (alignments); other one-piece costs the wavefront. Globally only: free ends,
 * extensions, local modes, bands and two-piece costs fail the batch with DINARA_INVALID_MODE. An
 * alignment's CIGAR is freed with dinara_free; its span is the whole of both sequences.
 */
int64_t dinara_distance(const char *reference, int64_t reference_length, const char *query, int64_t query_length,
                        const dinara_costs *costs, const dinara_mode *mode, const dinara_options *options);
int64_t dinara_align(const char *reference, int64_t reference_length, const char *query, int64_t query_length,
                     const dinara_costs *costs, const dinara_mode *mode, const dinara_options *options,
                     dinara_alignment *alignment);
int64_t dinara_score(const char *reference, int64_t reference_length, const char *query, int64_t query_length,
                     const dinara_costs *costs, const dinara_mode *mode, const dinara_options *options, int64_t *score);
int64_t dinara_distances(int64_t pairs, const char *const *references, const int64_t *reference_lengths,
                         const char *const *queries, const int64_t *query_lengths, const dinara_costs *costs,
                         const dinara_mode *mode, const dinara_options *options, int64_t threads, int64_t *results);
int64_t dinara_alignments(int64_t pairs, const char *const *references, const int64_t *reference_lengths,
                          const char *const *queries, const int64_t *query_lengths, const dinara_costs *costs,
                          const dinara_mode *mode, const dinara_options *options, int64_t threads,
                          dinara_alignment *alignments, int64_t *statuses);

/*
 * Unit-cost global edit distances (replaces api.mojo:1216-1312 `distances(placement=on_gpu)` ->
 * `gpu_distances` -> device_edit.mojo:80-173, and the reference's CPU band doubling,
 * band.mojo:526-657, which its GPU path lacks). Costs must be unit (null, or {1,0,1,-1,0,...}), the
 * mode global and the options without band or cap, as the reference's GPU placement requires
 * (api.mojo:1240-1246); otherwise the batch fails with DINARA_INVALID_MODE. Every byte matches only
 * itself; 0xFE and 0xFF are refused per pair (-1). results[i] is the distance or the pair's code.
 */
int64_t dinara_gpu_distances(dinara_gpu *gpu, int64_t pairs, const char *const *references,
                             const int64_t *reference_lengths, const char *const *queries, const int64_t *query_lengths,
                             const dinara_costs *costs, const dinara_mode *mode, const dinara_options *options,
                             int64_t *results);

/* How a band-doubling batch chooses each pair's first threshold. */
#define DINARA_BAND_PLAIN 0   /* the default: the length difference plus 256 (band.mojo:521 DOUBLING_START) */
#define DINARA_BAND_LEARNED 1 /* the context's trained predictor's cost, with its margin */
#define DINARA_BAND_GIVEN 2   /* thresholds the caller gives in `start_thresholds` */

typedef struct {
    int64_t policy;                  /* DINARA_BAND_PLAIN / _LEARNED / _GIVEN */
    const int64_t *start_thresholds; /* DINARA_BAND_GIVEN: one per pair */
    int64_t default_start;           /* added to the length difference for PLAIN; 0 for 256 */
} dinara_band_plan;

typedef struct {
    int64_t rounds;          /* launches of the band kernels (all pairs, all rounds) */
    int64_t pair_rounds;     /* summed over pairs: rounds each took */
    int64_t words_swept;     /* 64-cell words updated, all rounds (the band cells actually swept / 64) */
    int64_t full_cells;      /* sum of |A| * |B| (GCUPS denominator) */
    int64_t first_round_hits;/* pairs settled by their first threshold */
    int64_t overshoot;       /* pairs whose first threshold was at least twice their distance */
    int64_t undershoot;      /* pairs whose first threshold was below their distance */
    double kernel_ms;        /* device time of the band kernels */
    double predict_ms;       /* device time of the learned band's predictions (DINARA_BAND_LEARNED) */
    int64_t round_pairs[16]; /* pairs swept in each of the first 16 rounds */
    int64_t round_launches[16]; /* band kernel launches (window shapes) in each round */
    double round_ms[16];     /* device time of each round's band kernels */
} dinara_band_report;

/* Distances over one tape by band doubling from the plan's first thresholds; `report` may be null. */
int64_t dinara_gpu_distances_tape(dinara_gpu *gpu, int64_t pairs, const char *letters, const int64_t *offsets,
                                  const dinara_band_plan *plan, int64_t *results, dinara_band_report *report);

/*
 * The band autotuner (no reference counterpart; the reference's band doubling runs on the host with one
 * code path). A unit-cost round sweeps each pair's band with a window of G lanes x K 64-bit words, one of
 * DINARA_BAND_SHAPES shapes; which shape a band takes is set by figures the autotuner measures on the
 * context's own device: each shape's sweep rate (words a millisecond, as a relative word cost), and the
 * share of a round's work per lane that bounds a pair's chain of word steps (text letters x K), with the
 * launches' grid scheme, that give the fastest band doubling over pairs drawn from the given distribution. Shapes only decide how a band is swept, so distances never depend
 * on the tuning. A context starts from fixed defaults until this runs.
 */
#define DINARA_BAND_SHAPES 39

typedef struct {
    uint64_t seed;           /* the probe pairs' generator seed (0: 77) */
    int64_t pairs;           /* pairs drawn for the chain search (0: 50,000) */
    double length_low;       /* their reference lengths, log-uniform (0: 100 to 20,000) */
    double length_high;
    double rate_low;         /* their error rates, uniform, 50/25/25 (0: 0.5% to 15%) */
    double rate_high;
    int64_t probe_length;    /* letters of the pairs each shape is timed on (0: 4,096) */
    int64_t measure_shapes;  /* nonzero: time every shape first; zero: search the chain bound alone */
} dinara_band_tune_options;

typedef struct {
    int64_t shapes;                  /* shapes timed (0 when measure_shapes was zero) */
    double words_per_ms[40];         /* each shape's sweep rate, shape 6 log2(G) + K - 1 for K <= 6 */
    int64_t chain_tried;             /* candidate chain bounds tried */
    int64_t chain_words_tried[8];    /* each one's floor */
    double chain_share_tried[8];     /* and share */
    int64_t reach_tried[8];          /* and reach */
    double chain_ms[8];              /* the band rounds' device time under each, plain and near starts */
    int64_t chain_words;             /* the bound's floor */
    double chain_share;              /* the share chosen */
    int64_t reach;                   /* the reach chosen */
    int64_t full_grids;              /* 1 when the chosen launches each fill the GPU, 0 when they share it */
    double seconds;                  /* wall time of the whole tuning */
    double chain_ms_near[8];         /* of chain_ms, the near starts' part (the rest is plain doubling's) */
} dinara_band_tune_report;

/* Measures and installs the context's band tuning; `options` may be null for the defaults. */
int64_t dinara_gpu_band_autotune(dinara_gpu *gpu, const dinara_band_tune_options *options,
                                 dinara_band_tune_report *report);
/* A context's band tuning. A round's bound on a pair's chain of word steps is the larger of chain_words
 * and chain_share times the round's word steps (in its smallest windows) over the GPU's lanes. */
typedef struct {
    int64_t chain_words;   /* the bound's floor */
    double chain_share;    /* 0: the floor alone */
    int64_t reach;         /* how much wider than the smallest window a long pair may take, in quarters (5-8) */
    int64_t full_grids;    /* 1: a round's launches each fill the GPU; 0: they share it by their time */
    float word_costs[40];  /* each shape's relative time a word step (DINARA_BAND_SHAPES of them) */
} dinara_band_tuning;

/* Reads the context's tuning (`set` 0) or installs one (`set` 1, as a previous run reported it). */
int64_t dinara_gpu_band_tuning(dinara_gpu *gpu, int64_t set, dinara_band_tuning *tuning);

/*
 * The learned band predictor (no reference counterpart): a 258 -> 64 -> 64 -> 1 fp32 network over a
 * pair's 4-mer count differences, its length ratio and the sum of its squared 6-mer count differences,
 * predicting its distance over its mean length; band
 * doubling with DINARA_BAND_LEARNED starts each pair at the prediction times the margin plus the slack,
 * never below the length difference. Parameters are one flat vector of DINARA_PREDICTOR_PARAMETERS
 * floats: w1 [258][64], b1 [64], w2 [64][64], b2 [64], w3 [64], b3.
 */
#define DINARA_PREDICTOR_PARAMETERS 20801

typedef struct {
    uint64_t seed;          /* the training pairs' generator seed */
    int64_t pairs;          /* training pairs generated on the device (a tenth held out) */
    double length_low;      /* reference lengths log-uniform in [length_low, length_high] */
    double length_high;
    double rate_low;        /* per-pair error rate uniform in [rate_low, rate_high], 50/25/25 */
    double rate_high;
    int64_t epochs;
    int64_t batch;
    double learning_rate;   /* Adam's */
    double coverage;        /* share of held-out pairs the first threshold should reach (0.5-0.999) */
    double slack;           /* letters added to every first threshold */
} dinara_train_options;

typedef struct {
    int64_t steps;
    double train_loss;      /* mean squared error of the last batch, distance over mean length */
    double validation_loss; /* the held-out pairs' */
    double margin;          /* the multiplier chosen for the coverage */
    double slack;
    int64_t held_out;
    double seconds;         /* wall time of generation, exact distances and training */
} dinara_train_report;

/* Trains the context's predictor on the device: generates the pairs, measures their exact distances by
 * plain band doubling, trains with Adam, and sets the margin from the held-out pairs. */
int64_t dinara_gpu_predictor_train(dinara_gpu *gpu, const dinara_train_options *options, dinara_train_report *report);
/* Installs parameters (and the margin and slack) on the context, or reads them back. */
int64_t dinara_gpu_predictor_set(dinara_gpu *gpu, const float *parameters, double margin, double slack);
int64_t dinara_gpu_predictor_get(dinara_gpu *gpu, float *parameters, double *margin, double *slack);
/* The predictor's margins by the pair's mean length (< 300, < 1,000, < 4,096, longer): read into
 * `margins` (4 doubles) when `set` is 0, else installed from it. Training sets them from its held-out
 * pairs; dinara_gpu_predictor_set sets all four to its one margin. */
int64_t dinara_gpu_predictor_margins(dinara_gpu *gpu, int64_t set, double *margins);

/* The 258 features of each pair of a tape, pair-major into `features` (pairs x 258 floats): the 256 4-mer
 * count differences squared times 32 over the mean length, the length ratio, and the 6-mer count
 * differences' squares summed over the mean length. */
int64_t dinara_gpu_predictor_features(dinara_gpu *gpu, int64_t pairs, const char *letters, const int64_t *offsets,
                                      float *features);
/* One batch's gradients for the installed parameters: features pair-major (batch x 258), targets
 * (distance over mean length); the gradient of the mean squared error into `gradients`, and the mean
 * squared error into *loss. For checking the training kernels against another implementation. */
int64_t dinara_gpu_predictor_gradients(dinara_gpu *gpu, int64_t batch, const float *features, const float *targets,
                                       float *gradients, double *loss);
/* Each pair's predicted distance and first threshold. */
int64_t dinara_gpu_predictor_predict(dinara_gpu *gpu, int64_t pairs, const char *letters, const int64_t *offsets,
                                     float *predicted, int64_t *thresholds);

/*
 * Resident batches (no reference counterpart; the reference re-creates its device scope, uploads and
 * frees on every call, scoring.mojo:1342-1409): a batch's letters uploaded and packed once and kept on
 * the device, so later calls run the device path alone. One resident batch a context.
 */
typedef struct {
    double total_ms;       /* device time of the whole call, first launch to last */
    double kernel_ms;      /* device time of the sweep kernels (scores or band rounds) */
    double record_ms;      /* device time of the recording sweep and walk (alignments) */
    int64_t launches;      /* kernels this library launched in the call */
    int64_t cells;         /* matrix cells the sweeps updated */
    /* Device time and launches by kernel class, each launch timed on its own stream: 0 the proven-band
     * sweep recording decisions, 1 the proven-band sweep for scores, 2 whole-matrix sweeps, 3 the walk,
     * 4 unit-cost band rounds (a round's window shapes, first launch to last), 5 the learned band's
     * sketch and prediction, 6 unit-cost CIGARs (recording band and trace), 7 other. */
    double class_ms[8];
    int64_t class_launches[8];
    int64_t band_cells;    /* of `cells`, those of proven bands (64 diagonals a row) */
    int64_t whole_cells;   /* of `cells`, those of whole matrices (including the bands' leftovers) */
} dinara_timing;

/* Uploads and packs `pairs` pairs for a Scoring (or, with `scoring` null, as bytes for unit-cost
 * distances) and keeps them. Returns 0 or a code; per-pair refusals come back from the runs. */
int64_t dinara_gpu_resident_load(dinara_gpu *gpu, int64_t pairs, const char *letters, const int64_t *offsets,
                                 const dinara_scoring *scoring);

/* Scores (and with `cigars` nonzero the alignments' CIGARs) of the resident batch, results left on the
 * device until dinara_gpu_resident_fetch. */
int64_t dinara_gpu_resident_align(dinara_gpu *gpu, const dinara_mode *mode, int64_t cigars, int64_t eqx,
                                  dinara_timing *timing);

/* Distances of the resident (unit-cost) batch by band doubling. */
int64_t dinara_gpu_resident_distances(dinara_gpu *gpu, const dinara_band_plan *plan, dinara_band_report *report,
                                      dinara_timing *timing);

/* Copies the last resident run's results to the host: `scores` (int32, per pair) for a scoring run or
 * `distances` (int64) for a distance run; either may be null. */
int64_t dinara_gpu_resident_fetch(dinara_gpu *gpu, int32_t *scores, int64_t *distances);

/*
 * A serving loop (no reference counterpart; the reference opens a device scope, uploads and frees on
 * every call, scoring.mojo:1342-1409). Requests, each a batch of pairs under a Scoring, are submitted at
 * any time and admitted first in first out as a worker slot and device memory free up; each slot keeps its
 * stream and device buffers between requests, and admitted requests run at once on the device. Waits are
 * bounded and return DINARA_DEVICE_TIMEOUT when they run out.
 */
typedef struct dinara_server dinara_server;

typedef struct {
    int64_t slots;        /* requests that may run at once (1 to 32; 0 for 4) */
    int64_t device_bytes; /* the device memory budget for the slots' buffers (0 for 40 GiB) */
} dinara_server_options;

typedef struct {
    double submitted, admitted, finished; /* seconds since the server started */
    int64_t pairs;
    int64_t device_bytes;                 /* the request's estimated device memory */
} dinara_request_timing;

typedef struct {
    int64_t queued, running, admitted, completed, refused, pairs_done;
    int64_t resident_bytes, budget_bytes;
    double clock;  /* seconds since the server started */
    int64_t calls; /* device calls made: admitted requests merged into fewer when they share a Scoring */
} dinara_server_stats_t;

dinara_server *dinara_server_new(dinara_gpu *gpu, const dinara_server_options *options);
void dinara_server_free(dinara_server *server);
/* Queues a request (its letters and Scoring copied); its ticket into *ticket. */
int64_t dinara_server_submit(dinara_server *server, int64_t pairs, const char *letters, const int64_t *offsets,
                             const dinara_scoring *scoring, const dinara_mode *mode, int64_t *ticket);
/* Waits up to `timeout_ms` for a request: its scores and statuses (each `pairs` long) and timing; the
 * request's code (DINARA_OUT_OF_MEMORY when it cannot fit the budget) or DINARA_DEVICE_TIMEOUT. */
int64_t dinara_server_wait(dinara_server *server, int64_t ticket, int64_t timeout_ms, int32_t *scores,
                           int64_t *statuses, dinara_request_timing *timing);
int64_t dinara_server_stats(dinara_server *server, dinara_server_stats_t *stats);

/*
 * Scores without allocating (no counterpart in the reference). For callers that cannot allocate device
 * memory themselves or through this library (code inside another framework's memory pool, or under a
 * budget that forbids growth): the caller passes its own device buffers, a packed batch and the room
 * for the scores, and the call allocates nothing, keeping its working memory in one fixed device array
 * of 20 MiB that every device loading this library holds until exit.
 *
 * `tape` holds each sequence's letters as 2-bit codes in the Scoring's alphabet order (alphabets of up
 * to 4 letters), 16 a 32-bit word, lowest bits first, each sequence from a 16-byte boundary; pair i is
 * described by shapes[i] (word offsets into `tape` and lengths). Writes scores[i] (int32, device) on
 * `stream` (a cudaStream_t; null is the default stream).
 * Every call first checks the pairs' shapes with a small kernel on `stream` and waits for that stream
 * to reach it, reading back one 4-byte verdict; it then enqueues the sweep and returns without waiting
 * for it. A refused batch runs nothing and writes no score:
 *   - DINARA_OUT_OF_MEMORY: a pair wider than 512 columns with more than 8,191 reference letters (past
 *     the fixed array);
 *   - DINARA_INVALID_COSTS: a pair whose scores could pass 2^28 (the reference's ScoreReach,
 *     scoring.mojo:218-249, which the other entry points report per pair), or a shifted table entry
 *     past 16 bits.
 * The first call on a device also sets its array up, so make it before any stream capture. Calls share
 * the array: two calls that overlap on the GPU race, so serialize them.
 */
typedef struct {
    uint32_t first_word; /* the reference's first word in `tape` */
    uint32_t rows;       /* the reference's letters */
    uint32_t second_word;/* the query's first word */
    uint32_t columns;    /* the query's letters */
} dinara_packed_pair;

int64_t dinara_gpu_scores_static(int64_t device, int64_t pairs, const uint32_t *tape, const dinara_packed_pair *shapes,
                                 const dinara_scoring *scoring, const dinara_mode *mode, int32_t *scores, void *stream);

/* The device's measured integer issue rate (no reference counterpart: the roofline the sweeps are
 * measured against): `kind` 0 DPX add-and-max, 1 min/max with an add (counted as two), 2 three-input add,
 * 3 DPX add-and-max on 16-bit pairs, 4 three-way max, 5 three-way max on 16-bit pairs, 6 byte permute,
 * 7 max alone, 8 16-bit pair compare to a mask, 9 16-bit pair max with predicates, 10 kind 3 floored at
 * zero, 11 16-bit pair subtraction; instructions per second into *instructions_per_second, from independent chains on every SM. */
int64_t dinara_gpu_int32_peak(dinara_gpu *gpu, int64_t kind, double *instructions_per_second);

#ifdef __cplusplus
}
#endif

#endif
