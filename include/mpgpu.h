/*
 * mpgpu.h -- C ABI of the B200 (sm_100a) realignment engine.
 *
 * The engine runs MarginPolish's anchored, banded 3-state pair-HMM
 * forward / backward / posterior pass (match, gap-x and gap-y posteriors,
 * run-length repeat-count emissions included) for batches of reads on one
 * GPU. Every entry point takes plain pointers and sizes and returns an
 * mp_status; mp_last_error() gives a thread-local message for the last
 * failure. There is no CPU fallback: without a usable sm_100 device every
 * compute call fails with MP_ERR_CUDA.
 *
 * Reference interfaces replaced (paths within the MarginPolish tree):
 *  - mp_realign_batch                 the per-read calls of
 *        getAlignedPairsWithIndelsUsingAnchors (impl/pairwiseAligner.c:1105-1130)
 *        made by getAlignedPairsWithIndelsCroppingReference
 *        (impl/polisher.c:605-654) inside poa_realign (impl/polisher.c:656-703),
 *        batched over all reads of all chunks;
 *  - mp_model_create                  the StateMachine built by
 *        hmm_getStateMachine + rleNucleotideEmissions_construct
 *        (impl/stateMachine.c:676-689, :724-736; impl/parser.c:235-245, :391-401),
 *        lowered to flat tables;
 *  - mp_params                        PairwiseAlignmentParameters
 *        (inc/pairwiseAligner.h:28-39);
 *  - mp_band / mp_split_points        band_constructDynamic / band_construct and
 *        getSplitPoints (impl/pairwiseAligner.c:120-226, :899-926).
 * The reference's own signatures (stList / StateMachine based) are exported
 * by the drop-in layer declared in mpgpu_dropin.h.
 */
#ifndef MPGPU_H_
#define MPGPU_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    MP_OK = 0,
    MP_ERR_ARGUMENT = 1,   /* malformed input (anchors, lengths, parameters, symbols) */
    MP_ERR_CUDA = 2,       /* CUDA runtime / device failure, or no usable device */
    MP_ERR_MEMORY = 3,     /* host or device allocation failed */
    MP_ERR_OVERFLOW = 4,   /* an internal bound was exceeded (reported, never silent) */
    MP_ERR_STATE = 5       /* call order / handle misuse */
} mp_status;

#define MP_MAX_REPEAT 51           /* repeat-count table dimension (inc/margin.h:123) */
#define MP_PROB_ONE 10000000       /* integer probability one (inc/pairwiseAligner.h:26) */

/* Lowered state machine for one read strand. States: 0 match, 1 gap-x, 2 gap-y.
 * All probabilities are natural-log values, -INFINITY for zero. */
typedef struct {
    double log_transitions[9];     /* index from*3+to */
    double log_start[3];
    double log_ragged_start[3];
    double log_end[3];
    double log_ragged_end[3];
    double log_match[25];          /* by base [x*5+y]; base 4 = 'N' */
    double log_gap_x[5];
    double log_gap_y[5];
    int32_t run_length;            /* 1: symbols carry repeat counts (base = sym & 255, count = sym >> 8) */
    int32_t strand;                /* strand flag of the repeat table lookup (1 forward) */
    int32_t max_repeat;            /* table dimension, MP_MAX_REPEAT */
    int32_t reserved;
    double repeat_scale;           /* multiplier on the log10 table (2.3025 in the reference) */
    const double *repeat_log10;    /* [4][max_repeat][max_repeat] = [base][underlying][observed]; NULL if !run_length */
} mp_model_desc;

typedef struct {
    double threshold;                       /* minimum posterior emitted */
    int64_t min_diags_between_traceback;
    int64_t traceback_diagonals;
    int64_t diagonal_expansion;
    int64_t constraint_diagonal_trim;       /* carried, unused on this path (as in the reference) */
    int64_t split_matrix_bigger_than_this;
    int32_t dynamic_anchor_expansion;
    int32_t reserved;
    double gap_gamma;                       /* carried, unused on this path */
} mp_params;

/* A batch of alignment jobs in HOST memory. Job j aligns sequence Y =
 * y_symbols[y_offsets[j] .. y_offsets[j+1]) (the read) against sequence X =
 * x_symbols[x_begin[j] .. x_end[j]) (the template; jobs may share one template
 * buffer), with anchors in those coordinates. Anchors are int32 triples
 * (x, y, expansion), strictly increasing in x and y, with 0 <= x < len(X),
 * 0 <= y < len(Y), expansion even and >= 0. */
typedef struct {
    int64_t n_jobs;
    const int64_t *x_begin;         /* n_jobs */
    const int64_t *x_end;           /* n_jobs */
    int64_t x_symbols_length;       /* length of x_symbols */
    const uint16_t *x_symbols;
    const int64_t *y_offsets;       /* n_jobs+1 */
    const uint16_t *y_symbols;
    const int64_t *anchor_offsets;  /* n_jobs+1, in triples */
    const int32_t *anchors;         /* 3 int32 per anchor */
    const uint8_t *strand;          /* 1 forward (model 0), 0 reverse (model 1) */
    const uint8_t *ragged_left;     /* NULL: all 0 */
    const uint8_t *ragged_right;    /* NULL: all 0 */
    const int64_t *x_shift;         /* NULL: 0. Added to output x (the crop start of the reference) */
} mp_batch;

typedef struct mp_engine mp_engine;
typedef struct mp_model mp_model;
typedef struct mp_result mp_result;

/* Result view: host arrays owned by the mp_result. For list k (0 match, 1 gap-x,
 * 2 gap-y), job j's tuples are [offsets[k][j], offsets[k][j+1]) of
 * weight[k], x[k], y[k], in the reference's output order. */
typedef struct {
    int64_t n_jobs;
    const int64_t *offsets[3];
    const int32_t *weight[3];
    const int32_t *x[3];
    const int32_t *y[3];
    const double *log_likelihood;   /* per job: sum over split sub-problems of the final segment's log total */
    const int64_t *cells;           /* per job: sum of band widths (cell updates counted by the metric) */
    int64_t total_cells;
    double device_ms;               /* device time of the posterior kernels for this call */
} mp_result_view;

const char *mp_last_error(void);
const char *mp_version(void);

/* Engine bound to one CUDA device (one process per GPU). */
mp_status mp_engine_create(int device, mp_engine **out);
void mp_engine_destroy(mp_engine *e);
/* Query: SM count, and whether the device is sm_100. */
mp_status mp_engine_info(const mp_engine *e, int *sm_count, int *cc_major, int *cc_minor);
/* Releases the device buffers the engine keeps between calls (the batches of the one-shot
 * calls and the slots of mp_realign_batch_into); later calls allocate them again. Each batch
 * holds forward checkpoints for its longest task in every task slot of its persistent grid, up
 * to half the device's memory (the grid shrinks beyond that; the pipelined call shares that
 * budget among its slots). */
mp_status mp_engine_release_buffers(mp_engine *e);

/* Lowered models for forward-strand (fwd) and reverse-strand (rev) reads. */
mp_status mp_model_create(mp_engine *e, const mp_model_desc *fwd, const mp_model_desc *rev, mp_model **out);
void mp_model_destroy(mp_model *m);

/* Tuning of the posterior kernel (0 = automatic everywhere):
 *   checkpoint_stride  unused (each kernel variant has a fixed stride), kept for layout;
 *   warps_per_block    resident warps per block, capped by the variant's shared memory;
 *   blocks_per_sm      persistent blocks per SM;
 *   lanes_per_task     32, 16 or 8: lanes that carry one banded sub-problem. With 16 or 8,
 *                      a warp advances 2 or 4 sub-problems of similar length in lockstep. */
typedef struct {
    int32_t checkpoint_stride;
    int32_t warps_per_block;
    int32_t blocks_per_sm;
    int32_t lanes_per_task;
} mp_tuning;
mp_status mp_engine_set_tuning(mp_engine *e, const mp_tuning *t);

/* CUDA graph capture of the device-resident pass (mp_device_batch_run): the band kernels,
 * the queue reset and the persistent posterior launches of a run are captured into one graph
 * per batch, replayed while the launches are identical (repeated runs of the batch) and
 * updated in place when they change. Re-runs after capacity, window or range retries stay
 * direct launches. Off by default. */
mp_status mp_engine_set_graph_capture(mp_engine *e, int enable);

/* Autotuner. The posterior kernel comes in variants that differ in band tile shape (lanes
 * per sub-problem x cells per lane: the window of S = lanes x cells slots), checkpoint
 * stride and resident warps. mp_engine_autotune plans `sample` (a batch like the ones to
 * come), groups its sub-problems by band hull into classes bounded by the FP32 variants'
 * window capacities, and times on each class with enough sub-problems every variant that
 * holds it, at several warps per block. Each candidate runs on a persistent grid cut to the
 * blocks that get at least six task loads per warp (no tail of idle warps) and its per-block
 * rate is scaled to the whole device. The fastest pair per class becomes the engine's
 * choice for later calls while lanes_per_task is 0 (automatic); classes without a
 * measurement keep the built-in choice. FP64 re-runs and the adjoint are not tuned.
 * `report` may be NULL. mp_engine_autotune_reset restores the built-in choice. */
#define MP_AUTOTUNE_MAX_CLASSES 8
typedef struct {
    int32_t n_classes;
    int32_t max_hull[MP_AUTOTUNE_MAX_CLASSES];          /* class bound, in window slots */
    int32_t tasks[MP_AUTOTUNE_MAX_CLASSES];             /* sub-problems of the sample in the class */
    int32_t candidates[MP_AUTOTUNE_MAX_CLASSES];        /* (variant, warps) pairs timed; 0 = not tuned */
    int32_t variant[MP_AUTOTUNE_MAX_CLASSES];           /* chosen kernel variant (-1: built-in choice) */
    int32_t lanes_per_task[MP_AUTOTUNE_MAX_CLASSES];    /* tile shape of the choice */
    int32_t cells_per_lane[MP_AUTOTUNE_MAX_CLASSES];
    int32_t checkpoint_stride[MP_AUTOTUNE_MAX_CLASSES];
    int32_t warps_per_block[MP_AUTOTUNE_MAX_CLASSES];
    double gcups[MP_AUTOTUNE_MAX_CLASSES];              /* the choice, posterior kernel time only */
    double default_gcups[MP_AUTOTUNE_MAX_CLASSES];      /* the built-in choice on the same tasks */
} mp_autotune_report;
mp_status mp_engine_autotune(mp_engine *e, const mp_model *m, const mp_params *p, const mp_batch *sample,
                             mp_autotune_report *report);
mp_status mp_engine_autotune_reset(mp_engine *e);

/* Full posterior pass over a batch of jobs held in host memory: host->device copies,
 * band construction, the persistent length-sorted posterior kernel, compaction and
 * device->host copies of the tuples. The engine keeps the device buffers of its last
 * one-shot batch, so repeated calls of similar size allocate no device memory; calls on
 * one engine are serialised. */
mp_status mp_realign_batch(mp_engine *e, const mp_model *m, const mp_params *p, const mp_batch *b,
                           mp_result **out);
mp_status mp_result_view_get(const mp_result *r, mp_result_view *v);

void mp_result_destroy(mp_result *r);

/* ---- device-resident path (inputs already in HBM; used for kernel timing) ---- */
typedef struct mp_device_batch mp_device_batch;
/* Copies a host batch to the device once and plans it (splits, band, queue order). */
mp_status mp_device_batch_create(mp_engine *e, const mp_model *m, const mp_params *p, const mp_batch *b,
                                 mp_device_batch **out);
/* Runs the posterior kernel(s) on the resident batch; outputs stay on the device.
 * If kernel_ms is non-NULL it receives the CUDA-event time of the posterior kernel(s). */
mp_status mp_device_batch_run(mp_engine *e, mp_device_batch *db, float *kernel_ms);
/* Replaces the batch's jobs (and parameters), reusing its device buffers. */
mp_status mp_device_batch_reset(mp_engine *e, mp_device_batch *db, const mp_params *p, const mp_batch *b);
/* Copies the last run's results to the host. */
mp_status mp_device_batch_fetch(mp_engine *e, mp_device_batch *db, mp_result **out);
/* Caller-owned host arrays that receive a batch's results (mp_device_batch_fetch_into):
 * offsets[k] has n_jobs + 1 entries, weight/x/y[k] have totals[k] entries, log_likelihood
 * and cells have n_jobs entries. Any pointer except the tuple arrays of a non-empty list
 * may be NULL. Page-locked arrays (mp_host_alloc) are filled by DMA at full link speed. */
typedef struct {
    int64_t *offsets[3];
    int32_t *weight[3];
    int32_t *x[3];
    int32_t *y[3];
    double *log_likelihood;
    int64_t *cells;
} mp_output;
/* Tuples of each list produced by the last run. */
mp_status mp_device_batch_counts(const mp_device_batch *db, int64_t totals[3]);
/* Copies the last run's results into caller-owned host arrays (no allocation on the host). */
mp_status mp_device_batch_fetch_into(mp_engine *e, mp_device_batch *db, const mp_output *out);
/* The end-to-end pass of mp_realign_batch, pipelined for throughput, into caller-owned arrays. The jobs are
 * cut into `parts` contiguous slices of similar work (0: automatic, 4 for large batches).
 * Two device batches on two streams take the slices in turn, so one slice's input copies and
 * kernels overlap the previous slice's compaction and tuple copies. Page-locked output arrays
 * (mp_host_alloc) are needed for the copies to overlap. `out` receives offsets,
 * log-likelihoods and cells for every job and the tuples of list k at weight/x/y[k], which
 * hold cap[k] tuples. A list that needs more gets no tuples; the call then returns
 * MP_ERR_OVERFLOW. need[k] (need may be NULL) receives the totals, so the caller can grow its
 * arrays and call again. The results equal mp_realign_batch's. The batch's host arrays must
 * stay valid until the call returns. */
mp_status mp_realign_batch_into(mp_engine *e, const mp_model *m, const mp_params *p, const mp_batch *b,
                                int32_t parts, const mp_output *out, const int64_t cap[3], int64_t need[3]);
/* Page-locked host memory for inputs and outputs (cudaHostAlloc / cudaFreeHost). */
mp_status mp_host_alloc(size_t bytes, void **out);
void mp_host_free(void *p);
/* Totals of the resident batch (cells = sum of band widths; launches per run). */
mp_status mp_device_batch_stats(const mp_device_batch *db, int64_t *total_cells, int64_t *n_tasks,
                                int32_t *kernel_launches_per_run);
void mp_device_batch_destroy(mp_device_batch *db);
/* CUDA-event times of the last run: band kernels and posterior kernels (ms). */
mp_status mp_device_batch_timing(const mp_device_batch *db, float *band_ms, float *posterior_ms);

/* ---- measurement ---- */
/* The plain one-read-per-launch form of the same kernel, for comparison with the batched
 * launch: the first max_tasks sub-problems of the batch, each in its own launch of one warp,
 * in batch order. kernel_ms receives the CUDA-event time of those launches and cells their
 * band cells. The batch must be run again before its results are fetched. */
mp_status mp_device_batch_run_plain(mp_engine *e, mp_device_batch *db, int64_t max_tasks, float *kernel_ms,
                                    int64_t *cells);
/* FP32 FMA throughput of the device measured with a dependent-chain-free FMA loop
 * (TFLOP/s, FMA = 2 flops), timed with CUDA events; the roofline denominator of the
 * posterior kernel, whose bound is the FP32 pipe. */
mp_status mp_measure_fp32_peak(mp_engine *e, double *tflops);
/* FP64 add / multiply issue rate of the device (G operations/s, one per instruction), measured
 * the same way; the roofline denominator of the bubble scorer, built of such operations. */
mp_status mp_measure_fp64_peak(mp_engine *e, double *gops);

/* ---- geometry helpers (host, integer-exact restatements used by the planner) ---- */
/* Band of one sub-problem: (xay, xmyL, xmyR) for d = 0..lX+lY into out[3*(lX+lY+1)]. */
mp_status mp_band(const int32_t *anchors, int64_t n_anchors, int64_t lx, int64_t ly, int64_t expansion,
                  int dynamic, int64_t *out);
/* Split rectangles (x1, y1, x2, y2); *n_out receives the count, at most cap are written. */
mp_status mp_split_points(const int32_t *anchors, int64_t n_anchors, int64_t lx, int64_t ly,
                          int64_t max_matrix_size, int ragged_left, int ragged_right, int64_t *out, int64_t cap,
                          int64_t *n_out);
/* Reference crop of getAlignedPairsWithIndelsCroppingReference (impl/polisher.c:613-628):
 * [*start, *end) of the template given the first/last anchor and the read length. */
mp_status mp_crop_range(const int32_t *anchors, int64_t n_anchors, int64_t template_length, int64_t read_length,
                        int64_t *start, int64_t *end);

/* ---- forward likelihood: computeForwardProbability (impl/pairwiseAligner.c:813-865) ----
 * log_prob[j] receives ln P(X_j, Y_j): the forward total at the last anti-diagonal with
 * the (ragged) end probabilities, over the band of band_construct
 * (impl/pairwiseAligner.c:175-226: every anchor box widened by p->diagonal_expansion; the
 * anchors' own expansions are ignored), with no split rectangles and no traceback
 * segments, as in the reference. Jobs with lx + ly = 0 give 0 (LOG_ONE). The band hull
 * must fit the widest kernel window (240 slots), else MP_ERR_OVERFLOW. The bubble-graph
 * callers (impl/bubbleGraph.c:924) pass no anchors: the band is then the whole matrix. */
mp_status mp_forward_batch(mp_engine *e, const mp_model *m, const mp_params *p, const mp_batch *b,
                           double *log_prob);

/* ---- bubble scoring: computeForwardProbability (impl/pairwiseAligner.c:813-865) as the
 * bubble graph calls it (impl/bubbleGraph.c:924: no anchors, no ragged ends), in the
 * reference's own arithmetic ----
 * Pair j aligns X = x_symbols[x_offset[j] .. + x_length[j]) (an allele) against
 * Y = y_symbols[y_offset[j] .. + y_length[j]) (a read substring) with the forward (strand[j]
 * = 1) or reverse model; pairs may share symbols. log_prob[j] gets the forward log
 * probability over the whole matrix computed as the reference computes it: FP64 log-space
 * cells, its approximate log-sum (impl/pairwiseAligner.c:279-299) and its operation order, so
 * the value equals the reference's bit for bit. x_length + y_length = 0 gives 0 (LOG_ONE).
 * Run lengths in the symbols must be below the model's table (51), as rleString_
 * constructSymbolString clamps them; otherwise MP_ERR_ARGUMENT. */
typedef struct {
    int64_t n_pairs;
    const int64_t *x_offset;
    const int32_t *x_length;
    const int64_t *y_offset;
    const int32_t *y_length;
    const uint8_t *strand;
    int64_t x_symbols_length;
    const uint16_t *x_symbols;
    int64_t y_symbols_length;
    const uint16_t *y_symbols;
} mp_pair_batch;

mp_status mp_forward_pairs(mp_engine *e, const mp_model *m, const mp_pair_batch *b, double *log_prob);
/* The last mp_forward_pairs call of the engine: device time of its launches (CUDA events on the
 * engine's stream), its matrix cells (sum of (x_length + 1) (y_length + 1)) and its pairs. */
mp_status mp_forward_pairs_timing(mp_engine *e, float *kernel_ms, int64_t *cells, int64_t *pairs);

/* ---- device-side node update of the POA graphs ----
 * The match part of poa_augment (impl/polisher.c:322-340) and the run-length estimate
 * (poa_estimateRepeatCountsUsingBayesianModel, impl/polisher.c:1556-1565, :1796-1865) for every
 * graph of a batch of chunks at once, on the GPU, from the aligner's match tuples. A chunk's graph
 * has node 0 (the 'N' prefix) and node i >= 1 for reference run i-1; a match (weight, x, y) of a
 * read adds to node x+1 the weight in the bin of the read's base at run y and in the bin of its
 * run length (clamped below max_repeat), and appends the observation (read number within the
 * chunk, y, weight). Observations keep poa_augment's order: reads in order, each read's tuples in
 * the given order. The run-length estimate of node i >= 1 is the reference's maximum-likelihood
 * count over its observations (1 when it has none), bit-identical: every product and sum is
 * rounded separately, in the reference's order. */
typedef struct {
    int64_t n_chunks;
    const int64_t *node_offsets;   /* n_chunks + 1 (starts at 0): chunk c's nodes, node 0 first */
    const char *node_bases;        /* per node: its base (the prefix node 'N') */
    const int64_t *chunk_reads;    /* n_chunks + 1 (starts at 0): chunk c's reads */
    const int64_t *read_offsets;   /* n_reads + 1 (starts at 0): runs of read r */
    const char *read_chars;        /* run characters of every read */
    const uint32_t *read_counts;   /* run lengths of every read */
    const uint8_t *strand;         /* per read: 1 forward strand */
    const int64_t *match_offsets;  /* n_reads + 1 (starts at 0): match tuples of read r */
    const int32_t *weight;         /* match tuples (weight, x, y): x a run of the chunk's reference, */
    const int32_t *x;              /* y a run of the read */
    const int32_t *y;
    int64_t max_repeat;            /* the graphs' maxRepeatCount (the repeat table's dimension M) */
    const double *repeat_log10;    /* [4][M][M] log10 P(observed | underlying) per base row (the
                                    * polish model's table); NULL: no run-length estimate */
} mp_node_batch;

/* Outputs of mp_node_update; any may be NULL. */
typedef struct {
    double *base_weights;    /* [nodes][5] (A C G T N) */
    double *repeat_weights;  /* [nodes][max_repeat] */
    int64_t *obs_offsets;    /* nodes + 1: node g's observations are [obs_offsets[g], obs_offsets[g+1]) */
    int64_t *obs_read;       /* [tuples]: read number within the chunk */
    int64_t *obs_offset;     /* [tuples]: run of the read */
    double *obs_weight;      /* [tuples] */
    uint64_t *repeat_counts; /* [nodes]: the estimate (0 for each chunk's node 0) */
} mp_node_result;

/* A tuple outside its chunk's graph or its read is MP_ERR_ARGUMENT. */
mp_status mp_node_update(mp_engine *e, const mp_node_batch *b, const mp_node_result *r);

/* ---- adjoint: expected counts = gradient of the summed log-likelihood ----
 * For the FP32 scaled-probability DP over each job's band (the posterior pass's band,
 * splits and ragged ends, but one walk over the whole lattice: no traceback segments), the
 * kernel accumulates, divided by each sub-problem's total P:
 *   transitions[m][i*3+j]  sum over cells of f_i(cell) * t_ij * e_j(next) * b_j(next)
 *                          = d ln P / d ln t_ij  (the Baum-Welch transition counts of
 *                          getExpectationsUsingAnchors, impl/pairwiseAligner.c:347-357,
 *                          :1151-1156, which the reference only has for transitions);
 *   match[m][xb*5+yb]      posterior of the match state at cells with bases (xb, yb)
 *                          = d ln P / d ln (match emission xb, yb);
 *   gap_x[m][xb], gap_y[m][yb]  posteriors of the gap states by base;
 *   repeat[table][row][i][j]    match posteriors by the run-length table entry used
 *                          (impl/polisher.c:1756-1775), = d ln P / d ln R[row][i][j];
 *                          when both strands share one table all counts are in table 0;
 *   start[m][s], end[m][s]  state posteriors at the first / last cell = d ln P / d ln of
 *                          the (ragged) start / end probability of state s (these vectors
 *                          are functions of the transitions, impl/stateMachine.c:518-557).
 * m is the model of the read's strand (0 forward, 1 reverse). log_lik (optional, n_jobs)
 * receives each job's ln P; log_likelihood their sum. Band hulls up to 120 slots. */
typedef struct {
    double transitions[2][9];
    double match[2][25];
    double gap_x[2][5];
    double gap_y[2][5];
    double start[2][3];
    double end[2][3];
    double repeat[2][4 * MP_MAX_REPEAT * MP_MAX_REPEAT];
    double log_likelihood;
} mp_expectations;
mp_status mp_expectations_batch(mp_engine *e, const mp_model *m, const mp_params *p, const mp_batch *b,
                                mp_expectations *out, double *log_lik);

/* ---- the POA loop: poa_realign / poa_realignIterative / poa_realignAll ----
 * A set of chunks, each a draft (run-length string) with its reads, runs the reference's
 * polishing loop (impl/polisher.c): every read is realigned to its chunk's reference and
 * folded into the chunk's partial-order graph (poa_realign, :656-703, with poa_augment,
 * :316-534); a new reference is proposed by the consensus walk (consensus mode,
 * poa_getConsensus, :1025-1275) or by the bubble graph (polish mode, poa_polish, :2008-2031:
 * candidate alleles between anchor nodes scored against every read substring,
 * impl/bubbleGraph.c:800-978); high-posterior observations become the next anchors
 * (poa_getAnchorAlignments, :536-592), the run lengths are re-estimated
 * (poa_estimateRepeatCountsUsingBayesianModel, :1556-1565) and the loop stops on an
 * unchanged reference or a score that does not improve (poa_realignIterative, :2034-2106).
 * All chunks advance together: each iteration's realignments of every chunk are one batched
 * posterior pass on the GPU, and all bubble scores one mp_forward_pairs call; graph work runs
 * on host threads, one chunk per thread. */
typedef struct {
    double reference_base_penalty;   /* referenceBasePenalty (0.5 shipped) */
    int32_t compare_repeat_counts;   /* poaConstructCompareRepeatCounts */
    int32_t use_run_length;          /* useRunLengthEncoding (then repeat_log10 is required) */
    const double *anchor_probs;      /* minPosteriorProbForAlignmentAnchors: (probability, expansion) pairs */
    int64_t n_anchor_probs;
    int64_t min_iterations;          /* minPoaConsensusIterations */
    int64_t max_iterations;          /* maxPoaConsensusIterations */
    /* polish mode (poa_polish, impl/polisher.c:2008-2031; the bubble graph of
     * impl/bubbleGraph.c:800-978), run by mp_poa_set_realign_all after the consensus iterations */
    int64_t min_polish_iterations;   /* minRealignmentPolishIterations (1 shipped) */
    int64_t max_polish_iterations;   /* maxRealignmentPolishIterations (1 shipped; 0: no polish mode) */
    int32_t use_read_alleles;        /* useReadAlleles: alleles are the reads' substrings (1 shipped; the
                                        other allele source is not built: 0 is refused when polishing) */
    int32_t reserved;
    double candidate_variant_weight; /* candidateVariantWeight (0.18 shipped) */
    int64_t column_anchor_trim;      /* columnAnchorTrim (5 shipped) */
    int64_t filter_reads_coverage;   /* filterReadsWhileHaveAtLeastThisCoverage (15 shipped) */
    double min_avg_base_quality;     /* minAvgBaseQuality (10 shipped) */
} mp_polish_params;

/* Chunks and reads in HOST memory. Chunk c's draft is runs [ref_offsets[c], ref_offsets[c+1])
 * of ref_chars / ref_counts; its reads are [chunk_reads[c], chunk_reads[c+1]) (chunk_reads[0]
 * = 0), read r is runs [read_offsets[r], read_offsets[r+1]) of read_chars / read_counts.
 * anchors: per read (anchor_offsets[r] .. [r+1]) triples (x, y, expansion) in draft and read
 * run coordinates, strictly increasing; anchor_offsets NULL aligns every read to the whole
 * draft without anchors (the no-anchor path of poa_realign). */
typedef struct {
    int64_t n_chunks;
    const int64_t *ref_offsets;
    const char *ref_chars;
    const uint32_t *ref_counts;
    const int64_t *chunk_reads;
    const int64_t *read_offsets;
    const char *read_chars;
    const uint32_t *read_counts;
    const uint8_t *strand;            /* per read, 1 forward */
    const int64_t *anchor_offsets;
    const int32_t *anchors;
    const uint8_t *read_qualities;    /* per read run, laid out like read_chars (the run-length form
                                         of rleString_rleQualities, impl/polisher.c:1692-1714); NULL:
                                         reads without qualities */
} mp_polish_batch;

typedef struct mp_poa_set mp_poa_set;
typedef struct {
    int64_t nodes;            /* graph nodes (reference runs + the leading 'N' node) */
    int64_t max_repeat;       /* repeat-count weights per node */
    int64_t reference_runs;   /* runs of the graph's reference string */
    int64_t observations, inserts, deletes, insert_runs;
    double score;             /* match weight - error weight (the stop rule's score) */
    int64_t iterations;       /* iterations the last mp_poa_set_iterate ran for this chunk */
} mp_poa_chunk_info;

/* repeat_log10: the [4][51][51] log10 run-length table (the model's); needed when
 * use_run_length. Nothing runs until mp_poa_set_realign. e and m may be NULL for a set that
 * only takes caller pairs (mp_poa_set_realign_pairs) and uses the host-side steps. */
mp_status mp_poa_set_create(mp_engine *e, const mp_model *m, const mp_params *p, const mp_polish_params *pp,
                            const mp_polish_batch *b, const double *repeat_log10, mp_poa_set **out);
void mp_poa_set_destroy(mp_poa_set *s);
/* poa_realign of every chunk against its draft with the batch's anchors. */
mp_status mp_poa_set_realign(mp_poa_set *s);
/* poa_augment of every chunk's draft with aligned pairs the caller supplies instead of the
 * GPU pass: for list k (0 match, 1 gap-x = deletes, 2 gap-y = inserts), read r's tuples
 * (weight, x, y), in draft and read coordinates, are rows pair_offsets[k][r] ..
 * pair_offsets[k][r+1] of pairs[k]. */
mp_status mp_poa_set_realign_pairs(mp_poa_set *s, const int64_t *const pair_offsets[3], const int64_t *const pairs[3]);
/* poa_realignIterative in consensus mode for every chunk (after mp_poa_set_realign). */
mp_status mp_poa_set_iterate(mp_poa_set *s);
/* poa_realignIterative in polish mode (poa_polish) for every chunk: each iteration builds every
 * chunk's bubble graph on host threads and scores all of them in one GPU launch
 * (mp_forward_pairs). */
mp_status mp_poa_set_iterate_polish(mp_poa_set *s);
/* poa_realignAll (impl/polisher.c:2109-2129): realign, the consensus iterations when
 * max_iterations > 0, then the polish iterations when max_polish_iterations > 0. */
mp_status mp_poa_set_realign_all(mp_poa_set *s);
/* The steps of one polish iteration, for inspection: bubbleGraph_constructFromPoa on every
 * chunk's current graph without the scores (it sorts each node's observations by read and
 * descending weight, as the reference does), then the scores of all chunks in one launch. */
mp_status mp_poa_set_build_bubbles(mp_poa_set *s);
mp_status mp_poa_set_score_bubbles(mp_poa_set *s);
/* sizes[4]: bubbles, alleles, allele runs and read substrings of a chunk's bubble graph. */
mp_status mp_poa_bubble_sizes(const mp_poa_set *s, int64_t chunk, int64_t sizes[4]);
/* The graph: per bubble six values (reference start, reference allele runs, first allele,
 * alleles, first read substring, read substrings); per allele its run count, its runs laid end
 * to end (chars, counts); per read substring (read index in the chunk, start run, runs) and its
 * mean quality (-1 without qualities); the supports, per bubble alleles x reads (allele-major),
 * bubbles in order (zeros before mp_poa_set_score_bubbles). Any output may be NULL. */
mp_status mp_poa_bubbles(const mp_poa_set *s, int64_t chunk, int64_t *bubbles, int64_t *allele_runs, char *chars,
                         uint64_t *counts, int64_t *reads, double *quals, float *supports);
/* bubbleGraph_getConsensusPath and bubbleGraph_getConsensusString of a scored graph: the
 * chosen allele per bubble, the new consensus (at most cap runs; *n_runs its length) and the
 * map from the graph's reference runs to the consensus runs (-1: none). */
mp_status mp_poa_bubble_consensus(const mp_poa_set *s, int64_t chunk, int64_t *path, char *chars, uint64_t *counts,
                                  int64_t cap, int64_t *n_runs, int64_t *map);
/* poa_estimateRepeatCountsUsingBayesianModel on every chunk's graph (sets the run lengths of
 * its reference string, as the caller of poa_realignAll does, marginPolish.c:558). */
mp_status mp_poa_set_estimate_repeat_counts(mp_poa_set *s);
/* Wall seconds the set has spent in each step of the loop since it was created, summed over
 * calls: [0] job arrays of a realignment (crop, symbols, anchors), [1] the posterior pass on the
 * GPU, [2] tuples into host arrays, [3] complete-indel candidates, [4] reads folded into the
 * graphs, [5] consensus walks and anchor alignments, [6] run-length estimates and scores, [7]
 * bubble graphs and their scores, [8] the graphs' observation lists put together, [9] waiting for the
 * GPU's run-length estimate after the merge. Entries past 10 are set to 0. Instrumentation of
 * this library's loop; the reference has no counterpart. */
mp_status mp_poa_set_phase_seconds(const mp_poa_set *s, double *seconds, int64_t n);
/* Steps of a realignment that run on the GPU instead of the host threads (both on by default;
 * every combination builds identical graphs). MP_POA_DEVICE_RUN_LENGTHS: the new graphs' run
 * lengths (impl/polisher.c:1556-1565) by mp_node_update, while the host threads fold the reads.
 * MP_POA_DEVICE_INDELS: every read's complete-indel candidates (poa_augment,
 * impl/polisher.c:354-522) in one GPU pass. Its buffers (device and page-locked) grow on first
 * use and are kept by the engine, so an engine's first realignment pays their allocation. */
#define MP_POA_DEVICE_RUN_LENGTHS 1
#define MP_POA_DEVICE_INDELS 2
mp_status mp_poa_set_device_steps(mp_poa_set *s, int32_t steps);
/* Inspection of a chunk's current graph (sizes from mp_poa_info). */
mp_status mp_poa_info(const mp_poa_set *s, int64_t chunk, mp_poa_chunk_info *info);
mp_status mp_poa_nodes(const mp_poa_set *s, int64_t chunk, char *bases, uint64_t *repeat_counts,
                       double *base_weights, double *repeat_count_weights, int64_t *n_obs, int64_t *n_ins,
                       int64_t *n_del);
mp_status mp_poa_observations(const mp_poa_set *s, int64_t chunk, int64_t *read, int64_t *offset, double *weight);
mp_status mp_poa_inserts(const mp_poa_set *s, int64_t chunk, double *weight_fwd, double *weight_rev,
                         int64_t *lengths, char *chars, uint64_t *counts, int64_t *n_obs);
mp_status mp_poa_deletes(const mp_poa_set *s, int64_t chunk, int64_t *lengths, double *weight_fwd,
                         double *weight_rev, int64_t *n_obs);
/* The graph's reference string (reference_runs runs). */
mp_status mp_poa_reference(const mp_poa_set *s, int64_t chunk, char *chars, uint64_t *counts);
/* poa_getConsensus: the consensus (at most cap runs; *n_runs gets its length) and the
 * node-to-consensus map (nodes - 1 entries, -1 for nodes not in the consensus). */
mp_status mp_poa_consensus(const mp_poa_set *s, int64_t chunk, char *chars, uint64_t *counts, int64_t cap,
                           int64_t *n_runs, int64_t *map);
/* poa_getAnchorAlignments with the given map (NULL: the identity): offsets[reads+1] and
 * triples (consensus position, read offset, expansion), at most cap. */
mp_status mp_poa_anchor_alignments(const mp_poa_set *s, int64_t chunk, const int64_t *map, int64_t *offsets,
                                   int64_t *triples, int64_t cap, int64_t *n_anchors);

/* ---- chunk stitching: mergeContigChunks (impl/chunker.c:50-112) with removeOverlap
 * (impl/polisher.c:1937-2006) ----
 * Joins the polished chunks of one contig (expanded strings, chunk c = chars[offsets[c] ..
 * offsets[c+1]), in order). At every boundary the last `overlap` characters of the previous
 * chunk (as cropped so far) and the first `overlap` characters of the next are aligned without
 * anchors, ragged at both ends, with model m (the reference uses its code-default nucleotide
 * machine, stateMachine3_constructNucleotide) and parameters p; both are cut at the first match
 * pair of the largest weight (the previous chunk before its x, the next from its y). A boundary
 * without match pairs puts `spacer_length` Ns in place of an empty chunk, or ten Ns at the seam
 * of a non-empty one (overlap > 0). All boundaries are aligned in one GPU batch. The merged
 * contig goes to out (at most cap characters; *out_length gets its length, MP_ERR_OVERFLOW when
 * it does not fit); report (NULL or 3 per chunk) gets each chunk's boundary weight with the
 * previous chunk, the characters cut from its start, and 1 for a spacer, 2 for a seam of Ns.
 * The reference's overlap is twice chunkBoundary (marginPolish.c:658; 100 shipped). The
 * alignments are computed in the reference's arithmetic (mp_match_pairs_reference), so the cuts
 * are the reference's; an overlap above about 2,000 characters is refused (MP_ERR_OVERFLOW). */
/* ---- ingest: a coordinate-sorted BAM to chunks, reads and anchors ----
 * bamChunker_construct2 (impl/htsIntegration.c:149-273) and convertToReadsAndAlignments
 * (:347-661), with the run-length forms the loop takes (rleString_rleQualities,
 * runLengthEncodeAlignment, impl/polisher.c:1692-1750). The BAM is read here (BGZF and the
 * record layout of the SAM/BAM specification; no index is needed: opening scans the file once
 * and keeps each record's offset, so a conversion seeks to the first record that can overlap its
 * chunks). Host-only code. */
typedef struct mp_bam mp_bam;
typedef struct {
    int64_t chunk_size;              /* chunkSize (0: whole contigs) */
    int64_t chunk_boundary;          /* chunkBoundary: the margin each chunk extends by */
    int32_t include_soft_clip;       /* includeSoftClipping */
    int32_t include_secondary;       /* includeSecondaryAlignments */
    int32_t include_supplementary;   /* includeSupplementaryAlignments */
    int32_t use_run_length;          /* useRunLengthEncoding */
    int64_t min_mapq;                /* filterAlignmentsWithMapQBelowThisThreshold (conversion only) */
    const char *region;              /* "contig:start-end" (0-based start, exclusive end) or NULL */
} mp_bam_params;

mp_status mp_bam_open(const char *path, const mp_bam_params *p, mp_bam **out);
void mp_bam_close(mp_bam *b);
mp_status mp_bam_chunk_count(const mp_bam *b, int64_t *n);
/* Chunk i: its contig name (at most cap bytes with the terminator) and bounds[4] = (boundary
 * start, start, end, boundary end), the reference's BamChunk fields. */
mp_status mp_bam_chunk(const mp_bam *b, int64_t i, char *contig, int64_t cap, int64_t bounds[4]);
/* Converts chunks [first, first + n): every record in the chunk's bounds that passes the filters
 * becomes a read trimmed to the chunk and its aligned pairs (reference, read, 10). ref_offsets /
 * ref_chars (NULL: none) give each chunk's reference over its bounds (expanded); with run
 * lengths the anchors need it (without it the reads come without anchors, as in the reference).
 * max_depth > 0 downsamples chunks whose depth reaches it, keeping each read with probability
 * max_depth / depth (poorMansDownsample, impl/htsIntegration.c:663-697) from a generator
 * seeded with seed; the reference draws from sonLib's, so its sample differs. */
mp_status mp_bam_convert(mp_bam *b, int64_t first, int64_t n, const int64_t *ref_offsets, const char *ref_chars,
                         int64_t max_depth, uint64_t seed);
/* sizes[4] of the k-th chunk of the last conversion: reads, read runs, anchors, name bytes. */
mp_status mp_bam_reads_sizes(const mp_bam *b, int64_t k, int64_t sizes[4]);
/* Its reads: runs laid end to end (read_offsets[reads+1], chars, counts), per-run qualities
 * (has_qualities per read), strand (1 forward), anchors (anchor_offsets[reads+1], int32 triples
 * (reference run, read run, 10)) and names (name_offsets[reads+1], names). Any output may be NULL. */
mp_status mp_bam_reads(const mp_bam *b, int64_t k, int64_t *read_offsets, char *chars, uint32_t *counts,
                       uint8_t *qualities, uint8_t *has_qualities, uint8_t *strand, int64_t *anchor_offsets,
                       int32_t *anchors, int64_t *name_offsets, char *names);

/* getAlignedPairs (impl/pairwiseAligner.c:1132-1139) for small anchor-free alignments, in the
 * reference's own arithmetic: FP64 log cells over the whole matrix, its approximate log-sum
 * (:279-299), its walk schedule and total refresh, so every match weight is the reference's (up
 * to CUDA's exp within one unit in the last place). For choices that depend on near-equal
 * weights. Jobs of b (no anchors; ragged ends and strand honoured) with a model without run
 * lengths, at most 2^22 matrix cells each. Job j's tuples are [offsets[j], offsets[j+1]) of
 * weight, x, y (at most cap in all; *total gets the count) in the reference's list order. */
mp_status mp_match_pairs_reference(mp_engine *e, const mp_model *m, const mp_params *p, const mp_batch *b,
                                   int64_t *offsets, int32_t *weight, int32_t *x, int32_t *y, int64_t cap,
                                   int64_t *total);

mp_status mp_merge_contig(mp_engine *e, const mp_model *m, const mp_params *p, int64_t n_chunks,
                          const int64_t *offsets, const char *chars, int64_t overlap, int64_t spacer_length,
                          char *out, int64_t cap, int64_t *out_length, int64_t *report);

/* ---- single read without any memory allocation ----
 * No counterpart in the reference. For callers that cannot allocate device memory
 * (their framework's pool owns the GPU, or allocation is not allowed where they
 * run): the pass uses only a fixed device array inside this library (8 MiB on
 * every GPU that loads it, held until exit) plus the caller's own host buffers.
 * Limits: lx + ly < MP_NOALLOC_MAX_DIAGONALS, one split rectangle, a band hull
 * of at most 60 window slots; beyond them MP_ERR_ARGUMENT. The first call on a
 * device looks the array up with cudaGetSymbolAddress (make it before any stream
 * capture). Calls share the array and serialise internally; two calls running on
 * the GPU at the same time would race. Output lists: the caller's host arrays of
 * `capacity` entries; `count` receives the tuple counts (MP_ERR_OVERFLOW when a
 * count exceeds its capacity), in the same order as mp_realign_batch. */
#define MP_NOALLOC_MAX_DIAGONALS 32768
#define MP_NOALLOC_SCRATCH_BYTES (8u << 20)
typedef struct {
    int32_t *weight[3];   /* list 0 match, 1 gap-x, 2 gap-y */
    int32_t *x[3];
    int32_t *y[3];
    int64_t capacity[3];
    int64_t count[3];     /* out */
    double log_likelihood; /* out */
    int64_t cells;        /* out */
} mp_noalloc_output;
mp_status mp_realign_single_noalloc(mp_engine *e, const mp_model *m, const mp_params *p, const uint16_t *x,
                                    int64_t lx, const uint16_t *y, int64_t ly, const int32_t *anchors,
                                    int64_t n_anchors, int strand, int ragged_left, int ragged_right,
                                    mp_noalloc_output *out);

/* ---- run-length encoding and anchors (host, integer-exact) ---- */
/* rleString_construct (impl/polisher.c:1357-1389): runs of identical characters.
 * run_chars / run_counts need room for n entries; *n_runs receives the run count. */
mp_status mp_rle_encode(const char *s, int64_t n, char *run_chars, uint32_t *run_counts, int64_t *n_runs);
/* rleString_constructSymbolString (impl/stateMachine.c:133-146) with the nucleotide
 * alphabet (impl/stateMachine.c:25-42): symbol = (min(count, max_exclusive-1) << 8) | base
 * when include_counts, else base. */
mp_status mp_rle_symbols(const char *run_chars, const uint32_t *run_counts, int64_t n, int include_counts,
                         uint32_t max_repeat_exclusive, uint16_t *out);
/* runLengthEncodeAlignment (impl/polisher.c:1732-1750): maps base-level aligned pairs
 * (x, y, expansion) through the non-RLE -> RLE coordinate maps of X and Y
 * (rleString_getNonRleToRleCoordinateMap, :1718-1730, built from the run counts)
 * and keeps the strictly increasing ones. out needs room for 3*n int32; returns the count. */
mp_status mp_rle_anchors(const int64_t *pairs, int64_t n, const uint32_t *x_run_counts, int64_t x_runs,
                         const uint32_t *y_run_counts, int64_t y_runs, int32_t *out, int64_t *n_out);

#ifdef __cplusplus
}
#endif

#endif
