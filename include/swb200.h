/*
 * swb200.h -- C ABI of the B200 Smith-Waterman protein DB search library
 * (libswb200.so).  Plain pointers and sizes only; every call returns a
 * sw_status (no exceptions, no exit()).
 *
 * The reference (SWhybrid) has no foreign-function layer: its GPU back end is
 * the C++ class CUDAWorker behind the abstract Worker (src/Worker.h:82-249).
 * These entry points are what a B200 Worker subclass calls from inside the
 * Worker virtuals; each declaration names the reference code it replaces.
 *
 * Residue codes: 0..22 = "ABCDEFGHIKLMNPQRSTVWXYZ", 23 = '@', 24 = any other
 * letter (the reference maps those to -1; both score 0 under BLOSUM62).
 * Scores: Smith-Waterman local alignment with affine gaps, first gap residue
 * costs gap_open + gap_extend, each further residue gap_extend, floor 0.
 * With SW_FLAG_REFERENCE_CAP (default) a score above 65535 is reported as
 * 65535, as the reference's 16-bit RecalcWorker pass does.
 */
#ifndef SWB200_H_
#define SWB200_H_

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SWB200_ABI_VERSION 1

typedef enum sw_status {
    SW_OK = 0,
    SW_ERR_INVALID = 1,      /* bad argument (null pointer, bad code, k out of range) */
    SW_ERR_CUDA = 2,         /* CUDA runtime error; text in sw_last_error() */
    SW_ERR_NOMEM = 3,        /* device or host allocation failed */
    SW_ERR_STATE = 4,        /* call out of order (e.g. search before sw_db_load) */
    SW_ERR_FORMAT = 5,       /* DB image: bad magic, version or checksum */
    SW_ERR_UNSUPPORTED = 6,  /* size beyond what this build handles */
    SW_ERR_BUSY = 7,         /* serving: admission refused, retry later */
    SW_ERR_TIMEOUT = 8,      /* a bounded device or host wait ran out */
    SW_ERR_NO_DEVICE = 9     /* no CUDA device / library built without GPU code */
} sw_status;

#define SW_FLAG_REFERENCE_CAP 1u   /* report min(score, 65535) like RecalcWorker */

/* Search parameters.  Replaces Param (src/Param.h:59-117): matrix[32*32] is
 * Param::plain_matrix indexed [query_code*32 + db_code], gap_open/gap_extend
 * are Param::gapOpen/gapExtend, top_k is Param::topNum. */
typedef struct sw_params {
    int32_t matrix[32 * 32];
    int32_t gap_open;
    int32_t gap_extend;
    int32_t top_k;          /* 1..1024 */
    uint32_t flags;         /* SW_FLAG_* */
} sw_params;

/* One hit of a result list.  Replaces Result<int> (src/ResultList.h:8-16);
 * index is the record's position in the DB as loaded (FASTA order), not a
 * layout position.  Order: score descending, then index ascending. */
typedef struct sw_hit {
    int32_t score;
    uint32_t reserved;
    uint64_t index;
} sw_hit;

/* Kernel shape.  group_width threads cooperate on one pair of DB records
 * (4..32 threads, a warp-cooperative anti-diagonal wavefront; narrow groups
 * behave like the reference's one-record-per-thread "inter-sequence" form,
 * wide groups are the "intra-sequence" form); rows_per_thread query rows are
 * kept in registers per thread (an even number).  Pairs of records with more
 * than cutover columns run concurrently in the long-pair kernel, whose query
 * passes are pipelined across the warps of a block: the long shape's rows per
 * thread when it is 32 x {8, 16, 24, 32, 64} and differs from the short shape,
 * otherwise chosen automatically (the smallest row count of at most 3 passes).
 * The rest use the short shape.  cutover 0: automatic (a split only when the
 * DB's longest pairs would dominate the bulk launch, else one shape -- the
 * long one -- for the whole DB).  sw_run_stats.used reports what ran. */
typedef struct sw_kernel_config {
    int32_t long_group_width;
    int32_t long_rows_per_thread;
    int32_t short_group_width;
    int32_t short_rows_per_thread;
    int32_t cutover;        /* columns; 0 = one shape for the whole DB */
} sw_kernel_config;

typedef struct sw_db_stats {
    uint64_t n_records;
    uint64_t n_residues;    /* sum of real record lengths */
    uint64_t n_pairs;
    uint64_t max_length;
    uint64_t device_bytes;  /* resident DB footprint on the device */
} sw_db_stats;

typedef struct sw_run_stats {
    double kernel_ms;       /* device time of the last call's kernels (CUDA events) */
    double first_pass_ms;   /* device time of its first-pass kernel launches */
    double total_ms;        /* host wall time of the last call */
    uint64_t cells;         /* sum over queries of qlen * n_residues */
    uint64_t rescored;      /* records re-scored by the 32-bit pass */
    uint32_t launches;      /* kernels this library launched in the last call */
    uint32_t queries;
    sw_kernel_config used;  /* shape of the last plain search (with a row-segment
                               plan: its first segment's shape as the short one) */
    double long_ms;         /* last plain search with a cut-over: long-pair launch time */
    double bulk_ms;         /* ... and the concurrent bulk launch time (else 0, 0) */
} sw_run_stats;

/* ---- parameters, encoding ------------------------------------------------ */

/* BLOSUM62, open 10, extend 2, top 10, reference cap on (Param.h:59-117). */
void sw_params_default(sw_params *p);

/* The -m option the reference documents (README.md:130) but does not parse
 * (its Param always uses the BLOSUM62 of Param.h:8-51).  Sets p->matrix from
 * a matrix in the common text layout: '#' comments, a line of column letters,
 * then per row its letter and one integer (-127..127) per column.  Letters of
 * the 23-letter alphabet (either case) are used; others ('*', J, O, U, ...)
 * are skipped, since those residues always score 0 (code 24), and letters the
 * text lacks score 0.  SW_ERR_FORMAT on a malformed text; message in
 * sw_last_error(NULL). */
sw_status sw_params_parse_matrix(sw_params *p, const char *text);

/* "blosum62" (any case): the built-in table; anything else: a file read with
 * sw_params_parse_matrix. */
sw_status sw_params_load_matrix(sw_params *p, const char *name_or_path);

/* Letters to residue codes.  Replaces DataPool::amino_acids_trans
 * (src/DataPool.cpp:33-47) as used by DataPool::getQuery (:312-344) and
 * FastaFile::nextSeq (src/FastaFile.cpp:110-145). */
sw_status sw_encode(const char *letters, uint64_t n, uint8_t *codes);

/* ---- context ------------------------------------------------------------- */

/* Replaces CUDAWorker::CUDAWorker + alloc (src/CUDAWorker.cu:24-82): binds a
 * device, copies the parameters, creates the stream. */
sw_status sw_ctx_create(int device, const sw_params *params, struct sw_ctx **out);

/* Replaces CUDAWorker::free / ~CUDAWorker. */
sw_status sw_ctx_destroy(struct sw_ctx *ctx);

/* Text of the last error on this context (never NULL).  With ctx NULL: the
 * last error of a context-free call (the DB image functions) on this thread. */
const char *sw_last_error(const struct sw_ctx *ctx);

/* ---- database ------------------------------------------------------------ */

/* Makes a DB resident on the device.  Replaces the per-query host feed
 * DataPool::fillChunk -> Worker::fill -> CUDAWorker::packDB -> asyncCopy
 * (src/DataPool.cpp:171-286, src/CUDAWorker.cu:144-223): records are given
 * once as codes back to back with n_records+1 offsets, sorted by length,
 * paired and interleaved on the host, and uploaded. */
sw_status sw_db_load(struct sw_ctx *ctx, const uint8_t *residues,
                     const uint64_t *offsets, uint64_t n_records);

sw_status sw_db_stats_get(const struct sw_ctx *ctx, sw_db_stats *out);

/* ---- DB image on disk ------------------------------------------------------ */

/* Replaces DBmaker's .seq/.map/.title files (FastaFile::makeDatabase,
 * src/FastaFile.cpp:182-359, read by DataPool::fill/getTitle,
 * src/DataPool.cpp:171-310) with one checksummed, mmap-able file: records
 * in FASTA order (a hit's index is its FASTA position), their offsets, a
 * title index and the stable longest-first order the device layout uses. */
typedef struct sw_image_info {
    uint64_t n_records;
    uint64_t n_residues;
    uint64_t file_bytes;
    uint64_t titles_bytes;
    uint64_t checksum;      /* 64-bit FNV-1a of everything after the header */
    uint32_t version;
    uint32_t reserved;
} sw_image_info;

/* Writes an image of records held in memory (codes 0..24; titles and
 * title_offsets (n_records+1) may be NULL for empty titles).  The file is
 * written under path + ".tmp" and renamed into place. */
sw_status sw_db_write_image(const char *path, const uint8_t *residues, const uint64_t *offsets,
                            uint64_t n_records, const char *titles,
                            const uint64_t *title_offsets);

/* FASTA -> image (replaces DBmaker; FastaFile::nextSeq, src/FastaFile.cpp:
 * 110-145).  A record is a '>' header line (its title, without the '>') and
 * the sequence lines up to the next header; letters map as in sw_encode
 * (either case; '@' = 23; other characters = 24, where the reference's table
 * gives -1); whitespace, including '\r', is skipped rather than stored.
 * Sequence text before the first header is SW_ERR_FORMAT.  info may be NULL. */
sw_status sw_fasta_to_image(const char *fasta_path, const char *image_path,
                            sw_image_info *info);

/* Checks an image (magic, version, section bounds, offset tables and, when
 * verify_checksum != 0, the checksum: SW_ERR_FORMAT on any mismatch) and
 * reports its sizes.  Needs no device. */
sw_status sw_image_get_info(const char *path, int verify_checksum, sw_image_info *info);

/* Read access to an image without a device: maps the file (checked as by
 * sw_image_get_info) and points into it.  The pointers stay valid until
 * sw_image_close.  For host code that needs the records or titles
 * themselves, such as a DataPool reading a DB for several workers. */
typedef struct sw_image_view {
    const uint8_t *residues;        /* codes 0..24, records back to back */
    const uint64_t *offsets;        /* n_records + 1 */
    const char *titles;
    const uint64_t *title_offsets;  /* n_records + 1 */
    const uint32_t *order;          /* records by length, longest first, stable */
    uint64_t n_records;
    uint64_t n_residues;
    const void *mapping;            /* for sw_image_close */
    uint64_t mapping_bytes;
} sw_image_view;

sw_status sw_image_open(const char *path, int verify_checksum, sw_image_view *view);
void sw_image_close(sw_image_view *view);

/* sw_db_load from an image: maps the file, checks it as sw_image_get_info
 * does, builds the device layout from the stored order (checked to be the
 * stable longest-first permutation) and keeps the file mapped for titles. */
sw_status sw_db_load_image(struct sw_ctx *ctx, const char *path, int verify_checksum);

/* A record's title from the image the resident DB was loaded from (replaces
 * DataPool::getTitle, src/DataPool.cpp:289-310).  *title points into the
 * mapping (not NUL-terminated, *length bytes) and stays valid until the next
 * sw_db_load* or sw_ctx_destroy.  SW_ERR_STATE when the DB did not come from
 * an image. */
sw_status sw_db_title(const struct sw_ctx *ctx, uint64_t record, const char **title,
                      uint64_t *length);

/* ---- plain search: one query per call ------------------------------------ */

/* Replaces CUDAWorker::setQuery + search (src/CUDAWorker.cu:84-142,224-246)
 * plus the RecalcWorker pass (src/RecalcWorker.cpp:99-268) plus the top-k
 * merge (src/ResultList.h:37-79, src/WorkerPool.cpp:99-105).
 * hits: top_k entries; *n_hits receives how many have score > 0.
 * scores: optional (NULL or n_records int32), every record's score in DB order.
 * Any query length up to 2^24 residues (SW_ERR_UNSUPPORTED beyond; the same
 * bound holds for sw_search_device and each query of sw_search_batch): a
 * query whose profile does not fit one block's shared memory (over ~8,000
 * residues with the wide shapes) is scored in row segments of whole passes by
 * consecutive launches, each handing its last row (H and F per column) to the
 * next, with the scores merged by maximum. */
sw_status sw_search(struct sw_ctx *ctx, const uint8_t *query, uint32_t qlen,
                    sw_hit *hits, uint32_t *n_hits, int32_t *scores);

/* Same as sw_search with the query already in device memory and no host
 * copies; results stay on the device (d_scores: n_records int32, DB order,
 * may be NULL).  Asynchronous: the work is only enqueued on the context's
 * stream (call sw_sync to wait).  The device query buffer must stay valid
 * until then.  Used to time the resident path. */
sw_status sw_search_device(struct sw_ctx *ctx, const uint8_t *d_query,
                           uint32_t qlen, int32_t *d_scores);

/* Overrides the kernel shape chosen for plain searches (NULL = automatic). */
sw_status sw_set_kernel_config(struct sw_ctx *ctx, const sw_kernel_config *cfg);

/* One step of a row-segment plan: whole passes of group_width x
 * rows_per_thread query rows.  In a tuning entry, passes = 0 means "the rest
 * of the query" (its last pass padded); group_width = 0 ends the plan. */
typedef struct sw_plan_step {
    int32_t group_width;
    int32_t rows_per_thread;
    int32_t passes;
} sw_plan_step;

#define SW_PLAN_STEPS 4

/* Shape table from the autotuner: for a query of qlen residues the first
 * entry (in the given order, sorted by max_qlen) with qlen <= max_qlen is used
 * when its shapes fit that length (else the cost model chooses).  A new
 * context starts with the table measured on B200 that is compiled into the
 * library (swhybrid_b200/tuned/b200.json); this call replaces it, and n = 0
 * clears it (the cost model alone chooses).
 *
 * plan (optional, plan[0].group_width = 0 for none): the query's rows in
 * consecutive row segments of different shapes, so that only the last
 * segment's last pass holds padding rows.  Each step with passes > 0 takes
 * exactly that many whole passes; the first step with passes = 0 (or, if
 * none, the shape cfg gives the bulk launch) takes the rest.  Each segment
 * reads the boundary row the one before it wrote, and scores merge by
 * maximum, as when a query too long for one block's profile is split.  cfg
 * still decides the long-pair cut-over; the plan covers the other pairs.
 * The plan is not used (cfg's shape runs the whole query) when a shape
 * override is set, when its fixed steps need more rows than the query has,
 * when a segment's profile does not fit one pass of shared memory, or when a
 * segment's shape would make its launch wait on one long record (the longest
 * record pair it scores has more columns than a group's even share of the
 * DB: such a shape only pays with the long-pair split).  sw_get_plan reports
 * what a length runs. */
typedef struct sw_tuning_entry {
    uint32_t max_qlen;
    sw_kernel_config cfg;
    sw_plan_step plan[SW_PLAN_STEPS];
} sw_tuning_entry;

sw_status sw_set_tuning(struct sw_ctx *ctx, const sw_tuning_entry *entries, uint32_t n);

/* The compiled kernel shapes: fills up to capacity (group width, rows per
 * thread, threads per block) entries (any array may be NULL); *n_shapes
 * receives the total. */
sw_status sw_get_shapes(int32_t *group_width, int32_t *rows_per_thread,
                        int32_t *threads_per_block, uint32_t capacity, uint32_t *n_shapes);

/* Shape the library would pick for a query of this length. */
sw_status sw_get_kernel_config(struct sw_ctx *ctx, uint32_t qlen, sw_kernel_config *cfg);

/* Row segments a plain search of this length runs on the DB's pairs below the
 * long-pair cut-over, in order: each step's shape and passes (the last step
 * holds the rest of the query, its last pass padded).  Fills up to capacity
 * steps; *n_steps receives the count (1 without a plan). */
sw_status sw_get_plan(struct sw_ctx *ctx, uint32_t qlen, sw_plan_step *steps, uint32_t capacity,
                      uint32_t *n_steps);

sw_status sw_get_run_stats(const struct sw_ctx *ctx, sw_run_stats *out);

/* Totals since the last sw_reset_totals, folded in by sw_sync.  first_pass_ms
 * sums the device time of every first-pass kernel launch (CUDA events on the
 * context's stream); search_ms sums whole searches. */
typedef struct sw_totals {
    double first_pass_ms;
    double search_ms;
    uint64_t first_pass_launches;
    uint64_t launches;
    uint64_t cells;
    uint64_t queries;
} sw_totals;

/* Runs the context's work on a caller-owned CUDA stream (cudaStream_t passed
 * as void*; NULL restores the context's own stream).  Replaces the two
 * streams CUDAWorker::alloc creates (src/CUDAWorker.cu:53-82). */
sw_status sw_set_stream(struct sw_ctx *ctx, void *cuda_stream);

/* Waits for all work enqueued on the context and folds event timings into
 * the totals. */
sw_status sw_sync(struct sw_ctx *ctx);
sw_status sw_reset_totals(struct sw_ctx *ctx);
sw_status sw_get_totals(const struct sw_ctx *ctx, sw_totals *out);

/* ---- batched search: many queries per call -------------------------------- */

/* No reference counterpart (the reference searches one query per run;
 * WorkerPool balances DB chunks over host threads, src/WorkerPool.cpp:10-82).
 * Options of sw_search_batch.  Queries shorter than stack_rows residues are
 * packed several to a "stack" (rows_per_thread-aligned blocks of one virtual
 * query) and scored by one launch of shape group_width x rows_per_thread;
 * longer queries form stacks of their own, grouped by the shape the tuning
 * table gives their length.  Pairs of records longer than cutover columns run
 * in a concurrent launch with the long shape (0 = no split).  use_graph != 0
 * captures each batch signature (query count and lengths) as a CUDA graph and
 * replays it. */
typedef struct sw_batch_options {
    int32_t cutover;
    int32_t long_group_width;
    int32_t long_rows_per_thread;
    int32_t use_graph;
    int32_t group_width;
    int32_t rows_per_thread;
    int32_t stack_rows;
    int32_t pair_rows;      /* queries of at most this many residues are scored two per
                               register (pair_group_width x pair_rows_per_thread); 0 = off */
    int32_t pair_group_width;
    int32_t pair_rows_per_thread;
    int32_t pair_long;      /* != 0: longer queries are paired too (a lane each, scored in
                               segments of pair_rows rows by consecutive launches) */
    int32_t pair_regions;   /* boundary regions for those segments: up to this many tall
                               double stacks share each segment launch (a region holds
                               8 bytes per DB column); 0 = automatic: up to 16, as many
                               as fit in a quarter of the free memory */
} sw_batch_options;

/* NULL restores the defaults (no cut-over, long shape 32x16, graphs on,
 * stacks of up to 4096 rows with shape 16x64 -- the best measured on B200
 * for a 64-query batch of lengths 50..5,000 against a 205 M-residue DB --
 * and queries up to 2048 residues paired two per register with shape 16x64).
 * Paired queries: two stacks of short queries share every register, one in
 * each 16-bit lane, against one record, with a pre-packed profile (no
 * per-row byte unpacking); a lane stack holds at most pair_rows rows. */
sw_status sw_set_batch_options(struct sw_ctx *ctx, const sw_batch_options *opt);

/* Searches n_queries queries (codes back to back; query_offsets has
 * n_queries+1 entries) against the resident DB in one device pass.
 * hits: n_queries * top_k entries (query q's list at q * top_k); n_hits:
 * n_queries counts; scores: optional n_queries * n_records (query-major).
 * Results equal n_queries calls of sw_search. */
sw_status sw_search_batch(struct sw_ctx *ctx, uint32_t n_queries, const uint8_t *queries,
                          const uint64_t *query_offsets, sw_hit *hits, uint32_t *n_hits,
                          int32_t *scores);

/* ---- alignments of chosen records ---------------------------------------- */

/* One alignment: the best local alignment of the query against a record. */
typedef struct sw_alignment {
    uint64_t index;       /* the record (DB order, as given to sw_db_load) */
    int32_t score;        /* its exact score (no 65535 cap) */
    uint32_t q_begin;     /* aligned query residues [q_begin, q_end) */
    uint32_t q_end;
    uint32_t d_begin;     /* aligned record residues [d_begin, d_end) */
    uint32_t d_end;
    uint32_t matches;     /* aligned pairs with identical residues */
    uint32_t n_ops;       /* CIGAR operations at ops[ops_offset ..] */
    uint32_t reserved;
    uint64_t ops_offset;
} sw_alignment;

/* No counterpart in the reference, which reports scores and titles only
 * (WorkerPool::showResult, src/WorkerPool.cpp:130-155).  For each of the n
 * records (typically the hits of a sw_search), the best local alignment of
 * the query against it: coordinates and a CIGAR, computed on the device
 * (exact int32 Gotoh with direction bits, then a walk back from the first
 * maximal cell in record-then-query order; ties prefer the diagonal, then a
 * gap in the query, then a gap in the record, and a gap opened over one
 * extended).  ops receives run-length CIGAR operations in BAM's encoding,
 * (length << 4) | op with op 0 = M, 1 = I (query residue against a gap),
 * 2 = D (record residue against a gap); *ops_used receives how many were
 * needed (SW_ERR_UNSUPPORTED when more than ops_cap).  Direction bits take
 * qlen x record length / 2 bytes of device memory per record (at most 8 GiB
 * per record; records are processed in rounds within that bound). */
sw_status sw_traceback(struct sw_ctx *ctx, const uint8_t *query, uint32_t qlen,
                       const uint64_t *records, uint32_t n, sw_alignment *out,
                       uint32_t *ops, uint64_t ops_cap, uint64_t *ops_used);

/* ---- serving ------------------------------------------------------------- */

/* The reference serves no requests: src/main.cpp runs one query per process
 * (Param -> DataPool -> WorkerPool::run).  A serving context keeps the DB
 * resident and runs a scheduler thread that batches the requests in flight
 * at every device round (continuous batching): the DB is a ring of `chunks`
 * chunks of record pairs with the same length mix; every round scores the
 * next chunk for all requests in flight, short ones packed into shared
 * stacks as in sw_search_batch; a request joins at the next round boundary
 * and completes after `chunks` rounds with the same hits sw_search gives.
 * While serving, sw_db_load, sw_search, sw_search_device, sw_search_batch
 * and sw_set_stream return SW_ERR_BUSY, and the context's error text belongs
 * to the scheduler thread: a failed request carries its status in
 * sw_serve_result; read sw_last_error(ctx) after sw_serve_stop. */
typedef struct sw_serve_options {
    uint32_t max_active;      /* requests in flight on the device (slots) */
    uint32_t chunks;          /* rounds per request: DB chunks of the ring */
    uint32_t max_pending;     /* waiting requests before SW_ERR_BUSY (0 = unbounded) */
    uint64_t memory_budget;   /* device bytes for the slots (0 = half the free memory) */
    int32_t group_width;      /* kernel shape of the rounds */
    int32_t rows_per_thread;
    int32_t stack_rows;       /* requests shorter than this share stacks */
    int32_t pair_rows;        /* requests of at most this many residues are scored two
                                 per register (paired lanes, as in sw_search_batch) with
                                 shape pair_group_width x pair_rows_per_thread; 0 = off */
    int32_t pair_group_width;
    int32_t pair_rows_per_thread;
    int32_t pair_long;        /* != 0: longer requests are paired too (a lane each, scored
                                 in pair_rows-row segments by consecutive launches) */
    int32_t pair_regions;     /* boundary regions for those segments: up to this many
                                 tall double stacks share each segment launch (a region
                                 holds 8 bytes per DB column); 0 = automatic: up to 16,
                                 as many as fit in an eighth of the free memory */
} sw_serve_options;

/* Defaults: 128 slots, 4 chunks, unbounded queue, half the free memory,
 * shape 16x64, stacks of 4096 rows, every request paired two per register
 * with shape 16x64, in lanes of up to 2048 rows (as sw_search_batch does),
 * automatic boundary regions. */
void sw_serve_options_default(sw_serve_options *opt);

typedef struct sw_serve_result {
    uint64_t request_id;
    int32_t status;           /* SW_OK, or the error of the round that failed it */
    uint32_t n_hits;
    double submit_ms;         /* sw_serve_clock_ms() at submission */
    double start_ms;          /* ... at admission into a slot */
    double done_ms;           /* ... when its last round ended */
} sw_serve_result;

typedef struct sw_serve_stats {
    uint64_t submitted, admitted, completed, failed;
    uint64_t rounds, launches, rescored;
    uint64_t cells;           /* query residues x DB residues of completed requests */
    double busy_ms;           /* wall time inside device rounds */
    uint32_t slots, chunks;   /* as sized by sw_serve_start */
    uint32_t active, pending; /* now */
    double device_ms;         /* device time of the rounds (CUDA events from each round's
                                 table upload to its result download); busy_ms minus this
                                 is time the device waited for the host */
} sw_serve_stats;

/* Starts the scheduler thread (opt NULL = defaults).  The slot count is
 * min(max_active, memory_budget / bytes per request in flight). */
sw_status sw_serve_start(struct sw_ctx *ctx, const sw_serve_options *opt);

/* Queues a request (codes 0..24, 1..2^24 residues).  SW_ERR_BUSY when
 * max_pending requests already wait; SW_ERR_STATE when not serving.  A
 * request longer than one stack of the serving shape holds (8,192 rows for
 * the default 16 x 64; its query profile must fit one block's shared memory)
 * is scored alone at a round boundary by the plain path, which splits its
 * rows over consecutive launches, instead of sharing the round's launches. */
sw_status sw_serve_submit(struct sw_ctx *ctx, uint64_t request_id, const uint8_t *query,
                          uint32_t qlen);

/* Takes up to max_results completed requests, oldest completion first:
 * results[i] and hits[i * top_k ..] (score desc, index asc; unused entries
 * zero).  Waits up to timeout_ms for the first one (0 = no wait, < 0 = no
 * limit). */
sw_status sw_serve_poll(struct sw_ctx *ctx, uint32_t max_results, sw_serve_result *results,
                        sw_hit *hits, uint32_t *n_results, int32_t timeout_ms);

sw_status sw_serve_get_stats(struct sw_ctx *ctx, sw_serve_stats *out);

/* The clock of the result timestamps (steady, milliseconds). */
double sw_serve_clock_ms(void);

/* Drops waiting requests, lets the ones in flight finish (their results stay
 * unread), joins the scheduler and frees the serving memory. */
sw_status sw_serve_stop(struct sw_ctx *ctx);

/* ---- scoring without allocation ------------------------------------------ */

/* No counterpart in the reference.  For callers that cannot call cudaMalloc
 * where they score: a request path that must not allocate once it has
 * started (an allocation can block on the driver and stall every request
 * behind it), or a plug-in inside a host process whose device memory is all
 * reserved by that process's own allocator.  Scores every record of a DB
 * that the caller already holds in device memory (codes 0..24 back to back,
 * n_records+1 device offsets) against a device query, exactly (int32;
 * min(score, 65535) with SW_FLAG_REFERENCE_CAP), into d_scores (n_records
 * int32, device).  Allocates nothing: its scratch is one static device array
 * of about 16 MiB inside libswb200.so, held by every GPU that loads the
 * library until the process exits.  Limits: records of at most 8192
 * residues (a longer one scores 0 and the call returns SW_ERR_UNSUPPORTED
 * after scoring the others), at most 2^31 - 1 records and 2^24 query
 * residues (SW_ERR_UNSUPPORTED, nothing scored).  The first call on a device
 * looks up the array's device address; make that first call before any
 * stream capture.  The call waits for its own work on cuda_stream (NULL =
 * the default stream) before it returns.  All calls share the array and
 * each starts by clearing its counter: calls that overlap on the GPU race. */
sw_status sw_score_noalloc(int device, const sw_params *params, const uint8_t *d_query,
                           uint32_t qlen, const uint8_t *d_residues,
                           const uint64_t *d_offsets, uint32_t n_records, int32_t *d_scores,
                           void *cuda_stream);

#ifdef __cplusplus
}
#endif

#endif /* SWB200_H_ */
