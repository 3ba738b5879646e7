/*
 * excl_gpu.h — C ABI of libexcl_gpu.so, the B200 (sm_100a) implementation of
 * ExCLucene's batched decode + conjunctive (AND) intersection of compressed
 * posting lists in the ParaPFD, LRC, LRCSeg, SegLRC and hash-segmentation (HS)
 * formats.
 *
 * Plain C types only: pointers, sizes, integer status codes. Every call returns
 * an excl_status; nothing aborts the caller. Reference paths below are relative
 * to the ExCLucene source tree.
 */
#ifndef EXCL_GPU_H_
#define EXCL_GPU_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. Replace the reference's exit()-on-error paths:
 * CUDA_SAFE_CALL (ParaPFD_Intersection_kernel.cu:8-15) and the capacity checks
 * of CPUPreprocess (ParaPFD_Intersection.cu:204-212). */
typedef enum {
    EXCL_OK = 0,
    EXCL_E_INVALID = 1,     /* bad argument (null pointer, unknown term id, ...) */
    EXCL_E_CUDA = 2,        /* a CUDA runtime call failed */
    EXCL_E_CAPACITY = 3,    /* a batch or buffer exceeds its capacity */
    EXCL_E_FORMAT = 4,      /* data not representable in / not valid for the format */
    EXCL_E_TIMEOUT = 5,     /* excl_wait timed out; the batch is still in flight */
    EXCL_E_DEVICE_FLAG = 6, /* a kernel raised its error flag (bounded wait expired, bad index) */
    EXCL_E_NOMEM = 7        /* host or device allocation failed */
} excl_status;

/* List formats (one codec per list). Block bytes are the reference ParaPFD
 * layout (ParaPFor.cpp:56-94); see excl_build_params for the segmentation. */
typedef enum {
    EXCL_CODEC_PARAPFD = 0,   /* d-gaps, ParaPFD blocks (ParaPFD_Compression/main.cpp:163-189) */
    EXCL_CODEC_LRC = 1,       /* list regression, int intercept (LRC_Generator.cu:155-287) */
    EXCL_CODEC_LRCSEG = 2,    /* list regression + per-segment base (LRCSeg_Generator*.cu) */
    EXCL_CODEC_SEGLRC = 3,    /* per-segment regression + base (SegLRC_Generator.cu:94-436) */
    EXCL_CODEC_HS_SEGLRC = 4, /* hash buckets, per-bucket regression + base (HS_SegLRC_Generator.cu) */
    EXCL_CODEC_HS_PARAPFD = 5, /* hash buckets, d-gap ParaPFD blocks inside each bucket */
    EXCL_CODEC_NEWPFD = 6      /* d-gaps, NewPFD blocks: exceptions as Simple-16 (NewPFD_Compression/main.cpp,
                                  NewPFor.cpp:52-139); decode as NewPFD_Decompression_kernel.cu:322-488 */
} excl_codec;

/* Search method for locating a probe in a longer list. Every method gives the
 * same (exact) results; they differ in how a probe reaches its docID:
 * - BSEARCH and HASHSEG are the plain comparators: no position model. They find
 *   the segment by binary search over the segment heads or by the top-bits
 *   bucket directory, then binary-search the block's docIDs (the reference's
 *   uncompressed mqSearch, cuda_binarySearch_kernel.cu:167-296, and
 *   cuda_hashSegment_kernel.cu:170-314, on the compressed index);
 * - SEGREG uses the codec's own linear model: the bucket directory, then the
 *   segment regression's window (SegLRC_Intersection_kernel.cu:366-371,
 *   LRCSeg_Intersection_kernel.cu:290-302) on SegLRC, LRCSeg and HS_SegLRC lists;
 * - LEARNED uses the two-stage learned position model with its exact error
 *   window on lists that have one, and falls back to HASHSEG elsewhere (and
 *   where a leaf's window exceeds its threshold);
 * - AUTO: the autotuner's choice when one was made, else the learned model
 *   where one exists and SEGREG elsewhere.
 * d-gap codecs (ParaPFD, HS_ParaPFD, NewPFD) have no random access inside a
 * block: every method walks the block from its head or median there. */
typedef enum {
    EXCL_ALGO_AUTO = 0,
    EXCL_ALGO_BSEARCH = 1,
    EXCL_ALGO_HASHSEG = 2,
    EXCL_ALGO_LEARNED = 3,
    EXCL_ALGO_SEGREG = 4
} excl_algo;

/* ---------------------------------------------------------------------------
 * Codec calls — replace `uint32_t encodeArray(const uint32_t*, uint32_t*, uint32_t)`
 * and `decodeArray` (Compressed/include/ParaPFor.h:15-16). Reentrant; FRAC is an
 * argument instead of the global `float FRAC` (ParaPFor.cpp:19). Byte-identical
 * blocks. `cap` is the capacity of `out` in words. */
int excl_parapfd_encode(const uint32_t *in, uint32_t n, float frac, uint32_t *out, size_t cap, size_t *words);
int excl_parapfd_decode(const uint32_t *in, size_t nwords, uint32_t n, uint32_t *out, size_t *consumed);

/* NewPFD blocks (NewPFor.cpp:52-139): descriptor b << 26 | exception count,
 * the b-bit low parts, then one Simple-16 stream with the exception positions
 * (first absolute, then gaps minus one) and their high parts. A high part of
 * more than 28 bits has no Simple-16 layout: EXCL_E_FORMAT. */
int excl_newpfd_encode(const uint32_t *in, uint32_t n, float frac, uint32_t *out, size_t cap, size_t *words);
int excl_newpfd_decode(const uint32_t *in, size_t nwords, uint32_t n, uint32_t *out, size_t *consumed);

/* Compatibility shims with the reference's exact signatures (ParaPFor.h:15-16);
 * they use the process-wide FRAC set by excl_set_frac (default 0.0). Return 0
 * where the reference would write an unrepresentable block. */
void excl_set_frac(float frac);
uint32_t encodeArray(const uint32_t *in, uint32_t *out, uint32_t n);
uint32_t decodeArray(const uint32_t *in, uint32_t *out, uint32_t n);

/* ---------------------------------------------------------------------------
 * Index build (host). Replaces the offline encoders X_Compression / X_Generator
 * (e.g. ParaPFD_Compression/main.cpp:81-232, SegLRC_Generator.cu:94-436,
 * HS_SegLRC_Generator.cu:503-594) that wrote the .ind1, .ind2, .segHead, .segOffset,
 * .segMedian, .segNum, .regression_info and .HashSeg files. Input: sorted, duplicate-free docID lists in CSR form. */
typedef struct {
    uint32_t codec;        /* excl_codec used for every list unless `codecs` is set */
    const uint8_t *codecs; /* optional per-list codec (nlists entries) or NULL */
    uint32_t block;        /* segment size for fixed-block codecs: 128 or 256 (reference: 256) */
    float frac;            /* ParaPFD exception fraction (reference sweep 0..0.64) */
    uint32_t hs_bucket;    /* HS: expected bucket size (reference kExceptedBucketSize = 256), used when hs_kbits = 0 */
    uint32_t hs_kbits;     /* HS: fixed number of top bits of a hs_ubits-bit universe (0 = derive from length) */
    uint32_t hs_ubits;     /* HS: universe bits for hs_kbits */
    uint32_t threads;      /* host threads for the build (0 = all cores) */
} excl_build_params;

typedef struct excl_index excl_index;

int excl_index_build(const uint32_t *docs, const uint64_t *list_offsets, uint32_t nlists,
                     const excl_build_params *params, excl_index **out);
int excl_index_free(excl_index *ix);

/* The same build on the GPU, for the ParaPFD, NewPFD, LRC, LRCSeg, SegLRC,
 * HS_SegLRC and HS_ParaPFD formats (one codec for all lists, `codecs` = NULL): the hash
 * partition, regression fits, residuals and minima, d-gaps and medians, and
 * the ParaPFD blocks are computed by kernels on the context's device
 * (HS_SegLRC_Generator.cu:503-594, SegLRC_Generator.cu:94-436,
 * LRC_Generator.cu:96-287, LRCSeg_Generator.cu:98-215, ParaPFD_Compression/
 * main.cpp:163-189, ParaPFor.cpp:31-94; the reference runs the fits and the
 * encoder on the host). Fits of lists longer than 65,536 postings run on host
 * threads, overlapped. d_docs is the CSR docID array in device memory; list l
 * is d_docs[list_offsets[l] .. list_offsets[l+1]) (list_offsets on the host,
 * nlists + 1 entries). The result is byte-identical to excl_index_build's and
 * still has to be uploaded. NewPFD blocks are built too: their Simple-16
 * exception streams are packed by one warp per block, the 16 layouts tested
 * in parallel per word (NewPFor.cpp's sequential greedy choice, same bytes).
 * Scratch: about 12 bytes per posting plus 100 bytes per segment, freed on return. */
struct excl_ctx;
int excl_index_build_device(struct excl_ctx *ctx, const uint32_t *d_docs, const uint64_t *list_offsets,
                            uint32_t nlists, const excl_build_params *params, excl_index **out);

/* Sizes and host arrays of a built index (for checkers and the file writers).
 * Layout per list: see excl_list_info. Per segment: head, rec {start, word
 * offset, aux (ParaPFD: median docID; residual codecs: base)}, reg {a, b, L, R}. */
typedef struct {
    uint64_t word_base;
    uint32_t n, seg_base, nseg, codec, log2_block, first_doc, last_doc;
    uint32_t reg[4];      /* list regression raw bits: LRC {slope, icpt, range, 0}; LRCSeg/SegLRC {a, b, L, R} */
    uint32_t dir_shift, dir_base, ndir;
    uint32_t tile_base, ntiles;
    uint32_t model;       /* learned model slot or 0xffffffff */
} excl_list_info;

typedef struct {
    uint32_t nlists;
    uint64_t nsegs, nwords, ndir, ntilemap, postings;
    uint64_t device_bytes; /* bytes the resident image takes in HBM */
} excl_index_sizes;

int excl_index_sizes_get(const excl_index *ix, excl_index_sizes *s);
int excl_index_export(const excl_index *ix, excl_list_info *lists, uint32_t *words, uint32_t *seg_head,
                      uint32_t *seg_rec /* 4 u32 per segment */, uint32_t *seg_reg /* 4 u32 per segment */,
                      uint32_t *dir);

/* ---------------------------------------------------------------------------
 * The reference's on-disk files. An index in the ParaPFD, NewPFD, SegLRC, LRC
 * or LRCSeg format with 256-entry segments (SegmentSize of the reference
 * encoders), or in HS_SegLRC with the reference's bucketing (shift from the
 * list length, expected bucket size 256), is written as the file set the
 * reference's intersection binaries read, and such a file set is loaded
 * without re-encoding. `<dir>/<name>` +
 *   ParaPFD, NewPFD: .ind1 .ind2 .segNum .segHead .segOffset .segMedian
 *     (ParaPFD_Compression/main.cpp:81-232)
 *   SegLRC: .ind1 .ind2 .segNum .segHead .segOffset .ind2_distance_base
 *     .regression_info (per segment) .regression_info_list (per list)
 *     (SegLRC_Compression/main.cpp:80-207, SegLRC_Generator.cu:338-412)
 *   LRC: .ind1 .ind2 .segNum .segHead .segOffset .regression_info
 *     ({float slope; i32 intercept; float range} per list; LRC_Compression/
 *     main.cpp:94-215, LRC_Generator.cu:96-191)
 *   LRCSeg: .ind1 .ind2 .segNum .segHead .segOffset .ind2_distance_base
 *     .regression_info (per list) (LRCSeg_Compression/main.cpp:78-200)
 *   HS_SegLRC: .ind1 .ind2 .HashSeg_offset .HashSeg_info .segNum .segOffset
 *     .ind2_distance_base .regression_info (per bucket, empty buckets included)
 *     (HS_SegLRC_Generator.cu:180-594, HS_SegLRC_Compression/main.cpp:78-190)
 * The reference keeps the regression and hash files in a second directory.
 * .ind1 records are {u32 length; u64 byte offset}, 16 bytes (main.cpp:32-35).
 * Loading checks that lists, segments and blocks are consistent and in bounds,
 * and that every hash bucket decodes to its own docID range (EXCL_E_FORMAT
 * otherwise). */
int excl_index_save_reference(const excl_index *ix, const char *dir, const char *name);
int excl_index_load_reference(const char *dir, const char *name, uint32_t codec /* PARAPFD NEWPFD SEGLRC LRC LRCSEG HS_SEGLRC */,
                              excl_index **out);

/* The reference's .query stream (ParaPFD_Intersection.cu:139-142): per query a
 * u32 term count, then the term ids. Parse into CSR form; with null outputs it
 * only counts (nq, nterms), so a caller can size the buffers first. */
int excl_query_parse(const void *buf, size_t bytes, uint32_t *terms, size_t terms_cap, uint32_t *term_offsets,
                     size_t queries_cap, uint32_t *nq, size_t *nterms);
/* Encode CSR queries as a .query stream; with buf = NULL only *bytes is set. */
int excl_query_encode(const uint32_t *terms, const uint32_t *term_offsets, uint32_t nq, void *buf, size_t cap,
                      size_t *bytes);

/* ---------------------------------------------------------------------------
 * Context and device residency. One context per device; its own streams. */
typedef struct excl_ctx excl_ctx;

typedef struct {
    uint32_t max_queries;    /* per batch (reference: 16380-word constant image, ParaPFD_Intersection_kernel.cu:134) */
    uint32_t max_terms;      /* per query, <= 32 (reference MAX_QUERY_LEN 80, of which 8 are used by the workloads) */
    uint64_t max_keys;       /* per batch, sum of shortest-list lengths (reference baseSize) */
    uint32_t warps_per_cta;  /* batch kernel CTA width: 8 warps (0 = 8; 4 is accepted and runs as 8) */
    uint32_t ctas_per_sm;    /* batch kernel: 4, 5 or 6 resident 8-warp CTAs per SM, i.e. a register
                                budget of 64, 48 or 40 per thread (0 = 5) */
    uint32_t use_graphs;     /* 1: excl_intersect_device replays a CUDA graph of the batch kernel
                                when called again with the same arguments (excl_last_stats then
                                times the graph launch) */
    uint32_t merge_segs;     /* probe phase: a tile whose keys span at most this many segments of a
                                longer list decodes that span into shared memory and merges instead
                                of probing key by key (0 = default 2, EXCL_MERGE_OFF = never; max 4) */
} excl_ctx_config;
#define EXCL_MERGE_OFF 0xffffffffu

int excl_ctx_create(int device, const excl_ctx_config *cfg, excl_ctx **out);
int excl_ctx_destroy(excl_ctx *ctx);
const char *excl_last_error(const excl_ctx *ctx);
void *excl_ctx_stream(excl_ctx *ctx); /* the cudaStream_t all of this context's work runs on */

/* Uploads the index image once; it stays resident (reference: allocateResource,
 * ParaPFD_Intersection.cu:76-123, copies the whole .ind2 once). The caller may
 * free its host arrays afterwards; the library owns the device copies. */
int excl_index_upload(excl_ctx *ctx, excl_index *ix);

/* Decode lists [l0, l1) on the device into `d_out` (device pointer, list-major,
 * concatenated). Replaces the X_Decompression kernels (ParaPFD_Decompression_kernel.cu:117-272,
 * LRC_Decompression_kernel.cu:122-258, SegLRC_Decompression_kernel.cu:124-256,
 * HS_SegLRC_Decompression_kernel.cu:139-). Asynchronous on the context stream. */
int excl_decode_lists_device(excl_ctx *ctx, excl_index *ix, uint32_t l0, uint32_t l1, uint32_t *d_out);
/* Host convenience: decode to a host buffer (synchronous). */
int excl_decode_lists(excl_ctx *ctx, excl_index *ix, uint32_t l0, uint32_t l1, uint32_t *out, size_t cap);

/* ---------------------------------------------------------------------------
 * Batched conjunctive queries. Replaces the per-batch pipeline
 * CPUPreprocess -> htodTransfer -> kernelInvoke -> dtohTransfer
 * (ParaPFD_Intersection.cu:126-309; same skeleton in LRC/LRCSeg/SegLRC/HS).
 * Query q's terms are terms[term_offsets[q] .. term_offsets[q+1]).
 * Results: offsets[nq+1] (exclusive prefix of per-query counts) and the
 * concatenated per-query docIDs, each query sorted ascending. The output is
 * identical whatever the batching. */
typedef struct excl_batch excl_batch;
/* Threads: host threads may share a context. Calls that use its stream,
 * buffers or settings are serialised by the context; excl_wait does not hold
 * it while waiting. An excl_submit batch's results live in the context's
 * buffers until the next excl_submit on it, and waiting on the older batch
 * then returns EXCL_E_INVALID; excl_submit_into batches write to their own
 * arrays and may be waited on in any order. Up to 256 batches of either kind
 * may be in flight on one context. */

int excl_submit(excl_ctx *ctx, excl_index *ix, const uint32_t *terms, const uint32_t *term_offsets, uint32_t nq,
                uint32_t algo, excl_batch **ticket);
int excl_wait(excl_batch *ticket, uint32_t *offsets, uint32_t *docids, size_t cap, int timeout_ms, uint64_t *total);
int excl_batch_free(excl_batch *ticket);

/* Zero-copy variant of excl_submit, same results. The inputs are read from
 * host memory (asynchronously when page-locked) and the batch kernel writes
 * offsets[nq+1] and up to cap docIDs straight into the caller's arrays, which
 * must be page-locked, device-mapped host memory (excl_host_alloc, or
 * cudaHostAlloc / cudaHostRegister with the mapped flag). Query q's terms are
 * terms[term_offsets[q] .. term_offsets[q+1]) as in excl_submit. All four
 * arrays stay untouched until excl_wait(ticket, NULL, NULL, 0, timeout, &total)
 * returns; more than cap results give EXCL_E_CAPACITY there (the first cap are
 * written). Up to 256 such batches may be in flight on one context; they run
 * in submission order. excl_batch_free of an unfinished batch waits for it.
 * Replaces the same pipeline as excl_submit, with the reference's separate
 * dtohTransfer step (ParaPFD_Intersection.cu:306) folded into the kernel. */
int excl_submit_into(excl_ctx *ctx, excl_index *ix, const uint32_t *terms, const uint32_t *term_offsets, uint32_t nq,
                     uint32_t algo, uint32_t *offsets, uint32_t *docids, uint64_t cap, excl_batch **ticket);
/* Page-locked, device-mapped host memory for excl_submit_into (cudaHostAlloc). */
int excl_host_alloc(size_t bytes, void **out);
int excl_host_free(void *p);

/* All-device variant: queries and outputs already in device memory; no host
 * synchronisation. d_offsets has nq+1 entries; d_docids capacity `cap`.
 * Writes the total to d_offsets[nq]; a total above cap raises EXCL_E_CAPACITY
 * on the next excl_ctx_check. */
int excl_intersect_device(excl_ctx *ctx, excl_index *ix, const uint32_t *d_terms, const uint32_t *d_term_offsets,
                          uint32_t nq, uint32_t algo, uint32_t *d_offsets, uint32_t *d_docids, uint64_t cap);
/* Synchronises the context stream and reports device-side error flags. */
int excl_ctx_check(excl_ctx *ctx);

/* Allocation-free form of excl_intersect_device; it has no counterpart in the
 * reference. For callers that cannot call cudaMalloc when they query (a host
 * that fixes its device memory budget at start-up, or an embedding without an
 * excl_ctx, whose creation allocates the batch buffers): the per-batch scratch
 * lives in one fixed device array inside the library (5.6 MiB on every GPU that
 * loads it, held until the process exits), so the call allocates nothing.
 * The index must already be uploaded, on the current device. The caller passes
 * the inputs and outputs as device pointers and the cudaStream_t to run on;
 * the call returns after that stream has finished the batch.
 * Limits: nq <= EXCL_NOALLOC_MAX_QUERIES (else EXCL_E_CAPACITY before any
 * work) and at most EXCL_NOALLOC_MAX_KEYS docIDs over the queries' shortest
 * lists (else EXCL_E_CAPACITY after the batch).
 * The first call on a device looks up the array's device address; make that
 * first call before any stream capture. All calls share the array: calls whose
 * work overlaps on the GPU race and must be serialised by the caller.
 * The call takes no context lock: the index must not be re-uploaded
 * (excl_index_upload) or closed (excl_index_close) while a call that uses it
 * is running, on any thread. */
#define EXCL_NOALLOC_MAX_QUERIES 4096u
#define EXCL_NOALLOC_MAX_KEYS (1u << 20)
int excl_intersect_device_noalloc(excl_index *ix, const uint32_t *d_terms, const uint32_t *d_term_offsets,
                                  uint32_t nq, uint32_t algo, uint32_t *d_offsets, uint32_t *d_docids, uint64_t cap,
                                  void *stream);

/* Timing of the last excl_intersect_device / excl_wait batch: total_ms by CUDA
 * events around the batch kernel; pack_ms, probe_ms and compact_ms are its
 * three phases (pack, probe, scatter), from the kernel's own globaltimer stamps. */
typedef struct {
    float pack_ms, probe_ms, compact_ms, total_ms;
    uint64_t tiles;     /* (query, tile) work items */
    uint64_t keys;      /* shortest-list docIDs decoded */
    uint64_t probes;    /* (key, longer list) probes */
    uint64_t fallbacks; /* learned probes that fell back to the directory search */
    uint64_t merges;    /* (tile, longer list) pairs merged in shared memory instead of probed */
} excl_batch_stats;
int excl_last_stats(excl_ctx *ctx, excl_batch_stats *st);

/* Autotuner (no counterpart in the reference, which fixes one launch shape per
 * binary). Runs a sample batch (host arrays, as excl_submit) under every
 * candidate setting: search method (bsearch, hash directory, segment
 * regression windows, learned where models exist), batch kernel launch shape (8-warp CTAs per SM: 4, 5 or 6, i.e. a
 * register budget of 64, 48 or 40 per thread) and merge
 * threshold (EXCL_MERGE_OFF, 1, 2, 4 segments); then, for the best of those,
 * tiles of whole segments or of halves / quarters of them. Each candidate is timed with
 * CUDA events (median of 3 after a warm-up); the fastest is kept in the
 * context and used by later batches submitted with EXCL_ALGO_AUTO. The sample
 * must fit the context's limits. */
typedef struct {
    uint32_t algo, warps_per_cta, ctas_per_sm, merge_segs; /* the setting kept */
    float best_ms;     /* its device time for the sample */
    float default_ms;  /* device time of the untuned default (auto, 8 warps, 5 CTAs/SM, merge 2) */
    uint32_t tried;    /* candidates timed */
    uint32_t tile_split; /* log2 of the tiles each fixed segment of a query's shortest list is cut into */
} excl_tune_report;
int excl_autotune(excl_ctx *ctx, excl_index *ix, const uint32_t *terms, const uint32_t *term_offsets, uint32_t nq,
                  excl_tune_report *report);
/* Applies a setting (a report of an earlier excl_autotune, or one the caller
 * fills: algo, warps_per_cta 8 (4 is accepted), ctas_per_sm 4-6, merge_segs 1-4 or
 * EXCL_MERGE_OFF, tile_split 0-2) to the context without timing anything, so a
 * host can keep its tuning across runs. EXCL_E_INVALID for values outside
 * those ranges. */
int excl_ctx_set_tuning(excl_ctx *ctx, const excl_tune_report *setting);

/* Index-layout autotuner (no counterpart in the reference, which fixes the
 * layout per binary: SegmentSize 256 in its encoders, the HS bucket shift
 * derived from the list length at HS_SegLRC_Generator.cu:554-557). For each
 * candidate layout (codec, block size, FRAC, HS top-k bits ...) it builds the
 * corpus on the GPU (excl_index_build_device), uploads it, runs
 * excl_autotune on the sample batch and records the tuned time; the layout
 * with the lowest time is kept: *out receives that index (uploaded, owned by
 * the caller), *best its candidate number, and the context keeps its launch
 * tuning. The other candidates' indexes are freed. d_docs and list_offsets as
 * for excl_index_build_device; the sample as for excl_autotune. A candidate
 * that cannot be built (format limits, NewPFD) records its status and is
 * skipped; EXCL_E_INVALID if none can. Every layout gives the same results. */
typedef struct {
    excl_build_params build;  /* the layout (in) */
    float best_ms;            /* its tuned device time for the sample (out) */
    excl_tune_report tuning;  /* the launch setting excl_autotune chose for it (out) */
    uint64_t device_bytes;    /* its resident size (out) */
    int status;               /* EXCL_OK, or why it was skipped (out) */
} excl_layout_candidate;
int excl_autotune_layout(excl_ctx *ctx, const uint32_t *d_docs, const uint64_t *list_offsets, uint32_t nlists,
                         excl_layout_candidate *cands, uint32_t ncands, const uint32_t *terms,
                         const uint32_t *term_offsets, uint32_t nq, uint32_t *best, excl_index **out);

/* Self-test of the device failure path (no counterpart in the reference, whose
 * kernels exit() the process on any error). With polls > 0 every later batch of
 * the context also runs one bounded device wait on a flag that nothing sets; it
 * gives up after `polls` polls and raises the same error bit as an expired
 * cross-CTA wait of the batch kernel, so the batch completes, its results are
 * still exact, and excl_wait / excl_ctx_check report EXCL_E_DEVICE_FLAG ("scan
 * wait expired"). The context stays usable; polls = 0 (the default) turns the
 * check off. Faults nothing and hangs nothing: every device wait is bounded. */
int excl_ctx_set_wait_check(excl_ctx *ctx, uint32_t polls);

/* ---------------------------------------------------------------------------
 * Serving loop: continuous batching of single queries. No counterpart in the
 * reference, whose benchmark binaries run fixed batches from a query file
 * (ParaPFD_Intersection.cu:406-540). The index stays resident; queries are
 * submitted one at a time from any thread. A dispatcher packs whatever has
 * arrived into a batch whenever one of `slots` streams is idle, admitting
 * queries (FIFO) only while the batch's device working set fits in the free
 * part of a fixed HBM pool of hbm_budget_bytes; batches on different slots
 * run concurrently. A query's result is the same whatever it was batched with.
 * The index must be uploaded (excl_index_upload) to `device` first and outlive
 * the server. */
typedef struct excl_server excl_server;

typedef struct {
    uint32_t slots;             /* concurrent batches (streams), 0 = 4 */
    uint32_t max_batch_queries; /* 0 = 4096 */
    uint64_t max_batch_keys;    /* shortest-list docIDs per batch, 0 = 2^22; a query above it is rejected */
    uint64_t hbm_budget_bytes;  /* working-set pool shared by the slots, 0 = room for every slot's largest batch */
    uint32_t algo;              /* EXCL_ALGO_* */
    uint32_t warps_per_cta;     /* batch kernel CTA width: 8 warps (0 = default) */
    uint32_t ctas_per_sm;
} excl_server_config;

typedef struct {
    uint64_t submitted, completed, batches, rejected;
    double mean_batch;           /* completed queries per batch */
    uint64_t pool_bytes, pool_peak_bytes;
    uint32_t max_inflight;       /* most batches on the device at once */
    double p50_us, p99_us, max_us; /* submit -> result, completed queries */
} excl_server_stats;

int excl_server_create(int device, excl_index *ix, const excl_server_config *cfg, excl_server **out);
/* Finishes the batches in flight, fails queued queries, frees everything. */
int excl_server_destroy(excl_server *s);
/* Queues one query (its term ids are copied). Never waits for the GPU. */
int excl_server_submit(excl_server *s, const uint32_t *terms, uint32_t nterms, uint64_t *ticket);
/* Waits for a submitted query; copies its docIDs (ascending) to docids and the
 * count to *n, then releases the ticket. EXCL_E_CAPACITY if cap is too small
 * (the ticket is kept), EXCL_E_TIMEOUT after timeout_ms (< 0: no limit). */
int excl_server_wait(excl_server *s, uint64_t ticket, uint32_t *docids, size_t cap, uint32_t *n, int timeout_ms);
int excl_server_stats_get(excl_server *s, excl_server_stats *st);
int excl_server_stats_reset(excl_server *s);
/* Open-loop load for measurements: query q (terms[term_offsets[q] ..
 * term_offsets[q+1])) is submitted arrival_s[q] seconds after the call starts
 * (non-decreasing); returns once all are answered, with each query's
 * submit -> result latency in latency_s[q] (may be NULL), the excl_checksum
 * triple of all results in cs (may be NULL) and the elapsed time in *wall_s. */
int excl_server_replay(excl_server *s, const uint32_t *terms, const uint32_t *term_offsets, uint32_t nq,
                       const double *arrival_s, double *latency_s, uint64_t cs[3], double *wall_s);

/* ---------------------------------------------------------------------------
 * Learned position models. The reference's analogue is SegLRC's two-level
 * linear model: a list-level regression bounding the segment window and a
 * per-segment regression with a safe range (SegLRC_Generator.cu:264-331,
 * SegLRC_Intersection_kernel.cu:281-371). Here a root FP32 MLP 1->32->32->1,
 * trained on the device on the list's (docID, rank) pairs, routes each key to
 * one of `nleaves` linear leaves; each leaf stores the exact rank-error window
 * of its keys, measured with the query-time arithmetic, so probes stay exact.
 * Leaves wider than max_window fall back to the directory search. Models are
 * built for fixed-block lists of at least min_postings postings and uploaded
 * with the index; EXCL_ALGO_LEARNED / EXCL_ALGO_AUTO use them. */
typedef struct {
    uint32_t min_postings; /* lists with fewer postings get no model (0 = 2^20) */
    uint32_t nleaves;      /* 0 = 4096 */
    uint32_t steps;        /* training steps (0 = 300) */
    uint32_t batch;        /* sampled (docID, rank) pairs per step (0 = 16384) */
    float lr;              /* Adam learning rate (0 = 3e-3), cosine decay */
    uint32_t max_window;   /* widest leaf window used (0 = 4096) */
    uint32_t seed;
} excl_learn_params;

typedef struct {
    uint32_t models;
    double train_ms, fit_ms;   /* device time of training and of the leaf fits */
    float final_loss;          /* largest final MSE on normalized rank over the models */
    double mean_window;        /* mean leaf window (ranks) over non-empty leaves */
    double wide_leaf_frac;     /* share of non-empty leaves wider than max_window */
    uint64_t params_bytes;
} excl_learn_report;

int excl_learn_models(excl_ctx *ctx, excl_index *ix, const excl_learn_params *params, excl_learn_report *report);
/* Model of one list: root parameters (1153 floats), header {kmin, kscale,
 * nleaves, max_window}, leaves as {a, b, elo, ehi} (4 x 32-bit each). */
int excl_model_export(const excl_index *ix, uint32_t list, float *root, float *hdr4, int32_t *leaves,
                      uint32_t *nleaves);
/* The stored routing of one list's model: because the root is trained with
 * non-negative weights its leaf is non-decreasing in the key, so it is kept as
 * bnd[l] = first key routed to a leaf >= l (0xffffffff if none) plus grid[j] =
 * leaf of key first + (j << grid_shift), j in [0, grid_n]. meta = {first,
 * grid_shift, grid_n, nleaves}. The probe routes with these tables. */
int excl_model_tables(const excl_index *ix, uint32_t list, uint16_t *grid, uint32_t *bnd, uint32_t meta[4]);
/* One forward/backward pass of the training kernels over n given (x, y)
 * samples: the gradient of the mean squared error w.r.t. the 1153 root
 * parameters (for checking the kernels against a CPU restatement). */
int excl_model_grad(excl_ctx *ctx, const float *params, const float *x, const float *y, uint32_t n, float *grad,
                    float *loss);

/* Checksum triple of the reference (ParaPFD_Intersection.cu:378-403): empty
 * queries, total results, XOR of first/middle/last result per query. */
int excl_checksum(uint32_t nq, const uint32_t *offsets, const uint32_t *docids, uint64_t cs[3]);

#ifdef __cplusplus
}
#endif
#endif /* EXCL_GPU_H_ */
