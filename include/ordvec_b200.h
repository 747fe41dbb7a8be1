/*
 * ordvec_b200.h -- C ABI of libordvec_b200.so, the B200 (sm_100a) drop-in for
 * ordvec's compressed-scan path.
 *
 * Part 1 re-declares ordvec's C ABI v1 (ordvec-ffi/include/ordvec.h) with the
 * same names, struct layouts (128/128/184/24 bytes), status codes, validation
 * order and semantics, so a binding written for ordvec.h links against this
 * library unchanged.  Each declaration cites the reference declaration it
 * replaces.  Searches run on the GPU; handles own device-resident codes.
 *
 * Part 2 adds v1-compatible extensions (prefix `ovb_`): index construction
 * from host or device float vectors (GPU encode), the index kinds ABI v1 does
 * not expose (SignBitmap, RankQuantFastscan, MultiBucketBitmap), batched
 * searches with rectangular sentinel-padded output, fused two-stage
 * pipelines, and device-pointer variants that run asynchronously on a
 * caller-supplied CUDA stream.
 *
 * Errors: every fallible entry point returns a status and sets a
 * thread-local message readable with ordvec_last_error() until the next
 * fallible call on the same thread.  No entry point aborts.
 */
#ifndef ORDVEC_B200_H
#define ORDVEC_B200_H

#include <stdbool.h>
#include <stdint.h>
#include <stdlib.h>

/* ===================== Part 1: ordvec C ABI v1 ===================== */

#define ORDVEC_ABI_VERSION 1                 /* ordvec.h:15 */
#define ORDVEC_CAP_FULL_SEARCH (1 << 0)      /* ordvec.h:17 */
#define ORDVEC_CAP_SUBSET_SEARCH (1 << 1)    /* ordvec.h:19 */
#define ORDVEC_CAP_STATS (1 << 2)            /* ordvec.h:26 */
#define ORDVEC_CAP_ID_EQUALS_ROW_ID (1 << 3) /* ordvec.h:28 */
#define ORDVEC_SEARCH_FLAG_NONE 0            /* ordvec.h:30 */

typedef struct ordvec_index_t ordvec_index_t; /* ordvec.h:32 */
typedef uint32_t ordvec_status_t;             /* ordvec.h:34 */

typedef struct { /* ordvec.h:36-48, 128 bytes */
  uint64_t struct_size;
  uint32_t kind;
  uint32_t format_version;
  uint64_t dim;
  uint32_t bit_width;
  uint32_t n_top;
  uint64_t vector_count;
  uint64_t bytes_per_vec;
  uint64_t source_file_size_bytes;
  uint64_t capabilities;
  uint64_t reserved[8];
} ordvec_index_info_t;

typedef struct { /* ordvec.h:50-64, 128 bytes */
  uint64_t struct_size;
  const float *query;
  uint64_t dim;
  uint64_t k;
  const uint32_t *candidate_rows;
  uint64_t candidate_count;
  uint64_t flags;
  uint64_t user_tag;
  uint64_t reserved[8];
} ordvec_search_params_t;

typedef struct { /* ordvec.h:74-93, 184 bytes */
  uint64_t struct_size;
  uint32_t abi_version;
  uint32_t kind;
  uint64_t dim;
  uint32_t bit_width;
  uint32_t n_top;
  uint64_t k;
  uint64_t user_tag;
  uint64_t vector_count;
  uint64_t candidate_count;
  uint64_t returned_count;
  uint64_t total_ns;
  uint64_t prepare_ns;
  uint64_t score_ns;
  uint64_t select_ns;
  uint64_t vectors_scored;
  uint64_t bytes_read;
  uint64_t reserved[8];
} ordvec_search_stats_t;

typedef struct { /* ordvec.h:95-100, 24 bytes */
  uint64_t row_id;
  uint64_t id;
  float score;
  uint32_t reserved;
} ordvec_hit_t;

typedef uint32_t ordvec_index_kind_t; /* ordvec.h:102 */

#define ORDVEC_STATUS_OK 0                     /* ordvec.h:104-130 */
#define ORDVEC_STATUS_NULL_POINTER 1
#define ORDVEC_STATUS_BAD_ARGUMENT 2
#define ORDVEC_STATUS_BAD_STRUCT_SIZE 3
#define ORDVEC_STATUS_UNSUPPORTED_FORMAT 4
#define ORDVEC_STATUS_CORRUPT_INDEX 5
#define ORDVEC_STATUS_IO 6
#define ORDVEC_STATUS_DIM_MISMATCH 7
#define ORDVEC_STATUS_NONFINITE_QUERY 8
#define ORDVEC_STATUS_ROW_ID_OUT_OF_RANGE 9
#define ORDVEC_STATUS_BUFFER_TOO_SMALL 10
#define ORDVEC_STATUS_UNSUPPORTED_OPERATION 11
#define ORDVEC_STATUS_PANIC 12
#define ORDVEC_STATUS_INTERNAL 13

#define ORDVEC_INDEX_KIND_UNKNOWN 0    /* ordvec.h:132-136 */
#define ORDVEC_INDEX_KIND_RANK_QUANT 1
#define ORDVEC_INDEX_KIND_BITMAP 2

#ifdef __cplusplus
extern "C" {
#endif

uint32_t ordvec_abi_version(void);                          /* ordvec.h:142 */
const char *ordvec_version_string(void);                    /* ordvec.h:144 */
const char *ordvec_status_name(ordvec_status_t status);     /* ordvec.h:146 */
const char *ordvec_last_error(void);                        /* ordvec.h:148 */
ordvec_status_t ordvec_init(void);                          /* ordvec.h:150; also selects the CUDA device */
void ordvec_index_info_init(ordvec_index_info_t *info);     /* ordvec.h:160 */
void ordvec_search_params_init(ordvec_search_params_t *p);  /* ordvec.h:170 */
void ordvec_search_stats_init(ordvec_search_stats_t *s);    /* ordvec.h:180 */
ordvec_status_t ordvec_index_load(const char *path, uint64_t flags,
                                  ordvec_index_t **out);    /* ordvec.h:191; uploads codes to HBM */
ordvec_status_t ordvec_index_probe(const char *path, uint64_t flags,
                                   ordvec_index_info_t *info_out); /* ordvec.h:208 */
ordvec_status_t ordvec_index_info(const ordvec_index_t *index,
                                  ordvec_index_info_t *info_out);  /* ordvec.h:218 */
void ordvec_index_free(ordvec_index_t *index);              /* ordvec.h:228 */
ordvec_status_t ordvec_index_search(const ordvec_index_t *index,
                                    const ordvec_search_params_t *params,
                                    ordvec_hit_t *hits_out, uint64_t hits_capacity,
                                    uint64_t *returned_out,
                                    ordvec_search_stats_t *stats_out); /* ordvec.h:249-254 */

/* ===================== Part 2: B200 extensions ===================== */

/* Index kinds beyond ABI v1 (reported by ordvec_index_info). */
#define OVB_INDEX_KIND_SIGN_BITMAP 3  /* src/sign_bitmap.rs SignBitmap */
#define OVB_INDEX_KIND_FASTSCAN 4     /* src/fastscan.rs RankQuantFastscan */
#define OVB_INDEX_KIND_MULTIBUCKET 5  /* src/multi_bucket.rs MultiBucketBitmap */
#define OVB_INDEX_KIND_RANK 6         /* src/rank.rs Rank (u16 rank per coordinate) */

/* Empty device-resident indices; parameters validated as the reference's
 * constructors do (src/quant.rs:375-491, src/sign_bitmap.rs:113-165,
 * src/bitmap.rs:71-125, src/fastscan.rs:568-589, src/multi_bucket.rs:70-93,
 * src/rank.rs:316-324). */
ordvec_status_t ovb_rankquant_new(uint32_t dim, uint32_t bits, ordvec_index_t **out);
ordvec_status_t ovb_sign_bitmap_new(uint32_t dim, ordvec_index_t **out);
ordvec_status_t ovb_bitmap_new(uint32_t dim, uint32_t n_top, ordvec_index_t **out);
ordvec_status_t ovb_fastscan_new(uint32_t dim, ordvec_index_t **out);
ordvec_status_t ovb_multibucket_new(uint32_t dim, uint32_t bits, ordvec_index_t **out);
/* Rank: one u16 rank per coordinate, 2 * dim bytes per document; 2 <= dim <= 65535
 * (adds and searches run the device rank transform: dim <= 16384). */
ordvec_status_t ovb_rank_new(uint32_t dim, ordvec_index_t **out);

/* `add` (RankQuant::add src/quant.rs:587, SignBitmap::add src/sign_bitmap.rs:180,
 * Bitmap::add src/bitmap.rs:140, RankQuantFastscan::add src/fastscan.rs:597,
 * MultiBucketBitmap::add src/multi_bucket.rs:95, Rank::add src/rank.rs:335): n row-major f32 vectors,
 * host or device memory; encoded on the GPU.  Non-finite input is
 * rejected with BAD_ARGUMENT (the reference panics). */
ordvec_status_t ovb_index_add(ordvec_index_t *index, const float *vectors, uint64_t n);
ordvec_status_t ovb_index_add_device(ordvec_index_t *index, const float *d_vectors, uint64_t n);
/* Persisted-format loaders for the scan formats and Rank (.ovrq .ovbm .ovsb
 * .ovfs .ovr, src/rank_io.rs), with the reference loader's validation. */
ordvec_status_t ovb_index_load_any(const char *path, uint64_t flags, ordvec_index_t **out);
ordvec_status_t ovb_index_write(const ordvec_index_t *index, const char *path);
/* Codes in the reference's persisted payload layout (the bytes after the
 * file header), copied back from HBM. */
ordvec_status_t ovb_index_payload_bytes(const ordvec_index_t *index, uint64_t *bytes_out);
ordvec_status_t ovb_index_payload(const ordvec_index_t *index, void *out, uint64_t bytes);

/* Batched searches, host buffers, synchronous.  Output rows are
 * rectangular: nq x min(k, n) (rows underfull for subsets padded with
 * (-inf, -1)), ordered exactly as the reference orders them. */
/* RankQuant::search_asymmetric (src/quant.rs:713-847). */
ordvec_status_t ovb_rankquant_search(const ordvec_index_t *rq, const float *queries,
                                     uint64_t nq, uint64_t k, float *scores, int64_t *ids);
/* The same full search scored by the split-BF16 tensor-core scan (no
 * counterpart in the reference): rank codes exact in BF16, the query split
 * into hi + lo BF16 parts, f32 accumulation; dim must be a multiple of 64.
 * exact = 1 rescores in FP64 every candidate within twice the split error
 * bound of the k-th split score, giving ovb_rankquant_search's results
 * (ovb_rankquant_search itself takes this path for >= 64 queries);
 * exact = 0 returns the split-BF16 scores and their top-k. */
ordvec_status_t ovb_rankquant_search_split(const ordvec_index_t *rq, const float *queries,
                                           uint64_t nq, uint64_t k, uint32_t exact,
                                           float *scores, int64_t *ids);
/* Full searches on device buffers, stream-ordered on `stream` (a
 * cudaStream_t; queries nq x dim f32, results nq x min(k, n) as in the host
 * entry points; query finiteness is the caller's responsibility).  method
 * OVB_SEARCH_DEFAULT is the kind's `search` (RankQuant and Rank: symmetric;
 * Bitmap; RankQuantFastscan), OVB_SEARCH_ASYMMETRIC its `search_asymmetric`
 * (RankQuant, Rank).  Calls from one thread share its workspace and must be
 * ordered on one stream. */
/* Failure-path self-tests (no counterpart in the reference).  The tensor-core
 * kernels bound every mbarrier wait (about 1 s); a wait that gives up sets the
 * calling thread's error word, drains, frees its TMEM and returns, and the host
 * entry point then fails with ORDVEC_STATUS_INTERNAL.
 * ovb_selftest_bounded_wait runs that bounded wait on a barrier nothing
 * arrives at: *timed_out = 1 and *waited_ns its duration.
 * ovb_selftest_arm_tc_error sets the calling thread's error word, so that its
 * next search that runs a tensor-core kernel reports INTERNAL (and re-arms). */
ordvec_status_t ovb_selftest_bounded_wait(uint32_t *timed_out, uint64_t *waited_ns);
ordvec_status_t ovb_selftest_arm_tc_error(void);

#define OVB_SEARCH_DEFAULT 0u
#define OVB_SEARCH_ASYMMETRIC 1u
ordvec_status_t ovb_index_search_device(const ordvec_index_t *index, uint32_t method, const float *d_queries,
                                        uint64_t nq, uint64_t k, float *d_scores, int64_t *d_ids, void *stream);
/* RankQuant::search, symmetric (src/quant.rs:629-695): the query is
 * rank-transformed and bucketed like a document; score = sum_d
 * centre(q_bucket) * centre(d_bucket) / norm^2, the reference's values bit for
 * bit (the integer-valued sum is exact in f32 for b <= 4). */
ordvec_status_t ovb_rankquant_search_symmetric(const ordvec_index_t *rq, const float *queries,
                                               uint64_t nq, uint64_t k, float *scores, int64_t *ids);
/* Rank::search (src/rank.rs:364-419): Spearman correlation of the query's
 * ranks with each document's, exact integer sum, then * 0.25 / norm^2 in f32. */
ordvec_status_t ovb_rank_search(const ordvec_index_t *rank, const float *queries, uint64_t nq,
                                uint64_t k, float *scores, int64_t *ids);
/* Rank::search_asymmetric (src/rank.rs:420-482): L2-normalised f32 query
 * against the stored ranks, (sum_d q[d] rank[d] - mean sum_d q[d]) / norm with
 * the reference's sequential f32 sums. */
ordvec_status_t ovb_rank_search_asymmetric(const ordvec_index_t *rank, const float *queries,
                                           uint64_t nq, uint64_t k, float *scores, int64_t *ids);
/* Mixed batch (no counterpart in the reference): query i is searched in full
 * in indices[index_of_query[i]] (RankQuant indices of one dim, e.g. one
 * corpus at bits 1, 2 and 4) for its own k_of_query[i] <= k_max, all in one
 * call.  Output rows hold k_max entries: row i's first min(k_of_query[i], n)
 * are its top-k (score desc, id asc, the results ovb_rankquant_search gives),
 * the rest (-inf, -1).  Queries are grouped by index; each group on the
 * split-BF16 tensor-core path runs through a plan cached per (index, group
 * size, k): its first call tunes the scan's tile shape and records the
 * pipeline as a CUDA graph, later calls replay it (falling back to the exact
 * pipeline when the fixed candidate count is too small for a query).
 * OVB_MIXED_GRAPH=0 disables the plans. */
ordvec_status_t ovb_rankquant_search_mixed(const ordvec_index_t *const *indices,
                                           uint32_t n_indices, const uint32_t *index_of_query,
                                           const uint32_t *k_of_query, const float *queries,
                                           uint64_t nq, uint64_t k_max, float *scores,
                                           int64_t *ids);
/* The cached plan of (rq, group size nq, k): the tuned queries per tile of its
 * scan, its candidate count and how many times its graph was replayed.
 * BAD_ARGUMENT when no plan exists. */
ordvec_status_t ovb_mixed_plan_info(const ordvec_index_t *rq, uint64_t nq, uint64_t k,
                                    uint32_t *q_per_tile, uint64_t *candidates,
                                    uint64_t *replays);
/* RankQuant::search_asymmetric_subset_batched_serial_into (src/quant.rs:1336-1394):
 * CSR candidates (offsets[nq+1]), output nq x min(k, n). */
ordvec_status_t ovb_rankquant_search_subset(const ordvec_index_t *rq, const float *queries,
                                            uint64_t nq, const uint64_t *offsets,
                                            const uint32_t *candidates, uint64_t k,
                                            float *scores, int64_t *ids);
/* SignBitmap::top_m_candidates_batched_serial_csr (src/sign_bitmap.rs:453-483):
 * nq x min(m, n) ids, (hamming asc, id asc). */
ordvec_status_t ovb_sign_bitmap_top_m(const ordvec_index_t *sign, const float *queries,
                                      uint64_t nq, uint64_t m, uint32_t *candidates);
/* SignBitmap::score_all (src/sign_bitmap.rs:492-505): dim - hamming per row. */
ordvec_status_t ovb_sign_bitmap_score_all(const ordvec_index_t *sign, const float *query,
                                          uint32_t *scores);
/* Bitmap::search (src/bitmap.rs:196-242) and top_m_candidates_batched
 * (src/bitmap.rs:304-367). */
ordvec_status_t ovb_bitmap_search(const ordvec_index_t *bm, const float *queries, uint64_t nq,
                                  uint64_t k, float *scores, int64_t *ids);
ordvec_status_t ovb_bitmap_top_m(const ordvec_index_t *bm, const float *queries, uint64_t nq,
                                 uint64_t m, uint32_t *candidates);
/* RankQuantFastscan::search (src/fastscan.rs:630-634). */
ordvec_status_t ovb_fastscan_search(const ordvec_index_t *fs, const float *queries,
                                    uint64_t nq, uint64_t k, float *scores, int64_t *ids);
/* MultiBucketBitmap::top_m_bilinear over rank-bucketed query bitmaps
 * (src/multi_bucket.rs:122-251) with a caller weight matrix (nb x nb f32);
 * order (score desc, id asc). */
ordvec_status_t ovb_multibucket_top_m(const ordvec_index_t *mb, const float *queries,
                                      uint64_t nq, const float *weights, uint64_t m,
                                      uint32_t *candidates);

/* Fused two-stage pipelines: candidates stay in HBM between the stages.
 * stage1 = SignBitmap (sign probe, m = 0 selects the reference's default
 * TwoStageCandidatePolicy, src/quant.rs:234-262), RankQuantFastscan, Bitmap
 * or MultiBucketBitmap (diagonal weights); stage 2 = RankQuant asymmetric
 * subset rerank (src/quant.rs:1453-1498).  Output nq x min(k, m_eff). */
ordvec_status_t ovb_two_stage_search(const ordvec_index_t *rq, const ordvec_index_t *stage1,
                                     const float *queries, uint64_t nq, uint64_t m, uint64_t k,
                                     float *scores, int64_t *ids);
/* Same, device pointers, asynchronous on `stream` (a cudaStream_t). */
ordvec_status_t ovb_two_stage_search_device(const ordvec_index_t *rq,
                                            const ordvec_index_t *stage1,
                                            const float *d_queries, uint64_t nq, uint64_t m,
                                            uint64_t k, float *d_scores, int64_t *d_ids,
                                            void *stream);
/* How the two-stage pipelines rerank (no counterpart in the reference, whose
 * rerank is its asymmetric subset scorer, src/quant.rs:1126-1281):
 *   OVB_RERANK_AUTO       FP64 (the faster form at the measured shapes); with the
 *                         environment variable OVB_RERANK_TC=1, the split form
 *                         where the shape allows it (dim % 64 == 0,
 *                         16 <= dim*bits/8 <= 256 and a multiple of 16, >= 16
 *                         queries, m >= 4k + 64), else FP64
 *   OVB_RERANK_FP64       every candidate scored in FP64 (per-query tables)
 *   OVB_RERANK_SPLIT      split-BF16 scores (codes exact in BF16, query = hi + lo
 *                         BF16, f32 accumulation on tcgen05), then the top
 *                         2k + 32 by that score rescored in FP64 after a margin
 *                         test against the stated error bound: the same ids as
 *                         FP64 (a failed margin test reranks the batch in FP64)
 *   OVB_RERANK_SPLIT_RAW  the split-BF16 scores themselves, top-k by them (for
 *                         measuring the split's error against FP64)
 * The default calls (ovb_two_stage_search, _device, _profile) use AUTO. */
#define OVB_RERANK_AUTO 0u
#define OVB_RERANK_FP64 1u
#define OVB_RERANK_SPLIT 2u
#define OVB_RERANK_SPLIT_RAW 3u
/* ovb_two_stage_search_device with an explicit OVB_RERANK_* mode. */
ordvec_status_t ovb_two_stage_search_device_ex(const ordvec_index_t *rq,
                                               const ordvec_index_t *stage1,
                                               const float *d_queries, uint64_t nq, uint64_t m,
                                               uint64_t k, float *d_scores, int64_t *d_ids,
                                               void *stream, uint32_t rerank_mode);
/* Same as ovb_two_stage_search_device, synchronous, with CUDA events recorded
 * on `stream` between the pipeline stages; stage_ms[0..5] receives the device
 * time of: query prep, stage-1 candidate threshold (sample scan + select; 0
 * when the stage-1 scan keeps its full key matrix), stage-1 scan, stage-1
 * select, rerank scoring, final select (benchmark instrumentation). */
ordvec_status_t ovb_two_stage_profile(const ordvec_index_t *rq, const ordvec_index_t *stage1,
                                      const float *d_queries, uint64_t nq, uint64_t m,
                                      uint64_t k, float *d_scores, int64_t *d_ids, void *stream,
                                      float *stage_ms);
/* Allocation-free RankQuant full search (no counterpart in the reference):
 * same results as ovb_rankquant_search, but device pointers in and out,
 * asynchronous on `stream`, and no device allocation at all -- for callers
 * that may not call cudaMalloc (latency-bound serving threads, processes whose
 * device memory belongs to one budgeted allocator).  Intermediates live in a
 * fixed 32 MiB device array inside this library (held by every GPU that loads
 * it): requests needing more (nq*dim*4 + nq*n*4 + 2*nq*k*4 bytes, each part
 * rounded up to 256) or k > 4096 are rejected with BAD_ARGUMENT.  The first
 * call on a device looks up the array's device address; make it before any
 * stream capture, and do not use the entry point across a cudaDeviceReset
 * (the cached address would be stale).  Calls that overlap on the GPU share
 * the array and race.  Queries must be finite: they are not checked (that
 * would need a device-to-host read), and a non-finite query's ranking is
 * unspecified. */
ordvec_status_t ovb_rankquant_search_noalloc(const ordvec_index_t *rq, const float *d_queries,
                                             uint64_t nq, uint64_t k, float *d_scores,
                                             int64_t *d_ids, void *stream);
/* Number of kernel launches the last device/host search on this thread
 * issued (instrumentation for benchmarks). */
uint64_t ovb_last_launch_count(void);
/* Select the CUDA device this library's calls on the current thread use
 * (the library carries its own CUDA runtime, so a framework's current-device
 * setting does not reach it). */
ordvec_status_t ovb_set_device(int device);

/* Seeded synthetic corpus of the benchmark configurations: 256 clusters with
 * unit-norm N(0, I) centres, doc = centre + N(0, sigma^2) per coordinate,
 * L2-normalised; queries = a uniformly chosen doc + N(0, 0.1^2), renormalised.
 * xoshiro256** streams seeded by SplitMix64 per row, Box-Muller in f64.
 * Deterministic for any thread count.  planted (optional) receives the
 * source doc of each query. */
ordvec_status_t ovb_synth_docs(uint64_t seed, uint64_t first, uint64_t n, uint32_t dim,
                               float sigma, float *out);
ordvec_status_t ovb_synth_queries(uint64_t seed, uint64_t n_docs, uint64_t nq, uint32_t dim,
                                  float doc_sigma, float query_sigma, float *out,
                                  uint64_t *planted);

/* ---- Serving loop (no counterpart in the reference) ----------------------
 * A request server over device-resident indices.  Requests (a block of
 * queries, k, and m = stage-1 candidates) are queued by ovb_server_submit and
 * answered by worker threads, each with its own CUDA stream: a free worker
 * takes the oldest pending request and batches every other pending request of
 * the same route, k and m behind it (up to max_batch queries: continuous
 * batching), admits the batch when the device bytes of all batches in flight
 * stay within hbm_budget_bytes, and runs it while other workers' batches run
 * on their streams.  A request's results are the ones it gets alone: every
 * kernel scores a query independently of the others in its batch.  Before a
 * worker serves a route it sizes its buffers with two synthetic batches
 * (31 and max_batch queries, k = 100), so buffer growth (whose frees wait for
 * the whole device) does not stall batches in flight. */
typedef struct ovb_server ovb_server_t;

typedef struct ovb_server_config_t {
    uint64_t struct_size;      /* sizeof(ovb_server_config_t) */
    uint32_t workers;          /* concurrent batches (streams); 0 -> 2 */
    uint32_t max_batch;        /* queries per batch; 0 -> 1024 */
    uint64_t hbm_budget_bytes; /* device bytes of the batches in flight; 0 -> 4 GiB */
    uint64_t reserved[5];      /* must be zero */
} ovb_server_config_t;

typedef struct ovb_server_stats_t {
    uint64_t struct_size;       /* sizeof(ovb_server_stats_t) */
    uint64_t requests;          /* completed requests */
    uint64_t queries;           /* completed queries */
    uint64_t batches;           /* batches run */
    uint64_t peak_inflight_bytes;
    uint64_t max_concurrent_batches;
    double p50_ms, p99_ms, mean_ms; /* submit -> results ready, per request */
    uint64_t warm_workers;      /* workers whose buffers are sized for every route */
    uint64_t reserved[3];
} ovb_server_stats_t;

ordvec_status_t ovb_server_new(const ovb_server_config_t *config, ovb_server_t **out);
/* A route is a RankQuant index searched in full (stage1 NULL) or a
 * two-stage pair (stage-1 SignBitmap / Bitmap / FastScan / MultiBucket index
 * -> RankQuant rerank).  Indices must outlive the server. */
ordvec_status_t ovb_server_add_route(ovb_server_t *server, const ordvec_index_t *rq,
                                     const ordvec_index_t *stage1, uint32_t *route_out);
/* Copies nq x dim queries; m = 0 applies the default candidate policy.  Fails
 * fast on bad arguments or non-finite queries (NONFINITE_QUERY). */
ordvec_status_t ovb_server_submit(ovb_server_t *server, uint32_t route, const float *queries,
                                  uint64_t nq, uint64_t k, uint64_t m, uint64_t *ticket_out);
/* Blocks until the request is answered; writes nq x k_out scores and ids
 * (k_out = min(k, candidates); capacity = entries available in each array).
 * A ticket can be waited on once. */
ordvec_status_t ovb_server_wait(ovb_server_t *server, uint64_t ticket, float *scores,
                                int64_t *ids, uint64_t capacity, uint64_t *k_out,
                                double *latency_ms);
ordvec_status_t ovb_server_stats(ovb_server_t *server, ovb_server_stats_t *out);
/* Drains the queue (pending requests still run), joins the workers. */
void ovb_server_free(ovb_server_t *server);

#ifdef __cplusplus
}
#endif

#endif /* ORDVEC_B200_H */
