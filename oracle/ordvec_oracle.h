/*
 * ordvec_oracle.h -- CPU restatement of ordvec 0.6.0's compressed-scan path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker the parity tests,
 * the smoke test and the benchmark's CPU-baseline leg compare against.  It is
 * never linked into, loaded by, or called from the product library
 * (libordvec_b200.so) or its Python mirror.
 *
 * Every function restates the reference's algorithm (Rust, crate `ordvec`
 * 0.6.0); the doc comment beside each one names the reference file:line it
 * follows.  The reference cannot be compiled here (no Rust toolchain), so the
 * restatement is pinned against the reference's own literal known-answer
 * tests (tests/determinism_contract.rs, tests/persistence_compat.rs,
 * src/util.rs TopK literals, ordvec-ffi fixtures) and against the
 * sort-based oracle that tests/tiled_candgen.rs defines; see the golden
 * fixtures under tests/golden/.
 *
 * Conventions: all arrays are caller-allocated, row-major, little-endian.
 * `k`/`m` arguments are the caller's request; functions clamp exactly as the
 * reference does and return the effective count.
 */
#ifndef ORDVEC_ORACLE_H
#define ORDVEC_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

/* ---- math primitives (src/rank.rs, src/util.rs) ---- */
void orc_rank_transform(const float *v, uint32_t d, uint16_t *out);
uint32_t orc_rank_to_bucket(uint32_t rank, uint32_t d, uint32_t bits);
void orc_pack_buckets(const uint8_t *buckets, uint32_t d, uint32_t bits, uint8_t *out);
void orc_unpack_buckets(const uint8_t *packed, uint32_t d, uint32_t bits, uint8_t *out);
float orc_bucket_centre(uint32_t bucket, uint32_t bits);
float orc_rankquant_norm(uint32_t d, uint32_t bits);
void orc_l2_normalise(const float *v, uint32_t d, float *out);
uint64_t orc_policy_candidate_count(uint64_t min_candidates, uint64_t k_multiplier,
                                    int has_max, uint64_t max_candidates, uint64_t k,
                                    uint64_t search_space);

/* ---- encoders (the `add` paths) ---- */
void orc_rankquant_encode(const float *vecs, uint64_t n, uint32_t dim, uint32_t bits,
                          uint8_t *out);
void orc_sign_encode(const float *vecs, uint64_t n, uint32_t dim, uint64_t *out);
void orc_bitmap_encode(const float *vecs, uint64_t n, uint32_t dim, uint32_t n_top,
                       uint64_t *out);
void orc_bitmap_query_fp32(const float *q, uint32_t dim, uint32_t n_top, uint64_t *out);
void orc_fastscan_pack(const float *vecs, uint64_t n, uint32_t dim, uint8_t *out);
void orc_multibucket_encode(const float *vecs, uint64_t n, uint32_t dim, uint32_t bits,
                            uint64_t *out);

/* ---- TopK (src/util.rs:386-600), exposed for the literal tests ---- */
typedef struct orc_topk orc_topk;
orc_topk *orc_topk_new(uint64_t k, const uint32_t *tie_keys, uint64_t n_tie_keys);
void orc_topk_set_score_offset(orc_topk *t, float offset);
void orc_topk_insert(orc_topk *t, float score, uint64_t idx);
void orc_topk_finalize(const orc_topk *t, float *scores, int64_t *indices, uint64_t len);
void orc_topk_free(orc_topk *t);

/* ---- RankQuant symmetric search; Rank (u16) index ---- */
uint64_t orc_rq_search_sym(const uint8_t *packed, uint64_t n, uint32_t dim, uint32_t bits,
                           const float *queries, uint64_t nq, uint64_t k, float *scores, int64_t *ids);
void orc_rank_encode(const float *vecs, uint64_t n, uint32_t dim, uint16_t *out);
float orc_rank_norm(uint32_t d);
uint64_t orc_rank_search_sym(const uint16_t *ranks, uint64_t n, uint32_t dim, const float *queries,
                             uint64_t nq, uint64_t k, float *scores, int64_t *ids);
uint64_t orc_rank_search_asym(const uint16_t *ranks, uint64_t n, uint32_t dim, const float *queries,
                              uint64_t nq, uint64_t k, float *scores, int64_t *ids);

/* ---- RankQuant asymmetric search (scalar LUT tier) ---- */
uint64_t orc_rq_search_asym(const uint8_t *packed, uint64_t n, uint32_t dim, uint32_t bits,
                            const float *queries, uint64_t nq, uint64_t k, float *scores,
                            int64_t *ids);
void orc_rq_scores_f64(const uint8_t *packed, uint64_t n, uint32_t dim, uint32_t bits,
                       const float *query, double *out);
void orc_rq_scores_f64_subset(const uint8_t *packed, uint32_t dim, uint32_t bits,
                              const float *query, const uint32_t *cands, uint64_t m,
                              double *out);
uint64_t orc_rq_subset(const uint8_t *packed, uint64_t n, uint32_t dim, uint32_t bits,
                       const float *query, const uint32_t *cands, uint64_t m, uint64_t k,
                       float *scores, int64_t *ids);
uint64_t orc_rq_subset_batched(const uint8_t *packed, uint64_t n, uint32_t dim,
                               uint32_t bits, const float *queries, uint64_t nq,
                               const uint64_t *offsets, const uint32_t *cands, uint64_t k,
                               float *scores, int64_t *ids);

/* ---- SignBitmap ---- */
void orc_sign_query(const float *q, uint32_t dim, uint64_t *out);
void orc_sign_hamming_all(const uint64_t *words, uint64_t n, uint32_t dim, const float *q,
                          uint32_t *out);
uint64_t orc_sign_top_m(const uint64_t *words, uint64_t n, uint32_t dim, const float *q,
                        uint64_t m, uint32_t *out);
uint64_t orc_sign_top_m_streamed(const uint64_t *words, uint64_t n, uint32_t dim,
                                 const float *queries, uint64_t nq, uint64_t m,
                                 uint32_t *out);

/* ---- Bitmap (constant weight) ---- */
void orc_bitmap_overlap_all(const uint64_t *words, uint64_t n, uint32_t dim,
                            const uint64_t *qbm, uint32_t *out);
uint64_t orc_bitmap_top_m(const uint64_t *words, uint64_t n, uint32_t dim, uint32_t n_top,
                          const float *q, uint64_t m, uint32_t *out);
uint64_t orc_bitmap_search(const uint64_t *words, uint64_t n, uint32_t dim, uint32_t n_top,
                           const float *queries, uint64_t nq, uint64_t k, float *scores,
                           int64_t *ids);
uint64_t orc_bitmap_search_subset(const uint64_t *words, uint64_t n, uint32_t dim,
                                  uint32_t n_top, const float *query, const uint32_t *ids_in,
                                  uint64_t m, uint64_t k, float *scores, int64_t *ids);

/* ---- FastScan b=2 ---- */
void orc_fastscan_query(const float *q_unit, uint32_t dim, uint8_t *lut, float *bias_sum,
                        float *inv_q);
void orc_fastscan_scores(const uint8_t *blocks, uint64_t n, uint32_t dim,
                         const float *query, float *out);
uint64_t orc_fastscan_search(const uint8_t *blocks, uint64_t n, uint32_t dim,
                             const float *queries, uint64_t nq, uint64_t k, float *scores,
                             int64_t *ids);

/* ---- MultiBucketBitmap ---- */
void orc_multibucket_query(const float *q, uint32_t dim, uint32_t bits, uint64_t *out);
void orc_multibucket_weights(uint32_t bits, int kind, uint32_t half_width, float *w);
void orc_multibucket_scores(const uint64_t *words, uint64_t n, uint32_t dim, uint32_t bits,
                            const uint64_t *qbm, const float *w, float *out);
uint64_t orc_multibucket_top_m(const uint64_t *words, uint64_t n, uint32_t dim,
                               uint32_t bits, const uint64_t *qbm, const float *w,
                               uint64_t m, uint32_t *out);

/* ---- test-corpus helper (tests/tiled_candgen.rs XorShift) ---- */
void orc_xorshift_f32(uint64_t seed, uint64_t count, float *out);

/* ---- benchmark corpus generator and a one-pass host encoder ---- */
void orc_synth_docs(uint64_t seed, uint64_t first, uint64_t n, uint32_t dim, float sigma, float *out);
void orc_synth_queries(uint64_t seed, uint64_t n_docs, uint64_t nq, uint32_t dim, float doc_sigma,
                       float query_sigma, float *out, uint64_t *planted);
void orc_encode_bitmap_rankquant(const float *vecs, uint64_t n, uint32_t dim, uint32_t n_top,
                                 uint32_t bits, uint64_t *bitmap_out, uint8_t *rq_out);

/* ---- AVX-512 + OpenMP restatement, used only as the timed CPU baseline ---- */
int orc_avx512_available(void);
int orc_max_threads(void);
void orc_cpu_fastscan_two_stage(const uint8_t *blocks, const uint8_t *packed_b2, uint64_t n,
                                uint32_t dim, const float *queries, uint64_t nq,
                                uint64_t n_candidates, uint64_t k, int nthreads,
                                float *scores, int64_t *ids, uint32_t *cands_out);
void orc_cpu_sign_two_stage(const uint64_t *sign_words, const uint8_t *packed, uint64_t n,
                            uint32_t dim, uint32_t bits, const float *queries, uint64_t nq,
                            uint64_t m, uint64_t k, int nthreads, float *scores,
                            int64_t *ids);
void orc_cpu_bitmap_two_stage(const uint64_t *bitmap_words, const uint8_t *packed, uint64_t n,
                              uint32_t dim, uint32_t n_top, uint32_t bits, const float *queries,
                              uint64_t nq, uint64_t m, uint64_t k, int nthreads, float *scores,
                              int64_t *ids, uint32_t *cands_out);
void orc_cpu_rq_search_asym(const uint8_t *packed, uint64_t n, uint32_t dim, uint32_t bits,
                            const float *queries, uint64_t nq, uint64_t k, int nthreads,
                            float *scores, int64_t *ids);

#ifdef __cplusplus
}
#endif
#endif
