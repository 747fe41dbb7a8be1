/*
 * ordvec_oracle.c -- CPU restatement of ordvec 0.6.0's compressed-scan path.
 *
 * TEST INFRASTRUCTURE ONLY (see ordvec_oracle.h).  The product library never
 * links or calls this file.  Compiled with -ffp-contract=off and without
 * -ffast-math so every f32 operation rounds exactly as the reference's Rust
 * code does (Rust never contracts a*b+c into an FMA); the AVX-512 kernels
 * below use explicit FMA intrinsics exactly where the reference does.
 *
 * Parity pins: tests/test_oracle_golden.py checks this file against the
 * reference's literal known-answer tests and the tiled-candgen sort oracle.
 */
#define _GNU_SOURCE
#include "ordvec_oracle.h"

#include <immintrin.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ------------------------------------------------------------------ */
/* helpers                                                            */
/* ------------------------------------------------------------------ */

/* f32::total_cmp as an order-preserving signed key (core::f32::total_cmp). */
static inline int32_t total_key(float f) {
    int32_t x;
    memcpy(&x, &f, 4);
    x ^= (int32_t)(((uint32_t)(x >> 31)) >> 1);
    return x;
}
static inline int total_cmp(float a, float b) {
    int32_t x = total_key(a), y = total_key(b);
    return (x > y) - (x < y);
}

typedef struct { float v; uint32_t i; } vi_t;

static int cmp_u64(const void *pa, const void *pb) {
    uint64_t a = *(const uint64_t *)pa, b = *(const uint64_t *)pb;
    return (a > b) - (a < b);
}

/* ------------------------------------------------------------------ */
/* math primitives                                                    */
/* ------------------------------------------------------------------ */

/* rank_transform (src/rank.rs:38-53): argsort with the index tiebreak,
 * then invert the permutation.  The order of cmp_finite_f32_then_index
 * (src/util.rs:19-30: values equal under ==, so -0.0 == +0.0, tie by index,
 * otherwise total_cmp) is the unsigned order of the
 * total_cmp key with -0.0 folded onto +0.0, broken by index; a stable LSD
 * radix sort over that 32-bit key, fed in index order, produces it without
 * a comparison callback (the 10M-row benchmark corpora are encoded on the
 * host with it).  NaN inputs, which the reference rejects, are ordered by
 * their bit patterns. */
void orc_rank_transform(const float *v, uint32_t d, uint16_t *out) {
    if (d == 0) return;
    uint32_t *key = (uint32_t *)malloc(4 * (size_t)d * 2);
    uint16_t *idx = (uint16_t *)malloc(2 * (size_t)d * 2);
    uint32_t *k2 = key + d;
    uint16_t *i2 = idx + d;
    for (uint32_t i = 0; i < d; i++) {
        float f = v[i] == 0.0f ? 0.0f : v[i];
        key[i] = (uint32_t)total_key(f) ^ 0x80000000u;
        idx[i] = (uint16_t)i;
    }
    for (int pass = 0; pass < 4; pass++) {
        uint32_t shift = 8u * (uint32_t)pass, cnt[257] = {0};
        for (uint32_t i = 0; i < d; i++) cnt[((key[i] >> shift) & 0xFF) + 1]++;
        if (cnt[((key[0] >> shift) & 0xFF) + 1] == d) continue; /* one digit value: order unchanged */
        for (int b = 0; b < 256; b++) cnt[b + 1] += cnt[b];
        for (uint32_t i = 0; i < d; i++) {
            uint32_t p = cnt[(key[i] >> shift) & 0xFF]++;
            k2[p] = key[i];
            i2[p] = idx[i];
        }
        uint32_t *tk = key; key = k2; k2 = tk;
        uint16_t *ti = idx; idx = i2; i2 = ti;
    }
    for (uint32_t r = 0; r < d; r++) out[idx[r]] = (uint16_t)r;
    free(key < k2 ? key : k2);
    free(idx < i2 ? idx : i2);
}

/* rank_to_bucket (src/rank.rs:89-95): floor(rank * 2^bits / d) in u64. */
uint32_t orc_rank_to_bucket(uint32_t rank, uint32_t d, uint32_t bits) {
    return (uint32_t)(((uint64_t)rank * ((uint64_t)1 << bits)) / (uint64_t)d);
}

/* pack_buckets (src/rank.rs:128-156): MSB-first, code 0 in the top bits. */
void orc_pack_buckets(const uint8_t *buckets, uint32_t d, uint32_t bits, uint8_t *out) {
    uint32_t cpb = 8 / bits;
    memset(out, 0, d / cpb);
    for (uint32_t i = 0; i < d; i++) {
        uint32_t shift = (cpb - 1 - i % cpb) * bits;
        out[i / cpb] |= (uint8_t)(buckets[i] << shift);
    }
}

/* unpack_buckets (src/rank.rs:161-178). */
void orc_unpack_buckets(const uint8_t *packed, uint32_t d, uint32_t bits, uint8_t *out) {
    uint32_t cpb = 8 / bits;
    uint8_t mask = (uint8_t)((1u << bits) - 1);
    for (uint32_t i = 0; i < d; i++) {
        uint32_t shift = (cpb - 1 - i % cpb) * bits;
        out[i] = (uint8_t)((packed[i / cpb] >> shift) & mask);
    }
}

/* bucket_centre (src/rank.rs:220-228): bucket as f32 - (n - 1.0) / 2.0. */
float orc_bucket_centre(uint32_t bucket, uint32_t bits) {
    float n = (float)(1u << bits);
    return (float)bucket - (n - 1.0f) / 2.0f;
}

/* rankquant_norm (src/rank.rs:275-280): f64 closed form, narrowed to f32. */
float orc_rankquant_norm(uint32_t d, uint32_t bits) {
    double n = (double)(1u << bits);
    double var = (n * n - 1.0) / 12.0;
    return (float)sqrt((double)d * var);
}

/* l2_normalise (src/util.rs:93-101): sequential f32 sum of squares, sqrt,
 * reciprocal, multiply; norm <= 1e-12 yields the zero vector. */
void orc_l2_normalise(const float *v, uint32_t d, float *out) {
    float s = -0.0f;
    for (uint32_t i = 0; i < d; i++) {
        float sq = v[i] * v[i];
        s = s + sq;
    }
    float norm = sqrtf(s);
    if (norm <= 1e-12f) {
        for (uint32_t i = 0; i < d; i++) out[i] = 0.0f;
    } else {
        float inv = 1.0f / norm;
        for (uint32_t i = 0; i < d; i++) out[i] = v[i] * inv;
    }
}

/* TwoStageCandidatePolicy::candidate_count (src/quant.rs:242-251). */
uint64_t orc_policy_candidate_count(uint64_t min_candidates, uint64_t k_multiplier,
                                    int has_max, uint64_t max_candidates, uint64_t k,
                                    uint64_t search_space) {
    if (k == 0 || search_space == 0) return 0;
    uint64_t prod;
    if (__builtin_mul_overflow(k, k_multiplier, &prod)) prod = UINT64_MAX;
    uint64_t count = min_candidates > prod ? min_candidates : prod;
    if (has_max && max_candidates < count) count = max_candidates;
    return count < search_space ? count : search_space;
}

/* ------------------------------------------------------------------ */
/* encoders                                                           */
/* ------------------------------------------------------------------ */

/* RankQuant::add (src/quant.rs:587-614): rank -> bucket -> pack per row. */
void orc_rankquant_encode(const float *vecs, uint64_t n, uint32_t dim, uint32_t bits,
                          uint8_t *out) {
    uint32_t bpv = dim * bits / 8;
#pragma omp parallel
    {
        uint16_t *r = (uint16_t *)malloc(2 * dim);
        uint8_t *b = (uint8_t *)malloc(dim);
#pragma omp for schedule(static)
        for (int64_t i = 0; i < (int64_t)n; i++) {
            orc_rank_transform(vecs + (uint64_t)i * dim, dim, r);
            for (uint32_t j = 0; j < dim; j++) b[j] = (uint8_t)orc_rank_to_bucket(r[j], dim, bits);
            orc_pack_buckets(b, dim, bits, out + (uint64_t)i * bpv);
        }
        free(r);
        free(b);
    }
}

/* SignBitmap::add (src/sign_bitmap.rs:180-200): bit j of word j/64 set iff
 * v[j] > 0.0 (so -0.0 and +0.0 are unset). */
void orc_sign_encode(const float *vecs, uint64_t n, uint32_t dim, uint64_t *out) {
    uint32_t qpv = dim / 64;
    memset(out, 0, n * qpv * 8);
    for (uint64_t i = 0; i < n; i++)
        for (uint32_t j = 0; j < dim; j++)
            if (vecs[i * dim + j] > 0.0f) out[i * qpv + j / 64] |= (uint64_t)1 << (j % 64);
}

/* SignBitmap::build_query_bitmap (src/sign_bitmap.rs:204-214). */
void orc_sign_query(const float *q, uint32_t dim, uint64_t *out) { orc_sign_encode(q, 1, dim, out); }

/* Bitmap::add (src/bitmap.rs:140-162): bit j set iff rank[j] >= dim - n_top. */
void orc_bitmap_encode(const float *vecs, uint64_t n, uint32_t dim, uint32_t n_top,
                       uint64_t *out) {
    uint32_t qpv = dim / 64;
    memset(out, 0, n * qpv * 8);
    uint16_t cutoff = (uint16_t)(dim - n_top);
#pragma omp parallel
    {
        uint16_t *r = (uint16_t *)malloc(2 * dim);
#pragma omp for schedule(static)
        for (int64_t i = 0; i < (int64_t)n; i++) {
            orc_rank_transform(vecs + (uint64_t)i * dim, dim, r);
            for (uint32_t j = 0; j < dim; j++)
                if (r[j] >= cutoff) out[(uint64_t)i * qpv + j / 64] |= (uint64_t)1 << (j % 64);
        }
        free(r);
    }
}

/* stable sort by value descending under partial_cmp (equal -> original order) */
static int cmp_desc_stable(const void *pa, const void *pb) {
    const vi_t *a = (const vi_t *)pa, *b = (const vi_t *)pb;
    if (a->v > b->v) return -1;
    if (a->v < b->v) return 1;
    return (a->i > b->i) - (a->i < b->i);
}

/* Bitmap::build_query_bitmap_fp32 (src/bitmap.rs:170-187): the n_top largest
 * coordinates by value, stable sort (ties keep the lower index first). */
void orc_bitmap_query_fp32(const float *q, uint32_t dim, uint32_t n_top, uint64_t *out) {
    vi_t *o = (vi_t *)malloc(sizeof(vi_t) * dim);
    for (uint32_t i = 0; i < dim; i++) { o[i].v = q[i]; o[i].i = i; }
    qsort(o, dim, sizeof(vi_t), cmp_desc_stable);
    memset(out, 0, (dim / 64) * 8);
    for (uint32_t t = 0; t < n_top; t++) out[o[t].i / 64] |= (uint64_t)1 << (o[t].i % 64);
    free(o);
}

/* RankQuantFastscan::add + pack_fastscan_b2 (src/fastscan.rs:87-110, 597-623):
 * nibble = (b[2p] << 2) | b[2p+1] at [block][pair][lane32], zero-padded tail. */
void orc_fastscan_pack(const float *vecs, uint64_t n, uint32_t dim, uint8_t *out) {
    uint32_t pairs = dim / 2;
    uint64_t n_blocks = (n + 31) / 32;
    memset(out, 0, n_blocks * pairs * 32);
#pragma omp parallel
    {
        uint16_t *r = (uint16_t *)malloc(2 * dim);
#pragma omp for schedule(static)
        for (int64_t i = 0; i < (int64_t)n; i++) {
            orc_rank_transform(vecs + (uint64_t)i * dim, dim, r);
            uint64_t blk = (uint64_t)i / 32, lane = (uint64_t)i % 32;
            for (uint32_t p = 0; p < pairs; p++) {
                uint32_t a = orc_rank_to_bucket(r[2 * p], dim, 2) & 3;
                uint32_t c = orc_rank_to_bucket(r[2 * p + 1], dim, 2) & 3;
                out[blk * pairs * 32 + (uint64_t)p * 32 + lane] = (uint8_t)((a << 2) | c);
            }
        }
        free(r);
    }
}

/* MultiBucketBitmap::add (src/multi_bucket.rs:95-117): one bitmap per bucket,
 * layout [doc][bucket][word]. */
void orc_multibucket_encode(const float *vecs, uint64_t n, uint32_t dim, uint32_t bits,
                            uint64_t *out) {
    uint32_t qpb = dim / 64, nb = 1u << bits;
    memset(out, 0, n * nb * qpb * 8);
#pragma omp parallel
    {
        uint16_t *r = (uint16_t *)malloc(2 * dim);
#pragma omp for schedule(static)
        for (int64_t i = 0; i < (int64_t)n; i++) {
            orc_rank_transform(vecs + (uint64_t)i * dim, dim, r);
            uint64_t *row = out + (uint64_t)i * nb * qpb;
            for (uint32_t j = 0; j < dim; j++) {
                uint32_t b = orc_rank_to_bucket(r[j], dim, bits);
                row[b * qpb + j / 64] |= (uint64_t)1 << (j % 64);
            }
        }
        free(r);
    }
}

/* MultiBucketBitmap::query_bitmaps_from_ranks (src/multi_bucket.rs:122-137). */
void orc_multibucket_query(const float *q, uint32_t dim, uint32_t bits, uint64_t *out) {
    orc_multibucket_encode(q, 1, dim, bits, out);
}

/* ------------------------------------------------------------------ */
/* TopK (src/util.rs:386-600)                                         */
/* ------------------------------------------------------------------ */

struct orc_topk {
    uint64_t k, filled, worst_pos, n_tie;
    float *scores;
    int64_t *indices, *tie_keys, *tie_by_index;
    float score_offset, worst_val;
    int64_t worst_tie;
};

orc_topk *orc_topk_new(uint64_t k, const uint32_t *tie_keys, uint64_t n_tie_keys) {
    orc_topk *t = (orc_topk *)calloc(1, sizeof(orc_topk));
    t->k = k;
    t->scores = (float *)malloc(sizeof(float) * (k ? k : 1));
    t->indices = (int64_t *)malloc(8 * (k ? k : 1));
    t->tie_keys = (int64_t *)malloc(8 * (k ? k : 1));
    for (uint64_t i = 0; i < k; i++) {
        t->scores[i] = -INFINITY;
        t->indices[i] = -1;
        t->tie_keys[i] = INT64_MAX;
    }
    if (tie_keys) {
        t->n_tie = n_tie_keys;
        t->tie_by_index = (int64_t *)malloc(8 * (n_tie_keys ? n_tie_keys : 1));
        for (uint64_t i = 0; i < n_tie_keys; i++) t->tie_by_index[i] = tie_keys[i];
    }
    t->worst_val = INFINITY;
    t->worst_tie = INT64_MAX;
    return t;
}

void orc_topk_free(orc_topk *t) {
    if (!t) return;
    free(t->scores);
    free(t->indices);
    free(t->tie_keys);
    free(t->tie_by_index);
    free(t);
}

void orc_topk_set_score_offset(orc_topk *t, float offset) { t->score_offset = offset; }

/* recompute_worst (src/util.rs:499-520): lowest score, then highest tie key. */
static void topk_recompute_worst(orc_topk *t) {
    float wv = INFINITY;
    int64_t wt = INT64_MIN;
    uint64_t wp = 0;
    for (uint64_t i = 0; i < t->filled; i++) {
        int c = total_cmp(t->scores[i], wv);
        int worse = c < 0 || (c == 0 && t->tie_keys[i] > wt);
        if (worse) { wv = t->scores[i]; wt = t->tie_keys[i]; wp = i; }
    }
    t->worst_val = wv;
    t->worst_tie = wt;
    t->worst_pos = wp;
}

/* maybe_insert (src/util.rs:451-494): offset applied before the compare. */
void orc_topk_insert(orc_topk *t, float score, uint64_t idx) {
    score = score + t->score_offset;
    int64_t id = (int64_t)idx;
    int64_t tie = t->tie_by_index ? t->tie_by_index[idx] : id;
    if (t->filled < t->k) {
        t->scores[t->filled] = score;
        t->indices[t->filled] = id;
        t->tie_keys[t->filled] = tie;
        t->filled++;
        if (t->filled == t->k) topk_recompute_worst(t);
    } else {
        int c = total_cmp(score, t->worst_val);
        int better = c > 0 || (c == 0 && tie < t->worst_tie);
        if (better) {
            t->scores[t->worst_pos] = score;
            t->indices[t->worst_pos] = id;
            t->tie_keys[t->worst_pos] = tie;
            topk_recompute_worst(t);
        }
    }
}

typedef struct { float s; int64_t i, t; uint64_t slot; } fin_t;
static int cmp_fin(const void *pa, const void *pb) {
    const fin_t *a = (const fin_t *)pa, *b = (const fin_t *)pb;
    int c = total_cmp(b->s, a->s);
    if (c) return c;
    if (a->t != b->t) return (a->t > b->t) - (a->t < b->t);
    return (a->slot > b->slot) - (a->slot < b->slot);
}

/* finalize_into (src/util.rs:547-600): sort (score desc, tie asc, slot asc),
 * pad with (-inf, -1). */
void orc_topk_finalize(const orc_topk *t, float *scores, int64_t *indices, uint64_t len) {
    for (uint64_t i = 0; i < len; i++) { scores[i] = -INFINITY; indices[i] = -1; }
    fin_t *o = (fin_t *)malloc(sizeof(fin_t) * (t->filled ? t->filled : 1));
    for (uint64_t i = 0; i < t->filled; i++) {
        o[i].s = t->scores[i];
        o[i].i = t->indices[i];
        o[i].t = t->tie_keys[i];
        o[i].slot = i;
    }
    qsort(o, t->filled, sizeof(fin_t), cmp_fin);
    for (uint64_t i = 0; i < t->filled && i < len; i++) {
        scores[i] = o[i].s;
        indices[i] = o[i].i;
    }
    free(o);
}

/* ------------------------------------------------------------------ */
/* RankQuant asymmetric scoring                                       */
/* ------------------------------------------------------------------ */

/* build_asym_lut_into (src/quant_kernels.rs:39-53). */
static float *build_asym_lut(const float *q_unit, uint32_t dim, uint32_t bits) {
    uint32_t nb = 1u << bits;
    float *lut = (float *)malloc(sizeof(float) * dim * nb);
    for (uint32_t d = 0; d < dim; d++)
        for (uint32_t b = 0; b < nb; b++) lut[d * nb + b] = q_unit[d] * orc_bucket_centre(b, bits);
    return lut;
}

/* scan_b{1,2,4}_to_topk (src/quant_kernels.rs:89-160): sequential f32 LUT
 * sum per document in code order, then acc * scale into the TopK. */
static float lut_doc_score(const uint8_t *doc, uint32_t dim, uint32_t bits, const float *lut) {
    float acc = 0.0f;
    uint32_t bpv = dim * bits / 8;
    if (bits == 1) {
        for (uint32_t g = 0; g < bpv; g++) {
            uint32_t base = g * 8 * 2;
            for (int i = 0; i < 8; i++) acc += lut[base + 2 * i + ((doc[g] >> (7 - i)) & 1)];
        }
    } else if (bits == 2) {
        for (uint32_t g = 0; g < bpv; g++) {
            uint32_t base = g * 4 * 4;
            for (int i = 0; i < 4; i++) acc += lut[base + 4 * i + ((doc[g] >> (6 - 2 * i)) & 3)];
        }
    } else {
        for (uint32_t g = 0; g < bpv; g++) {
            uint32_t base = g * 2 * 16;
            acc += lut[base + ((doc[g] >> 4) & 0xF)];
            acc += lut[base + 16 + (doc[g] & 0xF)];
        }
    }
    return acc;
}

/* RankQuant::search_asymmetric, scalar LUT tier (src/quant.rs:713-847,
 * src/quant_kernels.rs:23-160).  Writes nq * min(k, n) results. */
uint64_t orc_rq_search_asym(const uint8_t *packed, uint64_t n, uint32_t dim, uint32_t bits,
                            const float *queries, uint64_t nq, uint64_t k, float *scores,
                            int64_t *ids) {
    uint64_t ke = k < n ? k : n;
    if (ke == 0) return 0;
    float inv_norm = 1.0f / orc_rankquant_norm(dim, bits);
    uint32_t bpv = dim * bits / 8;
    float *qu = (float *)malloc(sizeof(float) * dim);
    for (uint64_t qi = 0; qi < nq; qi++) {
        orc_l2_normalise(queries + qi * dim, dim, qu);
        float *lut = build_asym_lut(qu, dim, bits);
        orc_topk *t = orc_topk_new(ke, NULL, 0);
        for (uint64_t di = 0; di < n; di++)
            orc_topk_insert(t, lut_doc_score(packed + di * bpv, dim, bits, lut) * inv_norm, di);
        orc_topk_finalize(t, scores + qi * ke, ids + qi * ke, ke);
        orc_topk_free(t);
        free(lut);
    }
    free(qu);
    return ke;
}

/* RankQuant::search, symmetric (src/quant.rs:629-695): the query is
 * rank-transformed and bucketed like a document; LUT[d][b] =
 * bucket_centre(q_bucket[d]) * bucket_centre(b); the per-document sum is the
 * scan_b{1,2,4}_to_topk sequential f32 LUT sum, times 1 / (norm * norm). */
uint64_t orc_rq_search_sym(const uint8_t *packed, uint64_t n, uint32_t dim, uint32_t bits,
                           const float *queries, uint64_t nq, uint64_t k, float *scores, int64_t *ids) {
    uint64_t ke = k < n ? k : n;
    if (ke == 0) return 0;
    float norm = orc_rankquant_norm(dim, bits);
    float inv_norm_sq = 1.0f / (norm * norm);
    uint32_t bpv = dim * bits / 8, nb = 1u << bits;
    uint16_t *qr = (uint16_t *)malloc(sizeof(uint16_t) * dim);
    float *lut = (float *)malloc(sizeof(float) * (size_t)dim * nb);
    for (uint64_t qi = 0; qi < nq; qi++) {
        orc_rank_transform(queries + qi * dim, dim, qr);
        for (uint32_t d = 0; d < dim; d++) {
            float qc = orc_bucket_centre(orc_rank_to_bucket(qr[d], dim, bits), bits);
            for (uint32_t b = 0; b < nb; b++) lut[d * nb + b] = qc * orc_bucket_centre(b, bits);
        }
        orc_topk *t = orc_topk_new(ke, NULL, 0);
        for (uint64_t di = 0; di < n; di++)
            orc_topk_insert(t, lut_doc_score(packed + di * bpv, dim, bits, lut) * inv_norm_sq, di);
        orc_topk_finalize(t, scores + qi * ke, ids + qi * ke, ke);
        orc_topk_free(t);
    }
    free(lut);
    free(qr);
    return ke;
}

/* Rank (src/rank.rs:283-482): one u16 rank per coordinate. */
void orc_rank_encode(const float *vecs, uint64_t n, uint32_t dim, uint16_t *out) {
    for (uint64_t i = 0; i < n; i++) orc_rank_transform(vecs + i * dim, dim, out + i * dim);
}

/* rank_norm (src/rank.rs:249-252): f64 closed form, narrowed to f32. */
float orc_rank_norm(uint32_t d) {
    double x = (double)d;
    return (float)sqrt(x * (x * x - 1.0) / 12.0);
}

/* Rank::search (src/rank.rs:364-419): Spearman in exact integers,
 * acc = sum (2 q_r - (D - 1)) (2 d_r - (D - 1)), score = (acc as f32) * 0.25
 * * (1 / (norm * norm)), left to right in f32. */
uint64_t orc_rank_search_sym(const uint16_t *ranks, uint64_t n, uint32_t dim, const float *queries,
                             uint64_t nq, uint64_t k, float *scores, int64_t *ids) {
    uint64_t ke = k < n ? k : n;
    if (ke == 0) return 0;
    float norm = orc_rank_norm(dim);
    float inv_norm_sq = 1.0f / (norm * norm);
    int32_t mean_2x = (int32_t)dim - 1;
    uint16_t *qr = (uint16_t *)malloc(sizeof(uint16_t) * dim);
    for (uint64_t qi = 0; qi < nq; qi++) {
        orc_rank_transform(queries + qi * dim, dim, qr);
        orc_topk *t = orc_topk_new(ke, NULL, 0);
        for (uint64_t di = 0; di < n; di++) {
            const uint16_t *doc = ranks + di * dim;
            int64_t acc = 0;
            for (uint32_t d = 0; d < dim; d++)
                acc += (int64_t)(2 * (int32_t)qr[d] - mean_2x) * (int64_t)(2 * (int32_t)doc[d] - mean_2x);
            orc_topk_insert(t, (float)acc * 0.25f * inv_norm_sq, di);
        }
        orc_topk_finalize(t, scores + qi * ke, ids + qi * ke, ke);
        orc_topk_free(t);
    }
    free(qr);
    return ke;
}

/* Rank::search_asymmetric (src/rank.rs:420-482): q_unit = l2_normalise(q),
 * q_sum = sequential f32 sum, acc = sequential f32 sum of q_unit[d] * rank,
 * score = (acc - mean * q_sum) * (1 / norm), mean = (D - 1) / 2 in f32. */
uint64_t orc_rank_search_asym(const uint16_t *ranks, uint64_t n, uint32_t dim, const float *queries,
                              uint64_t nq, uint64_t k, float *scores, int64_t *ids) {
    uint64_t ke = k < n ? k : n;
    if (ke == 0) return 0;
    float inv_norm = 1.0f / orc_rank_norm(dim);
    float mean = ((float)dim - 1.0f) / 2.0f;
    float *qu = (float *)malloc(sizeof(float) * dim);
    for (uint64_t qi = 0; qi < nq; qi++) {
        orc_l2_normalise(queries + qi * dim, dim, qu);
        float q_sum = -0.0f;
        for (uint32_t d = 0; d < dim; d++) q_sum += qu[d];
        orc_topk *t = orc_topk_new(ke, NULL, 0);
        for (uint64_t di = 0; di < n; di++) {
            const uint16_t *doc = ranks + di * dim;
            float acc = 0.0f;
            for (uint32_t d = 0; d < dim; d++) acc += qu[d] * (float)doc[d];
            orc_topk_insert(t, (acc - mean * q_sum) * inv_norm, di);
        }
        orc_topk_finalize(t, scores + qi * ke, ids + qi * ke, ke);
        orc_topk_free(t);
    }
    free(qu);
    return ke;
}

/* The FP64 reference score of the asymmetric definition
 * score = sum_j q_unit[j] * bucket_centre(code_j) * inv_norm
 * (src/quant.rs:697-704), with q_unit and inv_norm exactly as the
 * reference computes them in f32 and the sum carried in f64. */
static double f64_doc_score(const uint8_t *doc, uint32_t dim, uint32_t bits, const float *qu) {
    uint32_t cpb = 8 / bits;
    uint32_t mask = (1u << bits) - 1;
    double acc = 0.0;
    for (uint32_t j = 0; j < dim; j++) {
        uint32_t code = (doc[j / cpb] >> ((cpb - 1 - j % cpb) * bits)) & mask;
        acc += (double)qu[j] * (double)orc_bucket_centre(code, bits);
    }
    return acc;
}

void orc_rq_scores_f64(const uint8_t *packed, uint64_t n, uint32_t dim, uint32_t bits,
                       const float *query, double *out) {
    float *qu = (float *)malloc(sizeof(float) * dim);
    orc_l2_normalise(query, dim, qu);
    double inv_norm = (double)(1.0f / orc_rankquant_norm(dim, bits));
    uint32_t bpv = dim * bits / 8;
#pragma omp parallel for schedule(static)
    for (int64_t di = 0; di < (int64_t)n; di++)
        out[di] = f64_doc_score(packed + (uint64_t)di * bpv, dim, bits, qu) * inv_norm;
    free(qu);
}

void orc_rq_scores_f64_subset(const uint8_t *packed, uint32_t dim, uint32_t bits,
                              const float *query, const uint32_t *cands, uint64_t m,
                              double *out) {
    float *qu = (float *)malloc(sizeof(float) * dim);
    orc_l2_normalise(query, dim, qu);
    double inv_norm = (double)(1.0f / orc_rankquant_norm(dim, bits));
    uint32_t bpv = dim * bits / 8;
    for (uint64_t i = 0; i < m; i++)
        out[i] = f64_doc_score(packed + (uint64_t)cands[i] * bpv, dim, bits, qu) * inv_norm;
    free(qu);
}

/* subset_rerank_row_into (src/quant.rs:1126-1281), scalar LUT tier: gather,
 * TopK keyed on global ids, finalize, map local -> global. `qu` is the
 * already-normalised query; writes `out_k` slots. */
static void subset_row(const uint8_t *packed, uint32_t dim, uint32_t bits, const float *qu,
                       const uint32_t *cands, uint64_t m, uint64_t out_k, float *scores,
                       int64_t *ids) {
    uint32_t bpv = dim * bits / 8;
    float inv_norm = 1.0f / orc_rankquant_norm(dim, bits);
    float *lut = build_asym_lut(qu, dim, bits);
    orc_topk *t = orc_topk_new(out_k, cands, m);
    for (uint64_t i = 0; i < m; i++)
        orc_topk_insert(t, lut_doc_score(packed + (uint64_t)cands[i] * bpv, dim, bits, lut) * inv_norm, i);
    int64_t *local = (int64_t *)malloc(8 * (out_k ? out_k : 1));
    orc_topk_finalize(t, scores, local, out_k);
    for (uint64_t i = 0; i < out_k; i++) ids[i] = local[i] < 0 ? -1 : (int64_t)cands[local[i]];
    free(local);
    orc_topk_free(t);
    free(lut);
}

/* RankQuant::search_asymmetric_subset (src/quant.rs:1048-1083). */
uint64_t orc_rq_subset(const uint8_t *packed, uint64_t n, uint32_t dim, uint32_t bits,
                       const float *query, const uint32_t *cands, uint64_t m, uint64_t k,
                       float *scores, int64_t *ids) {
    (void)n;
    uint64_t out_k = k < m ? k : m;
    if (out_k == 0) return 0;
    float *qu = (float *)malloc(sizeof(float) * dim);
    orc_l2_normalise(query, dim, qu);
    subset_row(packed, dim, bits, qu, cands, m, out_k, scores, ids);
    free(qu);
    return out_k;
}

/* RankQuant::search_asymmetric_subset_batched_serial_into
 * (src/quant.rs:1336-1394): rectangular nq x min(k, n), empty rows
 * sentinel-padded (-inf, -1), underfull rows padded by finalize. */
uint64_t orc_rq_subset_batched(const uint8_t *packed, uint64_t n, uint32_t dim,
                               uint32_t bits, const float *queries, uint64_t nq,
                               const uint64_t *offsets, const uint32_t *cands, uint64_t k,
                               float *scores, int64_t *ids) {
    uint64_t out_k = k < n ? k : n;
    if (out_k == 0 || nq == 0) return out_k;
    float *qu = (float *)malloc(sizeof(float) * dim);
    for (uint64_t qi = 0; qi < nq; qi++) {
        const uint32_t *row = cands + offsets[qi];
        uint64_t m = offsets[qi + 1] - offsets[qi];
        float *os = scores + qi * out_k;
        int64_t *oi = ids + qi * out_k;
        if (m == 0) {
            for (uint64_t s = 0; s < out_k; s++) { os[s] = -INFINITY; oi[s] = -1; }
            continue;
        }
        orc_l2_normalise(queries + qi * dim, dim, qu);
        subset_row(packed, dim, bits, qu, row, m, out_k, os, oi);
    }
    free(qu);
    return out_k;
}

/* ------------------------------------------------------------------ */
/* SignBitmap                                                         */
/* ------------------------------------------------------------------ */

/* sign_scan_collect scalar (src/sign_bitmap.rs:674-692, util.rs:236-238). */
void orc_sign_hamming_all(const uint64_t *words, uint64_t n, uint32_t dim, const float *q,
                          uint32_t *out) {
    uint32_t qpv = dim / 64;
    uint64_t *qb = (uint64_t *)malloc(8 * qpv);
    orc_sign_query(q, dim, qb);
    for (uint64_t i = 0; i < n; i++) {
        uint32_t h = 0;
        for (uint32_t w = 0; w < qpv; w++) h += (uint32_t)__builtin_popcountll(words[i * qpv + w] ^ qb[w]);
        out[i] = h;
    }
    free(qb);
}

/* SignBitmap::top_m_candidates (src/sign_bitmap.rs:330-362): top m_eff by
 * (hamming asc, doc_id asc), sorted.  Stated as the full lexicographic sort
 * of tests/tiled_candgen.rs:41-49. */
uint64_t orc_sign_top_m(const uint64_t *words, uint64_t n, uint32_t dim, const float *q,
                        uint64_t m, uint32_t *out) {
    uint64_t me = m < n ? m : n;
    if (me == 0) return 0;
    uint32_t *h = (uint32_t *)malloc(4 * n);
    orc_sign_hamming_all(words, n, dim, q, h);
    uint64_t *key = (uint64_t *)malloc(8 * n);
    for (uint64_t i = 0; i < n; i++) key[i] = ((uint64_t)h[i] << 32) | i;
    qsort(key, n, 8, cmp_u64);
    for (uint64_t i = 0; i < me; i++) out[i] = (uint32_t)key[i];
    free(key);
    free(h);
    return me;
}

/* bounded max-heap on (hamming, id) keys packed in u64 */
static void heap_push(uint64_t *h, uint64_t *len, uint64_t v) {
    uint64_t i = (*len)++;
    h[i] = v;
    while (i > 0) {
        uint64_t p = (i - 1) / 2;
        if (h[p] >= h[i]) break;
        uint64_t t = h[p]; h[p] = h[i]; h[i] = t;
        i = p;
    }
}
static void heap_pop(uint64_t *h, uint64_t *len) {
    uint64_t n = --(*len);
    h[0] = h[n];
    uint64_t i = 0;
    for (;;) {
        uint64_t l = 2 * i + 1, r = l + 1, b = i;
        if (l < n && h[l] > h[b]) b = l;
        if (r < n && h[r] > h[b]) b = r;
        if (b == i) break;
        uint64_t t = h[b]; h[b] = h[i]; h[i] = t;
        i = b;
    }
}

/* top_m_candidates_streamed (src/sign_bitmap.rs:231-328): 256 KiB doc blocks
 * x 32-query tiles, per-query bounded max-heap with the `worst` early-out.
 * Output: nq rows of m_eff ids (CSR with uniform rows). */
uint64_t orc_sign_top_m_streamed(const uint64_t *words, uint64_t n, uint32_t dim,
                                 const float *queries, uint64_t nq, uint64_t m,
                                 uint32_t *out) {
    uint64_t me = m < n ? m : n;
    if (me == 0 || nq == 0) return me;
    uint32_t qpv = dim / 64;
    uint64_t *qb = (uint64_t *)malloc(8 * qpv * nq);
    for (uint64_t qi = 0; qi < nq; qi++) orc_sign_query(queries + qi * dim, dim, qb + qi * qpv);
    uint64_t block_docs = (256 * 1024) / ((uint64_t)qpv * 8);
    if (block_docs < 64) block_docs = 64;
    if (block_docs > n) block_docs = n;
    uint64_t **heaps = (uint64_t **)malloc(sizeof(uint64_t *) * nq);
    uint64_t *lens = (uint64_t *)calloc(nq, 8);
    uint32_t *worst = (uint32_t *)malloc(4 * nq);
    for (uint64_t qi = 0; qi < nq; qi++) {
        heaps[qi] = (uint64_t *)malloc(8 * (me + 1));
        worst[qi] = UINT32_MAX;
    }
    for (uint64_t bs = 0; bs < n; bs += block_docs) {
        uint64_t bn = block_docs < n - bs ? block_docs : n - bs;
        for (uint64_t qi = 0; qi < nq; qi++) {
            for (uint64_t d = 0; d < bn; d++) {
                uint32_t h = 0;
                for (uint32_t w = 0; w < qpv; w++)
                    h += (uint32_t)__builtin_popcountll(words[(bs + d) * qpv + w] ^ qb[qi * qpv + w]);
                if (h >= worst[qi]) continue;
                heap_push(heaps[qi], &lens[qi], ((uint64_t)h << 32) | (bs + d));
                if (lens[qi] > me) heap_pop(heaps[qi], &lens[qi]);
                if (lens[qi] == me) worst[qi] = (uint32_t)(heaps[qi][0] >> 32);
            }
        }
    }
    for (uint64_t qi = 0; qi < nq; qi++) {
        qsort(heaps[qi], lens[qi], 8, cmp_u64);
        for (uint64_t i = 0; i < me; i++) out[qi * me + i] = (uint32_t)heaps[qi][i];
        free(heaps[qi]);
    }
    free(heaps);
    free(lens);
    free(worst);
    free(qb);
    return me;
}

/* ------------------------------------------------------------------ */
/* Bitmap                                                             */
/* ------------------------------------------------------------------ */

/* bitmap_scan_collect scalar (src/bitmap.rs:607-630, util.rs:227-229). */
void orc_bitmap_overlap_all(const uint64_t *words, uint64_t n, uint32_t dim,
                            const uint64_t *qbm, uint32_t *out) {
    uint32_t qpv = dim / 64;
    for (uint64_t i = 0; i < n; i++) {
        uint32_t s = 0;
        for (uint32_t w = 0; w < qpv; w++) s += (uint32_t)__builtin_popcountll(words[i * qpv + w] & qbm[w]);
        out[i] = s;
    }
}

/* Bitmap::top_m_candidates (src/bitmap.rs:257-290): (overlap desc, id asc). */
uint64_t orc_bitmap_top_m(const uint64_t *words, uint64_t n, uint32_t dim, uint32_t n_top,
                          const float *q, uint64_t m, uint32_t *out) {
    uint64_t me = m < n ? m : n;
    if (me == 0) return 0;
    uint64_t *qbm = (uint64_t *)malloc(8 * (dim / 64));
    orc_bitmap_query_fp32(q, dim, n_top, qbm);
    uint32_t *s = (uint32_t *)malloc(4 * n);
    orc_bitmap_overlap_all(words, n, dim, qbm, s);
    uint64_t *key = (uint64_t *)malloc(8 * n);
    for (uint64_t i = 0; i < n; i++) key[i] = ((uint64_t)(0xFFFFFFFFu - s[i]) << 32) | i;
    qsort(key, n, 8, cmp_u64);
    for (uint64_t i = 0; i < me; i++) out[i] = (uint32_t)key[i];
    free(key);
    free(s);
    free(qbm);
    return me;
}

/* Bitmap::search (src/bitmap.rs:196-242): overlap as f32 through TopK. */
uint64_t orc_bitmap_search(const uint64_t *words, uint64_t n, uint32_t dim, uint32_t n_top,
                           const float *queries, uint64_t nq, uint64_t k, float *scores,
                           int64_t *ids) {
    uint64_t ke = k < n ? k : n;
    if (ke == 0) return 0;
    uint32_t qpv = dim / 64;
    uint64_t *qbm = (uint64_t *)malloc(8 * qpv);
    uint32_t *s = (uint32_t *)malloc(4 * n);
    for (uint64_t qi = 0; qi < nq; qi++) {
        orc_bitmap_query_fp32(queries + qi * dim, dim, n_top, qbm);
        orc_bitmap_overlap_all(words, n, dim, qbm, s);
        orc_topk *t = orc_topk_new(ke, NULL, 0);
        for (uint64_t di = 0; di < n; di++) orc_topk_insert(t, (float)s[di], di);
        orc_topk_finalize(t, scores + qi * ke, ids + qi * ke, ke);
        orc_topk_free(t);
    }
    free(s);
    free(qbm);
    return ke;
}

/* Bitmap::search_subset (src/bitmap.rs:470-494): (score desc, row asc). */
uint64_t orc_bitmap_search_subset(const uint64_t *words, uint64_t n, uint32_t dim,
                                  uint32_t n_top, const float *query, const uint32_t *ids_in,
                                  uint64_t m, uint64_t k, float *scores, int64_t *ids) {
    (void)n;
    uint64_t ke = k < m ? k : m;
    if (ke == 0) return 0;
    uint32_t qpv = dim / 64;
    uint64_t *qbm = (uint64_t *)malloc(8 * qpv);
    orc_bitmap_query_fp32(query, dim, n_top, qbm);
    uint64_t *key = (uint64_t *)malloc(8 * m);
    for (uint64_t i = 0; i < m; i++) {
        uint32_t s = 0;
        for (uint32_t w = 0; w < qpv; w++)
            s += (uint32_t)__builtin_popcountll(words[(uint64_t)ids_in[i] * qpv + w] & qbm[w]);
        key[i] = ((uint64_t)(0xFFFFFFFFu - s) << 32) | ids_in[i];
    }
    qsort(key, m, 8, cmp_u64);
    for (uint64_t i = 0; i < ke; i++) {
        scores[i] = (float)(0xFFFFFFFFu - (uint32_t)(key[i] >> 32));
        ids[i] = (int64_t)(uint32_t)key[i];
    }
    free(key);
    free(qbm);
    return ke;
}

/* ------------------------------------------------------------------ */
/* FastScan b=2                                                       */
/* ------------------------------------------------------------------ */

/* build_fastscan_b2_query (src/fastscan.rs:130-173).  Bit-exact: product,
 * product, add (no FMA); strict < / > running min/max in pair/nibble order;
 * round() half away from zero; clamp; truncating cast. */
void orc_fastscan_query(const float *q, uint32_t dim, uint8_t *lut, float *bias_sum,
                        float *inv_q) {
    static const float centres[4] = {-1.5f, -0.5f, 0.5f, 1.5f};
    uint32_t pairs = dim / 2;
    float *lf = (float *)malloc(sizeof(float) * pairs * 16);
    float gmin = INFINITY, gmax = -INFINITY;
    for (uint32_t p = 0; p < pairs; p++) {
        float qa = q[2 * p], qc = q[2 * p + 1];
        for (int a = 0; a < 4; a++)
            for (int c = 0; c < 4; c++) {
                float x = qa * centres[a];
                float y = qc * centres[c];
                float v = x + y;
                lf[p * 16 + (a << 2 | c)] = v;
                if (v < gmin) gmin = v;
                if (v > gmax) gmax = v;
            }
    }
    float span = gmax - gmin;
    if (!(span >= 1e-12f)) span = 1e-12f; /* f32::max(span, 1e-12) for finite span */
    float scale = 255.0f / span;
    *inv_q = 1.0f / scale;
    *bias_sum = (float)pairs * gmin;
    for (uint32_t i = 0; i < pairs * 16; i++) {
        float v = roundf((lf[i] - gmin) * scale);
        if (v < 0.0f) v = 0.0f;
        if (v > 255.0f) v = 255.0f;
        lut[i] = (uint8_t)v;
    }
    free(lf);
}

/* scan_b2_fastscan_scalar (src/fastscan.rs:316-347) score per document:
 * raw = bias_sum + (acc as f32) * inv_q; score = raw * inv_norm. */
static void fastscan_scores_lut(const uint8_t *blocks, uint64_t n, uint32_t dim,
                                const uint8_t *lut, float bias_sum, float inv_q,
                                float inv_norm, float *out) {
    uint32_t pairs = dim / 2;
    uint64_t n_blocks = (n + 31) / 32;
    for (uint64_t b = 0; b < n_blocks; b++) {
        const uint8_t *blk = blocks + b * pairs * 32;
        uint32_t acc[32] = {0};
        uint64_t din = n - b * 32 < 32 ? n - b * 32 : 32;
        for (uint32_t p = 0; p < pairs; p++)
            for (uint64_t l = 0; l < din; l++) acc[l] += lut[p * 16 + blk[p * 32 + l]];
        for (uint64_t l = 0; l < din; l++) {
            float t = (float)acc[l] * inv_q;
            float raw = bias_sum + t;
            out[b * 32 + l] = raw * inv_norm;
        }
    }
}

void orc_fastscan_scores(const uint8_t *blocks, uint64_t n, uint32_t dim,
                         const float *query, float *out) {
    float *qu = (float *)malloc(sizeof(float) * dim);
    uint8_t *lut = (uint8_t *)malloc(dim * 8);
    float bias, invq;
    orc_l2_normalise(query, dim, qu);
    orc_fastscan_query(qu, dim, lut, &bias, &invq);
    float inv_norm = 1.0f / orc_rankquant_norm(dim, 2);
    fastscan_scores_lut(blocks, n, dim, lut, bias, invq, inv_norm, out);
    free(lut);
    free(qu);
}

/* search_asymmetric_fastscan_b2 (src/fastscan.rs:357-476), scalar kernel. */
uint64_t orc_fastscan_search(const uint8_t *blocks, uint64_t n, uint32_t dim,
                             const float *queries, uint64_t nq, uint64_t k, float *scores,
                             int64_t *ids) {
    uint64_t ke = k < n ? k : n;
    if (ke == 0) return 0;
    float *s = (float *)malloc(sizeof(float) * n);
    for (uint64_t qi = 0; qi < nq; qi++) {
        orc_fastscan_scores(blocks, n, dim, queries + qi * dim, s);
        orc_topk *t = orc_topk_new(ke, NULL, 0);
        for (uint64_t d = 0; d < n; d++) orc_topk_insert(t, s[d], d);
        orc_topk_finalize(t, scores + qi * ke, ids + qi * ke, ke);
        orc_topk_free(t);
    }
    free(s);
    return ke;
}

/* ------------------------------------------------------------------ */
/* MultiBucketBitmap                                                  */
/* ------------------------------------------------------------------ */

/* diagonal / outer-product / banded weights (src/multi_bucket.rs:142-188).
 * kind 0 = diagonal, 1 = outer product, 2 = banded(half_width). */
void orc_multibucket_weights(uint32_t bits, int kind, uint32_t half_width, float *w) {
    uint32_t nb = 1u << bits;
    float c = ((float)nb - 1.0f) / 2.0f;
    for (uint32_t a = 0; a < nb; a++)
        for (uint32_t b = 0; b < nb; b++) {
            float v = 0.0f;
            if (kind == 0) v = a == b ? 1.0f : 0.0f;
            else if (kind == 1) v = ((float)a - c) * ((float)b - c);
            else {
                uint32_t diff = a > b ? a - b : b - a;
                if (diff <= half_width) v = ((float)a - c) * ((float)b - c);
            }
            w[a * nb + b] = v;
        }
}

/* bilinear_score (src/multi_bucket.rs:194-222): acc += w * overlap in
 * (a, b) order, zero weights skipped. */
void orc_multibucket_scores(const uint64_t *words, uint64_t n, uint32_t dim, uint32_t bits,
                            const uint64_t *qbm, const float *w, float *out) {
    uint32_t qpb = dim / 64, nb = 1u << bits;
    for (uint64_t di = 0; di < n; di++) {
        const uint64_t *doc = words + di * nb * qpb;
        float acc = 0.0f;
        for (uint32_t a = 0; a < nb; a++)
            for (uint32_t b = 0; b < nb; b++) {
                float weight = w[a * nb + b];
                if (weight == 0.0f) continue;
                uint32_t ov = 0;
                for (uint32_t k = 0; k < qpb; k++) ov += (uint32_t)__builtin_popcountll(qbm[a * qpb + k] & doc[b * qpb + k]);
                float prod = weight * (float)ov;
                acc = acc + prod;
            }
        out[di] = acc;
    }
}

typedef struct { float s; uint32_t i; } si_t;
static int cmp_mb(const void *pa, const void *pb) {
    const si_t *a = (const si_t *)pa, *b = (const si_t *)pb;
    if (a->s > b->s) return -1;
    if (a->s < b->s) return 1;
    return (a->i > b->i) - (a->i < b->i);
}

/* top_m_bilinear (src/multi_bucket.rs:228-251).  The reference orders by
 * score desc with no id tie-break (select_nth_unstable); this restatement
 * fixes the tie order to (score desc, id asc), the order the GPU path
 * produces, so sets agree exactly away from boundary ties. */
uint64_t orc_multibucket_top_m(const uint64_t *words, uint64_t n, uint32_t dim,
                               uint32_t bits, const uint64_t *qbm, const float *w,
                               uint64_t m, uint32_t *out) {
    uint64_t me = m < n ? m : n;
    if (me == 0) return 0;
    float *s = (float *)malloc(sizeof(float) * n);
    orc_multibucket_scores(words, n, dim, bits, qbm, w, s);
    si_t *o = (si_t *)malloc(sizeof(si_t) * n);
    for (uint64_t i = 0; i < n; i++) { o[i].s = s[i]; o[i].i = (uint32_t)i; }
    qsort(o, n, sizeof(si_t), cmp_mb);
    for (uint64_t i = 0; i < me; i++) out[i] = o[i].i;
    free(o);
    free(s);
    return me;
}

/* ------------------------------------------------------------------ */
/* test-corpus helper                                                 */
/* ------------------------------------------------------------------ */

/* XorShift::next_f32 of tests/tiled_candgen.rs:12-27 (state seeded with
 * seed | 1): x ^= x<<13; x ^= x>>7; x ^= x<<17; ((x>>40) as f32 / 2^23) - 1. */
void orc_xorshift_f32(uint64_t seed, uint64_t count, float *out) {
    uint64_t x = seed | 1;
    for (uint64_t i = 0; i < count; i++) {
        x ^= x << 13;
        x ^= x >> 7;
        x ^= x << 17;
        out[i] = ((float)(x >> 40) / 8388608.0f) - 1.0f;
    }
}

/* ------------------------------------------------------------------ */
/* benchmark corpus generator                                         */
/* ------------------------------------------------------------------ */

/* The seeded clustered-Gaussian corpus of the benchmark configurations,
 * restated here so the CPU legs of the benchmark build their inputs without
 * the product library: 256 clusters, centre = N(0, I) normalised to unit
 * norm, doc = centre[cluster] + N(0, sigma^2) per coordinate, L2-normalised
 * in f64 and stored as f32; a query is a uniformly chosen doc plus
 * N(0, query_sigma^2), renormalised.  Every row owns a xoshiro256** stream
 * seeded through SplitMix64 from (seed, tag, row) -- tag 1 centres, 2 docs,
 * 3 queries (whose stream uses seed + 1) -- and normals come from
 * Box-Muller in f64, so any row range is reproducible on its own. */
typedef struct { uint64_t s[4]; } synth_rng;

static uint64_t synth_splitmix(uint64_t *x) {
    uint64_t z = (*x += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

static void synth_seed(synth_rng *r, uint64_t seed, uint64_t tag, uint64_t row) {
    uint64_t x = seed ^ (tag * 0xD1B54A32D192ED03ull) ^ (row * 0x8CB92BA72F3D8DD7ull);
    for (int i = 0; i < 4; i++) r->s[i] = synth_splitmix(&x);
}

static inline uint64_t synth_rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }

static uint64_t synth_next(synth_rng *r) {
    uint64_t *s = r->s;
    const uint64_t out = synth_rotl(s[1] * 5, 7) * 9, t = s[1] << 17;
    s[2] ^= s[0];
    s[3] ^= s[1];
    s[1] ^= s[2];
    s[0] ^= s[3];
    s[2] ^= t;
    s[3] = synth_rotl(s[3], 45);
    return out;
}

static double synth_uniform(synth_rng *r) { return (double)(synth_next(r) >> 11) * 0x1.0p-53; }

static void synth_normals(synth_rng *r, double *out, uint32_t n) {
    for (uint32_t i = 0; i < n; i += 2) {
        const double u1 = 1.0 - synth_uniform(r), u2 = synth_uniform(r);
        const double rad = sqrt(-2.0 * log(u1)), a = 6.283185307179586 * u2;
        out[i] = rad * cos(a);
        if (i + 1 < n) out[i + 1] = rad * sin(a);
    }
}

static void synth_normalise(double *v, uint32_t dim) {
    double s = 0.0;
    for (uint32_t j = 0; j < dim; j++) s += v[j] * v[j];
    const double inv = s > 0.0 ? 1.0 / sqrt(s) : 0.0;
    for (uint32_t j = 0; j < dim; j++) v[j] *= inv;
}

#define SYNTH_CLUSTERS 256u

static double *synth_centres(uint64_t seed, uint32_t dim) {
    double *c = (double *)malloc(sizeof(double) * SYNTH_CLUSTERS * dim + 8);
#pragma omp parallel for schedule(static)
    for (int k = 0; k < (int)SYNTH_CLUSTERS; k++) {
        synth_rng r;
        synth_seed(&r, seed, 1, (uint64_t)k);
        synth_normals(&r, c + (size_t)k * dim, dim);
        synth_normalise(c + (size_t)k * dim, dim);
    }
    return c;
}

static void synth_doc_row(uint64_t seed, uint64_t row, uint32_t dim, double sigma, const double *cen,
                          double *tmp, float *out) {
    synth_rng r;
    synth_seed(&r, seed, 2, row);
    const uint32_t cl = (uint32_t)(synth_next(&r) >> 56);
    synth_normals(&r, tmp, dim);
    const double *c = cen + (size_t)cl * dim;
    for (uint32_t j = 0; j < dim; j++) tmp[j] = c[j] + sigma * tmp[j];
    synth_normalise(tmp, dim);
    for (uint32_t j = 0; j < dim; j++) out[j] = (float)tmp[j];
}

void orc_synth_docs(uint64_t seed, uint64_t first, uint64_t n, uint32_t dim, float sigma, float *out) {
    if (dim == 0 || n == 0) return;
    double *cen = synth_centres(seed, dim);
#pragma omp parallel
    {
        double *tmp = (double *)malloc(sizeof(double) * (dim + 1));
#pragma omp for schedule(static)
        for (int64_t i = 0; i < (int64_t)n; i++)
            synth_doc_row(seed, first + (uint64_t)i, dim, sigma, cen, tmp, out + (uint64_t)i * dim);
        free(tmp);
    }
    free(cen);
}

void orc_synth_queries(uint64_t seed, uint64_t n_docs, uint64_t nq, uint32_t dim, float doc_sigma,
                       float query_sigma, float *out, uint64_t *planted) {
    if (dim == 0 || nq == 0 || n_docs == 0) return;
    double *cen = synth_centres(seed, dim);
#pragma omp parallel
    {
        double *tmp = (double *)malloc(sizeof(double) * (dim + 1));
        double *noise = (double *)malloc(sizeof(double) * (dim + 1));
        float *doc = (float *)malloc(sizeof(float) * dim);
#pragma omp for schedule(static)
        for (int64_t i = 0; i < (int64_t)nq; i++) {
            synth_rng r;
            synth_seed(&r, seed + 1, 3, (uint64_t)i);
            const uint64_t src = (uint64_t)(((unsigned __int128)synth_next(&r) * n_docs) >> 64);
            synth_doc_row(seed, src, dim, doc_sigma, cen, tmp, doc);
            synth_normals(&r, noise, dim);
            for (uint32_t j = 0; j < dim; j++) tmp[j] = (double)doc[j] + query_sigma * noise[j];
            synth_normalise(tmp, dim);
            for (uint32_t j = 0; j < dim; j++) out[(uint64_t)i * dim + j] = (float)tmp[j];
            if (planted) planted[i] = src;
        }
        free(tmp);
        free(noise);
        free(doc);
    }
    free(cen);
}

/* Bitmap::add and RankQuant::add in one pass over the rows (one rank
 * transform per row, shared by both layouts): the same bytes as
 * orc_bitmap_encode and orc_rankquant_encode.  Either output may be NULL. */
void orc_encode_bitmap_rankquant(const float *vecs, uint64_t n, uint32_t dim, uint32_t n_top,
                                 uint32_t bits, uint64_t *bitmap_out, uint8_t *rq_out) {
    uint32_t qpv = dim / 64, bpv = dim * bits / 8;
    uint16_t cutoff = (uint16_t)(dim - n_top);
#pragma omp parallel
    {
        uint16_t *r = (uint16_t *)malloc(2 * dim);
        uint8_t *b = (uint8_t *)malloc(dim);
#pragma omp for schedule(static)
        for (int64_t i = 0; i < (int64_t)n; i++) {
            orc_rank_transform(vecs + (uint64_t)i * dim, dim, r);
            if (bitmap_out) {
                uint64_t *row = bitmap_out + (uint64_t)i * qpv;
                memset(row, 0, 8 * (size_t)qpv);
                for (uint32_t j = 0; j < dim; j++)
                    if (r[j] >= cutoff) row[j / 64] |= (uint64_t)1 << (j % 64);
            }
            if (rq_out) {
                for (uint32_t j = 0; j < dim; j++) b[j] = (uint8_t)orc_rank_to_bucket(r[j], dim, bits);
                orc_pack_buckets(b, dim, bits, rq_out + (uint64_t)i * bpv);
            }
        }
        free(r);
        free(b);
    }
}

/* ------------------------------------------------------------------ */
/* AVX-512 + OpenMP restatement (timed CPU baseline only)             */
/* ------------------------------------------------------------------ */

int orc_avx512_available(void) {
    __builtin_cpu_init();
    return __builtin_cpu_supports("avx512f") && __builtin_cpu_supports("avx512bw") &&
           __builtin_cpu_supports("avx512dq") && __builtin_cpu_supports("avx512vpopcntdq");
}

int orc_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

#define AVX512 __attribute__((target("avx512f,avx512bw,avx512dq,avx512vpopcntdq")))

/* scan_b2_fastscan_avx512 (src/fastscan.rs:184-311): VPSHUFB nibble LUT,
 * u16 accumulate, flush to u32 every 256 pairs. */
AVX512 static void fastscan_avx512(const uint8_t *blocks, uint64_t n, uint32_t dim,
                                   const uint8_t *lut, float bias_sum, float inv_q,
                                   float scale, orc_topk *top) {
    uint32_t pairs = dim / 2;
    uint64_t bytes_per_block = (uint64_t)pairs * 32;
    uint64_t n_blocks = (n + 31) / 32;
    for (uint64_t b = 0; b < n_blocks; b++) {
        const uint8_t *bp = blocks + b * bytes_per_block;
        __m512i acc32_lo = _mm512_setzero_si512(), acc32_hi = _mm512_setzero_si512();
        uint32_t p = 0;
        while (p < pairs) {
            uint32_t chunk = pairs - p < 256 ? pairs - p : 256;
            __m512i a16lo = _mm512_setzero_si512(), a16hi = _mm512_setzero_si512();
            for (uint32_t pp = p; pp < p + chunk; pp++) {
                __m256i codes = _mm256_loadu_si256((const __m256i *)(bp + (uint64_t)pp * 32));
                __m128i l128 = _mm_loadu_si128((const __m128i *)(lut + (uint64_t)pp * 16));
                __m256i l256 = _mm256_broadcastsi128_si256(l128);
                __m256i contrib = _mm256_shuffle_epi8(l256, codes);
                __m256i lo = _mm256_cvtepu8_epi16(_mm256_castsi256_si128(contrib));
                __m256i hi = _mm256_cvtepu8_epi16(_mm256_extracti128_si256(contrib, 1));
                a16lo = _mm512_add_epi16(a16lo, _mm512_castsi256_si512(lo));
                a16hi = _mm512_add_epi16(a16hi, _mm512_castsi256_si512(hi));
            }
            acc32_lo = _mm512_add_epi32(acc32_lo, _mm512_cvtepu16_epi32(_mm512_castsi512_si256(a16lo)));
            acc32_hi = _mm512_add_epi32(acc32_hi, _mm512_cvtepu16_epi32(_mm512_castsi512_si256(a16hi)));
            p += chunk;
        }
        uint32_t tl[16], th[16];
        _mm512_storeu_si512(tl, acc32_lo);
        _mm512_storeu_si512(th, acc32_hi);
        uint64_t din = n - b * 32 < 32 ? n - b * 32 : 32;
        for (uint64_t l = 0; l < din; l++) {
            uint32_t acc = l < 16 ? tl[l] : th[l - 16];
            float raw = bias_sum + (float)acc * inv_q;
            orc_topk_insert(top, raw * scale, b * 32 + l);
        }
    }
}

/* scan_b2_asym_avx512 / scan_b4_asym_avx512 (src/quant_kernels.rs:406-581):
 * centre-drop with 4 accumulators, offset applied in the TopK. */
AVX512 static void asym_avx512(const uint8_t *packed, uint64_t n, uint32_t dim, uint32_t bits,
                               const float *q, float scale, orc_topk *top) {
    uint32_t bpv = dim * bits / 8;
    if (bits == 2) {
        const __m512i shifts = _mm512_setr_epi32(30, 28, 26, 24, 22, 20, 18, 16, 14, 12, 10, 8, 6, 4, 2, 0);
        const __m512i mask3 = _mm512_set1_epi32(3);
        uint32_t outer = bpv / 4 / 4;
        for (uint64_t di = 0; di < n; di++) {
            const uint8_t *doc = packed + di * bpv;
            __m512i dummy = _mm512_setzero_si512();
            (void)dummy;
            __m512 acc[4] = {_mm512_setzero_ps(), _mm512_setzero_ps(), _mm512_setzero_ps(), _mm512_setzero_ps()};
            for (uint32_t o = 0; o < outer; o++)
                for (int u = 0; u < 4; u++) {
                    uint32_t c = o * 4 + u;
                    const uint8_t *cp = doc + c * 4;
                    uint32_t chunk = ((uint32_t)cp[0] << 24) | ((uint32_t)cp[1] << 16) | ((uint32_t)cp[2] << 8) | cp[3];
                    __m512i codes = _mm512_and_si512(_mm512_srlv_epi32(_mm512_set1_epi32((int)chunk), shifts), mask3);
                    acc[u] = _mm512_fmadd_ps(_mm512_cvtepi32_ps(codes), _mm512_loadu_ps(q + c * 16), acc[u]);
                }
            __m512 total = _mm512_add_ps(_mm512_add_ps(acc[0], acc[1]), _mm512_add_ps(acc[2], acc[3]));
            orc_topk_insert(top, _mm512_reduce_add_ps(total) * scale, di);
        }
    } else {
        const __m512i shifts = _mm512_setr_epi32(28, 24, 20, 16, 12, 8, 4, 0, 28, 24, 20, 16, 12, 8, 4, 0);
        const __m512i maskf = _mm512_set1_epi32(0xF);
        uint32_t outer = bpv / 8 / 4;
        for (uint64_t di = 0; di < n; di++) {
            const uint8_t *doc = packed + di * bpv;
            __m512 acc[4] = {_mm512_setzero_ps(), _mm512_setzero_ps(), _mm512_setzero_ps(), _mm512_setzero_ps()};
            for (uint32_t o = 0; o < outer; o++)
                for (int u = 0; u < 4; u++) {
                    uint32_t c = o * 4 + u;
                    const uint8_t *cp = doc + c * 8;
                    uint32_t lo = ((uint32_t)cp[0] << 24) | ((uint32_t)cp[1] << 16) | ((uint32_t)cp[2] << 8) | cp[3];
                    uint32_t hi = ((uint32_t)cp[4] << 24) | ((uint32_t)cp[5] << 16) | ((uint32_t)cp[6] << 8) | cp[7];
                    __m512i comb = _mm512_mask_blend_epi32((__mmask16)0xFF00, _mm512_set1_epi32((int)lo), _mm512_set1_epi32((int)hi));
                    __m512i codes = _mm512_and_si512(_mm512_srlv_epi32(comb, shifts), maskf);
                    acc[u] = _mm512_fmadd_ps(_mm512_cvtepi32_ps(codes), _mm512_loadu_ps(q + c * 16), acc[u]);
                }
            __m512 total = _mm512_add_ps(_mm512_add_ps(acc[0], acc[1]), _mm512_add_ps(acc[2], acc[3]));
            orc_topk_insert(top, _mm512_reduce_add_ps(total) * scale, di);
        }
    }
}

/* sign_scan_collect_avx512vpop (src/sign_bitmap.rs:696-753). */
AVX512 static void sign_collect_avx512(const uint64_t *words, uint64_t n, uint32_t qpv,
                                       const uint64_t *q, uint32_t *scores) {
    uint32_t lanes = qpv / 8, rem = qpv % 8;
    __mmask8 tm = rem ? (__mmask8)((1u << rem) - 1) : 0;
    __m512i qz[64];
    for (uint32_t l = 0; l < lanes && l < 64; l++) qz[l] = _mm512_loadu_si512(q + l * 8);
    __m512i qt = rem ? _mm512_maskz_loadu_epi64(tm, q + lanes * 8) : _mm512_setzero_si512();
    for (uint64_t di = 0; di < n; di++) {
        const uint64_t *d = words + di * qpv;
        __m512i acc = _mm512_setzero_si512();
        for (uint32_t l = 0; l < lanes; l++)
            acc = _mm512_add_epi64(acc, _mm512_popcnt_epi64(_mm512_xor_si512(_mm512_loadu_si512(d + l * 8), qz[l])));
        if (rem) acc = _mm512_add_epi64(acc, _mm512_popcnt_epi64(_mm512_xor_si512(_mm512_maskz_loadu_epi64(tm, d + lanes * 8), qt)));
        scores[di] = (uint32_t)_mm512_reduce_add_epi64(acc);
    }
}

/* quickselect on packed (score, id) u64 keys: the m smallest moved to the
 * front (the reference's select_nth_unstable_by + head sort). */
static void select_smallest(uint64_t *a, uint64_t n, uint64_t m) {
    uint64_t lo = 0, hi = n;
    while (hi - lo > 16) {
        uint64_t x = a[lo], y = a[lo + (hi - lo) / 2], z = a[hi - 1];
        uint64_t piv = (x < y) ? ((y < z) ? y : (x < z ? z : x)) : ((x < z) ? x : (y < z ? z : y));
        uint64_t lt = lo, i = lo, gt = hi, t;
        while (i < gt) {
            if (a[i] < piv) { t = a[lt]; a[lt] = a[i]; a[i] = t; lt++; i++; }
            else if (a[i] > piv) { gt--; t = a[gt]; a[gt] = a[i]; a[i] = t; }
            else i++;
        }
        if (m <= lt) hi = lt;
        else if (m >= gt) lo = gt;
        else return;
    }
    qsort(a + lo, hi - lo, 8, cmp_u64);
}

static float *alloc_unit(const float *q, uint32_t dim) {
    float *qu = (float *)malloc(sizeof(float) * dim);
    orc_l2_normalise(q, dim, qu);
    return qu;
}

/* subset rerank with the reference's dispatch: AVX-512 centre-drop for
 * b=2/4 when dim % 64 == 0, scalar LUT otherwise (src/quant.rs:1126-1281). */
static void cpu_subset_row(const uint8_t *packed, uint32_t dim, uint32_t bits, const float *qu,
                           const uint32_t *cands, uint64_t m, uint64_t out_k, uint8_t *scratch,
                           float *scores, int64_t *ids) {
    uint32_t bpv = dim * bits / 8;
    if ((bits == 2 || bits == 4) && dim % 64 == 0 && orc_avx512_available()) {
        float inv_norm = 1.0f / orc_rankquant_norm(dim, bits);
        float centre = ((float)(1u << bits) - 1.0f) / 2.0f;
        float qs = -0.0f;
        for (uint32_t j = 0; j < dim; j++) qs += qu[j];
        for (uint64_t i = 0; i < m; i++) memcpy(scratch + i * bpv, packed + (uint64_t)cands[i] * bpv, bpv);
        orc_topk *t = orc_topk_new(out_k, cands, m);
        orc_topk_set_score_offset(t, -centre * qs * inv_norm);
        asym_avx512(scratch, m, dim, bits, qu, inv_norm, t);
        int64_t *local = (int64_t *)malloc(8 * out_k);
        orc_topk_finalize(t, scores, local, out_k);
        for (uint64_t i = 0; i < out_k; i++) ids[i] = local[i] < 0 ? -1 : (int64_t)cands[local[i]];
        free(local);
        orc_topk_free(t);
    } else {
        subset_row(packed, dim, bits, qu, cands, m, out_k, scores, ids);
    }
}

/* RankQuantFastscan::search(q, n_candidates) -> RankQuant b=2
 * search_asymmetric_subset(q, ids, k) per query, parallel over queries the
 * way rayon's par_chunks is (src/fastscan.rs:430-468, src/quant.rs:1048).
 * `cands_out` (nq x min(n_candidates, n), may be NULL) receives each query's
 * FastScan candidate row in TopK order. */
void orc_cpu_fastscan_two_stage(const uint8_t *blocks, const uint8_t *packed_b2, uint64_t n,
                                uint32_t dim, const float *queries, uint64_t nq,
                                uint64_t n_candidates, uint64_t k, int nthreads,
                                float *scores, int64_t *ids, uint32_t *cands_out) {
    uint64_t cand = n_candidates < n ? n_candidates : n;
    uint64_t out_k = k < cand ? k : cand;
    float inv_norm = 1.0f / orc_rankquant_norm(dim, 2);
    int use_avx = orc_avx512_available();
#pragma omp parallel num_threads(nthreads)
    {
        float *cs = (float *)malloc(sizeof(float) * cand);
        int64_t *ci = (int64_t *)malloc(8 * cand);
        uint32_t *cu = (uint32_t *)malloc(4 * cand);
        uint8_t *lut = (uint8_t *)malloc(dim * 8);
        uint8_t *scratch = (uint8_t *)malloc(cand * (dim / 4));
        float *fs = use_avx ? NULL : (float *)malloc(sizeof(float) * n);
#pragma omp for schedule(dynamic, 1)
        for (int64_t qi = 0; qi < (int64_t)nq; qi++) {
            float *qu = alloc_unit(queries + (uint64_t)qi * dim, dim);
            float bias, invq;
            orc_fastscan_query(qu, dim, lut, &bias, &invq);
            orc_topk *t = orc_topk_new(cand, NULL, 0);
            if (use_avx) fastscan_avx512(blocks, n, dim, lut, bias, invq, inv_norm, t);
            else {
                fastscan_scores_lut(blocks, n, dim, lut, bias, invq, inv_norm, fs);
                for (uint64_t d = 0; d < n; d++) orc_topk_insert(t, fs[d], d);
            }
            orc_topk_finalize(t, cs, ci, cand);
            orc_topk_free(t);
            for (uint64_t i = 0; i < cand; i++) cu[i] = (uint32_t)ci[i];
            if (cands_out) memcpy(cands_out + (uint64_t)qi * cand, cu, 4 * cand);
            cpu_subset_row(packed_b2, dim, 2, qu, cu, cand, out_k, scratch,
                           scores + (uint64_t)qi * out_k, ids + (uint64_t)qi * out_k);
            free(qu);
        }
        free(cs); free(ci); free(cu); free(lut); free(scratch); free(fs);
    }
}

/* RankQuant::try_search_with_sign_probe (src/quant.rs:1453-1498) per query:
 * SignBitmap::top_m_candidates (AVX-512 VPOPCNTDQ scan + select_nth) then
 * the subset rerank. */
void orc_cpu_sign_two_stage(const uint64_t *sign_words, const uint8_t *packed, uint64_t n,
                            uint32_t dim, uint32_t bits, const float *queries, uint64_t nq,
                            uint64_t m, uint64_t k, int nthreads, float *scores,
                            int64_t *ids) {
    uint64_t me = m < n ? m : n;
    uint64_t out_k = k < me ? k : me;
    uint32_t qpv = dim / 64;
    int use_avx = orc_avx512_available();
#pragma omp parallel num_threads(nthreads)
    {
        uint32_t *h = (uint32_t *)malloc(4 * n);
        uint64_t *key = (uint64_t *)malloc(8 * n);
        uint64_t *qb = (uint64_t *)malloc(8 * qpv);
        uint32_t *cu = (uint32_t *)malloc(4 * (me ? me : 1));
        uint8_t *scratch = (uint8_t *)malloc((me ? me : 1) * (dim * bits / 8));
#pragma omp for schedule(dynamic, 1)
        for (int64_t qi = 0; qi < (int64_t)nq; qi++) {
            const float *q = queries + (uint64_t)qi * dim;
            orc_sign_query(q, dim, qb);
            if (use_avx) sign_collect_avx512(sign_words, n, qpv, qb, h);
            else {
                for (uint64_t i = 0; i < n; i++) {
                    uint32_t s = 0;
                    for (uint32_t w = 0; w < qpv; w++) s += (uint32_t)__builtin_popcountll(sign_words[i * qpv + w] ^ qb[w]);
                    h[i] = s;
                }
            }
            for (uint64_t i = 0; i < n; i++) key[i] = ((uint64_t)h[i] << 32) | i;
            select_smallest(key, n, me);
            qsort(key, me, 8, cmp_u64);
            for (uint64_t i = 0; i < me; i++) cu[i] = (uint32_t)key[i];
            float *qu = alloc_unit(q, dim);
            cpu_subset_row(packed, dim, bits, qu, cu, me, out_k, scratch,
                           scores + (uint64_t)qi * out_k, ids + (uint64_t)qi * out_k);
            free(qu);
        }
        free(h); free(key); free(qb); free(cu); free(scratch);
    }
}

/* bitmap_scan_collect_batched_avx512vpop (src/bitmap.rs:813-936): the doc
 * stream is read once per group of CHUNK = 8 queries; each doc's words are
 * ANDed with the group's query words, VPOPCNTQ'd and summed per query, the
 * trailing qpv % 8 words through a masked load; a final group of fewer
 * than 8 queries runs the same loop with a runtime bound. */
#define BITMAP_BATCH_CHUNK 8
AVX512 static void bitmap_batched_avx512(const uint64_t *words, uint64_t n, uint32_t qpv,
                                         const uint64_t *qb, uint32_t batch, uint32_t *scores) {
    uint32_t lanes = qpv / 8, rem = qpv % 8;
    __mmask8 tm = rem ? (__mmask8)((1u << rem) - 1) : 0;
    __m512i *qz = (__m512i *)aligned_alloc(64, 64 * ((size_t)batch * (lanes + 1) + 1));
    for (uint32_t b = 0; b < batch; b++) {
        for (uint32_t l = 0; l < lanes; l++) qz[b * (lanes + 1) + l] = _mm512_loadu_si512(qb + (uint64_t)b * qpv + l * 8);
        qz[b * (lanes + 1) + lanes] = rem ? _mm512_maskz_loadu_epi64(tm, qb + (uint64_t)b * qpv + lanes * 8)
                                          : _mm512_setzero_si512();
    }
    uint32_t start = 0;
    for (; start + BITMAP_BATCH_CHUNK <= batch; start += BITMAP_BATCH_CHUNK) {
        for (uint64_t di = 0; di < n; di++) {
            const uint64_t *d = words + di * qpv;
            __m512i acc[BITMAP_BATCH_CHUNK];
            for (int b = 0; b < BITMAP_BATCH_CHUNK; b++) acc[b] = _mm512_setzero_si512();
            for (uint32_t l = 0; l < lanes; l++) {
                __m512i dz = _mm512_loadu_si512(d + l * 8);
                for (int b = 0; b < BITMAP_BATCH_CHUNK; b++)
                    acc[b] = _mm512_add_epi64(acc[b], _mm512_popcnt_epi64(_mm512_and_si512(dz, qz[(start + b) * (lanes + 1) + l])));
            }
            if (rem) {
                __m512i dz = _mm512_maskz_loadu_epi64(tm, d + lanes * 8);
                for (int b = 0; b < BITMAP_BATCH_CHUNK; b++)
                    acc[b] = _mm512_add_epi64(acc[b], _mm512_popcnt_epi64(_mm512_and_si512(dz, qz[(start + b) * (lanes + 1) + lanes])));
            }
            for (int b = 0; b < BITMAP_BATCH_CHUNK; b++)
                scores[(uint64_t)(start + b) * n + di] = (uint32_t)_mm512_reduce_add_epi64(acc[b]);
        }
    }
    uint32_t tail = batch - start;
    if (tail) {
        for (uint64_t di = 0; di < n; di++) {
            const uint64_t *d = words + di * qpv;
            __m512i acc[BITMAP_BATCH_CHUNK];
            for (uint32_t b = 0; b < tail; b++) acc[b] = _mm512_setzero_si512();
            for (uint32_t l = 0; l < lanes; l++) {
                __m512i dz = _mm512_loadu_si512(d + l * 8);
                for (uint32_t b = 0; b < tail; b++)
                    acc[b] = _mm512_add_epi64(acc[b], _mm512_popcnt_epi64(_mm512_and_si512(dz, qz[(start + b) * (lanes + 1) + l])));
            }
            if (rem) {
                __m512i dz = _mm512_maskz_loadu_epi64(tm, d + lanes * 8);
                for (uint32_t b = 0; b < tail; b++)
                    acc[b] = _mm512_add_epi64(acc[b], _mm512_popcnt_epi64(_mm512_and_si512(dz, qz[(start + b) * (lanes + 1) + lanes])));
            }
            for (uint32_t b = 0; b < tail; b++)
                scores[(uint64_t)(start + b) * n + di] = (uint32_t)_mm512_reduce_add_epi64(acc[b]);
        }
    }
    free(qz);
}

static void bitmap_batched_scalar(const uint64_t *words, uint64_t n, uint32_t qpv, const uint64_t *qb,
                                  uint32_t batch, uint32_t *scores) {
    for (uint64_t di = 0; di < n; di++)
        for (uint32_t b = 0; b < batch; b++) {
            uint32_t s = 0;
            for (uint32_t w = 0; w < qpv; w++)
                s += (uint32_t)__builtin_popcountll(words[di * qpv + w] & qb[(uint64_t)b * qpv + w]);
            scores[(uint64_t)b * n + di] = s;
        }
}

/* Bitmap::top_m_candidates_batched_chunked(queries, m, 8)
 * (src/bitmap.rs:304-367, 376-399: groups of 8 queries in parallel, one
 * batched scan per group, then per query the top-m by (overlap desc, id asc),
 * sorted) followed by RankQuant::search_asymmetric_subset per query
 * (src/quant.rs:1048-1083, 1126-1281; AVX-512 centre-drop for b=2/4 at
 * dim % 64 == 0).  `cands_out` (nq x min(m, n), may be NULL) receives each
 * query's candidate row. */
void orc_cpu_bitmap_two_stage(const uint64_t *bitmap_words, const uint8_t *packed, uint64_t n,
                              uint32_t dim, uint32_t n_top, uint32_t bits, const float *queries,
                              uint64_t nq, uint64_t m, uint64_t k, int nthreads, float *scores,
                              int64_t *ids, uint32_t *cands_out) {
    uint64_t me = m < n ? m : n;
    uint64_t out_k = k < me ? k : me;
    if (me == 0 || nq == 0) return;
    uint32_t qpv = dim / 64;
    int use_avx = orc_avx512_available();
    int64_t groups = (int64_t)((nq + BITMAP_BATCH_CHUNK - 1) / BITMAP_BATCH_CHUNK);
#pragma omp parallel num_threads(nthreads)
    {
        uint32_t *sc = (uint32_t *)malloc(4 * n * BITMAP_BATCH_CHUNK);
        uint64_t *key = (uint64_t *)malloc(8 * n);
        uint64_t *qb = (uint64_t *)malloc(8 * (size_t)qpv * BITMAP_BATCH_CHUNK);
        uint32_t *cu = (uint32_t *)malloc(4 * me);
        uint8_t *scratch = (uint8_t *)malloc(me * (dim * bits / 8));
#pragma omp for schedule(dynamic, 1)
        for (int64_t g = 0; g < groups; g++) {
            uint64_t q0 = (uint64_t)g * BITMAP_BATCH_CHUNK;
            uint32_t batch = (uint32_t)(nq - q0 < BITMAP_BATCH_CHUNK ? nq - q0 : BITMAP_BATCH_CHUNK);
            for (uint32_t b = 0; b < batch; b++)
                orc_bitmap_query_fp32(queries + (q0 + b) * dim, dim, n_top, qb + (uint64_t)b * qpv);
            if (use_avx) bitmap_batched_avx512(bitmap_words, n, qpv, qb, batch, sc);
            else bitmap_batched_scalar(bitmap_words, n, qpv, qb, batch, sc);
            for (uint32_t b = 0; b < batch; b++) {
                const uint32_t *row = sc + (uint64_t)b * n;
                for (uint64_t i = 0; i < n; i++) key[i] = ((uint64_t)(UINT32_MAX - row[i]) << 32) | i;
                select_smallest(key, n, me);
                qsort(key, me, 8, cmp_u64);
                for (uint64_t i = 0; i < me; i++) cu[i] = (uint32_t)key[i];
                uint64_t qi = q0 + b;
                if (cands_out) memcpy(cands_out + qi * me, cu, 4 * me);
                float *qu = alloc_unit(queries + qi * dim, dim);
                cpu_subset_row(packed, dim, bits, qu, cu, me, out_k, scratch, scores + qi * out_k, ids + qi * out_k);
                free(qu);
            }
        }
        free(sc); free(key); free(qb); free(cu); free(scratch);
    }
}

/* RankQuant::search_asymmetric with the reference's tier dispatch
 * (src/quant.rs:713-847). */
void orc_cpu_rq_search_asym(const uint8_t *packed, uint64_t n, uint32_t dim, uint32_t bits,
                            const float *queries, uint64_t nq, uint64_t k, int nthreads,
                            float *scores, int64_t *ids) {
    uint64_t ke = k < n ? k : n;
    if (ke == 0) return;
    float inv_norm = 1.0f / orc_rankquant_norm(dim, bits);
    int simd = (bits == 2 || bits == 4) && dim % 64 == 0 && orc_avx512_available();
    float centre = ((float)(1u << bits) - 1.0f) / 2.0f;
    uint32_t bpv = dim * bits / 8;
#pragma omp parallel for num_threads(nthreads) schedule(dynamic, 1)
    for (int64_t qi = 0; qi < (int64_t)nq; qi++) {
        float *qu = alloc_unit(queries + (uint64_t)qi * dim, dim);
        orc_topk *t = orc_topk_new(ke, NULL, 0);
        if (simd) {
            float qs = -0.0f;
            for (uint32_t j = 0; j < dim; j++) qs += qu[j];
            orc_topk_set_score_offset(t, -centre * qs * inv_norm);
            asym_avx512(packed, n, dim, bits, qu, inv_norm, t);
        } else {
            float *lut = build_asym_lut(qu, dim, bits);
            for (uint64_t di = 0; di < n; di++)
                orc_topk_insert(t, lut_doc_score(packed + di * bpv, dim, bits, lut) * inv_norm, di);
            free(lut);
        }
        orc_topk_finalize(t, scores + (uint64_t)qi * ke, ids + (uint64_t)qi * ke, ke);
        orc_topk_free(t);
        free(qu);
    }
}
