// Seeded synthetic corpora for the benchmark configurations.
//
// Docs: 256 clusters; centre c = N(0, I) normalised to unit norm; doc =
// centre[cluster] + N(0, sigma^2) per coordinate, L2-normalised.  Queries: a
// uniformly chosen doc + N(0, query_sigma^2) per coordinate, renormalised.
// Every row owns an independent xoshiro256** stream seeded through SplitMix64
// from (seed, tag, row), so any row range is reproducible on its own and the
// output does not depend on the thread count.  Normals come from Box-Muller in
// f64; the stored vectors are f32.
#include <cmath>
#include <cstring>
#include <vector>

#include "ovb_host.h"

namespace ovb {
namespace {

struct Rng {
  uint64_t s[4];
  static uint64_t splitmix(uint64_t& x) {
    uint64_t z = (x += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  }
  Rng(uint64_t seed, uint64_t tag, uint64_t row) {
    uint64_t x = seed ^ (tag * 0xD1B54A32D192ED03ull) ^ (row * 0x8CB92BA72F3D8DD7ull);
    for (auto& v : s) v = splitmix(x);
  }
  static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
  uint64_t next() {
    const uint64_t r = rotl(s[1] * 5, 7) * 9, t = s[1] << 17;
    s[2] ^= s[0];
    s[3] ^= s[1];
    s[1] ^= s[2];
    s[0] ^= s[3];
    s[2] ^= t;
    s[3] = rotl(s[3], 45);
    return r;
  }
  double uniform() { return (double)(next() >> 11) * 0x1.0p-53; }
  // n normals (Box-Muller pairs)
  void normals(double* out, uint32_t n) {
    for (uint32_t i = 0; i < n; i += 2) {
      const double u1 = 1.0 - uniform(), u2 = uniform();
      const double r = std::sqrt(-2.0 * std::log(u1)), a = 6.283185307179586 * u2;
      out[i] = r * std::cos(a);
      if (i + 1 < n) out[i + 1] = r * std::sin(a);
    }
  }
};

constexpr uint32_t kClusters = 256;

void normalise(double* v, uint32_t dim) {
  double s = 0.0;
  for (uint32_t j = 0; j < dim; j++) s += v[j] * v[j];
  const double inv = s > 0.0 ? 1.0 / std::sqrt(s) : 0.0;
  for (uint32_t j = 0; j < dim; j++) v[j] *= inv;
}

std::vector<double> centres(uint64_t seed, uint32_t dim) {
  std::vector<double> c((size_t)kClusters * dim);
#pragma omp parallel for schedule(static)
  for (int k = 0; k < (int)kClusters; k++) {
    Rng r(seed, 1, (uint64_t)k);
    r.normals(&c[(size_t)k * dim], dim);
    normalise(&c[(size_t)k * dim], dim);
  }
  return c;
}

void doc_row(uint64_t seed, uint64_t row, uint32_t dim, double sigma, const double* cen, double* tmp,
             float* out) {
  Rng r(seed, 2, row);
  const uint32_t cl = (uint32_t)(r.next() >> 56);
  r.normals(tmp, dim);
  const double* c = cen + (size_t)cl * dim;
  for (uint32_t j = 0; j < dim; j++) tmp[j] = c[j] + sigma * tmp[j];
  normalise(tmp, dim);
  for (uint32_t j = 0; j < dim; j++) out[j] = (float)tmp[j];
}

}  // namespace
}  // namespace ovb

using namespace ovb;

extern "C" {

ordvec_status_t ovb_synth_docs(uint64_t seed, uint64_t first, uint64_t n, uint32_t dim, float sigma, float* out) {
  if (!out && n) return ORDVEC_STATUS_NULL_POINTER;
  if (dim == 0) return ORDVEC_STATUS_BAD_ARGUMENT;
  const std::vector<double> cen = centres(seed, dim);
#pragma omp parallel
  {
    std::vector<double> tmp(dim + 1);
#pragma omp for schedule(static)
    for (int64_t i = 0; i < (int64_t)n; i++) doc_row(seed, first + (uint64_t)i, dim, sigma, cen.data(), tmp.data(), out + (uint64_t)i * dim);
  }
  return ORDVEC_STATUS_OK;
}

ordvec_status_t ovb_synth_queries(uint64_t seed, uint64_t n_docs, uint64_t nq, uint32_t dim, float doc_sigma,
                                  float query_sigma, float* out, uint64_t* planted) {
  if ((!out && nq) || n_docs == 0) return n_docs == 0 ? ORDVEC_STATUS_BAD_ARGUMENT : ORDVEC_STATUS_NULL_POINTER;
  if (dim == 0) return ORDVEC_STATUS_BAD_ARGUMENT;
  const std::vector<double> cen = centres(seed, dim);
#pragma omp parallel
  {
    std::vector<double> tmp(dim + 1), noise(dim + 1);
    std::vector<float> doc(dim);
#pragma omp for schedule(static)
    for (int64_t i = 0; i < (int64_t)nq; i++) {
      Rng r(seed + 1, 3, (uint64_t)i);
      const uint64_t src = (uint64_t)(((unsigned __int128)r.next() * n_docs) >> 64);
      doc_row(seed, src, dim, doc_sigma, cen.data(), tmp.data(), doc.data());
      r.normals(noise.data(), dim);
      for (uint32_t j = 0; j < dim; j++) tmp[j] = (double)doc[j] + query_sigma * noise[j];
      normalise(tmp.data(), dim);
      for (uint32_t j = 0; j < dim; j++) out[(uint64_t)i * dim + j] = (float)tmp[j];
      if (planted) planted[i] = src;
    }
  }
  return ORDVEC_STATUS_OK;
}

}  // extern "C"
