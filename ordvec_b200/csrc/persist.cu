// Persisted formats (src/rank_io.rs) loaded straight into HBM.
//
// Little-endian headers, one contiguous payload, exact-length files:
//   OVRQ/TVRQ  magic | ver u8 | bits u8 | dim u32 | n u32       (14 B)  RankQuant
//   OVBM/TVBM  magic | ver u8 | dim u32 | n_top u32 | n u32     (17 B)  Bitmap
//   OVSB/TVSB  magic | ver u8 | dim u32 | n u32                 (13 B)  SignBitmap
//   OVFS       magic | ver u8 | dim u32 | n u32                 (13 B)  FastScan
//   OVR1/TVR1  magic | ver u8 | dim u32 | n u32                 (13 B)  Rank (u16 LE ranks;
//              ABI v1's loader refuses it as an unsupported format)
// The loaders replay the reference's validation in the same order
// (header domains, MAX_VECTORS, 128 GiB payload cap, exact payload length,
// then row invariants: RankQuant constant composition, Bitmap popcount ==
// n_top, FastScan nibble domain / composition / zero tail padding, Rank rows
// permutations of [0, dim)).
// Malformed files map to CORRUPT_INDEX, I/O failures to IO, known-but-not-v1
// formats to UNSUPPORTED_FORMAT (ordvec-ffi/src/lib.rs:241-250, 697-776).
#include <sys/stat.h>

#include <cerrno>
#include <cstdio>
#include <cstring>

#include "ovb_host.h"

namespace ovb {

namespace {

enum class Fmt { Rank, RankQuant, Bitmap, Sign, FastScan, Unknown };

Fmt lookup_magic(const uint8_t m[4]) {
  auto is = [&](const char* s) { return memcmp(m, s, 4) == 0; };
  if (is("OVR1") || is("TVR1")) return Fmt::Rank;
  if (is("OVRQ") || is("TVRQ")) return Fmt::RankQuant;
  if (is("OVBM") || is("TVBM")) return Fmt::Bitmap;
  if (is("OVSB") || is("TVSB")) return Fmt::Sign;
  if (is("OVFS")) return Fmt::FastScan;
  return Fmt::Unknown;
}

[[noreturn]] void corrupt(const std::string& m) { fail(ORDVEC_STATUS_CORRUPT_INDEX, m); }

struct File {
  FILE* f = nullptr;
  uint64_t size = 0;
  explicit File(const char* path, const char* ctx) {
    f = fopen(path, "rb");
    if (!f) fail(errno == ENOENT ? ORDVEC_STATUS_IO : ORDVEC_STATUS_IO, std::string(ctx) + ": " + strerror(errno));
    struct stat st;
    if (fstat(fileno(f), &st) != 0) fail(ORDVEC_STATUS_IO, std::string(ctx) + ": stat failed");
    size = (uint64_t)st.st_size;
  }
  ~File() {
    if (f) fclose(f);
  }
  void read(void* dst, size_t n, const char* label, const char* field) {
    if (fread(dst, 1, n, f) != n) corrupt(std::string(label) + " header truncated while reading " + field);
  }
  uint32_t u32(const char* label, const char* field) {
    uint8_t b[4];
    read(b, 4, label, field);
    return (uint32_t)b[0] | ((uint32_t)b[1] << 8) | ((uint32_t)b[2] << 16) | ((uint32_t)b[3] << 24);
  }
  uint8_t u8(const char* label, const char* field) {
    uint8_t b;
    read(&b, 1, label, field);
    return b;
  }
  uint64_t pos() { return (uint64_t)ftell(f); }
};

void check_version(File& f, const char* label) {
  uint8_t v = f.u8(label, "version");
  if (v != 1) corrupt(std::string("unsupported ") + label + " version: " + std::to_string(v));
}
void check_dim(uint64_t dim) {
  if (dim < 2 || dim > kMaxDim) corrupt("dim " + std::to_string(dim) + " out of range [2, 65535]");
}
void check_n(uint64_t n) {
  if (n > kMaxVectors) corrupt("n_vectors " + std::to_string(n) + " exceeds MAX_VECTORS=67108864");
}
void check_payload(File& f, const char* label, uint64_t payload) {
  if (payload > (128ull << 30)) corrupt("payload " + std::to_string(payload) + " B exceeds MAX_PAYLOAD");
  uint64_t rem = f.size - f.pos();
  if (payload > rem)
    corrupt(std::string(label) + " payload truncated: header declares " + std::to_string(payload) +
            " B but file has " + std::to_string(rem) + " B remaining");
  if (payload < rem)
    corrupt(std::string(label) + " payload has trailing bytes: header declares " + std::to_string(payload) +
            " B but file has " + std::to_string(rem) + " B remaining");
}

struct Header {
  Fmt fmt;
  uint32_t dim = 0, bits = 0, n_top = 0;
  uint64_t n = 0, payload = 0, bytes_per_vec = 0;
};

// Reads and validates the header; leaves the file positioned at the payload.
Header read_header(File& f) {
  uint8_t m[4];
  f.read(m, 4, "ordvec index", "magic");
  Header h;
  h.fmt = lookup_magic(m);
  switch (h.fmt) {
    case Fmt::Unknown:
      corrupt("unrecognized ordvec index magic");
    case Fmt::Rank: {
      check_version(f, "OVR1");
      h.dim = f.u32("OVR1", "dim");
      check_dim(h.dim);
      h.n = f.u32("OVR1", "n_vectors");
      check_n(h.n);
      h.bytes_per_vec = 2ull * h.dim;
      h.payload = h.n * h.bytes_per_vec;
      check_payload(f, "OVR1", h.payload);
      break;
    }
    case Fmt::RankQuant: {
      check_version(f, "OVRQ");
      h.bits = f.u8("OVRQ", "bits");
      if (h.bits != 1 && h.bits != 2 && h.bits != 4)
        corrupt("unsupported OVRQ bits: " + std::to_string(h.bits) + " (expected 1, 2, or 4)");
      h.dim = f.u32("OVRQ", "dim");
      check_dim(h.dim);
      if (h.dim % (1u << h.bits))
        corrupt("OVRQ dim " + std::to_string(h.dim) + " is not a multiple of 2^bits = " +
                std::to_string(1u << h.bits) + "; constant-composition invariant violated");
      if (h.dim % (8 / h.bits))
        corrupt("OVRQ dim " + std::to_string(h.dim) + " is not a multiple of codes_per_byte");
      h.n = f.u32("OVRQ", "n_vectors");
      check_n(h.n);
      h.bytes_per_vec = (uint64_t)h.dim * h.bits / 8;
      h.payload = h.n * h.bytes_per_vec;
      check_payload(f, "OVRQ", h.payload);
      break;
    }
    case Fmt::Bitmap: {
      check_version(f, "OVBM");
      h.dim = f.u32("OVBM", "dim");
      check_dim(h.dim);
      if (h.dim % 64) corrupt("OVBM dim " + std::to_string(h.dim) + " is not a multiple of 64");
      h.n_top = f.u32("OVBM", "n_top");
      if (h.n_top == 0 || h.n_top >= h.dim)
        corrupt("OVBM n_top " + std::to_string(h.n_top) + " must satisfy 0 < n_top < dim");
      h.n = f.u32("OVBM", "n_vectors");
      check_n(h.n);
      h.bytes_per_vec = h.dim / 8;
      h.payload = h.n * h.bytes_per_vec;
      check_payload(f, "OVBM", h.payload);
      break;
    }
    case Fmt::Sign: {
      check_version(f, "OVSB");
      uint64_t dim = f.u32("OVSB", "dim");
      if (dim < 64 || dim > kMaxSignDim) corrupt("OVSB dim " + std::to_string(dim) + " out of range");
      if (dim % 64) corrupt("OVSB dim " + std::to_string(dim) + " is not a multiple of 64");
      h.dim = (uint32_t)dim;
      h.n = f.u32("OVSB", "n_vectors");
      check_n(h.n);
      h.bytes_per_vec = h.dim / 8;
      h.payload = h.n * h.bytes_per_vec;
      check_payload(f, "OVSB", h.payload);
      break;
    }
    case Fmt::FastScan: {
      check_version(f, "OVFS");
      h.dim = f.u32("OVFS", "dim");
      check_dim(h.dim);
      if (h.dim % 4) corrupt("OVFS dim " + std::to_string(h.dim) + " is not a multiple of 4");
      h.n = f.u32("OVFS", "n_vectors");
      check_n(h.n);
      h.bytes_per_vec = h.dim / 2;
      h.payload = ((h.n + 31) / 32) * (uint64_t)(h.dim / 2) * 32;
      check_payload(f, "OVFS", h.payload);
      break;
    }
  }
  return h;
}

void validate_rankquant_rows(const std::vector<uint8_t>& p, const Header& h) {
  const uint32_t cpb = 8 / h.bits, nb = 1u << h.bits, mask = nb - 1;
  const uint64_t bpv = h.bytes_per_vec, expect = h.dim / nb;
  for (uint64_t r = 0; r < h.n; r++) {
    uint32_t hist[16] = {0};
    const uint8_t* row = p.data() + r * bpv;
    for (uint64_t b = 0; b < bpv; b++)
      for (uint32_t s = 0; s < cpb; s++) hist[(row[b] >> ((cpb - 1 - s) * h.bits)) & mask]++;
    for (uint32_t b = 0; b < nb; b++)
      if (hist[b] != expect)
        corrupt("OVRQ row " + std::to_string(r) + " violates constant composition: bucket " + std::to_string(b) +
                " has " + std::to_string(hist[b]) + " codes, expected " + std::to_string(expect));
  }
}

// load_rank_from_stream (src/rank_io.rs:581-633): every row a permutation of
// [0, dim); a stamp per value marks the row that last held it.
void validate_rank_rows(const std::vector<uint8_t>& p, const Header& h) {
  std::vector<uint32_t> seen(h.dim, 0);
  for (uint64_t r = 0; r < h.n; r++) {
    const uint32_t stamp = (uint32_t)r + 1;
    for (uint64_t j = 0; j < h.dim; j++) {
      const uint8_t* b = p.data() + (r * h.dim + j) * 2;
      const uint32_t v = (uint32_t)b[0] | ((uint32_t)b[1] << 8);
      if (v >= h.dim)
        corrupt("OVR1 rank value " + std::to_string(v) + " >= dim (" + std::to_string(h.dim) +
                "); ranks must be a permutation of [0, dim)");
      if (seen[v] == stamp)
        corrupt("OVR1 row " + std::to_string(r) + " is not a permutation of [0, dim): value " + std::to_string(v) +
                " repeats");
      seen[v] = stamp;
    }
  }
}

void validate_bitmap_rows(const std::vector<uint8_t>& p, const Header& h) {
  const uint64_t qpv = h.dim / 64;
  const uint64_t* w = (const uint64_t*)p.data();
  for (uint64_t r = 0; r < h.n; r++) {
    uint32_t pop = 0;
    for (uint64_t i = 0; i < qpv; i++) pop += (uint32_t)__builtin_popcountll(w[r * qpv + i]);
    if (pop != h.n_top)
      corrupt("OVBM row " + std::to_string(r) + " has " + std::to_string(pop) + " bits set, expected n_top = " +
              std::to_string(h.n_top));
  }
}

void validate_fastscan(const std::vector<uint8_t>& p, const Header& h) {
  const uint64_t pairs = h.dim / 2, nblk = (h.n + 31) / 32, expect = h.dim / 4;
  for (uint64_t b = 0; b < nblk; b++) {
    const uint64_t din = h.n - b * 32 < 32 ? h.n - b * 32 : 32;
    const uint8_t* blk = p.data() + b * pairs * 32;
    for (uint64_t l = 0; l < 32; l++) {
      uint64_t cnt[4] = {0, 0, 0, 0};
      for (uint64_t pr = 0; pr < pairs; pr++) {
        uint8_t byte = blk[pr * 32 + l];
        if (l >= din) {
          if (byte) corrupt("OVFS tail padding byte must be zero");
          continue;
        }
        if (byte & 0xF0) corrupt("OVFS payload has invalid FastScan nibble");
        cnt[(byte >> 2) & 3]++;
        cnt[byte & 3]++;
      }
      if (l < din && (cnt[0] != expect || cnt[1] != expect || cnt[2] != expect || cnt[3] != expect))
        corrupt("OVFS document " + std::to_string(b * 32 + l) + " violates b=2 constant composition");
    }
  }
}

}  // namespace

uint64_t Index::ref_bytes_per_vec() const {
  switch (kind) {
    case ORDVEC_INDEX_KIND_RANK_QUANT:
      return bpv();
    case ORDVEC_INDEX_KIND_BITMAP:
    case OVB_INDEX_KIND_SIGN_BITMAP:
      return dim / 8;
    case OVB_INDEX_KIND_FASTSCAN:
      return dim / 2;
    case OVB_INDEX_KIND_MULTIBUCKET:
      return (uint64_t)nb() * dim / 8;
    case OVB_INDEX_KIND_RANK:
      return (uint64_t)dim * 2;
  }
  return 0;
}

uint64_t Index::device_bytes(uint64_t rows) const {
  switch (kind) {
    case ORDVEC_INDEX_KIND_RANK_QUANT:
      return rows * bpv();
    case ORDVEC_INDEX_KIND_BITMAP:
    case OVB_INDEX_KIND_SIGN_BITMAP:
      return rows * qpv() * 8;
    case OVB_INDEX_KIND_FASTSCAN:
      return ((rows + 31) / 32) * fastscan_block_bytes(pairs_pad);
    case OVB_INDEX_KIND_MULTIBUCKET:
      return rows * nb() * (dim / 64) * 8;
    case OVB_INDEX_KIND_RANK:
      return rows * dim * 2;
  }
  return 0;
}

void upload_payload(Index& ix, const uint8_t* payload, uint64_t bytes) {
  Workspace& w = workspace();
  if (ix.kind == OVB_INDEX_KIND_FASTSCAN) {
    const uint64_t dev = ix.device_bytes(ix.n);
    ix.codes.ensure(dev ? dev : 1);
    if (!ix.n) return;
    uint8_t* stage = (uint8_t*)w.stage.ensure(bytes);
    OVB_CUDA(cudaMemcpyAsync(stage, payload, bytes, cudaMemcpyHostToDevice, w.stream));
    launch_fastscan_relayout(stage, ix.n, ix.dim / 2, ix.pairs_pad, ix.codes.as<uint8_t>(), w.stream);
  } else {
    ix.codes.ensure(bytes ? bytes : 1);
    if (bytes) OVB_CUDA(cudaMemcpyAsync(ix.codes.p, payload, bytes, cudaMemcpyHostToDevice, w.stream));
  }
  OVB_CUDA(cudaStreamSynchronize(w.stream));
}

std::unique_ptr<Index> load_index_file(const char* path, bool v1_only) {
  File f(path, "open index");
  // sniff the magic first: format support is decided before any parsing
  // (ordvec-ffi/src/lib.rs:734-764)
  uint8_t m[4];
  if (f.size < 4) corrupt("read index magic: failed to fill whole buffer");
  f.read(m, 4, "ordvec index", "magic");
  const Fmt fmt = lookup_magic(m);
  if (fmt == Fmt::Unknown) corrupt("unrecognized ordvec index magic");
  if (v1_only && (fmt == Fmt::Rank || fmt == Fmt::Sign))
    fail(ORDVEC_STATUS_UNSUPPORTED_FORMAT, "ABI v1 supports only RankQuant and Bitmap indexes");
  if (v1_only && fmt == Fmt::FastScan)
    fail(ORDVEC_STATUS_UNSUPPORTED_FORMAT, "ABI v1 does not support RankQuantFastscan indexes");
  fseek(f.f, 0, SEEK_SET);
  Header h = read_header(f);
  std::vector<uint8_t> payload(h.payload);
  if (h.payload && fread(payload.data(), 1, h.payload, f.f) != h.payload) corrupt("payload read failed");
  auto ix = std::make_unique<Index>();
  ix->dim = h.dim;
  ix->n = h.n;
  ix->file_size = f.size;
  switch (h.fmt) {
    case Fmt::Rank:
      validate_rank_rows(payload, h);
      ix->kind = OVB_INDEX_KIND_RANK;
      ix->bits = 16;
      break;
    case Fmt::RankQuant:
      validate_rankquant_rows(payload, h);
      ix->kind = ORDVEC_INDEX_KIND_RANK_QUANT;
      ix->bits = h.bits;
      break;
    case Fmt::Bitmap:
      validate_bitmap_rows(payload, h);
      ix->kind = ORDVEC_INDEX_KIND_BITMAP;
      ix->n_top = h.n_top;
      break;
    case Fmt::Sign:
      ix->kind = OVB_INDEX_KIND_SIGN_BITMAP;
      break;
    case Fmt::FastScan:
      validate_fastscan(payload, h);
      ix->kind = OVB_INDEX_KIND_FASTSCAN;
      ix->bits = 2;
      ix->pairs_pad = fastscan_pairs_pad(h.dim);
      break;
    default:
      corrupt("unrecognized ordvec index magic");
  }
  ensure_device();
  OVB_CUDA(cudaGetDevice(&ix->device));
  upload_payload(*ix, payload.data(), payload.size());
  return ix;
}

void probe_index_file(const char* path, ordvec_index_info_t* info) {
  File f(path, "probe index metadata");
  if (f.size < 4) corrupt("ordvec index header truncated while reading magic");
  uint8_t m[4];
  f.read(m, 4, "ordvec index", "magic");
  Fmt fmt = lookup_magic(m);
  if (fmt == Fmt::Unknown) corrupt("unknown ordvec index magic");
  if (fmt == Fmt::FastScan)
    corrupt("OVFS (RankQuantFastscan) metadata probing is not supported in this version");
  fseek(f.f, 0, SEEK_SET);
  Header h = read_header(f);
  if (h.fmt == Fmt::Rank || h.fmt == Fmt::Sign)
    fail(ORDVEC_STATUS_UNSUPPORTED_FORMAT, "ABI v1 supports metadata probes only for RankQuant and Bitmap indexes");
  ordvec_index_info_init(info);
  info->kind = h.fmt == Fmt::RankQuant ? ORDVEC_INDEX_KIND_RANK_QUANT : ORDVEC_INDEX_KIND_BITMAP;
  info->format_version = 1;
  info->dim = h.dim;
  info->vector_count = h.n;
  info->bytes_per_vec = h.bytes_per_vec;
  info->source_file_size_bytes = f.size;
  info->bit_width = h.fmt == Fmt::RankQuant ? h.bits : 0;
  info->n_top = h.fmt == Fmt::Bitmap ? h.n_top : 0;
  info->capabilities = ORDVEC_CAP_FULL_SEARCH | ORDVEC_CAP_SUBSET_SEARCH | ORDVEC_CAP_STATS |
                       ORDVEC_CAP_ID_EQUALS_ROW_ID;
}

// Device codes -> the reference's payload layout.
void read_payload(const Index& ix, std::vector<uint8_t>& out) {
  Workspace& w = workspace();
  if (ix.kind == OVB_INDEX_KIND_FASTSCAN) {
    const uint64_t pairs = ix.dim / 2, nblk = (ix.n + 31) / 32;
    std::vector<uint8_t> dev(ix.device_bytes(ix.n));
    if (!dev.empty())
      OVB_CUDA(cudaMemcpyAsync(dev.data(), ix.codes.p, dev.size(), cudaMemcpyDeviceToHost, w.stream));
    OVB_CUDA(cudaStreamSynchronize(w.stream));
    out.assign(nblk * pairs * 32, 0);
    const uint64_t bb = fastscan_block_bytes(ix.pairs_pad);
    for (uint64_t b = 0; b < nblk; b++)
      for (uint64_t p = 0; p < pairs; p++)
        for (uint64_t l = 0; l < 32; l++) {
          const uint64_t g = p / 32, byte = (p % 32) / 2;
          const uint8_t v = dev[b * bb + (g * 32 + l) * 16 + byte];
          out[b * pairs * 32 + p * 32 + l] = (p & 1) ? (v >> 4) : (v & 15);
        }
    return;
  }
  out.resize(ix.device_bytes(ix.n));
  if (!out.empty()) OVB_CUDA(cudaMemcpyAsync(out.data(), ix.codes.p, out.size(), cudaMemcpyDeviceToHost, w.stream));
  OVB_CUDA(cudaStreamSynchronize(w.stream));
}

void write_index_file(const Index& ix, const char* path) {
  std::vector<uint8_t> payload;
  read_payload(ix, payload);
  std::vector<uint8_t> hdr;
  auto put32 = [&](uint32_t v) {
    for (int i = 0; i < 4; i++) hdr.push_back((uint8_t)(v >> (8 * i)));
  };
  switch (ix.kind) {
    case ORDVEC_INDEX_KIND_RANK_QUANT:
      hdr = {'O', 'V', 'R', 'Q', 1, (uint8_t)ix.bits};
      put32(ix.dim);
      put32((uint32_t)ix.n);
      break;
    case ORDVEC_INDEX_KIND_BITMAP:
      hdr = {'O', 'V', 'B', 'M', 1};
      put32(ix.dim);
      put32(ix.n_top);
      put32((uint32_t)ix.n);
      break;
    case OVB_INDEX_KIND_SIGN_BITMAP:
      hdr = {'O', 'V', 'S', 'B', 1};
      put32(ix.dim);
      put32((uint32_t)ix.n);
      break;
    case OVB_INDEX_KIND_FASTSCAN:
      hdr = {'O', 'V', 'F', 'S', 1};
      put32(ix.dim);
      put32((uint32_t)ix.n);
      break;
    case OVB_INDEX_KIND_RANK:
      hdr = {'O', 'V', 'R', '1', 1};
      put32(ix.dim);
      put32((uint32_t)ix.n);
      break;
    default:
      fail(ORDVEC_STATUS_UNSUPPORTED_OPERATION, "this index kind has no persisted format");
  }
  FILE* f = fopen(path, "wb");
  if (!f) fail(ORDVEC_STATUS_IO, std::string("create index file: ") + strerror(errno));
  bool ok = fwrite(hdr.data(), 1, hdr.size(), f) == hdr.size() &&
            (payload.empty() || fwrite(payload.data(), 1, payload.size(), f) == payload.size());
  ok = (fclose(f) == 0) && ok;
  if (!ok) fail(ORDVEC_STATUS_IO, "write index file failed");
}

}  // namespace ovb
