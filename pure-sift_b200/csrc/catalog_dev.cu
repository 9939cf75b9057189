// Device-resident FeatureCatalog: every entry's features, 128-bit codes and the
// entry table in device memory; PSIFTCAT v1 load and save; search_features with
// the shortlist verified as batched launches.
//
// Reference: FeatureCatalog (src/catalog.rs:182-702): upsert_entry (:324-342),
// remove (:345-353), list_summaries (:355-366), atomic_write_bytes (:203-245),
// save_binary (:401-445), load_binary (:447-540), search_features (:576-702);
// CatalogEntry::new (:122-140) for the codes of an upserted entry.
//
// Layout in HBM: structure-of-arrays over all features of all entries in entry
// order; entry e owns [offset_e, offset_e + count_e).  Descriptors are f32
// (n x 128, row-major, 512 B rows), coordinates interleaved (x, y) as the
// matcher reads them, codes 2 x u64 (word 0 = bits 0..63).  A replace or remove
// rebuilds the arrays in the new entry order with device-to-device copies.
//
// A search: query upload + quantisation, coarse votes over the resident codes
// (one launch), shortlist on the host (the reference's sort by votes, then id),
// then Lowe matching of the query against every shortlisted entry (one batched
// matcher call), similarity and homography RANSAC of every non-empty match list
// (one CTA per list, one launch each), and the tracking statistics on the host.
#include <algorithm>
#include <cerrno>
#include <cstdio>
#include <cstring>
#include <string>
#include <unordered_map>
#include <vector>

#include <sys/stat.h>
#include <unistd.h>

#include "mih.cuh"
#include "psift_internal.cuh"

namespace psift {
cudaError_t launch_quantize(const float* desc, int n, uint64_t* codes, uint8_t* u8, cudaStream_t st);
cudaError_t launch_dequantize(const uint8_t* q, int n, float* out, cudaStream_t st);
cudaError_t launch_votes(const uint64_t* q, int nq, const uint64_t* cat, const long long* offsets, int n_entries,
                         int mih, uint32_t* votes, cudaStream_t st);

namespace {

constexpr char kMagic[8] = {'P', 'S', 'I', 'F', 'T', 'C', 'A', 'T'};  // BINARY_CATALOG_MAGIC
constexpr uint32_t kVersion = 1;                                        // BINARY_CATALOG_VERSION
constexpr int kRecordBytes = 5 * 4 + 16 + 128;                          // x y scale response orientation, sig, q[128]
constexpr uint64_t kMaxFeatures = 0x7FFFFFFFull;                        // int indexing of the kernels
constexpr float kDefaultRansacThreshold = 3.0f;                         // DEFAULT_RANSAC_REPROJ_THRESHOLD

// The six feature arrays of `cap` features.
struct FeatureArrays {
  uint64_t cap = 0;
  float* desc = nullptr;
  float2* xy = nullptr;
  float* scale = nullptr;
  float* resp = nullptr;
  float* ori = nullptr;
  uint64_t* codes = nullptr;
};

void free_arrays(FeatureArrays& a) {
  cudaFree(a.desc);
  cudaFree(a.xy);
  cudaFree(a.scale);
  cudaFree(a.resp);
  cudaFree(a.ori);
  cudaFree(a.codes);
  a = FeatureArrays{};
}

cudaError_t alloc_arrays(FeatureArrays& a, uint64_t cap) {
  a = FeatureArrays{};
  a.cap = cap;
  if (cap == 0) return cudaSuccess;
  cudaError_t e = cudaMalloc(&a.desc, cap * 512);
  if (e == cudaSuccess) e = cudaMalloc(&a.xy, cap * 8);
  if (e == cudaSuccess) e = cudaMalloc(&a.scale, cap * 4);
  if (e == cudaSuccess) e = cudaMalloc(&a.resp, cap * 4);
  if (e == cudaSuccess) e = cudaMalloc(&a.ori, cap * 4);
  if (e == cudaSuccess) e = cudaMalloc(&a.codes, cap * 16);
  if (e != cudaSuccess) free_arrays(a);
  return e;
}

// Copies features [src_off, src_off + n) of `s` to [dst_off, ...) of `d`.
cudaError_t copy_range(FeatureArrays& d, uint64_t dst_off, const FeatureArrays& s, uint64_t src_off, uint64_t n,
                       cudaStream_t st) {
  if (n == 0) return cudaSuccess;
  const cudaMemcpyKind k = cudaMemcpyDeviceToDevice;
  cudaError_t e = cudaMemcpyAsync(d.desc + dst_off * 128, s.desc + src_off * 128, n * 512, k, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d.xy + dst_off, s.xy + src_off, n * 8, k, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d.scale + dst_off, s.scale + src_off, n * 4, k, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d.resp + dst_off, s.resp + src_off, n * 4, k, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d.ori + dst_off, s.ori + src_off, n * 4, k, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d.codes + dst_off * 2, s.codes + src_off * 2, n * 16, k, st);
  return e;
}

// PSIFTCAT records -> feature arrays.  The records of entry e start at byte
// file_off[e] of the uploaded file (any alignment) and fill features
// [out_off[e], out_off[e + 1]); out_off has n_entries + 1 items, the last being
// the total.  A warp takes kSplitPerWarp consecutive records, finds the first
// one's entry by binary search and walks the entries forward.  Per record,
// lane l loads 32-bit words l and 32 + l of the record's span (whole words
// around its 164 bytes; the uploaded region is padded to 256 bytes, and the
// word after the record is read only when the record is not word-aligned), and
// funnel shifts give the record's own words 0..40: x, y, scale, response,
// orientation, the stored 128-bit signature (kept as it is), then the 128
// descriptor bytes, which go to q8 for dequantize_descriptor_u8 (one 128-byte
// store per record); the other fields are gathered in shared memory and stored
// once per warp, each array's 32 entries together.
constexpr int kSplitWarps = 8;
constexpr int kSplitPerWarp = 32;
constexpr int kSplitBatch = 4;
__global__ void __launch_bounds__(kSplitWarps * 32)
    psiftcat_split_kernel(const uint8_t* __restrict__ file, const long long* __restrict__ file_off,
                          const long long* __restrict__ out_off, int n_entries, long long total, float2* xy,
                          float* scale, float* resp, float* ori, uint64_t* codes, uint8_t* q8) {
  constexpr unsigned kFull = 0xffffffffu;
  // record words 0..8 (x, y, scale, response, orientation, signature) of the
  // warp's records, field-major, written out coalesced at the end
  __shared__ uint32_t s_fld[kSplitWarps][9][kSplitPerWarp + 1];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long long i0 = ((long long)blockIdx.x * kSplitWarps + warp) * kSplitPerWarp;
  if (i0 >= total) return;
  const long long i1 = i0 + kSplitPerWarp < total ? i0 + kSplitPerWarp : total;
  int lo = 0, hi = n_entries - 1;  // last entry with out_off[e] <= i0
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (out_off[mid] <= i0) lo = mid;
    else hi = mid - 1;
  }
  int e = lo;
  long long e_begin = out_off[e], e_end = out_off[e + 1], e_file = file_off[e];
  // kSplitBatch records at a time: every record's loads are issued before the first is used
  for (long long ib = i0; ib < i1; ib += kSplitBatch) {
    uint32_t a[kSplitBatch], b[kSplitBatch], sh[kSplitBatch];
#pragma unroll
    for (int j = 0; j < kSplitBatch; ++j) {
      const long long i = ib + j;
      a[j] = b[j] = sh[j] = 0u;
      if (i >= i1) continue;
      while (e_end <= i) {  // entries without records are passed over
        ++e;
        e_begin = e_end;
        e_end = out_off[e + 1];
        e_file = file_off[e];
      }
      const unsigned long long s = (unsigned long long)(e_file + (i - e_begin) * kRecordBytes);
      const uint32_t* wbase = reinterpret_cast<const uint32_t*>(file + (s & ~3ull));
      sh[j] = (uint32_t)(s & 3u) * 8u;
      a[j] = __ldg(wbase + lane);  // span words 0..31
      if (lane < 9 || (lane == 9 && sh[j] != 0u)) b[j] = __ldg(wbase + 32 + lane);  // 32..41
    }
#pragma unroll
    for (int j = 0; j < kSplitBatch; ++j) {
      const long long i = ib + j;
      if (i >= i1) break;
      const uint32_t a_next = __shfl_down_sync(kFull, a[j], 1);
      const uint32_t b_first = __shfl_sync(kFull, b[j], 0);
      const uint32_t b_next = __shfl_down_sync(kFull, b[j], 1);
      const uint32_t o0 = __funnelshift_r(a[j], lane == 31 ? b_first : a_next, sh[j]);  // record word lane
      const uint32_t o1 = __funnelshift_r(b[j], b_next, sh[j]);  // record word 32 + lane (lanes 0..8)
      // descriptor word l = record word 9 + l
      const uint32_t qa = __shfl_sync(kFull, o0, lane + 9 < 32 ? lane + 9 : 31);
      const uint32_t qb = __shfl_sync(kFull, o1, lane >= 23 ? lane - 23 : 0);
      reinterpret_cast<uint32_t*>(q8 + i * 128)[lane] = lane <= 22 ? qa : qb;
      if (lane < 9) s_fld[warp][lane][i - i0] = o0;
    }
  }
  __syncwarp();
  const long long i = i0 + lane;
  if (i < i1) {
    const uint32_t(*f)[kSplitPerWarp + 1] = s_fld[warp];
    xy[i] = make_float2(__uint_as_float(f[0][lane]), __uint_as_float(f[1][lane]));
    scale[i] = __uint_as_float(f[2][lane]);
    resp[i] = __uint_as_float(f[3][lane]);
    ori[i] = __uint_as_float(f[4][lane]);
    reinterpret_cast<uint4*>(codes)[i] = make_uint4(f[5][lane], f[6][lane], f[7][lane], f[8][lane]);
  }
}

// Rust's str::from_utf8 acceptance rule (shortest forms, no surrogates, <= U+10FFFF).
bool valid_utf8(const uint8_t* s, size_t n) {
  size_t i = 0;
  while (i < n) {
    const uint8_t c = s[i];
    if (c < 0x80) {
      ++i;
      continue;
    }
    int len;
    uint32_t cp;
    if ((c & 0xE0) == 0xC0) {
      len = 2;
      cp = c & 0x1F;
    } else if ((c & 0xF0) == 0xE0) {
      len = 3;
      cp = c & 0x0F;
    } else if ((c & 0xF8) == 0xF0) {
      len = 4;
      cp = c & 0x07;
    } else {
      return false;
    }
    if (i + len > n) return false;
    for (int k = 1; k < len; ++k) {
      if ((s[i + k] & 0xC0) != 0x80) return false;
      cp = (cp << 6) | (s[i + k] & 0x3F);
    }
    if ((len == 2 && cp < 0x80) || (len == 3 && cp < 0x800) || (len == 4 && cp < 0x10000)) return false;
    if (cp > 0x10FFFF || (cp >= 0xD800 && cp <= 0xDFFF)) return false;
    i += len;
  }
  return true;
}

// Sequential reads of a file of known size; a short read counts as EOF.
struct FileReader {
  FILE* f;
  uint64_t pos, size;
  uint64_t left() const { return size - pos; }
  bool take(void* dst, size_t n) {
    if (left() < n || (n && std::fread(dst, 1, n, f) != n)) return false;
    pos += n;
    return true;
  }
  bool skip(uint64_t n) {
    if (left() < n || fseeko(f, (off_t)n, SEEK_CUR) != 0) return false;
    pos += n;
    return true;
  }
};

template <typename T>
void put(std::vector<uint8_t>& b, T v) {
  const size_t o = b.size();
  b.resize(o + sizeof(T));
  std::memcpy(b.data() + o, &v, sizeof(T));  // little-endian host
}

// atomic_write_bytes (src/catalog.rs:203-245): parent directories, then
// "<file name>.tmp.<pid>" beside the target, renamed over it.
psift_status atomic_write(psift_ctx* ctx, const std::string& path, const std::vector<uint8_t>& bytes) {
  const size_t slash = path.find_last_of('/');
  const std::string dir = slash == std::string::npos ? std::string() : path.substr(0, slash);
  std::string name = slash == std::string::npos ? path : path.substr(slash + 1);
  if (name.empty() || name == "." || name == "..") name = "catalog";
  if (!dir.empty()) {
    for (size_t k = 1; k <= dir.size(); ++k) {
      if (k == dir.size() || dir[k] == '/') {
        const std::string part = dir.substr(0, k);
        if (mkdir(part.c_str(), 0777) != 0 && errno != EEXIST)
          return set_error(ctx, PSIFT_ERR_IO, "Failed to create catalog directory `" + dir + "`: " + strerror(errno));
      }
    }
  }
  const std::string tmp = (dir.empty() ? std::string() : dir + "/") + name + ".tmp." + std::to_string(getpid());
  FILE* f = std::fopen(tmp.c_str(), "wb");
  if (!f) return set_error(ctx, PSIFT_ERR_IO, "Failed to create temporary catalog `" + tmp + "`: " + strerror(errno));
  const bool ok = (bytes.empty() || std::fwrite(bytes.data(), 1, bytes.size(), f) == bytes.size()) &&
                  std::fflush(f) == 0;
  const bool closed = std::fclose(f) == 0;
  if (!ok || !closed) {
    std::remove(tmp.c_str());
    return set_error(ctx, PSIFT_ERR_IO, "Failed to write catalog `" + tmp + "`");
  }
  if (std::rename(tmp.c_str(), path.c_str()) != 0) {
    const std::string why = strerror(errno);
    std::remove(tmp.c_str());
    return set_error(ctx, PSIFT_ERR_IO, "Failed to atomically replace catalog `" + path + "`: " + why);
  }
  return PSIFT_OK;
}

}  // namespace
}  // namespace psift

using namespace psift;

struct psift_catalog {
  psift_ctx* ctx = nullptr;
  psift_catalog_params params{};
  struct Entry {
    std::string id;
    uint32_t width = 0, height = 0;
    uint64_t count = 0, offset = 0;
  };
  std::vector<Entry> entries;
  std::unordered_map<std::string, uint32_t> index;  // id_index (last duplicate wins, as rebuild_indices)
  FeatureArrays a;
  uint64_t total = 0;
  char* scratch = nullptr;  // grow-only search / load workspace
  size_t scratch_cap = 0;
  // Multi-index hashing tables (src/catalog.rs:291-321), rebuilt on the first
  // votes after a change of contents (version counts upserts, removals).
  MihIndex mih;
  uint64_t version = 0;
  int32_t search_votes = PSIFT_VOTES_AUTO;

  psift_status reserve_scratch(size_t bytes) {
    if (bytes <= scratch_cap) return PSIFT_OK;
    bytes = align_up(bytes, 1 << 20);
    PSIFT_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    cudaFree(scratch);
    scratch = nullptr;
    scratch_cap = 0;
    cudaError_t e = cudaMalloc(&scratch, bytes);
    if (e != cudaSuccess) return cuda_error(ctx, e, "cudaMalloc(catalog scratch)");
    scratch_cap = bytes;
    return PSIFT_OK;
  }

  void reindex() {
    index.clear();
    uint64_t off = 0;
    for (uint32_t i = 0; i < entries.size(); ++i) {
      entries[i].offset = off;
      off += entries[i].count;
      index[entries[i].id] = i;
    }
    total = off;
  }

  // New arrays holding, in order, the old entries `order` (index into the old
  // `entries`, or -1 for `fresh_count` features uploaded afterwards by the caller).
  psift_status rebuild(const std::vector<long long>& order, uint64_t fresh_count, std::vector<Entry> next,
                       uint64_t* fresh_offset) {
    uint64_t need = 0;
    for (long long o : order) need += o < 0 ? fresh_count : entries[(size_t)o].count;
    if (need > kMaxFeatures) return set_error(ctx, PSIFT_ERR_CAPACITY, "catalog larger than 2^31-1 features");
    FeatureArrays n;
    cudaError_t e = alloc_arrays(n, std::max<uint64_t>(std::max(need, a.cap), 1024));
    if (e != cudaSuccess) return cuda_error(ctx, e, "cudaMalloc(catalog)");
    uint64_t off = 0;
    for (long long o : order) {
      if (o < 0) {
        *fresh_offset = off;
        off += fresh_count;
        continue;
      }
      const Entry& E = entries[(size_t)o];
      e = copy_range(n, off, a, E.offset, E.count, ctx->stream);
      if (e != cudaSuccess) {
        free_arrays(n);
        return cuda_error(ctx, e, "catalog reorder copy");
      }
      off += E.count;
    }
    PSIFT_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    free_arrays(a);
    a = n;
    entries = std::move(next);
    reindex();
    return PSIFT_OK;
  }

  psift_status grow(uint64_t need) {
    if (need <= a.cap) return PSIFT_OK;
    if (need > kMaxFeatures) return set_error(ctx, PSIFT_ERR_CAPACITY, "catalog larger than 2^31-1 features");
    FeatureArrays n;
    cudaError_t e = alloc_arrays(n, std::max<uint64_t>(std::max(need, 2 * a.cap), 1024));
    if (e != cudaSuccess) return cuda_error(ctx, e, "cudaMalloc(catalog)");
    e = copy_range(n, 0, a, 0, total, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) {
      free_arrays(n);
      return cuda_error(ctx, e, "catalog grow copy");
    }
    free_arrays(a);
    a = n;
    return PSIFT_OK;
  }

  // Host SoA features -> [off, off + n); codes from the descriptors.
  psift_status upload(uint64_t off, const psift_features* f) {
    const uint64_t n = f->count;
    if (n == 0) return PSIFT_OK;
    std::vector<float2> xy(n);
    for (uint64_t i = 0; i < n; ++i) xy[i] = make_float2(f->x[i], f->y[i]);
    cudaStream_t st = ctx->stream;
    PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(a.desc + off * 128, f->descriptors, n * 512, cudaMemcpyHostToDevice, st));
    PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(a.xy + off, xy.data(), n * 8, cudaMemcpyHostToDevice, st));
    PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(a.scale + off, f->scale, n * 4, cudaMemcpyHostToDevice, st));
    PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(a.resp + off, f->response, n * 4, cudaMemcpyHostToDevice, st));
    PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(a.ori + off, f->orientation, n * 4, cudaMemcpyHostToDevice, st));
    cudaError_t e = launch_quantize(a.desc + off * 128, (int)n, a.codes + off * 2, nullptr, st);
    ctx->launches++;
    if (e != cudaSuccess) return cuda_error(ctx, e, "quantize_u128");
    PSIFT_CUDA_TRY(ctx, cudaStreamSynchronize(st));  // xy lives on the host stack
    return PSIFT_OK;
  }
};

namespace {

psift_status cat_begin(const psift_catalog* cat) {
  if (!cat || !cat->ctx) return PSIFT_ERR_INVALID_ARGUMENT;
  cudaError_t e = cudaSetDevice(cat->ctx->device);
  if (e != cudaSuccess) return cuda_error(cat->ctx, e, "cudaSetDevice");
  return PSIFT_OK;
}

bool features_ok(const psift_features* f) {
  return f && (f->count == 0 ||
               (f->x && f->y && f->scale && f->response && f->orientation && f->descriptors));
}

// Whether the MIH tables can answer nq queries: the (query, entry) bitmap, the
// grouped query lists and the tables within their limits.
bool mih_index_fits(const psift_catalog* cat, uint32_t nq) {
  return (uint64_t)nq * cat->entries.size() <= kMihBitmapMaxBits && nq <= (1u << 26) &&
         cat->total <= (1ull << 28);
}

// The tables of the catalog's current contents (built on first use after a change).
psift_status ensure_mih(psift_catalog* cat) {
  if (cat->mih.valid && cat->mih.version == cat->version) return PSIFT_OK;
  std::vector<long long> off(cat->entries.size() + 1);
  for (size_t e = 0; e < cat->entries.size(); ++e) off[e] = (long long)cat->entries[e].offset;
  off[cat->entries.size()] = (long long)cat->total;
  const psift_status st = mih_build(cat->ctx, cat->mih, cat->a.codes, cat->total, off);
  if (st == PSIFT_OK) cat->mih.version = cat->version;
  return st;
}

enum ResolvedVotes { kExhaustiveScan, kMihScan, kMihIndex };

ResolvedVotes resolve_votes(const psift_catalog* cat, uint32_t nq, int32_t path) {
  switch (path) {
    case PSIFT_VOTES_MIH_SCAN: return kMihScan;
    case PSIFT_VOTES_MIH_INDEX: return kMihIndex;
    case PSIFT_VOTES_EXHAUSTIVE: return kExhaustiveScan;
    default:
      if (cat->entries.size() <= 32) return kExhaustiveScan;
      return mih_index_fits(cat, nq) ? kMihIndex : kMihScan;
  }
}

// Device votes for device query codes: the scan kernel (d_off: device entry
// offsets) or the tables (mih_scratch: mih_votes_scratch_bytes).
cudaError_t launch_catalog_votes(psift_catalog* cat, ResolvedVotes how, const uint64_t* d_codes, uint32_t nq,
                                 const long long* d_off, void* mih_scratch, uint32_t* d_votes, cudaStream_t s) {
  const uint32_t n_entries = (uint32_t)cat->entries.size();
  if (how == kMihIndex) {
    cat->ctx->launches += 2;
    return mih_votes(cat->mih, cat->a.codes, d_codes, nq, d_votes, mih_scratch, s);
  }
  cat->ctx->launches++;
  return launch_votes(d_codes, (int)nq, cat->a.codes, d_off, (int)n_entries, how == kMihScan ? 1 : 0, d_votes, s);
}

}  // namespace

extern "C" {

psift_status psift_catalog_create(psift_ctx* ctx, const psift_catalog_params* params, psift_catalog** out) {
  if (!ctx || !params || !out) return PSIFT_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  if (params->descriptor_kind != 0 && params->descriptor_kind != 1)
    return set_error(ctx, PSIFT_ERR_INVALID_ARGUMENT, "descriptor_kind must be 0 (Sift) or 1 (RootSift)");
  psift_catalog* c = new psift_catalog;
  c->ctx = ctx;
  c->params = *params;
  *out = c;
  return PSIFT_OK;
}

psift_status psift_catalog_destroy(psift_catalog* cat) {
  if (!cat) return PSIFT_OK;
  if (cat_begin(cat) == PSIFT_OK) cudaStreamSynchronize(cat->ctx->stream);
  free_arrays(cat->a);
  cudaFree(cat->scratch);
  mih_free(cat->mih);
  delete cat;
  return PSIFT_OK;
}

psift_status psift_catalog_params_get(const psift_catalog* cat, psift_catalog_params* out) {
  if (!cat || !out) return PSIFT_ERR_INVALID_ARGUMENT;
  *out = cat->params;
  return PSIFT_OK;
}

uint32_t psift_catalog_size(const psift_catalog* cat) { return cat ? (uint32_t)cat->entries.size() : 0u; }

psift_status psift_catalog_entry(const psift_catalog* cat, uint32_t i, char* id, size_t id_capacity,
                                 uint32_t* id_len, uint32_t* width, uint32_t* height, uint64_t* feature_count) {
  if (!cat) return PSIFT_ERR_INVALID_ARGUMENT;
  if (i >= cat->entries.size()) return set_error(cat->ctx, PSIFT_ERR_INVALID_ARGUMENT, "entry index out of range");
  const psift_catalog::Entry& E = cat->entries[i];
  if (id && id_capacity) {
    const size_t n = std::min(E.id.size(), id_capacity - 1);
    std::memcpy(id, E.id.data(), n);
    id[n] = 0;
  }
  if (id_len) *id_len = (uint32_t)E.id.size();
  if (width) *width = E.width;
  if (height) *height = E.height;
  if (feature_count) *feature_count = E.count;
  return PSIFT_OK;
}

psift_status psift_catalog_find(const psift_catalog* cat, const char* id, uint32_t* index) {
  if (!cat || !id || !index) return PSIFT_ERR_INVALID_ARGUMENT;
  auto it = cat->index.find(id);
  if (it == cat->index.end()) return set_error(cat->ctx, PSIFT_ERR_INVALID_ARGUMENT, std::string("no entry `") + id + "`");
  *index = it->second;
  return PSIFT_OK;
}

psift_status psift_catalog_upsert(psift_catalog* cat, const char* id, uint32_t width, uint32_t height,
                                  const psift_features* f) {
  psift_status st = cat_begin(cat);
  if (st != PSIFT_OK) return st;
  if (!id || !features_ok(f)) return set_error(cat->ctx, PSIFT_ERR_INVALID_ARGUMENT, "null argument");
  ++cat->version;
  psift_catalog::Entry E;
  E.id = id;
  E.width = width;
  E.height = height;
  E.count = f->count;
  auto it = cat->index.find(E.id);
  if (it != cat->index.end()) {
    // entries[existing] = entry; rebuild_indices(): same position, new features
    const uint32_t at = it->second;
    std::vector<long long> order;
    std::vector<psift_catalog::Entry> next = cat->entries;
    next[at] = E;
    for (uint32_t k = 0; k < cat->entries.size(); ++k) order.push_back(k == at ? -1 : (long long)k);
    uint64_t off = 0;
    if ((st = cat->rebuild(order, E.count, std::move(next), &off)) != PSIFT_OK) return st;
    return cat->upload(off, f);
  }
  if ((st = cat->grow(cat->total + E.count)) != PSIFT_OK) return st;
  const uint64_t off = cat->total;
  if ((st = cat->upload(off, f)) != PSIFT_OK) return st;
  E.offset = off;
  cat->index[E.id] = (uint32_t)cat->entries.size();
  cat->entries.push_back(E);
  cat->total += E.count;
  return PSIFT_OK;
}

psift_status psift_catalog_remove(psift_catalog* cat, const char* id, int32_t* removed) {
  psift_status st = cat_begin(cat);
  if (st != PSIFT_OK) return st;
  if (!id || !removed) return set_error(cat->ctx, PSIFT_ERR_INVALID_ARGUMENT, "null argument");
  *removed = 0;
  auto it = cat->index.find(id);
  if (it == cat->index.end()) return PSIFT_OK;
  // entries.swap_remove(idx): the last entry takes the removed one's place
  const uint32_t at = it->second, last = (uint32_t)cat->entries.size() - 1;
  std::vector<long long> order;
  std::vector<psift_catalog::Entry> next;
  for (uint32_t k = 0; k < last; ++k) {
    const uint32_t src = k == at ? last : k;
    order.push_back(src);
    next.push_back(cat->entries[src]);
  }
  uint64_t unused = 0;
  ++cat->version;
  if ((st = cat->rebuild(order, 0, std::move(next), &unused)) != PSIFT_OK) return st;
  *removed = 1;
  return PSIFT_OK;
}

psift_status psift_catalog_features(psift_catalog* cat, uint32_t i, psift_features* out, uint64_t* codes) {
  psift_status st = cat_begin(cat);
  if (st != PSIFT_OK) return st;
  psift_ctx* ctx = cat->ctx;
  if (!out) return set_error(ctx, PSIFT_ERR_INVALID_ARGUMENT, "null output");
  if (i >= cat->entries.size()) return set_error(ctx, PSIFT_ERR_INVALID_ARGUMENT, "entry index out of range");
  const psift_catalog::Entry& E = cat->entries[i];
  out->count = (uint32_t)E.count;
  if (E.count > out->capacity) return set_error(ctx, PSIFT_ERR_CAPACITY, "feature output capacity too small");
  if (E.count == 0) return PSIFT_OK;
  psift_features probe = *out;
  probe.count = 1;
  if (!features_ok(&probe)) return set_error(ctx, PSIFT_ERR_INVALID_ARGUMENT, "null feature array");
  const uint64_t n = E.count, o = E.offset;
  std::vector<float2> xy(n);
  cudaStream_t s = ctx->stream;
  const cudaMemcpyKind k = cudaMemcpyDeviceToHost;
  PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(out->descriptors, cat->a.desc + o * 128, n * 512, k, s));
  PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(xy.data(), cat->a.xy + o, n * 8, k, s));
  PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(out->scale, cat->a.scale + o, n * 4, k, s));
  PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(out->response, cat->a.resp + o, n * 4, k, s));
  PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(out->orientation, cat->a.ori + o, n * 4, k, s));
  if (codes) PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(codes, cat->a.codes + o * 2, n * 16, k, s));
  PSIFT_CUDA_TRY(ctx, cudaStreamSynchronize(s));
  for (uint64_t j = 0; j < n; ++j) {
    out->x[j] = xy[j].x;
    out->y[j] = xy[j].y;
  }
  return PSIFT_OK;
}

psift_status psift_catalog_load_binary(psift_ctx* ctx, const char* path, psift_catalog** out) {
  if (!ctx || !path || !out) return PSIFT_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  cudaError_t ce = cudaSetDevice(ctx->device);
  if (ce != cudaSuccess) return cuda_error(ctx, ce, "cudaSetDevice");
  const std::string p = path;
  FILE* f = std::fopen(path, "rb");
  if (!f) return set_error(ctx, PSIFT_ERR_IO, "Failed to read binary catalog `" + p + "`: " + strerror(errno));
  struct Closer {
    FILE* f;
    ~Closer() { std::fclose(f); }
  } closer{f};
  struct stat sb;
  if (fstat(fileno(f), &sb) != 0)
    return set_error(ctx, PSIFT_ERR_IO, "Failed to read binary catalog `" + p + "`: " + strerror(errno));
  FileReader r{f, 0, (uint64_t)sb.st_size};
  // Pass 1: header and entry table (the reference's read order and messages),
  // seeking over the record blocks.
  const std::string eof = "Unexpected EOF while reading binary catalog";
  char magic[8];
  if (!r.take(magic, 8)) return set_error(ctx, PSIFT_ERR_FORMAT, eof);
  if (std::memcmp(magic, kMagic, 8) != 0)
    return set_error(ctx, PSIFT_ERR_FORMAT, "Invalid binary catalog magic header in `" + p + "`");
  uint32_t version = 0, octaves = 0, scales = 0;
  float threshold = 0.0f;
  uint8_t kind = 0;
  uint64_t n_entries = 0;
  if (!r.take(&version, 4)) return set_error(ctx, PSIFT_ERR_FORMAT, eof);
  if (version != kVersion)
    return set_error(ctx, PSIFT_ERR_FORMAT, "Unsupported binary catalog version " + std::to_string(version) + " in `" +
                                                p + "` (expected 1)");
  if (!r.take(&octaves, 4) || !r.take(&scales, 4) || !r.take(&threshold, 4) || !r.take(&kind, 1))
    return set_error(ctx, PSIFT_ERR_FORMAT, eof);
  if (kind > 1)
    return set_error(ctx, PSIFT_ERR_FORMAT,
                     "Unknown descriptor kind " + std::to_string(kind) + " in binary catalog `" + p + "`");
  if (!r.take(&n_entries, 8)) return set_error(ctx, PSIFT_ERR_FORMAT, eof);
  std::vector<psift_catalog::Entry> entries;
  std::vector<long long> file_off, out_off;
  uint64_t total = 0;
  for (uint64_t e = 0; e < n_entries; ++e) {
    uint32_t id_len = 0, w = 0, h = 0;
    uint64_t cnt = 0;
    if (!r.take(&id_len, 4)) return set_error(ctx, PSIFT_ERR_FORMAT, eof);
    if (r.left() < id_len) return set_error(ctx, PSIFT_ERR_FORMAT, "Truncated entry id in binary catalog");
    psift_catalog::Entry E;
    E.id.resize(id_len);
    if (!r.take(&E.id[0], id_len)) return set_error(ctx, PSIFT_ERR_IO, "Failed to read binary catalog `" + p + "`");
    if (!valid_utf8(reinterpret_cast<const uint8_t*>(E.id.data()), id_len))
      return set_error(ctx, PSIFT_ERR_FORMAT, "Invalid UTF-8 entry id in binary catalog");
    if (!r.take(&w, 4) || !r.take(&h, 4) || !r.take(&cnt, 8)) return set_error(ctx, PSIFT_ERR_FORMAT, eof);
    // every record must be present before the next header (the reference's reads)
    if (cnt > r.left() / kRecordBytes) return set_error(ctx, PSIFT_ERR_FORMAT, eof);
    E.width = w;
    E.height = h;
    E.count = cnt;
    E.offset = total;
    file_off.push_back((long long)r.pos);
    out_off.push_back((long long)total);
    if (!r.skip(cnt * kRecordBytes)) return set_error(ctx, PSIFT_ERR_IO, "Failed to read binary catalog `" + p + "`");
    total += cnt;
    if (total > kMaxFeatures) return set_error(ctx, PSIFT_ERR_CAPACITY, "catalog larger than 2^31-1 features");
    entries.push_back(std::move(E));
  }
  out_off.push_back((long long)total);

  psift_catalog_params prm{octaves, scales, threshold, (int32_t)kind};
  psift_catalog* cat = nullptr;
  psift_status st = psift_catalog_create(ctx, &prm, &cat);
  if (st != PSIFT_OK) return st;
  auto fail = [&](psift_status s) {
    psift_catalog_destroy(cat);
    return s;
  };
  cat->entries = std::move(entries);
  cat->reindex();
  if (total > 0) {
    ce = alloc_arrays(cat->a, std::max<uint64_t>(total, 1024));
    if (ce != cudaSuccess) return fail(cuda_error(ctx, ce, "cudaMalloc(catalog)"));
    // Device workspace: the file up to its last record, the two offset tables
    // and the u8 descriptors.
    const uint64_t used = r.pos;
    const size_t fb = align_up(used, 256), tb = align_up(8 * out_off.size(), 256);
    if ((st = cat->reserve_scratch(fb + 2 * tb + total * 128)) != PSIFT_OK) return fail(st);
    uint8_t* d_file = (uint8_t*)cat->scratch;
    long long* d_foff = (long long*)(cat->scratch + fb);
    long long* d_ooff = (long long*)(cat->scratch + fb + tb);
    uint8_t* d_q8 = (uint8_t*)(cat->scratch + fb + 2 * tb);
    // Pass 2: the file streamed into two pinned staging halves; the copy of one
    // half to the device overlaps the read into the other.
    constexpr size_t kChunk = 32u << 20;
    if ((st = pinned_reserve(ctx, 2 * kChunk)) != PSIFT_OK) return fail(st);
    if (std::fseek(f, 0, SEEK_SET) != 0) return fail(set_error(ctx, PSIFT_ERR_IO, "Failed to read binary catalog `" + p + "`"));
    cudaEvent_t ev[2] = {nullptr, nullptr};
    for (auto& x : ev)
      if ((ce = cudaEventCreateWithFlags(&x, cudaEventDisableTiming)) != cudaSuccess) break;
    bool used_buf[2] = {false, false}, short_read = false;
    for (uint64_t off = 0, k = 0; ce == cudaSuccess && off < used; off += kChunk, k ^= 1) {
      const size_t n = (size_t)std::min<uint64_t>(kChunk, used - off);
      if (used_buf[k]) cudaEventSynchronize(ev[k]);
      char* hbuf = ctx->pinned.base + k * kChunk;
      if (std::fread(hbuf, 1, n, f) != n) {
        short_read = true;
        break;
      }
      ce = cudaMemcpyAsync(d_file + off, hbuf, n, cudaMemcpyHostToDevice, ctx->stream);
      if (ce == cudaSuccess) ce = cudaEventRecord(ev[k], ctx->stream);
      used_buf[k] = true;
    }
    if (ce == cudaSuccess && !short_read) {
      ce = cudaMemcpyAsync(d_foff, file_off.data(), 8 * file_off.size(), cudaMemcpyHostToDevice, ctx->stream);
      if (ce == cudaSuccess)
        ce = cudaMemcpyAsync(d_ooff, out_off.data(), 8 * out_off.size(), cudaMemcpyHostToDevice, ctx->stream);
      if (ce == cudaSuccess) {
        const long long per_block = (long long)kSplitWarps * kSplitPerWarp;
        const long long blocks = ((long long)total + per_block - 1) / per_block;
        psiftcat_split_kernel<<<(unsigned)blocks, kSplitWarps * 32, 0, ctx->stream>>>(
            d_file, d_foff, d_ooff, (int)file_off.size(), (long long)total, cat->a.xy, cat->a.scale, cat->a.resp,
            cat->a.ori, cat->a.codes, d_q8);
        ctx->launches++;
        ce = cudaGetLastError();
      }
      if (ce == cudaSuccess) {
        ce = launch_dequantize(d_q8, (int)total, cat->a.desc, ctx->stream);
        ctx->launches++;
      }
    }
    const cudaError_t cs = cudaStreamSynchronize(ctx->stream);
    if (ce == cudaSuccess) ce = cs;
    for (auto& x : ev)
      if (x) cudaEventDestroy(x);
    if (ce != cudaSuccess) return fail(cuda_error(ctx, ce, "PSIFTCAT upload"));
    if (short_read) return fail(set_error(ctx, PSIFT_ERR_IO, "Failed to read binary catalog `" + p + "`"));
  }
  *out = cat;
  return PSIFT_OK;
}

psift_status psift_catalog_save_binary(psift_catalog* cat, const char* path) {
  psift_status st = cat_begin(cat);
  if (st != PSIFT_OK) return st;
  psift_ctx* ctx = cat->ctx;
  if (!path) return set_error(ctx, PSIFT_ERR_INVALID_ARGUMENT, "null path");
  const uint64_t n = cat->total;
  std::vector<float2> xy(n);
  std::vector<float> sc(n), rs(n), orr(n);
  std::vector<uint64_t> codes(2 * n);
  std::vector<uint8_t> q(128 * n);
  if (n) {
    // quantize_descriptor_u8 of the resident f32 descriptors, as the reference's save does
    if ((st = cat->reserve_scratch(n * 128)) != PSIFT_OK) return st;
    cudaError_t e = launch_quantize(cat->a.desc, (int)n, nullptr, (uint8_t*)cat->scratch, ctx->stream);
    ctx->launches++;
    if (e != cudaSuccess) return cuda_error(ctx, e, "quantize_u8");
    cudaStream_t s = ctx->stream;
    const cudaMemcpyKind k = cudaMemcpyDeviceToHost;
    PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(q.data(), cat->scratch, n * 128, k, s));
    PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(xy.data(), cat->a.xy, n * 8, k, s));
    PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(sc.data(), cat->a.scale, n * 4, k, s));
    PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(rs.data(), cat->a.resp, n * 4, k, s));
    PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(orr.data(), cat->a.ori, n * 4, k, s));
    PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(codes.data(), cat->a.codes, n * 16, k, s));
    PSIFT_CUDA_TRY(ctx, cudaStreamSynchronize(s));
  }
  std::vector<uint8_t> b;
  b.reserve(64 + cat->entries.size() * 64 + n * kRecordBytes);
  b.insert(b.end(), kMagic, kMagic + 8);
  put<uint32_t>(b, kVersion);
  put<uint32_t>(b, cat->params.octaves);
  put<uint32_t>(b, cat->params.scales);
  put<float>(b, cat->params.threshold);
  put<uint8_t>(b, (uint8_t)cat->params.descriptor_kind);
  put<uint64_t>(b, (uint64_t)cat->entries.size());
  for (const psift_catalog::Entry& E : cat->entries) {
    put<uint32_t>(b, (uint32_t)E.id.size());
    b.insert(b.end(), E.id.begin(), E.id.end());
    put<uint32_t>(b, E.width);
    put<uint32_t>(b, E.height);
    put<uint64_t>(b, E.count);
    for (uint64_t j = E.offset; j < E.offset + E.count; ++j) {
      put<float>(b, xy[j].x);
      put<float>(b, xy[j].y);
      put<float>(b, sc[j]);
      put<float>(b, rs[j]);
      put<float>(b, orr[j]);
      put<uint64_t>(b, codes[2 * j]);
      put<uint64_t>(b, codes[2 * j + 1]);
      b.insert(b.end(), q.begin() + 128 * j, q.begin() + 128 * (j + 1));
    }
  }
  return atomic_write(ctx, path, b);
}

psift_status psift_catalog_search(psift_catalog* cat, const psift_features* query, uint32_t top_k,
                                  uint32_t shortlist_k, float ratio, float ransac_threshold,
                                  psift_catalog_hit* hits, uint32_t capacity, uint32_t* count) {
  psift_status st = cat_begin(cat);
  if (st != PSIFT_OK) return st;
  psift_ctx* ctx = cat->ctx;
  if (!count || !features_ok(query)) return set_error(ctx, PSIFT_ERR_INVALID_ARGUMENT, "null argument");
  *count = 0;
  const uint32_t nq = query->count;
  const uint32_t n_entries = (uint32_t)cat->entries.size();
  if (n_entries == 0 || nq == 0 || top_k == 0) return PSIFT_OK;
  psift_match_options mopt{ratio, 0, PSIFT_PRECISION_BF16_RERANK};
  char msg[160];
  if ((st = psift_match_options_validate(&mopt, msg, sizeof msg)) != PSIFT_OK) return set_error(ctx, st, msg);
  psift_ransac_options ropt;
  psift_ransac_options_default(&ropt);
  ropt.reproj_threshold = ransac_threshold;
  if ((st = psift_ransac_options_validate(&ropt, msg, sizeof msg)) != PSIFT_OK) return set_error(ctx, st, msg);
  const bool own_tracking = ransac_threshold != kDefaultRansacThreshold;
  const uint32_t max_cands = std::min<uint32_t>(n_entries, std::max<uint32_t>(shortlist_k, 1));
  const ResolvedVotes how = n_entries <= 32 ? kExhaustiveScan : resolve_votes(cat, nq, cat->search_votes);
  if (how == kMihIndex && (st = ensure_mih(cat)) != PSIFT_OK) return st;
  const size_t mih_bytes = how == kMihIndex ? mih_votes_scratch_bytes(nq, n_entries) : 0;

  // Workspace (device): query, codes, offsets, votes, then per candidate the
  // match list, three masks and the model / flag / count words, then the MIH
  // votes' scratch.
  const size_t q_bytes = align_up((size_t)nq * 512, 256), xy_bytes = align_up((size_t)nq * 8, 256);
  const size_t code_bytes = align_up((size_t)nq * 16, 256), off_bytes = align_up(8 * (size_t)(n_entries + 1), 256);
  const size_t vote_bytes = align_up(4 * (size_t)n_entries, 256);
  const size_t m_bytes = align_up(sizeof(psift_match) * nq, 256), mask_bytes = align_up(nq, 256);
  constexpr size_t kWords = 64;  // [0] match count, [4..12) sim, [16..32) hom, [40..48) tracking sim
  const size_t per_cand = m_bytes + 3 * mask_bytes + kWords * 4;
  const size_t search_bytes = align_up(q_bytes + xy_bytes + code_bytes + off_bytes + vote_bytes +
                                      per_cand * max_cands, 256);
  if ((st = cat->reserve_scratch(search_bytes + mih_bytes)) != PSIFT_OK) return st;
  char* w = cat->scratch;
  float* d_q = (float*)w;
  float2* d_qxy = (float2*)(w + q_bytes);
  uint64_t* d_codes = (uint64_t*)(w + q_bytes + xy_bytes);
  long long* d_off = (long long*)(w + q_bytes + xy_bytes + code_bytes);
  uint32_t* d_votes = (uint32_t*)(w + q_bytes + xy_bytes + code_bytes + off_bytes);
  char* cand_base = w + q_bytes + xy_bytes + code_bytes + off_bytes + vote_bytes;
  cudaStream_t s = ctx->stream;

  // Step 1: coarse votes (src/catalog.rs:588-633).
  std::vector<float2> qxy(nq);
  for (uint32_t i = 0; i < nq; ++i) qxy[i] = make_float2(query->x[i], query->y[i]);
  std::vector<long long> off(n_entries + 1);
  for (uint32_t e = 0; e < n_entries; ++e) off[e] = (long long)cat->entries[e].offset;
  off[n_entries] = (long long)cat->total;
  const int mih = n_entries > 32 ? 1 : 0;
  std::vector<uint32_t> votes(n_entries);
  PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(d_q, query->descriptors, (size_t)nq * 512, cudaMemcpyHostToDevice, s));
  PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(d_qxy, qxy.data(), (size_t)nq * 8, cudaMemcpyHostToDevice, s));
  PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(d_off, off.data(), 8 * off.size(), cudaMemcpyHostToDevice, s));
  {
    StageScope sc(ctx, STAGE_HAMMING);
    cudaError_t e = launch_quantize(d_q, (int)nq, d_codes, nullptr, s);
    ctx->launches++;
    if (e == cudaSuccess) {
      e = launch_catalog_votes(cat, how, d_codes, nq, d_off, w + search_bytes, d_votes, s);
    }
    if (e != cudaSuccess) return cuda_error(ctx, e, "catalog votes");
  }
  PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(votes.data(), d_votes, 4 * (size_t)n_entries, cudaMemcpyDeviceToHost, s));
  PSIFT_CUDA_TRY(ctx, cudaStreamSynchronize(s));

  // Shortlist: MIH keeps entries with votes > 0; sort (votes desc, id asc) when too many.
  std::vector<std::pair<uint32_t, uint32_t>> cands;  // (entry, votes)
  for (uint32_t e = 0; e < n_entries; ++e)
    if (!mih || votes[e] > 0) cands.emplace_back(e, votes[e]);
  if (cands.size() > max_cands) {
    std::stable_sort(cands.begin(), cands.end(), [&](const auto& a, const auto& b) {
      if (a.second != b.second) return a.second > b.second;
      return cat->entries[a.first].id < cat->entries[b.first].id;
    });
    cands.resize(max_cands);
  }

  // Step 2: Lowe matching against every candidate with >= 2 features (one batched call).
  std::vector<uint32_t> live;  // positions into cands
  for (uint32_t c = 0; c < cands.size(); ++c)
    if (cat->entries[cands[c].first].count >= 2) live.push_back(c);
  struct Slot {
    psift_match* m;
    uint8_t* mask_sim;
    uint8_t* mask_hom;
    uint8_t* mask_trk;
    uint32_t* words;
  };
  std::vector<Slot> slot(live.size());
  std::vector<psift_match_job> mjobs;
  for (size_t k = 0; k < live.size(); ++k) {
    char* b = cand_base + per_cand * k;
    slot[k] = Slot{(psift_match*)b, (uint8_t*)(b + m_bytes), (uint8_t*)(b + m_bytes + mask_bytes),
                   (uint8_t*)(b + m_bytes + 2 * mask_bytes), (uint32_t*)(b + m_bytes + 3 * mask_bytes)};
    const psift_catalog::Entry& E = cat->entries[cands[live[k]].first];
    mjobs.push_back(psift_match_job{d_q, cat->a.desc + E.offset * 128, (const float*)d_qxy,
                                    (const float*)(cat->a.xy + E.offset), nq, (uint32_t)E.count, slot[k].m, nq,
                                    slot[k].words});
  }
  std::vector<uint32_t> n_raw(live.size(), 0);
  if (!live.empty()) {
    PSIFT_CUDA_TRY(ctx, cudaMemsetAsync(cand_base, 0, per_cand * live.size(), s));
    PSIFT_CUDA_TRY(ctx, cudaMemsetAsync(ctx->d_error, 0, sizeof(uint32_t), s));
    if ((st = psift_match_batch_dev(ctx, mjobs.data(), (uint32_t)mjobs.size(), &mopt)) != PSIFT_OK) return st;
    uint32_t err = 0;
    for (size_t k = 0; k < live.size(); ++k)
      PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(&n_raw[k], slot[k].words, 4, cudaMemcpyDeviceToHost, s));
    PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(&err, ctx->d_error, 4, cudaMemcpyDeviceToHost, s));
    PSIFT_CUDA_TRY(ctx, cudaStreamSynchronize(s));
    if (err & kErrTimeout) return set_error(ctx, PSIFT_ERR_TIMEOUT, "tensor-core matcher wait timed out");
  }

  // Step 3: similarity + homography RANSAC of every non-empty list (and the
  // tracking summary's own similarity RANSAC when the threshold differs from
  // the default it uses).
  std::vector<size_t> verified;  // indices into live with raw matches
  std::vector<psift_ransac_job> sim, hom, trk;
  for (size_t k = 0; k < live.size(); ++k) {
    if (n_raw[k] == 0) continue;
    verified.push_back(k);
    uint32_t* W = slot[k].words;
    sim.push_back(psift_ransac_job{slot[k].m, n_raw[k], slot[k].mask_sim, (float*)(W + 4), (int32_t*)(W + 1),
                                   W + 2, nullptr, nullptr});
    hom.push_back(psift_ransac_job{slot[k].m, n_raw[k], slot[k].mask_hom, (float*)(W + 16), (int32_t*)(W + 12),
                                   W + 13, nullptr, nullptr});
    if (own_tracking)
      trk.push_back(psift_ransac_job{slot[k].m, n_raw[k], slot[k].mask_trk, (float*)(W + 40), (int32_t*)(W + 36),
                                     W + 37, nullptr, nullptr});
  }
  if (!verified.empty()) {
    if ((st = psift_ransac_batch_dev(ctx, sim.data(), (uint32_t)sim.size(), &ropt, 0)) != PSIFT_OK) return st;
    if ((st = psift_ransac_batch_dev(ctx, hom.data(), (uint32_t)hom.size(), &ropt, 1)) != PSIFT_OK) return st;
    if (own_tracking) {
      psift_ransac_options dopt;
      psift_ransac_options_default(&dopt);
      if ((st = psift_ransac_batch_dev(ctx, trk.data(), (uint32_t)trk.size(), &dopt, 0)) != PSIFT_OK) return st;
    }
  }

  // Step 4: results to the host; tracking statistics and the hit list.
  std::vector<psift_catalog_hit> out;
  std::vector<const psift_catalog::Entry*> out_entry;
  if (!verified.empty()) {
    const size_t nv = verified.size();
    std::vector<std::vector<psift_match>> hm(nv);
    std::vector<std::vector<uint8_t>> hmask(nv);
    std::vector<std::vector<float>> tsc(nv), tor(nv);
    std::vector<uint32_t> words(nv * kWords);
    for (size_t v = 0; v < nv; ++v) {
      const size_t k = verified[v];
      const psift_catalog::Entry& E = cat->entries[cands[live[k]].first];
      hm[v].resize(n_raw[k]);
      hmask[v].resize(n_raw[k]);
      tsc[v].resize(E.count);
      tor[v].resize(E.count);
      PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(hm[v].data(), slot[k].m, sizeof(psift_match) * n_raw[k],
                                          cudaMemcpyDeviceToHost, s));
      PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(hmask[v].data(), own_tracking ? slot[k].mask_trk : slot[k].mask_sim,
                                          n_raw[k], cudaMemcpyDeviceToHost, s));
      PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(words.data() + v * kWords, slot[k].words, kWords * 4,
                                          cudaMemcpyDeviceToHost, s));
      PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(tsc[v].data(), cat->a.scale + E.offset, 4 * E.count,
                                          cudaMemcpyDeviceToHost, s));
      PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(tor[v].data(), cat->a.ori + E.offset, 4 * E.count,
                                          cudaMemcpyDeviceToHost, s));
    }
    PSIFT_CUDA_TRY(ctx, cudaStreamSynchronize(s));
    for (size_t v = 0; v < nv; ++v) {
      const size_t k = verified[v];
      const uint32_t* W = words.data() + v * kWords;
      psift_catalog_hit H;
      std::memset(&H, 0, sizeof H);
      H.entry = cands[live[k]].first;
      H.coarse_votes = cands[live[k]].second;
      tracking_stats(hm[v].data(), n_raw[k], hmask[v].data(), query->scale, query->orientation, tsc[v].data(),
                     tor[v].data(), &H.tracking);
      const uint32_t sim_in = W[2], hom_in = W[13];
      const uint32_t best = std::max(hom_in, sim_in);
      H.tracking.match_count = best;
      H.tracking.inlier_ratio = (float)best / (float)H.tracking.raw_match_count;
      H.has_similarity = (int32_t)W[1];
      std::memcpy(H.similarity, W + 4, sizeof H.similarity);
      H.has_homography = (int32_t)W[12];
      std::memcpy(H.homography, W + 16, sizeof H.homography);
      out.push_back(H);
    }
  }
  // match_count desc, inlier_ratio desc (NaN compares equal), votes desc, id asc
  std::vector<size_t> order(out.size());
  for (size_t i = 0; i < order.size(); ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](size_t i, size_t j) {
    const psift_catalog_hit &a = out[i], &b = out[j];
    if (a.tracking.match_count != b.tracking.match_count) return a.tracking.match_count > b.tracking.match_count;
    const float ra = a.tracking.inlier_ratio, rb = b.tracking.inlier_ratio;
    if (ra > rb) return true;
    if (ra < rb) return false;
    if (a.coarse_votes != b.coarse_votes) return a.coarse_votes > b.coarse_votes;
    return cat->entries[a.entry].id < cat->entries[b.entry].id;
  });
  const uint32_t n_out = (uint32_t)std::min<size_t>(order.size(), top_k);
  *count = n_out;
  if (n_out > capacity) return set_error(ctx, PSIFT_ERR_CAPACITY, "hit output capacity too small");
  if (n_out && !hits) return set_error(ctx, PSIFT_ERR_INVALID_ARGUMENT, "null hit output");
  for (uint32_t i = 0; i < n_out; ++i) hits[i] = out[order[i]];
  return PSIFT_OK;
}


psift_status psift_catalog_votes(psift_catalog* cat, const uint64_t* query_codes, uint32_t nq, int32_t path,
                                 uint32_t* votes) {
  psift_status st = cat_begin(cat);
  if (st != PSIFT_OK) return st;
  psift_ctx* ctx = cat->ctx;
  if (path < PSIFT_VOTES_AUTO || path > PSIFT_VOTES_EXHAUSTIVE)
    return set_error(ctx, PSIFT_ERR_INVALID_ARGUMENT, "votes path must be one of PSIFT_VOTES_*");
  const uint32_t n_entries = (uint32_t)cat->entries.size();
  if (n_entries == 0) return PSIFT_OK;
  if (!votes || (nq && !query_codes)) return set_error(ctx, PSIFT_ERR_INVALID_ARGUMENT, "null argument");
  const ResolvedVotes how = resolve_votes(cat, nq, path);
  if (how == kMihIndex && !mih_index_fits(cat, nq))
    return set_error(ctx, PSIFT_ERR_CAPACITY, "MIH tables cannot serve this query: (query, entry) bitmap above 2^30 bits");
  if (how == kMihIndex && (st = ensure_mih(cat)) != PSIFT_OK) return st;
  const size_t code_bytes = align_up((size_t)nq * 16 + 16, 256), off_bytes = align_up(8 * (size_t)(n_entries + 1), 256);
  const size_t vote_bytes = align_up(4 * (size_t)n_entries, 256);
  const size_t mih_bytes = how == kMihIndex ? mih_votes_scratch_bytes(nq, n_entries) : 0;
  if ((st = cat->reserve_scratch(code_bytes + off_bytes + vote_bytes + mih_bytes)) != PSIFT_OK) return st;
  char* w = cat->scratch;
  uint64_t* d_codes = (uint64_t*)w;
  long long* d_off = (long long*)(w + code_bytes);
  uint32_t* d_votes = (uint32_t*)(w + code_bytes + off_bytes);
  cudaStream_t s = ctx->stream;
  std::vector<long long> off(n_entries + 1);
  for (uint32_t e = 0; e < n_entries; ++e) off[e] = (long long)cat->entries[e].offset;
  off[n_entries] = (long long)cat->total;
  if (nq) PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(d_codes, query_codes, (size_t)nq * 16, cudaMemcpyHostToDevice, s));
  PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(d_off, off.data(), 8 * off.size(), cudaMemcpyHostToDevice, s));
  {
    StageScope sc(ctx, STAGE_HAMMING);
    const cudaError_t e = launch_catalog_votes(cat, how, d_codes, nq, d_off, w + code_bytes + off_bytes + vote_bytes,
                                               d_votes, s);
    if (e != cudaSuccess) return cuda_error(ctx, e, "catalog votes");
  }
  PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(votes, d_votes, 4 * (size_t)n_entries, cudaMemcpyDeviceToHost, s));
  PSIFT_CUDA_TRY(ctx, cudaStreamSynchronize(s));
  return PSIFT_OK;
}

psift_status psift_catalog_set_search_votes(psift_catalog* cat, int32_t path) {
  if (!cat) return PSIFT_ERR_INVALID_ARGUMENT;
  if (path != PSIFT_VOTES_AUTO && path != PSIFT_VOTES_MIH_SCAN)
    return set_error(cat->ctx, PSIFT_ERR_INVALID_ARGUMENT, "search votes must be PSIFT_VOTES_AUTO or PSIFT_VOTES_MIH_SCAN");
  cat->search_votes = path;
  return PSIFT_OK;
}

}  // extern "C"
