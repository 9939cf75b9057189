// Multi-index hashing (MIH) inverted tables of the device-resident catalog.
//
// Reference: FeatureCatalog's 16 x 256 tables (src/catalog.rs:291-321): for
// each byte band b of a signature and each key k, the (entry, signature) pairs
// whose byte b equals k; the MIH branch of search_features' coarse votes
// (:596-621) visits, per query, the 16 buckets its own bytes select and counts
// each entry at most once per query (seen_stamp).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "psift_internal.cuh"

namespace psift {

constexpr int kMihBands = 16, kMihKeys = 256, kMihBuckets = kMihBands * kMihKeys;
// Votes through the index need a (query, entry) bitmap; above this many bits the
// catalog search scans every code with the MIH acceptance rule instead (same votes).
constexpr uint64_t kMihBitmapMaxBits = 1ull << 30;  // 128 MB

// A run of at most kMihChunk consecutive items of one bucket: one CTA of the votes kernel.
constexpr int kMihChunk = 1024;
struct MihChunk {
  uint32_t bucket;
  uint32_t count;
  unsigned long long start;  // first item (global position in `items`)
};

// The index over `n` features (global feature order of the catalog arrays).
// Device arrays are grow-only; `valid` says whether they describe the catalog's
// current contents (`version`).
struct MihIndex {
  uint64_t n = 0;
  uint32_t n_entries = 0;
  uint64_t version = 0;
  bool valid = false;
  uint32_t* items = nullptr;             // [16 n] feature indices, bucket-major (b * 256 + k)
  unsigned long long* off = nullptr;     // [4097] bucket starts in `items`
  uint32_t* entry_of = nullptr;          // [n] entry of each feature
  uint32_t* block_hist = nullptr;        // build scratch: per build block, per bucket
  MihChunk* chunks = nullptr;            // work list of the votes kernel
  uint32_t n_chunks = 0;
  uint64_t cap_n = 0, cap_chunks = 0;
  uint64_t max_bucket = 0;               // largest bucket (items)
};

void mih_free(MihIndex& m);

// Builds the tables over codes[0..n) (2 x u64 per feature) with entry e owning
// features [offsets[e], offsets[e + 1]) (host array of n_entries + 1).  Runs on
// ctx->stream and synchronises it once (the chunk list is made on the host).
psift_status mih_build(psift_ctx* ctx, MihIndex& m, const uint64_t* codes, uint64_t n,
                       const std::vector<long long>& offsets);

// Device scratch bytes that mih_votes needs for nq queries over n_entries entries.
size_t mih_votes_scratch_bytes(uint32_t nq, uint32_t n_entries);

// votes[e] = number of queries with a signature of entry e that shares one of its
// 16 bytes with the query and is within 24 bits of it (the reference's MIH
// votes), through the tables.  qcodes: device, 2 x u64 per query; votes: device,
// n_entries words; scratch: mih_votes_scratch_bytes.  Launches 2 kernels and 2
// memsets on `st`; returns the first error.
cudaError_t mih_votes(const MihIndex& m, const uint64_t* catalog_codes, const uint64_t* qcodes, uint32_t nq,
                      uint32_t* votes, void* scratch, cudaStream_t st);

}  // namespace psift
