// Device-side description of one image's scale space and detection buffers.
//
// HBM layout per image (all fp32 planes row-major, pitch = width rounded up to
// 32 elements so every row starts on a 128-byte boundary):
//   octave o: G[0..S+2] (S+3 Gaussian levels), D[0..S+1] (S+2 DoG slices),
//             extremum bitmask  [S][h][words]  (bit x%32 of word x/32),
//   rows:     per (octave, slice, row) keypoint counts and exclusive offsets,
//   keypoints (capacity kp_cap) in the reference's (octave, slice, row, column) order,
//   selected keypoints (top max_features by |response|, stable), 1..4
//   orientations each, feature offsets, then the SoA feature outputs.
#pragma once

#include <stdint.h>

#include "psift_gpu.h"

namespace psift {

enum SrcKind : int { SRC_F32 = 0, SRC_U8 = 1 };

struct OctaveDev {
  int h, w;
  long long pitch;         // elements
  long long plane_stride;  // elements between consecutive planes
  float* g;                // S+3 planes
  float* d;                // S+2 planes
  uint32_t* masks;         // S * h * words
  int words;               // ceil(w / 32)
  int row_base;            // first row index of this octave in the image's row arrays
  float scale_factor;      // 0.5 or 1 times 2^o
};

struct ImagePlan {
  // input
  const void* src;         // u8 or f32, device
  long long src_stride;    // elements
  int src_h, src_w;
  int src_kind;
  int upsample;
  // scale space
  int n_oct;
  OctaveDev oct[8];
  int total_rows;          // sum over octaves of S * h
  uint32_t* row_counts;
  uint32_t* row_offsets;
  // keypoints
  psift_keypoint* kps;     // kp_cap
  uint32_t* kp_count;      // number found (may exceed kp_cap)
  psift_keypoint* sel;     // sel_cap
  uint32_t* sel_count;
  float* oris;             // sel_cap * 4
  uint32_t* ori_count;     // sel_cap
  uint32_t* feat_offsets;  // sel_cap
  uint32_t* feat_count;    // features produced (<= feat_cap)
  uint32_t* feat_total;    // features before truncation to feat_cap
  uint32_t* out_count;     // optional user-visible copy of feat_count (device), may be null
  // outputs (device)
  float* fx;
  float* fy;
  float* fscale;
  float* fresp;
  float* fori;
  float* fdesc;
  uint32_t feat_cap;
};

// Output tile of a blur CTA.
constexpr int kTileW = 64;
constexpr int kTileH = 64;

// Tile work list of a blur launch over images of different sizes: image z owns
// the linear tiles [prefix[z], prefix[z + 1]), tiles_x[z] per row of tiles.
// n = 0: the launch is a (tiles x, tiles y, images) grid over the largest image.
constexpr int kTileMapMax = 64;
struct TileMap {
  int n;
  int prefix[kTileMapMax + 1];
  int tiles_x[kTileMapMax];
};

// Kernel parameters of the extrema stage (passed by value).
struct ExtremaParams {
  float threshold;
  int scales;
  float k;                           // 2^(1/scales) in f32
  float eff_scale[8][11];            // BASE_SIGMA * mult(octave) * k.powi(s)
};

// Kernel parameters of the orientation / descriptor stages.
struct DescribeParams {
  int scales;
  uint32_t max_features;  // 0 = uncapped
  int descriptor_kind;    // 0 = Sift, 1 = RootSift
};

}  // namespace psift
