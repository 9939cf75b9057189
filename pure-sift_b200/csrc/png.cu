// Input step of the extract path for PNG: bytes -> u8 luma in device memory -> features.
//
// Reference: decode_validated_dynamic_image / decode_validated_luma8
// (src/cli.rs:129-170): the header's size is checked (MIN_IMAGE_DIM, and
// MAX_IMAGE_DIM / MAX_IMAGE_PIXELS when the pixel cap is enforced), the bytes are
// decoded by the image crate 0.25.10 with its png 0.18.1 decoder (neither is in
// the tree) and converted by DynamicImage::into_luma8.  PNG decoding is lossless
// and fully specified (ISO/IEC 15948: zlib stream of filtered scanlines, five
// filter types, Adam7 interlacing), so every conforming decoder yields the same
// samples; the luma conversion is the image crate's published rule:
//   * gray 1/2/4 bits: expanded to 8 bits by the png crate (v * 255 / (2^bits - 1));
//   * palette: expanded to the PLTE colour; RGB(A) and gray+alpha: alpha dropped;
//   * RGB: (2126 R + 7152 G + 722 B) / 10000 in u32 with truncation (rgb_to_luma),
//     computed on the samples' own type, 8 or 16 bits;
//   * 16-bit results to u8: (v + 128) / 257 (round(v * 255 / 65535)).
//
// Here the zlib stream is inflated on host threads (zlib; the sequential step,
// as nvJPEG's Huffman stage), the filtered scanlines are copied to the device and
// png_unfilter_kernel undoes the row filters there: a warp per image (or Adam7
// pass) takes 32 rows at a time as a wavefront, lane t on row t one pixel behind
// lane t - 1, so the pixel above (and above-left) comes from the neighbour lane
// by a shuffle and every filter type (Sub, Up, Average, Paeth) runs branch-free
// in lockstep.  png_luma_kernel then expands, de-interlaces and converts each
// pixel straight into the detection batch's input slot.
#include <zlib.h>

#include <algorithm>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "psift_internal.cuh"

namespace psift {
namespace {

constexpr uint8_t kPngSig[8] = {0x89, 'P', 'N', 'G', 0x0D, 0x0A, 0x1A, 0x0A};
constexpr int kMaxPngThreads = 16;

// Adam7 passes: first column / row and steps (ISO/IEC 15948, 8.2).
constexpr int kA7X0[7] = {0, 4, 0, 2, 0, 1, 0}, kA7DX[7] = {8, 8, 4, 4, 2, 2, 1};
constexpr int kA7Y0[7] = {0, 0, 4, 0, 2, 0, 1}, kA7DY[7] = {8, 8, 8, 4, 4, 2, 2};

uint32_t be32(const uint8_t* p) {
  return ((uint32_t)p[0] << 24) | ((uint32_t)p[1] << 16) | ((uint32_t)p[2] << 8) | (uint32_t)p[3];
}

struct PngImage {
  uint32_t w = 0, h = 0;
  int depth = 0, color = 0, interlace = 0;
  int channels = 0;
  uint32_t unit = 1;               // filter unit: bytes per complete pixel, at least 1
  std::vector<uint8_t> plte;       // RGB triples
  std::vector<std::pair<const uint8_t*, size_t>> idat;
  int n_pass = 1;
  uint32_t pass_w[7] = {0}, pass_h[7] = {0};
  size_t pass_rb[7] = {0};         // bytes per row, filter byte excluded
  size_t pass_in[7] = {0};         // offset of the pass's row slots in the inflated buffer
  size_t pass_stride[7] = {0};     // bytes per row slot: filter byte at +15, the row at +16 (16-byte aligned)
  size_t pass_out[7] = {0};        // offset of the pass in the unfiltered buffer (16-byte aligned)
  size_t pass_ostride[7] = {0};    // bytes per unfiltered row: the row rounded up to 16
  size_t raw_bytes = 0, unf_bytes = 0;
};

psift_status header_error(psift_ctx* ctx, const std::string& what) {
  return set_error(ctx, PSIFT_ERR_FORMAT, "Invalid or unsupported image header: " + what);
}
psift_status payload_error(psift_ctx* ctx, const std::string& what) {
  return set_error(ctx, PSIFT_ERR_FORMAT, "Failed to decode image payload: " + what);
}

// Chunk walk, IHDR checks and the reference's size checks.  With header_only the
// walk stops after IHDR (the dimensions); otherwise PLTE and the IDAT spans are
// collected and every chunk's CRC is checked.
psift_status parse_png(psift_ctx* ctx, const uint8_t* data, size_t len, bool enforce_cap, bool header_only,
                       PngImage* P) {
  if (!data || len < 8 || std::memcmp(data, kPngSig, 8) != 0) return header_error(ctx, "not a PNG signature");
  size_t pos = 8;
  bool seen_ihdr = false, idat_done = false;
  while (pos + 12 <= len) {
    const uint32_t clen = be32(data + pos);
    const uint8_t* type = data + pos + 4;
    if (clen > len - pos - 12) return (seen_ihdr ? payload_error : header_error)(ctx, "truncated chunk");
    const uint8_t* body = data + pos + 8;
    const bool is = [&](const char* t) { return std::memcmp(type, t, 4) == 0; }("IHDR");
    if (!seen_ihdr) {
      if (!is || clen != 13) return header_error(ctx, "IHDR must be the first chunk");
      P->w = be32(body);
      P->h = be32(body + 4);
      P->depth = body[8];
      P->color = body[9];
      P->interlace = body[12];
      if (body[10] != 0 || body[11] != 0 || P->interlace > 1)
        return header_error(ctx, "unknown compression, filter or interlace method");
      const int d = P->depth;
      switch (P->color) {
        case 0: P->channels = 1; if (d != 1 && d != 2 && d != 4 && d != 8 && d != 16) P->channels = 0; break;
        case 2: P->channels = 3; if (d != 8 && d != 16) P->channels = 0; break;
        case 3: P->channels = 1; if (d != 1 && d != 2 && d != 4 && d != 8) P->channels = 0; break;
        case 4: P->channels = 2; if (d != 8 && d != 16) P->channels = 0; break;
        case 6: P->channels = 4; if (d != 8 && d != 16) P->channels = 0; break;
        default: P->channels = 0;
      }
      if (P->channels == 0) return header_error(ctx, "invalid bit depth / colour type combination");
      if (P->w == 0 || P->h == 0 || P->w > 0x7FFFFFFFu || P->h > 0x7FFFFFFFu)
        return header_error(ctx, "invalid dimensions");
      psift_status st = check_image_dims(ctx, P->w, P->h, enforce_cap);
      if (st != PSIFT_OK) return st;
      seen_ihdr = true;
      if (header_only) return PSIFT_OK;
    } else {
      const uint32_t crc = (uint32_t)crc32(crc32(0L, Z_NULL, 0), type, 4 + clen);
      if (crc != be32(body + clen)) return payload_error(ctx, "CRC error");
      if (std::memcmp(type, "IDAT", 4) == 0) {
        if (idat_done) return payload_error(ctx, "IDAT chunks are not consecutive");
        P->idat.emplace_back(body, clen);
      } else {
        if (!P->idat.empty()) idat_done = true;
        if (std::memcmp(type, "PLTE", 4) == 0) {
          if (clen % 3 != 0 || clen == 0 || clen > 768) return payload_error(ctx, "invalid PLTE chunk");
          P->plte.assign(body, body + clen);
        } else if (std::memcmp(type, "IEND", 4) == 0) {
          break;
        } else if (std::memcmp(type, "IHDR", 4) == 0) {
          return payload_error(ctx, "duplicate IHDR");
        } else if (!(type[0] & 0x20)) {
          return payload_error(ctx, "unknown critical chunk");
        }
      }
    }
    pos += 12 + (size_t)clen;
  }
  if (!seen_ihdr) return header_error(ctx, "missing IHDR");
  if (P->idat.empty()) return payload_error(ctx, "no image data");
  if (P->color == 3 && P->plte.empty()) return payload_error(ctx, "palette image without PLTE");
  // a missing IEND after complete image data is accepted
  const uint32_t bits_pp = (uint32_t)P->depth * (uint32_t)P->channels;
  P->unit = std::max(1u, bits_pp / 8);
  P->n_pass = P->interlace ? 7 : 1;
  size_t in = 0, out = 0;
  for (int p = 0; p < P->n_pass; ++p) {
    uint32_t pw = P->w, ph = P->h;
    if (P->interlace) {
      pw = P->w > (uint32_t)kA7X0[p] ? (P->w - kA7X0[p] + kA7DX[p] - 1) / kA7DX[p] : 0;
      ph = P->h > (uint32_t)kA7Y0[p] ? (P->h - kA7Y0[p] + kA7DY[p] - 1) / kA7DY[p] : 0;
    }
    P->pass_w[p] = pw;
    P->pass_h[p] = ph;
    P->pass_rb[p] = (pw == 0 || ph == 0) ? 0 : ((size_t)pw * bits_pp + 7) / 8;
    P->pass_in[p] = in;
    P->pass_out[p] = out;
    P->pass_stride[p] = align_up(P->pass_rb[p], 16) + 16;
    P->pass_ostride[p] = align_up(P->pass_rb[p], 16);
    if (P->pass_rb[p]) {
      in += (size_t)ph * P->pass_stride[p];
      out += (size_t)ph * P->pass_ostride[p];
    }
  }
  P->raw_bytes = in;
  P->unf_bytes = out;
  return PSIFT_OK;
}

// The zlib stream of the IDAT chunks into dst, each scanline (filter byte, then
// the row) into its slot: filter byte at +15, row at +16, so that every row
// starts 16-byte aligned for the device's copies.  A stream with trailing data
// past the image is accepted.  Returns an empty string or the error.
std::string inflate_png(const PngImage& P, uint8_t* dst) {
  z_stream zs;
  std::memset(&zs, 0, sizeof zs);
  if (inflateInit(&zs) != Z_OK) return "zlib initialisation failed";
  size_t chunk = 0;
  zs.next_in = const_cast<Bytef*>(P.idat[0].first);
  zs.avail_in = (uInt)P.idat[0].second;
  int r = Z_OK;
  std::string err;
  for (int p = 0; p < P.n_pass && err.empty(); ++p) {
    if (!P.pass_rb[p]) continue;
    for (uint32_t row = 0; row < P.pass_h[p] && err.empty(); ++row) {
      zs.next_out = dst + P.pass_in[p] + (size_t)row * P.pass_stride[p] + 15;
      zs.avail_out = (uInt)(1 + P.pass_rb[p]);
      while (zs.avail_out > 0) {
        if (zs.avail_in == 0) {
          if (++chunk >= P.idat.size()) break;
          zs.next_in = const_cast<Bytef*>(P.idat[chunk].first);
          zs.avail_in = (uInt)P.idat[chunk].second;
          continue;
        }
        r = inflate(&zs, Z_NO_FLUSH);
        if (r == Z_STREAM_END) break;
        if (r != Z_OK) break;
      }
      if (r != Z_OK && r != Z_STREAM_END) err = "corrupt deflate stream (zlib " + std::to_string(r) + ")";
      else if (zs.avail_out > 0) err = "image data is truncated";
    }
  }
  inflateEnd(&zs);
  return err;
}

// ------------------------------------------------------------------ kernels
struct PngPlane {
  const uint8_t* in;  // row slots: filter byte at +15 (checked on the host), the filtered row at +16
  uint8_t* out;       // rows of row_bytes at ostride
  uint32_t rows;
  uint32_t row_bytes;
  uint32_t stride;    // bytes per row slot (a multiple of 16)
  uint32_t ostride;   // bytes per unfiltered row (row_bytes rounded up to 16)
};

// Adam7 constants of pass p as nibble p of a word (device code).
__device__ __forceinline__ uint32_t a7(uint32_t packed, int p) { return (packed >> (4 * p)) & 15u; }
constexpr uint32_t kA7X0w = 0x0102040u, kA7DXw = 0x1224488u, kA7Y0w = 0x1020400u, kA7DYw = 0x2244888u;

__device__ __forceinline__ uint32_t paeth(uint32_t a, uint32_t b, uint32_t c) {
  const int p = (int)a + (int)b - (int)c;
  const int pa = abs(p - (int)a), pb = abs(p - (int)b), pc = abs(p - (int)c);
  return (pa <= pb && pa <= pc) ? a : (pb <= pc ? b : c);
}

constexpr int kRing = 512;          // bytes of a lane's row staged in shared memory (four 128-byte chunks)
constexpr int kUnfWarps = 12;       // row groups of a plane in flight at once (one warp each)
constexpr uint32_t kUnfSpin = 1u << 22;  // bounded wait on the previous group (with nanosleep)

// One CTA (kUnfWarps warps) per plane.  Rows go in groups of 32; group k is
// warp k mod kUnfWarps's, so up to kUnfWarps groups run at once, each behind the
// one above it.  Inside a group, at step s lane t reconstructs unit (pixel) s - t
// of row 32k + t: the row above at that unit is what lane t - 1 reconstructed at
// step s - 1 (a shuffle) and the unit before it lane t - 1's value one step
// earlier.  Lane 0's row above is the previous group's last row: every 32 steps
// the warp waits until that row is done up to the units of its next 32 steps
// (the previous group's lane 31 publishes its count after each 32 steps with a
// release store; lanes read it with acquire loads), then copies those units to
// shared memory.  Each lane's filtered row streams through a ring of 128-byte
// chunks in shared memory, the next chunk copied asynchronously while the
// current one is consumed (lane 31 trails lane 0 by at most 31 units = 248
// bytes, inside the ring).  Units are UNIT bytes, the filter's byte distance.
// The waits are bounded: on timeout the warp records kErrTimeout and leaves
// (the groups after it then time out too).
template <int UNIT>
__global__ void __launch_bounds__(32 * kUnfWarps) png_unfilter_kernel(const PngPlane* __restrict__ planes,
                                                                      uint32_t* err) {
  extern __shared__ __align__(16) uint8_t psm[];
  unsigned long long* progress = reinterpret_cast<unsigned long long*>(psm);         // [kUnfWarps]
  uint8_t* abuf_all = psm + 16 * kUnfWarps;                                        // [kUnfWarps][32 * 8]
  uint8_t* ring_all = abuf_all + 256 * kUnfWarps;                                  // [kUnfWarps][32][kRing]
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const PngPlane P = planes[blockIdx.x];
  const uint32_t rb = P.row_bytes, npix = rb / UNIT;
  const uint32_t rb16 = (rb + 15) & ~15u;
  const uint32_t nchunks = (rb + 127) / 128;
  uint8_t* my_ring = ring_all + ((size_t)warp * 32 + lane) * kRing;
  uint8_t* abuf = abuf_all + warp * 256;
  if (threadIdx.x < kUnfWarps) progress[threadIdx.x] = 0ull;
  __syncthreads();
  const unsigned long long span = (unsigned long long)npix + 1ull;  // progress of group k = k * span + units
  const uint32_t groups = (P.rows + 31) / 32;
  for (uint32_t k = warp; k < groups; k += kUnfWarps) {
    const uint32_t g = 32 * k;
    const uint32_t r = g + lane;
    const bool row_ok = r < P.rows;
    const uint8_t* slot = P.in + (size_t)r * P.stride;
    const uint32_t f = row_ok ? slot[15] : 0u;
    const uint8_t* src = slot + 16;
    uint8_t* dst = P.out + (size_t)r * P.ostride;
    const uint8_t* above_g = (g > 0) ? P.out + (size_t)(g - 1) * P.ostride : nullptr;  // row g - 1 (lane 0's above)
    const unsigned long long* prev = progress + (k + kUnfWarps - 1) % kUnfWarps;
    unsigned long long* mine = progress + warp;
    // chunk c of this lane's row into ring slot c % 4 (16-byte copies inside the row slot)
    auto fetch = [&](uint32_t c) {
      if (row_ok && c < nchunks)
        for (uint32_t q = 0; q < 8 && c * 128 + 16 * q < rb16; ++q)
          asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(
                           (uint32_t)__cvta_generic_to_shared(my_ring + (c & 3) * 128 + 16 * q)),
                       "l"(src + c * 128 + 16 * q)
                       : "memory");
      asm volatile("cp.async.commit_group;" ::: "memory");
    };
    // chunk c of this lane's reconstructed row (written over its filtered bytes in
    // the ring) to the output row as 16-byte stores; rows are padded to 16 bytes
    auto flush = [&](uint32_t c) {
      if (!row_ok || c >= nchunks) return;
      const uint4* from = reinterpret_cast<const uint4*>(my_ring + (c & 3) * 128);
      for (uint32_t q = 0; q < 8 && c * 128 + 16 * q < rb16; ++q)
        *reinterpret_cast<uint4*>(dst + c * 128 + 16 * q) = from[q];
    };
    fetch(0);
    fetch(1);
    asm volatile("cp.async.wait_group 1;" ::: "memory");
    __syncwarp();
    uint32_t cur = 0;
    uint8_t a[UNIT], c[UNIT], mine_prev[UNIT];  // left unit, above-left unit, this lane's last unit
#pragma unroll
    for (int q = 0; q < UNIT; ++q) a[q] = c[q] = mine_prev[q] = 0;
    const uint32_t steps = npix + 31;
    for (uint32_t s0 = 0; s0 < steps; s0 += 32) {
      // lane 0's row above, units s0 .. s0 + 31
      if (g > 0 && s0 < npix) {
        const uint32_t need = min(npix, s0 + 32);
        const unsigned long long target = (unsigned long long)(k - 1) * span + need;
        bool ok = false;
        for (uint32_t it = 0; it < kUnfSpin; ++it) {
          unsigned long long v;
          asm volatile("ld.acquire.cta.shared.u64 %0, [%1];" : "=l"(v) : "r"((uint32_t)__cvta_generic_to_shared(prev))
                       : "memory");
          if (v >= target) {
            ok = true;
            break;
          }
          __nanosleep(64);
        }
        if (!__all_sync(0xffffffffu, ok)) {
          if (lane == 0) atomicOr(err, kErrTimeout);
          asm volatile("cp.async.wait_group 0;" ::: "memory");
          return;
        }
        const uint32_t u = s0 + lane;
        if (u < npix)
#pragma unroll
          for (int q = 0; q < UNIT; ++q) abuf[lane * UNIT + q] = __ldcg(above_g + (size_t)u * UNIT + q);
        __syncwarp();
      }
      const uint32_t s1 = min(steps, s0 + 32);
      for (uint32_t s = s0; s < s1; ++s) {
        // lane 0 (the leading lane) reached a new chunk with its unit's last byte:
        // the chunk's successor is copied, the chunk itself is waited for
        const uint32_t lead = min(s, npix - 1) * UNIT + UNIT - 1;
        if ((lead >> 7) != cur) {
          cur = lead >> 7;
          // every lane is past chunk cur - 3 (lane 31 trails lane 0 by at most 248
          // bytes): it leaves the ring before chunk cur + 1 takes its slot
          if (cur >= 3) flush(cur - 3);
          fetch(cur + 1);
          asm volatile("cp.async.wait_group 1;" ::: "memory");
          __syncwarp();
        }
        // the unit lane - 1 reconstructed at step s - 1 = this lane's above unit
        uint32_t w0 = 0, w1 = 0;
#pragma unroll
        for (int q = 0; q < UNIT; ++q) {
          if (q < 4) w0 |= (uint32_t)mine_prev[q] << (8 * q);
          else w1 |= (uint32_t)mine_prev[q] << (8 * (q - 4));
        }
        w0 = __shfl_up_sync(0xffffffffu, w0, 1);
        if (UNIT > 4) w1 = __shfl_up_sync(0xffffffffu, w1, 1);
        const int i = (int)s - lane;
        const bool act = row_ok && i >= 0 && (uint32_t)i < npix;
        uint8_t bb[UNIT];
#pragma unroll
        for (int q = 0; q < UNIT; ++q) bb[q] = (uint8_t)((q < 4 ? w0 >> (8 * q) : w1 >> (8 * (q - 4))) & 0xFF);
        if (lane == 0) {
#pragma unroll
          for (int q = 0; q < UNIT; ++q) bb[q] = (act && g > 0) ? abuf[(s - s0) * UNIT + q] : 0;
        }
        if (act) {
          if (i == 0) {
#pragma unroll
            for (int q = 0; q < UNIT; ++q) a[q] = c[q] = 0;
          }
#pragma unroll
          for (int q = 0; q < UNIT; ++q) {
            const uint32_t x = my_ring[((uint32_t)i * UNIT + q) & (kRing - 1)];
            const uint32_t av = a[q], bv = r > 0 ? bb[q] : 0u, cv = r > 0 ? c[q] : 0u;
            const uint32_t pred =
                f == 1 ? av : f == 2 ? bv : f == 3 ? (av + bv) >> 1 : f == 4 ? paeth(av, bv, cv) : 0u;
            const uint8_t v = (uint8_t)(x + pred);
            my_ring[((uint32_t)i * UNIT + q) & (kRing - 1)] = v;
            // the group's last row also goes out byte by byte: the next group reads it
            // as soon as its progress is published
            if (lane == 31) dst[(size_t)i * UNIT + q] = v;
            a[q] = v;
            c[q] = (uint8_t)bv;
            mine_prev[q] = v;
          }
        }
      }
      // this group's last row (lane 31) is done up to unit s1 - 32: publish
      __syncwarp();
      if (lane == 31) {
        const uint32_t done = s1 >= 32 ? min(npix, s1 - 31) : 0u;
        const unsigned long long v = (unsigned long long)k * span + done;
        asm volatile("st.release.cta.shared.u64 [%0], %1;" ::"r"((uint32_t)__cvta_generic_to_shared(mine)), "l"(v)
                     : "memory");
      }
    }
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    __syncwarp();
    // the chunks still in the ring
    for (uint32_t c = cur >= 2 ? cur - 2 : 0; c <= cur; ++c) flush(c);
    __syncwarp();
  }
}

struct PngLumaJob {
  const uint8_t* unf;     // unfiltered passes
  uint8_t* luma;          // w x h, dense rows
  const uint8_t* plte;    // 256 RGB triples (zero past the file's palette)
  uint32_t w, h;
  uint32_t pass_rb[7];
  uint32_t pass_ostride[7];
  uint32_t pass_out[7];
  int depth, color, interlace;
};

__device__ __forceinline__ uint32_t rgb_luma(uint32_t r, uint32_t g, uint32_t b) {
  return (2126u * r + 7152u * g + 722u * b) / 10000u;
}
__device__ __forceinline__ uint32_t u16_to_u8(uint32_t v) { return (v + 128u) / 257u; }

// Thread per pixel: the pixel's pass and position, its samples, the luma.
__global__ void png_luma_kernel(const PngLumaJob* __restrict__ jobs) {
  const PngLumaJob& J = jobs[blockIdx.y];
  const uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= J.w * J.h) return;
  const uint32_t y = idx / J.w, x = idx - y * J.w;
  int p = 0;
  uint32_t px = x, py = y;
  if (J.interlace) {
    // Adam7: the pass of (x, y) follows from (x mod 8, y mod 8)
    const uint32_t xm = x & 7, ym = y & 7;
    if ((ym & 1) == 1) p = 6;
    else if ((xm & 1) == 1) p = 5;
    else if ((ym & 3) == 2) p = 4;
    else if ((xm & 3) == 2) p = 3;
    else if (ym == 4) p = 2;
    else if (xm == 4) p = 1;
    else p = 0;
    px = (x - a7(kA7X0w, p)) / a7(kA7DXw, p);
    py = (y - a7(kA7Y0w, p)) / a7(kA7DYw, p);
  }
  const uint8_t* row = J.unf + J.pass_out[p] + (size_t)py * J.pass_ostride[p];
  const int d = J.depth;
  uint32_t L;
  if (J.color == 0 || J.color == 3) {
    uint32_t v;
    if (d == 16) {
      v = ((uint32_t)row[2 * px] << 8) | row[2 * px + 1];
    } else if (d == 8) {
      v = row[px];
    } else {
      const uint32_t bit = px * (uint32_t)d;
      v = (row[bit >> 3] >> (8 - d - (bit & 7))) & ((1u << d) - 1u);
    }
    if (J.color == 3) {
      const uint8_t* c = J.plte + 3 * v;
      L = rgb_luma(c[0], c[1], c[2]);
    } else if (d == 16) {
      L = u16_to_u8(v);
    } else {
      L = v * (255u / ((1u << d) - 1u));
    }
  } else if (J.color == 4) {  // gray + alpha: the gray sample
    L = d == 16 ? u16_to_u8(((uint32_t)row[4 * px] << 8) | row[4 * px + 1]) : row[2 * px];
  } else {  // RGB / RGBA: alpha dropped
    const uint32_t ch = J.color == 6 ? 4 : 3;
    if (d == 16) {
      const uint8_t* s = row + 2 * ch * px;
      L = u16_to_u8(rgb_luma(((uint32_t)s[0] << 8) | s[1], ((uint32_t)s[2] << 8) | s[3], ((uint32_t)s[4] << 8) | s[5]));
    } else {
      const uint8_t* s = row + ch * px;
      L = rgb_luma(s[0], s[1], s[2]);
    }
  }
  J.luma[idx] = (uint8_t)L;
}

// ------------------------------------------------------------------- host
// Staging of a batch: the inflated streams in pinned memory, then on the device
// the filtered streams, the unfiltered passes, the palettes and the kernels'
// descriptors; per image fixed offsets, so chunks decoded on different streams
// never share a region.  Grow-only.
struct PngState {
  uint8_t* pinned = nullptr;
  size_t pinned_cap = 0;
  uint8_t* dev = nullptr;
  size_t dev_cap = 0;
};

PngState* png_state(psift_ctx* ctx) {
  if (!ctx->png) ctx->png = new PngState();
  return static_cast<PngState*>(ctx->png);
}

struct PngLayout {
  std::vector<size_t> pin_raw, dev_raw, dev_unf;  // per image
  size_t pin_desc = 0, dev_desc = 0;              // per image: 7 planes, 1 luma job, 768 palette bytes
  static constexpr size_t kDescBytes = 7 * sizeof(PngPlane) + sizeof(PngLumaJob) + 768;
  size_t desc_stride = 0;
};

psift_status png_reserve(psift_ctx* ctx, const std::vector<PngImage>& P, PngLayout& L) {
  PngState* S = png_state(ctx);
  const size_t n = P.size();
  L.pin_raw.resize(n);
  L.dev_raw.resize(n);
  L.dev_unf.resize(n);
  L.desc_stride = align_up(PngLayout::kDescBytes, 256);
  size_t pin = 0, dev = 0;
  for (size_t i = 0; i < n; ++i) {
    L.pin_raw[i] = pin;
    pin += align_up(P[i].raw_bytes, 256);
    L.dev_raw[i] = dev;
    dev += align_up(P[i].raw_bytes, 256);
    L.dev_unf[i] = dev;
    dev += align_up(P[i].unf_bytes, 256);
  }
  L.pin_desc = pin;
  L.dev_desc = dev;
  pin += n * L.desc_stride;
  dev += n * L.desc_stride;
  if (pin > S->pinned_cap) {
    if (S->pinned) {
      cudaError_t e = cudaStreamSynchronize(ctx->stream);  // no earlier copy still reads it
      if (e == cudaSuccess) e = cudaDeviceSynchronize();
      if (e != cudaSuccess) return cuda_error(ctx, e, "png staging");
      cudaFreeHost(S->pinned);
    }
    S->pinned = nullptr;
    S->pinned_cap = 0;
    const size_t cap = align_up(pin, 1 << 20);
    cudaError_t e = cudaHostAlloc(&S->pinned, cap, cudaHostAllocDefault);
    if (e != cudaSuccess) return cuda_error(ctx, e, "cudaHostAlloc(png staging)");
    S->pinned_cap = cap;
  }
  if (dev > S->dev_cap) {
    cudaFree(S->dev);  // synchronises the device: no earlier decode still uses it
    S->dev = nullptr;
    S->dev_cap = 0;
    const size_t cap = align_up(dev, 1 << 20);
    cudaError_t e = cudaMalloc(&S->dev, cap);
    if (e != cudaSuccess) return cuda_error(ctx, e, "cudaMalloc(png staging)");
    S->dev_cap = cap;
  }
  return PSIFT_OK;
}

// Inflates images [b, e) on host threads into their pinned regions and checks
// every row's filter type; returns the first error (image order).
psift_status inflate_range(psift_ctx* ctx, const std::vector<PngImage>& P, const PngLayout& L, uint32_t b,
                           uint32_t e) {
  PngState* S = png_state(ctx);
  const uint32_t n = e - b;
  std::vector<std::string> errs(n);
  auto work = [&](uint32_t t, uint32_t T) {
    for (uint32_t i = b + t; i < e; i += T) {
      const PngImage& I = P[i];
      uint8_t* dst = S->pinned + L.pin_raw[i];
      std::string err = inflate_png(I, dst);
      for (int p = 0; err.empty() && p < I.n_pass; ++p) {
        if (!I.pass_rb[p]) continue;
        const uint8_t* row = dst + I.pass_in[p] + 15;
        for (uint32_t r = 0; r < I.pass_h[p]; ++r, row += I.pass_stride[p])
          if (*row > 4) {
            err = "invalid filter type " + std::to_string((int)*row);
            break;
          }
      }
      errs[i - b] = err;
    }
  };
  const unsigned hc = std::max(1u, std::thread::hardware_concurrency());
  const uint32_t T = std::min<uint32_t>(n, std::min<unsigned>(hc, kMaxPngThreads));
  if (T <= 1) {
    work(0, 1);
  } else {
    std::vector<std::thread> th;
    for (uint32_t t = 1; t < T; ++t) th.emplace_back(work, t, T);
    work(0, T);
    for (auto& x : th) x.join();
  }
  for (uint32_t i = 0; i < n; ++i)
    if (!errs[i].empty()) return payload_error(ctx, errs[i]);
  return PSIFT_OK;
}

template <int UNIT>
cudaError_t launch_unfilter(const PngPlane* planes, int n, uint32_t* err, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  const size_t smem = (size_t)kUnfWarps * (16 + 256 + 32 * kRing);
  cudaError_t e = ensure_smem_attr((const void*)png_unfilter_kernel<UNIT>, smem);
  if (e != cudaSuccess) return e;
  png_unfilter_kernel<UNIT><<<n, 32 * kUnfWarps, smem, st>>>(planes, err);
  return cudaGetLastError();
}

// Decodes images [b, e) (parsed, not yet inflated) into luma[i - b] (dense rows)
// on st: inflate on host threads, the filtered streams to the device, the row
// filters undone per filter unit, then expansion and luma.
psift_status decode_png_range(psift_ctx* ctx, const std::vector<PngImage>& P, const PngLayout& L, uint32_t b,
                              uint32_t e, uint8_t* const* luma, cudaStream_t st, bool inflated = false) {
  if (!inflated) {
    psift_status rs = inflate_range(ctx, P, L, b, e);
    if (rs != PSIFT_OK) return rs;
  }
  PngState* S = png_state(ctx);
  const uint32_t n = e - b;
  // descriptors of the chunk: its slots of the per-image regions (planes of
  // images b..e-1 grouped by filter unit into slots 7b.., jobs into slots b..)
  uint8_t* pin_desc = S->pinned + L.pin_desc;
  uint8_t* dev_desc = S->dev + L.dev_desc;
  const size_t plane_base = 0, job_base = 7 * sizeof(PngPlane) * P.size(),
               plte_base = job_base + sizeof(PngLumaJob) * P.size();
  PngPlane* hp = reinterpret_cast<PngPlane*>(pin_desc + plane_base) + 7 * (size_t)b;
  PngLumaJob* hj = reinterpret_cast<PngLumaJob*>(pin_desc + job_base) + b;
  const int units[6] = {1, 2, 3, 4, 6, 8};
  int count[6] = {0, 0, 0, 0, 0, 0};
  int np = 0;
  uint32_t max_px = 0;
  for (int u = 0; u < 6; ++u) {
    for (uint32_t i = b; i < e; ++i) {
      const PngImage& I = P[i];
      if ((int)I.unit != units[u]) continue;
      for (int p = 0; p < I.n_pass; ++p) {
        if (!I.pass_rb[p]) continue;
        hp[np++] = PngPlane{S->dev + L.dev_raw[i] + I.pass_in[p], S->dev + L.dev_unf[i] + I.pass_out[p],
                            I.pass_h[p], (uint32_t)I.pass_rb[p], (uint32_t)I.pass_stride[p],
                            (uint32_t)I.pass_ostride[p]};
        ++count[u];
      }
    }
  }
  for (uint32_t i = b; i < e; ++i) {
    const PngImage& I = P[i];
    uint8_t* hplte = pin_desc + plte_base + 768 * (size_t)i;
    std::memset(hplte, 0, 768);
    if (!I.plte.empty()) std::memcpy(hplte, I.plte.data(), I.plte.size());
    PngLumaJob& J = hj[i - b];
    std::memset(&J, 0, sizeof J);
    J.unf = S->dev + L.dev_unf[i];
    J.luma = luma[i - b];
    J.plte = dev_desc + plte_base + 768 * (size_t)i;
    J.w = I.w;
    J.h = I.h;
    for (int p = 0; p < 7; ++p) {
      J.pass_rb[p] = (uint32_t)I.pass_rb[p];
      J.pass_ostride[p] = (uint32_t)I.pass_ostride[p];
      J.pass_out[p] = (uint32_t)I.pass_out[p];
    }
    J.depth = I.depth;
    J.color = I.color;
    J.interlace = I.interlace;
    max_px = std::max(max_px, I.w * I.h);
    PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(S->dev + L.dev_raw[i], S->pinned + L.pin_raw[i], I.raw_bytes,
                                        cudaMemcpyHostToDevice, st));
  }
  // the chunk's planes, jobs and palettes (three contiguous slot ranges)
  PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(dev_desc + plane_base + 7 * sizeof(PngPlane) * b, hp, sizeof(PngPlane) * np,
                                      cudaMemcpyHostToDevice, st));
  PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(dev_desc + job_base + sizeof(PngLumaJob) * b, hj, sizeof(PngLumaJob) * n,
                                      cudaMemcpyHostToDevice, st));
  PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(dev_desc + plte_base + 768 * (size_t)b, pin_desc + plte_base + 768 * (size_t)b,
                                      768 * (size_t)n, cudaMemcpyHostToDevice, st));
  const PngPlane* dp = reinterpret_cast<const PngPlane*>(dev_desc + plane_base) + 7 * (size_t)b;
  int off = 0;
  cudaError_t ce = cudaSuccess;
  for (int u = 0; u < 6 && ce == cudaSuccess; ++u) {
    if (!count[u]) continue;
    switch (units[u]) {
      case 1: ce = launch_unfilter<1>(dp + off, count[u], ctx->d_error, st); break;
      case 2: ce = launch_unfilter<2>(dp + off, count[u], ctx->d_error, st); break;
      case 3: ce = launch_unfilter<3>(dp + off, count[u], ctx->d_error, st); break;
      case 4: ce = launch_unfilter<4>(dp + off, count[u], ctx->d_error, st); break;
      case 6: ce = launch_unfilter<6>(dp + off, count[u], ctx->d_error, st); break;
      default: ce = launch_unfilter<8>(dp + off, count[u], ctx->d_error, st); break;
    }
    off += count[u];
    ctx->launches++;
  }
  if (ce == cudaSuccess) {
    dim3 grid((max_px + 255) / 256, n);
    png_luma_kernel<<<grid, 256, 0, st>>>(reinterpret_cast<const PngLumaJob*>(dev_desc + job_base) + b);
    ce = cudaGetLastError();
    ctx->launches++;
  }
  if (ce != cudaSuccess) return cuda_error(ctx, ce, "png decode");
  return PSIFT_OK;
}

bool is_png(const uint8_t* data, size_t len) { return data && len >= 8 && std::memcmp(data, kPngSig, 8) == 0; }

}  // namespace

void png_release(psift_ctx* ctx) {
  if (!ctx->png) return;
  PngState* S = static_cast<PngState*>(ctx->png);
  if (S->pinned) cudaFreeHost(S->pinned);
  cudaFree(S->dev);
  delete S;
  ctx->png = nullptr;
}

bool bytes_are_png(const uint8_t* data, size_t len) { return is_png(data, len); }

}  // namespace psift

using namespace psift;

extern "C" {

psift_status psift_png_info(psift_ctx* ctx, const uint8_t* data, size_t length, int32_t enforce_pixel_cap,
                            uint32_t* width, uint32_t* height, uint32_t* components) {
  if (!ctx || !width || !height) return PSIFT_ERR_INVALID_ARGUMENT;
  PngImage I;
  psift_status st = parse_png(ctx, data, length, enforce_pixel_cap != 0, true, &I);
  *width = I.w;
  *height = I.h;
  if (components) *components = (uint32_t)I.channels;
  return st;
}

psift_status psift_decode_png_luma(psift_ctx* ctx, const uint8_t* data, size_t length, int32_t enforce_pixel_cap,
                                   uint8_t* luma, size_t capacity, uint32_t* width, uint32_t* height) {
  if (!ctx || !width || !height) return PSIFT_ERR_INVALID_ARGUMENT;
  PSIFT_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  std::vector<PngImage> P(1);
  psift_status st = parse_png(ctx, data, length, enforce_pixel_cap != 0, false, &P[0]);
  *width = P[0].w;
  *height = P[0].h;
  if (st != PSIFT_OK) return st;
  const size_t px = (size_t)P[0].w * P[0].h;
  if (px > capacity) return set_error(ctx, PSIFT_ERR_CAPACITY, "luma output capacity too small");
  if (!luma) return set_error(ctx, PSIFT_ERR_INVALID_ARGUMENT, "null luma output");
  if ((st = io_reserve(ctx, px)) != PSIFT_OK) return st;
  PngLayout L;
  if ((st = png_reserve(ctx, P, L)) != PSIFT_OK) return st;
  uint8_t* d_luma = (uint8_t*)ctx->io.base;
  uint8_t* const outs[1] = {d_luma};
  PSIFT_CUDA_TRY(ctx, cudaMemsetAsync(ctx->d_error, 0, 4, ctx->stream));
  if ((st = decode_png_range(ctx, P, L, 0, 1, outs, ctx->stream)) != PSIFT_OK) return st;
  PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(luma, d_luma, px, cudaMemcpyDeviceToHost, ctx->stream));
  uint32_t word = 0;  // pageable: the copy completes before the synchronisation returns
  PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(&word, ctx->d_error, 4, cudaMemcpyDeviceToHost, ctx->stream));
  PSIFT_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  if (word & kErrTimeout) return set_error(ctx, PSIFT_ERR_TIMEOUT, "device wait timed out (png row filters)");
  return PSIFT_OK;
}

psift_status psift_detect_and_compute_png_batch(psift_ctx* ctx, const uint8_t* const* data, const size_t* lengths,
                                                uint32_t n, int32_t enforce_pixel_cap, const psift_sift_config* cfg,
                                                psift_features* outs) {
  if (!ctx || !data || !lengths || !outs || n == 0) return PSIFT_ERR_INVALID_ARGUMENT;
  PSIFT_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  std::vector<PngImage> P(n);
  std::vector<psift_image_u8> imgs(n);
  for (uint32_t i = 0; i < n; ++i) {
    const psift_status st = parse_png(ctx, data[i], lengths[i], enforce_pixel_cap != 0, false, &P[i]);
    if (st != PSIFT_OK) return st;
    imgs[i] = psift_image_u8{nullptr, P[i].h, P[i].w, P[i].w};
  }
  PngLayout L;
  psift_status rs = png_reserve(ctx, P, L);
  if (rs != PSIFT_OK) return rs;
  // The whole batch is inflated before chunk 0's stages, on as many host threads
  // as there are images (up to 16): with fewer images than threads, inflating per
  // chunk would leave threads idle for longer than the overlap with chunk 0's
  // kernels gains.  Each chunk's device part runs on its own stream.
  const DeviceFill fill = [&](char* extra, const std::vector<size_t>& dev_off, uint32_t b, uint32_t e,
                              cudaStream_t st) -> psift_status {
    if (b == 0) {
      psift_status rs = inflate_range(ctx, P, L, 0, n);
      if (rs != PSIFT_OK) return rs;
    }
    std::vector<uint8_t*> luma(e - b);
    for (uint32_t i = b; i < e; ++i) luma[i - b] = (uint8_t*)extra + dev_off[i];
    return decode_png_range(ctx, P, L, b, e, luma.data(), st, true);
  };
  return detect_batch_host_out(ctx, imgs.data(), n, cfg, outs, &fill);
}

psift_status psift_detect_and_compute_image_batch(psift_ctx* ctx, const uint8_t* const* data, const size_t* lengths,
                                                  uint32_t n, int32_t enforce_pixel_cap, const psift_sift_config* cfg,
                                                  psift_features* outs) {
  if (!ctx || !data || !lengths || !outs || n == 0) return PSIFT_ERR_INVALID_ARGUMENT;
  // the format from the leading bytes (the reader's guessed format): PNG
  // signature, else JPEG (whose decoder reports anything else as a bad header)
  std::vector<const uint8_t*> pd, jd;
  std::vector<size_t> pl, jl;
  std::vector<psift_features> po, jo;
  std::vector<uint32_t> pi, ji;
  for (uint32_t i = 0; i < n; ++i) {
    const bool png = is_png(data[i], lengths[i]);
    (png ? pd : jd).push_back(data[i]);
    (png ? pl : jl).push_back(lengths[i]);
    (png ? po : jo).push_back(outs[i]);
    (png ? pi : ji).push_back(i);
  }
  psift_status st = PSIFT_OK;
  if (!jd.empty())
    st = psift_detect_and_compute_jpeg_batch(ctx, jd.data(), jl.data(), (uint32_t)jd.size(), enforce_pixel_cap, cfg,
                                             jo.data());
  if (st == PSIFT_OK && !pd.empty())
    st = psift_detect_and_compute_png_batch(ctx, pd.data(), pl.data(), (uint32_t)pd.size(), enforce_pixel_cap, cfg,
                                            po.data());
  // the feature counts (or required counts) land in the callers' structs
  for (size_t k = 0; k < ji.size(); ++k) outs[ji[k]] = jo[k];
  for (size_t k = 0; k < pi.size(); ++k) outs[pi[k]] = po[k];
  return st;
}

}  // extern "C"
