// JPEG decoding for the frames of a stack: baseline sequential Huffman, 8-bit
// samples, three components (Y, Cb, Cr) at 4:4:4, 4:2:2 or 4:2:0.  The result
// is the image libjpeg gives with its default decompression settings (the
// reference decodes through libjpeg, src/image_io.zig:160-173): the "islow"
// integer inverse DCT, fancy (triangle) chroma upsampling and the fixed-point
// YCbCr -> RGB conversion.  Those are restated here from the JPEG standard
// (ITU-T T.81) and the published IJG algorithms, in integer arithmetic, so
// the output is byte-identical to libjpeg's.
//
// Work split: the host parses the markers and removes the byte stuffing
// (0xFF 0x00 -> 0xFF) while it cuts the entropy-coded data at its restart
// markers; each restart interval is then decoded by one GPU thread (the
// intervals are independent: the DC predictions restart).  A file without
// restart markers is one interval and is entropy-decoded on the host.  The
// inverse DCT, the upsampling and the colour conversion run on the GPU.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include <string>
#include <vector>

#ifdef __CUDACC__
#define JPEG_HD __host__ __device__
#else
#define JPEG_HD
#endif

namespace fs {
namespace jpeg {

constexpr int kMaxComponents = 3;

// Canonical Huffman table (T.81 Annex C / F.2.2.3): a direct lookup of every
// code up to kLookBits long, and the per-length limits for longer codes.
constexpr int kLookBits = 9;
struct Huffman {
  uint16_t look[1 << kLookBits];  // (length << 8) | symbol, 0: code longer than kLookBits
  int32_t maxcode[18];            // largest code of each length (-1: none); [17] sentinel
  int32_t valoffset[17];          // symbol index of a code of that length = code + valoffset
  uint8_t symbols[256];
};

struct Component {
  int id, h, v, tq;       // identifier, sampling factors, quantisation table
  int td, ta;             // DC / AC Huffman table of the scan
  int bw, bh;             // blocks per row / column (whole MCUs)
  int cw, ch;             // samples per row / column (ceil(W * h / hmax), ...)
};

// Everything the GPU needs, copied to the device as one block.
struct Tables {
  Huffman dc[2], ac[2];
  uint16_t quant[4][64];   // natural order
  int32_t ncomp;
  int32_t hmax, vmax, mcus_x, mcus_y;
  int32_t restart;         // MCUs per restart interval (0: one interval)
  Component comp[kMaxComponents];
};

struct Parsed {
  uint32_t width = 0, height = 0;
  Tables t;
  std::vector<uint8_t> data;         // entropy-coded bytes, stuffing removed, intervals back to back
  std::vector<uint32_t> seg_begin;   // byte offset of each restart interval in `data`
  std::vector<uint32_t> seg_end;
};

// Parse a JPEG file; false with a reason for anything outside the decoder's
// scope (progressive or arithmetic coding, 12-bit samples, other layouts).
bool parse(const uint8_t* p, size_t n, Parsed* out, std::string* why);

// Sizes of a decode: coefficients (int16, 64 per block, all components) and
// component planes (u8, whole blocks), in elements.
size_t coef_count(const Tables& t);
size_t plane_bytes(const Tables& t);
size_t coef_offset(const Tables& t, int c);   // first coefficient of component c
size_t plane_offset(const Tables& t, int c);  // first sample of component c

// Entropy decoding of one restart interval into dequantisation-ready
// coefficients (natural order); shared by the device kernel and the host path.
// Returns false on a corrupt stream.
JPEG_HD bool decode_interval(const Tables& t, const uint8_t* data, uint32_t begin, uint32_t end, int64_t first_mcu,
                             int64_t mcus, int16_t* coef);

// Device steps (d_tables: a device copy of the parsed Tables).  Entropy
// decoding of nseg restart intervals, one thread each, into d_coef (cleared
// by the caller); *d_status becomes 1 on a corrupt interval.
cudaError_t launch_entropy(const Tables* d_tables, const uint8_t* d_data, const uint32_t* d_begin,
                           const uint32_t* d_end, int nseg, int16_t* d_coef, int* d_status, cudaStream_t s);
// Inverse DCT of every block into the component planes, then upsampling and
// colour conversion into interleaved RGB u8 (w x h, row pitch in bytes).
cudaError_t launch_idct_color(const Tables* d_tables, const Tables& t, const int16_t* d_coef, uint8_t* d_planes,
                              uint32_t w, uint32_t h, uint8_t* d_dst, int64_t dst_pitch, cudaStream_t s);

}  // namespace jpeg
}  // namespace fs
