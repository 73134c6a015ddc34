// JPEG decoding (see jpeg.h): marker parsing and restart-interval cutting on
// the host, entropy decoding per restart interval, the "islow" inverse DCT,
// fancy upsampling and YCbCr -> RGB on the GPU.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>

#include "jpeg.h"

namespace fs {
namespace jpeg {

// ----------------------------------------------------------------- parsing
namespace {

// Zigzag position -> natural (row-major) index (T.81 Figure A.6).
const uint8_t kNatural[64] = {0,  1,  8,  16, 9,  2,  3,  10, 17, 24, 32, 25, 18, 11, 4,  5,
                              12, 19, 26, 33, 40, 48, 41, 34, 27, 20, 13, 6,  7,  14, 21, 28,
                              35, 42, 49, 56, 57, 50, 43, 36, 29, 22, 15, 23, 30, 37, 44, 51,
                              58, 59, 52, 45, 38, 31, 39, 46, 53, 60, 61, 54, 47, 55, 62, 63};

// T.81 Annex C: code sizes and codes of a table given BITS and HUFFVAL.
bool build_huffman(const uint8_t bits[17], const uint8_t* vals, int nvals, Huffman* h) {
  std::memset(h, 0, sizeof(*h));
  std::memcpy(h->symbols, vals, (size_t)nvals);
  int code = 0, k = 0;
  for (int len = 1; len <= 16; ++len) {
    h->valoffset[len] = k - code;
    for (int i = 0; i < bits[len]; ++i, ++k, ++code) {
      if (code >= (1 << len)) return false;  // over-subscribed table
      if (len <= kLookBits) {
        const int shift = kLookBits - len;
        for (int f = 0; f < (1 << shift); ++f) h->look[(code << shift) | f] = (uint16_t)((len << 8) | vals[k]);
      }
    }
    h->maxcode[len] = bits[len] ? code - 1 : -1;
    code <<= 1;
  }
  h->maxcode[17] = 0x7fffffff;
  return k == nvals;
}

uint16_t be16(const uint8_t* p) { return (uint16_t)((p[0] << 8) | p[1]); }

}  // namespace

bool parse(const uint8_t* p, size_t n, Parsed* out, std::string* why) {
  auto fail = [&](const char* w) {
    *why = w;
    return false;
  };
  if (n < 4 || p[0] != 0xFF || p[1] != 0xD8) return fail("not a JPEG file (no SOI marker)");
  Tables& t = out->t;
  std::memset(&t, 0, sizeof(t));
  bool have_sof = false, have_huff[2][2] = {{false, false}, {false, false}};
  size_t i = 2;
  while (i + 4 <= n) {
    if (p[i] != 0xFF) return fail("marker expected");
    const uint8_t m = p[i + 1];
    if (m == 0xFF) {  // fill byte
      ++i;
      continue;
    }
    if (m == 0xD8 || (m >= 0xD0 && m <= 0xD7) || m == 0x01) {
      i += 2;
      continue;
    }
    if (m == 0xD9) break;
    const size_t len = be16(p + i + 2);
    if (len < 2 || i + 2 + len > n) return fail("truncated marker segment");
    const uint8_t* s = p + i + 4;
    const size_t sl = len - 2;
    if (m == 0xC0 || m == 0xC1) {  // baseline / extended sequential, Huffman
      if (sl < 6 || s[0] != 8) return fail("only 8-bit samples are decoded");
      out->height = be16(s + 1);
      out->width = be16(s + 3);
      t.ncomp = s[5];
      if (t.ncomp != 3) return fail("only three-component (YCbCr) JPEGs are decoded");
      if (sl < 6 + 3 * (size_t)t.ncomp || out->width == 0 || out->height == 0) return fail("bad frame header");
      for (int c = 0; c < t.ncomp; ++c) {
        t.comp[c].id = s[6 + 3 * c];
        t.comp[c].h = s[7 + 3 * c] >> 4;
        t.comp[c].v = s[7 + 3 * c] & 15;
        t.comp[c].tq = s[8 + 3 * c] & 3;
        t.hmax = std::max(t.hmax, t.comp[c].h);
        t.vmax = std::max(t.vmax, t.comp[c].v);
      }
      // the upsampler handles chroma at full, half-horizontal or half-both
      // resolution with a full-resolution luma
      if (t.comp[0].h != t.hmax || t.comp[0].v != t.vmax || t.hmax > 2 || t.vmax > 2 || t.comp[1].h != 1 ||
          t.comp[1].v != 1 || t.comp[2].h != 1 || t.comp[2].v != 1 || (t.vmax == 2 && t.hmax != 2))
        return fail("chroma subsampling other than 4:4:4, 4:2:2 or 4:2:0");
      t.mcus_x = (int)((out->width + 8 * t.hmax - 1) / (8 * t.hmax));
      t.mcus_y = (int)((out->height + 8 * t.vmax - 1) / (8 * t.vmax));
      for (int c = 0; c < t.ncomp; ++c) {
        Component& cc = t.comp[c];
        cc.bw = t.mcus_x * cc.h;
        cc.bh = t.mcus_y * cc.v;
        cc.cw = (int)((out->width * (uint32_t)cc.h + t.hmax - 1) / t.hmax);
        cc.ch = (int)((out->height * (uint32_t)cc.v + t.vmax - 1) / t.vmax);
      }
      have_sof = true;
    } else if (m >= 0xC2 && m <= 0xCF && m != 0xC4 && m != 0xC8 && m != 0xCC) {
      return fail("progressive, lossless or arithmetic-coded JPEG");
    } else if (m == 0xDB) {  // DQT
      size_t k = 0;
      while (k < sl) {
        const int pq = s[k] >> 4, tq = s[k] & 15;
        if (tq > 3 || k + 1 + 64 * (pq + 1) > sl) return fail("bad quantisation table");
        for (int z = 0; z < 64; ++z)
          t.quant[tq][kNatural[z]] = pq ? be16(s + k + 1 + 2 * z) : s[k + 1 + z];
        k += 1 + 64 * (pq + 1);
      }
    } else if (m == 0xC4) {  // DHT
      size_t k = 0;
      while (k < sl) {
        if (k + 17 > sl) return fail("bad Huffman table");
        const int tc = s[k] >> 4, th = s[k] & 15;
        if (tc > 1 || th > 1) return fail("Huffman table class / id out of range");
        uint8_t bits[17] = {0};
        int nv = 0;
        for (int l = 1; l <= 16; ++l) nv += bits[l] = s[k + l];
        if (nv > 256 || k + 17 + nv > sl) return fail("bad Huffman table");
        if (!build_huffman(bits, s + k + 17, nv, tc ? &t.ac[th] : &t.dc[th])) return fail("bad Huffman table");
        have_huff[tc][th] = true;
        k += 17 + nv;
      }
    } else if (m == 0xDD) {  // DRI
      if (sl < 2) return fail("bad restart interval");
      t.restart = be16(s);
    } else if (m == 0xDA) {  // SOS
      if (!have_sof) return fail("scan before the frame header");
      const int ns = s[0];
      if (ns != t.ncomp || sl < 1 + 2 * (size_t)ns + 3) return fail("only single-scan interleaved JPEGs are decoded");
      for (int q = 0; q < ns; ++q) {
        const int id = s[1 + 2 * q];
        int c = 0;
        while (c < t.ncomp && t.comp[c].id != id) ++c;
        if (c != q) return fail("scan components out of frame order");
        t.comp[c].td = s[2 + 2 * q] >> 4;
        t.comp[c].ta = s[2 + 2 * q] & 15;
        if (t.comp[c].td > 1 || t.comp[c].ta > 1 || !have_huff[0][t.comp[c].td] || !have_huff[1][t.comp[c].ta])
          return fail("scan refers to a missing Huffman table");
      }
      // entropy-coded data: unstuff, cut at restart markers
      size_t j = i + 2 + len;
      out->data.clear();
      out->data.reserve(n - j);
      out->seg_begin.assign(1, 0);
      out->seg_end.clear();
      while (j < n) {
        const uint8_t b = p[j];
        if (b != 0xFF) {
          out->data.push_back(b);
          ++j;
          continue;
        }
        if (j + 1 >= n) break;
        const uint8_t b2 = p[j + 1];
        if (b2 == 0x00) {
          out->data.push_back(0xFF);
          j += 2;
        } else if (b2 >= 0xD0 && b2 <= 0xD7) {
          out->seg_end.push_back((uint32_t)out->data.size());
          out->seg_begin.push_back((uint32_t)out->data.size());
          j += 2;
        } else if (b2 == 0xFF) {
          ++j;  // fill byte
        } else {
          break;  // EOI or another marker ends the scan
        }
      }
      out->seg_end.push_back((uint32_t)out->data.size());
      const int64_t mcus = (int64_t)t.mcus_x * t.mcus_y;
      const int64_t per = t.restart > 0 ? t.restart : mcus;
      if ((int64_t)out->seg_begin.size() != (mcus + per - 1) / per)
        return fail("restart markers do not match the restart interval");
      if (out->data.size() > 0xFFFFFFF0u) return fail("entropy-coded data too large");
      return true;
    }
    i += 2 + len;
  }
  return fail("no scan in the file");
}

size_t coef_count(const Tables& t) {
  size_t n = 0;
  for (int c = 0; c < t.ncomp; ++c) n += (size_t)t.comp[c].bw * t.comp[c].bh * 64;
  return n;
}
size_t coef_offset(const Tables& t, int c) {
  size_t n = 0;
  for (int q = 0; q < c; ++q) n += (size_t)t.comp[q].bw * t.comp[q].bh * 64;
  return n;
}
size_t plane_bytes(const Tables& t) { return coef_count(t); }
size_t plane_offset(const Tables& t, int c) { return coef_offset(t, c); }

// ------------------------------------------------------- entropy decoding
namespace {

struct BitReader {
  const uint8_t* p;
  uint32_t pos, end;
  uint64_t acc;
  int nbits;
  JPEG_HD void fill() {
    while (nbits <= 56) {
      if (pos < end) {
        acc |= (uint64_t)p[pos++] << (56 - nbits);
        nbits += 8;
      } else {  // past the interval: zeros, as libjpeg feeds after a marker
        nbits = 64;
      }
    }
  }
  JPEG_HD uint32_t peek16() {
    if (nbits < 16) fill();
    return (uint32_t)(acc >> 48);
  }
  JPEG_HD void skip(int n) {
    acc <<= n;
    nbits -= n;
  }
  JPEG_HD uint32_t bits(int n) {  // n in 0..16
    if (n == 0) return 0;
    if (nbits < n) fill();
    const uint32_t v = (uint32_t)(acc >> (64 - n));
    skip(n);
    return v;
  }
};

// T.81 F.2.2.3 DECODE: -1 on an invalid code.
JPEG_HD int decode_symbol(const Huffman& h, BitReader& br) {
  const uint32_t peek = br.peek16();
  const uint16_t look = h.look[peek >> (16 - kLookBits)];
  if (look) {
    br.skip(look >> 8);
    return look & 255;
  }
  for (int len = kLookBits + 1; len <= 16; ++len) {
    const int32_t code = (int32_t)(peek >> (16 - len));
    if (code <= h.maxcode[len]) {
      br.skip(len);
      const int idx = code + h.valoffset[len];
      return (idx >= 0 && idx < 256) ? h.symbols[idx] : -1;
    }
  }
  return -1;
}

// T.81 F.2.2.1 EXTEND
JPEG_HD int extend(uint32_t v, int s) { return (s && v < (1u << (s - 1))) ? (int)v - (1 << s) + 1 : (int)v; }

JPEG_HD const uint8_t* natural_order() {
#ifdef __CUDA_ARCH__
  __constant__ static const uint8_t k[64] = {0,  1,  8,  16, 9,  2,  3,  10, 17, 24, 32, 25, 18, 11, 4,  5,
                                            12, 19, 26, 33, 40, 48, 41, 34, 27, 20, 13, 6,  7,  14, 21, 28,
                                            35, 42, 49, 56, 57, 50, 43, 36, 29, 22, 15, 23, 30, 37, 44, 51,
                                            58, 59, 52, 45, 38, 31, 39, 46, 53, 60, 61, 54, 47, 55, 62, 63};
  return k;
#else
  return kNatural;
#endif
}

}  // namespace

JPEG_HD bool decode_interval(const Tables& t, const uint8_t* data, uint32_t begin, uint32_t end, int64_t first_mcu,
                             int64_t mcus, int16_t* coef) {
  BitReader br{data, begin, end, 0ull, 0};
  int pred[kMaxComponents] = {0, 0, 0};
  const uint8_t* nat = natural_order();
  size_t base[kMaxComponents];
  for (int c = 0, acc = 0; c < t.ncomp; ++c) {
    base[c] = (size_t)acc;
    acc += t.comp[c].bw * t.comp[c].bh * 64;
  }
  for (int64_t m = first_mcu; m < first_mcu + mcus; ++m) {
    const int mx = (int)(m % t.mcus_x), my = (int)(m / t.mcus_x);
    for (int c = 0; c < t.ncomp; ++c) {
      const Component& cc = t.comp[c];
      for (int v = 0; v < cc.v; ++v) {
        for (int h = 0; h < cc.h; ++h) {
          int16_t* blk = coef + base[c] + ((size_t)(my * cc.v + v) * cc.bw + (size_t)(mx * cc.h + h)) * 64;
          // DC
          const int s = decode_symbol(t.dc[cc.td], br);
          if (s < 0 || s > 11) return false;
          pred[c] += extend(br.bits(s), s);
          blk[0] = (int16_t)pred[c];
          // AC
          for (int k = 1; k < 64;) {
            const int rs = decode_symbol(t.ac[cc.ta], br);
            if (rs < 0) return false;
            const int r = rs >> 4, sz = rs & 15;
            if (sz == 0) {
              if (r != 15) break;  // EOB
              k += 16;
              continue;
            }
            k += r;
            if (k > 63) return false;
            blk[nat[k]] = (int16_t)extend(br.bits(sz), sz);
            ++k;
          }
        }
      }
    }
  }
  return true;
}

// ---------------------------------------------------------------- kernels
namespace {

__global__ void entropy_kernel(const Tables* tables, const uint8_t* data, const uint32_t* seg_begin,
                               const uint32_t* seg_end, int nseg, int16_t* coef, int* status) {
  __shared__ Tables t;
  for (int i = threadIdx.x; i < (int)(sizeof(Tables) / 4); i += blockDim.x)
    reinterpret_cast<uint32_t*>(&t)[i] = reinterpret_cast<const uint32_t*>(tables)[i];
  __syncthreads();
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nseg) return;
  const int64_t mcus = (int64_t)t.mcus_x * t.mcus_y;
  const int64_t per = t.restart > 0 ? t.restart : mcus;
  const int64_t first = (int64_t)s * per;
  const int64_t count = first + per <= mcus ? per : mcus - first;
  if (!decode_interval(t, data, seg_begin[s], seg_end[s], first, count, coef)) atomicExch(status, 1);
}

// islow inverse DCT: the Loeffler-Ligtenberg-Moschytz factorisation in
// 13-bit fixed point, columns first with 2 extra bits kept, rows second
// (the IJG integer algorithm).  The constants are the LLM rotation
// coefficients scaled by 2^13 and rounded.
constexpr int kConstBits = 13, kPass1Bits = 2;
constexpr int32_t fix13(double x) { return (int32_t)(x * 8192.0 + 0.5); }
constexpr int32_t F0298 = fix13(0.298631336), F0390 = fix13(0.390180644), F0541 = fix13(0.541196100),
                  F0765 = fix13(0.765366865), F0899 = fix13(0.899976223), F1175 = fix13(1.175875602),
                  F1501 = fix13(1.501321110), F1847 = fix13(1.847759065), F1961 = fix13(1.961570560),
                  F2053 = fix13(2.053119869), F2562 = fix13(2.562915447), F3072 = fix13(3.072711026);

__device__ __forceinline__ int32_t descale(int32_t x, int n) { return (x + (1 << (n - 1))) >> n; }

// One 8-point inverse transform of in[0..7] (stride 1) into out[0..7].
template <int SHIFT, bool FROM_WS>
__device__ __forceinline__ void idct8(const int32_t* in, int32_t* out) {
  // even part
  int32_t z2 = in[2], z3 = in[6];
  int32_t z1 = (z2 + z3) * F0541;
  int32_t tmp2 = z1 + z3 * (-F1847);
  int32_t tmp3 = z1 + z2 * F0765;
  z2 = in[0];
  z3 = in[4];
  int32_t tmp0 = (z2 + z3) * (1 << kConstBits);
  int32_t tmp1 = (z2 - z3) * (1 << kConstBits);
  const int32_t tmp10 = tmp0 + tmp3, tmp13 = tmp0 - tmp3, tmp11 = tmp1 + tmp2, tmp12 = tmp1 - tmp2;
  // odd part
  tmp0 = in[7];
  tmp1 = in[5];
  tmp2 = in[3];
  tmp3 = in[1];
  z1 = tmp0 + tmp3;
  z2 = tmp1 + tmp2;
  z3 = tmp0 + tmp2;
  int32_t z4 = tmp1 + tmp3;
  const int32_t z5 = (z3 + z4) * F1175;
  tmp0 *= F0298;
  tmp1 *= F2053;
  tmp2 *= F3072;
  tmp3 *= F1501;
  z1 *= -F0899;
  z2 *= -F2562;
  z3 *= -F1961;
  z4 *= -F0390;
  z3 += z5;
  z4 += z5;
  tmp0 += z1 + z3;
  tmp1 += z2 + z4;
  tmp2 += z2 + z3;
  tmp3 += z1 + z4;
  out[0] = descale(tmp10 + tmp3, SHIFT);
  out[7] = descale(tmp10 - tmp3, SHIFT);
  out[1] = descale(tmp11 + tmp2, SHIFT);
  out[6] = descale(tmp11 - tmp2, SHIFT);
  out[2] = descale(tmp12 + tmp1, SHIFT);
  out[5] = descale(tmp12 - tmp1, SHIFT);
  out[3] = descale(tmp13 + tmp0, SHIFT);
  out[4] = descale(tmp13 - tmp0, SHIFT);
}

// Post-IDCT range limit: clamp(v + 128, 0, 255) on the 10-bit wrapped value
// (libjpeg's masked table lookup).
__device__ __forceinline__ uint8_t range_limit(int32_t v) {
  const int i = v & 1023;
  if (i < 128) return (uint8_t)(128 + i);
  if (i < 512) return 255;
  if (i < 896) return 0;
  return (uint8_t)(i - 896);
}

// One block per thread: dequantise, columns, rows, range limit.
__global__ void idct_kernel(const Tables* tables, const int16_t* coef, uint8_t* planes, int64_t nblocks) {
  const int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nblocks) return;
  const Tables& t = *tables;
  int c = 0;
  int64_t first = 0;
  while (c + 1 < t.ncomp && b >= first + (int64_t)t.comp[c].bw * t.comp[c].bh) {
    first += (int64_t)t.comp[c].bw * t.comp[c].bh;
    ++c;
  }
  const Component& cc = t.comp[c];
  const uint16_t* q = t.quant[cc.tq];
  const int16_t* in = coef + b * 64;
  int32_t ws[64];
  for (int col = 0; col < 8; ++col) {
    int32_t v[8], o[8];
#pragma unroll
    for (int r = 0; r < 8; ++r) v[r] = (int32_t)in[r * 8 + col] * (int32_t)q[r * 8 + col];
    idct8<kConstBits - kPass1Bits, false>(v, o);
#pragma unroll
    for (int r = 0; r < 8; ++r) ws[r * 8 + col] = o[r];
  }
  const int64_t lb = b - first;
  const int bx = (int)(lb % cc.bw), by = (int)(lb / cc.bw);
  uint8_t* out = planes + first * 64 + (int64_t)(by * 8) * (cc.bw * 8) + bx * 8;
  for (int r = 0; r < 8; ++r) {
    int32_t o[8];
    idct8<kConstBits + kPass1Bits + 3, true>(ws + r * 8, o);
    uint32_t lo = 0, hi = 0;
#pragma unroll
    for (int x = 0; x < 4; ++x) {
      lo |= (uint32_t)range_limit(o[x]) << (8 * x);
      hi |= (uint32_t)range_limit(o[x + 4]) << (8 * x);
    }
    *reinterpret_cast<uint2*>(out + (int64_t)r * (cc.bw * 8)) = make_uint2(lo, hi);
  }
}

__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }
__device__ __forceinline__ uint8_t clamp255(int v) { return (uint8_t)clampi(v, 0, 255); }

// Chroma sample of output pixel (x, y) with fancy upsampling: the IJG
// triangle filter (3/4 nearer + 1/4 farther sample in each upsampled
// direction, alternating rounding biases), edge rows and columns replicated.
__device__ __forceinline__ int chroma_at(const uint8_t* p, int stride, const Component& c, int hmax, int vmax, int x,
                                         int y) {
  if (hmax == 1) return p[(int64_t)y * stride + x];
  const int cx = x >> 1;
  if (vmax == 1) {  // h2v1
    const uint8_t* row = p + (int64_t)y * stride;
    const int v = row[cx];
    if ((x & 1) == 0) return cx == 0 ? v : (v * 3 + row[cx - 1] + 1) >> 2;
    return cx == c.cw - 1 ? v : (v * 3 + row[cx + 1] + 2) >> 2;
  }
  // h2v2: column sums of the nearer row (x3) and the farther row
  const int cy = y >> 1;
  const int far = (y & 1) == 0 ? clampi(cy - 1, 0, c.ch - 1) : clampi(cy + 1, 0, c.ch - 1);
  const uint8_t* r0 = p + (int64_t)cy * stride;
  const uint8_t* r1 = p + (int64_t)far * stride;
  const int cur = r0[cx] * 3 + r1[cx];
  if ((x & 1) == 0) {
    if (cx == 0) return (cur * 4 + 8) >> 4;
    return (cur * 3 + (r0[cx - 1] * 3 + r1[cx - 1]) + 8) >> 4;
  }
  if (cx == c.cw - 1) return (cur * 4 + 7) >> 4;
  return (cur * 3 + (r0[cx + 1] * 3 + r1[cx + 1]) + 7) >> 4;
}

// YCbCr -> RGB in 16-bit fixed point (the JFIF equations as libjpeg's
// colour converter tabulates them).
constexpr int32_t fix16(double x) { return (int32_t)(x * 65536.0 + 0.5); }

__global__ void color_kernel(const Tables* tables, const uint8_t* planes, int w, int h, uint8_t* dst,
                             int64_t dst_pitch) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (int64_t)w * h) return;
  const Tables& t = *tables;
  const int x = (int)(i % w), y = (int)(i / w);
  const uint8_t* yp = planes;
  const int ys = t.comp[0].bw * 8;
  const uint8_t* cbp = planes + (int64_t)t.comp[0].bw * t.comp[0].bh * 64;
  const uint8_t* crp = cbp + (int64_t)t.comp[1].bw * t.comp[1].bh * 64;
  const int cs = t.comp[1].bw * 8;
  const int yy = yp[(int64_t)y * ys + x];
  const int cb = chroma_at(cbp, cs, t.comp[1], t.hmax, t.vmax, x, y) - 128;
  const int cr = chroma_at(crp, cs, t.comp[2], t.hmax, t.vmax, x, y) - 128;
  const int r = yy + ((fix16(1.40200) * cr + (1 << 15)) >> 16);
  const int g = yy + ((-fix16(0.34414) * cb + (1 << 15) - fix16(0.71414) * cr) >> 16);
  const int b = yy + ((fix16(1.77200) * cb + (1 << 15)) >> 16);
  uint8_t* o = dst + (int64_t)y * dst_pitch + (int64_t)x * 3;
  o[0] = clamp255(r);
  o[1] = clamp255(g);
  o[2] = clamp255(b);
}

}  // namespace

cudaError_t launch_entropy(const Tables* d_tables, const uint8_t* d_data, const uint32_t* d_begin,
                           const uint32_t* d_end, int nseg, int16_t* d_coef, int* d_status, cudaStream_t s) {
  entropy_kernel<<<(nseg + 63) / 64, 64, 0, s>>>(d_tables, d_data, d_begin, d_end, nseg, d_coef, d_status);
  return cudaGetLastError();
}

cudaError_t launch_idct_color(const Tables* d_tables, const Tables& t, const int16_t* d_coef, uint8_t* d_planes,
                              uint32_t w, uint32_t h, uint8_t* d_dst, int64_t dst_pitch, cudaStream_t s) {
  const int64_t nblocks = (int64_t)coef_count(t) / 64;
  idct_kernel<<<(unsigned)((nblocks + 127) / 128), 128, 0, s>>>(d_tables, d_coef, d_planes, nblocks);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  const int64_t n = (int64_t)w * h;
  color_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(d_tables, d_planes, (int)w, (int)h, d_dst, dst_pitch);
  return cudaGetLastError();
}

}  // namespace jpeg
}  // namespace fs
