// Host writers for exported images: the files stbi_write_png, stbi_write_tga
// (Src/image.cpp:222-243, 370-390) and tinyexr's SaveEXRImageToFile
// (:245-296, 299-356) produce in the reference, pixel for pixel and of the
// same kinds.  PNG as 8-bit RGB: each row takes the filter whose output has the
// smallest sum of absolute (signed) bytes, as stb_image_write chooses, and the
// rows are deflated by zlib (level 0: stored blocks); TGA as run-length-coded
// 24-bit BGR with a bottom-left origin, stb's default; EXR as a single-part
// scanline file without compression, one scanline per block, HALF channels
// converted as tinyexr converts FLOAT pixels when HALF is requested.
#include <zlib.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "fk_internal.h"

namespace {

bool ends_with(const std::string& s, const char* tail) {
  const size_t n = std::strlen(tail);
  return s.size() >= n && s.compare(s.size() - n, n, tail) == 0;
}

// CRC-32 (ISO 3309, reflected polynomial 0xEDB88320) by slicing-by-8: eight
// table lookups per 8 input bytes (Kounavis and Berry, 2008).
struct Crc32 {
  uint32_t t[8][256];
  Crc32() {
    for (uint32_t i = 0; i < 256; ++i) {
      uint32_t c = i;
      for (int k = 0; k < 8; ++k) c = (c & 1) ? 0xEDB88320u ^ (c >> 1) : c >> 1;
      t[0][i] = c;
    }
    for (int k = 1; k < 8; ++k)
      for (uint32_t i = 0; i < 256; ++i) t[k][i] = (t[k - 1][i] >> 8) ^ t[0][t[k - 1][i] & 0xFF];
  }
  uint32_t update(uint32_t crc, const uint8_t* p, size_t n) const {  // crc: running value, not inverted
    for (; n >= 8; p += 8, n -= 8) {
      uint32_t a, b;
      std::memcpy(&a, p, 4);  // little-endian host
      std::memcpy(&b, p + 4, 4);
      a ^= crc;
      crc = t[7][a & 0xFF] ^ t[6][(a >> 8) & 0xFF] ^ t[5][(a >> 16) & 0xFF] ^ t[4][a >> 24] ^ t[3][b & 0xFF] ^
            t[2][(b >> 8) & 0xFF] ^ t[1][(b >> 16) & 0xFF] ^ t[0][b >> 24];
    }
    for (; n; --n, ++p) crc = t[0][(crc ^ *p) & 0xFF] ^ (crc >> 8);
    return crc;
  }
};

uint32_t crc32(const uint8_t* p, size_t n) {
  static const Crc32 table;
  return ~table.update(0xFFFFFFFFu, p, n);
}

// Adler-32 (RFC 1950) with the modulo deferred over runs of 5552 bytes, the
// longest run whose sums cannot overflow 32 bits.
uint32_t adler32(const uint8_t* p, size_t n) {
  uint32_t a = 1, b = 0;
  while (n) {
    size_t run = n < 5552 ? n : 5552;
    n -= run;
    for (; run; --run) {
      a += *p++;
      b += a;
    }
    a %= 65521;
    b %= 65521;
  }
  return (b << 16) | a;
}

void put_be32(std::vector<uint8_t>& o, uint32_t v) {
  o.push_back((uint8_t)(v >> 24));
  o.push_back((uint8_t)(v >> 16));
  o.push_back((uint8_t)(v >> 8));
  o.push_back((uint8_t)v);
}
void put_le(std::vector<uint8_t>& o, uint64_t v, int bytes) {
  for (int k = 0; k < bytes; ++k) o.push_back((uint8_t)(v >> (8 * k)));
}

void png_chunk(std::vector<uint8_t>& o, const char* type, const std::vector<uint8_t>& body) {
  put_be32(o, (uint32_t)body.size());
  const size_t start = o.size();
  o.insert(o.end(), type, type + 4);
  o.insert(o.end(), body.begin(), body.end());
  put_be32(o, crc32(o.data() + start, body.size() + 4));
}

bool write_file(const char* path, const std::vector<uint8_t>& bytes) {
  FILE* f = std::fopen(path, "wb");
  if (!f) return false;
  const bool ok = std::fwrite(bytes.data(), 1, bytes.size(), f) == bytes.size();
  return std::fclose(f) == 0 && ok;
}

// PNG filter types 0-4 (PNG specification, section 9) of one row into
// out[0..row); prev is the row above (zeros for the first row).
void png_filter(int type, const uint8_t* cur, const uint8_t* prev, size_t row, uint8_t* out) {
  for (size_t i = 0; i < row; ++i) {
    const int a = i >= 3 ? cur[i - 3] : 0, b = prev[i], c = i >= 3 ? prev[i - 3] : 0;
    int pred = 0;
    switch (type) {
      case 1: pred = a; break;
      case 2: pred = b; break;
      case 3: pred = (a + b) >> 1; break;
      case 4: {
        const int p = a + b - c, pa = std::abs(p - a), pb = std::abs(p - b), pc = std::abs(p - c);
        pred = (pa <= pb && pa <= pc) ? a : (pb <= pc ? b : c);
      } break;
      default: break;
    }
    out[i] = (uint8_t)(cur[i] - pred);
  }
}

// Rows [y0, y1) of the filtered image: per row the filter byte and the row
// under the filter with the smallest sum of |(int8) byte|.
void png_rows(const uint8_t* rgb, size_t row, uint32_t y0, uint32_t y1, uint8_t* raw) {
  std::vector<uint8_t> zero(row, 0), trial(row), best(row);
  for (uint32_t y = y0; y < y1; ++y) {
    const uint8_t* cur = rgb + (size_t)y * row;
    const uint8_t* prev = y ? cur - row : zero.data();
    uint64_t best_sum = ~0ull;
    int best_type = 0;
    for (int t = 0; t < 5; ++t) {
      png_filter(t, cur, prev, row, trial.data());
      uint64_t sum = 0;
      for (size_t i = 0; i < row; ++i) sum += (uint64_t)std::abs((int)(int8_t)trial[i]);
      if (sum < best_sum) {
        best_sum = sum;
        best_type = t;
        best.swap(trial);
      }
    }
    uint8_t* dst = raw + (size_t)y * (row + 1);
    dst[0] = (uint8_t)best_type;
    std::memcpy(dst + 1, best.data(), row);
  }
}

// Raw deflate of one band (at most 1 GiB), ended by a sync flush (the band's
// output ends on a byte boundary, so bands concatenate) or, for the last
// band, by the final block.  One deflate call: the output has deflateBound
// bytes and more.  False on a zlib error.
bool deflate_band(const uint8_t* in, size_t n, int level, bool last, std::vector<uint8_t>& out) {
  z_stream zs;
  std::memset(&zs, 0, sizeof(zs));
  if (deflateInit2(&zs, level, Z_DEFLATED, -15, 8, Z_DEFAULT_STRATEGY) != Z_OK) return false;
  out.resize(deflateBound(&zs, (uLong)n) + 64);
  zs.next_in = const_cast<Bytef*>(in);
  zs.avail_in = (uInt)n;
  zs.next_out = out.data();
  zs.avail_out = (uInt)out.size();
  const int rc = deflate(&zs, last ? Z_FINISH : Z_SYNC_FLUSH);
  const bool ok = zs.avail_in == 0 && (last ? rc == Z_STREAM_END : (rc == Z_OK && zs.avail_out > 0));
  out.resize(zs.total_out);
  deflateEnd(&zs);
  return ok;
}

int write_png(const char* path, uint32_t w, uint32_t h, const uint8_t* rgb, int level) {
  const size_t row = 3 * (size_t)w, raw_size = (size_t)h * (row + 1);
  std::vector<uint8_t> raw(raw_size);
  std::vector<uint8_t> z = {0x78, 0x01};  // zlib header: deflate, 32 KB window, no preset dictionary
  if (level <= 0) {
    for (uint32_t y = 0; y < h; ++y) {
      raw[(size_t)y * (row + 1)] = 0;  // filter: none
      std::memcpy(&raw[(size_t)y * (row + 1) + 1], rgb + (size_t)y * row, row);
    }
    z.reserve(2 + raw.size() + 5 * (raw.size() / 65535 + 1) + 4);
    size_t pos = 0;
    do {
      const size_t n = std::min<size_t>(65535, raw.size() - pos);
      z.push_back(pos + n == raw.size() ? 1 : 0);  // stored block, final flag
      put_le(z, n, 2);
      put_le(z, (uint16_t)~n, 2);
      z.insert(z.end(), raw.begin() + pos, raw.begin() + pos + n);
      pos += n;
    } while (pos < raw.size());
  } else {
    // filtered rows and their deflate in bands of rows, one thread each for
    // large images; each band starts a fresh window (a little less ratio)
    level = std::min(level, 9);
    const size_t min_band = (size_t)2 << 20;
    size_t bands = std::max<size_t>(1, std::min<size_t>(std::thread::hardware_concurrency(), 32));
    bands = std::max<size_t>(1, std::min<size_t>(bands, raw_size / min_band));
    bands = std::max<size_t>(bands, (raw_size >> 30) + 1);  // no band above 1 GiB
    bands = std::min<size_t>(bands, h ? h : 1);
    std::vector<uint32_t> y(bands + 1);
    for (size_t k = 0; k <= bands; ++k) y[k] = (uint32_t)((uint64_t)h * k / bands);
    std::vector<std::vector<uint8_t>> part(bands);
    std::vector<char> ok(bands, 0);
    auto work = [&](size_t k) {
      try {
        png_rows(rgb, row, y[k], y[k + 1], raw.data());
        const size_t b0 = (size_t)y[k] * (row + 1), b1 = (size_t)y[k + 1] * (row + 1);
        ok[k] = deflate_band(raw.data() + b0, b1 - b0, level, k + 1 == bands, part[k]);
      } catch (const std::bad_alloc&) {
        ok[k] = 0;
      }
    };
    std::vector<std::thread> pool;
    size_t started = 0;
    try {
      for (; bands > 1 && started < bands; ++started) pool.emplace_back(work, started);
    } catch (const std::exception&) {  // no more threads: the rest on this one
    }
    for (size_t k = started; k < bands; ++k) work(k);
    for (auto& t : pool) t.join();
    size_t total = 2 + 4;
    for (size_t k = 0; k < bands; ++k) {
      if (!ok[k]) return FK_ERR_NOMEM;
      total += part[k].size();
    }
    z[1] = 0x9C;  // zlib header: default compression level hint
    z.reserve(total);
    for (const auto& p : part) z.insert(z.end(), p.begin(), p.end());
  }
  put_be32(z, adler32(raw.data(), raw.size()));  // of the uncompressed data
  std::vector<uint8_t> o = {0x89, 'P', 'N', 'G', '\r', '\n', 0x1a, '\n'};
  std::vector<uint8_t> ihdr;
  put_be32(ihdr, w);
  put_be32(ihdr, h);
  ihdr.insert(ihdr.end(), {8, 2, 0, 0, 0});  // 8-bit RGB, deflate, filter method 0, no interlace
  png_chunk(o, "IHDR", ihdr);
  // the zlib stream over IDAT chunks of at most 1 GiB (a chunk's length is
  // limited to 2^31 - 1 bytes; decoders join consecutive IDAT chunks)
  const size_t kIdat = (size_t)1 << 30;
  for (size_t at = 0; at < z.size(); at += kIdat) {
    const size_t n = std::min(kIdat, z.size() - at);
    put_be32(o, (uint32_t)n);
    const size_t start = o.size();
    o.insert(o.end(), {'I', 'D', 'A', 'T'});
    o.insert(o.end(), z.begin() + at, z.begin() + at + n);
    put_be32(o, crc32(o.data() + start, n + 4));
  }
  png_chunk(o, "IEND", {});
  return write_file(path, o) ? FK_OK : FK_ERR_INVALID;
}

int write_tga(const char* path, uint32_t w, uint32_t h, const uint8_t* rgb) {
  if (w > 65535 || h > 65535) return FK_ERR_INVALID;
  std::vector<uint8_t> o(18, 0);
  o[2] = 10;  // run-length-coded true colour
  o[12] = (uint8_t)w;
  o[13] = (uint8_t)(w >> 8);
  o[14] = (uint8_t)h;
  o[15] = (uint8_t)(h >> 8);
  o[16] = 24;
  o[17] = 0;  // bottom-left origin: the last buffer row is stored first
  o.reserve(18 + 3 * (size_t)w * h + (size_t)h * (w / 128 + 1));
  auto same = [](const uint8_t* a, const uint8_t* b) { return a[0] == b[0] && a[1] == b[1] && a[2] == b[2]; };
  auto put_bgr = [&](const uint8_t* p) {
    o.push_back(p[2]);
    o.push_back(p[1]);
    o.push_back(p[0]);
  };
  for (uint32_t r = h; r-- > 0;) {  // packets stay within a row
    const uint8_t* px = rgb + 3 * (size_t)r * w;
    uint32_t x = 0;
    while (x < w) {
      uint32_t run = 1;
      while (x + run < w && run < 128 && same(px + 3 * (x + run), px + 3 * x)) ++run;
      if (run > 1) {  // run packet: one pixel, repeated
        o.push_back((uint8_t)(0x80 | (run - 1)));
        put_bgr(px + 3 * x);
        x += run;
        continue;
      }
      uint32_t n = 1;  // raw packet: up to the next pair of equal pixels
      while (x + n < w && n < 128 && !(x + n + 1 < w && same(px + 3 * (x + n), px + 3 * (x + n + 1)))) ++n;
      o.push_back((uint8_t)(n - 1));
      for (uint32_t i = 0; i < n; ++i) put_bgr(px + 3 * (x + i));
      x += n;
    }
  }
  return write_file(path, o) ? FK_OK : FK_ERR_INVALID;
}

// FLOAT to HALF as tinyexr converts pixels for a HALF channel: the mantissa
// truncated and rounded up in magnitude when the first dropped bit is set,
// float denormals to zero, NaN to a quiet NaN, overflow to infinity.
uint16_t half_of(float f) {
  uint32_t u;
  std::memcpy(&u, &f, 4);
  const uint32_t sign = (u >> 16) & 0x8000u, m = u & 0x7FFFFFu;
  const int e = (int)((u >> 23) & 0xFF);
  if (e == 0) return (uint16_t)sign;
  if (e == 255) return (uint16_t)(sign | 0x7C00u | (m ? 0x200u : 0u));
  const int ne = e - 127 + 15;
  if (ne >= 31) return (uint16_t)(sign | 0x7C00u);
  if (ne <= 0) {
    if (14 - ne > 24) return (uint16_t)sign;
    const uint32_t mant = m | 0x800000u;
    uint32_t hm = mant >> (14 - ne);
    if ((mant >> (13 - ne)) & 1u) ++hm;
    return (uint16_t)(sign | hm);
  }
  uint32_t hv = ((uint32_t)ne << 10) | (m >> 13);
  if (m & 0x1000u) ++hv;
  return (uint16_t)(sign | hv);
}

void attr(std::vector<uint8_t>& o, const char* name, const char* type, const std::vector<uint8_t>& v) {
  o.insert(o.end(), name, name + std::strlen(name) + 1);
  o.insert(o.end(), type, type + std::strlen(type) + 1);
  put_le(o, v.size(), 4);
  o.insert(o.end(), v.begin(), v.end());
}

int write_exr(const char* path, uint32_t w, uint32_t h, uint32_t nplanes, const float* planes) {
  if (nplanes != 1 && nplanes != 3) return FK_ERR_INVALID;
  static const char* names[3] = {"B", "G", "R"};  // plane order = the header's (sorted) channel order
  std::vector<uint8_t> o = {0x76, 0x2f, 0x31, 0x01, 2, 0, 0, 0};
  std::vector<uint8_t> ch;
  for (uint32_t c = 0; c < nplanes; ++c) {
    ch.insert(ch.end(), names[c], names[c] + 2);
    put_le(ch, 1, 4);                   // HALF
    ch.insert(ch.end(), {0, 0, 0, 0});  // pLinear, reserved
    put_le(ch, 1, 4);                   // x sampling
    put_le(ch, 1, 4);                   // y sampling
  }
  ch.push_back(0);
  attr(o, "channels", "chlist", ch);
  attr(o, "compression", "compression", {0});
  std::vector<uint8_t> box;
  put_le(box, 0, 4);
  put_le(box, 0, 4);
  put_le(box, w - 1, 4);
  put_le(box, h - 1, 4);
  attr(o, "dataWindow", "box2i", box);
  attr(o, "displayWindow", "box2i", box);
  attr(o, "lineOrder", "lineOrder", {0});
  const float one = 1.0f, zero = 0.0f;
  std::vector<uint8_t> f1(4), v2(8, 0);
  std::memcpy(f1.data(), &one, 4);
  std::memcpy(v2.data(), &zero, 4);
  std::memcpy(v2.data() + 4, &zero, 4);
  attr(o, "pixelAspectRatio", "float", f1);
  attr(o, "screenWindowCenter", "v2f", v2);
  attr(o, "screenWindowWidth", "float", f1);
  o.push_back(0);
  const size_t table = o.size(), block = 8 + (size_t)nplanes * w * 2;
  for (uint32_t y = 0; y < h; ++y) put_le(o, table + 8 * (size_t)h + y * block, 8);
  size_t at = o.size();
  o.resize(at + (size_t)h * block);
  for (uint32_t y = 0; y < h; ++y) {
    const uint32_t head[2] = {y, (uint32_t)(nplanes * w * 2)};  // little-endian host
    std::memcpy(&o[at], head, 8);
    at += 8;
    for (uint32_t c = 0; c < nplanes; ++c) {
      const float* src = planes + ((size_t)c * h + y) * w;
      for (uint32_t x = 0; x < w; ++x, at += 2) {
        const uint16_t v = half_of(src[x]);
        std::memcpy(&o[at], &v, 2);
      }
    }
  }
  return write_file(path, o) ? FK_OK : FK_ERR_INVALID;
}

}  // namespace

extern "C" {

int fk_image_write_rgb8(const char* path, uint32_t w, uint32_t h, const uint8_t* rgb) {
  if (!path || !rgb || w == 0 || h == 0) return FK_ERR_INVALID;
  const std::string p(path);
  if (ends_with(p, ".png")) return write_png(path, w, h, rgb, 6);
  if (ends_with(p, ".tga")) return write_tga(path, w, h, rgb);
  return FK_ERR_INVALID;
}

int fk_image_write_png(const char* path, uint32_t w, uint32_t h, const uint8_t* rgb, int level) {
  if (!path || !rgb || w == 0 || h == 0 || level < 0 || level > 9) return FK_ERR_INVALID;
  return write_png(path, w, h, rgb, level);
}

int fk_image_write_exr(const char* path, uint32_t w, uint32_t h, uint32_t planes, const float* data) {
  if (!path || !data || w == 0 || h == 0 || !ends_with(path, ".exr")) return FK_ERR_INVALID;
  return write_exr(path, w, h, planes, data);
}

}  // extern "C"
