// PNG output of a rendered image (Renderer::render_to_file,
// src/renderer.rs:914-920, writes the RgbImage with the `image` crate's PNG
// encoder): 8-bit RGB, non-interlaced.  Decoded pixels are what matters;
// the file bytes depend on the encoder.
//
// Encoded on host threads:
//   * each row gets the PNG filter (none, sub, up, average, Paeth) with the
//     smallest sum of absolute filtered bytes (the usual adaptive choice);
//   * the filtered rows are cut into bands, each deflated on its own thread;
//     every band but the last ends with a sync flush (byte-aligned, an
//     empty stored block), so the bands concatenate into one deflate stream;
//   * the zlib Adler-32 and the chunk CRC-32 are combined from per-band
//     values.
#include <zlib.h>

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "../../include/rtrace_gpu.h"

namespace {

inline int paeth(int a, int b, int c) {
  const int p = a + b - c;
  const int pa = std::abs(p - a), pb = std::abs(p - b), pc = std::abs(p - c);
  if (pa <= pb && pa <= pc) return a;
  return pb <= pc ? b : c;
}

// Filters row y (3 bytes per pixel) into out (1 + 3w bytes: filter type,
// data); cand: 15w bytes of scratch.  Each filter is its own loop.
void filter_row(const uint8_t* img, uint32_t w, uint32_t y, uint8_t* out, std::vector<uint8_t>& cand) {
  const size_t n = 3 * (size_t)w;
  const uint8_t* cur = img + y * n;
  cand.resize(5 * n);
  uint8_t* none = &cand[0];
  uint8_t* sub = &cand[n];
  uint8_t* upf = &cand[2 * n];
  uint8_t* avg = &cand[3 * n];
  uint8_t* pth = &cand[4 * n];
  static thread_local std::vector<uint8_t> zrow;  // the row above the first
  if (!y && zrow.size() < n) zrow.assign(n, 0);
  const uint8_t* up = y ? cur - n : zrow.data();
  memcpy(none, cur, n);
  for (size_t i = 0; i < 3 && i < n; i++) {
    sub[i] = cur[i];
    upf[i] = (uint8_t)(cur[i] - up[i]);
    avg[i] = (uint8_t)(cur[i] - (up[i] >> 1));
    pth[i] = (uint8_t)(cur[i] - up[i]);  // Paeth with a = c = 0 predicts b
  }
  for (size_t i = 3; i < n; i++) sub[i] = (uint8_t)(cur[i] - cur[i - 3]);
  for (size_t i = 3; i < n; i++) upf[i] = (uint8_t)(cur[i] - up[i]);
  for (size_t i = 3; i < n; i++) avg[i] = (uint8_t)(cur[i] - ((cur[i - 3] + up[i]) >> 1));
  for (size_t i = 3; i < n; i++) pth[i] = (uint8_t)(cur[i] - paeth(cur[i - 3], up[i], up[i - 3]));
  uint64_t best_sum = UINT64_MAX;
  int best = 0;
  for (int f = 0; f < 5; f++) {
    const uint8_t* c = &cand[f * n];
    uint64_t sum = 0;
    for (size_t i = 0; i < n; i++) sum += c[i] < 128 ? c[i] : 256 - c[i];
    if (sum < best_sum) {
      best_sum = sum;
      best = f;
    }
  }
  out[0] = (uint8_t)best;
  memcpy(out + 1, &cand[best * n], n);
}

void put_u32(std::string& s, uint32_t v) {
  const char b[4] = {(char)(v >> 24), (char)(v >> 16), (char)(v >> 8), (char)v};
  s.append(b, 4);
}

void chunk(std::string& png, const char* type, const std::string& data, uLong crc_of_data_part, bool have_crc) {
  put_u32(png, (uint32_t)data.size());
  png.append(type, 4);
  png.append(data);
  uLong crc = crc32(0L, reinterpret_cast<const Bytef*>(type), 4);
  if (have_crc)
    crc = crc32_combine(crc, crc_of_data_part, (z_off_t)data.size());
  else
    crc = crc32(crc, reinterpret_cast<const Bytef*>(data.data()), (uInt)data.size());
  put_u32(png, (uint32_t)crc);
}

struct Band {
  size_t first, rows;
  std::string out;
  uLong adler = 1, crc = 0;
  int err = Z_OK;
};

}  // namespace

// Encodes an 8-bit RGB image as PNG into *out (malloc'ed; rt_png_free).
// level: zlib level 0-9 (-1: default).  Threads: all host threads.
extern "C" rt_status rt_png_encode(const uint8_t* rgb, uint32_t width, uint32_t height, int32_t level, uint8_t** out,
                                   size_t* out_len) {
  if (!rgb || !out || !out_len || width == 0 || height == 0) return RT_ERR_INVALID_ARGUMENT;
  if (level < -1 || level > 9) return RT_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  *out_len = 0;
  const size_t row = 1 + 3 * (size_t)width;
  std::vector<uint8_t> filt(row * height);
  const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
  const size_t nb = std::max<size_t>(1, std::min<size_t>(4 * (size_t)hw, (row * height) / (256 * 1024) + 1));
  std::vector<Band> bands(std::min<size_t>(nb, height));
  for (size_t b = 0; b < bands.size(); b++) {
    bands[b].first = height * b / bands.size();
    bands[b].rows = height * (b + 1) / bands.size() - bands[b].first;
  }
  auto work = [&](size_t b) {
    Band& B = bands[b];
    std::vector<uint8_t> cand;
    for (size_t y = B.first; y < B.first + B.rows; y++) filter_row(rgb, width, (uint32_t)y, &filt[y * row], cand);
    const Bytef* src = &filt[B.first * row];
    const size_t len = B.rows * row;
    B.adler = adler32(1L, src, (uInt)len);
    z_stream z{};
    if ((B.err = deflateInit2(&z, level, Z_DEFLATED, -15, 8, Z_DEFAULT_STRATEGY)) != Z_OK) return;
    B.out.resize(deflateBound(&z, (uLong)len) + 16);
    z.next_in = const_cast<Bytef*>(src);
    z.avail_in = (uInt)len;
    z.next_out = reinterpret_cast<Bytef*>(&B.out[0]);
    z.avail_out = (uInt)B.out.size();
    const bool last = b + 1 == bands.size();
    int r = deflate(&z, last ? Z_FINISH : Z_SYNC_FLUSH);
    if (r != (last ? Z_STREAM_END : Z_OK) || z.avail_in != 0) B.err = Z_BUF_ERROR;
    B.out.resize(B.out.size() - z.avail_out);
    deflateEnd(&z);
    B.crc = crc32(0L, reinterpret_cast<const Bytef*>(B.out.data()), (uInt)B.out.size());
  };
  {
    const size_t nthreads = std::min<size_t>(hw, bands.size());
    std::vector<std::thread> th;
    for (size_t t = 1; t < nthreads; t++)
      th.emplace_back([&, t] {
        for (size_t b = t; b < bands.size(); b += nthreads) work(b);
      });
    for (size_t b = 0; b < bands.size(); b += nthreads) work(b);
    for (auto& t : th) t.join();
  }
  for (const Band& B : bands)
    if (B.err != Z_OK) return RT_ERR_INVALID_ARGUMENT;
  // zlib stream: header (deflate, 32 KB window, check bits), the bands,
  // Adler-32 of the filtered rows
  uLong adler = bands[0].adler;
  for (size_t b = 1; b < bands.size(); b++)
    adler = adler32_combine(adler, bands[b].adler, (z_off_t)(bands[b].rows * row));
  std::string idat;
  size_t total = 6;
  for (const Band& B : bands) total += B.out.size();
  idat.reserve(total);
  idat.push_back((char)0x78);
  idat.push_back((char)0x9C);
  uLong crc_data = crc32(0L, reinterpret_cast<const Bytef*>(idat.data()), 2);
  for (const Band& B : bands) {
    idat.append(B.out);
    crc_data = crc32_combine(crc_data, B.crc, (z_off_t)B.out.size());
  }
  std::string tail;
  put_u32(tail, (uint32_t)adler);
  idat.append(tail);
  crc_data = crc32(crc_data, reinterpret_cast<const Bytef*>(tail.data()), 4);

  std::string png("\x89PNG\r\n\x1a\n", 8);
  std::string ihdr;
  put_u32(ihdr, width);
  put_u32(ihdr, height);
  ihdr.append("\x08\x02\x00\x00\x00", 5);  // 8 bits, RGB, deflate, adaptive filters, no interlace
  chunk(png, "IHDR", ihdr, 0, false);
  chunk(png, "IDAT", idat, crc_data, true);
  chunk(png, "IEND", std::string(), 0, false);
  uint8_t* buf = static_cast<uint8_t*>(malloc(png.size()));
  if (!buf) return RT_ERR_OUT_OF_MEMORY;
  memcpy(buf, png.data(), png.size());
  *out = buf;
  *out_len = png.size();
  return RT_OK;
}

extern "C" void rt_png_free(uint8_t* p) { free(p); }

// Renderer::render_to_file's write: the image as a PNG file at path, at
// zlib level 1 (about twice as fast as the default level for a few percent
// more bytes on rendered frames).
extern "C" rt_status rt_png_write(const char* path, const uint8_t* rgb, uint32_t width, uint32_t height) {
  if (!path) return RT_ERR_INVALID_ARGUMENT;
  uint8_t* buf = nullptr;
  size_t len = 0;
  rt_status st = rt_png_encode(rgb, width, height, 1, &buf, &len);
  if (st != RT_OK) return st;
  FILE* f = fopen(path, "wb");
  if (!f) {
    free(buf);
    return RT_ERR_IO;
  }
  const bool ok = fwrite(buf, 1, len, f) == len;
  free(buf);
  if (fclose(f) != 0 || !ok) return RT_ERR_IO;
  return RT_OK;
}
