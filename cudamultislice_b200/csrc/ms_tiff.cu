// ms_tiff.cu -- float32 TIFF output (replaces the GUI's LibTiff.NET export,
// CUDA Simulation GUI/MainWindow.xaml.cs:684-890): one uncompressed strip,
// 32-bit IEEE float samples (SampleFormat 3), one sample per pixel,
// MinIsBlack, top-left orientation, little-endian -- the fields the GUI sets.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

#include "ms_tiff.h"

namespace ms {

namespace {
void put16(std::vector<uint8_t>& b, size_t at, uint16_t v) {
  b[at] = (uint8_t)(v & 0xff);
  b[at + 1] = (uint8_t)(v >> 8);
}
void put32(std::vector<uint8_t>& b, size_t at, uint32_t v) {
  for (int i = 0; i < 4; ++i) b[at + i] = (uint8_t)(v >> (8 * i));
}
}  // namespace

int write_tiff_f32(const char* path, const float* data, int nx, int ny) {
  if (!path || !data || nx < 1 || ny < 1) return 1;
  struct Tag {
    uint16_t id, type;
    uint32_t value;
  };
  const uint32_t bytes = (uint32_t)nx * (uint32_t)ny * 4u;
  const int ntags = 13;
  const uint32_t ifd = 8, data_at = (uint32_t)((ifd + 2 + 12 * ntags + 4 + 15) / 16 * 16);
  // SHORT = 3, LONG = 4; tags in ascending order
  const Tag tags[ntags] = {{256, 4, (uint32_t)nx}, {257, 4, (uint32_t)ny}, {258, 3, 32}, {259, 3, 1},
                           {262, 3, 1},            {266, 3, 1},            {273, 4, data_at}, {274, 3, 1},
                           {277, 3, 1},            {278, 4, (uint32_t)ny}, {279, 4, bytes}, {284, 3, 1},
                           {339, 3, 3}};
  std::vector<uint8_t> head(data_at, 0);
  head[0] = 'I';
  head[1] = 'I';
  put16(head, 2, 42);
  put32(head, 4, ifd);
  put16(head, ifd, ntags);
  for (int i = 0; i < ntags; ++i) {
    const size_t at = ifd + 2 + 12 * (size_t)i;
    put16(head, at, tags[i].id);
    put16(head, at + 2, tags[i].type);
    put32(head, at + 4, 1);
    if (tags[i].type == 3)
      put16(head, at + 8, (uint16_t)tags[i].value);
    else
      put32(head, at + 8, tags[i].value);
  }
  put32(head, ifd + 2 + 12 * ntags, 0);  // no further IFD
  FILE* f = std::fopen(path, "wb");
  if (!f) return 2;
  bool ok = std::fwrite(head.data(), 1, head.size(), f) == head.size();
  // samples little-endian, rows top to bottom
  std::vector<uint8_t> row((size_t)nx * 4);
  for (int y = 0; y < ny && ok; ++y) {
    for (int x = 0; x < nx; ++x) {
      uint32_t u;
      std::memcpy(&u, data + (size_t)y * nx + x, 4);
      for (int k = 0; k < 4; ++k) row[(size_t)x * 4 + k] = (uint8_t)(u >> (8 * k));
    }
    ok = std::fwrite(row.data(), 1, row.size(), f) == row.size();
  }
  ok = (std::fclose(f) == 0) && ok;
  return ok ? 0 : 2;
}

}  // namespace ms
