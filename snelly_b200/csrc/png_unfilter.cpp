// png_unfilter.cpp - undoes the PNG scanline filters (ISO/IEC 15948, section 9: None, Sub, Up,
// Average, Paeth) of decompressed 8-bit image data, for the environment maps and SDF-PNG assets
// the host loads (snelly_b200/image.py inflates, this reconstructs the bytes).
#include <cstdint>
#include <cstdlib>

#include "snelly.h"

extern "C" int snelly_png_unfilter(const uint8_t* raw, size_t raw_bytes, int width, int height, int channels,
                                   uint8_t* out) {
  if (!raw || !out || width < 1 || height < 1 || channels < 1 || channels > 4) return SNELLY_EINVAL;
  const size_t stride = (size_t)width * channels;
  if (raw_bytes < (stride + 1) * (size_t)height) return SNELLY_EINVAL;
  for (int y = 0; y < height; ++y) {
    const uint8_t* line = raw + (size_t)y * (stride + 1);
    const uint8_t f = line[0];
    ++line;
    uint8_t* cur = out + (size_t)y * stride;
    const uint8_t* prev = y > 0 ? out + (size_t)(y - 1) * stride : nullptr;
    for (size_t i = 0; i < stride; ++i) {
      const int a = i >= (size_t)channels ? cur[i - channels] : 0;  // left
      const int b = prev ? prev[i] : 0;                              // up
      const int c = (prev && i >= (size_t)channels) ? prev[i - channels] : 0;  // up-left
      int pred;
      switch (f) {
        case 0: pred = 0; break;
        case 1: pred = a; break;
        case 2: pred = b; break;
        case 3: pred = (a + b) >> 1; break;
        case 4: {
          const int p = a + b - c, pa = std::abs(p - a), pb = std::abs(p - b), pc = std::abs(p - c);
          pred = (pa <= pb && pa <= pc) ? a : (pb <= pc ? b : c);
          break;
        }
        default: return SNELLY_EINVAL;
      }
      cur[i] = (uint8_t)(line[i] + pred);
    }
  }
  return SNELLY_OK;
}
