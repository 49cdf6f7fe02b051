/* CPU restatement of the reference's Integral / SqrIntegral.
 *
 * TEST INFRASTRUCTURE ONLY (see oracle.h). The reference computes an
 * inclusive 2-D prefix sum, D[y][x] = sum_{j<=y, i<=x} S[j][i] (or S^2), in
 * 64x8 tiles followed by junction passes (cl-files/Integral.cl:39-460,
 * dispatch C++/programs/Integral.cpp:97-241). The value is the same whatever
 * the tiling; this restatement computes it exactly: integer sources in
 * __int128, float sources in long double, channel by channel.
 */
#include <stdint.h>
#include <stdlib.h>

#include "oracle.h"

typedef __int128 i128;

static int type_bytes(int type) {
  static const int b[8] = {1, 1, 2, 2, 4, 4, 4, 8};
  return (type >= 0 && type < 8) ? b[type] : 0;
}

static inline long double load_ld(const void* p, int type) {
  switch (type) {
    case 0: return *(const uint8_t*)p;
    case 1: return *(const int8_t*)p;
    case 2: return *(const uint16_t*)p;
    case 3: return *(const int16_t*)p;
    case 4: return *(const uint32_t*)p;
    case 5: return *(const int32_t*)p;
    case 6: return *(const float*)p;
    default: return *(const double*)p;
  }
}

static inline i128 load_i(const void* p, int type) {
  switch (type) {
    case 0: return *(const uint8_t*)p;
    case 1: return *(const int8_t*)p;
    case 2: return *(const uint16_t*)p;
    case 3: return *(const int16_t*)p;
    case 4: return *(const uint32_t*)p;
    default: return *(const int32_t*)p;
  }
}

int orc_integral_exact(int sqr, int type, int nch, const void* src,
                       int src_step, double* dst, int W, int H) {
  if (type < 0 || type > 7) return -10;
  if (nch < 1 || nch > 4 || W <= 0 || H <= 0) return -30;
  const int eb = type_bytes(type);
  const size_t n = (size_t)W * nch;
  if (type <= 5) {
    i128* col = (i128*)calloc(n, sizeof(i128));
    if (!col) return -5;
    for (int y = 0; y < H; ++y) {
      const char* row = (const char*)src + (size_t)y * src_step;
      for (int c = 0; c < nch; ++c) {
        i128 run = 0;
        for (int x = 0; x < W; ++x) {
          const i128 v = load_i(row + ((size_t)x * nch + c) * eb, type);
          run += sqr ? v * v : v;
          col[(size_t)x * nch + c] += run;
          dst[(size_t)y * n + (size_t)x * nch + c] = (double)(long double)col[(size_t)x * nch + c];
        }
      }
    }
    free(col);
  } else {
    long double* col = (long double*)calloc(n, sizeof(long double));
    if (!col) return -5;
    for (int y = 0; y < H; ++y) {
      const char* row = (const char*)src + (size_t)y * src_step;
      for (int c = 0; c < nch; ++c) {
        long double run = 0;
        for (int x = 0; x < W; ++x) {
          const long double v = load_ld(row + ((size_t)x * nch + c) * eb, type);
          run += sqr ? v * v : v;
          col[(size_t)x * nch + c] += run;
          dst[(size_t)y * n + (size_t)x * nch + c] = (double)col[(size_t)x * nch + c];
        }
      }
    }
    free(col);
  }
  return 0;
}
