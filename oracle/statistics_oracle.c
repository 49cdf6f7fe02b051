/* Index reductions (MinIndx / MaxIndx / MinAbsIndx / MaxAbsIndx).
 *
 * TEST INFRASTRUCTURE ONLY (oracle). A C restatement of the reference's
 * algorithm, comparison for comparison:
 *   cl-files/Statistics.cl :326-500 (REDUCE_POS_STD / REDUCE_POS_FLUSH):
 *     work-groups of 16 x 16 work-items; work-item (lx, ly) of group (gx, gy)
 *     reads x = 256 gx + lx + 16 i (i = 0..15) of row 16 gy + ly and keeps
 *     the first value no later one beats strictly (in the source type, after
 *     fabs/abs for the Abs forms; OpenCL abs() of a signed value is unsigned
 *     and is stored back in the source type); then the group folds
 *     work-item lid + s into lid for s = 128, 64, ..., 1, on a strict win,
 *     between valid work-items only; the group result is stored as float.
 *   C++/programs/StatisticsHelpers.cpp :105-146 (ReduceMin / ReduceMax):
 *     the host folds the groups in group order (gid = gy * groupsX + gx),
 *     starting from group 0, strict comparison, and returns the float.
 * The reference's own Statistics.cl also holds reductions that need OpenCL
 * atomics and bit casts, which the kernel shim does not provide, so it is not
 * compiled here; parity rests on this restatement. */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "oracle.h"

enum { OP_MIN = 0, OP_MAX = 1, OP_MINABS = 2, OP_MAXABS = 3 };

#define DEFINE_REDUCE(NAME, T, ABSFN)                                                     \
  static int NAME(int op, const void* src, int step, int W, int H, double* value, int* ox,  \
                  int* oy) {                                                              \
    const int gxn = (W + 255) / 256, gyn = (H + 15) / 16;                                 \
    const int is_min = (op == OP_MIN || op == OP_MINABS);                                 \
    const int use_abs = (op == OP_MINABS || op == OP_MAXABS);                             \
    float gval = 0;                                                                       \
    int gxx = 0, gyy = 0;                                                                 \
    for (int gy = 0; gy < gyn; ++gy)                                                      \
      for (int gx = 0; gx < gxn; ++gx) {                                                  \
        T buf[256];                                                                       \
        int cx[256], cy[256], valid[256];                                                 \
        for (int ly = 0; ly < 16; ++ly)                                                   \
          for (int lx = 0; lx < 16; ++lx) {                                               \
            const int lid = ly * 16 + lx, x = gx * 256 + lx, y = gy * 16 + ly;            \
            valid[lid] = x < W && y < H;                                                  \
            if (!valid[lid]) continue;                                                    \
            const T* row = (const T*)((const char*)src + (size_t)y * step);               \
            T r = use_abs ? ABSFN(row[x]) : row[x];                                       \
            int bx = x;                                                                   \
            for (int i = 16; i < 256; i += 16)                                            \
              if (x + i < W) {                                                            \
                const T p = use_abs ? ABSFN(row[x + i]) : row[x + i];                     \
                if (is_min ? (p < r) : (p > r)) {                                         \
                  r = p;                                                                  \
                  bx = x + i;                                                             \
                }                                                                         \
              }                                                                           \
            buf[lid] = r;                                                                 \
            cx[lid] = bx;                                                                 \
            cy[lid] = y;                                                                  \
          }                                                                               \
        for (int s = 128; s >= 1; s >>= 1)                                                \
          for (int lid = 0; lid < s; ++lid)                                               \
            if (valid[lid] && valid[lid + s] &&                                           \
                (is_min ? (buf[lid + s] < buf[lid]) : (buf[lid + s] > buf[lid]))) {       \
              buf[lid] = buf[lid + s];                                                    \
              cx[lid] = cx[lid + s];                                                      \
              cy[lid] = cy[lid + s];                                                      \
            }                                                                             \
        const float v = (float)buf[0];                                                    \
        if ((gy == 0 && gx == 0) || (is_min ? (v < gval) : (v > gval))) {                 \
          gval = v;                                                                       \
          gxx = cx[0];                                                                    \
          gyy = cy[0];                                                                    \
        }                                                                                 \
      }                                                                                   \
    *value = gval;                                                                        \
    *ox = gxx;                                                                            \
    *oy = gyy;                                                                            \
    return 0;                                                                             \
  }

#define ABS_NONE(v) (v)
#define ABS_S8(v) ((int8_t)(uint8_t)((v) < 0 ? (uint8_t)(0u - (uint8_t)(v)) : (uint8_t)(v)))
#define ABS_S16(v) ((int16_t)(uint16_t)((v) < 0 ? (uint16_t)(0u - (uint16_t)(v)) : (uint16_t)(v)))
#define ABS_S32(v) ((int32_t)(uint32_t)((v) < 0 ? (uint32_t)(0u - (uint32_t)(v)) : (uint32_t)(v)))

DEFINE_REDUCE(red_u8, uint8_t, ABS_NONE)
DEFINE_REDUCE(red_s8, int8_t, ABS_S8)
DEFINE_REDUCE(red_u16, uint16_t, ABS_NONE)
DEFINE_REDUCE(red_s16, int16_t, ABS_S16)
DEFINE_REDUCE(red_u32, uint32_t, ABS_NONE)
DEFINE_REDUCE(red_s32, int32_t, ABS_S32)
DEFINE_REDUCE(red_f32, float, fabsf)
DEFINE_REDUCE(red_f64, double, fabs)

int orc_index_reduce(int op, int type, const void* src, int step, int W, int H, double* value,
                     int* x, int* y) {
  if (op < 0 || op > 3 || W <= 0 || H <= 0) return -30;
  switch (type) {
    case 0: return red_u8(op, src, step, W, H, value, x, y);
    case 1: return red_s8(op, src, step, W, H, value, x, y);
    case 2: return red_u16(op, src, step, W, H, value, x, y);
    case 3: return red_s16(op, src, step, W, H, value, x, y);
    case 4: return red_u32(op, src, step, W, H, value, x, y);
    case 5: return red_s32(op, src, step, W, H, value, x, y);
    case 6: return red_f32(op, src, step, W, H, value, x, y);
    case 7: return red_f64(op, src, step, W, H, value, x, y);
  }
  return -30;
}
