/* CPU restatement of the reference's ImageProximity measures.
 *
 * TEST INFRASTRUCTURE ONLY (see oracle.h). Every function here follows
 * cl-files/ImageProximity.cl (the five measures, lines 44-466) and the
 * argument semantics of C++/programs/ImageProximity.cpp:34-163:
 *   - output is the same size as the source ("same" geometry);
 *   - the window of output (x, y) starts at (x - tw/2, y - th/2)
 *     (ImageProximity.cl:52-53, C integer division);
 *   - pixels outside the source read as 0 (ImageProximity.cl:64-67);
 *   - the _Norm measures divide by sqrt(sum S^2 * sum T^2) over the window,
 *     raw energies without mean removal (ImageProximity.cl:155, :409).
 * The reference arithmetic comes in two forms: each operation rounded on its
 * own (an OpenCL compiler that does not contract), or every `acc += a * b`
 * contracted to fma(a, b, acc) (what GPU OpenCL compilers do by default;
 * OpenCL C allows it). Both forms are pinned against the reference kernel
 * source built without and with FP contraction.
 */
#include <math.h>
#include <stdint.h>
#include <string.h>

#include "oracle.h"

typedef __int128 i128;

static int type_bytes(int type) {
  static const int b[8] = {1, 1, 2, 2, 4, 4, 4, 8};
  return (type >= 0 && type < 8) ? b[type] : 0;
}

/* Element c of pixel (x, y). */
static inline const void* pix(const void* base, int step, int type, int nch,
                              int x, int y, int c) {
  return (const char*)base + (size_t)y * step +
         ((size_t)x * nch + c) * type_bytes(type);
}

static inline double load_d(const void* p, int type) {
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

/* convert_float(value): the reference's CONVERT_REAL for non-F64 programs
 * (cl-files/Buffers.h:86), a round-to-nearest conversion. */
static inline float load_f(const void* p, int type) {
  switch (type) {
    case 0: return (float)*(const uint8_t*)p;
    case 1: return (float)*(const int8_t*)p;
    case 2: return (float)*(const uint16_t*)p;
    case 3: return (float)*(const int16_t*)p;
    case 4: return (float)*(const uint32_t*)p;
    case 5: return (float)*(const int32_t*)p;
    case 6: return *(const float*)p;
    default: return (float)*(const double*)p;
  }
}

static inline int64_t load_i(const void* p, int type) {
  switch (type) {
    case 0: return *(const uint8_t*)p;
    case 1: return *(const int8_t*)p;
    case 2: return *(const uint16_t*)p;
    case 3: return *(const int16_t*)p;
    case 4: return *(const uint32_t*)p;
    default: return *(const int32_t*)p;
  }
}

static int check_args(int measure, int type, int nch, int W, int H, int tw,
                      int th) {
  if (measure < 0 || measure > 4) return -30;
  if (type < 0 || type > 7) return -10;
  if (nch < 1 || nch > 4) return -10;
  if (W <= 0 || H <= 0 || tw <= 0 || th <= 0) return -30;
  return 0;
}

/* Single precision body: REAL = float (ImageProximity.cl with any type other
 * than F64). The accumulation order is h outer, w inner, one rounding per
 * operation. */
static void ref_f32(int measure, int type, int nch, const void* src, int ss,
                    const void* tmpl, int ts, void* dst, int ds, int W, int H,
                    int tw, int th, int r0, int r1, int fused) {
  const int left = -tw / 2, top = -th / 2;
#pragma omp parallel for schedule(dynamic, 4)
  for (int gy = r0; gy < r1; ++gy) {
    float* out = (float*)((char*)dst + (size_t)gy * ds);
    for (int gx = 0; gx < W; ++gx) {
      for (int c = 0; c < nch; ++c) {
        float sum = 0.f, sumSS = 0.f, sumTT = 0.f;
        for (int h = 0; h < th; ++h) {
          for (int w = 0; w < tw; ++w) {
            const int px = gx + w + left, py = gy + h + top;
            const float t = load_f(pix(tmpl, ts, type, nch, w, h, c), type);
            float s = 0.f;
            if (!(px < 0 || py < 0 || px >= W || py >= H))
              s = load_f(pix(src, ss, type, nch, px, py, c), type);
            if (fused) {
              const float d = s - t;
              switch (measure) {
                case 0: sum = fmaf(d, d, sum); break;
                case 1:
                  sum = fmaf(d, d, sum);
                  sumSS = fmaf(s, s, sumSS);
                  sumTT = fmaf(t, t, sumTT);
                  break;
                case 2: sum += fabsf(d); break;
                case 3: sum = fmaf(s, t, sum); break;
                default:
                  sum = fmaf(s, t, sum);
                  sumSS = fmaf(s, s, sumSS);
                  sumTT = fmaf(t, t, sumTT);
                  break;
              }
              continue;
            }
            switch (measure) {
              case 0: sum += (s - t) * (s - t); break;
              case 1:
                sum += (s - t) * (s - t);
                sumSS += s * s;
                sumTT += t * t;
                break;
              case 2: sum += fabsf(s - t); break;
              case 3: sum += s * t; break;
              default:
                sum += s * t;
                sumSS += s * s;
                sumTT += t * t;
                break;
            }
          }
        }
        if (measure == 1 || measure == 4) sum = sum / sqrtf(sumSS * sumTT);
        out[(size_t)gx * nch + c] = sum;
      }
    }
  }
}

/* Double precision body: REAL = double (F64 sources, Buffers.h:57-64). */
static void ref_f64(int measure, int nch, const void* src, int ss,
                    const void* tmpl, int ts, void* dst, int ds, int W, int H,
                    int tw, int th, int r0, int r1, int fused) {
  const int left = -tw / 2, top = -th / 2;
#pragma omp parallel for schedule(dynamic, 4)
  for (int gy = r0; gy < r1; ++gy) {
    double* out = (double*)((char*)dst + (size_t)gy * ds);
    for (int gx = 0; gx < W; ++gx) {
      for (int c = 0; c < nch; ++c) {
        double sum = 0., sumSS = 0., sumTT = 0.;
        for (int h = 0; h < th; ++h) {
          for (int w = 0; w < tw; ++w) {
            const int px = gx + w + left, py = gy + h + top;
            const double t = load_d(pix(tmpl, ts, 7, nch, w, h, c), 7);
            double s = 0.;
            if (!(px < 0 || py < 0 || px >= W || py >= H))
              s = load_d(pix(src, ss, 7, nch, px, py, c), 7);
            if (fused) {
              const double d = s - t;
              switch (measure) {
                case 0: sum = fma(d, d, sum); break;
                case 1:
                  sum = fma(d, d, sum);
                  sumSS = fma(s, s, sumSS);
                  sumTT = fma(t, t, sumTT);
                  break;
                case 2: sum += fabs(d); break;
                case 3: sum = fma(s, t, sum); break;
                default:
                  sum = fma(s, t, sum);
                  sumSS = fma(s, s, sumSS);
                  sumTT = fma(t, t, sumTT);
                  break;
              }
              continue;
            }
            switch (measure) {
              case 0: sum += (s - t) * (s - t); break;
              case 1:
                sum += (s - t) * (s - t);
                sumSS += s * s;
                sumTT += t * t;
                break;
              case 2: sum += fabs(s - t); break;
              case 3: sum += s * t; break;
              default:
                sum += s * t;
                sumSS += s * s;
                sumTT += t * t;
                break;
            }
          }
        }
        if (measure == 1 || measure == 4) sum = sum / sqrt(sumSS * sumTT);
        out[(size_t)gx * nch + c] = sum;
      }
    }
  }
}

int orc_proximity_refexact(int measure, int type, int nch, const void* src,
                           int src_step, const void* tmpl, int tmpl_step,
                           void* dst, int dst_step, int W, int H, int tw, int th,
                           int row_begin, int row_end, int fused) {
  int e = check_args(measure, type, nch, W, H, tw, th);
  if (e) return e;
  if (row_end > H) row_end = H;
  if (type == 7)
    ref_f64(measure, nch, src, src_step, tmpl, tmpl_step, dst, dst_step, W, H,
            tw, th, row_begin, row_end, fused);
  else
    ref_f32(measure, type, nch, src, src_step, tmpl, tmpl_step, dst, dst_step,
            W, H, tw, th, row_begin, row_end, fused);
  return 0;
}

/* Exact window sums for integer sources: every product and sum in __int128. */
static void exact_int(int measure, int type, int nch, const void* src, int ss,
                      const void* tmpl, int ts, double* dst, int W, int H,
                      int tw, int th, const int* rows, int nrows) {
  const int left = -tw / 2, top = -th / 2;
  const int n = rows ? nrows : H;
#pragma omp parallel for schedule(dynamic, 1)
  for (int i = 0; i < n; ++i) {
    const int gy = rows ? rows[i] : i;
    for (int gx = 0; gx < W; ++gx) {
      for (int c = 0; c < nch; ++c) {
        i128 sum = 0, sS = 0, sT = 0;
        for (int h = 0; h < th; ++h) {
          for (int w = 0; w < tw; ++w) {
            const int px = gx + w + left, py = gy + h + top;
            const int64_t t = load_i(pix(tmpl, ts, type, nch, w, h, c), type);
            int64_t s = 0;
            if (!(px < 0 || py < 0 || px >= W || py >= H))
              s = load_i(pix(src, ss, type, nch, px, py, c), type);
            const i128 d = (i128)s - t;
            switch (measure) {
              case 0: sum += d * d; break;
              case 1: sum += d * d; sS += (i128)s * s; sT += (i128)t * t; break;
              case 2: sum += d < 0 ? -d : d; break;
              case 3: sum += (i128)s * t; break;
              default: sum += (i128)s * t; sS += (i128)s * s; sT += (i128)t * t; break;
            }
          }
        }
        long double v = (long double)sum;
        if (measure == 1 || measure == 4)
          v = v / sqrtl((long double)sS * (long double)sT);
        dst[((size_t)i * W + gx) * nch + c] = (double)v;
      }
    }
  }
}

/* Extended precision window sums for float sources (products of two F32
 * values are exact in long double). */
static void exact_flt(int measure, int type, int nch, const void* src, int ss,
                      const void* tmpl, int ts, double* dst, int W, int H,
                      int tw, int th, const int* rows, int nrows) {
  const int left = -tw / 2, top = -th / 2;
  const int n = rows ? nrows : H;
#pragma omp parallel for schedule(dynamic, 1)
  for (int i = 0; i < n; ++i) {
    const int gy = rows ? rows[i] : i;
    for (int gx = 0; gx < W; ++gx) {
      for (int c = 0; c < nch; ++c) {
        long double sum = 0, sS = 0, sT = 0;
        for (int h = 0; h < th; ++h) {
          for (int w = 0; w < tw; ++w) {
            const int px = gx + w + left, py = gy + h + top;
            const long double t = load_d(pix(tmpl, ts, type, nch, w, h, c), type);
            long double s = 0;
            if (!(px < 0 || py < 0 || px >= W || py >= H))
              s = load_d(pix(src, ss, type, nch, px, py, c), type);
            const long double d = s - t;
            switch (measure) {
              case 0: sum += d * d; break;
              case 1: sum += d * d; sS += s * s; sT += t * t; break;
              case 2: sum += fabsl(d); break;
              case 3: sum += s * t; break;
              default: sum += s * t; sS += s * s; sT += t * t; break;
            }
          }
        }
        if (measure == 1 || measure == 4) sum = sum / sqrtl(sS * sT);
        dst[((size_t)i * W + gx) * nch + c] = (double)sum;
      }
    }
  }
}

int orc_proximity_exact(int measure, int type, int nch, const void* src,
                        int src_step, const void* tmpl, int tmpl_step,
                        double* dst, int W, int H, int tw, int th) {
  int e = check_args(measure, type, nch, W, H, tw, th);
  if (e) return e;
  if (type <= 5)
    exact_int(measure, type, nch, src, src_step, tmpl, tmpl_step, dst, W, H, tw,
              th, 0, 0);
  else
    exact_flt(measure, type, nch, src, src_step, tmpl, tmpl_step, dst, W, H, tw,
              th, 0, 0);
  return 0;
}

int orc_proximity_exact_rows(int measure, int type, int nch, const void* src,
                             int src_step, const void* tmpl, int tmpl_step,
                             double* dst, int W, int H, int tw, int th,
                             const int* rows, int nrows) {
  int e = check_args(measure, type, nch, W, H, tw, th);
  if (e) return e;
  for (int i = 0; i < nrows; ++i)
    if (rows[i] < 0 || rows[i] >= H) return -30;
  if (type <= 5)
    exact_int(measure, type, nch, src, src_step, tmpl, tmpl_step, dst, W, H, tw,
              th, rows, nrows);
  else
    exact_flt(measure, type, nch, src, src_step, tmpl, tmpl_step, dst, W, H, tw,
              th, rows, nrows);
  return 0;
}

int orc_window_terms_exact(int type, int nch, const void* src, int src_step,
                           const void* tmpl, int tmpl_step, double* ssq,
                           double* st, double* tt, int W, int H, int tw,
                           int th) {
  int e = check_args(0, type, nch, W, H, tw, th);
  if (e) return e;
  const int left = -tw / 2, top = -th / 2;
  if (tt) {
    for (int c = 0; c < nch; ++c) {
      long double a = 0;
      for (int h = 0; h < th; ++h)
        for (int w = 0; w < tw; ++w) {
          const long double t = load_d(pix(tmpl, tmpl_step, type, nch, w, h, c), type);
          a += t * t;
        }
      tt[c] = (double)a;
    }
  }
  if (!ssq && !st) return 0;
#pragma omp parallel for schedule(dynamic, 4)
  for (int gy = 0; gy < H; ++gy) {
    for (int gx = 0; gx < W; ++gx) {
      for (int c = 0; c < nch; ++c) {
        long double a = 0, b = 0;
        for (int h = 0; h < th; ++h) {
          for (int w = 0; w < tw; ++w) {
            const int px = gx + w + left, py = gy + h + top;
            if (px < 0 || py < 0 || px >= W || py >= H) continue;
            const long double s = load_d(pix(src, src_step, type, nch, px, py, c), type);
            const long double t = load_d(pix(tmpl, tmpl_step, type, nch, w, h, c), type);
            a += s * s;
            b += s * t;
          }
        }
        const size_t o = ((size_t)gy * W + gx) * nch + c;
        if (ssq) ssq[o] = (double)a;
        if (st) st[o] = (double)b;
      }
    }
  }
  return 0;
}

/* Adjoints of the two differentiable measures, single channel.
 *   SqrDistance   O = sum (S - T)^2
 *       dO/dT[h][w] = -2 (S[p] - T[h][w]),  dO/dS[p] = 2 (S[p] - T[h][w])
 *   CrossCorr_Norm O = C / sqrt(E_S * E_T), C = sum S*T
 *       dO/dT[h][w] = S[p] / sqrt(E_S E_T) - O * T[h][w] / E_T
 *       dO/dS[p]    = T[h][w] / sqrt(E_S E_T) - O * S[p] / E_S
 * where p is the source pixel under template element (h, w); padded pixels
 * (outside the source) are constants and receive no gradient. */
int orc_proximity_backward(int measure, const double* S, const double* T,
                           const double* g, double* dS, double* dT, int W,
                           int H, int tw, int th) {
  if (measure != 0 && measure != 4) return -30;
  const int left = -tw / 2, top = -th / 2;
  long double* aT = (long double*)__builtin_alloca(sizeof(long double) * tw * th);
  for (int i = 0; i < tw * th; ++i) aT[i] = 0;
  long double eT = 0;
  for (int i = 0; i < tw * th; ++i) eT += (long double)T[i] * T[i];
  for (int i = 0; i < W * H; ++i) dS[i] = 0;
  for (int gy = 0; gy < H; ++gy) {
    for (int gx = 0; gx < W; ++gx) {
      const long double go = g[(size_t)gy * W + gx];
      long double eS = 0, C = 0;
      if (measure == 4) {
        for (int h = 0; h < th; ++h)
          for (int w = 0; w < tw; ++w) {
            const int px = gx + w + left, py = gy + h + top;
            if (px < 0 || py < 0 || px >= W || py >= H) continue;
            const long double s = S[(size_t)py * W + px];
            eS += s * s;
            C += s * T[h * tw + w];
          }
      }
      const long double inv = measure == 4 ? 1.0L / sqrtl(eS * eT) : 0;
      const long double O = C * inv;
      for (int h = 0; h < th; ++h)
        for (int w = 0; w < tw; ++w) {
          const int px = gx + w + left, py = gy + h + top;
          const int inside = !(px < 0 || py < 0 || px >= W || py >= H);
          const long double s = inside ? S[(size_t)py * W + px] : 0;
          const long double t = T[h * tw + w];
          if (measure == 0) {
            aT[h * tw + w] += go * (-2) * (s - t);
            if (inside) dS[(size_t)py * W + px] += (double)(go * 2 * (s - t));
          } else {
            aT[h * tw + w] += go * (s * inv - O * t / eT);
            if (inside)
              dS[(size_t)py * W + px] += (double)(go * (t * inv - O * s / eS));
          }
        }
    }
  }
  for (int i = 0; i < tw * th; ++i) dT[i] = (double)aT[i];
  return 0;
}
