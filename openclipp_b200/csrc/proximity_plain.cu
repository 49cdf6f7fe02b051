// Plain (CUDA-core) ImageProximity kernels for sm_100a.
//
// Computes the five measures of the reference's cl-files/ImageProximity.cl
// (SqrDistance :44, SqrDistance_Norm :122, AbsDistance :213, CrossCorr :290,
// CrossCorr_Norm :375) for every pixel type and 1, 2 or 4 interleaved
// channels, with the reference's geometry: same-size output, window of
// output (x, y) anchored at (x - tw/2, y - th/2), zero outside the source.
//
// Arithmetic. Each output is accumulated in one register in the reference's
// order (template row h outer, column w inner), one fused multiply-add per
// product term (sum += a*b -> fma(a, b, sum)), so for F32 and F64 sources the
// result is bit-identical to the reference kernel source compiled with FP
// contraction, which is what GPU OpenCL compilers do. Integer sources are
// accumulated exactly: in float when every partial sum is an integer below
// 2^24 (then identical to the reference), in double otherwise (exact while
// sums stay below 2^53, i.e. for every 8/16-bit case of practical size).
//
// Tiling. A CTA of 8 warps owns a 256 x (8*RY) output tile: lane l owns RX=8
// consecutive columns, warp w owns RY consecutive rows. Source rows of the
// tile (plus halo, converted to the compute type) and template rows sit in
// shared memory. For each source row q, a warp slides an RX+8 wide register
// window along x and applies it to all of its RY output rows at once, each
// with its own template row h = q - j, which keeps per-output order h-major.
// Shared-memory rows are stored in 16-byte chunks with one pad chunk after
// every 8, so the lanes' stride-2 (float) or stride-4 (double) chunk accesses
// hit distinct banks. Very tall templates are processed in row bands.
//
// FP32 compute types run on sm_100's packed FP32 arithmetic over pairs of
// output rows (PackedRows below), specialised on the width of the template's
// last column chunk so that the inner loop has no bounds tests.
#include <algorithm>
#include <cuda_runtime.h>
#include <type_traits>

#include "internal.h"

namespace ocipb {
namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int RX = 8;     // outputs per thread along x
constexpr int TX = 32 * RX;
constexpr int WCH = 8;    // template columns per inner step
constexpr int kSmemBudget = 200 * 1024;

template <int TYPE> struct ElemOf;
template <> struct ElemOf<U8> { typedef uint8_t T; };
template <> struct ElemOf<S8> { typedef int8_t T; };
template <> struct ElemOf<U16> { typedef uint16_t T; };
template <> struct ElemOf<S16> { typedef int16_t T; };
template <> struct ElemOf<U32> { typedef uint32_t T; };
template <> struct ElemOf<S32> { typedef int32_t T; };
template <> struct ElemOf<F32> { typedef float T; };
template <> struct ElemOf<F64> { typedef double T; };

struct PlainParams {
  const char* src;
  size_t src_pitch;
  const char* tmpl;
  size_t tmpl_pitch;
  char* dst;
  size_t dst_pitch;
  const void* tt;  // per-channel template energy (compute type), _Norm only
  int dst_f64;
  int W, H, nch, dst_nch;
  int tw, th, twp;
  int rowBytes;     // bytes per shared-memory source row (with pad chunks)
  int RB;           // source rows per band
  int TB;           // template rows per band
  int nbands;
};

__device__ __forceinline__ float mad(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double mad(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float dv(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ double dv(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ float sq(float a) { return __fsqrt_rn(a); }
__device__ __forceinline__ double sq(double a) { return __dsqrt_rn(a); }

// Byte offset of logical element e of a shared-memory row: 16-byte chunks,
// one pad chunk after every 8 chunks.
template <typename CT>
__device__ __forceinline__ int phys_off(int e) {
  constexpr int E = 16 / sizeof(CT);
  const int c = e / E;
  return (c + (c >> 3)) * 16 + (e % E) * (int)sizeof(CT);
}

template <typename CT>
__host__ __device__ inline int row_bytes_for(int L) {
  const int E = 16 / (int)sizeof(CT);
  const int chunks = (L + E - 1) / E;
  return (chunks + chunks / 8 + 1) * 16;
}

// Packed FP32 form (every measure, FP32 compute type). Output rows 2jp and
// 2jp + 1 of one column meet the same source element at every step (their
// template rows are h and h - 1), so the template is staged as row pairs
// (t(h, w), t(h - 1, w)) and each packed instruction (__fadd2_rn,
// __ffma2_rn: per component the same rounding as __fadd_rn, __fmaf_rn) does
// the two rows' operation of one term: the difference (the template staged
// negated, s + (-t) being s - t exactly: IEEE subtraction is the addition of
// the negation), the absolute-value add, the fused multiply-add of the
// product or of the square, the energy term s*s. Every per-output operation
// and its order are the scalar form's, so the results are bit-identical; the
// packed instructions halve the instruction count and, unlike scalar ones,
// load both halves of the FMA pipe.
template <typename CT, int MEAS>
struct PackedRows {
  // FP32 compute type: F32 sources, and 8-bit ones whose sums are exact in
  // float (integer arithmetic, so any order gives the same values).
  static constexpr bool value = std::is_same<CT, float>::value;
  // The template is staged negated for the measures that take differences.
  static constexpr bool neg = MEAS == kAbsDistance || MEAS == kSqrDistance ||
                              MEAS == kSqrDistanceNorm;
};

// One chunk of KMAX template columns for a pair of output rows whose template
// rows both lie inside the template: sd[e] holds window element e in both
// halves, tp[k] the pair's (possibly negated) template values of column k.
template <int MEAS, int KMAX>
__device__ __forceinline__ void pair_chunk(float2 (&acc)[RX], float2 (&acc2)[RX],
                                           const float2 (&sd)[RX + WCH], const float2 (&tp)[WCH]) {
#pragma unroll
  for (int k = 0; k < KMAX; ++k) {
#pragma unroll
    for (int i = 0; i < RX; ++i) {
      const float2 s = sd[i + k];
      if (MEAS == kAbsDistance) {
        const float2 d = __fadd2_rn(s, tp[k]);
        acc[i] = __fadd2_rn(acc[i], make_float2(fabsf(d.x), fabsf(d.y)));
      } else if (MEAS == kSqrDistance || MEAS == kSqrDistanceNorm) {
        const float2 d = __fadd2_rn(s, tp[k]);
        acc[i] = __ffma2_rn(d, d, acc[i]);
        if (MEAS == kSqrDistanceNorm) acc2[i] = __ffma2_rn(s, s, acc2[i]);
      } else {
        acc[i] = __ffma2_rn(s, tp[k], acc[i]);
        if (MEAS == kCrossCorrNorm) acc2[i] = __ffma2_rn(s, s, acc2[i]);
      }
    }
  }
}

// The same for one row of the pair (H = 0: row 2jp, the .x halves; H = 1: row
// 2jp + 1, the .y halves) when the other row's template row lies outside.
template <int MEAS, int KMAX, int H>
__device__ __forceinline__ void half_chunk(float2 (&acc)[RX], float2 (&acc2)[RX],
                                           const float (&win)[RX + WCH], const float (&tv)[WCH]) {
#pragma unroll
  for (int k = 0; k < KMAX; ++k) {
#pragma unroll
    for (int i = 0; i < RX; ++i) {
      const float s = win[i + k];
      float& a = H ? acc[i].y : acc[i].x;
      float& a2 = H ? acc2[i].y : acc2[i].x;
      if (MEAS == kAbsDistance) {
        a = __fadd_rn(a, fabsf(__fadd_rn(s, tv[k])));
      } else if (MEAS == kSqrDistance || MEAS == kSqrDistanceNorm) {
        const float d = __fadd_rn(s, tv[k]);
        a = __fmaf_rn(d, d, a);
        if (MEAS == kSqrDistanceNorm) a2 = __fmaf_rn(s, s, a2);
      } else {
        a = __fmaf_rn(s, tv[k], a);
        if (MEAS == kCrossCorrNorm) a2 = __fmaf_rn(s, s, a2);
      }
    }
  }
}

// One template-column chunk applied to one output row.
template <typename CT, int MEAS>
__device__ __forceinline__ void apply_chunk(CT (&acc)[RX], CT (&acc2)[RX],
                                            const CT (&win)[RX + WCH],
                                            const CT (&tv)[WCH], int kmax) {
#pragma unroll
  for (int k = 0; k < WCH; ++k) {
    if (k < kmax) {
#pragma unroll
      for (int i = 0; i < RX; ++i) {
        const CT s = win[i + k];
        const CT t = tv[k];
        if (MEAS == kCrossCorr) {
          acc[i] = mad(s, t, acc[i]);
        } else if (MEAS == kCrossCorrNorm) {
          acc[i] = mad(s, t, acc[i]);
          acc2[i] = mad(s, s, acc2[i]);
        } else if (MEAS == kSqrDistance) {
          const CT d = sub(s, t);
          acc[i] = mad(d, d, acc[i]);
        } else if (MEAS == kSqrDistanceNorm) {
          const CT d = sub(s, t);
          acc[i] = mad(d, d, acc[i]);
          acc2[i] = mad(s, s, acc2[i]);
        } else {  // kAbsDistance
          acc[i] = add(acc[i], fabs(sub(s, t)));
        }
      }
    }
  }
}

// KT: for the packed FP32 form, the columns of the template's last chunk,
// tw - WCH * ((tw - 1) / WCH), in 1 .. WCH; 0 for the other forms.
template <int TYPE, typename CT, int MEAS, int RY, int KT>
__global__ void __launch_bounds__(kThreads, sizeof(CT) == 4 ? 2 : 1)
    prox_plain_kernel(const PlainParams p) {
  using ET = typename ElemOf<TYPE>::T;
  constexpr bool kNorm = (MEAS == kCrossCorrNorm || MEAS == kSqrDistanceNorm);
  constexpr bool kPacked = PackedRows<CT, MEAS>::value;
  constexpr int TY = kWarps * RY;
  extern __shared__ __align__(16) unsigned char smem[];
  unsigned char* s_src = smem;
  CT* s_t = reinterpret_cast<CT*>(smem + (size_t)p.RB * p.rowBytes);

  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int c = blockIdx.z;
  const int x0 = blockIdx.x * TX;
  const int y0 = blockIdx.y * TY;
  const int left = -(p.tw / 2);
  const int top = -(p.th / 2);
  const int L = TX + p.twp;          // logical elements per source row
  const int qtot = TY + p.th - 1;    // source rows needed by the tile
  const int nwc = p.twp / WCH;
  const int tstride = kPacked ? 2 * p.twp : p.twp;  // template row stride in s_t

  CT acc[RY][RX];
  CT acc2[RY][RX];
  // Packed form: output rows (2jp, 2jp + 1) of column i.
  float2 accr[RY / 2][RX], accr2[RY / 2][RX];
#pragma unroll
  for (int j = 0; j < RY / 2; ++j)
#pragma unroll
    for (int i = 0; i < RX; ++i) {
      accr[j][i] = make_float2(0.f, 0.f);
      accr2[j][i] = make_float2(0.f, 0.f);
    }
#pragma unroll
  for (int j = 0; j < RY; ++j)
#pragma unroll
    for (int i = 0; i < RX; ++i) {
      acc[j][i] = CT(0);
      acc2[j][i] = CT(0);
    }

  for (int band = 0; band < p.nbands; ++band) {
    const int g0 = band * p.RB;
    const int g1 = min(g0 + p.RB, qtot);
    // Template rows h that source rows [g0, g1) meet: h = q - w*RY - j.
    const int tg0 = max(0, g0 - (TY - 1));
    const int tg1 = min(p.th, g1);
    if (band > 0) __syncthreads();
    // Stage source rows [g0, g1) x logical columns [0, L): a warp per row,
    // lanes along the row (coalesced), zero outside the image. Sources of the
    // compute type are copied asynchronously (no register round trip), the
    // copies overlapping the template staging below.
    for (int qq = warp; qq < g1 - g0; qq += kWarps) {
      const int gy = y0 + top + g0 + qq;
      const bool row_in = gy >= 0 && gy < p.H;
      const ET* grow =
          reinterpret_cast<const ET*>(p.src + (size_t)(row_in ? gy : 0) * p.src_pitch) + c;
      unsigned char* srow = s_src + (size_t)qq * p.rowBytes;
      if constexpr (std::is_same<CT, ET>::value) {
        // Asynchronous copies, zero-filled outside the image (source size 0).
#pragma unroll 4
        for (int e = lane; e < L; e += 32) {
          const int gx = x0 + left + e;
          const bool in = row_in && gx >= 0 && gx < p.W;
          const ET* g = grow + (size_t)(in ? gx : 0) * p.nch;
          const unsigned sa = (unsigned)__cvta_generic_to_shared(srow + phys_off<CT>(e));
          asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;\n" ::"r"(sa), "l"(g),
                       "n"((int)sizeof(ET)), "r"(in ? (int)sizeof(ET) : 0)
                       : "memory");
        }
      } else {
#pragma unroll 4
        for (int e = lane; e < L; e += 32) {
          const int gx = x0 + left + e;
          CT v = CT(0);
          if (row_in && gx >= 0 && gx < p.W) v = (CT)grow[(size_t)gx * p.nch];
          *reinterpret_cast<CT*>(srow + phys_off<CT>(e)) = v;
        }
      }
    }
    if constexpr (std::is_same<CT, ET>::value) asm volatile("cp.async.commit_group;\n" ::: "memory");
    // Stage template rows [tg0, tg1), zero-padded to twp columns. The packed
    // form stores row h as the pairs (t(h, w), t(h - 1, w)), negated for the
    // measures that take differences.
    // Read-only loads, unrolled, so that a thread's loads are in flight together.
    const int ntel = (tg1 - tg0) * tstride;
#pragma unroll 8
    for (int idx = threadIdx.x; idx < ntel; idx += kThreads) {
      const int hh = idx / tstride;
      int w = idx - hh * tstride;
      int trow = tg0 + hh;
      if (kPacked) {  // pairs (row h, row h - 1) of column w
        w = (idx - hh * tstride) >> 1;
        trow -= (idx - hh * tstride) & 1;
      }
      CT v = CT(0);
      if (w < p.tw && trow >= 0)
        v = (CT)__ldg(reinterpret_cast<const ET*>(
            p.tmpl + (size_t)trow * p.tmpl_pitch + ((size_t)w * p.nch + c) * sizeof(ET)));
      s_t[idx] = (kPacked && PackedRows<CT, MEAS>::neg) ? -v : v;
    }
    if constexpr (std::is_same<CT, ET>::value) asm volatile("cp.async.wait_all;\n" ::: "memory");
    __syncthreads();

    // Window of source row q for template columns wc*WCH ..: RX + WCH elements.
    auto load_window = [&](const unsigned char* srow, int wc, CT (&win)[RX + WCH]) {
      const int e0 = lane * RX + wc * WCH;
      constexpr int E = 16 / sizeof(CT);
#pragma unroll
      for (int v = 0; v < (RX + WCH) / E; ++v) {
        const int e = e0 + v * E;
        if (sizeof(CT) == 4) {
          const float4 f = *reinterpret_cast<const float4*>(srow + phys_off<CT>(e));
          win[v * 4 + 0] = (CT)f.x;
          win[v * 4 + 1] = (CT)f.y;
          win[v * 4 + 2] = (CT)f.z;
          win[v * 4 + 3] = (CT)f.w;
        } else {
          const double2 d = *reinterpret_cast<const double2*>(srow + phys_off<CT>(e));
          win[v * 2 + 0] = (CT)d.x;
          win[v * 2 + 1] = (CT)d.y;
        }
      }
    };
    auto load_tmpl = [&](const CT* trow, CT (&tv)[WCH]) {
      if (sizeof(CT) == 4) {
        const float4 a = reinterpret_cast<const float4*>(trow)[0];
        const float4 b = reinterpret_cast<const float4*>(trow)[1];
        tv[0] = (CT)a.x; tv[1] = (CT)a.y; tv[2] = (CT)a.z; tv[3] = (CT)a.w;
        tv[4] = (CT)b.x; tv[5] = (CT)b.y; tv[6] = (CT)b.z; tv[7] = (CT)b.w;
      } else {
#pragma unroll
        for (int k = 0; k < WCH / 2; ++k) {
          const double2 d = reinterpret_cast<const double2*>(trow)[k];
          tv[2 * k] = (CT)d.x;
          tv[2 * k + 1] = (CT)d.y;
        }
      }
    };

    // Source rows q meet template rows h = q - warp*RY - j of the warp's
    // output rows j. Rows where some h falls outside the template (the first
    // and last RY - 1 of the warp) take the checked loop; the others, where
    // every output row has a template row, take the unchecked one.
    const int qa = max(g0, warp * RY);
    const int qb = min(g1, warp * RY + RY + p.th - 1);
    const int lo = min(max(qa, warp * RY + RY - 1), qb);
    const int hi = min(max(lo, warp * RY + p.th), qb);
    auto row_checked = [&](int q) {
      const int r = q - warp * RY;
      const unsigned char* srow = s_src + (size_t)(q - g0) * p.rowBytes;
      for (int wc = 0; wc < nwc; ++wc) {
        CT win[RX + WCH];
        load_window(srow, wc, win);
        const int kmax = min(WCH, p.tw - wc * WCH);
#pragma unroll
        for (int j = 0; j < RY; ++j) {
          const int h = r - j;
          if (h < 0 || h >= p.th) continue;
          CT tv[WCH];
          load_tmpl(s_t + (size_t)(h - tg0) * tstride + wc * WCH, tv);
          if (kmax == WCH)
            apply_chunk<CT, MEAS>(acc[j], acc2[j], win, tv, WCH);
          else
            apply_chunk<CT, MEAS>(acc[j], acc2[j], win, tv, kmax);
        }
      }
    };
    if constexpr (kPacked) {
      // Chunks of WCH template columns: nfull full ones, then the last, of
      // KT columns. check: some of the rows' template rows may lie outside.
      const int nfull = (p.tw - 1) / WCH;
      auto rows = [&](int qbeg, int qend, auto check) {
        for (int q = qbeg; q < qend; ++q) {
          const unsigned char* srow = s_src + (size_t)(q - g0) * p.rowBytes;
          const CT* t0 = s_t + (size_t)(q - warp * RY - tg0) * tstride;
          auto chunk = [&](int wc, auto kmaxc) {
            constexpr int KMAX = decltype(kmaxc)::value;
            CT win[RX + WCH];
            load_window(srow, wc, win);
            float2 sd[RX + WCH];  // each window element in both halves
#pragma unroll
            for (int e = 0; e < RX + WCH; ++e) sd[e] = make_float2(win[e], win[e]);
#pragma unroll
            for (int jp = 0; jp < RY / 2; ++jp) {
              // Rows near the warp's first and last source rows: a pair whose
              // template rows are both inside the template is packed, a pair
              // with one inside takes only that half (scalar), else none.
              int both = 3;
              if (decltype(check)::value) {
                const int h = q - warp * RY - 2 * jp;
                both = (h >= 0 && h < p.th ? 1 : 0) | (h >= 1 && h - 1 < p.th ? 2 : 0);
              }
              if (both == 3) {
                const float4* tr =
                    reinterpret_cast<const float4*>(t0 - (size_t)(2 * jp) * tstride + 2 * wc * WCH);
                float2 tp[WCH];  // (t(h, k), t(h - 1, k)), h the template row of output row 2jp
#pragma unroll
                for (int m = 0; m < WCH / 2; ++m) {
                  const float4 f = tr[m];
                  tp[2 * m] = make_float2(f.x, f.y);
                  tp[2 * m + 1] = make_float2(f.z, f.w);
                }
                pair_chunk<MEAS, KMAX>(accr[jp], accr2[jp], sd, tp);
              } else if (both != 0) {
                // The one template row inside: h (output row 2jp) or h - 1
                // (row 2jp + 1), read from its own staged row.
                const float4* tr = reinterpret_cast<const float4*>(
                    t0 - (size_t)(2 * jp + (both == 2 ? 1 : 0)) * tstride + 2 * wc * WCH);
                float tv[WCH];
#pragma unroll
                for (int m = 0; m < WCH / 2; ++m) {
                  const float4 f = tr[m];
                  tv[2 * m] = f.x;
                  tv[2 * m + 1] = f.z;
                }
                if (both == 1)
                  half_chunk<MEAS, KMAX, 0>(accr[jp], accr2[jp], win, tv);
                else
                  half_chunk<MEAS, KMAX, 1>(accr[jp], accr2[jp], win, tv);
              }
            }
          };
          for (int wc = 0; wc < nfull; ++wc) chunk(wc, std::integral_constant<int, WCH>());
          chunk(nfull, std::integral_constant<int, KT>());
        }
      };
      rows(qa, lo, std::true_type());
      rows(lo, hi, std::false_type());
      rows(hi, qb, std::true_type());
    } else {
      for (int q = qa; q < lo; ++q) row_checked(q);
      for (int q = lo; q < hi; ++q) row_checked(q);
      for (int q = hi; q < qb; ++q) row_checked(q);
    }
  }

  // Epilogue: value = sum (or sum / sqrt(sumSS * sumTT)), stored as F32/F64.
  CT tt = CT(0);
  if (kNorm) tt = reinterpret_cast<const CT*>(p.tt)[c];
#pragma unroll
  for (int j = 0; j < RY; ++j) {
    const int y = y0 + warp * RY + j;
    if (y >= p.H) continue;
    CT v[RX];
#pragma unroll
    for (int i = 0; i < RX; ++i) {
      v[i] = acc[j][i];
      CT e2 = acc2[j][i];
      if constexpr (kPacked) {
        v[i] = (j & 1) ? accr[j / 2][i].y : accr[j / 2][i].x;
        e2 = (j & 1) ? accr2[j / 2][i].y : accr2[j / 2][i].x;
      }
      if (kNorm) v[i] = dv(v[i], sq(mul(e2, tt)));
    }
    char* o = p.dst + (size_t)y * p.dst_pitch;
    const int xl = x0 + lane * RX;
    float* of = reinterpret_cast<float*>(o) + (size_t)xl;
    if (!p.dst_f64 && p.dst_nch == 1 && xl + RX <= p.W && (reinterpret_cast<size_t>(of) & 15) == 0) {
      // One-channel F32 row segment: 16-byte stores.
#pragma unroll
      for (int i = 0; i < RX; i += 4)
        *reinterpret_cast<float4*>(of + i) =
            make_float4((float)v[i], (float)v[i + 1], (float)v[i + 2], (float)v[i + 3]);
      continue;
    }
#pragma unroll
    for (int i = 0; i < RX; ++i) {
      const int x = xl + i;
      if (x >= p.W) continue;
      if (p.dst_f64)
        reinterpret_cast<double*>(o)[(size_t)x * p.dst_nch + c] = (double)v[i];
      else
        reinterpret_cast<float*>(o)[(size_t)x * p.dst_nch + c] = (float)v[i];
    }
  }
}

// Template energy sum T^2 in the reference's order (h outer, w inner, one
// fused multiply-add per term), one value per channel: the reference
// recomputes it inside every output's loop (ImageProximity.cl:152, :406),
// always with the same operands in the same order.
template <int TYPE, typename CT>
__global__ void __launch_bounds__(256) template_energy_kernel(const char* tmpl, size_t pitch,
                                                              int nch, int tw, int th, CT* out) {
  using ET = typename ElemOf<TYPE>::T;
  constexpr int kMaxStage = 32768 / (int)sizeof(CT);
  __shared__ CT st[kMaxStage];
  const int c = blockIdx.x;
  CT s = CT(0);
  // The template is staged in shared memory in chunks (all threads load), then
  // one thread runs the chain: the order of the additions is the reference's.
  for (int base = 0; base < th * tw; base += kMaxStage) {
    const int n = min(kMaxStage, th * tw - base);
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      const int h = (base + i) / tw, w = (base + i) - h * tw;
      st[i] = (CT)reinterpret_cast<const ET*>(tmpl + (size_t)h * pitch)[(size_t)w * nch + c];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll 8
      for (int i = 0; i < n; ++i) s = mad(st[i], st[i], s);
    }
  }
  if (threadIdx.x == 0) out[c] = s;
}

template <int TYPE, typename CT, int MEAS>
cudaError_t launch_typed(const DevImage& src, const DevImage& tmpl,
                         const DevImage& dst, void* tt_buf, cudaStream_t st) {
  constexpr int RY = sizeof(CT) == 4 ? 4 : 2;
  constexpr int TY = kWarps * RY;
  PlainParams p;
  p.src = (const char*)src.ptr;
  p.src_pitch = src.pitch;
  p.tmpl = (const char*)tmpl.ptr;
  p.tmpl_pitch = tmpl.pitch;
  p.dst = (char*)dst.ptr;
  p.dst_pitch = dst.pitch;
  p.dst_f64 = dst.type == F64;
  p.W = src.width;
  p.H = src.height;
  p.nch = src.nch;
  p.dst_nch = dst.nch;
  p.tw = tmpl.width;
  p.th = tmpl.height;
  p.twp = (p.tw + WCH - 1) / WCH * WCH;
  p.tt = tt_buf;
  const int L = TX + p.twp;
  p.rowBytes = row_bytes_for<CT>(L);
  const int qtot = TY + p.th - 1;
  // Band size: all rows if they fit, else as many as the budget allows.
  int RB = qtot;
  auto bytes_for = [&](int rb) {
    const int tb = std::min(p.th, rb + TY - 1);
    return (size_t)rb * p.rowBytes +
           (size_t)tb * p.twp * sizeof(CT) * (PackedRows<CT, MEAS>::value ? 2 : 1);
  };
  while (RB > 1 && bytes_for(RB) > (size_t)kSmemBudget) RB = (RB + 1) / 2;
  if (bytes_for(RB) > (size_t)kSmemBudget) return cudaErrorInvalidValue;
  p.RB = RB;
  p.TB = std::min(p.th, RB + TY - 1);
  p.nbands = (qtot + RB - 1) / RB;
  const size_t smem = bytes_for(RB);

  constexpr bool kNorm = (MEAS == kCrossCorrNorm || MEAS == kSqrDistanceNorm);
  if (kNorm) {
    template_energy_kernel<TYPE, CT><<<src.nch, 256, 0, st>>>(
        (const char*)tmpl.ptr, tmpl.pitch, tmpl.nch, p.tw, p.th, (CT*)tt_buf);
    count_launches(1);
  }
  auto kern = prox_plain_kernel<TYPE, CT, MEAS, RY, PackedRows<CT, MEAS>::value ? WCH : 0>;
  if constexpr (PackedRows<CT, MEAS>::value) {
    switch (p.tw - WCH * ((p.tw - 1) / WCH)) {
      case 1: kern = prox_plain_kernel<TYPE, CT, MEAS, RY, 1>; break;
      case 2: kern = prox_plain_kernel<TYPE, CT, MEAS, RY, 2>; break;
      case 3: kern = prox_plain_kernel<TYPE, CT, MEAS, RY, 3>; break;
      case 4: kern = prox_plain_kernel<TYPE, CT, MEAS, RY, 4>; break;
      case 5: kern = prox_plain_kernel<TYPE, CT, MEAS, RY, 5>; break;
      case 6: kern = prox_plain_kernel<TYPE, CT, MEAS, RY, 6>; break;
      case 7: kern = prox_plain_kernel<TYPE, CT, MEAS, RY, 7>; break;
      default: kern = prox_plain_kernel<TYPE, CT, MEAS, RY, 8>; break;
    }
  }
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem);
  if (e != cudaSuccess) return e;
  dim3 grid((p.W + TX - 1) / TX, (p.H + TY - 1) / TY, src.nch);
  kern<<<grid, kThreads, smem, st>>>(p);
  count_launches(1);
  return cudaGetLastError();
}

template <int TYPE, typename CT>
cudaError_t launch_measure(Measure m, const DevImage& src, const DevImage& tmpl,
                           const DevImage& dst, void* tt, cudaStream_t st) {
  switch (m) {
    case kSqrDistance: return launch_typed<TYPE, CT, kSqrDistance>(src, tmpl, dst, tt, st);
    case kSqrDistanceNorm: return launch_typed<TYPE, CT, kSqrDistanceNorm>(src, tmpl, dst, tt, st);
    case kAbsDistance: return launch_typed<TYPE, CT, kAbsDistance>(src, tmpl, dst, tt, st);
    case kCrossCorr: return launch_typed<TYPE, CT, kCrossCorr>(src, tmpl, dst, tt, st);
    case kCrossCorrNorm: return launch_typed<TYPE, CT, kCrossCorrNorm>(src, tmpl, dst, tt, st);
  }
  return cudaErrorInvalidValue;
}

}  // namespace

// Whether float accumulation is exact for an 8-bit source: every partial sum
// is an integer of magnitude at most area * 255^2 (255 for AbsDistance).
static bool small_int_exact_in_float(Measure m, int area) {
  const double maxterm = (m == kAbsDistance) ? 255.0 : 65025.0;
  return (double)area * maxterm <= 16777216.0;
}

cudaError_t launch_proximity_plain(Measure m, const DevImage& src,
                                   const DevImage& tmpl, const DevImage& dst,
                                   void* tt_scratch, cudaStream_t st) {
  const int area = tmpl.width * tmpl.height;
  if (m == kAbsDistance && proximity_sad_8bit_supported(src, tmpl))
    return launch_proximity_sad_8bit(src, tmpl, dst, st);
  switch (src.type) {
    case U8:
      return small_int_exact_in_float(m, area)
                 ? launch_measure<U8, float>(m, src, tmpl, dst, tt_scratch, st)
                 : launch_measure<U8, double>(m, src, tmpl, dst, tt_scratch, st);
    case S8:
      return small_int_exact_in_float(m, area)
                 ? launch_measure<S8, float>(m, src, tmpl, dst, tt_scratch, st)
                 : launch_measure<S8, double>(m, src, tmpl, dst, tt_scratch, st);
    case U16: return launch_measure<U16, double>(m, src, tmpl, dst, tt_scratch, st);
    case S16: return launch_measure<S16, double>(m, src, tmpl, dst, tt_scratch, st);
    case U32: return launch_measure<U32, double>(m, src, tmpl, dst, tt_scratch, st);
    case S32: return launch_measure<S32, double>(m, src, tmpl, dst, tt_scratch, st);
    case F32: return launch_measure<F32, float>(m, src, tmpl, dst, tt_scratch, st);
    case F64: return launch_measure<F64, double>(m, src, tmpl, dst, tt_scratch, st);
  }
  return cudaErrorInvalidValue;
}

}  // namespace ocipb
