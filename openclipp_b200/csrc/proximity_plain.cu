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
#include <algorithm>
#include <cuda_runtime.h>

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

template <int TYPE, typename CT, int MEAS, int RY>
__global__ void __launch_bounds__(kThreads, sizeof(CT) == 4 ? 2 : 1)
    prox_plain_kernel(const PlainParams p) {
  using ET = typename ElemOf<TYPE>::T;
  constexpr bool kNorm = (MEAS == kCrossCorrNorm || MEAS == kSqrDistanceNorm);
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

  CT acc[RY][RX];
  CT acc2[RY][RX];
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
    // Stage source rows [g0, g1) x logical columns [0, L).
    const int nel = (g1 - g0) * L;
    for (int idx = threadIdx.x; idx < nel; idx += kThreads) {
      const int q = idx / L;
      const int e = idx - q * L;
      const int gy = y0 + top + g0 + q;
      const int gx = x0 + left + e;
      CT v = CT(0);
      if (gx >= 0 && gx < p.W && gy >= 0 && gy < p.H)
        v = (CT)(*reinterpret_cast<const ET*>(
            p.src + (size_t)gy * p.src_pitch + ((size_t)gx * p.nch + c) * sizeof(ET)));
      *reinterpret_cast<CT*>(s_src + (size_t)q * p.rowBytes + phys_off<CT>(e)) = v;
    }
    // Stage template rows [tg0, tg1), zero-padded to twp columns.
    const int ntel = (tg1 - tg0) * p.twp;
    for (int idx = threadIdx.x; idx < ntel; idx += kThreads) {
      const int hh = idx / p.twp;
      const int w = idx - hh * p.twp;
      CT v = CT(0);
      if (w < p.tw)
        v = (CT)(*reinterpret_cast<const ET*>(
            p.tmpl + (size_t)(tg0 + hh) * p.tmpl_pitch + ((size_t)w * p.nch + c) * sizeof(ET)));
      s_t[idx] = v;
    }
    __syncthreads();

    const int qa = max(g0, warp * RY);
    const int qb = min(g1, warp * RY + RY + p.th - 1);
    for (int q = qa; q < qb; ++q) {
      const int r = q - warp * RY;
      const unsigned char* srow = s_src + (size_t)(q - g0) * p.rowBytes;
      for (int wc = 0; wc < nwc; ++wc) {
        CT win[RX + WCH];
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
        const int kmax = min(WCH, p.tw - wc * WCH);
#pragma unroll
        for (int j = 0; j < RY; ++j) {
          const int h = r - j;
          if (h < 0 || h >= p.th) continue;
          const CT* trow = s_t + (size_t)(h - tg0) * p.twp + wc * WCH;
          CT tv[WCH];
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
          if (kmax == WCH)
            apply_chunk<CT, MEAS>(acc[j], acc2[j], win, tv, WCH);
          else
            apply_chunk<CT, MEAS>(acc[j], acc2[j], win, tv, kmax);
        }
      }
    }
  }

  // Epilogue: value = sum (or sum / sqrt(sumSS * sumTT)), stored as F32/F64.
  CT tt = CT(0);
  if (kNorm) tt = reinterpret_cast<const CT*>(p.tt)[c];
#pragma unroll
  for (int j = 0; j < RY; ++j) {
    const int y = y0 + warp * RY + j;
    if (y >= p.H) continue;
#pragma unroll
    for (int i = 0; i < RX; ++i) {
      const int x = x0 + lane * RX + i;
      if (x >= p.W) continue;
      CT v = acc[j][i];
      if (kNorm) v = dv(v, sq(mul(acc2[j][i], tt)));
      char* o = p.dst + (size_t)y * p.dst_pitch;
      if (p.dst_f64)
        reinterpret_cast<double*>(o)[(size_t)x * p.dst_nch + c] = (double)v;
      else
        reinterpret_cast<float*>(o)[(size_t)x * p.dst_nch + c] = (float)v;
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
    return (size_t)rb * p.rowBytes + (size_t)tb * p.twp * sizeof(CT);
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
  auto kern = prox_plain_kernel<TYPE, CT, MEAS, RY>;
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
