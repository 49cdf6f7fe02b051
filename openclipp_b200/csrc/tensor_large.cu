// Tensor-core ImageProximity for templates larger than 64 x 64.
//
// The reference serves large templates with its FFT path
// (C++/programs/ImageProximityFFT.cpp:112-210: an FFT correlation plus the
// window statistics of cl-files/ImageProximityFFT.cl:55-147 from a
// SqrIntegral). Here the product term is split over template tiles of at
// most 64 x 64: each tile is one launch of the tcgen05 kernel with the
// tile's offset folded into the window anchor, writing (first tile) or adding
// (the others) its product sums to an F64 map. Integer sums stay exact (i8
// MMA, int32 per tile, FP64 across tiles); split-BF16 sums keep their
// per-tile accuracy. A scoring pass then forms the measure per output from
// that map, the window energy (the row energies of row_energy.cu summed over
// th rows as a running FP64 sum down each column) and the template energy,
// with the same formulas as the one-launch kernel's epilogue: U8 results are
// bit-identical to the plain path's, F32 and U16 within its split-BF16 error.
#include <cuda_runtime.h>

#include <algorithm>
#include <type_traits>

#include "host.h"
#include "internal.h"
#include "row_energy.h"
#include "tensor.h"

namespace ocipb {
namespace {

// Template energy sum T^2 per channel, FP64 (exact for integer templates).
template <typename ET>
__global__ void template_energy_f64_kernel(const char* tmpl, size_t pitch, int tw, int th, int nch,
                                           double* out) {
  const int c = blockIdx.x;
  double e = 0.0;
  for (int i = threadIdx.x; i < tw * th; i += blockDim.x) {
    const int h = i / tw, w = i - h * tw;
    const double v = reinterpret_cast<const ET*>(tmpl + (size_t)h * pitch)[(size_t)w * nch + c];
    e += v * v;
  }
  __shared__ double part[32];
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) e += __shfl_xor_sync(0xffffffffu, e, d);
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = e;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) t += part[i];
    out[c] = t;
  }
}

struct ScoreParams {
  const char* cmap;     // F64 product sums, channels interleaved
  size_t c_pitch;
  const char* rmap;     // row energies (int32 for U8, FP32 otherwise), one plane per channel
  size_t r_pitch, r_plane;
  const double* et;     // template energy per channel
  char* dst;
  size_t dst_pitch;
  int dst_f64;
  int W, H, nch;
  int th, ay;
  int measure;
  int band;             // output rows per thread
  int u8_float;         // U8 _Norm in float arithmetic (the plain path's float sums are exact)
};

// One thread per (column, channel) and band of rows: the window energy is a
// running FP64 sum of row energies down the column (the row entering at the
// bottom added, the row leaving at the top dropped), read four rows ahead.
template <bool SPLIT>
__global__ void __launch_bounds__(256) large_score_kernel(const ScoreParams p) {
  typedef typename std::conditional<SPLIT, float, int>::type RT;
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int xc = (int)(idx % ((long long)p.W * p.nch));  // x * nch + c
  const int y0 = (int)(idx / ((long long)p.W * p.nch)) * p.band;
  if (y0 >= p.H) return;
  const int x = xc / p.nch, c = xc - x * p.nch;
  const int y1 = min(p.H, y0 + p.band);
  const char* rplane = p.rmap + c * p.r_plane;
  auto r_at = [&](int r) -> double {
    return (r >= 0 && r < p.H) ? static_cast<double>(
                                     reinterpret_cast<const RT*>(rplane + (size_t)r * p.r_pitch)[x])
                               : 0.0;
  };
  const bool need_e = p.measure != kCrossCorr;
  double e = 0.0;
  if (need_e)
    for (int r = y0 - p.ay; r < y0 - p.ay + p.th - 1; ++r) e += r_at(r);
  const double et = p.et[c];
  for (int yb = y0; yb < y1; yb += 4) {
    double cin[4], rin[4], rout[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int y = yb + u;
      const bool in = y < y1;
      cin[u] = in ? reinterpret_cast<const double*>(p.cmap + (size_t)y * p.c_pitch)[xc] : 0.0;
      rin[u] = in && need_e ? r_at(y - p.ay + p.th - 1) : 0.0;
      rout[u] = in && need_e ? r_at(y - p.ay) : 0.0;
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int y = yb + u;
      if (y >= y1) break;
      e += rin[u];
      const double cc = cin[u];
      double v;
      float vf;
      if (SPLIT) {
        const double num = (p.measure == kCrossCorr || p.measure == kCrossCorrNorm)
                               ? cc
                               : e - 2.0 * cc + et;
        v = (p.measure == kCrossCorr || p.measure == kSqrDistance) ? num : num * rsqrt(e * et);
        vf = (float)v;
      } else {
        // Exact integers in FP64; the plain path's float or double formulas.
        const double num = (p.measure == kCrossCorr || p.measure == kCrossCorrNorm)
                               ? cc
                               : e - 2.0 * cc + et;
        if (p.measure == kCrossCorr || p.measure == kSqrDistance) {
          v = num;
          vf = (float)num;
        } else if (p.u8_float) {
          vf = __fdiv_rn((float)num, __fsqrt_rn(__fmul_rn((float)e, (float)et)));
          v = vf;
        } else {
          v = __ddiv_rn(num, __dsqrt_rn(__dmul_rn(e, et)));
          vf = (float)v;
        }
      }
      char* orow = p.dst + (size_t)y * p.dst_pitch;
      if (p.dst_f64)
        reinterpret_cast<double*>(orow)[xc] = v;
      else
        reinterpret_cast<float*>(orow)[xc] = vf;
      e -= rout[u];
    }
  }
}

}  // namespace

cudaError_t launch_proximity_tensor_large(Context& ctx, Measure m, const DevImage& src,
                                          const DevImage& tmpl, const DevImage& dst) {
  const int tw = tmpl.width, th = tmpl.height, nch = src.nch;
  const int ax = tw / 2, ay = th / 2;
  const int es = type_bytes(tmpl.type);
  // Product sums: F64 map with the source's channels interleaved.
  const size_t c_pitch = ((size_t)src.width * nch * 8 + 127) / 128 * 128;
  char* cmap = reinterpret_cast<char*>(ctx.scratch(Context::kProductMap, c_pitch * src.height));
  DevImage cview;
  cview.ptr = cmap;
  cview.pitch = c_pitch;
  cview.width = src.width;
  cview.height = src.height;
  cview.nch = nch;
  cview.type = F64;
  // Tiles of at most 64 x 64, balanced: rows [i th / ntr, (i + 1) th / ntr).
  const int ntr = (th + 63) / 64, ntc = (tw + 63) / 64;
  for (int i = 0; i < ntr; ++i) {
    const int r0 = i * th / ntr, r1 = (i + 1) * th / ntr;
    for (int j = 0; j < ntc; ++j) {
      const int c0 = j * tw / ntc, c1 = (j + 1) * tw / ntc;
      DevImage tile = tmpl;
      tile.ptr = (char*)tmpl.ptr + (size_t)r0 * tmpl.pitch + (size_t)c0 * nch * es;
      tile.width = c1 - c0;
      tile.height = r1 - r0;
      const cudaError_t e =
          launch_tensor_product_sums(ctx, src, tile, cview, ax - c0, ay - r0, i + j > 0);
      if (e != cudaSuccess) return e;
    }
  }
  // Row energies of the whole template width (measures other than CrossCorr).
  const size_t r_pitch = row_energy_pitch(src.width), r_plane = r_pitch * src.height;
  char* rmap = nullptr;
  if (m != kCrossCorr) {
    rmap = reinterpret_cast<char*>(ctx.scratch(Context::kEnergyMap, r_plane * nch));
    const cudaError_t e = launch_row_energy(src, tw, ax, rmap, r_pitch, r_plane, ctx.stream);
    if (e != cudaSuccess) return e;
  }
  double* et = reinterpret_cast<double*>(ctx.scratch(Context::kTemplateStats, 64));
  switch (tmpl.type) {
    case U8:
      template_energy_f64_kernel<uint8_t><<<nch, 256, 0, ctx.stream>>>(
          (const char*)tmpl.ptr, tmpl.pitch, tw, th, nch, et);
      break;
    case U16:
      template_energy_f64_kernel<uint16_t><<<nch, 256, 0, ctx.stream>>>(
          (const char*)tmpl.ptr, tmpl.pitch, tw, th, nch, et);
      break;
    default:
      template_energy_f64_kernel<float><<<nch, 256, 0, ctx.stream>>>(
          (const char*)tmpl.ptr, tmpl.pitch, tw, th, nch, et);
      break;
  }
  count_launches(1);
  ScoreParams p;
  p.cmap = cmap;
  p.c_pitch = c_pitch;
  p.rmap = rmap;
  p.r_pitch = r_pitch;
  p.r_plane = r_plane;
  p.et = et;
  p.dst = (char*)dst.ptr;
  p.dst_pitch = dst.pitch;
  p.dst_f64 = dst.type == F64;
  p.W = src.width;
  p.H = src.height;
  p.nch = nch;
  p.th = th;
  p.ay = ay;
  p.measure = m;
  p.u8_float = (double)tw * th * 65025.0 <= 16777216.0;
  // Bands: about 2048 threads per SM, each band at least th rows tall (its
  // first th - 1 row energies are summed before the first output).
  const long long cols = (long long)src.width * nch;
  const long long want = std::max(1LL, (2048LL * ctx.sm_count + cols - 1) / cols);
  p.band = (int)std::max<long long>((src.height + want - 1) / want, std::min(src.height, th));
  const long long threads = cols * ((src.height + p.band - 1) / p.band);
  const int blocks = (int)((threads + 255) / 256);
  if (src.type == U8)
    large_score_kernel<false><<<blocks, 256, 0, ctx.stream>>>(p);
  else
    large_score_kernel<true><<<blocks, 256, 0, ctx.stream>>>(p);
  count_launches(1);
  return cudaGetLastError();
}

}  // namespace ocipb
