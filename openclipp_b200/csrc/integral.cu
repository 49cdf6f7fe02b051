// Integral / SqrIntegral scan for sm_100a.
//
// Computes the reference's inclusive 2-D prefix sum (cl-files/Integral.cl
// :39-460, launched by C++/programs/Integral.cpp:143-241): D(x, y) = sum of
// S (or S^2) over [0..x] x [0..y], per channel, into an F32 or F64 image.
// Accumulation is exact: int64 for integer sources (every value fits: |S| <
// 2^32 and |S|^2 < 2^32 for 8/16-bit types, W*H < 2^31), FP64 for float
// sources and for the squares of 32-bit integers. The destination receives
// one rounding of the accumulated value, where the reference accumulates in
// the destination type (its F32 result is exact only while sums stay below
// 2^24).
//
// Layout: the image is cut into 256 x 64 tiles, one warp per tile (lane l
// holds 8 consecutive columns). Three passes, each reading the source once
// with coalesced loads (the second read mostly hits L2):
//   1. tile reduce: per-row tile sums (RowSum) and the tile-local column
//      prefix of the tile's column sums (LB) -- the counterpart of the
//      reference's vertical/horizontal junction buffers;
//   2. junctions: RowLeft = exclusive scan of RowSum across tiles of a row,
//      BandLeft = exclusive scan of tile totals across a band, Top = exclusive
//      scan over bands of (BandLeft + LB) per column (the full integral of the
//      row just above each band);
//   3. final: D = Top + running sum over the band's rows of
//      (RowLeft + warp-scanned row prefix), one store per pixel.
#include <cuda_runtime.h>

#include "internal.h"

namespace ocipb {
namespace {

constexpr int kTW = 256;   // tile width (32 lanes x 8 columns)
constexpr int kTH = 64;    // tile height
constexpr int kPX = 8;     // columns per lane
constexpr int kWarpsPerCta = 4;

template <int TYPE> struct ElemOf;
template <> struct ElemOf<U8> { typedef uint8_t T; };
template <> struct ElemOf<S8> { typedef int8_t T; };
template <> struct ElemOf<U16> { typedef uint16_t T; };
template <> struct ElemOf<S16> { typedef int16_t T; };
template <> struct ElemOf<U32> { typedef uint32_t T; };
template <> struct ElemOf<S32> { typedef int32_t T; };
template <> struct ElemOf<F32> { typedef float T; };
template <> struct ElemOf<F64> { typedef double T; };

struct IntegralParams {
  const char* src;
  size_t src_pitch;
  char* dst;
  size_t dst_pitch;
  int dst_f64;
  int W, H, nch;
  int nBX, nBY;
  void* rowsum;    // [nch][H][nBX]     RowSum, then RowLeft
  void* lb;        // [nch][nBY][W]     LB, then Top
  void* bandleft;  // [nch][nBY][nBX]
};

template <typename A>
__device__ __forceinline__ A warp_incl_scan(A v, int lane) {
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const A o = __shfl_up_sync(0xffffffffu, v, d);
    if (lane >= d) v += o;
  }
  return v;
}

template <typename A>
__device__ __forceinline__ A warp_sum(A v) {
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) v += __shfl_xor_sync(0xffffffffu, v, d);
  return v;
}

// Loads the lane's 8 values of row y (zero outside the image), squared if SQR.
template <int TYPE, typename A, bool SQR>
__device__ __forceinline__ void load_row(const IntegralParams& p, int c, int y,
                                         int xl, A (&v)[kPX]) {
  using ET = typename ElemOf<TYPE>::T;
  const ET* row = reinterpret_cast<const ET*>(p.src + (size_t)y * p.src_pitch);
#pragma unroll
  for (int k = 0; k < kPX; ++k) {
    const int x = xl + k;
    A a = A(0);
    if (x < p.W) a = (A)row[(size_t)x * p.nch + c];
    v[k] = SQR ? a * a : a;
  }
}

template <int TYPE, typename A, bool SQR>
__global__ void __launch_bounds__(32 * kWarpsPerCta)
    integral_reduce_kernel(const IntegralParams p) {
  const int lane = threadIdx.x & 31;
  const int tile = blockIdx.x * kWarpsPerCta + (threadIdx.x >> 5);
  const int c = blockIdx.y;
  if (tile >= p.nBX * p.nBY) return;
  const int bx = tile % p.nBX, by = tile / p.nBX;
  const int xl = bx * kTW + lane * kPX;
  const int y0 = by * kTH;
  A* rowsum = reinterpret_cast<A*>(p.rowsum) + (size_t)c * p.H * p.nBX;
  A* lb = reinterpret_cast<A*>(p.lb) + (size_t)c * p.nBY * p.W;
  A col[kPX];
#pragma unroll
  for (int k = 0; k < kPX; ++k) col[k] = A(0);
  const int yend = min(p.H, y0 + kTH);
  for (int y = y0; y < yend; ++y) {
    A v[kPX];
    load_row<TYPE, A, SQR>(p, c, y, xl, v);
    A s = A(0);
#pragma unroll
    for (int k = 0; k < kPX; ++k) {
      s += v[k];
      col[k] += v[k];
    }
    s = warp_sum(s);
    if (lane == 0) rowsum[(size_t)y * p.nBX + bx] = s;
  }
  // Tile-local prefix of the column sums along x = the tile's local integral
  // at its bottom row.
#pragma unroll
  for (int k = 1; k < kPX; ++k) col[k] += col[k - 1];
  const A incl = warp_incl_scan(col[kPX - 1], lane);
  const A excl = incl - col[kPX - 1];
#pragma unroll
  for (int k = 0; k < kPX; ++k)
    if (xl + k < p.W) lb[(size_t)by * p.W + xl + k] = excl + col[k];
}

// RowLeft (thread per row) and BandLeft (thread per band), both exclusive
// scans across the tiles of a row / band.
template <typename A>
__global__ void integral_junction_rows_kernel(const IntegralParams p) {
  const int c = blockIdx.y;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  A* rowsum = reinterpret_cast<A*>(p.rowsum) + (size_t)c * p.H * p.nBX;
  const A* lb = reinterpret_cast<const A*>(p.lb) + (size_t)c * p.nBY * p.W;
  A* bl = reinterpret_cast<A*>(p.bandleft) + (size_t)c * p.nBY * p.nBX;
  if (i < p.H) {
    A run = A(0);
    for (int bx = 0; bx < p.nBX; ++bx) {
      const A v = rowsum[(size_t)i * p.nBX + bx];
      rowsum[(size_t)i * p.nBX + bx] = run;
      run += v;
    }
  } else if (i < p.H + p.nBY) {
    const int by = i - p.H;
    A run = A(0);
    for (int bx = 0; bx < p.nBX; ++bx) {
      bl[(size_t)by * p.nBX + bx] = run;
      const int xe = min(p.W, (bx + 1) * kTW) - 1;
      run += lb[(size_t)by * p.W + xe];
    }
  }
}

// Top[by][x] = sum over bands above of (BandLeft + LB), in place over LB.
template <typename A>
__global__ void integral_junction_cols_kernel(const IntegralParams p) {
  const int c = blockIdx.y;
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= p.W) return;
  A* lb = reinterpret_cast<A*>(p.lb) + (size_t)c * p.nBY * p.W;
  const A* bl = reinterpret_cast<const A*>(p.bandleft) + (size_t)c * p.nBY * p.nBX;
  const int bx = x / kTW;
  A run = A(0);
  for (int by = 0; by < p.nBY; ++by) {
    const A v = bl[(size_t)by * p.nBX + bx] + lb[(size_t)by * p.W + x];
    lb[(size_t)by * p.W + x] = run;
    run += v;
  }
}

__device__ __forceinline__ float to_f32(long long v) { return __ll2float_rn(v); }
__device__ __forceinline__ float to_f32(double v) { return __double2float_rn(v); }
__device__ __forceinline__ double to_f64(long long v) { return __ll2double_rn(v); }
__device__ __forceinline__ double to_f64(double v) { return v; }

template <int TYPE, typename A, bool SQR>
__global__ void __launch_bounds__(32 * kWarpsPerCta)
    integral_final_kernel(const IntegralParams p) {
  const int lane = threadIdx.x & 31;
  const int tile = blockIdx.x * kWarpsPerCta + (threadIdx.x >> 5);
  const int c = blockIdx.y;
  if (tile >= p.nBX * p.nBY) return;
  const int bx = tile % p.nBX, by = tile / p.nBX;
  const int xl = bx * kTW + lane * kPX;
  const int y0 = by * kTH;
  const A* rowleft = reinterpret_cast<const A*>(p.rowsum) + (size_t)c * p.H * p.nBX;
  const A* top = reinterpret_cast<const A*>(p.lb) + (size_t)c * p.nBY * p.W;
  A acc[kPX];
#pragma unroll
  for (int k = 0; k < kPX; ++k)
    acc[k] = (xl + k < p.W) ? top[(size_t)by * p.W + xl + k] : A(0);
  const int yend = min(p.H, y0 + kTH);
  for (int y = y0; y < yend; ++y) {
    A v[kPX];
    load_row<TYPE, A, SQR>(p, c, y, xl, v);
#pragma unroll
    for (int k = 1; k < kPX; ++k) v[k] += v[k - 1];
    const A incl = warp_incl_scan(v[kPX - 1], lane);
    const A base = incl - v[kPX - 1] + rowleft[(size_t)y * p.nBX + bx];
    char* drow = p.dst + (size_t)y * p.dst_pitch;
#pragma unroll
    for (int k = 0; k < kPX; ++k) {
      acc[k] += base + v[k];
      const int x = xl + k;
      if (x < p.W) {
        if (p.dst_f64)
          reinterpret_cast<double*>(drow)[(size_t)x * p.nch + c] = to_f64(acc[k]);
        else
          reinterpret_cast<float*>(drow)[(size_t)x * p.nch + c] = to_f32(acc[k]);
      }
    }
  }
}

template <int TYPE, typename A, bool SQR>
cudaError_t run(IntegralParams& p, cudaStream_t st) {
  const int ntiles = p.nBX * p.nBY;
  dim3 g1((ntiles + kWarpsPerCta - 1) / kWarpsPerCta, p.nch);
  integral_reduce_kernel<TYPE, A, SQR><<<g1, 32 * kWarpsPerCta, 0, st>>>(p);
  dim3 g2((p.H + p.nBY + 127) / 128, p.nch);
  integral_junction_rows_kernel<A><<<g2, 128, 0, st>>>(p);
  dim3 g3((p.W + 127) / 128, p.nch);
  integral_junction_cols_kernel<A><<<g3, 128, 0, st>>>(p);
  integral_final_kernel<TYPE, A, SQR><<<g1, 32 * kWarpsPerCta, 0, st>>>(p);
  count_launches(4);
  return cudaGetLastError();
}

template <int TYPE, typename AI>
cudaError_t run_sqr(bool sqr, IntegralParams& p, cudaStream_t st) {
  return sqr ? run<TYPE, AI, true>(p, st) : run<TYPE, AI, false>(p, st);
}

}  // namespace

size_t integral_scratch_bytes(int width, int height, int nch) {
  const size_t nBX = (width + kTW - 1) / kTW, nBY = (height + kTH - 1) / kTH;
  return 8 * (size_t)nch * ((size_t)height * nBX + nBY * (size_t)width + nBY * nBX) + 256;
}

cudaError_t launch_integral(bool sqr, const DevImage& src, const DevImage& dst,
                            void* scratch, size_t scratch_bytes,
                            cudaStream_t st) {
  IntegralParams p;
  p.src = (const char*)src.ptr;
  p.src_pitch = src.pitch;
  p.dst = (char*)dst.ptr;
  p.dst_pitch = dst.pitch;
  p.dst_f64 = dst.type == F64;
  p.W = src.width;
  p.H = src.height;
  p.nch = src.nch;
  p.nBX = (p.W + kTW - 1) / kTW;
  p.nBY = (p.H + kTH - 1) / kTH;
  if (scratch_bytes < integral_scratch_bytes(p.W, p.H, p.nch)) return cudaErrorInvalidValue;
  char* s = (char*)scratch;
  p.rowsum = s;
  s += 8 * (size_t)p.nch * p.H * p.nBX;
  p.lb = s;
  s += 8 * (size_t)p.nch * p.nBY * p.W;
  p.bandleft = s;
  switch (src.type) {
    case U8: return run_sqr<U8, long long>(sqr, p, st);
    case S8: return run_sqr<S8, long long>(sqr, p, st);
    case U16: return run_sqr<U16, long long>(sqr, p, st);
    case S16: return run_sqr<S16, long long>(sqr, p, st);
    case U32:
      return sqr ? run<U32, double, true>(p, st) : run<U32, long long, false>(p, st);
    case S32:
      return sqr ? run<S32, double, true>(p, st) : run<S32, long long, false>(p, st);
    case F32: return run_sqr<F32, double>(sqr, p, st);
    case F64: return run_sqr<F64, double>(sqr, p, st);
  }
  return cudaErrorInvalidValue;
}

}  // namespace ocipb

// ---- Integral without device allocation -------------------------------------
//
// Some callers cannot let a library allocate device memory: their device
// memory is owned by another allocator (a framework's memory pool that holds
// the whole budget), or they must not allocate once running, because
// cudaMalloc/cudaFree can block and synchronise the whole device (for example
// latency-bound video pipelines). ocipIntegralNoAlloc serves them: the scan's
// scratch lives in the fixed array below, reserved when the library is loaded
// on a device and held by every device that loads the library until the
// process exits.

namespace ocipb {
namespace {

// Largest scratch the allocation-free entry point can use: 8 MiB, enough for
// one channel up to about 6000 x 6000 pixels (integral_scratch_bytes()).
constexpr size_t kNoAllocScratchBytes = size_t(8) << 20;
__device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
void* g_noalloc_addr[kMaxDevices] = {};

// The device address of g_noalloc_scratch on the current device. Host code
// cannot use the array's name as a device address; cudaGetSymbolAddress gives
// the real one, once per device (on the first call made on that device).
cudaError_t noalloc_scratch(int dev, void** ptr) {
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  if (g_noalloc_addr[dev] == nullptr) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    g_noalloc_addr[dev] = p;
  }
  *ptr = g_noalloc_addr[dev];
  return cudaSuccess;
}

}  // namespace
}  // namespace ocipb

#include <string>

#include "../../include/OpenCLIPP.h"
#include "../../include/OpenCLIPP_B200.h"
#include "host.h"

extern "C" ocipError ocipIntegralNoAlloc(int Square, SImage SourceDesc, const void* Source,
                                         size_t SourcePitch, SImage DestDesc, void* Dest,
                                         size_t DestPitch, void* Stream) {
  using namespace ocipb;
  OCIP_GUARD(
    if (Source == nullptr || Dest == nullptr) fail(CL_INVALID_MEM_OBJECT, "NULL image pointer");
    if ((int)SourceDesc.Type < 0 || (int)SourceDesc.Type >= (int)SImage::NbDataTypes ||
        SourceDesc.Channels < 1 || SourceDesc.Channels > 4)
      fail(CL_IMAGE_FORMAT_NOT_SUPPORTED, "unsupported source format");
    if (DestDesc.Type != SImage::F32 && DestDesc.Type != SImage::F64)
      fail(CL_INVALID_VALUE, "Destination image of Integral must be F32 or F64");
    if (SourceDesc.Width != DestDesc.Width || SourceDesc.Height != DestDesc.Height)
      fail(CL_INVALID_IMAGE_SIZE, "Different image sizes used");
    if (SourceDesc.Channels != DestDesc.Channels)
      fail(CL_INVALID_VALUE, "Different number of channels used");
    if (SourceDesc.Width == 0 || SourceDesc.Height == 0)
      fail(CL_INVALID_BUFFER_SIZE, "empty image");
    if (SourcePitch < (size_t)SourceDesc.Width * SourceDesc.Channels * type_bytes((int)SourceDesc.Type) ||
        DestPitch < (size_t)DestDesc.Width * DestDesc.Channels * type_bytes((int)DestDesc.Type))
      fail(CL_INVALID_VALUE, "pitch smaller than one row of pixels");
    const size_t need = integral_scratch_bytes((int)SourceDesc.Width, (int)SourceDesc.Height,
                                               (int)SourceDesc.Channels);
    if (need > kNoAllocScratchBytes)
      fail(CL_INVALID_IMAGE_SIZE,
           "image too large for ocipIntegralNoAlloc: needs " + std::to_string(need) +
               " bytes of scratch, the fixed limit is " + std::to_string(kNoAllocScratchBytes));
    int dev = 0;
    check_cuda(cudaGetDevice(&dev), "cudaGetDevice");
    void* scratch = nullptr;
    check_cuda(noalloc_scratch(dev, &scratch), "cudaGetSymbolAddress");
    DevImage s, d;
    s.ptr = const_cast<void*>(Source);
    s.pitch = SourcePitch;
    s.width = (int)SourceDesc.Width;
    s.height = (int)SourceDesc.Height;
    s.nch = (int)SourceDesc.Channels;
    s.type = (int)SourceDesc.Type;
    d.ptr = Dest;
    d.pitch = DestPitch;
    d.width = (int)DestDesc.Width;
    d.height = (int)DestDesc.Height;
    d.nch = (int)DestDesc.Channels;
    d.type = (int)DestDesc.Type;
    check_cuda(launch_integral(Square != 0, s, d, scratch, kNoAllocScratchBytes,
                               reinterpret_cast<cudaStream_t>(Stream)),
               "integral kernel launch");
  )
}
