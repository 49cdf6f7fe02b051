// Row energies of the ImageProximity windows, for the tensor-core path.
//
// R(x, r, c) = sum_{w < tw} S(x + w - ax, r, c)^2 (zero outside the image):
// the energy of the template-wide row segment of source row r that output
// column x's window covers. The window energy of output (x, y) -- the
// counterpart of the reference's AreaSqSum over a SqrIntegral
// (cl-files/ImageProximityFFT.cl:55-84) and of the sum S^2 accumulator of
// the direct _Norm kernels (cl-files/ImageProximity.cl:122-211, 375-466) --
// is then the sum of R over the th rows y - ay .. y - ay + th - 1, which the
// tensor kernel's epilogue keeps as a running FP64 sum while it walks down
// the rows. Rows are independent here, so every warp streams its own row
// segment with all its loads in flight.
//
// R is stored as FP32 for F32 and U16 sources (an FP64 sum rounded once:
// relative error 2^-24; an FP64 running sum of FP32 values adds and later
// removes each value exactly) and as int32 for U8 sources (exact: at most
// 1024 * 255^2 < 2^31). Bound: HBM (the source read once, 4 bytes written per
// output column and source row).
#include <cuda_runtime.h>

#include <algorithm>
#include <type_traits>

#include "internal.h"
#include "row_energy.h"

namespace ocipb {
namespace {

constexpr int kWarps = 8;        // one row segment per warp
constexpr int kSeg = 256;        // output columns per segment (8 per lane)
constexpr int kMaxTw = 1024;

struct RowEnergyParams {
  const char* src;
  size_t src_pitch;
  char* dst;
  size_t dst_pitch;   // bytes
  size_t dst_plane;   // bytes between channel planes
  int W, H, nch;
  int tw, ax;
  int buf;            // shared-memory entries per warp
};

template <typename ET>
struct RowSumOf {
  // Exact accumulation: int64 for integers, FP64 for floats.
  typedef typename std::conditional<std::is_integral<ET>::value, long long, double>::type A;
  // Stored: int32 for 8-bit sources, FP32 otherwise.
  typedef typename std::conditional<sizeof(ET) == 1, int, float>::type R;
};

// Shared-memory slot of element i of a warp's buffer: one pad slot after
// every 8, so that lanes reading runs 8 apart fall in different banks.
__device__ __forceinline__ int rpad(int i) { return i + (i >> 3); }

template <typename ET>
__global__ void __launch_bounds__(kWarps * 32) row_energy_kernel(const RowEnergyParams p) {
  typedef typename RowSumOf<ET>::A A;
  typedef typename RowSumOf<ET>::R RT;
  extern __shared__ __align__(16) unsigned char smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int r = blockIdx.y * kWarps + warp;
  if (r >= p.H) return;  // whole warp
  const int c = blockIdx.z;
  const int x0 = blockIdx.x * kSeg;
  A* buf = reinterpret_cast<A*>(smem) + warp * p.buf;
  // Squares of source columns x0 - ax .. x0 - ax + kSeg + tw - 2, coalesced.
  const ET* row = reinterpret_cast<const ET*>(p.src + (size_t)r * p.src_pitch);
  const int n = kSeg + p.tw - 1;
  const int xs0 = x0 - p.ax;
  constexpr int U = 4;  // loads issued before any is used
  for (int i0 = 0; i0 < n; i0 += 32 * U) {
    ET v[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int i = i0 + u * 32 + lane;
      const int x = xs0 + i;
      v[u] = (i < n && x >= 0 && x < p.W) ? row[(size_t)x * p.nch + c] : ET(0);
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int i = i0 + u * 32 + lane;
      if (i < n) {
        const A a = static_cast<A>(v[u]);
        buf[rpad(i)] = a * a;
      }
    }
  }
  __syncwarp();
  const int xl = x0 + 8 * lane;
  if (xl >= p.W) return;
  A e = A(0);
  for (int w = 0; w < p.tw; ++w) e += buf[rpad(8 * lane + w)];
  RT o[8];
  o[0] = static_cast<RT>(e);
#pragma unroll
  for (int i = 1; i < 8; ++i) {
    e += buf[rpad(8 * lane + i - 1 + p.tw)] - buf[rpad(8 * lane + i - 1)];
    o[i] = static_cast<RT>(e);
  }
  RT* dst = reinterpret_cast<RT*>(p.dst + c * p.dst_plane + (size_t)r * p.dst_pitch) + xl;
  if (xl + 8 <= p.W) {
    reinterpret_cast<uint4*>(dst)[0] = *reinterpret_cast<const uint4*>(&o[0]);
    reinterpret_cast<uint4*>(dst)[1] = *reinterpret_cast<const uint4*>(&o[4]);
  } else {
    for (int i = 0; i < 8 && xl + i < p.W; ++i) dst[i] = o[i];
  }
}

template <typename ET>
cudaError_t launch_typed(RowEnergyParams p, cudaStream_t st) {
  typedef typename RowSumOf<ET>::A A;
  const int n = kSeg + p.tw - 1;
  p.buf = n + (n >> 3) + 1;
  const size_t smem = (size_t)kWarps * p.buf * sizeof(A);
  auto kern = row_energy_kernel<ET>;
  if (smem > 48 * 1024) {
    const cudaError_t e =
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  dim3 grid((p.W + kSeg - 1) / kSeg, (p.H + kWarps - 1) / kWarps, p.nch);
  kern<<<grid, kWarps * 32, smem, st>>>(p);
  count_launches(1);
  return cudaGetLastError();
}

}  // namespace

size_t row_energy_pitch(int width) { return ((size_t)width * 4 + 127) / 128 * 128; }

cudaError_t launch_row_energy(const DevImage& src, int tw, int ax, void* dst, size_t dst_pitch,
                              size_t dst_plane, cudaStream_t stream) {
  if (tw < 1 || tw > kMaxTw) return cudaErrorInvalidValue;
  RowEnergyParams p;
  p.src = (const char*)src.ptr;
  p.src_pitch = src.pitch;
  p.dst = (char*)dst;
  p.dst_pitch = dst_pitch;
  p.dst_plane = dst_plane;
  p.W = src.width;
  p.H = src.height;
  p.nch = src.nch;
  p.tw = tw;
  p.ax = ax;
  p.buf = 0;
  switch (src.type) {
    case U8: return launch_typed<uint8_t>(p, stream);
    case U16: return launch_typed<uint16_t>(p, stream);
    case F32: return launch_typed<float>(p, stream);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace ocipb
