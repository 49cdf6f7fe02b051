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
// R is stored as FP32 for F32 and U16 sources (a difference of FP64 prefix
// sums rounded once: relative error 2^-24; an FP64 running sum of FP32
// values adds and later removes each value exactly) and as int32 for U8
// sources (exact). Bound: HBM (the source read once, 4 bytes written per
// output column and source row).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <type_traits>

#include "internal.h"
#include "row_energy.h"

namespace ocipb {
namespace {

constexpr int kWarps = 8;        // one row segment per warp
constexpr int kSeg = 256;        // output columns per segment (8 per lane)
constexpr int kMaxTw = 1024;  // 256 + tw - 1 <= 32 * 41

struct RowEnergyParams {
  const char* src;
  size_t src_pitch;
  char* dst;
  size_t dst_pitch;   // bytes
  size_t dst_plane;   // bytes between channel planes
  int W, H, nch;
  int tw, ax;
};

template <typename ET>
struct RowSumOf {
  // Prefix sums, exact for integers: int32 for 8-bit sources (at most
  // 1279 * 255^2 < 2^31), FP64 otherwise (16-bit: below 2^53; F32: squares
  // exact, sums rounded in FP64).
  typedef typename std::conditional<sizeof(ET) == 1, int, double>::type A;
  // Stored: int32 for 8-bit sources, FP32 otherwise.
  typedef typename std::conditional<sizeof(ET) == 1, int, float>::type R;
};

// One warp per (source row, 256 output columns). The squares of the n =
// 256 + tw - 1 source pixels the segment's windows cover are staged in
// shared memory (coalesced loads); lane l turns its K contiguous entries
// into prefix sums (local prefix plus a warp scan of the lanes' totals),
// P(i) = sum of squares [0, i) stored at entry i - 1; output column x0 + j
// (j = lane + 32 u) is then P(j + tw) - P(j): two conflict-free reads, and
// the warp's stores are 128-byte rows.
template <typename ET, int K>
__global__ void __launch_bounds__(kWarps * 32) row_energy_kernel(const RowEnergyParams p) {
  typedef typename RowSumOf<ET>::A A;
  typedef typename RowSumOf<ET>::R RT;
  extern __shared__ __align__(16) unsigned char smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int r = blockIdx.y * kWarps + warp;
  if (r >= p.H) return;  // whole warp
  const int c = blockIdx.z;
  const int x0 = blockIdx.x * kSeg;
  A* buf = reinterpret_cast<A*>(smem) + warp * (32 * K);
  const ET* row = reinterpret_cast<const ET*>(p.src + (size_t)r * p.src_pitch) + c;
  const int n = kSeg + p.tw - 1;
  const int xs0 = x0 - p.ax;
  // Squares of source columns xs0 .. xs0 + n - 1 (zero outside the image).
#pragma unroll 4
  for (int i = lane; i < 32 * K; i += 32) {
    const int x = xs0 + i;
    A v = A(0);
    if (i < n && x >= 0 && x < p.W) {
      const A e = static_cast<A>(row[x * p.nch]);
      v = e * e;
    }
    buf[i] = v;
  }
  __syncwarp();
  // Lane l: entries K l .. K l + K - 1 -> inclusive prefix sums in place.
  A loc[K];
  A tot = A(0);
#pragma unroll
  for (int k = 0; k < K; ++k) {
    tot += buf[K * lane + k];
    loc[k] = tot;
  }
  A incl = tot;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const A o = __shfl_up_sync(0xffffffffu, incl, d);
    if (lane >= d) incl += o;
  }
  const A excl = incl - tot;
  __syncwarp();
#pragma unroll
  for (int k = 0; k < K; ++k) buf[K * lane + k] = excl + loc[k];
  __syncwarp();
  RT* dst = reinterpret_cast<RT*>(p.dst + c * p.dst_plane + (size_t)r * p.dst_pitch);
#pragma unroll
  for (int u = 0; u < kSeg / 32; ++u) {
    const int j = lane + 32 * u;
    const int x = x0 + j;
    if (x < p.W) {
      const A hi = buf[j + p.tw - 1];
      const A lo = j > 0 ? buf[j - 1] : A(0);
      dst[x] = static_cast<RT>(hi - lo);
    }
  }
}

// One-channel form: the segment's source pixels are staged raw with 16-byte
// loads (from the 16-byte group at or below its first pixel, so `sh` pixels
// lead), squared and prefix-summed in registers, and only the prefix sums
// are written back for the differences. Same sums, in the same order, as
// row_energy_kernel.
template <typename ET, int K>
__global__ void __launch_bounds__(kWarps * 32) row_energy_vec_kernel(const RowEnergyParams p) {
  typedef typename RowSumOf<ET>::A A;
  typedef typename RowSumOf<ET>::R RT;
  constexpr int kInner = 16 / (int)sizeof(ET);                      // pixels per group
  constexpr int kRawGroups = (32 * K + kInner - 1) / kInner + 1;     // covers sh + 32 K
  extern __shared__ __align__(16) unsigned char smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int r = blockIdx.y * kWarps + warp;
  if (r >= p.H) return;  // whole warp
  const int x0 = blockIdx.x * kSeg;
  A* buf = reinterpret_cast<A*>(smem) + warp * (32 * K);
  ET* raw = reinterpret_cast<ET*>(smem + (size_t)kWarps * 32 * K * sizeof(A)) +
            warp * (kRawGroups * kInner);
  const ET* row = reinterpret_cast<const ET*>(p.src + (size_t)r * p.src_pitch);
  const int n = kSeg + p.tw - 1;
  const int xs0 = x0 - p.ax;
  const int xa = xs0 >= 0 ? xs0 - xs0 % kInner : -((-xs0 + kInner - 1) / kInner) * kInner;
  const int sh = xs0 - xa;
  // Raw pixels xa .. xa + kRawGroups * kInner - 1, zero outside the image:
  // whole groups inside the row with one 16-byte load, the rest per pixel.
  for (int g = lane; g < kRawGroups; g += 32) {
    const int x = xa + g * kInner;
    uint4 v;
    if (x >= 0 && x + kInner <= p.W) {
      v = __ldg(reinterpret_cast<const uint4*>(row + x));
    } else {
      ET e[kInner];
#pragma unroll
      for (int i = 0; i < kInner; ++i) e[i] = (x + i >= 0 && x + i < p.W) ? row[x + i] : ET(0);
      memcpy(&v, e, sizeof(v));
    }
    reinterpret_cast<uint4*>(raw)[g] = v;
  }
  __syncwarp();
  // Lane l: staged entries K l .. K l + K - 1 (pixel xs0 + i is raw[sh + i]).
  A loc[K];
  A tot = A(0);
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const int i = K * lane + k;
    const A e = i < n ? static_cast<A>(raw[sh + i]) : A(0);
    tot += e * e;
    loc[k] = tot;
  }
  A incl = tot;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const A o = __shfl_up_sync(0xffffffffu, incl, d);
    if (lane >= d) incl += o;
  }
  const A excl = incl - tot;
#pragma unroll
  for (int k = 0; k < K; ++k) buf[K * lane + k] = excl + loc[k];
  __syncwarp();
  RT* dst = reinterpret_cast<RT*>(p.dst + (size_t)r * p.dst_pitch);
#pragma unroll
  for (int u = 0; u < kSeg / 32; ++u) {
    const int j = lane + 32 * u;
    const int x = x0 + j;
    if (x < p.W) {
      const A hi = buf[j + p.tw - 1];
      const A lo = j > 0 ? buf[j - 1] : A(0);
      dst[x] = static_cast<RT>(hi - lo);
    }
  }
}

template <typename ET, int K>
cudaError_t launch_k(const RowEnergyParams& p, cudaStream_t st) {
  typedef typename RowSumOf<ET>::A A;
  if (p.nch == 1 && (p.src_pitch % 16) == 0 && ((uintptr_t)p.src % 16) == 0) {
    constexpr int kInner = 16 / (int)sizeof(ET);
    constexpr int kRawGroups = (32 * K + kInner - 1) / kInner + 1;
    const size_t smem = (size_t)kWarps * (32 * K * sizeof(A) + kRawGroups * 16);
    auto kern = row_energy_vec_kernel<ET, K>;
    if (smem > 48 * 1024) {
      const cudaError_t e =
          cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      if (e != cudaSuccess) return e;
    }
    dim3 grid((p.W + kSeg - 1) / kSeg, (p.H + kWarps - 1) / kWarps, 1);
    kern<<<grid, kWarps * 32, smem, st>>>(p);
    count_launches(1);
    return cudaGetLastError();
  }
  const size_t smem = (size_t)kWarps * 32 * K * sizeof(A);
  auto kern = row_energy_kernel<ET, K>;
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

template <typename ET>
cudaError_t launch_typed(const RowEnergyParams& p, cudaStream_t st) {
  // K: staged entries per lane, 32 K >= 256 + tw - 1.
  const int n = kSeg + p.tw - 1;
  if (n <= 32 * 9) return launch_k<ET, 9>(p, st);
  if (n <= 32 * 11) return launch_k<ET, 11>(p, st);
  if (n <= 32 * 17) return launch_k<ET, 17>(p, st);
  return launch_k<ET, 41>(p, st);
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
  switch (src.type) {
    case U8: return launch_typed<uint8_t>(p, stream);
    case U16: return launch_typed<uint16_t>(p, stream);
    case F32: return launch_typed<float>(p, stream);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace ocipb
