// Index reductions of score maps: ocipMinIndx, ocipMaxIndx, ocipMinAbsIndx,
// ocipMaxAbsIndx (include/OpenCLIPP.h:560-563), the natural consumer of a
// template-matching map (best match = arg-min of SqrDistance, arg-max of
// CrossCorr_Norm).
//
// Same result as the reference, ties and NaNs included, by doing the same
// comparisons in the same order (cl-files/Statistics.cl :326-500, REDUCE_POS;
// C++/programs/StatisticsHelpers.cpp :105-146, ReduceMin / ReduceMax):
//   * one CTA per reference work-group of 16 x 16 work-items covering a
//     256 x 16 pixel rectangle; work-item (lx, ly) reads the 16 pixels
//     x = 256 gx + lx + 16 i, i = 0..15, of row 16 gy + ly and keeps the first
//     one that no later one beats strictly (compare in the source type, after
//     fabs / abs for the Abs forms);
//   * the CTA folds work-item lid + s into lid for s = 128, 64, ..., 1 (the
//     reference's tree), replacing only on a strict win and only between valid
//     work-items;
//   * each group's winner is stored as float with its (x, y), and the host
//     folds the groups in group order with a strict comparison, starting from
//     group 0, and returns that float as a double.
// One memory-bound pass over the map; the group results (12 bytes per 4096
// pixels) are read back and folded on the host, as the reference does.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <type_traits>
#include <vector>

#include "host.h"
#include "internal.h"
#include "statistics.h"

namespace ocipb {
namespace {

template <int TYPE> struct ElemOf;
template <> struct ElemOf<U8> { typedef uint8_t T; };
template <> struct ElemOf<S8> { typedef int8_t T; };
template <> struct ElemOf<U16> { typedef uint16_t T; };
template <> struct ElemOf<S16> { typedef int16_t T; };
template <> struct ElemOf<U32> { typedef uint32_t T; };
template <> struct ElemOf<S32> { typedef int32_t T; };
template <> struct ElemOf<F32> { typedef float T; };
template <> struct ElemOf<F64> { typedef double T; };

// Values are compared in a type that holds every source value exactly
// (int for 8/16-bit, long long for 32-bit integers, the float type itself).
template <typename T>
struct CmpOf {
  typedef typename std::conditional<
      std::is_floating_point<T>::value, T,
      typename std::conditional<(sizeof(T) < 4), int, long long>::type>::type type;
};

// Source value after the reference's pre-operation, widened. OpenCL abs()
// returns the unsigned type of the same width and the reference stores it
// back in the source type (Statistics.cl REDUCE_POS, `type Res`), so abs of
// the most negative value wraps to itself.
template <typename T, bool ABS>
__device__ __forceinline__ typename CmpOf<T>::type load_op(T v) {
  typedef typename CmpOf<T>::type C;
  if constexpr (!ABS) {
    return static_cast<C>(v);
  } else if constexpr (std::is_floating_point<T>::value) {
    return fabs(v);
  } else if constexpr (std::is_signed<T>::value) {
    // Two's-complement abs on the bits (in the unsigned type of the same
    // width), then the bits read as a signed value of that width.
    constexpr int kBits = 8 * sizeof(T);
    typedef typename std::make_unsigned<T>::type U;
    const U u = static_cast<U>(v);
    const U neg = static_cast<U>(u >> (kBits - 1));
    const U absu = static_cast<U>(static_cast<U>(u ^ static_cast<U>(U(0) - neg)) + neg);
    C r = static_cast<C>(absu);
    if ((absu >> (kBits - 1)) & 1u) r -= static_cast<C>(1) << kBits;
    return r;
  } else {
    return static_cast<C>(v);
  }
}

template <int OP, typename C>
__device__ __forceinline__ bool wins(C a, C b) {  // a replaces b
  return (OP == kIdxMin || OP == kIdxMinAbs) ? (a < b) : (a > b);
}

template <int TYPE, int OP>
__global__ void __launch_bounds__(256) index_reduce_kernel(const char* src, size_t pitch, int W,
                                                           int H, float* out_val,
                                                           int2* out_coord) {
  typedef typename ElemOf<TYPE>::T T;
  typedef typename CmpOf<T>::type C;
  constexpr bool kAbs = (OP == kIdxMinAbs || OP == kIdxMaxAbs);
  __shared__ C buffer[256];
  __shared__ int2 coords[256];
  __shared__ int valid[256];
  const int lx = threadIdx.x & 15, ly = threadIdx.x >> 4;
  const int lid = threadIdx.x;
  const int gx = blockIdx.x * 256 + lx;
  const int gy = blockIdx.y * 16 + ly;
  if (gx < W && gy < H) {
    const T* row = reinterpret_cast<const T*>(src + (size_t)gy * pitch);
    C res = load_op<T, kAbs>(row[gx]);
    int2 c = make_int2(gx, gy);
    for (int i = 16; i < 256; i += 16) {
      if (gx + i < W) {
        const C px = load_op<T, kAbs>(row[gx + i]);
        if (wins<OP>(px, res)) {
          res = px;
          c.x = gx + i;
        }
      }
    }
    buffer[lid] = res;
    coords[lid] = c;
    valid[lid] = 1;
  } else {
    valid[lid] = 0;
  }
  __syncthreads();
#pragma unroll
  for (int s = 128; s >= 1; s >>= 1) {
    if (lid < s && valid[lid] && valid[lid + s] && wins<OP>(buffer[lid + s], buffer[lid])) {
      buffer[lid] = buffer[lid + s];
      coords[lid] = coords[lid + s];
    }
    __syncthreads();
  }
  if (lid == 0) {
    const int gid = blockIdx.y * gridDim.x + blockIdx.x;
    out_val[gid] = static_cast<float>(buffer[0]);
    out_coord[gid] = coords[0];
  }
}

template <int TYPE>
cudaError_t launch_typed(int op, const DevImage& s, float* val, int2* coord, dim3 grid,
                         cudaStream_t st) {
  const char* p = (const char*)s.ptr;
  switch (op) {
    case kIdxMin: index_reduce_kernel<TYPE, kIdxMin><<<grid, 256, 0, st>>>(p, s.pitch, s.width, s.height, val, coord); break;
    case kIdxMax: index_reduce_kernel<TYPE, kIdxMax><<<grid, 256, 0, st>>>(p, s.pitch, s.width, s.height, val, coord); break;
    case kIdxMinAbs: index_reduce_kernel<TYPE, kIdxMinAbs><<<grid, 256, 0, st>>>(p, s.pitch, s.width, s.height, val, coord); break;
    default: index_reduce_kernel<TYPE, kIdxMaxAbs><<<grid, 256, 0, st>>>(p, s.pitch, s.width, s.height, val, coord); break;
  }
  count_launches(1);
  return cudaGetLastError();
}

}  // namespace

size_t index_reduce_scratch_bytes(int W, int H) {
  const size_t groups = (size_t)((W + 255) / 256) * ((H + 15) / 16);
  return groups * (sizeof(float) + sizeof(int2)) + 256;
}

cudaError_t index_reduce(Context& ctx, int op, const DevImage& s, void* scratch, double* value,
                         int* x, int* y) {
  const dim3 grid((s.width + 255) / 256, (s.height + 15) / 16);
  const size_t groups = (size_t)grid.x * grid.y;
  float* val = reinterpret_cast<float*>(scratch);
  int2* coord = reinterpret_cast<int2*>(reinterpret_cast<char*>(scratch) +
                                        (groups * sizeof(float) + 15) / 16 * 16);
  cudaError_t e = cudaSuccess;
  switch (s.type) {
    case U8: e = launch_typed<U8>(op, s, val, coord, grid, ctx.stream); break;
    case S8: e = launch_typed<S8>(op, s, val, coord, grid, ctx.stream); break;
    case U16: e = launch_typed<U16>(op, s, val, coord, grid, ctx.stream); break;
    case S16: e = launch_typed<S16>(op, s, val, coord, grid, ctx.stream); break;
    case U32: e = launch_typed<U32>(op, s, val, coord, grid, ctx.stream); break;
    case S32: e = launch_typed<S32>(op, s, val, coord, grid, ctx.stream); break;
    case F32: e = launch_typed<F32>(op, s, val, coord, grid, ctx.stream); break;
    default: e = launch_typed<F64>(op, s, val, coord, grid, ctx.stream); break;
  }
  if (e != cudaSuccess) return e;
  std::vector<float> hv(groups);
  std::vector<int2> hc(groups);
  e = cudaMemcpyAsync(hv.data(), val, groups * sizeof(float), cudaMemcpyDeviceToHost, ctx.stream);
  if (e != cudaSuccess) return e;
  e = cudaMemcpyAsync(hc.data(), coord, groups * sizeof(int2), cudaMemcpyDeviceToHost, ctx.stream);
  if (e != cudaSuccess) return e;
  e = cudaStreamSynchronize(ctx.stream);
  if (e != cudaSuccess) return e;
  // Host fold in group order, strict comparison (StatisticsHelpers.cpp:105-146).
  const bool is_min = (op == kIdxMin || op == kIdxMinAbs);
  float v = hv[0];
  int bx = hc[0].x, by = hc[0].y;
  for (size_t i = 0; i < groups; ++i) {
    if (is_min ? (hv[i] < v) : (hv[i] > v)) {
      v = hv[i];
      bx = hc[i].x;
      by = hc[i].y;
    }
  }
  *value = v;
  *x = bx;
  *y = by;
  return cudaSuccess;
}

}  // namespace ocipb
