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
// Layout: the image is cut into 128 x 32 tiles, one warp per tile (lane l
// holds 4 consecutive columns, so one vector load of a warp reads 128
// contiguous pixels when the image allows it). On that vector path the tile's
// rows stream through a per-lane cp.async ring in shared memory (RowStream);
// other layouts load groups of rows into registers. The kernels stay within
// 64 registers so that 32 warps share an SM: a 4096 x 4096 image is 4096
// tiles, all resident at once on 148 SMs. Three launches:
//   1. tile reduce (reads the source): per-row tile sums (RowSum) and the
//      tile's local integral at its bottom row (LB) -- the counterpart of the
//      reference's vertical/horizontal junction buffers;
//   2. junctions, one launch with two kinds of blocks: blocks of 32 columns
//      turn LB into ColTop (exclusive scan of LB over the bands), and warps
//      turn RowSum into RowLeft (exclusive scan across the tiles of a row);
//   3. final (reads the source again, mostly from L2): D = Top + running sum
//      over the band's rows of (RowLeft + warp-scanned row prefix), where the
//      integral of the row above the band is Top(x) = ColTop(x) + the sum of
//      ColTop at the last column of every tile left of x (LB at a tile's last
//      column is the tile's total, so that sum is the integral of the tiles
//      left of this one over the bands above).
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstring>
#include <map>
#include <mutex>
#include <set>
#include <utility>

#include "internal.h"

namespace ocipb {
namespace {

constexpr int kTW = 128;   // tile width (32 lanes x 4 columns)
constexpr int kTH = 32;    // tile height
constexpr int kPX = 4;     // columns per lane
constexpr int kWarpsPerCta = 4;
constexpr int kMinCtas = 8;      // 32 warps per SM: at most 64 registers
constexpr int kJThreads = 256;   // junction blocks
constexpr int kJCols = 32;       // columns per ColTop block
constexpr int kJBands = 16;      // bands per thread and chunk step in a ColTop block
constexpr int kJRows = 8;        // image rows per warp in a RowLeft block

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
  int vec_src;     // 1: one channel, 16-byte aligned base and pitch
  int vec_dst;     // 1: one channel, base and pitch aligned to a lane's 4 pixels
  void* rowsum;    // [nch][H][nBX]     RowSum, then RowLeft
  void* lb;        // [nch][nBY][W]     LB, then ColTop
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

// Totals of G rows across the warp with G - 1 + log2(32 / G) shuffles instead
// of 5 G: at each halving step a lane keeps the half of its rows selected by
// its lane bit and adds the partner's copy of them. On return every lane
// holds the total of row (lane >> (5 - log2 G)). G is a power of two <= 32.
template <int G, typename A>
__device__ __forceinline__ A warp_sum_rows(A (&s)[G], int lane) {
#pragma unroll
  for (int lvl = 0; (G >> lvl) > 1; ++lvl) {
    const int o = 16 >> lvl;
    constexpr int kMax = G / 2;
    const bool upper = (lane & o) != 0;
#pragma unroll
    for (int i = 0; i < kMax; ++i) {
      if (i < (G >> lvl) / 2) {
        const int h = (G >> lvl) / 2;
        const A send = upper ? s[i] : s[i + h];
        const A keep = upper ? s[i + h] : s[i];
        s[i] = keep + __shfl_xor_sync(0xffffffffu, send, o);
      }
    }
  }
  A v = s[0];
#pragma unroll
  for (int o = 16 / G; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

template <int G>
__host__ __device__ constexpr int log2_of() { return G <= 1 ? 0 : 1 + log2_of<G / 2>(); }

// Rows whose tile sums one multi-row warp reduction combines in the reduce
// pass (8, or 4 for 8-byte types); the register paths load a group of rows
// before they use any of them.
template <typename ET>
__host__ __device__ constexpr int group_rows() { return sizeof(ET) >= 8 ? 4 : 8; }

// The lane's 4 source values of a row, as one vector load (two for 8-byte
// types): the row is 16-byte aligned and the 4 columns are inside the image.
template <typename ET>
__device__ __forceinline__ void load_vec(const ET* row, int xl, ET (&e)[kPX]) {
  if constexpr (sizeof(ET) == 1) {
    const uint32_t q = *reinterpret_cast<const uint32_t*>(row + xl);
    memcpy(e, &q, sizeof(q));
  } else if constexpr (sizeof(ET) == 2) {
    const uint2 q = *reinterpret_cast<const uint2*>(row + xl);
    memcpy(e, &q, sizeof(q));
  } else {
    constexpr int NQ = sizeof(ET) * kPX / 16;
    uint4 q[NQ];
#pragma unroll
    for (int i = 0; i < NQ; ++i) q[i] = reinterpret_cast<const uint4*>(row + xl)[i];
    memcpy(e, q, sizeof(q));
  }
}

// The lane's 4 source values of row y, zero outside the image.
template <typename ET>
__device__ __forceinline__ void load_raw(const IntegralParams& p, int c, int y, int xl,
                                         ET (&e)[kPX]) {
  const ET* row = reinterpret_cast<const ET*>(p.src + (size_t)y * p.src_pitch);
  if (p.vec_src && xl + kPX <= p.W) {
    load_vec(row, xl, e);
    return;
  }
#pragma unroll
  for (int k = 0; k < kPX; ++k) {
    const int x = xl + k;
    e[k] = x < p.W ? row[(size_t)x * p.nch + c] : ET(0);
  }
}

// Rows yg .. yg + G - 1 of the lane's columns (zero from row yend on). When
// the whole group lies inside the image and the tile's columns are vector
// loadable (both warp-uniform), the G loads are issued back to back.
template <int G, typename ET>
__device__ __forceinline__ void load_group(const IntegralParams& p, int c, int yg, int yend,
                                           int xl, bool vec_tile, ET (&raw)[G][kPX]) {
  if (vec_tile && yg + G <= yend) {
    const char* base = p.src + (size_t)yg * p.src_pitch;
#pragma unroll
    for (int r = 0; r < G; ++r)
      load_vec(reinterpret_cast<const ET*>(base + (size_t)r * p.src_pitch), xl, raw[r]);
    return;
  }
#pragma unroll
  for (int r = 0; r < G; ++r) {
    if (yg + r < yend) {
      load_raw(p, c, yg + r, xl, raw[r]);
    } else {
#pragma unroll
      for (int k = 0; k < kPX; ++k) raw[r][k] = ET(0);
    }
  }
}

template <typename A, bool SQR, typename ET>
__device__ __forceinline__ A value_of(ET e) {
  const A a = (A)e;
  return SQR ? a * a : a;
}

// ---- Per-lane row stream through shared memory ------------------------------
//
// On the vector path each lane copies its own kPX pixels of every tile row
// into a ring of kDepth slots with cp.async, kDepth rows ahead of the row it
// consumes, and reads back only what it copied itself, so no lane waits for
// another. The copies in flight hold no registers: a warp keeps kDepth rows
// (4 KB for 4-byte pixels) in flight whatever its per-row work.

__device__ __forceinline__ uint32_t smem_u32(const void* ptr) {
  return (uint32_t)__cvta_generic_to_shared(ptr);
}

template <int BYTES>
__device__ __forceinline__ void cp_async(void* dst, const void* src) {
  if constexpr (BYTES == 16)
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)), "l"(src)
                 : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(smem_u32(dst)), "l"(src),
                 "n"(BYTES)
                 : "memory");
}

__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;" ::: "memory");
}

template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

template <typename ET>
struct RowStream {
  static constexpr int kLane = kPX * (int)sizeof(ET);  // bytes per lane and row
  static constexpr int kDepth = kLane > 16 ? 4 : 8;
  static constexpr int kSlot = 32 * kLane;             // one warp-row
  static constexpr int kWarpBytes = kDepth * kSlot;

  unsigned char* mine;  // this lane's bytes in slot 0
  const char* src;      // this lane's pixels in row 0 of the tile
  size_t pitch;
  int nrows;

  __device__ __forceinline__ RowStream(unsigned char* warp_ring, int lane, const char* row0,
                                       size_t pitch_, int nrows_)
      : mine(warp_ring + lane * kLane), src(row0), pitch(pitch_), nrows(nrows_) {}

  __device__ __forceinline__ void copy(int y) const {
    unsigned char* d = mine + (y & (kDepth - 1)) * kSlot;
    const char* g = src + (size_t)y * pitch;
    if constexpr (kLane <= 16) {
      cp_async<kLane>(d, g);
    } else {
      cp_async<16>(d, g);
      cp_async<16>(d + 16, g + 16);
    }
  }

  // Rows 0 .. kDepth - 1 in flight; one commit group per row, empty past the
  // tile's last row, so that group y always holds row y.
  __device__ __forceinline__ void start() const {
#pragma unroll
    for (int d = 0; d < kDepth; ++d) {
      if (d < nrows) copy(d);
      cp_async_commit();
    }
  }

  // Row y (y < nrows) once its group has landed.
  __device__ __forceinline__ void read(int y, ET (&e)[kPX]) const {
    cp_async_wait<kDepth - 1>();
    const unsigned char* d = mine + (y & (kDepth - 1)) * kSlot;
    if constexpr (kLane == 4) {
      const uint32_t q = *reinterpret_cast<const uint32_t*>(d);
      memcpy(e, &q, sizeof(q));
    } else if constexpr (kLane == 8) {
      const uint2 q = *reinterpret_cast<const uint2*>(d);
      memcpy(e, &q, sizeof(q));
    } else if constexpr (kLane == 16) {
      const uint4 q = *reinterpret_cast<const uint4*>(d);
      memcpy(e, &q, sizeof(q));
    } else {
      uint4 q[2];
      q[0] = reinterpret_cast<const uint4*>(d)[0];
      q[1] = reinterpret_cast<const uint4*>(d)[1];
      memcpy(e, q, sizeof(q));
    }
  }

  // Reuse row y's slot for row y + kDepth. The warp barrier orders the read
  // of the slot before the copy that overwrites it.
  __device__ __forceinline__ void refill(int y) const {
    __syncwarp();
    if (y + kDepth < nrows) copy(y + kDepth);
    cp_async_commit();
  }

  __device__ __forceinline__ void drain() const { cp_async_wait<0>(); }
};

template <int TYPE, typename A, bool SQR>
__global__ void __launch_bounds__(32 * kWarpsPerCta, kMinCtas)
    integral_reduce_kernel(const IntegralParams p) {
  using ET = typename ElemOf<TYPE>::T;
  constexpr int G = group_rows<ET>();
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
  const bool vec_tile = p.vec_src && (bx + 1) * kTW <= p.W;
  if (vec_tile) {
    using RS = RowStream<ET>;
    __shared__ __align__(16) unsigned char ring[kWarpsPerCta * RS::kWarpBytes];
    const int nrows = yend - y0;
    const RS rs(ring + (threadIdx.x >> 5) * RS::kWarpBytes, lane,
                p.src + (size_t)y0 * p.src_pitch + (size_t)xl * sizeof(ET), p.src_pitch, nrows);
    rs.start();
    for (int yg = 0; yg < nrows; yg += G) {
      A s[G];
#pragma unroll
      for (int r = 0; r < G; ++r) {
        s[r] = A(0);
        if (yg + r < nrows) {
          ET e[kPX];
          rs.read(yg + r, e);
#pragma unroll
          for (int k = 0; k < kPX; ++k) {
            const A v = value_of<A, SQR>(e[k]);
            s[r] += v;
            col[k] += v;
          }
          rs.refill(yg + r);
        }
      }
      const A tot = warp_sum_rows<G>(s, lane);
      const int r = lane >> (5 - log2_of<G>());
      if ((lane & (32 / G - 1)) == 0 && yg + r < nrows)
        rowsum[(size_t)(y0 + yg + r) * p.nBX + bx] = tot;
    }
    rs.drain();
  } else {
    // Generic layouts (several channels, unaligned rows, the image's right
    // edge): register groups of rows.
    constexpr int GG = G / 2;
    for (int yg = y0; yg < yend; yg += GG) {
      ET raw[GG][kPX];
      load_group<GG>(p, c, yg, yend, xl, false, raw);
      A s[GG];
#pragma unroll
      for (int r = 0; r < GG; ++r) {
        s[r] = A(0);
#pragma unroll
        for (int k = 0; k < kPX; ++k) {
          const A v = value_of<A, SQR>(raw[r][k]);
          s[r] += v;
          col[k] += v;
        }
      }
      const A tot = warp_sum_rows<GG>(s, lane);
      const int r = lane >> (5 - log2_of<GG>());
      if ((lane & (32 / GG - 1)) == 0 && yg + r < yend)
        rowsum[(size_t)(yg + r) * p.nBX + bx] = tot;
    }
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

// Junctions. Blocks [0, top_blocks): kJCols columns each, LB -> ColTop in
// place, bands taken in chunks of 8 x kJBands: thread (column, group g) loads
// kJBands bands, the groups' totals are combined through shared memory. These
// blocks have the longer dependency chain, so they come first in the grid.
// Blocks after them: a warp per kJRows image rows, RowSum -> RowLeft in place.
// Loads are issued from clamped (always valid) addresses and masked
// afterwards: a load whose use sits in the same branch would stall the warp
// before the next load issues.
template <typename A>
__global__ void __launch_bounds__(kJThreads)
    integral_junction_kernel(const IntegralParams p, int top_blocks) {
  constexpr int kGroups = kJThreads / kJCols;
  constexpr int kChunk = kGroups * kJBands;
  __shared__ A group_total[kGroups][kJCols];
  const int c = blockIdx.y;
  const int lane = threadIdx.x & 31;
  // Launched as a programmatic dependent of the reduce launch: everything
  // read here is written by it.
  cudaGridDependencySynchronize();
  if ((int)blockIdx.x >= top_blocks) {
    const int y0 = ((blockIdx.x - top_blocks) * (kJThreads / 32) + (threadIdx.x >> 5)) * kJRows;
    if (y0 >= p.H) return;
    A* rs = reinterpret_cast<A*>(p.rowsum) + (size_t)c * p.H * p.nBX;
    A carry[kJRows];
#pragma unroll
    for (int i = 0; i < kJRows; ++i) carry[i] = A(0);
    for (int b0 = 0; b0 < p.nBX; b0 += 32) {
      const int b = b0 + lane;
      A v[kJRows];
#pragma unroll
      for (int i = 0; i < kJRows; ++i)
        v[i] = rs[(size_t)min(y0 + i, p.H - 1) * p.nBX + min(b, p.nBX - 1)];
#pragma unroll
      for (int i = 0; i < kJRows; ++i) {
        if (b >= p.nBX) v[i] = A(0);
        const A incl = warp_incl_scan(v[i], lane);
        if (b < p.nBX && y0 + i < p.H) rs[(size_t)(y0 + i) * p.nBX + b] = carry[i] + (incl - v[i]);
        carry[i] += __shfl_sync(0xffffffffu, incl, 31);
      }
    }
    return;
  }
  A* lb = reinterpret_cast<A*>(p.lb) + (size_t)c * p.nBY * p.W;
  const int x = blockIdx.x * kJCols + lane;
  const int xc = min(x, p.W - 1);
  const int g = threadIdx.x >> 5;
  A carry = A(0);
  for (int b0 = 0; b0 < p.nBY; b0 += kChunk) {
    A v[kJBands];
#pragma unroll
    for (int j = 0; j < kJBands; ++j)
      v[j] = lb[(size_t)min(b0 + g * kJBands + j, p.nBY - 1) * p.W + xc];
    A s = A(0);
#pragma unroll
    for (int j = 0; j < kJBands; ++j) {
      if (b0 + g * kJBands + j >= p.nBY) v[j] = A(0);
      s += v[j];
    }
    group_total[g][lane] = s;
    __syncthreads();
    A run = carry;
    for (int h = 0; h < g; ++h) run += group_total[h][lane];
#pragma unroll
    for (int j = 0; j < kJBands; ++j) {
      const int by = b0 + g * kJBands + j;
      if (by < p.nBY && x < p.W) lb[(size_t)by * p.W + x] = run;
      run += v[j];
    }
#pragma unroll
    for (int h = 0; h < kGroups; ++h) carry += group_total[h][lane];
    __syncthreads();
  }
}

__device__ __forceinline__ float to_f32(long long v) { return __ll2float_rn(v); }
__device__ __forceinline__ float to_f32(double v) { return __double2float_rn(v); }
__device__ __forceinline__ double to_f64(long long v) { return __ll2double_rn(v); }
__device__ __forceinline__ double to_f64(double v) { return v; }

// A 32-byte store of 4 doubles (sm_100 has 256-bit global accesses): a
// warp's store covers 1 KB contiguous, every 32-byte sector written whole.
__device__ __forceinline__ void st_global_v4f64(double* ptr, const double (&v)[4]) {
  asm volatile("st.global.v4.f64 [%0], {%1, %2, %3, %4};" ::"l"(ptr), "d"(v[0]), "d"(v[1]),
               "d"(v[2]), "d"(v[3])
               : "memory");
}

// One row of the lane's 4 results: one vector store (32 bytes for F64, 16 for
// F32) when the destination allows it.
template <typename OT, typename A>
__device__ __forceinline__ void store_row(const IntegralParams& p, int c, int y, int xl,
                                          const A (&acc)[kPX]) {
  OT* row = reinterpret_cast<OT*>(p.dst + (size_t)y * p.dst_pitch);
  OT o[kPX];
#pragma unroll
  for (int k = 0; k < kPX; ++k) {
    if constexpr (sizeof(OT) == 8) o[k] = to_f64(acc[k]);
    else o[k] = to_f32(acc[k]);
  }
  if (p.vec_dst && xl + kPX <= p.W) {
    if constexpr (sizeof(OT) == 8) {
      st_global_v4f64(row + xl, o);
    } else {
      uint4 q;
      memcpy(&q, o, sizeof(q));
      *reinterpret_cast<uint4*>(row + xl) = q;
    }
    return;
  }
#pragma unroll
  for (int k = 0; k < kPX; ++k)
    if (xl + k < p.W) row[(size_t)(xl + k) * p.nch + c] = o[k];
}

// One row of the final pass: the lane's 4 values plus the row's RowLeft and
// the warp-scanned prefix of the lanes to its left, added to the running
// column sums and stored.
template <typename A, bool SQR, typename OT, typename ET>
__device__ __forceinline__ void final_row(const IntegralParams& p, int c, int y, int xl,
                                          int lane, const ET (&e)[kPX], A left,
                                          A (&acc)[kPX]) {
  A v[kPX];
#pragma unroll
  for (int k = 0; k < kPX; ++k) v[k] = value_of<A, SQR>(e[k]);
#pragma unroll
  for (int k = 1; k < kPX; ++k) v[k] += v[k - 1];
  const A incl = warp_incl_scan(v[kPX - 1], lane);
  const A base = incl - v[kPX - 1] + left;
#pragma unroll
  for (int k = 0; k < kPX; ++k) acc[k] += base + v[k];
  store_row<OT>(p, c, y, xl, acc);
}

static_assert(kTH <= 32, "a tile's RowLeft values are held one per lane");

template <int TYPE, typename A, bool SQR, typename OT>
__global__ void __launch_bounds__(32 * kWarpsPerCta, kMinCtas)
    integral_final_kernel(const IntegralParams p) {
  using ET = typename ElemOf<TYPE>::T;
  using RS = RowStream<ET>;
  __shared__ __align__(16) unsigned char ring[kWarpsPerCta * RS::kWarpBytes];
  const int lane = threadIdx.x & 31;
  const int tile = blockIdx.x * kWarpsPerCta + (threadIdx.x >> 5);
  const int c = blockIdx.y;
  if (tile >= p.nBX * p.nBY) return;
  const int bx = tile % p.nBX, by = tile / p.nBX;
  const int xl = bx * kTW + lane * kPX;
  const int y0 = by * kTH;
  const int nrows = min(p.H, y0 + kTH) - y0;
  const A* rowleft = reinterpret_cast<const A*>(p.rowsum) + (size_t)c * p.H * p.nBX;
  const A* top = reinterpret_cast<const A*>(p.lb) + (size_t)c * p.nBY * p.W;
  const bool vec_tile = p.vec_src && (bx + 1) * kTW <= p.W;
  const RS rs(ring + (threadIdx.x >> 5) * RS::kWarpBytes, lane,
              p.src + (size_t)y0 * p.src_pitch + (size_t)xl * sizeof(ET), p.src_pitch, nrows);
  // The first source rows are in flight while the junction launch (this
  // kernel's programmatic predecessor) finishes; Top and RowLeft after it.
  if (vec_tile) rs.start();
  cudaGridDependencySynchronize();
  // Top = ColTop + the sum of ColTop at the last column of the tiles to the
  // left (lane j takes tiles j, j + 32, ...).
  A left_tiles = A(0);
  for (int j0 = 0; j0 < bx; j0 += 32) {
    const int j = min(j0 + lane, bx - 1);
    const A v = top[(size_t)by * p.W + min(p.W, (j + 1) * kTW) - 1];
    if (j0 + lane < bx) left_tiles += v;
  }
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) left_tiles += __shfl_xor_sync(0xffffffffu, left_tiles, d);
  A acc[kPX];
#pragma unroll
  for (int k = 0; k < kPX; ++k) acc[k] = top[(size_t)by * p.W + min(xl + k, p.W - 1)];
#pragma unroll
  for (int k = 0; k < kPX; ++k) acc[k] = (xl + k < p.W) ? acc[k] + left_tiles : A(0);
  // RowLeft of the tile's rows: lane i holds row y0 + i.
  const A left_lane = rowleft[(size_t)(y0 + min(lane, nrows - 1)) * p.nBX + bx];
  if (vec_tile) {
    for (int y = 0; y < nrows; ++y) {
      ET e[kPX];
      rs.read(y, e);
      rs.refill(y);
      final_row<A, SQR, OT>(p, c, y0 + y, xl, lane, e, __shfl_sync(0xffffffffu, left_lane, y),
                            acc);
    }
    rs.drain();
    return;
  }
  // Generic layouts (several channels, unaligned rows, the image's right
  // edge): register groups of rows.
  constexpr int G = group_rows<ET>() / 4;
  for (int yg = 0; yg < nrows; yg += G) {
    ET raw[G][kPX];
    load_group<G>(p, c, y0 + yg, y0 + nrows, xl, false, raw);
#pragma unroll
    for (int r = 0; r < G; ++r) {
      const A left = __shfl_sync(0xffffffffu, left_lane, (yg + r) & 31);
      if (yg + r < nrows) final_row<A, SQR, OT>(p, c, y0 + yg + r, xl, lane, raw[r], left, acc);
    }
  }
}

// Launch on st as a programmatic dependent of the previous launch on st: its
// blocks may start as the previous launch's blocks exit, and
// cudaGridDependencySynchronize() in the kernel waits for that launch's
// completion and memory.
template <typename... KArgs, typename... Args>
cudaError_t launch_dependent(void (*kernel)(KArgs...), dim3 grid, dim3 block, cudaStream_t st,
                             Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = 0;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, args...);
}

// Asks for the largest shared-memory carveout for `kernel` on the current
// device, once per (kernel, device): the row rings take 16 KB per block and
// kMinCtas blocks should fit on an SM.
void prefer_shared(const void* kernel) {
  static std::mutex mu;
  static std::set<std::pair<const void*, int>> done;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return;
  std::lock_guard<std::mutex> lock(mu);
  if (done.insert({kernel, dev}).second)
    cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                         (int)cudaSharedmemCarveoutMaxShared);
}

// The reduce launch is an ordinary one: it overwrites the scratch that the
// previous call's final launch reads.
template <int TYPE, typename A, bool SQR>
cudaError_t run(IntegralParams& p, cudaStream_t st) {
  prefer_shared((const void*)integral_reduce_kernel<TYPE, A, SQR>);
  prefer_shared((const void*)integral_final_kernel<TYPE, A, SQR, double>);
  prefer_shared((const void*)integral_final_kernel<TYPE, A, SQR, float>);
  const int ntiles = p.nBX * p.nBY;
  dim3 g1((ntiles + kWarpsPerCta - 1) / kWarpsPerCta, p.nch);
  integral_reduce_kernel<TYPE, A, SQR><<<g1, 32 * kWarpsPerCta, 0, st>>>(p);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  const int top_blocks = (p.W + kJCols - 1) / kJCols;
  const int rows_per_block = kJThreads / 32 * kJRows;
  dim3 g2(top_blocks + (p.H + rows_per_block - 1) / rows_per_block, p.nch);
  e = launch_dependent(integral_junction_kernel<A>, g2, dim3(kJThreads), st, p, top_blocks);
  if (e != cudaSuccess) return e;
  if (p.dst_f64)
    e = launch_dependent(integral_final_kernel<TYPE, A, SQR, double>, g1,
                         dim3(32 * kWarpsPerCta), st, p);
  else
    e = launch_dependent(integral_final_kernel<TYPE, A, SQR, float>, g1,
                         dim3(32 * kWarpsPerCta), st, p);
  count_launches(3);
  return e;
}

template <int TYPE, typename AI>
cudaError_t run_sqr(bool sqr, IntegralParams& p, cudaStream_t st) {
  return sqr ? run<TYPE, AI, true>(p, st) : run<TYPE, AI, false>(p, st);
}

}  // namespace

size_t integral_scratch_bytes(int width, int height, int nch) {
  const size_t nBX = (width + kTW - 1) / kTW, nBY = (height + kTH - 1) / kTH;
  return 8 * (size_t)nch * ((size_t)height * nBX + nBY * (size_t)width) + 256;
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
  p.vec_src = p.nch == 1 && ((uintptr_t)p.src % 16) == 0 && (p.src_pitch % 16) == 0;
  // A lane stores 4 pixels: 32 bytes for F64, 16 for F32.
  const size_t dst_align = p.dst_f64 ? 32 : 16;
  p.vec_dst = p.nch == 1 && ((uintptr_t)p.dst % dst_align) == 0 && (p.dst_pitch % dst_align) == 0;
  if (scratch_bytes < integral_scratch_bytes(p.W, p.H, p.nch)) return cudaErrorInvalidValue;
  char* s = (char*)scratch;
  p.rowsum = s;
  s += 8 * (size_t)p.nch * p.H * p.nBX;
  p.lb = s;

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

// Largest scratch the allocation-free entry point can use: 16 MiB, enough for
// one channel up to about 7300 x 7300 pixels (integral_scratch_bytes()).
constexpr size_t kNoAllocScratchBytes = size_t(16) << 20;
__device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// Device addresses of g_noalloc_scratch, one per CUDA context that has used
// it, keyed by the context's process-unique ID. A context that is destroyed
// (cudaDeviceReset, or a primary context released and created again) loads
// the module afresh, possibly at another address; its successor has a new
// ID and therefore gets its own lookup, never a stale address.
std::mutex g_noalloc_mutex;
std::map<unsigned long long, void*> g_noalloc_addr;

typedef CUresult (*CtxGetCurrentFn)(CUcontext*);
typedef CUresult (*CtxGetIdFn)(CUcontext, unsigned long long*);

template <typename F>
F driver_fn(const char* name) {
  void* f = nullptr;
  cudaDriverEntryPointQueryResult q;
  if (cudaGetDriverEntryPoint(name, &f, cudaEnableDefault, &q) != cudaSuccess ||
      q != cudaDriverEntryPointSuccess)
    return nullptr;
  return reinterpret_cast<F>(f);
}

// ID of the calling thread's current context, or false if there is none yet
// (the runtime binds the device's primary context on its first real call).
bool current_ctx_id(unsigned long long* id) {
  static const CtxGetCurrentFn get_cur = driver_fn<CtxGetCurrentFn>("cuCtxGetCurrent");
  static const CtxGetIdFn get_id = driver_fn<CtxGetIdFn>("cuCtxGetId");
  CUcontext c = nullptr;
  if (!get_cur || !get_id || get_cur(&c) != CUDA_SUCCESS || c == nullptr) return false;
  return get_id(c, id) == CUDA_SUCCESS;
}

// The device address of g_noalloc_scratch in the current context. Host code
// cannot use the array's name as a device address; cudaGetSymbolAddress gives
// the real one. It is looked up once per context (the first call made in a
// context, which may also load the module) and then served from the map.
cudaError_t noalloc_scratch(void** ptr) {
  unsigned long long id = 0;
  bool have_id = current_ctx_id(&id);
  if (have_id) {
    std::lock_guard<std::mutex> lk(g_noalloc_mutex);
    auto it = g_noalloc_addr.find(id);
    if (it != g_noalloc_addr.end()) {
      *ptr = it->second;
      return cudaSuccess;
    }
  }
  void* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess) return e;
  // The lookup made the primary context current if nothing was.
  if (!have_id) have_id = current_ctx_id(&id);
  if (have_id) {
    std::lock_guard<std::mutex> lk(g_noalloc_mutex);
    g_noalloc_addr[id] = p;
  }
  *ptr = p;
  return cudaSuccess;
}

}  // namespace
}  // namespace ocipb

#include <climits>
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
    // Refused before the scratch size is computed in int arithmetic (a
    // dimension above INT_MAX would wrap); far above the fixed limit anyway.
    if (SourceDesc.Width > (unsigned)INT_MAX || SourceDesc.Height > (unsigned)INT_MAX)
      fail(CL_INVALID_IMAGE_SIZE, "image too large for ocipIntegralNoAlloc: a dimension "
                                  "exceeds INT_MAX, beyond the fixed scratch limit");
    const size_t need = integral_scratch_bytes((int)SourceDesc.Width, (int)SourceDesc.Height,
                                               (int)SourceDesc.Channels);
    if (need > kNoAllocScratchBytes)
      fail(CL_INVALID_IMAGE_SIZE,
           "image too large for ocipIntegralNoAlloc: needs " + std::to_string(need) +
               " bytes of scratch, the fixed limit is " + std::to_string(kNoAllocScratchBytes));
    void* scratch = nullptr;
    check_cuda(noalloc_scratch(&scratch), "cudaGetSymbolAddress");
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
