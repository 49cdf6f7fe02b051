// Packed-byte SAD kernel for AbsDistance of 8-bit sources (U8, S8), sm_100a.
//
// AbsDistance (reference cl-files/ImageProximity.cl:213-242) sums |S - T| over
// the window. For an 8-bit source every term is an integer in [0, 255], so the sum
// is exact in a uint32 register for any template of fewer than 2^24 pixels,
// and the result is rounded once to the destination type. That equals the
// plain kernel's result (float accumulation while sums stay below 2^24, exact
// double above) and the reference's wherever its float accumulation is exact.
//
// Four taps per instruction: vabsdiff4 with accumulate adds the four bytewise
// absolute differences of two packed words (bytes unsigned for U8, signed for
// S8) to a 32-bit sum.
//
// Tiling follows the plain kernel: a CTA of 8 warps owns a 256 x 32 output
// tile; lane l owns 8 consecutive columns, warp w owns 4 consecutive rows.
// The tile's source rows (plus halo) and the template rows are staged in
// shared memory as bytes (one channel of the interleaved pixels, zero outside
// the image; template rows zero-padded to a multiple of 8). For each source
// row q and 8-byte template chunk, a lane reads the 16 window bytes its
// outputs need (two 8-byte loads; a warp's load is 256 contiguous bytes),
// forms the 12 byte-shifted words (3 aligned, 9 by byte_perm) and applies
// them to its 4 output rows, each with its own template row h = q - j, so
// each output's terms are added in the reference's order (h outer, w inner)
// -- which for exact integer sums does not change the result anyway.
#include <cuda_runtime.h>

#include "internal.h"

namespace ocipb {
namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int RX = 8;             // outputs per lane along x
constexpr int RY = 4;             // output rows per warp
constexpr int TX = 32 * RX;       // 256
constexpr int TY = kWarps * RY;   // 32
constexpr int kSmemBudget = 200 * 1024;

struct SadParams {
  const unsigned char* src;
  size_t src_pitch;
  const unsigned char* tmpl;
  size_t tmpl_pitch;
  char* dst;
  size_t dst_pitch;
  int dst_f64;
  int W, H, nch, dst_nch;
  int tw, th;
  int tw8;    // template row length in shared memory (multiple of 8)
  int rowB;   // bytes per staged source row (multiple of 16)
};

// acc + |a0 - b0| + |a1 - b1| + |a2 - b2| + |a3 - b3| over the bytes of a, b
// (unsigned bytes, or signed bytes when SIGNED).
template <bool SIGNED>
__device__ __forceinline__ uint32_t sad4(uint32_t a, uint32_t b, uint32_t acc) {
  uint32_t d;
  if constexpr (SIGNED)
    asm("vabsdiff4.u32.s32.s32.add %0, %1, %2, %3;" : "=r"(d) : "r"(a), "r"(b), "r"(acc));
  else
    asm("vabsdiff4.u32.u32.u32.add %0, %1, %2, %3;" : "=r"(d) : "r"(a), "r"(b), "r"(acc));
  return d;
}

// Bytes [k, k + 4) of the little-endian byte string lo:hi (0 < k < 4).
__device__ __forceinline__ uint32_t shifted(uint32_t lo, uint32_t hi, int k) {
  return __byte_perm(lo, hi, 0x3210 + 0x1111 * k);
}

// One staged source row q (r = q - first row of the warp) applied to the
// warp's RY output rows. FULL: every output row j meets template row
// h = r - j (no range checks).
template <bool SIGNED, bool FULL>
__device__ __forceinline__ void sad_row(const SadParams& p, const unsigned char* s_src,
                                        const unsigned char* s_t, int q, int r, int nc,
                                        int lane, uint32_t mlast0, uint32_t mlast1,
                                        uint32_t (&acc)[RY][RX]) {
  const unsigned char* srow = s_src + (size_t)q * p.rowB + lane * RX;
  for (int ch = 0; ch < nc; ++ch) {
    const uint2 a = *reinterpret_cast<const uint2*>(srow + 8 * ch);
    const uint2 b = *reinterpret_cast<const uint2*>(srow + 8 * ch + 8);
    uint32_t sw[12];
    sw[0] = a.x;
    sw[4] = a.y;
    sw[8] = b.x;
#pragma unroll
    for (int k = 1; k < 4; ++k) {
      sw[k] = shifted(a.x, a.y, k);
      sw[4 + k] = shifted(a.y, b.x, k);
      sw[8 + k] = shifted(b.x, b.y, k);
    }
    // Output i reads word i against template bytes 0 .. 3 of the chunk and
    // word i + 4 against bytes 4 .. 7; in the last chunk each is masked to
    // the valid bytes it meets.
    uint32_t w0[RX], w1[RX];
#pragma unroll
    for (int i = 0; i < RX; ++i) {
      w0[i] = sw[i];
      w1[i] = sw[i + 4];
    }
    if (ch == nc - 1) {
#pragma unroll
      for (int i = 0; i < RX; ++i) {
        w0[i] &= mlast0;
        w1[i] &= mlast1;
      }
    }
#pragma unroll
    for (int j = 0; j < RY; ++j) {
      const int h = r - j;
      if (!FULL && (h < 0 || h >= p.th)) continue;
      const uint2 t = *reinterpret_cast<const uint2*>(s_t + (size_t)h * p.tw8 + 8 * ch);
#pragma unroll
      for (int i = 0; i < RX; ++i) {
        acc[j][i] = sad4<SIGNED>(w0[i], t.x, acc[j][i]);
        acc[j][i] = sad4<SIGNED>(w1[i], t.y, acc[j][i]);
      }
    }
  }
}

template <bool SIGNED>
__global__ void __launch_bounds__(kThreads) prox_sad_kernel(const SadParams p) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int c = blockIdx.z;
  const int x0 = blockIdx.x * TX;
  const int y0 = blockIdx.y * TY;
  const int left = -(p.tw / 2);
  const int top = -(p.th / 2);
  const int L = TX + p.tw8;           // staged bytes per source row
  const int qtot = TY + p.th - 1;     // staged source rows
  unsigned char* s_src = smem;
  unsigned char* s_t = smem + (size_t)qtot * p.rowB;

  // Stage the tile's source rows, a warp per row: each lane issues kStage
  // loads (clamped addresses, masked afterwards) before it stores any.
  constexpr int kStage = 10;  // 320 bytes per warp pass: one pass for tw <= 64
  for (int q = warp; q < qtot; q += kWarps) {
    const int gy = y0 + top + q;
    const bool row_in = gy >= 0 && gy < p.H;
    const unsigned char* grow = p.src + (size_t)min(max(gy, 0), p.H - 1) * p.src_pitch;
    unsigned char* srow = s_src + (size_t)q * p.rowB;
    for (int e0 = 0; e0 < L; e0 += 32 * kStage) {
      unsigned char v[kStage];
#pragma unroll
      for (int u = 0; u < kStage; ++u) {
        const int gx = min(max(x0 + left + e0 + lane + 32 * u, 0), p.W - 1);
        v[u] = grow[(size_t)gx * p.nch + c];
      }
#pragma unroll
      for (int u = 0; u < kStage; ++u) {
        const int e = e0 + lane + 32 * u;
        const int gx = x0 + left + e;
        if (e < L) srow[e] = (row_in && gx >= 0 && gx < p.W) ? v[u] : (unsigned char)0;
      }
    }
  }
  for (int idx = threadIdx.x; idx < p.th * p.tw8; idx += kThreads) {
    const int h = idx / p.tw8;
    const int w = idx - h * p.tw8;
    s_t[idx] = w < p.tw ? p.tmpl[(size_t)h * p.tmpl_pitch + (size_t)w * p.nch + c] : 0;
  }
  __syncthreads();

  uint32_t acc[RY][RX];
#pragma unroll
  for (int j = 0; j < RY; ++j)
#pragma unroll
    for (int i = 0; i < RX; ++i) acc[j][i] = 0;

  const int nc = p.tw8 / 8;
  // Template bytes past tw are zero; the window bytes that meet them are
  // masked off in the last chunk so that they add |0 - 0|.
  const int rem = p.tw - 8 * (nc - 1);  // valid bytes of the last chunk, 1 .. 8
  const uint32_t mlast0 = rem >= 4 ? 0xffffffffu : (1u << (8 * rem)) - 1u;
  const uint32_t mlast1 = rem >= 8 ? 0xffffffffu : rem <= 4 ? 0u : (1u << (8 * (rem - 4))) - 1u;

  // Staged rows q of this warp: r = q - warp * RY in [0, RY + th - 1). Rows
  // with r in [RY - 1, th - 1] meet a template row in every output row of
  // the warp and take the loop without range checks.
  const int qa = warp * RY;
  const int qb = min(qtot, warp * RY + RY + p.th - 1);
  const int fa = min(qb, qa + RY - 1);
  const int fb = max(fa, min(qb, qa + p.th));
  for (int q = qa; q < fa; ++q)
    sad_row<SIGNED, false>(p, s_src, s_t, q, q - qa, nc, lane, mlast0, mlast1, acc);
  for (int q = fa; q < fb; ++q)
    sad_row<SIGNED, true>(p, s_src, s_t, q, q - qa, nc, lane, mlast0, mlast1, acc);
  for (int q = fb; q < qb; ++q)
    sad_row<SIGNED, false>(p, s_src, s_t, q, q - qa, nc, lane, mlast0, mlast1, acc);

#pragma unroll
  for (int j = 0; j < RY; ++j) {
    const int y = y0 + warp * RY + j;
    if (y >= p.H) continue;
    char* o = p.dst + (size_t)y * p.dst_pitch;
#pragma unroll
    for (int i = 0; i < RX; ++i) {
      const int x = x0 + lane * RX + i;
      if (x >= p.W) continue;
      if (p.dst_f64)
        reinterpret_cast<double*>(o)[(size_t)x * p.dst_nch + c] = (double)acc[j][i];
      else
        reinterpret_cast<float*>(o)[(size_t)x * p.dst_nch + c] = __uint2float_rn(acc[j][i]);
    }
  }
}

}  // namespace

size_t proximity_sad_8bit_smem(int tw, int th) {
  const int tw8 = (tw + 7) / 8 * 8;
  const int rowB = (TX + tw8 + 15) / 16 * 16;
  return (size_t)(TY + th - 1) * rowB + (size_t)th * tw8;
}

bool proximity_sad_8bit_supported(const DevImage& src, const DevImage& tmpl) {
  if ((src.type != U8 && src.type != S8) || tmpl.type != src.type) return false;
  // Exact uint32 sums: every output adds tw * th terms of at most 255.
  if ((double)tmpl.width * tmpl.height * 255.0 >= 4294967296.0) return false;
  return proximity_sad_8bit_smem(tmpl.width, tmpl.height) <= (size_t)kSmemBudget;
}

cudaError_t launch_proximity_sad_8bit(const DevImage& src, const DevImage& tmpl,
                                    const DevImage& dst, cudaStream_t st) {
  SadParams p;
  p.src = (const unsigned char*)src.ptr;
  p.src_pitch = src.pitch;
  p.tmpl = (const unsigned char*)tmpl.ptr;
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
  p.tw8 = (p.tw + 7) / 8 * 8;
  p.rowB = (TX + p.tw8 + 15) / 16 * 16;
  const size_t smem = proximity_sad_8bit_smem(p.tw, p.th);
  auto kern = src.type == S8 ? prox_sad_kernel<true> : prox_sad_kernel<false>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem);
  if (e != cudaSuccess) return e;
  dim3 grid((p.W + TX - 1) / TX, (p.H + TY - 1) / TY, src.nch);
  kern<<<grid, kThreads, smem, st>>>(p);
  count_launches(1);
  return cudaGetLastError();
}

}  // namespace ocipb
