// Backward (adjoint) kernels of SqrDistance and CrossCorr_Norm for F32
// sources. No reference counterpart: the reference has no derivatives. The
// forward definitions are those of cl-files/ImageProximity.cl :44-73 and
// :375-412 (window anchor (tw/2, th/2), zero padding).
//
// With upstream gradients G1 of SqrDistance and G2 of CrossCorr_Norm (either
// may be absent), N = CrossCorr_Norm, E_S the window energy and E_T the
// template energy, the gradients of L = sum G1 SqrDistance + sum G2 N are
//   dS(u, v) = sum_{w,h} M(u - w + a, v - h + b) T(w, h)
//            + S(u, v) sum_{w,h} P(u - w + a, v - h + b)
//   dT(w, h) = sum_{x,y} M(x, y) S(x + w - a, y + h - b)
//            + T(w, h) (2 sum G1 - sum(G2 N) / E_T)
// with M = -2 G1 + G2 / sqrt(E_S E_T) and P = 2 G1 - G2 N / E_S (zero where
// E_S E_T = 0: those outputs have no derivative). So one pass serves both
// measures:
//   * E_S is recomputed as separable FP64 window sums of S^2 (not stored by
//     the forward pass);
//   * the first term of dS is a correlation of M with the flipped template
//     (anchor (tw-1-a, th-1-b)), run on the forward tensor kernel;
//   * the window sums of P are separable FP64 sums as well;
//   * the first term of dT is the weight-gradient reduction below, on the
//     tensor cores (BF16 hi/lo split of S and M, three MMAs), with per-CTA
//     partials summed in FP64.
//
// Weight-gradient kernel. dT(w, h) = sum_r sum_x S(x + w - a, r) M(x, r - h + b).
// A CTA takes a strip of 128 columns x and a band of source rows r. Its 128
// TMEM lanes hold PR source rows at a time (lane L = i WP + w: row r0 + i,
// template column w; PR = 4 for tw <= 32, 2 for tw <= 64):
//   A[i WP + w][k] = S(x0 + k + w - a, r0 + i)          (built with tcgen05.st)
//   B[n][k]        = M(x0 + k, r0 - th + 1 + b + n)      (staged once, BF16)
//   D[i WP + w][n] += sum_k A B                         (accumulated all band)
// D[i WP + w][n] belongs to dT(w, h) with h = i + th - 1 - n for every step, so
// D accumulates in TMEM over the whole band and is folded into dT once.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>

#include "sm100.cuh"
#include "tensor.h"

namespace ocipb {
namespace {

using namespace sm100;

constexpr int kXS = 128;        // columns x per CTA (the MMA K of one step)
constexpr int kBRmax = 128;     // source rows per CTA band (at most)
constexpr int kWgWarps = 9;     // 8 builders (and fold), 1 control
constexpr int kWgThreads = kWgWarps * 32;
constexpr int kWgStages = 4;    // TMA stages of PR source rows
constexpr int kWgA = 3;         // A stages in TMEM
constexpr int kWgCols = 512;
constexpr long long kWgSpin = 4000000000LL;

struct WgParams {
  int W, H, tw, th, ax, ay;
  int BR;          // source rows per CTA band (a multiple of PR)
  int nbox;        // 16-byte groups per staged S row
  int lead;        // staged rows start `lead` pixels before x0 - ax
  const float* M;  // M map, row pitch m_pitch bytes
  size_t m_pitch;
  float* partials;  // [CTA][th * tw]
  int* err;
};

template <int PR>
struct WgCfg {
  static constexpr int WP = 128 / PR;         // template columns per row phase
};

struct WgLayout {
  int raw_stage, raw, nrs, b_arr, b, part, bars, total;
};

__host__ __device__ inline int wg_align(int x) { return (x + 127) & ~127; }

template <int PR>
__host__ __device__ inline WgLayout wg_layout(int nbox, int NB, int tw, int th, int BR) {
  WgLayout L;
  L.raw_stage = wg_align(PR * nbox * 16);
  L.raw = 0;
  L.nrs = BR + NB;  // staged M rows
  L.b_arr = kXS / 8 * L.nrs * 16;       // one BF16 array (hi or lo)
  L.b = L.raw + kWgStages * L.raw_stage;
  L.part = L.b + 2 * wg_align(L.b_arr);
  L.bars = L.part + wg_align(tw * th * 4);
  L.total = L.bars + wg_align(8 * (kWgStages + 2 * kWgA + 1) + 16);
  return L;
}

__device__ __forceinline__ uint32_t bf2(float lo, float hi) {
  __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<uint32_t*>(&v);
}

template <int PR>
__global__ void __launch_bounds__(kWgThreads, 1)
    wgrad_kernel(const __grid_constant__ CUtensorMap tmS, const WgParams p) {
  typedef WgCfg<PR> C;
  constexpr int WP = C::WP;
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ uint32_t s_tmem;
  __shared__ int s_abort;
  const int NB = (p.th + PR - 1 + 15) / 16 * 16;
  const WgLayout L = wg_layout<PR>(p.nbox, NB, p.tw, p.th, p.BR);
  uint64_t* raw_full = reinterpret_cast<uint64_t*>(smem + L.bars);
  uint64_t* ready = raw_full + kWgStages;
  uint64_t* mma_done = ready + kWgA;
  uint64_t* done_bar = mma_done + kWgA;
  float* part = reinterpret_cast<float*>(smem + L.part);
  volatile int* abort_flag = &s_abort;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int x0 = blockIdx.x * kXS;
  const int r_lo = blockIdx.y * p.BR;
  const int r_hi = min(p.H, r_lo + p.BR);
  const int nsteps = (r_hi - r_lo + PR - 1) / PR;
  const int mbase = r_lo - p.th + 1 + p.ay;  // M row of staged row 0

  if (threadIdx.x == 0) {
    s_abort = 0;
    for (int i = 0; i < kWgStages; ++i) mbar_init(&raw_full[i], 1);
    for (int i = 0; i < kWgA; ++i) {
      mbar_init(&ready[i], 8);
      mbar_init(&mma_done[i], 1);
    }
    mbar_init(done_bar, 1);
    fence_barrier_init();
  }
  if (warp == 0) tmem_alloc(&s_tmem, kWgCols);
  // Stage M rows mbase .. mbase + nrs - 1, columns x0 .. x0 + 127, as BF16
  // hi/lo in the K-major core-matrix layout [k / 8][row][8] (rows 16 bytes
  // apart, so a window of consecutive rows is one descriptor).
  for (int idx = threadIdx.x; idx < L.nrs * (kXS / 2); idx += kWgThreads) {
    const int row = idx / (kXS / 2), k = (idx - row * (kXS / 2)) * 2;
    const int y = mbase + row, x = x0 + k;
    float v0 = 0.f, v1 = 0.f;
    if (y >= 0 && y < p.H) {
      const float* mr = reinterpret_cast<const float*>(reinterpret_cast<const char*>(p.M) +
                                                       (size_t)y * p.m_pitch);
      if (x < p.W) v0 = mr[x];
      if (x + 1 < p.W) v1 = mr[x + 1];
    }
    const uint32_t hi = bf2(v0, v1);
    const uint32_t lo = bf2(v0 - __uint_as_float(hi << 16), v1 - __uint_as_float(hi & 0xFFFF0000u));
    const int off = ((k >> 3) * L.nrs + row) * 16 + (k & 7) * 2;
    *reinterpret_cast<uint32_t*>(smem + L.b + off) = hi;
    *reinterpret_cast<uint32_t*>(smem + L.b + wg_align(L.b_arr) + off) = lo;
  }
  for (int i = threadIdx.x; i < p.tw * p.th; i += kWgThreads) part[i] = 0.f;
  fence_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = s_tmem;
  const uint32_t acol = NB;  // A stages after the D columns

  if (warp == 8) {
    // ---- Control: TMA loads of PR source rows per step, MMA issue -------------
    if (lane == 0) {
      tma_prefetch_desc(&tmS);
      const int gx = (x0 - p.ax - p.lead) / 4;
      int issued = 0;
      for (; issued < min(nsteps, kWgStages); ++issued) {
        mbar_arrive_expect_tx(&raw_full[issued], PR * p.nbox * 16);
        tma_load_4d(smem + L.raw + issued * L.raw_stage, &tmS, 0, gx, r_lo + issued * PR, 0,
                    &raw_full[issued]);
      }
      const uint32_t bhi = smem_u32(smem + L.b);
      const uint32_t blo = bhi + wg_align(L.b_arr);
      const uint32_t idesc = idesc_bf16_f32(128, NB);
      const uint32_t lbo = L.nrs * 16;
      int i = 0, st = 0;
      uint32_t ph = 0;
      for (int s = 0; s < nsteps; ++s) {
        if (!mbar_wait(&ready[i], ph, abort_flag, kWgSpin)) break;
        // Every builder has read the rows of step s: reuse their stage.
        if (issued < nsteps) {
          mbar_arrive_expect_tx(&raw_full[st], PR * p.nbox * 16);
          tma_load_4d(smem + L.raw + st * L.raw_stage, &tmS, 0, gx, r_lo + issued * PR, 0,
                      &raw_full[st]);
          ++issued;
        }
        tc_fence_after();
        const uint32_t a = tmem + acol + i * kXS;  // hi: K/2 columns, lo: the next K/2
        const uint32_t boff = (uint32_t)(PR * s) * 16;
#pragma unroll
        for (int kk = 0; kk < kXS / 16; ++kk) {
          const uint32_t kb = kk * 2 * lbo;
          mma_bf16_ts(tmem, a + kk * 8, smem_desc(bhi + boff + kb, lbo, 128), idesc,
                      (s > 0 || kk > 0) ? 1u : 0u);
          mma_bf16_ts(tmem, a + kk * 8, smem_desc(blo + boff + kb, lbo, 128), idesc, 1);
          mma_bf16_ts(tmem, a + kXS / 2 + kk * 8, smem_desc(bhi + boff + kb, lbo, 128), idesc,
                      1);
        }
        mma_commit(&mma_done[i]);
        if (++i == kWgA) { i = 0; ph ^= 1; }
        if (++st == kWgStages) st = 0;
      }
      mma_commit(done_bar);
      volatile int no_abort = 0;
      mbar_wait(done_bar, 0, &no_abort, kWgSpin);
      for (int b = max(0, issued - kWgStages); b < issued; ++b)
        mbar_wait(&raw_full[b % kWgStages], (b / kWgStages) & 1, &no_abort, kWgSpin);
    }
  } else {
    // ---- Builders: A rows of step s (two warps per TMEM sub-partition, one
    // half of the K columns each) -------------------------------------------
    const int sp = warp & 3, half = warp >> 2;
    const int Lr = sp * 32 + lane;       // TMEM lane
    const int ri = Lr / WP, w = Lr % WP;  // row phase, template column
    const uint32_t lane_base = tmem + (static_cast<uint32_t>(sp * 32) << 16);
    const int e0 = p.lead + w;  // first pixel of this lane's window in the staged row
    int i = 0, st = 0;
    uint32_t iph = 0, rph = 0;
    for (int s = 0; s < nsteps; ++s) {
      if (!mbar_wait(&raw_full[st], rph, abort_flag, kWgSpin)) break;
      if (!mbar_wait(&mma_done[i], iph ^ 1, abort_flag, kWgSpin)) break;
      tc_fence_after();
      const bool live = r_lo + PR * s + ri < r_hi;  // rows of the next band stay zero
      const float2* r2 = reinterpret_cast<const float2*>(smem + L.raw + st * L.raw_stage +
                                                         ri * p.nbox * 16) + (e0 >> 1);
      const bool odd = e0 & 1;
      const uint32_t a_addr = lane_base + acol + i * kXS;
#pragma unroll
      for (int c = half * 4; c < half * 4 + 4; ++c) {  // 4 chunks of 16 columns
        float2 v[9];
#pragma unroll
        for (int j = 0; j < 9; ++j) v[j] = r2[c * 8 + j];
        uint32_t hi[8], lo[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          float f0 = odd ? v[q].y : v[q].x;
          float f1 = odd ? v[q + 1].x : v[q].y;
          if (!live) f0 = f1 = 0.f;
          hi[q] = bf2(f0, f1);
          lo[q] = bf2(f0 - __uint_as_float(hi[q] << 16), f1 - __uint_as_float(hi[q] & 0xFFFF0000u));
        }
        tmem_st8(a_addr + c * 8, hi);
        tmem_st8(a_addr + kXS / 2 + c * 8, lo);
      }
      tmem_st_wait();
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&ready[i]);
      if (++i == kWgA) { i = 0; iph ^= 1; }
      if (++st == kWgStages) { st = 0; rph ^= 1; }
    }
    // ---- Fold D into the template gradient ---------------------------------
    volatile int no_abort = 0;
    if (!*abort_flag && mbar_wait(done_bar, 0, &no_abort, kWgSpin)) {
      tc_fence_after();
      // Each builder warp of a sub-partition reads half of the NB columns.
      for (int n0 = half * 16; n0 < NB; n0 += 32) {
        uint32_t v[32];
        tmem_ld16(lane_base + n0, v);
        tmem_ld_wait();
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const int h = ri + p.th - 1 - (n0 + j);
          if (w < p.tw && h >= 0 && h < p.th) atomicAdd(&part[h * p.tw + w], __uint_as_float(v[j]));
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  const int cta = blockIdx.y * gridDim.x + blockIdx.x;
  for (int k = threadIdx.x; k < p.tw * p.th; k += kWgThreads)
    p.partials[(size_t)cta * p.tw * p.th + k] = part[k];
  if (warp == 0) {
    tc_fence_after();
    tmem_dealloc(tmem, kWgCols);
  }
  if (threadIdx.x == 0 && s_abort) atomicExch(p.err, 1);
}

// ---- Element-wise kernels ------------------------------------------------------

// Window sums are separable: a row pass writes horizontal window sums (FP64)
// and the consumer adds th of them down a column (FP64, from L2).
template <typename T, bool SQR>
__global__ void box_rows_kernel(const T* src, size_t src_pitch, int W, int H, int lo, int len,
                                double* out, size_t out_pitch) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y;
  if (x >= W || y >= H) return;
  const T* r = reinterpret_cast<const T*>(reinterpret_cast<const char*>(src) + (size_t)y * src_pitch);
  const int a = max(x + lo, 0), b = min(x + lo + len - 1, W - 1);
  double acc = 0.0;
  for (int i = a; i <= b; ++i) {
    const double v = r[i];
    acc += SQR ? v * v : v;
  }
  reinterpret_cast<double*>(reinterpret_cast<char*>(out) + (size_t)y * out_pitch)[x] = acc;
}

__device__ __forceinline__ double col_sum(const double* Hr, size_t hp, int H, int x, int y0,
                                          int y1) {
  y0 = max(y0, 0);
  y1 = min(y1, H - 1);
  double acc = 0.0;
  for (int j = y0; j <= y1; ++j)
    acc += reinterpret_cast<const double*>(reinterpret_cast<const char*>(Hr) + (size_t)j * hp)[x];
  return acc;
}

struct PrepParams {
  int W, H, tw, th, ax, ay;
  int mw;           // M row length written (incl. the zero pitch tail)
  const double* HS2;  // horizontal window sums of S^2 (forward anchor)
  size_t hs2_pitch;
  const float* G1;  // SqrDistance upstream gradient (or null)
  size_t g1_pitch;
  const float* G2;  // CrossCorr_Norm upstream gradient (or null)
  size_t g2_pitch;
  const float* N2;  // CrossCorr_Norm forward map
  size_t n2_pitch;
  const double* ET;  // template energy
  float* M;
  size_t m_pitch;
  double* P;
  size_t p_pitch;
  double* sums;  // [0] += sum G1, [1] += sum G2 N2
};

template <typename T>
__device__ __forceinline__ T at2(const T* base, size_t pitch, int x, int y) {
  return reinterpret_cast<const T*>(reinterpret_cast<const char*>(base) + (size_t)y * pitch)[x];
}

__global__ void bw_prep_kernel(const PrepParams p) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y;
  double s1 = 0.0, s2 = 0.0;
  if (x < p.mw && y < p.H) {
    float m = 0.f;
    double pp = 0.0;
    if (x < p.W) {
      const double et = *p.ET;
      double g1 = p.G1 ? at2(p.G1, p.g1_pitch, x, y) : 0.0;
      double g2 = p.G2 ? at2(p.G2, p.g2_pitch, x, y) : 0.0;
      m = static_cast<float>(-2.0 * g1);
      pp = 2.0 * g1;
      s1 = g1;
      if (p.G2) {
        const double es = col_sum(p.HS2, p.hs2_pitch, p.H, x, y - p.ay, y - p.ay + p.th - 1);
        const double n = at2(p.N2, p.n2_pitch, x, y);
        if (es > 0.0 && et > 0.0) {
          m = static_cast<float>(-2.0 * g1 + g2 / sqrt(es * et));
          pp = 2.0 * g1 - g2 * n / es;
          s2 = g2 * n;
        }
      }
    }
    reinterpret_cast<float*>(reinterpret_cast<char*>(p.M) + (size_t)y * p.m_pitch)[x] = m;
    if (x < p.W)
      reinterpret_cast<double*>(reinterpret_cast<char*>(p.P) + (size_t)y * p.p_pitch)[x] = pp;
  }
  // Block sums of G1 and G2 N2, then one FP64 atomic per block.
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) {
    s1 += __shfl_xor_sync(0xffffffffu, s1, d);
    s2 += __shfl_xor_sync(0xffffffffu, s2, d);
  }
  __shared__ double b1[8], b2[8];
  const int wi = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) {
    b1[wi] = s1;
    b2[wi] = s2;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double t1 = 0.0, t2 = 0.0;
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) {
      t1 += b1[i];
      t2 += b2[i];
    }
    atomicAdd(&p.sums[0], t1);
    atomicAdd(&p.sums[1], t2);
  }
}

// Template energy (FP64) and the flipped template, one block.
__global__ void bw_template_kernel(const float* T, size_t t_pitch, int tw, int th, float* Tf,
                                   size_t tf_pitch, double* ET) {
  double e = 0.0;
  for (int i = threadIdx.x; i < tw * th; i += blockDim.x) {
    const int h = i / tw, w = i - h * tw;
    const float v = at2(T, t_pitch, w, h);
    e += (double)v * v;
    reinterpret_cast<float*>(reinterpret_cast<char*>(Tf) + (size_t)(th - 1 - h) * tf_pitch)[tw - 1 - w] = v;
  }
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) e += __shfl_xor_sync(0xffffffffu, e, d);
  __shared__ double part[32];
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = e;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) t += part[i];
    *ET = t;
  }
}

// dS(u, v) = Q(u, v) + S(u, v) * sum of P over the adjoint window (HP: the
// horizontal sums of P over [u - tw + 1 + ax, u + ax]).
__global__ void bw_image_grad_kernel(int W, int H, int tw, int th, int ax, int ay, const float* S,
                                     size_t s_pitch, const float* Q, size_t q_pitch,
                                     const double* HP, size_t hp_pitch, char* dS, size_t ds_pitch,
                                     int ds_f64) {
  const int u = blockIdx.x * blockDim.x + threadIdx.x;
  const int v = blockIdx.y;
  if (u >= W || v >= H) return;
  const double b = col_sum(HP, hp_pitch, H, u, v - th + 1 + ay, v + ay);
  const double g = (double)at2(Q, q_pitch, u, v) + (double)at2(S, s_pitch, u, v) * b;
  if (ds_f64)
    reinterpret_cast<double*>(dS + (size_t)v * ds_pitch)[u] = g;
  else
    reinterpret_cast<float*>(dS + (size_t)v * ds_pitch)[u] = static_cast<float>(g);
}

// dT(w, h) = sum of the CTA partials (FP64) + T(w, h) (2 sum G1 - sum G2 N2 / E_T).
// A block takes 32 entries; its 8 warps split the partials.
__global__ void bw_template_grad_kernel(int tw, int th, int nparts, const float* partials,
                                        const float* T, size_t t_pitch, const double* sums,
                                        const double* ET, char* dT, size_t dt_pitch, int dt_f64) {
  const int k = blockIdx.x * 32 + (threadIdx.x & 31);
  const int wi = threadIdx.x >> 5;
  double acc = 0.0;
  if (k < tw * th)
    for (int c = wi; c < nparts; c += 8) acc += partials[(size_t)c * tw * th + k];
  __shared__ double red[8][32];
  red[wi][threadIdx.x & 31] = acc;
  __syncthreads();
  if (wi != 0 || k >= tw * th) return;
  acc = 0.0;
  for (int i = 0; i < 8; ++i) acc += red[i][threadIdx.x & 31];
  const int h = k / tw, w = k - h * tw;
  const double et = *ET;
  const double coef = 2.0 * sums[0] - (et > 0.0 ? sums[1] / et : 0.0);
  const double g = acc + (double)at2(T, t_pitch, w, h) * coef;
  if (dt_f64)
    reinterpret_cast<double*>(dT + (size_t)h * dt_pitch)[w] = g;
  else
    reinterpret_cast<float*>(dT + (size_t)h * dt_pitch)[w] = static_cast<float>(g);
}

typedef CUresult (*EncodeFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                             const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                             const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                             CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeFn wg_encode() {
  static EncodeFn fn = nullptr;
  if (!fn) {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeFn>(f);
  }
  return fn;
}

// Band rows of the weight-gradient grid: the tallest band (fewer partials,
// less staging per row) that still gives most SMs a CTA.
int wg_band_rows(int W, int H, int PR, int sm_count) {
  const int nstrips = (W + kXS - 1) / kXS;
  int BR = kBRmax;
  while (BR > 4 * PR && (long long)nstrips * ((H + BR - 1) / BR) * 5 < sm_count * 4) BR /= 2;
  return BR;
}

template <int PR>
cudaError_t launch_wgrad(Context& ctx, const DevImage& S, int tw, int th, const float* M,
                         size_t m_pitch, float* partials, int* nparts) {
  WgParams p;
  p.W = S.width;
  p.H = S.height;
  p.tw = tw;
  p.th = th;
  p.ax = tw / 2;
  p.ay = th / 2;
  p.lead = (4 - p.ax % 4) % 4;
  // Lane window: pixels lead + w .. lead + w + 128 (+1 for odd starts).
  p.nbox = (p.lead + WgCfg<PR>::WP + kXS + 1 + 3) / 4;
  p.M = M;
  p.m_pitch = m_pitch;
  p.partials = partials;
  p.err = reinterpret_cast<int*>(ctx.scratch(Context::kTensorAux, 256));
  EncodeFn enc = wg_encode();
  if (!enc) return cudaErrorNotSupported;
  CUtensorMap map;
  const cuuint64_t gdim[4] = {4, (cuuint64_t)((p.W + 3) / 4), (cuuint64_t)p.H, 1};
  const cuuint64_t gstride[3] = {16, (cuuint64_t)S.pitch, (cuuint64_t)S.pitch * p.H};
  const cuuint32_t box[4] = {4, (cuuint32_t)p.nbox, (cuuint32_t)PR, 1};
  const cuuint32_t estr[4] = {1, 1, 1, 1};
  if (enc(&map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, S.ptr, gdim, gstride, box, estr,
          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
          CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
    return cudaErrorInvalidValue;
  const int nstrips = (p.W + kXS - 1) / kXS;
  p.BR = wg_band_rows(p.W, p.H, PR, ctx.sm_count);
  const int NB = (th + PR - 1 + 15) / 16 * 16;
  const WgLayout L = wg_layout<PR>(p.nbox, NB, tw, th, p.BR);
  auto kern = wgrad_kernel<PR>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, L.total);
  if (e != cudaSuccess) return e;
  dim3 grid(nstrips, (p.H + p.BR - 1) / p.BR);
  *nparts = grid.x * grid.y;
  kern<<<grid, kWgThreads, L.total, ctx.stream>>>(map, p);
  count_launches(1);
  return cudaGetLastError();
}

size_t pitch_of(int W, int bytes) { return ((size_t)W * bytes + 127) / 128 * 128; }

}  // namespace

cudaError_t proximity_backward(Context& ctx, const DevImage& S, const DevImage& T,
                               const DevImage* G1, const DevImage* G2, const DevImage* N2,
                               const DevImage* dS, const DevImage* dT) {
  const int W = S.width, H = S.height, tw = T.width, th = T.height;
  const int ax = tw / 2, ay = th / 2;
  // Scratch: row window sums HS2 / HP and the map P (FP64), M and Q (F32),
  // flipped template, template energy and sums, weight-gradient partials.
  const size_t p8 = pitch_of(W, 8), p4 = pitch_of(W, 4);
  const size_t tfp = pitch_of(tw, 4);
  const int PR = tw <= 32 ? 4 : 2;
  const size_t nparts =
      (size_t)((W + kXS - 1) / kXS) * ((H + wg_band_rows(W, H, PR, ctx.sm_count) - 1) /
                                        wg_band_rows(W, H, PR, ctx.sm_count));
  size_t off = 0;
  auto take = [&](size_t bytes) {
    const size_t o = off;
    off += (bytes + 255) / 256 * 256;
    return o;
  };
  const size_t o_hs2 = take(p8 * H), o_p = take(p8 * H), o_hp = take(p8 * H);
  const size_t o_m = take(p4 * H), o_q = take(p4 * H), o_tf = take(tfp * th);
  const size_t o_sc = take(64), o_part = take(nparts * tw * th * 4);
  char* base = reinterpret_cast<char*>(ctx.scratch(Context::kBackward, off));
  double* scal = reinterpret_cast<double*>(base + o_sc);  // [0] E_T, [1] sum G1, [2] sum G2 N2
  cudaError_t e = cudaMemsetAsync(scal, 0, 64, ctx.stream);
  if (e != cudaSuccess) return e;
  const dim3 rows((W + 255) / 256, H);

  bw_template_kernel<<<1, 256, 0, ctx.stream>>>((const float*)T.ptr, T.pitch, tw, th,
                                                 (float*)(base + o_tf), tfp, scal);
  count_launches(1);
  double* hs2 = (double*)(base + o_hs2);
  if (G2) {
    box_rows_kernel<float, true><<<rows, 256, 0, ctx.stream>>>((const float*)S.ptr, S.pitch, W,
                                                               H, -ax, tw, hs2, p8);
    count_launches(1);
  }

  PrepParams pp;
  pp.W = W;
  pp.H = H;
  pp.tw = tw;
  pp.th = th;
  pp.ax = ax;
  pp.ay = ay;
  pp.mw = (int)(p4 / 4);
  pp.HS2 = hs2;
  pp.hs2_pitch = p8;
  pp.G1 = G1 ? (const float*)G1->ptr : nullptr;
  pp.g1_pitch = G1 ? G1->pitch : 0;
  pp.G2 = G2 ? (const float*)G2->ptr : nullptr;
  pp.g2_pitch = G2 ? G2->pitch : 0;
  pp.N2 = N2 ? (const float*)N2->ptr : nullptr;
  pp.n2_pitch = N2 ? N2->pitch : 0;
  pp.ET = scal;
  pp.M = (float*)(base + o_m);
  pp.m_pitch = p4;
  pp.P = (double*)(base + o_p);
  pp.p_pitch = p8;
  pp.sums = scal + 1;
  const dim3 eg((pp.mw + 255) / 256, H);
  bw_prep_kernel<<<eg, 256, 0, ctx.stream>>>(pp);
  count_launches(1);

  if (dS) {
    // Q = correlation of M with the flipped template, adjoint anchor.
    DevImage m{pp.M, p4, W, H, 1, F32};
    DevImage tf{base + o_tf, tfp, tw, th, 1, F32};
    DevImage q{base + o_q, p4, W, H, 1, F32};
    e = launch_proximity_tensor_anchored(ctx, kCrossCorr, m, tf, q, tw - 1 - ax, th - 1 - ay);
    if (e != cudaSuccess) return e;
    double* hp = (double*)(base + o_hp);
    box_rows_kernel<double, false><<<rows, 256, 0, ctx.stream>>>(pp.P, p8, W, H, ax - tw + 1, tw,
                                                                 hp, p8);
    count_launches(1);
    bw_image_grad_kernel<<<rows, 256, 0, ctx.stream>>>(W, H, tw, th, ax, ay, (const float*)S.ptr,
                                                        S.pitch, (const float*)q.ptr, p4, hp, p8,
                                                        (char*)dS->ptr, dS->pitch,
                                                        dS->type == F64);
    count_launches(1);
  }
  if (dT) {
    int np = 0;
    float* parts = reinterpret_cast<float*>(base + o_part);
    e = PR == 4 ? launch_wgrad<4>(ctx, S, tw, th, pp.M, p4, parts, &np)
                : launch_wgrad<2>(ctx, S, tw, th, pp.M, p4, parts, &np);
    if (e != cudaSuccess) return e;
    bw_template_grad_kernel<<<(tw * th + 31) / 32, 256, 0, ctx.stream>>>(
        tw, th, np, parts, (const float*)T.ptr, T.pitch, scal + 1, scal, (char*)dT->ptr,
        dT->pitch, dT->type == F64);
    count_launches(1);
  }
  return cudaGetLastError();
}

}  // namespace ocipb
