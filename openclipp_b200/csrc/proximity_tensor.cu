// Tensor-core (tcgen05) ImageProximity path for sm_100a.
//
// The product term of SqrDistance[_Norm] and CrossCorr[_Norm]
// (cl-files/ImageProximity.cl :44, :122, :290, :375),
//   C(x, y) = sum_h sum_w S(x + w - tw/2, y + h - th/2) * T(w, h),
// is computed as one small GEMM per source row r and 128-column strip:
//   D_r[m][n] = sum_k A_r[m][k] * B[n][k],  A_r[m][k] = S(x0 + m + k - tw/2, r),
//   B[n][k] = T(k, n - (R - th)) (template rows in N, zero rows on top),
// M = 128 output positions, N = R (th rounded up to 16/32/64), K = tw rounded
// up. Then C(x0 + m, y) = sum_n D_{y + n - off}[m][n], off = R - th + th/2:
// every source row contributes to R output rows, one per template row. The
// epilogue thread of lane m keeps those R partial sums in a register ring and
// emits output row y as soon as its last template row has been added.
//
// A_r is a Hankel (sliding-window) matrix. In the canonical K-major
// SWIZZLE_NONE layout, core matrix (mb, kb) holds
// S(x0 + 8(mb + kb) + row + j); it depends on mb + kb only. So A_r is given to
// the tensor core as a descriptor with LBO = SBO = 128 bytes over an array of
// 16 + K/8 - 1 core matrices, row q of which holds pixels q .. q+7: an 8x
// expansion of the source row built in shared memory, instead of the 32x
// (K-fold) expansion of an explicit im2col. For 8-bit sources (16 elements
// per core-matrix row) the same holds with LBO = 256, SBO = 128.
//
// Precision. U8 sources use the i8 MMA with s32 accumulation: every product
// term is exact and so are the results. F32 sources are split into BF16 hi + lo
// parts (S = S_hi + S_lo + O(2^-18 S)); three MMAs (hi*hi, hi*lo, lo*hi)
// accumulate in FP32 in TMEM. The window energy sum S^2 of each output comes
// from FP64 running sums fused into the kernel (per row: a prefix sum over the
// staged row gives the row-window sums; per column: a running sum over rows
// and its value th rows earlier), the template energy is exact in FP64, and
// SqrDistance = E_S - 2C + E_T and the _Norm divisions are done in FP64.
//
// Roles (256 threads): warp 0 issues TMA loads of source rows (zero fill
// outside the image), warp 1 allocates TMEM and issues the MMAs, warps 2-3
// build the Hankel operands and row energies, warps 4-7 (TMEM lanes 0-127)
// run the epilogue. Stages are chained by mbarriers; every wait is bounded
// and sets an error flag instead of hanging.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <type_traits>

#include "sm100.cuh"
#include "tensor.h"

namespace ocipb {
namespace {

using namespace sm100;

constexpr int kM = 128;
constexpr int kThreads = 256;
constexpr int kRawRows = 4;
constexpr int kNRaw = 4;
constexpr int kNQ = 8;
constexpr int kSTM = 4;
constexpr int kG = 8;  // epilogue output staging depth (steps)
constexpr long long kSpinLimit = 4000000000LL;  // about 2 s of SM clock

enum Elem { kF32 = 0, kU8 = 1 };

struct TensorParams {
  int W, H;
  int tw, th;
  int K;         // padded template width
  int nblk;      // core-matrix blocks per Hankel array
  int boxw;      // TMA box width (elements) = 128 + K
  int xshift;    // strip b covers outputs [128 b - xshift, 128 b - xshift + 128)
  int left0;     // tw / 2
  int off;       // R - th + th / 2
  int BH;        // output rows per band
  int measure;
  int norm_float;  // U8 _Norm: float arithmetic as the plain path (exact sums)
  const char* tmpl;
  size_t tmpl_pitch;
  char* dst;
  size_t dst_pitch;
  int dst_f64;
  int* err;
};

// Shared-memory layout, identical on host and device.
struct Layout {
  int raw_stage, raw, q_arr, q_stage, q, b_arr, b, pre, cum, stg, bars, total;
};

__host__ __device__ inline int align128(int x) { return (x + 127) & ~127; }

__host__ __device__ inline Layout make_layout(int elem, int R, int K, int nblk, int boxw) {
  Layout L;
  const int esz = elem == kF32 ? 4 : 1;
  const int narr = elem == kF32 ? 2 : 1;
  L.raw_stage = align128(kRawRows * boxw * esz);
  L.raw = 0;
  L.q_arr = nblk * 128;
  L.q_stage = align128(narr * L.q_arr + kM * 8);
  L.q = L.raw + kNRaw * L.raw_stage;
  L.b_arr = R * K * (elem == kF32 ? 2 : 1);
  L.b = L.q + kNQ * L.q_stage;
  L.pre = L.b + align128(narr * L.b_arr);
  L.cum = L.pre + align128(2 * (boxw + 8) * 8);
  L.stg = L.cum + R * kM * 8;
  L.bars = L.stg + kG * kM * 16;
  // mbarriers (2 per raw, operand and TMEM stage, plus one), then the TMEM
  // address, the abort flag and the template energy.
  L.total = L.bars + align128(8 * (2 * kNRaw + 2 * kNQ + 2 * kSTM + 1) + 32);
  return L;
}

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
  __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<uint32_t*>(&v);
}
__device__ __forceinline__ float bf16lo_f(uint32_t w) { return __uint_as_float(w << 16); }
__device__ __forceinline__ float bf16hi_f(uint32_t w) { return __uint_as_float(w & 0xFFFF0000u); }

// Row `rr` (0..7) of a BF16 core-matrix block: pixels rr..rr+7 of the 16
// pixels held in w[0..3] (this lane's 8) and n[0..3] (the next lane's 8).
template <int RR>
__device__ __forceinline__ uint4 hankel_row_bf16(const uint32_t (&w)[4], const uint32_t (&n)[4]) {
  uint32_t c[8] = {w[0], w[1], w[2], w[3], n[0], n[1], n[2], n[3]};
  constexpr int a = RR / 2;
  if (RR % 2 == 0) return make_uint4(c[a], c[a + 1], c[a + 2], c[a + 3]);
  return make_uint4(__byte_perm(c[a], c[a + 1], 0x5432), __byte_perm(c[a + 1], c[a + 2], 0x5432),
                    __byte_perm(c[a + 2], c[a + 3], 0x5432), __byte_perm(c[a + 3], c[a + 4], 0x5432));
}

// Row `rr` (0..7) of a U8 core-matrix block: bytes rr..rr+15 of the 24 bytes
// in c[0..5].
template <int RR>
__device__ __forceinline__ uint4 hankel_row_u8(const uint32_t (&c)[6]) {
  constexpr int a = RR / 4, sh = RR % 4;
  constexpr uint32_t sel = sh == 1 ? 0x4321 : sh == 2 ? 0x5432 : 0x6543;
  if (sh == 0) return make_uint4(c[a], c[a + 1], c[a + 2], c[a + 3]);
  return make_uint4(__byte_perm(c[a], c[a + 1], sel), __byte_perm(c[a + 1], c[a + 2], sel),
                    __byte_perm(c[a + 2], c[a + 3], sel), __byte_perm(c[a + 3], c[a + 4], sel));
}

template <int ELEM, int R>
__global__ void __launch_bounds__(kThreads, 1)
    prox_tensor_kernel(const __grid_constant__ CUtensorMap tmap, const TensorParams p) {
  extern __shared__ __align__(1024) unsigned char smem[];
  const Layout L = make_layout(ELEM, R, p.K, p.nblk, p.boxw);
  constexpr int kTmemCols = (kSTM * R < 32) ? 32 : kSTM * R;
  constexpr int ESZ = ELEM == kF32 ? 4 : 1;

  uint64_t* raw_full = reinterpret_cast<uint64_t*>(smem + L.bars);
  uint64_t* raw_empty = raw_full + kNRaw;
  uint64_t* q_full = raw_empty + kNRaw;
  uint64_t* q_empty = q_full + kNQ;
  uint64_t* tm_full = q_empty + kNQ;
  uint64_t* tm_empty = tm_full + kSTM;
  uint64_t* done_bar = tm_empty + kSTM;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done_bar + 1);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);
  double* s_et = reinterpret_cast<double*>(tmem_slot + 2);

  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const bool need_e = p.measure != kCrossCorr;
  const int xs_out = blockIdx.x * kM - p.xshift;
  const int y0 = blockIdx.y * p.BH;
  const int yend = min(p.H, y0 + p.BH);
  const int r_begin = y0 - p.off;
  const int nsteps = (yend - y0) + R - 1;

  if (threadIdx.x == 0) {
    for (int i = 0; i < kNRaw; ++i) {
      mbar_init(&raw_full[i], 1);
      mbar_init(&raw_empty[i], kRawRows);
    }
    for (int i = 0; i < kNQ; ++i) {
      mbar_init(&q_full[i], 1);
      mbar_init(&q_empty[i], 1 + 4);
    }
    for (int i = 0; i < kSTM; ++i) {
      mbar_init(&tm_full[i], 1);
      mbar_init(&tm_empty[i], 4);
    }
    mbar_init(done_bar, 1);
    *abort_flag = 0;
    fence_barrier_init();
  }
  if (warp == 1) tmem_alloc(tmem_slot, kTmemCols);

  // Template operand B (N = R rows, zero rows on top) and its energy.
  {
    const int padrows = R - p.th;
    for (int idx = threadIdx.x; idx < R * p.K; idx += kThreads) {
      const int n = idx / p.K, k = idx - n * p.K;
      const int h = n - padrows;
      if (ELEM == kF32) {
        float t = 0.f;
        if (h >= 0 && k < p.tw)
          t = reinterpret_cast<const float*>(p.tmpl + (size_t)h * p.tmpl_pitch)[k];
        const __nv_bfloat16 th_ = __float2bfloat16_rn(t);
        const __nv_bfloat16 tl_ = __float2bfloat16_rn(t - __bfloat162float(th_));
        const int off = ((k >> 3) * R + n) * 16 + (k & 7) * 2;
        *reinterpret_cast<__nv_bfloat16*>(smem + L.b + off) = th_;
        *reinterpret_cast<__nv_bfloat16*>(smem + L.b + L.b_arr + off) = tl_;
      } else {
        uint8_t t = 0;
        if (h >= 0 && k < p.tw)
          t = reinterpret_cast<const uint8_t*>(p.tmpl + (size_t)h * p.tmpl_pitch)[k];
        const int off = ((k >> 4) * R + n) * 16 + (k & 15);
        smem[L.b + off] = t;
      }
    }
    if (warp == 2) {
      double e = 0.0;
      for (int idx = lane; idx < p.th * p.tw; idx += 32) {
        const int h = idx / p.tw, k = idx - h * p.tw;
        double t;
        if (ELEM == kF32)
          t = reinterpret_cast<const float*>(p.tmpl + (size_t)h * p.tmpl_pitch)[k];
        else
          t = reinterpret_cast<const uint8_t*>(p.tmpl + (size_t)h * p.tmpl_pitch)[k];
        e += t * t;
      }
#pragma unroll
      for (int d = 16; d > 0; d >>= 1) e += __shfl_xor_sync(0xffffffffu, e, d);
      if (lane == 0) *s_et = e;
    }
  }
  fence_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;

  if (warp == 0) {
    // ---- TMA producer -------------------------------------------------------
    if (lane == 0) {
      tma_prefetch_desc(&tmap);
      const int nb = (nsteps + kRawRows - 1) / kRawRows;
      const int xt = xs_out - p.left0;
      int issued = 0;
      for (int b = 0; b < nb; ++b) {
        const int st = b % kNRaw;
        if (!mbar_wait(&raw_empty[st], ((b / kNRaw) & 1) ^ 1, abort_flag, kSpinLimit)) break;
        mbar_arrive_expect_tx(&raw_full[st], kRawRows * p.boxw * ESZ);
        tma_load_2d(smem + L.raw + st * L.raw_stage, &tmap, xt, r_begin + b * kRawRows,
                    &raw_full[st]);
        issued = b + 1;
      }
      // Every load this thread issued has landed before the CTA exits.
      for (int b = max(0, issued - kNRaw); b < issued; ++b) {
        volatile int no_abort = 0;
        mbar_wait(&raw_full[b % kNRaw], (b / kNRaw) & 1, &no_abort, kSpinLimit);
      }
    }
  } else if (warp == 1) {
    // ---- MMA issuer -----------------------------------------------------------
    if (lane == 0) {
      const uint32_t q0 = smem_u32(smem + L.q);
      const uint32_t b0 = smem_u32(smem + L.b);
      for (int s = 0; s < nsteps; ++s) {
        const int qs = s % kNQ, ts = s % kSTM;
        if (!mbar_wait(&q_full[qs], (s / kNQ) & 1, abort_flag, kSpinLimit)) break;
        if (!mbar_wait(&tm_empty[ts], ((s / kSTM) & 1) ^ 1, abort_flag, kSpinLimit)) break;
        tc_fence_after();
        const uint32_t d = tmem_base + ts * R;
        const uint32_t qa = q0 + qs * L.q_stage;
        if (ELEM == kF32) {
          constexpr uint32_t idesc = idesc_bf16_f32(kM, R);
          const uint32_t qlo = qa + L.q_arr;
          const uint32_t blo = b0 + L.b_arr;
          const int nk = p.K / 16;
          for (int kk = 0; kk < nk; ++kk)
            mma_bf16(d, smem_desc(qa + kk * 256, 128, 128),
                     smem_desc(b0 + kk * 2 * R * 16, R * 16, 128), idesc, kk > 0);
          for (int kk = 0; kk < nk; ++kk)
            mma_bf16(d, smem_desc(qa + kk * 256, 128, 128),
                     smem_desc(blo + kk * 2 * R * 16, R * 16, 128), idesc, 1);
          for (int kk = 0; kk < nk; ++kk)
            mma_bf16(d, smem_desc(qlo + kk * 256, 128, 128),
                     smem_desc(b0 + kk * 2 * R * 16, R * 16, 128), idesc, 1);
        } else {
          constexpr uint32_t idesc = idesc_u8_s32(kM, R);
          const int nk = p.K / 32;
          for (int kk = 0; kk < nk; ++kk)
            mma_i8(d, smem_desc(qa + kk * 512, 256, 128),
                   smem_desc(b0 + kk * 2 * R * 16, R * 16, 128), idesc, kk > 0);
        }
        mma_commit(&tm_full[ts]);
        mma_commit(&q_empty[qs]);
      }
      // Every MMA this thread issued has completed before TMEM is freed.
      mma_commit(done_bar);
      volatile int no_abort = 0;
      mbar_wait(done_bar, 0, &no_abort, kSpinLimit);
    }
  } else if (warp < 4) {
    // ---- Hankel operand + row-energy builders ----------------------------------
    const int pw = warp - 2;
    double* pre = reinterpret_cast<double*>(smem + L.pre) + pw * (p.boxw + 8);
    const int epl = (p.boxw + 31) / 32;
    for (int s = pw; s < nsteps; s += 2) {
      const int b = s / kRawRows, st = b % kNRaw, rr = s % kRawRows;
      const int qs = s % kNQ;
      if (!mbar_wait(&raw_full[st], (b / kNRaw) & 1, abort_flag, kSpinLimit)) break;
      if (!mbar_wait(&q_empty[qs], ((s / kNQ) & 1) ^ 1, abort_flag, kSpinLimit)) break;
      const unsigned char* row = smem + L.raw + st * L.raw_stage + rr * p.boxw * ESZ;
      unsigned char* qst = smem + L.q + qs * L.q_stage;
      const int t = lane;
      if (ELEM == kF32) {
        uint32_t hi[4] = {0, 0, 0, 0}, lo[4] = {0, 0, 0, 0};
        if (t <= p.nblk) {
          const float4 a = reinterpret_cast<const float4*>(row)[2 * t];
          const float4 c = reinterpret_cast<const float4*>(row)[2 * t + 1];
          const float f[8] = {a.x, a.y, a.z, a.w, c.x, c.y, c.z, c.w};
#pragma unroll
          for (int j = 0; j < 4; ++j) {
            hi[j] = pack_bf16(f[2 * j], f[2 * j + 1]);
            lo[j] = pack_bf16(f[2 * j] - bf16lo_f(hi[j]), f[2 * j + 1] - bf16hi_f(hi[j]));
          }
        }
        uint32_t hn[4], ln[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          hn[j] = __shfl_down_sync(0xffffffffu, hi[j], 1);
          ln[j] = __shfl_down_sync(0xffffffffu, lo[j], 1);
        }
        if (t < p.nblk) {
          uint4* qh = reinterpret_cast<uint4*>(qst + t * 128);
          uint4* ql = reinterpret_cast<uint4*>(qst + L.q_arr + t * 128);
          qh[0] = hankel_row_bf16<0>(hi, hn); ql[0] = hankel_row_bf16<0>(lo, ln);
          qh[1] = hankel_row_bf16<1>(hi, hn); ql[1] = hankel_row_bf16<1>(lo, ln);
          qh[2] = hankel_row_bf16<2>(hi, hn); ql[2] = hankel_row_bf16<2>(lo, ln);
          qh[3] = hankel_row_bf16<3>(hi, hn); ql[3] = hankel_row_bf16<3>(lo, ln);
          qh[4] = hankel_row_bf16<4>(hi, hn); ql[4] = hankel_row_bf16<4>(lo, ln);
          qh[5] = hankel_row_bf16<5>(hi, hn); ql[5] = hankel_row_bf16<5>(lo, ln);
          qh[6] = hankel_row_bf16<6>(hi, hn); ql[6] = hankel_row_bf16<6>(lo, ln);
          qh[7] = hankel_row_bf16<7>(hi, hn); ql[7] = hankel_row_bf16<7>(lo, ln);
        }
      } else {
        uint32_t w[2] = {0, 0};
        if (t <= p.nblk + 1) {
          const uint2 v = reinterpret_cast<const uint2*>(row)[t];
          w[0] = v.x;
          w[1] = v.y;
        }
        uint32_t c[6];
        c[0] = w[0];
        c[1] = w[1];
        c[2] = __shfl_down_sync(0xffffffffu, w[0], 1);
        c[3] = __shfl_down_sync(0xffffffffu, w[1], 1);
        c[4] = __shfl_down_sync(0xffffffffu, w[0], 2);
        c[5] = __shfl_down_sync(0xffffffffu, w[1], 2);
        if (t < p.nblk) {
          uint4* q = reinterpret_cast<uint4*>(qst + t * 128);
          q[0] = hankel_row_u8<0>(c);
          q[1] = hankel_row_u8<1>(c);
          q[2] = hankel_row_u8<2>(c);
          q[3] = hankel_row_u8<3>(c);
          q[4] = hankel_row_u8<4>(c);
          q[5] = hankel_row_u8<5>(c);
          q[6] = hankel_row_u8<6>(c);
          q[7] = hankel_row_u8<7>(c);
        }
      }
      if (need_e) {
        // Prefix sums of S^2 over the staged row, then the row-window sums
        // rs[m] = sum_{w < tw} S(m + w)^2 for the 128 positions.
        double run = 0.0;
        double vals[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) {
          const int j = lane * epl + k;
          double v = 0.0;
          if (k < epl && j < p.boxw) {
            v = ELEM == kF32 ? (double)reinterpret_cast<const float*>(row)[j]
                             : (double)row[j];
            v = v * v;
          }
          run += v;
          vals[k] = run;
        }
        double incl = run;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
          const double o = __shfl_up_sync(0xffffffffu, incl, d);
          if (lane >= d) incl += o;
        }
        const double excl = incl - run;
        if (lane == 0) pre[0] = 0.0;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
          const int j = lane * epl + k;
          if (k < epl && j < p.boxw) pre[j + 1] = excl + vals[k];
        }
        __syncwarp();
        double* rs = reinterpret_cast<double*>(qst + (ELEM == kF32 ? 2 : 1) * L.q_arr);
#pragma unroll
        for (int j = 0; j < kM / 32; ++j) {
          const int m = lane + 32 * j;
          rs[m] = pre[m + p.tw] - pre[m];
        }
      }
      fence_async_smem();
      __syncwarp();
      if (lane == 0) {
        mbar_arrive(&raw_empty[st]);
        mbar_arrive(&q_full[qs]);
      }
    }
  } else {
    // ---- Epilogue: ring accumulation, window energy, output -----------------------
    const int ew = warp - 4;
    const int m = ew * 32 + lane;
    const int x = xs_out + m;
    const bool x_ok = (x >= 0 && x < p.W);
    // U8: exact integers carried in double (the s32 MMA results and their sums
    // stay far below 2^53).
    typedef typename std::conditional<ELEM == kF32, float, double>::type AT;
    AT acc[R];
#pragma unroll
    for (int i = 0; i < R; ++i) acc[i] = AT(0);
    double cum = 0.0;
    double* cumring = reinterpret_cast<double*>(smem + L.cum);
    const double et = *s_et;
    const uint32_t lane_addr = tmem_base + (static_cast<uint32_t>(ew * 32) << 16);
    AT* stage_v = reinterpret_cast<AT*>(smem + L.stg);
    double* stage_e = reinterpret_cast<double*>(smem + L.stg + kG * kM * 8);
    // Output of the completed rows staged in shared memory (kG steps at a
    // time): keeps the unrolled ring loop small.
    auto flush = [&](int sbase, int cnt) {
#pragma unroll 1
      for (int j = 0; j < cnt; ++j) {
        const int yd = r_begin + sbase + j + p.off - R + 1;
        if (yd < y0 || yd >= yend || !x_ok) continue;
        const AT a = stage_v[j * kM + m];
        const double e = stage_e[j * kM + m];
        double outd;
        float outf;
        if (ELEM == kF32) {
          const double cc = (double)a;
          if (p.measure == kCrossCorr) outd = cc;
          else if (p.measure == kSqrDistance) outd = e - 2.0 * cc + et;
          else if (p.measure == kCrossCorrNorm) outd = __ddiv_rn(cc, __dsqrt_rn(__dmul_rn(e, et)));
          else outd = __ddiv_rn(e - 2.0 * cc + et, __dsqrt_rn(__dmul_rn(e, et)));
          outf = (float)outd;
        } else {
          const long long cc = (long long)a;
          const long long es = (long long)e, ei = (long long)et;
          const long long num =
              (p.measure == kCrossCorr || p.measure == kCrossCorrNorm) ? cc : es - 2 * cc + ei;
          if (p.measure == kCrossCorr || p.measure == kSqrDistance) {
            outd = (double)num;
            outf = __ll2float_rn(num);
          } else if (p.norm_float) {
            outf = __fdiv_rn((float)num, __fsqrt_rn(__fmul_rn((float)es, (float)ei)));
            outd = outf;
          } else {
            outd = __ddiv_rn((double)num, __dsqrt_rn(__dmul_rn((double)es, (double)ei)));
            outf = (float)outd;
          }
        }
        char* o = p.dst + (size_t)yd * p.dst_pitch;
        if (p.dst_f64)
          reinterpret_cast<double*>(o)[x] = outd;
        else
          reinterpret_cast<float*>(o)[x] = outf;
      }
    };
    bool ok = true;
    for (int s0 = 0; s0 < nsteps && ok; s0 += R) {
#pragma unroll
      for (int i = 0; i < R; ++i) {
        const int s = s0 + i;
        if (s >= nsteps || !ok) break;
        const int ts = s % kSTM, qs = s % kNQ;
        if (!mbar_wait(&tm_full[ts], (s / kSTM) & 1, abort_flag, kSpinLimit)) {
          ok = false;
          break;
        }
        tc_fence_after();
#pragma unroll
        for (int c = 0; c < (R + 31) / 32; ++c) {
          uint32_t v[32];
          if (R >= 32)
            tmem_ld32(lane_addr + ts * R + c * 32, v);
          else
            tmem_ld16(lane_addr + ts * R, v);
          tmem_ld_wait();
#pragma unroll
          for (int j = 0; j < 32; ++j) {
            const int n = c * 32 + j;
            if (n < R) {
              if (ELEM == kF32)
                acc[(i - n + R) % R] += __uint_as_float(v[j]);
              else
                acc[(i - n + R) % R] += (double)static_cast<int>(v[j]);
            }
          }
        }
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(&tm_empty[ts]);
        double e = 0.0;
        if (need_e) {
          if (!mbar_wait(&q_full[qs], (s / kNQ) & 1, abort_flag, kSpinLimit)) {
            ok = false;
            break;
          }
          const double* rs =
              reinterpret_cast<const double*>(smem + L.q + qs * L.q_stage +
                                              (ELEM == kF32 ? 2 : 1) * L.q_arr);
          cum += rs[m];
          const double old = (s >= p.th) ? cumring[((s - p.th) % R) * kM + m] : 0.0;
          cumring[(s % R) * kM + m] = cum;
          e = cum - old;
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&q_empty[qs]);
        const int g = i % kG;
        const int slot = (i + 1) % R;
        stage_v[g * kM + m] = acc[slot];
        stage_e[g * kM + m] = e;
        acc[slot] = AT(0);
        if (g == kG - 1) flush(s - (kG - 1), kG);
      }
    }
    if (ok && (nsteps % kG) != 0) flush(nsteps - nsteps % kG, nsteps % kG);
  }

  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    tmem_dealloc(tmem_base, kTmemCols);
  }
  if (threadIdx.x == 0 && *abort_flag) atomicExch(p.err, 1);
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                  const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                  const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  if (!fn) {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(f);
  }
  return fn;
}

int ring_size(int th) { return th <= 16 ? 16 : th <= 32 ? 32 : 64; }

template <int ELEM, int R>
cudaError_t launch_elem(Context& ctx, Measure m, const DevImage& src, const DevImage& tmpl,
                        const DevImage& dst) {
  TensorParams p;
  p.W = src.width;
  p.H = src.height;
  p.tw = tmpl.width;
  p.th = tmpl.height;
  p.K = ELEM == kF32 ? (p.tw + 15) / 16 * 16 : (p.tw + 31) / 32 * 32;
  p.nblk = ELEM == kF32 ? 15 + p.K / 8 : 14 + p.K / 8;
  p.boxw = kM + p.K;
  p.left0 = p.tw / 2;
  const int align = ELEM == kF32 ? 4 : 16;
  p.xshift = ((p.left0 % align) == 0) ? 0 : align - (p.left0 % align);
  p.off = R - p.th + p.th / 2;
  p.BH = p.H >= 2048 ? 512 : std::max(64, (p.H + 3) / 4);
  p.measure = m;
  p.norm_float = (double)p.tw * p.th * 65025.0 <= 16777216.0;
  p.tmpl = (const char*)tmpl.ptr;
  p.tmpl_pitch = tmpl.pitch;
  p.dst = (char*)dst.ptr;
  p.dst_pitch = dst.pitch;
  p.dst_f64 = dst.type == F64;
  p.err = reinterpret_cast<int*>(ctx.scratch(Context::kTensorAux, 256));

  EncodeTiledFn enc = encode_fn();
  if (!enc) return cudaErrorNotSupported;
  CUtensorMap map;
  const cuuint64_t gdim[2] = {(cuuint64_t)p.W, (cuuint64_t)p.H};
  const cuuint64_t gstride[1] = {(cuuint64_t)src.pitch};
  const cuuint32_t box[2] = {(cuuint32_t)p.boxw, (cuuint32_t)kRawRows};
  const cuuint32_t estride[2] = {1, 1};
  CUresult r = enc(&map, ELEM == kF32 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_UINT8,
                   2, src.ptr, gdim, gstride, box, estride, CU_TENSOR_MAP_INTERLEAVE_NONE,
                   CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return cudaErrorInvalidValue;

  const Layout L = make_layout(ELEM, R, p.K, p.nblk, p.boxw);
  auto kern = prox_tensor_kernel<ELEM, R>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, L.total);
  if (e != cudaSuccess) return e;
  const int nstrips = (p.W + p.xshift + kM - 1) / kM;
  const int nbands = (p.H + p.BH - 1) / p.BH;
  dim3 grid(nstrips, nbands, 1);
  kern<<<grid, kThreads, L.total, ctx.stream>>>(map, p);
  count_launches(1);
  return cudaGetLastError();
}

template <int ELEM>
cudaError_t launch_r(Context& ctx, Measure m, const DevImage& s, const DevImage& t,
                     const DevImage& d) {
  switch (ring_size(t.height)) {
    case 16: return launch_elem<ELEM, 16>(ctx, m, s, t, d);
    case 32: return launch_elem<ELEM, 32>(ctx, m, s, t, d);
    default: return launch_elem<ELEM, 64>(ctx, m, s, t, d);
  }
}

}  // namespace

bool tensor_supports(Measure m, const DevImage& src, const DevImage& tmpl, const DevImage& dst,
                     bool forced) {
  if (m == kAbsDistance) return false;
  if (src.nch != 1 || tmpl.nch != 1 || dst.nch != 1) return false;
  if (tmpl.width > 64 || tmpl.height > 64) return false;
  if (src.type == U8) return true;
  // F32: the BF16 hi + lo split keeps about 16 bits of each operand, so one
  // product can be off by ~3e-5 relative; the <= 1e-5 bar needs the errors of
  // many terms to average, and tiny templates gain nothing from the MMA.
  if (src.type == F32) return forced && tmpl.width * tmpl.height >= 64;
  return false;
}

cudaError_t launch_proximity_tensor(Context& ctx, Measure m, const DevImage& src,
                                    const DevImage& tmpl, const DevImage& dst) {
  if (src.type == U8) return launch_r<kU8>(ctx, m, src, tmpl, dst);
  return launch_r<kF32>(ctx, m, src, tmpl, dst);
}

}  // namespace ocipb
