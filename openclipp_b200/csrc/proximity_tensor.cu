// Tensor-core (tcgen05) ImageProximity path for sm_100a.
//
// The product term of SqrDistance[_Norm] and CrossCorr[_Norm]
// (cl-files/ImageProximity.cl :44, :122, :290, :375),
//   C(x, y) = sum_h sum_w S(x + w - tw/2, y + h - th/2) * T(w, h),
// is computed per channel as one small GEMM per source row r and 256-position
// strip. Each TMEM lane m holds two output positions, x0 + 2m (phase 0) and
// x0 + 2m + 1 (phase 1), and the A row of lane m is the source-row window
//   A_r[m][k] = S(x0 - tw/2 + 2m + k, r),   k < K = roundup(tw + 1),
// so the two phases share A: phase p reads it one pixel later. The template
// operand has N = 2R rows (R = th rounded up to 16/32/64, zero rows on top),
//   B[p R + n][k] = Tpad(k - p, n),   Tpad(w, n) = T(w, n - (R - th)),
// and D_r[m][p R + n] is the contribution of template row n to position
// x0 + 2m + p. Source row r feeds output row y = r - n + off
// (off = R - th + th/2) through template row n, so every output row collects
// R consecutive steps. The epilogue keeps those R partial sums per position
// in registers, ordered by output row: at each step it adds the step's R
// columns and shifts by one (acc[c] <- acc[c + 1] + D[R - 2 - c]), and
// acc[0] + D[R - 1] is the finished output row.
//
// The A operand lives in tensor memory: builder warps write each lane's
// K-pixel window with tcgen05.st (BF16 hi/lo pairs for F32 and U16 sources,
// bytes for U8), and the MMA reads it from TMEM, which costs half as many
// cycles per instruction as an A operand read from shared memory.
//
// Channels. Interleaved multi-channel sources are first split into planes
// (one row-major plane per channel in scratch memory); blockIdx.z is the
// channel, the TMA view has the channel as its outermost dimension (so rows
// outside a plane read as zeros), and the template and the score map are
// addressed with the channel stride.
//
// Precision. U8 sources use the i8 MMA with s32 accumulation: every product
// term is exact and so are the results. F32 and U16 sources are split into
// BF16 hi + lo parts (S = S_hi + S_lo + O(2^-18 S); exact for U16); three MMAs
// (hi*hi, hi*lo, lo*hi) accumulate in FP32 in TMEM. The window energy sum S^2
// of each position is a per-row sum of tw squares (FP32 FMA for F32, FP64 for
// U16, exact integers for U8) and a running sum over the last th rows (FP64 /
// exact integers); the template energy is exact in FP64. SqrDistance =
// E_S - 2C + E_T and the _Norm scale are done in FP64 (F32, U16) or as the
// plain path does them (U8).
//
// Roles (17 warps; one CTA per SM, since it allocates all of TMEM):
//   warps 0-7   builders, two per TMEM sub-partition (tcgen05.ld/st reach
//               only the 32 lanes of the warp's sub-partition), one per phase:
//               the A operand of step t (the warp's half of the K columns) and
//               the window energy of its positions, handed to the epilogue
//               through a shared-memory ring;
//   warps 8-15  epilogue, same split: TMEM loads, running sums, output;
//   warp 16     control: TMA loads of source rows (zero fill outside the
//               image) and the MMAs of each step. Issuing an MMA or a commit
//               blocks the issuing thread for tens of cycles, so this thread
//               does nothing else: one wait (ready), the MMAs, one commit
//               (mma_done) per step.
// Stages are chained by mbarriers; every wait is bounded and sets an error
// flag instead of hanging.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cstring>
#include <type_traits>

#include "sm100.cuh"
#include "tensor.h"

namespace ocipb {
namespace {

using namespace sm100;

constexpr int kM = 128;                 // TMEM lanes = A rows
constexpr int kPos = 2 * kM;            // output positions per strip
constexpr int kBuilders = 8;
constexpr int kEpilogue = 8;
constexpr int kThreads = (kBuilders + kEpilogue + 1) * 32;  // + control warp
constexpr int kRB = 8;                  // source rows per TMA load
constexpr int kNRaw = 4;                // TMA stages
constexpr int kNE = 16;                 // window-energy ring depth (steps)
constexpr int kTmemCols = 512;
constexpr int kMinSmem = 120 * 1024;    // keeps one CTA per SM (it takes all of TMEM)
constexpr long long kSpinLimit = 4000000000LL;  // about 2 s of SM clock

enum Elem { kF32 = 0, kU8 = 1, kU16 = 2 };

template <int ELEM>
struct ElemTraits {
  static constexpr bool split = ELEM != kU8;  // BF16 hi/lo operands
  static constexpr int size = ELEM == kF32 ? 4 : ELEM == kU16 ? 2 : 1;
  static constexpr int inner = 16 / size;     // elements per 16-byte TMA group
  typedef typename std::conditional<split, float, int>::type AT;   // accumulators
  typedef typename std::conditional<split, double, int>::type ET;  // window energy
};

// TMEM stages: NS stages of D (2R columns) first, then NS stages of A.
template <int ELEM, int R, int K>
struct Stages {
  static constexpr int N2 = 2 * R;
  static constexpr int AC = ElemTraits<ELEM>::split ? K : K / 4;  // TMEM columns per A stage
  static constexpr int NS0 = kTmemCols / (N2 + AC);
  static constexpr int NS = NS0 > 4 ? 4 : NS0;
  static_assert(NS >= 2, "TMEM too small for two stages");
  static_assert(2 * NS <= kNE, "energy ring shorter than the pipeline");
};

struct TensorParams {
  int W, H;
  int tw, th;
  int nch;       // channels (blockIdx.z = channel)
  int nbox;      // 16-byte groups per staged row
  int lead;      // staged rows start `lead` pixels before the first window (TMA alignment)
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
  int row_bytes, raw_stage, raw, b_arr, b, rs, es, bars, total;
};

__host__ __device__ inline int align128(int x) { return (x + 127) & ~127; }

__host__ __device__ inline Layout make_layout(bool split, int R, int K, int nbox) {
  Layout L;
  L.row_bytes = nbox * 16;
  L.raw_stage = align128(kRB * L.row_bytes);
  L.raw = 0;
  L.b_arr = 2 * R * K * (split ? 2 : 1);
  L.b = L.raw + kNRaw * L.raw_stage;
  L.rs = L.b + align128((split ? 2 : 1) * L.b_arr);
  L.es = L.rs + R * kPos * 4;
  L.bars = L.es + kNE * kPos * (split ? 8 : 4);
  // mbarriers: raw full; ready and MMA done (4 each at most); energy full;
  // done. Then the TMEM address, the abort flag and the template energy.
  L.total = L.bars + align128(8 * (kNRaw + 2 * 4 + kNE + 1) + 32);
  return L;
}

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
  __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<uint32_t*>(&v);
}
__device__ __forceinline__ float bf16lo_f(uint32_t w) { return __uint_as_float(w << 16); }
__device__ __forceinline__ float bf16hi_f(uint32_t w) { return __uint_as_float(w & 0xFFFF0000u); }

// Template element (w, h) of channel c as a double (exact for every type).
template <int ELEM>
__device__ __forceinline__ double tmpl_at(const TensorParams& p, int h, int w, int c) {
  const char* row = p.tmpl + (size_t)h * p.tmpl_pitch;
  const int i = w * p.nch + c;
  if (ELEM == kF32) return reinterpret_cast<const float*>(row)[i];
  if (ELEM == kU16) return reinterpret_cast<const uint16_t*>(row)[i];
  return reinterpret_cast<const uint8_t*>(row)[i];
}

// Pixels e0 + 16c .. e0 + 16c + 15 of a staged row as floats (F32, U16).
template <int ELEM>
__device__ __forceinline__ void load_chunk(const unsigned char* row, int e0, int c, float (&f)[16]) {
  if (ELEM == kF32) {
    const float2* r2 = reinterpret_cast<const float2*>(row) + (e0 >> 1) + c * 8;
    if (e0 & 1) {  // odd start: aligned pairs from e0 - 1, shifted by one
      float prev = r2[0].y;
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const float2 v = r2[j + 1];
        f[2 * j] = prev;
        f[2 * j + 1] = v.x;
        prev = v.y;
      }
    } else {
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const float2 v = r2[j];
        f[2 * j] = v.x;
        f[2 * j + 1] = v.y;
      }
    }
  } else {
    // U16: 32-bit words hold two pixels; an odd start is realigned by bytes.
    const uint32_t* r32 = reinterpret_cast<const uint32_t*>(row) + (e0 >> 1) + c * 8;
    uint32_t w[9];
#pragma unroll
    for (int j = 0; j < 9; ++j) w[j] = r32[j];
    const bool odd = e0 & 1;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const uint32_t v = odd ? __byte_perm(w[j], w[j + 1], 0x5432) : w[j];
      f[2 * j] = static_cast<float>(v & 0xFFFFu);
      f[2 * j + 1] = static_cast<float>(v >> 16);
    }
  }
}

template <int ELEM, int R, int K>
__global__ void __launch_bounds__(kThreads, 1)
    prox_tensor_kernel(const __grid_constant__ CUtensorMap tmap, const TensorParams p) {
  extern __shared__ __align__(1024) unsigned char smem[];
  typedef ElemTraits<ELEM> TR;
  constexpr bool SPLIT = TR::split;
  const Layout L = make_layout(SPLIT, R, K, p.nbox);
  typedef Stages<ELEM, R, K> SG;
  constexpr int N2 = SG::N2, AC = SG::AC, NS = SG::NS;
  typedef typename TR::AT AT;
  typedef typename TR::ET ET;
  typedef typename std::conditional<ELEM == kF32, float, ET>::type RT;  // row energy sum
  // Row energies kept for th steps: FP32 for F32/U16 (the same rounded value
  // is added and later subtracted, so the FP64 running sum does not drift),
  // exact int for U8.
  typedef typename std::conditional<SPLIT, float, int>::type ST;

  // ready[i]: step t = i + k NS may be issued (its A operand is written and
  //           the D stage of step t - NS has been read); 8 builder + 8
  //           epilogue arrivals.
  // mma_done[i]: the MMAs of step t have completed (D readable, A reusable).
  uint64_t* raw_full = reinterpret_cast<uint64_t*>(smem + L.bars);
  uint64_t* ready = raw_full + kNRaw;
  uint64_t* mma_done = ready + 4;
  uint64_t* e_full = mma_done + 4;
  uint64_t* done_bar = e_full + kNE;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done_bar + 1);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);
  double* s_et = reinterpret_cast<double*>(tmem_slot + 2);
  ET* estage = reinterpret_cast<ET*>(smem + L.es);

  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const bool need_e = p.measure != kCrossCorr;
  const int xs_out = blockIdx.x * kPos;  // strip b covers outputs [256 b, 256 b + 256)
  const int y0 = blockIdx.y * p.BH;
  const int ch = blockIdx.z;
  const int yend = min(p.H, y0 + p.BH);
  const int r_begin = y0 - p.off;
  const int nsteps = (yend - y0) + R - 1;
  const int nb = (nsteps + kRB - 1) / kRB;  // TMA loads (kRB rows each)

  if (threadIdx.x == 0) {
    for (int i = 0; i < kNRaw; ++i) mbar_init(&raw_full[i], 1);
    for (int i = 0; i < NS; ++i) {
      mbar_init(&ready[i], kBuilders + kEpilogue);
      mbar_init(&mma_done[i], 1);
    }
    for (int i = 0; i < kNE; ++i) mbar_init(&e_full[i], kBuilders);
    mbar_init(done_bar, 1);
    *abort_flag = 0;
    fence_barrier_init();
    // The first NS steps have no earlier D stage to wait for.
    for (int i = 0; i < NS; ++i) mbar_arrive_n(&ready[i], kEpilogue);
  }
  if (warp == 0) tmem_alloc(tmem_slot, kTmemCols);

  // Template operand B (N2 = 2R rows: phase 0 then phase 1, zero rows on top
  // of each) and the template energy of this channel.
  {
    const int padrows = R - p.th;
    for (int idx = threadIdx.x; idx < N2 * K; idx += kThreads) {
      const int nn = idx / K, k = idx - nn * K;
      const int ph = nn >= R ? 1 : 0;
      const int h = nn - ph * R - padrows;
      const int w = k - ph;
      const bool in = h >= 0 && w >= 0 && w < p.tw;
      const double t = in ? tmpl_at<ELEM>(p, h, w, ch) : 0.0;
      if (SPLIT) {
        const float tf = static_cast<float>(t);
        const __nv_bfloat16 th_ = __float2bfloat16_rn(tf);
        const __nv_bfloat16 tl_ = __float2bfloat16_rn(tf - __bfloat162float(th_));
        const int off = ((k >> 3) * N2 + nn) * 16 + (k & 7) * 2;
        *reinterpret_cast<__nv_bfloat16*>(smem + L.b + off) = th_;
        *reinterpret_cast<__nv_bfloat16*>(smem + L.b + L.b_arr + off) = tl_;
      } else {
        const int off = ((k >> 4) * N2 + nn) * 16 + (k & 15);
        smem[L.b + off] = static_cast<uint8_t>(t);
      }
    }
    if (warp == 1) {
      double e = 0.0;
      for (int idx = lane; idx < p.th * p.tw; idx += 32) {
        const int h = idx / p.tw, k = idx - h * p.tw;
        const double t = tmpl_at<ELEM>(p, h, k, ch);
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
  constexpr uint32_t acol0 = NS * N2;  // first A column

  const int sp = warp & 3;  // TMEM sub-partition of this warp
  const int m = sp * 32 + lane;
  const uint32_t lane_base = tmem_base + (static_cast<uint32_t>(sp * 32) << 16);

  if (warp == kBuilders + kEpilogue) {
    // ---- Control: TMA loads of source rows, MMA issue ---------------------------
    if (lane == 0) {
      tma_prefetch_desc(&tmap);
      // Staged row = pixels from xs_out - left0 - lead, a whole 16-byte group.
      const int gx = (xs_out - p.left0 - p.lead) / TR::inner;
      int issued = 0;
      for (; issued < min(nb, kNRaw); ++issued) {
        mbar_arrive_expect_tx(&raw_full[issued], kRB * L.row_bytes);
        tma_load_4d(smem + L.raw + issued * L.raw_stage, &tmap, 0, gx, r_begin + issued * kRB,
                    ch, &raw_full[issued]);
      }
      const uint32_t b0 = smem_u32(smem + L.b);
      int i = 0, st = 0, rr = 0;
      uint32_t ph = 0;
      for (int t = 0; t < nsteps; ++t) {
        if (!mbar_wait(&ready[i], ph, abort_flag, kSpinLimit)) break;
        // Every builder has read row t: its stage is free after the last row.
        if (rr == kRB - 1 && issued < nb) {
          mbar_arrive_expect_tx(&raw_full[st], kRB * L.row_bytes);
          tma_load_4d(smem + L.raw + st * L.raw_stage, &tmap, 0, gx, r_begin + issued * kRB, ch,
                      &raw_full[st]);
          ++issued;
        }
        tc_fence_after();
        const uint32_t d = tmem_base + i * N2;
        const uint32_t a = tmem_base + acol0 + i * AC;
        if (SPLIT) {
          constexpr uint32_t idesc = idesc_bf16_f32(kM, N2);
          const uint32_t blo = b0 + L.b_arr;
#pragma unroll
          for (int kk = 0; kk < K / 16; ++kk)
            mma_bf16_ts(d, a + kk * 8, smem_desc(b0 + kk * 2 * N2 * 16, N2 * 16, 128), idesc,
                        kk > 0);
#pragma unroll
          for (int kk = 0; kk < K / 16; ++kk)
            mma_bf16_ts(d, a + kk * 8, smem_desc(blo + kk * 2 * N2 * 16, N2 * 16, 128), idesc,
                        1);
#pragma unroll
          for (int kk = 0; kk < K / 16; ++kk)
            mma_bf16_ts(d, a + K / 2 + kk * 8, smem_desc(b0 + kk * 2 * N2 * 16, N2 * 16, 128),
                        idesc, 1);
        } else {
          constexpr uint32_t idesc = idesc_u8_s32(kM, N2);
#pragma unroll
          for (int kk = 0; kk < K / 32; ++kk)
            mma_i8_ts(d, a + kk * 8, smem_desc(b0 + kk * 2 * N2 * 16, N2 * 16, 128), idesc,
                      kk > 0);
        }
        mma_commit(&mma_done[i]);
        if (++i == NS) { i = 0; ph ^= 1; }
        if (++rr == kRB) { rr = 0; if (++st == kNRaw) st = 0; }
      }
      // Every MMA issued has completed before TMEM is freed, and every TMA
      // load issued has landed before the CTA exits.
      mma_commit(done_bar);
      volatile int no_abort = 0;
      mbar_wait(done_bar, 0, &no_abort, kSpinLimit);
      for (int b = max(0, issued - kNRaw); b < issued; ++b)
        mbar_wait(&raw_full[b % kNRaw], (b / kNRaw) & 1, &no_abort, kSpinLimit);
    }
  } else if (warp < kBuilders) {
    // ---- Builders: A operand of step t and the window energies ------------------
    const int ph = warp >> 2;      // phase of the energies; K half of the A build
    const int pos = 2 * m + ph;
    const int e0 = p.lead + 2 * m;  // this lane's window starts at pixel e0 of the staged row
    ST* rsring = reinterpret_cast<ST*>(smem + L.rs);
    ET ewin = ET(0);
    int i = 0, st = 0, rr = 0;
    uint32_t iph = 0, rph = 0;
    for (int t = 0; t < nsteps; ++t) {
      if (rr == 0 && !mbar_wait(&raw_full[st], rph, abort_flag, kSpinLimit)) break;
      // A stage i is free once the MMAs of step t - NS have completed.
      if (!mbar_wait(&mma_done[i], iph ^ 1, abort_flag, kSpinLimit)) break;
      tc_fence_after();
      const unsigned char* row = smem + L.raw + st * L.raw_stage + rr * L.row_bytes;
      const uint32_t a_addr = lane_base + acol0 + i * AC;
      ET rs = ET(0);
      if (SPLIT) {
        // The window in chunks of 16 K columns. The chunks alternate between
        // the two builders of a lane; both read every chunk when energies are
        // needed.
        RT r0 = RT(0), r1 = RT(0);
#pragma unroll
        for (int c = 0; c < K / 16; ++c) {
          const bool mine = (c & 1) == ph;
          if (!mine && !need_e) continue;
          float f[16];
          load_chunk<ELEM>(row, e0, c, f);
          if (mine) {
            uint32_t hi[8], lo[8];
#pragma unroll
            for (int q = 0; q < 8; ++q) {
              hi[q] = pack_bf16(f[2 * q], f[2 * q + 1]);
              lo[q] = pack_bf16(f[2 * q] - bf16lo_f(hi[q]), f[2 * q + 1] - bf16hi_f(hi[q]));
            }
            tmem_st8(a_addr + c * 8, hi);
            tmem_st8(a_addr + K / 2 + c * 8, lo);
          }
          if (need_e) {
            // Sum of squares over k in [ph, ph + tw). K = roundup16(tw + 1),
            // so only k = 0 and the last chunk can fall outside.
#pragma unroll
            for (int j = 0; j < 16; ++j) {
              const int k = c * 16 + j;
              RT v = static_cast<RT>(f[j]);
              if (k == 0 || k >= K - 16) v = (k >= ph && k < ph + p.tw) ? v : RT(0);
              if (j & 1)
                r1 = fma(v, v, r1);
              else
                r0 = fma(v, v, r0);
            }
          }
        }
        rs = static_cast<ET>(r0) + static_cast<ET>(r1);
      } else {
        // Bytes e0 .. e0 + K - 1: words from the aligned base, shifted.
        const uint32_t* r32 = reinterpret_cast<const uint32_t*>(row) + (e0 >> 2);
        uint32_t w[K / 4 + 1];
#pragma unroll
        for (int j = 0; j <= K / 4; ++j) w[j] = r32[j];
        const uint32_t sh = (e0 & 3) * 8;
        uint32_t a[K / 4];
#pragma unroll
        for (int j = 0; j < K / 4; ++j) a[j] = __funnelshift_r(w[j], w[j + 1], sh);
        // Each builder stores its half of the K/4 columns, 4 at a time.
#pragma unroll
        for (int c = 0; c < K / 16; ++c) {
          if ((c & 1) == ph) tmem_st4(a_addr + c * 4, &a[c * 4]);
        }
        if (need_e) {
          const uint32_t sh2 = sh + 8 * ph;
          uint32_t acc = 0;
#pragma unroll
          for (int j = 0; j < K / 4; ++j) {
            const int rem = p.tw - 4 * j;
            uint32_t v = __funnelshift_rc(w[j], w[j + 1], sh2);  // sh2 may be 32
            if (rem <= 0) v = 0;
            else if (rem < 4) v &= (1u << (8 * rem)) - 1u;
            acc = __dp4a(v, v, acc);
          }
          rs = static_cast<ET>(acc);
        }
      }
      if (need_e) {
        // Window energy: add this row, drop the row th steps back (the ring
        // holds R >= th rows; read before write when th == R).
        ST* slot = rsring + (t & (R - 1)) * kPos + pos;
        const ST old = t >= p.th ? rsring[((t - p.th) & (R - 1)) * kPos + pos] : ST(0);
        const ST cur = static_cast<ST>(rs);
        *slot = cur;
        ewin += static_cast<ET>(cur) - static_cast<ET>(old);
        estage[(t & (kNE - 1)) * kPos + pos] = ewin;
      }
      tmem_st_wait();
      tc_fence_before();
      __syncwarp();
      if (lane == 0) {
        if (need_e) mbar_arrive(&e_full[t & (kNE - 1)]);
        mbar_arrive(&ready[i]);
      }
      if (++i == NS) { i = 0; iph ^= 1; }
      if (++rr == kRB) { rr = 0; if (++st == kNRaw) { st = 0; rph ^= 1; } }
    }
  } else {
    // ---- Epilogue: running sums over template rows, energies, output ------------
    const int ph = (warp - kBuilders) >> 2;  // positions 2m + ph, D columns [ph R, ph R + R)
    const int pos = 2 * m + ph;
    const int x = xs_out + pos;
    const bool x_ok = x < p.W;
    const size_t xo = (size_t)x * p.nch + ch;  // element of the score-map row
    AT acc[R];
#pragma unroll
    for (int j = 0; j < R; ++j) acc[j] = AT(0);
    const ET et = static_cast<ET>(*s_et);
    const double etd = *s_et;
    int i = 0;
    uint32_t iph = 0;
    for (int s = 0; s < nsteps; ++s) {
      if (!mbar_wait(&mma_done[i], iph, abort_flag, kSpinLimit)) break;
      tc_fence_after();
      // D[n] = column i*N2 + ph*R + n. Chunks are taken from the top so the
      // shift-add below runs with ascending c (acc[c - 1] <- acc[c] + D[R-1-c]).
      constexpr int CW = R == 32 ? 32 : 16;  // 16-column loads keep R = 64 in registers
      AT outv = AT(0);
#pragma unroll
      for (int q = R / CW - 1; q >= 0; --q) {
        uint32_t v[32];
        if (CW == 32)
          tmem_ld32(lane_base + i * N2 + ph * R + q * CW, v);
        else
          tmem_ld16(lane_base + i * N2 + ph * R + q * CW, v);
        tmem_ld_wait();
#pragma unroll
        for (int j = CW - 1; j >= 0; --j) {
          const int n = q * CW + j;
          const int c = R - 1 - n;
          const AT val = SPLIT ? (AT)__uint_as_float(v[j]) : (AT) static_cast<int>(v[j]);
          if (c == 0)
            outv = acc[0] + val;
          else
            acc[c - 1] = acc[c] + val;
        }
      }
      acc[R - 1] = AT(0);
      ET e = ET(0);
      if (need_e) {
        if (!mbar_wait(&e_full[s & (kNE - 1)], (s / kNE) & 1, abort_flag, kSpinLimit)) break;
        e = estage[(s & (kNE - 1)) * kPos + pos];
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&ready[i]);  // D stage i free for step s + NS
      if (++i == NS) { i = 0; iph ^= 1; }

      const int yd = y0 + s - R + 1;
      if (s >= R - 1 && yd < yend && x_ok) {
        double outd;
        float outf;
        if (SPLIT) {
          const double cc = (double)outv;
          const double ed = (double)e;
          if (p.measure == kCrossCorr) outd = cc;
          else if (p.measure == kSqrDistance) outd = ed - 2.0 * cc + etd;
          else if (p.measure == kCrossCorrNorm) outd = cc * rsqrt(ed * etd);
          else outd = (ed - 2.0 * cc + etd) * rsqrt(ed * etd);
          outf = (float)outd;
        } else {
          const long long cc = (long long)outv;
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
          reinterpret_cast<double*>(o)[xo] = outd;
        else
          reinterpret_cast<float*>(o)[xo] = outf;
      }
    }
  }

  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    tmem_dealloc(tmem_base, kTmemCols);
  }
  if (threadIdx.x == 0 && *abort_flag) atomicExch(p.err, 1);
}

// Interleaved channels -> planes: plane c holds channel c of every pixel, rows
// at `plane_pitch`, planes `plane_bytes` apart. Columns W .. pw - 1 (the pitch
// tail, which the TMA view reads in whole 16-byte groups) are written as zeros.
template <typename T>
__global__ void split_channels_kernel(const char* src, size_t src_pitch, char* planes,
                                      size_t plane_pitch, size_t plane_bytes, int W, int pw,
                                      int H, int nch) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y;
  if (x >= pw || y >= H) return;
  const T* s = reinterpret_cast<const T*>(src + (size_t)y * src_pitch) + (size_t)x * nch;
  for (int c = 0; c < nch; ++c)
    reinterpret_cast<T*>(planes + c * plane_bytes + (size_t)y * plane_pitch)[x] =
        x < W ? s[c] : T(0);
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

// Band height: the fewest waves of CTAs times the steps per band (output
// rows plus the R - 1 rows of ramp), over all band counts.
int band_height(int H, int R, long long columns, int sm_count) {
  long long best = LLONG_MAX;
  int best_bh = H;
  for (int nb = 1; nb <= std::max(1, H / 8); ++nb) {
    const int bh = (H + nb - 1) / nb;
    const int nbe = (H + bh - 1) / bh;
    const long long waves = (columns * nbe + sm_count - 1) / sm_count;
    const long long cost = waves * (bh + R - 1);
    if (cost < best) {
      best = cost;
      best_bh = bh;
    }
  }
  return best_bh;
}

template <int ELEM, int R, int K>
cudaError_t launch_elem(Context& ctx, Measure m, const DevImage& src, const DevImage& tmpl,
                        const DevImage& dst) {
  typedef ElemTraits<ELEM> TR;
  TensorParams p;
  p.W = src.width;
  p.H = src.height;
  p.tw = tmpl.width;
  p.th = tmpl.height;
  p.nch = src.nch;
  // Lane m reads pixels lead + 2m .. lead + 2m + K (one more for odd leads).
  p.nbox = (kPos + K + 2 * TR::inner + 1) / TR::inner;
  p.left0 = p.tw / 2;
  p.lead = (TR::inner - p.left0 % TR::inner) % TR::inner;
  p.off = R - p.th + p.th / 2;
  const int nstrips = (p.W + kPos - 1) / kPos;
  p.BH = band_height(p.H, R, (long long)nstrips * p.nch, ctx.sm_count);
  p.measure = m;
  p.norm_float = (double)p.tw * p.th * 65025.0 <= 16777216.0;
  p.tmpl = (const char*)tmpl.ptr;
  p.tmpl_pitch = tmpl.pitch;
  p.dst = (char*)dst.ptr;
  p.dst_pitch = dst.pitch;
  p.dst_f64 = dst.type == F64;
  p.err = reinterpret_cast<int*>(ctx.scratch(Context::kTensorAux, 256));

  // Source planes: the image itself for one channel, else a split copy.
  const char* planes = (const char*)src.ptr;
  size_t plane_pitch = src.pitch, plane_bytes = src.pitch * (size_t)p.H;
  if (p.nch > 1) {
    plane_pitch = ((size_t)p.W * TR::size + 127) / 128 * 128;
    plane_bytes = plane_pitch * p.H;
    char* pl = reinterpret_cast<char*>(ctx.scratch(Context::kPlanes, plane_bytes * p.nch));
    typedef typename std::conditional<TR::size == 4, uint32_t,
                                      typename std::conditional<TR::size == 2, uint16_t,
                                                                uint8_t>::type>::type PT;
    const int pw = static_cast<int>(plane_pitch / TR::size);  // row length incl. the tail
    dim3 sg((pw + 255) / 256, p.H);
    split_channels_kernel<PT><<<sg, 256, 0, ctx.stream>>>((const char*)src.ptr, src.pitch, pl,
                                                          plane_pitch, plane_bytes, p.W, pw, p.H,
                                                          p.nch);
    count_launches(1);
    planes = pl;
  }

  EncodeTiledFn enc = encode_fn();
  if (!enc) return cudaErrorNotSupported;
  // Rank-4 view of the source planes: 16-byte groups (dim 0), groups along the
  // row (dim 1), rows (dim 2), channels (dim 3). A staged row of 256 + K
  // pixels is one box of nbox groups, under the 256-element box limit. The
  // last group of a row may reach into the row pitch, which is zero (image
  // creation zero-fills device buffers; the split writes zeros there).
  CUtensorMap map;
  const CUtensorMapDataType dt = ELEM == kF32   ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32
                                 : ELEM == kU16 ? CU_TENSOR_MAP_DATA_TYPE_UINT16
                                                : CU_TENSOR_MAP_DATA_TYPE_UINT8;
  const cuuint64_t gdim[4] = {(cuuint64_t)TR::inner,
                              (cuuint64_t)((p.W + TR::inner - 1) / TR::inner), (cuuint64_t)p.H,
                              (cuuint64_t)p.nch};
  const cuuint64_t gstride[3] = {16, (cuuint64_t)plane_pitch, (cuuint64_t)plane_bytes};
  const cuuint32_t box[4] = {(cuuint32_t)TR::inner, (cuuint32_t)p.nbox, (cuuint32_t)kRB, 1};
  const cuuint32_t estride[4] = {1, 1, 1, 1};
  CUresult r = enc(&map, dt, 4, const_cast<char*>(planes), gdim, gstride, box, estride,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                   CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return cudaErrorInvalidValue;

  const Layout L = make_layout(TR::split, R, K, p.nbox);
  const int smem_bytes = std::max(L.total, kMinSmem);
  auto kern = prox_tensor_kernel<ELEM, R, K>;
  cudaError_t e =
      cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_bytes);
  if (e != cudaSuccess) return e;
  const int nbands = (p.H + p.BH - 1) / p.BH;
  dim3 grid(nstrips, nbands, p.nch);
  kern<<<grid, kThreads, smem_bytes, ctx.stream>>>(map, p);
  count_launches(1);
  return cudaGetLastError();
}

template <int ELEM, int R>
cudaError_t launch_k(Context& ctx, Measure m, const DevImage& s, const DevImage& t,
                     const DevImage& d) {
  const int tw = t.width;
  if constexpr (ElemTraits<ELEM>::split) {
    switch ((tw + 1 + 15) / 16) {
      case 1: return launch_elem<ELEM, R, 16>(ctx, m, s, t, d);
      case 2: return launch_elem<ELEM, R, 32>(ctx, m, s, t, d);
      case 3: return launch_elem<ELEM, R, 48>(ctx, m, s, t, d);
      case 4: return launch_elem<ELEM, R, 64>(ctx, m, s, t, d);
      default: return launch_elem<ELEM, R, 80>(ctx, m, s, t, d);
    }
  } else {
    switch ((tw + 1 + 31) / 32) {
      case 1: return launch_elem<ELEM, R, 32>(ctx, m, s, t, d);
      case 2: return launch_elem<ELEM, R, 64>(ctx, m, s, t, d);
      default: return launch_elem<ELEM, R, 96>(ctx, m, s, t, d);
    }
  }
}

template <int ELEM>
cudaError_t launch_r(Context& ctx, Measure m, const DevImage& s, const DevImage& t,
                     const DevImage& d) {
  switch (ring_size(t.height)) {
    case 16: return launch_k<ELEM, 16>(ctx, m, s, t, d);
    case 32: return launch_k<ELEM, 32>(ctx, m, s, t, d);
    default: return launch_k<ELEM, 64>(ctx, m, s, t, d);
  }
}

}  // namespace

bool tensor_supports(Measure m, const DevImage& src, const DevImage& tmpl, const DevImage& dst,
                     bool forced) {
  if (m == kAbsDistance) return false;
  if (src.nch != tmpl.nch || src.nch != dst.nch || src.nch < 1 || src.nch > 4) return false;
  if (tmpl.width > 64 || tmpl.height > 64) return false;
  if (src.type == U8) return true;
  // F32 and U16 use the BF16 hi + lo split: about 16 bits of each F32 operand
  // (all 16 of a U16), so one product can be off by ~3e-5 relative; the 1e-5
  // bar needs the errors of many terms to average, and tiny templates gain
  // nothing from the MMA. Taken only when asked for.
  if (src.type == F32 || src.type == U16) return forced && tmpl.width * tmpl.height >= 64;
  return false;
}

cudaError_t launch_proximity_tensor(Context& ctx, Measure m, const DevImage& src,
                                    const DevImage& tmpl, const DevImage& dst) {
  if (src.type == U8) return launch_r<kU8>(ctx, m, src, tmpl, dst);
  if (src.type == U16) return launch_r<kU16>(ctx, m, src, tmpl, dst);
  return launch_r<kF32>(ctx, m, src, tmpl, dst);
}

}  // namespace ocipb
