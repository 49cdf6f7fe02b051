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
#include <map>
#include <mutex>
#include <tuple>
#include <type_traits>
#include <vector>

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
constexpr int kMaxDynSmem = 226 * 1024; // opt-in dynamic shared memory limit of the kernel
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

// One work item: one channel of one 256-position strip x band of rows of one
// (image, template) pair.
struct ItemArgs {
  const CUtensorMap* tmap;  // source planes (rank 4: group, groups, rows, channel)
  int W, H;
  int tw, th;
  int ax, ay;    // window anchor: output (x, y) reads S(x + w - ax, y + h - ay)
  int nch, ch;
  int xs_out;    // strip covers outputs [xs_out, xs_out + 256)
  int y0, yend;  // band of output rows
  int nbox;      // 16-byte groups per staged row (the tensor map's box)
  const char* tmpl;
  size_t tmpl_pitch;
  char* dst;
  size_t dst_pitch;
  int dst_f64;
  int measure;
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
  // done.
  L.total = L.bars + align128(8 * (kNRaw + 2 * 4 + kNE + 1));
  return L;
}

// CTA state that outlives one work item.
struct CtaState {
  uint32_t tmem;  // TMEM base address (all 512 columns)
  int abort;      // set by a wait that gave up; the CTA stops taking items
  int next;       // work item fetched from the queue
  double et;      // template energy of the current item's channel
};

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
  __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<uint32_t*>(&v);
}
__device__ __forceinline__ float bf16lo_f(uint32_t w) { return __uint_as_float(w << 16); }
__device__ __forceinline__ float bf16hi_f(uint32_t w) { return __uint_as_float(w & 0xFFFF0000u); }

// Template element (w, h) of channel c as a double (exact for every type).
template <int ELEM>
__device__ __forceinline__ double tmpl_at(const ItemArgs& a, int h, int w, int c) {
  const char* row = a.tmpl + (size_t)h * a.tmpl_pitch;
  const int i = w * a.nch + c;
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

// Runs one work item with all 17 warps of the CTA. The caller has synchronised
// the CTA; TMEM (512 columns) is allocated. Barriers are initialised here and
// invalidated at the end, so consecutive items may use different layouts.
template <int ELEM, int R, int K>
__device__ __forceinline__ void run_item(const ItemArgs& a, unsigned char* smem, CtaState& cs) {
  typedef ElemTraits<ELEM> TR;
  constexpr bool SPLIT = TR::split;
  typedef Stages<ELEM, R, K> SG;
  constexpr int N2 = SG::N2, AC = SG::AC, NS = SG::NS;
  typedef typename TR::AT AT;
  typedef typename TR::ET ET;
  typedef typename std::conditional<ELEM == kF32, float, ET>::type RT;  // row energy sum
  // Row energies kept for th steps: FP32 for F32/U16 (the same rounded value
  // is added and later subtracted, so the FP64 running sum does not drift),
  // exact int for U8.
  typedef typename std::conditional<SPLIT, float, int>::type ST;
  const Layout L = make_layout(SPLIT, R, K, a.nbox);

  // ready[i]: step t = i + k NS may be issued (its A operand is written and
  //           the D stage of step t - NS has been read); 8 builder + 8
  //           epilogue arrivals.
  // mma_done[i]: the MMAs of step t have completed (D readable, A reusable).
  uint64_t* raw_full = reinterpret_cast<uint64_t*>(smem + L.bars);
  uint64_t* ready = raw_full + kNRaw;
  uint64_t* mma_done = ready + 4;
  uint64_t* e_full = mma_done + 4;
  uint64_t* done_bar = e_full + kNE;
  volatile int* abort_flag = &cs.abort;
  ET* estage = reinterpret_cast<ET*>(smem + L.es);

  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const bool need_e = a.measure != kCrossCorr;
  const int ch = a.ch;
  const int left0 = a.ax;
  // Staged rows start `lead` pixels before the strip's first window pixel,
  // at a whole 16-byte group (TMA alignment).
  const int lead = (TR::inner - left0 % TR::inner) % TR::inner;
  const int off = R - a.th + a.ay;
  const int r_begin = a.y0 - off;
  const int nsteps = (a.yend - a.y0) + R - 1;
  const int nb = (nsteps + kRB - 1) / kRB;  // TMA loads (kRB rows each)

  if (threadIdx.x == 0) {
    for (int i = 0; i < kNRaw; ++i) mbar_init(&raw_full[i], 1);
    for (int i = 0; i < NS; ++i) {
      mbar_init(&ready[i], kBuilders + kEpilogue);
      mbar_init(&mma_done[i], 1);
    }
    for (int i = 0; i < kNE; ++i) mbar_init(&e_full[i], kBuilders);
    mbar_init(done_bar, 1);
    fence_barrier_init();
    // The first NS steps have no earlier D stage to wait for.
    for (int i = 0; i < NS; ++i) mbar_arrive_n(&ready[i], kEpilogue);
  }

  // Template operand B (N2 = 2R rows: phase 0 then phase 1, zero rows on top
  // of each) and the template energy of this channel.
  {
    const int padrows = R - a.th;
    for (int idx = threadIdx.x; idx < N2 * K; idx += kThreads) {
      const int nn = idx / K, k = idx - nn * K;
      const int ph = nn >= R ? 1 : 0;
      const int h = nn - ph * R - padrows;
      const int w = k - ph;
      const bool in = h >= 0 && w >= 0 && w < a.tw;
      const double t = in ? tmpl_at<ELEM>(a, h, w, ch) : 0.0;
      if (SPLIT) {
        const float tf = static_cast<float>(t);
        const __nv_bfloat16 th_ = __float2bfloat16_rn(tf);
        const __nv_bfloat16 tl_ = __float2bfloat16_rn(tf - __bfloat162float(th_));
        const int boff = ((k >> 3) * N2 + nn) * 16 + (k & 7) * 2;
        *reinterpret_cast<__nv_bfloat16*>(smem + L.b + boff) = th_;
        *reinterpret_cast<__nv_bfloat16*>(smem + L.b + L.b_arr + boff) = tl_;
      } else {
        const int boff = ((k >> 4) * N2 + nn) * 16 + (k & 15);
        smem[L.b + boff] = static_cast<uint8_t>(t);
      }
    }
    if (warp == 1) {
      double e = 0.0;
      for (int idx = lane; idx < a.th * a.tw; idx += 32) {
        const int h = idx / a.tw, k = idx - h * a.tw;
        const double t = tmpl_at<ELEM>(a, h, k, ch);
        e += t * t;
      }
#pragma unroll
      for (int d = 16; d > 0; d >>= 1) e += __shfl_xor_sync(0xffffffffu, e, d);
      if (lane == 0) cs.et = e;
    }
  }
  fence_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem_base = cs.tmem;
  constexpr uint32_t acol0 = NS * N2;  // first A column

  const int sp = warp & 3;  // TMEM sub-partition of this warp
  const int m = sp * 32 + lane;
  const uint32_t lane_base = tmem_base + (static_cast<uint32_t>(sp * 32) << 16);

  if (warp == kBuilders + kEpilogue) {
    // ---- Control: TMA loads of source rows, MMA issue ---------------------------
    if (lane == 0) {
      tma_prefetch_desc(a.tmap);
      const int gx = (a.xs_out - left0 - lead) / TR::inner;
      int issued = 0;
      for (; issued < min(nb, kNRaw); ++issued) {
        mbar_arrive_expect_tx(&raw_full[issued], kRB * L.row_bytes);
        tma_load_4d(smem + L.raw + issued * L.raw_stage, a.tmap, 0, gx, r_begin + issued * kRB,
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
          tma_load_4d(smem + L.raw + st * L.raw_stage, a.tmap, 0, gx, r_begin + issued * kRB,
                      ch, &raw_full[st]);
          ++issued;
        }
        tc_fence_after();
        const uint32_t d = tmem_base + i * N2;
        const uint32_t at = tmem_base + acol0 + i * AC;
        if (SPLIT) {
          constexpr uint32_t idesc = idesc_bf16_f32(kM, N2);
          const uint32_t blo = b0 + L.b_arr;
#pragma unroll
          for (int kk = 0; kk < K / 16; ++kk)
            mma_bf16_ts(d, at + kk * 8, smem_desc(b0 + kk * 2 * N2 * 16, N2 * 16, 128), idesc,
                        kk > 0);
#pragma unroll
          for (int kk = 0; kk < K / 16; ++kk)
            mma_bf16_ts(d, at + kk * 8, smem_desc(blo + kk * 2 * N2 * 16, N2 * 16, 128), idesc,
                        1);
#pragma unroll
          for (int kk = 0; kk < K / 16; ++kk)
            mma_bf16_ts(d, at + K / 2 + kk * 8, smem_desc(b0 + kk * 2 * N2 * 16, N2 * 16, 128),
                        idesc, 1);
        } else {
          constexpr uint32_t idesc = idesc_u8_s32(kM, N2);
#pragma unroll
          for (int kk = 0; kk < K / 32; ++kk)
            mma_i8_ts(d, at + kk * 8, smem_desc(b0 + kk * 2 * N2 * 16, N2 * 16, 128), idesc,
                      kk > 0);
        }
        mma_commit(&mma_done[i]);
        if (++i == NS) { i = 0; ph ^= 1; }
        if (++rr == kRB) { rr = 0; if (++st == kNRaw) st = 0; }
      }
      // Every MMA issued has completed before the item ends (TMEM and the
      // operands are reused), and every TMA load issued has landed.
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
    const int e0 = lead + 2 * m;   // this lane's window starts at pixel e0 of the staged row
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
              if (k == 0 || k >= K - 16) v = (k >= ph && k < ph + a.tw) ? v : RT(0);
              if (j & 1)
                r1 = fma(v, v, r1);
              else
                r0 = fma(v, v, r0);
            }
          }
        }
        rs = static_cast<ET>(r0) + static_cast<ET>(r1);
      } else {
        // Bytes e0 .. e0 + K - 1 in chunks of 16 (4 TMEM columns): words
        // from the aligned base, shifted. Chunks alternate between the two
        // builders of a lane; both read every chunk when energies are needed.
        const uint32_t* r32 = reinterpret_cast<const uint32_t*>(row) + (e0 >> 2);
        const uint32_t sh = (e0 & 3) * 8;
        const uint32_t sh2 = sh + 8 * ph;  // window of this builder's phase
        uint32_t acc = 0;
#pragma unroll
        for (int c = 0; c < K / 16; ++c) {
          const bool mine = (c & 1) == ph;
          if (!mine && !need_e) continue;
          uint32_t w[5];
#pragma unroll
          for (int j = 0; j < 5; ++j) w[j] = r32[c * 4 + j];
          if (mine) {
            uint32_t av[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) av[j] = __funnelshift_r(w[j], w[j + 1], sh);
            tmem_st4(a_addr + c * 4, av);
          }
          if (need_e) {
#pragma unroll
            for (int j = 0; j < 4; ++j) {
              const int rem = a.tw - 16 * c - 4 * j;
              uint32_t v = __funnelshift_rc(w[j], w[j + 1], sh2);  // sh2 may be 32
              if (rem <= 0) v = 0;
              else if (rem < 4) v &= (1u << (8 * rem)) - 1u;
              acc = __dp4a(v, v, acc);
            }
          }
        }
        if (need_e) rs = static_cast<ET>(acc);
      }
      if (need_e) {
        // Window energy: add this row, drop the row th steps back (the ring
        // holds R >= th rows; read before write when th == R).
        ST* slot = rsring + (t & (R - 1)) * kPos + pos;
        const ST old = t >= a.th ? rsring[((t - a.th) & (R - 1)) * kPos + pos] : ST(0);
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
    // Values used only when a row is written are read from shared memory
    // (the item, cs.et) at that point, which keeps registers for the R sums.
    const int ph = (warp - kBuilders) >> 2;  // positions 2m + ph, D columns [ph R, ph R + R)
    const uint32_t d_col = lane_base + ph * R;
    AT acc[R];
#pragma unroll
    for (int j = 0; j < R; ++j) acc[j] = AT(0);
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
          tmem_ld32(d_col + i * N2 + q * CW, v);
        else
          tmem_ld16(d_col + i * N2 + q * CW, v);
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
      const int pos = 2 * m + ph;
      ET e = ET(0);
      if (need_e) {
        if (!mbar_wait(&e_full[s & (kNE - 1)], (s / kNE) & 1, abort_flag, kSpinLimit)) break;
        e = estage[(s & (kNE - 1)) * kPos + pos];
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&ready[i]);  // D stage i free for step s + NS
      if (++i == NS) { i = 0; iph ^= 1; }

      const int yd = a.y0 + s - R + 1;
      const int x = a.xs_out + pos;
      if (s >= R - 1 && yd < a.yend && x < a.W) {
        const size_t xo = (size_t)x * a.nch + ch;  // element of the score-map row
        const double etd = cs.et;
        const ET et = static_cast<ET>(etd);
        double outd;
        float outf;
        if (SPLIT) {
          const double cc = (double)outv;
          const double ed = (double)e;
          if (a.measure == kCrossCorr) outd = cc;
          else if (a.measure == kSqrDistance) outd = ed - 2.0 * cc + etd;
          else if (a.measure == kCrossCorrNorm) outd = cc * rsqrt(ed * etd);
          else outd = (ed - 2.0 * cc + etd) * rsqrt(ed * etd);
          outf = (float)outd;
        } else {
          // Exact in int32: each of C, E_S, E_T <= 64 * 64 * 255^2 < 2^28.
          const int cc = static_cast<int>(outv);
          const int es = static_cast<int>(e), ei = static_cast<int>(et);
          const int num =
              (a.measure == kCrossCorr || a.measure == kCrossCorrNorm) ? cc : es - 2 * cc + ei;
          if (a.measure == kCrossCorr || a.measure == kSqrDistance) {
            outd = (double)num;
            outf = __int2float_rn(num);
          } else if ((double)a.tw * a.th * 65025.0 <= 16777216.0) {  // float sums exact
            outf = __fdiv_rn((float)num, __fsqrt_rn(__fmul_rn((float)es, (float)ei)));
            outd = outf;
          } else {
            outd = __ddiv_rn((double)num, __dsqrt_rn(__dmul_rn((double)es, (double)ei)));
            outf = (float)outd;
          }
        }
        char* o = a.dst + (size_t)yd * a.dst_pitch;
        if (a.dst_f64)
          reinterpret_cast<double*>(o)[xo] = outd;
        else
          reinterpret_cast<float*>(o)[xo] = outf;
      }
    }
  }

  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (threadIdx.x == 0) {
    for (int i = 0; i < kNRaw; ++i) mbar_inval(&raw_full[i]);
    for (int i = 0; i < NS; ++i) {
      mbar_inval(&ready[i]);
      mbar_inval(&mma_done[i]);
    }
    for (int i = 0; i < kNE; ++i) mbar_inval(&e_full[i]);
    mbar_inval(done_bar);
  }
}

// Template classes: R in {16, 32, 64} (template rows) x K (template columns
// + 1, padded to 16 for BF16 / 32 for i8).
template <int ELEM>
struct Classes {
  static constexpr int nk = ElemTraits<ELEM>::split ? 5 : 3;
  static constexpr int kstep = ElemTraits<ELEM>::split ? 16 : 32;
  static constexpr int kmax = nk * kstep;
};

template <int ELEM>
inline int class_of(int tw, int th) {
  typedef Classes<ELEM> C;
  const int r = th <= 16 ? 0 : th <= 32 ? 1 : 2;
  const int k = (tw + 1 + C::kstep - 1) / C::kstep - 1;
  return r * C::nk + k;
}

template <int ELEM>
__host__ __device__ inline void class_rk(int cls, int* R, int* K) {
  typedef Classes<ELEM> C;
  *R = 16 << (cls / C::nk);
  *K = (cls % C::nk + 1) * C::kstep;
}

template <int ELEM>
__device__ __forceinline__ void dispatch(int cls, const ItemArgs& a, unsigned char* smem,
                                         CtaState& cs) {
  if constexpr (ElemTraits<ELEM>::split) {
    switch (cls) {
      case 0: run_item<ELEM, 16, 16>(a, smem, cs); break;
      case 1: run_item<ELEM, 16, 32>(a, smem, cs); break;
      case 2: run_item<ELEM, 16, 48>(a, smem, cs); break;
      case 3: run_item<ELEM, 16, 64>(a, smem, cs); break;
      case 4: run_item<ELEM, 16, 80>(a, smem, cs); break;
      case 5: run_item<ELEM, 32, 16>(a, smem, cs); break;
      case 6: run_item<ELEM, 32, 32>(a, smem, cs); break;
      case 7: run_item<ELEM, 32, 48>(a, smem, cs); break;
      case 8: run_item<ELEM, 32, 64>(a, smem, cs); break;
      case 9: run_item<ELEM, 32, 80>(a, smem, cs); break;
      case 10: run_item<ELEM, 64, 16>(a, smem, cs); break;
      case 11: run_item<ELEM, 64, 32>(a, smem, cs); break;
      case 12: run_item<ELEM, 64, 48>(a, smem, cs); break;
      case 13: run_item<ELEM, 64, 64>(a, smem, cs); break;
      default: run_item<ELEM, 64, 80>(a, smem, cs); break;
    }
  } else {
    switch (cls) {
      case 0: run_item<ELEM, 16, 32>(a, smem, cs); break;
      case 1: run_item<ELEM, 16, 64>(a, smem, cs); break;
      case 2: run_item<ELEM, 16, 96>(a, smem, cs); break;
      case 3: run_item<ELEM, 32, 32>(a, smem, cs); break;
      case 4: run_item<ELEM, 32, 64>(a, smem, cs); break;
      case 5: run_item<ELEM, 32, 96>(a, smem, cs); break;
      case 6: run_item<ELEM, 64, 32>(a, smem, cs); break;
      case 7: run_item<ELEM, 64, 64>(a, smem, cs); break;
      default: run_item<ELEM, 64, 96>(a, smem, cs); break;
    }
  }
}

// Batch tables (device memory).
struct BatchImage {
  int W, H, nch;
};
struct BatchTemplate {
  const char* ptr;
  size_t pitch;
  int tw, th, cls;
};
struct BatchDest {
  char* ptr;
  size_t pitch;
  int f64;
};
struct BatchItem {
  int img, tpl, dst;  // indices into the tables
  int ch, strip, y0, yend;
};

struct TensorLaunch {
  CUtensorMap map;     // single-image mode: the source planes
  int mode;            // 0: one (image, template) pair, items from blockIdx; 1: work queue
  int measure;
  int nbox;            // 16-byte groups per staged row (all tensor maps of the launch)
  int* err;
  // mode 0
  ItemArgs base;       // fields common to every item
  int cls, BH;
  // mode 1
  const CUtensorMap* maps;  // one per image (64-byte aligned)
  const BatchImage* imgs;
  const BatchTemplate* tpls;
  const BatchDest* dsts;
  const BatchItem* items;
  int nitems;
  int* counter;        // next item; reset to 0 before every launch
};

// One kernel per element type. Mode 0 (one image and template): CTA
// (x, y, z) = (strip, band, channel). Mode 1 (batch): one persistent CTA per
// SM takes items from a global counter until none are left.
template <int ELEM>
__global__ void __launch_bounds__(kThreads, 1)
    prox_tensor_kernel(const __grid_constant__ TensorLaunch P) {
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ CtaState cs;
  const int warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) cs.abort = 0;
  if (warp == 0) tmem_alloc(&cs.tmem, kTmemCols);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();

  // The item's arguments live in shared memory: read where they are used,
  // they take no registers from the roles' accumulators.
  __shared__ ItemArgs item;
  __shared__ int item_cls;
  if (P.mode == 0) {
    if (threadIdx.x == 0) {
      item = P.base;
      item.tmap = &P.map;
      item.ch = blockIdx.z;
      item.xs_out = blockIdx.x * kPos;
      item.y0 = blockIdx.y * P.BH;
      item.yend = min(item.H, item.y0 + P.BH);
    }
    __syncthreads();
    dispatch<ELEM>(P.cls, item, smem, cs);
  } else {
    for (;;) {
      if (threadIdx.x == 0) {
        const int it = cs.abort ? P.nitems : atomicAdd(P.counter, 1);
        cs.next = it;
        if (it < P.nitems) {
          const BatchItem bi = P.items[it];
          const BatchImage im = P.imgs[bi.img];
          const BatchTemplate tp = P.tpls[bi.tpl];
          const BatchDest ds = P.dsts[bi.dst];
          item.tmap = P.maps + bi.img;
          item.W = im.W;
          item.H = im.H;
          item.tw = tp.tw;
          item.th = tp.th;
          item.ax = tp.tw / 2;
          item.ay = tp.th / 2;
          item.nch = im.nch;
          item.ch = bi.ch;
          item.xs_out = bi.strip * kPos;
          item.y0 = bi.y0;
          item.yend = bi.yend;
          item.nbox = P.nbox;
          item.tmpl = tp.ptr;
          item.tmpl_pitch = tp.pitch;
          item.dst = ds.ptr;
          item.dst_pitch = ds.pitch;
          item.dst_f64 = ds.f64;
          item.measure = P.measure;
          item_cls = tp.cls;
        }
      }
      __syncthreads();
      const int it = cs.next;
      if (it >= P.nitems) break;
      dispatch<ELEM>(item_cls, item, smem, cs);
      __syncthreads();  // every thread has read the item before it is replaced
    }
  }

  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    tmem_dealloc(cs.tmem, kTmemCols);
  }
  if (threadIdx.x == 0 && cs.abort) atomicExch(P.err, 1);
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

template <int ELEM>
int nbox_for(int K) {
  typedef ElemTraits<ELEM> TR;
  // Lane m reads pixels lead + 2m .. lead + 2m + K (one more for odd leads).
  return (kPos + K + 2 * TR::inner + 1) / TR::inner;
}

// Rank-4 view of source planes: 16-byte groups (dim 0), groups along the row
// (dim 1), rows (dim 2), channels (dim 3). A staged row of 256 + K pixels is
// one box of nbox groups, under the 256-element box limit. The last group of
// a row may reach into the row pitch, which is zero (image creation
// zero-fills device buffers; the channel split writes zeros there).
template <int ELEM>
cudaError_t encode_planes(CUtensorMap* map, const void* planes, int W, int H, int nch,
                          size_t plane_pitch, size_t plane_bytes, int nbox) {
  typedef ElemTraits<ELEM> TR;
  EncodeTiledFn enc = encode_fn();
  if (!enc) return cudaErrorNotSupported;
  const CUtensorMapDataType dt = ELEM == kF32   ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32
                                 : ELEM == kU16 ? CU_TENSOR_MAP_DATA_TYPE_UINT16
                                                : CU_TENSOR_MAP_DATA_TYPE_UINT8;
  const cuuint64_t gdim[4] = {(cuuint64_t)TR::inner, (cuuint64_t)((W + TR::inner - 1) / TR::inner),
                              (cuuint64_t)H, (cuuint64_t)nch};
  const cuuint64_t gstride[3] = {16, (cuuint64_t)plane_pitch, (cuuint64_t)plane_bytes};
  const cuuint32_t box[4] = {(cuuint32_t)TR::inner, (cuuint32_t)nbox, (cuuint32_t)kRB, 1};
  const cuuint32_t estride[4] = {1, 1, 1, 1};
  CUresult r = enc(map, dt, 4, const_cast<void*>(planes), gdim, gstride, box, estride,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                   CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

// Splits an nch-channel image into planes at `planes` (row pitch rounded up
// to 128 bytes). Returns the plane pitch.
template <int ELEM>
size_t split_channels(const DevImage& src, char* planes, cudaStream_t stream, bool count = true) {
  typedef ElemTraits<ELEM> TR;
  const size_t plane_pitch = ((size_t)src.width * TR::size + 127) / 128 * 128;
  const size_t plane_bytes = plane_pitch * src.height;
  typedef typename std::conditional<TR::size == 4, uint32_t,
                                    typename std::conditional<TR::size == 2, uint16_t,
                                                              uint8_t>::type>::type PT;
  const int pw = static_cast<int>(plane_pitch / TR::size);  // row length incl. the tail
  dim3 sg((pw + 255) / 256, src.height);
  split_channels_kernel<PT><<<sg, 256, 0, stream>>>((const char*)src.ptr, src.pitch, planes,
                                                    plane_pitch, plane_bytes, src.width, pw,
                                                    src.height, src.nch);
  if (count) count_launches(1);
  return plane_pitch;
}

size_t plane_set_bytes(const DevImage& s) {
  const size_t pitch = ((size_t)s.width * type_bytes(s.type) + 127) / 128 * 128;
  return pitch * s.height * s.nch;
}

template <int ELEM>
int smem_for_class(int cls, int nbox) {
  int R, K;
  class_rk<ELEM>(cls, &R, &K);
  return std::max(make_layout(ElemTraits<ELEM>::split, R, K, nbox).total, kMinSmem);
}

template <int ELEM>
cudaError_t launch_one(Context& ctx, Measure m, const DevImage& src, const DevImage& tmpl,
                       const DevImage& dst, int ax, int ay) {
  const int cls = class_of<ELEM>(tmpl.width, tmpl.height);
  int R, K;
  class_rk<ELEM>(cls, &R, &K);
  TensorLaunch P;
  std::memset(&P, 0, sizeof(P));
  P.mode = 0;
  P.measure = m;
  P.nbox = nbox_for<ELEM>(K);
  P.err = reinterpret_cast<int*>(ctx.scratch(Context::kTensorAux, 256));
  P.cls = cls;
  const int nstrips = (src.width + kPos - 1) / kPos;
  P.BH = band_height(src.height, R, (long long)nstrips * src.nch, ctx.sm_count);
  ItemArgs& a = P.base;
  a.W = src.width;
  a.H = src.height;
  a.tw = tmpl.width;
  a.th = tmpl.height;
  a.ax = ax;
  a.ay = ay;
  a.nch = src.nch;
  a.nbox = P.nbox;
  a.tmpl = (const char*)tmpl.ptr;
  a.tmpl_pitch = tmpl.pitch;
  a.dst = (char*)dst.ptr;
  a.dst_pitch = dst.pitch;
  a.dst_f64 = dst.type == F64;
  a.measure = m;

  // Source planes: the image itself for one channel, else a split copy.
  const void* planes = src.ptr;
  size_t plane_pitch = src.pitch;
  if (src.nch > 1) {
    char* pl = reinterpret_cast<char*>(ctx.scratch(Context::kPlanes, plane_set_bytes(src)));
    plane_pitch = split_channels<ELEM>(src, pl, ctx.stream);
    planes = pl;
  }
  cudaError_t e = encode_planes<ELEM>(&P.map, planes, src.width, src.height, src.nch,
                                      plane_pitch, plane_pitch * src.height, P.nbox);
  if (e != cudaSuccess) return e;

  const int smem_bytes = smem_for_class<ELEM>(cls, P.nbox);
  auto kern = prox_tensor_kernel<ELEM>;
  e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           kMaxDynSmem);
  if (e != cudaSuccess) return e;
  dim3 grid(nstrips, (src.height + P.BH - 1) / P.BH, src.nch);
  kern<<<grid, kThreads, smem_bytes, ctx.stream>>>(P);
  count_launches(1);
  return cudaGetLastError();
}

// ---- Batches ------------------------------------------------------------------

// Autotuned band heights, per (element type, template class, channels).
std::mutex g_tune_mutex;
std::map<std::tuple<int, int, int>, int> g_tuned_bh;

}  // namespace

struct TensorBatch {
  Context* ctx = nullptr;
  int elem = 0;
  int measure = 0;
  int nbox = 0;
  int smem = 0;
  int nitems = 0;
  void* tables = nullptr;  // maps, images, templates, dests, items, counter
  char* planes = nullptr;  // channel planes of multi-channel images
  std::vector<std::pair<int, size_t>> plane_offsets;  // per image: (split?, offset)
  std::vector<DevImage> images;
  TensorLaunch launch;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  std::map<int, int> bh;  // class -> band height used
};

namespace {

// Channel splits, queue reset, persistent launch. `count` is false while the
// work is recorded into a graph (counted when the graph is launched).
template <int ELEM>
cudaError_t batch_record(TensorBatch& b, cudaStream_t stream, bool count) {
  for (size_t i = 0; i < b.images.size(); ++i) {
    if (b.plane_offsets[i].first)
      split_channels<ELEM>(b.images[i], b.planes + b.plane_offsets[i].second, stream, count);
  }
  cudaError_t e = cudaMemsetAsync(b.launch.counter, 0, sizeof(int), stream);
  if (e != cudaSuccess) return e;
  auto kern = prox_tensor_kernel<ELEM>;
  kern<<<b.ctx->sm_count, kThreads, b.smem, stream>>>(b.launch);
  if (count) count_launches(1);
  return cudaGetLastError();
}

// Builds the item list of a batch: every (image, template) pair, channel,
// strip and band; the largest items first, so the queue ends on small ones.
template <int ELEM>
std::vector<BatchItem> make_items(const std::vector<DevImage>& imgs,
                                  const std::vector<DevImage>& tpls,
                                  const std::vector<int>& pair_img,
                                  const std::vector<int>& pair_tpl,
                                  const std::vector<int>& pair_dst,
                                  const std::map<int, int>& bh) {
  std::vector<std::pair<long long, BatchItem>> v;
  for (size_t p = 0; p < pair_img.size(); ++p) {
    const DevImage& s = imgs[pair_img[p]];
    const DevImage& t = tpls[pair_tpl[p]];
    const int cls = class_of<ELEM>(t.width, t.height);
    int R, K;
    class_rk<ELEM>(cls, &R, &K);
    const int BH = bh.at(cls);
    const int nstrips = (s.width + kPos - 1) / kPos;
    for (int c = 0; c < s.nch; ++c)
      for (int st = 0; st < nstrips; ++st)
        for (int y0 = 0; y0 < s.height; y0 += BH) {
          BatchItem it;
          it.img = pair_img[p];
          it.tpl = pair_tpl[p];
          it.dst = pair_dst[p];
          it.ch = c;
          it.strip = st;
          it.y0 = y0;
          it.yend = std::min(s.height, y0 + BH);
          // steps x MMA work per step (K columns, plus a fixed part)
          const long long cost = (long long)(it.yend - y0 + R - 1) * (K + 64);
          v.push_back({cost, it});
        }
  }
  std::stable_sort(v.begin(), v.end(),
                   [](const std::pair<long long, BatchItem>& a,
                      const std::pair<long long, BatchItem>& b) { return a.first > b.first; });
  std::vector<BatchItem> out;
  out.reserve(v.size());
  for (auto& x : v) out.push_back(x.second);
  return out;
}

// Device tables of a batch in one allocation; returns the TensorLaunch
// pointers into it.
template <int ELEM>
cudaError_t upload_tables(TensorBatch& b, const std::vector<CUtensorMap>& maps,
                          const std::vector<BatchImage>& bimgs,
                          const std::vector<BatchTemplate>& btpls,
                          const std::vector<BatchDest>& bdsts,
                          const std::vector<BatchItem>& items, void** mem) {
  auto al = [](size_t x) { return (x + 255) / 256 * 256; };
  const size_t o_maps = 0;
  const size_t o_imgs = al(o_maps + maps.size() * sizeof(CUtensorMap));
  const size_t o_tpls = al(o_imgs + bimgs.size() * sizeof(BatchImage));
  const size_t o_dsts = al(o_tpls + btpls.size() * sizeof(BatchTemplate));
  const size_t o_items = al(o_dsts + bdsts.size() * sizeof(BatchDest));
  const size_t o_ctr = al(o_items + items.size() * sizeof(BatchItem));
  const size_t total = o_ctr + 256;
  std::vector<char> host(total, 0);
  std::memcpy(host.data() + o_maps, maps.data(), maps.size() * sizeof(CUtensorMap));
  std::memcpy(host.data() + o_imgs, bimgs.data(), bimgs.size() * sizeof(BatchImage));
  std::memcpy(host.data() + o_tpls, btpls.data(), btpls.size() * sizeof(BatchTemplate));
  std::memcpy(host.data() + o_dsts, bdsts.data(), bdsts.size() * sizeof(BatchDest));
  std::memcpy(host.data() + o_items, items.data(), items.size() * sizeof(BatchItem));
  char* d = nullptr;
  cudaError_t e = cudaMalloc(&d, total);
  if (e != cudaSuccess) return e;
  e = cudaMemcpy(d, host.data(), total, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    cudaFree(d);
    return e;
  }
  *mem = d;
  TensorLaunch& P = b.launch;
  P.maps = reinterpret_cast<const CUtensorMap*>(d + o_maps);
  P.imgs = reinterpret_cast<const BatchImage*>(d + o_imgs);
  P.tpls = reinterpret_cast<const BatchTemplate*>(d + o_tpls);
  P.dsts = reinterpret_cast<const BatchDest*>(d + o_dsts);
  P.items = reinterpret_cast<const BatchItem*>(d + o_items);
  P.nitems = static_cast<int>(items.size());
  P.counter = reinterpret_cast<int*>(d + o_ctr);
  return cudaSuccess;
}

// Autotuner: for one template class, times the persistent kernel on the
// probe pair (first image and template of that class) replicated so that
// every band height sees the same total work and enough items for all SMs,
// and keeps the band height with the least time per pair. The candidates
// span the trade-off between ramp rows (R - 1 per band, favouring tall
// bands) and load balance (favouring short ones).
template <int ELEM>
int autotune_bh(Context& ctx, int measure, const DevImage& img, const CUtensorMap& map,
                const DevImage& tpl, int cls, int nbox, char* probe_dst, size_t probe_pitch) {
  int R, K;
  class_rk<ELEM>(cls, &R, &K);
  std::vector<int> cand;
  for (int bh : {64, 128, 192, 256, 384, 512, 768, 1024})
    if (bh >= R && bh < img.height) cand.push_back(bh);
  cand.push_back(img.height);
  const int nstrips = (img.width + kPos - 1) / kPos;
  const long long units = (long long)nstrips * img.nch;
  // Replicas so that the shortest candidate has at least 4 items per SM.
  const int min_bh = cand.front();
  const long long items_min = units * ((img.height + min_bh - 1) / min_bh);
  const int reps = (int)std::max<long long>(
      1, std::min<long long>(64, (4LL * ctx.sm_count + items_min - 1) / items_min));
  std::vector<CUtensorMap> maps(1, map);
  std::vector<BatchImage> bimgs(1, BatchImage{img.width, img.height, img.nch});
  std::vector<BatchTemplate> btpls(1, BatchTemplate{(const char*)tpl.ptr, tpl.pitch, tpl.width,
                                                    tpl.height, cls});
  std::vector<BatchDest> bdsts(1, BatchDest{probe_dst, probe_pitch, 0});
  float best = 1e30f;
  int best_bh = cand.back();
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  for (int bh : cand) {
    std::vector<int> pi(reps, 0), pt(reps, 0), pd(reps, 0);
    std::map<int, int> m1{{cls, bh}};
    std::vector<BatchItem> items = make_items<ELEM>({img}, {tpl}, pi, pt, pd, m1);
    TensorBatch tb;
    tb.ctx = &ctx;
    std::memset(&tb.launch, 0, sizeof(tb.launch));
    tb.launch.mode = 1;
    tb.launch.measure = measure;
    tb.launch.nbox = nbox;
    tb.launch.err = reinterpret_cast<int*>(ctx.scratch(Context::kTensorAux, 256));
    tb.smem = smem_for_class<ELEM>(cls, nbox);
    void* mem = nullptr;
    if (upload_tables<ELEM>(tb, maps, bimgs, btpls, bdsts, items, &mem) != cudaSuccess) break;
    float ms = 1e30f;
    for (int rep = 0; rep < 3; ++rep) {
      cudaEventRecord(e0, ctx.stream);
      batch_record<ELEM>(tb, ctx.stream, true);
      cudaEventRecord(e1, ctx.stream);
      cudaEventSynchronize(e1);
      float t = 0.f;
      cudaEventElapsedTime(&t, e0, e1);
      if (rep > 0) ms = std::min(ms, t);  // the first run warms up
    }
    cudaFree(mem);
    if (ms < best) {
      best = ms;
      best_bh = bh;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return best_bh;
}

template <int ELEM>
TensorBatch* batch_create(Context& ctx, Measure m, const std::vector<DevImage>& imgs,
                          const std::vector<DevImage>& tpls, const std::vector<DevImage>& dsts,
                          cudaError_t* err) {
  typedef Classes<ELEM> C;
  TensorBatch* b = new TensorBatch();
  b->ctx = &ctx;
  b->elem = ELEM;
  b->measure = m;
  b->nbox = nbox_for<ELEM>(C::kmax);
  b->images = imgs;
  std::memset(&b->launch, 0, sizeof(b->launch));
  cudaError_t e = cudaSuccess;
  auto fail = [&](cudaError_t code) {
    *err = code;
    tensor_batch_destroy(b);
    return static_cast<TensorBatch*>(nullptr);
  };

  // Channel planes of multi-channel images (owned by the batch).
  size_t plane_total = 0;
  for (const DevImage& s : imgs) {
    b->plane_offsets.push_back({s.nch > 1 ? 1 : 0, plane_total});
    if (s.nch > 1) plane_total += plane_set_bytes(s);
  }
  if (plane_total) {
    e = cudaMalloc(&b->planes, plane_total);
    if (e != cudaSuccess) return fail(e);
  }
  std::vector<CUtensorMap> maps(imgs.size());
  for (size_t i = 0; i < imgs.size(); ++i) {
    const DevImage& s = imgs[i];
    const void* planes = s.ptr;
    size_t pitch = s.pitch;
    if (s.nch > 1) {
      planes = b->planes + b->plane_offsets[i].second;
      pitch = (plane_set_bytes(s) / s.nch) / s.height;
    }
    e = encode_planes<ELEM>(&maps[i], planes, s.width, s.height, s.nch, pitch,
                            pitch * s.height, b->nbox);
    if (e != cudaSuccess) return fail(e);
  }
  std::vector<BatchImage> bimgs;
  for (const DevImage& s : imgs) bimgs.push_back(BatchImage{s.width, s.height, s.nch});
  std::vector<BatchTemplate> btpls;
  for (const DevImage& t : tpls)
    btpls.push_back(BatchTemplate{(const char*)t.ptr, t.pitch, t.width, t.height,
                                  class_of<ELEM>(t.width, t.height)});
  std::vector<BatchDest> bdsts;
  for (const DevImage& d : dsts) bdsts.push_back(BatchDest{(char*)d.ptr, d.pitch, d.type == F64});

  auto kern = prox_tensor_kernel<ELEM>;
  e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
  if (e != cudaSuccess) return fail(e);

  // Multi-channel probes read the planes: split them once before tuning.
  for (size_t i = 0; i < imgs.size(); ++i)
    if (b->plane_offsets[i].first)
      split_channels<ELEM>(imgs[i], b->planes + b->plane_offsets[i].second, ctx.stream);

  // Band height per template class: autotuned once per (type, class,
  // channels) and kept for the process.
  std::map<int, int> bh;
  for (size_t j = 0; j < tpls.size(); ++j) {
    const int cls = btpls[j].cls;
    if (bh.count(cls)) continue;
    const auto key = std::make_tuple(ELEM, cls, imgs[0].nch);
    {
      std::lock_guard<std::mutex> lk(g_tune_mutex);
      auto it = g_tuned_bh.find(key);
      if (it != g_tuned_bh.end()) {
        bh[cls] = it->second;
        continue;
      }
    }
    const DevImage& probe = imgs[0];
    char* pd = nullptr;
    const size_t pp = ((size_t)probe.width * probe.nch * 4 + 127) / 128 * 128;
    e = cudaMalloc(&pd, pp * probe.height);
    if (e != cudaSuccess) return fail(e);
    const int v = autotune_bh<ELEM>(ctx, m, probe, maps[0], tpls[j], cls, b->nbox, pd, pp);
    cudaStreamSynchronize(ctx.stream);
    cudaFree(pd);
    e = cudaGetLastError();
    if (e != cudaSuccess) return fail(e);
    bh[cls] = v;
    std::lock_guard<std::mutex> lk(g_tune_mutex);
    g_tuned_bh[key] = v;
  }
  b->bh = bh;

  std::vector<int> pi, pt, pd;
  for (size_t i = 0; i < imgs.size(); ++i)
    for (size_t j = 0; j < tpls.size(); ++j) {
      pi.push_back((int)i);
      pt.push_back((int)j);
      pd.push_back((int)(i * tpls.size() + j));
    }
  std::vector<BatchItem> items = make_items<ELEM>(imgs, tpls, pi, pt, pd, bh);
  b->launch.mode = 1;
  b->launch.measure = m;
  b->launch.nbox = b->nbox;
  b->launch.err = reinterpret_cast<int*>(ctx.scratch(Context::kTensorAux, 256));
  e = upload_tables<ELEM>(*b, maps, bimgs, btpls, bdsts, items, &b->tables);
  if (e != cudaSuccess) return fail(e);
  b->nitems = b->launch.nitems;
  b->smem = 0;
  for (const auto& kv : bh) b->smem = std::max(b->smem, smem_for_class<ELEM>(kv.first, b->nbox));

  // Capture the batch (splits, queue reset, persistent launch) as a graph.
  e = cudaStreamSynchronize(ctx.stream);
  if (e != cudaSuccess) return fail(e);
  e = cudaStreamBeginCapture(ctx.stream, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) return fail(e);
  const cudaError_t re = batch_record<ELEM>(*b, ctx.stream, false);
  e = cudaStreamEndCapture(ctx.stream, &b->graph);
  if (re != cudaSuccess) return fail(re);
  if (e != cudaSuccess) return fail(e);
  e = cudaGraphInstantiate(&b->exec, b->graph, 0);
  if (e != cudaSuccess) return fail(e);
  *err = cudaSuccess;
  return b;
}

}  // namespace

namespace {

// One thread waits on an mbarrier that nothing arrives on, with the bounded
// wait of the tensor kernels: the wait expires, sets the abort flag, and the
// kernel raises the context's error flag and returns.
__global__ void bounded_wait_probe_kernel(long long limit, int* err) {
  __shared__ uint64_t bar;
  __shared__ int abort_flag;
  if (threadIdx.x == 0) {
    abort_flag = 0;
    mbar_init(&bar, 1);
    fence_barrier_init();
    const bool ok = mbar_wait(&bar, 0, &abort_flag, limit);
    if (!ok) atomicExch(err, 1);
    mbar_inval(&bar);
  }
}

}  // namespace

cudaError_t launch_bounded_wait_probe(Context& ctx, long long limit_cycles) {
  int* err = reinterpret_cast<int*>(ctx.scratch(Context::kTensorAux, 256));
  bounded_wait_probe_kernel<<<1, 32, 0, ctx.stream>>>(limit_cycles, err);
  count_launches(1);
  return cudaGetLastError();
}

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
  return launch_proximity_tensor_anchored(ctx, m, src, tmpl, dst, tmpl.width / 2,
                                          tmpl.height / 2);
}

cudaError_t launch_proximity_tensor_anchored(Context& ctx, Measure m, const DevImage& src,
                                             const DevImage& tmpl, const DevImage& dst, int ax,
                                             int ay) {
  if (src.type == U8) return launch_one<kU8>(ctx, m, src, tmpl, dst, ax, ay);
  if (src.type == U16) return launch_one<kU16>(ctx, m, src, tmpl, dst, ax, ay);
  return launch_one<kF32>(ctx, m, src, tmpl, dst, ax, ay);
}

TensorBatch* tensor_batch_create(Context& ctx, Measure m, const std::vector<DevImage>& imgs,
                                 const std::vector<DevImage>& tpls,
                                 const std::vector<DevImage>& dsts, cudaError_t* err) {
  if (imgs[0].type == U8) return batch_create<kU8>(ctx, m, imgs, tpls, dsts, err);
  if (imgs[0].type == U16) return batch_create<kU16>(ctx, m, imgs, tpls, dsts, err);
  return batch_create<kF32>(ctx, m, imgs, tpls, dsts, err);
}

cudaError_t tensor_batch_run(TensorBatch* b) {
  count_launches(1 + std::count_if(b->plane_offsets.begin(), b->plane_offsets.end(),
                                   [](const std::pair<int, size_t>& p) { return p.first != 0; }));
  return cudaGraphLaunch(b->exec, b->ctx->stream);
}

int tensor_batch_items(const TensorBatch* b) { return b->nitems; }

int tensor_batch_band_height(const TensorBatch* b, int tw, int th) {
  int cls = 0;
  if (b->elem == kU8) cls = class_of<kU8>(tw, th);
  else cls = class_of<kF32>(tw, th);
  auto it = b->bh.find(cls);
  return it == b->bh.end() ? 0 : it->second;
}

void tensor_batch_destroy(TensorBatch* b) {
  if (!b) return;
  if (b->ctx) cudaStreamSynchronize(b->ctx->stream);
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  if (b->tables) cudaFree(b->tables);
  if (b->planes) cudaFree(b->planes);
  delete b;
}

}  // namespace ocipb
