// Tensor-core (tcgen05) ImageProximity path for sm_100a.
//
// The product term of SqrDistance[_Norm] and CrossCorr[_Norm]
// (cl-files/ImageProximity.cl :44, :122, :290, :375),
//   C(x, y) = sum_h sum_w S(x + w - ax, y + h - ay) * T(w, h),
// is computed per channel and strip of P = 128 S output positions by one
// chain of MMAs per source row. TMEM lane m holds the S positions
// x0 + S m + p (p < S). R (template rows rounded up to 16, 32 or 64) and S
// satisfy S R = 128: S = 8, 4, 2. An MMA instruction (M = 128, K = 16) takes
// the same time for any N up to 256, so the kernel makes N as wide as the
// accumulators in TMEM allow.
//
// A operand (shared memory, no per-lane copies). Lane m's K window is the
// staged row itself, A[m][k] = raw(S m + k): a Hankel matrix. In the
// canonical K-major SWIZZLE_NONE layout a core matrix row is 16 bytes, so the
// row is stored once more per S pixels: buffer row q holds raw elements
// S q .. S q + 7 (BF16) or .. + 15 (i8), and core matrix c of lane m is buffer
// row m + c (8/S) [(16/S) for i8]: one descriptor per MMA with SBO = 128 and
// LBO = the distance of the next K core matrix.
//
// F32 and U16 sources are split into BF16 hi + lo (U16 exactly) and three
// products hi*Thi + hi*Tlo + lo*Thi accumulate in FP32. They are packed into
// MMAs of K = 16 by pairing core matrices along K: (hi_c, lo_c) x (Tlo_c, Thi_c)
// for every chunk c, then (hi_2i, hi_2i+1) x (Thi_2i, Thi_2i+1). U8 sources use
// the i8 MMA with s32 accumulation (exact).
//
// B operand: N = S R = 128 rows, row S j + p = template row th - 1 - j at phase
// p, shifted by the staged row's lead: B[S j + p][k] = T(k - p - lead, th-1-j).
// Source row t then adds to output-row slots t .. t + R - 1 (slot u is the
// output row whose last template row is source row u).
//
// Blocks. The steps (source rows) of an item are cut into blocks of
// B = 16 / S steps. Step q of a block adds into TMEM columns S q + [0, N) of
// the block's partial buffer: MMAs of N' = N + 16 = 144 columns at the
// buffer's first column with B read S q rows later (B is stored with 16 - S
// zero rows in front), so the block's partial sums of its B + R - 1 slots
// end up at columns S j + p. The block's first MMA does not accumulate, which
// clears the buffer. Partial buffers are double-buffered: the epilogue reads
// block k while the tensor cores fill block k + 1.
//
// Running sums. The epilogue adds each block's partials into a ring of
// running sums in TMEM that only it reads and writes (slot u at ring columns
// S (u mod NS) + p, NS S = 144 columns; FP32 round-to-nearest, exact int32
// for U8). The block's first 16 columns are the B slots it completes: the
// epilogue writes them out and clears their ring columns. The tensor cores'
// FP32 accumulation into one value thus never spans more than one block:
// that accumulator rounds every addition with a bias that grows with the
// number of additions, so the chains of a whole window (th rows x K chunks)
// would cost accuracy.
//
// Window energies sum S^2 of each position (measures other than CrossCorr):
// a separate pre-pass (row_energy.cu) writes the row energies R(x, r) =
// sum_{w < tw} S^2(x + w - ax, r) of every source row (int32 for U8, FP32
// otherwise); the epilogue keeps each position's window energy as an FP64
// running sum over the rows it walks (add R of the row a slot completes,
// drop R of the row th back), loading a block's R values before it waits for
// the block's MMAs. Exact for U8; 2^-24 relative for F32 and U16.
// SqrDistance = E_S - 2C + E_T and the _Norm scale are done in FP64 (F32,
// U16) or as the plain path does them (U8: the results are bit-identical to
// it).
//
// Roles (10 warps; one CTA per SM, which holds all 512 TMEM columns):
//   warps 0-3  builders: the A operand of each row (split into hi/lo);
//   warps 4-7  epilogue (warp 4 + k reads TMEM lanes 32k .. 32k + 31): running
//              sums in the TMEM ring, window energies, score map;
//   warp 8     TMA loads of source rows (zero fill outside the image);
//   warp 9     MMA issue (one commit per block of rows: the block's partial
//              and its A stages are free once it completes).
// Every wait is bounded: a wait that gives up sets the CTA's abort flag, the
// roles leave their loops, the MMA and TMA threads drain what they issued,
// and the kernel raises the context's error flag.
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
#include "row_energy.h"

namespace ocipb {
namespace {

using namespace sm100;

constexpr int kM = 128;                 // TMEM lanes = A rows
constexpr int kBuilders = 4;
constexpr int kEpilogue = 4;
constexpr int kTmaWarp = kBuilders + kEpilogue;
constexpr int kMmaWarp = kTmaWarp + 1;
constexpr int kThreads = (kMmaWarp + 1) * 32;
constexpr int kBuildThreads = kBuilders * 32;
constexpr int kNRaw = 6;                // staged source rows (TMA stages of one row)
constexpr int kMaxNA = 16;              // A operand stages at most (two blocks of rows)
constexpr int kSR = 128;                // S R: template rows x positions per lane
constexpr int kN = kSR;                 // B rows (MMA N without the slide)
constexpr int kNp = kN + 16;            // MMA N: a block's B - 1 slides fit in 16 more
constexpr int kPartCols = kNp;          // TMEM columns per partial buffer (two of them)
constexpr int kRingCol = 2 * kPartCols; // first TMEM column of the running-sum ring
constexpr int kRingCols = kNp;          // ring columns: NS S = 144 (9 chunks of 16)
constexpr int kTmemCols = 512;
constexpr int kMinSmem = 120 * 1024;    // keeps one CTA per SM (it takes all of TMEM)
constexpr int kMaxDynSmem = 226 * 1024; // opt-in dynamic shared memory limit of the kernel
constexpr long long kSpinLimit = 4000000000LL;  // about 2 s of SM clock
constexpr int kBarBuild = 1;            // named barrier of the builder warps

enum Elem { kF32 = 0, kU8 = 1, kU16 = 2 };

template <int ELEM>
struct ElemTraits {
  static constexpr bool split = ELEM != kU8;  // BF16 hi/lo operands
  static constexpr int size = ELEM == kF32 ? 4 : ELEM == kU16 ? 2 : 1;
  static constexpr int inner = 16 / size;     // elements per 16-byte TMA group
  static constexpr int cmk = split ? 8 : 16;  // K elements per core-matrix row
};

// Positions per TMEM lane for a template of R rows (S R = 128), and the steps
// of a block (S B = 16: a block's completed slots are one 16-column chunk).
__host__ __device__ constexpr int s_for(int R) { return kSR / R; }
__host__ __device__ constexpr int block_steps(int S) { return 16 / S; }

// Geometry of one work item (host and device).
struct Geo {
  int S, P, Q, R, B;
  int NB;          // B-operand rows stored per core matrix
  int KC;          // core matrices of one K segment
  int nmma;        // MMAs per source row
  int cma;         // A core matrices addressed per lane (hi, incl. the pairing's spare)
  int QR;          // buffer rows of one A plane
  int lbok;        // bytes between K-adjacent core matrices of A
  int nraw;        // staged elements the windows cover (lead + P - 1 + tw)
  int NA;          // A operand stages: two blocks of steps
};

__host__ __device__ inline Geo make_geo(bool split, int R, int tw, int lead) {
  Geo g;
  g.S = s_for(R);
  g.P = kM * g.S;
  g.Q = 16 / g.S;
  g.R = R;
  g.B = block_steps(g.S);
  g.NB = kN + 32 - g.S;
  const int cmk = split ? 8 : 16;
  const int keff = tw + g.S - 1 + lead;
  g.KC = (keff + cmk - 1) / cmk;
  if (split) {
    g.nmma = g.KC + (g.KC + 1) / 2;
    g.cma = 2 * ((g.KC + 1) / 2);
  } else {
    g.nmma = (g.KC + 1) / 2;
    g.cma = 2 * g.nmma;
  }
  g.lbok = 16 * (cmk / g.S);
  g.QR = kM + (cmk / g.S) * (g.cma - 1);
  g.nraw = lead + g.P - 1 + tw;
  g.NA = 2 * g.B;
  return g;
}

// Staged elements of one row: the last buffer row's end, and every element
// of the strip's windows.
__host__ __device__ inline int staged_elems(const Geo& g, bool split) {
  const int a = g.S * (g.QR - 1) + (split ? 8 : 16);
  return a > g.nraw ? a : g.nraw;
}

// One work item: one channel of one strip x band of rows of one
// (image, template) pair.
struct ItemArgs {
  const CUtensorMap* tmap;  // source planes (rank 4: group, groups, rows, channel)
  int W, H;
  int tw, th, R;
  int ax, ay;    // window anchor: output (x, y) reads S(x + w - ax, y + h - ay)
  int nch, ch;
  int xs_out;    // strip covers outputs [xs_out, xs_out + P)
  int y0, yend;  // band of output rows
  int nbox;      // 16-byte groups per staged row (box_split loads of box_part)
  const char* tmpl;
  size_t tmpl_pitch;
  char* dst;
  size_t dst_pitch;
  int dst_f64;
  int measure;
  // Row energies (measures other than CrossCorr): int32 (U8) or FP32 planes
  // of R(x, r), plane ch at energy + ch * e_plane bytes, rows e_pitch apart.
  const char* energy;
  size_t e_pitch, e_plane;
  // 1: add the scores (raw CrossCorr sums into an F64 map) to the
  // destination instead of writing them (templates tiled over launches).
  int accum;
  // Best match (ocipProximityIndx): -1 none, else the index reduction
  // (0 min, 1 max, 2 min |v|, 3 max |v|) of the F32 scores; each epilogue
  // warp writes one IdxRecord per item to idx_out[item * 4 + warp]. dst may
  // then be null (no map written).
  int idx_op;
  char* idx_out;
};

// Best score of an epilogue warp's positions in one item. Among equal values
// the smallest key wins: key = (reference work-group index << 12) |
// (bit-reversed work-item id << 4) | pixel index within the work-item, the
// order in which the reference's index reduction resolves ties
// (cl-files/Statistics.cl REDUCE_POS: a strict scan of 16 pixels per
// work-item, a tree fold over work-items that keeps the left one on ties, a
// strict fold over work-groups). NaN scores are only flagged: with a NaN in
// the map the reference's answer depends on where it lies, so the caller
// takes the map path then.
struct IdxRecord {
  float v;
  int have;
  unsigned long long key;
  int nan;
  int pad;
};

// Shared-memory layout, identical on host and device.
struct Layout {
  int row_bytes, raw_stage, raw, b, a_stage, a, bars, total;
};

__host__ __device__ inline int align128(int x) { return (x + 127) & ~127; }

// A staged row of nbox 16-byte groups is loaded by box_split(nbox) TMA copies
// of box_part(nbox) groups each: a box dimension holds at most 256, and every
// copy's shared-memory destination must be 128-byte aligned, so a part is a
// multiple of 8 groups.
__host__ __device__ inline int box_split(int nbox) { return (nbox + 255) / 256; }
__host__ __device__ inline int box_part(int nbox) {
  return ((nbox + box_split(nbox) - 1) / box_split(nbox) + 7) & ~7;
}

__host__ __device__ inline Layout make_layout(bool split, const Geo& g, int nbox) {
  Layout L;
  L.row_bytes = box_split(nbox) * box_part(nbox) * 16;
  L.raw_stage = align128(L.row_bytes);
  L.raw = 0;
  L.b = L.raw + kNRaw * L.raw_stage;
  L.a = L.b + align128(2 * g.nmma * g.NB * 16);
  L.a_stage = align128(g.QR * 16 * (split ? 2 : 1));
  L.bars = L.a + g.NA * L.a_stage;
  // raw full, raw free; ready (one per A stage); block full, buffer free; done.
  L.total = L.bars + align128(8 * (2 * kNRaw + kMaxNA + 4 + 1));
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

// 8 staged elements from element e0 as floats (F32, U16).
template <int ELEM, int S>
__device__ __forceinline__ void load8(const unsigned char* row, int e0, float (&f)[8]) {
  if (S == 1) {
    // Any start element: single-element loads.
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      if (ELEM == kF32)
        f[j] = reinterpret_cast<const float*>(row)[e0 + j];
      else
        f[j] = static_cast<float>(reinterpret_cast<const uint16_t*>(row)[e0 + j]);
    }
  } else if (ELEM == kF32) {
    if (S % 4 == 0) {
      const float4* p = reinterpret_cast<const float4*>(row + 4 * e0);
      const float4 u = p[0], v = p[1];
      f[0] = u.x; f[1] = u.y; f[2] = u.z; f[3] = u.w;
      f[4] = v.x; f[5] = v.y; f[6] = v.z; f[7] = v.w;
    } else {
      const float2* p = reinterpret_cast<const float2*>(row + 4 * e0);
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const float2 u = p[j];
        f[2 * j] = u.x;
        f[2 * j + 1] = u.y;
      }
    }
  } else {
    // U16: e0 is even (S = 2, 4 or 8), so 32-bit words hold pixel pairs.
    const uint32_t* p = reinterpret_cast<const uint32_t*>(row + 2 * e0);
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const uint32_t w = p[j];
      f[2 * j] = static_cast<float>(w & 0xFFFFu);
      f[2 * j + 1] = static_cast<float>(w >> 16);
    }
  }
}

// AND of `p` over the builder warps (a named barrier every builder reaches).
__device__ __forceinline__ bool builders_all(bool p) {
  uint32_t r;
  asm volatile(
      "{\n\t.reg .pred pi, po;\n\t"
      "setp.ne.u32 pi, %1, 0;\n\t"
      "barrier.red.and.pred po, %2, %3, pi;\n\t"
      "selp.u32 %0, 1, 0, po;\n\t}"
      : "=r"(r)
      : "r"((uint32_t)p), "n"(kBarBuild), "n"(kBuildThreads)
      : "memory");
  return r != 0;
}

// Running best of one lane (the fused best match): the value, its key and
// flags. A value replaces the best when strictly better, or equal with a
// smaller key; NaN values are only flagged.
struct IdxState {
  float v;
  unsigned long long key;
  int have, nan;
};

__device__ __forceinline__ unsigned long long idx_key_of(int x, int y, int ngx) {
  const unsigned lid = ((unsigned)(y & 15) << 4) | (unsigned)(x & 15);
  const unsigned long long grp = (unsigned long long)(y >> 4) * ngx + (x >> 8);
  return (grp << 12) | ((unsigned long long)(__brev(lid) >> 24) << 4) | (unsigned)((x & 255) >> 4);
}

__device__ __forceinline__ void idx_state_update(IdxState& st, float v, int x, int y, int op,
                                                 int ngx) {
  const float c = op >= 2 ? fabsf(v) : v;
  if (c != c) {
    st.nan = 1;
    return;
  }
  const bool is_min = op == 0 || op == 2;
  if (st.have && (is_min ? c > st.v : c < st.v)) return;
  const unsigned long long k = idx_key_of(x, y, ngx);
  if (st.have && c == st.v && k > st.key) return;
  st.v = c;
  st.key = k;
  st.have = 1;
}

// Runs one work item with all 10 warps of the CTA. The caller has
// synchronised the CTA; TMEM (512 columns) is allocated. Barriers are
// initialised here and invalidated at the end, so consecutive items may use
// different layouts.
template <int ELEM, int S, bool IDX>
__device__ __forceinline__ void run_item(const ItemArgs& a, unsigned char* smem, CtaState& cs) {
  typedef ElemTraits<ELEM> TR;
  constexpr bool SPLIT = TR::split;
  constexpr int R = kSR / S;
  constexpr int Q = 16 / S;
  constexpr int BS = block_steps(S);
  constexpr int CMK = TR::cmk;
  constexpr int NC = S * (BS + R - 1);  // open-slot columns of a block
  constexpr int NCH = (NC + 15) / 16;   // 16-column chunks of a partial
  static_assert(S * BS == 16, "a block's completed slots are one chunk");
  static_assert(NC <= kNp && NCH * 16 == kRingCols, "block does not fit the ring");
  const int lead = (TR::inner - a.ax % TR::inner) % TR::inner;
  const Geo G = make_geo(SPLIT, R, a.tw, lead);
  const Layout L = make_layout(SPLIT, G, a.nbox);

  uint64_t* raw_full = reinterpret_cast<uint64_t*>(smem + L.bars);
  uint64_t* raw_free = raw_full + kNRaw;
  // A of row t written. Stage t mod NA is free again once the MMAs of block
  // t / BS - 2 have completed (its blk_full commit): NA = 2 BS stages.
  uint64_t* ready = raw_free + kNRaw;
  uint64_t* blk_full = ready + kMaxNA;     // block's MMAs complete (2 buffers)
  uint64_t* buf_free = blk_full + 2;       // block's buffer read by the epilogue
  uint64_t* done_bar = buf_free + 2;
  volatile int* abort_flag = &cs.abort;

  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const bool need_e = a.measure != kCrossCorr;
  const int ch = a.ch;
  const int r_begin = a.y0 - a.ay - (R - a.th);
  const int nsteps = (a.yend - a.y0) + R - 1;

  if (threadIdx.x == 0) {
    for (int i = 0; i < kNRaw; ++i) {
      mbar_init(&raw_full[i], 1);
      mbar_init(&raw_free[i], kBuilders);
    }
    for (int i = 0; i < G.NA; ++i) mbar_init(&ready[i], kBuilders);
    for (int i = 0; i < 2; ++i) {
      mbar_init(&blk_full[i], 1);
      mbar_init(&buf_free[i], kEpilogue);
    }
    mbar_init(done_bar, 1);
    fence_barrier_init();
  }

  // Template operand B: per core matrix (two per MMA, in issue order) NB rows
  // of 16 bytes; rows 16 - S .. 16 - S + N - 1 hold B, the rest are zero.
  {
    const int zp = 16 - S;
    const int total = 2 * G.nmma * G.NB * CMK;
    for (int idx = threadIdx.x; idx < total; idx += kThreads) {
      const int e = idx % CMK;
      const int row = (idx / CMK) % G.NB;
      const int cm = idx / (CMK * G.NB);
      // Which part (0 zero, 1 Thi, 2 Tlo; U8: 1) and which K chunk.
      int part, c;
      if (SPLIT) {
        const int j = cm >> 1, half = cm & 1;
        if (j < G.KC) {
          c = j;
          part = half ? 1 : 2;  // (hi_c, lo_c) x (Tlo_c, Thi_c)
        } else {
          c = 2 * (j - G.KC) + half;
          part = c < G.KC ? 1 : 0;
        }
      } else {
        c = cm;
        part = c < G.KC ? 1 : 0;
      }
      const int n = row - zp;
      double t = 0.0;
      if (part && n >= 0 && n < kN) {
        const int j = n / S, p = n - (n / S) * S;
        const int h = a.th - 1 - j;
        const int w = c * CMK + e - p - lead;
        if (h >= 0 && w >= 0 && w < a.tw) t = tmpl_at<ELEM>(a, h, w, ch);
      }
      unsigned char* dst = smem + L.b + (cm * G.NB + row) * 16;
      if (SPLIT) {
        const float tf = static_cast<float>(t);
        const __nv_bfloat16 hi = __float2bfloat16_rn(tf);
        const __nv_bfloat16 lo = __float2bfloat16_rn(tf - __bfloat162float(hi));
        reinterpret_cast<__nv_bfloat16*>(dst)[e] = part == 2 ? lo : hi;
      } else {
        dst[e] = static_cast<uint8_t>(t);
      }
    }
    if (warp == kTmaWarp) {
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

  if (warp == kTmaWarp) {
    // ---- TMA: source rows, one per stage ----------------------------------------
    if (lane == 0) {
      tma_prefetch_desc(a.tmap);
      const int gx = (a.xs_out - a.ax - lead) / TR::inner;  // exact: a multiple of inner
      const int part = box_part(a.nbox), nsplit = box_split(a.nbox);
      int issued = 0;
      for (; issued < nsteps; ++issued) {
        const int st = issued % kNRaw;
        if (issued >= kNRaw &&
            !mbar_wait(&raw_free[st], ((issued / kNRaw) - 1) & 1, abort_flag, kSpinLimit))
          break;
        mbar_arrive_expect_tx(&raw_full[st], L.row_bytes);
        for (int j = 0; j < nsplit; ++j)
          tma_load_4d(smem + L.raw + st * L.raw_stage + j * part * 16, a.tmap, 0, gx + j * part,
                      r_begin + issued, ch, &raw_full[st]);
      }
      // Every load issued has landed before the item ends.
      volatile int no_abort = 0;
      for (int b = max(0, issued - kNRaw); b < issued; ++b)
        mbar_wait(&raw_full[b % kNRaw], (b / kNRaw) & 1, &no_abort, kSpinLimit);
    }
  } else if (warp == kMmaWarp) {
    // ---- MMA issue --------------------------------------------------------------
    if (lane == 0) {
      const uint32_t idesc = SPLIT ? idesc_bf16_f32(kM, kNp) : idesc_u8_s32(kM, kNp);
      const uint32_t a0 = smem_u32(smem + L.a);
      const uint32_t b0 = smem_u32(smem + L.b);
      const uint32_t bstride = G.NB * 16;  // between B core matrices
      const uint32_t dhi = desc_hi(128);     // every descriptor: SBO 128 bytes
      const uint32_t astep = G.lbok >> 4, bstep = (2 * bstride) >> 4;  // 16-byte units
      int i = 0;
      uint32_t ph = 0;
      for (int t = 0; t < nsteps; ++t) {
        const int k = t / BS, q = t - (t / BS) * BS;
        // The buffer of block k was read by the epilogue (block k - 2).
        if (q == 0 && k >= 2 &&
            !mbar_wait(&buf_free[k & 1], ((k >> 1) - 1) & 1, abort_flag, kSpinLimit))
          break;
        if (!mbar_wait(&ready[i], ph, abort_flag, kSpinLimit)) break;
        tc_fence_after();
        const uint32_t d = tmem_base + (k & 1) * kPartCols;  // the block's partial
        const uint32_t ah = a0 + i * L.a_stage;
        const uint32_t bq = b0 + 16 * S * (Q - 1 - q);
        // The block's first MMA overwrites all kNp columns of the partial.
        const uint32_t acc0 = q == 0 ? 0u : 1u;
        // Descriptors advance by one add of their low word per MMA: B by two
        // core matrices, A by one (split, hi/lo pairs) or two K core matrices.
        // The MMAs of a step issue back to back from this one thread, so the
        // work between two of them delays the tensor pipe directly.
        uint32_t bl = desc_lo(bq, bstride);
        if (SPLIT) {
          uint32_t al = desc_lo(ah, G.QR * 16), acc = acc0;
          for (int c = 0; c < G.KC; ++c) {
            mma_bf16_h(d, al, dhi, bl, dhi, idesc, acc);
            acc = 1u;
            al += astep;
            bl += bstep;
          }
          uint32_t al2 = desc_lo(ah, G.lbok);
          for (int j = G.KC; j < G.nmma; ++j) {
            mma_bf16_h(d, al2, dhi, bl, dhi, idesc, 1u);
            al2 += 2 * astep;
            bl += bstep;
          }
        } else {
          uint32_t al = desc_lo(ah, G.lbok), acc = acc0;
          for (int j = 0; j < G.nmma; ++j) {
            mma_i8_h(d, al, dhi, bl, dhi, idesc, acc);
            acc = 1u;
            al += 2 * astep;
            bl += bstep;
          }
        }
        // One commit per block: it frees the block's partial for the epilogue
        // and its A stages for the builders.
        if (q == BS - 1 || t == nsteps - 1) mma_commit(&blk_full[k & 1]);
        if (++i == G.NA) { i = 0; ph ^= 1; }
      }
      // Every MMA issued has completed before the item ends.
      mma_commit(done_bar);
      volatile int no_abort = 0;
      mbar_wait(done_bar, 0, &no_abort, kSpinLimit);
    }
  } else if (warp < kBuilders) {
    // ---- Builders: A operand ------------------------------------------------------
    const int b = threadIdx.x;  // 0 .. 127
    int i = 0, st = 0;
    uint32_t rph = 0;
    for (int t = 0; t < nsteps; ++t) {
      bool ok = mbar_wait(&raw_full[st], rph, abort_flag, kSpinLimit);
      // A stage i was last read by row t - NA, in block kb - 2: wait for that
      // block's commit. (The barrier cannot be a phase further on: block kb
      // needs these rows; and block kb - 4 was waited for two blocks ago.)
      const int kb = t / BS;
      ok = ok && (t < G.NA ||
                  mbar_wait(&blk_full[(kb - 2) & 1], ((kb - 2) >> 1) & 1, abort_flag, kSpinLimit));
      // All builders take the same branch (they meet at named barriers).
      if (!builders_all(ok)) break;
      const unsigned char* row = smem + L.raw + st * L.raw_stage;
      unsigned char* ahi = smem + L.a + i * L.a_stage;
      for (int q = b; q < G.QR; q += kBuildThreads) {
        if (SPLIT) {
          float f[8];
          load8<ELEM, S>(row, S * q, f);
          uint32_t hi[4], lo[4];
#pragma unroll
          for (int j = 0; j < 4; ++j) {
            hi[j] = pack_bf16(f[2 * j], f[2 * j + 1]);
            lo[j] = pack_bf16(f[2 * j] - bf16lo_f(hi[j]), f[2 * j + 1] - bf16hi_f(hi[j]));
          }
          *reinterpret_cast<uint4*>(ahi + q * 16) = make_uint4(hi[0], hi[1], hi[2], hi[3]);
          *reinterpret_cast<uint4*>(ahi + G.QR * 16 + q * 16) =
              make_uint4(lo[0], lo[1], lo[2], lo[3]);
        } else {
          // Bytes S q .. S q + 15 (S q is a multiple of 4 when S is).
          const int off = S * q;
          const uint32_t* w32 = reinterpret_cast<const uint32_t*>(row + (off & ~3));
          const uint32_t sh = (off & 3) * 8;
          uint32_t w[5];
#pragma unroll
          for (int j = 0; j < 5; ++j) w[j] = (S % 4 == 0 && j == 4) ? 0u : w32[j];
          uint32_t v[4];
#pragma unroll
          for (int j = 0; j < 4; ++j)
            v[j] = S % 4 == 0 ? w[j] : __funnelshift_r(w[j], w[j + 1], sh);
          *reinterpret_cast<uint4*>(ahi + q * 16) = make_uint4(v[0], v[1], v[2], v[3]);
        }
      }
      fence_async_smem();
      __syncwarp();
      if (lane == 0) {
        mbar_arrive(&ready[i]);
        mbar_arrive(&raw_free[st]);
      }
      if (++i == G.NA) i = 0;
      if (++st == kNRaw) { st = 0; rph ^= 1; }
    }
  } else {
    // ---- Epilogue ---------------------------------------------------------------
    typedef typename std::conditional<SPLIT, float, int>::type AT;  // running sums
    const int sp = warp - kBuilders;  // TMEM sub-partition (warp % 4)
    const int m = sp * 32 + lane;
    const uint32_t lane_base = tmem_base + (static_cast<uint32_t>(sp * 32) << 16);
    const uint32_t ring = lane_base + kRingCol;
    // The item's fields in registers: the item lives in shared memory, and
    // the score loop would otherwise reload them on every slot.
    const auto ea_W = a.W;
    const auto ea_accum = a.accum;
    const int ea_idx_op = IDX ? a.idx_op : -1;
    const auto ea_dst = a.dst;
    const auto ea_dst_f64 = a.dst_f64;
    const auto ea_dst_pitch = a.dst_pitch;
    const auto ea_measure = a.measure;
    const auto ea_nch = a.nch;
    const auto ea_xs_out = a.xs_out;
    const auto ea_y0 = a.y0;
    const auto ea_yend = a.yend;
    const double etd = cs.et;
    const float ret = (float)(1.0 / sqrt(etd));  // 1 / sqrt(E_T)
    // Score of one position from its product sum cv and window energy ev.
    // Split sources: SqrDistance's terms cancel near a match, so its
    // numerator is formed in FP64; the _Norm scale of an F32 map is taken in
    // FP32 (relative error a few 1e-7), of an F64 map in FP64. U8: exact
    // integers and the plain path's float or double formulas (bit-identical).
    // Best-match state of this lane (ocipProximityIndx).
    IdxState ib;
    ib.v = 0.f;
    ib.key = 0ull;
    ib.have = 0;
    ib.nan = 0;
    const int idx_ngx = (ea_W + 255) >> 8;
    auto idx_update = [&](float v, int x, int y) { idx_state_update(ib, v, x, y, ea_idx_op, idx_ngx); };
    // U8 _Norm: float arithmetic where the plain path's float sums are exact.
    const bool u8_float = (double)a.tw * a.th * 65025.0 <= 16777216.0;
    // Scores with the measure fixed at compile time (MT::value), so that the
    // S positions of a slot are straight-line, independent work.
    auto num_of = [&](auto mt, AT cv, double ev) -> double {
      constexpr int M = decltype(mt)::value;
      const double cc = (double)cv;
      if (M == kCrossCorr || M == kCrossCorrNorm) return cc;
      return ev - 2.0 * cc + etd;
    };
    auto score_f = [&](auto mt, AT cv, double ev) -> float {
      constexpr int M = decltype(mt)::value;
      if (SPLIT) {
        const double num = num_of(mt, cv, ev);
        if (M == kCrossCorr || M == kSqrDistance) return (float)num;
        return (float)num * (rsqrtf((float)ev) * ret);
      } else {
        // Exact in int32: each of C, E_S, E_T <= 64 * 64 * 255^2 < 2^28.
        const int cc = static_cast<int>(cv);
        const int es = static_cast<int>(ev);
        const int ei = static_cast<int>(etd);
        const int num = (M == kCrossCorr || M == kCrossCorrNorm) ? cc : es - 2 * cc + ei;
        if (M == kCrossCorr || M == kSqrDistance) return __int2float_rn(num);
        if (u8_float) return __fdiv_rn((float)num, __fsqrt_rn(__fmul_rn((float)es, (float)ei)));
        return (float)__ddiv_rn((double)num, __dsqrt_rn(__dmul_rn((double)es, (double)ei)));
      }
    };
    auto score_d = [&](auto mt, AT cv, double ev) -> double {
      constexpr int M = decltype(mt)::value;
      if (SPLIT) {
        const double num = num_of(mt, cv, ev);
        if (M == kCrossCorr || M == kSqrDistance) return num;
        return num * rsqrt(ev * etd);
      } else {
        const int cc = static_cast<int>(cv);
        const int es = static_cast<int>(ev);
        const int ei = static_cast<int>(etd);
        const int num = (M == kCrossCorr || M == kCrossCorrNorm) ? cc : es - 2 * cc + ei;
        if (M == kCrossCorr || M == kSqrDistance) return (double)num;
        if (u8_float)
          return (double)__fdiv_rn((float)num, __fsqrt_rn(__fmul_rn((float)es, (float)ei)));
        return __ddiv_rn((double)num, __dsqrt_rn(__dmul_rn((double)es, (double)ei)));
      }
    };
    // Row energies of the rows block kk's slots complete (entering: staged
    // row u; leaving: staged row u - th), S positions of this lane each,
    // loaded before the block's MMAs are waited for. The window energy of
    // each position is an FP64 running sum over the slots, in order.
    typedef typename std::conditional<SPLIT, float, int>::type RT;
    const int xl = ea_xs_out + S * m;
    RT rin[BS][S], rout[BS][S];
    double esum[S];
#pragma unroll
    for (int p = 0; p < S; ++p) esum[p] = 0.0;
#pragma unroll
    for (int g = 0; g < BS; ++g)
#pragma unroll
      for (int p = 0; p < S; ++p) rin[g][p] = rout[g][p] = RT(0);  // CrossCorr: no energies
    auto load_rows = [&](RT (&v)[S], int sr) {
      const bool row_ok = need_e && sr >= 0 && sr < a.H;
      const RT* er = reinterpret_cast<const RT*>(a.energy + (size_t)ch * a.e_plane +
                                                 (size_t)(row_ok ? sr : 0) * a.e_pitch);
      if (row_ok && xl + S <= ea_W) {
        if (S == 2) {
          const uint2 q = *reinterpret_cast<const uint2*>(er + xl);
          memcpy(v, &q, sizeof(q));
        } else {
#pragma unroll
          for (int j = 0; j < S / 4; ++j) {
            const uint4 q = reinterpret_cast<const uint4*>(er + xl)[j];
            memcpy(&v[4 * j], &q, sizeof(q));
          }
        }
      } else {
#pragma unroll
        for (int p = 0; p < S; ++p) v[p] = row_ok && xl + p < ea_W ? er[xl + p] : RT(0);
      }
    };
    auto load_energies = [&](int kk) {
#pragma unroll
      for (int g = 0; g < BS; ++g) {
        const int u = kk * BS + g;
        const bool in = u < nsteps;
        load_rows(rin[g], in ? r_begin + u : -1);
        load_rows(rout[g], in && u >= a.th ? r_begin + u - a.th : -1);
      }
    };
    uint32_t zero[16];
#pragma unroll
    for (int j = 0; j < 16; ++j) zero[j] = 0u;
    for (int c = 0; c < kRingCols; c += 16) tmem_st16(ring + c, zero);
    tmem_st_wait();
    for (int k = 0; k * BS < nsteps; ++k) {
      const int t0 = k * BS;
      if (need_e) load_energies(k);
      bool ok = mbar_wait(&blk_full[k & 1], (k >> 1) & 1, abort_flag, kSpinLimit);
      // tcgen05.ld/st are warp-collective: the whole warp takes one branch.
      if (!__all_sync(0xffffffffu, ok)) break;
      tc_fence_after();
      const uint32_t part = lane_base + (k & 1) * kPartCols;
      // Relative chunk i of the block lives at ring chunk (k + i) mod NCH.
      // Chunks 1 .. NCH - 1 hold open slots: ring += partial.
      for (int c16 = 1; c16 < NCH; ++c16) {
        const uint32_t rc = ring + 16 * ((k + c16) % NCH);
        uint32_t vp[16], vr[16];
        tmem_ld16x(part + 16 * c16, vp);
        tmem_ld16x(rc, vr);
        tmem_ld_wait();
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          if (SPLIT)
            vr[j] = __float_as_uint(__fadd_rn(__uint_as_float(vr[j]), __uint_as_float(vp[j])));
          else
            vr[j] += vp[j];  // exact int32 sums
        }
        tmem_st16(rc, vr);
      }
      // Chunk 0: the BS slots t0 .. t0 + BS - 1 this block completes. Their
      // ring columns are cleared for the slots NS later.
      AT val[16];
      {
        const uint32_t rc = ring + 16 * (k % NCH);
        uint32_t vp[16], vr[16];
        tmem_ld16x(part, vp);
        tmem_ld16x(rc, vr);
        tmem_ld_wait();
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          if (SPLIT)
            val[j] = __fadd_rn(__uint_as_float(vr[j]), __uint_as_float(vp[j]));
          else
            val[j] = static_cast<int>(vr[j] + vp[j]);
        }
        tmem_st16(rc, zero);
      }
      tmem_st_wait();
      // The partial has been read: the MMAs may refill it (block k + 2).
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&buf_free[k & 1]);
      // The block's completed slots: window energies (running sums, in
      // order), scores and stores, specialised per measure.
      auto slots = [&](auto mt) {
#pragma unroll
        for (int g = 0; g < BS; ++g) {
          const int u = t0 + g;
          const int yd = ea_y0 + u - R + 1;
          if (u >= nsteps) break;
          double e[S];
#pragma unroll
          for (int p = 0; p < S; ++p) {
            esum[p] += static_cast<double>(rin[g][p]) - static_cast<double>(rout[g][p]);
            e[p] = esum[p];
          }
          if (u >= R - 1 && yd < ea_yend) {
            char* orow = ea_dst + (size_t)yd * ea_dst_pitch;
            const int x0 = xl;
            if (ea_nch == 1 && !ea_dst_f64 && x0 + S <= ea_W) {
              float outf[S];
#pragma unroll
              for (int p = 0; p < S; ++p) outf[p] = score_f(mt, val[g * S + p], e[p]);
              if (IDX && ea_idx_op >= 0) {
#pragma unroll
                for (int p = 0; p < S; ++p) idx_update(outf[p], x0 + p, yd);
              }
              if (ea_dst != nullptr) {
                float* o = reinterpret_cast<float*>(orow) + x0;
                if (S % 4 == 0) {
#pragma unroll
                  for (int j = 0; j < S / 4; ++j)
                    reinterpret_cast<float4*>(o)[j] = make_float4(
                        outf[(4 * j) % S], outf[(4 * j + 1) % S], outf[(4 * j + 2) % S],
                        outf[(4 * j + 3) % S]);
                } else {
#pragma unroll
                  for (int j = 0; j < S / 2; ++j)
                    reinterpret_cast<float2*>(o)[j] =
                        make_float2(outf[(2 * j) % S], outf[(2 * j + 1) % S]);
                }
              }
            } else {
#pragma unroll
              for (int p = 0; p < S; ++p) {
                const int x = x0 + p;
                if (x >= ea_W) break;
                const size_t xo = (size_t)x * ea_nch + ch;
                if (ea_dst_f64 && ea_accum) {
                  reinterpret_cast<double*>(orow)[xo] += score_d(mt, val[g * S + p], e[p]);
                } else if (ea_dst_f64) {
                  reinterpret_cast<double*>(orow)[xo] = score_d(mt, val[g * S + p], e[p]);
                } else {
                  const float v = score_f(mt, val[g * S + p], e[p]);
                  if (IDX && ea_idx_op >= 0) idx_update(v, x, yd);
                  if (ea_dst != nullptr) reinterpret_cast<float*>(orow)[xo] = v;
                }
              }
            }
          }
        }
      };
      switch (ea_measure) {
        case kSqrDistance: slots(std::integral_constant<int, kSqrDistance>()); break;
        case kSqrDistanceNorm: slots(std::integral_constant<int, kSqrDistanceNorm>()); break;
        case kCrossCorrNorm: slots(std::integral_constant<int, kCrossCorrNorm>()); break;
        default: slots(std::integral_constant<int, kCrossCorr>()); break;
      }
      if (!__all_sync(0xffffffffu, ok)) break;
    }
    if (IDX && ea_idx_op >= 0) {
      // The warp's best: same rule, then lane 0 writes the warp's record.
      const bool is_min = ea_idx_op == 0 || ea_idx_op == 2;
#pragma unroll
      for (int d = 16; d > 0; d >>= 1) {
        const float ov = __shfl_xor_sync(0xffffffffu, ib.v, d);
        const unsigned long long ok2 = __shfl_xor_sync(0xffffffffu, ib.key, d);
        const int oh = __shfl_xor_sync(0xffffffffu, ib.have, d);
        ib.nan |= __shfl_xor_sync(0xffffffffu, ib.nan, d);
        const bool take = oh && (!ib.have || (is_min ? ov < ib.v : ov > ib.v) ||
                                 (ov == ib.v && ok2 < ib.key));
        if (take) {
          ib.v = ov;
          ib.key = ok2;
          ib.have = 1;
        }
      }
      if (lane == 0) {
        const int item = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
        IdxRecord r;
        r.v = ib.v;
        r.have = ib.have;
        r.key = ib.key;
        r.nan = ib.nan;
        r.pad = 0;
        reinterpret_cast<IdxRecord*>(a.idx_out)[item * kEpilogue + sp] = r;
      }
    }
  }

  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (threadIdx.x == 0) {
    for (int i = 0; i < kNRaw; ++i) {
      mbar_inval(&raw_full[i]);
      mbar_inval(&raw_free[i]);
    }
    for (int i = 0; i < G.NA; ++i) mbar_inval(&ready[i]);
    for (int i = 0; i < 2; ++i) {
      mbar_inval(&blk_full[i]);
      mbar_inval(&buf_free[i]);
    }
    mbar_inval(done_bar);
  }
}

// Template classes: R in {16, 32, 64} (template rows rounded up); the strip
// width is 128 S positions.
inline int class_of(int th) { return th <= 16 ? 0 : th <= 32 ? 1 : 2; }
__host__ __device__ inline int class_r(int cls) { return 16 << cls; }
template <int ELEM>
int strip_width(int cls) {
  return kM * s_for(class_r(cls));
}

template <int ELEM, bool IDX>
__device__ __forceinline__ void dispatch(const ItemArgs& a, unsigned char* smem, CtaState& cs) {
  if (a.R == 16)
    run_item<ELEM, 8, IDX>(a, smem, cs);
  else if (a.R == 32)
    run_item<ELEM, 4, IDX>(a, smem, cs);
  else
    run_item<ELEM, 2, IDX>(a, smem, cs);
}

// Batch tables (device memory).
struct BatchImage {
  int W, H, nch;
};
struct BatchTemplate {
  const char* ptr;
  size_t pitch;
  int tw, th, cls;  // cls: template rows class (R = 16 << cls)
};
struct BatchDest {
  char* ptr;
  size_t pitch;
  int f64;
};
struct BatchItem {
  int img, tpl, dst;  // indices into the tables
  int energy;         // index into the energy maps, -1 for CrossCorr
  int ch, strip, y0, yend;
};
// Window-energy map of one (image, template size) pair of a batch.
struct BatchEnergy {
  const char* ptr;
  size_t pitch, plane;
};

struct TensorLaunch {
  CUtensorMap map;     // single-image mode: the source planes
  int mode;            // 0: one (image, template) pair, items from blockIdx; 1: work queue
  int measure;
  int nbox;            // 16-byte groups per staged row (all tensor maps of the launch)
  int* err;
  // mode 0
  ItemArgs base;       // fields common to every item
  int BH;
  // mode 1
  const CUtensorMap* maps;  // one per image (64-byte aligned)
  const BatchImage* imgs;
  const BatchTemplate* tpls;
  const BatchDest* dsts;
  const BatchItem* items;
  const BatchEnergy* energies;
  int nitems;
  int* counter;        // next item; reset to 0 before every launch
};

// One kernel per element type. Mode 0 (one image and template): CTA
// (x, y, z) = (strip, band, channel). Mode 1 (batch): one persistent CTA per
// SM takes items from a global counter until none are left.
template <int ELEM, bool IDX = false>
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
  if (P.mode == 0) {
    if (threadIdx.x == 0) {
      item = P.base;
      item.tmap = &P.map;
      item.ch = blockIdx.z;
      item.xs_out = blockIdx.x * kM * s_for(item.R);
      item.y0 = blockIdx.y * P.BH;
      item.yend = min(item.H, item.y0 + P.BH);
    }
    __syncthreads();
    dispatch<ELEM, IDX>(item, smem, cs);
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
          item.R = class_r(tp.cls);
          item.ax = tp.tw / 2;
          item.ay = tp.th / 2;
          item.nch = im.nch;
          item.ch = bi.ch;
          item.xs_out = bi.strip * kM * s_for(item.R);
          item.y0 = bi.y0;
          item.yend = bi.yend;
          item.nbox = P.nbox;
          item.tmpl = tp.ptr;
          item.tmpl_pitch = tp.pitch;
          item.dst = ds.ptr;
          item.dst_pitch = ds.pitch;
          item.dst_f64 = ds.f64;
          item.measure = P.measure;
          item.accum = 0;
          item.idx_op = -1;
          item.idx_out = nullptr;
          item.energy = nullptr;
          item.e_pitch = item.e_plane = 0;
          if (bi.energy >= 0) {
            const BatchEnergy be = P.energies[bi.energy];
            item.energy = be.ptr;
            item.e_pitch = be.pitch;
            item.e_plane = be.plane;
          }
        }
      }
      __syncthreads();
      const int it = cs.next;
      if (it >= P.nitems) break;
      dispatch<ELEM, IDX>(item, smem, cs);
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

// Lead of the staged row (elements before the first window pixel, so that
// the TMA copy starts on a 16-byte group).
template <int ELEM>
int lead_for(int ax) {
  const int inner = ElemTraits<ELEM>::inner;
  return (inner - ax % inner) % inner;
}

template <int ELEM>
Geo geo_for(int cls, int tw, int ax) {
  return make_geo(ElemTraits<ELEM>::split, class_r(cls), tw, lead_for<ELEM>(ax));
}

// 16-byte groups a staged row needs for a template of this class and width.
template <int ELEM>
int nbox_for(int cls, int tw, int ax) {
  typedef ElemTraits<ELEM> TR;
  const Geo g = geo_for<ELEM>(cls, tw, ax);
  return (staged_elems(g, TR::split) + TR::inner - 1) / TR::inner;
}

template <int ELEM>
int smem_for(int cls, int tw, int ax, int nbox) {
  return std::max(make_layout(ElemTraits<ELEM>::split, geo_for<ELEM>(cls, tw, ax), nbox).total,
                  kMinSmem);
}

// Rank-4 view of source planes: 16-byte groups (dim 0), groups along the row
// (dim 1), rows (dim 2), channels (dim 3). A staged row (the strip plus the
// template width, nbox groups) is box_split(nbox) boxes of box_part(nbox)
// groups and one row. The last group of a row may reach into the row pitch,
// which is zero (image creation zero-fills device buffers; the channel split
// writes zeros there).
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
  const cuuint32_t box[4] = {(cuuint32_t)TR::inner, (cuuint32_t)box_part(nbox), 1, 1};
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
cudaError_t launch_one(Context& ctx, Measure m, const DevImage& src, const DevImage& tmpl,
                       const DevImage& dst, int ax, int ay, bool accum = false,
                       int idx_op = -1, void* idx_out = nullptr, int* nrec = nullptr) {
  const int cls = class_of(tmpl.height);
  const int R = class_r(cls);
  TensorLaunch P;
  std::memset(&P, 0, sizeof(P));
  P.mode = 0;
  P.measure = m;
  P.nbox = nbox_for<ELEM>(cls, tmpl.width, ax);
  P.err = reinterpret_cast<int*>(ctx.scratch(Context::kTensorAux, 256));
  const int sw = strip_width<ELEM>(cls);
  const int nstrips = (src.width + sw - 1) / sw;
  P.BH = ctx.band_rows > 0
             ? std::min(ctx.band_rows, src.height)
             : band_height(src.height, R, (long long)nstrips * src.nch, ctx.sm_count);
  ItemArgs& a = P.base;
  a.W = src.width;
  a.H = src.height;
  a.tw = tmpl.width;
  a.th = tmpl.height;
  a.R = R;
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
  a.accum = accum ? 1 : 0;
  a.idx_op = idx_op;
  a.idx_out = reinterpret_cast<char*>(idx_out);

  const int smem_bytes = smem_for<ELEM>(cls, tmpl.width, ax, P.nbox);
  if (smem_bytes > kMaxDynSmem) return cudaErrorInvalidValue;

  // Row energies of every source row, for the measures that use them.
  if (m != kCrossCorr) {
    const size_t ep = row_energy_pitch(src.width);
    const size_t eplane = ep * src.height;
    char* emap = reinterpret_cast<char*>(ctx.scratch(Context::kEnergyMap, eplane * src.nch));
    cudaError_t ee = launch_row_energy(src, tmpl.width, ax, emap, ep, eplane, ctx.stream);
    if (ee != cudaSuccess) return ee;
    a.energy = emap;
    a.e_pitch = ep;
    a.e_plane = eplane;
  }

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

  auto kern = idx_op >= 0 ? prox_tensor_kernel<ELEM, true> : prox_tensor_kernel<ELEM, false>;
  e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           kMaxDynSmem);
  if (e != cudaSuccess) return e;
  dim3 grid(nstrips, (src.height + P.BH - 1) / P.BH, src.nch);
  if (nrec) *nrec = (int)(grid.x * grid.y * grid.z) * kEpilogue;
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
  // Row-energy maps, one per (image, template width) of the batch (measures
  // other than CrossCorr), recomputed by every run.
  struct EnergyJob {
    int img, tw;
    size_t offset, pitch, plane;
  };
  std::vector<EnergyJob> ejobs;
  char* emaps = nullptr;
};

namespace {

// Channel splits, window energies, queue reset, persistent launch. `count`
// is false while the work is recorded into a graph (counted when the graph
// is launched).
template <int ELEM>
cudaError_t batch_record(TensorBatch& b, cudaStream_t stream, bool count) {
  for (size_t i = 0; i < b.images.size(); ++i) {
    if (b.plane_offsets[i].first)
      split_channels<ELEM>(b.images[i], b.planes + b.plane_offsets[i].second, stream, count);
  }
  for (const TensorBatch::EnergyJob& j : b.ejobs) {
    const unsigned long long before = g_launches;
    cudaError_t ee = launch_row_energy(b.images[j.img], j.tw, j.tw / 2, b.emaps + j.offset,
                                       j.pitch, j.plane, stream);
    if (ee != cudaSuccess) return ee;
    if (!count) g_launches = before;
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
                                  const std::vector<int>& pair_energy,
                                  const std::map<int, int>& bh) {
  std::vector<std::pair<long long, BatchItem>> v;
  for (size_t p = 0; p < pair_img.size(); ++p) {
    const DevImage& s = imgs[pair_img[p]];
    const DevImage& t = tpls[pair_tpl[p]];
    const int cls = class_of(t.height);
    const int R = class_r(cls);
    const Geo g = geo_for<ELEM>(cls, t.width, t.width / 2);
    const int BH = bh.at(cls);
    const int sw = strip_width<ELEM>(cls);
    const int nstrips = (s.width + sw - 1) / sw;
    for (int c = 0; c < s.nch; ++c)
      for (int st = 0; st < nstrips; ++st)
        for (int y0 = 0; y0 < s.height; y0 += BH) {
          BatchItem it;
          it.img = pair_img[p];
          it.tpl = pair_tpl[p];
          it.dst = pair_dst[p];
          it.energy = pair_energy[p];
          it.ch = c;
          it.strip = st;
          it.y0 = y0;
          it.yend = std::min(s.height, y0 + BH);
          // steps x MMA work per step (MMAs of Np columns, plus a fixed part)
          const long long cost = (long long)(it.yend - y0 + R - 1) * (g.nmma * kNp + 512);
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
                          const std::vector<BatchItem>& items,
                          const std::vector<BatchEnergy>& benergy, void** mem) {
  auto al = [](size_t x) { return (x + 255) / 256 * 256; };
  const size_t o_maps = 0;
  const size_t o_imgs = al(o_maps + maps.size() * sizeof(CUtensorMap));
  const size_t o_tpls = al(o_imgs + bimgs.size() * sizeof(BatchImage));
  const size_t o_dsts = al(o_tpls + btpls.size() * sizeof(BatchTemplate));
  const size_t o_items = al(o_dsts + bdsts.size() * sizeof(BatchDest));
  const size_t o_en = al(o_items + items.size() * sizeof(BatchItem));
  const size_t o_ctr = al(o_en + benergy.size() * sizeof(BatchEnergy));
  const size_t total = o_ctr + 256;
  std::vector<char> host(total, 0);
  std::memcpy(host.data() + o_maps, maps.data(), maps.size() * sizeof(CUtensorMap));
  std::memcpy(host.data() + o_imgs, bimgs.data(), bimgs.size() * sizeof(BatchImage));
  std::memcpy(host.data() + o_tpls, btpls.data(), btpls.size() * sizeof(BatchTemplate));
  std::memcpy(host.data() + o_dsts, bdsts.data(), bdsts.size() * sizeof(BatchDest));
  std::memcpy(host.data() + o_items, items.data(), items.size() * sizeof(BatchItem));
  if (!benergy.empty())
    std::memcpy(host.data() + o_en, benergy.data(), benergy.size() * sizeof(BatchEnergy));
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
  P.energies = reinterpret_cast<const BatchEnergy*>(d + o_en);
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
                const DevImage& tpl, int cls, int nbox, int smem, char* probe_dst,
                size_t probe_pitch) {
  const int R = class_r(cls);
  std::vector<int> cand;
  for (int bh : {64, 128, 192, 256, 384, 512, 768, 1024})
    if (bh >= R && bh < img.height) cand.push_back(bh);
  cand.push_back(img.height);
  const int sw = strip_width<ELEM>(cls);
  const int nstrips = (img.width + sw - 1) / sw;
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
  // The probe pair's row energies, computed once for every candidate.
  std::vector<BatchEnergy> benergy;
  char* probe_e = nullptr;
  if (measure != kCrossCorr) {
    const size_t ep = row_energy_pitch(img.width), eplane = ep * img.height;
    if (cudaMalloc(&probe_e, eplane * img.nch) != cudaSuccess) return cand.back();
    if (launch_row_energy(img, tpl.width, tpl.width / 2, probe_e, ep, eplane, ctx.stream) !=
        cudaSuccess) {
      cudaFree(probe_e);
      return cand.back();
    }
    benergy.push_back(BatchEnergy{probe_e, ep, eplane});
  }
  float best = 1e30f;
  int best_bh = cand.back();
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  for (int bh : cand) {
    std::vector<int> pi(reps, 0), pt(reps, 0), pd(reps, 0), pe(reps, probe_e ? 0 : -1);
    std::map<int, int> m1{{cls, bh}};
    std::vector<BatchItem> items = make_items<ELEM>({img}, {tpl}, pi, pt, pd, pe, m1);
    TensorBatch tb;
    tb.ctx = &ctx;
    std::memset(&tb.launch, 0, sizeof(tb.launch));
    tb.launch.mode = 1;
    tb.launch.measure = measure;
    tb.launch.nbox = nbox;
    tb.launch.err = reinterpret_cast<int*>(ctx.scratch(Context::kTensorAux, 256));
    tb.smem = smem;
    void* mem = nullptr;
    if (upload_tables<ELEM>(tb, maps, bimgs, btpls, bdsts, items, benergy, &mem) != cudaSuccess)
      break;
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
  if (probe_e) {
    cudaStreamSynchronize(ctx.stream);
    cudaFree(probe_e);
  }
  return best_bh;
}

template <int ELEM>
TensorBatch* batch_create(Context& ctx, Measure m, const std::vector<DevImage>& imgs,
                          const std::vector<DevImage>& tpls, const std::vector<DevImage>& dsts,
                          cudaError_t* err) {
  TensorBatch* b = new TensorBatch();
  b->ctx = &ctx;
  b->elem = ELEM;
  b->measure = m;
  // One staged-row width for every tensor map of the batch: the widest need.
  b->nbox = 1;
  for (const DevImage& t : tpls)
    b->nbox = std::max(b->nbox, nbox_for<ELEM>(class_of(t.height), t.width, t.width / 2));
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
                                  class_of(t.height)});
  std::vector<BatchDest> bdsts;
  for (const DevImage& d : dsts) bdsts.push_back(BatchDest{(char*)d.ptr, d.pitch, d.type == F64});

  auto kern = prox_tensor_kernel<ELEM>;
  e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
  if (e != cudaSuccess) return fail(e);
  // Shared memory: the largest need of any template (per class, the widest).
  std::map<int, int> cls_smem;
  for (const DevImage& t : tpls) {
    const int c = class_of(t.height);
    const int sm = smem_for<ELEM>(c, t.width, t.width / 2, b->nbox);
    if (sm > kMaxDynSmem) return fail(cudaErrorInvalidValue);
    cls_smem[c] = std::max(cls_smem[c], sm);
  }

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
    const int v = autotune_bh<ELEM>(ctx, m, probe, maps[0], tpls[j], cls, b->nbox,
                                    cls_smem[cls], pd, pp);
    cudaStreamSynchronize(ctx.stream);
    cudaFree(pd);
    e = cudaGetLastError();
    if (e != cudaSuccess) return fail(e);
    bh[cls] = v;
    std::lock_guard<std::mutex> lk(g_tune_mutex);
    g_tuned_bh[key] = v;
  }
  b->bh = bh;

  // Row-energy maps: one per (image, template width) for the measures that
  // use them, laid out back to back in one allocation owned by the batch.
  std::map<std::pair<int, int>, int> eidx;
  std::vector<BatchEnergy> benergy;
  if (m != kCrossCorr) {
    size_t total = 0;
    for (size_t i = 0; i < imgs.size(); ++i)
      for (const DevImage& t : tpls) {
        const auto key = std::make_pair((int)i, t.width);
        if (eidx.count(key)) continue;
        eidx[key] = (int)b->ejobs.size();
        const size_t ep = row_energy_pitch(imgs[i].width);
        const size_t eplane = ep * imgs[i].height;
        b->ejobs.push_back(TensorBatch::EnergyJob{(int)i, t.width, total, ep, eplane});
        total += eplane * imgs[i].nch;
      }
    e = cudaMalloc(&b->emaps, total);
    if (e != cudaSuccess) return fail(e);
    for (const TensorBatch::EnergyJob& j : b->ejobs)
      benergy.push_back(BatchEnergy{b->emaps + j.offset, j.pitch, j.plane});
  }
  std::vector<int> pi, pt, pd, pe;
  for (size_t i = 0; i < imgs.size(); ++i)
    for (size_t j = 0; j < tpls.size(); ++j) {
      pi.push_back((int)i);
      pt.push_back((int)j);
      pd.push_back((int)(i * tpls.size() + j));
      pe.push_back(m != kCrossCorr ? eidx[std::make_pair((int)i, tpls[j].width)] : -1);
    }
  std::vector<BatchItem> items = make_items<ELEM>(imgs, tpls, pi, pt, pd, pe, bh);
  b->launch.mode = 1;
  b->launch.measure = m;
  b->launch.nbox = b->nbox;
  b->launch.err = reinterpret_cast<int*>(ctx.scratch(Context::kTensorAux, 256));
  e = upload_tables<ELEM>(*b, maps, bimgs, btpls, bdsts, items, benergy, &b->tables);
  if (e != cudaSuccess) return fail(e);
  b->nitems = b->launch.nitems;
  b->smem = 0;
  for (const auto& kv : cls_smem) b->smem = std::max(b->smem, kv.second);

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
  // Templates beyond 64 x 64 run as tiles of at most 64 x 64 (tensor_large.cu);
  // the row energies take templates up to 1024 columns.
  if (tmpl.width > 1024) return false;
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
  if (tmpl.width > 64 || tmpl.height > 64) return launch_proximity_tensor_large(ctx, m, src, tmpl, dst);
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

size_t tensor_index_records_bytes(const Context& ctx, const DevImage& src, const DevImage& tmpl) {
  (void)ctx;
  const int cls = class_of(tmpl.height);
  const int sw = kM * s_for(class_r(cls));
  const size_t nstrips = (src.width + sw - 1) / sw;
  // At most one band per row (a fixed band height of 1).
  const size_t nbands = src.height;
  return nstrips * nbands * src.nch * kEpilogue * sizeof(IdxRecord);
}

cudaError_t launch_proximity_tensor_indexed(Context& ctx, Measure m, const DevImage& src,
                                            const DevImage& tmpl, const DevImage& dst, int idx_op,
                                            void* records, int* nrec, float* best, int* bx,
                                            int* by, bool* has_nan) {
  cudaError_t e;
  const int ax = tmpl.width / 2, ay = tmpl.height / 2;
  if (src.type == U8)
    e = launch_one<kU8>(ctx, m, src, tmpl, dst, ax, ay, false, idx_op, records, nrec);
  else if (src.type == U16)
    e = launch_one<kU16>(ctx, m, src, tmpl, dst, ax, ay, false, idx_op, records, nrec);
  else
    e = launch_one<kF32>(ctx, m, src, tmpl, dst, ax, ay, false, idx_op, records, nrec);
  if (e != cudaSuccess) return e;
  std::vector<IdxRecord> recs(*nrec);
  e = cudaMemcpyAsync(recs.data(), records, recs.size() * sizeof(IdxRecord),
                      cudaMemcpyDeviceToHost, ctx.stream);
  if (e != cudaSuccess) return e;
  e = cudaStreamSynchronize(ctx.stream);
  if (e != cudaSuccess) return e;
  const bool is_min = idx_op == 0 || idx_op == 2;
  bool have = false, nan = false;
  float v = 0.f;
  unsigned long long key = 0;
  for (const IdxRecord& r : recs) {
    nan = nan || r.nan;
    if (!r.have) continue;
    if (!have || (is_min ? r.v < v : r.v > v) || (r.v == v && r.key < key)) {
      v = r.v;
      key = r.key;
      have = true;
    }
  }
  *has_nan = nan;
  *best = v;
  // Key -> pixel: group, bit-reversed work-item id, pixel index in the work-item.
  const unsigned long long grp = key >> 12;
  const unsigned rl = (unsigned)((key >> 4) & 255);  // bit-reversed work-item id
  unsigned lid = 0;
  for (int b = 0; b < 8; ++b) lid |= ((rl >> b) & 1u) << (7 - b);
  const int i = (int)(key & 15);
  const int ngx = (src.width + 255) >> 8;
  *bx = (int)(grp % ngx) * 256 + (int)(lid & 15) + 16 * i;
  *by = (int)(grp / ngx) * 16 + (int)(lid >> 4);
  return have ? cudaSuccess : cudaErrorInvalidValue;
}

cudaError_t launch_tensor_product_sums(Context& ctx, const DevImage& src, const DevImage& tmpl,
                                       const DevImage& c_map, int ax, int ay, bool accumulate) {
  if (c_map.type != F64) return cudaErrorInvalidValue;
  if (src.type == U8) return launch_one<kU8>(ctx, kCrossCorr, src, tmpl, c_map, ax, ay, accumulate);
  if (src.type == U16)
    return launch_one<kU16>(ctx, kCrossCorr, src, tmpl, c_map, ax, ay, accumulate);
  return launch_one<kF32>(ctx, kCrossCorr, src, tmpl, c_map, ax, ay, accumulate);
}

TensorBatch* tensor_batch_create(Context& ctx, Measure m, const std::vector<DevImage>& imgs,
                                 const std::vector<DevImage>& tpls,
                                 const std::vector<DevImage>& dsts, cudaError_t* err) {
  if (imgs[0].type == U8) return batch_create<kU8>(ctx, m, imgs, tpls, dsts, err);
  if (imgs[0].type == U16) return batch_create<kU16>(ctx, m, imgs, tpls, dsts, err);
  return batch_create<kF32>(ctx, m, imgs, tpls, dsts, err);
}

cudaError_t tensor_batch_run(TensorBatch* b) {
  count_launches(1 + (int)b->ejobs.size() +
                 std::count_if(b->plane_offsets.begin(), b->plane_offsets.end(),
                               [](const std::pair<int, size_t>& p) { return p.first != 0; }));
  return cudaGraphLaunch(b->exec, b->ctx->stream);
}

int tensor_batch_items(const TensorBatch* b) { return b->nitems; }

int tensor_batch_band_height(const TensorBatch* b, int tw, int th) {
  (void)tw;
  auto it = b->bh.find(class_of(th));
  return it == b->bh.end() ? 0 : it->second;
}

void tensor_batch_destroy(TensorBatch* b) {
  if (!b) return;
  if (b->ctx) cudaStreamSynchronize(b->ctx->stream);
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  if (b->tables) cudaFree(b->tables);
  if (b->planes) cudaFree(b->planes);
  if (b->emaps) cudaFree(b->emaps);
  delete b;
}

}  // namespace ocipb
