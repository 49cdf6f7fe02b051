/* Driver that runs the reference's Integral kernels on the host.
 *
 * TEST INFRASTRUCTURE ONLY (oracle). Built by oracle/Makefile from the
 * reference's unmodified cl-files/Integral.cl, once per source pixel type
 * (1 channel, as include/OpenCLIPP.h:641-645 states). The launch sequence
 * restates C++/programs/Integral.cpp:143-241:
 *   scan1 (or sqr) with 8x8 work-groups of 8 pixels each (64x8 tiles,
 *   Integral.cpp:28-30 + WorkGroup.h:114-156), then scan2 over
 *   (groupsW-1) x H, scan3 over W x H, scan4 over W x (groupsH-1) and scan5
 *   over W x H, with the junction buffers of Integral.cpp:42-95.
 * scan1/sqr contain two barriers; every work-group is run three times in a
 * row (one pass per barrier phase, then the real one), which reproduces the
 * barrier semantics because each phase's local-memory writes depend only on
 * the source and on the previous phase's local memory.
 * The tile kernels read the source without x/y bounds checks
 * (Integral.cl:57,120,270,333); the driver copies the source into a buffer
 * padded to whole tiles so those reads stay inside memory it owns.
 */
#include <cstdlib>
#include <cstring>
#include <vector>

#include "ref_shim.h"

#ifndef REF_VARIANT
#error "REF_VARIANT must name the source pixel type in lower case, e.g. u8"
#endif
#define REF_CAT2(a, b) a##b
#define REF_CAT(a, b) REF_CAT2(a, b)

namespace REF_CAT(refi_, REF_VARIANT) {
#include "Integral.cl"

template <class DT, class Tile, class S2, class S3, class S4, class S5>
static int pipeline(Tile tile, S2 scan2, S3 scan3, S4 scan4, S5 scan5,
                    const void* src, int src_step, void* dst, int dst_step,
                    int W, int H) {
  const int gpw = 64, gph = 8;
  const int groupsW = (W + gpw - 1) / gpw, groupsH = (H + gph - 1) / gph;
  /* Padded copy of the source (whole tiles). */
  const int pstep = ((groupsW * gpw * (int)sizeof(TYPE) > src_step)
                         ? groupsW * gpw * (int)sizeof(TYPE)
                         : src_step);
  std::vector<char> psrc((size_t)pstep * groupsH * gph + 64, 0);
  for (int y = 0; y < H; ++y)
    std::memcpy(&psrc[(size_t)y * pstep], (const char*)src + (size_t)y * src_step,
                (size_t)W * sizeof(TYPE));
  DT* d = (DT*)dst;
  /* Tile pass. */
#pragma omp parallel for schedule(dynamic, 1) collapse(2)
  for (int gy = 0; gy < groupsH; ++gy) {
    for (int gx = 0; gx < groupsW; ++gx) {
      oclshim::g_lsize[0] = oclshim::g_lsize[1] = 8;
      oclshim::g_grp[0] = gx;
      oclshim::g_grp[1] = gy;
      for (int pass = 0; pass < 3; ++pass)
        for (int ly = 0; ly < 8; ++ly)
          for (int lx = 0; lx < 8; ++lx) {
            oclshim::g_gid[0] = gx * 8 + lx;
            oclshim::g_gid[1] = gy * 8 + ly;
            oclshim::g_lid[0] = lx;
            oclshim::g_lid[1] = ly;
            tile((const TYPE*)psrc.data(), d, pstep, dst_step, W, H);
          }
    }
  }
  const int vw = groupsW - 1 > 0 ? groupsW - 1 : 1;
  const int hh = groupsH - 1 > 0 ? groupsH - 1 : 1;
  std::vector<DT> vert((size_t)vw * H), horiz((size_t)W * hh);
  const int vstep = vw * (int)sizeof(DT), hstep = W * (int)sizeof(DT);
  oclshim::g_lsize[0] = oclshim::g_lsize[1] = 1;
  if (groupsW > 1)
    for (int y = 0; y < H; ++y)
      for (int x = 0; x < groupsW - 1; ++x) {
        oclshim::g_gid[0] = x;
        oclshim::g_gid[1] = y;
        scan2(d, vert.data(), dst_step, vstep);
      }
  for (int y = 0; y < H; ++y)
    for (int x = 0; x < W; ++x) {
      oclshim::g_gid[0] = x;
      oclshim::g_gid[1] = y;
      scan3(d, vert.data(), d, dst_step, vstep, dst_step);
    }
  if (groupsH > 1)
    for (int y = 0; y < groupsH - 1; ++y)
      for (int x = 0; x < W; ++x) {
        oclshim::g_gid[0] = x;
        oclshim::g_gid[1] = y;
        scan4(d, horiz.data(), dst_step, hstep);
      }
  for (int y = 0; y < H; ++y)
    for (int x = 0; x < W; ++x) {
      oclshim::g_gid[0] = x;
      oclshim::g_gid[1] = y;
      scan5(d, horiz.data(), d, dst_step, hstep, dst_step);
    }
  return 0;
}
}  // namespace

/* sqr: 0 = Integral, 1 = SqrIntegral. dst_f64: Dest type F64 (1) or F32 (0),
 * as Integral.cpp:97-141 dispatches on the destination type. */
extern "C" int REF_CAT(ocl_ref_integral_, REF_VARIANT)(int sqr, const void* src,
                                                       int src_step, void* dst,
                                                       int dst_step, int dst_f64,
                                                       int W, int H) {
  using namespace REF_CAT(refi_, REF_VARIANT);
  if (W <= 0 || H <= 0) return -30;
  if (dst_f64) {
    if (sqr)
      return pipeline<double>(sqr_F64, scan2_F64, scan3_F64, scan4_F64, scan5_F64,
                              src, src_step, dst, dst_step, W, H);
    return pipeline<double>(scan1_F64, scan2_F64, scan3_F64, scan4_F64, scan5_F64,
                            src, src_step, dst, dst_step, W, H);
  }
  /* An F64 source with an F32 destination is not reproduced: the F64
   * program's "_F32" kernels write doubles (REAL) into the F32 image. */
  if constexpr (sizeof(REAL) != sizeof(float)) {
    return -30;
  } else {
    if (sqr)
      return pipeline<float>(sqr_F32, scan2_F32, scan3_F32, scan4_F32, scan5_F32,
                             src, src_step, dst, dst_step, W, H);
    return pipeline<float>(scan1_F32, scan2_F32, scan3_F32, scan4_F32, scan5_F32,
                           src, src_step, dst, dst_step, W, H);
  }
}
