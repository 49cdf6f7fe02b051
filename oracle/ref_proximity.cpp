/* Driver that runs the reference's ImageProximity kernels on the host.
 *
 * TEST INFRASTRUCTURE ONLY (oracle). Built by oracle/Makefile from the
 * reference's unmodified cl-files/ImageProximity.cl, once per pixel type and
 * channel count (-D <TYPE> [-D NBCHAN=n], as the reference's program builder
 * does in C++/programs/Program.cpp:176-192). The output goes to oracle/_ref/.
 *
 * Dispatch mirrors C++/programs/ImageProximity.cpp:46-57: the _Cached kernel
 * (16x16 work-groups, global range rounded up to 16, C++/programs/WorkGroup.h
 * :114-156) when the template is at most 16x16, the plain kernel (global range
 * exactly W x H, C++/Image.cpp:41-44) otherwise. Work-item rows (plain) or
 * work-groups (cached) are spread over host threads with OpenMP, which is how
 * a CPU OpenCL runtime maps work-groups onto cores.
 */
#include "ref_shim.h"

#ifndef REF_VARIANT
#error "REF_VARIANT must name the pixel type and channel count, e.g. U8_C1"
#endif
#define REF_CAT2(a, b) a##b
#define REF_CAT(a, b) REF_CAT2(a, b)

namespace REF_CAT(refk_, REF_VARIANT) {
#include "ImageProximity.cl"

typedef void (*kfn)(INPUT, INPUT, OUTPUT, int, int, int, int, int, int, int);

static kfn pick(int measure, bool cached) {
  switch (measure) {
    case 0: return cached ? SqrDistance_Cached : SqrDistance;
    case 1: return cached ? SqrDistance_Norm_Cached : SqrDistance_Norm;
    case 2: return cached ? AbsDistance_Cached : AbsDistance;
    case 3: return cached ? CrossCorr_Cached : CrossCorr;
    case 4: return cached ? CrossCorr_Norm_Cached : CrossCorr_Norm;
    default: return nullptr;
  }
}

static int run(int measure, const void* src, int src_step, const void* tmpl,
               int tmpl_step, void* dst, int dst_step, int W, int H, int tw,
               int th, int mode, int row_begin, int row_end) {
  const bool cached = (mode == 2) || (mode == 0 && tw <= 16 && th <= 16);
  if (cached && (tw > 16 || th > 16)) return -30;
  kfn f = pick(measure, cached);
  if (!f) return -30;
  INPUT s = (INPUT)src;
  INPUT t = (INPUT)tmpl;
  OUTPUT d = (OUTPUT)dst;
  if (row_end > H) row_end = H;
  if (!cached) {
#pragma omp parallel for schedule(dynamic, 4)
    for (int gy = row_begin; gy < row_end; ++gy) {
      oclshim::g_lsize[0] = oclshim::g_lsize[1] = 1;
      for (int gx = 0; gx < W; ++gx) {
        oclshim::g_gid[0] = gx;
        oclshim::g_gid[1] = gy;
        oclshim::g_lid[0] = oclshim::g_lid[1] = 0;
        f(s, t, d, src_step, tmpl_step, dst_step, tw, th, W, H);
      }
    }
    return 0;
  }
  const int gw = (W + 15) / 16;
  const int gb = row_begin / 16, ge = (row_end + 15) / 16;
#pragma omp parallel for schedule(dynamic, 1) collapse(2)
  for (int gyg = gb; gyg < ge; ++gyg) {
    for (int gxg = 0; gxg < gw; ++gxg) {
      oclshim::g_lsize[0] = oclshim::g_lsize[1] = 16;
      oclshim::g_grp[0] = gxg;
      oclshim::g_grp[1] = gyg;
      /* Pass 0 runs every work-item of the group up to the barrier: with a
       * destination width of 0 each one stores its template element into the
       * local cache and returns at the kernel's range check, writing nothing.
       * Pass 1 runs the kernels for real with the cache complete. */
      for (int pass = 0; pass < 2; ++pass) {
        for (int ly = 0; ly < 16; ++ly) {
          for (int lx = 0; lx < 16; ++lx) {
            const int gy = gyg * 16 + ly;
            oclshim::g_gid[0] = gxg * 16 + lx;
            oclshim::g_gid[1] = gy;
            oclshim::g_lid[0] = lx;
            oclshim::g_lid[1] = ly;
            if (pass == 0) {
              f(s, t, d, src_step, tmpl_step, dst_step, tw, th, 0, H);
              continue;
            }
            if (gy < row_begin || gy >= row_end) continue;
            f(s, t, d, src_step, tmpl_step, dst_step, tw, th, W, H);
          }
        }
      }
    }
  }
  return 0;
}
}  // namespace

/* measure: 0 SqrDistance, 1 SqrDistance_Norm, 2 AbsDistance, 3 CrossCorr,
 * 4 CrossCorr_Norm. mode: 0 = the reference host's own choice, 1 = plain
 * kernel, 2 = _Cached kernel. Rows [row_begin, row_end) of Dest are written
 * (a band, so a bounded sample of a large image can be timed). Steps are in
 * bytes, as in SImage. Returns 0 or a negative OpenCL-style error code. */
extern "C" int REF_CAT(ocl_ref_proximity_, REF_VARIANT)(
    int measure, const void* src, int src_step, const void* tmpl, int tmpl_step,
    void* dst, int dst_step, int W, int H, int tw, int th, int mode,
    int row_begin, int row_end) {
  return REF_CAT(refk_, REF_VARIANT)::run(measure, src, src_step, tmpl, tmpl_step,
                                         dst, dst_step, W, H, tw, th, mode,
                                         row_begin, row_end);
}
