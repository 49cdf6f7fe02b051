// ocip* processing entry points: ImageProximity and Integral.
//
// Argument checks keep the reference's order and codes:
//   ImageProximity (C++/programs/ImageProximity.cpp:34-163): template larger
//   than source -> CL_INVALID_VALUE; SameType(S, T) (Program.cpp:440-446)
//   -> CL_INVALID_VALUE; CheckSameSize(S, D) -> CL_INVALID_IMAGE_SIZE;
//   CheckSameNbChannels(S, D) -> CL_INVALID_VALUE; CheckFloat(D) ->
//   CL_INVALID_VALUE.
//   Integral (C++/programs/Integral.cpp:97-141, :143-146): Dest type F32 or
//   F64 else CL_INVALID_VALUE, then CheckSameSize(S, D).
// A handle that is not an image gives CL_INVALID_MEM_OBJECT (the reference
// casts blindly), an image of another context CL_INVALID_CONTEXT.
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "../../include/OpenCLIPP.h"
#include "../../include/OpenCLIPP_B200.h"
#include "host.h"
#include "internal.h"
#include "statistics.h"
#include "tensor.h"

using namespace ocipb;

namespace ocipb {

const char* error_name(int code) {
  switch (code) {
    case 0: return "SUCCESS";
    case -1: return "CL_DEVICE_NOT_FOUND";
    case -2: return "CL_DEVICE_NOT_AVAILABLE";
    case -3: return "CL_COMPILER_NOT_AVAILABLE";
    case -4: return "CL_MEM_OBJECT_ALLOCATION_FAILURE";
    case -5: return "CL_OUT_OF_RESOURCES";
    case -6: return "CL_OUT_OF_HOST_MEMORY";
    case -7: return "CL_PROFILING_INFO_NOT_AVAILABLE";
    case -8: return "CL_MEM_COPY_OVERLAP";
    case -9: return "CL_IMAGE_FORMAT_MISMATCH";
    case -10: return "CL_IMAGE_FORMAT_NOT_SUPPORTED";
    case -11: return "CL_BUILD_PROGRAM_FAILURE";
    case -12: return "CL_MAP_FAILURE";
    case -30: return "CL_INVALID_VALUE";
    case -31: return "CL_INVALID_DEVICE_TYPE";
    case -32: return "CL_INVALID_PLATFORM";
    case -33: return "CL_INVALID_DEVICE";
    case -34: return "CL_INVALID_CONTEXT";
    case -35: return "CL_INVALID_QUEUE_PROPERTIES";
    case -36: return "CL_INVALID_COMMAND_QUEUE";
    case -37: return "CL_INVALID_HOST_PTR";
    case -38: return "CL_INVALID_MEM_OBJECT";
    case -39: return "CL_INVALID_IMAGE_FORMAT_DESCRIPTOR";
    case -40: return "CL_INVALID_IMAGE_SIZE";
    case -41: return "CL_INVALID_SAMPLER";
    case -42: return "CL_INVALID_BINARY";
    case -43: return "CL_INVALID_BUILD_OPTIONS";
    case -44: return "CL_INVALID_PROGRAM";
    case -45: return "CL_INVALID_PROGRAM_EXECUTABLE";
    case -46: return "CL_INVALID_KERNEL_NAME";
    case -47: return "CL_INVALID_KERNEL_DEFINITION";
    case -48: return "CL_INVALID_KERNEL";
    case -49: return "CL_INVALID_ARG_INDEX";
    case -50: return "CL_INVALID_ARG_VALUE";
    case -51: return "CL_INVALID_ARG_SIZE";
    case -52: return "CL_INVALID_KERNEL_ARGS";
    case -53: return "CL_INVALID_WORK_DIMENSION";
    case -54: return "CL_INVALID_WORK_GROUP_SIZE";
    case -55: return "CL_INVALID_WORK_ITEM_SIZE";
    case -56: return "CL_INVALID_GLOBAL_OFFSET";
    case -57: return "CL_INVALID_EVENT_WAIT_LIST";
    case -58: return "CL_INVALID_EVENT";
    case -59: return "CL_INVALID_OPERATION";
    case -60: return "CL_INVALID_GL_OBJECT";
    case -61: return "CL_INVALID_BUFFER_SIZE";
    default: return "Unknown CL error";
  }
}

namespace {

void same_context(const Context& ctx, const Image& img) {
  if (img.ctx != &ctx) fail(CL_INVALID_CONTEXT, "image belongs to another context");
}

bool same_type(const Image& a, const Image& b) {
  return a.desc.Type == b.desc.Type && a.desc.Channels == b.desc.Channels;
}

void proximity_run(Context& ctx, Measure m, Image& S, Image& T, Image& D, int path) {
  send_if_needed(S);
  send_if_needed(T);
  const DevImage s = dev_view(S), t = dev_view(T), d = dev_view(D);
  cudaError_t e = cudaSuccess;
  bool done = false;
  if (path != OCIP_PATH_PLAIN && tensor_supports(m, s, t, d, path == OCIP_PATH_TENSOR)) {
    e = launch_proximity_tensor(ctx, m, s, t, d);
    done = true;
    ctx.last_path = OCIP_PATH_TENSOR;
  }
  if (!done) {
    void* tt = ctx.scratch(Context::kTemplateEnergy, 64);
    e = launch_proximity_plain(m, s, t, d, tt, ctx.stream);
    ctx.last_path = OCIP_PATH_PLAIN;
  }
  check_cuda(e, "proximity kernel launch");
  mark_written(D);
}

void proximity(Measure m, ocipImage hs, ocipImage ht, ocipImage hd) {
  Context& ctx = current();
  Image& S = image(hs);
  Image& T = image(ht);
  Image& D = image(hd);
  same_context(ctx, S);
  same_context(ctx, T);
  same_context(ctx, D);
  if (T.desc.Width > S.desc.Width || T.desc.Height > S.desc.Height)
    fail(CL_INVALID_VALUE, "Template image must be smaller than the source image.");
  if (!same_type(S, T)) fail(CL_INVALID_VALUE, "Source and Template must have same type.");
  if (S.desc.Width != D.desc.Width || S.desc.Height != D.desc.Height)
    fail(CL_INVALID_IMAGE_SIZE, "Different image sizes used");
  if (S.desc.Channels != D.desc.Channels)
    fail(CL_INVALID_VALUE, "Different number of channels used");
  if (!type_is_float((int)D.desc.Type))
    fail(CL_INVALID_VALUE, "non-float image used when not allowed");
  proximity_run(ctx, m, S, T, D, ctx.path);
}

// The FFT-named entry points (C++/programs/ImageProximityFFT.cpp:112-210)
// check in their own order with their own codes, then compute the same
// measure; here on the tensor path where it applies (no FFT).
void proximity_fft(Measure m, ocipProgram hp, ocipImage hs, ocipImage ht, ocipImage hd) {
  Context& ctx = current();
  Program* prog = reinterpret_cast<Program*>(hp);
  if (prog == nullptr || prog->magic != Program::kMagic || prog->kind != Program::kProximityFFT)
    fail(CL_INVALID_PROGRAM, "invalid program handle");
  Image& S = image(hs);
  Image& T = image(ht);
  Image& D = image(hd);
  same_context(ctx, S);
  same_context(ctx, T);
  same_context(ctx, D);
  if (!type_is_float((int)D.desc.Type))
    fail(CL_INVALID_VALUE, "non-float image used when not allowed");
  if (S.desc.Channels != T.desc.Channels || S.desc.Channels != D.desc.Channels)
    fail(CL_INVALID_VALUE, "Different number of channels used");
  if (S.desc.Width != D.desc.Width || S.desc.Height != D.desc.Height)
    fail(CL_INVALID_IMAGE_SIZE, "Different image sizes used");
  if (T.desc.Width > S.desc.Width || T.desc.Height > S.desc.Height)
    fail(CL_IMAGE_FORMAT_NOT_SUPPORTED, "The template image must be smaller than source image.");
  if (!same_type(S, T))
    fail(CL_IMAGE_FORMAT_MISMATCH, "The source image and the template image must be same type.");
  proximity_run(ctx, m, S, T, D, OCIP_PATH_TENSOR);
}

Program& program(ocipProgram h, int kind) {
  Program* p = reinterpret_cast<Program*>(h);
  if (p == nullptr || p->magic != Program::kMagic || p->kind != kind)
    fail(CL_INVALID_PROGRAM, "invalid program handle");
  return *p;
}

void integral_prepare(Program& prog, const Image& src) {
  const size_t need = integral_scratch_bytes((int)src.desc.Width, (int)src.desc.Height,
                                             (int)src.desc.Channels);
  if (prog.scratch_bytes >= need) return;
  if (prog.scratch) {
    check_cuda(cudaStreamSynchronize(prog.ctx->stream), "integral scratch sync");
    cudaFree(prog.scratch);
    prog.scratch = nullptr;
    prog.scratch_bytes = 0;
  }
  check_cuda(cudaMalloc(&prog.scratch, need), "integral scratch allocation");
  prog.scratch_bytes = need;
}

void integral(bool sqr, ocipProgram hp, ocipImage hs, ocipImage hd) {
  Context& ctx = current();
  Program& prog = program(hp, Program::kIntegral);
  Image& S = image(hs);
  Image& D = image(hd);
  same_context(ctx, S);
  same_context(ctx, D);
  if (prog.ctx != &ctx) fail(CL_INVALID_CONTEXT, "program belongs to another context");
  if (D.desc.Type != SImage::F32 && D.desc.Type != SImage::F64)
    fail(CL_INVALID_VALUE, "Destination image of Integral must be F32 or F64");
  integral_prepare(prog, S);
  if (S.desc.Width != D.desc.Width || S.desc.Height != D.desc.Height)
    fail(CL_INVALID_IMAGE_SIZE, "Different image sizes used");
  if (S.desc.Channels != D.desc.Channels)
    fail(CL_INVALID_VALUE, "Different number of channels used");
  send_if_needed(S);
  check_cuda(launch_integral(sqr, dev_view(S), dev_view(D), prog.scratch, prog.scratch_bytes,
                             ctx.stream),
             "integral kernel launch");
  mark_written(D);
}

// Batched matching (extension, no reference counterpart): the checks of the
// one-pair calls for every pair, plus what the tensor path needs.
void batch_prepare(ocipProgram* out, int measure, const ocipImage* himgs, int nimg,
                   const ocipImage* htpls, int ntpl, const ocipImage* hdsts) {
  Context& ctx = current();
  if (out == nullptr) fail(CL_INVALID_VALUE, "Program is NULL");
  if (measure < 0 || measure > kCrossCorrNorm || measure == kAbsDistance)
    fail(CL_INVALID_VALUE, "measure not available in batches (AbsDistance has no product form)");
  if (nimg <= 0 || ntpl <= 0 || himgs == nullptr || htpls == nullptr || hdsts == nullptr)
    fail(CL_INVALID_VALUE, "empty batch");
  std::vector<Image*> imgs, tpls, dsts;
  for (int i = 0; i < nimg; ++i) imgs.push_back(&image(himgs[i]));
  for (int j = 0; j < ntpl; ++j) tpls.push_back(&image(htpls[j]));
  for (int k = 0; k < nimg * ntpl; ++k) dsts.push_back(&image(hdsts[k]));
  for (Image* x : imgs) same_context(ctx, *x);
  for (Image* x : tpls) same_context(ctx, *x);
  for (Image* x : dsts) same_context(ctx, *x);
  const Image& first = *imgs[0];
  for (Image* x : imgs)
    if (!same_type(first, *x)) fail(CL_INVALID_VALUE, "batch images must share type and channels");
  for (int i = 0; i < nimg; ++i) {
    const Image& S = *imgs[i];
    for (int j = 0; j < ntpl; ++j) {
      const Image& T = *tpls[j];
      const Image& D = *dsts[i * ntpl + j];
      if (T.desc.Width > S.desc.Width || T.desc.Height > S.desc.Height)
        fail(CL_INVALID_VALUE, "Template image must be smaller than the source image.");
      if (!same_type(S, T)) fail(CL_INVALID_VALUE, "Source and Template must have same type.");
      if (S.desc.Width != D.desc.Width || S.desc.Height != D.desc.Height)
        fail(CL_INVALID_IMAGE_SIZE, "Different image sizes used");
      if (S.desc.Channels != D.desc.Channels)
        fail(CL_INVALID_VALUE, "Different number of channels used");
      if (!type_is_float((int)D.desc.Type))
        fail(CL_INVALID_VALUE, "non-float image used when not allowed");
      // The persistent batch kernel takes one template per work item: 64 x 64
      // at most (larger templates are tiled over launches by the one-pair calls).
      if (!tensor_supports((Measure)measure, dev_view(S), dev_view(T), dev_view(D), true) ||
          T.desc.Width > 64 || T.desc.Height > 64)
        fail(CL_INVALID_VALUE,
             "batches run on the tensor path: U8, U16 or F32 sources, templates of 64 x 64 "
             "or less (F32 and U16: at least 64 pixels)");
    }
  }
  for (Image* x : imgs) send_if_needed(*x);
  for (Image* x : tpls) send_if_needed(*x);
  std::vector<DevImage> vi, vt, vd;
  for (Image* x : imgs) vi.push_back(dev_view(*x));
  for (Image* x : tpls) vt.push_back(dev_view(*x));
  for (Image* x : dsts) vd.push_back(dev_view(*x));
  cudaError_t e = cudaSuccess;
  TensorBatch* b = tensor_batch_create(ctx, (Measure)measure, vi, vt, vd, &e);
  check_cuda(e, "batch preparation");
  Program* p = new Program();
  p->kind = Program::kProximityBatch;
  p->ctx = &ctx;
  p->batch = b;
  for (Image* x : dsts) x->in_device = true;
  mark_untracked_writes(ctx);  // the band-height tuning runs write destinations
  *out = reinterpret_cast<ocipProgram>(p);
}

void backward(ocipImage hs, ocipImage ht, ocipImage hg1, ocipImage hg2, ocipImage hn2,
              ocipImage hds, ocipImage hdt) {
  Context& ctx = current();
  Image& S = image(hs);
  Image& T = image(ht);
  same_context(ctx, S);
  same_context(ctx, T);
  auto f32_1ch = [](const Image& x) {
    return x.desc.Type == SImage::F32 && x.desc.Channels == 1;
  };
  auto same_size = [](const Image& a, const Image& b) {
    return a.desc.Width == b.desc.Width && a.desc.Height == b.desc.Height;
  };
  if (!f32_1ch(S) || !f32_1ch(T))
    fail(CL_INVALID_VALUE, "backward: Source and Template must be F32 with one channel");
  if (T.desc.Width > S.desc.Width || T.desc.Height > S.desc.Height)
    fail(CL_INVALID_VALUE, "Template image must be smaller than the source image.");
  if (T.desc.Width > 64 || T.desc.Height > 64)
    fail(CL_INVALID_VALUE, "backward: templates up to 64 x 64");
  if (hg1 == nullptr && hg2 == nullptr)
    fail(CL_INVALID_VALUE, "backward: no upstream gradient");
  Image* G1 = hg1 ? &image(hg1) : nullptr;
  Image* G2 = hg2 ? &image(hg2) : nullptr;
  Image* N2 = hn2 ? &image(hn2) : nullptr;
  Image* dS = hds ? &image(hds) : nullptr;
  Image* dT = hdt ? &image(hdt) : nullptr;
  if (G2 && !N2) fail(CL_INVALID_VALUE, "backward: CrossCorrNorm map needed with its gradient");
  for (Image* x : {G1, G2, N2}) {
    if (!x) continue;
    same_context(ctx, *x);
    if (!f32_1ch(*x)) fail(CL_INVALID_VALUE, "backward: gradient maps must be F32, one channel");
    if (!same_size(*x, S)) fail(CL_INVALID_IMAGE_SIZE, "Different image sizes used");
  }
  for (Image* x : {dS, dT}) {
    if (!x) continue;
    same_context(ctx, *x);
    if (!type_is_float((int)x->desc.Type) || x->desc.Channels != 1)
      fail(CL_INVALID_VALUE, "backward: gradients are written as F32 or F64, one channel");
  }
  if (dS && !same_size(*dS, S)) fail(CL_INVALID_IMAGE_SIZE, "Different image sizes used");
  if (dT && !same_size(*dT, T)) fail(CL_INVALID_IMAGE_SIZE, "Different image sizes used");
  for (Image* x : {&S, &T, G1, G2, N2})
    if (x) send_if_needed(*x);
  DevImage vg1, vg2, vn2, vds, vdt;
  if (G1) vg1 = dev_view(*G1);
  if (G2) vg2 = dev_view(*G2);
  if (N2) vn2 = dev_view(*N2);
  if (dS) vds = dev_view(*dS);
  if (dT) vdt = dev_view(*dT);
  check_cuda(proximity_backward(ctx, dev_view(S), dev_view(T), G1 ? &vg1 : nullptr,
                                G2 ? &vg2 : nullptr, N2 ? &vn2 : nullptr, dS ? &vds : nullptr,
                                dT ? &vdt : nullptr),
             "backward launch");
  if (dS) mark_written(*dS);
  if (dT) mark_written(*dT);
}

// Statistics::Min/Max/MinAbs/MaxAbs with coordinates
// (C++/programs/Statistics.cpp:244-298): one channel only (Check1Channel,
// C++/programs/Program.cpp:501-505), synchronous.
void index_op(int op, ocipProgram hp, ocipImage hs, double* result, int* x, int* y) {
  Context& ctx = current();
  Program& prog = program(hp, Program::kStatistics);
  if (prog.ctx != &ctx) fail(CL_INVALID_CONTEXT, "program belongs to another context");
  Image& S = image(hs);
  same_context(ctx, S);
  if (S.desc.Channels > 1) fail(CL_INVALID_VALUE, "only 1 channel images are allowed");
  if (result == nullptr || x == nullptr || y == nullptr) fail(CL_INVALID_VALUE, "NULL result");
  const size_t need = index_reduce_scratch_bytes((int)S.desc.Width, (int)S.desc.Height);
  if (prog.scratch_bytes < need) {
    if (prog.scratch) {
      check_cuda(cudaStreamSynchronize(ctx.stream), "statistics scratch sync");
      cudaFree(prog.scratch);
      prog.scratch = nullptr;
      prog.scratch_bytes = 0;
    }
    check_cuda(cudaMalloc(&prog.scratch, need), "statistics scratch allocation");
    prog.scratch_bytes = need;
  }
  send_if_needed(S);
  check_cuda(index_reduce(ctx, op, dev_view(S), prog.scratch, result, x, y), "index reduction");
  ctx.check_device_errors();
}

// Best match in one call (extension): the measure, then the reference's
// index reduction of its map. On the tensor path the reduction is fused into
// the scoring epilogue and no map needs to be written; a NaN score (the
// reference's answer then depends on where it lies) or a shape the fused
// kernel does not take uses the written map and the reference-order
// reduction.
void proximity_index(int measure, int op, ocipImage hs, ocipImage ht, ocipImage hd,
                     double* value, int* x, int* y) {
  Context& ctx = current();
  if (measure < kSqrDistance || measure > kCrossCorrNorm) fail(CL_INVALID_VALUE, "unknown measure");
  if (op < kIdxMin || op > kIdxMaxAbs) fail(CL_INVALID_VALUE, "unknown index reduction");
  if (value == nullptr || x == nullptr || y == nullptr) fail(CL_INVALID_VALUE, "NULL result");
  Image& S = image(hs);
  Image& T = image(ht);
  Image* D = hd ? &image(hd) : nullptr;
  same_context(ctx, S);
  same_context(ctx, T);
  if (D) same_context(ctx, *D);
  if (T.desc.Width > S.desc.Width || T.desc.Height > S.desc.Height)
    fail(CL_INVALID_VALUE, "Template image must be smaller than the source image.");
  if (!same_type(S, T)) fail(CL_INVALID_VALUE, "Source and Template must have same type.");
  if (S.desc.Channels > 1) fail(CL_INVALID_VALUE, "only 1 channel images are allowed");
  if (D && (S.desc.Width != D->desc.Width || S.desc.Height != D->desc.Height))
    fail(CL_INVALID_IMAGE_SIZE, "Different image sizes used");
  if (D && (D->desc.Type != SImage::F32 || D->desc.Channels != 1))
    fail(CL_INVALID_VALUE, "Dest of ocipProximityIndx must be F32 with one channel");
  send_if_needed(S);
  send_if_needed(T);
  const Measure m = static_cast<Measure>(measure);
  const DevImage s = dev_view(S), t = dev_view(T);
  DevImage d;
  if (D) {
    d = dev_view(*D);
  } else {
    d.ptr = nullptr;
    d.pitch = 0;
    d.width = s.width;
    d.height = s.height;
    d.nch = 1;
    d.type = F32;
  }
  const bool fused = ctx.path != OCIP_PATH_PLAIN && t.width <= 64 && t.height <= 64 &&
                     tensor_supports(m, s, t, d, ctx.path == OCIP_PATH_TENSOR);
  bool wrote_map = false;
  if (fused) {
    void* rec = ctx.scratch(Context::kIndexRecords, tensor_index_records_bytes(ctx, s, t));
    int nrec = 0, bx = 0, by = 0;
    float best = 0.f;
    bool nan = false;
    check_cuda(launch_proximity_tensor_indexed(ctx, m, s, t, d, op, rec, &nrec, &best, &bx, &by,
                                               &nan),
               "fused best-match launch");
    ctx.last_path = OCIP_PATH_TENSOR;
    if (D) mark_written(*D);
    ctx.check_device_errors();
    if (!nan) {
      *value = best;
      *x = bx;
      *y = by;
      return;
    }
    wrote_map = D != nullptr;
  }
  // The map path: the measure's map (Dest, or scratch), then the reduction.
  DevImage map = d;
  if (!D) {
    map.pitch = ((size_t)s.width * 4 + 127) / 128 * 128;
    map.ptr = ctx.scratch(Context::kIndexMap, map.pitch * s.height);
  }
  if (!wrote_map) {
    cudaError_t e;
    if (ctx.path != OCIP_PATH_PLAIN && tensor_supports(m, s, t, map, ctx.path == OCIP_PATH_TENSOR)) {
      e = launch_proximity_tensor(ctx, m, s, t, map);
      ctx.last_path = OCIP_PATH_TENSOR;
    } else {
      void* tt = ctx.scratch(Context::kTemplateEnergy, 64);
      e = launch_proximity_plain(m, s, t, map, tt, ctx.stream);
      ctx.last_path = OCIP_PATH_PLAIN;
    }
    check_cuda(e, "proximity kernel launch");
    if (D) mark_written(*D);
  }
  void* scratch = ctx.scratch(Context::kIndexScratch, index_reduce_scratch_bytes(s.width, s.height));
  check_cuda(index_reduce(ctx, op, map, scratch, value, x, y), "index reduction");
  ctx.check_device_errors();
}

}  // namespace
}  // namespace ocipb

extern "C" {

ocipError ocipProximityIndx(int Measure, int IndexOp, ocipImage Source, ocipImage Template,
                            ocipImage Dest, double* Value, int* X, int* Y) {
  OCIP_GUARD(proximity_index(Measure, IndexOp, Source, Template, Dest, Value, X, Y))
}

ocipError ocipPrepareStatistics(ocipProgram* ProgramPtr, ocipImage Img) {
  OCIP_GUARD(
    Context& ctx = current();
    if (ProgramPtr == nullptr) fail(CL_INVALID_VALUE, "ProgramPtr is NULL");
    if (Img != nullptr) image(Img);
    Program* p = new Program();
    p->kind = Program::kStatistics;
    p->ctx = &ctx;
    *ProgramPtr = reinterpret_cast<ocipProgram>(p);
  )
}
ocipError ocipMinIndx(ocipProgram P, ocipImage S, double* R, int* X, int* Y) {
  OCIP_GUARD(index_op(kIdxMin, P, S, R, X, Y))
}
ocipError ocipMaxIndx(ocipProgram P, ocipImage S, double* R, int* X, int* Y) {
  OCIP_GUARD(index_op(kIdxMax, P, S, R, X, Y))
}
ocipError ocipMinAbsIndx(ocipProgram P, ocipImage S, double* R, int* X, int* Y) {
  OCIP_GUARD(index_op(kIdxMinAbs, P, S, R, X, Y))
}
ocipError ocipMaxAbsIndx(ocipProgram P, ocipImage S, double* R, int* X, int* Y) {
  OCIP_GUARD(index_op(kIdxMaxAbs, P, S, R, X, Y))
}

ocipError ocipProximityBackward(ocipImage Source, ocipImage Template, ocipImage GradSqrDistance,
                                ocipImage GradCrossCorrNorm, ocipImage CrossCorrNorm,
                                ocipImage GradSource, ocipImage GradTemplate) {
  OCIP_GUARD(backward(Source, Template, GradSqrDistance, GradCrossCorrNorm, CrossCorrNorm,
                      GradSource, GradTemplate))
}

ocipError ocipPrepareProximityBatch(ocipProgram* Program, int Measure, const ocipImage* Images,
                                    int NbImages, const ocipImage* Templates, int NbTemplates,
                                    const ocipImage* Dests) {
  OCIP_GUARD(batch_prepare(Program, Measure, Images, NbImages, Templates, NbTemplates, Dests))
}

ocipError ocipTestBoundedWait(int LimitCycles) {
  OCIP_GUARD(
    Context& ctx = current();
    if (LimitCycles <= 0) fail(CL_INVALID_VALUE, "LimitCycles must be positive");
    check_cuda(launch_bounded_wait_probe(ctx, LimitCycles), "bounded-wait probe");
    check_cuda(cudaStreamSynchronize(ctx.stream), "bounded-wait probe");
    ctx.check_device_errors();
  )
}

ocipError ocipRunProximityBatch(ocipProgram P) {
  OCIP_GUARD(
    Context& ctx = current();
    ocipb::Program& prog = program(P, ocipb::Program::kProximityBatch);
    if (prog.ctx != &ctx) fail(CL_INVALID_CONTEXT, "program belongs to another context");
    check_cuda(tensor_batch_run(prog.batch), "batch launch");
    mark_untracked_writes(ctx);
  )
}

ocipError ocipGetProximityBatchInfo(ocipProgram P, int TemplateWidth, int TemplateHeight,
                                    int* NbItems, int* BandHeight) {
  OCIP_GUARD(
    ocipb::Program& prog = program(P, ocipb::Program::kProximityBatch);
    if (NbItems) *NbItems = tensor_batch_items(prog.batch);
    if (BandHeight) *BandHeight = tensor_batch_band_height(prog.batch, TemplateWidth, TemplateHeight);
  )
}

ocipError ocipPrepareProximity(ocipImage Image) {
  OCIP_GUARD(
    current();
    if (Image != nullptr) image(Image);
  )
}

ocipError ocipSqrDistance_Norm(ocipImage S, ocipImage T, ocipImage D) {
  OCIP_GUARD(proximity(kSqrDistanceNorm, S, T, D))
}
ocipError ocipSqrDistance(ocipImage S, ocipImage T, ocipImage D) {
  OCIP_GUARD(proximity(kSqrDistance, S, T, D))
}
ocipError ocipAbsDistance(ocipImage S, ocipImage T, ocipImage D) {
  OCIP_GUARD(proximity(kAbsDistance, S, T, D))
}
ocipError ocipCrossCorr(ocipImage S, ocipImage T, ocipImage D) {
  OCIP_GUARD(proximity(kCrossCorr, S, T, D))
}
ocipError ocipCrossCorr_Norm(ocipImage S, ocipImage T, ocipImage D) {
  OCIP_GUARD(proximity(kCrossCorrNorm, S, T, D))
}

ocipError ocipPrepareIntegral(ocipProgram* ProgramPtr, ocipImage Img) {
  OCIP_GUARD(
    Context& ctx = current();
    if (ProgramPtr == nullptr) fail(CL_INVALID_VALUE, "ProgramPtr is NULL");
    Program* p = new Program();
    p->kind = Program::kIntegral;
    p->ctx = &ctx;
    *ProgramPtr = reinterpret_cast<ocipProgram>(p);
    if (Img != nullptr) integral_prepare(*p, image(Img));
  )
}

ocipBool ocipIsFFTAvailable(void) { return 1; }

ocipError ocipPrepareImageProximityFFT(ocipProgram* ProgramPtr, ocipImage Img, ocipImage Tmpl) {
  OCIP_GUARD(
    Context& ctx = current();
    if (ProgramPtr == nullptr) fail(CL_INVALID_VALUE, "ProgramPtr is NULL");
    if (Img != nullptr) image(Img);
    if (Tmpl != nullptr) image(Tmpl);
    Program* p = new Program();
    p->kind = Program::kProximityFFT;
    p->ctx = &ctx;
    *ProgramPtr = reinterpret_cast<ocipProgram>(p);
  )
}
ocipError ocipSqrDistanceFFT(ocipProgram P, ocipImage S, ocipImage T, ocipImage D) {
  OCIP_GUARD(proximity_fft(kSqrDistance, P, S, T, D))
}
ocipError ocipSqrDistanceFFT_Norm(ocipProgram P, ocipImage S, ocipImage T, ocipImage D) {
  OCIP_GUARD(proximity_fft(kSqrDistanceNorm, P, S, T, D))
}
ocipError ocipCrossCorrFFT(ocipProgram P, ocipImage S, ocipImage T, ocipImage D) {
  OCIP_GUARD(proximity_fft(kCrossCorr, P, S, T, D))
}
ocipError ocipCrossCorrFFT_Norm(ocipProgram P, ocipImage S, ocipImage T, ocipImage D) {
  OCIP_GUARD(proximity_fft(kCrossCorrNorm, P, S, T, D))
}

ocipError ocipIntegral(ocipProgram P, ocipImage S, ocipImage D) { OCIP_GUARD(integral(false, P, S, D)) }
ocipError ocipSqrIntegral(ocipProgram P, ocipImage S, ocipImage D) { OCIP_GUARD(integral(true, P, S, D)) }

}  // extern "C"
