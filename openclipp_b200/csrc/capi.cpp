// C ABI of the library: the reference's ocip* entry points for template
// matching (include/OpenCLIPP.h) plus the extensions of OpenCLIPP_B200.h.
//
// Mirrors OpenCLIPP/OpenCLIPP.cpp: a process-wide current context
// (:73-75), exceptions turned into negative error codes at the boundary (the
// H() macro, :82; here OCIP_GUARD), context checks before anything else
// (GetList(), :717-728),
// asynchronous processing calls on one in-order queue (here a CUDA stream),
// lazy upload of source images on first use (C++/Buffer.cpp:190-194) and a
// blocking ocipReadImage (:203-211).
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>

#include "../../include/OpenCLIPP.h"
#include "../../include/OpenCLIPP_B200.h"
#include "host.h"
#include "internal.h"
#include "tensor.h"

using namespace ocipb;

namespace ocipb {

thread_local std::string g_last_error;
unsigned long long g_launches = 0;
std::map<Context*, bool> g_contexts;
Context* g_current = nullptr;

[[noreturn]] void fail(int code, const std::string& msg) { throw Error{code, msg}; }

void check_cuda(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return;
  const int code = (e == cudaErrorMemoryAllocation) ? CL_MEM_OBJECT_ALLOCATION_FAILURE
                                                    : CL_OUT_OF_RESOURCES;
  fail(code, std::string(what) + ": " + cudaGetErrorString(e));
}

Context& current() {
  if (g_current == nullptr)
    fail(CL_INVALID_CONTEXT, "No current context - use ocipInitialize() first");
  auto it = g_contexts.find(g_current);
  if (it == g_contexts.end() || !it->second)
    fail(CL_INVALID_CONTEXT, "Invalid current context - ocipInitialize()");
  check_cuda(cudaSetDevice(g_current->device), "cudaSetDevice");
  return *g_current;
}

Image& image(ocipImage h) {
  Image* img = reinterpret_cast<Image*>(h);
  if (img == nullptr || img->magic != Image::kMagic)
    fail(CL_INVALID_MEM_OBJECT, "invalid image handle");
  return *img;
}

// Counts a transfer of the image's host buffer and page-locks a pageable
// buffer once it has been transferred Image::kRegisterAfter times. A buffer
// that cannot be registered (already registered as part of another range,
// or the pinned-memory limit reached) stays pageable; copies are correct
// either way.
void note_host_transfer(Image& img) {
  if (img.host_pinned || img.host_transfers < 0) return;
  if (++img.host_transfers < Image::kRegisterAfter) return;
  // The caller's rows: Step bytes apart, the last one row_bytes() long.
  const size_t bytes = (size_t)img.desc.Step * (img.desc.Height - 1) + img.row_bytes();
  const cudaError_t e = cudaHostRegister(img.host, bytes, cudaHostRegisterDefault);
  if (e == cudaSuccess) {
    img.host_pinned = img.host_registered = true;
  } else {
    cudaGetLastError();  // not sticky: clear it
    if (e == cudaErrorHostMemoryAlreadyRegistered) img.host_pinned = true;
    else img.host_transfers = -1;  // do not try again
  }
}

void send(Image& img) {
  if (img.host == nullptr) return;  // device-only image (Buffer.cpp:158)
  Context& ctx = *img.ctx;
  check_cuda(cudaSetDevice(ctx.device), "cudaSetDevice");
  note_host_transfer(img);
  const size_t row = img.row_bytes();
  check_cuda(cudaMemcpy2DAsync(img.dev, img.pitch, img.host, img.desc.Step, row,
                               img.desc.Height, cudaMemcpyHostToDevice, ctx.stream),
             "send image");
  mark_written(img);
}

void mark_written(Image& img) {
  img.in_device = true;
  if (img.written == nullptr)
    check_cuda(cudaEventCreateWithFlags(&img.written, cudaEventDisableTiming), "event");
  check_cuda(cudaEventRecord(img.written, img.ctx->stream), "event record");
}

void mark_untracked_writes(Context& ctx) {
  if (ctx.untracked == nullptr)
    check_cuda(cudaEventCreateWithFlags(&ctx.untracked, cudaEventDisableTiming), "event");
  check_cuda(cudaEventRecord(ctx.untracked, ctx.stream), "event record");
}

void send_if_needed(Image& img) {
  if (!img.in_device) send(img);
}

DevImage dev_view(const Image& img) {
  DevImage d;
  d.ptr = img.dev;
  d.pitch = img.pitch;
  d.width = (int)img.desc.Width;
  d.height = (int)img.desc.Height;
  d.nch = (int)img.desc.Channels;
  d.type = (int)img.desc.Type;
  return d;
}

void* Context::scratch(int slot, size_t bytes) {
  Scratch& s = scratch_[slot];
  if (s.bytes < bytes) {
    if (s.ptr) {
      check_cuda(cudaStreamSynchronize(stream), "scratch sync");
      cudaFree(s.ptr);
      s.ptr = nullptr;
      s.bytes = 0;
    }
    check_cuda(cudaMalloc(&s.ptr, bytes), "scratch allocation");
    s.bytes = bytes;
    // New scratch starts zeroed: the kernels' error flag lives in one slot.
    check_cuda(cudaMemsetAsync(s.ptr, 0, bytes, stream), "scratch initialisation");
  }
  return s.ptr;
}

void Context::check_device_errors() {
  const Scratch& s = scratch_[kTensorAux];
  if (s.ptr == nullptr) return;
  int flag = 0;
  check_cuda(cudaMemcpy(&flag, s.ptr, sizeof(int), cudaMemcpyDeviceToHost), "error flag");
  if (flag) {
    check_cuda(cudaMemset(s.ptr, 0, sizeof(int)), "error flag");
    fail(CL_OUT_OF_RESOURCES,
         "a tensor-core kernel gave up a bounded wait; results since the last ocipFinish or "
         "ocipReadImage are not valid");
  }
}

Context::~Context() {
  for (auto& s : scratch_)
    if (s.ptr) cudaFree(s.ptr);
  if (untracked) cudaEventDestroy(untracked);
  if (copy_stream) cudaStreamDestroy(copy_stream);
  if (stream) cudaStreamDestroy(stream);
}

}  // namespace ocipb



extern "C" {

// ---- Context ------------------------------------------------------------

ocipError ocipInitialize(ocipContext* ContextPtr, const char* PreferredPlatform,
                         cl_device_type deviceType) {
  OCIP_GUARD(
    if (ContextPtr == nullptr) fail(CL_INVALID_VALUE, "ContextPtr is NULL");
    const cl_device_type wanted = deviceType;
    const bool gpu_ok = (wanted & CL_DEVICE_TYPE_GPU) || (wanted & CL_DEVICE_TYPE_DEFAULT) ||
                        wanted == (cl_device_type)CL_DEVICE_TYPE_ALL;
    if (!gpu_ok) fail(CL_DEVICE_NOT_FOUND, "only GPU devices are available");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
      fail(CL_DEVICE_NOT_FOUND, "no CUDA device");
    int dev = -1;
    if (PreferredPlatform != nullptr) {
      char* end = nullptr;
      const long v = strtol(PreferredPlatform, &end, 10);
      if (end != PreferredPlatform && *end == '\0' && v >= 0 && v < ndev) dev = (int)v;
    }
    if (dev < 0) check_cuda(cudaGetDevice(&dev), "cudaGetDevice");
    check_cuda(cudaSetDevice(dev), "cudaSetDevice");
    Context* ctx = new Context();
    ctx->device = dev;
    cudaDeviceProp prop;
    check_cuda(cudaGetDeviceProperties(&prop, dev), "cudaGetDeviceProperties");
    ctx->name = prop.name;
    ctx->sm_count = prop.multiProcessorCount;
    ctx->cc_major = prop.major;
    ctx->cc_minor = prop.minor;
    cudaError_t e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
      delete ctx;
      check_cuda(e, "cudaStreamCreate");
    }
    g_contexts[ctx] = true;
    g_current = ctx;
    *ContextPtr = reinterpret_cast<ocipContext>(ctx);
  )
}

ocipError ocipUninitialize(ocipContext Context) {
  ocipb::Context* ctx = reinterpret_cast<ocipb::Context*>(Context);
  if (ctx == nullptr) return CL_INVALID_CONTEXT;
  auto it = g_contexts.find(ctx);
  if (it == g_contexts.end() || !it->second) return CL_INVALID_CONTEXT;
  if (ctx == g_current) g_current = nullptr;
  OCIP_GUARD(
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    g_contexts.erase(it);
    delete ctx;
  )
}

ocipError ocipChangeContext(ocipContext Context) {
  ocipb::Context* ctx = reinterpret_cast<ocipb::Context*>(Context);
  if (ctx == nullptr) return CL_INVALID_CONTEXT;
  auto it = g_contexts.find(ctx);
  if (it == g_contexts.end() || !it->second) return CL_INVALID_CONTEXT;
  g_current = ctx;
  return CL_SUCCESS;
}

void ocipSetCLFilesPath(const char*) {}

const char* ocipGetErrorName(ocipError Error) { return ocipb::error_name(Error); }

ocipError ocipGetDeviceName(char* Name, uint BufferLength) {
  if (g_current == nullptr) return CL_INVALID_CONTEXT;
  OCIP_GUARD(
    Context& ctx = current();
    if (Name == nullptr || BufferLength == 0) fail(CL_INVALID_VALUE, "no buffer");
    if (ctx.name.length() > BufferLength - 1) return CL_OUT_OF_RESOURCES;
    memcpy(Name, ctx.name.c_str(), ctx.name.length() + 1);
  )
}

ocipError ocipFinish(void) {
  if (g_current == nullptr) return CL_INVALID_CONTEXT;
  OCIP_GUARD(
    Context& ctx = current();
    check_cuda(cudaStreamSynchronize(ctx.stream), "ocipFinish");
    ctx.check_device_errors();
  )
}

// ---- Images -------------------------------------------------------------

ocipError ocipCreateImage(ocipImage* ImagePtr, SImage desc, void* ImageData,
                          cl_mem_flags) {
  if (g_current == nullptr) return CL_INVALID_CONTEXT;
  OCIP_GUARD(
    Context& ctx = current();
    if (ImagePtr == nullptr) fail(CL_INVALID_VALUE, "ImagePtr is NULL");
    if (desc.Channels < 1 || desc.Channels > 4)
      fail(CL_IMAGE_FORMAT_NOT_SUPPORTED, "Invalid number of channels");
    if ((int)desc.Type < 0 || (int)desc.Type >= (int)SImage::NbDataTypes)
      fail(CL_IMAGE_FORMAT_NOT_SUPPORTED, "Invalid data type");
    if (desc.Width == 0 || desc.Height == 0 || desc.Step == 0)
      fail(CL_INVALID_BUFFER_SIZE, "empty image");
    const size_t row = (size_t)desc.Width * desc.Channels * type_bytes((int)desc.Type);
    if (desc.Step < row) fail(CL_INVALID_VALUE, "Step is smaller than one row of pixels");
    Image* img = new Image();
    img->ctx = &ctx;
    img->desc = desc;
    img->host = ImageData;
    if (ImageData != nullptr) {
      cudaPointerAttributes attr;
      if (cudaPointerGetAttributes(&attr, ImageData) == cudaSuccess)
        img->host_pinned = attr.type == cudaMemoryTypeHost;
      else
        cudaGetLastError();
    }
    img->pitch = (row + 127) / 128 * 128;
    cudaError_t e = cudaMalloc(&img->dev, img->pitch * desc.Height);
    if (e != cudaSuccess) {
      delete img;
      check_cuda(e, "image allocation");
    }
    // Zero the whole buffer once: the bytes between a row's end and the next
    // row (pitch padding) are never written afterwards, so kernels that read
    // whole 16-byte chunks past the last pixel see zeros there.
    e = cudaMemsetAsync(img->dev, 0, img->pitch * desc.Height, ctx.stream);
    if (e != cudaSuccess) {
      cudaFree(img->dev);
      delete img;
      check_cuda(e, "image initialisation");
    }
    *ImagePtr = reinterpret_cast<ocipImage>(img);
  )
}

ocipError ocipSendImage(ocipImage h) {
  OCIP_GUARD(
    Image& img = image(h);
    send(img);
  )
}

ocipError ocipReadImage(ocipImage h) {
  OCIP_GUARD(
    Image& img = image(h);
    if (img.host == nullptr) return CL_SUCCESS;  // Buffer.cpp:125-126
    Context& ctx = *img.ctx;
    check_cuda(cudaSetDevice(ctx.device), "cudaSetDevice");
    // The copy waits for the image's last writer only, not for everything
    // queued since: kernels enqueued after that writer keep running while
    // this map travels to the host. The call still returns only once the
    // data is in the host buffer (Read is blocking, OpenCLIPP.cpp:203-211),
    // so no copy is ever left in flight across calls.
    note_host_transfer(img);
    if (img.exposed) mark_written(img);  // writes through the raw address: wait for all
    if (img.written) check_cuda(cudaStreamWaitEvent(ctx.copy_stream, img.written, 0), "read wait");
    if (ctx.untracked)
      check_cuda(cudaStreamWaitEvent(ctx.copy_stream, ctx.untracked, 0), "read wait");
    check_cuda(cudaMemcpy2DAsync(img.host, img.desc.Step, img.dev, img.pitch,
                                 img.row_bytes(), img.desc.Height,
                                 cudaMemcpyDeviceToHost, ctx.copy_stream),
               "read image");
    check_cuda(cudaStreamSynchronize(ctx.copy_stream), "read image");
    ctx.check_device_errors();
  )
}

ocipError ocipReleaseImage(ocipImage h) {
  Image* img = reinterpret_cast<Image*>(h);
  if (img != nullptr && img->magic == Image::kMagic) {
    if (g_contexts.count(img->ctx)) {
      cudaSetDevice(img->ctx->device);
      cudaStreamSynchronize(img->ctx->stream);
    }
    if (img->written) cudaEventDestroy(img->written);
    if (img->host_registered) cudaHostUnregister(img->host);
    cudaFree(img->dev);
    img->magic = 0;
    delete img;
  }
  return CL_SUCCESS;  // OpenCLIPP.cpp:213-218 always succeeds
}

ocipError ocipReleaseProgram(ocipProgram h) {
  Program* p = reinterpret_cast<Program*>(h);
  if (p != nullptr && p->magic == Program::kMagic) {
    if (p->batch) tensor_batch_destroy(p->batch);
    if (p->scratch) {
      if (g_contexts.count(p->ctx)) {
        cudaSetDevice(p->ctx->device);
        cudaStreamSynchronize(p->ctx->stream);
      }
      cudaFree(p->scratch);
    }
    p->magic = 0;
    delete p;
  }
  return CL_SUCCESS;
}

// ---- Extensions -----------------------------------------------------------

ocipError ocipSetProximityPath(int Path) {
  if (g_current == nullptr) return CL_INVALID_CONTEXT;
  OCIP_GUARD(
    Context& ctx = current();
    if (Path < OCIP_PATH_AUTO || Path > OCIP_PATH_TENSOR) fail(CL_INVALID_VALUE, "unknown path");
    ctx.path = Path;
  )
}

ocipError ocipGetProximityPath(int* Path) {
  if (g_current == nullptr) return CL_INVALID_CONTEXT;
  OCIP_GUARD(
    Context& ctx = current();
    if (Path == nullptr) fail(CL_INVALID_VALUE, "Path is NULL");
    *Path = ctx.path;
  )
}

ocipError ocipGetLastProximityPath(int* Path) {
  if (g_current == nullptr) return CL_INVALID_CONTEXT;
  OCIP_GUARD(
    Context& ctx = current();
    if (Path == nullptr) fail(CL_INVALID_VALUE, "Path is NULL");
    *Path = ctx.last_path;
  )
}

ocipError ocipSetProximityBandHeight(int Rows) {
  if (g_current == nullptr) return CL_INVALID_CONTEXT;
  OCIP_GUARD(
    Context& ctx = current();
    if (Rows < 0) fail(CL_INVALID_VALUE, "Rows is negative");
    ctx.band_rows = Rows;
  )
}

const char* ocipGetLastErrorMessage(void) { return g_last_error.c_str(); }

ocipError ocipGetStream(void** Stream) {
  if (g_current == nullptr) return CL_INVALID_CONTEXT;
  OCIP_GUARD(
    Context& ctx = current();
    if (Stream == nullptr) fail(CL_INVALID_VALUE, "Stream is NULL");
    *Stream = (void*)ctx.stream;
  )
}

ocipError ocipGetLaunchCount(uint64_t* Count) {
  if (Count == nullptr) return CL_INVALID_VALUE;
  *Count = g_launches;
  return CL_SUCCESS;
}

ocipError ocipGetImageDevicePtr(ocipImage h, void** DevicePtr, size_t* Pitch) {
  OCIP_GUARD(
    Image& img = image(h);
    if (DevicePtr) *DevicePtr = img.dev;
    if (Pitch) *Pitch = img.pitch;
    img.exposed = true;
  )
}

ocipError ocipGetProximityBand(unsigned int Height, unsigned int TemplateHeight, int Part,
                               int Parts, unsigned int Rows[4]) {
  if (Rows == nullptr || Parts < 1 || Part < 0 || Part >= Parts || TemplateHeight == 0 ||
      TemplateHeight > Height)
    return CL_INVALID_VALUE;
  // Owned rows: the first Height % Parts parts take one row more.
  const uint64_t base = Height / (unsigned)Parts, extra = Height % (unsigned)Parts;
  const uint64_t p = (uint64_t)Part;
  const uint64_t y0 = p * base + (p < extra ? p : extra);
  const uint64_t y1 = y0 + base + (p < extra ? 1 : 0);
  Rows[0] = (unsigned)y0;
  Rows[1] = (unsigned)y1;
  if (y1 == y0) {
    Rows[2] = Rows[3] = (unsigned)y0;
    return CL_SUCCESS;
  }
  // Destination row y reads source rows y - ay .. y - ay + th - 1.
  const int64_t ay = TemplateHeight / 2;
  const int64_t s0 = (int64_t)y0 - ay;
  const int64_t s1 = (int64_t)y1 - ay + TemplateHeight - 1;
  int64_t a = s0 < 0 ? 0 : s0, b = s1 > (int64_t)Height ? (int64_t)Height : s1;
  // Near an edge the clipped band can be shorter than the template; widen it
  // with real rows (which change none of the owned outputs) to pass the
  // template-size check of the measure calls.
  if (b - a < (int64_t)TemplateHeight) {
    if (a == 0) b = TemplateHeight;
    else a = b - (int64_t)TemplateHeight;
  }
  Rows[2] = (unsigned)a;
  Rows[3] = (unsigned)b;
  return CL_SUCCESS;
}

}  // extern "C"
